// fock_groups.cu -- table of the per-group Fock launchers
#include "fock_kernel.cuh"

extern "C" int gtf_fock_group_0(int la, int lb, int lc, int ld, const FockGrid &g, cudaStream_t st);
extern "C" int gtf_fock_group_1(int la, int lb, int lc, int ld, const FockGrid &g, cudaStream_t st);
extern "C" int gtf_fock_group_2(int la, int lb, int lc, int ld, const FockGrid &g, cudaStream_t st);
extern "C" int gtf_fock_group_3(int la, int lb, int lc, int ld, const FockGrid &g, cudaStream_t st);
extern "C" int gtf_fock_group_4(int la, int lb, int lc, int ld, const FockGrid &g, cudaStream_t st);
extern "C" int gtf_fock_group_5(int la, int lb, int lc, int ld, const FockGrid &g, cudaStream_t st);

typedef int (*fock_group_launch_t)(int la, int lb, int lc, int ld, const FockGrid &g, cudaStream_t st);
fock_group_launch_t gtf_fock_groups[] = {gtf_fock_group_0, gtf_fock_group_1, gtf_fock_group_2, gtf_fock_group_3, gtf_fock_group_4, gtf_fock_group_5};
extern const int gtf_fock_ngroups = 6;
