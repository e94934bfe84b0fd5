// fock_cls_2.cu -- instantiations of the Fock kernel for one group of
// angular class pairs (split for parallel compilation).
#include "fock_kernel.cuh"

extern "C" int gtf_fock_group_2(int la, int lb, int lc, int ld, const FockGrid &g, cudaStream_t st)
{
    FOCK_GROUP_CASE(2,1,2,1)
    FOCK_GROUP_CASE(2,2,0,0)
    FOCK_GROUP_CASE(2,2,1,0)
    return GTF_NOT_IN_GROUP;
}
