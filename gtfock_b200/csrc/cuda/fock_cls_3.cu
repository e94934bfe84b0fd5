// fock_cls_3.cu -- instantiations of the Fock kernel for one group of
// angular class pairs (split for parallel compilation).
#include "fock_kernel.cuh"

extern "C" int gtf_fock_group_3(int la, int lb, int lc, int ld, const FockGrid &g, cudaStream_t st)
{
    FOCK_GROUP_CASE(2,2,1,1)
    FOCK_GROUP_CASE(2,2,2,0)
    return GTF_NOT_IN_GROUP;
}
