// fock_cls_5.cu -- instantiations of the Fock kernel for one group of
// angular class pairs (split for parallel compilation).
#include "fock_kernel.cuh"

extern "C" int gtf_fock_group_5(int la, int lb, int lc, int ld, const FockGrid &g, cudaStream_t st)
{
    FOCK_GROUP_CASE(2,2,2,2)
    return GTF_NOT_IN_GROUP;
}
