/* mkl_trans.h -- nothing from it is called on the single-process path. */
#ifndef GTF_REF_MKL_TRANS_H
#define GTF_REF_MKL_TRANS_H
#endif
