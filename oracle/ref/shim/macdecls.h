/* macdecls.h -- Global Arrays type codes for the single-process GA shim. */
#ifndef GTF_REF_MACDECLS_H
#define GTF_REF_MACDECLS_H
#define C_INT 1099
#define C_DBL 1013
#define MT_C_INT C_INT
#define MT_C_DBL C_DBL
#define MT_DBL C_DBL
#define MT_INT C_INT
int MA_init(int type, long stack, long heap);
#endif
