/* ga.h -- single-process Global Arrays shim (test infrastructure only).
 * Each global array is one local row-major 2-D array; one-sided operations
 * become copies.  Covers the calls made by pfock/*.c and pscf/*.c. */
#ifndef GTF_REF_GA_H
#define GTF_REF_GA_H
#include "macdecls.h"
typedef int ga_nbhdl_t;
void GA_Initialize(void);
void GA_Terminate(void);
int NGA_Create_irreg(int type, int ndim, int dims[], char *name, int block[], int map[]);
int GA_Duplicate(int g_a, char *name);
void GA_Destroy(int g_a);
void GA_Fill(int g_a, void *val);
void GA_Sync(void);
void NGA_Put(int g_a, int lo[], int hi[], void *buf, int ld[]);
void NGA_Get(int g_a, int lo[], int hi[], void *buf, int ld[]);
void NGA_Acc(int g_a, int lo[], int hi[], void *buf, int ld[], void *alpha);
void NGA_NbPut(int g_a, int lo[], int hi[], void *buf, int ld[], ga_nbhdl_t *h);
void NGA_NbGet(int g_a, int lo[], int hi[], void *buf, int ld[], ga_nbhdl_t *h);
void NGA_NbAcc(int g_a, int lo[], int hi[], void *buf, int ld[], void *alpha, ga_nbhdl_t *h);
int NGA_NbWait(ga_nbhdl_t *h);
void NGA_Access(int g_a, int lo[], int hi[], void *ptr, int ld[]);
void NGA_Release(int g_a, int lo[], int hi[]);
void NGA_Release_update(int g_a, int lo[], int hi[]);
long NGA_Read_inc(int g_a, int subscript[], long inc);
void NGA_Distribution(int g_a, int iproc, int lo[], int hi[]);
void GA_Copy(int g_a, int g_b);
void GA_Add(void *alpha, int g_a, void *beta, int g_b, int g_c);
void GA_Transpose(int g_a, int g_b);
void GA_Symmetrize(int g_a);
void GA_Dgemm(char ta, char tb, int m, int n, int k, double alpha,
              int g_a, int g_b, double beta, int g_c);
#endif
