/*
 * gtf_basis.h -- in-memory layout of a loaded basis set (host side).
 *
 * The reference keeps this state inside its binary integral library
 * (libcint, reached through libcint/include/CInt.h:45-145); here it is a
 * plain C struct so that the PFock engine can upload it to the GPU as
 * structure-of-arrays.  Shells are ordered atom by atom, and within an atom in
 * the order of the .gbs element block (an SP shell becomes S then P).
 */
#ifndef GTF_BASIS_H
#define GTF_BASIS_H

#include "CInt.h"

#define GTF_MAX_L 2           /* s, p, d: what cc-pVDZ/6-31G/STO-3G need for H..Ne */
#define GTF_MAX_NPRIM 16      /* largest contraction accepted per shell */
#define GTF_BOHR_ANGSTROM 0.529177210903

struct BasisSet {
    int natoms;
    int nshells;
    int nbf;          /* number of basis functions (spherical or Cartesian) */
    int nbf_cart;     /* number of Cartesian functions (== nbf when !pure) */
    int nprims;       /* total primitives over all shells */
    int pure;         /* 1: spherical harmonics for L >= 2, 0: Cartesian */
    int maxdim;       /* largest shell dimension */
    int charge;
    int nneutral;     /* sum of nuclear charges */
    double enuc;      /* nuclear repulsion energy (Hartree) */

    int *Z;           /* [natoms] */
    double *xyz;      /* [3*natoms] bohr */
    int *atom_sstart; /* [natoms+1] first shell of each atom */

    int *sh_atom;     /* [nshells] */
    int *sh_L;        /* [nshells] */
    int *sh_nprim;    /* [nshells] */
    int *sh_pstart;   /* [nshells] offset into alpha/coef */
    int *f_start;     /* [nshells+1] first function of each shell */
    int *fc_start;    /* [nshells+1] first Cartesian function of each shell */
    double *alpha;    /* [nprims] exponents */
    double *coef;     /* [nprims] coefficients incl. primitive + contraction norm */

    char bsdir[1024]; /* directory of the .gbs file (initial-guess .dat files) */
    double **guess;   /* [natoms] lazily built initial-guess blocks */
};

#ifdef __cplusplus
extern "C" {
#endif

/* number of functions of a shell of angular momentum L */
static inline int gtf_shell_dim(int L, int pure)
{
    return pure ? 2 * L + 1 : (L + 1) * (L + 2) / 2;
}

static inline int gtf_cart_dim(int L) { return (L + 1) * (L + 2) / 2; }

/* element symbol <-> nuclear charge (H..Xe) */
int gtf_element_z(const char *sym);
const char *gtf_element_symbol(int z);

/* Build a basis set from an in-memory .gbs text and an atom list (bohr).
 * Used by CInt_loadBasisSet and by the request path that receives geometries
 * without files. */
CIntStatus_t gtf_basis_build(BasisSet_t basis, const char *gbs_text,
                             int natoms, const int *Z, const double *xyz_bohr,
                             const char *bsdir);

#ifdef __cplusplus
}
#endif

#endif
