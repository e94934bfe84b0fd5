/*
 * basis.c -- CInt basis-set API (libcint/include/CInt.h:45-86,123-145).
 *
 * Parses Gaussian-94 .gbs basis files (header line "spherical"/"cartesian",
 * element blocks terminated by "****", SP shells split into S + P, Fortran
 * 'D' exponents accepted) and .xyz geometries (natoms, title, "El x y z" in
 * Angstrom; tolerant of two atoms written on one line, as in
 * data/graphene/graphene_120_648_1464.xyz:77).  Called by pscf/scf.c:209-339
 * and pfock/pfock.c:829-903 in the reference.
 */
#define _GNU_SOURCE
#include <ctype.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "gtf_basis.h"

static const char *k_elements[] = {
    "X",  "H",  "He", "Li", "Be", "B",  "C",  "N",  "O",  "F",  "Ne",
    "Na", "Mg", "Al", "Si", "P",  "S",  "Cl", "Ar", "K",  "Ca", "Sc",
    "Ti", "V",  "Cr", "Mn", "Fe", "Co", "Ni", "Cu", "Zn", "Ga", "Ge",
    "As", "Se", "Br", "Kr", "Rb", "Sr", "Y",  "Zr", "Nb", "Mo", "Tc",
    "Ru", "Rh", "Pd", "Ag", "Cd", "In", "Sn", "Sb", "Te", "I",  "Xe"};
#define K_NELEM ((int)(sizeof(k_elements) / sizeof(k_elements[0])))

int gtf_element_z(const char *sym)
{
    for (int z = 1; z < K_NELEM; z++) {
        if (strcasecmp(sym, k_elements[z]) == 0) return z;
    }
    return -1;
}

const char *gtf_element_symbol(int z)
{
    return (z > 0 && z < K_NELEM) ? k_elements[z] : "X";
}

/* ------------------------------------------------------------------------ */
/* .gbs parsing                                                              */
/* ------------------------------------------------------------------------ */

typedef struct {
    int L;
    int nprim;
    double alpha[GTF_MAX_NPRIM];
    double d[GTF_MAX_NPRIM];
} raw_shell_t;

typedef struct {
    int nshell;
    raw_shell_t *sh;
} elem_basis_t;

static double parse_fortran_double(const char *s, int *ok)
{
    char buf[64];
    size_t n = strlen(s);
    if (n >= sizeof(buf)) n = sizeof(buf) - 1;
    for (size_t i = 0; i < n; i++) {
        buf[i] = (s[i] == 'D' || s[i] == 'd') ? 'E' : s[i];
    }
    buf[n] = 0;
    char *end = NULL;
    double v = strtod(buf, &end);
    *ok = (end != buf);
    return v;
}

static int shell_letter_L(const char *tok)
{
    if (strcasecmp(tok, "S") == 0) return 0;
    if (strcasecmp(tok, "P") == 0) return 1;
    if (strcasecmp(tok, "D") == 0) return 2;
    if (strcasecmp(tok, "F") == 0) return 3;
    if (strcasecmp(tok, "G") == 0) return 4;
    if (strcasecmp(tok, "SP") == 0 || strcasecmp(tok, "L") == 0) return -1;
    return -2;
}

/* next line of a NUL-terminated text buffer; returns NULL at the end */
static const char *next_line(const char *p, char *line, size_t cap)
{
    if (*p == 0) return NULL;
    size_t n = 0;
    while (*p && *p != '\n') {
        if (n + 1 < cap) line[n++] = *p;
        p++;
    }
    line[n] = 0;
    if (*p == '\n') p++;
    /* strip trailing CR/space */
    while (n > 0 && isspace((unsigned char)line[n - 1])) line[--n] = 0;
    return p;
}

static int is_blank_or_comment(const char *line)
{
    const char *q = line;
    while (*q && isspace((unsigned char)*q)) q++;
    return *q == 0 || *q == '!';
}

/* Parse a whole .gbs text into per-element shell lists.  Returns 0 on success. */
static int parse_gbs(const char *text, int *pure, elem_basis_t elems[K_NELEM])
{
    char line[512];
    const char *p = text;
    int have_header = 0;
    int cur = -1;            /* current element Z or -1 outside a block */
    memset(elems, 0, sizeof(elem_basis_t) * K_NELEM);
    while ((p = next_line(p, line, sizeof(line))) != NULL) {
        if (is_blank_or_comment(line)) continue;
        char t0[64] = {0}, t1[64] = {0}, t2[64] = {0}, t3[64] = {0};
        int nt = sscanf(line, "%63s %63s %63s %63s", t0, t1, t2, t3);
        if (!have_header) {
            if (strcasecmp(t0, "spherical") == 0) { *pure = 1; have_header = 1; continue; }
            if (strcasecmp(t0, "cartesian") == 0) { *pure = 0; have_header = 1; continue; }
        }
        if (strcmp(t0, "****") == 0) { cur = -1; continue; }
        if (cur < 0) {
            int z = gtf_element_z(t0);
            if (z > 0 && nt >= 2) {
                cur = z;
                have_header = 1;
                continue;
            }
            continue;
        }
        /* inside an element block: a shell header */
        int L = shell_letter_L(t0);
        if (L == -2 || nt < 2) return -1;
        int nprim = atoi(t1);
        if (nprim <= 0 || nprim > GTF_MAX_NPRIM) return -1;
        raw_shell_t s0, s1;
        memset(&s0, 0, sizeof(s0));
        memset(&s1, 0, sizeof(s1));
        s0.L = (L == -1) ? 0 : L;
        s1.L = 1;
        s0.nprim = s1.nprim = nprim;
        for (int i = 0; i < nprim; i++) {
            p = next_line(p, line, sizeof(line));
            if (p == NULL) return -1;
            char a[64] = {0}, c0[64] = {0}, c1[64] = {0};
            int nn = sscanf(line, "%63s %63s %63s", a, c0, c1);
            int ok0 = 0, ok1 = 0, ok2 = 0;
            s0.alpha[i] = s1.alpha[i] = parse_fortran_double(a, &ok0);
            s0.d[i] = parse_fortran_double(c0, &ok1);
            if (L == -1) {
                if (nn < 3) return -1;
                s1.d[i] = parse_fortran_double(c1, &ok2);
                if (!ok2) return -1;
            }
            if (!ok0 || !ok1) return -1;
        }
        elem_basis_t *e = &elems[cur];
        int add = (L == -1) ? 2 : 1;
        e->sh = (raw_shell_t *)realloc(e->sh, sizeof(raw_shell_t) * (e->nshell + add));
        if (e->sh == NULL) return -1;
        e->sh[e->nshell++] = s0;
        if (L == -1) e->sh[e->nshell++] = s1;
    }
    return have_header ? 0 : -1;
}

static double dfact(int n) /* (n)!! for odd n >= -1 */
{
    double r = 1.0;
    for (int k = n; k > 1; k -= 2) r *= k;
    return r;
}

/* Coefficients of the normalised contracted shell: each primitive is
 * normalised as x^L exp(-a r^2), then the contraction is rescaled to unit
 * self-overlap. */
static void normalise_shell(const raw_shell_t *s, double *coef)
{
    const int L = s->L;
    const double df = dfact(2 * L - 1);
    double nrm[GTF_MAX_NPRIM];
    for (int i = 0; i < s->nprim; i++) {
        double a = s->alpha[i];
        nrm[i] = pow(2.0 * a / M_PI, 0.75) * pow(4.0 * a, 0.5 * L) / sqrt(df);
    }
    double ss = 0.0;
    for (int i = 0; i < s->nprim; i++) {
        for (int j = 0; j < s->nprim; j++) {
            double p = s->alpha[i] + s->alpha[j];
            ss += s->d[i] * s->d[j] * nrm[i] * nrm[j] *
                  pow(M_PI / p, 1.5) * df / pow(2.0 * p, L);
        }
    }
    double f = 1.0 / sqrt(ss);
    for (int i = 0; i < s->nprim; i++) coef[i] = s->d[i] * nrm[i] * f;
}

static void free_basis_arrays(BasisSet_t b)
{
    free(b->Z); free(b->xyz); free(b->atom_sstart);
    free(b->sh_atom); free(b->sh_L); free(b->sh_nprim); free(b->sh_pstart);
    free(b->f_start); free(b->fc_start); free(b->alpha); free(b->coef);
    if (b->guess) {
        for (int i = 0; i < b->natoms; i++) free(b->guess[i]);
        free(b->guess);
    }
    char dir[1024];
    memcpy(dir, b->bsdir, sizeof(dir));
    memset(b, 0, sizeof(*b));
    memcpy(b->bsdir, dir, sizeof(dir));
}

static void finish_basis(BasisSet_t b)
{
    b->nbf = 0;
    b->nbf_cart = 0;
    b->maxdim = 0;
    for (int s = 0; s < b->nshells; s++) {
        b->f_start[s] = b->nbf;
        b->fc_start[s] = b->nbf_cart;
        int d = gtf_shell_dim(b->sh_L[s], b->pure);
        b->nbf += d;
        b->nbf_cart += gtf_cart_dim(b->sh_L[s]);
        if (d > b->maxdim) b->maxdim = d;
    }
    b->f_start[b->nshells] = b->nbf;
    b->fc_start[b->nshells] = b->nbf_cart;
    b->nneutral = 0;
    for (int a = 0; a < b->natoms; a++) b->nneutral += b->Z[a];
    double e = 0.0;
    for (int a = 0; a < b->natoms; a++) {
        for (int c = a + 1; c < b->natoms; c++) {
            double dx = b->xyz[3 * a] - b->xyz[3 * c];
            double dy = b->xyz[3 * a + 1] - b->xyz[3 * c + 1];
            double dz = b->xyz[3 * a + 2] - b->xyz[3 * c + 2];
            e += (double)b->Z[a] * b->Z[c] / sqrt(dx * dx + dy * dy + dz * dz);
        }
    }
    b->enuc = e;
    b->guess = (double **)calloc((size_t)b->natoms, sizeof(double *));
}

CIntStatus_t gtf_basis_build(BasisSet_t b, const char *gbs_text,
                             int natoms, const int *Z, const double *xyz_bohr,
                             const char *bsdir)
{
    if (b == NULL || gbs_text == NULL || natoms <= 0) return CINT_STATUS_INVALID_VALUE;
    elem_basis_t elems[K_NELEM];
    int pure = 0;
    if (parse_gbs(gbs_text, &pure, elems) != 0) {
        for (int z = 0; z < K_NELEM; z++) free(elems[z].sh);
        return CINT_STATUS_FILEIO_FAILED;
    }
    CIntStatus_t st = CINT_STATUS_SUCCESS;
    free_basis_arrays(b);
    if (bsdir) snprintf(b->bsdir, sizeof(b->bsdir), "%s", bsdir);
    b->pure = pure;
    b->natoms = natoms;
    int nsh = 0, npr = 0;
    for (int a = 0; a < natoms; a++) {
        if (Z[a] <= 0 || Z[a] >= K_NELEM || elems[Z[a]].nshell == 0) {
            st = CINT_STATUS_INVALID_VALUE;
            goto done;
        }
        for (int s = 0; s < elems[Z[a]].nshell; s++) {
            if (elems[Z[a]].sh[s].L > GTF_MAX_L) { st = CINT_STATUS_INVALID_VALUE; goto done; }
            npr += elems[Z[a]].sh[s].nprim;
        }
        nsh += elems[Z[a]].nshell;
    }
    b->nshells = nsh;
    b->nprims = npr;
    b->Z = (int *)malloc(sizeof(int) * natoms);
    b->xyz = (double *)malloc(sizeof(double) * 3 * natoms);
    b->atom_sstart = (int *)malloc(sizeof(int) * (natoms + 1));
    b->sh_atom = (int *)malloc(sizeof(int) * nsh);
    b->sh_L = (int *)malloc(sizeof(int) * nsh);
    b->sh_nprim = (int *)malloc(sizeof(int) * nsh);
    b->sh_pstart = (int *)malloc(sizeof(int) * nsh);
    b->f_start = (int *)malloc(sizeof(int) * (nsh + 1));
    b->fc_start = (int *)malloc(sizeof(int) * (nsh + 1));
    b->alpha = (double *)malloc(sizeof(double) * npr);
    b->coef = (double *)malloc(sizeof(double) * npr);
    if (!b->Z || !b->xyz || !b->atom_sstart || !b->sh_atom || !b->sh_L ||
        !b->sh_nprim || !b->sh_pstart || !b->f_start || !b->fc_start ||
        !b->alpha || !b->coef) {
        st = CINT_STATUS_ALLOC_FAILED;
        goto done;
    }
    nsh = 0;
    npr = 0;
    for (int a = 0; a < natoms; a++) {
        b->Z[a] = Z[a];
        b->xyz[3 * a] = xyz_bohr[3 * a];
        b->xyz[3 * a + 1] = xyz_bohr[3 * a + 1];
        b->xyz[3 * a + 2] = xyz_bohr[3 * a + 2];
        b->atom_sstart[a] = nsh;
        const elem_basis_t *e = &elems[Z[a]];
        for (int s = 0; s < e->nshell; s++) {
            b->sh_atom[nsh] = a;
            b->sh_L[nsh] = e->sh[s].L;
            b->sh_nprim[nsh] = e->sh[s].nprim;
            b->sh_pstart[nsh] = npr;
            normalise_shell(&e->sh[s], &b->coef[npr]);
            for (int i = 0; i < e->sh[s].nprim; i++) b->alpha[npr + i] = e->sh[s].alpha[i];
            npr += e->sh[s].nprim;
            nsh++;
        }
    }
    b->atom_sstart[natoms] = nsh;
    finish_basis(b);
done:
    for (int z = 0; z < K_NELEM; z++) free(elems[z].sh);
    if (st != CINT_STATUS_SUCCESS) free_basis_arrays(b);
    return st;
}

static char *read_file(const char *path)
{
    FILE *fp = fopen(path, "rb");
    if (!fp) return NULL;
    fseek(fp, 0, SEEK_END);
    long n = ftell(fp);
    fseek(fp, 0, SEEK_SET);
    char *buf = (char *)malloc((size_t)n + 1);
    if (!buf) { fclose(fp); return NULL; }
    size_t got = fread(buf, 1, (size_t)n, fp);
    fclose(fp);
    buf[got] = 0;
    return buf;
}

/* Parse an .xyz text: natoms, a title line, then natoms "El x y z" records
 * read as a token stream (so records need not be one per line). */
static int parse_xyz(const char *text, int *natoms_out, int **Z_out, double **xyz_out)
{
    char line[512];
    const char *p = next_line(text, line, sizeof(line));
    if (p == NULL) return -1;
    int natoms = atoi(line);
    if (natoms <= 0) return -1;
    p = next_line(p, line, sizeof(line)); /* title */
    if (p == NULL) return -1;
    int *Z = (int *)malloc(sizeof(int) * natoms);
    double *xyz = (double *)malloc(sizeof(double) * 3 * natoms);
    if (!Z || !xyz) { free(Z); free(xyz); return -1; }
    const char *q = p;
    for (int a = 0; a < natoms; a++) {
        while (*q && isspace((unsigned char)*q)) q++;
        char sym[8] = {0};
        int n = 0;
        while (*q && isalpha((unsigned char)*q) && n < 7) sym[n++] = *q++;
        int z = gtf_element_z(sym);
        if (z <= 0) { free(Z); free(xyz); return -1; }
        Z[a] = z;
        for (int k = 0; k < 3; k++) {
            char *end = NULL;
            double v = strtod(q, &end);
            if (end == q) { free(Z); free(xyz); return -1; }
            xyz[3 * a + k] = v / GTF_BOHR_ANGSTROM;
            q = end;
        }
    }
    *natoms_out = natoms;
    *Z_out = Z;
    *xyz_out = xyz;
    return 0;
}

CIntStatus_t CInt_createBasisSet(BasisSet_t *basis)
{
    if (basis == NULL) return CINT_STATUS_INVALID_VALUE;
    BasisSet_t b = (BasisSet_t)calloc(1, sizeof(struct BasisSet));
    if (b == NULL) return CINT_STATUS_ALLOC_FAILED;
    *basis = b;
    return CINT_STATUS_SUCCESS;
}

CIntStatus_t CInt_destroyBasisSet(BasisSet_t basis)
{
    if (basis == NULL) return CINT_STATUS_INVALID_VALUE;
    free_basis_arrays(basis);
    free(basis);
    return CINT_STATUS_SUCCESS;
}

CIntStatus_t CInt_loadBasisSet(BasisSet_t basis, char *bsfile, char *xyzfile)
{
    if (basis == NULL || bsfile == NULL || xyzfile == NULL) return CINT_STATUS_INVALID_VALUE;
    char *gbs = read_file(bsfile);
    if (gbs == NULL) return CINT_STATUS_FILEIO_FAILED;
    char *xyz = read_file(xyzfile);
    if (xyz == NULL) { free(gbs); return CINT_STATUS_FILEIO_FAILED; }
    int natoms = 0;
    int *Z = NULL;
    double *pos = NULL;
    CIntStatus_t st;
    if (parse_xyz(xyz, &natoms, &Z, &pos) != 0) {
        st = CINT_STATUS_FILEIO_FAILED;
    } else {
        char dir[1024];
        snprintf(dir, sizeof(dir), "%s", bsfile);
        char *slash = strrchr(dir, '/');
        if (slash) *slash = 0; else snprintf(dir, sizeof(dir), ".");
        st = gtf_basis_build(basis, gbs, natoms, Z, pos, dir);
    }
    free(Z);
    free(pos);
    free(gbs);
    free(xyz);
    return st;
}

CIntStatus_t CInt_importBasisSet(BasisSet_t basis, int natoms, int *Zs,
                                 double *X, double *Y, double *Z,
                                 int nprims, int nshells, int pure,
                                 int *shells_p_atom, int *prims_p_shell,
                                 int *L, double *cc, double *alpha)
{
    /* Coordinates are taken in bohr; cc are the raw contraction coefficients
     * of each shell (as written in a .gbs file) and are normalised here. */
    if (basis == NULL || natoms <= 0 || nshells <= 0 || nprims <= 0) return CINT_STATUS_INVALID_VALUE;
    free_basis_arrays(basis);
    BasisSet_t b = basis;
    b->natoms = natoms;
    b->nshells = nshells;
    b->nprims = nprims;
    b->pure = pure ? 1 : 0;
    b->Z = (int *)malloc(sizeof(int) * natoms);
    b->xyz = (double *)malloc(sizeof(double) * 3 * natoms);
    b->atom_sstart = (int *)malloc(sizeof(int) * (natoms + 1));
    b->sh_atom = (int *)malloc(sizeof(int) * nshells);
    b->sh_L = (int *)malloc(sizeof(int) * nshells);
    b->sh_nprim = (int *)malloc(sizeof(int) * nshells);
    b->sh_pstart = (int *)malloc(sizeof(int) * nshells);
    b->f_start = (int *)malloc(sizeof(int) * (nshells + 1));
    b->fc_start = (int *)malloc(sizeof(int) * (nshells + 1));
    b->alpha = (double *)malloc(sizeof(double) * nprims);
    b->coef = (double *)malloc(sizeof(double) * nprims);
    if (!b->Z || !b->xyz || !b->atom_sstart || !b->sh_atom || !b->sh_L ||
        !b->sh_nprim || !b->sh_pstart || !b->f_start || !b->fc_start ||
        !b->alpha || !b->coef) {
        free_basis_arrays(b);
        return CINT_STATUS_ALLOC_FAILED;
    }
    int s = 0, p = 0;
    for (int a = 0; a < natoms; a++) {
        b->Z[a] = Zs[a];
        b->xyz[3 * a] = X[a];
        b->xyz[3 * a + 1] = Y[a];
        b->xyz[3 * a + 2] = Z[a];
        b->atom_sstart[a] = s;
        for (int k = 0; k < shells_p_atom[a]; k++, s++) {
            if (s >= nshells || L[s] < 0 || L[s] > GTF_MAX_L ||
                prims_p_shell[s] <= 0 || prims_p_shell[s] > GTF_MAX_NPRIM ||
                p + prims_p_shell[s] > nprims) {
                free_basis_arrays(b);
                return CINT_STATUS_INVALID_VALUE;
            }
            raw_shell_t rs;
            rs.L = L[s];
            rs.nprim = prims_p_shell[s];
            for (int i = 0; i < rs.nprim; i++) {
                rs.alpha[i] = alpha[p + i];
                rs.d[i] = cc[p + i];
            }
            b->sh_atom[s] = a;
            b->sh_L[s] = L[s];
            b->sh_nprim[s] = rs.nprim;
            b->sh_pstart[s] = p;
            normalise_shell(&rs, &b->coef[p]);
            for (int i = 0; i < rs.nprim; i++) b->alpha[p + i] = rs.alpha[i];
            p += rs.nprim;
        }
    }
    if (s != nshells || p != nprims) {
        free_basis_arrays(b);
        return CINT_STATUS_INVALID_VALUE;
    }
    b->atom_sstart[natoms] = s;
    finish_basis(b);
    return CINT_STATUS_SUCCESS;
}

/* ------------------------------------------------------------------------ */
/* pack / unpack (pscf/scf.c:284-296 broadcasts this blob)                   */
/* ------------------------------------------------------------------------ */

#define PACK_MAGIC 0x47544642 /* "GTFB" */

static size_t pack_int_count(int natoms, int nshells)
{
    return 8 + (size_t)natoms + (size_t)(natoms + 1) + 4 * (size_t)nshells;
}

CIntStatus_t CInt_packBasisSet(BasisSet_t b, void **buf, int *bufsize)
{
    if (b == NULL || buf == NULL || bufsize == NULL) return CINT_STATUS_INVALID_VALUE;
    size_t ioff = (pack_int_count(b->natoms, b->nshells) * sizeof(int) + 7) & ~(size_t)7;
    size_t nd = (size_t)b->natoms * 3 + (size_t)b->nprims * 2;
    size_t bytes = ioff + nd * sizeof(double) + sizeof(b->bsdir);
    char *p = (char *)calloc(1, bytes);
    if (p == NULL) return CINT_STATUS_ALLOC_FAILED;
    int *ip = (int *)p;
    ip[0] = PACK_MAGIC; ip[1] = b->natoms; ip[2] = b->nshells; ip[3] = b->nprims;
    ip[4] = b->pure; ip[5] = b->charge; ip[6] = 0; ip[7] = 0;
    int k = 8;
    for (int a = 0; a < b->natoms; a++) ip[k++] = b->Z[a];
    for (int a = 0; a <= b->natoms; a++) ip[k++] = b->atom_sstart[a];
    for (int s = 0; s < b->nshells; s++) {
        ip[k++] = b->sh_atom[s]; ip[k++] = b->sh_L[s];
        ip[k++] = b->sh_nprim[s]; ip[k++] = b->sh_pstart[s];
    }
    double *dp = (double *)(p + ioff);
    size_t j = 0;
    for (int a = 0; a < 3 * b->natoms; a++) dp[j++] = b->xyz[a];
    for (int i = 0; i < b->nprims; i++) dp[j++] = b->alpha[i];
    for (int i = 0; i < b->nprims; i++) dp[j++] = b->coef[i];
    memcpy(dp + j, b->bsdir, sizeof(b->bsdir));
    *buf = p;
    *bufsize = (int)bytes;
    return CINT_STATUS_SUCCESS;
}

CIntStatus_t CInt_unpackBasisSet(BasisSet_t b, void *buf)
{
    if (b == NULL || buf == NULL) return CINT_STATUS_INVALID_VALUE;
    const char *p = (const char *)buf;
    const int *ip = (const int *)p;
    if (ip[0] != PACK_MAGIC) return CINT_STATUS_INVALID_VALUE;
    free_basis_arrays(b);
    b->natoms = ip[1]; b->nshells = ip[2]; b->nprims = ip[3];
    b->pure = ip[4]; b->charge = ip[5];
    int na = b->natoms, ns = b->nshells, np = b->nprims;
    b->Z = (int *)malloc(sizeof(int) * na);
    b->xyz = (double *)malloc(sizeof(double) * 3 * na);
    b->atom_sstart = (int *)malloc(sizeof(int) * (na + 1));
    b->sh_atom = (int *)malloc(sizeof(int) * ns);
    b->sh_L = (int *)malloc(sizeof(int) * ns);
    b->sh_nprim = (int *)malloc(sizeof(int) * ns);
    b->sh_pstart = (int *)malloc(sizeof(int) * ns);
    b->f_start = (int *)malloc(sizeof(int) * (ns + 1));
    b->fc_start = (int *)malloc(sizeof(int) * (ns + 1));
    b->alpha = (double *)malloc(sizeof(double) * np);
    b->coef = (double *)malloc(sizeof(double) * np);
    if (!b->Z || !b->xyz || !b->atom_sstart || !b->sh_atom || !b->sh_L ||
        !b->sh_nprim || !b->sh_pstart || !b->f_start || !b->fc_start ||
        !b->alpha || !b->coef) {
        free_basis_arrays(b);
        return CINT_STATUS_ALLOC_FAILED;
    }
    int k = 8;
    for (int a = 0; a < na; a++) b->Z[a] = ip[k++];
    for (int a = 0; a <= na; a++) b->atom_sstart[a] = ip[k++];
    for (int s = 0; s < ns; s++) {
        b->sh_atom[s] = ip[k++]; b->sh_L[s] = ip[k++];
        b->sh_nprim[s] = ip[k++]; b->sh_pstart[s] = ip[k++];
    }
    size_t ioff = (pack_int_count(na, ns) * sizeof(int) + 7) & ~(size_t)7;
    const double *dp = (const double *)(p + ioff);
    size_t j = 0;
    for (int a = 0; a < 3 * na; a++) b->xyz[a] = dp[j++];
    for (int i = 0; i < np; i++) b->alpha[i] = dp[j++];
    for (int i = 0; i < np; i++) b->coef[i] = dp[j++];
    memcpy(b->bsdir, dp + j, sizeof(b->bsdir));
    b->bsdir[sizeof(b->bsdir) - 1] = 0;
    finish_basis(b);
    return CINT_STATUS_SUCCESS;
}

/* ------------------------------------------------------------------------ */
/* queries                                                                   */
/* ------------------------------------------------------------------------ */

int CInt_getNumShells(BasisSet_t b) { return b->nshells; }
int CInt_getNumFuncs(BasisSet_t b) { return b->nbf; }
int CInt_getNumAtoms(BasisSet_t b) { return b->natoms; }
int CInt_getMaxShellDim(BasisSet_t b) { return b->maxdim; }
int CInt_getTotalCharge(BasisSet_t b) { return b->charge; }
int CInt_getNneutral(BasisSet_t b) { return b->nneutral; }
double CInt_getNucEnergy(BasisSet_t b) { return b->enuc; }

int CInt_getNumOccOrb(BasisSet_t b)
{
    /* closed-shell occupation: (sum Z - charge) / 2 */
    return (b->nneutral - b->charge) / 2;
}

int CInt_getShellDim(BasisSet_t b, int s) { return b->f_start[s + 1] - b->f_start[s]; }
int CInt_getFuncStartInd(BasisSet_t b, int s) { return b->f_start[s]; }
int CInt_getFuncEndInd(BasisSet_t b, int s) { return b->f_start[s + 1]; }
int CInt_getAtomStartInd(BasisSet_t b, int a) { return b->atom_sstart[a]; }

void CInt_getShellxyz(BasisSet_t b, int s, double *x, double *y, double *z)
{
    int a = b->sh_atom[s];
    *x = b->xyz[3 * a];
    *y = b->xyz[3 * a + 1];
    *z = b->xyz[3 * a + 2];
}

/* Initial-guess block of one atom: <basis dir>/<El>.dat holds nf*nf values
 * (row-major) for an atom with nf functions, as in data/opt-cc-pvdz/H.dat.
 * When the file is absent or has the wrong length the block is zero, which
 * makes the first SCF iteration a core-Hamiltonian guess. */
void CInt_getInitialGuess(BasisSet_t b, int atomid, double **guess, int *spos, int *epos)
{
    int s0 = b->atom_sstart[atomid];
    int s1 = b->atom_sstart[atomid + 1];
    int f0 = b->f_start[s0];
    int f1 = b->f_start[s1];
    int nf = f1 - f0;
    *spos = f0;
    *epos = f1 - 1;
    if (b->guess[atomid] == NULL) {
        double *g = (double *)calloc((size_t)nf * nf, sizeof(double));
        char path[1200];
        snprintf(path, sizeof(path), "%s/%s.dat", b->bsdir, gtf_element_symbol(b->Z[atomid]));
        FILE *fp = fopen(path, "r");
        if (fp && g) {
            int n = 0;
            double v;
            double *tmp = (double *)malloc(sizeof(double) * nf * nf);
            while (tmp && n < nf * nf && fscanf(fp, "%lf", &v) == 1) tmp[n++] = v;
            if (tmp && n == nf * nf && fscanf(fp, "%lf", &v) != 1) memcpy(g, tmp, sizeof(double) * nf * nf);
            free(tmp);
        }
        if (fp) fclose(fp);
        b->guess[atomid] = g;
    }
    *guess = b->guess[atomid];
}
