/*
 * mdgpu oracle -- CPU restatement of the reference's multifrontal Cholesky path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker for the CUDA product:
 * only tests, the smoke check and the benchmark's CPU-baseline leg may load it.
 * It restates, in plain C, the reference's host symbolic phase, its numeric
 * multifrontal factorization (CPU branch) and the CSparse solves, each function
 * citing the reference file:line it follows.  Its outputs are pinned against
 * the reference itself (oracle/_ref, built by oracle/Makefile) through the
 * golden fixtures in tests/golden/.
 *
 * Index type: int (the reference's cs uses 32-bit int).  Scalar: double (the
 * reference's FP64 build, types.h:13-22).
 */
#ifndef MDGPU_ORACLE_H
#define MDGPU_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* Supernode-tree construction mode. */
enum { ORC_NODAL = 0, ORC_SUPER = 1, ORC_RELAXED = 2 };

typedef struct orc_plan {
    int n;
    /* permuted lower triangle of A, as the reference's Factor receives it */
    int *Ap, *Ai;
    double *Ax;
    /* overall fill-reducing permutation (new -> old); NULL for natural order */
    int *perm;
    int *parent, *post, *count0; /* cs_etree / cs_post / cs_counts outputs */
    int *count;                  /* column counts used for Lp (mutated by -rn) */
    int *rn_perm;                /* GetRelaxedETree permutation (NULL otherwise) */
    /* supernodes in the driver's (post)order */
    int nsuper;
    int *sn_nodo, *sn_cols, *sn_childptr, *sn_child;
    int *Lp;
    long long lnz;
} orc_plan;

/* Full symbolic pipeline of mdgpu.cu:1745-1875 on a lower-triangular CSC. */
int orc_analyze(int n, const int *Ap, const int *Ai, const double *Ax, int use_amd, int mode,
                int rn_zeros, orc_plan **out);
void orc_plan_free(orc_plan *p);

/* Numeric multifrontal factor of Factor (mdgpu.cu:1394-1608) with the CPU
 * dense kernel FactorAux_CPU_3 (mdgpu.cu:1298-1361); block_size <= 0 means no
 * -b (one panel per front).  Fills Li/Lx (length lnz) like spL.  If rows_ptr /
 * rows / relmap are non-NULL they receive, per supernode s, its front row set
 * (rows_ptr[s]..rows_ptr[s+1]) and the composed extend-add map of its update
 * rows into its parent's front (relmap at rows_ptr[s]+cols[s]..rows_ptr[s+1]),
 * -1 for the root.  Returns 0, or -(col+1) of the first non-positive pivot. */
int orc_factor(const orc_plan *p, int block_size, int *Li, double *Lx, double *flops,
               int *rows_ptr, int *rows, int *relmap);

/* x = P L^-T L^-1 P^T b (mdgpu.cu:1952-1961 with cs_lsolve / cs_ltsolve). */
void orc_solve(const orc_plan *p, const int *Li, const double *Lx, const double *b, double *x);

/* Relative residual ||Ax-b||_inf / (||A||_1 ||x||_inf + ||b||_inf) of the
 * ORIGINAL (unpermuted) lower-stored matrix (mdgpu.cu:1963-1972). */
double orc_residual(int n, const int *Ap, const int *Ai, const double *Ax, const double *x,
                    const double *b);

/* Individual symbolic steps (CSparse semantics). */
int orc_amd(int n, const int *Up, const int *Ui, int *perm);          /* cs_amd(1, A_upper) */
int orc_etree(int n, const int *Ap, const int *Ai, int *parent);      /* cs_etree(A, 0) */
int orc_post(int n, const int *parent, int *post);                    /* cs_post */
int orc_counts(int n, const int *Ap, const int *Ai, const int *parent, const int *post,
               int *count);                                           /* cs_counts(A,..,0) */

/* Dense partial Cholesky of one column-major n x n front with `cols` pivot
 * columns: the FactorAux_CPU_3 blocked algorithm (mdgpu.cu:1312-1341). */
void orc_front_factor(int n, int cols, int block_size, double *F);

/* plan accessors for foreign-function callers */
int orc_plan_n(const orc_plan *p);
int orc_plan_nsuper(const orc_plan *p);
long long orc_plan_lnz(const orc_plan *p);
int orc_plan_nchild_total(const orc_plan *p);
int orc_plan_nnz_low(const orc_plan *p);
void orc_plan_copy(const orc_plan *p, const char *what, void *dst);

#ifdef __cplusplus
}
#endif
#endif
