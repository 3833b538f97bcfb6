/*
 * mdgpu_b200 -- C ABI of the B200 multifrontal sparse Cholesky.
 *
 * Plain pointers and sizes only.  Index arrays are 32-bit `int` like the
 * reference's CSparse `cs` struct (cs.h:20-29); values are `double` (the
 * reference's FLOTANTE in its FP64 build, types.h:13-22).  The input matrix is
 * the LOWER triangle, diagonal included, in compressed-column form with sorted
 * row indices -- what the reference holds after cs_load + cs_compress
 * (mdgpu.cu:1724-1729).
 *
 * Every function returns an mdgpu_status (0 = success).  There is no global
 * state: one handle per sparsity pattern; calls on different handles may run
 * concurrently from different host threads.  A handle must not be used by two
 * host threads at once.
 */
#ifndef MDGPU_B200_H
#define MDGPU_B200_H

#if defined(__GNUC__)
#define MDGPU_API __attribute__((visibility("default")))
#else
#define MDGPU_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

typedef struct mdgpu_handle_s *mdgpu_handle;

enum mdgpu_status {
    MDGPU_OK = 0,
    MDGPU_ERR_INVALID = -1,   /* bad argument or pattern */
    MDGPU_ERR_NOT_SPD = -2,   /* non-positive pivot; see mdgpu_not_spd_column */
    MDGPU_ERR_OOM = -3,       /* device or host allocation failed */
    MDGPU_ERR_CUDA = -4,      /* CUDA runtime error (message: mdgpu_last_error) */
    MDGPU_ERR_NOT_TREE = -5,  /* elimination tree is a forest (etree.cpp:27-31) */
    MDGPU_ERR_STATE = -6,     /* e.g. solve before factor */
    MDGPU_ERR_NO_DEVICE = -7  /* no CUDA device: the numeric phase never runs on the CPU */
};

enum mdgpu_ordering { MDGPU_ORDER_NATURAL = 0, MDGPU_ORDER_AMD = 1 };
enum mdgpu_tree { MDGPU_TREE_NODAL = 0, MDGPU_TREE_SUPER = 1, MDGPU_TREE_RELAXED = 2 };
enum mdgpu_precision {
    MDGPU_FP64 = 0, /* plain FP64 factor: the drop-in mode */
    MDGPU_FP32 = 1, /* FP32 factor; Schur updates of large fronts on the tensor cores in
                       3xTF32 (close to FP32 accuracy) */
    MDGPU_BF16 = 2, /* FP32 factor whose large-front Schur updates take BF16 operands (one
                       tensor-core product, FP32 accumulation): for GMRES-IR
                       (mdgpu_gmres_ir); a factorization that meets a non-positive pivot is
                       redone in FP32 (mdgpu_info "bf16_fallbacks", "precision_used") */
    MDGPU_TF32 = 3  /* FP32 factor whose large-front Schur updates are one TF32 tensor-core
                       product (the operands' low 13 mantissa bits dropped): for GMRES-IR;
                       redone in FP32 on a non-positive pivot as MDGPU_BF16 */
};

/*
 * Symbolic analysis.  Replaces the reference driver's symbolic sequence
 * (mdgpu.cu:1745-1875): cs_transpose + cs_amd + cs_pinv + cs_symperm +
 * make_sym, cs_etree, cs_post, cs_counts, GetETree, then GetSuperETree
 * (tree = SUPER, flag -sn) or GetRelaxedETree (tree = RELAXED, flag -rn z),
 * and the spL->p column pointers.  Bit-identical to the reference.  Also
 * uploads the numeric plan (front row sets, extend-add maps, schedules) to
 * the current CUDA device when one is present.
 */
MDGPU_API int mdgpu_analyze(int n, const int *Ap, const int *Ai, int ordering, int tree, int relax_zeros,
                  mdgpu_handle *out);

/*
 * Read a matrix file, the reference's cs_load + cs_compress (cs.cpp:4-27,
 * 251-270, as its driver calls them, mdgpu.cu:1725-1729).  format 0: the
 * reference's own input, 1-based "i j x" triples read until the first line
 * that is not one (an index below 1 is an error, as in cs_entry); format 1:
 * a Matrix Market real coordinate file ('%' lines skipped, then the
 * "rows cols entries" line, whose sizes are used and checked).  *m, *n: the
 * largest indices (format 0) or the stated sizes; *nnz: the entries read.
 * With Ap (n + 1 entries) non-NULL, also the compressed columns: Ai (row
 * indices, 0-based) and Ax (values) receive nnz entries each (either may be
 * NULL), a column's entries in file order, as cs_compress leaves them.  Call
 * once with Ap = NULL for the sizes, then with arrays of those sizes.  For
 * mdgpu_analyze the file holds the lower triangle (a Matrix Market
 * "symmetric" file does) with rows ascending within each column.
 */
MDGPU_API int mdgpu_load_triplet(const char *path, int format, int *m, int *n, int *nnz, int *Ap,
                                 int *Ai, double *Ax);

/*
 * Many independent SPD systems under one handle (the batched mode of the
 * many-systems workload; the reference handles one system per run).  System
 * b is the lower triangle (n[b], Ap[b], Ai[b]); each is analysed on its own
 * exactly as mdgpu_analyze would, then the systems are numbered one after
 * another as one block-diagonal matrix, so one factor / solve call works on
 * all of them in the same level-scheduled launches.  Values and right-hand
 * sides are the systems' arrays concatenated in order; mdgpu_get_array
 * "sys_row_off" and "sys_val_off" (nsys + 1 entries, mdgpu_info "nsys") give
 * each system's first row and first value.  MDGPU_ERR_NOT_TREE names a
 * system whose elimination tree is a forest.
 */
MDGPU_API int mdgpu_analyze_batch(int nsys, const int *n, const int *const *Ap,
                                  const int *const *Ai, int ordering, int tree, int relax_zeros,
                                  mdgpu_handle *out);

/*
 * Cost estimate of independent systems without a handle or a device (no
 * counterpart in the reference): the same symbolic analysis as
 * mdgpu_analyze_batch for each system (on all host cores), reduced to its
 * flop count (as mdgpu_info "flops") in flops[nsys] and its L entries in
 * lnz[nsys] (optional).  For partitioning systems across GPUs.
 */
MDGPU_API int mdgpu_estimate_batch(int nsys, const int *n, const int *const *Ap,
                                   const int *const *Ai, int ordering, int tree, int relax_zeros,
                                   double *flops, long long *lnz);
/*
 * Analysis from an already permuted lower triangle and a given assembly tree,
 * the inputs of the reference's Factor(cs *A, cs *spL, ETree **listaNodos,
 * int cantNodos) (mdgpu.cu:1394): supernode s eliminates columns
 * first_col[s] .. first_col[s]+ncols[s]-1, its children are
 * child[child_ptr[s] .. child_ptr[s+1]-1], supernodes in postorder (root
 * last), and count[] are the L column counts that define spL->p.
 */
MDGPU_API int mdgpu_analyze_tree(int n, const int *Ap, const int *Ai, int nsuper, const int *first_col,
                       const int *ncols, const int *child_ptr, const int *child, const int *count,
                       mdgpu_handle *out);

MDGPU_API void mdgpu_destroy(mdgpu_handle h);

/*
 * Diagnostic (no counterpart in the reference): check on the host every
 * invariant the device kernels rely on when they index the handle's tables
 * -- front row sets strictly increasing and inside n, relative maps pointing
 * at the same row of the parent, every A entry at its row and column, level
 * and warp lists holding each front once, assembly maps and solve task
 * order, the residual's CSR in range.  MDGPU_OK, or MDGPU_ERR_INVALID with
 * the failed invariant and its front in mdgpu_last_error().  Host only.
 * With the environment variable MDGPU_CHECK_PLAN=1 every analysis runs the
 * same check before its tables reach the device, and fails if it fails.
 */
MDGPU_API int mdgpu_check_plan(mdgpu_handle h);

/* Scalars: "n", "nsuper", "lnz", "nlevels", "nnz", "max_front", "flops"
 * (the reference's own count, mdgpu.cu:1354-1359), "lstore_bytes",
 * "ustore_bytes" (the update-matrix store, reused over the matrices'
 * lifetimes), "ustore_total_bytes" (the sum of every update matrix: the store
 * without reuse), "zustore_bytes" (the selected inverse's update parts),
 * "fp64_diag_tiles" (diagonal tiles of the last FP32 / BF16 factor whose
 * pivots were weak -- d^2 < a / 1024 or not positive -- and were factored
 * again in FP64), "bf16_fallbacks", "precision_used" (the current factor's
 * precision),
 * "rows_total", "nchild", "large_fronts", "small_fronts",
 * "nsys", "solve_work_rows", "amap_rows", "amap_entries". */
MDGPU_API int mdgpu_info(mdgpu_handle h, const char *key, long long *value);

/* Copy a symbolic array out: "perm" (n, new->old; identity if natural),
 * "parent", "post", "count0" (n; cs_etree / cs_post / cs_counts), "count"
 * (n; counts defining L, after GetRelaxedETree's padding), "relax_perm",
 * "sn_first", "sn_ncols" (nsuper), "child_ptr" (nsuper+1), "child",
 * "Lp" (n+1, as long long), "rows_ptr" (nsuper+1), "rows" (front row sets),
 * "relmap" (per front row: its position in the parent's front, -1 for pivot
 * rows and the root), "level" (nsuper).  Solve plan (diagnostics):
 * "warp_list" (small fronts per level by rows descending), "warp_cnt" (per
 * level the counts of more than 16, 9..16 and at most 8 rows), "amap_off"
 * (nsuper; -1 for small fronts), "amap_row", "amap_ent" (forward assembly
 * of the large fronts: front-vector rows summed into each front row, child
 * order; a front's vector starts at the sum of the rows of the supernodes
 * before it). */
MDGPU_API int mdgpu_get_array(mdgpu_handle h, const char *name, void *dst);

/*
 * Numeric factorization on the GPU.  Replaces Factor (mdgpu.cu:1394-1608)
 * with FactorAux_GPU_2 / FactorAux_CPU_3 (mdgpu.cu:903,1298) and ExtendAdd
 * (mdgpu.cu:802).  Ax: the values of the caller's lower triangle in the
 * caller's (original) ordering, host memory; _device: device memory.
 * stream: a cudaStream_t or NULL (the handle's own stream).  Returns
 * MDGPU_ERR_NOT_SPD if a pivot was not positive.
 */
MDGPU_API int mdgpu_factor(mdgpu_handle h, const double *Ax, int precision, void *stream);
MDGPU_API int mdgpu_factor_device(mdgpu_handle h, const double *dAx, int precision, void *stream);

/*
 * Autotuner (no counterpart in the reference): chooses the launch shapes of
 * the small-front factor kernels for this handle's fronts -- the tiny-front
 * kernel's grid cap and the threads per CTA of each small-front size bucket
 * (fronts of at most 64, 96, 128, 160 rows) -- by timing the whole factor of
 * Ax (host values) in the given precision with CUDA events (median of three
 * after one untimed run) over the candidates, one shape after another, the
 * fastest kept.  The choice stays with the handle; the factor's CUDA graphs
 * are captured again.  *ms_best (optional): the chosen shapes' factor time.
 * mdgpu_info keys "tuned", "tune_tiny_blocks", "tune_threads_b2" ..
 * "tune_threads_b5" report it.
 */
MDGPU_API int mdgpu_autotune(mdgpu_handle h, const double *Ax, int precision, double *ms_best);
MDGPU_API int mdgpu_not_spd_column(mdgpu_handle h); /* first failing column (permuted), -1 if none */

/*
 * x = A^-1 b with the last factor: the reference's cs_pvec + cs_lsolve +
 * cs_ltsolve + cs_ipvec sequence (mdgpu.cu:1952-1961, cs.cpp:1086-1146) as
 * supernodal GPU sweeps.  B, X: n x nrhs column-major (leading dims ldb,
 * ldx), original ordering; host memory, or device memory for _device.
 */
MDGPU_API int mdgpu_solve(mdgpu_handle h, const double *B, int ldb, double *X, int ldx, int nrhs,
                void *stream);
MDGPU_API int mdgpu_solve_device(mdgpu_handle h, const double *dB, int ldb, double *dX, int ldx, int nrhs,
                       void *stream);

/*
 * mdgpu_solve_device without any device allocation.  No counterpart in the
 * reference.  For callers that cannot allocate device memory when they solve
 * -- host frameworks whose own caching allocator owns the device memory (a
 * cudaMalloc behind its back can fail or fragment its pool), loops that
 * cannot afford cudaMalloc's implicit device synchronization -- the work
 * vectors come from a fixed 32 MiB
 * device array that every GPU loading this library holds until exit (the
 * handle's plan and factor were allocated earlier by mdgpu_analyze and
 * mdgpu_factor).  A call needs (n + w) x min(nrhs, 64) doubles, w =
 * mdgpu_info(h, "solve_work_rows") (front vector rows plus backward partial
 * sums), one more when n x min(nrhs, 64) is odd; larger requests return
 * MDGPU_ERR_INVALID.  All calls share the
 * array: calls whose work overlaps on one GPU race and must be serialized by
 * the caller.  The analysis (mdgpu_analyze and the other analyze entries)
 * looks up the array's address on the handle's device, which loads the
 * array's module and commits its memory then, so a solve does no module
 * load; should that look-up fail there, the first call on the device makes
 * it: make that first call before any stream capture.
 */
MDGPU_API int mdgpu_solve_device_noalloc(mdgpu_handle h, const double *dB, int ldb, double *dX,
                                         int ldx, int nrhs, void *stream);

/*
 * Solve with FP64 iterative refinement on the GPU: r = b - A x with the
 * caller's FP64 values (the reference's residual, mdgpu.cu:1963-1972), then
 * x += A_factor^-1 r until the backward error ||r||inf / (||A||inf ||x||inf +
 * ||b||inf) <= tol or maxit corrections.  berr[nrhs] (optional) receives the
 * final backward errors, *iters (optional) the number of corrections.
 */
MDGPU_API int mdgpu_refine(mdgpu_handle h, const double *B, int ldb, double *X, int ldx, int nrhs,
                 double tol, int maxit, double *berr, int *iters, void *stream);
MDGPU_API int mdgpu_refine_device(mdgpu_handle h, const double *dB, int ldb, double *dX, int ldx, int nrhs,
                        double tol, int maxit, double *berr, int *iters, void *stream);

/*
 * Solve with GMRES-based iterative refinement (GMRES-IR; no counterpart in the
 * reference): x = M^-1 b, then while the backward error (as for
 * mdgpu_refine) is above tol and fewer than maxit corrections were made,
 * r = b - A x with the caller's FP64 values and the correction d solves
 * M^-1 A d = M^-1 r by GMRES in FP64 from d = 0 (at most `restart` steps,
 * 1..64; stop when the preconditioned residual is inner_tol times its start),
 * x += d.  M^-1 is the solve with the current factor (FP32 or FP64).  Plain
 * refinement needs cond(A) u_factor < 1; GMRES-IR converges for cond(A) up to
 * about u_factor^-2.  Right-hand sides are refined one after another.
 * berr[nrhs], iters[nrhs] (corrections) and inner[nrhs] (GMRES steps, one
 * factor solve and one product with A each) are optional outputs.  Device
 * memory: (restart + 2) n doubles, kept with the handle.
 */
MDGPU_API int mdgpu_gmres_ir(mdgpu_handle h, const double *B, int ldb, double *X, int ldx, int nrhs,
                             double tol, int maxit, int restart, double inner_tol, double *berr,
                             int *iters, int *inner, void *stream);
MDGPU_API int mdgpu_gmres_ir_device(mdgpu_handle h, const double *dB, int ldb, double *dX, int ldx,
                                    int nrhs, double tol, int maxit, int restart, double inner_tol,
                                    double *berr, int *iters, int *inner, void *stream);

/*
 * Differentiation (no counterpart in the reference, whose driver only
 * factors and solves).  mdgpu_logdet: log det A = 2 sum log L(j, j) of the
 * current factor (FP64 or FP32).  mdgpu_selinv: the selected inverse
 * Z = A^-1 on the pattern of L of the current FP64 factor (Takahashi's
 * recurrence over the fronts from the root down; it reuses the factor's
 * update-matrix storage, so call it after the factor and before the next
 * one).  mdgpu_grad_lower: the gradient of loss = log det A + b' A^-1 b with
 * respect to the caller's lower-triangle values Ax, given x = A^-1 b in the
 * caller's ordering (x = NULL: the gradient of log det A alone): an
 * off-diagonal entry, which stands for A(i,j) and A(j,i), gets
 * 2 (Z(i,j) - x_i x_j), a diagonal entry Z(i,i) - x_i^2; dropped duplicates
 * get 0.  G has nnz (Ap[n]) entries; the gradient with respect to b is 2 x.
 * _device: x and G in device memory.
 */
MDGPU_API int mdgpu_logdet(mdgpu_handle h, double *logdet, void *stream);
MDGPU_API int mdgpu_selinv(mdgpu_handle h, void *stream);
MDGPU_API int mdgpu_grad_lower(mdgpu_handle h, const double *x, double *G, void *stream);
MDGPU_API int mdgpu_grad_lower_device(mdgpu_handle h, const double *dx, double *dG, void *stream);

/*
 * General reverse mode of the factorization (no counterpart in the
 * reference; the forward structure it reverses is Factor, mdgpu.cu:1394-1608):
 * given Lbar, the gradient of a loss with respect to the values of L (lnz
 * entries in the CSC order of mdgpu_get_L / the reference's spL), writes
 * Abar, the gradient with respect to the caller's lower-triangle values
 * (nnz entries, caller order; an off-diagonal value stands for A(i,j) and
 * A(j,i); a repeated entry the assembly drops gets 0).  Needs a current FP64
 * factor.  Front by front from the root: the adjoints of the Schur update,
 * the triangular solve and the diagonal-block Cholesky, and the transpose of
 * the extend-add; only L is read (no update matrix is stored or recomputed).
 * _device: device pointers, asynchronous on the stream.
 */
MDGPU_API int mdgpu_adjoint(mdgpu_handle h, const double *Lbar, double *Abar, void *stream);
MDGPU_API int mdgpu_adjoint_device(mdgpu_handle h, const double *dLbar, double *dAbar,
                                   void *stream);

/*
 * Copy L out as compressed columns, the spL contract of the reference
 * (mdgpu.cu:1346-1352, 1859-1875): Lp[n+1] (long long), Li[lnz] row indices
 * ascending with the diagonal first, Lx[lnz] values (FP64; an FP32 factor is
 * widened).  Any of the three may be NULL.
 */
MDGPU_API int mdgpu_get_L(mdgpu_handle h, long long *Lp, int *Li, double *Lx);

/*
 * Diagnostics (no counterpart in the reference, whose only instrumentation is
 * its tic/toc phase timers, mdgpu.cu:31-57,1901-1930).  mdgpu_profile(h, 1)
 * brackets every kernel launch of the numeric phase with CUDA events, grouped
 * by kernel class; mdgpu_profile(h, 0) (or a second enable) stops recording
 * and folds the recorded events into per-class totals read back with
 * mdgpu_profile_read: device milliseconds, launches, and the algorithmic flops
 * / bytes of those launches.  Classes: 0 small-front factor, 1 large-front
 * assembly, 2 first diagonal tile, 3 panel TRSM, 4 Schur tile update, 5 small-
 * front solve sweeps, 6 large-front solve steps, 7 other.
 */
MDGPU_API int mdgpu_profile(mdgpu_handle h, int enable);
MDGPU_API int mdgpu_profile_read(mdgpu_handle h, int cls, double *ms, long long *launches,
                                 double *flops, double *bytes);

MDGPU_API const char *mdgpu_status_string(int status);
MDGPU_API const char *mdgpu_last_error(void);

#ifdef __cplusplus
}
#endif
#endif
