// Residual and norm kernels used by iterative refinement.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace mdgpu {

// Full symmetric pattern of the caller's matrix, rows in original numbering;
// src[p] indexes the caller's lower-triangle value array.
struct SymCsr {
    int n = 0;
    int64_t nnz = 0;
    int* rowptr = nullptr;
    int* col = nullptr;
    int* src = nullptr;
};

void launch_residual(const SymCsr& A, const double* Ax, const double* x, int ldx,
                     const double* b, int ldb, double* r, int ldr, int nrhs, cudaStream_t st);
void launch_anorm(const SymCsr& A, const double* Ax, unsigned long long* out, cudaStream_t st);
void launch_absmax3(int n, int nrhs, const double* r, int ldr, const double* x, int ldx,
                    const double* b, int ldb, unsigned long long* out, cudaStream_t st);
void launch_axpy(int n, int nrhs, const double* d, double* x, int ldx, cudaStream_t st);

// GMRES-IR vector operations: w = A v; out[i] = <V(:, i), w> for i < k
// (deterministic two-stage sums; partial holds dots_partial_size(k) values);
// w += sign * V(:, 0:k) coef; w *= alpha.  k <= 64.
void launch_spmv(const SymCsr& A, const double* Ax, const double* v, double* w, cudaStream_t st);
int dots_partial_size(int kmax);
void launch_dots(int n, int k, const double* V, int64_t ldv, const double* w, double* partial,
                 double* out, cudaStream_t st);
void launch_gemv_acc(int n, int k, const double* V, int64_t ldv, const double* coef, double sign,
                     double* w, cudaStream_t st);
void launch_scale(int n, double alpha, double* w, cudaStream_t st);

}  // namespace mdgpu
