// FP64 residual, norms and updates for iterative refinement.
//
// The residual r = b - A x uses the caller's ORIGINAL matrix (lower triangle,
// CSC) through a full symmetric CSR pattern built once on the host whose
// entries point back into the caller's value array, so no permuted copy of
// the values is ever made.  One warp per row, deterministic.
#include <cstdint>

#include "ir.hpp"

namespace mdgpu {

__global__ void k_residual(int n, int nrhs, const int* __restrict__ rowptr,
                           const int* __restrict__ col, const int* __restrict__ src,
                           const double* __restrict__ Ax, const double* __restrict__ x, int ldx,
                           const double* __restrict__ b, int ldb, double* __restrict__ r, int ldr) {
    const int lane = threadIdx.x & 31;
    const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t row = warp; row < (int64_t)n * nrhs; row += nwarps) {
        int q = (int)(row / n), i = (int)(row - (int64_t)q * n);
        const double* xq = x + (int64_t)q * ldx;
        double acc = 0;
        for (int p = rowptr[i] + lane; p < rowptr[i + 1]; p += 32) acc += Ax[src[p]] * xq[col[p]];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
        if (lane == 0) r[i + (int64_t)q * ldr] = b[i + (int64_t)q * ldb] - acc;
    }
}

// max |A| row sum (= the 1-norm, A symmetric)
__global__ void k_row_abs_sum_max(int n, const int* __restrict__ rowptr,
                                  const int* __restrict__ src, const double* __restrict__ Ax,
                                  unsigned long long* __restrict__ out) {
    const int lane = threadIdx.x & 31;
    const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    double best = 0;
    for (int64_t i = warp; i < n; i += nwarps) {
        double acc = 0;
        for (int p = rowptr[i] + lane; p < rowptr[i + 1]; p += 32) acc += fabs(Ax[src[p]]);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
        best = fmax(best, acc);
    }
    if (lane == 0) atomicMax(out, (unsigned long long)__double_as_longlong(best));
}

// per right-hand side q: out[3q+0] = max|r|, out[3q+1] = max|x|, out[3q+2] = max|b|
__global__ void k_absmax3(int n, int nrhs, const double* __restrict__ r, int ldr,
                          const double* __restrict__ x, int ldx, const double* __restrict__ b,
                          int ldb, unsigned long long* __restrict__ out) {
    for (int q = 0; q < nrhs; ++q) {
        double m0 = 0, m1 = 0, m2 = 0;
        for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
             i += (int64_t)gridDim.x * blockDim.x) {
            m0 = fmax(m0, fabs(r[i + (int64_t)q * ldr]));
            m1 = fmax(m1, fabs(x[i + (int64_t)q * ldx]));
            m2 = fmax(m2, fabs(b[i + (int64_t)q * ldb]));
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            m0 = fmax(m0, __shfl_xor_sync(0xffffffffu, m0, o));
            m1 = fmax(m1, __shfl_xor_sync(0xffffffffu, m1, o));
            m2 = fmax(m2, __shfl_xor_sync(0xffffffffu, m2, o));
        }
        if ((threadIdx.x & 31) == 0) {
            atomicMax(out + 3 * q + 0, (unsigned long long)__double_as_longlong(m0));
            atomicMax(out + 3 * q + 1, (unsigned long long)__double_as_longlong(m1));
            atomicMax(out + 3 * q + 2, (unsigned long long)__double_as_longlong(m2));
        }
    }
}

__global__ void k_axpy(int64_t len, const double* __restrict__ d, double* __restrict__ x) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < len;
         i += (int64_t)gridDim.x * blockDim.x)
        x[i] += d[i];
}

// ---- GMRES-IR vector operations (one right-hand side) ----

// w = A v with the caller's FP64 values, one warp per row (the residual's
// access pattern without b)
__global__ void k_spmv(int n, const int* __restrict__ rowptr, const int* __restrict__ col,
                       const int* __restrict__ src, const double* __restrict__ Ax,
                       const double* __restrict__ v, double* __restrict__ w) {
    const int lane = threadIdx.x & 31;
    const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t i = warp; i < n; i += nwarps) {
        double acc = 0;
        for (int p = rowptr[i] + lane; p < rowptr[i + 1]; p += 32) acc += Ax[src[p]] * v[col[p]];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
        if (lane == 0) w[i] = acc;
    }
}

constexpr int kDotBlocks = 148 * 2;  // partial sums per dot product
constexpr int kDotThreads = 256;

// column i = blockIdx.y of V (leading dimension ldv) against w: this block's
// rows summed in a fixed order into partial[i * gridDim.x + blockIdx.x]
__global__ void __launch_bounds__(kDotThreads)
    k_dots_partial(int n, const double* __restrict__ V, int64_t ldv, const double* __restrict__ w,
                   double* __restrict__ partial) {
    __shared__ double red[kDotThreads / 32];
    const double* v = V + (int64_t)blockIdx.y * ldv;
    double acc = 0;
    for (int64_t r = blockIdx.x * (int64_t)kDotThreads + threadIdx.x; r < n;
         r += (int64_t)gridDim.x * kDotThreads)
        acc += v[r] * w[r];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0;
        for (int q = 0; q < kDotThreads / 32; ++q) s += red[q];
        partial[(int64_t)blockIdx.y * gridDim.x + blockIdx.x] = s;
    }
}

// out[i] = the nb partial sums of column i = blockIdx.x, one warp, fixed order
__global__ void k_dots_final(int nb, const double* __restrict__ partial, double* __restrict__ out) {
    const double* p = partial + (int64_t)blockIdx.x * nb;
    double s = 0;
    for (int b = threadIdx.x; b < nb; b += 32) s += p[b];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (threadIdx.x == 0) out[blockIdx.x] = s;
}

// w += sign * sum_{i < k} coef[i] V(:, i)
__global__ void k_gemv_acc(int n, int k, const double* __restrict__ V, int64_t ldv,
                           const double* __restrict__ coef, double sign, double* __restrict__ w) {
    for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < n;
         r += (int64_t)gridDim.x * blockDim.x) {
        double s = 0;
        for (int i = 0; i < k; ++i) s += coef[i] * V[r + i * ldv];
        w[r] += sign * s;
    }
}

__global__ void k_scale(int n, double alpha, double* __restrict__ w) {
    for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < n;
         r += (int64_t)gridDim.x * blockDim.x)
        w[r] *= alpha;
}

static int grid_for(int64_t work, int per_block) {
    int64_t g = (work + per_block - 1) / per_block;
    if (g > 148 * 32) g = 148 * 32;
    return (int)(g < 1 ? 1 : g);
}

void launch_residual(const SymCsr& A, const double* Ax, const double* x, int ldx,
                     const double* b, int ldb, double* r, int ldr, int nrhs, cudaStream_t st) {
    k_residual<<<grid_for((int64_t)A.n * nrhs * 32, 256), 256, 0, st>>>(
        A.n, nrhs, A.rowptr, A.col, A.src, Ax, x, ldx, b, ldb, r, ldr);
}

void launch_anorm(const SymCsr& A, const double* Ax, unsigned long long* out, cudaStream_t st) {
    cudaMemsetAsync(out, 0, sizeof(unsigned long long), st);
    k_row_abs_sum_max<<<grid_for((int64_t)A.n * 32, 256), 256, 0, st>>>(A.n, A.rowptr, A.src, Ax,
                                                                        out);
}

void launch_absmax3(int n, int nrhs, const double* r, int ldr, const double* x, int ldx,
                    const double* b, int ldb, unsigned long long* out, cudaStream_t st) {
    cudaMemsetAsync(out, 0, 3 * sizeof(unsigned long long) * nrhs, st);
    k_absmax3<<<grid_for(n, 256), 256, 0, st>>>(n, nrhs, r, ldr, x, ldx, b, ldb, out);
}

void launch_axpy(int64_t len, const double* d, double* x, cudaStream_t st) {
    k_axpy<<<grid_for(len, 256), 256, 0, st>>>(len, d, x);
}

void launch_spmv(const SymCsr& A, const double* Ax, const double* v, double* w, cudaStream_t st) {
    k_spmv<<<grid_for((int64_t)A.n * 32, 256), 256, 0, st>>>(A.n, A.rowptr, A.col, A.src, Ax, v,
                                                            w);
}

int dots_partial_size(int kmax) { return kmax * kDotBlocks; }

void launch_dots(int n, int k, const double* V, int64_t ldv, const double* w, double* partial,
                 double* out, cudaStream_t st) {
    k_dots_partial<<<dim3(kDotBlocks, k), kDotThreads, 0, st>>>(n, V, ldv, w, partial);
    k_dots_final<<<k, 32, 0, st>>>(kDotBlocks, partial, out);
}

void launch_gemv_acc(int n, int k, const double* V, int64_t ldv, const double* coef, double sign,
                     double* w, cudaStream_t st) {
    k_gemv_acc<<<grid_for(n, 256), 256, 0, st>>>(n, k, V, ldv, coef, sign, w);
}

void launch_scale(int n, double alpha, double* w, cudaStream_t st) {
    k_scale<<<grid_for(n, 256), 256, 0, st>>>(n, alpha, w);
}

}  // namespace mdgpu
