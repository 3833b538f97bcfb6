// FP64 residual, norms and updates for iterative refinement.
//
// The residual r = b - A x uses the caller's ORIGINAL matrix (lower triangle,
// CSC) through a full symmetric CSR pattern built once on the host whose
// entries point back into the caller's value array, so no permuted copy of
// the values is ever made.  One thread per (row, right-hand side), the row's
// entries summed in their CSR order: the rows of the 3D grids have about
// seven entries, too few to spread over a warp, and consecutive threads take
// consecutive rows of one right-hand side, so their index and value loads
// fall together.  Deterministic.
#include <algorithm>
#include <cstdint>

#include "ir.hpp"

namespace mdgpu {

__global__ void k_residual(int n, int nrhs, const int* __restrict__ rowptr,
                           const int* __restrict__ col, const int* __restrict__ src,
                           const double* __restrict__ Ax, const double* __restrict__ x, int ldx,
                           const double* __restrict__ b, int ldb, double* __restrict__ r, int ldr) {
    const int64_t total = (int64_t)n * nrhs;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;
         t += (int64_t)gridDim.x * blockDim.x) {
        const int q = (int)(t / n), i = (int)(t - (int64_t)q * n);
        const double* xq = x + (int64_t)q * ldx;
        double acc = 0;
        for (int p = rowptr[i], pe = rowptr[i + 1]; p < pe; ++p) acc += Ax[src[p]] * xq[col[p]];
        r[i + (int64_t)q * ldr] = b[i + (int64_t)q * ldb] - acc;
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

// per right-hand side q = blockIdx.y: out[3q+0] = max|r|, out[3q+1] =
// max|x|, out[3q+2] = max|b|; each block reduces its rows in shared memory
// and adds three atomics
__global__ void __launch_bounds__(256) k_absmax3(int n, const double* __restrict__ r, int ldr,
                                                 const double* __restrict__ x, int ldx,
                                                 const double* __restrict__ b, int ldb,
                                                 unsigned long long* __restrict__ out) {
    __shared__ double red[3][8];
    const int q = blockIdx.y;
    const double* rq = r + (int64_t)q * ldr;
    const double* xq = x + (int64_t)q * ldx;
    const double* bq = b + (int64_t)q * ldb;
    double m0 = 0, m1 = 0, m2 = 0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        m0 = fmax(m0, fabs(rq[i]));
        m1 = fmax(m1, fabs(xq[i]));
        m2 = fmax(m2, fabs(bq[i]));
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        m0 = fmax(m0, __shfl_xor_sync(0xffffffffu, m0, o));
        m1 = fmax(m1, __shfl_xor_sync(0xffffffffu, m1, o));
        m2 = fmax(m2, __shfl_xor_sync(0xffffffffu, m2, o));
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) red[0][warp] = m0, red[1][warp] = m1, red[2][warp] = m2;
    __syncthreads();
    if (threadIdx.x < 3) {
        double m = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) m = fmax(m, red[threadIdx.x][w]);
        atomicMax(out + 3 * q + threadIdx.x, (unsigned long long)__double_as_longlong(m));
    }
}

// x(:, q) += d(:, q) for every right-hand side q (d: n x nrhs, leading
// dimension n; x: leading dimension ldx)
__global__ void k_axpy(int n, int nrhs, const double* __restrict__ d, double* __restrict__ x,
                       int ldx) {
    const int64_t total = (int64_t)n * nrhs;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;
         t += (int64_t)gridDim.x * blockDim.x) {
        const int q = (int)(t / n), i = (int)(t - (int64_t)q * n);
        x[i + (int64_t)q * ldx] += d[t];
    }
}

// ---- GMRES-IR vector operations (one right-hand side) ----

// w = A v with the caller's FP64 values, one thread per row (the
// residual's access pattern without b)
__global__ void k_spmv(int n, const int* __restrict__ rowptr, const int* __restrict__ col,
                       const int* __restrict__ src, const double* __restrict__ Ax,
                       const double* __restrict__ v, double* __restrict__ w) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        double acc = 0;
        for (int p = rowptr[i], pe = rowptr[i + 1]; p < pe; ++p) acc += Ax[src[p]] * v[col[p]];
        w[i] = acc;
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
    k_residual<<<grid_for((int64_t)A.n * nrhs, 256), 256, 0, st>>>(
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
    // about four blocks per SM over all right-hand sides, at most one per 256
    // rows; grid rows of at most 65535 right-hand sides
    const int gx = (int)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256,
                                                                (148 * 4 + nrhs - 1) / nrhs));
    for (int q0 = 0; q0 < nrhs; q0 += 65535) {
        const int nq = std::min(65535, nrhs - q0);
        k_absmax3<<<dim3(gx, nq), 256, 0, st>>>(n, r + (int64_t)q0 * ldr, ldr,
                                                x + (int64_t)q0 * ldx, ldx,
                                                b + (int64_t)q0 * ldb, ldb, out + 3 * (int64_t)q0);
    }
}

void launch_axpy(int n, int nrhs, const double* d, double* x, int ldx, cudaStream_t st) {
    k_axpy<<<grid_for((int64_t)n * nrhs, 256), 256, 0, st>>>(n, nrhs, d, x, ldx);
}

void launch_spmv(const SymCsr& A, const double* Ax, const double* v, double* w, cudaStream_t st) {
    k_spmv<<<grid_for(A.n, 256), 256, 0, st>>>(A.n, A.rowptr, A.col, A.src, Ax, v, w);
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
