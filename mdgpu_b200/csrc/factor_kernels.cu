// Numeric factorization kernels (scalar T = double or float).
//
// Small fronts (m <= 160): one CTA per front does everything in shared memory:
// zero the front, scatter A's values, extend-add every child's update matrix
// (children one after another, so the sum is deterministic), factor the c
// pivot columns, write the L panel and the Schur complement U = F22 - L21 L21'.
//
// Large fronts: a tiled right-looking partial Cholesky over the [L | U] split
// storage, batched over all large fronts of one tree level:
//   k_big_assemble   CTA per (front, 32-column block): zero, scatter A, pull the
//                    children's update columns that land in the block
//   k_tile_potrf     CTA per front: Cholesky of the first diagonal tile
//   k_tile_trsm      CTA per (front, row tile below the panel): X = A L^-T
//   k_tile_update    CTA per (front, lower tile right of the panel):
//                    C -= A B'; the CTA holding the next diagonal tile also
//                    factors it, so the next step's TRSM can start at once.
#include <cstdio>

#include "device_common.cuh"
#include "kernels.hpp"

namespace mdgpu {

// ---------------------------------------------------------------------------
// fused small-front kernel
// ---------------------------------------------------------------------------

template <typename T>
__global__ void k_small_front(const FrontDesc* __restrict__ fronts, const int* __restrict__ list,
                              const int* __restrict__ child, const int* __restrict__ relmap,
                              const int* __restrict__ a_src, const int* __restrict__ a_pos,
                              const double* __restrict__ Ax, T* __restrict__ Ls,
                              T* __restrict__ Us, int LD, int* __restrict__ status) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* F = reinterpret_cast<T*>(smem_raw);
    int* rel = reinterpret_cast<int*>(F + (size_t)LD * (LD - 1));
    const int s = list[blockIdx.x];
    const FrontDesc f = fronts[s];
    const int m = f.m, c = f.c, u = m - c;
    const int tid = threadIdx.x, nt = blockDim.x;

    for (int idx = tid; idx < m * LD; idx += nt) F[idx] = T(0);
    __syncthreads();
    for (int e = f.a_beg + tid; e < f.a_end; e += nt) {
        int src = a_src[e];
        if (src >= 0) {
            int pos = a_pos[e];
            F[(pos & 0xffff) + (pos >> 16) * LD] = (T)Ax[src];
        }
    }
    __syncthreads();
    for (int h = f.child_beg; h < f.child_end; ++h) {
        const FrontDesc g = fronts[child[h]];
        const int uc = g.m - g.c;
        if (uc <= 0) continue;
        for (int i = tid; i < uc; i += nt) rel[i] = relmap[g.rows_off + g.c + i];
        __syncthreads();
        const T* U = Us + g.uoff;
        for (int idx = tid; idx < uc * uc; idx += nt) {
            int j = idx / uc, i = idx - j * uc;
            if (i >= j) F[rel[i] + rel[j] * LD] += U[i + (int64_t)j * g.ldu];
        }
        __syncthreads();
    }
    // partial Cholesky of the c pivot columns (right-looking, panel only)
    for (int k = 0; k < c; ++k) {
        const T dkk = F[k + k * LD];
        const T d = sqrt(dkk);
        if (tid == 0 && !(dkk > T(0))) flag_pivot(status, f.first_col + k);
        const T inv = T(1) / d;
        for (int i = k + 1 + tid; i < m; i += nt) F[i + k * LD] *= inv;
        __syncthreads();
        if (tid == 0) F[k + k * LD] = d;
        const int rows = m - k - 1, w = c - k - 1;
        for (int idx = tid; idx < rows * w; idx += nt) {
            int jj = idx / rows, ii = idx - jj * rows;
            int i = k + 1 + ii, j = k + 1 + jj;
            if (i >= j) F[i + j * LD] -= F[i + k * LD] * F[j + k * LD];
        }
        __syncthreads();
    }
    // Schur complement straight to the update store
    if (f.uoff >= 0) {
        T* Ud = Us + f.uoff;
        for (int idx = tid; idx < u * u; idx += nt) {
            int j = idx / u, i = idx - j * u;
            if (i >= j) {
                T acc = F[(c + i) + (c + j) * LD];
                const T* a = F + c + i;
                const T* b = F + c + j;
#pragma unroll 4
                for (int k = 0; k < c; ++k) acc -= a[k * LD] * b[k * LD];
                Ud[i + (int64_t)j * f.ldu] = acc;
            }
        }
    }
    T* Ld = Ls + f.loff;
    for (int idx = tid; idx < m * c; idx += nt) {
        int j = idx / m, i = idx - j * m;
        Ld[i + (int64_t)j * f.ldl] = (i >= j) ? F[i + j * LD] : T(0);
    }
}

// ---------------------------------------------------------------------------
// large fronts: assembly
// ---------------------------------------------------------------------------

template <typename T>
__global__ void __launch_bounds__(256)
    k_big_assemble(const FrontDesc* __restrict__ fronts, const int* __restrict__ items,
                   const int* __restrict__ before, int nitems, int CB,
                   const int* __restrict__ child, const int* __restrict__ relmap,
                   const int* __restrict__ a_src, const int* __restrict__ a_pos,
                   const int* __restrict__ a_colptr, const int* __restrict__ a_colptr_off,
                   const double* __restrict__ Ax, T* __restrict__ Ls, T* __restrict__ Us) {
    __shared__ int range[2];
    const int it = find_item(before, nitems, blockIdx.x);
    const int s = items[it];
    const int blk = blockIdx.x - before[it];
    const FrontDesc f = fronts[s];
    const int j0 = blk * CB, j1 = min(j0 + CB, f.m);
    const int tid = threadIdx.x, nt = blockDim.x;

    for (int jj = j0; jj < j1; ++jj) {
        if (jj < f.c) {
            T* col = Ls + f.loff + (int64_t)jj * f.ldl;
            for (int r = tid; r < f.m; r += nt) col[r] = T(0);
        } else {
            T* col = Us + f.uoff + (int64_t)(jj - f.c) * f.ldu;
            for (int r = jj - f.c + tid; r < f.m - f.c; r += nt) col[r] = T(0);
        }
    }
    __syncthreads();
    if (j0 < f.c) {
        const int* cp = a_colptr + a_colptr_off[s];
        int e0 = f.a_beg + cp[j0], e1 = f.a_beg + cp[min(j1, f.c)];
        for (int e = e0 + tid; e < e1; e += nt) {
            int src = a_src[e];
            if (src >= 0) {
                int pos = a_pos[e];
                Ls[f.loff + (pos & 0xffff) + (int64_t)(pos >> 16) * f.ldl] = (T)Ax[src];
            }
        }
    }
    __syncthreads();
    for (int h = f.child_beg; h < f.child_end; ++h) {
        const FrontDesc g = fronts[child[h]];
        const int uc = g.m - g.c;
        const int* rm = relmap + g.rows_off + g.c;
        if (tid == 0) {
            int lo = 0, hi = uc;  // first update column mapping to >= j0
            while (lo < hi) {
                int mid = (lo + hi) >> 1;
                if (rm[mid] < j0) lo = mid + 1; else hi = mid;
            }
            int a = lo;
            hi = uc;
            while (lo < hi) {
                int mid = (lo + hi) >> 1;
                if (rm[mid] < j1) lo = mid + 1; else hi = mid;
            }
            range[0] = a;
            range[1] = lo;
        }
        __syncthreads();
        const int jlo = range[0], jhi = range[1];
        const T* U = Us + g.uoff;
        for (int jc = jlo; jc < jhi; ++jc) {
            const int pc = rm[jc];
            for (int ic = jc + tid; ic < uc; ic += nt) {
                T v = U[ic + (int64_t)jc * g.ldu];
                *front_elem(Ls, Us, f, rm[ic], pc) += v;
            }
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// large fronts: tiles
// ---------------------------------------------------------------------------

// In-place Cholesky of an n x n lower tile held in shared memory (ld = LDS).
template <typename T>
__device__ void tile_potrf_smem(T* S, int LDS, int n, int* status, int col0) {
    const int tid = threadIdx.x, nt = blockDim.x;
    for (int k = 0; k < n; ++k) {
        const T dkk = S[k + k * LDS];
        const T d = sqrt(dkk);
        if (tid == 0 && !(dkk > T(0))) flag_pivot(status, col0 + k);
        const T inv = T(1) / d;
        for (int i = k + 1 + tid; i < n; i += nt) S[i + k * LDS] *= inv;
        __syncthreads();
        if (tid == 0) S[k + k * LDS] = d;
        const int r = n - k - 1;
        for (int idx = tid; idx < r * r; idx += nt) {
            int jj = idx / r, ii = idx - jj * r;
            if (ii >= jj) S[(k + 1 + ii) + (k + 1 + jj) * LDS] -= S[(k + 1 + ii) + k * LDS] * S[(k + 1 + jj) + k * LDS];
        }
        __syncthreads();
    }
}

template <typename T, int TB>
__device__ void potrf_diag_tile(const FrontDesc& f, int k, T* Ls, T* S, int* status) {
    const int tid = threadIdx.x, nt = blockDim.x;
    const TileRange tk = tile_range(k, f.m, f.c, TB);
    const int n = tk.size;
    T* base = Ls + f.loff + tk.start + (int64_t)tk.start * f.ldl;
    for (int idx = tid; idx < n * n; idx += nt) {
        int j = idx / n, i = idx - j * n;
        S[i + j * (TB + 1)] = (i >= j) ? base[i + (int64_t)j * f.ldl] : T(0);
    }
    __syncthreads();
    tile_potrf_smem(S, TB + 1, n, status, f.first_col + tk.start);
    for (int idx = tid; idx < n * n; idx += nt) {
        int j = idx / n, i = idx - j * n;
        if (i >= j) base[i + (int64_t)j * f.ldl] = S[i + j * (TB + 1)];
    }
}

template <typename T, int TB>
__global__ void __launch_bounds__(256)
    k_tile_potrf(const FrontDesc* __restrict__ fronts, const int* __restrict__ list, int k,
                 T* __restrict__ Ls, int* __restrict__ status) {
    __shared__ T S[TB * (TB + 1)];
    const FrontDesc f = fronts[list[blockIdx.x]];
    if (k >= tiles_l(f.c, TB)) return;
    potrf_diag_tile<T, TB>(f, k, Ls, S, status);
}

template <typename T, int TB>
__global__ void __launch_bounds__(TB)
    k_tile_trsm(const FrontDesc* __restrict__ fronts, const int* __restrict__ items,
                const int* __restrict__ before, int nitems, int k, T* __restrict__ Ls) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* Lkk = reinterpret_cast<T*>(smem_raw);  // TB x (TB + 1)
    T* X = Lkk + TB * (TB + 1);               // TB x (TB + 1), row-major rows
    T* dinv = X + TB * (TB + 1);              // TB
    const int it = find_item(before, nitems, blockIdx.x);
    const FrontDesc f = fronts[items[it]];
    const int i = k + 1 + (blockIdx.x - before[it]);
    const TileRange tk = tile_range(k, f.m, f.c, TB);
    const TileRange ti = tile_range(i, f.m, f.c, TB);
    const int tid = threadIdx.x, nt = blockDim.x;
    const int nk = tk.size, ni = ti.size;
    const T* lkk = Ls + f.loff + tk.start + (int64_t)tk.start * f.ldl;
    T* aik = Ls + f.loff + ti.start + (int64_t)tk.start * f.ldl;
    for (int idx = tid; idx < nk * nk; idx += nt) {
        int j = idx / nk, r = idx - j * nk;
        Lkk[r + j * (TB + 1)] = lkk[r + (int64_t)j * f.ldl];
    }
    for (int idx = tid; idx < ni * nk; idx += nt) {
        int j = idx / ni, r = idx - j * ni;
        X[r * (TB + 1) + j] = aik[r + (int64_t)j * f.ldl];  // row-major: row r contiguous
    }
    __syncthreads();
    for (int j = tid; j < nk; j += nt) dinv[j] = T(1) / Lkk[j + j * (TB + 1)];
    __syncthreads();
    // X L' = A, one row per thread: x_j = (a_j - sum_{l<j} x_l L_jl) / L_jj
    for (int r = tid; r < ni; r += nt) {
        T* x = X + r * (TB + 1);
        for (int j = 0; j < nk; ++j) {
            T acc = x[j];
            for (int l = 0; l < j; ++l) acc -= x[l] * Lkk[j + l * (TB + 1)];
            x[j] = acc * dinv[j];
        }
    }
    __syncthreads();
    for (int idx = tid; idx < ni * nk; idx += nt) {
        int j = idx / ni, r = idx - j * ni;
        aik[r + (int64_t)j * f.ldl] = X[r * (TB + 1) + j];
    }
}

template <typename T, int TB>
__global__ void __launch_bounds__(256)
    k_tile_update(const FrontDesc* __restrict__ fronts, const int* __restrict__ items,
                  const int* __restrict__ before, int nitems, int k, T* __restrict__ Ls,
                  T* __restrict__ Us, int* __restrict__ status) {
    static_assert(TB == 64, "4x4 register tile over 256 threads assumes TB = 64");
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* As = reinterpret_cast<T*>(smem_raw);  // [K][TB]
    T* Bs = As + TB * TB;                    // [K][TB]
    const int it = find_item(before, nitems, blockIdx.x);
    const FrontDesc f = fronts[items[it]];
    int ii, jj;
    lower_index(blockIdx.x - before[it], ii, jj);
    const int i = k + 1 + ii, j = k + 1 + jj;
    const TileRange tk = tile_range(k, f.m, f.c, TB);
    const TileRange ti = tile_range(i, f.m, f.c, TB);
    const TileRange tj = tile_range(j, f.m, f.c, TB);
    const int tid = threadIdx.x;
    const int K = tk.size;
    const T* pa = Ls + f.loff + ti.start + (int64_t)tk.start * f.ldl;
    const T* pb = Ls + f.loff + tj.start + (int64_t)tk.start * f.ldl;
    for (int idx = tid; idx < TB * K; idx += 256) {
        int q = idx / TB, r = idx - q * TB;
        As[q * TB + r] = r < ti.size ? pa[r + (int64_t)q * f.ldl] : T(0);
        Bs[q * TB + r] = r < tj.size ? pb[r + (int64_t)q * f.ldl] : T(0);
    }
    __syncthreads();
    const int r0 = (tid & 15) * 4, c0 = (tid >> 4) * 4;
    T acc[4][4];
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) acc[a][b] = T(0);
    for (int q = 0; q < K; ++q) {
        T av[4], bv[4];
#pragma unroll
        for (int a = 0; a < 4; ++a) av[a] = As[q * TB + r0 + a];
#pragma unroll
        for (int b = 0; b < 4; ++b) bv[b] = Bs[q * TB + c0 + b];
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
            for (int b = 0; b < 4; ++b) acc[a][b] += av[a] * bv[b];
    }
#pragma unroll
    for (int b = 0; b < 4; ++b) {
        int cc = c0 + b;
        if (cc >= tj.size) continue;
        int gc = tj.start + cc;
#pragma unroll
        for (int a = 0; a < 4; ++a) {
            int rr = r0 + a;
            if (rr >= ti.size) continue;
            int gr = ti.start + rr;
            if (gr < gc) continue;
            *front_elem(Ls, Us, f, gr, gc) -= acc[a][b];
        }
    }
    // the next diagonal tile is final now: factor it for the next step
    if (i == k + 1 && j == k + 1 && i < tiles_l(f.c, TB)) {
        __syncthreads();
        potrf_diag_tile<T, TB>(f, i, Ls, As, status);
    }
}

// ---------------------------------------------------------------------------
// host launchers
// ---------------------------------------------------------------------------

template <typename T>
static size_t trsm_smem() {
    return (size_t)(2 * 64 * 65 + 64) * sizeof(T);
}

template <typename T>
void launch_small_fronts(const DevPlan& D, int level, const T* /*tag*/, T* Ls, T* Us,
                         const double* Ax, int* status, cudaStream_t st) {
    for (int b = 0; b < kSmallBuckets; ++b) {
        int beg = D.h_small_ptr[level * kSmallBuckets + b];
        int end = D.h_small_ptr[level * kSmallBuckets + b + 1];
        if (end == beg) continue;
        int MB = Plan::small_limit[b];
        int LD = MB + 1;
        size_t smem = (size_t)MB * LD * sizeof(T) + (size_t)MB * sizeof(int);
        int threads = MB <= 16 ? 64 : (MB <= 32 ? 128 : 256);
        k_small_front<T><<<end - beg, threads, smem, st>>>(D.fronts, D.small_list + beg, D.child,
                                                          D.relmap, D.a_src, D.a_pos, Ax, Ls, Us,
                                                          LD, status);
    }
}

template <typename T>
void launch_large_level(const DevPlan& D, int level, T* Ls, T* Us, const double* Ax, int* status,
                        cudaStream_t st) {
    const int lb = D.h_large_ptr[level], le = D.h_large_ptr[level + 1];
    if (le == lb) return;
    const DevSchedule& S = D.sched64;
    const WorkList& asl = D.h_assemble[level];
    k_big_assemble<T><<<asl.nctas, 256, 0, st>>>(D.fronts, S.items + asl.off, S.before + asl.off,
                                                 asl.nitems, kAssembleCols, D.child, D.relmap,
                                                 D.a_src, D.a_pos, D.a_colptr, D.a_colptr_off, Ax,
                                                 Ls, Us);
    k_tile_potrf<T, 64><<<le - lb, 256, 0, st>>>(D.fronts, D.large_list + lb, 0, Ls, status);
    for (int q = S.h_level_beg[level]; q < S.h_level_beg[level + 1]; ++q) {
        const WorkList& tr = S.h_trsm[q];
        const WorkList& up = S.h_update[q];
        if (tr.nctas > 0)
            k_tile_trsm<T, 64><<<tr.nctas, 64, trsm_smem<T>(), st>>>(D.fronts, S.items + tr.off,
                                                        S.before + tr.off, tr.nitems, tr.step, Ls);
        if (up.nctas > 0)
            k_tile_update<T, 64><<<up.nctas, 256, 2 * 64 * 64 * sizeof(T), st>>>(
                D.fronts, S.items + up.off, S.before + up.off, up.nitems, up.step, Ls, Us, status);
    }
}

template <typename T>
void factor_levels(const DevPlan& D, T* Ls, T* Us, const double* Ax, int* status,
                   cudaStream_t st) {
    static bool attr_done = false;
    if (!attr_done) {
        cudaFuncSetAttribute(k_small_front<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             227 * 1024);
        cudaFuncSetAttribute(k_tile_update<T, 64>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             2 * 64 * 64 * sizeof(T));
        cudaFuncSetAttribute(k_tile_trsm<T, 64>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             trsm_smem<T>());
        attr_done = true;
    }
    for (int l = 0; l < D.nlevels; ++l) {
        launch_small_fronts<T>(D, l, nullptr, Ls, Us, Ax, status, st);
        launch_large_level<T>(D, l, Ls, Us, Ax, status, st);
    }
}

template void factor_levels<double>(const DevPlan&, double*, double*, const double*, int*,
                                    cudaStream_t);
template void factor_levels<float>(const DevPlan&, float*, float*, const double*, int*,
                                   cudaStream_t);

}  // namespace mdgpu
