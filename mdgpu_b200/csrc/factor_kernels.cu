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
//   k_tile_potrf     CTA per front: Cholesky of the first diagonal tile, and its
//                    inverse (kept: it turns every TRSM and every solve step
//                    with this tile into a small matrix product)
//   k_tile_trsm      CTA per (front, row tile below the panel): X = A inv(L)'
//   k_tile_update    CTA per (front, lower tile right of the panel):
//                    C -= A B'; the CTA holding the next diagonal tile also
//                    factors it, so the next step's TRSM can start at once.
#include <cstdio>

#include "device_common.cuh"
#include "kernels.hpp"
#include "tile_ops.cuh"

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

// Fronts of at most 32 rows: a group of W lanes per front (W = 32, 16, 8:
// one, two or four fronts per warp), the front in the group's own W x (W + 1)
// shared slice; the same steps and sums in the same order as k_small_front,
// with group syncs only.
constexpr int kTinyFrontRows = 32;

template <typename T, int W>
__device__ void tiny_front_group(int s, const FrontDesc* __restrict__ fronts,
                                 const int* __restrict__ child, const int* __restrict__ relmap,
                                 const int* __restrict__ a_src, const int* __restrict__ a_pos,
                                 const double* __restrict__ Ax, T* __restrict__ Ls,
                                 T* __restrict__ Us, int* __restrict__ status, T* Fm) {
    constexpr int LD = W + 1;
    const unsigned mask =
        W == 32 ? 0xffffffffu : (((1u << W) - 1u) << ((threadIdx.x & 31) & ~(W - 1)));
    const int gl = threadIdx.x & (W - 1);
    const FrontDesc f = fronts[s];
    const int m = f.m, c = f.c, u = m - c;
    for (int idx = gl; idx < m * LD; idx += W) Fm[idx] = T(0);
    __syncwarp(mask);
    for (int e = f.a_beg + gl; e < f.a_end; e += W) {
        const int src = a_src[e];
        if (src >= 0) {
            const int pos = a_pos[e];
            Fm[(pos & 0xffff) + (pos >> 16) * LD] = (T)Ax[src];
        }
    }
    __syncwarp(mask);
    for (int h = f.child_beg; h < f.child_end; ++h) {
        const FrontDesc g = fronts[child[h]];
        const int uc = g.m - g.c;
        if (uc <= 0) continue;
        const int* rm = relmap + g.rows_off + g.c;
        const T* U = Us + g.uoff;
        for (int idx = gl; idx < uc * uc; idx += W) {
            const int j = idx / uc, i = idx - j * uc;
            if (i >= j) Fm[rm[i] + rm[j] * LD] += U[i + (int64_t)j * g.ldu];
        }
        __syncwarp(mask);
    }
    // partial Cholesky of the c pivot columns (right-looking, panel only):
    // lane i of the group owns row i and touches only it; the multipliers of
    // the other rows arrive by shuffles
    for (int k = 0; k < c; ++k) {
        const T dkk = Fm[k + k * LD];
        if (gl == 0 && !(dkk > T(0))) flag_pivot(status, f.first_col + k);
        const T d = sqrt(dkk);
        const T inv = T(1) / d;
        const T lik = (gl > k && gl < m) ? Fm[gl + k * LD] * inv : T(0);
        if (gl == k) Fm[k + k * LD] = d;
        if (gl > k && gl < m) Fm[gl + k * LD] = lik;
        for (int j = k + 1; j < c; ++j) {
            const T ljk = __shfl_sync(mask, lik, j, W);
            if (gl >= j && gl < m) Fm[gl + j * LD] -= lik * ljk;
        }
        __syncwarp(mask);
    }
    // Schur complement straight to the update store
    if (f.uoff >= 0) {
        T* Ud = Us + f.uoff;
        for (int idx = gl; idx < u * u; idx += W) {
            const int j = idx / u, i = idx - j * u;
            if (i >= j) {
                T acc = Fm[(c + i) + (c + j) * LD];
                for (int k = 0; k < c; ++k) acc -= Fm[(c + i) + k * LD] * Fm[(c + j) + k * LD];
                Ud[i + (int64_t)j * f.ldu] = acc;
            }
        }
    }
    T* Ld = Ls + f.loff;
    for (int idx = gl; idx < m * c; idx += W) {
        const int j = idx / m, i = idx - j * m;
        Ld[i + (int64_t)j * f.ldl] = (i >= j) ? Fm[i + j * LD] : T(0);
    }
    __syncwarp(mask);  // the slice is reused by the group's next front
}

// One level's fronts of at most 32 rows as warp tasks over a rows-descending
// list: tasks [0, n32) one front each (17..32 rows), then two fronts of 9..16
// rows per task, then four of at most 8; persistent warps take tasks with
// the grid's warp count as stride.
template <typename T>
__global__ void __launch_bounds__(128)
    k_tiny_fronts(const FrontDesc* __restrict__ fronts, const int* __restrict__ list, int n32,
                  int n16, int n8, const int* __restrict__ child, const int* __restrict__ relmap,
                  const int* __restrict__ a_src, const int* __restrict__ a_pos,
                  const double* __restrict__ Ax, T* __restrict__ Ls, T* __restrict__ Us,
                  int* __restrict__ status) {
    constexpr int LD = kTinyFrontRows + 1;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, wpb = blockDim.x >> 5;
    T* slice = reinterpret_cast<T*>(smem_raw) + (size_t)warp * kTinyFrontRows * LD;
    const int t16 = (n16 + 1) / 2, t8 = (n8 + 3) / 4, ntask = n32 + t16 + t8;
    for (int t = blockIdx.x * wpb + warp; t < ntask; t += gridDim.x * wpb) {
        if (t < n32) {
            tiny_front_group<T, 32>(list[t], fronts, child, relmap, a_src, a_pos, Ax, Ls, Us,
                                    status, slice);
        } else if (t < n32 + t16) {
            const int k = 2 * (t - n32) + (lane >> 4);
            if (k < n16)
                tiny_front_group<T, 16>(list[n32 + k], fronts, child, relmap, a_src, a_pos, Ax,
                                        Ls, Us, status, slice + (lane >> 4) * 16 * 17);
        } else {
            const int k = 4 * (t - n32 - t16) + (lane >> 3);
            if (k < n8)
                tiny_front_group<T, 8>(list[n32 + n16 + k], fronts, child, relmap, a_src, a_pos,
                                       Ax, Ls, Us, status, slice + (lane >> 3) * 8 * 9);
        }
        __syncwarp();
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
                   const int* __restrict__ asm_off, const int* __restrict__ asm_range,
                   const double* __restrict__ Ax, T* __restrict__ Ls, T* __restrict__ Us) {
    extern __shared__ int rel_sh[];  // a child's relative map from its first column in range
    const int it = find_item(before, nitems, blockIdx.x);
    const int s = items[it];
    const int blk = blockIdx.x - before[it];
    const FrontDesc f = fronts[s];
    const int j0 = blk * CB, j1 = min(j0 + CB, f.m);
    const int tid = threadIdx.x, nt = blockDim.x;
    const int nch = f.child_end - f.child_beg;
    const int* ranges = asm_range + asm_off[s] + blk * nch * 2;

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
    // children one after another (deterministic sums); each child's update
    // columns that land in [j0, j1) were located on the host.  The child's
    // relative map goes to shared memory and every thread keeps four
    // independent loads in flight before its read-modify-writes.
    for (int h = 0; h < nch; ++h) {
        const int jlo = ranges[2 * h], jhi = ranges[2 * h + 1];
        if (jlo == jhi) continue;
        const FrontDesc g = fronts[child[f.child_beg + h]];
        const int uc = g.m - g.c;
        const int* rm = relmap + g.rows_off + g.c;
        for (int q = jlo + tid; q < uc; q += nt) rel_sh[q - jlo] = rm[q];
        __syncthreads();
        const T* U = Us + g.uoff;
        for (int jc = jlo; jc < jhi; ++jc) {
            const int pc = rel_sh[jc - jlo];
            const T* ucol = U + (int64_t)jc * g.ldu;
            for (int ic0 = jc + tid; ic0 < uc; ic0 += 4 * nt) {
                T v[4];
                int pr[4];
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    const int ic = ic0 + u * nt;
                    pr[u] = ic < uc ? rel_sh[ic - jlo] : -1;
                    v[u] = ic < uc ? ucol[ic] : T(0);
                }
#pragma unroll
                for (int u = 0; u < 4; ++u)
                    if (pr[u] >= 0) *front_elem(Ls, Us, f, pr[u], pc) += v[u];
            }
        }
        __syncthreads();
    }
}

// Warp-per-column variant: no block barriers, only warp syncs.  Each warp
// builds its column in windows of W rows (W a multiple of 16) in its own
// shared slice, so the slice does not grow with the front.  A child's columns
// landing in the CTA's block of CB columns are at most CB (the relative map
// is injective): the child column that lands in parent column jj is found by
// one ballot over the child's range.  The child rows landing in a window are
// one contiguous range (increasing relative map), read from the per-16-row
// block table asm_range.  Every front entry gets its A value (or zero), then
// the children's contributions in child order: the sums of a child-by-child
// extend-add.
template <typename T>
__global__ void __launch_bounds__(256)
    k_big_assemble_warp(const FrontDesc* __restrict__ fronts, const int* __restrict__ items,
                        const int* __restrict__ before, int nitems, int CB,
                        const int* __restrict__ child, const int* __restrict__ relmap,
                        const int* __restrict__ a_src, const int* __restrict__ a_pos,
                        const int* __restrict__ a_colptr, const int* __restrict__ a_colptr_off,
                        const int* __restrict__ asm_off, const int* __restrict__ asm_range,
                        const double* __restrict__ Ax, T* __restrict__ Ls, T* __restrict__ Us,
                        int W) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nw = blockDim.x >> 5;
    T* colbuf = reinterpret_cast<T*>(smem_raw) + (size_t)warp * W;
    const int it = find_item(before, nitems, blockIdx.x);
    const int s = items[it];
    const int blk = blockIdx.x - before[it];
    const FrontDesc f = fronts[s];
    const int j0 = blk * CB, j1 = min(j0 + CB, f.m);
    const int nch = f.child_end - f.child_beg;
    const int* rtab = asm_range + asm_off[s];  // [16-row block][child] -> [lo, hi)
    const int* ranges = rtab + blk * nch * 2;
    const int* cp = j0 < f.c ? a_colptr + a_colptr_off[s] : nullptr;
    for (int jj = j0 + warp; jj < j1; jj += nw) {
        const bool inL = jj < f.c;
        const int rlo = inL ? 0 : jj;
        for (int R0 = (rlo / W) * W; R0 < f.m; R0 += W) {
            const int R1 = min(R0 + W, f.m), w0 = max(R0, rlo);
            for (int r = w0 + lane; r < R1; r += 32) colbuf[r - R0] = T(0);
            __syncwarp();
            if (inL) {
                const int e0 = f.a_beg + cp[jj], e1 = f.a_beg + cp[jj + 1];
                for (int e = e0 + lane; e < e1; e += 32) {
                    const int src = a_src[e], row = a_pos[e] & 0xffff;
                    if (src >= 0 && row >= R0 && row < R1) colbuf[row - R0] = (T)Ax[src];
                }
                __syncwarp();
            }
            const int b0 = R0 / 16, b1 = (R1 - 1) / 16;
            for (int h = 0; h < nch; ++h) {
                const int jlo = ranges[2 * h], jhi = ranges[2 * h + 1];
                if (jlo == jhi) continue;
                const FrontDesc g = fronts[child[f.child_beg + h]];
                const int* rm = relmap + g.rows_off + g.c;
                const int cand = jlo + lane;
                const unsigned hit =
                    __ballot_sync(0xffffffffu, cand < jhi && __ldg(rm + cand) == jj);
                if (!hit) continue;
                const int jc = jlo + __ffs(hit) - 1;
                // child rows >= jc landing in rows [R0, R1) of the parent
                const int ilo = max(jc, rtab[(b0 * nch + h) * 2]);
                const int ihi = rtab[(b1 * nch + h) * 2 + 1];
                const T* ucol = Us + g.uoff + (int64_t)jc * g.ldu;
                for (int ic0 = ilo + lane; ic0 < ihi; ic0 += 8 * 32) {
                    int pr[8];
                    T v[8];
#pragma unroll
                    for (int u = 0; u < 8; ++u) {
                        const int ic = ic0 + u * 32;
                        pr[u] = ic < ihi ? __ldg(rm + ic) : -1;
                        v[u] = ic < ihi ? __ldg(ucol + ic) : T(0);
                    }
#pragma unroll
                    for (int u = 0; u < 8; ++u)
                        if (pr[u] >= 0) colbuf[pr[u] - R0] += v[u];
                }
                __syncwarp();
            }
            if (inL) {
                T* col = Ls + f.loff + (int64_t)jj * f.ldl;
                for (int r = w0 + lane; r < R1; r += 32) col[r] = colbuf[r - R0];
            } else {
                T* col = Us + f.uoff + (int64_t)(jj - f.c) * f.ldu;
                for (int r = w0 + lane; r < R1; r += 32) col[r - f.c] = colbuf[r - R0];
            }
            __syncwarp();
        }
    }
}

// ---------------------------------------------------------------------------
// large fronts: tiles
// ---------------------------------------------------------------------------

// Factor diagonal tile k of front f in place and store its inverse (TB x TB,
// column-major, zero above the diagonal) at Dk (potrf_tile_core on a copy in
// shared memory; a partial tile (n < 64) is padded with the identity).
// S, W: TB x kPotrfLD.
template <typename T, int TB>
__device__ void potrf_diag_tile(const FrontDesc& f, int k, T* Ls, T* Dk, T* S, T* W,
                                int* status) {
    constexpr int LD = kPotrfLD;
    const int tid = threadIdx.x, nt = blockDim.x;
    const TileRange tk = tile_range(k, f.m, f.c, TB);
    const int n = tk.size;
    T* base = Ls + f.loff + tk.start + (int64_t)tk.start * f.ldl;
    for (int idx = tid; idx < TB * TB; idx += nt) {
        int j = idx / TB, i = idx - j * TB;
        T v = (i == j) ? T(1) : T(0);
        if (i < n && j < n && i >= j) v = base[i + (int64_t)j * f.ldl];
        S[i + j * LD] = v;
    }
    potrf_tile_core<T, TB>(S, W, n, f.first_col + tk.start, status);
    for (int idx = tid; idx < TB * TB; idx += nt) {
        int j = idx / TB, i = idx - j * TB;
        if (i < n && j < n && i >= j) base[i + (int64_t)j * f.ldl] = S[i + j * LD];
        Dk[idx] = (i >= j && i < n && j < n) ? W[i + j * LD] : T(0);
    }
}

template <typename T, int TB>
__global__ void __launch_bounds__(256)
    k_tile_potrf(const FrontDesc* __restrict__ fronts, const int* __restrict__ list, int k,
                 const int64_t* __restrict__ dinv_off, T* __restrict__ Ls, T* __restrict__ Dinv,
                 int* __restrict__ status) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* S = reinterpret_cast<T*>(smem_raw);
    T* W = S + TB * kPotrfLD;
    const int s = list[blockIdx.x];
    const FrontDesc f = fronts[s];
    if (k >= tiles_l(f.c, TB)) return;
    potrf_diag_tile<T, TB>(f, k, Ls, Dinv + dinv_off[s] + (int64_t)k * TB * TB, S, W, status);
}

// X = A_ik inv(L_kk)' in place, CTA per row tile below the panel tile.
template <typename T, int TB>
__global__ void __launch_bounds__(256)
    k_tile_trsm(const FrontDesc* __restrict__ fronts, const int* __restrict__ items,
                const int* __restrict__ before, int nitems, int k,
                const int64_t* __restrict__ dinv_off, T* __restrict__ Ls,
                const T* __restrict__ Dinv) {
    static_assert(TB == 64, "4x4 register tile over 256 threads assumes TB = 64");
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* As = reinterpret_cast<T*>(smem_raw);  // [K][TB]
    T* Bs = As + TB * TB;                    // [K][TB]: inv(L_kk)' columns
    const int it = find_item(before, nitems, blockIdx.x);
    const int s = items[it];
    const FrontDesc f = fronts[s];
    const int i = k + 1 + (blockIdx.x - before[it]);
    const TileRange tk = tile_range(k, f.m, f.c, TB);
    const TileRange ti = tile_range(i, f.m, f.c, TB);
    const int tid = threadIdx.x;
    const int K = tk.size;
    T* aik = Ls + f.loff + ti.start + (int64_t)tk.start * f.ldl;
    const T* Dk = Dinv + dinv_off[s] + (int64_t)k * TB * TB;  // inv(L_kk), col-major TB
    for (int idx = tid; idx < TB * K; idx += 256) {
        int q = idx / TB, r = idx - q * TB;
        As[q * TB + r] = r < ti.size ? aik[r + (int64_t)q * f.ldl] : T(0);
        Bs[q * TB + r] = Dk[r + q * TB];  // Bs[q][j] = inv(L)[j][q]
    }
    __syncthreads();
    T acc[4][4];
    tile_gemm_nt_acc<T, TB>(As, Bs, K, acc);
    const int r0 = (tid & 15) * 4, c0 = (tid >> 4) * 4;
#pragma unroll
    for (int b = 0; b < 4; ++b) {
        int cc = c0 + b;
        if (cc >= K) continue;
#pragma unroll
        for (int a = 0; a < 4; ++a) {
            int rr = r0 + a;
            if (rr < ti.size) aik[rr + (int64_t)cc * f.ldl] = acc[a][b];
        }
    }
}

// jcap < 0: every lower tile right of panel tile k (the FP64 schedule).
// jcap >= 0: only tile columns k < j <= jcap (the rest of a 256-column panel;
// the trailing part then gets one tensor-core update per panel).
template <typename T, int TB>
__global__ void __launch_bounds__(256)
    k_tile_update(const FrontDesc* __restrict__ fronts, const int* __restrict__ items,
                  const int* __restrict__ before, int nitems, int k, int jcap,
                  const int64_t* __restrict__ dinv_off, T* __restrict__ Ls, T* __restrict__ Us,
                  T* __restrict__ Dinv, int* __restrict__ status) {
    static_assert(TB == 64, "4x4 register tile over 256 threads assumes TB = 64");
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* As = reinterpret_cast<T*>(smem_raw);  // [K][TB]
    T* Bs = As + TB * TB;                    // [K][TB]
    const int it = find_item(before, nitems, blockIdx.x);
    const int s = items[it];
    const FrontDesc f = fronts[s];
    int i, j;
    if (jcap < 0) {
        int ii, jj;
        lower_index(blockIdx.x - before[it], ii, jj);
        i = k + 1 + ii;
        j = k + 1 + jj;
    } else {  // column-major over the panel's remaining tile columns
        const int NT = tiles_l(f.c, TB) + (f.m - f.c + TB - 1) / TB;
        int l = blockIdx.x - before[it];
        j = k + 1;
        while (l >= NT - j) {
            l -= NT - j;
            ++j;
        }
        i = j + l;
    }
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
    T acc[4][4];
    tile_gemm_nt_acc<T, TB>(As, Bs, K, acc);
    const int r0 = (tid & 15) * 4, c0 = (tid >> 4) * 4;
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
    if (i == k + 1 && j == k + 1 && i < tiles_l(f.c, TB) && (jcap < 0 || i <= jcap)) {
        __syncthreads();
        potrf_diag_tile<T, TB>(f, i, Ls, Dinv + dinv_off[s] + (int64_t)i * TB * TB, As,
                               As + TB * kPotrfLD, status);
    }
}

// ---------------------------------------------------------------------------
// host launchers
// ---------------------------------------------------------------------------

// rows per window of the warp-per-column assembly's column buffers
constexpr int kAssembleWindow = 1024;
constexpr size_t kAssembleColsSmemMax = 8 * kAssembleWindow * sizeof(double);

// shared memory of the tile kernels: two 64 x kPotrfLD buffers (operands of
// the tile products in 64 x 65 of them, or S and W of the diagonal-tile
// factorization)
template <typename T>
static size_t diag_smem() {
    return (size_t)2 * kTile * kPotrfLD * sizeof(T);
}

// The level's small fronts in pieces, piece i on sts[i]: the tiny fronts
// (piece 0), then one k_small_front launch per size bucket.
template <typename T>
void launch_small_fronts(const DevPlan& D, int level, T* Ls, T* Us, const double* Ax,
                         int* status, const cudaStream_t* sts) {
    {  // fronts of at most 32 rows (the first two buckets): one, two or four per warp
        const int beg = D.h_small_ptr[level * kSmallBuckets];
        const int end = D.h_small_ptr[level * kSmallBuckets + Plan::kTinyBuckets];
        const cudaStream_t st = sts[0];
        if (end > beg) {
            double by = 0;
            for (int b = 0; b < Plan::kTinyBuckets; ++b)
                by += D.h_small_bytes[level * kSmallBuckets + b];
            ProfScope ps(D.prof, KC_SMALL_FRONT, st, 0, by * sizeof(T) / 8.0);
            const size_t smem = (size_t)4 * kTinyFrontRows * (kTinyFrontRows + 1) * sizeof(T);
            // the level's slice of the rows-descending warp list: its fronts
            // of 17..32 rows end the part above 16 rows, then 9..16, then <= 8
            const int* cnt = D.solve.warp_cnt.data() + 3 * level;
            const int n32 = D.h_small_ptr[level * kSmallBuckets + 2] -
                            D.h_small_ptr[level * kSmallBuckets + 1];
            const int n16 = cnt[1], n8 = cnt[2];
            const int ntask = n32 + (n16 + 1) / 2 + (n8 + 3) / 4;
            const int blocks = std::min((ntask + 3) / 4, D.tiny_blocks_cap);
            k_tiny_fronts<T><<<blocks, 128, smem, st>>>(
                D.fronts, D.solve.warp_list + beg + (cnt[0] - n32), n32, n16, n8, D.child,
                D.relmap, D.a_src, D.a_pos, Ax, Ls, Us, status);
        }
    }
    for (int b = Plan::kTinyBuckets; b < kSmallBuckets; ++b) {
        int beg = D.h_small_ptr[level * kSmallBuckets + b];
        int end = D.h_small_ptr[level * kSmallBuckets + b + 1];
        if (end == beg) continue;
        int MB = Plan::small_limit[b];
        int LD = MB + 1;
        size_t smem = (size_t)MB * LD * sizeof(T) + (size_t)MB * sizeof(int);
        const int threads = D.small_threads[b];
        const cudaStream_t st = sts[1 + b - Plan::kTinyBuckets];
        ProfScope ps(D.prof, KC_SMALL_FRONT, st, 0,
                     D.h_small_bytes[level * kSmallBuckets + b] * sizeof(T) / 8.0);
        k_small_front<T><<<end - beg, threads, smem, st>>>(D.fronts, D.small_list + beg, D.child,
                                                          D.relmap, D.a_src, D.a_pos, Ax, Ls, Us,
                                                          LD, status);
    }
}

template <typename T>
void launch_large_level(const DevPlan& D, int level, T* Ls, T* Us, T* Dinv, const double* Ax,
                        int* status, cudaStream_t st) {
    const int lb = D.h_large_ptr[level], le = D.h_large_ptr[level + 1];
    if (le == lb) return;
    const DevSchedule& S = D.sched64;
    const WorkList& asl = D.h_assemble[level];
    {
        ProfScope ps(D.prof, KC_ASSEMBLE, st);
        k_big_assemble<T><<<asl.nctas, 256, D.max_u * sizeof(int), st>>>(
            D.fronts, S.items + asl.off, S.before + asl.off, asl.nitems, kAssembleCols, D.child,
            D.relmap, D.a_src, D.a_pos, D.a_colptr, D.a_colptr_off, D.asm_off, D.asm_range, Ax,
            Ls, Us);
    }
    {
        ProfScope ps(D.prof, KC_POTRF, st);
        k_tile_potrf<T, kTile><<<le - lb, 256, diag_smem<T>(), st>>>(D.fronts, D.large_list + lb,
                                                                     0, D.dinv_off, Ls, Dinv,
                                                                     status);
    }
    const size_t gsm = diag_smem<T>();
    for (int q = S.h_level_beg[level]; q < S.h_level_beg[level + 1]; ++q) {
        const WorkList& tr = S.h_trsm[q];
        const WorkList& up = S.h_update[q];
        if (tr.nctas > 0) {
            ProfScope ps(D.prof, KC_TRSM, st);
            k_tile_trsm<T, kTile><<<tr.nctas, 256, gsm, st>>>(
                D.fronts, S.items + tr.off, S.before + tr.off, tr.nitems, tr.step, D.dinv_off, Ls,
                Dinv);
        }
        if (up.nctas > 0) {
            ProfScope ps(D.prof, KC_SCHUR, st, D.h_update_flops[q]);
            k_tile_update<T, kTile><<<up.nctas, 256, gsm, st>>>(
                D.fronts, S.items + up.off, S.before + up.off, up.nitems, up.step, -1, D.dinv_off,
                Ls, Us, Dinv, status);
        }
    }
}

// Large fronts in 256-column panels: per panel one launch of dependency-
// ordered row-tile tasks (k_panel: diagonal tiles, triangular solves and the
// panel's own updates), then one wide Schur update of the whole trailing
// part -- tcgen05 tensor cores (TF32) for FP32, the register-tiled FP64
// kernel for FP64.  status[1] receives a device wait's error code (1, 2:
// the tensor-core pipeline; 3: a panel dependency wait; 4: a panel ticket
// counter not cleared).
template <typename T>
static void launch_large_level_panels(const DevPlan& D, int level, T* Ls, T* Us, T* Dinv,
                                      const double* Ax, int* status, int smode,
                                      cudaStream_t st) {
    const DevSchedule& S = D.psched;
    const size_t gsm = diag_smem<T>();
    for (int q = S.h_op_beg[level]; q < S.h_op_beg[level + 1]; ++q) {
        const PanelOp& op = S.h_ops[q];
        const WorkList& w = op.w;
        if (op.kind == OP_PANEL ? op.ntasks == 0 : w.nctas == 0) continue;
        switch (op.kind) {
            case OP_ASSEMBLE: {
                ProfScope ps(D.prof, KC_ASSEMBLE, st, 0, op.elems * sizeof(T) + op.xbytes);
                // a warp per column, 8 warps, columns built in windows of
                // kAssembleWindow rows (the whole column when shorter)
                const int W = std::min(kAssembleWindow, (D.h_level_max_m[level] + 15) & ~15);
                k_big_assemble_warp<T><<<w.nctas, 256, (size_t)8 * W * sizeof(T), st>>>(
                    D.fronts, S.items + w.off, S.before + w.off, w.nitems, kAssembleCols, D.child,
                    D.relmap, D.a_src, D.a_pos, D.a_colptr, D.a_colptr_off, D.asm_off,
                    D.asm_range, Ax, Ls, Us, W);
                break;
            }
            case OP_POTRF: {
                ProfScope ps(D.prof, KC_POTRF, st, op.flops, op.elems * sizeof(T));
                k_tile_potrf<T, kTile><<<w.nitems, 256, diag_smem<T>(), st>>>(
                    D.fronts, S.items + w.off, op.arg, D.dinv_off, Ls, Dinv, status);
                break;
            }
            case OP_TRSM: {
                ProfScope ps(D.prof, KC_TRSM, st, op.flops, op.elems * sizeof(T));
                k_tile_trsm<T, kTile><<<w.nctas, 256, gsm, st>>>(
                    D.fronts, S.items + w.off, S.before + w.off, w.nitems, op.arg, D.dinv_off, Ls,
                    Dinv);
                break;
            }
            case OP_UPDATE_PANEL: {
                ProfScope ps(D.prof, KC_TRSM, st, op.flops, op.elems * sizeof(T));
                k_tile_update<T, kTile><<<w.nctas, 256, gsm, st>>>(
                    D.fronts, S.items + w.off, S.before + w.off, w.nitems, op.arg, op.arg2,
                    D.dinv_off, Ls, Us, Dinv, status);
                break;
            }
            case OP_PANEL: {
                ProfScope ps(D.prof, KC_TRSM, st, op.flops, op.elems * sizeof(T));
                // the panel scratch the tensor-core Schur update reads:
                // the 3xTF32 hi/lo split (1) or the BF16 copy (2)
                launch_panel<T>(D, op, Ls, Dinv, status,
                                sizeof(T) == 4 ? (smode == kSchurBF16 ? 2 : 1) : 0, st);
                break;
            }
            case OP_SCHUR_TC: {
                // one update per panel: the FP64 factor's (the tensor-core
                // path runs the deferred updates below instead)
                if constexpr (sizeof(T) == 8) {
                    ProfScope ps(D.prof, KC_SCHUR, st, op.flops, op.elems * sizeof(T));
                    launch_schur_f64(D, w, op.arg, kPanel, Ls, Us, st);
                }
                break;
            }
            case OP_SCHUR_NEXT:
            case OP_SCHUR_REST: {
                if constexpr (sizeof(T) == 4) {
                    ProfScope ps(D.prof, KC_SCHUR, st, op.flops, op.elems * sizeof(T));
                    launch_schur_tc(D, w, op.arg, kPanel, op.arg2, op.kind == OP_SCHUR_NEXT, Ls,
                                    Us, status + 1, smode, st);
                }
                break;
            }
        }
    }
}

template <typename T>
static void set_factor_attributes() {
    cudaFuncSetAttribute(k_small_front<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         227 * 1024);
    cudaFuncSetAttribute(k_tile_update<T, kTile>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)diag_smem<T>());
    cudaFuncSetAttribute(k_tile_trsm<T, kTile>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)diag_smem<T>());
    cudaFuncSetAttribute(k_tile_potrf<T, kTile>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)diag_smem<T>());
    cudaFuncSetAttribute(k_big_assemble<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         227 * 1024);
    cudaFuncSetAttribute(k_big_assemble_warp<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)kAssembleColsSmemMax);
}

void init_factor_kernels() {
    set_factor_attributes<double>();
    set_factor_attributes<float>();
}

// Level by level.  A level's small and large fronts depend only on lower
// levels, so its small fronts run beside its large fronts, each piece (the
// tiny fronts, each k_small_front size bucket) on a stream of its own (fork
// and join by events; inside a stream capture these become parallel graph
// branches).  Serial while the profiler records, so each class keeps its own
// time.
template <typename T>
void factor_levels(const DevPlan& D, T* Ls, T* Us, T* Dinv, const double* Ax, int* status,
                   cudaStream_t st, int smode) {
    const bool fork = D.fork_ev && !(D.prof && D.prof->on);
    if (D.fsync && D.nfsync > 0) cudaMemsetAsync(D.fsync, 0, (size_t)D.nfsync * sizeof(int), st);
    for (int l = 0; l < D.nlevels; ++l) {
        const bool has_small =
            D.h_small_ptr[(l + 1) * kSmallBuckets] > D.h_small_ptr[l * kSmallBuckets];
        const bool has_large = D.h_large_ptr[l + 1] > D.h_large_ptr[l];
        // pieces of the level's small fronts that have fronts
        bool piece[DevPlan::kSmallPieces];
        int npieces = 0;
        piece[0] = D.h_small_ptr[l * kSmallBuckets + Plan::kTinyBuckets] >
                   D.h_small_ptr[l * kSmallBuckets];
        for (int b = Plan::kTinyBuckets; b < kSmallBuckets; ++b)
            piece[1 + b - Plan::kTinyBuckets] =
                D.h_small_ptr[l * kSmallBuckets + b + 1] > D.h_small_ptr[l * kSmallBuckets + b];
        for (int i = 0; i < DevPlan::kSmallPieces; ++i) npieces += piece[i];
        const bool par = fork && D.piece_st[0] && has_small && (has_large || npieces > 1);
        if (par) {
            // every piece on its own stream beside the large fronts
            cudaEventRecord(D.fork_ev, st);
            for (int i = 0; i < DevPlan::kSmallPieces; ++i)
                if (piece[i]) cudaStreamWaitEvent(D.piece_st[i], D.fork_ev, 0);
            launch_small_fronts<T>(D, l, Ls, Us, Ax, status, D.piece_st);
            for (int i = 0; i < DevPlan::kSmallPieces; ++i)
                if (piece[i]) cudaEventRecord(D.piece_join[i], D.piece_st[i]);
        } else {
            cudaStream_t serial[DevPlan::kSmallPieces];
            for (int i = 0; i < DevPlan::kSmallPieces; ++i) serial[i] = st;
            launch_small_fronts<T>(D, l, Ls, Us, Ax, status, serial);
        }
        // FP32 needs the TMA descriptors of the tensor-core path; without them
        // (descriptor encoding unavailable) it keeps the 64-wide tile schedule
        if (sizeof(T) == 8 || (smode == kSchurBF16 ? D.tmaps_bf16 != nullptr : D.tmaps != nullptr))
            launch_large_level_panels<T>(D, l, Ls, Us, Dinv, Ax, status, smode, st);
        else
            launch_large_level<T>(D, l, Ls, Us, Dinv, Ax, status, st);
        if (par)
            for (int i = 0; i < DevPlan::kSmallPieces; ++i)
                if (piece[i]) cudaStreamWaitEvent(st, D.piece_join[i], 0);
    }
}

template void factor_levels<double>(const DevPlan&, double*, double*, double*, const double*,
                                    int*, cudaStream_t, int);
template void factor_levels<float>(const DevPlan&, float*, float*, float*, const double*, int*,
                                   cudaStream_t, int);

}  // namespace mdgpu
