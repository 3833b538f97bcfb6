// Selected inverse and the adjoint of logdet A + b' A^-1 b.
//
// For A = L L' (the FP64 factor), Z = A^-1 on the pattern of L satisfies the
// Takahashi recurrence, column by column from the last: with R the rows
// below the diagonal of column j (a clique of the filled graph),
//     y = L(R, j) / L(j, j),   Z(R, j) = -Z(R, R) y,
//     Z(j, j) = 1 / L(j, j)^2 - y' Z(R, j).
// Per front, with its pivot columns in blocks K of NB columns from the last
// and R the front rows below the block, the same in block form:
//     W = inv(L_KK),  Y = L_RK W,  Z_RK = -Z_RR Y,  Z_KK = W'W - Y' Z_RK.
// Z_RR lies inside the front: its pivot part was computed by the later
// blocks, its update part Z_UU is the parent front's Z on the front's update
// rows (gathered through the relative map -- the transpose of the
// extend-add).  So the fronts are processed level by level from the root:
// small fronts one CTA each (blocks of 16 columns), large fronts in blocks of
// 64 columns over many CTAs per front (below); Z of the pivot columns goes to
// a store laid out like the L panels, Z_UU to the selected inverse's own
// update store.
//
// The gradient of loss = logdet A + b' A^-1 b with respect to the caller's
// lower-triangle values: with x = A^-1 b, d loss / d A = Z - x x' (symmetric),
// so an off-diagonal entry (one value standing for A(i,j) and A(j,i)) gets
// 2 (Z(i,j) - x_i x_j) and a diagonal entry Z(i,i) - x_i^2.
#include <cuda_runtime.h>

#include <cstdint>

#include "device_common.cuh"
#include "kernels.hpp"

namespace mdgpu {

constexpr int kSelBlock = 16;  // pivot columns per block of the recurrence

// Z(r, col), r >= col, front-local indices of front f
// (Z's update part of front f at zoff in the Zu store)
__device__ __forceinline__ double& zelem(double* Zs, double* Zu, const FrontDesc& f,
                                         int64_t zoff, int r, int col) {
    if (col < f.c) return Zs[f.loff + r + (int64_t)col * f.ldl];
    return Zu[zoff + (r - f.c) + (int64_t)(col - f.c) * f.ldu];
}

__global__ void __launch_bounds__(256, 2)
    k_selinv_front(const FrontDesc* __restrict__ fronts, const int* __restrict__ list,
                   const int* __restrict__ relmap, const double* __restrict__ Ls,
                   double* __restrict__ Zs, double* __restrict__ Zu,
                   const int64_t* __restrict__ zuoff, double* __restrict__ Yscr,
                   const int64_t* __restrict__ yoff) {
    constexpr int NB = kSelBlock;
    __shared__ double Lk[NB][NB + 1];
    __shared__ double Wk[NB][NB + 1];
    const int tid = threadIdx.x, nt = blockDim.x;
    const int s = list[blockIdx.x];
    const FrontDesc f = fronts[s];
    const int m = f.m, c = f.c, u = m - c;
    const int64_t zf = (f.parent >= 0 && u > 0) ? zuoff[s] : -1;
    // the update part: the parent's Z on this front's update rows
    if (f.parent >= 0 && u > 0) {
        const FrontDesc p = fronts[f.parent];
        const int64_t zp = zuoff[f.parent];
        const int* rm = relmap + f.rows_off + c;
        for (int b = 0; b < u; ++b) {
            const int pb = rm[b];
            for (int a = b + tid; a < u; a += nt)
                Zu[zf + a + (int64_t)b * f.ldu] = zelem(Zs, Zu, p, zp, rm[a], pb);
        }
        __syncthreads();
    }
    double* Y = Yscr + yoff[s];  // (m - k1) x NB, row-major
    const double* L = Ls + f.loff;
    const int nblk = (c + NB - 1) / NB;
    for (int kb = nblk - 1; kb >= 0; --kb) {
        const int k0 = kb * NB, k1 = min(k0 + NB, c), nb = k1 - k0;
        // W = inv(L_KK): a column per thread, forward substitution
        for (int e = tid; e < NB * NB; e += nt) {
            const int i = e % NB, j = e / NB;
            Lk[i][j] = (i < nb && j < nb && i >= j) ? L[(k0 + i) + (int64_t)(k0 + j) * f.ldl] : 0.0;
        }
        __syncthreads();
        if (tid < NB) {
            const int j = tid;
            for (int i = 0; i < NB; ++i) {
                double v = 0.0;
                if (i < nb && j < nb && i >= j) {
                    v = (i == j) ? 1.0 : 0.0;
                    for (int k = j; k < i; ++k) v -= Lk[i][k] * Wk[k][j];
                    v /= Lk[i][i];
                }
                Wk[i][j] = v;
            }
        }
        __syncthreads();
        // Y = L_RK W, a row per thread
        for (int a = k1 + tid; a < m; a += nt) {
            double l[NB];
#pragma unroll
            for (int k = 0; k < NB; ++k) l[k] = k < nb ? L[a + (int64_t)(k0 + k) * f.ldl] : 0.0;
            double* y = Y + (int64_t)(a - k1) * NB;
#pragma unroll 1
            for (int j = 0; j < NB; ++j) {
                double v = 0.0;
#pragma unroll
                for (int k = 0; k < NB; ++k) v += l[k] * Wk[k][j];
                y[j] = v;
            }
        }
        __syncthreads();
        // Z_RK = -Z_RR Y, a row per thread
        for (int a = k1 + tid; a < m; a += nt) {
            double acc[NB];
#pragma unroll
            for (int j = 0; j < NB; ++j) acc[j] = 0.0;
            for (int b = k1; b < m; ++b) {
                const double z = b <= a ? zelem(Zs, Zu, f, zf, a, b) : zelem(Zs, Zu, f, zf, b, a);
                const double* y = Y + (int64_t)(b - k1) * NB;
#pragma unroll
                for (int j = 0; j < NB; ++j) acc[j] += z * y[j];
            }
            for (int j = 0; j < nb; ++j) Zs[f.loff + a + (int64_t)(k0 + j) * f.ldl] = -acc[j];
        }
        __syncthreads();
        // Z_KK = W'W - Y' Z_RK, lower part, an entry per thread
        for (int e = tid; e < NB * NB; e += nt) {
            const int i = e % NB, j = e / NB;
            if (i >= nb || j >= nb || i < j) continue;
            double v = 0.0;
            for (int k = i; k < nb; ++k) v += Wk[k][i] * Wk[k][j];
            for (int a = k1; a < m; ++a)
                v -= Y[(int64_t)(a - k1) * NB + i] * Zs[f.loff + a + (int64_t)(k0 + j) * f.ldl];
            Zs[f.loff + (k0 + i) + (int64_t)(k0 + j) * f.ldl] = v;
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// large fronts: the same recurrence in blocks of kSelT = 64 pivot columns
// (the factor's diagonal tiles, whose inverses W it stored), one launch per
// phase and block step over every large front of the level, many CTAs per
// front:
//   gather  Z_UU from the parent's Z (CTA per front and 16 columns)
//   y       Y = L_RK W                (CTA per front and 64-row tile of R)
//   zrk     Z_RK = -Z_RR Y            (CTA per front and 64-row tile of R)
//   zkk     Z_KK = W'W - Y' Z_RK      (CTA per front)
// Y and a row-major copy of Z_RK sit in the front's scratch (2 m x 64).
// ---------------------------------------------------------------------------

constexpr int kSelT = 64;
// dynamic shared memory of the tiled phases: two 64 x 65 FP64 blocks
constexpr int kSelSmem = 2 * kSelT * (kSelT + 1) * (int)sizeof(double);

__device__ __forceinline__ double zget(const double* __restrict__ Zs,
                                       const double* __restrict__ Zu, const FrontDesc& f,
                                       int64_t zoff, int r, int col) {
    if (r < col) {
        const int t = r;
        r = col;
        col = t;
    }
    if (col < f.c) return Zs[f.loff + r + (int64_t)col * f.ldl];
    return Zu[zoff + (r - f.c) + (int64_t)(col - f.c) * f.ldu];
}

// acc[a][b] += sum over q < K of As[q lda + r0 + a] Bs[q ldb + c0 + b]
__device__ __forceinline__ void sel_gemm(const double* As, int lda, const double* Bs, int ldb,
                                         int K, double (&acc)[4][4]) {
    const int tid = threadIdx.x;
    const int r0 = (tid & 15) * 4, c0 = (tid >> 4) * 4;
    for (int q = 0; q < K; ++q) {
        double av[4], bv[4];
#pragma unroll
        for (int a = 0; a < 4; ++a) av[a] = As[q * lda + r0 + a];
#pragma unroll
        for (int b = 0; b < 4; ++b) bv[b] = Bs[q * ldb + c0 + b];
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
            for (int b = 0; b < 4; ++b) acc[a][b] += av[a] * bv[b];
    }
}

struct SelStep {
    int kb, k0, k1, nb;
};
__device__ __forceinline__ SelStep sel_step(const FrontDesc& f, int step) {
    SelStep t;
    const int nblk = (f.c + kSelT - 1) / kSelT;
    t.kb = nblk - 1 - step;
    t.k0 = t.kb * kSelT;
    t.k1 = min(t.k0 + kSelT, f.c);
    t.nb = t.k1 - t.k0;
    return t;
}

__global__ void __launch_bounds__(256)
    k_sel_gather(const FrontDesc* __restrict__ fronts, const int* __restrict__ items,
                 const int* __restrict__ before, int nitems, const int* __restrict__ relmap,
                 double* __restrict__ Zs, double* __restrict__ Zu,
                 const int64_t* __restrict__ zuoff) {
    const int it = find_item(before, nitems, blockIdx.x);
    const int s = items[it], blk = blockIdx.x - before[it];
    const FrontDesc f = fronts[s];
    const FrontDesc p = fronts[f.parent];
    const int u = f.m - f.c;
    const int64_t zf = zuoff[s], zp = zuoff[f.parent];
    const int* rm = relmap + f.rows_off + f.c;
    for (int b = 16 * blk; b < min(16 * blk + 16, u); ++b) {
        const int pb = rm[b];
        for (int a = b + (int)threadIdx.x; a < u; a += blockDim.x)
            Zu[zf + a + (int64_t)b * f.ldu] = zelem(Zs, Zu, p, zp, rm[a], pb);
    }
}

__global__ void __launch_bounds__(256)
    k_sel_y(const FrontDesc* __restrict__ fronts, const int* __restrict__ items,
            const int* __restrict__ before, int nitems, int step, const double* __restrict__ Ls,
            const double* __restrict__ Dinv, const int64_t* __restrict__ dinv_off,
            double* __restrict__ Yscr, const int64_t* __restrict__ yoff) {
    extern __shared__ double sel_sm[];
    double* As = sel_sm;                  // kSelT x kSelT
    double* Bs = As + kSelT * kSelT;      // kSelT x (kSelT + 1)
    const int it = find_item(before, nitems, blockIdx.x);
    const int s = items[it], rt = blockIdx.x - before[it];
    const FrontDesc f = fronts[s];
    const SelStep t = sel_step(f, step);
    const int a0 = t.k1 + kSelT * rt, rows = min(kSelT, f.m - a0);
    const double* W = Dinv + dinv_off[s] + (int64_t)t.kb * kSelT * kSelT;
    for (int idx = threadIdx.x; idx < kSelT * kSelT; idx += 256) {
        const int r = idx & 63, q = idx >> 6;
        As[q * kSelT + r] =
            (r < rows && q < t.nb) ? Ls[f.loff + a0 + r + (int64_t)(t.k0 + q) * f.ldl] : 0.0;
        // W(r, q) column-major: Bs[k][c] = W(k, c) with k = r, c = q
        Bs[r * (kSelT + 1) + q] = W[r + q * kSelT];
    }
    __syncthreads();
    double acc[4][4] = {};
    sel_gemm(As, kSelT, Bs, kSelT + 1, t.nb, acc);
    const int r0 = (threadIdx.x & 15) * 4, c0 = (threadIdx.x >> 4) * 4;
    double* Y = Yscr + yoff[s];
#pragma unroll
    for (int a = 0; a < 4; ++a)
        if (r0 + a < rows)
#pragma unroll
            for (int b = 0; b < 4; ++b) Y[(int64_t)(a0 + r0 + a - t.k1) * kSelT + c0 + b] = acc[a][b];
}

__global__ void __launch_bounds__(256)
    k_sel_zrk(const FrontDesc* __restrict__ fronts, const int* __restrict__ items,
              const int* __restrict__ before, int nitems, int step, double* __restrict__ Zs,
              const double* __restrict__ Zu, const int64_t* __restrict__ zuoff,
              double* __restrict__ Yscr, const int64_t* __restrict__ yoff) {
    extern __shared__ double sel_sm[];
    double* As = sel_sm;                      // kSelT x (kSelT + 1)
    double* Bs = As + kSelT * (kSelT + 1);    // kSelT x kSelT
    const int it = find_item(before, nitems, blockIdx.x);
    const int s = items[it], rt = blockIdx.x - before[it];
    const FrontDesc f = fronts[s];
    const SelStep t = sel_step(f, step);
    const int a0 = t.k1 + kSelT * rt, rows = min(kSelT, f.m - a0);
    const int64_t zf = (f.parent >= 0 && f.m > f.c) ? zuoff[s] : -1;
    double* Y = Yscr + yoff[s];
    const int ylen = f.m - t.k1;
    double* Zrk = Y + (int64_t)f.m * kSelT;
    double acc[4][4] = {};
    for (int b0 = t.k1; b0 < f.m; b0 += kSelT) {
        const int cols = min(kSelT, f.m - b0);
        // As[q][r] = Z(a0 + r, b0 + q): read along the stored columns
        const bool upper = b0 >= a0 + kSelT;  // every b above every a
        for (int idx = threadIdx.x; idx < kSelT * kSelT; idx += 256) {
            const int fast = idx & 63, slow = idx >> 6;
            const int r = upper ? slow : fast, q = upper ? fast : slow;
            As[q * (kSelT + 1) + r] =
                (r < rows && q < cols) ? zget(Zs, Zu, f, zf, a0 + r, b0 + q) : 0.0;
        }
        for (int idx = threadIdx.x; idx < kSelT * kSelT; idx += 256) {
            const int c = idx & 63, q = idx >> 6;
            Bs[q * kSelT + c] = q < cols ? Y[(int64_t)(b0 + q - t.k1) * kSelT + c] : 0.0;
        }
        __syncthreads();
        sel_gemm(As, kSelT + 1, Bs, kSelT, kSelT, acc);
        __syncthreads();
    }
    (void)ylen;
    const int r0 = (threadIdx.x & 15) * 4, c0 = (threadIdx.x >> 4) * 4;
#pragma unroll
    for (int a = 0; a < 4; ++a) {
        const int r = r0 + a;
        if (r >= rows) continue;
#pragma unroll
        for (int b = 0; b < 4; ++b) {
            const int c = c0 + b;
            const double v = -acc[a][b];
            Zrk[(int64_t)(a0 + r - t.k1) * kSelT + c] = v;
            if (c < t.nb) Zs[f.loff + a0 + r + (int64_t)(t.k0 + c) * f.ldl] = v;
        }
    }
}

__global__ void __launch_bounds__(256)
    k_sel_zkk(const FrontDesc* __restrict__ fronts, const int* __restrict__ items, int step,
              double* __restrict__ Zs, const double* __restrict__ Dinv,
              const int64_t* __restrict__ dinv_off, const double* __restrict__ Yscr,
              const int64_t* __restrict__ yoff) {
    extern __shared__ double sel_sm[];
    double* As = sel_sm;                      // kSelT x (kSelT + 1) each
    double* Bs = As + kSelT * (kSelT + 1);
    const int s = items[blockIdx.x];
    const FrontDesc f = fronts[s];
    const SelStep t = sel_step(f, step);
    const double* W = Dinv + dinv_off[s] + (int64_t)t.kb * kSelT * kSelT;
    const double* Y = Yscr + yoff[s];
    const double* Zrk = Y + (int64_t)f.m * kSelT;
    // W'W: As[q][i] = W(q, i)
    for (int idx = threadIdx.x; idx < kSelT * kSelT; idx += 256) {
        const int q = idx & 63, i = idx >> 6;
        const double w = W[q + i * kSelT];
        As[q * (kSelT + 1) + i] = w;
        Bs[q * (kSelT + 1) + i] = w;
    }
    __syncthreads();
    double pos[4][4] = {}, neg[4][4] = {};
    sel_gemm(As, kSelT + 1, Bs, kSelT + 1, t.nb, pos);
    __syncthreads();
    // Y' Z_RK over the rows of R
    for (int a0 = t.k1; a0 < f.m; a0 += kSelT) {
        const int rows = min(kSelT, f.m - a0);
        for (int idx = threadIdx.x; idx < kSelT * kSelT; idx += 256) {
            const int i = idx & 63, q = idx >> 6;
            const int64_t o = (int64_t)(a0 + q - t.k1) * kSelT + i;
            As[q * (kSelT + 1) + i] = q < rows ? Y[o] : 0.0;
            Bs[q * (kSelT + 1) + i] = q < rows ? Zrk[o] : 0.0;
        }
        __syncthreads();
        sel_gemm(As, kSelT + 1, Bs, kSelT + 1, kSelT, neg);
        __syncthreads();
    }
    const int r0 = (threadIdx.x & 15) * 4, c0 = (threadIdx.x >> 4) * 4;
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) {
            const int i = r0 + a, j = c0 + b;
            if (i < t.nb && j < t.nb && i >= j)
                Zs[f.loff + (t.k0 + i) + (int64_t)(t.k0 + j) * f.ldl] = pos[a][b] - neg[a][b];
        }
}

// G (caller order; zeroed by the caller) of every lower-triangle entry e:
// its front position (a_pos: row | column << 16 within front a_front[e]).
__global__ void k_grad_lower(int nnz, const FrontDesc* __restrict__ fronts,
                             const int* __restrict__ a_front, const int* __restrict__ a_src,
                             const int* __restrict__ a_pos, const int* __restrict__ rows,
                             const int* __restrict__ perm, const double* __restrict__ Zs,
                             const double* __restrict__ x, double* __restrict__ G) {
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < nnz; e += gridDim.x * blockDim.x) {
        const int src = a_src[e];
        if (src < 0) continue;  // a duplicate the assembly drops: gradient 0
        const FrontDesc f = fronts[a_front[e]];
        const int pos = a_pos[e], r = pos & 0xffff, jj = pos >> 16;
        double z = Zs[f.loff + r + (int64_t)jj * f.ldl];
        const int pr = rows[f.rows_off + r], pc = f.first_col + jj;
        if (x) {
            const int i = perm ? perm[pr] : pr, j = perm ? perm[pc] : pc;
            z -= x[i] * x[j];
        }
        G[src] = pr == pc ? z : 2.0 * z;
    }
}

// logdet = 2 sum log L(j, j): per block a fixed-order sum over its
// supernodes, then one block sums the partials (deterministic)
template <typename T>
__global__ void k_logdet_partial(int nsuper, const FrontDesc* __restrict__ fronts,
                                 const T* __restrict__ Ls, double* __restrict__ partial) {
    __shared__ double red[256];
    double v = 0.0;
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < nsuper; s += gridDim.x * blockDim.x) {
        const FrontDesc f = fronts[s];
        for (int j = 0; j < f.c; ++j) v += log((double)Ls[f.loff + j + (int64_t)j * f.ldl]);
    }
    red[threadIdx.x] = v;
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) partial[blockIdx.x] = red[0];
}

__global__ void k_logdet_final(int nparts, const double* __restrict__ partial,
                               double* __restrict__ out) {
    __shared__ double red[256];
    double v = 0.0;
    for (int i = threadIdx.x; i < nparts; i += blockDim.x) v += partial[i];
    red[threadIdx.x] = v;
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) out[0] = 2.0 * red[0];
}

constexpr int kLogdetBlocks = 148 * 2;

// Level by level from the root: the small fronts one CTA each
// (k_selinv_front), the large fronts by the tiled phases above, block step
// by block step (fronts with fewer pivot blocks join the later steps).
void launch_selinv(const DevPlan& D, const double* Ls, const double* Dinv, double* Zs,
                   double* Zu, double* Yscr, cudaStream_t st) {
    const SelSchedule& S = D.sel;
    for (int l = D.nlevels - 1; l >= 0; --l) {
        const int sb = D.h_small_ptr[l * kSmallBuckets], se = D.h_small_ptr[(l + 1) * kSmallBuckets];
        if (se > sb)
            k_selinv_front<<<se - sb, 256, 0, st>>>(D.fronts, D.small_list + sb, D.relmap, Ls, Zs,
                                                    Zu, D.zuoff, Yscr, D.yoff);
        const WorkList& g = S.h_gather[l];
        if (g.nctas > 0)
            k_sel_gather<<<g.nctas, 256, 0, st>>>(D.fronts, S.items + g.off, S.before + g.off,
                                                  g.nitems, D.relmap, Zs, Zu, D.zuoff);
        for (int q = S.h_step_beg[l]; q < S.h_step_beg[l + 1]; ++q) {
            const WorkList& w = S.h_steps[q];
            if (w.nctas > 0) {
                k_sel_y<<<w.nctas, 256, kSelSmem, st>>>(D.fronts, S.items + w.off,
                                                        S.before + w.off, w.nitems, w.step, Ls,
                                                        Dinv, D.dinv_off, Yscr, D.yoff);
                k_sel_zrk<<<w.nctas, 256, kSelSmem, st>>>(D.fronts, S.items + w.off,
                                                          S.before + w.off, w.nitems, w.step, Zs,
                                                          Zu, D.zuoff, Yscr, D.yoff);
            }
            k_sel_zkk<<<w.nitems, 256, kSelSmem, st>>>(D.fronts, S.items + w.off, w.step, Zs,
                                                       Dinv, D.dinv_off, Yscr, D.yoff);
        }
    }
}

void launch_grad_lower(const DevPlan& D, int nnz, const int* perm, const double* Zs,
                       const double* x, double* G, cudaStream_t st) {
    const int blocks = std::max(1, std::min((nnz + 255) / 256, 148 * 8));
    k_grad_lower<<<blocks, 256, 0, st>>>(nnz, D.fronts, D.a_front, D.a_src, D.a_pos, D.rows, perm,
                                         Zs, x, G);
}

template <typename T>
void launch_logdet(const DevPlan& D, const T* Ls, double* partial, double* out, cudaStream_t st) {
    k_logdet_partial<T><<<kLogdetBlocks, 256, 0, st>>>(D.nsuper, D.fronts, Ls, partial);
    k_logdet_final<<<1, 256, 0, st>>>(kLogdetBlocks, partial, out);
}
template void launch_logdet<double>(const DevPlan&, const double*, double*, double*, cudaStream_t);
template void launch_logdet<float>(const DevPlan&, const float*, double*, double*, cudaStream_t);

int logdet_partials() { return kLogdetBlocks; }
int selinv_block() { return kSelBlock; }

void init_selinv() {
    cudaFuncSetAttribute(k_sel_y, cudaFuncAttributeMaxDynamicSharedMemorySize, kSelSmem);
    cudaFuncSetAttribute(k_sel_zrk, cudaFuncAttributeMaxDynamicSharedMemorySize, kSelSmem);
    cudaFuncSetAttribute(k_sel_zkk, cudaFuncAttributeMaxDynamicSharedMemorySize, kSelSmem);
}
int selinv_tile() { return kSelT; }

}  // namespace mdgpu
