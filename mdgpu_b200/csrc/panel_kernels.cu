// One launch per (tree level, 256-column panel) for the pivot panels of the
// large fronts: the whole panel factorization of every large front of the
// level that has this panel, as dependency-ordered row-tile tasks.
//
// Panel p of front f covers pivot tiles [klo, khi) (klo = 4p, at most four
// 64-column tiles).  Task (f, i) owns row tile i >= klo of the panel
// (64 rows x the panel's columns, kept in shared memory for the whole task)
// and computes, for every pivot tile k of the panel below its own row,
//     tile(i, k) -= sum over k' in [klo, k) of X(i, k') X(k, k')'
//     X(i, k)     = tile(i, k) inv(L_kk)'
// A diagonal task (i < khi) stops at k = i: it then forms
//     tile(i, i) -= sum over k' in [klo, i) of X(i, k') X(i, k')'
// (accumulated step by step as its X(i, k') appear), factors it with its
// inverse (potrf_tile_core), stores L_ii and inv(L_ii), and publishes a flag.
// Every task reads the published X(k, .) and inv(L_kk) through L2 (ld.cg:
// never a stale L1 line).  The update products of step k need only the
// blocks X(k, k') that the diagonal task of tile k has written; it counts
// them in a step word per tile as it goes, so every task runs them while the
// diagonal tile is still being factored, and only the TRSM product waits for
// the tile's flag.  Per pivot tile the chain is then one TRSM product, one
// SYRK product and one 64 x 64 factorization.
//
// Tasks take atomic tickets; the list holds every front's diagonal tasks
// first (tile by tile), then the rest, so a task only waits on tasks with a
// lower ticket, held by CTAs that are already running: the waits cannot
// deadlock.  Every wait polls with an iteration limit; on timeout the launch
// is aborted (all waiters leave) and an error code reaches the host.
//
// This replaces, per panel, the 64-wide steps of TRSM, in-panel update and
// diagonal factorization as separate launches (about nine per panel): the
// critical path of a panel is the chain of its diagonal tiles, each one
// TRSM product, one SYRK product and one 64 x 64 factorization behind the
// previous (the in-panel updates run ahead on the step words).  FP32
// factors with tensor-core Schur updates: every task finally writes its rows
// of the finished panel into a panel scratch, row-major (the K-major
// operands of the update), columns past the last pivot column as zeros --
// split for 3xTF32 (hi = X with the low 13 mantissa bits cleared, lo =
// X - hi) or rounded to BF16 -- a diagonal task after publishing its flag,
// so the copy stays off the chain.
//
// FP32 factors: each diagonal tile's pivots are compared with the tile's
// diagonal before its factorization; if one lost more than ten bits to
// cancellation (or is not positive) the tile is factored again in FP64 from
// the same values (the FP64 safeguard for weak pivots; the count is
// reported in status[3]).
#include <cuda_bf16.h>

#include <climits>
#include <cstdio>

#include "device_common.cuh"
#include "kernels.hpp"
#include "tile_ops.cuh"

namespace mdgpu {

namespace {

constexpr int kPanelWaitPolls = 1 << 20;  // ~0.5-1 s at ~1 us per poll
// FP32 diagonal tiles: a pivot d with d^2 < a / kWeakPivotInv (a: the
// tile's diagonal entry before the factorization) sends the tile to FP64
constexpr float kWeakPivotInv = 1024.f;

__device__ __forceinline__ int pn_ld_acquire(const int* p) {
    int v;
    asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ int pn_ld_relaxed(const int* p) {
    int v;
    asm volatile("ld.relaxed.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void pn_st_release(int* p, int v) {
    asm volatile("st.release.gpu.global.b32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// bounded wait for a published word to reach v (a pivot tile's flag: 1; a
// step count); false = aborted (this wait ran out, or another one did)
__device__ bool pn_wait(const int* flag, int* abort_flag, int* err, int v = 1) {
    for (int it = 0; it < kPanelWaitPolls; ++it) {
        if (pn_ld_acquire(flag) >= v) return true;
        if (pn_ld_relaxed(abort_flag)) return false;
        if (it > 8) __nanosleep(it < 256 ? 32 : 256);
    }
    atomicExch(abort_flag, 1);
    atomicExch(err, 3);
    return false;
}

// 64 x 64 operand block into registers: Bs[q][c] = src[c + q ld] for c <
// nrows (zero beyond), through L2; thread t holds elements t + 256 u.
template <typename T>
__device__ __forceinline__ void pn_load_block(T (&pre)[16], const T* __restrict__ src, int64_t ld,
                                              int nrows) {
#pragma unroll
    for (int u = 0; u < 16; ++u) {
        const int idx = threadIdx.x + 256 * u;
        const int q = idx >> 6, c = idx & 63;
        pre[u] = c < nrows ? __ldcg(src + c + (int64_t)q * ld) : T(0);
    }
}
template <typename T>
__device__ __forceinline__ void pn_store_block(T* Bs, const T (&pre)[16]) {
#pragma unroll
    for (int u = 0; u < 16; ++u) Bs[threadIdx.x + 256 * u] = pre[u];
}

// one 64-column block of the task's row block (rows r < nrows, columns cc <
// ncols) to the L panel
template <typename T>
__device__ __forceinline__ void pn_write_block(const T* Xk, T* dst, int64_t ldl, int nrows,
                                               int ncols) {
    for (int idx = threadIdx.x; idx < kTile * kTile; idx += 256) {
        const int q = idx >> 6, r = idx & 63;
        if (r < nrows && q < ncols) dst[r + (int64_t)q * ldl] = Xk[idx];
    }
}

// The task's rows of the finished panel (read back from the L store, which
// this CTA wrote: zeros above the diagonal and past the last pivot column)
// into the panel scratch for the tensor-core Schur update, row-major (a
// kScrCols-wide row, this panel's kPanel columns from column kofs: the
// K-major operand layout), all kPanel columns (zeros past the last pivot
// column):
//   mode 1 (3xTF32): hi = x with the low 13 mantissa bits cleared, lo =
//          x - hi; hi rows from the front's base, lo rows mpad further;
//   mode 2 (BF16): x rounded to BF16 (nearest even), one copy.
// 32-column blocks go through buf (64 x 33 floats) so the global reads run
// down columns and the writes along rows.  ps: the front's scratch base;
// row0: the task's first row.
__device__ __forceinline__ void pn_split_rows(const float* rowp, int64_t ldl, int nrows,
                                              int ncols, float* ps, int row0, int kofs, int mpad,
                                              int mode, float* buf) {
    for (int cb = 0; cb < kPanel; cb += 32) {
        __syncthreads();  // buf free
        for (int idx = threadIdx.x; idx < kTile * 32; idx += 256) {
            const int q = idx >> 6, r = idx & 63;
            buf[r * 33 + q] = (r < nrows && cb + q < ncols) ? rowp[r + (int64_t)(cb + q) * ldl]
                                                             : 0.f;
        }
        __syncthreads();
        for (int idx = threadIdx.x; idx < kTile * 32; idx += 256) {
            const int r = idx >> 5, q = idx & 31;
            if (r >= nrows) continue;
            const float x = buf[r * 33 + q];
            const int64_t e = (int64_t)(row0 + r) * kScrCols + kofs + cb + q;
            if (mode == 2) {
                reinterpret_cast<__nv_bfloat16*>(ps)[e] = __float2bfloat16_rn(x);
            } else {
                const float h = __uint_as_float(__float_as_uint(x) & 0xffffe000u);
                ps[e] = h;
                ps[e + (int64_t)mpad * kScrCols] = x - h;
            }
        }
    }
}

}  // namespace

// shared memory: the row block (kPanel columns x 64 rows), then one operand
// block, which the diagonal factorization reuses as its S and W
template <typename T>
constexpr size_t panel_smem_bytes() {
    return ((size_t)kPanel * kTile + 2 * (size_t)kTile * kPotrfLD) * sizeof(T);
}

template <typename T>
__global__ void __launch_bounds__(256, sizeof(T) == 4 ? 2 : 1)
    k_panel(const FrontDesc* __restrict__ fronts, const int2* __restrict__ tasks, int ntasks,
            int panel, int* __restrict__ counter, int* __restrict__ flags,
            int* __restrict__ steps, int* __restrict__ abort_flag, int* __restrict__ err,
            const int64_t* __restrict__ dinv_off, T* __restrict__ Ls, T* __restrict__ Dinv,
            float* __restrict__ pscr, const int64_t* __restrict__ pscr_off, int split_mode,
            int* __restrict__ status) {
    constexpr int TB = kTile, PT = kPanel / kTile, LDS = kPotrfLD;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* Xs = reinterpret_cast<T*>(smem_raw);  // row block: column q at Xs + q * TB
    T* Bs = Xs + (size_t)kPanel * TB;        // operand block; S and W of the factorization
    __shared__ int s_task, s_ok;
    const int tid = threadIdx.x;
    if (tid == 0) s_task = atomicAdd(counter, 1);
    __syncthreads();
    if (s_task >= ntasks) {  // counter not cleared: refuse rather than read past the list
        if (tid == 0) atomicExch(err, 4);
        return;
    }
    const int2 tk = tasks[s_task];
    const int s = tk.x, i = tk.y;
    const FrontDesc f = fronts[s];
    const int nt1 = tiles_l(f.c, TB);
    const int klo = panel * PT, khi = min(klo + PT, nt1);
    const bool diag = i < khi;
    const int kend = diag ? i : khi;  // steps [klo, kend)
    const TileRange ti = tile_range(i, f.m, f.c, TB);
    const int col0 = klo * TB;
    const int ncol = (diag ? min((i + 1) * TB, f.c) : min(khi * TB, f.c)) - col0;
    const int64_t tile0 = dinv_off[s] / (TB * TB);  // flag of pivot tile k: flags[tile0 + k]
    T* rowp = Ls + f.loff + ti.start + (int64_t)col0 * f.ldl;
    float* ps = nullptr;  // the front's panel scratch (row-major), if any
    const int mpad = panel_mpad(f.m);
    if constexpr (sizeof(T) == 4)
        if (pscr && split_mode) ps = pscr + pscr_off[s];

    for (int idx = tid; idx < kPanel * TB; idx += 256) {
        const int q = idx >> 6, r = idx & 63;
        Xs[idx] = (r < ti.size && q < ncol) ? rowp[r + (int64_t)q * f.ldl] : T(0);
    }
    const int r0 = (tid & 15) * 4, c0 = (tid >> 4) * 4;
    T accd[4][4];  // diagonal task: sum of X(i, k) X(i, k)' so far
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) accd[a][b] = T(0);

    // tid 0 waits for a word to reach v; false (uniform) = aborted
    auto wait_word = [&](const int* w, int v) -> bool {
        if (tid == 0) s_ok = pn_wait(w, abort_flag, err, v) ? 1 : 0;
        __syncthreads();
        return s_ok != 0;
    };
    for (int k = klo; k < kend; ++k) {
        const int ksz = min(TB, f.c - k * TB);
        const T* Lk = Ls + f.loff + k * TB;  // rows of pivot tile k
        const T* Dk = Dinv + dinv_off[s] + (int64_t)k * TB * TB;
        const int nupd = k - klo;
        T* Xk = Xs + (size_t)(k - klo) * TB * TB;
        T pre[16];
        T acc[4][4];
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
            for (int b = 0; b < 4; ++b) acc[a][b] = T(0);
        // tile(i, k) -= X(i, k') X(k, k')' over the panel's earlier tiles,
        // each block once the diagonal task of tile k has counted it in (the
        // next block loads during a product)
        for (int j = 0; j < nupd; ++j) {
            if (j == 0) {
                if (!wait_word(steps + tile0 + k, 1)) return;
                pn_load_block(pre, Lk + (int64_t)col0 * f.ldl, f.ldl, ksz);
            }
            __syncthreads();  // the previous product is done with Bs
            pn_store_block(Bs, pre);
            if (j + 1 < nupd) {
                if (!wait_word(steps + tile0 + k, j + 2)) return;
                pn_load_block(pre, Lk + (int64_t)(col0 + (j + 1) * TB) * f.ldl, f.ldl, ksz);
            }
            __syncthreads();
            tile_gemm_nt_add<T, TB>(Xs + (size_t)j * TB * TB, Bs, acc);
        }
        // the TRSM product waits for the diagonal tile
        if (!wait_word(flags + tile0 + k, 1)) return;
        pn_load_block(pre, Dk, TB, TB);
        __syncthreads();
        if (nupd > 0) {
#pragma unroll
            for (int a = 0; a < 4; ++a)
#pragma unroll
                for (int b = 0; b < 4; ++b) Xk[(c0 + b) * TB + r0 + a] -= acc[a][b];
        }
        pn_store_block(Bs, pre);  // inv(L_kk): Bs[q][c] = inv(L_kk)[c][q]
        __syncthreads();
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
            for (int b = 0; b < 4; ++b) acc[a][b] = T(0);
        tile_gemm_nt_add<T, TB>(Xk, Bs, acc);  // X(i, k) = tile(i, k) inv(L_kk)'
        __syncthreads();
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
            for (int b = 0; b < 4; ++b) {
                const bool in = r0 + a < ti.size && c0 + b < ksz;
                Xk[(c0 + b) * TB + r0 + a] = in ? acc[a][b] : T(0);
            }
        __syncthreads();
        pn_write_block(Xk, rowp + (int64_t)(k - klo) * TB * f.ldl, f.ldl, ti.size, ksz);
        if (diag) {
            // X(i, k) counted in for the tasks' step-i updates
            __threadfence();
            __syncthreads();
            if (tid == 0) pn_st_release(steps + tile0 + i, k - klo + 1);
            tile_gemm_nt_add<T, TB>(Xk, Xk, accd);
        }
    }
    // columns of the panel this task's rows hold (beyond: zeros in the split)
    const int pcols = min(kPanel, f.c - col0);
    if (!diag) {
        if constexpr (sizeof(T) == 4)
            if (ps) pn_split_rows(rowp, f.ldl, ti.size, pcols, ps, ti.start, (panel & 1) * kPanel, mpad,
                              split_mode, Bs);
        return;
    }

    // diagonal tile (i, i): update, factor with its inverse, store, publish
    T* S = Bs;
    T* W = Bs + TB * LDS;
    const int n = ti.size;
    const T* Xi = Xs + (size_t)(i - klo) * TB * TB;
    const int col0g = f.first_col + i * TB;
    __syncthreads();  // every reader of Bs and of the X blocks is done
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) {
            const int r = r0 + a, c = c0 + b;
            T v = (r == c) ? T(1) : T(0);
            if (r < n && c < n) v = r >= c ? Xi[c * TB + r] - accd[a][b] : T(0);
            S[r + c * LDS] = v;
        }
    T* base = Ls + f.loff + i * TB + (int64_t)(i * TB) * f.ldl;
    T* Di = Dinv + dinv_off[s] + (int64_t)i * TB * TB;
    bool redo64 = false;
    if constexpr (sizeof(T) == 4) {
        // FP32 pivots checked against the tile's diagonal before the
        // factorization: a pivot that lost more than ten bits to
        // cancellation (d^2 < a / 1024), or a non-positive one, and the tile
        // is factored again in FP64 from the same updated values
        __shared__ int s_stat;
        if (tid == 0) s_stat = INT_MAX;
        __syncthreads();
        const float dpre = tid < n ? S[tid * (LDS + 1)] : 1.f;
        potrf_tile_core<T, TB>(S, W, n, col0g, &s_stat);
        bool weak = false;
        if (tid < n) {
            const float d = S[tid * (LDS + 1)];
            weak = !(d * d >= dpre * (1.f / kWeakPivotInv));
        }
        redo64 = __syncthreads_or(weak || (tid == 0 && s_stat != INT_MAX)) != 0;
        if (redo64) {
            double sd[4][4];
#pragma unroll
            for (int a = 0; a < 4; ++a)
#pragma unroll
                for (int b = 0; b < 4; ++b) {
                    const int r = r0 + a, c = c0 + b;
                    double v = (r == c) ? 1.0 : 0.0;
                    if (r < n && c < n)
                        v = r >= c ? (double)Xi[c * TB + r] - (double)accd[a][b] : 0.0;
                    sd[a][b] = v;
                }
            __syncthreads();  // the row block and S, W are reused below
            double* S64 = reinterpret_cast<double*>(Xs);  // 2 TB kPotrfLD doubles fit in
            double* W64 = S64 + TB * LDS;                 // the row block + operand block
#pragma unroll
            for (int a = 0; a < 4; ++a)
#pragma unroll
                for (int b = 0; b < 4; ++b) S64[(r0 + a) + (c0 + b) * LDS] = sd[a][b];
            potrf_tile_core<double, TB>(S64, W64, n, col0g, status);
            for (int idx = tid; idx < TB * TB; idx += 256) {
                const int j = idx >> 6, r = idx & 63;
                const bool in = r < n && j < n && r >= j;
                if (in) base[r + (int64_t)j * f.ldl] = (T)S64[r + j * LDS];
                Di[idx] = in ? (T)W64[r + j * LDS] : T(0);
            }
            if (tid == 0) atomicAdd(status + 3, 1);
        }
    } else {
        potrf_tile_core<T, TB>(S, W, n, col0g, status);
    }
    if (!redo64)
        for (int idx = tid; idx < TB * TB; idx += 256) {
            const int j = idx >> 6, r = idx & 63;
            const bool in = r < n && j < n && r >= j;
            if (in) base[r + (int64_t)j * f.ldl] = S[r + j * LDS];
            Di[idx] = in ? W[r + j * LDS] : T(0);
        }
    __threadfence();
    __syncthreads();
    if (tid == 0) pn_st_release(flags + tile0 + i, 1);
    // the split for the Schur update, after the flag: off the panel's chain
    if constexpr (sizeof(T) == 4)
        if (ps) pn_split_rows(rowp, f.ldl, ti.size, pcols, ps, ti.start, (panel & 1) * kPanel, mpad,
                              split_mode, Bs);
}

template <typename T>
void launch_panel(const DevPlan& D, const PanelOp& op, T* Ls, T* Dinv, int* status,
                  int split_mode, cudaStream_t st) {
    int* counter = D.fsync + op.counter;
    int* flags = D.fsync + D.fsync_flags;
    int* abort_flag = D.fsync + D.fsync_flags + D.nflags_factor;
    int* steps = abort_flag + 1;
    k_panel<T><<<op.ntasks, 256, panel_smem_bytes<T>(), st>>>(
        D.fronts, D.psched.tasks + op.toff, op.ntasks, op.arg, counter, flags, steps, abort_flag,
        status + 1, D.dinv_off, Ls, Dinv, split_mode ? D.pscr : nullptr, D.pscr_off, split_mode,
        status);
}

template void launch_panel<float>(const DevPlan&, const PanelOp&, float*, float*, int*, int,
                                  cudaStream_t);
template void launch_panel<double>(const DevPlan&, const PanelOp&, double*, double*, int*, int,
                                   cudaStream_t);

void init_panel_kernels() {
    cudaFuncSetAttribute(k_panel<float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)panel_smem_bytes<float>());
    cudaFuncSetAttribute(k_panel<double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)panel_smem_bytes<double>());
}

}  // namespace mdgpu
