// Supernodal triangular solves L y = b (forward, leaves to root) and
// L' x = y (backward, root to leaves) on the panel storage of the factor.
//
// Forward is multifrontal like the factor: supernode s forms its front vector
// f (m_s x nrhs) from the right-hand side rows of its pivot columns and the
// update parts of its children's front vectors (pulled child by child, so the
// sums are deterministic), solves with the diagonal block, and leaves
// f[c:m] - L21 y as its own update part.  Backward reads the already final
// solution entries of its update rows (ancestors) directly.
//
// Small fronts: one CTA per front.  Large fronts: tiled, one launch per
// 64-row block of the diagonal block, many CTAs per launch; every CTA applies
// the block's inverse (stored by the factorization) redundantly -- a 64 x 64
// product, no serial substitution -- so no launch needs a second phase.
#include <algorithm>

#include "device_common.cuh"
#include "kernels.hpp"

namespace mdgpu {

// Front vector of supernode s: rows fv_off[s] .. fv_off[s] + m - 1 of one
// array whose row holds the nrhs right-hand sides side by side, so row r,
// right-hand side q is front_vec(...)[r * nrhs + q].
template <typename TV>
__device__ inline TV* front_vec(TV* fv, const int64_t* fv_off, int s, int nrhs) {
    return fv + fv_off[s] * nrhs;
}

// ---------------------------------------------------------------------------
// one launch per level and direction: dependency-ordered tile tasks
//
// Each CTA takes the next task by an atomic ticket, so every task that
// started before it holds a lower ticket; the task lists are ordered so that
// a task only waits for tasks earlier in its list, hence for CTAs that are
// already resident, and the waits cannot deadlock.  A pivot tile publishes
// its solution values and then a flag (release); a dependent task polls the
// flag (acquire) with an iteration limit, after which the solve is aborted
// (every waiter leaves) and the error word is set for the host.
// ---------------------------------------------------------------------------

constexpr int kSolveWaitPolls = 1 << 18;  // ~0.1-0.3 s at ~1 us per poll
constexpr int kWarpSolveRhs = 4;   // right-hand sides per pass of the warp path
constexpr int kSolvePassRhs = 32;  // right-hand sides per pass of the solve launches

__device__ __forceinline__ int ld_acquire_gpu(const int* p) {
    int v;
    asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ int ld_relaxed_gpu(const int* p) {
    int v;
    asm volatile("ld.relaxed.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release_gpu(int* p, int v) {
    asm volatile("st.release.gpu.global.b32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
// load of a value another CTA of this launch published (ordered after the
// acquire by the CTA barrier; never served from this SM's L1)
__device__ __forceinline__ double ld_shared_value(const double* p) {
    double v;
    asm volatile("ld.relaxed.gpu.global.f64 %0, [%1];" : "=d"(v) : "l"(p) : "memory");
    return v;
}

__device__ bool wait_flag(const int* flag, int target, int* abort_flag, int* err) {
    for (int it = 0; it < kSolveWaitPolls; ++it) {
        if (ld_acquire_gpu(flag) >= target) return true;
        if (ld_relaxed_gpu(abort_flag)) return false;
        __nanosleep(64);
    }
    atomicExch(abort_flag, 1);
    atomicOr(err, 1);
    return false;
}

// Published pivot-tile values: every slot starts as the all-ones bit pattern
// (a NaN that arithmetic never produces), and a producer stores final values
// only (aligned 8-byte stores are single-copy atomic), so a consumer that
// sees no sentinel has the data: one round trip instead of flag then data.
// All threads poll together (uniform result): the warps that hold slot
// elements spin on their own elements (a warp vote per round, no block
// barrier, a short sleep and an abort check every 32 rounds), the others go
// straight to the closing barrier; iteration limit as wait_flag.
__device__ __forceinline__ double ld_relaxed_f64(const double* p) {
    double v;
    asm volatile("ld.relaxed.gpu.global.f64 %0, [%1];" : "=d"(v) : "l"(p) : "memory");
    return v;
}
// every publication goes through here: a NaN that carries the sentinel's
// all-ones pattern (a right-hand side's own payload passed along) is
// published as the default NaN, so a slot is never read as unpublished once
// written
__device__ __forceinline__ void st_relaxed_f64(double* p, double v) {
    if (__double_as_longlong(v) == -1ll) v = __longlong_as_double(0x7ff8000000000000ll);
    asm volatile("st.relaxed.gpu.global.f64 [%0], %1;" ::"l"(p), "d"(v) : "memory");
}
__device__ __forceinline__ bool is_unpublished(double v) {
    return __double_as_longlong(v) == -1ll;
}
__device__ bool poll_published(double* dst, const double* src, int nk, int nrhs, int* abort_flag,
                               int* err) {
    constexpr int T = kTile;
    const int total = T * nrhs, lane = threadIdx.x & 31;  // total: a multiple of 64
    bool ok = true;
    for (int base = threadIdx.x & ~31; ok && base < total; base += blockDim.x) {
        const int e = base + lane;
        const bool need = (e & (T - 1)) < nk;
        double v = 0.0;
        for (int it = 0;; ++it) {
            if (need) v = ld_relaxed_f64(src + e);
            if (__all_sync(0xffffffffu, !need || !is_unpublished(v))) break;
            if (it + 1 >= kSolveWaitPolls) {
                if (lane == 0) {
                    atomicExch(abort_flag, 1);
                    atomicOr(err, 1);
                }
                ok = false;
                break;
            }
            if ((it & 31) == 31) {
                const int a = lane == 0 ? ld_relaxed_gpu(abort_flag) : 0;
                if (__shfl_sync(0xffffffffu, a, 0)) {
                    ok = false;
                    break;
                }
                __nanosleep(32);
            }
        }
        if (ok) dst[e] = need ? v : 0.0;
    }
    return __syncthreads_and(ok);
}

template <typename TL>
__device__ __forceinline__ void cp_async_elem(TL* dst, const TL* src) {
    const uint32_t d = static_cast<uint32_t>(__cvta_generic_to_shared(dst));
    if constexpr (sizeof(TL) == 4)
        asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(d), "l"(src) : "memory");
    else
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit_group() {
    asm volatile("cp.async.commit_group;" ::: "memory");
}
template <int N>
__device__ __forceinline__ void cp_async_wait_groups() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// Stage layout of a 64 x 64 block of L (or of a diagonal inverse): column-
// major, columns of blk_ld elements (a multiple of 16 bytes), copied in
// 16-byte chunks from the 16-byte boundary at or below the block's first
// row, so row r of column c sits at c * blk_ld + d + r with d =
// blk_off(first row).  Rows past the block and columns past nc are
// zero-filled by the copies themselves (source size below 16 bytes).  The L
// store's columns start on 32-byte boundaries (ldl a multiple of 8, front
// offsets of 32), the inverses' on 64 * 64 elements.
template <typename TL>
__host__ __device__ constexpr int blk_ld() {
    return kTile + 16 / (int)sizeof(TL);
}
template <typename TL>
__device__ __forceinline__ int blk_off(int start) {
    return start & (16 / (int)sizeof(TL) - 1);
}
// rows start .. start + nr - 1 and columns 0 .. nc - 1 of the matrix at src
// (column stride ld)
template <typename TL>
__device__ __forceinline__ void load_block_async(TL* dst, const TL* src, int64_t ld, int start,
                                                 int nr, int nc) {
    constexpr int E = 16 / (int)sizeof(TL), LDB = blk_ld<TL>(), CH = LDB / E;
    const int r0 = start - blk_off<TL>(start);
    for (int e = threadIdx.x; e < kTile * CH; e += blockDim.x) {
        const int col = e / CH, u = e - col * CH;
        const int row = r0 + u * E;
        const int bytes = col < nc ? min(max(start + nr - row, 0), E) * (int)sizeof(TL) : 0;
        const TL* sp = bytes ? src + row + (int64_t)col * ld : src;
        const uint32_t da = static_cast<uint32_t>(__cvta_generic_to_shared(dst + col * LDB + u * E));
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(da), "l"(sp), "r"(bytes)
                     : "memory");
    }
}

// ---------------------------------------------------------------------------
// large-front tile tasks: a pipeline of `stg` stages streams the L blocks a
// task multiplies, each with the vector block it is multiplied by (a pivot
// tile's published solution, or gathered solution rows), by cp.async; the
// block in use is consumed while the next ones load.  Published vectors come
// through L2 (16-byte cp.async.cg); a stage whose copy still holds a
// sentinel falls back to polling that slot.
// ---------------------------------------------------------------------------

template <typename TL>
__host__ __device__ constexpr int level_stages(int nrhs) {
    return 2;
}

// shared memory: diagonal inverse block, stg L blocks, stg vector blocks, a
// vector, the quarter reduction, the gather's row indices
template <typename TL, typename TV>
__host__ __device__ constexpr size_t level_smem_bytes(int nrhs) {
    return (((1 + (size_t)level_stages<TL>(nrhs)) * kTile * blk_ld<TL>() * sizeof(TL) + 15) / 16) * 16 +
           (((size_t)level_stages<TL>(nrhs) + 1) * kTile * nrhs + 4 * kTile) * sizeof(TV) +
           (size_t)SolveScheduleHost::kGatherTiles * kTile * sizeof(int);
}

template <typename TL, typename TV>
struct LevelSmem {
    TL* Dk;   // T x LD
    TL* Lst;  // stg x T x LD
    TV* Vst;  // stg x T x nrhs
    TV* Y;    // T x nrhs
    TV* red;  // 4 x T
    int* idx; // kGatherTiles x T
    int stg;
    __device__ explicit LevelSmem(int nrhs) {
        constexpr int T = kTile, LD = blk_ld<TL>();
        extern __shared__ __align__(16) unsigned char smem_raw[];
        stg = level_stages<TL>(nrhs);
        Dk = reinterpret_cast<TL*>(smem_raw);
        Lst = Dk + T * LD;
        Vst = reinterpret_cast<TV*>(smem_raw +
                                    (((1 + (size_t)stg) * T * LD * sizeof(TL) + 15) / 16) * 16);
        Y = Vst + (size_t)stg * T * nrhs;
        red = Y + T * nrhs;
        idx = reinterpret_cast<int*>(red + 4 * T);
    }
    __device__ TL* lb(int p) const { return Lst + (p % stg) * kTile * blk_ld<TL>(); }
    __device__ TV* vb(int p, int nrhs) const { return Vst + (size_t)(p % stg) * kTile * nrhs; }
};

__device__ __forceinline__ void cp_async_wait_stages(int stg) {
    if (stg >= 3)
        cp_async_wait_groups<2>();
    else
        cp_async_wait_groups<1>();
}

// a published T x nrhs slot into a stage (16-byte copies through L2; T * nrhs
// is even and slots start on 16 bytes)
__device__ __forceinline__ void load_slot_async(double* dst, const double* src, int nrhs) {
    for (int q = threadIdx.x; q < kTile * nrhs / 2; q += blockDim.x) {
        const uint32_t da = static_cast<uint32_t>(__cvta_generic_to_shared(dst + 2 * q));
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(da), "l"(src + 2 * q)
                     : "memory");
    }
}

// After the stage's copy landed: rows >= nk zeroed, rows < nk checked for
// the sentinel; an unpublished row sends the CTA to poll the slot.  Uniform
// result; false = the solve was aborted.
__device__ __forceinline__ bool settle_slot(double* v, const double* src, int nk, int nrhs,
                                            int* abort_flag, int* err) {
    bool mine = true;
    for (int e = threadIdx.x; e < kTile * nrhs; e += blockDim.x) {
        if ((e & (kTile - 1)) >= nk)
            v[e] = 0.0;
        else if (is_unpublished(v[e]))
            mine = false;
    }
    if (__syncthreads_and(mine)) return true;
    return poll_published(v, src, nk, nrhs, abort_flag, err);
}

// Forward, task (s, i0 | cnt << 16): row tiles i0 .. i0 + cnt - 1 of front s.
// Each gathers its rows of the front vector (right-hand side on the pivot
// rows plus the children's update rows, child by child; one tile ahead) and
// accumulates acc = sum_{k < min(i, nt1)} L(i, k) y_k over the pivot tiles.
// A pivot tile (i0 < nt1, cnt = 1) then solves y_i = inv(L_ii) (f_i - acc)
// into the solution and publishes it; an update tile leaves f_i - acc in the
// front vector for the parent.  Threads: r = row in the tile; one
// right-hand side splits the 64 columns of a block over four column phases
// held by lanes of one warp, several split the right-hand sides (NQ per
// thread).
template <typename TL, typename TV, int NQ>
__device__ void fwd_tile_task(int2 tk, const FrontDesc* __restrict__ fronts,
                              double* __restrict__ pub, int* __restrict__ abort_flag,
                              int* __restrict__ err, const int64_t* __restrict__ fv_off,
                              const int* __restrict__ amap_off, const int* __restrict__ amap_row,
                              const int* __restrict__ amap_ent,
                              const int64_t* __restrict__ dinv_off, const TL* __restrict__ Ls,
                              const TL* __restrict__ Dinv, TV* __restrict__ xp,
                              TV* __restrict__ fv, int n, int nrhs) {
    static_assert(sizeof(TV) == 8, "solve vectors are double");
    constexpr int T = kTile, LD = blk_ld<TL>();
    const LevelSmem<TL, TV> sm(nrhs);
    const bool lsplit = nrhs == 1;
    // one right-hand side: r = row, g = column phase (columns g, g + 4, ...),
    // the four phases of a row in one warp (rows 8w .. 8w + 7 of warp w), so
    // a row's sum is two shuffles; several: r = row, g = quarter of the
    // right-hand sides
    const int tid = threadIdx.x;
    const int r = lsplit ? 8 * (tid >> 5) + (tid & 7) : tid & (T - 1);
    const int g = lsplit ? (tid >> 3) & 3 : tid >> 6;
    const int s = tk.x, i0 = tk.y & 0xffff, cnt = tk.y >> 16;
    const FrontDesc F = fronts[s];
    const int nt1 = tiles_l(F.c, T);
    const bool pivot = i0 < nt1;
    const int kend = pivot ? i0 : nt1;  // L blocks per tile
    const int P = cnt * kend;
    const TL* L = Ls + F.loff;
    double* pb = pub + (dinv_off[s] / (T * T)) * T * nrhs;  // this front's pivot tiles
    TV* f = front_vec(fv, fv_off, s, nrhs);
    // the row offset of this task's blocks in their stage columns (every row
    // tile of a task starts at the same residue: 0 for a pivot tile, c for
    // update tiles)
    const int db = blk_off<TL>(tile_range(i0, F.m, F.c, T).start);
    const int aoff = amap_off[s];
    // rows of tile i of the front vector into v (this thread's share)
    auto gather_rows = [&](int i, TV (&v)[NQ]) {
        const TileRange ti = tile_range(i, F.m, F.c, T);
        const int R = ti.start + r;
        int e0 = 0, e1 = 0;
        if (r < ti.size) {
            e0 = amap_row[aoff + R];
            e1 = amap_row[aoff + R + 1];
        }
#pragma unroll
        for (int j = 0; j < NQ; ++j) {
            const int q = lsplit ? 0 : g + 4 * j;
            TV x = TV(0);
            if (r < ti.size && q < nrhs && (!lsplit || (g == 0 && j == 0))) {
                if (R < F.c) x = xp[F.first_col + R + (int64_t)q * n];
                for (int e = e0; e < e1; ++e) x += __ldcg(fv + (int64_t)amap_ent[e] * nrhs + q);
            }
            v[j] = x;
        }
    };
    auto issue = [&](int p) {
        if (p < P) {
            const int i = i0 + p / kend, k = p % kend;
            const TileRange ti = tile_range(i, F.m, F.c, T);
            load_block_async(sm.lb(p), L + (int64_t)k * T * F.ldl, F.ldl, ti.start, ti.size,
                             min(T, F.c - k * T));
            load_slot_async(sm.vb(p, nrhs), pb + (int64_t)k * T * nrhs, nrhs);
        }
        cp_async_commit_group();
    };
    if (pivot) {
        const TileRange ti = tile_range(i0, F.m, F.c, T);
        load_block_async(sm.Dk, Dinv + dinv_off[s] + (int64_t)i0 * T * T, T, 0, ti.size, ti.size);
    }
    for (int p = 0; p < sm.stg - 1; ++p) issue(p);
    TV fcur[NQ], fnext[NQ], acc[NQ];
    gather_rows(i0, fcur);
#pragma unroll
    for (int j = 0; j < NQ; ++j) {
        fnext[j] = TV(0);
        acc[j] = TV(0);
    }
    if (cnt > 1) gather_rows(i0 + 1, fnext);
    bool ok = true;
    for (int p = 0; p < P; ++p) {
        issue(p + sm.stg - 1);
        cp_async_wait_stages(sm.stg);
        __syncthreads();
        const int i = i0 + p / kend, k = p % kend;
        TV* Yk = sm.vb(p, nrhs);
        if (!settle_slot(Yk, pb + (int64_t)k * T * nrhs, min(T, F.c - k * T), nrhs, abort_flag,
                         err)) {
            ok = false;
            break;
        }
        const TL* B = sm.lb(p);
        if (lsplit) {
#pragma unroll
            for (int l = 0; l < 16; ++l)
                acc[0] += (TV)B[db + r + (g + 4 * l) * LD] * Yk[g + 4 * l];
        } else {
#pragma unroll 4
            for (int l = 0; l < T; ++l) {
                const TV lv = (TV)B[db + r + l * LD];
#pragma unroll
                for (int j = 0; j < NQ; ++j) {
                    const int q = g + 4 * j;
                    if (q < nrhs) acc[j] += lv * Yk[l + T * q];
                }
            }
        }
        if (!pivot && k == kend - 1) {  // update tile i complete: f_i - acc to the front vector
            const TileRange ti = tile_range(i, F.m, F.c, T);
            if (lsplit) {
                TV v = acc[0] + __shfl_xor_sync(0xffffffffu, acc[0], 8);
                v += __shfl_xor_sync(0xffffffffu, v, 16);
                if (g == 0 && r < ti.size) f[ti.start + r] = fcur[0] - v;
            } else if (r < ti.size) {
#pragma unroll
                for (int j = 0; j < NQ; ++j) {
                    const int q = g + 4 * j;
                    if (q < nrhs) f[(int64_t)(ti.start + r) * nrhs + q] = fcur[j] - acc[j];
                }
            }
#pragma unroll
            for (int j = 0; j < NQ; ++j) {
                acc[j] = TV(0);
                fcur[j] = fnext[j];
            }
            if (i + 2 < i0 + cnt) gather_rows(i + 2, fnext);
        }
        if (p + 1 < P) __syncthreads();  // the stages are reused; after the last, nothing is
    }
    cp_async_wait_groups<0>();
    if (!ok || !pivot) return;
    // pivot tile: F = f_i - acc (zero beyond the tile), then y = Dk F
    const TileRange ti = tile_range(i0, F.m, F.c, T);
    TV* Y = sm.Y;
    const TL* Dk = sm.Dk;
    if (lsplit) {
        // one right-hand side, one barrier: the row's phases summed by
        // shuffles, F into sm.Y, then y = Dk F the same way
        TV a = acc[0] + __shfl_xor_sync(0xffffffffu, acc[0], 8);
        a += __shfl_xor_sync(0xffffffffu, a, 16);
        if (g == 0) Y[r] = r < ti.size ? fcur[0] - a : TV(0);
        __syncthreads();
        TV y = TV(0);
#pragma unroll
        for (int l = 0; l < 16; ++l) y += (TV)Dk[r + (g + 4 * l) * LD] * Y[g + 4 * l];
        y += __shfl_xor_sync(0xffffffffu, y, 8);
        y += __shfl_xor_sync(0xffffffffu, y, 16);
        if (g == 0 && r < ti.size) {
            xp[F.first_col + ti.start + r] = y;
            st_relaxed_f64(pb + (int64_t)i0 * T + r, y);
        }
        return;
    }
    __syncthreads();
#pragma unroll
    for (int j = 0; j < NQ; ++j) {
        const int q = g + 4 * j;
        if (q < nrhs) Y[r + T * q] = r < ti.size ? fcur[j] - acc[j] : TV(0);
    }
    __syncthreads();
    {
        TV y[NQ];
#pragma unroll
        for (int j = 0; j < NQ; ++j) y[j] = TV(0);
#pragma unroll 4
        for (int l = 0; l < T; ++l) {
            const TV dv = (TV)Dk[r + l * LD];
#pragma unroll
            for (int j = 0; j < NQ; ++j) {
                const int q = g + 4 * j;
                if (q < nrhs) y[j] += dv * Y[l + T * q];
            }
        }
        if (r < ti.size) {
#pragma unroll
            for (int j = 0; j < NQ; ++j) {
                const int q = g + 4 * j;
                if (q < nrhs) {
                    xp[F.first_col + ti.start + r + (int64_t)q * n] = y[j];
                    st_relaxed_f64(pb + ((int64_t)i0 * nrhs + q) * T + r, y[j]);
                }
            }
        }
    }
}

// Backward, update rows, task (s, j | h << 16): the partial sum
// L(k, j)' x_k over the update row tiles k of chunk h (kGatherTiles tiles;
// x final: ancestors, read through the row list) for pivot column tile j,
// written as a T x nrhs vector for the pivot task to add in chunk order, then
// counted in.  Threads: l = column in the tile, g = quarter.
template <typename TL, typename TV, int NQ>
__device__ void bwd_gather_task(int2 tk, const FrontDesc* __restrict__ fronts,
                                const int* __restrict__ rows, const int* __restrict__ gather_nch,
                                const int* __restrict__ gather_off, int* __restrict__ gcount,
                                const int64_t* __restrict__ dinv_off, const TL* __restrict__ Ls,
                                const TV* __restrict__ xp, TV* __restrict__ part, int n,
                                int nrhs) {
    constexpr int T = kTile, LD = blk_ld<TL>(), GC = SolveScheduleHost::kGatherTiles;
    const LevelSmem<TL, TV> sm(nrhs);
    const int tid = threadIdx.x, l = tid & (T - 1), g = tid >> 6;
    const int s = tk.x, j = tk.y & 0xffff, h = tk.y >> 16;
    const FrontDesc F = fronts[s];
    const int nt1 = tiles_l(F.c, T), NT = nt1 + tiles_l(F.m - F.c, T);
    const TileRange tj = tile_range(j, F.m, F.c, T);
    const bool lsplit = nrhs == 1;
    const TL* Lc = Ls + F.loff + (int64_t)tj.start * F.ldl;
    const int* rw = rows + F.rows_off;
    const int k0 = nt1 + h * GC, P = min(NT, k0 + GC) - k0;
    // update row tiles start at c + 64 u: one row offset for every block
    const int db = blk_off<TL>(F.c);
    // one right-hand side: warp w takes columns 8w .. 8w + 7, lane (c1 =
    // column, q1 = row phase) the rows q1, q1 + 4, ...: conflict-free reads
    // of the 16-byte-column stage layout, the phases summed by shuffles
    const int c1 = 8 * (tid >> 5) + (tid & 7), q1 = (tid >> 3) & 3;
    // the chunk's solution rows (ancestors), then the pipeline
    for (int e = tid; e < P * T; e += blockDim.x) {
        const TileRange tkr = tile_range(k0 + e / T, F.m, F.c, T);
        const int rr = e & (T - 1);
        sm.idx[e] = rr < tkr.size ? rw[tkr.start + rr] : -1;
    }
    __syncthreads();
    // two stages: the L blocks by cp.async; the ancestors' solution rows
    // (written in this launch) through L2 into registers one stage ahead,
    // stored into their stage after the previous stage's products
    static_assert(kTile * kSolvePassRhs % 256 == 0, "whole vector elements per thread");
    constexpr int VPT = kTile * kSolvePassRhs / 256;
    TV pend[VPT];
    auto fetch = [&](int p) {
#pragma unroll
        for (int k = 0; k < VPT; ++k) {
            const int e = tid + 256 * k;
            pend[k] = TV(0);
            if (p < P && e < T * nrhs) {
                const int row = sm.idx[p * T + (e & (T - 1))], q = e / T;
                if (row >= 0) pend[k] = __ldcg(xp + row + (int64_t)q * n);
            }
        }
    };
    auto put = [&](int p) {
        if (p >= P) return;
        TV* v = sm.vb(p, nrhs);
#pragma unroll
        for (int k = 0; k < VPT; ++k) {
            const int e = tid + 256 * k;
            if (e < T * nrhs) v[e] = pend[k];
        }
    };
    auto issue = [&](int p) {
        if (p < P) {
            const TileRange tkr = tile_range(k0 + p, F.m, F.c, T);
            load_block_async(sm.lb(p), Lc, F.ldl, tkr.start, tkr.size, tj.size);
        }
        cp_async_commit_group();
    };
    static_assert(level_stages<TL>(1) == 2, "the gather's vector pipeline has two stages");
    issue(0);
    fetch(0);
    put(0);
    TV acc[NQ];
#pragma unroll
    for (int a = 0; a < NQ; ++a) acc[a] = TV(0);
    for (int p = 0; p < P; ++p) {
        issue(p + 1);
        fetch(p + 1);
        cp_async_wait_groups<1>();
        __syncthreads();
        const TL* Bk = sm.lb(p);
        const TV* X = sm.vb(p, nrhs);
        if (lsplit) {
#pragma unroll
            for (int u = 0; u < 16; ++u)
                acc[0] += (TV)Bk[db + q1 + 4 * u + c1 * LD] * X[q1 + 4 * u];
        } else {
#pragma unroll 4
            for (int r = 0; r < T; ++r) {
                const TV lv = (TV)Bk[db + r + l * LD];
#pragma unroll
                for (int a = 0; a < NQ; ++a) {
                    const int q = g + 4 * a;
                    if (q < nrhs) acc[a] += lv * X[r + T * q];
                }
            }
        }
        __syncthreads();
        put(p + 1);
    }
    cp_async_wait_groups<0>();
    TV* out = part + ((int64_t)gather_off[s] + (int64_t)j * gather_nch[s] + h) * T * nrhs;
    if (lsplit) {
        TV v = acc[0] + __shfl_xor_sync(0xffffffffu, acc[0], 8);
        v += __shfl_xor_sync(0xffffffffu, v, 16);
        if (q1 == 0) out[c1] = v;
    } else {
#pragma unroll
        for (int a = 0; a < NQ; ++a) {
            const int q = g + 4 * a;
            if (q < nrhs) out[l + T * q] = acc[a];
        }
    }
    // count this chunk in for the pivot task (s, j): the CTA's stores, then
    // a device-scope fence, then the increment
    __syncthreads();
    if (tid == 0) {
        __threadfence();
        atomicAdd(gcount + dinv_off[s] / (T * T) + j, 1);
    }
}

// ---------------------------------------------------------------------------
// small fronts: a warp per front, the right-hand sides in passes of NQ
// (kWarpSolveRhs, or one), lane l holding rows l, l + 32, ... (R slots,
// m <= 32 R) of the pass's right-hand sides in registers.  Forward: the
// pivot value is broadcast by a shuffle and every lane updates its rows
// below it; backward: a warp reduction per pivot column (dot product with
// the final rows below it).  No block barriers; the children's update parts
// are summed into a per-warp shared buffer (child by child, deterministic)
// before the rows are taken into registers.
// ---------------------------------------------------------------------------

// Dependency words of the one-launch solve.  Forward: front s starts once
// done[s] (its finished children) reaches its child count, and counts
// itself in at its parent once its update rows are written.  Backward:
// front s starts once done[parent] reaches target[parent] (the parent's
// solution rows are final), and counts one completion of its own once its
// solution rows are written.  Data written inside the launch by other CTAs
// (children's update rows, ancestors' solution rows) are read through L2.
struct FrontDeps {
    int* done;
    const int* target;  // backward only
    int* abort_flag;
    int* err;
};

// Fronts of at most W rows (W = 8, 16, 32) on a group of W lanes of a warp
// (32 / W fronts per warp), one row per lane.  mask: the group's lanes; the
// group's rows of the warp buffer are wbuf[q * 32 + r].
template <int W>
__device__ __forceinline__ unsigned group_mask() {
    return W == 32 ? 0xffffffffu : (((1u << W) - 1u) << ((threadIdx.x & 31) & ~(W - 1)));
}

// the group's first lane waits (bounded) for *word >= target; uniform result
template <int W>
__device__ __forceinline__ bool group_wait(const int* word, int target, const FrontDeps& d,
                                           unsigned mask) {
    int ok = 1;
    if ((threadIdx.x & (W - 1)) == 0) ok = wait_flag(word, target, d.abort_flag, d.err) ? 1 : 0;
    return __shfl_sync(mask, ok, 0, W) != 0;
}
// every lane's stores, a device-scope fence, then one increment of *word
template <int W>
__device__ __forceinline__ void group_signal(int* word, unsigned mask) {
    __threadfence();
    __syncwarp(mask);
    if (word && (threadIdx.x & (W - 1)) == 0) atomicAdd(word, 1);
}

template <typename TL, typename TV, int W, int NQ>
__device__ void fwd_group_front(int s, const FrontDesc& F, const FrontDeps& deps,
                                const FrontDesc* __restrict__ fronts,
                                const int* __restrict__ child, const int* __restrict__ relmap,
                                const int64_t* __restrict__ fv_off, const TL* __restrict__ Ls,
                                TV* __restrict__ xp, TV* __restrict__ out, TV* __restrict__ fv,
                                int n, int nrhs, TV* wbuf) {
    const unsigned mask = group_mask<W>();
    if (!group_wait<W>(deps.done + s, F.child_end - F.child_beg, deps, mask)) return;
    const int r = threadIdx.x & (W - 1);
    const int m = F.m, c = F.c;
    const int64_t ldl = F.ldl;
    const TL* L = Ls + F.loff;
    for (int q0 = 0; q0 < nrhs; q0 += NQ) {
        const int nq = min(NQ, nrhs - q0);
#pragma unroll
        for (int q = 0; q < NQ; ++q)
            if (q < nq && r < m)
                wbuf[q * 32 + r] = r < c ? xp[F.first_col + r + (int64_t)(q0 + q) * n] : TV(0);
        __syncwarp(mask);
        for (int h = F.child_beg; h < F.child_end; ++h) {  // children in order
            const int ch = child[h];
            const FrontDesc g = fronts[ch];
            const int uc = g.m - g.c;
            const TV* w = front_vec(fv, fv_off, ch, nrhs) + g.c * nrhs + q0;
            if (r < uc) {  // uc < m <= W
                const int p = relmap[g.rows_off + g.c + r];
#pragma unroll
                for (int q = 0; q < NQ; ++q)
                    if (q < nq) wbuf[q * 32 + p] += __ldcg(w + r * nrhs + q);
            }
            __syncwarp(mask);
        }
        TV v[NQ];
#pragma unroll
        for (int q = 0; q < NQ; ++q) v[q] = (q < nq && r < m) ? wbuf[q * 32 + r] : TV(0);
        __syncwarp(mask);
        // column j of L for this lane's row, one column ahead of its use
        TV lc = (r > 0 && r < m) ? (TV)L[r] : TV(0), d = (TV)L[0];
        for (int j = 0; j < c; ++j) {
            TV ln = TV(0), dn = TV(1);
            if (j + 1 < c) {
                const TL* cn = L + (j + 1) * ldl;
                dn = (TV)cn[j + 1];
                ln = (r > j + 1 && r < m) ? (TV)cn[r] : TV(0);
            }
            // several right-hand sides: one reciprocal per column
            const TV rd = NQ > 1 ? TV(1) / d : TV(0);
#pragma unroll
            for (int q = 0; q < NQ; ++q) {
                const TV sv = __shfl_sync(mask, v[q], j, W);
                const TV y = NQ > 1 ? sv * rd : sv / d;
                if (r == j)
                    v[q] = y;
                else if (r > j)
                    v[q] -= lc * y;
            }
            lc = ln;
            d = dn;
        }
#pragma unroll
        for (int q = 0; q < NQ; ++q) {
            if (q >= nq || r >= m) continue;
            if (r < c)
                xp[F.first_col + r + (int64_t)(q0 + q) * n] = v[q];
            else
                out[r * nrhs + q0 + q] = v[q];
        }
    }
    group_signal<W>(F.parent >= 0 ? deps.done + F.parent : nullptr, mask);
}

template <typename TL, typename TV, int W, int NQ>
__device__ void bwd_group_front(int s, const FrontDesc& F, const FrontDeps& deps,
                                const int* __restrict__ rows, const TL* __restrict__ Ls,
                                TV* __restrict__ xp, int n, int nrhs) {
    const unsigned mask = group_mask<W>();
    if (F.parent >= 0 && !group_wait<W>(deps.done + F.parent, deps.target[F.parent], deps, mask))
        return;
    const int r = threadIdx.x & (W - 1);
    const int m = F.m, c = F.c;
    const int64_t ldl = F.ldl;
    const TL* L = Ls + F.loff;
    // this lane's row in the solution: a pivot row, else an ancestor's
    const int src = r < c ? F.first_col + r : (r < m ? rows[F.rows_off + r] : 0);
    for (int q0 = 0; q0 < nrhs; q0 += NQ) {
        const int nq = min(NQ, nrhs - q0);
        TV v[NQ];  // y on the pivot rows (x once solved), final x on the others
#pragma unroll
        for (int q = 0; q < NQ; ++q)
            v[q] = (q < nq && r < m) ? __ldcg(xp + src + (int64_t)(q0 + q) * n) : TV(0);
        const int jl = c - 1;
        TV lc = (r > jl && r < m) ? (TV)L[r + jl * ldl] : TV(0), d = (TV)L[jl + jl * ldl];
        for (int j = jl; j >= 0; --j) {
            TV ln = TV(0), dn = TV(1);
            if (j > 0) {
                const TL* cn = L + (j - 1) * ldl;
                dn = (TV)cn[j - 1];
                ln = (r > j - 1 && r < m) ? (TV)cn[r] : TV(0);
            }
            TV p[NQ];
#pragma unroll
            for (int q = 0; q < NQ; ++q) p[q] = lc * v[q];
#pragma unroll
            for (int o = W / 2; o > 0; o >>= 1)
#pragma unroll
                for (int q = 0; q < NQ; ++q) p[q] += __shfl_xor_sync(mask, p[q], o, W);
            if (r == j) {
#pragma unroll
                for (int q = 0; q < NQ; ++q) v[q] = (v[q] - p[q]) / d;
            }
            lc = ln;
            d = dn;
        }
#pragma unroll
        for (int q = 0; q < NQ; ++q)
            if (q < nq && r < c) xp[F.first_col + r + (int64_t)(q0 + q) * n] = v[q];
    }
    group_signal<W>(deps.done + s, mask);
}

// Fronts of 33..160 rows: the same sweeps with the front vector kept in the
// warp's shared buffer (ld MR rows per right-hand side) instead of registers.
template <typename TL, typename TV, int NQ>
__device__ void fwd_warp_front_smem(int s, const FrontDesc& F, const FrontDeps& deps,
                                    const FrontDesc* __restrict__ fronts,
                                    const int* __restrict__ child, const int* __restrict__ relmap,
                                    const int64_t* __restrict__ fv_off, const TL* __restrict__ Ls,
                                    TV* __restrict__ xp, TV* __restrict__ out, TV* __restrict__ fv,
                                    int n, int nrhs, TV* f, int MR) {
    if (!group_wait<32>(deps.done + s, F.child_end - F.child_beg, deps, 0xffffffffu)) return;
    const int lane = threadIdx.x & 31;
    const int m = F.m, c = F.c;
    const int64_t ldl = F.ldl;
    const TL* L = Ls + F.loff;
    for (int q0 = 0; q0 < nrhs; q0 += NQ) {
        const int nq = min(NQ, nrhs - q0);
        for (int r = lane; r < m; r += 32)
#pragma unroll
            for (int q = 0; q < NQ; ++q)
                if (q < nq)
                    f[q * MR + r] = r < c ? xp[F.first_col + r + (int64_t)(q0 + q) * n] : TV(0);
        __syncwarp();
        for (int h = F.child_beg; h < F.child_end; ++h) {  // children in order
            const int ch = child[h];
            const FrontDesc g = fronts[ch];
            const int uc = g.m - g.c;
            const TV* w = front_vec(fv, fv_off, ch, nrhs) + g.c * nrhs + q0;
            const int* rm = relmap + g.rows_off + g.c;
            for (int rr = lane; rr < uc; rr += 32) {
                const int p = rm[rr];
#pragma unroll
                for (int q = 0; q < NQ; ++q)
                    if (q < nq) f[q * MR + p] += __ldcg(w + rr * nrhs + q);
            }
            __syncwarp();
        }
        for (int j = 0; j < c; ++j) {
            const TL* col = L + j * ldl;
            const TV d = (TV)col[j];
            const TV rd = NQ > 1 ? TV(1) / d : TV(0);  // several right-hand sides
            TV y[NQ];
#pragma unroll
            for (int q = 0; q < NQ; ++q) y[q] = NQ > 1 ? f[q * MR + j] * rd : f[q * MR + j] / d;
            if (lane == (j & 31)) {
#pragma unroll
                for (int q = 0; q < NQ; ++q)
                    if (q < nq) xp[F.first_col + j + (int64_t)(q0 + q) * n] = y[q];
            }
            for (int r = j + 1 + lane; r < m; r += 32) {
                const TV l = (TV)col[r];
#pragma unroll
                for (int q = 0; q < NQ; ++q) f[q * MR + r] -= l * y[q];
            }
            __syncwarp();
        }
        for (int r = c + lane; r < m; r += 32)
#pragma unroll
            for (int q = 0; q < NQ; ++q)
                if (q < nq) out[r * nrhs + q0 + q] = f[q * MR + r];
        __syncwarp();
    }
    group_signal<32>(F.parent >= 0 ? deps.done + F.parent : nullptr, 0xffffffffu);
}

template <typename TL, typename TV, int NQ>
__device__ void bwd_warp_front_smem(int s, const FrontDesc& F, const FrontDeps& deps,
                                    const int* __restrict__ rows, const TL* __restrict__ Ls,
                                    TV* __restrict__ xp, int n, int nrhs, TV* x, int MR) {
    if (F.parent >= 0 &&
        !group_wait<32>(deps.done + F.parent, deps.target[F.parent], deps, 0xffffffffu))
        return;
    const int lane = threadIdx.x & 31;
    const int m = F.m, c = F.c;
    const int64_t ldl = F.ldl;
    const TL* L = Ls + F.loff;
    const int* rw = rows + F.rows_off;
    for (int q0 = 0; q0 < nrhs; q0 += NQ) {
        const int nq = min(NQ, nrhs - q0);
        for (int r = lane; r < m; r += 32) {
            const int src = r < c ? F.first_col + r : rw[r];
#pragma unroll
            for (int q = 0; q < NQ; ++q)
                x[q * MR + r] = q < nq ? __ldcg(xp + src + (int64_t)(q0 + q) * n) : TV(0);
        }
        __syncwarp();
        for (int j = c - 1; j >= 0; --j) {
            const TL* col = L + j * ldl;
            TV p[NQ];
#pragma unroll
            for (int q = 0; q < NQ; ++q) p[q] = TV(0);
            for (int r = j + 1 + lane; r < m; r += 32) {
                const TV l = (TV)col[r];
#pragma unroll
                for (int q = 0; q < NQ; ++q) p[q] += l * x[q * MR + r];
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1)
#pragma unroll
                for (int q = 0; q < NQ; ++q) p[q] += __shfl_xor_sync(0xffffffffu, p[q], o);
            const TV d = (TV)col[j];
            if (lane == (j & 31)) {
#pragma unroll
                for (int q = 0; q < NQ; ++q) {
                    const TV v = (x[q * MR + j] - p[q]) / d;
                    x[q * MR + j] = v;
                    if (q < nq) xp[F.first_col + j + (int64_t)(q0 + q) * n] = v;
                }
            }
            __syncwarp();
        }
    }
    group_signal<32>(deps.done + s, 0xffffffffu);
}

// dispatch on the front's rows: registers up to 32, the shared buffer above
template <typename TL, typename TV, int NQ>
__device__ void fwd_warp_front(int s, const FrontDeps& deps, const FrontDesc* __restrict__ fronts,
                               const int* __restrict__ child, const int* __restrict__ relmap,
                               const int64_t* __restrict__ fv_off, const TL* __restrict__ Ls,
                               TV* __restrict__ xp, TV* __restrict__ fv, int n, int nrhs,
                               TV* wbuf, int MR) {
    const FrontDesc F = fronts[s];
    TV* out = front_vec(fv, fv_off, s, nrhs);
    if (F.m <= 32)
        fwd_group_front<TL, TV, 32, NQ>(s, F, deps, fronts, child, relmap, fv_off, Ls, xp, out,
                                        fv, n, nrhs, wbuf);
    else
        fwd_warp_front_smem<TL, TV, NQ>(s, F, deps, fronts, child, relmap, fv_off, Ls, xp, out,
                                        fv, n, nrhs, wbuf, MR);
}

template <typename TL, typename TV, int NQ>
__device__ void bwd_warp_front(int s, const FrontDeps& deps, const FrontDesc* __restrict__ fronts,
                               const int* __restrict__ rows, const TL* __restrict__ Ls,
                               TV* __restrict__ xp, int n, int nrhs, TV* wbuf, int MR) {
    const FrontDesc F = fronts[s];
    if (F.m <= 32)
        bwd_group_front<TL, TV, 32, NQ>(s, F, deps, rows, Ls, xp, n, nrhs);
    else
        bwd_warp_front_smem<TL, TV, NQ>(s, F, deps, rows, Ls, xp, n, nrhs, wbuf, MR);
}

// per-warp shared buffer of the warp path: MR = rows rounded up to 32, times
// the right-hand sides of one pass
__host__ __device__ constexpr int warp_rows(int msmall) { return ((msmall + 31) / 32) * 32; }
__host__ __device__ constexpr int warp_buf_stride(int msmall, int nrhs) {
    return warp_rows(msmall) * (nrhs == 1 ? 1 : kWarpSolveRhs);
}

// Warp tasks of one warp item (its slice of the direction's warp list):
// tasks [0, n1) one front each, then two fronts of 9..16 rows per task, then
// four of at most 8 rows.
struct WarpTasks {
    const int* list;
    int n1, n2, n4;
    __host__ __device__ int count() const { return n1 + (n2 + 1) / 2 + (n4 + 3) / 4; }
};


template <typename TL, typename TV, int NQ>
__device__ void fwd_warp_task(const WarpTasks& wt, int t, const FrontDeps& deps,
                              const FrontDesc* __restrict__ fronts,
                              const int* __restrict__ child, const int* __restrict__ relmap,
                              const int64_t* __restrict__ fv_off, const TL* __restrict__ Ls,
                              TV* __restrict__ xp, TV* __restrict__ fv, int n, int nrhs, TV* wbuf,
                              int MR) {
    const int lane = threadIdx.x & 31;
    if (t < wt.n1) {
        fwd_warp_front<TL, TV, NQ>(wt.list[t], deps, fronts, child, relmap, fv_off, Ls, xp, fv, n,
                                   nrhs, wbuf, MR);
        return;
    }
    t -= wt.n1;
    const int t2 = (wt.n2 + 1) / 2;
    if (t < t2) {
        const int k = 2 * t + (lane >> 4);
        if (k < wt.n2) {
            const int s = wt.list[wt.n1 + k];
            const FrontDesc F = fronts[s];
            fwd_group_front<TL, TV, 16, NQ>(s, F, deps, fronts, child, relmap, fv_off, Ls, xp,
                                            front_vec(fv, fv_off, s, nrhs), fv, n, nrhs,
                                            wbuf + (lane & 16));
        }
        return;
    }
    const int k = 4 * (t - t2) + (lane >> 3);
    if (k < wt.n4) {
        const int s = wt.list[wt.n1 + wt.n2 + k];
        const FrontDesc F = fronts[s];
        fwd_group_front<TL, TV, 8, NQ>(s, F, deps, fronts, child, relmap, fv_off, Ls, xp,
                                       front_vec(fv, fv_off, s, nrhs), fv, n, nrhs,
                                       wbuf + (lane & 24));
    }
}

template <typename TL, typename TV, int NQ>
__device__ void bwd_warp_task(const WarpTasks& wt, int t, const FrontDeps& deps,
                              const FrontDesc* __restrict__ fronts, const int* __restrict__ rows,
                              const TL* __restrict__ Ls, TV* __restrict__ xp, int n, int nrhs,
                              TV* wbuf, int MR) {
    const int lane = threadIdx.x & 31;
    if (t < wt.n1) {
        bwd_warp_front<TL, TV, NQ>(wt.list[t], deps, fronts, rows, Ls, xp, n, nrhs, wbuf, MR);
        return;
    }
    t -= wt.n1;
    const int t2 = (wt.n2 + 1) / 2;
    if (t < t2) {
        const int k = 2 * t + (lane >> 4);
        if (k < wt.n2) {
            const int s = wt.list[wt.n1 + k];
            bwd_group_front<TL, TV, 16, NQ>(s, fronts[s], deps, rows, Ls, xp, n, nrhs);
        }
        return;
    }
    const int k = 4 * (t - t2) + (lane >> 3);
    if (k < wt.n4) {
        const int s = wt.list[wt.n1 + wt.n2 + k];
        bwd_group_front<TL, TV, 8, NQ>(s, fronts[s], deps, rows, Ls, xp, n, nrhs);
    }
}

// Backward, task (s, j): pivot column tile j of front s accumulates, once
// the update-row gathers of (s, j) have all counted in, their partial sums
// in chunk order, then acc += sum_{k > j} L(k, j)' x_k over the pivot tiles
// nt1-1 .. j+1 of this front as they publish, and solves
// x_j = inv(L_jj)' (y_j - acc).  Threads: l = column in the tile.
template <typename TL, typename TV, int NQ>
__device__ void bwd_chain_task(int2 tk, const FrontDesc* __restrict__ fronts,
                               double* __restrict__ pub, int* __restrict__ abort_flag,
                               int* __restrict__ err, const int* __restrict__ gather_nch,
                               const int* __restrict__ gather_off, const int* __restrict__ gcount,
                               const TV* __restrict__ part, const int64_t* __restrict__ dinv_off,
                               const TL* __restrict__ Ls, const TL* __restrict__ Dinv,
                               TV* __restrict__ xp, int n, int nrhs) {
    static_assert(sizeof(TV) == 8, "solve vectors are double");
    constexpr int T = kTile, LD = blk_ld<TL>();
    const LevelSmem<TL, TV> sm(nrhs);
    __shared__ int s_ok;
    const int tid = threadIdx.x, l = tid & (T - 1), g = tid >> 6;
    // one right-hand side: warp w takes columns 8w .. 8w + 7, lane (c1 =
    // column, q1 = row phase) the rows q1, q1 + 4, ...: conflict-free reads
    // of the 16-byte-column stage layout, the phases summed by shuffles
    const int c1 = 8 * (tid >> 5) + (tid & 7), q1 = (tid >> 3) & 3;
    const int s = tk.x, j = tk.y;
    const FrontDesc F = fronts[s];
    const int nt1 = tiles_l(F.c, T);
    const TileRange tj = tile_range(j, F.m, F.c, T);
    const bool lsplit = nrhs == 1;
    const TL* Lc = Ls + F.loff + (int64_t)tj.start * F.ldl;  // column tile j
    const int64_t tile0 = dinv_off[s] / (T * T);               // this front's first pivot tile
    double* pb = pub + tile0 * T * nrhs;
    const int P = nt1 - 1 - j;  // pivot row tiles k = nt1-1 down to j+1
    auto issue = [&](int p) {
        if (p < P) {
            const TileRange tkr = tile_range(nt1 - 1 - p, F.m, F.c, T);
            load_block_async(sm.lb(p), Lc, F.ldl, tkr.start, tkr.size, tj.size);
            load_slot_async(sm.vb(p, nrhs), pb + (int64_t)(nt1 - 1 - p) * T * nrhs, nrhs);
        }
        cp_async_commit_group();
    };
    load_block_async(sm.Dk, Dinv + dinv_off[s] + (int64_t)j * T * T, T, 0, tj.size, tj.size);
    for (int p = 0; p < sm.stg - 1; ++p) issue(p);
    TV acc[NQ];
#pragma unroll
    for (int a = 0; a < NQ; ++a) acc[a] = TV(0);
    // this tile's y_j, before the first wait
    const int64_t xj = F.first_col + tj.start;
    TV ypre[NQ];
#pragma unroll
    for (int a = 0; a < NQ; ++a) {
        if (lsplit)
            ypre[a] = (a == 0 && q1 == 0 && c1 < tj.size) ? __ldcg(xp + xj + c1) : TV(0);
        else
            ypre[a] = (l < tj.size && g + 4 * a < nrhs)
                          ? __ldcg(xp + xj + l + (int64_t)(g + 4 * a) * n)
                          : TV(0);
    }
    // the update-row partial sums of (s, j) (gathers hold lower tickets), in
    // chunk order, before the chain's first wait
    {
        const int nch = gather_nch[s];
        if (nch > 0) {
            if (tid == 0) s_ok = wait_flag(gcount + tile0 + j, nch, abort_flag, err) ? 1 : 0;
            __syncthreads();
            if (!s_ok) {
                cp_async_wait_groups<0>();
                return;
            }
            const TV* pj = part + ((int64_t)gather_off[s] + (int64_t)j * nch) * T * nrhs;
            for (int h = 0; h < nch; ++h, pj += (int64_t)T * nrhs) {
                if (lsplit) {
                    if (q1 == 0) acc[0] += __ldcg(pj + c1);
                } else {
#pragma unroll
                    for (int a = 0; a < NQ; ++a) {
                        const int q = g + 4 * a;
                        if (q < nrhs) acc[a] += __ldcg(pj + l + T * q);
                    }
                }
            }
        }
    }
    bool ok = true;
    for (int p = 0; p < P; ++p) {
        issue(p + sm.stg - 1);
        cp_async_wait_stages(sm.stg);
        __syncthreads();
        const int k = nt1 - 1 - p;
        TV* X = sm.vb(p, nrhs);
        if (!settle_slot(X, pb + (int64_t)k * T * nrhs, tile_range(k, F.m, F.c, T).size, nrhs,
                         abort_flag, err)) {
            ok = false;
            break;
        }
        const TL* B = sm.lb(p);
        if (lsplit) {
#pragma unroll
            for (int u = 0; u < 16; ++u) acc[0] += (TV)B[q1 + 4 * u + c1 * LD] * X[q1 + 4 * u];
        } else {
#pragma unroll 4
            for (int r = 0; r < T; ++r) {
                const TV lv = (TV)B[r + l * LD];
#pragma unroll
                for (int a = 0; a < NQ; ++a) {
                    const int q = g + 4 * a;
                    if (q < nrhs) acc[a] += lv * X[r + T * q];
                }
            }
        }
        if (p + 1 < P) __syncthreads();  // the stages are reused; after the last, nothing is
    }
    cp_async_wait_groups<0>();
    if (!ok) return;
    TV* X = sm.Y;
    const TL* Dk = sm.Dk;
    // t = y_j - acc (y_j: this front's forward solution), then x_j = Dk' t
    if (lsplit) {
        // one right-hand side, one barrier: the row phases' sums by
        // shuffles, t into sm.Y, then x_j = Dk' t the same way
        TV a = acc[0] + __shfl_xor_sync(0xffffffffu, acc[0], 8);
        a += __shfl_xor_sync(0xffffffffu, a, 16);
        if (q1 == 0) X[c1] = c1 < tj.size ? ypre[0] - a : TV(0);
        __syncthreads();
        TV x = TV(0);
#pragma unroll
        for (int u = 0; u < 16; ++u) x += (TV)Dk[q1 + 4 * u + c1 * LD] * X[q1 + 4 * u];
        x += __shfl_xor_sync(0xffffffffu, x, 8);
        x += __shfl_xor_sync(0xffffffffu, x, 16);
        if (q1 == 0 && c1 < tj.size) {
            xp[xj + c1] = x;
            st_relaxed_f64(pb + (int64_t)j * T + c1, x);
        }
        return;
    }
    __syncthreads();
#pragma unroll
    for (int a = 0; a < NQ; ++a) {
        const int q = g + 4 * a;
        if (q < nrhs) X[l + T * q] = l < tj.size ? ypre[a] - acc[a] : TV(0);
    }
    __syncthreads();
    {
        TV x[NQ];
#pragma unroll
        for (int a = 0; a < NQ; ++a) x[a] = TV(0);
#pragma unroll 4
        for (int r = 0; r < T; ++r) {
            const TV dv = (TV)Dk[r + l * LD];
#pragma unroll
            for (int a = 0; a < NQ; ++a) {
                const int q = g + 4 * a;
                if (q < nrhs) x[a] += dv * X[r + T * q];
            }
        }
        if (l < tj.size) {
#pragma unroll
            for (int a = 0; a < NQ; ++a) {
                const int q = g + 4 * a;
                if (q < nrhs) {
                    xp[xj + l + (int64_t)q * n] = x[a];
                    st_relaxed_f64(pb + ((int64_t)j * nrhs + q) * T + l, x[a]);
                }
            }
        }
    }
}

// ---------------------------------------------------------------------------
// forward update tiles with one right-hand side: L read straight from global
// memory into registers, coalesced (a thread per row), the next columns'
// loads issued before the current ones are used, no block barrier per L
// block.  The pivot tiles' published vectors come through poll_published
// into a shared double buffer (a buffer is rewritten two polls later, after
// the barrier of the poll between).
// ---------------------------------------------------------------------------

// (fronts of one pivot tile only: with more, one column group of loads in
// flight per iteration leaves a tail of one memory latency per 16 columns
// after the last pivot tile, where the staged tile path keeps two 64-column
// blocks in flight)
constexpr int kRt1MaxPivotTiles = 1;

struct Rt1Smem {
    double* Ys;  // 2 x T: published slots
    __device__ Rt1Smem() {
        extern __shared__ __align__(16) unsigned char smem_raw[];
        Ys = reinterpret_cast<double*>(smem_raw);
    }
};
template <typename TL>
__host__ __device__ constexpr size_t rt1_smem_bytes() {
    return 2 * (size_t)kTile * sizeof(double);
}

template <typename TL>
__device__ __forceinline__ TL ldL(const TL* p) {
    return __ldg(p);
}

// Forward update rows [R0, R1) of front s (at most 256; one right-hand side):
// thread = row; columns in groups of 16, the next group's loads issued
// before the current group's products.
template <typename TL>
__device__ void fwd_update_rt1(int s, int R0, int R1, const FrontDesc& F, double* __restrict__ pb,
                               int* __restrict__ abort_flag, int* __restrict__ err,
                               const int* __restrict__ amap_off, const int* __restrict__ amap_row,
                               const int* __restrict__ amap_ent, const TL* __restrict__ Ls,
                               const double* __restrict__ xp, double* __restrict__ f,
                               const double* __restrict__ fv) {
    constexpr int T = kTile;
    const Rt1Smem sm;
    const int R = R0 + threadIdx.x;
    const bool rv = R < R1;
    const TL* Lr = Ls + F.loff + R;
    double f0 = 0.0;
    if (rv) {
        const int* ar = amap_row + amap_off[s] + R;
        const int e0 = ar[0], e1 = ar[1];
        for (int e = e0; e < e1; ++e) f0 += __ldcg(fv + amap_ent[e]);
    }
    constexpr int GW = sizeof(TL) == 4 ? 16 : 8;  // columns per group (registers)
    constexpr int GPB = T / GW;                     // groups per 64-column block
    const int ng = (F.c + GW - 1) / GW;
    auto load = [&](int cg, TL (&v)[GW]) {
#pragma unroll
        for (int l = 0; l < GW; ++l) {
            const int col = GW * cg + l;
            v[l] = (rv && col < F.c) ? ldL(Lr + (int64_t)col * F.ldl) : TL(0);
        }
    };
    double acc = 0.0;
    TL lv[GW], ln[GW];
    load(0, lv);
    for (int cg = 0; cg < ng; ++cg) {
        if (cg + 1 < ng) load(cg + 1, ln);
        const int k = cg / GPB;
        double* Yk = sm.Ys + (k & 1) * T;
        if (cg % GPB == 0 &&
            !poll_published(Yk, pb + (int64_t)k * T, min(T, F.c - k * T), 1, abort_flag, err))
            return;
        const double* y = Yk + GW * (cg % GPB);
#pragma unroll
        for (int l = 0; l < GW; ++l) acc += (double)lv[l] * y[l];
#pragma unroll
        for (int l = 0; l < GW; ++l) lv[l] = ln[l];
    }
    if (rv) f[R] = f0 - acc;
}

// One launch per direction over all work items (the item lists, in a
// topological order by critical-path priority, and their kinds are
// described with the solve schedule): persistent CTAs take items by atomic
// ticket.  An item only waits for items with lower tickets -- children's
// (forward) and parents' (backward) items come earlier in the list, and so
// do a front's earlier pivot tiles and its backward gathers -- and a CTA
// takes a ticket only while it runs, so every wait is for a CTA that is
// running or done.
// Forward: a front's items wait for its children (the count of finished
// children), a small front counts itself in at its parent once written, a
// large front once its last update tile is (a per-front count of finished
// update tiles).  Backward: a front's items wait for its parent's solution
// rows (the parent's count of completions: one per pivot tile of a large
// front, one for a small front); the pivot tasks wait for their gathers'
// counts as before.  Every wait polls with an iteration limit; on timeout
// the launch is aborted (every later wait returns at once) and the error
// word reaches the host.

// a CTA's tid 0 waits (bounded) for *word >= target; uniform result
__device__ __forceinline__ bool cta_wait(const int* word, int target, int* abort_flag, int* err) {
    __shared__ int s_wok;
    if (threadIdx.x == 0) s_wok = wait_flag(word, target, abort_flag, err) ? 1 : 0;
    __syncthreads();
    return s_wok != 0;
}

template <typename TL, typename TV, int NQ>
__global__ void __launch_bounds__(256, NQ == 1 ? 4 : 2)
    k_fwd_solve(const FrontDesc* __restrict__ fronts, const int4* __restrict__ items, int nitems,
                int* __restrict__ counter, double* __restrict__ pub, int* __restrict__ abort_flag,
                int* __restrict__ err, int* __restrict__ fdone, int* __restrict__ udone,
                const int64_t* __restrict__ fv_off, const int* __restrict__ amap_off,
                const int* __restrict__ amap_row, const int* __restrict__ amap_ent,
                const int64_t* __restrict__ dinv_off, const int* __restrict__ wlist,
                const int* __restrict__ child,
                const int* __restrict__ relmap, const TL* __restrict__ Ls,
                const TL* __restrict__ Dinv, TV* __restrict__ xp, TV* __restrict__ fv, int n,
                int nrhs, int MR) {
    constexpr int T = kTile;
    __shared__ int s_item;
    const FrontDeps deps{fdone, nullptr, abort_flag, err};
    for (;;) {
        if (threadIdx.x == 0) s_item = atomicAdd(counter, 1);
        __syncthreads();
        const int k = s_item;
        if (k >= nitems) return;
        const int4 it = items[k];
        if (it.x == SolveScheduleHost::kItemWarps) {
            extern __shared__ __align__(16) unsigned char smem_raw[];
            const WarpTasks wt{wlist + it.y, it.z & 0xff, (it.z >> 8) & 0xff, it.z >> 16};
            const int w = threadIdx.x >> 5, t = w;
            TV* wbuf = reinterpret_cast<TV*>(smem_raw) + w * warp_buf_stride(MR, nrhs);
            if (t < wt.count()) {
                if (nrhs == 1)
                    fwd_warp_task<TL, TV, 1>(wt, t, deps, fronts, child, relmap, fv_off, Ls, xp,
                                             fv, n, nrhs, wbuf, MR);
                else
                    fwd_warp_task<TL, TV, kWarpSolveRhs>(wt, t, deps, fronts, child, relmap,
                                                         fv_off, Ls, xp, fv, n, nrhs, wbuf, MR);
            }
        } else {
            // a tile task of a large front: its children first
            const int2 tk = make_int2(it.y, it.z);
            const int s = tk.x, i0 = tk.y & 0xffff, cnt = tk.y >> 16;
            const FrontDesc F = fronts[s];
            const int nt1 = tiles_l(F.c, T);
            if (cta_wait(fdone + s, F.child_end - F.child_beg, abort_flag, err)) {
                bool done = false;
                if constexpr (NQ == 1) {
                    // update tiles of fronts with at most kRt1MaxPivotTiles
                    // pivot tiles, one right-hand side: registers straight
                    // from L (measured faster there; the staged pipeline
                    // streams long column ranges better)
                    if (nrhs == 1 && i0 >= nt1 && nt1 <= kRt1MaxPivotTiles) {
                        double* pb = pub + (dinv_off[s] / (T * T)) * T;
                        const TileRange a = tile_range(i0, F.m, F.c, T);
                        const TileRange b = tile_range(i0 + cnt - 1, F.m, F.c, T);
                        fwd_update_rt1<TL>(s, a.start, b.start + b.size, F, pb, abort_flag, err,
                                           amap_off, amap_row, amap_ent, Ls, xp,
                                           front_vec(fv, fv_off, s, 1), fv);
                        done = true;
                    }
                }
                if (!done)
                    fwd_tile_task<TL, TV, NQ>(tk, fronts, pub, abort_flag, err, fv_off, amap_off,
                                              amap_row, amap_ent, dinv_off, Ls, Dinv, xp, fv, n,
                                              nrhs);
                // update tiles counted in; the front's last one counts the
                // front in at its parent
                if (i0 >= nt1) {
                    __syncthreads();
                    if (threadIdx.x == 0) {
                        __threadfence();
                        const int ntu = tiles_l(F.m - F.c, T);
                        if (atomicAdd(udone + s, cnt) + cnt == ntu && F.parent >= 0) {
                            __threadfence();
                            atomicAdd(fdone + F.parent, 1);
                        }
                    }
                }
            }
        }
        __syncthreads();  // shared memory and s_item free for the next item
    }
}

template <typename TL, typename TV, int NQ>
__global__ void __launch_bounds__(256, NQ == 1 ? 4 : 2)
    k_bwd_solve(const FrontDesc* __restrict__ fronts, const int4* __restrict__ items, int nitems,
                int* __restrict__ counter, double* __restrict__ pub, int* __restrict__ abort_flag,
                int* __restrict__ err, int* __restrict__ bdone, const int* __restrict__ btarget,
                const int* __restrict__ gather_nch, const int* __restrict__ gather_off,
                int* __restrict__ gcount, TV* __restrict__ part,
                const int64_t* __restrict__ dinv_off, const int* __restrict__ wlist,
                const int* __restrict__ rows,
                const TL* __restrict__ Ls, const TL* __restrict__ Dinv, TV* __restrict__ xp,
                int n, int nrhs, int MR) {
    __shared__ int s_item;
    const FrontDeps deps{bdone, btarget, abort_flag, err};
    for (;;) {
        if (threadIdx.x == 0) s_item = atomicAdd(counter, 1);
        __syncthreads();
        const int k = s_item;
        if (k >= nitems) return;
        const int4 it = items[k];
        if (it.x == SolveScheduleHost::kItemWarps) {
            extern __shared__ __align__(16) unsigned char smem_raw[];
            const WarpTasks wt{wlist + it.y, it.z & 0xff, (it.z >> 8) & 0xff, it.z >> 16};
            const int w = threadIdx.x >> 5, t = w;
            TV* wbuf = reinterpret_cast<TV*>(smem_raw) + w * warp_buf_stride(MR, nrhs);
            if (t < wt.count()) {
                if (nrhs == 1)
                    bwd_warp_task<TL, TV, 1>(wt, t, deps, fronts, rows, Ls, xp, n, nrhs, wbuf, MR);
                else
                    bwd_warp_task<TL, TV, kWarpSolveRhs>(wt, t, deps, fronts, rows, Ls, xp, n,
                                                         nrhs, wbuf, MR);
            }
        } else if (it.x == SolveScheduleHost::kItemGather) {
            // the update rows' partial sums need the ancestors' solution
            const int2 tk = make_int2(it.y, it.z);
            const int p = fronts[tk.x].parent;
            if (p < 0 || cta_wait(bdone + p, btarget[p], abort_flag, err))
                bwd_gather_task<TL, TV, NQ>(tk, fronts, rows, gather_nch, gather_off, gcount,
                                            dinv_off, Ls, xp, part, n, nrhs);
        } else {
            // a pivot tile: its gathers (counted) waited for the ancestors
            const int2 tk = make_int2(it.y, it.z);
            bwd_chain_task<TL, TV, NQ>(tk, fronts, pub, abort_flag, err, gather_nch, gather_off,
                                       gcount, part, dinv_off, Ls, Dinv, xp, n, nrhs);
            __syncthreads();
            if (threadIdx.x == 0) {
                __threadfence();
                atomicAdd(bdone + tk.x, 1);
            }
        }
        __syncthreads();  // shared memory and s_item free for the next item
    }
}

// ---------------------------------------------------------------------------
// permutations
// ---------------------------------------------------------------------------

__global__ void k_perm_gather(const int* __restrict__ perm, const double* __restrict__ b,
                              double* __restrict__ xp, int n, int nrhs, int ldb) {
    int64_t total = (int64_t)n * nrhs;
    for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < total;
         idx += (int64_t)gridDim.x * blockDim.x) {
        int q = (int)(idx / n), k = (int)(idx - (int64_t)q * n);
        xp[idx] = b[(perm ? perm[k] : k) + (int64_t)q * ldb];
    }
}

__global__ void k_perm_scatter(const int* __restrict__ perm, const double* __restrict__ xp,
                               double* __restrict__ x, int n, int nrhs, int ldx) {
    int64_t total = (int64_t)n * nrhs;
    for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < total;
         idx += (int64_t)gridDim.x * blockDim.x) {
        int q = (int)(idx / n), k = (int)(idx - (int64_t)q * n);
        x[(perm ? perm[k] : k) + (int64_t)q * ldx] = xp[idx];
    }
}

void permute_gather(const int* perm, const double* b, double* xp, int n, int nrhs, int ldb,
                    cudaStream_t st) {
    int64_t total = (int64_t)n * nrhs;
    int blocks = (int)std::min<int64_t>((total + 255) / 256, 148 * 16);
    k_perm_gather<<<blocks, 256, 0, st>>>(perm, b, xp, n, nrhs, ldb);
}

void permute_scatter(const int* perm, const double* xp, double* x, int n, int nrhs, int ldx,
                     cudaStream_t st) {
    int64_t total = (int64_t)n * nrhs;
    int blocks = (int)std::min<int64_t>((total + 255) / 256, 148 * 16);
    k_perm_scatter<<<blocks, 256, 0, st>>>(perm, xp, x, n, nrhs, ldx);
}

// ---------------------------------------------------------------------------
// launch sequence
// ---------------------------------------------------------------------------

// rows of a small front's warp buffer (every level's largest small front)
constexpr int kWarpBufRows = ((Plan::kSmallMaxRows + 31) / 32) * 32;

// dynamic shared memory of a solve launch: the tile tasks' stages or the
// eight warps' buffers, whichever is larger
template <typename TL, typename TV>
static size_t solve_smem(int nrhs) {
    size_t m = level_smem_bytes<TL, TV>(nrhs);
    if (nrhs == 1) m = std::max(m, rt1_smem_bytes<TL>());
    return std::max(m, 8 * (size_t)warp_buf_stride(kWarpBufRows, nrhs) * sizeof(TV));
}

template <typename TL, typename TV, int NQ>
static void set_solve_attributes_nq() {
    const int sm = (int)solve_smem<TL, TV>(kSolvePassRhs);
    cudaFuncSetAttribute(k_fwd_solve<TL, TV, NQ>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
    cudaFuncSetAttribute(k_bwd_solve<TL, TV, NQ>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
}

template <typename TL, typename TV>
static void set_solve_attributes() {
    set_solve_attributes_nq<TL, TV, 1>();
    set_solve_attributes_nq<TL, TV, 4>();
    set_solve_attributes_nq<TL, TV, 8>();
}

void init_solve_kernels() {
    set_solve_attributes<double, double>();
    set_solve_attributes<float, double>();
}

template <typename TL, typename TV, int NQ>
static void solve_levels_nq(const DevPlan& D, const TL* Ls, const TL* Dinv, TV* xp, TV* fv,
                            int nrhs, cudaStream_t st) {
    const SolveSchedule& S = D.solve;
    static_assert(Plan::kSmallMaxRows <= 32 * 5, "the warp path holds 160 rows in shared memory");
    // sync: the two ticket counters, the gathers' counts per pivot tile, the
    // abort word, then per front the forward finished-children and
    // finished-update-tile counts and the backward completions
    int* counters = S.sync;
    int* gcount = S.sync + 2;
    int* abort_flag = gcount + S.nflags;
    int* fdone = abort_flag + 1;
    int* udone = fdone + S.nfronts;
    int* bdone = udone + S.nfronts;
    cudaMemsetAsync(S.sync, 0, (size_t)S.nsync * sizeof(int), st);
    // publication slots of the forward and backward pivot tiles: all-ones bits
    cudaMemsetAsync(fv + D.fv_pub_off * nrhs, 0xff,
                    (size_t)2 * S.nflags * kTile * nrhs * sizeof(TV), st);
    const size_t sm = solve_smem<TL, TV>(nrhs);
    const int sms = D.num_sms > 0 ? D.num_sms : 148;
    const int grid = sms * (NQ == 1 ? 4 : 2);  // the launch bounds' residency
    double fbytes = 0, bbytes = 0;
    for (int l = 0; l < D.nlevels; ++l) {
        fbytes += (S.small_elems[l] + S.fwd_elems[l]) * sizeof(TL);
        bbytes += (S.small_elems[l] + S.bwd_elems[l]) * sizeof(TL);
    }
    if (S.nfwd_items > 0) {
        ProfScope ps(D.prof, KC_SOLVE_LARGE, st, 0, fbytes);
        k_fwd_solve<TL, TV, NQ><<<std::min(grid, S.nfwd_items), 256, sm, st>>>(
            D.fronts, S.fwd_items, S.nfwd_items, counters, fv + D.fv_pub_off * nrhs, abort_flag,
            S.err, fdone, udone, D.fv_off, S.amap_off, S.amap_row, S.amap_ent, D.dinv_off,
            S.fwd_wlist, D.child, D.relmap, Ls, Dinv, xp, fv, D.n, nrhs,
            kWarpBufRows);
    }
    if (S.nbwd_items > 0) {
        ProfScope ps(D.prof, KC_SOLVE_LARGE, st, 0, bbytes);
        k_bwd_solve<TL, TV, NQ><<<std::min(grid, S.nbwd_items), 256, sm, st>>>(
            D.fronts, S.bwd_items, S.nbwd_items, counters + 1,
            fv + (D.fv_pub_off + (int64_t)S.nflags * kTile) * nrhs, abort_flag, S.err, bdone,
            S.bwd_target, S.gather_nch, S.gather_off, gcount, fv + D.fv_fronts * nrhs,
            D.dinv_off, S.bwd_wlist, D.rows, Ls, Dinv, xp, D.n, nrhs,
            kWarpBufRows);
    }
}

template <typename TL, typename TV>
void solve_levels(const DevPlan& D, const TL* Ls, const TL* Dinv, TV* xp, TV* fv, int nrhs,
                  cudaStream_t st) {
    // passes of at most kSolvePassRhs right-hand sides (xp columns q0 ..;
    // the work vectors, sized for more, are reused with the pass's count)
    for (int q0 = 0; q0 < nrhs; q0 += kSolvePassRhs) {
        const int nq = std::min(kSolvePassRhs, nrhs - q0);
        TV* x = xp + (int64_t)q0 * D.n;
        if (nq <= 4)
            solve_levels_nq<TL, TV, 1>(D, Ls, Dinv, x, fv, nq, st);
        else if (nq <= 16)
            solve_levels_nq<TL, TV, 4>(D, Ls, Dinv, x, fv, nq, st);
        else
            solve_levels_nq<TL, TV, 8>(D, Ls, Dinv, x, fv, nq, st);
    }
}

template void solve_levels<double, double>(const DevPlan&, const double*, const double*, double*,
                                           double*, int, cudaStream_t);
template void solve_levels<float, double>(const DevPlan&, const float*, const float*, double*,
                                          double*, int, cudaStream_t);

}  // namespace mdgpu
