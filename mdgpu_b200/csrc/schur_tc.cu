// Tensor-core Schur-complement update for FP32 fronts (3xTF32 products, or
// one BF16 product, FP32 accumulation) on sm_100a: tcgen05.mma with the
// accumulators in TMEM, operands brought into shared memory by TMA straight
// from the L panels.
//
// After pivot panel p (columns [k0, k0 + K), K <= 256) of a large front, the
// trailing lower part is updated in 128 x 128 tiles (I, J), I >= J >= J0:
//     C(I, J) -= A_I A_J'      A_I = rows 128 I .. of the panel's columns
// in 3xTF32: A = hi + lo with hi = A with the low 13 mantissa bits cleared
// (an exact TF32 value) and lo = A - hi (exact in FP32), and
// C -= lo hi' + hi lo' + hi hi' (close to FP32 accuracy, which keeps the
// iterative refinement short).
//
// Persistent CTAs take tiles round-robin over the launch's tile list, with
// three roles:
//   loader     3xTF32: lane 0 of warp 0 issues per 32-column chunk one TMA
//              load each of A_hi, B_hi, A_lo, B_lo (128 rows x 128 bytes,
//              128-byte swizzle: K-major) from the split scratch the panel
//              kernel wrote (hi = A with the low 13 mantissa bits cleared,
//              lo = A - hi; per front 2 mpad rows of 256 columns, row-major;
//              rows past it read as zeros); BF16: warps 0-3, the TMA of
//              64-column FP32 chunks of the L panel, then the rounding to
//              BF16 into a K-major copy (below);
//   MMA        one elected thread: per 8-column step three tcgen05.mma
//              kind::tf32 (M = N = 128), or one kind::f16 per 16 columns,
//              into the tile's TMEM accumulator; each stage is committed
//              back to the loader, each finished tile to the epilogue;
//   epilogue   eight warps, two per 32 TMEM lanes (tile rows), each two
//              32-column blocks: the tile's old C values loaded first (under
//              the tile's MMAs), then tcgen05.ld of the accumulator, handed
//              back once read, and C -= acc in place (coalesced along the
//              columns).
// The TMEM accumulator is double-buffered (2 x 128 columns), so tile t's
// epilogue runs under tile t + 1's MMAs.  320 threads, one CTA per SM;
// 3xTF32: three 64 KB stages; BF16: six 32 KB stages.
//
// BF16 mode (the MDGPU_BF16 factor): the loaders round each FP32 chunk to
// BF16 (nearest even) into a K-major copy with the 128-byte swizzle, and one
// tcgen05.mma kind::f16 per 16 columns replaces the three TF32 products.
// Per-front power-of-two scaling is not applied: BF16 keeps FP32's 8-bit
// exponent, so scaling by 2^k would only shift exponents and leave every
// rounded bit as it is.
//
// Both modes feed the MMA K-major operands with the 128-byte swizzle: rows
// of 128 bytes (32 TF32 or 64 BF16 values along K), 8-row atoms of 1024
// bytes, the 16-byte chunk c of row r at c ^ (r mod 8) -- the pattern the
// TMA writes with CU_TENSOR_MAP_SWIZZLE_128B (3xTF32) and the BF16
// conversion writes by hand.  A K-step of the MMA (8 TF32 or 16 BF16) is 32
// bytes along the row: the descriptor's start address advances by 32.
//
// Every wait on an mbarrier is bounded: on timeout the CTA records an error
// code in *err and sets its abort word, every role leaves its loop, the
// loaders wait (bounded) for their TMA loads in flight and the MMA warp for
// its MMAs, then the TMEM is freed and the CTA returns; the host reports the
// error.  The TMA loads never use cluster multicast and only ever read this
// GPU's own memory.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstdio>

#include "device_common.cuh"
#include "kernels.hpp"

namespace mdgpu {

namespace tc {

constexpr int BM = 128, BN = 128;
constexpr uint32_t TMEM_COLS = 2 * BN;  // two accumulators

// Per-mode constants: a chunk is 128 bytes of K per operand row (32 TF32 or
// 64 BF16 columns); a stage holds A_hi, B_hi, A_lo, B_lo (3xTF32) or A, B
// (BF16), 16 KB each, as the panel kernel wrote them.  One TMA warp, one MMA
// warp, eight epilogue warps (two per 32 TMEM lanes, two 32-column blocks
// each); one CTA per SM.
template <int MODE>
struct Cfg {
    static constexpr bool BF = MODE == kSchurBF16;
    static constexpr int BK = BF ? 64 : 32;       // K columns per chunk
    static constexpr int ESZ = BF ? 2 : 4;        // operand element bytes
    static constexpr int OPER = BM * BK * ESZ;    // bytes of one operand chunk (16 KB)
    static constexpr int NOPER = MODE == kSchur3xTF32 ? 4 : 2;
    static constexpr int STAGE_TMA = NOPER * OPER;
    static constexpr int STAGE_BYTES = STAGE_TMA;
    static constexpr int STAGES = NOPER == 4 ? 3 : 6;  // 192 KB of stages either way
    static constexpr int SMEM_BYTES = STAGES * STAGE_BYTES + 1024;  // + alignment slack
    static constexpr int NLOAD = 1;
    static constexpr int MMA_WARP = NLOAD;
    static constexpr int NEPI = 8;
    static constexpr int NTHREADS = (NLOAD + 1 + NEPI) * 32;
    static constexpr int CTAS_PER_SM = 1;
};
constexpr long long WAIT_LIMIT = 1ll << 22;                  // polls (with backoff)

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
                 "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t phase) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(phase)
        : "memory");
    return ok != 0;
}

// bounded wait; false on timeout or when the CTA's abort word is set
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t phase, volatile int* abort) {
    for (long long i = 0; i < WAIT_LIMIT; ++i) {
        if (mbar_try_wait(bar, phase)) return true;
        if (i > 64) {
            if (*abort) return false;
            __nanosleep(64);
        }
    }
    return false;
}
__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, uint64_t* bar,
                                            int x, int y) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%3, %4}], [%2];" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(smem_u32(bar)), "r"(x), "r"(y)
        : "memory");
}

// instruction descriptor: D f32, A/B tf32, both K-major, M = 128, N = 128
constexpr uint32_t IDESC = (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(BN >> 3) << 17) |
                           ((uint32_t)(BM >> 4) << 24);

__device__ __forceinline__ void mma_tf32(uint32_t tmem_d, uint64_t da, uint64_t db,
                                         uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}" ::"r"(
            tmem_d),
        "l"(da), "l"(db), "r"(IDESC), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u)
        : "memory");
}

// UMMA shared-memory descriptor: K-major, 128-byte swizzle (layout type 2):
// rows of 128 B along K, 8-row atoms 1024 B apart (SBO); the 16-byte chunks
// of row r of an atom sit at chunk ^ (r mod 8).  A K-step (8 TF32, 16 BF16)
// inside the 128-byte row advances the start address by 32 B.
__device__ __forceinline__ uint64_t make_desc_kmajor(uint32_t saddr) {
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFF);
    d |= (uint64_t)1 << 16;                   // LBO (unused for swizzled K-major)
    d |= (uint64_t)((1024 >> 4) & 0x3FFF) << 32;  // SBO: 8 rows of 128 B
    d |= (uint64_t)1 << 46;                   // descriptor version for sm_100
    d |= (uint64_t)2 << 61;                   // SWIZZLE_128B
    return d;
}

// instruction descriptor: D f32, A/B bf16 (kind::f16), both K-major,
// M = 128, N = 128
constexpr uint32_t IDESC_BF16 = (1u << 4) | (1u << 7) | (1u << 10) |
                                ((uint32_t)(BN >> 3) << 17) | ((uint32_t)(BM >> 4) << 24);

__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t da, uint64_t db,
                                         uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}" ::"r"(
            tmem_d),
        "l"(da), "l"(db), "r"(IDESC_BF16), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u)
        : "memory");
}

__device__ __forceinline__ void mma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::
                     "r"(smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32]) {
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
        "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];\n\t"
        "tcgen05.wait::ld.sync.aligned;"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
          "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]),
          "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]),
          "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
          "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]),
          "=r"(r[31])
        : "r"(taddr)
        : "memory");
    // the wait is in the same asm statement: the registers are defined only
    // once the asynchronous TMEM load has landed
#pragma unroll
    for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

// Tile number b of the launch -> front s and tile (I, J); the CTAs of a front
// enumerate the lower 128-tiles (I, J) with J >= J0 = cbeg / 128 row by row.
// The launch's update (upd = npan | strip << 4): the trailing part after
// panel `panel` (columns from cbeg = (panel + 1) PW) takes the products of
// the npan panels ending at `panel` (K = npan PW pivot columns from k0, read
// from scratch column kofs: panel q sits at column (q mod 2) PW); strip: only
// the two tile columns of the next panel, else the whole lower trailing part.
struct TileJob {
    int s, I, J, nk, k0, kofs, cbeg, cend;  // columns [cbeg, cend) are updated
};
__device__ __forceinline__ TileJob tile_job(const FrontDesc* __restrict__ fronts,
                                            const int* __restrict__ items,
                                            const int* __restrict__ before, int nitems, int b,
                                            int panel, int PW, int BK, int upd) {
    TileJob t;
    const int it = find_item(before, nitems, b);
    t.s = items[it];
    const FrontDesc f = fronts[t.s];
    const int npan = upd & 15;
    const int pf = panel - npan + 1;  // first panel of the update
    t.k0 = pf * PW;
    t.kofs = (pf & 1) * PW;
    const int K = min(npan * PW, f.c - t.k0);
    t.cbeg = min((panel + 1) * PW, f.c);
    // a strip stops at the next panel's end (the columns after it take this
    // panel's product with the next one's, in the following update)
    t.cend = (upd >> 4) ? min((panel + 2) * PW, f.c) : f.m;
    const int J0 = t.cbeg / BM;
    int ii, jj;
    const int q = b - before[it];
    if (upd >> 4) {  // strip: column J0 (rows J0 ..), then column J0 + 1
        const int nb = (f.m + BM - 1) / BM - J0;
        if (q < nb) {
            ii = q;
            jj = 0;
        } else {
            ii = q - nb + 1;
            jj = 1;
        }
    } else {
        lower_index(q, ii, jj);
    }
    t.I = J0 + ii;
    t.J = J0 + jj;
    t.nk = (K + BK - 1) / BK;
    return t;
}

}  // namespace tc

// items/before: one entry per large front (its tile count); ntiles: the
// launch's total.  maps: per large front a tensor map over its panel scratch
// (two panels side by side); upd: the update's shape (tile_job).
template <int MODE>
__global__ void __launch_bounds__(tc::Cfg<MODE>::NTHREADS, tc::Cfg<MODE>::CTAS_PER_SM)
    k_schur_tc(const FrontDesc* __restrict__ fronts, const int* __restrict__ items,
               const int* __restrict__ before, int nitems, int ntiles,
               const int* __restrict__ tmap_idx, const CUtensorMap* __restrict__ maps, int panel,
               int PW, int upd, float* __restrict__ Ls, float* __restrict__ Us,
               int* __restrict__ err) {
    using namespace tc;
    using C = Cfg<MODE>;
    constexpr int BK = C::BK, STAGES = C::STAGES, OPER = C::OPER, STAGE_TMA = C::STAGE_TMA,
                  STAGE_BYTES = C::STAGE_BYTES, NLOAD_WARPS = C::NLOAD,
                  MMA_WARP = C::MMA_WARP;
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    __shared__ __align__(8) uint64_t full_bar[STAGES];   // TMA bytes landed
    __shared__ __align__(8) uint64_t empty_bar[STAGES];  // MMAs done reading the stage
    __shared__ __align__(8) uint64_t accf_bar[2];        // accumulator complete
    __shared__ __align__(8) uint64_t acce_bar[2];        // accumulator read out (4 warps)
    __shared__ __align__(8) uint64_t drain_bar;          // every MMA issued has completed
    __shared__ uint32_t tmem_base_sh;
    __shared__ volatile int abort_sh;

    // 1024-byte aligned in the shared window (the 128-byte swizzle phase)
    unsigned char* smem = smem_raw + ((1024u - (tc::smem_u32(smem_raw) & 1023u)) & 1023u);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

    if (tid == 0) {
        for (int q = 0; q < STAGES; ++q) {
            tc::mbar_init(&full_bar[q], 1);
            tc::mbar_init(&empty_bar[q], 1);
        }
        for (int a = 0; a < 2; ++a) {
            tc::mbar_init(&accf_bar[a], 1);
            tc::mbar_init(&acce_bar[a], C::NEPI);
        }
        tc::mbar_init(&drain_bar, 1);
        abort_sh = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == MMA_WARP) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         tc::smem_u32(&tmem_base_sh)),
                     "r"(TMEM_COLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = tmem_base_sh;

    if (warp < NLOAD_WARPS) {
        // ---- loader: TMA (warp 0, lane 0)
        long long g = 0;  // chunk counter over this CTA's tiles
        long long issued = 0;
        bool ok = true;
        for (int b = blockIdx.x; b < ntiles && ok; b += gridDim.x) {
            const TileJob t = tile_job(fronts, items, before, nitems, b, panel, PW, BK, upd);
            const CUtensorMap* map = maps + tmap_idx[t.s];
            const int mpad = panel_mpad(fronts[t.s].m);
            for (int ch = 0; ch < t.nk; ++ch, ++g) {
                const int st = (int)(g % STAGES);
                const uint32_t use = (uint32_t)(g / STAGES);
                unsigned char* a = smem + st * STAGE_BYTES;
                if (tid == 0) {
                    if (use > 0 && !tc::mbar_wait(&empty_bar[st], (use - 1) & 1, &abort_sh)) {
                        ok = false;
                    } else {
                        // the panel scratch (row-major): K columns ch * BK ..,
                        // 128 rows per box; 3xTF32: hi rows, then lo rows
                        // from mpad
                        tc::mbar_expect_tx(&full_bar[st], STAGE_TMA);
                        const int col = t.kofs + ch * BK, ra = t.I * BM, rb = t.J * BN;
                        tc::tma_load_2d(a, map, &full_bar[st], col, ra);
                        tc::tma_load_2d(a + OPER, map, &full_bar[st], col, rb);
                        if constexpr (MODE == kSchur3xTF32) {
                            tc::tma_load_2d(a + 2 * OPER, map, &full_bar[st], col, mpad + ra);
                            tc::tma_load_2d(a + 3 * OPER, map, &full_bar[st], col, mpad + rb);
                        }
                        issued = g + 1;
                    }
                }
                ok = __shfl_sync(0xffffffffu, ok ? 1 : 0, 0) != 0;
                if (!ok) break;
            }
        }
        if (!ok && tid == 0) {
            atomicExch(err, 1);
            abort_sh = 1;
            // drain: wait (bounded, ignoring the abort word) for the loads issued
            volatile int never = 0;
            for (long long q = (issued > STAGES ? issued - STAGES : 0); q < issued; ++q)
                tc::mbar_wait(&full_bar[q % STAGES], (uint32_t)(q / STAGES) & 1, &never);
        }
    } else if (warp == MMA_WARP) {
        // ---- MMA issue
        if (lane == 0) {
            long long g = 0;
            int tl = 0;  // tiles of this CTA
            bool ok = true, any = false;
            for (int b = blockIdx.x; b < ntiles && ok; b += gridDim.x, ++tl) {
                const TileJob t = tile_job(fronts, items, before, nitems, b, panel, PW, BK, upd);
                const int acc = tl & 1;
                const uint32_t use_acc = (uint32_t)(tl >> 1);
                if (use_acc > 0 && !tc::mbar_wait(&acce_bar[acc], (use_acc - 1) & 1, &abort_sh)) {
                    ok = false;
                    break;
                }
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                const uint32_t d = tmem + (uint32_t)(acc * BN);
                for (int ch = 0; ch < t.nk; ++ch, ++g) {
                    const int st = (int)(g % STAGES);
                    if (!tc::mbar_wait(&full_bar[st], (uint32_t)(g / STAGES) & 1, &abort_sh)) {
                        ok = false;
                        break;
                    }
                    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                    if constexpr (MODE == kSchur3xTF32) {
                        const uint32_t ah = tc::smem_u32(smem + st * STAGE_BYTES);
                        const uint32_t bh = ah + OPER;
                        const uint32_t al = ah + 2 * OPER, bl = bh + 2 * OPER;
#pragma unroll
                        for (int k = 0; k < BK / 8; ++k) {
                            const uint32_t o = k * 32;
                            tc::mma_tf32(d, tc::make_desc_kmajor(al + o),
                                         tc::make_desc_kmajor(bh + o),
                                         (ch > 0 || k > 0) ? 1u : 0u);
                            tc::mma_tf32(d, tc::make_desc_kmajor(ah + o),
                                         tc::make_desc_kmajor(bl + o), 1u);
                            tc::mma_tf32(d, tc::make_desc_kmajor(ah + o),
                                         tc::make_desc_kmajor(bh + o), 1u);
                        }
                    } else if constexpr (MODE == kSchur1xTF32) {
                        // hi hi' only: one TF32 product
                        const uint32_t ah = tc::smem_u32(smem + st * STAGE_BYTES);
                        const uint32_t bh = ah + OPER;
#pragma unroll
                        for (int k = 0; k < BK / 8; ++k)
                            tc::mma_tf32(d, tc::make_desc_kmajor(ah + k * 32),
                                         tc::make_desc_kmajor(bh + k * 32),
                                         (ch > 0 || k > 0) ? 1u : 0u);
                    } else {
                        const uint32_t ab = tc::smem_u32(smem + st * STAGE_BYTES);
                        const uint32_t bb = ab + OPER;
#pragma unroll
                        for (int k = 0; k < BK / 16; ++k)
                            tc::mma_bf16(d, tc::make_desc_kmajor(ab + k * 32),
                                         tc::make_desc_kmajor(bb + k * 32),
                                         (ch > 0 || k > 0) ? 1u : 0u);
                    }
                    tc::mma_commit(&empty_bar[st]);
                    any = true;
                }
                if (!ok) break;
                tc::mma_commit(&accf_bar[acc]);
            }
            if (!ok) {
                atomicExch(err, 1);
                abort_sh = 1;
            }
            // completes once every MMA issued above has
            if (any) {
                tc::mma_commit(&drain_bar);
                volatile int never = 0;
                if (!tc::mbar_wait(&drain_bar, 0, &never)) atomicExch(err, 2);
            }
        }
        __syncwarp();
    } else {
        // ---- epilogue: warp w reads TMEM lanes 32 (w % 4) .. + 31 (tile
        // rows) and NCB 32-column blocks of them (two warps per lane
        // quarter).  The tile's old C values are loaded before the
        // accumulator is waited for, so their latency hides under the MMAs.
        constexpr int NCB = BN / 32 / (C::NEPI / 4);  // 32-column blocks per warp
        const int quarter = warp & 3;
        const int cb0 = ((warp - MMA_WARP - 1) >> 2) * NCB;
        int tl = 0;
        for (int b = blockIdx.x; b < ntiles; b += gridDim.x, ++tl) {
            const TileJob t = tile_job(fronts, items, before, nitems, b, panel, PW, BK, upd);
            const FrontDesc f = fronts[t.s];
            const int acc = tl & 1;
            const int row = t.I * BM + quarter * 32 + lane;
            const int col0 = t.J * BN + cb0 * 32;
            float* const Lrow = Ls + f.loff + row;          // C(row, col), col < c
            float* const Urow = Us + f.uoff + (row - f.c);  // C(row, col), col >= c
            // 32 columns from c0 of this lane's row: a pointer walked along
            // them (L panel, then the update store from column c on)
            auto start = [&](int c0) -> float* {
                return c0 < f.c ? Lrow + (int64_t)c0 * f.ldl : Urow + (int64_t)(c0 - f.c) * f.ldu;
            };
            // valid columns of this lane's row: [t.cbeg, chi)
            const int chi = row < f.m ? min(t.cend, row + 1) : t.cbeg;
            // old C values of a 32-column block into o (zeros outside)
            auto load_block = [&](int c0, float (&o)[32]) {
                float* p = start(c0);
#pragma unroll
                for (int q = 0; q < 32; ++q) {
                    const int col = c0 + q;
                    if (col == f.c) p = Urow;
                    o[q] = (col >= t.cbeg && col < chi) ? *p : 0.f;
                    p += col < f.c ? f.ldl : f.ldu;
                }
            };
            auto store_block = [&](int c0, const float (&o)[32], const float (&v)[32]) {
                float* p = start(c0);
#pragma unroll
                for (int q = 0; q < 32; ++q) {
                    const int col = c0 + q;
                    if (col == f.c) p = Urow;
                    if (col >= t.cbeg && col < chi) *p = o[q] - v[q];
                    p += col < f.c ? f.ldl : f.ldu;
                }
            };
            // the first block's old values load before the wait (under the
            // tile's MMAs), each later block's after the previous store
            float old[32], v[32];
            load_block(col0, old);
            if (!tc::mbar_wait(&accf_bar[acc], (uint32_t)(tl >> 1) & 1, &abort_sh)) break;
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const uint32_t taddr = tmem + ((uint32_t)(quarter * 32) << 16) + acc * BN + cb0 * 32;
#pragma unroll 1
            for (int k = 0; k < NCB; ++k) {
                if (k > 0) load_block(col0 + 32 * k, old);
                tc::tmem_ld32(taddr + 32 * k, v);
                if (k == NCB - 1) {
                    // this warp's TMEM reads of the accumulator are done
                    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
                    __syncwarp();
                    if (lane == 0) tc::mbar_arrive(&acce_bar[acc]);
                }
                store_block(col0 + 32 * k, old, v);
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == MMA_WARP)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                     "r"(TMEM_COLS));
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------

typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*,
                                  const cuuint64_t*, const cuuint64_t*, const cuuint32_t*,
                                  const cuuint32_t*, CUtensorMapInterleave, CUtensorMapSwizzle,
                                  CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static EncodeTiledFn encode_fn() {
    static EncodeTiledFn fn = nullptr;
    if (!fn) {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
                cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<EncodeTiledFn>(p);
    }
    return fn;
}

// One tensor map per large front, over its panel scratch (row-major: kScrCols
// columns -- two panels side by side -- the inner dimension, of 2 KB (TF32)
// or 1 KB (BF16) per row):
// 3xTF32, FP32 values, 2 mpad rows (hi then lo); BF16, BF16 values, mpad
// rows.  Boxes of 128 bytes of columns x 128 rows with the 128-byte swizzle;
// reads past the rows return zeros.
int build_panel_maps(const Plan& P, const float* base, const std::vector<int64_t>& scr_off,
                     std::vector<CUtensorMap>& maps, std::vector<int>& idx, bool bf16) {
    EncodeTiledFn enc = encode_fn();
    if (!enc) return -1;
    maps.resize(P.large_list.size());
    idx.assign(P.nsuper, -1);
    for (size_t q = 0; q < P.large_list.size(); ++q) {
        const int s = P.large_list[q];
        const FrontDesc& f = P.fronts[s];
        idx[s] = (int)q;
        const int mpad = panel_mpad(f.m);
        const int esz = bf16 ? 2 : 4;
        cuuint64_t dims[2] = {(cuuint64_t)kScrCols, (cuuint64_t)(bf16 ? mpad : 2 * mpad)};
        cuuint64_t strides[1] = {(cuuint64_t)kScrCols * esz};
        cuuint32_t box[2] = {(cuuint32_t)(bf16 ? tc::Cfg<kSchurBF16>::BK
                                               : tc::Cfg<kSchur3xTF32>::BK),
                             (cuuint32_t)tc::BM};
        cuuint32_t estr[2] = {1, 1};
        void* ptr = const_cast<float*>(base + scr_off[s]);
        CUresult r = enc(&maps[q],
                         bf16 ? CU_TENSOR_MAP_DATA_TYPE_BFLOAT16 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32,
                         2, ptr, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                         CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                         CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
        if (r != CUDA_SUCCESS) return -2;
    }
    return 0;
}

void init_schur_tc() {
    cudaFuncSetAttribute(k_schur_tc<kSchur3xTF32>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         tc::Cfg<kSchur3xTF32>::SMEM_BYTES);
    cudaFuncSetAttribute(k_schur_tc<kSchurBF16>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         tc::Cfg<kSchurBF16>::SMEM_BYTES);
    cudaFuncSetAttribute(k_schur_tc<kSchur1xTF32>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         tc::Cfg<kSchur1xTF32>::SMEM_BYTES);
}

template <int MODE>
static void launch_schur_mode(const DevPlan& D, const WorkList& w, int panel, int PW, int upd,
                              float* Ls, float* Us, int* err, const CUtensorMap* maps,
                              cudaStream_t st) {
    using C = tc::Cfg<MODE>;
    const int sms = D.num_sms > 0 ? D.num_sms : 148;
    k_schur_tc<MODE><<<std::min(w.nctas, sms * C::CTAS_PER_SM), C::NTHREADS, C::SMEM_BYTES, st>>>(
        D.fronts, D.psched.items + w.off, D.psched.before + w.off, w.nitems, w.nctas, D.tmap_idx,
        maps, panel, PW, upd, Ls, Us, err);
}

void launch_schur_tc(const DevPlan& D, const WorkList& w, int panel, int PW, int npan,
                     bool strip, float* Ls, float* Us, int* err, int mode, cudaStream_t st) {
    const int upd = npan | (strip ? 16 : 0);
    if (mode == kSchurBF16)
        launch_schur_mode<kSchurBF16>(D, w, panel, PW, upd, Ls, Us, err, D.tmaps_bf16, st);
    else if (mode == kSchur1xTF32)
        launch_schur_mode<kSchur1xTF32>(D, w, panel, PW, upd, Ls, Us, err, D.tmaps, st);
    else
        launch_schur_mode<kSchur3xTF32>(D, w, panel, PW, upd, Ls, Us, err, D.tmaps, st);
}

}  // namespace mdgpu
