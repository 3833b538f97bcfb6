// Tensor-core Schur-complement update for FP32 fronts (TF32 inputs, FP32
// accumulation) on sm_100a: tcgen05.mma with the accumulator in TMEM,
// operands staged in shared memory by TMA.
//
// One CTA computes one 128 x 128 tile (I, J), I >= J, of the trailing part of
// a large front after a pivot panel of K <= PW (256) columns:
//     C(I, J) -= A_I * A_J'      A_I = rows 128I.. of the panel columns
// in 3xTF32: A = hi + lo with hi an exact TF32 value and lo = A - hi, and
// C -= hi*hi' + hi*lo' + lo*hi' (close to FP32 accuracy, which keeps the
// iterative refinement short).  The panel's TRSMs write hi and lo into a
// per-front scratch (column-major, rows hi then lo), so A_I and A_J arrive
// split: a 32-row x 16-column TMA box (rows contiguous, 128 bytes per panel column)
// lands MN-major.  For 32-bit MN-major operands the only UMMA shared-memory
// layout is the 128-byte swizzle with 32-byte atoms (32-byte chunks of each
// 128-byte row permuted by row mod 4, atoms of 4 K-rows); the TMA writes
// exactly that pattern with CU_TENSOR_MAP_SWIZZLE_128B_ATOM_32B.  Four boxes
// make a 128-row x 16-column operand; a stage holds A_hi, B_hi, A_lo, B_lo
// (32 KB), and the K loop runs over 16-column chunks through a 3-stage ring
// (97 KB of shared memory: two CTAs per SM, so one CTA's epilogue overlaps
// the other's MMAs).
//
// Roles: thread 0 issues the TMA loads (refilling a stage once the MMAs that
// read it have completed), thread 32 issues the MMAs (single-issued per
// CTA) and commits each stage back to the producer; then all 128 threads
// read the accumulator out of TMEM (warp w owns TMEM lanes 32w..32w+31 =
// tile rows) and subtract it from C in place -- coalesced along the column.
//
// Every wait on an mbarrier is bounded: on timeout the CTA records an error
// code in *err, drains what it issued (bounded again), frees its TMEM and
// returns; the host reports the error.  The TMA loads never use cluster
// multicast and only ever read this GPU's own memory.
#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>

#include "device_common.cuh"
#include "kernels.hpp"

namespace mdgpu {

namespace tc {

constexpr int BM = 128, BN = 128, BK = 16, STAGES = 3;
constexpr int BOX = 32;                                   // TMA box: 32 rows x BK columns (fp32)
constexpr int STAGE_A = BM * BK * 4, STAGE_B = BN * BK * 4;  // bytes
constexpr int STAGE_TMA = STAGE_A + STAGE_B;              // one of hi / lo: A and B
// per stage: A_hi, B_hi, then A_lo, B_lo at the same offsets + STAGE_TMA
constexpr int STAGE_BYTES = 2 * STAGE_TMA;
constexpr int SMEM_BYTES = STAGES * STAGE_BYTES + 1024;   // + alignment slack
constexpr uint32_t TMEM_COLS = 128;
constexpr long long WAIT_LIMIT = 1ll << 22;               // polls (with backoff) before giving up

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

// bounded wait; false on timeout
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t phase) {
    for (long long i = 0; i < WAIT_LIMIT; ++i) {
        if (mbar_try_wait(bar, phase)) return true;
        if (i > 64) __nanosleep(64);
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

// UMMA shared-memory descriptor: MN-major, 128-byte swizzle with 32-byte
// atoms (layout type 1).  LBO = distance between 32-element (128 B) blocks
// along M/N (one TMA box, BK K-rows x 128 B), SBO = distance between groups
// of 4 K-rows (512 B); version 1 (sm_100).
__device__ __forceinline__ uint64_t make_desc(uint32_t saddr) {
    constexpr uint64_t LBO = BOX * BK * 4, SBO = 512;
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFF);
    d |= (uint64_t)((LBO >> 4) & 0x3FFF) << 16;
    d |= (uint64_t)((SBO >> 4) & 0x3FFF) << 32;
    d |= (uint64_t)1 << 46;  // descriptor version for sm_100
    d |= (uint64_t)1 << 61;  // SWIZZLE_128B_BASE32B
    return d;
}

// instruction descriptor: D f32, A/B tf32, both MN-major, M = 128, N = 128
constexpr uint32_t IDESC = (1u << 4) | (2u << 7) | (2u << 10) | (1u << 15) | (1u << 16) |
                           ((uint32_t)(BN >> 3) << 17) | ((uint32_t)(BM >> 4) << 24);

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

}  // namespace tc

// items/before: one entry per large front; the CTAs of a front enumerate the
// lower 128-tiles (I, J) with J >= J0 = cbeg / 128 in row-major order.
__global__ void __launch_bounds__(128, 2)
    k_schur_tc(const FrontDesc* __restrict__ fronts, const int* __restrict__ items,
               const int* __restrict__ before, int nitems, const int* __restrict__ tmap_idx,
               const CUtensorMap* __restrict__ maps, int panel, int PW,
               float* __restrict__ Ls, float* __restrict__ Us, int* __restrict__ err) {
    using namespace tc;
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    __shared__ __align__(8) uint64_t full_bar[STAGES];
    __shared__ __align__(8) uint64_t empty_bar[STAGES];
    __shared__ __align__(8) uint64_t done_bar;
    __shared__ uint32_t tmem_base_sh;
    __shared__ volatile int abort_sh;

    // 1024-byte aligned in the shared window (the 128-byte swizzle phase)
    unsigned char* smem = smem_raw + ((1024u - (tc::smem_u32(smem_raw) & 1023u)) & 1023u);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int it = find_item(before, nitems, blockIdx.x);
    const int s = items[it];
    const FrontDesc f = fronts[s];
    const CUtensorMap* map = maps + tmap_idx[s];
    const int mpad = panel_mpad(f.m);
    // panel columns [k0, k0 + K); trailing columns start at cbeg
    const int k0 = panel * PW;
    const int K = min(PW, f.c - k0);
    const int cbeg = min(k0 + PW, f.c);
    const int J0 = cbeg / BM;
    int ii, jj;
    lower_index(blockIdx.x - before[it], ii, jj);
    const int I = J0 + ii, J = J0 + jj;
    const int nk = (K + BK - 1) / BK;

    if (tid == 0) {
        for (int q = 0; q < STAGES; ++q) {
            tc::mbar_init(&full_bar[q], 1);
            tc::mbar_init(&empty_bar[q], 1);
        }
        tc::mbar_init(&done_bar, 1);
        abort_sh = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         tc::smem_u32(&tmem_base_sh)),
                     "r"(TMEM_COLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = tmem_base_sh;

    if (tid == 0) {
        // producer: A_hi, B_hi, A_lo, B_lo of each BK-column chunk
        int issued = 0;
        bool ok = true;
        for (int ch = 0; ch < nk; ++ch) {
            const int st = ch % STAGES;
            if (ch >= STAGES && !tc::mbar_wait(&empty_bar[st], ((ch / STAGES) - 1) & 1)) {
                ok = false;
                break;
            }
            if (abort_sh) break;
            unsigned char* a = smem + st * STAGE_BYTES;
            unsigned char* b = a + STAGE_A;
            tc::mbar_expect_tx(&full_bar[st], STAGE_BYTES);
            const int col = ch * BK;
#pragma unroll
            for (int q = 0; q < BM / BOX; ++q) {
                const int ra = I * BM + q * BOX, rb = J * BN + q * BOX;
                tc::tma_load_2d(a + q * BOX * BK * 4, map, &full_bar[st], ra, col);
                tc::tma_load_2d(b + q * BOX * BK * 4, map, &full_bar[st], rb, col);
                tc::tma_load_2d(a + STAGE_TMA + q * BOX * BK * 4, map, &full_bar[st], mpad + ra,
                                col);
                tc::tma_load_2d(b + STAGE_TMA + q * BOX * BK * 4, map, &full_bar[st], mpad + rb,
                                col);
            }
            issued = ch + 1;
        }
        if (!ok) {
            atomicExch(err, 1);
            abort_sh = 1;
        }
        if (!ok || abort_sh) {
            // drain: wait (bounded) for the loads already issued
            for (int ch = 0; ch < issued; ++ch)
                tc::mbar_wait(&full_bar[ch % STAGES], (ch / STAGES) & 1);
        }
    } else if (tid == 32) {
        // MMA issuer
        int committed = 0;
        bool ok = true;
        for (int ch = 0; ch < nk; ++ch) {
            const int st = ch % STAGES;
            if (!tc::mbar_wait(&full_bar[st], (ch / STAGES) & 1)) {
                ok = false;
                break;
            }
            if (abort_sh) break;
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const uint32_t ah = tc::smem_u32(smem + st * STAGE_BYTES);
            const uint32_t bh = ah + STAGE_A;
            const uint32_t al = ah + STAGE_TMA, bl = bh + STAGE_TMA;
#pragma unroll
            for (int t = 0; t < BK / 8; ++t) {
                const uint32_t o = t * 1024;
                tc::mma_tf32(tmem, tc::make_desc(al + o), tc::make_desc(bh + o),
                             (ch > 0 || t > 0) ? 1u : 0u);
                tc::mma_tf32(tmem, tc::make_desc(ah + o), tc::make_desc(bl + o), 1u);
                tc::mma_tf32(tmem, tc::make_desc(ah + o), tc::make_desc(bh + o), 1u);
            }
            tc::mma_commit(&empty_bar[st]);
            committed = ch + 1;
        }
        if (!ok) {
            atomicExch(err, 1);
            abort_sh = 1;
        }
        // completes once every MMA issued above has (a partial accumulator
        // after an abort is not written back)
        if (committed > 0) tc::mma_commit(&done_bar);
    }
    __syncthreads();
    const bool have_acc = nk > 0 && tc::mbar_wait(&done_bar, 0);
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (!have_acc && nk > 0 && tid == 0) atomicExch(err, 2);
    if (have_acc && !abort_sh) {
        const int row = I * BM + warp * 32 + lane;
#pragma unroll 1
        for (int cb = 0; cb < BN / 32; ++cb) {
            float v[32];
            tc::tmem_ld32(tmem + ((uint32_t)(warp * 32) << 16) + cb * 32, v);
            if (row < f.m) {
                // gather all 32 addresses and old values first (independent
                // loads in flight), then write
                float* p[32];
                float old[32];
#pragma unroll
                for (int q = 0; q < 32; ++q) {
                    const int col = J * BN + cb * 32 + q;
                    const bool ok = col >= cbeg && col < f.m && row >= col;
                    p[q] = ok ? front_elem(Ls, Us, f, row, col) : nullptr;
                }
#pragma unroll
                for (int q = 0; q < 32; ++q) old[q] = p[q] ? *p[q] : 0.f;
#pragma unroll
                for (int q = 0; q < 32; ++q)
                    if (p[q]) *p[q] = old[q] - v[q];
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0)
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

// One tensor map per large front over its split panel scratch: 2 * mpad rows
// (hi then lo) x PW panel columns, column-major.
int build_panel_maps(const Plan& P, const float* pscr, const std::vector<int64_t>& pscr_off,
                     int PW, std::vector<CUtensorMap>& maps, std::vector<int>& idx) {
    EncodeTiledFn enc = encode_fn();
    if (!enc) return -1;
    maps.resize(P.large_list.size());
    idx.assign(P.nsuper, -1);
    for (size_t q = 0; q < P.large_list.size(); ++q) {
        int s = P.large_list[q];
        const int mpad = panel_mpad(P.fronts[s].m);
        idx[s] = (int)q;
        cuuint64_t dims[2] = {(cuuint64_t)(2 * mpad), (cuuint64_t)PW};
        cuuint64_t strides[1] = {(cuuint64_t)(2 * mpad) * 4};
        cuuint32_t box[2] = {tc::BOX, tc::BK};
        cuuint32_t estr[2] = {1, 1};
        void* base = const_cast<float*>(pscr + pscr_off[s]);
        CUresult r = enc(&maps[q], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, base, dims, strides, box,
                         estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B_ATOM_32B,
                         CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
        if (r != CUDA_SUCCESS) return -2;
    }
    return 0;
}

void init_schur_tc() {
    cudaFuncSetAttribute(k_schur_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, tc::SMEM_BYTES);
}

void launch_schur_tc(const DevPlan& D, const WorkList& w, int panel, int PW, float* Ls,
                     float* Us, int* err, cudaStream_t st) {
    k_schur_tc<<<w.nctas, 128, tc::SMEM_BYTES, st>>>(D.fronts, D.psched.items + w.off,
                                                     D.psched.before + w.off, w.nitems,
                                                     D.tmap_idx, D.tmaps, panel, PW, Ls, Us,
                                                     err);
}

}  // namespace mdgpu
