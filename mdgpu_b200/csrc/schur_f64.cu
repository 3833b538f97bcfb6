// FP64 Schur-complement update of a large front after a 256-column pivot
// panel (the FP64 counterpart of the tensor-core kernel in schur_tc.cu, same
// work lists and tile enumeration):
//     C(I, J) -= A_I * A_J'     128 x 128 tile, K <= 256 panel columns
// FP64 has no tcgen05 kind, so this is a register-tiled FMA kernel: 256
// threads, 8 x 8 outputs per thread (rows ty*4+{0..3} and ty*4+64+{0..3},
// columns likewise, which keeps shared-memory reads conflict-free), operand
// chunks of 16 columns double-buffered in shared memory with cp.async.
#include <cuda_runtime.h>

#include <cstdint>

#include "device_common.cuh"
#include "kernels.hpp"

namespace mdgpu {

namespace f64k {
constexpr int BM = 128, KC = 16, THREADS = 256;
constexpr int STAGE = 2 * KC * BM;  // doubles: A and B chunk
constexpr size_t SMEM_BYTES = 2 * STAGE * sizeof(double);
}  // namespace f64k

__device__ __forceinline__ void cp_async16(void* dst, const void* src, int src_bytes) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(
                     static_cast<uint32_t>(__cvta_generic_to_shared(dst))),
                 "l"(src), "r"(src_bytes)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_one() { asm volatile("cp.async.wait_group 1;" ::: "memory"); }

__global__ void __launch_bounds__(256)
    k_schur_f64(const FrontDesc* __restrict__ fronts, const int* __restrict__ items,
                const int* __restrict__ before, int nitems, int panel, int PW,
                double* __restrict__ Ls, double* __restrict__ Us) {
    using namespace f64k;
    extern __shared__ __align__(16) double sm[];
    const int it = find_item(before, nitems, blockIdx.x);
    const FrontDesc f = fronts[items[it]];
    const int k0 = panel * PW;
    const int K = min(PW, f.c - k0);
    const int cbeg = min(k0 + PW, f.c);
    int ii, jj;
    lower_index(blockIdx.x - before[it], ii, jj);
    const int I = cbeg / BM + ii, J = cbeg / BM + jj;
    const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
    const double* panelp = Ls + f.loff;
    const int nchunks = (K + KC - 1) / KC;

    // each thread copies 4 x 16 bytes of A and 4 x 16 bytes of B per chunk:
    // element pair (row 2*(tid & 63), column (tid >> 6) + 4*u)
    auto load_chunk = [&](int ch, int stage) {
        double* As = sm + stage * STAGE;
        double* Bs = As + KC * BM;
        const int r2 = (tid & 63) * 2;
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int q = (tid >> 6) + 4 * u;  // chunk column
            const int col = k0 + ch * KC + q;
            const bool colok = (ch * KC + q) < K;
            const int ra = I * BM + r2, rb = J * BM + r2;
            // rows beyond the front (or a partial pair) and columns beyond the
            // panel are zero-filled; the source address then stays in bounds
            const int na = (colok && ra < f.m) ? min(2, f.m - ra) * 8 : 0;
            const int nb = (colok && rb < f.m) ? min(2, f.m - rb) * 8 : 0;
            const double* sa = panelp + (na ? (int64_t)col * f.ldl + ra : 0);
            const double* sb = panelp + (nb ? (int64_t)col * f.ldl + rb : 0);
            cp_async16(As + q * BM + r2, sa, na);
            cp_async16(Bs + q * BM + r2, sb, nb);
        }
        cp_async_commit();
    };

    double acc[8][8];
#pragma unroll
    for (int a = 0; a < 8; ++a)
#pragma unroll
        for (int b = 0; b < 8; ++b) acc[a][b] = 0.0;

    load_chunk(0, 0);
    for (int ch = 0; ch < nchunks; ++ch) {
        if (ch + 1 < nchunks) {
            load_chunk(ch + 1, (ch + 1) & 1);
            cp_async_wait_one();
        } else {
            cp_async_wait_all();
        }
        __syncthreads();
        const double* As = sm + (ch & 1) * STAGE;
        const double* Bs = As + KC * BM;
#pragma unroll 4
        for (int q = 0; q < KC; ++q) {
            const double2* ar = reinterpret_cast<const double2*>(As + q * BM);
            const double2* br = reinterpret_cast<const double2*>(Bs + q * BM);
            double2 a0 = ar[ty * 2], a1 = ar[ty * 2 + 1], a2 = ar[32 + ty * 2],
                    a3 = ar[32 + ty * 2 + 1];
            double2 b0 = br[tx * 2], b1 = br[tx * 2 + 1], b2 = br[32 + tx * 2],
                    b3 = br[32 + tx * 2 + 1];
            const double av[8] = {a0.x, a0.y, a1.x, a1.y, a2.x, a2.y, a3.x, a3.y};
            const double bv[8] = {b0.x, b0.y, b1.x, b1.y, b2.x, b2.y, b3.x, b3.y};
#pragma unroll
            for (int a = 0; a < 8; ++a)
#pragma unroll
                for (int b = 0; b < 8; ++b) acc[a][b] = fma(av[a], bv[b], acc[a][b]);
        }
        __syncthreads();
    }
    // epilogue: gather addresses and old values of a row, then write
#pragma unroll
    for (int a = 0; a < 8; ++a) {
        const int row = I * BM + (a < 4 ? ty * 4 + a : 64 + ty * 4 + (a - 4));
        if (row >= f.m) continue;
        double* p[8];
        double old[8];
#pragma unroll
        for (int b = 0; b < 8; ++b) {
            const int col = J * BM + (b < 4 ? tx * 4 + b : 64 + tx * 4 + (b - 4));
            const bool ok = col >= cbeg && col < f.m && row >= col;
            p[b] = ok ? front_elem(Ls, Us, f, row, col) : nullptr;
        }
#pragma unroll
        for (int b = 0; b < 8; ++b) old[b] = p[b] ? *p[b] : 0.0;
#pragma unroll
        for (int b = 0; b < 8; ++b)
            if (p[b]) *p[b] = old[b] - acc[a][b];
    }
}

void init_schur_f64() {
    cudaFuncSetAttribute(k_schur_f64, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)f64k::SMEM_BYTES);
}

void launch_schur_f64(const DevPlan& D, const WorkList& w, int panel, int PW, double* Ls,
                      double* Us, cudaStream_t st) {
    k_schur_f64<<<w.nctas, f64k::THREADS, f64k::SMEM_BYTES, st>>>(
        D.fronts, D.psched.items + w.off, D.psched.before + w.off, w.nitems, panel, PW, Ls, Us);
}

}  // namespace mdgpu
