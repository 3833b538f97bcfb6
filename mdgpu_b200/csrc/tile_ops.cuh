// 64 x 64 tile operations shared by the large-front factor kernels: the
// diagonal-tile Cholesky with its inverse, and the register-tiled products
// C -= A B' over 256 threads (a 4 x 4 block of outputs each).
#pragma once

#include <cuda_runtime.h>

#include "device_common.cuh"

namespace mdgpu {

__device__ __forceinline__ float recip_sqrt(float x) { return rsqrtf(x); }
__device__ __forceinline__ double recip_sqrt(double x) { return rsqrt(x); }

// Cholesky of the TB x TB tile held in S (lower part; a partial tile of n <
// TB rows padded with the identity) and its inverse.  On exit S holds L in
// its lower blocks and W holds inv(L) in its lower blocks (the blocks above
// the diagonal of W are not written); S, W: TB x (TB + 1), column-major.
// The 256 threads form a 16 x 16 grid; thread (tr, tc), tr >= tc, keeps the
// 4 x 4 block (tr, tc) of the tile in registers, and its block of X = inv(L).
// Sixteen blocked steps (two barriers each) of right-looking Cholesky with
// the inverse alongside:
//   (a) the diagonal owner factors its 4 x 4 block and inverts it (Y);
//   (b) the owners below it form their panel block A Y'; at the same time
//       the owners of block row kb of X finalise it, X(kb, tc) = Y x;
//   (c) every lower block right of the panel takes the rank-4 update; at the
//       same time the X blocks below take x -= L(tr, kb) X(kb, tc);
// with L going to S and X to W block by block.  One reciprocal square root
// per pivot; a non-positive (or NaN) pivot of row r < n is recorded at
// global column col0 + r.  Starts and ends with a CTA barrier.
template <typename T, int TB>
__device__ void potrf_tile_core(T* S, T* W, int n, int col0, int* status) {
    static_assert(TB == 64, "16 x 16 grid of 4 x 4 blocks over 256 threads");
    constexpr int LD = TB + 1, B = 4, NB = TB / B;
    const int tid = threadIdx.x;
    const int tr = tid & (NB - 1), tc = tid >> 4;
    const bool low = tr >= tc;
    __syncthreads();
    T a[B][B], x[B][B];  // this thread's block of A -> L, and of inv(L)
#pragma unroll
    for (int r = 0; r < B; ++r)
#pragma unroll
        for (int c = 0; c < B; ++c) {
            a[r][c] = low ? S[(B * tr + r) + (B * tc + c) * LD] : T(0);
            x[r][c] = (tr == tc && r == c) ? T(1) : T(0);
        }
    __syncthreads();
#pragma unroll 1
    for (int kb = 0; kb < NB; ++kb) {
        if (tr == kb && tc == kb) {  // (a) L_kk and its inverse Y = X(kb, kb)
#pragma unroll
            for (int i = 0; i < B; ++i) {
                const T piv = a[i][i];
                if (B * kb + i < n && !(piv > T(0))) flag_pivot(status, col0 + B * kb + i);
                // one reciprocal square root per pivot: d = piv / sqrt(piv)
                const T rd = recip_sqrt(piv);
                const T d = piv * rd;
                a[i][i] = d;
                x[i][i] = rd;  // diagonal of Y
#pragma unroll
                for (int r = i + 1; r < B; ++r) a[r][i] *= rd;
#pragma unroll
                for (int r = i + 1; r < B; ++r)
#pragma unroll
                    for (int c = i + 1; c <= r; ++c) a[r][c] -= a[r][i] * a[c][i];
            }
            // Y = inv(L_kk) by forward substitution, column by column
#pragma unroll
            for (int c = 0; c < B; ++c)
#pragma unroll
                for (int r = c + 1; r < B; ++r) {
                    T v = T(0);
#pragma unroll
                    for (int m = c; m < r; ++m) v -= a[r][m] * x[m][c];
                    x[r][c] = v * x[r][r];
                }
#pragma unroll
            for (int r = 0; r < B; ++r)
#pragma unroll
                for (int c = 0; c < B; ++c) {
                    S[(B * kb + r) + (B * kb + c) * LD] = (c <= r) ? a[r][c] : T(0);
                    W[(B * kb + r) + (B * kb + c) * LD] = (c <= r) ? x[r][c] : T(0);
                }
        }
        __syncthreads();
        if (tc == kb && tr > kb) {  // (b) panel block: A Y'
            T y[B][B];
#pragma unroll
            for (int r = 0; r < B; ++r)
#pragma unroll
                for (int c = 0; c < B; ++c) y[r][c] = W[(B * kb + r) + (B * kb + c) * LD];
            T o[B][B];
#pragma unroll
            for (int r = 0; r < B; ++r)
#pragma unroll
                for (int c = 0; c < B; ++c) {
                    T v = T(0);
#pragma unroll
                    for (int m = 0; m <= c; ++m) v += a[r][m] * y[c][m];
                    o[r][c] = v;
                }
#pragma unroll
            for (int r = 0; r < B; ++r)
#pragma unroll
                for (int c = 0; c < B; ++c) {
                    a[r][c] = o[r][c];
                    S[(B * tr + r) + (B * kb + c) * LD] = o[r][c];
                }
        } else if (tr == kb && tc < kb) {  // (b) inverse block row kb: X = Y x
            T y[B][B];
#pragma unroll
            for (int r = 0; r < B; ++r)
#pragma unroll
                for (int c = 0; c < B; ++c) y[r][c] = W[(B * kb + r) + (B * kb + c) * LD];
            T o[B][B];
#pragma unroll
            for (int r = 0; r < B; ++r)
#pragma unroll
                for (int c = 0; c < B; ++c) {
                    T v = T(0);
#pragma unroll
                    for (int m = 0; m <= r; ++m) v += y[r][m] * x[m][c];
                    o[r][c] = v;
                }
#pragma unroll
            for (int r = 0; r < B; ++r)
#pragma unroll
                for (int c = 0; c < B; ++c) {
                    x[r][c] = o[r][c];
                    W[(B * kb + r) + (B * tc + c) * LD] = o[r][c];
                }
        }
        __syncthreads();
        if (tc > kb && low) {  // (c) trailing update with the panel
            T p[B][B], q[B][B];
#pragma unroll
            for (int r = 0; r < B; ++r)
#pragma unroll
                for (int m = 0; m < B; ++m) {
                    p[r][m] = S[(B * tr + r) + (B * kb + m) * LD];
                    q[r][m] = S[(B * tc + r) + (B * kb + m) * LD];
                }
#pragma unroll
            for (int r = 0; r < B; ++r)
#pragma unroll
                for (int c = 0; c < B; ++c)
#pragma unroll
                    for (int m = 0; m < B; ++m) a[r][c] -= p[r][m] * q[c][m];
        } else if (tr > kb && tc <= kb) {  // (c) inverse rows below: x -= L(tr, kb) X(kb, tc)
            T p[B][B], q[B][B];
#pragma unroll
            for (int r = 0; r < B; ++r)
#pragma unroll
                for (int m = 0; m < B; ++m) {
                    p[r][m] = S[(B * tr + r) + (B * kb + m) * LD];
                    q[m][r] = W[(B * kb + m) + (B * tc + r) * LD];
                }
#pragma unroll
            for (int r = 0; r < B; ++r)
#pragma unroll
                for (int c = 0; c < B; ++c)
#pragma unroll
                    for (int m = 0; m < B; ++m) x[r][c] -= p[r][m] * q[m][c];
        }
    }
    __syncthreads();
}

// acc = sum over q < K of As[q][r0 + a] * Bs[q][c0 + b] (As, Bs: K x TB,
// row q at q * TB), r0 = 4 (tid mod 16), c0 = 4 (tid / 16).
template <typename T, int TB>
__device__ void tile_gemm_nt_acc(const T* As, const T* Bs, int K, T (&acc)[4][4]) {
    const int tid = threadIdx.x;
    const int r0 = (tid & 15) * 4, c0 = (tid >> 4) * 4;
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
}

// acc += the full-K (TB) product of two TB x TB blocks, as tile_gemm_nt_acc;
// both blocks 16-byte aligned, so each thread reads its four rows and four
// columns of a K step with vector loads.
template <typename T, int TB>
__device__ __forceinline__ void tile_gemm_nt_add(const T* __restrict__ As,
                                                 const T* __restrict__ Bs, T (&acc)[4][4]) {
    const int tid = threadIdx.x;
    const int r0 = (tid & 15) * 4, c0 = (tid >> 4) * 4;
#pragma unroll 4
    for (int q = 0; q < TB; ++q) {
        T av[4], bv[4];
        if constexpr (sizeof(T) == 4) {
            const float4 a4 = *reinterpret_cast<const float4*>(As + q * TB + r0);
            const float4 b4 = *reinterpret_cast<const float4*>(Bs + q * TB + c0);
            av[0] = a4.x, av[1] = a4.y, av[2] = a4.z, av[3] = a4.w;
            bv[0] = b4.x, bv[1] = b4.y, bv[2] = b4.z, bv[3] = b4.w;
        } else {
            const double2 a0 = *reinterpret_cast<const double2*>(As + q * TB + r0);
            const double2 a1 = *reinterpret_cast<const double2*>(As + q * TB + r0 + 2);
            const double2 b0 = *reinterpret_cast<const double2*>(Bs + q * TB + c0);
            const double2 b1 = *reinterpret_cast<const double2*>(Bs + q * TB + c0 + 2);
            av[0] = a0.x, av[1] = a0.y, av[2] = a1.x, av[3] = a1.y;
            bv[0] = b0.x, bv[1] = b0.y, bv[2] = b1.x, bv[3] = b1.y;
        }
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
            for (int b = 0; b < 4; ++b) acc[a][b] += av[a] * bv[b];
    }
}

}  // namespace mdgpu
