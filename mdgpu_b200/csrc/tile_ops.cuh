// 64 x 64 tile operations shared by the large-front factor kernels: the
// diagonal-tile Cholesky with its inverse, and the register-tiled products
// C -= A B' over 256 threads (a 4 x 4 block of outputs each).
#pragma once

#include <cuda_runtime.h>

#include "device_common.cuh"

namespace mdgpu {

__device__ __forceinline__ float recip_sqrt(float x) { return rsqrtf(x); }
__device__ __forceinline__ double recip_sqrt(double x) { return rsqrt(x); }

// Leading dimension of the diagonal-tile factorization's S and W: a 4x4
// block's columns are 16-byte vectors (4 floats or 2 x 2 doubles).
constexpr int kPotrfLD = 64 + 4;

// a 4x4 block at (r0, c0) of a kPotrfLD column-major array, in and out
template <typename T>
__device__ __forceinline__ void blk_ld(const T* M, int r0, int c0, T (&b)[4][4]) {
#pragma unroll
    for (int c = 0; c < 4; ++c) {
        const T* p = M + r0 + (c0 + c) * kPotrfLD;
        if constexpr (sizeof(T) == 4) {
            const float4 v = *reinterpret_cast<const float4*>(p);
            b[0][c] = v.x, b[1][c] = v.y, b[2][c] = v.z, b[3][c] = v.w;
        } else {
            const double2 v0 = *reinterpret_cast<const double2*>(p);
            const double2 v1 = *reinterpret_cast<const double2*>(p + 2);
            b[0][c] = v0.x, b[1][c] = v0.y, b[2][c] = v1.x, b[3][c] = v1.y;
        }
    }
}
template <typename T>
__device__ __forceinline__ void blk_st(T* M, int r0, int c0, const T (&b)[4][4]) {
#pragma unroll
    for (int c = 0; c < 4; ++c) {
        T* p = M + r0 + (c0 + c) * kPotrfLD;
        if constexpr (sizeof(T) == 4) {
            *reinterpret_cast<float4*>(p) = make_float4(b[0][c], b[1][c], b[2][c], b[3][c]);
        } else {
            *reinterpret_cast<double2*>(p) = make_double2(b[0][c], b[1][c]);
            *reinterpret_cast<double2*>(p + 2) = make_double2(b[2][c], b[3][c]);
        }
    }
}

// Factor a 4x4 diagonal block in registers: a -> L (lower, zeros above), y =
// inv(L).  One reciprocal square root per pivot (d = piv / sqrt(piv)); a
// non-positive (or NaN) pivot of a row < n is recorded at global column
// col0 + row0 + i.
template <typename T>
__device__ __forceinline__ void diag4(T (&a)[4][4], T (&y)[4][4], int row0, int n, int col0,
                                      int* status) {
#pragma unroll
    for (int r = 0; r < 4; ++r)
#pragma unroll
        for (int c = 0; c < 4; ++c) y[r][c] = T(0);
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const T piv = a[i][i];
        if (row0 + i < n && !(piv > T(0))) flag_pivot(status, col0 + row0 + i);
        const T rd = recip_sqrt(piv);
        a[i][i] = piv * rd;
        y[i][i] = rd;
#pragma unroll
        for (int r = i + 1; r < 4; ++r) a[r][i] *= rd;
#pragma unroll
        for (int r = i + 1; r < 4; ++r)
#pragma unroll
            for (int c = i + 1; c <= r; ++c) a[r][c] -= a[r][i] * a[c][i];
    }
#pragma unroll
    for (int c = 0; c < 4; ++c)
#pragma unroll
        for (int r = c + 1; r < 4; ++r) {
            T v = T(0);
#pragma unroll
            for (int m = c; m < r; ++m) v -= a[r][m] * y[m][c];
            y[r][c] = v * y[r][r];
        }
#pragma unroll
    for (int r = 0; r < 4; ++r)
#pragma unroll
        for (int c = r + 1; c < 4; ++c) a[r][c] = T(0);
}

// Cholesky of the TB x TB tile held in S (lower part; a partial tile of n <
// TB rows padded with the identity) and its inverse.  On exit S holds L in
// its lower blocks and W holds inv(L) in its lower blocks (the blocks above
// the diagonal of W are not written); S, W: TB x kPotrfLD, column-major.
// The tile is a 16 x 16 grid of 4 x 4 blocks held in registers: threads
// 0..119 own the strictly lower blocks (column by column: block (tr, tc)
// and its block of X = inv(L)), lanes 0..15 of warp 7 the diagonal blocks,
// so the chain of diagonal factors runs on one warp that no other block's
// work makes diverge.  Sixteen blocked steps of right-looking Cholesky with
// the inverse alongside, two barriers each:
//   (b) the owners of column kb form their panel block A Y' (Y = the
//       inverse of diagonal block kb); the owners of block row kb of X
//       finalise it, X(kb, tc) = Y x;
//   (c) every lower block right of the panel takes the rank-4 update, the
//       X blocks below take x -= L(tr, kb) X(kb, tc), and the diagonal
//       owners update their blocks -- the owner of block kb + 1 factoring it
//       at once (L and Y to S and W for the next step).
// Starts and ends with a CTA barrier.
template <typename T, int TB>
__device__ void potrf_tile_core(T* S, T* W, int n, int col0, int* status) {
    static_assert(TB == 64 && TB + 4 == kPotrfLD, "16 x 16 grid of 4 x 4 blocks over 256 threads");
    constexpr int B = 4, NB = TB / B, NSTRICT = NB * (NB - 1) / 2, DIAG0 = 224;
    const int tid = threadIdx.x;
    const bool strict = tid < NSTRICT;
    const bool diag = tid >= DIAG0 && tid < DIAG0 + NB;
    int tr = 0, tc = 0;
    if (strict) {  // column-major order of the strictly lower blocks
        int p = tid;
        while (p >= NB - 1 - tc) p -= NB - 1 - tc, ++tc;
        tr = tc + 1 + p;
    } else if (diag) {
        tr = tc = tid - DIAG0;
    }
    __syncthreads();
    T a[B][B], x[B][B];
#pragma unroll
    for (int r = 0; r < B; ++r)
#pragma unroll
        for (int c = 0; c < B; ++c) a[r][c] = x[r][c] = T(0);
    if (strict || diag) blk_ld(S, B * tr, B * tc, a);
    __syncthreads();
    if (diag && tr == 0) {
        T y[B][B];
        diag4(a, y, 0, n, col0, status);
        blk_st(S, 0, 0, a);
        blk_st(W, 0, 0, y);
    }
    __syncthreads();
#pragma unroll 1
    for (int kb = 0; kb < NB; ++kb) {
        if (strict) {
            if (tc == kb) {  // (b) panel block: A Y'
                T y[B][B], o[B][B];
                blk_ld(W, B * kb, B * kb, y);
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
                    for (int c = 0; c < B; ++c) a[r][c] = o[r][c];
                blk_st(S, B * tr, B * kb, a);
            } else if (tr == kb) {  // (b) inverse block row kb: Y x
                T y[B][B], o[B][B];
                blk_ld(W, B * kb, B * kb, y);
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
                    for (int c = 0; c < B; ++c) x[r][c] = o[r][c];
                blk_st(W, B * kb, B * tc, x);
            }
        }
        __syncthreads();
        if (diag && tr > kb) {  // (c) own diagonal block; the next one factored at once
            T p[B][B];
            blk_ld(S, B * tr, B * kb, p);
#pragma unroll
            for (int r = 0; r < B; ++r)
#pragma unroll
                for (int c = 0; c <= r; ++c)
#pragma unroll
                    for (int m = 0; m < B; ++m) a[r][c] -= p[r][m] * p[c][m];
            if (tr == kb + 1) {
                T y[B][B];
                diag4(a, y, B * tr, n, col0, status);
                blk_st(S, B * tr, B * tr, a);
                blk_st(W, B * tr, B * tr, y);
            }
        } else if (strict && tc > kb) {  // (c) trailing update with the panel
            T p[B][B], q[B][B];
            blk_ld(S, B * tr, B * kb, p);
            blk_ld(S, B * tc, B * kb, q);
#pragma unroll
            for (int r = 0; r < B; ++r)
#pragma unroll
                for (int c = 0; c < B; ++c)
#pragma unroll
                    for (int m = 0; m < B; ++m) a[r][c] -= p[r][m] * q[c][m];
        } else if (strict && tr > kb) {  // (c) inverse rows below: x -= L(tr, kb) X(kb, tc)
            T p[B][B], q[B][B];
            blk_ld(S, B * tr, B * kb, p);
            blk_ld(W, B * kb, B * tc, q);
#pragma unroll
            for (int r = 0; r < B; ++r)
#pragma unroll
                for (int c = 0; c < B; ++c)
#pragma unroll
                    for (int m = 0; m < B; ++m) x[r][c] -= p[r][m] * q[m][c];
        }
        __syncthreads();
    }
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
