// Reverse mode of the multifrontal Cholesky factorization (FP64): from the
// gradient Lbar of a loss with respect to the entries of L (on L's pattern)
// to the gradient Abar with respect to the caller's lower-triangle values.
//
// The factor (the forward structure of Factor, mdgpu.cu:1394-1608) per front
// s with pivot block K (c columns) and update rows R (u rows):
//     F     = A_s + sum over children of extend(U_child)
//     L11   = chol(F11),   L21 = F21 L11^-T,   U = F22 - L21 L21'
// Reversed front by front from the root (all gradients with respect to the
// stored lower entries; an off-diagonal entry stands for both triangles):
//     Ubar  = Fbar of the parent on this front's update rows (the transpose
//             of the extend-add: a gather through the relative map)
//     L21bar -= (Ubar + Ubar') L21
//     F21bar  = L21bar L11^-1
//     L11bar -= tril(F21bar' L21)
//     F11bar  = the Cholesky adjoint of L11 (Murray 2016):
//               P = Phi(L11' L11bar), S = L11^-T P L11^-1,
//               F11bar = tril(S + S') with the diagonal of S
//     F22bar  = Ubar
// and Abar is Fbar at the positions where the front assembly put A's
// entries.  Only L and the gradients flowing down the tree are needed: the
// update matrices are neither stored for the reverse sweep nor recomputed.
//
// Fbar's pivot columns live in a store laid out like the L panels (it starts
// as Lbar, scattered there, and is turned into Fbar in place), Ubar in a
// store with the selected inverse's lifetimes (plan zuoff).  One CTA per
// front and level; the dense steps run in the CTA from global memory (a
// c x c scratch per front for the Cholesky adjoint).
#include <cuda_runtime.h>

#include <cstdint>

#include "device_common.cuh"
#include "kernels.hpp"

namespace mdgpu {

namespace {

// Fbar (r, col), r >= col, front-local, of front f (pivot columns in Fb,
// the update part in Fu at zoff)
__device__ __forceinline__ double fbar_get(const double* __restrict__ Fb,
                                           const double* __restrict__ Fu, const FrontDesc& f,
                                           int64_t zoff, int r, int col) {
    if (col < f.c) return Fb[f.loff + r + (int64_t)col * f.ldl];
    return Fu[zoff + (r - f.c) + (int64_t)(col - f.c) * f.ldu];
}

}  // namespace

// Lbar (CSC of L: column j holds rows j.. in ascending order, diagonal
// first) into the panel store: panel (r, jj) of front s is entry
// Lp[first + jj] + r - jj for r >= jj; zero above the diagonal.
__global__ void __launch_bounds__(256)
    k_adj_scatter(const FrontDesc* __restrict__ fronts, const int64_t* __restrict__ Lp,
                  const double* __restrict__ Lbar, double* __restrict__ Fb) {
    const FrontDesc f = fronts[blockIdx.x];
    for (int jj = 0; jj < f.c; ++jj) {
        const int64_t p0 = Lp[f.first_col + jj];
        double* col = Fb + f.loff + (int64_t)jj * f.ldl;
        for (int r = threadIdx.x; r < f.m; r += blockDim.x) col[r] = r >= jj ? Lbar[p0 + r - jj] : 0.0;
    }
}

// Ubar of front s = Fbar of its parent on s's update rows (lower part)
__global__ void __launch_bounds__(256)
    k_adj_gather(const FrontDesc* __restrict__ fronts, const int* __restrict__ items,
                 const int* __restrict__ before, int nitems, const int* __restrict__ relmap,
                 const double* __restrict__ Fb, double* __restrict__ Fu,
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
            Fu[zf + a + (int64_t)b * f.ldu] = fbar_get(Fb, Fu, p, zp, rm[a], pb);
    }
}

// One front: Lbar (pivot columns of Fb, rows 0..m) -> Fbar in place, with
// Ubar from Fu; W: c x c scratch.
__global__ void __launch_bounds__(256)
    k_adj_front(const FrontDesc* __restrict__ fronts, const int* __restrict__ list,
                const double* __restrict__ Ls, double* __restrict__ Fb,
                const double* __restrict__ Fu, const int64_t* __restrict__ zuoff,
                double* __restrict__ Wscr, const int64_t* __restrict__ woff) {
    const int s = list[blockIdx.x];
    const FrontDesc f = fronts[s];
    const int m = f.m, c = f.c, u = m - c;
    const int tid = threadIdx.x, nt = blockDim.x;
    const double* L = Ls + f.loff;  // L(r, k) = L[r + k ldl]
    double* G = Fb + f.loff;        // Lbar -> Fbar, same layout
    const int64_t zf = (f.parent >= 0 && u > 0) ? zuoff[s] : -1;
    double* W = Wscr + woff[s];     // c x c, column-major
    auto ubar = [&](int a, int b) -> double {  // (Ubar + Ubar')(a, b)
        if (a == b) return 2.0 * Fu[zf + a + (int64_t)a * f.ldu];
        const int hi = a > b ? a : b, lo = a > b ? b : a;
        return Fu[zf + hi + (int64_t)lo * f.ldu];
    };
    if (u > 0) {
        // L21bar -= (Ubar + Ubar') L21: outputs (a, k) (each reads L21 and
        // Ubar only)
        if (zf >= 0) {
            for (int64_t e = tid; e < (int64_t)u * c; e += nt) {
                const int a = (int)(e % u), k = (int)(e / u);
                double v = 0.0;
                for (int b = 0; b < u; ++b) v += ubar(a, b) * L[c + b + (int64_t)k * f.ldl];
                G[c + a + (int64_t)k * f.ldl] -= v;
            }
            __syncthreads();
        }
        // F21bar = L21bar L11^-1: row a solves x L11 = l, columns from last
        for (int a = tid; a < u; a += nt) {
            double* x = G + c + a;
            for (int k = c - 1; k >= 0; --k) {
                double v = x[(int64_t)k * f.ldl];
                for (int j = k + 1; j < c; ++j) v -= x[(int64_t)j * f.ldl] * L[j + (int64_t)k * f.ldl];
                x[(int64_t)k * f.ldl] = v / L[k + (int64_t)k * f.ldl];
            }
        }
        __syncthreads();
        // L11bar -= tril(F21bar' L21)
        for (int64_t e = tid; e < (int64_t)c * c; e += nt) {
            const int i = (int)(e % c), j = (int)(e / c);
            if (i < j) continue;
            double v = 0.0;
            for (int a = 0; a < u; ++a)
                v += G[c + a + (int64_t)i * f.ldl] * L[c + a + (int64_t)j * f.ldl];
            W[i + (int64_t)j * c] = v;
        }
        __syncthreads();
        for (int64_t e = tid; e < (int64_t)c * c; e += nt) {
            const int i = (int)(e % c), j = (int)(e / c);
            if (i >= j) G[i + (int64_t)j * f.ldl] -= W[i + (int64_t)j * c];
        }
        __syncthreads();
    }
    // Cholesky adjoint of the pivot block.  P = Phi(L11' L11bar) into W
    // (lower; P(i, j) = sum over k >= i of L(k, i) Lbar(k, j), diagonal halved)
    for (int64_t e = tid; e < (int64_t)c * c; e += nt) {
        const int i = (int)(e % c), j = (int)(e / c);
        double v = 0.0;
        if (i >= j) {
            for (int k = i; k < c; ++k) v += L[k + (int64_t)i * f.ldl] * G[k + (int64_t)j * f.ldl];
            if (i == j) v *= 0.5;
        }
        W[i + (int64_t)j * c] = v;
    }
    __syncthreads();
    // X = P L^-1: row i solves x L = p (columns from last), in place
    for (int i = tid; i < c; i += nt) {
        for (int k = c - 1; k >= 0; --k) {
            double v = W[i + (int64_t)k * c];
            for (int j = k + 1; j < c; ++j) v -= W[i + (int64_t)j * c] * L[j + (int64_t)k * f.ldl];
            W[i + (int64_t)k * c] = v / L[k + (int64_t)k * f.ldl];
        }
    }
    __syncthreads();
    // S = L^-T X: column j solves L' s = x (rows from last), in place
    for (int j = tid; j < c; j += nt) {
        double* sc = W + (int64_t)j * c;
        for (int k = c - 1; k >= 0; --k) {
            double v = sc[k];
            for (int r = k + 1; r < c; ++r) v -= L[r + (int64_t)k * f.ldl] * sc[r];
            sc[k] = v / L[k + (int64_t)k * f.ldl];
        }
    }
    __syncthreads();
    // F11bar = tril(S + S'), diagonal S(i, i)
    for (int64_t e = tid; e < (int64_t)c * c; e += nt) {
        const int i = (int)(e % c), j = (int)(e / c);
        if (i < j) continue;
        G[i + (int64_t)j * f.ldl] =
            i == j ? W[i + (int64_t)i * c] : W[i + (int64_t)j * c] + W[j + (int64_t)i * c];
    }
}

// Abar of every lower-triangle entry e (caller order; zeroed by the caller):
// Fbar at the front position the assembly gave it
__global__ void k_adj_abar(int nnz, const FrontDesc* __restrict__ fronts,
                           const int* __restrict__ a_front, const int* __restrict__ a_src,
                           const int* __restrict__ a_pos, const double* __restrict__ Fb,
                           double* __restrict__ Abar) {
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < nnz; e += gridDim.x * blockDim.x) {
        const int src = a_src[e];
        if (src < 0) continue;  // a duplicate the assembly drops: gradient 0
        const FrontDesc f = fronts[a_front[e]];
        const int pos = a_pos[e], r = pos & 0xffff, jj = pos >> 16;
        Abar[src] = Fb[f.loff + r + (int64_t)jj * f.ldl];
    }
}

void launch_adjoint(const DevPlan& D, int nnz, const double* Ls, const double* Lbar, double* Fb,
                    double* Fu, double* Wscr, double* Abar, cudaStream_t st) {
    const AdjSchedule& S = D.adj;
    k_adj_scatter<<<D.nsuper, 256, 0, st>>>(D.fronts, S.Lp, Lbar, Fb);
    for (int l = D.nlevels - 1; l >= 0; --l) {
        const WorkList& g = S.h_gather[l];
        if (g.nctas > 0)
            k_adj_gather<<<g.nctas, 256, 0, st>>>(D.fronts, S.items + g.off, S.before + g.off,
                                                  g.nitems, D.relmap, Fb, Fu, D.zuoff);
        const int b = D.h_level_ptr[l], e = D.h_level_ptr[l + 1];
        if (e > b)
            k_adj_front<<<e - b, 256, 0, st>>>(D.fronts, D.level_list + b, Ls, Fb, Fu, D.zuoff,
                                               Wscr, S.woff);
    }
    cudaMemsetAsync(Abar, 0, (size_t)nnz * sizeof(double), st);
    const int blocks = std::max(1, std::min((nnz + 255) / 256, 148 * 8));
    k_adj_abar<<<blocks, 256, 0, st>>>(nnz, D.fronts, D.a_front, D.a_src, D.a_pos, Fb, Abar);
}

}  // namespace mdgpu
