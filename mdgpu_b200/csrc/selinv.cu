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
// extend-add).  So the fronts are processed level by level from the root,
// one CTA per front; Z of the pivot columns goes to a store laid out like the
// L panels, Z_UU to the update store (the factor's update matrices are no
// longer needed).
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

void launch_selinv(const DevPlan& D, const double* Ls, double* Zs, double* Zu, double* Yscr,
                   cudaStream_t st) {
    for (int l = D.nlevels - 1; l >= 0; --l) {
        const int b = D.h_level_ptr[l], e = D.h_level_ptr[l + 1];
        if (e > b)
            k_selinv_front<<<e - b, 256, 0, st>>>(D.fronts, D.level_list + b, D.relmap, Ls, Zs, Zu,
                                                  D.zuoff, Yscr, D.yoff);
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

}  // namespace mdgpu
