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
#include "device_common.cuh"
#include "kernels.hpp"

namespace mdgpu {

template <typename TV>
__device__ inline TV* front_vec(TV* fv, const int64_t* fv_off, int s, int nrhs) {
    return fv + fv_off[s] * nrhs;
}

// ---------------------------------------------------------------------------
// small fronts
// ---------------------------------------------------------------------------

template <typename TL, typename TV>
__global__ void __launch_bounds__(128)
    k_fwd_small(const FrontDesc* __restrict__ fronts, const int* __restrict__ list,
                const int* __restrict__ child, const int* __restrict__ relmap,
                const int64_t* __restrict__ fv_off, const TL* __restrict__ Ls, TV* __restrict__ xp,
                TV* __restrict__ fv, int n, int nrhs) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    TV* f = reinterpret_cast<TV*>(smem_raw);
    const int s = list[blockIdx.x];
    const FrontDesc F = fronts[s];
    const int m = F.m, c = F.c;
    const int tid = threadIdx.x, nt = blockDim.x;
    const TL* L = Ls + F.loff;
    for (int idx = tid; idx < m * nrhs; idx += nt) {
        int q = idx / m, r = idx - q * m;
        f[idx] = r < c ? xp[F.first_col + r + (int64_t)q * n] : TV(0);
    }
    __syncthreads();
    for (int h = F.child_beg; h < F.child_end; ++h) {
        const int ch = child[h];
        const FrontDesc g = fronts[ch];
        const int uc = g.m - g.c;
        const TV* w = front_vec(fv, fv_off, ch, nrhs);
        const int* rm = relmap + g.rows_off + g.c;
        for (int idx = tid; idx < uc * nrhs; idx += nt) {
            int q = idx / uc, r = idx - q * uc;
            f[rm[r] + q * m] += w[g.c + r + q * g.m];
        }
        __syncthreads();
    }
    for (int j = 0; j < c; ++j) {
        const TV inv = TV(1) / (TV)L[j + (int64_t)j * F.ldl];
        for (int q = tid; q < nrhs; q += nt) f[j + q * m] *= inv;
        __syncthreads();
        const int rows = m - j - 1;
        for (int idx = tid; idx < rows * nrhs; idx += nt) {
            int q = idx / rows, r = j + 1 + (idx - q * rows);
            f[r + q * m] -= (TV)L[r + (int64_t)j * F.ldl] * f[j + q * m];
        }
        __syncthreads();
    }
    TV* out = front_vec(fv, fv_off, s, nrhs);
    for (int idx = tid; idx < m * nrhs; idx += nt) {
        int q = idx / m, r = idx - q * m;
        if (r < c)
            xp[F.first_col + r + (int64_t)q * n] = f[idx];
        else
            out[idx] = f[idx];
    }
}

template <typename TL, typename TV>
__global__ void __launch_bounds__(128)
    k_bwd_small(const FrontDesc* __restrict__ fronts, const int* __restrict__ list,
                const int* __restrict__ rows, const TL* __restrict__ Ls, TV* __restrict__ xp, int n,
                int nrhs, int umax) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    TV* xb = reinterpret_cast<TV*>(smem_raw);  // u x nrhs
    TV* t = xb + (size_t)umax * nrhs;          // c x nrhs
    const int s = list[blockIdx.x];
    const FrontDesc F = fronts[s];
    const int m = F.m, c = F.c, u = m - c;
    const int tid = threadIdx.x, nt = blockDim.x;
    const int lane = tid & 31, warp = tid >> 5, nw = nt >> 5;
    const TL* L = Ls + F.loff;
    const int* rw = rows + F.rows_off + c;
    for (int idx = tid; idx < u * nrhs; idx += nt) {
        int q = idx / u, r = idx - q * u;
        xb[idx] = xp[rw[r] + (int64_t)q * n];
    }
    for (int idx = tid; idx < c * nrhs; idx += nt) {
        int q = idx / c, j = idx - q * c;
        t[idx] = xp[F.first_col + j + (int64_t)q * n];
    }
    __syncthreads();
    for (int j = warp; j < c; j += nw) {
        const TL* col = L + c + (int64_t)j * F.ldl;
        for (int q = 0; q < nrhs; ++q) {
            TV acc = TV(0);
            for (int r = lane; r < u; r += 32) acc += (TV)col[r] * xb[r + q * u];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
            if (lane == 0) t[j + q * c] -= acc;
        }
    }
    __syncthreads();
    for (int j = c - 1; j >= 0; --j) {
        const TV inv = TV(1) / (TV)L[j + (int64_t)j * F.ldl];
        for (int q = tid; q < nrhs; q += nt) t[j + q * c] *= inv;
        __syncthreads();
        for (int idx = tid; idx < j * nrhs; idx += nt) {
            int q = idx / j, l = idx - q * j;
            t[l + q * c] -= (TV)L[j + (int64_t)l * F.ldl] * t[j + q * c];
        }
        __syncthreads();
    }
    for (int idx = tid; idx < c * nrhs; idx += nt) {
        int q = idx / c, j = idx - q * c;
        xp[F.first_col + j + (int64_t)q * n] = t[idx];
    }
}

// ---------------------------------------------------------------------------
// large fronts
// ---------------------------------------------------------------------------

template <typename TV>
__global__ void __launch_bounds__(256)
    k_fwd_assemble(const FrontDesc* __restrict__ fronts, const int* __restrict__ list,
                   const int* __restrict__ child, const int* __restrict__ relmap,
                   const int64_t* __restrict__ fv_off, const TV* __restrict__ xp,
                   TV* __restrict__ fv, int n, int nrhs) {
    const int s = list[blockIdx.x];
    const FrontDesc F = fronts[s];
    const int m = F.m, c = F.c;
    const int tid = threadIdx.x, nt = blockDim.x;
    TV* f = front_vec(fv, fv_off, s, nrhs);
    for (int idx = tid; idx < m * nrhs; idx += nt) {
        int q = idx / m, r = idx - q * m;
        f[idx] = r < c ? xp[F.first_col + r + (int64_t)q * n] : TV(0);
    }
    __syncthreads();
    for (int h = F.child_beg; h < F.child_end; ++h) {
        const int ch = child[h];
        const FrontDesc g = fronts[ch];
        const int uc = g.m - g.c;
        const TV* w = front_vec(fv, fv_off, ch, nrhs);
        const int* rm = relmap + g.rows_off + g.c;
        for (int idx = tid; idx < uc * nrhs; idx += nt) {
            int q = idx / uc, r = idx - q * uc;
            f[rm[r] + q * m] += w[g.c + r + q * g.m];
        }
        __syncthreads();
    }
}

// y = inv(L_kk) f or x = inv(L_kk)' t for one pivot tile, with the inverse
// stored by the factorization (Dk: T x T column-major, zero above the
// diagonal); in and out are nk x nrhs in shared memory.
template <typename TV>
__device__ void apply_tile_inverse(const TV* Dk, const TV* in, TV* out, int nk, int nrhs,
                                   bool transpose) {
    constexpr int T = kTile;
    for (int idx = threadIdx.x; idx < nk * nrhs; idx += blockDim.x) {
        int q = idx / nk, r = idx - q * nk;
        const TV* v = in + q * nk;
        TV acc = TV(0);
        if (!transpose) {
            for (int l = 0; l <= r; ++l) acc += Dk[r + l * T] * v[l];
        } else {
            for (int l = r; l < nk; ++l) acc += Dk[l + r * T] * v[l];
        }
        out[idx] = acc;
    }
    __syncthreads();
}

template <typename TL, typename TV>
__global__ void __launch_bounds__(256)
    k_fwd_step(const FrontDesc* __restrict__ fronts, const int* __restrict__ items,
               const int* __restrict__ before, int nitems, int kb,
               const int64_t* __restrict__ fv_off, const int64_t* __restrict__ dinv_off,
               const TL* __restrict__ Ls, const TL* __restrict__ Dinv, TV* __restrict__ xp,
               TV* __restrict__ fv, int n, int nrhs) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    constexpr int T = kTile;
    TV* Dk = reinterpret_cast<TV*>(smem_raw);  // T x T
    TV* fk = Dk + T * T;                       // nk x nrhs
    TV* y = fk + T * nrhs;                     // nk x nrhs
    const int it = find_item(before, nitems, blockIdx.x);
    const int s = items[it];
    const FrontDesc F = fronts[s];
    const int i = kb + (blockIdx.x - before[it]);
    const TileRange tk = tile_range(kb, F.m, F.c, T);
    const int nk = tk.size;
    const int tid = threadIdx.x, nt = blockDim.x;
    const TL* L = Ls + F.loff;
    TV* f = front_vec(fv, fv_off, s, nrhs);
    const TL* dk = Dinv + dinv_off[s] + (int64_t)kb * T * T;
    for (int idx = tid; idx < T * T; idx += nt) Dk[idx] = (TV)dk[idx];
    for (int idx = tid; idx < nk * nrhs; idx += nt) {
        int q = idx / nk, r = idx - q * nk;
        fk[idx] = f[tk.start + r + (int64_t)q * F.m];
    }
    __syncthreads();
    apply_tile_inverse(Dk, fk, y, nk, nrhs, false);
    if (i == kb) {
        for (int idx = tid; idx < nk * nrhs; idx += nt) {
            int q = idx / nk, r = idx - q * nk;
            xp[F.first_col + tk.start + r + (int64_t)q * n] = y[idx];
        }
        return;
    }
    // f[tile i] -= L(tile i, tile kb) y: warp w takes columns w, w+8, ...; lanes
    // take rows lane, lane+32 (coalesced, 16 independent loads per thread);
    // the eight partial sums per row meet in shared memory
    const TileRange ti = tile_range(i, F.m, F.c, T);
    TV* part = y + T * nrhs;  // 8 x T, one right-hand side at a time
    const int lane = tid & 31, warp = tid >> 5;
    const TL* blk = L + ti.start + (int64_t)tk.start * F.ldl;
    for (int q = 0; q < nrhs; ++q) {
        TV a0 = TV(0), a1 = TV(0);
        for (int j = warp; j < nk; j += 8) {
            const TV yj = y[j + q * nk];
            const TL* col = blk + (int64_t)j * F.ldl;
            if (lane < ti.size) a0 += (TV)col[lane] * yj;
            if (lane + 32 < ti.size) a1 += (TV)col[lane + 32] * yj;
        }
        part[warp * T + lane] = a0;
        part[warp * T + lane + 32] = a1;
        __syncthreads();
        for (int r = tid; r < ti.size; r += nt) {
            TV acc = TV(0);
#pragma unroll
            for (int w = 0; w < 8; ++w) acc += part[w * T + r];
            f[ti.start + r + (int64_t)q * F.m] -= acc;
        }
        __syncthreads();
    }
}

template <typename TL, typename TV>
__global__ void __launch_bounds__(256)
    k_bwd_gather(const FrontDesc* __restrict__ fronts, const int* __restrict__ items,
                 const int* __restrict__ before, int nitems, const int* __restrict__ rows,
                 const int64_t* __restrict__ fv_off, const TL* __restrict__ Ls,
                 const TV* __restrict__ xp, TV* __restrict__ fv, int n, int nrhs) {
    // t[cols of tile jb] = y - L21' x_below, written into the front vector.
    // x_below (the already final solution at the front's update rows) is
    // gathered into shared memory a chunk of rows at a time, so the L21
    // column reads stream without waiting on the row-index indirection.
    constexpr int T = kTile, CH = 2048;
    __shared__ TV xs[CH];
    const int it = find_item(before, nitems, blockIdx.x);
    const int s = items[it];
    const FrontDesc F = fronts[s];
    const int jb = blockIdx.x - before[it];
    const TileRange tj = tile_range(jb, F.m, F.c, T);
    const int c = F.c, u = F.m - c;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const TL* L = Ls + F.loff;
    const int* rw = rows + F.rows_off + c;
    TV* f = front_vec(fv, fv_off, s, nrhs);
    for (int q = 0; q < nrhs; ++q) {
        TV acc[T / 8];  // this warp's columns: warp, warp + 8, ...
#pragma unroll
        for (int a = 0; a < T / 8; ++a) acc[a] = TV(0);
        for (int r0 = 0; r0 < u; r0 += CH) {
            const int nr = min(CH, u - r0);
            for (int r = tid; r < nr; r += blockDim.x) xs[r] = xp[rw[r0 + r] + (int64_t)q * n];
            __syncthreads();
#pragma unroll
            for (int a = 0; a < T / 8; ++a) {
                const int l = warp + 8 * a;
                if (l >= tj.size) break;
                const TL* col = L + c + r0 + (int64_t)(tj.start + l) * F.ldl;
                TV sum = TV(0);
                for (int r = lane; r < nr; r += 32) sum += (TV)col[r] * xs[r];
                acc[a] += sum;
            }
            __syncthreads();
        }
#pragma unroll
        for (int a = 0; a < T / 8; ++a) {
            const int l = warp + 8 * a;
            if (l >= tj.size) break;
            TV v = acc[a];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
            const int j = tj.start + l;
            if (lane == 0) f[j + (int64_t)q * F.m] = xp[F.first_col + j + (int64_t)q * n] - v;
        }
    }
}

template <typename TL, typename TV>
__global__ void __launch_bounds__(256)
    k_bwd_step(const FrontDesc* __restrict__ fronts, const int* __restrict__ items,
               const int* __restrict__ before, int nitems, int kb,
               const int64_t* __restrict__ fv_off, const int64_t* __restrict__ dinv_off,
               const TL* __restrict__ Ls, const TL* __restrict__ Dinv, TV* __restrict__ xp,
               TV* __restrict__ fv, int n, int nrhs) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    constexpr int T = kTile;
    TV* Dk = reinterpret_cast<TV*>(smem_raw);  // T x T
    TV* tk_ = Dk + T * T;                      // nk x nrhs
    TV* x = tk_ + T * nrhs;                    // nk x nrhs
    const int it = find_item(before, nitems, blockIdx.x);
    const int s = items[it];
    const FrontDesc F = fronts[s];
    const int jb = blockIdx.x - before[it];
    const TileRange tk = tile_range(kb, F.m, F.c, T);
    const int nk = tk.size;
    const int tid = threadIdx.x, nt = blockDim.x;
    const int lane = tid & 31, warp = tid >> 5, nw = nt >> 5;
    const TL* L = Ls + F.loff;
    TV* f = front_vec(fv, fv_off, s, nrhs);
    const TL* dk = Dinv + dinv_off[s] + (int64_t)kb * T * T;
    for (int idx = tid; idx < T * T; idx += nt) Dk[idx] = (TV)dk[idx];
    for (int idx = tid; idx < nk * nrhs; idx += nt) {
        int q = idx / nk, r = idx - q * nk;
        tk_[idx] = f[tk.start + r + (int64_t)q * F.m];
    }
    __syncthreads();
    apply_tile_inverse(Dk, tk_, x, nk, nrhs, true);
    if (jb == kb) {
        for (int idx = tid; idx < nk * nrhs; idx += nt) {
            int q = idx / nk, r = idx - q * nk;
            xp[F.first_col + tk.start + r + (int64_t)q * n] = x[idx];
        }
        return;
    }
    const TileRange tj = tile_range(jb, F.m, F.c, T);
    for (int l = warp; l < tj.size; l += nw) {
        const TL* col = L + tk.start + (int64_t)(tj.start + l) * F.ldl;  // L[kb rows, col]
        for (int q = 0; q < nrhs; ++q) {
            TV acc = TV(0);
            for (int r = lane; r < nk; r += 32) acc += (TV)col[r] * x[r + q * nk];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
            if (lane == 0) f[tj.start + l + (int64_t)q * F.m] -= acc;
        }
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

template <typename TL, typename TV>
static void set_solve_attributes() {
    cudaFuncSetAttribute(k_fwd_small<TL, TV>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         200 * 1024);
    cudaFuncSetAttribute(k_bwd_small<TL, TV>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         200 * 1024);
    cudaFuncSetAttribute(k_fwd_step<TL, TV>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         200 * 1024);
    cudaFuncSetAttribute(k_bwd_step<TL, TV>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         200 * 1024);
}

void init_solve_kernels() {
    set_solve_attributes<double, double>();
    set_solve_attributes<float, double>();
}

template <typename TL, typename TV>
void solve_levels(const DevPlan& D, const TL* Ls, const TL* Dinv, TV* xp, TV* fv, int nrhs,
                  cudaStream_t st) {
    const int n = D.n;
    const int msmall = Plan::small_limit[kSmallBuckets - 1];
    const size_t step_smem = (size_t)(kTile * kTile + 2 * kTile * nrhs + 8 * kTile) * sizeof(TV);
    const SolveSchedule& S = D.solve;
    for (int l = 0; l < D.nlevels; ++l) {
        int beg = D.h_small_ptr[l * kSmallBuckets], end = D.h_small_ptr[(l + 1) * kSmallBuckets];
        if (end > beg) {
            ProfScope ps(D.prof, KC_SOLVE_SMALL, st);
            k_fwd_small<TL, TV><<<end - beg, 128, (size_t)msmall * nrhs * sizeof(TV), st>>>(
                D.fronts, D.small_list + beg, D.child, D.relmap, D.fv_off, Ls, xp, fv, n, nrhs);
        }
        int lb = D.h_large_ptr[l], le = D.h_large_ptr[l + 1];
        if (le > lb) {
            ProfScope ps(D.prof, KC_SOLVE_LARGE, st);
            k_fwd_assemble<TV><<<le - lb, 256, 0, st>>>(D.fronts, D.large_list + lb, D.child,
                                                        D.relmap, D.fv_off, xp, fv, n, nrhs);
            for (int q = S.fwd_beg[l]; q < S.fwd_beg[l + 1]; ++q) {
                const WorkList& w = S.fwd[q];
                if (w.nctas == 0) continue;
                k_fwd_step<TL, TV><<<w.nctas, 256, step_smem, st>>>(
                    D.fronts, S.items + w.off, S.before + w.off, w.nitems, w.step, D.fv_off,
                    D.dinv_off, Ls, Dinv, xp, fv, n, nrhs);
            }
        }
    }
    for (int l = D.nlevels - 1; l >= 0; --l) {
        int lb = D.h_large_ptr[l], le = D.h_large_ptr[l + 1];
        if (le > lb) {
            ProfScope ps(D.prof, KC_SOLVE_LARGE, st);
            const WorkList& g = S.gather[l];
            if (g.nctas > 0)
                k_bwd_gather<TL, TV><<<g.nctas, 256, 0, st>>>(D.fronts, S.items + g.off,
                                                              S.before + g.off, g.nitems, D.rows,
                                                              D.fv_off, Ls, xp, fv, n, nrhs);
            for (int q = S.bwd_beg[l]; q < S.bwd_beg[l + 1]; ++q) {
                const WorkList& w = S.bwd[q];
                if (w.nctas == 0) continue;
                k_bwd_step<TL, TV><<<w.nctas, 256, step_smem, st>>>(
                    D.fronts, S.items + w.off, S.before + w.off, w.nitems, w.step, D.fv_off,
                    D.dinv_off, Ls, Dinv, xp, fv, n, nrhs);
            }
        }
        int beg = D.h_small_ptr[l * kSmallBuckets], end = D.h_small_ptr[(l + 1) * kSmallBuckets];
        if (end > beg) {
            int umax = msmall;
            size_t smem = (size_t)(umax + msmall) * nrhs * sizeof(TV);
            ProfScope ps(D.prof, KC_SOLVE_SMALL, st);
            k_bwd_small<TL, TV><<<end - beg, 128, smem, st>>>(D.fronts, D.small_list + beg,
                                                              D.rows, Ls, xp, n, nrhs, umax);
        }
    }
}

template void solve_levels<double, double>(const DevPlan&, const double*, const double*, double*,
                                           double*, int, cudaStream_t);
template void solve_levels<float, double>(const DevPlan&, const float*, const float*, double*,
                                          double*, int, cudaStream_t);

}  // namespace mdgpu
