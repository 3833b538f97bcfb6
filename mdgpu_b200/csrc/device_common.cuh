// Device-side helpers shared by the factor and solve kernels.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "plan.hpp"

namespace mdgpu {

// Rows/columns [start, start + size) of tile t of a front with m rows and c
// pivot columns: tiles 0..nt1-1 cover [0, c), the rest cover [c, m).
struct TileRange {
    int start, size;
    bool in_u;
};

__host__ __device__ inline int tiles_l(int c, int T) { return (c + T - 1) / T; }

__host__ __device__ inline TileRange tile_range(int t, int m, int c, int T) {
    int nt1 = tiles_l(c, T);
    TileRange r;
    if (t < nt1) {
        r.start = t * T;
        r.size = min(T, c - r.start);
        r.in_u = false;
    } else {
        r.start = c + (t - nt1) * T;
        r.size = min(T, m - r.start);
        r.in_u = true;
    }
    return r;
}

// Address of front element (row r, column col), r >= col, for the split
// [L panel | U] storage of front f.
template <typename T>
__device__ inline T* front_elem(T* Ls, T* Us, const FrontDesc& f, int r, int col) {
    if (col < f.c) return Ls + f.loff + r + (int64_t)col * f.ldl;
    return Us + f.uoff + (r - f.c) + (int64_t)(col - f.c) * f.ldu;
}

// Which item of a work list does CTA `b` belong to (binary search over the
// list's prefix counts, nitems + 1 entries).
__device__ inline int find_item(const int* before, int nitems, int b) {
    int lo = 0, hi = nitems - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (before[mid] <= b)
            lo = mid;
        else
            hi = mid - 1;
    }
    return lo;
}

// (i, j), i >= j, of entry l of the row-major enumeration of a lower triangle.
__device__ inline void lower_index(int l, int& i, int& j) {
    int r = (int)((sqrt(8.0 * (double)l + 1.0) - 1.0) * 0.5);
    while ((r + 1) * (r + 2) / 2 <= l) ++r;
    while (r * (r + 1) / 2 > l) --r;
    i = r;
    j = l - r * (r + 1) / 2;
}

// Record a non-positive (or NaN) pivot at global column col: the smallest
// such column wins.
__device__ inline void flag_pivot(int* status, int col) { atomicMin(status, col); }

}  // namespace mdgpu
