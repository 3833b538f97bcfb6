// Host-side view of the device-resident plan and the kernel launchers.
#pragma once

#include <cuda_runtime.h>

#include <vector>

#include "plan.hpp"

namespace mdgpu {

constexpr int kAssembleCols = 32;  // columns per CTA in the large-front assembly
constexpr int kTile = 64;          // tile of the large-front factor and solve kernels

// A work-list schedule resident on the device (items/before arrays) with the
// host copy of the per-launch descriptors.
struct DevSchedule {
    int* items = nullptr;
    int* before = nullptr;
    std::vector<int> h_level_beg;
    std::vector<WorkList> h_trsm, h_update;
};

struct SolveSchedule {
    int* items = nullptr;
    int* before = nullptr;
    // per level: large-front forward steps, backward steps and the L21'x
    // gather; each WorkList names its step
    std::vector<int> fwd_beg, bwd_beg;
    std::vector<WorkList> fwd, bwd;
    std::vector<WorkList> gather;  // per level
};

struct DevPlan {
    int n = 0, nsuper = 0, nlevels = 0;
    FrontDesc* fronts = nullptr;
    int* child = nullptr;
    int* rows = nullptr;
    int* relmap = nullptr;
    int* a_src = nullptr;
    int* a_pos = nullptr;
    int* a_colptr = nullptr;
    int* a_colptr_off = nullptr;
    int* small_list = nullptr;
    int* large_list = nullptr;
    int64_t* fv_off = nullptr;  // per supernode: offset of its front vector (m entries)
    std::vector<int> h_small_ptr, h_large_ptr;
    std::vector<WorkList> h_assemble;  // per level, offsets into sched64 arrays
    DevSchedule sched64;
    SolveSchedule solve;
    int64_t fv_total = 0;  // sum of m over supernodes
};

template <typename T>
void factor_levels(const DevPlan& D, T* Ls, T* Us, const double* Ax, int* status,
                   cudaStream_t st);

// Solves with the factor L (scalar TL) on vectors of type TV.  xp holds the
// permuted right-hand sides on entry (n x nrhs, ld n) and the permuted
// solution on exit; fv is scratch of fv_total * nrhs entries.
template <typename TL, typename TV>
void solve_levels(const DevPlan& D, const TL* Ls, TV* xp, TV* fv, int nrhs, cudaStream_t st);

// gather / scatter with the fill-reducing permutation (perm: new -> old)
void permute_gather(const int* perm, const double* b, double* xp, int n, int nrhs, int ldb,
                    cudaStream_t st);
void permute_scatter(const int* perm, const double* xp, double* x, int n, int nrhs, int ldx,
                     cudaStream_t st);

}  // namespace mdgpu
