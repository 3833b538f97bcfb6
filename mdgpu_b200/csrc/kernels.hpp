// Host-side view of the device-resident plan and the kernel launchers.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "plan.hpp"

namespace mdgpu {

constexpr int kAssembleCols = 16;  // columns per CTA in the large-front assembly

// Kernel classes timed by the profiler.
enum KernelClass {
    KC_SMALL_FRONT = 0,  // fused small-front factor
    KC_ASSEMBLE,         // large-front assembly
    KC_POTRF,            // first diagonal tile of large fronts
    KC_TRSM,             // panel factorization (diagonal tiles, triangular solves, in-panel updates)
    KC_SCHUR,            // Schur-complement tile updates (dominant flops)
    KC_SOLVE_SMALL,      // small-front forward/backward sweeps
    KC_SOLVE_LARGE,      // large-front forward/backward steps
    KC_OTHER,            // permutations, residual, norms
    KC_COUNT
};

// Optional per-launch CUDA-event timing, grouped by kernel class; off by
// default (no events recorded).  Algorithmic flops / bytes per launch are
// accumulated alongside for roofline figures.
struct Profiler {
    bool on = false;
    struct Rec {
        int cls;
        cudaEvent_t a, b;
        double flops, bytes;
    };
    std::vector<Rec> recs;
    std::vector<cudaEvent_t> pool;
    size_t used = 0;
    cudaEvent_t take() {
        if (used == pool.size()) {
            cudaEvent_t e;
            cudaEventCreate(&e);
            pool.push_back(e);
        }
        return pool[used++];
    }
    ~Profiler() {
        for (auto e : pool) cudaEventDestroy(e);
    }
};

// RAII helper: records a begin/end event pair around the launches in scope.
struct ProfScope {
    Profiler* p;
    int cls;
    double flops, bytes;
    cudaStream_t st;
    cudaEvent_t a = nullptr;
    ProfScope(Profiler* p_, int cls_, cudaStream_t st_, double fl = 0, double by = 0)
        : p(p_), cls(cls_), flops(fl), bytes(by), st(st_) {
        if (p && p->on) {
            a = p->take();
            cudaEventRecord(a, st);
        }
    }
    ~ProfScope() {
        if (a) {
            cudaEvent_t b = p->take();
            cudaEventRecord(b, st);
            p->recs.push_back({cls, a, b, flops, bytes});
        }
    }
};
constexpr int kTile = 64;          // tile of the large-front factor and solve kernels
constexpr int kPanel = 256;        // pivot columns per panel of the large fronts
constexpr int kScrCols = 2 * kPanel;  // panel scratch row: panels of even and odd index

// A work-list schedule resident on the device (items/before arrays) with the
// host copy of the per-launch descriptors.
struct DevSchedule {
    int* items = nullptr;
    int* before = nullptr;
    int2* tasks = nullptr;  // OP_PANEL tasks (front, row tile)
    std::vector<int> h_level_beg;
    std::vector<WorkList> h_trsm, h_update;
    // panel schedule (FP32): per level a run of operations
    std::vector<int> h_op_beg;
    std::vector<PanelOp> h_ops;
};

// Solve: one launch per direction over every level's work items (see
// SolveScheduleHost).  sync holds the two ticket counters, one count per
// pivot tile (backward gathers counted in), the abort word, then per front
// the forward count of finished children, the forward count of finished
// update tiles and the backward count of finished completions; it is
// cleared at the start of every solve.  err (not cleared by the solve) gets
// bit 0 when a dependency wait ran out.
struct SolveSchedule {
    int2* tasks = nullptr;
    int4* fwd_items = nullptr;
    int4* bwd_items = nullptr;
    int nfwd_items = 0, nbwd_items = 0;
    int* fwd_wlist = nullptr;    // the warp items' fronts, per direction
    int* bwd_wlist = nullptr;
    int* bwd_target = nullptr;   // per front
    int nfronts = 0;
    std::vector<int> fwd_task_beg, bwd_task_beg;  // nlevels + 1
    std::vector<double> fwd_elems, bwd_elems;     // per level: L + Dinv elements
    std::vector<double> small_elems;              // per level: L elements of small fronts
    int* sync = nullptr;
    int nsync = 0, nflags = 0;
    int* err = nullptr;
    // backward update-row partial sums (see SolveScheduleHost)
    std::vector<int> gather_task_beg;
    int* gather_nch = nullptr;
    int* gather_off = nullptr;
    // forward assembly of the large fronts as a gather (see SolveScheduleHost)
    int* amap_off = nullptr;
    int* amap_row = nullptr;
    int* amap_ent = nullptr;
    // small fronts per level by rows descending, and per level the counts
    // taking one, two and four fronts per warp (see SolveScheduleHost)
    int* warp_list = nullptr;
    std::vector<int> warp_cnt;
};

// Selected inverse of the large fronts: per level a gather list (front, CTAs
// = 16-column blocks of its update part) and per (level, block step) a list
// (front, CTAs = 64-row tiles below the step's pivot block); WorkList.step
// is the block step (0 = the front's last pivot block).
struct SelSchedule {
    int* items = nullptr;
    int* before = nullptr;
    std::vector<WorkList> h_gather;  // per level
    std::vector<int> h_step_beg;     // nlevels + 1
    std::vector<WorkList> h_steps;
};

// General reverse mode (adjoint.cu): per level the fronts with an update
// part and a parent, for the gather of their Ubar (CTA per 16 columns); L's
// column pointers; per front the offset of its c x c scratch (a level's
// fronts side by side, levels reuse it).
struct AdjSchedule {
    int* items = nullptr;
    int* before = nullptr;
    std::vector<WorkList> h_gather;  // per level
    int64_t* Lp = nullptr;
    int64_t* woff = nullptr;
    int64_t wtotal = 0;
};

struct DevPlan {
    int n = 0, nsuper = 0, nlevels = 0;
    int num_sms = 0;  // of the handle's device (persistent grids)
    // launch shapes of the small-front factor kernels, chosen by
    // mdgpu_autotune (these defaults otherwise): the tiny-front kernel's grid
    // cap (blocks of four warps) and the threads of k_small_front per size
    // bucket
    int tiny_blocks_cap = 148 * 8;
    int small_threads[kSmallBuckets] = {64, 128, 256, 256, 256, 256};
    // the factor runs a level's small fronts beside its large fronts (both
    // depend only on lower levels), and the small fronts' pieces (the tiny
    // fronts, then each k_small_front size bucket) beside one another: a
    // fork event, and a stream and a join event per piece
    cudaEvent_t fork_ev = nullptr;
    static constexpr int kSmallPieces = 1 + kSmallBuckets - Plan::kTinyBuckets;
    cudaStream_t piece_st[kSmallPieces] = {};
    cudaEvent_t piece_join[kSmallPieces] = {};
    int max_u = 0;  // largest update-matrix order (child relative maps in shared memory)
    int max_m_large = 0, max_nch_large = 0;  // largest large front, most children of one
    std::vector<int> h_level_max_m;          // per level: largest large front
    FrontDesc* fronts = nullptr;
    int* child = nullptr;
    int* rows = nullptr;
    int* relmap = nullptr;
    int* a_src = nullptr;
    int* a_pos = nullptr;
    // selected inverse: every supernode by level (root level last), the
    // Y scratch offset per supernode, and per lower-triangle entry its front
    int* level_list = nullptr;
    std::vector<int> h_level_ptr;  // nlevels + 1
    int64_t* yoff = nullptr;
    SelSchedule sel;
    AdjSchedule adj;
    int64_t* zuoff = nullptr;  // per supernode: Z's update part in the selinv Zu store
    int64_t yscr_total = 0;
    int* a_front = nullptr;
    int* a_colptr = nullptr;
    int* a_colptr_off = nullptr;
    int* small_list = nullptr;
    int* large_list = nullptr;
    int64_t* fv_off = nullptr;  // per supernode: offset of its front vector (m entries)
    int64_t* dinv_off = nullptr;  // per supernode: inverted diagonal tiles (large fronts)
    int* asm_off = nullptr;       // per supernode: child column ranges (large fronts)
    int* asm_range = nullptr;
    int64_t dinv_total = 0;
    // FP32 path: per large front a TMA descriptor of its L panel (the
    // operands of the tensor-core Schur updates)
    CUtensorMap* tmaps = nullptr;
    CUtensorMap* tmaps_bf16 = nullptr;  // over the same scratch as BF16, for the BF16 Schur update
    // FP32 tensor-core path: the last two panels of every large front of a
    // level (panel q at columns (q mod 2) kPanel of a kScrCols-wide row),
    // row-major, split: per front 2 mpad rows of kScrCols floats (rows [0,
    // mpad) the TF32 parts hi, rows [mpad, 2 mpad) lo = x - hi; or mpad rows
    // of BF16 values), mpad = m rounded up to 128; written by the panel
    // kernel, read by the tensor-core Schur update through tmaps (fronts of
    // a level side by side, levels reuse it)
    float* pscr = nullptr;
    int64_t* pscr_off = nullptr;  // per supernode (-1 if small)
    int64_t pscr_total = 0;
    int* tmap_idx = nullptr;
    DevSchedule psched;
    // sync words of the panel launches, cleared at the start of every
    // factor: one ticket counter per OP_PANEL launch, then one flag per pivot
    // tile of the large fronts (flag of tile k of front s at fsync_flags +
    // dinv_off[s] / kTile^2 + k), then the abort word, then one step count
    // per pivot tile (the blocks X(k, .) its diagonal task has written)
    int* fsync = nullptr;
    int nfsync = 0;
    int fsync_flags = 0;
    int nflags_factor = 0;
    std::vector<int> h_small_ptr, h_large_ptr;
    std::vector<WorkList> h_assemble;  // per level, offsets into sched64 arrays
    DevSchedule sched64;
    SolveSchedule solve;
    // work vectors per right-hand side: the front vectors (sum of m over
    // supernodes), the backward gather partials (T rows each), then the
    // publication slots of the pivot tiles (T rows each, forward then backward)
    int64_t fv_fronts = 0;
    int64_t fv_pub_off = 0;
    int64_t fv_total = 0;
    std::vector<double> h_update_flops;  // per update work list (algorithmic)
    std::vector<double> h_small_bytes;   // per (level, bucket) small-front launch
    Profiler* prof = nullptr;
};

// one-time kernel attribute setup (dynamic shared memory limits); must run
// before any launch sequence is captured into a CUDA graph
void init_factor_kernels();
void init_solve_kernels();
void init_schur_tc();
void init_schur_f64();
void init_panel_kernels();
void init_selinv();

// panel scratch rows of a large front (m rounded up to the 128-row tile)
__host__ __device__ inline int panel_mpad(int m) { return (m + 127) & ~127; }

// Schur-update modes of an FP32 factor's large fronts on the tensor cores:
// 3xTF32 (close to FP32 accuracy, MDGPU_FP32), BF16 operands (MDGPU_BF16),
// one TF32 product (MDGPU_TF32)
enum SchurMode { kSchur3xTF32 = 0, kSchurBF16 = 1, kSchur1xTF32 = 2 };

// smode (T = float only): the SchurMode of the large fronts' updates (FP64
// for T = double).  status: [0] smallest failing pivot column, [1] device
// wait error code, [3] count of diagonal tiles refactored in FP64 (weak FP32
// pivots)
template <typename T>
void factor_levels(const DevPlan& D, T* Ls, T* Us, T* Dinv, const double* Ax, int* status,
                   cudaStream_t st, int smode = kSchur3xTF32);

// Solves with the factor L (scalar TL) on vectors of type TV.  xp holds the
// permuted right-hand sides on entry (n x nrhs, ld n) and the permuted
// solution on exit; fv is scratch of fv_total * nrhs entries.
template <typename TL, typename TV>
void solve_levels(const DevPlan& D, const TL* Ls, const TL* Dinv, TV* xp, TV* fv, int nrhs,
                  cudaStream_t st);

// Per large front a map over its panel scratch (base scr + scr_off[s],
// row-major, kPanel columns): bf16, the BF16 copy (mpad rows); else the
// TF32 hi/lo split (2 mpad rows); boxes of 128 bytes x 128 rows, 128-byte
// swizzle
int build_panel_maps(const Plan& P, const float* base, const std::vector<int64_t>& scr_off,
                     std::vector<CUtensorMap>& maps, std::vector<int>& idx, bool bf16);
// one panel launch (OP_PANEL): every row-tile task of the panel's fronts
// split: also write the panel split for 3xTF32 into the panel scratch
template <typename T>
void launch_panel(const DevPlan& D, const PanelOp& op, T* Ls, T* Dinv, int* status, int split_mode,
                  cudaStream_t st);
// the update after panel `panel` with the npan panels ending there; strip:
// only the next panel's two tile columns (see PanelOpKind)
void launch_schur_tc(const DevPlan& D, const WorkList& w, int panel, int PW, int npan,
                     bool strip, float* Ls, float* Us, int* err, int mode, cudaStream_t st);
void launch_schur_f64(const DevPlan& D, const WorkList& w, int panel, int PW, double* Ls,
                      double* Us, cudaStream_t st);

// fixed device scratch of the no-allocation solve (noalloc.cu)
long long noalloc_scratch_capacity();
double* noalloc_scratch(std::string& msg);

// gather / scatter with the fill-reducing permutation (perm: new -> old)
void permute_gather(const int* perm, const double* b, double* xp, int n, int nrhs, int ldb,
                    cudaStream_t st);
void permute_scatter(const int* perm, const double* xp, double* x, int n, int nrhs, int ldx,
                     cudaStream_t st);

// selected inverse and adjoint (selinv.cu)
void launch_selinv(const DevPlan& D, const double* Ls, const double* Dinv, double* Zs,
                   double* Zu, double* Yscr, cudaStream_t st);
void launch_grad_lower(const DevPlan& D, int nnz, const int* perm, const double* Zs,
                       const double* x, double* G, cudaStream_t st);
template <typename T>
void launch_logdet(const DevPlan& D, const T* Ls, double* partial, double* out, cudaStream_t st);
int logdet_partials();
// Abar (nnz entries, caller order) from Lbar (L's CSC values) with the FP64
// factor Ls: Fb, Fu, Wscr stores of plan lstore, zustore, adj.wtotal doubles
void launch_adjoint(const DevPlan& D, int nnz, const double* Ls, const double* Lbar, double* Fb,
                    double* Fu, double* Wscr, double* Abar, cudaStream_t st);
int selinv_block();  // pivot columns per block of the one-CTA (small-front) kernel
int selinv_tile();   // pivot columns per block step of the large fronts

}  // namespace mdgpu
