// Numeric plan: everything the GPU factor and solve need, computed once per
// sparsity pattern on the host and uploaded once.
//
// Layout in HBM (element offsets, all 256-byte aligned):
//   L store   one column-major m_s x c_s panel per supernode s, leading
//             dimension ldl_s = m_s rounded up to 8.  The panel holds the
//             supernode's columns of L (rows = the front's row set); it is the
//             factor's final storage and the input of the solves.
//   U store   one column-major u_s x u_s update matrix per non-root supernode
//             (u_s = m_s - c_s, leading dimension ldu_s = u_s rounded up to 8),
//             lower triangle only; written when s is factored (tree level
//             lev(s)), read when its parent is assembled (level lev(parent)).
//             Storage is reused over the matrices' lifetimes: two update
//             matrices whose level intervals [lev(s), lev(parent)] overlap
//             share no element, others may, so the store is about the
//             largest sum of update matrices live at one level, not their
//             total (the role of a postorder stack in a sequential code).
// Front s is the m_s x m_s matrix [L panel | U]; its rows are the sorted
// global (permuted) column indices rows_s, the first c_s of which are
// first_col_s .. first_col_s + c_s - 1.
#pragma once

#include <cstdint>
#include <memory>
#include <new>
#include <type_traits>
#include <utility>
#include <vector>

#include "symbolic.hpp"

namespace mdgpu {

// std::allocator whose resize() leaves new elements default-initialised
// (for int and plain structs: untouched), so a plan's large arrays are first
// written -- and their pages first touched -- by the threads that fill them.
template <typename T>
struct UninitAlloc : std::allocator<T> {
    template <typename U>
    struct rebind {
        using other = UninitAlloc<U>;
    };
    UninitAlloc() = default;
    template <typename U>
    UninitAlloc(const UninitAlloc<U>&) noexcept {}
    template <typename U>
    void construct(U* p) noexcept(std::is_nothrow_default_constructible<U>::value) {
        ::new (static_cast<void*>(p)) U;
    }
    template <typename U, typename... A>
    void construct(U* p, A&&... a) {
        ::new (static_cast<void*>(p)) U(std::forward<A>(a)...);
    }
};
template <typename T>
using HostArray = std::vector<T, UninitAlloc<T>>;

// Per-supernode record mirrored on the device.
struct FrontDesc {
    int64_t loff;    // L store offset of the panel
    int64_t uoff;    // U store offset of the update matrix (-1 for the root)
    int m, c;        // front rows, pivot columns
    int ldl, ldu;    // leading dimensions
    int rows_off;    // offset of rows_s / relmap_s in the row arrays
    int first_col;   // global (permuted) index of the first pivot column
    int child_beg, child_end;  // range in the child list
    int a_beg, a_end;          // range in the A-entry lists
    int parent;                // parent supernode (-1 for the root)
    int pad_;
};

// A tiled work list for one (level, step) launch of a multi-CTA kernel over
// the large fronts: CTA b belongs to item[k] where ctas_before[k] <= b <
// ctas_before[k+1].
struct WorkList {
    int64_t off;   // offset into the shared work-list arrays
    int nitems;
    int nctas;
    int step;
};

constexpr int kSmallBuckets = 6;

struct Plan {
    int n = 0;
    int nsuper = 0;
    int64_t nnz_user = 0;       // entries of the caller's lower triangle
    std::vector<int> perm;      // new -> old (empty: natural)
    std::vector<int> iperm;     // old -> new
    HostArray<FrontDesc> fronts;
    std::vector<int> child;     // children lists
    HostArray<int> rows;        // front row sets, concatenated
    HostArray<int> relmap;      // per row r >= c_s of front s: position in the parent's front
    HostArray<int> a_src;       // per A entry: index in the caller's value array
    HostArray<int> a_pos;       // per A entry: local (row | col << 16) inside the front
    std::vector<int> a_colptr;  // per large front: c+1 offsets into its A entries
    std::vector<int> a_colptr_off;  // per supernode: offset into a_colptr (-1 if small)
    // large fronts: inverted diagonal tiles (T x T each, one per pivot tile)
    std::vector<int64_t> dinv_off;  // per supernode (-1 if small)
    int64_t dinv_total = 0;         // elements
    // large fronts: per 32-column block of the front and per child, the
    // child's update columns [lo, hi) that land in the block
    std::vector<int> asm_off;       // per supernode (-1 if small)
    std::vector<int> asm_range;
    std::vector<int64_t> Lp;    // CSC column pointers of L (reference spL->p)
    int64_t lstore = 0, ustore = 0;  // element counts
    // selected inverse: the update part Z_UU of every front with an update
    // matrix, at zuoff[s] of a store of zustore elements (see build_plan)
    std::vector<int64_t> zuoff;
    int64_t zustore = 0;
    int64_t lnz = 0;
    double flops = 0;           // sum over columns of count^2 (the reference's count)
    int max_m = 0, max_u = 0;

    // level schedule: supernodes grouped by tree height (leaves = level 0)
    int nlevels = 0;
    // small fronts of each level, bucketed by m (bucket limits small_limit[])
    std::vector<int> small_ptr;     // nlevels * kSmallBuckets + 1
    std::vector<int> small_list;
    // large fronts of each level
    std::vector<int> large_ptr;     // nlevels + 1
    std::vector<int> large_list;

    static const int small_limit[kSmallBuckets];
    static constexpr int kTinyBuckets = 2;  // buckets of fronts with m <= 32
    static constexpr int kSmallMaxRows = 160;  // small_limit[kSmallBuckets - 1]
};

// Offsets for blocks with inclusive lifetimes [beg_i, end_i] (levels 0 ..
// nlev - 1): blocks whose lifetimes overlap get disjoint ranges.  Sweep over
// the levels: the blocks whose lifetime ended at l - 1 are freed (coalesced),
// then the blocks starting at l are placed, largest first, in the smallest
// free range that holds them, else on top.  Blocks of size 0 get -1.
// Returns the store size (the highest end reached).
int64_t lifetime_alloc(const std::vector<int>& beg, const std::vector<int>& end,
                       const std::vector<int64_t>& size, int nlev, std::vector<int64_t>& off);

// Build the plan from a completed symbolic analysis.  `large_threshold` is
// the row count above which a front takes the tiled multi-CTA path.
void build_plan(const Symbolic& S, int64_t nnz_user, int large_threshold, Plan& P);
// Fill dinv_off / asm_off / asm_range for tile size T and assembly width CB.
void build_large_tables(Plan& P, int T, int CB);

// Work-list storage: every list is a run of (front id, CTAs before it)
// pairs closed by a sentinel carrying the list's CTA total.
struct ListStore {
    std::vector<int> items;
    std::vector<int> ctas_before;
    WorkList add(const std::vector<std::pair<int, int>>& fronts_ctas, int step);
};

// Work lists of the tiled factor kernels, for tile size T.
struct TileSchedule {
    int T = 64;
    ListStore store;
    std::vector<int> level_beg;          // per level: range of (trsm, update) pairs
    std::vector<WorkList> trsm, update;  // one pair per (level, step)
    std::vector<WorkList> assemble;      // per level: CTA per (front, column block)
};

// Panel schedule of the large fronts: per level, operations in launch order:
// the assembly, then per 256-column panel one panel factorization (OP_PANEL)
// and the Schur updates after it.  FP64 factors run one update of the whole
// trailing part per panel (OP_SCHUR_TC).  The tensor-core FP32 factors defer
// the bulk of it to every second panel, so the trailing matrix is read and
// written once per two panels: after an even panel p, OP_SCHUR_NEXT updates
// only the next panel's columns (two 128-column tiles) of the fronts that
// have panel p + 1, and OP_SCHUR_REST (arg2 = 1) the whole trailing part of
// the fronts that do not; after an odd panel p, OP_SCHUR_REST (arg2 = 2)
// updates the trailing part after panel p with panels p - 1 and p together
// (K = 512).  OP_POTRF, OP_TRSM and OP_UPDATE_PANEL are the 64-wide steps of
// the tile schedule.
enum PanelOpKind {
    OP_ASSEMBLE = 0,
    OP_POTRF,
    OP_TRSM,
    OP_UPDATE_PANEL,
    OP_SCHUR_TC,
    OP_PANEL,
    OP_SCHUR_NEXT,
    OP_SCHUR_REST
};
struct PanelOp {
    int kind;
    int arg;      // tile step k (POTRF/TRSM/UPDATE_PANEL) or panel index (SCHUR_*, PANEL)
    int arg2;     // UPDATE_PANEL: last tile index of the panel; SCHUR_REST: panels (1, 2)
    WorkList w;
    double flops;  // algorithmic flops of the launch
    double elems;  // algorithmic factor-scalar traffic (elements read + written)
    double xbytes; // other algorithmic traffic in bytes (FP64 values, indices)
    // OP_PANEL: tasks [toff, toff + ntasks) of PanelSchedule::tasks (pairs),
    // taken by ticket from counter number `counter`
    int64_t toff = 0;
    int ntasks = 0;
    int counter = -1;
};
struct PanelSchedule {
    ListStore store;
    std::vector<int> op_beg;  // per level
    std::vector<PanelOp> ops;
    // OP_PANEL tasks (front s, row tile i) as int pairs: per launch every
    // diagonal task first (pivot tile by pivot tile), then the other row
    // tiles front by front, so that a task waits only on lower tickets
    std::vector<int> tasks;
    int ncounters = 0;   // one ticket counter per OP_PANEL launch
    int64_t nflags = 0;  // one flag per pivot tile of a large front (dinv_total / T^2)
};
void build_panel_schedule(const Plan& P, int T, int PW, int CB, PanelSchedule& S);

// Tasks of the large-front solve kernels (one launch per level and direction).
struct SolveScheduleHost {
    int T = 64;
    // one launch per level and direction: tasks (front, tile) as int pairs,
    // ordered so that every task's dependencies come earlier (a task only
    // waits on tasks that took a lower ticket, hence already run)
    // forward task (s, i | cnt << 16): row tiles i .. i + cnt - 1 of front s
    // (a pivot tile alone; update tiles grouped to about kFwdGroupBlocks L
    // blocks per task); backward task (s, j): pivot column tile j
    static constexpr int kFwdGroupBlocks = 8;
    static constexpr int kFwdGroupTiles = 4;  // at most 256 rows: a thread per row
    std::vector<int> tasks;
    std::vector<int> fwd_task_beg, bwd_task_beg;  // nlevels + 1 each, in tasks
    std::vector<double> fwd_elems, bwd_elems;     // per level, L + Dinv elements read
    std::vector<double> small_elems;              // per level: L elements of its small fronts
    int nflags = 0;                               // one per pivot tile of a large front
    // backward, update rows: one task per (front, pivot column tile j,
    // chunk of kGatherTiles update row tiles), packed (s, j | chunk << 16);
    // each writes a T x nrhs partial sum of L(chunk, j)' x; per front the
    // chunk count and the first partial (pivot tile j, chunk h at
    // gather_off + j * gather_nch + h; every level's partials side by side,
    // the levels' launches being one)
    static constexpr int kGatherTiles = 4;
    std::vector<int> gather_task_beg;   // nlevels + 1, in tasks
    std::vector<int> gather_nch, gather_off;  // per supernode
    int64_t gather_vecs = 0;            // partial vectors of all levels
    // The solve runs one launch per direction over all work items in a
    // topological order (every item's dependencies come earlier), fronts by
    // critical-path priority, four ints per item {kind, a, b, c}:
    //   kItemTile    a large-front tile task: front a, task spec b (as in
    //                tasks: the forward row tiles or the backward pivot tile)
    //   kItemGather  a backward update-row gather: front a, spec b
    //   kItemWarps   small fronts on up to kWarpsPerItem warps: entries
    //                a .. of the direction's warp list, b = n1 | n2 << 8 |
    //                n4 << 16: n1 fronts of more than 16 rows (a warp each),
    //                then n2 of 9..16 rows (two per warp), then n4 of at
    //                most 8 rows (four per warp)
    static constexpr int kItemTile = 0, kItemGather = 1, kItemWarps = 2;
    static constexpr int kWarpsPerItem = 8;
    std::vector<int> fwd_items, bwd_items;
    std::vector<int> fwd_wlist, bwd_wlist;  // the warp items' fronts
    // backward: the solution rows of front s are final once bwd_target[s]
    // completions are counted (one per pivot tile of a large front, one for
    // a small front)
    std::vector<int> bwd_target;
    // small fronts of each level for the warp-per-front factor, by rows
    // descending (same level ranges as small_list): warp_cnt[3 l + k] fronts
    // of more than 16 rows (k = 0, a warp each), of 9..16 rows (k = 1, two
    // per warp) and of at most 8 rows (k = 2, four per warp)
    std::vector<int> warp_list;
    std::vector<int> warp_cnt;
    // front vectors: front s holds rows fv_off[s] .. fv_off[s] + m_s - 1 of
    // one array (a row holds the right-hand sides side by side)
    std::vector<int64_t> fv_off;
    int64_t fv_rows = 0;
    // forward assembly of the large fronts as a gather: row r of large front
    // s sums the front-vector rows amap_ent[amap_row[amap_off[s] + r] ..
    // amap_row[amap_off[s] + r + 1] - 1] (children's update rows, in child
    // order, so the sums are those of a child-by-child scatter)
    std::vector<int> amap_off;  // per supernode, -1 for small fronts
    HostArray<int> amap_row;
    HostArray<int> amap_ent;
};

int front_tiles(int m, int c, int T);  // tiles in the [0,c) + [c,m) tiling
void build_factor_schedule(const Plan& P, int T, int assemble_cols, TileSchedule& S);
void build_solve_schedule(const Plan& P, int T, SolveScheduleHost& S);
// per supernode: tree level (leaves 0)
std::vector<int> front_levels(const Plan& P);

}  // namespace mdgpu
