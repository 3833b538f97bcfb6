// C ABI implementation (include/mdgpu_b200.h): symbolic on the host, plan
// resident on the device, numeric factor / solve / refinement on the GPU.
#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

#include <algorithm>
#include <atomic>
#include <climits>
#include <cstdio>
#include <map>
#include <cstdlib>
#include <cstring>
#include <exception>
#include <new>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

#include "gmres_ir.hpp"
#include "ir.hpp"
#include "kernels.hpp"
#include "mdgpu_b200.h"
#include "parallel.hpp"
#include "plan.hpp"
#include "plan_check.hpp"
#include "symbolic.hpp"

using namespace mdgpu;

namespace {

thread_local std::string g_last_error;

// An NVTX range over one API-level phase (factor, solve, refinement, ...),
// so a profiler can select a phase's kernels by name (ncu --nvtx
// --nvtx-include "mdgpu_factor/").  Header-only NVTX: without a tool
// attached each call returns at once.
struct NvtxRange {
    explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
    ~NvtxRange() { nvtxRangePop(); }
    NvtxRange(const NvtxRange&) = delete;
    NvtxRange& operator=(const NvtxRange&) = delete;
};

struct CudaError : std::runtime_error {
    cudaError_t code;
    CudaError(cudaError_t c, const char* what) : std::runtime_error(what), code(c) {}
};

void ck(cudaError_t e, const char* where) {
    if (e != cudaSuccess)
        throw CudaError(e, (std::string(where) + ": " + cudaGetErrorString(e)).c_str());
}

template <typename T>
T* dalloc(size_t count) {
    void* p = nullptr;
    if (count == 0) count = 1;
    cudaError_t e = cudaMalloc(&p, count * sizeof(T));
    if (e != cudaSuccess) {
        cudaGetLastError();
        throw std::bad_alloc();
    }
    return static_cast<T*>(p);
}

template <typename T, typename A>
T* upload(const std::vector<T, A>& v) {
    T* d = dalloc<T>(v.size());
    if (!v.empty()) ck(cudaMemcpy(d, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice), "upload");
    return d;
}

int device_available() {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return n > 0;
}

}  // namespace

struct mdgpu_handle_s {
    Symbolic sym;
    Plan plan;
    TileSchedule fsched;
    SolveScheduleHost ssched;
    // batch of independent systems (mdgpu_analyze_batch): per system its first
    // row and its first entry in the concatenated lower-triangle values
    std::vector<int> sys_row_off, sys_val_off;
    PanelSchedule pschedh;
    std::vector<int64_t> pscr_off;  // panel scratch offset per supernode
    bool use_tensor_cores = true;
    DevPlan D;
    std::vector<int> level;
    SymCsr csr;
    std::vector<int> h_csr_rowptr;
    HostArray<int> h_csr_col, h_csr_src;  // every entry written by the CSR build
    bool on_device = false;
    int device = 0;
    cudaStream_t stream = nullptr;
    std::vector<void*> owned;  // device allocations of the plan
    int* d_perm = nullptr;
    int* d_status = nullptr;
    unsigned long long* d_norms = nullptr;  // [0] = ||A||, then 3 per rhs
    double* d_Ax = nullptr;
    double* dL64 = nullptr;
    double* dU64 = nullptr;
    float* dL32 = nullptr;
    float* dU32 = nullptr;
    double* dD64 = nullptr;  // inverted diagonal tiles of the large fronts
    float* dD32 = nullptr;
    double *d_xp = nullptr, *d_fv = nullptr, *d_B = nullptr, *d_X = nullptr, *d_R = nullptr,
           *d_D = nullptr;
    int nrhs_cap = 0;
    // CUDA graphs of the numeric launch sequences (captured once, replayed)
    bool use_graphs = true;
    cudaGraphExec_t fgraph[4] = {nullptr, nullptr, nullptr, nullptr};  // per precision
    std::map<int, cudaGraphExec_t> sgraph;  // key: precision * 1024 + rhs count
    int factored = -1;  // precision of the current factor, -1 none
    int fp64_diag_tiles = 0;  // of the last factor: diagonal tiles redone in FP64
    int bf16_fallbacks = 0;   // BF16 or 1xTF32 factors redone in FP32 (non-positive pivot)
    bool tuned = false;       // launch shapes chosen by mdgpu_autotune
    bool selinv_done = false;      // Z of the current FP64 factor in dZ64 / dZu64
    double* dZ64 = nullptr;        // selected inverse, laid out as the L panels
    double* dZu64 = nullptr;       // its update parts (plan.zuoff offsets)
    // general reverse mode: Fbar panels, Ubar store, c x c scratch, Lbar / Abar
    double *d_Fb = nullptr, *d_Fu = nullptr, *d_W = nullptr, *d_Lbar = nullptr,
           *d_Abar = nullptr;
    double* d_Y = nullptr;         // its Y scratch
    double* d_logdet = nullptr;    // logdet partial sums, then the result
    double* d_gx = nullptr;        // gradient: x and G on the device (host entry)
    double* d_gG = nullptr;
    double* d_gm = nullptr;  // GMRES-IR basis, scratch vector, slots, partial sums
    int64_t gm_cap = 0;      // its size in doubles
    int status_init[2] = {0, 0};
    int not_spd = -1;
    Profiler prof;
    std::vector<double> prof_ms, prof_flops, prof_bytes;
    std::vector<long long> prof_n;

    template <typename T>
    T* keep(T* p) {
        owned.push_back(p);
        return p;
    }
    void drop_solve_graphs() {
        for (auto& kv : sgraph) cudaGraphExecDestroy(kv.second);
        sgraph.clear();
    }
    ~mdgpu_handle_s() {
        if (!on_device) return;
        cudaSetDevice(device);
        for (auto g : fgraph)
            if (g) cudaGraphExecDestroy(g);
        drop_solve_graphs();
        for (void* p : owned) cudaFree(p);
        for (void* p : {(void*)d_Fb, (void*)d_Fu, (void*)d_W, (void*)d_Lbar, (void*)d_Abar})
            if (p) cudaFree(p);
        for (void* p : {(void*)dZ64, (void*)dZu64, (void*)d_Y, (void*)d_logdet, (void*)d_gx, (void*)d_gG,
                        (void*)d_gm})
            if (p) cudaFree(p);
        for (void* p : {(void*)d_Ax, (void*)dL64, (void*)dU64, (void*)dL32, (void*)dU32,
                        (void*)dD64, (void*)dD32,
                        (void*)d_xp, (void*)d_fv, (void*)d_B, (void*)d_X, (void*)d_R, (void*)d_D})
            if (p) cudaFree(p);
        for (int i = 0; i < DevPlan::kSmallPieces; ++i) {
            if (D.piece_join[i]) cudaEventDestroy(D.piece_join[i]);
            if (D.piece_st[i]) cudaStreamDestroy(D.piece_st[i]);
        }
        if (D.fork_ev) cudaEventDestroy(D.fork_ev);
        if (stream) cudaStreamDestroy(stream);
    }
};

namespace {

constexpr int kLargeThreshold = 160;  // rows above which a front is tiled

void build_csr(mdgpu_handle_s* h, int n, const int* Ap, const int* Ai) {
    // full symmetric CSR of the caller's lower triangle, rows in original order
    std::vector<int> cnt(n, 0);
    for (int j = 0; j < n; ++j)
        for (int p = Ap[j]; p < Ap[j + 1]; ++p) {
            int i = Ai[p];
            cnt[i]++;
            if (i != j) cnt[j]++;
        }
    h->h_csr_rowptr.assign(n + 1, 0);
    for (int i = 0; i < n; ++i) h->h_csr_rowptr[i + 1] = h->h_csr_rowptr[i] + cnt[i];
    int64_t nnz = h->h_csr_rowptr[n];
    h->h_csr_col.resize(nnz);
    h->h_csr_src.resize(nnz);
    std::vector<int> next(h->h_csr_rowptr.begin(), h->h_csr_rowptr.end() - 1);
    for (int j = 0; j < n; ++j)
        for (int p = Ap[j]; p < Ap[j + 1]; ++p) {
            int i = Ai[p];
            int q = next[i]++;
            h->h_csr_col[q] = j;
            h->h_csr_src[q] = p;
            if (i != j) {
                q = next[j]++;
                h->h_csr_col[q] = i;
                h->h_csr_src[q] = p;
            }
        }
    h->csr.n = n;
    h->csr.nnz = nnz;
}

void finish_plan(mdgpu_handle_s* h) {
    build_plan(h->sym, h->sym.lower.nnz(), kLargeThreshold, h->plan);
    build_large_tables(h->plan, kTile, kAssembleCols);
    build_factor_schedule(h->plan, kTile, kAssembleCols, h->fsched);
    build_solve_schedule(h->plan, kTile, h->ssched);
    build_panel_schedule(h->plan, kTile, kPanel, kAssembleCols, h->pschedh);
    h->level = front_levels(h->plan);
}

void init_kernels_once() {
    static bool done = false;
    if (done) return;
    init_factor_kernels();
    init_solve_kernels();
    init_schur_tc();
    init_schur_f64();
    init_panel_kernels();
    init_selinv();
    done = true;
}

// Capture fn(stream) on the handle's own stream into an executable graph.
template <typename F>
cudaGraphExec_t capture(mdgpu_handle_s* h, F&& fn) {
    cudaGraph_t g = nullptr;
    ck(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal), "begin capture");
    fn(h->stream);
    cudaError_t e = cudaStreamEndCapture(h->stream, &g);
    ck(e, "end capture");
    cudaGraphExec_t ex = nullptr;
    ck(cudaGraphInstantiate(&ex, g, 0), "instantiate graph");
    cudaGraphDestroy(g);
    return ex;
}

void upload_plan(mdgpu_handle_s* h, bool check = false) {
    // check (or MDGPU_CHECK_PLAN=1): check every table the kernels index by
    // before any of it reaches the device (the analysis fails with the
    // broken invariant)
    const char* e = std::getenv("MDGPU_CHECK_PLAN");
    if (check || (e && e[0] == '1')) {
        std::string why =
            check_plan(h->plan, h->sym, h->ssched, h->level, h->h_csr_rowptr, h->h_csr_col.data(),
                       h->h_csr_src.data(), (int64_t)h->h_csr_col.size());
        if (why.empty()) why = check_panel_schedule(h->plan, h->pschedh, h->level, kTile, kPanel);
        if (!why.empty()) throw std::runtime_error("plan check: " + why);
    }
    if (!device_available()) return;
    init_kernels_once();
    ck(cudaGetDevice(&h->device), "cudaGetDevice");
    ck(cudaDeviceGetAttribute(&h->D.num_sms, cudaDevAttrMultiProcessorCount, h->device),
       "SM count");
    {
        // the no-allocation solve's scratch array: its address on this device
        // now, so that no solve loads its module (a failure here is reported
        // by that solve, which retries the look-up)
        std::string msg;
        if (!noalloc_scratch(msg)) cudaGetLastError();
    }
    h->on_device = true;
    ck(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking), "stream");
    ck(cudaEventCreateWithFlags(&h->D.fork_ev, cudaEventDisableTiming), "event");
    for (int i = 0; i < DevPlan::kSmallPieces; ++i) {
        ck(cudaStreamCreateWithFlags(&h->D.piece_st[i], cudaStreamNonBlocking), "stream");
        ck(cudaEventCreateWithFlags(&h->D.piece_join[i], cudaEventDisableTiming), "event");
    }
    const Plan& P = h->plan;
    DevPlan& D = h->D;
    D.n = P.n;
    D.nsuper = P.nsuper;
    D.nlevels = P.nlevels;
    D.max_u = std::max(P.max_u, 1);
    D.h_level_max_m.assign(P.nlevels, 0);
    for (int l = 0; l < P.nlevels; ++l)
        for (int q = P.large_ptr[l]; q < P.large_ptr[l + 1]; ++q)
            D.h_level_max_m[l] = std::max(D.h_level_max_m[l], P.fronts[P.large_list[q]].m);
    for (int s : P.large_list) {
        D.max_m_large = std::max(D.max_m_large, P.fronts[s].m);
        D.max_nch_large = std::max(D.max_nch_large, P.fronts[s].child_end - P.fronts[s].child_beg);
    }
    if ((size_t)D.max_u * sizeof(int) > 227 * 1024)
        throw std::runtime_error("update matrix order exceeds the assembly kernel's shared memory");
    D.fronts = h->keep(upload(P.fronts));
    D.child = h->keep(upload(P.child));
    D.rows = h->keep(upload(P.rows));
    D.relmap = h->keep(upload(P.relmap));
    D.a_src = h->keep(upload(P.a_src));
    D.a_pos = h->keep(upload(P.a_pos));
    D.a_colptr = h->keep(upload(P.a_colptr));
    D.a_colptr_off = h->keep(upload(P.a_colptr_off));
    D.small_list = h->keep(upload(P.small_list));
    D.large_list = h->keep(upload(P.large_list));
    D.h_small_ptr = P.small_ptr;
    D.h_large_ptr = P.large_ptr;
    const int64_t acc = h->ssched.fv_rows;
    D.fv_fronts = acc;
    // publication slots start on 16 bytes (copied with 16-byte cp.async)
    D.fv_pub_off = (acc + h->ssched.gather_vecs * kTile + 1) & ~(int64_t)1;
    D.fv_total = D.fv_pub_off + 2 * (int64_t)h->ssched.nflags * kTile;
    D.fv_off = h->keep(upload(h->ssched.fv_off));
    D.dinv_off = h->keep(upload(P.dinv_off));
    {
        // panel scratch (3xTF32 path): fronts of one level side by side,
        // levels reuse it
        h->pscr_off.assign(P.nsuper, -1);
        D.pscr_total = 0;
        for (int l = 0; l < P.nlevels; ++l) {
            int64_t off = 0;
            for (int q = P.large_ptr[l]; q < P.large_ptr[l + 1]; ++q) {
                const int s = P.large_list[q];
                h->pscr_off[s] = off;
                off += 2 * (int64_t)panel_mpad(P.fronts[s].m) * kScrCols;
            }
            D.pscr_total = std::max(D.pscr_total, off);
        }
        D.pscr_off = h->keep(upload(h->pscr_off));
    }
    D.asm_off = h->keep(upload(P.asm_off));
    D.asm_range = h->keep(upload(P.asm_range));
    D.dinv_total = P.dinv_total;
    {
        // selected inverse: supernodes by level, Y scratch per level's fronts
        // side by side (levels reuse it), each lower entry's front
        const std::vector<int>& lv = h->level;
        D.h_level_ptr.assign(P.nlevels + 1, 0);
        for (int s = 0; s < P.nsuper; ++s) D.h_level_ptr[lv[s] + 1]++;
        for (int l = 0; l < P.nlevels; ++l) D.h_level_ptr[l + 1] += D.h_level_ptr[l];
        std::vector<int> ll(std::max(P.nsuper, 1)), nxt(D.h_level_ptr.begin(), D.h_level_ptr.end() - 1);
        for (int s = 0; s < P.nsuper; ++s) ll[nxt[lv[s]]++] = s;
        D.level_list = h->keep(upload(ll));
        // Y scratch: m x 16 for a small front (one CTA), 2 m x 64 for a
        // large one (Y and a row-major copy of Z_RK); a level's fronts side
        // by side, levels reuse it
        std::vector<char> large(P.nsuper, 0);
        for (int s : P.large_list) large[s] = 1;
        std::vector<int64_t> yo(P.nsuper, 0);
        D.yscr_total = 0;
        for (int l = 0; l < P.nlevels; ++l) {
            int64_t off = 0;
            for (int q = D.h_level_ptr[l]; q < D.h_level_ptr[l + 1]; ++q) {
                const int s = ll[q];
                yo[s] = off;
                off += (int64_t)P.fronts[s].m * (large[s] ? 2 * selinv_tile() : selinv_block());
            }
            D.yscr_total = std::max(D.yscr_total, off);
        }
        D.yoff = h->keep(upload(yo));
        // the large fronts' selected-inverse work lists
        {
            const int T = selinv_tile();
            ListStore st;
            SelSchedule& SS = D.sel;
            SS.h_gather.assign(P.nlevels, WorkList{0, 0, 0, 0});
            SS.h_step_beg.assign(P.nlevels + 1, 0);
            for (int l = 0; l < P.nlevels; ++l) {
                SS.h_step_beg[l] = (int)SS.h_steps.size();
                std::vector<std::pair<int, int>> g;
                int maxb = 0;
                for (int q = P.large_ptr[l]; q < P.large_ptr[l + 1]; ++q) {
                    const FrontDesc& f = P.fronts[P.large_list[q]];
                    if (f.parent >= 0 && f.m > f.c) g.push_back({P.large_list[q], (f.m - f.c + 15) / 16});
                    maxb = std::max(maxb, (f.c + T - 1) / T);
                }
                if (!g.empty()) SS.h_gather[l] = st.add(g, 0);
                for (int t = 0; t < maxb; ++t) {
                    std::vector<std::pair<int, int>> w;
                    for (int q = P.large_ptr[l]; q < P.large_ptr[l + 1]; ++q) {
                        const int s = P.large_list[q];
                        const FrontDesc& f = P.fronts[s];
                        const int nblk = (f.c + T - 1) / T;
                        if (t >= nblk) continue;
                        const int k1 = std::min((nblk - t) * T, f.c);
                        w.push_back({s, (f.m - k1 + T - 1) / T});
                    }
                    SS.h_steps.push_back(st.add(w, t));
                }
            }
            SS.h_step_beg[P.nlevels] = (int)SS.h_steps.size();
            if (st.items.empty()) {
                st.items.assign(1, -1);
                st.ctas_before.assign(1, 0);
            }
            SS.items = h->keep(upload(st.items));
            SS.before = h->keep(upload(st.ctas_before));
        }
        // the general reverse mode: gather lists, L's column pointers, the
        // c x c scratch of every front (a level's fronts side by side)
        {
            AdjSchedule& AS = D.adj;
            ListStore st;
            AS.h_gather.assign(P.nlevels, WorkList{0, 0, 0, 0});
            std::vector<int64_t> wo(P.nsuper, 0);
            AS.wtotal = 1;
            for (int l = 0; l < P.nlevels; ++l) {
                std::vector<std::pair<int, int>> g;
                int64_t off = 0;
                for (int q = D.h_level_ptr[l]; q < D.h_level_ptr[l + 1]; ++q) {
                    const int s = ll[q];
                    const FrontDesc& f = P.fronts[s];
                    wo[s] = off;
                    off += (int64_t)f.c * f.c;
                    if (f.parent >= 0 && f.m > f.c) g.push_back({s, (f.m - f.c + 15) / 16});
                }
                AS.wtotal = std::max(AS.wtotal, off);
                if (!g.empty()) AS.h_gather[l] = st.add(g, 0);
            }
            if (st.items.empty()) {
                st.items.assign(1, -1);
                st.ctas_before.assign(1, 0);
            }
            AS.items = h->keep(upload(st.items));
            AS.before = h->keep(upload(st.ctas_before));
            AS.woff = h->keep(upload(wo));
            AS.Lp = h->keep(upload(P.Lp));
        }
        {
            std::vector<int64_t> zo = P.zuoff;
            if (zo.empty()) zo.assign(1, -1);
            D.zuoff = h->keep(upload(zo));
        }
        std::vector<int> af(std::max<size_t>(P.a_src.size(), 1), 0);
        for (int s = 0; s < P.nsuper; ++s)
            for (int e = P.fronts[s].a_beg; e < P.fronts[s].a_end; ++e) af[e] = s;
        D.a_front = h->keep(upload(af));
    }
    D.sched64.items = h->keep(upload(h->fsched.store.items));
    D.sched64.before = h->keep(upload(h->fsched.store.ctas_before));
    D.sched64.h_level_beg = h->fsched.level_beg;
    D.sched64.h_trsm = h->fsched.trsm;
    D.sched64.h_update = h->fsched.update;
    D.h_assemble = h->fsched.assemble;
    D.psched.items = h->keep(upload(h->pschedh.store.items));
    D.psched.before = h->keep(upload(h->pschedh.store.ctas_before));
    D.psched.h_op_beg = h->pschedh.op_beg;
    D.psched.h_ops = h->pschedh.ops;
    {
        std::vector<int> pt = h->pschedh.tasks;
        if (pt.empty()) pt.assign(2, 0);
        D.psched.tasks = reinterpret_cast<int2*>(h->keep(upload(pt)));
        D.fsync_flags = h->pschedh.ncounters;
        D.nflags_factor = (int)h->pschedh.nflags;
        D.nfsync = D.fsync_flags + 2 * D.nflags_factor + 1;
        D.fsync = h->keep(dalloc<int>(D.nfsync));
        ck(cudaMemset(D.fsync, 0, (size_t)D.nfsync * sizeof(int)), "panel sync words");
    }
    {
        const SolveScheduleHost& SS = h->ssched;
        std::vector<int> tasks = SS.tasks;
        if (tasks.empty()) tasks.assign(2, 0);
        D.solve.tasks = reinterpret_cast<int2*>(h->keep(upload(tasks)));
        D.solve.fwd_task_beg = SS.fwd_task_beg;
        D.solve.bwd_task_beg = SS.bwd_task_beg;
        D.solve.fwd_elems = SS.fwd_elems;
        D.solve.bwd_elems = SS.bwd_elems;
        D.solve.small_elems = SS.small_elems;
        D.solve.gather_task_beg = SS.gather_task_beg;
        D.solve.amap_off = h->keep(upload(SS.amap_off));
        D.solve.amap_row = h->keep(upload(SS.amap_row));
        D.solve.amap_ent = h->keep(upload(SS.amap_ent));
        D.solve.warp_list = h->keep(upload(SS.warp_list));
        D.solve.warp_cnt = SS.warp_cnt;
        D.solve.gather_nch = h->keep(upload(SS.gather_nch));
        D.solve.gather_off = h->keep(upload(SS.gather_off));
        D.solve.nflags = SS.nflags;
        auto items = [&](const std::vector<int>& v, int& n) {
            n = (int)(v.size() / 4);
            std::vector<int> w = v;
            if (w.empty()) w.assign(4, 0);
            return reinterpret_cast<int4*>(h->keep(upload(w)));
        };
        D.solve.fwd_items = items(SS.fwd_items, D.solve.nfwd_items);
        D.solve.bwd_items = items(SS.bwd_items, D.solve.nbwd_items);
        {
            std::vector<int> wf = SS.fwd_wlist, wb = SS.bwd_wlist;
            if (wf.empty()) wf.assign(1, 0);
            if (wb.empty()) wb.assign(1, 0);
            D.solve.fwd_wlist = h->keep(upload(wf));
            D.solve.bwd_wlist = h->keep(upload(wb));
        }
        D.solve.bwd_target = h->keep(upload(SS.bwd_target));
        D.solve.nfronts = P.nsuper;
        D.solve.nsync = 3 + SS.nflags + 3 * P.nsuper;
        D.solve.sync = h->keep(dalloc<int>(D.solve.nsync));
    }
    // algorithmic work per launch, for the profiler's roofline figures
    {
        const TileSchedule& TS = h->fsched;
        D.h_update_flops.assign(TS.update.size(), 0.0);
        for (size_t q = 0; q < TS.update.size(); ++q) {
            const WorkList& w = TS.update[q];
            int k = w.step;
            double fl = 0;
            for (int it = 0; it < w.nitems; ++it) {
                const FrontDesc& f = P.fronts[TS.store.items[w.off + it]];
                int NT = front_tiles(f.m, f.c, kTile);
                double K = std::min(kTile, f.c - k * kTile);
                auto sz = [&](int t) {
                    int nt1 = (f.c + kTile - 1) / kTile;
                    if (t < nt1) return std::min(kTile, f.c - t * kTile);
                    int s0 = f.c + (t - nt1) * kTile;
                    return std::min(kTile, f.m - s0);
                };
                for (int i = k + 1; i < NT; ++i) {
                    double ri = sz(i);
                    fl += K * ri * (ri + 1);  // diagonal tile, lower part
                    for (int j = k + 1; j < i; ++j) fl += 2.0 * K * ri * sz(j);
                }
            }
            D.h_update_flops[q] = fl;
        }
        D.h_small_bytes.assign(P.small_ptr.size(), 0.0);
        for (size_t b = 0; b + 1 < P.small_ptr.size(); ++b) {
            double by = 0;
            for (int q = P.small_ptr[b]; q < P.small_ptr[b + 1]; ++q) {
                const FrontDesc& f = P.fronts[P.small_list[q]];
                double u = f.m - f.c;
                by += (f.a_end - f.a_beg) * 16.0 + 8.0 * f.m * f.c;
                if (f.uoff >= 0) by += 8.0 * u * (u + 1) / 2;
                for (int hh = f.child_beg; hh < f.child_end; ++hh) {
                    const FrontDesc& g = P.fronts[P.child[hh]];
                    double uc = g.m - g.c;
                    by += 8.0 * uc * (uc + 1) / 2 + 4.0 * uc;
                }
            }
            D.h_small_bytes[b] = by;
        }
    }
    D.prof = &h->prof;
    if (!P.perm.empty()) h->d_perm = h->keep(upload(P.perm));
    // not-SPD column, device wait error, solve error, FP64 diagonal tiles
    h->d_status = h->keep(dalloc<int>(4));
    D.solve.err = h->d_status + 2;
    h->d_Ax = dalloc<double>(std::max<int64_t>(P.nnz_user, 1));
    h->csr.rowptr = h->keep(upload(h->h_csr_rowptr));
    h->csr.col = h->keep(upload(h->h_csr_col));
    h->csr.src = h->keep(upload(h->h_csr_src));
}

int fail(int status, const std::string& msg) {
    g_last_error = msg;
    return status;
}

template <typename F>
int guarded(F&& f) {
    try {
        return f();
    } catch (const CudaError& e) {
        return fail(MDGPU_ERR_CUDA, e.what());
    } catch (const std::bad_alloc&) {
        return fail(MDGPU_ERR_OOM, "allocation failed");
    } catch (const std::exception& e) {
        return fail(MDGPU_ERR_INVALID, e.what());
    }
}

cudaStream_t pick_stream(mdgpu_handle_s* h, void* s) {
    return s ? static_cast<cudaStream_t>(s) : h->stream;
}

void ensure_factor_storage(mdgpu_handle_s* h, int precision) {
    const Plan& P = h->plan;
    if (precision == MDGPU_FP64) {
        if (!h->dL64) h->dL64 = dalloc<double>(P.lstore);
        if (!h->dU64) h->dU64 = dalloc<double>(P.ustore);
        if (!h->dD64) h->dD64 = dalloc<double>(P.dinv_total);
    } else {
        if (!h->dL32) {
            h->dL32 = dalloc<float>(P.lstore);
            // the split panel scratch and its TMA descriptors (3xTF32
            // tensor-core Schur updates)
            if (h->use_tensor_cores && !P.large_list.empty()) {
                h->D.pscr = h->keep(dalloc<float>(std::max<int64_t>(h->D.pscr_total, 1)));
                std::vector<CUtensorMap> maps;
                std::vector<int> idx;
                if (build_panel_maps(P, h->D.pscr, h->pscr_off, maps, idx, false) == 0) {
                    h->D.tmaps = h->keep(upload(maps));
                    h->D.tmap_idx = h->keep(upload(idx));
                }
            }
        }
        if (!h->dU32) h->dU32 = dalloc<float>(P.ustore);
        if (!h->dD32) h->dD32 = dalloc<float>(P.dinv_total);
        // the same scratch read as the BF16 copy of the panels (BF16 Schur
        // updates)
        if (precision == MDGPU_BF16 && !h->D.tmaps_bf16 && h->D.pscr) {
            std::vector<CUtensorMap> maps;
            std::vector<int> idx;
            if (build_panel_maps(P, h->D.pscr, h->pscr_off, maps, idx, true) == 0)
                h->D.tmaps_bf16 = h->keep(upload(maps));
        }
    }
}

void ensure_solve_storage(mdgpu_handle_s* h, int nrhs) {
    if (nrhs <= h->nrhs_cap) return;
    h->drop_solve_graphs();  // they reference the buffers replaced below
    for (double** p : {&h->d_xp, &h->d_fv, &h->d_B, &h->d_X, &h->d_R, &h->d_D})
        if (*p) {
            cudaFree(*p);
            *p = nullptr;
        }
    if (h->d_norms) {
        cudaFree(h->d_norms);
        h->d_norms = nullptr;
    }
    int64_t n = h->plan.n;
    int chunk = std::min(nrhs, 64);
    h->d_xp = dalloc<double>(n * nrhs);
    h->d_fv = dalloc<double>(h->D.fv_total * chunk);
    h->d_B = dalloc<double>(n * nrhs);
    h->d_X = dalloc<double>(n * nrhs);
    h->d_R = dalloc<double>(n * nrhs);
    h->d_D = dalloc<double>(n * nrhs);
    h->d_norms = dalloc<unsigned long long>(1 + 3 * nrhs);
    h->nrhs_cap = nrhs;
}

int do_factor_once(mdgpu_handle_s* h, const double* dAx, int precision, cudaStream_t st);

// MDGPU_BF16 or MDGPU_TF32 whose factorization meets a non-positive pivot
// (the rounding of the Schur updates' operands can destroy definiteness when
// cond(A) u is near 1) is factored again in FP32; precision_used records
// which factor the handle holds.
int do_factor(mdgpu_handle_s* h, const double* dAx, int precision, cudaStream_t st) {
    int rc = do_factor_once(h, dAx, precision, st);
    if (rc == MDGPU_ERR_NOT_SPD && (precision == MDGPU_BF16 || precision == MDGPU_TF32)) {
        rc = do_factor_once(h, h->d_Ax, MDGPU_FP32, st);
        if (rc == MDGPU_OK) h->bf16_fallbacks++;
    }
    return rc;
}

int do_factor_once(mdgpu_handle_s* h, const double* dAx, int precision, cudaStream_t st) {
    NvtxRange nvtx("mdgpu_factor");
    if (precision != MDGPU_FP64 && precision != MDGPU_FP32 && precision != MDGPU_BF16 &&
        precision != MDGPU_TF32)
        return fail(MDGPU_ERR_INVALID, "unknown precision");
    ck(cudaSetDevice(h->device), "cudaSetDevice");
    ensure_factor_storage(h, precision);
    h->selinv_done = false;
    if (dAx != h->d_Ax)
        ck(cudaMemcpyAsync(h->d_Ax, dAx, h->plan.nnz_user * sizeof(double),
                           cudaMemcpyDeviceToDevice, st),
           "copy values");
    const int big = INT_MAX;
    h->status_init[0] = big;
    h->status_init[1] = 0;
    ck(cudaMemcpyAsync(h->d_status, h->status_init, 2 * sizeof(int), cudaMemcpyHostToDevice, st),
       "status");
    ck(cudaMemsetAsync(h->d_status + 3, 0, sizeof(int), st), "status");
    auto run = [h, precision](cudaStream_t s) {
        if (precision == MDGPU_FP64)
            factor_levels<double>(h->D, h->dL64, h->dU64, h->dD64, h->d_Ax, h->d_status, s);
        else
            factor_levels<float>(h->D, h->dL32, h->dU32, h->dD32, h->d_Ax, h->d_status, s,
                                 precision == MDGPU_BF16   ? kSchurBF16
                                 : precision == MDGPU_TF32 ? kSchur1xTF32
                                                           : kSchur3xTF32);
    };
    if (h->use_graphs && !h->prof.on) {
        cudaGraphExec_t& g = h->fgraph[precision];
        if (!g) g = capture(h, run);
        ck(cudaGraphLaunch(g, st), "factor graph");
    } else {
        run(st);
    }
    ck(cudaGetLastError(), "factor launch");
    int stat[4] = {big, 0, 0, 0};
    ck(cudaMemcpyAsync(stat, h->d_status, 4 * sizeof(int), cudaMemcpyDeviceToHost, st), "status");
    ck(cudaStreamSynchronize(st), "factor");
    h->fp64_diag_tiles = stat[3];
    int col = stat[0];
    if (stat[1] != 0) {
        h->factored = -1;
        return fail(MDGPU_ERR_CUDA,
                    "factor: a device wait timed out (code " + std::to_string(stat[1]) +
                        ": 1-2 tensor-core pipeline, 3 panel dependency, 4 panel ticket)");
    }
    h->factored = precision;
    h->selinv_done = false;
    h->not_spd = (col == big) ? -1 : col;
    if (h->not_spd >= 0) {
        h->factored = -1;
        return fail(MDGPU_ERR_NOT_SPD,
                    "non-positive pivot at permuted column " + std::to_string(h->not_spd));
    }
    return MDGPU_OK;
}

// dB, dX device, original ordering; chunks of at most 64 right-hand sides
void do_solve(mdgpu_handle_s* h, const double* dB, int ldb, double* dX, int ldx, int nrhs,
              cudaStream_t st) {
    NvtxRange nvtx("mdgpu_solve");
    const int n = h->plan.n;
    for (int q0 = 0; q0 < nrhs; q0 += 64) {
        int nq = std::min(64, nrhs - q0);
        permute_gather(h->d_perm, dB + (int64_t)q0 * ldb, h->d_xp, n, nq, ldb, st);
        const int prec = h->factored;
        auto run = [h, prec, nq](cudaStream_t s) {
            if (prec == MDGPU_FP64)
                solve_levels<double, double>(h->D, h->dL64, h->dD64, h->d_xp, h->d_fv, nq, s);
            else
                solve_levels<float, double>(h->D, h->dL32, h->dD32, h->d_xp, h->d_fv, nq, s);
        };
        if (h->use_graphs && !h->prof.on) {
            cudaGraphExec_t& g = h->sgraph[prec * 1024 + nq];
            if (!g) g = capture(h, run);
            ck(cudaGraphLaunch(g, st), "solve graph");
        } else {
            run(st);
        }
        permute_scatter(h->d_perm, h->d_xp, dX + (int64_t)q0 * ldx, n, nq, ldx, st);
    }
    ck(cudaGetLastError(), "solve launch");
}

int do_refine(mdgpu_handle_s* h, const double* dB, int ldb, double* dX, int ldx, int nrhs,
              double tol, int maxit, double* berr, int* iters, cudaStream_t st) {
    NvtxRange nvtx("mdgpu_refine");
    const int n = h->plan.n;
    ensure_solve_storage(h, nrhs);
    launch_anorm(h->csr, h->d_Ax, h->d_norms, st);
    do_solve(h, dB, ldb, dX, ldx, nrhs, st);
    std::vector<unsigned long long> raw(1 + 3 * nrhs);
    std::vector<double> be(nrhs, 0.0);
    int it = 0;
    for (;; ++it) {
        launch_residual(h->csr, h->d_Ax, dX, ldx, dB, ldb, h->d_R, n, nrhs, st);
        launch_absmax3(n, nrhs, h->d_R, n, dX, ldx, dB, ldb, h->d_norms + 1, st);
        ck(cudaMemcpyAsync(raw.data(), h->d_norms, raw.size() * sizeof(unsigned long long),
                           cudaMemcpyDeviceToHost, st),
           "norms");
        ck(cudaStreamSynchronize(st), "refine");
        double anorm;
        std::memcpy(&anorm, &raw[0], sizeof(double));
        bool done = true;
        for (int q = 0; q < nrhs; ++q) {
            double nr, nx, nb;
            std::memcpy(&nr, &raw[1 + 3 * q], sizeof(double));
            std::memcpy(&nx, &raw[2 + 3 * q], sizeof(double));
            std::memcpy(&nb, &raw[3 + 3 * q], sizeof(double));
            double den = anorm * nx + nb;
            be[q] = den > 0 ? nr / den : 0.0;
            if (!(be[q] <= tol)) done = false;
        }
        if (done || it >= maxit) break;
        do_solve(h, h->d_R, n, h->d_D, n, nrhs, st);
        launch_axpy(n, nrhs, h->d_D, dX, ldx, st);
    }
    if (berr) std::copy(be.begin(), be.end(), berr);
    if (iters) *iters = it;
    return MDGPU_OK;
}

// GMRES-IR on the device: the vector backend of gmres_ir() over one
// right-hand side; the preconditioner is the solve with the current factor.
struct DeviceGmresOps {
    mdgpu_handle_s* h;
    cudaStream_t st;
    int n, kmax;
    double anorm;
    double *V, *tmp, *slots, *coef, *partial;

    double* basis(int k) { return V + (int64_t)k * n; }
    double* scratch() { return tmp; }
    void residual(const double* x, const double* b, double* r) {
        launch_residual(h->csr, h->d_Ax, x, n, b, n, r, n, 1, st);
    }
    double backward_error(const double* r, const double* x, const double* b) {
        launch_absmax3(n, 1, r, n, x, n, b, n, h->d_norms + 1, st);
        unsigned long long raw[3];
        ck(cudaMemcpyAsync(raw, h->d_norms + 1, sizeof(raw), cudaMemcpyDeviceToHost, st), "norms");
        ck(cudaStreamSynchronize(st), "gmres-ir");
        double nr, nx, nb;
        std::memcpy(&nr, &raw[0], sizeof(double));
        std::memcpy(&nx, &raw[1], sizeof(double));
        std::memcpy(&nb, &raw[2], sizeof(double));
        const double den = anorm * nx + nb;
        return den > 0 ? nr / den : 0.0;
    }
    void precond(const double* r, double* z) { do_solve(h, r, n, z, n, 1, st); }
    void spmv(const double* v, double* w) { launch_spmv(h->csr, h->d_Ax, v, w, st); }
    void dots(int k, const double* w, int s) {
        launch_dots(n, k, V, n, w, partial, slots + (int64_t)s * kmax, st);
    }
    void sub(int k, int s, double* w) {
        launch_gemv_acc(n, k, V, n, slots + (int64_t)s * kmax, -1.0, w, st);
    }
    void norm2_to_slot(const double* w) {
        launch_dots(n, 1, w, n, w, partial, slots + 2 * (int64_t)kmax, st);
    }
    void fetch(double* host) {
        ck(cudaMemcpyAsync(host, slots, (2 * (size_t)kmax + 1) * sizeof(double),
                           cudaMemcpyDeviceToHost, st),
           "gmres slots");
        ck(cudaStreamSynchronize(st), "gmres-ir");
    }
    void scale(double alpha, double* w) { launch_scale(n, alpha, w, st); }
    void add(int k, const double* y, double* x) {
        ck(cudaMemcpyAsync(coef, y, k * sizeof(double), cudaMemcpyHostToDevice, st), "gmres y");
        launch_gemv_acc(n, k, V, n, coef, 1.0, x, st);
    }
};

int do_gmres_ir(mdgpu_handle_s* h, const double* dB, int ldb, double* dX, int ldx, int nrhs,
                const GmresIrParams& prm, double* berr, int* outer, int* inner, cudaStream_t st) {
    NvtxRange nvtx("mdgpu_gmres_ir");
    const int n = h->plan.n, kmax = prm.restart;
    ensure_solve_storage(h, 1);
    // basis (kmax + 1 vectors), one scratch vector, the slots (2 kmax + 1) and
    // the correction's coefficients (kmax), the partial sums of the dots
    const int64_t need = (int64_t)n * (kmax + 2) + 3 * (int64_t)kGmresMaxRestart + 1 +
                         dots_partial_size(kGmresMaxRestart);
    if (need > h->gm_cap) {
        if (h->d_gm) cudaFree(h->d_gm);
        h->d_gm = nullptr;
        h->gm_cap = 0;
        h->d_gm = dalloc<double>(need);
        h->gm_cap = need;
    }
    DeviceGmresOps ops;
    ops.h = h;
    ops.st = st;
    ops.n = n;
    ops.kmax = kmax;
    ops.V = h->d_gm;
    ops.tmp = ops.V + (int64_t)n * (kmax + 1);
    ops.slots = ops.tmp + n;
    ops.coef = ops.slots + 2 * kGmresMaxRestart + 1;
    ops.partial = ops.coef + kGmresMaxRestart;
    launch_anorm(h->csr, h->d_Ax, h->d_norms, st);
    unsigned long long raw;
    ck(cudaMemcpyAsync(&raw, h->d_norms, sizeof(raw), cudaMemcpyDeviceToHost, st), "norm");
    ck(cudaStreamSynchronize(st), "gmres-ir");
    std::memcpy(&ops.anorm, &raw, sizeof(double));
    for (int q = 0; q < nrhs; ++q) {
        const GmresIrResult r =
            gmres_ir(ops, dX + (int64_t)q * ldx, dB + (int64_t)q * ldb, prm);
        if (berr) berr[q] = r.berr;
        if (outer) outer[q] = r.outer;
        if (inner) inner[q] = r.inner;
    }
    return MDGPU_OK;
}

// The same full symmetric CSR for independent systems given one by one: the
// block-diagonal matrix's rows hold only their own system's entries, in the
// same order as build_csr over the concatenation; the systems are filled in
// parallel.
void build_csr_batch(mdgpu_handle_s* h, int nsys, const int* n, const int* const* Ap,
                     const int* const* Ai, const std::vector<int>& row_off,
                     const std::vector<int>& val_off) {
    const int N = row_off[nsys];
    std::vector<int> cnt(N, 0);
    parallel_for(nsys, [&](int b) {
        int* cb = cnt.data() + row_off[b];
        for (int j = 0; j < n[b]; ++j)
            for (int p = Ap[b][j]; p < Ap[b][j + 1]; ++p) {
                const int i = Ai[b][p];
                cb[i]++;
                if (i != j) cb[j]++;
            }
    });
    h->h_csr_rowptr.assign(N + 1, 0);
    for (int i = 0; i < N; ++i) h->h_csr_rowptr[i + 1] = h->h_csr_rowptr[i] + cnt[i];
    const int64_t nnz = h->h_csr_rowptr[N];
    h->h_csr_col.resize(nnz);
    h->h_csr_src.resize(nnz);
    parallel_for(nsys, [&](int b) {
        const int r0 = row_off[b];
        std::vector<int> next(h->h_csr_rowptr.begin() + r0, h->h_csr_rowptr.begin() + r0 + n[b]);
        for (int j = 0; j < n[b]; ++j)
            for (int p = Ap[b][j]; p < Ap[b][j + 1]; ++p) {
                const int i = Ai[b][p];
                int q = next[i]++;
                h->h_csr_col[q] = j + r0;
                h->h_csr_src[q] = p + val_off[b];
                if (i != j) {
                    q = next[j]++;
                    h->h_csr_col[q] = i + r0;
                    h->h_csr_src[q] = p + val_off[b];
                }
            }
    });
    h->csr.n = N;
    h->csr.nnz = nnz;
}

// One symbolic result for independent systems: the block-diagonal matrix of
// their lower triangles, each system analysed on its own (so each keeps its
// own bit-exact ordering and tree); rows, supernodes, L columns and the
// value sources are offset system by system.  The assembly forest has one
// tree per system.
void combine_symbolic(const std::vector<Symbolic>& parts, const std::vector<int>& val_off,
                      Symbolic& S) {
    S = Symbolic();
    const int nsys = (int)parts.size();
    // each system's first row, supernode, lower entry, child entry, L entry
    // and value in the concatenated arrays
    std::vector<int64_t> ro(nsys + 1, 0), so(nsys + 1, 0), eo(nsys + 1, 0), co(nsys + 1, 0),
        lo(nsys + 1, 0), vo(nsys + 1, 0);
    bool any_perm = false, any_relax = false;
    for (int b = 0; b < nsys; ++b) {
        const Symbolic& p = parts[b];
        ro[b + 1] = ro[b] + p.n;
        so[b + 1] = so[b] + p.tree.size();
        eo[b + 1] = eo[b] + p.lower.nnz();
        co[b + 1] = co[b] + (int64_t)p.tree.child.size();
        lo[b + 1] = lo[b] + p.Lp.back();
        vo[b + 1] = vo[b] + (int64_t)p.lower.val.size();
        any_perm = any_perm || !p.perm.empty();
        any_relax = any_relax || !p.relax_perm.empty();
    }
    if (eo[nsys] > INT_MAX) throw std::runtime_error("batch too large for 32-bit entry indices");
    const int n = (int)ro[nsys];
    const int ns = (int)so[nsys];
    S.n = n;
    S.lower.nrows = S.lower.ncols = n;
    if (any_perm) S.perm.resize(n);
    if (any_relax) S.relax_perm.resize(n);
    S.parent.resize(n);
    S.post.resize(n);
    S.count0.resize(n);
    S.count.resize(n);
    S.lower.colptr.resize(n + 1);
    S.lower.rowidx.resize(eo[nsys]);
    S.lower.val.resize(vo[nsys]);
    S.lower_src.resize(eo[nsys]);
    S.tree.first_col.resize(ns);
    S.tree.ncols.resize(ns);
    S.tree.child_ptr.resize(ns + 1);
    S.tree.child.resize(co[nsys]);
    S.Lp.resize(n + 1);
    S.lower.colptr[0] = 0;
    S.tree.child_ptr[0] = 0;
    S.Lp[0] = 0;
    // the systems' slices are disjoint: filled in parallel
    parallel_for(nsys, [&](int b) {
        const Symbolic& p = parts[b];
        const int r0 = (int)ro[b], s0 = (int)so[b];
        const int64_t e0 = eo[b], c0 = co[b], l0 = lo[b];
        for (int i = 0; i < p.n; ++i) {
            if (any_perm) S.perm[r0 + i] = p.perm.empty() ? r0 + i : p.perm[i] + r0;
            if (any_relax)
                S.relax_perm[r0 + i] = p.relax_perm.empty() ? r0 + i : p.relax_perm[i] + r0;
            S.parent[r0 + i] = p.parent[i] < 0 ? p.parent[i] : p.parent[i] + r0;
            S.post[r0 + i] = p.post[i] + r0;
            S.count0[r0 + i] = p.count0[i];
            S.count[r0 + i] = p.count[i];
            S.lower.colptr[r0 + i + 1] = (int)(e0 + p.lower.colptr[i + 1]);
            S.Lp[r0 + i + 1] = l0 + p.Lp[i + 1];
        }
        for (int64_t q = 0; q < p.lower.nnz(); ++q) {
            S.lower.rowidx[e0 + q] = p.lower.rowidx[q] + r0;
            const int src = p.lower_src[q];
            S.lower_src[e0 + q] = src < 0 ? src : src + val_off[b];
        }
        std::copy(p.lower.val.begin(), p.lower.val.end(), S.lower.val.begin() + vo[b]);
        for (int s = 0; s < p.tree.size(); ++s) {
            S.tree.first_col[s0 + s] = p.tree.first_col[s] + r0;
            S.tree.ncols[s0 + s] = p.tree.ncols[s];
            S.tree.child_ptr[s0 + s + 1] = (int)(c0 + p.tree.child_ptr[s + 1]);
        }
        for (size_t k = 0; k < p.tree.child.size(); ++k)
            S.tree.child[c0 + k] = p.tree.child[k] + s0;
    });
}

// Solve error word (d_status[2]): cleared before a public solve call, read
// after it; bit 0 = a dependency wait of the large-front solve ran out,
// bit 1 = a solve kernel found its ticket counter not cleared.
void solve_status_reset(mdgpu_handle_s* h, cudaStream_t st) {
    ck(cudaMemsetAsync(h->d_status + 2, 0, sizeof(int), st), "clear solve status");
}
int solve_status_check(mdgpu_handle_s* h, cudaStream_t st) {
    int e = 0;
    ck(cudaMemcpyAsync(&e, h->d_status + 2, sizeof(int), cudaMemcpyDeviceToHost, st),
       "solve status");
    ck(cudaStreamSynchronize(st), "solve");
    if (e != 0)
        return fail(MDGPU_ERR_CUDA, "large-front solve aborted (status " + std::to_string(e) +
                                        "): a dependency wait ran out");
    return MDGPU_OK;
}

// Validation and symbolic analysis of independent systems, shared by the
// batch analysis and the cost estimate.  The analyses are independent: one
// host thread per core, systems taken in order from a shared counter; the
// first failing system (lowest index) is reported.  With offsets, row_off /
// val_off receive the systems' first row and first value in the
// concatenation (32-bit, checked); given flops, each system's analysis is
// reduced to its flop count (sum over columns of count^2 + 1, as the plan's)
// and its L entries (lnz, optional), then dropped, and parts stays empty.
int analyze_systems(int nsys, const int* n, const int* const* Ap, const int* const* Ai,
                    int ordering, int tree, int relax_zeros, bool offsets,
                    std::vector<Symbolic>& parts, std::vector<int>& row_off,
                    std::vector<int>& val_off, double* flops, long long* lnz) {
    row_off.assign(nsys + 1, 0);
    val_off.assign(nsys + 1, 0);
    for (int b = 0; b < nsys; ++b) {
        const int nb = n[b];
        if (nb <= 0 || !Ap[b] || !Ai[b])
            return fail(MDGPU_ERR_INVALID, "bad arguments of system " + std::to_string(b));
        for (int j = 0; j < nb; ++j) {
            if (Ap[b][j + 1] < Ap[b][j])
                return fail(MDGPU_ERR_INVALID,
                            "column pointers decrease in system " + std::to_string(b));
            for (int p = Ap[b][j]; p < Ap[b][j + 1]; ++p)
                if (Ai[b][p] < j || Ai[b][p] >= nb)
                    return fail(MDGPU_ERR_INVALID,
                                "entry outside the lower triangle in system " + std::to_string(b));
        }
        if (offsets) {
            if ((int64_t)row_off[b] + nb > INT_MAX || (int64_t)val_off[b] + Ap[b][nb] > INT_MAX)
                return fail(MDGPU_ERR_INVALID, "batch too large for 32-bit indices");
            row_off[b + 1] = row_off[b] + nb;
            val_off[b + 1] = val_off[b] + Ap[b][nb];
        }
    }
    const bool keep = flops == nullptr;
    std::vector<int> rc(nsys, 0);
    std::vector<std::string> what(nsys);
    parallel_for(nsys, [&](int b) {
        Symbolic one;
        Symbolic& S = keep ? parts[b] : one;
        try {
            rc[b] = analyze(n[b], Ap[b], Ai[b], nullptr, ordering == MDGPU_ORDER_AMD,
                            (TreeKind)tree, relax_zeros, S) != 0
                        ? 1
                        : 0;
            if (!keep && rc[b] == 0) {
                double f = 0.0;
                for (int j = 0; j < n[b]; ++j) f += (double)S.count[j] * S.count[j] + 1.0;
                flops[b] = f;
                if (lnz) lnz[b] = (long long)S.Lp[n[b]];
            }
        } catch (const std::bad_alloc&) {
            rc[b] = 2;
        } catch (const std::exception& e) {
            rc[b] = 3;
            what[b] = e.what();
        }
    });
    for (int b = 0; b < nsys; ++b) {
        if (rc[b] == 1)
            return fail(MDGPU_ERR_NOT_TREE,
                        "the elimination tree of system " + std::to_string(b) + " is a forest");
        if (rc[b] == 2) throw std::bad_alloc();
        if (rc[b] == 3) throw std::runtime_error("system " + std::to_string(b) + ": " + what[b]);
    }
    return MDGPU_OK;
}

// Argument check of the GMRES-IR entry points.
int check_gmres_args(int maxit, int restart, double inner_tol) {
    if (maxit < 0) return fail(MDGPU_ERR_INVALID, "maxit must be >= 0");
    if (restart < 1 || restart > kGmresMaxRestart)
        return fail(MDGPU_ERR_INVALID, "restart must be in 1..64");
    if (!(inner_tol >= 0.0)) return fail(MDGPU_ERR_INVALID, "inner_tol must be >= 0");
    return MDGPU_OK;
}

// Argument check shared by the solve entry points; names the offending argument.
int check_solve_args(mdgpu_handle_s* h, const void* B, int ldb, const void* X, int ldx,
                     int nrhs) {
    if (!h) return fail(MDGPU_ERR_INVALID, "null handle");
    if (!B || !X) return fail(MDGPU_ERR_INVALID, "null right-hand side or solution pointer");
    if (nrhs <= 0) return fail(MDGPU_ERR_INVALID, "nrhs must be positive, got " + std::to_string(nrhs));
    if (ldb < h->plan.n || ldx < h->plan.n)
        return fail(MDGPU_ERR_INVALID, "leading dimensions (" + std::to_string(ldb) + ", " +
                                           std::to_string(ldx) + ") below n = " +
                                           std::to_string(h->plan.n));
    return MDGPU_OK;
}

}  // namespace

extern "C" {

int mdgpu_analyze(int n, const int* Ap, const int* Ai, int ordering, int tree, int relax_zeros,
                  mdgpu_handle* out) {
    if (!out || n <= 0 || !Ap || !Ai) return fail(MDGPU_ERR_INVALID, "bad arguments");
    if (tree < 0 || tree > 2 || ordering < 0 || ordering > 1)
        return fail(MDGPU_ERR_INVALID, "bad ordering or tree kind");
    *out = nullptr;
    return guarded([&]() -> int {
        for (int j = 0; j < n; ++j) {
            if (Ap[j + 1] < Ap[j]) return fail(MDGPU_ERR_INVALID, "column pointers decrease");
            for (int p = Ap[j]; p < Ap[j + 1]; ++p)
                if (Ai[p] < j || Ai[p] >= n)
                    return fail(MDGPU_ERR_INVALID, "entry outside the lower triangle");
        }
        auto* h = new mdgpu_handle_s();
        int rc = analyze(n, Ap, Ai, nullptr, ordering == MDGPU_ORDER_AMD, (TreeKind)tree,
                         relax_zeros, h->sym);
        if (rc != 0) {
            delete h;
            return fail(MDGPU_ERR_NOT_TREE, "the elimination tree is a forest");
        }
        try {
            finish_plan(h);
            build_csr(h, n, Ap, Ai);
            upload_plan(h);
        } catch (...) {
            delete h;
            throw;
        }
        *out = h;
        return MDGPU_OK;
    });
}

int mdgpu_load_triplet(const char* path, int format, int* m, int* n, int* nnz, int* Ap, int* Ai,
                       double* Ax) {
    if (!path || !m || !n || !nnz || (format != 0 && format != 1))
        return fail(MDGPU_ERR_INVALID, "bad arguments");
    return guarded([&]() -> int {
        FILE* f = std::fopen(path, "r");
        if (!f) return fail(MDGPU_ERR_INVALID, std::string("cannot open ") + path);
        long long msize = -1, nsize = -1;
        if (format == 1) {  // Matrix Market: '%' lines, then "rows cols entries"
            char line[4096];
            bool have = false;
            while (std::fgets(line, sizeof line, f)) {
                if (line[0] == '%') continue;
                long long a, b, c;
                if (std::sscanf(line, "%lld %lld %lld", &a, &b, &c) != 3 || a < 0 || b < 0 ||
                    a > INT_MAX || b > INT_MAX) {
                    std::fclose(f);
                    return fail(MDGPU_ERR_INVALID, "bad Matrix Market size line");
                }
                msize = a;
                nsize = b;
                have = true;
                break;
            }
            if (!have) {
                std::fclose(f);
                return fail(MDGPU_ERR_INVALID, "no Matrix Market size line");
            }
        }
        // 1-based "i j x" triples, read until the first that does not parse
        std::vector<int> ti, tj;
        std::vector<double> tx;
        int i, j;
        double x;
        while (std::fscanf(f, "%d %d %lg", &i, &j, &x) == 3) {
            if (i < 1 || j < 1) {
                std::fclose(f);
                return fail(MDGPU_ERR_INVALID, "index below 1 in entry " + std::to_string(ti.size()));
            }
            if ((msize >= 0 && i > msize) || (nsize >= 0 && j > nsize)) {
                std::fclose(f);
                return fail(MDGPU_ERR_INVALID,
                            "entry " + std::to_string(ti.size()) + " outside the stated size");
            }
            ti.push_back(i - 1);
            tj.push_back(j - 1);
            tx.push_back(x);
        }
        std::fclose(f);
        int mm = 0, nn = 0;
        for (size_t k = 0; k < ti.size(); ++k) {
            mm = std::max(mm, ti[k] + 1);
            nn = std::max(nn, tj[k] + 1);
        }
        if (msize >= 0) {
            mm = (int)msize;
            nn = (int)nsize;
        }
        if (ti.size() > (size_t)INT_MAX) return fail(MDGPU_ERR_INVALID, "too many entries");
        *m = mm;
        *n = nn;
        *nnz = (int)ti.size();
        if (Ap) {  // compressed columns, entries of a column in file order
            std::vector<int> w(nn + 1, 0);
            for (int c : tj) w[c + 1]++;
            for (int c = 0; c < nn; ++c) w[c + 1] += w[c];
            std::copy(w.begin(), w.end(), Ap);
            for (size_t k = 0; k < ti.size(); ++k) {
                const int p = w[tj[k]]++;
                if (Ai) Ai[p] = ti[k];
                if (Ax) Ax[p] = tx[k];
            }
        }
        return MDGPU_OK;
    });
}

int mdgpu_estimate_batch(int nsys, const int* n, const int* const* Ap, const int* const* Ai,
                         int ordering, int tree, int relax_zeros, double* flops,
                         long long* lnz) {
    if (nsys <= 0 || !n || !Ap || !Ai || !flops) return fail(MDGPU_ERR_INVALID, "bad arguments");
    if (tree < 0 || tree > 2 || ordering < 0 || ordering > 1)
        return fail(MDGPU_ERR_INVALID, "bad ordering or tree kind");
    return guarded([&]() -> int {
        std::vector<Symbolic> parts;
        std::vector<int> row_off, val_off;
        return analyze_systems(nsys, n, Ap, Ai, ordering, tree, relax_zeros, false, parts,
                               row_off, val_off, flops, lnz);
    });
}

int mdgpu_analyze_batch(int nsys, const int* n, const int* const* Ap, const int* const* Ai,
                        int ordering, int tree, int relax_zeros, mdgpu_handle* out) {
    if (!out || nsys <= 0 || !n || !Ap || !Ai) return fail(MDGPU_ERR_INVALID, "bad arguments");
    if (tree < 0 || tree > 2 || ordering < 0 || ordering > 1)
        return fail(MDGPU_ERR_INVALID, "bad ordering or tree kind");
    *out = nullptr;
    return guarded([&]() -> int {
        std::vector<Symbolic> parts(nsys);
        std::vector<int> row_off, val_off;
        if (int rc = analyze_systems(nsys, n, Ap, Ai, ordering, tree, relax_zeros, true, parts,
                                     row_off, val_off, nullptr, nullptr))
            return rc;
        auto* h = new mdgpu_handle_s();
        try {
            combine_symbolic(parts, val_off, h->sym);
            h->sys_row_off = row_off;
            h->sys_val_off = val_off;
            finish_plan(h);
            build_csr_batch(h, nsys, n, Ap, Ai, row_off, val_off);
            upload_plan(h);
        } catch (...) {
            delete h;
            throw;
        }
        *out = h;
        return MDGPU_OK;
    });
}

namespace {

// The caller's lower triangle and assembly tree, checked before any of it is
// used as an index (O(n + nnz + nsuper)); empty when valid.  The tree must be
// the reference's ETree list (etree.h:6-19) in the form Factor consumes it:
// supernodes of consecutive columns that together cover 0..n-1 once each,
// listed in postorder (every supernode but the root, the last, is the child
// of exactly one later supernode), and column counts of a supernodal L
// (count[j + i] = count[j] - i inside a supernode, count[j] <= n - j).
std::string validate_tree(int n, const int* Ap, const int* Ai, int nsuper, const int* first_col,
                          const int* ncols, const int* child_ptr, const int* child,
                          const int* count) {
    if (Ap[0] != 0) return "Ap[0] must be 0";
    for (int j = 0; j < n; ++j) {
        if (Ap[j + 1] < Ap[j]) return "column pointers decrease at column " + std::to_string(j);
        for (int p = Ap[j]; p < Ap[j + 1]; ++p)
            if (Ai[p] < j || Ai[p] >= n)
                return "entry " + std::to_string(p) + " outside the lower triangle";
    }
    if (nsuper > n) return "more supernodes than columns";
    std::vector<char> covered(n, 0);
    for (int s = 0; s < nsuper; ++s) {
        if (first_col[s] < 0 || first_col[s] >= n)
            return "supernode " + std::to_string(s) + ": first column out of range";
        if (ncols[s] < 1 || ncols[s] > n - first_col[s])
            return "supernode " + std::to_string(s) + ": column count out of range";
        for (int j = first_col[s]; j < first_col[s] + ncols[s]; ++j)
            if (covered[j]++)
                return "column " + std::to_string(j) + " belongs to two supernodes";
    }
    for (int j = 0; j < n; ++j)
        if (!covered[j]) return "column " + std::to_string(j) + " belongs to no supernode";
    for (int j = 0; j < n; ++j)
        if (count[j] < 1 || count[j] > n - j)
            return "count[" + std::to_string(j) + "] out of range";
    for (int s = 0; s < nsuper; ++s)
        for (int i = 1; i < ncols[s]; ++i)
            if (count[first_col[s] + i] != count[first_col[s]] - i)
                return "supernode " + std::to_string(s) + ": column counts are not those of a "
                       "supernode";
    if (child_ptr[0] != 0) return "child_ptr[0] must be 0";
    for (int s = 0; s < nsuper; ++s)
        if (child_ptr[s + 1] < child_ptr[s])
            return "child_ptr decreases at supernode " + std::to_string(s);
    if (child_ptr[nsuper] != nsuper - 1)
        return "child lists must name every supernode but the root once";
    std::vector<char> seen(nsuper, 0);
    for (int s = 0; s < nsuper; ++s)
        for (int h = child_ptr[s]; h < child_ptr[s + 1]; ++h) {
            const int ch = child[h];
            if (ch < 0 || ch >= s)
                return "child " + std::to_string(ch) + " of supernode " + std::to_string(s) +
                       " is not an earlier supernode (postorder)";
            if (seen[ch]++) return "supernode " + std::to_string(ch) + " has two parents";
        }
    return std::string();
}

}  // namespace

int mdgpu_analyze_tree(int n, const int* Ap, const int* Ai, int nsuper, const int* first_col,
                       const int* ncols, const int* child_ptr, const int* child, const int* count,
                       mdgpu_handle* out) {
    if (!out || n <= 0 || !Ap || !Ai || nsuper <= 0 || !first_col || !ncols || !child_ptr ||
        !count)
        return fail(MDGPU_ERR_INVALID, "bad arguments");
    *out = nullptr;
    return guarded([&]() -> int {
        const std::string why =
            validate_tree(n, Ap, Ai, nsuper, first_col, ncols, child_ptr, child, count);
        if (!why.empty()) return fail(MDGPU_ERR_INVALID, "bad assembly tree: " + why);
        auto* h = new mdgpu_handle_s();
        Symbolic& S = h->sym;
        S.n = n;
        S.lower.nrows = S.lower.ncols = n;
        S.lower.colptr.assign(Ap, Ap + n + 1);
        S.lower.rowidx.assign(Ai, Ai + Ap[n]);
        S.lower_src.resize(Ap[n]);
        for (int p = 0; p < Ap[n]; ++p) S.lower_src[p] = p;
        S.count.assign(count, count + n);
        S.count0 = S.count;
        S.tree.first_col.assign(first_col, first_col + nsuper);
        S.tree.ncols.assign(ncols, ncols + nsuper);
        S.tree.child_ptr.assign(child_ptr, child_ptr + nsuper + 1);
        S.tree.child.assign(child, child + child_ptr[nsuper]);
        S.Lp.assign(n + 1, 0);
        for (int j = 0; j < n; ++j) S.Lp[j + 1] = S.Lp[j] + S.count[j];
        try {
            finish_plan(h);
            build_csr(h, n, Ap, Ai);
            // a caller's tree: every table the kernels index by is checked
            // on the host before any of it reaches the device
            upload_plan(h, true);
        } catch (...) {
            delete h;
            throw;
        }
        *out = h;
        return MDGPU_OK;
    });
}

void mdgpu_destroy(mdgpu_handle h) { delete h; }

int mdgpu_info(mdgpu_handle h, const char* key, long long* value) {
    if (!h || !key || !value) return fail(MDGPU_ERR_INVALID, "bad arguments");
    const Plan& P = h->plan;
    std::string k(key);
    if (k == "n") *value = P.n;
    else if (k == "nsuper") *value = P.nsuper;
    else if (k == "lnz") *value = P.lnz;
    else if (k == "nlevels") *value = P.nlevels;
    else if (k == "nnz") *value = P.nnz_user;
    else if (k == "max_front") *value = P.max_m;
    else if (k == "flops") *value = (long long)P.flops;
    else if (k == "lstore_bytes") *value = P.lstore * 8;
    else if (k == "ustore_bytes") *value = P.ustore * 8;
    else if (k == "zustore_bytes") *value = P.zustore * 8;
    else if (k == "fp64_diag_tiles") *value = h->fp64_diag_tiles;
    else if (k == "bf16_fallbacks") *value = h->bf16_fallbacks;
    else if (k == "precision_used") *value = h->factored;
    else if (k == "tuned") *value = h->tuned;
    else if (k == "tune_tiny_blocks") *value = h->D.tiny_blocks_cap;
    else if (k.rfind("tune_threads_b", 0) == 0 && k.size() == 15 && k[14] >= '0' &&
             k[14] < '0' + kSmallBuckets)
        *value = h->D.small_threads[k[14] - '0'];
    else if (k == "ustore_total_bytes") {
        long long t = 0;
        for (const FrontDesc& f : P.fronts)
            if (f.uoff >= 0) t += ((long long)f.ldu * (f.m - f.c) + 31) / 32 * 32;
        *value = t * 8;
    }
    else if (k == "rows_total") *value = (long long)P.rows.size();
    else if (k == "nchild") *value = (long long)P.child.size();
    else if (k == "large_fronts") *value = (long long)P.large_list.size();
    else if (k == "on_device") *value = h->on_device;
    else if (k == "solve_work_rows") *value = h->D.fv_total;
    else if (k == "nsys") *value = h->sys_row_off.empty() ? 1 : (long long)h->sys_row_off.size() - 1;
    else if (k == "small_fronts") *value = (long long)P.small_list.size();
    else if (k == "amap_rows") *value = (long long)h->ssched.amap_row.size();
    else if (k == "amap_entries") *value = (long long)h->ssched.amap_ent.size();
    else return fail(MDGPU_ERR_INVALID, "unknown key " + k);
    return MDGPU_OK;
}

int mdgpu_get_array(mdgpu_handle h, const char* name, void* dst) {
    if (!h || !name || !dst) return fail(MDGPU_ERR_INVALID, "bad arguments");
    const Plan& P = h->plan;
    const Symbolic& S = h->sym;
    std::string k(name);
    auto put = [&](const auto& v) {
        if (!v.empty()) std::memcpy(dst, v.data(), v.size() * sizeof(int));
        return MDGPU_OK;
    };
    if (k == "perm") {
        if (P.perm.empty()) {
            int* d = static_cast<int*>(dst);
            for (int i = 0; i < P.n; ++i) d[i] = i;
            return MDGPU_OK;
        }
        return put(P.perm);
    }
    if (k == "parent") return put(S.parent);
    if (k == "post") return put(S.post);
    if (k == "count0") return put(S.count0);
    if (k == "count") return put(S.count);
    if (k == "relax_perm") return put(S.relax_perm);
    if (k == "sn_first") return put(S.tree.first_col);
    if (k == "sn_ncols") return put(S.tree.ncols);
    if (k == "child_ptr") return put(S.tree.child_ptr);
    if (k == "child") return put(S.tree.child);
    if (k == "level") return put(h->level);
    if (k == "sys_row_off") return put(h->sys_row_off);
    if (k == "sys_val_off") return put(h->sys_val_off);
    if (k == "rows") return put(P.rows);
    if (k == "warp_list") return put(h->ssched.warp_list);
    if (k == "warp_cnt") return put(h->ssched.warp_cnt);
    if (k == "amap_off") return put(h->ssched.amap_off);
    if (k == "amap_row") return put(h->ssched.amap_row);
    if (k == "amap_ent") return put(h->ssched.amap_ent);
    if (k == "relmap") return put(P.relmap);
    if (k == "rows_ptr") {
        int* d = static_cast<int*>(dst);
        for (int s = 0; s < P.nsuper; ++s) d[s] = P.fronts[s].rows_off;
        d[P.nsuper] = (int)P.rows.size();
        return MDGPU_OK;
    }
    if (k == "Lp") {
        std::memcpy(dst, P.Lp.data(), P.Lp.size() * sizeof(int64_t));
        return MDGPU_OK;
    }
    return fail(MDGPU_ERR_INVALID, "unknown array " + k);
}

int mdgpu_factor_device(mdgpu_handle h, const double* dAx, int precision, void* stream) {
    if (!h || !dAx) return fail(MDGPU_ERR_INVALID, "bad arguments");
    if (!h->on_device) return fail(MDGPU_ERR_NO_DEVICE, "no CUDA device");
    return guarded([&] { return do_factor(h, dAx, precision, pick_stream(h, stream)); });
}

int mdgpu_factor(mdgpu_handle h, const double* Ax, int precision, void* stream) {
    if (!h || !Ax) return fail(MDGPU_ERR_INVALID, "bad arguments");
    if (!h->on_device) return fail(MDGPU_ERR_NO_DEVICE, "no CUDA device");
    return guarded([&] {
        cudaStream_t st = pick_stream(h, stream);
        ck(cudaSetDevice(h->device), "cudaSetDevice");
        ck(cudaMemcpyAsync(h->d_Ax, Ax, h->plan.nnz_user * sizeof(double),
                           cudaMemcpyHostToDevice, st),
           "upload values");
        return do_factor(h, h->d_Ax, precision, st);
    });
}

int mdgpu_check_plan(mdgpu_handle h) {
    if (!h) return fail(MDGPU_ERR_INVALID, "null handle");
    return guarded([&]() -> int {
        std::string why =
            check_plan(h->plan, h->sym, h->ssched, h->level, h->h_csr_rowptr, h->h_csr_col.data(),
                       h->h_csr_src.data(), (int64_t)h->h_csr_col.size());
        if (why.empty()) why = check_panel_schedule(h->plan, h->pschedh, h->level, kTile, kPanel);
        if (!why.empty()) return fail(MDGPU_ERR_INVALID, "plan check: " + why);
        return MDGPU_OK;
    });
}

int mdgpu_not_spd_column(mdgpu_handle h) { return h ? h->not_spd : -1; }

int mdgpu_solve_device(mdgpu_handle h, const double* dB, int ldb, double* dX, int ldx, int nrhs,
                       void* stream) {
    if (int rc = check_solve_args(h, dB, ldb, dX, ldx, nrhs)) return rc;
    if (!h->on_device) return fail(MDGPU_ERR_NO_DEVICE, "no CUDA device");
    if (h->factored < 0) return fail(MDGPU_ERR_STATE, "no valid factor");
    return guarded([&] {
        cudaStream_t st = pick_stream(h, stream);
        ck(cudaSetDevice(h->device), "cudaSetDevice");
        ensure_solve_storage(h, nrhs);
        solve_status_reset(h, st);
        do_solve(h, dB, ldb, dX, ldx, nrhs, st);
        return solve_status_check(h, st);
    });
}

int mdgpu_solve(mdgpu_handle h, const double* B, int ldb, double* X, int ldx, int nrhs,
                void* stream) {
    if (int rc = check_solve_args(h, B, ldb, X, ldx, nrhs)) return rc;
    if (!h->on_device) return fail(MDGPU_ERR_NO_DEVICE, "no CUDA device");
    if (h->factored < 0) return fail(MDGPU_ERR_STATE, "no valid factor");
    return guarded([&] {
        cudaStream_t st = pick_stream(h, stream);
        ck(cudaSetDevice(h->device), "cudaSetDevice");
        ensure_solve_storage(h, nrhs);
        const int n = h->plan.n;
        ck(cudaMemcpy2DAsync(h->d_B, n * sizeof(double), B, ldb * sizeof(double),
                             n * sizeof(double), nrhs, cudaMemcpyHostToDevice, st),
           "upload rhs");
        solve_status_reset(h, st);
        do_solve(h, h->d_B, n, h->d_X, n, nrhs, st);
        ck(cudaMemcpy2DAsync(X, ldx * sizeof(double), h->d_X, n * sizeof(double),
                             n * sizeof(double), nrhs, cudaMemcpyDeviceToHost, st),
           "download solution");
        return solve_status_check(h, st);
    });
}

int mdgpu_refine_device(mdgpu_handle h, const double* dB, int ldb, double* dX, int ldx, int nrhs,
                        double tol, int maxit, double* berr, int* iters, void* stream) {
    if (int rc = check_solve_args(h, dB, ldb, dX, ldx, nrhs)) return rc;
    if (maxit < 0) return fail(MDGPU_ERR_INVALID, "maxit must be >= 0");
    if (!h->on_device) return fail(MDGPU_ERR_NO_DEVICE, "no CUDA device");
    if (h->factored < 0) return fail(MDGPU_ERR_STATE, "no valid factor");
    return guarded([&] {
        cudaStream_t st = pick_stream(h, stream);
        ck(cudaSetDevice(h->device), "cudaSetDevice");
        solve_status_reset(h, st);
        int rc = do_refine(h, dB, ldb, dX, ldx, nrhs, tol, maxit, berr, iters, st);
        int rs = solve_status_check(h, st);
        return rs != MDGPU_OK ? rs : rc;
    });
}

int mdgpu_refine(mdgpu_handle h, const double* B, int ldb, double* X, int ldx, int nrhs,
                 double tol, int maxit, double* berr, int* iters, void* stream) {
    if (int rc = check_solve_args(h, B, ldb, X, ldx, nrhs)) return rc;
    if (maxit < 0) return fail(MDGPU_ERR_INVALID, "maxit must be >= 0");
    if (!h->on_device) return fail(MDGPU_ERR_NO_DEVICE, "no CUDA device");
    if (h->factored < 0) return fail(MDGPU_ERR_STATE, "no valid factor");
    return guarded([&] {
        cudaStream_t st = pick_stream(h, stream);
        ck(cudaSetDevice(h->device), "cudaSetDevice");
        ensure_solve_storage(h, nrhs);
        const int n = h->plan.n;
        ck(cudaMemcpy2DAsync(h->d_B, n * sizeof(double), B, ldb * sizeof(double),
                             n * sizeof(double), nrhs, cudaMemcpyHostToDevice, st),
           "upload rhs");
        solve_status_reset(h, st);
        int rc = do_refine(h, h->d_B, n, h->d_X, n, nrhs, tol, maxit, berr, iters, st);
        ck(cudaMemcpy2DAsync(X, ldx * sizeof(double), h->d_X, n * sizeof(double),
                             n * sizeof(double), nrhs, cudaMemcpyDeviceToHost, st),
           "download solution");
        int rs = solve_status_check(h, st);
        return rs != MDGPU_OK ? rs : rc;
    });
}

int mdgpu_gmres_ir_device(mdgpu_handle h, const double* dB, int ldb, double* dX, int ldx,
                          int nrhs, double tol, int maxit, int restart, double inner_tol,
                          double* berr, int* iters, int* inner, void* stream) {
    if (int rc = check_solve_args(h, dB, ldb, dX, ldx, nrhs)) return rc;
    if (int rc = check_gmres_args(maxit, restart, inner_tol)) return rc;
    if (!h->on_device) return fail(MDGPU_ERR_NO_DEVICE, "no CUDA device");
    if (h->factored < 0) return fail(MDGPU_ERR_STATE, "no valid factor");
    return guarded([&] {
        cudaStream_t st = pick_stream(h, stream);
        ck(cudaSetDevice(h->device), "cudaSetDevice");
        solve_status_reset(h, st);
        const GmresIrParams prm{tol, maxit, restart, inner_tol};
        int rc = do_gmres_ir(h, dB, ldb, dX, ldx, nrhs, prm, berr, iters, inner, st);
        int rs = solve_status_check(h, st);
        return rs != MDGPU_OK ? rs : rc;
    });
}

int mdgpu_gmres_ir(mdgpu_handle h, const double* B, int ldb, double* X, int ldx, int nrhs,
                   double tol, int maxit, int restart, double inner_tol, double* berr, int* iters,
                   int* inner, void* stream) {
    if (int rc = check_solve_args(h, B, ldb, X, ldx, nrhs)) return rc;
    if (int rc = check_gmres_args(maxit, restart, inner_tol)) return rc;
    if (!h->on_device) return fail(MDGPU_ERR_NO_DEVICE, "no CUDA device");
    if (h->factored < 0) return fail(MDGPU_ERR_STATE, "no valid factor");
    return guarded([&] {
        cudaStream_t st = pick_stream(h, stream);
        ck(cudaSetDevice(h->device), "cudaSetDevice");
        ensure_solve_storage(h, nrhs);
        const int n = h->plan.n;
        ck(cudaMemcpy2DAsync(h->d_B, n * sizeof(double), B, ldb * sizeof(double),
                             n * sizeof(double), nrhs, cudaMemcpyHostToDevice, st),
           "upload rhs");
        solve_status_reset(h, st);
        const GmresIrParams prm{tol, maxit, restart, inner_tol};
        int rc = do_gmres_ir(h, h->d_B, n, h->d_X, n, nrhs, prm, berr, iters, inner, st);
        ck(cudaMemcpy2DAsync(X, ldx * sizeof(double), h->d_X, n * sizeof(double),
                             n * sizeof(double), nrhs, cudaMemcpyDeviceToHost, st),
           "download solution");
        int rs = solve_status_check(h, st);
        return rs != MDGPU_OK ? rs : rc;
    });
}

int mdgpu_logdet(mdgpu_handle h, double* logdet, void* stream) {
    if (!h || !logdet) return fail(MDGPU_ERR_INVALID, "bad arguments");
    if (!h->on_device) return fail(MDGPU_ERR_NO_DEVICE, "no CUDA device");
    if (h->factored < 0) return fail(MDGPU_ERR_STATE, "no valid factor");
    return guarded([&]() -> int {
        cudaStream_t st = pick_stream(h, stream);
        ck(cudaSetDevice(h->device), "cudaSetDevice");
        if (!h->d_logdet) h->d_logdet = dalloc<double>(logdet_partials() + 1);
        double* out = h->d_logdet + logdet_partials();
        if (h->factored == MDGPU_FP64)
            launch_logdet<double>(h->D, h->dL64, h->d_logdet, out, st);
        else
            launch_logdet<float>(h->D, h->dL32, h->d_logdet, out, st);
        ck(cudaGetLastError(), "logdet launch");
        ck(cudaMemcpyAsync(logdet, out, sizeof(double), cudaMemcpyDeviceToHost, st), "logdet");
        ck(cudaStreamSynchronize(st), "logdet");
        return MDGPU_OK;
    });
}

int mdgpu_selinv(mdgpu_handle h, void* stream) {
    if (!h) return fail(MDGPU_ERR_INVALID, "bad arguments");
    if (!h->on_device) return fail(MDGPU_ERR_NO_DEVICE, "no CUDA device");
    if (h->factored != MDGPU_FP64) return fail(MDGPU_ERR_STATE, "the selected inverse needs an FP64 factor");
    return guarded([&]() -> int {
        cudaStream_t st = pick_stream(h, stream);
        ck(cudaSetDevice(h->device), "cudaSetDevice");
        if (!h->dZ64) h->dZ64 = dalloc<double>(h->plan.lstore);
        if (!h->dZu64) h->dZu64 = dalloc<double>(h->plan.zustore);
        if (!h->d_Y) h->d_Y = dalloc<double>(std::max<int64_t>(h->D.yscr_total, 1));
        NvtxRange nvtx("mdgpu_selinv");
        launch_selinv(h->D, h->dL64, h->dD64, h->dZ64, h->dZu64, h->d_Y, st);
        ck(cudaGetLastError(), "selected inverse launch");
        ck(cudaStreamSynchronize(st), "selected inverse");
        h->selinv_done = true;
        return MDGPU_OK;
    });
}

int mdgpu_grad_lower_device(mdgpu_handle h, const double* dx, double* dG, void* stream) {
    if (!h || !dG) return fail(MDGPU_ERR_INVALID, "bad arguments");
    if (!h->on_device) return fail(MDGPU_ERR_NO_DEVICE, "no CUDA device");
    if (!h->selinv_done) return fail(MDGPU_ERR_STATE, "no selected inverse of the current factor");
    return guarded([&]() -> int {
        cudaStream_t st = pick_stream(h, stream);
        ck(cudaSetDevice(h->device), "cudaSetDevice");
        ck(cudaMemsetAsync(dG, 0, (size_t)h->plan.nnz_user * sizeof(double), st), "zero G");
        launch_grad_lower(h->D, (int)h->plan.a_src.size(), h->d_perm, h->dZ64, dx, dG, st);
        ck(cudaGetLastError(), "gradient launch");
        return MDGPU_OK;
    });
}

int mdgpu_grad_lower(mdgpu_handle h, const double* x, double* G, void* stream) {
    if (!h || !G) return fail(MDGPU_ERR_INVALID, "bad arguments");
    if (!h->on_device) return fail(MDGPU_ERR_NO_DEVICE, "no CUDA device");
    if (!h->selinv_done) return fail(MDGPU_ERR_STATE, "no selected inverse of the current factor");
    return guarded([&]() -> int {
        cudaStream_t st = pick_stream(h, stream);
        ck(cudaSetDevice(h->device), "cudaSetDevice");
        const int64_t n = h->plan.n, nnz = h->plan.nnz_user;
        if (!h->d_gx) h->d_gx = dalloc<double>(n);
        if (!h->d_gG) h->d_gG = dalloc<double>(std::max<int64_t>(nnz, 1));
        if (x) ck(cudaMemcpyAsync(h->d_gx, x, n * sizeof(double), cudaMemcpyHostToDevice, st), "x");
        int rc = mdgpu_grad_lower_device(h, x ? h->d_gx : nullptr, h->d_gG, stream);
        if (rc != MDGPU_OK) return rc;
        ck(cudaMemcpyAsync(G, h->d_gG, nnz * sizeof(double), cudaMemcpyDeviceToHost, st), "G");
        ck(cudaStreamSynchronize(st), "gradient");
        return MDGPU_OK;
    });
}

int mdgpu_autotune(mdgpu_handle h, const double* Ax, int precision, double* ms_best) {
    if (!h || !Ax) return fail(MDGPU_ERR_INVALID, "bad arguments");
    if (!h->on_device) return fail(MDGPU_ERR_NO_DEVICE, "no CUDA device");
    if (precision != MDGPU_FP64 && precision != MDGPU_FP32 && precision != MDGPU_BF16 &&
        precision != MDGPU_TF32)
        return fail(MDGPU_ERR_INVALID, "unknown precision");
    return guarded([&]() -> int {
        NvtxRange nvtx("mdgpu_autotune");
        ck(cudaSetDevice(h->device), "cudaSetDevice");
        cudaStream_t st = h->stream;
        ck(cudaMemcpyAsync(h->d_Ax, Ax, h->plan.nnz_user * sizeof(double), cudaMemcpyHostToDevice,
                           st),
           "values");
        cudaEvent_t e0, e1;
        ck(cudaEventCreate(&e0), "event");
        ck(cudaEventCreate(&e1), "event");
        DevPlan& D = h->D;
        // the factor's device time with the current shapes: the graph is
        // captured again, one untimed factor, then the median of three
        auto measure = [&]() -> double {
            for (auto& g : h->fgraph)
                if (g) {
                    cudaGraphExecDestroy(g);
                    g = nullptr;
                }
            int rc = do_factor_once(h, h->d_Ax, precision, st);
            if (rc != MDGPU_OK) throw std::runtime_error(std::string("autotune factor: ") +
                                                         g_last_error);
            float t[3];
            for (float& x : t) {
                ck(cudaEventRecord(e0, st), "event");
                do_factor_once(h, h->d_Ax, precision, st);
                ck(cudaEventRecord(e1, st), "event");
                ck(cudaEventSynchronize(e1), "event");
                ck(cudaEventElapsedTime(&x, e0, e1), "event");
            }
            std::sort(t, t + 3);
            return t[1];
        };
        // coordinate descent, one pass: each shape over its candidates with
        // the others held, the fastest kept
        double best = measure();
        {
            const int cand[] = {148 * 4, 148 * 8, 148 * 16};
            int keep = D.tiny_blocks_cap;
            for (int c : cand) {
                if (c == keep) continue;
                D.tiny_blocks_cap = c;
                const double t = measure();
                if (t < best) {
                    best = t;
                    keep = c;
                }
            }
            D.tiny_blocks_cap = keep;
        }
        for (int b = Plan::kTinyBuckets; b < kSmallBuckets; ++b) {
            const int cand[] = {128, 256, 512};
            int keep = D.small_threads[b];
            for (int c : cand) {
                if (c == keep) continue;
                D.small_threads[b] = c;
                const double t = measure();
                if (t < best) {
                    best = t;
                    keep = c;
                }
            }
            D.small_threads[b] = keep;
        }
        for (auto& g : h->fgraph)
            if (g) {
                cudaGraphExecDestroy(g);
                g = nullptr;
            }
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        h->tuned = true;
        if (ms_best) *ms_best = best;
        return MDGPU_OK;
    });
}

int mdgpu_adjoint_device(mdgpu_handle h, const double* dLbar, double* dAbar, void* stream) {
    if (!h || !dLbar || !dAbar) return fail(MDGPU_ERR_INVALID, "bad arguments");
    if (!h->on_device) return fail(MDGPU_ERR_NO_DEVICE, "no CUDA device");
    if (h->factored != MDGPU_FP64) return fail(MDGPU_ERR_STATE, "the adjoint needs an FP64 factor");
    return guarded([&]() -> int {
        NvtxRange nvtx("mdgpu_adjoint");
        cudaStream_t st = pick_stream(h, stream);
        ck(cudaSetDevice(h->device), "cudaSetDevice");
        const Plan& P = h->plan;
        if (!h->d_Fb) h->d_Fb = dalloc<double>(P.lstore);
        if (!h->d_Fu) h->d_Fu = dalloc<double>(P.zustore);
        if (!h->d_W) h->d_W = dalloc<double>(h->D.adj.wtotal);
        launch_adjoint(h->D, (int)P.a_src.size(), h->dL64, dLbar, h->d_Fb, h->d_Fu, h->d_W,
                       dAbar, st);
        ck(cudaGetLastError(), "adjoint launch");
        return MDGPU_OK;
    });
}

int mdgpu_adjoint(mdgpu_handle h, const double* Lbar, double* Abar, void* stream) {
    if (!h || !Lbar || !Abar) return fail(MDGPU_ERR_INVALID, "bad arguments");
    if (!h->on_device) return fail(MDGPU_ERR_NO_DEVICE, "no CUDA device");
    if (h->factored != MDGPU_FP64) return fail(MDGPU_ERR_STATE, "the adjoint needs an FP64 factor");
    return guarded([&]() -> int {
        cudaStream_t st = pick_stream(h, stream);
        ck(cudaSetDevice(h->device), "cudaSetDevice");
        const int64_t lnz = h->plan.lnz, nnz = h->plan.nnz_user;
        if (!h->d_Lbar) h->d_Lbar = dalloc<double>(std::max<int64_t>(lnz, 1));
        if (!h->d_Abar) h->d_Abar = dalloc<double>(std::max<int64_t>(nnz, 1));
        ck(cudaMemcpyAsync(h->d_Lbar, Lbar, lnz * sizeof(double), cudaMemcpyHostToDevice, st),
           "Lbar");
        int rc = mdgpu_adjoint_device(h, h->d_Lbar, h->d_Abar, stream);
        if (rc != MDGPU_OK) return rc;
        ck(cudaMemcpyAsync(Abar, h->d_Abar, nnz * sizeof(double), cudaMemcpyDeviceToHost, st),
           "Abar");
        ck(cudaStreamSynchronize(st), "adjoint");
        return MDGPU_OK;
    });
}

int mdgpu_get_L(mdgpu_handle h, long long* Lp, int* Li, double* Lx) {
    if (!h) return fail(MDGPU_ERR_INVALID, "bad arguments");
    const Plan& P = h->plan;
    if (Lp) std::memcpy(Lp, P.Lp.data(), P.Lp.size() * sizeof(int64_t));
    if (Li) {
        for (int s = 0; s < P.nsuper; ++s) {
            const FrontDesc& f = P.fronts[s];
            const int* r = P.rows.data() + f.rows_off;
            for (int j = 0; j < f.c; ++j) {
                int64_t p0 = P.Lp[f.first_col + j];
                for (int i = j; i < f.m; ++i) Li[p0 + i - j] = r[i];
            }
        }
    }
    if (!Lx) return MDGPU_OK;
    if (!h->on_device) return fail(MDGPU_ERR_NO_DEVICE, "no CUDA device");
    if (h->factored < 0) return fail(MDGPU_ERR_STATE, "no valid factor");
    return guarded([&] {
        ck(cudaSetDevice(h->device), "cudaSetDevice");
        ck(cudaStreamSynchronize(h->stream), "sync");
        std::vector<double> L64;
        std::vector<float> L32;
        if (h->factored == MDGPU_FP64) {
            L64.resize(P.lstore);
            ck(cudaMemcpy(L64.data(), h->dL64, P.lstore * sizeof(double), cudaMemcpyDeviceToHost),
               "download L");
        } else {
            L32.resize(P.lstore);
            ck(cudaMemcpy(L32.data(), h->dL32, P.lstore * sizeof(float), cudaMemcpyDeviceToHost),
               "download L");
        }
        for (int s = 0; s < P.nsuper; ++s) {
            const FrontDesc& f = P.fronts[s];
            for (int j = 0; j < f.c; ++j) {
                int64_t p0 = P.Lp[f.first_col + j];
                int64_t base = f.loff + (int64_t)j * f.ldl;
                for (int i = j; i < f.m; ++i)
                    Lx[p0 + i - j] = h->factored == MDGPU_FP64 ? L64[base + i] : (double)L32[base + i];
            }
        }
        return MDGPU_OK;
    });
}

int mdgpu_solve_device_noalloc(mdgpu_handle h, const double* dB, int ldb, double* dX, int ldx,
                               int nrhs, void* stream) {
    if (int rc = check_solve_args(h, dB, ldb, dX, ldx, nrhs)) return rc;
    if (!h->on_device) return fail(MDGPU_ERR_NO_DEVICE, "no CUDA device");
    if (h->factored < 0) return fail(MDGPU_ERR_STATE, "no valid factor");
    return guarded([&]() -> int {
        cudaStream_t st = pick_stream(h, stream);
        ck(cudaSetDevice(h->device), "cudaSetDevice");
        std::string msg;
        double* scratch = noalloc_scratch(msg);
        if (!scratch) return fail(MDGPU_ERR_CUDA, msg);
        const int n = h->plan.n;
        const int chunk = std::min(nrhs, 64);
        // the work vectors start on 16 bytes (the solve copies published
        // vectors from them in 16-byte pieces): the permuted right-hand sides
        // take an even number of doubles
        const long long xrows = ((long long)n * chunk + 1) & ~1ll;
        const long long need = xrows + h->D.fv_total * chunk;
        if (need > noalloc_scratch_capacity())
            return fail(MDGPU_ERR_INVALID,
                        "no-allocation solve needs " + std::to_string(need) +
                            " scratch doubles ((n + solve_work_rows) x min(nrhs, 64), n x "
                            "min(nrhs, 64) rounded up to even), limit " +
                            std::to_string(noalloc_scratch_capacity()));
        double* xp = scratch;
        double* fv = scratch + xrows;
        solve_status_reset(h, st);
        for (int q0 = 0; q0 < nrhs; q0 += 64) {
            const int nq = std::min(64, nrhs - q0);
            permute_gather(h->d_perm, dB + (int64_t)q0 * ldb, xp, n, nq, ldb, st);
            if (h->factored == MDGPU_FP64)
                solve_levels<double, double>(h->D, h->dL64, h->dD64, xp, fv, nq, st);
            else
                solve_levels<float, double>(h->D, h->dL32, h->dD32, xp, fv, nq, st);
            permute_scatter(h->d_perm, xp, dX + (int64_t)q0 * ldx, n, nq, ldx, st);
        }
        ck(cudaGetLastError(), "solve launch");
        return solve_status_check(h, st);
    });
}

int mdgpu_profile(mdgpu_handle h, int enable) {
    if (!h) return fail(MDGPU_ERR_INVALID, "bad arguments");
    if (!h->on_device) return fail(MDGPU_ERR_NO_DEVICE, "no CUDA device");
    return guarded([&] {
        Profiler& P = h->prof;
        if (!P.recs.empty()) {
            ck(cudaDeviceSynchronize(), "profile sync");
            h->prof_ms.assign(KC_COUNT, 0.0);
            h->prof_flops.assign(KC_COUNT, 0.0);
            h->prof_bytes.assign(KC_COUNT, 0.0);
            h->prof_n.assign(KC_COUNT, 0);
            for (auto& r : P.recs) {
                float ms = 0;
                ck(cudaEventElapsedTime(&ms, r.a, r.b), "event time");
                h->prof_ms[r.cls] += ms;
                h->prof_flops[r.cls] += r.flops;
                h->prof_bytes[r.cls] += r.bytes;
                h->prof_n[r.cls] += 1;
            }
        }
        P.recs.clear();
        P.used = 0;
        P.on = enable != 0;
        return MDGPU_OK;
    });
}

int mdgpu_profile_read(mdgpu_handle h, int cls, double* ms, long long* launches, double* flops,
                       double* bytes) {
    if (!h || cls < 0 || cls >= KC_COUNT) return fail(MDGPU_ERR_INVALID, "bad arguments");
    bool have = (int)h->prof_ms.size() == KC_COUNT;
    if (ms) *ms = have ? h->prof_ms[cls] : 0.0;
    if (launches) *launches = have ? h->prof_n[cls] : 0;
    if (flops) *flops = have ? h->prof_flops[cls] : 0.0;
    if (bytes) *bytes = have ? h->prof_bytes[cls] : 0.0;
    return MDGPU_OK;
}

const char* mdgpu_status_string(int status) {
    switch (status) {
        case MDGPU_OK: return "ok";
        case MDGPU_ERR_INVALID: return "invalid argument";
        case MDGPU_ERR_NOT_SPD: return "matrix is not positive definite";
        case MDGPU_ERR_OOM: return "out of memory";
        case MDGPU_ERR_CUDA: return "CUDA error";
        case MDGPU_ERR_NOT_TREE: return "elimination tree is a forest";
        case MDGPU_ERR_STATE: return "invalid call order";
        case MDGPU_ERR_NO_DEVICE: return "no CUDA device";
        default: return "unknown status";
    }
}

const char* mdgpu_last_error(void) { return g_last_error.c_str(); }

}  // extern "C"
