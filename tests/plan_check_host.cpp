// Host check of the plan self-check (mdgpu_b200/csrc/plan_check.cpp): the
// library's own analysis and plan builders on a 3D 7-point grid, the check
// on the intact plan, then on copies with one invariant broken each.  Test
// infrastructure: compiled and run by tests/test_plan_check.py.
//
// Usage: plan_check_host <side>.  Prints "intact: <message or ok>", then one
// line "<corruption>: <message>" per corruption.
#include <cstdio>
#include <cstdlib>
#include <string>
#include <utility>
#include <vector>

#include "plan.hpp"
#include "plan_check.hpp"
#include "symbolic.hpp"

using namespace mdgpu;

namespace {

// lower triangle (CSC) of the 7-point stencil on a side^3 grid
void grid(int side, int& n, std::vector<int>& Ap, std::vector<int>& Ai) {
    n = side * side * side;
    Ap.assign(1, 0);
    Ai.clear();
    for (int z = 0; z < side; ++z)
        for (int y = 0; y < side; ++y)
            for (int x = 0; x < side; ++x) {
                const int k = (z * side + y) * side + x;
                Ai.push_back(k);
                if (x + 1 < side) Ai.push_back(k + 1);
                if (y + 1 < side) Ai.push_back(k + side);
                if (z + 1 < side) Ai.push_back(k + side * side);
                Ap.push_back((int)Ai.size());
            }
}

struct Case {
    Plan P;
    SolveScheduleHost Q;
    PanelSchedule PS;
    std::vector<int> level, rowptr, col, src;
};

std::string run(const Case& c, const Symbolic& S) {
    std::string m = check_plan(c.P, S, c.Q, c.level, c.rowptr, c.col.data(), c.src.data(),
                               (int64_t)c.col.size());
    if (m.empty()) m = check_panel_schedule(c.P, c.PS, c.level, 64, 256);
    return m.empty() ? "ok" : m;
}

}  // namespace

int main(int argc, char** argv) {
    if (argc != 2) return 2;
    int n;
    std::vector<int> Ap, Ai;
    grid(std::atoi(argv[1]), n, Ap, Ai);
    Symbolic S;
    if (analyze(n, Ap.data(), Ai.data(), nullptr, true, TreeKind::Super, 0, S) != 0) return 3;
    Case base;
    build_plan(S, Ap[n], Plan::kSmallMaxRows, base.P);
    build_solve_schedule(base.P, 64, base.Q);
    build_large_tables(base.P, 64, 16);
    build_panel_schedule(base.P, 64, 256, 16, base.PS);
    base.level = front_levels(base.P);
    // the residual's CSR: only its ranges are checked, so rows in order
    base.rowptr.assign(n + 1, 0);
    for (int j = 0; j < n; ++j) {
        for (int p = Ap[j]; p < Ap[j + 1]; ++p) {
            base.col.push_back(Ai[p]);
            base.src.push_back(p);
        }
        base.rowptr[j + 1] = (int)base.col.size();
    }
    std::printf("intact: %s\n", run(base, S).c_str());
    const Plan& P = base.P;
    // a front with two update rows, a non-root front with an update row, a
    // level with two small fronts, a large front with two pivot tiles
    int s_rows = -1, s_rel = -1, s_piv = -1, l_warp = -1;
    for (int s = 0; s < P.nsuper; ++s) {
        const FrontDesc& f = P.fronts[s];
        if (s_rows < 0 && f.m >= f.c + 2) s_rows = s;
        if (s_rel < 0 && f.parent >= 0 && f.m > f.c) s_rel = s;
    }
    for (int s : P.large_list)
        if (s_piv < 0 && P.fronts[s].c > 64) s_piv = s;
    for (int l = 0; l < P.nlevels && l_warp < 0; ++l)
        if (P.small_ptr[(l + 1) * kSmallBuckets] - P.small_ptr[l * kSmallBuckets] >= 2) l_warp = l;
    if (s_rows < 0 || s_rel < 0 || s_piv < 0 || l_warp < 0) return 4;
    std::vector<std::pair<std::string, Case>> bad;
    {
        Case c = base;
        const FrontDesc& f = c.P.fronts[s_rows];
        std::swap(c.P.rows[f.rows_off + f.c], c.P.rows[f.rows_off + f.c + 1]);
        bad.push_back({"rows", c});
    }
    {
        Case c = base;
        const FrontDesc& f = c.P.fronts[s_rel];
        c.P.relmap[f.rows_off + f.c] += 1;
        bad.push_back({"relmap", c});
    }
    {
        Case c = base;
        c.P.a_pos[0] += 1;
        bad.push_back({"a_pos", c});
    }
    {
        Case c = base;
        c.P.fronts[s_rows].loff += 1;
        bad.push_back({"loff", c});
    }
    {
        Case c = base;
        const int b = c.P.small_ptr[l_warp * kSmallBuckets];
        c.Q.warp_list[b + 1] = c.Q.warp_list[b];
        bad.push_back({"warp_list", c});
    }
    {
        Case c = base;
        const int l = c.level[s_piv];
        int q0 = -1, q1 = -1;  // its pivot tiles 0 and 1, swapped
        for (int q = c.Q.fwd_task_beg[l]; q < c.Q.fwd_task_beg[l + 1]; ++q)
            if (c.Q.tasks[2 * q] == s_piv) {
                if ((c.Q.tasks[2 * q + 1] & 0xffff) == 0) q0 = q;
                if ((c.Q.tasks[2 * q + 1] & 0xffff) == 1) q1 = q;
            }
        if (q0 < 0 || q1 < 0) return 5;
        std::swap(c.Q.tasks[2 * q0 + 1], c.Q.tasks[2 * q1 + 1]);
        bad.push_back({"tasks", c});
    }
    {
        // the forward item list: a large front's first item swapped with
        // the last item of one of its children
        Case c = base;
        const FrontDesc& f = c.P.fronts[s_piv];
        if (f.child_end <= f.child_beg) return 7;
        const int ch = c.P.child[f.child_beg];
        const std::vector<int>& it = c.Q.fwd_items;
        int64_t kc = -1, kp = -1;
        for (int64_t k = 0; k < (int64_t)it.size() / 4; ++k) {
            const int* e = it.data() + 4 * k;
            if (e[0] == SolveScheduleHost::kItemWarps) {
                const int nf = (e[2] & 0xff) + ((e[2] >> 8) & 0xff) + (e[2] >> 16);
                for (int q = 0; q < nf; ++q)
                    if (c.Q.fwd_wlist[e[1] + q] == ch) kc = k;
            } else {
                if (e[1] == ch) kc = k;
                if (e[1] == s_piv && kp < 0) kp = k;
            }
        }
        if (kc < 0 || kp < 0 || kc >= kp) return 8;
        for (int q = 0; q < 4; ++q) std::swap(c.Q.fwd_items[4 * kc + q], c.Q.fwd_items[4 * kp + q]);
        bad.push_back({"items", c});
    }
    {
        Case c = base;
        const int off = c.Q.amap_off[s_piv];
        const int e = c.Q.amap_row[off + c.P.fronts[s_piv].m - 1];  // an entry of a late row
        c.Q.amap_ent[e < (int)c.Q.amap_ent.size() ? e : 0] += 1;
        bad.push_back({"amap", c});
    }
    {
        Case c = base;
        c.col[3] = n;
        bad.push_back({"csr", c});
    }
    {
        Case c = base;
        const int s = P.fronts[s_rel].parent;
        c.level[s_rel] = c.level[s];
        bad.push_back({"level", c});
    }
    {
        // a front's second diagonal task moved behind a task that waits on it
        Case c = base;
        int64_t td = -1, tl = -1;
        for (const PanelOp& o : c.PS.ops) {
            if (o.kind != OP_PANEL || o.arg != 0) continue;
            for (int64_t t = o.toff; t < o.toff + o.ntasks; ++t)
                if (c.PS.tasks[2 * t] == s_piv && c.PS.tasks[2 * t + 1] == 1) td = t;
            if (td >= 0) {
                tl = o.toff + o.ntasks - 1;
                break;
            }
        }
        if (td < 0) return 6;
        std::swap(c.PS.tasks[2 * td], c.PS.tasks[2 * tl]);
        std::swap(c.PS.tasks[2 * td + 1], c.PS.tasks[2 * tl + 1]);
        bad.push_back({"panel", c});
    }
    {
        // two update matrices live at the same level given the same storage
        Case c = base;
        int a = -1, b = -1;
        for (int s = 0; s < P.nsuper && b < 0; ++s)
            if (P.fronts[s].uoff >= 0 && c.level[s] == 0) {
                if (a < 0)
                    a = s;
                else
                    b = s;
            }
        if (b < 0) return 7;
        c.P.fronts[b].uoff = c.P.fronts[a].uoff;
        bad.push_back({"uoff", c});
    }
    for (auto& b : bad) std::printf("%s: %s\n", b.first.c_str(), run(b.second, S).c_str());
    return 0;
}
