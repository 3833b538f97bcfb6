// Host self-check of a plan before (or after) its upload: every invariant the
// device kernels rely on when they index the plan's tables, checked from
// its definition rather than from the builder's steps.  A violation is
// reported with the front it concerns; nothing here touches the device.
#include "plan_check.hpp"

#include <algorithm>
#include <map>
#include <string>
#include <vector>

namespace mdgpu {

namespace {

struct Fail {
    std::string msg;
};

[[noreturn]] void bad(const std::string& what, int s = -1) {
    throw Fail{s >= 0 ? "front " + std::to_string(s) + ": " + what : what};
}

int round8(int x) { return (x + 7) & ~7; }

}  // namespace

std::string check_plan(const Plan& P, const Symbolic& S, const SolveScheduleHost& Q,
                       const std::vector<int>& level, const std::vector<int>& csr_rowptr,
                       const int* csr_col, const int* csr_src, int64_t csr_nnz) {
    try {
        const int n = P.n, ns = P.nsuper, T = Q.T;
        if ((int)P.fronts.size() != ns || (int)level.size() != ns) bad("table sizes");
        // fronts: sizes, storage ranges, row sets, children, columns owned
        std::vector<int> owner(n, -1);
        int64_t rows_next = 0, lprev = -1;
        for (int s = 0; s < ns; ++s) {
            const FrontDesc& f = P.fronts[s];
            const int u = f.m - f.c;
            if (f.c < 1 || f.m < f.c) bad("rows / pivot columns out of range", s);
            if (f.ldl != round8(f.m) || f.ldu != round8(u)) bad("leading dimensions", s);
            if (f.loff % 32 || f.loff <= lprev || f.loff + (int64_t)f.ldl * f.c > P.lstore)
                bad("L panel offset", s);
            lprev = f.loff + (int64_t)f.ldl * f.c - 1;
            if ((f.parent >= 0 && u > 0) != (f.uoff >= 0)) bad("update matrix presence", s);
            if (f.uoff >= 0 && (f.uoff % 32 || f.uoff + (int64_t)f.ldu * u > P.ustore))
                bad("update matrix offset", s);
            if (f.uoff >= 0 && ((int)P.zuoff.size() != ns || P.zuoff[s] < 0 || P.zuoff[s] % 32 ||
                                P.zuoff[s] + (int64_t)f.ldu * u > P.zustore))
                bad("selected-inverse update offset", s);
            if (f.rows_off != rows_next) bad("row set offset", s);
            rows_next += f.m;
            if (rows_next > (int64_t)P.rows.size()) bad("row set past the row array", s);
            if (f.first_col < 0 || f.first_col + f.c > n) bad("pivot columns past n", s);
            for (int j = f.first_col; j < f.first_col + f.c; ++j) {
                if (owner[j] >= 0) bad("column " + std::to_string(j) + " in two fronts", s);
                owner[j] = s;
            }
            const int* r = P.rows.data() + f.rows_off;
            for (int i = 0; i < f.c; ++i)
                if (r[i] != f.first_col + i) bad("pivot rows", s);
            for (int i = 1; i < f.m; ++i)
                if (r[i] <= r[i - 1]) bad("rows not strictly increasing", s);
            if (r[f.m - 1] >= n) bad("row past n", s);
            if (f.child_beg < 0 || f.child_end < f.child_beg || f.child_end > (int)P.child.size())
                bad("child range", s);
            for (int h = f.child_beg; h < f.child_end; ++h) {
                const int ch = P.child[h];
                if (ch < 0 || ch >= s || P.fronts[ch].parent != s) bad("child not before it", s);
                if (level[ch] >= level[s]) bad("child level not below", s);
            }
            if (f.parent >= ns || (f.parent >= 0 && f.parent <= s)) bad("parent after it", s);
        }
        if (rows_next != (int64_t)P.rows.size() || P.relmap.size() != P.rows.size())
            bad("row array size");
        for (int j = 0; j < n; ++j)
            if (owner[j] < 0) bad("column " + std::to_string(j) + " in no front");
        // relative maps: update row i of s sits at relmap in its parent
        for (int s = 0; s < ns; ++s) {
            const FrontDesc& f = P.fronts[s];
            const int* r = P.rows.data() + f.rows_off;
            const int* rm = P.relmap.data() + f.rows_off;
            for (int i = 0; i < (f.parent < 0 ? f.m : f.c); ++i)
                if (rm[i] != -1) bad("relative map of a row with no parent row", s);
            if (f.parent < 0) continue;
            const FrontDesc& p = P.fronts[f.parent];
            const int* rp = P.rows.data() + p.rows_off;
            for (int i = f.c; i < f.m; ++i) {
                const int q = rm[i];
                if (q < 0 || q >= p.m || rp[q] != r[i]) bad("relative map entry", s);
                if (i > f.c && q <= rm[i - 1]) bad("relative map not increasing", s);
            }
        }
        // A entries: each in its column's front, at its row and column
        const SparseCol& A = S.lower;
        if ((int64_t)P.a_src.size() != A.nnz() || (int64_t)P.a_pos.size() != A.nnz())
            bad("A map sizes");
        for (int j = 0; j < n; ++j) {
            const FrontDesc& f = P.fronts[owner[j]];
            const int* r = P.rows.data() + f.rows_off;
            for (int p = A.colptr[j]; p < A.colptr[j + 1]; ++p) {
                const int pos = P.a_pos[p] & 0xffff, jj = P.a_pos[p] >> 16;
                if (jj != j - f.first_col || pos >= f.m || r[pos] != A.rowidx[p])
                    bad("A entry position", owner[j]);
                if (P.a_src[p] != S.lower_src[p] && P.a_src[p] != -1)
                    bad("A entry source", owner[j]);
                if (P.a_src[p] >= P.nnz_user) bad("A entry source past the values", owner[j]);
            }
            if (j == f.first_col &&
                (f.a_beg != A.colptr[j] || f.a_end != A.colptr[j + f.c]))
                bad("A entry range", owner[j]);
        }
        // level lists: every front once, small ones by size bucket
        std::vector<int> seen(ns, 0);
        std::vector<char> is_large(ns, 0);
        for (int l = 0; l < P.nlevels; ++l) {
            for (int q = P.small_ptr[l * kSmallBuckets]; q < P.small_ptr[(l + 1) * kSmallBuckets];
                 ++q) {
                const int s = P.small_list[q];
                if (s < 0 || s >= ns) bad("small list entry out of range");
                if (level[s] != l || P.fronts[s].m > Plan::kSmallMaxRows) bad("small list", s);
                seen[s]++;
            }
            for (int q = P.large_ptr[l]; q < P.large_ptr[l + 1]; ++q) {
                const int s = P.large_list[q];
                if (s < 0 || s >= ns) bad("large list entry out of range");
                if (level[s] != l) bad("large list", s);
                seen[s]++;
                is_large[s] = 1;
            }
        }
        for (int s = 0; s < ns; ++s)
            if (seen[s] != 1) bad("not exactly once in the level lists", s);
        // warp lists: the level's small fronts, rows descending, with counts
        if (Q.warp_list.size() != P.small_list.size()) bad("warp list size");
        for (int l = 0; l < P.nlevels; ++l) {
            const int b = P.small_ptr[l * kSmallBuckets], e = P.small_ptr[(l + 1) * kSmallBuckets];
            std::vector<int> a(P.small_list.begin() + b, P.small_list.begin() + e),
                w(Q.warp_list.begin() + b, Q.warp_list.begin() + e);
            int cnt[3] = {0, 0, 0};
            for (int q = 0; q < e - b; ++q) {
                if (w[q] < 0 || w[q] >= ns) bad("warp list entry out of range");
                const int m = P.fronts[w[q]].m;
                if (q && m > P.fronts[w[q - 1]].m) bad("warp list not by rows descending");
                cnt[m > 16 ? 0 : (m > 8 ? 1 : 2)]++;
            }
            std::sort(a.begin(), a.end());
            std::sort(w.begin(), w.end());
            if (a != w) bad("warp list of level " + std::to_string(l));
            for (int k = 0; k < 3; ++k)
                if (Q.warp_cnt[3 * l + k] != cnt[k]) bad("warp counts of level " + std::to_string(l));
        }
        // front vectors and the forward assembly map of the large fronts
        int64_t fv = 0;
        for (int s = 0; s < ns; ++s) {
            if (Q.fv_off[s] != fv) bad("front vector offset", s);
            fv += P.fronts[s].m;
        }
        if (Q.fv_rows != fv) bad("front vector rows");
        for (int s = 0; s < ns; ++s) {
            const FrontDesc& f = P.fronts[s];
            if (!is_large[s]) {
                if (Q.amap_off[s] != -1) bad("assembly map of a small front", s);
                continue;
            }
            const int off = Q.amap_off[s];
            if (off < 0 || off + f.m >= (int64_t)Q.amap_row.size()) bad("assembly map offset", s);
            int64_t want = 0;
            for (int h = f.child_beg; h < f.child_end; ++h)
                want += P.fronts[P.child[h]].m - P.fronts[P.child[h]].c;
            if (Q.amap_row[off + f.m] - Q.amap_row[off] != want) bad("assembly map size", s);
            for (int r = 0; r < f.m; ++r) {
                const int e0 = Q.amap_row[off + r], e1 = Q.amap_row[off + r + 1];
                if (e1 < e0 || e0 < 0 || e1 > (int64_t)Q.amap_ent.size()) bad("assembly map row", s);
                for (int e = e0; e < e1; ++e) {
                    const int64_t row = Q.amap_ent[e];
                    const int ch = (int)(std::upper_bound(Q.fv_off.begin(), Q.fv_off.end(), row) -
                                         Q.fv_off.begin()) - 1;
                    if (ch < 0 || P.fronts[ch].parent != s) bad("assembly map child", s);
                    const FrontDesc& g = P.fronts[ch];
                    const int64_t i = row - Q.fv_off[ch];
                    if (i < g.c || i >= g.m || P.relmap[g.rows_off + i] != r)
                        bad("assembly map entry", s);
                }
            }
        }
        // update matrices sharing storage have disjoint lifetimes: at every
        // level, the ranges of the matrices live there do not overlap (the
        // factor's [lev(s), lev(parent)]; the selected inverse's [lowest
        // child level, lev(s)])
        {
            int nlev = 0;
            for (int s = 0; s < ns; ++s) nlev = std::max(nlev, level[s] + 1);
            for (int pass = 0; pass < 2; ++pass) {
                std::vector<std::vector<int>> live(nlev);
                for (int s = 0; s < ns; ++s) {
                    const FrontDesc& f = P.fronts[s];
                    if (f.uoff < 0) continue;
                    int b = level[s], e = level[s];
                    if (pass == 0) {
                        e = level[f.parent];
                    } else {
                        for (int h = f.child_beg; h < f.child_end; ++h)
                            b = std::min(b, level[P.child[h]]);
                    }
                    for (int l = b; l <= e; ++l) live[l].push_back(s);
                }
                for (int l = 0; l < nlev; ++l) {
                    std::vector<std::pair<int64_t, int64_t>> rg;
                    for (int s : live[l]) {
                        const FrontDesc& f = P.fronts[s];
                        const int64_t o = pass == 0 ? f.uoff : P.zuoff[s];
                        rg.push_back({o, o + (int64_t)f.ldu * (f.m - f.c)});
                    }
                    std::sort(rg.begin(), rg.end());
                    for (size_t q = 1; q < rg.size(); ++q)
                        if (rg[q].first < rg[q - 1].second)
                            bad(pass == 0 ? "update matrices live together share storage"
                                          : "selected-inverse update parts live together share "
                                            "storage");
                }
            }
        }
        // solve tasks: each tile of each large front once per direction, in
        // dependency order (forward pivot tiles ascending before the front's
        // update tiles; backward pivot tiles descending)
        for (int dir = 0; dir < 2; ++dir) {
            const std::vector<int>& beg = dir == 0 ? Q.fwd_task_beg : Q.bwd_task_beg;
            for (int l = 0; l < P.nlevels; ++l) {
                std::vector<int> done_piv(ns, 0), upd(ns, 0);
                for (int q = beg[l]; q < beg[l + 1]; ++q) {
                    const int s = Q.tasks[2 * q], t = Q.tasks[2 * q + 1];
                    if (s < 0 || s >= ns || level[s] != l || !is_large[s]) bad("solve task front");
                    const FrontDesc& f = P.fronts[s];
                    const int nt1 = (f.c + T - 1) / T, NT = front_tiles(f.m, f.c, T);
                    if (dir == 0) {
                        const int i = t & 0xffff, cnt = t >> 16;
                        if (cnt < 1 || i + cnt > NT) bad("forward task tiles", s);
                        if (i < nt1) {
                            if (cnt != 1 || i != done_piv[s] || upd[s]) bad("forward pivot order", s);
                            done_piv[s]++;
                        } else {
                            if (done_piv[s] != nt1 || i != nt1 + upd[s]) bad("forward update order", s);
                            upd[s] += cnt;
                        }
                    } else {
                        if (t != nt1 - 1 - done_piv[s]) bad("backward pivot order", s);
                        done_piv[s]++;
                    }
                }
                for (int q = P.large_ptr[l]; q < P.large_ptr[l + 1]; ++q) {
                    const int s = P.large_list[q];
                    const FrontDesc& f = P.fronts[s];
                    const int nt1 = (f.c + T - 1) / T, NT = front_tiles(f.m, f.c, T);
                    if (done_piv[s] != nt1 || (dir == 0 && upd[s] != NT - nt1))
                        bad("solve tasks do not cover the front", s);
                }
            }
        }
        // the one-launch solve's item lists: every front's work exactly once
        // (forward: each pivot tile alone and in order, then update tasks
        // covering the update tiles in order; backward: each gather (j, h)
        // once, each pivot tile once, descending, after its gathers; small
        // fronts in warp items of at most kWarpsPerItem warps, each once), in
        // a topological order: forward all of a front's items after all of
        // its children's, backward after all of its parent's
        {
            const int WPI = SolveScheduleHost::kWarpsPerItem;
            for (int dir = 0; dir < 2; ++dir) {
                const std::vector<int>& it = dir == 0 ? Q.fwd_items : Q.bwd_items;
                const std::vector<int>& wl = dir == 0 ? Q.fwd_wlist : Q.bwd_wlist;
                if (it.size() % 4) bad("solve items");
                if (wl.size() != P.small_list.size()) bad("solve warp list size");
                const int64_t nit = (int64_t)it.size() / 4;
                std::vector<int64_t> first(ns, -1), last(ns, -1);
                std::vector<int> piv(ns, 0), upd(ns, 0), wseen(ns, 0);
                std::vector<std::vector<char>> gseen(ns);
                std::vector<int> gcnt(ns, 0);
                std::vector<char> wl_used(wl.size(), 0);
                auto touch = [&](int s, int64_t k) {
                    if (first[s] < 0) first[s] = k;
                    last[s] = k;
                };
                for (int64_t k = 0; k < nit; ++k) {
                    const int* e = it.data() + 4 * k;
                    if (e[0] == SolveScheduleHost::kItemWarps) {
                        const int n1 = e[2] & 0xff, n2 = (e[2] >> 8) & 0xff, n4 = e[2] >> 16;
                        const int nf = n1 + n2 + n4;
                        if (nf < 1 || n1 + (n2 + 1) / 2 + (n4 + 3) / 4 > WPI || e[1] < 0 ||
                            (size_t)e[1] + nf > wl.size())
                            bad("solve warp item");
                        for (int q = 0; q < nf; ++q) {
                            if (wl_used[e[1] + q]++) bad("solve warp list entry used twice");
                            const int s = wl[e[1] + q];
                            if (s < 0 || s >= ns || is_large[s]) bad("solve warp list entry");
                            const int m = P.fronts[s].m;
                            if ((q < n1) != (m > 16) || (q >= n1 + n2) != (m <= 8))
                                bad("solve warp item size class", s);
                            wseen[s]++;
                            touch(s, k);
                        }
                        continue;
                    }
                    const int s = e[1], t = e[2];
                    if (s < 0 || s >= ns || !is_large[s]) bad("solve item front");
                    const FrontDesc& f = P.fronts[s];
                    const int nt1 = (f.c + T - 1) / T, NT = front_tiles(f.m, f.c, T);
                    const int nch = Q.gather_nch[s];
                    if (gseen[s].empty()) gseen[s].assign((size_t)nt1 * std::max(nch, 1), 0);
                    touch(s, k);
                    if (e[0] == SolveScheduleHost::kItemGather) {
                        const int j = t & 0xffff, h = t >> 16;
                        if (dir != 1 || j >= nt1 || h >= nch || gseen[s][(size_t)j * nch + h]++ ||
                            piv[s] > nt1 - 1 - j)
                            bad("solve gather item", s);
                        gcnt[s]++;
                    } else if (e[0] != SolveScheduleHost::kItemTile) {
                        bad("solve item kind", s);
                    } else if (dir == 0) {
                        const int i = t & 0xffff, cnt = t >> 16;
                        if (cnt < 1 || i + cnt > NT) bad("forward item tiles", s);
                        if (i < nt1) {
                            if (cnt != 1 || i != piv[s] || upd[s]) bad("forward pivot order", s);
                            piv[s]++;
                        } else {
                            if (piv[s] != nt1 || i != nt1 + upd[s]) bad("forward update order", s);
                            upd[s] += cnt;
                        }
                    } else {
                        if (t != nt1 - 1 - piv[s]) bad("backward pivot order", s);
                        for (int h = 0; h < nch; ++h)
                            if (!gseen[s][(size_t)t * nch + h]) bad("backward pivot before its gathers", s);
                        piv[s]++;
                    }
                }
                for (int s = 0; s < ns; ++s) {
                    const FrontDesc& f = P.fronts[s];
                    if (is_large[s]) {
                        const int nt1 = (f.c + T - 1) / T, NT = front_tiles(f.m, f.c, T);
                        if (piv[s] != nt1 || (dir == 0 && upd[s] != NT - nt1) ||
                            (dir == 1 && gcnt[s] != nt1 * Q.gather_nch[s]))
                            bad("solve items do not cover the front", s);
                    } else if (wseen[s] != 1) {
                        bad("small front not in exactly one warp item", s);
                    }
                    if (f.parent >= 0) {
                        const bool ok = dir == 0 ? last[s] < first[f.parent]
                                                 : last[f.parent] < first[s];
                        if (!ok) bad("solve items out of dependency order", s);
                    }
                }
            }
            if ((int)Q.bwd_target.size() != ns) bad("backward targets");
            for (int s = 0; s < ns; ++s)
                if (Q.bwd_target[s] != (is_large[s] ? (P.fronts[s].c + T - 1) / T : 1))
                    bad("backward target", s);
        }
        // the residual's CSR of the caller's matrix
        if ((int)csr_rowptr.size() != n + 1 || csr_rowptr[0] != 0 || csr_rowptr[n] != csr_nnz)
            bad("CSR row pointers");
        for (int i = 0; i < n; ++i)
            if (csr_rowptr[i + 1] < csr_rowptr[i]) bad("CSR row pointers decrease");
        for (int64_t q = 0; q < csr_nnz; ++q)
            if (csr_col[q] < 0 || csr_col[q] >= n || csr_src[q] < 0 || csr_src[q] >= P.nnz_user)
                bad("CSR entry out of range");
    } catch (const Fail& f) {
        return f.msg;
    }
    return std::string();
}

std::string check_panel_schedule(const Plan& P, const PanelSchedule& S,
                                 const std::vector<int>& level, int T, int PW) {
    try {
        const int ns = P.nsuper, TPP = PW / T;
        std::vector<char> is_large(ns, 0);
        for (int s : P.large_list) is_large[s] = 1;
        std::vector<char> counter_used(S.ncounters, 0);
        for (int l = 0; l < P.nlevels; ++l) {
            for (int q = S.op_beg[l]; q < S.op_beg[l + 1]; ++q) {
                const PanelOp& op = S.ops[q];
                if (op.kind != OP_PANEL) continue;
                const int klo = op.arg * TPP;
                if (op.counter < 0 || op.counter >= S.ncounters || counter_used[op.counter]++)
                    bad("panel ticket counter");
                if (op.toff < 0 || op.ntasks < 1 ||
                    2 * (op.toff + op.ntasks) > (int64_t)S.tasks.size())
                    bad("panel task range");
                // every task's waits (the pivot tiles of the panel above its
                // row) name diagonal tasks earlier in the list
                std::map<int, std::vector<char>> done;
                for (int64_t t = op.toff; t < op.toff + op.ntasks; ++t) {
                    const int s = S.tasks[2 * t], i = S.tasks[2 * t + 1];
                    if (s < 0 || s >= ns || !is_large[s] || level[s] != l) bad("panel task front");
                    const FrontDesc& f = P.fronts[s];
                    const int nt1 = (f.c + T - 1) / T, NT = front_tiles(f.m, f.c, T);
                    const int khi = std::min(klo + TPP, nt1);
                    if (klo >= nt1 || i < klo || i >= NT) bad("panel task row tile", s);
                    if (P.dinv_off[s] < 0 || P.dinv_off[s] % ((int64_t)T * T) ||
                        P.dinv_off[s] / ((int64_t)T * T) + nt1 > S.nflags)
                        bad("panel flag range", s);
                    std::vector<char>& d = done[s];
                    d.resize(NT, 0);
                    for (int k = klo; k < std::min(i, khi); ++k)
                        if (!d[k]) bad("panel task order", s);
                    if (d[i]++) bad("panel task repeated", s);
                }
                for (int qq = P.large_ptr[l]; qq < P.large_ptr[l + 1]; ++qq) {
                    const int s = P.large_list[qq];
                    const FrontDesc& f = P.fronts[s];
                    const int nt1 = (f.c + T - 1) / T, NT = front_tiles(f.m, f.c, T);
                    if (klo >= nt1) continue;
                    auto it = done.find(s);
                    for (int i = klo; i < NT; ++i)
                        if (it == done.end() || !it->second[i])
                            bad("panel tasks do not cover the front", s);
                }
            }
        }
    } catch (const Fail& f) {
        return f.msg;
    }
    return std::string();
}

}  // namespace mdgpu
