// Numeric plan construction (see plan.hpp).
#include "plan.hpp"

#include <algorithm>
#include <map>
#include <set>
#include <atomic>
#include <cmath>
#include <exception>
#include <stdexcept>
#include <string>
#include <thread>

#include "parallel.hpp"

namespace mdgpu {

// The trees of an assembly forest (a batch of independent systems) as
// contiguous supernode ranges [beg, end): each tree ends at its root and holds
// only its own descendants.  A single range when that does not hold.
static std::vector<std::pair<int, int>> tree_ranges(const AssemblyTree& t,
                                                    const std::vector<int>& parent) {
    const int ns = t.size();
    std::vector<std::pair<int, int>> r;
    int beg = 0;
    for (int s = 0; s < ns; ++s) {
        for (int h = t.child_ptr[s]; h < t.child_ptr[s + 1]; ++h)
            if (t.child[h] < beg || t.child[h] >= s) return {{0, ns}};
        if (parent[s] < 0) {
            r.push_back({beg, s + 1});
            beg = s + 1;
        }
    }
    if (beg != ns || r.empty()) return {{0, ns}};
    return r;
}

// fn(beg, end) on every range, ranges shared out to the host's cores
template <typename F>
static void for_each_range(const std::vector<std::pair<int, int>>& rg, F&& fn) {
    parallel_for((int)rg.size(), [&](int i) { fn(rg[i].first, rg[i].second); });
}

const int Plan::small_limit[kSmallBuckets] = {16, 32, 64, 96, 128, 160};

static int64_t align_up(int64_t x, int64_t a) { return (x + a - 1) / a * a; }
static int round8(int x) { return (x + 7) & ~7; }

int64_t lifetime_alloc(const std::vector<int>& beg, const std::vector<int>& end,
                       const std::vector<int64_t>& size, int nlev, std::vector<int64_t>& off) {
    const int nb = (int)size.size();
    off.assign(nb, -1);
    std::vector<std::vector<int>> starts(std::max(nlev, 1)), ends(std::max(nlev, 1));
    for (int i = 0; i < nb; ++i)
        if (size[i] > 0) {
            starts[beg[i]].push_back(i);
            ends[end[i]].push_back(i);
        }
    std::map<int64_t, int64_t> by_off;                 // free ranges: offset -> size
    std::set<std::pair<int64_t, int64_t>> by_size;     // (size, offset)
    auto drop = [&](std::map<int64_t, int64_t>::iterator it) {
        by_size.erase({it->second, it->first});
        by_off.erase(it);
    };
    int64_t top = 0, peak = 0;
    for (int l = 0; l < nlev; ++l) {
        if (l > 0)
            for (int i : ends[l - 1]) {
                int64_t o = off[i], z = size[i];
                auto nx = by_off.lower_bound(o);
                if (nx != by_off.end() && nx->first == o + z) {
                    z += nx->second;
                    auto d = nx++;
                    drop(d);
                }
                if (nx != by_off.begin()) {
                    auto pv = std::prev(nx);
                    if (pv->first + pv->second == o) {
                        o = pv->first;
                        z += pv->second;
                        drop(pv);
                    }
                }
                if (o + z == top) {
                    top = o;
                } else {
                    by_off[o] = z;
                    by_size.insert({z, o});
                }
            }
        std::vector<int>& st = starts[l];
        std::sort(st.begin(), st.end(), [&](int a, int b) {
            return size[a] != size[b] ? size[a] > size[b] : a < b;
        });
        for (int i : st) {
            const int64_t z = size[i];
            // best fit: the smallest free range that holds it (lowest
            // offset among equals)
            auto fit = by_size.lower_bound({z, INT64_MIN});
            if (fit != by_size.end()) {
                const int64_t o = fit->second, fz = fit->first;
                drop(by_off.find(o));
                off[i] = o;
                if (fz > z) {
                    by_off[o + z] = fz - z;
                    by_size.insert({fz - z, o + z});
                }
            } else {
                off[i] = top;
                top += z;
                peak = std::max(peak, top);
            }
        }
    }
    return peak;
}

int front_tiles(int m, int c, int T) { return (c + T - 1) / T + (m - c + T - 1) / T; }

void build_plan(const Symbolic& S, int64_t nnz_user, int large_threshold, Plan& P) {
    P = Plan();
    if (large_threshold > Plan::kSmallMaxRows ||
        Plan::small_limit[kSmallBuckets - 1] != Plan::kSmallMaxRows)
        throw std::runtime_error("small fronts must have at most 160 rows");
    const AssemblyTree& t = S.tree;
    int n = S.n, ns = t.size();
    P.n = n;
    P.nsuper = ns;
    P.nnz_user = nnz_user;
    P.perm = S.perm;
    if (!P.perm.empty()) {
        P.iperm.resize(n);
        for (int k = 0; k < n; ++k) P.iperm[P.perm[k]] = k;
    }
    P.Lp = S.Lp;
    P.lnz = S.Lp[n];
    for (int j = 0; j < n; ++j) P.flops += (double)S.count[j] * S.count[j] + 1.0;

    std::vector<int> parent(ns, -1);
    for (int s = 0; s < ns; ++s)
        for (int h = t.child_ptr[s]; h < t.child_ptr[s + 1]; ++h) parent[t.child[h]] = s;

    // Front row sets, bottom-up in visiting order: the pivot rows, then the
    // sorted union of A's rows below the supernode and the children's update
    // rows.  This is the row set the reference builds with MatrizGetFk_3 and
    // VectorMerge (mdgpu.cu:180-291,1456,1489-1508,1566).
    // The row count of front s is the column count of its first column, so
    // the sets go straight into one flat array (checked as they are formed).
    const SparseCol& A = S.lower;
    std::vector<int64_t> rows_off(ns + 1, 0);
    for (int s = 0; s < ns; ++s) {
        const int cnt = S.count[t.first_col[s]];
        if (cnt < t.ncols[s] || cnt > n - t.first_col[s])
            throw std::runtime_error("front " + std::to_string(s) + ": column count " +
                                     std::to_string(cnt) + " out of range");
        rows_off[s + 1] = rows_off[s] + cnt;
    }
    if (rows_off[ns] > INT32_MAX) throw std::runtime_error("row arrays exceed 2^31 entries");
    P.rows.resize(rows_off[ns]);    // every entry is written below
    P.relmap.resize(rows_off[ns]);  // likewise (-1 where there is no parent row)
    const auto ranges = tree_ranges(t, parent);
    for_each_range(ranges, [&](int s0, int s1) {
        std::vector<int> scratch;
        for (int s = s0; s < s1; ++s) {
            int k = t.first_col[s], c = t.ncols[s];
            scratch.clear();
            for (int j = k; j < k + c; ++j)
                for (int p = A.colptr[j]; p < A.colptr[j + 1]; ++p)
                    if (A.rowidx[p] >= k + c) scratch.push_back(A.rowidx[p]);
            for (int h = t.child_ptr[s]; h < t.child_ptr[s + 1]; ++h) {
                int ch = t.child[h];
                for (int64_t i = rows_off[ch] + t.ncols[ch]; i < rows_off[ch + 1]; ++i) {
                    const int rc = P.rows[i];
                    if (rc < k) throw std::runtime_error("child update row below its parent");
                    if (rc >= k + c) scratch.push_back(rc);
                }
            }
            std::sort(scratch.begin(), scratch.end());
            scratch.erase(std::unique(scratch.begin(), scratch.end()), scratch.end());
            const int64_t m = c + (int64_t)scratch.size();
            if (m != rows_off[s + 1] - rows_off[s])
                throw std::runtime_error("front " + std::to_string(s) + " has " + std::to_string(m) +
                                         " rows but column count " + std::to_string(S.count[k]));
            int* r = P.rows.data() + rows_off[s];
            for (int i = 0; i < c; ++i) r[i] = k + i;
            std::copy(scratch.begin(), scratch.end(), r + c);
        }
        // relative maps: position of each update row of s inside its parent's
        // rows; -1 for the pivot rows and for a root's rows
        for (int s = s0; s < s1; ++s) {
            int p = parent[s];
            int* rm = P.relmap.data() + rows_off[s];
            std::fill(rm, rm + (p < 0 ? rows_off[s + 1] - rows_off[s] : t.ncols[s]), -1);
            if (p < 0) continue;
            const int* rs = P.rows.data() + rows_off[s];
            const int* rp = P.rows.data() + rows_off[p];
            const int64_t ms = rows_off[s + 1] - rows_off[s], mp = rows_off[p + 1] - rows_off[p];
            int64_t q = 0;
            for (int64_t i = t.ncols[s]; i < ms; ++i) {
                while (q < mp && rp[q] < rs[i]) ++q;
                if (q == mp || rp[q] != rs[i]) throw std::runtime_error("row not in parent");
                P.relmap[rows_off[s] + i] = (int)q;
            }
        }
    });

    // storage offsets and descriptors.  The offsets are prefix sums of the
    // 32-aligned panel and update sizes (offsets start at 0 and stay aligned,
    // so align_up(off + size) = off + align_up(size)): sums per range, then
    // the ranges filled in parallel from their bases.
    P.fronts.resize(ns);  // every descriptor is written below
    const int nrg = (int)ranges.size();
    std::vector<int64_t> rg_l(nrg + 1, 0), rg_u(nrg + 1, 0);
    std::vector<int> rg_maxm(nrg, 0), rg_maxu(nrg, 0);
    auto panel_size = [&](int s, int64_t& lsz, int64_t& usz) {
        const int m = (int)(rows_off[s + 1] - rows_off[s]), c = t.ncols[s], u = m - c;
        lsz = align_up((int64_t)round8(m) * c, 32);
        usz = (parent[s] >= 0 && u > 0) ? align_up((int64_t)round8(u) * u, 32) : -1;
    };
    parallel_for(nrg, [&](int r) {
        int64_t sl = 0, su = 0;
        for (int s = ranges[r].first; s < ranges[r].second; ++s) {
            int64_t lsz, usz;
            panel_size(s, lsz, usz);
            sl += lsz;
            if (usz >= 0) su += usz;
        }
        rg_l[r + 1] = sl;
        rg_u[r + 1] = su;
    });
    for (int r = 0; r < nrg; ++r) {
        rg_l[r + 1] += rg_l[r];
        rg_u[r + 1] += rg_u[r];
    }
    parallel_for(nrg, [&](int r) {
        int64_t lo = rg_l[r], uo = rg_u[r];
        for (int s = ranges[r].first; s < ranges[r].second; ++s) {
            int64_t lsz, usz;
            panel_size(s, lsz, usz);
            FrontDesc& f = P.fronts[s];
            f.m = (int)(rows_off[s + 1] - rows_off[s]);
            f.c = t.ncols[s];
            f.ldl = round8(f.m);
            const int u = f.m - f.c;
            f.ldu = round8(u);
            f.loff = lo;
            lo += lsz;
            if (usz >= 0) {
                f.uoff = uo;
                uo += usz;
            } else {
                f.uoff = -1;
            }
            f.rows_off = (int)rows_off[s];
            f.first_col = t.first_col[s];
            f.child_beg = t.child_ptr[s];
            f.child_end = t.child_ptr[s + 1];
            f.a_beg = A.colptr[f.first_col];
            f.a_end = A.colptr[f.first_col + f.c];
            f.parent = parent[s];
            f.pad_ = 0;
            rg_maxm[r] = std::max(rg_maxm[r], f.m);
            rg_maxu[r] = std::max(rg_maxu[r], u);
        }
    });
    for (int r = 0; r < nrg; ++r) {
        P.max_m = std::max(P.max_m, rg_maxm[r]);
        P.max_u = std::max(P.max_u, rg_maxu[r]);
    }
    const int64_t lo = rg_l[nrg];
    P.lstore = std::max<int64_t>(lo, 32);
    P.child = t.child;
    {
        // update matrices over their lifetimes in the level schedule: the
        // factor writes U_s at level lev(s) and its parent's assembly reads
        // it at lev(parent); the selected inverse (top-down) writes Z_UU of s
        // at lev(s) and its children read it down to their lowest level
        const std::vector<int> lev = front_levels(P);
        int nlev = 0;
        for (int s = 0; s < ns; ++s) nlev = std::max(nlev, lev[s] + 1);
        std::vector<int> fb(ns), fe(ns), zb(ns), ze(ns);
        std::vector<int64_t> usz(ns, 0), uoff, zoff;
        for (int s = 0; s < ns; ++s) {
            const FrontDesc& f = P.fronts[s];
            fb[s] = fe[s] = zb[s] = ze[s] = lev[s];
            if (f.uoff < 0) continue;
            usz[s] = align_up((int64_t)f.ldu * (f.m - f.c), 32);
            fe[s] = lev[f.parent];
            for (int h = f.child_beg; h < f.child_end; ++h)
                zb[s] = std::min(zb[s], lev[P.child[h]]);
        }
        P.ustore = std::max<int64_t>(lifetime_alloc(fb, fe, usz, nlev, uoff), 32);
        P.zustore = std::max<int64_t>(lifetime_alloc(zb, ze, usz, nlev, zoff), 32);
        P.zuoff = zoff;
        for (int s = 0; s < ns; ++s) P.fronts[s].uoff = usz[s] > 0 ? uoff[s] : -1;
    }

    // A entries: the lower triangle's entries of the supernode's columns are
    // contiguous (columns are consecutive).  A repeated (row, col) keeps the
    // last occurrence, as the reference's front assembly overwrites
    // (mdgpu.cu:274-282).
    int nnz = A.nnz();
    P.a_src.resize(nnz);
    P.a_pos.resize(nnz);
    for_each_range(ranges, [&](int s0, int s1) {
        for (int s = s0; s < s1; ++s) {
            const FrontDesc& f = P.fronts[s];
            const int* r = P.rows.data() + f.rows_off;
            for (int jj = 0; jj < f.c; ++jj) {
                int j = f.first_col + jj;
                for (int p = A.colptr[j]; p < A.colptr[j + 1]; ++p) {
                    int row = A.rowidx[p];
                    int pos = (int)(std::lower_bound(r, r + f.m, row) - r);
                    if (pos >= f.m || r[pos] != row)
                        throw std::runtime_error("A entry outside front");
                    if (f.m >= 65536) throw std::runtime_error("front too large for packed A map");
                    P.a_src[p] = S.lower_src[p];
                    P.a_pos[p] = pos | (jj << 16);
                }
            }
            // duplicates: keep the last in storage order
            bool dup = false;
            for (int jj = 0; jj < f.c && !dup; ++jj) {
                int j = f.first_col + jj;
                for (int p = A.colptr[j] + 1; p < A.colptr[j + 1]; ++p)
                    if (A.rowidx[p] <= A.rowidx[p - 1]) dup = true;
            }
            if (dup) {
                for (int jj = 0; jj < f.c; ++jj) {
                    int j = f.first_col + jj;
                    for (int p = A.colptr[j]; p < A.colptr[j + 1]; ++p)
                        for (int q = p + 1; q < A.colptr[j + 1]; ++q)
                            if (A.rowidx[q] == A.rowidx[p]) {
                                P.a_src[p] = -1;
                                break;
                            }
                }
            }
        }
    });

    // levels
    std::vector<int> level(ns, 0);
    for (int s = 0; s < ns; ++s)
        for (int h = t.child_ptr[s]; h < t.child_ptr[s + 1]; ++h)
            level[s] = std::max(level[s], level[t.child[h]] + 1);
    P.nlevels = ns ? *std::max_element(level.begin(), level.end()) + 1 : 0;
    int L = P.nlevels;
    std::vector<std::vector<int>> small(L * kSmallBuckets), large(L);
    for (int s = 0; s < ns; ++s) {
        int m = P.fronts[s].m;
        if (m > large_threshold) {
            large[level[s]].push_back(s);
            continue;
        }
        int b = 0;
        while (b < kSmallBuckets - 1 && m > Plan::small_limit[b]) ++b;
        small[level[s] * kSmallBuckets + b].push_back(s);
    }
    P.small_ptr.assign(L * kSmallBuckets + 1, 0);
    for (int i = 0; i < L * kSmallBuckets; ++i) {
        P.small_ptr[i + 1] = P.small_ptr[i] + (int)small[i].size();
        P.small_list.insert(P.small_list.end(), small[i].begin(), small[i].end());
    }
    P.large_ptr.assign(L + 1, 0);
    P.a_colptr_off.assign(ns, -1);
    for (int l = 0; l < L; ++l) {
        P.large_ptr[l + 1] = P.large_ptr[l] + (int)large[l].size();
        P.large_list.insert(P.large_list.end(), large[l].begin(), large[l].end());
        for (int s : large[l]) {
            const FrontDesc& f = P.fronts[s];
            P.a_colptr_off[s] = (int)P.a_colptr.size();
            for (int jj = 0; jj <= f.c; ++jj)
                P.a_colptr.push_back(A.colptr[f.first_col + jj] - f.a_beg);
        }
    }
    if (P.a_colptr.empty()) P.a_colptr.push_back(0);
}

void build_large_tables(Plan& P, int T, int CB) {
    P.dinv_off.assign(P.nsuper, -1);
    P.asm_off.assign(P.nsuper, -1);
    P.asm_range.clear();
    int64_t d = 0;
    for (int s : P.large_list) {
        const FrontDesc& f = P.fronts[s];
        P.dinv_off[s] = d;
        d += (int64_t)((f.c + T - 1) / T) * T * T;
        int nblk = (f.m + CB - 1) / CB;
        P.asm_off[s] = (int)P.asm_range.size();
        for (int b = 0; b < nblk; ++b) {
            int j0 = b * CB, j1 = std::min(j0 + CB, f.m);
            for (int h = f.child_beg; h < f.child_end; ++h) {
                const FrontDesc& g = P.fronts[P.child[h]];
                const int* rm = P.relmap.data() + g.rows_off + g.c;
                int uc = g.m - g.c;
                int lo = (int)(std::lower_bound(rm, rm + uc, j0) - rm);
                int hi = (int)(std::lower_bound(rm, rm + uc, j1) - rm);
                P.asm_range.push_back(lo);
                P.asm_range.push_back(hi);
            }
        }
    }
    P.dinv_total = std::max<int64_t>(d, 32);
    if (P.asm_range.empty()) P.asm_range.push_back(0);
}

WorkList ListStore::add(const std::vector<std::pair<int, int>>& it, int step) {
    WorkList w;
    w.off = (int64_t)items.size();
    w.nitems = (int)it.size();
    w.step = step;
    int acc = 0;
    for (auto& [s, cnt] : it) {
        items.push_back(s);
        ctas_before.push_back(acc);
        acc += cnt;
    }
    items.push_back(-1);
    ctas_before.push_back(acc);
    w.nctas = acc;
    return w;
}

void build_factor_schedule(const Plan& P, int T, int assemble_cols, TileSchedule& S) {
    S = TileSchedule();
    S.T = T;
    S.level_beg.assign(P.nlevels + 1, 0);
    for (int l = 0; l < P.nlevels; ++l) {
        S.level_beg[l] = (int)S.trsm.size();
        std::vector<std::pair<int, int>> as;
        int maxsteps = 0;
        for (int q = P.large_ptr[l]; q < P.large_ptr[l + 1]; ++q) {
            const FrontDesc& f = P.fronts[P.large_list[q]];
            maxsteps = std::max(maxsteps, (f.c + T - 1) / T);
            as.push_back({P.large_list[q], (f.m + assemble_cols - 1) / assemble_cols});
        }
        S.assemble.push_back(S.store.add(as, 0));
        for (int k = 0; k < maxsteps; ++k) {
            std::vector<std::pair<int, int>> tr, up;
            for (int q = P.large_ptr[l]; q < P.large_ptr[l + 1]; ++q) {
                int s = P.large_list[q];
                const FrontDesc& f = P.fronts[s];
                int nt1 = (f.c + T - 1) / T;
                if (k >= nt1) continue;
                int rem = front_tiles(f.m, f.c, T) - k - 1;
                if (rem > 0) {
                    tr.push_back({s, rem});
                    up.push_back({s, rem * (rem + 1) / 2});
                }
            }
            S.trsm.push_back(S.store.add(tr, k));
            S.update.push_back(S.store.add(up, k));
        }
    }
    S.level_beg[P.nlevels] = (int)S.trsm.size();
}

void build_solve_schedule(const Plan& P, int T, SolveScheduleHost& S) {
    S = SolveScheduleHost();
    S.T = T;
    // level tasks.  Forward: row tile i of front s; pivot tiles (i < nt1)
    // wait for pivot tiles 0..i-1, update tiles for all nt1 of them, so the
    // key i (pivot) / nt1 (update) orders dependencies first.  Backward:
    // pivot column tile j waits for pivot tiles j+1..nt1-1: key nt1-1-j.
    S.tasks.clear();
    S.fwd_task_beg.assign(P.nlevels + 1, 0);
    S.bwd_task_beg.assign(P.nlevels + 1, 0);
    S.fwd_elems.assign(P.nlevels, 0.0);
    S.bwd_elems.assign(P.nlevels, 0.0);
    S.small_elems.assign(P.nlevels, 0.0);
    for (int l = 0; l < P.nlevels; ++l)
        for (int q = P.small_ptr[l * kSmallBuckets]; q < P.small_ptr[(l + 1) * kSmallBuckets]; ++q) {
            const FrontDesc& f = P.fronts[P.small_list[q]];
            S.small_elems[l] += (double)f.c * (f.c + 1) / 2 + (double)(f.m - f.c) * f.c;
        }
    int64_t ntiles_piv = 0;
    for (int s : P.large_list) ntiles_piv += (P.fronts[s].c + T - 1) / T;
    S.nflags = (int)ntiles_piv;
    struct Key {
        int key, ord, s, t;
    };
    auto emit = [&](std::vector<Key>& ks) {
        std::stable_sort(ks.begin(), ks.end(), [](const Key& a, const Key& b) {
            return a.key != b.key ? a.key < b.key : a.ord < b.ord;
        });
        for (const Key& k : ks) {
            S.tasks.push_back(k.s);
            S.tasks.push_back(k.t);
        }
    };
    for (int dir = 0; dir < 2; ++dir) {
        for (int l = 0; l < P.nlevels; ++l) {
            (dir == 0 ? S.fwd_task_beg : S.bwd_task_beg)[l] = (int)(S.tasks.size() / 2);
            std::vector<Key> ks;
            double bytes = 0;
            int ord = 0;
            for (int q = P.large_ptr[l]; q < P.large_ptr[l + 1]; ++q) {
                const int s = P.large_list[q];
                const FrontDesc& f = P.fronts[s];
                const int nt1 = (f.c + T - 1) / T, NT = front_tiles(f.m, f.c, T);
                bytes += (double)f.c * (f.c + 1) / 2 + (double)(f.m - f.c) * f.c +
                         (double)nt1 * T * T;
                if (dir == 0) {
                    // pivot tiles one per task; update tiles in groups of
                    // kFwdGroupBlocks / nt1 (streamed by one CTA)
                    for (int i = 0; i < nt1; ++i) ks.push_back({i, ord++, s, i | (1 << 16)});
                    const int G = std::max(1, std::min(SolveScheduleHost::kFwdGroupBlocks / nt1,
                                                       SolveScheduleHost::kFwdGroupTiles));
                    for (int i = nt1; i < NT; i += G)
                        ks.push_back({nt1, ord++, s, i | (std::min(G, NT - i) << 16)});
                } else
                    for (int j = 0; j < nt1; ++j) ks.push_back({nt1 - 1 - j, ord++, s, j});
            }
            (dir == 0 ? S.fwd_elems : S.bwd_elems)[l] = bytes;
            emit(ks);
        }
        (dir == 0 ? S.fwd_task_beg : S.bwd_task_beg)[P.nlevels] = (int)(S.tasks.size() / 2);
    }
    S.warp_list.assign(P.small_list.size(), 0);
    S.warp_cnt.assign(3 * (size_t)P.nlevels, 0);
    {
        // per level a stable counting sort of the small fronts by rows,
        // descending (small fronts have at most kSmallMaxRows rows)
        constexpr int MX = Plan::kSmallMaxRows;
        std::vector<int> at(MX + 2);
        for (int l = 0; l < P.nlevels; ++l) {
            const int b = P.small_ptr[l * kSmallBuckets], e = P.small_ptr[(l + 1) * kSmallBuckets];
            std::fill(at.begin(), at.end(), 0);
            for (int q = b; q < e; ++q) {
                const int m = P.fronts[P.small_list[q]].m;
                if (m < 1 || m > MX) throw std::runtime_error("small front of unexpected size");
                at[MX - m + 1]++;  // slot of m: fronts with more rows first
                S.warp_cnt[3 * l + (m > 16 ? 0 : (m > 8 ? 1 : 2))]++;
            }
            for (int k = 0; k <= MX; ++k) at[k + 1] += at[k];
            for (int q = b; q < e; ++q) {
                const int s = P.small_list[q];
                S.warp_list[b + at[MX - P.fronts[s].m]++] = s;
            }
        }
    }
    S.fv_off.assign(P.nsuper, 0);
    S.fv_rows = 0;
    for (int s = 0; s < P.nsuper; ++s) {
        S.fv_off[s] = S.fv_rows;
        S.fv_rows += P.fronts[s].m;
    }
    if (S.fv_rows > INT32_MAX) throw std::runtime_error("front vectors exceed 2^31 rows");
    // assembly maps of the large fronts: sizes first (rows m + 1, entries =
    // the children's update rows), then each front filled on its own
    S.amap_off.assign(P.nsuper, -1);
    const int nlarge = (int)P.large_list.size();
    std::vector<int64_t> row_base(nlarge + 1, 0), ent_base(nlarge + 1, 0);
    for (int k = 0; k < nlarge; ++k) {
        const FrontDesc& f = P.fronts[P.large_list[k]];
        int64_t ent = 0;
        for (int h = f.child_beg; h < f.child_end; ++h) {
            const FrontDesc& g = P.fronts[P.child[h]];
            ent += g.m - g.c;
        }
        row_base[k + 1] = row_base[k] + f.m + 1;
        ent_base[k + 1] = ent_base[k] + ent;
    }
    if (ent_base[nlarge] > INT32_MAX) throw std::runtime_error("assembly map exceeds 2^31 entries");
    if (row_base[nlarge] > INT32_MAX) throw std::runtime_error("assembly map exceeds 2^31 rows");
    S.amap_row.resize(row_base[nlarge]);  // every entry is written below
    S.amap_ent.resize(ent_base[nlarge]);
    parallel_for(nlarge, [&](int k) {
        const int s = P.large_list[k];
        const FrontDesc& f = P.fronts[s];
        std::vector<int> cnt(f.m + 1, 0);
        for (int h = f.child_beg; h < f.child_end; ++h) {
            const FrontDesc& g = P.fronts[P.child[h]];
            const int* rm = P.relmap.data() + g.rows_off + g.c;
            for (int rr = 0; rr < g.m - g.c; ++rr) cnt[rm[rr] + 1]++;
        }
        for (int r = 0; r < f.m; ++r) cnt[r + 1] += cnt[r];
        const int64_t base = ent_base[k];
        S.amap_off[s] = (int)row_base[k];
        for (int r = 0; r <= f.m; ++r) S.amap_row[row_base[k] + r] = (int)(base + cnt[r]);
        for (int h = f.child_beg; h < f.child_end; ++h) {  // child order kept per row
            const int ch = P.child[h];
            const FrontDesc& g = P.fronts[ch];
            const int* rm = P.relmap.data() + g.rows_off + g.c;
            for (int rr = 0; rr < g.m - g.c; ++rr)
                S.amap_ent[base + cnt[rm[rr]]++] = (int)(S.fv_off[ch] + g.c + rr);
        }
    });
    const int GC = SolveScheduleHost::kGatherTiles;
    S.gather_task_beg.assign(P.nlevels + 1, 0);
    S.gather_nch.assign(P.nsuper, 0);
    S.gather_off.assign(P.nsuper, 0);
    S.gather_vecs = 0;
    int64_t vecs = 0;
    for (int l = 0; l < P.nlevels; ++l) {
        S.gather_task_beg[l] = (int)(S.tasks.size() / 2);
        for (int q = P.large_ptr[l]; q < P.large_ptr[l + 1]; ++q) {
            const int s = P.large_list[q];
            const FrontDesc& f = P.fronts[s];
            const int nt1 = (f.c + T - 1) / T, nu = (f.m - f.c + T - 1) / T;
            const int nch = (nu + GC - 1) / GC;
            S.gather_nch[s] = nch;
            if (vecs + (int64_t)nt1 * nch > INT32_MAX)
                throw std::runtime_error("update-row partial sums exceed 2^31 vectors");
            S.gather_off[s] = (int)vecs;
            vecs += (int64_t)nt1 * nch;
            for (int j = 0; j < nt1; ++j)
                for (int h = 0; h < nch; ++h) {
                    S.tasks.push_back(s);
                    S.tasks.push_back(j | (h << 16));
                }
        }
    }
    S.gather_vecs = vecs;
    S.gather_task_beg[P.nlevels] = (int)(S.tasks.size() / 2);
    // the fused launches' item lists: fronts level by level (forward
    // bottom-up, backward top-down), within a level by critical-path
    // priority (an estimate of the latency from the front to the end of the
    // sweep: forward, the front and its ancestors up to the root; backward,
    // the front and its longest descendant chain), highest first.  A front's
    // dependencies (forward: its children; backward: its parent) sit on
    // earlier levels, so the order is topological.  Each large
    // front's items stay together (forward: pivot tiles in order, then the
    // update tasks; backward: the gathers, then the pivot tasks from the last
    // pivot tile down); small fronts are packed into warp items of at most
    // kWarpsPerItem warps in the same order, and an open warp item is emitted
    // before any front that depends on one of its fronts.
    {
        const int ns = P.nsuper;
        std::vector<int64_t> lat(ns, 4), pf(ns, 0), pb(ns, 0);
        for (int s : P.large_list) lat[s] = 6 + 3 * (int64_t)((P.fronts[s].c + T - 1) / T);
        auto level_fronts = [&](int l, auto&& fn) {
            for (int q = P.small_ptr[l * kSmallBuckets]; q < P.small_ptr[(l + 1) * kSmallBuckets]; ++q)
                fn(P.small_list[q]);
            for (int q = P.large_ptr[l]; q < P.large_ptr[l + 1]; ++q) fn(P.large_list[q]);
        };
        for (int l = P.nlevels - 1; l >= 0; --l)  // parents first
            level_fronts(l, [&](int s) {
                const int par = P.fronts[s].parent;
                pf[s] = lat[s] + (par >= 0 ? pf[par] : 0);
            });
        for (int l = 0; l < P.nlevels; ++l)  // children first
            level_fronts(l, [&](int s) {
                int64_t h = 0;
                for (int q = P.fronts[s].child_beg; q < P.fronts[s].child_end; ++q)
                    h = std::max(h, pb[P.child[q]]);
                pb[s] = lat[s] + h;
            });
        std::vector<char> large(ns, 0);
        for (int s : P.large_list) large[s] = 1;
        const int WPI = SolveScheduleHost::kWarpsPerItem;
        std::vector<int> lev(ns, 0);
        for (int l = 0; l < P.nlevels; ++l) level_fronts(l, [&](int s) { lev[s] = l; });
        for (int dir = 0; dir < 2; ++dir) {
            const std::vector<int64_t>& pr = dir == 0 ? pf : pb;
            std::vector<int> order(ns);
            for (int s = 0; s < ns; ++s) order[s] = s;
            std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
                if (lev[a] != lev[b]) return dir == 0 ? lev[a] < lev[b] : lev[a] > lev[b];
                return pr[a] > pr[b];
            });
            std::vector<int>& it = dir == 0 ? S.fwd_items : S.bwd_items;
            std::vector<int>& wl = dir == 0 ? S.fwd_wlist : S.bwd_wlist;
            it.clear();
            wl.clear();
            std::vector<char> open(ns, 0);
            std::vector<int> cls[3];
            auto warps = [](size_t a, size_t b, size_t c) {
                return (int)(a + (b + 1) / 2 + (c + 3) / 4);
            };
            auto flush = [&]() {
                if (cls[0].empty() && cls[1].empty() && cls[2].empty()) return;
                const int off = (int)wl.size();
                for (int k = 0; k < 3; ++k)
                    for (int f : cls[k]) {
                        wl.push_back(f);
                        open[f] = 0;
                    }
                it.insert(it.end(), {SolveScheduleHost::kItemWarps, off,
                                     (int)cls[0].size() | (int)cls[1].size() << 8 |
                                         (int)cls[2].size() << 16,
                                     0});
                for (auto& v : cls) v.clear();
            };
            for (int s : order) {
                const FrontDesc& f = P.fronts[s];
                bool dep_open = false;
                if (dir == 0) {
                    for (int q = f.child_beg; q < f.child_end; ++q) dep_open |= open[P.child[q]] != 0;
                } else {
                    dep_open = f.parent >= 0 && open[f.parent];
                }
                if (dep_open) flush();
                if (large[s]) {
                    const int nt1 = (f.c + T - 1) / T, NT = front_tiles(f.m, f.c, T);
                    if (dir == 0) {
                        for (int i = 0; i < nt1; ++i)
                            it.insert(it.end(), {SolveScheduleHost::kItemTile, s, i | (1 << 16), 0});
                        const int G = std::max(1, std::min(SolveScheduleHost::kFwdGroupBlocks / nt1,
                                                           SolveScheduleHost::kFwdGroupTiles));
                        for (int i = nt1; i < NT; i += G)
                            it.insert(it.end(), {SolveScheduleHost::kItemTile, s,
                                                 i | (std::min(G, NT - i) << 16), 0});
                    } else {
                        for (int j = nt1 - 1; j >= 0; --j)
                            for (int h = 0; h < S.gather_nch[s]; ++h)
                                it.insert(it.end(),
                                          {SolveScheduleHost::kItemGather, s, j | (h << 16), 0});
                        for (int j = nt1 - 1; j >= 0; --j)
                            it.insert(it.end(), {SolveScheduleHost::kItemTile, s, j, 0});
                    }
                } else {
                    const int k = f.m > 16 ? 0 : (f.m > 8 ? 1 : 2);
                    const size_t a = cls[0].size() + (k == 0), b = cls[1].size() + (k == 1),
                                 c = cls[2].size() + (k == 2);
                    if (warps(a, b, c) > WPI) flush();
                    cls[k].push_back(s);
                    open[s] = 1;
                }
            }
            flush();
        }
    }
    S.bwd_target.assign(P.nsuper, 1);
    for (int s : P.large_list) S.bwd_target[s] = (P.fronts[s].c + T - 1) / T;
}

void build_panel_schedule(const Plan& P, int T, int PW, int CB, PanelSchedule& S) {
    S = PanelSchedule();
    const int TPP = PW / T;  // tiles per panel
    S.op_beg.assign(P.nlevels + 1, 0);
    auto tsize = [&](const FrontDesc& f, int t) {
        int nt1 = (f.c + T - 1) / T;
        if (t < nt1) return std::min(T, f.c - t * T);
        return std::min(T, f.m - (f.c + (t - nt1) * T));
    };
    for (int l = 0; l < P.nlevels; ++l) {
        S.op_beg[l] = (int)S.ops.size();
        std::vector<int> fr(P.large_list.begin() + P.large_ptr[l],
                            P.large_list.begin() + P.large_ptr[l + 1]);
        if (fr.empty()) continue;
        std::vector<std::pair<int, int>> as;
        int maxpanels = 0;
        double asm_el = 0, asm_x = 0;
        // diagonal tile t of f: factor (n^3/3), read + write its lower part,
        // write the T x T inverse
        auto potrf_cost = [&](const FrontDesc& f, int t, double& fl, double& el) {
            double nn = tsize(f, t);
            fl += nn * nn * nn / 3.0;
            el += nn * (nn + 1) + (double)T * T;
        };
        for (int s : fr) {
            const FrontDesc& f = P.fronts[s];
            as.push_back({s, (f.m + CB - 1) / CB});
            maxpanels = std::max(maxpanels, (f.c + PW - 1) / PW);
            // assembly: write the L panel and the U store, read every child's
            // update matrix; FP64 values with their source index and position
            double u = f.m - f.c;
            asm_el += (double)f.m * f.c + u * (u + 1) / 2;
            for (int h = f.child_beg; h < f.child_end; ++h) {
                const FrontDesc& g = P.fronts[P.child[h]];
                double uc = g.m - g.c;
                asm_el += uc * (uc + 1) / 2;
                asm_x += 4.0 * uc;  // relative map
            }
            asm_x += 16.0 * (f.a_end - f.a_beg);
        }
        S.ops.push_back({OP_ASSEMBLE, 0, 0, S.store.add(as, 0), 0, asm_el, asm_x});
        for (int p = 0; p < maxpanels; ++p) {
            // one launch for the whole panel: diagonal tasks first
            const int64_t toff = (int64_t)S.tasks.size() / 2;
            double fl = 0, el = 0;
            for (int t = 0; t < TPP; ++t)
                for (int s : fr) {
                    const FrontDesc& f = P.fronts[s];
                    const int nt1 = (f.c + T - 1) / T;
                    const int klo = p * TPP, khi = std::min(klo + TPP, nt1);
                    if (klo + t < khi) {
                        S.tasks.push_back(s);
                        S.tasks.push_back(klo + t);
                    }
                }
            for (int s : fr) {
                const FrontDesc& f = P.fronts[s];
                const int nt1 = (f.c + T - 1) / T, NT = front_tiles(f.m, f.c, T);
                const int klo = p * TPP, khi = std::min(klo + TPP, nt1);
                if (klo >= nt1) continue;
                for (int i = khi; i < NT; ++i) {
                    S.tasks.push_back(s);
                    S.tasks.push_back(i);
                }
                // algorithmic work: per pivot tile k its factorization, the
                // triangular solve of every row below it and the update of
                // the panel's later columns; every panel element read and
                // written once, every inverse written once
                for (int k = klo; k < khi; ++k) {
                    const double K = tsize(f, k);
                    potrf_cost(f, k, fl, el);
                    for (int i = k + 1; i < NT; ++i) fl += tsize(f, i) * K * K;
                    for (int j = k + 1; j < khi; ++j) {
                        const double rj = tsize(f, j);
                        fl += K * rj * (rj + 1);
                        for (int i = j + 1; i < NT; ++i) fl += 2.0 * K * tsize(f, i) * rj;
                    }
                    for (int i = k + 1; i < NT; ++i) el += 2.0 * tsize(f, i) * K;
                }
            }
            const int ntasks = (int)((int64_t)S.tasks.size() / 2 - toff);
            if (ntasks > 0) {
                PanelOp op{OP_PANEL, p, 0, WorkList{0, 0, 0, p}, fl, el, 0};
                op.toff = toff;
                op.ntasks = ntasks;
                op.counter = S.ncounters++;
                S.ops.push_back(op);
            }
            std::vector<std::pair<int, int>> big;
            double sfl = 0, sel = 0;
            for (int s : fr) {
                const FrontDesc& f = P.fronts[s];
                int k0 = p * PW;
                if (k0 >= f.c) continue;
                int K = std::min(PW, f.c - k0);
                int cbeg = std::min(k0 + PW, f.c);
                if (cbeg < f.m) {
                    int NB = (f.m + 127) / 128, J0 = cbeg / 128;
                    int nb = NB - J0;
                    big.push_back({s, nb * (nb + 1) / 2});
                    double tr = f.m - cbeg;
                    sfl += (double)K * tr * (tr + 1);  // lower trailing part, 2 flops per FMA
                    sel += (double)K * tr + tr * (tr + 1);  // read the panel, update the trailing part
                }
            }
            if (!big.empty()) S.ops.push_back({OP_SCHUR_TC, p, 0, S.store.add(big, p), sfl, sel, 0});
            // the tensor-core path's deferred updates (see PanelOpKind)
            std::vector<std::pair<int, int>> nxt, rest;
            double nfl = 0, nel = 0, rfl = 0, rel = 0;
            for (int s : fr) {
                const FrontDesc& f = P.fronts[s];
                const int k0 = p * PW;
                if (k0 >= f.c) continue;
                const int cbeg = std::min(k0 + PW, f.c);
                if (cbeg >= f.m) continue;
                const int NB = (f.m + 127) / 128, J0 = cbeg / 128, nb = NB - J0;
                const double tr = f.m - cbeg;
                const bool hasnext = cbeg < f.c;
                if (p % 2 == 0 && hasnext) {
                    // the next panel's columns [cbeg, min(cbeg + 256, c)): two
                    // tile columns
                    const double K = std::min(PW, f.c - k0);
                    const double w = std::min(PW, f.c - cbeg);
                    const double area = w * tr - w * (w - 1) / 2;
                    nxt.push_back({s, nb + std::max(nb - 1, 0)});
                    nfl += 2.0 * K * area;
                    nel += K * (tr + w) + 2.0 * area;
                } else {
                    const int np = p % 2 == 1 ? 2 : 1;
                    const double K = std::min(np * PW, f.c - (p - np + 1) * PW);
                    rest.push_back({s, nb * (nb + 1) / 2});
                    rfl += K * tr * (tr + 1);
                    rel += K * tr + tr * (tr + 1);
                }
            }
            if (!nxt.empty())
                S.ops.push_back({OP_SCHUR_NEXT, p, 1, S.store.add(nxt, p), nfl, nel, 0});
            if (!rest.empty())
                S.ops.push_back({OP_SCHUR_REST, p, p % 2 == 1 ? 2 : 1, S.store.add(rest, p), rfl,
                                 rel, 0});
        }
    }
    S.op_beg[P.nlevels] = (int)S.ops.size();
    S.nflags = (P.dinv_total + (int64_t)T * T - 1) / ((int64_t)T * T);
}

std::vector<int> front_levels(const Plan& P) {
    std::vector<int> level(P.nsuper, 0);
    for (int s = 0; s < P.nsuper; ++s)
        for (int h = P.fronts[s].child_beg; h < P.fronts[s].child_end; ++h)
            level[s] = std::max(level[s], level[P.child[h]] + 1);
    return level;
}

}  // namespace mdgpu
