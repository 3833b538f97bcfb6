// Host symbolic analysis (see symbolic.hpp).  The orderings and trees must be
// identical to the reference's, so each algorithm below takes the same steps
// in the same order as the routine it is named after; ties, hash buckets and
// list orders all matter for the resulting permutation.
#include "symbolic.hpp"

#include <algorithm>
#include <cmath>
#include <stdexcept>

namespace mdgpu {

// ---------------------------------------------------------------------------
// sparse helpers
// ---------------------------------------------------------------------------

static void prefix_counts(std::vector<int>& ptr, std::vector<int>& cnt) {
    // ptr[k] = sum cnt[0..k-1]; cnt[k] <- ptr[k]  (cs_cumsum, cs.cpp:273)
    int n = (int)cnt.size();
    ptr.assign(n + 1, 0);
    int run = 0;
    for (int k = 0; k < n; ++k) {
        ptr[k] = run;
        run += cnt[k];
        cnt[k] = ptr[k];
    }
    ptr[n] = run;
}

SparseCol transpose(const SparseCol& A, bool values) {
    // cs_transpose, cs.cpp:407
    SparseCol T;
    T.nrows = A.ncols;
    T.ncols = A.nrows;
    int nz = A.nnz();
    std::vector<int> next(A.nrows, 0);
    for (int p = 0; p < nz; ++p) next[A.rowidx[p]]++;
    prefix_counts(T.colptr, next);
    T.rowidx.resize(nz);
    bool v = values && A.has_values();
    if (v) T.val.resize(nz);
    for (int j = 0; j < A.ncols; ++j) {
        for (int p = A.colptr[j]; p < A.colptr[j + 1]; ++p) {
            int q = next[A.rowidx[p]]++;
            T.rowidx[q] = j;
            if (v) T.val[q] = A.val[p];
        }
    }
    return T;
}

// union of two matrices' patterns with values summed; column j lists A's rows
// in stored order followed by B's rows that A lacks (cs_add, cs.cpp:510)
static SparseCol add_patterns(const SparseCol& A, const SparseCol& B, bool values) {
    SparseCol C;
    C.nrows = A.nrows;
    C.ncols = B.ncols;
    C.colptr.assign(C.ncols + 1, 0);
    C.rowidx.reserve(A.nnz() + B.nnz());
    bool v = values && A.has_values() && B.has_values();
    std::vector<int> seen(C.nrows, 0);
    std::vector<double> acc(v ? C.nrows : 0);
    for (int j = 0; j < C.ncols; ++j) {
        int start = (int)C.rowidx.size();
        C.colptr[j] = start;
        for (const SparseCol* S : {&A, &B}) {
            for (int p = S->colptr[j]; p < S->colptr[j + 1]; ++p) {
                int i = S->rowidx[p];
                if (seen[i] < j + 1) {
                    seen[i] = j + 1;
                    C.rowidx.push_back(i);
                    if (v) acc[i] = S->val[p];
                } else if (v) {
                    acc[i] += S->val[p];
                }
            }
        }
        if (v)
            for (int p = start; p < (int)C.rowidx.size(); ++p) C.val.push_back(acc[C.rowidx[p]]);
    }
    C.colptr[C.ncols] = (int)C.rowidx.size();
    return C;
}

static void remove_diagonal(SparseCol& A) {
    // cs_fkeep with the off-diagonal predicate, cs.cpp:595
    int w = 0;
    bool v = A.has_values();
    for (int j = 0; j < A.ncols; ++j) {
        int p = A.colptr[j], end = A.colptr[j + 1];
        A.colptr[j] = w;
        for (; p < end; ++p) {
            if (A.rowidx[p] == j) continue;
            if (v) A.val[w] = A.val[p];
            A.rowidx[w++] = A.rowidx[p];
        }
    }
    A.colptr[A.ncols] = w;
    A.rowidx.resize(w);
    if (v) A.val.resize(w);
}

SparseCol symmetric_from_lower(const SparseCol& lower) {
    SparseCol up = transpose(lower, true);
    remove_diagonal(up);
    return add_patterns(lower, up, true);
}

SparseCol permute_upper(const SparseCol& A, const std::vector<int>& pinv) {
    // cs_symperm, cs.cpp:1005
    int n = A.ncols;
    SparseCol C;
    C.nrows = C.ncols = n;
    std::vector<int> cnt(n, 0);
    auto newidx = [&](int i) { return pinv.empty() ? i : pinv[i]; };
    for (int j = 0; j < n; ++j)
        for (int p = A.colptr[j]; p < A.colptr[j + 1]; ++p) {
            int i = A.rowidx[p];
            if (i > j) continue;
            cnt[std::max(newidx(i), newidx(j))]++;
        }
    prefix_counts(C.colptr, cnt);
    C.rowidx.resize(C.colptr[n]);
    bool v = A.has_values();
    if (v) C.val.resize(C.colptr[n]);
    for (int j = 0; j < n; ++j) {
        int j2 = newidx(j);
        for (int p = A.colptr[j]; p < A.colptr[j + 1]; ++p) {
            int i = A.rowidx[p];
            if (i > j) continue;
            int i2 = newidx(i);
            int q = cnt[std::max(i2, j2)]++;
            C.rowidx[q] = std::min(i2, j2);
            if (v) C.val[q] = A.val[p];
        }
    }
    return C;
}

// ---------------------------------------------------------------------------
// approximate minimum degree (quotient-graph elimination, cs.cpp:645-991)
// ---------------------------------------------------------------------------

namespace {

inline int flip(int i) { return -i - 2; }

// Depth-first postorder of the subtree rooted at `root` using `head`/`next`
// child lists that are consumed (cs_tdfs, cs.cpp:456).
int dfs_postorder(int root, int k, std::vector<int>& head, const std::vector<int>& next,
                  int* out, int* stack) {
    int top = 0;
    stack[0] = root;
    while (top >= 0) {
        int v = stack[top];
        int c = head[v];
        if (c == -1) {
            --top;
            out[k++] = v;
        } else {
            head[v] = next[c];
            stack[++top] = c;
        }
    }
    return k;
}

class MinDegree {
   public:
    explicit MinDegree(const SparseCol& upper) : n_(upper.ncols) {
        // quotient graph starts as A + A' without the diagonal
        SparseCol at = transpose(upper, false);
        SparseCol pat = add_patterns(upper, at, false);
        remove_diagonal(pat);
        adjptr_ = pat.colptr;
        used_ = adjptr_[n_];
        capacity_ = used_ + used_ / 5 + 2 * n_;  // elbow room (cs.cpp:691)
        adj_ = pat.rowidx;
        adj_.resize(std::max(capacity_, 1));
        double d = 10 * std::sqrt((double)n_);
        dense_ = (int)(16 > d ? 16 : d);
        dense_ = std::min(n_ - 2, dense_);
        int m = n_ + 1;
        len_.assign(m, 0);
        nv_.assign(m, 1);
        next_.assign(m, -1);
        head_.assign(m, -1);
        elen_.assign(m, 0);
        degree_.assign(m, 0);
        w_.assign(m, 1);
        hhead_.assign(m, -1);
        last_.assign(m, -1);
    }

    std::vector<int> run() {
        initialize();
        while (eliminated_ < n_) {
            int k = pick_pivot();
            int elenk = elen_[k];
            int nvk = nv_[k];
            eliminated_ += nvk;
            if (elenk > 0 && used_ + mindeg_ >= capacity_) compact();
            form_element(k, elenk, nvk);
            measure_set_differences();
            update_degrees(k);
            detect_indistinguishable();
            finish_element(k, elenk);
        }
        return postorder();
    }

   private:
    int n_;
    int used_ = 0, capacity_ = 0, dense_ = 0;
    int lemax_ = 0, mindeg_ = 0, eliminated_ = 0, mark_ = 0;
    int dk_ = 0, nvk_ = 0, pk1_ = 0, pk2_ = 0;
    std::vector<int> adjptr_, adj_;
    std::vector<int> len_, nv_, next_, head_, elen_, degree_, w_, hhead_, last_;

    // cs_wclear, cs.cpp:630; the sum wraps exactly as 32-bit arithmetic does
    int reset_if_needed(int mark) {
        int sum = (int)((unsigned)mark + (unsigned)lemax_);
        if (mark < 2 || sum < 0) {
            for (int k = 0; k < n_; ++k)
                if (w_[k] != 0) w_[k] = 1;
            mark = 2;
        }
        return mark;
    }

    void list_insert(int i, int d) {
        if (head_[d] != -1) last_[head_[d]] = i;
        next_[i] = head_[d];
        head_[d] = i;
    }

    void initialize() {
        for (int k = 0; k < n_; ++k) len_[k] = adjptr_[k + 1] - adjptr_[k];
        len_[n_] = 0;
        for (int i = 0; i <= n_; ++i) degree_[i] = len_[i];
        mark_ = reset_if_needed(0);
        elen_[n_] = -2;
        adjptr_[n_] = -1;
        w_[n_] = 0;
        for (int i = 0; i < n_; ++i) {
            int d = degree_[i];
            if (d == 0) {  // isolated node: eliminated immediately
                elen_[i] = -2;
                ++eliminated_;
                adjptr_[i] = -1;
                w_[i] = 0;
            } else if (d > dense_) {  // dense node: absorbed into the placeholder n
                nv_[i] = 0;
                elen_[i] = -1;
                ++eliminated_;
                adjptr_[i] = flip(n_);
                nv_[n_]++;
            } else {
                list_insert(i, d);
            }
        }
    }

    int pick_pivot() {
        int k = -1;
        for (; mindeg_ < n_ && (k = head_[mindeg_]) == -1; ++mindeg_) {
        }
        if (next_[k] != -1) last_[next_[k]] = -1;
        head_[mindeg_] = next_[k];
        return k;
    }

    void compact() {
        // garbage collection of the adjacency store (cs.cpp:753-773)
        for (int j = 0; j < n_; ++j) {
            int p = adjptr_[j];
            if (p >= 0) {
                adjptr_[j] = adj_[p];
                adj_[p] = flip(j);
            }
        }
        int q = 0;
        for (int p = 0; p < used_;) {
            int j = flip(adj_[p++]);
            if (j >= 0) {
                adj_[q] = adjptr_[j];
                adjptr_[j] = q++;
                for (int t = 0; t < len_[j] - 1; ++t) adj_[q++] = adj_[p++];
            }
        }
        used_ = q;
    }

    void unlink(int i) {
        if (next_[i] != -1) last_[next_[i]] = last_[i];
        if (last_[i] != -1)
            next_[last_[i]] = next_[i];
        else
            head_[degree_[i]] = next_[i];
    }

    void form_element(int k, int elenk, int nvk) {
        // Lk = union of the pivot's variables and its elements' variables
        // (cs.cpp:775-821)
        dk_ = 0;
        nvk_ = nvk;
        nv_[k] = -nvk;
        int p = adjptr_[k];
        pk1_ = (elenk == 0) ? p : used_;
        pk2_ = pk1_;
        for (int k1 = 1; k1 <= elenk + 1; ++k1) {
            int e, pj, ln;
            if (k1 > elenk) {
                e = k;
                pj = p;
                ln = len_[k] - elenk;
            } else {
                e = adj_[p++];
                pj = adjptr_[e];
                ln = len_[e];
            }
            for (int k2 = 1; k2 <= ln; ++k2) {
                int i = adj_[pj++];
                int nvi = nv_[i];
                if (nvi <= 0) continue;
                dk_ += nvi;
                nv_[i] = -nvi;
                adj_[pk2_++] = i;
                unlink(i);
            }
            if (e != k) {
                adjptr_[e] = flip(k);
                w_[e] = 0;
            }
        }
        if (elenk != 0) used_ = pk2_;
        degree_[k] = dk_;
        adjptr_[k] = pk1_;
        len_[k] = pk2_ - pk1_;
        elen_[k] = -2;
    }

    void measure_set_differences() {
        // w[e] - mark = |Le \ Lk| for elements adjacent to Lk (cs.cpp:823-842)
        mark_ = reset_if_needed(mark_);
        for (int pk = pk1_; pk < pk2_; ++pk) {
            int i = adj_[pk];
            int eln = elen_[i];
            if (eln <= 0) continue;
            int nvi = -nv_[i];
            int base = mark_ - nvi;
            for (int p = adjptr_[i]; p <= adjptr_[i] + eln - 1; ++p) {
                int e = adj_[p];
                if (w_[e] >= mark_)
                    w_[e] -= nvi;
                else if (w_[e] != 0)
                    w_[e] = degree_[e] + base;
            }
        }
    }

    void update_degrees(int k) {
        // approximate external degrees, pruning and hashing (cs.cpp:844-905)
        for (int pk = pk1_; pk < pk2_; ++pk) {
            int i = adj_[pk];
            int p1 = adjptr_[i];
            int p2 = p1 + elen_[i] - 1;
            int pn = p1;
            unsigned int h = 0;
            int d = 0;
            for (int p = p1; p <= p2; ++p) {
                int e = adj_[p];
                if (w_[e] == 0) continue;
                int dext = w_[e] - mark_;
                if (dext > 0) {
                    d += dext;
                    adj_[pn++] = e;
                    h += e;
                } else {  // aggressive absorption of e into k
                    adjptr_[e] = flip(k);
                    w_[e] = 0;
                }
            }
            elen_[i] = pn - p1 + 1;
            int p3 = pn;
            int p4 = p1 + len_[i];
            for (int p = p2 + 1; p < p4; ++p) {
                int j = adj_[p];
                int nvj = nv_[j];
                if (nvj <= 0) continue;
                d += nvj;
                adj_[pn++] = j;
                h += j;
            }
            if (d == 0) {  // mass elimination
                adjptr_[i] = flip(k);
                int nvi = -nv_[i];
                dk_ -= nvi;
                nvk_ += nvi;
                eliminated_ += nvi;
                nv_[i] = 0;
                elen_[i] = -1;
            } else {
                degree_[i] = std::min(degree_[i], d);
                adj_[pn] = adj_[p3];
                adj_[p3] = adj_[p1];
                adj_[p1] = k;
                len_[i] = pn - p1 + 1;
                h %= (unsigned)n_;
                next_[i] = hhead_[h];
                hhead_[h] = i;
                last_[i] = (int)h;
            }
        }
        degree_[k] = dk_;
        lemax_ = std::max(lemax_, dk_);
        mark_ = reset_if_needed((int)((unsigned)mark_ + (unsigned)lemax_));
    }

    void detect_indistinguishable() {
        // merge variables with identical adjacency (cs.cpp:907-943)
        for (int pk = pk1_; pk < pk2_; ++pk) {
            int i = adj_[pk];
            if (nv_[i] >= 0) continue;
            unsigned int h = (unsigned)last_[i];
            i = hhead_[h];
            hhead_[h] = -1;
            for (; i != -1 && next_[i] != -1; i = next_[i], ++mark_) {
                int ln = len_[i];
                int eln = elen_[i];
                for (int p = adjptr_[i] + 1; p <= adjptr_[i] + ln - 1; ++p) w_[adj_[p]] = mark_;
                int jlast = i;
                for (int j = next_[i]; j != -1;) {
                    bool same = (len_[j] == ln) && (elen_[j] == eln);
                    for (int p = adjptr_[j] + 1; same && p <= adjptr_[j] + ln - 1; ++p)
                        if (w_[adj_[p]] != mark_) same = false;
                    if (same) {
                        adjptr_[j] = flip(i);
                        nv_[i] += nv_[j];
                        nv_[j] = 0;
                        elen_[j] = -1;
                        j = next_[j];
                        next_[jlast] = j;
                    } else {
                        jlast = j;
                        j = next_[j];
                    }
                }
            }
        }
    }

    void finish_element(int k, int elenk) {
        // restore nv, compute external degrees, refill degree lists (cs.cpp:945-966)
        int pw = pk1_;
        for (int pk = pk1_; pk < pk2_; ++pk) {
            int i = adj_[pk];
            int nvi = -nv_[i];
            if (nvi <= 0) continue;
            nv_[i] = nvi;
            int d = degree_[i] + dk_ - nvi;
            d = std::min(d, n_ - eliminated_ - nvi);
            if (head_[d] != -1) last_[head_[d]] = i;
            next_[i] = head_[d];
            last_[i] = -1;
            head_[d] = i;
            mindeg_ = std::min(mindeg_, d);
            degree_[i] = d;
            adj_[pw++] = i;
        }
        nv_[k] = nvk_;
        if ((len_[k] = pw - pk1_) == 0) {
            adjptr_[k] = -1;
            w_[k] = 0;
        }
        if (elenk != 0) used_ = pw;
    }

    std::vector<int> postorder() {
        // postorder of the assembly tree (cs.cpp:969-989)
        std::vector<int> P(n_ + 1);
        for (int i = 0; i < n_; ++i) adjptr_[i] = flip(adjptr_[i]);
        for (int j = 0; j <= n_; ++j) head_[j] = -1;
        for (int j = n_; j >= 0; --j) {
            if (nv_[j] > 0) continue;
            next_[j] = head_[adjptr_[j]];
            head_[adjptr_[j]] = j;
        }
        for (int e = n_; e >= 0; --e) {
            if (nv_[e] <= 0) continue;
            if (adjptr_[e] != -1) {
                next_[e] = head_[adjptr_[e]];
                head_[adjptr_[e]] = e;
            }
        }
        for (int k = 0, i = 0; i <= n_; ++i)
            if (adjptr_[i] == -1) k = dfs_postorder(i, k, head_, next_, P.data(), w_.data());
        P.resize(n_);
        return P;
    }
};

}  // namespace

std::vector<int> amd_order(const SparseCol& upper) { return MinDegree(upper).run(); }

// ---------------------------------------------------------------------------
// elimination tree, postorder, column counts
// ---------------------------------------------------------------------------

std::vector<int> elimination_tree(const SparseCol& A) {
    // cs_etree(A, 0), cs.cpp:480: path-compressed ancestor walk over triu(A)
    int n = A.ncols;
    std::vector<int> parent(n, -1), anc(n, -1);
    for (int k = 0; k < n; ++k) {
        for (int p = A.colptr[k]; p < A.colptr[k + 1]; ++p) {
            for (int i = A.rowidx[p]; i != -1 && i < k;) {
                int up = anc[i];
                anc[i] = k;
                if (up == -1) parent[i] = k;
                i = up;
            }
        }
    }
    return parent;
}

std::vector<int> tree_postorder(const std::vector<int>& parent) {
    int n = (int)parent.size();
    std::vector<int> head(n, -1), next(n, -1), stack(n), post(n);
    for (int j = n - 1; j >= 0; --j) {
        if (parent[j] == -1) continue;
        next[j] = head[parent[j]];
        head[parent[j]] = j;
    }
    int k = 0;
    for (int j = 0; j < n; ++j)
        if (parent[j] == -1) k = dfs_postorder(j, k, head, next, post.data(), stack.data());
    return post;
}

std::vector<int> column_counts(const SparseCol& A, const std::vector<int>& parent,
                               const std::vector<int>& post) {
    // cs_counts(A, parent, post, 0), cs.cpp:338: skeleton-matrix leaves and
    // least common ancestors (cs_leaf, cs.cpp:385)
    int n = A.ncols;
    SparseCol AT = transpose(A, false);
    std::vector<int> anc(n), maxfirst(n, -1), prevleaf(n, -1), first(n, -1), cc(n);
    for (int k = 0; k < n; ++k) {
        int j = post[k];
        cc[j] = (first[j] == -1) ? 1 : 0;
        for (; j != -1 && first[j] == -1; j = parent[j]) first[j] = k;
    }
    for (int i = 0; i < n; ++i) anc[i] = i;
    for (int k = 0; k < n; ++k) {
        int j = post[k];
        if (parent[j] != -1) cc[parent[j]]--;
        for (int p = AT.colptr[j]; p < AT.colptr[j + 1]; ++p) {
            int i = AT.rowidx[p];
            if (i <= j || first[j] <= maxfirst[i]) continue;
            maxfirst[i] = first[j];
            int jprev = prevleaf[i];
            prevleaf[i] = j;
            cc[j]++;
            if (jprev == -1) continue;
            int q = jprev;
            while (q != anc[q]) q = anc[q];
            for (int s = jprev; s != q;) {
                int sp = anc[s];
                anc[s] = q;
                s = sp;
            }
            cc[q]--;
        }
        if (parent[j] != -1) anc[j] = parent[j];
    }
    for (int j = 0; j < n; ++j)
        if (parent[j] != -1) cc[parent[j]] += cc[j];
    return cc;
}

// ---------------------------------------------------------------------------
// assembly trees (etree.cpp)
// ---------------------------------------------------------------------------

namespace {

struct TreeNode {
    int first = 0, ncols = 1, rows = 0, zeros = 0;
    std::vector<int> kids;     // child ids
    std::vector<int> members;  // member columns (relaxed tree)
};

// children lists in ascending column order (GetETree, etree.cpp:26-39)
std::vector<std::vector<int>> children_of(const std::vector<int>& parent) {
    std::vector<std::vector<int>> ch(parent.size());
    for (int i = 0; i < (int)parent.size(); ++i)
        if (parent[i] != -1) ch[parent[i]].push_back(i);
    return ch;
}

AssemblyTree flatten(const std::vector<TreeNode>& nodes, int count) {
    AssemblyTree t;
    t.first_col.resize(count);
    t.ncols.resize(count);
    t.child_ptr.assign(count + 1, 0);
    for (int s = 0; s < count; ++s) {
        t.first_col[s] = nodes[s].first;
        t.ncols[s] = nodes[s].ncols;
        t.child_ptr[s + 1] = t.child_ptr[s] + (int)nodes[s].kids.size();
    }
    t.child.reserve(t.child_ptr[count]);
    for (int s = 0; s < count; ++s)
        t.child.insert(t.child.end(), nodes[s].kids.begin(), nodes[s].kids.end());
    return t;
}

}  // namespace

AssemblyTree nodal_tree(const std::vector<int>& parent, const std::vector<int>& post) {
    int n = (int)parent.size();
    std::vector<int> pos(n);
    for (int k = 0; k < n; ++k) pos[post[k]] = k;
    auto ch = children_of(parent);
    std::vector<TreeNode> nodes(n);
    for (int k = 0; k < n; ++k) {
        int j = post[k];
        nodes[k].first = j;
        for (int c : ch[j]) nodes[k].kids.push_back(pos[c]);
    }
    return flatten(nodes, n);
}

AssemblyTree super_tree(const std::vector<int>& parent, const std::vector<int>& post,
                        const std::vector<int>& count) {
    // GetSuperETree (etree.cpp:50-118): walk the columns in postorder; a column
    // whose last (largest) child is the previous column with exactly one more
    // row absorbs that child's supernode.  Children are kept in visiting order.
    int n = (int)parent.size();
    auto ch = children_of(parent);
    std::vector<TreeNode> out;
    out.reserve(n);
    std::vector<int> stack;
    stack.reserve(n);
    for (int k = 0; k < n; ++k) {
        int j = post[k];
        const auto& kids = ch[j];
        int nk = (int)kids.size();
        bool absorb = nk >= 1 && count[kids.back()] == count[j] + 1 && kids.back() == j - 1;
        if (!absorb) {
            TreeNode t;
            t.first = j;
            t.ncols = 1;
            t.rows = count[j];
            t.kids.resize(nk);
            for (int i = nk - 1; i >= 0; --i) {
                t.kids[i] = stack.back();
                stack.pop_back();
            }
            out.push_back(std::move(t));
            stack.push_back((int)out.size() - 1);
        } else {
            int sid = stack.back();  // the chain being extended = the list's last entry
            stack.pop_back();
            if (sid != (int)out.size() - 1) throw std::logic_error("supernode chain order");
            TreeNode& t = out[sid];
            std::vector<int> grandkids = std::move(t.kids);
            t.kids.assign(nk - 1, 0);
            for (int i = nk - 2; i >= 0; --i) {
                t.kids[i] = stack.back();
                stack.pop_back();
            }
            t.kids.insert(t.kids.end(), grandkids.begin(), grandkids.end());
            t.ncols += 1;
            t.rows -= 1;
            stack.push_back(sid);
        }
    }
    return flatten(out, (int)out.size());
}

AssemblyTree relaxed_tree(const std::vector<int>& parent, const std::vector<int>& post,
                          std::vector<int>& count, int max_zeros, std::vector<int>& perm) {
    // GetRelaxedETree (etree.cpp:194-342) over the nodal tree.
    int n = (int)parent.size();
    auto ch = children_of(parent);
    std::vector<int> rows0(count);  // node rows are fixed when the nodal tree is built
    std::vector<TreeNode> R(n);
    std::vector<char> absorbed(n, 0);
    std::vector<int> stack;
    stack.reserve(n);
    for (int k = 0; k < n; ++k) {
        int j = post[k];
        int nk = (int)ch[j].size();
        std::vector<int> kids(stack.end() - nk, stack.end());
        std::vector<char> take(nk, 0);
        TreeNode& r = R[j];
        r.first = j;
        r.ncols = 1;
        r.rows = rows0[j];
        r.members = {j};
        int zeros = 0, cols = 1;
        for (;;) {
            int best = -1, best_z = -1;
            for (int h = 0; h < nk; ++h) {
                const TreeNode& c = R[kids[h]];
                int z = (r.rows + cols - c.rows) * c.ncols + c.zeros;
                if (!take[h] && z <= max_zeros && (best_z == -1 || z < best_z)) {
                    best_z = z;
                    best = h;
                }
            }
            if (best < 0) break;
            take[best] = 1;
            const TreeNode& c = R[kids[best]];
            zeros += best_z;
            cols += c.ncols;
            for (int m : c.members) count[m] += (best_z - c.zeros) / c.ncols;
        }
        r.zeros = zeros;
        for (int h = 0; h < nk; ++h) {
            TreeNode& c = R[kids[h]];
            if (!take[h]) {
                r.kids.push_back(kids[h]);
            } else {
                absorbed[kids[h]] = 1;
                r.members.insert(r.members.end(), c.members.begin(), c.members.end());
                r.kids.insert(r.kids.end(), c.kids.begin(), c.kids.end());
            }
        }
        r.ncols = (int)r.members.size();
        for (int m : r.members) r.first = std::min(r.first, m);
        // selection sort of the members by their (updated) counts, etree.cpp:180
        auto& a = r.members;
        for (int i = 0; i < (int)a.size(); ++i) {
            int x = -1;
            for (int t = i; t < (int)a.size(); ++t)
                if (x == -1 || count[a[t]] < count[a[x]]) x = t;
            std::swap(a[x], a[i]);
        }
        stack.resize(stack.size() - nk);
        stack.push_back(j);
    }
    // renumber by a depth-first walk from the last root (etree.cpp:165-178)
    perm.assign(n, 0);
    std::vector<int> pos(n, -1), order;
    order.reserve(n);
    std::vector<std::pair<int, int>> st;
    st.push_back({stack.back(), 0});
    int c = 0;
    std::vector<TreeNode> out;
    while (!st.empty()) {
        auto& [v, it] = st.back();
        if (it < (int)R[v].kids.size()) {
            int kid = R[v].kids[it++];
            st.push_back({kid, 0});
        } else {
            int vv = v;
            st.pop_back();
            pos[vv] = (int)out.size();
            TreeNode t = R[vv];
            t.first = c;
            for (int i = t.ncols - 1; i >= 0; --i) perm[c++] = t.members[i];
            out.push_back(std::move(t));
        }
    }
    for (auto& t : out)
        for (int& kid : t.kids) kid = pos[kid];
    return flatten(out, (int)out.size());
}

// ---------------------------------------------------------------------------
// driver (mdgpu.cu:1745-1875)
// ---------------------------------------------------------------------------

int analyze(int n, const int* Ap, const int* Ai, const double* /*Ax*/, bool use_amd, TreeKind kind,
            int relax_zeros, Symbolic& S) {
    S = Symbolic();
    S.n = n;
    // The value channel carries each entry's index in the caller's arrays, so
    // the numeric phase can read the caller's values in any ordering.
    SparseCol low;
    low.nrows = low.ncols = n;
    low.colptr.assign(Ap, Ap + n + 1);
    low.rowidx.assign(Ai, Ai + Ap[n]);
    low.val.resize(Ap[n]);
    for (int p = 0; p < Ap[n]; ++p) low.val[p] = (double)p;

    if (use_amd) {
        SparseCol up = transpose(low, true);
        S.perm = amd_order(up);
        std::vector<int> pinv(n);
        for (int k = 0; k < n; ++k) pinv[S.perm[k]] = k;
        SparseCol upp = permute_upper(up, pinv);
        low = transpose(upp, true);
    }
    SparseCol full = symmetric_from_lower(low);
    S.parent = elimination_tree(full);
    S.post = tree_postorder(S.parent);
    S.count0 = column_counts(full, S.parent, S.post);
    S.count = S.count0;
    int roots = 0;
    for (int p : S.parent) roots += (p == -1);
    if (roots != 1) return -1;  // GetETree requires a single tree (etree.cpp:27-31)

    if (kind == TreeKind::Relaxed) {
        std::vector<int> rp;
        S.tree = relaxed_tree(S.parent, S.post, S.count, relax_zeros, rp);
        std::vector<int> irp(n);
        for (int k = 0; k < n; ++k) irp[rp[k]] = k;
        SparseCol up = transpose(low, true);
        SparseCol upp = permute_upper(up, irp);
        low = transpose(upp, true);
        std::vector<int> c2(n), p2(n);
        for (int k = 0; k < n; ++k) {
            c2[k] = S.count[rp[k]];
            p2[k] = S.perm.empty() ? rp[k] : S.perm[rp[k]];
        }
        S.count = c2;
        S.perm = p2;
        S.relax_perm = rp;
    } else if (kind == TreeKind::Super) {
        S.tree = super_tree(S.parent, S.post, S.count);
    } else {
        S.tree = nodal_tree(S.parent, S.post);
    }
    S.lower_src.resize(low.nnz());
    for (int p = 0; p < low.nnz(); ++p) S.lower_src[p] = (int)low.val[p];
    low.val.clear();
    S.lower = std::move(low);
    S.Lp.assign(n + 1, 0);
    for (int j = 0; j < n; ++j) S.Lp[j + 1] = S.Lp[j] + S.count[j];
    return 0;
}

}  // namespace mdgpu
