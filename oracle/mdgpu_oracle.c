/*
 * mdgpu oracle -- CPU restatement of the reference's multifrontal Cholesky path.
 *
 * TEST INFRASTRUCTURE ONLY (the checker, never the product).  Every routine
 * restates one reference routine, cited by file:line; loop orders of the
 * reference's f2c BLAS branches are kept so that rounding matches.  The
 * outputs are pinned against the reference itself through tests/golden/.
 */
#include "mdgpu_oracle.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------------ */
/* compressed-column helpers (CSparse semantics, cs.cpp)                     */
/* ------------------------------------------------------------------------ */

typedef struct {
    int m, n, nzmax;
    int *p, *i;
    double *x;
} ccol;

static void *xmalloc(size_t n, size_t sz) {
    void *p = malloc((n > 0 ? n : 1) * sz);
    if (!p) {
        fprintf(stderr, "oracle: out of memory\n");
        abort();
    }
    return p;
}
static void *xcalloc(size_t n, size_t sz) {
    void *p = calloc(n > 0 ? n : 1, sz);
    if (!p) {
        fprintf(stderr, "oracle: out of memory\n");
        abort();
    }
    return p;
}

static ccol *ccol_new(int m, int n, int nzmax, int values) {
    ccol *A = (ccol *)xcalloc(1, sizeof(ccol));
    A->m = m;
    A->n = n;
    A->nzmax = nzmax > 1 ? nzmax : 1;
    A->p = (int *)xmalloc(n + 1, sizeof(int));
    A->i = (int *)xmalloc(A->nzmax, sizeof(int));
    A->x = values ? (double *)xmalloc(A->nzmax, sizeof(double)) : NULL;
    return A;
}
static void ccol_free(ccol *A) {
    if (!A) return;
    free(A->p);
    free(A->i);
    free(A->x);
    free(A);
}

/* p[0..n] = running sum of c[0..n-1]; c <- p[0..n-1]   (cs_cumsum, cs.cpp:273) */
static void running_sum(int *p, int *c, int n) {
    int nz = 0;
    for (int k = 0; k < n; k++) {
        p[k] = nz;
        nz += c[k];
        c[k] = p[k];
    }
    p[n] = nz;
}

/* C = A'  (cs_transpose, cs.cpp:407-429) */
static ccol *ccol_transpose(const ccol *A, int values) {
    int m = A->m, n = A->n;
    int nnz = A->p[n];
    ccol *C = ccol_new(n, m, nnz, values && A->x);
    int *cnt = (int *)xcalloc(m, sizeof(int));
    for (int p = 0; p < nnz; p++) cnt[A->i[p]]++;
    running_sum(C->p, cnt, m);
    for (int j = 0; j < n; j++) {
        for (int p = A->p[j]; p < A->p[j + 1]; p++) {
            int q = cnt[A->i[p]]++;
            C->i[q] = j;
            if (C->x) C->x[q] = A->x[p];
        }
    }
    free(cnt);
    return C;
}

/* C = alpha A + beta B  (cs_add + cs_scatter, cs.cpp:510-592): column j of C
 * lists A(:,j)'s rows in stored order, then B(:,j)'s rows not yet present. */
static ccol *ccol_add(const ccol *A, const ccol *B, double alpha, double beta) {
    int m = A->m, n = B->n;
    int values = A->x && B->x;
    ccol *C = ccol_new(m, n, A->p[A->n] + B->p[n], values);
    int *mark = (int *)xcalloc(m, sizeof(int));
    double *acc = values ? (double *)xmalloc(m, sizeof(double)) : NULL;
    int nz = 0;
    for (int j = 0; j < n; j++) {
        C->p[j] = nz;
        const ccol *S[2] = {A, B};
        double sc[2] = {alpha, beta};
        for (int s = 0; s < 2; s++) {
            for (int p = S[s]->p[j]; p < S[s]->p[j + 1]; p++) {
                int i = S[s]->i[p];
                if (mark[i] < j + 1) {
                    mark[i] = j + 1;
                    C->i[nz++] = i;
                    if (acc) acc[i] = sc[s] * S[s]->x[p];
                } else if (acc) {
                    acc[i] += sc[s] * S[s]->x[p];
                }
            }
        }
        if (values)
            for (int p = C->p[j]; p < nz; p++) C->x[p] = acc[C->i[p]];
    }
    C->p[n] = nz;
    free(mark);
    free(acc);
    return C;
}

/* drop diagonal entries in place  (cs_fkeep with cs_diag, cs.cpp:595-617,642) */
static void ccol_drop_diag(ccol *A) {
    int nz = 0;
    for (int j = 0; j < A->n; j++) {
        int p = A->p[j], end = A->p[j + 1];
        A->p[j] = nz;
        for (; p < end; p++) {
            if (A->i[p] != j) {
                if (A->x) A->x[nz] = A->x[p];
                A->i[nz++] = A->i[p];
            }
        }
    }
    A->p[A->n] = nz;
}

/* C = A(p,p), upper part stored, given pinv  (cs_symperm, cs.cpp:1005-1041) */
static ccol *ccol_symperm_upper(const ccol *A, const int *pinv, int values) {
    int n = A->n;
    ccol *C = ccol_new(n, n, A->p[n], values && A->x);
    int *cnt = (int *)xcalloc(n, sizeof(int));
    for (int j = 0; j < n; j++) {
        int j2 = pinv ? pinv[j] : j;
        for (int p = A->p[j]; p < A->p[j + 1]; p++) {
            int i = A->i[p];
            if (i > j) continue;
            int i2 = pinv ? pinv[i] : i;
            cnt[i2 > j2 ? i2 : j2]++;
        }
    }
    running_sum(C->p, cnt, n);
    for (int j = 0; j < n; j++) {
        int j2 = pinv ? pinv[j] : j;
        for (int p = A->p[j]; p < A->p[j + 1]; p++) {
            int i = A->i[p];
            if (i > j) continue;
            int i2 = pinv ? pinv[i] : i;
            int q = cnt[i2 > j2 ? i2 : j2]++;
            C->i[q] = i2 < j2 ? i2 : j2;
            if (C->x) C->x[q] = A->x[p];
        }
    }
    free(cnt);
    return C;
}

/* full symmetric A from its lower triangle  (make_sym, mdgpu.cu:1630-1638) */
static ccol *ccol_sym_from_lower(const ccol *L) {
    ccol *T = ccol_transpose(L, 1);
    ccol_drop_diag(T);
    ccol *C = ccol_add(L, T, 1, 1);
    ccol_free(T);
    return C;
}

static ccol *ccol_wrap(int n, const int *Ap, const int *Ai, const double *Ax) {
    ccol *A = ccol_new(n, n, Ap[n], Ax != NULL);
    memcpy(A->p, Ap, (n + 1) * sizeof(int));
    memcpy(A->i, Ai, Ap[n] * sizeof(int));
    if (Ax) memcpy(A->x, Ax, Ap[n] * sizeof(double));
    return A;
}

/* ------------------------------------------------------------------------ */
/* approximate minimum degree  (cs_amd with order = 1, cs.cpp:645-991)       */
/* ------------------------------------------------------------------------ */

#define FLIP(i) (-(i)-2)

/* reset the marker array when the mark would wrap  (cs_wclear, cs.cpp:630-639);
 * the sum is taken with wrap-around arithmetic, as the compiled reference does */
static int reset_marks(int mark, int lemax, int *w, int n) {
    int sum = (int)((unsigned)mark + (unsigned)lemax);
    if (mark < 2 || sum < 0) {
        for (int k = 0; k < n; k++)
            if (w[k] != 0) w[k] = 1;
        mark = 2;
    }
    return mark;
}

/* depth-first postorder of the subtree at j  (cs_tdfs, cs.cpp:456-477) */
static int tree_dfs(int j, int k, int *head, const int *next, int *post, int *stack) {
    int top = 0;
    stack[0] = j;
    while (top >= 0) {
        int p = stack[top];
        int i = head[p];
        if (i == -1) {
            top--;
            post[k++] = p;
        } else {
            head[p] = next[i];
            stack[++top] = i;
        }
    }
    return k;
}

int orc_amd(int n, const int *Up, const int *Ui, int *P) {
    ccol A = {n, n, Up[n], (int *)Up, (int *)Ui, NULL};
    ccol *AT = ccol_transpose(&A, 0);
    double dd = 10 * sqrt((double)n);
    int dense = (int)(16 > dd ? 16 : dd);
    dense = (n - 2 < dense) ? n - 2 : dense;
    ccol *C = ccol_add(&A, AT, 0, 0);
    ccol_free(AT);
    ccol_drop_diag(C);
    int *Cp = C->p;
    int cnz = Cp[n];
    int nzmax = cnz + cnz / 5 + 2 * n; /* elbow room, cs.cpp:691 */
    int *Ci = (int *)xmalloc(nzmax, sizeof(int));
    memcpy(Ci, C->i, cnz * sizeof(int));
    int *W = (int *)xmalloc(8 * (size_t)(n + 1), sizeof(int));
    int *len = W, *nv = W + (n + 1), *next = W + 2 * (n + 1), *head = W + 3 * (n + 1);
    int *elen = W + 4 * (n + 1), *degree = W + 5 * (n + 1), *w = W + 6 * (n + 1);
    int *hhead = W + 7 * (n + 1);
    int *last = P; /* P doubles as the `last` workspace, as in cs.cpp:696 */
    int lemax = 0, mindeg = 0, nel = 0, mark;

    for (int k = 0; k < n; k++) len[k] = Cp[k + 1] - Cp[k];
    len[n] = 0;
    for (int i = 0; i <= n; i++) {
        head[i] = -1;
        last[i] = -1;
        next[i] = -1;
        hhead[i] = -1;
        nv[i] = 1;
        w[i] = 1;
        elen[i] = 0;
        degree[i] = len[i];
    }
    mark = reset_marks(0, 0, w, n);
    elen[n] = -2;
    Cp[n] = -1;
    w[n] = 0;
    /* initial degree lists, cs.cpp:718-742 */
    for (int i = 0; i < n; i++) {
        int d = degree[i];
        if (d == 0) {
            elen[i] = -2;
            nel++;
            Cp[i] = -1;
            w[i] = 0;
        } else if (d > dense) {
            nv[i] = 0;
            elen[i] = -1;
            nel++;
            Cp[i] = FLIP(n);
            nv[n]++;
        } else {
            if (head[d] != -1) last[head[d]] = i;
            next[i] = head[d];
            head[d] = i;
        }
    }
    while (nel < n) {
        /* pivot of least approximate degree, cs.cpp:746-751 */
        int k = -1;
        for (; mindeg < n && (k = head[mindeg]) == -1; mindeg++)
            ;
        if (next[k] != -1) last[next[k]] = -1;
        head[mindeg] = next[k];
        int elenk = elen[k];
        int nvk = nv[k];
        nel += nvk;
        /* compaction of the element/node lists, cs.cpp:753-773 */
        if (elenk > 0 && cnz + mindeg >= nzmax) {
            for (int j = 0; j < n; j++) {
                int p = Cp[j];
                if (p >= 0) {
                    Cp[j] = Ci[p];
                    Ci[p] = FLIP(j);
                }
            }
            int q = 0;
            for (int p = 0; p < cnz;) {
                int j = FLIP(Ci[p++]);
                if (j >= 0) {
                    Ci[q] = Cp[j];
                    Cp[j] = q++;
                    for (int k3 = 0; k3 < len[j] - 1; k3++) Ci[q++] = Ci[p++];
                }
            }
            cnz = q;
        }
        /* new element Lk, cs.cpp:775-821 */
        int dk = 0;
        nv[k] = -nvk;
        int p = Cp[k];
        int pk1 = (elenk == 0) ? p : cnz;
        int pk2 = pk1;
        for (int k1 = 1; k1 <= elenk + 1; k1++) {
            int e, pj, ln;
            if (k1 > elenk) {
                e = k;
                pj = p;
                ln = len[k] - elenk;
            } else {
                e = Ci[p++];
                pj = Cp[e];
                ln = len[e];
            }
            for (int k2 = 1; k2 <= ln; k2++) {
                int i = Ci[pj++];
                int nvi = nv[i];
                if (nvi <= 0) continue;
                dk += nvi;
                nv[i] = -nvi;
                Ci[pk2++] = i;
                if (next[i] != -1) last[next[i]] = last[i];
                if (last[i] != -1)
                    next[last[i]] = next[i];
                else
                    head[degree[i]] = next[i];
            }
            if (e != k) {
                Cp[e] = FLIP(k);
                w[e] = 0;
            }
        }
        if (elenk != 0) cnz = pk2;
        degree[k] = dk;
        Cp[k] = pk1;
        len[k] = pk2 - pk1;
        elen[k] = -2;
        /* |Le \ Lk| for every element e adjacent to Lk, cs.cpp:823-842 */
        mark = reset_marks(mark, lemax, w, n);
        for (int pk = pk1; pk < pk2; pk++) {
            int i = Ci[pk];
            int eln = elen[i];
            if (eln <= 0) continue;
            int nvi = -nv[i];
            int wnvi = mark - nvi;
            for (int pp = Cp[i]; pp <= Cp[i] + eln - 1; pp++) {
                int e = Ci[pp];
                if (w[e] >= mark)
                    w[e] -= nvi;
                else if (w[e] != 0)
                    w[e] = degree[e] + wnvi;
            }
        }
        /* approximate degrees and hashes, cs.cpp:844-902 */
        for (int pk = pk1; pk < pk2; pk++) {
            int i = Ci[pk];
            int p1 = Cp[i];
            int p2 = p1 + elen[i] - 1;
            int pn = p1;
            unsigned int h = 0;
            int d = 0;
            for (int pp = p1; pp <= p2; pp++) {
                int e = Ci[pp];
                if (w[e] != 0) {
                    int dext = w[e] - mark;
                    if (dext > 0) {
                        d += dext;
                        Ci[pn++] = e;
                        h += e;
                    } else {
                        Cp[e] = FLIP(k);
                        w[e] = 0;
                    }
                }
            }
            elen[i] = pn - p1 + 1;
            int p3 = pn;
            int p4 = p1 + len[i];
            for (int pp = p2 + 1; pp < p4; pp++) {
                int j = Ci[pp];
                int nvj = nv[j];
                if (nvj <= 0) continue;
                d += nvj;
                Ci[pn++] = j;
                h += j;
            }
            if (d == 0) {
                Cp[i] = FLIP(k);
                int nvi = -nv[i];
                dk -= nvi;
                nvk += nvi;
                nel += nvi;
                nv[i] = 0;
                elen[i] = -1;
            } else {
                degree[i] = degree[i] < d ? degree[i] : d;
                Ci[pn] = Ci[p3];
                Ci[p3] = Ci[p1];
                Ci[p1] = k;
                len[i] = pn - p1 + 1;
                h %= (unsigned)n;
                next[i] = hhead[h];
                hhead[h] = i;
                last[i] = (int)h;
            }
        }
        degree[k] = dk;
        lemax = lemax > dk ? lemax : dk;
        mark = reset_marks((int)((unsigned)mark + (unsigned)lemax), lemax, w, n);
        /* indistinguishable nodes, cs.cpp:907-943 */
        for (int pk = pk1; pk < pk2; pk++) {
            int i = Ci[pk];
            if (nv[i] >= 0) continue;
            unsigned int h = (unsigned)last[i];
            i = hhead[h];
            hhead[h] = -1;
            for (; i != -1 && next[i] != -1; i = next[i], mark++) {
                int ln = len[i];
                int eln = elen[i];
                for (int pp = Cp[i] + 1; pp <= Cp[i] + ln - 1; pp++) w[Ci[pp]] = mark;
                int jlast = i;
                for (int j = next[i]; j != -1;) {
                    int ok = (len[j] == ln) && (elen[j] == eln);
                    for (int pp = Cp[j] + 1; ok && pp <= Cp[j] + ln - 1; pp++)
                        if (w[Ci[pp]] != mark) ok = 0;
                    if (ok) {
                        Cp[j] = FLIP(i);
                        nv[i] += nv[j];
                        nv[j] = 0;
                        elen[j] = -1;
                        j = next[j];
                        next[jlast] = j;
                    } else {
                        jlast = j;
                        j = next[j];
                    }
                }
            }
        }
        /* finalize Lk, cs.cpp:945-966 */
        int pw = pk1;
        for (int pk = pk1; pk < pk2; pk++) {
            int i = Ci[pk];
            int nvi = -nv[i];
            if (nvi <= 0) continue;
            nv[i] = nvi;
            int d = degree[i] + dk - nvi;
            d = d < n - nel - nvi ? d : n - nel - nvi;
            if (head[d] != -1) last[head[d]] = i;
            next[i] = head[d];
            last[i] = -1;
            head[d] = i;
            mindeg = mindeg < d ? mindeg : d;
            degree[i] = d;
            Ci[pw++] = i;
        }
        nv[k] = nvk;
        if ((len[k] = pw - pk1) == 0) {
            Cp[k] = -1;
            w[k] = 0;
        }
        if (elenk != 0) cnz = pw;
    }
    /* postorder the assembly tree, cs.cpp:969-989 */
    for (int i = 0; i < n; i++) Cp[i] = FLIP(Cp[i]);
    for (int j = 0; j <= n; j++) head[j] = -1;
    for (int j = n; j >= 0; j--) {
        if (nv[j] > 0) continue;
        next[j] = head[Cp[j]];
        head[Cp[j]] = j;
    }
    for (int e = n; e >= 0; e--) {
        if (nv[e] <= 0) continue;
        if (Cp[e] != -1) {
            next[e] = head[Cp[e]];
            head[Cp[e]] = e;
        }
    }
    for (int k = 0, i = 0; i <= n; i++) {
        if (Cp[i] == -1) k = tree_dfs(i, k, head, next, P, w);
    }
    free(Ci);
    free(W);
    ccol_free(C);
    return 0;
}

/* ------------------------------------------------------------------------ */
/* elimination tree, postorder, column counts                               */
/* ------------------------------------------------------------------------ */

/* cs_etree(A, 0), cs.cpp:480-507 */
int orc_etree(int n, const int *Ap, const int *Ai, int *parent) {
    int *anc = (int *)xmalloc(n, sizeof(int));
    for (int k = 0; k < n; k++) {
        parent[k] = -1;
        anc[k] = -1;
        for (int p = Ap[k]; p < Ap[k + 1]; p++) {
            int i = Ai[p];
            while (i != -1 && i < k) {
                int inext = anc[i];
                anc[i] = k;
                if (inext == -1) parent[i] = k;
                i = inext;
            }
        }
    }
    free(anc);
    return 0;
}

/* cs_post, cs.cpp:432-453 */
int orc_post(int n, const int *parent, int *post) {
    int *w = (int *)xmalloc(3 * (size_t)n, sizeof(int));
    int *head = w, *next = w + n, *stack = w + 2 * n;
    for (int j = 0; j < n; j++) head[j] = -1;
    for (int j = n - 1; j >= 0; j--) {
        if (parent[j] == -1) continue;
        next[j] = head[parent[j]];
        head[parent[j]] = j;
    }
    int k = 0;
    for (int j = 0; j < n; j++) {
        if (parent[j] != -1) continue;
        k = tree_dfs(j, k, head, next, post, stack);
    }
    free(w);
    return 0;
}

/* cs_leaf, cs.cpp:385-404 */
static int skel_leaf(int i, int j, const int *first, int *maxfirst, int *prevleaf, int *ancestor,
                     int *jleaf) {
    *jleaf = 0;
    if (i <= j || first[j] <= maxfirst[i]) return -1;
    maxfirst[i] = first[j];
    int jprev = prevleaf[i];
    prevleaf[i] = j;
    *jleaf = (jprev == -1) ? 1 : 2;
    if (*jleaf == 1) return i;
    int q;
    for (q = jprev; q != ancestor[q]; q = ancestor[q])
        ;
    for (int s = jprev, sp; s != q; s = sp) {
        sp = ancestor[s];
        ancestor[s] = q;
    }
    return q;
}

/* cs_counts(A, parent, post, 0), cs.cpp:338-382, A full symmetric */
int orc_counts(int n, const int *Ap, const int *Ai, const int *parent, const int *post,
               int *colcount) {
    ccol A = {n, n, Ap[n], (int *)Ap, (int *)Ai, NULL};
    ccol *AT = ccol_transpose(&A, 0);
    int *w = (int *)xmalloc(4 * (size_t)n, sizeof(int));
    int *ancestor = w, *maxfirst = w + n, *prevleaf = w + 2 * n, *first = w + 3 * n;
    int *delta = colcount;
    for (int k = 0; k < 4 * n; k++) w[k] = -1;
    for (int k = 0; k < n; k++) {
        int j = post[k];
        delta[j] = (first[j] == -1) ? 1 : 0;
        for (; j != -1 && first[j] == -1; j = parent[j]) first[j] = k;
    }
    for (int i = 0; i < n; i++) ancestor[i] = i;
    for (int k = 0; k < n; k++) {
        int j = post[k];
        if (parent[j] != -1) delta[parent[j]]--;
        for (int p = AT->p[j]; p < AT->p[j + 1]; p++) {
            int jleaf;
            int q = skel_leaf(AT->i[p], j, first, maxfirst, prevleaf, ancestor, &jleaf);
            if (jleaf >= 1) delta[j]++;
            if (jleaf == 2) delta[q]--;
        }
        if (parent[j] != -1) ancestor[j] = parent[j];
    }
    for (int j = 0; j < n; j++)
        if (parent[j] != -1) colcount[parent[j]] += colcount[j];
    free(w);
    ccol_free(AT);
    return 0;
}

/* ------------------------------------------------------------------------ */
/* assembly trees  (etree.cpp)                                               */
/* ------------------------------------------------------------------------ */

typedef struct {
    int nodo, cols, rows, ceros;
    int nkids, *kids; /* indices into the owning node array */
    int nmem, *mem;   /* member columns (relaxed tree only) */
} tnode;

/* GetETree, etree.cpp:12-48: node per column, children ascending, list in
 * postorder.  Returns the node array; order[] receives the postorder. */
static tnode *nodal_tree(int n, const int *parent, const int *post, const int *count) {
    tnode *t = (tnode *)xcalloc(n, sizeof(tnode));
    int *nk = (int *)xcalloc(n, sizeof(int));
    for (int i = 0; i < n; i++)
        if (parent[i] != -1) nk[parent[i]]++;
    for (int i = 0; i < n; i++) {
        t[i].nodo = i;
        t[i].cols = 1;
        t[i].rows = count[i];
        t[i].ceros = 0;
        t[i].kids = (int *)xmalloc(nk[i], sizeof(int));
        t[i].nmem = 1;
        t[i].mem = (int *)xmalloc(1, sizeof(int));
        t[i].mem[0] = i;
    }
    for (int i = 0; i < n; i++) {
        if (parent[i] != -1) {
            tnode *pp = &t[parent[i]];
            pp->kids[pp->nkids++] = i;
        }
    }
    free(nk);
    (void)post;
    return t;
}

static void free_nodes(tnode *t, int n) {
    for (int i = 0; i < n; i++) {
        free(t[i].kids);
        free(t[i].mem);
    }
    free(t);
}

/* GetSuperETree, etree.cpp:50-118, with every node's children kept in
 * postorder (the reference stores the non-last ones reversed at
 * etree.cpp:101-103, which its own Factor cannot pair; the partition is the
 * same).  Supernode ids are positions in the output list. */
static int super_tree(int n, const tnode *nt, const int *post, tnode *out) {
    int *stack = (int *)xmalloc(n, sizeof(int));
    int top = 0, ns = 0;
    for (int idx = 0; idx < n; idx++) {
        const tnode *t = &nt[post[idx]];
        int merge = 0;
        if (t->nkids >= 1) {
            const tnode *lastk = &nt[t->kids[t->nkids - 1]];
            if (lastk->rows == t->rows + 1 && lastk->nodo == t->nodo - 1) merge = 1;
        }
        tnode r;
        memset(&r, 0, sizeof(r));
        int slot;
        if (!merge) {
            r.nodo = t->nodo;
            r.cols = t->cols;
            r.rows = t->rows;
            r.nkids = t->nkids;
            r.kids = (int *)xmalloc(r.nkids, sizeof(int));
            for (int i = t->nkids - 1; i >= 0; i--) r.kids[i] = stack[--top];
            slot = ns++;
        } else {
            int hm = stack[--top];
            tnode *h = &out[hm];
            r.nodo = h->nodo;
            r.cols = h->cols + 1;
            r.rows = h->rows - 1;
            r.nkids = t->nkids - 1 + h->nkids;
            r.kids = (int *)xmalloc(r.nkids, sizeof(int));
            for (int i = 0; i < h->nkids; i++) r.kids[t->nkids - 1 + i] = h->kids[i];
            for (int i = t->nkids - 2; i >= 0; i--) r.kids[i] = stack[--top];
            free(h->kids);
            slot = hm; /* replaces the list's last entry, etree.cpp:107-109 */
            if (slot != ns - 1) {
                fprintf(stderr, "oracle: supernode merge is not the last entry\n");
                abort();
            }
        }
        out[slot] = r;
        stack[top++] = slot;
    }
    free(stack);
    return ns;
}

/* selection sort of a[] by c[a[]] ascending, etree.cpp:180-192 */
static void sort_by_count(int *a, const int *c, int n) {
    for (int i = 0; i < n; i++) {
        int x = -1;
        for (int j = i; j < n; j++)
            if (x == -1 || c[a[j]] < c[a[x]]) x = j;
        int tmp = a[x];
        a[x] = a[i];
        a[i] = tmp;
    }
}

/* GetRelaxedETree, etree.cpp:194-342, on the nodal tree; mutates count,
 * writes the column permutation (new -> old) and the relaxed nodes in dfs
 * postorder into out (ids = output positions).  Returns the node count. */
static int relaxed_tree(int n, const tnode *nt, const int *post, int max_zeros, int *count,
                        int *perm, tnode *out) {
    tnode *R = (tnode *)xcalloc(n, sizeof(tnode)); /* one per nodal node */
    int *stack = (int *)xmalloc(n, sizeof(int));
    int top = 0;
    for (int idx = 0; idx < n; idx++) {
        const tnode *t = &nt[post[idx]];
        int nk = t->nkids;
        int *kids = &stack[top - nk]; /* the children's relaxed roots */
        int *merged = (int *)xcalloc(nk, sizeof(int));
        int zeros = t->ceros;
        int rid = post[idx];
        tnode *r = &R[rid];
        r->nodo = t->nodo;
        r->cols = t->cols;
        r->rows = t->rows;
        r->ceros = 0;
        r->nmem = 1;
        r->mem = (int *)xmalloc(1, sizeof(int));
        r->mem[0] = r->nodo;
        int cols = 1;
        for (;;) {
            int best = -1, best_z = -1;
            for (int h = 0; h < nk; h++) {
                const tnode *k = &R[kids[h]];
                int z = (t->rows + cols - k->rows) * k->cols + k->ceros;
                if (!merged[h] && z <= max_zeros && (best_z == -1 || z < best_z)) {
                    best_z = z;
                    best = h;
                }
            }
            if (best < 0) break;
            merged[best] = 1;
            const tnode *k = &R[kids[best]];
            zeros += best_z;
            cols += k->cols;
            for (int h = 0; h < k->cols; h++) count[k->mem[h]] += (best_z - k->ceros) / k->cols;
        }
        r->ceros = zeros;
        int nkids = nk;
        for (int h = 0; h < nk; h++)
            if (merged[h]) nkids += R[kids[h]].nkids - 1;
        r->kids = (int *)xmalloc(nkids, sizeof(int));
        r->nkids = 0;
        for (int h = 0; h < nk; h++) {
            tnode *k = &R[kids[h]];
            if (!merged[h]) {
                r->kids[r->nkids++] = kids[h];
            } else {
                r->mem = (int *)realloc(r->mem, (r->cols + k->cols) * sizeof(int));
                for (int c = 0; c < k->cols; c++) r->mem[r->cols++] = k->mem[c];
                r->nmem = r->cols;
                for (int hh = 0; hh < k->nkids; hh++) r->kids[r->nkids++] = k->kids[hh];
            }
        }
        for (int c = 0; c < r->cols; c++)
            if (r->mem[c] < r->nodo) r->nodo = r->mem[c];
        sort_by_count(r->mem, count, r->cols);
        free(merged);
        top -= nk;
        stack[top++] = rid;
    }
    /* dfs from the last root, etree.cpp:165-178,329-331 (iterative, same order) */
    int *map = (int *)xmalloc(n, sizeof(int)); /* relaxed id -> output position */
    for (int i = 0; i < n; i++) map[i] = -1;
    int *st = (int *)xmalloc(n, sizeof(int));
    int *it = (int *)xmalloc(n, sizeof(int));
    int sp = 0, nout = 0, c = 0;
    st[sp] = stack[top - 1];
    it[sp] = 0;
    sp++;
    while (sp > 0) {
        int v = st[sp - 1];
        if (it[sp - 1] < R[v].nkids) {
            int ch = R[v].kids[it[sp - 1]++];
            st[sp] = ch;
            it[sp] = 0;
            sp++;
        } else {
            sp--;
            map[v] = nout;
            out[nout] = R[v];
            out[nout].nodo = c;
            for (int i = R[v].cols - 1; i >= 0; i--) perm[c++] = R[v].mem[i];
            nout++;
        }
    }
    for (int s = 0; s < nout; s++)
        for (int h = 0; h < out[s].nkids; h++) out[s].kids[h] = map[out[s].kids[h]];
    for (int i = 0; i < n; i++) /* nodes absorbed into a parent */
        if (map[i] == -1) {
            free(R[i].mem);
            free(R[i].kids);
        }
    free(R);
    free(map);
    free(st);
    free(it);
    free(stack);
    return nout;
}

/* ------------------------------------------------------------------------ */
/* symbolic driver  (mdgpu.cu:1745-1875)                                     */
/* ------------------------------------------------------------------------ */

int orc_analyze(int n, const int *Ap, const int *Ai, const double *Ax, int use_amd, int mode,
                int rn_zeros, orc_plan **out) {
    orc_plan *P = (orc_plan *)xcalloc(1, sizeof(orc_plan));
    P->n = n;
    ccol *C_low = ccol_wrap(n, Ap, Ai, Ax);
    ccol *A_low;
    if (use_amd) {
        ccol *C_up = ccol_transpose(C_low, 1);
        P->perm = (int *)xmalloc(n + 1, sizeof(int));
        orc_amd(n, C_up->p, C_up->i, P->perm);
        int *pinv = (int *)xmalloc(n, sizeof(int));
        for (int k = 0; k < n; k++) pinv[P->perm[k]] = k;
        ccol *U = ccol_symperm_upper(C_up, pinv, 1);
        ccol_free(C_up);
        A_low = ccol_transpose(U, 1);
        ccol_free(U);
        free(pinv);
        ccol_free(C_low);
    } else {
        A_low = C_low;
    }
    ccol *A = ccol_sym_from_lower(A_low);
    P->parent = (int *)xmalloc(n, sizeof(int));
    P->post = (int *)xmalloc(n, sizeof(int));
    P->count0 = (int *)xmalloc(n, sizeof(int));
    P->count = (int *)xmalloc(n, sizeof(int));
    orc_etree(n, A->p, A->i, P->parent);
    orc_post(n, P->parent, P->post);
    orc_counts(n, A->p, A->i, P->parent, P->post, P->count0);
    memcpy(P->count, P->count0, n * sizeof(int));
    ccol_free(A);

    int nroots = 0;
    for (int i = 0; i < n; i++) nroots += P->parent[i] == -1;
    if (nroots != 1) { /* GetETree rejects a forest, etree.cpp:27-31 */
        ccol_free(A_low);
        orc_plan_free(P);
        return -1;
    }
    tnode *nt = nodal_tree(n, P->parent, P->post, P->count);
    tnode *sn = (tnode *)xcalloc(n, sizeof(tnode));
    int ns;
    if (mode == ORC_RELAXED) {
        int *permR = (int *)xmalloc(n, sizeof(int));
        ns = relaxed_tree(n, nt, P->post, rn_zeros, P->count, permR, sn);
        int *ipermR = (int *)xmalloc(n, sizeof(int));
        for (int k = 0; k < n; k++) ipermR[permR[k]] = k;
        ccol *t1 = ccol_transpose(A_low, 1);
        ccol *t2 = ccol_symperm_upper(t1, ipermR, 1);
        ccol_free(t1);
        ccol_free(A_low);
        A_low = ccol_transpose(t2, 1);
        ccol_free(t2);
        int *c2 = (int *)xmalloc(n, sizeof(int));
        for (int k = 0; k < n; k++) c2[k] = P->count[permR[k]];
        free(P->count);
        P->count = c2;
        int *p2 = (int *)xmalloc(n, sizeof(int));
        for (int k = 0; k < n; k++) p2[k] = P->perm ? P->perm[permR[k]] : permR[k];
        free(P->perm);
        P->perm = p2;
        P->rn_perm = permR;
        free(ipermR);
    } else if (mode == ORC_SUPER) {
        ns = super_tree(n, nt, P->post, sn);
    } else {
        ns = n;
        int *pos = (int *)xmalloc(n, sizeof(int));
        for (int k = 0; k < n; k++) pos[P->post[k]] = k;
        for (int k = 0; k < n; k++) {
            const tnode *t = &nt[P->post[k]];
            sn[k] = *t;
            sn[k].kids = (int *)xmalloc(t->nkids, sizeof(int));
            for (int h = 0; h < t->nkids; h++) sn[k].kids[h] = pos[t->kids[h]];
            sn[k].mem = NULL;
        }
        free(pos);
    }
    P->nsuper = ns;
    P->sn_nodo = (int *)xmalloc(ns, sizeof(int));
    P->sn_cols = (int *)xmalloc(ns, sizeof(int));
    P->sn_childptr = (int *)xmalloc(ns + 1, sizeof(int));
    int nk = 0;
    for (int s = 0; s < ns; s++) nk += sn[s].nkids;
    P->sn_child = (int *)xmalloc(nk, sizeof(int));
    P->sn_childptr[0] = 0;
    for (int s = 0; s < ns; s++) {
        P->sn_nodo[s] = sn[s].nodo;
        P->sn_cols[s] = sn[s].cols;
        P->sn_childptr[s + 1] = P->sn_childptr[s] + sn[s].nkids;
        memcpy(P->sn_child + P->sn_childptr[s], sn[s].kids, sn[s].nkids * sizeof(int));
        free(sn[s].kids);
        if (mode == ORC_RELAXED) free(sn[s].mem);
    }
    free(sn);
    free_nodes(nt, n);

    P->Lp = (int *)xmalloc(n + 1, sizeof(int));
    long long nz = 0;
    for (int i = 0; i < n; i++) {
        P->Lp[i] = (int)nz;
        nz += P->count[i];
    }
    P->Lp[n] = (int)nz;
    P->lnz = nz;
    P->Ap = A_low->p;
    P->Ai = A_low->i;
    P->Ax = A_low->x;
    free(A_low);
    *out = P;
    return 0;
}

void orc_plan_free(orc_plan *P) {
    if (!P) return;
    free(P->Ap);
    free(P->Ai);
    free(P->Ax);
    free(P->perm);
    free(P->parent);
    free(P->post);
    free(P->count0);
    free(P->count);
    free(P->rn_perm);
    free(P->sn_nodo);
    free(P->sn_cols);
    free(P->sn_childptr);
    free(P->sn_child);
    free(P->Lp);
    free(P);
}

/* ------------------------------------------------------------------------ */
/* dense kernels: the used branches of the reference's f2c BLAS              */
/* ------------------------------------------------------------------------ */

/* A := alpha x x' + A, lower, incx = 1  (dsyr.cpp:200-214) */
static void syr_lower(int n, double alpha, const double *x, double *a, int lda) {
    for (int j = 0; j < n; j++) {
        if (x[j] != 0.) {
            double temp = alpha * x[j];
            for (int i = j; i < n; i++) a[i + (size_t)j * lda] += x[i] * temp;
        }
    }
}

/* B := B inv(A'), A lower non-unit, alpha = 1  (dtrsm.cpp, Right/Lower/Trans) */
static void trsm_rltn(int m, int n, const double *a, int lda, double *b, int ldb) {
    for (int k = 0; k < n; k++) {
        double temp = 1. / a[k + (size_t)k * lda];
        for (int i = 0; i < m; i++) b[i + (size_t)k * ldb] = temp * b[i + (size_t)k * ldb];
        for (int j = k + 1; j < n; j++) {
            if (a[j + (size_t)k * lda] != 0.) {
                temp = a[j + (size_t)k * lda];
                for (int i = 0; i < m; i++) b[i + (size_t)j * ldb] -= temp * b[i + (size_t)k * ldb];
            }
        }
    }
}

/* C := alpha A B' + C, beta = 1  (dgemm.cpp:325-356, 'N','T') */
static void gemm_nt(int m, int n, int k, double alpha, const double *a, int lda, const double *b,
                    int ldb, double *c, int ldc) {
    for (int j = 0; j < n; j++) {
        for (int l = 0; l < k; l++) {
            if (b[j + (size_t)l * ldb] != 0.) {
                double temp = alpha * b[j + (size_t)l * ldb];
                for (int i = 0; i < m; i++) c[i + (size_t)j * ldc] += temp * a[i + (size_t)l * lda];
            }
        }
    }
}

/* FactorAux_CPU_3's blocked right-looking partial Cholesky, mdgpu.cu:1312-1341 */
void orc_front_factor(int n, int cols, int block_size, double *M) {
    int w = n;
    int b = block_size <= 0 ? n : block_size;
    for (int i = 0; i < cols; i += b) {
        int nb = (i + b < cols) ? i + b : cols;
        int b2 = nb - i;
        for (int c = i; c < nb; c++) {
            double raiz = sqrt(M[c + (size_t)c * w]);
            for (int j = c; j < nb; j++) M[j + (size_t)c * w] = M[j + (size_t)c * w] / raiz;
            syr_lower(nb - c - 1, -1.0, M + (c + 1) + (size_t)c * w, M + (c + 1) + (size_t)(c + 1) * w,
                      w);
        }
        if (n - nb > 0) {
            trsm_rltn(n - nb, nb - i, M + i + (size_t)i * w, w, M + (i + b2) + (size_t)i * w, w);
            gemm_nt(n - nb, n - nb, b2, -1.0, M + (i + b2) + (size_t)i * w, w,
                    M + (i + b2) + (size_t)i * w, w, M + (i + b2) + (size_t)(i + b2) * w, w);
        }
    }
}

/* ------------------------------------------------------------------------ */
/* multifrontal numeric factorization  (Factor, mdgpu.cu:1394-1608)          */
/* ------------------------------------------------------------------------ */

typedef struct {
    int n, offset;
    int *q;  /* global row ids */
    int *ql; /* relative map into the destination front */
    double *x; /* n x n column-major, ld = n */
} front;

static front *front_new(int n, int *q, int offset) {
    front *f = (front *)xcalloc(1, sizeof(front));
    f->n = n;
    f->q = q;
    f->offset = offset;
    f->x = (double *)xcalloc((size_t)n * n, sizeof(double));
    return f;
}
static void front_free(front *f) {
    if (!f) return;
    free(f->q);
    free(f->ql);
    free(f->x);
    free(f);
}

/* sorted union without duplicates  (VectorMerge, mdgpu.cu:535-583) */
static int *merge_rows(const int *q1, int n1, const int *q2, int n2, int *nout) {
    int *q = (int *)xmalloc(n1 + n2, sizeof(int));
    int nn = 0, k1 = 0, k2 = 0;
    while (k1 < n1 || k2 < n2) {
        int v;
        if (k1 < n1 && (k2 >= n2 || q1[k1] < q2[k2]))
            v = q1[k1++];
        else
            v = q2[k2++];
        if (nn == 0 || q[nn - 1] != v) q[nn++] = v;
    }
    *nout = nn;
    return q;
}

/* position of each q[i] inside Q  (VectorMergeIndices, mdgpu.cu:585-595) */
static int *positions_in(const int *Q, const int *q, int n) {
    int *ql = (int *)xmalloc(n, sizeof(int));
    int j = 0;
    for (int i = 0; i < n; i++) {
        while (Q[j] != q[i]) j++;
        ql[i] = j;
    }
    return ql;
}

/* front of supernode (k, c) assembled from lower A  (MatrizGetFk_3,
 * mdgpu.cu:180-291): rows k..k+c-1 then the sorted union of the rows >= k+c
 * of A's columns k..k+c-1; A's values scattered into the first c columns. */
static front *front_from_A(int n_all, const int *Ap, const int *Ai, const double *Ax, int k,
                           int c) {
    int cap = c;
    for (int i = 0; i < c; i++) cap += Ap[k + i + 1] - Ap[k + i];
    int *rows = (int *)xmalloc(cap, sizeof(int));
    int nr = 0;
    for (int i = 0; i < c; i++) rows[nr++] = k + i;
    int *pos = (int *)xmalloc(c, sizeof(int));
    for (int i = 0; i < c; i++) {
        int p = Ap[k + i];
        while (p < Ap[k + i + 1] && Ai[p] < k + c) p++;
        pos[i] = p;
    }
    for (;;) {
        int mn = 0x7fffffff;
        for (int i = 0; i < c; i++)
            if (pos[i] < Ap[k + i + 1] && Ai[pos[i]] < mn) mn = Ai[pos[i]];
        if (mn == 0x7fffffff) break;
        rows[nr++] = mn;
        for (int i = 0; i < c; i++)
            if (pos[i] < Ap[k + i + 1] && Ai[pos[i]] == mn) pos[i]++;
    }
    free(pos);
    front *f = front_new(nr, rows, 0);
    for (int i = 0; i < c; i++) {
        int r = 0;
        for (int p = Ap[k + i]; p < Ap[k + i + 1]; p++) {
            while (rows[r] < Ai[p]) r++;
            f->x[r + (size_t)i * nr] = Ax[p];
        }
    }
    (void)n_all;
    return f;
}

/* dst[ql[i], ql[j]] += src[off+i, off+j] over the full trailing square
 * (ExtendAdd_CPU, mdgpu.cu:748-767) */
static void extend_add(const front *src, front *dst) {
    int m = src->n - src->offset;
    for (int j = 0; j < m; j++) {
        int qj = src->ql[j];
        for (int i = 0; i < m; i++) {
            int qi = src->ql[i];
            dst->x[qi + (size_t)qj * dst->n] +=
                src->x[(src->offset + i) + (size_t)(src->offset + j) * src->n];
        }
    }
}

typedef struct {
    const orc_plan *P;
    int block;
    int *Li;
    double *Lx;
    double flops;
    int bad;
    int *rows_ptr, *rows, *relmap;
    int **pending; /* per supernode: map of its update rows into its parent's Uk */
} fctx;

/* factor a front whose `offset` leading columns are pivots and copy them into
 * L (FactorAux_CPU_3, mdgpu.cu:1298-1361) */
static void factor_front(fctx *X, front *f, int s) {
    const orc_plan *P = X->P;
    int n = f->n, cols = f->offset, k = P->sn_nodo[s];
    orc_front_factor(n, cols, X->block, f->x);
    for (int c = 0; c < cols; c++) {
        double dc = f->x[c + (size_t)c * n];
        if (!(dc > 0) && !X->bad) X->bad = -(k + c + 1);
        for (int j = c; j < n; j++) {
            long long x = P->Lp[k + c] + j - c;
            X->Li[x] = f->q[j];
            X->Lx[x] = f->x[j + (size_t)c * n];
        }
        X->flops += (n - c) + 1;
        X->flops += (double)(n - c) * (n - c - 1);
    }
    if (X->rows_ptr) {
        if (X->rows_ptr[s + 1] - X->rows_ptr[s] != n) {
            fprintf(stderr, "oracle: front %d has %d rows, plan expects %d\n", s, n,
                    X->rows_ptr[s + 1] - X->rows_ptr[s]);
            abort();
        }
        memcpy(X->rows + X->rows_ptr[s], f->q, n * sizeof(int));
    }
}

/* record child maps composed with the map of their Uk into the new front */
static void compose_maps(fctx *X, int t, const int *ukql) {
    const orc_plan *P = X->P;
    for (int h = P->sn_childptr[t]; h < P->sn_childptr[t + 1]; h++) {
        int ch = P->sn_child[h];
        int *pm = X->pending[ch];
        if (!pm) continue;
        int m = X->rows_ptr[ch + 1] - X->rows_ptr[ch] - P->sn_cols[ch];
        for (int r = 0; r < m; r++)
            X->relmap[X->rows_ptr[ch] + P->sn_cols[ch] + r] = ukql[pm[r]];
        free(pm);
        X->pending[ch] = NULL;
    }
}

int orc_factor(const orc_plan *P, int block_size, int *Li, double *Lx, double *flops,
               int *rows_ptr, int *rows, int *relmap) {
    fctx X;
    memset(&X, 0, sizeof(X));
    X.P = P;
    X.block = block_size;
    X.Li = Li;
    X.Lx = Lx;
    X.rows_ptr = rows_ptr;
    X.rows = rows;
    X.relmap = relmap;
    int ns = P->nsuper;
    if (rows_ptr) {
        /* front of supernode s has count[nodo] rows (one L column each) */
        rows_ptr[0] = 0;
        for (int s = 0; s < ns; s++) rows_ptr[s + 1] = rows_ptr[s] + P->count[P->sn_nodo[s]];
        X.pending = (int **)xcalloc(ns, sizeof(int *));
    }
    front **stack = (front **)xmalloc(ns, sizeof(front *));
    int top = 0;

    for (int t = 0; t < ns; t++) {
        int c0 = P->sn_childptr[t], nk = P->sn_childptr[t + 1] - c0;
        if (nk == 0) continue; /* leaves are formed by their parent, mdgpu.cu:1407 */
        front **F = (front **)xmalloc(nk, sizeof(front *));
        front **U = (front **)xmalloc(nk, sizeof(front *));
        front **U2 = (front **)xmalloc(nk, sizeof(front *));
        for (int i = 0; i < nk; i++) {
            int ch = P->sn_child[c0 + i];
            F[i] = front_from_A(P->n, P->Ap, P->Ai, P->Ax, P->sn_nodo[ch], P->sn_cols[ch]);
            F[i]->offset = P->sn_cols[ch];
        }
        for (int i = nk - 1; i >= 0; i--) {
            int ch = P->sn_child[c0 + i];
            int chk = P->sn_childptr[ch + 1] - P->sn_childptr[ch];
            U[i] = chk == 0 ? NULL : stack[--top];
        }
        for (int i = 0; i < nk; i++) {
            int ch = P->sn_child[c0 + i];
            if (!U[i]) {
                U2[i] = F[i];
                F[i] = NULL;
                continue;
            }
            int nq;
            int *q = merge_rows(F[i]->q, F[i]->n, U[i]->q + U[i]->offset, U[i]->n - U[i]->offset, &nq);
            F[i]->ql = positions_in(q, F[i]->q, F[i]->n);
            U[i]->ql = positions_in(q, U[i]->q, U[i]->n);
            if (X.pending) compose_maps(&X, ch, U[i]->ql);
            U2[i] = front_new(nq, q, P->sn_cols[ch]);
            F[i]->offset = 0;
            extend_add(F[i], U2[i]);
            extend_add(U[i], U2[i]);
        }
        for (int i = 0; i < nk; i++) factor_front(&X, U2[i], P->sn_child[c0 + i]);
        int n = U2[0]->n - U2[0]->offset;
        int *q = (int *)xmalloc(n, sizeof(int));
        memcpy(q, U2[0]->q + U2[0]->offset, n * sizeof(int));
        for (int i = 1; i < nk; i++) {
            int n2;
            int *q2 = merge_rows(q, n, U2[i]->q + U2[i]->offset, U2[i]->n - U2[i]->offset, &n2);
            free(q);
            q = q2;
            n = n2;
        }
        for (int i = 0; i < nk; i++) {
            U2[i]->ql = positions_in(q, U2[i]->q + U2[i]->offset, U2[i]->n - U2[i]->offset);
            if (X.pending) {
                int m = U2[i]->n - U2[i]->offset;
                int *pm = (int *)xmalloc(m, sizeof(int));
                memcpy(pm, U2[i]->ql, m * sizeof(int));
                X.pending[P->sn_child[c0 + i]] = pm;
            }
        }
        front *Uk = front_new(n, q, 0);
        for (int i = 0; i < nk; i++) extend_add(U2[i], Uk);
        for (int i = 0; i < nk; i++) {
            front_free(F[i]);
            front_free(U[i]);
            front_free(U2[i]);
        }
        free(F);
        free(U);
        free(U2);
        stack[top++] = Uk;
    }
    /* the root, mdgpu.cu:1551-1607 */
    int root = ns - 1;
    front *Fr = front_from_A(P->n, P->Ap, P->Ai, P->Ax, P->sn_nodo[root], P->sn_cols[root]);
    front *U2;
    if (top > 0) {
        front *U = stack[--top];
        int nq;
        int *q = merge_rows(U->q, U->n, Fr->q, Fr->n, &nq);
        U->ql = positions_in(q, U->q, U->n);
        Fr->ql = positions_in(q, Fr->q, Fr->n);
        if (X.pending) compose_maps(&X, root, U->ql);
        U2 = front_new(nq, q, P->sn_cols[root]);
        extend_add(Fr, U2);
        extend_add(U, U2);
        front_free(Fr);
        front_free(U);
    } else {
        U2 = Fr;
        U2->offset = P->sn_cols[root];
    }
    factor_front(&X, U2, root);
    front_free(U2);
    if (relmap)
        for (int r = rows_ptr[root]; r < rows_ptr[root + 1]; r++) relmap[r] = -1;
    free(stack);
    if (X.pending) {
        for (int s = 0; s < ns; s++) free(X.pending[s]);
        free(X.pending);
    }
    if (flops) *flops = X.flops;
    return X.bad;
}

/* ------------------------------------------------------------------------ */
/* solves and residual  (cs.cpp:1069-1146, mdgpu.cu:1941-1972)               */
/* ------------------------------------------------------------------------ */

void orc_solve(const orc_plan *P, const int *Li, const double *Lx, const double *b, double *x) {
    int n = P->n;
    const int *Lp = P->Lp;
    double *y = (double *)xmalloc(n, sizeof(double));
    for (int k = 0; k < n; k++) y[k] = P->perm ? b[P->perm[k]] : b[k]; /* cs_pvec */
    for (int j = 0; j < n; j++) {                                        /* cs_lsolve */
        y[j] /= Lx[Lp[j]];
        for (int p = Lp[j] + 1; p < Lp[j + 1]; p++) y[Li[p]] -= Lx[p] * y[j];
    }
    for (int j = n - 1; j >= 0; j--) { /* cs_ltsolve */
        for (int p = Lp[j] + 1; p < Lp[j + 1]; p++) y[j] -= Lx[p] * y[Li[p]];
        y[j] /= Lx[Lp[j]];
    }
    for (int k = 0; k < n; k++) { /* cs_ipvec */
        if (P->perm)
            x[P->perm[k]] = y[k];
        else
            x[k] = y[k];
    }
    free(y);
}

double orc_residual(int n, const int *Ap, const int *Ai, const double *Ax, const double *x,
                    const double *b) {
    ccol *L = ccol_wrap(n, Ap, Ai, Ax);
    ccol *A = ccol_sym_from_lower(L);
    double *r = (double *)xmalloc(n, sizeof(double));
    for (int i = 0; i < n; i++) r[i] = -b[i];
    for (int j = 0; j < n; j++) /* cs_gaxpy */
        for (int p = A->p[j]; p < A->p[j + 1]; p++) r[A->i[p]] += A->x[p] * x[j];
    double nr = 0, nx = 0, nb = 0, na = 0;
    for (int i = 0; i < n; i++) {
        nr = fmax(nr, fabs(r[i]));
        nx = fmax(nx, fabs(x[i]));
        nb = fmax(nb, fabs(b[i]));
    }
    for (int j = 0; j < n; j++) { /* cs_norm */
        double s = 0;
        for (int p = A->p[j]; p < A->p[j + 1]; p++) s += fabs(A->x[p]);
        na = fmax(na, s);
    }
    free(r);
    ccol_free(A);
    ccol_free(L);
    return nr / (na * nx + nb);
}

/* ------------------------------------------------------------------------ */
/* accessors                                                                */
/* ------------------------------------------------------------------------ */

int orc_plan_n(const orc_plan *p) { return p->n; }
int orc_plan_nsuper(const orc_plan *p) { return p->nsuper; }
long long orc_plan_lnz(const orc_plan *p) { return p->lnz; }
int orc_plan_nchild_total(const orc_plan *p) { return p->sn_childptr[p->nsuper]; }
int orc_plan_nnz_low(const orc_plan *p) { return p->Ap[p->n]; }

void orc_plan_copy(const orc_plan *p, const char *what, void *dst) {
    int n = p->n, ns = p->nsuper;
#define CP(name, ptr, cnt, T)                                    \
    if (!strcmp(what, name)) {                                   \
        if (ptr) memcpy(dst, ptr, (size_t)(cnt) * sizeof(T));    \
        return;                                                  \
    }
    CP("perm", p->perm, n, int);
    CP("parent", p->parent, n, int);
    CP("post", p->post, n, int);
    CP("count0", p->count0, n, int);
    CP("count", p->count, n, int);
    CP("rn_perm", p->rn_perm, n, int);
    CP("sn_nodo", p->sn_nodo, ns, int);
    CP("sn_cols", p->sn_cols, ns, int);
    CP("sn_childptr", p->sn_childptr, ns + 1, int);
    CP("sn_child", p->sn_child, p->sn_childptr[ns], int);
    CP("Lp", p->Lp, n + 1, int);
    CP("Ap", p->Ap, n + 1, int);
    CP("Ai", p->Ai, p->Ap[n], int);
    CP("Ax", p->Ax, p->Ap[n], double);
#undef CP
    fprintf(stderr, "oracle: unknown plan field %s\n", what);
}
