/*
 * The drop-in binding a maintainer of the reference adds (test
 * infrastructure: linked into oracle/_ref/mdgpu_ref_shim_harness, the
 * reference's own driver sequence with its Factor replaced by this one).
 *
 * Factor(cs* A, cs* spL, ETree** listaNodos, int cantNodos) (mdgpu.cu:1394)
 * receives the permuted lower triangle, the pre-sized spL (spL->p = the
 * column counts' prefix sums, mdgpu.cu:1859-1875) and the postordered
 * supernode list; it must fill spL->i and spL->x.  Here the whole numeric
 * phase goes through the C ABI: mdgpu_analyze_tree builds the plan from the
 * given tree, mdgpu_factor factors on the GPU, mdgpu_get_L writes L in the
 * reference's layout (rows ascending, diagonal first).  Errors print the
 * library's message and exit, as the reference does (cutil.h:9-35).
 *
 * The value type follows the reference's FLOTANTE (types.h:4-24).  In its
 * FP64 build the values pass straight through and the factor is FP64.  In
 * its default build (FLOTANTE float) the shim widens A->x to double for the
 * C ABI, factors in FP32 (the reference's precision; 3xTF32 tensor-core Schur
 * updates), and narrows L back to float into spL->x.
 */
#include <stdio.h>
#include <stdlib.h>

#include <map>
#include <vector>

#include "cs.h"
#include "etree.h"
#include "mdgpu_b200.h"

static void check(int rc, const char* what) {
    if (rc != MDGPU_OK) {
        fprintf(stderr, "%s: %s (%d): %s\n", what, mdgpu_status_string(rc), rc,
                mdgpu_last_error());
        exit(3);
    }
}

// FP64 build: the values pass straight through, FP64 factor
static void numeric(mdgpu_handle h, int nnz, const double* Ax, int lnz, int* Li, double* Lx,
                    long long* Lp) {
    (void)nnz;
    (void)lnz;
    check(mdgpu_factor(h, Ax, MDGPU_FP64, NULL), "mdgpu_factor");
    check(mdgpu_get_L(h, Lp, Li, Lx), "mdgpu_get_L");
}

// default (FP32) build: widen A, FP32 factor, narrow L
static void numeric(mdgpu_handle h, int nnz, const float* Ax, int lnz, int* Li, float* Lx,
                    long long* Lp) {
    std::vector<double> ax(Ax, Ax + nnz), lx(lnz > 0 ? lnz : 1);
    check(mdgpu_factor(h, ax.data(), MDGPU_FP32, NULL), "mdgpu_factor");
    check(mdgpu_get_L(h, Lp, Li, lx.data()), "mdgpu_get_L");
    for (int q = 0; q < lnz; q++) Lx[q] = (float)lx[q];
}

void Factor(cs* A, cs* spL, struct ETree** lista, int cant) {
    std::map<struct ETree*, int> pos;
    for (int s = 0; s < cant; s++) pos[lista[s]] = s;
    std::vector<int> first(cant), ncols(cant), cptr(cant + 1, 0), child, count(A->n);
    for (int s = 0; s < cant; s++) {
        first[s] = lista[s]->nodo;
        ncols[s] = lista[s]->cols;
        cptr[s + 1] = cptr[s] + lista[s]->nHijos;
        for (int h = 0; h < lista[s]->nHijos; h++) child.push_back(pos[lista[s]->hijos[h]]);
    }
    for (int j = 0; j < A->n; j++) count[j] = spL->p[j + 1] - spL->p[j];
    mdgpu_handle h = NULL;
    check(mdgpu_analyze_tree(A->n, A->p, A->i, cant, first.data(), ncols.data(), cptr.data(),
                             child.data(), count.data(), &h),
          "mdgpu_analyze_tree");
    std::vector<long long> Lp(A->n + 1);
    numeric(h, A->p[A->n], A->x, spL->p[A->n], spL->i, spL->x, Lp.data());
    mdgpu_destroy(h);
}
