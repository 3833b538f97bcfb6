/*
 * Harness that drives the reference's own CPU path (test infrastructure only).
 *
 * It links the reference objects compiled from their sources as they lie (see
 * oracle/Makefile) and replays the reference driver's sequence:
 *   load + compress           mdgpu.cu:1724-1729  (cs_load, cs_compress)
 *   symbolic                  mdgpu.cu:1745-1875  (cs_amd, cs_symperm, make_sym,
 *                                                  cs_etree, cs_post, cs_counts,
 *                                                  GetETree, GetSuperETree /
 *                                                  GetRelaxedETree, spL->p)
 *   numeric factor            mdgpu.cu:1888-1890  (Factor with GPU = false)
 *   solve + residual          mdgpu.cu:1941-1973  (cs_pvec, cs_lsolve, cs_ltsolve,
 *                                                  cs_ipvec, cs_gaxpy, cs_norm)
 * with three fixes that make the reference's CPU path usable as an oracle,
 * each applied here rather than in the reference sources:
 *   - spL->x is allocated (its allocation is commented out at mdgpu.cu:1873,
 *     yet FactorAux_CPU_3 writes it at mdgpu.cu:1350);
 *   - the children of every supernode are put back in postorder after
 *     GetSuperETree (etree.cpp:93,101-103 stores the non-last children in
 *     reverse, which Factor's update-matrix stack at mdgpu.cu:1434-1440 cannot
 *     pair correctly); the supernode partition itself is untouched;
 *   - without -amd the solution vector is the un-permuted one (mdgpu.cu:1959-1961
 *     leaves x2 unwritten in that case).
 *
 * Usage: mdgpu_ref_harness [-amd] [-sn | -rn z] [-b bs] [-nofactor] [-bfile f]
 *                          <matrix triplet file> <output dir>
 * Outputs raw little-endian arrays (.i32 / .f64) and meta.json in <output dir>.
 * The scalar is the reference's FLOTANTE (types.h:4-24): double in the FP64
 * build, float in the reference's default build; values are written as f64
 * either way and the right-hand side file holds f64 values.
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>
#include <vector>
#include <map>
#include <string>
#include <algorithm>

#include "cs.h"
#include "etree.h"

extern bool GPU;
extern int block_size;
extern bool pad;
extern double flops;
void Factor(cs* A, cs* spL, struct ETree** listaNodos, int cantNodos);

static double now_s() {
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return ts.tv_sec + 1e-9 * ts.tv_nsec;
}

/* make_sym is file-static in mdgpu.cu:1630-1638; same three CSparse calls. */
typedef FLOTANTE Val;
static int keep_offdiag(int i, int j, Val, void*) { return i != j; }
static cs* sym_from_lower(cs* A) {
    cs* AT = cs_transpose(A, 1);
    cs_fkeep(AT, &keep_offdiag, NULL);
    cs* C = cs_add(A, AT, 1, 1);
    cs_spfree(AT);
    return C;
}

static double inf_norm(const Val* x, int n) {
    double m = 0;
    for (int i = 0; i < n; i++) m = std::max(m, fabs((double)x[i]));
    return m;
}

static std::string g_out;
static void dump(const char* name, const void* data, size_t bytes) {
    std::string path = g_out + "/" + name;
    FILE* f = fopen(path.c_str(), "wb");
    if (!f) { fprintf(stderr, "cannot write %s\n", path.c_str()); exit(2); }
    if (bytes) fwrite(data, 1, bytes, f);
    fclose(f);
}
static void dump_i32(const char* name, const int* v, size_t n) { dump(name, v, n * sizeof(int)); }
static void dump_f64(const char* name, const Val* v, size_t n) {
    std::vector<double> d(v, v + n);
    dump(name, d.data(), n * sizeof(double));
}

int main(int argc, char** argv) {
    bool amd = false, sn = false, rn = false, do_factor = true;
    int rn_zeros = 0;
    const char* bfile = NULL;
    int a = 1;
    for (; a < argc - 2; a++) {
        if (!strcmp(argv[a], "-amd")) amd = true;
        else if (!strcmp(argv[a], "-sn")) sn = true;
        else if (!strcmp(argv[a], "-rn")) { rn = true; rn_zeros = atoi(argv[++a]); }
        else if (!strcmp(argv[a], "-b")) block_size = atoi(argv[++a]);
        else if (!strcmp(argv[a], "-nofactor")) do_factor = false;
        else if (!strcmp(argv[a], "-bfile")) bfile = argv[++a];
        else { fprintf(stderr, "unknown flag %s\n", argv[a]); return 2; }
    }
    if (argc - a != 2) { fprintf(stderr, "usage: %s [flags] matrix outdir\n", argv[0]); return 2; }
    const char* mfile = argv[a];
    g_out = argv[a + 1];
    GPU = false;
    pad = false;

    double t0 = now_s();
    FILE* f = fopen(mfile, "r");
    if (!f) { fprintf(stderr, "cannot open %s\n", mfile); return 2; }
    cs* T = cs_load(f);
    fclose(f);
    cs* C_low = cs_compress(T);
    cs_spfree(T);
    double t_load = now_s() - t0;
    int n = C_low->n;

    /* ---- symbolic: mdgpu.cu:1745-1875 ---- */
    double t1 = now_s();
    cs* A_low = NULL;
    cs* A = NULL;
    int* amd_perm = NULL;
    if (amd) {
        cs* C_up = cs_transpose(C_low, 1);
        amd_perm = cs_amd(1, C_up);
        int* amd_pinv = cs_pinv(amd_perm, C_up->n);
        cs* A_amd_U = cs_symperm(C_up, amd_pinv, 1);
        cs_spfree(C_up);
        A_low = cs_transpose(A_amd_U, 1);
        cs_spfree(A_amd_U);
        free(amd_pinv);
    } else {
        A_low = C_low;
    }
    A = sym_from_lower(A_low);
    int* parent = cs_etree(A, 0);
    int* post = cs_post(parent, A->n);
    int* count = cs_counts(A, parent, post, 0);
    std::vector<int> count0(count, count + n);

    struct ETree** listaNodos;
    int cantNodos;
    GetETree(A, parent, post, count, &listaNodos, &cantNodos);
    struct ETree** lista;
    int cant;
    if (sn) {
        GetSuperETree(listaNodos, cantNodos, &lista, &cant);
    } else {
        lista = listaNodos;
        cant = cantNodos;
    }
    std::vector<int> rn_perm;
    if (rn) {
        int* permR;
        GetRelaxedETree(listaNodos, cantNodos, rn_zeros, count, &permR, &lista, &cant);
        int* ipermR = cs_pinv(permR, cantNodos);
        cs* tmp1 = cs_transpose(A_low, 1);
        cs* tmp2 = cs_symperm(tmp1, ipermR, 1);
        cs_spfree(tmp1);
        cs* A_low2 = cs_transpose(tmp2, 1);
        cs_spfree(tmp2);
        if (A_low != C_low) cs_spfree(A_low);
        A_low = A_low2;
        int* count2 = (int*)malloc(cantNodos * sizeof(int));
        cs_pvec(permR, count, count2, cantNodos);
        count = count2;
        if (amd_perm) {
            int* amd_perm2 = (int*)malloc(cantNodos * sizeof(int));
            cs_pvec(permR, amd_perm, amd_perm2, cantNodos);
            amd_perm = amd_perm2;
        } else {
            /* without -amd the reference applies no amd_perm; record the
               relaxed permutation as the overall one */
            amd_perm = (int*)malloc(cantNodos * sizeof(int));
            memcpy(amd_perm, permR, cantNodos * sizeof(int));
        }
        rn_perm.assign(permR, permR + cantNodos);
        free(ipermR);
    }
    /* put every node's children in postorder (see header) */
    std::map<struct ETree*, int> pos;
    for (int s = 0; s < cant; s++) pos[lista[s]] = s;
    for (int s = 0; s < cant; s++) {
        struct ETree* t = lista[s];
        std::sort(t->hijos, t->hijos + t->nHijos,
                  [&](struct ETree* x, struct ETree* y) { return pos[x] < pos[y]; });
    }

    cs* spL = (cs*)calloc(1, sizeof(cs));
    spL->n = A->n;
    spL->m = A->m;
    spL->p = (int*)malloc((spL->n + 1) * sizeof(int));
    long long nz = 0;
    for (int i = 0; i < spL->n; i++) { spL->p[i] = (int)nz; nz += count[i]; }
    spL->p[spL->n] = (int)nz;
    spL->nzmax = (int)nz;
    spL->nz = -1;
    spL->i = (int*)calloc(nz > 0 ? nz : 1, sizeof(int));
    spL->x = (Val*)calloc(nz > 0 ? nz : 1, sizeof(Val));
    double t_symbolic = now_s() - t1;

    /* ---- dump symbolic ---- */
    if (amd_perm) dump_i32("perm.i32", amd_perm, n);
    dump_i32("parent.i32", parent, n);
    dump_i32("post.i32", post, n);
    dump_i32("count0.i32", count0.data(), n);
    dump_i32("count.i32", count, n);
    if (rn) dump_i32("rn_perm.i32", rn_perm.data(), n);
    {
        std::vector<int> nodo(cant), cols(cant), cptr(cant + 1, 0), child;
        for (int s = 0; s < cant; s++) {
            nodo[s] = lista[s]->nodo;
            cols[s] = lista[s]->cols;
            cptr[s + 1] = cptr[s] + lista[s]->nHijos;
            for (int h = 0; h < lista[s]->nHijos; h++) child.push_back(pos[lista[s]->hijos[h]]);
        }
        dump_i32("sn_nodo.i32", nodo.data(), cant);
        dump_i32("sn_cols.i32", cols.data(), cant);
        dump_i32("sn_childptr.i32", cptr.data(), cant + 1);
        dump_i32("sn_child.i32", child.data(), child.size());
    }
    dump_i32("Lp.i32", spL->p, n + 1);
    /* permuted lower A as Factor sees it */
    dump_i32("Ap.i32", A_low->p, n + 1);
    dump_i32("Ai.i32", A_low->i, A_low->p[n]);
    dump_f64("Ax.f64", A_low->x, A_low->p[n]);

    double t_factor = 0, t_solve = 0, resid_rel = -1, resid_abs = -1;
    if (do_factor) {
        double t2 = now_s();
        Factor(A_low, spL, lista, cant);
        t_factor = now_s() - t2;
        dump_i32("Li.i32", spL->i, nz);
        dump_f64("Lx.f64", spL->x, nz);

        /* ---- solve + residual: mdgpu.cu:1941-1973 ---- */
        std::vector<Val> b(n), x(n), x2(n);
        if (bfile) {
            std::vector<double> bd(n);
            FILE* fb = fopen(bfile, "rb");
            if (!fb || fread(bd.data(), sizeof(double), n, fb) != (size_t)n) {
                fprintf(stderr, "cannot read %s\n", bfile);
                return 2;
            }
            fclose(fb);
            for (int i = 0; i < n; i++) b[i] = (Val)bd[i];
        } else {
            for (int i = 0; i < n; i++) b[i] = 1 + ((Val)i) / n;
        }
        double t3 = now_s();
        x = b;
        if (amd_perm) cs_pvec(amd_perm, b.data(), x.data(), n);
        cs_lsolve(spL, x.data());
        cs_ltsolve(spL, x.data());
        if (amd_perm) cs_ipvec(amd_perm, x.data(), x2.data(), n);
        else x2 = x;
        t_solve = now_s() - t3;
        std::vector<Val> r(n);
        for (int i = 0; i < n; i++) r[i] = -b[i];
        cs* C = sym_from_lower(C_low);
        cs_gaxpy(C, x2.data(), r.data());
        resid_abs = inf_norm(r.data(), n);
        resid_rel = resid_abs / (cs_norm(A) * inf_norm(x.data(), n) + inf_norm(b.data(), n));
        dump_f64("b.f64", b.data(), n);
        dump_f64("x.f64", x2.data(), n);
    }

    std::string meta = g_out + "/meta.json";
    FILE* fm = fopen(meta.c_str(), "w");
    fprintf(fm,
            "{\"n\": %d, \"nnz_low\": %d, \"lnz\": %lld, \"nsuper\": %d, \"flops\": %.17g, "
            "\"t_load\": %.9f, \"t_symbolic\": %.9f, \"t_factor\": %.9f, \"t_solve\": %.9f, "
            "\"resid_rel\": %.17g, \"resid_abs\": %.17g}\n",
            n, C_low->p[n], nz, cant, flops, t_load, t_symbolic, t_factor, t_solve, resid_rel,
            resid_abs);
    fclose(fm);
    printf("n=%d lnz=%lld nsuper=%d flops=%.6g factor=%.6fs solve=%.6fs resid=%.3e\n", n, nz,
           cant, flops, t_factor, t_solve, resid_rel);
    return 0;
}
