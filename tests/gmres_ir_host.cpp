// Host check of the GMRES-IR driver (mdgpu_b200/csrc/gmres_ir.hpp): the same
// template the library instantiates with its device vector operations, here
// over plain loops on the CPU, with a dense lower-triangular preconditioner
// factor given by the test.  Test infrastructure: compiled and run by
// tests/test_gmres_ir.py.
//
// Input (binary, native byte order): int32 n, restart, maxit, nnz; double
// tol, inner_tol; int32 rowptr[n + 1], col[nnz]; double val[nnz] (the full
// symmetric matrix, CSR); double L[n * n] (row-major lower triangle of the
// preconditioner factor, M = L L'); double b[n].
// Output (text): "outer inner berr", then the backward errors seen, then x.
#include <cmath>
#include <cstdio>
#include <vector>

#include "gmres_ir.hpp"

namespace {

struct HostOps {
    int n = 0, kmax = 0;
    std::vector<int> rp, ci;
    std::vector<double> va, L, V, tmp, y, slots, hist;
    double anorm = 0.0;

    double* basis(int k) { return V.data() + (size_t)k * n; }
    double* scratch() { return tmp.data(); }
    void residual(const double* x, const double* b, double* r) {
        for (int i = 0; i < n; ++i) {
            double s = 0.0;
            for (int p = rp[i]; p < rp[i + 1]; ++p) s += va[p] * x[ci[p]];
            r[i] = b[i] - s;
        }
    }
    double backward_error(const double* r, const double* x, const double* b) {
        double nr = 0.0, nx = 0.0, nb = 0.0;
        for (int i = 0; i < n; ++i) {
            nr = std::fmax(nr, std::fabs(r[i]));
            nx = std::fmax(nx, std::fabs(x[i]));
            nb = std::fmax(nb, std::fabs(b[i]));
        }
        const double den = anorm * nx + nb;
        const double be = den > 0 ? nr / den : 0.0;
        hist.push_back(be);
        return be;
    }
    void precond(const double* r, double* z) {
        for (int i = 0; i < n; ++i) {
            double s = r[i];
            for (int k = 0; k < i; ++k) s -= L[(size_t)i * n + k] * y[k];
            y[i] = s / L[(size_t)i * n + i];
        }
        for (int i = n - 1; i >= 0; --i) {
            double s = y[i];
            for (int k = i + 1; k < n; ++k) s -= L[(size_t)k * n + i] * z[k];
            z[i] = s / L[(size_t)i * n + i];
        }
    }
    void spmv(const double* v, double* w) {
        for (int i = 0; i < n; ++i) {
            double s = 0.0;
            for (int p = rp[i]; p < rp[i + 1]; ++p) s += va[p] * v[ci[p]];
            w[i] = s;
        }
    }
    void dots(int k, const double* w, int s) {
        for (int i = 0; i < k; ++i) {
            double a = 0.0;
            for (int r = 0; r < n; ++r) a += basis(i)[r] * w[r];
            slots[(size_t)s * kmax + i] = a;
        }
    }
    void sub(int k, int s, double* w) {
        for (int r = 0; r < n; ++r) {
            double a = 0.0;
            for (int i = 0; i < k; ++i) a += slots[(size_t)s * kmax + i] * basis(i)[r];
            w[r] -= a;
        }
    }
    void norm2_to_slot(const double* w) {
        double a = 0.0;
        for (int r = 0; r < n; ++r) a += w[r] * w[r];
        slots[2 * (size_t)kmax] = a;
    }
    void fetch(double* host) {
        for (size_t i = 0; i < slots.size(); ++i) host[i] = slots[i];
    }
    void scale(double alpha, double* w) {
        for (int r = 0; r < n; ++r) w[r] *= alpha;
    }
    void add(int k, const double* c, double* x) {
        for (int r = 0; r < n; ++r) {
            double a = 0.0;
            for (int i = 0; i < k; ++i) a += c[i] * basis(i)[r];
            x[r] += a;
        }
    }
};

template <typename T>
bool rd(FILE* f, T* p, size_t cnt) {
    return std::fread(p, sizeof(T), cnt, f) == cnt;
}

}  // namespace

int main(int argc, char** argv) {
    if (argc != 3) return 2;
    FILE* f = std::fopen(argv[1], "rb");
    if (!f) return 2;
    int hdr[4];
    double tols[2];
    if (!rd(f, hdr, 4) || !rd(f, tols, 2)) return 2;
    HostOps ops;
    const int n = hdr[0], nnz = hdr[3];
    mdgpu::GmresIrParams prm;
    prm.restart = hdr[1];
    prm.maxit = hdr[2];
    prm.tol = tols[0];
    prm.inner_tol = tols[1];
    ops.n = n;
    ops.kmax = prm.restart;
    ops.rp.resize(n + 1);
    ops.ci.resize(nnz);
    ops.va.resize(nnz);
    ops.L.resize((size_t)n * n);
    std::vector<double> b(n), x(n, 0.0);
    if (!rd(f, ops.rp.data(), n + 1) || !rd(f, ops.ci.data(), nnz) || !rd(f, ops.va.data(), nnz) ||
        !rd(f, ops.L.data(), (size_t)n * n) || !rd(f, b.data(), n))
        return 2;
    std::fclose(f);
    ops.V.assign((size_t)n * (prm.restart + 1), 0.0);
    ops.tmp.assign(n, 0.0);
    ops.y.assign(n, 0.0);
    ops.slots.assign(2 * (size_t)prm.restart + 1, 0.0);
    for (int i = 0; i < n; ++i) {
        double s = 0.0;
        for (int p = ops.rp[i]; p < ops.rp[i + 1]; ++p) s += std::fabs(ops.va[p]);
        ops.anorm = std::fmax(ops.anorm, s);
    }
    const mdgpu::GmresIrResult res = mdgpu::gmres_ir(ops, x.data(), b.data(), prm);
    FILE* o = std::fopen(argv[2], "w");
    if (!o) return 2;
    std::fprintf(o, "%d %d %.17g\n", res.outer, res.inner, res.berr);
    for (double h : ops.hist) std::fprintf(o, "%.17g ", h);
    std::fprintf(o, "\n");
    for (double v : x) std::fprintf(o, "%.17g\n", v);
    std::fclose(o);
    return 0;
}
