// GMRES-based iterative refinement (GMRES-IR) of one right-hand side.
//
// Carson & Higham, "Accelerating the solution of linear systems by iterative
// refinement in three precisions", SIAM J. Sci. Comput. 40(2), A817-A847
// (2018), Algorithm 3.1, with the working and residual precisions FP64 and
// the factor's precision (FP32, later BF16) as the low one:
//
//     x = M^-1 b
//     repeat: r = b - A x;  stop when the backward error
//             ||r||inf / (||A||inf ||x||inf + ||b||inf) <= tol, or after
//             maxit corrections;
//             solve M^-1 A d = M^-1 r by GMRES from d = 0 (at most `restart`
//             steps; stop when the preconditioned residual falls to
//             inner_tol times its start);  x += d
//
// M^-1 is the solve with the current (low-precision) factor.  Plain
// refinement (x += M^-1 r) converges only while cond(A) u_factor < 1; GMRES
// on the preconditioned system converges for cond(A) up to about u_factor^-2,
// which is what a BF16 factor needs.  The Arnoldi basis is orthogonalised by
// classical Gram-Schmidt applied twice (two block passes per step, no
// dependent dot-product chain), the Hessenberg matrix is reduced by Givens
// rotations as it grows, so its last entry is the residual norm of the
// preconditioned system.
//
// The driver is written once over a vector-operations backend `Ops` (all
// vectors length n, FP64, in the backend's memory):
//     double* basis(int k)           vector k of the Arnoldi basis, k <= restart
//     double* scratch()              one more vector
//     void residual(x, b, r)         r = b - A x with the caller's FP64 A
//     double backward_error(r, x, b) the stopping measure above
//     void precond(r, z)             z = M^-1 r (r is not modified)
//     void spmv(v, w)                w = A v
//     void dots(k, w, s)             slot s (0 or 1) [i] = <basis(i), w>, i < k
//     void sub(k, s, w)              w -= sum_i slot s [i] basis(i)
//     void norm2_to_slot(w)          the norm slot = <w, w>
//     void fetch(double* host)       the slots to the host, laid out as
//                                    [slot 0 (restart), slot 1 (restart), norm]
//     void scale(alpha, w)           w *= alpha
//     void add(k, y, x)              x += sum_i y[i] basis(i), y on the host
// The slots live in the backend, so a device backend keeps the Arnoldi step
// on the device and copies back once per step.
#pragma once

#include <algorithm>
#include <cmath>
#include <vector>

namespace mdgpu {

struct GmresIrParams {
    double tol = 1e-14;        // backward error to reach
    int maxit = 10;            // corrections at most
    int restart = 30;          // GMRES steps per correction at most
    double inner_tol = 1e-8;   // GMRES stop: preconditioned residual / its start
};

struct GmresIrResult {
    double berr = 0.0;  // final backward error
    int outer = 0;      // corrections applied
    int inner = 0;      // GMRES steps over all corrections
};

constexpr int kGmresMaxRestart = 64;

// x: on entry ignored, on exit the solution; b: right-hand side.
template <class Ops>
GmresIrResult gmres_ir(Ops& ops, double* x, const double* b, const GmresIrParams& p) {
    const int kmax = p.restart;
    GmresIrResult res;
    std::vector<double> H((size_t)(kmax + 1) * kmax), cs(kmax), sn(kmax), g(kmax + 1), y(kmax);
    std::vector<double> slots(2 * (size_t)kmax + 1);
    auto h_at = [&](int i, int j) -> double& { return H[(size_t)j * (kmax + 1) + i]; };
    double* r = ops.scratch();
    ops.precond(b, x);
    for (int outer = 0;; ++outer) {
        ops.residual(x, b, r);
        res.berr = ops.backward_error(r, x, b);
        res.outer = outer;
        if (!(res.berr > p.tol) || outer >= p.maxit) break;
        // the preconditioned residual starts the basis
        double* v0 = ops.basis(0);
        ops.precond(r, v0);
        ops.norm2_to_slot(v0);
        ops.fetch(slots.data());
        const double beta = std::sqrt(slots[2 * kmax]);
        if (!(beta > 0.0) || !std::isfinite(beta)) break;
        ops.scale(1.0 / beta, v0);
        std::fill(g.begin(), g.end(), 0.0);
        g[0] = beta;
        int k = 0;
        for (int j = 0; j < kmax; ++j) {
            // w = M^-1 A v_j, built in the next basis slot
            double* w = ops.basis(j + 1);
            ops.spmv(ops.basis(j), r);
            ops.precond(r, w);
            ops.dots(j + 1, w, 0);
            ops.sub(j + 1, 0, w);
            ops.dots(j + 1, w, 1);
            ops.sub(j + 1, 1, w);
            ops.norm2_to_slot(w);
            ops.fetch(slots.data());
            for (int i = 0; i <= j; ++i) h_at(i, j) = slots[i] + slots[kmax + i];
            const double hn = std::sqrt(slots[2 * kmax]);
            h_at(j + 1, j) = hn;
            for (int i = 0; i < j; ++i) {
                const double t = cs[i] * h_at(i, j) + sn[i] * h_at(i + 1, j);
                h_at(i + 1, j) = -sn[i] * h_at(i, j) + cs[i] * h_at(i + 1, j);
                h_at(i, j) = t;
            }
            const double d = std::hypot(h_at(j, j), h_at(j + 1, j));
            if (!(d > 0.0)) break;  // M^-1 A singular on the basis: keep k = j
            cs[j] = h_at(j, j) / d;
            sn[j] = h_at(j + 1, j) / d;
            h_at(j, j) = d;
            h_at(j + 1, j) = 0.0;
            g[j + 1] = -sn[j] * g[j];
            g[j] = cs[j] * g[j];
            k = j + 1;
            if (std::fabs(g[j + 1]) <= p.inner_tol * beta || !(hn > 0.0)) break;
            ops.scale(1.0 / hn, w);
        }
        // d = V_k y with H(0:k, 0:k) y = g(0:k), upper triangular
        for (int i = k - 1; i >= 0; --i) {
            double s = g[i];
            for (int c = i + 1; c < k; ++c) s -= h_at(i, c) * y[c];
            y[i] = s / h_at(i, i);
        }
        ops.add(k, y.data(), x);
        res.inner += k;
    }
    return res;
}

}  // namespace mdgpu
