"""ctypes front-end of the oracle (liboracle.so) -- TEST INFRASTRUCTURE ONLY.

Only the tests, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` may import this module; the product never does.  ``run`` mirrors
the reference driver (mdgpu.cu:1745-1972) on a lower-triangular CSC matrix and
returns every intermediate the parity tests compare.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
REF_HARNESS = os.path.join(HERE, "_ref", "mdgpu_ref_harness")

MODES = {"nodal": 0, "sn": 1, "rn": 2}

_lib = None


def build():
    """Compile the restatement with gcc (oracle/Makefile)."""
    subprocess.check_call(["make", "-s", "-C", HERE, "liboracle.so"])


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH) or os.path.getmtime(LIB_PATH) < os.path.getmtime(
            os.path.join(HERE, "mdgpu_oracle.c")
        ):
            build()
        L = C.CDLL(LIB_PATH)
        i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
        f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
        L.orc_analyze.argtypes = [C.c_int, i32p, i32p, f64p, C.c_int, C.c_int, C.c_int,
                                  C.POINTER(C.c_void_p)]
        L.orc_analyze.restype = C.c_int
        L.orc_plan_free.argtypes = [C.c_void_p]
        for f in ("orc_plan_n", "orc_plan_nsuper", "orc_plan_nchild_total", "orc_plan_nnz_low"):
            getattr(L, f).argtypes = [C.c_void_p]
            getattr(L, f).restype = C.c_int
        L.orc_plan_lnz.argtypes = [C.c_void_p]
        L.orc_plan_lnz.restype = C.c_longlong
        L.orc_plan_copy.argtypes = [C.c_void_p, C.c_char_p, C.c_void_p]
        L.orc_factor.argtypes = [C.c_void_p, C.c_int, i32p, f64p, C.POINTER(C.c_double),
                                 C.c_void_p, C.c_void_p, C.c_void_p]
        L.orc_factor.restype = C.c_int
        L.orc_solve.argtypes = [C.c_void_p, i32p, f64p, f64p, f64p]
        L.orc_residual.argtypes = [C.c_int, i32p, i32p, f64p, f64p, f64p]
        L.orc_residual.restype = C.c_double
        L.orc_amd.argtypes = [C.c_int, i32p, i32p, i32p]
        L.orc_etree.argtypes = [C.c_int, i32p, i32p, i32p]
        L.orc_post.argtypes = [C.c_int, i32p, i32p]
        L.orc_counts.argtypes = [C.c_int, i32p, i32p, i32p, i32p, i32p]
        L.orc_front_factor.argtypes = [C.c_int, C.c_int, C.c_int, f64p]
        _lib = L
    return _lib


class Plan:
    """Owns an orc_plan*; fields are copied out as numpy arrays."""

    def __init__(self, n, Ap, Ai, Ax, amd=True, mode="sn", rn_zeros=0):
        L = lib()
        self._p = C.c_void_p()
        rc = L.orc_analyze(int(n), np.ascontiguousarray(Ap, np.int32),
                           np.ascontiguousarray(Ai, np.int32),
                           np.ascontiguousarray(Ax, np.float64), int(bool(amd)), MODES[mode],
                           int(rn_zeros), C.byref(self._p))
        if rc != 0:
            raise ValueError("oracle analyze failed (%d)" % rc)
        self.n = L.orc_plan_n(self._p)
        self.nsuper = L.orc_plan_nsuper(self._p)
        self.lnz = L.orc_plan_lnz(self._p)
        nk = L.orc_plan_nchild_total(self._p)
        nnz = L.orc_plan_nnz_low(self._p)
        n, ns = self.n, self.nsuper
        sizes = {"perm": n, "parent": n, "post": n, "count0": n, "count": n, "rn_perm": n,
                 "sn_nodo": ns, "sn_cols": ns, "sn_childptr": ns + 1, "sn_child": nk,
                 "Lp": n + 1, "Ap": n + 1, "Ai": nnz}
        self.has_perm = bool(amd) or mode == "rn"
        for k, sz in sizes.items():
            if k == "perm" and not self.has_perm:
                setattr(self, k, None)
                continue
            if k == "rn_perm" and mode != "rn":
                setattr(self, k, None)
                continue
            a = np.zeros(max(sz, 1), np.int32)
            L.orc_plan_copy(self._p, k.encode(), a.ctypes.data)
            setattr(self, k, a[:sz])
        self.Ax = np.zeros(max(nnz, 1), np.float64)
        L.orc_plan_copy(self._p, b"Ax", self.Ax.ctypes.data)
        self.Ax = self.Ax[:nnz]

    def factor(self, block_size=0, maps=False):
        L = lib()
        Li = np.zeros(max(self.lnz, 1), np.int32)
        Lx = np.zeros(max(self.lnz, 1), np.float64)
        flops = C.c_double()
        rows_ptr = rows = relmap = None
        args = [None, None, None]
        if maps:
            rows_ptr = np.zeros(self.nsuper + 1, np.int32)
            tot = int(sum(self.count[self.sn_nodo]))
            rows = np.zeros(max(tot, 1), np.int32)
            relmap = np.zeros(max(tot, 1), np.int32)
            args = [rows_ptr.ctypes.data, rows.ctypes.data, relmap.ctypes.data]
        rc = L.orc_factor(self._p, int(block_size), Li, Lx, C.byref(flops), *args)
        out = {"Li": Li[: self.lnz], "Lx": Lx[: self.lnz], "flops": flops.value, "status": rc}
        if maps:
            out.update(rows_ptr=rows_ptr, rows=rows[: rows_ptr[-1]], relmap=relmap[: rows_ptr[-1]])
        return out

    def solve(self, Li, Lx, b):
        x = np.zeros(self.n, np.float64)
        lib().orc_solve(self._p, np.ascontiguousarray(Li, np.int32),
                        np.ascontiguousarray(Lx, np.float64),
                        np.ascontiguousarray(b, np.float64), x)
        return x

    def __del__(self):
        try:
            if self._p:
                lib().orc_plan_free(self._p)
        except Exception:
            pass


def residual(n, Ap, Ai, Ax, x, b):
    return lib().orc_residual(int(n), np.ascontiguousarray(Ap, np.int32),
                              np.ascontiguousarray(Ai, np.int32),
                              np.ascontiguousarray(Ax, np.float64),
                              np.ascontiguousarray(x, np.float64),
                              np.ascontiguousarray(b, np.float64))


def front_factor(F, cols, block_size=0):
    """Dense partial Cholesky of one column-major square front (in place copy)."""
    F = np.array(F, dtype=np.float64, order="F")
    n = F.shape[0]
    buf = np.ascontiguousarray(F.T).ravel()  # column-major flattening
    lib().orc_front_factor(n, int(cols), int(block_size), buf)
    return buf.reshape(n, n).T


def run_reference(matrix_file, outdir, amd=True, mode="sn", rn_zeros=0, block=0, bfile=None,
                  factor=True, timeout=None):
    """Run the compiled reference (oracle/_ref) and load its outputs."""
    args = [REF_HARNESS]
    if amd:
        args.append("-amd")
    if mode == "sn":
        args.append("-sn")
    elif mode == "rn":
        args += ["-rn", str(rn_zeros)]
    if block:
        args += ["-b", str(block)]
    if not factor:
        args.append("-nofactor")
    if bfile:
        args += ["-bfile", bfile]
    args += [matrix_file, outdir]
    os.makedirs(outdir, exist_ok=True)
    subprocess.run(args, check=True, capture_output=True, timeout=timeout)
    return load_dir(outdir)


def load_dir(d):
    import json

    out = {}
    for f in os.listdir(d):
        p = os.path.join(d, f)
        if f.endswith(".i32"):
            out[f[:-4]] = np.fromfile(p, dtype=np.int32)
        elif f.endswith(".f64"):
            out[f[:-4]] = np.fromfile(p, dtype=np.float64)
        elif f == "meta.json":
            with open(p) as fh:
                out["meta"] = json.load(fh)
    return out


def selected_inverse(n, Lp, Li, Lx):
    """Z = A^-1 on the pattern of L (and its transpose) from the CSC factor
    A = L L' (rows ascending, diagonal first): the Takahashi recurrence,
    column by column from the last --
        y = L(R, j) / L(j, j),  Z(R, j) = -Z(R, R) y,
        Z(j, j) = 1 / L(j, j)^2 - y' Z(R, j)
    with R the rows below the diagonal of column j (a clique of the filled
    graph, so Z(R, R) lies on the pattern).  Dense n x n storage: for the
    small test sizes only.  TEST INFRASTRUCTURE ONLY."""
    Z = np.zeros((n, n))
    for j in range(n - 1, -1, -1):
        p0, p1 = int(Lp[j]), int(Lp[j + 1])
        d = Lx[p0]
        R = np.asarray(Li[p0 + 1:p1], dtype=np.int64)
        y = Lx[p0 + 1:p1] / d
        zr = -Z[np.ix_(R, R)] @ y
        Z[R, j] = zr
        Z[j, R] = zr
        Z[j, j] = 1.0 / (d * d) - y @ zr
    return Z


def gmres_ir(matvec, precond, b, anorm, tol=1e-14, maxit=10, restart=30, inner_tol=1e-10):
    """GMRES-based iterative refinement, restated from Carson & Higham,
    "Accelerating the solution of linear systems by iterative refinement in
    three precisions", SIAM J. Sci. Comput. 40(2), A817-A847 (2018),
    Algorithm 3.1, with the working and residual precisions both FP64:

        x = M^-1 b
        repeat: r = b - A x;  stop when ||r||inf / (anorm ||x||inf + ||b||inf)
                <= tol or after maxit corrections;
                solve M^-1 A d = M^-1 r by GMRES (zero start, at most
                `restart` steps, stop when the preconditioned residual falls
                to inner_tol times its start);  x += d

    where M^-1 applies the low-precision factor.  The Arnoldi basis is
    orthogonalised by classical Gram-Schmidt applied twice, the Hessenberg
    matrix reduced by Givens rotations as it grows.  matvec(v) = A v and
    precond(r) = M^-1 r take and return FP64 vectors.  Returns (x, berr
    history, inner step counts).  TEST INFRASTRUCTURE ONLY."""
    b = np.asarray(b, np.float64)
    n = b.size
    x = precond(b)
    hist, inner = [], []
    for outer in range(maxit + 1):
        r = b - matvec(x)
        den = anorm * np.abs(x).max() + np.abs(b).max()
        be = np.abs(r).max() / den if den > 0 else 0.0
        hist.append(be)
        if be <= tol or outer == maxit:
            break
        z = precond(r)
        beta = np.sqrt(z @ z)
        if beta == 0.0:
            break
        V = np.zeros((n, restart + 1))
        H = np.zeros((restart + 1, restart))
        cs, sn = np.zeros(restart), np.zeros(restart)
        g = np.zeros(restart + 1)
        g[0] = beta
        V[:, 0] = z / beta
        k = 0
        for j in range(restart):
            w = precond(matvec(V[:, j]))
            h1 = V[:, :j + 1].T @ w
            w = w - V[:, :j + 1] @ h1
            h2 = V[:, :j + 1].T @ w
            w = w - V[:, :j + 1] @ h2
            H[:j + 1, j] = h1 + h2
            hn = np.sqrt(w @ w)
            H[j + 1, j] = hn
            for i in range(j):
                t = cs[i] * H[i, j] + sn[i] * H[i + 1, j]
                H[i + 1, j] = -sn[i] * H[i, j] + cs[i] * H[i + 1, j]
                H[i, j] = t
            den2 = np.hypot(H[j, j], H[j + 1, j])
            cs[j], sn[j] = H[j, j] / den2, H[j + 1, j] / den2
            H[j, j] = den2
            H[j + 1, j] = 0.0
            g[j + 1] = -sn[j] * g[j]
            g[j] = cs[j] * g[j]
            k = j + 1
            if abs(g[j + 1]) <= inner_tol * beta or hn == 0.0:
                break
            V[:, j + 1] = w / hn
        y = np.zeros(k)
        for i in range(k - 1, -1, -1):
            y[i] = (g[i] - H[i, i + 1:k] @ y[i + 1:k]) / H[i, i]
        x = x + V[:, :k] @ y
        inner.append(k)
    return x, hist, inner


def round_bf16(a):
    """Round FP64 values to the nearest BF16 (8 significant bits, ties to
    even), returned as FP64: the factor a BF16 tensor-core path would keep.
    TEST INFRASTRUCTURE ONLY."""
    u = np.asarray(a, np.float32).copy().view(np.uint32)
    u += np.uint32(0x7FFF) + ((u >> np.uint32(16)) & np.uint32(1))
    u &= np.uint32(0xFFFF0000)
    return u.view(np.float32).astype(np.float64)


def truncate_tf32(a):
    """FP32 values with the low 13 mantissa bits cleared (an exact TF32
    value, rounded toward zero): the operand a TF32 tensor-core product reads
    from an FP32 register, and the 'hi' part of a 3xTF32 split.  TEST
    INFRASTRUCTURE ONLY."""
    u = np.asarray(a, np.float32).copy().view(np.uint32)
    u &= np.uint32(0xFFFFE000)
    return u.view(np.float32)


def rounded_update_cholesky(A, nb=64, rounding=None):
    """Dense right-looking blocked Cholesky in FP32 whose trailing (Schur)
    updates take their operands through `rounding` (an FP32 -> FP32 map; None:
    plain FP32 products) and accumulate in FP32; the diagonal-block factor and
    the panel solve stay in FP32.  rounding=truncate_tf32 is a 1xTF32
    tensor-core Schur update, None the FP32 arithmetic a 3xTF32 update
    approaches.  Returns the lower factor in FP64.  TEST INFRASTRUCTURE ONLY."""
    import scipy.linalg as sl

    W = np.array(A, dtype=np.float32)
    n = W.shape[0]
    for k in range(0, n, nb):
        e = min(k + nb, n)
        L11 = np.linalg.cholesky(W[k:e, k:e].astype(np.float64)).astype(np.float32)
        W[k:e, k:e] = L11
        if e < n:
            L21 = sl.solve_triangular(L11, W[e:, k:e].T, lower=True).T.astype(np.float32)
            W[e:, k:e] = L21
            Q = L21 if rounding is None else rounding(L21)
            W[e:, e:] -= Q @ Q.T
    return np.tril(W).astype(np.float64)


def bf16_update_cholesky(A, nb=64, pow2_scale=False):
    """Dense right-looking blocked Cholesky in FP32 whose trailing (Schur)
    updates take their operands rounded to BF16 and accumulate in FP32 -- the
    arithmetic of a BF16 tensor-core Schur update (A22 -= L21 L21' with BF16
    inputs, FP32 accumulators); the diagonal-block factor and the panel solve
    stay in FP32.  pow2_scale: before rounding, each panel is multiplied by
    the power of two that brings its largest magnitude into [1, 2) and the
    product is scaled back (per-front power-of-two scaling).  Returns the
    lower factor in FP64.  TEST INFRASTRUCTURE ONLY."""
    import scipy.linalg as sl

    W = np.array(A, dtype=np.float32)
    n = W.shape[0]
    for k in range(0, n, nb):
        e = min(k + nb, n)
        L11 = np.linalg.cholesky(W[k:e, k:e].astype(np.float64)).astype(np.float32)
        W[k:e, k:e] = L11
        if e < n:
            L21 = sl.solve_triangular(L11, W[e:, k:e].T, lower=True).T.astype(np.float32)
            W[e:, k:e] = L21
            s = 1.0
            if pow2_scale:
                mx = float(np.abs(L21).max())
                if mx > 0:
                    s = 2.0 ** -np.floor(np.log2(mx))
            Q = (round_bf16(L21 * np.float32(s))).astype(np.float32)
            W[e:, e:] -= (Q @ Q.T) * np.float32(1.0 / (s * s))
    return np.tril(W).astype(np.float64)


def cholesky_adjoint_dense(L, Lbar):
    """Reverse mode of the Cholesky factorization A = L L' (dense, FP64):
    given L and Lbar (the loss's gradient with respect to the entries of the
    lower triangle of L), the gradient with respect to the entries of the
    lower triangle of A, each stored entry a free variable (an off-diagonal
    one stands for A(i, j) and A(j, i)).  With Phi(X) = the lower triangle
    of X with its diagonal halved (Murray 2016, "Differentiation of the
    Cholesky decomposition"):
        P = Phi(L' Lbar),  S = L^-T P L^-1,
        Abar = tril(S + S') with the diagonal S(i, i).
    TEST INFRASTRUCTURE ONLY."""
    import scipy.linalg as sl

    L = np.asarray(L, dtype=np.float64)
    Lb = np.tril(np.asarray(Lbar, dtype=np.float64))
    P = np.tril(L.T @ Lb)
    P[np.diag_indices_from(P)] *= 0.5
    X = sl.solve_triangular(L, P.T, lower=True, trans="T").T  # X = P L^-1 (L' X' = P')
    S = sl.solve_triangular(L, X, lower=True, trans="T")        # L^-T X
    G = np.tril(S + S.T)
    G[np.diag_indices_from(G)] = np.diag(S)
    return G
