"""The one-product TF32 factor (MDGPU_TF32, -m gpu).

Its large fronts' Schur updates are one tcgen05 kind::tf32 product of the
panel's hi parts (the FP32 values with the low 13 mantissa bits cleared),
FP32 accumulation.  The factor's error against the oracle's FP64 L lies
between the 3xTF32 factor's and that of a dense blocked Cholesky whose every
trailing update takes truncated TF32 operands (oracle.rounded_update_cholesky
with oracle.truncate_tf32, the upper bound: here only the large fronts' Schur
updates drop the bits); it is far above the 3xTF32 factor's, so the one-product
path is in use.  GMRES-IR on it reaches backward error 1e-14.
"""
import numpy as np
import pytest

import mdgpu_b200 as M
from mdgpu_b200 import matgen as mg
from oracle import oracle as O

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover - collected only on GPU boxes
    pytest.skip("needs a CUDA device", allow_module_level=True)


def _rel_fro(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def _truncate_tf32_f32(a):
    return O.truncate_tf32(np.asarray(a, dtype=np.float32)).astype(np.float32)


def test_tf32_factor_error_between_3xtf32_and_dense_tf32():
    n, Ap, Ai, Ax = mg.laplacian_3d_varcoef(16, seed=0, sigma=0.5, shift=1e-2)
    S = M.Solver(n, Ap, Ai)
    assert S.info("large_fronts") > 0
    P = O.Plan(n, Ap, Ai, Ax, amd=True, mode="sn")
    ref = P.factor()
    S.factor(Ax, M.FP32)
    e32 = _rel_fro(S.get_L()[2], ref["Lx"])
    S.factor(Ax, M.TF32)
    assert S.info("precision_used") == M.TF32
    _, Li, Lx = S.get_L()
    np.testing.assert_array_equal(Li, ref["Li"])
    etf = _rel_fro(Lx, ref["Lx"])
    perm = S.array("perm")
    Ad = mg.lower_to_full_scipy(n, Ap, Ai, Ax).toarray()[np.ix_(perm, perm)]
    L64 = np.linalg.cholesky(Ad)
    e_dense = _rel_fro(O.rounded_update_cholesky(Ad, rounding=_truncate_tf32_f32), L64)
    assert etf <= 3.0 * e_dense, (etf, e_dense)
    assert etf >= 30.0 * e32, (etf, e32)


def test_tf32_factor_with_gmres_ir_reaches_fp64_accuracy():
    n, Ap, Ai, Ax = mg.laplacian_3d_varcoef(16, seed=2, sigma=1.0, shift=1e-3)
    S = M.Solver(n, Ap, Ai)
    assert S.info("large_fronts") > 0
    S.factor(Ax, M.TF32)
    b = mg.rhs_uniform(n, seed=4)
    x, berr, it, inner = S.gmres_ir(b, tol=1e-14, maxit=10)
    assert np.max(berr) <= 1e-14, (berr, it, inner)
    assert O.residual(n, Ap, Ai, Ax, x, b) <= 1e-14
    S64 = M.Solver(n, Ap, Ai)
    S64.factor(Ax, M.FP64)
    x64 = S64.solve(b)
    assert np.abs(x - x64).max() / np.abs(x64).max() <= 1e-9
