"""The BF16 factor (MDGPU_BF16) and the FP64 safeguard for weak pivots (-m gpu).

* BF16 Schur updates (tcgen05 kind::f16, BF16 operands rounded to nearest
  even, FP32 accumulation): the factor's error against the oracle's FP64 L
  lies between the FP32 factor's and that of a dense blocked Cholesky whose
  every trailing update takes BF16 operands (oracle.rounded_update_cholesky
  with BF16 rounding, the upper bound: here only the large fronts' Schur
  updates are BF16); it is far above the FP32 factor's, so the BF16 path is
  in use.  GMRES-IR on it reaches backward error 1e-14 (elasticity system).
* Weak pivots: on a nearly singular system (shift 1e-8) the last pivots
  lose far more than ten bits to cancellation; those diagonal tiles are
  factored again in FP64 (mdgpu_info "fp64_diag_tiles" > 0) and GMRES-IR on
  the FP32 factor reaches backward error 1e-14.
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


def _round_bf16_f32(a):
    return O.round_bf16(a).astype(np.float32)


def test_bf16_factor_error_between_fp32_and_dense_bf16():
    n, Ap, Ai, Ax = mg.laplacian_3d_varcoef(16, seed=0, sigma=0.5, shift=1e-2)
    S = M.Solver(n, Ap, Ai)
    assert S.info("large_fronts") > 0
    P = O.Plan(n, Ap, Ai, Ax, amd=True, mode="sn")
    ref = P.factor()
    S.factor(Ax, M.FP32)
    e32 = _rel_fro(S.get_L()[2], ref["Lx"])
    S.factor(Ax, M.BF16)
    assert S.info("precision_used") == M.BF16
    _, Li, Lx = S.get_L()
    np.testing.assert_array_equal(Li, ref["Li"])
    ebf = _rel_fro(Lx, ref["Lx"])
    perm = S.array("perm")
    Ad = mg.lower_to_full_scipy(n, Ap, Ai, Ax).toarray()[np.ix_(perm, perm)]
    L64 = np.linalg.cholesky(Ad)
    e_dense = _rel_fro(O.rounded_update_cholesky(Ad, rounding=_round_bf16_f32), L64)
    assert ebf <= 3.0 * e_dense, (ebf, e_dense)
    assert ebf >= 30.0 * e32, (ebf, e32)


def test_bf16_factor_with_gmres_ir_reaches_fp64_accuracy():
    n, Ap, Ai, Ax = mg.elasticity_3dof(8, seed=0, sigma=1.0, shift=1e-2)
    S = M.Solver(n, Ap, Ai)
    assert S.info("large_fronts") > 0
    S.factor(Ax, M.BF16)
    b = mg.rhs_uniform(n, seed=4)
    x, berr, it, inner = S.gmres_ir(b, tol=1e-14, maxit=10)
    assert np.max(berr) <= 1e-14, (berr, it, inner)
    assert O.residual(n, Ap, Ai, Ax, x, b) <= 1e-14
    S64 = M.Solver(n, Ap, Ai)
    S64.factor(Ax, M.FP64)
    x64 = S64.solve(b)
    assert np.abs(x - x64).max() / np.abs(x64).max() <= 1e-9


def test_weak_pivots_refactored_in_fp64():
    n, Ap, Ai, Ax = mg.laplacian_3d_varcoef(14, seed=1, sigma=0.5, shift=1e-8)
    S = M.Solver(n, Ap, Ai)
    assert S.info("large_fronts") > 0
    S.factor(Ax, M.FP32)
    assert S.info("fp64_diag_tiles") > 0
    b = mg.rhs_uniform(n, seed=5)
    x, berr, it, inner = S.gmres_ir(b, tol=1e-14, maxit=10)
    assert np.max(berr) <= 1e-14, (berr, it, inner)
    # a well-conditioned system keeps every diagonal tile in FP32
    n2, Ap2, Ai2, Ax2 = mg.laplacian_3d_varcoef(14, seed=1, sigma=0.5, shift=1.0)
    S2 = M.Solver(n2, Ap2, Ai2)
    S2.factor(Ax2, M.FP32)
    assert S2.info("fp64_diag_tiles") == 0
