"""GPU parity: the CUDA factor and solves against the oracle (-m gpu).

Tolerances: FP64 factor L within 1e-12 relative Frobenius of the oracle's L
(the oracle is bit-identical to the reference's CPU path); FP64 solutions
within 1e-10 relative (inf-norm) and backward error <= 1e-14; an FP32 factor
with FP64 iterative refinement reaches backward error <= 1e-14.
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

TREE = {"nodal": M.TREE_NODAL, "sn": M.TREE_SUPER, "rn": M.TREE_RELAXED}

CASES = [
    ("2d100_amd_sn", lambda: mg.laplacian_2d_5pt(100), True, "sn", 0),
    ("2d100_amd_nodal", lambda: mg.laplacian_2d_5pt(100), True, "nodal", 0),
    ("2d60_nat_sn", lambda: mg.laplacian_2d_5pt(60), False, "sn", 0),
    ("2d100_amd_rn16", lambda: mg.laplacian_2d_5pt(100), True, "rn", 16),
    ("3d10_amd_sn", lambda: mg.laplacian_3d_varcoef(10, seed=0), True, "sn", 0),
    ("3d16_amd_sn", lambda: mg.laplacian_3d_varcoef(16, seed=0), True, "sn", 0),
    ("3d16_amd_rn4", lambda: mg.laplacian_3d_varcoef(16, seed=0), True, "rn", 4),
    ("3d20_amd_sn", lambda: mg.laplacian_3d_varcoef(20, seed=3), True, "sn", 0),
    ("rnd300_amd_sn", lambda: mg.random_spd(300, 0.02, seed=1), True, "sn", 0),
    ("rnd500_nat_nodal", lambda: mg.random_spd(500, 0.02, seed=2), False, "nodal", 0),
]


def _rel_fro(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


@pytest.mark.parametrize("name,gen,amd,mode,z", CASES, ids=[c[0] for c in CASES])
def test_fp64_factor_and_solve_match_oracle(name, gen, amd, mode, z):
    n, Ap, Ai, Ax = gen()
    P = O.Plan(n, Ap, Ai, Ax, amd=amd, mode=mode, rn_zeros=z)
    ref = P.factor()
    S = M.Solver(n, Ap, Ai, ordering=int(amd), tree=TREE[mode], relax_zeros=z)
    S.factor(Ax, M.FP64)
    Lp, Li, Lx = S.get_L()
    np.testing.assert_array_equal(Lp.astype(np.int32), P.Lp)
    np.testing.assert_array_equal(Li, ref["Li"])
    assert _rel_fro(Lx, ref["Lx"]) <= 1e-12
    b = mg.rhs_uniform(n, seed=0)
    x = S.solve(b)
    xr = P.solve(ref["Li"], ref["Lx"], b)
    assert np.abs(x - xr).max() / np.abs(xr).max() <= 1e-10
    assert O.residual(n, Ap, Ai, Ax, x, b) <= 1e-14


def test_fp64_refactor_is_deterministic():
    n, Ap, Ai, Ax = mg.laplacian_3d_varcoef(16, seed=0)
    S = M.Solver(n, Ap, Ai)
    S.factor(Ax)
    L1 = S.get_L()[2].copy()
    S.factor(Ax)
    L2 = S.get_L()[2]
    np.testing.assert_array_equal(L1, L2)


def test_multiple_rhs_and_device_api():
    n, Ap, Ai, Ax = mg.laplacian_3d_varcoef(16, seed=1)
    S = M.Solver(n, Ap, Ai)
    dAx = torch.from_numpy(Ax).cuda()
    S.factor(dAx, M.FP64)
    B = mg.rhs_uniform(n, seed=5, nrhs=70)  # more than one 64-column chunk
    X = S.solve(B)
    for q in (0, 33, 69):
        assert O.residual(n, Ap, Ai, Ax, X[:, q], B[:, q]) <= 1e-14
    dB = torch.from_numpy(np.asfortranarray(B)).cuda()
    dB = dB.t().contiguous().t()
    dX = S.solve(dB)
    np.testing.assert_allclose(dX.cpu().numpy(), X, rtol=0, atol=1e-12 * np.abs(X).max())


@pytest.mark.parametrize("name", ["2d100_amd_sn", "3d16_amd_rn4", "rnd300_amd_sn"])
def test_solves_with_each_rhs_count_match_oracle(name):
    """Small fronts take a warp each (rows in registers up to 32, in the warp's
    shared buffer up to 160) with at most 4 right-hand sides, a CTA each with
    more; every count must give the oracle's solution column by column."""
    _, gen, amd, mode, z = next(c for c in CASES if c[0] == name)
    n, Ap, Ai, Ax = gen()
    P = O.Plan(n, Ap, Ai, Ax, amd=amd, mode=mode, rn_zeros=z)
    ref = P.factor()
    S = M.Solver(n, Ap, Ai, ordering=int(amd), tree=TREE[mode], relax_zeros=z)
    assert S.array("rows_ptr").size > 1
    S.factor(Ax, M.FP64)
    B = mg.rhs_uniform(n, seed=9, nrhs=9)
    xr = [P.solve(ref["Li"], ref["Lx"], B[:, q]) for q in range(9)]
    for k in (1, 2, 3, 4, 5, 9):
        X = S.solve(B[:, :k]).reshape(n, k)
        for q in range(k):
            assert np.abs(X[:, q] - xr[q]).max() / np.abs(xr[q]).max() <= 1e-10, (k, q)
    S.factor(Ax, M.FP32)
    for k in (1, 3, 4, 5):
        X = S.solve(B[:, :k]).reshape(n, k)
        for q in range(k):
            assert np.abs(X[:, q] - xr[q]).max() / np.abs(xr[q]).max() <= 1e-3, (k, q)


@pytest.mark.parametrize("side", [16, 24])
def test_fp32_factor_with_refinement_reaches_fp64_accuracy(side):
    n, Ap, Ai, Ax = mg.laplacian_3d_varcoef(side, seed=0)
    S = M.Solver(n, Ap, Ai)
    S.factor(Ax, M.FP32)
    b = mg.rhs_uniform(n, seed=0)
    x, berr, iters = S.refine(b, tol=1e-14, maxit=20)
    assert berr[0] <= 1e-14
    assert O.residual(n, Ap, Ai, Ax, x, b) <= 1e-14
    S64 = M.Solver(n, Ap, Ai)
    S64.factor(Ax, M.FP64)
    x64 = S64.solve(b)
    assert np.abs(x - x64).max() / np.abs(x64).max() <= 1e-9


def test_not_spd_reports_first_failing_column():
    n, Ap, Ai, Ax = mg.laplacian_2d_5pt(20)
    Ax = Ax.copy()
    # make the first diagonal entry negative
    Ax[Ap[0]] = -4.0
    S = M.Solver(n, Ap, Ai, ordering=M.ORDER_NATURAL)
    with pytest.raises(M.NotSPDError) as ei:
        S.factor(Ax)
    assert ei.value.column == 0
    with pytest.raises(M.MdgpuError):
        S.solve(np.ones(n))


@pytest.mark.parametrize("side", [24, 32])
def test_fp32_tensor_core_factor_close_to_reference(side):
    """FP32 factor whose large-front Schur updates run on the tcgen05 tensor
    cores (TF32 inputs, FP32 accumulation) over 256-column panels: L within
    TF32 accuracy of the reference's FP64 L (relative Frobenius <= 5e-3), the
    same pattern, and FP64 refinement to backward error <= 1e-14."""
    n, Ap, Ai, Ax = mg.laplacian_3d_varcoef(side, seed=0)
    P = O.Plan(n, Ap, Ai, Ax, amd=True, mode="sn")
    ref = P.factor()
    S = M.Solver(n, Ap, Ai)
    assert S.info("large_fronts") > 0
    S.factor(Ax, M.FP32)
    _, Li, Lx = S.get_L()
    np.testing.assert_array_equal(Li, ref["Li"])
    assert _rel_fro(Lx, ref["Lx"]) <= 5e-3
    b = mg.rhs_uniform(n, seed=1)
    x, berr, iters = S.refine(b, tol=1e-14, maxit=30)
    assert berr[0] <= 1e-14
    assert O.residual(n, Ap, Ai, Ax, x, b) <= 1e-14


@pytest.mark.parametrize("prec", [M.FP32, M.FP64], ids=["fp32", "fp64"])
def test_refine_device_with_padded_leading_dimensions(prec):
    """Refinement on device arrays whose columns are longer than n (leading
    dimensions n + 3 for B and n + 5 for X, five right-hand sides): the same
    numbers as the host-buffer entry point (the residual, the max-norms and
    the column updates take their leading dimensions from the caller), the
    padding rows left as they were, and a backward error below 1e-14 by the
    host's own product with A."""
    from scipy.sparse.linalg import norm as sparse_norm

    n, Ap, Ai, Ax = mg.laplacian_3d_varcoef(12, seed=6)
    S = M.Solver(n, Ap, Ai)
    S.factor(Ax, prec)
    k = 5
    B = mg.rhs_uniform(n, seed=7, nrhs=k).reshape(n, k)
    xh, berr_h, it_h = S.refine(B)
    bbig = torch.full((k, n + 3), 7.0, dtype=torch.float64, device="cuda")
    xbig = torch.full((k, n + 5), float("nan"), dtype=torch.float64, device="cuda")
    dB = bbig.t()[:n]
    dX = xbig.t()[:n]
    dB.copy_(torch.from_numpy(B))
    berr_d, it_d = S.refine_device(dB, dX)
    torch.cuda.synchronize()
    x = dX.cpu().numpy()
    assert it_d == it_h
    np.testing.assert_array_equal(x, xh)
    np.testing.assert_array_equal(berr_d, berr_h)
    assert torch.isnan(xbig[:, n:]).all() and (bbig[:, n:] == 7.0).all()
    A = mg.lower_to_full_scipy(n, Ap, Ai, Ax)
    r = B - A @ x
    den = sparse_norm(A, np.inf) * np.abs(x).max(axis=0) + np.abs(B).max(axis=0)
    assert (np.abs(r).max(axis=0) / den).max() <= 1e-14
