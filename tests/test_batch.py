"""Many independent systems under one handle (mdgpu_analyze_batch).

Each system must come out exactly as if analysed and factored alone: its
symbolic arrays are the individual ones shifted by the system's row /
supernode offsets, its block of L matches its own factor, its solution its
own solution.  The mix follows the many-systems workload: 2D and 3D grids of
different sizes, variable coefficients.
"""
import numpy as np
import pytest

import mdgpu_b200 as M
from mdgpu_b200 import matgen as mg


def _systems(seed=0, k=6):
    rng = np.random.default_rng(seed)
    out = []
    for q in range(k):
        if q % 2 == 0:
            out.append(mg.laplacian_2d_5pt(int(rng.integers(6, 20))))
        else:
            out.append(mg.laplacian_3d_varcoef(int(rng.integers(4, 9)), seed=int(rng.integers(100)),
                                               sigma=0.5, shift=1e-2))
    return out


def test_batch_symbolic_is_the_individual_symbolic_shifted():
    syss = _systems()
    B = M.Solver.batch([(n, Ap, Ai) for (n, Ap, Ai, _) in syss])
    assert B.info("nsys") == len(syss)
    assert B.n == sum(s[0] for s in syss)
    so = 0
    Lp = B.array("Lp")
    for b, (n, Ap, Ai, _) in enumerate(syss):
        S = M.Solver(n, Ap, Ai)
        r0, r1 = B.row_off[b], B.row_off[b + 1]
        assert r1 - r0 == n and B.val_off[b + 1] - B.val_off[b] == Ap[-1]
        assert np.array_equal(B.array("perm")[r0:r1] - r0, S.array("perm"))
        par = B.array("parent")[r0:r1]
        exp = S.array("parent")
        assert np.array_equal(np.where(exp < 0, exp, exp + r0), par)
        assert np.array_equal(B.array("count")[r0:r1], S.array("count"))
        ns = S.info("nsuper")
        assert np.array_equal(B.array("sn_first")[so:so + ns] - r0, S.array("sn_first"))
        assert np.array_equal(B.array("sn_ncols")[so:so + ns], S.array("sn_ncols"))
        assert np.array_equal(Lp[r0:r1 + 1] - Lp[r0], S.array("Lp"))
        so += ns
    assert so == B.info("nsuper")


def test_batch_rejects_a_system_whose_tree_is_a_forest():
    n, Ap, Ai, _ = mg.laplacian_2d_5pt(6)
    # two disconnected diagonal entries: a forest
    bad = (2, np.array([0, 1, 2], np.int32), np.array([0, 1], np.int32))
    with pytest.raises(M.MdgpuError) as e:
        M.Solver.batch([(n, Ap, Ai), bad])
    assert e.value.status == -5 and "system 1" in str(e.value)


@pytest.mark.gpu
def test_batch_factor_and_solve_match_each_system_alone():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    syss = _systems(seed=1, k=8)
    B = M.Solver.batch([(n, Ap, Ai) for (n, Ap, Ai, _) in syss])
    Ax = np.concatenate([s[3] for s in syss])
    b = np.concatenate([mg.rhs_uniform(s[0], seed=7 + q) for q, s in enumerate(syss)])
    B.factor(Ax, M.FP64)
    x = B.solve(b)
    Lp, Li, Lx = B.get_L()
    for q, (n, Ap, Ai, Axq) in enumerate(syss):
        S = M.Solver(n, Ap, Ai)
        S.factor(Axq, M.FP64)
        r0, r1 = B.row_off[q], B.row_off[q + 1]
        xq = S.solve(b[r0:r1])
        np.testing.assert_allclose(x[r0:r1], xq, rtol=0, atol=1e-12 * np.abs(xq).max())
        lp, li, lx = S.get_L()
        seg = slice(Lp[r0], Lp[r1])
        assert np.array_equal(Li[seg] - r0, li)
        assert np.linalg.norm(Lx[seg] - lx) <= 1e-12 * np.linalg.norm(lx)
    # FP32 factor + FP64 refinement on the whole batch
    B.factor(Ax, M.FP32)
    xr, berr, it = B.refine(b, tol=1e-14, maxit=20)
    assert berr[0] <= 1e-14
    for q, (n, Ap, Ai, Axq) in enumerate(syss):
        r0, r1 = B.row_off[q], B.row_off[q + 1]
        A = mg.lower_to_full_scipy(n, Ap, Ai, Axq)
        r = b[r0:r1] - A @ xr[r0:r1]
        den = abs(A).sum(axis=1).max() * np.abs(xr[r0:r1]).max() + np.abs(b[r0:r1]).max()
        assert np.abs(r).max() / den <= 1e-13


@pytest.mark.gpu
def test_batch_matches_the_oracle_system_by_system():
    """Every system's block of the batch factor against the oracle (the
    restatement of the reference's CPU path) run on that system alone: the
    same L pattern, L within 1e-12 relative Frobenius, the solution within
    1e-10 of the oracle's.  The mix includes 3D grids large enough for tiled
    fronts, so the batch's panel launches hold fronts of several systems."""
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    from oracle import oracle as O

    syss = _systems(seed=2, k=6) + [mg.laplacian_3d_varcoef(14, seed=5, sigma=0.5, shift=1e-2),
                                    mg.laplacian_3d_varcoef(12, seed=6)]
    B = M.Solver.batch([(n, Ap, Ai) for (n, Ap, Ai, _) in syss])
    assert B.info("large_fronts") > 0
    Ax = np.concatenate([s[3] for s in syss])
    b = np.concatenate([mg.rhs_uniform(s[0], seed=11 + q) for q, s in enumerate(syss)])
    B.factor(Ax, M.FP64)
    x = B.solve(b)
    Lp, Li, Lx = B.get_L()
    for q, (n, Ap, Ai, Axq) in enumerate(syss):
        P = O.Plan(n, Ap, Ai, Axq, amd=True, mode="sn")
        ref = P.factor()
        r0, r1 = B.row_off[q], B.row_off[q + 1]
        seg = slice(Lp[r0], Lp[r1])
        np.testing.assert_array_equal(Li[seg] - r0, ref["Li"])
        assert np.linalg.norm(Lx[seg] - ref["Lx"]) <= 1e-12 * np.linalg.norm(ref["Lx"]), q
        xr = P.solve(ref["Li"], ref["Lx"], b[r0:r1])
        assert np.abs(x[r0:r1] - xr).max() <= 1e-10 * np.abs(xr).max(), q
