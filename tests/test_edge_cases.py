"""Edge cases of the symbolic phase (CPU) and of the GPU factor (-m gpu).

The reference rejects a forest (GetETree, etree.cpp:27-31) and overwrites
repeated entries in front assembly (last one wins, mdgpu.cu:274-282); a
1 x 1 system and a dense matrix (one supernode) are the degenerate trees.
"""
import numpy as np
import pytest

import mdgpu_b200 as M
from oracle import oracle as O


def _lower_csc(A):
    n = A.shape[0]
    Ap, Ai, Ax = [0], [], []
    for j in range(n):
        for i in range(j, n):
            if A[i, j] != 0:
                Ai.append(i)
                Ax.append(A[i, j])
        Ap.append(len(Ai))
    return n, np.array(Ap, np.int32), np.array(Ai, np.int32), np.array(Ax)


def _dense_spd(n, seed):
    rng = np.random.default_rng(seed)
    X = rng.standard_normal((n, n))
    return X @ X.T + n * np.eye(n)


@pytest.mark.parametrize("n", [1, 2, 7, 40, 200])
def test_dense_matrix_is_one_supernode(n):
    n, Ap, Ai, Ax = _lower_csc(_dense_spd(n, n))
    S = M.Solver(n, Ap, Ai)
    assert S.info("nsuper") == 1
    P = O.Plan(n, Ap, Ai, Ax, amd=True, mode="sn")
    assert P.nsuper == 1
    np.testing.assert_array_equal(S.array("perm"), P.perm)


def test_diagonal_matrix_is_a_forest():
    n, Ap, Ai, Ax = _lower_csc(np.diag(np.arange(1.0, 6.0)))
    with pytest.raises(M.MdgpuError) as ei:
        M.Solver(n, Ap, Ai)
    assert ei.value.status == -5
    with pytest.raises(ValueError):
        O.Plan(n, Ap, Ai, Ax)


def test_empty_matrix_is_rejected():
    with pytest.raises(M.MdgpuError):
        M.Solver(0, np.zeros(1, np.int32), np.zeros(0, np.int32))


torch = pytest.importorskip("torch")


@pytest.mark.gpu
@pytest.mark.skipif(not torch.cuda.is_available(), reason="needs a CUDA device")
@pytest.mark.parametrize("n", [1, 2, 40, 200, 700])
@pytest.mark.parametrize("prec", [M.FP64, M.FP32])
def test_dense_factor_and_solve(n, prec):
    A = _dense_spd(n, 3 * n + 1)
    n, Ap, Ai, Ax = _lower_csc(A)
    S = M.Solver(n, Ap, Ai)
    S.factor(Ax, prec)
    b = np.random.default_rng(n).uniform(-1, 1, n)
    if prec == M.FP64:
        x = S.solve(b)
        P = O.Plan(n, Ap, Ai, Ax)
        ref = P.factor()
        Lx = S.get_L()[2]
        assert np.linalg.norm(Lx - ref["Lx"]) <= 1e-12 * np.linalg.norm(ref["Lx"])
    else:
        x, berr, _ = S.refine(b, tol=1e-14, maxit=30)
    assert O.residual(n, Ap, Ai, Ax, x, b) <= 1e-14


@pytest.mark.gpu
@pytest.mark.skipif(not torch.cuda.is_available(), reason="needs a CUDA device")
def test_repeated_entries_keep_the_last_value():
    """A repeated (i, j) entry: the reference's front assembly overwrites, so
    the last occurrence in the column is the value factored."""
    A = _dense_spd(30, 5)
    n, Ap, Ai, Ax = _lower_csc(A)
    # duplicate the diagonal entry of column 3 with a bogus first copy
    j = 3
    p = Ap[j]
    Ai2 = np.insert(Ai, p, Ai[p])
    Ax2 = np.insert(Ax, p, -123.0)
    Ap2 = Ap.copy()
    Ap2[j + 1:] += 1
    S = M.Solver(n, Ap2, Ai2, ordering=M.ORDER_NATURAL)
    S.factor(Ax2)
    S0 = M.Solver(n, Ap, Ai, ordering=M.ORDER_NATURAL)
    S0.factor(Ax)
    np.testing.assert_allclose(S.get_L()[2], S0.get_L()[2], rtol=1e-13, atol=1e-13)


@pytest.mark.gpu
@pytest.mark.skipif(not torch.cuda.is_available(), reason="needs a CUDA device")
def test_nan_with_the_sentinel_payload_in_the_rhs_solves_to_nan_quickly():
    """The solve marks unpublished pivot-tile slots with the all-ones bit
    pattern (a NaN).  A right-hand side holding a NaN with exactly that
    payload must come out as NaN in the solution, promptly and with status
    OK, not stall the dependent tiles until their waits run out; the other
    right-hand side of the same call is unaffected."""
    import time

    from mdgpu_b200 import matgen as mg

    n, Ap, Ai, Ax = mg.laplacian_3d_varcoef(16, seed=0)  # large fronts: tile tasks
    S = M.Solver(n, Ap, Ai)
    assert S.info("large_fronts") > 0
    S.factor(Ax, M.FP64)
    B = mg.rhs_uniform(n, seed=2, nrhs=2).reshape(n, 2).copy()
    ref = S.solve(B[:, 1].copy())
    bad = np.array([-1], dtype=np.int64).view(np.float64)[0]
    perm = S.array("perm")
    B[perm[-1], 0] = bad  # the last pivot: the root's last tile
    B[perm[n // 2], 0] = bad
    for cols in ([0], [0, 1]):
        t0 = time.perf_counter()
        X = S.solve(np.asfortranarray(B[:, cols])).reshape(n, len(cols))
        assert time.perf_counter() - t0 < 2.0
        assert np.isnan(X[:, 0]).any()
        if len(cols) == 2:
            np.testing.assert_allclose(X[:, 1], ref, rtol=0, atol=1e-12 * np.abs(ref).max())
