"""The general reverse mode (mdgpu_adjoint: Lbar -> Abar).

CPU: the oracle's dense Cholesky adjoint (oracle.cholesky_adjoint_dense,
Murray 2016) against central differences of loss(A) = <Lbar, chol(A)>.
GPU (-m gpu): the library's reverse sweep over the assembly tree against the
dense adjoint of the permuted matrix on A's pattern (1e-10 relative), for
supernodal and relaxed trees with large fronts; against central differences
of the GPU factor itself; and for Lbar = the gradient of log det A = 2 sum
log L(j, j), against the selected-inverse gradient mdgpu_grad_lower.
"""
import numpy as np
import pytest

import mdgpu_b200 as M
from mdgpu_b200 import matgen as mg
from oracle import oracle as O


def test_oracle_cholesky_adjoint_matches_central_differences():
    rng = np.random.default_rng(0)
    n = 11
    X = rng.standard_normal((n, n))
    A = X @ X.T + n * np.eye(n)
    Lb = np.tril(rng.standard_normal((n, n)))
    Al = np.tril(A)

    def loss(v):
        Af = np.tril(v) + np.tril(v, -1).T
        return float(np.sum(Lb * np.linalg.cholesky(Af)))

    G = O.cholesky_adjoint_dense(np.linalg.cholesky(A), Lb)
    for i in range(n):
        for j in range(i + 1):
            h = 1e-6
            P, Q = Al.copy(), Al.copy()
            P[i, j] += h
            Q[i, j] -= h
            fd = (loss(P) - loss(Q)) / (2 * h)
            assert abs(fd - G[i, j]) <= 1e-7 * max(1.0, abs(G[i, j])), (i, j, fd, G[i, j])


def _dense_reference(S, n, Ap, Ai, Ax, Lbar):
    """Abar on A's pattern from the dense adjoint of the permuted matrix."""
    perm = S.array("perm")
    iperm = np.empty(n, np.int64)
    iperm[perm] = np.arange(n)
    A = mg.lower_to_full_scipy(n, Ap, Ai, Ax).toarray()[np.ix_(perm, perm)]
    Lp, Li, _ = S.get_L(values=False)
    Lbd = np.zeros((n, n))
    for j in range(n):
        Lbd[Li[Lp[j]:Lp[j + 1]], j] = Lbar[Lp[j]:Lp[j + 1]]
    G = O.cholesky_adjoint_dense(np.linalg.cholesky(A), Lbd)
    out = np.zeros(Ap[-1])
    for j in range(n):
        for p in range(Ap[j], Ap[j + 1]):
            a, b = iperm[Ai[p]], iperm[j]
            out[p] = G[max(a, b), min(a, b)]
    return out


CASES = [
    ("3d8_sn", lambda: mg.laplacian_3d_varcoef(8, seed=2, sigma=0.5, shift=1e-2), M.TREE_SUPER, 0),
    ("3d9_rn4", lambda: mg.laplacian_3d_varcoef(9, seed=3, sigma=1.0, shift=1e-2),
     M.TREE_RELAXED, 4),
    ("3d14_sn", lambda: mg.laplacian_3d_varcoef(14, seed=4, sigma=0.5, shift=1e-2), M.TREE_SUPER, 0),
]


@pytest.mark.gpu
@pytest.mark.parametrize("name,gen,tree,z", CASES, ids=[c[0] for c in CASES])
def test_adjoint_matches_dense_reverse_mode(name, gen, tree, z):
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    n, Ap, Ai, Ax = gen()
    S = M.Solver(n, Ap, Ai, tree=tree, relax_zeros=z)
    if name == "3d14_sn":
        assert S.info("large_fronts") > 0
    S.factor(Ax, M.FP64)
    rng = np.random.default_rng(5)
    Lbar = rng.standard_normal(S.info("lnz"))
    G = S.adjoint(Lbar)
    Gd = _dense_reference(S, n, Ap, Ai, Ax, Lbar)
    np.testing.assert_allclose(G, Gd, rtol=0, atol=1e-10 * np.abs(Gd).max())
    # device in, device out: the same numbers
    dG = S.adjoint(torch.from_numpy(Lbar).cuda()).cpu().numpy()
    np.testing.assert_array_equal(dG, G)


@pytest.mark.gpu
def test_adjoint_matches_central_differences_of_the_gpu_factor():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    n, Ap, Ai, Ax = mg.laplacian_3d_varcoef(8, seed=6, sigma=0.5, shift=1e-2)
    S = M.Solver(n, Ap, Ai)
    rng = np.random.default_rng(7)
    Lbar = rng.standard_normal(S.info("lnz"))

    def loss(v):
        S.factor(v, M.FP64)
        return float(Lbar @ S.get_L()[2])

    loss(Ax)
    G = S.adjoint(Lbar)
    for p in rng.choice(Ap[-1], 16, replace=False):
        h = 1e-6 * max(abs(Ax[p]), 1e-3)
        vp, vm = Ax.copy(), Ax.copy()
        vp[p] += h
        vm[p] -= h
        fd = (loss(vp) - loss(vm)) / (2 * h)
        assert abs(fd - G[p]) <= 1e-6 * max(abs(G[p]), 1e-3 * np.abs(G).max()), (p, fd, G[p])


@pytest.mark.gpu
def test_adjoint_of_logdet_equals_the_selected_inverse_gradient():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    n, Ap, Ai, Ax = mg.laplacian_3d_varcoef(14, seed=8, sigma=1.0, shift=1e-2)
    S = M.Solver(n, Ap, Ai)
    S.factor(Ax, M.FP64)
    Lp, Li, Lx = S.get_L()
    Lbar = np.zeros_like(Lx)
    diag = Lp[:-1]  # the diagonal leads every column
    Lbar[diag] = 2.0 / Lx[diag]
    G = S.adjoint(Lbar)
    S.selinv()
    Gz = S.grad_lower()
    np.testing.assert_allclose(G, Gz, rtol=0, atol=1e-10 * np.abs(Gz).max())
