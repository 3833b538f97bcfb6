"""The adjoint: log det A, the selected inverse Z = A^-1 on the pattern of L,
and d(log det A + b' A^-1 b)/d Ax for the caller's lower-triangle values.

Checked against dense FP64 (numpy inverse and slogdet) on small 2D / 3D
grids (supernodal and relaxed trees, fronts above 160 rows included), by
central finite differences on single entries, against a reference gradient
by FP64 solves on a 32^3 grid, and through the torch autograd front-end.  The oracle's Takahashi restatement is itself checked
against the dense inverse on the CPU.
"""
import numpy as np
import pytest

import mdgpu_b200 as M
from mdgpu_b200 import matgen as mg
from oracle import oracle as O


def test_oracle_selected_inverse_matches_dense():
    import scipy.sparse as sp

    n, Ap, Ai, Ax = mg.laplacian_3d_varcoef(6, seed=3)
    P = O.Plan(n, Ap, Ai, Ax, amd=True, mode="sn")
    ref = P.factor()
    Z = O.selected_inverse(n, P.Lp, ref["Li"], ref["Lx"])
    L = sp.csc_matrix((ref["Lx"], ref["Li"], P.Lp), shape=(n, n)).toarray()
    Ainv = np.linalg.inv(L @ L.T)
    mask = (L != 0) | (L.T != 0)
    assert np.abs((Z - Ainv)[mask]).max() <= 1e-12 * np.abs(Ainv).max()


def _dense(n, Ap, Ai, Ax):
    return mg.lower_to_full_scipy(n, Ap, Ai, Ax).toarray()


def _dense_grad(n, Ap, Ai, Ax, b=None):
    A = _dense(n, Ap, Ai, Ax)
    Ainv = np.linalg.inv(A)
    Z = Ainv.copy()
    if b is not None:
        x = Ainv @ b
        Z -= np.outer(x, x)
    G = np.zeros(Ap[-1])
    for j in range(n):
        for p in range(Ap[j], Ap[j + 1]):
            i = Ai[p]
            G[p] = Z[i, j] if i == j else 2.0 * Z[i, j]
    return G


CASES = [
    ("2d14_sn", lambda: mg.laplacian_2d_5pt(14), M.TREE_SUPER, 0),
    ("3d9_sn", lambda: mg.laplacian_3d_varcoef(9, seed=2, sigma=1.0, shift=1e-2), M.TREE_SUPER, 0),
    ("3d9_rn4", lambda: mg.laplacian_3d_varcoef(9, seed=2, sigma=1.0, shift=1e-2), M.TREE_RELAXED, 4),
    ("3d16_sn", lambda: mg.laplacian_3d_varcoef(16, seed=5, sigma=1.0, shift=1e-2), M.TREE_SUPER, 0),
]


@pytest.mark.gpu
@pytest.mark.parametrize("name,gen,tree,z", CASES, ids=[c[0] for c in CASES])
def test_logdet_and_gradient_match_dense(name, gen, tree, z):
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    n, Ap, Ai, Ax = gen()
    S = M.Solver(n, Ap, Ai, tree=tree, relax_zeros=z)
    if name == "3d16_sn":
        assert np.diff(S.array("rows_ptr")).max() > 160  # large fronts too
    S.factor(Ax, M.FP64)
    A = _dense(n, Ap, Ai, Ax)
    sign, ld = np.linalg.slogdet(A)
    assert sign > 0 and abs(S.logdet() - ld) <= 1e-11 * abs(ld)
    b = mg.rhs_uniform(n, seed=4)
    x = S.solve(b)
    S.selinv()
    G0 = S.grad_lower()
    Gd0 = _dense_grad(n, Ap, Ai, Ax)
    np.testing.assert_allclose(G0, Gd0, rtol=0, atol=1e-10 * np.abs(Gd0).max())
    G = S.grad_lower(x)
    Gd = _dense_grad(n, Ap, Ai, Ax, b)
    np.testing.assert_allclose(G, Gd, rtol=0, atol=1e-10 * np.abs(Gd).max())
    # twice in a row, and from device vectors: the same numbers
    dG = S.grad_lower(torch.from_numpy(x).cuda()).cpu().numpy()
    np.testing.assert_array_equal(dG, G)


@pytest.mark.gpu
def test_theta_gradient_matches_a_solve_reference_at_32_cubed():
    """d loss / d theta_e (loss = log det A + b' A^-1 b, edge conductances
    theta lognormal(0, 1) on a 32^3 grid, shift 1e-2) from the selected
    inverse, against an FP64 reference gradient on 64 random edges computed
    by solves instead: u' A^-1 u - (x_i - x_j)^2 with u = e_i - e_j.  The grid
    is too large for a dense gradient, and central differences lose digits to
    the size of the loss; the two FP64 routes agree to 1e-8 relative."""
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    n, Ap, Ai, Ax, lo, hi, cond = mg.laplacian_grid_edges((32,) * 3, seed=3, sigma=1.0,
                                                          shift=1e-2)
    S = M.Solver(n, Ap, Ai)
    assert np.diff(S.array("rows_ptr")).max() > 1000  # tiled large fronts on the path
    S.factor(Ax, M.FP64)
    b = mg.rhs_uniform(n, seed=4)
    x = S.solve(b)
    S.selinv()
    G = S.grad_lower(x)

    def pos(r, c):
        seg = Ai[Ap[c]:Ap[c + 1]]
        return Ap[c] + int(np.searchsorted(seg, r))

    picked = np.random.default_rng(5).choice(len(cond), 64, replace=False)
    U = np.zeros((n, len(picked)))
    U[lo[picked], np.arange(len(picked))] = 1.0
    U[hi[picked], np.arange(len(picked))] = -1.0
    Zu = S.solve(U)
    g = np.array([G[pos(lo[e], lo[e])] + G[pos(hi[e], hi[e])] - G[pos(hi[e], lo[e])]
                  for e in picked])
    gref = np.array([Zu[lo[e], k] - Zu[hi[e], k] - (x[lo[e]] - x[hi[e]]) ** 2
                     for k, e in enumerate(picked)])
    err = np.abs(g - gref) / np.maximum(np.abs(gref), 1e-6 * np.abs(gref).max())
    assert err.max() <= 1e-8, (err.max(), int(np.argmax(err)))


@pytest.mark.gpu
def test_gradient_matches_central_differences():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    n, Ap, Ai, Ax = mg.laplacian_3d_varcoef(10, seed=7, sigma=1.0, shift=1e-2)
    S = M.Solver(n, Ap, Ai)
    b = mg.rhs_uniform(n, seed=8)

    def loss(v):
        S.factor(v, M.FP64)
        return S.logdet() + float(b @ S.solve(b))

    loss(Ax)
    S.selinv()
    G = S.grad_lower(S.solve(b))
    rng = np.random.default_rng(0)
    for p in rng.choice(Ap[-1], 12, replace=False):
        h = 1e-6 * abs(Ax[p])
        vp, vm = Ax.copy(), Ax.copy()
        vp[p] += h
        vm[p] -= h
        fd = (loss(vp) - loss(vm)) / (2 * h)
        assert abs(fd - G[p]) <= 1e-6 * max(abs(G[p]), 1e-3 * np.abs(G).max()), (p, fd, G[p])


@pytest.mark.gpu
def test_autograd_front_end():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    from mdgpu_b200.autograd import logdet_quad

    n, Ap, Ai, Ax = mg.laplacian_3d_varcoef(8, seed=9, sigma=0.5, shift=1e-2)
    S = M.Solver(n, Ap, Ai)
    tAx = torch.from_numpy(Ax).cuda().requires_grad_(True)
    tb = torch.from_numpy(mg.rhs_uniform(n, seed=10)).cuda().requires_grad_(True)
    loss = logdet_quad(S, tAx, tb)
    loss.backward()
    b = tb.detach().cpu().numpy()
    Gd = _dense_grad(n, Ap, Ai, Ax, b)
    np.testing.assert_allclose(tAx.grad.cpu().numpy(), Gd, rtol=0, atol=1e-10 * np.abs(Gd).max())
    x = np.linalg.solve(_dense(n, Ap, Ai, Ax), b)
    np.testing.assert_allclose(tb.grad.cpu().numpy(), 2 * x, rtol=1e-10, atol=0)
    sign, ld = np.linalg.slogdet(_dense(n, Ap, Ai, Ax))
    assert abs(float(loss.detach()) - (ld + b @ x)) <= 1e-10 * abs(ld + b @ x)


@pytest.mark.gpu
def test_autograd_two_forwards_on_one_solver_then_backwards():
    """Two forwards on one Solver (the second refactors it) before either
    backward: each backward differentiates its own values (it refactors them
    when the Solver's factor generation moved on), matching the dense
    gradient of each."""
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    from mdgpu_b200.autograd import logdet_quad

    n, Ap, Ai, Ax1 = mg.laplacian_3d_varcoef(7, seed=11, sigma=0.5, shift=1e-2)
    Ax2 = mg.laplacian_3d_varcoef(7, seed=12, sigma=0.5, shift=1e-2)[3]
    b = mg.rhs_uniform(n, seed=13)
    S = M.Solver(n, Ap, Ai)
    t1 = torch.from_numpy(Ax1).cuda().requires_grad_(True)
    t2 = torch.from_numpy(Ax2).cuda().requires_grad_(True)
    tb = torch.from_numpy(b).cuda()
    l1 = logdet_quad(S, t1, tb)
    l2 = logdet_quad(S, t2, tb)
    l1.backward()
    l2.backward()
    for t, A in ((t1, Ax1), (t2, Ax2)):
        Gd = _dense_grad(n, Ap, Ai, A, b)
        np.testing.assert_allclose(t.grad.cpu().numpy(), Gd, rtol=0,
                                   atol=1e-10 * np.abs(Gd).max())
