"""GMRES-based iterative refinement (GMRES-IR).

CPU: the oracle's restatement (Carson & Higham 2018, Algorithm 3.1) reaches
backward error 1e-14 with a factor rounded to BF16, where plain refinement
does not; the library's driver template (mdgpu_b200/csrc/gmres_ir.hpp),
compiled here over host loops (tests/gmres_ir_host.cpp), takes the same
steps as the oracle; the entry points' argument checks.
GPU: the entry points with the FP32 and FP64 factors on the multi-unknown
(3 per node) system, host and device buffers.
"""
import os
import shutil
import subprocess

import numpy as np
import pytest
import scipy.linalg as sl
import scipy.sparse as sp

import mdgpu_b200 as M
from mdgpu_b200 import matgen as mg
from oracle import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _system(side, seed, sigma=1.0):
    n, Ap, Ai, Ax = mg.elasticity_3dof(side, seed=seed, sigma=sigma)
    A = mg.lower_to_full_scipy(n, Ap, Ai, Ax).toarray()
    return n, Ap, Ai, Ax, A


def _precond(L):
    return lambda r: sl.solve_triangular(L.T, sl.solve_triangular(L, r, lower=True), lower=False)


def _berr(A, x, b):
    return np.abs(b - A @ x).max() / (np.abs(A).sum(1).max() * np.abs(x).max() + np.abs(b).max())


def test_oracle_gmres_ir_reaches_fp64_accuracy_with_a_bf16_factor():
    n, _, _, _, A = _system(6, seed=1, sigma=2.0)  # cond(A) ~ 5e5
    L = O.round_bf16(np.linalg.cholesky(A))
    Minv = _precond(L)
    b = np.random.default_rng(0).uniform(-1, 1, n)
    anorm = np.abs(A).sum(1).max()
    # plain refinement with the same factor: ten corrections fall short
    x = Minv(b)
    for _ in range(10):
        x = x + Minv(b - A @ x)
    assert _berr(A, x, b) > 1e-10
    x, hist, inner = O.gmres_ir(lambda v: A @ v, Minv, b, anorm, tol=1e-14, maxit=10)
    assert hist[-1] <= 1e-14 and len(hist) <= 4, hist
    assert all(1 <= k <= 30 for k in inner)
    xe = np.linalg.solve(A, b)
    assert np.abs(x - xe).max() <= 1e-12 * np.abs(xe).max()


def test_bf16_schur_update_factor_plain_ir_vs_gmres_ir():
    """The arithmetic of a BF16 tensor-core Schur update (operands rounded to
    BF16, FP32 accumulation; diagonal blocks and panel solves in FP32) on the
    multi-unknown system (cond ~2e4): the factor is good to ~3e-4, plain
    refinement gains about one digit per correction, GMRES-IR reaches 1e-14
    in two.  Per-panel power-of-two scaling changes no bit: BF16 keeps FP32's
    exponent range, so the scaling only shifts exponents."""
    n, _, _, _, A = _system(8, seed=1, sigma=1.0)
    L = O.bf16_update_cholesky(A)
    assert np.array_equal(L, O.bf16_update_cholesky(A, pow2_scale=True))
    rel = np.linalg.norm(L @ L.T - A) / np.linalg.norm(A)
    assert 1e-5 < rel < 1e-3, rel
    Minv = _precond(L)
    b = np.random.default_rng(0).uniform(-1, 1, n)
    x = Minv(b)
    for _ in range(10):
        x = x + Minv(b - A @ x)
    assert _berr(A, x, b) > 1e-12
    anorm = np.abs(A).sum(1).max()
    x, hist, inner = O.gmres_ir(lambda v: A @ v, Minv, b, anorm, tol=1e-14, maxit=10)
    assert hist[-1] <= 1e-14 and len(hist) <= 4, hist


def _harness(tmp_path):
    cxx = shutil.which("g++")
    if cxx is None:
        pytest.skip("needs g++")
    exe = str(tmp_path / "gmres_ir_host")
    subprocess.run([cxx, "-O2", "-std=c++17", "-I", os.path.join(ROOT, "mdgpu_b200", "csrc"),
                    os.path.join(ROOT, "tests", "gmres_ir_host.cpp"), "-o", exe], check=True)
    return exe


def _run_harness(exe, tmp_path, A, L, b, tol, maxit, restart, inner_tol):
    n = A.shape[0]
    C = sp.csr_matrix(A)
    C.sort_indices()
    fin, fout = str(tmp_path / "in.bin"), str(tmp_path / "out.txt")
    with open(fin, "wb") as f:
        np.array([n, restart, maxit, C.nnz], np.int32).tofile(f)
        np.array([tol, inner_tol], np.float64).tofile(f)
        C.indptr.astype(np.int32).tofile(f)
        C.indices.astype(np.int32).tofile(f)
        C.data.astype(np.float64).tofile(f)
        np.ascontiguousarray(np.tril(L), np.float64).tofile(f)
        np.asarray(b, np.float64).tofile(f)
    subprocess.run([exe, fin, fout], check=True)
    with open(fout) as f:
        outer, inner, berr = f.readline().split()
        hist = np.array([float(v) for v in f.readline().split()])
        x = np.array([float(v) for v in f.read().split()])
    return int(outer), int(inner), float(berr), hist, x


HARNESS_CASES = [
    # name, factor rounding, restart, maxit, inner_tol
    ("bf16_r30", "bf16", 30, 10, 1e-8),
    ("bf16_r3", "bf16", 3, 30, 1e-8),
    ("bf16_loose", "bf16", 30, 10, 1e-4),
    ("fp32_r30", "fp32", 30, 10, 1e-8),
    ("bf16_update_r30", "bf16_update", 30, 10, 1e-8),
    ("bf16_maxit0", "bf16", 30, 0, 1e-8),
]


@pytest.mark.parametrize("name,rounding,restart,maxit,inner_tol", HARNESS_CASES,
                         ids=[c[0] for c in HARNESS_CASES])
def test_driver_template_takes_the_oracles_steps(tmp_path, name, rounding, restart, maxit,
                                                 inner_tol):
    exe = _harness(tmp_path)
    n, _, _, _, A = _system(5, seed=3, sigma=1.5)
    if rounding == "bf16_update":
        L = O.bf16_update_cholesky(A)
    else:
        L = np.linalg.cholesky(A)
        L = O.round_bf16(L) if rounding == "bf16" else L.astype(np.float32).astype(np.float64)
    b = np.random.default_rng(7).uniform(-1, 1, n)
    anorm = np.abs(A).sum(1).max()
    x0, hist0, inner0 = O.gmres_ir(lambda v: A @ v, _precond(L), b, anorm, tol=1e-14,
                                   maxit=maxit, restart=restart, inner_tol=inner_tol)
    outer, inner, berr, hist, x = _run_harness(exe, tmp_path, A, L, b, 1e-14, maxit, restart,
                                               inner_tol)
    assert outer == len(hist0) - 1 and inner == sum(inner0), (outer, inner, hist0, inner0)
    hist0 = np.array(hist0)
    assert len(hist) == len(hist0)
    # the backward errors agree to the residual's roundoff (~1e-16 absolute)
    np.testing.assert_allclose(hist, hist0, rtol=1e-3, atol=1e-15)
    assert berr == hist[-1]
    assert np.abs(x - x0).max() <= 1e-11 * np.abs(x0).max()
    if maxit > 0:
        assert berr <= 1e-14


def test_gmres_ir_argument_checks():
    n, Ap, Ai, Ax = mg.laplacian_2d_5pt(6)
    S = M.Solver(n, Ap, Ai)
    b = np.ones(n)
    for kw in ({"restart": 0}, {"restart": 65}, {"maxit": -1}, {"inner_tol": -1.0}):
        with pytest.raises(M.MdgpuError) as e:
            S.gmres_ir(b, **kw)
        assert e.value.status == -1, kw
    # valid arguments: stopped by the missing device or the missing factor
    with pytest.raises(M.MdgpuError) as e:
        S.gmres_ir(b)
    assert e.value.status in (-6, -7)


def _node_ordered(side, seed, sigma):
    """The multi-unknown system in the node-graph AMD ordering, expanded to
    the three unknowns of each node, analysed in natural order."""
    n, Ap, Ai, Ax = mg.elasticity_3dof(side, seed=seed, sigma=sigma)
    nn, gp, gi, _ = mg.node_graph_lower(side)
    perm = mg.expand_node_perm(M.Solver(nn, gp, gi, ordering=M.ORDER_AMD).array("perm"))
    return mg.permute_lower(n, Ap, Ai, Ax, perm)


def _need_cuda():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    return torch


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [M.FP32, M.FP64], ids=["fp32", "fp64"])
def test_gmres_ir_on_the_multi_unknown_system(precision):
    torch = _need_cuda()
    n, Ap, Ai, Ax = _node_ordered(8, seed=4, sigma=1.0)
    S = M.Solver(n, Ap, Ai, ordering=M.ORDER_NATURAL)
    S.factor(Ax, precision)
    A = mg.lower_to_full_scipy(n, Ap, Ai, Ax).toarray()
    B = np.random.default_rng(5).uniform(-1, 1, (n, 3))
    X, berr, it, inner = S.gmres_ir(B, tol=1e-14, maxit=10)
    Xe = np.linalg.solve(A, B)
    # forward error <= cond(A) (~2e4) x backward error (<= 1e-14)
    for q in range(3):
        assert berr[q] <= 1e-14 and it[q] <= 3, (berr, it, inner)
        assert _berr(A, X[:, q], B[:, q]) <= 2e-14
        assert np.abs(X[:, q] - Xe[:, q]).max() <= 1e-9 * np.abs(Xe[:, q]).max()
    # a single right-hand side, and device buffers with a leading dimension > n
    x1, b1, i1, k1 = S.gmres_ir(B[:, 1])
    assert b1 <= 1e-14 and np.abs(x1 - Xe[:, 1]).max() <= 1e-9 * np.abs(Xe[:, 1]).max()
    ld = n + 3
    dB = torch.zeros((3, ld), dtype=torch.float64, device="cuda")
    dB[:, :n] = torch.from_numpy(B.T.copy()).cuda()
    dX = torch.zeros((3, ld), dtype=torch.float64, device="cuda")
    berr_d, it_d, inner_d = S.gmres_ir_device(dB[:, :n].t(), dX[:, :n].t())
    Xd = dX[:, :n].cpu().numpy().T
    assert np.all(berr_d <= 1e-14)
    assert np.abs(Xd - Xe).max() <= 1e-9 * np.abs(Xe).max()
    assert torch.all(dX[:, n:] == 0)  # nothing written past n in a column


@pytest.mark.gpu
def test_gmres_ir_short_restarts_and_no_correction():
    _need_cuda()
    n, Ap, Ai, Ax = _node_ordered(7, seed=6, sigma=1.5)
    S = M.Solver(n, Ap, Ai, ordering=M.ORDER_NATURAL)
    S.factor(Ax, M.FP32)
    A = mg.lower_to_full_scipy(n, Ap, Ai, Ax).toarray()
    b = np.random.default_rng(8).uniform(-1, 1, n)
    # restart 2: more corrections, same accuracy
    x, berr, it, inner = S.gmres_ir(b, tol=1e-14, maxit=30, restart=2)
    assert berr <= 1e-14 and inner <= 2 * it
    # maxit 0: the factor's solve alone, its backward error reported
    x0, berr0, it0, inner0 = S.gmres_ir(b, maxit=0)
    assert it0 == 0 and inner0 == 0
    assert abs(berr0 - _berr(A, x0, b)) <= 1e-3 * berr0
    np.testing.assert_allclose(x0, S.solve(b), rtol=0, atol=1e-14 * np.abs(x0).max())
