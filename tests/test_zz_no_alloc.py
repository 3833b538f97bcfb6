"""The solve that allocates no device memory (mdgpu_solve_device_noalloc).

For callers that cannot allocate at solve time (under a framework whose
caching allocator owns the device memory, or in loops that cannot pay
cudaMalloc's implicit synchronization), the work vectors come from a fixed
32 MiB device array instead of cudaMalloc.  Checked through the C ABI against
mdgpu_solve_device on two calls in a row (the array keeps the previous call's
contents), and the size limit is enforced with a clear error.

This file is collected last on purpose: it must pass after every other test
and alone in a fresh process.
"""
import ctypes as C

import numpy as np
import pytest

import mdgpu_b200 as M
from mdgpu_b200 import matgen as mg

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover - collected only on GPU boxes
    pytest.skip("needs a CUDA device", allow_module_level=True)


def _noalloc(S, dB, dX, nrhs):
    return M.lib().mdgpu_solve_device_noalloc(S._h, C.c_void_p(dB.data_ptr()), S.n,
                                              C.c_void_p(dX.data_ptr()), S.n, nrhs, None)


def _colmajor(a):
    t = torch.from_numpy(np.asfortranarray(a)).cuda()
    return t.t().contiguous().t() if t.dim() == 2 else t


@pytest.mark.parametrize("prec,gen", [
    (M.FP64, lambda: mg.laplacian_3d_varcoef(14, seed=2)),
    (M.FP32, lambda: mg.laplacian_3d_varcoef(14, seed=2)),
    # odd n with an odd right-hand-side count: the work vectors after the
    # permuted right-hand sides still start on 16 bytes
    (M.FP32, lambda: mg.laplacian_3d_varcoef(13, seed=4)),
], ids=["fp64", "fp32", "fp32_odd_n"])
def test_noalloc_solve_matches_regular_solve_twice(prec, gen):
    n, Ap, Ai, Ax = gen()
    S = M.Solver(n, Ap, Ai)
    S.factor(Ax, prec)
    for call, (seed, nrhs) in enumerate([(10, 3), (11, 1)]):
        B = mg.rhs_uniform(n, seed=seed, nrhs=nrhs).reshape(n, nrhs)
        dB = _colmajor(B)
        ref = S.solve(dB)
        dX = torch.full_like(dB, float("nan"))
        rc = _noalloc(S, dB, dX, nrhs)
        assert rc == 0, M.lib().mdgpu_last_error().decode()
        torch.cuda.synchronize()
        x, xr = dX.cpu().numpy(), ref.cpu().numpy()
        assert np.all(np.isfinite(x)), call
        np.testing.assert_allclose(x, xr, rtol=1e-12, atol=1e-12 * np.abs(xr).max())


def test_noalloc_solve_rejects_requests_beyond_its_scratch():
    n, Ap, Ai, Ax = mg.laplacian_2d_5pt(300)  # n = 90000: 64 rhs need > 4M doubles
    S = M.Solver(n, Ap, Ai)
    S.factor(Ax, M.FP64)
    nrhs = 64
    dB = _colmajor(mg.rhs_uniform(n, seed=1, nrhs=nrhs))
    dX = torch.empty_like(dB)
    rc = _noalloc(S, dB, dX, nrhs)
    assert rc == -1
    msg = M.lib().mdgpu_last_error().decode()
    assert "limit" in msg and "scratch" in msg
    # one right-hand side fits and still solves
    db1 = dB[:, 0].contiguous()
    dx1 = torch.empty_like(db1)
    assert _noalloc(S, db1, dx1, 1) == 0
    x1 = S.solve(db1)
    np.testing.assert_allclose(dx1.cpu().numpy(), x1.cpu().numpy(), rtol=1e-12,
                               atol=1e-12 * float(x1.abs().max()))


def test_noalloc_solve_allocates_nothing_and_chunks_more_than_64_rhs():
    """After one warm-up call, further calls -- 70 and 65 right-hand sides
    (two 64-column chunks reusing the same work vectors) and one -- leave the
    device's free memory unchanged, and each matches the regular solve."""
    n, Ap, Ai, Ax = mg.laplacian_3d_varcoef(10, seed=3)
    S = M.Solver(n, Ap, Ai)
    S.factor(Ax, M.FP32)
    B = mg.rhs_uniform(n, seed=21, nrhs=70).reshape(n, 70)
    dB = _colmajor(B)
    refs = {k: S.solve(_colmajor(B[:, :k])).cpu().numpy().reshape(n, k) for k in (70, 65, 1)}
    dX = torch.full_like(dB, float("nan"))
    assert _noalloc(S, dB, dX, 70) == 0, M.lib().mdgpu_last_error().decode()
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for k in (70, 65, 1, 70):
        dX.fill_(float("nan"))
        rc = _noalloc(S, dB, dX, k)
        assert rc == 0, M.lib().mdgpu_last_error().decode()
        torch.cuda.synchronize()
        x = dX[:, :k].cpu().numpy()
        xr = refs[k]
        assert np.all(np.isfinite(x)), k
        np.testing.assert_allclose(x, xr, rtol=1e-12, atol=1e-12 * np.abs(xr).max())
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0, (free0, free1)
