"""The autotuner (mdgpu_autotune, -m gpu): it picks launch shapes from its
candidate sets by timing the factor, the handle keeps them, and the factor
with the chosen shapes still matches the oracle (FP64 L within 1e-12) --
the shapes change who does the work, not the sums."""
import numpy as np
import pytest

import mdgpu_b200 as M
from mdgpu_b200 import matgen as mg
from oracle import oracle as O

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover - collected only on GPU boxes
    pytest.skip("needs a CUDA device", allow_module_level=True)


def test_autotune_keeps_the_factor_exact():
    n, Ap, Ai, Ax = mg.laplacian_3d_varcoef(16, seed=0)
    S = M.Solver(n, Ap, Ai)
    S.factor(Ax, M.FP64)
    L0 = S.get_L()[2].copy()
    assert S.info("tuned") == 0
    shapes = S.autotune(Ax, M.FP64)
    assert S.info("tuned") == 1 and shapes["ms"] > 0
    assert shapes["tiny_blocks"] in (148 * 4, 148 * 8, 148 * 16)
    for b in range(2, 6):
        assert shapes["threads_b%d" % b] in (128, 256, 512)
    S.factor(Ax, M.FP64)
    np.testing.assert_array_equal(S.get_L()[2], L0)  # same sums, bit for bit
    P = O.Plan(n, Ap, Ai, Ax, amd=True, mode="sn")
    ref = P.factor()
    assert np.linalg.norm(L0 - ref["Lx"]) <= 1e-12 * np.linalg.norm(ref["Lx"])
