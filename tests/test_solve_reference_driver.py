"""The drop-in through the reference's own driver: oracle/_ref/
mdgpu_ref_shim_harness is the reference's driver sequence (load, cs_amd,
etree, counts, supernode tree, spL sizing; then cs_lsolve / cs_ltsolve and the
residual on the filled spL) compiled from the reference sources, with its
Factor replaced by the C-ABI binding oracle/ref/ref_factor_shim.cpp.

CPU: the binary links against the library and binds Factor to the shim (the
symbolic outputs equal the plain reference's; the numeric call reports that
there is no device instead of factoring on the CPU).
GPU: the L the shim writes into spL has the reference's pattern and values
(FP64, 1e-12), and the reference's own solve on it reaches its residual.
Both binaries are built from the reference sources by ``make -C oracle ref
ref-shim``; the tests skip where they were not built.
"""
import os
import subprocess

import numpy as np
import pytest

from mdgpu_b200 import matgen as mg
from oracle import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SHIM = os.path.join(ROOT, "oracle", "_ref", "mdgpu_ref_shim_harness")
# the reference's default build (FLOTANTE float, types.h:4): its own driver
# and the same driver with Factor bound to the shim
REF32 = os.path.join(ROOT, "oracle", "_ref", "mdgpu_ref_harness_f32")
SHIM32 = os.path.join(ROOT, "oracle", "_ref", "mdgpu_ref_shim_harness_f32")

SYMBOLIC = ("perm", "parent", "post", "count0", "count", "sn_nodo", "sn_cols", "sn_childptr",
            "sn_child", "Lp", "Ap", "Ai")


def _need_binaries():
    if not (os.path.exists(SHIM) and os.path.exists(O.REF_HARNESS)):
        pytest.skip("reference harnesses not built (make -C oracle ref ref-shim)")


def _run(exe, flags, mfile, out, check=True):
    os.makedirs(out, exist_ok=True)
    return subprocess.run([exe] + flags + [mfile, out], capture_output=True, text=True,
                          timeout=600, check=check)


def test_shim_binds_factor_to_the_library(tmp_path):
    _need_binaries()
    n, Ap, Ai, Ax = mg.laplacian_3d_varcoef(7, seed=1)
    mfile = str(tmp_path / "A.txt")
    mg.write_triplets(mfile, n, Ap, Ai, Ax)
    _run(O.REF_HARNESS, ["-amd", "-sn", "-nofactor"], mfile, str(tmp_path / "ref"))
    _run(SHIM, ["-amd", "-sn", "-nofactor"], mfile, str(tmp_path / "shim"))
    ref = O.load_dir(str(tmp_path / "ref"))
    shim = O.load_dir(str(tmp_path / "shim"))
    for k in SYMBOLIC:
        assert np.array_equal(ref[k], shim[k]), k
    try:
        import torch

        has_gpu = torch.cuda.is_available()
    except ImportError:
        has_gpu = False
    if not has_gpu:
        r = _run(SHIM, ["-amd", "-sn"], mfile, str(tmp_path / "shim2"), check=False)
        assert r.returncode == 3 and "mdgpu_factor" in r.stderr and "device" in r.stderr, r.stderr


CASES = [
    ("2d30_amd_sn", lambda: mg.laplacian_2d_5pt(30), ["-amd", "-sn"]),
    ("3d10_amd_sn", lambda: mg.laplacian_3d_varcoef(10, seed=2), ["-amd", "-sn"]),
    ("3d9_amd_rn4", lambda: mg.laplacian_3d_varcoef(9, seed=3), ["-amd", "-rn", "4"]),
    ("3d14_amd_sn", lambda: mg.laplacian_3d_varcoef(14, seed=4), ["-amd", "-sn"]),
]


@pytest.mark.gpu
@pytest.mark.parametrize("name,gen,flags", CASES, ids=[c[0] for c in CASES])
def test_reference_driver_with_the_shim_factor(tmp_path, name, gen, flags):
    _need_binaries()
    n, Ap, Ai, Ax = gen()
    mfile = str(tmp_path / "A.txt")
    mg.write_triplets(mfile, n, Ap, Ai, Ax)
    _run(O.REF_HARNESS, flags, mfile, str(tmp_path / "ref"))
    _run(SHIM, flags, mfile, str(tmp_path / "shim"))
    ref = O.load_dir(str(tmp_path / "ref"))
    shim = O.load_dir(str(tmp_path / "shim"))
    if name == "3d14_amd_sn":
        assert np.diff(ref["Lp"]).max() > 160  # large fronts on the GPU too
    assert np.array_equal(ref["Lp"], shim["Lp"])
    assert np.array_equal(ref["Li"], shim["Li"])
    d = np.linalg.norm(shim["Lx"] - ref["Lx"]) / np.linalg.norm(ref["Lx"])
    assert d <= 1e-12, d
    # the reference's own solve on the shim's L
    assert shim["meta"]["resid_rel"] <= 1e-14, shim["meta"]
    np.testing.assert_allclose(shim["x"], ref["x"], rtol=0, atol=1e-10 * np.abs(ref["x"]).max())


def _need_f32_binaries():
    if not (os.path.exists(SHIM32) and os.path.exists(REF32)):
        pytest.skip("FP32 reference harnesses not built (make -C oracle ref32 ref-shim32)")


def test_fp32_build_shim_binds_factor_to_the_library(tmp_path):
    """The reference's default FP32 build links the shim too: same symbolic
    phase as its own FP32 driver; without a GPU the numeric call reports that
    there is no device."""
    _need_f32_binaries()
    n, Ap, Ai, Ax = mg.laplacian_3d_varcoef(7, seed=1)
    mfile = str(tmp_path / "A.txt")
    mg.write_triplets(mfile, n, Ap, Ai, Ax)
    _run(REF32, ["-amd", "-sn", "-nofactor"], mfile, str(tmp_path / "ref"))
    _run(SHIM32, ["-amd", "-sn", "-nofactor"], mfile, str(tmp_path / "shim"))
    ref = O.load_dir(str(tmp_path / "ref"))
    shim = O.load_dir(str(tmp_path / "shim"))
    for k in SYMBOLIC:
        assert np.array_equal(ref[k], shim[k]), k
    try:
        import torch

        has_gpu = torch.cuda.is_available()
    except ImportError:
        has_gpu = False
    if not has_gpu:
        r = _run(SHIM32, ["-amd", "-sn"], mfile, str(tmp_path / "shim2"), check=False)
        assert r.returncode == 3 and "mdgpu_factor" in r.stderr and "device" in r.stderr, r.stderr


@pytest.mark.gpu
@pytest.mark.parametrize("name,gen,flags", CASES, ids=[c[0] for c in CASES])
def test_fp32_reference_driver_with_the_shim_factor(tmp_path, name, gen, flags):
    """FLOTANTE float: the shim factors in FP32 on the GPU and hands L back as
    float.  L has the reference's pattern and lies as close to the FP64 L as
    the reference's own FP32 factor does (both are FP32 factors: within 20x
    its error, and below 1e-5); the reference's FP32 solve on it reaches the
    residual of the reference's FP32 build (within 20x, below 1e-5)."""
    _need_binaries()
    _need_f32_binaries()
    n, Ap, Ai, Ax = gen()
    mfile = str(tmp_path / "A.txt")
    mg.write_triplets(mfile, n, Ap, Ai, Ax)
    _run(O.REF_HARNESS, flags, mfile, str(tmp_path / "ref64"))
    _run(REF32, flags, mfile, str(tmp_path / "ref32"))
    _run(SHIM32, flags, mfile, str(tmp_path / "shim32"))
    ref64 = O.load_dir(str(tmp_path / "ref64"))
    ref32 = O.load_dir(str(tmp_path / "ref32"))
    shim = O.load_dir(str(tmp_path / "shim32"))
    assert np.array_equal(ref32["Lp"], shim["Lp"])
    assert np.array_equal(ref32["Li"], shim["Li"])
    nrm = np.linalg.norm(ref64["Lx"])
    e_ref = np.linalg.norm(ref32["Lx"] - ref64["Lx"]) / nrm
    e_shim = np.linalg.norm(shim["Lx"] - ref64["Lx"]) / nrm
    assert e_shim <= max(20 * e_ref, 1e-7) and e_shim <= 1e-5, (e_shim, e_ref)
    r_ref, r_shim = ref32["meta"]["resid_rel"], shim["meta"]["resid_rel"]
    assert r_shim <= max(20 * r_ref, 1e-7) and r_shim <= 1e-5, (r_shim, r_ref)
