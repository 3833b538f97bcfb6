"""The plan self-check (mdgpu_check_plan, mdgpu_b200/csrc/plan_check.cpp):
every invariant the device kernels rely on when they index the plan's tables
holds on the plans of many kinds of input, and each of twelve broken
invariants is caught and named (tests/plan_check_host.cpp compiles the
library's own host analysis, plan builders and check with g++).  CPU only.
"""
import os
import shutil
import subprocess

import numpy as np
import pytest

import mdgpu_b200 as M
from mdgpu_b200 import matgen as mg

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "mdgpu_b200", "csrc")


def _plans():
    yield "2d60", M.Solver(*mg.laplacian_2d_5pt(60)[:3])
    yield "3d18", M.Solver(*mg.laplacian_3d_varcoef(18, seed=1)[:3])
    yield "3d12_relaxed8", M.Solver(*mg.laplacian_3d_varcoef(12, seed=2)[:3],
                                    tree=M.TREE_RELAXED, relax_zeros=8)
    yield "3d9_nodal", M.Solver(*mg.laplacian_3d_varcoef(9, seed=3)[:3], tree=M.TREE_NODAL)
    yield "3d9_natural", M.Solver(*mg.laplacian_3d_varcoef(9, seed=3)[:3],
                                  ordering=M.ORDER_NATURAL)
    yield "elasticity6", M.Solver(*mg.elasticity_3dof(6, seed=1)[:3])
    syss = [mg.laplacian_grid((s,) * d, seed=s, sigma=0.5, shift=1e-2)
            for s, d in ((12, 2), (7, 3), (30, 2), (10, 3), (5, 3))]
    yield "batch5", M.Solver.batch([s[:3] for s in syss])
    # repeated entries: the assembly keeps the last, the map drops the rest
    n, Ap, Ai, _ = mg.laplacian_2d_5pt(5)
    Ap2 = Ap.copy()
    Ai2 = np.insert(Ai, Ap[3], Ai[Ap[3]])
    Ap2[4:] += 1
    yield "repeated", M.Solver(n, Ap2, Ai2)


@pytest.mark.parametrize("name", [p[0] for p in _plans()])
def test_plans_pass_the_check(name):
    S = dict(_plans())[name]
    S.check_plan()
    if name == "3d18":
        assert S.info("large_fronts") > 0  # assembly maps and solve tasks checked too


EXPECT = {
    "rows": "rows not strictly increasing",
    "relmap": "relative map entry",
    "a_pos": "A entry position",
    "loff": "L panel offset",
    "warp_list": "warp list",
    "tasks": "forward pivot order",
    "items": "solve items out of dependency order",
    "amap": "assembly map",
    "csr": "CSR entry out of range",
    "level": "child level not below",
    "panel": "panel task order",
    "uoff": "update matrices live together share storage",
}


def test_each_broken_invariant_is_caught(tmp_path):
    cxx = shutil.which("g++")
    if cxx is None:
        pytest.skip("needs g++")
    exe = str(tmp_path / "plan_check_host")
    subprocess.run([cxx, "-O2", "-std=c++17", "-I", CSRC,
                    os.path.join(ROOT, "tests", "plan_check_host.cpp"),
                    os.path.join(CSRC, "plan.cpp"), os.path.join(CSRC, "symbolic.cpp"),
                    os.path.join(CSRC, "plan_check.cpp"), "-o", exe, "-lpthread"], check=True)
    out = subprocess.run([exe, "16"], check=True, capture_output=True, text=True).stdout
    got = dict(line.split(": ", 1) for line in out.strip().splitlines())
    assert got.pop("intact") == "ok"
    assert set(got) == set(EXPECT)
    for k, v in EXPECT.items():
        assert v in got[k], (k, got[k])


def _random_connected_lower(n, extra, rng):
    """Lower CSC of a random connected pattern: a random spanning tree plus
    `extra` random edges (so the elimination tree is one tree)."""
    edges = set()
    order = rng.permutation(n)
    for k in range(1, n):
        a, b = order[k], order[rng.integers(0, k)]
        edges.add((max(a, b), min(a, b)))
    for _ in range(extra):
        a, b = rng.integers(0, n, 2)
        if a != b:
            edges.add((max(a, b), min(a, b)))
    cols = [[j] for j in range(n)]
    for i, j in edges:
        cols[j].append(i)
    Ap, Ai = [0], []
    for j in range(n):
        Ai.extend(sorted(cols[j]))
        Ap.append(len(Ai))
    return n, np.array(Ap, np.int32), np.array(Ai, np.int32)


@pytest.mark.parametrize("seed", range(12))
def test_random_patterns_pass_the_check(seed):
    rng = np.random.default_rng(100 + seed)
    n = int(rng.integers(1, 400))
    n, Ap, Ai = _random_connected_lower(n, int(rng.integers(0, 6 * n + 1)), rng)
    for kw in ({}, {"tree": M.TREE_NODAL}, {"tree": M.TREE_RELAXED, "relax_zeros": 6},
               {"ordering": M.ORDER_NATURAL}):
        S = M.Solver(n, Ap, Ai, **kw)
        S.check_plan()


def test_check_before_upload_when_asked():
    """MDGPU_CHECK_PLAN=1 runs the check inside every analysis, before the
    tables would reach the device."""
    import sys

    code = ("import mdgpu_b200 as M; from mdgpu_b200 import matgen as mg; "
            "M.Solver(*mg.laplacian_3d_varcoef(14, seed=1)[:3]); "
            "M.Solver.batch([mg.laplacian_2d_5pt(9)[:3], mg.laplacian_2d_5pt(6)[:3]]); "
            "print('analysed')")
    env = dict(os.environ, MDGPU_CHECK_PLAN="1", PYTHONPATH=ROOT)
    out = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True,
                         timeout=300, check=True).stdout
    assert "analysed" in out
