"""Host symbolic phase through the C ABI: bit-exact with the reference (CPU).

The golden digests were produced by the reference itself; the product's own
C++ symbolic code (mdgpu_b200/csrc/symbolic.cpp) must reproduce every array.
"""
import os
import re

import numpy as np
import pytest

import mdgpu_b200 as M
from oracle import oracle as O
from tests import golden_cases as G

MAN = G.manifest()
TREE = {"nodal": M.TREE_NODAL, "sn": M.TREE_SUPER, "rn": M.TREE_RELAXED}
KEYS = {"perm": "perm", "parent": "parent", "post": "post", "count0": "count0",
        "count": "count", "sn_first": "sn_nodo", "sn_ncols": "sn_cols",
        "child_ptr": "sn_childptr", "child": "sn_child", "relax_perm": "rn_perm"}
FAST = [k for k, v in MAN.items() if v["meta"]["n"] <= 40000]
SLOW = [k for k in MAN if k not in FAST]


def _solver(e, n, Ap, Ai):
    f = e["flags"]
    return M.Solver(n, Ap, Ai, ordering=int(f["amd"]), tree=TREE[f["mode"]],
                    relax_zeros=f.get("rn_zeros", 0))


def _check(name):
    e = MAN[name]
    n, Ap, Ai, _ = G.make_matrix(e["spec"])
    S = _solver(e, n, Ap, Ai)
    assert S.info("nsuper") == e["meta"]["nsuper"]
    assert S.info("lnz") == e["meta"]["lnz"]
    for k, gk in KEYS.items():
        if gk in e["sha"]:
            assert G.digest(S.array(k)) == e["sha"][gk], k
    assert G.digest(S.array("Lp").astype(np.int32)) == e["sha"]["Lp"]
    if "Li" in e["sha"]:
        _, Li, _ = S.get_L(values=False)
        assert G.digest(Li) == e["sha"]["Li"]
    if e["factor"]:
        assert S.info("flops") == int(e["meta"]["flops"])


@pytest.mark.parametrize("name", FAST)
def test_symbolic_bit_exact(name):
    _check(name)


@pytest.mark.slow
@pytest.mark.parametrize("name", SLOW)
def test_symbolic_bit_exact_large(name):
    _check(name)


@pytest.mark.parametrize("name", ["cfg1_2d100_amd_sn", "3d16_amd_sn", "3d16_amd_rn4",
                                  "rnd300_nat_nodal", "2d100_amd_nodal"])
def test_front_rows_and_extend_add_maps_match_reference_merges(name):
    """Front row sets and the child->parent relative index maps equal the ones
    the reference builds with MatrizGetFk_3 / VectorMerge / VectorMergeIndices
    (composed U2.ql -> Uk.ql, as restated by the oracle)."""
    e = MAN[name]
    n, Ap, Ai, Ax = G.make_matrix(e["spec"])
    f = e["flags"]
    P = O.Plan(n, Ap, Ai, Ax, amd=f["amd"], mode=f["mode"], rn_zeros=f.get("rn_zeros", 0))
    ref = P.factor(maps=True)
    S = _solver(e, n, Ap, Ai)
    np.testing.assert_array_equal(S.array("rows_ptr"), ref["rows_ptr"])
    np.testing.assert_array_equal(S.array("rows"), ref["rows"])
    relmap = S.array("relmap")
    cols = S.array("sn_ncols")
    rp = ref["rows_ptr"]
    mask = np.ones(len(relmap), bool)
    for s in range(len(cols)):
        mask[rp[s]:rp[s] + cols[s]] = False  # pivot rows carry no map
    np.testing.assert_array_equal(relmap[mask], ref["relmap"][mask])


def test_analyze_tree_matches_analyze():
    """mdgpu_analyze_tree (the Factor(cs*, cs*, ETree**, int) entry) builds the
    same plan from the reference's own symbolic outputs."""
    from mdgpu_b200 import matgen as mg

    n, Ap, Ai, Ax = mg.laplacian_3d_varcoef(10, seed=0)
    P = O.Plan(n, Ap, Ai, Ax, amd=True, mode="sn")
    S1 = M.Solver(n, Ap, Ai)
    S2 = M.Solver.from_tree(n, P.Ap, P.Ai, P.sn_nodo, P.sn_cols, P.sn_childptr, P.sn_child,
                            P.count)
    for k in ("rows_ptr", "rows", "relmap", "sn_first", "sn_ncols", "child"):
        np.testing.assert_array_equal(S1.array(k), S2.array(k))
    np.testing.assert_array_equal(S1.get_L(values=False)[1], S2.get_L(values=False)[1])


def test_vector_merge_known_answer():
    """testVectorMerge (mdgpu.cu:1610-1624): a front whose rows merge {2,5}
    into {0..5} maps them to positions {2,5}.  Built as a 2-supernode tree:
    child rows {2,5} (pivot 2) feeding a root with rows 0..5 (natural order,
    nodal tree of a matrix shaped to make those fronts)."""
    # column 2 couples to 5; columns 0..5 all couple to 5 (arrow into 5)
    n = 6
    cols = {0: [0, 5], 1: [1, 5], 2: [2, 5], 3: [3, 5], 4: [4, 5], 5: [5]}
    Ap = [0]
    Ai = []
    for j in range(n):
        Ai += cols[j]
        Ap.append(len(Ai))
    S = M.Solver(n, np.array(Ap), np.array(Ai), ordering=M.ORDER_NATURAL, tree=M.TREE_NODAL)
    rp = S.array("rows_ptr")
    rows = S.array("rows")
    first = S.array("sn_first")
    s2 = int(np.where(first == 2)[0][0])
    assert list(rows[rp[s2]:rp[s2 + 1]]) == [2, 5]
    root = len(first) - 1
    assert list(rows[rp[root]:rp[root + 1]]) == [5]
    relmap = S.array("relmap")
    assert relmap[rp[s2] + 1] == 0


def test_forest_is_rejected():
    # two disconnected blocks: the reference's GetETree rejects a forest
    n = 4
    Ap = np.array([0, 2, 3, 5, 6], np.int32)
    Ai = np.array([0, 1, 1, 2, 3, 3], np.int32)
    with pytest.raises(M.MdgpuError) as ei:
        M.Solver(n, Ap, Ai)
    assert ei.value.status == -5


def test_invalid_input_is_rejected():
    n = 3
    Ap = np.array([0, 1, 2, 3], np.int32)
    Ai = np.array([1, 0, 2], np.int32)  # entry above the diagonal in column 1
    with pytest.raises(M.MdgpuError) as ei:
        M.Solver(n, Ap, Ai)
    assert ei.value.status == -1


def test_library_exports_every_declared_symbol():
    header = open(os.path.join(G.HERE, "..", "..", "include", "mdgpu_b200.h")).read()
    declared = set(re.findall(r"MDGPU_API[^;(]*?\b(mdgpu_\w+)\s*\(", header))
    assert declared == set(M.EXPORTS)
    L = M.lib()
    for name in declared:
        assert hasattr(L, name), name


def test_numeric_calls_fail_loudly_without_a_device():
    torch = pytest.importorskip("torch")
    if torch.cuda.is_available():
        pytest.skip("a device is present")
    from mdgpu_b200 import matgen as mg

    n, Ap, Ai, Ax = mg.laplacian_2d_5pt(10)
    S = M.Solver(n, Ap, Ai)
    assert S.info("on_device") == 0
    with pytest.raises(M.MdgpuError) as ei:
        S.factor(Ax)
    assert ei.value.status == -7
