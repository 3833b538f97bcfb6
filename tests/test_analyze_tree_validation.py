"""mdgpu_analyze_tree checks the caller's lower triangle and assembly tree
before using any of it as an index (the inputs of the reference's
Factor(cs *A, cs *spL, ETree **listaNodos, int cantNodos), mdgpu.cu:1394,
ETree at etree.h:6-19): each malformed tree is rejected with
MDGPU_ERR_INVALID and a message naming what is wrong, the same message on
every run, and a valid tree still analyses (CPU only)."""
import numpy as np
import pytest

import mdgpu_b200 as M
from mdgpu_b200 import matgen as mg
from oracle import oracle as O


@pytest.fixture(scope="module")
def tree():
    n, Ap, Ai, Ax = mg.laplacian_3d_varcoef(8, seed=0)
    P = O.Plan(n, Ap, Ai, Ax, amd=True, mode="sn")
    return dict(n=n, Ap=np.array(P.Ap, np.int32), Ai=np.array(P.Ai, np.int32),
                first_col=np.array(P.sn_nodo, np.int32), ncols=np.array(P.sn_cols, np.int32),
                child_ptr=np.array(P.sn_childptr, np.int32),
                child=np.array(P.sn_child, np.int32), count=np.array(P.count, np.int32))


def _analyze(t):
    return M.Solver.from_tree(t["n"], t["Ap"], t["Ai"], t["first_col"], t["ncols"],
                              t["child_ptr"], t["child"], t["count"])


def _copy(t):
    return {k: (v.copy() if isinstance(v, np.ndarray) else v) for k, v in t.items()}


def test_valid_tree_analyses(tree):
    S = _analyze(tree)
    assert S.info("nsuper") == len(tree["first_col"])


def _parent_of_first_child(t):
    return int(np.nonzero(np.diff(t["child_ptr"]) > 0)[0][0])


def _bad_child_out_of_range(t):
    t["child"][0] = 999999


def _bad_child_not_earlier(t):
    s = _parent_of_first_child(t)
    t["child"][t["child_ptr"][s]] = s  # its own child: not an earlier supernode


def _bad_child_ptr_decreasing(t):
    cp = t["child_ptr"]
    s = int(np.nonzero(np.diff(cp) > 0)[0][0])
    cp[s + 1] = cp[s] - 1 if cp[s] > 0 else -1


def _bad_two_parents(t):
    t["child"][1] = t["child"][0]  # the second child entry repeats the first


def _bad_missing_child(t):
    t["child_ptr"][-1] -= 1


def _bad_uncovered_column(t):
    s = int(np.nonzero(t["ncols"] > 1)[0][0])
    t["ncols"][s] -= 1  # its last column is then covered by no supernode


def _bad_first_col_out_of_range(t):
    t["first_col"][0] = t["n"] + 5


def _bad_shared_column(t):
    ones = np.nonzero(t["ncols"] == 1)[0]
    t["first_col"][ones[1]] = t["first_col"][ones[0]]


def _bad_zero_columns(t):
    t["ncols"][0] = 0


def _bad_count_too_large(t):
    t["count"][t["n"] - 1] = 2


def _bad_count_not_supernodal(t):
    s = int(np.nonzero(t["ncols"] > 1)[0][0])
    t["count"][t["first_col"][s] + 1] += 1


def _bad_entry_above_diagonal(t):
    j = 5
    t["Ai"][t["Ap"][j]] = j - 1


def _bad_first_colptr(t):
    t["Ap"][0] = 1


CASES = [
    (_bad_child_out_of_range, "not an earlier supernode"),
    (_bad_child_not_earlier, "not an earlier supernode"),
    (_bad_child_ptr_decreasing, "child_ptr"),
    (_bad_two_parents, "two parents"),
    (_bad_missing_child, "child lists"),
    (_bad_uncovered_column, "belongs to no supernode"),
    (_bad_first_col_out_of_range, "first column out of range"),
    (_bad_shared_column, "belongs to two supernodes"),
    (_bad_zero_columns, "column count out of range"),
    (_bad_count_too_large, "count["),
    (_bad_count_not_supernodal, "not those of a supernode"),
    (_bad_entry_above_diagonal, "outside the lower triangle"),
    (_bad_first_colptr, "Ap[0]"),
]


@pytest.mark.parametrize("mutate,what", CASES, ids=[c[0].__name__[5:] for c in CASES])
def test_malformed_tree_is_rejected(tree, mutate, what):
    msgs = set()
    for _ in range(3):
        t = _copy(tree)
        mutate(t)
        with pytest.raises(M.MdgpuError) as ei:
            _analyze(t)
        assert ei.value.status == -1, str(ei.value)
        assert what in str(ei.value), str(ei.value)
        msgs.add(str(ei.value))
    assert len(msgs) == 1  # the same diagnosis every time: nothing read out of bounds first
