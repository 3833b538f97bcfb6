"""The file reader mdgpu_load_triplet against a restatement of the reference's
cs_load + cs_compress (cs.cpp:4-27, 251-270): 1-based "i j x" triples read
until the first line that is not one, sizes from the largest indices, a
column's entries in file order; and the Matrix Market variant (comment
lines, the size line, its sizes checked).  CPU only.
"""
import numpy as np
import pytest

import mdgpu_b200 as M
from mdgpu_b200 import matgen as mg


def _restated(triples):
    """cs_load + cs_compress on a list of 1-based (i, j, x)."""
    m = max((t[0] for t in triples), default=0)
    n = max((t[1] for t in triples), default=0)
    cnt = np.zeros(n + 1, np.int64)
    for _, j, _ in triples:
        cnt[j] += 1
    Ap = np.cumsum(cnt).astype(np.int32)
    nxt = Ap[:-1].copy()
    Ai = np.zeros(len(triples), np.int32)
    Ax = np.zeros(len(triples))
    for i, j, x in triples:
        p = nxt[j - 1]
        nxt[j - 1] += 1
        Ai[p], Ax[p] = i - 1, x
    return m, n, Ap, Ai, Ax


def test_reference_format_matches_restatement(tmp_path):
    rng = np.random.default_rng(3)
    triples = [(int(rng.integers(1, 30)), int(rng.integers(1, 25)), float(rng.standard_normal()))
               for _ in range(200)]
    f = tmp_path / "a.txt"
    # the reading stops at the first line that is not a triple
    f.write_text("".join(f"{i} {j} {x!r}\n" for i, j, x in triples) + "end\n7 7 1.0\n")
    m, n, Ap, Ai, Ax = M.load_triplet(f)
    em, en, eAp, eAi, eAx = _restated(triples)
    assert (m, n) == (em, en)
    np.testing.assert_array_equal(Ap, eAp)
    np.testing.assert_array_equal(Ai, eAi)
    np.testing.assert_array_equal(Ax, eAx)


def test_matrix_market_round_trip_gives_the_same_analysis(tmp_path):
    n, Ap, Ai, Ax = mg.laplacian_3d_varcoef(9, seed=5)
    f = tmp_path / "lap.mtx"
    lines = ["%%MatrixMarket matrix coordinate real symmetric", "% lower triangle",
             f"{n} {n} {Ap[-1]}"]
    for j in range(n):
        for p in range(Ap[j], Ap[j + 1]):
            lines.append(f"{Ai[p] + 1} {j + 1} {float(Ax[p])!r}")
    f.write_text("\n".join(lines) + "\n")
    m2, n2, Ap2, Ai2, Ax2 = M.load_triplet(f, matrix_market=True)
    assert (m2, n2) == (n, n)
    np.testing.assert_array_equal(Ap2, Ap)
    np.testing.assert_array_equal(Ai2, Ai)
    np.testing.assert_array_equal(Ax2, Ax)
    S1, S2 = M.Solver(n, Ap, Ai), M.Solver(n2, Ap2, Ai2)
    for name in ("perm", "sn_first", "Lp"):
        np.testing.assert_array_equal(S1.array(name), S2.array(name))


def test_matrix_market_stated_size_kept_and_checked(tmp_path):
    f = tmp_path / "s.mtx"
    f.write_text("%%MatrixMarket matrix coordinate real symmetric\n5 5 2\n1 1 2.0\n3 2 -1.0\n")
    m, n, Ap, Ai, Ax = M.load_triplet(f, matrix_market=True)
    assert (m, n) == (5, 5) and Ap.tolist() == [0, 1, 2, 2, 2, 2]
    g = tmp_path / "t.mtx"
    g.write_text("%%MatrixMarket matrix coordinate real symmetric\n2 2 1\n3 1 1.0\n")
    with pytest.raises(M.MdgpuError) as e:
        M.load_triplet(g, matrix_market=True)
    assert "outside" in str(e.value)


def test_index_below_one_and_missing_file_are_errors(tmp_path):
    f = tmp_path / "z.txt"
    f.write_text("1 1 4.0\n0 1 -1.0\n")
    with pytest.raises(M.MdgpuError) as e:
        M.load_triplet(f)
    assert "below 1" in str(e.value)
    with pytest.raises(M.MdgpuError):
        M.load_triplet(tmp_path / "missing.txt")
