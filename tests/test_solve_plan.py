"""Host logic of the solve plan, checked on CPU against a restatement from
the front row sets: the warp lists (small fronts of each level by rows
descending, split into fronts taking a warp, half a warp and a quarter warp)
and the forward assembly map of the large fronts (per front row, the
children's front-vector rows that add into it, in child order -- the same
sums as a child-by-child scatter through the relative maps).
"""
import numpy as np
import pytest

import mdgpu_b200 as M
from mdgpu_b200 import matgen as mg

LARGE = 160  # rows above which a front is tiled


def _cases():
    return [
        ("3d16", mg.laplacian_3d_varcoef(16, seed=0), M.TREE_SUPER, 0),
        ("3d12_rn4", mg.laplacian_3d_varcoef(12, seed=1), M.TREE_RELAXED, 4),
        ("2d60", mg.laplacian_2d_5pt(60), M.TREE_SUPER, 0),
    ]


@pytest.mark.parametrize("name,sys,tree,z", _cases(), ids=[c[0] for c in _cases()])
def test_warp_lists_and_assembly_map(name, sys, tree, z):
    n, Ap, Ai, _ = sys
    S = M.Solver(n, Ap, Ai, tree=tree, relax_zeros=z)
    ptr = S.array("rows_ptr")
    m = np.diff(ptr)
    c = S.array("sn_ncols")
    level = S.array("level")
    cp, ch = S.array("child_ptr"), S.array("child")
    relmap = S.array("relmap")
    nl = S.info("nlevels")
    fv_off = np.concatenate([[0], np.cumsum(m)[:-1]])

    # warp lists: per level the small fronts, rows descending, and the counts
    wl, wc = S.array("warp_list"), S.array("warp_cnt").reshape(nl, 3)
    pos = 0
    for lv in range(nl):
        small = np.flatnonzero((level == lv) & (m <= LARGE))
        got = wl[pos:pos + small.size]
        pos += small.size
        assert sorted(got.tolist()) == sorted(small.tolist())
        assert np.all(np.diff(m[got]) <= 0)
        mm = m[got]
        assert wc[lv].tolist() == [int((mm > 16).sum()), int(((mm > 8) & (mm <= 16)).sum()),
                                   int((mm <= 8).sum())]
    assert pos == wl.size

    # assembly map: restated from the children's update rows in child order
    aoff, arow, aent = S.array("amap_off"), S.array("amap_row"), S.array("amap_ent")
    nlarge = 0
    for s in range(m.size):
        if m[s] <= LARGE:
            assert aoff[s] == -1
            continue
        nlarge += 1
        want = [[] for _ in range(m[s])]
        for h in range(cp[s], cp[s + 1]):
            g = ch[h]
            for rr in range(m[g] - c[g]):
                want[relmap[ptr[g] + c[g] + rr]].append(fv_off[g] + c[g] + rr)
        r0 = arow[aoff[s]:aoff[s] + m[s] + 1]
        for r in range(m[s]):
            assert aent[r0[r]:r0[r + 1]].tolist() == want[r]
    assert nlarge == S.info("large_fronts")


def test_assembly_map_gather_equals_scatter():
    """Numerically: gathering through the map gives the scatter's sums bit
    for bit (same terms in the same order)."""
    n, Ap, Ai, _ = mg.laplacian_3d_varcoef(16, seed=2)
    S = M.Solver(n, Ap, Ai)
    ptr = S.array("rows_ptr")
    m, c = np.diff(ptr), S.array("sn_ncols")
    cp, ch, relmap = S.array("child_ptr"), S.array("child"), S.array("relmap")
    aoff, arow, aent = S.array("amap_off"), S.array("amap_row"), S.array("amap_ent")
    fv = np.random.default_rng(0).standard_normal(int(m.sum()))
    fv_off = np.concatenate([[0], np.cumsum(m)[:-1]])
    for s in np.flatnonzero(m > LARGE):
        scat = np.zeros(m[s])
        for h in range(cp[s], cp[s + 1]):
            g = ch[h]
            for rr in range(m[g] - c[g]):
                scat[relmap[ptr[g] + c[g] + rr]] += fv[fv_off[g] + c[g] + rr]
        r0 = arow[aoff[s]:aoff[s] + m[s] + 1]
        gath = np.zeros(m[s])
        for r in range(m[s]):
            acc = 0.0
            for e in range(r0[r], r0[r + 1]):
                acc += fv[aent[e]]
            gath[r] = acc
        np.testing.assert_array_equal(gath, scat)
