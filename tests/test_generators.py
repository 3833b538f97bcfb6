"""Host-side generators for the multi-unknown workload: the 3-unknowns-per-
node elasticity-like system on a 27-point node grid, its node graph, the
expansion of a node ordering to the unknowns and the symmetric permutation
of a lower triangle.  CPU only.
"""
import numpy as np

import mdgpu_b200 as M
from mdgpu_b200 import matgen as mg


def _dense(n, Ap, Ai, Ax):
    return mg.lower_to_full_scipy(n, Ap, Ai, Ax).toarray()


def test_elasticity_system_is_spd_with_the_stated_blocks():
    side = 3
    n, Ap, Ai, Ax = mg.elasticity_3dof(side, seed=2, sigma=1.0, shift=1e-2)
    assert n == 3 * side ** 3
    A = _dense(n, Ap, Ai, Ax)
    assert np.allclose(A, A.T)
    # edge terms annihilate equal displacements: the smallest eigenvalue is
    # the diagonal shift
    ev = np.linalg.eigvalsh(A)
    assert abs(ev[0] - 1e-2) <= 1e-9 and np.all(ev > 0)
    # the block of nodes 0 and 1 (offset +x): -w (I + 0.5 e e'), e = x
    B = -A[3:6, 0:3]
    w = B[1, 1]
    assert w > 0
    np.testing.assert_allclose(B, w * (np.eye(3) + 0.5 * np.diag([1.0, 0, 0])), atol=1e-14)
    # each node couples to at most 26 others (27-point connectivity)
    G = _dense(*mg.node_graph_lower(side))
    assert (G != 0).sum(axis=1).max() == 27


def test_node_ordering_expanded_and_applied():
    side = 3
    n, Ap, Ai, Ax = mg.elasticity_3dof(side, seed=3)
    nn, gp, gi, gx = mg.node_graph_lower(side)
    perm_nodes = M.Solver(nn, gp, gi, ordering=M.ORDER_AMD).array("perm")
    perm = mg.expand_node_perm(perm_nodes)
    assert sorted(perm.tolist()) == list(range(n))
    np.testing.assert_array_equal(perm[3 * 5:3 * 6], 3 * perm_nodes[5] + np.arange(3))
    n2, Ap2, Ai2, Ax2 = mg.permute_lower(n, Ap, Ai, Ax, perm)
    A = _dense(n, Ap, Ai, Ax)
    np.testing.assert_allclose(_dense(n2, Ap2, Ai2, Ax2), A[np.ix_(perm, perm)], atol=0)
    # the permuted system analyses in natural order
    S = M.Solver(n2, Ap2, Ai2, ordering=M.ORDER_NATURAL)
    assert S.info("lnz") > 0
