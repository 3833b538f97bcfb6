"""Seeded synthetic SPD test matrices with the shapes of the benchmark workloads.

All generators return the LOWER triangle (diagonal included) in compressed
sparse column form ``(n, Ap, Ai, Ax)`` with int32 indices, row indices sorted
ascending inside each column -- the layout the reference's ``cs`` struct holds
after ``cs_compress`` of a column-sorted triplet file (cs.cpp:251).

``write_triplets`` writes the reference's input format: a headerless text file
of 1-based ``i j x`` lines (cs.cpp:4-27), lower triangle only, one entry per
line in column-major order, values printed with 17 significant digits so the
reference parses exactly the doubles generated here.

Grid numbering is lexicographic, node (x, y, z) -> x + nx*(y + ny*z).  Edge
conductances are drawn from ``numpy.random.default_rng(seed)`` (PCG64) in a
fixed order: all x-edges, then y-edges, then z-edges, each block in node
order of the edge's lower endpoint.
"""
from __future__ import annotations

import numpy as np


def _edges_grid(dims):
    """Return (lo, hi, axis) arrays of the 2*d-point stencil edges of a grid."""
    dims = tuple(int(d) for d in dims)
    idx = np.arange(int(np.prod(dims)), dtype=np.int64).reshape(dims[::-1])  # [z][y][x]
    los, his = [], []
    nd = len(dims)
    for ax in range(nd):
        # axis 0 is x which is the last axis of idx
        a = nd - 1 - ax
        sl_lo = [slice(None)] * nd
        sl_hi = [slice(None)] * nd
        sl_lo[a] = slice(0, dims[ax] - 1)
        sl_hi[a] = slice(1, dims[ax])
        lo = idx[tuple(sl_lo)].ravel()
        hi = idx[tuple(sl_hi)].ravel()
        order = np.argsort(lo, kind="stable")
        los.append(lo[order])
        his.append(hi[order])
    return los, his


def _assemble_lower(n, rows, cols, vals):
    """Sum duplicate (row, col) lower-triangle entries and build sorted CSC."""
    rows = np.asarray(rows, dtype=np.int64)
    cols = np.asarray(cols, dtype=np.int64)
    vals = np.asarray(vals, dtype=np.float64)
    assert np.all(rows >= cols)
    key = cols * n + rows
    order = np.argsort(key, kind="stable")
    key = key[order]
    vals = vals[order]
    uniq, start = np.unique(key, return_index=True)
    sums = np.add.reduceat(vals, start) if len(vals) else vals
    c = (uniq // n).astype(np.int64)
    r = (uniq % n).astype(np.int32)
    Ap = np.zeros(n + 1, dtype=np.int64)
    np.add.at(Ap, c + 1, 1)
    Ap = np.cumsum(Ap).astype(np.int32)
    return n, Ap, r.astype(np.int32), sums.astype(np.float64)


def laplacian_grid(dims, *, seed=None, sigma=1.0, shift=0.0, const=None):
    """Variable- or constant-coefficient 2D/3D grid Laplacian, lower CSC.

    ``const=(diag, off)`` gives the constant stencil (e.g. ``(4, -1)`` for the
    2D 5-point Dirichlet Laplacian).  Otherwise each edge has conductance
    c ~ lognormal(0, sigma) drawn from ``default_rng(seed)``; off-diagonals
    are -c and the diagonal is the sum of incident conductances + ``shift``.
    """
    dims = tuple(int(d) for d in dims)
    n = int(np.prod(dims))
    los, his = _edges_grid(dims)
    lo = np.concatenate(los)
    hi = np.concatenate(his)
    if const is not None:
        d, off = const
        cond = np.full(lo.shape, -float(off))
        diag = np.full(n, float(d))
    else:
        rng = np.random.default_rng(seed)
        cond = np.concatenate([rng.lognormal(0.0, sigma, size=len(l)) for l in los])
        diag = np.full(n, float(shift))
        np.add.at(diag, lo, cond)
        np.add.at(diag, hi, cond)
    rows = np.concatenate([np.arange(n), hi])
    cols = np.concatenate([np.arange(n), lo])
    vals = np.concatenate([diag, -cond])
    return _assemble_lower(n, rows, cols, vals)


def laplacian_grid_edges(dims, *, seed=None, sigma=1.0, shift=0.0):
    """laplacian_grid with its edges: (n, Ap, Ai, Ax, lo, hi, cond), edge e
    joining unknowns lo[e] < hi[e] with conductance cond[e] (the same draws
    as laplacian_grid for the same arguments)."""
    dims = tuple(int(d) for d in dims)
    n = int(np.prod(dims))
    los, his = _edges_grid(dims)
    lo = np.concatenate(los)
    hi = np.concatenate(his)
    rng = np.random.default_rng(seed)
    cond = np.concatenate([rng.lognormal(0.0, sigma, size=len(l)) for l in los])
    diag = np.full(n, float(shift))
    np.add.at(diag, lo, cond)
    np.add.at(diag, hi, cond)
    rows = np.concatenate([np.arange(n), hi])
    cols = np.concatenate([np.arange(n), lo])
    vals = np.concatenate([diag, -cond])
    n, Ap, Ai, Ax = _assemble_lower(n, rows, cols, vals)
    return n, Ap, Ai, Ax, lo, hi, cond


def laplacian_2d_5pt(side=100):
    """2D 5-point Dirichlet Laplacian: diagonal 4, off-diagonals -1."""
    return laplacian_grid((side, side), const=(4.0, -1.0))


def laplacian_3d_varcoef(side=64, seed=0, sigma=1.0, shift=1e-3):
    """3D 7-point Laplacian with lognormal(0, sigma) edge conductances."""
    return laplacian_grid((side, side, side), seed=seed, sigma=sigma, shift=shift)


def random_spd(n, density=0.05, seed=0):
    """Random sparse SPD matrix (diagonally dominant), lower CSC."""
    rng = np.random.default_rng(seed)
    m = max(1, int(density * n * (n - 1) / 2))
    r = rng.integers(0, n, size=m)
    c = rng.integers(0, n, size=m)
    keep = r != c
    r, c = r[keep], c[keep]
    lo = np.minimum(r, c)
    hi = np.maximum(r, c)
    v = -rng.uniform(0.1, 1.0, size=len(lo))
    diag = np.full(n, 1.0)
    np.add.at(diag, lo, -v)
    np.add.at(diag, hi, -v)
    rows = np.concatenate([np.arange(n), hi])
    cols = np.concatenate([np.arange(n), lo])
    vals = np.concatenate([diag, v])
    return _assemble_lower(n, rows, cols, vals)


def rhs_uniform(n, seed=0, nrhs=1):
    """Right-hand sides with entries i.i.d. U(-1, 1), column-major (n, nrhs)."""
    rng = np.random.default_rng(seed)
    b = rng.uniform(-1.0, 1.0, size=(nrhs, n)).T
    return np.ascontiguousarray(b if nrhs > 1 else b[:, 0])


def lower_to_full_scipy(n, Ap, Ai, Ax):
    """Full symmetric scipy CSC matrix from the lower CSC triple."""
    import scipy.sparse as sp

    L = sp.csc_matrix((Ax, Ai, Ap), shape=(n, n))
    return (L + sp.tril(L, -1).T).tocsc()


def write_triplets(path, n, Ap, Ai, Ax):
    """Write the reference's headerless 1-based ``i j x`` triplet file."""
    cols = np.repeat(np.arange(n, dtype=np.int64), np.diff(Ap))
    with open(path, "w") as f:
        lines = [
            "%d %d %.17g\n" % (int(i) + 1, int(j) + 1, float(x))
            for i, j, x in zip(Ai, cols, Ax)
        ]
        f.writelines(lines)


def elasticity_3dof(side=40, seed=0, sigma=1.0, shift=1e-2):
    """3 unknowns per node of a side^3 node grid with 27-point connectivity,
    elasticity-like: for an edge (i, j) with stencil offset unit vector e,
    B_ij = w_ij (I_3 + 0.5 e e') with w_ij ~ lognormal(0, sigma); the
    off-diagonal block is -B_ij and the diagonal block sum_j B_ij + shift I_3
    (a sum of positive semidefinite edge terms plus shift I: SPD).  Unknown
    3 k + c is component c of node k.  Lower CSC of the 3 side^3 system."""
    side = int(side)
    nn = side ** 3
    idx = np.arange(nn, dtype=np.int64).reshape(side, side, side)  # [z][y][x]
    rng = np.random.default_rng(seed)
    rows, cols, vals = [], [], []
    diag = np.zeros((nn, 3, 3))
    # the 13 offsets with a positive first nonzero component: each edge once
    offs = [(dz, dy, dx) for dz in (-1, 0, 1) for dy in (-1, 0, 1) for dx in (-1, 0, 1)
            if (dz, dy, dx) > (0, 0, 0)]
    for dz, dy, dx in offs:
        e = np.array([dx, dy, dz], dtype=np.float64)
        e /= np.linalg.norm(e)
        K = np.eye(3) + 0.5 * np.outer(e, e)
        sz = slice(max(0, -dz), side - max(0, dz))
        sy = slice(max(0, -dy), side - max(0, dy))
        sx = slice(max(0, -dx), side - max(0, dx))
        a = idx[sz, sy, sx].ravel()
        b = idx[sz.start + dz:sz.stop + dz, sy.start + dy:sy.stop + dy,
                sx.start + dx:sx.stop + dx].ravel()
        w = rng.lognormal(0.0, sigma, size=a.size)
        Bs = w[:, None, None] * K[None]
        np.add.at(diag, a, Bs)
        np.add.at(diag, b, Bs)
        lo, hi = np.minimum(a, b), np.maximum(a, b)
        for ci in range(3):
            for cj in range(3):
                rows.append(3 * hi + ci)
                cols.append(3 * lo + cj)
                vals.append(-Bs[:, ci, cj])
    diag += shift * np.eye(3)[None]
    k = np.arange(nn)
    for ci in range(3):
        for cj in range(ci + 1):
            rows.append(3 * k + ci)
            cols.append(3 * k + cj)
            vals.append(diag[:, ci, cj])
    return _assemble_lower(3 * nn, np.concatenate(rows), np.concatenate(cols),
                           np.concatenate(vals))


def node_graph_lower(side=40):
    """Pattern of the side^3 node grid with 27-point connectivity (lower CSC,
    unit values): the graph the 3-unknown systems are ordered on."""
    side = int(side)
    nn = side ** 3
    idx = np.arange(nn, dtype=np.int64).reshape(side, side, side)
    rows, cols = [np.arange(nn)], [np.arange(nn)]
    for dz, dy, dx in [(dz, dy, dx) for dz in (-1, 0, 1) for dy in (-1, 0, 1)
                       for dx in (-1, 0, 1) if (dz, dy, dx) > (0, 0, 0)]:
        sz = slice(max(0, -dz), side - max(0, dz))
        sy = slice(max(0, -dy), side - max(0, dy))
        sx = slice(max(0, -dx), side - max(0, dx))
        a = idx[sz, sy, sx].ravel()
        b = idx[sz.start + dz:sz.stop + dz, sy.start + dy:sy.stop + dy,
                sx.start + dx:sx.stop + dx].ravel()
        rows.append(np.maximum(a, b))
        cols.append(np.minimum(a, b))
    r, c = np.concatenate(rows), np.concatenate(cols)
    return _assemble_lower(nn, r, c, np.ones(r.size))


def expand_node_perm(perm, dof=3):
    """A node permutation (new -> old) as one of the node's unknowns."""
    perm = np.asarray(perm, dtype=np.int64)
    return (dof * perm[:, None] + np.arange(dof)[None, :]).ravel().astype(np.int32)


def permute_lower(n, Ap, Ai, Ax, perm):
    """Lower CSC of P A P' (perm: new -> old) from the lower CSC of A."""
    perm = np.asarray(perm, dtype=np.int64)
    inv = np.empty(n, dtype=np.int64)
    inv[perm] = np.arange(n)
    cols = np.repeat(np.arange(n), np.diff(Ap))
    r, c = inv[np.asarray(Ai, dtype=np.int64)], inv[cols]
    return _assemble_lower(n, np.maximum(r, c), np.minimum(r, c), np.asarray(Ax, dtype=np.float64))
