"""Independent systems across GPUs, one process per GPU.

The systems of a batch share nothing, so a multi-GPU run needs no exchange
on the data path: every rank computes the same partition of the systems from
their flop estimates (``estimate_batch``, deterministic, so no collective is
needed to agree on it), builds one batch handle over its own share and
factors and solves it on its own GPU.  The one exchange is host-side, after
the solve: ``ShardedBatch.gather`` collects per-system results on one rank
(``torch.distributed.gather_object``, any backend).

Partition: longest processing time first -- systems by estimated flops,
largest first, each to the rank with the least work so far -- which keeps the
slowest rank within 4/3 of the best possible split (Graham 1969).
"""
from __future__ import annotations

import numpy as np

from . import ORDER_AMD, TREE_SUPER, Solver, estimate_batch


def lpt_partition(costs, nparts):
    """Split item indices into nparts lists by longest processing time first:
    items by cost descending (ties: lower index first), each to the part with
    the least total so far (ties: lower part).  Each part's indices come back
    ascending, so a shard keeps the callers' system order."""
    costs = np.asarray(costs, dtype=np.float64)
    if nparts < 1:
        raise ValueError("nparts must be >= 1")
    order = sorted(range(costs.size), key=lambda i: (-costs[i], i))
    load = [0.0] * nparts
    parts = [[] for _ in range(nparts)]
    for i in order:
        p = min(range(nparts), key=lambda q: (load[q], q))
        parts[p].append(i)
        load[p] += costs[i]
    return [np.array(sorted(p), dtype=np.int64) for p in parts]


class ShardedBatch:
    """This rank's share of independent systems [(n, Ap, Ai), ...] under one
    batch ``Solver`` (``solver`` is None when the share is empty).

    ``systems[i]`` may carry more than (n, Ap, Ai); only those are used.
    ``local_values`` / ``local_rhs`` concatenate per-system arrays of this
    rank's systems in the solver's order; ``split`` cuts a local solution back
    into per-system pieces; ``gather`` brings every system's piece to one
    rank in the callers' order."""

    def __init__(self, systems, rank, world, ordering=ORDER_AMD, tree=TREE_SUPER, relax_zeros=0,
                 costs=None):
        if not 0 <= rank < world:
            raise ValueError("rank must be in [0, world)")
        self.rank, self.world, self.nsys = rank, world, len(systems)
        trip = [(int(s[0]), s[1], s[2]) for s in systems]
        if costs is None:
            costs, _ = estimate_batch(trip, ordering, tree, relax_zeros)
        self.costs = np.asarray(costs, dtype=np.float64)
        self.parts = lpt_partition(self.costs, world)
        self.mine = self.parts[rank]
        self.sizes = np.array([trip[i][0] for i in self.mine], dtype=np.int64)
        self.row_off = np.concatenate([[0], np.cumsum(self.sizes)]).astype(np.int64)
        self.solver = None
        if self.mine.size:
            self.solver = Solver.batch([trip[i] for i in self.mine], ordering, tree, relax_zeros)
        self.n = int(self.row_off[-1])

    def load(self):
        """Estimated flops of each rank's share."""
        return np.array([self.costs[p].sum() for p in self.parts])

    def local_values(self, values):
        """values[i] = system i's lower-triangle values, for all systems."""
        if not self.mine.size:
            return np.zeros(0)
        return np.concatenate([np.asarray(values[i], dtype=np.float64) for i in self.mine])

    def local_rhs(self, rhs):
        """rhs[i] = system i's right-hand side(s), shape (n_i,) or (n_i, k)."""
        if not self.mine.size:
            return np.zeros(0)
        return np.concatenate([np.asarray(rhs[i], dtype=np.float64) for i in self.mine], axis=0)

    def split(self, x_local):
        """{system index: its rows of x_local} for this rank's systems."""
        x_local = np.asarray(x_local)
        if x_local.shape[0] != self.n:
            raise ValueError("local solution has %d rows, expected %d" % (x_local.shape[0], self.n))
        return {int(i): x_local[self.row_off[k]:self.row_off[k + 1]]
                for k, i in enumerate(self.mine)}

    def gather(self, x_local, dst=0, group=None):
        """Every system's rows of the ranks' local solutions, on rank dst, as
        a list in the callers' system order (None on the other ranks).  With
        world 1 no process group is needed."""
        mine = self.split(x_local)
        if self.world == 1:
            return [mine[i] for i in range(self.nsys)]
        import torch.distributed as dist

        got = [None] * self.world if self.rank == dst else None
        dist.gather_object(mine, got, dst=dst, group=group)
        if self.rank != dst:
            return None
        out = [None] * self.nsys
        for piece in got:
            for i, v in piece.items():
                out[i] = v
        return out
