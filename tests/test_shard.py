"""Independent systems across GPUs (mdgpu_b200/shard.py): the cost estimate
against each system's own analysis, the longest-processing-time partition,
and the host-side plumbing of a sharded batch over 2 gloo ranks on the CPU
(every rank derives the same partition with no exchange; the gather brings
every system's rows back in the callers' order, empty shards included).
The numeric calls are the batch solver's own, tested on the GPU elsewhere."""
import os
import socket

import numpy as np
import pytest

import mdgpu_b200 as M
from mdgpu_b200 import matgen as mg
from mdgpu_b200.shard import ShardedBatch, lpt_partition


def _systems(count, seed=0):
    rng = np.random.default_rng(seed)
    out = []
    for q in range(count):
        if q % 2 == 0:
            dims = (int(rng.integers(6, 20)),) * 2
        else:
            dims = (int(rng.integers(4, 9)),) * 3
        out.append(mg.laplacian_grid(dims, seed=q, sigma=0.5, shift=1e-2))
    return out


def test_estimate_matches_each_systems_analysis():
    syss = _systems(9)
    flops, lnz = M.estimate_batch([s[:3] for s in syss])
    for i, (n, Ap, Ai, _) in enumerate(syss):
        S = M.Solver(n, Ap, Ai)
        assert flops[i] == S.info("flops") and lnz[i] == S.info("lnz")
    # relaxed trees change the counts; the estimate follows the tree kind
    f2, _ = M.estimate_batch([s[:3] for s in syss], tree=M.TREE_RELAXED, relax_zeros=8)
    S = M.Solver(*syss[3][:3], tree=M.TREE_RELAXED, relax_zeros=8)
    assert f2[3] == S.info("flops")


def test_estimate_rejects_bad_input():
    n, Ap, Ai, _ = mg.laplacian_2d_5pt(4)
    bad_Ap = Ap.copy()
    bad_Ap[2] = bad_Ap[1] - 1  # decreasing column pointers
    with pytest.raises(M.MdgpuError) as e:
        M.estimate_batch([(n, Ap, Ai), (n, bad_Ap, Ai)])
    assert e.value.status == -1 and "system 1" in str(e.value)
    bad_Ai = Ai.copy()
    bad_Ai[Ap[1]] = 0  # column 1 holding row 0: above the diagonal
    with pytest.raises(M.MdgpuError) as e:
        M.estimate_batch([(n, Ap, bad_Ai)])
    assert e.value.status == -1


def test_lpt_partition():
    costs = [7, 5, 4, 4, 3, 3, 3, 1]
    parts = lpt_partition(costs, 3)
    # largest first, each to the least-loaded part (ties: lower part)
    assert [p.tolist() for p in parts] == [[0, 5], [1, 4, 6], [2, 3, 7]]  # loads 10, 11, 9
    rng = np.random.default_rng(1)
    for m in (1, 2, 3, 5, 8):
        c = rng.lognormal(0, 2, 200)
        parts = lpt_partition(c, m)
        allidx = np.sort(np.concatenate(parts))
        assert np.array_equal(allidx, np.arange(200))
        loads = [c[p].sum() for p in parts]
        assert max(loads) <= 4 / 3 * max(c.sum() / m, c.max()) + 1e-9
        assert all(np.all(np.diff(p) > 0) for p in parts)
    # more parts than items: the extra parts are empty
    parts = lpt_partition([2.0, 1.0], 4)
    assert [p.tolist() for p in parts] == [[0], [1], [], []]


def test_one_rank_holds_everything():
    syss = _systems(5, seed=2)
    B = ShardedBatch(syss, 0, 1)
    assert B.mine.tolist() == list(range(5))
    S = M.Solver.batch([s[:3] for s in syss])
    assert B.n == S.n and np.array_equal(B.row_off, S.row_off)
    assert np.array_equal(B.solver.array("perm"), S.array("perm"))
    x = np.arange(B.n, dtype=np.float64)
    got = B.gather(x)
    for i, (n, *_rest) in enumerate(syss):
        assert np.array_equal(got[i], x[S.row_off[i]:S.row_off[i + 1]])


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port):
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        syss = _systems(11, seed=3)
        B = ShardedBatch(syss, rank, world)
        # the same partition on every rank, derived without an exchange
        every = [None] * world
        dist.all_gather_object(every, [p.tolist() for p in B.parts])
        assert all(e == every[0] for e in every)
        # this rank's solver covers exactly its systems, in order
        assert B.solver is not None
        assert B.solver.n == sum(syss[i][0] for i in B.mine)
        vals = B.local_values([s[3] for s in syss])
        assert vals.size == sum(syss[i][1][-1] for i in B.mine)
        rhs = B.local_rhs([np.full((s[0], 2), i, dtype=np.float64) for i, s in enumerate(syss)])
        assert rhs.shape == (B.n, 2)
        # a stand-in solution: system i's rows hold 1000 i + row
        x = np.concatenate([1000.0 * i + np.arange(syss[i][0]) for i in B.mine])
        got = B.gather(x, dst=0)
        if rank == 0:
            for i, s in enumerate(syss):
                assert np.array_equal(got[i], 1000.0 * i + np.arange(s[0])), i
        else:
            assert got is None
        # one system, two ranks: rank 1 holds nothing and still takes part
        one = ShardedBatch(syss[:1], rank, world)
        assert (one.solver is None) == (rank == 1)
        x1 = np.arange(one.n, dtype=np.float64)
        got1 = one.gather(x1, dst=1)
        if rank == 1:
            assert len(got1) == 1 and np.array_equal(got1[0], np.arange(syss[0][0]))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_partition_and_gather():
    mp = pytest.importorskip("torch.multiprocessing")
    mp.spawn(_worker, args=(2, _free_port()), nprocs=2, join=True)
