"""World-size-2 gloo tests of the wedge-range sharding (CPU only). Each
rank counts its range with the oracle's wedge-check count (the checker) and
the ranks' partial counts are summed by the same all-reduce the GPU path
uses."""
from __future__ import annotations

import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from conftest import ORACLE, PKG, random_pairs


def test_shard_ranges_cover_exactly():
    from wetric.parallel import shard_range

    for W in (0, 1, 2, 7, 10**12 + 3):
        for world in (1, 2, 3, 8):
            cuts = [shard_range(W, r, world) for r in range(world)]
            assert cuts[0][0] == 0 and cuts[-1][1] == W
            assert all(a[1] == b[0] for a, b in zip(cuts, cuts[1:]))
            sizes = [e - b for b, e in cuts]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        shard_range(10, 2, 2)


def test_cost_balanced_cuts():
    """Cuts rise from 0 to W, give every rank the same estimated time (the
    core's wedges cheaper than the rest), and fall back to equal shares
    when both parts cost the same per wedge."""
    from wetric.parallel import cost_balanced_cuts

    W, Wc = 7_209_050_446, 4_576_079_111
    main_ms, core_ms = 8.86, 2.34
    for world in (1, 2, 4, 8):
        cuts = cost_balanced_cuts(W, Wc, main_ms, core_ms, world)
        assert len(cuts) == world + 1 and cuts[0] == 0 and cuts[-1] == W
        assert all(a <= b for a, b in zip(cuts, cuts[1:]))
        Wm = W - Wc

        def cost(x):
            return min(x, Wm) * main_ms / Wm + max(0, x - Wm) * core_ms / Wc

        shares = [cost(b) - cost(a) for a, b in zip(cuts, cuts[1:])]
        assert max(shares) - min(shares) < 1e-6 * (main_ms + core_ms)
    # ranks below the core's start get fewer wedges than those above it
    cuts = cost_balanced_cuts(W, Wc, main_ms, core_ms, 4)
    assert cuts[1] - cuts[0] < cuts[4] - cuts[3]
    # equal cost per wedge: equal shares (within rounding)
    cuts = cost_balanced_cuts(1000, 400, 6.0, 4.0, 4)
    assert cuts == [0, 250, 500, 750, 1000]
    assert cost_balanced_cuts(0, 0, 1.0, 0.0, 3) == [0, 0, 0, 0]
    with pytest.raises(ValueError):
        cost_balanced_cuts(10, 0, 1.0, 0.0, 0)


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, seed, out):
    import sys

    sys.path.insert(0, PKG)
    sys.path.insert(0, ORACLE)
    import datetime

    import torch.distributed as dist

    import oracle
    from wetric.parallel import distributed_count, host_wedge_total

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        src, dst = random_pairs(3000, 60000, seed)
        g = oracle.oriented_from_pairs(src, dst)
        W = host_wedge_total(g.row_ptr)
        assert W == oracle.wedge_total(g)
        total = distributed_count(lambda b, e: oracle.count_wedges(g, 64, b, e), W)
        # the same with uneven, cost-balanced boundaries
        from wetric.parallel import cost_balanced_cuts

        cuts = cost_balanced_cuts(W, W // 3, 3.0, 0.5, world)
        again = distributed_count(lambda b, e: oracle.count_wedges(g, 64, b, e), W, cuts=cuts)
        assert again == total
        out[rank] = total
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("seed", [1, 2])
def test_distributed_count_gloo_world2(seed):
    import oracle

    ctx = mp.get_context("spawn")
    manager = ctx.Manager()
    out = manager.dict()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, seed, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    src, dst = random_pairs(3000, 60000, seed)
    want = oracle.count_merge(oracle.oriented_from_pairs(src, dst))
    assert out[0] == out[1] == want


def _bcast_worker(rank, world, port, seed, out):
    import sys

    sys.path.insert(0, PKG)
    sys.path.insert(0, ORACLE)
    import datetime

    import torch.distributed as dist

    import oracle
    from wetric.parallel import broadcast_csr, distributed_count, host_wedge_total

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        rp = ci = None
        if rank == 0:
            src, dst = random_pairs(2500, 50000, seed)
            g = oracle.oriented_from_pairs(src, dst)
            rp, ci = g.row_ptr, g.col_ind
        rp_t, ci_t = broadcast_csr(rp, ci, src=0)
        rp_np = rp_t.numpy().astype(np.uint64)
        ci_np = ci_t.numpy().view(np.uint32)
        W = host_wedge_total(rp_np)
        # every rank checks its replica against a local rebuild, then counts
        src, dst = random_pairs(2500, 50000, seed)
        ref = oracle.oriented_from_pairs(src, dst)
        assert np.array_equal(rp_np, np.asarray(ref.row_ptr, dtype=np.uint64))
        assert np.array_equal(ci_np, np.asarray(ref.col_ind, dtype=np.uint32))
        out[rank] = distributed_count(lambda b, e: oracle.count_wedges(ref, 64, b, e), W)
    finally:
        dist.destroy_process_group()


def test_broadcast_csr_gloo_world2():
    """Rank 0's oriented CSR reaches rank 1 bit for bit (header + two
    broadcasts), and the sharded count over the replicas is exact."""
    import oracle

    ctx = mp.get_context("spawn")
    manager = ctx.Manager()
    out = manager.dict()
    port = _free_port()
    procs = [ctx.Process(target=_bcast_worker, args=(r, 2, port, 5, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    src, dst = random_pairs(2500, 50000, 5)
    want = oracle.count_merge(oracle.oriented_from_pairs(src, dst))
    assert out[0] == out[1] == want


def test_shard_graphs_balance_and_cover():
    """Whole-graph sharding: every graph on exactly one rank, the same
    assignment on every call, and the heaviest graph never shares a rank
    with more work than the lightest rank plus that graph."""
    from wetric.parallel import shard_graphs

    rng = np.random.default_rng(3)
    for world in (1, 2, 3, 8):
        for G in (0, 1, 5, 100):
            w = rng.integers(0, 10**9, size=G).tolist()
            parts = shard_graphs(w, world)
            assert parts == shard_graphs(w, world)
            flat = sorted(i for p in parts for i in p)
            assert flat == list(range(G))
            if G:
                loads = [sum(w[i] for i in p) for p in parts]
                assert max(loads) - min(loads) <= max(w)
    with pytest.raises(ValueError):
        shard_graphs([1, 2], 0)


def _batch_worker(rank, world, port, out):
    import sys

    sys.path.insert(0, PKG)
    sys.path.insert(0, ORACLE)
    import datetime

    import torch.distributed as dist

    import oracle
    from wetric.parallel import distributed_batch_counts, host_wedge_total, shard_graphs

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        graphs = [oracle.oriented_from_pairs(*random_pairs(40 + 37 * i, 300 + 211 * i, 60 + i))
                  for i in range(9)]
        weights = [host_wedge_total(g.row_ptr) for g in graphs]
        seen = []

        def count_graphs(idx):
            seen.extend(idx)
            return [oracle.count_wedges(graphs[i], 64) for i in idx]

        out[rank] = (distributed_batch_counts(count_graphs, weights), sorted(seen),
                     shard_graphs(weights, world)[rank])
    finally:
        dist.destroy_process_group()


def test_distributed_batch_counts_gloo_world2():
    """Each rank counts only its graphs (the checker's count), and one
    all-reduce of the count vector gives both ranks every graph's count."""
    import oracle

    ctx = mp.get_context("spawn")
    manager = ctx.Manager()
    out = manager.dict()
    port = _free_port()
    procs = [ctx.Process(target=_batch_worker, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    want = [oracle.count_merge(oracle.oriented_from_pairs(*random_pairs(40 + 37 * i, 300 + 211 * i, 60 + i)))
            for i in range(9)]
    (c0, s0, p0), (c1, s1, p1) = out[0], out[1]
    assert c0 == c1 == want
    assert s0 == p0 and s1 == p1 and sorted(s0 + s1) == list(range(9))


def _failing_worker(rank, world, port, mode, out):
    import sys

    sys.path.insert(0, PKG)
    sys.path.insert(0, ORACLE)
    import datetime

    import torch.distributed as dist

    import oracle
    from wetric.parallel import RankFailed, distributed_batch_counts, distributed_count

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=30))
    try:
        graphs = [oracle.oriented_from_pairs(*random_pairs(50 + 20 * i, 400 + 90 * i, 90 + i))
                  for i in range(6)]
        weights = [1 + i for i in range(6)]

        if mode == "batch_wrong_length":
            def count_graphs(idx):
                c = [oracle.count_wedges(graphs[i], 64) for i in idx]
                return c[:-1] if rank == 1 else c
            fn = lambda: distributed_batch_counts(count_graphs, weights)
        elif mode == "batch_raises":
            def count_graphs(idx):
                if rank == 0:
                    raise MemoryError("planted on the host")
                return [oracle.count_wedges(graphs[i], 64) for i in idx]
            fn = lambda: distributed_batch_counts(count_graphs, weights)
        else:  # range_raises
            def count_range(b, e):
                if rank == 1:
                    raise RuntimeError("planted on the host")
                return oracle.count_wedges(graphs[0], 64, b, e)
            fn = lambda: distributed_count(count_range, 10**6)
        try:
            fn()
            out[rank] = ("returned", None)
        except RankFailed as ex:
            out[rank] = ("raised", ex.failed_ranks)
        # the group is still usable: one more collective in step on both ranks
        from wetric.parallel import reduce_count
        out[f"after{rank}"] = reduce_count(rank + 1)
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("mode,bad", [("batch_wrong_length", [1]), ("batch_raises", [0]),
                                      ("range_raises", [1])])
def test_one_rank_failing_raises_on_every_rank(mode, bad):
    """A rank whose local count fails (wrong number of counts, or an
    exception) still reaches the all-reduce; both ranks then raise
    RankFailed naming it, neither waits in the collective, and the group
    stays usable for the next collective."""
    ctx = mp.get_context("spawn")
    manager = ctx.Manager()
    out = manager.dict()
    port = _free_port()
    procs = [ctx.Process(target=_failing_worker, args=(r, 2, port, mode, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    for p in procs:
        if p.exitcode is None:
            p.kill()
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    assert out[0] == ("raised", bad) and out[1] == ("raised", bad)
    assert out["after0"] == out["after1"] == 3
