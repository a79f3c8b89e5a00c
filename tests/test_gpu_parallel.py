"""World-size-2 runs of the sharded count where each rank counts its wedge
range through the library's CUDA path (wetric.count with wedge_begin /
wedge_end, and wetric.Batch for whole-graph sharding); the ranks exchange
only the counts, over gloo. Both ranks share the one visible GPU: their
kernels are independent (no rank waits on another's kernel), the exchange
is on the host."""
from __future__ import annotations

import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from conftest import ORACLE, PKG, random_pairs

pytestmark = pytest.mark.gpu


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import sys

    sys.path.insert(0, PKG)
    sys.path.insert(0, ORACLE)
    import datetime

    import torch
    import torch.distributed as dist

    import oracle
    import wetric
    from wetric.parallel import distributed_batch_counts, distributed_count, host_wedge_total

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=120))
    try:
        torch.cuda.set_device(0)
        src, dst = wetric.gen_rmat(16, 16 << 16, seed=41)
        g = oracle.oriented_from_pairs(src, dst)
        W = host_wedge_total(g.row_ptr)
        out[f"count{rank}"] = distributed_count(
            lambda b, e: wetric.count(g.row_ptr, g.col_ind, 5, 8192, wedge_begin=b,
                                      wedge_end=e)[0], W)
        graphs = [random_pairs(300 + 97 * i, 3000 + 900 * i, 500 + i) for i in range(10)]
        weights = [host_wedge_total(oracle.oriented_from_pairs(s, d).row_ptr) for s, d in graphs]

        def count_graphs(idx):
            # a batch of this rank's graphs, each with its own (local) ids
            s_ = np.concatenate([graphs[i][0] for i in idx]).astype(np.uint32)
            d_ = np.concatenate([graphs[i][1] for i in idx]).astype(np.uint32)
            off = np.zeros(len(idx) + 1, np.uint64)
            off[1:] = np.cumsum([len(graphs[i][0]) for i in idx])
            nn = np.array([300 + 97 * i for i in idx], np.uint32)
            b = wetric.Batch(s_, d_, off, nn, spread=5, a=64)
            c, _ = b.count()
            b.free()
            return [int(x) for x in c]

        out[f"batch{rank}"] = distributed_batch_counts(count_graphs, weights)
    finally:
        dist.destroy_process_group()


def test_sharded_counts_through_the_library_world2(oracle_mod):
    ctx = mp.get_context("spawn")
    manager = ctx.Manager()
    out = manager.dict()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=300)
    for p in procs:
        if p.exitcode is None:
            p.kill()
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    import wetric

    src, dst = wetric.gen_rmat(16, 16 << 16, seed=41)
    want = oracle_mod.count_merge(oracle_mod.oriented_from_pairs(src, dst))
    assert out["count0"] == out["count1"] == want
    graphs = [random_pairs(300 + 97 * i, 3000 + 900 * i, 500 + i) for i in range(10)]
    want_b = [oracle_mod.count_merge(oracle_mod.oriented_from_pairs(s, d, 300 + 97 * i))
              for i, (s, d) in enumerate(graphs)]
    assert out["batch0"] == out["batch1"] == want_b
