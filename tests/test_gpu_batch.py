"""GPU tests of batched counting: every graph's count in the batch equals
the oracle's count of that graph alone, and equals the single-graph path."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import complete_graph, comb3, random_pairs, wheel_graph

pytestmark = pytest.mark.gpu


def make_batch(graphs):
    """graphs: list of (src, dst, n) with local ids -> concatenated arrays."""
    src = np.concatenate([g[0] for g in graphs]).astype(np.uint32)
    dst = np.concatenate([g[1] for g in graphs]).astype(np.uint32)
    off = np.zeros(len(graphs) + 1, np.uint64)
    off[1:] = np.cumsum([len(g[0]) for g in graphs])
    n = np.array([g[2] for g in graphs], np.uint64)
    return src, dst, off, n


def mixed_graphs(seed, count=40):
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        kind = i % 4
        if kind == 0:
            n = int(rng.integers(2, 3000))
            s, d = random_pairs(n, int(rng.integers(0, 12 * n)), seed * 1000 + i)
        elif kind == 1:
            k = int(rng.integers(3, 60))
            s, d = complete_graph(k)
            n = k
        elif kind == 2:
            k = int(rng.integers(4, 500))
            s, d = wheel_graph(k)
            n = k + 1
        else:
            n = int(rng.integers(1000, 20000))
            s, d = random_pairs(n, 15 * n, seed * 1000 + i)
        out.append((s, d, n))
    return out


@pytest.mark.parametrize("seed", [1, 2])
@pytest.mark.parametrize("spread,a,graph", [(5, 8192, True), (1, 64, False), (0, 4096, True)])
def test_batch_counts_equal_single_graph(wetric_mod, oracle_mod, seed, spread, a, graph):
    graphs = mixed_graphs(seed)
    src, dst, off, n = make_batch(graphs)
    b = wetric_mod.Batch(src, dst, off, n, spread=spread, a=a, use_cuda_graph=graph)
    counts, st = b.count()
    wedges, edges = b.info()
    for g, (s, d, ng) in enumerate(graphs):
        og = oracle_mod.oriented_from_pairs(s, d, ng)
        assert counts[g] == oracle_mod.count_merge(og), g
        assert wedges[g] == oracle_mod.wedge_total(og), g
        assert edges[g] == og.m, g
    # replays give the same counts
    again, _ = b.count()
    assert np.array_equal(again, counts)
    assert st.wedges == int(wedges.sum())
    b.free()


@pytest.mark.parametrize("use_graph", [True, False])
def test_batch_pair_streams_on_and_off(wetric_mod, oracle_mod, use_graph):
    """Short rows of every graph counted by pair streams (the default) or by
    wedge checks give the same per-graph counts, equal to the oracle's; the
    statistics and per-graph wedges cover both parts."""
    graphs = mixed_graphs(5, count=24)
    rng = np.random.default_rng(5)
    for i in range(6):  # Erdos-Renyi graphs whose rows are all short
        n = int(rng.integers(20_000, 80_000))
        s, d = random_pairs(n, 12 * n, 5000 + i)
        graphs.append((s, d, n))
    src, dst, off, n = make_batch(graphs)
    want = [oracle_mod.count_merge(oracle_mod.oriented_from_pairs(s, d, ng))
            for s, d, ng in graphs]
    W = [oracle_mod.wedge_total(oracle_mod.oriented_from_pairs(s, d, ng))
         for s, d, ng in graphs]
    on = wetric_mod.Batch(src, dst, off, n, use_cuda_graph=use_graph)
    off_ = wetric_mod.Batch(src, dst, off, n, use_cuda_graph=use_graph, pair_streams=False)
    c_on, st_on = on.count()
    c_off, st_off = off_.count()
    assert list(c_on) == want and list(c_off) == want
    assert st_on.pair_rows > 0 and st_on.pair_wedges > 0
    assert st_off.pair_rows == 0
    assert st_on.wedges == st_off.wedges == sum(W)
    assert list(on.info()[0]) == W
    again, _ = on.count()
    assert list(again) == want
    on.free()
    off_.free()


def test_batch_alone_equals_mix(wetric_mod, oracle_mod, torch_mod=None):
    """A graph's count is the same alone and inside a mix, from device pairs."""
    import torch

    graphs = mixed_graphs(7, count=25)
    src, dst, off, n = make_batch(graphs)
    b = wetric_mod.Batch(torch.from_numpy(src.view(np.int32)).cuda(),
                         torch.from_numpy(dst.view(np.int32)).cuda(), off, n, spread=3)
    mix, _ = b.count()
    for g, (s, d, ng) in enumerate(graphs):
        alone = wetric_mod.Batch(s, d, np.array([0, len(s)], np.uint64),
                                 np.array([ng], np.uint64), spread=3)
        c, _ = alone.count()
        assert c[0] == mix[g]
        og = wetric_mod.orient_edges(s, d, n=ng)
        assert og.count(3, 8192)[0] == mix[g]
        og.free()
        alone.free()
    b.free()


def test_batch_errors(wetric_mod):
    s, d = complete_graph(5)
    with pytest.raises(wetric_mod.WetricError):   # id >= n of its graph
        wetric_mod.Batch(s, d, np.array([0, len(s)], np.uint64), np.array([4], np.uint64))
    with pytest.raises(wetric_mod.WetricError):   # n == 0
        wetric_mod.Batch(s, d, np.array([0, len(s)], np.uint64), np.array([0], np.uint64))
    b = wetric_mod.Batch(s, d, np.array([0, len(s)], np.uint64), np.array([5], np.uint64))
    assert b.count()[0][0] == comb3(5)
    b.free()


def test_batch_empty_graphs(wetric_mod):
    s, d = complete_graph(4)
    src = np.concatenate([s, np.zeros(0, np.uint32)])
    off = np.array([0, 0, len(s), len(s)], np.uint64)
    n = np.array([3, 4, 1], np.uint64)
    b = wetric_mod.Batch(src, d, off, n)
    counts, _ = b.count()
    assert counts.tolist() == [0, 4, 0]
    b.free()


def test_batch_autotune(wetric_mod, oracle_mod):
    """The autotuner picks a candidate spread for every bucket with enough
    wedges to time, counts stay exact, and a second batch with graphs of the
    same buckets reuses the device's table (same spreads)."""
    from wetric import workloads as Wl

    graphs = []
    for i, scale in enumerate((12, 13, 13)):
        s, d, n = Wl.host_pairs(Wl.RmatSpec(scale=scale, edge_factor=16, seed=300 + i))
        graphs.append((s, d, n))
    for i in range(6):
        n = 20000
        s, d = random_pairs(n, 40 * n, 400 + i)
        graphs.append((s, d, n))
    src, dst, off, n = make_batch(graphs)
    b = wetric_mod.Batch(src, dst, off, n, spread=0, autotune=True)
    counts, _ = b.count()
    for g, (s, d, ng) in enumerate(graphs):
        assert counts[g] == oracle_mod.count_merge(oracle_mod.oriented_from_pairs(s, d, ng)), g
    sp = b.spreads()
    assert set(sp.tolist()) <= {1, 2, 5, 10, 20}
    b.free()
    b2 = wetric_mod.Batch(src, dst, off, n, spread=0, autotune=True)
    assert np.array_equal(b2.spreads(), sp)
    assert np.array_equal(b2.count()[0], counts)
    b2.free()
    # a fixed spread bypasses the tuner
    b3 = wetric_mod.Batch(src, dst, off, n, spread=3, autotune=True)
    assert set(b3.spreads().tolist()) == {3}
    assert np.array_equal(b3.count()[0], counts)
    b3.free()
