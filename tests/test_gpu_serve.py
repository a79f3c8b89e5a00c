"""GPU tests of the counting service: every request's count is the same as
the graph's count alone (exact), whether it arrives alone or in a mix that
overlaps on the device; admission keeps the memory under the budget."""
from __future__ import annotations

import threading
import time

import numpy as np
import pytest

from conftest import comb3, complete_graph, random_pairs

pytestmark = pytest.mark.gpu


def _graphs(seed, count):
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        n = int(rng.integers(3, 5000))
        s, d = random_pairs(n, int(rng.integers(0, 20 * n)), seed * 100 + i)
        out.append((s, d, n))
    return out


def test_server_counts_match_alone(wetric_mod, oracle_mod):
    graphs = _graphs(3, 60)
    want = [oracle_mod.count_merge(oracle_mod.oriented_from_pairs(s, d, n)) for s, d, n in graphs]
    srv = wetric_mod.Server(max_batch_graphs=16)
    tickets = [srv.submit(s, d, n) for s, d, n in graphs]
    got = [srv.wait(t)[0] for t in tickets]
    assert got == want
    st = srv.stats()
    assert st["completed"] == len(graphs) and st["failed"] == 0
    # the same graphs one at a time
    for (s, d, n), w in zip(graphs[:10], want[:10]):
        assert srv.wait(srv.submit(s, d, n))[0] == w
    srv.close()


@pytest.mark.parametrize("large_pairs", [0, 20000])
def test_server_size_lanes(wetric_mod, oracle_mod, large_pairs):
    """With a large-request threshold, graphs above it run in their own lane
    (own worker thread and stream); with 0 there is one lane. Every count
    matches the graph alone either way."""
    graphs = _graphs(11, 40)
    want = [oracle_mod.count_merge(oracle_mod.oriented_from_pairs(s, d, n)) for s, d, n in graphs]
    big = sum(1 for s, _, _ in graphs if len(s) >= 20000)
    assert 0 < big < len(graphs)
    srv = wetric_mod.Server(max_batch_graphs=12, large_pairs=large_pairs)
    tickets = [srv.submit(s, d, n) for s, d, n in graphs]
    assert [srv.wait(t)[0] for t in tickets] == want
    st = srv.stats()
    assert st["completed"] == len(graphs) and st["failed"] == 0
    srv.close()


def test_server_concurrent_submitters_and_device_inputs(wetric_mod, oracle_mod):
    import torch

    graphs = _graphs(5, 48)
    want = [oracle_mod.count_merge(oracle_mod.oriented_from_pairs(s, d, n)) for s, d, n in graphs]
    srv = wetric_mod.Server(max_batch_graphs=8)
    got = [None] * len(graphs)

    def client(idx):
        for i in idx:
            s, d, n = graphs[i]
            if i % 2:
                s = torch.from_numpy(s.view(np.int32)).cuda()
                d = torch.from_numpy(d.view(np.int32)).cuda()
                torch.cuda.synchronize()
            t = srv.submit(s, d, n)
            time.sleep(0.001)
            got[i] = srv.wait(t)[0]

    threads = [threading.Thread(target=client, args=(range(k, len(graphs), 4),))
               for k in range(4)]
    for th in threads:
        th.start()
    for th in threads:
        th.join(timeout=120)
    assert got == want
    srv.close()


def test_server_budget_admission(wetric_mod):
    """A budget that fits about one request at a time still completes every
    request exactly (admission waits for memory to free up)."""
    s, d = complete_graph(40)
    srv = wetric_mod.Server(hbm_budget=4 << 20, max_batch_graphs=64)
    tickets = [srv.submit(s, d, 40) for _ in range(20)]
    assert [srv.wait(t)[0] for t in tickets] == [comb3(40)] * 20
    st = srv.stats()
    assert st["batches"] >= 2 and st["admitted_bytes"] == 0
    srv.close()


def test_server_errors(wetric_mod):
    srv = wetric_mod.Server()
    s, d = complete_graph(5)
    with pytest.raises(wetric_mod.WetricError):
        srv.submit(s, d, 0)
    t = srv.submit(s, d, 4)          # id 4 >= n: the request fails, not the server
    with pytest.raises(wetric_mod.WetricError):
        srv.wait(t)
    assert srv.wait(srv.submit(s, d, 5))[0] == comb3(5)
    with pytest.raises(wetric_mod.WetricError):
        srv.poll(123456789)
    # a bad request batched with good ones fails alone
    srv2 = wetric_mod.Server(max_batch_graphs=64)
    good = [srv2.submit(s, d, 5) for _ in range(5)]
    bad = srv2.submit(s, d, 3)
    good += [srv2.submit(s, d, 5) for _ in range(5)]
    assert [srv2.wait(t)[0] for t in good] == [comb3(5)] * 10
    with pytest.raises(wetric_mod.WetricError):
        srv2.wait(bad)
    srv2.close()
    srv.close()
