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


@pytest.fixture(scope="module")
def torch_mod_serve():
    import torch

    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    return torch


def _graphs(seed, count):
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        n = int(rng.integers(3, 5000))
        s, d = random_pairs(n, int(rng.integers(0, 20 * n)), seed * 100 + i)
        out.append((s, d, n))
    return out


@pytest.mark.parametrize("resident", [True, False])
def test_server_counts_match_alone(wetric_mod, oracle_mod, resident):
    graphs = _graphs(3, 60)
    want = [oracle_mod.count_merge(oracle_mod.oriented_from_pairs(s, d, n)) for s, d, n in graphs]
    srv = wetric_mod.Server(max_batch_graphs=16, resident=resident)
    tickets = [srv.submit(s, d, n) for s, d, n in graphs]
    got = [srv.wait(t)[0] for t in tickets]
    assert got == want
    st = srv.stats()
    assert st["completed"] == len(graphs) and st["failed"] == 0
    # the same graphs one at a time
    for (s, d, n), w in zip(graphs[:10], want[:10]):
        assert srv.wait(srv.submit(s, d, n))[0] == w
    srv.close()


@pytest.mark.parametrize("resident", [False, True])
@pytest.mark.parametrize("large_pairs", [0, 20000])
def test_server_size_lanes(wetric_mod, oracle_mod, large_pairs, resident):
    """With a large-request threshold, graphs above it run in their own lane
    (own worker thread and stream); with 0 there is one lane. Every count
    matches the graph alone either way."""
    graphs = _graphs(11, 40)
    want = [oracle_mod.count_merge(oracle_mod.oriented_from_pairs(s, d, n)) for s, d, n in graphs]
    big = sum(1 for s, _, _ in graphs if len(s) >= 20000)
    assert 0 < big < len(graphs)
    srv = wetric_mod.Server(max_batch_graphs=12, large_pairs=large_pairs, resident=resident)
    tickets = [srv.submit(s, d, n) for s, d, n in graphs]
    assert [srv.wait(t)[0] for t in tickets] == want
    st = srv.stats()
    assert st["completed"] == len(graphs) and st["failed"] == 0
    srv.close()


@pytest.mark.parametrize("resident", [False, True])
def test_server_concurrent_submitters_and_device_inputs(wetric_mod, oracle_mod, resident):
    import torch

    graphs = _graphs(5, 48)
    want = [oracle_mod.count_merge(oracle_mod.oriented_from_pairs(s, d, n)) for s, d, n in graphs]
    srv = wetric_mod.Server(max_batch_graphs=8, resident=resident)
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
    srv = wetric_mod.Server(hbm_budget=4 << 20, max_batch_graphs=64, resident=False)
    tickets = [srv.submit(s, d, 40) for _ in range(20)]
    assert [srv.wait(t)[0] for t in tickets] == [comb3(40)] * 20
    st = srv.stats()
    assert st["batches"] >= 2 and st["admitted_bytes"] == 0
    srv.close()
    # resident: the budget is returned once the kernel has idled out and the
    # completed requests' memory is freed
    srv = wetric_mod.Server(hbm_budget=4 << 20, resident=True)
    tickets = [srv.submit(s, d, 40) for _ in range(20)]
    assert [srv.wait(t)[0] for t in tickets] == [comb3(40)] * 20
    for _ in range(200):
        if srv.stats()["admitted_bytes"] == 0:
            break
        time.sleep(0.01)
    assert srv.stats()["admitted_bytes"] == 0
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


def test_server_wait_runs_out_then_completes(wetric_mod, oracle_mod):
    """A 1 ms wait on a request queued behind a long one in the same lane
    returns ETIMEDOUT (the ticket stays valid); a later wait gets the exact
    count. The long request is an R-MAT scale-20 graph (tens of ms of
    preprocessing and counting)."""
    from wetric import workloads as Wl

    src, dst, n = Wl.host_pairs(Wl.RmatSpec(scale=20, edge_factor=16, seed=31))
    s_small, d_small = complete_graph(30)
    srv = wetric_mod.Server(large_pairs=0)  # one lane: the small one queues
    t_big = srv.submit(src, dst, n)
    t_small = srv.submit(s_small, d_small, 30)
    with pytest.raises(wetric_mod.WetricError) as e:
        srv.wait(t_small, timeout_ms=1)
    assert e.value.status == wetric_mod.ETIMEDOUT
    assert srv.wait(t_small, timeout_ms=120000)[0] == comb3(30)
    want = oracle_mod.count_merge(oracle_mod.oriented_from_pairs(src, dst, n))
    assert srv.wait(t_big, timeout_ms=120000)[0] == want
    srv.close()


def test_resident_folds_arrivals_into_the_running_kernel(wetric_mod, oracle_mod):
    """Small requests submitted while a large one is being counted by the
    resident kernel are folded into that kernel's queue: they complete
    while the large request is still pending, with no launch of their own,
    and every count equals the graph's count alone."""
    from wetric import workloads as Wl

    big_s, big_d, big_n = Wl.host_pairs(Wl.RmatSpec(scale=23, edge_factor=16, seed=77))
    og = wetric_mod.orient_edges(big_s, big_d, n=big_n)
    want_big = og.count(5, 8192)[0]  # the large graph counted alone
    og.free()
    small = _graphs(17, 6)
    want_small = [oracle_mod.count_merge(oracle_mod.oriented_from_pairs(s, d, n))
                  for s, d, n in small]
    srv = wetric_mod.Server(item_tiles=2048, resident=True)
    t_big = srv.submit(big_s, big_d, big_n)
    # wait until the large request's tiles are on the resident kernel
    for _ in range(30000):
        if srv.stats()["resident_launches"] >= 1:
            break
        time.sleep(0.001)
    launches0 = srv.stats()["resident_launches"]
    assert launches0 >= 1
    t_small = [srv.submit(s, d, n) for s, d, n in small]
    got_small = [srv.wait(t, timeout_ms=120000)[0] for t in t_small]
    big_now = srv.poll(t_big)  # None while the large request is pending
    folded_launches = srv.stats()["resident_launches"]
    got_big = big_now[0] if big_now is not None else srv.wait(t_big, timeout_ms=120000)[0]
    assert got_small == want_small
    assert got_big == want_big
    assert big_now is None, "the large request finished before the small ones"
    # the small requests share the kernel's queue with the large one: no
    # launch of their own (a relaunch after a brief idle gap of the queue
    # may add one, never one per request)
    assert folded_launches - launches0 <= 1 < len(small), (launches0, folded_launches)
    st = srv.stats()
    assert st["completed"] == len(small) + 1 and st["failed"] == 0
    srv.close()


def test_resident_kernel_gives_up_waiting_and_relaunches(wetric_mod, oracle_mod):
    """With nothing left in its queue the resident kernel's bounded wait runs
    out: it ends by itself with status 2 (gave up waiting), no fault and no
    hang, and the next request relaunches it."""
    srv = wetric_mod.Server(resident=True)
    s, d = complete_graph(50)
    assert srv.wait(srv.submit(s, d, 50))[0] == comb3(50)
    st = None
    for _ in range(500):
        st = srv.stats()
        if st["resident_last_exit"] == 2:
            break
        time.sleep(0.002)
    assert st["resident_last_exit"] == 2, st
    first = st["resident_launches"]
    assert first >= 1
    g = oracle_mod.oriented_from_pairs(*random_pairs(3000, 40000, 5), 3000)
    s2, d2 = random_pairs(3000, 40000, 5)
    assert srv.wait(srv.submit(s2, d2, 3000))[0] == oracle_mod.count_merge(g)
    assert srv.stats()["resident_launches"] > first
    srv.close()


def test_resident_stream_of_arrivals_all_complete(wetric_mod, oracle_mod):
    """A stream of arrivals like the serving workload, at test size: 300
    small graphs submitted one every 0.2 ms while two R-MAT scale-18 graphs
    are fed to the resident kernel in many small queue items. Hundreds of
    items pass the queue head in quick succession; every request completes
    (a wait that runs out fails the test instead of hanging it) with the
    graph's count alone."""
    from wetric import workloads as Wl

    big = [Wl.host_pairs(Wl.RmatSpec(scale=18, edge_factor=16, seed=s)) for s in (41, 42)]
    want_big = []
    for s, d, n in big:
        og = wetric_mod.orient_edges(s, d, n=n)
        want_big.append(og.count(5, 8192)[0])
        og.free()
    small = _graphs(23, 300)
    want_small = [oracle_mod.count_merge(oracle_mod.oriented_from_pairs(s, d, n))
                  for s, d, n in small]
    srv = wetric_mod.Server(item_tiles=8, large_pairs=1 << 20, resident=True)
    tickets = []
    for i, (s, d, n) in enumerate(small):
        if i in (10, 150):
            bs, bd, bn = big[0 if i == 10 else 1]
            tickets.append(("big", 0 if i == 10 else 1, srv.submit(bs, bd, bn)))
        tickets.append(("small", i, srv.submit(s, d, n)))
        time.sleep(0.0002)
    for kind, i, t in tickets:
        c = srv.wait(t, timeout_ms=60000)[0]
        assert c == (want_big[i] if kind == "big" else want_small[i]), (kind, i)
    st = srv.stats()
    assert st["completed"] == len(tickets) and st["failed"] == 0
    assert st["resident_launches"] >= 1
    srv.close()


def test_resident_device_inputs_default_items(wetric_mod, torch_mod_serve):
    """The serving workload's shape at test size: device inputs, the
    default item size, R-MAT scale-21 requests (dense core, fed in items) in
    the large lane between small Erdos-Renyi and Chung-Lu requests. Every
    request completes with the graph's count alone; a wait that runs out
    reports the server's queue state."""
    from wetric import workloads as Wl

    torch = torch_mod_serve
    specs = [Wl.ErdosRenyiSpec(n=50_000, draws=600_000, seed=61),
             Wl.chung_lu_for(60_000, 20.0, 2.5, 62),
             Wl.RmatSpec(scale=21, edge_factor=16, seed=63),
             Wl.ErdosRenyiSpec(n=5_000, draws=60_000, seed=64),
             Wl.RmatSpec(scale=20, edge_factor=16, seed=65),
             Wl.chung_lu_for(200_000, 30.0, 2.3, 66)]
    pool = []
    for sp in specs:
        s_, d_, n_ = Wl.device_pairs(sp, 0)
        og = wetric_mod.orient_edges(s_, d_, n=n_)
        pool.append((s_, d_, n_, og.count(5, 8192)[0]))
        og.free()
    torch.cuda.synchronize()
    srv = wetric_mod.Server(large_pairs=8 << 20, resident=True)
    order = [0, 1, 3, 2, 0, 3, 1, 4, 5, 3, 2, 0, 1, 3, 5, 4, 0, 3]
    tickets = []
    for i in order:
        s_, d_, n_, _ = pool[i]
        tickets.append((i, srv.submit(s_, d_, n_)))
        time.sleep(0.003)
    for i, t in tickets:
        try:
            c = srv.wait(t, timeout_ms=60000)[0]
        except wetric_mod.WetricError as e:
            raise AssertionError(f"request {i} (ticket {t}) did not complete: "
                                 f"{srv.stats()}") from e
        assert c == pool[i][3], i
    st = srv.stats()
    assert st["completed"] == len(order) and st["failed"] == 0
    srv.close()


@pytest.mark.parametrize("resident", [False, True])
def test_server_submit_csr(wetric_mod, oracle_mod, torch_mod_serve, resident):
    """A graph submitted as a CSR -- oriented or symmetric, host or device,
    u64 or u32 offsets -- counts the same as the graph alone; the caller's
    arrays can be dropped right after the call."""
    torch = torch_mod_serve
    graphs = _graphs(31, 6)
    want = [oracle_mod.count_merge(oracle_mod.oriented_from_pairs(s, d, n)) for s, d, n in graphs]
    srv = wetric_mod.Server(resident=resident)
    tickets = []
    for i, (s, d, n) in enumerate(graphs):
        if i % 3 == 0:
            g = oracle_mod.oriented_from_pairs(s, d, n)
            rp, ci, oriented = g.row_ptr, g.col_ind, True
        elif i % 3 == 1:
            g = oracle_mod.csr_from_pairs(s, d, n)
            rp, ci, oriented = g.row_ptr.astype(np.uint32), g.col_ind, False
        else:
            g = oracle_mod.oriented_from_pairs(s, d, n)
            rp = torch.from_numpy(g.row_ptr.astype(np.int64)).cuda()
            ci = torch.from_numpy(g.col_ind.astype(np.int32)).cuda()
            oriented = True
        tickets.append(srv.submit_csr(rp, ci, oriented=oriented))
        del rp, ci, g
    assert [srv.wait(t, timeout_ms=60000)[0] for t in tickets] == want
    srv.close()
