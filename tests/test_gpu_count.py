"""GPU parity tests: every count, CSR and statistic from libwetric's CUDA
path is compared bit-exactly with the oracle (and, where recorded, with the
reference's own binaries) on the same seeded inputs."""
from __future__ import annotations

import json
import os
import subprocess

import numpy as np
import pytest

from conftest import (GOLDEN, PKG, bipartite_graph, comb3, complete_graph,
                      random_pairs, star_graph, wheel_graph)

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch_mod():
    import torch

    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    return torch


def host_oriented(oracle_mod, src, dst, n=0):
    g = oracle_mod.oriented_from_pairs(src, dst, n)
    return g.row_ptr, g.col_ind, g


# ------------------------------------------------------------ closed forms


@pytest.mark.parametrize("k", [3, 4, 5, 8, 17, 33, 64, 100])
def test_complete_graphs(wetric_mod, oracle_mod, k):
    rp, ci, _ = host_oriented(oracle_mod, *complete_graph(k))
    for s, a in ((1, 0), (5, 8192), (3, 32), (7, 64)):
        got, st = wetric_mod.count(rp, ci, s, a)
        assert got == comb3(k), (k, s, a)
        assert st.wedges == comb3(k)  # sum of C(d+, 2) over K_k


def test_rows_longer_than_the_stage(wetric_mod, oracle_mod):
    """K_1500: out-degrees up to 1499 exceed the shared-memory stage, so the
    warp-staged kernel mixes staged and global searches."""
    rp, ci, _ = host_oriented(oracle_mod, *complete_graph(1500))
    for kernel in KERNELS:
        for s, a in ((1, 0), (5, 0), (7, 512)):
            assert wetric_mod.count(rp, ci, s, a, kernel=kernel)[0] == comb3(1500)


def test_zero_triangle_families(wetric_mod, oracle_mod):
    for src, dst in (star_graph(300), bipartite_graph(20, 31)):
        rp, ci, _ = host_oriented(oracle_mod, src, dst)
        for s, a in ((1, 0), (5, 64), (16, 8192)):
            assert wetric_mod.count(rp, ci, s, a)[0] == 0


@pytest.mark.parametrize("k", [4, 5, 9, 100, 1000])
def test_wheels(wetric_mod, oracle_mod, k):
    rp, ci, _ = host_oriented(oracle_mod, *wheel_graph(k))
    assert wetric_mod.count(rp, ci, 5, 64)[0] == k
    assert wetric_mod.count(rp, ci, 1, 0)[0] == k


def test_empty_inputs(wetric_mod, oracle_mod):
    # no vertices with wedges
    rp = np.array([0, 1, 1], np.uint64)
    ci = np.array([1], np.uint32)
    assert wetric_mod.count(rp, ci, 5, 64)[0] == 0
    # no edges at all
    rp = np.zeros(5, np.uint64)
    assert wetric_mod.count(rp, np.zeros(0, np.uint32), 5, 64)[0] == 0
    # no vertices
    assert wetric_mod.count(np.zeros(1, np.uint64), np.zeros(0, np.uint32), 5, 0)[0] == 0
    # device preprocessing of self-loops only: n = 1 + the largest id of a
    # non-loop pair, 0 when there is none (tc.cu:587, 625)
    og = wetric_mod.orient_edges(np.array([2, 2], np.uint32), np.array([2, 2], np.uint32))
    assert (og.n, og.m) == (1, 0)
    assert og.count(5, 64)[0] == 0
    og.free()
    og = wetric_mod.orient_edges(np.zeros(0, np.uint32), np.zeros(0, np.uint32))
    assert (og.n, og.m) == (1, 0)
    og.free()


# ----------------------------------------------------------------- parity


SPREADS = (1, 2, 3, 5, 8, 16, 47)
BITMAPS = (0, 32, 64, 96, 4096, 8192)
KERNELS = (1, 2, 3, 4, 5, 6, 7, 8)  # block-tile, warp-staged, row-walk variants


@pytest.mark.parametrize("seed", range(8))
def test_random_graph_parity(wetric_mod, oracle_mod, seed):
    rng = np.random.default_rng(100 + seed)
    n = int(rng.integers(50, 20000))
    m = int(rng.integers(n, 30 * n))
    src, dst = random_pairs(n, m, seed)
    rp, ci, g = host_oriented(oracle_mod, src, dst)
    want = oracle_mod.count_merge(g)
    W = oracle_mod.wedge_total(g)
    for kernel in KERNELS:
        for s in SPREADS:
            for a in BITMAPS:
                got, st = wetric_mod.count(rp, ci, s, a, kernel=kernel)
                assert got == want, (n, m, s, a, kernel)
                assert st.wedges == W


@pytest.mark.parametrize("scale,ef,seed", [(10, 16, 1), (13, 16, 2), (15, 8, 3), (17, 16, 4)])
def test_rmat_parity(wetric_mod, oracle_mod, scale, ef, seed):
    from wetric import workloads as Wl

    spec = Wl.RmatSpec(scale=scale, edge_factor=ef, seed=seed)
    src, dst, _ = Wl.host_pairs(spec)
    rp, ci, g = host_oriented(oracle_mod, src, dst)
    want = oracle_mod.count_merge(g)
    assert oracle_mod.count_wedges(g, 4096) == want
    for kernel in KERNELS:
        for s, a in ((1, 0), (2, 4096), (5, 8192), (10, 16384), (5, 0)):
            assert wetric_mod.count(rp, ci, s, a, kernel=kernel)[0] == want, (spec, s, a)


def test_skewed_chung_lu_parity(wetric_mod, oracle_mod):
    from wetric import workloads as Wl

    spec = Wl.ChungLuSpec(n=50_000, gamma=2.1, i0=2.0, draws=600_000, seed=5)
    src, dst, _ = Wl.host_pairs(spec)
    rp, ci, g = host_oriented(oracle_mod, src, dst)
    want = oracle_mod.count_merge(g)
    for s, a in ((1, 0), (5, 8192), (32, 64)):
        assert wetric_mod.count(rp, ci, s, a)[0] == want


@pytest.mark.parametrize("kind", ["er", "chung_lu", "rmat", "small"])
def test_pair_streams_parity(wetric_mod, oracle_mod, torch_mod, kind):
    """Short rows counted by pair streams (the default) give the oracle's
    count, from host and device input and at several s / a; with the pair
    streams off the count is the same; the statistics split the wedges
    between the two; a forced dense core over pair vertices and a wedge
    range (which the pair streams do not take) still count exactly."""
    from wetric import workloads as Wl

    torch = torch_mod
    if kind == "er":
        src, dst = random_pairs(200_000, 3_000_000, 31)
    elif kind == "chung_lu":
        src, dst, _ = Wl.host_pairs(Wl.chung_lu_for(120_000, 30.0, 2.5, 32))
    elif kind == "rmat":
        src, dst, _ = Wl.host_pairs(Wl.RmatSpec(scale=16, edge_factor=16, seed=33))
    else:
        src, dst = random_pairs(300, 4000, 34)
    rp, ci, g = host_oriented(oracle_mod, src, dst)
    want = oracle_mod.count_merge(g)
    W = oracle_mod.wedge_total(g)
    drp = torch.from_numpy(rp.astype(np.int64)).cuda()
    dci = torch.from_numpy(ci.astype(np.int32)).cuda()
    for s, a in ((5, 8192), (1, 0), (10, 64)):
        on, st_on = wetric_mod.count(drp, dci, s, a)
        off, st_off = wetric_mod.count(drp, dci, s, a, pair_streams=False)
        host, st_host = wetric_mod.count(rp, ci, s, a)
        assert on == off == host == want, (kind, s, a)
        assert st_on.wedges == st_off.wedges == st_host.wedges == W
        assert st_on.wedges_counted == W
        assert st_off.pair_rows == 0 and st_off.pair_wedges == 0
        assert st_host.pair_rows == st_on.pair_rows
        assert 0 <= st_on.pair_wedges <= W
        if kind == "er":
            assert st_on.pair_rows > 0 and st_on.pair_wedges > 0
    # a forced core over rows that also take pair streams: each vertex is
    # counted once (the core's blocks skip the pair vertices)
    c_core, st_core = wetric_mod.count(drp, dci, 5, 8192, core_len=4096)
    assert c_core == want and st_core.core_len == min(4096, len(rp) - 1)
    # a wedge range is counted by the wedge check alone
    cuts = [0, W // 2, W]
    parts = [wetric_mod.count(drp, dci, 5, 8192, wedge_begin=b, wedge_end=e)
             for b, e in zip(cuts, cuts[1:])]
    assert sum(c for c, _ in parts) == want
    assert all(st.pair_rows == 0 for _, st in parts)


def test_config1_chung_lu_exact(wetric_mod, oracle_mod):
    """The plain single-graph case: n = 262,111, 899,792 edges, s=5, a=8192."""
    from wetric import workloads as Wl

    src, dst, _ = Wl.host_pairs(Wl.CHUNG_LU_262K)
    rp, ci, g = host_oriented(oracle_mod, src, dst)
    assert (g.n, g.m) == (262_111, 899_792)
    want = oracle_mod.count_merge(g)
    got, st = wetric_mod.count(rp, ci, 5, 8192)
    assert got == want
    assert st.wedges == oracle_mod.wedge_total(g)
    # the reference-shaped entry point on the u64 graph
    t = wetric_mod.GPUTime()
    assert wetric_mod.tc_GPU(wetric_mod.Graph(rp, ci), 5, 8192, t) == want
    assert t.copy > 0 and t.exec > 0


# ------------------------------------------------------ layouts and inputs


def test_u64_offset_kernels(wetric_mod, oracle_mod):
    """The u64-offset instantiations (used when m >= 2^32) on a graph small
    enough for the oracle, by keeping the offsets wide."""
    from wetric import workloads as Wl

    src, dst, _ = Wl.host_pairs(Wl.RmatSpec(scale=14, edge_factor=16, seed=11))
    rp, ci, g = host_oriented(oracle_mod, src, dst)
    want = oracle_mod.count_merge(g)
    for kernel in KERNELS:
        for s, a in ((1, 0), (5, 8192), (3, 64)):
            assert wetric_mod.count(rp, ci, s, a, kernel=kernel,
                                    keep_u64_offsets=True)[0] == want


def test_one_pass_launch(wetric_mod, oracle_mod):
    """WETRIC_OPT_ONE_PASS (one warp per tile, no tile counter) gives the
    persistent launch's count for every row-walk kernel, whole graph and
    wedge ranges."""
    from wetric import workloads as Wl

    src, dst, _ = Wl.host_pairs(Wl.RmatSpec(scale=13, edge_factor=16, seed=12))
    rp, ci, g = host_oriented(oracle_mod, src, dst)
    want = oracle_mod.count_merge(g)
    W = oracle_mod.wedge_total(g)
    for kernel in (3, 4, 5, 6, 7, 8):
        for s, a in ((1, 0), (5, 8192)):
            assert wetric_mod.count(rp, ci, s, a, kernel=kernel, one_pass=True)[0] == want
        cuts = [0, W // 3, W // 3 + 37, W]
        assert sum(wetric_mod.count(rp, ci, 2, 64, kernel=kernel, one_pass=True,
                                    wedge_begin=b, wedge_end=e)[0]
                   for b, e in zip(cuts, cuts[1:])) == want


def test_offsets_and_device_inputs(wetric_mod, oracle_mod, torch_mod):
    torch = torch_mod
    src, dst = random_pairs(3000, 40000, 21)
    rp, ci, g = host_oriented(oracle_mod, src, dst)
    want = oracle_mod.count_merge(g)
    assert wetric_mod.count(rp.astype(np.uint32), ci, 5, 64)[0] == want
    assert wetric_mod.count_simple(rp, ci, 5, 64) == want
    drp = torch.from_numpy(rp.astype(np.int64)).cuda()
    dci = torch.from_numpy(ci.astype(np.int32)).cuda()
    assert wetric_mod.count(drp, dci, 5, 64)[0] == want
    assert wetric_mod.count(drp.to(torch.int32), dci, 3, 0)[0] == want
    # a caller stream
    s = torch.cuda.Stream()
    assert wetric_mod.count(drp, dci, 5, 64, stream=s)[0] == want
    # symmetric input oriented on the device
    sym = oracle_mod.csr_from_pairs(src, dst)
    assert wetric_mod.count(sym.row_ptr, sym.col_ind, 5, 64, oriented=False)[0] == want
    assert wetric_mod.count(sym.row_ptr.astype(np.uint32), sym.col_ind, 2, 0,
                            oriented=False)[0] == want


def test_wedge_ranges(wetric_mod, oracle_mod):
    src, dst = random_pairs(5000, 80000, 22)
    rp, ci, g = host_oriented(oracle_mod, src, dst)
    W = oracle_mod.wedge_total(g)
    want = oracle_mod.count_merge(g)
    cuts = sorted({0, W, *np.random.default_rng(1).integers(0, W, 9).tolist()})
    total = 0
    for b, e in zip(cuts, cuts[1:]):
        part, st = wetric_mod.count(rp, ci, 5, 64, wedge_begin=b, wedge_end=e)
        assert part == oracle_mod.count_wedges(g, 64, b, e)
        assert st.wedges_counted == e - b
        total += part
    assert total == want
    # empty and out-of-range ranges
    assert wetric_mod.count(rp, ci, 5, 64, wedge_begin=W, wedge_end=W + 10)[0] == 0
    assert wetric_mod.count(rp, ci, 5, 64, wedge_begin=7, wedge_end=7)[0] == 0


def test_host_input_row_chunks(wetric_mod, oracle_mod):
    """Host CSRs of 2^22 columns or more are copied in row chunks, highest
    rows first, and counted chunk by chunk as they arrive: the count equals
    the oracle's and the unchunked (validated) count's for u32 and u64
    offsets, every row-walk kernel and the block-tile kernel, one-pass
    launches and wedge ranges that cut across chunks."""
    src, dst = wetric_mod.gen_rmat(19, 16 << 19, seed=12)
    rp, ci, g = host_oriented(oracle_mod, src, dst)
    assert g.m >= 1 << 22
    want = oracle_mod.count_merge(g)
    W = oracle_mod.wedge_total(g)
    rp32 = rp.astype(np.uint32)
    for kernel in (1, 4, 7, 8):
        for s, a in ((5, 8192), (1, 0), (10, 4096)):
            got, st = wetric_mod.count(rp32, ci, s, a, kernel=kernel)
            assert got == want, (kernel, s, a)
            assert st.wedges_counted == W
    assert wetric_mod.count(rp, ci, 5, 8192)[0] == want
    assert wetric_mod.count(rp32, ci, 5, 8192, validate=True)[0] == want
    assert wetric_mod.count(rp32, ci, 5, 8192, one_pass=True)[0] == want
    cuts = sorted({0, W, *np.random.default_rng(4).integers(0, W, 5).tolist()})
    total = 0
    for b, e in zip(cuts, cuts[1:]):
        part, st = wetric_mod.count(rp32, ci, 5, 8192, wedge_begin=b, wedge_end=e)
        assert st.wedges_counted == e - b
        total += part
    assert total == want
    # broken row offsets in a chunk-sized CSR: rejected by the device row
    # check (before any column copy), whatever the chunk boundaries see
    n = len(rp32) - 1
    for bad in (n // 2, n // 8, n - 1):
        rpb = rp32.copy()
        rpb[bad] = rpb[-1] + 5
        with pytest.raises(wetric_mod.WetricError) as e:
            wetric_mod.count(rpb, ci, 5, 8192)
        assert e.value.status == wetric_mod.EINVAL
    rpb = rp32.copy()
    rpb[-1] -= 1  # offsets end short of m
    with pytest.raises(wetric_mod.WetricError):
        wetric_mod.count(rpb, ci, 5, 8192)
    assert wetric_mod.count(rp32, ci, 5, 8192)[0] == want


def test_validation_and_errors(wetric_mod, oracle_mod):
    rp = np.array([0, 2, 3, 3], np.uint64)
    # unsorted row 0
    ci = np.array([2, 1, 2], np.uint32)
    with pytest.raises(wetric_mod.WetricError) as e:
        wetric_mod.count(rp, ci, 5, 64, validate=True)
    assert e.value.status == wetric_mod.EINVAL
    # column below its row (not oriented)
    ci = np.array([1, 2, 0], np.uint32)
    with pytest.raises(wetric_mod.WetricError):
        wetric_mod.count(rp, ci, 5, 64, validate=True)
    # column out of range: rejected by validation, harmless without it
    ci = np.array([1, 9, 2], np.uint32)
    with pytest.raises(wetric_mod.WetricError):
        wetric_mod.count(rp, ci, 5, 64, validate=True)
    wetric_mod.count(rp, ci, 5, 64)
    # broken row offsets are always rejected
    with pytest.raises(wetric_mod.WetricError) as e:
        wetric_mod.count(np.array([0, 3, 2, 3], np.uint64), np.array([1, 2, 2], np.uint32), 5, 64)
    assert e.value.status == wetric_mod.EINVAL
    with pytest.raises(wetric_mod.WetricError):
        wetric_mod.count(np.array([0, 2, 3, 5], np.uint64), np.array([1, 2, 2], np.uint32), 5, 64)
    # the library stays usable after errors
    rp2, ci2, _ = host_oriented(oracle_mod, *complete_graph(6))
    assert wetric_mod.count(rp2, ci2, 5, 64)[0] == 20


def test_hbm_budget_rejects_then_recovers(wetric_mod, oracle_mod):
    rp, ci, _ = host_oriented(oracle_mod, *complete_graph(30))
    wetric_mod.set_hbm_budget(1024)
    try:
        with pytest.raises(wetric_mod.WetricError) as e:
            wetric_mod.count(rp, ci, 5, 64)
        assert e.value.status == wetric_mod.ENOMEM
    finally:
        wetric_mod.set_hbm_budget(0)
    assert wetric_mod.count(rp, ci, 5, 64)[0] == comb3(30)


# ------------------------------------------------------- preprocessing


def test_device_orientation_bit_exact(wetric_mod, oracle_mod, torch_mod):
    torch = torch_mod
    for seed, (n, m) in enumerate([(10, 30), (1000, 20000), (70000, 300000), (1 << 20, 50000)]):
        src, dst = random_pairs(n, m, 40 + seed)
        want = oracle_mod.oriented_from_pairs(src, dst)
        og = wetric_mod.orient_edges(src, dst)
        got = og.download()
        assert np.array_equal(got.row_ptr, want.row_ptr)
        assert np.array_equal(got.col_ind, want.col_ind)
        # device-resident pairs give the same CSR
        og2 = wetric_mod.orient_edges(torch.from_numpy(src.astype(np.int32)).cuda(),
                                      torch.from_numpy(dst.astype(np.int32)).cuda())
        got2 = og2.download()
        assert np.array_equal(got2.col_ind, want.col_ind)
        assert og2.count(5, 64)[0] == oracle_mod.count_merge(want)
        og.free()
        og2.free()


def test_reference_mirrors_bit_exact(wetric_mod, oracle_mod):
    """read_graph / preprocess mirrors equal the oracle's restatements."""
    with open(os.path.join(GOLDEN, "hand_graphs.json")) as f:
        hand = json.load(f)
    for h in hand["graphs"]:
        path = os.path.join(GOLDEN, h["file"])
        sym = wetric_mod.read_graph(path, h["mm"], h["zero_indexed"])
        want = oracle_mod.read_graph(path, h["mm"], h["zero_indexed"])
        assert np.array_equal(sym.row_ptr, want.row_ptr), h["file"]
        assert np.array_equal(sym.col_ind, want.col_ind), h["file"]
        g = wetric_mod.preprocess(sym)
        gw = oracle_mod.preprocess(want)
        assert np.array_equal(g.row_ptr, gw.row_ptr) and np.array_equal(g.col_ind, gw.col_ind)
        assert wetric_mod.tc_GPU(g, 5, 8192) == h["triangles"]
        assert (g.n, g.m) == (h["n"], h["m"])
    for h in hand["errors"]:
        with pytest.raises(wetric_mod.WetricError):
            wetric_mod.read_graph(os.path.join(GOLDEN, h["file"]), h["mm"], h["zero_indexed"])


def test_read_graph_file_roundtrip(tmp_path, wetric_mod, oracle_mod):
    s, d = wetric_mod.gen_rmat(15, 400_000, seed=77)
    path = str(tmp_path / "r.mtx")
    wetric_mod.write_mm(path, 1 << 15, s, d)
    sym = wetric_mod.read_graph(path, True, False)
    want = oracle_mod.read_graph(path, True, False)
    assert np.array_equal(sym.row_ptr, want.row_ptr)
    assert np.array_equal(sym.col_ind, want.col_ind)


def test_device_generators_match_host(wetric_mod, torch_mod):
    s, d = wetric_mod.gen_rmat(20, 1_000_003, seed=3)
    ds, dd = wetric_mod.gen_rmat_device(20, 1_000_003, seed=3)
    assert np.array_equal(ds.cpu().numpy().view(np.uint32), s)
    assert np.array_equal(dd.cpu().numpy().view(np.uint32), d)
    cdf = wetric_mod.chung_lu_cdf(10_000, 2.5, 10.0)
    s, d = wetric_mod.gen_weighted(cdf, 10_000, 100_000, seed=8)
    ds, dd = wetric_mod.gen_weighted_device(cdf, 10_000, 100_000, seed=8)
    assert np.array_equal(ds.cpu().numpy().view(np.uint32), s)
    s, d = wetric_mod.gen_weighted(None, 999, 5000, seed=2)
    ds, dd = wetric_mod.gen_weighted_device(None, 999, 5000, seed=2)
    assert np.array_equal(dd.cpu().numpy().view(np.uint32), d)


# -------------------------------------------------- statistics and bytes


def test_stats_match_oracle(wetric_mod, oracle_mod, torch_mod):
    torch = torch_mod
    src, dst = random_pairs(4000, 60000, 9)
    g = oracle_mod.oriented_from_pairs(src, dst)
    drp = torch.from_numpy(g.row_ptr.astype(np.int64)).cuda()
    dci = torch.from_numpy(g.col_ind.astype(np.int32)).cuda()
    W, md = wetric_mod.wedge_total(drp)
    assert W == oracle_mod.wedge_total(g) and md == oracle_mod.max_out_degree(g)
    assert wetric_mod.algorithmic_bytes(drp, dci) == oracle_mod.algorithmic_bytes(g)


# -------------------------------------- against the reference's own outputs


REF_JSON = os.path.join(GOLDEN, "reference_counts.json")


@pytest.mark.skipif(not os.path.exists(REF_JSON), reason="reference outputs not generated")
def test_against_recorded_reference_outputs(wetric_mod):
    from wetric import workloads as Wl

    with open(REF_JSON) as f:
        ref = json.load(f)
    kinds = {"RmatSpec": Wl.RmatSpec, "ChungLuSpec": Wl.ChungLuSpec,
             "ErdosRenyiSpec": Wl.ErdosRenyiSpec}
    for entry in ref["seeded"]:
        d = dict(entry["spec"])
        spec = kinds[d.pop("kind")](**{k: v for k, v in d.items() if k != "name"})
        src, dst, _ = Wl.host_pairs(spec)
        og = wetric_mod.orient_edges(src, dst)
        for run in entry["runs"]:
            assert (og.n, og.m) == (run["n"], run["m"]), spec
            assert og.count(run["s"], run["a"])[0] == run["triangles"], (spec, run)
        og.free()


def _ref_bin():
    import oracle

    return oracle.have_reference_binary()


@pytest.mark.skipif(not _ref_bin(), reason="reference tc not built (make -C oracle ref)")
def test_cli_matches_reference_binary(tmp_path, wetric_mod, oracle_mod):
    """Our tc and the reference's tc (sm_100a build) print the same header
    and the same n, m, s, a, triangles on the same file."""
    s, d = wetric_mod.gen_rmat(14, 16 << 14, seed=31)
    path = str(tmp_path / "g.mtx")
    wetric_mod.write_mm(path, 1 << 14, s, d)
    ours = subprocess.run([os.path.join(PKG, "bin", "tc"), "-m", path, "-s", "5", "-a", "8192",
                           "-l", "2"], capture_output=True, text=True, timeout=300)
    assert ours.returncode == 0, ours.stderr
    theirs = subprocess.run([oracle_mod.REF_TC, "-m", path, "-s", "5", "-a", "8192", "-l", "2"],
                            capture_output=True, text=True, timeout=300)
    assert theirs.returncode == 0, theirs.stderr
    ol, tl = ours.stdout.splitlines(), theirs.stdout.splitlines()
    assert ol[0] == tl[0]  # header line, byte for byte
    assert len(ol) == len(tl) == 3
    end = max(60, len(path)) + 17 * 5  # through the triangles column
    for a, b in zip(ol[1:], tl[1:]):
        assert a.split()[:6] == b.split()[:6]
        assert a[:end] == b[:end]


@pytest.mark.skipif(not os.path.exists(os.path.join(PKG, "bin", "tc")), reason="tc not built")
def test_cli_flags(tmp_path):
    tc = os.path.join(PKG, "bin", "tc")
    k4 = os.path.join(GOLDEN, "k4.mtx")
    out = subprocess.run([tc, "-m", k4, "-s", "1", "-a", "64", "-l", "3"], capture_output=True,
                         text=True, timeout=120)
    assert out.returncode == 0
    rows = out.stdout.splitlines()[1:]
    assert len(rows) == 3 and all(r.split()[5] == "4" for r in rows)
    z = os.path.join(GOLDEN, "wheel8_zero.el")
    out = subprocess.run([tc, "-z", "-e", z, "-s", "2", "-a", "0", "-p", "0"],
                         capture_output=True, text=True, timeout=120)
    assert out.returncode == 0 and out.stdout.splitlines()[1].split()[5] == "8"
    for bad in (["-m", k4, "-s", "0", "-a", "64"], ["-m", k4, "-s", "1", "-a", "33"],
                ["-m", k4, "-s", "1", "-q"], ["-s", "1"], ["-m", k4, "-s", "1", "-p", "3"]):
        r = subprocess.run([tc, *bad], capture_output=True, text=True, timeout=60)
        assert r.returncode != 0
    r = subprocess.run([tc, "-e", os.path.join(GOLDEN, "zero_id.el"), "-s", "1"],
                       capture_output=True, text=True, timeout=60)
    assert r.returncode != 0
    # -w writes the preprocessed CSR; -c counts from it without parsing
    cache = str(tmp_path / "k5.wcsr")
    k5 = os.path.join(GOLDEN, "k5_dups_loops.el")
    a = subprocess.run([tc, "-e", k5, "-s", "1", "-a", "64", "-w", cache],
                       capture_output=True, text=True, timeout=120)
    b = subprocess.run([tc, "-c", cache, "-s", "3", "-a", "0"],
                       capture_output=True, text=True, timeout=120)
    assert a.returncode == 0 and b.returncode == 0
    assert a.stdout.splitlines()[1].split()[5] == b.stdout.splitlines()[1].split()[5] == "10"
    bad = str(tmp_path / "bad.wcsr")
    open(bad, "wb").write(b"not a cache")
    r = subprocess.run([tc, "-c", bad, "-s", "1"], capture_output=True, text=True, timeout=60)
    assert r.returncode != 0
    # -j appends one JSON line per printed run (K_4: 4 wedges, 4 triangles)
    js = str(tmp_path / "runs.jsonl")
    r = subprocess.run([tc, "-m", k4, "-s", "1", "-a", "64", "-l", "2", "-j", js],
                       capture_output=True, text=True, timeout=120)
    assert r.returncode == 0
    lines = [json.loads(x) for x in open(js).read().splitlines()]
    assert len(lines) == 2
    assert all(x["triangles"] == 4 and x["wedges"] == 4 and x["n"] == 4 for x in lines)


# --------------------------------------------- size-independent properties


def test_large_rmat_invariants(wetric_mod, torch_mod):
    """R-MAT scale 21 on the device: the count is invariant under spread,
    bitmap length, wedge-range splits and a relabelling of the ids."""
    torch = torch_mod
    from wetric import workloads as Wl

    spec = Wl.RmatSpec(scale=21, edge_factor=16, seed=9)
    src, dst, _ = Wl.device_pairs(spec)
    og = wetric_mod.orient_edges(src, dst)
    base, st = og.count(5, 8192)
    W = st.wedges
    for s, a in ((1, 0), (2, 4096), (10, 16384), (16, 64)):
        assert og.count(s, a)[0] == base
    parts = [og.count(5, 8192, wedge_begin=W * i // 5, wedge_end=W * (i + 1) // 5)[0]
             for i in range(5)]
    assert sum(parts) == base
    perm = torch.randperm(1 << 21, device="cuda", generator=torch.Generator("cuda").manual_seed(1))
    perm = perm.to(torch.int32)
    og2 = wetric_mod.orient_edges(perm[src.long()], perm[dst.long()], n=1 << 21)
    assert og2.count(5, 8192)[0] == base
    og.free()
    og2.free()


def test_pageable_host_columns_concurrent(wetric_mod, oracle_mod):
    """Pageable (numpy) host columns are staged through the library's pinned
    buffers; two threads counting at once (one stages, the other copies
    directly while the buffers are held) and a pinned copy of the same CSR
    all give the oracle's count."""
    import threading

    import torch

    src, dst = wetric_mod.gen_rmat(19, 16 << 19, seed=17)
    g = oracle_mod.oriented_from_pairs(src, dst)
    assert g.m >= 1 << 22
    want = oracle_mod.count_merge(g)
    rp32 = g.row_ptr.astype(np.uint32)
    got = {}

    def run(k):
        for i in range(3):
            got[(k, i)] = wetric_mod.count(rp32, g.col_ind, 5, 8192)[0]

    ths = [threading.Thread(target=run, args=(k,)) for k in range(2)]
    for t in ths:
        t.start()
    for t in ths:
        t.join(timeout=300)
    assert len(got) == 6 and set(got.values()) == {want}
    ci_pin = torch.from_numpy(g.col_ind.view(np.int32)).pin_memory()
    assert wetric_mod.count(rp32, ci_pin.numpy().view(np.uint32), 5, 8192)[0] == want
