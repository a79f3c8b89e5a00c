"""CPU tests of the oracle: closed forms, hand fixtures, the reference's own
outputs (tests/golden/reference_counts.json), and the two independent
counting algorithms against each other."""
from __future__ import annotations

import json
import math
import os

import numpy as np
import pytest

from conftest import (GOLDEN, bipartite_graph, comb3, complete_graph,
                      random_pairs, star_graph, wheel_graph)


def oriented(oracle_mod, src, dst, n=0):
    return oracle_mod.oriented_from_pairs(src, dst, n)


@pytest.mark.parametrize("k", [3, 4, 5, 6, 9, 12, 20])
def test_complete_graph_closed_form(oracle_mod, k):
    g = oriented(oracle_mod, *complete_graph(k))
    assert g.m == k * (k - 1) // 2
    assert oracle_mod.count_merge(g) == comb3(k)
    for a in (0, 32, 64, 128):
        assert oracle_mod.count_wedges(g, a) == comb3(k)


def test_star_bipartite_wheel(oracle_mod):
    g = oriented(oracle_mod, *star_graph(50))
    assert oracle_mod.wedge_total(g) == 0 or oracle_mod.count_merge(g) == 0
    assert oracle_mod.count_wedges(g, 64) == 0
    g = oriented(oracle_mod, *bipartite_graph(7, 9))
    assert oracle_mod.count_merge(g) == 0 and oracle_mod.count_wedges(g, 0) == 0
    for k in (4, 5, 10, 33):
        g = oriented(oracle_mod, *wheel_graph(k))
        assert oracle_mod.count_merge(g) == k
        assert oracle_mod.count_wedges(g, 64) == k


def test_empty_and_loops_only(oracle_mod):
    g = oriented(oracle_mod, np.array([3, 3], np.uint32), np.array([3, 3], np.uint32))
    assert g.m == 0 and g.n == 1
    assert oracle_mod.count_merge(g) == 0
    assert oracle_mod.count_wedges(g, 64) == 0


@pytest.mark.parametrize("seed", range(6))
def test_merge_equals_wedge_check(oracle_mod, seed):
    rng = np.random.default_rng(seed)
    n = int(rng.integers(20, 3000))
    m = int(rng.integers(n, 20 * n))
    g = oriented(oracle_mod, *random_pairs(n, m, seed))
    want = oracle_mod.count_merge(g)
    for a in (0, 64, 96 if n > 96 else 64, 4096):
        assert oracle_mod.count_wedges(g, a) == want


def test_wedge_ranges_partition(oracle_mod):
    g = oriented(oracle_mod, *random_pairs(500, 6000, 11))
    W = oracle_mod.wedge_total(g)
    total = oracle_mod.count_merge(g)
    cuts = sorted({0, W, *np.random.default_rng(3).integers(0, W, 7).tolist()})
    parts = [oracle_mod.count_wedges(g, 64, b, e) for b, e in zip(cuts, cuts[1:]) if e > b]
    assert sum(parts) == total


def test_orientation_invariants(oracle_mod):
    """The oriented graph has every column above its row, sorted rows, no
    reverse edge (the check of experiments/edge_get.cu:311-317) and one entry
    per undirected edge; vertices are in stable ascending-degree order."""
    src, dst = random_pairs(2000, 30000, 5)
    sym = oracle_mod.csr_from_pairs(src, dst)
    g = oracle_mod.preprocess(sym)
    assert g.m * 2 == sym.m
    rp, ci = g.row_ptr, g.col_ind
    rows = np.repeat(np.arange(g.n), np.diff(rp).astype(np.int64))
    assert np.all(ci > rows)
    for v in range(g.n):
        r = ci[rp[v]:rp[v + 1]]
        assert np.all(np.diff(r.astype(np.int64)) > 0)
    deg = np.diff(sym.row_ptr).astype(np.int64)
    order = np.lexsort((np.arange(sym.n), deg))
    # rank(v) = position in order; in-degree + out-degree of new id r equals
    # the symmetric degree of order[r]
    indeg = np.bincount(ci, minlength=g.n)
    outdeg = np.diff(rp).astype(np.int64)
    assert np.array_equal(indeg + outdeg, deg[order])


def _int_decode(iv: int, d: int):
    """Integer restatement used by the device decode (csrc/count.cu)."""
    W = d * (d - 1) // 2
    j = W - 1 - iv
    q = (math.isqrt(8 * j + 1) - 1) >> 1
    p = j - q * (q + 1) // 2
    return d - 2 - q, d - 1 - p


def test_integer_decode_matches_reference_formula(oracle_mod):
    for d in range(2, 120):
        for iv in range(d * (d - 1) // 2):
            assert _int_decode(iv, d) == oracle_mod.decode_wedge(iv, d)
    rng = np.random.default_rng(0)
    for d in [1000, 4095, 65535, 70000, 1 << 20, 3_000_001]:
        W = d * (d - 1) // 2
        for iv in [0, 1, W - 1, W - 2, *rng.integers(0, W, 200).tolist()]:
            assert _int_decode(int(iv), d) == oracle_mod.decode_wedge(int(iv), d)


def test_row_major_wedge_order(oracle_mod):
    d = 7
    seen = [_int_decode(i, d) for i in range(d * (d - 1) // 2)]
    assert seen == [(w, u) for w in range(d) for u in range(w + 1, d)]


def test_hand_fixtures(oracle_mod):
    with open(os.path.join(GOLDEN, "hand_graphs.json")) as f:
        hand = json.load(f)
    for h in hand["graphs"]:
        sym = oracle_mod.read_graph(os.path.join(GOLDEN, h["file"]), h["mm"], h["zero_indexed"])
        g = oracle_mod.preprocess(sym)
        assert (g.n, g.m) == (h["n"], h["m"]), h["file"]
        assert oracle_mod.count_merge(g) == h["triangles"], h["file"]
        assert oracle_mod.count_wedges(g, 8192) == h["triangles"], h["file"]
    for h in hand["errors"]:
        with pytest.raises(oracle_mod.OracleError):
            oracle_mod.read_graph(os.path.join(GOLDEN, h["file"]), h["mm"], h["zero_indexed"])
    # The weighted file: the reference's token-stream parse keeps the first
    # line's pair and the next line's, then stops at the weight "1.5".
    w = hand["deviations"][0]
    g = oracle_mod.preprocess(oracle_mod.read_graph(os.path.join(GOLDEN, w["file"]), True, False))
    assert (g.n, g.m) == (3, 2)


REF_JSON = os.path.join(GOLDEN, "reference_counts.json")


def _spec(d):
    from wetric import workloads as W

    kind = d.pop("kind")
    d.pop("name")
    return {"RmatSpec": W.RmatSpec, "ChungLuSpec": W.ChungLuSpec,
            "ErdosRenyiSpec": W.ErdosRenyiSpec}[kind](**d)


@pytest.mark.skipif(not os.path.exists(REF_JSON), reason="reference outputs not generated")
def test_oracle_pinned_to_reference_outputs(oracle_mod):
    """The oracle reproduces every count the reference's own binaries
    printed on the seeded graphs and the hand fixtures."""
    from wetric import workloads as W

    with open(REF_JSON) as f:
        ref = json.load(f)
    assert ref["seeded"], "no seeded reference rows"
    for entry in ref["seeded"]:
        spec = _spec(dict(entry["spec"]))
        src, dst, _ = W.host_pairs(spec)
        g = oracle_mod.oriented_from_pairs(src, dst)
        tri = oracle_mod.count_merge(g)
        for run in entry["runs"]:
            assert run["n"] == g.n, spec
            assert run["m"] == g.m, spec
            assert run["triangles"] == tri, (spec, run)
            assert oracle_mod.count_wedges(g, run["a"]) == tri
    with open(os.path.join(GOLDEN, "hand_graphs.json")) as f:
        hand = {h["file"]: h for h in json.load(f)["graphs"]}
    for row in ref["hand"]:
        if row["file"] in hand:
            h = hand[row["file"]]
            assert (row["n"], row["m"], row["triangles"]) == (h["n"], h["m"], h["triangles"])
        else:  # the weighted deviation file: the reference keeps two pairs
            assert (row["n"], row["m"], row["triangles"]) == (3, 2, 0)


def test_oracle_rmat_stream_and_mm_writer_match_the_library(tmp_path):
    """The oracle's R-MAT stream and Matrix Market writer (used by the
    benchmark's reference arm so that arm never loads the product library)
    give the same pairs and the same bytes as the library's own."""
    import oracle
    import wetric

    for scale, ef, seed in ((10, 16, 1), (16, 8, 3), (13, 16, 77)):
        s1, d1 = oracle.gen_rmat(scale, ef << scale, seed=seed)
        s2, d2 = wetric.gen_rmat(scale, ef << scale, seed=seed)
        assert np.array_equal(s1, s2) and np.array_equal(d1, d2)
        oracle.write_mm(str(tmp_path / "o.mtx"), 1 << scale, s1, d1)
        wetric.write_mm(str(tmp_path / "w.mtx"), 1 << scale, s2, d2)
        assert (tmp_path / "o.mtx").read_bytes() == (tmp_path / "w.mtx").read_bytes()


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_wedge_total_from_pairs_two_ways(seed):
    """W and the max out-degree from raw pairs: the C radix-sort form, the
    numpy form and the oriented CSR all agree (self-loops, duplicates and
    both directions present)."""
    import oracle

    rng = np.random.default_rng(seed)
    n = int(rng.integers(50, 3000))
    src = rng.integers(0, n, 20 * n).astype(np.uint32)
    dst = rng.integers(0, n, 20 * n).astype(np.uint32)
    src[:5] = dst[:5]  # self-loops
    g = oracle.oriented_from_pairs(src, dst)
    want = (oracle.wedge_total(g), oracle.max_out_degree(g))
    assert oracle.wedge_total_from_pairs(src, dst) == want
    assert oracle.wedge_total_from_pairs_numpy(src, dst) == want
    assert oracle.wedge_total_from_pairs(np.zeros(0, np.uint32), np.zeros(0, np.uint32)) == (0, 0)
