"""CPU tests of the host-side tools: generators, the Matrix Market writer
and the product's parser (against the oracle's restatement of
read_graph)."""
from __future__ import annotations

import json
import os

import numpy as np
import pytest

from conftest import GOLDEN


def test_rmat_deterministic_and_in_range(wetric_mod):
    s1, d1 = wetric_mod.gen_rmat(12, 50_000, seed=9)
    s2, d2 = wetric_mod.gen_rmat(12, 50_000, seed=9)
    s3, _ = wetric_mod.gen_rmat(12, 50_000, seed=10)
    assert np.array_equal(s1, s2) and np.array_equal(d1, d2)
    assert not np.array_equal(s1, s3)
    assert s1.max() < 4096 and d1.max() < 4096
    # quadrant probabilities at the top level: P(src bit) = c + d = 0.24,
    # P(dst bit) = b + d = 0.24
    top_s = (s1 >> 11).mean()
    top_d = (d1 >> 11).mean()
    assert abs(top_s - 0.24) < 0.01 and abs(top_d - 0.24) < 0.01
    # prefix property: edge k does not depend on the stream length
    s4, d4 = wetric_mod.gen_rmat(12, 1000, seed=9)
    assert np.array_equal(s4, s1[:1000]) and np.array_equal(d4, d1[:1000])


def test_chung_lu_degrees(wetric_mod):
    from wetric import workloads as W

    src, dst, n = W.host_pairs(W.CHUNG_LU_262K)
    assert n == 262_111
    keep = src != dst
    lo = np.minimum(src[keep], dst[keep]).astype(np.uint64)
    hi = np.maximum(src[keep], dst[keep]).astype(np.uint64)
    k = np.unique(lo << np.uint64(32) | hi)
    assert len(k) == 899_792
    deg = np.bincount(np.concatenate([(k >> np.uint64(32)).astype(np.int64),
                                      (k & np.uint64(0xFFFFFFFF)).astype(np.int64)]),
                      minlength=n)
    assert 400 <= deg.max() <= 440
    assert abs(deg.mean() - 6.87) < 0.05


def test_erdos_renyi_uniform(wetric_mod):
    s, d = wetric_mod.gen_weighted(None, 1000, 200_000, seed=3)
    c = np.bincount(np.concatenate([s, d]), minlength=1000)
    assert c.min() > 300 and c.max() < 500


def test_write_mm_roundtrip(tmp_path, wetric_mod, oracle_mod):
    s, d = wetric_mod.gen_rmat(10, 8000, seed=4)
    path = str(tmp_path / "g.mtx")
    wetric_mod.write_mm(path, 1024, s, d)
    via_file = oracle_mod.read_graph(path, True, False)
    direct = oracle_mod.csr_from_pairs(s, d)
    assert np.array_equal(via_file.row_ptr, direct.row_ptr)
    assert np.array_equal(via_file.col_ind, direct.col_ind)
    with open(path) as f:
        assert f.readline().startswith("%%MatrixMarket matrix coordinate pattern symmetric")


def _csr_of_pairs(oracle_mod, s, d, n):
    return oracle_mod.csr_from_pairs(s, d, n)


def test_parser_matches_reference_rules(tmp_path, wetric_mod, oracle_mod):
    """Product parser == oracle read_graph (the reference's rules) on
    two-column files, big enough to split across parser threads."""
    s, d = wetric_mod.gen_rmat(16, 300_000, seed=12)
    path = str(tmp_path / "big.mtx")
    wetric_mod.write_mm(path, 1 << 16, s, d)
    ps, pd, n = wetric_mod.parse_file(path, True, False)
    want = oracle_mod.read_graph(path, True, False)
    got = oracle_mod.csr_from_pairs(ps, pd, n)
    assert n == want.n
    assert np.array_equal(got.row_ptr, want.row_ptr)
    assert np.array_equal(got.col_ind, want.col_ind)
    assert not np.any(ps == pd)  # self-loops dropped


def test_parser_hand_fixtures(wetric_mod, oracle_mod):
    with open(os.path.join(GOLDEN, "hand_graphs.json")) as f:
        hand = json.load(f)
    for h in hand["graphs"]:
        path = os.path.join(GOLDEN, h["file"])
        ps, pd, n = wetric_mod.parse_file(path, h["mm"], h["zero_indexed"])
        assert n == h["n"], h["file"]
        g = oracle_mod.preprocess(oracle_mod.csr_from_pairs(ps, pd, n))
        assert g.m == h["m"]
        assert oracle_mod.count_merge(g) == h["triangles"]
    for h in hand["errors"]:
        with pytest.raises(wetric_mod.WetricError) as e:
            wetric_mod.parse_file(os.path.join(GOLDEN, h["file"]), h["mm"], h["zero_indexed"])
        assert e.value.status in (wetric_mod.EIO, wetric_mod.EINVAL)
    # zero_id.el parses when zero-indexing is set: a triangle on 0, 1, 2
    ps, pd, n = wetric_mod.parse_file(os.path.join(GOLDEN, "zero_id.el"), False, True)
    assert n == 3 and len(ps) == 3
    # weighted: every line's pair is read, the third column ignored
    dev = hand["deviations"][0]
    ps, pd, n = wetric_mod.parse_file(os.path.join(GOLDEN, dev["file"]), True, False)
    g = oracle_mod.preprocess(oracle_mod.csr_from_pairs(ps, pd, n))
    assert (g.n, g.m, oracle_mod.count_merge(g)) == (dev["n"], dev["m"], dev["triangles"])


def test_parser_edge_cases(tmp_path, wetric_mod):
    p = tmp_path / "x.el"
    p.write_text("c header\n\n1 2\n\n  2 3   \n3 1\nbad line\n4 5\n")
    s, d, n = wetric_mod.parse_file(str(p), False, False)
    # parse stops at "bad line"; blank and indented lines inside the body
    # are read like fscanf's whitespace skip
    assert list(zip(s.tolist(), d.tolist())) == [(0, 1), (1, 2), (2, 0)]
    assert n == 3
    p.write_text("%%MatrixMarket\n5 5 1\n")
    s, d, n = wetric_mod.parse_file(str(p), True, False)
    assert len(s) == 0 and n == 1
    p.write_text("1 -2\n")
    with pytest.raises(wetric_mod.WetricError):
        wetric_mod.parse_file(str(p), False, False)
    p.write_text("1 99999999999\n")
    with pytest.raises(wetric_mod.WetricError):
        wetric_mod.parse_file(str(p), False, False)
    with pytest.raises(wetric_mod.WetricError):
        wetric_mod.parse_file(str(tmp_path / "missing.el"), False, False)


def test_csr_cache_round_trip_and_rejects_bad_files(wetric_mod, oracle_mod, tmp_path):
    """wetric_save_csr / wetric_load_csr: u64 and u32 offsets round-trip
    bit for bit with their orientation flag; truncated, foreign or
    inconsistent files are errors, not graphs."""
    from conftest import random_pairs

    src, dst = random_pairs(500, 6000, 77)
    g = oracle_mod.oriented_from_pairs(src, dst)
    rp, ci = np.asarray(g.row_ptr, np.uint64), np.asarray(g.col_ind, np.uint32)
    p = str(tmp_path / "g.wcsr")
    for offsets, oriented in ((rp, True), (rp.astype(np.uint32), False)):
        wetric_mod.save_csr(p, offsets, ci, oriented=oriented)
        rp2, ci2, o2 = wetric_mod.load_csr(p)
        assert rp2.dtype == np.uint64 and np.array_equal(rp2, rp)
        assert np.array_equal(ci2, ci) and o2 == oriented
    # empty graph
    wetric_mod.save_csr(p, np.zeros(1, np.uint64), np.zeros(0, np.uint32))
    rp3, ci3, _ = wetric_mod.load_csr(p)
    assert rp3.tolist() == [0] and ci3.size == 0
    # damaged files
    wetric_mod.save_csr(p, rp, ci)
    raw = open(p, "rb").read()
    bad = []
    bad.append(raw[:-4])                                   # truncated
    bad.append(b"NOTACSR!" + raw[8:])                      # foreign magic
    b = bytearray(raw)
    b[32 + 8 * 3:32 + 8 * 4] = (10**9).to_bytes(8, "little")  # offset past m
    bad.append(bytes(b))
    b = bytearray(raw)
    off = 32 + 8 * (len(rp)) + 4 * 3
    b[off:off + 4] = (10**6).to_bytes(4, "little")         # column >= n
    bad.append(bytes(b))
    for k, data in enumerate(bad):
        q = str(tmp_path / f"bad{k}.wcsr")
        open(q, "wb").write(data)
        with pytest.raises(wetric_mod.WetricError) as e:
            wetric_mod.load_csr(q)
        assert e.value.status == wetric_mod.EIO, k
    with pytest.raises(wetric_mod.WetricError):
        wetric_mod.load_csr(str(tmp_path / "missing.wcsr"))


def test_parser_fuzz_matches_oracle(tmp_path, wetric_mod, oracle_mod):
    """Seeded random files in the reference's accepted forms -- header lines
    that do not start with a digit, an MM size line, pairs split by spaces,
    tabs and blank lines, duplicates and self-loops, 0- or 1-based ids --
    parse to the same graph as the oracle's read_graph."""
    rng = np.random.default_rng(2024)
    for case in range(60):
        mm = bool(case % 2)
        zero = bool((case // 2) % 2)
        n = int(rng.integers(1, 60))
        k = int(rng.integers(0, 120))
        lo = 0 if zero else 1
        src = rng.integers(lo, n + lo, size=k)
        dst = rng.integers(lo, n + lo, size=k)
        lines = []
        for _ in range(int(rng.integers(0, 4))):
            lines.append(rng.choice(["%", "#", "c", "p", "%%MatrixMarket x"]) + " header")
        if mm:
            lines.append(f"{n} {n} {k}")
        for a, b in zip(src.tolist(), dst.tolist()):
            sep = rng.choice([" ", "  ", "\t", " \t "])
            lines.append(f"{a}{sep}{b}" + rng.choice(["", " ", "\t"]))
            if rng.random() < 0.1:
                lines.append("")
        path = tmp_path / f"f{case}.{'mtx' if mm else 'el'}"
        path.write_text("\n".join(lines) + ("\n" if rng.random() < 0.5 else ""))
        want = oracle_mod.read_graph(str(path), mm, zero)
        ps, pd, pn = wetric_mod.parse_file(str(path), mm, zero)
        got = oracle_mod.csr_from_pairs(ps, pd, pn)
        assert pn == want.n, case
        assert np.array_equal(got.row_ptr, want.row_ptr), case
        assert np.array_equal(got.col_ind, want.col_ind), case
