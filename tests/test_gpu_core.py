"""GPU parity tests of the dense-core count (k_core_bitmap + k_core_count):
with any core length -- none, chosen by the library, not a multiple of 32
or 128, larger than the graph -- every count equals the oracle's, for host
and device inputs, u32 and u64 offsets, the chunked host-input path and
wedge ranges that cut the core's pairs anywhere."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import comb3, complete_graph, random_pairs

pytestmark = pytest.mark.gpu

CORE_LENS = (None, 0, 32, 33, 100, 1000, 4096, 32768, 65536)  # None: no core


def _core(wetric_mod, c):
    return wetric_mod.CORE_OFF if c is None else c


def dense_top_graph(oracle_mod, seed, n, m, top, top_edges):
    """Random pairs plus a dense block among the last `top` ids, so the
    degree order puts a triangle-rich core at the end."""
    src, dst = random_pairs(n, m, seed)
    rng = np.random.default_rng(seed + 7)
    t = rng.integers(n - top, n, size=(top_edges, 2)).astype(np.uint32)
    src = np.concatenate([src, t[:, 0]])
    dst = np.concatenate([dst, t[:, 1]])
    return oracle_mod.oriented_from_pairs(src, dst)


@pytest.mark.parametrize("seed", range(4))
def test_core_lengths_parity(wetric_mod, oracle_mod, seed):
    rng = np.random.default_rng(300 + seed)
    n = int(rng.integers(2000, 20000))
    g = dense_top_graph(oracle_mod, seed, n, 8 * n, int(rng.integers(100, 1500)), 30 * n)
    want = oracle_mod.count_merge(g)
    W = oracle_mod.wedge_total(g)
    rp32 = g.row_ptr.astype(np.uint32)
    for c in CORE_LENS:
        for kernel in (7, 8):
            for s, a in ((5, 8192), (1, 0), (3, 96)):
                got, st = wetric_mod.count(g.row_ptr, g.col_ind, s, a, kernel=kernel,
                                           core_len=_core(wetric_mod, c))
                assert got == want, (n, c, kernel, s, a)
                assert st.wedges == W
                if c is None:
                    assert st.core_len == 0 and st.core_wedges == 0
                elif c:
                    assert st.core_len == min(c, 65536, g.n) or (c < 32 and st.core_len == 0)
        # without pair streams (which take short rows out of the core's
        # hands) the core's wedges are those of the top core_len vertices
        got, st = wetric_mod.count(rp32, g.col_ind, 5, 4096, core_len=_core(wetric_mod, c),
                                   pair_streams=False)
        assert got == want
        if st.core_len:
            d = np.diff(g.row_ptr.astype(np.int64))[g.n - st.core_len:]
            assert st.core_wedges == int((d * (d - 1) // 2).sum())


def test_core_wedge_ranges(wetric_mod, oracle_mod):
    """Ranges that start or end inside a core vertex and inside one of its
    pairs count exactly the oracle's wedges of that range."""
    g = dense_top_graph(oracle_mod, 11, 6000, 40000, 600, 120000)
    W = oracle_mod.wedge_total(g)
    want = oracle_mod.count_merge(g)
    d = np.diff(g.row_ptr.astype(np.int64))
    for c in (300, 1000, 5000):
        Wc = int((d[: g.n - c] * (d[: g.n - c] - 1) // 2).sum())
        rng = np.random.default_rng(c)
        cuts = sorted({0, W, Wc, Wc + 1, *rng.integers(Wc, W, 9).tolist(),
                       *rng.integers(0, W, 3).tolist()})
        total = 0
        for b, e in zip(cuts, cuts[1:]):
            part, st = wetric_mod.count(g.row_ptr, g.col_ind, 5, 64, wedge_begin=b,
                                        wedge_end=e, core_len=c)
            assert part == oracle_mod.count_wedges(g, 64, b, e), (c, b, e)
            assert st.wedges_counted == e - b
            total += part
        assert total == want


def test_core_covering_the_whole_graph(wetric_mod, oracle_mod):
    """A core longer than the graph holds every vertex: the wedge-check
    kernel has nothing left and the core counts everything."""
    for k in (64, 129, 700):
        g = oracle_mod.oriented_from_pairs(*complete_graph(k))
        for c in (0, k, 32768):
            got, st = wetric_mod.count(g.row_ptr, g.col_ind, 5, 64, core_len=c)
            assert got == comb3(k)
            # without pair streams the core counts every wedge
            got, st = wetric_mod.count(g.row_ptr, g.col_ind, 5, 64, core_len=c,
                                       pair_streams=False)
            assert got == comb3(k)
            if c:
                assert st.core_len == k and st.core_wedges == st.wedges


def test_core_on_rmat_auto_and_device_inputs(wetric_mod, oracle_mod):
    """On R-MAT graphs the library picks a core by itself; device and host
    inputs, one-pass launches and u64 offsets all agree with the oracle."""
    import torch

    from wetric import workloads as Wl

    for scale, seed in ((15, 3), (17, 4)):
        src, dst, _ = Wl.host_pairs(Wl.RmatSpec(scale=scale, edge_factor=16, seed=seed))
        g = oracle_mod.oriented_from_pairs(src, dst)
        want = oracle_mod.count_merge(g)
        got, st = wetric_mod.count(g.row_ptr, g.col_ind, 5, 8192)
        assert got == want and st.core_len > 0, (scale, st.core_len)
        rp_d = torch.from_numpy(g.row_ptr.view(np.int64)).cuda()
        ci_d = torch.from_numpy(g.col_ind.view(np.int32)).cuda()
        for kw in ({}, {"one_pass": True}, {"keep_u64_offsets": True},
                   {"core_len": 2048}, {"core_len": 777, "kernel": 7}):
            assert wetric_mod.count(rp_d, ci_d, 5, 8192, **kw)[0] == want, kw


def test_core_with_host_row_chunks(wetric_mod, oracle_mod):
    """A host CSR large enough for the chunked copy: the core's rows arrive
    over several chunks, and the count (whole and in wedge ranges across
    the core boundary) equals the oracle's for several core lengths."""
    src, dst = wetric_mod.gen_rmat(19, 16 << 19, seed=21)
    g = oracle_mod.oriented_from_pairs(src, dst)
    assert g.m >= 1 << 22
    want = oracle_mod.count_merge(g)
    W = oracle_mod.wedge_total(g)
    rp32 = g.row_ptr.astype(np.uint32)
    d = np.diff(g.row_ptr.astype(np.int64))
    for c in (0, 4096, 32768, None):
        got, st = wetric_mod.count(rp32, g.col_ind, 5, 8192, core_len=_core(wetric_mod, c))
        assert got == want, c
        h = st.core_len
        Wc = int((d[: g.n - h] * (d[: g.n - h] - 1) // 2).sum()) if h else W
        cuts = sorted({0, W, max(Wc - 3, 0), min(Wc + 5, W),
                       *np.random.default_rng(9).integers(0, W, 3).tolist()})
        total = 0
        for b, e in zip(cuts, cuts[1:]):
            total += wetric_mod.count(rp32, g.col_ind, 5, 8192, wedge_begin=b, wedge_end=e,
                                      core_len=_core(wetric_mod, c))[0]
        assert total == want, c


@pytest.mark.parametrize("seed", range(3))
def test_core_shell_parity(wetric_mod, oracle_mod, seed):
    """A shell below the core (the core matrix as the bitmap): every shell
    length -- none (the default), small, three times the core, reaching vertex 0 -- gives
    the oracle's count, whole and in wedge ranges across the shell's
    boundaries, and the stats report the shell's vertices and wedges."""
    rng = np.random.default_rng(600 + seed)
    n = int(rng.integers(3000, 15000))
    g = dense_top_graph(oracle_mod, 40 + seed, n, 10 * n, int(rng.integers(300, 1500)), 40 * n)
    want = oracle_mod.count_merge(g)
    W = oracle_mod.wedge_total(g)
    d = np.diff(g.row_ptr.astype(np.int64))
    pre = np.concatenate([[0], np.cumsum(d * (d - 1) // 2)])
    for core_len, shell_len in ((512, wetric_mod.CORE_OFF), (512, 0), (700, 100), (300, 10**6),
                                (2048, 1536), (512, 1536)):
        for kernel in (7, 8):
            for a in (0, 64, 256):
                got, st = wetric_mod.count(g.row_ptr, g.col_ind, 5, a, kernel=kernel,
                                           core_len=core_len, shell_len=shell_len)
                assert got == want, (core_len, shell_len, kernel, a)
                # the shell's statistics without pair streams (which take
                # short rows out of the shell's hands)
                got, st = wetric_mod.count(g.row_ptr, g.col_ind, 5, a, kernel=kernel,
                                           core_len=core_len, shell_len=shell_len,
                                           pair_streams=False)
                assert got == want, (core_len, shell_len, kernel, a)
                h = st.core_len
                assert h == min(core_len, g.n)
                want_shell = 0 if shell_len in (wetric_mod.CORE_OFF, 0) else min(
                    shell_len, g.n - h)
                assert st.shell_len == want_shell
                v0, v1 = g.n - h, g.n - h - st.shell_len
                assert st.shell_wedges == int(pre[v0] - pre[v1])
        h = min(core_len, g.n)
        v0 = g.n - h
        v1 = max(0, v0 - (0 if shell_len in (wetric_mod.CORE_OFF, 0) else shell_len))
        cuts = sorted({0, W, int(pre[v1]), int(pre[v1]) + 1, int(pre[v0]), int(pre[v0]) - 1,
                       *rng.integers(int(pre[v1]), int(pre[v0]) + 1, 5).tolist()})
        total = 0
        for b, e in zip(cuts, cuts[1:]):
            if e <= b:
                continue
            part, _ = wetric_mod.count(g.row_ptr, g.col_ind, 5, 64, wedge_begin=b, wedge_end=e,
                                       core_len=core_len, shell_len=shell_len)
            assert part == oracle_mod.count_wedges(g, 64, b, e), (core_len, shell_len, b, e)
            total += part
        assert total == want
