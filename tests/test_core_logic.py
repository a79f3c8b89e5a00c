"""CPU restatement of the dense-core count (csrc/count_kernels.cuh:
core_row_off / core_row_first, k_core_bitmap, k_core_count, k_core_plan and
the split of a wedge range between the wedge-check kernel and the core in
csrc/count.cu), checked against the oracle's wedge-check count on random
oriented graphs, core lengths that are not multiples of 32 or 128, and
wedge ranges that cut pairs of wedges anywhere."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import random_pairs


def row_first(r):
    return (r >> 7) << 2


def row_off(H4, r):
    q, Q, R = r >> 5, r >> 7, (r >> 5) & 3
    S = 2 * Q * max(Q - 1, 0) + R * Q
    return 32 * (q * H4 - 4 * S) + (r & 31) * (H4 - 4 * Q)


def h4_of(h):
    return 4 * -(-h // 128)


@pytest.mark.parametrize("h", [1, 31, 32, 33, 127, 128, 129, 300, 1000, 4096, 32768])
def test_core_layout_rows_are_disjoint_aligned_and_hold_their_columns(h):
    """Every row starts on a 16-byte boundary, rows follow one another with
    no gap or overlap, and the word of every column c > r of row r lies in
    row r's words."""
    H4 = h4_of(h)
    rows = range(h) if h <= 4096 else list(range(0, h, 97)) + [h - 1]
    for r in rows:
        off, first = row_off(H4, r), row_first(r)
        length = H4 - first
        assert off % 4 == 0 and length % 4 == 0 and length >= 4
        assert row_off(H4, r + 1) == off + length
        for c in (r + 1, (r + h) // 2, h - 1):
            if r < c < h:
                w = off + (c >> 5) - first
                assert off <= w < off + length
    total = row_off(H4, h)
    assert total == sum(H4 - row_first(r) for r in range(h)) if h <= 4096 else True


def build_core(rp, ci, v0, h):
    """k_core_bitmap: bits of every core row (columns in (v, v0 + h))."""
    H4 = h4_of(h)
    core = np.zeros(row_off(H4, h) + 4, np.uint32)
    for r in range(h):
        v = v0 + r
        base = row_off(H4, r) - row_first(r)
        for j in range(rp[v], rp[v + 1]):
            u = int(ci[j])
            c = u - v0
            if u > v and 0 <= c < h:
                core[base + (c >> 5)] |= np.uint32(1 << (c & 31))
    return core, H4


def masked_popc(x, jj, cmin, cmax):
    lo = jj << 5
    m = 0xFFFFFFFF
    if cmin > lo:
        m = 0 if cmin >= lo + 32 else (m << (cmin - lo)) & 0xFFFFFFFF
    if cmax < lo + 32:
        m &= 0 if cmax <= lo else (0xFFFFFFFF >> (lo + 32 - cmax))
    return bin(int(x) & m).count("1")


CORE_WARPS = 8  # kCoreBlock / 32


def core_pairs(d):
    """k_core_count's split of a vertex's pairs wi in [0, d - 1): warp q
    takes groups base = q, q + 256, ...; lane p of a group sets up the pair
    base + 8p, and the group holds the lanes whose pair exists (a prefix of
    the warp: cnt = popc(ballot(wl + 1 < d))). Yields (warp, base, p, wi)."""
    for q in range(CORE_WARPS):
        base = q
        while base + 1 < d:
            valid = [base + CORE_WARPS * lane + 1 < d for lane in range(32)]
            cnt = sum(valid)
            assert valid == [True] * cnt + [False] * (32 - cnt)
            for p in range(cnt):
                yield q, base, p, base + CORE_WARPS * p
            base += 32 * CORE_WARPS


def core_count(rp, ci, core, v0, h, H4, lo, hi, exclude=frozenset()):
    """k_core_count over the active core vertices, wedges [lo, hi) only
    (vertices in `exclude` are not active: they took pair streams)."""
    n = len(rp) - 1
    deg = np.diff(rp)
    act = [v for v in range(n) if deg[v] >= 2 and v not in exclude]
    wp = [0]
    for v in act:
        wp.append(wp[-1] + int(deg[v]) * (int(deg[v]) - 1) // 2)
    total = 0
    for k, v in enumerate(act):
        if v < v0:
            continue
        P, d, rb = wp[k], int(deg[v]), int(rp[v])
        Wv = d * (d - 1) // 2
        if P + Wv <= lo or P >= hi:
            continue
        rv = np.zeros(H4, np.uint32)
        for j in range(d):
            c = int(ci[rb + j]) - v0
            if 0 <= c < h:
                rv[c >> 5] |= np.uint32(1 << (c & 31))
        whole = P >= lo and P + Wv <= hi
        for _, _, _, wi in core_pairs(d):
            cw = int(ci[rb + wi]) - v0
            if not 0 <= cw < h:
                continue
            j0 = row_first(cw)
            row = row_off(H4, cw)
            cut, cmin, cmax = False, 0, h
            if not whole:
                ps = P + wi * (d - 1) - wi * max(wi - 1, 0) // 2
                pl = d - 1 - wi
                if ps + pl <= lo or ps >= hi:
                    continue
                if ps < lo or ps + pl > hi:
                    cut = True
                    ulo = wi + 1 + (lo - ps if ps < lo else 0)
                    uhi = wi + 1 + (hi - ps if ps + pl > hi else pl)
                    cmin = int(ci[rb + ulo]) - v0
                    cmax = int(ci[rb + uhi - 1]) - v0 + 1
            for jj in range(j0, H4):
                x = int(core[row + jj - j0]) & int(rv[jj])
                total += masked_popc(x, jj, cmin, cmax) if cut else bin(x).count("1")
    return total, wp


def test_core_pairs_cover_each_pair_once():
    """Every pair of a vertex goes to exactly one (warp, group, lane), and
    the warps' shares differ by at most one group's worth of pairs per
    round (the strided split gives each warp every 8th pair)."""
    for d in list(range(0, 70)) + [255, 256, 257, 258, 300, 511, 512, 513, 1000, 2049]:
        got = sorted(wi for _, _, _, wi in core_pairs(d))
        assert got == list(range(max(d - 1, 0)))
        per_warp = [sum(1 for q, _, _, _ in core_pairs(d) if q == w) for w in range(CORE_WARPS)]
        assert max(per_warp) - min(per_warp) <= 1


def _graph(seed, n, m):
    import oracle

    src, dst = random_pairs(n, m, seed)
    # a denser top: extra edges among the last ids so the core has triangles
    rng = np.random.default_rng(seed + 1000)
    top = rng.integers(max(0, n - 200), n, size=(m // 3, 2)).astype(np.uint32)
    src = np.concatenate([src, top[:, 0]])
    dst = np.concatenate([dst, top[:, 1]])
    return oracle.oriented_from_pairs(src, dst)


@pytest.mark.parametrize("seed,n,m,h", [(1, 400, 3000, 37), (2, 600, 5000, 150),
                                         (3, 300, 6000, 300), (4, 900, 4000, 129)])
def test_core_count_with_wedge_ranges_matches_oracle(seed, n, m, h):
    """The wedge-check share [wb, min(we, Wc)) (the oracle's count stands in
    for the wedge-check kernel) plus the core share [max(wb, Wc), we) equals
    the oracle's count of [wb, we), for whole and cut ranges."""
    import oracle

    g = _graph(seed, n, m)
    rp = np.asarray(g.row_ptr, np.int64)
    ci = np.asarray(g.col_ind, np.int64)
    n = g.n
    h = min(h, n)
    v0 = n - h
    core, H4 = build_core(rp, ci, v0, h)
    W = oracle.wedge_total(g)
    deg = np.diff(rp)
    Wc = int(sum(int(d) * (int(d) - 1) // 2 for d in deg[:v0]))
    rng = np.random.default_rng(seed)
    ranges = [(0, W), (Wc, W), (0, Wc)] + [tuple(sorted(rng.integers(0, W + 1, 2)))
                                           for _ in range(12)]
    ranges += [(Wc + 1, W - 1), (Wc - 1, Wc + 2)]
    for wb, we in ranges:
        wb, we = int(max(0, wb)), int(min(W, we))
        if we <= wb:
            continue
        want = oracle.count_wedges(g, 0, wb, we)
        main = oracle.count_wedges(g, 0, wb, min(we, Wc)) if min(we, Wc) > wb else 0
        lo, hi = max(wb, Wc), we
        got_core = core_count(rp, ci, core, v0, h, H4, lo, hi)[0] if hi > lo else 0
        assert main + got_core == want, (wb, we, Wc, main, got_core, want)


# core_candidate(c) of csrc/count_kernels.cuh, largest first
CORE_CANDIDATES = [65536 - 8192 * c for c in range(5)] + [32768 >> c for c in range(1, 5)]
CORE_MIN_WEDGES, CORE_WORDS_PER_WEDGE, CORE_WORDS_PER_CHECK = 1 << 22, 2, 8.0


def core_pick(plan):
    """core_pick: the eligible candidate (enough wedges, at most 2 words per
    wedge) with the least words - 8 * wedges; the first of equal ones; -1
    for none."""
    pick, best = -1, 0.0
    for c in range(len(CORE_CANDIDATES)):
        wedges, words = plan[2 * c], plan[2 * c + 1]
        if wedges < CORE_MIN_WEDGES or words > CORE_WORDS_PER_WEDGE * wedges:
            continue
        score = float(words) - CORE_WORDS_PER_CHECK * float(wedges)
        if pick < 0 or score < best:
            pick, best = c, score
    return pick


def test_core_pick_rule():
    """The automatic core length: R-MAT scale 22's plan (wedges, words of
    the top h vertices for h = 65536 ... 2048) picks 49,152 vertices; a plan
    whose rows read more than 2 words per wedge, or with too few wedges,
    picks none; lengths that n caps to the same value tie on the first."""
    assert CORE_CANDIDATES == [65536, 57344, 49152, 40960, 32768, 16384, 8192, 4096, 2048]
    s22 = [(5.515e9, 9.475e9), (5.347e9, 7.879e9), (5.185e9, 6.516e9), (5.025e9, 5.375e9),
           (4.576e9, 3.998e9), (2.849e9, 1.072e9), (1.913e9, 3.910e8), (1.2e9, 1.0e8),
           (0.7e9, 3.0e7)]
    plan = [int(x) for pair in s22 for x in pair]
    assert CORE_CANDIDATES[core_pick(plan)] == 49152
    sparse = [int(x) for w, _ in s22 for x in (w, 3 * w)]
    assert core_pick(sparse) == -1
    assert core_pick([1000, 10] * 9) == -1
    capped = [int(x) for _ in range(9) for x in (5e6, 1e6)]
    assert core_pick(capped) == 0


def test_core_plan_candidates():
    """k_core_plan: the wedges of each candidate's top vertices are exact;
    the word estimate is at least the number of pairs."""
    import oracle

    g = _graph(7, 3000, 30000)
    rp = np.asarray(g.row_ptr, np.int64)
    n = g.n
    d = np.diff(rp)
    for hc in CORE_CANDIDATES:
        h = min(n, hc)
        top = d[n - h:]
        wedges = int((top * (top - 1) // 2).sum())
        r = np.arange(h)
        words = int((top * (h - r) // 64 + top).sum())
        assert wedges == oracle.wedge_total(oracle.CSR(
            np.concatenate([[0], np.cumsum(top)]).astype(np.uint64),
            np.zeros(int(top.sum()), np.uint32)))
        assert words >= int(top.sum())


@pytest.mark.parametrize("seed,n,m,h", [(5, 500, 6000, 200), (6, 800, 9000, 333)])
def test_core_matrix_as_bitmap(seed, n, m, h):
    """When the core covers the bitmap's rows the count checks edges (w, u)
    of core rows in the core matrix: check_wedge's word
    off(r) - first(r) + (c >> 5), bit c & 31 (r = w - v0, c = u - v0), and
    segment_hits' x = (u - w - 1) + r + 1 from the row's column-0 word,
    both give exactly the adjacency of the oriented graph."""
    g = _graph(seed, n, m)
    rp = np.asarray(g.row_ptr, np.int64)
    ci = np.asarray(g.col_ind, np.int64)
    n = g.n
    h = min(h, n)
    v0 = n - h
    core, H4 = build_core(rp, ci, v0, h)
    rng = np.random.default_rng(seed)
    for _ in range(3000):
        w = int(rng.integers(v0, n))
        u = int(rng.integers(w + 1, n + 1)) if w + 1 < n else None
        if u is None or u >= n:
            continue
        r, c = w - v0, u - v0
        word = row_off(H4, r) - row_first(r) + (c >> 5)
        bit = (int(core[word]) >> (c & 31)) & 1
        t = u - w - 1
        x = t + r + 1
        assert x == c
        want = int(u in set(ci[rp[w]:rp[w + 1]].tolist()))
        assert bit == want, (w, u)


def shell_count(rp, ci, core, v0, h, H4, v1, lo, hi):
    """k_shell_count over the active vertices in [v1, v0), wedges [lo, hi):
    each pair by a row AND (core w, when its 16-byte words are no more than
    its wedges) or by edge checks of its columns [ulo, uhi)."""
    n = len(rp) - 1
    deg = np.diff(rp)
    adj = [set(ci[rp[v]:rp[v + 1]].tolist()) for v in range(n)]
    act = [v for v in range(n) if deg[v] >= 2]
    wp = [0]
    for v in act:
        wp.append(wp[-1] + int(deg[v]) * (int(deg[v]) - 1) // 2)
    total, ands = 0, 0
    for k, v in enumerate(act):
        if not v1 <= v < v0:
            continue
        P, d, rb = wp[k], int(deg[v]), int(rp[v])
        Wv = d * (d - 1) // 2
        if P + Wv <= lo or P >= hi:
            continue
        rv = np.zeros(H4, np.uint32)
        for j in range(d):
            c = int(ci[rb + j]) - v0
            if 0 <= c < h:
                rv[c >> 5] |= np.uint32(1 << (c & 31))
        whole = P >= lo and P + Wv <= hi
        for wi in range(d - 1):
            w = int(ci[rb + wi])
            ulo, uhi, cut = wi + 1, d, False
            if not whole:
                ps = P + wi * (d - 1) - wi * max(wi - 1, 0) // 2
                pl = d - 1 - wi
                if ps + pl <= lo or ps >= hi:
                    continue
                if ps < lo or ps + pl > hi:
                    cut = True
                    ulo = wi + 1 + (lo - ps if ps < lo else 0)
                    uhi = wi + 1 + (hi - ps if ps + pl > hi else pl)
            cw = w - v0
            if 0 <= cw < h:
                j0 = row_first(cw)
                nq = (H4 - j0) >> 2
                if nq <= uhi - ulo:
                    ands += 1
                    row = row_off(H4, cw)
                    cmin = int(ci[rb + ulo]) - v0 if cut else 0
                    cmax = int(ci[rb + uhi - 1]) - v0 + 1 if cut else h
                    for jj in range(j0, H4):
                        x = int(core[row + jj - j0]) & int(rv[jj])
                        total += masked_popc(x, jj, cmin, cmax) if cut else bin(x).count("1")
                    continue
            total += sum(1 for j in range(ulo, uhi) if int(ci[rb + j]) in adj[w])
    return total, ands


@pytest.mark.parametrize("seed,n,m,h,shell", [(8, 900, 20000, 100, 300), (9, 1200, 30000, 130, 500),
                                               (10, 700, 25000, 64, 2000)])
def test_core_shell_split_matches_oracle(seed, n, m, h, shell):
    """The wedge-check share [wb, min(we, W1)), the shell's [W1, Wc) and the
    core's [Wc, W) of a range add up to the oracle's count of the range;
    some shell pairs take the row AND and some the edge checks."""
    import oracle

    g = _graph(seed, n, m)
    rp = np.asarray(g.row_ptr, np.int64)
    ci = np.asarray(g.col_ind, np.int64)
    n = g.n
    h = min(h, n)
    v0 = n - h
    v1 = max(0, v0 - shell)
    core, H4 = build_core(rp, ci, v0, h)
    W = oracle.wedge_total(g)
    deg = np.diff(rp)
    pre = lambda v: int(sum(int(d) * (int(d) - 1) // 2 for d in deg[:v]))
    Wc, W1 = pre(v0), pre(v1)
    rng = np.random.default_rng(seed)
    ranges = [(0, W), (W1, Wc), (W1 + 1, Wc - 1)] + [tuple(sorted(rng.integers(0, W + 1, 2)))
                                                     for _ in range(6)]
    total_ands = 0
    for wb, we in ranges:
        wb, we = int(wb), int(we)
        if we <= wb:
            continue
        want = oracle.count_wedges(g, 0, wb, we)
        main = oracle.count_wedges(g, 0, wb, min(we, W1)) if min(we, W1) > wb else 0
        slo, shi = max(wb, W1), min(we, Wc)
        sh, ands = shell_count(rp, ci, core, v0, h, H4, v1, slo, shi) if shi > slo else (0, 0)
        total_ands += ands
        clo = max(wb, Wc)
        co = core_count(rp, ci, core, v0, h, H4, clo, we)[0] if we > clo else 0
        assert main + sh + co == want, (wb, we, main, sh, co, want)
    assert total_ands > 0
