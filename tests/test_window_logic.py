"""CPU restatement of the warp-staged kernel's index logic
(csrc/count_kernels.cuh, k_count_staged): the 32-entry vertex window, the
5-step shuffle search and the cursor advance between rounds. Checks on
degree sequences with many one-wedge vertices that every lane finds the
vertex owning its wedge and that the cursor always starts the next round on
the right vertex."""
from __future__ import annotations

import numpy as np
import pytest


def active_prefix(deg):
    d = np.asarray(deg, np.int64)
    d = d[d >= 2]
    wp = np.zeros(len(d) + 1, np.int64)
    wp[1:] = np.cumsum(d * (d - 1) // 2)
    return wp, len(d)


def simulate(deg, spread, wb=0, we=None):
    wp, K = active_prefix(deg)
    W = int(wp[-1])
    we = W if we is None else we
    G = 256 * spread
    tiles = -(-(we - wb) // G) if we > wb else 0
    INF = np.iinfo(np.int64).max

    owner_of = np.repeat(np.arange(K), np.diff(wp))

    def owner(i):
        return int(owner_of[i])

    for t in range(tiles):
        base = wb + t * G
        end = min(base + G, we)
        kcur = owner(base)  # k_tile_map
        while base < end:
            E = [int(wp[kcur + l]) if kcur + l <= K else INF for l in range(32)]
            for lane in range(32):
                i = base + lane
                if i >= end:
                    continue
                j = 0
                for step in (16, 8, 4, 2, 1):
                    if E[j + step] <= i:
                        j += step
                assert kcur + j == owner(i), (t, base, lane)
                assert 0 <= i - E[j] < int(wp[kcur + j + 1] - wp[kcur + j])
            # cursor advance (lane 31's j, then the entry after it)
            i31 = base + 31
            j31 = 0
            for step in (16, 8, 4, 2, 1):
                if E[j31 + step] <= i31:
                    j31 += step
            E32 = int(wp[kcur + 32]) if kcur + 32 <= K else INF
            e_next = E[j31 + 1] if j31 < 31 else E32
            kcur += j31 + (1 if e_next <= base + 32 else 0)
            base += 32
            if base < end:
                assert kcur == owner(base), (t, base)
    return W


@pytest.mark.parametrize("seed", range(6))
def test_window_on_one_wedge_vertices(seed):
    rng = np.random.default_rng(seed)
    # long runs of d = 2 (one wedge each), mixed with hubs and d < 2
    deg = rng.choice([0, 1, 2, 2, 2, 2, 3, 9, 40], size=1500)
    for s in (1, 2, 5):
        simulate(deg, s)


def test_window_all_one_wedge():
    simulate(np.full(3000, 2), 1)
    simulate(np.full(3000, 2), 3)


def test_window_ranges():
    rng = np.random.default_rng(9)
    deg = rng.choice([2, 2, 3, 5, 30], size=800)
    W = simulate(deg, 1)
    for wb, we in ((0, W), (17, W - 5), (W // 3, 2 * W // 3), (W - 1, W)):
        simulate(deg, 2, wb, we)


# ------------------------------------------------- whole-kernel emulation

STAGE_CAP = 1024


def _isqrt_kernel(x: int) -> int:
    """isqrt64 of csrc/count_kernels.cuh: float/double estimate plus two
    bounded corrections each way."""
    import math

    y = int(math.sqrt(float(x)))
    y = min(y, 0xFFFFFFFF)
    for _ in range(2):
        y -= 1 if y * y > x else 0
    for _ in range(2):
        y += 1 if (y + 1) * (y + 1) <= x else 0
    return y


def _decode(iv, d):
    W = d * (d - 1) // 2
    if d < 2 or iv >= W:
        return None
    j = W - 1 - iv
    q = (_isqrt_kernel(8 * j + 1) - 1) >> 1
    p = j - q * (q + 1) // 2
    if q > d - 2 or p > q:
        return None
    return d - 2 - q, d - 1 - p


def emulate_staged(rp, ci, s, a, wb=0, we=None):
    """Counts like k_count_staged (single graph): tiles of 256*s wedges per
    warp, rounds of 32 lanes, bitmap for w in the last a ids, N+(w) of the
    last searching lane staged when d+(w) <= 1024, global search otherwise."""
    n = len(rp) - 1
    d_all = np.diff(rp).astype(np.int64)
    act = np.nonzero(d_all >= 2)[0]
    K = len(act)
    wp = np.zeros(K + 1, np.int64)
    wp[1:] = np.cumsum(d_all[act] * (d_all[act] - 1) // 2)
    W = int(wp[-1])
    we = W if we is None else min(we, W)
    if we <= wb:
        return 0
    owner_of = np.repeat(np.arange(K), np.diff(wp))
    S = a * (a - 1) // 2 if a else 0
    bm_first = max(n, a) - a
    edges = set()
    for v in range(n):
        for x in ci[rp[v]:rp[v + 1]]:
            edges.add((v, int(x)))
    G = 256 * s
    tiles = -(-(we - wb) // G)
    INF = 1 << 62
    total = 0
    for t in range(tiles):
        staged, staged_row = None, None
        base = wb + t * G
        end = min(base + G, we)
        kcur = int(owner_of[base])
        while base < end:
            E = [int(wp[kcur + l]) if kcur + l <= K else INF for l in range(32)]
            lanes = []
            for lane in range(32):
                i = base + lane
                j = 0
                for step in (16, 8, 4, 2, 1):
                    if E[j + step] <= i:
                        j += step
                lanes.append((i, j))
            j31 = lanes[31][1]
            E32 = int(wp[kcur + 32]) if kcur + 32 <= K else INF
            e_next = E[j31 + 1] if j31 < 31 else E32
            wu = []
            for i, j in lanes:
                if i >= end:
                    wu.append(None)
                    continue
                k = kcur + j
                v = int(act[k]) if k < K else 0
                dec = _decode(i - E[j], int(d_all[v])) if k < K and E[j] <= i else None
                assert dec is not None, "window logic gave a lane no wedge"
                wi, ui = dec
                wu.append((int(ci[rp[v] + wi]), int(ci[rp[v] + ui])))
            kcur += j31 + (1 if e_next <= base + 32 else 0)
            is_bm = [x is not None and x[0] >= bm_first for x in wu]
            is_srch = [x is not None and not b and x[0] < n for x, b in zip(wu, is_bm)]
            if any(is_srch):
                src = max(l for l in range(32) if is_srch[l])
                wc = wu[src][0]
                if wc != staged:
                    dw = int(rp[wc + 1] - rp[wc])
                    if dw <= STAGE_CAP:
                        staged, staged_row = wc, ci[rp[wc]:rp[wc + 1]]
            for l in range(32):
                if wu[l] is None:
                    continue
                w, u = wu[l]
                if is_bm[l]:
                    hit = u > w and u < n and (w, u) in edges
                elif is_srch[l]:
                    row = staged_row if w == staged else ci[rp[w]:rp[w + 1]]
                    hit = u in set(row.tolist())
                else:
                    hit = False
                total += int(hit)
            base += 32
    return total


@pytest.mark.parametrize("seed", range(4))
def test_staged_kernel_emulation_matches_oracle(seed):
    import oracle
    from conftest import random_pairs

    rng = np.random.default_rng(seed)
    n = int(rng.integers(30, 400))
    src, dst = random_pairs(n, int(rng.integers(n, 6 * n)), 500 + seed)
    g = oracle.oriented_from_pairs(src, dst)
    want = oracle.count_merge(g)
    W = oracle.wedge_total(g)
    for s, a in ((1, 0), (2, 64), (1, 4096)):
        assert emulate_staged(g.row_ptr.astype(np.int64), g.col_ind, s, a) == want
    cut = W // 3
    parts = (emulate_staged(g.row_ptr.astype(np.int64), g.col_ind, 1, 64, 0, cut)
             + emulate_staged(g.row_ptr.astype(np.int64), g.col_ind, 1, 64, cut, W))
    assert parts == want


def test_staged_kernel_emulation_one_wedge_vertices():
    """Many vertices with exactly one wedge: a star forest of 2-paths plus
    triangles (each triangle's lowest vertex has d+ = 2)."""
    import oracle

    tri = np.arange(0, 900, 3, dtype=np.uint32)
    src = np.concatenate([tri, tri + 1, tri])
    dst = np.concatenate([tri + 1, tri + 2, tri + 2])
    g = oracle.oriented_from_pairs(src, dst)
    assert emulate_staged(g.row_ptr.astype(np.int64), g.col_ind, 1, 0) == 300
    assert emulate_staged(g.row_ptr.astype(np.int64), g.col_ind, 2, 64) == 300


def emulate_rows(rp, ci, s, a, wb=0, we=None, stats=None, segs=False):
    """Counts like k_count_rows (single graph): warp-uniform (k, w_i, u_i)
    walked in rounds of 32; fast rounds inside rows w_i and w_i + 1, general
    rounds with the vertex window and per-lane decode; with segs, the
    long-row segments of kSegs (whole rounds inside row w_i, row-uniform
    check of segment_hits over the rest of the row or tile) come first
    whenever 16 or more wedges are left in the row."""
    n = len(rp) - 1
    d_all = np.diff(rp).astype(np.int64)
    act = np.nonzero(d_all >= 2)[0]
    K = len(act)
    wp = np.zeros(K + 1, np.int64)
    wp[1:] = np.cumsum(d_all[act] * (d_all[act] - 1) // 2)
    W = int(wp[-1])
    we = W if we is None else min(we, W)
    if we <= wb:
        return 0
    S = a * (a - 1) // 2 if a else 0
    bm_first = max(n, a) - a
    rows = {v: set(ci[rp[v]:rp[v + 1]].tolist()) for v in range(n)}
    owner_of = np.repeat(np.arange(K), np.diff(wp))
    G = 256 * s
    tiles = -(-(we - wb) // G)
    INF = 1 << 62
    total = 0
    fast = general = segments = 0

    def check(w, u):
        if w >= bm_first:
            return u > w and u < n and u in rows[w]
        return w < n and u in rows[w]

    for t in range(tiles):
        base = wb + t * G
        end = min(base + G, we)
        kcur = int(owner_of[base])
        rb, d = int(rp[act[kcur]]), int(d_all[act[kcur]])
        dec = _decode(base - int(wp[kcur]), d)
        assert dec is not None
        wi, ui = dec
        while base < end:
            if segs and d - ui >= 16:
                segments += 1
                nseg = min(end - base, d - ui)
                assert nseg >= 1
                w = int(ci[rb + wi])
                for k in range(nseg):
                    assert _decode(base + k - int(wp[kcur]), d) == (wi, ui + k)
                for k in range(nseg):
                    total += int(_segment_check(w, int(ci[rb + ui + k]), n,
                                                bm_first, rows))
                base += nseg
                ui += nseg
                if ui == d:
                    wi += 1
                    ui = wi + 1
                    assert ui < d
                if base < end:
                    assert kcur == owner_of[base]
                    assert _decode(base - int(wp[kcur]), d) == (wi, ui)
                continue
            n_round = min(32, end - base)
            rem0 = d - ui
            len1 = d - wi - 2 if wi + 2 < d else 0
            wu = [None] * 32
            if n_round <= rem0 + len1:
                fast += 1
                for lane in range(n_round):
                    in1 = lane >= rem0
                    my_ui = wi + 2 + (lane - rem0) if in1 else ui + lane
                    my_wi = wi + 1 if in1 else wi
                    assert my_ui < d and my_wi < my_ui
                    wu[lane] = (int(ci[rb + my_wi]), int(ci[rb + my_ui]))
                    # the lane's wedge index must be base + lane
                    v = act[owner_of[base + lane]]
                    assert v == act[kcur]
                    assert _decode(base + lane - int(wp[kcur]), d) == (my_wi, my_ui)
                if n_round < rem0:
                    ui += n_round
                else:
                    c1 = n_round - rem0
                    if c1 < len1:
                        wi += 1
                        ui = wi + 1 + c1
                    elif wi + 3 < d:
                        wi += 2
                        ui = wi + 1
                    elif base + n_round < end:
                        kcur += 1
                        rb, d = int(rp[act[kcur]]), int(d_all[act[kcur]])
                        wi, ui = 0, 1
            else:
                general += 1
                E = [int(wp[kcur + l]) if kcur + l <= K else INF for l in range(32)]
                # prefix entries relative to base, saturated to 32 bits
                Er = [0 if e <= base else min(e - base, 0xFFFFFFFF) for e in E]
                js = []
                for lane in range(32):
                    i = base + lane
                    j = 0
                    for step in (16, 8, 4, 2, 1):
                        if Er[j + step] <= lane:
                            j += step
                    js.append(j)
                    if lane < n_round:
                        k = kcur + j
                        v = int(act[k])
                        dec = _decode(i - E[j], int(d_all[v]))
                        assert dec is not None
                        wu[lane] = (int(ci[rp[v] + dec[0]]), int(ci[rp[v] + dec[1]]))
                j31 = js[31]
                if base + n_round < end:
                    # successor of lane 31's wedge (vertex kcur + j31)
                    v31 = int(act[kcur + j31])
                    d31 = int(d_all[v31])
                    w31, u31 = _decode(base + 31 - E[j31], d31)
                    adv = j31
                    if u31 + 1 < d31:
                        wi, ui = w31, u31 + 1
                    elif w31 + 2 < d31:
                        wi, ui = w31 + 1, w31 + 2
                    else:
                        wi, ui = 0, 1
                        adv = j31 + 1
                    kcur += adv
                    rb, d = int(rp[act[kcur]]), int(d_all[act[kcur]])
            for x in wu:
                if x is not None:
                    total += int(check(*x))
            base += n_round
            if base < end:
                assert kcur == owner_of[base]
                assert _decode(base - int(wp[kcur]), d) == (wi, ui)
    if stats is not None:
        stats.update(fast=fast, general=general, segments=segments)
    return total


def _segment_check(w, u, n, bm_first, rows):
    """segment_hits for one lane: the bitmap row of w through the row-local
    bit offset t = u - w - 1 < n - w - 1 (u32 wrap for u <= w), else
    membership in N+(w)."""
    if w >= n:
        return False
    if w >= bm_first:
        t = (u - w - 1) & 0xFFFFFFFF
        return t < n - w - 1 and u in rows[w]
    return u in rows[w]


@pytest.mark.parametrize("seed", range(4))
def test_rows_kernel_emulation_matches_oracle(seed):
    import oracle
    from conftest import random_pairs

    rng = np.random.default_rng(seed)
    n = int(rng.integers(30, 400))
    src, dst = random_pairs(n, int(rng.integers(n, 8 * n)), 700 + seed)
    g = oracle.oriented_from_pairs(src, dst)
    want = oracle.count_merge(g)
    W = oracle.wedge_total(g)
    rp = g.row_ptr.astype(np.int64)
    for s, a in ((1, 0), (2, 64), (1, 4096)):
        assert emulate_rows(rp, g.col_ind, s, a) == want
    cuts = sorted({0, W, W // 3, W // 2 + 7})
    assert sum(emulate_rows(rp, g.col_ind, 1, 64, b, e)
               for b, e in zip(cuts, cuts[1:]) if e > b) == want


def test_rows_kernel_emulation_long_rows_and_one_wedge_vertices():
    import oracle
    from conftest import complete_graph

    # K_70 (long rows: fast rounds) + 300 disjoint triangles (one-wedge
    # vertices: general rounds), in one graph
    s1, d1 = complete_graph(70)
    tri = np.arange(100, 1000, 3, dtype=np.uint32)
    src = np.concatenate([s1, tri, tri + 1, tri])
    dst = np.concatenate([d1, tri + 1, tri + 2, tri + 2])
    g = oracle.oriented_from_pairs(src, dst)
    want = oracle.count_merge(g)
    st = {}
    assert emulate_rows(g.row_ptr.astype(np.int64), g.col_ind, 1, 0, stats=st) == want
    assert st["fast"] > 0 and st["general"] > 0
    assert emulate_rows(g.row_ptr.astype(np.int64), g.col_ind, 3, 64) == want


@pytest.mark.parametrize("seed", range(3))
def test_rows_kernel_segments_emulation(seed):
    """kSegs: long-row segments, then fast and general rounds for the rest;
    every wedge is visited once in order, over whole graphs and wedge
    ranges, with and without the bitmap."""
    import oracle
    from conftest import complete_graph, random_pairs

    rng = np.random.default_rng(40 + seed)
    s1, d1 = complete_graph(int(rng.integers(40, 90)))
    s2, d2 = random_pairs(600, 9000, 900 + seed)
    s2 = s2 + 200
    d2 = d2 + 200
    tri = np.arange(1000, 1600, 3, dtype=np.uint32)
    src = np.concatenate([s1, s2, tri, tri + 1, tri])
    dst = np.concatenate([d1, d2, tri + 1, tri + 2, tri + 2])
    g = oracle.oriented_from_pairs(src, dst)
    want = oracle.count_merge(g)
    W = oracle.wedge_total(g)
    rp = g.row_ptr.astype(np.int64)
    for s, a in ((1, 0), (2, 64), (5, 4096)):
        st = {}
        assert emulate_rows(rp, g.col_ind, s, a, stats=st, segs=True) == want
        assert st["segments"] > 0 and st["fast"] > 0 and st["general"] > 0
    cuts = sorted({0, W, W // 5, W // 2 + 13, W - 33})
    assert sum(emulate_rows(rp, g.col_ind, 1, 64, b, e, segs=True)
               for b, e in zip(cuts, cuts[1:]) if e > b) == want


# ------------------------------------------------ 32-bit decode path


def _isqrt_small(j, rel_err):
    """isqrt_small (csrc/count_kernels.cuh) with the approximate square
    root modelled as float32 sqrt times (1 + rel_err)."""
    f = np.float32(np.float32(8.0) * np.float32(j) + np.float32(1.0))
    r = np.float32(np.sqrt(f, dtype=np.float32) * np.float32(1.0 + rel_err))
    y = int(r)
    x = 8 * j + 1
    if y * y > x:
        y -= 1
    if (y + 1) * (y + 1) <= x:
        y += 1
    return y


def test_isqrt_small_exact_under_sqrt_error():
    """floor(sqrt(8j + 1)) for j below C(2^16, 2) (vertices with d < 2^16),
    with the square root off by up to 2^-21 relative either way (the bound
    the kernel relies on is below 2^-22)."""
    import math

    top = (65535 * 65534) // 2
    rng = np.random.default_rng(9)
    js = np.concatenate([np.arange(0, 5000), rng.integers(0, top, 20000)])
    # values of j next to perfect squares, where the floor changes
    ks = rng.integers(1, 1 << 17, 5000)
    near = np.concatenate([(ks * ks - 1) // 8 + o for o in (-1, 0, 1)])
    js = np.concatenate([js, near[(near >= 0) & (near < top)]])
    for j in js.tolist():
        want = math.isqrt(8 * j + 1)
        for e in (-2.0 ** -21, 0.0, 2.0 ** -21):
            assert _isqrt_small(j, e) == want, (j, e)


# ------------------------------------------------ per-row hash set logic

HASH_BUCKET = 8
EMPTY = 0xFFFFFFFF


def _buckets_for(d, min_degree, keys_per_bucket):
    return 0 if d < min_degree or d == 0 else -(-d // keys_per_bucket)


def _bucket(x, nbk):
    return (((x * 2654435761) & 0xFFFFFFFF) * nbk) >> 32


def _fill(b):
    f = 0
    while f < HASH_BUCKET and b[f] != EMPTY:
        f += 1
    return f


def _warp_build(row, nbk):
    """k_hash_build for one row: rounds of 32 columns; lanes sharing a
    bucket take slots fill + rank; lanes past a full bucket continue one at
    a time (lowest lane first) into the following buckets."""
    tab = [[EMPTY] * HASH_BUCKET for _ in range(nbk)]
    for j0 in range(0, len(row), 32):
        xs = [int(x) for x in row[j0:j0 + 32]]
        bks = [_bucket(x, nbk) for x in xs]
        fills = {b: _fill(tab[b]) for b in set(bks)}
        slots = []
        for lane, b in enumerate(bks):
            rank = sum(1 for q in bks[:lane] if q == b)
            slots.append(fills[b] + rank)
        for x, b, sl in zip(xs, bks, slots):
            if sl < HASH_BUCKET:
                assert tab[b][sl] == EMPTY
                tab[b][sl] = x
        for x, b, sl in zip(xs, bks, slots):
            if sl >= HASH_BUCKET:
                for _ in range(1, nbk):
                    b = 0 if b + 1 == nbk else b + 1
                    f = _fill(tab[b])
                    if f < HASH_BUCKET:
                        tab[b][f] = x
                        break
                else:
                    raise AssertionError("table full")
    return tab


def _contains(tab, u):
    """hash_contains: first bucket, then the following ones while full."""
    nbk = len(tab)
    bk = _bucket(u, nbk)
    for _ in range(nbk):
        b = tab[bk]
        if u in b:
            return True
        if b[-1] == EMPTY:
            return False
        bk = 0 if bk + 1 == nbk else bk + 1
    return False


@pytest.mark.parametrize("min_degree,keys_per_bucket", [(32, 2), (64, 3), (1, 8)])
def test_hash_sets_membership(min_degree, keys_per_bucket):
    """Restates k_hash_build / hash_contains (csrc/count_kernels.cuh) for the
    single-graph sizing (32, 2), the batch sizing (64, 3) and the densest
    legal one (8 columns per bucket): every column is found, no other id is,
    slots fill in order, and no column sits past a bucket with a free slot."""
    rng = np.random.default_rng(3)
    for d in (1, 16, 31, 32, 33, 64, 100, 513, 2000):
        nbk = _buckets_for(d, min_degree, keys_per_bucket)
        if nbk == 0:
            assert d < min_degree
            continue
        # ids drawn from a narrow range too, so buckets collide heavily
        hi = (1 << 31) if d % 2 else 4 * d
        row = np.sort(rng.choice(hi, size=d, replace=False)).astype(np.int64)
        tab = _warp_build(row, nbk)
        for b in tab:
            f = _fill(b)
            assert all(x == EMPTY for x in b[f:])
        members = set(row.tolist())
        assert sum(_fill(b) for b in tab) == d
        for x in row.tolist():
            assert _contains(tab, x)
        for u in rng.integers(0, hi, size=2000).tolist():
            assert _contains(tab, u) == (u in members)


def _pack16(bucket):
    """A near bucket's 8 16-bit slots as the 4 words one 16-byte load gives
    (slot 2i in the low half of word i), empty slots 0xFFFF."""
    h = [0xFFFF if x == EMPTY else int(x) for x in bucket]
    return [h[2 * i] | (h[2 * i + 1] << 16) for i in range(4)]


def _bucket16_has(words, t):
    """bucket16_has: a 16-bit half of y = word ^ (t * 0x10001) is zero iff
    (y - 0x10001) & ~y & 0x80008000 is non-zero."""
    kk = (t * 0x10001) & 0xFFFFFFFF
    z = 0
    for w in words:
        y = w ^ kk
        z |= ((y - 0x10001) & 0xFFFFFFFF) & (~y & 0xFFFFFFFF)
    return (z & 0x80008000) != 0


def _near_contains(tab, t):
    nbk = len(tab)
    bk = _bucket(t, nbk)
    for _ in range(nbk):
        words = _pack16(tab[bk])
        if _bucket16_has(words, t):
            return True
        if (words[3] >> 16) == 0xFFFF:
            return False
        bk = 0 if bk + 1 == nbk else bk + 1
    return False


def test_bucket16_compare_exact():
    """The packed compare against every slot position, key values at the
    ends of the 16-bit range and words whose halves differ by one."""
    rng = np.random.default_rng(11)
    for _ in range(3000):
        slots = rng.integers(0, 65535, size=8).tolist()
        nfill = int(rng.integers(0, 9))
        b = slots[:nfill] + [EMPTY] * (8 - nfill)
        words = _pack16(b)
        for t in [0, 1, 65534, int(rng.integers(0, 65535))] + slots[:nfill] + \
                [(x + 1) % 65535 for x in slots[:nfill]] + [max(x - 1, 0) for x in slots[:nfill]]:
            assert _bucket16_has(words, t) == (t in slots[:nfill])


def test_near_sets_membership():
    """k_near_build / near_contains (csrc/count_kernels.cuh): rows with
    n - v <= 65536 store u - v - 1 as 16-bit keys, 8 slots per bucket,
    three keys per bucket on average; every column is found, no other id
    in (v, n) is, and ids outside (v, n) are rejected before the lookup."""
    rng = np.random.default_rng(5)
    n = 1 << 20
    for span, d in ((65536, 16), (65536, 700), (40000, 3000), (2000, 1999), (100, 40)):
        v = n - span
        row = np.sort(rng.choice(np.arange(v + 1, n), size=d, replace=False)).astype(np.int64)
        keys = (row - v - 1).tolist()
        assert max(keys) <= 65534
        nbk = _buckets_for(d, 16, 3)
        tab = _warp_build(keys, nbk)
        lim = n - v - 1
        members = set(row.tolist())
        for u in row.tolist():
            assert _near_contains(tab, u - v - 1)
        for u in rng.integers(v + 1, n, size=3000).tolist():
            assert _near_contains(tab, u - v - 1) == (u in members)
        for u in (v, v - 1, n, n + 5):
            t = (u - v - 1) & 0xFFFFFFFF
            assert t >= lim  # the lookup's range test rejects these


def _chunk_rows(rp, m, tops=(1, 4, 8, 16, 32, 48)):
    """The row chunks a host-input count copies (csrc/api.cu,
    column_chunks): highest rows first, each starting at the first row whose
    columns begin at or after the top t/64 of the columns, t in `tops`; the
    last chunk starts at row 0."""
    n = len(rp) - 1
    out, prev = [], n
    for t in tops:
        target = m - m * t // 64
        lo = int(np.searchsorted(rp[:prev], target, side="left"))
        if 0 < lo < prev:
            out.append(lo)
            prev = lo
    out.append(0)
    return out


@pytest.mark.parametrize("seed", range(3))
def test_row_chunks_partition_the_wedges(seed):
    """Wedge order is vertex order, so the chunks' vertex ranges map to
    contiguous wedge ranges [P(lo), P(hi)); counting each chunk's range
    (clipped to a requested wedge range) gives the whole count, and every
    edge check of a chunk reads only rows at or above its first row."""
    import oracle
    from conftest import random_pairs

    src, dst = random_pairs(3000, 60000, 300 + seed)
    g = oracle.oriented_from_pairs(src, dst)
    rp = g.row_ptr.astype(np.int64)
    ci = g.col_ind.astype(np.int64)
    n, m = len(rp) - 1, int(rp[-1])
    d = np.diff(rp)
    P = np.zeros(n + 1, np.int64)
    P[1:] = np.cumsum(d * (d - 1) // 2)
    W = int(P[-1])
    want = oracle.count_merge(g)
    los = _chunk_rows(rp, m)
    assert los[-1] == 0 and all(a > b for a, b in zip(los, los[1:]))
    his = [n] + los[:-1]
    for lo, hi in zip(los, his):
        # columns of rows >= lo are > lo: the chunk's checks stay above it
        assert (ci[rp[lo]:] > lo).all() if rp[lo] < m else True
    for wb, we in ((0, W), (W // 7, W - W // 5)):
        total = 0
        for lo, hi in zip(los, his):
            cb, ce = max(P[lo], wb), min(P[hi], we)
            if ce > cb:
                total += oracle.count_wedges(g, 64, int(cb), int(ce))
        assert total == (want if (wb, we) == (0, W) else oracle.count_wedges(g, 64, wb, we))


def _near_segment_ks(lane, nseg):
    """The columns k one lane probes in segment_hits' near-set loop: three
    rounds at a time (k, k + 32, k + 64 while k + 64 < nseg), then one."""
    ks, k = [], lane
    while k + 64 < nseg:
        ks += [k, k + 32, k + 64]
        k += 96
    while k < nseg:
        ks.append(k)
        k += 32
    return ks


def _far_segment_ks(lane, nseg):
    """The 32-bit hash-set loop: two rounds at a time, then at most one."""
    ks, k = [], lane
    while k + 32 < nseg:
        ks += [k, k + 32]
        k += 64
    if k < nseg:
        ks.append(k)
    return ks


def test_segment_loops_visit_every_column_once():
    """Over a warp, the near (three in flight) and far (two in flight)
    segment loops probe each of the segment's nseg columns exactly once."""
    for nseg in range(1, 400):
        for fn in (_near_segment_ks, _far_segment_ks):
            seen = sorted(k for lane in range(32) for k in fn(lane, nseg))
            assert seen == list(range(nseg)), (fn.__name__, nseg)
