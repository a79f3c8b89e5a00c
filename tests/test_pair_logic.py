"""CPU restatement of the pair streams for short rows
(csrc/pair_streams.cuh: pair_budget, k_pair_plan, k_count_pairs with its
warp-wide search from stream positions to pairs, and the split of the
vertices between the pair streams and the wedge check in csrc/count.cu),
checked against the oracle's per-vertex merge counts on random graphs, with
tiles that cut vertices anywhere."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import random_pairs

MAX_DEG, VERTEX_COST, ROUND_COST, WEDGE_COST, SEG_WEDGE_COST, SEG_MIN = 64, 160, 30, 7, 2, 16
INF = 0xFFFFFFFF


def pair_budget(d):
    """Wedges of row tails shorter than a segment at WEDGE_COST, the rest at
    SEG_WEDGE_COST, against VERTEX_COST + ROUND_COST per 32 columns."""
    if d < 2 or d > MAX_DEG:
        return 0
    t = min(d - 1, SEG_MIN - 1)
    short_w, all_w = t * (t + 1) // 2, d * (d - 1) // 2
    wc = WEDGE_COST * short_w + SEG_WEDGE_COST * (all_w - short_w)
    return 0 if wc <= VERTEX_COST else (wc - VERTEX_COST) * 32 // ROUND_COST


def pair_plan(rp, ci, v_end):
    """k_pair_plan: (pair vertices, their stream lengths R, their wedges)."""
    pv, R, W = [], [], 0
    for v in range(v_end):
        b, d = int(rp[v]), int(rp[v + 1] - rp[v])
        budget = pair_budget(d)
        if not budget:
            continue
        r = 0
        for j in range(d - 1):
            if r > budget:
                break
            u = int(ci[b + j])
            r += int(rp[u + 1] - rp[u])
        if r <= budget:
            pv.append(v)
            R.append(r)
            W += d * (d - 1) // 2
    return pv, R, W


def popc(x):
    return bin(x & 0xFFFFFFFF).count("1")


def vertex_rounds(rp, ci, v, q0, q1):
    """The rounds of k_count_pairs for positions [q0, q1) of v's stream,
    lane by lane, with the warp's search (ballot counts of the starts
    before the round, OR of the starts inside it)."""
    b, d = int(rp[v]), int(rp[v + 1] - rp[v])
    u = [int(x) for x in ci[b:b + d]]
    vset = set(u)
    row, length = [0] * 64, [0] * 64
    for i in range(d - 1):
        row[i] = int(rp[u[i]])
        length[i] = int(rp[u[i] + 1]) - row[i]
    # compacted entries with columns, their starts (exclusive prefix)
    erow, estart, pos = [], [], 0
    for i in range(64):
        if length[i]:
            erow.append(row[i])
            estart.append(pos)
        pos += length[i]
    ne = len(erow)
    c = [estart[e] if e < ne else INF for e in range(64)]
    # column index of stream position 0 of each entry, mod 2^32
    eoff = [(erow[e] - estart[e]) & 0xFFFFFFFF for e in range(ne)]
    hits = 0
    # entries starting before the first round, then carried round to round
    before = sum(1 for e in range(64) if c[e] < q0)
    for base in range(q0, q1, 32):
        assert before == sum(1 for e in range(64) if c[e] < base)
        starts = 0
        for e in range(64):
            if 0 <= c[e] - base < 32:
                starts |= 1 << (c[e] - base)
        for lane in range(32):
            q = base + lane
            if q >= q1:
                continue
            e = before + popc(starts & (0xFFFFFFFF >> (31 - lane))) - 1
            assert 0 <= e < ne and estart[e] <= q
            x = int(ci[(eoff[e] + q) & 0xFFFFFFFF])
            hits += x in vset
        before += popc(starts)
    return hits


def pair_count(rp, ci, pv, R, T):
    """k_count_pairs over tiles of T streamed columns: every tile walks the
    vertices its range touches (from its tile_k entry)."""
    ps = np.concatenate([[0], np.cumsum(R)]).astype(np.int64)
    total_R = int(ps[-1])
    total = 0
    tiles = -(-total_R // T)
    for t in range(tiles):
        tb, te = t * T, min(t * T + T, total_R)
        k = int(np.searchsorted(ps[:len(pv)], tb, side="right")) - 1  # k_tile_map
        while k < len(pv):
            s0, s1 = int(ps[k]), int(ps[k + 1])
            if s0 >= te:
                break
            if s1 > tb and s1 != s0:
                total += vertex_rounds(rp, ci, pv[k], max(tb - s0, 0), min(te, s1) - s0)
            k += 1
    return total


def _graph(kind, seed, n, m):
    import oracle

    if kind == "er":
        src, dst = random_pairs(n, m, seed)
    else:  # mild power law: a few hubs
        rng = np.random.default_rng(seed)
        w = (1.0 + np.arange(n) / 20.0) ** -0.7
        p = w / w.sum()
        src = rng.choice(n, m, p=p).astype(np.uint32)
        dst = rng.choice(n, m, p=p).astype(np.uint32)
    return oracle.oriented_from_pairs(src, dst)


def test_pair_budget_rule():
    # seven columns (21 wedges, 147 instructions) never pay for the setup
    assert [pair_budget(d) for d in (0, 1, 2, 4, 5, 6, 7, 65)] == [0] * 8
    assert pair_budget(8) == (7 * 28 - 160) * 32 // 30
    # 64 columns: 120 wedges in tails below 16, 1896 in segment tails
    assert pair_budget(64) == (7 * 120 + 2 * 1896 - 160) * 32 // 30
    # the budget grows with the wedges it replaces
    assert all(pair_budget(d) < pair_budget(d + 1) for d in range(8, 64))


@pytest.mark.parametrize("kind,seed,n,m", [("er", 1, 400, 6000), ("er", 2, 1500, 30000),
                                           ("skew", 3, 800, 12000), ("skew", 4, 300, 9000)])
@pytest.mark.parametrize("T", [32, 256, 2048])
def test_pair_streams_match_oracle_per_vertex(kind, seed, n, m, T):
    """The pair streams' hits equal the oracle's merge count of the pair
    vertices, for tiles that start and end inside vertices; with the rest
    of the vertices to the wedge check, every vertex is counted once."""
    import oracle

    g = _graph(kind, seed, n, m)
    rp, ci = np.asarray(g.row_ptr, np.int64), np.asarray(g.col_ind, np.int64)
    nv = len(rp) - 1
    pv, R, W = pair_plan(rp, ci, nv)
    assert pv, "the graph should have short rows that take pair streams"
    got = pair_count(rp, ci, pv, R, T)
    want = sum(oracle.count_merge_range(g, v, v + 1) for v in pv)
    assert got == want
    assert W == sum(int(rp[v + 1] - rp[v]) * int(rp[v + 1] - rp[v] - 1) // 2 for v in pv)


def test_pair_plan_takes_short_rows_only():
    """Rows with more than 64 columns, or too few wedges to pay for the
    setup, never take pair streams."""
    g = _graph("er", 7, 600, 20000)
    rp, ci = np.asarray(g.row_ptr, np.int64), np.asarray(g.col_ind, np.int64)
    nv = len(rp) - 1
    pv, _, _ = pair_plan(rp, ci, nv)
    assert pv
    assert all(8 <= rp[v + 1] - rp[v] <= 64 for v in pv)


@pytest.mark.parametrize("seed,n,m,h", [(11, 500, 9000, 200), (12, 400, 12000, 400)])
def test_pair_vertices_inside_the_core_are_counted_once(seed, n, m, h):
    """Pair vertices leave the active set, so the core's blocks (one per
    active core vertex) skip them and the pair streams count them: the
    core's count over the remaining core vertices plus the pair streams plus
    the wedge checks of the rest equals the oracle's count."""
    import oracle
    from test_core_logic import build_core, core_count

    g = _graph("er", seed, n, m)
    rp, ci = np.asarray(g.row_ptr, np.int64), np.asarray(g.col_ind, np.int64)
    nv = len(rp) - 1
    pv, R, _ = pair_plan(rp, ci, nv)
    v0 = nv - min(nv, h)
    assert any(v >= v0 for v in pv), "the test wants pair vertices inside the core"
    core, H4 = build_core(rp, ci, v0, nv - v0)
    # the core over its active (non-pair) vertices: all their wedges
    core_part, wp = core_count(rp, ci, core, v0, nv - v0, H4, 0, 1 << 62, exclude=set(pv))
    pair_part = pair_count(rp, ci, pv, R, 256)
    rest = sum(oracle.count_merge_range(g, v, v + 1)
               for v in range(v0) if v not in set(pv))
    assert core_part + pair_part + rest == oracle.count_merge(g)
