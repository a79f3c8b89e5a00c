"""Multi-GPU wedge-range sharding.

The wedge index space [0, W) of one oriented graph splits into equal
contiguous ranges, one per rank (the reference already parameterises a
kernel launch by a wedge window, experiments/tc_big_graphs.cu:173-174 and
394-420). Every rank holds a replica of the CSR, counts the triangles closed
by its range, and one 8-byte all-reduce sums the partial counts -- the only
exchange the path has. A replica made on one rank reaches the others with
broadcast_csr. A batch of many graphs shards whole graphs instead
(shard_graphs / distributed_batch_counts): each rank counts its own graphs
and one all-reduce of the per-graph count vector gives every rank all of
them. One process per GPU, torch.distributed for the plumbing (NCCL on
GPUs, gloo on CPU for tests).
"""
from __future__ import annotations

import heapq
from typing import Callable, List, Optional, Sequence, Tuple

import numpy as np


def shard_range(W: int, rank: int, world: int) -> Tuple[int, int]:
    """[begin, end) of rank's share of [0, W); shares differ by at most one."""
    if world <= 0 or not 0 <= rank < world:
        raise ValueError(f"bad rank {rank} of {world}")
    return W * rank // world, W * (rank + 1) // world


def cost_balanced_cuts(W: int, core_wedges: int, main_ms: float, core_ms: float,
                       world: int) -> List[int]:
    """Rank boundaries (world + 1 values, 0 .. W) that give every rank the
    same estimated device time instead of the same number of wedges.

    The dense core holds the last ``core_wedges`` wedges of the wedge order
    and counts them far faster per wedge than the wedge check counts the
    rest (``main_ms`` and ``core_ms``: the two kernels' times of one
    whole-graph count, e.g. ``stats.count_ms - stats.core_ms`` and
    ``stats.core_ms``), so equal wedge ranges would leave the low ranks with
    most of the time. The cost is linear in each part; the cuts split it
    evenly. Every rank must pass the same figures (broadcast them) so the
    ranges tile [0, W) exactly."""
    if world <= 0:
        raise ValueError(f"bad world size {world}")
    Wc = max(0, min(int(core_wedges), int(W)))
    Wm = int(W) - Wc
    cm = max(float(main_ms), 1e-9) / max(Wm, 1)
    cc = max(float(core_ms), 1e-9) / Wc if Wc else cm
    total = Wm * cm + Wc * cc
    cuts = [0]
    for r in range(1, world):
        c = total * r / world
        x = int(c / cm) if c <= Wm * cm else Wm + int((c - Wm * cm) / cc)
        cuts.append(min(int(W), max(cuts[-1], x)))
    cuts.append(int(W))
    return cuts


def host_wedge_total(row_ptr: np.ndarray) -> int:
    """W = sum over v of C(d+(v), 2) of a host oriented CSR."""
    d = np.diff(np.asarray(row_ptr, dtype=np.int64))
    return int((d * (d - 1) // 2).sum())


class RankFailed(RuntimeError):
    """Raised on every rank when the local work of one or more ranks failed.

    The failing rank's own exception is chained as ``__cause__`` on that
    rank; the others learn only which ranks failed (``failed_ranks``)."""

    def __init__(self, failed_ranks: List[int], cause: Optional[BaseException] = None):
        self.failed_ranks = failed_ranks
        what = f": {type(cause).__name__}: {cause}" if cause is not None else ""
        super().__init__(f"local count failed on rank(s) {failed_ranks}{what}")


def _reduce_with_status(values: List[int], failed: bool, group, device):
    """All-reduces (sum) ``values`` plus one status slot per rank.

    Every rank reaches the collective whether or not its own work failed, so
    no rank is left waiting in it; the status slots tell every rank which
    ranks failed. Returns (sums, failed_ranks)."""
    import torch
    import torch.distributed as dist

    rank, world = dist.get_rank(group), dist.get_world_size(group)
    host = [0 if failed else int(v) for v in values] + [0] * world
    if failed:
        host[len(values) + rank] = 1
    t = torch.tensor(host, dtype=torch.int64, device=device or "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    host = t.tolist()
    bad = [r for r in range(world) if host[len(values) + r]]
    return [int(x) for x in host[: len(values)]], bad


def reduce_count(value: int, group=None, device: Optional[str] = None) -> int:
    """Sum of an exact integer count over the ranks of `group`."""
    import torch
    import torch.distributed as dist

    t = torch.tensor([value], dtype=torch.int64, device=device or "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    return int(t.item())


def broadcast_csr(row_ptr, col_ind, src: int = 0, group=None, device: Optional[str] = None):
    """Gives every rank of `group` a replica of rank `src`'s oriented CSR.

    On rank `src`, ``row_ptr`` / ``col_ind`` are the CSR (torch tensors or
    numpy arrays); other ranks pass None. Returns (row_ptr, col_ind) as
    torch tensors on ``device`` (int64 offsets, int32 columns holding the
    u32 ids bit for bit): a header broadcast with the sizes, then one
    broadcast per array -- over NVLink with NCCL when ``device`` is a GPU,
    through gloo on CPU.
    """
    import torch
    import torch.distributed as dist

    rank = dist.get_rank(group)
    dev = torch.device(device or "cpu")
    if rank == src:
        rp = torch.as_tensor(np.asarray(row_ptr, dtype=np.int64) if not torch.is_tensor(row_ptr)
                             else row_ptr.to(torch.int64)).to(dev)
        ci_np = None if torch.is_tensor(col_ind) else np.asarray(col_ind, dtype=np.uint32)
        ci = (torch.from_numpy(ci_np.view(np.int32)) if ci_np is not None
              else col_ind.view(torch.int32) if col_ind.dtype in (torch.int32,)
              else col_ind.to(torch.int32)).to(dev)
        hdr = torch.tensor([rp.numel(), ci.numel()], dtype=torch.int64, device=dev)
    else:
        hdr = torch.zeros(2, dtype=torch.int64, device=dev)
    dist.broadcast(hdr, src, group=group)
    if rank != src:
        rp = torch.empty(int(hdr[0]), dtype=torch.int64, device=dev)
        ci = torch.empty(int(hdr[1]), dtype=torch.int32, device=dev)
    dist.broadcast(rp, src, group=group)
    if ci.numel():
        dist.broadcast(ci, src, group=group)
    return rp, ci


def distributed_count(count_range: Callable[[int, int], int], W: int, group=None,
                      device: Optional[str] = None,
                      cuts: Optional[Sequence[int]] = None) -> int:
    """Counts the triangles of one graph across the ranks of `group`.

    ``count_range(begin, end)`` returns the triangles closed by wedges
    [begin, end) on this rank (for example ``lambda b, e: og.count(s, a,
    wedge_begin=b, wedge_end=e)[0]`` on an :class:`wetric.OrientedGraph`).
    Every rank must call this with the same W. ``device`` is where the
    all-reduce buffer lives ("cuda:i" for NCCL, None for gloo): the count
    plus one status slot per rank. If ``count_range`` raises on any rank,
    every rank still reaches the all-reduce and then raises
    :class:`RankFailed` (no rank is left waiting in the collective).
    ``cuts`` (world + 1 boundaries, the same on every rank, e.g. from
    :func:`cost_balanced_cuts`) replaces the equal wedge shares.
    """
    import torch.distributed as dist

    rank, world = dist.get_rank(group), dist.get_world_size(group)
    if cuts is not None:
        if len(cuts) != world + 1 or cuts[0] != 0 or cuts[-1] != W or any(
                cuts[i] > cuts[i + 1] for i in range(world)):
            raise ValueError("cuts must rise from 0 to W with world + 1 entries")
        b, e = int(cuts[rank]), int(cuts[rank + 1])
    else:
        b, e = shard_range(W, rank, world)
    err: Optional[BaseException] = None
    part = 0
    try:
        part = int(count_range(b, e)) if e > b else 0
    except Exception as ex:  # reported after the collective, on every rank
        err = ex
    (total,), bad = _reduce_with_status([part], err is not None, group, device)
    if bad:
        raise RankFailed(bad, err) from err
    return total


def shard_graphs(weights: Sequence[int], world: int) -> List[List[int]]:
    """Whole graphs of a batch assigned to `world` ranks by estimated work.

    ``weights[i]`` is graph i's estimated work (its wedge count W). Graphs
    are dealt heaviest first, each to the rank with the least work so far
    (ties: the lower rank), so every rank computes the same assignment with
    no exchange and the heaviest graphs spread first. Returns each rank's
    graph indices in ascending order.
    """
    if world <= 0:
        raise ValueError(f"bad world size {world}")
    order = sorted(range(len(weights)), key=lambda i: (-int(weights[i]), i))
    heap = [(0, r) for r in range(world)]
    parts: List[List[int]] = [[] for _ in range(world)]
    for i in order:
        load, r = heapq.heappop(heap)
        parts[r].append(i)
        heapq.heappush(heap, (load + int(weights[i]), r))
    return [sorted(p) for p in parts]


def distributed_batch_counts(count_graphs: Callable[[List[int]], Sequence[int]],
                             weights: Sequence[int], group=None,
                             device: Optional[str] = None) -> List[int]:
    """Per-graph triangle counts of a batch counted across the ranks.

    ``count_graphs(indices)`` counts this rank's graphs (in the given order;
    for example a :class:`wetric.Batch` built from them). Every rank must
    pass the same ``weights``. Each rank writes its counts into a vector of
    all graphs, zeros elsewhere, and one all-reduce (sum) gives every rank
    every count -- the only exchange. The vector carries one status slot per
    rank: if ``count_graphs`` raises or returns the wrong number of counts on
    any rank, every rank still reaches the all-reduce and then raises
    :class:`RankFailed`.
    """
    import torch.distributed as dist

    rank, world = dist.get_rank(group), dist.get_world_size(group)
    mine = shard_graphs(weights, world)[rank]
    err: Optional[BaseException] = None
    vec = [0] * len(weights)
    try:
        counts = list(count_graphs(mine)) if mine else []
        if len(counts) != len(mine):
            raise ValueError(f"count_graphs returned {len(counts)} counts for {len(mine)} graphs")
        for i, c in zip(mine, counts):
            vec[i] = int(c)
    except Exception as ex:  # reported after the collective, on every rank
        err = ex
    sums, bad = _reduce_with_status(vec, err is not None, group, device)
    if bad:
        raise RankFailed(bad, err) from err
    return sums
