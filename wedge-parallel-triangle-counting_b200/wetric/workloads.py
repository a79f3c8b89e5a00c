"""Seeded synthetic workloads that stand in for the reference's datasets.

* ``CHUNG_LU_262K``: the plain single-graph case -- a Chung-Lu graph with
  n = 262,111, power-law exponent 2.6 and 899,990 seeded endpoint draws,
  which leaves 899,792 unique undirected edges (mean degree 6.87, max 419).
  It stands in for the reference README's example graph (same n and m);
  run with s = 5, a = 8192.
* ``RMAT_S22``: R-MAT scale 22 (n = 4,194,304), edge factor 16
  (67,108,864 draws), (a, b, c, d) = (0.57, 0.19, 0.19, 0.05), seed 1;
  symmetrised, deduplicated, self-loops removed by preprocessing.
* ``RMAT_S27``: the large-graph case, R-MAT scale 27, edge factor 40
  (5,368,709,120 draws), same (a, b, c, d); m > 2^32 after symmetrising.
* ``mixed_batch(count, seed)``: the uneven batch -- half Erdos-Renyi, half
  Chung-Lu with exponent uniform in [2.2, 3.0]; n log-uniform in
  [1,000, 1,000,000]; mean degree uniform in [4, 64]; graph i seeded with
  seed + i.

Generators are counter-based (see csrc/gen.cuh), so the host and device
streams are identical and every workload is reproducible from its seed.
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import Tuple

import numpy as np


@dataclass(frozen=True)
class RmatSpec:
    scale: int
    edge_factor: int
    a: float = 0.57
    b: float = 0.19
    c: float = 0.19
    seed: int = 1

    @property
    def n(self) -> int:
        return 1 << self.scale

    @property
    def draws(self) -> int:
        return self.edge_factor << self.scale

    @property
    def name(self) -> str:
        return f"rmat-s{self.scale}-ef{self.edge_factor}-seed{self.seed}"


@dataclass(frozen=True)
class ChungLuSpec:
    n: int
    gamma: float
    i0: float
    draws: int
    seed: int = 1

    @property
    def name(self) -> str:
        return f"chunglu-n{self.n}-g{self.gamma}-seed{self.seed}"


@dataclass(frozen=True)
class ErdosRenyiSpec:
    n: int
    draws: int
    seed: int = 1

    @property
    def name(self) -> str:
        return f"er-n{self.n}-e{self.draws}-seed{self.seed}"


CHUNG_LU_262K = ChungLuSpec(n=262_111, gamma=2.6, i0=84.0, draws=899_990, seed=1)
RMAT_S22 = RmatSpec(scale=22, edge_factor=16)
RMAT_S27 = RmatSpec(scale=27, edge_factor=40)


def chung_lu_for(n: int, mean_degree: float, gamma: float, seed: int) -> ChungLuSpec:
    """A Chung-Lu graph with n vertices, about n * mean_degree / 2 edges and
    expected degrees following a power law of exponent gamma, with the
    largest expected degree near sqrt(n * mean_degree) (the natural cutoff
    that keeps edge probabilities below one)."""
    alpha = 1.0 / (gamma - 1.0)
    target_max = max(2.0, (n * mean_degree) ** 0.5)
    # weights (1 + i/i0)^-alpha: max/mean ~ (n/i0)^alpha * (1 - alpha); pick
    # i0 so that the largest expected degree lands near target_max.
    ratio = max(1.5, target_max / mean_degree)
    i0 = max(1.0, n / (ratio / max(1e-3, 1.0 - alpha)) ** (1.0 / alpha)) if alpha < 1 else max(1.0, n / ratio)
    return ChungLuSpec(n=n, gamma=gamma, i0=float(i0), draws=int(n * mean_degree / 2), seed=seed)


def mixed_batch(count: int = 4096, seed: int = 1000):
    """The uneven-batch workload: list of graph specs, half Erdos-Renyi and
    half Chung-Lu, n log-uniform in [1e3, 1e6], mean degree U[4, 64]."""
    rng = np.random.default_rng(seed)
    specs = []
    for i in range(count):
        n = int(round(10 ** rng.uniform(3.0, 6.0)))
        deg = float(rng.uniform(4.0, 64.0))
        gamma = float(rng.uniform(2.2, 3.0))
        if i % 2 == 0:
            specs.append(ErdosRenyiSpec(n=n, draws=int(n * deg / 2), seed=seed + i))
        else:
            specs.append(chung_lu_for(n, deg, gamma, seed + i))
    return specs


def batch_pairs_device(specs, device: int = 0):
    """Concatenated device pairs of a list of graph specs:
    (src, dst, pair_off, n) ready for :class:`wetric.Batch`."""
    import torch

    draws = np.array([s.draws for s in specs], np.uint64)
    off = np.zeros(len(specs) + 1, np.uint64)
    off[1:] = np.cumsum(draws)
    total = int(off[-1])
    dev = f"cuda:{device}"
    src = torch.empty(total, dtype=torch.int32, device=dev)
    dst = torch.empty(total, dtype=torch.int32, device=dev)
    import wetric

    for i, sp in enumerate(specs):
        lo, hi = int(off[i]), int(off[i + 1])
        if hi == lo:
            continue
        if isinstance(sp, RmatSpec):
            s, d = wetric.gen_rmat_device(sp.scale, sp.draws, sp.a, sp.b, sp.c, sp.seed, device)
        elif isinstance(sp, ChungLuSpec):
            cdf = wetric.chung_lu_cdf(sp.n, sp.gamma, sp.i0)
            s, d = wetric.gen_weighted_device(cdf, sp.n, sp.draws, sp.seed, device)
        else:
            s, d = wetric.gen_weighted_device(None, sp.n, sp.draws, sp.seed, device)
        src[lo:hi] = s
        dst[lo:hi] = d
        del s, d
    n = np.array([sp.n for sp in specs], np.uint64)
    return src, dst, off, n


def host_pairs(spec) -> Tuple[np.ndarray, np.ndarray, int]:
    """(src, dst, n) of a workload on the host (0-based, raw: self-loops
    and repeats included)."""
    import wetric

    if isinstance(spec, RmatSpec):
        s, d = wetric.gen_rmat(spec.scale, spec.draws, spec.a, spec.b, spec.c, spec.seed)
        return s, d, spec.n
    if isinstance(spec, ChungLuSpec):
        cdf = wetric.chung_lu_cdf(spec.n, spec.gamma, spec.i0)
        s, d = wetric.gen_weighted(cdf, spec.n, spec.draws, spec.seed)
        return s, d, spec.n
    if isinstance(spec, ErdosRenyiSpec):
        s, d = wetric.gen_weighted(None, spec.n, spec.draws, spec.seed)
        return s, d, spec.n
    raise TypeError(spec)


def device_pairs(spec, device: int = 0):
    """(src, dst, n) of a workload as CUDA torch tensors."""
    import wetric

    if isinstance(spec, RmatSpec):
        s, d = wetric.gen_rmat_device(spec.scale, spec.draws, spec.a, spec.b,
                                      spec.c, spec.seed, device)
        return s, d, spec.n
    if isinstance(spec, ChungLuSpec):
        cdf = wetric.chung_lu_cdf(spec.n, spec.gamma, spec.i0)
        s, d = wetric.gen_weighted_device(cdf, spec.n, spec.draws, spec.seed, device)
        return s, d, spec.n
    if isinstance(spec, ErdosRenyiSpec):
        s, d = wetric.gen_weighted_device(None, spec.n, spec.draws, spec.seed, device)
        return s, d, spec.n
    raise TypeError(spec)
