"""Seeded synthetic workloads that stand in for the reference's datasets.

* ``CHUNG_LU_262K``: the plain single-graph case -- a Chung-Lu graph with
  n = 262,111, power-law exponent 2.6 and 899,990 seeded endpoint draws,
  which leaves 899,792 unique undirected edges (mean degree 6.87, max 419).
  It stands in for the reference README's example graph (same n and m);
  run with s = 5, a = 8192.
* ``RMAT_S22``: R-MAT scale 22 (n = 4,194,304), edge factor 16
  (67,108,864 draws), (a, b, c, d) = (0.57, 0.19, 0.19, 0.05), seed 1;
  symmetrised, deduplicated, self-loops removed by preprocessing.

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
