"""Shared test setup: import paths, the `gpu` marker, small graph builders."""
from __future__ import annotations

import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "wedge-parallel-triangle-counting_b200")
ORACLE = os.path.join(ROOT, "oracle")
GOLDEN = os.path.join(ROOT, "tests", "golden")
for p in (ROOT, PKG, ORACLE):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


# ------------------------------------------------------------ graph builders


def complete_graph(k: int):
    """K_k as 0-based pairs (each unordered pair once)."""
    iu = np.triu_indices(k, 1)
    return iu[0].astype(np.uint32), iu[1].astype(np.uint32)


def star_graph(k: int):
    return np.zeros(k, np.uint32), np.arange(1, k + 1, dtype=np.uint32)


def wheel_graph(k: int):
    """Hub 0 + cycle 1..k: k triangles for k >= 4."""
    hub_s = np.zeros(k, np.uint32)
    hub_d = np.arange(1, k + 1, dtype=np.uint32)
    cyc_s = np.arange(1, k + 1, dtype=np.uint32)
    cyc_d = np.array([(i % k) + 1 for i in range(1, k + 1)], np.uint32)
    return np.concatenate([hub_s, cyc_s]), np.concatenate([hub_d, cyc_d])


def bipartite_graph(p: int, q: int):
    a, b = np.meshgrid(np.arange(p), np.arange(p, p + q), indexing="ij")
    return a.ravel().astype(np.uint32), b.ravel().astype(np.uint32)


def random_pairs(n: int, m: int, seed: int):
    rng = np.random.default_rng(seed)
    return (rng.integers(0, n, m).astype(np.uint32),
            rng.integers(0, n, m).astype(np.uint32))


def comb3(k: int) -> int:
    return k * (k - 1) * (k - 2) // 6


@pytest.fixture(scope="session")
def oracle_mod():
    import oracle

    return oracle


@pytest.fixture(scope="session")
def wetric_mod():
    import wetric

    return wetric
