"""GPU test of wetric_count_noalloc, the count entry point for callers that
cannot allocate device memory when they count (code inside another
framework's memory pool or under a device-memory quota, hosts that forbid
allocation after start-up). It must give exactly the count of the
allocating entry point, wetric_count_ex, on the same device CSR, on two
calls in a row (the static scratch keeps the previous call's contents, so
the second call checks that everything which must start at zero is
cleared). Collected last on purpose; it needs nothing from other tests."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _noalloc_fn(wetric_mod):
    fn = wetric_mod._lib.wetric_count_noalloc
    fn.restype = C.c_int
    fn.argtypes = [C.POINTER(wetric_mod._Csr), C.c_uint32, C.c_uint32, C.c_int,
                   C.c_void_p, C.POINTER(C.c_uint64)]
    return fn


def _device_csr(wetric_mod, spec, offsets32):
    import torch

    from wetric import workloads as Wl

    src, dst, _ = Wl.host_pairs(spec)
    og = wetric_mod.orient_edges(src, dst)
    g = og.download()
    og.free()
    rp = torch.from_numpy(g.row_ptr.astype(np.uint32 if offsets32 else np.uint64)
                          .view(np.int32 if offsets32 else np.int64)).cuda()
    ci = torch.from_numpy(g.col_ind.view(np.int32)).cuda()
    flags = wetric_mod.CSR_ORIENTED | wetric_mod.CSR_DEVICE
    if offsets32:
        flags |= wetric_mod.CSR_OFFSETS32
    csr = wetric_mod._Csr(g.n, g.m, rp.data_ptr(), ci.data_ptr(), flags)
    return csr, (rp, ci)


@pytest.mark.parametrize("offsets32", [False, True])
def test_noalloc_matches_allocating_count(wetric_mod, offsets32):
    import torch

    from wetric import workloads as Wl

    fn = _noalloc_fn(wetric_mod)
    for spec, s, a in ((Wl.CHUNG_LU_262K, 5, 8192),
                       (Wl.RmatSpec(scale=16, edge_factor=16, seed=3), 5, 8192),
                       (Wl.RmatSpec(scale=12, edge_factor=16, seed=4), 2, 64)):
        csr, keep = _device_csr(wetric_mod, spec, offsets32)
        o = wetric_mod._Opts()
        wetric_mod._opts_init(C.byref(o))
        o.spread, o.bitmap_len = s, a
        want = C.c_uint64(0)
        assert wetric_mod._count_ex(C.byref(csr), C.byref(o), C.byref(want), None) == 0
        stream = torch.cuda.current_stream().cuda_stream
        for _ in range(2):  # two calls in a row
            got = C.c_uint64(12345)
            rc = fn(C.byref(csr), s, a, 0, stream, C.byref(got))
            assert rc == 0, wetric_mod.last_error()
            assert got.value == want.value
        del keep


def test_noalloc_rejects_sizes_beyond_its_scratch(wetric_mod):
    fn = _noalloc_fn(wetric_mod)
    rp = np.zeros(2, np.uint64)
    csr = wetric_mod._Csr(2_000_000, 0, rp.ctypes.data, None,
                          wetric_mod.CSR_ORIENTED | wetric_mod.CSR_DEVICE)
    out = C.c_uint64(0)
    assert fn(C.byref(csr), 5, 64, 0, None, C.byref(out)) == wetric_mod.ERANGE
    csr.n = 10
    assert fn(C.byref(csr), 5, 16384, 0, None, C.byref(out)) == wetric_mod.ERANGE
    host = wetric_mod._Csr(10, 0, rp.ctypes.data, None, wetric_mod.CSR_ORIENTED)
    assert fn(C.byref(host), 5, 64, 0, None, C.byref(out)) == wetric_mod.EINVAL


def _pairs_csr(wetric_mod, src, dst, offsets32):
    """Oriented device CSR of a small hand-made pair list."""
    import torch

    og = wetric_mod.orient_edges(np.asarray(src, np.uint32), np.asarray(dst, np.uint32))
    g = og.download()
    og.free()
    rp = torch.from_numpy(g.row_ptr.astype(np.uint32 if offsets32 else np.uint64)
                          .view(np.int32 if offsets32 else np.int64)).cuda()
    ci = torch.from_numpy(np.ascontiguousarray(g.col_ind).view(np.int32)).cuda()
    flags = wetric_mod.CSR_ORIENTED | wetric_mod.CSR_DEVICE
    if offsets32:
        flags |= wetric_mod.CSR_OFFSETS32
    return wetric_mod._Csr(g.n, g.m, rp.data_ptr(), ci.data_ptr() if g.m else None, flags), (rp, ci)


def _edge_case(wetric_mod, name):
    """(pairs, s, a) of the small cases whose scratch layout differs."""
    n = 5000
    path = (list(range(n - 1)), list(range(1, n)))             # W = 0: no active vertex
    rng = np.random.default_rng(11)
    src = rng.integers(0, 3000, 40000)
    dst = rng.integers(0, 3000, 40000)
    return {"path_no_wedges": (path, 5, 8192),
            "random_no_bitmap": ((src, dst), 1, 0),            # a = 0: no bitmap words
            "triangle_only": (([0, 1, 2], [1, 2, 0]), 3, 32)}[name]


@pytest.mark.parametrize("offsets32", [False, True])
@pytest.mark.parametrize("name", ["path_no_wedges", "random_no_bitmap", "triangle_only"])
def test_noalloc_small_layouts_match(wetric_mod, name, offsets32):
    """Graphs that reach the entry point's early returns and its other
    scratch layouts (no wedges, no bitmap, a single triangle) give the
    allocating count's answer, twice in a row, after a call on a larger
    graph has left its contents in the shared scratch."""
    import torch

    from wetric import workloads as Wl

    fn = _noalloc_fn(wetric_mod)
    stream = torch.cuda.current_stream().cuda_stream
    big, keep_big = _device_csr(wetric_mod, Wl.RmatSpec(scale=12, edge_factor=16, seed=4), offsets32)
    junk = C.c_uint64(0)
    assert fn(C.byref(big), 1, 64, 0, stream, C.byref(junk)) == 0
    (src, dst), s, a = _edge_case(wetric_mod, name)
    csr, keep = _pairs_csr(wetric_mod, src, dst, offsets32)
    o = wetric_mod._Opts()
    wetric_mod._opts_init(C.byref(o))
    o.spread, o.bitmap_len = s, a
    want = C.c_uint64(0)
    assert wetric_mod._count_ex(C.byref(csr), C.byref(o), C.byref(want), None) == 0
    if name == "path_no_wedges":
        assert want.value == 0
    if name == "triangle_only":
        assert want.value == 1
    for _ in range(2):
        got = C.c_uint64(777)
        rc = fn(C.byref(csr), s, a, 0, stream, C.byref(got))
        assert rc == 0, wetric_mod.last_error()
        assert got.value == want.value
    del keep, keep_big


def test_noalloc_empty_graph(wetric_mod):
    """n = 0 counts zero triangles without touching the scratch."""
    import torch

    fn = _noalloc_fn(wetric_mod)
    rp = torch.zeros(1, dtype=torch.int64, device="cuda")
    csr = wetric_mod._Csr(0, 0, rp.data_ptr(), None,
                          wetric_mod.CSR_ORIENTED | wetric_mod.CSR_DEVICE)
    for _ in range(2):
        got = C.c_uint64(99)
        assert fn(C.byref(csr), 5, 8192, 0, None, C.byref(got)) == 0, wetric_mod.last_error()
        assert got.value == 0
