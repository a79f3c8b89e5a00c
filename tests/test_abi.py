"""CPU tests of the C ABI: the library loads, exports every entry point the
headers declare, lays out its structs exactly as the reference's
GRAPH_TYPE / BIG_GRAPH_TYPE / GPU_time (tc.cu:58-79,
experiments/tc_big_graphs.cu:58-63), and refuses to count without a GPU
(there is no CPU fallback)."""
from __future__ import annotations

import ctypes as C
import os
import re
import subprocess

import numpy as np
import pytest

from conftest import PKG, ROOT

HEADERS = [os.path.join(ROOT, "include", "wetric.h"),
           os.path.join(PKG, "csrc", "wetric_tools.h")]


def declared_functions(path):
    text = open(path).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(wetric_[a-z0-9_]+)\s*\(", text)))


def test_headers_declare_expected_entry_points():
    names = declared_functions(HEADERS[0])
    for must in ("wetric_count", "wetric_count_ex", "wetric_tc_gpu", "wetric_read_graph",
                 "wetric_preprocess", "wetric_free_graph", "wetric_last_error",
                 "wetric_strerror"):
        assert must in names


@pytest.mark.parametrize("header", HEADERS)
def test_library_exports_every_declared_symbol(wetric_mod, header):
    lib = C.CDLL(wetric_mod.LIB_PATH)
    missing = [f for f in declared_functions(header) if not hasattr(lib, f)]
    assert not missing, missing


def test_python_binding_covers_header(wetric_mod):
    declared = set(declared_functions(HEADERS[0]))
    assert set(wetric_mod.EXPORTED_SYMBOLS) <= declared


LAYOUT_C = r"""
#include <stddef.h>
#include <stdio.h>
#include "wetric.h"
int main(void) {
  printf("%zu %zu %zu %zu %zu\n", sizeof(wetric_graph), sizeof(wetric_big_graph),
         offsetof(wetric_big_graph, numEdges), offsetof(wetric_big_graph, rowPtr),
         sizeof(wetric_gpu_time));
  printf("%zu %zu %zu %zu\n", sizeof(wetric_csr), sizeof(wetric_opts),
         offsetof(wetric_opts, stream), sizeof(wetric_stats));
  printf("%zu %zu %zu %zu %zu\n", offsetof(wetric_opts, core_len),
         offsetof(wetric_stats, core_wedges), sizeof(wetric_server_opts),
         sizeof(wetric_server_stats), offsetof(wetric_server_stats, resident_last_exit));
  return 0;
}
"""


def test_struct_layouts(tmp_path, wetric_mod):
    src = tmp_path / "layout.c"
    src.write_text(LAYOUT_C)
    exe = tmp_path / "layout"
    subprocess.check_call(["gcc", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)])
    lines = subprocess.check_output([str(exe)], text=True).split("\n")
    g, bg, bg_ne, bg_rp, gt = map(int, lines[0].split())
    csr, opts, opts_stream, stats = map(int, lines[1].split())
    # GRAPH_TYPE = {u32, u32, u32*, u32*}; BIG_GRAPH_TYPE = {u32, u64, u64*, u32*}
    assert (g, bg, bg_ne, bg_rp, gt) == (24, 32, 8, 16, 16)
    assert C.sizeof(wetric_mod._Graph) == g
    assert C.sizeof(wetric_mod._BigGraph) == bg
    assert C.sizeof(wetric_mod._GPUTime) == gt
    assert C.sizeof(wetric_mod._Csr) == csr
    assert C.sizeof(wetric_mod._Opts) == opts
    assert wetric_mod._Opts.stream.offset == opts_stream
    assert C.sizeof(wetric_mod._Stats) == stats
    core_off, core_w, sopts, sstats, last_exit = map(int, lines[2].split())
    assert wetric_mod._Opts.core_len.offset == core_off
    assert wetric_mod._Stats.core_wedges.offset == core_w
    assert C.sizeof(wetric_mod._ServerOpts) == sopts
    assert C.sizeof(wetric_mod._ServerStats) == sstats
    assert wetric_mod._ServerStats.resident_last_exit.offset == last_exit


def test_strerror_and_opts(wetric_mod):
    assert wetric_mod._strerror(0) == b"ok"
    assert b"invalid" in wetric_mod._strerror(wetric_mod.EINVAL)
    o = wetric_mod._Opts()
    wetric_mod._opts_init(C.byref(o))
    assert (o.spread, o.bitmap_len, o.device, o.wedge_end, o.kernel) == (5, 8192, 0, 0, 0)


def _has_gpu():
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.mark.skipif(_has_gpu(), reason="checks the no-GPU failure path")
def test_no_cpu_fallback(wetric_mod):
    """Without a GPU every count fails loudly with ENODEV."""
    rp = np.array([0, 2, 3, 3], np.uint64)
    ci = np.array([1, 2, 2], np.uint32)
    with pytest.raises(wetric_mod.WetricError) as e:
        wetric_mod.count(rp, ci, 5, 64)
    assert e.value.status == wetric_mod.ENODEV
    assert wetric_mod._count(C.byref(wetric_mod._csr_struct(rp, ci, True)[0]), 5, 64) == (1 << 64) - 1
    assert wetric_mod.last_error()[0] == wetric_mod.ENODEV


def test_argument_errors_before_device(wetric_mod):
    """Bad arguments are rejected with EINVAL before any device work."""
    rp = np.array([0, 1, 1], np.uint64)
    ci = np.array([1], np.uint32)
    for s, a in ((0, 64), (5, 33)):
        with pytest.raises(wetric_mod.WetricError) as e:
            wetric_mod.count(rp, ci, s, a)
        assert e.value.status == wetric_mod.EINVAL
    # the Python layer refuses arrays that are not 1-D integer arrays
    with pytest.raises(TypeError):
        wetric_mod.count(rp.astype(np.float64), ci, 5, 64)
    with pytest.raises(TypeError):
        wetric_mod.count(rp, ci.astype(np.float32), 5, 64)
    with pytest.raises(ValueError):
        wetric_mod.count(rp.reshape(1, -1), ci, 5, 64)
    with pytest.raises(ValueError):
        wetric_mod.count(np.zeros(0, np.uint64), ci, 5, 64)
