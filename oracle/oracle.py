"""ctypes binding of the CPU oracle (oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, by the smoke() check of
__graft_entry__.py and by bench.py's CPU-baseline / reference legs, always
as the checker. The product (libwetric, the tc tool, the wetric package)
never imports it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from dataclasses import dataclass
from typing import Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
REF_TC = os.path.join(HERE, "_ref", "tc")
REF_TC_BIG = os.path.join(HERE, "_ref", "tc_big_graphs")


def build() -> None:
    subprocess.check_call(["make", "-s", "-C", HERE, "liboracle.so"])


if not os.path.exists(LIB_PATH):
    build()

_lib = C.CDLL(LIB_PATH)


class _OCsr(C.Structure):
    _fields_ = [
        ("n", C.c_uint64),
        ("m", C.c_uint64),
        ("rp", C.POINTER(C.c_uint64)),
        ("ci", C.POINTER(C.c_uint32)),
    ]


def _sig(name, restype, *args):
    f = getattr(_lib, name)
    f.restype = restype
    f.argtypes = list(args)
    return f


_free = _sig("oracle_free", None, C.POINTER(_OCsr))
_read_graph = _sig("oracle_read_graph", C.c_int, C.c_char_p, C.c_int, C.c_int, C.POINTER(_OCsr))
_from_pairs = _sig("oracle_csr_from_pairs", C.c_int, C.c_void_p, C.c_void_p,
                   C.c_uint64, C.c_uint64, C.POINTER(_OCsr))
_preprocess = _sig("oracle_preprocess", C.c_int, C.POINTER(_OCsr), C.POINTER(_OCsr))
_wedge_total = _sig("oracle_wedge_total", C.c_uint64, C.POINTER(_OCsr))
_max_out = _sig("oracle_max_out_degree", C.c_uint64, C.POINTER(_OCsr))
_count_wedges = _sig("oracle_count_wedges", C.c_uint64, C.POINTER(_OCsr),
                     C.c_uint64, C.c_uint64, C.c_uint32)
_count_merge = _sig("oracle_count_merge", C.c_uint64, C.POINTER(_OCsr))
_count_merge_range = _sig("oracle_count_merge_range", C.c_uint64, C.POINTER(_OCsr),
                          C.c_uint64, C.c_uint64)
_wedges_range = _sig("oracle_wedges_range", C.c_uint64, C.POINTER(_OCsr),
                     C.c_uint64, C.c_uint64)
_alg_bytes = _sig("oracle_algorithmic_bytes", C.c_uint64, C.POINTER(_OCsr))
_decode = _sig("oracle_decode_wedge", None, C.c_uint64, C.c_uint64,
               C.POINTER(C.c_uint64), C.POINTER(C.c_uint64))
_max_threads = _sig("oracle_max_threads", C.c_int)
_gen_rmat = _sig("oracle_gen_rmat", C.c_int, C.c_uint32, C.c_uint64, C.c_double, C.c_double,
                 C.c_double, C.c_uint64, C.c_void_p, C.c_void_p)
_write_mm = _sig("oracle_write_mm", C.c_int, C.c_char_p, C.c_uint64, C.c_void_p, C.c_void_p,
                 C.c_uint64)


@dataclass
class CSR:
    row_ptr: np.ndarray  # u64[n+1]
    col_ind: np.ndarray  # u32[m]

    @property
    def n(self) -> int:
        return int(self.row_ptr.shape[0] - 1)

    @property
    def m(self) -> int:
        return int(self.col_ind.shape[0])

    def _struct(self):
        rp = np.ascontiguousarray(self.row_ptr, dtype=np.uint64)
        ci = np.ascontiguousarray(self.col_ind, dtype=np.uint32)
        if ci.shape[0] == 0:
            ci = np.zeros(1, np.uint32)
        s = _OCsr(rp.shape[0] - 1, self.m, rp.ctypes.data_as(C.POINTER(C.c_uint64)),
                  ci.ctypes.data_as(C.POINTER(C.c_uint32)))
        return s, (rp, ci)


def _take(s: _OCsr) -> CSR:
    n, m = int(s.n), int(s.m)
    rp = np.ctypeslib.as_array(s.rp, shape=(n + 1,)).copy()
    ci = np.ctypeslib.as_array(s.ci, shape=(m,)).copy() if m else np.zeros(0, np.uint32)
    _free(C.byref(s))
    return CSR(rp, ci)


class OracleError(RuntimeError):
    pass


def read_graph(path: str, matrix_market: bool = False, zero_indexed: bool = False) -> CSR:
    """read_graph (tc.cu:561-685) restated: symmetric deduplicated CSR."""
    s = _OCsr()
    rc = _read_graph(os.fsencode(path), int(matrix_market), int(zero_indexed), C.byref(s))
    if rc != 0:
        raise OracleError({-1: "cannot open/allocate", -2: "no data line",
                           -3: "zero id without zero_indexed"}.get(rc, str(rc)))
    return _take(s)


def csr_from_pairs(src: np.ndarray, dst: np.ndarray, n: int = 0) -> CSR:
    src = np.ascontiguousarray(src, dtype=np.uint32)
    dst = np.ascontiguousarray(dst, dtype=np.uint32)
    s = _OCsr()
    if _from_pairs(src.ctypes.data, dst.ctypes.data, src.shape[0], n, C.byref(s)) != 0:
        raise OracleError("allocation failed")
    return _take(s)


def preprocess(g: CSR) -> CSR:
    """preprocess (tc.cu:687-787) restated with the stable degree order."""
    si, keep = g._struct()
    so = _OCsr()
    if _preprocess(C.byref(si), C.byref(so)) != 0:
        raise OracleError("allocation failed")
    del keep
    return _take(so)


def oriented_from_pairs(src, dst, n: int = 0) -> CSR:
    return preprocess(csr_from_pairs(src, dst, n))


def _call(fn, g: CSR, *args):
    s, keep = g._struct()
    r = fn(C.byref(s), *args)
    del keep
    return int(r)


def wedge_total(g: CSR) -> int:
    return _call(_wedge_total, g)


def max_out_degree(g: CSR) -> int:
    return _call(_max_out, g)


def count_wedges(g: CSR, a: int = 0, wedge_begin: int = 0, wedge_end: int = 0) -> int:
    """Wedge-check count (tc.cu:173-293 + bitmap of tc.cu:329-346)."""
    return _call(_count_wedges, g, wedge_begin, wedge_end, a)


def count_merge(g: CSR) -> int:
    """Independent merge-intersection count (OpenMP)."""
    return _call(_count_merge, g)


def count_merge_range(g: CSR, vbegin: int, vend: int) -> int:
    return _call(_count_merge_range, g, vbegin, vend)


def wedges_range(g: CSR, vbegin: int, vend: int) -> int:
    return _call(_wedges_range, g, vbegin, vend)


def algorithmic_bytes(g: CSR) -> int:
    return _call(_alg_bytes, g)


def decode_wedge(iv: int, d: int):
    """The reference's floating-point first-wedge decode (tc.cu:206-212)."""
    wi, ui = C.c_uint64(0), C.c_uint64(0)
    _decode(iv, d, C.byref(wi), C.byref(ui))
    return int(wi.value), int(ui.value)


def max_threads() -> int:
    return int(_max_threads())


def have_reference_binary(big: bool = False) -> bool:
    return os.access(REF_TC_BIG if big else REF_TC, os.X_OK)


def run_reference(path: str, s: int, a: int, loops: int = 1, matrix_market: bool = True,
                  big: bool = False, zero_indexed: bool = False,
                  timeout: Optional[float] = None):
    """Runs the reference's own tc (built for sm_100a into _ref/) and parses
    its table: returns a list of row dicts (n, m, s, a, triangles, prepro,
    copy, exec, total, cpu_gpu). Needs a GPU."""
    exe = REF_TC_BIG if big else REF_TC
    cmd = [exe, "-m" if matrix_market else "-e", path, "-s", str(s), "-a", str(a),
           "-l", str(loops)]
    if zero_indexed:
        cmd.insert(1, "-z")
    out = subprocess.run(cmd, capture_output=True, text=True, timeout=timeout)
    if out.returncode != 0:
        raise OracleError(f"reference tc failed ({out.returncode}): {out.stderr[-500:]}")
    rows = []
    for line in out.stdout.splitlines()[1:]:
        f = line.split()
        if len(f) < 11:
            continue
        rows.append(dict(graph=f[0], n=int(f[1]), m=int(f[2]), s=int(f[3]), a=int(f[4]),
                         triangles=int(f[5]), prepro=float(f[6]), copy=float(f[7]),
                         exec=float(f[8]), total=float(f[9]), cpu_gpu=float(f[10])))
    return rows


_wt_pairs = _sig("oracle_wedge_total_from_pairs", C.c_int, C.c_void_p, C.c_void_p, C.c_uint64,
                 C.POINTER(C.c_uint64), C.POINTER(C.c_uint64))


def wedge_total_from_pairs(src: np.ndarray, dst: np.ndarray):
    """(W, max out-degree) of the oriented graph of raw pairs (the same rules
    as csr_from_pairs + preprocess, without building the CSR), in C."""
    s = np.ascontiguousarray(src, dtype=np.uint32)
    d = np.ascontiguousarray(dst, dtype=np.uint32)
    W, md = C.c_uint64(0), C.c_uint64(0)
    if _wt_pairs(s.ctypes.data, d.ctypes.data, s.shape[0], C.byref(W), C.byref(md)) != 0:
        raise OracleError("allocation failed")
    return int(W.value), int(md.value)


def wedge_total_from_pairs_numpy(src: np.ndarray, dst: np.ndarray):
    """(W, max out-degree) of the oriented graph of raw pairs, computed with
    numpy (the same rules as csr_from_pairs + preprocess, without building
    the CSR): unique undirected edges, stable (degree, id) rank, each edge
    charged to its lower-ranked end."""
    keep = src != dst
    lo = np.minimum(src[keep], dst[keep]).astype(np.uint64)
    hi = np.maximum(src[keep], dst[keep]).astype(np.uint64)
    k = np.unique((lo << np.uint64(32)) | hi)
    a = (k >> np.uint64(32)).astype(np.int64)
    b = (k & np.uint64(0xFFFFFFFF)).astype(np.int64)
    n = int(max(a.max(), b.max())) + 1 if len(k) else 1
    deg = np.bincount(a, minlength=n) + np.bincount(b, minlength=n)
    order = np.lexsort((np.arange(n), deg))
    rank = np.empty(n, np.int64)
    rank[order] = np.arange(n)
    dplus = np.bincount(np.minimum(rank[a], rank[b]), minlength=n).astype(np.int64)
    return int((dplus * (dplus - 1) // 2).sum()), int(dplus.max() if n else 0)


def gen_rmat(scale: int, edges: int, a: float = 0.57, b: float = 0.19, c: float = 0.19,
             seed: int = 1):
    """The benchmark's seeded R-MAT pair stream (src, dst) on the CPU."""
    src = np.empty(edges, np.uint32)
    dst = np.empty(edges, np.uint32)
    if _gen_rmat(scale, edges, a, b, c, seed, src.ctypes.data, dst.ctypes.data) != 0:
        raise OracleError("bad R-MAT arguments")
    return src, dst


def write_mm(path: str, n: int, src: np.ndarray, dst: np.ndarray) -> None:
    """Pairs -> 'coordinate pattern symmetric' Matrix Market file (1-based)."""
    s = np.ascontiguousarray(src, dtype=np.uint32)
    d = np.ascontiguousarray(dst, dtype=np.uint32)
    if _write_mm(os.fsencode(path), n, s.ctypes.data, d.ctypes.data, s.shape[0]) != 0:
        raise OracleError(f"cannot write {path}")


def cpu_model() -> str:
    """The host CPU's model name (from /proc/cpuinfo), or '' if unknown."""
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return ""
