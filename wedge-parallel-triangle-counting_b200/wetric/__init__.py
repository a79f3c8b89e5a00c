"""wetric -- Python host interface of the B200-native wedge-parallel
triangle counter.

A thin ctypes layer over ``libwetric.so`` (the C ABI of
``include/wetric.h``). The functions that mirror the reference keep its
names and argument meaning:

* :func:`read_graph`  -- ``read_graph``  (tc.cu:561)
* :func:`preprocess`  -- ``preprocess``  (tc.cu:687)
* :func:`tc_GPU`      -- ``tc_GPU``      (tc.cu:315), adding milliseconds into
  a :class:`GPUTime` like the reference's ``GPU_time`` (tc.cu:76-79)

plus :func:`count` (host numpy or device torch CSR, options, statistics),
:func:`orient_edges` (device preprocessing of a raw edge list) and the
seeded generators used for synthetic inputs.

Every count runs in libwetric's CUDA kernels: there is no CPU path. If the
shared library is missing this module raises on import, and every count
raises :class:`WetricError` when no GPU is present.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass, field
from typing import Optional, Tuple

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
# WETRIC_LIB selects another build of the library (same C ABI).
LIB_PATH = os.environ.get("WETRIC_LIB") or os.path.join(_HERE, "libwetric.so")

if not os.path.exists(LIB_PATH):
    raise ImportError(
        f"{LIB_PATH} is not built; run `make` in {os.path.dirname(_HERE)}"
    )

_lib = C.CDLL(LIB_PATH)

# ------------------------------------------------------------------ status

OK, EINVAL, ENOMEM, ETIMEDOUT, ECUDA, ERANGE, EIO, ENODEV, EBUSY = range(9)

CSR_ORIENTED = 0x1
CSR_SYMMETRIC = 0x2
CSR_DEVICE = 0x4
CSR_OFFSETS32 = 0x8
OPT_KEEP_U64_OFFSETS = 0x1
OPT_ONE_PASS = 0x2
OPT_NO_PAIR_STREAMS = 0x4
CORE_OFF = 0xFFFFFFFF

PREPROCESS_CPU, PREPROCESS_GPU, PREPROCESS_GPU_CONSTRAINED = 0, 1, 2


class WetricError(RuntimeError):
    """A libwetric call failed; ``status`` is the WETRIC_* code."""

    def __init__(self, status: int, message: str):
        super().__init__(f"[{status}] {message}")
        self.status = status


# ------------------------------------------------------------------ structs


class _Graph(C.Structure):
    """GRAPH_TYPE layout (tc.cu:58-63)."""

    _fields_ = [
        ("numVertices", C.c_uint32),
        ("numEdges", C.c_uint32),
        ("rowPtr", C.POINTER(C.c_uint32)),
        ("colInd", C.POINTER(C.c_uint32)),
    ]


class _BigGraph(C.Structure):
    """BIG_GRAPH_TYPE layout (experiments/tc_big_graphs.cu:58-63)."""

    _fields_ = [
        ("numVertices", C.c_uint32),
        ("numEdges", C.c_uint64),
        ("rowPtr", C.POINTER(C.c_uint64)),
        ("colInd", C.POINTER(C.c_uint32)),
    ]


class _GPUTime(C.Structure):
    _fields_ = [("copy", C.c_double), ("exec", C.c_double)]


class _Csr(C.Structure):
    _fields_ = [
        ("n", C.c_uint64),
        ("m", C.c_uint64),
        ("row_ptr", C.c_void_p),
        ("col_ind", C.c_void_p),
        ("flags", C.c_uint32),
    ]


class _Opts(C.Structure):
    _fields_ = [
        ("spread", C.c_uint32),
        ("bitmap_len", C.c_uint32),
        ("block", C.c_uint32),
        ("validate", C.c_uint32),
        ("wedge_begin", C.c_uint64),
        ("wedge_end", C.c_uint64),
        ("device", C.c_int32),
        ("l2_persist", C.c_uint32),
        ("kernel", C.c_uint32),
        ("opt_flags", C.c_uint32),
        ("stream", C.c_void_p),
        ("core_len", C.c_uint32),
        ("shell_len", C.c_uint32),
    ]


class _Stats(C.Structure):
    _fields_ = [
        ("copy_ms", C.c_double),
        ("prep_ms", C.c_double),
        ("exec_ms", C.c_double),
        ("count_ms", C.c_double),
        ("n", C.c_uint64),
        ("m", C.c_uint64),
        ("wedges", C.c_uint64),
        ("wedges_counted", C.c_uint64),
        ("max_out_degree", C.c_uint64),
        ("spread", C.c_uint32),
        ("bitmap_len", C.c_uint32),
        ("block", C.c_uint32),
        ("grid", C.c_uint32),
        ("launches", C.c_uint32),
        ("core_len", C.c_uint32),
        ("core_wedges", C.c_uint64),
        ("core_ms", C.c_double),
        ("shell_len", C.c_uint64),
        ("shell_wedges", C.c_uint64),
        ("shell_ms", C.c_double),
        ("pair_rows", C.c_uint64),
        ("pair_wedges", C.c_uint64),
        ("pair_ms", C.c_double),
    ]


def _sig(name, restype, *argtypes):
    fn = getattr(_lib, name)
    fn.restype = restype
    fn.argtypes = list(argtypes)
    return fn


_last_error = _sig("wetric_last_error", C.c_int)
_strerror = _sig("wetric_strerror", C.c_char_p, C.c_int)
_last_msg = _sig("wetric_last_error_message", C.c_char_p)
_opts_init = _sig("wetric_opts_init", None, C.POINTER(_Opts))
_set_budget = _sig("wetric_set_hbm_budget", C.c_int, C.c_int, C.c_uint64)
_count = _sig("wetric_count", C.c_uint64, C.POINTER(_Csr), C.c_uint32, C.c_uint32)
_count_ex = _sig(
    "wetric_count_ex", C.c_int, C.POINTER(_Csr), C.POINTER(_Opts),
    C.POINTER(C.c_uint64), C.POINTER(_Stats)
)
_tc_gpu = _sig(
    "wetric_tc_gpu", C.c_uint64, C.POINTER(_Graph), C.c_uint32, C.c_uint32,
    C.POINTER(_GPUTime)
)
_tc_gpu_big = _sig(
    "wetric_tc_gpu_big", C.c_uint64, C.POINTER(_BigGraph), C.c_uint32,
    C.c_uint32, C.POINTER(_GPUTime)
)
_read_graph = _sig(
    "wetric_read_graph", C.POINTER(_Graph), C.c_char_p, C.c_int, C.c_int, C.c_int
)
_read_big_graph = _sig(
    "wetric_read_big_graph", C.POINTER(_BigGraph), C.c_char_p, C.c_int,
    C.c_int, C.c_int
)
_preprocess = _sig("wetric_preprocess", C.POINTER(_Graph), C.POINTER(_Graph), C.c_int)
_preprocess_big = _sig(
    "wetric_preprocess_big", C.POINTER(_BigGraph), C.POINTER(_BigGraph), C.c_int
)
_free_graph = _sig("wetric_free_graph", None, C.POINTER(_Graph))
_free_big_graph = _sig("wetric_free_big_graph", None, C.POINTER(_BigGraph))
_wedge_total = _sig(
    "wetric_wedge_total", C.c_int, C.POINTER(_Csr), C.c_int,
    C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)
)
_alg_bytes = _sig(
    "wetric_algorithmic_bytes", C.c_int, C.POINTER(_Csr), C.c_int,
    C.POINTER(C.c_uint64)
)
_orient_edges = _sig(
    "wetric_orient_edges", C.c_int, C.c_void_p, C.c_void_p, C.c_uint64,
    C.c_uint64, C.c_uint32, C.c_int, C.POINTER(C.c_void_p), C.POINTER(_Stats)
)
_oriented_csr = _sig("wetric_oriented_csr", C.c_int, C.c_void_p, C.POINTER(_Csr))
_oriented_download = _sig(
    "wetric_oriented_download", C.c_int, C.c_void_p, C.c_void_p, C.c_void_p
)
_oriented_free = _sig("wetric_oriented_free", None, C.c_void_p)
_gen_rmat = _sig(
    "wetric_gen_rmat", C.c_int, C.c_uint32, C.c_uint64, C.c_double, C.c_double,
    C.c_double, C.c_uint64, C.c_void_p, C.c_void_p
)
_gen_rmat_dev = _sig(
    "wetric_gen_rmat_device", C.c_int, C.c_uint32, C.c_uint64, C.c_double,
    C.c_double, C.c_double, C.c_uint64, C.c_void_p, C.c_void_p, C.c_int
)
_chung_lu_cdf = _sig(
    "wetric_chung_lu_cdf", C.c_int, C.c_uint32, C.c_double, C.c_double, C.c_void_p
)
_gen_weighted = _sig(
    "wetric_gen_weighted", C.c_int, C.c_void_p, C.c_uint32, C.c_uint64,
    C.c_uint64, C.c_void_p, C.c_void_p
)
_gen_weighted_dev = _sig(
    "wetric_gen_weighted_device", C.c_int, C.c_void_p, C.c_uint32, C.c_uint64,
    C.c_uint64, C.c_void_p, C.c_void_p, C.c_int
)
_write_mm = _sig(
    "wetric_write_mm", C.c_int, C.c_char_p, C.c_uint64, C.c_void_p, C.c_void_p,
    C.c_uint64
)

EXPORTED_SYMBOLS = (
    "wetric_last_error", "wetric_strerror", "wetric_last_error_message",
    "wetric_read_graph", "wetric_read_big_graph", "wetric_preprocess",
    "wetric_preprocess_big", "wetric_free_graph", "wetric_free_big_graph",
    "wetric_tc_gpu", "wetric_tc_gpu_big", "wetric_set_hbm_budget",
    "wetric_opts_init", "wetric_count", "wetric_count_ex",
    "wetric_wedge_total", "wetric_algorithmic_bytes", "wetric_orient_edges",
    "wetric_oriented_csr", "wetric_oriented_download", "wetric_oriented_free",
    "wetric_batch_opts_init", "wetric_batch_create", "wetric_batch_count",
    "wetric_batch_info", "wetric_batch_spreads", "wetric_batch_free",
    "wetric_server_opts_init",
    "wetric_server_create", "wetric_server_submit", "wetric_server_poll",
    "wetric_server_wait", "wetric_server_get_stats", "wetric_server_destroy",
    "wetric_save_csr", "wetric_load_csr", "wetric_free_buffer",
)


def last_error() -> Tuple[int, str]:
    code = _last_error()
    return code, (_last_msg() or b"").decode(errors="replace")


def _raise(status: Optional[int] = None, what: str = "") -> None:
    code, msg = last_error()
    if status is None:
        status = code
    text = _strerror(status).decode()
    raise WetricError(status, f"{what}: {text}: {msg}" if what else f"{text}: {msg}")


def _check(status: int, what: str) -> None:
    if status != OK:
        _raise(status, what)


def set_hbm_budget(nbytes: int, device: int = 0) -> None:
    """Cap the device memory libwetric may hold on ``device`` (0 = none)."""
    _check(_set_budget(device, nbytes), "set_hbm_budget")


# ------------------------------------------------------------ host graphs


@dataclass
class GPUTime:
    """GPU_time (tc.cu:76-79): milliseconds, accumulated across calls."""

    copy: float = 0.0
    exec: float = 0.0


@dataclass
class Graph:
    """A host CSR: ``row_ptr`` (u64, or u32 when built so) and ``col_ind``."""

    row_ptr: np.ndarray
    col_ind: np.ndarray

    @property
    def numVertices(self) -> int:
        return int(self.row_ptr.shape[0] - 1)

    @property
    def numEdges(self) -> int:
        return int(self.col_ind.shape[0])

    n = numVertices
    m = numEdges


def _graph_from_big(p) -> Graph:
    g = p.contents
    n, m = int(g.numVertices), int(g.numEdges)
    rp = np.ctypeslib.as_array(g.rowPtr, shape=(n + 1,)).copy()
    ci = (
        np.ctypeslib.as_array(g.colInd, shape=(m,)).copy()
        if m
        else np.zeros(0, np.uint32)
    )
    _free_big_graph(p)
    return Graph(rp.astype(np.uint64, copy=False), ci.astype(np.uint32, copy=False))


def _as_big(graph: Graph):
    rp = np.ascontiguousarray(graph.row_ptr, dtype=np.uint64)
    ci = np.ascontiguousarray(graph.col_ind, dtype=np.uint32)
    s = _BigGraph()
    s.numVertices = rp.shape[0] - 1
    s.numEdges = ci.shape[0]
    s.rowPtr = rp.ctypes.data_as(C.POINTER(C.c_uint64))
    s.colInd = ci.ctypes.data_as(C.POINTER(C.c_uint32))
    return s, (rp, ci)


def read_graph(filename: str, matrix_market: bool = False,
               zero_indexed: bool = False,
               preprocess_style: int = PREPROCESS_GPU_CONSTRAINED) -> Graph:
    """read_graph (tc.cu:561): symmetric, deduplicated CSR of a text edge
    list or Matrix Market file (dedup on the GPU)."""
    p = _read_big_graph(os.fsencode(filename), int(matrix_market),
                        int(zero_indexed), int(preprocess_style))
    if not p:
        _raise(what="read_graph")
    return _graph_from_big(p)


def preprocess(graph: Graph, preprocess_style: int = PREPROCESS_GPU_CONSTRAINED) -> Graph:
    """preprocess (tc.cu:687): stable ascending-degree relabel, orientation
    toward the higher id, sorted rows (on the GPU)."""
    s, keep = _as_big(graph)
    p = _preprocess_big(C.byref(s), int(preprocess_style))
    del keep
    if not p:
        _raise(what="preprocess")
    return _graph_from_big(p)


def tc_GPU(graph: Graph, spread: int, adjacency_matrix_len: int,
           t: Optional[GPUTime] = None) -> int:
    """tc_GPU (tc.cu:315): triangles of a host oriented CSR; adds copy and
    exec milliseconds into ``t``."""
    s, keep = _as_big(graph)
    gt = _GPUTime(t.copy if t else 0.0, t.exec if t else 0.0)
    r = _tc_gpu_big(C.byref(s), spread, adjacency_matrix_len, C.byref(gt))
    del keep
    if r == (1 << 64) - 1:
        _raise(what="tc_GPU")
    if t is not None:
        t.copy, t.exec = gt.copy, gt.exec
    return int(r)


# ----------------------------------------------------------- count / stats


@dataclass
class Stats:
    copy_ms: float = 0.0
    prep_ms: float = 0.0
    exec_ms: float = 0.0
    count_ms: float = 0.0
    n: int = 0
    m: int = 0
    wedges: int = 0
    wedges_counted: int = 0
    max_out_degree: int = 0
    spread: int = 0
    bitmap_len: int = 0
    block: int = 0
    grid: int = 0
    launches: int = 0
    core_len: int = 0
    core_wedges: int = 0
    core_ms: float = 0.0
    shell_len: int = 0
    shell_wedges: int = 0
    shell_ms: float = 0.0
    pair_rows: int = 0
    pair_wedges: int = 0
    pair_ms: float = 0.0


def _stats(s: _Stats) -> Stats:
    return Stats(**{f: getattr(s, f) for f in Stats.__dataclass_fields__})


def _is_torch(x) -> bool:
    return type(x).__module__.startswith("torch")


def _csr_struct(row_ptr, col_ind, oriented: bool):
    """Builds a wetric_csr from numpy (host) or torch CUDA (device) arrays."""
    flags = CSR_ORIENTED if oriented else CSR_SYMMETRIC
    if _is_torch(row_ptr):
        import torch

        assert row_ptr.is_cuda and col_ind.is_cuda, "torch tensors must be on CUDA"
        assert col_ind.dtype in (torch.int32, torch.uint32)
        if row_ptr.dtype in (torch.int32, torch.uint32):
            flags |= CSR_OFFSETS32
        elif row_ptr.dtype not in (torch.int64, torch.uint64):
            raise TypeError("row_ptr must be a 32- or 64-bit integer tensor")
        row_ptr = row_ptr.contiguous()
        col_ind = col_ind.contiguous()
        flags |= CSR_DEVICE
        csr = _Csr(row_ptr.numel() - 1, col_ind.numel(), row_ptr.data_ptr(),
                   col_ind.data_ptr(), flags)
        return csr, (row_ptr, col_ind), row_ptr.device.index or 0
    rp = np.ascontiguousarray(row_ptr)
    ci = np.ascontiguousarray(col_ind)
    if rp.dtype.kind not in "iu" or ci.dtype.kind not in "iu":
        raise TypeError("row_ptr and col_ind must be integer arrays")
    if rp.ndim != 1 or ci.ndim != 1 or rp.shape[0] < 1:
        raise ValueError("row_ptr must be 1-D with n + 1 entries, col_ind 1-D")
    if rp.dtype in (np.uint32, np.int32):
        rp = rp.view(np.uint32)
        flags |= CSR_OFFSETS32
    else:
        rp = np.ascontiguousarray(rp, dtype=np.uint64)
    ci = ci.view(np.uint32) if ci.dtype in (np.uint32, np.int32) else np.ascontiguousarray(ci, dtype=np.uint32)
    csr = _Csr(rp.shape[0] - 1, ci.shape[0], rp.ctypes.data, ci.ctypes.data, flags)
    return csr, (rp, ci), None


def count(row_ptr, col_ind, s: int = 5, a: int = 8192, *, oriented: bool = True,
          device: Optional[int] = None, validate: bool = False,
          wedge_begin: int = 0, wedge_end: int = 0, block: int = 0,
          l2_persist: bool = False, stream=None, kernel: int = 0,
          keep_u64_offsets: bool = False, one_pass: bool = False,
          core_len: int = 0, shell_len: int = 0,
          pair_streams: bool = True) -> Tuple[int, Stats]:
    """Exact triangle count of a CSR with spread ``s`` and bitmap length ``a``.

    ``row_ptr``/``col_ind`` are numpy arrays (host; copied to the GPU inside
    the call) or CUDA torch tensors (device-resident). ``oriented=False``
    takes a symmetric adjacency and orients it on the device first. With a
    wedge range only the triangles closed by those wedges are counted.
    ``stream`` is a ``torch.cuda.Stream`` (or raw handle) to run on.
    ``kernel`` picks the count kernel (``wetric_opts.kernel``: 0 = the
    default, 8, the row walk with long-row segments and 16-bit near hash
    sets; 1-7 the earlier variants). ``core_len`` sizes the dense core
    (``wetric_opts.core_len``: 0 = chosen by the library, :data:`CORE_OFF` =
    none, else that many top vertices counted by row ANDs) and ``shell_len``
    the shell below it (0 = none). ``pair_streams=False`` turns off the
    pair streams for short rows (``WETRIC_OPT_NO_PAIR_STREAMS``). A host CSR of
    2^22 columns or more is copied in row chunks, highest rows first, and
    counted as it arrives.
    """
    csr, keep, dev = _csr_struct(row_ptr, col_ind, oriented)
    o = _Opts()
    _opts_init(C.byref(o))
    o.spread, o.bitmap_len, o.block = s, a, block
    o.validate = int(validate)
    o.wedge_begin, o.wedge_end = wedge_begin, wedge_end
    o.device = device if device is not None else (dev or 0)
    o.l2_persist = int(l2_persist)
    o.kernel = kernel
    o.core_len = core_len
    o.shell_len = shell_len
    o.opt_flags = ((OPT_KEEP_U64_OFFSETS if keep_u64_offsets else 0)
                   | (OPT_ONE_PASS if one_pass else 0)
                   | (0 if pair_streams else OPT_NO_PAIR_STREAMS))
    if stream is not None:
        o.stream = getattr(stream, "cuda_stream", stream)
    out = C.c_uint64(0)
    st = _Stats()
    rc = _count_ex(C.byref(csr), C.byref(o), C.byref(out), C.byref(st))
    del keep
    _check(rc, "count")
    return int(out.value), _stats(st)


def count_simple(row_ptr, col_ind, s: int = 5, a: int = 8192) -> int:
    """wetric_count: the plain C entry point (UINT64_MAX on error -> raises)."""
    csr, keep, _ = _csr_struct(row_ptr, col_ind, True)
    r = _count(C.byref(csr), s, a)
    del keep
    if r == (1 << 64) - 1:
        _raise(what="wetric_count")
    return int(r)


def wedge_total(row_ptr, device: int = 0) -> Tuple[int, int]:
    """(W, max out-degree) of a device oriented CSR (torch row offsets)."""
    import torch

    n = row_ptr.numel() - 1
    flags = CSR_ORIENTED | CSR_DEVICE
    if row_ptr.dtype in (torch.int32, torch.uint32):
        flags |= CSR_OFFSETS32
    csr = _Csr(n, 0, row_ptr.data_ptr(), None, flags)
    W, md = C.c_uint64(0), C.c_uint64(0)
    _check(_wedge_total(C.byref(csr), device, C.byref(W), C.byref(md)), "wedge_total")
    return int(W.value), int(md.value)


def algorithmic_bytes(row_ptr, col_ind, device: int = 0) -> int:
    """Algorithmic bytes of the wedge-check count on a device oriented CSR."""
    csr, keep, _ = _csr_struct(row_ptr, col_ind, True)
    out = C.c_uint64(0)
    _check(_alg_bytes(C.byref(csr), device, C.byref(out)), "algorithmic_bytes")
    del keep
    return int(out.value)


# ----------------------------------------------- device preprocessing handle


class OrientedGraph:
    """An oriented CSR in libwetric-owned device memory (wetric_orient_edges)."""

    def __init__(self, handle: int, stats: Stats):
        self._h = C.c_void_p(handle)
        self.stats = stats
        csr = _Csr()
        _check(_oriented_csr(self._h, C.byref(csr)), "oriented_csr")
        self.n, self.m = int(csr.n), int(csr.m)
        self.row_ptr_ptr, self.col_ind_ptr = csr.row_ptr, csr.col_ind

    def csr(self) -> _Csr:
        return _Csr(self.n, self.m, self.row_ptr_ptr, self.col_ind_ptr,
                    CSR_ORIENTED | CSR_DEVICE)

    def count(self, s: int = 5, a: int = 8192, device: int = 0, **kw) -> Tuple[int, Stats]:
        o = _Opts()
        _opts_init(C.byref(o))
        o.spread, o.bitmap_len, o.device = s, a, device
        o.block = kw.get("block", 0)
        o.wedge_begin = kw.get("wedge_begin", 0)
        o.wedge_end = kw.get("wedge_end", 0)
        o.validate = int(kw.get("validate", False))
        o.l2_persist = int(kw.get("l2_persist", False))
        o.kernel = kw.get("kernel", 0)
        o.core_len = kw.get("core_len", 0)
        o.shell_len = kw.get("shell_len", 0)
        o.opt_flags = ((OPT_KEEP_U64_OFFSETS if kw.get("keep_u64_offsets") else 0)
                       | (OPT_ONE_PASS if kw.get("one_pass") else 0)
                       | (0 if kw.get("pair_streams", True) else OPT_NO_PAIR_STREAMS))
        stream = kw.get("stream")
        if stream is not None:
            o.stream = getattr(stream, "cuda_stream", stream)
        csr = self.csr()
        out, st = C.c_uint64(0), _Stats()
        _check(_count_ex(C.byref(csr), C.byref(o), C.byref(out), C.byref(st)), "count")
        return int(out.value), _stats(st)

    def download(self) -> Graph:
        rp = np.empty(self.n + 1, np.uint64)
        ci = np.empty(max(self.m, 1), np.uint32)
        _check(_oriented_download(self._h, rp.ctypes.data, ci.ctypes.data), "download")
        return Graph(rp, ci[: self.m])

    def free(self) -> None:
        if self._h:
            _oriented_free(self._h)
            self._h = C.c_void_p(None)

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


def orient_edges(src, dst, n: int = 0, device: int = 0) -> OrientedGraph:
    """Raw 0-based pairs (numpy host or torch CUDA) -> device oriented CSR.
    Self-loops dropped, direction and duplicates ignored; n = max id + 1
    unless given."""
    flags = 0
    if _is_torch(src):
        flags = CSR_DEVICE
        sp, dp, P = src.data_ptr(), dst.data_ptr(), src.numel()
        keep = (src, dst)
    else:
        s = np.ascontiguousarray(src, dtype=np.uint32)
        d = np.ascontiguousarray(dst, dtype=np.uint32)
        sp, dp, P = s.ctypes.data, d.ctypes.data, s.shape[0]
        keep = (s, d)
    h = C.c_void_p()
    st = _Stats()
    rc = _orient_edges(sp, dp, P, n, flags, device, C.byref(h), C.byref(st))
    del keep
    _check(rc, "orient_edges")
    return OrientedGraph(h.value, _stats(st))


# ---------------------------------------------------------------- generators


def gen_rmat(scale: int, edges: int, a: float = 0.57, b: float = 0.19,
             c: float = 0.19, seed: int = 1) -> Tuple[np.ndarray, np.ndarray]:
    """Seeded R-MAT pairs on the host (identical to :func:`gen_rmat_device`)."""
    src = np.empty(edges, np.uint32)
    dst = np.empty(edges, np.uint32)
    _check(_gen_rmat(scale, edges, a, b, c, seed, src.ctypes.data, dst.ctypes.data),
           "gen_rmat")
    return src, dst


def gen_rmat_device(scale: int, edges: int, a: float = 0.57, b: float = 0.19,
                    c: float = 0.19, seed: int = 1, device: int = 0):
    """The same R-MAT pairs written into CUDA torch tensors."""
    import torch

    src = torch.empty(edges, dtype=torch.int32, device=f"cuda:{device}")
    dst = torch.empty(edges, dtype=torch.int32, device=f"cuda:{device}")
    torch.cuda.synchronize(device)
    _check(_gen_rmat_dev(scale, edges, a, b, c, seed, src.data_ptr(),
                         dst.data_ptr(), device), "gen_rmat_device")
    return src, dst


def chung_lu_cdf(n: int, gamma: float, i0: float) -> np.ndarray:
    cdf = np.empty(n, np.uint64)
    _check(_chung_lu_cdf(n, gamma, i0, cdf.ctypes.data), "chung_lu_cdf")
    return cdf


def gen_weighted(cdf: Optional[np.ndarray], n: int, edges: int,
                 seed: int = 1) -> Tuple[np.ndarray, np.ndarray]:
    """Chung-Lu (cdf given) or Erdos-Renyi (cdf None) pairs on the host."""
    src = np.empty(edges, np.uint32)
    dst = np.empty(edges, np.uint32)
    cp = None
    if cdf is not None:
        cdf = np.ascontiguousarray(cdf, dtype=np.uint64)
        cp = cdf.ctypes.data
    _check(_gen_weighted(cp, n, edges, seed, src.ctypes.data, dst.ctypes.data),
           "gen_weighted")
    return src, dst


def gen_weighted_device(cdf, n: int, edges: int, seed: int = 1, device: int = 0):
    """Device form of :func:`gen_weighted` (cdf: numpy, copied, or None)."""
    import torch

    dev = f"cuda:{device}"
    cdf_t = None
    if cdf is not None:
        cdf_t = torch.from_numpy(np.ascontiguousarray(cdf, dtype=np.uint64).view(np.int64)).to(dev)
    src = torch.empty(edges, dtype=torch.int32, device=dev)
    dst = torch.empty(edges, dtype=torch.int32, device=dev)
    torch.cuda.synchronize(device)
    _check(_gen_weighted_dev(cdf_t.data_ptr() if cdf_t is not None else None, n,
                             edges, seed, src.data_ptr(), dst.data_ptr(), device),
           "gen_weighted_device")
    return src, dst


def write_mm(path: str, n: int, src: np.ndarray, dst: np.ndarray) -> None:
    """Pairs -> 'coordinate pattern symmetric' Matrix Market file (1-based)."""
    s = np.ascontiguousarray(src, dtype=np.uint32)
    d = np.ascontiguousarray(dst, dtype=np.uint32)
    _check(_write_mm(os.fsencode(path), n, s.ctypes.data, d.ctypes.data, s.shape[0]),
           "write_mm")


_parse_file = _sig(
    "wetric_parse_file", C.c_int, C.c_char_p, C.c_int, C.c_int,
    C.POINTER(C.POINTER(C.c_uint32)), C.POINTER(C.POINTER(C.c_uint32)),
    C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)
)
_free_buffer = _sig("wetric_free_buffer", None, C.c_void_p)


def parse_file(path: str, matrix_market: bool = False,
               zero_indexed: bool = False) -> Tuple[np.ndarray, np.ndarray, int]:
    """Host-only parse with the input rules of :func:`read_graph`: returns
    0-based non-loop pairs and n = max id + 1."""
    ps, pd = C.POINTER(C.c_uint32)(), C.POINTER(C.c_uint32)()
    cnt, n = C.c_uint64(0), C.c_uint64(0)
    rc = _parse_file(os.fsencode(path), int(matrix_market), int(zero_indexed),
                     C.byref(ps), C.byref(pd), C.byref(cnt), C.byref(n))
    if rc != OK:
        raise WetricError(rc, f"parse_file: {_strerror(rc).decode()}")
    k = int(cnt.value)
    try:
        src = np.ctypeslib.as_array(ps, shape=(k,)).copy() if k else np.zeros(0, np.uint32)
        dst = np.ctypeslib.as_array(pd, shape=(k,)).copy() if k else np.zeros(0, np.uint32)
    finally:
        _free_buffer(C.cast(ps, C.c_void_p))
        _free_buffer(C.cast(pd, C.c_void_p))
    return src, dst, int(n.value)


_save_csr = _sig("wetric_save_csr", C.c_int, C.c_char_p, C.POINTER(_Csr))
_load_csr = _sig("wetric_load_csr", C.c_int, C.c_char_p, C.POINTER(_Csr))


def save_csr(path: str, row_ptr, col_ind, oriented: bool = True) -> None:
    """Writes a host CSR (numpy; u64 or u32 offsets) to the binary cache
    read by :func:`load_csr` (wetric_save_csr)."""
    rp = np.ascontiguousarray(row_ptr)
    if rp.dtype not in (np.uint64, np.int64, np.uint32, np.int32):
        rp = rp.astype(np.uint64)
    ci = np.ascontiguousarray(col_ind, dtype=np.uint32)
    c = _Csr()
    c.n, c.m = rp.shape[0] - 1, ci.shape[0]
    c.row_ptr = rp.ctypes.data
    c.col_ind = ci.ctypes.data
    c.flags = (CSR_ORIENTED if oriented else CSR_SYMMETRIC) | (
        CSR_OFFSETS32 if rp.dtype.itemsize == 4 else 0)
    _check(_save_csr(os.fsencode(path), C.byref(c)), "save_csr")


def load_csr(path: str) -> Tuple[np.ndarray, np.ndarray, bool]:
    """(row_ptr u64, col_ind u32, oriented) from a binary cache file
    (wetric_load_csr); the file is checked against its header and the CSR."""
    c = _Csr()
    _check(_load_csr(os.fsencode(path), C.byref(c)), "load_csr")
    n, m = int(c.n), int(c.m)
    try:
        rp = np.ctypeslib.as_array(C.cast(c.row_ptr, C.POINTER(C.c_uint64)), shape=(n + 1,)).copy()
        ci = (np.ctypeslib.as_array(C.cast(c.col_ind, C.POINTER(C.c_uint32)), shape=(m,)).copy()
              if m else np.zeros(0, np.uint32))
    finally:
        _free_buffer(C.cast(c.row_ptr, C.c_void_p))
        _free_buffer(C.cast(c.col_ind, C.c_void_p))
    return rp, ci, bool(c.flags & CSR_ORIENTED)


# ------------------------------------------------------------------ batches


class _BatchOpts(C.Structure):
    _fields_ = [
        ("spread", C.c_uint32),
        ("bitmap_len", C.c_uint32),
        ("use_cuda_graph", C.c_uint32),
        ("autotune", C.c_uint32),
        ("bitmap_cap_bytes", C.c_uint64),
        ("no_pair_streams", C.c_uint32),
    ]


_batch_opts_init = _sig("wetric_batch_opts_init", None, C.POINTER(_BatchOpts))
_batch_create = _sig(
    "wetric_batch_create", C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
    C.c_uint32, C.c_uint32, C.c_int, C.POINTER(_BatchOpts), C.POINTER(C.c_void_p)
)
_batch_count = _sig("wetric_batch_count", C.c_int, C.c_void_p, C.c_void_p, C.POINTER(_Stats))
_batch_info = _sig("wetric_batch_info", C.c_int, C.c_void_p, C.c_void_p, C.c_void_p)
_batch_spreads = _sig("wetric_batch_spreads", C.c_int, C.c_void_p, C.c_void_p)
_batch_free = _sig("wetric_batch_free", None, C.c_void_p)


class Batch:
    """Many graphs preprocessed once, kept on the device and counted by one
    persistent launch (wetric_batch_*).

    ``src``/``dst`` hold every graph's 0-based pairs back to back (numpy or
    CUDA torch), ``pair_off`` (G+1) delimits them and ``n`` (G) gives each
    graph's vertex count. ``spread=0`` picks s per graph size, or, with
    ``autotune=True``, per size/skew bucket by timing candidate spreads (the
    results are kept per device and reused by later batches).
    ``pair_streams=False`` counts every short row by wedge checks too.
    """

    def __init__(self, src, dst, pair_off, n, device: int = 0, spread: int = 5,
                 a: int = 8192, use_cuda_graph: bool = True, bitmap_cap_bytes: int = 0,
                 autotune: bool = False, pair_streams: bool = True):
        po = np.ascontiguousarray(pair_off, dtype=np.uint64)
        nn = np.ascontiguousarray(n, dtype=np.uint64)
        self.G = int(nn.shape[0])
        assert po.shape[0] == self.G + 1
        flags = 0
        if _is_torch(src):
            flags = CSR_DEVICE
            sp, dp, keep = src.data_ptr(), dst.data_ptr(), (src, dst)
        else:
            s_ = np.ascontiguousarray(src, dtype=np.uint32)
            d_ = np.ascontiguousarray(dst, dtype=np.uint32)
            sp, dp, keep = s_.ctypes.data, d_.ctypes.data, (s_, d_)
        o = _BatchOpts()
        _batch_opts_init(C.byref(o))
        o.spread, o.bitmap_len = spread, a
        o.use_cuda_graph = int(use_cuda_graph)
        o.bitmap_cap_bytes = bitmap_cap_bytes
        o.autotune = int(autotune)
        o.no_pair_streams = int(not pair_streams)
        h = C.c_void_p()
        rc = _batch_create(sp, dp, po.ctypes.data, nn.ctypes.data, self.G, flags,
                           device, C.byref(o), C.byref(h))
        del keep
        _check(rc, "batch_create")
        self._h = h

    def count(self) -> Tuple[np.ndarray, Stats]:
        out = np.zeros(self.G, np.uint64)
        st = _Stats()
        _check(_batch_count(self._h, out.ctypes.data, C.byref(st)), "batch_count")
        return out, _stats(st)

    def info(self) -> Tuple[np.ndarray, np.ndarray]:
        w = np.zeros(self.G, np.uint64)
        e = np.zeros(self.G, np.uint64)
        _check(_batch_info(self._h, w.ctypes.data, e.ctypes.data), "batch_info")
        return w, e

    def spreads(self) -> np.ndarray:
        """The spread s_g each graph is counted with."""
        out = np.zeros(self.G, np.uint32)
        _check(_batch_spreads(self._h, out.ctypes.data), "batch_spreads")
        return out

    def free(self) -> None:
        if self._h:
            _batch_free(self._h)
            self._h = C.c_void_p(None)

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


# ------------------------------------------------------------------ serving


class _ServerOpts(C.Structure):
    _fields_ = [
        ("hbm_budget", C.c_uint64),
        ("max_batch_pairs", C.c_uint64),
        ("max_batch_graphs", C.c_uint32),
        ("spread", C.c_uint32),
        ("bitmap_len", C.c_uint32),
        ("queue_capacity", C.c_uint32),
        ("large_pairs", C.c_uint64),
        ("reserve_bytes", C.c_uint64),
        ("resident", C.c_uint32),
        ("item_tiles", C.c_uint32),
    ]


class _ServerStats(C.Structure):
    _fields_ = [
        ("completed", C.c_uint64),
        ("failed", C.c_uint64),
        ("batches", C.c_uint64),
        ("waiting", C.c_uint64),
        ("admitted_bytes", C.c_uint64),
        ("mean_batch_graphs", C.c_double),
        ("p50_ms", C.c_double),
        ("p99_ms", C.c_double),
        ("count_busy_ms", C.c_double),
        ("admit_busy_ms", C.c_double),
        ("pairs_admitted", C.c_uint64),
        ("queue_p50_ms", C.c_double),
        ("small_p50_ms", C.c_double),
        ("small_p99_ms", C.c_double),
        ("large_p50_ms", C.c_double),
        ("large_p99_ms", C.c_double),
        ("large_completed", C.c_uint64),
        ("resident_launches", C.c_uint64),
        ("recycles", C.c_uint64),
        ("resident_last_exit", C.c_uint32),
        ("launch_error_code", C.c_uint32),
        ("live", C.c_uint64),
        ("feeding", C.c_uint64),
        ("items_published", C.c_uint64),
        ("items_taken", C.c_uint64),
        ("draining", C.c_uint32),
        ("launch_errors", C.c_uint32),
        ("lane_phase", C.c_uint32 * 2),
    ]


_server_opts_init = _sig("wetric_server_opts_init", None, C.POINTER(_ServerOpts))
_server_create = _sig("wetric_server_create", C.c_int, C.c_int, C.POINTER(_ServerOpts),
                      C.POINTER(C.c_void_p))
_server_submit = _sig("wetric_server_submit", C.c_int, C.c_void_p, C.c_void_p, C.c_void_p,
                      C.c_uint64, C.c_uint64, C.c_uint32, C.POINTER(C.c_uint64))
_server_submit_csr = _sig("wetric_server_submit_csr", C.c_int, C.c_void_p, C.POINTER(_Csr),
                          C.POINTER(C.c_uint64))
_server_poll = _sig("wetric_server_poll", C.c_int, C.c_void_p, C.c_uint64,
                    C.POINTER(C.c_uint64), C.POINTER(C.c_double))
_server_wait = _sig("wetric_server_wait", C.c_int, C.c_void_p, C.c_uint64, C.c_uint32,
                    C.POINTER(C.c_uint64), C.POINTER(C.c_double))
_server_stats = _sig("wetric_server_get_stats", C.c_int, C.c_void_p, C.POINTER(_ServerStats))
_server_destroy = _sig("wetric_server_destroy", None, C.c_void_p)


class Server:
    """A counting service (wetric_server_*): submit graphs any time, get
    exact counts back; requests are admitted against an HBM budget and
    batched per lane (the default), or, with ``resident=True``, folded into
    the resident counting kernel's work queue as soon as they are
    preprocessed. Submitted buffers must stay alive until their ticket
    completes (the object keeps a reference until then)."""

    def __init__(self, device: int = 0, hbm_budget: int = 0, max_batch_graphs: int = 0,
                 max_batch_pairs: int = 0, spread: int = 5, a: int = 8192,
                 queue_capacity: int = 0, large_pairs: Optional[int] = None,
                 resident: bool = False, item_tiles: int = 0):
        o = _ServerOpts()
        _server_opts_init(C.byref(o))
        if hbm_budget:
            o.hbm_budget = hbm_budget
        if max_batch_graphs:
            o.max_batch_graphs = max_batch_graphs
        if max_batch_pairs:
            o.max_batch_pairs = max_batch_pairs
        if queue_capacity:
            o.queue_capacity = queue_capacity
        o.spread, o.bitmap_len = spread, a
        if large_pairs is not None:
            o.large_pairs = large_pairs
        o.resident = int(resident)
        if item_tiles:
            o.item_tiles = item_tiles
        h = C.c_void_p()
        _check(_server_create(device, C.byref(o), C.byref(h)), "server_create")
        self._h = h
        self._keep = {}

    def submit(self, src, dst, n: int) -> int:
        if _is_torch(src):
            flags, sp, dp, P = CSR_DEVICE, src.data_ptr(), dst.data_ptr(), src.numel()
            keep = (src, dst)
        else:
            s_ = np.ascontiguousarray(src, dtype=np.uint32)
            d_ = np.ascontiguousarray(dst, dtype=np.uint32)
            flags, sp, dp, P = 0, s_.ctypes.data, d_.ctypes.data, s_.shape[0]
            keep = (s_, d_)
        t = C.c_uint64(0)
        _check(_server_submit(self._h, sp, dp, P, n, flags, C.byref(t)), "server_submit")
        self._keep[int(t.value)] = keep
        return int(t.value)

    def submit_csr(self, row_ptr, col_ind, oriented: bool = True) -> int:
        """Submits a graph given as a CSR (numpy or CUDA torch arrays; u64 or
        u32 offsets); the server copies it before returning."""
        csr, keep, _ = _csr_struct(row_ptr, col_ind, oriented)
        t = C.c_uint64(0)
        rc = _server_submit_csr(self._h, C.byref(csr), C.byref(t))
        del keep
        _check(rc, "server_submit_csr")
        return int(t.value)

    def poll(self, ticket: int):
        """(count, latency_ms), or None while pending."""
        c, lat = C.c_uint64(0), C.c_double(0)
        rc = _server_poll(self._h, ticket, C.byref(c), C.byref(lat))
        if rc == EBUSY:
            return None
        self._keep.pop(ticket, None)
        _check(rc, "server_poll")
        return int(c.value), float(lat.value)

    def wait(self, ticket: int, timeout_ms: int = 60000):
        c, lat = C.c_uint64(0), C.c_double(0)
        rc = _server_wait(self._h, ticket, timeout_ms, C.byref(c), C.byref(lat))
        if rc != ETIMEDOUT:
            self._keep.pop(ticket, None)
        _check(rc, "server_wait")
        return int(c.value), float(lat.value)

    def stats(self) -> dict:
        st = _ServerStats()
        _check(_server_stats(self._h, C.byref(st)), "server_stats")
        out = {f: getattr(st, f) for f, _ in _ServerStats._fields_}
        out["lane_phase"] = list(st.lane_phase)
        return out

    def close(self) -> None:
        if self._h:
            _server_destroy(self._h)
            self._h = C.c_void_p(None)
            self._keep.clear()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


from . import workloads  # noqa: E402,F401  (seeded workload definitions)
