"""tdfs_b200 -- B200-native subgraph enumeration (drop-in for lyuheng/tdfs).

Python mirror of the reference's host interface over the C ABI of
libtdfs_b200.so (include/tdfs.h):

* ``GraphPreprocessor(prefix, labeled)`` -- reads the reference's binary CSR
  files and keeps the graph resident on the GPU (src/graph.h:26-50).
* ``PatternPreprocessor(gfile, labeled)`` -- compiles a ``.g`` pattern into a
  plan table (src/pattern.h:90-108).
* ``count(graph, pattern)`` -- one launch of the DFS kernel; returns the count
  ``ulb``/``lb`` print (cu_test.cu:81-107).

There is no CPU execution path: every count runs the sm_100a kernels, and the
module raises ``TdfsError`` when the library or a GPU is missing.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "lib", "libtdfs_b200.so")
BIN_DIR = os.path.join(_HERE, "bin")
CONVERT = os.path.join(BIN_DIR, "tdfs_convert")  # host-only graph writer / converter

ERR_NAMES = {1: "IO", 2: "FORMAT", 3: "PATTERN", 4: "CUDA", 5: "CAPACITY", 6: "TIMEOUT", 7: "ARG",
             8: "ADMISSION"}

# every symbol include/tdfs.h declares (checked by the CPU tests)
EXPORTS = [
    "tdfs_last_error", "tdfs_version", "tdfs_options_default",
    "tdfs_graph_open", "tdfs_graph_from_csr", "tdfs_graph_info", "tdfs_graph_free",
    "tdfs_plan_compile", "tdfs_plan_from_text", "tdfs_plan_dump", "tdfs_plan_info", "tdfs_plan_free",
    "tdfs_count", "tdfs_count_batch", "tdfs_count_batch_status", "tdfs_selftest_wait_limit",
    "tdfs_last_launch",
    "tdfs_csr_read", "tdfs_csr_view", "tdfs_csr_write", "tdfs_csr_set_labels", "tdfs_csr_free",
    "tdfs_csr_from_arrays", "tdfs_csr_relabel", "tdfs_csr_halve",
    "tdfs_gen_er", "tdfs_gen_chung_lu", "tdfs_gen_rmat", "tdfs_gen_pattern", "tdfs_estimate",
    "tdfs_autotune", "tdfs_count_static", "tdfs_server_options_default", "tdfs_server_create", "tdfs_server_submit", "tdfs_server_wait",
    "tdfs_server_stats", "tdfs_server_destroy",
]


class TdfsError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"TDFS_ERR_{ERR_NAMES.get(code, code)}: {msg}")
        self.code = code


class Options(C.Structure):
    """Launch knobs (tdfs_options)."""
    _fields_ = [
        ("warps_per_block", C.c_int),
        ("blocks_per_sm", C.c_int),
        ("chunk_cap", C.c_int),
        ("steal", C.c_int),
        ("merge_window", C.c_int),
        ("edge_begin", C.c_int64),
        ("edge_end", C.c_int64),
        ("edge_stride", C.c_int),
        ("edge_phase", C.c_int),
        ("stream", C.c_void_p),
        ("steal_min", C.c_int),
        ("merge_ratio", C.c_int),
        ("graph_capture", C.c_int),
        ("edge_chunk", C.c_int),
        ("fixed_stage", C.c_int),
        ("split_after_us", C.c_int),
        ("steal_first", C.c_int),
        ("lane_list", C.c_int),
        ("work_budget", C.c_int64),
        ("wait_limit_ms", C.c_int),
        ("split_rush_us", C.c_int),
        ("leaf_steal_min", C.c_int),
        ("label_index", C.c_int),
        ("level_hoist", C.c_int),
        ("label_rows", C.c_int),
        ("tail_count", C.c_int),
        ("dead_prune", C.c_int),
    ]


class ServerOptions(C.Structure):
    """tdfs_server_options."""
    _fields_ = [
        ("max_inflight", C.c_int),
        ("max_k", C.c_int),
        ("labeled", C.c_int),
        ("idle_exit_ms", C.c_int),
        ("mem_budget", C.c_size_t),
        ("launch", Options),
    ]


class ServeStats(C.Structure):
    """tdfs_serve_stats."""
    _fields_ = [
        ("completed", C.c_uint64),
        ("pending", C.c_uint64),
        ("inflight", C.c_uint64),
        ("p50_us", C.c_double),
        ("p99_us", C.c_double),
        ("max_us", C.c_double),
        ("queries_per_s", C.c_double),
        ("aborted", C.c_uint64),
    ]


_lib = None


def lib() -> C.CDLL:
    """Load libtdfs_b200.so (fails loudly when it was not built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise TdfsError(4, f"{LIB_PATH} not built; run `python -m tdfs_b200.build`")
    L = C.CDLL(LIB_PATH)
    vp, i64, i32, ci = C.c_void_p, C.c_int64, C.c_int32, C.c_int
    pp = C.POINTER(C.c_void_p)
    L.tdfs_last_error.restype = C.c_char_p
    L.tdfs_options_default.argtypes = [C.POINTER(Options)]
    L.tdfs_options_default.restype = None
    L.tdfs_graph_open.argtypes = [C.c_char_p, ci, ci, pp]
    L.tdfs_graph_from_csr.argtypes = [i64, i64, vp, vp, vp, ci, pp]
    L.tdfs_graph_info.argtypes = [vp, C.POINTER(i64), C.POINTER(i64), C.POINTER(i32), C.POINTER(ci),
                                  C.POINTER(C.c_size_t)]
    L.tdfs_graph_free.argtypes = [vp]
    L.tdfs_plan_compile.argtypes = [C.c_char_p, ci, pp]
    L.tdfs_plan_from_text.argtypes = [C.c_char_p, ci, pp]
    L.tdfs_plan_dump.argtypes = [vp, C.c_char_p, C.c_size_t, C.POINTER(C.c_size_t)]
    L.tdfs_plan_info.argtypes = [vp, C.POINTER(ci), C.POINTER(ci), C.POINTER(i64)]
    L.tdfs_plan_free.argtypes = [vp]
    L.tdfs_count.argtypes = [vp, vp, C.POINTER(Options), C.POINTER(C.c_uint64), C.POINTER(C.c_float)]
    L.tdfs_count_batch.argtypes = [vp, C.POINTER(vp), ci, C.POINTER(Options), C.POINTER(C.c_uint64),
                                   C.POINTER(C.c_float)]
    L.tdfs_count_batch_status.argtypes = [vp, C.POINTER(vp), ci, C.POINTER(Options), C.POINTER(C.c_uint64),
                                          C.POINTER(ci), C.POINTER(C.c_float)]
    L.tdfs_selftest_wait_limit.argtypes = [vp, ci, C.POINTER(C.c_float)]
    L.tdfs_last_launch.argtypes = [vp, vp]
    L.tdfs_csr_read.argtypes = [C.c_char_p, ci, pp]
    L.tdfs_csr_view.argtypes = [vp, C.POINTER(i64), C.POINTER(i64), pp, pp, pp, C.POINTER(i32)]
    L.tdfs_csr_write.argtypes = [vp, C.c_char_p]
    L.tdfs_csr_set_labels.argtypes = [vp, ci, C.c_uint64]
    L.tdfs_csr_free.argtypes = [vp]
    L.tdfs_csr_from_arrays.argtypes = [i64, i64, vp, vp, vp, pp]
    L.tdfs_csr_relabel.argtypes = [vp, pp]
    L.tdfs_csr_halve.argtypes = [vp, pp]
    L.tdfs_gen_er.argtypes = [i64, C.c_double, C.c_uint64, pp]
    L.tdfs_gen_chung_lu.argtypes = [i64, i64, C.c_double, i32, C.c_uint64, pp]
    L.tdfs_gen_rmat.argtypes = [ci, ci, C.c_double, C.c_double, C.c_double, C.c_uint64, pp]
    L.tdfs_gen_pattern.argtypes = [ci, C.c_double, ci, C.c_uint64, C.c_char_p, C.c_size_t]
    L.tdfs_estimate.argtypes = [vp, vp, i64, i64, i64, C.c_uint64, vp]
    L.tdfs_autotune.argtypes = [vp, C.POINTER(vp), ci, C.POINTER(Options), ci, C.POINTER(Options),
                                C.POINTER(C.c_float)]
    L.tdfs_count_static.argtypes = [ci, i64, i64, vp, vp, vp, vp, C.POINTER(Options), C.POINTER(C.c_uint64)]
    L.tdfs_server_options_default.argtypes = [C.POINTER(ServerOptions)]
    L.tdfs_server_options_default.restype = None
    L.tdfs_server_create.argtypes = [vp, C.POINTER(ServerOptions), pp]
    L.tdfs_server_submit.argtypes = [vp, vp, C.POINTER(C.c_uint64)]
    L.tdfs_server_wait.argtypes = [vp, C.c_uint64, C.POINTER(C.c_uint64), C.POINTER(C.c_double)]
    L.tdfs_server_stats.argtypes = [vp, C.POINTER(ServeStats)]
    L.tdfs_server_destroy.argtypes = [vp]
    _lib = L
    return L


def _check(rc: int):
    if rc:
        raise TdfsError(rc, lib().tdfs_last_error().decode())


def default_options(**kw) -> Options:
    o = Options()
    lib().tdfs_options_default(C.byref(o))
    for k, v in kw.items():
        setattr(o, k, v)
    return o


# --------------------------------------------------------------------------
# host CSR graphs (generators and the reference file format)
# --------------------------------------------------------------------------

class HostCSR:
    """Host CSR owned by the library; numpy views share its memory."""

    def __init__(self, handle: C.c_void_p):
        self._h = handle
        n, e, md = C.c_int64(), C.c_int64(), C.c_int32()
        rp, ci, lb = C.c_void_p(), C.c_void_p(), C.c_void_p()
        _check(lib().tdfs_csr_view(handle, C.byref(n), C.byref(e), C.byref(rp), C.byref(ci), C.byref(lb),
                                   C.byref(md)))
        self.n, self.nedges, self.max_degree = n.value, e.value, md.value
        self.rowptr = np.ctypeslib.as_array(C.cast(rp, C.POINTER(C.c_int64)), shape=(self.n + 1,))
        self.colidx = (np.ctypeslib.as_array(C.cast(ci, C.POINTER(C.c_int32)), shape=(self.nedges,))
                       if self.nedges else np.zeros(0, np.int32))
        self.labels = (np.ctypeslib.as_array(C.cast(lb, C.POINTER(C.c_int32)), shape=(self.n,))
                       if lb.value else None)

    def set_labels(self, nlabels: int, seed: int) -> "HostCSR":
        _check(lib().tdfs_csr_set_labels(self._h, nlabels, seed))
        self.__init__(self._h)
        return self

    def write(self, prefix: str):
        _check(lib().tdfs_csr_write(self._h, prefix.encode()))

    def relabel(self) -> "HostCSR":
        """Descending-degree relabelling (graph_converter/relabel.cpp:11-71)."""
        h = C.c_void_p()
        _check(lib().tdfs_csr_relabel(self._h, C.byref(h)))
        return HostCSR(h)

    def halve(self) -> "HostCSR":
        """Degree orientation: one direction of every edge
        (graph_converter/halve.cpp:10-42)."""
        h = C.c_void_p()
        _check(lib().tdfs_csr_halve(self._h, C.byref(h)))
        return HostCSR(h)

    def __del__(self):
        if getattr(self, "_h", None) and _lib is not None:
            _lib.tdfs_csr_free(self._h)
            self._h = None


def csr_from_arrays(rowptr, colidx, labels=None) -> HostCSR:
    """Host CSR copied from arrays (int64 rowptr, int32 colidx, optional
    int32 labels), checked like the file reader."""
    rowptr = np.ascontiguousarray(rowptr, dtype=np.int64)
    colidx = np.ascontiguousarray(colidx, dtype=np.int32)
    lab = None if labels is None else np.ascontiguousarray(labels, dtype=np.int32)
    h = C.c_void_p()
    _check(lib().tdfs_csr_from_arrays(len(rowptr) - 1, len(colidx), rowptr.ctypes.data, colidx.ctypes.data,
                                      None if lab is None else lab.ctypes.data, C.byref(h)))
    return HostCSR(h)


def read_csr(prefix: str, labeled: bool = False) -> HostCSR:
    h = C.c_void_p()
    _check(lib().tdfs_csr_read(prefix.encode(), int(labeled), C.byref(h)))
    return HostCSR(h)


def gen_er(n: int, avg_degree: float, seed: int) -> HostCSR:
    h = C.c_void_p()
    _check(lib().tdfs_gen_er(n, avg_degree, seed, C.byref(h)))
    return HostCSR(h)


def gen_chung_lu(n: int, undirected_edges: int, gamma: float, max_degree: int, seed: int) -> HostCSR:
    h = C.c_void_p()
    _check(lib().tdfs_gen_chung_lu(n, undirected_edges, gamma, max_degree, seed, C.byref(h)))
    return HostCSR(h)


def gen_rmat(scale: int, edge_factor: int, a: float, b: float, c: float, seed: int) -> HostCSR:
    h = C.c_void_p()
    _check(lib().tdfs_gen_rmat(scale, edge_factor, a, b, c, seed, C.byref(h)))
    return HostCSR(h)


class EstimateResult(C.Structure):
    """Result of tdfs_estimate."""
    _fields_ = [("matches", C.c_double), ("nodes", C.c_double * 7), ("scanned", C.c_double),
                ("matches_rse", C.c_double), ("scanned_rse", C.c_double), ("probes", C.c_int64)]


def estimate(csr: HostCSR, pattern: "PatternPreprocessor", probes: int = 1000, seed: int = 0,
             edge_begin: int = 0, edge_end: int = -1) -> EstimateResult:
    """Expected count and work of a query (tdfs_estimate) over the level-0 edge
    range [edge_begin, edge_end), from random DFS probes over the host copy
    of the graph."""
    r = EstimateResult()
    _check(lib().tdfs_estimate(csr._h, pattern._h, edge_begin, edge_end, probes, seed, C.byref(r)))
    return r


def gen_pattern(k: int, density: float, nlabels: int, seed: int) -> str:
    buf = C.create_string_buffer(1024)
    _check(lib().tdfs_gen_pattern(k, density, nlabels, seed, buf, len(buf)))
    return buf.value.decode()


# --------------------------------------------------------------------------
# reference-shaped front ends
# --------------------------------------------------------------------------

class GraphPreprocessor:
    """Device-resident data graph (src/graph.h:26-50)."""

    def __init__(self, prefix: str | None = None, labeled: bool = False, device: int = 0, *,
                 csr: HostCSR | None = None, rowptr=None, colidx=None, labels=None):
        h = C.c_void_p()
        if prefix is not None:
            _check(lib().tdfs_graph_open(prefix.encode(), int(labeled), device, C.byref(h)))
        else:
            if csr is not None:
                rowptr, colidx = csr.rowptr, csr.colidx
                labels = csr.labels if labeled else None
            rowptr = np.ascontiguousarray(rowptr, dtype=np.int64)
            colidx = np.ascontiguousarray(colidx, dtype=np.int32)
            lab = None if (labels is None or not labeled) else np.ascontiguousarray(labels, dtype=np.int32)
            _check(lib().tdfs_graph_from_csr(len(rowptr) - 1, len(colidx), rowptr.ctypes.data,
                                             colidx.ctypes.data, None if lab is None else lab.ctypes.data,
                                             device, C.byref(h)))
        self._h = h
        n, e, md, lb, by = C.c_int64(), C.c_int64(), C.c_int32(), C.c_int(), C.c_size_t()
        _check(lib().tdfs_graph_info(h, C.byref(n), C.byref(e), C.byref(md), C.byref(lb), C.byref(by)))
        self.n, self.nedges, self.max_degree = n.value, e.value, md.value
        self.labeled, self.device_bytes = bool(lb.value), by.value

    def close(self):
        if getattr(self, "_h", None):
            lib().tdfs_graph_free(self._h)
            self._h = None

    def __del__(self):
        if _lib is not None:
            self.close()


class PatternPreprocessor:
    """Compiled pattern plan (src/pattern.h:90-108)."""

    def __init__(self, gfile: str | None = None, labeled: bool = False, *, text: str | None = None):
        h = C.c_void_p()
        if text is not None:
            _check(lib().tdfs_plan_from_text(text.encode(), int(labeled), C.byref(h)))
        else:
            _check(lib().tdfs_plan_compile(gfile.encode(), int(labeled), C.byref(h)))
        self._h = h
        k, lb, m = C.c_int(), C.c_int(), C.c_int64()
        _check(lib().tdfs_plan_info(h, C.byref(k), C.byref(lb), C.byref(m)))
        self.nnodes, self.labeled, self.PatternMultiplicity = k.value, bool(lb.value), m.value

    def dump(self) -> dict:
        import json
        n = C.c_size_t()
        _check(lib().tdfs_plan_dump(self._h, None, 0, C.byref(n)))
        buf = C.create_string_buffer(n.value)
        _check(lib().tdfs_plan_dump(self._h, buf, n.value, None))
        return json.loads(buf.value.decode())

    def close(self):
        if getattr(self, "_h", None):
            lib().tdfs_plan_free(self._h)
            self._h = None

    def __del__(self):
        if _lib is not None:
            self.close()


@dataclass
class CountResult:
    count: int
    kernel_ms: float


def count(graph: GraphPreprocessor, pattern: PatternPreprocessor, options: Options | None = None) -> CountResult:
    """Count embeddings as ulb/lb would print them."""
    c = C.c_uint64()
    ms = C.c_float()
    _check(lib().tdfs_count(graph._h, pattern._h, None if options is None else C.byref(options), C.byref(c),
                            C.byref(ms)))
    return CountResult(c.value, ms.value)


def count_batch(graph: GraphPreprocessor, patterns, options: Options | None = None):
    """Counts for many patterns; returns (list of counts, kernel ms)."""
    arr = (C.c_void_p * len(patterns))(*[p._h.value for p in patterns])
    out = (C.c_uint64 * len(patterns))()
    ms = C.c_float()
    _check(lib().tdfs_count_batch(graph._h, arr, len(patterns), None if options is None else C.byref(options),
                                  out, C.byref(ms)))
    return list(out), ms.value


def count_batch_status(graph: GraphPreprocessor, patterns, options: Options | None = None):
    """Counts and per-pattern status (0, or the TDFS_ERR_TIMEOUT code when a
    pattern ran out of options.work_budget); returns (counts, status, kernel ms)."""
    n = len(patterns)
    arr = (C.c_void_p * n)(*[p._h.value for p in patterns])
    out = (C.c_uint64 * n)()
    st = (C.c_int * n)()
    ms = C.c_float()
    _check(lib().tdfs_count_batch_status(graph._h, arr, n, None if options is None else C.byref(options), out, st,
                                         C.byref(ms)))
    return list(out), list(st), ms.value


def selftest_wait_limit(graph: GraphPreprocessor, wait_limit_ms: int):
    """Run the match kernel over a slot that can never complete; returns
    (status code the launch reported, kernel ms).  TDFS_ERR_TIMEOUT (6) means
    every warp's bounded wait ran out as designed."""
    ms = C.c_float()
    rc = lib().tdfs_selftest_wait_limit(graph._h, wait_limit_ms, C.byref(ms))
    return rc, ms.value


class LaunchStats(C.Structure):
    """tdfs_launch_stats: diagnostics of the last count launch."""
    _fields_ = [("steals", C.c_uint64), ("splits", C.c_uint64), ("warps", C.c_int64),
                ("idle_fraction", C.c_double), ("mean_warp_ms", C.c_double)]


def last_launch(graph: GraphPreprocessor) -> dict:
    """Steals, split units, grid warps, idle share and mean warp time of the
    last count launch on this graph."""
    st = LaunchStats()
    _check(lib().tdfs_last_launch(graph._h, C.byref(st)))
    return {f: getattr(st, f) for f, _ in LaunchStats._fields_}


EDGE_CHUNK = 32  # directed edges per level-0 ticket (kEdgeChunk in match.cuh)


def shard_options(rank: int, world: int, **kw) -> Options:
    """Options for rank `rank` of `world` GPUs: level-0 edge chunks are dealt
    round-robin, chunk t going to rank t % world, so the ranks' counts sum to
    the whole count with no data-path collective (one u64 reduction).  The
    chunk is 32 edges unless edge_chunk is given; every rank must use the
    same chunk."""
    if not 0 <= rank < world:
        raise ValueError("rank out of range")
    return default_options(edge_stride=world, edge_phase=rank, **kw)


def shard_edge_ranges(nedges: int, rank: int, world: int, chunk: int = EDGE_CHUNK, begin: int = 0):
    """The [begin, end) edge ranges rank `rank` covers under shard_options
    over the level-0 range [begin, nedges) with `chunk`-edge chunks (the
    kernel's ticket t covers begin + (t * world + rank) * chunk)."""
    out = []
    t = 0
    while True:
        b = begin + (t * world + rank) * chunk
        if b >= nedges:
            return out
        out.append((b, min(nedges, b + chunk)))
        t += 1


def count_static(device: int, n: int, nedges: int, d_rowptr: int, d_colidx: int, d_labels: int | None,
                 pattern: PatternPreprocessor, options: Options | None = None) -> int:
    """Count with no device allocation (tdfs_count_static): the graph is
    given as device pointers, the working memory is the library's fixed
    per-GPU array."""
    c = C.c_uint64()
    _check(lib().tdfs_count_static(device, n, nedges, d_rowptr, d_colidx, d_labels, pattern._h,
                                   None if options is None else C.byref(options), C.byref(c)))
    return c.value


def autotune(graph: GraphPreprocessor, patterns, base: Options | None = None, sample_stride: int = 16):
    """Fastest launch options for this graph and batch of patterns, timed on
    every sample_stride-th level-0 chunk.  Returns (Options, sample ms)."""
    arr = (C.c_void_p * len(patterns))(*[p._h.value for p in patterns])
    best = Options()
    ms = C.c_float()
    _check(lib().tdfs_autotune(graph._h, arr, len(patterns), None if base is None else C.byref(base), sample_stride,
                               C.byref(best), C.byref(ms)))
    return best, ms.value


class Server:
    """Continuous-batching query server over one device-resident graph
    (tdfs_server_*): submit() admits queries into a running persistent
    kernel; wait() returns (count, latency in microseconds)."""

    def __init__(self, graph: GraphPreprocessor, labeled: bool = False, max_inflight: int = 256, max_k: int = 7,
                 mem_budget: int = 0, idle_exit_ms: int = 50, **launch):
        o = ServerOptions()
        lib().tdfs_server_options_default(C.byref(o))
        o.max_inflight, o.max_k, o.labeled = max_inflight, max_k, int(labeled)
        o.mem_budget, o.idle_exit_ms = mem_budget, idle_exit_ms
        for k, v in launch.items():
            setattr(o.launch, k, v)
        h = C.c_void_p()
        _check(lib().tdfs_server_create(graph._h, C.byref(o), C.byref(h)))
        self._h = h
        self.graph = graph

    def submit(self, pattern: PatternPreprocessor) -> int:
        t = C.c_uint64()
        _check(lib().tdfs_server_submit(self._h, pattern._h, C.byref(t)))
        return t.value

    def wait(self, ticket: int):
        c, lat = C.c_uint64(), C.c_double()
        _check(lib().tdfs_server_wait(self._h, ticket, C.byref(c), C.byref(lat)))
        return c.value, lat.value

    def stats(self) -> dict:
        st = ServeStats()
        _check(lib().tdfs_server_stats(self._h, C.byref(st)))
        return {f: getattr(st, f) for f, _ in ServeStats._fields_}

    def close(self):
        if getattr(self, "_h", None):
            h, self._h = self._h, None
            _check(lib().tdfs_server_destroy(h))

    def __del__(self):
        if _lib is not None and getattr(self, "_h", None):
            _lib.tdfs_server_destroy(self._h)
            self._h = None
