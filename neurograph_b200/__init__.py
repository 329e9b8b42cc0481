"""neurograph-b200: B200-native all-sources shortest paths for neurograph connectomes.

Python binding of the C ABI in ``include/ngx_b200.h`` (``neurograph_b200/lib/libngx_b200.so``). The library is
the product; this module only marshals host arrays through ctypes. There is no CPU fallback: importing works
without a GPU, but every call needs the CUDA library and a B200, and fails loudly otherwise.

Mapping to the reference (paths relative to the reference project):

* ``Graph(...)``                 DistributedGraph::construct_graph (source/graph/DistributedGraph.cpp:46-127)
* ``Graph.apsp()``               AllPairsShortestPath::compute_apsp / compute_apsp_inverse /
                                 compute_apsp_delta_stepping (source/metrics/paths/AllPairsShortestPath.h:54-98)
* ``Graph.sssp_rows()``          Dijkstra::compute_sssp's distance rows (source/metrics/paths/Dijkstra.h:55-98)
* ``Graph.brandes()``            BetweennessCentrality::compute_average_betweenness_centrality with the Brandes
                                 variant (source/metrics/paths/BetweennessCentrality.h:46-80)
* ``Graph.apsp_grad()``          new: gradient of CPL and global efficiency w.r.t. every arc length
* ``Batch(...)``                 new: many graphs in one handle and one persistent launch (the per-graph loop of
                                 source/neurograph.cpp:139-416 run for every graph at once)
"""

from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass, field

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.environ.get("NGX_B200_LIBRARY") or os.path.join(HERE, "lib", "libngx_b200.so")

NGX_OK = 0
STATUS_NAMES = {0: "OK", 1: "INVALID_ARGUMENT", 2: "OUT_OF_MEMORY", 3: "CUDA_ERROR", 4: "TIMEOUT", 5: "ABORTED", 6: "UNSUPPORTED"}
METRICS = {"regular": 0, "inverse": 1}
MODES = {"batched": 0, "plain": 1}
TASKS = {"apsp": 0, "brandes": 1, "grad": 2}
SIZE_CLASSES = 32
BUILD_ON_HOST = 1
TILE = 32
ACC_DIGITS = 72


class NgxError(RuntimeError):
    """A non-OK status from the CUDA library."""

    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


class _Csr(C.Structure):
    _fields_ = [("n", C.c_int64), ("m", C.c_int64), ("row_ptr", C.c_void_p), ("col", C.c_void_p), ("w", C.c_void_p)]


class _Opts(C.Structure):
    _fields_ = [
        ("metric", C.c_int), ("mode", C.c_int), ("sources", C.c_void_p), ("num_sources", C.c_int64),
        ("delta", C.c_double), ("block_threads", C.c_int), ("ctas_per_sm", C.c_int), ("hist_bins", C.c_int64),
        ("hist_max", C.c_double), ("max_iterations", C.c_uint64), ("tile_ctas", C.c_int),
    ]


class _BatchOpts(C.Structure):
    _fields_ = [
        ("task", C.c_int), ("metric", C.c_int), ("delta_scale", C.c_double), ("block_threads", C.c_int),
        ("hist_bins", C.c_int64), ("hist_max", C.c_double), ("use_cuda_graph", C.c_int), ("max_iterations", C.c_uint64),
        ("tile_ctas", C.c_int),
    ]


class _Tuning(C.Structure):
    _fields_ = [("delta_scale", C.c_double), ("block_threads", C.c_int), ("ctas_per_sm", C.c_int), ("tile_ctas", C.c_int),
                ("trials", C.c_int), ("gteps", C.c_double)]


class _Result(C.Structure):
    _fields_ = [
        ("sum_distances", C.c_double), ("sum_inverse", C.c_double), ("diameter", C.c_double),
        ("unreachable", C.c_uint64), ("reached_pairs", C.c_uint64), ("traversed_arcs", C.c_uint64),
        ("hist_overflow", C.c_uint64), ("hist_max", C.c_double), ("cpl", C.c_double), ("efficiency", C.c_double),
        ("kernel_ms", C.c_double), ("phases", C.c_uint64), ("expansions", C.c_uint64), ("lane_expansions", C.c_uint64),
        ("dag_levels", C.c_uint64), ("dag_entries", C.c_uint64), ("dag_scan_tiles", C.c_uint64),
        ("phase_cycles", C.c_uint64 * 5),
        ("hist", C.c_void_p), ("src_sum", C.c_void_p), ("src_max", C.c_void_p), ("src_sum_inverse", C.c_void_p),
        ("src_unreachable", C.c_void_p), ("src_arcs", C.c_void_p), ("acc_digits", C.c_void_p),
    ]


_LIB = None

# Every symbol include/ngx_b200.h declares (checked by the CPU test suite against the built library).
EXPORTED = [
    "ngx_status_string", "ngx_last_error", "ngx_version", "ngx_graph_create", "ngx_graph_destroy", "ngx_graph_size",
    "ngx_graph_request_abort", "ngx_graph_set_stream", "ngx_graph_set_memory_budget", "ngx_apsp", "ngx_sssp_rows", "ngx_brandes",
    "ngx_apsp_grad", "ngx_batch_create", "ngx_batch_run", "ngx_batch_autotune", "ngx_graph_update_weights", "ngx_apsp_noalloc", "ngx_exact_accumulate", "ngx_exact_round", "ngx_graph_source_order",
    "ngx_network_load", "ngx_network_size", "ngx_network_csr", "ngx_graph_create_from_network", "ngx_network_destroy",
    "ngx_diameter_contract", "ngx_diameter_approximation", "ngx_scc",
]


def library() -> C.CDLL:
    """Loads libngx_b200.so (raises if it has not been built)."""
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m neurograph_b200.build`")
        lib = C.CDLL(LIB_PATH)
        lib.ngx_status_string.restype = C.c_char_p
        lib.ngx_last_error.restype = C.c_char_p
        lib.ngx_version.restype = C.c_char_p
        lib.ngx_graph_create.argtypes = [C.POINTER(_Csr), C.c_int, C.POINTER(C.c_void_p)]
        lib.ngx_graph_create_ex.argtypes = [C.POINTER(_Csr), C.c_int, C.c_int, C.POINTER(C.c_void_p)]
        lib.ngx_graph_layout.argtypes = [C.c_void_p] + [C.c_void_p] * 7
        lib.ngx_graph_autotune.argtypes = [C.c_void_p, C.c_int, C.c_int64, C.POINTER(_Tuning)]
        lib.ngx_graph_tuning.argtypes = [C.c_void_p, C.c_int, C.POINTER(_Tuning)]
        lib.ngx_graph_destroy.argtypes = [C.c_void_p]
        lib.ngx_graph_destroy.restype = None
        lib.ngx_graph_size.argtypes = [C.c_void_p, C.POINTER(C.c_int64), C.POINTER(C.c_int64)]
        lib.ngx_graph_request_abort.argtypes = [C.c_void_p]
        lib.ngx_graph_set_memory_budget.argtypes = [C.c_void_p, C.c_uint64]
        lib.ngx_graph_set_stream.argtypes = [C.c_void_p, C.c_void_p]
        lib.ngx_apsp.argtypes = [C.c_void_p, C.POINTER(_Opts), C.POINTER(_Result)]
        lib.ngx_sssp_rows.argtypes = [C.c_void_p, C.POINTER(_Opts), C.c_void_p]
        if hasattr(lib, "ngx_brandes"):
            lib.ngx_brandes.argtypes = [C.c_void_p, C.POINTER(_Opts), C.c_void_p, C.POINTER(_Result)]
        if hasattr(lib, "ngx_apsp_grad"):
            lib.ngx_apsp_grad.argtypes = [C.c_void_p, C.POINTER(_Opts), C.c_void_p, C.c_void_p, C.POINTER(_Result)]
        lib.ngx_brandes_fixed.argtypes = [C.c_void_p, C.POINTER(_Opts), C.c_void_p, C.POINTER(_Result)]
        lib.ngx_apsp_grad_fixed.argtypes = [C.c_void_p, C.POINTER(_Opts), C.c_void_p, C.c_void_p, C.POINTER(_Result)]
        lib.ngx_fixed_to_double.argtypes = [C.c_void_p, C.c_int64, C.c_double, C.c_double, C.c_void_p]
        lib.ngx_batch_create.argtypes = [C.POINTER(_Csr), C.c_int64, C.c_int, C.POINTER(C.c_void_p)]
        lib.ngx_batch_run.argtypes = [C.c_void_p, C.POINTER(_BatchOpts), C.POINTER(_Result), C.c_void_p, C.c_void_p, C.c_void_p]
        lib.ngx_batch_autotune.argtypes = [C.c_void_p, C.c_int, C.c_void_p]
        lib.ngx_graph_update_weights.argtypes = [C.c_void_p, C.c_void_p]
        lib.ngx_apsp_noalloc.argtypes = [C.c_void_p, C.POINTER(_Opts), C.POINTER(_Result)]
        lib.ngx_graph_source_order.argtypes = [C.c_void_p, C.c_void_p]
        lib.ngx_network_load.argtypes = [C.c_char_p, C.c_int32, C.c_char_p, C.c_int, C.c_int, C.POINTER(C.c_void_p)]
        lib.ngx_network_size.argtypes = [C.c_void_p, C.POINTER(C.c_int64), C.POINTER(C.c_int64)]
        lib.ngx_network_csr.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
        lib.ngx_graph_create_from_network.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.c_void_p)]
        lib.ngx_network_destroy.argtypes = [C.c_void_p]
        lib.ngx_network_destroy.restype = None
        lib.ngx_diameter_contract.argtypes = [C.POINTER(_Csr), C.c_uint64, C.c_void_p, C.c_int64, C.c_uint32, C.POINTER(C.c_void_p)]
        lib.ngx_diameter_approximation.argtypes = [C.POINTER(_Csr), C.c_uint64, C.c_void_p, C.c_int64, C.c_uint32, C.c_int,
                                                   C.POINTER(C.c_uint64)]
        lib.ngx_scc.argtypes = [C.c_void_p, C.c_void_p, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64), C.c_void_p]
        lib.ngx_exact_accumulate.argtypes = [C.c_void_p, C.c_int64, C.c_void_p]
        lib.ngx_exact_round.argtypes = [C.c_void_p]
        lib.ngx_exact_round.restype = C.c_double
        _LIB = lib
    return _LIB


def _check(status: int) -> None:
    if status != NGX_OK:
        raise NgxError(status, library().ngx_last_error().decode())


@dataclass
class ApspResult:
    """Mirror of ApspGlobalResult (source/Types.h:237-244) plus the new outputs."""

    cpl: float
    efficiency: float
    diameter: float
    unreachable: int
    reached_pairs: int
    traversed_arcs: int
    sum_distances: float
    sum_inverse: float
    hist_max: float
    hist_overflow: int
    kernel_ms: float
    phases: int = 0
    expansions: int = 0
    lane_expansions: int = 0
    dag_levels: int = 0
    dag_entries: int = 0
    dag_scan_tiles: int = 0
    phase_cycles: tuple = ()
    hist: np.ndarray | None = None
    per_source: dict | None = None
    cluster_sizes: dict = field(default_factory=dict)
    acc_digits: np.ndarray | None = None  # (2, ACC_DIGITS) exact sums of d and 1/d before rounding (exact=True)

    @property
    def gteps(self) -> float:
        return self.traversed_arcs / (self.kernel_ms * 1e-3) / 1e9 if self.kernel_ms > 0 else 0.0


def _out_array(a, size):
    """A caller's output array, checked: C-contiguous float64 with at least `size` entries."""
    if not isinstance(a, np.ndarray) or a.dtype != np.float64 or not a.flags["C_CONTIGUOUS"] or a.size < size or not a.flags["WRITEABLE"]:
        raise ValueError(f"out arrays must be writeable C-contiguous float64 arrays of at least {size} entries")
    return a.reshape(-1)


class Graph:
    """A graph resident on one GPU (device CSR + reverse CSR)."""

    def __init__(self, n: int, row_ptr, col, w, device: int = 0, build: str = "device"):
        """build: "device" (the arrays are built by GPU kernels, the default) or "host" (host threads, then uploaded);
        both give the same arrays bit for bit."""
        lib = library()
        self.n = int(n)
        self.row_ptr = np.ascontiguousarray(row_ptr, dtype=np.int64)
        self.col = np.ascontiguousarray(col, dtype=np.int32)
        self.w = np.ascontiguousarray(w, dtype=np.float64)
        self.m = int(self.col.size)
        csr = _Csr(self.n, self.m, self.row_ptr.ctypes.data, self.col.ctypes.data if self.m else None,
                   self.w.ctypes.data if self.m else None)
        handle = C.c_void_p()
        if build not in ("device", "host"):
            raise ValueError(f"unknown build {build!r}")
        _check(lib.ngx_graph_create_ex(C.byref(csr), int(device), BUILD_ON_HOST if build == "host" else 0, C.byref(handle)))
        self._handle = handle

    def layout(self) -> dict:
        """The handle's device arrays (ngx_graph_layout): row_ptr, arcs / arcs_inverse / rarcs as (col, id, len)
        record arrays, rrow_ptr, arc_src and the mean lengths."""
        m = int(self._stored_arcs())
        rec = np.dtype([("col", np.int32), ("id", np.int32), ("len", np.float64)])
        out = {"row_ptr": np.zeros(self.n + 1, np.int64), "rrow_ptr": np.zeros(self.n + 1, np.int64),
               "arcs": np.zeros(max(m, 1), rec), "arcs_inverse": np.zeros(max(m, 1), rec), "rarcs": np.zeros(max(m, 1), rec),
               "arc_src": np.zeros(max(m, 1), np.int32), "mean_lengths": np.zeros(2)}
        _check(library().ngx_graph_layout(self._handle, *(out[k].ctypes.data for k in
                                                          ("row_ptr", "arcs", "arcs_inverse", "rrow_ptr", "rarcs", "arc_src", "mean_lengths"))))
        for k in ("arcs", "arcs_inverse", "rarcs", "arc_src"):
            out[k] = out[k][:m]
        return out

    def _stored_arcs(self) -> int:
        rows = np.zeros(self.n + 1, np.int64)
        _check(library().ngx_graph_layout(self._handle, rows.ctypes.data, None, None, None, None, None, None))
        return int(rows[-1])

    @classmethod
    def from_network(cls, directory: str, number_ranks: int, file_prefix: str = "", remove_self_arcs: bool = False,
                     undirected: bool = False, one_weight: bool = False, threads: int = 0, device: int = 0) -> "Graph":
        """Loads neurograph's per-rank network files (ngx_network_load) straight into a device graph
        (ngx_graph_create_from_network); the CSR is also kept on the host as row_ptr / col / w."""
        lib = library()
        flags = (LOAD_REMOVE_SELF_ARCS if remove_self_arcs else 0) | (LOAD_UNDIRECTED if undirected else 0) | \
            (LOAD_ONE_WEIGHT if one_weight else 0)
        net = C.c_void_p()
        _check(lib.ngx_network_load(os.fsencode(directory), int(number_ranks), file_prefix.encode(), flags, int(threads), C.byref(net)))
        try:
            n, m = C.c_int64(), C.c_int64()
            _check(lib.ngx_network_size(net, C.byref(n), C.byref(m)))
            self = cls.__new__(cls)
            self.n, self.m = n.value, m.value
            self.row_ptr = np.zeros(self.n + 1, np.int64)
            self.col = np.zeros(max(self.m, 1), np.int32)
            self.w = np.zeros(max(self.m, 1), np.float64)
            _check(lib.ngx_network_csr(net, self.row_ptr.ctypes.data, self.col.ctypes.data, self.w.ctypes.data))
            self.col, self.w = self.col[: self.m], self.w[: self.m]
            handle = C.c_void_p()
            _check(lib.ngx_graph_create_from_network(net, int(device), C.byref(handle)))
            self._handle = handle
        finally:
            lib.ngx_network_destroy(net)
        return self

    def close(self) -> None:
        if getattr(self, "_handle", None):
            library().ngx_graph_destroy(self._handle)
            self._handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:  # noqa: BLE001 - interpreter shutdown
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def request_abort(self) -> None:
        _check(library().ngx_graph_request_abort(self._handle))

    def set_stream(self, stream_handle: int | None) -> None:
        """Issue the graph's work on a caller-owned cudaStream_t (e.g. torch.cuda.Stream().cuda_stream)."""
        _check(library().ngx_graph_set_stream(self._handle, stream_handle))

    def set_memory_budget(self, nbytes: int) -> None:
        _check(library().ngx_graph_set_memory_budget(self._handle, int(nbytes)))

    def autotune(self, task="apsp", sample_sources: int = 0) -> dict:
        """ngx_graph_autotune: times the task on a sample of the all-sources order for bucket widths, block shapes and
        CTAs per tile, keeps the fastest for later runs that leave those options at 0, and returns it."""
        t = _Tuning()
        _check(library().ngx_graph_autotune(self._handle, TASKS[task] if isinstance(task, str) else int(task), int(sample_sources),
                                            C.byref(t)))
        return {name: getattr(t, name) for name, _ in _Tuning._fields_}

    def source_order(self) -> np.ndarray:
        """The order in which all-sources runs take the sources (tiles of nearby vertices); contiguous chunks of it
        split an all-sources job into batches with the same tiles."""
        out = np.zeros(max(self.n, 1), np.int64)
        _check(library().ngx_graph_source_order(self._handle, out.ctypes.data))
        return out[: self.n]

    def scc(self) -> dict:
        """Strongly connected components (ngx_scc), as the reference's SccResult: number_components,
        largest_component_size, component_sizes {size: number of components}; plus `component`, each vertex's
        component named by its largest vertex."""
        comp = np.zeros(max(self.n, 1), np.int32)
        hist = np.zeros(self.n + 1, np.uint64)
        count, largest = C.c_uint64(0), C.c_uint64(0)
        _check(library().ngx_scc(self._handle, comp.ctypes.data, C.byref(count), C.byref(largest), hist.ctypes.data))
        sizes = {int(k): int(hist[k]) for k in np.nonzero(hist)[0]}
        return {"number_components": count.value, "largest_component_size": largest.value, "component_sizes": sizes,
                "component": comp[: self.n]}

    def update_weights(self, w) -> None:
        """Replaces the arc weights in place (same arcs; no weight may change between zero and non-zero)."""
        w = np.ascontiguousarray(w, dtype=np.float64)
        if w.size != self.m:
            raise ValueError(f"expected {self.m} weights, got {w.size}")
        _check(library().ngx_graph_update_weights(self._handle, w.ctypes.data if self.m else None))
        self.w = w

    def _opts(self, sources, metric, mode, delta, hist_bins, hist_max, block_threads, ctas_per_sm, max_iterations, tile_ctas=0):
        srcs = None if sources is None else np.ascontiguousarray(sources, dtype=np.int64)
        opts = _Opts(
            METRICS[metric] if isinstance(metric, str) else int(metric),
            MODES[mode] if isinstance(mode, str) else int(mode),
            None if srcs is None else srcs.ctypes.data,
            0 if srcs is None else srcs.size,
            float(delta), int(block_threads), int(ctas_per_sm), int(hist_bins), float(hist_max), int(max_iterations), int(tile_ctas),
        )
        k = self.n if srcs is None else srcs.size
        return opts, srcs, k

    def _result(self, r: _Result, hist, per, k) -> ApspResult:
        out = ApspResult(
            cpl=r.cpl, efficiency=r.efficiency, diameter=r.diameter, unreachable=r.unreachable,
            reached_pairs=r.reached_pairs, traversed_arcs=r.traversed_arcs, sum_distances=r.sum_distances,
            sum_inverse=r.sum_inverse, hist_max=r.hist_max, hist_overflow=r.hist_overflow, kernel_ms=r.kernel_ms,
            phases=r.phases, expansions=r.expansions, lane_expansions=r.lane_expansions, dag_levels=r.dag_levels, dag_entries=r.dag_entries, dag_scan_tiles=r.dag_scan_tiles,
            phase_cycles=tuple(int(x) for x in r.phase_cycles), hist=hist, per_source=per,
        )
        if per is not None:
            sizes: dict[int, int] = {}
            for u in per["unreachable"].astype(np.int64):
                sizes[int(self.n - u)] = sizes.get(int(self.n - u), 0) + 1
            out.cluster_sizes = sizes
        return out

    @staticmethod
    def _result_struct(hist_bins, per_source, k, exact=False):
        r = _Result()
        hist = np.zeros(hist_bins, np.uint64) if hist_bins > 0 else None
        per = None
        if per_source:
            per = {"sum": np.zeros(k), "max": np.zeros(k), "sum_inv": np.zeros(k),
                   "unreachable": np.zeros(k, np.uint64), "arcs": np.zeros(k, np.uint64)}
            r.src_sum, r.src_max, r.src_sum_inverse = per["sum"].ctypes.data, per["max"].ctypes.data, per["sum_inv"].ctypes.data
            r.src_unreachable, r.src_arcs = per["unreachable"].ctypes.data, per["arcs"].ctypes.data
        if hist is not None:
            r.hist = hist.ctypes.data
        if exact:
            digits = np.zeros((2, ACC_DIGITS), np.uint64)
            r.acc_digits = digits.ctypes.data
            r._digits = digits  # kept alive with the struct
        return r, hist, per

    def apsp(self, sources=None, metric="regular", mode="batched", delta=0.0, hist_bins=0, hist_max=0.0,
             per_source=False, block_threads=0, ctas_per_sm=0, max_iterations=0, exact=False, tile_ctas=0) -> ApspResult:
        """exact=True also returns the unrounded exact sums (acc_digits), for merging the runs of several ranks.
        tile_ctas: CTAs that work on one source tile together (0 = the library's choice)."""
        opts, srcs, k = self._opts(sources, metric, mode, delta, hist_bins, hist_max, block_threads, ctas_per_sm, max_iterations, tile_ctas)
        r, hist, per = self._result_struct(hist_bins, per_source, k, exact)
        _check(library().ngx_apsp(self._handle, C.byref(opts), C.byref(r)))
        out = self._result(r, hist, per, k)
        if exact:
            out.acc_digits = r._digits
        return out

    def apsp_noalloc(self, sources=None, metric="regular", delta=0.0, hist_bins=0, hist_max=0.0, per_source=False,
                     block_threads=0, ctas_per_sm=0, max_iterations=0) -> ApspResult:
        """ngx_apsp_noalloc: apsp() in the batched form with no device allocation (graphs of up to 32768 vertices;
        hist_max is required with hist_bins). Calls on one device must not overlap."""
        opts, srcs, k = self._opts(sources, metric, "batched", delta, hist_bins, hist_max, block_threads, ctas_per_sm, max_iterations)
        r, hist, per = self._result_struct(hist_bins, per_source, k)
        _check(library().ngx_apsp_noalloc(self._handle, C.byref(opts), C.byref(r)))
        return self._result(r, hist, per, k)

    def sssp_rows(self, sources, metric="regular", mode="batched", delta=0.0, tile_ctas=0) -> np.ndarray:
        opts, srcs, k = self._opts(sources, metric, mode, delta, 0, 0.0, 0, 0, 0, tile_ctas)
        rows = np.zeros((k, self.n), np.float64)
        _check(library().ngx_sssp_rows(self._handle, C.byref(opts), rows.ctypes.data))
        return rows

    def brandes(self, sources=None, delta=0.0, hist_bins=0, hist_max=0.0, per_source=False, block_threads=0,
                ctas_per_sm=0, max_iterations=0, fixed=False, exact=False, tile_ctas=0, mode="batched", out=None):
        """Betweenness (sum of pair dependencies over the sources) and the run's APSP result. fixed=True returns the
        unconverted sums instead (ngx_brandes_fixed): an (n, 2) uint64 array of 128-bit fixed-point words.
        mode="plain" runs one source per CTA (the per-source baseline form); its dependencies are summed in another
        order than the batched form's, so its betweenness agrees with the batched one to rounding, not bit for bit.
        out: a C-contiguous float64 array of at least max(n, 1) entries to write the betweenness into (a view of it is
        returned)."""
        opts, srcs, k = self._opts(sources, "regular", mode, delta, hist_bins, hist_max, block_threads, ctas_per_sm, max_iterations,
                                   tile_ctas)
        r, hist, per = self._result_struct(hist_bins, per_source, k, exact)
        if fixed:
            if out is not None:
                raise ValueError("out= takes converted betweenness; the fixed-point words are returned as a new array")
            words = np.zeros((max(self.n, 1), 2), np.uint64)
            _check(library().ngx_brandes_fixed(self._handle, C.byref(opts), words.ctypes.data, C.byref(r)))
            bc = words[: self.n]
        else:
            bc = _out_array(out, max(self.n, 1)) if out is not None else np.zeros(max(self.n, 1), np.float64)
            _check(library().ngx_brandes(self._handle, C.byref(opts), bc.ctypes.data, C.byref(r)))
            bc = bc[: self.n]
        out = self._result(r, hist, per, k)
        if exact:
            out.acc_digits = r._digits
        return bc, out

    def apsp_grad(self, sources=None, delta=0.0, block_threads=0, ctas_per_sm=0, max_iterations=0, fixed=False, tile_ctas=0,
                  out=None):
        """Gradients of CPL and efficiency w.r.t. every arc length, and the run's APSP result. fixed=True returns the
        unconverted sums instead (ngx_apsp_grad_fixed): two (m, 2) uint64 arrays, before the division by R.
        out=(dcpl, deff): two C-contiguous float64 arrays of at least max(m, 1) entries to write into (for instance
        page-locked ones reused from call to call, which the device writes directly); views of them are returned."""
        opts, srcs, k = self._opts(sources, "regular", "batched", delta, 0, 0.0, block_threads, ctas_per_sm, max_iterations, tile_ctas)
        r, hist, per = self._result_struct(0, False, k)
        if fixed:
            if out is not None:
                raise ValueError("out= takes converted gradients; the fixed-point words are returned as new arrays")
            dcpl = np.zeros((max(self.m, 1), 2), np.uint64)
            deff = np.zeros((max(self.m, 1), 2), np.uint64)
            _check(library().ngx_apsp_grad_fixed(self._handle, C.byref(opts), dcpl.ctypes.data, deff.ctypes.data, C.byref(r)))
        else:
            dcpl, deff = (_out_array(out[0], max(self.m, 1)), _out_array(out[1], max(self.m, 1))) if out is not None else \
                (np.zeros(max(self.m, 1), np.float64), np.zeros(max(self.m, 1), np.float64))
            _check(library().ngx_apsp_grad(self._handle, C.byref(opts), dcpl.ctypes.data, deff.ctypes.data, C.byref(r)))
        return dcpl[: self.m], deff[: self.m], self._result(r, hist, per, k)


class Batch:
    """Many independent graphs resident on one GPU in one handle; every run covers all sources of all graphs.

    ``graphs`` is a sequence of ``(n, row_ptr, col, w)``. Results, betweenness and gradients keep per-graph numbering.
    """

    def __init__(self, graphs, device: int = 0):
        lib = library()
        self.graphs = [(int(n), np.ascontiguousarray(rp, dtype=np.int64), np.ascontiguousarray(c, dtype=np.int32),
                        np.ascontiguousarray(w, dtype=np.float64)) for n, rp, c, w in graphs]
        self.ns = [g[0] for g in self.graphs]
        self.ms = [int(g[2].size) for g in self.graphs]
        csrs = (_Csr * max(1, len(self.graphs)))()
        for i, (n, rp, c, w) in enumerate(self.graphs):
            csrs[i] = _Csr(n, c.size, rp.ctypes.data, c.ctypes.data if c.size else None, w.ctypes.data if c.size else None)
        handle = C.c_void_p()
        _check(lib.ngx_batch_create(csrs, len(self.graphs), int(device), C.byref(handle)))
        self._handle = handle

    def close(self) -> None:
        if getattr(self, "_handle", None):
            library().ngx_graph_destroy(self._handle)
            self._handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:  # noqa: BLE001 - interpreter shutdown
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def set_stream(self, stream_handle: int | None) -> None:
        _check(library().ngx_graph_set_stream(self._handle, stream_handle))

    def run(self, task="apsp", metric="regular", delta_scale=0.0, hist_bins=0, hist_max=0.0, per_source=False,
            use_cuda_graph=False, block_threads=0, max_iterations=0, tile_ctas=0):
        """Runs `task` for every graph. Returns (results, extra): a list of ApspResult and, per graph, the betweenness
        vector (task "brandes"), the (dcpl, deff) pair (task "grad") or None."""
        t = TASKS[task] if isinstance(task, str) else int(task)
        opts = _BatchOpts(t, METRICS[metric] if isinstance(metric, str) else int(metric), float(delta_scale),
                          int(block_threads), int(hist_bins), float(hist_max), int(bool(use_cuda_graph)), int(max_iterations),
                          int(tile_ctas))
        count = len(self.graphs)
        structs = (_Result * max(1, count))()
        keep = []
        for i, n in enumerate(self.ns):
            r, hist, per = Graph._result_struct(hist_bins, per_source, n)
            structs[i] = r
            keep.append((hist, per))
        n_total, m_total = sum(self.ns), sum(self.ms)
        bc = np.zeros(max(1, n_total)) if t == 1 else None
        dcpl = np.zeros(max(1, m_total)) if t == 2 else None
        deff = np.zeros(max(1, m_total)) if t == 2 else None
        _check(library().ngx_batch_run(self._handle, C.byref(opts), structs,
                                       None if bc is None else bc.ctypes.data,
                                       None if dcpl is None else dcpl.ctypes.data,
                                       None if deff is None else deff.ctypes.data))
        results, extras = [], []
        v_off = a_off = 0
        for i, n in enumerate(self.ns):
            hist, per = keep[i]
            view = Graph.__new__(Graph)
            view.n = n
            results.append(Graph._result(view, structs[i], hist, per, n))
            m = self.ms[i]
            if bc is not None:
                extras.append(bc[v_off:v_off + n].copy())
            elif dcpl is not None:
                extras.append((dcpl[a_off:a_off + m].copy(), deff[a_off:a_off + m].copy()))
            else:
                extras.append(None)
            v_off += n
            a_off += m
        return results, extras

    def tuning(self, task="apsp") -> dict:
        """The launch shape ngx_batch_autotune picked for the task (ngx_graph_tuning)."""
        t = _Tuning()
        _check(library().ngx_graph_tuning(self._handle, TASKS[task] if isinstance(task, str) else int(task), C.byref(t)))
        return {name: getattr(t, name) for name, _ in _Tuning._fields_}

    def autotune(self, task="apsp") -> np.ndarray:
        """Tunes the bucket width per size class (floor(log2 n)) and the batch's launch shape; returns the chosen scales
        (0 = class empty)."""
        scales = np.zeros(SIZE_CLASSES)
        _check(library().ngx_batch_autotune(self._handle, TASKS[task] if isinstance(task, str) else int(task), scales.ctypes.data))
        return scales

    def update_weights(self, weights) -> None:
        """Replaces all graphs' weights in place: one array per graph, caller arc order."""
        flat = np.ascontiguousarray(np.concatenate([np.asarray(w, dtype=np.float64) for w in weights]) if weights else np.zeros(0))
        if flat.size != sum(self.ms):
            raise ValueError("weights do not match the batch's arcs")
        _check(library().ngx_graph_update_weights(self._handle, flat.ctypes.data if flat.size else None))


LOAD_REMOVE_SELF_ARCS, LOAD_UNDIRECTED, LOAD_ONE_WEIGHT = 1, 2, 4


def load_network(directory: str, number_ranks: int, file_prefix: str = "", remove_self_arcs: bool = False,
                 undirected: bool = False, one_weight: bool = False, threads: int = 0):
    """Reads neurograph's per-rank network files (ngx_network_load, host only) and returns (n, row_ptr, col, w), the
    global CSR a Graph is built from."""
    flags = (LOAD_REMOVE_SELF_ARCS if remove_self_arcs else 0) | (LOAD_UNDIRECTED if undirected else 0) | \
        (LOAD_ONE_WEIGHT if one_weight else 0)
    lib = library()
    handle = C.c_void_p()
    _check(lib.ngx_network_load(os.fsencode(directory), int(number_ranks), file_prefix.encode(), flags, int(threads), C.byref(handle)))
    try:
        n, m = C.c_int64(), C.c_int64()
        _check(lib.ngx_network_size(handle, C.byref(n), C.byref(m)))
        row_ptr = np.zeros(n.value + 1, np.int64)
        col = np.zeros(max(m.value, 1), np.int32)
        w = np.zeros(max(m.value, 1), np.float64)
        _check(lib.ngx_network_csr(handle, row_ptr.ctypes.data, col.ctypes.data, w.ctypes.data))
    finally:
        lib.ngx_network_destroy(handle)
    return n.value, row_ptr, col[: m.value], w[: m.value]


def _csr_struct(n, row_ptr, col, w):
    rp = np.ascontiguousarray(row_ptr, dtype=np.int64)
    c = np.ascontiguousarray(col, dtype=np.int32)
    ww = np.ascontiguousarray(w, dtype=np.float64)
    return _Csr(int(n), c.size, rp.ctypes.data, c.ctypes.data if c.size else None, ww.ctypes.data if c.size else None), (rp, c, ww)


def _network_arrays(lib, handle):
    n, m = C.c_int64(), C.c_int64()
    _check(lib.ngx_network_size(handle, C.byref(n), C.byref(m)))
    row_ptr = np.zeros(n.value + 1, np.int64)
    col = np.zeros(max(m.value, 1), np.int32)
    w = np.zeros(max(m.value, 1), np.float64)
    _check(lib.ngx_network_csr(handle, row_ptr.ctypes.data, col.ctypes.data, w.ctypes.data))
    return n.value, row_ptr, col[: m.value], w[: m.value]


def diameter_contract(n, row_ptr, col, w, r: int, draws=None, seed: int = 0):
    """The contracted graph of the diameter approximation (ngx_diameter_contract, host only): (n, row_ptr, col, w)."""
    lib = library()
    csr, keep = _csr_struct(n, row_ptr, col, w)
    d = None if draws is None else np.ascontiguousarray(draws, np.float64)
    handle = C.c_void_p()
    _check(lib.ngx_diameter_contract(C.byref(csr), int(r), None if d is None else d.ctypes.data, 0 if d is None else d.size, int(seed),
                                     C.byref(handle)))
    try:
        return _network_arrays(lib, handle)
    finally:
        lib.ngx_network_destroy(handle)


def diameter_approximation(n, row_ptr, col, w, r: int, draws=None, seed: int = 0, device: int = 0) -> int:
    """DiameterApproximation::compute_approximation: the contracted graph's exact diameter (GPU) plus 2r."""
    lib = library()
    csr, keep = _csr_struct(n, row_ptr, col, w)
    d = None if draws is None else np.ascontiguousarray(draws, np.float64)
    out = C.c_uint64()
    _check(lib.ngx_diameter_approximation(C.byref(csr), int(r), None if d is None else d.ctypes.data, 0 if d is None else d.size, int(seed),
                                          int(device), C.byref(out)))
    return int(out.value)


def exact_accumulate(values, digits=None) -> np.ndarray:
    """Adds non-negative finite doubles exactly into an accumulator ((ACC_DIGITS,) uint64, new if None). Host only."""
    v = np.ascontiguousarray(values, dtype=np.float64)
    d = np.zeros(ACC_DIGITS, np.uint64) if digits is None else digits
    if d.dtype != np.uint64 or d.size != ACC_DIGITS or not d.flags.c_contiguous:
        raise ValueError("digits must be a contiguous uint64 array of ACC_DIGITS words")
    _check(library().ngx_exact_accumulate(v.ctypes.data if v.size else None, v.size, d.ctypes.data))
    return d


def fixed_to_double(words, divisor: float = 1.0, sign: float = 1.0) -> np.ndarray:
    """Converts (count, 2) 128-bit fixed-point words (as ngx_brandes_fixed / ngx_apsp_grad_fixed return them, or their
    merged sums) to doubles the way the library converts its own sums: sign * value / divisor."""
    w = np.ascontiguousarray(words, dtype=np.uint64).reshape(-1, 2)
    out = np.zeros(max(w.shape[0], 1), np.float64)
    _check(library().ngx_fixed_to_double(w.ctypes.data, w.shape[0], float(divisor), float(sign), out.ctypes.data))
    return out[: w.shape[0]]


def exact_round(digits) -> float:
    """The accumulator's value rounded once to nearest-even (digits may be a sum of several normalized accumulators)."""
    d = np.array(digits, dtype=np.uint64, copy=True)
    if d.size != ACC_DIGITS:
        raise ValueError("expected ACC_DIGITS words")
    return float(library().ngx_exact_round(d.ctypes.data))


def version() -> str:
    return library().ngx_version().decode()
