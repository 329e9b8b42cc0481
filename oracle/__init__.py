"""Python bindings of the checkers for the all-sources shortest-path hot path.

TEST INFRASTRUCTURE ONLY. Nothing in the product library imports this package: only ``tests/``,
``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py`` use it, as the checker and as the
timed CPU baseline, never as the thing measured or shipped.

Two checkers live here:

* ``Restatement`` binds ``libngx_oracle.so``, the project's C restatement (``ngx_oracle.c``) of the
  reference's Dijkstra, APSP summary, Brandes and the CPL/efficiency gradient, with FP64 arc lengths.
* ``Reference`` binds ``_ref/libngx_ref.so``, the reference implementation's own C++ sources compiled
  against single-rank shims (``ref_harness.cpp``, ``Makefile``). It exists only where the reference
  sources were present at build time; on other machines the committed golden fixtures under
  ``tests/golden/`` carry its outputs.
"""

from __future__ import annotations

import ctypes as C
import os
import subprocess
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
RESTATEMENT_SO = os.path.join(HERE, "libngx_oracle.so")
REFERENCE_SO = os.path.join(HERE, "_ref", "libngx_ref.so")
REFERENCE_GTESTS = os.path.join(HERE, "_ref", "ref_gtests")
INTEGRATION_CHECK = os.path.join(HERE, "_ref", "integration_check")
REFERENCE_DIR_RECORD = os.path.join(HERE, "_ref", "reference_dir.txt")


def _reference_sources() -> str | None:
    """The reference source tree: $NGX_REFERENCE_DIR, else the tree the reference build was made from."""
    path = os.environ.get("NGX_REFERENCE_DIR")
    if not path and os.path.exists(REFERENCE_DIR_RECORD):
        with open(REFERENCE_DIR_RECORD) as f:
            path = f.read().strip()
    return path if path and os.path.isdir(os.path.join(path, "source")) else None


REFERENCE_SOURCES = _reference_sources()

METRIC_REGULAR = 0
METRIC_INVERSE = 1

_i64p = np.ctypeslib.ndpointer(dtype=np.int64, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_u64p = np.ctypeslib.ndpointer(dtype=np.uint64, flags="C_CONTIGUOUS")


def build(reference_dir: str | None = None, quiet: bool = True) -> None:
    """Compile the restatement and, when `reference_dir` (or $NGX_REFERENCE_DIR) holds the reference sources, the
    reference harness built from them."""
    global REFERENCE_SOURCES
    out = subprocess.DEVNULL if quiet else None
    subprocess.run(["make", "-C", HERE, "restatement"], check=True, stdout=out)
    ref = reference_dir or os.environ.get("NGX_REFERENCE_DIR")
    if ref and os.path.isdir(os.path.join(ref, "source")):
        ref = os.path.abspath(ref)
        subprocess.run(["make", "-C", HERE, "-j8", "reference", f"REF={ref}"], check=True, stdout=out)
        if os.path.exists(os.path.join(os.path.dirname(HERE), "neurograph_b200", "lib", "libngx_b200.so")):
            subprocess.run(["make", "-C", HERE, "integration", f"REF={ref}"], check=True, stdout=out)
        REFERENCE_SOURCES = _reference_sources() or ref


class _Graph(C.Structure):
    _fields_ = [
        ("n", C.c_int64),
        ("m", C.c_int64),
        ("row_ptr", C.POINTER(C.c_int64)),
        ("col", C.POINTER(C.c_int32)),
        ("w", C.POINTER(C.c_double)),
    ]


class _Totals(C.Structure):
    _fields_ = [
        ("sum_distances", C.c_double),
        ("sum_inverse", C.c_double),
        ("sum_distances_sequential", C.c_double),
        ("sum_inverse_sequential", C.c_double),
        ("diameter", C.c_double),
        ("unreachable", C.c_uint64),
        ("reached_pairs", C.c_uint64),
        ("traversed_arcs", C.c_uint64),
        ("hist_overflow", C.c_uint64),
        ("cpl", C.c_double),
        ("efficiency", C.c_double),
    ]


@dataclass
class Csr:
    """Out-arc CSR with FP64 weights (int32 targets, int64 offsets)."""

    n: int
    row_ptr: np.ndarray
    col: np.ndarray
    w: np.ndarray

    @property
    def m(self) -> int:
        return int(self.row_ptr[-1]) if self.n > 0 else 0

    @staticmethod
    def from_arrays(n, row_ptr, col, w) -> "Csr":
        return Csr(
            int(n),
            np.ascontiguousarray(row_ptr, dtype=np.int64),
            np.ascontiguousarray(col, dtype=np.int32),
            np.ascontiguousarray(w, dtype=np.float64),
        )


def _totals_dict(t: _Totals) -> dict:
    return {name: getattr(t, name) for name, _ in _Totals._fields_}


class Restatement:
    """ctypes binding of libngx_oracle.so (see ngx_oracle.h)."""

    def __init__(self, path: str = RESTATEMENT_SO):
        if not os.path.exists(path):
            build(reference=False)
        lib = C.CDLL(path)
        lib.ngxo_sssp.argtypes = [C.POINTER(_Graph), C.c_int64, C.c_int, _f64p]
        lib.ngxo_apsp.argtypes = [
            C.POINTER(_Graph), C.c_void_p, C.c_int64, C.c_int, C.c_int64, C.c_double, C.c_void_p,
            C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(_Totals),
        ]
        lib.ngxo_brandes.argtypes = [C.POINTER(_Graph), C.c_void_p, C.c_int64, _f64p]
        lib.ngxo_apsp_grad.argtypes = [C.POINTER(_Graph), C.c_void_p, C.c_int64, _f64p, _f64p, C.POINTER(_Totals)]
        lib.ngxo_exact_sum.argtypes = [_f64p, C.c_int64]
        lib.ngxo_scc.argtypes = [C.POINTER(_Graph), C.c_void_p]
        lib.ngxo_scc.restype = C.c_int64
        lib.ngxo_exact_sum.restype = C.c_double
        self.lib = lib

    @staticmethod
    def _graph(g: Csr) -> _Graph:
        return _Graph(
            g.n, g.m,
            g.row_ptr.ctypes.data_as(C.POINTER(C.c_int64)),
            g.col.ctypes.data_as(C.POINTER(C.c_int32)),
            g.w.ctypes.data_as(C.POINTER(C.c_double)),
        )

    def exact_sum(self, x) -> float:
        x = np.ascontiguousarray(x, dtype=np.float64)
        return self.lib.ngxo_exact_sum(x, x.size)

    def scc(self, g: Csr) -> dict:
        """Tarjan's strongly connected components (ngxo_scc): the SccResult summary plus `component`, each vertex's
        component named by its largest vertex."""
        comp = np.zeros(max(g.n, 1), np.int32)
        count = self.lib.ngxo_scc(C.byref(self._graph(g)), comp.ctypes.data)
        if count < 0:
            raise RuntimeError(f"ngxo_scc failed ({count})")
        out = _scc_summary(comp[: g.n])
        assert out["number_components"] == count
        out["component"] = comp[: g.n]
        return out

    def sssp(self, g: Csr, source: int, metric: int = METRIC_REGULAR) -> np.ndarray:
        dist = np.empty(max(g.n, 1), dtype=np.float64)
        rc = self.lib.ngxo_sssp(C.byref(self._graph(g)), source, metric, dist)
        if rc != 0:
            raise ValueError(f"ngxo_sssp failed ({rc})")
        return dist[: g.n]

    def apsp(self, g: Csr, sources=None, metric: int = METRIC_REGULAR, bins: int = 0, hist_max: float = 0.0) -> dict:
        srcs = None if sources is None else np.ascontiguousarray(sources, dtype=np.int64)
        k = g.n if srcs is None else srcs.size
        per = {
            "sum": np.zeros(k, np.float64), "max": np.zeros(k, np.float64), "sum_inv": np.zeros(k, np.float64),
            "sum_inv_seq": np.zeros(k, np.float64), "unreachable": np.zeros(k, np.uint64),
            "arcs": np.zeros(k, np.uint64),
        }
        hist = np.zeros(bins, np.uint64) if bins > 0 else None
        totals = _Totals()
        ptr = lambda a: None if a is None else a.ctypes.data  # noqa: E731
        rc = self.lib.ngxo_apsp(
            C.byref(self._graph(g)), ptr(srcs), k, metric, bins, hist_max, ptr(hist),
            ptr(per["sum"]), ptr(per["max"]), ptr(per["sum_inv"]), ptr(per["sum_inv_seq"]),
            ptr(per["unreachable"]), ptr(per["arcs"]), C.byref(totals),
        )
        if rc != 0:
            raise ValueError(f"ngxo_apsp failed ({rc})")
        out = _totals_dict(totals)
        out["per_source"] = per
        out["hist"] = hist
        out["cluster_sizes"] = _cluster_sizes(g.n, per["unreachable"])
        return out

    def brandes(self, g: Csr, sources=None) -> np.ndarray:
        srcs = None if sources is None else np.ascontiguousarray(sources, dtype=np.int64)
        k = g.n if srcs is None else srcs.size
        bc = np.zeros(max(g.n, 1), np.float64)
        rc = self.lib.ngxo_brandes(C.byref(self._graph(g)), None if srcs is None else srcs.ctypes.data, k, bc)
        if rc != 0:
            raise ValueError(f"ngxo_brandes failed ({rc})")
        return bc[: g.n]

    def apsp_grad(self, g: Csr, sources=None):
        srcs = None if sources is None else np.ascontiguousarray(sources, dtype=np.int64)
        k = g.n if srcs is None else srcs.size
        dcpl = np.zeros(max(g.m, 1), np.float64)
        deff = np.zeros(max(g.m, 1), np.float64)
        totals = _Totals()
        rc = self.lib.ngxo_apsp_grad(C.byref(self._graph(g)), None if srcs is None else srcs.ctypes.data, k, dcpl, deff, C.byref(totals))
        if rc != 0:
            raise ValueError(f"ngxo_apsp_grad failed ({rc})")
        return dcpl[: g.m], deff[: g.m], _totals_dict(totals)


def _chunks(sources, threads: int) -> list[np.ndarray]:
    srcs = np.ascontiguousarray(sources, dtype=np.int64)
    parts = max(1, min(int(threads) if threads else (os.cpu_count() or 1), srcs.size))
    return [c for c in np.array_split(srcs, parts) if c.size]


def _pool_map(fn, items, threads: int):
    """fn over items on host threads (the C calls release the interpreter lock), in item order."""
    from concurrent.futures import ThreadPoolExecutor

    with ThreadPoolExecutor(max(1, int(threads) if threads else (os.cpu_count() or 1))) as ex:
        return list(ex.map(fn, items))


class ParallelRestatement(Restatement):
    """The restatement over a source list on host threads, for parity checks on large graphs. Every per-source value
    is computed exactly as by the sequential calls; only totals that sum over sources (betweenness, gradients) are
    combined in another order (relative differences of a few units in the last place)."""

    def __init__(self, threads: int = 0, path: str = RESTATEMENT_SO):
        super().__init__(path)
        self.threads = threads

    def sssp_rows(self, g: Csr, sources, metric: int = METRIC_REGULAR) -> np.ndarray:
        return np.stack(_pool_map(lambda s: self.sssp(g, int(s), metric), list(sources), self.threads))

    def apsp_sources(self, g: Csr, sources, metric: int = METRIC_REGULAR, bins: int = 0, hist_max: float = 0.0) -> dict:
        """Per-source summaries (bit-identical to apsp()'s), histogram, overflow, unreachable and traversed arcs."""
        parts = _pool_map(lambda c: self.apsp(g, c, metric, bins, hist_max), _chunks(sources, self.threads), self.threads)
        per = {k: np.concatenate([p["per_source"][k] for p in parts]) for k in parts[0]["per_source"]}
        out = {"per_source": per, "hist": None if bins <= 0 else np.sum([p["hist"] for p in parts], axis=0).astype(np.uint64)}
        for key in ("unreachable", "reached_pairs", "traversed_arcs", "hist_overflow"):
            out[key] = int(sum(int(p[key]) for p in parts))
        out["diameter"] = max(p["diameter"] for p in parts)
        return out

    def brandes_sources(self, g: Csr, sources) -> np.ndarray:
        return np.sum(_pool_map(lambda c: self.brandes(g, c), _chunks(sources, self.threads), self.threads), axis=0)

    def apsp_grad_sources(self, g: Csr, sources=None):
        """(dcpl, deff, reached_pairs): each chunk's gradient scaled back by its own R and divided by the total R."""
        srcs = np.arange(g.n) if sources is None else sources
        parts = _pool_map(lambda c: self.apsp_grad(g, c), _chunks(srcs, self.threads), self.threads)
        total = sum(int(p[2]["reached_pairs"]) for p in parts)
        dcpl = np.sum([p[0] * float(p[2]["reached_pairs"]) for p in parts], axis=0) / float(total)
        deff = np.sum([p[1] * float(p[2]["reached_pairs"]) for p in parts], axis=0) / float(total)
        return dcpl, deff, total


def _scc_summary(component: np.ndarray) -> dict:
    """SccResult of the reference from per-vertex component names: number, largest size, {size: components}."""
    _, sizes = np.unique(component, return_counts=True)
    keys, counts = np.unique(sizes, return_counts=True)
    return {"number_components": int(sizes.size), "largest_component_size": int(sizes.max()) if sizes.size else 0,
            "component_sizes": {int(k): int(c) for k, c in zip(keys, counts)}}


def _cluster_sizes(n: int, unreachable: np.ndarray) -> dict:
    """cluster_sizes of AllPairsShortestPath.h:139-140: reachable count (incl. the source) -> number of sources."""
    out: dict[int, int] = {}
    for u in np.asarray(unreachable, dtype=np.int64):
        key = int(n - u)
        out[key] = out.get(key, 0) + 1
    return out


class Reference:
    """ctypes binding of the reference's own code built from source (oracle/_ref/libngx_ref.so)."""

    def __init__(self, path: str = REFERENCE_SO):
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        lib = C.CDLL(path)
        lib.ngxref_last_error.restype = C.c_char_p
        lib.ngxref_fixture_name.restype = C.c_char_p
        self.lib = lib

    @staticmethod
    def available(path: str = REFERENCE_SO) -> bool:
        return os.path.exists(path)

    def _check(self, rc: int) -> None:
        if rc != 0:
            raise RuntimeError(self.lib.ngxref_last_error().decode())

    def fixture_names(self) -> list[str]:
        return [self.lib.ngxref_fixture_name(i).decode() for i in range(self.lib.ngxref_fixture_count())]

    def _read_csr(self, call) -> tuple[int, np.ndarray, np.ndarray, np.ndarray]:
        n, m = C.c_int64(), C.c_int64()
        self._check(call(C.byref(n), C.byref(m), None, None, None, C.c_int64(0)))
        row_ptr = np.zeros(n.value + 1, np.int64)
        col = np.zeros(max(m.value, 1), np.int32)
        w = np.zeros(max(m.value, 1), np.int32)
        self._check(call(C.byref(n), C.byref(m), row_ptr.ctypes.data_as(C.c_void_p), col.ctypes.data_as(C.c_void_p),
                         w.ctypes.data_as(C.c_void_p), C.c_int64(m.value)))
        return n.value, row_ptr, col[: m.value], w[: m.value]

    def fixture_csr(self, index: int):
        return self._read_csr(lambda *a: self.lib.ngxref_fixture_csr(C.c_int(index), *a))

    def load_csr(self, path: str, remove_self_arcs=False, undirected=False, one_weight=False):
        return self._read_csr(lambda *a: self.lib.ngxref_load_csr(path.encode(), int(remove_self_arcs), int(undirected), int(one_weight), *a))

    def graph(self, n, row_ptr, col, w_int) -> "RefGraph":
        handle = C.c_void_p()
        row_ptr = np.ascontiguousarray(row_ptr, np.int64)
        col = np.ascontiguousarray(col, np.int32)
        w_int = np.ascontiguousarray(w_int, np.int32)
        self._check(self.lib.ngxref_graph_create(C.c_int64(n), row_ptr.ctypes.data_as(C.c_void_p), col.ctypes.data_as(C.c_void_p),
                                                  w_int.ctypes.data_as(C.c_void_p), C.byref(handle)))
        return RefGraph(self, handle, n)

    def fixture_graph(self, index: int) -> "RefGraph":
        handle = C.c_void_p()
        self._check(self.lib.ngxref_fixture_graph(C.c_int(index), C.byref(handle)))
        n, _, _, _ = self.fixture_csr(index)
        return RefGraph(self, handle, n)


class RefGraph:
    def __init__(self, ref: Reference, handle, n: int):
        self.ref, self.handle, self.n = ref, handle, n

    def __del__(self):
        try:
            self.ref.lib.ngxref_graph_destroy(self.handle)
        except Exception:  # noqa: BLE001 - interpreter shutdown
            pass

    def csr(self):
        """(n, row_ptr, col, w_int32) in the reference's stored arc order."""
        return self.ref._read_csr(lambda *a: self.ref.lib.ngxref_graph_csr(self.handle, *a))

    def _apsp_out(self, call) -> dict:
        cpl, eff, dia, un, ln = C.c_double(), C.c_double(), C.c_double(), C.c_uint64(), C.c_int64()
        cap = 4096
        keys = np.zeros(cap, np.uint64)
        cnts = np.zeros(cap, np.uint64)
        self.ref._check(call(C.byref(cpl), C.byref(eff), C.byref(dia), C.byref(un), keys.ctypes.data_as(C.c_void_p),
                             cnts.ctypes.data_as(C.c_void_p), C.c_int64(cap), C.byref(ln)))
        return {"cpl": cpl.value, "efficiency": eff.value, "diameter": dia.value, "unreachable": un.value,
                "cluster_sizes": {int(keys[i]): int(cnts[i]) for i in range(min(ln.value, cap))}}

    def apsp(self, inverse=False, queue=0) -> dict:
        return self._apsp_out(lambda *a: self.ref.lib.ngxref_apsp(self.handle, int(inverse), int(queue), *a))

    def apsp_delta_stepping(self, delta: int, epoch: int) -> dict:
        return self._apsp_out(lambda *a: self.ref.lib.ngxref_apsp_delta_stepping(self.handle, C.c_uint64(delta), int(epoch), *a))

    def sssp_rows(self, sources, inverse=False, queue=0):
        srcs = np.ascontiguousarray(sources, np.int64)
        rows = np.zeros((srcs.size, self.n), np.float64 if inverse else np.uint64)
        summary = np.zeros((srcs.size, 4), np.float64)
        self.ref._check(self.ref.lib.ngxref_sssp_rows(self.handle, int(inverse), int(queue), srcs.ctypes.data_as(C.c_void_p),
                                                      C.c_int64(srcs.size), rows.ctypes.data_as(C.c_void_p), summary.ctypes.data_as(C.c_void_p)))
        return rows, summary

    def delta_stepping(self, sources, delta: int, epoch: int):
        srcs = np.ascontiguousarray(sources, np.int64)
        summary = np.zeros((srcs.size, 4), np.float64)
        self.ref._check(self.ref.lib.ngxref_delta_stepping(self.handle, C.c_uint64(delta), int(epoch), srcs.ctypes.data_as(C.c_void_p),
                                                           C.c_int64(srcs.size), summary.ctypes.data_as(C.c_void_p)))
        return summary

    def diameter_approximation(self, r: int, draws=None, seed: int = 0) -> int:
        """DiameterApproximation::compute_approximation of the reference (draws: replayed generator values)."""
        out = C.c_uint64()
        d = None if draws is None else np.ascontiguousarray(draws, np.float64)
        self.ref._check(self.ref.lib.ngxref_diameter_approximation(self.handle, C.c_uint64(r), None if d is None else d.ctypes.data_as(C.c_void_p),
                                                                    C.c_int64(0 if d is None else d.size), C.c_uint(seed), C.byref(out)))
        return int(out.value)

    def scc(self, algorithm: int = 3, tail_threshold: int = 0) -> dict:
        """StronglyConnectedComponents::compute_strongly_connected_components (algorithm: 0 TarjanGathered,
        1 ForwardBackward, 2 Coloring, 3 Multistep)."""
        count, largest = C.c_uint64(), C.c_uint64()
        sizes = np.zeros(self.n + 1, np.uint64)
        self.ref._check(self.ref.lib.ngxref_scc(self.handle, int(algorithm), C.c_uint64(tail_threshold), C.byref(count), C.byref(largest),
                                                sizes.ctypes.data_as(C.c_void_p), C.c_int64(sizes.size)))
        return {"number_components": int(count.value), "largest_component_size": int(largest.value),
                "component_sizes": {int(k): int(sizes[k]) for k in np.nonzero(sizes)[0]}}

    def betweenness(self, algorithm=0):
        bc = np.zeros(max(self.n, 1), np.float64)
        avg = C.c_double()
        self.ref._check(self.ref.lib.ngxref_betweenness(self.handle, int(algorithm), bc.ctypes.data_as(C.c_void_p), C.byref(avg)))
        return bc[: self.n], avg.value
