"""The C ABI library without a GPU: it loads, exports every symbol include/ngx_b200.h declares, and rejects invalid
graphs on the host before touching a device (the host validation of ngx_graph_create)."""

from __future__ import annotations

import ctypes as C
import os
import re

import numpy as np
import pytest

import neurograph_b200 as ngx

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for header in os.listdir(os.path.join(ROOT, "include")):
        if header.endswith(".h"):
            with open(os.path.join(ROOT, "include", header)) as f:
                names |= set(re.findall(r"^NGX_API\s+[^;(]*?\b(ngx_\w+)\s*\(", f.read(), flags=re.M))
    return sorted(names)


def test_library_exports_every_declared_symbol():
    lib = ngx.library()
    names = declared_symbols()
    assert "ngx_apsp" in names and "ngx_graph_create" in names
    missing = [name for name in names if not hasattr(lib, name)]
    assert not missing, missing
    assert set(ngx.EXPORTED) <= set(names)


def test_status_strings():
    lib = ngx.library()
    assert lib.ngx_status_string(0) == b"ok"
    assert lib.ngx_status_string(4) == b"iteration cap reached"
    assert b"sm_100a" in lib.ngx_version()


def _create(n, row_ptr, col, w):
    lib = ngx.library()
    row_ptr = np.ascontiguousarray(row_ptr, np.int64)
    col = np.ascontiguousarray(col, np.int32)
    w = np.ascontiguousarray(w, np.float64)
    csr = ngx._Csr(n, col.size, row_ptr.ctypes.data, col.ctypes.data if col.size else None, w.ctypes.data if w.size else None)
    handle = C.c_void_p()
    return lib.ngx_graph_create(C.byref(csr), 0, C.byref(handle))


@pytest.mark.parametrize(
    "graph",
    [
        (3, [0, 2, 1, 3], [1, 2, 0], [1.0, 1.0, 1.0]),        # row_ptr not monotone
        (3, [0, 1, 2, 3], [1, 5, 0], [1.0, 1.0, 1.0]),        # target out of range
        (3, [0, 1, 2, 3], [1, 2, -1], [1.0, 1.0, 1.0]),       # negative target
        (3, [0, 1, 2, 3], [1, 2, 0], [1.0, np.nan, 1.0]),     # NaN weight
        (3, [0, 1, 2, 3], [1, 2, 0], [1.0, np.inf, 1.0]),     # infinite weight
        (3, [1, 1, 2, 3], [1, 2, 0], [1.0, 1.0, 1.0]),        # row_ptr[0] != 0
        (3, [0, 1, 2, 2], [1, 2, 0], [1.0, 1.0, 1.0]),        # row_ptr[n] != m
    ],
)
def test_invalid_graphs_are_rejected_on_the_host(graph):
    assert _create(*graph) == 1  # NGX_INVALID_ARGUMENT
    assert ngx.library().ngx_last_error().startswith(b"ngx_graph_create")


def test_null_arguments():
    lib = ngx.library()
    assert lib.ngx_graph_create(None, 0, None) == 1
    assert lib.ngx_apsp(None, None, None) == 1
    assert lib.ngx_graph_size(None, None, None) == 1


def test_exact_sums_on_the_host():
    """ngx_exact_accumulate / ngx_exact_round (host only): the exactly rounded sum whatever the split or order,
    equal to math.fsum; negative or non-finite values are rejected."""
    import math

    rng = np.random.default_rng(4)
    x = np.concatenate([rng.lognormal(0.0, 6.0, 50000), [0.0, 5e-324, 2.2250738585072014e-308, 1.7976931348623157e308 / 4]])
    whole = ngx.exact_accumulate(x)
    assert ngx.exact_round(whole) == math.fsum(x)
    parts = [ngx.exact_accumulate(p) for p in np.array_split(rng.permutation(x), 7)]
    assert ngx.exact_round(sum(parts)) == math.fsum(x)
    assert ngx.exact_round(np.zeros(ngx.ACC_DIGITS, np.uint64)) == 0.0
    # ties to even at the rounding boundary: 1 + 2^-53 rounds to 1, 1 + 3 * 2^-53 to 1 + 2^-51
    assert ngx.exact_round(ngx.exact_accumulate([1.0, 2.0 ** -53])) == 1.0
    assert ngx.exact_round(ngx.exact_accumulate([1.0, 2.0 ** -53, 2.0 ** -52])) == 1.0 + 2.0 ** -51
    for bad in ([-1.0], [float("nan")], [float("inf")]):
        with pytest.raises(ngx.NgxError):
            ngx.exact_accumulate(bad)


def test_caller_output_arrays_are_checked():
    """out= arrays (betweenness, gradients) must be writeable C-contiguous float64 arrays with room for every entry;
    anything else is refused before the library is called."""
    good = np.zeros(8)
    assert ngx._out_array(good, 8) is not None and ngx._out_array(good, 5).size == 8
    ro = np.zeros(8)
    ro.flags.writeable = False
    for bad in (np.zeros(8, np.float32), np.zeros(7), np.zeros((8, 2))[:, 0], ro, [0.0] * 8):
        with pytest.raises(ValueError):
            ngx._out_array(bad, 8)
