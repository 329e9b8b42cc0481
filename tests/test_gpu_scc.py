"""ngx_scc through the C ABI: the GPU's strongly connected components must equal the reference's golden values and,
vertex by vertex, the oracle's Tarjan components (both name a component by its largest vertex), on the golden fixtures,
on generated graphs with many components of mixed sizes and on a full-size synthetic connectome."""

from __future__ import annotations

import ctypes

import numpy as np
import pytest

import neurograph_b200 as ngx
import oracle
from neurograph_b200 import synth
from test_scc import FAMILIES, GOLDEN, scc_family, summary

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name,count,largest,sizes,line", GOLDEN, ids=[g[0] for g in GOLDEN])
def test_reference_golden_values(golden, restatement, name, count, largest, sizes, line):
    g = golden[name]
    got = ngx.Graph(g.n, g.row_ptr, g.col, g.w).scc()
    assert summary(got) == {"number_components": count, "largest_component_size": largest, "component_sizes": sizes}, \
        f"tests/scc/test_tarjan_gathered.cpp:{line}"
    assert np.array_equal(got["component"], restatement.scc(g.csr())["component"])


@pytest.mark.parametrize("kind", FAMILIES)
@pytest.mark.parametrize("n", [1, 2, 257, 20000])
def test_matches_the_oracle(restatement, kind, n):
    n, rp, c, w = scc_family(kind, n, seed=n)
    want = restatement.scc(oracle.Csr.from_arrays(n, rp, c, w))
    got = ngx.Graph(n, rp, c, w).scc()
    assert np.array_equal(got["component"], want["component"])
    assert summary(got) == summary(want)


def test_full_size_connectome(restatement):
    c = synth.connectome(100_000, 100, 0.08, weights="lognormal", seed=1, use_gpu=True)
    want = restatement.scc(oracle.Csr.from_arrays(c.n, c.row_ptr, c.col, c.w))
    g = ngx.Graph(c.n, c.row_ptr, c.col, c.w)
    got = g.scc()
    assert np.array_equal(got["component"], want["component"])
    assert summary(g.scc()) == summary(want)  # a second call on the same handle reuses its buffers


def test_empty_graph_and_batch_handle():
    got = ngx.Graph(0, np.zeros(1, np.int64), np.zeros(0, np.int32), np.zeros(0)).scc()
    assert summary(got) == {"number_components": 0, "largest_component_size": 0, "component_sizes": {}}
    rp = np.array([0, 1, 2], np.int64)
    b = ngx.Batch([(2, rp, np.array([1, 0], np.int32), np.ones(2))] * 2)
    count, largest = ctypes.c_uint64(), ctypes.c_uint64()
    with pytest.raises(ngx.NgxError, match="batch"):
        ngx._check(ngx.library().ngx_scc(b._handle, None, ctypes.byref(count), ctypes.byref(largest), None))
