"""ngx_apsp_noalloc (APSP from the library's fixed scratch array, no device allocation) against ngx_apsp.

Tolerance: none. Every output of both entry points is exact or exactly rounded (integer counts, the exact sums of d
and 1/d rounded once, maxima of stored lengths, histogram counts), and both run the same tile kernel, so the two must
agree bit for bit; NaN averages (no reached pairs) count as equal. Each case calls the new entry point twice in a row,
so the second call runs on scratch that the first one left behind.
"""

from __future__ import annotations

import numpy as np
import pytest

import neurograph_b200 as ngx
from neurograph_b200 import synth

pytestmark = pytest.mark.gpu

FIELDS = ("sum_distances", "sum_inverse", "diameter", "unreachable", "reached_pairs", "traversed_arcs", "hist_overflow",
          "cpl", "efficiency")


def same(a: ngx.ApspResult, b: ngx.ApspResult, label):
    for k in FIELDS:
        x, y = getattr(a, k), getattr(b, k)
        assert x == y or (x != x and y != y), (label, k, x, y)
    assert a.cluster_sizes == b.cluster_sizes, label
    if b.hist is not None:
        assert np.array_equal(a.hist, b.hist), label
    if b.per_source is not None:
        for k, v in b.per_source.items():
            assert np.array_equal(a.per_source[k], v), (label, k)


CASES = [
    ("connectome int", lambda: synth.connectome(3000, 10, 0.15, weights="int", seed=21, use_gpu=False)),
    ("connectome lognormal", lambda: synth.connectome(6000, 12, 0.1, weights="lognormal", seed=22, use_gpu=False)),
    ("random unit", lambda: synth.random_graph(2500, 4, weights="unit", seed=23)),
]


@pytest.mark.parametrize("name,make", CASES, ids=[c[0] for c in CASES])
@pytest.mark.parametrize("metric", ["regular", "inverse"])
def test_matches_ngx_apsp_twice_in_a_row(name, make, metric):
    c = make()
    kw = dict(metric=metric, hist_bins=512, hist_max=40.0, per_source=True)
    with ngx.Graph(c.n, c.row_ptr, c.col, c.w) as g:
        want = g.apsp(**kw)
        first = g.apsp_noalloc(**kw)
        second = g.apsp_noalloc(**kw)
    same(first, want, (name, "first"))
    same(second, want, (name, "second"))


def test_source_subset_and_no_optional_outputs():
    c = synth.connectome(5000, 8, 0.2, weights="lognormal", seed=24, use_gpu=False)
    sources = np.random.default_rng(5).choice(c.n, size=777, replace=False)
    with ngx.Graph(c.n, c.row_ptr, c.col, c.w) as g:
        want = g.apsp(sources=sources, per_source=True)
        got = [g.apsp_noalloc(sources=sources, per_source=True) for _ in range(2)]
        bare_want = g.apsp()
        bare = [g.apsp_noalloc() for _ in range(2)]
    for r in got:
        same(r, want, "subset")
    for r in bare:
        same(r, bare_want, "all sources, summaries only")


def test_largest_graph_with_few_workspace_slots():
    """At the vertex limit a workspace slot is ~9.2 MB, so only three fit beside the outputs: ten source tiles then
    reuse each slot several times, as they never do on the smaller graphs above."""
    c = synth.random_graph(ngx_limit(), 3, weights="lognormal", seed=27)
    sources = np.random.default_rng(8).choice(c.n, size=300, replace=False)
    kw = dict(sources=sources, per_source=True, hist_bins=256, hist_max=20.0)
    with ngx.Graph(c.n, c.row_ptr, c.col, c.w) as g:
        want = g.apsp(**kw)
        got = [g.apsp_noalloc(**kw) for _ in range(2)]
    for r in got:
        same(r, want, "n = 32768")


def test_limits_are_rejected():
    big = synth.random_graph(ngx_limit() + 1, 1, weights="int", seed=25)
    with ngx.Graph(big.n, big.row_ptr, big.col, big.w) as g:
        with pytest.raises(ngx.NgxError, match="at most 32768"):
            g.apsp_noalloc()
    c = synth.connectome(500, 6, 0.2, weights="int", seed=26, use_gpu=False)
    with ngx.Graph(c.n, c.row_ptr, c.col, c.w) as g:
        with pytest.raises(ngx.NgxError, match="hist_max"):
            g.apsp_noalloc(hist_bins=64)
        with pytest.raises(ngx.NgxError):
            g.apsp_noalloc(sources=np.arange(40000) % c.n)
        with pytest.raises(ngx.NgxError):
            g.apsp_noalloc(sources=[c.n])
        # a rejected call leaves the scratch usable
        same(g.apsp_noalloc(hist_bins=64, hist_max=30.0), g.apsp(hist_bins=64, hist_max=30.0), "after rejections")


def ngx_limit() -> int:
    return 32768
