"""Parity at the benchmark's full size (connectome N=100000, ~9.9M arcs, log-normal FP64 weights).

The oracle is too slow for all 1e5 sources, so this checks a seeded sample of sources against it (per-source exact
sums, maxima, unreachable and traversed-arc counts bit for bit; betweenness of the sample within 1e-12 relative), and
size-independent properties of a full wave of 9,472 sources: the exact sums of disjoint chunks merge to the sum of the
whole wave, per-source sums add up to the wave total exactly (a checksum of checksums), and a repeated run gives the
same bits.
"""

from __future__ import annotations

import numpy as np
import pytest

import neurograph_b200 as ngx
import oracle
from neurograph_b200 import synth

pytestmark = pytest.mark.gpu

REL = 1e-12


@pytest.fixture(scope="module")
def graph():
    c = synth.connectome(100_000, 100, 0.08, weights="lognormal", mu=0.0, sigma=1.0, seed=2)
    try:
        import torch

        torch.cuda.empty_cache()
    except Exception:  # noqa: BLE001
        pass
    return c


def test_sampled_sources_match_the_oracle(graph, restatement):
    c = graph
    csr = oracle.Csr.from_arrays(c.n, c.row_ptr, c.col, c.w)
    sample = np.random.default_rng(7).choice(c.n, size=3, replace=False)
    want = restatement.apsp(csr, sources=sample, bins=1024, hist_max=2.0)
    with ngx.Graph(c.n, c.row_ptr, c.col, c.w) as g:
        got = g.apsp(sources=sample, per_source=True, hist_bins=1024, hist_max=2.0)
        bc, _ = g.brandes(sources=sample)
    for k in ("sum", "sum_inv", "max", "unreachable", "arcs"):
        assert np.array_equal(got.per_source[k], want["per_source"][k]), k
    assert got.sum_distances == want["sum_distances"] and got.sum_inverse == want["sum_inverse"]
    assert np.array_equal(got.hist, want["hist"]) and got.hist_overflow == want["hist_overflow"]
    want_bc = restatement.brandes(csr, sources=sample)
    floor = REL * max(1.0, float(np.abs(want_bc).mean()))
    assert np.all(np.abs(bc - want_bc) <= np.maximum(REL * np.abs(want_bc), floor))


def test_full_wave_properties(graph):
    c = graph
    with ngx.Graph(c.n, c.row_ptr, c.col, c.w) as g:
        wave = g.source_order()[: 296 * 32]
        whole = g.apsp(sources=wave, per_source=True, exact=True)
        again = g.apsp(sources=wave, per_source=True, exact=True)
        digits = np.zeros((2, ngx.ACC_DIGITS), np.uint64)
        for chunk in np.array_split(wave, 3):
            digits += g.apsp(sources=chunk, exact=True).acc_digits
    assert np.array_equal(whole.acc_digits, again.acc_digits)
    assert whole.sum_distances == again.sum_distances and whole.diameter == again.diameter
    assert ngx.exact_round(digits[0]) == whole.sum_distances
    assert ngx.exact_round(digits[1]) == whole.sum_inverse
    # checksum of checksums: the exactly rounded per-source sums, summed exactly, round to the wave's total
    # (each per-source sum is itself exactly rounded, so compare within one rounding per source)
    total = ngx.exact_round(ngx.exact_accumulate(whole.per_source["sum"]))
    assert abs(total - whole.sum_distances) <= wave.size * np.spacing(whole.per_source["sum"].max())
    assert whole.traversed_arcs == int(whole.per_source["arcs"].sum())
    assert whole.unreachable == int(whole.per_source["unreachable"].sum())
