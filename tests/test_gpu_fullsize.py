"""Parity at the benchmark's full size (connectome N=100000, ~9.9M arcs, log-normal FP64 weights).

The oracle is too slow for all 1e5 sources, so this checks 64 seeded sources against it, on host threads: the full
distance rows bit for bit, the per-source exact sums, maxima, unreachable and traversed-arc counts and the 1024-bin
histogram bit for bit, and the betweenness of those sources within 1e-12 relative. A full wave of 9,472 sources is
checked through size-independent properties: the exact sums of disjoint chunks merge to the sum of the whole wave,
per-source sums add up to the wave total (a checksum of checksums), and a repeated run gives the same bits.
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


def test_sampled_sources_match_the_oracle(graph):
    c = graph
    csr = oracle.Csr.from_arrays(c.n, c.row_ptr, c.col, c.w)
    sample = np.random.default_rng(7).choice(c.n, size=64, replace=False)
    check = oracle.ParallelRestatement()
    want_rows = check.sssp_rows(csr, sample)
    want = check.apsp_sources(csr, sample, bins=1024, hist_max=2.0)
    want_bc = check.brandes_sources(csr, sample)
    with ngx.Graph(c.n, c.row_ptr, c.col, c.w) as g:
        rows = g.sssp_rows(sample)
        got = g.apsp(sources=sample, per_source=True, hist_bins=1024, hist_max=2.0)
        bc, _ = g.brandes(sources=sample)
    assert np.array_equal(rows, want_rows)
    for k in ("sum", "sum_inv", "max", "unreachable", "arcs"):
        assert np.array_equal(got.per_source[k], want["per_source"][k]), k
    assert np.array_equal(got.hist, want["hist"]) and got.hist_overflow == want["hist_overflow"]
    assert got.unreachable == want["unreachable"] and got.traversed_arcs == want["traversed_arcs"]
    assert got.diameter == want["diameter"]
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
