"""Cancellation and the workspace budget, exercised without any GPU fault.

* Cancellation: a long all-sources run goes on in one host thread while another thread calls request_abort (the
  mapped host flag that every tile polls once per phase). The run must return NGX_ABORTED, and the same handle must
  then give results equal to the oracle's.
* Memory budget: a budget below one workspace slot must fail with NGX_OUT_OF_MEMORY before any launch; budgets that
  allow one or a few slots run the same tiles with fewer CTAs, so every output must be bit-identical to an
  unbudgeted run (the sums are exact, betweenness is summed in fixed point).
"""

from __future__ import annotations

import threading
import time

import numpy as np
import pytest

import neurograph_b200 as ngx
import oracle
from neurograph_b200 import synth

pytestmark = pytest.mark.gpu

NGX_ABORTED = 5
NGX_OUT_OF_MEMORY = 2


def _run_with_abort(run):
    """Runs `run()` on a thread and requests an abort every 5 ms until it returns (a run resets the flag when it
    starts, so one early request could be lost). Returns (exception or None, seconds the run took)."""
    box = {}

    def target():
        t0 = time.perf_counter()
        try:
            run()
            box["error"] = None
        except ngx.NgxError as e:  # noqa: PERF203
            box["error"] = e
        box["seconds"] = time.perf_counter() - t0

    th = threading.Thread(target=target)
    th.start()
    return th, box


@pytest.fixture(scope="module")
def long_graph():
    # ~1e11 traversed arcs over all sources: a second or more per run, so the abort lands in flight
    return synth.connectome(50_000, 40, 0.08, weights="lognormal", seed=31)


@pytest.mark.parametrize("task", ["apsp", "brandes"])
def test_abort_from_another_thread(long_graph, restatement, task):
    c = long_graph
    with ngx.Graph(c.n, c.row_ptr, c.col, c.w) as g:
        run = (lambda: g.apsp(hist_bins=64, hist_max=5.0)) if task == "apsp" else (lambda: g.brandes())
        th, box = _run_with_abort(run)
        time.sleep(0.05)
        while th.is_alive():
            g.request_abort()
            th.join(0.005)
        err = box["error"]
        assert err is not None, f"the run finished in {box['seconds']:.2f} s before an abort landed"
        assert err.status == NGX_ABORTED, err
        assert "abort" in str(err)
        # the same handle, a small oracle-checked run
        sources = np.arange(0, c.n, 997)[:48]
        csr = oracle.Csr.from_arrays(c.n, c.row_ptr, c.col, c.w)
        got = g.apsp(sources=sources, per_source=True)
        want = restatement.apsp(csr, sources=sources)
        for k in ("sum", "sum_inv", "max", "unreachable", "arcs"):
            assert np.array_equal(got.per_source[k], want["per_source"][k]), k
        bc, _ = g.brandes(sources=sources)
        bc_want = restatement.brandes(csr, sources=sources)
        floor = 1e-12 * max(1.0, float(np.abs(bc_want).mean()))
        assert np.all(np.abs(bc - bc_want) <= np.maximum(1e-12 * np.abs(bc_want), floor))


def test_abort_request_between_runs_does_not_leak_into_the_next_run():
    c = synth.connectome(2000, 8, 0.15, weights="int", seed=32, use_gpu=False)
    with ngx.Graph(c.n, c.row_ptr, c.col, c.w) as g:
        g.request_abort()
        r = g.apsp()  # a run clears the flag when it starts
        assert r.reached_pairs > 0


@pytest.fixture(scope="module")
def budget_graph():
    return synth.connectome(20_000, 20, 0.1, weights="lognormal", seed=33)


def test_budget_below_one_slot_is_out_of_memory(budget_graph):
    c = budget_graph
    with ngx.Graph(c.n, c.row_ptr, c.col, c.w) as g:
        g.set_memory_budget(1 << 20)  # 1 MiB: a slot of a 20,000-vertex graph needs several MB
        for call in (lambda: g.apsp(), lambda: g.brandes(), lambda: g.apsp_grad()):
            with pytest.raises(ngx.NgxError) as e:
                call()
            assert e.value.status == NGX_OUT_OF_MEMORY
            assert "slot" in str(e.value)
        g.set_memory_budget(0)  # no cap: the handle works again
        assert g.apsp().reached_pairs > 0


@pytest.mark.parametrize("budget_mb", [40, 150])
def test_budgeted_runs_are_bit_identical(budget_graph, budget_mb):
    c = budget_graph
    sources = np.random.default_rng(34).choice(c.n, size=1500, replace=False)
    with ngx.Graph(c.n, c.row_ptr, c.col, c.w) as g:
        free_apsp = g.apsp(sources=sources, per_source=True, hist_bins=256, hist_max=4.0, exact=True)
        free_bc, _ = g.brandes(sources=sources)
        free_dcpl, free_deff, _ = g.apsp_grad(sources=sources)
        g.set_memory_budget(budget_mb << 20)
        cap_apsp = g.apsp(sources=sources, per_source=True, hist_bins=256, hist_max=4.0, exact=True)
        cap_bc, _ = g.brandes(sources=sources)
        cap_dcpl, cap_deff, _ = g.apsp_grad(sources=sources)
    assert np.array_equal(free_apsp.acc_digits, cap_apsp.acc_digits)
    assert np.array_equal(free_apsp.hist, cap_apsp.hist)
    for k, v in free_apsp.per_source.items():
        assert np.array_equal(v, cap_apsp.per_source[k]), k
    assert free_apsp.diameter == cap_apsp.diameter and free_apsp.unreachable == cap_apsp.unreachable
    assert np.array_equal(free_bc, cap_bc)
    assert np.array_equal(free_dcpl, cap_dcpl) and np.array_equal(free_deff, cap_deff)
