"""ngx_diameter_approximation through the C ABI: the contracted graph's diameter from the batched GPU kernel plus 2r
must equal the reference's golden values and the host contraction + oracle APSP, exactly (integers)."""

from __future__ import annotations

import numpy as np
import pytest

import neurograph_b200 as ngx
from test_diameter import GOLDEN, approximation, symmetric_graph

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name,r,draws,value,line", GOLDEN, ids=[f"{g[0]}-r{g[1]}-{len(g[2])}" for g in GOLDEN])
def test_reference_golden_values(golden, name, r, draws, value, line):
    g = golden[name]
    assert ngx.diameter_approximation(g.n, g.row_ptr, g.col, g.w, r, draws=draws) == value, f"test_diameter_approximation.cpp:{line}"


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_matches_the_host_path(restatement, seed):
    n, rp, c, w = symmetric_graph(1500, 8, seed=60 + seed)
    for r in (1, 3):
        want = approximation(restatement, n, rp, c, w, r, seed=seed)
        assert ngx.diameter_approximation(n, rp, c, w, r, seed=seed) == want
