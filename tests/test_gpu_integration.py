"""The reference-side adapter (neurograph_b200/host/ngx_neurograph.h) compiled into the reference's own code.

oracle/_ref/integration_check (built where the reference sources exist, see oracle/Makefile) runs the reference's
fixture graphs through AllPairsShortestPath / BetweennessCentrality and through the adapter's GPU entry points and
exits non-zero on any mismatch.
"""

from __future__ import annotations

import os
import subprocess

import pytest

import oracle

pytestmark = pytest.mark.gpu


@pytest.mark.skipif(not os.path.exists(oracle.INTEGRATION_CHECK), reason="integration check not built (no reference sources at build time)")
def test_reference_fixtures_through_the_adapter():
    out = subprocess.run([oracle.INTEGRATION_CHECK], capture_output=True, text=True, timeout=300)
    print(out.stdout)
    assert out.returncode == 0, out.stdout[-3000:] + out.stderr[-2000:]
    assert "MISMATCH" not in out.stdout
    assert out.stdout.count("apsp ok") >= 8
