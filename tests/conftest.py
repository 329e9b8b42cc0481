"""Test configuration: the `gpu` marker and shared fixtures (golden fixtures of the reference, the oracle)."""

from __future__ import annotations

import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 and the built CUDA library")


class GoldenGraph:
    """One graph of tests/golden/reference_fixtures.npz with the reference's outputs."""

    def __init__(self, data, name):
        self.name = name
        self._d = data
        self.row_ptr = data[f"{name}/row_ptr"]
        self.col = data[f"{name}/col"]
        self.w_int = data[f"{name}/w"]
        self.n = self.row_ptr.size - 1
        self.w = self.w_int.astype(np.float64)

    def get(self, key):
        k = f"{self.name}/{key}"
        return self._d[k] if k in self._d else None

    def csr(self):
        import oracle

        return oracle.Csr.from_arrays(self.n, self.row_ptr, self.col, self.w)

    def apsp(self, metric="regular"):
        s = self.get(f"{metric}/scalars")
        keys = self.get(f"{metric}/cluster_keys")
        counts = self.get(f"{metric}/cluster_counts")
        return {"cpl": s[0], "efficiency": s[1], "diameter": s[2], "unreachable": int(s[3]),
                "cluster_sizes": {int(k): int(c) for k, c in zip(keys, counts)}}


@pytest.fixture(scope="session")
def golden():
    data = np.load(os.path.join(GOLDEN, "reference_fixtures.npz"))
    names = [str(x) for x in data["names"]]
    return {name: GoldenGraph(data, name) for name in names}


@pytest.fixture(scope="session")
def expectations():
    with open(os.path.join(GOLDEN, "reference_expectations.json")) as f:
        return json.load(f)


@pytest.fixture(scope="session")
def restatement():
    import oracle

    return oracle.Restatement()
