"""Strongly connected components, host side (no GPU): the oracle's Tarjan (oracle/ngx_oracle.c, ngxo_scc) pinned to
the golden values of the reference's SCC tests (tests/scc/test_tarjan_gathered.cpp; the forward-backward, coloring and
multistep files assert the same values) and to the reference's own StronglyConnectedComponents, all four algorithms,
built from source (oracle/_ref), on generated graphs with many components of mixed sizes; and the component names
(largest member) checked against brute-force reachability on small graphs."""

from __future__ import annotations

import numpy as np
import pytest

import oracle

# fixture -> (number_components, largest_component_size, component_sizes, line of the assertion)
GOLDEN = [
    ("standard", 1, 10, {10: 1}, 37), ("standard_uu", 1, 10, {10: 1}, 53), ("full", 1, 10, {10: 1}, 69),
    ("empty", 0, 0, {}, 84), ("negative_weight", 4, 1, {1: 4}, 100),
    ("multi_component_four_rank_on_one_rank", 7, 4, {1: 4, 2: 2, 4: 1}, 117),
    ("standard_four_rank_on_one_rank", 1, 40, {40: 1}, 134), ("full_four_rank_on_one_rank", 1, 36, {36: 1}, 149),
    ("standard_seven_rank_on_one_rank", 12, 40, {1: 10, 20: 1, 40: 1}, 213),
    ("standard_uu_seven_rank_on_one_rank", 8, 40, {1: 3, 2: 2, 3: 1, 20: 1, 40: 1}, 230),
    ("full_seven_rank_on_one_rank", 1, 63, {63: 1}, 245),
]
ALGORITHMS = {"tarjan_gathered": 0, "forward_backward": 1, "coloring": 2, "multistep": 3}


def summary(out):
    return {k: out[k] for k in ("number_components", "largest_component_size", "component_sizes")}


def csr_from_pairs(n, src, dst, w=None, rng=None):
    """CSR of the arcs (src[i] -> dst[i]) in that order within each source row; weights 1..9 unless given."""
    src = np.asarray(src, np.int64)
    dst = np.asarray(dst, np.int64)
    order = np.argsort(src, kind="stable")
    row_ptr = np.zeros(n + 1, np.int64)
    np.add.at(row_ptr, src + 1, 1)
    if w is None:
        w = (rng or np.random.default_rng(0)).integers(1, 10, src.size)
    return n, np.cumsum(row_ptr), dst[order].astype(np.int32), np.asarray(w, np.float64)[order]


def scc_family(kind, n, seed):
    """Graphs with many strongly connected components of mixed sizes (all with integer weights)."""
    rng = np.random.default_rng(seed)
    if kind == "sparse":  # random digraph near its giant-component threshold: components of every size
        m = int(1.3 * n)
        return csr_from_pairs(n, rng.integers(0, n, m), rng.integers(0, n, m), rng=rng)
    if kind == "cycles_dag":  # cycles of random lengths, joined by forward arcs only (a DAG of cycles), plus self arcs
        cuts = np.sort(rng.choice(np.arange(1, n), size=min(n - 1, max(1, n // 7)), replace=False))
        perm = rng.permutation(n)
        src, dst = [], []
        for block in np.split(np.arange(n), cuts):
            ring = perm[block]
            if ring.size > 1 and rng.random() < 0.8:
                src += list(ring)
                dst += list(np.roll(ring, -1))
        pos = np.empty(n, np.int64)
        pos[perm] = np.arange(n)
        for _ in range(2 * n):
            a, b = rng.integers(0, n, 2)
            if pos[a] < pos[b] and np.searchsorted(cuts, pos[a], "right") != np.searchsorted(cuts, pos[b], "right"):
                src.append(a)
                dst.append(b)
        loops = rng.integers(0, n, n // 10)
        return csr_from_pairs(n, src + list(loops), dst + list(loops), rng=rng)
    if kind == "zero_weights":  # zero-weight arcs are absent arcs: they must not join components
        m = 3 * n
        src, dst = rng.integers(0, n, m), rng.integers(0, n, m)
        w = rng.integers(1, 10, m) * (rng.random(m) < 0.6)
        return csr_from_pairs(n, src, dst, w=w)
    if kind == "isolated":  # a strongly connected core, a tail of arcs into and out of it, and vertices without arcs
        core = max(1, n // 3)
        src = list(range(core)) + list(rng.integers(0, core, core))
        dst = [(i + 1) % core for i in range(core)] + list(rng.integers(0, core, core))
        for v in range(core, 2 * n // 3):
            if rng.random() < 0.5:
                src.append(v), dst.append(int(rng.integers(0, core)))
            else:
                src.append(int(rng.integers(0, core))), dst.append(v)
        return csr_from_pairs(n, src, dst, rng=rng)
    if kind == "path":  # one long path and one long cycle: the longest trims and colourings
        half = n // 2
        src = list(range(half - 1)) + list(range(half, n))
        dst = list(range(1, half)) + list(range(half + 1, n)) + [half]
        return csr_from_pairs(n, src, dst[: len(src)], rng=rng)
    raise ValueError(kind)


FAMILIES = ["sparse", "cycles_dag", "zero_weights", "isolated", "path"]


def reachability(n, row_ptr, col, w):
    reach = np.eye(n, dtype=bool)
    for u in range(n):
        for e in range(row_ptr[u], row_ptr[u + 1]):
            if w[e] != 0:
                reach[u, col[e]] = True
    for k in range(n):  # Warshall
        reach |= reach[:, k:k + 1] & reach[k:k + 1, :]
    return reach


@pytest.mark.parametrize("name,count,largest,sizes,line", GOLDEN, ids=[g[0] for g in GOLDEN])
def test_oracle_matches_the_reference_golden_values(golden, restatement, name, count, largest, sizes, line):
    g = golden[name]
    got = restatement.scc(g.csr())
    assert summary(got) == {"number_components": count, "largest_component_size": largest, "component_sizes": sizes}, \
        f"tests/scc/test_tarjan_gathered.cpp:{line}"


@pytest.mark.parametrize("kind", FAMILIES)
@pytest.mark.parametrize("seed", [0, 1])
def test_oracle_names_match_brute_force_reachability(restatement, kind, seed):
    n, rp, c, w = scc_family(kind, 60, seed)
    reach = reachability(n, rp, c, w)
    mutual = reach & reach.T
    want = np.array([np.nonzero(mutual[v])[0].max() for v in range(n)], np.int32)
    got = restatement.scc(oracle.Csr.from_arrays(n, rp, c, w))
    assert np.array_equal(got["component"], want)


@pytest.mark.parametrize("kind", FAMILIES)
def test_oracle_matches_the_reference_algorithms(restatement, kind):
    if not oracle.Reference.available():
        pytest.skip("the reference build (oracle/_ref) is not here")
    ref = oracle.Reference()
    for seed in (3, 4):
        n, rp, c, w = scc_family(kind, 2000, seed)
        want = summary(restatement.scc(oracle.Csr.from_arrays(n, rp, c, w)))
        assert want["number_components"] > (1 if kind != "path" else 2)
        rg = ref.graph(n, rp, c, w.astype(np.int32))
        for name, algorithm in ALGORITHMS.items():
            assert rg.scc(algorithm) == want, name
        assert rg.scc(3, tail_threshold=500) == want
