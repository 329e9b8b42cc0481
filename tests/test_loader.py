"""ngx_network_load (host only, no GPU): neurograph's per-rank network files into a global CSR.

Checked against the reference's own loader (DistributedGraph::construct_graph through the shim build, one rank) on its
sample input and on generated files full of the cases the reference's line rules handle (repeated arcs, zero and
negative weights, plastic flags, self arcs, comments, malformed and out-of-range lines), for every combination of the
three transforms; and the same network split over 3 ranks must load to the same global CSR as the 1-rank files.
Arcs are compared as sorted (source, target, weight) triples: the reference stores a vertex's arcs in hash-map order.
"""

from __future__ import annotations

import itertools
import os

import numpy as np
import pytest

import neurograph_b200 as ngx
import oracle

FLAGS = list(itertools.product([False, True], repeat=3))
SAMPLE = os.path.join(oracle.REFERENCE_SOURCES or "", "input", "rank_1_nodes_5000_arcs_6")


def triples(n, row_ptr, col, w):
    u = np.repeat(np.arange(n, dtype=np.int64), np.diff(row_ptr))
    t = np.stack([u, np.asarray(col, np.int64), np.asarray(w, np.float64).astype(np.int64)], 1)
    return t[np.lexsort((t[:, 2], t[:, 1], t[:, 0]))]


def reference():
    if not oracle.Reference.available():
        pytest.skip("the reference build (oracle/_ref) is not here")
    return oracle.Reference()


def write_network(directory, n, ranks, rng):
    """A random network with every kind of line the loader must handle, written as `ranks` per-rank file sets; the
    same seed gives the same global network for any number of ranks."""
    bounds = np.linspace(0, n, ranks + 1).astype(np.int64)

    def where(g):
        r = int(np.searchsorted(bounds, g, side="right") - 1)
        return r, int(g - bounds[r]) + 1  # 1-based local id

    arcs = []  # (source, target, weight, plastic or None)
    for _ in range(6 * n):
        u, v = (int(x) for x in rng.integers(0, n, 2))
        if rng.random() < 0.05:
            v = u  # self arc
        w = int(rng.integers(-5, 6))  # zeros and negatives included
        plastic = None if rng.random() < 0.5 else int(rng.random() < 0.9)
        arcs.append((u, v, w, plastic))
        if rng.random() < 0.2:
            arcs.append((u, v, int(rng.integers(-5, 6)), None))  # repeated arc: weights sum
    in_arcs = [(u, v, w, p) for (u, v, w, p) in arcs if rng.random() < 0.7]  # in files need not mirror out files
    os.makedirs(os.path.join(directory, "positions"), exist_ok=True)
    os.makedirs(os.path.join(directory, "network"), exist_ok=True)
    width = len(str(ranks - 1))
    for r in range(ranks):
        name = f"rank_{r:0{width}d}"
        with open(os.path.join(directory, "positions", f"{name}_positions.txt"), "w") as f:
            f.write(f"# {bounds[r + 1] - bounds[r]} of {n}\n# <local id> <pos x> <pos y> <pos z> <type>\n")
            for i in range(int(bounds[r + 1] - bounds[r])):
                f.write(f"{i + 1} {rng.random():.6f} {rng.random():.6f} {rng.random():.6f} {'ex' if rng.random() < 0.8 else 'in'}\n")

        def line(u, v, w, p):
            tr, tid = where(v)
            sr, sid = where(u)
            tail = "" if p is None else f"\t{p}"
            return f"{tr} {tid}\t{sr} {sid}\t{w}{tail}\n"

        for kind, selected in (("out", [a for a in arcs if where(a[0])[0] == r]), ("in", [a for a in in_arcs if where(a[1])[0] == r])):
            with open(os.path.join(directory, "network", f"{name}_{kind}_network.txt"), "w") as f:
                f.write("# Total number neurons: %d\n# <target rank> <target neuron id>\t<source rank> <source neuron id>\t<weight>\n" % n)
                for a in selected:
                    f.write(line(*a))
                f.write("\n")
                f.write("this line does not parse\n")
                f.write(f"{r} 0 {r} 1 3\n")  # id 0: out of range after the 1-based shift
                f.write(f"{r} {n + 5} {r} 1 3\n")  # target beyond the rank's vertices
                f.write(f"{ranks + 2} 1 {r} 1 3\n" if kind == "out" else f"{r} 1 {ranks + 2} 1 3\n")  # unknown rank


@pytest.mark.skipif(not os.path.isdir(SAMPLE), reason="the reference's sample input is not here")
@pytest.mark.parametrize("remove_self_arcs,undirected,one_weight", FLAGS)
def test_sample_input_matches_the_reference_loader(remove_self_arcs, undirected, one_weight):
    ref = reference()
    want = ref.load_csr(SAMPLE, remove_self_arcs=remove_self_arcs, undirected=undirected, one_weight=one_weight)
    got = ngx.load_network(SAMPLE, 1, remove_self_arcs=remove_self_arcs, undirected=undirected, one_weight=one_weight)
    assert got[0] == want[0]
    assert np.array_equal(triples(*got), triples(*want))


@pytest.mark.parametrize("remove_self_arcs,undirected,one_weight", FLAGS)
def test_generated_files_match_the_reference_loader(tmp_path, remove_self_arcs, undirected, one_weight):
    ref = reference()
    write_network(str(tmp_path), 300, 1, np.random.default_rng(5))
    want = ref.load_csr(str(tmp_path), remove_self_arcs=remove_self_arcs, undirected=undirected, one_weight=one_weight)
    got = ngx.load_network(str(tmp_path), 1, remove_self_arcs=remove_self_arcs, undirected=undirected, one_weight=one_weight, threads=3)
    assert got[0] == want[0] == 300
    assert np.array_equal(triples(*got), triples(*want))
    assert (got[3] != 0).all()
    for v in range(got[0]):
        row = got[2][got[1][v]:got[1][v + 1]]
        assert (np.diff(row) > 0).all()  # each row sorted by target, no repeats


@pytest.mark.parametrize("remove_self_arcs,undirected,one_weight", FLAGS)
def test_ranks_split_loads_the_same_global_graph(tmp_path, remove_self_arcs, undirected, one_weight):
    one, three = tmp_path / "one", tmp_path / "three"
    write_network(str(one), 400, 1, np.random.default_rng(9))
    write_network(str(three), 400, 3, np.random.default_rng(9))
    kw = dict(remove_self_arcs=remove_self_arcs, undirected=undirected, one_weight=one_weight)
    a = ngx.load_network(str(one), 1, **kw)
    b = ngx.load_network(str(three), 3, **kw)
    assert a[0] == b[0] == 400
    assert np.array_equal(a[1], b[1]) and np.array_equal(a[2], b[2]) and np.array_equal(a[3], b[3])


def test_missing_files_are_errors(tmp_path):
    with pytest.raises(ngx.NgxError, match="cannot read"):
        ngx.load_network(str(tmp_path), 1)
    write_network(str(tmp_path), 50, 2, np.random.default_rng(1))
    with pytest.raises(ngx.NgxError, match="cannot read"):
        ngx.load_network(str(tmp_path), 3)  # rank_2 files do not exist
