"""The Python host mirror's own logic, without a device: Sparsifier.insert (sparsifier.rs:357-376) collects
edges as the reference's Triplet does (upper triangle, zero values and self-loops skipped, duplicates summed
by to_csc, sparsifier.rs:48-70,83-87), the threshold is n * round(beta) * row_constant (sparsifier.rs:264-266,
f64::round rounding half away from zero), and building one or inserting into one needs no GPU."""
import math

import numpy as np
import pytest


def test_insert_collects_a_symmetric_graph(ssp):
    prm = ssp.SparsifierParameters.new_default()
    sp = ssp.Sparsifier(6, prm)
    for v1, v2, w in [(0, 1, 1.5), (1, 0, 0.5), (2, 3, 2.0), (4, 4, 9.0), (3, 5, 0.0), (5, 2, 1.0)]:
        sp.insert(v1, v2, w)
    G = sp.graph
    A = G.to_scipy().toarray()
    want = np.zeros((6, 6))
    want[0, 1] = want[1, 0] = 2.0  # both orientations of one edge, summed
    want[2, 3] = want[3, 2] = 2.0
    want[2, 5] = want[5, 2] = 1.0
    assert np.array_equal(A, want)
    assert np.all(np.diff(G.colptr) >= 0) and sp.num_edges() is None  # nothing sparsified yet


def test_insert_rejects_vertices_out_of_range(ssp):
    sp = ssp.Sparsifier(4, ssp.SparsifierParameters.new_default())
    for v1, v2 in [(-1, 2), (0, 4), (7, 1)]:
        with pytest.raises(ssp.SspError):
            sp.insert(v1, v2, 1.0)
    assert sp.graph.nnz == 0


@pytest.mark.parametrize("n", [10, 1000, 123_457])
def test_threshold(ssp, n):
    prm = ssp.SparsifierParameters.new_default()
    sp = ssp.Sparsifier(n, prm)
    beta = math.pow(prm.epsilon, -2.0) * prm.beta_constant * math.log(n)
    assert sp.threshold == n * int(math.floor(beta + 0.5)) * prm.row_constant


def test_built_from_a_graph_all_edges_pending(ssp):
    G = ssp.gen_grid2d(7, 5)
    sp = ssp.Sparsifier(G, ssp.SparsifierParameters.cli(0.5))
    P = sp.graph
    assert P.n == G.n and np.array_equal(P.colptr, G.colptr) and np.array_equal(P.rowidx, G.rowidx)
    assert np.array_equal(P.values, G.values)


def test_streaming_off_never_triggers(ssp):
    """With params.streaming unset, insert only collects (the trigger would need a device)."""
    prm = ssp.SparsifierParameters.new_default()
    assert prm.streaming == 0
    sp = ssp.Sparsifier(50, prm)
    rng = np.random.default_rng(1)
    for _ in range(2000):
        a, b = rng.integers(0, 50, 2)
        sp.insert(int(a), int(b), float(rng.uniform(0.5, 2.0)))
    assert sp.current_laplacian is None and sp.stats is None
