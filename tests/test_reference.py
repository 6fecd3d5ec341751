"""The oracle's solve stage pinned against the reference's own solver.

oracle/_ref/ref_solve is the reference's src/example.cc factorization_driver (parallel randomized Cholesky +
the PCG driver of include/custom_cg.hpp) compiled from the reference's sources with an MKL protocol shim.
Its factorization is randomized and thread-scheduled, so agreement is measured on what the sparsifier
consumes: the per-edge norms d_e = ||Z[v1_e] - Z[v2_e]|| of the solutions (sparsifier.rs:622-640), which
must agree to 1e-3 relative -- both solvers stop at ||r|| <= sqrt(2e-7) (custom_cg.hpp:159,213), which
leaves them within ~1e-4 of an exact solve on these graphs.
"""
import math

import numpy as np
import pytest

refsolver = pytest.importorskip("refsolver")
pytestmark = pytest.mark.skipif(not refsolver.available(), reason="oracle/_ref/ref_solve is not built")

CASES = {
    "grid30": lambda S: S.gen_grid2d(30, 30),
    "er5k": lambda S: S.gen_er(5000, 20.0, 0.5, 2.0, 1),
    "grid3d": lambda S: S.gen_grid3d(10, 9, 8, -3, 3, 2),
    "er2k_isolated_vertex": lambda S: S.gen_er(2000, 10.0, 0.5, 2.0, 3),
}
ABS_TOL = math.sqrt(2e-7)  # custom_cg.hpp:159 (dpar[0] = 2e-7, compared as sqrt, :213)


def _lap(ora, G):
    v1, v2, w = ora.extract_edges(G.n, G.colptr, G.rowidx, G.values)
    return (v1, v2, w), ora.laplacian(G.n, v1, v2, w)


@pytest.mark.parametrize("name", list(CASES))
def test_reference_solver_leverage_matches_oracle(ssp, ora, name):
    G = CASES[name](ssp)
    (v1, v2, w), (cp, ri, va) = _lap(ora, G)
    k = 24
    Y = ora.sketch(G.n, v1, v2, w, k, 1 / math.sqrt(k), 0)
    status, _, Xr = refsolver.solve(G.n, cp, ri, va, Y, threads=2)
    assert status == 0
    F = ora.Factor(G.n, cp, ri, va, 0, 4096, 0)
    Xo, iters, rel, rc = ora.pcg(G.n, cp, ri, va, F, Y, 0.0, ABS_TOL, 400)
    assert rc == 0 and iters.max() < 400
    dr, do = ora.diff_norms(v1, v2, Xr), ora.diff_norms(v1, v2, Xo)
    live = do > 1e-12
    assert live.sum() > 0.99 * len(do)
    assert np.max(np.abs(dr[live] - do[live]) / do[live]) < 1e-3
    beta = math.pow(0.5, -2) * 4 * math.log(G.n)  # sparsifier.rs:264
    pr, po = ora.probs(w, dr, beta, 1.0), ora.probs(w, do, beta, 1.0)
    assert np.max(np.abs(pr - po) / np.maximum(po, 1e-300)) < 2.5e-3


def test_reference_and_oracle_both_reject_inconsistent_rhs(ssp, ora):
    # a random zero-sum right-hand side is not in the range of a Laplacian with an isolated vertex: the
    # reference throws "solver did not converge" (example.cc:566), the oracle reports non-convergence
    G = CASES["er2k_isolated_vertex"](ssp)
    (v1, v2, w), (cp, ri, va) = _lap(ora, G)
    assert np.any(np.diff(cp) == 0)
    B = np.random.default_rng(0).standard_normal((G.n, 2))
    B -= B.mean(0)
    status, _, _ = refsolver.solve(G.n, cp, ri, va, B, threads=2)
    assert status == 2
    F = ora.Factor(G.n, cp, ri, va, 0, 4096, 0)
    _, iters, rel, rc = ora.pcg(G.n, cp, ri, va, F, B, 0.0, ABS_TOL, 400)
    assert rc != 0 and iters.max() == 400 and rel.max() >= 0.01


def test_reference_solve_start_times(ora):
    # the MKL shim records when each of the reference's sequential PCG solves starts (example.cc:551-568):
    # one start per right-hand side, after the set-up and factorization, in increasing order, within the run
    n = 3000
    v1, v2, w = ora.gen_er(n, 12.0, 0.5, 2.0, 4)
    cp, ri, va = ora.laplacian(n, v1, v2, w)
    Y = ora.sketch(n, v1, v2, w, 5, 1 / math.sqrt(5), 0)
    status, secs, X, starts = refsolver.solve(n, cp, ri, va, Y, threads=2, timings=True)
    assert status == 0 and X.shape == (n, 5)
    assert len(starts) == 5 and starts[0] > 0 and np.all(np.diff(starts) > 0) and starts[-1] < secs
