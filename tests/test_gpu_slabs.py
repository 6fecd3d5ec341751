"""Column slabs of the PCG's Laplacian product: on a random graph whose gathered tile is larger than the slab
budget the SpMM runs one pass per column slab (the first writes q, the others add into it).  The budget is an
environment knob (SSP_SPMM_SLAB_MB), so small graphs here take the same code path as n = 1M does at the
default budget.  Tolerance as the single-pass solve: diff norms within 1e-7 of the oracle's at tol 1e-10."""
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SMALL_BUDGET_MB = "0.25"  # 1024 rows of 32 FP64 columns per slab


def _oracle_graph(ora, G):
    v1, v2, w = ora.extract_edges(G.n, G.colptr, G.rowidx, G.values)
    return (v1, v2, w), ora.laplacian(G.n, v1, v2, w)


CASES = {
    "er6k": lambda ssp: ssp.gen_er(6000, 20.0, 0.5, 2.0, 11),
    # hubs: a hub's share of one slab is still longer than a chunk and takes the long-row path
    "rmat12": lambda ssp: ssp.gen_rmat(12, 16, 0.57, 0.19, 0.19, 5),
}


@pytest.mark.parametrize("name", list(CASES))
@pytest.mark.parametrize("k", [5, 40])
def test_slab_solve_matches_oracle(ssp, ora, ctx, monkeypatch, name, k):
    G = CASES[name](ssp)
    (v1, v2, w), (cp, ri, va) = _oracle_graph(ora, G)
    lap = ssp.CSC(G.n, cp, ri, va)
    Y = ora.sketch(G.n, v1, v2, w, k, 1 / math.sqrt(k), 7)
    monkeypatch.setenv("SSP_SPMM_SLAB_MB", SMALL_BUDGET_MB)
    Z, rep = ctx.solve_lap(lap, Y, tol=1e-10, abs_tol=0.0, max_iters=400, factor_seed=2, max_degree=16)
    monkeypatch.setenv("SSP_SPMM_SLAB_MB", "0")
    Z1, rep1 = ctx.solve_lap(lap, Y, tol=1e-10, abs_tol=0.0, max_iters=400, factor_seed=2, max_degree=16)
    assert rep["spmm_slabs"] == math.ceil(G.n / 1024) and rep1["spmm_slabs"] == 1
    assert rep["not_converged"] == 0 and rep["max_relres"] < 1e-8
    F = ora.Factor(G.n, cp, ri, va, 2, 4096, 16)
    Zo, it, _, rc = ora.pcg(G.n, cp, ri, va, F, Y, 1e-10, 0.0, 400)
    assert rc == 0
    dz, d1, do = Z[v1] - Z[v2], Z1[v1] - Z1[v2], Zo[v1] - Zo[v2]
    assert np.abs(dz - do).max() <= 1e-7 * np.abs(do).max()
    assert np.abs(dz - d1).max() <= 1e-7 * np.abs(d1).max()
    assert abs(rep["max_iters_used"] - it.max()) <= 2


def test_slabs_skipped_when_the_matrix_is_local(ssp, ctx, monkeypatch):
    """A grid's entries sit within a few rows of the diagonal: a row sweep already reuses L2, no slabs."""
    G = ssp.gen_grid2d(100, 100)
    monkeypatch.setenv("SSP_SPMM_SLAB_MB", SMALL_BUDGET_MB)
    _, st = ctx.sparsify(G, ssp.SparsifierParameters.baseline(1.0, pcg_tol=1e-8))
    assert st["spmm_slabs"] == 1


def test_slab_mixed_precision_reaches_tolerance(ssp, ora, ctx, monkeypatch):
    G = CASES["er6k"](ssp)
    (v1, v2, w), (cp, ri, va) = _oracle_graph(ora, G)
    lap = ssp.CSC(G.n, cp, ri, va)
    Y = ora.sketch(G.n, v1, v2, w, 21, 1 / math.sqrt(21), 9)
    monkeypatch.setenv("SSP_SPMM_SLAB_MB", SMALL_BUDGET_MB)
    Zm, rm = ctx.solve_lap(lap, Y, tol=1e-9, abs_tol=0.0, max_iters=600, precision=1)
    assert rm["spmm_slabs"] == 6 and rm["refinements"] >= 1 and rm["max_relres"] <= 1e-9 * 1.0001
    F = ora.Factor(G.n, cp, ri, va, 0, 4096, rm["factor_max_degree_used"])
    Zo, _, _, rc = ora.pcg(G.n, cp, ri, va, F, Y, 1e-9, 0.0, 600)
    assert rc == 0
    dm, do = ora.diff_norms(v1, v2, Zm), ora.diff_norms(v1, v2, Zo)
    live = do > 1e-12 * do.max()
    assert np.max(np.abs(dm[live] - do[live]) / do[live]) < 1e-6


def test_slab_sparsify_matches_oracle(ssp, ora, ctx, monkeypatch):
    G = ssp.gen_er(6000, 40.0, 0.5, 2.0, 13)
    prm = ssp.SparsifierParameters.baseline(1.5, pcg_tol=1e-10)
    monkeypatch.setenv("SSP_SPMM_SLAB_MB", SMALL_BUDGET_MB)
    H, st = ctx.sparsify(G, prm)
    assert st["spmm_slabs"] == 6
    (v1, v2, w), (cp, ri, va) = _oracle_graph(ora, G)
    k, s = prm.jl_dim(G.n), prm.jl_scale(prm.jl_dim(G.n))
    Y = ora.sketch(G.n, v1, v2, w, k, s, prm.sketch_seed, prm.sketch_uniform)
    F = ora.Factor(G.n, cp, ri, va, prm.factor_seed, prm.dense_threshold, st["factor_max_degree_used"])
    Z, _, _, rc = ora.pcg(G.n, cp, ri, va, F, Y, prm.pcg_tol, prm.pcg_abs_tol, prm.pcg_max_iters)
    assert rc == 0
    p = ora.probs(w, ora.diff_norms(v1, v2, Z), prm.beta(G.n), k * s * s)
    (hcp, hri, hva), keep = ora.sample_apply(G.n, v1, v2, w, p, ora.coins(prm.sampling_seed, len(w)), prm.reweight,
                                             (cp, ri, va))
    assert st["m_out"] == int(keep.sum()) and 0 < st["m_out"] < st["m_in"]
    assert np.array_equal(H.colptr, hcp) and np.array_equal(H.rowidx, hri)
    np.testing.assert_allclose(H.values, hva, rtol=1e-12, atol=1e-12)
