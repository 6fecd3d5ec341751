"""SSP_PRECISION_PC32: FP64 PCG whose preconditioner runs in FP32 (the triangular solves of
custom_cg.hpp:224-235 on FP32 factor values and FP32 rows).  The PCG recurrences, the Laplacian product and
every dot product stay FP64, and the stopping test is the FP64 one, so the solution meets the requested
tolerance; the FP32 preconditioner changes only how fast it gets there.  Stated tolerance against the FP64
oracle: diff norms within 1e-6 relative at solve tolerance 1e-9."""
import math

import numpy as np
import pytest
import scipy.sparse as sp

pytestmark = pytest.mark.gpu

CASES = {
    "grid3d_logw": lambda ssp: ssp.gen_grid3d(16, 16, 16, -3, 3, 2),
    "er5k": lambda ssp: ssp.gen_er(5000, 20.0, 0.5, 2.0, 1),
    "rmat12": lambda ssp: ssp.gen_rmat(12, 16, 0.57, 0.19, 0.19, 3),
}


@pytest.mark.parametrize("name", list(CASES))
@pytest.mark.parametrize("max_degree", [0, -1])
def test_pc32_reaches_fp64_tolerance(ssp, ora, ctx, name, max_degree):
    G = CASES[name](ssp)
    v1, v2, w = ora.extract_edges(G.n, G.colptr, G.rowidx, G.values)
    cp, ri, va = ora.laplacian(G.n, v1, v2, w)
    lap = ssp.CSC(G.n, cp, ri, va)
    k = 37
    Y = ora.sketch(G.n, v1, v2, w, k, 1 / math.sqrt(k), 5)
    Zp, rp = ctx.solve_lap(lap, Y, tol=1e-9, abs_tol=0.0, max_iters=600, max_degree=max_degree,
                           precision=ssp.SSP_PRECISION_PC32)
    Zd, rd = ctx.solve_lap(lap, Y, tol=1e-9, abs_tol=0.0, max_iters=600, max_degree=max_degree, precision=0)
    assert rp["not_converged"] == 0 and rp["refinements"] == 0
    assert rp["max_relres"] <= 1e-9 * 1.0001
    # the FP32 preconditioner costs at most a few iterations
    assert rp["max_iters_used"] <= rd["max_iters_used"] + max(3, rd["max_iters_used"] // 4)
    Lg = sp.csc_matrix((va, ri, cp), shape=(G.n, G.n))
    b = Y - Y.mean(0)
    rel = np.linalg.norm(b - Lg @ Zp, axis=0) / np.linalg.norm(b, axis=0)
    assert rel.max() <= 1.01e-9
    F = ora.Factor(G.n, cp, ri, va, 0, 4096, rd["factor_max_degree_used"])
    Zo, it, _, rc = ora.pcg(G.n, cp, ri, va, F, Y, 1e-9, 0.0, 600)
    assert rc == 0
    dp, do = ora.diff_norms(v1, v2, Zp), ora.diff_norms(v1, v2, Zo)
    live = do > 1e-12 * do.max()
    assert np.max(np.abs(dp[live] - do[live]) / do[live]) < 1e-6


def test_pc32_sparsify_end_to_end(ssp, ctx):
    G = ssp.gen_grid3d(20, 20, 20, -3, 3, 2)
    prm = ssp.SparsifierParameters.baseline(0.5, pcg_tol=1e-8)
    H0, s0 = ctx.sparsify(G, prm)
    prm.precision = ssp.SSP_PRECISION_PC32
    H1, s1 = ctx.sparsify(G, prm)
    assert s1["pcg_max_relres"] <= 1e-8 * 1.0001 and s1["pcg_refinements"] == 0
    # probabilities move by about the solve tolerance: at most a handful of coin decisions can flip
    assert abs(s1["m_out"] - s0["m_out"]) <= 3 and 0 < s0["m_out"] < s0["m_in"]
    _, LG = ssp.stage_graph(ctx, G)
    r = ctx.probe_quadratic_form(LG, H1, 0.5, probes=100, seed=11)
    assert r["upper_bound_violations"] == 0 and r["lower_bound_violations"] == 0
