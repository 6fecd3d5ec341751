"""Every output H passes the spectral check (1 +- eps).

The checks follow the reference's probe_quadratic_form (experiments.rs:88-122) and compute_quadratic_form
(sparsifier.rs:820-826): x^T L_H x against x^T L_G x on 100 seeded uniform(-1, 1) probes, which must give no
violation of (1 - eps) x^T L_G x < x^T L_H x < (1 + eps) x^T L_G x.  On graphs of at most 4000 vertices the
extremal eigenvalues of the pencil (L_H, L_G) on the complement of the constant vector -- the exact spectral
bound that the probes sample -- are found by Lanczos (scipy eigsh) and must lie in [1 - eps, 1 + eps].

The graphs have the shapes of the benchmark configurations, at sizes a test runs in seconds: a dense ER graph
that the sampler thins to about 60% of its edges at eps = 0.5, 3-D grids whose weights span six decades
(eps 0.5), R-MAT (eps 0.3) and random geometric graphs (eps 0.3).  Sparsification runs on the GPU through
the C ABI with the benchmark parameters (k = ceil(24 ln n / eps^2), w/p reweighting); the checks run on the
host in FP64.
"""
import numpy as np
import pytest
import scipy.linalg as sl
import scipy.sparse as sp
import scipy.sparse.linalg as sla

pytestmark = pytest.mark.gpu

# name: (generator, eps, largest kept fraction expected (None: no claim), Lanczos check)
CASES = {
    "er_n2000_deg400": (lambda S: S.gen_er(2000, 400.0, 0.5, 2.0, 7), 0.5, 0.75, True),
    "grid3d_15_logw": (lambda S: S.gen_grid3d(15, 15, 15, -3.0, 3.0, 2), 0.5, 0.9, True),
    "rmat_s12": (lambda S: S.gen_rmat(12, 16, 0.57, 0.19, 0.19, 3), 0.3, None, True),
    "rgg_n3000_deg32": (lambda S: S.gen_rgg(3000, 32.0, 0.1, 10.0, 5), 0.3, None, True),
    "grid3d_32_logw": (lambda S: S.gen_grid3d(32, 32, 32, -3.0, 3.0, 2), 0.5, 0.9, False),
    "rmat_s14": (lambda S: S.gen_rmat(14, 16, 0.57, 0.19, 0.19, 3), 0.3, None, False),
    "rgg_n50k_deg16": (lambda S: S.gen_rgg(50_000, 16.0, 0.1, 10.0, 9), 0.5, None, False),
    "er_n20k_deg200": (lambda S: S.gen_er(20_000, 200.0, 0.5, 2.0, 4), 0.5, None, False),
}


def pencil_extremes(LG, LH):
    """Smallest and largest eigenvalue of L_H y = lam L_G y for y orthogonal to the constant vector (G
    connected), by Lanczos on C^-1 L_H C^-T with C C^T = L_G + 11^T / n: that shift maps the constant vector
    to eigenvalue 0 and leaves the pencil's other eigenvalues unchanged."""
    n = LG.shape[0]
    C = np.linalg.cholesky(LG.toarray() + np.full((n, n), 1.0 / n))

    def mv(x):
        y = sl.solve_triangular(C, x, lower=True, trans="T")
        return sl.solve_triangular(C, LH @ y, lower=True)

    op = sla.LinearOperator((n, n), matvec=mv, dtype=np.float64)
    hi = sla.eigsh(op, k=1, which="LA", tol=1e-8, return_eigenvectors=False)[0]
    lo = np.sort(sla.eigsh(op, k=2, which="SA", tol=1e-8, return_eigenvectors=False))
    assert abs(lo[0]) < 1e-8  # the constant vector
    return float(lo[1]), float(hi)


@pytest.mark.parametrize("name", list(CASES))
def test_sparsifier_passes_spectral_check(ssp, ctx, name):
    gen, eps, kept_max, lanczos = CASES[name]
    G = gen(ssp)
    prm = ssp.SparsifierParameters.baseline(eps, pcg_tol=1e-8)
    assert prm.reweight == ssp.SSP_REWEIGHT_INV_P
    H, st = ctx.sparsify(G, prm)
    _, LG = ssp.stage_graph(ctx, G)
    kept = st["m_out"] / st["m_in"]
    if kept_max is not None:
        assert kept < kept_max, f"{name}: kept {kept:.3f}, expected real sparsification"
    assert ctx.check_laplacian(H)["ok"]
    assert ctx.verify_ccs(G, H)
    r = ctx.probe_quadratic_form(LG, H, eps, probes=100, seed=11)
    assert r["probes"] == 100
    assert r["upper_bound_violations"] == 0 and r["lower_bound_violations"] == 0, r
    assert r["max_relative_error"] < eps
    if lanczos:
        assert G.n <= 4000
        lo, hi = pencil_extremes(LG.to_scipy(), H.to_scipy())
        assert 1 - eps <= lo <= hi <= 1 + eps, (name, kept, lo, hi)


def test_reference_reweight_is_biased_low(ssp, ctx):
    """The reference's w/sqrt(p) (sparsifier.rs:657) on the dense ER graph: the same kept edges, but the
    pencil's spectrum shifts down (every kept edge with p < 1 weighs w/sqrt(p) < w/p), which is why the
    benchmark configurations reweight by w/p."""
    G = CASES["er_n2000_deg400"][0](ssp)
    prm = ssp.SparsifierParameters.baseline(0.5, pcg_tol=1e-8)
    Hp, _ = ctx.sparsify(G, prm)
    prm.reweight = ssp.SSP_REWEIGHT_INV_SQRT_P
    Hs, _ = ctx.sparsify(G, prm)
    _, LG = ssp.stage_graph(ctx, G)
    assert np.array_equal(Hp.colptr, Hs.colptr) and np.array_equal(Hp.rowidx, Hs.rowidx)
    lo_p, hi_p = pencil_extremes(LG.to_scipy(), Hp.to_scipy())
    lo_s, hi_s = pencil_extremes(LG.to_scipy(), Hs.to_scipy())
    assert hi_s < hi_p and lo_s < lo_p and hi_s < 1.0 < hi_p
