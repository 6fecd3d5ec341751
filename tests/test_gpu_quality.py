"""a15 checks on the GPU against numpy/scipy: check_diagonal, quadratic forms, the probe experiment and
connected components (sparsifier.rs:806-826, experiments.rs:58-122)."""
import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.csgraph as csg

from conftest import rand_graph

pytestmark = pytest.mark.gpu


def _lap_of(ssp, ora, G):
    v1, v2, w = ora.extract_edges(G.n, G.colptr, G.rowidx, G.values)
    cp, ri, va = ora.laplacian(G.n, v1, v2, w)
    return ssp.CSC(G.n, cp, ri, va)


def test_check_laplacian(ssp, ora, ctx):
    L = _lap_of(ssp, ora, ssp.gen_er(3000, 12.0, 0.5, 2.0, 3))
    r = ctx.check_laplacian(L)
    A = L.to_scipy()
    assert r["ok"] and r["max_abs_colsum"] <= 1e-10 and r["bad_columns"] == 0
    assert abs(r["max_abs_colsum"] - np.abs(np.asarray(A.sum(axis=0))).max()) <= 1e-12
    # a changed diagonal breaks one column sum; a changed off-diagonal value breaks symmetry twice
    va = L.values.copy()
    d0 = L.colptr[5] + int(np.where(L.rowidx[L.colptr[5]:L.colptr[6]] == 5)[0][0])
    va[d0] += 1e-6
    o1 = L.colptr[7] + int(np.where(L.rowidx[L.colptr[7]:L.colptr[8]] != 7)[0][0])
    va[o1] *= 1.5
    r2 = ctx.check_laplacian(ssp.CSC(L.n, L.colptr, L.rowidx, va))
    assert r2["bad_columns"] == 2 and r2["asymmetric_entries"] == 2 and not r2["ok"]


def test_quadratic_forms_and_probes(ssp, ora, ctx):
    G = ssp.gen_er(5000, 30.0, 0.5, 2.0, 6)
    LG = _lap_of(ssp, ora, G)
    X = ctx.probe_vectors(G.n, 7, seed=11)
    # Philox layout: X[i, j] = 2 u53(philox((i, j), (seed, "PROB")) word 0) - 1
    for (i, j) in [(0, 0), (17, 3), (G.n - 1, 6)]:
        w = ora.philox4x64((i, j, 0, 0), 11, 0x50524F42)
        assert X[i, j] == 2.0 * ((int(w[0]) >> 11) * 2.0 ** -53) - 1.0
    assert np.all(np.abs(X) < 1.0) and abs(X.mean()) < 0.02
    A = LG.to_scipy()
    ref = np.einsum("ij,ij->j", X, A @ X)
    np.testing.assert_allclose(ctx.quadratic_forms(LG, X), ref, rtol=1e-12)
    prm = ssp.SparsifierParameters.baseline(0.5, pcg_tol=1e-8)
    prm.reweight = ssp.SSP_REWEIGHT_INV_P
    H, st = ctx.sparsify(G, prm)
    res = ctx.probe_quadratic_form(LG, H, 0.5, probes=50, seed=2)
    Xp = ctx.probe_vectors(G.n, 50, seed=2)
    qg = np.einsum("ij,ij->j", Xp, A @ Xp)
    qh = np.einsum("ij,ij->j", Xp, H.to_scipy() @ Xp)
    rel = np.abs(qh - qg) / np.abs(qg)
    assert res["probes"] == 50
    assert res["upper_bound_violations"] == int((qh >= 1.5 * qg).sum())
    assert res["lower_bound_violations"] == int((qh <= 0.5 * qg).sum())
    assert abs(res["mean_relative_error"] - rel.mean()) <= 1e-9 and abs(res["max_relative_error"] - rel.max()) <= 1e-9
    assert abs(res["std_dev_relative_error"] - rel.std()) <= 1e-9


@pytest.mark.parametrize("seed", [0, 1])
def test_connected_components(ssp, ctx, seed):
    A = rand_graph(4000, 2300, seed)  # sparse: many components
    G = ssp.CSC.from_scipy(A)
    cnt, labels = ctx.connected_components(G)
    nref, lref = csg.connected_components(A, directed=False)
    assert cnt == nref
    # same partition, each label the smallest vertex of its component
    for c in range(nref):
        members = np.where(lref == c)[0]
        assert np.all(labels[members] == members.min())
    H, st = ctx.sparsify(G, ssp.SparsifierParameters.cli(0.5))
    assert ctx.verify_ccs(G, H)
