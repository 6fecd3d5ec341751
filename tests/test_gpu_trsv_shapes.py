"""Launch shapes of the preconditioner's level solves, chosen by measurement.

A level launch gives each warp row 8, 16 or 32 columns.  Every width forms each (row, column) sum the same way
-- rows longer than one chunk included, whose entries go to a fixed set of accumulators combined by a fixed
tree -- so M^{-1} r is the same bit for bit whatever the widths, and the autotuner's choice changes only the
time.  The measured shapes are cached per factor shape in the context; a sparsification with measured shapes
equals the one with the fixed rule bit for bit.  The preconditioner's algebra is custom_cg.hpp:224-235's.
"""
import numpy as np
import pytest

from conftest import rand_graph

pytestmark = pytest.mark.gpu

GRAPHS = {
    # average degree 300: the early levels' columns of L hold hundreds of entries (more than one chunk)
    "er_dense": lambda ssp: ssp.CSC.from_scipy(rand_graph(3000, 450_000, 5)),
    # power-law hubs: rows and columns of thousands of entries
    "rmat12": lambda ssp: ssp.gen_rmat(12, 16, 0.57, 0.19, 0.19, 3),
    "grid3d": lambda ssp: ssp.gen_grid3d(12, 11, 10, -3, 3, 2),
    "er5k": lambda ssp: ssp.gen_er(5000, 20.0, 0.5, 2.0, 1),
}


def _laplacian(ssp, ctx, G):
    _, L = ssp.stage_graph(ctx, G)
    return L


@pytest.mark.parametrize("name,maxdeg", [("er_dense", 0), ("er_dense", 350), ("rmat12", 0), ("rmat12", 40),
                                         ("grid3d", 0), ("er5k", 23)])
def test_every_width_gives_the_same_bits(ssp, ctx, monkeypatch, name, maxdeg):
    G = GRAPHS[name](ssp)
    L = _laplacian(ssp, ctx, G)
    R = np.random.default_rng(3).standard_normal((G.n, 40))
    monkeypatch.setenv("SSP_TRSV_TUNE", "0")
    rule = ssp.stage_precond(ctx, L, 7, R, 4096, maxdeg)
    monkeypatch.delenv("SSP_TRSV_TUNE")
    outs = {}
    for w in ("8", "16", "32"):
        monkeypatch.setenv("SSP_TRSV_WIDTH", w)
        outs[w] = ssp.stage_precond(ctx, L, 7, R, 4096, maxdeg)
    monkeypatch.delenv("SSP_TRSV_WIDTH")
    # measured shapes (the stage entry measures from any size here)
    monkeypatch.setenv("SSP_TRSV_TUNE_MIN", "0")
    outs["measured"] = ssp.stage_precond(ctx, L, 7, R, 4096, maxdeg)
    assert np.isfinite(rule).all()
    for w, Z in outs.items():
        np.testing.assert_array_equal(Z.view(np.uint64), rule.view(np.uint64), err_msg=f"width {w}")


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_sparsify_with_measured_shapes_equals_rule(ssp, monkeypatch, precision):
    """First call measures (SSP_TRSV_TUNED, device time reported), the second takes the context's cached
    shapes (SSP_TRSV_CACHED), and the fixed rule (SSP_TRSV_TUNE=0) gives the same L_H bit for bit."""
    G = ssp.gen_er(20000, 20.0, 0.5, 2.0, 4)
    prm = ssp.SparsifierParameters.baseline(0.5, pcg_tol=1e-8)
    if precision == "mixed":
        prm.precision = ssp.SSP_PRECISION_MIXED
    c = ssp.Context(0)
    try:
        monkeypatch.setenv("SSP_TRSV_TUNE_MIN", "0")
        H1, s1 = c.sparsify(G, prm)
        H2, s2 = c.sparsify(G, prm)
        monkeypatch.setenv("SSP_TRSV_TUNE", "0")
        H3, s3 = c.sparsify(G, prm)
    finally:
        c.close()
    assert s1["trsv_shapes"] == ssp.SSP_TRSV_TUNED and s1["ms_trsv_tune"] > 0
    assert s2["trsv_shapes"] == ssp.SSP_TRSV_CACHED and s2["ms_trsv_tune"] == 0
    assert s3["trsv_shapes"] == ssp.SSP_TRSV_RULE
    nlev = s1["trsv_levels_w8"] + s1["trsv_levels_w16"] + s1["trsv_levels_w32"]
    assert nlev > 0 and nlev == s3["trsv_levels_w8"] + s3["trsv_levels_w16"] + s3["trsv_levels_w32"]
    assert (s1["trsv_levels_w8"], s1["trsv_levels_w16"], s1["trsv_levels_w32"]) == \
        (s2["trsv_levels_w8"], s2["trsv_levels_w16"], s2["trsv_levels_w32"])
    for H in (H2, H3):
        np.testing.assert_array_equal(H.colptr, H1.colptr)
        np.testing.assert_array_equal(H.rowidx, H1.rowidx)
        np.testing.assert_array_equal(H.values.view(np.uint64), H1.values.view(np.uint64))
    assert s1["pcg_max_iters_used"] == s3["pcg_max_iters_used"]
