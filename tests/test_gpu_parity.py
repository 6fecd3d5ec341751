"""GPU parity: every stage of the CUDA path against the CPU oracle, through the C ABI.

Bit-exact: edges, L_G, sketch, factor (L, D, levels), diff norms given Z, probabilities, coins, keep set and
L_H given p and coins.  Tolerance: M^{-1} application (1e-12 relative) and PCG solutions (1e-7 relative on
edge differences at tol 1e-10; the residual itself must meet the requested tolerance).
"""
import math

import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.csgraph as csg

from conftest import rand_graph

pytestmark = pytest.mark.gpu


def _csc(ssp, A):
    return ssp.CSC.from_scipy(A)


GRAPHS = {
    "rand300": lambda ssp: _csc(ssp, rand_graph(300, 1500, 1)),
    "rand2k_disconnected": lambda ssp: _csc(ssp, rand_graph(2000, 2200, 2)),
    "grid40": lambda ssp: ssp.gen_grid2d(40, 40),
    "grid3d": lambda ssp: ssp.gen_grid3d(10, 9, 8, -3, 3, 2),
    "er5k": lambda ssp: ssp.gen_er(5000, 20.0, 0.5, 2.0, 1),
}


def _oracle_graph(ora, G):
    v1, v2, w = ora.extract_edges(G.n, G.colptr, G.rowidx, G.values)
    lg = ora.laplacian(G.n, v1, v2, w)
    return (v1, v2, w), lg


@pytest.mark.parametrize("name", list(GRAPHS))
def test_graph_assembly_bit_exact(ssp, ora, ctx, name):
    G = GRAPHS[name](ssp)
    (v1, v2, w), L = ssp.stage_graph(ctx, G)
    (o1, o2, ow), (cp, ri, va) = _oracle_graph(ora, G)
    assert np.array_equal(v1, o1) and np.array_equal(v2, o2) and np.array_equal(w, ow)
    assert np.array_equal(L.colptr, cp) and np.array_equal(L.rowidx, ri) and np.array_equal(L.values, va)


@pytest.mark.parametrize("k", [1, 7, 256, 300, 885])
@pytest.mark.parametrize("uniform", [False, True])
def test_sketch_bit_exact(ssp, ora, ctx, k, uniform):
    G = GRAPHS["rand300"](ssp)
    (v1, v2, w), _ = _oracle_graph(ora, G)
    scale = 1.0 / math.sqrt(k) if not uniform else math.sqrt(3.0)
    Y = ssp.stage_sketch(ctx, G.n, v1, v2, w, k, scale, 17, uniform)
    Yo = ora.sketch(G.n, v1, v2, w, k, scale, 17, uniform)
    assert np.array_equal(Y, Yo)


def _canon_cols(colptr, rows, vals, n):
    return [sorted(zip(rows[colptr[v]:colptr[v + 1]].tolist(), vals[colptr[v]:colptr[v + 1]].tolist()))
            for v in range(n)]


@pytest.mark.parametrize("name", ["rand300", "rand2k_disconnected", "grid40", "grid3d", "er5k"])
@pytest.mark.parametrize("dense,maxdeg", [(0, 0), (64, 0), (4096, 0), (4096, 12), (0, 30)])
def test_factor_bit_exact(ssp, ora, ctx, name, dense, maxdeg):
    G = GRAPHS[name](ssp)
    (v1, v2, w), (cp, ri, va) = _oracle_graph(ora, G)
    lap = ssp.CSC(G.n, cp, ri, va)
    seed = 5
    f = ssp.stage_factor(ctx, lap, seed, dense, maxdeg)
    o = ora.Factor(G.n, cp, ri, va, seed, dense, maxdeg)
    assert f["num_levels"] == o.num_levels
    assert np.array_equal(f["level"], o.level)
    assert np.array_equal(f["D"], o.D)
    assert _canon_cols(f["colptr"], f["rows"], f["vals"], G.n) == _canon_cols(o.colstart, o.rows, o.vals, G.n)


def test_factor_deterministic(ssp, ora, ctx):
    G = GRAPHS["er5k"](ssp)
    (_, _, _), (cp, ri, va) = _oracle_graph(ora, G)
    lap = ssp.CSC(G.n, cp, ri, va)
    a = ssp.stage_factor(ctx, lap, 9, 256, 40)
    b = ssp.stage_factor(ctx, lap, 9, 256, 40)
    for key in ("colptr", "D", "level"):
        assert np.array_equal(a[key], b[key])


@pytest.mark.parametrize("dense,maxdeg", [(0, 0), (128, 0), (4096, 8)])
def test_precond_matches_oracle(ssp, ora, ctx, dense, maxdeg):
    G = GRAPHS["grid3d"](ssp)
    (_, _, _), (cp, ri, va) = _oracle_graph(ora, G)
    lap = ssp.CSC(G.n, cp, ri, va)
    rng = np.random.default_rng(0)
    R = rng.standard_normal((G.n, 19))
    Z = ssp.stage_precond(ctx, lap, 3, R, dense, maxdeg)
    o = ora.Factor(G.n, cp, ri, va, 3, dense, maxdeg)
    Zo = np.column_stack([o.precond(R[:, j].copy()) for j in range(R.shape[1])])
    assert np.abs(Z - Zo).max() <= 1e-12 * np.abs(Zo).max()


@pytest.mark.parametrize("name,k,maxdeg", [("er5k", 70, 23), ("er5k", 5, 23), ("grid3d", 33, 8),
                                            ("rand2k_disconnected", 40, 6), ("er5k", 40, 0)])
def test_precond_last_level_finished_by_forward_solve(ssp, ora, ctx, monkeypatch, name, k, maxdeg):
    """The last level's rows are finished (z = y / D) by the forward solve and the backward launch of that
    level is skipped (k_fwd_last): the result equals the two separate launches bit for bit, and the oracle.
    Truncated factors end in a wide diagonal level of short rows (the case the kernel is for); complete
    elimination ends in a one-vertex level."""
    G = GRAPHS[name](ssp)
    (_, _, _), (cp, ri, va) = _oracle_graph(ora, G)
    lap = ssp.CSC(G.n, cp, ri, va)
    R = np.random.default_rng(k).standard_normal((G.n, k))
    monkeypatch.setenv("SSP_PRECOND_FUSE_LAST", "1")
    Zf = ssp.stage_precond(ctx, lap, 7, R, 4096, maxdeg)
    monkeypatch.setenv("SSP_PRECOND_FUSE_LAST", "0")
    Zs = ssp.stage_precond(ctx, lap, 7, R, 4096, maxdeg)
    np.testing.assert_array_equal(Zf.view(np.uint64), Zs.view(np.uint64))
    o = ora.Factor(G.n, cp, ri, va, 7, 4096, maxdeg)
    Zo = np.column_stack([o.precond(R[:, j].copy()) for j in range(k)])
    assert np.abs(Zf - Zo).max() <= 1e-12 * np.abs(Zo).max()


@pytest.mark.parametrize("k", [5, 40])
@pytest.mark.parametrize("dense", [0, 1024])
def test_precond_step_schedule_matches_oracle(ssp, ora, ctx, k, dense):
    """Thin-level runs solved by dependency steps: a 3-D grid's factor ends in hundreds of one-row levels (a
    one-vertex-per-level dense tail when dense > 0) that the schedule packs into far fewer steps, with rows
    split over warps; k = 5 takes the 8-column warp layout, k = 40 two tiles with padding columns."""
    G = ssp.gen_grid3d(16, 16, 16, -3, 3, 2)
    (_, _, _), (cp, ri, va) = _oracle_graph(ora, G)
    lap = ssp.CSC(G.n, cp, ri, va)
    R = np.random.default_rng(1).standard_normal((G.n, k))
    Z = ssp.stage_precond(ctx, lap, 5, R, dense, 0)
    o = ora.Factor(G.n, cp, ri, va, 5, dense, 0)
    assert o.num_levels > 100
    Zo = np.column_stack([o.precond(R[:, j].copy()) for j in range(k)])
    assert np.abs(Z - Zo).max() <= 1e-12 * np.abs(Zo).max()


@pytest.mark.parametrize("name", ["rand300", "grid40", "er5k"])
def test_pcg_matches_oracle(ssp, ora, ctx, name):
    G = GRAPHS[name](ssp)
    (v1, v2, w), (cp, ri, va) = _oracle_graph(ora, G)
    lap = ssp.CSC(G.n, cp, ri, va)
    k = 13
    Y = ora.sketch(G.n, v1, v2, w, k, 1 / math.sqrt(k), 3)
    Z, rep = ctx.solve_lap(lap, Y, tol=1e-10, abs_tol=0.0, max_iters=400, factor_seed=4, dense_threshold=256,
                           max_degree=16)
    F = ora.Factor(G.n, cp, ri, va, 4, 256, 16)
    Zo, it, rel, rc = ora.pcg(G.n, cp, ri, va, F, Y, 1e-10, 0.0, 400)
    assert rc == 0 and rep["not_converged"] == 0 and rep["max_relres"] < 1e-8
    dz, do = Z[v1] - Z[v2], Zo[v1] - Zo[v2]
    assert np.abs(dz - do).max() <= 1e-7 * np.abs(do).max()
    assert abs(rep["max_iters_used"] - it.max()) <= 2


MIXED_CASES = {
    "grid40": lambda ssp: ssp.gen_grid2d(40, 40),
    "er5k": lambda ssp: ssp.gen_er(5000, 20.0, 0.5, 2.0, 1),
    # weights spread over six decades: FP32 inner solves stop contracting and FP64 rounds take over
    "grid3d_logw": lambda ssp: ssp.gen_grid3d(16, 16, 16, -3, 3, 2),
}


@pytest.mark.parametrize("name", list(MIXED_CASES))
@pytest.mark.parametrize("max_degree", [0, -1])
def test_mixed_precision_reaches_fp64_tolerance(ssp, ora, ctx, name, max_degree):
    """SSP_PRECISION_MIXED: FP32 inner PCG inside FP64 refinement stops on the same FP64 residual test, so
    the solution matches the FP64 oracle's to the solve tolerance (stated: diff norms within 1e-6)."""
    G = MIXED_CASES[name](ssp)
    (v1, v2, w), (cp, ri, va) = _oracle_graph(ora, G)
    lap = ssp.CSC(G.n, cp, ri, va)
    k = 21
    Y = ora.sketch(G.n, v1, v2, w, k, 1 / math.sqrt(k), 5)
    Zm, rm = ctx.solve_lap(lap, Y, tol=1e-9, abs_tol=0.0, max_iters=600, max_degree=max_degree, precision=1)
    Zd, rd = ctx.solve_lap(lap, Y, tol=1e-9, abs_tol=0.0, max_iters=600, max_degree=max_degree, precision=0)
    assert rm["not_converged"] == 0 and rm["refinements"] >= 1 and rd["refinements"] == 0
    assert rm["max_relres"] <= 1e-9 * 1.0001 and rd["max_relres"] <= 1e-9 * 1.0001
    # the true residual of the mixed solution, computed here in FP64
    Lg = sp.csc_matrix((va, ri, cp), shape=(G.n, G.n))
    b = Y - Y.mean(0)
    rel = np.linalg.norm(b - Lg @ Zm, axis=0) / np.linalg.norm(b, axis=0)
    assert rel.max() <= 1.01e-9
    F = ora.Factor(G.n, cp, ri, va, 0, 4096, rd["factor_max_degree_used"])
    Zo, it, _, rc = ora.pcg(G.n, cp, ri, va, F, Y, 1e-9, 0.0, 600)
    assert rc == 0
    dm, do = ora.diff_norms(v1, v2, Zm), ora.diff_norms(v1, v2, Zo)
    live = do > 1e-12 * do.max()
    assert np.max(np.abs(dm[live] - do[live]) / do[live]) < 1e-6


def test_mixed_precision_sparsify_end_to_end(ssp, ctx):
    G = ssp.gen_er(4000, 80.0, 0.5, 2.0, 2)
    prm = ssp.SparsifierParameters.baseline(1.5, pcg_tol=1e-8)
    H0, s0 = ctx.sparsify(G, prm)
    prm.precision = ssp.SSP_PRECISION_MIXED
    H1, s1 = ctx.sparsify(G, prm)
    assert s1["pcg_refinements"] >= 1 and s0["pcg_refinements"] == 0
    assert s1["pcg_max_relres"] <= 1e-8 * 1.0001
    # probabilities move by ~1e-8 relative: at most a handful of coin decisions can flip
    assert abs(s1["m_out"] - s0["m_out"]) <= 3 and 0 < s0["m_out"] < s0["m_in"]


def test_run_solve_lap_dropin(ssp, ora, ctx):
    """ffi::run_solve_lap semantics (lib.rs:103, example.cc:668-703): FlattenedVec row-major n x k in and
    out, ||r||^2 <= 2e-7 stop, success iff relative residual < 0.01."""
    G = GRAPHS["grid40"](ssp)
    (v1, v2, w), (cp, ri, va) = _oracle_graph(ora, G)
    k = 24
    Y = ora.sketch(G.n, v1, v2, w, k, math.sqrt(3.0), 0)
    sol, nr, nc = ssp.run_solve_lap((Y.ravel(), G.n, k), cp.astype(np.int32), ri, va, "", G.n, False)
    assert (nr, nc) == (G.n, k)
    Z = sol.reshape(G.n, k)
    Lg = sp.csc_matrix((va, ri, cp), shape=(G.n, G.n))
    b = Y - Y.mean(0)
    res = np.linalg.norm(b - Lg @ Z, axis=0)
    assert (res <= math.sqrt(2e-7) * 1.0000001).all()
    assert (res / np.linalg.norm(b, axis=0) < 0.01).all()


def test_run_solve_lap_not_converged_is_an_error(ssp, ora):
    G = GRAPHS["grid3d"](ssp)
    (v1, v2, w), (cp, ri, va) = _oracle_graph(ora, G)
    lap = ssp.CSC(G.n, cp, ri, va)
    ctx2 = ssp.Context(0)
    Y = ora.sketch(G.n, v1, v2, w, 4, 1.0, 0)
    with pytest.raises(ssp.SspError) as e:
        ctx2.solve_lap(lap, Y, tol=1e-12, abs_tol=0.0, max_iters=1)
    assert e.value.code == -4
    ctx2.close()


def test_leverage_stages_bit_exact(ssp, ora, ctx):
    G = GRAPHS["er5k"](ssp)
    (v1, v2, w), _ = _oracle_graph(ora, G)
    rng = np.random.default_rng(3)
    Z = rng.standard_normal((G.n, 77))
    d = ssp.stage_diff_norms(ctx, v1, v2, Z)
    assert np.array_equal(d, ora.diff_norms(v1, v2, Z))
    p = ssp.stage_probs(ctx, w, d, 123.4, 77.0)
    assert np.array_equal(p, ora.probs(w, d, 123.4, 77.0))
    c = ssp.stage_coins(ctx, len(w), 99)
    assert np.array_equal(c, ora.coins(99, len(w)))


@pytest.mark.parametrize("reweight", [0, 1])
def test_sample_apply_bit_exact(ssp, ora, ctx, reweight):
    G = GRAPHS["grid3d"](ssp)
    (v1, v2, w), lg = _oracle_graph(ora, G)
    rng = np.random.default_rng(reweight)
    p = rng.uniform(0, 1, len(w))
    p[::7] = 1.0
    p[::11] = 0.0
    coins = ora.coins(5, len(w))
    H, keep = ssp.stage_sample_apply(ctx, G, p, coins, reweight)
    (hcp, hri, hva), okeep = ora.sample_apply(G.n, v1, v2, w, p, coins, reweight, lg)
    assert np.array_equal(keep, okeep)
    assert np.array_equal(H.colptr, hcp) and np.array_equal(H.rowidx, hri) and np.array_equal(H.values, hva)


def _oracle_pipeline(ora, ssp, G, params, max_degree):
    (v1, v2, w), (cp, ri, va) = _oracle_graph(ora, G)
    n = G.n
    k = params.jl_dim(n)
    s = params.jl_scale(k)
    Y = ora.sketch(n, v1, v2, w, k, s, params.sketch_seed, params.sketch_uniform)
    F = ora.Factor(n, cp, ri, va, params.factor_seed, params.dense_threshold, max_degree)
    Z, it, rel, rc = ora.pcg(n, cp, ri, va, F, Y, params.pcg_tol, params.pcg_abs_tol, params.pcg_max_iters)
    d = ora.diff_norms(v1, v2, Z)
    denom = k * s * s if params.prob_variance_correction else float(k)
    p = ora.probs(w, d, params.beta(n), denom)
    coins = ora.coins(params.sampling_seed, len(w))
    (hcp, hri, hva), keep = ora.sample_apply(n, v1, v2, w, p, coins, params.reweight, (cp, ri, va))
    return dict(k=k, Z=Z, d=d, p=p, keep=keep, H=(hcp, hri, hva), iters=it, v=(v1, v2, w), lg=(cp, ri, va))


def test_sparsify_config_grid2d_100(ssp, ora, ctx):
    """Configuration C1: 2-D 4-neighbour grid 100x100, unit weights, eps 0.5, k = ceil(24 ln n / eps^2) = 885
    columns of +-1/sqrt(k) Philox signs (seed 0), PCG tol 1e-8."""
    G = ssp.gen_grid2d(100, 100)
    prm = ssp.SparsifierParameters.baseline(0.5, pcg_tol=1e-8)
    H, st = ctx.sparsify(G, prm)
    assert st["k"] == 885 and st["m_in"] == 19_800
    o = _oracle_pipeline(ora, ssp, G, prm, st["factor_max_degree_used"])
    # leverage estimates agree to the solver tolerance; p equals wherever it is clipped at 1
    assert st["pcg_max_relres"] < 1e-7
    sp_run = ssp.Sparsifier(G, prm, ctx)
    sp_run.sparsify()
    Hm = sp_run.current_laplacian.to_scipy()
    Ho = sp.csc_matrix((o["H"][2], o["H"][1], o["H"][0]), shape=(G.n, G.n))
    assert (Hm != 0).nnz == (Ho != 0).nnz
    assert abs(Hm - Ho).max() <= 1e-12 * abs(Ho).max()
    assert st["m_out"] == int(o["keep"].sum())


def test_sparsify_config_rmat_small(ssp, ora, ctx):
    """The R-MAT configuration (power-law LCC, lognormal weights, eps 0.3) at scale 12: hubs of degree
    > 1000 take the long-row path of every gather kernel.  End to end against the oracle."""
    G = ssp.gen_rmat(12, 16, 0.57, 0.19, 0.19, 3)
    prm = ssp.SparsifierParameters.baseline(0.3, pcg_tol=1e-8)
    H, st = ctx.sparsify(G, prm)
    o = _oracle_pipeline(ora, ssp, G, prm, st["factor_max_degree_used"])
    assert st["pcg_max_relres"] < 1e-7 and st["m_in"] == len(o["keep"])
    assert st["m_out"] == int(o["keep"].sum()) and st["m_out"] < st["m_in"]
    Hm, Ho = H.to_scipy(), sp.csc_matrix((o["H"][2], o["H"][1], o["H"][0]), shape=(G.n, G.n))
    assert (Hm != 0).nnz == (Ho != 0).nnz and abs(Hm - Ho).max() <= 1e-12 * abs(Ho).max()


def test_spectral_check_dense_graph(ssp, ora, ctx):
    """A graph that actually gets sparsified: K_300 with eps = 0.7 and unbiased w/p reweighting.
    Every probe x^T L_H x / x^T L_G x and every eigenvalue of L_G^+ L_H must lie within 1 +- eps."""
    n = 300
    A = sp.csc_matrix(np.triu(np.ones((n, n)), 1))
    A = (A + A.T).tocsc()
    A.sort_indices()
    G = ssp.CSC.from_scipy(A)
    eps = 0.7
    prm = ssp.SparsifierParameters.baseline(eps, pcg_tol=1e-10)
    prm.reweight = ssp.SSP_REWEIGHT_INV_P
    H, st = ctx.sparsify(G, prm)
    assert st["m_out"] < 0.6 * st["m_in"]
    Lg = sp.diags(np.asarray(A.sum(0)).ravel()) - A
    Lh = H.to_scipy()
    rng = np.random.default_rng(0)
    for _ in range(100):
        x = rng.uniform(-1, 1, n)
        x -= x.mean()
        r = (x @ (Lh @ x)) / (x @ (Lg @ x))
        assert 1 - eps <= r <= 1 + eps
    Lgd, Lhd = Lg.toarray(), Lh.toarray()
    ev = np.linalg.eigvals(np.linalg.pinv(Lgd) @ Lhd).real
    ev = np.sort(ev)[1:]  # drop the shared nullspace
    assert ev.min() >= 1 - eps and ev.max() <= 1 + eps


def test_sparsify_deterministic(ssp, ctx):
    G = ssp.gen_er(20_000, 20.0, 0.5, 2.0, 7)
    prm = ssp.SparsifierParameters.baseline(0.5, pcg_tol=1e-6)
    H1, s1 = ctx.sparsify(G, prm)
    H2, s2 = ctx.sparsify(G, prm)
    assert np.array_equal(H1.colptr, H2.colptr) and np.array_equal(H1.values, H2.values)
    assert s1["pcg_mean_iters"] == s2["pcg_mean_iters"]


def test_invalid_inputs_rejected(ssp, ctx):
    A = rand_graph(100, 300, 4)
    bad = A.copy()
    bad.data = -bad.data
    with pytest.raises(ssp.SspError) as e:
        ctx.sparsify(ssp.CSC.from_scipy(bad), ssp.SparsifierParameters.cli(0.5))
    assert e.value.code == -1
    G = ssp.CSC.from_scipy(A)
    ri = G.rowidx.copy()
    s0, s1 = G.colptr[3], G.colptr[4]
    ri[s0], ri[s0 + 1] = ri[s0 + 1], ri[s0]
    with pytest.raises(ssp.SspError):
        ctx.sparsify(ssp.CSC(G.n, G.colptr, ri, G.values), ssp.SparsifierParameters.cli(0.5))
    # the context stays usable after a rejected call
    H, st = ctx.sparsify(G, ssp.SparsifierParameters.cli(0.5))
    assert st["m_in"] == G.nnz // 2


def test_sparsify_dataset_mtx(ssp, tmp_path):
    G = ssp.gen_grid2d(30, 30)
    src, dst = str(tmp_path / "in.mtx"), str(tmp_path / "out.mtx")
    ssp.write_mtx(src, G)
    st = ssp.sparsify_dataset(src, "grid", dst, 0.5, False, 0, 0, True)
    H = ssp.read_mtx(dst)
    assert st.original_num_edges == 2 * 30 * 29
    assert H.num_edges() == st.final_num_edges
    Lh = H.to_scipy()
    assert np.abs(np.asarray(Lh.sum(axis=0))).max() < 1e-9


@pytest.mark.parametrize("split", [(0, 16, 37), (0, 8, 37), (0, 37, 37)])
def test_column_split_phases_match_single_call(ssp, ora, ctx, split):
    """ssp_shard_leverage over two column shares + ssp_shard_finish on their summed squares equals
    ssp_sparsify up to the order of the final sum over columns; the autotuned factor is the same (the graph
    is large enough to be worth truncating)."""
    import torch
    G = ssp.gen_er(24000, 40.0, 0.5, 2.0, 9)
    prm = ssp.SparsifierParameters.baseline(1.5, pcg_tol=1e-10)
    prm.jl_dim_override = 37
    H1, st1 = ctx.sparsify(G, prm)
    m = ctx.num_edges(G)
    assert m == st1["m_in"]
    a, b, k = split
    dev = torch.device("cuda", 0)
    sq = torch.zeros((2, m), dtype=torch.float64, device=dev)
    torch.cuda.synchronize()
    sa = ctx.shard_leverage(G, prm, a, b, sq[0].data_ptr())
    degs = [sa["factor_max_degree_used"]]
    if b < k:
        sb = ctx.shard_leverage(G, prm, b, k, sq[1].data_ptr())
        degs.append(sb["factor_max_degree_used"])
    assert all(dg == st1["factor_max_degree_used"] for dg in degs) and st1["factor_max_degree_used"] > 0
    tot = (sq[0] + sq[1]).contiguous()
    torch.cuda.synchronize()
    H2, st2 = ctx.shard_finish(G, prm, tot.data_ptr())
    assert st2["m_out"] == st1["m_out"] and 0 < st1["m_out"] < m
    assert np.array_equal(H2.colptr, H1.colptr) and np.array_equal(H2.rowidx, H1.rowidx)
    np.testing.assert_allclose(H2.values, H1.values, rtol=1e-12, atol=1e-12)
    # the summed squares against the oracle's solve of all 37 columns with the same factor
    v1, v2, w = ora.extract_edges(G.n, G.colptr, G.rowidx, G.values)
    cp, ri, va = ora.laplacian(G.n, v1, v2, w)
    Y = ora.sketch(G.n, v1, v2, w, k, prm.jl_scale(k), prm.sketch_seed)
    F = ora.Factor(G.n, cp, ri, va, prm.factor_seed, prm.dense_threshold, st1["factor_max_degree_used"])
    Z, _, _, rc = ora.pcg(G.n, cp, ri, va, F, Y, prm.pcg_tol, prm.pcg_abs_tol, prm.pcg_max_iters)
    assert rc == 0
    np.testing.assert_allclose(tot.cpu().numpy(), ora.diff_norms(v1, v2, Z) ** 2, rtol=1e-7)


@pytest.mark.parametrize("n", [0, 1, 4095, 4096, 4097, 16_777_216, 16_777_217, 40_000_123])
def test_device_scan_every_depth(ssp, ctx, n):
    """The exclusive scan every stage builds its offsets with: one tile, several, and past 4096^2 elements,
    where an int32 scan recurses twice into the int64 one (each level with its own tile-sum buffer)."""
    a = np.random.default_rng(n).integers(0, 100, n, dtype=np.int32)
    out = ssp.stage_scan(ctx, a)
    ref = np.zeros(n + 1, np.int64)
    np.cumsum(a, dtype=np.int64, out=ref[1:])
    assert np.array_equal(out, ref)


@pytest.mark.parametrize("name", ["er5k", "grid3d", "rand2k_disconnected"])
def test_fused_diff_norms_equal_separate_pass(ssp, ctx, monkeypatch, name):
    """The solve's final product forms the edges' squared diff norms while it gathers x (per 32-column tile
    a butterfly, tiles added in order); the separate pass over the edges forms the same sums: the two
    sparsifiers must be identical bit for bit, for k in one tile (k = 13) and across several (baseline k)."""
    G = GRAPHS[name](ssp)
    for prm in (ssp.SparsifierParameters.cli(0.5), ssp.SparsifierParameters.baseline(1.0, pcg_tol=1e-8)):
        monkeypatch.setenv("SSP_DIFF_FUSED", "1")
        H1, s1 = ctx.sparsify(G, prm)
        monkeypatch.setenv("SSP_DIFF_FUSED", "0")
        H0, s0 = ctx.sparsify(G, prm)
        # (the residual products sum in different orders: relres agrees to rounding only)
        assert s1["m_out"] == s0["m_out"] and abs(s1["pcg_max_relres"] - s0["pcg_max_relres"]) <= 1e-6 * s0["pcg_max_relres"]
        assert np.array_equal(H1.colptr, H0.colptr) and np.array_equal(H1.rowidx, H0.rowidx)
        assert np.array_equal(H1.values.view(np.uint64), H0.values.view(np.uint64))


def test_large_host_buffers_match_device_buffers(ssp, ctx, tmp_path):
    """A graph whose value arrays exceed the staged-copy threshold (64 MB): host in / host out goes through the
    pinned ring and the pre-faulted result buffers, and must return exactly the device path's L_H (both
    written with the device writer, whose %.17g text round-trips every value)."""
    import ctypes
    import torch
    from spec_spars_b200 import _lib as L
    G = ssp.gen_er(1_000_000, 10.0, 0.5, 2.0, 4)
    assert G.values.nbytes > 64 << 20
    prm = ssp.SparsifierParameters.baseline(1.5, pcg_tol=1e-6)
    H, st = ctx.sparsify(G, prm)
    assert H.values.nbytes > 64 << 20
    dev = torch.device("cuda", 0)
    cp, ri, va = (torch.from_numpy(a).to(dev) for a in (G.colptr, G.rowidx, G.values))
    (nnz, dcp, dri, dva), st2 = ctx.sparsify_device(G.n, G.nnz, cp.data_ptr(), ri.data_ptr(), va.data_ptr(), prm)
    torch.cuda.synchronize()
    assert nnz == H.nnz and st["m_out"] == st2["m_out"]
    pd, ph = tmp_path / "dev.mtx", tmp_path / "host.mtx"
    s = L._Csc(G.n, nnz, dcp, dri, dva, L.SSP_MEM_DEVICE)
    L._check(L.lib().ssp_write_mtx_device(ctx._h, str(pd).encode(), ctypes.byref(s)))
    ctx.write_mtx(str(ph), H)
    assert ph.read_bytes() == pd.read_bytes()


@pytest.mark.parametrize("precision", [0, 1])
def test_column_batches_match_single_pass(ssp, ctx, monkeypatch, precision):
    """Columns solved in memory-sized batches (forced here to 64 columns: k = 205 in four batches, the last
    partial): the factor is built once and the squared diff norms accumulate tile by tile, so the sparsifier
    equals the single pass up to the solves' rounding (FP64: the same keep set, weights within 1e-9)."""
    G = GRAPHS["er5k"](ssp)
    prm = ssp.SparsifierParameters.baseline(1.0, pcg_tol=1e-9)
    prm.precision = precision
    monkeypatch.delenv("SSP_COLUMN_BATCH", raising=False)
    H1, s1 = ctx.sparsify(G, prm)
    monkeypatch.setenv("SSP_COLUMN_BATCH", "64")
    H4, s4 = ctx.sparsify(G, prm)
    assert s1["k"] == s4["k"] == 205 and s4["pcg_max_relres"] <= 1e-9 * 1.0001
    assert abs(s1["m_out"] - s4["m_out"]) <= (0 if precision == 0 else 3)
    if precision == 0:
        assert np.array_equal(H1.colptr, H4.colptr) and np.array_equal(H1.rowidx, H4.rowidx)
        np.testing.assert_allclose(H4.values, H1.values, rtol=1e-9, atol=0)
