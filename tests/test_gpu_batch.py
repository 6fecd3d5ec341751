"""Several graphs sparsified as one disjoint union (ssp_sparsify_batch) and served in batches.

Each graph of a batch keeps its own parameters (epsilon, seeds, JL rule and scale) and every PCG scalar is
per (graph, column), so its result must equal the same graph sparsified alone: the same kept edges and L_H
values within 1e-8 relative (the lone and the batched solve differ only in how their dot products are
blocked, and both run to relative residual 1e-8).  Iteration counts may differ by one where a column's
residual lands within rounding of its threshold."""
import threading

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

RTOL = 1e-8


def _prm(ssp, eps, seed, mixed=False, max_degree=24):
    p = ssp.SparsifierParameters.baseline(eps, pcg_tol=1e-8, sampling_seed=seed, sketch_seed=seed + 7)
    p.dense_threshold = 0           # no dense tail: a batch eliminates in the sparse phase
    p.factor_max_degree = max_degree  # a fixed truncation, applied graph by graph (0: complete elimination)
    if mixed:
        p.precision = ssp.SSP_PRECISION_MIXED
    return p


def _graphs(ssp):
    return [ssp.gen_grid2d(30, 31), ssp.gen_er(3000, 12.0, 0.1, 10.0, 3), ssp.gen_rgg(2000, 16.0, 0.1, 10.0, 5),
            ssp.gen_grid3d(12, 11, 10, -3.0, 3.0, 2), ssp.gen_rmat(10, 16, 0.57, 0.19, 0.19, 3),
            ssp.gen_er(800, 200.0, 0.5, 2.0, 9)]


def _close(H, H0):
    assert H.n == H0.n
    assert np.array_equal(H.colptr, H0.colptr) and np.array_equal(H.rowidx, H0.rowidx)
    np.testing.assert_allclose(H.values, H0.values, rtol=RTOL, atol=0)


@pytest.mark.parametrize("max_degree", [24, 0, 6, -1])
def test_batch_equals_each_graph_alone(ssp, ctx, max_degree):
    """Truncated at average live degree 24 (graphs stop at different levels), 6 (early), eliminated completely
    (0), or each graph's own autotuned choice (-1: the probe runs graph by graph inside the batch)."""
    graphs = _graphs(ssp)
    params = [_prm(ssp, [0.5, 0.3][i % 2], i, max_degree=max_degree) for i in range(len(graphs))]
    got = ctx.sparsify_batch(graphs, params)
    assert len(got) == len(graphs)
    for G, prm, (H, st) in zip(graphs, params, got):
        H0, st0 = ctx.sparsify(G, prm)
        _close(H, H0)
        assert st["n"] == G.n and st["m_in"] == st0["m_in"] and st["m_out"] == st0["m_out"]
        assert st["k"] == st0["k"]
        assert abs(st["pcg_max_iters_used"] - st0["pcg_max_iters_used"]) <= 1
        assert st["factor_max_degree_used"] == st0["factor_max_degree_used"]
        if max_degree >= 0:
            assert st["factor_max_degree_used"] == max_degree
        assert st["pcg_max_relres"] < 1e-7


def test_mixed_precision_batch_meets_the_tolerance(ssp, ctx):
    """FP32 inner solves in FP64 refinement over a batch: when to fall back to FP64 inner solves is decided for
    the batch as a whole, so a graph's iterates can follow another path than alone; both stop at relative
    residual 1e-8, so the kept counts agree to 0.5% and every result passes the (1 +- eps) probes."""
    graphs = _graphs(ssp)
    params = [_prm(ssp, [0.5, 0.3][i % 2], i, mixed=True) for i in range(len(graphs))]
    got = ctx.sparsify_batch(graphs, params)
    for G, prm, (H, st) in zip(graphs, params, got):
        _, st0 = ctx.sparsify(G, prm)
        assert st["m_in"] == st0["m_in"] and abs(st["m_out"] - st0["m_out"]) <= 0.005 * st0["m_out"] + 1
        assert st["pcg_max_relres"] < 1e-7
        _, LG = ssp.stage_graph(ctx, G)
        r = ctx.probe_quadratic_form(LG, H, prm.epsilon, probes=50, seed=3)
        assert r["upper_bound_violations"] == 0 and r["lower_bound_violations"] == 0


def test_batch_of_one_and_a_dense_graph_really_sparsifies(ssp, ctx):
    G = ssp.gen_er(2000, 400.0, 0.5, 2.0, 7)
    prm = _prm(ssp, 0.5, 4)
    (H, st), = ctx.sparsify_batch([G], prm)
    H0, st0 = ctx.sparsify(G, prm)
    _close(H, H0)
    assert st["m_out"] < 0.8 * st["m_in"]


def test_batch_rejects_mixed_options(ssp, ctx):
    a, b = ssp.gen_grid2d(10, 10), ssp.gen_grid2d(12, 12)
    p, q = _prm(ssp, 0.5, 1), _prm(ssp, 0.5, 2)
    q.factor_seed = 99
    with pytest.raises(ssp.SspError, match="must agree"):
        ctx.sparsify_batch([a, b], [p, q])
    r = _prm(ssp, 0.5, 3)
    r.dense_threshold = 4096
    with pytest.raises(ssp.SspError, match="sparse-phase elimination"):
        ctx.sparsify_batch([a], [r])


def test_served_batches_equal_lone_calls(ssp, ctx):
    """Requests submitted from several threads are batched by the server (ssp_result.batch > 1 for some), and
    each result equals the lone call within the stated tolerance; a request that asks for the autotuned factor
    runs alone and is bit-identical."""
    graphs = _graphs(ssp) * 2
    params = [_prm(ssp, 0.5 if i % 3 else 0.3, i, max_degree=-1 if i % 2 else 24) for i in range(len(graphs))]
    lone_G, lone_p = ssp.gen_er(2500, 10.0, 0.1, 10.0, 77), ssp.SparsifierParameters.baseline(0.5, pcg_tol=1e-8)
    alone = [ctx.sparsify(G, p) for G, p in zip(graphs, params)]
    alone_auto = ctx.sparsify(lone_G, lone_p)
    tickets = [None] * len(graphs)
    with ssp.Server(0, slots=2, max_batch=8) as srv:
        def submit(idx):
            for i in idx:
                tickets[i] = srv.submit(graphs[i], params[i])
        th = [threading.Thread(target=submit, args=(range(t, len(graphs), 2),)) for t in range(2)]
        for t in th:
            t.start()
        t_auto = srv.submit(lone_G, lone_p)
        for t in th:
            t.join()
        results = [srv.wait(t) for t in tickets]
        H_auto, st_auto, tm_auto = srv.wait(t_auto)
        info = srv.info()
    assert info["completed"] == len(graphs) + 1 and info["failed"] == 0
    assert info["peak_batch"] > 1 and info["batches"] < len(graphs) + 1
    assert any(tm["batch"] > 1 for _, _, tm in results)
    for (H, st, tm), (H0, st0) in zip(results, alone):
        _close(H, H0)
        assert st["m_out"] == st0["m_out"]
    assert tm_auto["batch"] == 1
    H0, _ = alone_auto
    assert np.array_equal(H_auto.values, H0.values) and np.array_equal(H_auto.rowidx, H0.rowidx)
