"""Streaming resparsification (ssp_sparsify_update; Sparsifier::insert + sparsify, sparsifier.rs:357-376,
693-709,735-790): the current L_H plus newly inserted edges, sketched over the new edges only, solved and
sampled over all of them -- against the oracle restatement of the same steps."""
import numpy as np
import pytest
import scipy.sparse as sp

pytestmark = pytest.mark.gpu


def _empty(ssp, n):
    return ssp.CSC(n, np.zeros(n + 1, np.int64), np.zeros(0, np.int32), np.zeros(0, np.float64))


def _same(a, b):
    return (np.array_equal(a.colptr, b.colptr) and np.array_equal(a.rowidx, b.rowidx)
            and np.array_equal(a.values, b.values))


def test_update_from_empty_equals_sparsify(ssp, ctx):
    G = ssp.gen_er(3000, 40.0, 0.5, 2.0, 5)
    prm = ssp.SparsifierParameters.baseline(1.5, pcg_tol=1e-8)
    H0, s0 = ctx.sparsify(G, prm)
    H1, s1 = ctx.sparsify_update(_empty(ssp, G.n), G, prm)
    assert _same(H0, H1) and s0["m_out"] == s1["m_out"] and 0 < s0["m_out"] < s0["m_in"]


@pytest.mark.parametrize("uniform", [0, 1])
def test_second_batch_matches_oracle(ssp, ora, ctx, uniform):
    n = 2500
    A = ssp.gen_er(n, 30.0, 0.5, 2.0, 1)
    B = ssp.gen_er(n, 10.0, 0.5, 2.0, 2)  # overlaps some pairs of A: their weights add
    prm = ssp.SparsifierParameters.baseline(1.5, pcg_tol=1e-10)
    prm.sketch_uniform = uniform
    H1, s1 = ctx.sparsify(A, prm)
    H2, s2 = ctx.sparsify_update(H1, B, prm)
    # oracle: the merged graph is -offdiag(H1) + B; the sketch uses B's edges alone
    L1 = H1.to_scipy()
    M = (-(L1 - sp.diags(L1.diagonal())) + B.to_scipy()).tocsc()
    M.eliminate_zeros()
    M.sort_indices()
    v1, v2, w = ora.extract_edges(n, M.indptr, M.indices, M.data)
    cp, ri, va = ora.laplacian(n, v1, v2, w)
    b1, b2, bw = ora.extract_edges(n, B.colptr, B.rowidx, B.values)
    k = prm.jl_dim(n)
    sc = prm.jl_scale(k)
    Y = ora.sketch(n, b1, b2, bw, k, sc, prm.sketch_seed, bool(uniform))
    F = ora.Factor(n, cp, ri, va, prm.factor_seed, prm.dense_threshold, s2["factor_max_degree_used"])
    Z, _, _, rc = ora.pcg(n, cp, ri, va, F, Y, prm.pcg_tol, prm.pcg_abs_tol, prm.pcg_max_iters)
    assert rc == 0
    p = ora.probs(w, ora.diff_norms(v1, v2, Z), prm.beta(n), k * sc * sc)
    (hcp, hri, hva), keep = ora.sample_apply(n, v1, v2, w, p, ora.coins(prm.sampling_seed, len(w)), prm.reweight,
                                             (cp, ri, va))
    assert s2["m_in"] == len(w) and s2["m_out"] == int(keep.sum()) and 0 < keep.sum() < len(w)
    assert np.array_equal(H2.colptr, hcp) and np.array_equal(H2.rowidx, hri)
    np.testing.assert_allclose(H2.values, hva, rtol=1e-12, atol=1e-12)


def test_sparsifier_insert_and_streaming_trigger(ssp, ctx):
    n = 1500
    G = ssp.gen_er(n, 60.0, 0.5, 2.0, 3)
    extra = ssp.gen_er(n, 6.0, 0.5, 2.0, 4).to_scipy().tocoo()
    prm = ssp.SparsifierParameters.baseline(1.5, pcg_tol=1e-8)
    prm.row_constant = 1
    s = ssp.Sparsifier(n, prm, ctx)
    A = G.to_scipy().tocoo()
    for a, b, x in zip(A.row, A.col, A.data):
        if a < b:
            s.insert(int(a), int(b), float(x))
    s.insert(0, 0, 3.0)  # self-loops and zero values are skipped
    s.insert(1, 2, 0.0)
    st1 = s.sparsify()
    H_direct, _ = ctx.sparsify(G, prm)
    assert _same(s.current_laplacian, H_direct)
    # without streaming, inserts only queue
    first = [(int(a), int(b), float(x)) for a, b, x in zip(extra.row, extra.col, extra.data) if a < b]
    s.insert(*first[0])
    assert _same(s.current_laplacian, H_direct)
    # threshold = n * round(beta) * row_constant (sparsifier.rs:266), round half away from zero
    assert s.threshold == n * int(np.floor(prm.beta(n) + 0.5)) * prm.row_constant
    # with streaming, the reference's trigger compares the current Laplacian's edges with the threshold
    s.params.streaming = 1
    s.threshold = s.num_edges() + 1
    s.insert(*first[1])  # not above the threshold: queued
    assert _same(s.current_laplacian, H_direct)
    s.threshold = s.num_edges() - 1
    s.insert(*first[2])  # above it: sparsifies the three queued edges into the current Laplacian
    assert not _same(s.current_laplacian, H_direct) and s.graph.nnz == 0
    assert st1.final_num_edges == H_direct.num_edges()
