"""A graph Laplacian as the sparsifier's input, as Sparsifier::from_matrix reads one (sparsifier.rs:299-300):
laplacian_to_graph must invert the oracle's Laplacian bit for bit (the off-diagonal negated, the diagonal
dropped, the stored order kept), and sparsify_laplacian must return exactly what sparsify returns on the
graph itself."""
import ctypes
import math

import numpy as np
import pytest


def _same(a, b):
    return (a.n == b.n and np.array_equal(a.colptr, b.colptr) and np.array_equal(a.rowidx, b.rowidx)
            and np.array_equal(a.values.view(np.uint64), b.values.view(np.uint64)))


def _laplacian_of(ssp, ora, G):
    v1, v2, w = ora.extract_edges(G.n, G.colptr, G.rowidx, G.values)
    return ssp.CSC(G.n, *ora.laplacian(G.n, v1, v2, w))


GRAPHS = {
    "er": lambda ssp: ssp.gen_er(5000, 12.0, 1e-3, 1e3, 3),
    "rmat": lambda ssp: ssp.gen_rmat(11, 16, 0.57, 0.19, 0.19, 4),  # hubs and isolated vertices
    "grid3d": lambda ssp: ssp.gen_grid3d(12, 10, 9, -3, 3, 5),
}
# the graphs the other GPU tests already sparsify with the CLI parameters
SPARSIFY = {
    "er5k": lambda ssp: ssp.gen_er(5000, 20.0, 0.5, 2.0, 1),
    "grid3d": lambda ssp: ssp.gen_grid3d(10, 9, 8, -3, 3, 2),
}


@pytest.mark.parametrize("name", list(GRAPHS))
def test_laplacian_to_graph_inverts_the_oracle_laplacian(ssp, ora, name):
    G = GRAPHS[name](ssp)
    L = _laplacian_of(ssp, ora, G)
    assert L.nnz > G.nnz
    assert _same(ssp.laplacian_to_graph(L), G)


def test_laplacian_to_graph_edge_cases(ssp):
    # no off-diagonal at all: an empty graph of the same order
    d = ssp.laplacian_to_graph(ssp.CSC(3, [0, 1, 2, 3], [0, 1, 2], [0.0, 0.0, 0.0]))
    assert d.n == 3 and d.nnz == 0 and list(d.colptr) == [0, 0, 0, 0]
    # a Laplacian with its diagonal left out converts the same way; a zero off-diagonal stays an entry
    L = ssp.CSC(3, [0, 2, 4, 6], [1, 2, 0, 2, 0, 1], [-2.0, 0.0, -2.0, -0.5, 0.0, -0.5])
    g = ssp.laplacian_to_graph(L)
    assert list(g.colptr) == [0, 2, 4, 6] and list(g.rowidx) == [1, 2, 0, 2, 0, 1]
    assert g.values.tolist() == [2.0, -0.0, 2.0, 0.5, -0.0, 0.5]


def test_laplacian_to_graph_rejects_bad_descriptors(ssp):
    import spec_spars_b200._lib as Lb
    ri, va = np.array([1, 0], np.int32), np.array([-1.0, -1.0])
    out = Lb._CscOut()
    for colptr, mem in (([0, 1, 3], Lb.SSP_MEM_HOST),   # does not end at nnz
                        ([1, 1, 2], Lb.SSP_MEM_HOST),   # does not start at 0
                        ([0, 5, 2], Lb.SSP_MEM_HOST),   # decreasing (a column past nnz)
                        ([0, 1, 2], Lb.SSP_MEM_DEVICE)):  # host only
        cp = np.array(colptr, np.int64)
        s = Lb._Csc(2, 2, cp.ctypes.data, ri.ctypes.data, va.ctypes.data, mem)
        assert Lb.lib().ssp_laplacian_to_graph(ctypes.byref(s), ctypes.byref(out)) == -1, colptr
        assert Lb.lib().ssp_last_error()


@pytest.mark.gpu
@pytest.mark.parametrize("name", list(SPARSIFY))
def test_sparsify_laplacian_equals_sparsify(ssp, ora, ctx, name):
    G = SPARSIFY[name](ssp)
    L = _laplacian_of(ssp, ora, G)
    prm = ssp.SparsifierParameters.cli(0.5)
    H, st = ctx.sparsify(G, prm)
    HL, stL = ctx.sparsify_laplacian(L, prm)
    assert _same(H, HL) and st["m_in"] == stL["m_in"] and st["m_out"] == stL["m_out"]


@pytest.mark.gpu
def test_sparsify_laplacian_from_device_memory(ssp, ora, ctx):
    import torch
    import spec_spars_b200._lib as Lb
    G = SPARSIFY["er5k"](ssp)
    L = _laplacian_of(ssp, ora, G)
    prm = ssp.SparsifierParameters.cli(0.5)
    H, _ = ctx.sparsify(G, prm)
    dev = torch.device("cuda", 0)
    cp, ri, va = (torch.from_numpy(a).to(dev) for a in (L.colptr, L.rowidx, L.values))
    torch.cuda.synchronize()
    s = Lb._Csc(L.n, L.nnz, cp.data_ptr(), ri.data_ptr(), va.data_ptr(), Lb.SSP_MEM_DEVICE)
    out, st = Lb._CscOut(), Lb._Stats()
    Lb._check(Lb.lib().ssp_sparsify_laplacian(ctx._h, ctypes.byref(s), ctypes.byref(prm._s), Lb.SSP_MEM_HOST,
                                              ctypes.byref(out), ctypes.byref(st)))
    assert _same(H, Lb._take_out(out))


def test_sparsifier_from_matrix(ssp, ora, tmp_path):
    """Sparsifier.from_matrix (sparsifier.rs:299-335): the Laplacian file becomes the current Laplacian as
    read_mtx gives it, nothing is pending, and its edges are the row < col entries in CSC order with values
    -w, the same edges in the same order as the graph's."""
    G = GRAPHS["er"](ssp)
    L = _laplacian_of(ssp, ora, G)
    path = tmp_path / "lap.mtx"
    ssp.write_mtx(str(path), L)
    prm = ssp.SparsifierParameters.new_default()
    sp = ssp.Sparsifier.from_matrix(str(path), prm)
    assert sp.num_nodes == G.n and _same(sp.current_laplacian, ssp.read_mtx(str(path)))
    v1, v2, w = ora.extract_edges(G.n, G.colptr, G.rowidx, G.values)
    r, c, val = sp.laplacian_edges()
    assert np.array_equal(r, v1) and np.array_equal(c, v2) and np.array_equal(-val, w)
    assert sp.num_edges() == len(w) and sp.graph.nnz == 0
    beta = prm.beta(G.n)
    assert sp.threshold == G.n * int(math.floor(beta + 0.5)) * prm.row_constant  # sparsifier.rs:264-266


@pytest.mark.gpu
def test_sparsifier_from_matrix_probabilities(ssp, ora, ctx, tmp_path):
    """compute_diff_norms / compute_probs on a loaded Laplacian (as tests.rs:747-764 uses them) equal the
    oracle's stages on the same edges, bit for bit."""
    G = GRAPHS["er"](ssp)
    L = _laplacian_of(ssp, ora, G)
    path = tmp_path / "lap.mtx"
    ssp.write_mtx(str(path), L)
    prm = ssp.SparsifierParameters.new_default()
    sp = ssp.Sparsifier.from_matrix(str(path), prm, ctx=ctx)
    X = np.random.default_rng(5).standard_normal((G.n, 21))
    d = sp.compute_diff_norms(X)
    v1, v2, w = ora.extract_edges(G.n, G.colptr, G.rowidx, G.values)
    assert np.array_equal(d, ora.diff_norms(v1, v2, X))
    p = sp.compute_probs(d)
    assert np.array_equal(p, ora.probs(w, d, prm.beta(G.n), float(prm.jl_dim(G.n))))
    assert np.all((p >= 0) & (p <= 1))


@pytest.mark.gpu
def test_sparsify_laplacian_rejects_bad_colptr_on_the_device(ssp, ctx):
    """The Laplacian's graph is formed on the device; column pointers that decrease, or that do not start at
    0 and end at nnz, are rejected there with the host conversion's messages."""
    import spec_spars_b200._lib as Lb
    prm = ssp.SparsifierParameters.cli(0.5)
    ri = np.array([0, 1, 0, 1, 2, 1, 2], np.int32)
    va = np.array([1.0, -1.0, -1.0, 2.0, -1.0, -1.0, 1.0])
    for colptr, msg in (([0, 2, 1, 7], b"non-decreasing"), ([0, 2, 5, 6], b"start at 0 and end at nnz")):
        cp = np.array(colptr, np.int64)
        s = Lb._Csc(3, 7, cp.ctypes.data, ri.ctypes.data, va.ctypes.data, Lb.SSP_MEM_HOST)
        out, st = Lb._CscOut(), Lb._Stats()
        rc = Lb.lib().ssp_sparsify_laplacian(ctx._h, ctypes.byref(s), ctypes.byref(prm._s), Lb.SSP_MEM_HOST,
                                             ctypes.byref(out), ctypes.byref(st))
        assert rc != 0 and msg in Lb.lib().ssp_last_error(), colptr
    # a valid path graph 0 - 1 - 2 goes through
    cp = np.array([0, 2, 5, 7], np.int64)
    s = Lb._Csc(3, 7, cp.ctypes.data, ri.ctypes.data, va.ctypes.data, Lb.SSP_MEM_HOST)
    out, st = Lb._CscOut(), Lb._Stats()
    Lb._check(Lb.lib().ssp_sparsify_laplacian(ctx._h, ctypes.byref(s), ctypes.byref(prm._s), Lb.SSP_MEM_HOST,
                                              ctypes.byref(out), ctypes.byref(st)))
    assert st.m_in == 2
