"""C ABI checks that need no GPU: the library loads, exports every symbol the header declares, derived
parameters follow the reference formulas, host-side I/O and generators, and device entry points fail
cleanly (status code, message) when no device is visible."""
import math
import os

import numpy as np
import pytest
import scipy.sparse as sp


def test_library_exports_header_symbols(ssp):
    L = ssp.lib()
    assert len(ssp.HEADER_SYMBOLS) >= 30
    missing = [s for s in ssp.HEADER_SYMBOLS if not hasattr(L, s)]
    assert missing == []


def test_params_presets(ssp):
    d = ssp.SparsifierParameters.new_default()  # sparsifier.rs:182-209
    assert (d.epsilon, d.beta_constant, d.row_constant, d.jl_factor) == (0.5, 4, 2, 1.5)
    assert d.jl_scaling_factor == math.sqrt(3.0) and d.sketch_seed == 1 and d.sampling_seed == 1
    assert d.sketch_uniform == 1 and d.streaming == 0
    c = ssp.SparsifierParameters.cli(0.3, False, 7, 9)  # lib.rs:149-156
    assert (c.jl_factor, c.beta_constant, c.row_constant, c.sketch_uniform) == (4.0, 4, 2, 0)
    assert (c.sketch_seed, c.sampling_seed) == (7, 9)
    assert c.pcg_max_iters == 400 and c.pcg_abs_tol == math.sqrt(2e-7)


@pytest.mark.parametrize("n", [100, 10_000, 1_000_000, 4_194_304])
def test_derived_parameters(ssp, n):
    c = ssp.SparsifierParameters.cli(0.5)
    # sparsifier.rs:264 beta = eps^-2 * beta_constant * ln(n); :272 k = ceil(log2(n) * jl_factor)
    assert c.beta(n) == math.pow(0.5, -2.0) * 4 * math.log(n)
    assert c.jl_dim(n) == math.ceil(math.log2(n) * 4.0)
    b = ssp.SparsifierParameters.baseline(0.5)
    assert b.jl_dim(n) == math.ceil(24 * math.log(n) / 0.25)
    k = b.jl_dim(n)
    assert b.jl_scale(k) == 1.0 / math.sqrt(k)


def test_baseline_k_values(ssp):
    b5 = ssp.SparsifierParameters.baseline(0.5)
    b3 = ssp.SparsifierParameters.baseline(0.3)
    assert b5.jl_dim(10_000) == 885 and b5.jl_dim(1_000_000) == 1327 and b5.jl_dim(2_097_152) == 1398
    assert b3.jl_dim(4_194_304) == 4067


def test_generators(ssp):
    g = ssp.gen_grid2d(100, 100)
    assert g.n == 10_000 and g.nnz == 2 * 19_800
    A = g.to_scipy()
    assert abs(A - A.T).max() == 0
    g3 = ssp.gen_grid3d(8, 8, 8, -3, 3, 2)
    assert g3.n == 512 and g3.nnz == 2 * 3 * 8 * 8 * 7
    w = g3.values
    assert w.min() >= 1e-3 and w.max() <= 1e3
    er = ssp.gen_er(20_000, 20.0, 0.5, 2.0, 1)
    m = er.nnz // 2
    assert abs(m - 200_000) < 5 * math.sqrt(200_000)
    assert (er.values >= 0.5).all() and (er.values <= 2.0).all()
    assert np.array_equal(er.values.astype(np.float32).astype(np.float64), er.values)
    er2 = ssp.gen_er(20_000, 20.0, 0.5, 2.0, 1)
    assert np.array_equal(er.rowidx, er2.rowidx) and np.array_equal(er.values, er2.values)


def test_mtx_roundtrip(ssp, tmp_path):
    g = ssp.gen_grid3d(5, 4, 3, -1, 1, 3)
    p = str(tmp_path / "g.mtx")
    ssp.write_mtx(p, g)
    h = ssp.read_mtx(p)
    assert np.array_equal(g.colptr, h.colptr) and np.array_equal(g.rowidx, h.rowidx)
    assert np.array_equal(g.values, h.values)


def test_mtx_symmetric_and_pattern(ssp, tmp_path):
    p = tmp_path / "s.mtx"
    p.write_text("%%MatrixMarket matrix coordinate real symmetric\n% c\n3 3 3\n2 1 1.5\n3 2 2.5\n1 1 4\n")
    h = ssp.read_mtx(str(p))
    A = h.to_scipy().toarray()
    assert np.array_equal(A, np.array([[4, 1.5, 0], [1.5, 0, 2.5], [0, 2.5, 0]]))
    q = tmp_path / "p.mtx"
    q.write_text("%%MatrixMarket matrix coordinate pattern general\n2 2 2\n1 2\n2 1\n")
    hp = ssp.read_mtx(str(q))
    assert np.array_equal(hp.to_scipy().toarray(), np.array([[0, 1.0], [1.0, 0]]))
    r = tmp_path / "d.mtx"
    r.write_text("%%MatrixMarket matrix coordinate real general\n2 2 2\n1 2 1\n1 2 2\n")
    assert ssp.read_mtx(str(r)).to_scipy().toarray()[0, 1] == 3.0  # duplicates summed


def test_mtx_errors(ssp, tmp_path):
    with pytest.raises(ssp.SspError) as e:
        ssp.read_mtx(str(tmp_path / "missing.mtx"))
    assert e.value.code == -6
    p = tmp_path / "rect.mtx"
    p.write_text("%%MatrixMarket matrix coordinate real general\n2 3 1\n1 1 1\n")
    with pytest.raises(ssp.SspError):
        ssp.read_mtx(str(p))


def test_no_device_is_a_clean_error(ssp):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a device is visible")
    with pytest.raises(ssp.SspError) as e:
        ssp.Context(0)
    assert e.value.code == -7 and "no CUDA device" in str(e.value)
    with pytest.raises(ssp.SspError):
        ssp.run_solve_lap((np.zeros(4), 2, 2), [0, 1, 2], [0, 1], [1.0, 1.0], "", 2, False)


def test_missing_library_fails_loudly(monkeypatch, tmp_path):
    import spec_spars_b200._lib as L
    monkeypatch.setattr(L, "LIB_PATH", str(tmp_path / "nope.so"))
    monkeypatch.setattr(L, "_LIB", None)
    with pytest.raises(L.SspError):
        L.lib()


def test_server_api_without_device(ssp):
    """The serving entry points load and fail cleanly on a machine without a GPU; the footprint estimate
    grows with the problem."""
    G = ssp.gen_rgg(3000, 12.0, 0.1, 10.0, 5)
    assert abs(G.nnz / G.n - 12.0) < 2.0
    small = ssp.request_footprint(G, ssp.SparsifierParameters.baseline(0.5))
    tight = ssp.request_footprint(G, ssp.SparsifierParameters.baseline(0.3))
    mixed = ssp.SparsifierParameters.baseline(0.5)
    mixed.precision = ssp.SSP_PRECISION_MIXED
    assert 0 < small < tight and ssp.request_footprint(G, mixed) > small
    try:
        import torch
        has_gpu = torch.cuda.is_available()
    except Exception:
        has_gpu = False
    if not has_gpu:
        with pytest.raises(ssp.SspError) as e:
            ssp.Server(0, slots=2)
        assert e.value.code == -7


def test_edge_list_to_matrix_market(ssp, tmp_path):
    """edge_list_to_matrix_market (utils.rs:413-526): header line, optional weights, (min, max) pairs,
    first weight of a repeated pair wins, sorted output, weights printed as Rust displays an f64."""
    src = tmp_path / "g.txt"
    lines = ["6 9", "0 1 2.5", "1 0 7.0", "", "3 2", "2 4 0.0025", "5 5 1e-10", "4 2 9", "1 3 12345678.5",
             "0 5 0.1"]
    src.write_text("\n".join(lines) + "\n")
    dst = tmp_path / "g.mtx"
    ssp.edge_list_to_matrix_market(src, dst, 1.5)
    first = {}
    for ln in lines[1:]:
        if not ln.strip():
            continue
        t = ln.split()
        u, v = int(t[0]), int(t[1])
        w = float(t[2]) if len(t) > 2 else 1.5
        first.setdefault((min(u, v), max(u, v)), w)
    expect = ["%%MatrixMarket matrix coordinate real symmetric", f"% Converted from {src}", f"6 6 {len(first)}"]
    expect += [f"{i} {j} {np.format_float_positional(w, trim='-')}" for (i, j), w in sorted(first.items())]
    assert dst.read_text().splitlines() == expect
    assert "0 1 2.5" in expect and "5 5 0.0000000001" in expect and "2 3 1.5" in expect
    with pytest.raises(ssp.SspError) as e:
        ssp.edge_list_to_matrix_market(tmp_path / "missing.txt", dst, 1.0)
    assert e.value.code == -6


def test_rmat_generator(ssp):
    """R-MAT (the scale-22 configuration, run small): symmetric, one connected component (the LCC),
    FP32-rounded lognormal weights, deterministic for a seed."""
    import scipy.sparse.csgraph as csg
    g = ssp.gen_rmat(11, 16, 0.57, 0.19, 0.19, 3)
    A = g.to_scipy()
    assert abs(A - A.T).max() == 0 and A.diagonal().max() == 0
    assert csg.connected_components(A, directed=False)[0] == 1
    assert np.all(g.values == g.values.astype(np.float32).astype(np.float64)) and g.values.min() > 0
    assert np.diff(g.colptr).max() > 20 * np.diff(g.colptr).mean()  # skewed degrees
    h = ssp.gen_rmat(11, 16, 0.57, 0.19, 0.19, 3)
    assert np.array_equal(g.rowidx, h.rowidx) and np.array_equal(g.values, h.values)
