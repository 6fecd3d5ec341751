"""ssp_stage_leverage_probs_static: the allocation-free leverage stage, called through the C ABI with device
buffers, against the context-based entry points (ssp_stage_diff_norms + ssp_stage_probs) on two calls in a
row.  Both paths use the same per-edge arithmetic in the same order, so the probabilities must agree bit for
bit.  The file sorts last so that it also runs after every other GPU test in one session."""
import ctypes

import numpy as np
import pytest


def _edges(ssp, ctx, G):
    (v1, v2, w), _ = ssp.stage_graph(ctx, G)
    return v1, v2, w


def _static_probs(ssp, torch, stream, n, v1, v2, Z, w, beta, denom, check_free=False):
    dev = torch.device("cuda", 0)
    tv1 = torch.from_numpy(v1).to(dev)
    tv2 = torch.from_numpy(v2).to(dev)
    tZ = torch.from_numpy(np.ascontiguousarray(Z)).to(dev)
    tw = torch.from_numpy(w).to(dev)
    tp = torch.full((len(w),), -7.0, dtype=torch.float64, device=dev)
    torch.cuda.synchronize()
    free_before = torch.cuda.mem_get_info(0)[0]
    rc = ssp.lib().ssp_stage_leverage_probs_static(stream, n, len(w), tv1.data_ptr(), tv2.data_ptr(), tZ.data_ptr(),
                                                    Z.shape[1], tw.data_ptr(), beta, denom, tp.data_ptr())
    assert rc == 0, ssp.lib().ssp_last_error()
    torch.cuda.synchronize()
    if check_free:
        assert torch.cuda.mem_get_info(0)[0] == free_before
    return tp.cpu().numpy()


def test_static_rejects_oversize_before_launch(ssp):
    L = ssp.lib()
    cap = 1 << 20
    buf = (ctypes.c_double * 4)()
    ib = (ctypes.c_int32 * 4)()
    rc = L.ssp_stage_leverage_probs_static(None, 10, cap + 1, ctypes.addressof(ib), ctypes.addressof(ib),
                                           ctypes.addressof(buf), 1, ctypes.addressof(buf), 1.0, 1.0,
                                           ctypes.addressof(buf))
    assert rc == -5
    assert b"exceeds the static scratch capacity" in L.ssp_last_error()
    assert L.ssp_stage_leverage_probs_static(None, 10, 3, None, None, None, 0, None, 1.0, 1.0, None) == -1
    assert L.ssp_stage_leverage_probs_static(None, 10, 0, None, None, None, 4, None, 1.0, 1.0, None) == 0


@pytest.mark.gpu
def test_static_matches_context_entry_points_twice(ssp, ctx):
    import torch
    stream = torch.cuda.current_stream(0).cuda_stream
    cases = [(ssp.gen_er(40_000, 20.0, 0.5, 2.0, 5), 61, 123.4, 77.0),
             (ssp.gen_grid3d(30, 20, 25, -3, 3, 7), 130, 9.5, 130.0)]
    prepared = []
    for G, k, beta, denom in cases:
        v1, v2, w = _edges(ssp, ctx, G)
        Z = np.random.default_rng(k).standard_normal((G.n, k))
        ref = ssp.stage_probs(ctx, w, ssp.stage_diff_norms(ctx, v1, v2, Z), beta, denom)
        prepared.append((G.n, v1, v2, Z, w, beta, denom, ref))
    # the first call per device loads the device code and looks the scratch up (start-up); the two calls
    # after it must not change free device memory
    _static_probs(ssp, torch, stream, *prepared[0][:7])
    outs = [(_static_probs(ssp, torch, stream, *c[:7], check_free=True), c[7]) for c in prepared]
    for got, ref in outs:
        assert got.shape == ref.shape and np.all((got >= 0) & (got <= 1))
        np.testing.assert_array_equal(got.view(np.uint64), ref.view(np.uint64))


@pytest.mark.gpu
def test_static_out_of_range_endpoint_gets_probability_one(ssp, ctx):
    """An edge whose endpoint lies outside [0, n) is not read: it gets p = 1, the others are unchanged; the
    context entry point gives NaN for it from device input and rejects it from host input."""
    import torch
    stream = torch.cuda.current_stream(0).cuda_stream
    G = ssp.gen_grid2d(30, 30)
    v1, v2, w = _edges(ssp, ctx, G)
    k = 40
    Z = np.random.default_rng(3).standard_normal((G.n, k))
    beta, denom = 0.5, 40.0
    ref = ssp.stage_probs(ctx, w, ssp.stage_diff_norms(ctx, v1, v2, Z), beta, denom)
    bad = v2.copy()
    bad[17] = G.n
    got = _static_probs(ssp, torch, stream, G.n, v1, bad, Z, w, beta, denom)
    assert got[17] == 1.0
    keep = np.arange(len(w)) != 17
    np.testing.assert_array_equal(got[keep].view(np.uint64), ref[keep].view(np.uint64))
    with pytest.raises(ssp.SspError, match="outside"):
        ssp.stage_diff_norms(ctx, v1, bad, Z)
    dev = torch.device("cuda", 0)
    td = torch.full((len(w),), -1.0, dtype=torch.float64, device=dev)
    tv1, tbad = torch.from_numpy(v1).to(dev), torch.from_numpy(bad).to(dev)
    tZ = torch.from_numpy(Z).to(dev)
    torch.cuda.synchronize()
    rc = ssp.lib().ssp_stage_diff_norms(ctx._h, G.n, len(w), tv1.data_ptr(), tbad.data_ptr(), tZ.data_ptr(), k,
                                        1, td.data_ptr())
    assert rc == 0, ssp.lib().ssp_last_error()
    d = td.cpu().numpy()
    assert np.isnan(d[17]) and not np.isnan(d[keep]).any()
