"""The column-split sparsification (spec_spars_b200/sharded.py) on CPU ranks over gloo.

The stages here are the oracle's, not the GPU's: this covers the host logic of the multi-GPU path (the
column shares, the all-reduce of per-edge partial squares, the replicated finish) with world_size 2 and 3.
The GPU phases themselves are covered by tests/test_gpu_parity.py through the C ABI.
"""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


class OracleStages:
    """Both phases computed by the CPU oracle (test-only stand-in for CudaStages)."""

    def __init__(self, ora):
        self.ora = ora

    def _prep(self, graph, params):
        ora = self.ora
        v1, v2, w = ora.extract_edges(graph.n, graph.colptr, graph.rowidx, graph.values)
        lg = ora.laplacian(graph.n, v1, v2, w)
        k = params.jl_dim(graph.n)
        return v1, v2, w, lg, k, params.jl_scale(k)

    def num_edges(self, graph):
        return len(self.ora.extract_edges(graph.n, graph.colptr, graph.rowidx, graph.values)[0])

    def zeros(self, m):
        return torch.zeros(max(m, 1), dtype=torch.float64)

    def leverage(self, graph, params, c0, c1, sq):
        ora = self.ora
        v1, v2, w, (cp, ri, va), k, scale = self._prep(graph, params)
        Y = ora.sketch(graph.n, v1, v2, w, k, scale, params.sketch_seed, bool(params.sketch_uniform))[:, c0:c1]
        F = ora.Factor(graph.n, cp, ri, va, params.factor_seed, params.dense_threshold, params.factor_max_degree)
        Z, _, _, rc = ora.pcg(graph.n, cp, ri, va, F, Y, params.pcg_tol, params.pcg_abs_tol, params.pcg_max_iters)
        assert rc == 0
        d = Z[v1] - Z[v2]
        sq[:len(v1)] = torch.from_numpy((d * d).sum(axis=1))
        return {"pcg_max_iters_used": 0}

    def finish(self, graph, params, sq):
        ora = self.ora
        v1, v2, w, lg, k, scale = self._prep(graph, params)
        d = np.sqrt(sq[:len(v1)].numpy())
        denom = k * scale * scale if params.prob_variance_correction else float(k)
        p = ora.probs(w, d, params.beta(graph.n), denom)
        H, keep = ora.sample_apply(graph.n, v1, v2, w, p, ora.coins(params.sampling_seed, len(v1)),
                                   params.reweight, lg)
        return (H, keep, p), {}


def _params(ssp):
    prm = ssp.SparsifierParameters.baseline(1.5, pcg_tol=1e-10)  # large eps: some edges are dropped
    prm.jl_dim_override = 37  # not a multiple of the column tile: the last share is ragged
    prm.factor_max_degree = 0
    prm.dense_threshold = 64
    return prm


def _graph(ssp):
    return ssp.gen_er(600, 40.0, 0.5, 2.0, 4)


def _worker(rank, world, port, outdir):
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    sys.path.insert(0, os.path.join(root, "oracle"))
    import pyoracle as ora
    import spec_spars_b200 as ssp
    from spec_spars_b200.sharded import sparsify_sharded
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        (H, keep, p), st = sparsify_sharded(_graph(ssp), _params(ssp), OracleStages(ora))
        np.savez(os.path.join(outdir, f"r{rank}.npz"), cp=H[0], ri=H[1], va=H[2], keep=keep, p=p,
                 c0=st["columns"][0], c1=st["columns"][1])
    finally:
        dist.destroy_process_group()


def test_column_range_partitions_k():
    from spec_spars_b200.sharded import column_range, TILE
    for k in (1, 7, 8, 37, 885, 1327):
        for world in (1, 2, 3, 8, 200):
            shares = [column_range(k, world, r) for r in range(world)]
            assert shares[0][0] == 0 and shares[-1][1] == k
            for (a0, a1), (b0, b1) in zip(shares, shares[1:]):
                assert a1 == b0 and a0 <= a1
            tiles = [(b - a + TILE - 1) // TILE for a, b in shares]
            assert all(a % TILE == 0 for a, b in shares if b > a)
            assert max(tiles) - min(tiles) <= 1
    with pytest.raises(ValueError):
        column_range(10, 2, 2)


@pytest.mark.parametrize("world", [2, 3])
def test_sharded_matches_single_rank(ssp, ora, tmp_path, world):
    port = _free_port()
    mp.start_processes(_worker, args=(world, port, str(tmp_path)), nprocs=world, join=True, start_method="spawn")
    outs = [np.load(tmp_path / f"r{r}.npz") for r in range(world)]
    # shares cover the 37 columns once, and every rank ends with the same L_H
    assert int(outs[0]["c0"]) == 0 and int(outs[-1]["c1"]) == 37
    for o in outs[1:]:
        for key in ("cp", "ri", "va", "keep", "p"):
            assert np.array_equal(o[key], outs[0][key])
    # against the whole computation on one rank (diff_norms over all 37 columns at once)
    G, prm = _graph(ssp), _params(ssp)
    v1, v2, w = ora.extract_edges(G.n, G.colptr, G.rowidx, G.values)
    cp, ri, va = ora.laplacian(G.n, v1, v2, w)
    k = prm.jl_dim(G.n)
    Y = ora.sketch(G.n, v1, v2, w, k, prm.jl_scale(k), prm.sketch_seed)
    F = ora.Factor(G.n, cp, ri, va, prm.factor_seed, prm.dense_threshold, 0)
    Z, _, _, rc = ora.pcg(G.n, cp, ri, va, F, Y, prm.pcg_tol, prm.pcg_abs_tol, prm.pcg_max_iters)
    p = ora.probs(w, ora.diff_norms(v1, v2, Z), prm.beta(G.n), k * prm.jl_scale(k) ** 2)
    np.testing.assert_allclose(outs[0]["p"], p, rtol=1e-12, atol=0)
    _, keep = ora.sample_apply(G.n, v1, v2, w, p, ora.coins(prm.sampling_seed, len(v1)), prm.reweight,
                               (cp, ri, va))
    assert np.array_equal(outs[0]["keep"], keep)
    assert 0 < keep.sum() < len(keep)
