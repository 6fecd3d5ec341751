"""One sparsification with its JL columns split across ranks, one GPU per rank (torch.distributed).

The k sketch columns are independent once the preconditioner exists.
* Every rank builds the same deterministic factor.
* Each rank sketches and solves a contiguous, tile-aligned share of the k global columns. Philox sketch
  entries depend only on the global column, so no sketch data is exchanged.
* Each rank leaves the per-edge partial sums of squared solution differences in an m-vector.
* The only exchange is one all-reduce(sum) of those m doubles over the process group.
* Every rank then derives the same probabilities, coins and L_H.

This replaces the reference's sequential per-column solve loop (example.cc:551-568) and its diff-norm pass
(sparsifier.rs:565-583) when the columns live on several GPUs.

The stage implementation is passed in. CudaStages runs on this rank's GPU through the C ABI, and is the
only one this package provides.
"""
import torch
import torch.distributed as dist

TILE = 32  # columns per PCG tile (SSP_TILE): shares are whole tiles so no rank pays for a partial tile twice


def column_range(k, world, rank, align=TILE):
    """Contiguous share [begin, end) of the k global columns for `rank`, in whole tiles, balanced to one
    tile.  Ranks beyond the tile count get an empty share."""
    if not (0 <= rank < world) or k < 0:
        raise ValueError("need 0 <= rank < world and k >= 0")
    tiles = (k + align - 1) // align
    per, extra = divmod(tiles, world)
    t0 = rank * per + min(rank, extra)
    t1 = t0 + per + (1 if rank < extra else 0)
    return min(t0 * align, k), min(t1 * align, k)


class CudaStages:
    """The two phases on this rank's GPU (ssp_shard_leverage / ssp_shard_finish).  The context runs on the
    current torch stream, so the all-reduce in between is stream-ordered with both phases."""

    def __init__(self, ctx, device):
        self.ctx = ctx
        self.device = torch.device("cuda", device)
        ctx.set_stream(torch.cuda.current_stream(self.device).cuda_stream)

    def num_edges(self, graph):
        return self.ctx.num_edges(graph)

    def zeros(self, m):
        return torch.zeros(max(m, 1), dtype=torch.float64, device=self.device)

    def leverage(self, graph, params, col_begin, col_end, sq):
        return self.ctx.shard_leverage(graph, params, col_begin, col_end, sq.data_ptr())

    def finish(self, graph, params, sq):
        return self.ctx.shard_finish(graph, params, sq.data_ptr())


def sparsify_sharded(graph, params, stages, group=None):
    """Sparsify `graph` with the JL columns split over the ranks of `group`; every rank returns the same
    L_H.  The stats are this rank's: stats["columns"] says which columns it solved."""
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    k = params.jl_dim(graph.n)
    c0, c1 = column_range(k, world, rank)
    m = stages.num_edges(graph)
    sq = stages.zeros(m)
    part = stages.leverage(graph, params, c0, c1, sq) if c1 > c0 else {}
    dist.all_reduce(sq, op=dist.ReduceOp.SUM, group=group)
    H, st = stages.finish(graph, params, sq)
    st = dict(st)
    for key in ("nnz_factor", "factor_levels", "pcg_max_iters_used", "pcg_mean_iters", "pcg_max_relres",
                "ms_factor", "ms_solve", "factor_max_degree_used"):
        if key in part:
            st[key] = part[key]
    st["columns"] = (c0, c1)
    st["k_local"] = c1 - c0
    return H, st
