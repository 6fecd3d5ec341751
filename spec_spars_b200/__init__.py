"""spec_spars_b200: B200-native spectral sparsification (JL sketch -> approximate Cholesky PCG ->
leverage-score sampling), driven through the C ABI in include/specspars.h.

The Python layer mirrors the reference crate's entry points (tenchd/spec_spars):
  SparsifierParameters.new / new_default / cli   <- src/sparsifier.rs:163-209, src/lib.rs:149-156
  Sparsifier(graph, params).sparsify()           <- src/sparsifier.rs:722-770
  InputStream(path).run_stream(params, ...)      <- src/stream.rs:18-64
  sparsify_dataset(...)                          <- src/lib.rs:145-166
  run_solve_lap(...)                             <- src/lib.rs:103 (cxx bridge)
All numerical work happens in libspecspars.so on the GPU; importing works without a GPU, and the
first call that needs one raises SspError if no device is visible.
"""
from ._lib import (  # noqa: F401
    SspError, lib, Context, CSC, DeviceCSC, SparsifierParameters, Sparsifier, InputStream, SparsificationStats,
    sparsify_dataset, run_solve_lap, solve_lap, read_mtx, write_mtx, laplacian_to_graph, parse_decimal, format_g17, gen_grid2d, gen_grid3d, gen_er, gen_rgg, gen_rmat,
    Server, request_footprint, edge_list_to_matrix_market, format_shortest,
    stage_graph, stage_sketch, stage_factor, stage_precond, stage_diff_norms, stage_probs, stage_coins, stage_scan,
    stage_sample_apply, SSP_JL_DIM_REF, SSP_JL_DIM_24, SSP_JL_SCALE_FIXED, SSP_JL_SCALE_INV_SQRT_K,
    SSP_REWEIGHT_INV_SQRT_P, SSP_REWEIGHT_INV_P, SSP_PRECISION_FP64, SSP_PRECISION_MIXED, SSP_PRECISION_PC32, LIB_PATH, HEADER_SYMBOLS,
    SSP_TRSV_RULE, SSP_TRSV_TUNED, SSP_TRSV_CACHED, SSP_TRSV_FORCED,
)
