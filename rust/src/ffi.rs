//! The C ABI of libspecspars.so (include/specspars.h), declared for Rust.
//!
//! Every struct is `#[repr(C)]` with the header's fields in the header's order and types, one field per
//! line; tests/test_rust_ffi_layout.py parses these declarations and checks every offset and size against
//! the header as a C compiler lays it out.  Every function returns an `int` status (SSP_OK = 0) unless
//! noted; `ssp_last_error` gives the calling thread's last message.

use std::os::raw::{c_char, c_int, c_void};

pub const SSP_OK: c_int = 0;
pub const SSP_ERR_INVALID: c_int = -1;
pub const SSP_ERR_CUDA: c_int = -2;
pub const SSP_ERR_NOMEM: c_int = -3;
pub const SSP_ERR_NOT_CONVERGED: c_int = -4;
pub const SSP_ERR_CAPACITY: c_int = -5;
pub const SSP_ERR_IO: c_int = -6;
pub const SSP_ERR_NO_DEVICE: c_int = -7;
pub const SSP_ERR_PENDING: c_int = -8;

pub const SSP_MEM_HOST: i32 = 0;
pub const SSP_MEM_DEVICE: i32 = 1;
pub const SSP_JL_DIM_REF: i32 = 0;
pub const SSP_JL_DIM_24: i32 = 1;
pub const SSP_JL_SCALE_FIXED: i32 = 0;
pub const SSP_JL_SCALE_INV_SQRT_K: i32 = 1;
pub const SSP_PRECISION_FP64: i32 = 0;
pub const SSP_PRECISION_MIXED: i32 = 1;
pub const SSP_PRECISION_PC32: i32 = 2;
pub const SSP_REWEIGHT_INV_SQRT_P: i32 = 0;
pub const SSP_REWEIGHT_INV_P: i32 = 1;
pub const SSP_TRSV_RULE: i32 = 0;
pub const SSP_TRSV_TUNED: i32 = 1;
pub const SSP_TRSV_CACHED: i32 = 2;
pub const SSP_TRSV_FORCED: i32 = 3;
pub const SSP_REQ_SPARSIFY: i32 = 0;

/// ssp_csc: a square matrix in compressed-sparse-column form (CSC == CSR for the symmetric matrices here).
#[repr(C)]
#[derive(Clone, Copy, Debug)]
pub struct SspCsc {
    pub n: i64,
    pub nnz: i64,
    pub colptr: *const i64,
    pub rowidx: *const i32,
    pub values: *const f64,
    pub mem: i32,
}

/// ssp_csc_out: a library-allocated CSC result, released with ssp_csc_free.
#[repr(C)]
#[derive(Debug)]
pub struct SspCscOut {
    pub n: i64,
    pub nnz: i64,
    pub colptr: *mut i64,
    pub rowidx: *mut i32,
    pub values: *mut f64,
    pub mem: i32,
    pub owned_by_context: i32,
}

/// ssp_params: SparsifierParameters (sparsifier.rs:146-159) plus this library's options.
#[repr(C)]
#[derive(Clone, Copy, Debug)]
pub struct SspParams {
    pub epsilon: f64,
    pub beta_constant: i32,
    pub row_constant: i32,
    pub verbose: i32,
    pub jl_factor: f64,
    pub jl_scaling_factor: f64,
    pub sketch_seed: u64,
    pub sampling_seed: u64,
    pub bench: i32,
    pub sketch_uniform: i32,
    pub streaming: i32,
    pub output_file: *const c_char,
    pub jl_dim_rule: i32,
    pub jl_scale_rule: i32,
    pub prob_variance_correction: i32,
    pub reweight: i32,
    pub pcg_tol: f64,
    pub pcg_abs_tol: f64,
    pub pcg_max_iters: i32,
    pub factor_seed: u64,
    pub dense_threshold: i64,
    pub factor_max_degree: i64,
    pub jl_dim_override: i32,
    pub precision: i32,
}

/// ssp_stats: what one sparsification did (SparsificationStats and the Benchmarker phases).
#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct SspStats {
    pub n: i64,
    pub m_in: i64,
    pub m_out: i64,
    pub k: i32,
    pub beta: f64,
    pub nnz_factor: i64,
    pub factor_levels: i32,
    pub pcg_max_iters_used: i32,
    pub pcg_mean_iters: f64,
    pub pcg_max_relres: f64,
    pub ms_assembly: f64,
    pub ms_sketch: f64,
    pub ms_factor: f64,
    pub ms_solve: f64,
    pub ms_leverage: f64,
    pub ms_sample: f64,
    pub ms_total: f64,
    pub kernels_launched: i64,
    pub ms_spmm: f64,
    pub n_spmm: i64,
    pub ms_precond: f64,
    pub n_precond: i64,
    pub nnz_laplacian: i64,
    pub factor_max_degree_used: i64,
    pub ms_autotune: f64,
    pub pcg_refinements: i32,
    pub pcg_fp64_rounds: i32,
    pub spmm_slabs: i32,
    pub trsv_shapes: i32,
    pub trsv_levels_w8: i32,
    pub trsv_levels_w16: i32,
    pub trsv_levels_w32: i32,
    pub ms_trsv_tune: f64,
}

/// ssp_solve_opts: options of ssp_solve_lap.
#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct SspSolveOpts {
    pub tol: f64,
    pub abs_tol: f64,
    pub max_iters: i32,
    pub factor_seed: u64,
    pub dense_threshold: i64,
    pub verbose: i32,
    pub factor_max_degree: i64,
    pub precision: i32,
}

/// ssp_solve_report: what ssp_solve_lap did.
#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct SspSolveReport {
    pub k: i32,
    pub max_iters_used: i32,
    pub mean_iters: f64,
    pub max_relres: f64,
    pub not_converged: i32,
    pub nnz_factor: i64,
    pub factor_levels: i32,
    pub ms_factor: f64,
    pub ms_solve: f64,
    pub factor_max_degree_used: i64,
    pub refinements: i32,
    pub fp64_rounds: i32,
    pub spmm_slabs: i32,
    pub trsv_shapes: i32,
    pub trsv_levels_w8: i32,
    pub trsv_levels_w16: i32,
    pub trsv_levels_w32: i32,
    pub ms_trsv_tune: f64,
}

/// ssp_server_opts: the persistent request loop's device, slots, HBM budget and queue limit.
#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct SspServerOpts {
    pub device: i32,
    pub slots: i32,
    pub hbm_budget_bytes: i64,
    pub max_pending: i32,
    pub max_batch: i32,
}

/// ssp_request: one sparsification request (graph and parameters are copied by ssp_submit).
#[repr(C)]
#[derive(Clone, Copy, Debug)]
pub struct SspRequest {
    pub kind: i32,
    pub graph: SspCsc,
    pub params: SspParams,
    pub check_probes: i32,
}

/// ssp_result: a finished request; `out` then belongs to the caller (ssp_csc_free).
#[repr(C)]
pub struct SspResult {
    pub status: i32,
    pub error: [c_char; 256],
    pub out: SspCscOut,
    pub stats: SspStats,
    pub est_bytes: i64,
    pub queue_ms: f64,
    pub run_ms: f64,
    pub latency_ms: f64,
    pub slot: i32,
    pub checked: i32,
    pub probe_upper_violations: i64,
    pub probe_lower_violations: i64,
    pub probe_mean_relative_error: f64,
    pub probe_max_relative_error: f64,
    pub components_graph: i64,
    pub components_sparsifier: i64,
    pub check_ms: f64,
    pub batch: i32,
}

/// ssp_server_info: counters of the request loop.
#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct SspServerInfo {
    pub submitted: i64,
    pub completed: i64,
    pub failed: i64,
    pub rejected: i64,
    pub pending: i64,
    pub inflight: i32,
    pub peak_inflight: i32,
    pub slots: i32,
    pub waiters: i32,
    pub peak_inflight_bytes: i64,
    pub budget_bytes: i64,
    pub batches: i64,
    pub peak_batch: i32,
}

/// ssp_probe_result: probe_quadratic_form's counts (experiments.rs:88-122).
#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct SspProbeResult {
    pub upper_bound_violations: i64,
    pub lower_bound_violations: i64,
    pub mean_relative_error: f64,
    pub std_dev_relative_error: f64,
    pub max_relative_error: f64,
    pub probes: i32,
}

/// Opaque handles.
pub type SspContext = c_void;
pub type SspServer = c_void;

extern "C" {
    pub fn ssp_last_error() -> *const c_char;

    pub fn ssp_context_create(device: i32, ctx: *mut *mut SspContext) -> c_int;
    pub fn ssp_context_destroy(ctx: *mut SspContext) -> c_int;
    pub fn ssp_context_set_stream(ctx: *mut SspContext, stream: *mut c_void) -> c_int;
    pub fn ssp_context_kernels_launched(ctx: *const SspContext) -> i64;
    pub fn ssp_context_workspace_bytes(ctx: *const SspContext) -> i64;
    pub fn ssp_context_release_workspace(ctx: *mut SspContext) -> c_int;

    pub fn ssp_params_default(p: *mut SspParams);
    pub fn ssp_params_new(p: *mut SspParams, epsilon: f64, beta_constant: i32, row_constant: i32, verbose: i32,
                          jl_factor: f64, jl_scaling_factor: f64, sketch_seed: u64, sampling_seed: u64, bench: i32,
                          sketch_uniform: i32, output_file: *const c_char, streaming: i32);
    pub fn ssp_params_cli(p: *mut SspParams, epsilon: f64, verbose: i32, sketch_seed: u64, sampling_seed: u64,
                          bench: i32, output_file: *const c_char);
    pub fn ssp_params_jl_dim(p: *const SspParams, n: i64) -> i32;
    pub fn ssp_params_beta(p: *const SspParams, n: i64) -> f64;
    pub fn ssp_params_jl_scale(p: *const SspParams, k: i32) -> f64;

    /// drop-in for ffi::run_solve_lap (lib.rs:103): row-major num_rows x num_cols in and out
    pub fn ssp_run_solve_lap(shared_jl_cols: *const f64, num_rows: usize, num_cols: usize, col_ptrs: *const i32,
                             col_ptrs_len: usize, row_indices: *const i32, values: *const f64, nnz: usize,
                             solver_output_filename: *const c_char, num_nodes: i32, verbose: i32,
                             solution_out: *mut f64) -> c_int;
    pub fn ssp_solve_opts_default(o: *mut SspSolveOpts);
    pub fn ssp_solve_lap(ctx: *mut SspContext, lap: *const SspCsc, y: *const f64, k: i32, z: *mut f64, mem: i32,
                         opts: *const SspSolveOpts, rep: *mut SspSolveReport) -> c_int;

    pub fn ssp_sparsify(ctx: *mut SspContext, graph: *const SspCsc, params: *const SspParams, out_mem: i32,
                        out: *mut SspCscOut, stats: *mut SspStats) -> c_int;
    pub fn ssp_sparsify_batch(ctx: *mut SspContext, count: i32, graphs: *const SspCsc, params: *const SspParams,
                              outs: *mut SspCscOut, stats: *mut SspStats) -> c_int;
    pub fn ssp_sparsify_laplacian(ctx: *mut SspContext, lap: *const SspCsc, params: *const SspParams, out_mem: i32,
                                  out: *mut SspCscOut, stats: *mut SspStats) -> c_int;
    pub fn ssp_laplacian_to_graph(lap: *const SspCsc, graph: *mut SspCscOut) -> c_int;
    pub fn ssp_csc_free(out: *mut SspCscOut) -> c_int;
    pub fn ssp_sparsify_update(ctx: *mut SspContext, laplacian: *const SspCsc, new_edges: *const SspCsc,
                               params: *const SspParams, out_mem: i32, out: *mut SspCscOut,
                               stats: *mut SspStats) -> c_int;

    pub fn ssp_shard_leverage(ctx: *mut SspContext, graph: *const SspCsc, params: *const SspParams, col_begin: i32,
                              col_end: i32, sq: *mut f64, m: *mut i64, stats: *mut SspStats) -> c_int;
    pub fn ssp_shard_finish(ctx: *mut SspContext, graph: *const SspCsc, params: *const SspParams,
                            sq_total: *const f64, out_mem: i32, out: *mut SspCscOut, stats: *mut SspStats) -> c_int;

    pub fn ssp_server_opts_default(opts: *mut SspServerOpts);
    pub fn ssp_request_footprint(graph: *const SspCsc, params: *const SspParams) -> i64;
    pub fn ssp_server_create(opts: *const SspServerOpts, server: *mut *mut SspServer) -> c_int;
    pub fn ssp_submit(server: *mut SspServer, req: *const SspRequest, ticket: *mut u64) -> c_int;
    pub fn ssp_wait(server: *mut SspServer, ticket: u64, timeout_ms: i64, res: *mut SspResult) -> c_int;
    pub fn ssp_poll(server: *mut SspServer, ticket: u64, res: *mut SspResult) -> c_int;
    pub fn ssp_server_info_get(server: *mut SspServer, info: *mut SspServerInfo) -> c_int;
    pub fn ssp_server_destroy(server: *mut SspServer) -> c_int;

    pub fn ssp_check_laplacian(ctx: *mut SspContext, lap: *const SspCsc, tol: f64, bad_columns: *mut i64,
                               max_abs_colsum: *mut f64, asymmetric_entries: *mut i64) -> c_int;
    pub fn ssp_probe_quadratic_form(ctx: *mut SspContext, lap_g: *const SspCsc, lap_h: *const SspCsc, epsilon: f64,
                                    probes: i32, seed: u64, res: *mut SspProbeResult) -> c_int;
    pub fn ssp_connected_components(ctx: *mut SspContext, m: *const SspCsc, mem: i32, labels: *mut i32,
                                    count: *mut i64) -> c_int;

    pub fn ssp_sparsify_mtx(input_file: *const c_char, output_file: *const c_char, params: *const SspParams,
                            stats: *mut SspStats) -> c_int;
    pub fn ssp_read_mtx(path: *const c_char, out: *mut SspCscOut) -> c_int;
    pub fn ssp_write_mtx(path: *const c_char, m: *const SspCsc) -> c_int;
    pub fn ssp_read_mtx_device(ctx: *mut SspContext, path: *const c_char, out_mem: i32, out: *mut SspCscOut) -> c_int;
    pub fn ssp_write_mtx_device(ctx: *mut SspContext, path: *const c_char, m: *const SspCsc) -> c_int;
    pub fn ssp_edgelist_to_mtx(input_path: *const c_char, output_path: *const c_char, default_weight: f64) -> c_int;
    pub fn ssp_edgelist_to_mtx_device(ctx: *mut SspContext, input_path: *const c_char, output_path: *const c_char,
                                      default_weight: f64, on_device: *mut i32) -> c_int;
}
