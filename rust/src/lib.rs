//! spec_spars_b200: the reference crate's sparsification entry points (tenchd/spec_spars) over the B200
//! library libspecspars.so.
//!
//! Replaces, for the sparsification path:
//!   `SparsifierParameters::new` / `new_default`   src/sparsifier.rs:163-209
//!   `Sparsifier::sparsify` (one call on a graph)   src/sparsifier.rs:735-790
//!   `ffi::run_solve_lap` (the cxx bridge)          src/lib.rs:103, src/example.cc:668-703
//!   `sparsify_dataset`                             src/lib.rs:158-168
//!   `read_mtx` / `write_mtx`                       src/utils.rs:149-154,189-191
//! All numerical work runs on the GPU inside the library; this crate only marshals plain pointers and
//! sizes across the C ABI (`ffi`) and turns status codes into `Result`s.

pub mod ffi;

use std::ffi::{CStr, CString};
use std::fmt;
use std::ptr;

/// A failed call: the library's status code (ffi::SSP_ERR_*) and its message.
#[derive(Debug, Clone)]
pub struct Error {
    pub code: i32,
    pub message: String,
}

impl fmt::Display for Error {
    fn fmt(&self, f: &mut fmt::Formatter<'_>) -> fmt::Result {
        write!(f, "spec_spars_b200 error {}: {}", self.code, self.message)
    }
}

impl std::error::Error for Error {}

fn check(rc: i32) -> Result<(), Error> {
    if rc == ffi::SSP_OK {
        return Ok(());
    }
    let message = unsafe {
        let p = ffi::ssp_last_error();
        if p.is_null() { String::new() } else { CStr::from_ptr(p).to_string_lossy().into_owned() }
    };
    Err(Error { code: rc, message })
}

fn cstring(s: &str) -> Result<CString, Error> {
    CString::new(s).map_err(|_| Error { code: ffi::SSP_ERR_INVALID, message: "string contains a NUL byte".into() })
}

/// A square matrix in compressed-sparse-column form on the host (CSC == CSR for the symmetric matrices of
/// this path): column j holds rows rowidx[colptr[j]..colptr[j + 1]], sorted.
#[derive(Debug, Clone, Default, PartialEq)]
pub struct Csc {
    pub n: usize,
    pub colptr: Vec<i64>,
    pub rowidx: Vec<i32>,
    pub values: Vec<f64>,
}

impl Csc {
    fn raw(&self) -> ffi::SspCsc {
        ffi::SspCsc {
            n: self.n as i64,
            nnz: self.values.len() as i64,
            colptr: self.colptr.as_ptr(),
            rowidx: self.rowidx.as_ptr(),
            values: self.values.as_ptr(),
            mem: ffi::SSP_MEM_HOST,
        }
    }

    /// Copies a library-allocated host result and frees it.
    fn take(mut out: ffi::SspCscOut) -> Csc {
        let n = out.n as usize;
        let nnz = out.nnz as usize;
        let m = unsafe {
            Csc {
                n,
                colptr: std::slice::from_raw_parts(out.colptr, n + 1).to_vec(),
                rowidx: if nnz > 0 { std::slice::from_raw_parts(out.rowidx, nnz).to_vec() } else { Vec::new() },
                values: if nnz > 0 { std::slice::from_raw_parts(out.values, nnz).to_vec() } else { Vec::new() },
            }
        };
        unsafe {
            ffi::ssp_csc_free(&mut out);
        }
        m
    }

    /// Edges of a Laplacian or adjacency: off-diagonal nonzeros with row < column (sparsifier.rs:346-353).
    pub fn num_edges(&self) -> usize {
        let mut e = 0;
        for j in 0..self.n {
            for p in self.colptr[j] as usize..self.colptr[j + 1] as usize {
                if (self.rowidx[p] as usize) < j && self.values[p] != 0.0 {
                    e += 1;
                }
            }
        }
        e
    }
}

fn empty_out() -> ffi::SspCscOut {
    ffi::SspCscOut { n: 0, nnz: 0, colptr: ptr::null_mut(), rowidx: ptr::null_mut(), values: ptr::null_mut(), mem: 0,
                     owned_by_context: 0 }
}

/// SparsifierParameters (sparsifier.rs:146-159): the reference's knobs with their meanings, plus the
/// library's additions (JL dimension and scale rules, reweighting, PCG tolerances, factor seed, precision)
/// as public fields of `raw`.
#[derive(Debug)]
pub struct SparsifierParameters {
    pub raw: ffi::SspParams,
    output_file: CString,
}

impl Clone for SparsifierParameters {
    // the copy's raw.output_file must point at its own string
    fn clone(&self) -> SparsifierParameters {
        let mut p = SparsifierParameters { raw: self.raw, output_file: self.output_file.clone() };
        p.raw.output_file = p.output_file.as_ptr();
        p
    }
}

impl SparsifierParameters {
    /// SparsifierParameters::new (sparsifier.rs:163-179), same arguments in the same order.
    #[allow(clippy::too_many_arguments)]
    pub fn new(epsilon: f64, beta_constant: i32, row_constant: i32, verbose: bool, jl_factor: f64,
               jl_scaling_factor: f64, sketch_seed: u64, sampling_seed: u64, benchmark: bool, sketch_uniform: bool,
               output_filename: String, streaming: bool) -> SparsifierParameters {
        let output_file = CString::new(output_filename).unwrap_or_default();
        let mut raw = unsafe { std::mem::zeroed::<ffi::SspParams>() };
        unsafe {
            ffi::ssp_params_new(&mut raw, epsilon, beta_constant, row_constant, verbose as i32, jl_factor,
                                jl_scaling_factor, sketch_seed, sampling_seed, benchmark as i32,
                                sketch_uniform as i32, output_file.as_ptr(), streaming as i32);
        }
        let mut p = SparsifierParameters { raw, output_file };
        p.raw.output_file = p.output_file.as_ptr();
        p
    }

    /// SparsifierParameters::new_default (sparsifier.rs:182-209).
    pub fn new_default(benchmark: bool) -> SparsifierParameters {
        let output_file = CString::default();
        let mut raw = unsafe { std::mem::zeroed::<ffi::SspParams>() };
        unsafe {
            ffi::ssp_params_default(&mut raw);
        }
        raw.bench = benchmark as i32;
        let mut p = SparsifierParameters { raw, output_file };
        p.raw.output_file = p.output_file.as_ptr();
        p
    }

    /// The knobs sparsify_dataset fixes (lib.rs:149-156): jl_factor 4, scale sqrt(3), beta 4, row 2,
    /// discrete signs, not streaming.
    pub fn cli(epsilon: f64, verbose: bool, sketch_seed: u64, sampling_seed: u64, benchmark: bool,
               output_filename: &str) -> SparsifierParameters {
        let output_file = CString::new(output_filename).unwrap_or_default();
        let mut raw = unsafe { std::mem::zeroed::<ffi::SspParams>() };
        unsafe {
            ffi::ssp_params_cli(&mut raw, epsilon, verbose as i32, sketch_seed, sampling_seed, benchmark as i32,
                                output_file.as_ptr());
        }
        let mut p = SparsifierParameters { raw, output_file };
        p.raw.output_file = p.output_file.as_ptr();
        p
    }

    /// k = ceil(log2(n) * jl_factor) (sparsifier.rs:272), or the rule/override the parameters name.
    pub fn jl_dim(&self, n: usize) -> i32 {
        unsafe { ffi::ssp_params_jl_dim(&self.raw, n as i64) }
    }

    /// beta = epsilon^-2 * beta_constant * ln n (sparsifier.rs:264).
    pub fn beta(&self, n: usize) -> f64 {
        unsafe { ffi::ssp_params_beta(&self.raw, n as i64) }
    }
}

/// One GPU and its stream and reusable device workspace.
pub struct Context {
    raw: *mut ffi::SspContext,
}

unsafe impl Send for Context {}

impl Context {
    pub fn new(device: i32) -> Result<Context, Error> {
        let mut raw = ptr::null_mut();
        check(unsafe { ffi::ssp_context_create(device, &mut raw) })?;
        Ok(Context { raw })
    }

    /// Sparsifier::sparsify on a graph given as a symmetric matrix whose upper triangle holds the edges:
    /// returns L_H (the full Laplacian of the sparsifier) and the statistics.
    pub fn sparsify(&mut self, graph: &Csc, params: &SparsifierParameters) -> Result<(Csc, ffi::SspStats), Error> {
        let g = graph.raw();
        let mut out = empty_out();
        let mut stats = ffi::SspStats::default();
        check(unsafe { ffi::ssp_sparsify(self.raw, &g, &params.raw, ffi::SSP_MEM_HOST, &mut out, &mut stats) })?;
        Ok((Csc::take(out), stats))
    }

    /// The same with a graph Laplacian as input (as Sparsifier::from_matrix loads one, sparsifier.rs:299-300).
    pub fn sparsify_laplacian(&mut self, lap: &Csc, params: &SparsifierParameters)
                              -> Result<(Csc, ffi::SspStats), Error> {
        let l = lap.raw();
        let mut out = empty_out();
        let mut stats = ffi::SspStats::default();
        check(unsafe {
            ffi::ssp_sparsify_laplacian(self.raw, &l, &params.raw, ffi::SSP_MEM_HOST, &mut out, &mut stats)
        })?;
        Ok((Csc::take(out), stats))
    }

    /// probe_quadratic_form (experiments.rs:88-122): (1 +- epsilon) violations of L_H against L_G on
    /// `probes` seeded uniform(-1, 1) probes.
    pub fn probe_quadratic_form(&mut self, lap_g: &Csc, lap_h: &Csc, epsilon: f64, probes: i32, seed: u64)
                                -> Result<ffi::SspProbeResult, Error> {
        let (g, h) = (lap_g.raw(), lap_h.raw());
        let mut r = ffi::SspProbeResult::default();
        check(unsafe { ffi::ssp_probe_quadratic_form(self.raw, &g, &h, epsilon, probes, seed, &mut r) })?;
        Ok(r)
    }
}

impl Drop for Context {
    fn drop(&mut self) {
        if !self.raw.is_null() {
            unsafe {
                ffi::ssp_context_destroy(self.raw);
            }
        }
    }
}

/// The cxx bridge's matrix type (lib.rs:81-85): `vec` holds num_rows x num_cols values row by row.
#[derive(Debug, Clone, Default, PartialEq)]
pub struct FlattenedVec {
    pub vec: Vec<f64>,
    pub num_cols: usize,
    pub num_rows: usize,
}

/// ffi::run_solve_lap (lib.rs:103) with the same arguments: solves L x_j = b_j for the columns of
/// shared_jl_cols (num_nodes x k, row-major) with the Laplacian in CSC (int32 pointers, as the bridge passes
/// it) and returns the solutions in the same layout.  The reference's C++ throws when a solve does not
/// converge (example.cc:566); this panics with the library's message, as the bridge would abort.
pub fn run_solve_lap(shared_jl_cols: FlattenedVec, rust_col_ptrs: Vec<i32>, rust_row_indices: Vec<i32>,
                     rust_values: Vec<f64>, solver_output_filename: &str, num_nodes: i32, verbose: bool)
                     -> FlattenedVec {
    try_run_solve_lap(&shared_jl_cols, &rust_col_ptrs, &rust_row_indices, &rust_values, solver_output_filename,
                      num_nodes, verbose)
        .unwrap_or_else(|e| panic!("run_solve_lap: {}", e))
}

/// run_solve_lap without the panic: SSP_ERR_NOT_CONVERGED (-4) where the reference throws.
pub fn try_run_solve_lap(shared_jl_cols: &FlattenedVec, col_ptrs: &[i32], row_indices: &[i32], values: &[f64],
                         solver_output_filename: &str, num_nodes: i32, verbose: bool)
                         -> Result<FlattenedVec, Error> {
    let name = cstring(solver_output_filename)?;
    let mut out = vec![0.0f64; shared_jl_cols.num_rows * shared_jl_cols.num_cols];
    check(unsafe {
        ffi::ssp_run_solve_lap(shared_jl_cols.vec.as_ptr(), shared_jl_cols.num_rows, shared_jl_cols.num_cols,
                               col_ptrs.as_ptr(), col_ptrs.len(), row_indices.as_ptr(), values.as_ptr(),
                               values.len(), name.as_ptr(), num_nodes, verbose as i32, out.as_mut_ptr())
    })?;
    Ok(FlattenedVec { vec: out, num_cols: shared_jl_cols.num_cols, num_rows: shared_jl_cols.num_rows })
}

/// read_mtx (utils.rs:149-154): a Matrix Market coordinate file, symmetric storage expanded, duplicates summed.
pub fn read_mtx(path: &str) -> Result<Csc, Error> {
    let p = cstring(path)?;
    let mut out = empty_out();
    check(unsafe { ffi::ssp_read_mtx(p.as_ptr(), &mut out) })?;
    Ok(Csc::take(out))
}

/// write_mtx (utils.rs:189-191).
pub fn write_mtx(path: &str, m: &Csc) -> Result<(), Error> {
    let p = cstring(path)?;
    let r = m.raw();
    check(unsafe { ffi::ssp_write_mtx(p.as_ptr(), &r) })
}

/// edge_list_to_matrix_market (utils.rs:413-526), same arguments: the edge list as a symmetric .mtx, first
/// weight of a repeated pair kept, weights written as Display writes an f64.
pub fn edge_list_to_matrix_market(input_path: &str, output_path: &str, default_weight: f64) -> Result<(), Error> {
    let (i, o) = (cstring(input_path)?, cstring(output_path)?);
    check(unsafe { ffi::ssp_edgelist_to_mtx(i.as_ptr(), o.as_ptr(), default_weight) })
}

impl Context {
    /// edge_list_to_matrix_market on this context's GPU: the same file byte for byte.  Returns whether the GPU
    /// wrote it (a file its line parser does not mirror is converted on the host instead).
    pub fn edge_list_to_matrix_market(&mut self, input_path: &str, output_path: &str, default_weight: f64)
                                      -> Result<bool, Error> {
        let (i, o) = (cstring(input_path)?, cstring(output_path)?);
        let mut on_device = 0i32;
        check(unsafe {
            ffi::ssp_edgelist_to_mtx_device(self.raw, i.as_ptr(), o.as_ptr(), default_weight, &mut on_device)
        })?;
        Ok(on_device != 0)
    }
}

/// sparsify_dataset (lib.rs:158-168), same arguments: read the .mtx graph, sparsify it with the knobs the
/// reference fixes for this call, and write L_H to output_filename (nothing written when it is empty).
#[allow(clippy::too_many_arguments)]
pub fn sparsify_dataset(input_filename: &str, dataset_name: &str, output_filename: &str, epsilon: f64,
                        verbose: bool, sketch_seed: u64, sampling_seed: u64, benchmark: bool)
                        -> Result<ffi::SspStats, Error> {
    println!("sparsifying {}", input_filename);
    let _ = dataset_name;
    let params = SparsifierParameters::cli(epsilon, verbose, sketch_seed, sampling_seed, benchmark, output_filename);
    let input = cstring(input_filename)?;
    let output = cstring(output_filename)?;
    let mut stats = ffi::SspStats::default();
    check(unsafe { ffi::ssp_sparsify_mtx(input.as_ptr(), output.as_ptr(), &params.raw, &mut stats) })?;
    Ok(stats)
}
