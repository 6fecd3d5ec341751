"""ctypes bindings of include/specspars.h and the reference-shaped Python API on top of them."""
import ctypes
import math
import os
import re

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libspecspars.so")
HEADER = os.path.join(HERE, "..", "include", "specspars.h")

SSP_OK = 0
SSP_MEM_HOST, SSP_MEM_DEVICE = 0, 1
SSP_JL_DIM_REF, SSP_JL_DIM_24 = 0, 1
SSP_JL_SCALE_FIXED, SSP_JL_SCALE_INV_SQRT_K = 0, 1
SSP_REWEIGHT_INV_SQRT_P, SSP_REWEIGHT_INV_P = 0, 1
SSP_TRSV_RULE, SSP_TRSV_TUNED, SSP_TRSV_CACHED, SSP_TRSV_FORCED = 0, 1, 2, 3
SSP_PRECISION_FP64, SSP_PRECISION_MIXED, SSP_PRECISION_PC32 = 0, 1, 2

ERROR_NAMES = {-1: "SSP_ERR_INVALID", -2: "SSP_ERR_CUDA", -3: "SSP_ERR_NOMEM", -4: "SSP_ERR_NOT_CONVERGED",
               -5: "SSP_ERR_CAPACITY", -6: "SSP_ERR_IO", -7: "SSP_ERR_NO_DEVICE", -8: "SSP_ERR_PENDING"}


def _header_symbols():
    try:
        txt = open(HEADER).read()
    except OSError:
        return []
    return sorted(set(re.findall(r"^\s*(?:const\s+)?[a-z_0-9]+\s*\**\s+(ssp_[a-z_0-9]+)\s*\(", txt, re.M)))


HEADER_SYMBOLS = _header_symbols()


class SspError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{ERROR_NAMES.get(code, code)}: {msg}")
        self.code = code


class _Csc(ctypes.Structure):
    _fields_ = [("n", ctypes.c_int64), ("nnz", ctypes.c_int64), ("colptr", ctypes.c_void_p),
                ("rowidx", ctypes.c_void_p), ("values", ctypes.c_void_p), ("mem", ctypes.c_int32)]


class _CscOut(ctypes.Structure):
    _fields_ = [("n", ctypes.c_int64), ("nnz", ctypes.c_int64), ("colptr", ctypes.c_void_p),
                ("rowidx", ctypes.c_void_p), ("values", ctypes.c_void_p), ("mem", ctypes.c_int32),
                ("owned_by_context", ctypes.c_int32)]


class _Params(ctypes.Structure):
    _fields_ = [("epsilon", ctypes.c_double), ("beta_constant", ctypes.c_int32), ("row_constant", ctypes.c_int32),
                ("verbose", ctypes.c_int32), ("jl_factor", ctypes.c_double), ("jl_scaling_factor", ctypes.c_double),
                ("sketch_seed", ctypes.c_uint64), ("sampling_seed", ctypes.c_uint64), ("bench", ctypes.c_int32),
                ("sketch_uniform", ctypes.c_int32), ("streaming", ctypes.c_int32), ("output_file", ctypes.c_char_p),
                ("jl_dim_rule", ctypes.c_int32), ("jl_scale_rule", ctypes.c_int32),
                ("prob_variance_correction", ctypes.c_int32), ("reweight", ctypes.c_int32),
                ("pcg_tol", ctypes.c_double), ("pcg_abs_tol", ctypes.c_double), ("pcg_max_iters", ctypes.c_int32),
                ("factor_seed", ctypes.c_uint64), ("dense_threshold", ctypes.c_int64),
                ("factor_max_degree", ctypes.c_int64), ("jl_dim_override", ctypes.c_int32),
                ("precision", ctypes.c_int32)]


class _Stats(ctypes.Structure):
    _fields_ = [("n", ctypes.c_int64), ("m_in", ctypes.c_int64), ("m_out", ctypes.c_int64), ("k", ctypes.c_int32),
                ("beta", ctypes.c_double), ("nnz_factor", ctypes.c_int64), ("factor_levels", ctypes.c_int32),
                ("pcg_max_iters_used", ctypes.c_int32), ("pcg_mean_iters", ctypes.c_double),
                ("pcg_max_relres", ctypes.c_double), ("ms_assembly", ctypes.c_double),
                ("ms_sketch", ctypes.c_double), ("ms_factor", ctypes.c_double), ("ms_solve", ctypes.c_double),
                ("ms_leverage", ctypes.c_double), ("ms_sample", ctypes.c_double), ("ms_total", ctypes.c_double),
                ("kernels_launched", ctypes.c_int64), ("ms_spmm", ctypes.c_double), ("n_spmm", ctypes.c_int64),
                ("ms_precond", ctypes.c_double), ("n_precond", ctypes.c_int64), ("nnz_laplacian", ctypes.c_int64),
                ("factor_max_degree_used", ctypes.c_int64), ("ms_autotune", ctypes.c_double),
                ("pcg_refinements", ctypes.c_int32), ("pcg_fp64_rounds", ctypes.c_int32),
                ("spmm_slabs", ctypes.c_int32), ("trsv_shapes", ctypes.c_int32),
                ("trsv_levels_w8", ctypes.c_int32), ("trsv_levels_w16", ctypes.c_int32),
                ("trsv_levels_w32", ctypes.c_int32), ("ms_trsv_tune", ctypes.c_double)]


class _SolveOpts(ctypes.Structure):
    _fields_ = [("tol", ctypes.c_double), ("abs_tol", ctypes.c_double), ("max_iters", ctypes.c_int32),
                ("factor_seed", ctypes.c_uint64), ("dense_threshold", ctypes.c_int64), ("verbose", ctypes.c_int32),
                ("factor_max_degree", ctypes.c_int64), ("precision", ctypes.c_int32)]


class _SolveReport(ctypes.Structure):
    _fields_ = [("k", ctypes.c_int32), ("max_iters_used", ctypes.c_int32), ("mean_iters", ctypes.c_double),
                ("max_relres", ctypes.c_double), ("not_converged", ctypes.c_int32),
                ("nnz_factor", ctypes.c_int64), ("factor_levels", ctypes.c_int32), ("ms_factor", ctypes.c_double),
                ("ms_solve", ctypes.c_double), ("factor_max_degree_used", ctypes.c_int64),
                ("refinements", ctypes.c_int32), ("fp64_rounds", ctypes.c_int32), ("spmm_slabs", ctypes.c_int32),
                ("trsv_shapes", ctypes.c_int32), ("trsv_levels_w8", ctypes.c_int32),
                ("trsv_levels_w16", ctypes.c_int32), ("trsv_levels_w32", ctypes.c_int32),
                ("ms_trsv_tune", ctypes.c_double)]


class _ServerOpts(ctypes.Structure):
    _fields_ = [("device", ctypes.c_int32), ("slots", ctypes.c_int32), ("hbm_budget_bytes", ctypes.c_int64),
                ("max_pending", ctypes.c_int32), ("max_batch", ctypes.c_int32)]


class _Request(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_int32), ("graph", _Csc), ("params", _Params), ("check_probes", ctypes.c_int32)]


class _Result(ctypes.Structure):
    _fields_ = [("status", ctypes.c_int32), ("error", ctypes.c_char * 256), ("out", _CscOut), ("stats", _Stats),
                ("est_bytes", ctypes.c_int64), ("queue_ms", ctypes.c_double), ("run_ms", ctypes.c_double),
                ("latency_ms", ctypes.c_double), ("slot", ctypes.c_int32), ("checked", ctypes.c_int32),
                ("probe_upper_violations", ctypes.c_int64), ("probe_lower_violations", ctypes.c_int64),
                ("probe_mean_relative_error", ctypes.c_double), ("probe_max_relative_error", ctypes.c_double),
                ("components_graph", ctypes.c_int64), ("components_sparsifier", ctypes.c_int64),
                ("check_ms", ctypes.c_double), ("batch", ctypes.c_int32)]


class _ServerInfo(ctypes.Structure):
    _fields_ = [("submitted", ctypes.c_int64), ("completed", ctypes.c_int64), ("failed", ctypes.c_int64),
                ("rejected", ctypes.c_int64), ("pending", ctypes.c_int64), ("inflight", ctypes.c_int32),
                ("peak_inflight", ctypes.c_int32), ("slots", ctypes.c_int32), ("waiters", ctypes.c_int32),
                ("peak_inflight_bytes", ctypes.c_int64), ("budget_bytes", ctypes.c_int64),
                ("batches", ctypes.c_int64), ("peak_batch", ctypes.c_int32)]


class _ProbeResult(ctypes.Structure):
    _fields_ = [("upper_bound_violations", ctypes.c_int64), ("lower_bound_violations", ctypes.c_int64),
                ("mean_relative_error", ctypes.c_double), ("std_dev_relative_error", ctypes.c_double),
                ("max_relative_error", ctypes.c_double), ("probes", ctypes.c_int32)]


_LIB = None
P = ctypes.c_void_p
I32, I64, U64, DBL = ctypes.c_int32, ctypes.c_int64, ctypes.c_uint64, ctypes.c_double


def lib():
    """Load libspecspars.so from the package directory.  Missing library is an error, not a fallback."""
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            raise SspError(-1, f"{LIB_PATH} is not built; run `python -m spec_spars_b200.build`")
        L = ctypes.CDLL(LIB_PATH)
        sig = {
            "ssp_last_error": ([], ctypes.c_char_p),
            "ssp_context_create": ([I32, ctypes.POINTER(P)], ctypes.c_int),
            "ssp_context_destroy": ([P], ctypes.c_int),
            "ssp_context_set_stream": ([P, P], ctypes.c_int),
            "ssp_context_kernels_launched": ([P], I64),
            "ssp_context_workspace_bytes": ([P], I64),
            "ssp_params_default": ([ctypes.POINTER(_Params)], None),
            "ssp_params_new": ([ctypes.POINTER(_Params), DBL, I32, I32, I32, DBL, DBL, U64, U64, I32, I32,
                                ctypes.c_char_p, I32], None),
            "ssp_params_cli": ([ctypes.POINTER(_Params), DBL, I32, U64, U64, I32, ctypes.c_char_p], None),
            "ssp_params_jl_dim": ([ctypes.POINTER(_Params), I64], I32),
            "ssp_params_beta": ([ctypes.POINTER(_Params), I64], DBL),
            "ssp_params_jl_scale": ([ctypes.POINTER(_Params), I32], DBL),
            "ssp_run_solve_lap": ([P, ctypes.c_size_t, ctypes.c_size_t, P, ctypes.c_size_t, P, P, ctypes.c_size_t,
                                   ctypes.c_char_p, I32, I32, P], ctypes.c_int),
            "ssp_solve_opts_default": ([ctypes.POINTER(_SolveOpts)], None),
            "ssp_solve_lap": ([P, ctypes.POINTER(_Csc), P, I32, P, I32, ctypes.POINTER(_SolveOpts),
                               ctypes.POINTER(_SolveReport)], ctypes.c_int),
            "ssp_sparsify_batch": ([P, I32, ctypes.POINTER(_Csc), ctypes.POINTER(_Params), ctypes.POINTER(_CscOut),
                                    ctypes.POINTER(_Stats)], ctypes.c_int),
            "ssp_sparsify": ([P, ctypes.POINTER(_Csc), ctypes.POINTER(_Params), I32, ctypes.POINTER(_CscOut),
                              ctypes.POINTER(_Stats)], ctypes.c_int),
            "ssp_sparsify_laplacian": ([P, ctypes.POINTER(_Csc), ctypes.POINTER(_Params), I32,
                                        ctypes.POINTER(_CscOut), ctypes.POINTER(_Stats)], ctypes.c_int),
            "ssp_laplacian_to_graph": ([ctypes.POINTER(_Csc), ctypes.POINTER(_CscOut)], ctypes.c_int),
            "ssp_csc_free": ([ctypes.POINTER(_CscOut)], ctypes.c_int),
            "ssp_sparsify_mtx": ([ctypes.c_char_p, ctypes.c_char_p, ctypes.POINTER(_Params),
                                  ctypes.POINTER(_Stats)], ctypes.c_int),
            "ssp_read_mtx": ([ctypes.c_char_p, ctypes.POINTER(_CscOut)], ctypes.c_int),
            "ssp_read_mtx_device": ([P, ctypes.c_char_p, I32, ctypes.POINTER(_CscOut)], ctypes.c_int),
            "ssp_write_mtx_device": ([P, ctypes.c_char_p, ctypes.POINTER(_Csc)], ctypes.c_int),
            "ssp_stage_scan": ([P, P, I64, P], ctypes.c_int),
            "ssp_parse_decimal": ([ctypes.c_char_p, ctypes.c_size_t, ctypes.POINTER(ctypes.c_double)], ctypes.c_int),
            "ssp_format_g17": ([ctypes.c_double, ctypes.c_char_p, ctypes.c_size_t], ctypes.c_int),
            "ssp_write_mtx": ([ctypes.c_char_p, ctypes.POINTER(_Csc)], ctypes.c_int),
            "ssp_gen_grid2d": ([I64, I64, DBL, ctypes.POINTER(_CscOut)], ctypes.c_int),
            "ssp_gen_grid3d": ([I64, I64, I64, DBL, DBL, U64, ctypes.POINTER(_CscOut)], ctypes.c_int),
            "ssp_gen_er": ([I64, DBL, DBL, DBL, U64, ctypes.POINTER(_CscOut)], ctypes.c_int),
            "ssp_edgelist_to_mtx": ([ctypes.c_char_p, ctypes.c_char_p, DBL], ctypes.c_int),
            "ssp_edgelist_to_mtx_device": ([P, ctypes.c_char_p, ctypes.c_char_p, DBL, ctypes.POINTER(I32)],
                                           ctypes.c_int),
            "ssp_format_shortest": ([DBL, ctypes.c_char_p, ctypes.c_size_t], ctypes.c_int),
            "ssp_gen_rmat": ([I32, I32, DBL, DBL, DBL, U64, ctypes.POINTER(_CscOut)], ctypes.c_int),
            "ssp_gen_rgg": ([I64, DBL, DBL, DBL, U64, ctypes.POINTER(_CscOut)], ctypes.c_int),
            "ssp_check_laplacian": ([P, ctypes.POINTER(_Csc), DBL, ctypes.POINTER(I64), ctypes.POINTER(DBL),
                                     ctypes.POINTER(I64)], ctypes.c_int),
            "ssp_probe_vectors": ([P, I64, I32, U64, I32, P], ctypes.c_int),
            "ssp_quadratic_forms": ([P, ctypes.POINTER(_Csc), P, I32, I32, P], ctypes.c_int),
            "ssp_probe_quadratic_form": ([P, ctypes.POINTER(_Csc), ctypes.POINTER(_Csc), DBL, I32, U64,
                                          ctypes.POINTER(_ProbeResult)], ctypes.c_int),
            "ssp_connected_components": ([P, ctypes.POINTER(_Csc), I32, P, ctypes.POINTER(I64)], ctypes.c_int),
            "ssp_context_release_workspace": ([P], ctypes.c_int),
            "ssp_server_opts_default": ([ctypes.POINTER(_ServerOpts)], None),
            "ssp_request_footprint": ([ctypes.POINTER(_Csc), ctypes.POINTER(_Params)], I64),
            "ssp_server_create": ([ctypes.POINTER(_ServerOpts), ctypes.POINTER(P)], ctypes.c_int),
            "ssp_submit": ([P, ctypes.POINTER(_Request), ctypes.POINTER(U64)], ctypes.c_int),
            "ssp_wait": ([P, U64, I64, ctypes.POINTER(_Result)], ctypes.c_int),
            "ssp_poll": ([P, U64, ctypes.POINTER(_Result)], ctypes.c_int),
            "ssp_server_info_get": ([P, ctypes.POINTER(_ServerInfo)], ctypes.c_int),
            "ssp_server_destroy": ([P], ctypes.c_int),
            "ssp_stage_graph": ([P, ctypes.POINTER(_Csc), ctypes.POINTER(I64), ctypes.POINTER(I64), P, P, P, P, P, P],
                                ctypes.c_int),
            "ssp_stage_sketch": ([P, I64, I64, P, P, P, I32, I32, DBL, U64, I32, P], ctypes.c_int),
            "ssp_stage_factor": ([P, ctypes.POINTER(_Csc), U64, I64, I64, ctypes.POINTER(I64), P, P, P, P, P,
                                  ctypes.POINTER(I32)], ctypes.c_int),
            "ssp_stage_precond": ([P, ctypes.POINTER(_Csc), U64, I64, I64, P, I32, P], ctypes.c_int),
            "ssp_stage_diff_norms": ([P, I64, I64, P, P, P, I32, I32, P], ctypes.c_int),
            "ssp_stage_probs": ([P, I64, P, P, DBL, DBL, I32, P], ctypes.c_int),
            "ssp_stage_coins": ([P, I64, U64, I32, P], ctypes.c_int),
            "ssp_stage_sample_apply": ([P, ctypes.POINTER(_Csc), P, P, I32, I32, P, ctypes.POINTER(_CscOut)],
                                       ctypes.c_int),
            "ssp_stage_leverage_probs_static": ([P, I64, I64, P, P, P, I32, P, DBL, DBL, P], ctypes.c_int),
            "ssp_shard_leverage": ([P, ctypes.POINTER(_Csc), ctypes.POINTER(_Params), I32, I32, P,
                                    ctypes.POINTER(I64), ctypes.POINTER(_Stats)], ctypes.c_int),
            "ssp_sparsify_update": ([P, ctypes.POINTER(_Csc), ctypes.POINTER(_Csc), ctypes.POINTER(_Params), I32,
                                     ctypes.POINTER(_CscOut), ctypes.POINTER(_Stats)], ctypes.c_int),
            "ssp_shard_finish": ([P, ctypes.POINTER(_Csc), ctypes.POINTER(_Params), P, I32, ctypes.POINTER(_CscOut),
                                  ctypes.POINTER(_Stats)], ctypes.c_int),
        }
        for name, (args, res) in sig.items():
            f = getattr(L, name)
            f.argtypes = args
            f.restype = res
        _LIB = L
    return _LIB


def _check(rc):
    if rc != SSP_OK:
        msg = lib().ssp_last_error()
        raise SspError(rc, msg.decode() if msg else "")


def _ptr(a):
    if a is None:
        return None
    if isinstance(a, int):
        return a
    if hasattr(a, "data_ptr"):  # torch tensor
        return a.data_ptr()
    return a.ctypes.data


# ---------------------------------------------------------------- CSC container
class CSC:
    """Host CSC matrix (colptr int64, rowidx int32, values float64)."""

    def __init__(self, n, colptr, rowidx, values):
        self.n = int(n)
        self.colptr = np.ascontiguousarray(colptr, np.int64)
        self.rowidx = np.ascontiguousarray(rowidx, np.int32)
        self.values = np.ascontiguousarray(values, np.float64)

    @property
    def nnz(self):
        return int(self.colptr[-1])

    def _struct(self):
        return _Csc(self.n, self.nnz, _ptr(self.colptr), _ptr(self.rowidx), _ptr(self.values), SSP_MEM_HOST)

    @classmethod
    def _from_out(cls, out):
        n, nnz = out.n, out.nnz
        cp = np.ctypeslib.as_array((ctypes.c_int64 * (n + 1)).from_address(out.colptr)).copy()
        if nnz:
            ri = np.ctypeslib.as_array((ctypes.c_int32 * nnz).from_address(out.rowidx)).copy()
            va = np.ctypeslib.as_array((ctypes.c_double * nnz).from_address(out.values)).copy()
        else:
            ri = np.zeros(0, np.int32)
            va = np.zeros(0, np.float64)
        return cls(n, cp, ri, va)

    def to_scipy(self):
        import scipy.sparse as sp
        return sp.csc_matrix((self.values, self.rowidx, self.colptr), shape=(self.n, self.n))

    @classmethod
    def from_scipy(cls, m):
        import scipy.sparse as sp
        m = sp.csc_matrix(m)
        m.sort_indices()
        m.sum_duplicates()
        return cls(m.shape[0], m.indptr, m.indices, m.data)

    def num_edges(self):
        """(nnz - stored diagonal) / 2 (Sparsifier::num_edges, sparsifier.rs:346-353)."""
        cols = np.repeat(np.arange(self.n), np.diff(self.colptr))
        diag = int(np.count_nonzero(cols == self.rowidx))
        return (self.nnz - diag) // 2


class DeviceCSC:
    """A CSC whose arrays live on the device, given as raw pointers (for example the L_H that
    Context.sparsify_device returns, or torch tensors' data_ptr()); usable wherever the API takes a CSC."""

    def __init__(self, n, nnz, colptr_ptr, rowidx_ptr, values_ptr):
        self.n, self.nnz = int(n), int(nnz)
        self._p = (colptr_ptr, rowidx_ptr, values_ptr)

    def _struct(self):
        return _Csc(self.n, self.nnz, self._p[0], self._p[1], self._p[2], SSP_MEM_DEVICE)


class _HostOut:
    """Owns a library-allocated host CSC; frees it once no array views it any more."""

    def __init__(self, out):
        self.out = out

    def __del__(self):
        try:
            lib().ssp_csc_free(ctypes.byref(self.out))
        except Exception:
            pass


def _take_out(out):
    """Host CSC result as numpy arrays viewing the library's buffers (no copy); they are freed with the
    last array."""
    if out.mem != SSP_MEM_HOST or out.nnz == 0:
        try:
            return CSC._from_out(out)
        finally:
            lib().ssp_csc_free(ctypes.byref(out))
    holder = _HostOut(out)
    views = []
    for addr, ct, cnt, dt in ((out.colptr, ctypes.c_int64, out.n + 1, np.int64),
                              (out.rowidx, ctypes.c_int32, out.nnz, np.int32),
                              (out.values, ctypes.c_double, out.nnz, np.float64)):
        buf = (ct * cnt).from_address(addr)
        buf._owner = holder
        views.append(np.frombuffer(buf, dtype=dt))
    return CSC(out.n, *views)


def read_mtx(path):
    out = _CscOut()
    _check(lib().ssp_read_mtx(path.encode(), ctypes.byref(out)))
    return _take_out(out)


def laplacian_to_graph(lap):
    """The graph whose Laplacian is lap: entry (i, j) = -lap[i, j] off the diagonal, the diagonal dropped
    (host only, no GPU needed)."""
    s = lap._struct()
    out = _CscOut()
    _check(lib().ssp_laplacian_to_graph(ctypes.byref(s), ctypes.byref(out)))
    return _take_out(out)


def write_mtx(path, m):
    s = m._struct()
    _check(lib().ssp_write_mtx(path.encode(), ctypes.byref(s)))


def parse_decimal(token):
    """(status, value): status 1 = exact device conversion, 0 = left to the host's strtod, -1 = malformed."""
    b = token.encode() if isinstance(token, str) else bytes(token)
    v = ctypes.c_double(0.0)
    rc = lib().ssp_parse_decimal(b, len(b), ctypes.byref(v))
    return rc, v.value


def format_g17(x):
    """printf("%.17g", x) as the device formats it, or None where the host formats it."""
    buf = ctypes.create_string_buffer(40)
    n = lib().ssp_format_g17(float(x), buf, 40)
    return None if n < 0 else buf.raw[:n].decode()


def gen_grid2d(nx, ny, w=1.0):
    out = _CscOut()
    _check(lib().ssp_gen_grid2d(nx, ny, w, ctypes.byref(out)))
    return _take_out(out)


def gen_grid3d(nx, ny, nz, wlog10_lo=-3.0, wlog10_hi=3.0, seed=2):
    out = _CscOut()
    _check(lib().ssp_gen_grid3d(nx, ny, nz, wlog10_lo, wlog10_hi, seed, ctypes.byref(out)))
    return _take_out(out)


def gen_er(n, avg_degree, wlo=0.5, whi=2.0, seed=1):
    out = _CscOut()
    _check(lib().ssp_gen_er(n, avg_degree, wlo, whi, seed, ctypes.byref(out)))
    return _take_out(out)


def edge_list_to_matrix_market(input_path, output_path, default_weight=1.0, ctx=None):
    """edge_list_to_matrix_market (utils.rs:413-526).  With a Context the conversion runs on its GPU
    (ssp_edgelist_to_mtx_device) and returns True when the GPU wrote the file, False when the file went to the
    host converter; the file is the same either way."""
    if ctx is not None:
        dev = I32(0)
        _check(lib().ssp_edgelist_to_mtx_device(ctx._h, str(input_path).encode(), str(output_path).encode(),
                                                default_weight, ctypes.byref(dev)))
        return bool(dev.value)
    _check(lib().ssp_edgelist_to_mtx(str(input_path).encode(), str(output_path).encode(), default_weight))


def format_shortest(v):
    """The edge-list converter's device formatter, run on the host: v as Rust displays an f64 (shortest
    round-trip digits, no exponent), or None for values it leaves to the host."""
    buf = ctypes.create_string_buffer(64)
    n = lib().ssp_format_shortest(float(v), buf, 64)
    return buf.value.decode() if n >= 0 else None


def gen_rmat(scale, edge_factor=16, a=0.57, b=0.19, c=0.19, seed=3):
    """R-MAT graph, largest connected component (the R-MAT configuration: scale 22, edge factor 16)."""
    out = _CscOut()
    _check(lib().ssp_gen_rmat(scale, edge_factor, a, b, c, seed, ctypes.byref(out)))
    return _take_out(out)


def gen_rgg(n, avg_degree, wlo=0.1, whi=10.0, seed=1):
    out = _CscOut()
    _check(lib().ssp_gen_rgg(n, avg_degree, wlo, whi, seed, ctypes.byref(out)))
    return _take_out(out)


# ---------------------------------------------------------------- parameters
class SparsifierParameters:
    """SparsifierParameters (sparsifier.rs:146-210) plus this build's options."""

    _FIELDS = [f for f, _ in _Params._fields_]

    def __init__(self, s=None):
        object.__setattr__(self, "_s", s if s is not None else _Params())
        object.__setattr__(self, "_out", b"")

    @classmethod
    def new(cls, epsilon, beta_constant, row_constant, verbose, jl_factor, jl_scaling_factor, sketch_seed,
            sampling_seed, bench, sketch_uniform, output_file, streaming):
        p = cls()
        out = (output_file or "").encode()
        object.__setattr__(p, "_out", out)
        lib().ssp_params_new(ctypes.byref(p._s), epsilon, beta_constant, row_constant, int(verbose), jl_factor,
                             jl_scaling_factor, sketch_seed, sampling_seed, int(bench), int(sketch_uniform), out,
                             int(streaming))
        return p

    @classmethod
    def new_default(cls, bench=False):
        p = cls()
        lib().ssp_params_default(ctypes.byref(p._s))
        p._s.bench = int(bench)
        return p

    @classmethod
    def cli(cls, epsilon=0.5, verbose=False, sketch_seed=0, sampling_seed=0, bench=False, output_file=""):
        """The knobs sparsify_dataset hard-codes (lib.rs:149-156)."""
        p = cls()
        out = (output_file or "").encode()
        object.__setattr__(p, "_out", out)
        lib().ssp_params_cli(ctypes.byref(p._s), epsilon, int(verbose), sketch_seed, sampling_seed, int(bench), out)
        return p

    @classmethod
    def baseline(cls, epsilon=0.5, pcg_tol=1e-8, sketch_seed=0, sampling_seed=0):
        """k = ceil(24 ln n / eps^2) columns of +-1/sqrt(k) signs, variance-corrected probabilities, kept
        edges reweighted by w/p.  These are the benchmark configurations, whose outputs are checked against
        (1 +- eps) on probes and extremal eigenvalues: w/p keeps E[L_H] = L_G, while the reference's w/sqrt(p)
        (sparsifier.rs:657) leaves L_H biased low wherever p < 1."""
        p = cls.cli(epsilon=epsilon, sketch_seed=sketch_seed, sampling_seed=sampling_seed)
        p.jl_dim_rule = SSP_JL_DIM_24
        p.jl_scale_rule = SSP_JL_SCALE_INV_SQRT_K
        p.prob_variance_correction = 1
        p.reweight = SSP_REWEIGHT_INV_P
        p.pcg_tol = pcg_tol
        p.pcg_abs_tol = 0.0
        return p

    def __getattr__(self, k):
        if k in SparsifierParameters._FIELDS:
            v = getattr(self._s, k)
            return v.decode() if isinstance(v, bytes) else v
        raise AttributeError(k)

    def __setattr__(self, k, v):
        if k == "output_file":
            b = (v or "").encode()
            object.__setattr__(self, "_out", b)
            self._s.output_file = b
        elif k in SparsifierParameters._FIELDS:
            setattr(self._s, k, v)
        else:
            raise AttributeError(k)

    def jl_dim(self, n):
        return lib().ssp_params_jl_dim(ctypes.byref(self._s), n)

    def beta(self, n):
        return lib().ssp_params_beta(ctypes.byref(self._s), n)

    def jl_scale(self, k):
        return lib().ssp_params_jl_scale(ctypes.byref(self._s), k)


def _stats_dict(st):
    return {f: getattr(st, f) for f, _ in _Stats._fields_}


class SparsificationStats:
    """SparsificationStats (sparsifier.rs:213-237)."""

    def __init__(self, d):
        self.__dict__.update(d)
        self.original_num_edges = d["m_in"]
        self.final_num_edges = d["m_out"]

    def sparsification_rate(self):
        return self.final_num_edges / self.original_num_edges if self.original_num_edges else 0.0


# ---------------------------------------------------------------- context
class Context:
    def __init__(self, device=0):
        h = P()
        _check(lib().ssp_context_create(device, ctypes.byref(h)))
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            lib().ssp_context_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def read_mtx(self, path):
        """utils::read_mtx parsed on the GPU (host CSC result, identical to read_mtx)."""
        out = _CscOut()
        _check(lib().ssp_read_mtx_device(self._h, path.encode(), SSP_MEM_HOST, ctypes.byref(out)))
        return _take_out(out)

    def write_mtx(self, path, m):
        """utils::write_mtx formatted on the GPU (the bytes write_mtx writes)."""
        s = m._struct()
        _check(lib().ssp_write_mtx_device(self._h, path.encode(), ctypes.byref(s)))

    def set_stream(self, stream_ptr):
        _check(lib().ssp_context_set_stream(self._h, stream_ptr))

    @property
    def kernels_launched(self):
        return lib().ssp_context_kernels_launched(self._h)

    def release_workspace(self):
        """Free the context's cached device workspace (it grows again on the next call)."""
        _check(lib().ssp_context_release_workspace(self._h))

    @property
    def workspace_bytes(self):
        return lib().ssp_context_workspace_bytes(self._h)

    def sparsify(self, graph, params):
        """Host CSC in, host CSC L_H out."""
        g = graph._struct()
        out = _CscOut()
        st = _Stats()
        _check(lib().ssp_sparsify(self._h, ctypes.byref(g), ctypes.byref(params._s), SSP_MEM_HOST,
                                  ctypes.byref(out), ctypes.byref(st)))
        return _take_out(out), _stats_dict(st)

    def sparsify_batch(self, graphs, params):
        """Several host graphs sparsified as one disjoint union (ssp_sparsify_batch): one factorization and one
        all-columns PCG for the batch, every PCG scalar per (graph, column).  params: one SparsifierParameters
        per graph, or one for all; they must agree on the factor seed, precision, PCG options, reweighting and a
        fixed truncation (factor_max_degree >= 0), with dense_threshold = 0.  Returns [(L_H, stats)]."""
        graphs = list(graphs)
        if isinstance(params, SparsifierParameters):
            params = [params] * len(graphs)
        params = list(params)
        if len(params) != len(graphs) or not graphs:
            raise ValueError("sparsify_batch: need one SparsifierParameters per graph")
        cnt = len(graphs)
        gs = (_Csc * cnt)(*[g._struct() for g in graphs])
        ps = (_Params * cnt)(*[p._s for p in params])
        outs = (_CscOut * cnt)()
        sts = (_Stats * cnt)()
        _check(lib().ssp_sparsify_batch(self._h, cnt, gs, ps, outs, sts))
        res = []
        for i in range(cnt):
            out = _CscOut()
            ctypes.memmove(ctypes.byref(out), ctypes.byref(outs[i]), ctypes.sizeof(_CscOut))
            res.append((_take_out(out), _stats_dict(sts[i])))
        return res

    def sparsify_laplacian(self, lap, params):
        """Host Laplacian L_G in (as Sparsifier::from_matrix reads one, sparsifier.rs:299-300), host L_H out;
        the same result as sparsify on laplacian_to_graph(lap)."""
        g = lap._struct()
        out = _CscOut()
        st = _Stats()
        _check(lib().ssp_sparsify_laplacian(self._h, ctypes.byref(g), ctypes.byref(params._s), SSP_MEM_HOST,
                                            ctypes.byref(out), ctypes.byref(st)))
        return _take_out(out), _stats_dict(st)

    def sparsify_device(self, n, nnz, colptr_ptr, rowidx_ptr, values_ptr, params):
        """Device CSC in (raw pointers), device CSC out (context-owned until the next call)."""
        g = _Csc(n, nnz, colptr_ptr, rowidx_ptr, values_ptr, SSP_MEM_DEVICE)
        out = _CscOut()
        st = _Stats()
        _check(lib().ssp_sparsify(self._h, ctypes.byref(g), ctypes.byref(params._s), SSP_MEM_DEVICE,
                                  ctypes.byref(out), ctypes.byref(st)))
        return (out.nnz, out.colptr, out.rowidx, out.values), _stats_dict(st)

    # ---- checks (a15): check_diagonal, compute_quadratic_form, probe_quadratic_form, verify_ccs
    def check_laplacian(self, lap, tol=1e-10):
        """Sparsifier::check_diagonal (sparsifier.rs:806-817) as counts instead of asserts."""
        bad, mx, asym = I64(0), DBL(0), I64(0)
        g = lap._struct()
        _check(lib().ssp_check_laplacian(self._h, ctypes.byref(g), tol, ctypes.byref(bad), ctypes.byref(mx),
                                         ctypes.byref(asym)))
        return {"bad_columns": bad.value, "max_abs_colsum": mx.value, "asymmetric_entries": asym.value,
                "ok": bad.value == 0 and asym.value == 0}

    def probe_vectors(self, n, p, seed=0):
        X = np.zeros((p, n), np.float64)  # column-major n x p = p contiguous vectors
        _check(lib().ssp_probe_vectors(self._h, n, p, seed, SSP_MEM_HOST, _ptr(X)))
        return X.T

    def quadratic_forms(self, lap, X):
        """x_j^T L x_j for the columns of X (n x p)."""
        X = np.asarray(X, np.float64)
        if X.ndim == 1:
            X = X[:, None]
        Xc = np.ascontiguousarray(X.T)
        out = np.zeros(X.shape[1], np.float64)
        g = lap._struct()
        _check(lib().ssp_quadratic_forms(self._h, ctypes.byref(g), _ptr(Xc), X.shape[1], SSP_MEM_HOST, _ptr(out)))
        return out

    def probe_quadratic_form(self, lap_g, lap_h, epsilon, probes=100, seed=0):
        """probe_quadratic_form (experiments.rs:88-122) with Philox probes."""
        r = _ProbeResult()
        g, h = lap_g._struct(), lap_h._struct()
        _check(lib().ssp_probe_quadratic_form(self._h, ctypes.byref(g), ctypes.byref(h), epsilon, probes, seed,
                                              ctypes.byref(r)))
        return {f: getattr(r, f) for f, _ in _ProbeResult._fields_}

    def connected_components(self, m):
        """(number of components, label = smallest vertex of the component) over off-diagonal nonzeros."""
        labels = np.zeros(m.n, np.int32)
        cnt = I64(0)
        g = m._struct()
        _check(lib().ssp_connected_components(self._h, ctypes.byref(g), SSP_MEM_HOST, _ptr(labels),
                                              ctypes.byref(cnt)))
        return cnt.value, labels

    def verify_ccs(self, graph, sparsifier):
        """verify_ccs (experiments.rs:58-64): the sparsifier keeps the number of connected components."""
        return self.connected_components(graph)[0] == self.connected_components(sparsifier)[0]

    def sparsify_update(self, laplacian, new_edges, params):
        """Sparsify again after inserting edges: current L_H + the new edges (sketched alone), as
        Sparsifier::insert + sparsify (sparsifier.rs:357-376,735-790).  Returns (L_H, stats)."""
        a, b = laplacian._struct(), new_edges._struct()
        out = _CscOut()
        st = _Stats()
        _check(lib().ssp_sparsify_update(self._h, ctypes.byref(a), ctypes.byref(b), ctypes.byref(params._s),
                                         SSP_MEM_HOST, ctypes.byref(out), ctypes.byref(st)))
        return _take_out(out), _stats_dict(st)

    def num_edges(self, graph):
        """Edges of a host graph as the sparsifier counts them (upper triangle, value != 0)."""
        m = I64(0)
        g = graph._struct()
        _check(lib().ssp_shard_leverage(self._h, ctypes.byref(g), None, 0, 0, None, ctypes.byref(m), None))
        return m.value

    def shard_leverage(self, graph, params, col_begin, col_end, sq_ptr):
        """Phase 1 of a column-split sparsification: solve the global JL columns [col_begin, col_end) and
        write the per-edge partial sums of squared differences into the device buffer at sq_ptr."""
        g = graph._struct()
        m = I64(0)
        st = _Stats()
        _check(lib().ssp_shard_leverage(self._h, ctypes.byref(g), ctypes.byref(params._s), col_begin, col_end,
                                        sq_ptr, ctypes.byref(m), ctypes.byref(st)))
        return _stats_dict(st)

    def shard_finish(self, graph, params, sq_total_ptr, device_out=False):
        """Phase 2: probabilities, coins and L_H from the per-edge squares summed over all columns.  With
        device_out, L_H stays in the context (nnz, colptr, rowidx, values device pointers, valid until the
        context's next call), as sparsify_device returns it."""
        g = graph._struct()
        out = _CscOut()
        st = _Stats()
        _check(lib().ssp_shard_finish(self._h, ctypes.byref(g), ctypes.byref(params._s), sq_total_ptr,
                                      SSP_MEM_DEVICE if device_out else SSP_MEM_HOST, ctypes.byref(out),
                                      ctypes.byref(st)))
        if device_out:
            return (out.nnz, out.colptr, out.rowidx, out.values), _stats_dict(st)
        return _take_out(out), _stats_dict(st)

    def solve_lap(self, lap, Y, tol=0.0, abs_tol=np.sqrt(2e-7), max_iters=400, factor_seed=0,
                  dense_threshold=4096, max_degree=-1, raise_on_failure=True, precision=0, verbose=False):
        Y = np.ascontiguousarray(Y, np.float64)
        n, k = Y.shape
        Z = np.zeros_like(Y)
        o = _SolveOpts(tol, abs_tol, max_iters, factor_seed, dense_threshold, int(verbose), max_degree, precision)
        rep = _SolveReport()
        s = lap._struct()
        rc = lib().ssp_solve_lap(self._h, ctypes.byref(s), _ptr(Y), k, _ptr(Z), SSP_MEM_HOST, ctypes.byref(o),
                                 ctypes.byref(rep))
        if rc != SSP_OK and (raise_on_failure or rc != -4):
            _check(rc)
        return Z, {f: getattr(rep, f) for f, _ in _SolveReport._fields_}


_DEFAULT_CTX = None


def _ctx():
    global _DEFAULT_CTX
    if _DEFAULT_CTX is None:
        _DEFAULT_CTX = Context(0)
    return _DEFAULT_CTX


def solve_lap(lap, Y, **kw):
    return _ctx().solve_lap(lap, Y, **kw)


def run_solve_lap(shared_jl_cols, col_ptrs, row_indices, values, solver_output_filename, num_nodes, verbose):
    """Drop-in for ffi::run_solve_lap (lib.rs:103): FlattenedVec-like (vec, num_rows, num_cols) in,
    row-major solution out.  Raises SspError where the reference throws."""
    vec, num_rows, num_cols = shared_jl_cols
    vec = np.ascontiguousarray(vec, np.float64)
    cp = np.ascontiguousarray(col_ptrs, np.int32)
    ri = np.ascontiguousarray(row_indices, np.int32)
    va = np.ascontiguousarray(values, np.float64)
    sol = np.zeros(num_rows * num_cols, np.float64)
    _check(lib().ssp_run_solve_lap(_ptr(vec), num_rows, num_cols, _ptr(cp), len(cp), _ptr(ri), _ptr(va), len(va),
                                   (solver_output_filename or "").encode(), num_nodes, int(verbose), _ptr(sol)))
    return sol, num_rows, num_cols


class Sparsifier:
    """Sparsifier (sparsifier.rs:244-297, 357-376, 735-790): a current Laplacian plus the edges inserted since
    the last sparsification.  Built from a graph (all its edges pending), from a vertex count (empty), or with
    from_matrix from a Laplacian file (the current Laplacian, nothing pending).

    insert() skips zero values and checks the reference's streaming trigger: with params.streaming set, it
    sparsifies when the current Laplacian has more than threshold = n * round(beta) * row_constant edges
    (sparsifier.rs:266,370-374; as there, the count is of the current Laplacian, not of the pending edges).
    sparsify() adds the pending edges and runs the GPU path; the JL sketch covers the pending edges only."""

    def __init__(self, graph, parameters, ctx=None):
        self.params = parameters
        self._ctx = ctx  # the device context is taken on first use, so building one needs no GPU
        self.stats = None
        if isinstance(graph, (int, np.integer)):
            self.num_nodes = int(graph)
            self._rows, self._cols, self._vals = [], [], []
        else:
            self.num_nodes = graph.n
            A = graph.to_scipy().tocoo()
            up = A.row < A.col
            self._rows, self._cols, self._vals = list(A.row[up]), list(A.col[up]), list(A.data[up])
        beta = parameters.beta(self.num_nodes)
        # f64::round rounds half away from zero (sparsifier.rs:266)
        self.threshold = self.num_nodes * int(math.floor(beta + 0.5)) * parameters.row_constant
        self.current_laplacian = None

    @classmethod
    def from_matrix(cls, filename, parameters, ctx=None):
        """Sparsifier::from_matrix (sparsifier.rs:299-335): the current Laplacian read from a .mtx file, no
        edges pending, the same threshold."""
        lap = read_mtx(filename)
        sp = cls(lap.n, parameters, ctx)
        sp.current_laplacian = lap
        return sp

    @property
    def ctx(self):
        if self._ctx is None:
            self._ctx = _ctx()
        return self._ctx

    @property
    def graph(self):
        return self._pending_csc()

    def laplacian_edges(self):
        """(row, col, value) of the current Laplacian's entries with row < col in CSC order: the edges, in the
        order compute_diff_norms and compute_probs walk them (sparsifier.rs:546-547,571-572)."""
        L = self.current_laplacian
        cols = np.repeat(np.arange(L.n, dtype=np.int32), np.diff(L.colptr))
        up = L.rowidx < cols
        return np.ascontiguousarray(L.rowidx[up], np.int32), np.ascontiguousarray(cols[up]), L.values[up]

    def compute_diff_norms(self, solution):
        """Per edge of the current Laplacian, ||X[row] - X[col]|| over the columns of the n x k solution
        (compute_diff_norms, sparsifier.rs:565-583).  On the GPU; the squares are summed per 32-column tile
        and the tiles in order, where the reference adds the columns one by one."""
        v1, v2, _ = self.laplacian_edges()
        return stage_diff_norms(self.ctx, v1, v2, solution)

    def compute_probs(self, diff_norms):
        """Per edge, min(1, beta * (-value) * d^2 / jl_dim) (compute_probs, sparsifier.rs:542-562), with
        beta and jl_dim of this Sparsifier's vertex count.  On the GPU."""
        _, _, val = self.laplacian_edges()
        n = self.num_nodes
        return stage_probs(self.ctx, -val, diff_norms, self.params.beta(n), float(self.params.jl_dim(n)))

    def insert(self, v1, v2, value):
        if not (0 <= v1 < self.num_nodes and 0 <= v2 < self.num_nodes):
            raise SspError(-1, "vertex id out of range")
        if value != 0.0 and v1 != v2:
            a, b = (v1, v2) if v1 < v2 else (v2, v1)
            self._rows.append(a)
            self._cols.append(b)
            self._vals.append(float(value))
        if self.params.streaming and (self.num_edges() or 0) > self.threshold:
            self.sparsify()

    def _pending_csc(self):
        import scipy.sparse as sp
        n = self.num_nodes
        U = sp.coo_matrix((np.asarray(self._vals, np.float64), (np.asarray(self._rows, np.int64),
                                                                 np.asarray(self._cols, np.int64))), shape=(n, n))
        A = (U + U.T).tocsc()  # duplicates summed, as Triplet::to_csc
        A.sum_duplicates()
        A.sort_indices()
        return CSC.from_scipy(A)

    def sparsify(self):
        new = self._pending_csc()
        if self.current_laplacian is None:
            self.current_laplacian, st = self.ctx.sparsify(new, self.params)
        else:
            self.current_laplacian, st = self.ctx.sparsify_update(self.current_laplacian, new, self.params)
        self._rows, self._cols, self._vals = [], [], []
        self.stats = SparsificationStats(st)
        return self.stats

    def num_edges(self):
        return self.current_laplacian.num_edges() if self.current_laplacian is not None else None


class InputStream:
    """Reads a .mtx file (InputStream::new, stream.rs:18-37)."""

    def __init__(self, filename, dataset_name=""):
        self.input_matrix = read_mtx(filename)
        self.num_nodes = self.input_matrix.n
        self.dataset_name = dataset_name

    def run_stream(self, parameters, test=False, writeout=False):
        sp = Sparsifier(self.input_matrix, parameters)
        stats = sp.sparsify()
        if writeout and not test and parameters.output_file:
            write_mtx(parameters.output_file, sp.current_laplacian)
        return sp, stats


def sparsify_dataset(input_filename, dataset_name, output_filename, epsilon, verbose, sketch_seed, sampling_seed,
                     benchmark):
    """sparsify_dataset (lib.rs:145-166)."""
    p = SparsifierParameters.cli(epsilon, verbose, sketch_seed, sampling_seed, benchmark, output_filename)
    st = _Stats()
    _check(lib().ssp_sparsify_mtx(input_filename.encode(), (output_filename or "").encode(), ctypes.byref(p._s),
                                  ctypes.byref(st)))
    return SparsificationStats(_stats_dict(st))


# ---------------------------------------------------------------- stage entry points (parity tests)
def stage_graph(ctx, graph):
    """Edges (v1, v2, w) and L_G as built on the device."""
    m, lnnz = I64(), I64()
    g = graph._struct()
    _check(lib().ssp_stage_graph(ctx._h, ctypes.byref(g), ctypes.byref(m), ctypes.byref(lnnz), None, None, None,
                                 None, None, None))
    mm, nn = m.value, lnnz.value
    v1 = np.zeros(max(mm, 1), np.int32); v2 = np.zeros(max(mm, 1), np.int32); w = np.zeros(max(mm, 1), np.float64)
    cp = np.zeros(graph.n + 1, np.int64); ri = np.zeros(max(nn, 1), np.int32); va = np.zeros(max(nn, 1), np.float64)
    _check(lib().ssp_stage_graph(ctx._h, ctypes.byref(g), ctypes.byref(m), ctypes.byref(lnnz), _ptr(v1), _ptr(v2),
                                 _ptr(w), _ptr(cp), _ptr(ri), _ptr(va)))
    return (v1[:mm], v2[:mm], w[:mm]), CSC(graph.n, cp, ri[:nn], va[:nn])


def stage_sketch(ctx, n, v1, v2, w, k, scale, seed, uniform=False):
    v1 = np.ascontiguousarray(v1, np.int32); v2 = np.ascontiguousarray(v2, np.int32)
    w = np.ascontiguousarray(w, np.float64)
    Y = np.zeros((n, k), np.float64)
    _check(lib().ssp_stage_sketch(ctx._h, n, len(v1), _ptr(v1), _ptr(v2), _ptr(w), SSP_MEM_HOST, k, scale, seed,
                                  int(uniform), _ptr(Y)))
    return Y


def stage_factor(ctx, lap, seed, dense_threshold=4096, max_degree=0):
    s = lap._struct()
    nnz = I64()
    nl = I32()
    _check(lib().ssp_stage_factor(ctx._h, ctypes.byref(s), seed, dense_threshold, max_degree, ctypes.byref(nnz),
                                  None, None, None, None, None, ctypes.byref(nl)))
    n = lap.n
    cp = np.zeros(n + 1, np.int64); rows = np.zeros(max(nnz.value, 1), np.int32)
    vals = np.zeros(max(nnz.value, 1), np.float64); D = np.zeros(n, np.float64); lvl = np.zeros(n, np.int32)
    _check(lib().ssp_stage_factor(ctx._h, ctypes.byref(s), seed, dense_threshold, max_degree, ctypes.byref(nnz),
                                  _ptr(cp), _ptr(rows), _ptr(vals), _ptr(D), _ptr(lvl), ctypes.byref(nl)))
    return {"colptr": cp, "rows": rows[:nnz.value], "vals": vals[:nnz.value], "D": D, "level": lvl,
            "num_levels": nl.value}


def stage_precond(ctx, lap, seed, R, dense_threshold=4096, max_degree=0):
    R = np.ascontiguousarray(R, np.float64)
    if R.ndim == 1:
        R = R[:, None]
    Z = np.zeros_like(R)
    s = lap._struct()
    _check(lib().ssp_stage_precond(ctx._h, ctypes.byref(s), seed, dense_threshold, max_degree, _ptr(R), R.shape[1],
                                   _ptr(Z)))
    return Z


def stage_diff_norms(ctx, v1, v2, Z):
    Z = np.ascontiguousarray(Z, np.float64)
    v1 = np.ascontiguousarray(v1, np.int32); v2 = np.ascontiguousarray(v2, np.int32)
    d = np.zeros(len(v1), np.float64)
    _check(lib().ssp_stage_diff_norms(ctx._h, Z.shape[0], len(v1), _ptr(v1), _ptr(v2), _ptr(Z), Z.shape[1],
                                      SSP_MEM_HOST, _ptr(d)))
    return d


def stage_probs(ctx, w, d, beta, denom):
    w = np.ascontiguousarray(w, np.float64); d = np.ascontiguousarray(d, np.float64)
    p = np.zeros_like(w)
    _check(lib().ssp_stage_probs(ctx._h, len(w), _ptr(w), _ptr(d), beta, denom, SSP_MEM_HOST, _ptr(p)))
    return p


def stage_scan(ctx, a):
    a = np.ascontiguousarray(a, np.int32)
    out = np.zeros(len(a) + 1, np.int64)
    _check(lib().ssp_stage_scan(ctx._h, _ptr(a), len(a), _ptr(out)))
    return out


def stage_coins(ctx, m, seed):
    c = np.zeros(m, np.float64)
    _check(lib().ssp_stage_coins(ctx._h, m, seed, SSP_MEM_HOST, _ptr(c)))
    return c


def stage_sample_apply(ctx, graph, p, coins, reweight):
    p = np.ascontiguousarray(p, np.float64); coins = np.ascontiguousarray(coins, np.float64)
    keep = np.zeros(max(len(p), 1), np.uint8)
    out = _CscOut()
    g = graph._struct()
    _check(lib().ssp_stage_sample_apply(ctx._h, ctypes.byref(g), _ptr(p), _ptr(coins), int(reweight), SSP_MEM_HOST,
                                        _ptr(keep), ctypes.byref(out)))
    return _take_out(out), keep[:len(p)].astype(bool)


# ---------------------------------------------------------------- serving
SSP_ERR_PENDING = -8


def request_footprint(graph, params):
    """Estimated device bytes of one sparsification (what the server admits against its HBM budget)."""
    g = graph._struct()
    return lib().ssp_request_footprint(ctypes.byref(g), ctypes.byref(params._s))


class Server:
    """Persistent request loop on one device (ssp_server_*): submit from any thread, collect with wait/poll."""

    def __init__(self, device=0, slots=4, hbm_budget_bytes=0, max_pending=0, max_batch=32):
        """max_batch: requests that may share one run (ssp_sparsify_batch); 1 runs every request alone."""
        o = _ServerOpts(device, slots, hbm_budget_bytes, max_pending, max_batch)
        h = P()
        _check(lib().ssp_server_create(ctypes.byref(o), ctypes.byref(h)))
        self._h = h

    def submit(self, graph, params, check_probes=0):
        """Queue one sparsification; check_probes > 0 also checks the result on the device (a15)."""
        req = _Request(0, graph._struct(), params._s, check_probes)
        t = U64(0)
        _check(lib().ssp_submit(self._h, ctypes.byref(req), ctypes.byref(t)))
        return t.value

    def _collect(self, res):
        info = {"queue_ms": res.queue_ms, "run_ms": res.run_ms, "latency_ms": res.latency_ms, "slot": res.slot,
                "est_bytes": res.est_bytes, "batch": res.batch}
        if res.checked:
            info["check"] = {"upper_bound_violations": res.probe_upper_violations,
                             "lower_bound_violations": res.probe_lower_violations,
                             "mean_relative_error": res.probe_mean_relative_error,
                             "max_relative_error": res.probe_max_relative_error,
                             "components_graph": res.components_graph,
                             "components_sparsifier": res.components_sparsifier,
                             "ccs_equal": res.components_graph == res.components_sparsifier,
                             "check_ms": res.check_ms}
        if res.status != SSP_OK:
            raise SspError(res.status, res.error.decode(errors="replace"))
        return _take_out(res.out), _stats_dict(res.stats), info

    def wait(self, ticket, timeout_ms=-1):
        """(L_H, stats, timing) of a finished request; None if timeout_ms passes first."""
        res = _Result()
        rc = lib().ssp_wait(self._h, ticket, timeout_ms, ctypes.byref(res))
        if rc == SSP_ERR_PENDING:
            return None
        _check(rc)
        return self._collect(res)

    def poll(self, ticket):
        return self.wait(ticket, 0)

    def info(self):
        i = _ServerInfo()
        _check(lib().ssp_server_info_get(self._h, ctypes.byref(i)))
        return {f: getattr(i, f) for f, _ in _ServerInfo._fields_}

    def close(self):
        if getattr(self, "_h", None):
            lib().ssp_server_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
