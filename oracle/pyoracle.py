"""ctypes front end of the CPU oracle (oracle/ssp_oracle.c).

Test infrastructure only: imported by tests/, __graft_entry__.smoke() and the
cpu_baseline leg of bench.py, as the checker.  The product library never
loads it.
"""
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
i64p = np.ctypeslib.ndpointer(np.int64, flags="C_CONTIGUOUS")
f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
u8p = np.ctypeslib.ndpointer(np.uint8, flags="C_CONTIGUOUS")
u64p = np.ctypeslib.ndpointer(np.uint64, flags="C_CONTIGUOUS")


def build():
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


class _Factor(ctypes.Structure):
    _fields_ = [("n", ctypes.c_int64), ("nnz", ctypes.c_int64),
                ("colstart", ctypes.c_void_p), ("rows", ctypes.c_void_p), ("vals", ctypes.c_void_p),
                ("D", ctypes.c_void_p), ("level", ctypes.c_void_p), ("order", ctypes.c_void_p),
                ("num_levels", ctypes.c_int32), ("dense_start", ctypes.c_int32)]


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "libssp_oracle.so")
        if not os.path.exists(path):
            build()
        L = ctypes.CDLL(path)
        L.ora_philox4x64.argtypes = [u64p, ctypes.c_uint64, ctypes.c_uint64, u64p]
        L.ora_sketch_entry.argtypes = [ctypes.c_uint64, ctypes.c_int, ctypes.c_int64, ctypes.c_int64]
        L.ora_sketch_entry.restype = ctypes.c_double
        L.ora_coin.argtypes = [ctypes.c_uint64, ctypes.c_int64]
        L.ora_coin.restype = ctypes.c_double
        L.ora_priority.argtypes = [ctypes.c_uint64, ctypes.c_int64]
        L.ora_priority.restype = ctypes.c_uint64
        L.ora_factor_uniform.argtypes = [ctypes.c_uint64, ctypes.c_int64, ctypes.c_int64]
        L.ora_factor_uniform.restype = ctypes.c_double
        L.ora_extract_edges.argtypes = [ctypes.c_int64, i64p, i32p, f64p,
                                        ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
        L.ora_extract_edges.restype = ctypes.c_int64
        L.ora_laplacian_nnz.argtypes = [ctypes.c_int64, ctypes.c_int64, i32p, i32p, f64p]
        L.ora_laplacian_nnz.restype = ctypes.c_int64
        L.ora_laplacian.argtypes = [ctypes.c_int64, ctypes.c_int64, i32p, i32p, f64p, i64p, i32p, f64p]
        L.ora_sketch.argtypes = [ctypes.c_int64, ctypes.c_int64, i32p, i32p, f64p, ctypes.c_int32,
                                 ctypes.c_double, ctypes.c_uint64, ctypes.c_int, f64p]
        L.ora_factor.argtypes = [ctypes.c_int64, i64p, i32p, f64p, ctypes.c_uint64, ctypes.c_int64,
                                 ctypes.c_int64, ctypes.POINTER(_Factor)]
        L.ora_factor.restype = ctypes.c_int
        L.ora_factor_free.argtypes = [ctypes.POINTER(_Factor)]
        L.ora_factor_export.argtypes = [ctypes.POINTER(_Factor), i64p, i32p, f64p, f64p, i32p, i32p]
        L.ora_precond.argtypes = [ctypes.POINTER(_Factor), f64p, f64p]
        L.ora_pcg.argtypes = [ctypes.c_int64, i64p, i32p, f64p, ctypes.POINTER(_Factor), f64p,
                              ctypes.c_int32, ctypes.c_double, ctypes.c_double, ctypes.c_int32,
                              f64p, i32p, f64p]
        L.ora_pcg.restype = ctypes.c_int
        L.ora_diff_norms.argtypes = [ctypes.c_int64, ctypes.c_int64, i32p, i32p, f64p, ctypes.c_int32,
                                     ctypes.c_int64, f64p]
        L.ora_probs.argtypes = [ctypes.c_int64, f64p, f64p, ctypes.c_double, ctypes.c_double, f64p]
        L.ora_sample_apply.argtypes = [ctypes.c_int64, ctypes.c_int64, i32p, i32p, f64p, f64p, f64p,
                                       ctypes.c_int, i64p, i32p, f64p,
                                       ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
        L.ora_sample_apply.restype = ctypes.c_int64
        L.ora_gen_er.argtypes = [ctypes.c_int64, ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_uint64,
                                 ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64]
        L.ora_gen_er.restype = ctypes.c_int64
        _LIB = L
    return _LIB


def philox4x64(ctr, key0, key1):
    c = np.ascontiguousarray(ctr, dtype=np.uint64)
    out = np.zeros(4, np.uint64)
    lib().ora_philox4x64(c, key0, key1, out)
    return out


def sketch_entry(seed, uniform, e, j):
    return lib().ora_sketch_entry(seed, int(uniform), e, j)


def coin(seed, e):
    return lib().ora_coin(seed, e)


def coins(seed, m):
    L = lib()
    return np.array([L.ora_coin(seed, e) for e in range(m)], dtype=np.float64)


def priority(seed, v):
    return lib().ora_priority(seed, v)


def extract_edges(n, colptr, rowidx, val):
    colptr = np.ascontiguousarray(colptr, np.int64)
    rowidx = np.ascontiguousarray(rowidx, np.int32)
    val = np.ascontiguousarray(val, np.float64)
    m = lib().ora_extract_edges(n, colptr, rowidx, val, None, None, None)
    if m < 0:
        raise ValueError(f"oracle edge extraction failed ({m})")
    v1 = np.zeros(m, np.int32); v2 = np.zeros(m, np.int32); w = np.zeros(m, np.float64)
    lib().ora_extract_edges(n, colptr, rowidx, val, v1.ctypes.data, v2.ctypes.data, w.ctypes.data)
    return v1, v2, w


def gen_er(n, avg_degree, wlo, whi, seed):
    """Edges (v1 < v2, CSC-upper order) and weights of the synthetic ER graph the library's gen_er builds."""
    m = lib().ora_gen_er(n, avg_degree, wlo, whi, seed, None, None, None, 0)
    v1 = np.zeros(m, np.int32); v2 = np.zeros(m, np.int32); w = np.zeros(m, np.float64)
    if lib().ora_gen_er(n, avg_degree, wlo, whi, seed, v1.ctypes.data, v2.ctypes.data, w.ctypes.data, m) != m:
        raise RuntimeError("oracle ER generator: edge count changed between passes")
    return v1, v2, w


def laplacian(n, v1, v2, w):
    v1 = np.ascontiguousarray(v1, np.int32); v2 = np.ascontiguousarray(v2, np.int32)
    w = np.ascontiguousarray(w, np.float64)
    m = len(v1)
    nnz = lib().ora_laplacian_nnz(n, m, v1, v2, w)
    cp = np.zeros(n + 1, np.int64); ri = np.zeros(max(nnz, 1), np.int32); va = np.zeros(max(nnz, 1), np.float64)
    lib().ora_laplacian(n, m, v1, v2, w, cp, ri, va)
    return cp, ri[:nnz], va[:nnz]


def sketch(n, v1, v2, w, k, scale, seed, uniform=False):
    v1 = np.ascontiguousarray(v1, np.int32); v2 = np.ascontiguousarray(v2, np.int32)
    w = np.ascontiguousarray(w, np.float64)
    Y = np.zeros((n, k), np.float64)
    lib().ora_sketch(n, len(v1), v1, v2, w, k, scale, seed, int(uniform), Y)
    return Y


class Factor:
    """L (strictly lower, columns = vertex ids), D, levels and elimination order."""

    def __init__(self, n, colptr, rowidx, val, seed, dense_threshold=0, max_degree=0):
        self._f = _Factor()
        colptr = np.ascontiguousarray(colptr, np.int64)
        rowidx = np.ascontiguousarray(rowidx, np.int32)
        val = np.ascontiguousarray(val, np.float64)
        rc = lib().ora_factor(n, colptr, rowidx, val, seed, dense_threshold, max_degree, ctypes.byref(self._f))
        if rc != 0:
            raise RuntimeError("oracle factorization failed")
        nnz = self._f.nnz
        self.n = n
        self.colstart = np.zeros(n + 1, np.int64)
        self.rows = np.zeros(max(nnz, 1), np.int32)
        self.vals = np.zeros(max(nnz, 1), np.float64)
        self.D = np.zeros(n, np.float64)
        self.level = np.zeros(n, np.int32)
        self.order = np.zeros(n, np.int32)
        lib().ora_factor_export(ctypes.byref(self._f), self.colstart, self.rows, self.vals, self.D,
                                self.level, self.order)
        self.rows = self.rows[:nnz]; self.vals = self.vals[:nnz]
        self.num_levels = self._f.num_levels
        self.dense_start = self._f.dense_start

    def __del__(self):
        try:
            lib().ora_factor_free(ctypes.byref(self._f))
        except Exception:
            pass

    def precond(self, r):
        r = np.ascontiguousarray(r, np.float64)
        z = np.zeros_like(r)
        lib().ora_precond(ctypes.byref(self._f), r, z)
        return z

    def dense_L(self):
        n = self.n
        L = np.eye(n)
        for v in range(n):
            for p in range(self.colstart[v], self.colstart[v + 1]):
                L[self.rows[p], v] = self.vals[p]
        return L


def pcg(n, colptr, rowidx, val, factor, Y, tol, abs_tol, max_iters):
    Y = np.ascontiguousarray(Y, np.float64)
    k = Y.shape[1]
    Z = np.zeros_like(Y)
    iters = np.zeros(k, np.int32); rel = np.zeros(k, np.float64)
    rc = lib().ora_pcg(n, np.ascontiguousarray(colptr, np.int64), np.ascontiguousarray(rowidx, np.int32),
                       np.ascontiguousarray(val, np.float64), ctypes.byref(factor._f), Y, k, tol, abs_tol,
                       max_iters, Z, iters, rel)
    return Z, iters, rel, rc


def diff_norms(v1, v2, Z, k=None, ldz=None):
    Z = np.ascontiguousarray(Z, np.float64)
    n = Z.shape[0]
    if k is None:
        k = Z.shape[1]
    if ldz is None:
        ldz = Z.shape[1]
    m = len(v1)
    d = np.zeros(m, np.float64)
    lib().ora_diff_norms(n, m, np.ascontiguousarray(v1, np.int32), np.ascontiguousarray(v2, np.int32),
                         Z, k, ldz, d)
    return d


def probs(w, d, beta, denom):
    w = np.ascontiguousarray(w, np.float64); d = np.ascontiguousarray(d, np.float64)
    p = np.zeros_like(w)
    lib().ora_probs(len(w), w, d, beta, denom, p)
    return p


def sample_apply(n, v1, v2, w, p, coin_arr, reweight, lg):
    cp, ri, va = lg
    args = (n, len(v1), np.ascontiguousarray(v1, np.int32), np.ascontiguousarray(v2, np.int32),
            np.ascontiguousarray(w, np.float64), np.ascontiguousarray(p, np.float64),
            np.ascontiguousarray(coin_arr, np.float64), int(reweight),
            np.ascontiguousarray(cp, np.int64), np.ascontiguousarray(ri, np.int32),
            np.ascontiguousarray(va, np.float64))
    nnz = lib().ora_sample_apply(*args, None, None, None, None)
    hcp = np.zeros(n + 1, np.int64); hri = np.zeros(max(nnz, 1), np.int32)
    hva = np.zeros(max(nnz, 1), np.float64); keep = np.zeros(max(len(v1), 1), np.uint8)
    lib().ora_sample_apply(*args, hcp.ctypes.data, hri.ctypes.data, hva.ctypes.data, keep.ctypes.data)
    return (hcp, hri[:nnz], hva[:nnz]), keep[:len(v1)].astype(bool)
