"""Runs the reference's own CPU Laplacian solver (src/example.cc factorization_driver + include/custom_cg.hpp,
built into oracle/_ref/ref_solve by oracle/ref/Makefile) as a subprocess.

Test infrastructure only: tests/ and bench.py's reference/CPU legs use it to check the oracle and to time
the reference's CPU path.  It is a separate process because the reference asserts and throws on failure.
"""
import os
import struct
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
BIN = os.path.join(HERE, "_ref", "ref_solve")


def available():
    return os.path.exists(BIN) and os.access(BIN, os.X_OK)


def build(ref_root=None):
    """Compile ref_solve from the reference sources at ref_root (default: $SSP_REFERENCE_DIR) when they are
    present; without them (a machine that only has the prebuilt binary) nothing is compiled."""
    ref_root = ref_root or os.environ.get("SSP_REFERENCE_DIR")
    if not ref_root or not os.path.exists(os.path.join(ref_root, "src", "example.cc")):
        return available()
    r = subprocess.run(["make", "-s", f"REF={ref_root}"], cwd=os.path.join(HERE, "ref"), capture_output=True,
                       text=True)
    if r.returncode != 0:
        raise RuntimeError("building the reference solver failed:\n" + r.stdout + r.stderr)
    return available()


def solve(n, colptr, rowidx, values, rhs, threads=1, verbose=False, timeout=600, timings=False):
    """Solve L x_j = b_j for the columns of rhs (n x k) with the reference solver.

    Returns (status, seconds, X): status 0 = every column converged (relative residual < 0.01,
    custom_cg.hpp:256), 1 = the driver returned false, 2 = it threw (example.cc:566); seconds covers the
    solver's set-up (elimination tree), factorization and all solves.  With timings=True a fourth item
    holds, per right-hand side, the seconds from the start to the beginning of its PCG solve: the first one
    is the set-up + factorization time, the differences are the per-column solve times.
    """
    rhs = np.asarray(rhs, np.float64)
    if rhs.ndim == 1:
        rhs = rhs[:, None]
    k = rhs.shape[1]
    colptr = np.ascontiguousarray(colptr, np.int32)
    rowidx = np.ascontiguousarray(rowidx, np.int32)
    values = np.ascontiguousarray(values, np.float64)
    with tempfile.TemporaryDirectory() as d:
        fin, fout = os.path.join(d, "in.bin"), os.path.join(d, "out.bin")
        with open(fin, "wb") as f:
            f.write(b"SSPR" + struct.pack("<4iq", n, k, threads, int(verbose), len(values)))
            f.write(colptr.tobytes())
            f.write(rowidx.tobytes())
            f.write(values.tobytes())
            f.write(np.ascontiguousarray(rhs.T).tobytes())
        env = dict(os.environ, OMP_NUM_THREADS=str(threads))
        r = subprocess.run([BIN, fin, fout], capture_output=True, text=True, timeout=timeout, env=env)
        if r.returncode != 0:
            raise RuntimeError(f"ref_solve exited {r.returncode}: {r.stderr[-2000:]}")
        raw = open(fout, "rb").read()
    status, secs, ns = struct.unpack_from("<idi", raw, 0)
    starts = np.frombuffer(raw, np.float64, count=ns, offset=16).copy()
    off = 16 + 8 * ns
    X = np.frombuffer(raw, np.float64, count=k * n, offset=off).reshape(k, n).T.copy()
    if timings:
        return status, secs, X, starts
    return status, secs, X
