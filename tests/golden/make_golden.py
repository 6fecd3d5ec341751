"""Writes the golden fixtures of tests/golden/: outputs of the reference's own Laplacian solver.

The solver is the reference's src/example.cc factorization_driver + include/custom_cg.hpp PCG, compiled from
the reference's sources into oracle/_ref/ref_solve (oracle/ref/Makefile, with the MKL protocol shim).  For
each case the fixture holds the solver's input (the Laplacian CSC, i32 pointers as in lib.rs:103, and the
n x k right-hand side), its status (0 converged, 2 threw "solver did not converge", example.cc:566) and what
the sparsifier consumes from the solution: the per-edge norms d_e = ||X[v1_e] - X[v2_e]|| over the k columns
(sparsifier.rs:565-583), computed here with numpy.

The reference's factorization draws from std::random_device, so a fixture records one run of it; a rerun
gives other bits but, both stopping at ||r|| <= sqrt(2e-7) (custom_cg.hpp:159,213), the same d_e to ~1e-4.

Run from the repository root on a machine that has the reference's sources and a C++ compiler:
    python tests/golden/make_golden.py [path-to-reference]
"""
import math
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import pyoracle as ora  # noqa: E402
import refsolver  # noqa: E402
import spec_spars_b200 as S  # noqa: E402

K = 8  # right-hand sides per case: the sketch's +-1/sqrt(k) Philox signs, seed 0

CASES = {
    "grid20": lambda: S.gen_grid2d(20, 20),
    "er800": lambda: S.gen_er(800, 8.0, 0.5, 2.0, 1),
    "grid3d_8x7x6": lambda: S.gen_grid3d(8, 7, 6, -3, 3, 2),  # weights over six decades
    "er400_isolated_vertex": lambda: S.gen_er(400, 5.0, 0.5, 2.0, 3),
    "rmat_s9": lambda: S.gen_rmat(9, 8, 0.57, 0.19, 0.19, 4),  # power law: hubs, LogNormal weights
    "rgg500": lambda: S.gen_rgg(500, 10.0, 0.1, 10.0, 6),  # random geometric: mesh-like, local
}


def edge_norms(v1, v2, X):
    d = X[v1] - X[v2]
    return np.sqrt((d * d).sum(axis=1))


def make(name, G):
    v1, v2, w = ora.extract_edges(G.n, G.colptr, G.rowidx, G.values)
    cp, ri, va = ora.laplacian(G.n, v1, v2, w)
    if name.endswith("isolated_vertex"):
        # a random zero-sum right-hand side: not in the range of a Laplacian with an isolated vertex
        assert np.any(np.diff(cp) == 0)
        Y = np.random.default_rng(0).standard_normal((G.n, 2))
        Y -= Y.mean(0)
    else:
        Y = ora.sketch(G.n, v1, v2, w, K, 1 / math.sqrt(K), 0)
    status, _, X = refsolver.solve(G.n, cp, ri, va, Y, threads=2)
    d = edge_norms(v1, v2, X) if status == 0 else np.zeros(0)
    np.savez_compressed(os.path.join(HERE, f"ref_solve_{name}.npz"), n=np.int64(G.n),
                        colptr=cp.astype(np.int32), rowidx=ri.astype(np.int32), values=va, rhs=Y,
                        v1=v1.astype(np.int32), v2=v2.astype(np.int32), w=w, status=np.int32(status), d=d)
    return status, len(w)


def main():
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("SSP_REFERENCE_DIR")
    if not ref:
        raise SystemExit("usage: make_golden.py <reference source tree>  (or set SSP_REFERENCE_DIR)")
    if not refsolver.build(ref):
        raise SystemExit("oracle/_ref/ref_solve could not be built: the reference's sources are needed")
    for name, gen in CASES.items():
        status, m = make(name, gen())
        print(f"{name}: status {status}, {m} edges")


if __name__ == "__main__":
    main()
