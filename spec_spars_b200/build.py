"""Builds spec_spars_b200/libspecspars.so for sm_100a with nvcc (in-tree, no JIT cache).

Usage: python -m spec_spars_b200.build [-j N] [--force]
"""
import argparse
import concurrent.futures as cf
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libspecspars.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-O2",
          "--expt-relaxed-constexpr", "-Xptxas", "-O3"]
# Translation units whose results must be bit-identical to the CPU oracle: no FMA contraction.
EXACT = {"ssp_graph.cu", "ssp_sketch.cu", "ssp_factor.cu", "ssp_sample.cu", "ssp_noalloc.cu"}
SOURCES = ["ssp_util.cu", "ssp_graph.cu", "ssp_sketch.cu", "ssp_factor.cu", "ssp_pcg.cu", "ssp_sample.cu",
           "ssp_autotune.cu", "ssp_noalloc.cu", "ssp_quality.cu", "ssp_mtxio.cu", "ssp_api.cu", "ssp_host.cpp",
           "ssp_server.cpp"]
HEADERS = ["ssp_internal.cuh", "ssp_sort.cuh", "ssp_host.h", "ssp_decimal.cuh"]


def _nvcc():
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if c and (os.path.isabs(c) and os.path.exists(c) or not os.path.isabs(c)):
            return c
    return "nvcc"


def _newest_dep():
    paths = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(HERE, "..", "include", "specspars.h"),
                                                        os.path.abspath(__file__)]
    return max(os.path.getmtime(p) for p in paths if os.path.exists(p))


def _compile(src, force, verbose):
    obj = os.path.join(BUILD, src + ".o")
    s = os.path.join(CSRC, src)
    if not force and os.path.exists(obj) and os.path.getmtime(obj) >= max(os.path.getmtime(s), _newest_dep()):
        return obj, None
    cmd = [_nvcc()] + ARCH + COMMON
    if src in EXACT:
        cmd += ["-fmad=false"]
    if src.endswith(".cpp"):
        cmd += ["-x", "cu"]
    cmd += ["-c", s, "-o", obj]
    if verbose:
        cmd += ["-Xptxas", "-v"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        return obj, f"{' '.join(cmd)}\n{r.stdout}\n{r.stderr}"
    if verbose and r.stderr:
        sys.stderr.write(r.stderr)
    return obj, None


def build(jobs=8, force=False, verbose=False):
    os.makedirs(BUILD, exist_ok=True)
    with cf.ThreadPoolExecutor(max_workers=jobs) as ex:
        results = list(ex.map(lambda s: _compile(s, force, verbose), SOURCES))
    errs = [e for _, e in results if e]
    if errs:
        raise RuntimeError("nvcc failed:\n" + "\n".join(errs))
    objs = [o for o, _ in results]
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < max(os.path.getmtime(o) for o in objs):
        cmd = [_nvcc()] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("-j", type=int, default=8)
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-v", action="store_true")
    a = ap.parse_args()
    print(build(a.j, a.force, a.v))
