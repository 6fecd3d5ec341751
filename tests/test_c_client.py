"""The C ABI from plain C (tests/c_client/sparsify_file.c, compiled here against include/specspars.h and
linked to libspecspars.so): the calls a Rust or other FFI caller makes, with no Python in between.  Without a
device the client must get the library's clean SSP_ERR_NO_DEVICE after the host-only calls succeed; on a B200
its output file must be byte-identical to the Python host's result for the same graph."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "c_client", "sparsify_file.c")
LIBDIR = os.path.join(ROOT, "spec_spars_b200")


@pytest.fixture(scope="module")
def client(ssp, tmp_path_factory):
    if shutil.which("gcc") is None:
        pytest.skip("needs a C compiler")
    exe = tmp_path_factory.mktemp("c_client") / "sparsify_file"
    subprocess.run(["gcc", "-std=c11", "-O1", "-I", os.path.join(ROOT, "include"), SRC, "-o", str(exe),
                    "-L", LIBDIR, "-lspecspars", f"-Wl,-rpath,{LIBDIR}"], check=True, capture_output=True)
    return str(exe)


def _graph_file(ssp, tmp_path):
    G = ssp.gen_grid2d(30, 30)
    path = tmp_path / "grid.mtx"
    ssp.write_mtx(str(path), G)
    return G, path


def test_c_client_without_device(ssp, client, tmp_path):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a device is visible")
    G, path = _graph_file(ssp, tmp_path)
    r = subprocess.run([client, str(path), str(tmp_path / "out.mtx")], capture_output=True, text=True)
    assert r.returncode == 3, r.stdout + r.stderr
    k = ssp.SparsifierParameters.cli(0.5).jl_dim(G.n)
    assert f"n {G.n} nnz {G.nnz} jl_dim {k}" in r.stdout and "no CUDA device" in r.stdout


def _shared_compute_mode():
    """The client runs in its own process beside this one's context: only in the default compute mode."""
    try:
        r = subprocess.run(["nvidia-smi", "--id=0", "--query-gpu=compute_mode", "--format=csv,noheader"],
                           capture_output=True, text=True, timeout=30)
    except (OSError, subprocess.TimeoutExpired):
        return False
    return r.returncode == 0 and r.stdout.strip().lower() == "default"


@pytest.mark.gpu
def test_c_client_output_equals_python_host(ssp, ctx, client, tmp_path):
    if not _shared_compute_mode():
        pytest.skip("the GPU is not in the default (shared) compute mode")
    G, path = _graph_file(ssp, tmp_path)
    out = tmp_path / "out.mtx"
    r = subprocess.run([client, str(path), str(out)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    H, st = ctx.sparsify(ssp.read_mtx(str(path)), ssp.SparsifierParameters.cli(0.5))
    ref = tmp_path / "ref.mtx"
    ssp.write_mtx(str(ref), H)
    assert out.read_bytes() == ref.read_bytes()
    assert f"m_in {st['m_in']} m_out {st['m_out']}" in r.stdout
