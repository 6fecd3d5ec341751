"""Matrix Market on the GPU (ssp_read_mtx_device / ssp_write_mtx_device) against the host reader and writer
(read_mtx / write_mtx, which restate utils::read_mtx / write_mtx): the same CSC bit for bit, the same bytes,
the same errors -- over symmetric, general, pattern and integer files, duplicates, comments, blank lines,
CRLF endings, every number form, and values the device hands to the host."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _same(a, b):
    return (a.n == b.n and np.array_equal(a.colptr, b.colptr) and np.array_equal(a.rowidx, b.rowidx)
            and np.array_equal(a.values.view(np.uint64), b.values.view(np.uint64)))


def _both(ssp, ctx, path):
    return ssp.read_mtx(str(path)), ctx.read_mtx(str(path))


def test_symmetric_file_with_duplicates_and_odd_tokens(ssp, ctx, tmp_path):
    lines = ["%%MatrixMarket matrix coordinate real symmetric", "% a comment", "%another", "6 6 14",
             "1 2 0.5", "2 1 .25", "1 2 1e-5",            # (0,1) summed in file order, mirrored too
             "3 3 +2", "4 3 1E+2", "5 4 -3.5e-3",
             "", "6 5 123456789012345678901234",          # more than 19 digits: strtod on the host
             "6 1 1e-320", "   2   6   7.000000000000000001  ",  # subnormal; trailing digits beyond 19
             "5 5 0", "6 6 1", "3 1 9007199254740993", "4 2 0.1", "2 2 5."]
    p = tmp_path / "a.mtx"
    p.write_text("\n".join(lines) + "\n")
    h, d = _both(ssp, ctx, p)
    assert _same(h, d) and h.n == 6


def test_general_pattern_integer_and_crlf(ssp, ctx, tmp_path):
    cases = {
        "gen.mtx": "%%MatrixMarket matrix coordinate real general\r\n3 3 4\r\n1 1 1.5\r\n3 1 2\r\n1 3 -2\r\n2 2 4e0\r\n",
        "pat.mtx": "%%MatrixMarket matrix coordinate pattern symmetric\n4 4 3\n2 1\n3 2\n4 3\n",
        "int.mtx": "%%MatrixMarket matrix coordinate integer general\n3 3 3\n1 2 7\n2 3 -4\n3 1 12\n\n\n",
    }
    for name, text in cases.items():
        p = tmp_path / name
        p.write_bytes(text.encode())
        h, d = _both(ssp, ctx, p)
        assert _same(h, d), name


@pytest.mark.parametrize("body,what", [
    ("1 2 0.5\n9 1 1.0\n", "row out of range"),
    ("1 2 0.5\n", "fewer entries than declared"),
    ("1 2 0.5\n% late comment\n2 3 1.0\n", "comment among the entries"),
    ("1 2 0.5 7\n2 3 1.0\n", "an extra token"),
    ("1 2\n0.5 2 3 1.0\n", "an entry split over lines"),
    ("1 2 x\n2 3 1.0\n", "a malformed value"),
])
def test_malformed_bodies_behave_as_the_host_reader(ssp, ctx, tmp_path, body, what):
    p = tmp_path / "bad.mtx"
    p.write_text("%%MatrixMarket matrix coordinate real general\n3 3 2\n" + body)
    try:
        h = ssp.read_mtx(str(p))
    except ssp.SspError as e:
        with pytest.raises(ssp.SspError) as e2:
            ctx.read_mtx(str(p))
        assert e2.value.code == e.code and str(e2.value) == str(e), what
        return
    assert _same(h, ctx.read_mtx(str(p))), what


@pytest.mark.parametrize("gen", ["er", "rmat"])
def test_large_round_trip(ssp, ctx, tmp_path, gen):
    G = ssp.gen_er(100_000, 12.0, 1e-3, 1e3, 7) if gen == "er" else ssp.gen_rmat(14, 16, 0.57, 0.19, 0.19, 2)
    p = tmp_path / "g.mtx"
    ssp.write_mtx(str(p), G)  # host writer
    h, d = _both(ssp, ctx, p)
    assert _same(h, d) and _same(h, G)
    q = tmp_path / "g_dev.mtx"
    ctx.write_mtx(str(q), G)  # device writer
    assert q.read_bytes() == p.read_bytes()


def test_writer_values_formatted_on_the_host(ssp, ctx, tmp_path):
    A = ssp.gen_grid2d(20, 20).to_scipy().tocsc()
    rng = np.random.default_rng(3)
    special = np.array([1e-25, 3e300, 5e-324, 1e-20, 9.87e38, 1.5e39, 2.0 ** -1074 * 7, 1 / 3])
    A.data = rng.uniform(0.1, 10.0, A.nnz)
    A.data[: len(special)] = special
    M = ssp.CSC.from_scipy(A)
    p, q = tmp_path / "h.mtx", tmp_path / "d.mtx"
    ssp.write_mtx(str(p), M)
    ctx.write_mtx(str(q), M)
    assert q.read_bytes() == p.read_bytes()
    assert _same(ssp.read_mtx(str(q)), ctx.read_mtx(str(q)))


def test_sparsify_dataset_file_unchanged(ssp, ctx, tmp_path):
    """ssp_sparsify_mtx reads and writes on the GPU: its output file has the host writer's bytes for the
    sparsifier the in-memory call returns."""
    G = ssp.gen_er(3000, 30.0, 0.5, 2.0, 9)
    src, out = tmp_path / "in.mtx", tmp_path / "out.mtx"
    ssp.write_mtx(str(src), G)
    ssp.sparsify_dataset(str(src), "er3000", str(out), 0.5, False, 0, 0, False)
    H, _ = ctx.sparsify(ssp.read_mtx(str(src)), ssp.SparsifierParameters.cli(0.5))
    ref = tmp_path / "ref.mtx"
    ssp.write_mtx(str(ref), H)
    assert out.read_bytes() == ref.read_bytes()
