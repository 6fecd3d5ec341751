"""The edge-list converter on the GPU (ssp_edgelist_to_mtx_device) against the host converter
(ssp_edgelist_to_mtx), both restating edge_list_to_matrix_market (utils.rs:413-526): the output files must be
equal byte for byte, and a file the device parser leaves to the host must give the host's result or error."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _convert_both(ssp, ctx, tmp_path, text, default_weight=1.5):
    src = tmp_path / "in.txt"
    src.write_bytes(text.encode() if isinstance(text, str) else text)
    dh, dd = tmp_path / "host.mtx", tmp_path / "dev.mtx"
    eh = ed = None
    on_device = None
    try:
        ssp.edge_list_to_matrix_market(src, dh, default_weight)
    except ssp.SspError as e:
        eh = (e.code, str(e))
    try:
        on_device = ssp.edge_list_to_matrix_market(src, dd, default_weight, ctx=ctx)
    except ssp.SspError as e:
        ed = (e.code, str(e))
    assert eh == ed
    if eh is None:
        assert dd.read_bytes() == dh.read_bytes()
        return dd.read_text(), on_device
    return None, on_device


def _random_list(rng, n, m, weights):
    lines = [f"{n} {m}"]
    u = rng.integers(0, n, size=m)
    v = rng.integers(0, n, size=m)
    for k in range(m):
        sep = rng.choice([" ", "\t", "  ", " \t "])
        ln = f"{u[k]}{sep}{v[k]}"
        r = rng.random()
        weighted = weights is not None and r < 0.8
        if weighted:
            w = weights(rng)
            ln += f"{rng.choice([' ', chr(9)])}{w}"
        if rng.random() < 0.05:
            # text after the weight is ignored; after the endpoints it would be read as the weight
            ln += rng.choice([" ", "\r", " trailing text"] if weighted else [" ", "\r"])
        lines.append(ln)
        if rng.random() < 0.02:
            lines.append(rng.choice(["", "   ", "\t"]))
    return "\n".join(lines) + ("\n" if rng.random() < 0.5 else "")


def _weight(rng):
    k = rng.integers(0, 6)
    if k == 0:
        return repr(float(rng.uniform(0.1, 10.0)))
    if k == 1:
        return f"{rng.uniform(0, 1000):.{int(rng.integers(0, 6))}f}"
    if k == 2:
        return f"{rng.uniform(1, 9):.3f}e{int(rng.integers(-12, 12))}"
    if k == 3:
        return str(int(rng.integers(1, 100)))
    if k == 4:
        return repr(float(np.exp(rng.normal(0, 3))))
    return "0." + "".join(str(d) for d in rng.integers(0, 10, size=25))  # beyond 19 digits: strtod on the host


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_random_lists_equal_host_bytes(ssp, ctx, tmp_path, seed):
    rng = np.random.default_rng(seed)
    text = _random_list(rng, 500, 20000, _weight)
    out, on_device = _convert_both(ssp, ctx, tmp_path, text)
    assert out is not None and out.count("\n") > 1000 and on_device


def test_large_list_with_duplicates(ssp, ctx, tmp_path):
    rng = np.random.default_rng(7)
    n, m = 200_000, 2_000_000
    u = rng.integers(0, n, size=m)
    v = rng.integers(0, n, size=m)
    w = rng.uniform(0.5, 2.0, size=m)
    body = "\n".join(f"{a} {b} {float(c)!r}" for a, b, c in zip(u, v, w))
    out, on_device = _convert_both(ssp, ctx, tmp_path, f"{n} {m}\n" + body + "\n")
    assert out is not None and on_device


# (text, written by the GPU)
@pytest.mark.parametrize("text,dev", [
    ("3 2\n0 1 2.5\n1 2\n", True),                       # default weight
    ("3 2\r\n0 1 2.5\r\n1 2\r\n", True),                 # CRLF
    ("3 1\n0 1 2.5", True),                              # no final newline
    ("3 0\n", True),                                     # no edges
    ("3 0", True),                                       # header only, no newline
    ("4 2\n0 1 0x1p3\n2 3 1e-5\n", True),                 # hex: strtod on the host for that weight
    ("4 1\n0 1 2.5abc\n", True),                         # strtod reads the prefix
    ("4 3\n0 1 inf\n1 2 nan\n2 3 -0.0\n", False),         # host text for inf / NaN
    ("4 2\n+0 1 2.0\n2 3 1.0\n", False),                  # a sign
    ("4 2\n0 1 2.5\n2 3x 1.0\n", None),                   # text glued to an endpoint: the host's error
    ("4 2\n0 1 2.5\n2\n", None),                          # missing endpoint: the host's error
    ("4 1\n0 1 abc\n", None),                            # bad weight: the host's error
    ("", None),                                          # empty file: the host's error
    ("x y\n0 1\n", None),                                # bad header: the host's error
    ("5 1\n4294967296 1 2.0\n", False),                   # endpoint >= 2^32
    ("3 2\n0 1 1e-30\n1 2 1e300\n", False),               # weights whose text the device leaves to the host
])
def test_edge_cases_match_host(ssp, ctx, tmp_path, text, dev):
    out, on_device = _convert_both(ssp, ctx, tmp_path, text)
    if dev is None:
        assert out is None
    else:
        assert out is not None and on_device == dev
