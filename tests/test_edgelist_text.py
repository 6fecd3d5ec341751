"""The weight text of edge_list_to_matrix_market (utils.rs:519): an f64 as Rust's Display writes it -- the
shortest digits that read back as the value, without an exponent, padded with zeros (2^70 prints as
1180591620717411300000, not its exact integer).  numpy's format_float_positional(unique=True) follows the same
rule and is the checker here.  Two implementations are checked: the device formatter of the GPU converter
(run on the host through ssp_format_shortest) and the host converter's text (through its output file)."""
import math

import numpy as np
import pytest


def _rust(v):
    if math.isnan(v):
        return "NaN"
    if math.isinf(v):
        return "inf" if v > 0 else "-inf"
    return np.format_float_positional(v, unique=True, trim="-")


def _samples(seed, count):
    rng = np.random.default_rng(seed)
    # random bit patterns over the formatter's range, short decimals, integers, and powers of two / ten
    bits = rng.integers(0, 2**63, size=count, dtype=np.int64).view(np.float64)
    bits = bits[np.isfinite(bits) & (np.abs(bits) > 1e-22) & (np.abs(bits) < 3e38)]
    dec = np.array([round(x, int(d)) for x, d in zip(rng.uniform(-1000, 1000, size=count),
                                                     rng.integers(0, 8, size=count))])
    ints = rng.integers(-10**17, 10**17, size=count).astype(np.float64)
    specials = [0.0, -0.0, 1.0, 0.1, 0.2, 0.3, 1e-7, 123456.789, 2.0**53, 2.0**53 + 2, 2.0**70, 1e21, 1e22,
                2.2250738585072014e-308, 1.7976931348623157e308, 9.999999999999999e22,
                0.30000000000000004, 2.5e15, 1e16, 12345678901234567890.0]
    specials += [2.0**k for k in range(-70, 127)] + [10.0**k for k in range(-22, 38)]
    return np.concatenate([bits, dec, ints, np.array(specials, np.float64)])


def test_device_formatter_matches_rust_display(ssp):
    vals = _samples(1, 60000)
    done = 0
    for v in vals:
        got = ssp.format_shortest(float(v))
        if got is None:
            # left to the host: not finite, subnormal, outside about [1e-22, 3e38], or longer than the buffer
            a = abs(float(v))
            assert not math.isfinite(a) or a < 1e-21 or a > 1e38 or len(_rust(float(v))) >= 63, v
            continue
        assert got == _rust(float(v)), (float(v).hex(), got, _rust(float(v)))
        done += 1
    assert done > 0.95 * len(vals)


def test_host_converter_weights_match_rust_display(ssp, tmp_path):
    vals = list(_samples(2, 3000)) + [float("inf"), float("-inf"), 5e-324, 1e300, -1e-300]
    src = tmp_path / "w.txt"
    with open(src, "w") as f:
        f.write(f"{len(vals) + 1} {len(vals)}\n")
        for i, v in enumerate(vals):
            f.write(f"{i} {i + 1} {float(v)!r}\n")
    dst = tmp_path / "w.mtx"
    ssp.edge_list_to_matrix_market(src, dst, 1.0)
    body = dst.read_text().splitlines()[3:]
    assert len(body) == len(vals)
    for i, (ln, v) in enumerate(zip(body, vals)):
        assert ln == f"{i} {i + 1} {_rust(float(v))}", (ln, float(v))


@pytest.mark.parametrize("v,text", [(2.0**70, "1180591620717411300000"), (1e21, "1000000000000000000000"),
                                    (1.5, "1.5"), (-0.0, "-0"), (100.0, "100"), (1e-7, "0.0000001")])
def test_known_texts(ssp, v, text):
    assert ssp.format_shortest(v) == text
