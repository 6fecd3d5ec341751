"""The exact decimal conversions of the GPU Matrix Market reader and writer, run on the host through the C ABI:
parse_decimal must return strtod's correctly rounded binary64 bit for bit (or hand the token to the host),
format_g17 must write printf("%.17g")'s bytes (or hand the value to the host).  Random tokens and values over
the converters' whole domain, plus the round-half-even ties both directions have."""
import ctypes
import random
import struct

import pytest

_LIBC = ctypes.CDLL(None)


def _g17(x):
    buf = ctypes.create_string_buffer(64)
    _LIBC.snprintf(buf, 64, b"%.17g", ctypes.c_double(x))
    return buf.value.decode()


def _bits(x):
    return struct.unpack("<Q", struct.pack("<d", x))[0]


def _random_token(rng):
    nd = rng.randint(1, 19)
    digits = "".join(rng.choice("0123456789") for _ in range(nd))
    lead = "0" * rng.choice([0, 0, 0, 1, 3])
    sign = rng.choice(["", "", "-", "+"])
    point = rng.randint(0, nd)
    body = lead + digits[:point] + "." + digits[point:] if rng.random() < 0.8 else lead + digits
    if body.startswith(".") and rng.random() < 0.5:
        body = "0" + body
    exp = ""
    if rng.random() < 0.6:
        exp = rng.choice("eE") + rng.choice(["", "-", "+"]) + str(rng.randint(0, 40))
    return sign + body + exp


def test_parse_matches_strtod(ssp):
    rng = random.Random(11)
    host = 0
    tokens = [_random_token(rng) for _ in range(60000)]
    # what the writer produces: %.17g of random doubles over many decades
    tokens += [_g17(rng.uniform(1, 10) * 10.0 ** rng.randint(-30, 30)) for _ in range(40000)]
    # ties: integers half-way between two doubles (2^53 + odd, scaled by powers of two), written exactly
    for k in range(1, 200, 2):
        for j in range(0, 9):
            tokens.append(str((2 ** 53 + k) * 2 ** j))
        for j in range(1, 4):  # (2^53 + k) / 2^j written exactly: digits of (2^53 + k) 5^j, point j from the end
            d = str((2 ** 53 + k) * 5 ** j)
            tokens.append(d[:-j] + "." + d[-j:])
    for t in tokens:
        rc, v = ssp.parse_decimal(t)
        assert rc in (0, 1), t
        if rc == 1:
            assert _bits(v) == _bits(float(t)), (t, v, float(t))
        else:
            host += 1
    # only tokens outside the exact domain (|exponent| > 38, subnormal) go to the host
    assert host < 0.2 * len(tokens)


@pytest.mark.parametrize("token", ["1e", "abc", "", "-", "e5", "--1"])
def test_parse_rejects_malformed(ssp, token):
    assert ssp.parse_decimal(token)[0] == -1


# strtod decides these: forms it may accept (or reject) and values outside the exact domain
@pytest.mark.parametrize("token", ["inf", "nan", "1e400", "1e-320", "0x1p3", "1234567890123456789012", "1e-39",
                                   "1.2.3"])
def test_parse_leaves_the_rest_to_the_host(ssp, token):
    assert ssp.parse_decimal(token)[0] == 0


def test_format_matches_printf(ssp):
    rng = random.Random(5)
    xs = [rng.uniform(-1, 1) * 10.0 ** rng.uniform(-22, 40) for _ in range(80000)]
    xs += [struct.unpack("<d", struct.pack("<Q", rng.getrandbits(64)))[0] for _ in range(20000)]
    # 18-significant-digit values whose 17-digit rounding is an exact tie
    xs += [(10 ** 15 + k) / 16.0 for k in range(1, 4000, 2)]
    xs += [0.0, -0.0, 1.0, 0.1, 1e16, 1e17, 9.999999999999998e16, 2.0 ** -60, 1e-20, 9.9e38]
    host = 0
    for x in xs:
        s = ssp.format_g17(x)
        if s is None:
            host += 1
            ax = abs(x)
            assert x != x or ax == float("inf") or ax < 1.1e-20 or ax >= 9.9e38, x
        else:
            assert s == _g17(x), (x, s, _g17(x))
    assert host < 0.3 * len(xs)
