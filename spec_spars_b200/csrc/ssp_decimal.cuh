// ssp_decimal.cuh -- exact decimal <-> binary64 conversions for the Matrix Market reader and writer, usable
// on the host and on the device.
//
// parse_decimal: the correctly rounded (round-half-even) binary64 nearest to a decimal token, as strtod and
// Rust's str::parse::<f64> return it.  With at most 19 significant digits the token is m * 10^E exactly
// (m < 2^64); for 0 <= E <= 38 the product is an exact 128-bit integer, and for -38 <= E < 0 the quotient
// m / 10^-E is formed by binary long division to 55+ bits plus a sticky remainder.  Either way the result is
// rounded once.  Tokens outside that domain (more significant digits, |E| > 38, results that would be
// subnormal, inf / nan / hex forms) return NEEDS_HOST: the caller converts those few on the host.
//
// format_g17: the text printf("%.17g") writes for a binary64 (17 significant digits, round-half-even on the
// exact binary value, %g's choice of fixed or exponent form, trailing zeros removed).  The 17-digit integer
// is computed exactly with 192-bit arithmetic for decimal exponents in [-20, 38]; other values return -1 and
// are formatted on the host.
#pragma once
#include <math.h>
#include <stdint.h>

#if defined(__CUDACC__)
#define SSP_HD __host__ __device__ __forceinline__
#else
#define SSP_HD inline
#endif

namespace ssp {
namespace dec {

typedef unsigned __int128 u128;

enum { PARSE_OK = 1, PARSE_NEEDS_HOST = 0, PARSE_SYNTAX = -1 };

SSP_HD int bitlen64(uint64_t x) {
#if defined(__CUDA_ARCH__)
    return x ? 64 - __clzll((long long)x) : 0;
#else
    return x ? 64 - __builtin_clzll(x) : 0;
#endif
}
SSP_HD int bitlen128(u128 x) {
    const uint64_t hi = (uint64_t)(x >> 64);
    return hi ? 64 + bitlen64(hi) : bitlen64((uint64_t)x);
}
SSP_HD u128 pow10_128(int k) {  // 0 <= k <= 38
    u128 p = 1;
    for (int i = 0; i < k; i++) p *= 10;
    return p;
}
// 2^s for -1022 <= s <= 1023
SSP_HD double pow2(int s) {
    union {
        uint64_t u;
        double d;
    } c;
    c.u = (uint64_t)(1023 + s) << 52;
    return c.d;
}
// mant * 2^e2 for an integer mant < 2^53, exact when the result is normal (every partial product lies
// between mant and the result, so it is normal too)
SSP_HD double ldexp_exact(uint64_t mant, int e2) {
    double v = (double)mant;
    while (e2 > 1000) {
        v *= pow2(1000);
        e2 -= 1000;
    }
    while (e2 < -1000) {
        v *= pow2(-1000);
        e2 += 1000;
    }
    return v * pow2(e2);
}
// round an exact value N * 2^scale2 (+ a positive fraction below N's last bit when sticky) to binary64;
// false when the result would be subnormal or overflow
SSP_HD bool round_to_double(u128 N, bool sticky_in, int scale2, double* out) {
    const int L = bitlen128(N);
    uint64_t mant;
    int sh = 0;
    if (L <= 53) {
        if (sticky_in) return false;  // callers pass a fraction only with 55+ bits of N
        mant = (uint64_t)N;
    } else {
        sh = L - 53;
        mant = (uint64_t)(N >> sh);
        const bool guard = (N >> (sh - 1)) & 1;
        const u128 below = sh >= 2 ? (N & ((((u128)1) << (sh - 1)) - 1)) : (u128)0;
        const bool sticky = below != 0 || sticky_in;
        if (guard && (sticky || (mant & 1))) mant++;
        if (mant == (1ull << 53)) {
            mant >>= 1;
            sh++;
        }
    }
    if (mant == 0) {
        *out = 0.0;
        return true;
    }
    // value = mant * 2^(sh + scale2); normal iff its exponent lies in [-1022, 1023]
    const int e = sh + scale2 + bitlen64(mant) - 1;
    if (e < -1022 || e > 1023) return false;
    *out = ldexp_exact(mant, sh + scale2);
    return true;
}

// value of m * 10^E, m > 0
SSP_HD bool m10e_to_double(uint64_t m, int E, double* out) {
    if (E >= 0) {
        if (E > 38) return false;
        const u128 P = pow10_128(E);
        if (bitlen64(m) + bitlen128(P) > 128) return false;
        return round_to_double((u128)m * P, false, 0, out);
    }
    if (-E > 38) return false;
    const u128 P = pow10_128(-E);
    const int bm = bitlen64(m), bp = bitlen128(P);
    const int s = bp - bm + 55 > 0 ? bp - bm + 55 : 0;
    // long division of (m << s) by P, one numerator bit at a time; rem < P < 2^127 throughout
    u128 rem = 0;
    uint64_t Q = 0;
    for (int i = bm + s - 1; i >= 0; i--) {
        const uint64_t bit = (i >= s && i - s < 64) ? (m >> (i - s)) & 1 : 0;
        rem = (rem << 1) | bit;
        Q <<= 1;
        if (rem >= P) {
            rem -= P;
            Q |= 1;
        }
    }
    return round_to_double((u128)Q, rem != 0, -s, out);
}

SSP_HD bool is_digit(char c) { return c >= '0' && c <= '9'; }

// the token [p, e) (no surrounding whitespace)
SSP_HD int parse_decimal(const char* p, const char* e, double* out) {
    bool neg = false;
    if (p < e && (*p == '+' || *p == '-')) {
        neg = *p == '-';
        p++;
    }
    uint64_t m = 0;
    int nd = 0, exp10 = 0;
    bool any = false, trunc = false;
    for (; p < e && is_digit(*p); p++) {
        any = true;
        const int d = *p - '0';
        if (nd < 19) {
            if (m || d) {
                m = m * 10 + d;
                nd++;
            }
        } else {
            exp10++;
            if (d) trunc = true;
        }
    }
    if (p < e && *p == '.') {
        p++;
        for (; p < e && is_digit(*p); p++) {
            any = true;
            const int d = *p - '0';
            if (nd < 19) {
                if (m || d) {
                    m = m * 10 + d;
                    nd++;
                }
                exp10--;
            } else if (d) {
                trunc = true;
            }
        }
    }
    if (!any) {
        // inf, nan, hex: leave to the host's strtod
        return (p < e && (*p == 'i' || *p == 'I' || *p == 'n' || *p == 'N')) ? PARSE_NEEDS_HOST : PARSE_SYNTAX;
    }
    if (p < e && (*p == 'e' || *p == 'E')) {
        p++;
        bool eneg = false;
        if (p < e && (*p == '+' || *p == '-')) {
            eneg = *p == '-';
            p++;
        }
        if (!(p < e && is_digit(*p))) return PARSE_SYNTAX;
        int x = 0;
        for (; p < e && is_digit(*p); p++)
            if (x < 100000) x = x * 10 + (*p - '0');
        exp10 += eneg ? -x : x;
    }
    if (p != e) {
        // hex floats ("0x...") and other forms strtod may still accept
        return PARSE_NEEDS_HOST;
    }
    if (trunc) return PARSE_NEEDS_HOST;
    if (m == 0) {
        *out = neg ? -0.0 : 0.0;
        return PARSE_OK;
    }
    double v;
    if (!m10e_to_double(m, exp10, &v)) return PARSE_NEEDS_HOST;
    *out = neg ? -v : v;
    return PARSE_OK;
}

// ---------------------------------------------------------------- %.17g
// 192-bit unsigned integers as three 64-bit limbs (little end first)
struct U192 {
    uint64_t w[3];
};
SSP_HD void u192_mul_small(U192& a, uint64_t f) {
    u128 c = 0;
    for (int i = 0; i < 3; i++) {
        const u128 t = (u128)a.w[i] * f + c;
        a.w[i] = (uint64_t)t;
        c = t >> 64;
    }
}
SSP_HD bool u192_bit(const U192& a, int i) { return (a.w[i >> 6] >> (i & 63)) & 1; }
SSP_HD int u192_bitlen(const U192& a) {
    for (int i = 2; i >= 0; i--)
        if (a.w[i]) return 64 * i + bitlen64(a.w[i]);
    return 0;
}
// floor(a / 2^t) as u128 (the caller guarantees it fits)
SSP_HD u128 u192_shr(const U192& a, int t) {
    u128 r = 0;
    for (int i = u192_bitlen(a) - 1; i >= t; i--) r = (r << 1) | (u128)u192_bit(a, i);
    return r;
}
// floor(a / P) and whether the remainder is zero, compared at half: returns quotient, sets cmp to
// -1 / 0 / +1 for remainder below / at / above P / 2
SSP_HD u128 u192_div(const U192& a, u128 P, int* cmp) {
    u128 rem = 0, q = 0;
    for (int i = u192_bitlen(a) - 1; i >= 0; i--) {
        // rem < P <= 2^80 here, so the shift cannot overflow
        rem = (rem << 1) | (u128)u192_bit(a, i);
        q <<= 1;
        if (rem >= P) {
            rem -= P;
            q |= 1;
        }
    }
    const u128 twice = rem << 1;
    *cmp = twice < P ? -1 : (twice == P ? 0 : 1);
    return q;
}

// D = v * 10^(16 - X) rounded half-even to an integer, for positive finite v = mant * 2^e2; false outside the
// supported range
SSP_HD bool scaled17(uint64_t mant, int e2, int X, uint64_t* D) {
    const int k = 16 - X;
    if (k >= 0) {
        if (k > 37) return false;
        U192 N = {{mant, 0, 0}};
        for (int i = 0; i < k; i++) u192_mul_small(N, 10);
        if (e2 >= 0) {
            // only values >= 2^52 have e2 >= 0, so k <= 1 here
            if (e2 > 8) return false;
            u128 r = ((u128)N.w[1] << 64 | N.w[0]) << e2;
            if (N.w[2] || u192_bitlen(N) + e2 > 127) return false;
            *D = (uint64_t)r;
            return true;
        }
        const int t = -e2;
        if (t >= 192 || u192_bitlen(N) - t > 120) return false;
        u128 r = u192_shr(N, t);
        const bool guard = u192_bit(N, t - 1);
        bool below = false;
        for (int i = 0; i < t - 1; i++) below |= u192_bit(N, i);
        if (guard && (below || (r & 1))) r++;
        *D = (uint64_t)r;
        return true;
    }
    // k < 0: D = mant * 2^e2 / 10^-k, with e2 >= 0 (v >= 1e17)
    if (-k > 23 || e2 < 0 || e2 > 120) return false;
    U192 N = {{mant, 0, 0}};
    for (int i = 0; i < e2; i++) u192_mul_small(N, 2);
    int cmp = 0;
    u128 q = u192_div(N, pow10_128(-k), &cmp);
    if (cmp > 0 || (cmp == 0 && (q & 1))) q++;
    *D = (uint64_t)q;
    return true;
}

// printf("%.17g", v) into buf (at least 32 bytes); returns the length, or -1 (format on the host)
SSP_HD int format_g17(double v, char* buf) {
    union { double d; uint64_t u; } c;
    c.d = v;
    const bool neg = c.u >> 63;
    const int be = (int)((c.u >> 52) & 0x7ff);
    const uint64_t frac = c.u & ((1ull << 52) - 1);
    int n = 0;
    if (be == 0x7ff) return -1;  // inf / nan
    if (neg) buf[n++] = '-';
    if (be == 0 && frac == 0) {
        buf[n++] = '0';
        return n;
    }
    if (be == 0) return -1;  // subnormal
    const uint64_t mant = frac | (1ull << 52);
    const int e2 = be - 1075;
    // X = floor(log10 v): an estimate, corrected below by the digit count of D
    int X = (int)floor(log10(neg ? -v : v));
    if (X < -21 || X > 39) return -1;
    uint64_t D = 0;
    const uint64_t LO = 10000000000000000ull, HI = 100000000000000000ull;  // 1e16, 1e17
    for (int tries = 0; tries < 4; tries++) {
        if (X < -21 || X > 39) return -1;
        if (!scaled17(mant, e2, X, &D)) return -1;
        if (D >= HI) {
            // either X is one too small, or rounding carried to 10^17
            uint64_t D2;
            if (!scaled17(mant, e2, X + 1, &D2)) return -1;
            if (D2 >= LO) {
                X++;
                D = D2;
                if (D >= HI) continue;
                break;
            }
            return -1;
        }
        if (D < LO) {
            X--;
            continue;
        }
        break;
    }
    if (D < LO || D >= HI || X < -20 || X > 38) return -1;
    char dig[17];
    for (int i = 16; i >= 0; i--) {
        dig[i] = (char)('0' + D % 10);
        D /= 10;
    }
    int last = 16;  // last significant digit kept after stripping trailing zeros
    while (last > 0 && dig[last] == '0') last--;
    if (X < -4 || X >= 17) {
        buf[n++] = dig[0];
        if (last > 0) {
            buf[n++] = '.';
            for (int i = 1; i <= last; i++) buf[n++] = dig[i];
        }
        buf[n++] = 'e';
        int x = X;
        buf[n++] = x < 0 ? '-' : '+';
        if (x < 0) x = -x;
        if (x >= 100) buf[n++] = (char)('0' + x / 100);
        buf[n++] = (char)('0' + (x / 10) % 10);
        buf[n++] = (char)('0' + x % 10);
    } else if (X >= 0) {
        for (int i = 0; i <= X; i++) buf[n++] = dig[i];
        if (last > X) {
            buf[n++] = '.';
            for (int i = X + 1; i <= last; i++) buf[n++] = dig[i];
        }
    } else {
        buf[n++] = '0';
        buf[n++] = '.';
        for (int i = 0; i < -X - 1; i++) buf[n++] = '0';
        for (int i = 0; i <= last; i++) buf[n++] = dig[i];
    }
    return n;
}

// ---------------------------------------------------------------- shortest round-trip, fixed notation
// a / P and a % P (bit by bit; P < 2^127)
SSP_HD u128 u192_divmod(const U192& a, u128 P, u128* rem) {
    u128 r = 0, q = 0;
    for (int i = u192_bitlen(a) - 1; i >= 0; i--) {
        r = (r << 1) | (u128)u192_bit(a, i);
        q <<= 1;
        if (r >= P) {
            r -= P;
            q |= 1;
        }
    }
    *rem = r;
    return q;
}

// q = floor(mant * 2^e2 * 10^k), with the remainder compared at half (cmp -1 / 0 / +1 below / at / above) and
// whether it is zero; false outside the supported range (|k| <= 38, q < 2^64, operands within 192 bits)
SSP_HD bool scaled_floor(uint64_t mant, int e2, int k, uint64_t* q, int* cmp, bool* exact) {
    if (k > 38 || k < -38) return false;
    if (k >= 0) {
        U192 N = {{mant, 0, 0}};
        for (int i = 0; i < k; i++) u192_mul_small(N, 10);
        if (e2 >= 0) {
            if (u192_bitlen(N) + e2 > 63) return false;
            *q = N.w[0] << e2;
            *cmp = -1;
            *exact = true;
            return true;
        }
        const int t = -e2;
        if (t >= 192 || u192_bitlen(N) - t > 63) return false;
        *q = (uint64_t)u192_shr(N, t);
        const bool guard = u192_bit(N, t - 1);
        bool sticky = false;
        for (int i = 0; i < t - 1 && !sticky; i++) sticky = u192_bit(N, i);
        *cmp = guard ? (sticky ? 1 : 0) : -1;
        *exact = !guard && !sticky;
        return true;
    }
    u128 P = pow10_128(-k);
    U192 N = {{mant, 0, 0}};
    if (e2 >= 0) {
        if (e2 > 127) return false;
        for (int i = 0; i < e2; i++) u192_mul_small(N, 2);
    } else {
        if (bitlen128(P) + (-e2) > 126) return false;
        P <<= -e2;
    }
    u128 rem = 0;
    const u128 qq = u192_divmod(N, P, &rem);
    if (qq >> 64) return false;
    *q = (uint64_t)qq;
    const u128 twice = rem << 1;
    *cmp = twice < P ? -1 : (twice == P ? 0 : 1);
    *exact = rem == 0;
    return true;
}

// The shortest decimal that reads back as v (the closest such one; an exact tie keeps the even last digit), in
// fixed notation without an exponent: the text Rust's Display writes for an f64 and C++'s
// to_chars(..., chars_format::fixed) writes.  Returns the length written to buf (at most cap), or -1 when v is
// not finite, subnormal, outside about [1e-22, 1e54], or its text is longer than cap (format on the host).
SSP_HD int format_shortest_fixed(double v, char* buf, int cap) {
    union { double d; uint64_t u; } c;
    c.d = v;
    const bool neg = c.u >> 63;
    const int be = (int)((c.u >> 52) & 0x7ff);
    const uint64_t frac = c.u & ((1ull << 52) - 1);
    if (be == 0x7ff || (be == 0 && frac != 0)) return -1;  // inf / nan / subnormal
    int n = 0;
    if (neg) {
        if (cap < 1) return -1;
        buf[n++] = '-';
    }
    if (be == 0) {
        if (n + 1 > cap) return -1;
        buf[n++] = '0';
        return n;
    }
    const uint64_t mant = frac | (1ull << 52);
    const int e2 = be - 1075;
    // X = floor(log10 |v|) exactly: 17 digits of the floor fall in [1e16, 1e17)
    int X = (int)floor(log10(neg ? -v : v));
    const uint64_t LO = 10000000000000000ull, HI = 100000000000000000ull;
    uint64_t q = 0;
    int cmp = 0;
    bool exact = false;
    for (int tries = 0;; tries++) {
        if (tries > 3 || !scaled_floor(mant, e2, 16 - X, &q, &cmp, &exact)) return -1;
        if (q >= HI) X++;
        else if (q < LO) X--;
        else break;
    }
    // the fewest significant digits P whose floor or ceiling reads back as v
    uint64_t digits = 0;
    int dexp = 0;  // v's text = digits * 10^dexp
    for (int P = 1; P <= 17; P++) {
        const int k = P - 1 - X;
        if (!scaled_floor(mant, e2, k, &q, &cmp, &exact)) return -1;
        if (exact) {
            digits = q;
            dexp = -k;
            break;
        }
        double d1 = 0, d2 = 0;
        const int E = -k;
        const bool in1 = m10e_to_double(q, E, &d1), in2 = m10e_to_double(q + 1, E, &d2);
        if (!in1 || !in2) return -1;
        const bool ok1 = d1 == (neg ? -v : v), ok2 = d2 == (neg ? -v : v);
        if (!ok1 && !ok2) continue;
        bool up = ok2 && (!ok1 || cmp > 0 || (cmp == 0 && (q & 1)));
        digits = up ? q + 1 : q;
        dexp = E;
        break;
    }
    if (digits == 0) return -1;
    while (digits % 10 == 0) {
        digits /= 10;
        dexp++;
    }
    char dig[20];
    int L = 0;
    for (uint64_t t = digits; t; t /= 10) dig[L++] = (char)('0' + t % 10);
    // dig holds the digits lowest first
    if (dexp >= 0) {
        if (n + L + dexp > cap) return -1;
        for (int i = L - 1; i >= 0; i--) buf[n++] = dig[i];
        for (int i = 0; i < dexp; i++) buf[n++] = '0';
    } else if (L + dexp > 0) {
        if (n + L + 1 > cap) return -1;
        const int ip = L + dexp;  // digits before the point
        for (int i = 0; i < L; i++) {
            if (i == ip) buf[n++] = '.';
            buf[n++] = dig[L - 1 - i];
        }
    } else {
        const int z = -dexp - L;  // zeros after the point
        if (n + 2 + z + L > cap) return -1;
        buf[n++] = '0';
        buf[n++] = '.';
        for (int i = 0; i < z; i++) buf[n++] = '0';
        for (int i = L - 1; i >= 0; i--) buf[n++] = dig[i];
    }
    return n;
}

}  // namespace dec
}  // namespace ssp
