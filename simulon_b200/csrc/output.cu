// Host-side helpers of the simulator's output files (no device work): the
// trajectory rows "<symbol> <x> <y> <z>" with six decimals, as
// MDSimulator._dump_step_outputs writes them (core/md_simulation.py:125-168).
//
// A double is m 2^e exactly (m a 53-bit integer), so x 10^6 = m 10^6 2^e is
// formed exactly in 128-bit integers and rounded half to even on the exact
// value: the digits equal Python's format(x, ".6f") (correctly rounded, ties
// to even) and C's printf("%.6f").  Magnitudes of 2^40 and above and
// infinities go through snprintf; NaN prints as "nan" (as Python).
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>

#include "../../include/simb200.h"

namespace {

// x in fixed notation with six decimals into p (room for at least 64 bytes);
// returns the length.
int fixed6(double x, char* p) {
    if (std::isnan(x)) {                  // Python prints NaN unsigned
        std::memcpy(p, "nan", 3);
        return 3;
    }
    if (!std::isfinite(x) || std::fabs(x) >= 1099511627776.0) return snprintf(p, 64, "%.6f", x);
    uint64_t bits;
    std::memcpy(&bits, &x, sizeof bits);
    const bool neg = (bits >> 63) != 0;
    const int be = (int)((bits >> 52) & 0x7FF);
    uint64_t m = bits & ((1ull << 52) - 1);
    int e;
    if (be == 0) {
        e = -1074;                        // subnormal (or zero)
    } else {
        m |= 1ull << 52;
        e = be - 1075;
    }
    // v = round_half_even(m * 10^6 * 2^e), m * 10^6 < 2^73
    unsigned __int128 v = (unsigned __int128)m * 1000000u;
    if (e >= 0) {
        v <<= e;                          // not reached: |x| < 2^40 gives e <= -13
    } else {
        const int s = -e;
        if (s >= 128) {
            v = 0;                        // x 10^6 < 2^-54: rounds to 0
        } else {
            const unsigned __int128 q = v >> s;
            const unsigned __int128 rem = v - (q << s);
            const unsigned __int128 half = (unsigned __int128)1 << (s - 1);
            v = q;
            if (rem > half || (rem == half && (q & 1))) v += 1;
        }
    }
    const uint64_t whole = (uint64_t)(v / 1000000u);
    const uint32_t frac = (uint32_t)(v % 1000000u);
    char tmp[32];
    int n = 0;
    uint64_t w = whole;
    do {
        tmp[n++] = (char)('0' + (int)(w % 10));
        w /= 10;
    } while (w);
    int len = 0;
    if (neg) p[len++] = '-';
    while (n) p[len++] = tmp[--n];
    p[len++] = '.';
    uint32_t f = frac;
    for (int k = 5; k >= 0; --k) {
        p[len + k] = (char)('0' + (int)(f % 10));
        f /= 10;
    }
    return len + 6;
}

}  // namespace

extern "C" int64_t sim_format_xyz_rows(const double* xyz, const int32_t* type, int64_t n, const char* const* symbols,
                                       int32_t n_symbols, char* out, int64_t cap) {
    if (n < 0 || !out || cap < 0 || (n > 0 && (!xyz || !symbols || n_symbols <= 0))) return -1;
    int64_t w = 0;
    for (int64_t i = 0; i < n; ++i) {
        const int32_t t = type ? type[i] : 0;
        if (t < 0 || t >= n_symbols || !symbols[t]) return -1;
        const size_t ls = std::strlen(symbols[t]);
        if (cap - w < (int64_t)ls + 3 * 64 + 4) return -1;   // room for the widest row
        std::memcpy(out + w, symbols[t], ls);
        w += (int64_t)ls;
        for (int c = 0; c < 3; ++c) {
            out[w++] = ' ';
            w += fixed6(xyz[3 * i + c], out + w);
        }
        out[w++] = '\n';
    }
    return w;
}
