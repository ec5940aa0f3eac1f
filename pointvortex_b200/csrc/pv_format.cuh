// pv_format.cuh — exact decimal text of doubles as `std::ostream << std::setprecision(17)` writes
// them (the reference's trajectory and checkpoint files, src/print.cpp:20, src/checkpoint.cpp:41),
// for one value per GPU thread.
//
// With precision 17 and no floatfield flag, libstdc++ formats a double through "%.*g", so every
// value is printed with 17 significant digits, correctly rounded (ties to even) from its exact
// binary value, in the shorter of the fixed and exponent forms that %g chooses, with trailing
// zeros removed. Correct rounding needs the exact value, so the scaling by a power of ten is done
// in integer arithmetic on up to 1152-bit numbers:
//
//   |v| = m 2^e (53-bit m), k = floor(log10 |v|), s = 16 - k,
//   D = round_half_even(|v| 10^s) in [10^16, 10^17]   (D = 10^17 -> D = 10^16, k + 1)
//   s >= 0:  |v| 10^s = m 5^s 2^(e+s)         (one big product, then a shift)
//   s <  0:  |v| 10^s = m 2^e / (5^-s 2^-s)   (a 61-bit quotient by binary long division)
//
// k starts from floor(b log10 2) for the top bit b of |v| ((b * 78913) >> 18, exact for
// |b| <= 1100) and moves up by one when the scaled value reaches 10^17. The functions are
// __host__ __device__ so that the same source can be checked on the CPU.
#pragma once

#include <stdint.h>

#if defined(__CUDACC__)
#define PVF_HD __host__ __device__ __forceinline__
#else
#define PVF_HD inline
#endif

namespace pvb {
namespace fmt {

constexpr int kMaxDoubleChars = 24;  // "-1.2345678901234567e-308"
constexpr int kMaxU64Chars = 20;     // 18446744073709551615
constexpr int kLimbs = 18;           // 1152 bits: m 2^971 and 5^292 2^288 fit

struct Big {
    uint64_t w[kLimbs];  // little-endian limbs; all limbs are kept valid (no length field)
};

PVF_HD void mul_wide(uint64_t a, uint64_t b, uint64_t &lo, uint64_t &hi) {
#if defined(__CUDA_ARCH__)
    lo = a * b;
    hi = __umul64hi(a, b);
#else
    const unsigned __int128 p = static_cast<unsigned __int128>(a) * b;
    lo = static_cast<uint64_t>(p);
    hi = static_cast<uint64_t>(p >> 64);
#endif
}

PVF_HD int clz64(uint64_t x) {
#if defined(__CUDA_ARCH__)
    return __clzll(static_cast<long long>(x));
#else
    return x ? __builtin_clzll(x) : 64;
#endif
}

PVF_HD void big_set(Big &a, uint64_t v) {
    a.w[0] = v;
    for (int i = 1; i < kLimbs; ++i)
        a.w[i] = 0;
}

PVF_HD void big_mul_small(Big &a, uint64_t f) {
    uint64_t carry = 0;
    for (int i = 0; i < kLimbs; ++i) {
        uint64_t lo, hi;
        mul_wide(a.w[i], f, lo, hi);
        lo += carry;
        hi += (lo < carry) ? 1 : 0;
        a.w[i] = lo;
        carry = hi;
    }
}

// a *= 5^p
PVF_HD void big_mul_pow5(Big &a, int p) {
    const uint64_t p27 = 7450580596923828125ull;  // 5^27, the largest power of 5 below 2^63
    while (p >= 27) {
        big_mul_small(a, p27);
        p -= 27;
    }
    uint64_t f = 1;
    for (int i = 0; i < p; ++i)
        f *= 5;
    if (f != 1)
        big_mul_small(a, f);
}

PVF_HD void big_shl(Big &a, int bits) {
    const int limbs = bits >> 6, r = bits & 63;
    for (int i = kLimbs - 1; i >= 0; --i) {
        const int src = i - limbs;
        uint64_t v = 0;
        if (src >= 0) {
            v = a.w[src] << r;
            if (r && src >= 1)
                v |= a.w[src - 1] >> (64 - r);
        }
        a.w[i] = v;
    }
}

PVF_HD void big_shr1(Big &a) {
    for (int i = 0; i < kLimbs; ++i)
        a.w[i] = (a.w[i] >> 1) | (i + 1 < kLimbs ? (a.w[i + 1] << 63) : 0);
}

PVF_HD int big_cmp(const Big &a, const Big &b) {
    for (int i = kLimbs - 1; i >= 0; --i)
        if (a.w[i] != b.w[i])
            return a.w[i] < b.w[i] ? -1 : 1;
    return 0;
}

PVF_HD void big_sub(Big &a, const Big &b) {
    uint64_t borrow = 0;
    for (int i = 0; i < kLimbs; ++i) {
        const uint64_t d = a.w[i] - b.w[i];
        const uint64_t d2 = d - borrow;
        borrow = (a.w[i] < b.w[i]) || (d < borrow) ? 1 : 0;
        a.w[i] = d2;
    }
}

PVF_HD bool big_bit(const Big &a, int bit) { return (a.w[bit >> 6] >> (bit & 63)) & 1; }

PVF_HD bool big_any_below(const Big &a, int bit) {  // any set bit in [0, bit)
    const int full = bit >> 6, r = bit & 63;
    for (int i = 0; i < full; ++i)
        if (a.w[i])
            return true;
    return r && (a.w[full] & ((uint64_t{1} << r) - 1));
}

PVF_HD uint64_t big_bits64(const Big &a, int from) {  // bits [from, from + 64)
    const int l = from >> 6, r = from & 63;
    uint64_t v = l < kLimbs ? a.w[l] >> r : 0;
    if (r && l + 1 < kLimbs)
        v |= a.w[l + 1] << (64 - r);
    return v;
}

// floor(m 2^e 10^s) and where the dropped fraction lies against one half (-1 below, 0 at,
// +1 above). The quotient is below 2^61 for the s this file uses.
PVF_HD uint64_t scaled_floor(uint64_t m, int e, int s, int &half_cmp) {
    Big n;
    big_set(n, m);
    if (s >= 0) {
        big_mul_pow5(n, s);
        const int t = e + s;
        if (t >= 0) {
            big_shl(n, t);
            half_cmp = -1;
            return n.w[0];
        }
        const int sh = -t;
        const uint64_t q = big_bits64(n, sh);
        const bool half = big_bit(n, sh - 1);
        half_cmp = !half ? -1 : (big_any_below(n, sh - 1) ? 1 : 0);
        return q;
    }
    const int r = -s;
    Big d;
    big_set(d, 1);
    big_mul_pow5(d, r);
    if (e >= r)
        big_shl(n, e - r);
    else
        big_shl(d, r - e);
    // binary long division, quotient bits 60..0
    Big ds = d;
    big_shl(ds, 60);
    uint64_t q = 0;
    for (int bit = 60; bit >= 0; --bit) {
        if (big_cmp(n, ds) >= 0) {
            big_sub(n, ds);
            q |= uint64_t{1} << bit;
        }
        big_shr1(ds);
    }
    big_shl(n, 1);  // compare 2 * remainder with the divisor
    half_cmp = big_cmp(n, d);
    return q;
}

PVF_HD int format_u64(uint64_t v, char *out) {
    char tmp[kMaxU64Chars];
    int n = 0;
    do {
        tmp[n++] = static_cast<char>('0' + v % 10);
        v /= 10;
    } while (v);
    for (int i = 0; i < n; ++i)
        out[i] = tmp[n - 1 - i];
    return n;
}

// "%.17g" of v into out (at most kMaxDoubleChars bytes, no terminator); returns the length.
PVF_HD int format_g17(double v, char *out) {
#if defined(__CUDA_ARCH__)
    const uint64_t bits = static_cast<uint64_t>(__double_as_longlong(v));
#else
    uint64_t bits;
    __builtin_memcpy(&bits, &v, sizeof bits);
#endif
    int len = 0;
    const bool negative = bits >> 63;
    const int be = static_cast<int>((bits >> 52) & 0x7ff);
    const uint64_t frac = bits & ((uint64_t{1} << 52) - 1);
    if (negative)
        out[len++] = '-';
    if (be == 0x7ff) {
        const char *t = frac ? "nan" : "inf";
        for (int i = 0; i < 3; ++i)
            out[len++] = t[i];
        return len;
    }
    if (be == 0 && frac == 0) {
        out[len++] = '0';
        return len;
    }
    const uint64_t m = be ? (frac | (uint64_t{1} << 52)) : frac;
    const int e = be ? be - 1075 : -1074;
    const int top = e + 63 - clz64(m);
    int k = (top * 78913) >> 18;  // floor(top log10 2); arithmetic shift floors negatives
    int half_cmp = 0;
    uint64_t q = scaled_floor(m, e, 16 - k, half_cmp);
    const uint64_t p17 = 100000000000000000ull, p16 = 10000000000000000ull;
    if (q >= p17) {
        ++k;
        q = scaled_floor(m, e, 16 - k, half_cmp);
    }
    if (half_cmp > 0 || (half_cmp == 0 && (q & 1)))
        ++q;
    if (q == p17) {
        q = p16;
        ++k;
    }
    char dig[17];
    for (int i = 16; i >= 0; --i) {
        dig[i] = static_cast<char>('0' + q % 10);
        q /= 10;
    }
    int last = 16;  // last significant digit after trailing zeros go
    while (last > 0 && dig[last] == '0')
        --last;
    if (k >= -4 && k < 17) {
        if (k >= 0) {
            for (int i = 0; i <= k; ++i)
                out[len++] = dig[i];
            if (last > k) {
                out[len++] = '.';
                for (int i = k + 1; i <= last; ++i)
                    out[len++] = dig[i];
            }
        } else {
            out[len++] = '0';
            out[len++] = '.';
            for (int i = 0; i < -k - 1; ++i)
                out[len++] = '0';
            for (int i = 0; i <= last; ++i)
                out[len++] = dig[i];
        }
        return len;
    }
    out[len++] = dig[0];
    if (last > 0) {
        out[len++] = '.';
        for (int i = 1; i <= last; ++i)
            out[len++] = dig[i];
    }
    out[len++] = 'e';
    out[len++] = k < 0 ? '-' : '+';
    const int ak = k < 0 ? -k : k;
    if (ak >= 100)
        out[len++] = static_cast<char>('0' + ak / 100);
    out[len++] = static_cast<char>('0' + (ak / 10) % 10);
    out[len++] = static_cast<char>('0' + ak % 10);
    return len;
}

}  // namespace fmt
}  // namespace pvb
