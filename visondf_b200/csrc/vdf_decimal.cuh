// vdf_decimal.cuh -- text fields to numbers with the semantics the reference's
// CSV reader gets from its parsers:
//   * doubles: fast_float::from_chars (v8.1.0, vendored at
//     V/external/fast_float, called from V/inlines/classify_column.inl:42 and
//     V/inlines/read/read_csv/type_inference/type_classification.inl:106-108):
//     the C++17 from_chars grammar for chars_format::general (optional '-',
//     digits with an optional '.', optional exponent; "nan", "inf",
//     "infinity" in any case), the longest valid prefix, correctly rounded to
//     nearest-even; the caller stores 0 when it is invalid or out of range
//     (overflow to infinity, or a nonzero decimal that rounds to zero);
//   * unsigned / signed 32-bit integers: std::from_chars into unsigned int /
//     int (classify_column.inl:98-117), 0 when invalid or out of range.
//
// The conversion to double is exact in three steps (own code; published
// methods named at each step):
//   1. Clinger's fast path (W. D. Clinger, "How to read floating point numbers
//      accurately", PLDI 1990): w <= 2^53 and |q| <= 22 need one IEEE
//      multiplication or division by an exact power of ten;
//   2. otherwise the product of w and a 128-bit truncation F of 5^q (the
//      product form of Eisel-Lemire, D. Lemire, "Number parsing at a gigabyte
//      per second", SPE 2021).  The true product lies in [P, P + 2^64 - 1]
//      (F_true - F < 1, w < 2^64); when both ends round to the same double,
//      so does the true value (rounding is monotone);
//   3. when they do not (a halfway point falls inside the interval, or more
//      than 19 significant digits make w and w + 1 disagree), the field is
//      decided exactly: big-integer comparison of the decimal against the
//      halfway point between the two candidate doubles (slow_decide below).
// Everything here is __host__ __device__ so the same code can be checked on
// the host against the reference's parser.
#pragma once
#include <stdint.h>

#ifdef __CUDACC__
#define VDF_HD __host__ __device__ __forceinline__
#define VDF_HDN __host__ __device__ __noinline__
#else
#define VDF_HD inline
#define VDF_HDN inline
#endif

#include "vdf_pow5.inc"

namespace vdfdec {

#ifdef __CUDACC__
__device__ const uint64_t kPow5HiDev[] = {VDF_POW5_HI_DATA};
__device__ const uint64_t kPow5LoDev[] = {VDF_POW5_LO_DATA};
__device__ const int16_t kPow5EDev[] = {VDF_POW5_E_DATA};
#endif
static const uint64_t kPow5HiHost[] = {VDF_POW5_HI_DATA};
static const uint64_t kPow5LoHost[] = {VDF_POW5_LO_DATA};
static const int16_t kPow5EHost[] = {VDF_POW5_E_DATA};

VDF_HD uint64_t pow5_hi(int i) {
#ifdef __CUDA_ARCH__
    return __ldg(&kPow5HiDev[i]);
#else
    return kPow5HiHost[i];
#endif
}
VDF_HD uint64_t pow5_lo(int i) {
#ifdef __CUDA_ARCH__
    return __ldg(&kPow5LoDev[i]);
#else
    return kPow5LoHost[i];
#endif
}
VDF_HD int pow5_e(int i) {
#ifdef __CUDA_ARCH__
    return kPow5EDev[i];
#else
    return kPow5EHost[i];
#endif
}

VDF_HD uint64_t mulhi64(uint64_t a, uint64_t b) {
#ifdef __CUDA_ARCH__
    return __umul64hi(a, b);
#else
    return (uint64_t)(((unsigned __int128)a * b) >> 64);
#endif
}
VDF_HD int clz64(uint64_t x) {  // x != 0
#ifdef __CUDA_ARCH__
    return __clzll((long long)x);
#else
    return __builtin_clzll(x);
#endif
}
VDF_HD double bits_to_double(uint64_t b) {
#ifdef __CUDA_ARCH__
    return __longlong_as_double((long long)b);
#else
    double d;
    __builtin_memcpy(&d, &b, 8);
    return d;
#endif
}
VDF_HD double dmul_rn(double a, double b) {
#ifdef __CUDA_ARCH__
    return __dmul_rn(a, b);
#else
    return a * b;
#endif
}
VDF_HD double ddiv_rn(double a, double b) {
#ifdef __CUDA_ARCH__
    return __ddiv_rn(a, b);
#else
    return a / b;
#endif
}

VDF_HD bool is_digit(unsigned char c) { return (unsigned)(c - '0') < 10u; }
VDF_HD unsigned char lower(unsigned char c) { return (c >= 'A' && c <= 'Z') ? (unsigned char)(c + 32) : c; }

// ---------------------------------------------------------------- scanning
enum Kind : int { kInvalid = 0, kFinite = 1, kInf = 2, kNaN = 3 };

// A scanned decimal: value = w * 10^q (plus dropped digits when `many`).
struct Number {
    uint64_t w;
    int64_t q;
    int kind;
    bool neg;
    bool many;  // a nonzero significant digit after the 19th was dropped
};

constexpr int kMaxW = 19;          // 10^19 - 1 < 2^64
constexpr int64_t kExpCap = 1 << 30;

// `p`..`end`: the field's bytes, read through `at(i)` so device callers can
// supply their own cached byte reader.
template <typename At>
VDF_HD Number scan_number(At at, uint32_t len) {
    Number r{0, 0, kInvalid, false, false};
    uint32_t i = 0;
    if (len == 0) return r;
    r.neg = at(0) == '-';
    if (r.neg) i = 1;
    const uint32_t sign_end = i;
    uint64_t w = 0;
    int nd = 0;
    int64_t q = 0;
    bool seen = false, many = false;
    while (i < len) {
        const unsigned char c = at(i);
        if (!is_digit(c)) break;
        const uint32_t d = c - '0';
        seen = true;
        if (nd == 0 && d == 0) {
        } else if (nd < kMaxW) {
            w = w * 10 + d;
            ++nd;
        } else {
            ++q;
            many |= d != 0;
        }
        ++i;
    }
    if (i < len && at(i) == '.') {
        ++i;
        while (i < len) {
            const unsigned char c = at(i);
            if (!is_digit(c)) break;
            const uint32_t d = c - '0';
            seen = true;
            if (nd == 0 && d == 0) {
                --q;
            } else if (nd < kMaxW) {
                w = w * 10 + d;
                ++nd;
                --q;
            } else {
                many |= d != 0;
            }
            ++i;
        }
    }
    if (!seen) {
        // not a number: "nan" / "inf" after the optional '-'
        i = sign_end;
        if (len - i >= 3) {
            const unsigned char a = lower(at(i)), b = lower(at(i + 1)), c = lower(at(i + 2));
            if (a == 'n' && b == 'a' && c == 'n') r.kind = kNaN;
            else if (a == 'i' && b == 'n' && c == 'f') r.kind = kInf;
        }
        return r;
    }
    if (i < len && (at(i) == 'e' || at(i) == 'E')) {
        uint32_t j = i + 1;
        bool eneg = false;
        if (j < len && (at(j) == '+' || at(j) == '-')) {
            eneg = at(j) == '-';
            ++j;
        }
        if (j < len && is_digit(at(j))) {
            int64_t e = 0;
            while (j < len && is_digit(at(j))) {
                if (e < kExpCap) e = e * 10 + (at(j) - '0');
                ++j;
            }
            q += eneg ? -e : e;
        }
    }
    r.w = w;
    r.q = q;
    r.kind = kFinite;
    r.many = many;
    return r;
}

// ------------------------------------------------------ eight at a time
// Top bit of each byte set exactly where the byte is an ASCII digit: for a
// byte b below 0x80, (b & 0x7f) + 0x50 reaches 0x80 iff b >= '0' and
// (b & 0x7f) + 0x46 reaches 0x80 iff b > '9'; neither sum carries into the
// next byte.
VDF_HD uint64_t digit_bytes(uint64_t v) {
    const uint64_t low = v & 0x7f7f7f7f7f7f7f7full;
    const uint64_t ge0 = low + 0x5050505050505050ull;
    const uint64_t gt9 = low + 0x4646464646464646ull;
    return ge0 & ~gt9 & ~v & 0x8080808080808080ull;
}

// Number of leading digit bytes (byte 0 first) of v, 0..8.
VDF_HD int digit_run(uint64_t v) {
    const uint64_t stop = ~digit_bytes(v) & 0x8080808080808080ull;
    if (!stop) return 8;
#ifdef __CUDA_ARCH__
    return (__ffsll((long long)stop) - 1) >> 3;
#else
    return __builtin_ctzll(stop) >> 3;
#endif
}

// The value of the k leading digit bytes of v (k <= 8): the digits are moved
// to the top k bytes (zeros before them read as leading zeros), then adjacent
// digits combine pairwise three times -- x*10 + y per byte pair, per 16-bit
// pair (x*100 + y) and per 32-bit pair (x*10^4 + y) -- each by one multiply
// whose cross terms land outside the kept lanes.
VDF_HD uint64_t digits_value(uint64_t v, int k) {
    if (k == 0) return 0;
    const uint64_t mask = k == 8 ? ~0ull : ((1ull << (8 * k)) - 1);
    uint64_t d = (v & mask) - (0x3030303030303030ull & mask);
    d <<= 8 * (8 - k);
    d = ((d * (1 + (10ull << 8))) >> 8) & 0x00ff00ff00ff00ffull;
    d = ((d * (1 + (100ull << 16))) >> 16) & 0x0000ffff0000ffffull;
    return (d * (1 + (10000ull << 32))) >> 32;
}

VDF_HD uint64_t pow10_small(int k) {  // 10^k, k <= 8
    uint64_t p = 1;
    for (int i = 0; i < k; ++i) p *= 10;
    return p;
}

// The common field shape [-]d{0,7}[.d{0,7}] (at least one digit, then the
// end of the field or a byte other than 'e' / 'E') read eight bytes at a
// time; any other shape returns false and goes through scan_number, which
// gives the same Number for the shapes accepted here.  `src.get8(i, avail)`
// returns the 8 bytes at i with the bytes at and past `avail` zeroed.
template <typename Src>
VDF_HD bool scan_number_fast(Src& src, uint64_t fs, uint32_t len, Number& out) {
    if (len == 0) return false;
    uint32_t i = 0;
    const bool neg = src.get(fs) == '-';
    if (neg) i = 1;
    const uint64_t v1 = src.get8(fs + i, len - i);
    const int k1 = digit_run(v1);
    if (k1 == 8) return false;
    uint64_t w = digits_value(v1, k1);
    int64_t q = 0;
    i += k1;
    if (i < len) {
        const unsigned char c = (unsigned char)(v1 >> (8 * k1));
        if (c == '.') {
            ++i;
            const uint64_t v2 = i < len ? src.get8(fs + i, len - i) : 0;
            const int k2 = digit_run(v2);
            if (k2 == 8 || k1 + k2 == 0) return false;
            w = w * pow10_small(k2) + digits_value(v2, k2);
            q = -k2;
            i += k2;
            if (i < len) {
                const unsigned char e = (unsigned char)(v2 >> (8 * k2));
                if (e == 'e' || e == 'E') return false;
            }
        } else if (c == 'e' || c == 'E' || k1 == 0) {
            return false;
        }
    } else if (k1 == 0) {
        return false;
    }
    out.w = w;
    out.q = q;
    out.kind = kFinite;
    out.neg = neg;
    out.many = false;
    return true;
}

// ---------------------------------------------------------- conversion
struct U192 {
    uint64_t p0, p1, p2;
};

VDF_HD U192 mul_64x128(uint64_t a, uint64_t hi, uint64_t lo) {
    const uint64_t l0 = a * lo, l1 = mulhi64(a, lo);
    const uint64_t h0 = a * hi, h1 = mulhi64(a, hi);
    U192 r;
    r.p0 = l0;
    r.p1 = l1 + h0;
    r.p2 = h1 + (r.p1 < l1 ? 1u : 0u);
    return r;
}

// The approximate product for w * 10^q: P (192 bits) with value = P * 2^scale,
// P in [2^190, 2^192); `exact` when the table entry is exact.
struct Product {
    U192 p;
    int scale;
    bool exact;
};

VDF_HD Product product_of(uint64_t w, int q) {
    const int lz = clz64(w);
    const int i = q - VDF_POW5_QMIN;
    Product r;
    r.p = mul_64x128(w << lz, pow5_hi(i), pow5_lo(i));
    r.scale = pow5_e(i) - lz + q;
    r.exact = q >= 0 && q <= 55;
    return r;
}

// Rounds P * 2^scale (P >= 2^190) to nearest-even; returns the magnitude's
// bits (0x7ff0... for overflow).
VDF_HD uint64_t round_product(U192 p, int scale) {
    const int t = (p.p2 >> 63) ? 191 : 190;
    const int E = t + scale;  // value in [2^E, 2^(E+1))
    if (E > 1023) return 0x7ff0000000000000ull;
    const int ulp_exp = E - 52 > -1074 ? E - 52 : -1074;
    const int s = ulp_exp - scale;  // bit index of the ulp inside P
    if (s > 192) return 0;  // the half-ulp bit (s - 1) lies above P: below 2^-1075
    if (s == 192) {
        // half-ulp (2^-1075) is bit 191: below it when P < 2^191, a tie when
        // P == 2^191 exactly (rounds to even, 0), above it otherwise
        if (t == 190) return 0;
        const bool exact_pow2 = p.p2 == (1ull << 63) && p.p1 == 0 && p.p0 == 0;
        return exact_pow2 ? 0 : 1;
    }
    // s in [138, 191]: the kept bits and the rounding bits are all in p2 / below
    const int sh = s - 128;  // in [10, 63]
    uint64_t m = p.p2 >> sh;
    const uint64_t rest = p.p2 & ((1ull << sh) - 1);
    const uint64_t half = 1ull << (sh - 1);
    bool up;
    if (rest != half) up = rest > half;
    else if (p.p1 | p.p0) up = true;
    else up = (m & 1) != 0;
    m += up ? 1 : 0;
    const uint64_t bits = ((uint64_t)(ulp_exp + 1074) << 52) + m;
    return bits >= 0x7ff0000000000000ull ? 0x7ff0000000000000ull : bits;
}

// The double nearest w * 10^q for w in [1, 2^64), q in the table's range, or
// `ambiguous` when the truncated table cannot decide.
VDF_HD uint64_t product_bits(uint64_t w, int q, bool& ambiguous) {
    const Product pr = product_of(w, q);
    const uint64_t lo = round_product(pr.p, pr.scale);
    if (pr.exact) return lo;
    U192 u = pr.p;  // P + 2^64 - 1 (no overflow: P <= (2^64-1)(2^128-1))
    const uint64_t add = ~0ull;
    const uint64_t n0 = u.p0 + add;
    const uint64_t c0 = n0 < u.p0 ? 1 : 0;
    const uint64_t n1 = u.p1 + c0;
    const uint64_t c1 = n1 < u.p1 ? 1 : 0;
    u.p0 = n0;
    u.p1 = n1;
    u.p2 += c1;
    if (round_product(u, pr.scale) != lo) ambiguous = true;
    return lo;
}

struct Conv {
    double v;        // the value the reference stores (0 when invalid / out of range)
    bool ambiguous;  // needs slow_decide
};

VDF_HD Conv convert(const Number& n) {
    Conv r{0.0, false};
    const uint64_t sign = n.neg ? (1ull << 63) : 0;
    if (n.kind == kInvalid) return r;
    if (n.kind == kNaN) {
        r.v = bits_to_double(sign | 0x7ff8000000000000ull);
        return r;
    }
    if (n.kind == kInf) {
        r.v = bits_to_double(sign | 0x7ff0000000000000ull);
        return r;
    }
    if (n.w == 0) {
        r.v = bits_to_double(sign);
        return r;
    }
    if (!n.many && n.w <= (1ull << 53) && n.q >= -22 && n.q <= 22) {
        // exact powers of ten 1e0..1e22 (each fits in 53 bits times a power of two)
        double p10 = 1.0;
        const int aq = n.q < 0 ? (int)-n.q : (int)n.q;
        double b = 10.0;
        for (int e = aq; e; e >>= 1, b = b * b)
            if (e & 1) p10 *= b;
        const double x = (double)n.w;
        const double v = n.q < 0 ? ddiv_rn(x, p10) : dmul_rn(x, p10);
        r.v = n.neg ? -v : v;
        return r;
    }
    if (n.q < VDF_POW5_QMIN) return r;  // below 1e-323 / 2: rounds to zero -> out of range
    if (n.q > VDF_POW5_QMAX) return r;  // at least 1e309: infinity -> out of range
    bool amb = false;
    uint64_t bits = product_bits(n.w, (int)n.q, amb);
    if (n.many) {
        // the true digits lie in [w, w + 1) * 10^q
        const uint64_t hi = product_bits(n.w + 1, (int)n.q, amb);
        if (hi != bits) amb = true;
    }
    if (amb) {
        r.ambiguous = true;
        return r;
    }
    if (bits == 0 || bits >= 0x7ff0000000000000ull) return r;  // out of range
    r.v = bits_to_double(sign | bits);
    return r;
}

// ------------------------------------------------------------ slow path
// Exact decision by big-integer comparison.  The decimal D = M * 10^Q (M the
// first kSlowDigits significant digits, `sticky` when nonzero digits follow)
// is compared with the halfway point H = (2m + 1) * 2^(ulp_exp - 1) above the
// candidate m * 2^ulp_exp that truncating the (lower-bound) product gives.
// A halfway point between doubles has at most 767 significant decimal digits,
// so digits past kSlowDigits only break an exact tie (sticky => D > H).
constexpr int kSlowDigits = 800;
constexpr int kLimbs = 48;  // 3072 bits: M < 2^2658, (2m+1) * 5^1142 < 2^2707

struct Big {
    uint64_t l[kLimbs];
    int n;  // used limbs
};

VDF_HD void big_set(Big& a, uint64_t v) {
    a.l[0] = v;
    a.n = v ? 1 : 0;
}
// a = a * m + add; false on overflow
VDF_HD bool big_muladd(Big& a, uint64_t m, uint64_t add) {
    uint64_t carry = add;
    for (int i = 0; i < a.n; ++i) {
        const uint64_t lo = a.l[i] * m, hi = mulhi64(a.l[i], m);
        const uint64_t s = lo + carry;
        carry = hi + (s < lo ? 1 : 0);
        a.l[i] = s;
    }
    if (carry) {
        if (a.n == kLimbs) return false;
        a.l[a.n++] = carry;
    }
    return true;
}
VDF_HD bool big_mulpow5(Big& a, int k) {
    const uint64_t p27 = 7450580596923828125ull;  // 5^27
    while (k >= 27) {
        if (!big_muladd(a, p27, 0)) return false;
        k -= 27;
    }
    uint64_t p = 1;
    while (k-- > 0) p *= 5;
    return big_muladd(a, p, 0);
}
VDF_HD bool big_shl(Big& a, int bits) {
    if (a.n == 0 || bits == 0) return true;
    const int limbs = bits >> 6, b = bits & 63;
    const int nn = a.n + limbs + 1;
    if (nn > kLimbs + 1) return false;
    uint64_t top = b ? (a.l[a.n - 1] >> (64 - b)) : 0;
    if (nn == kLimbs + 1 && top) return false;
    for (int i = a.n - 1; i >= 0; --i) {
        const uint64_t hi = a.l[i] << b;
        const uint64_t lo = (b && i > 0) ? (a.l[i - 1] >> (64 - b)) : 0;
        a.l[i + limbs] = hi | lo;
    }
    for (int i = 0; i < limbs; ++i) a.l[i] = 0;
    a.n += limbs;
    if (top) a.l[a.n++] = top;
    return true;
}
VDF_HD int big_cmp(const Big& a, const Big& b) {
    if (a.n != b.n) return a.n < b.n ? -1 : 1;
    for (int i = a.n - 1; i >= 0; --i)
        if (a.l[i] != b.l[i]) return a.l[i] < b.l[i] ? -1 : 1;
    return 0;
}

// Re-scans the field and decides it exactly.  `ok` false only if the numbers
// exceed the fixed-size integers (not expected for any input).
template <typename At>
VDF_HDN double slow_decide(At at, uint32_t len, bool& ok) {
    ok = true;
    const Number n = scan_number(at, len);
    // candidate from the lower-bound product of the first 19 digits
    const Product pr = product_of(n.w, (int)n.q);
    const int t = (pr.p.p2 >> 63) ? 191 : 190;
    const int E = t + pr.scale;
    const int ulp_exp = E - 52 > -1074 ? E - 52 : -1074;
    const int s = ulp_exp - pr.scale;
    uint64_t m = 0;
    if (s < 192) m = pr.p.p2 >> (s - 128);
    // M: the first kSlowDigits significant digits (sticky: a nonzero digit
    // after them).  Every kept digit past the 19th moves one decimal place
    // below the point relative to the 19-digit scan, so Q = q - (nd - 19).
    Big a;
    big_set(a, 0);
    bool sticky = false;
    int nd = 0;
    uint64_t chunk = 0, cmul = 1;
    bool frac = false;
    for (uint32_t i = n.neg ? 1 : 0; i < len; ++i) {
        const unsigned char c = at(i);
        if (c == '.' && !frac) {
            frac = true;
            continue;
        }
        if (!is_digit(c)) break;
        const uint32_t d = c - '0';
        if (nd == 0 && d == 0) continue;
        if (nd < kSlowDigits) {
            chunk = chunk * 10 + d;
            cmul *= 10;
            ++nd;
            if (cmul == 10000000000000000000ull) {
                if (!big_muladd(a, cmul, chunk)) ok = false;
                chunk = 0;
                cmul = 1;
            }
        } else {
            sticky |= d != 0;
        }
    }
    if (cmul > 1 && !big_muladd(a, cmul, chunk)) ok = false;
    const int64_t Q = n.q - (int64_t)(nd - (nd < kMaxW ? nd : kMaxW));
    // H = (2m + 1) * 2^(ulp_exp - 1); compare M * 5^Q * 2^Q with it
    Big b;
    big_set(b, 2 * m + 1);
    int64_t e2a = Q, e2b = ulp_exp - 1;
    if (Q >= 0) {
        if (!big_mulpow5(a, (int)Q)) ok = false;
    } else {
        if (!big_mulpow5(b, (int)-Q)) ok = false;
    }
    if (e2a > e2b) {
        if (!big_shl(a, (int)(e2a - e2b))) ok = false;
    } else if (e2b > e2a) {
        if (!big_shl(b, (int)(e2b - e2a))) ok = false;
    }
    int c = big_cmp(a, b);
    if (c == 0 && sticky) c = 1;
    if (c > 0 || (c == 0 && (m & 1))) ++m;
    uint64_t bits = ((uint64_t)(ulp_exp + 1074) << 52) + m;
    if (bits == 0 || bits >= 0x7ff0000000000000ull) return 0.0;  // out of range
    if (n.neg) bits |= 1ull << 63;
    return bits_to_double(bits);
}

// ---------------------------------------------------------- integers
// std::from_chars into unsigned int: digits only, 0 when none or > 2^32 - 1.
template <typename At>
VDF_HD uint32_t parse_u32(At at, uint32_t len) {
    uint64_t v = 0;
    uint32_t i = 0;
    bool over = false;
    while (i < len && is_digit(at(i))) {
        v = v * 10 + (at(i) - '0');
        if (v > 0xffffffffull) {
            over = true;
            v = 0xffffffffull + 1;  // stays above; keep consuming digits
        }
        ++i;
    }
    if (i == 0 || over) return 0;
    return (uint32_t)v;
}
// std::from_chars into int: optional '-', digits; 0 when none or out of range.
template <typename At>
VDF_HD int32_t parse_i32(At at, uint32_t len) {
    uint32_t i = 0;
    const bool neg = len > 0 && at(0) == '-';
    if (neg) i = 1;
    const uint32_t d0 = i;
    uint64_t v = 0;
    bool over = false;
    while (i < len && is_digit(at(i))) {
        v = v * 10 + (at(i) - '0');
        if (v > 0x80000000ull) {
            over = true;
            v = 0x80000001ull;
        }
        ++i;
    }
    if (i == d0 || over) return 0;
    if (!neg && v > 0x7fffffffull) return 0;
    return neg ? (int32_t)(0 - v) : (int32_t)v;
}

}  // namespace vdfdec
