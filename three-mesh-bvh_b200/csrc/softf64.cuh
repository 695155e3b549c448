// IEEE-754 binary64 arithmetic in 64-bit integer operations (round to nearest, ties to even).
//
// The device never executes an FP64 instruction; where a result must match the reference's
// JavaScript double arithmetic bit for bit (the SAH build's split decisions, bin indices and split
// positions, the exact fallback of the oriented-box tests), these functions compute the correctly
// rounded binary64 result of each operation on the same operands, so a sequence of them reproduces
// the reference's sequence of double operations exactly.
//
// Methods: the operand unpacking, alignment with a sticky bit and round-to-nearest-even packing
// follow IEEE 754-2008 section 4.3 and the guard/round/sticky argument of D. Goldberg, "What
// every computer scientist should know about floating-point arithmetic" (1991), section 1.4;
// division is restoring binary long division and the square root is the digit-by-digit
// (two bits per step) integer square root, both with the remainder folded into a sticky bit.
//
// Values are carried as their bit patterns (uint64_t).  Internally a finite nonzero operand is
// (biased exponent e, significand m) with m's leading one at bit 62, i.e. value = m * 2^(e-1023-62);
// the low 10 bits of m are guard bits.  NaN results are the canonical quiet NaN (the reference
// only ever tests NaN-ness).  Compiles for host and device.
#pragma once

#include <cstdint>

// Small helpers are inlined; the arithmetic routines are kept out of line (one copy per
// translation unit) so that kernels calling them from many places stay small in the
// instruction cache.
#ifdef __CUDACC__
#define BVHC_SF_HD __host__ __device__ __forceinline__
#define BVHC_SF_NI static __host__ __device__ __noinline__
#else
#define BVHC_SF_HD inline
#define BVHC_SF_NI [[maybe_unused]] static
#endif

namespace bvhc {
namespace sf {

typedef uint64_t f64;

constexpr uint64_t kSign = 0x8000000000000000ull;
constexpr uint64_t kFrac = 0x000FFFFFFFFFFFFFull;
constexpr f64 kInf = 0x7FF0000000000000ull;
constexpr f64 kNaN = 0x7FF8000000000000ull;
constexpr f64 kOne = 0x3FF0000000000000ull;

BVHC_SF_HD int clz64(uint64_t x) {  // x != 0
#ifdef __CUDA_ARCH__
  return __clzll((long long)x);
#else
  return __builtin_clzll(x);
#endif
}

BVHC_SF_HD int clz32(uint32_t x) {  // x != 0
#ifdef __CUDA_ARCH__
  return __clz((int)x);
#else
  return __builtin_clz(x);
#endif
}

BVHC_SF_HD uint64_t mul_hi(uint64_t a, uint64_t b) {
#ifdef __CUDA_ARCH__
  return __umul64hi(a, b);
#else
  return (uint64_t)(((unsigned __int128)a * b) >> 64);
#endif
}

BVHC_SF_HD bool is_nan(f64 a) { return (a & ~kSign) > kInf; }
BVHC_SF_HD bool is_inf(f64 a) { return (a & ~kSign) == kInf; }
BVHC_SF_HD bool is_zero(f64 a) { return (a & ~kSign) == 0; }
BVHC_SF_HD f64 neg(f64 a) { return a ^ kSign; }
BVHC_SF_HD f64 abs(f64 a) { return a & ~kSign; }

// x >> n, with every bit shifted out OR-ed into bit 0.
BVHC_SF_HD uint64_t shr_jam(uint64_t x, int n) {
  if (n <= 0) return x;
  if (n >= 64) return x != 0;
  return (x >> n) | (uint64_t)((x << (64 - n)) != 0);
}

// Rounds sign * m * 2^(e-1023-62) to binary64 (m normalised to bit 62 when e >= 1).
BVHC_SF_NI f64 round_pack(uint64_t sign, int e, uint64_t m) {
  if (e >= 0x7FF) return sign | kInf;
  if (e < 1) {  // below the normal range: denormalise to the scale of e = 1
    m = shr_jam(m, 1 - e);
    e = 1;
  }
  const uint64_t rb = m & 0x3FF;
  m >>= 10;
  if (rb > 0x200 || (rb == 0x200 && (m & 1))) ++m;
  if (m >= (1ull << 53)) {  // the rounding carried into a new leading bit
    m >>= 1;
    ++e;
    if (e >= 0x7FF) return sign | kInf;
  }
  if (m < (1ull << 52)) return sign | m;  // subnormal (exponent field 0) or zero
  return sign | ((uint64_t)e << 52) | (m & kFrac);
}

// Finite nonzero a: biased exponent (may be <= 0 for subnormals) and m with its leading one at bit 62.
BVHC_SF_HD int unpack(f64 a, uint64_t& m) {
  const int e = (int)((a >> 52) & 0x7FF);
  const uint64_t f = a & kFrac;
  if (e != 0) {
    m = (f | (1ull << 52)) << 10;
    return e;
  }
  const int lead = 63 - clz64(f);  // subnormal: value = f * 2^-1074
  m = f << (62 - lead);
  return 1 - (52 - lead);
}

BVHC_SF_NI f64 add(f64 a, f64 b) {
  if (is_nan(a) || is_nan(b)) return kNaN;
  uint64_t sa = a & kSign, sb = b & kSign;
  if (is_inf(a)) return (is_inf(b) && sa != sb) ? kNaN : a;
  if (is_inf(b)) return b;
  if (is_zero(a)) return is_zero(b) ? (sa & sb) : b;
  if (is_zero(b)) return a;
  uint64_t ma, mb;
  int ea = unpack(a, ma), eb = unpack(b, mb);
  if (ea < eb || (ea == eb && ma < mb)) {  // a gets the larger magnitude (and the result's sign)
    uint64_t t = ma; ma = mb; mb = t;
    int te = ea; ea = eb; eb = te;
    t = sa; sa = sb; sb = t;
  }
  mb = shr_jam(mb, ea - eb);
  if (sa == sb) {
    uint64_t s = ma + mb;  // both below 2^63
    if (s & kSign) {
      s = shr_jam(s, 1);
      ++ea;
    }
    return round_pack(sa, ea, s);
  }
  uint64_t d = ma - mb;
  if (d == 0) return 0;  // exact cancellation is +0 when rounding to nearest
  const int sh = clz64(d) - 1;
  return round_pack(sa, ea - sh, d << sh);
}

BVHC_SF_HD f64 sub(f64 a, f64 b) { return add(a, is_nan(b) ? b : neg(b)); }

BVHC_SF_NI f64 mul(f64 a, f64 b) {
  if (is_nan(a) || is_nan(b)) return kNaN;
  const uint64_t s = (a ^ b) & kSign;
  if (is_inf(a) || is_inf(b)) return (is_zero(a) || is_zero(b)) ? kNaN : (s | kInf);
  if (is_zero(a) || is_zero(b)) return s;
  uint64_t ma, mb;
  int e = unpack(a, ma) + unpack(b, mb) - 1023;
  const uint64_t x = ma >> 10, y = mb >> 10;  // 53-bit significands
  const uint64_t lo = x * y, hi = mul_hi(x, y);  // product in [2^104, 2^106)
  uint64_t m = (hi << 22) | (lo >> 42) | (uint64_t)((lo & ((1ull << 42) - 1)) != 0);
  if (m & kSign) {
    m = shr_jam(m, 1);
    ++e;
  }
  return round_pack(s, e, m);
}

BVHC_SF_NI f64 div(f64 a, f64 b) {
  if (is_nan(a) || is_nan(b)) return kNaN;
  const uint64_t s = (a ^ b) & kSign;
  if (is_inf(a)) return is_inf(b) ? kNaN : (s | kInf);
  if (is_inf(b)) return s;
  if (is_zero(b)) return is_zero(a) ? kNaN : (s | kInf);
  if (is_zero(a)) return s;
  uint64_t ma, mb;
  int e = unpack(a, ma) - unpack(b, mb) + 1023;
  const uint64_t y = mb >> 10;
  uint64_t r = ma >> 10, q = 0;
  if (r >= y) {
    r -= y;
    q = 1;
  }
  for (int i = 0; i < 62; ++i) {  // q = floor(x * 2^62 / y), r the remainder
    r <<= 1;
    q <<= 1;
    if (r >= y) {
      r -= y;
      q |= 1;
    }
  }
  q |= (uint64_t)(r != 0);
  if (!(q & (1ull << 62))) {
    q <<= 1;
    --e;
  }
  return round_pack(s, e, q);
}

BVHC_SF_NI f64 sqrt(f64 a) {
  if (is_nan(a)) return kNaN;
  if (is_zero(a)) return a;
  if (a & kSign) return kNaN;
  if (is_inf(a)) return a;
  uint64_t m;
  int u = unpack(a, m) - 1023;  // a = m * 2^(u-62)
  unsigned __int128 x = (unsigned __int128)m << 62;
  if (u & 1) {
    x <<= 1;
    --u;
  }
  // root = floor(sqrt(x)) in [2^62, 2^63): two radicand bits per step
  unsigned __int128 rem = 0, root = 0;
  for (int i = 63; i >= 0; --i) {
    rem = (rem << 2) | (unsigned __int128)((x >> (2 * i)) & 3);
    const unsigned __int128 trial = (root << 2) | 1;
    if (rem >= trial) {
      rem -= trial;
      root = (root << 1) | 1;
    } else {
      root <<= 1;
    }
  }
  return round_pack(0, u / 2 + 1023, (uint64_t)root | (uint64_t)(rem != 0));
}

// Ordering key: monotone in the value, with -0 and +0 equal.
BVHC_SF_HD int64_t order_key(f64 a) {
  return (a & kSign) ? -(int64_t)(a & ~kSign) : (int64_t)a;
}
BVHC_SF_HD bool lt(f64 a, f64 b) { return !is_nan(a) && !is_nan(b) && order_key(a) < order_key(b); }
BVHC_SF_HD bool le(f64 a, f64 b) { return !is_nan(a) && !is_nan(b) && order_key(a) <= order_key(b); }
BVHC_SF_HD bool eq(f64 a, f64 b) { return !is_nan(a) && !is_nan(b) && order_key(a) == order_key(b); }

BVHC_SF_HD uint32_t f32_bits(float x) {
#ifdef __CUDA_ARCH__
  return (uint32_t)__float_as_uint(x);
#else
  uint32_t u;
  __builtin_memcpy(&u, &x, 4);
  return u;
#endif
}
BVHC_SF_HD float f32_from_bits(uint32_t u) {
#ifdef __CUDA_ARCH__
  return __uint_as_float(u);
#else
  float x;
  __builtin_memcpy(&x, &u, 4);
  return x;
#endif
}

// Exact widening of a float32.
BVHC_SF_HD f64 from_f32(float x) {
  const uint32_t u = f32_bits(x);
  const uint64_t s = (uint64_t)(u >> 31) << 63;
  const int e = (int)((u >> 23) & 0xFF);
  const uint32_t f = u & 0x7FFFFF;
  if (e == 0xFF) return f ? kNaN : (s | kInf);
  if (e == 0) {
    if (f == 0) return s;
    const int lead = 31 - clz32(f);  // subnormal: f * 2^-149
    return s | ((uint64_t)(lead - 149 + 1023) << 52) | (((uint64_t)f << (52 - lead)) & kFrac);
  }
  return s | ((uint64_t)(e - 127 + 1023) << 52) | ((uint64_t)f << 29);
}

// Round to the nearest float32, ties to even (JavaScript's Math.fround / a Float32Array store).
BVHC_SF_NI float to_f32(f64 a) {
  const uint32_t s = (uint32_t)(a >> 63) << 31;
  if (is_nan(a)) return f32_from_bits(0x7FC00000u);
  if (is_inf(a)) return f32_from_bits(s | 0x7F800000u);
  const int e = (int)((a >> 52) & 0x7FF);
  if (e == 0) return f32_from_bits(s);  // binary64 subnormals are far below float32's range
  const uint64_t m = (a & kFrac) | (1ull << 52);  // a = m * 2^(e-1075)
  int E = e - 896;                                // float32 biased exponent
  int shift = E >= 1 ? 29 : 29 + (1 - E);         // bits of m below the float32 result's unit
  if (shift > 54) return f32_from_bits(s);
  uint64_t q = m >> shift;
  const uint64_t rem = m & ((1ull << shift) - 1), half = 1ull << (shift - 1);
  if (rem > half || (rem == half && (q & 1))) ++q;
  if (E >= 1) {
    if (q >= (1u << 24)) {
      q >>= 1;
      ++E;
    }
    if (E >= 0xFF) return f32_from_bits(s | 0x7F800000u);
    return f32_from_bits(s | ((uint32_t)E << 23) | ((uint32_t)q & 0x7FFFFF));
  }
  return f32_from_bits(s | (uint32_t)q);  // subnormal; q == 2^23 encodes the smallest normal
}

// Nonnegative integers (exact below 2^53, rounded above).
BVHC_SF_NI f64 from_u64(uint64_t x) {
  if (x == 0) return 0;
  const int lead = 63 - clz64(x);
  const uint64_t m = lead <= 62 ? x << (62 - lead) : shr_jam(x, lead - 62);
  return round_pack(0, lead + 1023, m);
}

// Truncation toward zero for |a| < 2^31 (JavaScript's `~~a` there); NaN gives 0.
BVHC_SF_NI int to_i32_trunc(f64 a) {
  if (is_nan(a)) return 0;
  const int e = (int)((a >> 52) & 0x7FF);
  if (e < 1023) return 0;
  const uint64_t m = (a & kFrac) | (1ull << 52);
  const int sh = 1075 - e;
  const uint64_t v = sh >= 0 ? (sh >= 64 ? 0 : m >> sh) : m << (-sh);
  return (a & kSign) ? -(int)v : (int)v;
}

}  // namespace sf
}  // namespace bvhc
