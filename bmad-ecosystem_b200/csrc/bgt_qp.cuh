// bgt_qp.cuh -- IEEE 754 binary128 ("quad precision") arithmetic in software,
// for the device and the host.
//
// The reference carries a particle's time in real(qp) (coord_struct%t,
// bmad_struct.f90:546-574): every element adds a real(rp) step to it
// (track_a_drift.f90:79-80; track_a_quadrupole.f90:144 and the same line in
// track_a_bend / track_a_thick_multipole), and with absolute time tracking
// the RF phase is computed from it in real(qp) before being rounded to
// real(rp) (particle_rf_time.f90:74-76,116-118; track_a_rfcavity.f90:78-80).
// A double-double holds ~106 bits, not binary128's 113, and rounds
// differently; over thousands of additions per turn the difference reaches
// the last bit of the phase.  These routines round exactly as binary128 does
// (to nearest, ties to even), so the device's time and phase are the
// reference's bit for bit.
//
// Scope: finite operands that are normal or zero (a particle time, a double
// converted to binary128, an RF frequency) and results in the normal range.
// NaN or infinite operands give a NaN (a lost particle whose coordinates
// overflowed).  Values keep the binary128 bit layout (lo = bits 0-63,
// hi = bits 64-127: the memory order of a C __float128 or a Fortran real(qp)
// on x86-64), so host arrays pass through unchanged.
#pragma once
#include <stdint.h>
#include <string.h>

#if defined(__CUDACC__)
#define BGT_QP_HD __host__ __device__ __forceinline__
#else
#define BGT_QP_HD static inline
#endif

namespace bgt {
namespace qp {

typedef unsigned __int128 u128;

struct Q {
  uint64_t lo, hi;  // binary128 bits
};

constexpr int BIAS = 16383;
constexpr uint64_t EXP_MASK = 0x7fffull;
constexpr uint64_t FRAC_HI_MASK = (1ull << 48) - 1;

BGT_QP_HD Q make_nan() { return Q{0ull, 0x7fff800000000000ull}; }
BGT_QP_HD Q make_zero(uint64_t sign) { return Q{0ull, sign << 63}; }
BGT_QP_HD bool is_zero(Q a) { return ((a.hi << 1) | a.lo) == 0; }
BGT_QP_HD bool is_special(Q a) { return ((a.hi >> 48) & EXP_MASK) == EXP_MASK; }
BGT_QP_HD Q neg(Q a) { return Q{a.lo, a.hi ^ (1ull << 63)}; }

// leading zeros of a nonzero 64-bit word
BGT_QP_HD int clz64(uint64_t x) {
#if defined(__CUDA_ARCH__)
  return __clzll((long long)x);
#else
  return __builtin_clzll(x);
#endif
}

BGT_QP_HD int clz128(u128 x) {
  const uint64_t h = (uint64_t)(x >> 64);
  if (h) return clz64(h);
  const uint64_t l = (uint64_t)x;
  return l ? 64 + clz64(l) : 128;
}

// Significand with the hidden bit (113 bits) and unbiased exponent of a
// normal value.
BGT_QP_HD u128 sig_of(Q a) { return ((u128)((a.hi & FRAC_HI_MASK) | (1ull << 48)) << 64) | a.lo; }
BGT_QP_HD int exp_of(Q a) { return (int)((a.hi >> 48) & EXP_MASK) - BIAS; }

// Pack sign, unbiased exponent e of the leading bit and a significand m in
// [2^115, 2^116) that carries 3 extra low bits (guard, round, sticky) --
// the value m * 2^(e - 115) -- rounding to nearest, ties to even.
BGT_QP_HD Q round_pack(uint64_t sign, int e, u128 m) {
  const uint32_t grs = (uint32_t)(m & 7u);
  m >>= 3;  // 113 bits
  if (grs > 4 || (grs == 4 && (m & 1u))) {
    m += 1;
    if (m >> 113) {  // carried into a new leading bit
      m >>= 1;
      e += 1;
    }
  }
  const uint64_t be = (uint64_t)(e + BIAS);
  return Q{(uint64_t)m, (sign << 63) | (be << 48) | ((uint64_t)(m >> 64) & FRAC_HI_MASK)};
}

// Right shift keeping a sticky bit (any bit shifted out ORed into bit 0).
BGT_QP_HD u128 shr_sticky(u128 x, int s) {
  if (s <= 0) return x;
  if (s >= 128) return x != 0 ? 1 : 0;
  const u128 out = x >> s;
  return out | ((x << (128 - s)) != 0 ? 1 : 0);
}

// Exact conversion of a double.
BGT_QP_HD Q from_double(double d) {
  uint64_t b;
  memcpy(&b, &d, 8);
  const uint64_t sign = b >> 63;
  const int ex = (int)((b >> 52) & 0x7ff);
  uint64_t fr = b & ((1ull << 52) - 1);
  if (ex == 0x7ff) return make_nan();
  if (ex == 0) {
    if (fr == 0) return make_zero(sign);
    // subnormal double fr * 2^-1074: normalised (binary128 holds it as a
    // normal number); lz = 52 - (index of the leading bit)
    const int lz = clz64(fr) - 11;
    fr = (fr << lz) & ((1ull << 52) - 1);
    const int e = -1022 - lz;
    return Q{fr << 60, (sign << 63) | ((uint64_t)(e + BIAS) << 48) | (fr >> 4)};
  }
  const int e = ex - 1023;
  return Q{fr << 60, (sign << 63) | ((uint64_t)(e + BIAS) << 48) | (fr >> 4)};
}

// Nearest double, ties to even (results in the normal double range, or
// zero).
BGT_QP_HD double to_double(Q a) {
  const uint64_t sign = a.hi >> 63;
  double r;
  if (is_special(a)) {
    const uint64_t nb = 0x7ff8000000000000ull;
    memcpy(&r, &nb, 8);
    return r;
  }
  if (is_zero(a)) {
    const uint64_t zb = sign << 63;
    memcpy(&r, &zb, 8);
    return r;
  }
  int e = exp_of(a);
  const u128 m = sig_of(a);  // 113 bits
  const u128 rest = m & ((((u128)1) << 60) - 1);
  uint64_t k = (uint64_t)(m >> 60);  // 53 bits
  const u128 half = ((u128)1) << 59;
  if (rest > half || (rest == half && (k & 1u))) {
    k += 1;
    if (k >> 53) {
      k >>= 1;
      e += 1;
    }
  }
  const uint64_t bits = (sign << 63) | ((uint64_t)(e + 1023) << 52) | (k & ((1ull << 52) - 1));
  memcpy(&r, &bits, 8);
  return r;
}

// a + b, correctly rounded.
BGT_QP_HD Q add(Q a, Q b) {
  if (is_special(a) || is_special(b)) return make_nan();
  if (is_zero(a)) {
    if (is_zero(b)) return make_zero((a.hi >> 63) & (b.hi >> 63));  // -0 only for -0 + -0
    return b;
  }
  if (is_zero(b)) return a;
  int ea = exp_of(a), eb = exp_of(b);
  u128 ma = sig_of(a) << 3, mb = sig_of(b) << 3;  // room for guard, round and sticky bits
  uint64_t sa = a.hi >> 63, sb = b.hi >> 63;
  // order by magnitude: |a| >= |b|
  if (eb > ea || (eb == ea && mb > ma)) {
    const int te = ea;
    ea = eb;
    eb = te;
    const u128 tm = ma;
    ma = mb;
    mb = tm;
    const uint64_t ts = sa;
    sa = sb;
    sb = ts;
  }
  mb = shr_sticky(mb, ea - eb);
  int e = ea;
  u128 m;
  if (sa == sb) {
    m = ma + mb;
    if (m >> 116) {  // one more leading bit
      m = shr_sticky(m, 1);
      e += 1;
    }
  } else {
    m = ma - mb;
    if (m == 0) return make_zero(0);  // exact cancellation: +0 when rounding to nearest
    // the leading bit back to bit 115 (exact: when more than one bit
    // cancels, b was shifted by at most one place and lost nothing)
    const int lz = clz128(m) - (127 - 115);
    if (lz > 0) {
      m <<= lz;
      e -= lz;
    }
  }
  return round_pack(sa, e, m);
}

BGT_QP_HD Q sub(Q a, Q b) { return add(a, neg(b)); }

// a * b, correctly rounded.
BGT_QP_HD Q mul(Q a, Q b) {
  if (is_special(a) || is_special(b)) return make_nan();
  const uint64_t sign = (a.hi ^ b.hi) >> 63;
  if (is_zero(a) || is_zero(b)) return make_zero(sign);
  const u128 ma = sig_of(a), mb = sig_of(b);
  const uint64_t a0 = (uint64_t)ma, a1 = (uint64_t)(ma >> 64);  // a1 < 2^49
  const uint64_t b0 = (uint64_t)mb, b1 = (uint64_t)(mb >> 64);
  // the 226-bit product as (hi:lo) 128-bit halves
  const u128 p00 = (u128)a0 * b0;
  const u128 p01 = (u128)a0 * b1;
  const u128 p10 = (u128)a1 * b0;
  const u128 p11 = (u128)a1 * b1;
  u128 lo = p00;
  u128 hi = p11;
  const u128 mid = p01 + p10;  // < 2^114, no overflow
  const u128 mid_lo = mid << 64;
  lo += mid_lo;
  hi += (mid >> 64) + (lo < mid_lo ? 1 : 0);
  // product in [2^224, 2^226): keep 116 bits (113 + guard, round, sticky)
  int e = exp_of(a) + exp_of(b);
  const int top = (hi >> 97) ? 225 : 224;  // index of the leading bit
  if (top == 225) e += 1;
  const int shift = top - 115;  // 109 or 110
  const u128 keep = (hi << (128 - shift)) | (lo >> shift);
  const u128 lost = lo << (128 - shift);
  return round_pack(sign, e, keep | (lost != 0 ? 1 : 0));
}

// |a| < |b| for normal or zero values.
BGT_QP_HD bool mag_less(Q a, Q b) {
  const uint64_t ah = a.hi & ~(1ull << 63), bh = b.hi & ~(1ull << 63);
  return ah < bh || (ah == bh && a.lo < b.lo);
}

// a >= b for normal or zero values (-0 == +0).
BGT_QP_HD bool ge(Q a, Q b) {
  const bool za = is_zero(a), zb = is_zero(b);
  if (za && zb) return true;
  const uint64_t sa = za ? 0 : a.hi >> 63, sb = zb ? 0 : b.hi >> 63;
  if (sa != sb) return sb == 1;  // a positive, b negative
  if (za) return sb == 1;
  if (zb) return sa == 0;
  const bool less = mag_less(a, b);
  const bool equal = a.hi == b.hi && a.lo == b.lo;
  return sa == 0 ? !less : (less || equal);
}

// fmod(x, p): the exact remainder x - trunc(x / p) * p, with the sign of x
// (representable: no rounding).
BGT_QP_HD Q fmod(Q x, Q p) {
  if (is_special(x) || is_special(p) || is_zero(p)) return make_nan();
  if (is_zero(x) || mag_less(x, p)) return x;
  const uint64_t sign = x.hi >> 63;
  const int ex = exp_of(x), ep = exp_of(p);
  const u128 mp = sig_of(p);
  u128 r = sig_of(x);
  if (r >= mp) r -= mp;
  for (int k = 0; k < ex - ep; k++) {
    r <<= 1;
    if (r >= mp) r -= mp;
  }
  if (r == 0) return make_zero(sign);
  // r * 2^(ep - 112): the leading bit to bit 112
  const int lz = clz128(r) - (127 - 112);
  r <<= lz;
  const int e = ep - lz;
  return Q{(uint64_t)r, (sign << 63) | ((uint64_t)(e + BIAS) << 48) | ((uint64_t)(r >> 64) & FRAC_HI_MASK)};
}

// 2 a, exact for the normal values here (far from the exponent limit).
BGT_QP_HD Q twice(Q a) {
  if (is_zero(a) || is_special(a)) return a;
  return Q{a.lo, a.hi + (1ull << 48)};
}

// modulo2(x, amp) in real(qp): x folded into [-amp, amp)
// (sim_utils/special_functions/modulo2_mod.f90:121-134): Fortran's
// MODULO(x, 2 amp) -- fmod, then shifted into the sign of 2 amp -- less
// 2 amp when it reaches amp.
BGT_QP_HD Q modulo2(Q x, Q amp) {
  const Q per = twice(amp);
  Q r = fmod(x, per);
  if (!is_zero(r) && ((r.hi >> 63) != (per.hi >> 63))) r = add(r, per);
  if (ge(r, amp)) r = sub(r, per);
  return r;
}

}  // namespace qp
}  // namespace bgt
