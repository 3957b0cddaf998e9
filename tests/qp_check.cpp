// Host check of bgt_qp.cuh (software binary128) against GCC's __float128
// (libquadmath): add, sub, mul, fmod, modulo2 and the conversions from and to
// double, bit for bit, on random operands shaped like the tracker's (a
// particle time of up to seconds plus per-element steps, products with an RF
// frequency, folds into an RF half-period) and on edge cases (exact
// cancellation, carries, ties, zeros, signs, subnormal doubles).
//   qp_check N SEED   -> prints "mismatches M of K" and exits 1 on any mismatch
#include <math.h>
#include <quadmath.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "../bmad-ecosystem_b200/csrc/bgt_qp.cuh"

using bgt::qp::Q;

static Q q_of(__float128 x) {
  Q q;
  memcpy(&q, &x, 16);
  return q;
}
static __float128 f_of(Q q) {
  __float128 x;
  memcpy(&x, &q, 16);
  return x;
}
static bool same(Q a, __float128 b) {
  const Q qb = q_of(b);
  if (isnanq(b)) return bgt::qp::is_special(a);
  return a.lo == qb.lo && a.hi == qb.hi;
}

static uint64_t rng_state;
static uint64_t rnd() {
  rng_state ^= rng_state << 13;
  rng_state ^= rng_state >> 7;
  rng_state ^= rng_state << 17;
  return rng_state;
}
static double urand() { return (rnd() >> 11) * 0x1.0p-53; }
// a random binary128: random 112-bit fraction, exponent in [elo, ehi], sign
static __float128 rq(int elo, int ehi) {
  Q q;
  q.lo = rnd();
  const int e = elo + (int)(rnd() % (uint64_t)(ehi - elo + 1));
  q.hi = ((rnd() & 1ull) << 63) | ((uint64_t)(e + 16383) << 48) | (rnd() & ((1ull << 48) - 1));
  return f_of(q);
}
static double rd(int elo, int ehi) {
  const int e = elo + (int)(rnd() % (uint64_t)(ehi - elo + 1));
  return ldexp(1.0 + urand(), e) * ((rnd() & 1) ? -1 : 1);
}

int main(int argc, char** argv) {
  const long n = argc > 1 ? atol(argv[1]) : 1000000;
  rng_state = argc > 2 ? strtoull(argv[2], 0, 10) : 88172645463325252ull;
  if (rng_state == 0) rng_state = 1;
  long bad = 0, total = 0;
#define CHECK(got, want, what)                                 \
  do {                                                         \
    total++;                                                   \
    if (!same((got), (want))) {                                \
      if (bad < 10) fprintf(stderr, "mismatch in %s\n", what); \
      bad++;                                                   \
    }                                                          \
  } while (0)
  for (long i = 0; i < n; i++) {
    // a time of up to seconds and element-sized steps
    const __float128 t = rq(-40, 2);
    const double d = rd(-60, 0);
    const Q qt = q_of(t), qd = bgt::qp::from_double(d);
    CHECK(qd, (__float128)d, "from_double");
    CHECK(bgt::qp::add(qt, qd), t + (__float128)d, "add t+d");
    CHECK(bgt::qp::sub(qt, qd), t - (__float128)d, "sub t-d");
    // general operands, and near-cancellation
    const __float128 a = rq(-80, 20), b = rq(-80, 20);
    CHECK(bgt::qp::add(q_of(a), q_of(b)), a + b, "add a+b");
    const __float128 c = a * (1 + rq(-120, -100));
    CHECK(bgt::qp::sub(q_of(a), q_of(c)), a - c, "sub near-cancel");
    CHECK(bgt::qp::mul(q_of(a), q_of(b)), a * b, "mul a*b");
    CHECK(bgt::qp::mul(qt, bgt::qp::from_double(d)), t * (__float128)d, "mul t*d");
    // the RF phase chain: modulo2(t - t0, 0.5/f), (time - 0) * f, phi0 - that, twopi * that
    const double f = 4.9e8 + 2e7 * urand();
    const __float128 amp = ((__float128)0.5) / (__float128)f;
    const __float128 x = t - (__float128)rd(-30, -1);
    const __float128 per = 2 * amp;
    __float128 r = fmodq(x, per);
    if (r != 0 && ((r < 0) != (per < 0))) r += per;
    if (r >= amp) r = r - 2 * amp;
    const Q qr = bgt::qp::modulo2(q_of(x), q_of(amp));
    CHECK(qr, r, "modulo2");
    CHECK(bgt::qp::fmod(q_of(x), q_of(per)), fmodq(x, per), "fmod");
    const double phi0 = rd(-10, -1);
    const __float128 ph = (__float128)(2 * M_PI) * ((__float128)phi0 - (r - (__float128)0.0) * (__float128)f);
    const Q qph = bgt::qp::mul(bgt::qp::from_double(2 * M_PI),
                               bgt::qp::sub(bgt::qp::from_double(phi0),
                                            bgt::qp::mul(bgt::qp::sub(qr, bgt::qp::from_double(0.0)),
                                                         bgt::qp::from_double(f))));
    CHECK(qph, ph, "rf phase");
    total++;
    if (bgt::qp::to_double(qph) != (double)ph) {
      if (bad < 10) fprintf(stderr, "mismatch in to_double\n");
      bad++;
    }
    // to_double on arbitrary operands, every seventh an exact tie
    Q qt2 = q_of(a);
    if (i % 7 == 0) qt2.lo = (qt2.lo & ~((1ull << 60) - 1)) | (1ull << 59);
    total++;
    if (bgt::qp::to_double(qt2) != (double)f_of(qt2)) {
      if (bad < 10) fprintf(stderr, "mismatch in to_double (tie)\n");
      bad++;
    }
  }
  // edge cases
  const double eds[] = {0.0, -0.0, 1.0, -1.0, 0x1p-1074, -0x1p-1074, 0x1.fffffffffffffp-1023, 0x1p-1022,
                        0x1.fffffffffffffp+1023, 3e-300};
  for (double d : eds) {
    CHECK(bgt::qp::from_double(d), (__float128)d, "from_double edge");
    for (double e : eds) {
      if (fabs(d) > 1e300 || fabs(e) > 1e300) continue;
      CHECK(bgt::qp::add(bgt::qp::from_double(d), bgt::qp::from_double(e)), (__float128)d + (__float128)e,
            "add edge");
      CHECK(bgt::qp::mul(bgt::qp::from_double(d), bgt::qp::from_double(e)), (__float128)d * (__float128)e,
            "mul edge");
    }
  }
  const __float128 one = 1, ulp = ldexpq((__float128)1, -112);
  CHECK(bgt::qp::add(q_of(one), q_of(ulp / 2)), one + ulp / 2, "tie to even down");
  CHECK(bgt::qp::add(q_of(one + ulp), q_of(ulp / 2)), (one + ulp) + ulp / 2, "tie to even up");
  CHECK(bgt::qp::add(q_of(2 - ulp), q_of(ulp)), (2 - ulp) + ulp, "carry");
  CHECK(bgt::qp::sub(q_of(one), q_of(one)), one - one, "exact cancel");
  CHECK(bgt::qp::sub(q_of(one), q_of(one - ulp / 2)), one - (one - ulp / 2), "one-bit cancel");
  printf("mismatches %ld of %ld\n", bad, total);
  return bad ? 1 : 0;
}
