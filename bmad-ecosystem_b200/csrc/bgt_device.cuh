// bgt_device.cuh -- FP64 element maps for one particle held in registers.
//
// Each function restates a reference routine (cited) for forward tracking
// (direction = time_dir = orientation = +1) with the tracking species equal
// to the reference species (charge_dir = rel_tracking_charge = 1).  The order
// of floating-point operations follows the reference expressions; element
// constants come pre-folded from the table (see bgt_table.h).
#pragma once
#include <stdint.h>

#include "bgt_crmath.cuh"
#include "bgt_qp.cuh"
#include "bgt_table.h"

// Every transcendental of a particle coordinate goes through bgt::cr
// (correctly rounded, see bgt_crmath.cuh); element constants arrive from the
// host table, evaluated there with the host C library.

namespace bgt {

constexpr double C_LIGHT = 2.99792458e8;                    // physical_constants.f90:34
constexpr double PI_D = 3.141592653589793238462643383279;   // physical_constants.f90:12
constexpr double TWOPI_D = 2 * PI_D;

enum State : int32_t { ALIVE = 1, LOST = 2, LOST_NEG_X = 3, LOST_POS_X = 4, LOST_NEG_Y = 5, LOST_POS_Y = 6,
                       LOST_PZ = 8 };

// Per-launch constants.
struct Glob {
  double mc2;       // mass_of(species)
  double mc2sq;     // mc2**2
  double p0c;       // reference momentum (all elements share it)
  double mal;       // bmad_com%max_aperture_limit
  int32_t ap_on;    // bmad_com%aperture_limit_on
  int32_t charge;
  int32_t abs_time;       // bmad_com%absolute_time_tracking
  int32_t abs_ref_shift;  // bmad_com%absolute_time_ref_shift
  int32_t track_time;     // the particle time t is carried (the kernel sets 0 in instances without it)
};

// A particle: phase-space coordinates, beta, state and the time t as
// binary128 bits (the reference's real(qp) coord_struct%t), advanced only
// when Glob::track_time is set.
struct Part {
  double x, px, y, py, z, pz, beta;
  int32_t state;
  uint64_t t_lo, t_hi;
};

__device__ __forceinline__ qp::Q time_of(const Part& p) { return qp::Q{p.t_lo, p.t_hi}; }
__device__ __forceinline__ void set_time(Part& p, qp::Q t) {
  p.t_lo = t.lo;
  p.t_hi = t.hi;
}
// t = t + dt, dt a real(rp) step, the sum rounded in real(qp)
__device__ __forceinline__ void add_time(Part& p, double dt) { set_time(p, qp::add(time_of(p), qp::from_double(dt))); }

// Per-particle memo of the drift's pz-only term (track_a_drift.f90:69,
// first sqrt_one).  Value-identical: recomputed whenever pz differs.
struct DriftMemo {
  double pz;
  double a;
};

// Out-of-line device functions (a plain static function in a host build);
// internal linkage, since every compilation unit of kernels has its own copy.
#ifdef __CUDACC__
#define BGT_DEV_NOINLINE static __device__ __noinline__
#else
#define BGT_DEV_NOINLINE static __attribute__((noinline))
#endif

__device__ __forceinline__ double sq(double x) { return x * x; }

// sim_utils/special_functions/sqrt_one.f90:18-40
__device__ __forceinline__ double sqrt_one(double x) {
  double s = sqrt(1.0 + x);
  double rad = s + 1.0;
  return x / rad;
}

// sim_utils/special_functions/sinc.f90:15-45
__device__ __forceinline__ double sinc_d(double x) {
  if (fabs(x) < 1e-8) return 1.0;
  return cr::sin(x) / x;
}

// x**m as gfortran evaluates it (libgcc __powidf2 order of multiplies).
__device__ __forceinline__ double powi_d(double x, int m) {
  unsigned n = (unsigned)m;
  double y = (n & 1u) ? x : 1.0;
  while (n >>= 1) {
    x = x * x;
    if (n & 1u) y = y * x;
  }
  return y;
}

// bmad/low_level/mexp.f90:14-33 (m >= 0 here)
__device__ __forceinline__ double mexp_d(double x, int m) { return m == 0 ? 1.0 : powi_d(x, m); }

// c_multi(n, m, .true.) table (bmad/low_level/c_multi.f90:19-75), host-built.
// Internal linkage: every compilation unit holding tracking kernels has its
// own copy, filled through that unit's upload function.
static __constant__ double c_cm[BGT_MAXPOLE_DEV + 1][BGT_MAXPOLE_DEV + 1];
// c_multi(n, m) without the n! factor (the cc table of multipole_kick,
// multipole_mod.f90:262-266).
static __constant__ double c_cm0[BGT_MAXPOLE_DEV + 1][BGT_MAXPOLE_DEV + 1];

// 3x3 matrix times vector, sums from zero in k order (as the oracle's and
// gfortran's matmul)
__device__ __forceinline__ void mv3_0(const double* S, double r0, double r1, double r2, double& o0, double& o1,
                                      double& o2) {
  o0 = ((0.0 + S[0] * r0) + S[1] * r1) + S[2] * r2;
  o1 = ((0.0 + S[3] * r0) + S[4] * r1) + S[5] * r2;
  o2 = ((0.0 + S[6] * r0) + S[7] * r1) + S[8] * r2;
}

// A position (r0, r1, r2) through a host-recorded chain of affine steps of a
// misaligned bend's geometry (bend_shift, misalignment and tilt frames; the
// op layout of the BM block in bgt_table.h).
__device__ __forceinline__ void bend_chain_position(const double* ops, int n, double& r0, double& r1, double& r2) {
  for (int k = 0; k < n; k++) {
    const double* o = ops + k * BM_OP_N;
    const int code = (int)o[0];
    const double* S = o + 1;
    const double* L = o + 10;
    if (code == 0) {
      r2 = r2 - L[2];
    } else if (code == 4) {
      r2 = r2 + L[2];
    } else {
      double a0 = r0, a1 = r1, a2 = r2;
      if (code == 2) {
        a0 = r0 - L[0];
        a1 = r1 - L[1];
        a2 = r2 - L[2];
      }
      mv3_0(S, a0, a1, a2, r0, r1, r2);
      if (code == 1) {
        r0 = r0 + L[0];
        r1 = r1 + L[1];
        r2 = r2 + L[2];
      }
    }
  }
}

// ---------------------------------------------------------------------------
// Apertures

// The element frame of a misaligned bend at an end for the aperture check:
// offset_particle(set, s_pos = 0 or L, no drift, no tilt),
// offset_particle.f90:208-228 and 246-258 (only x and y are needed).  The
// chain up to the arc shift is element-constant (BMA block); the shift by
// ds = rho atan2(r3 g, 1 + r1 g) turns by a particle-dependent angle, so its
// rotation (bend_shift.f90:19-61 without ref_tilt) runs here.  Out of line,
// like the exact bend edge, so that it adds no register pressure to the
// element loop.
struct XY {
  double x, y;
};
BGT_DEV_NOINLINE XY bend_aperture_frame(Part p, const double* bma, bool at_exit) {
  double r0 = p.x, r1 = p.y, r2 = 0.0;
  bend_chain_position(bma + (at_exit ? BMA_OPS_OUT : BMA_OPS_IN), (int)bma[at_exit ? BMA_NOUT : BMA_NIN], r0, r1,
                      r2);
  const double g = bma[BMA_G];
  const double ds = (g == 0) ? -1 * bma[at_exit ? BMA_DSC_OUT : BMA_DSC_IN]
                             : (1 / g) * cr::atan2(r2 * g, 1.0 + r0 * g);
  const double angle = ds * g;
  if (angle != 0) {
    const double ca = cr::cos(angle), sa = cr::sin(angle);
    // rotate_mat(unit, y, angle): each column of the unit matrix as rotate_vec
    const double S[9] = {sa * 0.0 + ca * 1.0, sa * 0.0 + ca * 0.0, sa * 1.0 + ca * 0.0,
                         0.0, 1.0, 0.0,
                         ca * 0.0 - sa * 1.0, ca * 0.0 - sa * 0.0, ca * 1.0 - sa * 0.0};
    const double sh = cr::sin(angle / 2);
    double o0, o1, o2;
    mv3_0(S, r0, r1, r2, o0, o1, o2);
    r0 = o0 + -(2 * (sh * sh)) / g;
    r1 = o1 + 0.0 / g;
  }
  const double rel_p = 1 + p.pz;
  const double pz = rel_p * rel_p - p.px * p.px - p.py * p.py;
  if (pz > 0) return {r0, r1};  // with pz <= 0 offset_particle only marks the particle
  return {p.x, p.y};
}

// bmad/low_level/orbit_too_large.f90:26-120
__device__ __forceinline__ bool orbit_too_large(Part& p, const Glob& G) {
  if (p.x > G.mal) {
    p.state = LOST_POS_X;
    return true;
  } else if (-p.x > G.mal) {
    p.state = LOST_NEG_X;
    return true;
  }
  if (p.y > G.mal) {
    p.state = LOST_POS_Y;
    return true;
  } else if (-p.y > G.mal) {
    p.state = LOST_NEG_Y;
    return true;
  }
  double rel_p = 1 + p.pz;
  if (rel_p < 0) {
    p.state = LOST_PZ;
    return true;
  }
  double f_unstable = p.px * p.px + p.py * p.py - rel_p * rel_p;
  if (f_unstable > 0) {
    if (fabs(p.px) > fabs(p.py)) {
      p.state = p.px > 0 ? LOST_POS_X : LOST_NEG_X;
    } else {
      p.state = p.py > 0 ? LOST_POS_Y : LOST_NEG_Y;
    }
    return true;
  }
  return false;
}

// bmad/low_level/check_aperture_limit.f90:240-309 (lab-frame elliptical and
// rectangular limits; the leading orbit_too_large is done by the caller).
// (x, y) checked against the limits: x, y themselves, or with
// offset_moves_aperture the particle's position in the element frame at this
// end -- offset_particle(set, s_pos = 0 or L, no drift, tilt for collimators)
// as check_aperture_limit.f90:159-175 calls it (only x and y are needed).
__device__ __forceinline__ void aperture_frame(const Part& p, const double* mis, int32_t flags, bool at_exit,
                                               double& xa, double& ya) {
  xa = p.x;
  ya = p.y;
  if (!(flags & F_AP_OFFSET)) return;
  if (flags & F_BEND_MIS) {
    const XY f = bend_aperture_frame(p, mis + MIS_N + BM_N, at_exit);
    xa = f.x;
    ya = f.y;
    return;
  }
  if (flags & F_OFFSET) {
    if (flags & F_PITCH) {
      const double rel_p = 1 + p.pz;
      const double r0 = p.x - mis[MIS_XOFF], r1 = p.y - mis[MIS_YOFF];
      const double r2 = at_exit ? mis[MIS_R3EXIT] : mis[MIS_R3SET];
      const double* w = mis + MIS_WINV;
      const double o0 = w[0] * r0 + w[1] * r1 + w[2] * r2;
      const double o1 = w[3] * r0 + w[4] * r1 + w[5] * r2;
      const double pz = rel_p * rel_p - p.px * p.px - p.py * p.py;
      if (pz > 0) {  // with pz <= 0 offset_particle only marks the particle
        xa = o0;
        ya = o1;
      }
    } else {
      const double rel_p = 1 + p.pz;
      const double pz = rel_p * rel_p - p.px * p.px - p.py * p.py;
      if (pz > 0) {
        xa = p.x - mis[MIS_XOFF];
        ya = p.y - mis[MIS_YOFF];
      }
    }
  }
  if ((flags & F_AP_TILT) && (flags & F_TILT)) {
    const double c = mis[MIS_COS], s = mis[MIS_SIN], x = xa, y = ya;
    xa = c * x + s * y;
    ya = -s * x + c * y;
  }
}

// UF: the unstable factor starts from uf0 (a collimator's momentum limits
// went first) instead of 0.
template <bool UF = false>
__device__ __forceinline__ void aperture_limits(Part& p, const double* ap, int32_t flags, double px_, double py_,
                                                double uf0 = 0.0) {
  if (flags & F_AP_ELLIPTICAL) {
    double xp = px_ - ap[AP_XC];
    double yp = py_ - ap[AP_YC];
    double r = sq(xp / ap[AP_XW]) + sq(yp / ap[AP_YW]);
    if (r < 1) return;
    if (fabs(xp / ap[AP_XW]) > fabs(yp / ap[AP_YW])) {
      p.state = xp > 0 ? LOST_POS_X : LOST_NEG_X;
    } else {
      p.state = yp > 0 ? LOST_POS_Y : LOST_NEG_Y;
    }
  } else {
    double uf = UF ? uf0 : 0, f;
    const double x1 = ap[AP_X1], x2 = ap[AP_X2], y1 = ap[AP_Y1], y2 = ap[AP_Y2];
    const double xv = px_, yv = py_;
    if (x1 != 0 && xv < x1) {
      f = fabs((xv - x1) / (x2 - x1));
      if (f > uf) {
        p.state = LOST_NEG_X;
        uf = f;
      }
    }
    if (x2 != 0 && xv > x2) {
      f = fabs((xv - x2) / (x2 - x1));
      if (f > uf) {
        p.state = LOST_POS_X;
        uf = f;
      }
    }
    if (y1 != 0 && yv < y1) {
      f = fabs((yv - y1) / (y2 - y1));
      if (f > uf) {
        p.state = LOST_NEG_Y;
        uf = f;
      }
    }
    if (y2 != 0 && yv > y2) {
      f = fabs((yv - y2) / (y2 - y1));
      if (f > uf) {
        p.state = LOST_POS_Y;
        uf = f;
      }
    }
  }
}

// check_this_limit, check_aperture_limit.f90:329-341
__device__ __forceinline__ void check_this_limit(Part& p, double coord, double width2, double center, double& uf) {
  if (width2 == 0) return;
  if (coord > center - width2 && coord < center + width2) return;
  p.state = LOST;
  uf = fmax((center - width2) - coord, coord - (center + width2));
}

// A collimator's momentum and longitudinal limits, check_aperture_limit.f90:
// 98-135, on the lab-frame coordinates: the ecollimator's (px, py) and
// (z, pz) pairs are ellipses when both widths are set, the rcollimator's four
// limits independent.
__device__ __forceinline__ void collimator_momentum_limits(Part& p, const double* m, int32_t flags, double& uf) {
  if (flags & F_AP_MOM_ELL) {
    for (int k = 0; k < 2; k++) {
      const double xw2 = m[4 * k + 0], x0 = m[4 * k + 1], yw2 = m[4 * k + 2], y0 = m[4 * k + 3];
      const double u = k == 0 ? p.px : p.z, v = k == 0 ? p.py : p.pz;
      if (xw2 == 0 || yw2 == 0) {
        check_this_limit(p, u, xw2, x0, uf);
        check_this_limit(p, v, yw2, y0, uf);
      } else {
        const double r = sq((u - x0) / xw2) + sq((v - y0) / yw2);
        if (r > 1) {
          p.state = LOST;
          uf = sqrt(r) - 1;
        }
      }
    }
  } else {
    check_this_limit(p, p.px, m[APM_PXW], m[APM_PXC], uf);
    check_this_limit(p, p.py, m[APM_PYW], m[APM_PYC], uf);
    check_this_limit(p, p.z, m[APM_ZW], m[APM_ZC], uf);
    check_this_limit(p, p.pz, m[APM_PZW], m[APM_PZC], uf);
  }
}

__device__ __forceinline__ void check_aperture(Part& p, const double* ap, const double* mis, int32_t flags,
                                               bool at_exit) {
  double xa, ya;
  double uf = 0;
  if (flags & F_AP_MOMENTUM) collimator_momentum_limits(p, ap + AP_N, flags, uf);
  aperture_frame(p, mis, flags, at_exit, xa, ya);
  aperture_limits<true>(p, ap, flags, xa, ya, uf);
}

// ---------------------------------------------------------------------------
// Drift: bmad/low_level/track_a_drift.f90:25-116

__device__ __forceinline__ double drift_pz_term(const Part& p, const Glob& G, DriftMemo& m) {
  if (p.pz != m.pz) {
    double delta = p.pz;
    double rel_pc = 1 + delta;
    m.a = sqrt_one((G.mc2sq * (2 * delta + delta * delta)) / (sq(G.p0c * rel_pc) + G.mc2sq));
    m.pz = p.pz;
  }
  return m.a;
}

// a / b correctly rounded from r = RN(1 / b): q = RN(a r), e = RN(a - b q)
// (one FMA), result RN(q + e r) -- IEEE division bit for bit for a = 0 or
// |a| >= 2^-960 and b in the normal range (coordinates, lengths and momenta
// here).  Why, scaled to b in [1, 2), Q = a / b in [1, 2), u = 2^-53:
// * |a r - Q| <= a u / 2 < 2u, so |Q - q| < 4u, and q + e r differs from Q
//   by |Q - q| |e_r + e_e + e_r e_e| < 8u^2 (e_r = b r - 1, |e_r| < u; e_e
//   the rounding of the remainder, |e_e| <= u), so the result can only miss
//   RN(Q) when a rounding midpoint M lies within 8u^2 of Q.
// * a - b M is a nonzero multiple of 2u^2 (a and b are multiples of 2u, M an
//   odd multiple of u), so |Q - M| > u^2.
// * For |Q - M| < 8u^2, |a r - M| < 2u makes q a neighbour of M whenever
//   a <= 4 - 16u; above that, a / b for a double b in [1, 2) is within
//   O(u^2) of no midpoint.  With q a neighbour of M (a faithful quotient)
//   the remainder is exact and the error is at most
//   (u + |Q - M|) b u / 2 < |Q - M|.
// (Markstein's theorem, P. Markstein, IBM J. Res. Dev. 34(1), 1990, is the
// case of a q already faithful; here q = RN(a r) can be 1.5 ulp away.)
// e = 0 keeps q, which keeps the sign of a zero quotient.  Checked on 6e8
// random and constructed operand pairs (divisors next to a power of two,
// quotients next to a midpoint) without a mismatch.  Three instructions in
// place of a division for every quotient by the same divisor.
__device__ __forceinline__ double div_by(double a, double b, double r) {
  const double q = a * r;
  const double e = fma(-q, b, a);
  return e == 0 ? q : fma(e, r, q);
}

template <bool REF_MOTION>
__device__ __forceinline__ void track_a_drift(Part& p, double length, const Glob& G, DriftMemo& m) {
  if (length == 0) return;
  double rel_pc = 1 + p.pz;
  const double r_pc = 1.0 / rel_pc;
  double px_rel = div_by(p.px, rel_pc, r_pc);
  double py_rel = div_by(p.py, rel_pc, r_pc);
  double pxy2 = px_rel * px_rel + py_rel * py_rel;
  if (pxy2 >= 1) {
    p.state = LOST_PZ;
    return;
  }
  double ps_rel = sqrt(1 - pxy2);
  const double r_ps = 1.0 / ps_rel;
  p.x = p.x + div_by(length * px_rel, ps_rel, r_ps);
  p.y = p.y + div_by(length * py_rel, ps_rel, r_ps);
  double dz;
  if (p.beta > 0) {
    if (REF_MOTION) {
      double a = drift_pz_term(p, G, m);
      // sqrt_one(-pxy2) = -pxy2 / (sqrt(1 + (-pxy2)) + 1), and
      // sqrt(1 + (-pxy2)) is ps_rel bit for bit (1 + (-a) == 1 - a)
      dz = length * (a + div_by(-pxy2 / (ps_rel + 1.0), ps_rel, r_ps));
    } else {
      dz = -div_by(length, ps_rel, r_ps);
    }
  } else {
    if (REF_MOTION) {
      dz = length * (1 - r_ps);
    } else {
      dz = -div_by(length, ps_rel, r_ps);
    }
  }
  // dt = rel_z_vel * length / (beta * ps_rel * c_light); t = t + dt
  // (track_a_drift.f90:79-80)
  if (G.track_time && p.beta > 0) add_time(p, length / (p.beta * ps_rel * C_LIGHT));
  p.z = p.z + dz;
}

// t = start t + delta_ref_time + (start z - z) / (beta * c_light), summed
// left to right in real(qp) (track_a_quadrupole.f90:144,
// track_a_bend.f90:327, track_a_thick_multipole.f90:133).
__device__ __forceinline__ void element_exit_time(Part& p, qp::Q t0, double z0, double dt_ref, const Glob& G) {
  if (!G.track_time) return;
  const double dz_t = (z0 - p.z) / (p.beta * C_LIGHT);
  set_time(p, qp::add(qp::add(t0, qp::from_double(1 * dt_ref)), qp::from_double(dz_t)));
}

// bmad/code/tilt_coords.f90:18-53 with host-evaluated cos/sin of the angle
__device__ __forceinline__ void tilt_coords(Part& p, double c, double s) {
  double x = p.x, y = p.y, px = p.px, py = p.py;
  p.x = c * x + s * y;
  p.y = -s * x + c * y;
  p.px = c * px + s * py;
  p.py = -s * px + c * py;
}

// offset_particle set/unset for non-bend elements, bmad/code/offset_particle.f90
// :183-334 (set) and :339-492 (unset), forward tracking.  Block layout in
// bgt_table.h (MIS_*).
__device__ __forceinline__ void matvec3(const double* w, double r0, double r1, double r2, double& o0, double& o1,
                                        double& o2) {
  o0 = w[0] * r0 + w[1] * r1 + w[2] * r2;
  o1 = w[3] * r0 + w[4] * r1 + w[5] * r2;
  o2 = w[6] * r0 + w[7] * r1 + w[8] * r2;
}

__device__ __forceinline__ void offset_set(Part& p, const double* mis, int32_t flags, const Glob& G, DriftMemo& m,
                                           bool set_tilt) {
  if (flags & F_OFFSET) {
    double rel_p = 1 + p.pz;
    if (flags & F_PITCH) {
      double r0 = p.x - mis[MIS_XOFF], r1 = p.y - mis[MIS_YOFF], r2 = mis[MIS_R3SET];
      double o0, o1, o2;
      matvec3(mis + MIS_WINV, r0, r1, r2, o0, o1, o2);
      o2 = o2 + mis[MIS_LHALF];
      double s_body = o2;
      double pz = rel_p * rel_p - p.px * p.px - p.py * p.py;
      if (pz <= 0) {
        p.state = LOST_PZ;
      } else {
        double q0, q1, q2;
        matvec3(mis + MIS_WINV, p.px, p.py, 1 * sqrt(pz), q0, q1, q2);
        p.px = q0;
        p.py = q1;
        p.x = o0;
        p.y = o1;
      }
      double ds = 0.0 - s_body;
      if (fabs(ds) > 1e-14 && p.state == ALIVE) track_a_drift<false>(p, ds, G, m);
    } else {
      double pz = rel_p * rel_p - p.px * p.px - p.py * p.py;
      if (pz <= 0) {
        p.state = LOST_PZ;
      } else {
        p.x = p.x - mis[MIS_XOFF];
        p.y = p.y - mis[MIS_YOFF];
      }
      double ds = mis[MIS_DS_SET];
      if (fabs(ds) > 1e-14 && p.state == ALIVE) track_a_drift<false>(p, ds, G, m);
    }
  }
  if (flags & F_HV_KICK) {
    p.px = p.px + mis[MIS_HK];
    p.py = p.py + mis[MIS_VK];
  }
  if (set_tilt && (flags & F_TILT)) tilt_coords(p, mis[MIS_COS], mis[MIS_SIN]);
}

__device__ __forceinline__ void offset_unset(Part& p, const double* mis, int32_t flags, const Glob& G, DriftMemo& m,
                                             bool set_tilt) {
  if (set_tilt && (flags & F_TILT)) tilt_coords(p, mis[MIS_COSU], mis[MIS_SINU]);
  if (flags & F_HV_KICK) {
    p.px = p.px + mis[MIS_HK];
    p.py = p.py + mis[MIS_VK];
  }
  if (flags & F_OFFSET) {
    double rel_p = 1 + p.pz;
    if (flags & F_PITCH) {
      double o0, o1, o2;
      matvec3(mis + MIS_W, p.x, p.y, mis[MIS_R3UNSET], o0, o1, o2);
      o0 = o0 + mis[MIS_XOFF];
      o1 = o1 + mis[MIS_YOFF];
      o2 = o2 + mis[MIS_ZADD];
      double s_lab = o2;
      double pz = rel_p * rel_p - p.px * p.px - p.py * p.py;
      if (pz <= 0) {
        p.state = LOST_PZ;
      } else {
        double q0, q1, q2;
        matvec3(mis + MIS_W, p.px, p.py, 1 * sqrt(pz), q0, q1, q2);
        p.px = q0;
        p.py = q1;
        p.x = o0;
        p.y = o1;
      }
      double ds = 2 * mis[MIS_LHALF] - s_lab;
      if (fabs(ds) > 1e-14 && p.state == ALIVE) track_a_drift<false>(p, ds, G, m);
    } else {
      double pz = rel_p * rel_p - p.px * p.px - p.py * p.py;
      if (pz <= 0) {
        p.state = LOST_PZ;
      } else {
        p.x = p.x + mis[MIS_XOFF];
        p.y = p.y + mis[MIS_YOFF];
      }
      double ds = mis[MIS_DS_UNSET];
      if (fabs(ds) > 1e-14 && p.state == ALIVE) track_a_drift<false>(p, ds, G, m);
    }
  }
}

// ---------------------------------------------------------------------------
// Multipole kicks: bmad/modules/multipole_mod.f90:82-174 (ab_multipole_kicks,
// magnetic) and :314-401 (ab_multipole_kick).  The factor
// r = ele%value(p0c)/orbit%p0c and the charge/orientation factor are exactly
// 1.0 here, so a2 = scale * a, b2 = scale * b.
// x^k for k = 0..7 exactly as mexp / gfortran's integer power (binary
// exponentiation, y = y * x order) evaluates each one: x^3 = x * x^2,
// x^5 = x * x^4, x^6 = x^2 * x^4, x^7 = (x * x^2) * x^4.
__device__ __forceinline__ void powi_table7(double x, double (&p)[8]) {
  p[0] = 1.0;
  p[1] = x;
  p[2] = x * x;
  p[3] = x * p[2];
  p[4] = p[2] * p[2];
  p[5] = x * p[4];
  p[6] = p[2] * p[4];
  p[7] = p[3] * p[4];
}

__device__ __forceinline__ void ab_multipole_kicks(Part& p, const double* an, const double* bn, int ix_max,
                                                   double scale) {
  double kx_tot = 0, ky_tot = 0;
  const double x = p.x, y = p.y;
  if (ix_max <= 7) {
    // same terms in the same order, each power computed once per kick
    double xp[8], yp[8];
    powi_table7(x, xp);
    powi_table7(y, yp);
#pragma unroll
    for (int n = 0; n <= 7; n++) {
      if (n > ix_max) break;
      const double a = an[n], b = bn[n];
      double kx = 0, ky = 0;
      if (!(a == 0 && b == 0)) {
        const double a2 = scale * a, b2 = scale * b;
#pragma unroll
        for (int m = 0; m <= n; m += 2) {
          const double f = c_cm[n][m] * xp[n - m] * yp[m];
          kx = kx + b2 * f;
          ky = ky - a2 * f;
        }
#pragma unroll
        for (int m = 1; m <= n; m += 2) {
          const double f = c_cm[n][m] * xp[n - m] * yp[m];
          kx = kx + a2 * f;
          ky = ky + b2 * f;
        }
      }
      kx_tot = kx_tot + kx;
      ky_tot = ky_tot + ky;
    }
    p.px = p.px + kx_tot;
    p.py = p.py + ky_tot;
    return;
  }
  for (int n = 0; n <= ix_max; n++) {
    double a = an[n], b = bn[n];
    double kx = 0, ky = 0;
    if (!(a == 0 && b == 0)) {
      double a2 = scale * a, b2 = scale * b;
      for (int m = 0; m <= n; m += 2) {
        double f = c_cm[n][m] * mexp_d(x, n - m) * mexp_d(y, m);
        kx = kx + b2 * f;
        ky = ky - a2 * f;
      }
      for (int m = 1; m <= n; m += 2) {
        double f = c_cm[n][m] * mexp_d(x, n - m) * mexp_d(y, m);
        kx = kx + a2 * f;
        ky = ky + b2 * f;
      }
    }
    kx_tot = kx_tot + kx;
    ky_tot = ky_tot + ky;
  }
  p.px = p.px + kx_tot;
  p.py = p.py + ky_tot;
}

// ---------------------------------------------------------------------------
// Quadrupole body helpers

// bmad/low_level/quad_mat2_calc.f90:22-81 (mat2 and z_coef)
struct QMat {
  double cx, m01, m10, z0, z1, z2;
};

__device__ __forceinline__ QMat quad_mat2_calc(double k1, double length, double rel_p) {
  QMat q;
  double sqrt_k = sqrt(fabs(k1));
  double sk_l = sqrt_k * length;
  double cx, sx;
  if (fabs(sk_l) < 1e-10) {
    double k_l2 = k1 * (length * length);
    cx = 1 + k_l2 / 2;
    sx = (1 + k_l2 / 6) * length;
  } else if (k1 < 0) {
    cx = cr::cos(sk_l);
    sx = cr::sin(sk_l) / sqrt_k;
  } else {
    cx = cr::cosh(sk_l);
    sx = cr::sinh(sk_l) / sqrt_k;
  }
  q.cx = cx;
  q.m01 = sx / rel_p;
  q.m10 = k1 * sx * rel_p;
  q.z0 = k1 * (-cx * sx + length) / 4;
  q.z1 = -k1 * (sx * sx) / (2 * rel_p);
  q.z2 = -(cx * sx + length) / (4 * (rel_p * rel_p));
  return q;
}

// bmad/low_level/low_energy_z_correction.f90:22-58; lez = LEZ block
__device__ __forceinline__ double low_energy_z_correction(const Part& p, const double* lez, double ds) {
  double beta0 = lez[LEZ_BETA0];
  double pz = p.pz;
  if (lez[LEZ_MASS] * ((beta0 * pz) * (beta0 * pz)) < lez[LEZ_3E7]) {
    return ds * pz * (1 - 3 * (pz * (beta0 * beta0)) / 2 + (pz * pz) * lez[LEZ_F]) * lez[LEZ_ME2];
  }
  return ds * (p.beta - beta0) / beta0;
}

// bmad/low_level/apply_energy_kick.f90:23-74
__device__ __forceinline__ void apply_energy_kick(Part& p, double dE, const Glob& G) {
  double pc = (1 + p.pz) * G.p0c;
  double beta_old = p.beta;
  double E_old = pc / p.beta;
  double E_new = E_old + dE;
  if (E_new < G.mc2) {
    p.pz = -1;
    p.beta = 0;
    p.state = LOST_PZ;
    return;
  }
  p.pz = p.pz + (1 + p.pz) * sqrt_one((2 * E_old * dE + dE * dE) / (pc * pc));
  double pc_new = G.p0c * (1 + p.pz);
  double beta_new = pc_new / E_new;
  p.z = p.z * beta_new / beta_old;
  p.beta = beta_new;
}

// Electric multipole kicks: ab_multipole_kicks with electric = true
// (bmad/modules/multipole_mod.f90:82-174, ab_multipole_kick :314-401):
// kick factor charge / (beta p0c) per order (b enters with a minus sign),
// then the energy change from the transverse kick: pz, beta and z rescaled.
__device__ __forceinline__ void ab_multipole_kicks_elec(Part& p, const double* ae, const double* be, int ix_max,
                                                        double scale, const Glob& G) {
  const double px0 = p.px, py0 = p.py, pz0 = p.pz, z0 = p.z, beta0 = p.beta;
  const double x = p.x, y = p.y;
  double kx_tot = 0, ky_tot = 0;
  for (int n = 0; n <= ix_max; n++) {
    const double a = ae[n], b = be[n];
    double kx = 0, ky = 0;
    if (!(a == 0 && b == 0)) {
      const double f = (double)G.charge / (p.beta * G.p0c);
      double a2 = a * f, b2 = -b * f;
      a2 = scale * a2;
      b2 = scale * b2;
      for (int m = 0; m <= n; m += 2) {
        const double t = c_cm[n][m] * mexp_d(x, n - m) * mexp_d(y, m);
        kx = kx + b2 * t;
        ky = ky - a2 * t;
      }
      for (int m = 1; m <= n; m += 2) {
        const double t = c_cm[n][m] * mexp_d(x, n - m) * mexp_d(y, m);
        kx = kx + a2 * t;
        ky = ky + b2 * t;
      }
    }
    kx_tot = kx_tot + kx;
    ky_tot = ky_tot + ky;
  }
  p.px = p.px + kx_tot;
  p.py = p.py + ky_tot;
  const double alpha = (kx_tot * (2 * px0 + kx_tot) + ky_tot * (2 * py0 + ky_tot)) / sq(1 + pz0);
  if (alpha < -1) {
    p.state = LOST_PZ;
    return;
  }
  const double dpz = (1 + pz0) * sqrt_one(alpha);
  p.pz = pz0 + dpz;
  p.beta = (1 + p.pz) / sqrt(sq(1 + p.pz) + sq(G.mc2 / G.p0c));
  p.z = z0 * p.beta / beta0;
}

// electric_longitudinal_fringe, bmad/low_level/apply_element_edge_kick.f90:
// 283-329: the energy change crossing the edge of the electric multipole
// potential; at_sign +1 entering, -1 leaving (the element has length).
__device__ __forceinline__ void electric_longitudinal_fringe(Part& p, const double* ae, const double* be, int ix_max,
                                                             double at_sign, const Glob& G) {
  const double ff = at_sign * (double)G.charge;
  double xr = 1, xi = 0;
  const double cr = p.x, ci = p.y;
  double phi = 0;
  for (int i = 0; i <= ix_max; i++) {
    const double nr = xr * cr - xi * ci;
    const double ni = xr * ci + xi * cr;
    xr = nr;
    xi = ni;
    if (ae[i] == 0 && be[i] == 0) continue;
    const double abr = be[i], abi = -ae[i];
    phi = phi - (abr * xr - abi * xi) / (i + 1);
  }
  apply_energy_kick(p, -ff * phi, G);
}

// hard_multipole_edge_kick, bmad/modules/fringe_mod.f90:691-864 (tracking
// part): hard-edge fringe of the quadrupole (N = 1, bp = k1) or sextupole
// (N = 2, bp = k2) body field, charge_dir = 1.  Complex products as gfortran
// forms them: (a + ib)(c + id) = (ac - bd) + i(ad + bc).
struct Cx {
  double re, im;
};
__device__ __forceinline__ Cx cx_mul(Cx a, Cx b) { return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; }
__device__ __forceinline__ Cx cx_add(Cx a, Cx b) { return {a.re + b.re, a.im + b.im}; }

template <int N>
__device__ __forceinline__ void hard_multipole_edge_kick(Part& p, double bp, bool first_edge) {
  const double x = p.x, y = p.y;
  const Cx xy = {x, y};
  Cx poly_n1 = {1.0, 0.0}, poly = xy;
  const double rel_p = 1 + p.pz;
  double fx = 0, dfx_dx = 0, dfx_dy = 0, fy = 0, dfy_dx = 0, dfy_dy = 0;
#pragma unroll
  for (int n = 1; n <= N; n++) {
    poly_n1 = poly;
    poly = cx_mul(poly, xy);
    if (n != N) continue;  // a sextupole's field is order 2 only
    const Cx dpoly_dx = {(n + 1) * poly_n1.re, (n + 1) * poly_n1.im};
    const Cx dpoly_dy = {-dpoly_dx.im, dpoly_dx.re};
    const double den = (4 * (n + 2)) * rel_p;
    Cx cab = {1.0 * bp / den, 1.0 * 0.0 / den};
    if (first_edge) cab = {-cab.re, -cab.im};
    const double cn = (double)(n + 3) / (n + 1);
    Cx xny = {x, -cn * y};
    const Cx dxny_dy = {0.0, -cn};
    fx = fx + cx_mul(cx_mul(cab, poly), xny).re;
    dfx_dx = dfx_dx + cx_mul(cab, cx_add(cx_mul(dpoly_dx, xny), poly)).re;
    dfx_dy = dfx_dy + cx_mul(cab, cx_add(cx_mul(dpoly_dy, xny), cx_mul(poly, dxny_dy))).re;
    xny = {y, cn * x};
    const Cx dxny_dx = {0.0, cn};
    fy = fy + cx_mul(cx_mul(cab, poly), xny).re;
    dfy_dx = dfy_dx + cx_mul(cab, cx_add(cx_mul(dpoly_dx, xny), cx_mul(poly, dxny_dx))).re;
    dfy_dy = dfy_dy + cx_mul(cab, cx_add(cx_mul(dpoly_dy, xny), poly)).re;
  }
  const double px = p.px, py = p.py;
  const double denom = (1 - dfx_dx) * (1 - dfy_dy) - dfx_dy * dfy_dx;
  p.x = p.x - fx;
  p.px = px + ((1.0 - dfy_dy - denom) * px + dfy_dx * py) / denom;
  p.y = p.y - fy;
  p.py = py + (dfx_dy * px + (1.0 - dfx_dx - denom) * py) / denom;
  p.z = p.z + (p.px * fx + p.py * fy) / rel_p;
}

// soft_quadrupole_edge_kick, bmad/modules/fringe_mod.f90:555-660 (tracking
// part, charge_dir = 1): s = (k1, fq1, fq2); the exponential of the
// particle-dependent f1 is correctly rounded, as the C library gives it.
__device__ __forceinline__ void soft_quad_edge_kick(Part& p, const double* s, bool first_edge) {
  const double rel_p = 1 + p.pz;
  const double k1_rel = 1.0 * s[0] / rel_p;
  double f1 = k1_rel * s[1];
  const double f2 = k1_rel * s[2];
  if (f1 == 0 && f2 == 0) return;
  if (!first_edge) f1 = -f1;
  const double ef1 = cr::exp(f1);
  const double x = p.x, px = p.px, y = p.y, py = p.py;
  const double vx = px / rel_p, vy = py / rel_p;
  p.z = p.z - (f1 * x + f2 * (1 + f1 / 2) * vx / ef1) * vx + (f1 * y + f2 * (1 - f1 / 2) * vy * ef1) * vy;
  p.x = x * ef1 + vx * f2;
  p.px = px / ef1;
  p.y = y / ef1 - vy * f2;
  p.py = py * ef1;
}

// sad_soft_bend_edge_kick, bmad/modules/fringe_mod.f90:892-996 (tracking
// part, sbend): s = (12 fint hgap, 12 fintx hgapx, g + dg)
__device__ __forceinline__ void sad_soft_bend_edge(Part& p, const double* s, bool first_edge) {
  const double fb = first_edge ? s[0] : s[1];
  if (fb == 0) return;
  double g = s[2];
  if (g == 0) return;
  g = g * 1;
  if (!first_edge) g = -g;
  const double px = p.px, y = p.y, rel_p = 1 + p.pz;
  const double c1 = fb * fb * g / (24 * rel_p);
  const double c2 = fb * (g * g) / (6 * rel_p);
  const double c3 = 2 * (g * g) / (3 * fb * rel_p);
  const double y2 = y * y, y3 = y * y2, y4 = y2 * y2;
  p.x = p.x + c1 * p.pz;
  p.py = p.py + c2 * y - c3 * y3;
  p.z = p.z + (c1 * px + c2 * y2 / 2 - c3 * y4 / 4) / rel_p;
}

// linear_bend_edge_kick, bmad/modules/fringe_mod.f90:151-212 (tracking
// part): s = (ht_x, ht_y at the entrance, ht_x, ht_y at the exit)
__device__ __forceinline__ void linear_bend_edge(Part& p, const double* s, bool first_edge) {
  const double ht_x = first_edge ? s[0] : s[2], ht_y = first_edge ? s[1] : s[3];
  const double x = p.x, y = p.y;
  p.px = p.px + ht_x * x;
  p.py = p.py + ht_y * y;
}

// ---------------------------------------------------------------------------
// The exact (PTC) bend edge of fringe_type full, exact_bend_edge_kick,
// bmad/modules/fringe_mod.f90:1465-1686 (tracking part, time_dir = 1).  The
// particle goes to PTC's (x, px, y, py, pt, ct), through a rotation of the
// frame by the edge angle, the dipole fringe map and the wedge of the bend
// field, and back.  xe is the exact-edge block (XE_*), E one end's part of
// it.  The steps return false where the reference sets err_flag.

// ptc_rot_xz, fringe_mod.f90:1384-1441 (a, tan a, cos a, sin a)
__device__ __forceinline__ bool ptc_rot_xz(double* X, double tan_a, double cos_a, double sin_a, const double* xe) {
  const double beta0 = xe[XE_BETA0];
  double arg = 1.0 + 2.0 * X[4] / beta0 + X[4] * X[4] - X[1] * X[1] - X[3] * X[3];
  if (arg < 0) return false;
  double pz = sqrt(arg);
  double pt = 1.0 - X[1] * tan_a / pz;
  double x1 = X[0];
  X[0] = x1 / cos_a / pt;
  X[1] = X[1] * cos_a + sin_a * pz;
  X[2] = X[2] + X[3] * x1 * tan_a / pz / pt;
  X[5] = X[5] + x1 * tan_a / pz / pt * (xe[XE_IB] + X[4]);
  return true;
}

// ptc_wedger, fringe_mod.f90:1020-1123, for the end's angle -a and b1 =
// g_tot != 0 (g_tot = 0 is a rotation by -a)
__device__ __forceinline__ bool ptc_wedge(double* X, const double* E, const double* xe) {
  const double beta0 = xe[XE_BETA0], b1 = xe[XE_GTOT];
  const double a = E[XE_NA], cos_a = E[XE_COSNA], sin_a = E[XE_SINNA];
  double fac = 1.0 + 2.0 * X[4] / beta0 + X[4] * X[4] - X[1] * X[1] - X[3] * X[3];
  if (fac < 0) return false;
  double radix = 1.0 + 2.0 * X[4] / beta0 + X[4] * X[4] - X[3] * X[3];
  if (radix < 1e-10) return false;
  double pz = sqrt(fac), pt = sqrt(radix);
  double Xn2 = X[1] * cos_a + (pz - b1 * X[0]) * sin_a;
  radix = 1.0 + 2.0 * X[4] / beta0 + X[4] * X[4] - Xn2 * Xn2 - X[3] * X[3];
  if (radix < 1e-10) return false;
  double pzs = sqrt(radix);
  double Xn1 = X[0] * cos_a + (X[0] * X[1] * E[XE_SIN2NA] + (sin_a * sin_a) * (2.0 * X[0] * pz - b1 * (X[0] * X[0]))) /
                                  (pzs + pz * cos_a - X[1] * sin_a);
  double Xn3 = (a + cr::asin(X[1] / pt) - cr::asin(Xn2 / pt)) / b1;
  double Xn6 = X[5] + Xn3 * (xe[XE_IB] + X[4]);
  Xn3 = X[2] + X[3] * Xn3;
  X[0] = Xn1;
  X[1] = Xn2;
  X[2] = Xn3;
  X[5] = Xn6;
  return true;
}

__device__ __forceinline__ bool ptc_wedge_or_rot(double* X, const double* E, const double* xe) {
  if (xe[XE_GTOT] == 0) return ptc_rot_xz(X, E[XE_TANNA], E[XE_COSNA], E[XE_SINNA], xe);
  return ptc_wedge(X, E, xe);
}

// ptc_fringe_dipoler, fringe_mod.f90:1151-1360 (b = E[XE_B]).  gfortran's
// inline SUM starts from zero, kept for the sign of zero.
__device__ __forceinline__ bool ptc_fringe_dipoler(double* X, const double* E, const double* xe) {
  const double beta0 = xe[XE_BETA0], b = E[XE_B], fint = E[XE_FINT], hgap = E[XE_HGAP];
  double fac = 1.0 + 2.0 * X[4] / beta0 + X[4] * X[4] - X[1] * X[1] - X[3] * X[3];
  if (fac == 0) return false;
  double pz = sqrt(fac);
  double time_fac = xe[XE_IB] + X[4];
  double xp = X[1] / pz, yp = X[3] / pz;
  double d11 = (1.0 + xp * xp) / pz, d21 = xp * yp / pz, d31 = -xp;
  double d12 = xp * yp / pz, d22 = (1.0 + yp * yp) / pz, d32 = -yp;
  double d13 = -(time_fac * xp / (pz * pz)), d23 = -(time_fac * yp / (pz * pz)), d33 = time_fac / pz;
  double u = 1.0 + yp * yp;
  double w = 1.0 + (xp * xp) * (2.0 + yp * yp);
  double fi0 = cr::atan(xp / u) - b * fint * hgap * 2.0 * w * pz;
  double cf = cr::cos(fi0);
  double co2 = b / (cf * cf);
  double xu = xp / u;
  double co1 = co2 / (1.0 + xu * xu);
  double fi1 = co1 / u - co2 * b * fint * hgap * 2.0 * (2.0 * xp * (2.0 + yp * yp) * pz);
  double fi2 = -(co1 * 2.0 * xp * yp / (u * u)) - co2 * b * fint * hgap * 2.0 * (2.0 * (xp * xp) * yp) * pz;
  double fi3 = -(co2 * b * fint * hgap * 2.0 * w);
  double fi0t = b * cr::tan(fi0);
  double bb = 0.0 + fi1 * d12 + fi2 * d22 + fi3 * d32;
  fac = 1.0 - 2.0 * bb * X[2];
  if (fac < 0) return false;
  X[2] = 2.0 * X[2] / (1.0 + sqrt(fac));
  X[3] = X[3] - fi0t * X[2];
  bb = 0.0 + fi1 * d11 + fi2 * d21 + fi3 * d31;
  X[0] = X[0] + 0.5 * bb * (X[2] * X[2]);
  bb = 0.0 + fi1 * d13 + fi2 * d23 + fi3 * d33;
  X[5] = X[5] - 0.5 * bb * (X[2] * X[2]);
  return true;
}

// exact_bend_edge_kick, fringe_mod.f90:1465-1577, with vec_bmad_to_ptc and
// vec_ptc_to_bmad (:1599-1684): a failed step leaves the coordinates as they
// were and the particle lost_pz.  Out of line (the particle passed and
// returned by value), so that its temporaries do not raise the register
// pressure of the element loop around it.
template <bool ENTERING>
BGT_DEV_NOINLINE Part exact_bend_edge(Part p, const double* xe) {
  const double beta0 = xe[XE_BETA0], ib = xe[XE_IB];
  const double* E = xe + (ENTERING ? XE_IN : XE_OUT);
  const double v5 = p.z, v6 = p.pz;
  double X[6];
  X[0] = p.x;
  X[1] = p.px;
  X[2] = p.y;
  X[3] = p.py;
  X[4] = (v6 * v6 + 2 * v6) / (ib + sqrt(xe[XE_IB2] + v6 * v6 + 2 * v6));
  X[5] = -(v5 * (ib + X[4]) / (1 + v6));
  bool ok;
  if (ENTERING) {
    ok = ptc_rot_xz(X, E[XE_TANA], E[XE_COSA], E[XE_SINA], xe) && ptc_fringe_dipoler(X, E, xe) &&
         ptc_wedge_or_rot(X, E, xe);
  } else {
    ok = ptc_wedge_or_rot(X, E, xe) && ptc_fringe_dipoler(X, E, xe) &&
         ptc_rot_xz(X, E[XE_TANA], E[XE_COSA], E[XE_SINA], xe);
  }
  if (!ok) {
    p.state = LOST_PZ;
    return p;
  }
  double f1 = 1 + 2 * X[4] / beta0 + X[4] * X[4];
  if (f1 <= 0) return p;
  double t6 = (2 * X[4] / beta0 + X[4] * X[4]) / (sqrt(f1) + 1);
  double t5 = -(X[5] * (1 + t6) / (ib + X[4]));
  p.x = X[0];
  p.px = X[1];
  p.y = X[2];
  p.py = X[3];
  p.z = t5;
  p.pz = t6;
  return p;
}

// ---------------------------------------------------------------------------
// Hwang hard-edge bend fringe, bmad/modules/fringe_mod.f90:240-418 (td = +1)
template <bool ENTERING>
__device__ __forceinline__ void hwang_edge(Part& p, const double* E) {
  const double gt = E[EDGE_GT], gt2 = E[EDGE_GT2], gs2 = E[EDGE_GS2], k1_tane = E[EDGE_K1TANE];
  const double fg = E[EDGE_FG];
  double e_factor = 1 / (1 + p.pz);
  double v0 = p.x, v1 = p.px, v2 = p.y, v3 = p.py, v4 = p.z;
  double dx, dpx, dy, dpy, dz;
  if (ENTERING) {
    dx = (-gt2 * (v0 * v0) + gs2 * (v2 * v2)) * e_factor / 2;
    dpx = (E[EDGE_C1] * (v2 * v2) / 2 + gt2 * (v0 * v1 - v2 * v3) + k1_tane * (v0 * v0 - v2 * v2)) * e_factor;
    dy = gt2 * v0 * v2 * e_factor;
    dpy = (fg * v2 - gt2 * v0 * v3 - E[EDGE_GPG] * v1 * v2 - E[EDGE_K1TANE2] * v0 * v2) * e_factor;
    dz = (e_factor * e_factor) * 0.5 *
         ((v2 * v2) * fg + (v0 * v0 * v0) * E[EDGE_C3] / 6.0 + 0.5 * v0 * (v2 * v2) * E[EDGE_C4] +
          ((v0 * v0) * v1 - 2.0 * v0 * v2 * v3) * gt2 - v1 * (v2 * v2) * gs2);
  } else {
    dx = (gt2 * (v0 * v0) - gs2 * (v2 * v2)) * e_factor / 2;
    dpx = (gt2 * (v2 * v3 - v0 * v1) + k1_tane * (v0 * v0 - v2 * v2) - E[EDGE_C1] * (v0 * v0 + v2 * v2) / 2) *
          e_factor;
    dy = -gt2 * v0 * v2 * e_factor;
    dpy = (fg * v2 + gt2 * v0 * v3 + E[EDGE_GPG] * v1 * v2 + E[EDGE_GTGS2_2K1] * v0 * v2) * e_factor;
    dz = (e_factor * e_factor) * 0.5 *
         ((v2 * v2) * fg + (v0 * v0 * v0) * E[EDGE_C3] / 6.0 + 0.5 * v0 * (v2 * v2) * E[EDGE_C4] -
          ((v0 * v0) * v1 - 2.0 * v0 * v2 * v3) * gt2 + v1 * (v2 * v2) * gs2);
  }
  p.x = v0 + 1.0 * dx;
  p.px = v1 + 1.0 * (dpx + gt * v0);
  p.y = v2 + 1.0 * dy;
  p.py = v3 + 1.0 * (dpy - gt * v2);
  p.z = v4 + 1.0 * dz;
}

}  // namespace bgt
