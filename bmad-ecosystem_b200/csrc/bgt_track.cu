// bgt_track.cu -- persistent FP64 tracking kernel for sm_100a and the C ABI
// declared in include/bgt.h.
//
// Launch model: one thread per particle, the particle's phase-space vector in
// registers for whole turns.  A CTA owns a tile of particles ("slots") of one
// lattice variant; it stages that variant's element table into shared memory
// with one bulk TMA copy (cp.async.bulk, no multicast) completed on an
// mbarrier, then walks turns x records reading the table by broadcast.  The
// grid is persistent (a multiple of the SM count); CTAs pull tiles from an
// atomic counter so uneven survival balances across SMs.  Every few turns a
// CTA compacts its surviving particles onto the lowest lanes (warp ballot +
// block prefix sum through shared memory) so dead lanes stop costing issue
// slots; fully dead warps skip the element loop.
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <string>
#include <unordered_map>
#include <vector>

#include "../../include/bgt.h"
#include "bgt_device.cuh"
#include "bgt_table.h"

namespace bgt {

// ===========================================================================
// Element bodies (device)

struct Rec {
  const RecHdr* h;
  const double* mis;   // misalignment block or nullptr
  const double* ap;    // aperture block or nullptr
  const double* kb;    // kind block
};

__device__ __forceinline__ Rec decode(const double* r) {
  Rec R;
  R.h = reinterpret_cast<const RecHdr*>(r);
  const double* q = r + HDR_DW;
  int32_t fl = R.h->flags;
  R.mis = nullptr;
  R.ap = nullptr;
  if (fl & F_MISALIGN) {
    R.mis = q;
    q += MIS_N;
  }
  if (fl & (F_AP_ENTRANCE | F_AP_EXIT)) {
    R.ap = q;
    q += AP_N;
  }
  R.kb = q;
  return R;
}

// Per-thread memo of quad_mat2_calc results for up to QMEMO_CLASSES quad
// strength classes (same b1, length and step), in shared memory:
// qm[(cls * 13 + j) * stride], j = 0..11 the two QMat, j = 12 the rel_p key.
// quad_mat2_calc is a pure function of (b1, length, step, rel_p) and rel_p
// changes only at energy kicks, so ring quads of one class reuse it until the
// next RF pass: value-identical, ~2 evaluations per turn instead of 128.
constexpr int QMEMO_CLASSES = 2;
struct QMemo {
  double* q;  // this thread's column
  int stride;
};

// bmad/low_level/track_a_quadrupole.f90:134-265 (magnetic and electric
// multipoles; no quadrupole fringe)
__device__ __forceinline__ void body_quad(Part& p, const Rec& R, const Glob& G, DriftMemo& m, QMemo qm) {
  const double* q = R.kb;
  const int32_t fl = R.h->flags;
  const int ix = R.h->ix_mag_max;
  const int ixe = R.h->aux1;
  const int n_step = R.h->n_step;
  const double* an = q + Q_N;
  const double* bn = an + (ix + 1);
  const double* ae = an + 2 * (ix + 1);
  const double* be = ae + (ixe + 1);
  const double* hard = ae + ((fl & F_ELEC) ? 2 * (ixe + 1) : 0);
  if (fl & F_MISALIGN) offset_set(p, R.mis, fl, G, m, true);
  if (fl & F_FRINGE_INFO) {
    // apply_element_edge_kick.f90:160-176, first edge: magnetic, then electric
    if (fl & F_EDGE_IN) {
      if (fl & F_HARD_EDGE) hard_multipole_edge_kick<1>(p, hard[0], true);
      if (fl & F_ELEC_EDGE) electric_longitudinal_fringe(p, ae, be, ixe, 1.0, G);
    }
    if (p.state != ALIVE) return;
  }
  if (ix > -1) ab_multipole_kicks(p, an, bn, ix, q[Q_RHALF]);
  if (ixe > -1) ab_multipole_kicks_elec(p, ae, be, ixe, q[Q_STEP] / 2, G);
  const double step = q[Q_STEP];
  // rel_p changes only through electric fields, absent here: quad_mat2_calc
  // has identical inputs at every step, so it is evaluated once.
  QMat mx, my;
  double rel_p_m = NAN;
  for (int i = 1; i <= n_step; i++) {
    double rel_p = 1 + p.pz;
    if (!(rel_p == rel_p_m)) {
      const int cls = R.h->aux0;
      double* c = qm.q + (cls * 13) * qm.stride;
      if (cls >= 0 && c[12 * qm.stride] == rel_p) {
        mx = {c[0], c[qm.stride], c[2 * qm.stride], c[3 * qm.stride], c[4 * qm.stride], c[5 * qm.stride]};
        my = {c[6 * qm.stride], c[7 * qm.stride], c[8 * qm.stride], c[9 * qm.stride], c[10 * qm.stride],
              c[11 * qm.stride]};
      } else {
        double k1 = q[Q_B1] / (q[Q_LEN] * rel_p);
        mx = quad_mat2_calc(-k1, step, rel_p);
        my = quad_mat2_calc(k1, step, rel_p);
        if (cls >= 0) {
          const double v[12] = {mx.cx, mx.m01, mx.m10, mx.z0, mx.z1, mx.z2,
                                my.cx, my.m01, my.m10, my.z0, my.z1, my.z2};
#pragma unroll
          for (int j = 0; j < 12; j++) c[j * qm.stride] = v[j];
          c[12 * qm.stride] = rel_p;
        }
      }
      rel_p_m = rel_p;
    }
    double x = p.x, px = p.px, y = p.y, py = p.py;
    p.z = p.z + (mx.z0 * (x * x) + mx.z1 * x * px + mx.z2 * (px * px) + my.z0 * (y * y) + my.z1 * y * py +
                 my.z2 * (py * py));
    p.x = mx.cx * x + mx.m01 * px;
    p.px = mx.m10 * x + mx.cx * px;
    p.y = my.cx * y + my.m01 * py;
    p.py = my.m10 * y + my.cx * py;
    p.z = p.z + low_energy_z_correction(p, q + Q_LEZ, step);
    if (ix > -1) ab_multipole_kicks(p, an, bn, ix, (i == n_step) ? q[Q_RHALF] : q[Q_RSTEP]);
    if (ixe > -1) ab_multipole_kicks_elec(p, ae, be, ixe, (i == n_step) ? q[Q_STEP] / 2 : q[Q_STEP], G);
  }
  if (fl & F_FRINGE_INFO) {
    // second edge: electric, then magnetic
    if (fl & F_EDGE_OUT) {
      if (fl & F_ELEC_EDGE) electric_longitudinal_fringe(p, ae, be, ixe, -1.0, G);
      if (fl & F_HARD_EDGE) hard_multipole_edge_kick<1>(p, hard[0], false);
    }
    if (p.state != ALIVE) return;
  }
  if (fl & F_MISALIGN) offset_unset(p, R.mis, fl, G, m, true);
}

// bmad/low_level/track_a_thick_multipole.f90:18-134
__device__ __forceinline__ void body_thick(Part& p, const Rec& R, const Glob& G, DriftMemo& m) {
  const double* q = R.kb;
  const int32_t fl = R.h->flags;
  const int ix = R.h->ix_mag_max;
  const int n_step = R.h->n_step;
  const int ixe = R.h->aux1;
  const double* an = q + TM_N;
  const double* bn = an + (ix + 1);
  const double* ae = an + 2 * (ix + 1);
  const double* be = ae + (ixe + 1);
  const double* hard = ae + ((fl & F_ELEC) ? 2 * (ixe + 1) : 0);
  if (fl & F_MISALIGN) offset_set(p, R.mis, fl, G, m, true);
  if (fl & F_FRINGE_INFO) {
    if (fl & F_EDGE_IN) {
      if (fl & F_HARD_EDGE) hard_multipole_edge_kick<2>(p, hard[0], true);
      if (fl & F_ELEC_EDGE) electric_longitudinal_fringe(p, ae, be, ixe, 1.0, G);
    }
    if (p.state != ALIVE) return;
  }
  if (ix > -1) ab_multipole_kicks(p, an, bn, ix, q[TM_RHALF]);
  if (ixe > -1) ab_multipole_kicks_elec(p, ae, be, ixe, q[TM_STEP] / 2, G);
  for (int i = 1; i <= n_step; i++) {
    track_a_drift<true>(p, q[TM_STEP], G, m);
    if (ix > -1) ab_multipole_kicks(p, an, bn, ix, (i == n_step) ? q[TM_RHALF] : q[TM_RSTEP]);
    if (ixe > -1) ab_multipole_kicks_elec(p, ae, be, ixe, (i == n_step) ? q[TM_STEP] / 2 : q[TM_STEP], G);
  }
  if (fl & F_FRINGE_INFO) {
    if (fl & F_EDGE_OUT) {
      if (fl & F_ELEC_EDGE) electric_longitudinal_fringe(p, ae, be, ixe, -1.0, G);
      if (fl & F_HARD_EDGE) hard_multipole_edge_kick<2>(p, hard[0], false);
    }
    if (p.state != ALIVE) return;
  }
  if (fl & F_MISALIGN) offset_unset(p, R.mis, fl, G, m, true);
}

// multipole_kick, bmad/modules/multipole_mod.f90:203-286
__device__ __forceinline__ void multipole_kick(Part& p, int n, double knl, double c, double s, bool t_zero,
                                               bool ref_orb_offset) {
  double x, y;
  if (t_zero) {
    s = 0;
    c = 1;
    x = p.x;
    y = p.y;
  } else {
    x = p.x * c + p.y * s;
    y = -p.x * s + p.y * c;
  }
  if (n == 0 && ref_orb_offset) {
    p.px = p.px + 1.0 * knl * c * p.pz;
    p.py = p.py + 1.0 * knl * s * p.pz;
    p.z = p.z - 1.0 * knl * (c * p.x + s * p.y);
    return;
  }
  double x_value = 0, y_value = 0;
  for (int mm = 0; mm <= n; mm++) {
    // x_terms(mm) = x**(n-mm), y_terms(mm) = y**mm, both by repeated products
    double xt = 1.0, yt = 1.0;
    for (int k = 0; k < n - mm; k++) xt = xt * x;
    for (int k = 0; k < mm; k++) yt = yt * y;
    double term = c_cm0[n][mm] * xt * yt;
    if (mm & 1) y_value = y_value + term;
    else x_value = x_value + term;
  }
  double x_vel = 1.0 * knl * x_value;
  double y_vel = 1.0 * knl * y_value;
  if (t_zero) {
    p.px = p.px + x_vel;
    p.py = p.py + y_vel;
  } else {
    p.px = p.px + x_vel * c - y_vel * s;
    p.py = p.py + x_vel * s + y_vel * c;
  }
}

// track1_bmad.f90:142-166 (multipole, ab_multipole)
__device__ __forceinline__ void body_thin(Part& p, const Rec& R, const Glob& G, DriftMemo& m) {
  const double* q = R.kb;
  const int32_t fl = R.h->flags;
  const int ix = R.h->ix_mag_max;
  if (fl & F_MISALIGN) offset_set(p, R.mis, fl, G, m, false);
  const bool ref_orb = q[TH_REFORB] != 0;
  for (int n = 0; n <= ix; n++) {
    const double* pp = q + TH_N + TH_POLE * n;
    if (pp[0] == 0) continue;
    multipole_kick(p, n, pp[0], pp[1], pp[2], pp[3] != 0, ref_orb);
  }
  if (fl & F_MISALIGN) offset_unset(p, R.mis, fl, G, m, false);
}

// Double-double helpers for particle_rf_time's quad-precision modulo2
// (bmad/code/particle_rf_time.f90:116-118) and the phase0 product
// (track_a_rfcavity.f90:78-80).
struct DD {
  double hi, lo;
};
__device__ __forceinline__ DD two_sum(double a, double b) {
  double s = a + b;
  double bb = s - a;
  double e = (a - (s - bb)) + (b - bb);
  return {s, e};
}
__device__ __forceinline__ DD dd_norm(double hi, double lo) {
  double s = hi + lo;
  return {s, lo - (s - hi)};
}
__device__ __forceinline__ DD dd_add(DD a, DD b) {
  DD s = two_sum(a.hi, b.hi);
  DD t = two_sum(a.lo, b.lo);
  s.lo += t.hi;
  s = dd_norm(s.hi, s.lo);
  s.lo += t.lo;
  return dd_norm(s.hi, s.lo);
}
__device__ __forceinline__ DD dd_mul_d(DD a, double b) {
  double p = a.hi * b;
  double e = fma(a.hi, b, -p);
  e = fma(a.lo, b, e);
  return dd_norm(p, e);
}
__device__ __forceinline__ DD dd_neg(DD a) { return {-a.hi, -a.lo}; }

// modulo2(time, amp) with amp a double-double (modulo2_mod.f90:121-134)
__device__ __forceinline__ DD dd_modulo2(double x, DD amp) {
  DD per = {2 * amp.hi, 2 * amp.lo};
  double q = floor(x / per.hi);
  DD r = dd_add({x, 0.0}, dd_neg(dd_mul_d(per, q)));
  // fix the quotient so that 0 <= r < per
  if (r.hi < 0) r = dd_add(r, per);
  if (r.hi > per.hi || (r.hi == per.hi && r.lo >= per.lo)) r = dd_add(r, dd_neg(per));
  if (r.hi > amp.hi || (r.hi == amp.hi && r.lo >= amp.lo)) r = dd_add(r, dd_neg(per));
  return r;
}

// bmad/low_level/track_a_rfcavity.f90:17-146, relative time, no coupler
__device__ __forceinline__ void body_rf(Part& p, const Rec& R, const Glob& G, DriftMemo& m) {
  const double* q = R.kb;
  const int32_t fl = R.h->flags;
  const int ix = R.h->ix_mag_max;
  const double* an = q + RF_N;
  const double* bn = an + (ix + 1);
  offset_set(p, R.mis, fl, G, m, true);
  if (ix > -1) ab_multipole_kicks(p, an, bn, ix, q[RF_RHALF]);
  const double voltage = q[RF_VOLT];
  const double f = q[RF_FREQ];
  // particle_rf_time, relative time: time = -z / (beta * c_light)
  double time = -p.z / (p.beta * C_LIGHT);
  DD t = {time, 0.0};
  if (f != 0) t = dd_modulo2(time, DD{q[RF_HALF_AMP_HI], q[RF_HALF_AMP_LO]});
  DD tf = dd_mul_d(t, f);
  DD u = dd_add({q[RF_PHI0], 0.0}, dd_neg(tf));
  DD v = dd_mul_d(u, TWOPI_D);
  double phase0 = v.hi + v.lo;
  phase0 = phase0 + q[RF_PHI0_MP];
  // modulo2(phase0, pi) in double
  double per = 2 * PI_D;
  double mod = fmod(phase0, per);
  if (mod != 0 && ((mod < 0) != (per < 0))) mod += per;
  if (mod >= PI_D) mod = mod - per;
  double phase = mod;
  const int n_slice = R.h->n_step;
  const double slice_l = q[RF_SLICE_L];
  for (int i = 0; i <= n_slice; i++) {
    double dE = 1 * voltage * cr::sin(phase) / n_slice;
    if (i == 0 || i == n_slice) dE = dE / 2;
    apply_energy_kick(p, dE, G);
    if (p.pz == -1) {
      p.state = LOST_PZ;
      return;
    }
    if (i != n_slice) {
      double z0 = p.z;
      track_a_drift<true>(p, slice_l, G, m);
      phase = phase + q[RF_TWOPI_F] * (p.z - z0) / (C_LIGHT * p.beta);
    }
  }
  if (ix > -1) ab_multipole_kicks(p, an, bn, ix, q[RF_RHALF]);
  offset_unset(p, R.mis, fl, G, m, true);
}

// bmad/low_level/track_a_bend.f90:338-471, apply_multipole_kicks (magnetic,
// non-exact multipoles).  ab_multipole_kick is called with ele_orientation 0
// and no scale, so a2 = an(i), b2 = bn(i).
__device__ __forceinline__ void bend_multipole_kicks(Part& p, const double* q, const double* an, const double* bn,
                                                     int ix, double coef, const Glob& G) {
  double B0 = 0, B1 = 0;
  const double f_p0c = q[B_FP0C];
  const double x = p.x, y = p.y;
  for (int n = 0; n <= ix; n++) {
    double a2 = an[n], b2 = bn[n];
    if (a2 == 0 && b2 == 0) continue;
    double kx = 0, ky = 0;
    for (int mm = 0; mm <= n; mm += 2) {
      double f = c_cm[n][mm] * mexp_d(x, n - mm) * mexp_d(y, mm);
      kx = kx + b2 * f;
      ky = ky - a2 * f;
    }
    for (int mm = 1; mm <= n; mm += 2) {
      double f = c_cm[n][mm] * mexp_d(x, n - mm) * mexp_d(y, mm);
      kx = kx + a2 * f;
      ky = ky + b2 * f;
    }
    B0 = B0 + f_p0c * ky;
    B1 = B1 - f_p0c * kx;
  }
  double f_coef = coef * q[B_CDIR] * (1 + q[B_G] * p.x) * C_LIGHT / G.p0c;
  p.px = p.px - f_coef * B1;
  p.py = p.py + f_coef * B0;
}

// sbend_body_with_k1_map, track_a_bend.f90:500-659 (no matrix)
__device__ __forceinline__ void sbend_k1_body(Part& p, const double* q) {
  const double g = q[B_G];
  const double k1 = q[B_K1 + 0];
  const double length = q[B_K1 + 1];
  const double g_tot = q[B_K1 + 2];
  double rel_p = (1 + p.pz);
  double rel_p2 = rel_p * rel_p;
  double k_x = k1 + g * g_tot;
  double x_c = (g * rel_p - g_tot) / k_x;
  double om_x = sqrt(fabs(k_x) / rel_p);
  double om_y = sqrt(fabs(k1) / rel_p);
  double tau_x = -copysign(1.0, k_x);
  double tau_y = copysign(1.0, k1);
  double s_x, c_x, z2, s_y, c_y;
  double arg = om_x * length;
  if (arg < 1e-6) {
    s_x = (1 + tau_x * (arg * arg) / 6) * length;
    c_x = 1 + tau_x * (arg * arg) / 2;
    z2 = g * (length * length) / (2 * rel_p);
  } else if (k_x > 0) {
    s_x = cr::sin(arg) / om_x;
    c_x = cr::cos(arg);
    z2 = tau_x * g * (1 - c_x) / (rel_p * (om_x * om_x));
  } else {
    s_x = cr::sinh(arg) / om_x;
    c_x = cr::cosh(arg);
    z2 = tau_x * g * (1 - c_x) / (rel_p * (om_x * om_x));
  }
  arg = om_y * length;
  if (arg < 1e-6) {
    s_y = (1 + tau_y * (arg * arg) / 6) * length;
    c_y = 1 + tau_y * (arg * arg) / 2;
  } else if (k1 < 0) {
    s_y = cr::sin(om_y * length) / om_y;
    c_y = cr::cos(om_y * length);
  } else {
    s_y = cr::sinh(om_y * length) / om_y;
    c_y = cr::cosh(om_y * length);
  }
  double r0 = p.x - x_c, r1 = p.px, r2 = p.y, r3 = p.py, r4 = p.z;
  double z0 = -g * x_c * length;
  double z1 = -g * s_x;
  double z11 = tau_x * (om_x * om_x) * (length - c_x * s_x) / 4;
  double z12 = -tau_x * (om_x * om_x) * (s_x * s_x) / (2 * rel_p);
  double z22 = -(length + c_x * s_x) / (4 * rel_p2);
  double z33 = tau_y * (om_y * om_y) * (length - c_y * s_y) / 4;
  double z34 = -tau_y * (om_y * om_y) * (s_y * s_y) / (2 * rel_p);
  double z44 = -(length + c_y * s_y) / (4 * rel_p2);
  p.x = c_x * r0 + s_x * r1 / rel_p + x_c;
  p.px = tau_x * (om_x * om_x) * rel_p * s_x * r0 + c_x * r1;
  p.y = c_y * r2 + s_y * r3 / rel_p;
  p.py = tau_y * (om_y * om_y) * rel_p * s_y * r2 + c_y * r3;
  p.z = r4 + 1 * 1 * z0 + z1 * r0 + z2 * r1 + z11 * (r0 * r0) + z12 * r0 * r1 + z22 * (r1 * r1) +
        z33 * (r2 * r2) + z34 * r2 * r3 + z44 * (r3 * r3);
}

// Returns false when the element ends the particle (lost inside and
// track_a_bend returns early).  bmad/low_level/track_a_bend.f90:18-333.
__device__ __forceinline__ void body_bend(Part& p, const Rec& R, const Glob& G, DriftMemo& m) {
  const double* q = R.kb;
  const int32_t fl = R.h->flags;
  const int ix = R.h->ix_mag_max;
  const int n_step = R.h->n_step;
  const double* an = q + B_N;
  const double* bn = an + (ix + 1);
  if (fl & F_MISALIGN) offset_set(p, R.mis, fl, G, m, true);
  if (fl & F_EDGE_IN) hwang_edge<true>(p, q + B_EDGE);
  if (orbit_too_large(p, G)) return;
  if (ix > -1) bend_multipole_kicks(p, q, an, bn, ix, 0.5, G);
  const double g = q[B_G];
  const double step_len = q[B_STEP];
  for (int n = 1; n <= n_step; n++) {
    if (fl & F_K1_BODY) {
      sbend_k1_body(p, q);
      p.z = p.z + low_energy_z_correction(p, q + B_LEZ, step_len);
    } else if (fl & F_DRIFT_BODY) {
      track_a_drift<true>(p, step_len, G, m);
    } else {
      const double x = p.x, px = p.px, y = p.y, py = p.py, z = p.z, pz = p.pz;
      const double rel_p = 1 + pz;
      const double rel_p2 = rel_p * rel_p;
      if ((fl & F_SEMI_LINEAR_OK) && fabs(x * g) < 1e-9 && fabs(px) < 1e-9 && fabs(py) < 1e-9 &&
          fabs(pz) < 1e-9) {
        const double ll = step_len;
        double gam2 = G.mc2sq / (sq(rel_p * G.p0c) + G.mc2sq);
        double m56 = ll * (gam2 - q[B_M56C]);
        p.x = q[B_COSA] * x + q[B_LLSINC] * px + q[B_GLL2COSC] * pz;
        p.px = -(q[B_GSIN] * x) + q[B_COSA] * px + q[B_GLLSINC] * pz;
        p.y = y + ll * py;
        p.z = -(q[B_GLLSINC] * x) - q[B_GLL2COSC] * px + z + m56 * pz;
      } else {
        const double g_tot = q[B_GTOT];
        const double angle = q[B_ANGLE];
        const double sinc_a = q[B_SINCA];
        double pt = sqrt(rel_p2 - py * py);
        if (fabs(px) > pt) {
          p.state = LOST_PZ;
          return;
        }
        double g_p = g_tot / pt;
        double phi_1 = cr::asin(px / pt);
        double sin_plus = cr::sin(angle + phi_1), cos_plus = cr::cos(angle + phi_1);
        double gx1 = 1 + g * x;
        double t1 = gx1 * step_len * sinc_a;
        double alpha = 2 * gx1 * sin_plus * step_len * sinc_a - g_p * (t1 * t1);
        double r = cos_plus * cos_plus + g_p * alpha;
        if (r < 0 || (fabs(g_p) < 1e-5 && fabs(cos_plus) < 1e-5)) {
          p.state = LOST;
          p.x = 2 * G.mal;
          return;
        }
        double rad = sqrt(r);
        double xi;
        if (cos_plus > 0) {
          xi = alpha / (rad + cos_plus);
        } else {
          xi = (rad - cos_plus) / g_p;
        }
        p.x = x * q[B_COSA] - q[B_LL2GCOSC] + xi;
        if (fabs(p.x) > G.mal) {
          p.state = LOST;
          return;
        }
        double L_u = xi;
        double L_v = -(q[B_LLSINC] + x * q[B_SINA]);
        double L_c = sqrt(L_v * L_v + L_u * L_u);
        double angle_p = 2 * (angle + phi_1 - 1 * cr::atan2(L_u, -L_v));
        double L_p = 1 * L_c / sinc_d(angle_p / 2);
        p.px = pt * cr::sin(phi_1 + angle - angle_p);
        p.y = y + py * L_p / pt;
        p.z = z + p.beta * step_len / q[B_BETAREF] - rel_p * L_p / pt;
      }
    }
    if (ix > -1) bend_multipole_kicks(p, q, an, bn, ix, (n == n_step) ? 0.5 : 1.0, G);
  }
  if (orbit_too_large(p, G)) return;
  if (fl & F_EDGE_OUT) hwang_edge<false>(p, q + B_EDGE + EDGE_N);
  if (fl & F_MISALIGN) offset_unset(p, R.mis, fl, G, m, true);
}

// track1, bmad/code/track1.f90:43-342 for one alive particle and one record:
// entrance aperture, body, orbit_too_large, exit aperture.  Returns the
// particle's state (ALIVE or a lost code).
__device__ __forceinline__ void track1_rec(Part& p, const double* rec, const Glob& G, DriftMemo& m, QMemo qm) {
  Rec R = decode(rec);
  const int32_t fl = R.h->flags;
  if ((fl & F_AP_ENTRANCE) && G.ap_on) {
    check_aperture(p, R.ap, R.mis, fl, false);
    if (p.state != ALIVE) return;
  }
  switch (R.h->kind) {
    case K_DRIFT:
      track_a_drift<true>(p, R.kb[DR_L], G, m);
      break;
    case K_QUAD:
      body_quad(p, R, G, m, qm);
      break;
    case K_BEND:
      body_bend(p, R, G, m);
      break;
    case K_THICK_MULT:
      body_thick(p, R, G, m);
      break;
    case K_THIN_MULT:
      body_thin(p, R, G, m);
      break;
    case K_RFCAVITY:
      body_rf(p, R, G, m);
      break;
    default:
      break;
  }
  if (orbit_too_large(p, G)) return;
  if (p.state != ALIVE) return;
  if ((fl & F_AP_EXIT) && G.ap_on) check_aperture(p, R.ap, R.mis, fl, true);
}

// ===========================================================================
// TMA bulk copy + mbarrier (inline PTX, sm_90+ forms valid on sm_100a).

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void tma_bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}
// Bounded wait on the mbarrier phase.  Returns false after max_iters tries.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, uint32_t max_iters) {
  for (uint32_t it = 0; it < max_iters; it++) {
    uint32_t done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

// ===========================================================================
// Kernel

struct KArgs {
  // particles (SoA)
  double* vec6;  // [6][n_stride]
  double* beta;
  int32_t* state;
  int32_t* ix_ele_lost;
  int32_t* ix_turn_lost;
  const int32_t* slot_particle;  // slot -> particle index, -1 = padding (nullptr = identity)
  const int32_t* tile_variant;   // tile -> variant (nullptr = variant 0)
  int64_t n;                     // particles
  int64_t n_stride;              // coordinate stride in vec6
  int64_t n_slots;               // slots (multiple of block size when tile_variant is set)
  // tables
  const double* tables;           // all variants, each 16-byte aligned
  // Per variant: [sequence: n_rec x (int32 record offset in doubles, int32
  // ix_ele)] [pool of unique records].  Identical elements share one record.
  const int64_t* table_off_dw;    // [variant] offset in doubles
  int32_t table_dw;               // doubles per table (max over variants, multiple of 2)
  int32_t rec_begin, rec_end;     // element range [begin, end) per turn
  int32_t n_rec;                  // elements per table
  int32_t turn0, n_turns;
  int32_t compact_every;
  int32_t* tile_counter;
  int32_t* error_flag;
  Glob G;
};

constexpr int MAX_BLOCK = 256;

// TMODE 0: the variant's element table is staged in shared memory.
// TMODE 1: it is read from global memory (L2 / L1) instead -- for tables
//   larger than the shared-memory budget (e.g. every quadrupole and sextupole
//   misaligned and carrying its own multipole errors), or to leave shared
//   memory to more resident CTAs; CTA-wide tiles as in TMODE 0.
// TMODE 2: global-memory tables with every warp scheduled on its own.
template <int BLOCK, int MINB, int TMODE>
__global__ void __launch_bounds__(BLOCK, MINB) track_kernel(KArgs a) {
  constexpr bool GTAB = TMODE != 0;
  extern __shared__ __align__(128) double smem[];
  __shared__ __align__(8) uint64_t bar;
  __shared__ int32_t s_tile;
  __shared__ int32_t s_warp_cnt[BLOCK / 32];
  const double* table = smem;
  // compaction staging area sits after the table
  double* stage = smem + (GTAB ? 0 : a.table_dw);  // [9][BLOCK] doubles; rows 7-8 hold int32 ids and loss records
  int32_t* stage_i = reinterpret_cast<int32_t*>(stage + 7 * BLOCK);  // [3][BLOCK]
  // quad memo after the (optional) compaction stage
  double* qmemo_base = stage + (a.compact_every > 0 ? 9 * BLOCK : 0);
  const QMemo qmemo{qmemo_base + threadIdx.x, BLOCK};

  const int tid = threadIdx.x;
  if (TMODE == 2) {
    // Tables in global memory: no CTA-wide state to share, so every warp
    // runs its own persistent loop over 32-slot tiles and never waits at a
    // CTA barrier for warps whose particles live longer (DA scans mix
    // short- and long-lived probes in one tile).  No compaction here.
    const int lane = tid & 31;
    const int64_t n_wtiles = (a.n_slots + 31) / 32;
    while (true) {
      int64_t wt = 0;
      if (lane == 0) wt = atomicAdd(a.tile_counter, 1);
      wt = __shfl_sync(0xffffffffu, wt, 0);
      if (wt >= n_wtiles) break;
      const int64_t slot = wt * 32 + lane;
      // slots are grouped per variant in multiples of the CTA size, so the
      // 32 slots of a warp tile share one variant
      const int variant = a.tile_variant ? a.tile_variant[(wt * 32) / BLOCK] : 0;
      const double* wtable = a.tables + a.table_off_dw[variant];
      const int2* wseq = reinterpret_cast<const int2*>(wtable);
      int64_t pidx = -1;
      if (slot < a.n_slots) pidx = a.slot_particle ? a.slot_particle[slot] : slot;
      if (pidx >= a.n) pidx = -1;
      Part p;
      int32_t ixe = -1, ixt = -1;
      p.state = 0;
      if (pidx >= 0) {
        p.x = a.vec6[0 * a.n_stride + pidx];
        p.px = a.vec6[1 * a.n_stride + pidx];
        p.y = a.vec6[2 * a.n_stride + pidx];
        p.py = a.vec6[3 * a.n_stride + pidx];
        p.z = a.vec6[4 * a.n_stride + pidx];
        p.pz = a.vec6[5 * a.n_stride + pidx];
        p.beta = a.beta[pidx];
        p.state = a.state[pidx];
        ixe = a.ix_ele_lost[pidx];
        if (a.ix_turn_lost) ixt = a.ix_turn_lost[pidx];
      }
      DriftMemo memo;
      memo.pz = NAN;
      memo.a = 0;
#pragma unroll
      for (int c = 0; c < QMEMO_CLASSES; c++) qmemo.q[(c * 13 + 12) * qmemo.stride] = NAN;
      if (p.state == ALIVE && orbit_too_large(p, a.G)) {
        ixe = wseq[a.rec_begin].y;
        ixt = a.turn0;
      }
      for (int t = 0; t < a.n_turns; t++) {
        if (__all_sync(0xffffffffu, p.state != ALIVE)) break;  // whole warp lost
        const int turn = a.turn0 + t;
        for (int r = a.rec_begin; r < a.rec_end; r++) {
          const int2 e = wseq[r];
          if (p.state == ALIVE) {
            track1_rec(p, wtable + e.x, a.G, memo, qmemo);
            if (p.state != ALIVE) {
              ixe = e.y;
              ixt = turn;
            }
          }
        }
      }
      if (pidx >= 0) {
        a.vec6[0 * a.n_stride + pidx] = p.x;
        a.vec6[1 * a.n_stride + pidx] = p.px;
        a.vec6[2 * a.n_stride + pidx] = p.y;
        a.vec6[3 * a.n_stride + pidx] = p.py;
        a.vec6[4 * a.n_stride + pidx] = p.z;
        a.vec6[5 * a.n_stride + pidx] = p.pz;
        a.beta[pidx] = p.beta;
        a.state[pidx] = p.state;
        a.ix_ele_lost[pidx] = ixe;
        if (a.ix_turn_lost) a.ix_turn_lost[pidx] = ixt;
      }
    }
    return;
  }
  if (tid == 0) mbar_init(&bar, 1);
  __syncthreads();
  uint32_t parity = 0;
  int loaded_variant = -1;
  const uint32_t table_bytes = (uint32_t)a.table_dw * 8u;
  const int64_t n_tiles = (a.n_slots + BLOCK - 1) / BLOCK;

  while (true) {
    if (tid == 0) s_tile = atomicAdd(a.tile_counter, 1);
    __syncthreads();
    const int64_t tile = s_tile;
    if (tile >= n_tiles) break;
    const int variant = a.tile_variant ? a.tile_variant[tile] : 0;
    if (GTAB) {
      table = a.tables + a.table_off_dw[variant];
    } else if (variant != loaded_variant) {
      // all threads finished reading the previous table (barrier above)
      if (tid == 0) {
        mbar_expect_tx(&bar, table_bytes);
        tma_bulk_g2s(smem, a.tables + a.table_off_dw[variant], table_bytes, &bar);
      }
      const int bad = __syncthreads_or(!mbar_wait(&bar, parity, 1u << 26));
      if (bad) {
        if (tid == 0) atomicExch(a.error_flag, 1);
        return;
      }
      parity ^= 1u;
      loaded_variant = variant;
    }
    const int2* seq = reinterpret_cast<const int2*>(table);

    // ---- load my particle ----
    const int64_t slot = tile * BLOCK + tid;
    int64_t pidx = -1;
    if (slot < a.n_slots) pidx = a.slot_particle ? a.slot_particle[slot] : slot;
    if (pidx >= a.n) pidx = -1;
    Part p;
    int32_t ixe = -1, ixt = -1;
    p.state = 0;
    if (pidx >= 0) {
      p.x = a.vec6[0 * a.n_stride + pidx];
      p.px = a.vec6[1 * a.n_stride + pidx];
      p.y = a.vec6[2 * a.n_stride + pidx];
      p.py = a.vec6[3 * a.n_stride + pidx];
      p.z = a.vec6[4 * a.n_stride + pidx];
      p.pz = a.vec6[5 * a.n_stride + pidx];
      p.beta = a.beta[pidx];
      p.state = a.state[pidx];
      ixe = a.ix_ele_lost[pidx];
      if (a.ix_turn_lost) ixt = a.ix_turn_lost[pidx];
    }
    DriftMemo memo;
    memo.pz = NAN;
    memo.a = 0;
#pragma unroll
    for (int c = 0; c < QMEMO_CLASSES; c++) qmemo.q[(c * 13 + 12) * qmemo.stride] = NAN;
    int32_t my_idx = (int32_t)pidx;  // particle carried by this lane (changes on compaction)

    // entrance check of the first element (check_aperture_limit ->
    // orbit_too_large, track1.f90:195)
    if (p.state == ALIVE) {
      if (orbit_too_large(p, a.G)) {
        ixe = seq[a.rec_begin].y;
        ixt = a.turn0;
      }
    }

    for (int t = 0; t < a.n_turns; t++) {
      const int turn = a.turn0 + t;
      if (__all_sync(0xffffffffu, p.state != ALIVE)) {
        // whole warp dead: nothing to do this turn (no block barrier inside
        // the turn unless compaction is on)
      } else {
        for (int r = a.rec_begin; r < a.rec_end; r++) {
          const int2 e = seq[r];
          if (p.state == ALIVE) {
            track1_rec(p, table + e.x, a.G, memo, qmemo);
            if (p.state != ALIVE) {
              ixe = e.y;
              ixt = turn;
            }
          }
        }
      }
      // ---- intra-tile compaction (warp ballot + block prefix sum) ----
      if (a.compact_every > 0 && ((t + 1) % a.compact_every) == 0 && t + 1 < a.n_turns) {
        const bool alive = (p.state == ALIVE);
        const unsigned ballot = __ballot_sync(0xffffffffu, alive);
        const int warp = tid >> 5, lane = tid & 31;
        if (lane == 0) s_warp_cnt[warp] = __popc(ballot);
        __syncthreads();
        int base = 0, total = 0;
        for (int w = 0; w < BLOCK / 32; w++) {
          int c = s_warp_cnt[w];
          if (w < warp) base += c;
          total += c;
        }
        // Only worth moving when at least one warp can go idle.
        const bool do_move = total <= BLOCK - 32 && total > 0;
        if (do_move) {
          // dead particles write their final state back now (their lane is reused)
          if (!alive && my_idx >= 0) {
            a.vec6[0 * a.n_stride + my_idx] = p.x;
            a.vec6[1 * a.n_stride + my_idx] = p.px;
            a.vec6[2 * a.n_stride + my_idx] = p.y;
            a.vec6[3 * a.n_stride + my_idx] = p.py;
            a.vec6[4 * a.n_stride + my_idx] = p.z;
            a.vec6[5 * a.n_stride + my_idx] = p.pz;
            a.beta[my_idx] = p.beta;
            a.state[my_idx] = p.state;
            a.ix_ele_lost[my_idx] = ixe;
            if (a.ix_turn_lost) a.ix_turn_lost[my_idx] = ixt;
          }
          const int dst = base + __popc(ballot & ((1u << lane) - 1u));
          if (alive) {
            stage[0 * BLOCK + dst] = p.x;
            stage[1 * BLOCK + dst] = p.px;
            stage[2 * BLOCK + dst] = p.y;
            stage[3 * BLOCK + dst] = p.py;
            stage[4 * BLOCK + dst] = p.z;
            stage[5 * BLOCK + dst] = p.pz;
            stage[6 * BLOCK + dst] = p.beta;
            stage_i[dst] = my_idx;
            stage_i[BLOCK + dst] = ixe;
            stage_i[2 * BLOCK + dst] = ixt;
          }
          __syncthreads();
          if (tid < total) {
            p.x = stage[0 * BLOCK + tid];
            p.px = stage[1 * BLOCK + tid];
            p.y = stage[2 * BLOCK + tid];
            p.py = stage[3 * BLOCK + tid];
            p.z = stage[4 * BLOCK + tid];
            p.pz = stage[5 * BLOCK + tid];
            p.beta = stage[6 * BLOCK + tid];
            my_idx = stage_i[tid];
            ixe = stage_i[BLOCK + tid];
            ixt = stage_i[2 * BLOCK + tid];
            p.state = ALIVE;
            memo.pz = NAN;
#pragma unroll
            for (int c = 0; c < QMEMO_CLASSES; c++) qmemo.q[(c * 13 + 12) * qmemo.stride] = NAN;
          } else {
            p.state = 0;
            my_idx = -1;
          }
        }
        __syncthreads();
      }
    }

    // ---- store ----
    if (my_idx >= 0) {
      a.vec6[0 * a.n_stride + my_idx] = p.x;
      a.vec6[1 * a.n_stride + my_idx] = p.px;
      a.vec6[2 * a.n_stride + my_idx] = p.y;
      a.vec6[3 * a.n_stride + my_idx] = p.py;
      a.vec6[4 * a.n_stride + my_idx] = p.z;
      a.vec6[5 * a.n_stride + my_idx] = p.pz;
      a.beta[my_idx] = p.beta;
      a.state[my_idx] = p.state;
      a.ix_ele_lost[my_idx] = ixe;
      if (a.ix_turn_lost) a.ix_turn_lost[my_idx] = ixt;
    }
    __syncthreads();
  }
}

}  // namespace bgt

// ===========================================================================
// Host side: table compiler, handle, C ABI.
// Element constants are evaluated here with the host C library (glibc libm),
// the same library the reference evaluates them with.

namespace bgt {
namespace host {

static const double PI_H = 3.141592653589793238462643383279;
static const double TWOPI_H = 2 * PI_H;

static double sinc_h(double x) { return fabs(x) < 1e-8 ? 1.0 : sin(x) / x; }
static double cosc_h(double x) {
  if (fabs(x) < 1e-8) return 0.50;
  double s = sinc_h(x / 2);
  return 0.5 * (s * s);
}
static double sincc_h(double x) {
  const double c0 = 1.0 / 6.0, c1 = -1.0 / 120.0, c2 = 1.0 / 5040.0, c3 = -1.0 / 362880.0;
  double x2 = x * x;
  if (fabs(x) < 0.1) return c0 + x2 * (c1 + x2 * (c2 + x2 * c3));
  return (x - sin(x)) / (x * x2);
}
static int nint_h(double x) { return (int)lround(x); }

static int max_nonzero(const double* a, const double* b, int n) {
  for (int i = n - 1; i >= 0; i--) {
    if (a[i] != 0) return i;
    if (b && b[i] != 0) return i;
  }
  return -1;
}

// floor_angles_to_w_mat, bmad/geometry/floor_angles_to_w_mat.f90:17-57, psi = 0
static void w_mats(double theta, double phi, double w[9], double winv[9]) {
  double s_the = sin(theta), c_the = cos(theta);
  double s_phi = sin(phi), c_phi = cos(phi);
  double s_psi = sin(0.0), c_psi = cos(0.0);
  w[0] = c_the * c_psi - s_the * s_phi * s_psi;
  w[1] = -c_the * s_psi - s_the * s_phi * c_psi;
  w[2] = s_the * c_phi;
  w[3] = c_phi * s_psi;
  w[4] = c_phi * c_psi;
  w[5] = s_phi;
  w[6] = -s_the * c_psi - c_the * s_phi * s_psi;
  w[7] = s_the * s_psi - c_the * s_phi * c_psi;
  w[8] = c_the * c_phi;
  winv[0] = c_the * c_psi - s_the * s_phi * s_psi;
  winv[1] = c_phi * s_psi;
  winv[2] = -s_the * c_psi - c_the * s_phi * s_psi;
  winv[3] = -c_the * s_psi - s_the * s_phi * c_psi;
  winv[4] = c_phi * c_psi;
  winv[5] = s_the * s_psi - c_the * s_phi * c_psi;
  winv[6] = s_the * c_phi;
  winv[7] = s_phi;
  winv[8] = c_the * c_phi;
}

struct Builder {
  std::vector<double>& out;
  size_t start;
  explicit Builder(std::vector<double>& o) : out(o), start(o.size()) { out.resize(start + HDR_DW, 0.0); }
  RecHdr* hdr() { return reinterpret_cast<RecHdr*>(out.data() + start); }
  // Appends n zeros and returns a pointer to them (valid until the next append).
  double* ptr_after_push(int n) {
    size_t at = out.size();
    out.resize(at + n, 0.0);
    return out.data() + at;
  }
  void finish() {
    // keep every record 16-byte aligned
    if ((out.size() - start) % 2) out.push_back(0.0);
    hdr()->size_dw = (int32_t)(out.size() - start);
  }
};

static std::string ename(const bgt_element& e) { return "element ix_ele=" + std::to_string(e.ix_ele); }

// low_energy_z_correction element constants (low_energy_z_correction.f90:22-58)
static void put_lez(double* q, const bgt_element& e, double mass, double p0c) {
  double beta0 = p0c / e.e_tot;
  q[LEZ_BETA0] = beta0;
  q[LEZ_F] = (beta0 * beta0) * (2 * (beta0 * beta0) - ((mass / e.e_tot) * (mass / e.e_tot)) / 2);
  q[LEZ_ME2] = (mass / e.e_tot) * (mass / e.e_tot);
  q[LEZ_MASS] = mass;
  q[LEZ_3E7] = 3e-7 * e.e_tot;
}

// Hwang edge constants (fringe_mod.f90:240-300)
static void put_edge(double* E, const bgt_element& e, bool entering) {
  double c_dir = 1.0;
  double g_tot = e.is_on ? (e.g + e.dg) * c_dir : 0.0;
  double k1 = e.is_on ? e.k1 : 0.0;
  double ang = entering ? e.e1 : e.e2;
  double fint_gap = entering ? e.fint * e.hgap : e.fintx * e.hgapx;
  if (e.fringe_type == BGT_FRINGE_HARD_EDGE_ONLY) fint_gap = 0;
  double cos_e = cos(ang), sin_e = sin(ang);
  double tan_e = sin_e / cos_e, sec_e = 1 / cos_e;
  double gt = g_tot * tan_e;
  double gt2 = g_tot * (tan_e * tan_e);
  double gs2 = g_tot * (sec_e * sec_e);
  double k1_tane = k1 * tan_e * c_dir;
  double fg = 2 * fint_gap * gs2 * g_tot * sec_e * (1 + sin_e * sin_e);
  E[EDGE_GT] = gt;
  E[EDGE_GT2] = gt2;
  E[EDGE_GS2] = gs2;
  E[EDGE_K1TANE] = k1_tane;
  E[EDGE_K1TANE2] = 2 * k1_tane;
  E[EDGE_FG] = fg;
  E[EDGE_C1] = entering ? (gt * g_tot) * (1 + 2 * (tan_e * tan_e)) : gt * gt2;
  E[EDGE_C3] = 4.0 * k1_tane - gt * gt2;
  E[EDGE_C4] = -4.0 * k1_tane + gt * gs2;
  E[EDGE_GPG] = g_tot + gt2;
  E[EDGE_GTGS2_2K1] = gt * gs2 - 2 * k1_tane;
}

// Compile one element into a record.  Returns 0 or BGT_EUNSUPPORTED with err set.
static int compile_element(const bgt_element& e, const bgt_species& sp, double p0c, std::vector<double>& out,
                           std::string& err) {
  const int ixe = max_nonzero(e.an_elec, e.bn_elec, BGT_N_POLE);
  if (ixe > -1 && e.is_on && e.key != BGT_QUADRUPOLE && e.key != BGT_SEXTUPOLE && e.key != BGT_OCTUPOLE &&
      e.key != BGT_THICK_MULTIPOLE) {
    err = ename(e) + ": electric multipoles are supported on quadrupoles and thick multipoles only";
    return BGT_EUNSUPPORTED;
  }
  if (e.p0c != p0c) {
    err = ename(e) + ": element p0c differs from the lattice reference momentum";
    return BGT_EUNSUPPORTED;
  }
  Builder B(out);
  int32_t flags = 0;
  int key = e.key;
  int kind;
  bool off = !e.is_on;
  // track1_bmad.f90:51-60: an element that is off becomes a drift (multipoles do nothing)
  if (off) {
    if (key == BGT_MULTIPOLE || key == BGT_AB_MULTIPOLE || key == BGT_MARKER) kind = K_MARKER;
    else if (key == BGT_SBEND) kind = K_BEND;
    else kind = K_DRIFT;
  } else {
    switch (key) {
      case BGT_DRIFT: kind = K_DRIFT; break;
      case BGT_MARKER: kind = K_MARKER; break;
      case BGT_QUADRUPOLE: kind = K_QUAD; break;
      case BGT_SBEND: kind = K_BEND; break;
      case BGT_SEXTUPOLE: case BGT_OCTUPOLE: case BGT_THICK_MULTIPOLE: case BGT_MONITOR: case BGT_INSTRUMENT:
      case BGT_PIPE: case BGT_RCOLLIMATOR: case BGT_ECOLLIMATOR: case BGT_KICKER: case BGT_HKICKER:
      case BGT_VKICKER:
        kind = K_THICK_MULT;
        break;
      case BGT_MULTIPOLE: case BGT_AB_MULTIPOLE: kind = K_THIN_MULT; break;
      case BGT_RFCAVITY: kind = K_RFCAVITY; break;
      default:
        err = ename(e) + ": element key " + std::to_string(key) + " is not supported";
        return BGT_EUNSUPPORTED;
    }
  }

  // ---- misalignment (offset_particle) ----
  bool offset = e.x_offset != 0 || e.y_offset != 0 || e.z_offset != 0 || e.x_pitch != 0 || e.y_pitch != 0;
  bool pitch = e.x_pitch != 0 || e.y_pitch != 0;
  bool use_mis = false;
  double tilt = 0;
  if (kind == K_QUAD || kind == K_THICK_MULT || kind == K_THIN_MULT) {
    use_mis = e.has_misalign != 0;
    tilt = e.tilt;
  } else if (kind == K_RFCAVITY) {
    use_mis = true;  // track_a_rfcavity calls offset_particle unconditionally
    tilt = e.tilt;
  } else if (kind == K_BEND) {
    if (offset || e.roll != 0) {
      err = ename(e) + ": bend offsets/pitches/roll are not supported";
      return BGT_EUNSUPPORTED;
    }
    use_mis = e.has_misalign != 0 && e.ref_tilt != 0;
    tilt = e.ref_tilt;
  }
  if (use_mis) {
    flags |= F_MISALIGN;
    if (offset) flags |= F_OFFSET;
    if (pitch) flags |= F_PITCH;
    if (tilt != 0 && kind != K_THIN_MULT) flags |= F_TILT;
    if (kind == K_RFCAVITY && e.is_on && (e.hkick != 0 || e.vkick != 0)) flags |= F_HV_KICK;
  }
  // ---- aperture ----
  bool ap_any = e.aperture_type != BGT_APERTURE_NONE && e.aperture_at != BGT_NO_END;
  bool ap_ell = e.aperture_type == BGT_APERTURE_ELLIPTICAL;
  if (ap_any) {
    if (ap_ell) {
      double x1 = -e.x1_limit, x2 = e.x2_limit, y1 = -e.y1_limit, y2 = e.y2_limit;
      // elliptical_params_setup error (check_aperture_limit.f90:344-349) -> no check
      if ((x1 == 0 && x2 != 0) || (x1 != 0 && x2 == 0) || (y1 == 0 && y2 != 0) || (y1 != 0 && y2 == 0))
        ap_any = false;
    } else if (e.x1_limit == 0 && e.x2_limit == 0 && e.y1_limit == 0 && e.y2_limit == 0) {
      ap_any = false;
    }
  }
  if (ap_any) {
    if (e.offset_moves_aperture && (flags & F_MISALIGN) && (offset || tilt != 0)) {
      if (kind == K_BEND) {
        err = ename(e) + ": offset_moves_aperture on a bend is not supported";
        return BGT_EUNSUPPORTED;
      }
      flags |= F_AP_OFFSET;
      if (key == BGT_ECOLLIMATOR || key == BGT_RCOLLIMATOR) flags |= F_AP_TILT;
    }
    if (e.aperture_at == BGT_ENTRANCE_END || e.aperture_at == BGT_BOTH_ENDS) flags |= F_AP_ENTRANCE;
    if (e.aperture_at == BGT_EXIT_END || e.aperture_at == BGT_BOTH_ENDS) flags |= F_AP_EXIT;
    flags |= ap_ell ? F_AP_ELLIPTICAL : F_AP_RECT;
  }

  if (flags & F_MISALIGN) {
    double* m = B.ptr_after_push(MIS_N);
    double L = e.l;
    double L_half = 0.5 * L;
    m[MIS_XOFF] = e.x_offset;
    m[MIS_YOFF] = e.y_offset;
    m[MIS_ZOFF] = e.z_offset;
    m[MIS_LHALF] = L_half;
    m[MIS_COS] = cos(tilt);
    m[MIS_SIN] = sin(tilt);
    m[MIS_COSU] = cos(-tilt);
    m[MIS_SINU] = sin(-tilt);
    w_mats(e.x_pitch, e.y_pitch, m + MIS_W, m + MIS_WINV);
    m[MIS_HK] = 0.5 * 1.0 * e.hkick;
    m[MIS_VK] = 0.5 * 1.0 * e.vkick;
    // set: ds_center = L_half - s_pos0 (s_pos0 = 0); r(3) = 0 - (z_off + ds_center) then + L_half
    double ds_center_set = L_half - 0.0;
    m[MIS_R3SET] = 0.0 - (e.z_offset + 1 * ds_center_set);
    double s_body = m[MIS_R3SET] + L_half;
    m[MIS_DS_SET] = (1 - 1) * L_half - s_body;
    // unset: s_pos0 = L; r(3) = 0 - ds_center, then + (z_off + L_half)
    double ds_center_unset = L_half - L;
    m[MIS_R3UNSET] = 0.0 - ds_center_unset;
    m[MIS_ZADD] = e.z_offset + L_half;
    // aperture in the element frame at the exit: s_pos = L
    double ds_center_exit = L_half - L;
    m[MIS_R3EXIT] = 0.0 - (e.z_offset + 1 * ds_center_exit);
    double s_lab = m[MIS_R3UNSET] + m[MIS_ZADD];
    m[MIS_DS_UNSET] = (1 + 1) * L_half - s_lab;
  }
  if (flags & (F_AP_ENTRANCE | F_AP_EXIT)) {
    double* a = B.ptr_after_push(AP_N);
    a[AP_X1] = -e.x1_limit;
    a[AP_X2] = e.x2_limit;
    a[AP_Y1] = -e.y1_limit;
    a[AP_Y2] = e.y2_limit;
    if (ap_ell) {
      double w = (a[AP_X2] - a[AP_X1]) / 2, c = (a[AP_X2] + a[AP_X1]) / 2;
      if (w == 0) w = sp.max_aperture_limit;
      a[AP_XW] = std::max(w, 0.0);
      a[AP_XC] = c;
      w = (a[AP_Y2] - a[AP_Y1]) / 2;
      c = (a[AP_Y2] + a[AP_Y1]) / 2;
      if (w == 0) w = sp.max_aperture_limit;
      a[AP_YW] = std::max(w, 0.0);
      a[AP_YC] = c;
    }
  }

  RecHdr h{};
  h.kind = kind;
  h.ix_ele = e.ix_ele;
  h.ix_mag_max = -1;
  h.n_step = 0;
  double an[BGT_N_POLE], bn[BGT_N_POLE];
  memcpy(an, e.an, sizeof(an));
  memcpy(bn, e.bn, sizeof(bn));
  int ix = max_nonzero(an, bn, BGT_N_POLE);

  switch (kind) {
    case K_MARKER:
      break;
    case K_DRIFT: {
      double* q = B.ptr_after_push(DR_N);
      q[DR_L] = e.l * 1;
      break;
    }
    case K_QUAD: {
      // pull_this_b1 (multipole_ele_to_ab.f90:660-676)
      double b1 = bn[1];
      bn[1] = 0;
      if (ix <= 1) ix = max_nonzero(an, bn, 2);
      double length = 1 * e.l;
      int n_step = 1;
      if (ix > -1 || ixe > -1) n_step = std::max(nint_h(fabs(length) / e.ds_step), 1);
      double r_step = 1.0 / n_step;
      double step_len = e.l * r_step;
      if (length == 0) n_step = 0;
      double* q = B.ptr_after_push(Q_N);
      q[Q_LEN] = length;
      q[Q_B1] = 1.0 * b1;
      q[Q_STEP] = step_len;
      q[Q_RHALF] = r_step / 2;
      q[Q_RSTEP] = r_step;
      put_lez(q + Q_LEZ, e, sp.mass, p0c);
      h.n_step = n_step;
      h.ix_mag_max = ix;
      break;
    }
    case K_THICK_MULT: {
      if (key == BGT_PIPE) ix = -1;  // multipole_ele_to_ab returns nothing for pipes
      double length = e.l * 1;
      int n_step = (ix == -1 && ixe == -1) ? 1 : std::max(nint_h(fabs(length / e.ds_step)), 1);
      double r_step = 1.0 / n_step;
      double step_len = length / n_step;
      double* q = B.ptr_after_push(TM_N);
      q[TM_STEP] = step_len;
      q[TM_RHALF] = 1 * r_step / 2;
      q[TM_RSTEP] = 1 * r_step;
      h.n_step = n_step;
      h.ix_mag_max = ix;
      break;
    }
    case K_THIN_MULT: {
      int ixk = max_nonzero(e.knl, nullptr, BGT_N_POLE);
      double* q = B.ptr_after_push(TH_N + TH_POLE * (ixk + 1));
      q[TH_REFORB] = (key == BGT_MULTIPOLE) ? 1.0 : 0.0;
      for (int n = 0; n <= ixk; n++) {
        double* pp = q + TH_N + TH_POLE * n;
        pp[0] = e.knl[n];
        pp[1] = cos(e.tn[n]);
        pp[2] = sin(e.tn[n]);
        pp[3] = (e.tn[n] == 0) ? 1.0 : 0.0;
      }
      h.ix_mag_max = ixk;
      ix = -1;  // no (an, bn) arrays
      break;
    }
    case K_RFCAVITY: {
      if (e.coupler_strength != 0) {
        err = ename(e) + ": rf coupler kicks are not supported";
        return BGT_EUNSUPPORTED;
      }
      if (e.rf_frequency == 0 && e.voltage != 0) {
        err = ename(e) + ": rfcavity has zero rf_frequency";
        return BGT_EINVAL;
      }
      double length = e.l * 1;
      int n_step = 1;
      double r_step = 1.0 / n_step;
      int n_slice = std::max(1, nint_h(fabs(length) / e.ds_step));
      double* q = B.ptr_after_push(RF_N);
      q[RF_LEN] = length;
      q[RF_VOLT] = (e.is_on ? e.voltage * 1 : 0.0) * 1.0;
      q[RF_PHI0] = e.phi0;
      q[RF_FREQ] = e.rf_frequency;
      q[RF_NSLICE] = n_slice;
      q[RF_SLICE_L] = length / n_slice;
      q[RF_TWOPI_F] = TWOPI_H * e.rf_frequency;
      if (e.rf_frequency != 0) {
        __float128 amp = ((__float128)0.5) / (__float128)e.rf_frequency;
        double hi = (double)amp;
        q[RF_HALF_AMP_HI] = hi;
        q[RF_HALF_AMP_LO] = (double)(amp - (__float128)hi);
      }
      q[RF_PHI0_MP] = TWOPI_H * e.phi0_multipass;
      q[RF_RHALF] = 0.5 * r_step;
      h.n_step = n_slice;
      h.ix_mag_max = ix;
      break;
    }
    case K_BEND: {
      if (e.exact_multipoles != 0) {
        err = ename(e) + ": exact_multipoles is not supported";
        return BGT_EUNSUPPORTED;
      }
      bool edges = e.fringe_type != BGT_FRINGE_NONE;
      if (edges && e.fringe_type != BGT_FRINGE_BASIC_BEND && e.fringe_type != BGT_FRINGE_HARD_EDGE_ONLY) {
        err = ename(e) + ": bend fringe_type other than basic_bend/hard_edge_only is not supported";
        return BGT_EUNSUPPORTED;
      }
      // multipole_ele_to_ab(..., include_kicks$, b1) then track_a_bend.f90:58-94
      double b1 = bn[1];
      bn[1] = 0;
      if (ix <= 1) ix = max_nonzero(an, bn, 2);
      b1 = b1 * 1.0;
      if (fabs(b1) < 1e-10) {
        bn[1] = b1;
        b1 = 0;
      }
      double length = 1 * e.l;
      double g = e.g, dg;
      if (length == 0) {
        dg = 0;
      } else {
        dg = bn[0] / e.l;
        bn[0] = 0;
      }
      double g_tot = (g + dg) * 1.0;
      if (off) {
        dg = -g;
        g_tot = 0;
        b1 = 0;
      }
      int n_step = 1;
      if (ix > -1) n_step = std::max(nint_h(fabs(length) / e.ds_step), 1);
      double r_step = 1.0 / n_step;
      double step_len = length / n_step;
      double angle = g * step_len;
      double* q = B.ptr_after_push(B_N);
      q[B_LEN] = length;
      q[B_G] = g;
      q[B_DG] = dg;
      q[B_GTOT] = g_tot;
      q[B_STEP] = step_len;
      q[B_ANGLE] = angle;
      q[B_RSTEP] = r_step;
      double cos_a = cos(angle), sin_a = sin(angle), sinc_a = sinc_h(angle), cosc_a = cosc_h(angle);
      q[B_COSA] = cos_a;
      q[B_SINA] = sin_a;
      q[B_SINCA] = sinc_a;
      q[B_COSCA] = cosc_a;
      q[B_BETAREF] = e.p0c / e.e_tot;
      q[B_B1] = b1;
      double ll = step_len;
      q[B_LL2GCOSC] = ((step_len * step_len) * g) * cosc_a;
      q[B_LLSINC] = ll * sinc_a;
      q[B_M56C] = ((g * ll) * (g * ll)) * sincc_h(angle);
      q[B_GLLSINC] = (g * ll) * sinc_a;
      q[B_GLL2COSC] = (g * (ll * ll)) * cosc_a;
      q[B_GSIN] = g * sin_a;
      q[B_FP0C] = r_step * e.p0c / (C_LIGHT * sp.charge);
      q[B_CDIR] = 1 * 1 * (double)sp.charge;
      put_lez(q + B_LEZ, e, sp.mass, p0c);
      q[B_K1 + 0] = b1 / e.l;
      q[B_K1 + 1] = 1 * e.l / n_step;
      q[B_K1 + 2] = g_tot;
      if (edges) {
        if (e.fringe_at == BGT_ENTRANCE_END || e.fringe_at == BGT_BOTH_ENDS) flags |= F_EDGE_IN;
        if (e.fringe_at == BGT_EXIT_END || e.fringe_at == BGT_BOTH_ENDS) flags |= F_EDGE_OUT;
      }
      put_edge(q + B_EDGE, e, true);
      put_edge(q + B_EDGE + EDGE_N, e, false);
      if (b1 != 0) flags |= F_K1_BODY;
      else if ((g == 0 && dg == 0) || step_len == 0) flags |= F_DRIFT_BODY;
      if (dg == 0) flags |= F_SEMI_LINEAR_OK;
      if (off) flags |= F_IS_OFF;
      h.n_step = n_step;
      h.ix_mag_max = ix;
      break;
    }
    default:
      err = ename(e) + ": internal: unknown kind";
      return BGT_EUNSUPPORTED;
  }
  if (ix > -1 && (kind == K_QUAD || kind == K_THICK_MULT || kind == K_BEND || kind == K_RFCAVITY)) {
    double* q = B.ptr_after_push(2 * (ix + 1));
    for (int n = 0; n <= ix; n++) {
      q[n] = an[n];
      q[ix + 1 + n] = bn[n];
    }
  }
  h.aux1 = -1;
  if (kind == K_QUAD || kind == K_THICK_MULT) {
    // init_fringe_info (bmad/low_level/init_fringe_info.f90:22-60); the edge
    // kicks act at the ends fringe_at names (apply_element_edge_kick.f90:104)
    const bool fringe = (e.fringe_type != BGT_FRINGE_NONE && e.fringe_at != BGT_NO_END) || ixe > -1;
    if (fringe) flags |= F_FRINGE_INFO;
    if (e.fringe_at == BGT_ENTRANCE_END || e.fringe_at == BGT_BOTH_ENDS) flags |= F_EDGE_IN;
    if (e.fringe_at == BGT_EXIT_END || e.fringe_at == BGT_BOTH_ENDS) flags |= F_EDGE_OUT;
    if (ixe > -1) {
      flags |= F_ELEC;
      h.aux1 = ixe;
      double* q = B.ptr_after_push(2 * (ixe + 1));
      for (int n = 0; n <= ixe; n++) {
        q[n] = e.an_elec[n];
        q[ixe + 1 + n] = e.bn_elec[n];
      }
      // electric_longitudinal_fringe (apply_element_edge_kick.f90:283-329)
      // does nothing for zero length
      if (e.l != 0) flags |= F_ELEC_EDGE;
    }
    // hard_multipole_edge_kick (fringe_mod.f90:691-864) for quadrupoles and
    // sextupoles; soft_quadrupole_edge_kick is zero for fq1 = fq2 = 0 (the
    // defaults, the only values this table carries)
    if ((e.fringe_type == BGT_FRINGE_FULL || e.fringe_type == BGT_FRINGE_HARD_EDGE_ONLY) &&
        (key == BGT_QUADRUPOLE || key == BGT_SEXTUPOLE)) {
      flags |= F_HARD_EDGE;
      double* q = B.ptr_after_push(1);
      q[0] = (key == BGT_QUADRUPOLE) ? e.k1 : e.k2;
    }
  }
  h.flags = flags;
  *B.hdr() = h;
  B.finish();
  return 0;
}

// c_multi table, bmad/low_level/c_multi.f90:19-75
static void c_multi_tables(double cm[BGT_MAXPOLE_DEV + 1][BGT_MAXPOLE_DEV + 1],
                           double cm0[BGT_MAXPOLE_DEV + 1][BGT_MAXPOLE_DEV + 1]) {
  const int N = BGT_MAXPOLE_DEV + 1;
  double c[BGT_MAXPOLE_DEV + 1][BGT_MAXPOLE_DEV + 1] = {};
  double nf[BGT_MAXPOLE_DEV + 1];
  c[0][0] = 1;
  for (int in = 1; in < N; in++) {
    c[in][0] = 1;
    c[in][in] = 1;
    for (int im = 1; im <= in - 1; im++) c[in][im] = c[in - 1][im - 1] + c[in - 1][im];
  }
  nf[0] = 1;
  for (int in = 0; in < N; in++) {
    if (in > 0) nf[in] = in * nf[in - 1];
    for (int im = 0; im <= in; im++) {
      c[in][im] = c[in][im] / nf[in];
      if (im % 4 == 0) c[in][im] = -c[in][im];
      if (im % 4 == 3) c[in][im] = -c[in][im];
    }
  }
  for (int in = 0; in < N; in++)
    for (int im = 0; im < N; im++) {
      cm0[in][im] = c[in][im];
      cm[in][im] = c[in][im] * nf[in];
    }
}

}  // namespace host
}  // namespace bgt

// ===========================================================================
// Handle and C ABI

using namespace bgt;

struct bgt_handle {
  int device = 0;
  int num_sms = 148;
  int32_t n_ele = 0, n_variants = 0;
  bgt_species sp{};
  Glob G{};
  int32_t table_dw = 0;
  std::vector<double> h_tables;
  std::vector<int64_t> h_table_off;
  double* d_tables = nullptr;
  int64_t* d_table_off = nullptr;
  int32_t* d_scratch = nullptr;  // [0] tile counter, [1] error flag
  bgt_tuning tuning{128, 4, 0, 0, 0};
  std::string err;
  int64_t launches = 0;
  // host-API staging
  double* d_vec6 = nullptr;
  double* d_beta = nullptr;
  int32_t* d_i32 = nullptr;  // state, ixe, ixt, slot map, tile variant
  int64_t cap = 0, cap_slots = 0, cap_tiles = 0;
  // device-API grouping by variant: slot map, tile variant, and per variant
  // first index / count / first slot (int64) plus a check flag
  int32_t* d_grp = nullptr;
  int64_t* d_grp_v = nullptr;
  int64_t grp_cap_slots = 0, grp_cap_tiles = 0;
};

static int set_err(bgt_handle* h, int code, const std::string& msg) {
  if (h) h->err = msg;
  return code;
}

#define CU(h, call)                                                                              \
  do {                                                                                           \
    cudaError_t e_ = (call);                                                                     \
    if (e_ != cudaSuccess)                                                                       \
      return set_err((h), BGT_ECUDA, std::string(#call) + ": " + cudaGetErrorString(e_));        \
  } while (0)

// dynamic shared memory per CTA: B200 allows 227 KB per block, less the
// kernel's static shared memory
constexpr size_t SMEM_LIMIT = 224 * 1024;

static size_t smem_bytes(const bgt_handle* h, int block, bool compact, bool gtab = false) {
  size_t b = gtab ? 0 : (size_t)h->table_dw * 8;
  if (compact) b += (size_t)9 * block * 8;
  b += (size_t)QMEMO_CLASSES * 13 * block * 8;
  return b;
}

template <int BLOCK, int MINB, int TMODE = 0>
static cudaError_t launch_track(const KArgs& a, int grid, size_t smem, cudaStream_t st) {
  static bool attr_set[64] = {};
  int dev = 0;
  cudaGetDevice(&dev);
  if (!attr_set[dev & 63]) {
    cudaError_t e = cudaFuncSetAttribute(track_kernel<BLOCK, MINB, TMODE>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SMEM_LIMIT);
    if (e != cudaSuccess) return e;
    attr_set[dev & 63] = true;
  }
  track_kernel<BLOCK, MINB, TMODE><<<grid, BLOCK, smem, st>>>(a);
  return cudaGetLastError();
}

// Enqueue tracking of slots on `st`.
static int enqueue_track(bgt_handle* h, KArgs a, int64_t n_tiles, cudaStream_t st) {
  int block = h->tuning.threads_per_block;
  bool compact = a.compact_every > 0;
  const bool fits = smem_bytes(h, block, compact) <= SMEM_LIMIT;
  if (h->tuning.table_mode == 1 && !fits)
    return set_err(h, BGT_ETOOLARGE, "element table does not fit in shared memory (table_mode 1)");
  const bool gtab = h->tuning.table_mode >= 2 || !fits;
  const bool warp_sched = h->tuning.table_mode == 3;
  size_t smem = smem_bytes(h, block, compact, gtab);
  if (smem > SMEM_LIMIT) return set_err(h, BGT_ETOOLARGE, "tracking state does not fit in shared memory");
  int64_t grid = (int64_t)h->num_sms * std::max(1, h->tuning.blocks_per_sm);
  if (grid > n_tiles) grid = n_tiles;
  if (grid < 1) grid = 1;
  a.tile_counter = h->d_scratch;
  a.error_flag = h->d_scratch + 1;
  CU(h, cudaMemsetAsync(h->d_scratch, 0, sizeof(int32_t), st));
  cudaError_t e;
  // (threads per CTA, resident CTAs per SM) pairs compiled with matching
  // __launch_bounds__, i.e. register caps of 128, 102, 85 and 64 per thread
  const int bps = h->tuning.blocks_per_sm;
  if (gtab) {
    // (128, 3): 170 registers per thread, no spills -- for small,
    // long-lived sets where one particle's turn latency sets the time
    switch ((block * 100 + bps) * 10 + (warp_sched ? 2 : 1)) {
      case 128031: e = launch_track<128, 3, 1>(a, (int)grid, smem, st); break;
      case 128041: e = launch_track<128, 4, 1>(a, (int)grid, smem, st); break;
      case 128051: e = launch_track<128, 5, 1>(a, (int)grid, smem, st); break;
      case 256021: e = launch_track<256, 2, 1>(a, (int)grid, smem, st); break;
      case 256031: e = launch_track<256, 3, 1>(a, (int)grid, smem, st); break;
      case 128032: e = launch_track<128, 3, 2>(a, (int)grid, smem, st); break;
      case 128042: e = launch_track<128, 4, 2>(a, (int)grid, smem, st); break;
      case 128052: e = launch_track<128, 5, 2>(a, (int)grid, smem, st); break;
      case 256022: e = launch_track<256, 2, 2>(a, (int)grid, smem, st); break;
      case 256032: e = launch_track<256, 3, 2>(a, (int)grid, smem, st); break;
      default:
        return set_err(h, BGT_ETOOLARGE,
                       "element table read from global memory: tuning must be (128: 3,4,5) or (256: 2,3)");
    }
    if (e != cudaSuccess)
      return set_err(h, BGT_ECUDA, std::string("track_kernel launch: ") + cudaGetErrorString(e));
    h->launches++;
    return 0;
  }
  switch (block * 100 + bps) {
    case 6408: e = launch_track<64, 8>(a, (int)grid, smem, st); break;
    case 6410: e = launch_track<64, 10>(a, (int)grid, smem, st); break;
    case 6412: e = launch_track<64, 12>(a, (int)grid, smem, st); break;
    case 6416: e = launch_track<64, 16>(a, (int)grid, smem, st); break;
    case 12804: e = launch_track<128, 4>(a, (int)grid, smem, st); break;
    case 12805: e = launch_track<128, 5>(a, (int)grid, smem, st); break;
    case 12806: e = launch_track<128, 6>(a, (int)grid, smem, st); break;
    case 12808: e = launch_track<128, 8>(a, (int)grid, smem, st); break;
    case 25602: e = launch_track<256, 2>(a, (int)grid, smem, st); break;
    case 25603: e = launch_track<256, 3>(a, (int)grid, smem, st); break;
    case 25604: e = launch_track<256, 4>(a, (int)grid, smem, st); break;
    default:
      return set_err(h, BGT_EINVAL,
                     "tuning (threads_per_block, blocks_per_sm) must be one of (64: 8,10,12,16), "
                     "(128: 4,5,6,8), (256: 2,3,4)");
  }
  if (e != cudaSuccess) return set_err(h, BGT_ECUDA, std::string("track_kernel launch: ") + cudaGetErrorString(e));
  h->launches++;
  return 0;
}

static KArgs base_args(bgt_handle* h) {
  KArgs a{};
  a.tables = h->d_tables;
  a.table_off_dw = h->d_table_off;
  a.table_dw = h->table_dw;
  a.n_rec = h->n_ele;
  a.rec_begin = 0;
  a.rec_end = h->n_ele;
  a.G = h->G;
  a.compact_every = h->tuning.compact_every;
  return a;
}

extern "C" {

int bgt_create(bgt_handle** out, const bgt_element* eles, int32_t n_ele, int32_t n_variants,
               const bgt_species* species, int32_t device) {
  if (!out || !eles || !species || n_ele <= 0 || n_variants <= 0) return BGT_EINVAL;
  *out = nullptr;
  bgt_handle* h = new bgt_handle();
  h->device = device;
  h->n_ele = n_ele;
  h->n_variants = n_variants;
  h->sp = *species;
  double p0c = eles[0].p0c;
  h->G.mc2 = species->mass;
  h->G.mc2sq = species->mass * species->mass;
  h->G.p0c = p0c;
  h->G.mal = species->max_aperture_limit;
  h->G.ap_on = species->aperture_limit_on;
  h->G.charge = species->charge;
  // compile tables
  std::vector<double> all;
  const int32_t seq_dw = n_ele + (n_ele % 2);  // (offset, ix_ele) int32 pairs, padded to 16 bytes
  for (int v = 0; v < n_variants; v++) {
    std::vector<double> tab(seq_dw, 0.0);
    std::unordered_map<std::string, int32_t> pool;  // record bytes -> offset (identical elements share)
    std::unordered_map<std::string, int32_t> qclass;  // quad (length, b1, step) -> memo class
    for (int e = 0; e < n_ele; e++) {
      std::vector<double> rec;
      int rc = host::compile_element(eles[(int64_t)v * n_ele + e], *species, p0c, rec, h->err);
      if (rc) {
        std::string m = h->err;
        delete h;
        // no handle to carry the message: print it once so the caller sees why
        fprintf(stderr, "bgt_create: %s\n", m.c_str());
        return rc;
      }
      RecHdr* rh = reinterpret_cast<RecHdr*>(rec.data());
      rh->ix_ele = 0;  // carried by the sequence instead
      if (rh->kind == K_QUAD) {
        // quad-matrix memo class: same (b1, length, step) -> same quad_mat2_calc
        const double* kb = rec.data() + HDR_DW + ((rh->flags & F_MISALIGN) ? MIS_N : 0) +
                           ((rh->flags & (F_AP_ENTRANCE | F_AP_EXIT)) ? AP_N : 0);
        std::string ck(reinterpret_cast<const char*>(kb), 3 * sizeof(double));  // Q_LEN, Q_B1, Q_STEP
        auto ci = qclass.find(ck);
        if (ci != qclass.end()) {
          rh->aux0 = ci->second;
        } else if ((int)qclass.size() < QMEMO_CLASSES) {
          rh->aux0 = (int32_t)qclass.size();
          qclass.emplace(ck, rh->aux0);
        } else {
          rh->aux0 = -1;
        }
      }
      std::string key(reinterpret_cast<const char*>(rec.data()), rec.size() * sizeof(double));
      auto it = pool.find(key);
      int32_t off;
      if (it != pool.end()) {
        off = it->second;
      } else {
        off = (int32_t)tab.size();
        tab.insert(tab.end(), rec.begin(), rec.end());
        pool.emplace(std::move(key), off);
      }
      int32_t* s = reinterpret_cast<int32_t*>(tab.data()) + 2 * e;
      s[0] = off;
      s[1] = eles[(int64_t)v * n_ele + e].ix_ele;
    }
    h->table_dw = std::max(h->table_dw, (int32_t)tab.size());
    h->h_table_off.push_back((int64_t)all.size());
    all.insert(all.end(), tab.begin(), tab.end());
    while (all.size() % 2) all.push_back(0.0);
  }
  // every table is read as table_dw doubles: pad the tail
  all.resize(h->h_table_off.back() + h->table_dw + 2, 0.0);
  if (h->table_dw % 2) h->table_dw++;
  h->h_tables = all;
  cudaError_t e;
  if ((e = cudaSetDevice(device)) != cudaSuccess ||
      (e = cudaDeviceGetAttribute(&h->num_sms, cudaDevAttrMultiProcessorCount, device)) != cudaSuccess ||
      (e = cudaMalloc(&h->d_tables, all.size() * 8)) != cudaSuccess ||
      (e = cudaMalloc(&h->d_table_off, h->h_table_off.size() * 8)) != cudaSuccess ||
      (e = cudaMalloc(&h->d_scratch, 64)) != cudaSuccess ||
      (e = cudaMemcpy(h->d_tables, all.data(), all.size() * 8, cudaMemcpyHostToDevice)) != cudaSuccess ||
      (e = cudaMemcpy(h->d_table_off, h->h_table_off.data(), h->h_table_off.size() * 8, cudaMemcpyHostToDevice)) !=
          cudaSuccess ||
      (e = cudaMemset(h->d_scratch, 0, 64)) != cudaSuccess) {
    fprintf(stderr, "bgt_create: CUDA error: %s\n", cudaGetErrorString(e));
    bgt_destroy(h);
    return BGT_ECUDA;
  }
  static double cm[BGT_MAXPOLE_DEV + 1][BGT_MAXPOLE_DEV + 1], cm0[BGT_MAXPOLE_DEV + 1][BGT_MAXPOLE_DEV + 1];
  host::c_multi_tables(cm, cm0);
  if ((e = cudaMemcpyToSymbol(c_cm, cm, sizeof(cm))) != cudaSuccess ||
      (e = cudaMemcpyToSymbol(c_cm0, cm0, sizeof(cm0))) != cudaSuccess) {
    fprintf(stderr, "bgt_create: CUDA error: %s\n", cudaGetErrorString(e));
    bgt_destroy(h);
    return BGT_ECUDA;
  }
  *out = h;
  return 0;
}

int bgt_destroy(bgt_handle* h) {
  if (!h) return 0;
  cudaFree(h->d_tables);
  cudaFree(h->d_table_off);

  cudaFree(h->d_scratch);
  cudaFree(h->d_vec6);
  cudaFree(h->d_beta);
  cudaFree(h->d_i32);
  cudaFree(h->d_grp);
  cudaFree(h->d_grp_v);
  delete h;
  return 0;
}

const char* bgt_last_error(const bgt_handle* h) { return h ? h->err.c_str() : "null handle"; }

int bgt_table_info(const bgt_handle* h, int64_t* table_bytes, int32_t* n_records) {
  if (!h) return BGT_EINVAL;
  if (table_bytes) *table_bytes = (int64_t)h->table_dw * 8;
  if (n_records) *n_records = h->n_ele;
  return 0;
}

int bgt_set_tuning(bgt_handle* h, const bgt_tuning* t) {
  if (!h || !t) return BGT_EINVAL;
  bgt_tuning n = *t;
  if (n.threads_per_block == 0) n.threads_per_block = 128;
  if (n.blocks_per_sm == 0) n.blocks_per_sm = 4;
  if (n.threads_per_block != 64 && n.threads_per_block != 128 && n.threads_per_block != 256)
    return set_err(h, BGT_EINVAL, "threads_per_block must be 64, 128 or 256");
  if (n.compact_every < 0 || n.turns_per_launch < 0) return set_err(h, BGT_EINVAL, "negative tuning value");
  if (n.table_mode < 0 || n.table_mode > 3) return set_err(h, BGT_EINVAL, "table_mode must be 0, 1, 2 or 3");
  h->tuning = n;
  return 0;
}

int bgt_get_tuning(const bgt_handle* h, bgt_tuning* t) {
  if (!h || !t) return BGT_EINVAL;
  *t = h->tuning;
  return 0;
}

int64_t bgt_kernel_launch_count(const bgt_handle* h) { return h ? h->launches : -1; }

// Track device-resident particles for turns [turn0, turn0 + n_turns) in
// segments of tuning.turns_per_launch turns (one persistent launch each).
static int track_device_impl(bgt_handle* h, double* d_vec6, int64_t n_stride, double* d_beta, int32_t* d_state,
                             int32_t* d_ixe, int32_t* d_ixt, const int32_t* d_slot, const int32_t* d_tile_var,
                             int64_t n, int64_t n_slots, int32_t turn0, int32_t n_turns, int32_t rec_begin,
                             int32_t rec_end, cudaStream_t st) {
  KArgs a = base_args(h);
  a.vec6 = d_vec6;
  a.n_stride = n_stride;
  a.beta = d_beta;
  a.state = d_state;
  a.ix_ele_lost = d_ixe;
  a.ix_turn_lost = d_ixt;
  a.slot_particle = d_slot;
  a.tile_variant = d_tile_var;
  a.n = n;
  a.n_slots = n_slots;
  a.rec_begin = rec_begin;
  a.rec_end = rec_end;
  int64_t n_tiles = (n_slots + h->tuning.threads_per_block - 1) / h->tuning.threads_per_block;
  int32_t seg = h->tuning.turns_per_launch > 0 ? h->tuning.turns_per_launch : n_turns;
  for (int32_t t = 0; t < n_turns; t += seg) {
    a.turn0 = turn0 + t;
    a.n_turns = std::min(seg, n_turns - t);
    int rc = enqueue_track(h, a, n_tiles, st);
    if (rc) return rc;
  }
  return 0;
}

// Per-variant particle counts of a variant-sorted device array, with a check
// that ids are in range (bad bit 1) and non-decreasing (bad bit 2).
__global__ void variant_count_kernel(const int32_t* var, int64_t n, int32_t n_var, int64_t* first, int64_t* count,
                                     int32_t* bad) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  int32_t v = var[i];
  if (v < 0 || v >= n_var) {
    atomicOr(bad, 1);
    return;
  }
  if (i > 0 && var[i - 1] > v) atomicOr(bad, 2);
  if (i == 0 || var[i - 1] != v) first[v] = i;
  atomicAdd((unsigned long long*)&count[v], 1ull);
}

// slot of particle i: its variant's first slot + its rank inside the variant
__global__ void variant_slot_kernel(const int32_t* var, int64_t n, const int64_t* first, const int64_t* slot0,
                                    int32_t* slot) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  int32_t v = var[i];
  slot[slot0[v] + (i - first[v])] = (int32_t)i;
}

int bgt_track_turns_device(bgt_handle* h, double* d_vec6, double* d_beta, int32_t* d_state, int32_t* d_ix_ele_lost,
                           int32_t* d_ix_turn_lost, const int32_t* d_variant, int64_t n, int32_t turn0,
                           int32_t n_turns, void* stream) {
  if (!h || !d_vec6 || !d_beta || !d_state || !d_ix_ele_lost || n < 0 || n_turns < 0) return BGT_EINVAL;
  if (n == 0 || n_turns == 0) return 0;
  if (n > INT32_MAX) return set_err(h, BGT_EINVAL, "bgt_track_turns_device: n exceeds 2^31 - 1");
  CU(h, cudaSetDevice(h->device));
  cudaStream_t st = (cudaStream_t)stream;
  if (!d_variant || h->n_variants == 1)
    return track_device_impl(h, d_vec6, n, d_beta, d_state, d_ix_ele_lost, d_ix_turn_lost, nullptr, nullptr, n, n,
                             turn0, n_turns, 0, h->n_ele, st);
  // Group by variant into tile-aligned slot ranges.  The variant ids must be
  // sorted (non-decreasing); the per-variant counts are read back once.
  const int32_t nv = h->n_variants;
  const int block = h->tuning.threads_per_block;
  if (!h->d_grp_v) CU(h, cudaMalloc(&h->d_grp_v, ((size_t)3 * nv + 1) * 8));
  int64_t* d_first = h->d_grp_v;
  int64_t* d_count = d_first + nv;
  int64_t* d_slot0 = d_count + nv;
  int32_t* d_bad = (int32_t*)(d_slot0 + nv);
  CU(h, cudaMemsetAsync(d_first, 0, ((size_t)3 * nv + 1) * 8, st));
  variant_count_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(d_variant, n, nv, d_first, d_count, d_bad);
  h->launches++;
  std::vector<int64_t> cnt((size_t)nv + 1);
  CU(h, cudaMemcpyAsync(cnt.data(), d_count, (size_t)nv * 8, cudaMemcpyDeviceToHost, st));
  int32_t bad = 0;
  CU(h, cudaMemcpyAsync(&bad, d_bad, 4, cudaMemcpyDeviceToHost, st));
  CU(h, cudaStreamSynchronize(st));
  if (bad & 1) return set_err(h, BGT_EINVAL, "bgt_track_turns_device: variant id out of range");
  if (bad & 2) return set_err(h, BGT_EINVAL, "bgt_track_turns_device: variant ids must be sorted");
  std::vector<int64_t> slot0(nv);
  std::vector<int32_t> tvar;
  int64_t s = 0;
  for (int32_t v = 0; v < nv; v++) {
    slot0[v] = s;
    int64_t tiles = (cnt[v] + block - 1) / block;
    for (int64_t t = 0; t < tiles; t++) tvar.push_back(v);
    s += tiles * block;
  }
  const int64_t n_slots = s, n_tiles = (int64_t)tvar.size();
  if (n_slots > h->grp_cap_slots || n_tiles > h->grp_cap_tiles) {
    CU(h, cudaStreamSynchronize(st));
    cudaFree(h->d_grp);
    h->d_grp = nullptr;
    h->grp_cap_slots = std::max(n_slots, h->grp_cap_slots);
    h->grp_cap_tiles = std::max(n_tiles, h->grp_cap_tiles);
    CU(h, cudaMalloc(&h->d_grp, (size_t)(h->grp_cap_slots + h->grp_cap_tiles) * 4));
  }
  int32_t* d_slot = h->d_grp;
  int32_t* d_tvar = d_slot + h->grp_cap_slots;
  CU(h, cudaMemcpyAsync(d_slot0, slot0.data(), (size_t)nv * 8, cudaMemcpyHostToDevice, st));
  CU(h, cudaMemcpyAsync(d_tvar, tvar.data(), (size_t)n_tiles * 4, cudaMemcpyHostToDevice, st));
  CU(h, cudaMemsetAsync(d_slot, 0xff, (size_t)n_slots * 4, st));
  variant_slot_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(d_variant, n, d_first, d_slot0, d_slot);
  h->launches++;
  // (copies from pageable host memory return once the data is staged, so
  // slot0 and tvar may go out of scope before the copies complete)
  return track_device_impl(h, d_vec6, n, d_beta, d_state, d_ix_ele_lost, d_ix_turn_lost, d_slot, d_tvar, n, n_slots,
                           turn0, n_turns, 0, h->n_ele, st);
}

// Grow the host-API staging buffers.
static int ensure_staging(bgt_handle* h, int64_t n, int64_t n_slots, int64_t n_tiles) {
  if (n <= h->cap && n_slots <= h->cap_slots && n_tiles <= h->cap_tiles) return 0;
  cudaFree(h->d_vec6);
  cudaFree(h->d_beta);
  cudaFree(h->d_i32);
  h->d_vec6 = nullptr;
  h->d_beta = nullptr;
  h->d_i32 = nullptr;
  h->cap = std::max(n, h->cap);
  h->cap_slots = std::max(n_slots, h->cap_slots);
  h->cap_tiles = std::max(n_tiles, h->cap_tiles);
  CU(h, cudaMalloc(&h->d_vec6, (size_t)h->cap * 6 * 8));
  CU(h, cudaMalloc(&h->d_beta, (size_t)h->cap * 8));
  CU(h, cudaMalloc(&h->d_i32, (size_t)(3 * h->cap + h->cap_slots + h->cap_tiles) * 4));
  return 0;
}

// Host-buffer tracking shared by bgt_track_turns and bgt_track_elements.
static int track_host(bgt_handle* h, double* vec6, double* beta, int32_t* state, int32_t* ixe, int32_t* ixt,
                      const int32_t* variant, int64_t n, int32_t turn0, int32_t n_turns, int32_t rec_begin,
                      int32_t rec_end) {
  if (!h || !vec6 || !beta || !state || !ixe || n < 0) return BGT_EINVAL;
  if (n == 0 || n_turns == 0) return 0;
  CU(h, cudaSetDevice(h->device));
  const int block = h->tuning.threads_per_block;
  // group particles by variant into tile-aligned slot ranges
  std::vector<int32_t> slot_map, tile_var;
  int64_t n_slots = n;
  bool multi = variant && h->n_variants > 1;
  if (multi) {
    std::vector<int64_t> count(h->n_variants, 0);
    for (int64_t i = 0; i < n; i++) {
      if (variant[i] < 0 || variant[i] >= h->n_variants) return set_err(h, BGT_EINVAL, "variant out of range");
      count[variant[i]]++;
    }
    std::vector<int64_t> start(h->n_variants, 0);
    int64_t s = 0;
    for (int v = 0; v < h->n_variants; v++) {
      start[v] = s;
      int64_t tiles = (count[v] + block - 1) / block;
      for (int64_t t = 0; t < tiles; t++) tile_var.push_back(v);
      s += tiles * block;
    }
    n_slots = s;
    slot_map.assign(n_slots, -1);
    std::vector<int64_t> fill = start;
    for (int64_t i = 0; i < n; i++) slot_map[fill[variant[i]]++] = (int32_t)i;
  }
  int64_t n_tiles = (n_slots + block - 1) / block;
  int rc = ensure_staging(h, n, n_slots, n_tiles);
  if (rc) return rc;
  int32_t* d_state = h->d_i32;
  int32_t* d_ixe = d_state + h->cap;
  int32_t* d_ixt = d_ixe + h->cap;
  int32_t* d_slot = d_ixt + h->cap;
  int32_t* d_tvar = d_slot + h->cap_slots;
  CU(h, cudaMemcpy2D(h->d_vec6, h->cap * 8, vec6, n * 8, n * 8, 6, cudaMemcpyHostToDevice));
  CU(h, cudaMemcpy(h->d_beta, beta, n * 8, cudaMemcpyHostToDevice));
  CU(h, cudaMemcpy(d_state, state, n * 4, cudaMemcpyHostToDevice));
  CU(h, cudaMemcpy(d_ixe, ixe, n * 4, cudaMemcpyHostToDevice));
  if (ixt) CU(h, cudaMemcpy(d_ixt, ixt, n * 4, cudaMemcpyHostToDevice));
  if (multi) {
    CU(h, cudaMemcpy(d_slot, slot_map.data(), n_slots * 4, cudaMemcpyHostToDevice));
    CU(h, cudaMemcpy(d_tvar, tile_var.data(), tile_var.size() * 4, cudaMemcpyHostToDevice));
  } else if (variant && h->n_variants == 1) {
    for (int64_t i = 0; i < n; i++)
      if (variant[i] != 0) return set_err(h, BGT_EINVAL, "variant out of range");
  }
  rc = track_device_impl(h, h->d_vec6, h->cap, h->d_beta, d_state, d_ixe, ixt ? d_ixt : nullptr,
                         multi ? d_slot : nullptr, multi ? d_tvar : nullptr, n, n_slots, turn0, n_turns, rec_begin,
                         rec_end, 0);
  if (rc) return rc;
  CU(h, cudaDeviceSynchronize());
  int32_t flag = 0;
  CU(h, cudaMemcpy(&flag, h->d_scratch + 1, 4, cudaMemcpyDeviceToHost));
  if (flag) return set_err(h, BGT_ETIMEOUT, "element-table staging did not complete");
  CU(h, cudaMemcpy2D(vec6, n * 8, h->d_vec6, h->cap * 8, n * 8, 6, cudaMemcpyDeviceToHost));
  CU(h, cudaMemcpy(beta, h->d_beta, n * 8, cudaMemcpyDeviceToHost));
  CU(h, cudaMemcpy(state, d_state, n * 4, cudaMemcpyDeviceToHost));
  CU(h, cudaMemcpy(ixe, d_ixe, n * 4, cudaMemcpyDeviceToHost));
  if (ixt) CU(h, cudaMemcpy(ixt, d_ixt, n * 4, cudaMemcpyDeviceToHost));
  return 0;
}

int bgt_track_turns(bgt_handle* h, double* vec6, double* beta, int32_t* state, int32_t* ix_ele_lost,
                    int32_t* ix_turn_lost, const int32_t* variant, int64_t n, int32_t turn0, int32_t n_turns) {
  if (!h) return BGT_EINVAL;
  return track_host(h, vec6, beta, state, ix_ele_lost, ix_turn_lost, variant, n, turn0, n_turns, 0, h->n_ele);
}

int bgt_track_elements(bgt_handle* h, double* vec6, double* beta, int32_t* state, int32_t* ix_ele_lost,
                       const int32_t* variant, int64_t n, int32_t e_begin, int32_t e_end) {
  if (!h) return BGT_EINVAL;
  if (e_begin < 0 || e_end > h->n_ele || e_begin >= e_end) return set_err(h, BGT_EINVAL, "bad element range");
  return track_host(h, vec6, beta, state, ix_ele_lost, nullptr, variant, n, 0, 1, e_begin, e_end);
}

}  // extern "C"

// ===========================================================================
// Dynamic-aperture polar grid (bmad/modules/dynamic_aperture_mod.f90:27-207,
// 284-398 with the bisection replaced by a fixed grid of radii).

namespace bgt {

struct DAArgs {
  const double* ref;  // [(v*n_delta + d)*6 + c]
  const double* cs;   // [a] = (cos(angle_a), sin(angle_a)), host-evaluated
  int32_t n_var, n_delta, n_angle, n_radius;
  double a0, da, dr, y_scale;
  int32_t block;
  int64_t per_var, slots_per_var;
  double p0c, mc2;
  double* vec6;
  int64_t stride;
  double* beta;
  int32_t* state;
  int32_t* ixe;
  int32_t* ixt;
  int32_t* slot;
};

// particle index p = ((v*n_delta + d)*n_angle + a)*n_radius + r
__global__ void da_init_kernel(DAArgs A, int64_t n) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  int32_t r = (int32_t)(i % A.n_radius);
  int64_t q = i / A.n_radius;
  int32_t a = (int32_t)(q % A.n_angle);
  q /= A.n_angle;
  int32_t d = (int32_t)(q % A.n_delta);
  int32_t v = (int32_t)(q / A.n_delta);
  const double* ref = A.ref + ((int64_t)v * A.n_delta + d) * 6;
  double rad = A.dr * r;
  double x1 = A.cs[2 * a] * rad;
  double y1 = A.cs[2 * a + 1] * rad * A.y_scale;
  A.vec6[0 * A.stride + i] = ref[0] + x1;
  A.vec6[1 * A.stride + i] = ref[1];
  A.vec6[2 * A.stride + i] = ref[2] + y1;
  A.vec6[3 * A.stride + i] = ref[3];
  A.vec6[4 * A.stride + i] = ref[4];
  A.vec6[5 * A.stride + i] = ref[5];
  double pc = (1 + ref[5]) * A.p0c;
  A.beta[i] = pc / sqrt(pc * pc + A.mc2 * A.mc2);
  A.state[i] = ALIVE;
  A.ixe[i] = -1;
  A.ixt[i] = -1;
  // slot of this particle: variant-major, padded per variant; inside a
  // variant radius-major ((d * n_radius + r) * n_angle + a), so that a warp
  // (and a CTA) holds probes of one or few radii across the angles -- they
  // are lost at similar turns, and warps of a CTA finish together instead of
  // idling at the end-of-tile barrier.  Results do not depend on the slot.
  int64_t within = ((int64_t)d * A.n_radius + r) * A.n_angle + a;
  A.slot[(int64_t)v * A.slots_per_var + within] = (int32_t)i;
}

__global__ void da_tile_var_kernel(int32_t* tvar, int64_t tiles_per_var, int64_t n_tiles) {
  int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t < n_tiles) tvar[t] = (int32_t)(t / tiles_per_var);
}

__global__ void da_reduce_kernel(const int32_t* state, const int32_t* ixt, int64_t n_rays, int32_t n_radius,
                                 double dr, int32_t turn0, int32_t n_turns, double* da_radius,
                                 int32_t* survive) {
  int64_t ray = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (ray >= n_rays) return;
  int64_t base = ray * n_radius;
  int32_t first_lost = n_radius;
  for (int32_t r = 0; r < n_radius; r++) {
    int32_t s = state[base + r];
    if (s != ALIVE && first_lost == n_radius) first_lost = r;
    if (survive) survive[base + r] = (s == ALIVE) ? n_turns : (ixt[base + r] - turn0);
  }
  int32_t last_ok = first_lost - 1;
  da_radius[ray] = last_ok < 0 ? 0.0 : dr * last_ok;
}

// FP64 fused multiply-add throughput probe: 8 independent chains per thread.
__global__ void fp64_peak_kernel(double* out, int iters, double a, double b) {
  double x0 = threadIdx.x * 1e-9, x1 = x0 + 1, x2 = x0 + 2, x3 = x0 + 3, x4 = x0 + 4, x5 = x0 + 5, x6 = x0 + 6,
         x7 = x0 + 7;
  for (int i = 0; i < iters; i++) {
    x0 = fma(x0, a, b);
    x1 = fma(x1, a, b);
    x2 = fma(x2, a, b);
    x3 = fma(x3, a, b);
    x4 = fma(x4, a, b);
    x5 = fma(x5, a, b);
    x6 = fma(x6, a, b);
    x7 = fma(x7, a, b);
  }
  double s = x0 + x1 + x2 + x3 + x4 + x5 + x6 + x7;
  if (s == 12345.678) out[0] = s;  // keeps the chains live
}

}  // namespace bgt

extern "C" {

int bgt_da_scan_grid(bgt_handle* h, const double* ref_orbit, int32_t n_variants_used, const double* deltas,
                     int32_t n_delta, int32_t n_angle, double angle_min, double angle_max, int32_t n_radius,
                     double r_max, double y_scale, int32_t n_turns, double* da_radius, int32_t* survive_turns) {
  (void)deltas;
  if (!h || !ref_orbit || !da_radius || n_variants_used <= 0 || n_variants_used > h->n_variants || n_delta <= 0 ||
      n_angle <= 0 || n_radius <= 1 || n_turns <= 0)
    return BGT_EINVAL;
  CU(h, cudaSetDevice(h->device));
  const int block = h->tuning.threads_per_block;
  DAArgs A{};
  A.n_var = n_variants_used;
  A.n_delta = n_delta;
  A.n_angle = n_angle;
  A.n_radius = n_radius;
  A.a0 = angle_min;
  A.da = n_angle > 1 ? (angle_max - angle_min) / (n_angle - 1) : 0.0;
  A.dr = r_max / (n_radius - 1);
  A.y_scale = y_scale;
  A.per_var = (int64_t)n_delta * n_angle * n_radius;
  int64_t tiles_per_var = (A.per_var + block - 1) / block;
  A.slots_per_var = tiles_per_var * block;
  int64_t n = A.per_var * n_variants_used;
  int64_t n_slots = A.slots_per_var * n_variants_used;
  int64_t n_tiles = tiles_per_var * n_variants_used;
  A.p0c = h->G.p0c;
  A.mc2 = h->G.mc2;
  int rc = ensure_staging(h, n, n_slots, n_tiles);
  if (rc) return rc;
  int32_t* d_state = h->d_i32;
  int32_t* d_ixe = d_state + h->cap;
  int32_t* d_ixt = d_ixe + h->cap;
  int32_t* d_slot = d_ixt + h->cap;
  int32_t* d_tvar = d_slot + h->cap_slots;
  double* d_ref = nullptr;
  double* d_da = nullptr;
  int32_t* d_surv = nullptr;
  int64_t n_rays = (int64_t)n_variants_used * n_delta * n_angle;
  // ray directions: angle_j = j * delta_angle + min_angle
  // (dynamic_aperture_mod.f90:88-95), cos/sin by the host C library
  std::vector<double> cs(2 * (size_t)n_angle);
  for (int j = 0; j < n_angle; j++) {
    double ang = (n_angle == 1) ? (angle_min + angle_max) / 2 : j * A.da + angle_min;
    cs[2 * j] = cos(ang);
    cs[2 * j + 1] = sin(ang);
  }
  double* d_cs = nullptr;
  CU(h, cudaMalloc(&d_cs, cs.size() * 8));
  CU(h, cudaMemcpy(d_cs, cs.data(), cs.size() * 8, cudaMemcpyHostToDevice));
  A.cs = d_cs;
  CU(h, cudaMalloc(&d_ref, (size_t)n_variants_used * n_delta * 6 * 8));
  CU(h, cudaMalloc(&d_da, (size_t)n_rays * 8));
  if (survive_turns) CU(h, cudaMalloc(&d_surv, (size_t)n * 4));
  CU(h, cudaMemcpy(d_ref, ref_orbit, (size_t)n_variants_used * n_delta * 6 * 8, cudaMemcpyHostToDevice));
  CU(h, cudaMemset(d_slot, 0xff, (size_t)n_slots * 4));
  A.ref = d_ref;
  A.vec6 = h->d_vec6;
  A.stride = h->cap;
  A.beta = h->d_beta;
  A.state = d_state;
  A.ixe = d_ixe;
  A.ixt = d_ixt;
  A.slot = d_slot;
  A.block = block;
  da_init_kernel<<<(unsigned)((n + 255) / 256), 256>>>(A, n);
  da_tile_var_kernel<<<(unsigned)((n_tiles + 255) / 256), 256>>>(d_tvar, tiles_per_var, n_tiles);
  h->launches += 2;
  rc = track_device_impl(h, h->d_vec6, h->cap, h->d_beta, d_state, d_ixe, d_ixt, d_slot, d_tvar, n, n_slots, 0,
                         n_turns, 0, h->n_ele, 0);
  if (rc) {
    cudaFree(d_ref);
    cudaFree(d_da);
    cudaFree(d_surv);
    cudaFree(d_cs);
    return rc;
  }
  da_reduce_kernel<<<(unsigned)((n_rays + 127) / 128), 128>>>(d_state, d_ixt, n_rays, n_radius, A.dr, 0, n_turns,
                                                              d_da, d_surv);
  h->launches++;
  CU(h, cudaDeviceSynchronize());
  int32_t flag = 0;
  CU(h, cudaMemcpy(&flag, h->d_scratch + 1, 4, cudaMemcpyDeviceToHost));
  CU(h, cudaMemcpy(da_radius, d_da, (size_t)n_rays * 8, cudaMemcpyDeviceToHost));
  if (survive_turns) CU(h, cudaMemcpy(survive_turns, d_surv, (size_t)n * 4, cudaMemcpyDeviceToHost));
  cudaFree(d_ref);
  cudaFree(d_da);
  cudaFree(d_surv);
  cudaFree(d_cs);
  if (flag) return set_err(h, BGT_ETIMEOUT, "element-table staging did not complete");
  return 0;
}

// Measured FP64 FMA throughput of the current device in TFLOP/s (2 flops per
// FMA).  Measurement helper for roofline reporting; no reference counterpart.
int bgt_fp64_peak_tflops(int32_t device, double* tflops) {
  if (!tflops) return BGT_EINVAL;
  cudaError_t e = cudaSetDevice(device);
  if (e != cudaSuccess) return BGT_ECUDA;
  int sms = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  double* d_out = nullptr;
  if (cudaMalloc(&d_out, 8) != cudaSuccess) return BGT_ECUDA;
  const int threads = 256, blocks = sms * 8, iters = 1 << 14;
  cudaEvent_t t0, t1;
  cudaEventCreate(&t0);
  cudaEventCreate(&t1);
  fp64_peak_kernel<<<blocks, threads>>>(d_out, iters, 0.999999, 1e-9);
  cudaEventRecord(t0);
  const int reps = 5;
  for (int r = 0; r < reps; r++) fp64_peak_kernel<<<blocks, threads>>>(d_out, iters, 0.999999, 1e-9);
  cudaEventRecord(t1);
  cudaEventSynchronize(t1);
  float ms = 0;
  cudaEventElapsedTime(&ms, t0, t1);
  cudaEventDestroy(t0);
  cudaEventDestroy(t1);
  cudaFree(d_out);
  if (cudaGetLastError() != cudaSuccess) return BGT_ECUDA;
  double flops = 2.0 * 8.0 * iters * (double)threads * blocks * reps;
  *tflops = flops / (ms * 1e-3) / 1e12;
  return 0;
}

}  // extern "C"

// ===========================================================================
// Allocation-free tracking entry point.
//
// For callers that cannot allocate device memory from inside this library:
// hosts whose framework owns the device memory (a caching allocator that has
// reserved the GPU, so a cudaMalloc here could fail or fragment its pool) and
// loops that must not allocate per call.  The element table, the tile
// counter and the error flag live in one file-scope device array instead of
// handle-owned cudaMalloc buffers; the caller passes the particle arrays.
//
// The array holds BGT_NOALLOC_SCRATCH_BYTES on every GPU that loads this
// library, until the process exits.  Tables larger than that are rejected.
// Every call uses the same array and leaves its contents behind: calls that
// overlap on the GPU (different streams, or threads) race and must be
// serialised by the caller.  The first call on a device resolves the array's
// address (cudaGetSymbolAddress) and uploads the multipole coefficient
// tables; make that first call before any stream capture.

#define BGT_NOALLOC_SCRATCH_BYTES (256 * 1024)

namespace bgt {

// [0..15]: tile counter (int32), error flag (int32); table from byte 256 on
static __device__ __align__(256) unsigned char g_noalloc_scratch[BGT_NOALLOC_SCRATCH_BYTES];

namespace {
constexpr int kNoallocMaxDevices = 64;
unsigned char* g_noalloc_ptr[kNoallocMaxDevices] = {};
}  // namespace

}  // namespace bgt

extern "C" int bgt_track_turns_device_noalloc(const bgt_element* eles, int32_t n_ele, const bgt_species* species,
                                              double* d_vec6, double* d_beta, int32_t* d_state,
                                              int32_t* d_ix_ele_lost, int32_t* d_ix_turn_lost, int64_t n,
                                              int32_t turn0, int32_t n_turns, const bgt_tuning* tuning,
                                              int32_t device, void* stream, char* err, int32_t err_len) {
  auto fail = [&](int code, const std::string& msg) {
    if (err && err_len > 0) {
      snprintf(err, (size_t)err_len, "%s", msg.c_str());
    }
    return code;
  };
  if (!eles || !species || n_ele <= 0 || !d_vec6 || !d_beta || !d_state || !d_ix_ele_lost || n < 0 ||
      n_turns < 0 || device < 0 || device >= bgt::kNoallocMaxDevices)
    return fail(BGT_EINVAL, "bgt_track_turns_device_noalloc: invalid argument");
  if (n == 0 || n_turns == 0) return 0;
  cudaError_t ce = cudaSetDevice(device);
  if (ce != cudaSuccess) return fail(BGT_ECUDA, std::string("cudaSetDevice: ") + cudaGetErrorString(ce));

  // one-time set-up on this device (this device current)
  if (!bgt::g_noalloc_ptr[device]) {
    void* p = nullptr;
    ce = cudaGetSymbolAddress(&p, bgt::g_noalloc_scratch);
    if (ce != cudaSuccess) return fail(BGT_ECUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(ce));
    static double cm[BGT_MAXPOLE_DEV + 1][BGT_MAXPOLE_DEV + 1], cm0[BGT_MAXPOLE_DEV + 1][BGT_MAXPOLE_DEV + 1];
    bgt::host::c_multi_tables(cm, cm0);
    if ((ce = cudaMemcpyToSymbol(bgt::c_cm, cm, sizeof(cm))) != cudaSuccess ||
        (ce = cudaMemcpyToSymbol(bgt::c_cm0, cm0, sizeof(cm0))) != cudaSuccess)
      return fail(BGT_ECUDA, std::string("coefficient upload: ") + cudaGetErrorString(ce));
    bgt::g_noalloc_ptr[device] = static_cast<unsigned char*>(p);
  }
  unsigned char* base = bgt::g_noalloc_ptr[device];

  // compile the table on the host (same records as bgt_create, one variant)
  std::vector<double> tab((size_t)(n_ele + (n_ele % 2)), 0.0);
  std::unordered_map<std::string, int32_t> pool;
  std::string msg;
  const double p0c = eles[0].p0c;
  for (int e = 0; e < n_ele; e++) {
    std::vector<double> rec;
    int rc = bgt::host::compile_element(eles[e], *species, p0c, rec, msg);
    if (rc) return fail(rc, msg);
    bgt::RecHdr* rh = reinterpret_cast<bgt::RecHdr*>(rec.data());
    rh->ix_ele = 0;
    if (rh->kind == bgt::K_QUAD) rh->aux0 = -1;  // no quad memo classes on this path
    std::string key(reinterpret_cast<const char*>(rec.data()), rec.size() * sizeof(double));
    auto it = pool.find(key);
    int32_t off;
    if (it != pool.end()) {
      off = it->second;
    } else {
      off = (int32_t)tab.size();
      tab.insert(tab.end(), rec.begin(), rec.end());
      pool.emplace(std::move(key), off);
    }
    int32_t* s = reinterpret_cast<int32_t*>(tab.data()) + 2 * e;
    s[0] = off;
    s[1] = eles[e].ix_ele;
  }
  if (tab.size() % 2) tab.push_back(0.0);
  const size_t table_bytes = tab.size() * sizeof(double);
  if (256 + table_bytes > BGT_NOALLOC_SCRATCH_BYTES)
    return fail(BGT_ETOOLARGE, "bgt_track_turns_device_noalloc: element table needs " +
                                   std::to_string(table_bytes) + " bytes, the scratch array holds " +
                                   std::to_string(BGT_NOALLOC_SCRATCH_BYTES - 256));
  cudaStream_t st = (cudaStream_t)stream;
  int32_t* d_counter = reinterpret_cast<int32_t*>(base);
  double* d_table = reinterpret_cast<double*>(base + 256);
  // table offset 0 for the single variant, kept in the scratch header
  int64_t* d_table_off = reinterpret_cast<int64_t*>(base + 16);
  const int64_t zero_off = 0;
  if ((ce = cudaMemcpyAsync(d_table, tab.data(), table_bytes, cudaMemcpyHostToDevice, st)) != cudaSuccess ||
      (ce = cudaMemcpyAsync(d_table_off, &zero_off, sizeof(zero_off), cudaMemcpyHostToDevice, st)) != cudaSuccess)
    return fail(BGT_ECUDA, std::string("table upload: ") + cudaGetErrorString(ce));

  bgt_tuning t = tuning ? *tuning : bgt_tuning{128, 4, 0, 0};
  if (t.threads_per_block == 0) t.threads_per_block = 128;
  if (t.blocks_per_sm == 0) t.blocks_per_sm = 4;
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);

  bgt::KArgs a{};
  a.vec6 = d_vec6;
  a.beta = d_beta;
  a.state = d_state;
  a.ix_ele_lost = d_ix_ele_lost;
  a.ix_turn_lost = d_ix_turn_lost;
  a.n = n;
  a.n_stride = n;
  a.n_slots = n;
  a.tables = d_table;
  a.table_off_dw = d_table_off;
  a.table_dw = (int32_t)tab.size();
  a.rec_begin = 0;
  a.rec_end = n_ele;
  a.n_rec = n_ele;
  a.compact_every = t.compact_every;
  a.tile_counter = d_counter;
  a.error_flag = d_counter + 1;
  a.G.mc2 = species->mass;
  a.G.mc2sq = species->mass * species->mass;
  a.G.p0c = p0c;
  a.G.mal = species->max_aperture_limit;
  a.G.ap_on = species->aperture_limit_on;
  a.G.charge = species->charge;
  const int block = t.threads_per_block;
  size_t smem = (size_t)a.table_dw * 8 + (t.compact_every > 0 ? (size_t)9 * block * 8 : 0) +
                (size_t)bgt::QMEMO_CLASSES * 13 * block * 8;
  if (smem > 200 * 1024) return fail(BGT_ETOOLARGE, "element table does not fit in shared memory");
  const int64_t n_tiles = (n + block - 1) / block;
  int64_t grid = std::min<int64_t>((int64_t)sms * t.blocks_per_sm, n_tiles);
  if (grid < 1) grid = 1;
  // the counter and error flag must start at zero for every launch
  if ((ce = cudaMemsetAsync(d_counter, 0, 2 * sizeof(int32_t), st)) != cudaSuccess)
    return fail(BGT_ECUDA, std::string("scratch clear: ") + cudaGetErrorString(ce));
  const int32_t seg = t.turns_per_launch > 0 ? t.turns_per_launch : n_turns;
  for (int32_t k = 0; k < n_turns; k += seg) {
    a.turn0 = turn0 + k;
    a.n_turns = std::min(seg, n_turns - k);
    if (k > 0 && (ce = cudaMemsetAsync(d_counter, 0, sizeof(int32_t), st)) != cudaSuccess)
      return fail(BGT_ECUDA, std::string("scratch clear: ") + cudaGetErrorString(ce));
    switch (block * 100 + t.blocks_per_sm) {
      case 12804: ce = launch_track<128, 4>(a, (int)grid, smem, st); break;
      case 25602: ce = launch_track<256, 2>(a, (int)grid, smem, st); break;
      default:
        return fail(BGT_EINVAL, "bgt_track_turns_device_noalloc: tuning must be (128, 4) or (256, 2)");
    }
    if (ce != cudaSuccess) return fail(BGT_ECUDA, std::string("track_kernel launch: ") + cudaGetErrorString(ce));
  }
  return 0;
}
