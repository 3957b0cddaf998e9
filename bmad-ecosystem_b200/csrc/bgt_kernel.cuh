// bgt_kernel.cuh -- the persistent FP64 tracking kernel (device code) and
// its launcher, shared by bgt_track.cu (host side, C ABI) and
// bgt_track_kernels.cu (explicit instantiations, compiled in groups).
//
// Launch model: one thread per particle, the particle's phase-space vector in
// registers for whole turns.  A CTA owns a tile of particles ("slots") of one
// lattice variant; it stages that variant's element table into shared memory
// with one bulk TMA copy (cp.async.bulk into its own shared memory) completed on an
// mbarrier, then walks turns x records reading the table by broadcast.  The
// grid is persistent (a multiple of the SM count); CTAs pull tiles from an
// atomic counter so uneven survival balances across SMs.  Every few turns a
// CTA compacts its surviving particles onto the lowest lanes (warp ballot +
// block prefix sum through shared memory) so dead lanes stop costing issue
// slots; fully dead warps skip the element loop.
//
// Everything up to track1_rec is per-particle arithmetic with no CUDA
// construct beyond the __device__ qualifiers; a plain C++ compiler that
// defines those away compiles it for the host (the tests run the element
// maps that way).  The kernel and its launcher need nvcc.
#pragma once

#ifdef __CUDACC__
#include <cuda_runtime.h>

#include <atomic>
#endif
#include <math.h>
#include <stdint.h>

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

template <bool RARE>
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
    if (RARE && (fl & F_BEND_MIS)) {
      q += BM_N;  // the bend geometry follows the block
      if (fl & F_AP_OFFSET) q += BMA_N;  // and its aperture frames
    }
  }
  if (fl & (F_AP_ENTRANCE | F_AP_EXIT)) {
    R.ap = q;
    q += AP_N;
    if (RARE && (fl & F_AP_MOMENTUM)) q += APM_N;  // collimator momentum limits follow
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
template <bool RARE>
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
  const double* soft = hard + ((fl & F_HARD_EDGE) ? 1 : 0);
  const qp::Q t0 = time_of(p);  // start_orb = orbit (track_a_quadrupole.f90:40)
  const double z0 = p.z;
  if (fl & F_MISALIGN) offset_set(p, R.mis, fl, G, m, true);
  if (RARE && (fl & F_FRINGE_INFO)) {
    // apply_element_edge_kick.f90:160-176, first edge: magnetic (hard, then
    // soft), then electric
    if (fl & F_EDGE_IN) {
      if (fl & F_HARD_EDGE) hard_multipole_edge_kick<1>(p, hard[0], true);
      if (fl & F_SOFT_EDGE) soft_quad_edge_kick(p, soft, true);
      if (fl & F_ELEC_EDGE) electric_longitudinal_fringe(p, ae, be, ixe, 1.0, G);
    }
    if (p.state != ALIVE) return;
  }
  if (ix > -1) ab_multipole_kicks(p, an, bn, ix, q[Q_RHALF]);
  if (RARE && ixe > -1) ab_multipole_kicks_elec(p, ae, be, ixe, q[Q_STEP] / 2, G);
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
    if (RARE && ixe > -1) ab_multipole_kicks_elec(p, ae, be, ixe, (i == n_step) ? q[Q_STEP] / 2 : q[Q_STEP], G);
  }
  if (RARE && (fl & F_FRINGE_INFO)) {
    // second edge: electric, then magnetic (soft, then hard)
    if (fl & F_EDGE_OUT) {
      if (fl & F_ELEC_EDGE) electric_longitudinal_fringe(p, ae, be, ixe, -1.0, G);
      if (fl & F_SOFT_EDGE) soft_quad_edge_kick(p, soft, false);
      if (fl & F_HARD_EDGE) hard_multipole_edge_kick<1>(p, hard[0], false);
    }
    if (p.state != ALIVE) return;
  }
  if (fl & F_MISALIGN) offset_unset(p, R.mis, fl, G, m, true);
  element_exit_time(p, t0, z0, q[Q_DTREF], G);
}

// bmad/low_level/track_a_thick_multipole.f90:18-134
template <bool RARE>
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
  const qp::Q t0 = time_of(p);  // start_orb = orbit (track_a_thick_multipole.f90:41)
  const double z0 = p.z;
  if (fl & F_MISALIGN) offset_set(p, R.mis, fl, G, m, true);
  if (RARE && (fl & F_FRINGE_INFO)) {
    if (fl & F_EDGE_IN) {
      if (fl & F_HARD_EDGE) hard_multipole_edge_kick<2>(p, hard[0], true);
      if (fl & F_ELEC_EDGE) electric_longitudinal_fringe(p, ae, be, ixe, 1.0, G);
    }
    if (p.state != ALIVE) return;
  }
  if (ix > -1) ab_multipole_kicks(p, an, bn, ix, q[TM_RHALF]);
  if (RARE && ixe > -1) ab_multipole_kicks_elec(p, ae, be, ixe, q[TM_STEP] / 2, G);
  for (int i = 1; i <= n_step; i++) {
    track_a_drift<true>(p, q[TM_STEP], G, m);
    if (ix > -1) ab_multipole_kicks(p, an, bn, ix, (i == n_step) ? q[TM_RHALF] : q[TM_RSTEP]);
    if (RARE && ixe > -1) ab_multipole_kicks_elec(p, ae, be, ixe, (i == n_step) ? q[TM_STEP] / 2 : q[TM_STEP], G);
  }
  if (RARE && (fl & F_FRINGE_INFO)) {
    if (fl & F_EDGE_OUT) {
      if (fl & F_ELEC_EDGE) electric_longitudinal_fringe(p, ae, be, ixe, -1.0, G);
      if (fl & F_HARD_EDGE) hard_multipole_edge_kick<2>(p, hard[0], false);
    }
    if (p.state != ALIVE) return;
  }
  if (fl & F_MISALIGN) offset_unset(p, R.mis, fl, G, m, true);
  element_exit_time(p, t0, z0, q[TM_DTREF], G);
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
// rf_coupler_kick, bmad/low_level/rf_coupler_kick.f90:20-104 (tracking part)
// for an rfcavity: ph = pi/2 - phase + twopi * coupler_phase, the transverse
// kick dp cos(ph) / p0c and the energy change (dp_x x + dp_y y) f2.
__device__ __forceinline__ void rf_coupler_kick(Part& p, const double* q, double phase, const Glob& G) {
  double ph = phase;
  ph = PI_D / 2 - ph;
  ph = ph + q[RF_CPL_PH];
  const double dp_x = q[RF_CPL_DPX], dp_y = q[RF_CPL_DPY];
  const double c = cr::cos(ph);
  p.px = p.px + 1 * dp_x * c / G.p0c;
  p.py = p.py + 1 * dp_y * c / G.p0c;
  const double f2 = 1 * cr::sin(ph) * TWOPI_D * q[RF_FREQ] / C_LIGHT;
  const double dE = (dp_x * p.x + dp_y * p.y) * f2;
  apply_energy_kick(p, dE, G);
}

template <bool RARE>
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
  double phase0;
  if (RARE && G.abs_time) {
    // particle_rf_time, absolute time (particle_rf_time.f90:74-76): t less
    // the cavity's ref_time_start, folded by modulo2 and multiplied out in
    // real(qp) (:116-118, track_a_rfcavity.f90:78-80) with the binary128
    // arithmetic of bgt_qp.cuh, then rounded to real(rp); no phi0_multipass
    // (:81)
    qp::Q time = time_of(p);
    if (G.abs_ref_shift) time = qp::sub(time, qp::from_double(q[RF_TSTART]));
    if (f != 0) {
      qp::Q amp;
      memcpy(&amp, q + RF_AMPQ, 16);
      time = qp::modulo2(time, amp);
    }
    const qp::Q ph = qp::mul(qp::from_double(TWOPI_D),
                             qp::sub(qp::from_double(q[RF_PHI0]),
                                     qp::mul(qp::sub(time, qp::from_double(0.0)), qp::from_double(f))));
    phase0 = qp::to_double(ph);
  } else {
    // particle_rf_time, relative time: time = -z / (beta * c_light)
    double time = -p.z / (p.beta * C_LIGHT);
    DD t = {time, 0.0};
    if (f != 0) t = dd_modulo2(time, DD{q[RF_HALF_AMP_HI], q[RF_HALF_AMP_LO]});
    DD tf = dd_mul_d(t, f);
    DD u = dd_add({q[RF_PHI0], 0.0}, dd_neg(tf));
    DD v = dd_mul_d(u, TWOPI_D);
    phase0 = v.hi + v.lo;
    phase0 = phase0 + q[RF_PHI0_MP];
  }
  // modulo2(phase0, pi) in double
  double per = 2 * PI_D;
  double mod = fmod(phase0, per);
  if (mod != 0 && ((mod < 0) != (per < 0))) mod += per;
  if (mod >= PI_D) mod = mod - per;
  double phase = mod;
  if (RARE && (fl & F_COUPLER_IN)) rf_coupler_kick(p, q, phase, G);
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
  if (RARE && (fl & F_COUPLER_OUT)) rf_coupler_kick(p, q, phase, G);
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

// apply_multipole_kicks, electric part (track_a_bend.f90:379-385 field,
// :421-438 kick): the field of elec_multipole_field (bmad/code/
// elec_multipole_field.f90:20-65) summed over the orders, then the kick that
// changes px, py, pz, beta and z.  Called after the magnetic kick, which does
// not move x and y, so the field is the one the reference evaluates first.
__device__ __forceinline__ void bend_elec_kicks(Part& p, const double* ae, const double* be, int ixe, double coef,
                                                double step_len, double g, const Glob& G) {
  double E0 = 0, E1 = 0;
  const double x = p.x, y = p.y;
  for (int n = 0; n <= ixe; n++) {
    const double a = ae[n], b = be[n];
    if (a == 0 && b == 0) continue;
    double Ex = 0, Ey = 0;
    for (int mm = 0; mm <= n; mm += 2) {
      const double f = c_cm[n][mm] * mexp_d(x, n - mm) * mexp_d(y, mm);
      Ex = Ex - b * f;
      Ey = Ey - a * f;
    }
    for (int mm = 1; mm <= n; mm += 2) {
      const double f = c_cm[n][mm] * mexp_d(x, n - mm) * mexp_d(y, mm);
      Ex = Ex + a * f;
      Ey = Ey - b * f;
    }
    E0 = E0 + Ex;
    E1 = E1 + Ey;
  }
  const double px0 = p.px, py0 = p.py, pz0 = p.pz, z0 = p.z, beta0 = p.beta;
  const double rel_p0 = 1 + pz0;
  const double ps2 = rel_p0 * rel_p0 - px0 * px0 - py0 * py0;
  const double ps = sqrt(ps2) / rel_p0;
  const double f_coef = step_len * coef * (1 + g * x) * (double)G.charge / (ps * beta0 * G.p0c);
  const double Kx = f_coef * E0;
  const double Ky = f_coef * E1;
  const double alpha = (Kx * (2 * px0 + Kx) + Ky * (2 * py0 + Ky)) / (rel_p0 * rel_p0);
  p.px = px0 + Kx;
  p.py = py0 + Ky;
  p.pz = pz0 + rel_p0 * sqrt_one(alpha);
  p.beta = (1 + p.pz) / sqrt(ps2 + p.px * p.px + p.py * p.py + sq(G.mc2 / G.p0c));
  p.z = z0 * p.beta / beta0;
}

// offset_particle for a misaligned bend (offset_particle.f90:208-235 set,
// :393-425 unset, drift to the edge): (x, y, 0) through the BM block's
// affine steps, the momentum through their product W, then the drift to the
// nominal edge (s = 0 on set, L on unset).
__device__ __forceinline__ void bend_offset(Part& p, const double* bm, bool set, double L_half, const Glob& G,
                                            DriftMemo& m) {
  const int n = (int)bm[set ? BM_NSET : BM_NUNSET];
  const double* ops = bm + (set ? BM_OPS_SET : BM_OPS_UNSET);
  const double* W = bm + (set ? BM_WSET : BM_WUNSET);
  double r0 = p.x, r1 = p.y, r2 = 0.0;
  bend_chain_position(ops, n, r0, r1, r2);
  const double s_pos = r2;
  const double rel_p = 1 + p.pz;
  const double pz = rel_p * rel_p - p.px * p.px - p.py * p.py;
  if (pz <= 0) {
    p.state = LOST_PZ;
  } else {
    double q0, q1, q2;
    mv3_0(W, p.px, p.py, 1 * sqrt(pz), q0, q1, q2);
    p.px = q0;
    p.py = q1;
    p.x = r0;
    p.y = r1;
  }
  const double ds = (set ? 0.0 : 2 * L_half) - s_pos;
  if (fabs(ds) > 1e-14 && p.state == ALIVE) track_a_drift<false>(p, ds, G, m);
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

// bmad/low_level/track_a_bend.f90:18-333.  With RARE: misaligned bends
// (offset_particle's bend geometry) and electric multipoles.
template <bool RARE>
__device__ __forceinline__ void body_bend(Part& p, const Rec& R, const Glob& G, DriftMemo& m) {
  const double* q = R.kb;
  const int32_t fl = R.h->flags;
  const int ix = R.h->ix_mag_max;
  const int n_step = R.h->n_step;
  const double* an = q + B_N;
  const double* bn = an + (ix + 1);
  const int ixe = RARE ? R.h->aux1 : -1;
  const double* ae = an + 2 * (ix + 1);
  const double* be = ae + (ixe + 1);
  const qp::Q t0 = time_of(p);  // start_orb = orbit (track_a_bend.f90:42)
  const double z0 = p.z;
  if (fl & F_MISALIGN) {
    if (RARE && (fl & F_BEND_MIS))
      bend_offset(p, R.mis + MIS_N, true, R.mis[MIS_LHALF], G, m);
    else
      offset_set(p, R.mis, fl, G, m, true);
  }
  const double* ext = ae + ((fl & F_ELEC) ? 2 * (ixe + 1) : 0);  // soft / linear / exact edge constants
  if (fl & F_EDGE_IN) {
    // apply_element_edge_kick.f90:160-201: entering, magnetic (bend_edge_kick,
    // fringe_mod.f90:39-127) then electric
    if (RARE && (fl & F_EXACT_EDGE)) {
      hard_multipole_edge_kick<1>(p, ext[XE_K1], true);
      p = exact_bend_edge<true>(p, ext);
    }
    if (RARE && (fl & F_SOFT_EDGE)) sad_soft_bend_edge(p, ext, true);
    if (!(RARE && (fl & F_NO_HWANG))) hwang_edge<true>(p, q + B_EDGE);
    if (RARE && (fl & F_LINEAR_EDGE)) linear_bend_edge(p, ext, true);
    if (RARE && (fl & F_ELEC_EDGE)) electric_longitudinal_fringe(p, ae, be, ixe, 1.0, G);
  }
  if (orbit_too_large(p, G)) return;
  if (ix > -1) bend_multipole_kicks(p, q, an, bn, ix, 0.5, G);
  if (RARE && ixe > -1) bend_elec_kicks(p, ae, be, ixe, 0.5, q[B_STEP], q[B_G], G);
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
        const double r_pt = 1.0 / pt;  // the four quotients by pt from one reciprocal
        double g_p = div_by(g_tot, pt, r_pt);
        double phi_1 = cr::asin(div_by(px, pt, r_pt));
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
        p.y = y + div_by(py * L_p, pt, r_pt);
        p.z = z + div_by(p.beta * step_len, q[B_BETAREF], q[B_RBETAREF]) - div_by(rel_p * L_p, pt, r_pt);
      }
    }
    if (ix > -1) bend_multipole_kicks(p, q, an, bn, ix, (n == n_step) ? 0.5 : 1.0, G);
    if (RARE && ixe > -1) bend_elec_kicks(p, ae, be, ixe, (n == n_step) ? 0.5 : 1.0, step_len, g, G);
  }
  if (orbit_too_large(p, G)) return;
  if (fl & F_EDGE_OUT) {
    // leaving: electric then magnetic
    if (RARE && (fl & F_ELEC_EDGE)) electric_longitudinal_fringe(p, ae, be, ixe, -1.0, G);
    if (RARE && (fl & F_EXACT_EDGE)) {
      p = exact_bend_edge<false>(p, ext);
      hard_multipole_edge_kick<1>(p, ext[XE_K1], false);
    }
    if (RARE && (fl & F_LINEAR_EDGE)) linear_bend_edge(p, ext, false);
    if (!(RARE && (fl & F_NO_HWANG))) hwang_edge<false>(p, q + B_EDGE + EDGE_N);
    if (RARE && (fl & F_SOFT_EDGE)) sad_soft_bend_edge(p, ext, false);
  }
  if (fl & F_MISALIGN) {
    if (RARE && (fl & F_BEND_MIS))
      bend_offset(p, R.mis + MIS_N, false, R.mis[MIS_LHALF], G, m);
    else
      offset_unset(p, R.mis, fl, G, m, true);
  }
  element_exit_time(p, t0, z0, q[B_DTREF], G);
}

// track1, bmad/code/track1.f90:43-342 for one alive particle and one record:
// entrance aperture, body, orbit_too_large, exit aperture.  Returns the
// particle's state (ALIVE or a lost code).
template <bool RARE>
__device__ __forceinline__ void track1_rec(Part& p, const double* rec, const Glob& G, DriftMemo& m, QMemo qm) {
  Rec R = decode<RARE>(rec);
  const int32_t fl = R.h->flags;
  if ((fl & F_AP_ENTRANCE) && G.ap_on) {
    if (RARE)
      check_aperture(p, R.ap, R.mis, fl, false);
    else
      aperture_limits(p, R.ap, fl, p.x, p.y);
    if (p.state != ALIVE) return;
  }
  switch (R.h->kind) {
    case K_DRIFT:
      track_a_drift<true>(p, R.kb[DR_L], G, m);
      break;
    case K_QUAD:
      body_quad<RARE>(p, R, G, m, qm);
      break;
    case K_BEND:
      body_bend<RARE>(p, R, G, m);
      break;
    case K_THICK_MULT:
      body_thick<RARE>(p, R, G, m);
      break;
    case K_THIN_MULT:
      body_thin(p, R, G, m);
      break;
    case K_RFCAVITY:
      body_rf<RARE>(p, R, G, m);
      break;
    default:
      break;
  }
  if (orbit_too_large(p, G)) return;
  if (p.state != ALIVE) return;
  if ((fl & F_AP_EXIT) && G.ap_on) {
    if (RARE)
      check_aperture(p, R.ap, R.mis, fl, true);
    else
      aperture_limits(p, R.ap, fl, p.x, p.y);
  }
}

#ifdef __CUDACC__
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
__device__ __forceinline__ uint64_t global_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t done;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(done)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return done != 0;
}
// Bounded wait on the mbarrier phase: false once limit_ns nanoseconds of
// %globaltimer have passed without the phase completing.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, uint64_t limit_ns) {
  if (mbar_try_wait(bar, parity)) return true;
  const uint64_t t0 = global_ns();
  while (!mbar_try_wait(bar, parity)) {
    if (global_ns() - t0 > limit_ns) return false;
  }
  return true;
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
  uint64_t* t;                   // particle times, binary128 bits [n][2] (nullptr = not tracked; RARE only)
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
  int32_t* error_flag;            // this call's flag: 1 = a table-staging wait ran out
  int32_t* status;                // the handle's sticky flag (ORed with error_flag; may be null)
  uint64_t wait_ns;               // bound of every wait on the staging mbarrier
  int32_t skip_table_copy;        // test only: arm the mbarrier but issue no copy, so the wait runs out
  Glob G;
};

constexpr int MAX_BLOCK = 256;

// Particle time in and out of global memory, binary128 bits per particle
// (t[2 i], t[2 i + 1]); only the kernel instances that track time touch them.
template <bool RARE>
__device__ __forceinline__ void load_time(Part& p, const uint64_t* t, int64_t i) {
  if (RARE && t) {
    p.t_lo = t[2 * i];
    p.t_hi = t[2 * i + 1];
  }
}
template <bool RARE>
__device__ __forceinline__ void store_time(const Part& p, uint64_t* t, int64_t i) {
  if (RARE && t) {
    t[2 * i] = p.t_lo;
    t[2 * i + 1] = p.t_hi;
  }
}

// TMODE 0: the variant's element table is staged in shared memory.
// TMODE 1: it is read from global memory (L2 / L1) instead -- for tables
//   larger than the shared-memory budget (e.g. every quadrupole and sextupole
//   misaligned and carrying its own multipole errors), or to leave shared
//   memory to more resident CTAs; CTA-wide tiles as in TMODE 0.
// TMODE 2: global-memory tables with every warp scheduled on its own.
// RARE: the element loop also handles the rarely used record features --
//   electric multipoles, the quadrupole/sextupole hard-edge multipole fringe,
//   apertures checked in the element frame, misaligned bends, RF couplers and
//   the bend edges other than Hwang's (F_FRINGE_INFO, F_ELEC, F_AP_OFFSET,
//   F_BEND_MIS, F_COUPLER_*, F_SOFT_EDGE, F_LINEAR_EDGE, F_EXACT_EDGE,
//   F_NO_HWANG).  Lattices without them run the RARE = false kernel, whose
//   element loop carries none of that code (a smaller instruction footprint
//   and register budget for the common case); the host picks the variant
//   from the compiled tables, never the other way round.
template <int BLOCK, int MINB, int TMODE, bool RARE>
__global__ void __launch_bounds__(BLOCK, MINB) track_kernel(KArgs a) {
  constexpr bool GTAB = TMODE != 0;
  extern __shared__ __align__(128) double smem[];
  __shared__ __align__(8) uint64_t bar;
  __shared__ int32_t s_tile;
  __shared__ int32_t s_warp_cnt[BLOCK / 32];
  const double* table = smem;
  // compaction staging area sits after the table
  // [STAGE_ROWS][BLOCK] doubles; rows 7-8 hold int32 ids and loss records,
  // rows 9-10 the particle times (RARE)
  constexpr int STAGE_ROWS = RARE ? 11 : 9;
  double* stage = smem + (GTAB ? 0 : a.table_dw);
  int32_t* stage_i = reinterpret_cast<int32_t*>(stage + 7 * BLOCK);   // [3][BLOCK]
  uint64_t* stage_t = reinterpret_cast<uint64_t*>(stage + 9 * BLOCK);  // [2][BLOCK]
  // quad memo after the (optional) compaction stage
  double* qmemo_base = stage + (a.compact_every > 0 ? STAGE_ROWS * BLOCK : 0);
  const QMemo qmemo{qmemo_base + threadIdx.x, BLOCK};

  // the instances without time tracking (RARE = false) never carry the
  // particle time: track_time = 0 is then a constant and the time arithmetic
  // is compiled out
  Glob G = a.G;
  if (!RARE) G.track_time = 0;
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
      p.t_lo = 0;
      p.t_hi = 0;
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
        load_time<RARE>(p, a.t, pidx);
      }
      DriftMemo memo;
      memo.pz = NAN;
      memo.a = 0;
#pragma unroll
      for (int c = 0; c < QMEMO_CLASSES; c++) qmemo.q[(c * 13 + 12) * qmemo.stride] = NAN;
      if (p.state == ALIVE && orbit_too_large(p, G)) {
        ixe = wseq[a.rec_begin].y;
        ixt = a.turn0;
      }
      for (int t = 0; t < a.n_turns; t++) {
        if (__all_sync(0xffffffffu, p.state != ALIVE)) break;  // whole warp lost
        const int turn = a.turn0 + t;
        for (int r = a.rec_begin; r < a.rec_end; r++) {
          const int2 e = wseq[r];
          if (p.state == ALIVE) {
            track1_rec<RARE>(p, wtable + e.x, G, memo, qmemo);
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
        store_time<RARE>(p, a.t, pidx);
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
        if (!a.skip_table_copy) tma_bulk_g2s(smem, a.tables + a.table_off_dw[variant], table_bytes, &bar);
      }
      const int bad = __syncthreads_or(!mbar_wait(&bar, parity, a.wait_ns));
      if (bad) {
        // Give the copy in flight (if one was issued) one more bounded wait
        // to land before the CTA's shared memory is released, then report.
        if (tid == 0) {
          if (!a.skip_table_copy) mbar_wait(&bar, parity, a.wait_ns);
          atomicExch(a.error_flag, 1);
          if (a.status) atomicOr(a.status, 1);
        }
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
    p.t_lo = 0;
    p.t_hi = 0;
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
      load_time<RARE>(p, a.t, pidx);
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
      if (orbit_too_large(p, G)) {
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
            track1_rec<RARE>(p, table + e.x, G, memo, qmemo);
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
            store_time<RARE>(p, a.t, my_idx);
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
            if (RARE) {
              stage_t[dst] = p.t_lo;
              stage_t[BLOCK + dst] = p.t_hi;
            }
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
            if (RARE) {
              p.t_lo = stage_t[tid];
              p.t_hi = stage_t[BLOCK + tid];
            }
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
      store_time<RARE>(p, a.t, my_idx);
    }
    __syncthreads();
  }
}

}  // namespace bgt

namespace bgt {

// dynamic shared memory per CTA: B200 allows 227 KB per block, less the
// kernel's static shared memory
constexpr size_t SMEM_LIMIT = 224 * 1024;

template <int BLOCK, int MINB, int TMODE, bool RARE>
cudaError_t launch_track(const KArgs& a, int grid, size_t smem, cudaStream_t st) {
  // the attribute is per device; setting it twice (two threads racing on
  // the first launch) is harmless
  static std::atomic<bool> attr_set[64];
  int dev = 0;
  cudaGetDevice(&dev);
  if (!attr_set[dev & 63].load(std::memory_order_acquire)) {
    cudaError_t e = cudaFuncSetAttribute(track_kernel<BLOCK, MINB, TMODE, RARE>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SMEM_LIMIT);
    if (e != cudaSuccess) return e;
    attr_set[dev & 63].store(true, std::memory_order_release);
  }
  track_kernel<BLOCK, MINB, TMODE, RARE><<<grid, BLOCK, smem, st>>>(a);
  return cudaGetLastError();
}

// One compiled (threads per CTA, resident CTAs per SM, table mode, RARE)
// instance of track_kernel and the group it was compiled in.  Every group is
// its own compilation unit with its own copy of the __constant__ multipole
// coefficient tables, which upload_cm fills.
using LaunchFn = cudaError_t (*)(const KArgs&, int grid, size_t smem, cudaStream_t st);
struct TrackKernel {
  int block, minb, tmode;
  bool rare;
  LaunchFn launch;
};
struct TrackKernelGroup {
  const TrackKernel* kernels;
  int n;
  cudaError_t (*upload_cm)(const double* cm, const double* cm0, size_t bytes);
};
constexpr int N_KERNEL_GROUPS = 10;
TrackKernelGroup track_kernel_group(int g);
#endif  // __CUDACC__

}  // namespace bgt
