// bgt_compile.h -- the element-table compiler, host only (no CUDA): turns
// bgt_element descriptions into the table records laid out in bgt_table.h.
// Element constants are evaluated here with the host C library (glibc libm),
// the same library the reference evaluates them with.  bgt_track.cu includes
// it for bgt_create and the no-allocation path; the host build of the element
// maps (tests) includes it with a plain C++ compiler.
#pragma once
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <string>
#include <unordered_map>
#include <vector>

#include "../../include/bgt.h"
#include "bgt_table.h"

namespace bgt {
namespace host {

static const double C_LIGHT_H = 2.99792458e8;  // physical_constants.f90:34

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

// ---- bend geometry of offset_particle (F_BEND_MIS) ----
// offset_particle.f90:208-235 (set) and :393-425 (unset) for a misaligned
// bend, recorded as the affine steps of the BM block.  The matrices and
// vectors are computed by the same steps, in the same floating-point order,
// as the oracle's bend_offset_position; the device applies them to (x, y, 0).
enum { AX_X = 0, AX_Y = 1, AX_Z = 2 };

// sim_utils/special_functions/cos_one.f90:16-26
static double cos_one_h(double angle) {
  double s = sin(angle / 2);
  return -(2 * (s * s));
}

// rotate_vec, sim_utils/math/rotation_3d_mod.f90:737-760
static void rotate_vec_h(double v[3], int axis, double angle) {
  if (angle == 0) return;
  double ca = cos(angle), sa = sin(angle), a, b;
  if (axis == AX_X) {
    a = ca * v[1] - sa * v[2];
    b = sa * v[1] + ca * v[2];
    v[1] = a;
    v[2] = b;
  } else if (axis == AX_Y) {
    a = sa * v[2] + ca * v[0];
    b = ca * v[2] - sa * v[0];
    v[0] = a;
    v[2] = b;
  } else {
    a = ca * v[0] - sa * v[1];
    b = sa * v[0] + ca * v[1];
    v[0] = a;
    v[1] = b;
  }
}

// rotate_mat without right_multiply (mat = Rot . mat),
// rotation_3d_mod.f90:781-835: every column as rotate_vec
static void rotate_mat_h(double m[3][3], int axis, double angle) {
  if (angle == 0) return;
  for (int j = 0; j < 3; j++) {
    double v[3] = {m[0][j], m[1][j], m[2][j]};
    rotate_vec_h(v, axis, angle);
    m[0][j] = v[0];
    m[1][j] = v[1];
    m[2][j] = v[2];
  }
}

// 3x3 matmul with k-ordered sums from zero (gfortran's inline matmul)
static void matmul33_h(const double a[3][3], const double b[3][3], double out[3][3]) {
  double t[3][3];
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) {
      double s = 0;
      for (int k = 0; k < 3; k++) s = s + a[i][k] * b[k][j];
      t[i][j] = s;
    }
  memcpy(out, t, sizeof(t));
}

// floor_angles_to_w_mat (not inverse), floor_angles_to_w_mat.f90:17-57
static void floor_w_h(double theta, double phi, double psi, double w[3][3]) {
  double s_the = sin(theta), c_the = cos(theta);
  double s_phi = sin(phi), c_phi = cos(phi);
  double s_psi = sin(psi), c_psi = cos(psi);
  w[0][0] = c_the * c_psi - s_the * s_phi * s_psi;
  w[0][1] = -c_the * s_psi - s_the * s_phi * c_psi;
  w[0][2] = s_the * c_phi;
  w[1][0] = c_phi * s_psi;
  w[1][1] = c_phi * c_psi;
  w[1][2] = s_phi;
  w[2][0] = -s_the * c_psi - c_the * s_phi * s_psi;
  w[2][1] = s_the * s_psi - c_the * s_phi * c_psi;
  w[2][2] = c_the * c_phi;
}

struct BendChain {
  double* ops;
  int n = 0;
  double W[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
  explicit BendChain(double* o) : ops(o) {}
  void op(int code, const double S[3][3], const double L[3]) {
    double* o = ops + n * BM_OP_N;
    o[0] = code;
    for (int i = 0; i < 3; i++)
      for (int j = 0; j < 3; j++) o[1 + 3 * i + j] = S[i][j];
    for (int i = 0; i < 3; i++) o[10 + i] = L[i];
    if (code >= 1 && code <= 3) matmul33_h(S, W, W);
    n++;
  }
  // bend_shift, bmad/geometry/bend_shift.f90:19-61 (has_tilt: ref_tilt given)
  void shift(double g, double delta_s, bool has_tilt, double ref_tilt) {
    const double I[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
    double angle = delta_s * g;
    if (angle == 0) {
      const double L[3] = {0.0, 0.0, delta_s};
      op(0, I, L);
      return;
    }
    double tlt = has_tilt ? ref_tilt : 0.0;
    double S[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
    if (tlt != 0) {
      rotate_mat_h(S, AX_Z, -ref_tilt);
      rotate_mat_h(S, AX_Y, angle);
      rotate_mat_h(S, AX_Z, ref_tilt);
    } else {
      rotate_mat_h(S, AX_Y, angle);
    }
    double L[3] = {cos_one_h(angle) / g, 0.0 / g, -sin(angle) / g};
    if (has_tilt) rotate_vec_h(L, AX_Z, ref_tilt);
    op(1, S, L);
  }
};

// ele_misalignment_L_S_calc, bmad/geometry/ele_misalignment_L_S_calc.f90:
// 16-50, sbend branch (angle = g L, rho = 1/g)
static void bend_L_S(const bgt_element& e, double L_mis[3], double S[3][3]) {
  L_mis[0] = e.x_offset;
  L_mis[1] = e.y_offset;
  L_mis[2] = e.z_offset;
  if (e.roll != 0) {
    double angle = e.g * e.l;
    double rho = e.g == 0 ? 0.0 : 1 / e.g;
    double Lc[3] = {rho * cos_one_h(angle / 2), rho * 0.0, rho * sin(angle / 2)};
    rotate_vec_h(Lc, AX_Y, angle / 2);
    rotate_vec_h(Lc, AX_Z, e.ref_tilt);
    for (int i = 0; i < 3; i++) L_mis[i] = L_mis[i] - Lc[i];
    rotate_vec_h(Lc, AX_Z, e.roll);
    for (int i = 0; i < 3; i++) L_mis[i] = L_mis[i] + Lc[i];
  }
  floor_w_h(e.x_pitch, e.y_pitch, e.roll, S);
}

// w_mat_for_tilt, bmad/geometry/w_mat_for_tilt.f90:13-40 (not inverse)
static void w_tilt_h(double tilt, double w[3][3]) {
  double c = cos(tilt), s = sin(tilt);
  const double t[3][3] = {{c, -s, 0.0}, {s, c, 0.0}, {0.0, 0.0, 1.0}};
  memcpy(w, t, sizeof(t));
}

// The BM block: the set chain (drift to the entrance edge) and the unset
// chain (drift to the exit edge).
static void bend_mis_block(const bgt_element& e, double* bm) {
  const double g = e.g, rt = e.ref_tilt, L = e.l, L_half = 0.5 * L;
  const double I[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
  const double zero[3] = {0.0, 0.0, 0.0};
  double L_mis[3], ws[3][3], wt[3][3], wm[3][3];
  bend_L_S(e, L_mis, ws);
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) wt[i][j] = ws[j][i];
  {
    BendChain c(bm + BM_OPS_SET);
    const double ds_center = L_half - 0.0;
    c.shift(g, 1 * ds_center, true, rt);
    c.op(2, wt, L_mis);
    if (rt != 0) {
      c.shift(g, -L_half, true, rt);
      w_tilt_h(-rt, wm);
      c.op(3, wm, zero);
      c.shift(g, L_half, false, 0.0);
    }
    c.shift(g, -1 * 1 * L_half, false, 0.0);
    const double add[3] = {0.0, 0.0, (1 - 1 * 1) * L_half};
    c.op(4, I, add);
    bm[BM_NSET] = c.n;
    for (int i = 0; i < 3; i++)
      for (int j = 0; j < 3; j++) bm[BM_WSET + 3 * i + j] = c.W[i][j];
  }
  {
    BendChain c(bm + BM_OPS_UNSET);
    const double ds_center = L_half - L;
    c.shift(g, ds_center, false, 0.0);
    if (rt != 0) {
      c.shift(g, -L_half, false, 0.0);
      w_tilt_h(rt, wm);
      c.op(3, wm, zero);
      c.shift(g, L_half, true, rt);
    }
    c.op(1, ws, L_mis);
    c.shift(g, 1 * 1 * L_half, true, rt);
    const double add[3] = {0.0, 0.0, (1 + 1 * 1) * L_half};
    c.op(4, I, add);
    bm[BM_NUNSET] = c.n;
    for (int i = 0; i < 3; i++)
      for (int j = 0; j < 3; j++) bm[BM_WUNSET + 3 * i + j] = c.W[i][j];
  }
}

// The BMA block: offset_particle's set transform at s_pos = 0 and s_pos = L
// without the drift (offset_particle.f90:208-228), up to the arc shift that
// depends on the particle.
static void bend_ap_block(const bgt_element& e, double* bma) {
  const double g = e.g, rt = e.ref_tilt, L = e.l, L_half = 0.5 * L;
  const double zero[3] = {0.0, 0.0, 0.0};
  double L_mis[3], ws[3][3], wt[3][3], wm[3][3];
  bend_L_S(e, L_mis, ws);
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) wt[i][j] = ws[j][i];
  bma[BMA_G] = g;
  for (int end = 0; end < 2; end++) {
    const double ds_center = L_half - (end == 0 ? 0.0 : L);
    BendChain c(bma + (end == 0 ? BMA_OPS_IN : BMA_OPS_OUT));
    c.shift(g, 1 * ds_center, true, rt);
    c.op(2, wt, L_mis);
    if (rt != 0) {
      c.shift(g, -L_half, true, rt);
      w_tilt_h(-rt, wm);
      c.op(3, wm, zero);
      c.shift(g, L_half, false, 0.0);
    }
    bma[end == 0 ? BMA_NIN : BMA_NOUT] = c.n;
    bma[end == 0 ? BMA_DSC_IN : BMA_DSC_OUT] = ds_center;
  }
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
  if (e.fringe_type == BGT_FRINGE_HARD_EDGE_ONLY || e.fringe_type == BGT_FRINGE_SAD_FULL) fint_gap = 0;
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
      e.key != BGT_THICK_MULTIPOLE && e.key != BGT_SBEND) {
    err = ename(e) + ": electric multipoles are supported on quadrupoles, bends and thick multipoles only";
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
  bool use_mis = false, bend_mis = false;
  double tilt = 0;
  if (kind == K_QUAD || kind == K_THICK_MULT || kind == K_THIN_MULT) {
    use_mis = e.has_misalign != 0;
    tilt = e.tilt;
  } else if (kind == K_RFCAVITY) {
    use_mis = true;  // track_a_rfcavity calls offset_particle unconditionally
    tilt = e.tilt;
  } else if (kind == K_BEND) {
    // is_misaligned, offset_particle.f90:195-196
    const bool misaligned = offset || e.roll != 0;
    if (misaligned && (e.g != 0 || e.ref_tilt != 0 || e.roll != 0)) {
      use_mis = bend_mis = true;  // the bend geometry (BM block)
    } else if (misaligned) {
      use_mis = true;  // g = ref_tilt = roll = 0: the straight-element geometry
    } else {
      use_mis = e.has_misalign != 0 && e.ref_tilt != 0;
      tilt = e.ref_tilt;
    }
  }
  if (use_mis) {
    flags |= F_MISALIGN;
    if (bend_mis) flags |= F_BEND_MIS;
    if (offset && !bend_mis) flags |= F_OFFSET;
    if (pitch && !bend_mis) flags |= F_PITCH;
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
    if (kind == K_BEND) {
      // offset_particle(set, s_pos, no tilt) of a bend (offset_particle.f90:
      // 180-258): the bend geometry when misaligned with g, ref_tilt or roll
      // (BMA block), the straight geometry when misaligned otherwise, and a
      // bare ref_tilt rotation when not misaligned
      const bool misaligned = offset || e.roll != 0;
      if (e.offset_moves_aperture && (misaligned || e.ref_tilt != 0)) {
        if (!(flags & F_MISALIGN)) {
          err = ename(e) + ": offset_moves_aperture on a bend with ref_tilt needs has_misalign set";
          return BGT_EUNSUPPORTED;
        }
        flags |= F_AP_OFFSET;
        if (!misaligned) flags |= F_AP_TILT;
      }
    } else if (e.offset_moves_aperture && (flags & F_MISALIGN) && (offset || tilt != 0)) {
      flags |= F_AP_OFFSET;
      if (key == BGT_ECOLLIMATOR || key == BGT_RCOLLIMATOR) flags |= F_AP_TILT;
    }
    if (e.aperture_at == BGT_ENTRANCE_END || e.aperture_at == BGT_BOTH_ENDS) flags |= F_AP_ENTRANCE;
    if (e.aperture_at == BGT_EXIT_END || e.aperture_at == BGT_BOTH_ENDS) flags |= F_AP_EXIT;
    flags |= ap_ell ? F_AP_ELLIPTICAL : F_AP_RECT;
  }
  // a collimator's momentum and longitudinal limits (check_aperture_limit.f90:
  // 98-135) are checked at the ends aperture_at names whatever the transverse
  // limits; without transverse limits the aperture block holds zeros (no
  // transverse check)
  const bool ap_mom = (key == BGT_ECOLLIMATOR || key == BGT_RCOLLIMATOR) && e.aperture_at != BGT_NO_END &&
                      (e.px_aperture_width2 != 0 || e.py_aperture_width2 != 0 || e.z_aperture_width2 != 0 ||
                       e.pz_aperture_width2 != 0);
  if (ap_mom) {
    if (!ap_any) {
      if (e.aperture_at == BGT_ENTRANCE_END || e.aperture_at == BGT_BOTH_ENDS) flags |= F_AP_ENTRANCE;
      if (e.aperture_at == BGT_EXIT_END || e.aperture_at == BGT_BOTH_ENDS) flags |= F_AP_EXIT;
      flags |= F_AP_RECT;
    }
    flags |= F_AP_MOMENTUM;
    if (key == BGT_ECOLLIMATOR) flags |= F_AP_MOM_ELL;
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
    if (flags & F_BEND_MIS) bend_mis_block(e, B.ptr_after_push(BM_N));
    if ((flags & F_BEND_MIS) && (flags & F_AP_OFFSET)) bend_ap_block(e, B.ptr_after_push(BMA_N));
  }
  if (flags & (F_AP_ENTRANCE | F_AP_EXIT)) {
    double* a = B.ptr_after_push(AP_N);
    a[AP_X1] = ap_any ? -e.x1_limit : 0.0;
    a[AP_X2] = ap_any ? e.x2_limit : 0.0;
    a[AP_Y1] = ap_any ? -e.y1_limit : 0.0;
    a[AP_Y2] = ap_any ? e.y2_limit : 0.0;
    if (ap_any && ap_ell) {
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
    if (flags & F_AP_MOMENTUM) {
      double* m = B.ptr_after_push(APM_N);
      m[APM_PXW] = e.px_aperture_width2;
      m[APM_PXC] = e.px_aperture_center;
      m[APM_PYW] = e.py_aperture_width2;
      m[APM_PYC] = e.py_aperture_center;
      m[APM_ZW] = e.z_aperture_width2;
      m[APM_ZC] = e.z_aperture_center;
      m[APM_PZW] = e.pz_aperture_width2;
      m[APM_PZC] = e.pz_aperture_center;
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
      q[Q_DTREF] = e.delta_ref_time;
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
      q[TM_DTREF] = e.delta_ref_time;
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
        memcpy(q + RF_AMPQ, &amp, 16);
      }
      q[RF_TSTART] = e.ref_time_start;
      q[RF_PHI0_MP] = TWOPI_H * e.phi0_multipass;
      q[RF_RHALF] = 0.5 * r_step;
      // rf_coupler_kick.f90:41-60: e_accel_field(ele, gradient$) is voltage / l
      // (attribute_bookkeeper.f90:730-736) times field_autoscale = 1
      if (e.coupler_strength != 0) {
        const int cat = e.coupler_at;
        if (cat == BGT_ENTRANCE_END || cat == BGT_BOTH_ENDS) flags |= F_COUPLER_IN;
        if (cat == BGT_EXIT_END || cat == BGT_BOTH_ENDS) flags |= F_COUPLER_OUT;
        double gradient = e.voltage == 0 ? 0.0 : (e.l == 0 ? 1e30 : e.voltage / e.l);
        double field = e.is_on ? gradient * 1.0 : 0.0;
        double dp_coef = field * e.coupler_strength;
        double dp_x = dp_coef * cos(TWOPI_H * e.coupler_angle);
        double dp_y = dp_coef * sin(TWOPI_H * e.coupler_angle);
        if (cat == BGT_BOTH_ENDS) {
          dp_x = dp_x / 2;
          dp_y = dp_y / 2;
        }
        q[RF_CPL_DPX] = dp_x;
        q[RF_CPL_DPY] = dp_y;
        q[RF_CPL_PH] = TWOPI_H * e.coupler_phase;
      }
      h.n_step = n_slice;
      h.ix_mag_max = ix;
      break;
    }
    case K_BEND: {
      if (e.exact_multipoles != 0) {
        err = ename(e) + ": exact_multipoles is not supported";
        return BGT_EUNSUPPORTED;
      }
      const int ft = e.fringe_type;
      bool edges = ft != BGT_FRINGE_NONE;
      if (edges && ft != BGT_FRINGE_BASIC_BEND && ft != BGT_FRINGE_HARD_EDGE_ONLY && ft != BGT_FRINGE_SAD_FULL &&
          ft != BGT_FRINGE_SOFT_EDGE_ONLY && ft != BGT_FRINGE_LINEAR_EDGE && ft != BGT_FRINGE_FULL) {
        err = ename(e) + ": bend fringe_type " + std::to_string(ft) + " is not supported";
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
      if (ix > -1 || ixe > -1) n_step = std::max(nint_h(fabs(length) / e.ds_step), 1);
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
      q[B_FP0C] = r_step * e.p0c / (C_LIGHT_H * sp.charge);
      q[B_CDIR] = 1 * 1 * (double)sp.charge;
      put_lez(q + B_LEZ, e, sp.mass, p0c);
      q[B_K1 + 0] = b1 / e.l;
      q[B_K1 + 1] = 1 * e.l / n_step;
      q[B_K1 + 2] = g_tot;
      // the ends act for a fringe type or for the electric longitudinal
      // fringe alone (fringe_type none with electric multipoles:
      // apply_element_edge_kick.f90:101-103, 152-153)
      if (edges || ixe > -1) {
        if (e.fringe_at == BGT_ENTRANCE_END || e.fringe_at == BGT_BOTH_ENDS) flags |= F_EDGE_IN;
        if (e.fringe_at == BGT_EXIT_END || e.fringe_at == BGT_BOTH_ENDS) flags |= F_EDGE_OUT;
      }
      if (!edges && ixe > -1) flags |= F_NO_HWANG;
      put_edge(q + B_EDGE, e, true);
      put_edge(q + B_EDGE + EDGE_N, e, false);
      q[B_DTREF] = e.delta_ref_time;
      q[B_RBETAREF] = 1.0 / q[B_BETAREF];
      // bend_edge_kick (fringe_mod.f90:39-127): the Hwang map for basic_bend,
      // hard_edge_only and sad_full; the SAD soft edge for soft_edge_only and
      // sad_full (nothing when fint hgap or g + dg is zero); the linear edge;
      // for full the exact edge inside the k1 hard-edge multipole fringe
      if (edges && (ft == BGT_FRINGE_SOFT_EDGE_ONLY || ft == BGT_FRINGE_LINEAR_EDGE || ft == BGT_FRINGE_FULL))
        flags |= F_NO_HWANG;
      if (ft == BGT_FRINGE_FULL && (flags & (F_EDGE_IN | F_EDGE_OUT))) flags |= F_EXACT_EDGE;
      if ((ft == BGT_FRINGE_SOFT_EDGE_ONLY || ft == BGT_FRINGE_SAD_FULL) && e.g + e.dg != 0 &&
          (12 * e.fint * e.hgap != 0 || 12 * e.fintx * e.hgapx != 0))
        flags |= F_SOFT_EDGE;
      if (ft == BGT_FRINGE_LINEAR_EDGE) flags |= F_LINEAR_EDGE;
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
  if (kind == K_BEND && ixe > -1) {
    // electric multipoles of a bend: kicks in apply_multipole_kicks
    // (track_a_bend.f90:379-466), longitudinal fringe at the ends the Hwang
    // edges act (apply_element_edge_kick.f90:160-163)
    flags |= F_ELEC;
    h.aux1 = ixe;
    double* q = B.ptr_after_push(2 * (ixe + 1));
    for (int n = 0; n <= ixe; n++) {
      q[n] = e.an_elec[n];
      q[ixe + 1 + n] = e.bn_elec[n];
    }
    if (e.l != 0) flags |= F_ELEC_EDGE;
  }
  if (kind == K_BEND && (flags & F_SOFT_EDGE)) {
    // sad_soft_bend_edge_kick, fringe_mod.f90:913-930
    double* q = B.ptr_after_push(3);
    q[0] = 12 * e.fint * e.hgap;
    q[1] = 12 * e.fintx * e.hgapx;
    q[2] = e.g + e.dg;
  }
  if (kind == K_BEND && (flags & F_EXACT_EDGE)) {
    // exact_bend_edge_kick, fringe_mod.f90:1486-1511 (time_dir = 1) and the
    // strength of hard_multipole_edge_kick (fringe_mod.f90:737-738, 772-774)
    double* q = B.ptr_after_push(XE_N);
    const double beta0 = e.p0c / e.e_tot;
    q[XE_BETA0] = beta0;
    q[XE_IB] = 1 / beta0;
    q[XE_IB2] = 1 / (beta0 * beta0);
    const double g_tot = e.is_on ? e.g + e.dg : 0.0;
    q[XE_GTOT] = g_tot;
    q[XE_K1] = e.k1;
    for (int end = 0; end < 2; end++) {
      double* E = q + (end == 0 ? XE_IN : XE_OUT);
      const double a = 1 * (end == 0 ? e.e1 : e.e2);
      E[XE_A] = a;
      E[XE_TANA] = tan(a);
      E[XE_COSA] = cos(a);
      E[XE_SINA] = sin(a);
      E[XE_NA] = -a;
      E[XE_TANNA] = tan(-a);
      E[XE_COSNA] = cos(-a);
      E[XE_SINNA] = sin(-a);
      E[XE_SIN2NA] = sin(2.0 * -a);
      E[XE_B] = end == 0 ? g_tot : -g_tot;
      E[XE_FINT] = 1 * (end == 0 ? e.fint : e.fintx);
      E[XE_HGAP] = end == 0 ? e.hgap : e.hgapx;
    }
  }
  if (kind == K_BEND && (flags & F_LINEAR_EDGE)) {
    // linear_bend_edge_kick, fringe_mod.f90:170-201 (c_dir = 1)
    double* q = B.ptr_after_push(4);
    const double g_tot = e.is_on ? (e.g + e.dg) * 1.0 : 0.0;
    for (int end = 0; end < 2; end++) {
      const double ang = end == 0 ? e.e1 : e.e2, fint = end == 0 ? e.fint : e.fintx;
      const double hgap = end == 0 ? e.hgap : e.hgapx;
      const double cos_e = cos(ang), sin_e = sin(ang), tan_e = sin_e / cos_e;
      double ht_x = g_tot * tan_e, ht_y;
      if (fint == 0)
        ht_y = -ht_x;
      else
        ht_y = -g_tot * tan(ang - 2 * fint * g_tot * hgap * (1 + sin_e * sin_e) / cos_e);
      q[2 * end] = 1 * ht_x;
      q[2 * end + 1] = 1 * ht_y;
    }
  }
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
    // sextupoles
    if ((e.fringe_type == BGT_FRINGE_FULL || e.fringe_type == BGT_FRINGE_HARD_EDGE_ONLY) &&
        (key == BGT_QUADRUPOLE || key == BGT_SEXTUPOLE)) {
      flags |= F_HARD_EDGE;
      double* q = B.ptr_after_push(1);
      q[0] = (key == BGT_QUADRUPOLE) ? e.k1 : e.k2;
    }
    // soft_quadrupole_edge_kick (fringe_mod.f90:555-660): nothing unless fq1
    // or fq2 is nonzero
    if ((e.fringe_type == BGT_FRINGE_FULL || e.fringe_type == BGT_FRINGE_SOFT_EDGE_ONLY) &&
        key == BGT_QUADRUPOLE && (e.fq1 != 0 || e.fq2 != 0)) {
      flags |= F_SOFT_EDGE;
      double* q = B.ptr_after_push(3);
      q[0] = e.k1;
      q[1] = e.fq1;
      q[2] = e.fq2;
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

// Whether a compiled record uses a feature only the RARE kernels handle.
static bool record_is_rare(const RecHdr* rh) {
  return (rh->flags & (F_FRINGE_INFO | F_ELEC | F_AP_OFFSET | F_BEND_MIS | F_COUPLER_IN | F_COUPLER_OUT |
                       F_SOFT_EDGE | F_LINEAR_EDGE | F_NO_HWANG | F_EXACT_EDGE | F_AP_MOMENTUM)) != 0;
}

// The element tables of all variants, as bgt_create uploads them.  Per
// variant: the sequence of n_ele (int32 record offset in doubles, int32
// ix_ele) pairs, padded to 16 bytes, then the pool of unique records
// (identical elements share one).  Each table starts at table_off[v]
// doubles, 16-byte aligned; table_dw is the largest table rounded up to an
// even count and `all` is padded so that every table can be read as
// table_dw doubles.  Quadrupole records get a quad-matrix memo class in
// aux0 (same length, b1 and step -> same class; -1 past qmemo_classes).
// rare: some record needs the RARE kernels.  Returns 0 or
// BGT_EUNSUPPORTED with err set.
static int compile_tables(const bgt_element* eles, int32_t n_ele, int32_t n_variants, const bgt_species& sp,
                          int qmemo_classes, std::vector<double>& all, std::vector<int64_t>& table_off,
                          int32_t& table_dw, bool& rare, std::string& err) {
  const double p0c = eles[0].p0c;
  const int32_t seq_dw = n_ele + (n_ele % 2);  // (offset, ix_ele) int32 pairs, padded to 16 bytes
  all.clear();
  table_off.clear();
  table_dw = 0;
  rare = false;
  for (int v = 0; v < n_variants; v++) {
    std::vector<double> tab(seq_dw, 0.0);
    std::unordered_map<std::string, int32_t> pool;  // record bytes -> offset (identical elements share)
    std::unordered_map<std::string, int32_t> qclass;  // quad (length, b1, step) -> memo class
    for (int e = 0; e < n_ele; e++) {
      std::vector<double> rec;
      int rc = compile_element(eles[(int64_t)v * n_ele + e], sp, p0c, rec, err);
      if (rc) return rc;
      RecHdr* rh = reinterpret_cast<RecHdr*>(rec.data());
      rh->ix_ele = 0;  // carried by the sequence instead
      if (record_is_rare(rh)) rare = true;
      if (rh->kind == K_QUAD) {
        // quad-matrix memo class: same (b1, length, step) -> same quad_mat2_calc
        const double* kb = rec.data() + HDR_DW + ((rh->flags & F_MISALIGN) ? MIS_N : 0) +
                           ((rh->flags & (F_AP_ENTRANCE | F_AP_EXIT)) ? AP_N : 0);
        std::string ck(reinterpret_cast<const char*>(kb), 3 * sizeof(double));  // Q_LEN, Q_B1, Q_STEP
        auto ci = qclass.find(ck);
        if (ci != qclass.end()) {
          rh->aux0 = ci->second;
        } else if ((int)qclass.size() < qmemo_classes) {
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
    table_dw = std::max(table_dw, (int32_t)tab.size());
    table_off.push_back((int64_t)all.size());
    all.insert(all.end(), tab.begin(), tab.end());
    while (all.size() % 2) all.push_back(0.0);
  }
  // every table is read as table_dw doubles: pad the tail
  all.resize(table_off.back() + table_dw + 2, 0.0);
  if (table_dw % 2) table_dw++;
  return 0;
}

}  // namespace host
}  // namespace bgt
