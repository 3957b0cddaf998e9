// bgt_track.cu -- host side of the FP64 tracker: the element-table compiler,
// the handle, the launch dispatch and the C ABI declared in include/bgt.h.
// The kernel itself is in bgt_kernel.cuh (instances in bgt_track_kernels.cu).
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
#include "bgt_kernel.cuh"

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
    if (flags & F_BEND_MIS) bend_mis_block(e, B.ptr_after_push(BM_N));
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
          ft != BGT_FRINGE_SOFT_EDGE_ONLY && ft != BGT_FRINGE_LINEAR_EDGE) {
        err = ename(e) + ": bend fringe_type full (the exact bend edge) is not supported";
        return BGT_EUNSUPPORTED;
      }
      if (ixe > -1 && !edges && e.fringe_at != BGT_NO_END) {
        err = ename(e) + ": electric multipoles on a bend with fringe_type none are not supported";
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
      // bend_edge_kick (fringe_mod.f90:39-127): the Hwang map for basic_bend,
      // hard_edge_only and sad_full; the SAD soft edge for soft_edge_only and
      // sad_full (nothing when fint hgap or g + dg is zero); the linear edge
      if (edges && (ft == BGT_FRINGE_SOFT_EDGE_ONLY || ft == BGT_FRINGE_LINEAR_EDGE)) flags |= F_NO_HWANG;
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
  bool rare = false;  // some record needs the RARE kernels
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


static size_t smem_bytes(const bgt_handle* h, int block, bool compact, bool gtab = false) {
  size_t b = gtab ? 0 : (size_t)h->table_dw * 8;
  if (compact) b += (size_t)9 * block * 8;
  b += (size_t)QMEMO_CLASSES * 13 * block * 8;
  return b;
}

namespace bgt {
TrackKernelGroup track_kernel_group_0();
TrackKernelGroup track_kernel_group_1();
TrackKernelGroup track_kernel_group_2();
TrackKernelGroup track_kernel_group_3();
TrackKernelGroup track_kernel_group_4();
TrackKernelGroup track_kernel_group_5();
TrackKernelGroup track_kernel_group_6();
TrackKernelGroup track_kernel_group_7();
TrackKernelGroup track_kernel_group_8();
TrackKernelGroup track_kernel_group_9();
TrackKernelGroup track_kernel_group(int g) {
  static TrackKernelGroup (*const groups[N_KERNEL_GROUPS])() = {
      track_kernel_group_0, track_kernel_group_1, track_kernel_group_2, track_kernel_group_3,
      track_kernel_group_4, track_kernel_group_5, track_kernel_group_6, track_kernel_group_7,
      track_kernel_group_8, track_kernel_group_9};
  return groups[g]();
}
}  // namespace bgt

// The compiled kernel for a shape, table mode and feature set, or nullptr.
static LaunchFn find_track_kernel(int block, int minb, int tmode, bool rare) {
  for (int g = 0; g < N_KERNEL_GROUPS; g++) {
    const TrackKernelGroup grp = track_kernel_group(g);
    for (int i = 0; i < grp.n; i++) {
      const TrackKernel& k = grp.kernels[i];
      if (k.block == block && k.minb == minb && k.tmode == tmode && k.rare == rare) return k.launch;
    }
  }
  return nullptr;
}

// Fill every kernel group's copy of the multipole coefficient tables on the
// current device.
static cudaError_t upload_multipole_tables() {
  static double cm[BGT_MAXPOLE_DEV + 1][BGT_MAXPOLE_DEV + 1], cm0[BGT_MAXPOLE_DEV + 1][BGT_MAXPOLE_DEV + 1];
  host::c_multi_tables(cm, cm0);
  for (int g = 0; g < N_KERNEL_GROUPS; g++) {
    cudaError_t e = track_kernel_group(g).upload_cm(&cm[0][0], &cm0[0][0], sizeof(cm));
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

// Whether a compiled record uses a feature only the RARE kernels handle.
static bool record_is_rare(const RecHdr* rh) {
  return (rh->flags & (F_FRINGE_INFO | F_ELEC | F_AP_OFFSET | F_BEND_MIS | F_COUPLER_IN | F_COUPLER_OUT |
                       F_SOFT_EDGE | F_LINEAR_EDGE | F_NO_HWANG)) != 0;
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
  const int bps = h->tuning.blocks_per_sm;
  const LaunchFn launch = find_track_kernel(block, bps, gtab ? (warp_sched ? 2 : 1) : 0, h->rare);
  if (!launch) {
    if (gtab)
      return set_err(h, BGT_ETOOLARGE,
                     "element table read from global memory: tuning must be (128: 3,4,5) or (256: 2,3)");
    return set_err(h, BGT_EINVAL,
                   "tuning (threads_per_block, blocks_per_sm) must be one of (64: 8,10,12,16), "
                   "(128: 4,5,6,8), (256: 2,3,4)");
  }
  const cudaError_t e = launch(a, (int)grid, smem, st);
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
      if (record_is_rare(rh)) h->rare = true;
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
  if ((e = upload_multipole_tables()) != cudaSuccess) {
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
    if ((ce = upload_multipole_tables()) != cudaSuccess)
      return fail(BGT_ECUDA, std::string("coefficient upload: ") + cudaGetErrorString(ce));
    bgt::g_noalloc_ptr[device] = static_cast<unsigned char*>(p);
  }
  unsigned char* base = bgt::g_noalloc_ptr[device];

  // compile the table on the host (same records as bgt_create, one variant)
  std::vector<double> tab((size_t)(n_ele + (n_ele % 2)), 0.0);
  std::unordered_map<std::string, int32_t> pool;
  std::string msg;
  bool rare = false;
  const double p0c = eles[0].p0c;
  for (int e = 0; e < n_ele; e++) {
    std::vector<double> rec;
    int rc = bgt::host::compile_element(eles[e], *species, p0c, rec, msg);
    if (rc) return fail(rc, msg);
    bgt::RecHdr* rh = reinterpret_cast<bgt::RecHdr*>(rec.data());
    rh->ix_ele = 0;
    if (record_is_rare(rh)) rare = true;
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
    if (!((block == 128 && t.blocks_per_sm == 4) || (block == 256 && t.blocks_per_sm == 2)))
      return fail(BGT_EINVAL, "bgt_track_turns_device_noalloc: tuning must be (128, 4) or (256, 2)");
    ce = find_track_kernel(block, t.blocks_per_sm, 0, rare)(a, (int)grid, smem, st);
    if (ce != cudaSuccess) return fail(BGT_ECUDA, std::string("track_kernel launch: ") + cudaGetErrorString(ce));
  }
  return 0;
}
