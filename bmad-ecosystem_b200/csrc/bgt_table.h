// bgt_table.h -- device element table: one variable-length record per
// lattice element, packed as doubles so the whole table of a ring (a few
// tens of KB) is staged once per CTA into shared memory by a bulk TMA copy
// and then read by broadcast from there for every turn.
//
// Record = 4-double header (8 x int32) + kind-specific FP64 parameters.
// Every value that depends only on the element (never on the particle) is
// computed on the host with the same operation order the reference uses
// (e.g. sin/cos of tilts, Hwang edge coefficients, element-constant products
// that sit leftmost in a reference expression), so device results are
// value-identical to evaluating the reference expression in full.
#pragma once
#include <stdint.h>

#define BGT_MAXPOLE_DEV 21  // highest multipole order (n_pole_maxx)

namespace bgt {

enum Kind : int32_t {
  K_MARKER = 0,       // nothing but aperture checks
  K_DRIFT = 1,        // track_a_drift
  K_QUAD = 2,         // track_a_quadrupole
  K_BEND = 3,         // track_a_bend (+ Hwang edges)
  K_THICK_MULT = 4,   // track_a_thick_multipole (sext, oct, thick_multipole, kickers, collimators ...)
  K_THIN_MULT = 5,    // multipole / ab_multipole (track1_bmad.f90:142-166)
  K_RFCAVITY = 6,     // track_a_rfcavity
};

enum Flag : int32_t {
  F_OFFSET = 1 << 0,      // x/y/z offset or pitch -> offset_particle translation
  F_PITCH = 1 << 1,       // x/y pitch -> W rotation and drift to the edge
  F_TILT = 1 << 2,        // tilt_coords with tilt_tot (or ref_tilt for bends)
  F_AP_ENTRANCE = 1 << 3, // aperture checked at the entrance edge
  F_AP_EXIT = 1 << 4,     // aperture checked at the exit edge
  F_AP_ELLIPTICAL = 1 << 5,
  F_AP_RECT = 1 << 6,
  F_HV_KICK = 1 << 7,      // offset_particle set_hv1 kicks (rfcavity only)
  F_EDGE_IN = 1 << 8,      // Hwang edge at entrance
  F_EDGE_OUT = 1 << 9,     // Hwang edge at exit
  F_MISALIGN = 1 << 10,    // has_misalign (offset_particle is called)
  F_SEMI_LINEAR_OK = 1 << 11, // bend: dg == 0 so the near-axis semi-linear map may apply
  F_K1_BODY = 1 << 12,     // bend: sbend_body_with_k1_map
  F_DRIFT_BODY = 1 << 13,  // bend: body is a plain drift (g == dg == 0 or step_len == 0)
  F_IS_OFF = 1 << 14,      // bend is off (is_on = F)
  // quadrupole / thick multipole: init_fringe_info is true (a fringe type or
  // electric multipoles): the state is checked after each edge kick
  F_FRINGE_INFO = 1 << 15,
  // quadrupole / thick multipole / bend: electric multipoles, ae[aux1+1]
  // and be[aux1+1] follow the magnetic an/bn arrays.  For these kinds
  // F_EDGE_IN / F_EDGE_OUT mark the ends fringe_at names
  F_ELEC = 1 << 16,
  // the electric longitudinal fringe acts (electric multipoles, length != 0)
  F_ELEC_EDGE = 1 << 17,
  // quadrupole / sextupole hard-edge multipole fringe (fringe_type full or
  // hard_edge_only); the body strength (k1 or k2) follows the arrays
  F_HARD_EDGE = 1 << 18,
  // offset_moves_aperture: the aperture is checked in the element frame
  // (check_aperture_limit.f90:159-175); F_AP_TILT: with the tilt as well
  // (collimators)
  F_AP_OFFSET = 1 << 19,
  F_AP_TILT = 1 << 20,
  // misaligned bend with g, ref_tilt or roll nonzero: offset_particle's bend
  // geometry (offset_particle.f90:208-235, 393-425), a bend-misalignment
  // block (BM_*) after the misalignment block
  F_BEND_MIS = 1 << 21,
  // rfcavity coupler kick at the entrance / exit (rf_coupler_kick.f90)
  F_COUPLER_IN = 1 << 22,
  F_COUPLER_OUT = 1 << 23,
  // soft-edge fringe: a quadrupole's (fringe_type full or soft_edge_only,
  // fq1 or fq2 nonzero: k1, fq1, fq2 follow the hard-edge strength) or a
  // bend's SAD soft edge (soft_edge_only, sad_full: fb_in, fb_out, g + dg
  // after the electric multipoles)
  F_SOFT_EDGE = 1 << 24,
  // bend linear_edge fringe: ht_x, ht_y at the entrance, then at the exit,
  // after the electric multipoles
  F_LINEAR_EDGE = 1 << 25,
  // bend edges without the Hwang map (soft_edge_only, linear_edge, full)
  F_NO_HWANG = 1 << 26,
  // bend fringe_type full: the exact (PTC) bend edge and the k1 hard-edge
  // multipole fringe, an exact-edge block (XE_*) after the electric
  // multipoles
  F_EXACT_EDGE = 1 << 27,
  // collimator momentum / longitudinal limits (check_aperture_limit.f90:
  // 98-135), a block of APM_N doubles after the aperture block;
  // F_AP_MOM_ELL: the ecollimator's elliptical pairs
  F_AP_MOMENTUM = 1 << 28,
  F_AP_MOM_ELL = 1 << 29,
};

struct RecHdr {
  int32_t kind;
  int32_t ix_ele;
  int32_t size_dw;    // record size in doubles, header included
  int32_t flags;
  int32_t n_step;     // body steps (quad, bend, thick multipole), slices (rf)
  int32_t ix_mag_max; // highest multipole order with a kick (-1 = none)
  int32_t aux0;       // kind-specific
  int32_t aux1;       // kind-specific
};
static_assert(sizeof(RecHdr) == 32, "header is 4 doubles");

constexpr int HDR_DW = 4;

// ---- parameter offsets (in doubles, relative to the record start) ----
// Common blocks appear in this order after the header when their flag is set:
//   misalignment block (F_MISALIGN):      MIS_N doubles
//   bend-misalignment block (F_BEND_MIS): BM_N doubles
//   aperture block (F_AP_*):              AP_N doubles
// then the kind block.
constexpr int MIS_XOFF = 0, MIS_YOFF = 1, MIS_ZOFF = 2, MIS_LHALF = 3, MIS_COS = 4, MIS_SIN = 5;
constexpr int MIS_WINV = 6;   // 9 doubles: w_mat_inv (set), row-major
constexpr int MIS_W = 15;     // 9 doubles: w_mat (unset), row-major
constexpr int MIS_HK = 24, MIS_VK = 25;  // 0.5*charge_dir*hkick, 0.5*charge_dir*vkick
constexpr int MIS_DS_SET = 26;    // drift length to the body edge after the set translation (no pitch)
constexpr int MIS_DS_UNSET = 27;  // drift length back to the lab edge after unset (no pitch)
constexpr int MIS_R3SET = 28;     // 0 - (z_offset + ds_center) on set
constexpr int MIS_R3UNSET = 29;   // 0 - ds_center on unset
constexpr int MIS_ZADD = 30;      // z_offset + L/2 on unset
constexpr int MIS_COSU = 31, MIS_SINU = 32;  // cos/sin of -tilt (unset)
constexpr int MIS_R3EXIT = 33;    // 0 - (z_offset + ds_center) with s = L (aperture at the exit)
constexpr int MIS_N = 34;

// Bend-misalignment block (F_BEND_MIS).  The position (x, y, 0) goes through
// a short list of affine steps with element-constant matrices -- the
// bend_shift / misalignment / tilt frames offset_particle chains -- and the
// momentum (px, py, ps) through the product W of their matrices:
//   op (BM_OP_N doubles): [code, S (9, row-major), L (3)]
//   code 0: r3 = r3 - L3        (bend_shift with zero angle)
//   code 1: r = S r + L         (bend_shift; unset misalignment S r + L_mis)
//   code 2: r = S (r - L)       (set misalignment S^T (r - L_mis))
//   code 3: r = S r             (w_mat_for_tilt)
//   code 4: r3 = r3 + L3
constexpr int BM_NSET = 0, BM_NUNSET = 1;
constexpr int BM_WSET = 2, BM_WUNSET = 11;  // 9 doubles each, row-major
constexpr int BM_OP_N = 13, BM_MAX_OPS = 7;
constexpr int BM_OPS_SET = 20, BM_OPS_UNSET = BM_OPS_SET + BM_MAX_OPS * BM_OP_N;
constexpr int BM_N = BM_OPS_UNSET + BM_MAX_OPS * BM_OP_N;
// Bend aperture-frame block (F_BEND_MIS with F_AP_OFFSET), after the BM
// block: offset_particle(set, s_pos = 0 or L, no drift, no tilt) as
// check_aperture_limit.f90:159-175 calls it.  Per end the affine steps up to
// the particle-dependent arc shift (op layout as above) and ds_center; g.
constexpr int BMA_NIN = 0, BMA_NOUT = 1, BMA_G = 2, BMA_DSC_IN = 3, BMA_DSC_OUT = 4;
constexpr int BMA_OPS_IN = 5, BMA_OPS_OUT = BMA_OPS_IN + BM_MAX_OPS * BM_OP_N;
constexpr int BMA_N = BMA_OPS_OUT + BM_MAX_OPS * BM_OP_N;

constexpr int AP_X1 = 0, AP_X2 = 1, AP_Y1 = 2, AP_Y2 = 3;  // x1_lim = -x1_limit, ...
constexpr int AP_XW = 4, AP_XC = 5, AP_YW = 6, AP_YC = 7;  // elliptical width2/center
constexpr int AP_N = 8;
// Collimator momentum block (F_AP_MOMENTUM): width2 and center of px, py, z, pz
constexpr int APM_PXW = 0, APM_PXC = 1, APM_PYW = 2, APM_PYC = 3, APM_ZW = 4, APM_ZC = 5, APM_PZW = 6,
              APM_PZC = 7, APM_N = 8;

// Drift: L
constexpr int DR_L = 0, DR_N = 1;

// Quadrupole
constexpr int Q_LEN = 0;      // length (time_dir * L)
constexpr int Q_B1 = 1;       // charge_dir * b1
constexpr int Q_STEP = 2;     // step_len
constexpr int Q_RHALF = 3;    // r_step / 2
constexpr int Q_RSTEP = 4;    // r_step
constexpr int Q_LEZ = 5;      // low_energy_z_correction constants, LEZ_N doubles
constexpr int Q_DTREF = Q_LEZ + 6;  // delta_ref_time
constexpr int Q_N = Q_DTREF + 1;
constexpr int LEZ_BETA0 = 0, LEZ_MB2_THRESH = 1, LEZ_F = 2, LEZ_ME2 = 3, LEZ_MASS = 4, LEZ_3E7 = 5;

// Thick multipole: step_len, r_step/2, r_step, delta_ref_time
constexpr int TM_STEP = 0, TM_RHALF = 1, TM_RSTEP = 2, TM_DTREF = 3, TM_N = 4;

// Bend
constexpr int B_LEN = 0, B_G = 1, B_DG = 2, B_GTOT = 3, B_STEP = 4, B_ANGLE = 5, B_RSTEP = 6;
constexpr int B_COSA = 7, B_SINA = 8, B_SINCA = 9, B_COSCA = 10, B_BETAREF = 11, B_B1 = 12;
constexpr int B_LL2GCOSC = 13;    // ((step_len*step_len)*g)*cosc_a      (exact body)
constexpr int B_LLSINC = 14;      // step_len*sinc_a                     (exact body, semi-linear)
constexpr int B_M56C = 15;        // (g*ll)**2 * sincc(angle)            (semi-linear)
constexpr int B_GLLSINC = 16;     // (g*ll)*sinc_a                       (semi-linear)
constexpr int B_GLL2COSC = 17;    // (g*ll**2)*cosc_a                    (semi-linear)
constexpr int B_GSIN = 18;        // g*sin_a                             (semi-linear)
constexpr int B_FP0C = 19;        // multipole kick: r_step * p0c / (c_light * charge)
constexpr int B_CDIR = 20;        // c_dir = charge (multipole kick)
constexpr int B_LEZ = 21;         // low_energy_z_correction block (k1 body)
constexpr int B_K1 = B_LEZ + 6;   // k1 body: k1 = b1/L, length (= L/n_step), g_tot
constexpr int B_EDGE = B_K1 + 3;  // Hwang edge constants, entrance block then exit block
// Hwang edge block (fringe_mod.f90:240-418); C1 is (gt*g_tot)*(1+2*tan_e**2)
// at the entrance and gt*gt2 at the exit, the leftmost constant factors of
// the dpx terms.
constexpr int EDGE_GT = 0, EDGE_GT2 = 1, EDGE_GS2 = 2, EDGE_K1TANE = 3, EDGE_K1TANE2 = 4, EDGE_FG = 5,
              EDGE_C1 = 6, EDGE_C3 = 7, EDGE_C4 = 8, EDGE_GPG = 9, EDGE_GTGS2_2K1 = 10;
constexpr int EDGE_N = 11;
constexpr int B_DTREF = B_EDGE + 2 * EDGE_N;  // delta_ref_time
constexpr int B_RBETAREF = B_DTREF + 1;       // RN(1 / beta_ref): divides by beta_ref via div_by
constexpr int B_N = B_RBETAREF + 1;

// Exact bend edge block (F_EXACT_EDGE, exact_bend_edge_kick,
// fringe_mod.f90:1465-1686): beta0 = p0c / e_tot, 1 / beta0,
// 1 / beta0**2, g_tot (0 for a bend that is off), k1 (hard-edge multipole
// fringe), then one block per end, entrance first.  Per end, with a the
// edge angle (e1 or e2): a, tan / cos / sin of a (the frame rotation),
// -a, tan / cos / sin of -a and sin(-2a) (the wedge, or a rotation when
// g_tot = 0), then the dipole fringe's b (g_tot at the entrance, -g_tot at
// the exit), fint and hgap (fintx and hgapx at the exit).
constexpr int XE_BETA0 = 0, XE_IB = 1, XE_IB2 = 2, XE_GTOT = 3, XE_K1 = 4, XE_IN = 5;
constexpr int XE_A = 0, XE_TANA = 1, XE_COSA = 2, XE_SINA = 3, XE_NA = 4, XE_TANNA = 5, XE_COSNA = 6,
              XE_SINNA = 7, XE_SIN2NA = 8, XE_B = 9, XE_FINT = 10, XE_HGAP = 11, XE_END_N = 12;
constexpr int XE_OUT = XE_IN + XE_END_N, XE_N = XE_IN + 2 * XE_END_N;

// Thin multipole: per pole n (0..ix_mag_max): knl, cos(tilt), sin(tilt), tilt_is_zero
constexpr int TH_REFORB = 0;  // ref_orb_offset (1.0 for multipole$, else 0)
constexpr int TH_N = 1;
constexpr int TH_POLE = 4;    // doubles per pole

// RF cavity
constexpr int RF_LEN = 0, RF_VOLT = 1, RF_PHI0 = 2, RF_FREQ = 3, RF_NSLICE = 4, RF_SLICE_L = 5;
constexpr int RF_TWOPI_F = 6;  // twopi * rf_frequency
constexpr int RF_HALF_AMP_HI = 7, RF_HALF_AMP_LO = 8;  // 0.5/f as double-double
constexpr int RF_PHI0_MP = 9;  // twopi * phi0_multipass
constexpr int RF_RHALF = 10;   // 0.5 * r_step (multipole kicks)
constexpr int RF_CPL_DPX = 11, RF_CPL_DPY = 12;  // coupler dp_x, dp_y (halved for both ends)
constexpr int RF_CPL_PH = 13;  // twopi * coupler_phase
constexpr int RF_TSTART = 14;  // ref_time_start (absolute time)
constexpr int RF_AMPQ = 15;    // 0.5/f in real(qp): binary128 bits in two doubles (absolute time)
constexpr int RF_N = 17;

// Multipole arrays for quad / bend / thick multipole / rf follow the kind
// block: an[0..ix_mag_max], bn[0..ix_mag_max].

}  // namespace bgt
