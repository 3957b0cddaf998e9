/*
 * bmad_oracle.h -- CPU oracle for the bgt tracker.  TEST INFRASTRUCTURE ONLY.
 *
 * This is a plain-C, FP64 restatement of the reference's `bmad_standard`
 * element-by-element tracking path (Bmad, Fortran).  It exists to check the
 * CUDA tracker: only tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline leg may load it.  Nothing in the product links or calls it.
 *
 * Every routine names the reference file:line it follows.  Operation order is
 * kept as written in the Fortran so that, compiled without FMA contraction
 * (-ffp-contract=off), results match the reference gfortran -O2 build up to
 * libm differences.
 *
 * Parity pins: the reference's own golden vectors
 *   regression_tests/tracking_method_test/output.correct  (Bmad_Standard rows)
 *   regression_tests/fringe_test/output.correct           (Hwang edge kick)
 *   regression_tests/aperture_test/output.correct         (aperture states)
 * are checked against this oracle by tests/test_oracle_golden.py.
 *
 * Scope: forward tracking only (orbit%direction = +1, time_dir = +1,
 * ele%orientation = +1), relative-time RF (bmad_com%absolute_time_tracking
 * = F, the reference default), no radiation, no spin, no slaves/lords.
 */
#ifndef BMAD_ORACLE_H
#define BMAD_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

#define BGO_N_POLE 22 /* n_pole_maxx = 21, bmad_struct.f90:48 */

/* Element keys (subset of bmad_struct.f90 key list used on the path). */
enum {
  BGO_DRIFT = 1,
  BGO_QUADRUPOLE = 2,
  BGO_SBEND = 3,
  BGO_SEXTUPOLE = 4,
  BGO_OCTUPOLE = 5,
  BGO_THICK_MULTIPOLE = 6,
  BGO_MULTIPOLE = 7,
  BGO_AB_MULTIPOLE = 8,
  BGO_RFCAVITY = 9,
  BGO_MARKER = 10,
  BGO_ECOLLIMATOR = 11,
  BGO_RCOLLIMATOR = 12,
  BGO_INSTRUMENT = 13,
  BGO_MONITOR = 14,
  BGO_PIPE = 15,
  BGO_HKICKER = 16,
  BGO_VKICKER = 17,
  BGO_KICKER = 18
};

/* coord_struct%state codes, bmad_struct.f90:522-527 */
enum {
  BGO_ALIVE = 1,
  BGO_LOST = 2,
  BGO_LOST_NEG_X = 3,
  BGO_LOST_POS_X = 4,
  BGO_LOST_NEG_Y = 5,
  BGO_LOST_POS_Y = 6,
  BGO_LOST_Z = 7,
  BGO_LOST_PZ = 8
};

/* fringe_type values (names as in bmad_struct.f90) */
enum {
  BGO_FRINGE_NONE = 0,
  BGO_FRINGE_BASIC_BEND = 1,
  BGO_FRINGE_FULL = 2,
  BGO_FRINGE_HARD_EDGE_ONLY = 3,
  BGO_FRINGE_SOFT_EDGE_ONLY = 4,
  BGO_FRINGE_SAD_FULL = 5,
  BGO_FRINGE_LINEAR_EDGE = 6
};

/* fringe_at / aperture_at values */
enum {
  BGO_NO_END = 0,
  BGO_ENTRANCE_END = 1,
  BGO_EXIT_END = 2,
  BGO_BOTH_ENDS = 3
};

/* aperture_type values */
enum {
  BGO_APERTURE_RECTANGULAR = 0,
  BGO_APERTURE_ELLIPTICAL = 1
};

typedef struct bgo_param {
  double mass;               /* mass_of(species) [eV] */
  int charge;                /* charge_of(species) [e] */
  double max_aperture_limit; /* bmad_com%max_aperture_limit = 1e3, bmad_struct.f90:2297 */
  int aperture_limit_on;     /* bmad_com%aperture_limit_on, default T */
  double unstable_factor;    /* lat_param_struct%unstable_factor (output) */
  int absolute_time_tracking;  /* bmad_com%absolute_time_tracking, default F (bmad_struct.f90:2333) */
  int absolute_time_ref_shift; /* bmad_com%absolute_time_ref_shift, default T (bmad_struct.f90:2334) */
} bgo_param;

typedef struct bgo_coord {
  double vec[6];
  double beta;
  double p0c;
  int state;
  __float128 t; /* coord_struct%t: the particle time, real(qp) (bmad_struct.f90:546-574) */
} bgo_coord;

typedef struct bgo_ele {
  int key, ix_ele, is_on;
  int fringe_type, fringe_at, aperture_type, aperture_at, offset_moves_aperture;
  int has_mag_poles, has_elec_poles; /* associated(ele%a_pole), associated(ele%a_pole_elec) */
  int scale_multipoles, field_master;
  int has_misalign;                  /* ele%bookkeeping_state%has_misalign (set by bgo_bookkeeper) */
  int num_steps;
  int coupler_at; /* rfcavity: ends with the coupler kick */
  double l, k1, k2, k3, g, dg, e1, e2, fint, hgap, fintx, hgapx;
  double voltage, phi0, phi0_multipass, rf_frequency;
  double p0c, e_tot, ds_step;
  double x_offset, y_offset, z_offset, x_pitch, y_pitch, tilt, ref_tilt, roll;
  double hkick, vkick, kick;
  double x1_limit, x2_limit, y1_limit, y2_limit;
  double px_aperture_width2, px_aperture_center, py_aperture_width2, py_aperture_center;
  double z_aperture_width2, z_aperture_center, pz_aperture_width2, pz_aperture_center;
  double r0_mag, r0_elec;
  double coupler_strength, coupler_angle, coupler_phase;
  double fq1, fq2;
  /* ele%value(delta_ref_time$), ele%value(ref_time_start$): the reference
   * particle's time through the element and at its entrance
   * (lat_compute_reference_energy.f90:540-760) */
  double delta_ref_time, ref_time_start;
  /* For BGO_MULTIPOLE: a_pole = knl, b_pole = tn, ksl_pole = ksl (pointer_to_ele_multipole). */
  double a_pole[BGO_N_POLE], b_pole[BGO_N_POLE], ksl_pole[BGO_N_POLE];
  double a_pole_elec[BGO_N_POLE], b_pole_elec[BGO_N_POLE];
} bgo_ele;

/* ---- bookkeeping (host setup) ---- */
void bgo_ele_init(bgo_ele* ele, int key);
int bgo_bookkeeper(bgo_ele* ele);
int bgo_multipole_ele_to_ab(const bgo_ele* ele, int use_ele_tilt, int electric, int include_kicks,
                            double* a, double* b, double* b1 /* may be NULL */);
int bgo_multipole_ele_to_kt(const bgo_ele* ele, int use_ele_tilt, double* knl, double* tilt);
double bgo_c_multi(int n, int m, int no_n_fact);

/* ---- single particle ---- */
void bgo_init_coord(bgo_coord* orb, const double vec[6], double p0c, const bgo_param* param);
void bgo_track1(bgo_coord* orb, const bgo_ele* ele, bgo_param* param);
int bgo_orbit_too_large(bgo_coord* orb, bgo_param* param);
void bgo_check_aperture_limit(bgo_coord* orb, const bgo_ele* ele, int at_exit, bgo_param* param);
void bgo_hwang_bend_edge_kick(const bgo_ele* ele, int entering, bgo_coord* orb, const bgo_param* param);
void bgo_offset_particle(const bgo_ele* ele, int set, bgo_coord* orb, int s_pos_mode, double s_pos,
                         const bgo_param* param, double* s_out);

/* ---- lattice / multi-turn drivers ----
 * Coordinates are SoA: x[n], px[n], ... (six arrays packed as vec6[6*n], index c*n+i)
 * plus beta[n]; state/ix_ele_lost/ix_turn_lost are int32.
 * ix_ele_lost is the element's ix_ele (Bmad element index), ix_turn_lost the
 * 0-based turn index in which the loss happened (-1 while alive).
 */
/* t (may be NULL): the particle times t[n], real(qp) like coord_struct%t. */
void bgo_track_turns(const bgo_ele* eles, int n_ele, const bgo_param* param, double p0c, double* vec6,
                     double* beta, __float128* t, int* state, int* ix_ele_lost, int* ix_turn_lost, long n,
                     int turn0, int n_turns, int n_threads, int element_outer);

/* Count of FP64 operations (add/sub/mul/div/sqrt = 1, libm call = 1 each,
 * tallied separately) executed by bgo_track1 since the last reset. */
void bgo_flop_counter_reset(void);
void bgo_flop_counter_read(double* flops, double* libm_calls);

#ifdef __cplusplus
}
#endif
#endif
