/*
 * bmad_oracle.c -- CPU oracle for the bgt tracker.  TEST INFRASTRUCTURE ONLY.
 *
 * Plain-C FP64 restatement of the reference's `bmad_standard` tracking path.
 * Each function cites the reference file:line it restates (paths relative to
 * the Bmad project root).  Build flags: -O2 -ffp-contract=off (no FMA
 * contraction, like gfortran -O2 on x86-64), -fopenmp.  libm supplies
 * sin/cos/asin/atan2/sinh/cosh as it does for the reference.
 *
 * Only forward tracking (direction = time_dir = orientation = +1) and
 * relative-time RF are restated; the tracking species equals the reference
 * species, so rel_tracking_charge_to_mass = 1.
 */
#include "bmad_oracle.h"

#include <math.h>
#include <quadmath.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* sim_utils/interfaces/physical_constants.f90:12-13,34 */
static const double PI = 3.141592653589793238462643383279;
#define TWOPI (2 * PI)
static const double C_LIGHT = 2.99792458e8;

#ifdef BGO_COUNT_FLOPS
static double g_flops = 0, g_libm = 0;
#define FL(n) (g_flops += (n))
#define LM(n) (g_libm += (n))
#else
#define FL(n) ((void)0)
#define LM(n) ((void)0)
#endif

void bgo_flop_counter_reset(void) {
#ifdef BGO_COUNT_FLOPS
  g_flops = 0;
  g_libm = 0;
#endif
}

void bgo_flop_counter_read(double* flops, double* libm_calls) {
#ifdef BGO_COUNT_FLOPS
  *flops = g_flops;
  *libm_calls = g_libm;
#else
  *flops = -1;
  *libm_calls = -1;
#endif
}

static double sq(double x) { return x * x; }

/* Transcendentals of particle coordinates.  The default build calls the C
 * library (as the reference does); the BGO_CR_LIBM build rounds libquadmath's
 * quad-precision values to double, i.e. correctly rounded results.  Element
 * constants (tilts, bend angles, edge angles) always use the C library. */
#ifdef BGO_CR_LIBM
static double P_SIN(double x) { return (double)sinq((__float128)x); }
static double P_COS(double x) { return (double)cosq((__float128)x); }
static double P_ASIN(double x) { return (double)asinq((__float128)x); }
static double P_ATAN2(double y, double x) { return (double)atan2q((__float128)y, (__float128)x); }
static double P_SINH(double x) { return (double)sinhq((__float128)x); }
static double P_COSH(double x) { return (double)coshq((__float128)x); }
static double P_EXP(double x) { return (double)expq((__float128)x); }
static double P_TAN(double x) { return (double)tanq((__float128)x); }
static double P_ATAN(double x) { return (double)atanq((__float128)x); }
#else
#define P_SIN sin
#define P_COS cos
#define P_ASIN asin
#define P_ATAN2 atan2
#define P_SINH sinh
#define P_COSH cosh
#define P_EXP exp
#define P_TAN tan
#define P_ATAN atan
#endif

/* x**m for integer m, as gfortran evaluates it (repeated squaring,
 * libgcc __powidf2 / libgfortran pow_r8_i4 order of multiplies). */
static double powi_f(double x, int m) {
  unsigned n = (unsigned)(m < 0 ? -m : m);
  double y = (n % 2) ? x : 1;
  while (n >>= 1) {
    x = x * x;
    FL(1);
    if (n % 2) {
      y = y * x;
      FL(1);
    }
  }
  return m < 0 ? 1 / y : y;
}

/* sim_utils/special_functions/sqrt_one.f90:18-40 (nd = 0) */
static double sqrt_one(double x) {
  double sqv = sqrt(1 + x);
  double rad = sqv + 1;
  FL(4);
  return x / rad;
}

/* sim_utils/special_functions/sinc.f90:15-45 (nd = 0) */
static double sinc_f(double x) {
  if (fabs(x) < 1e-8) return 1.0;
  LM(1);
  FL(1);
  return sin(x) / x;
}

/* sinc of a particle-dependent argument */
static double sinc_p(double x) {
  if (fabs(x) < 1e-8) return 1.0;
  LM(1);
  FL(1);
  return P_SIN(x) / x;
}

/* sim_utils/special_functions/cosc.f90:15-35 (nd = 0) */
static double cosc_f(double x) {
  if (fabs(x) < 1e-8) return 0.50;
  double s = sinc_f(x / 2);
  FL(3);
  return 0.5 * (s * s);
}

/* sim_utils/special_functions/sincc.f90:15-45 (nd = 0) */
static double sincc_f(double x) {
  const double c0 = 1.0 / 6.0, c1 = -1.0 / 120.0, c2 = 1.0 / 5040.0, c3 = -1.0 / 362880.0;
  double x2 = x * x;
  if (fabs(x) < 0.1) {
    FL(7);
    return c0 + x2 * (c1 + x2 * (c2 + x2 * c3));
  }
  LM(1);
  FL(4);
  return (x - sin(x)) / (x * x2);
}

/* Fortran MODULO(a, p) for reals as gfortran evaluates it: fmod, then shift
 * into the sign of p. */
static double fmodulo(double a, double p) {
  double r = fmod(a, p);
  if (r != 0 && ((r < 0) != (p < 0))) r += p;
  return r;
}

/* sim_utils/special_functions/modulo2_mod.f90:85-98 */
static double modulo2_dp(double x, double amp) {
  double m2 = fmodulo(x, 2 * amp);
  if (m2 >= amp) m2 = m2 - 2 * amp;
  return m2;
}

/* sim_utils/special_functions/modulo2_mod.f90:121-134 (quad precision) */
static __float128 modulo2_qp(__float128 x, __float128 amp) {
  __float128 p = 2 * amp;
  __float128 r = fmodq(x, p);
  if (r != 0 && ((r < 0) != (p < 0))) r += p;
  if (r >= amp) r = r - 2 * amp;
  return r;
}

/* ------------------------------------------------------------------ */
/* c_multi, bmad/low_level/c_multi.f90:19-75                           */

static double g_cm[BGO_N_POLE][BGO_N_POLE];
static double g_nfact[BGO_N_POLE];
static int g_cm_init = 0;

static void c_multi_init(void) {
  if (g_cm_init) return;
  memset(g_cm, 0, sizeof(g_cm));
  g_cm[0][0] = 1;
  for (int in = 1; in < BGO_N_POLE; in++) {
    g_cm[in][0] = 1;
    g_cm[in][in] = 1;
    for (int im = 1; im <= in - 1; im++) g_cm[in][im] = g_cm[in - 1][im - 1] + g_cm[in - 1][im];
  }
  g_nfact[0] = 1;
  for (int in = 0; in < BGO_N_POLE; in++) {
    if (in > 0) g_nfact[in] = in * g_nfact[in - 1];
    for (int im = 0; im <= in; im++) {
      g_cm[in][im] = g_cm[in][im] / g_nfact[in];
      if (im % 4 == 0) g_cm[in][im] = -g_cm[in][im];
      if (im % 4 == 3) g_cm[in][im] = -g_cm[in][im];
    }
  }
  g_cm_init = 1;
}

double bgo_c_multi(int n, int m, int no_n_fact) {
  c_multi_init();
  if (no_n_fact) return g_cm[n][m] * g_nfact[n];
  return g_cm[n][m];
}

/* sim_utils factorial (real result, exact product for n <= 21 as doubles) */
static double factorial_f(int n) {
  double f = 1;
  for (int i = 2; i <= n; i++) f = f * i;
  return f;
}

/* bmad/low_level/mexp.f90:14-33 */
static double mexp(double x, int m) {
  if (m < 0) return 0;
  if (m == 0) return 1;
  return powi_f(x, m);
}

/* sim_utils/math/max_nonzero.f90:19-45 */
static int max_nonzero2(const double* a, const double* b, int n) {
  for (int i = n - 1; i >= 0; i--) {
    if (a[i] != 0) return i;
    if (b && b[i] != 0) return i;
  }
  return -1;
}

static int sign_of(double x) { return x < 0 ? -1 : 1; }

/* ------------------------------------------------------------------ */
/* Element init + bookkeeping                                          */

void bgo_ele_init(bgo_ele* ele, int key) {
  memset(ele, 0, sizeof(*ele));
  ele->key = key;
  ele->is_on = 1;
  ele->scale_multipoles = 1;
  ele->aperture_at = BGO_EXIT_END; /* bmad_struct.f90:1495 */
  ele->aperture_type = (key == BGO_ECOLLIMATOR) ? BGO_APERTURE_ELLIPTICAL : BGO_APERTURE_RECTANGULAR;
  ele->fringe_at = BGO_BOTH_ENDS; /* set_ele_defaults.f90:35 */
  ele->fringe_type = BGO_FRINGE_NONE; /* set_ele_defaults.f90:36 */
  if (key == BGO_SBEND) ele->fringe_type = BGO_FRINGE_BASIC_BEND; /* set_ele_defaults.f90:298 */
  if (key == BGO_RFCAVITY) {
    ele->fringe_type = BGO_FRINGE_FULL; /* set_ele_defaults.f90:315 */
    ele->num_steps = 10;                /* set_ele_defaults.f90:317 */
    ele->coupler_at = BGO_EXIT_END;     /* set_ele_defaults.f90:309 */
  }
  if (key == BGO_RCOLLIMATOR || key == BGO_ECOLLIMATOR) ele->offset_moves_aperture = 1;
  ele->fintx = NAN; /* real_garbage$ until bookkeeping copies fint */
  ele->hgapx = NAN;
}

/* PTC check_bend, forest/code/So_fitting.f90:3504-3536 */
static int check_bend(double xl, double ggi, double rhoi, double xbend1, double gf[8]) {
  double co[8] = {0};
  double gg = (double)(long)ggi; /* int(ggi) */
  if (gg == 0) gg = 1;
  co[2] = 1.0 / 12.0;
  co[4] = 0.17;
  co[6] = 0.17e-1;
  for (int i = 0; i < 8; i++) gf[i] = 0;
  for (int i = 3; i <= 7; i += 2) {
    double ar = i - 1;
    gf[i] = pow(co[i - 1] / xbend1, 1.0 / ar) * fabs(rhoi) * xl;
    if (gf[i] < gg) gf[i] = gg;
  }
  gf[2] = gf[3];
  gf[4] = gf[5] * 3;
  gf[6] = gf[7] * 7;
  int met = 2;
  if (gf[4] < gf[2]) met = 4;
  if (gf[6] < gf[4] && gf[6] < gf[2]) met = 6;
  return met;
}

static int nint_f(double x) { return (int)lround(x); }

/* bmad/code/attribute_bookkeeper.f90:150-180 (tilt_tot / has_misalign) and
 * :295-404 (ds_step / num_steps).  Returns 0 on success. */
int bgo_bookkeeper(bgo_ele* ele) {
  c_multi_init();
  if (isnan(ele->fintx)) ele->fintx = ele->fint;
  if (isnan(ele->hgapx)) ele->hgapx = ele->hgap;

  if (ele->key == BGO_SBEND) {
    ele->has_misalign = (ele->ref_tilt != 0 || ele->roll != 0);
  } else {
    ele->has_misalign = (ele->tilt != 0);
  }
  ele->has_misalign = ele->has_misalign || ele->x_offset != 0 || ele->y_offset != 0 || ele->z_offset != 0 ||
                      ele->x_pitch != 0 || ele->y_pitch != 0;

  int has_ds = 0;
  switch (ele->key) {
    case BGO_DRIFT: case BGO_QUADRUPOLE: case BGO_SBEND: case BGO_SEXTUPOLE: case BGO_OCTUPOLE:
    case BGO_THICK_MULTIPOLE: case BGO_RFCAVITY: case BGO_ECOLLIMATOR: case BGO_RCOLLIMATOR:
    case BGO_INSTRUMENT: case BGO_MONITOR: case BGO_PIPE: case BGO_HKICKER: case BGO_VKICKER:
    case BGO_KICKER:
      has_ds = 1;
      break;
    default:
      has_ds = 0;
  }
  if (!has_ds || ele->p0c <= 0) return 0;

  if (ele->ds_step == 0 && ele->num_steps == 0) {
    switch (ele->key) {
      case BGO_DRIFT: case BGO_PIPE: case BGO_ECOLLIMATOR: case BGO_RCOLLIMATOR: case BGO_INSTRUMENT:
      case BGO_MONITOR:
        ele->num_steps = 1;
        ele->ds_step = ele->l;
        break;
      case BGO_SBEND: case BGO_QUADRUPOLE: case BGO_SEXTUPOLE:
        if (ele->l != 0) {
          double knl[BGO_N_POLE], tl[BGO_N_POLE], gf[8];
          double a[BGO_N_POLE], b[BGO_N_POLE];
          bgo_multipole_ele_to_ab(ele, 0, 0, 1, a, b, NULL);
          for (int n = 0; n < BGO_N_POLE; n++) {
            /* multipole1_ab_to_kt, bmad/low_level/multipole1_ab_to_kt.f90 */
            knl[n] = (a[n] == 0 && b[n] == 0) ? 0 : factorial_f(n) * sqrt(a[n] * a[n] + b[n] * b[n]);
            knl[n] = fabs(knl[n]);
            tl[n] = 0;
          }
          double bend_factor = knl[0] / ele->l;
          double radius0 = ele->r0_mag;
          if (radius0 == 0) radius0 = 0.01;
          double quad_factor = 0;
          if (ele->key == BGO_SBEND) {
            bend_factor = bend_factor + fmax(fabs(ele->g), fabs(ele->g + ele->dg));
            quad_factor = knl[1] + knl[2] * radius0 + ele->l * sq(bend_factor);
          } else if (ele->key == BGO_QUADRUPOLE) {
            quad_factor = 50 * (knl[1] + ele->l * sq(bend_factor));
          } else {
            quad_factor = knl[2] * radius0 + ele->l * sq(bend_factor);
          }
          if (ele->has_elec_poles) {
            double ae[BGO_N_POLE], be[BGO_N_POLE];
            double r0e = ele->r0_elec;
            if (r0e == 0) r0e = 0.01;
            bgo_multipole_ele_to_ab(ele, 0, 1, 0, ae, be, NULL);
            bend_factor = bend_factor + (fabs(ae[0]) + fabs(be[0])) / ele->p0c;
            quad_factor = quad_factor + (fabs(ae[1]) + fabs(be[1]) + r0e * (fabs(ae[2]) + fabs(be[2]))) / ele->p0c;
          }
          int ixm = check_bend(ele->l, quad_factor, bend_factor, 1e-8, gf);
          if (ixm > 4) ixm = 4;
          int ns = nint_f(gf[ixm + 1]);
          ele->num_steps = ns > 1 ? ns : 1;
          ele->ds_step = fabs(ele->l) / ele->num_steps;
          (void)tl;
        }
        break;
      case BGO_KICKER: case BGO_HKICKER: case BGO_VKICKER:
        if (ele->l != 0) {
          double gf[8];
          double km = (ele->key == BGO_KICKER) ? sqrt(sq(ele->hkick) + sq(ele->vkick)) / ele->l : ele->kick / ele->l;
          int ixm = check_bend(ele->l, 0.0, km, 1e-8, gf);
          int ns = nint_f(gf[ixm + 1]);
          ele->num_steps = ns > 1 ? ns : 1;
          ele->ds_step = fabs(ele->l) / ele->num_steps;
        }
        break;
      default:
        break;
    }
  }
  if (ele->ds_step <= 0) {
    if (ele->num_steps <= 0 || fabs(ele->l) == 0) {
      ele->ds_step = 0.2; /* bmad_com%default_ds_step */
    } else {
      ele->ds_step = fabs(ele->l) / ele->num_steps;
    }
  }
  {
    int ns = nint_f(fabs(ele->l / ele->ds_step));
    ele->num_steps = ns > 1 ? ns : 1;
  }
  return 0;
}

/* ------------------------------------------------------------------ */
/* multipole_ele_to_ab, bmad/code/multipole_ele_to_ab.f90:31-678       */

/* tilt_this_multipole, multipole_ele_to_ab.f90:436-457 */
static void tilt_this_multipole(const bgo_ele* ele, int sgn, double* a, double* b, int ix_pole_max) {
  double tilt = (ele->key == BGO_SBEND) ? sgn * ele->ref_tilt : sgn * ele->tilt;
  if (tilt == 0) return;
  for (int n = 0; n <= ix_pole_max; n++) {
    if (a[n] == 0 && b[n] == 0) continue;
    double an = a[n], bn = b[n];
    double cos_t = cos((n + 1) * tilt);
    double sin_t = sin((n + 1) * tilt);
    b[n] = bn * cos_t + an * sin_t;
    a[n] = -bn * sin_t + an * cos_t;
  }
}

/* convert_this_ab, multipole_ele_to_ab.f90:463-575 (non-slave, so the
 * relative tilt is zero) */
static int convert_this_ab(const bgo_ele* ele, int electric, const double* a_pole, const double* b_pole, double* a,
                           double* b) {
  for (int n = 0; n < BGO_N_POLE; n++) {
    a[n] = a_pole[n];
    b[n] = b_pole[n];
  }
  int ix_max = max_nonzero2(a, b, BGO_N_POLE);
  if (ix_max < 0) return 0;
  /* field_master scaling (field_master = F for all inputs here) */
  if (!ele->scale_multipoles) return 0;
  if (electric) {
    double radius = ele->r0_elec;
    if (radius != 0 && radius != 1) {
      double factor = radius;
      for (int n = 0; n < BGO_N_POLE; n++) {
        factor = factor / radius;
        a[n] = factor * a[n];
        b[n] = factor * b[n];
      }
    }
    return 0;
  }
  double cnst = 0;
  int ref_exp = 0;
  switch (ele->key) {
    case BGO_SBEND:
      cnst = ele->l * (ele->g + ele->dg);
      ref_exp = 0;
      break;
    case BGO_KICKER:
      if (ele->hkick == 0) cnst = ele->vkick;
      else if (ele->vkick == 0) cnst = ele->hkick;
      else cnst = sqrt(sq(ele->hkick) + sq(ele->vkick));
      ref_exp = 0;
      break;
    case BGO_HKICKER: case BGO_VKICKER:
      cnst = ele->kick;
      ref_exp = 0;
      break;
    case BGO_QUADRUPOLE:
      cnst = ele->k1 * ele->l;
      ref_exp = 1;
      break;
    case BGO_SEXTUPOLE:
      cnst = ele->k2 * ele->l;
      ref_exp = 2;
      break;
    case BGO_OCTUPOLE:
      cnst = ele->k3 * ele->l;
      ref_exp = 3;
      break;
    case BGO_AB_MULTIPOLE: case BGO_THICK_MULTIPOLE: case BGO_RFCAVITY:
      return 0;
    default:
      return -1; /* CONFUSION! TRYING TO SCALE NON-SCALABLE ELEMENT */
  }
  double radius = ele->r0_mag;
  if (radius == 0) {
    for (int n = 0; n < BGO_N_POLE; n++) {
      a[n] = cnst * a[n];
      b[n] = cnst * b[n];
    }
  } else {
    double factor = cnst * powi_f(radius, ref_exp + 1);
    for (int n = 0; n < BGO_N_POLE; n++) {
      factor = factor / radius;
      a[n] = factor * a[n];
      b[n] = factor * b[n];
    }
  }
  return 0;
}

static int has_hkick_attributes(int key) {
  switch (key) {
    case BGO_QUADRUPOLE: case BGO_SBEND: case BGO_SEXTUPOLE: case BGO_OCTUPOLE: case BGO_THICK_MULTIPOLE:
    case BGO_RFCAVITY: case BGO_ECOLLIMATOR: case BGO_RCOLLIMATOR: case BGO_INSTRUMENT: case BGO_MONITOR:
    case BGO_PIPE: case BGO_KICKER:
      return 1;
    default:
      return 0;
  }
}

/* this_ele_non_multipoles, multipole_ele_to_ab.f90:324-410 */
static void this_ele_non_multipoles(const bgo_ele* ele, int electric, double a_kick[4], double b_kick[4]) {
  for (int i = 0; i < 4; i++) a_kick[i] = b_kick[i] = 0;
  if (electric) return; /* elseparator only */
  switch (ele->key) {
    case BGO_HKICKER:
      b_kick[0] = -ele->kick;
      break;
    case BGO_VKICKER:
      a_kick[0] = ele->kick;
      break;
    case BGO_KICKER:
      b_kick[0] = -ele->hkick;
      a_kick[0] = ele->vkick;
      break;
    default: {
      double hk = ele->hkick, vk = ele->vkick;
      if (has_hkick_attributes(ele->key) && (hk != 0 || vk != 0)) {
        double tilt = (ele->key == BGO_SBEND) ? ele->ref_tilt : ele->tilt;
        if (tilt != 0) {
          double cos_t = cos(tilt), sin_t = sin(tilt);
          b_kick[0] = -hk * cos_t - vk * sin_t;
          a_kick[0] = -hk * sin_t + vk * cos_t;
        } else {
          b_kick[0] = -hk;
          a_kick[0] = vk;
        }
      }
    }
  }
  switch (ele->key) {
    case BGO_QUADRUPOLE:
      b_kick[1] = ele->k1 * ele->l;
      break;
    case BGO_SBEND:
      b_kick[0] = b_kick[0] + ele->dg * ele->l;
      b_kick[1] = ele->k1 * ele->l;
      b_kick[2] = ele->k2 * ele->l / 2.0;
      break;
    case BGO_SEXTUPOLE:
      b_kick[2] = ele->k2 * ele->l / 2.0;
      break;
    case BGO_OCTUPOLE:
      b_kick[3] = ele->k3 * ele->l / 6.0;
      break;
    default:
      break;
  }
}

/* pull_this_b1, multipole_ele_to_ab.f90:660-676 */
static double pull_this_b1(double* a, double* b, int* ix_pole_max) {
  double b1 = b[1];
  b[1] = 0;
  if (*ix_pole_max > 1) return b1;
  *ix_pole_max = max_nonzero2(a, b, 2);
  return b1;
}

/* multipole1_kt_to_ab, bmad/low_level/multipole1_kt_to_ab.f90 */
static void multipole1_kt_to_ab(double knl, double knsl, double tn, int n, double* an, double* bn) {
  if (knl == 0 && knsl == 0) {
    *bn = 0;
    *an = 0;
  } else {
    double angle = -tn * (n + 1);
    *bn = (knl * cos(angle) - knsl * sin(angle)) / factorial_f(n);
    *an = (knl * sin(angle) + knsl * cos(angle)) / factorial_f(n);
  }
}

/* multipole1_ab_to_kt, bmad/low_level/multipole1_ab_to_kt.f90 */
static void multipole1_ab_to_kt(double an, double bn, int n, double* knl, double* tn) {
  if (an == 0 && bn == 0) {
    *knl = 0;
    *tn = 0;
  } else {
    double a = an, b = bn;
    *knl = factorial_f(n) * sqrt(a * a + b * b);
    *tn = -atan2(a, b) / (n + 1);
    if (2 * (n + 1) * fabs(*tn) > PI) {
      *knl = -*knl;
      *tn = sign_of(*tn) * (fabs(*tn) - PI / (n + 1));
    }
  }
}

/* Returns ix_pole_max (>= -1) or -2 on error. */
int bgo_multipole_ele_to_ab(const bgo_ele* ele, int use_ele_tilt, int electric, int include_kicks, double* a,
                            double* b, double* b1) {
  c_multi_init();
  for (int n = 0; n < BGO_N_POLE; n++) a[n] = b[n] = 0;
  if (b1) *b1 = 0;
  int ix_pole_max = -1;
  if (!ele->is_on || ele->key == BGO_PIPE) return -1;

  if (ele->key == BGO_MULTIPOLE) {
    if (electric || !ele->has_mag_poles) return -1;
    for (int n = 0; n < BGO_N_POLE; n++)
      multipole1_kt_to_ab(ele->a_pole[n], ele->ksl_pole[n], ele->b_pole[n], n, &a[n], &b[n]);
    ix_pole_max = max_nonzero2(a, b, BGO_N_POLE);
    if (b1) *b1 = pull_this_b1(a, b, &ix_pole_max);
    return ix_pole_max;
  }

  int has_poles = electric ? ele->has_elec_poles : ele->has_mag_poles;
  if (has_poles) {
    int rc = convert_this_ab(ele, electric, electric ? ele->a_pole_elec : ele->a_pole,
                             electric ? ele->b_pole_elec : ele->b_pole, a, b);
    if (rc) return -2;
  }
  double a_kick[4], b_kick[4];
  this_ele_non_multipoles(ele, electric, a_kick, b_kick);
  if (include_kicks) {
    for (int i = 0; i < 4; i++) {
      a[i] = a[i] + a_kick[i];
      b[i] = b[i] + b_kick[i];
    }
  }
  ix_pole_max = max_nonzero2(a, b, BGO_N_POLE);
  if (use_ele_tilt) tilt_this_multipole(ele, +1, a, b, ix_pole_max);
  if (b1) *b1 = pull_this_b1(a, b, &ix_pole_max);
  return ix_pole_max;
}

/* multipole_ele_to_kt, bmad/code/multipole_ele_to_kt.f90:29-95 (magnetic) */
int bgo_multipole_ele_to_kt(const bgo_ele* ele, int use_ele_tilt, double* knl, double* tilt) {
  if (ele->key == BGO_MULTIPOLE) {
    int all_zero = 1;
    for (int n = 0; n < BGO_N_POLE; n++)
      if (ele->ksl_pole[n] != 0) all_zero = 0;
    if (!ele->has_mag_poles) {
      for (int n = 0; n < BGO_N_POLE; n++) knl[n] = tilt[n] = 0;
    } else if (all_zero) {
      for (int n = 0; n < BGO_N_POLE; n++) {
        knl[n] = ele->a_pole[n];
        tilt[n] = ele->b_pole[n] + ele->tilt;
      }
    } else {
      for (int n = 0; n < BGO_N_POLE; n++) {
        knl[n] = sqrt(sq(ele->a_pole[n]) + sq(ele->ksl_pole[n]));
        tilt[n] = ele->b_pole[n] - atan2(ele->ksl_pole[n], ele->a_pole[n]) / (n + 1);
        if (2 * (n + 1) * fabs(tilt[n]) > PI) {
          knl[n] = -knl[n];
          tilt[n] = sign_of(tilt[n]) * (fabs(tilt[n]) - PI / (n + 1));
        }
      }
    }
    return max_nonzero2(knl, NULL, BGO_N_POLE);
  }
  double a[BGO_N_POLE], b[BGO_N_POLE];
  int ix = bgo_multipole_ele_to_ab(ele, use_ele_tilt, 0, 0, a, b, NULL);
  if (ix > -1) {
    for (int n = 0; n < BGO_N_POLE; n++) multipole1_ab_to_kt(a[n], b[n], n, &knl[n], &tilt[n]);
  } else {
    for (int n = 0; n < BGO_N_POLE; n++) knl[n] = tilt[n] = 0;
  }
  return ix;
}

/* ------------------------------------------------------------------ */
/* Kicks: bmad/modules/multipole_mod.f90                               */

/* ab_multipole_kick, multipole_mod.f90:314-401 (no dk).  ele_orientation
 * = 0 selects the "ignore orientation" form used by track_a_bend. */
static void ab_multipole_kick(double a, double b, int n, int ele_orientation, const bgo_coord* coord,
                              const bgo_param* param, int electric, const double* scale, double* kx, double* ky) {
  double a2, b2, f;
  *kx = 0;
  *ky = 0;
  if (a == 0 && b == 0) return;
  if (electric) {
    f = param->charge / (coord->beta * coord->p0c);
    a2 = a * f;
    b2 = -b * f;
    FL(4);
  } else {
    if (ele_orientation == 0) {
      a2 = a;
      b2 = b;
    } else {
      /* direction * orientation * charge_to_mass / charge_to_mass = 1 */
      f = 1.0;
      a2 = a * f;
      b2 = b * f;
    }
  }
  if (scale) {
    a2 = *scale * a2;
    b2 = *scale * b2;
    FL(2);
  }
  double x = coord->vec[0], y = coord->vec[2];
  for (int m = 0; m <= n; m += 2) {
    f = bgo_c_multi(n, m, 1) * mexp(x, n - m) * mexp(y, m);
    *kx = *kx + b2 * f;
    *ky = *ky - a2 * f;
    FL(6);
  }
  for (int m = 1; m <= n; m += 2) {
    f = bgo_c_multi(n, m, 1) * mexp(x, n - m) * mexp(y, m);
    *kx = *kx + a2 * f;
    *ky = *ky + b2 * f;
    FL(6);
  }
}

/* apply_energy_kick, bmad/low_level/apply_energy_kick.f90:23-74 */
static void apply_energy_kick(double dE, bgo_coord* orbit, const bgo_param* param) {
  double mc2 = param->mass;
  double p0c = orbit->p0c;
  double pc = (1 + orbit->vec[5]) * p0c;
  double beta_old = orbit->beta;
  double E_old = pc / orbit->beta;
  double E_new = E_old + dE;
  FL(4);
  if (E_new < mc2) {
    orbit->vec[5] = -1;
    orbit->beta = 0;
    orbit->state = BGO_LOST_PZ;
    return;
  }
  orbit->vec[5] = orbit->vec[5] + (1 + orbit->vec[5]) * sqrt_one((2 * E_old * dE + dE * dE) / (pc * pc));
  double pc_new = p0c * (1 + orbit->vec[5]);
  double beta_new = pc_new / E_new;
  orbit->vec[4] = orbit->vec[4] * beta_new / beta_old;
  orbit->beta = beta_new;
  FL(14);
}

/* ab_multipole_kicks, multipole_mod.f90:82-174 (no matrix) */
static void ab_multipole_kicks(const double* an, const double* bn, int ix_pole_max, const bgo_ele* ele,
                               bgo_coord* orbit, const bgo_param* param, int electric, double scale) {
  double kx_tot = 0, ky_tot = 0, kx, ky;
  bgo_coord orb0 = *orbit;
  double r = ele->p0c / orbit->p0c;
  FL(1);
  for (int n = 0; n <= ix_pole_max; n++) {
    ab_multipole_kick(r * an[n], r * bn[n], n, 1, orbit, param, electric, &scale, &kx, &ky);
    kx_tot = kx_tot + kx;
    ky_tot = ky_tot + ky;
    FL(4);
  }
  orbit->vec[1] = orbit->vec[1] + kx_tot;
  orbit->vec[3] = orbit->vec[3] + ky_tot;
  FL(2);
  if (!electric) return;
  double alpha = (kx_tot * (2 * orb0.vec[1] + kx_tot) + ky_tot * (2 * orb0.vec[3] + ky_tot)) / sq(1 + orb0.vec[5]);
  if (alpha < -1) {
    orbit->state = BGO_LOST_PZ;
    return;
  }
  double dpz = (1 + orb0.vec[5]) * sqrt_one(alpha);
  orbit->vec[5] = orb0.vec[5] + dpz;
  orbit->beta = (1 + orbit->vec[5]) / sqrt(sq(1 + orbit->vec[5]) + sq(param->mass / orbit->p0c));
  orbit->vec[4] = orb0.vec[4] * orbit->beta / orb0.beta;
  FL(24);
}

/* multipole_kick, multipole_mod.f90:203-286 (thin, knl/tilt form) */
static void multipole_kick(double knl, double tilt, int n, bgo_coord* coord, int ref_orb_offset) {
  double x, y, sin_ang, cos_ang, xt[BGO_N_POLE], yt[BGO_N_POLE];
  if (knl == 0) return;
  c_multi_init();
  double t = tilt;
  double charge = 1.0; /* direction*time_dir*orientation*ctm/ctm */
  if (t == 0) {
    sin_ang = 0;
    cos_ang = 1;
    x = coord->vec[0];
    y = coord->vec[2];
  } else {
    sin_ang = sin(t);
    cos_ang = cos(t);
    x = coord->vec[0] * cos_ang + coord->vec[2] * sin_ang;
    y = -coord->vec[0] * sin_ang + coord->vec[2] * cos_ang;
    LM(2);
    FL(6);
  }
  if (n == 0 && ref_orb_offset) {
    coord->vec[1] = coord->vec[1] + charge * knl * cos_ang * coord->vec[5];
    coord->vec[3] = coord->vec[3] + charge * knl * sin_ang * coord->vec[5];
    coord->vec[4] = coord->vec[4] - charge * knl * (cos_ang * coord->vec[0] + sin_ang * coord->vec[2]);
    FL(16);
    return;
  }
  xt[n] = 1.0;
  yt[0] = 1.0;
  for (int m = 1; m <= n; m++) {
    xt[n - m] = xt[n - m + 1] * x;
    yt[m] = yt[m - 1] * y;
    FL(2);
  }
  double x_value = 0, y_value = 0;
  for (int m = 0; m <= n; m += 2) {
    x_value = x_value + g_cm[n][m] * xt[m] * yt[m];
    FL(3);
  }
  for (int m = 1; m <= n; m += 2) {
    y_value = y_value + g_cm[n][m] * xt[m] * yt[m];
    FL(3);
  }
  double x_vel = charge * knl * x_value;
  double y_vel = charge * knl * y_value;
  FL(4);
  if (t == 0) {
    coord->vec[1] = coord->vec[1] + x_vel;
    coord->vec[3] = coord->vec[3] + y_vel;
    FL(2);
  } else {
    coord->vec[1] = coord->vec[1] + x_vel * cos_ang - y_vel * sin_ang;
    coord->vec[3] = coord->vec[3] + x_vel * sin_ang + y_vel * cos_ang;
    FL(8);
  }
}

/* ------------------------------------------------------------------ */
/* Drift: bmad/low_level/track_a_drift.f90:25-116 (forward)             */

static void track_a_drift(bgo_coord* orb, double length, int include_ref_motion, const bgo_param* param) {
  if (length == 0) return;
  double delta = orb->vec[5];
  double rel_pc = 1 + delta;
  double px_rel = orb->vec[1] / rel_pc;
  double py_rel = orb->vec[3] / rel_pc;
  double pxy2 = px_rel * px_rel + py_rel * py_rel;
  FL(6);
  if (pxy2 >= 1) {
    orb->state = BGO_LOST_PZ;
    return;
  }
  double ps_rel = sqrt(1 - pxy2);
  orb->vec[0] = orb->vec[0] + length * px_rel / ps_rel;
  orb->vec[2] = orb->vec[2] + length * py_rel / ps_rel;
  FL(8);
  double dz;
  if (orb->beta > 0) {
    if (include_ref_motion) {
      double mc2 = param->mass;
      dz = length * (sqrt_one((mc2 * mc2 * (2 * delta + delta * delta)) / (sq(orb->p0c * rel_pc) + mc2 * mc2)) +
                     sqrt_one(-pxy2) / ps_rel);
      FL(14);
    } else {
      dz = -length / ps_rel;
      FL(2);
    }
  } else {
    if (include_ref_motion) {
      dz = length * (1 - 1 / ps_rel);
      FL(3);
    } else {
      dz = -length / ps_rel;
      FL(2);
    }
  }
  /* dt = rel_z_vel * length / (beta * ps_rel * c_light); orb%t = orb%t + dt
   * (track_a_drift.f90:79-80): a real(rp) step added to the real(qp) time
   * (time bookkeeping, not counted in the FP64 operation tally) */
  if (orb->beta > 0) {
    double dt = length / (orb->beta * ps_rel * C_LIGHT);
    orb->t = orb->t + (__float128)dt;
  }
  orb->vec[4] = orb->vec[4] + dz;
  FL(1);
}

/* orbit%t = start_orb%t + direction * time_dir * delta_ref_time +
 * (start_orb%vec(5) - orbit%vec(5)) / (orbit%beta * c_light), summed left to
 * right in real(qp) (track_a_quadrupole.f90:144, track_a_bend.f90:327,
 * track_a_thick_multipole.f90:133). */
static void element_exit_time(bgo_coord* orbit, const bgo_ele* ele, __float128 t0, double z0) {
  double dz_t = (z0 - orbit->vec[4]) / (orbit->beta * C_LIGHT);
  orbit->t = t0 + (__float128)(1 * ele->delta_ref_time) + (__float128)dz_t;
}

/* tilt_coords, bmad/code/tilt_coords.f90:18-53 */
static void tilt_coords(double tilt_val, double* v) {
  if (tilt_val == 0) return;
  double s = sin(tilt_val), c = cos(tilt_val);
  double x = v[0], y = v[2], px = v[1], py = v[3];
  v[0] = c * x + s * y;
  v[2] = -s * x + c * y;
  v[1] = c * px + s * py;
  v[3] = -s * px + c * py;
  LM(2);
  FL(12);
}

/* floor_angles_to_w_mat, bmad/geometry/floor_angles_to_w_mat.f90:17-57 (psi = 0) */
static void floor_angles_to_w_mat(double theta, double phi, double psi, double w[3][3], int inverse) {
  double s_the = sin(theta), c_the = cos(theta);
  double s_phi = sin(phi), c_phi = cos(phi);
  double s_psi = sin(psi), c_psi = cos(psi);
  if (!inverse) {
    w[0][0] = c_the * c_psi - s_the * s_phi * s_psi;
    w[0][1] = -c_the * s_psi - s_the * s_phi * c_psi;
    w[0][2] = s_the * c_phi;
    w[1][0] = c_phi * s_psi;
    w[1][1] = c_phi * c_psi;
    w[1][2] = s_phi;
    w[2][0] = -s_the * c_psi - c_the * s_phi * s_psi;
    w[2][1] = s_the * s_psi - c_the * s_phi * c_psi;
    w[2][2] = c_the * c_phi;
  } else {
    w[0][0] = c_the * c_psi - s_the * s_phi * s_psi;
    w[0][1] = c_phi * s_psi;
    w[0][2] = -s_the * c_psi - c_the * s_phi * s_psi;
    w[1][0] = -c_the * s_psi - s_the * s_phi * c_psi;
    w[1][1] = c_phi * c_psi;
    w[1][2] = s_the * s_psi - c_the * s_phi * c_psi;
    w[2][0] = s_the * c_phi;
    w[2][1] = s_phi;
    w[2][2] = c_the * c_phi;
  }
}

static void matvec3(double w[3][3], const double r[3], double out[3]) {
  for (int i = 0; i < 3; i++) {
    double s = 0;
    for (int k = 0; k < 3; k++) s = s + w[i][k] * r[k];
    out[i] = s;
  }
}

/* ------------------------------------------------------------------ */
/* Bend geometry of offset_particle (offset_particle.f90:208-235 set,
 * :393-425 unset).  Element constants (angles, tilts) use the C library. */

enum { AX_X = 0, AX_Y = 1, AX_Z = 2 };

typedef struct {
  double r[3];
  double w[3][3];
} bgo_pos;

/* sim_utils/special_functions/cos_one.f90:16-26 */
static double cos_one(double angle) {
  double s = sin(angle / 2);
  return -(2 * (s * s));
}

/* rotate_vec, sim_utils/math/rotation_3d_mod.f90:737-760 */
static void rotate_vec(double v[3], int axis, double angle) {
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

/* rotate_mat without right_multiply (mat = Rot . mat),
 * sim_utils/math/rotation_3d_mod.f90:781-835: each column as rotate_vec */
static void rotate_mat(double m[3][3], int axis, double angle) {
  if (angle == 0) return;
  for (int j = 0; j < 3; j++) {
    double v[3] = {m[0][j], m[1][j], m[2][j]};
    rotate_vec(v, axis, angle);
    m[0][j] = v[0];
    m[1][j] = v[1];
    m[2][j] = v[2];
  }
}

/* matmul of 3x3 matrices (k-ordered sums, as gfortran's inline matmul) */
static void matmul33(double a[3][3], double b[3][3], double out[3][3]) {
  double t[3][3];
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) {
      double s = 0;
      for (int k = 0; k < 3; k++) s = s + a[i][k] * b[k][j];
      t[i][j] = s;
    }
  memcpy(out, t, sizeof(t));
}

/* w_mat_for_tilt, bmad/geometry/w_mat_for_tilt.f90:13-40 (not inverse) */
static void w_mat_for_tilt(double tilt, double w[3][3]) {
  double c = cos(tilt), s = sin(tilt);
  double t[3][3] = {{c, -s, 0.0}, {s, c, 0.0}, {0.0, 0.0, 1.0}};
  memcpy(w, t, sizeof(t));
}

static void pos_apply(bgo_pos* p, double m[3][3]) {
  double r[3];
  matvec3(m, p->r, r);
  memcpy(p->r, r, sizeof(r));
  matmul33(m, p->w, p->w);
}

/* bend_shift, bmad/geometry/bend_shift.f90:19-61; has_tilt says whether
 * the optional ref_tilt argument is present. */
static void bend_shift(bgo_pos* p, double g, double delta_s, int has_tilt, double ref_tilt) {
  double angle = delta_s * g;
  if (angle == 0) {
    p->r[2] = p->r[2] - delta_s;
    return;
  }
  double tlt = has_tilt ? ref_tilt : 0.0;
  double S[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
  if (tlt != 0) {
    rotate_mat(S, AX_Z, -ref_tilt);
    rotate_mat(S, AX_Y, angle);
    rotate_mat(S, AX_Z, ref_tilt);
  } else {
    rotate_mat(S, AX_Y, angle);
  }
  double L[3] = {cos_one(angle) / g, 0.0 / g, -sin(angle) / g};
  if (has_tilt) rotate_vec(L, AX_Z, ref_tilt);
  double r[3];
  matvec3(S, p->r, r);
  for (int i = 0; i < 3; i++) p->r[i] = r[i] + L[i];
  matmul33(S, p->w, p->w);
}

/* bend_shift for a particle-dependent arc length (the s_pos form of the bend
 * geometry): the same operations, with the rotation by the particle's angle
 * taken through the particle transcendentals (P_SIN / P_COS); ref_tilt
 * rotations, element constants, through the C library. */
static void bend_shift_particle(bgo_pos* p, double g, double delta_s, int has_tilt, double ref_tilt) {
  double angle = delta_s * g;
  if (angle == 0) {
    p->r[2] = p->r[2] - delta_s;
    return;
  }
  double tlt = has_tilt ? ref_tilt : 0.0;
  double S[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
  if (tlt != 0) rotate_mat(S, AX_Z, -ref_tilt);
  double ca = P_COS(angle), sa = P_SIN(angle);
  for (int j = 0; j < 3; j++) { /* rotate_mat(S, AX_Y, angle), each column as rotate_vec */
    double a = sa * S[2][j] + ca * S[0][j];
    double b = ca * S[2][j] - sa * S[0][j];
    S[0][j] = a;
    S[2][j] = b;
  }
  if (tlt != 0) rotate_mat(S, AX_Z, ref_tilt);
  double sh = P_SIN(angle / 2);
  double L[3] = {-(2 * (sh * sh)) / g, 0.0 / g, -sa / g};
  if (has_tilt) rotate_vec(L, AX_Z, ref_tilt);
  double r[3];
  matvec3(S, p->r, r);
  for (int i = 0; i < 3; i++) p->r[i] = r[i] + L[i];
  matmul33(S, p->w, p->w);
}

/* ele_misalignment_L_S_calc, bmad/geometry/ele_misalignment_L_S_calc.f90:
 * 16-50, sbend branch (angle = g L, rho = 1/g as the bookkeeper sets them) */
static void bend_misalignment_L_S(const bgo_ele* ele, double L_mis[3], double S[3][3]) {
  L_mis[0] = ele->x_offset;
  L_mis[1] = ele->y_offset;
  L_mis[2] = ele->z_offset;
  if (ele->roll != 0) {
    double angle = ele->g * ele->l;
    double rho = ele->g == 0 ? 0.0 : 1 / ele->g;
    double Lc[3] = {rho * cos_one(angle / 2), rho * 0.0, rho * sin(angle / 2)};
    rotate_vec(Lc, AX_Y, angle / 2);
    rotate_vec(Lc, AX_Z, ele->ref_tilt);
    for (int i = 0; i < 3; i++) L_mis[i] = L_mis[i] - Lc[i];
    rotate_vec(Lc, AX_Z, ele->roll);
    for (int i = 0; i < 3; i++) L_mis[i] = L_mis[i] + Lc[i];
  }
  floor_angles_to_w_mat(ele->x_pitch, ele->y_pitch, ele->roll, S, 0);
}

/* The bend branch of offset_particle for a misaligned bend with g, ref_tilt
 * or roll nonzero: (x, y) -> position (r, w) in the body frame (set) or the
 * lab frame (unset).  drift_to = 0: s_pos given, no drift (rho*atan2 form). */
static void bend_offset_position(const bgo_ele* ele, int set, int drift_to, double ds_center, double L_half,
                                 double x, double y, bgo_pos* pos) {
  const double g = ele->g, ref_tilt = ele->ref_tilt;
  double L_mis[3], ws[3][3], wt[3][3];
  pos->r[0] = x;
  pos->r[1] = y;
  pos->r[2] = 0.0;
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) pos->w[i][j] = (i == j) ? 1.0 : 0.0;
  if (set) {
    bend_shift(pos, g, 1 * ds_center, 1, ref_tilt);
    bend_misalignment_L_S(ele, L_mis, ws);
    for (int i = 0; i < 3; i++)
      for (int j = 0; j < 3; j++) wt[i][j] = ws[j][i];
    for (int i = 0; i < 3; i++) pos->r[i] = pos->r[i] - L_mis[i];
    pos_apply(pos, wt);
    if (ref_tilt != 0) {
      bend_shift(pos, g, -L_half, 1, ref_tilt);
      w_mat_for_tilt(-ref_tilt, ws);
      pos_apply(pos, ws);
      bend_shift(pos, g, L_half, 0, 0.0);
    }
    if (drift_to != 0) {
      bend_shift(pos, g, -1 * 1 * L_half, 0, 0.0);
      pos->r[2] = pos->r[2] + (1 - 1 * 1) * L_half;
    } else {
      double ds = (g == 0) ? -1 * ds_center : (1 / g) * P_ATAN2(pos->r[2] * g, 1.0 + pos->r[0] * g);
      bend_shift_particle(pos, g, ds, 0, 0.0);
      pos->r[2] = pos->r[2] + L_half + ds;
    }
  } else {
    bend_shift(pos, g, ds_center, 0, 0.0);
    if (ref_tilt != 0) {
      bend_shift(pos, g, -L_half, 0, 0.0);
      w_mat_for_tilt(ref_tilt, ws);
      pos_apply(pos, ws);
      bend_shift(pos, g, L_half, 1, ref_tilt);
    }
    bend_misalignment_L_S(ele, L_mis, ws);
    pos_apply(pos, ws);
    for (int i = 0; i < 3; i++) pos->r[i] = pos->r[i] + L_mis[i];
    if (drift_to != 0) {
      bend_shift(pos, g, 1 * 1 * L_half, 1, ref_tilt);
      pos->r[2] = pos->r[2] + (1 + 1 * 1) * L_half;
    } else {
      double ds = (g == 0) ? -ds_center : (1 / g) * P_ATAN2(pos->r[2] * g, 1.0 + pos->r[0] * g);
      bend_shift_particle(pos, g, ds, 1, ref_tilt);
      pos->r[2] = pos->r[2] + L_half + ds;
    }
  }
}

/* offset_particle, bmad/code/offset_particle.f90:66-530, forward tracking.
 * s_pos_mode: 0 = normal (drift to the edge), 1 = s_pos given (no drift),
 * with s_pos the lab (set) / body (unset) position.  s_out (may be NULL):
 * the edge drifted to, or the body (set) / lab (unset) position (:334-336,
 * :486-492). */
static void offset_particle_s(const bgo_ele* ele, int set, bgo_coord* orbit, int set_tilt, int set_hvkicks,
                              int s_pos_mode, double s_pos, const bgo_param* param, double* s_out) {
  double length = ele->l;
  double L_half = 0.5 * length;
  int has_orient = !(ele->key == BGO_MULTIPOLE && 0); /* all path elements carry orientation attributes */
  int drift_to; /* 0 = no, 1 = upstream, 2 = downstream */
  if (!has_orient) drift_to = 0;
  else if (s_pos_mode) drift_to = 0;
  else if (set) drift_to = 1;
  else drift_to = 2;

  double s_pos0;
  if (s_pos_mode) s_pos0 = s_pos;
  else if (set) s_pos0 = 0;
  else s_pos0 = length;
  double ds_center = L_half - s_pos0;
  double s_target = (drift_to == 1) ? (1 - 1) * L_half : (1 + 1) * L_half;

  double rel_p = 1 + orbit->vec[5];
  int set_hv = set_hvkicks && ele->is_on && has_hkick_attributes(ele->key);
  int set_hv1 = set_hv && !(ele->key == BGO_KICKER || ele->key == BGO_HKICKER || ele->key == BGO_VKICKER);
  int set_hv2 = set_hv && !set_hv1;
  double charge_dir = 1.0;
  int set_t = set_tilt;
  int key = ele->key;
  int is_misaligned = (ele->x_offset != 0 || ele->y_offset != 0 || ele->z_offset != 0 || ele->x_pitch != 0 ||
                       ele->y_pitch != 0 || (key == BGO_SBEND && ele->roll != 0));
  double w[3][3], r[3], r2[3];

  if (set) {
    double s_body;
    if (is_misaligned) {
      if (key == BGO_SBEND && (ele->g != 0 || ele->ref_tilt != 0 || ele->roll != 0)) {
        bgo_pos pos;
        bend_offset_position(ele, 1, drift_to, ds_center, L_half, orbit->vec[0], orbit->vec[2], &pos);
        memcpy(r2, pos.r, sizeof(r2));
        memcpy(w, pos.w, sizeof(w));
      } else {
        r[0] = orbit->vec[0] - ele->x_offset;
        r[1] = orbit->vec[2] - ele->y_offset;
        r[2] = 0.0 - (ele->z_offset + 1 * ds_center);
        floor_angles_to_w_mat(ele->x_pitch, ele->y_pitch, 0.0, w, 1);
        matvec3(w, r, r2);
        r2[2] = r2[2] + L_half;
      }
      s_body = r2[2];
      double pz = rel_p * rel_p - orbit->vec[1] * orbit->vec[1] - orbit->vec[3] * orbit->vec[3];
      if (pz <= 0) {
        orbit->state = BGO_LOST_PZ;
      } else {
        double p0[3] = {orbit->vec[1], orbit->vec[3], 1 * sqrt(pz)}, p1[3];
        matvec3(w, p0, p1);
        orbit->vec[1] = p1[0];
        orbit->vec[3] = p1[1];
        orbit->vec[0] = r2[0];
        orbit->vec[2] = r2[1];
      }
    } else {
      if (key == BGO_SBEND && ele->ref_tilt != 0) tilt_coords(ele->ref_tilt, orbit->vec);
      s_body = s_pos0;
    }
    double ds = s_target - s_body;
    if (fabs(ds) > 1e-14 && drift_to != 0 && orbit->state == BGO_ALIVE) track_a_drift(orbit, ds, 0, param);
    if (s_out) *s_out = drift_to != 0 ? s_target : s_body;
    if (set_hv1) {
      orbit->vec[1] = orbit->vec[1] + 0.5 * charge_dir * ele->hkick;
      orbit->vec[3] = orbit->vec[3] + 0.5 * charge_dir * ele->vkick;
    }
    if (set_t && key != BGO_SBEND && ele->tilt != 0) tilt_coords(ele->tilt, orbit->vec);
    if (set_hv2) {
      if (key == BGO_HKICKER) {
        orbit->vec[1] = orbit->vec[1] + 0.5 * charge_dir * ele->kick;
      } else if (key == BGO_VKICKER) {
        orbit->vec[3] = orbit->vec[3] + 0.5 * charge_dir * ele->kick;
      } else {
        orbit->vec[1] = orbit->vec[1] + 0.5 * charge_dir * ele->hkick;
        orbit->vec[3] = orbit->vec[3] + 0.5 * charge_dir * ele->vkick;
      }
    }
  } else {
    if (set_hv2) {
      if (key == BGO_HKICKER) {
        orbit->vec[1] = orbit->vec[1] + 0.5 * charge_dir * ele->kick;
      } else if (key == BGO_VKICKER) {
        orbit->vec[3] = orbit->vec[3] + 0.5 * charge_dir * ele->kick;
      } else {
        orbit->vec[1] = orbit->vec[1] + 0.5 * charge_dir * ele->hkick;
        orbit->vec[3] = orbit->vec[3] + 0.5 * charge_dir * ele->vkick;
      }
    }
    if (set_t && key != BGO_SBEND) tilt_coords(-ele->tilt, orbit->vec);
    if (set_hv1) {
      orbit->vec[1] = orbit->vec[1] + 0.5 * charge_dir * ele->hkick;
      orbit->vec[3] = orbit->vec[3] + 0.5 * charge_dir * ele->vkick;
    }
    double s_lab;
    if (is_misaligned) {
      if (key == BGO_SBEND && (ele->g != 0 || ele->ref_tilt != 0 || ele->roll != 0)) {
        bgo_pos pos;
        bend_offset_position(ele, 0, drift_to, ds_center, L_half, orbit->vec[0], orbit->vec[2], &pos);
        memcpy(r2, pos.r, sizeof(r2));
        memcpy(w, pos.w, sizeof(w));
      } else {
        r[0] = orbit->vec[0];
        r[1] = orbit->vec[2];
        r[2] = 0.0;
        r[2] = r[2] - ds_center;
        floor_angles_to_w_mat(ele->x_pitch, ele->y_pitch, 0.0, w, 0);
        matvec3(w, r, r2);
        r2[0] = r2[0] + ele->x_offset;
        r2[1] = r2[1] + ele->y_offset;
        r2[2] = r2[2] + (ele->z_offset + L_half);
      }
      s_lab = r2[2];
      double pz = rel_p * rel_p - orbit->vec[1] * orbit->vec[1] - orbit->vec[3] * orbit->vec[3];
      if (pz <= 0) {
        orbit->state = BGO_LOST_PZ;
      } else {
        double p0[3] = {orbit->vec[1], orbit->vec[3], 1 * sqrt(pz)}, p1[3];
        matvec3(w, p0, p1);
        orbit->vec[1] = p1[0];
        orbit->vec[3] = p1[1];
        orbit->vec[0] = r2[0];
        orbit->vec[2] = r2[1];
      }
    } else {
      if (key == BGO_SBEND && ele->ref_tilt != 0) tilt_coords(-ele->ref_tilt, orbit->vec);
      s_lab = s_pos0;
    }
    double ds = s_target - s_lab;
    if (fabs(ds) > 1e-14 && drift_to != 0 && orbit->state == BGO_ALIVE) track_a_drift(orbit, ds, 0, param);
    if (s_out) *s_out = drift_to != 0 ? s_target : s_lab;
  }
}

static void offset_particle(const bgo_ele* ele, int set, bgo_coord* orbit, int set_tilt, int set_hvkicks,
                            int s_pos_mode, double s_pos, const bgo_param* param) {
  offset_particle_s(ele, set, orbit, set_tilt, set_hvkicks, s_pos_mode, s_pos, param, NULL);
}

/* offset_particle(ele, set$ or unset$, orbit) with its default tilt and hv
 * kicks; drift_to_edge = no$ with s_pos when s_pos_mode is 1 (the form the
 * reference's coord_test exercises).  Test entry point. */
void bgo_offset_particle(const bgo_ele* ele, int set, bgo_coord* orb, int s_pos_mode, double s_pos,
                         const bgo_param* param, double* s_out) {
  offset_particle_s(ele, set, orb, 1, 1, s_pos_mode, s_pos, param, s_out);
}

/* ------------------------------------------------------------------ */
/* Apertures                                                           */

/* orbit_too_large, bmad/low_level/orbit_too_large.f90:26-120 */
int bgo_orbit_too_large(bgo_coord* orbit, bgo_param* param) {
  double mal = param->max_aperture_limit;
  if (orbit->vec[0] > mal) {
    orbit->state = BGO_LOST_POS_X;
    param->unstable_factor = (fabs(orbit->vec[0]) - mal) / mal;
    return 1;
  } else if (-orbit->vec[0] > mal) {
    orbit->state = BGO_LOST_NEG_X;
    param->unstable_factor = (fabs(orbit->vec[0]) - mal) / mal;
    return 1;
  }
  if (orbit->vec[2] > mal) {
    orbit->state = BGO_LOST_POS_Y;
    param->unstable_factor = (fabs(orbit->vec[2]) - mal) / mal;
    return 1;
  } else if (-orbit->vec[2] > mal) {
    orbit->state = BGO_LOST_NEG_Y;
    param->unstable_factor = (fabs(orbit->vec[2]) - mal) / mal;
    return 1;
  }
  double rel_p = 1 + orbit->vec[5];
  if (rel_p < 0) {
    orbit->state = BGO_LOST_PZ;
    param->unstable_factor = fabs(rel_p) + 1e-6;
    return 1;
  }
  double f_unstable = orbit->vec[1] * orbit->vec[1] + orbit->vec[3] * orbit->vec[3] - rel_p * rel_p;
  FL(6);
  if (f_unstable > 0) {
    param->unstable_factor = sqrt(f_unstable);
    if (fabs(orbit->vec[1]) > fabs(orbit->vec[3])) {
      orbit->state = orbit->vec[1] > 0 ? BGO_LOST_POS_X : BGO_LOST_NEG_X;
    } else {
      orbit->state = orbit->vec[3] > 0 ? BGO_LOST_POS_Y : BGO_LOST_NEG_Y;
    }
    return 1;
  }
  return 0;
}

/* check_this_limit, check_aperture_limit.f90:325-337 */
static void check_this_limit(bgo_coord* orbit, double coord, double width2, double center, double* uf) {
  if (width2 == 0) return;
  if (coord > center - width2 && coord < center + width2) return;
  orbit->state = BGO_LOST;
  *uf = fmax((center - width2) - coord, coord - (center + width2));
}

/* elliptical_params_setup, check_aperture_limit.f90:341-365 */
static int elliptical_params_setup(double lim1, double lim2, double* pos, double* width2, double* center,
                                   const bgo_param* param) {
  if ((lim1 == 0 && lim2 != 0) || (lim1 != 0 && lim2 == 0)) return 1;
  *width2 = (lim2 - lim1) / 2;
  *center = (lim2 + lim1) / 2;
  *pos = *pos - *center;
  if (*width2 == 0) *width2 = param->max_aperture_limit;
  *width2 = fmax(*width2, 0.0);
  return 0;
}

/* check_aperture_limit, bmad/low_level/check_aperture_limit.f90:30-372
 * (no lords, custom, wall3d or wall_transition apertures). */
void bgo_check_aperture_limit(bgo_coord* orb, const bgo_ele* ele, int at_exit, bgo_param* param) {
  double uf = 0, r, x0, y0, xw2, yw2;
  param->unstable_factor = 0;
  if (bgo_orbit_too_large(orb, param)) return;
  if (!param->aperture_limit_on) return;
  int physical_end = at_exit ? BGO_EXIT_END : BGO_ENTRANCE_END;
  int here = 0;
  if (ele->aperture_at == BGO_BOTH_ENDS) here = 1;
  else if (ele->aperture_at == physical_end) here = 1;
  if (!here) return;

  if (ele->key == BGO_ECOLLIMATOR) {
    xw2 = ele->px_aperture_width2;
    yw2 = ele->py_aperture_width2;
    x0 = ele->px_aperture_center;
    y0 = ele->py_aperture_center;
    if (xw2 == 0 || yw2 == 0) {
      check_this_limit(orb, orb->vec[1], xw2, x0, &uf);
      check_this_limit(orb, orb->vec[3], yw2, y0, &uf);
    } else {
      r = sq((orb->vec[1] - x0) / xw2) + sq((orb->vec[3] - y0) / yw2);
      if (r > 1) {
        orb->state = BGO_LOST;
        uf = sqrt(r) - 1;
      }
    }
    xw2 = ele->z_aperture_width2;
    yw2 = ele->pz_aperture_width2;
    x0 = ele->z_aperture_center;
    y0 = ele->pz_aperture_center;
    if (xw2 == 0 || yw2 == 0) {
      check_this_limit(orb, orb->vec[4], xw2, x0, &uf);
      check_this_limit(orb, orb->vec[5], yw2, y0, &uf);
    } else {
      r = sq((orb->vec[4] - x0) / xw2) + sq((orb->vec[5] - y0) / yw2);
      if (r > 1) {
        orb->state = BGO_LOST;
        uf = sqrt(r) - 1;
      }
    }
  } else if (ele->key == BGO_RCOLLIMATOR) {
    check_this_limit(orb, orb->vec[1], ele->px_aperture_width2, ele->px_aperture_center, &uf);
    check_this_limit(orb, orb->vec[3], ele->py_aperture_width2, ele->py_aperture_center, &uf);
    check_this_limit(orb, orb->vec[4], ele->z_aperture_width2, ele->z_aperture_center, &uf);
    check_this_limit(orb, orb->vec[5], ele->pz_aperture_width2, ele->pz_aperture_center, &uf);
  }

  double xp, yp;
  if (ele->offset_moves_aperture) {
    bgo_coord orb2 = *orb;
    int do_tilt = (ele->key == BGO_ECOLLIMATOR || ele->key == BGO_RCOLLIMATOR);
    double s_here = at_exit ? ele->l : 0.0;
    offset_particle(ele, 1, &orb2, do_tilt, 0, 1, s_here, param);
    xp = orb2.vec[0];
    yp = orb2.vec[2];
  } else {
    xp = orb->vec[0];
    yp = orb->vec[2];
  }

  double x1_lim = -ele->x1_limit, x2_lim = ele->x2_limit, y1_lim = -ele->y1_limit, y2_lim = ele->y2_limit;

  if (ele->aperture_type == BGO_APERTURE_ELLIPTICAL) {
    if (elliptical_params_setup(x1_lim, x2_lim, &xp, &xw2, &x0, param)) return;
    if (elliptical_params_setup(y1_lim, y2_lim, &yp, &yw2, &y0, param)) return;
    r = sq(xp / xw2) + sq(yp / yw2);
    FL(6);
    if (r < 1) {
      param->unstable_factor = uf;
      return;
    }
    if (fabs(xp / xw2) > fabs(yp / yw2)) {
      orb->state = xp > 0 ? BGO_LOST_POS_X : BGO_LOST_NEG_X;
    } else {
      orb->state = yp > 0 ? BGO_LOST_POS_Y : BGO_LOST_NEG_Y;
    }
    uf = sqrt(r) - 1;
  } else {
    double f;
    if (x1_lim != 0 && xp < x1_lim) {
      f = fabs((xp - x1_lim) / (x2_lim - x1_lim));
      if (f > uf) {
        orb->state = BGO_LOST_NEG_X;
        uf = f;
      }
    }
    if (x2_lim != 0 && xp > x2_lim) {
      f = fabs((xp - x2_lim) / (x2_lim - x1_lim));
      if (f > uf) {
        orb->state = BGO_LOST_POS_X;
        uf = f;
      }
    }
    if (y1_lim != 0 && yp < y1_lim) {
      f = fabs((yp - y1_lim) / (y2_lim - y1_lim));
      if (f > uf) {
        orb->state = BGO_LOST_NEG_Y;
        uf = f;
      }
    }
    if (y2_lim != 0 && yp > y2_lim) {
      f = fabs((yp - y2_lim) / (y2_lim - y1_lim));
      if (f > uf) {
        orb->state = BGO_LOST_POS_Y;
        uf = f;
      }
    }
  }
  param->unstable_factor = uf;
}

/* ------------------------------------------------------------------ */
/* Edge kicks                                                          */

/* hwang_bend_edge_kick, bmad/modules/fringe_mod.f90:240-418 (forward,
 * td = +1 so the backward-time re-evaluation does not apply). */
void bgo_hwang_bend_edge_kick(const bgo_ele* ele, int entering, bgo_coord* orb, const bgo_param* param) {
  (void)param;
  double c_dir = 1.0;
  double e_factor = 1 / (1 + orb->vec[5]);
  double td = 1.0;
  double g_tot, k1, e, fint_gap;
  if (ele->is_on) {
    g_tot = (ele->g + ele->dg) * c_dir;
    k1 = ele->k1;
  } else {
    g_tot = 0;
    k1 = 0;
  }
  if (entering) {
    e = ele->e1;
    fint_gap = ele->fint * ele->hgap;
  } else {
    e = ele->e2;
    fint_gap = ele->fintx * ele->hgapx;
  }
  if (ele->fringe_type == BGO_FRINGE_HARD_EDGE_ONLY || ele->fringe_type == BGO_FRINGE_SAD_FULL) fint_gap = 0;
  double cos_e = cos(e), sin_e = sin(e);
  double tan_e = sin_e / cos_e, sec_e = 1 / cos_e;
  double gt = g_tot * tan_e;
  double gt2 = g_tot * (tan_e * tan_e);
  double gs2 = g_tot * (sec_e * sec_e);
  double k1_tane = k1 * tan_e * c_dir;
  double fg_factor = 2 * fint_gap * gs2 * g_tot * sec_e * (1 + sin_e * sin_e);
  double v[6];
  for (int i = 0; i < 6; i++) v[i] = orb->vec[i];
  double dx, dpx, dy, dpy, dz;
  LM(2);
  FL(20);
  if (entering) {
    dx = (-gt2 * (v[0] * v[0]) + gs2 * (v[2] * v[2])) * e_factor / 2;
    dpx = (gt * g_tot * (1 + 2 * (tan_e * tan_e)) * (v[2] * v[2]) / 2 + gt2 * (v[0] * v[1] - v[2] * v[3]) +
           k1_tane * (v[0] * v[0] - v[2] * v[2])) *
          e_factor;
    dy = gt2 * v[0] * v[2] * e_factor;
    dpy = (fg_factor * v[2] - gt2 * v[0] * v[3] - (g_tot + gt2) * v[1] * v[2] - 2 * k1_tane * v[0] * v[2]) * e_factor;
    dz = (e_factor * e_factor) * 0.5 *
         ((v[2] * v[2]) * fg_factor + (v[0] * v[0] * v[0]) * (4.0 * k1_tane - gt * gt2) / 6.0 +
          0.5 * v[0] * (v[2] * v[2]) * (-4.0 * k1_tane + gt * gs2) +
          ((v[0] * v[0]) * v[1] - 2.0 * v[0] * v[2] * v[3]) * gt2 - v[1] * (v[2] * v[2]) * gs2);
  } else {
    dx = (gt2 * (v[0] * v[0]) - gs2 * (v[2] * v[2])) * e_factor / 2;
    dpx = (gt2 * (v[2] * v[3] - v[0] * v[1]) + k1_tane * (v[0] * v[0] - v[2] * v[2]) -
           gt * gt2 * (v[0] * v[0] + v[2] * v[2]) / 2) *
          e_factor;
    dy = -gt2 * v[0] * v[2] * e_factor;
    dpy = (fg_factor * v[2] + gt2 * v[0] * v[3] + (g_tot + gt2) * v[1] * v[2] + (gt * gs2 - 2 * k1_tane) * v[0] * v[2]) *
          e_factor;
    dz = (e_factor * e_factor) * 0.5 *
         ((v[2] * v[2]) * fg_factor + (v[0] * v[0] * v[0]) * (4.0 * k1_tane - gt * gt2) / 6.0 +
          0.5 * v[0] * (v[2] * v[2]) * (-4.0 * k1_tane + gt * gs2) -
          ((v[0] * v[0]) * v[1] - 2.0 * v[0] * v[2] * v[3]) * gt2 + v[1] * (v[2] * v[2]) * gs2);
  }
  FL(80);
  orb->vec[0] = v[0] + td * dx;
  orb->vec[1] = v[1] + td * (dpx + gt * v[0]);
  orb->vec[2] = v[2] + td * dy;
  orb->vec[3] = v[3] + td * (dpy - gt * v[2]);
  orb->vec[4] = v[4] + td * dz;
  FL(14);
}

/* electric_longitudinal_fringe, apply_element_edge_kick.f90:283-329 */
static void electric_longitudinal_fringe(bgo_coord* orb, const bgo_ele* ele, const double* ae, const double* be,
                                         int ix_elec_max, double at_sign, const bgo_param* param) {
  if (ele->l == 0) return;
  if (ix_elec_max < 0) return;
  double ff = at_sign * param->charge;
  double xr = 1, xi = 0, cr = orb->vec[0], ci = orb->vec[2];
  double phi = 0, Er0 = 0, Er1 = 0;
  for (int i = 0; i <= ix_elec_max; i++) {
    double xor_ = xr, xoi = xi;
    double nr = xr * cr - xi * ci;
    double ni = xr * ci + xi * cr;
    xr = nr;
    xi = ni;
    if (ae[i] == 0 && be[i] == 0) continue;
    double abr = be[i], abi = -ae[i];
    phi = phi - (abr * xr - abi * xi) / (i + 1);
    Er0 = Er0 + (abr * xor_ - abi * xoi);
    Er1 = Er1 + (-(abr * xoi + abi * xor_));
  }
  (void)Er0;
  (void)Er1;
  apply_energy_kick(-ff * phi, orb, param);
}

/* hard_multipole_edge_kick, bmad/modules/fringe_mod.f90:691-864, tracking
 * part (no matrix): the hard-edge fringe of the quadrupole (n = 1, k1) or
 * sextupole (n = 2, k2) body field; charge_dir = 1 (forward tracking of the
 * reference species).  Complex products are written out as gfortran forms
 * them: (a + ib)(c + id) = (ac - bd) + i(ad + bc). */
typedef struct {
  double re, im;
} bgo_cplx;
static bgo_cplx cmul(bgo_cplx a, bgo_cplx b) {
  bgo_cplx r = {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
  FL(6);
  return r;
}
static bgo_cplx cadd(bgo_cplx a, bgo_cplx b) {
  bgo_cplx r = {a.re + b.re, a.im + b.im};
  FL(2);
  return r;
}

static void hard_multipole_edge_kick(const bgo_ele* ele, int first_edge, bgo_coord* orb) {
  int n_max;
  if (ele->key == BGO_QUADRUPOLE || ele->key == BGO_SBEND) n_max = 1; /* fringe_mod.f90:737-738 */
  else if (ele->key == BGO_SEXTUPOLE) n_max = 2;
  else return;
  double x = orb->vec[0], y = orb->vec[2];
  bgo_cplx xy = {x, y}, poly_n1 = {1.0, 0.0}, poly = xy, poly_n2;
  double rel_p = 1 + orb->vec[5];
  double fx = 0, dfx_dx = 0, dfx_dy = 0, fy = 0, dfy_dx = 0, dfy_dy = 0;
  FL(1);
  for (int n = 1; n <= n_max; n++) {
    poly_n2 = poly_n1;
    poly_n1 = poly;
    poly = cmul(poly, xy);
    double ap = 0, bp;
    if (ele->key == BGO_QUADRUPOLE || ele->key == BGO_SBEND) {
      bp = ele->k1;
    } else {
      bp = ele->k2;
      if (n != 2) continue;
    }
    (void)poly_n2;
    bgo_cplx dpoly_dx = {(n + 1) * poly_n1.re, (n + 1) * poly_n1.im};
    bgo_cplx dpoly_dy = {-dpoly_dx.im, dpoly_dx.re}; /* i * dpoly_dx */
    double den = (4 * (n + 2)) * rel_p;
    bgo_cplx cab = {1.0 * bp / den, 1.0 * ap / den};
    if (first_edge) {
      cab.re = -cab.re;
      cab.im = -cab.im;
    }
    double cn = (double)(n + 3) / (n + 1);
    bgo_cplx xny = {x, -cn * y};
    bgo_cplx dxny_dy = {0.0, -cn};
    FL(8);
    fx = fx + cmul(cmul(cab, poly), xny).re;
    dfx_dx = dfx_dx + cmul(cab, cadd(cmul(dpoly_dx, xny), poly)).re;
    dfx_dy = dfx_dy + cmul(cab, cadd(cmul(dpoly_dy, xny), cmul(poly, dxny_dy))).re;
    xny = (bgo_cplx){y, cn * x};
    bgo_cplx dxny_dx = {0.0, cn};
    fy = fy + cmul(cmul(cab, poly), xny).re;
    dfy_dx = dfy_dx + cmul(cab, cadd(cmul(dpoly_dx, xny), cmul(poly, dxny_dx))).re;
    dfy_dy = dfy_dy + cmul(cab, cadd(cmul(dpoly_dy, xny), poly)).re;
    FL(7);
  }
  double px = orb->vec[1], py = orb->vec[3];
  double denom = (1 - dfx_dx) * (1 - dfy_dy) - dfx_dy * dfy_dx;
  orb->vec[0] = orb->vec[0] - fx;
  orb->vec[1] = px + ((1.0 - dfy_dy - denom) * px + dfy_dx * py) / denom;
  orb->vec[2] = orb->vec[2] - fy;
  orb->vec[3] = py + (dfx_dy * px + (1.0 - dfx_dx - denom) * py) / denom;
  orb->vec[4] = orb->vec[4] + (orb->vec[1] * fx + orb->vec[3] * fy) / rel_p;
  FL(26);
}

/* apply_element_edge_kick, bmad/low_level/apply_element_edge_kick.f90:37-278
 * for the bmad_standard field_calc case.  Returns -1 for unsupported forms. */
/* sad_soft_bend_edge_kick, bmad/modules/fringe_mod.f90:892-996 (tracking
 * part, sbend): the soft-edge bend fringe of fringe_type soft_edge_only and
 * sad_full, fb = 12 fint hgap at the entrance (fintx, hgapx at the exit). */
static void sad_soft_bend_edge_kick(const bgo_ele* ele, int first_edge, bgo_coord* orb) {
  if (ele->fringe_type != BGO_FRINGE_SOFT_EDGE_ONLY && ele->fringe_type != BGO_FRINGE_SAD_FULL) return;
  double fb = first_edge ? 12 * ele->fint * ele->hgap : 12 * ele->fintx * ele->hgapx;
  if (fb == 0) return;
  double g = ele->g + ele->dg;
  if (g == 0) return;
  g = g * 1;
  if (!first_edge) g = -g;
  double px = orb->vec[1];
  double y = orb->vec[2];
  double rel_p = 1 + orb->vec[5];
  double c1 = fb * fb * g / (24 * rel_p);
  double c2 = fb * (g * g) / (6 * rel_p);
  double c3 = 2 * (g * g) / (3 * fb * rel_p);
  double y2 = y * y, y3 = y * y2, y4 = y2 * y2;
  orb->vec[0] = orb->vec[0] + c1 * orb->vec[5];
  orb->vec[3] = orb->vec[3] + c2 * y - c3 * y3;
  orb->vec[4] = orb->vec[4] + (c1 * px + c2 * y2 / 2 - c3 * y4 / 4) / rel_p;
  FL(30);
}

/* linear_bend_edge_kick, bmad/modules/fringe_mod.f90:151-212 (tracking
 * part): the linear edge focusing of fringe_type linear_edge. */
static void linear_bend_edge_kick(const bgo_ele* ele, int first_edge, bgo_coord* orb) {
  double c_dir = 1.0;
  double g_tot = ele->is_on ? (ele->g + ele->dg) * c_dir : 0.0;
  double e, fint, hgap;
  if (first_edge) {
    e = ele->e1;
    fint = ele->fint;
    hgap = ele->hgap;
  } else {
    e = ele->e2;
    fint = ele->fintx;
    hgap = ele->hgapx;
  }
  double cos_e = cos(e), sin_e = sin(e), tan_e = sin_e / cos_e;
  double ht_x = g_tot * tan_e, ht_y;
  if (fint == 0) {
    ht_y = -ht_x;
  } else {
    ht_y = -g_tot * tan(e - 2 * fint * g_tot * hgap * (1 + sin_e * sin_e) / cos_e);
  }
  ht_x = 1 * ht_x;
  ht_y = 1 * ht_y;
  double x = orb->vec[0], y = orb->vec[2];
  orb->vec[1] = orb->vec[1] + ht_x * x;
  orb->vec[3] = orb->vec[3] + ht_y * y;
  FL(4);
}

/* soft_quadrupole_edge_kick, bmad/modules/fringe_mod.f90:555-660 (tracking
 * part): the soft-edge fringe of a quadrupole with the fringe integrals
 * fq1, fq2; charge_dir = 1 (forward tracking of the reference species). */
static void soft_quadrupole_edge_kick(const bgo_ele* ele, int first_edge, bgo_coord* orb) {
  if (ele->fringe_type != BGO_FRINGE_SOFT_EDGE_ONLY && ele->fringe_type != BGO_FRINGE_FULL) return;
  double rel_p = 1 + orb->vec[5];
  double k1_rel = 1.0 * ele->k1 / rel_p;
  double f1 = k1_rel * ele->fq1;
  double f2 = k1_rel * ele->fq2;
  if (f1 == 0 && f2 == 0) return;
  if (!first_edge) f1 = -f1;
  double ef1 = P_EXP(f1);
  double x = orb->vec[0], px = orb->vec[1], y = orb->vec[2], py = orb->vec[3];
  double vx = px / rel_p, vy = py / rel_p;
  orb->vec[4] = orb->vec[4] - (f1 * x + f2 * (1 + f1 / 2) * vx / ef1) * vx +
                (f1 * y + f2 * (1 - f1 / 2) * vy * ef1) * vy;
  orb->vec[0] = x * ef1 + vx * f2;
  orb->vec[1] = px / ef1;
  orb->vec[2] = y / ef1 - vy * f2;
  orb->vec[3] = py * ef1;
  LM(1);
  FL(40);
}

/* The exact (PTC) bend edge of fringe_type full: exact_bend_edge_kick,
 * bmad/modules/fringe_mod.f90:1465-1686, tracking part, forward
 * (time_dir = 1).  The particle goes to PTC's (x, px, y, py, pt, ct)
 * coordinates, through a rotation of the frame by the edge angle, the
 * dipole fringe map and the wedge of the bend field, and back.  Each step
 * returns 0 where the reference sets err_flag (the particle is then lost_pz
 * with its Bmad coordinates untouched). */

/* ptc_rot_xz, fringe_mod.f90:1384-1441: rotation of the frame about y. */
static int ptc_rot_xz(double a, double X[6], double beta0) {
  double arg = 1.0 + 2.0 * X[4] / beta0 + X[4] * X[4] - X[1] * X[1] - X[3] * X[3];
  if (arg < 0) return 0;
  double pz = sqrt(arg);
  double pt = 1.0 - X[1] * tan(a) / pz;
  double x1 = X[0];
  X[0] = x1 / cos(a) / pt;
  X[1] = X[1] * cos(a) + sin(a) * pz;
  X[2] = X[2] + X[3] * x1 * tan(a) / pz / pt;
  X[5] = X[5] + x1 * tan(a) / pz / pt * (1.0 / beta0 + X[4]);
  FL(30);
  return 1;
}

/* ptc_wedger, fringe_mod.f90:1020-1123: a wedge of angle a of the bend
 * field g_tot (a plain rotation when g_tot = 0). */
static int ptc_wedger(double a, double g_tot, double beta0, double X[6]) {
  double b1 = g_tot;
  if (b1 == 0) return ptc_rot_xz(a, X, beta0);
  double fac = 1.0 + 2.0 * X[4] / beta0 + X[4] * X[4] - X[1] * X[1] - X[3] * X[3];
  if (fac < 0) return 0;
  double radix = 1.0 + 2.0 * X[4] / beta0 + X[4] * X[4] - X[3] * X[3];
  if (radix < 1e-10) return 0;
  double pz = sqrt(fac), pt = sqrt(radix);
  double Xn1, Xn2, Xn3, Xn6;
  Xn2 = X[1] * cos(a) + (pz - b1 * X[0]) * sin(a);
  radix = 1.0 + 2.0 * X[4] / beta0 + X[4] * X[4] - Xn2 * Xn2 - X[3] * X[3];
  if (radix < 1e-10) return 0;
  double pzs = sqrt(radix);
  double sa = sin(a);
  Xn1 = X[0] * cos(a) + (X[0] * X[1] * sin(2.0 * a) + (sa * sa) * (2.0 * X[0] * pz - b1 * (X[0] * X[0]))) /
                            (pzs + pz * cos(a) - X[1] * sin(a));
  Xn3 = (a + P_ASIN(X[1] / pt) - P_ASIN(Xn2 / pt)) / b1;
  Xn6 = X[5] + Xn3 * (1.0 / beta0 + X[4]);
  Xn3 = X[2] + X[3] * Xn3;
  X[0] = Xn1;
  X[1] = Xn2;
  X[2] = Xn3;
  X[5] = Xn6;
  LM(2);
  FL(60);
  return 1;
}

/* ptc_fringe_dipoler, fringe_mod.f90:1151-1360: the dipole fringe with the
 * field integral fint * hgap; b = g_tot at the entrance, -g_tot at the exit.
 * gfortran's inline SUM starts from zero, kept here for the sign of zero. */
static int ptc_fringe_dipoler(double X[6], double g_tot, double beta0, double fint, double hgap, int first_edge) {
  double b = first_edge ? g_tot : -g_tot;
  double fac = 1.0 + 2.0 * X[4] / beta0 + X[4] * X[4] - X[1] * X[1] - X[3] * X[3];
  if (fac == 0) return 0;
  double pz = sqrt(fac);
  double time_fac = 1.0 / beta0 + X[4];
  double xp = X[1] / pz, yp = X[3] / pz;
  double d11 = (1.0 + xp * xp) / pz, d21 = xp * yp / pz, d31 = -xp;
  double d12 = xp * yp / pz, d22 = (1.0 + yp * yp) / pz, d32 = -yp;
  double d13 = -(time_fac * xp / (pz * pz)), d23 = -(time_fac * yp / (pz * pz)), d33 = time_fac / pz;
  double u = 1.0 + yp * yp;
  double w = 1.0 + (xp * xp) * (2.0 + yp * yp);
  double fi0 = P_ATAN(xp / u) - b * fint * hgap * 2.0 * w * pz;
  double cf = P_COS(fi0);
  double co2 = b / (cf * cf);
  double xu = xp / u;
  double co1 = co2 / (1.0 + xu * xu);
  double fi1 = co1 / u - co2 * b * fint * hgap * 2.0 * (2.0 * xp * (2.0 + yp * yp) * pz);
  double fi2 = -(co1 * 2.0 * xp * yp / (u * u)) - co2 * b * fint * hgap * 2.0 * (2.0 * (xp * xp) * yp) * pz;
  double fi3 = -(co2 * b * fint * hgap * 2.0 * w);
  double fi0t = b * P_TAN(fi0);
  double bb = 0.0 + fi1 * d12 + fi2 * d22 + fi3 * d32;
  fac = 1.0 - 2.0 * bb * X[2];
  if (fac < 0) return 0;
  X[2] = 2.0 * X[2] / (1.0 + sqrt(fac));
  X[3] = X[3] - fi0t * X[2];
  bb = 0.0 + fi1 * d11 + fi2 * d21 + fi3 * d31;
  X[0] = X[0] + 0.5 * bb * (X[2] * X[2]);
  bb = 0.0 + fi1 * d13 + fi2 * d23 + fi3 * d33;
  X[5] = X[5] - 0.5 * bb * (X[2] * X[2]);
  LM(3);
  FL(110);
  return 1;
}

/* exact_bend_edge_kick, fringe_mod.f90:1465-1577, with vec_bmad_to_ptc and
 * vec_ptc_to_bmad (:1599-1684).  orb%t is not tracked (relative RF time). */
static void exact_bend_edge_kick(const bgo_ele* ele, int first_edge, bgo_coord* orb) {
  double beta0 = ele->p0c / ele->e_tot;
  double g_tot = ele->is_on ? ele->g + ele->dg : 0.0;
  double X[6];
  double v5 = orb->vec[4], v6 = orb->vec[5];
  X[0] = orb->vec[0];
  X[1] = orb->vec[1];
  X[2] = orb->vec[2];
  X[3] = orb->vec[3];
  X[4] = (v6 * v6 + 2 * v6) / (1 / beta0 + sqrt(1 / (beta0 * beta0) + v6 * v6 + 2 * v6));
  X[5] = -(v5 * (1 / beta0 + X[4]) / (1 + v6));
  double edge_angle, fint, hgap;
  if (first_edge) {
    edge_angle = 1 * ele->e1;
    fint = ele->fint;
    hgap = ele->hgap;
  } else {
    edge_angle = 1 * ele->e2;
    fint = ele->fintx;
    hgap = ele->hgapx;
  }
  int ok;
  if (first_edge) {
    ok = ptc_wedger(edge_angle, 0.0, beta0, X) && ptc_fringe_dipoler(X, g_tot, beta0, 1 * fint, hgap, 1) &&
         ptc_wedger(-edge_angle, g_tot, beta0, X);
  } else {
    ok = ptc_wedger(-edge_angle, g_tot, beta0, X) && ptc_fringe_dipoler(X, g_tot, beta0, 1 * fint, hgap, 0) &&
         ptc_wedger(edge_angle, 0.0, beta0, X);
  }
  FL(20);
  if (!ok) {
    orb->state = BGO_LOST_PZ;
    return;
  }
  double f1 = 1 + 2 * X[4] / beta0 + X[4] * X[4];
  if (f1 <= 0) return;
  double t6 = (2 * X[4] / beta0 + X[4] * X[4]) / (sqrt(f1) + 1);
  double t5 = -(X[5] * (1 + t6) / (1 / beta0 + X[4]));
  orb->vec[0] = X[0];
  orb->vec[1] = X[1];
  orb->vec[2] = X[2];
  orb->vec[3] = X[3];
  orb->vec[4] = t5;
  orb->vec[5] = t6;
  FL(12);
}

static int apply_element_edge_kick(bgo_coord* orb, const bgo_ele* ele, int first_edge, const bgo_param* param,
                                   const double* ae, const double* be, int ix_elec_max) {
  int physical_end = first_edge ? BGO_ENTRANCE_END : BGO_EXIT_END;
  int fat = ele->fringe_at;
  int here = (fat == BGO_BOTH_ENDS) || (fat == physical_end);
  if (!here) return 0;
  double at_sign = first_edge ? 1.0 : -1.0;
  if (!first_edge) electric_longitudinal_fringe(orb, ele, ae, be, ix_elec_max, at_sign, param);
  switch (ele->key) {
    case BGO_QUADRUPOLE:
    case BGO_SEXTUPOLE: {
      /* apply_element_edge_kick.f90:173-186: quadrupole entrance hard then
       * soft, exit soft then hard; sextupole hard only. */
      int hard = ele->fringe_type == BGO_FRINGE_FULL || ele->fringe_type == BGO_FRINGE_HARD_EDGE_ONLY;
      int soft = ele->key == BGO_QUADRUPOLE;
      if (first_edge) {
        if (hard) hard_multipole_edge_kick(ele, first_edge, orb);
        if (soft) soft_quadrupole_edge_kick(ele, first_edge, orb);
      } else {
        if (soft) soft_quadrupole_edge_kick(ele, first_edge, orb);
        if (hard) hard_multipole_edge_kick(ele, first_edge, orb);
      }
      break;
    }
    case BGO_SBEND:
      /* bend_edge_kick, fringe_mod.f90:39-127 */
      if (ele->fringe_type == BGO_FRINGE_NONE) break;
      if (ele->fringe_type == BGO_FRINGE_BASIC_BEND || ele->fringe_type == BGO_FRINGE_HARD_EDGE_ONLY) {
        bgo_hwang_bend_edge_kick(ele, first_edge, orb, param);
      } else if (ele->fringe_type == BGO_FRINGE_SAD_FULL) {
        if (first_edge) {
          sad_soft_bend_edge_kick(ele, first_edge, orb);
          bgo_hwang_bend_edge_kick(ele, first_edge, orb, param);
        } else {
          bgo_hwang_bend_edge_kick(ele, first_edge, orb, param);
          sad_soft_bend_edge_kick(ele, first_edge, orb);
        }
      } else if (ele->fringe_type == BGO_FRINGE_SOFT_EDGE_ONLY) {
        sad_soft_bend_edge_kick(ele, first_edge, orb);
      } else if (ele->fringe_type == BGO_FRINGE_LINEAR_EDGE) {
        linear_bend_edge_kick(ele, first_edge, orb);
      } else {
        /* full: the k1 hard-edge multipole fringe (fringe_mod.f90:63-65,
         * 102-104) around the exact edge */
        if (first_edge) hard_multipole_edge_kick(ele, first_edge, orb);
        exact_bend_edge_kick(ele, first_edge, orb);
        if (!first_edge) hard_multipole_edge_kick(ele, first_edge, orb);
      }
      break;
    default:
      break;
  }
  if (first_edge) electric_longitudinal_fringe(orb, ele, ae, be, ix_elec_max, at_sign, param);
  return 0;
}

static int has_fringe_info(const bgo_ele* ele) {
  /* init_fringe_info, bmad/low_level/init_fringe_info.f90:22-60 */
  if (ele->key == BGO_RFCAVITY) return 1;
  if ((ele->fringe_type == BGO_FRINGE_NONE || ele->fringe_at == BGO_NO_END) && !ele->has_elec_poles) return 0;
  return 1;
}

/* ------------------------------------------------------------------ */
/* Element trackers                                                    */

/* quad_mat2_calc, bmad/low_level/quad_mat2_calc.f90:22-81 */
static void quad_mat2_calc(double k1, double length, double rel_p, double m[2][2], double zc[3]) {
  double sqrt_k = sqrt(fabs(k1));
  double sk_l = sqrt_k * length;
  double cx, sx;
  if (fabs(sk_l) < 1e-10) {
    double k_l2 = k1 * (length * length);
    cx = 1 + k_l2 / 2;
    sx = (1 + k_l2 / 6) * length;
    FL(8);
  } else if (k1 < 0) {
    cx = P_COS(sk_l);
    sx = P_SIN(sk_l) / sqrt_k;
    LM(2);
    FL(1);
  } else {
    cx = P_COSH(sk_l);
    sx = P_SINH(sk_l) / sqrt_k;
    LM(2);
    FL(1);
  }
  m[0][0] = cx;
  m[0][1] = sx / rel_p;
  m[1][0] = k1 * sx * rel_p;
  m[1][1] = cx;
  zc[0] = k1 * (-cx * sx + length) / 4;
  zc[1] = -k1 * (sx * sx) / (2 * rel_p);
  zc[2] = -(cx * sx + length) / (4 * rel_p * rel_p);
  FL(22);
}

/* low_energy_z_correction, bmad/low_level/low_energy_z_correction.f90:22-58 */
static double low_energy_z_correction(const bgo_coord* orbit, const bgo_ele* ele, double ds,
                                      const bgo_param* param) {
  double mass = param->mass;
  double p0c = orbit->p0c;
  double e_tot = ele->e_tot;
  double beta0 = p0c / e_tot;
  double pz = orbit->vec[5];
  double dz;
  FL(5);
  if (mass * ((beta0 * pz) * (beta0 * pz)) < 3e-7 * e_tot) {
    double f = (beta0 * beta0) * (2 * (beta0 * beta0) - ((mass / e_tot) * (mass / e_tot)) / 2);
    dz = ds * pz * (1 - 3 * (pz * (beta0 * beta0)) / 2 + (pz * pz) * f) * ((mass / e_tot) * (mass / e_tot));
    FL(24);
  } else {
    dz = ds * (orbit->beta - beta0) / beta0;
    FL(3);
  }
  return dz;
}

/* track_a_quadrupole, bmad/low_level/track_a_quadrupole.f90:17-148 */
static int track_a_quadrupole(bgo_coord* orbit, const bgo_ele* ele, const bgo_param* param) {
  double an[BGO_N_POLE], bn[BGO_N_POLE], ae[BGO_N_POLE], be[BGO_N_POLE], b1;
  const __float128 t0 = orbit->t; /* start_orb = orbit (:40) */
  const double z0 = orbit->vec[4];
  double charge_dir = 1.0;
  double length = 1 * ele->l;
  int ix_mag_max = bgo_multipole_ele_to_ab(ele, 0, 0, 1, an, bn, &b1);
  int ix_elec_max = bgo_multipole_ele_to_ab(ele, 0, 1, 0, ae, be, NULL);
  if (ix_mag_max < -1 || ix_elec_max < -1) return -1;
  int n_step = 1;
  if (ix_mag_max > -1 || ix_elec_max > -1) {
    int ns = nint_f(fabs(length) / ele->ds_step);
    n_step = ns > 1 ? ns : 1;
  }
  double r_step = 1.0 / n_step;
  double step_len = ele->l * r_step;
  if (length == 0) n_step = 0;

  if (ele->has_misalign) offset_particle(ele, 1, orbit, 1, 0, 0, 0, param);
  int has_fringe = has_fringe_info(ele);
  if (has_fringe) {
    if (apply_element_edge_kick(orbit, ele, 1, param, ae, be, ix_elec_max)) return -1;
    if (orbit->state != BGO_ALIVE) return 0;
  }
  if (ix_mag_max > -1) ab_multipole_kicks(an, bn, ix_mag_max, ele, orbit, param, 0, r_step / 2);
  if (ix_elec_max > -1) ab_multipole_kicks(ae, be, ix_elec_max, ele, orbit, param, 1, step_len / 2);

  for (int i = 1; i <= n_step; i++) {
    double mx[2][2], my[2][2], dzx[3], dzy[3];
    double rel_p = 1 + orbit->vec[5];
    double k1 = charge_dir * b1 / (length * rel_p);
    FL(4);
    quad_mat2_calc(-k1, step_len, rel_p, mx, dzx);
    quad_mat2_calc(k1, step_len, rel_p, my, dzy);
    double* v = orbit->vec;
    v[4] = v[4] + (dzx[0] * (v[0] * v[0]) + dzx[1] * v[0] * v[1] + dzx[2] * (v[1] * v[1]) + dzy[0] * (v[2] * v[2]) +
                   dzy[1] * v[2] * v[3] + dzy[2] * (v[3] * v[3]));
    double x = v[0], px = v[1], y = v[2], py = v[3];
    v[0] = mx[0][0] * x + mx[0][1] * px;
    v[1] = mx[1][0] * x + mx[1][1] * px;
    v[2] = my[0][0] * y + my[0][1] * py;
    v[3] = my[1][0] * y + my[1][1] * py;
    FL(32);
    v[4] = v[4] + low_energy_z_correction(orbit, ele, step_len, param);
    FL(1);
    if (i == n_step) {
      if (ix_mag_max > -1) ab_multipole_kicks(an, bn, ix_mag_max, ele, orbit, param, 0, r_step / 2);
      if (ix_elec_max > -1) ab_multipole_kicks(ae, be, ix_elec_max, ele, orbit, param, 1, step_len / 2);
    } else {
      if (ix_mag_max > -1) ab_multipole_kicks(an, bn, ix_mag_max, ele, orbit, param, 0, r_step);
      if (ix_elec_max > -1) ab_multipole_kicks(ae, be, ix_elec_max, ele, orbit, param, 1, step_len);
    }
  }
  if (has_fringe) {
    if (apply_element_edge_kick(orbit, ele, 0, param, ae, be, ix_elec_max)) return -1;
    if (orbit->state != BGO_ALIVE) return 0;
  }
  if (ele->has_misalign) offset_particle(ele, 0, orbit, 1, 0, 0, 0, param);
  element_exit_time(orbit, ele, t0, z0);
  return 0;
}

/* track_a_thick_multipole, bmad/low_level/track_a_thick_multipole.f90:18-134
 * (no elseparator / ac_kicker forms). */
static int track_a_thick_multipole(bgo_coord* orbit, const bgo_ele* ele, const bgo_param* param) {
  double an[BGO_N_POLE], bn[BGO_N_POLE], ae[BGO_N_POLE], be[BGO_N_POLE];
  const __float128 t0 = orbit->t; /* start_orb = orbit (:41) */
  const double z0 = orbit->vec[4];
  double length = ele->l * 1;
  int ix_mag_max = bgo_multipole_ele_to_ab(ele, 0, 0, 1, an, bn, NULL);
  int ix_elec_max = bgo_multipole_ele_to_ab(ele, 0, 1, 0, ae, be, NULL);
  if (ix_mag_max < -1 || ix_elec_max < -1) return -1;
  int n_step;
  if (ix_mag_max == -1 && ix_elec_max == -1) {
    n_step = 1;
  } else {
    int ns = nint_f(fabs(length / ele->ds_step));
    n_step = ns > 1 ? ns : 1;
  }
  double r_step = 1.0 / n_step;
  double step_len = length / n_step;
  if (ele->has_misalign) offset_particle(ele, 1, orbit, 1, 0, 0, 0, param);
  int has_fringe = has_fringe_info(ele);
  if (has_fringe) {
    if (apply_element_edge_kick(orbit, ele, 1, param, ae, be, ix_elec_max)) return -1;
    if (orbit->state != BGO_ALIVE) return 0;
  }
  double ac_amp = 1;
  if (ix_mag_max > -1) ab_multipole_kicks(an, bn, ix_mag_max, ele, orbit, param, 0, ac_amp * r_step / 2);
  if (ix_elec_max > -1) ab_multipole_kicks(ae, be, ix_elec_max, ele, orbit, param, 1, ac_amp * step_len / 2);
  for (int i = 1; i <= n_step; i++) {
    track_a_drift(orbit, step_len, 1, param);
    if (i == n_step) {
      if (ix_mag_max > -1) ab_multipole_kicks(an, bn, ix_mag_max, ele, orbit, param, 0, ac_amp * r_step / 2);
      if (ix_elec_max > -1) ab_multipole_kicks(ae, be, ix_elec_max, ele, orbit, param, 1, ac_amp * step_len / 2);
    } else {
      if (ix_mag_max > -1) ab_multipole_kicks(an, bn, ix_mag_max, ele, orbit, param, 0, ac_amp * r_step);
      if (ix_elec_max > -1) ab_multipole_kicks(ae, be, ix_elec_max, ele, orbit, param, 1, ac_amp * step_len);
    }
  }
  if (has_fringe) {
    if (apply_element_edge_kick(orbit, ele, 0, param, ae, be, ix_elec_max)) return -1;
    if (orbit->state != BGO_ALIVE) return 0;
  }
  if (ele->has_misalign) offset_particle(ele, 0, orbit, 1, 0, 0, 0, param);
  element_exit_time(orbit, ele, t0, z0);
  return 0;
}

/* sbend_body_with_k1_map, bmad/low_level/track_a_bend.f90:500-659 (no matrix) */
static void sbend_body_with_k1_map(const bgo_ele* ele, double dg, double b1, int n_step, bgo_coord* orbit) {
  double rel_charge_dir = 1.0;
  double g = ele->g;
  double length = 1 * ele->l / n_step;
  double k1 = b1 / ele->l;
  double g_tot = (g + dg) * rel_charge_dir;
  double rel_p = (1 + orbit->vec[5]);
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
    s_x = P_SIN(arg) / om_x;
    c_x = P_COS(arg);
    z2 = tau_x * g * (1 - c_x) / (rel_p * (om_x * om_x));
  } else {
    s_x = P_SINH(arg) / om_x;
    c_x = P_COSH(arg);
    z2 = tau_x * g * (1 - c_x) / (rel_p * (om_x * om_x));
  }
  arg = om_y * length;
  if (arg < 1e-6) {
    s_y = (1 + tau_y * (arg * arg) / 6) * length;
    c_y = 1 + tau_y * (arg * arg) / 2;
  } else if (k1 < 0) {
    s_y = P_SIN(om_y * length) / om_y;
    c_y = P_COS(om_y * length);
  } else {
    s_y = P_SINH(om_y * length) / om_y;
    c_y = P_COSH(om_y * length);
  }
  double r[6];
  for (int i = 0; i < 6; i++) r[i] = orbit->vec[i];
  r[0] = r[0] - x_c;
  double z0 = -g * x_c * length;
  double z1 = -g * s_x;
  double z11 = tau_x * (om_x * om_x) * (length - c_x * s_x) / 4;
  double z12 = -tau_x * (om_x * om_x) * (s_x * s_x) / (2 * rel_p);
  double z22 = -(length + c_x * s_x) / (4 * rel_p2);
  double z33 = tau_y * (om_y * om_y) * (length - c_y * s_y) / 4;
  double z34 = -tau_y * (om_y * om_y) * (s_y * s_y) / (2 * rel_p);
  double z44 = -(length + c_y * s_y) / (4 * rel_p2);
  orbit->vec[0] = c_x * r[0] + s_x * r[1] / rel_p + x_c;
  orbit->vec[1] = tau_x * (om_x * om_x) * rel_p * s_x * r[0] + c_x * r[1];
  orbit->vec[2] = c_y * r[2] + s_y * r[3] / rel_p;
  orbit->vec[3] = tau_y * (om_y * om_y) * rel_p * s_y * r[2] + c_y * r[3];
  orbit->vec[4] = r[4] + 1 * 1 * z0 + z1 * r[0] + z2 * r[1] + z11 * (r[0] * r[0]) + z12 * r[0] * r[1] +
                  z22 * (r[1] * r[1]) + z33 * (r[2] * r[2]) + z34 * r[2] * r[3] + z44 * (r[3] * r[3]);
  LM(2);
  FL(110);
}

/* elec_multipole_field, bmad/code/elec_multipole_field.f90:20-65 (no dE) */
static void elec_multipole_field(double a, double b, int n, const bgo_coord* coord, double* Ex, double* Ey) {
  *Ex = 0;
  *Ey = 0;
  if (a == 0 && b == 0) return;
  double x = coord->vec[0], y = coord->vec[2];
  for (int m = 0; m <= n; m += 2) {
    double f = bgo_c_multi(n, m, 1) * mexp(x, n - m) * mexp(y, m);
    *Ex = *Ex - b * f;
    *Ey = *Ey - a * f;
  }
  for (int m = 1; m <= n; m += 2) {
    double f = bgo_c_multi(n, m, 1) * mexp(x, n - m) * mexp(y, m);
    *Ex = *Ex + a * f;
    *Ey = *Ey - b * f;
  }
}

/* apply_multipole_kicks (contained in track_a_bend), track_a_bend.f90:338-471,
 * non-exact form: the magnetic field B and electric field E at the particle,
 * then the magnetic kick, then the electric kick (which changes pz, beta, z). */
static void bend_apply_multipole_kicks(double coef, double step_len, double r_step, int ix_mag_max,
                                       const double* an, const double* bn, int ix_elec_max, const double* ae,
                                       const double* be, const bgo_ele* ele, bgo_coord* orbit,
                                       const bgo_param* param) {
  double B0 = 0, B1 = 0, E0 = 0, E1 = 0, kx, ky;
  int charge = param->charge;
  double c_dir = 1 * 1 * (double)param->charge;
  double f_p0c = r_step * ele->p0c / (C_LIGHT * param->charge);
  for (int i = 0; i <= ix_mag_max; i++) {
    if (an[i] == 0 && bn[i] == 0) continue;
    ab_multipole_kick(an[i], bn[i], i, 0, orbit, param, 0, NULL, &kx, &ky);
    B0 = B0 + f_p0c * ky;
    B1 = B1 - f_p0c * kx;
    FL(4);
  }
  for (int i = 0; i <= ix_elec_max; i++) {
    if (ae[i] == 0 && be[i] == 0) continue;
    double Ex, Ey;
    elec_multipole_field(ae[i], be[i], i, orbit, &Ex, &Ey);
    E0 = E0 + Ex;
    E1 = E1 + Ey;
  }
  if (ix_mag_max > -1) {
    double f_coef = coef * c_dir * (1 + ele->g * orbit->vec[0]) * C_LIGHT / orbit->p0c;
    orbit->vec[1] = orbit->vec[1] - f_coef * B1;
    orbit->vec[3] = orbit->vec[3] + f_coef * B0;
    FL(10);
  }
  if (ix_elec_max > -1) {
    bgo_coord orb0 = *orbit;
    double rel_p0 = 1 + orb0.vec[5];
    double ps2 = rel_p0 * rel_p0 - orb0.vec[1] * orb0.vec[1] - orb0.vec[3] * orb0.vec[3];
    double ps = sqrt(ps2) / rel_p0;
    double f_coef =
        step_len * coef * (1 + ele->g * orb0.vec[0]) * (double)charge / (ps * orb0.beta * orb0.p0c);
    double Kx = f_coef * E0;
    double Ky = f_coef * E1;
    double alpha = (Kx * (2 * orb0.vec[1] + Kx) + Ky * (2 * orb0.vec[3] + Ky)) / (rel_p0 * rel_p0);
    orbit->vec[1] = orb0.vec[1] + Kx;
    orbit->vec[3] = orb0.vec[3] + Ky;
    orbit->vec[5] = orb0.vec[5] + rel_p0 * sqrt_one(alpha);
    orbit->beta = (1 + orbit->vec[5]) / sqrt(ps2 + orbit->vec[1] * orbit->vec[1] + orbit->vec[3] * orbit->vec[3] +
                                             sq(param->mass / orbit->p0c));
    orbit->vec[4] = orb0.vec[4] * orbit->beta / orb0.beta;
  }
}

/* track_a_bend, bmad/low_level/track_a_bend.f90:18-333 */
static int track_a_bend(bgo_coord* orbit, const bgo_ele* ele, bgo_param* param) {
  double an[BGO_N_POLE], bn[BGO_N_POLE], ae[BGO_N_POLE], be[BGO_N_POLE], b1;
  const __float128 t0 = orbit->t; /* start_orb = orbit (:42) */
  const double z0 = orbit->vec[4];
  if (ele->has_misalign) offset_particle(ele, 1, orbit, 1, 0, 0, 0, param);
  double rel_charge_dir = 1.0;
  int ix_elec_max = bgo_multipole_ele_to_ab(ele, 0, 1, 0, ae, be, NULL);
  if (apply_element_edge_kick(orbit, ele, 1, param, ae, be, ix_elec_max)) return -1;
  if (bgo_orbit_too_large(orbit, param)) return 0;

  int ix_mag_max = bgo_multipole_ele_to_ab(ele, 0, 0, 1, an, bn, &b1);
  if (ix_mag_max < -1) return -1;
  b1 = b1 * rel_charge_dir;
  if (fabs(b1) < 1e-10) {
    bn[1] = b1;
    b1 = 0;
  }
  double length = 1 * ele->l;
  double g = ele->g, dg;
  if (length == 0) {
    dg = 0;
  } else {
    dg = bn[0] / ele->l;
    bn[0] = 0;
  }
  double g_tot = (g + dg) * rel_charge_dir;
  if (!ele->is_on) {
    dg = -g;
    g_tot = 0;
    b1 = 0;
  }
  int n_step = 1;
  if (ix_mag_max > -1 || ix_elec_max > -1) {
    int ns = nint_f(fabs(length) / ele->ds_step);
    n_step = ns > 1 ? ns : 1;
  }
  double r_step = 1.0 / n_step;
  double step_len = length / n_step;
  double angle = g * step_len;
  FL(4);
  if (ix_mag_max > -1 || ix_elec_max > -1)
    bend_apply_multipole_kicks(0.5, step_len, r_step, ix_mag_max, an, bn, ix_elec_max, ae, be, ele, orbit, param);

  for (int n = 1; n <= n_step; n++) {
    if (b1 != 0) {
      sbend_body_with_k1_map(ele, dg, b1, n_step, orbit);
      orbit->vec[4] = orbit->vec[4] + low_energy_z_correction(orbit, ele, step_len, param);
    } else if ((g == 0 && dg == 0) || step_len == 0) {
      track_a_drift(orbit, step_len, 1, param);
    } else {
      double x = orbit->vec[0], px = orbit->vec[1], y = orbit->vec[2], py = orbit->vec[3], z = orbit->vec[4],
             pz = orbit->vec[5];
      double rel_p = 1 + pz;
      double rel_p2 = rel_p * rel_p;
      if (dg == 0 && fabs(x * g) < 1e-9 && fabs(px) < 1e-9 && fabs(py) < 1e-9 && fabs(pz) < 1e-9) {
        double ll = step_len;
        double cos_a = cos(angle), sin_a = sin(angle), sinc_a = sinc_f(angle), cosc_a = cosc_f(angle);
        double m2 = param->mass * param->mass;
        double gam2 = m2 / (sq(rel_p * orbit->p0c) + m2);
        double m56 = ll * (gam2 - sq(g * ll) * sincc_f(angle));
        orbit->vec[0] = cos_a * x + ll * sinc_a * px + g * (ll * ll) * cosc_a * pz;
        orbit->vec[1] = -(g * sin_a * x) + cos_a * px + g * ll * sinc_a * pz;
        orbit->vec[2] = y + ll * py;
        orbit->vec[4] = -(g * ll * sinc_a * x) - g * (ll * ll) * cosc_a * px + z + m56 * pz;
        LM(2);
        FL(40);
      } else {
        double beta_ref = ele->p0c / ele->e_tot;
        double sinc_a = sinc_f(angle);
        double pt = sqrt(rel_p2 - py * py);
        FL(5);
        if (fabs(px) > pt) {
          orbit->state = BGO_LOST_PZ;
          return 0;
        }
        double g_p = g_tot / pt;
        double phi_1 = P_ASIN(px / pt);
        double cos_a = cos(angle), sin_a = sin(angle), cosc_a = cosc_f(angle);
        double cos_plus = P_COS(angle + phi_1), sin_plus = P_SIN(angle + phi_1);
        double gx1 = 1 + g * x;
        double alpha = 2 * gx1 * sin_plus * step_len * sinc_a - g_p * sq(gx1 * step_len * sinc_a);
        double r = cos_plus * cos_plus + g_p * alpha;
        LM(5);
        FL(22);
        if (r < 0 || (fabs(g_p) < 1e-5 && fabs(cos_plus) < 1e-5)) {
          orbit->state = BGO_LOST;
          orbit->vec[0] = 2 * param->max_aperture_limit;
          return 0;
        }
        double rad = sqrt(r), denom, xi;
        if (cos_plus > 0) {
          denom = rad + cos_plus;
          xi = alpha / denom;
        } else {
          denom = rad - cos_plus;
          xi = denom / g_p;
        }
        orbit->vec[0] = x * cos_a - (step_len * step_len) * g * cosc_a + xi;
        FL(9);
        if (fabs(orbit->vec[0]) > param->max_aperture_limit) {
          orbit->state = BGO_LOST;
          return 0;
        }
        double L_u = xi;
        double L_v = -(step_len * sinc_a + x * sin_a);
        double L_c = sqrt(L_v * L_v + L_u * L_u);
        double angle_p = 2 * (angle + phi_1 - 1 * P_ATAN2(L_u, -L_v));
        double L_p = 1 * L_c / sinc_p(angle_p / 2);
        orbit->vec[1] = pt * P_SIN(phi_1 + angle - angle_p);
        orbit->vec[2] = y + py * L_p / pt;
        orbit->vec[4] = z + orbit->beta * step_len / beta_ref - rel_p * L_p / pt;
        LM(2);
        FL(28);
      }
    }
    if (ix_mag_max > -1 || ix_elec_max > -1) {
      if (n == n_step)
        bend_apply_multipole_kicks(0.5, step_len, r_step, ix_mag_max, an, bn, ix_elec_max, ae, be, ele, orbit,
                                   param);
      else
        bend_apply_multipole_kicks(1.0, step_len, r_step, ix_mag_max, an, bn, ix_elec_max, ae, be, ele, orbit,
                                   param);
    }
  }
  if (bgo_orbit_too_large(orbit, param)) return 0;
  if (apply_element_edge_kick(orbit, ele, 0, param, ae, be, ix_elec_max)) return -1;
  if (ele->has_misalign) offset_particle(ele, 0, orbit, 1, 0, 0, 0, param);
  element_exit_time(orbit, ele, t0, z0);
  return 0;
}

/* rf_coupler_kick, bmad/low_level/rf_coupler_kick.f90:20-104 (tracking part)
 * for an rfcavity: the coupler's transverse kick with the energy change it
 * implies.  e_accel_field(ele, gradient$) = voltage / l (attribute_bookkeeper
 * .f90:730-736) times field_autoscale = 1, the value bmad_standard tracking
 * keeps (autoscale_phase_and_amp.f90:108-115). */
static void rf_coupler_kick(const bgo_ele* ele, int first_edge, double phase, bgo_coord* orbit,
                            const bgo_param* param) {
  int physical_end = first_edge ? BGO_ENTRANCE_END : BGO_EXIT_END;
  if (!(ele->coupler_at == BGO_BOTH_ENDS || ele->coupler_at == physical_end)) return;
  if (ele->coupler_strength == 0) return;
  double ph = phase;
  ph = PI / 2 - ph;
  ph = ph + TWOPI * ele->coupler_phase;
  double gradient = ele->voltage == 0 ? 0.0 : (ele->l == 0 ? 1e30 : ele->voltage / ele->l);
  double field = ele->is_on ? gradient * 1.0 : 0.0;
  double dp_coef = field * ele->coupler_strength;
  double dp_x = dp_coef * cos(TWOPI * ele->coupler_angle);
  double dp_y = dp_coef * sin(TWOPI * ele->coupler_angle);
  if (ele->coupler_at == BGO_BOTH_ENDS) {
    dp_x = dp_x / 2;
    dp_y = dp_y / 2;
  }
  double c = P_COS(ph);
  orbit->vec[1] = orbit->vec[1] + 1 * dp_x * c / orbit->p0c;
  orbit->vec[3] = orbit->vec[3] + 1 * dp_y * c / orbit->p0c;
  double f2 = 1 * P_SIN(ph) * TWOPI * ele->rf_frequency / C_LIGHT;
  double dE = (dp_x * orbit->vec[0] + dp_y * orbit->vec[2]) * f2;
  LM(2);
  FL(16);
  apply_energy_kick(dE, orbit, param);
}

/* track_a_rfcavity, bmad/low_level/track_a_rfcavity.f90:17-146 with
 * particle_rf_time (bmad/code/particle_rf_time.f90:32-120) in relative-time
 * mode, rf_ref_time_offset = 0 (rf_ref_time_offset.f90:33) and no coupler
 * kick (rf_coupler_kick.f90:41 returns for coupler_strength = 0). */
static int track_a_rfcavity(bgo_coord* orbit, const bgo_ele* ele, const bgo_param* param) {
  double an[BGO_N_POLE], bn[BGO_N_POLE], ae[BGO_N_POLE], be[BGO_N_POLE];
  if (ele->rf_frequency == 0 && ele->voltage != 0) {
    orbit->state = BGO_LOST;
    return 0;
  }
  double length = ele->l * 1;
  int n_step = 1;
  double r_step = 1.0 / n_step;
  double step_len = length / n_step;
  int n_slice = nint_f(fabs(length) / ele->ds_step);
  if (n_slice < 1) n_slice = 1;
  double charge_dir = 1.0;
  int ix_mag_max = bgo_multipole_ele_to_ab(ele, 0, 0, 1, an, bn, NULL);
  int ix_elec_max = bgo_multipole_ele_to_ab(ele, 0, 1, 0, ae, be, NULL);
  if (ix_mag_max < -1 || ix_elec_max < -1) return -1;
  offset_particle(ele, 1, orbit, 1, 1, 0, 0, param);
  if (ix_mag_max > -1) ab_multipole_kicks(an, bn, ix_mag_max, ele, orbit, param, 0, 0.5 * r_step);
  if (ix_elec_max > -1) ab_multipole_kicks(ae, be, ix_elec_max, ele, orbit, param, 1, 0.5 * step_len);

  double voltage = (ele->is_on ? ele->voltage * 1 : 0.0) * charge_dir;
  double f = ele->rf_frequency;
  /* particle_rf_time (particle_rf_time.f90:74-90): with absolute time
   * tracking the particle time t less ref_time_start (absolute_time_ref_shift),
   * else the relative time -z / (beta * c_light) in real(rp); then modulo2
   * in real(qp) (:116-118).  rf_ref_time_offset is 0 for an element that is
   * not a slave (rf_ref_time_offset.f90:30-43). */
  __float128 time;
  if (param->absolute_time_tracking) {
    time = orbit->t;
    if (param->absolute_time_ref_shift) time = time - (__float128)ele->ref_time_start;
  } else {
    double time_dp = -orbit->vec[4] / (orbit->beta * C_LIGHT);
    time = (__float128)time_dp;
  }
  if (f != 0) time = modulo2_qp(time, ((__float128)0.5) / (__float128)f);
  __float128 ph = (__float128)TWOPI * ((__float128)ele->phi0 - (time - (__float128)0.0) * (__float128)f);
  double phase0 = (double)ph;
  /* no phi0_multipass with absolute time (track_a_rfcavity.f90:81) */
  if (!param->absolute_time_tracking) phase0 = phase0 + TWOPI * ele->phi0_multipass;
  double phase = modulo2_dp(phase0, PI);
  LM(0);
  FL(8);
  rf_coupler_kick(ele, 1, phase, orbit, param);

  for (int i = 0; i <= n_slice; i++) {
    double dE = 1 * voltage * P_SIN(phase) / n_slice;
    if (i == 0 || i == n_slice) dE = dE / 2;
    LM(1);
    FL(3);
    apply_energy_kick(dE, orbit, param);
    if (orbit->vec[5] == -1) {
      orbit->state = BGO_LOST_PZ;
      return 0;
    }
    if (i != n_slice) {
      double z = orbit->vec[4];
      track_a_drift(orbit, length / n_slice, 1, param);
      phase = phase + TWOPI * f * (orbit->vec[4] - z) / (C_LIGHT * orbit->beta);
      FL(7);
    }
  }
  rf_coupler_kick(ele, 0, phase, orbit, param);
  if (ix_elec_max > -1) ab_multipole_kicks(ae, be, ix_elec_max, ele, orbit, param, 1, 0.5 * step_len);
  if (ix_mag_max > -1) ab_multipole_kicks(an, bn, ix_mag_max, ele, orbit, param, 0, 0.5 * r_step);
  offset_particle(ele, 0, orbit, 1, 1, 0, 0, param);
  return 0;
}

/* track1_bmad, bmad/low_level/track1_bmad.f90:22-283 (subset). */
static int track1_bmad(bgo_coord* orbit, const bgo_ele* ele, bgo_param* param) {
  int key = ele->key;
  if (!ele->is_on) {
    switch (key) {
      case BGO_AB_MULTIPOLE: case BGO_MULTIPOLE: case BGO_MARKER:
        key = -1; /* do_nothing */
        break;
      case BGO_SBEND:
        break;
      default:
        key = BGO_DRIFT;
    }
  }
  switch (key) {
    case -1:
      return 0;
    case BGO_MARKER: /* track1_bmad.f90:123-125 */
      orbit->t = orbit->t + (__float128)ele->delta_ref_time;
      return 0;
    case BGO_RCOLLIMATOR: case BGO_ECOLLIMATOR: case BGO_MONITOR: case BGO_INSTRUMENT: case BGO_PIPE:
    case BGO_KICKER: case BGO_HKICKER: case BGO_VKICKER: case BGO_OCTUPOLE: case BGO_THICK_MULTIPOLE:
    case BGO_SEXTUPOLE:
      return track_a_thick_multipole(orbit, ele, param);
    case BGO_DRIFT:
      track_a_drift(orbit, ele->l * 1, 1, param);
      return 0;
    case BGO_MULTIPOLE: case BGO_AB_MULTIPOLE: {
      double knl[BGO_N_POLE], tl[BGO_N_POLE];
      if (ele->has_misalign) offset_particle(ele, 1, orbit, 0, 1, 0, 0, param);
      int ix = bgo_multipole_ele_to_kt(ele, 1, knl, tl);
      if (ix > -1) {
        for (int n = 0; n < BGO_N_POLE; n++) {
          if (knl[n] == 0) continue;
          multipole_kick(knl[n], tl[n], n, orbit, ele->key == BGO_MULTIPOLE);
        }
      }
      if (ele->has_misalign) offset_particle(ele, 0, orbit, 0, 1, 0, 0, param);
      return 0;
    }
    case BGO_QUADRUPOLE:
      return track_a_quadrupole(orbit, ele, param);
    case BGO_RFCAVITY:
      return track_a_rfcavity(orbit, ele, param);
    case BGO_SBEND:
      return track_a_bend(orbit, ele, param);
    default:
      return -1;
  }
}

void bgo_init_coord(bgo_coord* orb, const double vec[6], double p0c, const bgo_param* param) {
  for (int i = 0; i < 6; i++) orb->vec[i] = vec[i];
  orb->p0c = p0c;
  /* convert_pc_to: beta = pc / sqrt(pc**2 + mc2**2) */
  double pc = (1 + vec[5]) * p0c;
  orb->beta = pc / sqrt(pc * pc + param->mass * param->mass);
  orb->state = BGO_ALIVE;
  /* init_coord.f90:222 with ref_time = 0 */
  orb->t = (__float128)(0.0 - orb->vec[4] / (orb->beta * C_LIGHT));
}

/* track1, bmad/code/track1.f90:43-342 (no hooks, radiation, spin). */
void bgo_track1(bgo_coord* orb, const bgo_ele* ele, bgo_param* param) {
  if (orb->state != BGO_ALIVE) return;
  bgo_check_aperture_limit(orb, ele, 0, param);
  if (orb->state != BGO_ALIVE) return;
  if (track1_bmad(orb, ele, param)) {
    orb->state = -1; /* setup error: form not restated */
    return;
  }
  if (bgo_orbit_too_large(orb, param)) return;
  if (orb->state != BGO_ALIVE) return;
  bgo_check_aperture_limit(orb, ele, 1, param);
}

/* ------------------------------------------------------------------ */
/* Multi-turn driver.                                                  */
/* Turn loop: bsim/modules/lt_tracking_mod.f90:1631-1695; element loop:  */
/* bmad/multiparticle/beam_mod.f90:152-167; OpenMP over particles per    */
/* element: bmad/multiparticle/beam_utils.f90:69-74.                     */

static void track_one_particle(const bgo_ele* eles, int n_ele, bgo_param* p, double p0c, double* vec6, double* beta,
                               __float128* tt, int* state, int* ixe, int* ixt, long n, long i, int turn0,
                               int n_turns) {
  bgo_coord orb;
  for (int c = 0; c < 6; c++) orb.vec[c] = vec6[c * n + i];
  orb.beta = beta[i];
  orb.p0c = p0c;
  orb.state = state[i];
  orb.t = tt ? tt[i] : 0;
  if (orb.state != BGO_ALIVE) return;
  for (int t = turn0; t < turn0 + n_turns && orb.state == BGO_ALIVE; t++) {
    for (int e = 0; e < n_ele; e++) {
      bgo_track1(&orb, &eles[e], p);
      if (orb.state != BGO_ALIVE) {
        ixe[i] = eles[e].ix_ele;
        ixt[i] = t;
        break;
      }
    }
  }
  for (int c = 0; c < 6; c++) vec6[c * n + i] = orb.vec[c];
  beta[i] = orb.beta;
  state[i] = orb.state;
  if (tt) tt[i] = orb.t;
}

void bgo_track_turns(const bgo_ele* eles, int n_ele, const bgo_param* param, double p0c, double* vec6,
                     double* beta, __float128* tq, int* state, int* ix_ele_lost, int* ix_turn_lost, long n,
                     int turn0, int n_turns, int n_threads, int element_outer) {
  c_multi_init();
#ifdef _OPENMP
  if (n_threads > 0) omp_set_num_threads(n_threads);
#else
  (void)n_threads;
#endif
  if (!element_outer) {
#pragma omp parallel for schedule(dynamic, 64)
    for (long i = 0; i < n; i++) {
      bgo_param p = *param;
      track_one_particle(eles, n_ele, &p, p0c, vec6, beta, tq, state, ix_ele_lost, ix_turn_lost, n, i, turn0,
                         n_turns);
    }
    return;
  }
  /* Reference structure: element-outer, parallel over particles per element. */
  for (int t = turn0; t < turn0 + n_turns; t++) {
    for (int e = 0; e < n_ele; e++) {
#pragma omp parallel for schedule(static)
      for (long i = 0; i < n; i++) {
        if (state[i] != BGO_ALIVE) continue;
        bgo_param p = *param;
        bgo_coord orb;
        for (int c = 0; c < 6; c++) orb.vec[c] = vec6[c * n + i];
        orb.beta = beta[i];
        orb.p0c = p0c;
        orb.state = state[i];
        orb.t = tq ? tq[i] : 0;
        bgo_track1(&orb, &eles[e], &p);
        for (int c = 0; c < 6; c++) vec6[c * n + i] = orb.vec[c];
        beta[i] = orb.beta;
        state[i] = orb.state;
        if (tq) tq[i] = orb.t;
        if (orb.state != BGO_ALIVE) {
          ix_ele_lost[i] = eles[e].ix_ele;
          ix_turn_lost[i] = t;
        }
      }
    }
  }
}
