/*
 * bgt.h -- C ABI of libbgt, the B200 FP64 multi-particle tracker for Bmad
 * `bmad_standard` lattices.
 *
 * The entry points replace, for the tracking methods and element types listed
 * below, the reference's multi-particle tracking call surface:
 *
 *   bgt_track_turns   <- the turn loop of long_term_tracking in BEAM mode,
 *                        bsim/modules/lt_tracking_mod.f90:1631-1695, i.e.
 *                        ltt_track_bmad_bunch (:3186-3225) -> track_bunch
 *                        (bmad/multiparticle/beam_mod.f90:103-170) ->
 *                        track1_bunch_hom (beam_utils.f90:32-160) ->
 *                        track1 (bmad/code/track1.f90:43) per particle per
 *                        element.  Installed through track1_bunch_hook_ptr
 *                        (bmad/modules/bmad_routine_interface.f90:3927-3936)
 *                        or as a 'GPU' case of lttp%tracking_method
 *                        (lt_tracking_mod.f90:1636-1670).
 *   bgt_track_elements <- track_all / track_many over a contiguous range of
 *                        elements (bmad/code/track_all.f90:25,
 *                        bmad/code/track_many.f90:50), and, with a range of
 *                        one element, track1 (bmad/code/track1.f90:43).
 *   bgt_da_scan_grid  <- dynamic_aperture_scan / dynamic_aperture_point
 *                        (bmad/modules/dynamic_aperture_mod.f90:27,284) with
 *                        the bisection replaced by a polar amplitude grid.
 *
 * Conventions (kept from the reference so the shim is a pass-through):
 *  - Element keys, fringe_type, fringe_at/aperture_at and aperture_type use
 *    Bmad's integer codes (bmad/modules/bmad_struct.f90:157-168,372,1681-1695).
 *  - Particle state codes are Bmad's coord_struct%state codes
 *    (bmad_struct.f90:522-527): alive = 1, lost = 2, lost_neg_x = 3,
 *    lost_pos_x = 4, lost_neg_y = 5, lost_pos_y = 6, lost_pz = 8.
 *    A lost particle is a state, not an error (track1.f90:38-40).
 *  - Coordinates are Bmad phase-space coordinates (x, px, y, py, z, pz),
 *    stored structure-of-arrays: vec6[c * n + i] is coordinate c of particle i.
 *  - ix_ele_lost is the lost-at element's ix_ele (the `track_state` of
 *    track_all, track_all.f90:17-18); ix_turn_lost is the 0-based turn index in
 *    which the particle was lost (bunch%ix_turn before that turn,
 *    lt_tracking_mod.f90:1633).  Both stay -1 for particles that survive.
 *  - Every function returns 0 on success or a negative BGT_E* code; the
 *    message is available from bgt_last_error() on the same thread.
 *    Nothing aborts.
 *  - Host buffers are caller-owned; device buffers are owned by the handle or
 *    by the caller (the *_device entry points).
 *
 * Threading.  The reference calls track1 from OpenMP threads
 * (bmad/multiparticle/beam_utils.f90:69-74) and track_many from the parallel
 * sections of its DA scan (bmad/modules/dynamic_aperture_mod.f90:163-196).
 * Every entry point that takes a handle is re-entrant: any number of threads
 * may call it on one handle at the same time.  Each call takes a context of
 * its own from the handle's pool -- a library-owned stream, staging buffers
 * and the kernel's tile counter and error flag -- so concurrent calls never
 * share buffers; the host-buffer calls wait for their own stream only (no
 * device-wide synchronisation).  Device-buffer calls run on the caller's
 * stream, ordered after the previous GPU work of the context they use, and
 * are serialised per stream as CUDA orders them.  bgt_set_tuning takes
 * effect for calls that start after it returns.  bgt_destroy must not run
 * concurrently with other calls on the same handle.
 *
 * Scope: forward tracking (direction = time_dir = orientation = +1), relative
 * or absolute RF time (bmad_com%absolute_time_tracking), magnetic and electric
 * multipoles (electric ones on quadrupoles, sextupoles, octupoles, thick
 * multipoles and bends), misaligned elements including bends, the bend
 * edges of every fringe type (the exact PTC edge of fringe_type full
 * included), RF coupler kicks, no radiation/spin, no exact bend multipoles.
 * bgt_create rejects any element outside that scope with BGT_EUNSUPPORTED
 * and names the element.
 */
#ifndef BGT_H
#define BGT_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define BGT_N_POLE 22 /* n_pole_maxx + 1, bmad_struct.f90:48 */

/* Bmad element keys (bmad_struct.f90:1681-1695). */
enum {
  BGT_DRIFT = 1,
  BGT_SBEND = 2,
  BGT_QUADRUPOLE = 3,
  BGT_SEXTUPOLE = 5,
  BGT_RFCAVITY = 9,
  BGT_MARKER = 14,
  BGT_KICKER = 15,
  BGT_OCTUPOLE = 17,
  BGT_MULTIPOLE = 19,
  BGT_AB_MULTIPOLE = 22,
  BGT_MONITOR = 31,
  BGT_INSTRUMENT = 32,
  BGT_HKICKER = 33,
  BGT_VKICKER = 34,
  BGT_RCOLLIMATOR = 35,
  BGT_ECOLLIMATOR = 36,
  BGT_PIPE = 44,
  BGT_THICK_MULTIPOLE = 67
};

/* fringe_type (bmad_struct.f90:164-168); 1 = none$ */
enum { BGT_FRINGE_NONE = 1, BGT_FRINGE_SOFT_EDGE_ONLY = 2, BGT_FRINGE_HARD_EDGE_ONLY = 3,
       BGT_FRINGE_FULL = 4, BGT_FRINGE_SAD_FULL = 5, BGT_FRINGE_LINEAR_EDGE = 6, BGT_FRINGE_BASIC_BEND = 7 };
/* fringe_at / aperture_at (bmad_struct.f90:372) */
enum { BGT_ENTRANCE_END = 1, BGT_EXIT_END = 2, BGT_BOTH_ENDS = 3, BGT_NO_END = 4 };
/* aperture_type (bmad_struct.f90:157); 0 = no aperture limits set */
enum { BGT_APERTURE_NONE = 0, BGT_APERTURE_RECTANGULAR = 2, BGT_APERTURE_ELLIPTICAL = 3 };

/* coord_struct%state (bmad_struct.f90:522-527) */
enum { BGT_ALIVE = 1, BGT_LOST = 2, BGT_LOST_NEG_X = 3, BGT_LOST_POS_X = 4, BGT_LOST_NEG_Y = 5,
       BGT_LOST_POS_Y = 6, BGT_LOST_PZ = 8 };

/* error codes */
enum { BGT_OK = 0, BGT_EINVAL = -1, BGT_EUNSUPPORTED = -2, BGT_ECUDA = -3, BGT_ENOMEM = -4,
       BGT_ETIMEOUT = -5, BGT_ETOOLARGE = -6 };

/*
 * One lattice element, i.e. the ele_struct fields the bmad_standard path
 * reads (ele%value(...) entries by name, bmad_struct.f90:1762-1879).
 * an/bn and an_elec/bn_elec are what
 *   multipole_ele_to_ab(ele, .false., ix, an, bn, magnetic$, include_kicks$)
 *   multipole_ele_to_ab(ele, .false., ix, an_elec, bn_elec, electric$)
 * return (bmad/code/multipole_ele_to_ab.f90:31) -- b1 NOT pulled out; the
 * library pulls it where track_a_quadrupole / track_a_bend do.  knl/tn are
 * multipole_ele_to_kt(ele, .true., ix, knl, tn) (multipole_ele_to_kt.f90:29),
 * used by multipole and ab_multipole elements.
 */
typedef struct bgt_element {
  int32_t key;
  int32_t ix_ele;
  int32_t is_on;
  int32_t num_steps;
  int32_t fringe_type;
  int32_t fringe_at;
  int32_t aperture_type;
  int32_t aperture_at;
  int32_t offset_moves_aperture;
  int32_t exact_multipoles; /* 0 = off$ */
  int32_t has_misalign;     /* ele%bookkeeping_state%has_misalign */
  int32_t coupler_at;       /* rfcavity: coupler_at (end codes as fringe_at; default exit end) */
  double l, k1, k2, k3, g, dg, e1, e2, fint, hgap, fintx, hgapx;
  double voltage, phi0, phi0_multipass, rf_frequency, coupler_strength;
  double p0c, e_tot, ds_step;
  double x_offset, y_offset, z_offset, x_pitch, y_pitch, tilt, ref_tilt, roll;
  double hkick, vkick, kick;
  double x1_limit, x2_limit, y1_limit, y2_limit;
  double an[BGT_N_POLE], bn[BGT_N_POLE];
  double an_elec[BGT_N_POLE], bn_elec[BGT_N_POLE];
  double knl[BGT_N_POLE], tn[BGT_N_POLE];
  double coupler_angle, coupler_phase; /* rfcavity coupler (with coupler_strength) */
  double fq1, fq2;                     /* quadrupole soft-edge fringe integrals */
  /* ecollimator / rcollimator momentum and longitudinal limits
   * (check_aperture_limit.f90:98-135); width2 = 0: no limit */
  double px_aperture_width2, px_aperture_center, py_aperture_width2, py_aperture_center;
  double z_aperture_width2, z_aperture_center, pz_aperture_width2, pz_aperture_center;
  /* reference time through the element and at its entrance
   * (ele%value(delta_ref_time$), ele%value(ref_time_start$), set by
   * lat_compute_reference_energy.f90): the particle time's per-element step
   * and, with absolute time tracking, the origin of the RF phase */
  double delta_ref_time, ref_time_start;
} bgt_element;

/* Tracked species (lat%param%particle) and bmad_com switches. */
typedef struct bgt_species {
  double mass;               /* mass_of(species) [eV] */
  int32_t charge;            /* charge_of(species) [e] */
  int32_t aperture_limit_on; /* bmad_com%aperture_limit_on (default 1) */
  double max_aperture_limit; /* bmad_com%max_aperture_limit (default 1e3 m) */
  int32_t absolute_time_tracking;  /* bmad_com%absolute_time_tracking (default 0): the RF phase
                                      from the particle time t instead of -z / (beta c) */
  int32_t absolute_time_ref_shift; /* bmad_com%absolute_time_ref_shift (default 1) */
} bgt_species;

/* Launch tiles chosen by the autotuner (0 = let the library choose). */
typedef struct bgt_tuning {
  int32_t threads_per_block; /* particles per CTA */
  int32_t blocks_per_sm;     /* resident CTAs per SM for the persistent grid */
  int32_t turns_per_launch;  /* turns per persistent-kernel launch (graph node) */
  int32_t compact_every;     /* compact lost particles every this many turns (0 = never) */
  int32_t table_mode;        /* element table: 0 = staged in shared memory when it fits, else read
                                from global memory; 1 = shared memory only; 2 = global memory;
                                3 = global memory with every warp scheduled on its own (no
                                CTA-wide tiles: for small, long-lived particle sets) */
  int32_t wait_limit_us;     /* bound of the kernel's wait for its element-table copy, in
                                microseconds (0 = 2 s); when it runs out the kernel sets its error
                                flag and returns: BGT_ETIMEOUT from host-buffer calls, from
                                bgt_device_status for device-buffer calls */
  int32_t test_skip_table_copy; /* tests only: 1 = arm the table copy's barrier but issue no copy,
                                   so every staging wait runs out (exercises the bounded wait and
                                   the error path); 0 in normal use */
} bgt_tuning;

typedef struct bgt_handle bgt_handle;

/*
 * Flattens n_variants lattices of n_ele elements each (eles[v * n_ele + e])
 * into the device element tables (structure-of-records, one table per
 * variant).  Each variant is a copy of the same ring with its own element
 * values (error seeds, sextupole settings).  `device` is the CUDA ordinal.
 */
int bgt_create(bgt_handle** out, const bgt_element* eles, int32_t n_ele, int32_t n_variants,
               const bgt_species* species, int32_t device);
int bgt_destroy(bgt_handle* h);
const char* bgt_last_error(const bgt_handle* h);

/* Table bytes per variant and the tuning currently in use. */
int bgt_table_info(const bgt_handle* h, int64_t* table_bytes, int32_t* n_records);
int bgt_set_tuning(bgt_handle* h, const bgt_tuning* t);
int bgt_get_tuning(const bgt_handle* h, bgt_tuning* t);

/*
 * Track n particles for n_turns turns starting at turn index turn0, in place.
 * HOST buffers (the long_term_tracking drop-in): vec6[6*n], beta[n] (FP64),
 * state/ix_ele_lost/ix_turn_lost[n] (int32).  variant[n] selects each
 * particle's lattice variant (NULL = variant 0).  Particles whose state is
 * not alive are left untouched.  Copies in, tracks, copies out.
 *
 * t (may be NULL) is the particle time coord_struct%t: n IEEE binary128
 * values (16 bytes each: a Fortran real(qp) array or C __float128[n]),
 * advanced in every element in binary128 arithmetic exactly as the
 * reference advances it (track_a_drift.f90:79-80,
 * track_a_quadrupole.f90:144, track_a_bend.f90:327,
 * track_a_thick_multipole.f90:133).  It is required with absolute time
 * tracking, where the RF phase comes from it (particle_rf_time.f90:74-76).
 * Tracking time runs the RARE kernel instances.
 */
int bgt_track_turns(bgt_handle* h, double* vec6, double* beta, void* t, int32_t* state, int32_t* ix_ele_lost,
                    int32_t* ix_turn_lost, const int32_t* variant, int64_t n, int32_t turn0, int32_t n_turns);

/*
 * Same, DEVICE buffers already resident in HBM, enqueued on `stream`
 * (a cudaStream_t, NULL = legacy default stream); d_t as t above, in device
 * memory.  Asynchronous: a staging timeout on the device is reported by
 * bgt_device_status.
 * Uses library-owned scratch sized on first use (grown as needed).
 * d_variant (device int32[n], may be NULL = variant 0) must be sorted
 * (non-decreasing); with it and more than one variant the call counts the
 * particles per variant on the device and synchronises `stream` once to read
 * the counts back (BGT_EINVAL for unsorted or out-of-range ids).
 */
int bgt_track_turns_device(bgt_handle* h, double* d_vec6, double* d_beta, void* d_t, int32_t* d_state,
                           int32_t* d_ix_ele_lost, int32_t* d_ix_turn_lost, const int32_t* d_variant, int64_t n,
                           int32_t turn0, int32_t n_turns, void* stream);

/*
 * Waits for `stream` and reports whether any device-buffer call on this
 * handle hit a table-staging timeout on the device since the last check
 * (BGT_ETIMEOUT), clearing the flag; 0 otherwise.  The device-side
 * counterpart of the err_flag the reference's tracking routines return
 * (track1.f90:38-40 keeps particle loss a state, not an error).
 */
int bgt_device_status(bgt_handle* h, void* stream);

/*
 * Track n particles through table elements [e_begin, e_end) of their variant
 * once (no turn wrap), HOST buffers (t as for bgt_track_turns).
 * e_end - e_begin == 1 is track1
 * (bmad/code/track1.f90:43) including its two check_aperture_limit calls.
 */
int bgt_track_elements(bgt_handle* h, double* vec6, double* beta, void* t, int32_t* state, int32_t* ix_ele_lost,
                       const int32_t* variant, int64_t n, int32_t e_begin, int32_t e_end);

/*
 * Dynamic-aperture scan on a polar grid, one launch for all variants:
 * for each variant v, momentum offset d (n_delta of them), angle a (n_angle
 * in [angle_min, angle_max]) and radius r (n_radius from 0 to r_max), the
 * particle starts at ref_orbit[(v * n_delta + d) * 6 + c] -- the reference
 * orbit of variant v at the d-th momentum offset: its closed orbit with pz
 * set to that offset, plus eta*pz when the caller includes it, as
 * dynamic_aperture_mod.f90:132-140 forms it -- plus (r cos a, 0,
 * r sin a * y_scale, 0, 0, 0), and is tracked n_turns turns.  The
 * momentum offsets are part of ref_orbit (its pz entries).
 * da_radius[((v * n_delta) + d) * n_angle + a] receives
 * the largest grid radius below the first lost one along that ray (the
 * lower bracket x0 of dynamic_aperture_point, dynamic_aperture_mod.f90:
 * 335-388); survive_turns (optional, may be NULL) receives, per particle in
 * (v, d, a, r) order, the turns survived (n_turns if never lost).
 */
int bgt_da_scan_grid(bgt_handle* h, const double* ref_orbit, int32_t n_variants_used, int32_t n_delta,
                     int32_t n_angle, double angle_min, double angle_max, int32_t n_radius, double r_max,
                     double y_scale, int32_t n_turns, double* da_radius, int32_t* survive_turns);

/* Number of this library's kernels launched since the handle was created. */
int64_t bgt_kernel_launch_count(const bgt_handle* h);

/*
 * Allocation-free variant of bgt_track_turns_device (no counterpart in the
 * reference).  For callers that cannot let this library allocate device
 * memory: hosts whose framework owns the GPU's memory through its own
 * caching allocator, and loops that must not allocate per call.  It needs no
 * handle: it compiles the n_ele elements (one lattice) on the host, copies
 * the table into a fixed device array inside the library, and tracks the
 * caller's device particle arrays in place on `stream`.  It never calls
 * cudaMalloc or cudaFree.
 *
 * Limits: the array holds 256 KiB (table plus a 256-byte header) on every
 * GPU that loads the library, until the process exits; larger tables are
 * rejected with BGT_ETOOLARGE.  A table that fits the array but not the
 * kernel's shared memory is read in place from the array.  Every call
 * reuses the same array and leaves its contents behind, so calls that
 * overlap on the GPU (other streams or threads) race: serialise them.  The
 * first call on a device looks up the array's address and uploads constant
 * tables; make it before any stream capture.  It carries no particle
 * times, so a species with absolute time tracking is refused
 * (BGT_EUNSUPPORTED).  tuning may be NULL; otherwise
 * (threads, CTAs per SM) must be (128, 4) or (256, 2), checked before
 * anything is enqueued (table_mode is ignored).  d_status (device int32, may
 * be NULL) receives, in stream order, the call's error flag: 1 when a
 * table-staging wait on the device ran out, else 0.  The caller's current
 * device is left as it was.  On error a message is written to err (err_len
 * bytes).
 */
int bgt_track_turns_device_noalloc(const bgt_element* eles, int32_t n_ele, const bgt_species* species,
                                   double* d_vec6, double* d_beta, int32_t* d_state, int32_t* d_ix_ele_lost,
                                   int32_t* d_ix_turn_lost, int64_t n, int32_t turn0, int32_t n_turns,
                                   const bgt_tuning* tuning, int32_t device, void* stream, int32_t* d_status,
                                   char* err, int32_t err_len);

/* Measured FP64 FMA throughput of `device` in TFLOP/s (2 flops per FMA):
 * the roofline denominator for the tracking kernel.  No reference
 * counterpart (measurement helper). */
int bgt_fp64_peak_tflops(int32_t device, double* tflops);

#ifdef __cplusplus
}
#endif
#endif
