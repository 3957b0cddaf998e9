!+
! Module bgt_mod
!
! Fortran (ISO_C_BINDING) side of libbgt, the B200 FP64 tracker for Bmad's
! bmad_standard element-by-element path.  The C ABI is include/bgt.h; every
! interface below mirrors one of its prototypes, and the derived types mirror
! its structs field for field (bind(c): the same layout as the C compiler's).
!
! What Bmad code calls:
!   bgt_ring_init          -- flatten a branch (one turn starting after a given
!                             element) into the library's element table once
!   bgt_track_bunch_turns  -- a whole bunch, n turns, on the GPU: the 'GPU'
!                             case of ltt_run_beam_mode
!                             (bsim/modules/lt_tracking_mod.f90:1636-1670;
!                             include file bgt_ltt_gpu_case.inc)
!   bgt_track_one_turn     -- one particle, one turn: the 'GPU' case of the
!                             dynamic_aperture program's track_many_hook
!                             (bsim/dynamic_aperture/track_many_hook.f90:69-95;
!                             include file bgt_track_many_gpu_case.inc)
!   bgt_ring_free          -- release the handle
!
! Elements and particles are passed in Bmad's own units and integer codes
! (coord_struct%t as the real(qp) array the library's time argument takes);
! multipole arrays come from Bmad's multipole_ele_to_ab / multipole_ele_to_kt,
! so the library sees exactly what track1 would use.  Particle loss is a
! state (coord_struct%state), not an error; err_flag is set only when the
! library refuses the lattice (an element outside its scope: the caller keeps
! Bmad's own tracking) or a CUDA call fails.
!
! Needs gfortran (or another Fortran 2008 compiler), a Bmad build (module
! bmad) and libbgt.so at link time.
!-

module bgt_mod

use iso_c_binding
use bmad

implicit none

integer, parameter :: bgt_n_pole = n_pole_maxx + 1

! Return codes (bgt.h).
integer(c_int), parameter :: bgt_ok$ = 0, bgt_einval$ = -1, bgt_eunsupported$ = -2, bgt_ecuda$ = -3, &
                             bgt_enomem$ = -4, bgt_etimeout$ = -5, bgt_etoolarge$ = -6

! bgt_element (bgt.h): the ele_struct values the bmad_standard path reads.
type, bind(c) :: bgt_element_c
  integer(c_int32_t) :: key, ix_ele, is_on, num_steps, fringe_type, fringe_at, aperture_type, aperture_at
  integer(c_int32_t) :: offset_moves_aperture, exact_multipoles, has_misalign, coupler_at
  real(c_double) :: l, k1, k2, k3, g, dg, e1, e2, fint, hgap, fintx, hgapx
  real(c_double) :: voltage, phi0, phi0_multipass, rf_frequency, coupler_strength
  real(c_double) :: p0c, e_tot, ds_step
  real(c_double) :: x_offset, y_offset, z_offset, x_pitch, y_pitch, tilt, ref_tilt, roll
  real(c_double) :: hkick, vkick, kick
  real(c_double) :: x1_limit, x2_limit, y1_limit, y2_limit
  real(c_double) :: an(bgt_n_pole), bn(bgt_n_pole), an_elec(bgt_n_pole), bn_elec(bgt_n_pole)
  real(c_double) :: knl(bgt_n_pole), tn(bgt_n_pole)
  real(c_double) :: coupler_angle, coupler_phase
  real(c_double) :: fq1, fq2
  real(c_double) :: px_aperture_width2, px_aperture_center, py_aperture_width2, py_aperture_center
  real(c_double) :: z_aperture_width2, z_aperture_center, pz_aperture_width2, pz_aperture_center
  real(c_double) :: delta_ref_time, ref_time_start
end type

! bgt_species (bgt.h): the tracked species and the bmad_com switches used.
type, bind(c) :: bgt_species_c
  real(c_double) :: mass
  integer(c_int32_t) :: charge, aperture_limit_on
  real(c_double) :: max_aperture_limit
  integer(c_int32_t) :: absolute_time_tracking, absolute_time_ref_shift
end type

! bgt_tuning (bgt.h); all zero = the library's defaults.
type, bind(c) :: bgt_tuning_c
  integer(c_int32_t) :: threads_per_block, blocks_per_sm, turns_per_launch, compact_every, table_mode
  integer(c_int32_t) :: wait_limit_us, test_skip_table_copy
end type

interface
  integer(c_int) function bgt_create(h, eles, n_ele, n_variants, species, device) bind(c, name='bgt_create')
    import
    type(c_ptr) :: h
    type(bgt_element_c) :: eles(*)
    integer(c_int32_t), value :: n_ele, n_variants, device
    type(bgt_species_c) :: species
  end function
  integer(c_int) function bgt_destroy(h) bind(c, name='bgt_destroy')
    import
    type(c_ptr), value :: h
  end function
  type(c_ptr) function bgt_last_error(h) bind(c, name='bgt_last_error')
    import
    type(c_ptr), value :: h
  end function
  integer(c_int) function bgt_set_tuning(h, t) bind(c, name='bgt_set_tuning')
    import
    type(c_ptr), value :: h
    type(bgt_tuning_c) :: t
  end function
  integer(c_int) function bgt_track_turns(h, vec6, beta, t, state, ix_ele_lost, ix_turn_lost, variant, n, &
                                          turn0, n_turns) bind(c, name='bgt_track_turns')
    import
    type(c_ptr), value :: h, variant
    real(c_double) :: vec6(*), beta(*)
    real(qp) :: t(*)
    integer(c_int32_t) :: state(*), ix_ele_lost(*), ix_turn_lost(*)
    integer(c_int64_t), value :: n
    integer(c_int32_t), value :: turn0, n_turns
  end function
  integer(c_int) function bgt_track_elements(h, vec6, beta, t, state, ix_ele_lost, variant, n, e_begin, e_end) &
                                             bind(c, name='bgt_track_elements')
    import
    type(c_ptr), value :: h, variant
    real(c_double) :: vec6(*), beta(*)
    real(qp) :: t(*)
    integer(c_int32_t) :: state(*), ix_ele_lost(*)
    integer(c_int64_t), value :: n
    integer(c_int32_t), value :: e_begin, e_end
  end function
  integer(c_int) function bgt_da_scan_grid(h, ref_orbit, n_variants_used, n_delta, n_angle, angle_min, &
                      angle_max, n_radius, r_max, y_scale, n_turns, da_radius, survive_turns) &
                      bind(c, name='bgt_da_scan_grid')
    import
    type(c_ptr), value :: h, survive_turns
    real(c_double) :: ref_orbit(*), da_radius(*)
    integer(c_int32_t), value :: n_variants_used, n_delta, n_angle, n_radius, n_turns
    real(c_double), value :: angle_min, angle_max, r_max, y_scale
  end function
  integer(c_size_t) function bgt_c_strlen(s) bind(c, name='strlen')
    import
    type(c_ptr), value :: s
  end function
end interface

! One tracking ring per process: the branch flattened into one turn that
! starts after element ix_start (usually 0, the beginning).
type bgt_ring_struct
  type(c_ptr) :: h = c_null_ptr
  integer :: ix_branch = -1
  integer :: ix_start = -1
  integer :: n_ele = 0
end type

type(bgt_ring_struct), save, target :: bgt_ring_global

contains

!+
! Function bgt_error_string (h) result (str)
!
! The library's message for the last failed call on this thread.
!-

function bgt_error_string (h) result (str)
type(c_ptr), value :: h
character(:), allocatable :: str
type(c_ptr) p
character(kind=c_char), pointer :: chars(:)
integer n, i

p = bgt_last_error(h)
if (.not. c_associated(p)) then
  str = ''
  return
endif
n = int(bgt_c_strlen(p))
call c_f_pointer(p, chars, [n])
allocate (character(n) :: str)
do i = 1, n
  str(i:i) = chars(i)
enddo
end function bgt_error_string

!+
! Subroutine bgt_flatten (branch, ix_start, eles)
!
! One turn of branch%ele(1:n_ele_track), starting after element ix_start
! (ix_start+1 .. n_ele_track, then 1 .. ix_start), into the C element array.
! The (a, b) arrays come from Bmad's own multipole_ele_to_ab /
! multipole_ele_to_kt; offsets are the *_tot values.
!-

subroutine bgt_flatten (branch, ix_start, eles)
type (branch_struct), target :: branch
integer ix_start
type (bgt_element_c) eles(:)
type (ele_struct), pointer :: ele
real(rp) a(0:n_pole_maxx), b(0:n_pole_maxx)
integer i, k, ix

do k = 1, branch%n_ele_track
  i = modulo(ix_start + k - 1, branch%n_ele_track) + 1
  ele => branch%ele(i)
  eles(k)%key = ele%key
  eles(k)%ix_ele = ele%ix_ele
  eles(k)%is_on = merge(1, 0, ele%is_on)
  eles(k)%num_steps = nint(ele%value(num_steps$))
  eles(k)%fringe_type = nint(ele%value(fringe_type$))
  eles(k)%fringe_at = nint(ele%value(fringe_at$))
  eles(k)%aperture_type = ele%aperture_type
  eles(k)%aperture_at = ele%aperture_at
  eles(k)%offset_moves_aperture = merge(1, 0, ele%offset_moves_aperture)
  eles(k)%exact_multipoles = nint(ele%value(exact_multipoles$))
  eles(k)%has_misalign = merge(1, 0, ele%bookkeeping_state%has_misalign)
  eles(k)%coupler_at = nint(ele%value(coupler_at$))
  eles(k)%l = ele%value(l$)
  eles(k)%k1 = ele%value(k1$)
  eles(k)%k2 = ele%value(k2$)
  eles(k)%k3 = ele%value(k3$)
  eles(k)%g = ele%value(g$)
  eles(k)%dg = ele%value(dg$)
  eles(k)%e1 = ele%value(e1$)
  eles(k)%e2 = ele%value(e2$)
  eles(k)%fint = ele%value(fint$)
  eles(k)%hgap = ele%value(hgap$)
  eles(k)%fintx = ele%value(fintx$)
  eles(k)%hgapx = ele%value(hgapx$)
  eles(k)%voltage = ele%value(voltage$)
  eles(k)%phi0 = ele%value(phi0$)
  eles(k)%phi0_multipass = ele%value(phi0_multipass$)
  eles(k)%rf_frequency = ele%value(rf_frequency$)
  eles(k)%coupler_strength = ele%value(coupler_strength$)
  eles(k)%p0c = ele%value(p0c$)
  eles(k)%e_tot = ele%value(e_tot$)
  eles(k)%ds_step = ele%value(ds_step$)
  eles(k)%x_offset = ele%value(x_offset_tot$)
  eles(k)%y_offset = ele%value(y_offset_tot$)
  eles(k)%z_offset = ele%value(z_offset_tot$)
  eles(k)%x_pitch = ele%value(x_pitch_tot$)
  eles(k)%y_pitch = ele%value(y_pitch_tot$)
  eles(k)%tilt = ele%value(tilt_tot$)
  eles(k)%ref_tilt = ele%value(ref_tilt_tot$)
  eles(k)%roll = ele%value(roll_tot$)
  eles(k)%hkick = ele%value(hkick$)
  eles(k)%vkick = ele%value(vkick$)
  eles(k)%kick = ele%value(kick$)
  eles(k)%x1_limit = ele%value(x1_limit$)
  eles(k)%x2_limit = ele%value(x2_limit$)
  eles(k)%y1_limit = ele%value(y1_limit$)
  eles(k)%y2_limit = ele%value(y2_limit$)
  eles(k)%coupler_angle = ele%value(coupler_angle$)
  eles(k)%coupler_phase = ele%value(coupler_phase$)
  eles(k)%fq1 = ele%value(fq1$)
  eles(k)%fq2 = ele%value(fq2$)
  eles(k)%px_aperture_width2 = ele%value(px_aperture_width2$)
  eles(k)%px_aperture_center = ele%value(px_aperture_center$)
  eles(k)%py_aperture_width2 = ele%value(py_aperture_width2$)
  eles(k)%py_aperture_center = ele%value(py_aperture_center$)
  eles(k)%z_aperture_width2 = ele%value(z_aperture_width2$)
  eles(k)%z_aperture_center = ele%value(z_aperture_center$)
  eles(k)%pz_aperture_width2 = ele%value(pz_aperture_width2$)
  eles(k)%pz_aperture_center = ele%value(pz_aperture_center$)
  eles(k)%delta_ref_time = ele%value(delta_ref_time$)
  eles(k)%ref_time_start = ele%value(ref_time_start$)
  eles(k)%an = 0;  eles(k)%bn = 0;  eles(k)%an_elec = 0;  eles(k)%bn_elec = 0
  eles(k)%knl = 0;  eles(k)%tn = 0
  if (ele%key == multipole$ .or. ele%key == ab_multipole$) then
    call multipole_ele_to_kt(ele, .true., ix, a, b)
    eles(k)%knl = a
    eles(k)%tn = b
  else
    call multipole_ele_to_ab(ele, .false., ix, a, b, magnetic$, include_kicks$)
    eles(k)%an = a
    eles(k)%bn = b
    call multipole_ele_to_ab(ele, .false., ix, a, b, electric$)
    eles(k)%an_elec = a
    eles(k)%bn_elec = b
  endif
enddo
end subroutine bgt_flatten

!+
! Subroutine bgt_ring_init (branch, ix_start, err_flag)
!
! Makes bgt_ring_global track one turn of `branch` starting after element
! ix_start, creating the library handle on the first call (or when the
! branch or start changes).  err_flag = .true. when the library refuses the
! lattice; its message is printed.
!-

subroutine bgt_ring_init (branch, ix_start, err_flag)
type (branch_struct), target :: branch
integer ix_start
logical err_flag
type (bgt_element_c), allocatable :: eles(:)
type (bgt_species_c) sp
integer(c_int) rc
character(*), parameter :: r_name = 'bgt_ring_init'

err_flag = .false.
if (c_associated(bgt_ring_global%h) .and. bgt_ring_global%ix_branch == branch%ix_branch .and. &
    bgt_ring_global%ix_start == ix_start .and. bgt_ring_global%n_ele == branch%n_ele_track) return
call bgt_ring_free()

allocate (eles(branch%n_ele_track))
call bgt_flatten (branch, ix_start, eles)
sp%mass = mass_of(branch%param%particle)
sp%charge = charge_of(branch%param%particle)
sp%aperture_limit_on = merge(1, 0, bmad_com%aperture_limit_on)
sp%max_aperture_limit = bmad_com%max_aperture_limit
sp%absolute_time_tracking = merge(1, 0, bmad_com%absolute_time_tracking)
sp%absolute_time_ref_shift = merge(1, 0, bmad_com%absolute_time_ref_shift)
rc = bgt_create(bgt_ring_global%h, eles, int(branch%n_ele_track, c_int32_t), 1_c_int32_t, sp, 0_c_int32_t)
if (rc /= bgt_ok$) then
  call out_io (s_error$, r_name, 'libbgt refused the lattice: ' // bgt_error_string(c_null_ptr))
  bgt_ring_global%h = c_null_ptr
  err_flag = .true.
  return
endif
bgt_ring_global%ix_branch = branch%ix_branch
bgt_ring_global%ix_start = ix_start
bgt_ring_global%n_ele = branch%n_ele_track
end subroutine bgt_ring_init

!+
! Subroutine bgt_ring_free ()
!-

subroutine bgt_ring_free ()
integer(c_int) rc
if (c_associated(bgt_ring_global%h)) rc = bgt_destroy(bgt_ring_global%h)
bgt_ring_global%h = c_null_ptr
bgt_ring_global%ix_branch = -1
bgt_ring_global%ix_start = -1
bgt_ring_global%n_ele = 0
end subroutine bgt_ring_free

!+
! Subroutine bgt_track_bunch_turns (branch, ele_start, bunch, i_turn, n_turns, err_flag)
!
! Tracks every alive particle of the bunch n_turns turns from ele_start on
! the GPU (what ltt_track_bmad_bunch does for one turn: track1 per particle
! per element, lt_tracking_mod.f90:3186-3225).  Coordinates, beta and state
! come back in place; a particle lost here gets ix_ele = the lost-at element
! (track_all's track_state).  i_turn is the turn index before tracking
! (bunch%ix_turn).
!-

subroutine bgt_track_bunch_turns (branch, ele_start, bunch, i_turn, n_turns, err_flag)
type (branch_struct), target :: branch
type (ele_struct) ele_start
type (bunch_struct), target :: bunch
integer i_turn, n_turns
logical err_flag
type (coord_struct), pointer :: p
real(c_double), allocatable :: vec6(:), beta(:)
real(qp), allocatable :: t(:)
integer(c_int32_t), allocatable :: state(:), ix_ele_lost(:), ix_turn_lost(:)
integer(c_int) rc
integer n, ip, c
character(*), parameter :: r_name = 'bgt_track_bunch_turns'

call bgt_ring_init (branch, ele_start%ix_ele, err_flag)
if (err_flag) return
n = size(bunch%particle)
if (n == 0) return
allocate (vec6(6*n), beta(n), t(n), state(n), ix_ele_lost(n), ix_turn_lost(n))
do ip = 1, n
  p => bunch%particle(ip)
  do c = 1, 6
    vec6((c-1)*n + ip) = p%vec(c)
  enddo
  beta(ip) = p%beta
  t(ip) = p%t
  state(ip) = p%state
  ix_ele_lost(ip) = -1
  ix_turn_lost(ip) = -1
enddo
rc = bgt_track_turns(bgt_ring_global%h, vec6, beta, t, state, ix_ele_lost, ix_turn_lost, c_null_ptr, &
                     int(n, c_int64_t), int(i_turn, c_int32_t), int(n_turns, c_int32_t))
if (rc /= bgt_ok$) then
  call out_io (s_error$, r_name, 'libbgt: ' // bgt_error_string(bgt_ring_global%h))
  err_flag = .true.
  return
endif
do ip = 1, n
  p => bunch%particle(ip)
  if (p%state /= alive$) cycle
  do c = 1, 6
    p%vec(c) = vec6((c-1)*n + ip)
  enddo
  p%beta = beta(ip)
  p%t = t(ip)
  p%state = state(ip)
  if (p%state /= alive$) p%ix_ele = ix_ele_lost(ip)
enddo
end subroutine bgt_track_bunch_turns

!+
! Subroutine bgt_track_one_turn (branch, ele_start, orb, err_flag)
!
! One particle, one turn from ele_start back to it on the GPU: what
! ltt_track_bmad_single does in the dynamic_aperture program's
! track_many_hook (track_many_hook.f90:69-95).  For a whole scan,
! bgt_da_scan_grid tracks every probe of every angle in one launch instead.
!-

subroutine bgt_track_one_turn (branch, ele_start, orb, err_flag)
type (branch_struct), target :: branch
type (ele_struct) ele_start
type (coord_struct) orb
logical err_flag
real(c_double) vec6(6), beta(1)
real(qp) t(1)
integer(c_int32_t) state(1), ix_ele_lost(1), ix_turn_lost(1)
integer(c_int) rc
character(*), parameter :: r_name = 'bgt_track_one_turn'

call bgt_ring_init (branch, ele_start%ix_ele, err_flag)
if (err_flag) return
if (orb%state /= alive$) return
vec6 = orb%vec
beta(1) = orb%beta
t(1) = orb%t
state(1) = orb%state
ix_ele_lost(1) = -1
ix_turn_lost(1) = -1
rc = bgt_track_turns(bgt_ring_global%h, vec6, beta, t, state, ix_ele_lost, ix_turn_lost, c_null_ptr, &
                     1_c_int64_t, 0_c_int32_t, 1_c_int32_t)
if (rc /= bgt_ok$) then
  call out_io (s_error$, r_name, 'libbgt: ' // bgt_error_string(bgt_ring_global%h))
  err_flag = .true.
  return
endif
orb%vec = vec6
orb%beta = beta(1)
orb%t = t(1)
orb%state = state(1)
if (orb%state /= alive$) orb%ix_ele = ix_ele_lost(1)
end subroutine bgt_track_one_turn

end module bgt_mod
