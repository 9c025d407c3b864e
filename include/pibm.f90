! pibm.f90 -- ISO_C_BINDING interface of libpibm (the C ABI of include/pibm.h)
! for a Fortran host such as the reference's driver
! (SRC/FLO/dtibm_main_scal_flo.F90).  Every derived type mirrors the C struct
! of the same name member for member (bind(C) gives them the C layout); every
! interface mirrors one entry point.  Arrays keep the reference's layout:
! complex(8) u(nx+1,my2,mz,3), nl(...), p(nx,my2,mz); real(8) xc(nbody,3).
! Pass arrays with c_loc(...) where an argument is type(c_ptr), value.
module pibm_c
  use iso_c_binding
  implicit none

  integer(c_int), parameter :: PIBM_OK = 0, PIBM_ERR_ARG = -1, PIBM_ERR_BLOWUP = -2, &
       PIBM_ERR_PIVOT = -3, PIBM_ERR_NAN = -4, PIBM_ERR_DEM_MOVE = -5, &
       PIBM_ERR_NEIGH_OVERFLOW = -6, PIBM_ERR_TIMEOUT = -7, PIBM_ERR_CUDA = -8, &
       PIBM_ERR_NOMEM = -9, PIBM_ERR_SPREAD_OVERFLOW = -10
  integer(c_int32_t), parameter :: PIBM_SCHEME_CENTER = 0, PIBM_SCHEME_UPWIND = 1
  integer(c_int32_t), parameter :: PIBM_LIMITER_NONE = 0, PIBM_LIMITER_MINMOD = 1
  integer(c_int), parameter :: PIBM_NPHASE = 7, PIBM_NKERNEL = 12

  type, bind(C) :: pibm_params
     integer(c_int32_t) :: my, mz
     real(c_double) :: lybyd, dbydx, dia_phys, vis, re, cfl, cfl_max, vfl, dr, f1, f2
     real(c_double) :: flo_ang(3), mpg(3)
     real(c_double) :: rhof, rhos, coeff_rest
     integer(c_int32_t) :: ramp_frac_steps, discr_scheme, limiter, adaptive, set_mpg
     integer(c_int32_t) :: initialize_zero, dorpr, revernorm, include_frmeanfluid, imove
     integer(c_int32_t) :: collision_softsphere, iscalon
     real(c_double) :: pr_or_sc_nu, phisurf, phistream
     integer(c_int32_t) :: rk3
     integer(c_int32_t) :: dobnd, aliasflag, nlcons_false      ! must be 0: DOBND=F, ALIASFLAG=0, NLCONS=T
     integer(c_int32_t) :: reserved(4)
  end type pibm_params

  type, bind(C) :: pibm_particles
     integer(c_int32_t) :: nbody
     type(c_ptr) :: xc              ! real(8) xc(nbody,3), grid units
     type(c_ptr) :: velbdy          ! real(8) velbdy(nbody,3) or c_null_ptr
  end type pibm_particles

  type, bind(C) :: pibm_state_view
     type(c_ptr) :: u, nl, p        ! complex(8) u(nx+1,my2,mz,3), nl(nx+1,my2,mz,3), p(nx,my2,mz)
     real(c_double) :: umean(3), mpg(3), ufmean(3)
     real(c_double) :: t, dt, cf
  end type pibm_state_view

  type, bind(C) :: pibm_step_report
     real(c_double) :: dt, t, cf
     real(c_double) :: umax
     real(c_double) :: divmax
     real(c_double) :: ufmean(3), usmean(3), umean(3)
     real(c_double) :: mpg(3), frmean(3)
     real(c_double) :: pres_total(3), visc_total(3)
     real(c_double) :: norm_drag, ferror
     real(c_double) :: pres_drag, visc_drag, total_drag
     real(c_double) :: mixmeanslipmod
     integer(c_int64_t) :: nrpr_active_total
     real(c_double) :: heat_ratio
     real(c_double) :: nusselt
  end type pibm_step_report

  type, bind(C) :: pibm_info
     integer(c_int32_t) :: nx, my, mz, my2, nbody, nbnd
     real(c_double) :: dx, dt, radbdy, maxvolfrac
     integer(c_int64_t) :: count_solid, count_fluid
     integer(c_int32_t) :: npts_active
     integer(c_int32_t) :: kernels_per_step
  end type pibm_info

  type, bind(C) :: pibm_adjoint_report
     real(c_double) :: J
     real(c_double) :: forward_ms
     real(c_double) :: reverse_ms
     integer(c_int32_t) :: nsteps, checkpoint_every
     integer(c_int32_t) :: adjoint_kernels_per_step
     integer(c_int32_t) :: reserved
  end type pibm_adjoint_report

  interface
     ! ---- one run ----
     integer(c_int) function pibm_create(prm, parts, h) bind(C, name="pibm_create")
       import :: c_int, c_ptr, pibm_params, pibm_particles
       type(pibm_params), intent(in) :: prm
       type(pibm_particles), intent(in) :: parts
       type(c_ptr), intent(out) :: h
     end function
     integer(c_int) function pibm_info_get(h, info) bind(C, name="pibm_info_get")
       import :: c_int, c_ptr, pibm_info
       type(c_ptr), value :: h
       type(pibm_info), intent(out) :: info
     end function
     integer(c_int) function pibm_set_state(h, s) bind(C, name="pibm_set_state")
       import :: c_int, c_ptr, pibm_state_view
       type(c_ptr), value :: h
       type(pibm_state_view), intent(in) :: s
     end function
     integer(c_int) function pibm_step(h, rks, rep) bind(C, name="pibm_step")
       import :: c_int, c_ptr, pibm_step_report
       type(c_ptr), value :: h
       integer(c_int), value :: rks
       type(pibm_step_report), intent(out) :: rep
     end function
     integer(c_int) function pibm_run(h, nsteps, last) bind(C, name="pibm_run")
       import :: c_int, c_ptr, pibm_step_report
       type(c_ptr), value :: h
       integer(c_int), value :: nsteps
       type(pibm_step_report), intent(out) :: last
     end function
     integer(c_int) function pibm_run_timed(h, nsteps, last, total_ms) bind(C, name="pibm_run_timed")
       import :: c_int, c_ptr, c_double, pibm_step_report
       type(c_ptr), value :: h
       integer(c_int), value :: nsteps
       type(pibm_step_report), intent(out) :: last
       real(c_double), intent(out) :: total_ms
     end function
     integer(c_int) function pibm_run_profiled(h, nsteps, last, total_ms, phase_ms, nphase) &
          bind(C, name="pibm_run_profiled")
       import :: c_int, c_ptr, c_double, pibm_step_report
       type(c_ptr), value :: h
       integer(c_int), value :: nsteps
       type(pibm_step_report), intent(out) :: last
       real(c_double), intent(out) :: total_ms
       real(c_double), intent(out) :: phase_ms(*)
       integer(c_int), value :: nphase
     end function
     integer(c_int) function pibm_kernel_times(h, nsteps, total_ms, kernel_ms, nkernel) &
          bind(C, name="pibm_kernel_times")
       import :: c_int, c_ptr, c_double
       type(c_ptr), value :: h
       integer(c_int), value :: nsteps
       real(c_double), intent(out) :: total_ms
       real(c_double), intent(out) :: kernel_ms(*)
       integer(c_int), value :: nkernel
     end function
     type(c_ptr) function pibm_kernel_name(k) bind(C, name="pibm_kernel_name")
       import :: c_ptr, c_int
       integer(c_int), value :: k
     end function
     integer(c_int) function pibm_get_state(h, s) bind(C, name="pibm_get_state")
       import :: c_int, c_ptr, pibm_state_view
       type(c_ptr), value :: h
       type(pibm_state_view), intent(inout) :: s
     end function
     integer(c_int) function pibm_get_particles(h, pres, visc, force, xc, vel) bind(C, name="pibm_get_particles")
       import :: c_int, c_ptr
       type(c_ptr), value :: h, pres, visc, force, xc, vel     ! real(8) (nbody,3) each, or c_null_ptr
     end function
     integer(c_int) function pibm_get_scalar(h, phif, flux_body, ratios) bind(C, name="pibm_get_scalar")
       import :: c_int, c_ptr
       type(c_ptr), value :: h, phif, flux_body, ratios         ! complex(8) phif(nx+1,my2,mz), real(8) flux_body(nbody), ratios(3)
     end function
     integer(c_int) function pibm_set_desired_means(h, usmean_des, ufmean_des) bind(C, name="pibm_set_desired_means")
       import :: c_int, c_ptr, c_double
       type(c_ptr), value :: h
       real(c_double), intent(in) :: usmean_des(3), ufmean_des(3)
     end function
     integer(c_int) function pibm_get_scalar_nl(h, nlphif) bind(C, name="pibm_get_scalar_nl")
       import :: c_int, c_ptr
       type(c_ptr), value :: h, nlphif                          ! complex(8) nlphif(nx+1,my2,mz)
     end function
     integer(c_int) function pibm_set_scalar(h, phif, nlphif, ratios) bind(C, name="pibm_set_scalar")
       import :: c_int, c_ptr
       type(c_ptr), value :: h, phif, nlphif, ratios            ! ratios(2): heat_ratio, heat_ratio_old
     end function
     integer(c_int) function pibm_get_contacts(h, maxn, neigh, pn, pv) bind(C, name="pibm_get_contacts")
       import :: c_int, c_ptr, c_int32_t
       type(c_ptr), value :: h
       integer(c_int32_t), value :: maxn
       integer(c_int32_t), intent(out) :: neigh(*), pn(*), pv(*)   ! (nbody, maxn) like NEIGHBOURS / PN / PV
     end function
     integer(c_int) function pibm_get_surface_points(h, bnd) bind(C, name="pibm_get_surface_points")
       import :: c_int, c_ptr, c_double
       type(c_ptr), value :: h
       real(c_double), intent(out) :: bnd(*)                    ! (3, nbnd): direction of point l in bnd(1:3, l)
     end function
     integer(c_int) function pibm_get_frame(h, frame_vel, frame_pos) bind(C, name="pibm_get_frame")
       import :: c_int, c_ptr, c_double
       type(c_ptr), value :: h
       real(c_double), intent(out) :: frame_vel(3), frame_pos(3)
     end function
     integer(c_int) function pibm_set_frame(h, frame_vel, frame_pos) bind(C, name="pibm_set_frame")
       import :: c_int, c_ptr, c_double
       type(c_ptr), value :: h
       real(c_double), intent(in) :: frame_vel(3), frame_pos(3)
     end function
     integer(c_int) function pibm_get_if_rev(h, if_rev) bind(C, name="pibm_get_if_rev")
       import :: c_int, c_ptr, c_int8_t
       type(c_ptr), value :: h
       integer(c_int8_t), intent(out) :: if_rev(*)              ! (nbnd, nbody), 0/1
     end function
     integer(c_int) function pibm_get_fluid_mask(h, mask) bind(C, name="pibm_get_fluid_mask")
       import :: c_int, c_ptr, c_int8_t
       type(c_ptr), value :: h
       integer(c_int8_t), intent(out) :: mask(*)                ! fluid_atijk(nx,my,mz), 0/1
     end function
     subroutine pibm_destroy(h) bind(C, name="pibm_destroy")
       import :: c_ptr
       type(c_ptr), value :: h
     end subroutine
     type(c_ptr) function pibm_last_error() bind(C, name="pibm_last_error")
       import :: c_ptr
     end function

     ! ---- plane transforms (ff2rc / ff2cr over nplanes planes, host arrays) ----
     integer(c_int) function pibm_ff2rc(my, mz, nplanes, a, b) bind(C, name="pibm_ff2rc")
       import :: c_int, c_double
       integer(c_int), value :: my, mz, nplanes
       real(c_double), intent(in) :: a(*)
       real(c_double), intent(out) :: b(*)
     end function
     integer(c_int) function pibm_ff2cr(my, mz, nplanes, a, b) bind(C, name="pibm_ff2cr")
       import :: c_int, c_double
       integer(c_int), value :: my, mz, nplanes
       real(c_double), intent(in) :: a(*)
       real(c_double), intent(out) :: b(*)
     end function
     integer(c_int) function pibm_ff2cr_noalloc(my, mz, nplanes, d_a, d_b, stream) bind(C, name="pibm_ff2cr_noalloc")
       import :: c_int, c_ptr
       integer(c_int), value :: my, mz, nplanes
       type(c_ptr), value :: d_a, d_b, stream                   ! device pointers, cudaStream_t
     end function

     ! ---- discrete adjoint ----
     integer(c_int) function pibm_adjoint_run(h, nsteps, ckpt, e, g_xc, g_mpg, rep) bind(C, name="pibm_adjoint_run")
       import :: c_int, c_ptr, c_double
       type(c_ptr), value :: h
       integer(c_int), value :: nsteps, ckpt
       real(c_double), intent(in) :: e(3)
       real(c_double), intent(out) :: g_xc(*), g_mpg(3)
       type(c_ptr), value :: rep                                ! c_loc(pibm_adjoint_report) or c_null_ptr
     end function
     integer(c_int) function pibm_adjoint_begin(h, nsteps, e) bind(C, name="pibm_adjoint_begin")
       import :: c_int, c_ptr, c_double
       type(c_ptr), value :: h
       integer(c_int), value :: nsteps
       real(c_double), intent(in) :: e(3)
     end function
     integer(c_int) function pibm_adjoint_step(h) bind(C, name="pibm_adjoint_step")
       import :: c_int, c_ptr
       type(c_ptr), value :: h
     end function
     integer(c_int) function pibm_adjoint_end(h, g_xc, g_mpg) bind(C, name="pibm_adjoint_end")
       import :: c_int, c_ptr, c_double
       type(c_ptr), value :: h
       real(c_double), intent(out) :: g_xc(*), g_mpg(3)
     end function

     ! ---- tile shapes and measurement ----
     integer(c_int) function pibm_get_tuning(h, lines_per_cta, lines_ms) bind(C, name="pibm_get_tuning")
       import :: c_int, c_ptr, c_int32_t, c_double
       type(c_ptr), value :: h
       integer(c_int32_t), intent(out) :: lines_per_cta
       real(c_double), intent(out) :: lines_ms(2)
     end function
     integer(c_int) function pibm_set_tuning(h, lines_per_cta) bind(C, name="pibm_set_tuning")
       import :: c_int, c_ptr, c_int32_t
       type(c_ptr), value :: h
       integer(c_int32_t), value :: lines_per_cta
     end function
     integer(c_int) function pibm_fp64_peak(tflops, ms) bind(C, name="pibm_fp64_peak")
       import :: c_int, c_double
       real(c_double), intent(out) :: tflops, ms
     end function
     integer(c_int) function pibm_qdiv_check(a, n, b, nb, mismatches) bind(C, name="pibm_qdiv_check")
       import :: c_int, c_double, c_long_long
       real(c_double), intent(in) :: a(*)
       integer(c_long_long), value :: n
       real(c_double), intent(in) :: b(*)
       integer(c_int), value :: nb
       integer(c_long_long), intent(out) :: mismatches
     end function

     ! ---- batched independent realizations ----
     integer(c_int) function pibm_batch_create(n, prm, parts, b) bind(C, name="pibm_batch_create")
       import :: c_int, c_ptr, pibm_params, pibm_particles
       integer(c_int), value :: n
       type(pibm_params), intent(in) :: prm(*)
       type(pibm_particles), intent(in) :: parts(*)
       type(c_ptr), intent(out) :: b
     end function
     integer(c_int) function pibm_batch_run(b, nsteps) bind(C, name="pibm_batch_run")
       import :: c_int, c_ptr
       type(c_ptr), value :: b
       integer(c_int), value :: nsteps
     end function
     integer(c_int) function pibm_batch_time(b, nsteps, sequential, ms) bind(C, name="pibm_batch_time")
       import :: c_int, c_ptr, c_double
       type(c_ptr), value :: b
       integer(c_int), value :: nsteps, sequential
       real(c_double), intent(out) :: ms
     end function
     type(c_ptr) function pibm_batch_member(b, i) bind(C, name="pibm_batch_member")
       import :: c_ptr, c_int
       type(c_ptr), value :: b
       integer(c_int), value :: i
     end function
     subroutine pibm_batch_destroy(b) bind(C, name="pibm_batch_destroy")
       import :: c_ptr
       type(c_ptr), value :: b
     end subroutine
  end interface
end module pibm_c
