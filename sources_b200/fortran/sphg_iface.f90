!-----------------------------------------------------------------------
! sphg_iface.f90 -- ISO_C_BINDING interface of libsphg (include/sphg.h)
! for the Fortran host of cwang2015/sources.  It replaces the calls to
! time_integration / time_integration_for_water / time_integration_for_soil
! (sph.f90:51-57) with the GPU step; the particles objects keep owning
! their arrays.  No Fortran compiler exists in the build image, so this
! module is compiled only where one does (gfortran/ifort, -std=f2008).
!-----------------------------------------------------------------------
module sphg_iface
  use, intrinsic :: iso_c_binding
  implicit none

  integer(c_int), parameter :: SPHG_WATER = 1, SPHG_SOIL = 2
  integer(c_int), parameter :: SPHG_FP64 = 0, SPHG_FP32 = 1

  type, bind(C) :: sphg_material
     real(c_double) :: rho0, b, gamma, c, viscosity
     real(c_double) :: k, porosity, permeability, G, E, niu, cohesion, phi
  end type

  type, bind(C) :: sphg_params
     integer(c_int32_t) :: abi_version, dim, skf, single_phase, first_material
     integer(c_int32_t) :: summation_density, average_velocity, visc_artificial
     integer(c_int32_t) :: artificial_density, soil_artificial_stress, volume_fraction
     integer(c_int32_t) :: water_artificial_volume, volume_fraction_renorm
     integer(c_int32_t) :: stress_integration, yield_criterion, plasticity
     integer(c_int32_t) :: integrate_scheme, precision, reorder_interval, renorm_interval
     real(c_double) :: gravity, numeric_gravity, alpha, beta, etq, dd, p1, p2
     real(c_double) :: delta, epsilon, dt, x_min, x_max, y_min, y_max
     integer(c_int64_t) :: max_interaction
     type(sphg_material) :: water, soil
     real(c_double) :: forchheimer_b
  end type

  type, bind(C) :: sphg_phase_host
     integer(c_int32_t) :: ntotal, nvirt, material, nfail
     real(c_double) :: dspp
     type(c_ptr) :: x = c_null_ptr, vx = c_null_ptr, dvx = c_null_ptr, av = c_null_ptr, v_min = c_null_ptr
     type(c_ptr) :: rho = c_null_ptr, rho_min = c_null_ptr, drho = c_null_ptr, p = c_null_ptr
     type(c_ptr) :: c = c_null_ptr, mass = c_null_ptr, hsml = c_null_ptr
     type(c_ptr) :: vof = c_null_ptr, vof_min = c_null_ptr, dvof = c_null_ptr, vof2 = c_null_ptr
     type(c_ptr) :: sxx = c_null_ptr, sxy = c_null_ptr, syy = c_null_ptr
     type(c_ptr) :: dsxx = c_null_ptr, dsxy = c_null_ptr, dsyy = c_null_ptr, dp = c_null_ptr
     type(c_ptr) :: sxx_min = c_null_ptr, sxy_min = c_null_ptr, syy_min = c_null_ptr, p_min = c_null_ptr
     type(c_ptr) :: epsilon_p = c_null_ptr, vcc = c_null_ptr
     type(c_ptr) :: txx = c_null_ptr, tyy = c_null_ptr, txy = c_null_ptr
     type(c_ptr) :: itype = c_null_ptr, fail = c_null_ptr
  end type

  ! scene generators (the input_*.f90 routines of the reference)
  integer(c_int), parameter :: SPHG_SCENE_DAM_BREAK = 1, SPHG_SCENE_GRANULAR_COLUMN = 2, SPHG_SCENE_TWO_PHASE = 3
  type, bind(C) :: sphg_scene_spec
     integer(c_int32_t) :: kind, skf, precision, pad
     real(c_double) :: dx, box_w, box_h, col_w, col_h, water_h, phi_deg
     real(c_double) :: porosity, permeability, forchheimer_b
  end type

  type, bind(C) :: sphg_stats_t
     integer(c_int64_t) :: niac(3)
     integer(c_int32_t) :: maxiac(2), miniac(2), noiac(2)
     integer(c_int32_t) :: nfail, n_out_of_domain, itimestep, pad
     real(c_double) :: time, last_step_ms
  end type

  interface
     subroutine sphg_default_params(p) bind(C, name="sphg_default_params")
       import :: sphg_params
       type(sphg_params), intent(out) :: p
     end subroutine
     integer(c_int) function sphg_create(p, n_phase, ctx) bind(C, name="sphg_create")
       import :: sphg_params, c_int, c_ptr
       type(sphg_params), intent(in) :: p
       integer(c_int), value :: n_phase
       type(c_ptr), intent(out) :: ctx
     end function
     integer(c_int) function sphg_upload_phase(ctx, phase, v) bind(C, name="sphg_upload_phase")
       import :: sphg_phase_host, c_int, c_ptr
       type(c_ptr), value :: ctx
       integer(c_int), value :: phase
       type(sphg_phase_host), intent(in) :: v
     end function
     integer(c_int) function sphg_single_step(ctx, itimestep) bind(C, name="sphg_single_step")
       import :: c_int, c_ptr
       type(c_ptr), value :: ctx
       integer(c_int), value :: itimestep
     end function
     integer(c_int) function sphg_time_integration(ctx, maxtimestep, itimestep, time) &
          bind(C, name="sphg_time_integration")
       import :: c_int, c_ptr, c_double
       type(c_ptr), value :: ctx
       integer(c_int), value :: maxtimestep
       integer(c_int), intent(inout) :: itimestep
       real(c_double), intent(inout) :: time
     end function
     integer(c_int) function sphg_download_phase(ctx, phase, v) bind(C, name="sphg_download_phase")
       import :: sphg_phase_host, c_int, c_ptr
       type(c_ptr), value :: ctx
       integer(c_int), value :: phase
       type(sphg_phase_host), intent(inout) :: v
     end function
     integer(c_int) function sphg_export_pairs(ctx, which, pair_i, pair_j, cap, n) &
          bind(C, name="sphg_export_pairs")
       import :: c_int, c_ptr, c_int32_t, c_int64_t
       type(c_ptr), value :: ctx
       integer(c_int), value :: which
       integer(c_int32_t), intent(out) :: pair_i(*), pair_j(*)
       integer(c_int64_t), value :: cap
       integer(c_int64_t), intent(out) :: n
     end function
     ! interaction statistics and nfail of the last step (interaction_statistics)
     integer(c_int) function sphg_stats(ctx, out) bind(C, name="sphg_stats")
       import :: sphg_stats_t, c_int, c_ptr
       type(c_ptr), value :: ctx
       type(sphg_stats_t), intent(out) :: out
     end function
     ! Tecplot output of every phase (output, declarations_sph.f90:1703); the
     ! paths end with c_null_char, path_second and the zone arrays may be c_null_ptr
     integer(c_int) function sphg_write_tecplot(ctx, path_first, path_second, append, zone_first, zone_second) &
          bind(C, name="sphg_write_tecplot")
       import :: c_int, c_ptr, c_char
       type(c_ptr), value :: ctx
       character(kind=c_char), intent(in) :: path_first(*)
       type(c_ptr), value :: path_second
       integer(c_int), value :: append
       type(c_ptr), value :: zone_first, zone_second
     end function
     ! run the context on a caller's CUDA stream (c_null_ptr: its own stream)
     integer(c_int) function sphg_set_stream(ctx, stream) bind(C, name="sphg_set_stream")
       import :: c_int, c_ptr
       type(c_ptr), value :: ctx, stream
     end function
     integer(c_int) function sphg_kernel_profile(ctx, enable) bind(C, name="sphg_kernel_profile")
       import :: c_int, c_ptr
       type(c_ptr), value :: ctx
       integer(c_int), value :: enable
     end function
     ! positions / velocities of one phase to or from DEVICE arrays (original order)
     integer(c_int) function sphg_export_xv_device(ctx, phase, x_dev, v_dev) bind(C, name="sphg_export_xv_device")
       import :: c_int, c_ptr
       type(c_ptr), value :: ctx
       integer(c_int), value :: phase
       type(c_ptr), value :: x_dev, v_dev
     end function
     integer(c_int) function sphg_import_xv_device(ctx, phase, x_dev, v_dev) bind(C, name="sphg_import_xv_device")
       import :: c_int, c_ptr
       type(c_ptr), value :: ctx
       integer(c_int), value :: phase
       type(c_ptr), value :: x_dev, v_dev
     end function
     ! several contexts stepped together, one CUDA graph per step (not to be
     ! stepped once a context is destroyed); itimesteps and times hold one entry per context
     integer(c_int) function sphg_group_create(ctxs, n, group) bind(C, name="sphg_group_create")
       import :: c_int, c_ptr
       type(c_ptr), intent(in) :: ctxs(*)
       integer(c_int), value :: n
       type(c_ptr), intent(out) :: group
     end function
     integer(c_int) function sphg_group_time_integration(group, maxtimestep, itimesteps, times) &
          bind(C, name="sphg_group_time_integration")
       import :: c_int, c_ptr, c_double
       type(c_ptr), value :: group
       integer(c_int), value :: maxtimestep
       integer(c_int), intent(inout) :: itimesteps(*)
       real(c_double), intent(inout) :: times(*)
     end function
     subroutine sphg_group_destroy(group) bind(C, name="sphg_group_destroy")
       import :: c_ptr
       type(c_ptr), value :: group
     end subroutine
     ! scene generators: sizes first, then the host allocates its particles
     ! arrays (x is (2,n)) and points the phase views at them
     subroutine sphg_scene_default(kind, s) bind(C, name="sphg_scene_default")
       import :: c_int, sphg_scene_spec
       integer(c_int), value :: kind
       type(sphg_scene_spec), intent(out) :: s
     end subroutine
     integer(c_int) function sphg_scene_size(s, n_phase, ntotal, nvirt) bind(C, name="sphg_scene_size")
       import :: c_int, c_int32_t, sphg_scene_spec
       type(sphg_scene_spec), intent(in) :: s
       integer(c_int32_t), intent(out) :: n_phase, ntotal(2), nvirt(2)
     end function
     integer(c_int) function sphg_make_scene(s, p, first, second) bind(C, name="sphg_make_scene")
       import :: c_int, sphg_scene_spec, sphg_params, sphg_phase_host
       type(sphg_scene_spec), intent(in) :: s
       type(sphg_params), intent(out) :: p
       type(sphg_phase_host), intent(inout) :: first, second
     end function
     subroutine sphg_destroy(ctx) bind(C, name="sphg_destroy")
       import :: c_ptr
       type(c_ptr), value :: ctx
     end subroutine
     type(c_ptr) function sphg_strerror(code) bind(C, name="sphg_strerror")
       import :: c_ptr, c_int
       integer(c_int), value :: code
     end function
  end interface
end module sphg_iface
