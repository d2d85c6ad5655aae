! gfsph_c.f90 — ISO_C_BINDING interface of libgfsph (include/gfsph.h) for the
! Geoflow-SPH Fortran host.  Source only: the image that builds the library has
! no Fortran compiler.  A maintainer adds this module to the reference's build
! and, in Driver_Flow (SPH_FEM_Driver_2019.f90:1580-1697), replaces the calls
! to adaptive_dt_sph and time_integration_sph with one gfsph_step per output
! interval, uploading x, vx, rho, mass, hsml once after Init_sph and
! downloading them before each Out_PLOT / Out_Save.
module gfsph_c
  use, intrinsic :: iso_c_binding
  implicit none

  integer(c_int), parameter :: GFSPH_NCONST = 110, GFSPH_NTOPO = 16
  integer(c_int), parameter :: GFSPH_OK = 0, GFSPH_T_END_REACHED = 1
  integer(c_int), parameter :: GFSPH_ERR_ARG = -1, GFSPH_ERR_CUDA = -2, GFSPH_ERR_CAPACITY = -3, &
                               GFSPH_ERR_UNSUPPORTED = -4, GFSPH_ERR_STATE = -5, GFSPH_ERR_NO_DEVICE = -6, &
                               GFSPH_ERR_NONFINITE = -7, GFSPH_ERR_DOMAIN = -8, GFSPH_ERR_HOST = -9
  integer(c_int), parameter :: GFSPH_RASTER_DEPTH_IDW = 0, GFSPH_RASTER_MAX_DEPTH = 1, &
                               GFSPH_RASTER_MAX_VEL = 2, GFSPH_RASTER_SUM_DEPTH = 3, &
                               GFSPH_RASTER_SUM_VEL = 4, GFSPH_RASTER_COUNT = 5, &
                               GFSPH_RASTER_Z = 6, GFSPH_RASTER_ERODED = 7, GFSPH_RASTER_AVAILABLE = 8

  type, bind(c) :: gfsph_params
     real(c_float)  :: cst(GFSPH_NCONST)        ! const(1..110)
     integer(c_int) :: pa_sph, nnps, sle, skf
     integer(c_int) :: summation_density, average_velocity, nor_density
     integer(c_int) :: ic_adapt
     real(c_float)  :: h_inf, dt
     integer(c_int) :: dem_deriv, max_neighbours
     integer(c_int) :: icpwp                   ! 0 or 3 (Get_Pwp_SW, nUaux = 1)
     real(c_float)  :: pwp0rel                 ! initial Uaux = pwp0rel * rho * const(14)
     integer(c_int) :: ws_interact              ! ic_ws_Interact (0 or 1)
     integer(c_int) :: sw_alg                   ! ic_SWalg (0 or 1) with ws_interact = 1
     integer(c_int) :: reserved(4)
  end type gfsph_params

  type, bind(c) :: gfsph_dem
     integer(c_int) :: nx, ny                  ! npoigx, npoigy
     real(c_float)  :: xmin, ymin, dx, dy      ! xming, yming, deltxg, deltyg
     type(c_ptr)    :: topol                   ! c_loc(topol) of topol(ntopo, npoig)
     integer(c_int) :: ntopo
     type(c_ptr)    :: z
  end type gfsph_dem

  type, bind(c) :: gfsph_gfl_params
     real(c_float)  :: constF(15)              ! constF(1:15) of the GFL .dat as Input_GFL keeps them
     integer(c_int) :: ntype                   ! 2 under a still-water level, 3 over a dry bed
     integer(c_int) :: ngaus                   ! Gauss points per triangle (1 or 3)
     integer(c_int) :: niter                   ! consistent-mass sweeps of solve
     real(c_float)  :: swl                     ! still-water level
     real(c_float)  :: comp                    ! dry depth of check
  end type gfsph_gfl_params

  interface
     integer(c_int) function gfsph_create(params, dem, handle) bind(c, name="gfsph_create")
       import :: c_int, c_ptr, gfsph_params, gfsph_dem
       type(gfsph_params), intent(in) :: params
       type(gfsph_dem), intent(in) :: dem
       type(c_ptr), intent(out) :: handle
     end function
     integer(c_int) function gfsph_destroy(handle) bind(c, name="gfsph_destroy")
       import :: c_int, c_ptr
       type(c_ptr), value :: handle
     end function
     integer(c_int) function gfsph_upload(handle, n, x, vx, rho, mass, hsml, itype, out_flag) &
          bind(c, name="gfsph_upload")
       import :: c_int, c_ptr, c_float
       type(c_ptr), value :: handle
       integer(c_int), value :: n
       real(c_float), intent(in) :: x(2, n), vx(2, n), rho(n), mass(n), hsml(n)
       integer(c_int), intent(in) :: itype(n), out_flag(n)
     end function
     integer(c_int) function gfsph_download(handle, x, vx, rho, mass, hsml, out_flag) &
          bind(c, name="gfsph_download")
       import :: c_int, c_ptr, c_float
       type(c_ptr), value :: handle
       real(c_float), intent(out) :: x(2, *), vx(2, *), rho(*), mass(*), hsml(*)
       integer(c_int), intent(out) :: out_flag(*)
     end function
     integer(c_int) function gfsph_step(handle, nsteps, t_end, t_out, steps_done) bind(c, name="gfsph_step")
       import :: c_int, c_ptr, c_double
       type(c_ptr), value :: handle
       integer(c_int), value :: nsteps
       real(c_double), value :: t_end
       real(c_double), intent(out) :: t_out
       integer(c_int), intent(out) :: steps_done
     end function
     integer(c_int) function gfsph_get_time(handle, t, dt) bind(c, name="gfsph_get_time")
       import :: c_int, c_ptr, c_double, c_float
       type(c_ptr), value :: handle
       real(c_double), intent(out) :: t
       real(c_float), intent(out) :: dt
     end function
     ! the handle's kernels on a CUDA stream (c_null_ptr: the handle's own)
     integer(c_int) function gfsph_set_stream(handle, stream) bind(c, name="gfsph_set_stream")
       import :: c_int, c_ptr
       type(c_ptr), value :: handle, stream
     end function
     integer(c_int) function gfsph_set_time(handle, t, dt) bind(c, name="gfsph_set_time")
       import :: c_int, c_ptr, c_double, c_float
       type(c_ptr), value :: handle
       real(c_double), value :: t
       real(c_float), value :: dt
     end function
     integer(c_int) function gfsph_density(handle, rho) bind(c, name="gfsph_density")
       import :: c_int, c_ptr, c_float
       type(c_ptr), value :: handle
       real(c_float), intent(out) :: rho(*)
     end function
     integer(c_int) function gfsph_neighbours(handle, cap, offsets, idx) bind(c, name="gfsph_neighbours")
       import :: c_int, c_ptr
       type(c_ptr), value :: handle
       integer(c_int), value :: cap
       integer(c_int), intent(out) :: offsets(*), idx(*)
     end function
     integer(c_int) function gfsph_internal_forces(handle, indvxdt) bind(c, name="gfsph_internal_forces")
       import :: c_int, c_ptr, c_float
       type(c_ptr), value :: handle
       real(c_float), intent(out) :: indvxdt(2, *)
     end function
     integer(c_int) function gfsph_raster(handle, kind, out) bind(c, name="gfsph_raster")
       import :: c_int, c_ptr, c_float
       type(c_ptr), value :: handle
       integer(c_int), value :: kind
       real(c_float), intent(out) :: out(*)
     end function
     integer(c_int) function gfsph_raster_misfit(h, target, loss, gx, gh) bind(c, name="gfsph_raster_misfit")
       import :: c_int, c_ptr, c_float, c_double
       type(c_ptr), value :: h
       real(c_float), intent(in) :: target(*)
       real(c_double), intent(out) :: loss
       real(c_float), intent(out) :: gx(*), gh(*)
     end function
     integer(c_int) function gfsph_hazard_sample(handle) bind(c, name="gfsph_hazard_sample")
       import :: c_int, c_ptr
       type(c_ptr), value :: handle
     end function
     integer(c_int) function gfsph_hazard_reset(handle) bind(c, name="gfsph_hazard_reset")
       import :: c_int, c_ptr
       type(c_ptr), value :: handle
     end function
     integer(c_int) function gfsph_profile(handle, enable) bind(c, name="gfsph_profile")
       import :: c_int, c_ptr
       type(c_ptr), value :: handle
       integer(c_int), value :: enable
     end function
     integer(c_int) function gfsph_profile_read(handle, kernel, total_ms, launches) bind(c, name="gfsph_profile_read")
       import :: c_int, c_ptr, c_double, c_long_long
       type(c_ptr), value :: handle
       integer(c_int), value :: kernel
       real(c_double), intent(out) :: total_ms
       integer(c_long_long), intent(out) :: launches
     end function
     integer(c_int) function gfsph_num_kernels() bind(c, name="gfsph_num_kernels")
       import :: c_int
     end function
     type(c_ptr) function gfsph_kernel_name(kernel) bind(c, name="gfsph_kernel_name")
       import :: c_int, c_ptr
       integer(c_int), value :: kernel
     end function
     integer(c_long_long) function gfsph_launch_count(handle) bind(c, name="gfsph_launch_count")
       import :: c_long_long, c_ptr
       type(c_ptr), value :: handle
     end function
     integer(c_int) function gfsph_stats(handle, out, nout) bind(c, name="gfsph_stats")
       import :: c_int, c_ptr
       type(c_ptr), value :: handle
       integer(c_int), intent(out) :: out(*)
       integer(c_int), value :: nout
     end function
     integer(c_int) function gfsph_dem_topol(mode, nx, ny, dx, dy, topol) bind(c, name="gfsph_dem_topol")
       import :: c_int, c_float
       integer(c_int), value :: mode, nx, ny
       real(c_float), value :: dx, dy
       real(c_float), intent(inout) :: topol(GFSPH_NTOPO, *)
     end function
     integer(c_int) function gfsph_set_search(h, level_factor, cell_div) bind(c, name="gfsph_set_search")
       import :: c_int, c_ptr, c_float
       type(c_ptr), value :: h
       real(c_float), value :: level_factor, cell_div
     end function
     integer(c_int) function gfsph_get_search(h, level_factor, cell_div) bind(c, name="gfsph_get_search")
       import :: c_int, c_ptr, c_float
       type(c_ptr), value :: h
       real(c_float), intent(out) :: level_factor, cell_div
     end function
     integer(c_int) function gfsph_autotune(h, steps, level_factor, cell_div, best_ms) bind(c, name="gfsph_autotune")
       import :: c_int, c_ptr, c_float
       type(c_ptr), value :: h
       integer(c_int), value :: steps
       real(c_float), intent(out) :: level_factor, cell_div, best_ms
     end function
     integer(c_int) function gfsph_adjoint_forward(h, nsteps, every, adj) bind(c, name="gfsph_adjoint_forward")
       import :: c_int, c_ptr
       type(c_ptr), value :: h
       integer(c_int), value :: nsteps, every
       type(c_ptr), intent(out) :: adj
     end function
     integer(c_int) function gfsph_adjoint_backward(adj, gx, gv, gh, gx0, gv0, gm, gmu, gxi) &
         bind(c, name="gfsph_adjoint_backward")
       import :: c_int, c_ptr, c_float, c_double
       type(c_ptr), value :: adj
       real(c_float), intent(in) :: gx(*), gv(*), gh(*)
       real(c_float), intent(out) :: gx0(*), gv0(*), gm(*)
       real(c_double), intent(out) :: gmu, gxi
     end function
     integer(c_int) function gfsph_adjoint_param(a, which, val) bind(c, name="gfsph_adjoint_param")
       import :: c_int, c_ptr, c_double
       type(c_ptr), value :: a
       integer(c_int), value :: which
       real(c_double), intent(out) :: val
     end function
     integer(c_int) function gfsph_adjoint_destroy(adj) bind(c, name="gfsph_adjoint_destroy")
       import :: c_int, c_ptr
       type(c_ptr), value :: adj
     end function
     integer(c_int) function gfsph_gradhs(h, ix0, iy0, nwx, nwy, niter, tol, hs_w, gradhs_w) &
         bind(c, name="gfsph_gradhs")
       import :: c_int, c_ptr, c_float
       type(c_ptr), value :: h
       integer(c_int), value :: ix0, iy0, nwx, nwy, niter
       real(c_float), value :: tol
       real(c_float), intent(out) :: hs_w(*), gradhs_w(*)
     end function
     integer(c_int) function gfsph_set_pwp(h, pwp) bind(c, name="gfsph_set_pwp")
       import :: c_int, c_ptr, c_float
       type(c_ptr), value :: h
       real(c_float), intent(in) :: pwp(*)
     end function
     integer(c_int) function gfsph_get_pwp(h, pwp) bind(c, name="gfsph_get_pwp")
       import :: c_int, c_ptr, c_float
       type(c_ptr), value :: h
       real(c_float), intent(out) :: pwp(*)
     end function
     integer(c_int) function gfsph_ensemble_create(params, dem, nreal, ens) bind(c, name="gfsph_ensemble_create")
       import :: c_int, c_ptr, gfsph_params, gfsph_dem
       type(gfsph_params), intent(in) :: params(*)
       type(gfsph_dem), intent(in) :: dem
       integer(c_int), value :: nreal
       type(c_ptr), intent(out) :: ens
     end function
     integer(c_int) function gfsph_ensemble_destroy(ens) bind(c, name="gfsph_ensemble_destroy")
       import :: c_int, c_ptr
       type(c_ptr), value :: ens
     end function
     integer(c_int) function gfsph_ensemble_member(ens, r, member) bind(c, name="gfsph_ensemble_member")
       import :: c_int, c_ptr
       type(c_ptr), value :: ens
       integer(c_int), value :: r
       type(c_ptr), intent(out) :: member
     end function
     integer(c_int) function gfsph_ensemble_step(ens, nsteps, t_end, min_steps_done) bind(c, name="gfsph_ensemble_step")
       import :: c_int, c_ptr, c_double
       type(c_ptr), value :: ens
       integer(c_int), value :: nsteps
       real(c_double), value :: t_end
       integer(c_int), intent(out) :: min_steps_done
     end function
     integer(c_int) function gfsph_ensemble_sample(ens) bind(c, name="gfsph_ensemble_sample")
       import :: c_int, c_ptr
       type(c_ptr), value :: ens
     end function
     integer(c_int) function gfsph_ensemble_exceedance(ens, threshold, prob) bind(c, name="gfsph_ensemble_exceedance")
       import :: c_int, c_ptr, c_float
       type(c_ptr), value :: ens
       real(c_float), value :: threshold
       real(c_float), intent(out) :: prob(*)
     end function
     integer(c_int) function gfsph_cg_create(npoin, nelem, nnode, ndofn, intmat, gstif, cg) bind(c, name="gfsph_cg_create")
       import :: c_int, c_ptr, c_float
       integer(c_int), value :: npoin, nelem, nnode, ndofn
       integer(c_int), intent(in) :: intmat(nnode, nelem)
       real(c_float), intent(in) :: gstif(nnode*ndofn, nnode*ndofn, nelem)
       type(c_ptr), intent(out) :: cg
     end function
     integer(c_int) function gfsph_cg_solve(cg, iffix, fixed, rcg, ficg, tol, iterations) bind(c, name="gfsph_cg_solve")
       import :: c_int, c_ptr, c_float
       type(c_ptr), value :: cg
       integer(c_int), intent(inout) :: iffix(*)
       real(c_float), intent(in) :: fixed(*)
       real(c_float), intent(inout) :: rcg(*)
       real(c_float), intent(out) :: ficg(*)
       real(c_float), value :: tol
       integer(c_int), intent(out) :: iterations
     end function
     integer(c_int) function gfsph_cg_destroy(cg) bind(c, name="gfsph_cg_destroy")
       import :: c_int, c_ptr
       type(c_ptr), value :: cg
     end function
     integer(c_long_long) function gfsph_cg_launch_count(cg) bind(c, name="gfsph_cg_launch_count")
       import :: c_long_long, c_ptr
       type(c_ptr), value :: cg
     end function
     integer(c_int) function gfsph_cg_device_ms(cg, ms) bind(c, name="gfsph_cg_device_ms")
       import :: c_int, c_ptr, c_double
       type(c_ptr), value :: cg
       real(c_double), intent(out) :: ms
     end function
     ! drop-in for: call solvegc2(npoin, nelem, nnode, ndofn, ntotv, nevab, intmat, iffix, fixed, gstif, rcg, ficg, tolCG)
     integer(c_int) function gfsph_solvegc2(npoin, nelem, nnode, ndofn, intmat, iffix, fixed, gstif, rcg, ficg, &
          tol, iterations) bind(c, name="gfsph_solvegc2")
       import :: c_int, c_float
       integer(c_int), value :: npoin, nelem, nnode, ndofn
       integer(c_int), intent(in) :: intmat(nnode, nelem)
       integer(c_int), intent(inout) :: iffix(*)
       real(c_float), intent(in) :: fixed(*), gstif(nnode*ndofn, nnode*ndofn, nelem)
       real(c_float), intent(inout) :: rcg(*)
       real(c_float), intent(out) :: ficg(*)
       real(c_float), value :: tol
       integer(c_int), intent(out) :: iterations
     end function
     ! allocation-free depth raster: device pointers in and out (c_devptr from CUDA Fortran or c_loc)
     integer(c_int) function gfsph_raster_idw_noalloc(n, d_x, d_rho, d_flag, nx, ny, xmin, ymin, dx, dy, d_out, &
          stream) bind(c, name="gfsph_raster_idw_noalloc")
       import :: c_int, c_ptr, c_float
       integer(c_int), value :: n, nx, ny
       type(c_ptr), value :: d_x, d_rho, d_flag, d_out, stream
       real(c_float), value :: xmin, ymin, dx, dy
     end function
     ! the GFL step: replaces Init_GFL's set-up and calls of time_integration_gfl on one mesh
     integer(c_int) function gfsph_gfl_create(params, npoin, nelem, coord, intmat, z, gfl) &
          bind(c, name="gfsph_gfl_create")
       import :: c_int, c_ptr, c_float, gfsph_gfl_params
       type(gfsph_gfl_params), intent(in) :: params
       integer(c_int), value :: npoin, nelem
       real(c_float), intent(in) :: coord(2, npoin), z(npoin)
       integer(c_int), intent(in) :: intmat(3, nelem)
       type(c_ptr), intent(out) :: gfl
     end function
     integer(c_int) function gfsph_gfl_destroy(gfl) bind(c, name="gfsph_gfl_destroy")
       import :: c_int, c_ptr
       type(c_ptr), value :: gfl
     end function
     integer(c_int) function gfsph_gfl_set_state(gfl, unkno, time) bind(c, name="gfsph_gfl_set_state")
       import :: c_int, c_ptr, c_float, c_double
       type(c_ptr), value :: gfl
       real(c_float), intent(in) :: unkno(3, *)
       real(c_double), value :: time
     end function
     integer(c_int) function gfsph_gfl_get_state(gfl, unkno, time) bind(c, name="gfsph_gfl_get_state")
       import :: c_int, c_ptr, c_float, c_double
       type(c_ptr), value :: gfl
       real(c_float), intent(out) :: unkno(3, *)
       real(c_double), intent(out) :: time
     end function
     integer(c_int) function gfsph_gfl_set_wir(gfl, hs_w, gradhs_w) bind(c, name="gfsph_gfl_set_wir")
       import :: c_int, c_ptr, c_float
       type(c_ptr), value :: gfl
       real(c_float), intent(in) :: hs_w(*), gradhs_w(2, *)
     end function
     integer(c_int) function gfsph_gfl_step(gfl, nsteps, dt) bind(c, name="gfsph_gfl_step")
       import :: c_int, c_ptr, c_float
       type(c_ptr), value :: gfl
       integer(c_int), value :: nsteps
       real(c_float), value :: dt
     end function
     integer(c_int) function gfsph_gfl_topol(gfl, topol, topel) bind(c, name="gfsph_gfl_topol")
       import :: c_int, c_ptr, c_float
       type(c_ptr), value :: gfl
       real(c_float), intent(out) :: topol(9, *), topel(9, *)
     end function
     integer(c_long_long) function gfsph_gfl_launch_count(gfl) bind(c, name="gfsph_gfl_launch_count")
       import :: c_long_long, c_ptr
       type(c_ptr), value :: gfl
     end function
     integer(c_int) function gfsph_gfl_device_ms(gfl, ms) bind(c, name="gfsph_gfl_device_ms")
       import :: c_int, c_ptr, c_double
       type(c_ptr), value :: gfl
       real(c_double), intent(out) :: ms
     end function
     type(c_ptr) function gfsph_strerror(status) bind(c, name="gfsph_strerror")
       import :: c_int, c_ptr
       integer(c_int), value :: status
     end function
     integer(c_int) function gfsph_version() bind(c, name="gfsph_version")
       import :: c_int
     end function
     integer(c_int) function gfsph_binary_version(version) bind(c, name="gfsph_binary_version")
       import :: c_int
       integer(c_int), intent(out) :: version
     end function
  end interface
end module gfsph_c
