! moons_gpu_mod.f90 -- ISO_C_BINDING interfaces to include/moons_gpu.h.
!
! The module a Fortran host (the reference's solve_MOONS, init_mom,
! init_induction, Euler_time_*, clean_div_*) uses to call the B200 library.
! Every function returns an integer status (0 = OK); the caller decides
! whether to stop, as the reference's own error paths do.  Arrays are passed
! with c_loc of the contiguous grid_field array f(sx,sy,sz) for the duration
! of the call only.  Written against the C header; it is not compiled in
! this repository's build (no Fortran compiler in the image).
module moons_gpu_mod
  use, intrinsic :: iso_c_binding
  implicit none

  integer(c_int), parameter :: MOONS_OK = 0, MOONS_ERR_ARG = 1, MOONS_ERR_SHAPE = 2, MOONS_ERR_CUDA = 3
  integer(c_int), parameter :: MOONS_ERR_NAN = 4, MOONS_ERR_STATE = 5, MOONS_ERR_NOMEM = 6
  integer(c_int), parameter :: MOONS_ERR_LIMIT = 7
  integer(c_int), parameter :: MOONS_CC = 0, MOONS_FX = 1, MOONS_FY = 2, MOONS_FZ = 3
  integer(c_int), parameter :: MOONS_EX = 4, MOONS_EY = 5, MOONS_EZ = 6, MOONS_NODE = 7
  integer(c_int), parameter :: MOONS_BC_NONE = 0, MOONS_BC_DIRICHLET = 1, MOONS_BC_NEUMANN = 2
  integer(c_int), parameter :: MOONS_BC_PERIODIC = 3, MOONS_BC_ROBIN = 4
  integer(c_int), parameter :: MOONS_OP_LAP_UNIFORM = 1, MOONS_OP_LAP_PROPS = 2
  integer(c_int), parameter :: MOONS_OP_IND_DIFFUSION = 3, MOONS_OP_MOM_DIFFUSION = 4
  integer(c_int), parameter :: MOONS_OP_NRG_DIFFUSION = 5
  integer(c_int), parameter :: MOONS_PREC_IDENTITY = 0, MOONS_PREC_LAP = 1
  integer(c_int), parameter :: MOONS_PREC_MOM = 2, MOONS_PREC_IND = 3
  integer(c_int), parameter :: MOONS_PREC_MG = 4, MOONS_PREC_MG_MIXED = 5, MOONS_PREC_UNET = 6
  integer(c_int), parameter :: MOONS_PREC_FD = 7
  integer(c_int), parameter :: MOONS_PREC_UNET_MG = 8
  ! the MHD step: induction forms and field handles of moons_mhd_field
  integer(c_int), parameter :: MOONS_IND_OFF = 0, MOONS_IND_B = 1, MOONS_IND_POTENTIAL = 2
  integer(c_int), parameter :: MOONS_MHD_U = 0, MOONS_MHD_P = 1, MOONS_MHD_B = 2, MOONS_MHD_B0 = 3
  integer(c_int), parameter :: MOONS_MHD_PHI = 4, MOONS_MHD_J = 5, MOONS_MHD_SIGMA_INV = 6
  integer(c_int), parameter :: MOONS_MHD_JXB = 7, MOONS_MHD_DIVU = 8, MOONS_MHD_DIVB = 9
  integer(c_int), parameter :: MOONS_MHD_T = 10, MOONS_MHD_KT = 11, MOONS_MHD_GRAVITY = 12
  integer(c_int), parameter :: MOONS_MHD_SIGMA_INV_CC = 13, MOONS_MHD_U_CC = 14
  ! largest face temporary (points) that moons_lap_var_noalloc accepts
  integer(c_long_long), parameter :: MOONS_LAP_VAR_NOALLOC_MAX_POINTS = 131072_c_long_long

  type, bind(C) :: moons_bc_spec
    integer(c_int) :: type(6)
    integer(c_int) :: prescribed(6)
    real(c_double) :: value(6)
    real(c_double) :: c_w(6)
    integer(c_int) :: order(6)
    integer(c_int) :: all_neumann
  end type

  type, bind(C) :: moons_isp
    integer(c_int) :: iter_max
    real(c_double) :: tol_rel
    real(c_double) :: tol_abs
    integer(c_int) :: n_skip_check_res
  end type

  type, bind(C) :: moons_solve_info
    integer(c_int) :: iterations
    real(c_double) :: res0, res, rel
    integer(c_int) :: exit_reason
    real(c_double) :: ms
  end type

  ! parameters of the MHD step (solve_MOONS); the meaning of each field is
  ! given in the C header
  type, bind(C) :: moons_mhd_params
    real(c_double) :: dt
    integer(c_int) :: induction
    integer(c_int) :: finite_Rem
    integer(c_int) :: mpg_dir
    real(c_double) :: mpg_scale
    real(c_double) :: scale_advection_U
    real(c_double) :: scale_diffusion_U
    real(c_double) :: scale_JxB
    real(c_double) :: scale_advection_B
    real(c_double) :: scale_diffusion_B
    real(c_double) :: scale_current
    real(c_double) :: coeff_implicit_U
    real(c_double) :: coeff_implicit_B
    type(moons_isp) :: isp_U, isp_p, isp_B, isp_phi
    type(moons_bc_spec) :: bc_U(3), bc_p, bc_B(3), bc_phi
    integer(c_int) :: ind_offset(3)
    integer(c_int) :: prescribed_Ustar
    integer(c_int) :: prescribed_Bstar
    integer(c_int) :: prec_poisson
    integer(c_int) :: energy
    integer(c_int) :: solve_method_T
    real(c_double) :: coeff_implicit_T
    real(c_double) :: scale_advection_T
    real(c_double) :: scale_diffusion_T
    real(c_double) :: scale_heating_T
    real(c_double) :: scale_buoyancy
    type(moons_isp) :: isp_T
    type(moons_bc_spec) :: bc_T
    real(c_double) :: scale_KE_diffusion_T
    real(c_double) :: scale_viscous_dissipation_T
    real(c_double) :: scale_joule_heating_T
    integer(c_int) :: solve_method_U
    integer(c_int) :: solve_method_B
    integer(c_int) :: rk_stages
    real(c_double) :: scale_diffusion_linear_U
    real(c_double) :: scale_diffusion_linear_B
  end type

  type, bind(C) :: moons_step_info
    integer(c_int) :: steps
    integer(c_int) :: iters_U, iters_p, iters_B, iters_phi
    real(c_double) :: res_p, res_phi
    real(c_double) :: ms
    integer(c_int) :: iters_T
  end type

  interface
    function moons_last_error() bind(C, name="moons_last_error") result(p)
      import :: c_ptr
      type(c_ptr) :: p
    end function

    function moons_mesh_create(m, hn_x, sn_x, hn_y, sn_y, hn_z, sn_z, device) &
        bind(C, name="moons_mesh_create") result(st)
      import :: c_ptr, c_int, c_double
      type(c_ptr) :: m
      real(c_double), intent(in) :: hn_x(*), hn_y(*), hn_z(*)
      integer(c_int), value :: sn_x, sn_y, sn_z, device
      integer(c_int) :: st
    end function

    function moons_mesh_destroy(m) bind(C, name="moons_mesh_destroy") result(st)
      import :: c_ptr, c_int
      type(c_ptr), value :: m
      integer(c_int) :: st
    end function

    function moons_sf_create(m, data_loc, f) bind(C, name="moons_sf_create") result(st)
      import :: c_ptr, c_int
      type(c_ptr), value :: m
      integer(c_int), value :: data_loc
      type(c_ptr) :: f
      integer(c_int) :: st
    end function

    function moons_sf_destroy(f) bind(C, name="moons_sf_destroy") result(st)
      import :: c_ptr, c_int
      type(c_ptr), value :: f
      integer(c_int) :: st
    end function

    function moons_sf_upload(f, host, n) bind(C, name="moons_sf_upload") result(st)
      import :: c_ptr, c_int, c_double, c_long_long
      type(c_ptr), value :: f
      real(c_double), intent(in) :: host(*)
      integer(c_long_long), value :: n
      integer(c_int) :: st
    end function

    function moons_sf_download(f, host, n) bind(C, name="moons_sf_download") result(st)
      import :: c_ptr, c_int, c_double, c_long_long
      type(c_ptr), value :: f
      real(c_double), intent(out) :: host(*)
      integer(c_long_long), value :: n
      integer(c_int) :: st
    end function

    function moons_sf_set_bcs(f, spec) bind(C, name="moons_sf_set_bcs") result(st)
      import :: c_ptr, c_int, moons_bc_spec
      type(c_ptr), value :: f
      type(moons_bc_spec), intent(in) :: spec
      integer(c_int) :: st
    end function

    function moons_apply_bcs(f) bind(C, name="moons_apply_bcs") result(st)
      import :: c_ptr, c_int
      type(c_ptr), value :: f
      integer(c_int) :: st
    end function

    function moons_grad(gx, gy, gz, u) bind(C, name="moons_grad") result(st)
      import :: c_ptr, c_int
      type(c_ptr), value :: gx, gy, gz, u
      integer(c_int) :: st
    end function

    function moons_div(out, ux, uy, uz) bind(C, name="moons_div") result(st)
      import :: c_ptr, c_int
      type(c_ptr), value :: out, ux, uy, uz
      integer(c_int) :: st
    end function

    function moons_curl(ox, oy, oz, ux, uy, uz) bind(C, name="moons_curl") result(st)
      import :: c_ptr, c_int
      type(c_ptr), value :: ox, oy, oz, ux, uy, uz
      integer(c_int) :: st
    end function

    function moons_lap_var(out, u, kx, ky, kz) bind(C, name="moons_lap_var") result(st)
      import :: c_ptr, c_int
      type(c_ptr), value :: out, u, kx, ky, kz
      integer(c_int) :: st
    end function

    ! the same operator without device allocation (temporaries in the
    ! library's built-in device array; fields beyond the limit above are
    ! rejected with MOONS_ERR_LIMIT)
    function moons_lap_var_noalloc(out, u, kx, ky, kz) bind(C, name="moons_lap_var_noalloc") result(st)
      import :: c_ptr, c_int
      type(c_ptr), value :: out, u, kx, ky, kz
      integer(c_int) :: st
    end function

    function moons_pcg_create(m, op, prec, ncomp, x, x_bc, k, s) &
        bind(C, name="moons_pcg_create") result(st)
      import :: c_ptr, c_int
      type(c_ptr), value :: m
      integer(c_int), value :: op, prec, ncomp
      type(c_ptr), intent(in) :: x(*), x_bc(*), k(*)
      type(c_ptr) :: s
      integer(c_int) :: st
    end function

    function moons_pcg_update_mfp(s, coeff, upd) bind(C, name="moons_pcg_update_mfp") result(st)
      import :: c_ptr, c_int, c_double
      type(c_ptr), value :: s
      real(c_double), value :: coeff
      integer(c_int), value :: upd
      integer(c_int) :: st
    end function

    function moons_pcg_solve(s, x, b, isp, info) bind(C, name="moons_pcg_solve") result(st)
      import :: c_ptr, c_int, moons_isp, moons_solve_info
      type(c_ptr), value :: s
      type(c_ptr), intent(in) :: x(*), b(*)
      type(moons_isp), intent(in) :: isp
      type(moons_solve_info), intent(out) :: info
      integer(c_int) :: st
    end function

    function moons_pcg_destroy(s) bind(C, name="moons_pcg_destroy") result(st)
      import :: c_ptr, c_int
      type(c_ptr), value :: s
      integer(c_int) :: st
    end function

    ! learned preconditioner: a trained U-Net attached to a MOONS_PREC_UNET solver
    function moons_unet_create(m, seed, u) bind(C, name="moons_unet_create") result(st)
      import :: c_ptr, c_int, c_long_long
      type(c_ptr), value :: m
      integer(c_long_long), value :: seed
      type(c_ptr), intent(out) :: u
      integer(c_int) :: st
    end function

    function moons_unet_set_params(u, p, n) bind(C, name="moons_unet_set_params") result(st)
      import :: c_ptr, c_int, c_float, c_long_long
      type(c_ptr), value :: u
      real(c_float), intent(in) :: p(*)
      integer(c_long_long), value :: n
      integer(c_int) :: st
    end function

    function moons_unet_set_out_scale(u, c) bind(C, name="moons_unet_set_out_scale") result(st)
      import :: c_ptr, c_int, c_double
      type(c_ptr), value :: u
      real(c_double), value :: c
      integer(c_int) :: st
    end function

    function moons_unet_set_coeff(u, kx, ky, kz) bind(C, name="moons_unet_set_coeff") result(st)
      import :: c_ptr, c_int
      type(c_ptr), value :: u, kx, ky, kz
      integer(c_int) :: st
    end function

    function moons_pcg_set_unet(s, u) bind(C, name="moons_pcg_set_unet") result(st)
      import :: c_ptr, c_int
      type(c_ptr), value :: s, u
      integer(c_int) :: st
    end function

    function moons_mhd_set_unet(s, which, u) bind(C, name="moons_mhd_set_unet") result(st)
      import :: c_ptr, c_int
      type(c_ptr), value :: s, u
      integer(c_int), value :: which
      integer(c_int) :: st
    end function

    function moons_clean_div(s, x, xstar, phi, scale, temp_f, temp_cc, isp, info) &
        bind(C, name="moons_clean_div") result(st)
      import :: c_ptr, c_int, c_double, moons_isp, moons_solve_info
      type(c_ptr), value :: s, phi, temp_cc
      type(c_ptr), intent(in) :: x(*), xstar(*), temp_f(*)
      real(c_double), value :: scale
      type(moons_isp), intent(in) :: isp
      type(moons_solve_info), intent(out) :: info
      integer(c_int) :: st
    end function

    function moons_pcg_apply_op(s, ax, x) bind(C, name="moons_pcg_apply_op") result(st)
      import :: c_ptr, c_int
      type(c_ptr), value :: s
      type(c_ptr), intent(in) :: ax(*), x(*)
      integer(c_int) :: st
    end function

    function moons_pcg_apply_prec(s, z, r) bind(C, name="moons_pcg_apply_prec") result(st)
      import :: c_ptr, c_int
      type(c_ptr), value :: s
      type(c_ptr), intent(in) :: z(*), r(*)
      integer(c_int) :: st
    end function

    function moons_unet_destroy(u) bind(C, name="moons_unet_destroy") result(st)
      import :: c_ptr, c_int
      type(c_ptr), value :: u
      integer(c_int) :: st
    end function

    ! fields, BCs and the remaining discrete operators
    function moons_sf_shape(f, shp) bind(C, name="moons_sf_shape") result(st)
      import :: c_ptr, c_int
      type(c_ptr), value :: f
      integer(c_int), intent(out) :: shp(3)
      integer(c_int) :: st
    end function

    function moons_sf_fill(f, val) bind(C, name="moons_sf_fill") result(st)
      import :: c_ptr, c_int, c_double
      type(c_ptr), value :: f
      real(c_double), value :: val
      integer(c_int) :: st
    end function

    function moons_mesh_sync(m) bind(C, name="moons_mesh_sync") result(st)
      import :: c_ptr, c_int
      type(c_ptr), value :: m
      integer(c_int) :: st
    end function

    function moons_apply_bcs_implicit(f) bind(C, name="moons_apply_bcs_implicit") result(st)
      import :: c_ptr, c_int
      type(c_ptr), value :: f
      integer(c_int) :: st
    end function

    ! del%assign/add/subtract (ops_del.f90:236-261): gen 1 assign, 2 add,
    ! 3 subtract; n the derivative order, dir 1..3, pad 0/1
    function moons_del(out, in, n, dir, pad, gen) bind(C, name="moons_del") result(st)
      import :: c_ptr, c_int
      type(c_ptr), value :: out, in
      integer(c_int), value :: n, dir, pad, gen
      integer(c_int) :: st
    end function

    function moons_interp(out, in, dir) bind(C, name="moons_interp") result(st)
      import :: c_ptr, c_int
      type(c_ptr), value :: out, in
      integer(c_int), value :: dir
      integer(c_int) :: st
    end function

    function moons_lap_centered(out, u) bind(C, name="moons_lap_centered") result(st)
      import :: c_ptr, c_int
      type(c_ptr), value :: out, u
      integer(c_int) :: st
    end function

    ! the solver's residual r = vol*(b - A x_BC - A x) for the iterate x
    function moons_pcg_residual(s, x, b, r) bind(C, name="moons_pcg_residual") result(st)
      import :: c_ptr, c_int
      type(c_ptr), value :: s
      type(c_ptr), intent(in) :: x(*), b(*), r(*)
      integer(c_int) :: st
    end function

    ! the whole step on the device (solve_MOONS, MOONS_solver.f90:47-144):
    ! create from the two meshes and the parameters, upload the initial U, B,
    ! B0 and sigma through the field handles, init, then step
    function moons_mhd_create(mesh_mom, mesh_ind, prm, s) bind(C, name="moons_mhd_create") result(st)
      import :: c_ptr, c_int, moons_mhd_params
      type(c_ptr), value :: mesh_mom, mesh_ind
      type(moons_mhd_params), intent(in) :: prm
      type(c_ptr) :: s
      integer(c_int) :: st
    end function

    function moons_mhd_destroy(s) bind(C, name="moons_mhd_destroy") result(st)
      import :: c_ptr, c_int
      type(c_ptr), value :: s
      integer(c_int) :: st
    end function

    function moons_mhd_field(s, which, comp, f) bind(C, name="moons_mhd_field") result(st)
      import :: c_ptr, c_int
      type(c_ptr), value :: s
      integer(c_int), value :: which, comp
      type(c_ptr) :: f
      integer(c_int) :: st
    end function

    function moons_mhd_init(s) bind(C, name="moons_mhd_init") result(st)
      import :: c_ptr, c_int
      type(c_ptr), value :: s
      integer(c_int) :: st
    end function

    function moons_mhd_step(s, nsteps, info) bind(C, name="moons_mhd_step") result(st)
      import :: c_ptr, c_int, moons_step_info
      type(c_ptr), value :: s
      integer(c_int), value :: nsteps
      type(moons_step_info), intent(out) :: info
      integer(c_int) :: st
    end function

    function moons_mhd_divergence(s, l2_divu, l2_divb) bind(C, name="moons_mhd_divergence") result(st)
      import :: c_ptr, c_int, c_double
      type(c_ptr), value :: s
      real(c_double), intent(out) :: l2_divu, l2_divb
      integer(c_int) :: st
    end function
  end interface
end module moons_gpu_mod
