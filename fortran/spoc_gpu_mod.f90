! ISO_C_BINDING interface to the C ABI in include/spoc_gpu.h.
!
! A Fortran driver (src/shwwnl.f, src/shw_cpu.f, src/shwwnl_adap.f) has two
! ways in:
!   1. Link-time drop-in: link libspoc_gpu.so instead of calvar*.o.  The
!      library exports cal_var_ with the reference argument list, so
!      `call cal_var(...)` is unchanged; call spoc_register_commons_f once
!      after the two dpotrf calls (src/shwwnl.f:153-156).
!   2. Handle API: spoc_create / spoc_set_params / spoc_rk4_steps keep the
!      state on the GPU between steps.
! This file is compiled with the driver (gfortran -c spoc_gpu_mod.f90).
module spoc_gpu_mod
  use iso_c_binding
  implicit none

  integer(c_int), parameter :: SPOC_LIN = 0, SPOC_FS = 1, SPOC_NS = 2, SPOC_INV = 3
  integer(c_int), parameter :: SPOC_FP64 = 0

  type, bind(c) :: spoc_tables
    integer(c_int) :: nc, nm, ng, ngf
    type(c_ptr) :: wi, xi, yi, wif, tif
    type(c_ptr) :: pi2
    integer(c_int) :: ld_pi2
    type(c_ptr) :: pico
    integer(c_int) :: ld_pico1, ld_pico2
    type(c_ptr) :: amm, amml, agx, agy, ammo
    integer(c_int) :: ld_mat
    type(c_ptr) :: cip
  end type spoc_tables

  type, bind(c) :: spoc_mesh
    integer(c_int) :: ne, nf
    type(c_ptr) :: itm, its, tseg, ssit, norm, vect, normt, bdl
  end type spoc_mesh

  type, bind(c) :: spoc_params
    real(c_double) :: mu0, mb0, g0
    type(c_ptr) :: fc, w0, z0, hb
    integer(c_int) :: ld
  end type spoc_params

  interface
    integer(c_int) function spoc_register_commons(t, variant, precision) bind(c, name='spoc_register_commons')
      import :: c_int, spoc_tables
      type(spoc_tables), intent(in) :: t
      integer(c_int), value :: variant, precision
    end function

    function spoc_cal_var_status() bind(c, name='spoc_cal_var_status')
      import :: c_ptr
      type(c_ptr) :: spoc_cal_var_status
    end function

    subroutine spoc_cal_var_refresh() bind(c, name='spoc_cal_var_refresh')
    end subroutine

    subroutine spoc_release_commons() bind(c, name='spoc_release_commons')
    end subroutine

    integer(c_int) function spoc_create(t, m, variant, precision, h) bind(c, name='spoc_create')
      import :: c_int, c_ptr, spoc_tables, spoc_mesh
      type(spoc_tables), intent(in) :: t
      type(spoc_mesh), intent(in) :: m
      integer(c_int), value :: variant, precision
      type(c_ptr), intent(out) :: h
    end function

    subroutine spoc_destroy(h) bind(c, name='spoc_destroy')
      import :: c_ptr
      type(c_ptr), value :: h
    end subroutine

    integer(c_int) function spoc_set_params(h, p) bind(c, name='spoc_set_params')
      import :: c_int, c_ptr, spoc_params
      type(c_ptr), value :: h
      type(spoc_params), intent(in) :: p
    end function

    integer(c_int) function spoc_cal_var(h, ld, u0, v0, h0, u1, v1, h1) bind(c, name='spoc_cal_var')
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: h
      integer(c_int), value :: ld
      real(c_double), intent(in) :: u0(ld,*), v0(ld,*), h0(ld,*)
      real(c_double), intent(out) :: u1(ld,*), v1(ld,*), h1(ld,*)
    end function

    integer(c_int) function spoc_set_state(h, ld, u, v, hh) bind(c, name='spoc_set_state')
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: h
      integer(c_int), value :: ld
      real(c_double), intent(in) :: u(ld,*), v(ld,*), hh(ld,*)
    end function

    integer(c_int) function spoc_get_state(h, ld, u, v, hh) bind(c, name='spoc_get_state')
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: h
      integer(c_int), value :: ld
      real(c_double), intent(out) :: u(ld,*), v(ld,*), hh(ld,*)
    end function

    integer(c_int) function spoc_rk4_steps(h, dt, nsteps) bind(c, name='spoc_rk4_steps')
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: h
      real(c_double), value :: dt
      integer(c_int), value :: nsteps
    end function

    integer(c_int) function spoc_energy(h, ke, pe, mass) bind(c, name='spoc_energy')
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: h
      real(c_double), intent(out) :: ke, pe, mass
    end function

    ! Regridding (src/shwwnl_adap.f:375-450): cal_conv's flags on the device,
    ! then interpol / verif_rot / checkcfl2 of the state onto a new handle.
    ! fconv, fderaff are logical*4 arrays in the reference (0 / 1 here).
    integer(c_int) function spoc_cal_conv(h, fac1, fac2, fac3, fconv, fderaff, flags, supmax) &
        bind(c, name='spoc_cal_conv')
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: h
      real(c_double), value :: fac1, fac2, fac3
      integer(c_int), intent(out) :: fconv(*), fderaff(*), flags(3)
      real(c_double), intent(out) :: supmax
    end function

    integer(c_int) function spoc_inter_only_new(ne, nenew, in, innew, tinter) &
        bind(c, name='spoc_inter_only_new')
      import :: c_int
      integer(c_int), value :: ne, nenew
      integer(c_int), intent(in) :: in(3,*), innew(3,*)
      integer(c_int), intent(out) :: tinter(*)
    end function

    integer(c_int) function spoc_locate_points(ne, in, itm, tseg, pseg, xgr, ygr, nenew, &
        innew, xgrnew, ygrnew, tinter, ng, xi, yi, pt_elem, pt_x, pt_y) &
        bind(c, name='spoc_locate_points')
      import :: c_int, c_double
      integer(c_int), value :: ne, nenew, ng
      integer(c_int), intent(in) :: in(3,*), itm(3,*), tseg(2,*), pseg(2,*), innew(3,*), tinter(*)
      real(c_double), intent(in) :: xgr(*), ygr(*), xgrnew(*), ygrnew(*), xi(*), yi(*)
      integer(c_int), intent(out) :: pt_elem(ng,*)
      real(c_double), intent(out) :: pt_x(ng,*), pt_y(ng,*)
    end function

    integer(c_int) function spoc_interpol(dst, src, tinter, pt_elem, pt_x, pt_y) &
        bind(c, name='spoc_interpol')
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: dst, src
      integer(c_int), intent(in) :: tinter(*), pt_elem(*)
      real(c_double), intent(in) :: pt_x(*), pt_y(*)
    end function

    integer(c_int) function spoc_verif_rot(h) bind(c, name='spoc_verif_rot')
      import :: c_int, c_ptr
      type(c_ptr), value :: h
    end function

    ! write_gra's values for all elements: out(5, np, ne) = x, y, u, v, h
    integer(c_int) function spoc_lattice(h, ngraph, nn, in, xgr, ygr, out) &
        bind(c, name='spoc_lattice')
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: h
      integer(c_int), value :: ngraph, nn
      integer(c_int), intent(in) :: in(3,*)
      real(c_double), intent(in) :: xgr(*), ygr(*)
      real(c_double), intent(out) :: out(5,*)
    end function

    integer(c_int) function spoc_cfl2(h, ngraph, nn, in, xgr, ygr, dt_in, cflmin, dt) &
        bind(c, name='spoc_cfl2')
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: h
      integer(c_int), value :: ngraph, nn
      integer(c_int), intent(in) :: in(3,*)
      real(c_double), intent(in) :: xgr(*), ygr(*)
      real(c_double), value :: dt_in
      real(c_double), intent(out) :: cflmin, dt
    end function
  end interface

contains

  ! Register the COMMON tables of src/shwwnl.f:60-71 (after dpotrf).  All
  ! arrays keep their reference declarations: pi2(ng_max,nnmod),
  ! pico(ngf_max,nnmod,3), matrices (nnmod,nnmod), cip(2,0:nnmod).
  integer(c_int) function spoc_register_commons_f(variant, nc, nm, ng, ngf, ng_max, ngf_max, &
      nnmod, wi, xi, yi, wif, tif, pi2, pico, amm, amml, agx, agy, ammo, cip) result(rc)
    integer, intent(in) :: variant, nc, nm, ng, ngf, ng_max, ngf_max, nnmod
    real(c_double), target, intent(in) :: wi(*), xi(*), yi(*), wif(*), tif(*)
    real(c_double), target, intent(in) :: pi2(ng_max,*), pico(ngf_max,nnmod,*)
    real(c_double), target, intent(in) :: amm(nnmod,*), amml(nnmod,*), agx(nnmod,*), agy(nnmod,*), ammo(nnmod,*)
    integer(c_int), target, intent(in) :: cip(2,0:*)
    type(spoc_tables) :: t
    t%nc = nc; t%nm = nm; t%ng = ng; t%ngf = ngf
    t%wi = c_loc(wi(1)); t%xi = c_loc(xi(1)); t%yi = c_loc(yi(1))
    t%wif = c_loc(wif(1)); t%tif = c_loc(tif(1))
    t%pi2 = c_loc(pi2(1,1)); t%ld_pi2 = ng_max
    t%pico = c_loc(pico(1,1,1)); t%ld_pico1 = ngf_max; t%ld_pico2 = nnmod
    t%amm = c_loc(amm(1,1)); t%amml = c_loc(amml(1,1)); t%agx = c_loc(agx(1,1))
    t%agy = c_loc(agy(1,1)); t%ammo = c_loc(ammo(1,1)); t%ld_mat = nnmod
    t%cip = c_loc(cip(1,0))
    rc = spoc_register_commons(t, int(variant, c_int), SPOC_FP64)
  end function

end module spoc_gpu_mod
