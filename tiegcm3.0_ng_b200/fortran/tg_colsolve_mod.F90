! ISO_C_BINDING interface to libtg_colsolve.so (include/tg_colsolve.h) for the
! TIE-GCM NG Fortran host.  It declares the C entry points; the drop-in
! wrappers that keep the reference's subroutine names and arguments are shown
! in INTEGRATION.md (they need the model's params_module / fields_ng_module).
!
! No Fortran compiler exists in the build image, so this module is not
! compiled here; the C ABI it binds is exercised from C and Python instead.
module tg_colsolve_mod
  use iso_c_binding, only: c_int, c_long, c_double, c_ptr, c_null_ptr
  implicit none

  integer(c_int), parameter :: TG_OK = 0, TG_EINVAL = 1, TG_EPIVOT = 2, TG_ENONFINITE = 3, &
    TG_ENOCONV = 4, TG_ETIMEOUT = 5, TG_ECUDA = 6, TG_ENOMEM = 7, TG_ENODEV = 8
  integer(c_int), parameter :: TG_PREC_F64 = 0, TG_PREC_F32_REFINE = 1

  interface
    ! trsolv (src/trsolv.F:2): one latitude slab (lev0:lev1, lon0:lon1)
    integer(c_int) function tg_trsolv(a, b, c, f, x, lev0, lev1, k1, k2, lon0, lon1, lonmax) &
        bind(C, name="tg_trsolv")
      import :: c_int, c_double
      real(c_double), intent(in) :: a(*), b(*), c(*), f(*)
      real(c_double), intent(inout) :: x(*)
      integer(c_int), value :: lev0, lev1, k1, k2, lon0, lon1, lonmax
    end function tg_trsolv

    ! trsolv_ng (src/trsolv_ng.F90:1): all ghost-inclusive columns of a nest
    integer(c_int) function tg_trsolv_ng(a, b, c, f, x, nk, k2, ncol) bind(C, name="tg_trsolv_ng")
      import :: c_int, c_double
      real(c_double), intent(in) :: a(*), b(*), c(*), f(*)
      real(c_double), intent(inout) :: x(*)
      integer(c_int), value :: nk, k2, ncol
    end function tg_trsolv_ng

    ! blktri (src/duv.F:801): 2x2 blocks on one slab
    integer(c_int) function tg_blktri(a, b, c, f, x, lev0, lev1, lon0, lon1, nlonp4) &
        bind(C, name="tg_blktri")
      import :: c_int, c_double
      real(c_double), intent(in) :: a(*), b(*), c(*), f(*)
      real(c_double), intent(inout) :: x(*)
      integer(c_int), value :: lev0, lev1, lon0, lon1, nlonp4
    end function tg_blktri

    ! comp_ng 3x3 block solve (src/comp_ng.F90:166-332); ubc_add may be c_null_ptr
    integer(c_int) function tg_comp_blksolve_ng(nb, p, q, r, f, ubc_ratio, ubc_add, u, nk, ncol) &
        bind(C, name="tg_comp_blksolve_ng")
      import :: c_int, c_double, c_ptr
      integer(c_int), value :: nb, nk, ncol
      real(c_double), intent(in) :: p(*), q(*), r(*), f(*)
      type(c_ptr), value :: ubc_ratio, ubc_add
      real(c_double), intent(inout) :: u(*)
    end function tg_comp_blksolve_ng

    integer(c_int) function tg_set_host_precision(precision) bind(C, name="tg_set_host_precision")
      import :: c_int
      integer(c_int), value :: precision
    end function tg_set_host_precision

    integer(c_int) function tg_release_buffers() bind(C, name="tg_release_buffers")
      import :: c_int
    end function tg_release_buffers
  end interface
end module tg_colsolve_mod
