! ISO_C_BINDING interface to libtg_colsolve.so (include/tg_colsolve.h) for the
! TIE-GCM NG Fortran host.  It declares the C entry points; the drop-in
! wrappers that keep the reference's subroutine names and arguments belong to
! the model's side, since they need its params_module / fields_ng_module.
!
! No Fortran compiler exists in the build image, so this module is not
! compiled here; the C ABI it binds is exercised from C and Python instead.
module tg_colsolve_mod
  use iso_c_binding, only: c_int, c_long, c_double, c_ptr, c_null_ptr
  implicit none

  integer(c_int), parameter :: TG_OK = 0, TG_EINVAL = 1, TG_EPIVOT = 2, TG_ENONFINITE = 3, &
    TG_ENOCONV = 4, TG_ETIMEOUT = 5, TG_ECUDA = 6, TG_ENOMEM = 7, TG_ENODEV = 8
  integer(c_int), parameter :: TG_PREC_F64 = 0, TG_PREC_F32_REFINE = 1
  integer(c_int), parameter :: TG_FILTER_DT = 0, TG_FILTER_MINOR = 1, TG_FILTER_OPLUS = 2
  integer(c_int), parameter :: TG_LAYOUT_COLUMN = 0, TG_LAYOUT_LEVEL = 1
  integer(c_int), parameter :: TG_KIND_SCALAR = 0, TG_KIND_BLOCK2 = 2, TG_KIND_BLOCK3 = 3

  ! One system of a batched host call (tg_solve_host): c_loc() of the
  ! Fortran arrays, block systems with P, Q, R in a, b, c and u in x.
  type, bind(C) :: tg_host_system
    integer(c_int) :: kind, nk, k2, ncol
    type(c_ptr) :: a = c_null_ptr, b = c_null_ptr, c = c_null_ptr, f = c_null_ptr, x = c_null_ptr
    type(c_ptr) :: ubc_ratio = c_null_ptr, ubc_add = c_null_ptr
  end type tg_host_system

  ! One segment of a GPU-resident plan: device pointers (CUDA Fortran
  ! c_devloc, OpenACC host_data use_device), level-major with stride ld.
  type, bind(C) :: tg_segment
    integer(c_int) :: kind, nk, k2, ncol
    integer(c_long) :: ld
    type(c_ptr) :: a = c_null_ptr, b = c_null_ptr, c = c_null_ptr, f = c_null_ptr, x = c_null_ptr
    type(c_ptr) :: ubc_ratio = c_null_ptr, ubc_add = c_null_ptr
  end type tg_segment

  ! Field tables of the fused assembly + solve entries: c_loc() of each
  ! Fortran array (3-D fields (nk, ncol), 2-D (ncol), level profiles (nk)),
  ! in the order of the C structs in include/tg_colsolve.h.
  type, bind(C) :: tg_dt_fields
    type(c_ptr) :: tn, tnsmooth, horadv, un, vn, o1
    type(c_ptr) :: mbar, xnmbar, scht, schti, cp, kt
    type(c_ptr) :: km, hdt, qji_tn, cool_imp, cool_exp, w
    type(c_ptr) :: qtotal, rkm12, tlbc, t_lbc, ulbc, vlbc
    type(c_ptr) :: expz, dift
  end type tg_dt_fields

  type, bind(C) :: tg_dt_consts
    real(c_double) :: dz, dtx2inv, expzmid_inv, grav, p0, avo, gask, tsurplus, rmassinv_o1
  end type tg_dt_consts

  type, bind(C) :: tg_minor_fields
    type(c_ptr) :: tn, o2, o1, he, mbar, barm
    type(c_ptr) :: xnmbar, w, ftm1_smooth, hadvec, sloss, sprod
    type(c_ptr) :: tlbc, flbc1, flbc2, flbc3, fubc, dfactor
    type(c_ptr) :: expz, difk
  end type tg_minor_fields

  type, bind(C) :: tg_minor_consts
    real(c_double) :: rmx, alfax, phix(4), dzp, dtx2inv, expzmid, expzmid_inv
    real(c_double) :: rmassinv_o2, rmassinv_o1, rmassinv_n2, rmassinv_he
    real(c_double) :: rmass_o2, rmass_o1, rmass_he, rmass_n2, p0, grav, avo
    real(c_double) :: b(9), fb(3)
  end type tg_minor_consts

  type, bind(C) :: tg_comp_fields
    type(c_ptr) :: tn, o2, o1, he, w, mbar
    type(c_ptr) :: o2nm_smooth, o1nm_smooth, henm_smooth, o2_advec, o1_advec, he_advec
    type(c_ptr) :: hdo2, hdo1, hdhe, fs, tlbc, flx_he
    type(c_ptr) :: dfactor, expz, difk
  end type tg_comp_fields

  type, bind(C) :: tg_comp_consts
    real(c_double) :: dz, dtx2inv, expzmid, expzmid_inv
    real(c_double) :: rmassinv_o2, rmassinv_o1, rmassinv_he, rmassinv_n2
    real(c_double) :: rmass_o2, rmass_o1, rmass_he, p0, grav
    real(c_double) :: b(9), fb(3)
    real(c_double) :: pshelb
    integer(c_int) :: calc_helium
  end type tg_comp_consts

  type, bind(C) :: tg_settei_fields
    type(c_ptr) :: tn, o2, o1, he, n2, ne
    type(c_ptr) :: te, ti, op, o2p, nplus, n2p
    type(c_ptr) :: nop, xnmbar, xnmbari, scht, schti, qji_ti
    type(c_ptr) :: qop2p, qop2d, qo2p, qop, qn2p, qnp
    type(c_ptr) :: qnop, Q1, Q2, t_lbc, chi, rlatm
    type(c_ptr) :: dipmag, qteaur
  end type tg_settei_fields

  type, bind(C) :: tg_settei_consts
    real(c_double) :: f107, dipmin, dz, evergs, avo, rmass_o1
    real(c_double) :: rmassinv_o2, rmassinv_o1, rmassinv_he, rmassinv_n2, rmassinv_n4s, rmassinv_no
    real(c_double) :: b(9), fb(3)
    integer(c_int) :: et, electron_heating
  end type tg_settei_consts

  type, bind(C) :: tg_oplus_fields
    type(c_ptr) :: tn, te, ti, o2, o1, n2
    type(c_ptr) :: he, n2d, ne, u, v, w
    type(c_ptr) :: wi, xnmbar, scht, qop2p, qop2d, qop
    type(c_ptr) :: rk1, rk2, rk19, rk20, rk25, op
    type(c_ptr) :: optm1_smooth2, explicit_h, bdotdh_djbz, bx, by, bz
    type(c_ptr) :: dvb, rlatm, chi, dipmag, sndec, csdec
    type(c_ptr) :: zpint
  end type tg_oplus_fields

  type, bind(C) :: tg_oplus_consts
    real(c_double) :: rmass_op, gask, grav, re, rmassinv_o2, rmassinv_o1, rmassinv_n2, rmassinv_n2d, rmassinv_he
    real(c_double) :: rk10, rk16, rk17, rk18, rk21, rk22, rk23, rk24, rk26, rk27
    real(c_double) :: colfac, opdiffcap, dtx2inv, dz, dlev
    integer(c_int) :: nstep_sub
  end type tg_oplus_consts

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

    ! every system of a step in one call (host arrays, pipelined copies)
    integer(c_int) function tg_solve_host(sys, nsys) bind(C, name="tg_solve_host")
      import :: c_int, tg_host_system
      type(tg_host_system), intent(in) :: sys(*)
      integer(c_int), value :: nsys
    end function tg_solve_host

    ! device pointers, stream-ordered; status_dev and stream may be c_null_ptr
    integer(c_int) function tg_trsolv_dev(a, b, c, f, x, nk, k2, ncol, layout, ld, precision, status_dev, &
        stream) bind(C, name="tg_trsolv_dev")
      import :: c_int, c_long, c_ptr
      type(c_ptr), value :: a, b, c, f, x, status_dev, stream
      integer(c_int), value :: nk, k2, ncol, layout, precision
      integer(c_long), value :: ld
    end function tg_trsolv_dev

    integer(c_int) function tg_blksolve_dev(nb, p, q, r, f, ubc_ratio, ubc_add, u, nk, k2, ncol, layout, ld, &
        precision, status_dev, stream) bind(C, name="tg_blksolve_dev")
      import :: c_int, c_long, c_ptr
      integer(c_int), value :: nb, nk, k2, ncol, layout, precision
      type(c_ptr), value :: p, q, r, f, ubc_ratio, ubc_add, u, status_dev, stream
      integer(c_long), value :: ld
    end function tg_blksolve_dev

    ! GPU-resident plans over many segments (one persistent launch per kind)
    integer(c_int) function tg_plan_create(segs, nseg, precision, plan) bind(C, name="tg_plan_create")
      import :: c_int, c_ptr, tg_segment
      type(tg_segment), intent(in) :: segs(*)
      integer(c_int), value :: nseg, precision
      type(c_ptr), intent(out) :: plan
    end function tg_plan_create

    integer(c_int) function tg_plan_execute(plan, stream) bind(C, name="tg_plan_execute")
      import :: c_int, c_ptr
      type(c_ptr), value :: plan, stream
    end function tg_plan_execute

    integer(c_int) function tg_plan_capture_graph(plan, stream) bind(C, name="tg_plan_capture_graph")
      import :: c_int, c_ptr
      type(c_ptr), value :: plan, stream
    end function tg_plan_capture_graph

    integer(c_int) function tg_plan_status(plan, per_segment_status) bind(C, name="tg_plan_status")
      import :: c_int, c_ptr
      type(c_ptr), value :: plan
      integer(c_int), intent(out) :: per_segment_status(*)
    end function tg_plan_status

    integer(c_int) function tg_plan_destroy(plan) bind(C, name="tg_plan_destroy")
      import :: c_int, c_ptr
      type(c_ptr), value :: plan
    end function tg_plan_destroy

    integer(c_int) function tg_set_refine(max_sweeps, rel_tol) bind(C, name="tg_set_refine")
      import :: c_int, c_double
      integer(c_int), value :: max_sweeps
      real(c_double), value :: rel_tol
    end function tg_set_refine
    ! fused column assembly + solve (host arrays, Fortran layout)
    integer(c_int) function tg_dt_ng(fl, cn, tn_upd, nk, ncol) bind(C, name="tg_dt_ng")
      import :: c_int, c_double, tg_dt_fields, tg_dt_consts
      type(tg_dt_fields), intent(in) :: fl
      type(tg_dt_consts), intent(in) :: cn
      real(c_double), intent(inout) :: tn_upd(*)
      integer(c_int), value :: nk, ncol
    end function tg_dt_ng

    integer(c_int) function tg_minor_ng(fl, cn, fcomp_out, nk, ncol) bind(C, name="tg_minor_ng")
      import :: c_int, c_double, tg_minor_fields, tg_minor_consts
      type(tg_minor_fields), intent(in) :: fl
      type(tg_minor_consts), intent(in) :: cn
      real(c_double), intent(inout) :: fcomp_out(*)
      integer(c_int), value :: nk, ncol
    end function tg_minor_ng

    integer(c_int) function tg_comp_ng(fl, cn, o2_upd, o1_upd, he_upd, nk, ncol) bind(C, name="tg_comp_ng")
      import :: c_int, c_double, tg_comp_fields, tg_comp_consts
      type(tg_comp_fields), intent(in) :: fl
      type(tg_comp_consts), intent(in) :: cn
      real(c_double), intent(inout) :: o2_upd(*), o1_upd(*), he_upd(*)
      integer(c_int), value :: nk, ncol
    end function tg_comp_ng

    integer(c_int) function tg_comp_post_ng(o2, o1, he, o2_nm, o1_nm, he_nm, xnmbar, zpmid, dz, dtsmooth, &
        dtsmooth_div2, nk, ncol, o2_upd, o1_upd, he_upd, o2nm_upd, o1nm_upd, henm_upd) bind(C, name="tg_comp_post_ng")
      import :: c_int, c_double
      real(c_double), intent(in) :: o2(*), o1(*), he(*), o2_nm(*), o1_nm(*), he_nm(*), xnmbar(*), zpmid(*)
      real(c_double), value :: dz, dtsmooth, dtsmooth_div2
      integer(c_int), value :: nk, ncol
      real(c_double), intent(inout) :: o2_upd(*), o1_upd(*), he_upd(*), o2nm_upd(*), o1nm_upd(*), henm_upd(*)
    end function tg_comp_post_ng

    ! device form: level-major device arrays (stride ld), zpmid on the device
    integer(c_int) function tg_comp_post_ng_dev(o2, o1, he, o2_nm, o1_nm, he_nm, xnmbar, zpmid, dz, dtsmooth, &
        dtsmooth_div2, nk, ncol, ld, o2_upd, o1_upd, he_upd, o2nm_upd, o1nm_upd, henm_upd, bnd_mask, o2_bnd, &
        o1_bnd, he_bnd, stream) bind(C, name="tg_comp_post_ng_dev")
      import :: c_int, c_long, c_double, c_ptr
      type(c_ptr), value :: o2, o1, he, o2_nm, o1_nm, he_nm, xnmbar, zpmid
      real(c_double), value :: dz, dtsmooth, dtsmooth_div2
      integer(c_int), value :: nk, ncol
      integer(c_long), value :: ld
      type(c_ptr), value :: o2_upd, o1_upd, he_upd, o2nm_upd, o1nm_upd, henm_upd
      type(c_ptr), value :: bnd_mask, o2_bnd, o1_bnd, he_bnd, stream
    end function tg_comp_post_ng_dev

    ! which = TG_FILTER_DT / _MINOR / _OPLUS: the time filter and floor after
    ! the lateral-boundary hook (dt_ng.F90:208-213, minor_ng.F90:234-237,
    ! oplus_ng.F90:337-340); upd floored in place, nm_upd the filtered field
    integer(c_int) function tg_time_filter_ng(which, cur, prev, dtsmooth, dtsmooth_div2, nk, ncol, upd, nm_upd) &
        bind(C, name="tg_time_filter_ng")
      import :: c_int, c_double
      integer(c_int), value :: which, nk, ncol
      real(c_double), intent(in) :: cur(*), prev(*)
      real(c_double), value :: dtsmooth, dtsmooth_div2
      real(c_double), intent(inout) :: upd(*), nm_upd(*)
    end function tg_time_filter_ng

    ! advec_ng / smooth_ng (src/advec_ng.F90, src/smooth_ng.F90) for a nest
    ! held as one subdomain: f, un, vn, hadvec, fin, fout (nk, lond0:lond1,
    ! latd0:latd1), racs (latd0:latd1)
    integer(c_int) function tg_advec_ng(f, un, vn, racs, dlamda, dphi, re_inv, nk, nlon, nlat, hadvec) &
        bind(C, name="tg_advec_ng")
      import :: c_int, c_double
      real(c_double), intent(in) :: f(*), un(*), vn(*), racs(*)
      real(c_double), value :: dlamda, dphi, re_inv
      integer(c_int), value :: nk, nlon, nlat
      real(c_double), intent(inout) :: hadvec(*)
    end function tg_advec_ng

    integer(c_int) function tg_smooth_ng(fin, shapiro, nk, nlon, nlat, fout) bind(C, name="tg_smooth_ng")
      import :: c_int, c_double
      real(c_double), intent(in) :: fin(*)
      real(c_double), value :: shapiro
      integer(c_int), value :: nk, nlon, nlat
      real(c_double), intent(inout) :: fout(*)
    end function tg_smooth_ng

    integer(c_int) function tg_settei_ng(fl, cn, te_out, ti_out, qtotal, nk, ncol) bind(C, name="tg_settei_ng")
      import :: c_int, c_double, tg_settei_fields, tg_settei_consts
      type(tg_settei_fields), intent(in) :: fl
      type(tg_settei_consts), intent(in) :: cn
      real(c_double), intent(inout) :: te_out(*), ti_out(*), qtotal(*)
      integer(c_int), value :: nk, ncol
    end function tg_settei_ng

    ! Fe and Fn may be c_null_ptr (both or neither)
    integer(c_int) function tg_oplus_ng(fl, cn, opout, xiop2p, xiop2d, fe, fn, nk, ncol) bind(C, name="tg_oplus_ng")
      import :: c_int, c_double, c_ptr, tg_oplus_fields, tg_oplus_consts
      type(tg_oplus_fields), intent(in) :: fl
      type(tg_oplus_consts), intent(in) :: cn
      real(c_double), intent(inout) :: opout(*), xiop2p(*), xiop2d(*)
      type(c_ptr), value :: fe, fn
      integer(c_int), value :: nk, ncol
    end function tg_oplus_ng

    ! the polar ring filter of a global field held whole, f(nk, nlonp4, nlat):
    ! filter_o2o's latscan loop over ringfilter (comp.F:1109-1125) becomes
    !   istat = tg_filter_o2o(fkij, nlevs, nlon, nlat, chunk_array, nlat_filter, dlamda)
    integer(c_int) function tg_ringfilter(f, nk, nlon, nlat, order, poly, chunk_array, nlat_filter, dlamda) &
        bind(C, name="tg_ringfilter")
      import :: c_int, c_double
      real(c_double), intent(inout) :: f(*)
      integer(c_int), value :: nk, nlon, nlat, order, poly, nlat_filter
      integer(c_int), intent(in) :: chunk_array(*)
      real(c_double), value :: dlamda
    end function tg_ringfilter

    integer(c_int) function tg_filter_o2o(fout, nk, nlon, nlat, chunk_array, nlat_filter, dlamda) &
        bind(C, name="tg_filter_o2o")
      import :: c_int, c_double
      real(c_double), intent(inout) :: fout(*)
      integer(c_int), value :: nk, nlon, nlat, nlat_filter
      integer(c_int), intent(in) :: chunk_array(*)
      real(c_double), value :: dlamda
    end function tg_filter_o2o
  end interface
end module tg_colsolve_mod
