"""Python mirror of the reference's column-solver interface over the C ABI of
libtg_colsolve.so (include/tg_colsolve.h).

The functions keep the reference's names, argument order and meaning:

  trsolv(a,b,c,f,x,lev0,lev1,k1,k2,lon0,lon1,lonmax,lat,idebug)   src/trsolv.F:2
  trsolv_ng(a,b,c,f,x,k2,i_ng)                                     src/trsolv_ng.F90:1
  blktri(a,b,c,f,beta,gamma,y,x,lev0,lev1,lon0,lon1,nlonp4)        src/duv.F:801
  comp_blksolve_ng(P,Q,R,f,u,ubc_ratio,ubc_add)                    src/comp_ng.F90:166-332

Host arrays are numpy float64 arrays in the reference's Fortran layouts
(order='F'); x/u are written in place, as the Fortran intent(out) arguments
are.  Like the reference, a zero pivot does not raise: the numbers come out
as Inf/NaN exactly as the Fortran would produce them, and the call returns the
status code (TG_EPIVOT).  Argument and CUDA errors raise TgError.

Device entry points (trsolv_dev, blksolve_dev, Plan) take raw device
pointers (ints) or torch CUDA tensors.

There is no CPU fallback: if the CUDA library is missing the import of this
module's functions fails with an error.
"""
import ctypes
import os

import numpy as np

TG_OK, TG_EINVAL, TG_EPIVOT, TG_ENONFINITE, TG_ENOCONV, TG_ETIMEOUT, TG_ECUDA, TG_ENOMEM, TG_ENODEV = range(9)
STATUS_NAMES = {0: "TG_OK", 1: "TG_EINVAL", 2: "TG_EPIVOT", 3: "TG_ENONFINITE", 4: "TG_ENOCONV",
                5: "TG_ETIMEOUT", 6: "TG_ECUDA", 7: "TG_ENOMEM", 8: "TG_ENODEV"}
TG_PREC_F64, TG_PREC_F32_REFINE = 0, 1
TG_LAYOUT_COLUMN, TG_LAYOUT_LEVEL = 0, 1
TG_KIND_SCALAR, TG_KIND_BLOCK2, TG_KIND_BLOCK3 = 0, 2, 3
TG_FILTER_DT, TG_FILTER_MINOR, TG_FILTER_OPLUS = 0, 1, 2
NUMERIC_STATUS = (TG_OK, TG_EPIVOT, TG_ENONFINITE, TG_ENOCONV)

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libtg_colsolve.so")

# Every symbol include/tg_colsolve.h declares.
EXPORTS = ("tg_solve_host", "tg_dt_ng", "tg_dt_ng_dev", "tg_minor_ng", "tg_minor_ng_dev", "tg_comp_ng",
           "tg_comp_ng_dev", "tg_comp_post_ng", "tg_comp_post_ng_dev", "tg_comp_diag_ng", "tg_comp_diag_ng_dev", "tg_oplus_ng_factor_doubles", "tg_oplus_diag_ng", "tg_oplus_diag_ng_dev", "tg_oplus_ng_factor_dev", "tg_oplus_ng_solve_dev", "tg_time_filter_ng", "tg_time_filter_ng_dev", "tg_advec_ng", "tg_advec_ng_dev", "tg_smooth_ng", "tg_smooth_ng_dev", "tg_settei_ng", "tg_settei_ng_dev", "tg_oplus_ng",
           "tg_oplus_ng_dev", "tg_trsolv", "tg_trsolv_ng", "tg_blktri", "tg_comp_blksolve_ng", "tg_blksolve", "tg_trsolv_dev",
           "tg_blksolve_dev", "tg_blksolve_dev_noalloc", "tg_plan_create", "tg_plan_execute", "tg_plan_capture_graph",
           "tg_plan_status", "tg_plan_launches", "tg_plan_describe", "tg_set_cache_hints", "tg_set_block_rows", "tg_set_block_width", "tg_set_stage_levels", "tg_set_column_residency", "tg_set_assembly_mode", "tg_set_walk_prefetch", "tg_set_block_scratch_budget", "tg_set_scalar_scratch_budget", "tg_set_kind_overlap", "tg_set_host_pipeline", "tg_selftest_wait", "tg_plan_sweep_histogram", "tg_plan_destroy",
           "tg_set_refine", "tg_set_host_precision", "tg_set_tile", "tg_set_pipeline", "tg_set_prefetch", "tg_set_scratch_global", "tg_selftest_division", "tg_selftest_walk", "tg_release_buffers", "tg_version", "tg_kernel_arch", "tg_ringfilter", "tg_ringfilter_dev", "tg_filter_o2o", "tg_trsolv_defer", "tg_trsolv_flush", "tg_dt_diag_ng", "tg_dt_diag_ng_dev", "tg_minor_diag_ng", "tg_minor_diag_ng_dev", "tg_dt_ng_post_dev", "tg_minor_ng_post_dev", "tg_oplus_ng_post_dev", "tg_last_error")


class PostStepArgs(ctypes.Structure):
    """tg_post_step of include/tg_colsolve.h."""
    _fields_ = [("cur", ctypes.c_void_p), ("prev", ctypes.c_void_p), ("nm_upd", ctypes.c_void_p),
                ("bnd_mask", ctypes.c_void_p), ("bnd", ctypes.c_void_p), ("dtsmooth", ctypes.c_double),
                ("dtsmooth_div2", ctypes.c_double)]


class TgError(RuntimeError):
    def __init__(self, status, where):
        self.status = status
        msg = lib().tg_last_error().decode(errors="replace")
        super().__init__(f"{where}: {STATUS_NAMES.get(status, status)}: {msg}")


class Segment(ctypes.Structure):
    """tg_segment of include/tg_colsolve.h."""
    _fields_ = [("kind", ctypes.c_int), ("nk", ctypes.c_int), ("k2", ctypes.c_int), ("ncol", ctypes.c_int),
                ("ld", ctypes.c_long),
                ("a", ctypes.c_void_p), ("b", ctypes.c_void_p), ("c", ctypes.c_void_p), ("f", ctypes.c_void_p),
                ("x", ctypes.c_void_p), ("ubc_ratio", ctypes.c_void_p), ("ubc_add", ctypes.c_void_p)]


DT_FIELDS = ("tn", "tnsmooth", "horadv", "un", "vn", "o1", "mbar", "xnmbar", "scht", "schti", "cp", "kt", "km",
             "hdt", "qji_tn", "cool_imp", "cool_exp", "w", "qtotal", "rkm12", "tlbc", "t_lbc", "ulbc", "vlbc",
             "expz", "dift")
DT_CONSTS = ("dz", "dtx2inv", "expzmid_inv", "grav", "p0", "avo", "gask", "tsurplus", "rmassinv_o1")


class HostSystem(ctypes.Structure):
    """tg_host_system of include/tg_colsolve.h."""
    _fields_ = [("kind", ctypes.c_int), ("nk", ctypes.c_int), ("k2", ctypes.c_int), ("ncol", ctypes.c_int),
                ("a", ctypes.c_void_p), ("b", ctypes.c_void_p), ("c", ctypes.c_void_p), ("f", ctypes.c_void_p),
                ("x", ctypes.c_void_p), ("ubc_ratio", ctypes.c_void_p), ("ubc_add", ctypes.c_void_p)]


class DtFields(ctypes.Structure):
    """tg_dt_fields of include/tg_colsolve.h."""
    _fields_ = [(n, ctypes.c_void_p) for n in DT_FIELDS]


class DtConsts(ctypes.Structure):
    """tg_dt_consts of include/tg_colsolve.h."""
    _fields_ = [(n, ctypes.c_double) for n in DT_CONSTS]


MINOR_FIELDS = ("tn", "o2", "o1", "he", "mbar", "barm", "xnmbar", "w", "ftm1_smooth", "hadvec", "sloss", "sprod",
                "tlbc", "flbc1", "flbc2", "flbc3", "fubc", "dfactor", "expz", "difk")
MINOR_SCALARS = ("rmx", "alfax")
MINOR_CONSTS2 = ("dzp", "dtx2inv", "expzmid", "expzmid_inv", "rmassinv_o2", "rmassinv_o1", "rmassinv_n2",
                 "rmassinv_he", "rmass_o2", "rmass_o1", "rmass_he", "rmass_n2", "p0", "grav", "avo")


class MinorFields(ctypes.Structure):
    """tg_minor_fields of include/tg_colsolve.h."""
    _fields_ = [(n, ctypes.c_void_p) for n in MINOR_FIELDS]


class MinorConsts(ctypes.Structure):
    """tg_minor_consts of include/tg_colsolve.h."""
    _fields_ = ([("rmx", ctypes.c_double), ("alfax", ctypes.c_double), ("phix", ctypes.c_double * 4)] +
                [(n, ctypes.c_double) for n in MINOR_CONSTS2] +
                [("b", ctypes.c_double * 9), ("fb", ctypes.c_double * 3)])


def minor_consts(c):
    return MinorConsts(c["rmx"], c["alfax"], (ctypes.c_double * 4)(*c["phix"]), *[float(c[n]) for n in MINOR_CONSTS2],
                       (ctypes.c_double * 9)(*np.ravel(c["b"], order="F")), (ctypes.c_double * 3)(*c["fb"]))


COMP_FIELDS = ("tn", "o2", "o1", "he", "w", "mbar", "o2nm_smooth", "o1nm_smooth", "henm_smooth", "o2_advec",
               "o1_advec", "he_advec", "hdo2", "hdo1", "hdhe", "fs", "tlbc", "flx_he", "dfactor", "expz", "difk")
COMP_CONSTS = ("dz", "dtx2inv", "expzmid", "expzmid_inv", "rmassinv_o2", "rmassinv_o1", "rmassinv_he",
               "rmassinv_n2", "rmass_o2", "rmass_o1", "rmass_he", "p0", "grav")


class CompFields(ctypes.Structure):
    """tg_comp_fields of include/tg_colsolve.h."""
    _fields_ = [(n, ctypes.c_void_p) for n in COMP_FIELDS]


class CompConsts(ctypes.Structure):
    """tg_comp_consts of include/tg_colsolve.h."""
    _fields_ = ([(n, ctypes.c_double) for n in COMP_CONSTS] +
                [("b", ctypes.c_double * 9), ("fb", ctypes.c_double * 3), ("pshelb", ctypes.c_double),
                 ("calc_helium", ctypes.c_int)])


def comp_consts(c):
    return CompConsts(*[float(c[n]) for n in COMP_CONSTS], (ctypes.c_double * 9)(*np.ravel(c["b"], order="F")),
                      (ctypes.c_double * 3)(*c["fb"]), float(c.get("pshelb", 0.1154e-5)),
                      int(c.get("calc_helium", 1)))


SETTEI_FIELDS = ("tn", "o2", "o1", "he", "n2", "ne", "te", "ti", "op", "o2p", "nplus", "n2p", "nop", "xnmbar",
                 "xnmbari", "scht", "schti", "qji_ti", "qop2p", "qop2d", "qo2p", "qop", "qn2p", "qnp", "qnop",
                 "Q1", "Q2", "t_lbc", "chi", "rlatm", "dipmag", "qteaur")
SETTEI_CONSTS = ("f107", "dipmin", "dz", "evergs", "avo", "rmass_o1", "rmassinv_o2", "rmassinv_o1",
                 "rmassinv_he", "rmassinv_n2", "rmassinv_n4s", "rmassinv_no")


class SetteiFields(ctypes.Structure):
    """tg_settei_fields of include/tg_colsolve.h."""
    _fields_ = [(n, ctypes.c_void_p) for n in SETTEI_FIELDS]


class SetteiConsts(ctypes.Structure):
    """tg_settei_consts of include/tg_colsolve.h."""
    _fields_ = ([(n, ctypes.c_double) for n in SETTEI_CONSTS] +
                [("b", ctypes.c_double * 9), ("fb", ctypes.c_double * 3), ("et", ctypes.c_int),
                 ("electron_heating", ctypes.c_int)])


def settei_consts(c):
    return SetteiConsts(*[float(c[n]) for n in SETTEI_CONSTS], (ctypes.c_double * 9)(*np.ravel(c["b"], order="F")),
                        (ctypes.c_double * 3)(*c["fb"]), int(c.get("et", 0)), int(c.get("electron_heating", 0)))


OPLUS_FIELDS = ("tn", "te", "ti", "o2", "o1", "n2", "he", "n2d", "ne", "u", "v", "w", "wi", "xnmbar", "scht",
                "qop2p", "qop2d", "qop", "rk1", "rk2", "rk19", "rk20", "rk25", "op", "optm1_smooth2", "explicit_h",
                "bdotdh_djbz", "bx", "by", "bz", "dvb", "rlatm", "chi", "dipmag", "sndec", "csdec", "zpint")
OPLUS_CONSTS = ("rmass_op", "gask", "grav", "re", "rmassinv_o2", "rmassinv_o1", "rmassinv_n2", "rmassinv_n2d",
                "rmassinv_he", "rk10", "rk16", "rk17", "rk18", "rk21", "rk22", "rk23", "rk24", "rk26", "rk27",
                "colfac", "opdiffcap", "dtx2inv", "dz", "dlev")


class OplusFields(ctypes.Structure):
    """tg_oplus_fields of include/tg_colsolve.h."""
    _fields_ = [(n, ctypes.c_void_p) for n in OPLUS_FIELDS]


class OplusConsts(ctypes.Structure):
    """tg_oplus_consts of include/tg_colsolve.h."""
    _fields_ = [(n, ctypes.c_double) for n in OPLUS_CONSTS] + [("nstep_sub", ctypes.c_int)]


def oplus_consts(c):
    return OplusConsts(*[float(c[n]) for n in OPLUS_CONSTS], int(c["nstep_sub"]))


_lib = None


def lib():
    """Loads libtg_colsolve.so; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: build it with tiegcm3.0_ng_b200/build.py "
                              "(there is no CPU fallback)")
        L = ctypes.CDLL(LIB_PATH)
        P, I, Lg, D = ctypes.c_void_p, ctypes.c_int, ctypes.c_long, ctypes.c_double
        sig = {
            "tg_trsolv": [P, P, P, P, P, I, I, I, I, I, I, I],
            "tg_dt_ng": [ctypes.POINTER(DtFields), ctypes.POINTER(DtConsts), P, I, I],
            "tg_solve_host": [ctypes.POINTER(HostSystem), I],
            "tg_minor_ng": [ctypes.POINTER(MinorFields), ctypes.POINTER(MinorConsts), P, I, I],
            "tg_comp_ng": [ctypes.POINTER(CompFields), ctypes.POINTER(CompConsts), P, P, P, I, I],
            "tg_settei_ng": [ctypes.POINTER(SetteiFields), ctypes.POINTER(SetteiConsts), P, P, P, I, I],
            "tg_oplus_ng": [ctypes.POINTER(OplusFields), ctypes.POINTER(OplusConsts), P, P, P, P, P, I, I],
            "tg_oplus_ng_dev": [ctypes.POINTER(OplusFields), ctypes.POINTER(OplusConsts), P, P, P, P, P, I, I, Lg, P,
                                P, P],
            "tg_settei_ng_dev": [ctypes.POINTER(SetteiFields), ctypes.POINTER(SetteiConsts), P, P, P, I, I, Lg, P, P,
                                 P],
            "tg_comp_ng_dev": [ctypes.POINTER(CompFields), ctypes.POINTER(CompConsts), P, I, I, Lg, P, P, P],
            "tg_comp_diag_ng": [ctypes.POINTER(CompFields), ctypes.POINTER(CompConsts), P, P, P, P, I, I],
            "tg_comp_diag_ng_dev": [ctypes.POINTER(CompFields), ctypes.POINTER(CompConsts), P, P, I, I, Lg, P],
            "tg_comp_post_ng": [P] * 8 + [D, D, D, I, I] + [P] * 6,
            "tg_comp_post_ng_dev": [P] * 8 + [D, D, D, I, I, Lg] + [P] * 11,
            "tg_oplus_ng_factor_doubles": [I, Lg],
            "tg_oplus_diag_ng": [ctypes.POINTER(OplusFields), ctypes.POINTER(OplusConsts), P, P, P, P, P, I, I],
            "tg_oplus_diag_ng_dev": [ctypes.POINTER(OplusFields), ctypes.POINTER(OplusConsts), P, P, P, P, P, I, I,
                                     Lg, P],
            "tg_oplus_ng_factor_dev": [ctypes.POINTER(OplusFields), ctypes.POINTER(OplusConsts), P, P, P, I, I, Lg, P,
                                       P],
            "tg_oplus_ng_solve_dev": [ctypes.POINTER(OplusFields), ctypes.POINTER(OplusConsts), P, P, I, I, Lg,
                                      ctypes.POINTER(PostStepArgs), P, P],
            "tg_time_filter_ng": [I, P, P, D, D, I, I, P, P],
            "tg_time_filter_ng_dev": [I, P, P, D, D, I, I, Lg, P, P, P],
            "tg_advec_ng": [P, P, P, P, D, D, D, I, I, I, P],
            "tg_advec_ng_dev": [P, P, P, P, D, D, D, P, I, I, I, Lg, P],
            "tg_smooth_ng": [P, D, I, I, I, P],
            "tg_smooth_ng_dev": [P, D, P, I, I, I, Lg, P],
            "tg_minor_ng_dev": [ctypes.POINTER(MinorFields), ctypes.POINTER(MinorConsts), P, I, I, Lg, P, P, P],
            "tg_dt_ng_dev": [ctypes.POINTER(DtFields), ctypes.POINTER(DtConsts), P, I, I, Lg, P, P, P],
            "tg_trsolv_ng": [P, P, P, P, P, I, I, I],
            "tg_blktri": [P, P, P, P, P, I, I, I, I, I],
            "tg_comp_blksolve_ng": [I, P, P, P, P, P, P, P, I, I],
            "tg_blksolve": [I, P, P, P, P, P, P, P, I, I, I],
            "tg_trsolv_dev": [P, P, P, P, P, I, I, I, I, Lg, I, P, P],
            "tg_blksolve_dev": [I, P, P, P, P, P, P, P, I, I, I, I, Lg, I, P, P],
            "tg_blksolve_dev_noalloc": [I, P, P, P, P, P, P, P, I, I, I, Lg, P, P],
            "tg_plan_create": [ctypes.POINTER(Segment), I, I, ctypes.POINTER(P)],
            "tg_plan_execute": [P, P],
            "tg_plan_capture_graph": [P, P],
            "tg_plan_status": [P, P],
            "tg_plan_launches": [P],
            "tg_plan_describe": [P, ctypes.c_char_p, I],
            "tg_set_cache_hints": [I],
            "tg_set_block_rows": [I, I],
            "tg_set_block_width": [I, I],
            "tg_set_stage_levels": [I, I, I],
            "tg_set_column_residency": [I, I, I],
            "tg_kernel_arch": [ctypes.POINTER(I)],
            "tg_ringfilter": [P, I, I, I, I, I, P, I, D],
            "tg_trsolv_defer": [P, P, P, P, P, I, I, I, I, I, I, I],
            "tg_trsolv_flush": [],
            "tg_dt_ng_post_dev": [ctypes.POINTER(DtFields), ctypes.POINTER(DtConsts), P, I, I, Lg,
                                  ctypes.POINTER(PostStepArgs), P, P],
            "tg_minor_ng_post_dev": [ctypes.POINTER(MinorFields), ctypes.POINTER(MinorConsts), P, I, I, Lg,
                                     ctypes.POINTER(PostStepArgs), P, P],
            "tg_oplus_ng_post_dev": [ctypes.POINTER(OplusFields), ctypes.POINTER(OplusConsts), P, P, P, P, P, I, I,
                                     Lg, ctypes.POINTER(PostStepArgs), P, P],
            "tg_dt_diag_ng": [ctypes.POINTER(DtFields), ctypes.POINTER(DtConsts), P, P, I, I],
            "tg_dt_diag_ng_dev": [ctypes.POINTER(DtFields), ctypes.POINTER(DtConsts), P, P, I, I, Lg, P],
            "tg_minor_diag_ng": [ctypes.POINTER(MinorFields), ctypes.POINTER(MinorConsts), P, P, I, I],
            "tg_minor_diag_ng_dev": [ctypes.POINTER(MinorFields), ctypes.POINTER(MinorConsts), P, P, I, I, Lg, P],
            "tg_filter_o2o": [P, I, I, I, P, I, D],
            "tg_ringfilter_dev": [P, I, I, I, I, I, P, I, D, Lg, P],
            "tg_set_assembly_mode": [I],
            "tg_set_walk_prefetch": [I],
            "tg_set_block_scratch_budget": [D],
            "tg_set_scalar_scratch_budget": [D],
            "tg_set_kind_overlap": [I],
            "tg_set_host_pipeline": [I, I],
            "tg_selftest_wait": [ctypes.c_uint, P, P],
            "tg_plan_sweep_histogram": [P, ctypes.POINTER(Lg), I],
            "tg_plan_destroy": [P],
            "tg_set_refine": [I, D],
            "tg_set_host_precision": [I],
            "tg_set_tile": [I, I, I, I],
            "tg_set_pipeline": [I, I, I, I],
            "tg_set_scratch_global": [I, I, I],
            "tg_set_prefetch": [I, I, I],
            "tg_selftest_division": [P, P, P, Lg, P],
            "tg_selftest_walk": [I, P, I, I, I, I, Lg, P, P],
            "tg_release_buffers": [],
            "tg_version": [],
            "tg_last_error": [],
        }
        for name, args in sig.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = I
        L.tg_version.restype = ctypes.c_char_p
        L.tg_oplus_ng_factor_doubles.restype = Lg
        L.tg_last_error.restype = ctypes.c_char_p
        _lib = L
    return _lib


def version():
    return lib().tg_version().decode()


def _chunks(chunk_array):
    ch = np.ascontiguousarray(chunk_array, dtype=np.int32)
    return ch, ch.ctypes.data, int(ch.size)


def ringfilter(f, order, poly, chunk_array, dlamda):
    """ringfilter (src/ringfilter.F) over every latitude of the global field
    f (nk, nlon+4, nlat), Fortran-ordered float64, filtered in place."""
    if f.ndim != 3:
        raise ValueError("ringfilter: f must be (nk, nlon+4, nlat)")
    nk, nlonp4, nlat = f.shape
    ch, cp, nf = _chunks(chunk_array)
    return _check(lib().tg_ringfilter(_host(f, "f"), nk, nlonp4 - 4, nlat, int(order), int(poly), cp, nf,
                                      float(dlamda)), "tg_ringfilter", numeric_ok=False)


def filter_o2o(fout, chunk_array, dlamda):
    """filter_o2o (src/comp.F:1065-1145): the order-1 ring filter of one species, in place."""
    if fout.ndim != 3:
        raise ValueError("filter_o2o: fout must be (nk, nlon+4, nlat)")
    nk, nlonp4, nlat = fout.shape
    ch, cp, nf = _chunks(chunk_array)
    return _check(lib().tg_filter_o2o(_host(fout, "fout"), nk, nlonp4 - 4, nlat, cp, nf, float(dlamda)),
                  "tg_filter_o2o", numeric_ok=False)


def ringfilter_dev(f, nk, nlon, nlat, order, poly, chunk_array, dlamda, ld, stream=None):
    """Device form on level-major planes (k, i + (nlon+4)*j) at stride ld."""
    ch, cp, nf = _chunks(chunk_array)
    return _check(lib().tg_ringfilter_dev(_dptr(f), nk, nlon, nlat, int(order), int(poly), cp, nf, float(dlamda),
                                          int(ld), _stream(stream)), "tg_ringfilter_dev", numeric_ok=False)


def kernel_arch():
    """SASS target of the library's kernels on the current device (100 for sm_100a)."""
    v = ctypes.c_int(0)
    _check(lib().tg_kernel_arch(ctypes.byref(v)), "tg_kernel_arch", numeric_ok=False)
    return v.value


def _check(rc, where, numeric_ok=True):
    if rc == TG_OK or (numeric_ok and rc in NUMERIC_STATUS):
        return rc
    raise TgError(rc, where)


def _host(a, name):
    if not isinstance(a, np.ndarray) or a.dtype != np.float64 or not (a.flags.f_contiguous or a.ndim <= 1):
        raise TypeError(f"{name}: a Fortran-ordered float64 numpy array is required")
    return a.ctypes.data


def _out(x, name):
    p = _host(x, name)
    if not x.flags.writeable:
        raise TypeError(f"{name}: output array is read-only")
    return p


def _check_sizes(where, fields, names, nk, ncol, two_d=(), one_d=(), outs=()):
    """Every field holds the values the C entry reads: 3-D fields nk*ncol,
    2-D fields ncol, level profiles nk (a short array would be over-read)."""
    for n in names:
        want = nk if n in one_d else ncol if n in two_d else 12 * nk * ncol if n == "fs" else nk * ncol
        if np.size(fields[n]) != want:
            raise ValueError(f"{where}: {n} has {np.size(fields[n])} values, expected {want}")
    for n, x in outs:
        if np.size(x) != nk * ncol:
            raise ValueError(f"{where}: {n} must hold nk*ncol = {nk * ncol} values")


# ---------------------------------------------------------------------------
# Drop-ins (host arrays, synchronous)
# ---------------------------------------------------------------------------
def trsolv(a, b, c, f, x, lev0, lev1, k1, k2, lon0, lon1, lonmax, lat=None, idebug=0):
    """trsolv (src/trsolv.F): one latitude slab (lev0:lev1, lon0:lon1).
    lat and idebug only feed the reference's debug output and are ignored."""
    nlev, nlon = lev1 - lev0 + 1, lon1 - lon0 + 1
    for v, n in ((a, "a"), (b, "b"), (c, "c"), (f, "f"), (x, "x")):
        if v.shape != (nlev, nlon):
            raise ValueError(f"trsolv: {n} must have shape {(nlev, nlon)}")
    rc = lib().tg_trsolv(_host(a, "a"), _host(b, "b"), _host(c, "c"), _host(f, "f"), _out(x, "x"),
                         lev0, lev1, k1, k2, lon0, lon1, lonmax)
    return _check(rc, "tg_trsolv")


_deferred_x = []   # the x arrays of queued slabs, kept alive until the flush


def trsolv_defer(a, b, c, f, x, lev0, lev1, k1, k2, lon0, lon1, lonmax, lat=None, idebug=0):
    """tg_trsolv_defer: queue one latitude slab (arguments as trsolv); a, b,
    c, f are copied now and may be reused; x is written by trsolv_flush()."""
    nlev, nlon = lev1 - lev0 + 1, lon1 - lon0 + 1
    for v, n in ((a, "a"), (b, "b"), (c, "c"), (f, "f"), (x, "x")):
        if v.shape != (nlev, nlon):
            raise ValueError(f"trsolv_defer: {n} must have shape {(nlev, nlon)}")
    rc = lib().tg_trsolv_defer(_host(a, "a"), _host(b, "b"), _host(c, "c"), _host(f, "f"), _out(x, "x"),
                               lev0, lev1, k1, k2, lon0, lon1, lonmax)
    _check(rc, "tg_trsolv_defer", numeric_ok=False)
    _deferred_x.append(x)
    return rc


def trsolv_flush():
    """tg_trsolv_flush: solve every queued slab and write their x."""
    try:
        return _check(lib().tg_trsolv_flush(), "tg_trsolv_flush")
    finally:
        _deferred_x.clear()


def trsolv_ng(a, b, c, f, x, k2, i_ng=None):
    """trsolv_ng (src/trsolv_ng.F90): arrays (nk, lond0:lond1, latd0:latd1)
    (any trailing shape), all ghost-inclusive columns solved, rows 1..k2."""
    nk = a.shape[0]
    ncol = a.size // nk if nk else 0
    for v, n in ((b, "b"), (c, "c"), (f, "f"), (x, "x")):
        if v.shape != a.shape:
            raise ValueError(f"trsolv_ng: {n} must have the shape of a {a.shape}")
    rc = lib().tg_trsolv_ng(_host(a, "a"), _host(b, "b"), _host(c, "c"), _host(f, "f"), _out(x, "x"),
                            nk, k2, ncol)
    return _check(rc, "tg_trsolv_ng")


def blktri(a, b, c, f, beta, gamma, y, x, lev0, lev1, lon0, lon1, nlonp4):
    """blktri (src/duv.F:801): 2x2 blocks (2,2,lev0:lev1,lon0:lon1), vectors
    (2,lev0:lev1,lon0:lon1).  beta, gamma and y are the reference's work
    arrays; they are accepted for signature compatibility and not written."""
    nlev, nlon = lev1 - lev0 + 1, lon1 - lon0 + 1
    for v, n in ((a, "a"), (b, "b"), (c, "c")):
        if v.shape != (2, 2, nlev, nlon):
            raise ValueError(f"blktri: {n} must have shape {(2, 2, nlev, nlon)}")
    for v, n in ((f, "f"), (x, "x")):
        if v.shape != (2, nlev, nlon):
            raise ValueError(f"blktri: {n} must have shape {(2, nlev, nlon)}")
    rc = lib().tg_blktri(_host(a, "a"), _host(b, "b"), _host(c, "c"), _host(f, "f"), _out(x, "x"),
                         lev0, lev1, lon0, lon1, nlonp4)
    return _check(rc, "tg_blktri")


def comp_blksolve_ng(P, Q, R, f, u, ubc_ratio=None, ubc_add=None):
    """The comp_ng block solve (src/comp_ng.F90:166-332): P,Q,R (B,B,nk,ncol),
    f,u (B,nk,ncol); rows 1..nk-1 solved, row nk from the UBC if ubc_ratio
    (B,ncol) is given."""
    B, nk = f.shape[0], f.shape[1]
    ncol = f.size // (B * nk)
    for v, n in ((P, "P"), (Q, "Q"), (R, "R")):
        if v.shape[:3] != (B, B, nk) or v.size != B * B * nk * ncol:
            raise ValueError(f"comp_blksolve_ng: {n} has the wrong shape")
    if u.shape != f.shape:
        raise ValueError("comp_blksolve_ng: u must have the shape of f")
    ur = None if ubc_ratio is None else _host(ubc_ratio, "ubc_ratio")
    ua = None if ubc_add is None else _host(ubc_add, "ubc_add")
    rc = lib().tg_comp_blksolve_ng(B, _host(P, "P"), _host(Q, "Q"), _host(R, "R"), _host(f, "f"), ur, ua,
                                   _out(u, "u"), nk, ncol)
    return _check(rc, "tg_comp_blksolve_ng")


def blksolve(P, Q, R, f, u, k2, ubc_ratio=None, ubc_add=None):
    """General block solve on host arrays: rows 1..k2 of (B,B,nk,ncol) blocks;
    row k2+1 from the UBC if ubc_ratio is given."""
    B, nk = f.shape[0], f.shape[1]
    ncol = f.size // (B * nk)
    for v, n in ((P, "P"), (Q, "Q"), (R, "R")):
        if v.shape[:3] != (B, B, nk) or v.size != B * B * nk * ncol:
            raise ValueError(f"blksolve: {n} has the wrong shape")
    if u.shape != f.shape:
        raise ValueError("blksolve: u must have the shape of f")
    ur = None if ubc_ratio is None else _host(ubc_ratio, "ubc_ratio")
    ua = None if ubc_add is None else _host(ubc_add, "ubc_add")
    rc = lib().tg_blksolve(B, _host(P, "P"), _host(Q, "Q"), _host(R, "R"), _host(f, "f"), ur, ua,
                           _out(u, "u"), nk, k2, ncol)
    return _check(rc, "tg_blksolve")


def solve_host(systems):
    """tg_solve_host: systems is a list of dicts with kind and the host arrays
    a, b, c, f, x (Fortran layout; block kinds P, Q, R in a, b, c), k2, and
    optionally ubc_ratio / ubc_add; all solved in one pipelined call."""
    arr = (HostSystem * max(len(systems), 1))()
    for i, q in enumerate(systems):
        kind = q["kind"]
        f = q["f"]
        nk = f.shape[0] if kind == TG_KIND_SCALAR else f.shape[1]
        B = 1 if kind == TG_KIND_SCALAR else kind
        ncol = f.size // (B * nk)
        arr[i] = HostSystem(kind, nk, q.get("k2", nk), ncol, _host(q["a"], "a"), _host(q["b"], "b"),
                            _host(q["c"], "c"), _host(f, "f"), _out(q["x"], "x"),
                            None if q.get("ubc_ratio") is None else _host(q["ubc_ratio"], "ubc_ratio"),
                            None if q.get("ubc_add") is None else _host(q["ubc_add"], "ubc_add"))
    return _check(lib().tg_solve_host(arr, len(systems)), "tg_solve_host")


def dt_ng(fields, consts, tn_upd):
    """dt_ng's vertical column step (src/dt_ng.F90:57-167) on host arrays:
    fields is a dict of the DT_FIELDS arrays (3-D (nk,ncol...) Fortran-ordered,
    2-D (ncol...), expz/dift (nk)), consts a dict of DT_CONSTS; tn_upd
    (nk, ...) receives the solution."""
    nk = tn_upd.shape[0]
    ncol = tn_upd.size // nk
    _check_sizes("dt_ng", fields, DT_FIELDS, nk, ncol, two_d=("tlbc", "t_lbc", "ulbc", "vlbc"),
                 one_d=("expz", "dift"))
    F = DtFields(*[_host(fields[n], n) for n in DT_FIELDS])
    C = DtConsts(*[float(consts[n]) for n in DT_CONSTS])
    rc = lib().tg_dt_ng(ctypes.byref(F), ctypes.byref(C), _out(tn_upd, "tn_upd"), nk, ncol)
    return _check(rc, "tg_dt_ng")


def minor_ng(fields, consts, fcomp_out):
    """minor_ng's vertical column step (src/minor_ng.F90:60-200) on host
    arrays (fields: MINOR_FIELDS; consts: rmx, alfax, phix(4), b(3,3), fb(3)
    and the MINOR_CONSTS2 constants); fcomp_out (nk, ...) receives the solution."""
    nk = fcomp_out.shape[0]
    ncol = fcomp_out.size // nk
    _check_sizes("minor_ng", fields, MINOR_FIELDS, nk, ncol,
                 two_d=("tlbc", "flbc1", "flbc2", "flbc3", "fubc", "dfactor"), one_d=("expz", "difk"))
    F = MinorFields(*[_host(fields[n], n) for n in MINOR_FIELDS])
    C = minor_consts(consts)
    rc = lib().tg_minor_ng(ctypes.byref(F), ctypes.byref(C), _out(fcomp_out, "fcomp_out"), nk, ncol)
    return _check(rc, "tg_minor_ng")


DT_DIAG_NAMES = ("DTDT", "DT_SOLAR", "DT_HORDIF", "DT_RECOMB", "DT_JOULE", "DT_MOLDIF", "DT_COOL", "DT_HORADV",
                 "DT_VERADV", "DT_ADIA", "DT_CONDUCT", "DEN")
MINOR_DIAG_NAMES = ("DPDT", "PROD", "LOSS", "MOLDIF", "EDDYDIF", "VERADV", "HORADV")


def dt_diag_ng(fields, consts, tn_upd):
    """dt_ng's history diagnostics (src/dt_ng.F90:169-191, DEN :133) from the
    fields and the solution; returns a dict name -> (nk, ncol) array."""
    nk = tn_upd.shape[0]
    ncol = tn_upd.size // nk
    _check_sizes("dt_diag_ng", fields, DT_FIELDS, nk, ncol, two_d=("tlbc", "t_lbc", "ulbc", "vlbc"),
                 one_d=("expz", "dift"), outs=(("tn_upd", tn_upd),))
    F = DtFields(*[_host(fields[n], n) for n in DT_FIELDS])
    C = DtConsts(*[float(consts[n]) for n in DT_CONSTS])
    out = np.zeros((nk, ncol, len(DT_DIAG_NAMES)), order="F")
    _check(lib().tg_dt_diag_ng(ctypes.byref(F), ctypes.byref(C), _host(tn_upd, "tn_upd"), out.ctypes.data, nk, ncol),
           "tg_dt_diag_ng", numeric_ok=False)
    return {n: out[:, :, i] for i, n in enumerate(DT_DIAG_NAMES)}


def minor_diag_ng(fields, consts, fcomp_out):
    """minor_ng's history diagnostics (src/minor_ng.F90:202-224) from the
    fields and the solution; returns a dict name -> (nk, ncol) array."""
    nk = fcomp_out.shape[0]
    ncol = fcomp_out.size // nk
    _check_sizes("minor_diag_ng", fields, MINOR_FIELDS, nk, ncol,
                 two_d=("tlbc", "flbc1", "flbc2", "flbc3", "fubc", "dfactor"), one_d=("expz", "difk"),
                 outs=(("fcomp_out", fcomp_out),))
    F = MinorFields(*[_host(fields[n], n) for n in MINOR_FIELDS])
    C = minor_consts(consts)
    out = np.zeros((nk, ncol, len(MINOR_DIAG_NAMES)), order="F")
    _check(lib().tg_minor_diag_ng(ctypes.byref(F), ctypes.byref(C), _host(fcomp_out, "fcomp_out"), out.ctypes.data,
                                  nk, ncol), "tg_minor_diag_ng", numeric_ok=False)
    return {n: out[:, :, i] for i, n in enumerate(MINOR_DIAG_NAMES)}


def dt_diag_ng_dev(fields, consts, tn_upd, diag, nk, ncol, ld, stream=None):
    """Device form: level-major fields, diag 12 planes of nk*ld."""
    F = DtFields(*[_dptr(fields[n]) for n in DT_FIELDS])
    C = DtConsts(*[float(consts[n]) for n in DT_CONSTS])
    rc = lib().tg_dt_diag_ng_dev(ctypes.byref(F), ctypes.byref(C), _dptr(tn_upd), _dptr(diag), nk, ncol, ld,
                                 _stream(stream))
    return _check(rc, "tg_dt_diag_ng_dev", numeric_ok=False)


def minor_diag_ng_dev(fields, consts, fcomp_out, diag, nk, ncol, ld, stream=None):
    """Device form: level-major fields, diag 7 planes of nk*ld."""
    F = MinorFields(*[_dptr(fields[n]) for n in MINOR_FIELDS])
    C = minor_consts(consts)
    rc = lib().tg_minor_diag_ng_dev(ctypes.byref(F), ctypes.byref(C), _dptr(fcomp_out), _dptr(diag), nk, ncol, ld,
                                    _stream(stream))
    return _check(rc, "tg_minor_diag_ng_dev", numeric_ok=False)


COMP_DIAG_NAMES = ("DO2DT", "DO1DT", "DHEDT", "O2_PROD", "O1_PROD", "HE_PROD", "O2_LOSS", "O1_LOSS", "HE_LOSS",
                   "O2_HORDIF", "O1_HORDIF", "HE_HORDIF", "O2_MOLDIF", "O1_MOLDIF", "HE_MOLDIF", "O2_EDDYDIF",
                   "O1_EDDYDIF", "HE_EDDYDIF", "O2_VERADV", "O1_VERADV", "HE_VERADV", "O2_HORADV", "O1_HORADV",
                   "HE_HORADV")


def comp_diag_ng(fields, consts, o2_upd, o1_upd, he_upd):
    """comp_ng's history diagnostics (src/comp_ng.F90:334-380) from the fields
    and the solution; returns a dict name -> (nk, ncol) array."""
    nk = o2_upd.shape[0]
    ncol = o2_upd.size // nk
    if np.asarray(fields["fs"]).size != 12 * nk * ncol:
        raise ValueError("fs must hold 12 slabs of nk*ncol")
    _check_sizes("comp_diag_ng", fields, COMP_FIELDS, nk, ncol, two_d=("tlbc", "flx_he", "dfactor"),
                 one_d=("expz", "difk"), outs=(("o1_upd", o1_upd), ("he_upd", he_upd)))
    arrs = {n: np.ascontiguousarray(fields[n], dtype=np.float64).reshape(-1) if n == "fs" else fields[n]
            for n in COMP_FIELDS}
    F = CompFields(*[_host(arrs[n], n) for n in COMP_FIELDS])
    C = comp_consts(consts)
    out = np.zeros((nk, ncol, len(COMP_DIAG_NAMES)), order="F")
    _check(lib().tg_comp_diag_ng(ctypes.byref(F), ctypes.byref(C), _host(o2_upd, "o2_upd"), _host(o1_upd, "o1_upd"),
                                 _host(he_upd, "he_upd"), out.ctypes.data, nk, ncol), "tg_comp_diag_ng",
           numeric_ok=False)
    return {n: out[:, :, i] for i, n in enumerate(COMP_DIAG_NAMES)}


def comp_diag_ng_dev(fields, consts, upd, diag, nk, ncol, ld, stream=None):
    """Device form: level-major fields, upd the (3, nk, ld) solution, diag 24 planes of nk*ld."""
    F = CompFields(*[_dptr(fields[n]) for n in COMP_FIELDS])
    C = comp_consts(consts)
    rc = lib().tg_comp_diag_ng_dev(ctypes.byref(F), ctypes.byref(C), _dptr(upd), _dptr(diag), nk, ncol, ld,
                                   _stream(stream))
    return _check(rc, "tg_comp_diag_ng_dev", numeric_ok=False)


def comp_ng(fields, consts, o2_upd, o1_upd, he_upd):
    """comp_ng's column step (src/comp_ng.F90:74-332) on host arrays: fields
    COMP_FIELDS ((nk, ncol) Fortran order, fs (12, ncol, nk) C order = the
    reference's fs(nk, ncol, 3, 0:3)); outputs (nk, ncol) O2, O, He."""
    nk = o2_upd.shape[0]
    ncol = o2_upd.size // nk
    if np.asarray(fields["fs"]).size != 12 * nk * ncol:
        raise ValueError("fs must hold 12 slabs of nk*ncol")
    _check_sizes("comp_ng", fields, COMP_FIELDS, nk, ncol, two_d=("tlbc", "flx_he", "dfactor"),
                 one_d=("expz", "difk"), outs=(("o1_upd", o1_upd), ("he_upd", he_upd)))
    arrs = {n: np.ascontiguousarray(fields[n], dtype=np.float64).reshape(-1) if n == "fs" else fields[n]
            for n in COMP_FIELDS}
    F = CompFields(*[_host(arrs[n], n) for n in COMP_FIELDS])
    C = comp_consts(consts)
    rc = lib().tg_comp_ng(ctypes.byref(F), ctypes.byref(C), _out(o2_upd, "o2_upd"), _out(o1_upd, "o1_upd"),
                          _out(he_upd, "he_upd"), nk, ncol)
    return _check(rc, "tg_comp_ng")


def settei_ng(fields, consts, te_out, ti_out, qtotal):
    """settei_ng's column step (src/settei_ng.F90:60-261) on host arrays:
    fields SETTEI_FIELDS ((nk, ncol) Fortran order, 2-D (ncol)); te_out and
    ti_out receive Te and Ti; qtotal (nk, ncol) is updated in place."""
    nk = te_out.shape[0]
    ncol = te_out.size // nk
    _check_sizes("settei_ng", fields, SETTEI_FIELDS, nk, ncol,
                 two_d=("t_lbc", "chi", "rlatm", "dipmag", "qteaur"), outs=(("ti_out", ti_out), ("qtotal", qtotal)))
    F = SetteiFields(*[_host(fields[n], n) for n in SETTEI_FIELDS])
    C = settei_consts(consts)
    rc = lib().tg_settei_ng(ctypes.byref(F), ctypes.byref(C), _out(te_out, "te_out"), _out(ti_out, "ti_out"),
                            _out(qtotal, "qtotal"), nk, ncol)
    return _check(rc, "tg_settei_ng")


def oplus_ng(fields, consts, opout, xiop2p, xiop2d, Fe=None, Fn=None):
    """oplus_ng's vertical column step (src/oplus_ng.F90:88-307) on host
    arrays: fields OPLUS_FIELDS ((nk, ncol) Fortran order, 2-D (ncol), zpint
    (nk)); outputs (nk, ncol)."""
    nk = opout.shape[0]
    ncol = opout.size // nk
    _check_sizes("oplus_ng", fields, OPLUS_FIELDS, nk, ncol,
                 two_d=("bx", "by", "bz", "dvb", "rlatm", "chi", "dipmag", "sndec", "csdec"), one_d=("zpint",),
                 outs=(("xiop2p", xiop2p), ("xiop2d", xiop2d)))
    F = OplusFields(*[_host(fields[n], n) for n in OPLUS_FIELDS])
    C = oplus_consts(consts)
    rc = lib().tg_oplus_ng(ctypes.byref(F), ctypes.byref(C), _out(opout, "opout"), _out(xiop2p, "xiop2p"),
                           _out(xiop2d, "xiop2d"), None if Fe is None else _out(Fe, "Fe"),
                           None if Fn is None else _out(Fn, "Fn"), nk, ncol)
    return _check(rc, "tg_oplus_ng")


def oplus_ng_dev(fields, consts, opout, xiop2p, xiop2d, nk, ncol, ld, Fe=None, Fn=None, system_out=None,
                 status=None, stream=None):
    F = OplusFields(*[_dptr(fields[n]) for n in OPLUS_FIELDS])
    C = oplus_consts(consts)
    rc = lib().tg_oplus_ng_dev(ctypes.byref(F), ctypes.byref(C), _dptr(opout), _dptr(xiop2p), _dptr(xiop2d),
                               _dptr(Fe), _dptr(Fn), nk, ncol, ld, _dptr(system_out),
                               None if status is None else _int_dptr(status), _stream(stream))
    return _check(rc, "tg_oplus_ng_dev", numeric_ok=False)


def _post(post):
    """post: dict cur, prev, nm_upd (CUDA tensors or device pointers), optional
    bnd_mask (uint8 per column) and bnd, dtsmooth, dtsmooth_div2."""
    m = post.get("bnd_mask")
    if m is not None and not isinstance(m, int):
        if not m.is_cuda or str(m.dtype) != "torch.uint8":
            raise TypeError("bnd_mask must be a uint8 CUDA tensor")
        m = m.data_ptr()
    return PostStepArgs(_dptr(post["cur"]), _dptr(post["prev"]), _dptr(post["nm_upd"]), m, _dptr(post.get("bnd")),
                        float(post["dtsmooth"]), float(post["dtsmooth_div2"]))


def dt_ng_post_dev(fields, consts, tn_upd, nk, ncol, ld, post, status=None, stream=None):
    """dt_ng with the lateral overwrite, time filter and floor fused into its back sweep."""
    F = DtFields(*[_dptr(fields[n]) for n in DT_FIELDS])
    C = DtConsts(*[float(consts[n]) for n in DT_CONSTS])
    Pp = _post(post)
    rc = lib().tg_dt_ng_post_dev(ctypes.byref(F), ctypes.byref(C), _dptr(tn_upd), nk, ncol, ld, ctypes.byref(Pp),
                                 None if status is None else _int_dptr(status), _stream(stream))
    return _check(rc, "tg_dt_ng_post_dev", numeric_ok=False)


def minor_ng_post_dev(fields, consts, fcomp_out, nk, ncol, ld, post, status=None, stream=None):
    """minor_ng with the lateral overwrite, time filter and floors fused into its back sweep."""
    F = MinorFields(*[_dptr(fields[n]) for n in MINOR_FIELDS])
    C = minor_consts(consts)
    Pp = _post(post)
    rc = lib().tg_minor_ng_post_dev(ctypes.byref(F), ctypes.byref(C), _dptr(fcomp_out), nk, ncol, ld,
                                    ctypes.byref(Pp), None if status is None else _int_dptr(status), _stream(stream))
    return _check(rc, "tg_minor_ng_post_dev", numeric_ok=False)


def oplus_ng_post_dev(fields, consts, opout, xiop2p, xiop2d, nk, ncol, ld, post, Fe=None, Fn=None, status=None,
                      stream=None):
    """oplus_ng with the lateral overwrite, time filter and floors fused into its back sweep."""
    F = OplusFields(*[_dptr(fields[n]) for n in OPLUS_FIELDS])
    C = oplus_consts(consts)
    Pp = _post(post)
    rc = lib().tg_oplus_ng_post_dev(ctypes.byref(F), ctypes.byref(C), _dptr(opout), _dptr(xiop2p), _dptr(xiop2d),
                                    _dptr(Fe), _dptr(Fn), nk, ncol, ld, ctypes.byref(Pp),
                                    None if status is None else _int_dptr(status), _stream(stream))
    return _check(rc, "tg_oplus_ng_post_dev", numeric_ok=False)


OPLUS_DIAG_NAMES = ("DOPDT", "OP_PROD", "OP_LOSS", "OP_DIFF", "OP_DRIFT", "OP_WIND")


def oplus_diag_ng(fields, consts, opout, diffexp=None, vdotn_h=None, bdotdh_bvel=None):
    """oplus_ng's history diagnostics (src/oplus_ng.F90:309-330) of the solution
    on host arrays, with the horizontal terms (None: 0); returns a dict name ->
    (nk, ncol) array."""
    nk = opout.shape[0]
    ncol = opout.size // nk
    _check_sizes("oplus_diag_ng", fields, OPLUS_FIELDS, nk, ncol,
                 two_d=("bx", "by", "bz", "dvb", "rlatm", "chi", "dipmag", "sndec", "csdec"), one_d=("zpint",),
                 outs=(("opout", opout),))
    for a, n in ((diffexp, "diffexp"), (vdotn_h, "vdotn_h"), (bdotdh_bvel, "bdotdh_bvel")):
        if a is not None and np.size(a) != nk * ncol:
            raise ValueError(f"oplus_diag_ng: {n} must hold nk*ncol values")
    F = OplusFields(*[_host(fields[n], n) for n in OPLUS_FIELDS])
    C = oplus_consts(consts)
    h = [None if a is None else _host(a, n) for a, n in ((diffexp, "diffexp"), (vdotn_h, "vdotn_h"),
                                                          (bdotdh_bvel, "bdotdh_bvel"))]
    out = np.zeros((nk, ncol, len(OPLUS_DIAG_NAMES)), order="F")
    _check(lib().tg_oplus_diag_ng(ctypes.byref(F), ctypes.byref(C), _host(opout, "opout"), *h, out.ctypes.data, nk,
                                  ncol), "tg_oplus_diag_ng", numeric_ok=False)
    return {n: out[:, :, i] for i, n in enumerate(OPLUS_DIAG_NAMES)}


def oplus_diag_ng_dev(fields, consts, opout, diag, nk, ncol, ld, diffexp=None, vdotn_h=None, bdotdh_bvel=None,
                      stream=None):
    """Device form: level-major fields and solution, diag 6 planes of nk*ld."""
    F = OplusFields(*[_dptr(fields[n]) for n in OPLUS_FIELDS])
    C = oplus_consts(consts)
    rc = lib().tg_oplus_diag_ng_dev(ctypes.byref(F), ctypes.byref(C), _dptr(opout), _dptr(diffexp), _dptr(vdotn_h),
                                    _dptr(bdotdh_bvel), _dptr(diag), nk, ncol, ld, _stream(stream))
    return _check(rc, "tg_oplus_diag_ng_dev", numeric_ok=False)


def oplus_ng_factor_doubles(nk, ld):
    """Doubles of the factor buffer tg_oplus_ng_factor_dev fills."""
    return int(lib().tg_oplus_ng_factor_doubles(int(nk), int(ld)))


def oplus_ng_factor_dev(fields, consts, xiop2p, xiop2d, factor, nk, ncol, ld, status=None, stream=None):
    """The O+ sub-cycle's rows and pivots, once per step, into factor (a float64
    CUDA tensor of oplus_ng_factor_doubles(nk, ld) elements)."""
    F = OplusFields(*[_dptr(fields[n]) for n in OPLUS_FIELDS])
    C = oplus_consts(consts)
    rc = lib().tg_oplus_ng_factor_dev(ctypes.byref(F), ctypes.byref(C), _dptr(xiop2p), _dptr(xiop2d), _dptr(factor),
                                      nk, ncol, ld, None if status is None else _int_dptr(status), _stream(stream))
    return _check(rc, "tg_oplus_ng_factor_dev", numeric_ok=False)


def oplus_ng_solve_dev(fields, consts, factor, opout, nk, ncol, ld, post=None, status=None, stream=None):
    """One O+ sub-step from the factor with fields' current explicit_h and
    optm1_smooth2; post (as for oplus_ng_post_dev) fuses the post-solve steps."""
    F = OplusFields(*[_dptr(fields[n]) for n in OPLUS_FIELDS])
    C = oplus_consts(consts)
    Pp = None if post is None else ctypes.byref(_post(post))
    rc = lib().tg_oplus_ng_solve_dev(ctypes.byref(F), ctypes.byref(C), _dptr(factor), _dptr(opout), nk, ncol, ld,
                                     Pp, None if status is None else _int_dptr(status), _stream(stream))
    return _check(rc, "tg_oplus_ng_solve_dev", numeric_ok=False)


def settei_ng_dev(fields, consts, te_out, ti_out, qtotal, nk, ncol, ld, system_out=None, status=None, stream=None):
    F = SetteiFields(*[_dptr(fields[n]) for n in SETTEI_FIELDS])
    C = settei_consts(consts)
    rc = lib().tg_settei_ng_dev(ctypes.byref(F), ctypes.byref(C), _dptr(te_out), _dptr(ti_out), _dptr(qtotal), nk,
                                ncol, ld, _dptr(system_out), None if status is None else _int_dptr(status),
                                _stream(stream))
    return _check(rc, "tg_settei_ng_dev", numeric_ok=False)


def comp_ng_dev(fields, consts, out, nk, ncol, ld, system_out=None, status=None, stream=None):
    F = CompFields(*[_dptr(fields[n]) for n in COMP_FIELDS])
    C = comp_consts(consts)
    rc = lib().tg_comp_ng_dev(ctypes.byref(F), ctypes.byref(C), _dptr(out), nk, ncol, ld, _dptr(system_out),
                              None if status is None else _int_dptr(status), _stream(stream))
    return _check(rc, "tg_comp_ng_dev", numeric_ok=False)


POST_INPUTS = ("o2", "o1", "he", "o2_nm", "o1_nm", "he_nm", "xnmbar")


def comp_post_ng(fields, consts, upd, nm_out):
    """comp_ng's post-solve steps (src/comp_ng.F90:415-457): upd = [o2, o1, he]
    (nk, ncol) updated in place, nm_out = [o2nm, o1nm, henm] receive the
    filtered fields."""
    nk = upd[0].shape[0]
    ncol = upd[0].size // nk
    ins = [_host(fields[n], n) for n in POST_INPUTS]
    zp = np.ascontiguousarray(fields["zpmid"], dtype=np.float64)
    rc = lib().tg_comp_post_ng(*ins, zp.ctypes.data, float(consts["dz"]), float(consts["dtsmooth"]),
                               float(consts["dtsmooth_div2"]), nk, ncol,
                               *[_out(u, "upd") for u in upd], *[_out(u, "nm_out") for u in nm_out])
    return _check(rc, "tg_comp_post_ng")


def comp_post_ng_dev(fields, zpmid, consts, upd, nm_out, nk, ncol, ld, bnd_mask=None, bnd=None, stream=None):
    """Device form of comp_post_ng on level-major (nk, ld) fields: fields holds
    POST_INPUTS as CUDA tensors, zpmid (nk) on the device, upd = [o2, o1, he]
    (comp_ng's solution, updated in place), nm_out = [o2nm, o1nm, henm].
    bnd_mask (uint8 per column) and bnd = [o2, o1, he] boundary values: the
    lateral-boundary overwrite before the post steps."""
    ins = [_dptr(fields[n]) for n in POST_INPUTS]
    if (bnd_mask is None) != (bnd is None):
        raise ValueError("comp_post_ng_dev: give bnd_mask and bnd together")
    if bnd_mask is not None and (not bnd_mask.is_cuda or str(bnd_mask.dtype) != "torch.uint8"):
        raise TypeError("bnd_mask must be a uint8 CUDA tensor")
    bp = [None] * 3 if bnd is None else [_dptr(b) for b in bnd]
    rc = lib().tg_comp_post_ng_dev(*ins, _dptr(zpmid), float(consts["dz"]), float(consts["dtsmooth"]),
                                   float(consts["dtsmooth_div2"]), nk, ncol, ld, *[_dptr(u) for u in upd],
                                   *[_dptr(u) for u in nm_out], None if bnd_mask is None else bnd_mask.data_ptr(),
                                   *bp, _stream(stream))
    return _check(rc, "tg_comp_post_ng_dev", numeric_ok=False)


def time_filter_ng(which, cur, prev, dtsmooth, dtsmooth_div2, upd, nm_out):
    """Post-solve time filter and floor (which = TG_FILTER_DT: src/dt_ng.F90:208-213,
    TG_FILTER_MINOR: src/minor_ng.F90:234-237, TG_FILTER_OPLUS:
    src/oplus_ng.F90:337-340) on host (nk, ncol) arrays: upd is floored in
    place and nm_out receives the filtered field."""
    for n, x in (("cur", cur), ("prev", prev), ("nm_out", nm_out)):
        if np.shape(x) != np.shape(upd):
            raise ValueError(f"time_filter_ng: {n} must have the shape of upd {upd.shape}")
    nk = upd.shape[0]
    ncol = upd.size // nk
    rc = lib().tg_time_filter_ng(int(which), _host(cur, "cur"), _host(prev, "prev"), float(dtsmooth),
                                 float(dtsmooth_div2), nk, ncol, _out(upd, "upd"), _out(nm_out, "nm_out"))
    return _check(rc, "tg_time_filter_ng", numeric_ok=False)


def time_filter_ng_dev(which, cur, prev, dtsmooth, dtsmooth_div2, upd, nm_out, nk, ncol, ld, stream=None):
    """Device form of time_filter_ng on level-major (nk, ld) fields."""
    rc = lib().tg_time_filter_ng_dev(int(which), _dptr(cur), _dptr(prev), float(dtsmooth), float(dtsmooth_div2), nk,
                                     ncol, ld, _dptr(upd), _dptr(nm_out), _stream(stream))
    return _check(rc, "tg_time_filter_ng_dev", numeric_ok=False)


def advec_ng(f, un, vn, racs, dlamda, dphi, re_inv, hadvec):
    """advec_ng (src/advec_ng.F90) for a nest held as one subdomain: f, un, vn
    and hadvec are (nk, nlon+4, nlat+4) Fortran arrays, racs (nlat+4)."""
    if np.ndim(f) != 3:
        raise ValueError("advec_ng: f must be (nk, nlon+4, nlat+4)")
    for n, x in (("un", un), ("vn", vn), ("hadvec", hadvec)):
        if np.shape(x) != f.shape:
            raise ValueError(f"advec_ng: {n} must have the shape of f {f.shape}")
    nk, nlond, nlatd = f.shape
    r = np.ascontiguousarray(racs, dtype=np.float64)
    if r.shape != (nlatd,):
        raise ValueError(f"advec_ng: racs must have {nlatd} values")
    rc = lib().tg_advec_ng(_host(f, "f"), _host(un, "un"), _host(vn, "vn"), r.ctypes.data, float(dlamda),
                           float(dphi), float(re_inv), nk, nlond - 4, nlatd - 4, _out(hadvec, "hadvec"))
    return _check(rc, "tg_advec_ng", numeric_ok=False)


def smooth_ng(fin, shapiro, fout):
    """smooth_ng (src/smooth_ng.F90) for a nest held as one subdomain; fin and
    fout are (nk, nlon+4, nlat+4) Fortran arrays."""
    if np.ndim(fin) != 3 or np.shape(fout) != np.shape(fin):
        raise ValueError("smooth_ng: fin and fout must both be (nk, nlon+4, nlat+4)")
    nk, nlond, nlatd = fin.shape
    rc = lib().tg_smooth_ng(_host(fin, "fin"), float(shapiro), nk, nlond - 4, nlatd - 4, _out(fout, "fout"))
    return _check(rc, "tg_smooth_ng", numeric_ok=False)


def advec_ng_dev(f, un, vn, racs, dlamda, dphi, re_inv, hadvec, nk, nlon, nlat, ld, stream=None):
    """Device form of advec_ng on level-major planes (k*ld + i + (nlon+4)*j)."""
    rc = lib().tg_advec_ng_dev(_dptr(f), _dptr(un), _dptr(vn), _dptr(racs), float(dlamda), float(dphi),
                               float(re_inv), _dptr(hadvec), nk, nlon, nlat, ld, _stream(stream))
    return _check(rc, "tg_advec_ng_dev", numeric_ok=False)


def smooth_ng_dev(fin, shapiro, fout, nk, nlon, nlat, ld, stream=None):
    """Device form of smooth_ng on level-major planes (k*ld + i + (nlon+4)*j)."""
    rc = lib().tg_smooth_ng_dev(_dptr(fin), float(shapiro), _dptr(fout), nk, nlon, nlat, ld, _stream(stream))
    return _check(rc, "tg_smooth_ng_dev", numeric_ok=False)


def minor_ng_dev(fields, consts, out, nk, ncol, ld, system_out=None, status=None, stream=None):
    F = MinorFields(*[_dptr(fields[n]) for n in MINOR_FIELDS])
    C = minor_consts(consts)
    rc = lib().tg_minor_ng_dev(ctypes.byref(F), ctypes.byref(C), _dptr(out), nk, ncol, ld, _dptr(system_out),
                               None if status is None else _int_dptr(status), _stream(stream))
    return _check(rc, "tg_minor_ng_dev", numeric_ok=False)


def dt_ng_dev(fields, consts, tn_upd, nk, ncol, ld, system_out=None, status=None, stream=None):
    """Device form of dt_ng: fields are device pointers / CUDA tensors in the
    level-major layout (3-D (nk, ld)); system_out (4*nk*ld) receives p,q,r,rhs."""
    F = DtFields(*[_dptr(fields[n]) for n in DT_FIELDS])
    C = DtConsts(*[float(consts[n]) for n in DT_CONSTS])
    rc = lib().tg_dt_ng_dev(ctypes.byref(F), ctypes.byref(C), _dptr(tn_upd), nk, ncol, ld, _dptr(system_out),
                            None if status is None else _int_dptr(status), _stream(stream))
    return _check(rc, "tg_dt_ng_dev", numeric_ok=False)


# ---------------------------------------------------------------------------
# Device entry points
# ---------------------------------------------------------------------------
def _dptr(t):
    if t is None:
        return None
    if isinstance(t, int):
        return t
    if hasattr(t, "data_ptr"):
        if not t.is_cuda or str(t.dtype) != "torch.float64":
            raise TypeError("a float64 CUDA tensor is required")
        return t.data_ptr()
    raise TypeError("device pointer (int) or torch CUDA tensor expected")


def _stream(stream):
    if stream is None:
        return None
    if isinstance(stream, int):
        return stream
    return stream.cuda_stream


def trsolv_dev(a, b, c, f, x, nk, k2, ncol, layout=TG_LAYOUT_LEVEL, ld=None, precision=TG_PREC_F64,
               status=None, stream=None):
    ld = ncol if ld is None else ld
    rc = lib().tg_trsolv_dev(_dptr(a), _dptr(b), _dptr(c), _dptr(f), _dptr(x), nk, k2, ncol, layout, ld,
                             precision, None if status is None else _int_dptr(status), _stream(stream))
    return _check(rc, "tg_trsolv_dev", numeric_ok=False)


def blksolve_dev(B, P, Q, R, f, u, nk, k2, ncol, ubc_ratio=None, ubc_add=None, layout=TG_LAYOUT_LEVEL,
                 ld=None, precision=TG_PREC_F64, status=None, stream=None):
    ld = ncol if ld is None else ld
    rc = lib().tg_blksolve_dev(B, _dptr(P), _dptr(Q), _dptr(R), _dptr(f), _dptr(ubc_ratio), _dptr(ubc_add),
                               _dptr(u), nk, k2, ncol, layout, ld, precision,
                               None if status is None else _int_dptr(status), _stream(stream))
    return _check(rc, "tg_blksolve_dev", numeric_ok=False)


def blksolve_dev_noalloc(B, P, Q, R, f, u, nk, k2, ncol, ubc_ratio=None, ubc_add=None, ld=None, status=None,
                         stream=None):
    """tg_blksolve_dev_noalloc: the FP64 level-major block solve with its
    scratch in a fixed array of the library (no device allocation)."""
    ld = ncol if ld is None else ld
    rc = lib().tg_blksolve_dev_noalloc(B, _dptr(P), _dptr(Q), _dptr(R), _dptr(f), _dptr(ubc_ratio),
                                       _dptr(ubc_add), _dptr(u), nk, k2, ncol, ld,
                                       None if status is None else _int_dptr(status), _stream(stream))
    return _check(rc, "tg_blksolve_dev_noalloc", numeric_ok=False)


def _int_dptr(t):
    if isinstance(t, int):
        return t
    if not t.is_cuda or str(t.dtype) != "torch.int32":
        raise TypeError("status must be an int32 CUDA tensor")
    return t.data_ptr()


def set_refine(max_sweeps=3, rel_tol=1e-11):
    return _check(lib().tg_set_refine(max_sweeps, rel_tol), "tg_set_refine", numeric_ok=False)


def set_host_precision(precision=TG_PREC_F64):
    """Precision used by the host-array drop-ins (default FP64)."""
    return _check(lib().tg_set_host_precision(precision), "tg_set_host_precision", numeric_ok=False)


def set_tile(kind, precision, cols_per_block=0, cols_per_thread=0):
    return _check(lib().tg_set_tile(kind, precision, cols_per_block, cols_per_thread), "tg_set_tile",
                  numeric_ok=False)


def set_pipeline(kind, precision, stages=-1, warps=0):
    """Ring depth of the bulk-copy staged FP64 kernels (0: register prefetch,
    -1: default) and their warps per CTA (0: default)."""
    return _check(lib().tg_set_pipeline(kind, precision, stages, warps), "tg_set_pipeline", numeric_ok=False)


def set_prefetch(kind, precision, levels=-1):
    """Register prefetch depth (levels) of the scalar kernels: 4, 8, 16; -1 default."""
    return _check(lib().tg_set_prefetch(kind, precision, levels), "tg_set_prefetch", numeric_ok=False)


def set_scratch_global(kind, precision, on=-1):
    """Scalar FP64 register kernel: w2 in global scratch (1) or shared memory (0)."""
    return _check(lib().tg_set_scratch_global(kind, precision, on), "tg_set_scratch_global", numeric_ok=False)


def selftest_division(a, b, q, stream=None):
    """q = a/b on the device through the kernels' division routine."""
    return _check(lib().tg_selftest_division(_dptr(a), _dptr(b), _dptr(q), int(q.numel()), _stream(stream)),
                  "tg_selftest_division", numeric_ok=False)


def selftest_walk(which, buf, nk, K, top, ncol, ld, status, stream=None):
    """One column walk of the assembly routines on caller-formed level-major
    rows (which 0: the Thomas walk over planes p, q, r, f, x of buf; which 1:
    oplus_ng's factor pass over a factor buffer); the walk's status goes to
    the device int `status`."""
    need = (5 if which == 0 else 1) * nk * ld
    if which == 1:
        need = oplus_ng_factor_doubles(nk, ld)
    if buf.numel() < need:
        raise ValueError(f"selftest_walk: buf holds {buf.numel()} doubles, expected {need}")
    return _check(lib().tg_selftest_walk(int(which), _dptr(buf), int(nk), int(K), int(top), int(ncol), int(ld),
                                         _int_dptr(status), _stream(stream)), "tg_selftest_walk", numeric_ok=False)


def set_cache_hints(on):
    """L2 eviction-priority hints of the ring kernels (1 on, 0 off, -1 default)."""
    return _check(lib().tg_set_cache_hints(int(on)), "tg_set_cache_hints")


def set_block_rows(kind, on):
    """FP64 block ring kernel with one lane per block row (1 on, 0 off, -1 default)."""
    return _check(lib().tg_set_block_rows(int(kind), int(on)), "tg_set_block_rows")


def set_block_width(kind, width):
    """Columns per warp of the FP64 block ring kernel (32, 16 or 8; other values: default)."""
    return _check(lib().tg_set_block_width(int(kind), int(width)), "tg_set_block_width")


def set_stage_levels(kind, precision, levels):
    """Levels per ring stage of the scalar FP64 ring with w2 in global scratch (1, 2, 4, 8)."""
    return _check(lib().tg_set_stage_levels(int(kind), int(precision), int(levels)), "tg_set_stage_levels")


def set_column_residency(kind, precision, mode):
    """FP64 ring kernels: scalar 0 w2 in L2 scratch, 1 w2 in shared memory, 2 w2 and w3 in shared memory;
    block kinds 0 Gamma in L2 scratch, 1 Gamma in shared memory; -1 default."""
    return _check(lib().tg_set_column_residency(int(kind), int(precision), int(mode)), "tg_set_column_residency")


def set_assembly_mode(mode):
    """Assembly kernels: 2 three passes where built (default), 1 two passes, 0 one fused column walk, -1 default."""
    return _check(lib().tg_set_assembly_mode(int(mode)), "tg_set_assembly_mode")


def set_walk_prefetch(levels):
    """Levels the assembly walks read ahead: 1..32, or -1 automatic (8 up to 16384 columns, else 1)."""
    return _check(lib().tg_set_walk_prefetch(int(levels)), "tg_set_walk_prefetch")


def set_scalar_scratch_budget(megabytes):
    """L2 budget (MB) of the scalar ring kernels' w2 scratch and parked results (<= 0: default)."""
    return _check(lib().tg_set_scalar_scratch_budget(float(megabytes)), "tg_set_scalar_scratch_budget")


def set_kind_overlap(mode):
    """Kinds of a plan: 1 side by side, 0 one after the other, -1 side by side when each fits in one wave."""
    return _check(lib().tg_set_kind_overlap(int(mode)), "tg_set_kind_overlap")


def set_host_pipeline(chunk_kb=0, streams=0):
    """Host-array entries: input KiB per pipelined column chunk and streams (<= 0: defaults)."""
    return _check(lib().tg_set_host_pipeline(int(chunk_kb), int(streams)), "tg_set_host_pipeline")


def set_block_scratch_budget(megabytes):
    """Budget (MB) of the block kernels' Gamma scratch (<= 0: default 160)."""
    return _check(lib().tg_set_block_scratch_budget(float(megabytes)), "tg_set_block_scratch_budget")


def selftest_wait(polls, status, stream=None):
    """Bounded mbarrier wait on a barrier nothing completes; status (int32 CUDA
    tensor) receives TG_ETIMEOUT."""
    return _check(lib().tg_selftest_wait(int(polls), _int_dptr(status), _stream(stream)), "tg_selftest_wait",
                  numeric_ok=False)


def release_buffers():
    return lib().tg_release_buffers()


class Plan:
    """A batched, GPU-resident solve of many segments (tg_plan_*).

    segments: list of dicts with keys kind, nk, k2, ncol, ld, a, b, c, f, x
    and optionally ubc_ratio, ubc_add (device pointers or torch tensors, in
    the level-major plan layout of include/tg_colsolve.h).  The tensors are
    referenced, not copied; keep them alive while the plan is used."""

    def __init__(self, segments, precision=TG_PREC_F64):
        arr = (Segment * max(len(segments), 1))()
        self._keep = []
        for i, s in enumerate(segments):
            arr[i] = Segment(s["kind"], s["nk"], s["k2"], s["ncol"], s.get("ld", s["ncol"]),
                             _dptr(s["a"]), _dptr(s["b"]), _dptr(s["c"]), _dptr(s["f"]), _dptr(s["x"]),
                             _dptr(s.get("ubc_ratio")), _dptr(s.get("ubc_add")))
            self._keep.append(s)
        self.nseg = len(segments)
        self.precision = precision
        h = ctypes.c_void_p()
        rc = lib().tg_plan_create(arr, len(segments), precision, ctypes.byref(h))
        _check(rc, "tg_plan_create", numeric_ok=False)
        self._h = h

    def execute(self, stream=None):
        _check(lib().tg_plan_execute(self._h, _stream(stream)), "tg_plan_execute", numeric_ok=False)

    def capture_graph(self, stream):
        _check(lib().tg_plan_capture_graph(self._h, _stream(stream)), "tg_plan_capture_graph", numeric_ok=False)

    @property
    def launches(self):
        return lib().tg_plan_launches(self._h)

    def describe(self):
        """Kernel and launch shape of each group, e.g. 'k_scalar_f64_ring<4,1> kind=0 ...'."""
        buf = ctypes.create_string_buffer(1024)
        _check(lib().tg_plan_describe(self._h, buf, len(buf)), "tg_plan_describe", numeric_ok=False)
        return buf.value.decode()

    def status(self):
        per = (ctypes.c_int * max(self.nseg, 1))()
        rc = lib().tg_plan_status(self._h, per)
        _check(rc, "tg_plan_status")
        return rc, list(per)[: self.nseg]

    def sweep_histogram(self, nbins=8):
        h = (ctypes.c_long * nbins)()
        n = lib().tg_plan_sweep_histogram(self._h, h, nbins)
        if n < 0:
            raise TgError(-n, "tg_plan_sweep_histogram")
        return list(h)[:n]

    def close(self):
        if getattr(self, "_h", None):
            lib().tg_plan_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
