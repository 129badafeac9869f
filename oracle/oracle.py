"""ctypes binding of the CPU oracle (oracle/liboracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline legs of bench.py, always as the checker or the timed baseline,
never by the product library.  Parity of the oracle with the reference is
unpinned (no Fortran compiler here, no reference tests); it is pinned against
LAPACK, manufactured solutions and a long-double restatement instead.

Arrays are numpy float64 in the reference's column-major layouts:
  scalar (nk, ncol), block matrices (B, B, nk, ncol), block vectors (B, nk, ncol),
stored Fortran-ordered (``order='F'``), i.e. the level index fastest.
"""
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")
_lib = None


def build(force=False):
    """Compile oracle/liboracle.so with its Makefile (gcc, -ffp-contract=off)."""
    src = os.path.join(_HERE, "tg_oracle.c")
    if force or not os.path.exists(_LIB_PATH) or os.path.getmtime(_LIB_PATH) < os.path.getmtime(src):
        subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(_LIB_PATH)
        P = ctypes.c_void_p
        i, l = ctypes.c_int, ctypes.c_long
        L.oracle_trsolv_ng.argtypes = [P, P, P, P, P, i, i, l, i]
        L.oracle_trsolv_ng_ld.argtypes = [P, P, P, P, P, i, i, l]
        L.oracle_trsolv.argtypes = [P, P, P, P, P, i, i, i, i, i, i, i]
        L.oracle_matinv3.argtypes = [P, P]
        L.oracle_matinv2.argtypes = [P, P]
        L.oracle_blksolve.argtypes = [i, P, P, P, P, P, i, i, l, P, P, i]
        L.oracle_blksolve_ld.argtypes = [i, P, P, P, P, P, i, i, l, P, P]
        L.oracle_blktri.argtypes = [P, P, P, P, P, i, i, i, i, i]
        L.oracle_max_threads.restype = i
        for fn in (L.oracle_trsolv_ng, L.oracle_trsolv_ng_ld, L.oracle_trsolv, L.oracle_matinv3,
                   L.oracle_matinv2, L.oracle_blksolve, L.oracle_blksolve_ld, L.oracle_blktri):
            fn.restype = None
        _lib = L
    return _lib


def _p(a):
    if a is None:
        return None
    assert a.dtype == np.float64 and (a.flags.f_contiguous or a.ndim == 1), "float64 Fortran-ordered array expected"
    return a.ctypes.data


def _fcopy(a):
    return np.asfortranarray(np.asarray(a, dtype=np.float64))


def max_threads():
    return lib().oracle_max_threads()


def trsolv_ng(a, b, c, f, k2, x=None, nthreads=1, long_double=False):
    """trsolv_ng (src/trsolv_ng.F90) over (nk, ncol) arrays; returns x.

    Rows k2+1..nk of x keep the values of the ``x`` passed in (NaN if none)."""
    a, b, c, f = (_fcopy(v) for v in (a, b, c, f))
    nk = a.shape[0]
    ncol = a.size // nk
    if x is None:
        x = np.full(a.shape, np.nan, order="F")
    else:
        x = _fcopy(x).copy(order="F")
    if long_double:
        lib().oracle_trsolv_ng_ld(_p(a), _p(b), _p(c), _p(f), _p(x), nk, k2, ncol)
    else:
        lib().oracle_trsolv_ng(_p(a), _p(b), _p(c), _p(f), _p(x), nk, k2, ncol, nthreads)
    return x


def trsolv(a, b, c, f, x, lev0, lev1, k1, k2, lon0, lon1, lonmax):
    """trsolv (src/trsolv.F) on one (lev0:lev1, lon0:lon1) slab; returns x."""
    a, b, c, f = (_fcopy(v) for v in (a, b, c, f))
    x = _fcopy(x).copy(order="F")
    lib().oracle_trsolv(_p(a), _p(b), _p(c), _p(f), _p(x), lev0, lev1, k1, k2, lon0, lon1, lonmax)
    return x


def matinv3(A):
    A = _fcopy(A)
    B = np.empty((3, 3), order="F")
    lib().oracle_matinv3(_p(A), _p(B))
    return B


def matinv2(A):
    A = _fcopy(A)
    B = np.empty((2, 2), order="F")
    lib().oracle_matinv2(_p(A), _p(B))
    return B


def blksolve(P, Q, R, f, k2, ubc_ratio=None, ubc_add=None, u=None, nthreads=1, long_double=False):
    """Block-tridiagonal solve (comp_ng.F90:166-332 / duv.F blktri) over
    (B,B,nk,ncol) blocks and (B,nk,ncol) vectors; returns u."""
    P, Q, R, f = (_fcopy(v) for v in (P, Q, R, f))
    B, nk = f.shape[0], f.shape[1]
    ncol = f.size // (B * nk)
    u = np.full(f.shape, np.nan, order="F") if u is None else _fcopy(u).copy(order="F")
    ur = None if ubc_ratio is None else _fcopy(ubc_ratio)
    ua = None if ubc_add is None else _fcopy(ubc_add)
    if long_double:
        lib().oracle_blksolve_ld(B, _p(P), _p(Q), _p(R), _p(f), _p(u), nk, k2, ncol, _p(ur), _p(ua))
    else:
        lib().oracle_blksolve(B, _p(P), _p(Q), _p(R), _p(f), _p(u), nk, k2, ncol, _p(ur), _p(ua), nthreads)
    return u


def blktri(a, b, c, f, x, lev0, lev1, lon0, lon1, nlonp4):
    """blktri (src/duv.F:801-908) on one slab; returns x."""
    a, b, c, f = (_fcopy(v) for v in (a, b, c, f))
    x = _fcopy(x).copy(order="F")
    lib().oracle_blktri(_p(a), _p(b), _p(c), _p(f), _p(x), lev0, lev1, lon0, lon1, nlonp4)
    return x


# ---- dt_ng column assembly ----------------------------------------------------
DT_FIELD_ORDER = ("tn", "tnsmooth", "horadv", "un", "vn", "o1", "mbar", "xnmbar", "scht", "schti", "cp", "kt",
                  "km", "hdt", "qji_tn", "cool_imp", "cool_exp", "w", "qtotal", "rkm12",
                  "tlbc", "t_lbc", "ulbc", "vlbc", "expz", "dift")
DT_CONST_ORDER = ("dz", "dtx2inv", "expzmid_inv", "grav", "p0", "avo", "gask", "tsurplus", "rmassinv_o1")


class DtFields(ctypes.Structure):
    _fields_ = [(n, ctypes.c_void_p) for n in DT_FIELD_ORDER]


class DtConsts(ctypes.Structure):
    _fields_ = [(n, ctypes.c_double) for n in DT_CONST_ORDER]


def dt_ng(fields, consts, with_system=False):
    """dt_ng assembly + solve (src/dt_ng.F90:57-167); returns tn_upd and, if
    with_system, (p, q, r, rhs) rows 1..nk-1."""
    L = lib()
    if not hasattr(L, "_dt_bound"):
        L.oracle_dt_ng.argtypes = [ctypes.POINTER(DtFields), ctypes.POINTER(DtConsts), ctypes.c_int,
                                   ctypes.c_long, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                   ctypes.c_void_p, ctypes.c_void_p]
        L.oracle_dt_ng.restype = None
        L._dt_bound = True
    arrs = {k: _fcopy(fields[k]) for k in DT_FIELD_ORDER}
    nk, ncol = arrs["tn"].shape[0], arrs["tn"].size // arrs["tn"].shape[0]
    F = DtFields(*[arrs[k].ctypes.data for k in DT_FIELD_ORDER])
    C = DtConsts(*[float(consts[k]) for k in DT_CONST_ORDER])
    tn_upd = np.zeros((nk, ncol), order="F")
    sysarr = [np.zeros((nk, ncol), order="F") for _ in range(4)] if with_system else [None] * 4
    L.oracle_dt_ng(ctypes.byref(F), ctypes.byref(C), nk, ncol, *[_p(s) for s in sysarr], _p(tn_upd))
    return (tn_upd, tuple(sysarr)) if with_system else tn_upd


DT_DIAG_NAMES = ("DTDT", "DT_SOLAR", "DT_HORDIF", "DT_RECOMB", "DT_JOULE", "DT_MOLDIF", "DT_COOL", "DT_HORADV",
                 "DT_VERADV", "DT_ADIA", "DT_CONDUCT", "DEN")


def dt_diag_ng(fields, consts, tn_upd):
    """dt_ng's history diagnostics (src/dt_ng.F90:169-191, DEN :133) from the
    fields and the solution tn_upd (nk, ncol); returns a dict name -> (nk, ncol)."""
    L = lib()
    if not hasattr(L, "_dt_diag_bound"):
        L.oracle_dt_diag_ng.argtypes = [ctypes.POINTER(DtFields), ctypes.POINTER(DtConsts), ctypes.c_int,
                                        ctypes.c_long, ctypes.c_void_p, ctypes.c_void_p]
        L.oracle_dt_diag_ng.restype = None
        L._dt_diag_bound = True
    arrs = {k: _fcopy(fields[k]) for k in DT_FIELD_ORDER}
    nk, ncol = arrs["tn"].shape[0], arrs["tn"].size // arrs["tn"].shape[0]
    F = DtFields(*[arrs[k].ctypes.data for k in DT_FIELD_ORDER])
    C = DtConsts(*[float(consts[k]) for k in DT_CONST_ORDER])
    x = _fcopy(tn_upd)
    out = np.zeros((nk, ncol, len(DT_DIAG_NAMES)), order="F")
    L.oracle_dt_diag_ng(ctypes.byref(F), ctypes.byref(C), nk, ncol, _p(x), _p(out))
    return {n: out[:, :, i] for i, n in enumerate(DT_DIAG_NAMES)}


MINOR_FIELD_ORDER = ("tn", "o2", "o1", "he", "mbar", "barm", "xnmbar", "w", "ftm1_smooth", "hadvec", "sloss",
                     "sprod", "tlbc", "flbc1", "flbc2", "flbc3", "fubc", "dfactor", "expz", "difk")
MINOR_CONST_ORDER = ("dzp", "dtx2inv", "expzmid", "expzmid_inv", "rmassinv_o2", "rmassinv_o1", "rmassinv_n2",
                     "rmassinv_he", "rmass_o2", "rmass_o1", "rmass_he", "rmass_n2", "p0", "grav", "avo")


class MinorFields(ctypes.Structure):
    _fields_ = [(n, ctypes.c_void_p) for n in MINOR_FIELD_ORDER]


class MinorConsts(ctypes.Structure):
    _fields_ = ([("rmx", ctypes.c_double), ("alfax", ctypes.c_double), ("phix", ctypes.c_double * 4)] +
                [(n, ctypes.c_double) for n in MINOR_CONST_ORDER] +
                [("b", ctypes.c_double * 9), ("fb", ctypes.c_double * 3)])


def _minor_consts(consts):
    return MinorConsts(consts["rmx"], consts["alfax"], (ctypes.c_double * 4)(*consts["phix"]),
                       *[float(consts[k]) for k in MINOR_CONST_ORDER],
                       (ctypes.c_double * 9)(*np.ravel(consts["b"], order="F")), (ctypes.c_double * 3)(*consts["fb"]))


MINOR_DIAG_NAMES = ("DPDT", "PROD", "LOSS", "MOLDIF", "EDDYDIF", "VERADV", "HORADV")


def minor_diag_ng(fields, consts, fcomp_out):
    """minor_ng's history diagnostics (src/minor_ng.F90:202-224) from the
    fields and the solution; returns a dict name -> (nk, ncol) holding the
    values passed to addfld (VERADV and HORADV with the reference's sign)."""
    L = lib()
    if not hasattr(L, "_minor_diag_bound"):
        L.oracle_minor_diag_ng.argtypes = [ctypes.POINTER(MinorFields), ctypes.POINTER(MinorConsts), ctypes.c_int,
                                           ctypes.c_long, ctypes.c_void_p, ctypes.c_void_p]
        L.oracle_minor_diag_ng.restype = None
        L._minor_diag_bound = True
    arrs = {k: _fcopy(fields[k]) for k in MINOR_FIELD_ORDER}
    nk, ncol = arrs["tn"].shape[0], arrs["tn"].size // arrs["tn"].shape[0]
    F = MinorFields(*[arrs[k].ctypes.data for k in MINOR_FIELD_ORDER])
    C = _minor_consts(consts)
    x = _fcopy(fcomp_out)
    out = np.zeros((nk, ncol, len(MINOR_DIAG_NAMES)), order="F")
    L.oracle_minor_diag_ng(ctypes.byref(F), ctypes.byref(C), nk, ncol, _p(x), _p(out))
    return {n: out[:, :, i] for i, n in enumerate(MINOR_DIAG_NAMES)}


def minor_ng(fields, consts, with_system=False):
    """minor_ng assembly + solve (src/minor_ng.F90:60-200); returns fcomp_out
    (before the max(.,small) clamp) and, if with_system, (p, q, r, f) rows 1..nk."""
    L = lib()
    if not hasattr(L, "_minor_bound"):
        L.oracle_minor_ng.argtypes = [ctypes.POINTER(MinorFields), ctypes.POINTER(MinorConsts), ctypes.c_int,
                                      ctypes.c_long] + [ctypes.c_void_p] * 5
        L.oracle_minor_ng.restype = None
        L._minor_bound = True
    arrs = {k: _fcopy(fields[k]) for k in MINOR_FIELD_ORDER}
    nk, ncol = arrs["tn"].shape[0], arrs["tn"].size // arrs["tn"].shape[0]
    F = MinorFields(*[arrs[k].ctypes.data for k in MINOR_FIELD_ORDER])
    C = _minor_consts(consts)
    out = np.zeros((nk, ncol), order="F")
    sysarr = [np.zeros((nk, ncol), order="F") for _ in range(4)] if with_system else [None] * 4
    L.oracle_minor_ng(ctypes.byref(F), ctypes.byref(C), nk, ncol, *[_p(s) for s in sysarr], _p(out))
    return (out, tuple(sysarr)) if with_system else out


COMP_FIELD_ORDER = ("tn", "o2", "o1", "he", "w", "mbar", "o2nm_smooth", "o1nm_smooth", "henm_smooth",
                    "o2_advec", "o1_advec", "he_advec", "hdo2", "hdo1", "hdhe", "fs",
                    "tlbc", "flx_he", "dfactor", "expz", "difk")
COMP_CONST_ORDER = ("dz", "dtx2inv", "expzmid", "expzmid_inv", "rmassinv_o2", "rmassinv_o1", "rmassinv_he",
                    "rmassinv_n2", "rmass_o2", "rmass_o1", "rmass_he", "p0", "grav")


class CompFields(ctypes.Structure):
    _fields_ = [(n, ctypes.c_void_p) for n in COMP_FIELD_ORDER]


class CompConsts(ctypes.Structure):
    _fields_ = ([(n, ctypes.c_double) for n in COMP_CONST_ORDER] +
                [("b", ctypes.c_double * 9), ("fb", ctypes.c_double * 3), ("pshelb", ctypes.c_double),
                 ("calc_helium", ctypes.c_int)])


def comp_consts(c, cls=CompConsts):
    return cls(*[float(c[k]) for k in COMP_CONST_ORDER], (ctypes.c_double * 9)(*np.ravel(c["b"], order="F")),
               (ctypes.c_double * 3)(*c["fb"]), float(c["pshelb"]), int(c["calc_helium"]))


def _bind_comp(L):
    if not hasattr(L, "_comp_bound"):
        L.oracle_comp_ng.argtypes = [ctypes.POINTER(CompFields), ctypes.POINTER(CompConsts), ctypes.c_int,
                                     ctypes.c_long] + [ctypes.c_void_p] * 8
        L.oracle_comp_ng.restype = None
        L.oracle_comp_post_ng.argtypes = [ctypes.c_void_p] * 8 + [ctypes.c_double] * 3 + \
            [ctypes.c_int, ctypes.c_long] + [ctypes.c_void_p] * 6
        L.oracle_comp_post_ng.restype = None
        L.oracle_comp_diag_ng.argtypes = [ctypes.POINTER(CompFields), ctypes.POINTER(CompConsts), ctypes.c_int,
                                          ctypes.c_long] + [ctypes.c_void_p] * 4
        L.oracle_comp_diag_ng.restype = None
        L._comp_bound = True
    return L


def comp_ng(fields, consts, with_system=False):
    """comp_ng column step (src/comp_ng.F90:74-332); returns (o2, o1, he)
    upd arrays (nk, ncol) and, if with_system, (P, Q, R, f, ubc) with P,Q,R
    (3,3,nk,ncol), f (3,nk,ncol) rows 1..nk-1 and ubc (6,ncol)."""
    L = _bind_comp(lib())
    arrs = {k: (np.ascontiguousarray(fields[k]) if k == "fs" else _fcopy(fields[k])) for k in COMP_FIELD_ORDER}
    nk, ncol = arrs["tn"].shape[0], arrs["tn"].size // arrs["tn"].shape[0]
    assert arrs["fs"].size == 12 * nk * ncol
    F = CompFields(*[arrs[k].ctypes.data for k in COMP_FIELD_ORDER])
    C = comp_consts(consts)
    upd = [np.zeros((nk, ncol), order="F") for _ in range(3)]
    if with_system:
        sysarr = [np.zeros((3, 3, nk, ncol), order="F") for _ in range(3)] + \
                 [np.zeros((3, nk, ncol), order="F"), np.zeros((6, ncol), order="F")]
    else:
        sysarr = [None] * 5
    L.oracle_comp_ng(ctypes.byref(F), ctypes.byref(C), nk, ncol, *[_p(u) for u in upd], *[_p(s) for s in sysarr])
    return (tuple(upd), tuple(sysarr)) if with_system else tuple(upd)


COMP_DIAG_NAMES = ("DO2DT", "DO1DT", "DHEDT", "O2_PROD", "O1_PROD", "HE_PROD", "O2_LOSS", "O1_LOSS", "HE_LOSS",
                   "O2_HORDIF", "O1_HORDIF", "HE_HORDIF", "O2_MOLDIF", "O1_MOLDIF", "HE_MOLDIF", "O2_EDDYDIF",
                   "O1_EDDYDIF", "HE_EDDYDIF", "O2_VERADV", "O1_VERADV", "HE_VERADV", "O2_HORADV", "O1_HORADV",
                   "HE_HORADV")


def comp_diag_ng(fields, consts, upd):
    """comp_ng's history diagnostics (src/comp_ng.F90:334-380) of the solution
    upd = (o2, o1, he) (nk, ncol): a dict of (nk, ncol) arrays by the names of
    the addfld calls (VERADV and HORADV negated as they are handed over;
    MOLDIF, EDDYDIF, VERADV 0 on the first and top levels)."""
    L = _bind_comp(lib())
    arrs = {k: (np.ascontiguousarray(fields[k]) if k == "fs" else _fcopy(fields[k])) for k in COMP_FIELD_ORDER}
    nk, ncol = arrs["tn"].shape[0], arrs["tn"].size // arrs["tn"].shape[0]
    F = CompFields(*[arrs[k].ctypes.data for k in COMP_FIELD_ORDER])
    C = comp_consts(consts)
    x = [_fcopy(u) for u in upd]
    out = np.zeros((nk, ncol, len(COMP_DIAG_NAMES)), order="F")
    L.oracle_comp_diag_ng(ctypes.byref(F), ctypes.byref(C), nk, ncol, *[_p(u) for u in x], _p(out))
    return {n: out[:, :, i] for i, n in enumerate(COMP_DIAG_NAMES)}


POST_INPUTS = ("o2", "o1", "he", "o2_nm", "o1_nm", "he_nm", "xnmbar")


def comp_post_ng(fields, consts):
    """comp_ng post-solve steps (src/comp_ng.F90:415-457); returns
    (o2_upd, o1_upd, he_upd, o2nm_upd, o1nm_upd, henm_upd)."""
    L = _bind_comp(lib())
    a = {k: _fcopy(fields[k]) for k in POST_INPUTS}
    nk, ncol = a["o2"].shape[0], a["o2"].size // a["o2"].shape[0]
    upd = [_fcopy(fields[k]).copy(order="F") for k in ("o2_upd", "o1_upd", "he_upd")]
    nm = [np.zeros((nk, ncol), order="F") for _ in range(3)]
    zp = np.ascontiguousarray(fields["zpmid"], dtype=np.float64)
    L.oracle_comp_post_ng(*[_p(a[k]) for k in POST_INPUTS], zp.ctypes.data, float(consts["dz"]),
                          float(consts["dtsmooth"]), float(consts["dtsmooth_div2"]), nk, ncol,
                          *[_p(u) for u in upd], *[_p(u) for u in nm])
    return tuple(upd) + tuple(nm)


FILTER_DT, FILTER_MINOR, FILTER_OPLUS = 0, 1, 2


def time_filter_ng(which, cur, prev, upd, dtsmooth, dtsmooth_div2):
    """Post-solve time filter and floor of dt_ng (src/dt_ng.F90:208-213),
    minor_ng (src/minor_ng.F90:234-237) or oplus_ng (src/oplus_ng.F90:337-340);
    returns (upd floored, nm) as new (nk, ncol) arrays."""
    L = lib()
    if not hasattr(L, "_filter_bound"):
        L.oracle_time_filter_ng.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_double,
                                            ctypes.c_double, ctypes.c_long, ctypes.c_void_p, ctypes.c_void_p]
        L.oracle_time_filter_ng.restype = None
        L._filter_bound = True
    c, p = _fcopy(cur), _fcopy(prev)
    u = _fcopy(upd).copy(order="F")
    nm = np.zeros_like(u, order="F")
    L.oracle_time_filter_ng(int(which), _p(c), _p(p), float(dtsmooth), float(dtsmooth_div2), u.size, _p(u), _p(nm))
    return u, nm


SETTEI_FIELD_ORDER = ("tn", "o2", "o1", "he", "n2", "ne", "te", "ti", "op", "o2p", "nplus", "n2p", "nop", "xnmbar",
                      "xnmbari", "scht", "schti", "qji_ti", "qop2p", "qop2d", "qo2p", "qop", "qn2p", "qnp", "qnop",
                      "Q1", "Q2", "t_lbc", "chi", "rlatm", "dipmag", "qteaur")
SETTEI_CONST_ORDER = ("f107", "dipmin", "dz", "evergs", "avo", "rmass_o1", "rmassinv_o2", "rmassinv_o1",
                      "rmassinv_he", "rmassinv_n2", "rmassinv_n4s", "rmassinv_no")


class SetteiFields(ctypes.Structure):
    _fields_ = [(n, ctypes.c_void_p) for n in SETTEI_FIELD_ORDER]


class SetteiConsts(ctypes.Structure):
    _fields_ = ([(n, ctypes.c_double) for n in SETTEI_CONST_ORDER] +
                [("b", ctypes.c_double * 9), ("fb", ctypes.c_double * 3), ("et", ctypes.c_int),
                 ("electron_heating", ctypes.c_int)])


def settei_consts(c, cls=SetteiConsts):
    return cls(*[float(c[k]) for k in SETTEI_CONST_ORDER], (ctypes.c_double * 9)(*np.ravel(c["b"], order="F")),
               (ctypes.c_double * 3)(*c["fb"]), int(c["et"]), int(c["electron_heating"]))


def settei_ng(fields, consts, qtotal, with_system=False):
    """settei_ng column step (src/settei_ng.F90:60-261); returns (te_out,
    ti_out, qtotal_out) and, if with_system, (p, q, r, rhs) rows 1..nk-1."""
    L = lib()
    if not hasattr(L, "_settei_bound"):
        L.oracle_settei_ng.argtypes = [ctypes.POINTER(SetteiFields), ctypes.POINTER(SetteiConsts), ctypes.c_int,
                                       ctypes.c_long] + [ctypes.c_void_p] * 7
        L.oracle_settei_ng.restype = None
        L._settei_bound = True
    arrs = {k: _fcopy(fields[k]) for k in SETTEI_FIELD_ORDER}
    nk, ncol = arrs["tn"].shape[0], arrs["tn"].size // arrs["tn"].shape[0]
    F = SetteiFields(*[arrs[k].ctypes.data for k in SETTEI_FIELD_ORDER])
    C = settei_consts(consts)
    te_out, ti_out = np.zeros((nk, ncol), order="F"), np.zeros((nk, ncol), order="F")
    qt = _fcopy(qtotal).copy(order="F")
    sysarr = [np.zeros((nk, ncol), order="F") for _ in range(4)] if with_system else [None] * 4
    L.oracle_settei_ng(ctypes.byref(F), ctypes.byref(C), nk, ncol, _p(te_out), _p(ti_out), _p(qt),
                       *[_p(s) for s in sysarr])
    return ((te_out, ti_out, qt), tuple(sysarr)) if with_system else (te_out, ti_out, qt)


OPLUS_FIELD_ORDER = ("tn", "te", "ti", "o2", "o1", "n2", "he", "n2d", "ne", "u", "v", "w", "wi", "xnmbar", "scht",
                     "qop2p", "qop2d", "qop", "rk1", "rk2", "rk19", "rk20", "rk25", "op", "optm1_smooth2",
                     "explicit_h", "bdotdh_djbz", "bx", "by", "bz", "dvb", "rlatm", "chi", "dipmag", "sndec", "csdec",
                     "zpint")
OPLUS_CONST_ORDER = ("rmass_op", "gask", "grav", "re", "rmassinv_o2", "rmassinv_o1", "rmassinv_n2", "rmassinv_n2d",
                     "rmassinv_he", "rk10", "rk16", "rk17", "rk18", "rk21", "rk22", "rk23", "rk24", "rk26", "rk27",
                     "colfac", "opdiffcap", "dtx2inv", "dz", "dlev")


class OplusFields(ctypes.Structure):
    _fields_ = [(n, ctypes.c_void_p) for n in OPLUS_FIELD_ORDER]


class OplusConsts(ctypes.Structure):
    _fields_ = [(n, ctypes.c_double) for n in OPLUS_CONST_ORDER] + [("nstep_sub", ctypes.c_int)]


def oplus_consts(c, cls=OplusConsts):
    return cls(*[float(c[k]) for k in OPLUS_CONST_ORDER], int(c["nstep_sub"]))


def oplus_ng(fields, consts, with_system=False):
    """oplus_ng vertical column step (src/oplus_ng.F90:125-307); returns
    (opout, xiop2p, xiop2d, Fe, Fn) and, if with_system, (p, q, r, explicit)."""
    L = lib()
    if not hasattr(L, "_oplus_bound"):
        L.oracle_oplus_ng.argtypes = [ctypes.POINTER(OplusFields), ctypes.POINTER(OplusConsts), ctypes.c_int,
                                      ctypes.c_long] + [ctypes.c_void_p] * 9
        L.oracle_oplus_ng.restype = None
        L._oplus_bound = True
    arrs = {k: _fcopy(fields[k]) for k in OPLUS_FIELD_ORDER}
    nk, ncol = arrs["tn"].shape[0], arrs["tn"].size // arrs["tn"].shape[0]
    F = OplusFields(*[arrs[k].ctypes.data for k in OPLUS_FIELD_ORDER])
    C = oplus_consts(consts)
    outs = [np.zeros((nk, ncol), order="F") for _ in range(5)]
    sysarr = [np.zeros((nk, ncol), order="F") for _ in range(4)] if with_system else [None] * 4
    L.oracle_oplus_ng(ctypes.byref(F), ctypes.byref(C), nk, ncol, *[_p(a) for a in outs], *[_p(s) for s in sysarr])
    return (tuple(outs), tuple(sysarr)) if with_system else tuple(outs)


OPLUS_DIAG_NAMES = ("DOPDT", "OP_PROD", "OP_LOSS", "OP_DIFF", "OP_DRIFT", "OP_WIND")


def oplus_diag_ng(fields, consts, opout, diffexp=None, vdotn_h=None, bdotdh_bvel=None):
    """oplus_ng's history diagnostics (src/oplus_ng.F90:309-330) of the
    solution opout (nk, ncol), with the horizontal terms (None: 0); a dict of
    (nk, ncol) arrays by the names of the addfld calls."""
    L = lib()
    if not hasattr(L, "_oplus_diag_bound"):
        L.oracle_oplus_diag_ng.argtypes = [ctypes.POINTER(OplusFields), ctypes.POINTER(OplusConsts), ctypes.c_int,
                                           ctypes.c_long] + [ctypes.c_void_p] * 5
        L.oracle_oplus_diag_ng.restype = None
        L._oplus_diag_bound = True
    arrs = {k: _fcopy(fields[k]) for k in OPLUS_FIELD_ORDER}
    nk, ncol = arrs["tn"].shape[0], arrs["tn"].size // arrs["tn"].shape[0]
    F = OplusFields(*[arrs[k].ctypes.data for k in OPLUS_FIELD_ORDER])
    C = oplus_consts(consts)
    x = _fcopy(opout)
    h = [None if a is None else _fcopy(a) for a in (diffexp, vdotn_h, bdotdh_bvel)]
    out = np.zeros((nk, ncol, len(OPLUS_DIAG_NAMES)), order="F")
    L.oracle_oplus_diag_ng(ctypes.byref(F), ctypes.byref(C), nk, ncol, _p(x), *[_p(a) for a in h], _p(out))
    return {n: out[:, :, i] for i, n in enumerate(OPLUS_DIAG_NAMES)}


def _bind_horiz(L):
    if not hasattr(L, "_horiz_bound"):
        P, D, I = ctypes.c_void_p, ctypes.c_double, ctypes.c_int
        L.oracle_advec_ng.argtypes = [P, P, P, P, D, D, D, I, I, I, P]
        L.oracle_advec_ng.restype = None
        L.oracle_smooth_ng.argtypes = [P, D, I, I, I, P]
        L.oracle_smooth_ng.restype = None
        L._horiz_bound = True
    return L


def advec_ng(f, un, vn, racs, dlamda, dphi, re_inv):
    """advec_ng (src/advec_ng.F90:1-52) on one nest held as a single
    subdomain; f, un, vn (nk, nlon+4, nlat+4), racs (nlat+4).  Returns hadvec."""
    L = _bind_horiz(lib())
    a = [_fcopy(x) for x in (f, un, vn)]
    r = np.ascontiguousarray(racs, dtype=np.float64)
    nk, nlond, nlatd = a[0].shape
    out = np.zeros_like(a[0], order="F")
    L.oracle_advec_ng(*[_p(x) for x in a], r.ctypes.data, float(dlamda), float(dphi), float(re_inv), nk,
                      nlond - 4, nlatd - 4, _p(out))
    return out


def smooth_ng(fin, shapiro):
    """smooth_ng (src/smooth_ng.F90:1-42) on one nest held as a single
    subdomain; fin (nk, nlon+4, nlat+4).  Returns fout."""
    L = _bind_horiz(lib())
    a = _fcopy(fin)
    nk, nlond, nlatd = a.shape
    out = np.zeros_like(a, order="F")
    L.oracle_smooth_ng(_p(a), float(shapiro), nk, nlond - 4, nlatd - 4, _p(out))
    return out


def ringfilter(f, order, poly, chunk_array, dlamda):
    """ringfilter (src/ringfilter.F:1-111) over every latitude of a global
    field f (nk, nlon+4, nlat); returns the filtered copy."""
    L = lib()
    if not hasattr(L, "_ring_bound"):
        P, D, I = ctypes.c_void_p, ctypes.c_double, ctypes.c_int
        L.oracle_ringfilter.argtypes = [P, I, I, I, I, I, P, I, D]
        L.oracle_ringfilter.restype = I
        L._ring_bound = True
    out = np.array(f, dtype=np.float64, order="F", copy=True)
    nk, nlonp4, nlat = out.shape
    ch = np.ascontiguousarray(chunk_array, dtype=np.int32)
    rc = L.oracle_ringfilter(_p(out), nk, nlonp4 - 4, nlat, int(order), int(poly), ch.ctypes.data, ch.size,
                             float(dlamda))
    if rc:
        raise ValueError("ringfilter: order >= nlon")
    return out
