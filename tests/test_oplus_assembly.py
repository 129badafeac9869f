"""The oplus_ng vertical column step of the oracle (src/oplus_ng.F90:88-307),
checked bit for bit against an independent numpy transcription of the
Fortran array statements (transcendental functions through Python's math
module, the C library's)."""
import math

import numpy as np
import pytest

from conftest import prec_fn

COS, SIN, LOG10, POW = (prec_fn(math.cos, np.cos), prec_fn(math.sin, np.sin), prec_fn(math.log10, np.log10),
                        prec_fn(math.pow, np.power))


def interp_up(a):
    """x(k) = .5*(a(k)+a(k+1)), x(nk) = 1.5*a(nk)-.5*a(nk-1)"""
    out = np.empty_like(a)
    out[:-1] = .5 * (a[:-1] + a[1:])
    out[-1] = 1.5 * a[-1] - .5 * a[-2]
    return out


def oplus_numpy(F, C, parts=None):
    """The system rows, rates and fluxes; parts (a dict) receives the raw
    diffusion / drift / wind coefficients, op_loss and op_prod."""
    pi = 4.0 * math.atan(1.0)
    rtd = 180. / pi
    phid, phin, ppolar = 2.0e8, -2.0e8, 0.
    nk, ncol = F["tn"].shape
    g = lambda k: F[k]
    tn, te, ti, o2, o1, n2, he, n2d, ne = (g(k) for k in ("tn", "te", "ti", "o2", "o1", "n2", "he", "n2d", "ne"))
    xnmbar, op, bx, by, bz = g("xnmbar"), g("op"), g("bx"), g("by"), g("bz")
    arl, chi = np.abs(g("rlatm")), g("chi")
    a = np.full(ncol, np.nan, dtype=F["tn"].dtype)
    a = np.where(arl >= pi / 4.5, 1., a)
    a = np.where((arl < pi / 4.5) & (arl > pi / 18), .5 * (1. + COS(arl * 6. - pi * 4. / 3.)), a)
    a = np.where(arl <= pi / 18, 0., a)
    fed, fen = phid * a, phin * a
    opflux = np.where(chi >= 0.5 * pi, fen, fed)
    opflux = np.where((chi * rtd - 80.) * (chi * rtd - 100.) < 0.,
                      .5 * (fed + fen) + .5 * (fed - fen) * COS(pi * (chi * rtd - 80.) / 20.), opflux)
    opflux = np.where(arl >= pi / 3., opflux + ppolar, opflux)
    tr = 0.5 * (tn + ti)
    wni, wii = interp_up(g("w")), interp_up(g("wi"))
    qop2pi, qop2di, qopi = interp_up(g("qop2p")), interp_up(g("qop2d")), interp_up(g("qop"))
    lg = 1. - 0.064 * LOG10(tr)
    vni = (18.1 * o2 * C["rmassinv_o2"] + o1 * C["rmassinv_o1"] * np.sqrt(tr) * (lg * lg) * C["colfac"] +
           3.6 * he * C["rmassinv_he"] + 18.6 * n2 * C["rmassinv_n2"])
    dj = 1.42E17 / (xnmbar * vni)
    vni = 16 * 3.53E-11 * vni
    if not abs(C["opdiffcap"] - 0.) < 1e-9:
        cap = C["opdiffcap"] / (1 + POW(2., g("zpint") - 6))[:, None]
        dj = np.where(dj < cap, dj, cap)
    tp = te + ti
    hj = g("scht")
    bdotu = bx * g("u") + by * g("v") + hj * bz * wni
    tp_op = tp * op
    d = np.empty_like(tn)
    d[1:nk - 1] = (tp_op[2:] - tp_op[:nk - 2]) / 2.
    d[nk - 2] = tp_op[nk - 2] - tp_op[nk - 3]
    d[nk - 1] = tp_op[nk - 1] - tp_op[nk - 2]
    d[0] = tp_op[1] - tp_op[0]
    diffj = 1. / (hj * C["dlev"]) * d + C["rmass_op"] * C["grav"] / C["gask"] * op
    wd = vni * diffj * dj
    sncsdip = SIN(g("dipmag")) * COS(g("dipmag"))
    Fe = wd * sncsdip * g("sndec")
    Fn = wd * sncsdip * g("csdec")
    dvb = g("dvb") / bz
    dz = C["dz"]
    hdz = 1. / (hj * dz)
    tp1 = 0.5 * (ti + te)
    hdzi = np.empty_like(tn)
    hdzi[1:nk - 1] = 0.5 * (hdz[:nk - 2] + hdz[1:nk - 1])
    hdzi[0] = 1.5 * hdz[0] - 0.5 * hdz[1]
    hdzi[nk - 1] = 1.5 * hdz[nk - 2] - 0.5 * hdz[nk - 3]
    gmr = C["grav"] * C["rmass_op"] / (2. * C["gask"])
    tph1 = 2. * tp1 * hdzi + gmr
    tph0 = np.empty_like(tn)
    tph0[1:] = 2. * tp1[:nk - 1] * hdzi[1:] - gmr
    tph1[nk - 1] = 2. * (2. * tp1[nk - 2] - tp1[nk - 3]) * hdzi[nk - 1] + gmr
    tph0[0] = 2. * (2. * tp1[0] - tp1[1]) * hdzi[0] - gmr
    djint = np.empty_like(tn)
    djint[1:nk - 1] = 0.5 * (dj[:nk - 2] + dj[1:nk - 1])
    djint[0] = 1.5 * dj[0] - 0.5 * dj[1]
    djint[nk - 1] = 1.5 * dj[nk - 2] - 0.5 * dj[nk - 3]
    divbz = dvb + g("bdotdh_djbz") / (dj * (bz * bz))
    hdzmbz = (hdz - 0.5 * divbz) * (bz * bz)
    hdzpbz = (hdz + 0.5 * divbz) * (bz * bz)
    explicit = g("explicit_h") - g("optm1_smooth2") * C["dtx2inv"] * C["nstep_sub"]
    diffp = hdzmbz * djint * tph0
    diffq, diffr = np.empty_like(tn), np.empty_like(tn)
    diffq[:nk - 1] = -(hdzpbz[:nk - 1] * djint[1:] * tph0[1:] + hdzmbz[:nk - 1] * djint[:nk - 1] * tph1[:nk - 1])
    diffr[:nk - 1] = hdzpbz[:nk - 1] * djint[1:] * tph1[1:]
    driftp = wii * 0.5 * hdz
    driftq = -wii * 6. / C["re"]
    driftr = -wii * 0.5 * hdz
    windp, windq, windr = (np.zeros_like(tn) for _ in range(3))
    windp[1:nk - 1] = bz * bdotu[:nk - 2] * 0.5 * hdz[1:nk - 1]
    windq[:nk - 2] = -bdotu[:nk - 2] * dvb * bz
    windr[:nk - 2] = -bz * bdotu[1:nk - 1] * 0.5 * hdz[:nk - 2]
    windp[0] = bz * (2. * bdotu[0] - bdotu[1]) * 0.5 * hdz[0]
    windq[nk - 2] = -bdotu[nk - 2] * dvb * bz
    windr[nk - 2] = bz * (2. * bdotu[nk - 2] - bdotu[nk - 3]) * 0.5 * hdz[nk - 2]
    if parts is not None:
        parts.update(diffp=diffp, diffq=diffq, diffr=diffr, driftp=driftp, driftq=driftq, driftr=driftr,
                     windp=windp, windq=windq, windr=windr)
    p = diffp + driftp + windp
    q = diffq + driftq + windq - C["dtx2inv"] * C["nstep_sub"]
    r = diffr + driftr + windr
    ubcb = -(bz * bz) * djint[nk - 1] * tph0[nk - 1]
    ubca = -(bz * bz) * djint[nk - 1] * tph1[nk - 1]
    q[nk - 2] = q[nk - 2] + ubcb / ubca * r[nk - 2]
    explicit[nk - 2] = explicit[nk - 2] - opflux * r[nk - 2] / ubca
    r[nk - 2] = 0.
    rk19, rk20, rk25 = g("rk19"), g("rk20"), g("rk25")
    xiop2p = qop2pi / (xnmbar * ((C["rk16"] + C["rk17"]) * n2 * C["rmassinv_n2"] + C["rk18"] * o1 * C["rmassinv_o1"]) +
                       (rk19 + rk20) * ne + C["rk21"] + C["rk22"])
    xiop2d = (qop2di + (rk20 * ne + C["rk22"]) * xiop2p) / \
        (xnmbar * (C["rk23"] * n2 * C["rmassinv_n2"] + C["rk24"] * o1 * C["rmassinv_o1"] +
                   C["rk26"] * o2 * C["rmassinv_o2"]) + rk25 * ne + C["rk27"])
    op_loss = xnmbar * (g("rk1") * o2 * C["rmassinv_o2"] + g("rk2") * n2 * C["rmassinv_n2"] +
                        C["rk10"] * n2d * C["rmassinv_n2d"])
    q = q - op_loss
    op_prod = (qopi + (rk19 * ne + C["rk21"]) * xiop2p + (rk25 * ne + C["rk27"]) * xiop2d +
               (C["rk18"] * xiop2p + C["rk24"] * xiop2d) * o1 * C["rmassinv_o1"] * xnmbar)
    explicit = explicit - op_prod
    if parts is not None:
        parts.update(op_loss=op_loss, op_prod=op_prod)
    q[0] = q[0] - p[0]
    explicit[0] = explicit[0] - 2. * p[0] * g("qop")[0] / (1.5 * op_loss[0] - 0.5 * op_loss[1])
    p[0] = 0.
    return p, q, r, explicit, xiop2p, xiop2d, Fe, Fn


@pytest.mark.parametrize("nk,dz,cap", [(29, 0.5, 0.0), (57, 0.25, 1e7), (57, 0.25, 0.0), (3, 0.5, 1e5)])
def test_oplus_matches_independent_transcription(pkg, orc, nk, dz, cap):
    F, C = pkg.synth.oplus_inputs(nk, 61, dz, 13 + nk, opdiffcap=cap)
    (op, x2p, x2d, fe, fn), (p, q, r, ex) = orc.oplus_ng(F, C, with_system=True)
    pn, qn, rn, exn, x2pn, x2dn, fen, fnn = oplus_numpy(F, C)
    for got, want in ((p, pn), (q, qn), (r, rn), (ex, exn)):
        assert np.array_equal(got[:nk - 1], want[:nk - 1])
    for got, want in ((x2p, x2pn), (x2d, x2dn), (fe, fen), (fn, fnn)):
        assert np.array_equal(got, want)
    x = orc.trsolv_ng(pn, qn, rn, exn, nk - 1)
    assert np.array_equal(op[:nk - 1], x[:nk - 1])
    assert np.array_equal(op[nk - 1], x[nk - 2] * x[nk - 2] / x[nk - 3])


def oplus_diag_numpy(F, C, x, h3):
    """The addfld diagnostics of oplus_ng.F90:309-330 as its array statements
    write them, on levels 2..nk-1 for the three sums."""
    parts = {}
    oplus_numpy(F, C, parts)
    nk = x.shape[0]
    out = {"DOPDT": (x - F["optm1_smooth2"]) * C["dtx2inv"] * C["nstep_sub"], "OP_PROD": parts["op_prod"],
           "OP_LOSS": -(parts["op_loss"] * x)}
    for name, pre, hz in (("OP_DIFF", "diff", h3[0]), ("OP_DRIFT", "drift", -h3[1]), ("OP_WIND", "wind", -h3[2])):
        s = np.zeros_like(x)
        k = slice(1, nk - 1)
        s[k] = (hz[k] + parts[pre + "p"][k] * x[:nk - 2] + parts[pre + "q"][k] * x[1:nk - 1] +
                parts[pre + "r"][k] * x[2:])
        out[name] = s
    return out


@pytest.mark.parametrize("nk,dz,cap", [(29, 0.5, 0.0), (57, 0.25, 1e7), (3, 0.5, 1e5)])
def test_oplus_diagnostics_match_independent_transcription(pkg, orc, nk, dz, cap):
    F, C = pkg.synth.oplus_inputs(nk, 61, dz, 23 + nk, opdiffcap=cap)
    op = orc.oplus_ng(F, C)[0]
    rng = np.random.default_rng(nk)
    h3 = [np.asfortranarray(rng.uniform(-1e-3, 1e-3, op.shape)) for _ in range(3)]
    got = orc.oplus_diag_ng(F, C, op, *h3)
    want = oplus_diag_numpy(F, C, op, h3)
    assert sorted(got) == sorted(orc.OPLUS_DIAG_NAMES)
    for name in orc.OPLUS_DIAG_NAMES:
        assert np.array_equal(got[name], want[name]), name
    # without the horizontal terms the sums hold the vertical parts alone
    zero = orc.oplus_diag_ng(F, C, op)
    want0 = oplus_diag_numpy(F, C, op, [np.zeros_like(op)] * 3)
    for name in orc.OPLUS_DIAG_NAMES:
        assert np.array_equal(zero[name], want0[name]), name
