"""The settei_ng column step of the oracle (src/settei_ng.F90:60-261),
checked bit for bit against an independent numpy transcription of the
Fortran array statements.  Transcendental functions go through Python's math
module (the C library's, as the oracle uses)."""
import math

import numpy as np
import pytest

from conftest import prec_fn

EXP, LOG, SQRT, COS, SIN = (prec_fn(math.exp, np.exp), prec_fn(math.log, np.log), np.sqrt,
                            prec_fn(math.cos, np.cos), prec_fn(math.sin, np.sin))
POW = prec_fn(math.pow, np.power)


def settei_numpy(F, C, qtotal):
    pi = 4.0 * math.atan(1.0)
    rtd = 180.0 / pi
    ev, dz, b, fb = C["evergs"], C["dz"], C["b"], C["fb"]
    fpolar, dl, alam, ad, sd = -3.0e+9, 1.e-6, 0.0069, 0.0091, 2.3e-11
    tn, o2, o1, he, n2, ne, te, ti = (F[k] for k in ("tn", "o2", "o1", "he", "n2", "ne", "te", "ti"))
    xnmbar, xnmbari, h_mid, h_int = F["xnmbar"], F["xnmbari"], F["scht"], F["schti"]
    nk, ncol = tn.shape
    f107te = min(C["f107"], 235.)
    arl, chi = np.abs(F["rlatm"]), F["chi"]
    a = np.full(ncol, np.nan, dtype=F["tn"].dtype)
    a = np.where(arl >= pi / 4.5, 1., a)
    a = np.where((arl < pi / 4.5) & (arl > pi / 18), .5 * (1. + COS(arl * 6. - pi * 4. / 3.)), a)
    a = np.where(arl <= pi / 18, 0., a)
    fed = -9.0e+7 * f107te * a
    fen = fed / 2.
    fed = fed + F["qteaur"]
    fen = fen + F["qteaur"]
    fe = np.where(chi >= .5 * pi, fen, fed)
    fe = np.where((chi * rtd - 80.) * (chi * rtd - 100.) >= 0., fe * ev,
                  (.5 * (fed + fen) + .5 * (fed - fen) * COS(pi * (chi * rtd - 80.) / 20.)) * ev)
    fe = np.where(arl >= pi / 3., fe + fpolar * ev, fe)
    te_int, o2n, o1n, hen, n2n, tn_int = (np.empty_like(tn) for _ in range(6))
    for dst, src in ((te_int, te), (o2n, o2), (o1n, o1), (hen, he), (n2n, n2), (tn_int, tn)):
        dst[1:nk - 1] = .5 * (src[1:nk - 1] + src[0:nk - 2])
    te_int[0] = np.maximum(1.5 * te[0] - .5 * te[1], F["t_lbc"])
    o2n[0] = .5 * (fb[0] + (b[0, 0] + 1.) * o2[0] + b[0, 1] * o1[0] + b[0, 2] * he[0])
    o1n[0] = .5 * (fb[0] + b[0, 0] * o2[0] + (b[0, 1] + 1.) * o1[0] + b[0, 2] * he[0])
    hen[0] = .5 * (fb[0] + b[0, 0] * o2[0] + b[0, 1] * o1[0] + (b[0, 2] + 1.) * he[0])
    n2n[0] = np.maximum(1. - o2n[0] - o1n[0] - hen[0], 0.)
    tn_int[0] = F["t_lbc"]
    te_int[nk - 1] = 1.5 * te[nk - 2] - .5 * te[nk - 3]
    for dst, src in ((o2n, o2), (o1n, o1), (hen, he), (n2n, n2)):
        dst[nk - 1] = .5 * (src[nk - 1] + src[nk - 2])
    tn_int[nk - 1] = 1.5 * tn[nk - 2] - .5 * tn[nk - 3]
    n2n = np.maximum(n2n, 0.)
    o2n = xnmbari * o2n * C["rmassinv_o2"]
    o1n = xnmbari * o1n * C["rmassinv_o1"]
    hen = xnmbari * hen * C["rmassinv_he"]
    n2n = xnmbari * n2n * C["rmassinv_n2"]
    root_te = SQRT(te_int)
    tek0 = 7.5e5 / (1. + 3.22e4 * (te_int * te_int) / ne *
                    ((2.20e-16 + 7.92e-18 * root_te) * o2n + 1.10e-16 * (1. + 5.7e-4 * te_int) * o1n +
                     5.60e-16 * hen + (2.82e-17 - 3.41e-21 * te_int) * root_te * n2n)) * ev
    s = SIN(np.maximum(np.abs(F["dipmag"]), C["dipmin"]))
    sindipmag = np.maximum(s * s, .10)
    p = 2. / 7. / (h_mid * (dz * dz))
    p = p * sindipmag
    th = tek0 / h_int
    th1 = np.empty_like(th)
    th1[:nk - 1] = th[1:]
    th1[nk - 1] = 2. * th[nk - 1] - th[nk - 2]
    r = p * th1
    p = p * th
    q = -(p + r)
    rhs = np.zeros_like(tn)
    q[0] = q[0] - p[0]
    rhs[0] = rhs[0] - 2. * p[0] * POW(tn_int[0], 3.5)
    p[0] = 0.
    q[nk - 2] = q[nk - 2] + r[nk - 2]
    rhs[nk - 2] = rhs[nk - 2] + r[nk - 2] * dz * 3.5 * h_int[nk - 1] * fe / tek0[nk - 1]
    r[nk - 2] = 0.
    qtot = np.maximum(F["qo2p"] + F["qop"] + F["qn2p"] + F["qnop"] + F["qnp"] + F["qop2d"] + F["qop2p"], 1.e-20)
    qtot[:nk - 1] = SQRT(qtot[:nk - 1] * qtot[1:])
    qtot[nk - 1] = 0.
    root_ne = np.empty_like(tn)
    root_ne[:nk - 1] = ne[:nk - 1] * ne[1:]
    root_ne[nk - 1] = ne[nk - 1] * ne[nk - 1] * ne[nk - 1] / ne[nk - 2]
    root_ne = SQRT(np.maximum(root_ne, 1.e4))
    o2n = xnmbar * o2 * C["rmassinv_o2"]
    o1n = xnmbar * o1 * C["rmassinv_o1"]
    hen = xnmbar * he * C["rmassinv_he"]
    n2n = xnmbar * n2 * C["rmassinv_n2"]
    if C["electron_heating"] == 6:
        qe = LOG(root_ne / (o2n + n2n + o1n))
        qe = EXP(((((((-1.249e-5 * qe - 5.755e-4) * qe - 9.346e-3) * qe - 5.900e-2) * qe - 4.392e-2) * qe + 1.056) *
                  qe + 5.342))
    else:
        qe = LOG(root_ne / (o2n + n2n + 0.1 * o1n))
        qe = EXP(-((((0.001996 * qe + 0.08034) * qe + 1.166) * qe + 6.941) * qe + 12.75))
    rhs = rhs - qe * qtot * ev
    if C["et"]:
        rhs = rhs - (F["Q1"] + F["Q2"]) * 10.0
    root_te = SQRT(te)
    coll = np.where(te >= 1000., 2.e-7 * EXP(-4605.2 / te), 5.71e-8 * EXP(-3352.6 / te))
    coll = np.where(te > 2000., 2.53e-6 * root_te * EXP(-17620. / te), coll)
    with np.errstate(divide="ignore", invalid="ignore"):
        l2v = np.where(np.abs(te - tn) < dl, 3200. / (tn * tn),
                       1. / (te - tn) * (1. - EXP(-3200. * (te - tn) / (te * tn))))
    l2v = 1.3e-4 * l2v * coll
    leo2 = o2n * (1.21e-18 * (1. + 3.6e-2 * root_te) * root_te + 6.9e-14 / root_te + 3.125e-21 * (te * te))
    leo1d = 0.
    leo1 = o1n * (7.9e-19 * (1. + 5.7e-4 * te) * root_te + 3.4e-12 * (1. - 7.e-5 * te) / tn * (150. / te + 0.4))
    lehe = hen * 2.46e-17 * root_te
    len2 = n2n * (1.77E-19 * (1. - 1.21E-4 * te) * te + 2.9e-14 / root_te + l2v)
    len_ = leo2 + leo1 + lehe + len2
    if C["et"]:
        len_ = np.where((te > 500.0) & (F["Q2"] > 0.0), len_ * EXP(-7.54E-4 * (te - 500.0)), len_)
    lxen = (len_ + o1n * (1. - alam / (ad + sd * n2n)) * leo1d) * root_ne * ev
    len_ = (len_ + o1n * leo1d) * root_ne * ev
    ion = (F["op"] * C["rmassinv_o1"] + F["o2p"] * C["rmassinv_o2"] + F["nplus"] * C["rmassinv_n4s"] +
           F["n2p"] * C["rmassinv_n2"] + F["nop"] * C["rmassinv_no"])
    loss_ei = 3.2e-8 * root_ne / (root_te * te) * 15. * ev * C["rmass_o1"] * ion
    root_tn = SQRT(2 * tn)
    op, o2p, nplus, n2p, nop = (F[k] for k in ("op", "o2p", "nplus", "n2p", "nop"))
    loss_in = 1e-14 * ev * (op * (5.8 * o2n + 0.21 * o1n * root_tn + 2.8 * hen + 6.6 * n2n) +
                            o2p * (0.14 * o2n * root_tn + 4.36 * o1n + 1.63 * hen + 5.81 * n2n) +
                            nplus * (5.84 * o2n + 5.84 * o1n + 3.05 * hen + 6.56 * n2n) +
                            n2p * (5.54 * o2n + 4.65 * o1n + 1.82 * hen + 0.27 * n2n * root_tn) +
                            nop * (5.45 * o2n + 4.5 * o1n + 1.72 * hen + 5.92 * n2n))
    q = q - (len_ + loss_ei) / POW(te, 2.5)
    rhs = rhs - len_ * tn - loss_ei * ti
    q_eni = loss_ei * np.maximum(te - ti, 0.)
    q_eni = (lxen * (te - tn) + q_eni) * C["avo"] / xnmbar
    qi = np.empty_like(tn)
    qi[1:nk - 1] = .5 * (q_eni[:nk - 2] + q_eni[1:nk - 1])
    qi[0] = 1.5 * q_eni[0] - 0.5 * q_eni[1]
    qi[nk - 1] = 1.5 * q_eni[nk - 2] - 0.5 * q_eni[nk - 3]
    return p, q, r, rhs, qtotal + qi, loss_ei, loss_in


@pytest.mark.parametrize("nk,dz,et,eh", [(29, 0.5, 0, 0), (57, 0.25, 1, 6), (57, 0.25, 0, 6), (3, 0.5, 1, 0)])
def test_settei_matches_independent_transcription(pkg, orc, nk, dz, et, eh):
    F, C, qt = pkg.synth.settei_inputs(nk, 53, dz, 7 + nk, et=et, electron_heating=eh)
    (te, ti, q2), (p, q, r, rhs) = orc.settei_ng(F, C, qt, with_system=True)
    pn, qn, rn, rhsn, q2n, lei, lin = settei_numpy(F, C, qt)
    for got, want in ((p, pn), (q, qn), (r, rn), (rhs, rhsn)):
        assert np.array_equal(got[:nk - 1], want[:nk - 1])
    assert np.array_equal(q2, q2n)
    x = orc.trsolv_ng(pn, qn, rn, rhsn, nk - 1)
    x[:nk - 1] = POW(x[:nk - 1], 2. / 7.)
    x[nk - 1] = x[nk - 2] * x[nk - 2] / x[nk - 3]
    te_n = np.maximum(x, F["tn"])
    ti_n = np.maximum((F["qji_ti"] * F["xnmbar"] / C["avo"] + lei * te_n + lin * F["tn"]) / (lei + lin), F["tn"])
    assert np.array_equal(te, te_n)
    assert np.array_equal(ti, ti_n)
    assert np.all(np.isfinite(te)) and np.all(np.isfinite(ti))


def test_settei_inputs_cover_the_branches(pkg):
    F, C, qt = pkg.synth.settei_inputs(57, 400, 0.25, 1)
    arl, chi_deg = np.abs(F["rlatm"]), np.degrees(F["chi"])
    assert np.any(arl >= np.pi / 3) and np.any(arl <= np.pi / 18) and np.any((arl > np.pi / 18) & (arl < np.pi / 4.5))
    assert np.any((chi_deg > 80) & (chi_deg < 100)) and np.any(chi_deg >= 90) and np.any(chi_deg < 80)
    te = F["te"]
    assert np.any(te > 2000.) and np.any((te >= 1000.) & (te <= 2000.)) and np.any(te < 1000.)
    assert np.any(np.abs(te - F["tn"]) < 1e-6)
