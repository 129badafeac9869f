"""The comp_ng column step of the oracle (src/comp_ng.F90:74-332) and its
post-solve steps (:415-457), checked bit for bit against an independent
numpy transcription that follows the Fortran array statements, and the
oracle's block solve of comp_ng's system against the generic block solve."""
import math

import numpy as np
import pytest

from conftest import prec_fn
from test_minor_assembly import PHI, SS, matinv3

TAU, T00, THDIFFALPHA = 1.86e3, 273., -0.38
_pow = prec_fn(math.pow, np.power)
_log = prec_fn(math.log, np.log)
_exp = prec_fn(math.exp, np.exp)


def _comp_levels(F, C):
    """Interface quantities (comp_ng.F90:74-102) and level(j, thermal): ep, the
    alpha matrix, ak and wks4 of level j (:128-211); also wi."""
    nk, ncol = F["tn"].shape
    tn, o2, o1, he, w, mbar = (F[k] for k in ("tn", "o2", "o1", "he", "w", "mbar"))
    b, fb, dz = C["b"], C["fb"], C["dz"]
    dt = F["tn"].dtype
    ps0 = [b[i, 0] * o2[0] + b[i, 1] * o1[0] + b[i, 2] * he[0] + fb[i] for i in range(3)]
    embar0 = 1. / (ps0[0] * C["rmassinv_o2"] + ps0[1] * C["rmassinv_o1"] + ps0[2] * C["rmassinv_he"] +
                   (1. - ps0[0] - ps0[1] - ps0[2]) * C["rmassinv_n2"])
    o2i, o1i, hei, embari, tni, dembardz, dtndz = (np.empty_like(tn) for _ in range(7))
    o2i[0] = .5 * (ps0[0] + o2[0])
    o1i[0] = .5 * (ps0[1] + o1[0])
    hei[0] = .5 * (ps0[2] + he[0])
    embari[0] = .5 * (embar0 + mbar[0])
    tni[0] = F["tlbc"]
    dembardz[0] = mbar[0] - embar0
    dtndz[0] = (tn[0] - F["tlbc"]) * 2
    o2i[1:] = .5 * (o2[:-1] + o2[1:])
    o1i[1:] = .5 * (o1[:-1] + o1[1:])
    hei[1:] = .5 * (he[:-1] + he[1:])
    embari[1:] = .5 * (mbar[:-1] + mbar[1:])
    tni[1:] = .5 * (tn[:-1] + tn[1:])
    dembardz[1:] = mbar[1:] - mbar[:-1]
    dtndz[1:] = tn[1:] - tn[:-1]
    dembardz = dembardz / dz
    dtndz = dtndz / dz
    wi = np.empty_like(tn)
    wi[:-1] = .5 * (w[:-1] + w[1:])
    wi[-1] = 1.5 * w[-1] - .5 * w[-2]
    df = [_pow(tni / T00, 1.75 - SS[n]) for n in range(3)]
    phi = lambda i, j: PHI[i - 1, j - 1]
    rmass = (C["rmass_o2"], C["rmass_o1"], C["rmass_he"])

    def level(j, thermal):
        ep = [1. - 1. / embari[j] * (rmass[i] + dembardz[j]) for i in range(3)]
        if thermal:
            ep[2] = ep[2] - THDIFFALPHA * dtndz[j] / tni[j]
        a = np.empty((3, 3, ncol), dtype=dt)
        a[0, 0] = -(phi(1, 4) + (phi(1, 2) - phi(1, 4)) * o1i[j] + (df[0][j] * phi(1, 3) - phi(1, 4)) * hei[j])
        a[1, 1] = -(phi(2, 4) + (phi(2, 1) - phi(2, 4)) * o2i[j] + (df[1][j] * phi(2, 3) - phi(2, 4)) * hei[j])
        a[2, 2] = -(df[2][j] * phi(3, 4) + (df[0][j] * phi(3, 1) - df[2][j] * phi(3, 4)) * o2i[j] +
                    (df[1][j] * phi(3, 2) - df[2][j] * phi(3, 4)) * o1i[j])
        a[0, 1] = (phi(1, 2) - phi(1, 4)) * o2i[j]
        a[0, 2] = (df[0][j] * phi(1, 3) - phi(1, 4)) * o2i[j]
        a[1, 0] = (phi(2, 1) - phi(2, 4)) * o1i[j]
        a[1, 2] = (df[1][j] * phi(2, 3) - phi(2, 4)) * o1i[j]
        a[2, 0] = (df[0][j] * phi(3, 1) - df[2][j] * phi(3, 4)) * hei[j]
        a[2, 1] = (df[1][j] * phi(3, 2) - df[2][j] * phi(3, 4)) * hei[j]
        wks1 = embari[j] * C["rmassinv_n2"] * _pow(T00 / tni[j], 0.25) / TAU
        ak = matinv3(a) * wks1
        return ep, a, ak, dembardz[j] / (embari[j] * 2.)

    return level, wi, embari


def comp_numpy(F, C):
    """Returns (upd (3, nk, ncol), P, Q, R (3,3,nk-1,ncol), f (3,nk-1,ncol))."""
    nk, ncol = F["tn"].shape
    tn = F["tn"]
    b, fb, dz = C["b"], C["fb"], C["dz"]
    dt = F["tn"].dtype
    flx_he = F["flx_he"] if C["calc_helium"] else np.zeros(ncol, dtype=dt)
    fs = F["fs"].reshape(4, 3, ncol, nk)          # fs(k, col, isp, m) -> [m, isp, col, k]
    level, wi, embari = _comp_levels(F, C)
    ep_kp, a_kp, ak_kp, wks4 = level(0, True)
    nms = (F["o2nm_smooth"], F["o1nm_smooth"], F["henm_smooth"])
    adv = (F["o2_advec"], F["o1_advec"], F["he_advec"])
    hd = (F["hdo2"], F["hdo1"], F["hdhe"])
    dfac = F["dfactor"]
    P, Q, R = (np.zeros((3, 3, nk - 1, ncol), dtype=dt) for _ in range(3))
    fv = np.zeros((3, nk - 1, ncol), dtype=dt)
    gama = np.zeros((nk, 3, 3, ncol), dtype=dt)
    zz = np.zeros((nk, 3, ncol), dtype=dt)
    for k in range(nk - 1):
        ep_km, ak_km, wks3 = ep_kp, ak_kp, wks4
        ep_kp, a_kp, ak_kp, wks4 = level(k + 1, k + 1 != nk - 1)
        eddyp = C["expzmid_inv"] * F["difk"][k] * (1. / dz - wks3)
        eddyr = C["expzmid"] * F["difk"][k + 1] * (1. / dz + wks4)
        eddyq = (C["expzmid_inv"] * F["difk"][k] * (1. / dz + wks3) +
                 C["expzmid"] * F["difk"][k + 1] * (1. / dz - wks4))
        ez = F["expz"][k]
        pk, qk, rk = (np.empty((3, 3, ncol), dtype=dt) for _ in range(3))
        for isp in range(3):
            for m in range(3):
                d = 1. if isp == m else 0.
                molp = ak_km[isp, m] * (1. / dz + ep_km[m] / 2.)
                molr = ak_kp[isp, m] * (1. / dz - ep_kp[m] / 2.)
                molq = ak_km[isp, m] * (1. / dz - ep_km[m] / 2.) + ak_kp[isp, m] * (1. / dz + ep_kp[m] / 2.)
                pk[isp, m] = molp / dz - ez * d / dz * (eddyp * dfac + .5 * wi[k])
                rk[isp, m] = molr / dz - ez * d / dz * (eddyr * dfac - .5 * wi[k])
                qk[isp, m] = -molq / dz + ez * d * (eddyq * dfac / dz + C["dtx2inv"]) - ez * fs[m + 1, isp, :, k]
        fk = np.array([ez * (nms[i][k] * C["dtx2inv"] - (adv[i][k] - fs[0, i, :, k]) + hd[i][k]) for i in range(3)])
        if k == 0:
            for m in range(3):
                for n in range(3):
                    qk[:, m] = qk[:, m] + pk[:, n] * b[n, m]
            for m in range(3):
                fk = fk - pk[:, m] * fb[m]
            pk[...] = 0.
        elif k == nk - 2:
            for m in range(3):
                qk[:, m] = qk[:, m] + (1. + .5 * ep_kp[m] * dz) / (1. - .5 * ep_kp[m] * dz) * rk[:, m]
            a22, a33, a23, a32 = a_kp[1, 1], a_kp[2, 2], a_kp[1, 2], a_kp[2, 1]
            flx00 = embari[k] * C["rmassinv_n2"] * C["p0"] * _pow(T00 / tn[k], 0.25) / (TAU * C["grav"])
            fk = (fk - rk[:, 1] * (a23 - a22) * flx_he / (flx00 * (1. / dz - 0.5 * ep_kp[1])) -
                  rk[:, 2] * (a33 - a32) * flx_he / (flx00 * (1. / dz - 0.5 * ep_kp[2])))
            rk[...] = 0.
        P[:, :, k], Q[:, :, k], R[:, :, k], fv[:, k] = pk, qk, rk, fk
        for m in range(3):
            for n in range(3):
                qk[:, m] = qk[:, m] - pk[:, n] * gama[k, n, m]
        wkm1 = matinv3(qk)
        wkv1 = fk.copy()
        for m in range(3):
            wkv1 = wkv1 - pk[:, m] * zz[k, m]
            for n in range(3):
                gama[k + 1, :, m] = gama[k + 1, :, m] + wkm1[:, n] * rk[n, m]
        for m in range(3):
            zz[k + 1] = zz[k + 1] + wkm1[:, m] * wkv1[m]
    upd = np.zeros((3, nk, ncol), dtype=dt)
    for k in range(nk - 2, -1, -1):
        upd[:, k] = zz[k + 1]
        for isp in range(3):
            for m in range(3):
                upd[isp, k] = upd[isp, k] - gama[k + 1, isp, m] * upd[m, k + 1]
    for isp in range(3):
        upd[isp, nk - 1] = (1. + .5 * ep_kp[isp] * dz) / (1. - .5 * ep_kp[isp] * dz) * upd[isp, nk - 2]
    upd[1, nk - 1] = upd[1, nk - 1] + (a23 - a22) * flx_he / (flx00 * (1. / dz - 0.5 * ep_kp[1]))
    upd[2, nk - 1] = upd[2, nk - 1] + (a33 - a32) * flx_he / (flx00 * (1. / dz - 0.5 * ep_kp[2]))
    if not C["calc_helium"]:
        upd[2] = C["pshelb"]
    return upd, P, Q, R, fv


def comp_diag_numpy(F, C, upd):
    """comp_ng's addfld diagnostics (comp_ng.F90:334-380) as the array
    statements write them: sum(loss, dim=4) and sum(moldif, dim=4) add over
    the row's species, accumulated from 0."""
    nk, ncol = F["tn"].shape
    dz = C["dz"]
    fs = F["fs"].reshape(4, 3, ncol, nk)
    level, wi, _ = _comp_levels(F, C)
    L = [level(j, j != nk - 1) for j in range(nk)]
    nms = (F["o2nm_smooth"], F["o1nm_smooth"], F["henm_smooth"])
    adv = (F["o2_advec"], F["o1_advec"], F["he_advec"])
    hd = (F["hdo2"], F["hdo1"], F["hdhe"])
    names = ("O2", "O1", "HE")
    out = {}
    for i, n in enumerate(names):
        out["D" + n + "DT"] = C["dtx2inv"] * (upd[i] - nms[i])
        out[n + "_PROD"] = fs[0, i].T.copy()
        out[n + "_HORDIF"] = hd[i]
        out[n + "_HORADV"] = -adv[i]
    for m, n in enumerate(names):
        s = np.zeros((nk, ncol))
        for isp in range(3):
            s = s + fs[m + 1, isp].T * upd[m]
        out[n + "_LOSS"] = s
    moldif = np.zeros((3, nk, ncol))
    eddydif = np.zeros((3, nk, ncol))
    veradv = np.zeros((3, nk, ncol))
    for k in range(1, nk - 1):
        ep_km, _, ak_km, wks3 = L[k]
        ep_kp, _, ak_kp, wks4 = L[k + 1]
        eddyp = C["expzmid_inv"] * F["difk"][k] * (1. / dz - wks3)
        eddyr = C["expzmid"] * F["difk"][k + 1] * (1. / dz + wks4)
        eddyq = (C["expzmid_inv"] * F["difk"][k] * (1. / dz + wks3) +
                 C["expzmid"] * F["difk"][k + 1] * (1. / dz - wks4))
        for m in range(3):
            s = np.zeros(ncol)
            for isp in range(3):
                molp = ak_km[isp, m] * (1. / dz + ep_km[m] / 2.)
                molr = ak_kp[isp, m] * (1. / dz - ep_kp[m] / 2.)
                molq = ak_km[isp, m] * (1. / dz - ep_km[m] / 2.) + ak_kp[isp, m] * (1. / dz + ep_kp[m] / 2.)
                s = s + -(1. / F["expz"][k] / dz * (molp * upd[m, k - 1] - molq * upd[m, k] + molr * upd[m, k + 1]))
            moldif[m, k] = s
        for isp in range(3):
            eddydif[isp, k] = 1. / dz * (eddyp * upd[isp, k - 1] - eddyq * upd[isp, k] + eddyr * upd[isp, k + 1])
            veradv[isp, k] = wi[k] / (2 * dz) * (upd[isp, k + 1] - upd[isp, k - 1])
    eddydif = eddydif * F["dfactor"]
    for i, n in enumerate(names):
        out[n + "_MOLDIF"] = moldif[i]
        out[n + "_EDDYDIF"] = eddydif[i]
        out[n + "_VERADV"] = -veradv[i]
    return out


@pytest.mark.parametrize("nk,dz,calc_helium", [(29, 0.5, 1), (57, 0.25, 1), (3, 0.5, 1), (29, 0.5, 0)])
def test_comp_diagnostics_match_independent_transcription(pkg, orc, nk, dz, calc_helium):
    F, C = pkg.synth.comp_inputs(nk, 40, dz, 13 + nk, calc_helium=calc_helium)
    upd = orc.comp_ng(F, C)
    got = orc.comp_diag_ng(F, C, upd)
    want = comp_diag_numpy(F, C, np.array(upd))
    assert sorted(got) == sorted(orc.COMP_DIAG_NAMES)
    for name in orc.COMP_DIAG_NAMES:
        assert np.array_equal(got[name], want[name]), name


@pytest.mark.parametrize("nk,dz,calc_helium", [(29, 0.5, 1), (57, 0.25, 1), (3, 0.5, 1), (29, 0.5, 0)])
def test_comp_matches_independent_transcription(pkg, orc, nk, dz, calc_helium):
    F, C = pkg.synth.comp_inputs(nk, 37, dz, 3 + nk, calc_helium=calc_helium)
    upd, (P, Q, R, f, ubc) = orc.comp_ng(F, C, with_system=True)
    un, Pn, Qn, Rn, fn = comp_numpy(F, C)
    for i in range(3):
        assert np.array_equal(upd[i], un[i])
    for got, want in ((P, Pn), (Q, Qn), (R, Rn)):
        assert np.array_equal(got[:, :, :nk - 1], want)
    assert np.array_equal(f[:, :nk - 1], fn)
    assert np.all(np.isfinite(un))


@pytest.mark.parametrize("nk,dz", [(29, 0.5), (57, 0.25)])
def test_comp_solve_equals_block_solve(pkg, orc, nk, dz):
    """comp_ng's inline block solve (:280-332) is the generic block solve with
    k2 = nk-1 and the upper-boundary relation u(nk) = ratio*u(nk-1) + add."""
    F, C = pkg.synth.comp_inputs(nk, 41, dz, 17)
    upd, (P, Q, R, f, ubc) = orc.comp_ng(F, C, with_system=True)
    u = orc.blksolve(P, Q, R, f, nk - 1, ubc_ratio=ubc[:3], ubc_add=ubc[3:])
    for i in range(3):
        assert np.array_equal(u[i], upd[i])


def comp_post_numpy(F, C):
    o2u, o1u, heu = (F[k].copy() for k in ("o2_upd", "o1_upd", "he_upd"))
    ds, ds2, dz = C["dtsmooth"], C["dtsmooth_div2"], C["dz"]
    o2n = ds2 * (F["o2_nm"] + o2u) + ds * F["o2"]
    o1n = ds2 * (F["o1_nm"] + o1u) + ds * F["o1"]
    hen = ds2 * (F["he_nm"] + heu) + ds * F["he"]
    n2 = 1. - o2u - o1u - heu
    n2nm = 1. - o2n - o1n - hen
    nk, ncol = n2.shape
    zp, xn = F["zpmid"], F["xnmbar"]
    for i in range(ncol):
        below = np.nonzero(n2[:, i] < 0.01)[0]
        ktop = below[0] if below.size else nk
        if 0 < ktop < nk - 1:
            n2top = math.log(n2[ktop, i] * xn[ktop, i])
            n2top1 = math.log(n2[ktop - 1, i] * xn[ktop - 1, i])
            dn2dz = (n2top - n2top1) / dz
            for k in range(ktop + 1, nk):
                n2[k, i] = math.exp(n2top + dn2dz * (zp[k] - zp[ktop])) / xn[k, i]
    small = 1e-9
    out = []
    for a, b, c, d in ((o2u, o1u, heu, n2), (o2n, o1n, hen, n2nm)):
        a, b, c, d = (np.maximum(v, small) for v in (a, b, c, d))
        s = a + b + c + d
        out.append((a / s, b / s, c / s))
    return out[0] + out[1]


@pytest.mark.parametrize("nk,dz", [(29, 0.5), (57, 0.25)])
def test_comp_post_matches_independent_transcription(pkg, orc, nk, dz):
    F, C = pkg.synth.comp_post_inputs(nk, 64, dz, 5)
    got = orc.comp_post_ng(F, C)
    want = comp_post_numpy(F, C)
    for g, w in zip(got, want):
        assert np.array_equal(g, w)
    # about half the columns take the N2 extrapolation
    n2 = 1. - F["o2_upd"] - F["o1_upd"] - F["he_upd"]
    hit = np.any(n2[1:-1] < 0.01, axis=0).mean()
    assert 0.1 < hit < 0.95
