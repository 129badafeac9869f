"""The dt_ng column assembly of the oracle (src/dt_ng.F90:57-167), checked
bit for bit against an independent numpy transcription that follows the
Fortran array statements line by line."""
import numpy as np
import pytest


def dt_numpy(F, C, keep=None):
    """The assembled rows; keep (a dict), if given, receives the intermediates."""
    nk = F["tn"].shape[0]
    tn, w, cp, km, un, vn, qt = (F[k] for k in ("tn", "w", "cp", "km", "un", "vn", "qtotal"))
    expz, dift = F["expz"][:, None], F["dift"][:, None]
    dz, dtx2inv = C["dz"], C["dtx2inv"]
    vad = np.empty_like(tn)
    vad[0] = (tn[0] - F["t_lbc"]) * w[0] * 2.
    vad[nk - 1] = 0.
    vad[1:nk - 1] = (tn[1:nk - 1] - tn[0:nk - 2]) * w[1:nk - 1]
    for k in range(nk - 1):
        vad[k] = (vad[k] + vad[k + 1]) * .5
    vad = vad / dz
    advec = F["horadv"] + vad
    cpi, kmi, wi = (np.empty_like(tn) for _ in range(3))
    for dst, src in ((cpi, cp), (kmi, km), (wi, w)):
        dst[:nk - 1] = .5 * (src[:nk - 1] + src[1:])
        dst[nk - 1] = 1.5 * src[nk - 1] - .5 * src[nk - 2]
    cptn = cpi * (advec - dtx2inv * F["tnsmooth"])
    cptn = cptn * expz
    dudz, dvdz = np.empty_like(tn), np.empty_like(tn)
    dudz[1:nk - 2] = (un[2:nk - 1] - un[0:nk - 3]) / (2. * dz)
    dvdz[1:nk - 2] = (vn[2:nk - 1] - vn[0:nk - 3]) / (2. * dz)
    dudz[0] = (un[0] + 1. / 3. * un[1] - 4. / 3. * F["ulbc"]) / dz
    dvdz[0] = (vn[0] + 1. / 3. * vn[1] - 4. / 3. * F["vlbc"]) / dz
    dudz[nk - 2] = dudz[nk - 3] / 3.
    dvdz[nk - 2] = dvdz[nk - 3] / 3.
    dudz[nk - 1] = dudz[nk - 2] / 3.
    dvdz[nk - 1] = dvdz[nk - 2] / 3.
    qsolar = np.empty_like(tn)
    qsolar[:nk - 1] = .5 * (qt[:nk - 1] + qt[1:])
    qsolar[nk - 1] = 1.5 * qt[nk - 1] - .5 * qt[nk - 2]
    qrecomb = C["tsurplus"] * F["rkm12"] * (F["xnmbar"] * F["o1"] * C["rmassinv_o1"]) ** 2 * C["avo"] / F["mbar"]
    qm = C["grav"] * kmi / (C["p0"] * F["scht"]) * (dudz ** 2 + dvdz ** 2)
    qm = qm / expz
    total_heat = qsolar + F["hdt"] + qrecomb + F["qji_tn"] + qm
    cptn = cptn - total_heat * expz
    tni = np.empty_like(tn)
    tni[1:nk - 1] = .5 * (tn[0:nk - 2] + tn[1:nk - 1])
    tni[0] = F["tlbc"]
    tni[nk - 1] = tn[nk - 2]
    h = F["schti"]
    rho = C["p0"] * C["expzmid_inv"] / (h * C["grav"])
    rho = rho * expz
    gpart = h ** 2 * rho * cp
    g = C["grav"] * (F["kt"] + gpart * dift) / (C["p0"] * h * dz ** 2)
    f = C["grav"] ** 2 * h ** 2 * rho / (tni * C["p0"] * 2. * dz)
    f = f * dift
    p, q, r = (np.zeros_like(tn) for _ in range(3))
    p[:nk - 1] = g[:nk - 1] - f[:nk - 1]
    q[:nk - 1] = -(g[1:] - f[1:] + g[:nk - 1] + f[:nk - 1])
    r[:nk - 1] = g[1:] + f[1:]
    q[nk - 2] = -g[nk - 2] - f[nk - 2]
    r[nk - 2] = 0.
    rhs = cptn
    qpart = cpi * (dtx2inv + F["cool_imp"]) + wi * C["gask"] / F["mbar"]
    rhs = rhs + F["cool_exp"]
    q = q - qpart * expz
    q[0] = q[0] - p[0]
    rhs[0] = rhs[0] - 2. * p[0] * F["t_lbc"]
    p[0] = 0.
    if keep is not None:
        keep.update(vad=vad, cpi=cpi, wi=wi, qsolar=qsolar, qrecomb=qrecomb, qm=qm, g=g, f=f, rho=rho)
    return p, q, r, rhs


def dt_diag_numpy(F, C, tn_upd):
    """dt_ng.F90:169-191 (and DEN, :133) as the Fortran array statements."""
    m = {}
    dt_numpy(F, C, keep=m)
    nk = F["tn"].shape[0]
    expz = F["expz"][:, None]
    cpi, g, f, x = m["cpi"], m["g"], m["f"], tn_upd
    out = {"DTDT": C["dtx2inv"] * (x - F["tnsmooth"]), "DT_SOLAR": m["qsolar"] / cpi, "DT_HORDIF": F["hdt"] / cpi,
           "DT_RECOMB": m["qrecomb"] / cpi, "DT_JOULE": F["qji_tn"] / cpi, "DT_MOLDIF": m["qm"] / cpi}
    dt_cool_exp = F["cool_exp"] / cpi
    dt_cool_exp = dt_cool_exp / expz
    out["DT_COOL"] = -dt_cool_exp - F["cool_imp"] * x
    out["DT_HORADV"] = -F["horadv"]
    out["DT_VERADV"] = -m["vad"]
    out["DT_ADIA"] = -m["wi"] * C["gask"] / (cpi * F["mbar"]) * x
    cond = np.zeros_like(x)
    k = slice(1, nk - 1)
    km1, kp1 = slice(0, nk - 2), slice(2, nk)
    cond[k] = 1 / expz[k] * ((g[k] - f[k]) * x[km1] - (g[kp1] - f[kp1] + g[k] + f[k]) * x[k] +
                             (g[kp1] + f[kp1]) * x[kp1])
    out["DT_CONDUCT"] = cond / cpi
    out["DEN"] = m["rho"] * np.ones_like(x)
    return out


@pytest.mark.parametrize("nk,dz", [(29, 0.5), (57, 0.25), (3, 0.5)])
def test_dt_assembly_matches_independent_transcription(pkg, orc, nk, dz):
    F, C = pkg.synth.dt_inputs(nk, 47, dz, 11 + nk)
    tn_upd, (p, q, r, rhs) = orc.dt_ng(F, C, with_system=True)
    pn, qn, rn, rhsn = dt_numpy(F, C)
    for got, want in ((p, pn), (q, qn), (r, rn), (rhs, rhsn)):
        assert np.array_equal(got[:nk - 1], want[:nk - 1])
    # the solve of the assembled system, and the top row
    x = orc.trsolv_ng(pn, qn, rn, rhsn, nk - 1)
    assert np.array_equal(tn_upd[:nk - 1], x[:nk - 1])
    assert np.array_equal(tn_upd[nk - 1], x[nk - 2] ** 2 / x[nk - 3])
    assert np.all(np.isfinite(tn_upd))


@pytest.mark.parametrize("nk,dz", [(29, 0.5), (57, 0.25), (3, 0.5)])
def test_dt_diagnostics_match_independent_transcription(pkg, orc, nk, dz):
    F, C = pkg.synth.dt_inputs(nk, 47, dz, 13 + nk)
    tn_upd = orc.dt_ng(F, C)
    got = orc.dt_diag_ng(F, C, tn_upd)
    want = dt_diag_numpy(F, C, tn_upd)
    assert set(got) == set(want)
    for name in got:
        # -x and (-1)*x differ only in the sign of zero; compare values
        assert np.array_equal(got[name], want[name]), name
    assert np.all(got["DT_CONDUCT"][[0, nk - 1]] == 0.0)
