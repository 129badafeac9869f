"""The dt_ng column assembly of the oracle (src/dt_ng.F90:57-167), checked
bit for bit against an independent numpy transcription that follows the
Fortran array statements line by line."""
import numpy as np
import pytest


def dt_numpy(F, C):
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
    return p, q, r, rhs


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
