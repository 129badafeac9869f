"""The minor_ng column assembly of the oracle (src/minor_ng.F90:60-200),
checked bit for bit against an independent numpy transcription that follows
the Fortran array statements line by line.  The fractional powers go through
math.pow (the C library's pow, as the oracle uses)."""
import math

import numpy as np
import pytest

TAU, T00 = 1.86e3, 273.
SS = (1.710, 1.749, 1.718)
PHI = np.array([0., 0.673, 0.270, 1.35, 0., 0.404, 2.16, 1.616, 0., 1.11, 0.769, 0.322]).reshape((3, 4), order="F")
from conftest import prec_fn  # noqa: E402

_pow = prec_fn(math.pow, np.power)


def matinv3(a):
    """matutil.F90 matinv3 = matadj3 / matdet3 on (3, 3, ...) arrays."""
    d = (a[0, 0] * a[1, 1] * a[2, 2] - a[0, 0] * a[1, 2] * a[2, 1] - a[0, 1] * a[1, 0] * a[2, 2] +
         a[0, 1] * a[1, 2] * a[2, 0] + a[0, 2] * a[1, 0] * a[2, 1] - a[0, 2] * a[1, 1] * a[2, 0])
    adj = np.empty_like(a)
    adj[0, 0] = (a[1, 1] * a[2, 2] - a[1, 2] * a[2, 1])
    adj[1, 0] = -(a[1, 0] * a[2, 2] - a[1, 2] * a[2, 0])
    adj[2, 0] = (a[1, 0] * a[2, 1] - a[1, 1] * a[2, 0])
    adj[0, 1] = -(a[0, 1] * a[2, 2] - a[0, 2] * a[2, 1])
    adj[1, 1] = (a[0, 0] * a[2, 2] - a[0, 2] * a[2, 0])
    adj[2, 1] = -(a[0, 0] * a[2, 1] - a[0, 1] * a[2, 0])
    adj[0, 2] = (a[0, 1] * a[1, 2] - a[0, 2] * a[1, 1])
    adj[1, 2] = -(a[0, 0] * a[1, 2] - a[0, 2] * a[1, 0])
    adj[2, 2] = (a[0, 0] * a[1, 1] - a[0, 1] * a[1, 0])
    return adj / d


def minor_numpy(F, C, keep=None):
    nk = F["tn"].shape[0]
    tn, o2, o1, he, mbar, barm, w = (F[k] for k in ("tn", "o2", "o1", "he", "mbar", "barm", "w"))
    b, fb, dzp, rmx = C["b"], C["fb"], C["dzp"], C["rmx"]
    phix = np.asarray(C["phix"])
    salfax = phix[:3] - phix[3]
    bo2 = b[0, 0] * o2[0] + b[0, 1] * o1[0] + b[0, 2] * he[0] + fb[0]
    bo1 = b[1, 0] * o2[0] + b[1, 1] * o1[0] + b[1, 2] * he[0] + fb[1]
    bhe = b[2, 0] * o2[0] + b[2, 1] * o1[0] + b[2, 2] * he[0] + fb[2]
    xmbari = 1. / (bo2 * C["rmassinv_o2"] + bo1 * C["rmassinv_o1"] + (1. - bo2 - bo1 - bhe) * C["rmassinv_n2"] +
                   bhe * C["rmassinv_he"])
    dmdz, pso1, pso2, pshe, do1dz, do2dz, dhedz = (np.empty_like(tn) for _ in range(7))
    dmdz[0] = (mbar[0] - xmbari) / dzp
    pso1[0] = .5 * (bo1 + o1[0])
    pso2[0] = .5 * (bo2 + o2[0])
    pshe[0] = .5 * (bhe + he[0])
    do1dz[0] = (o1[0] - bo1) / dzp
    do2dz[0] = (o2[0] - bo2) / dzp
    dhedz[0] = (he[0] - bhe) / dzp
    dmdz[1:] = (mbar[1:] - mbar[:-1]) / dzp
    pso1[1:] = .5 * (o1[1:] + o1[:-1])
    pso2[1:] = .5 * (o2[1:] + o2[:-1])
    pshe[1:] = .5 * (he[1:] + he[:-1])
    do1dz[1:] = (o1[1:] - o1[:-1]) / dzp
    do2dz[1:] = (o2[1:] - o2[:-1]) / dzp
    dhedz[1:] = (he[1:] - he[:-1]) / dzp
    tni = np.empty_like(tn)
    tni[0] = F["tlbc"]
    tni[nk - 1] = tn[nk - 2]
    tni[1:nk - 1] = .5 * (tn[1:nk - 1] + tn[0:nk - 2])
    s0prod = F["sprod"] * rmx / F["xnmbar"]
    df = [_pow(tni / T00, 1.75 - SS[n]) for n in range(3)]
    phi = lambda i, j: PHI[i - 1, j - 1]
    alfa = np.empty((3, 3) + tn.shape, dtype=tn.dtype)
    alfa[0, 0] = -(phi(1, 4) + (phi(1, 2) - phi(1, 4)) * pso1 + (df[0] * phi(1, 3) - phi(1, 4)) * pshe)
    alfa[1, 1] = -(phi(2, 4) + (phi(2, 1) - phi(2, 4)) * pso2 + (df[1] * phi(2, 3) - phi(2, 4)) * pshe)
    alfa[2, 2] = -(df[2] * phi(3, 4) + (df[0] * phi(3, 1) - df[2] * phi(3, 4)) * pso2 +
                   (df[1] * phi(3, 2) - df[2] * phi(3, 4)) * pso1)
    alfa[0, 1] = (phi(1, 2) - phi(1, 4)) * pso2
    alfa[0, 2] = (df[0] * phi(1, 3) - phi(1, 4)) * pso2
    alfa[1, 0] = (phi(2, 1) - phi(2, 4)) * pso1
    alfa[1, 2] = (df[1] * phi(2, 3) - phi(2, 4)) * pso1
    alfa[2, 0] = (df[0] * phi(3, 1) - df[2] * phi(3, 4)) * pshe
    alfa[2, 1] = (df[1] * phi(3, 2) - df[2] * phi(3, 4)) * pshe
    inv = matinv3(alfa)
    # dot_product(salfax, invalfa(:,n)), summed left to right
    sa = [salfax[0] * inv[0, n] + salfax[1] * inv[1, n] + salfax[2] * inv[2, n] for n in range(3)]
    ex = (1. - (rmx + dmdz) / barm +
          sa[0] * (do2dz - (1. - (C["rmass_o2"] + dmdz) / barm) * pso2) +
          sa[1] * (do1dz - (1. - (C["rmass_o1"] + dmdz) / barm) * pso1) +
          sa[2] * (dhedz - (1. - (C["rmass_he"] + dmdz) / barm) * pshe))
    dmdz = dmdz / barm
    ax = -(barm / (TAU * C["rmass_n2"]) * _pow(T00 / tni, 0.25) /
           (phix[2] + salfax[0] * pso2 + salfax[1] * pso1 + salfax[2] * pshe))
    dtnidz = np.empty_like(tn)
    dtnidz[1:nk - 1] = (tni[2:] - tni[:nk - 2]) / 2.
    dtnidz[0] = tni[1] - tni[0]
    dtnidz[nk - 1] = tni[nk - 1] - tni[nk - 2]
    thdiff = ex - C["alfax"] * dtnidz / (dzp * tni)
    wi = np.empty_like(tn)
    wi[:nk - 1] = .5 * (w[:nk - 1] + w[1:])
    wi[nk - 1] = 1.5 * w[nk - 1] - .5 * w[nk - 2]
    difk, expz, dfac = F["difk"][:, None], F["expz"][:, None], F["dfactor"]
    molp = ax[:-1] * (1. / dzp + .5 * thdiff[:-1])
    molr = ax[1:] * (1. / dzp - .5 * thdiff[1:])
    molq = ax[:-1] * (1. / dzp - .5 * thdiff[:-1]) + ax[1:] * (1. / dzp + .5 * thdiff[1:])
    eddyp = C["expzmid_inv"] * difk[:-1] * (1. / dzp - .5 * dmdz[:-1])
    eddyr = C["expzmid"] * difk[1:] * (1. / dzp + .5 * dmdz[1:])
    eddyq = (C["expzmid_inv"] * difk[:-1] * (1. / dzp + .5 * dmdz[:-1]) +
             C["expzmid"] * difk[1:] * (1. / dzp - .5 * dmdz[1:]))
    p, q, r = (np.empty_like(tn) for _ in range(3))
    p[:-1] = molp / dzp - expz[:-1] * (eddyp * dfac + .5 * wi[:-1]) / dzp
    r[:-1] = molr / dzp - expz[:-1] * (eddyr * dfac - .5 * wi[:-1]) / dzp
    q[:-1] = -molq / dzp + expz[:-1] * (eddyq * dfac / dzp + C["dtx2inv"] - F["sloss"][:-1])
    f = F["ftm1_smooth"] * C["dtx2inv"] - F["hadvec"] + s0prod
    f = f * expz
    l1, l2, l3 = F["flbc1"], F["flbc2"], F["flbc3"]
    q[0] = q[0] + p[0] * (l1 + .5 * l2 * dzp) / (l1 - .5 * l2 * dzp)
    f[0] = f[0] - p[0] * l3 * dzp / (l1 - .5 * l2 * dzp)
    p[0] = 0.
    p[nk - 1] = 1. + .5 * dzp * thdiff[nk - 1]
    q[nk - 1] = p[nk - 1] - 2.
    r[nk - 1] = 0.
    f[nk - 1] = -C["grav"] * rmx * F["fubc"] * dzp / (C["p0"] * ax[nk - 1] * C["avo"])
    if keep is not None:
        keep.update(molp=molp, molq=molq, molr=molr, eddyp=eddyp, eddyq=eddyq, eddyr=eddyr, wi=wi, s0prod=s0prod)
    return p, q, r, f


def minor_diag_numpy(F, C, x):
    """minor_ng.F90:202-224: the values the reference passes to addfld."""
    m = {}
    minor_numpy(F, C, keep=m)
    nk = x.shape[0]
    dzp, expz = C["dzp"], F["expz"][:, None]
    k, km1, kp1 = slice(1, nk - 1), slice(0, nk - 2), slice(2, nk)
    moldif, eddydif, veradv = (np.zeros_like(x) for _ in range(3))
    # molp(k) etc. are the rows k of the k = 1..nk-1 arrays
    moldif[k] = -1 / expz[k] / dzp * (m["molp"][k] * x[km1] - m["molq"][k] * x[k] + m["molr"][k] * x[kp1])
    eddydif[k] = 1 / dzp * (m["eddyp"][k] * x[km1] - m["eddyq"][k] * x[k] + m["eddyr"][k] * x[kp1])
    veradv[k] = m["wi"][k] / (2 * dzp) * (x[kp1] - x[km1])
    eddydif = eddydif * F["dfactor"]
    return {"DPDT": C["dtx2inv"] * (x - F["ftm1_smooth"]), "PROD": m["s0prod"] * np.ones_like(x),
            "LOSS": F["sloss"] * x, "MOLDIF": moldif, "EDDYDIF": eddydif, "VERADV": -veradv, "HORADV": -F["hadvec"]}


@pytest.mark.parametrize("nk,dz", [(29, 0.5), (57, 0.25), (3, 0.5)])
def test_minor_assembly_matches_independent_transcription(pkg, orc, nk, dz):
    F, C = pkg.synth.minor_inputs(nk, 41, dz, 5 + nk)
    x, (p, q, r, f) = orc.minor_ng(F, C, with_system=True)
    pn, qn, rn, fn = minor_numpy(F, C)
    for got, want in ((p, pn), (q, qn), (r, rn), (f, fn)):
        assert np.array_equal(got, want)
    assert np.array_equal(x, orc.trsolv_ng(pn, qn, rn, fn, nk))
    assert np.all(np.isfinite(x))


def test_minor_inputs_give_a_well_posed_system(pkg, orc):
    F, C = pkg.synth.minor_inputs(57, 64, 0.25, 1)
    x = orc.minor_ng(F, C)
    # the column solution stays at the species' mixing-ratio scale
    assert np.all(np.isfinite(x)) and np.max(np.abs(x)) < 1e-3


@pytest.mark.parametrize("nk,dz", [(29, 0.5), (57, 0.25), (3, 0.5)])
def test_minor_diagnostics_match_independent_transcription(pkg, orc, nk, dz):
    F, C = pkg.synth.minor_inputs(nk, 41, dz, 7 + nk)
    x = orc.minor_ng(F, C)
    got = orc.minor_diag_ng(F, C, x)
    want = minor_diag_numpy(F, C, x)
    assert set(got) == set(want)
    for name in got:
        assert np.array_equal(got[name], want[name]), name
