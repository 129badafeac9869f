"""History diagnostics of dt_ng (src/dt_ng.F90:169-191) and minor_ng
(src/minor_ng.F90:202-224) on the GPU against the oracle's restatement:
dt_ng's bit for bit; minor_ng's bit for bit except MOLDIF and EDDYDIF, which
carry the device's fractional powers (the level quantities of the solve)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MINOR_TOL = 1e-12


def _rel(got, want):
    scale = np.maximum(np.max(np.abs(want), axis=0), 1e-300)
    return float(np.max(np.abs(got - want) / scale))


def _level(pkg, torch, F, nk, ncol, one_d):
    ld = pkg.batch.pad_ld(ncol)
    dev = {}
    for k, v in F.items():
        if v.ndim == 2:
            dev[k] = pkg.batch.level_scalar(v, ld, "cuda")
        elif k in one_d:
            dev[k] = torch.from_numpy(np.ascontiguousarray(v)).cuda()
        else:
            t = torch.zeros(ld, dtype=torch.float64, device="cuda")
            t[:ncol] = torch.from_numpy(v)
            dev[k] = t
    return dev, ld


@pytest.mark.parametrize("nk,dz,ncol", [(57, 0.25, 3001), (29, 0.5, 777), (113, 0.125, 300), (3, 0.5, 33),
                                        (4, 0.5, 65)])
def test_dt_diag_host_bit_exact(cuda, pkg, orc, nk, dz, ncol):
    F, C = pkg.synth.dt_inputs(nk, ncol, dz, 70 + nk)
    tn_upd = orc.dt_ng(F, C)
    got = pkg.dt_diag_ng(F, C, tn_upd)
    want = orc.dt_diag_ng(F, C, tn_upd)
    for name in pkg.colsolve.DT_DIAG_NAMES:
        assert np.array_equal(got[name], want[name]), name


def test_dt_diag_device_bit_exact(cuda, pkg, orc):
    torch = cuda
    nk, ncol, dz = 57, 1000, 0.25
    F, C = pkg.synth.dt_inputs(nk, ncol, dz, 12)
    tn_upd = orc.dt_ng(F, C)
    dev, ld = _level(pkg, torch, F, nk, ncol, ("expz", "dift"))
    x = pkg.batch.level_scalar(tn_upd, ld, "cuda")
    diag = torch.full((12, nk, ld), 7.0, dtype=torch.float64, device="cuda")
    stream = torch.cuda.Stream()
    pkg.dt_diag_ng_dev(dev, C, x, diag, nk, ncol, ld, stream=stream)
    stream.synchronize()
    want = orc.dt_diag_ng(F, C, tn_upd)
    for i, name in enumerate(pkg.colsolve.DT_DIAG_NAMES):
        assert np.array_equal(pkg.batch.from_level_scalar(diag[i], ncol), want[name]), name


EXACT_MINOR = ("DPDT", "PROD", "LOSS", "VERADV", "HORADV")


@pytest.mark.parametrize("nk,dz,ncol", [(57, 0.25, 3001), (29, 0.5, 2592), (113, 0.125, 500), (3, 0.5, 33)])
def test_minor_diag_host(cuda, pkg, orc, nk, dz, ncol):
    F, C = pkg.synth.minor_inputs(nk, ncol, dz, 80 + nk)
    fcomp = orc.minor_ng(F, C)
    got = pkg.minor_diag_ng(F, C, fcomp)
    want = orc.minor_diag_ng(F, C, fcomp)
    for name in pkg.colsolve.MINOR_DIAG_NAMES:
        if name in EXACT_MINOR:
            assert np.array_equal(got[name], want[name]), name
        else:
            assert _rel(got[name], want[name]) <= MINOR_TOL, name
            assert np.all(got[name][0] == 0.0) and np.all(got[name][-1] == want[name][-1])


def test_minor_diag_device(cuda, pkg, orc):
    torch = cuda
    nk, ncol, dz = 57, 1000, 0.25
    F, C = pkg.synth.minor_inputs(nk, ncol, dz, 14)
    fcomp = orc.minor_ng(F, C)
    dev, ld = _level(pkg, torch, F, nk, ncol, ("expz", "difk"))
    x = pkg.batch.level_scalar(fcomp, ld, "cuda")
    diag = torch.full((7, nk, ld), 7.0, dtype=torch.float64, device="cuda")
    pkg.minor_diag_ng_dev(dev, C, x, diag, nk, ncol, ld)
    torch.cuda.synchronize()
    want = orc.minor_diag_ng(F, C, fcomp)
    for i, name in enumerate(pkg.colsolve.MINOR_DIAG_NAMES):
        got = pkg.batch.from_level_scalar(diag[i], ncol)
        if name in EXACT_MINOR:
            assert np.array_equal(got, want[name]), name
        else:
            assert _rel(got, want[name]) <= MINOR_TOL, name


# comp_ng: MOLDIF and EDDYDIF carry the level quantities ak, ep, wks4 with the
# device's fractional powers, and MOLDIF's three-point difference of large
# terms cancels (measured on B200: 1.02e-12 of the column's largest value);
# the other 18 planes are bit-identical.
COMP_TOL = 1e-11


def _comp_check(pkg, got, want):
    for name in pkg.colsolve.COMP_DIAG_NAMES:
        if name.endswith("_MOLDIF") or name.endswith("_EDDYDIF"):
            assert _rel(got[name], want[name]) <= COMP_TOL, name
        else:
            assert np.array_equal(got[name], want[name]), name


@pytest.mark.parametrize("nk,dz,ncol,calc_helium", [(57, 0.25, 2001, 1), (29, 0.5, 777, 0), (113, 0.125, 300, 1),
                                                    (3, 0.5, 33, 1)])
def test_comp_diag_host(cuda, pkg, orc, nk, dz, ncol, calc_helium):
    F, C = pkg.synth.comp_inputs(nk, ncol, dz, 90 + nk, calc_helium=calc_helium)
    upd = orc.comp_ng(F, C)
    got = pkg.comp_diag_ng(F, C, *[np.asfortranarray(u) for u in upd])
    want = orc.comp_diag_ng(F, C, upd)
    _comp_check(pkg, got, want)


def test_comp_diag_device(cuda, pkg, orc):
    torch = cuda
    nk, ncol, dz = 57, 1500, 0.25
    F, C = pkg.synth.comp_inputs(nk, ncol, dz, 19)
    upd = orc.comp_ng(F, C)
    ld = pkg.batch.pad_ld(ncol)
    grid = type("G", (), dict(nk=nk, ncol=ncol, ld=ld))()
    dev = pkg.dynamics._dev_fields(F, grid, ("expz", "difk"), "cuda")
    x = torch.stack([pkg.batch.level_scalar(np.asfortranarray(u), ld, "cuda") for u in upd])
    diag = torch.full((24, nk, ld), 7.0, dtype=torch.float64, device="cuda")
    stream = torch.cuda.Stream()
    pkg.comp_diag_ng_dev(dev, C, x, diag, nk, ncol, ld, stream=stream)
    stream.synchronize()
    got = {n: pkg.batch.from_level_scalar(diag[i], ncol) for i, n in enumerate(pkg.colsolve.COMP_DIAG_NAMES)}
    _comp_check(pkg, got, orc.comp_diag_ng(F, C, upd))


# oplus_ng: OP_DIFF carries dj, whose collision frequency takes the device's
# log10 (and pow with the diffusion cap); the other five are bit-identical.
OPLUS_TOL = 1e-12


def _oplus_check(pkg, got, want):
    for name in pkg.colsolve.OPLUS_DIAG_NAMES:
        if name == "OP_DIFF":
            assert _rel(got[name], want[name]) <= OPLUS_TOL, name
        else:
            assert np.array_equal(got[name], want[name]), name


@pytest.mark.parametrize("nk,dz,ncol,cap,horizontal", [(57, 0.25, 2001, 0.0, True), (29, 0.5, 777, 1e7, False),
                                                       (3, 0.5, 33, 0.0, True)])
def test_oplus_diag_host(cuda, pkg, orc, nk, dz, ncol, cap, horizontal):
    F, C = pkg.synth.oplus_inputs(nk, ncol, dz, 95 + nk, opdiffcap=cap)
    op = orc.oplus_ng(F, C)[0]
    rng = np.random.default_rng(nk)
    h3 = [np.asfortranarray(rng.uniform(-1e-3, 1e-3, op.shape)) for _ in range(3)] if horizontal else [None] * 3
    got = pkg.oplus_diag_ng(F, C, np.asfortranarray(op), *h3)
    want = orc.oplus_diag_ng(F, C, op, *h3)
    _oplus_check(pkg, got, want)


def test_oplus_diag_device(cuda, pkg, orc):
    torch = cuda
    nk, ncol, dz = 57, 1500, 0.25
    F, C = pkg.synth.oplus_inputs(nk, ncol, dz, 29)
    op = orc.oplus_ng(F, C)[0]
    rng = np.random.default_rng(3)
    h3 = [np.asfortranarray(rng.uniform(-1e-3, 1e-3, op.shape)) for _ in range(3)]
    dev, ld = _level(pkg, torch, F, nk, ncol, ("zpint",))
    x = pkg.batch.level_scalar(np.asfortranarray(op), ld, "cuda")
    hd = [pkg.batch.level_scalar(h, ld, "cuda") for h in h3]
    diag = torch.full((6, nk, ld), 7.0, dtype=torch.float64, device="cuda")
    stream = torch.cuda.Stream()
    pkg.oplus_diag_ng_dev(dev, C, x, diag, nk, ncol, ld, *hd, stream=stream)
    stream.synchronize()
    got = {n: pkg.batch.from_level_scalar(diag[i], ncol) for i, n in enumerate(pkg.colsolve.OPLUS_DIAG_NAMES)}
    _oplus_check(pkg, got, orc.oplus_diag_ng(F, C, op, *h3))
