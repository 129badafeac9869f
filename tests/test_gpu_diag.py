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
