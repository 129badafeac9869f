"""dt_ng fused assembly + solve on the GPU against the oracle, bit for bit."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("nk,dz,ncol", [(57, 0.25, 3001), (29, 0.5, 2592), (113, 0.125, 500), (3, 0.5, 33)])
def test_dt_ng_host_bit_exact(cuda, pkg, orc, nk, dz, ncol):
    F, C = pkg.synth.dt_inputs(nk, ncol, dz, 7 + nk)
    tn_upd = np.zeros((nk, ncol), order="F")
    assert pkg.dt_ng(F, C, tn_upd) == pkg.TG_OK
    assert np.array_equal(tn_upd, orc.dt_ng(F, C))


def test_dt_ng_device_system_and_solution(cuda, pkg, orc):
    torch = cuda
    nk, ncol, dz = 57, 1000, 0.25
    F, C = pkg.synth.dt_inputs(nk, ncol, dz, 3)
    ref, (p, q, r, rhs) = orc.dt_ng(F, C, with_system=True)
    ld = pkg.batch.pad_ld(ncol)
    dev = {}
    for k, v in F.items():
        if v.ndim == 2:
            dev[k] = pkg.batch.level_scalar(v, ld, "cuda")
        elif k in ("expz", "dift"):
            dev[k] = torch.from_numpy(np.ascontiguousarray(v)).cuda()
        else:
            t = torch.zeros(ld, dtype=torch.float64, device="cuda")
            t[:ncol] = torch.from_numpy(v)
            dev[k] = t
    out = torch.zeros((nk, ld), dtype=torch.float64, device="cuda")
    sysout = torch.zeros((4, nk, ld), dtype=torch.float64, device="cuda")
    st = torch.zeros(1, dtype=torch.int32, device="cuda")
    pkg.dt_ng_dev(dev, C, out, nk, ncol, ld, system_out=sysout, status=st)
    torch.cuda.synchronize()
    assert int(st.item()) == pkg.TG_OK
    assert np.array_equal(pkg.batch.from_level_scalar(out, ncol), ref)
    for i, want in enumerate((p, q, r, rhs)):
        got = pkg.batch.from_level_scalar(sysout[i], ncol)
        assert np.array_equal(got[:nk - 1], want[:nk - 1])


def _rel(got, want):
    scale = np.maximum(np.max(np.abs(want), axis=0), 1e-300)
    return float(np.max(np.abs(got - want) / scale))


# minor_ng: the device pow differs from the C library's pow in the last bit
# now and then, so the fused kernel agrees with the oracle to a tolerance.
MINOR_TOL = 1e-12


@pytest.mark.parametrize("nk,dz,ncol", [(57, 0.25, 3001), (29, 0.5, 2592), (113, 0.125, 500), (3, 0.5, 33),
                                        (300, 0.05, 70)])
def test_minor_ng_host(cuda, pkg, orc, nk, dz, ncol):
    F, C = pkg.synth.minor_inputs(nk, ncol, dz, 9 + nk)
    out = np.zeros((nk, ncol), order="F")
    assert pkg.minor_ng(F, C, out) == pkg.TG_OK
    assert _rel(out, orc.minor_ng(F, C)) <= MINOR_TOL


def test_minor_ng_device_system_and_solution(cuda, pkg, orc):
    torch = cuda
    nk, ncol, dz = 57, 1000, 0.25
    F, C = pkg.synth.minor_inputs(nk, ncol, dz, 4)
    ref, sysref = orc.minor_ng(F, C, with_system=True)
    ld = pkg.batch.pad_ld(ncol)
    dev = {}
    for k, v in F.items():
        if v.ndim == 2:
            dev[k] = pkg.batch.level_scalar(v, ld, "cuda")
        elif k in ("expz", "difk"):
            dev[k] = torch.from_numpy(np.ascontiguousarray(v)).cuda()
        else:
            t = torch.zeros(ld, dtype=torch.float64, device="cuda")
            t[:ncol] = torch.from_numpy(v)
            dev[k] = t
    out = torch.zeros((nk, ld), dtype=torch.float64, device="cuda")
    sysout = torch.zeros((4, nk, ld), dtype=torch.float64, device="cuda")
    st = torch.zeros(1, dtype=torch.int32, device="cuda")
    pkg.minor_ng_dev(dev, C, out, nk, ncol, ld, system_out=sysout, status=st)
    torch.cuda.synchronize()
    assert int(st.item()) == pkg.TG_OK
    assert _rel(pkg.batch.from_level_scalar(out, ncol), ref) <= MINOR_TOL
    for i, want in enumerate(sysref):
        assert _rel(pkg.batch.from_level_scalar(sysout[i], ncol), want) <= MINOR_TOL
