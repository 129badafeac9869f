"""The column walks of the three-pass assembly routines on rows the test forms
itself (tg_selftest_walk).  Both walks divide by Markstein's sequence without
a branch and, from the first level whose operands leave the sequence's safe
range (zeros, extreme magnitudes), walk the rest again with IEEE division;
the bits must be the oracle's Thomas solve (src/trsolv_ng.F90:14-26) and, for
oplus_ng's factor pass, the IEEE recurrence w1 = q - p*w2, 1/w1, w2 = r/w1
(src/oplus_ng.F90:230-305 through trsolv), in the shared-memory tile walk
(up to 16384 columns) and in the global-memory walk alike."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _planted(pkg, nk, ncol, seed):
    """A diffusion-like system with operands outside the safe range planted
    in a few columns, the last (ragged) tile included."""
    a, b, c, f = (np.array(v) for v in pkg.synth.scalar_system(nk, ncol, 0.25, seed))
    f[0, 3] = 0.0                      # a zero numerator at level 0
    c[10, 40] = 0.0                    # a zero w2 from level 10 on
    f[20:, 77] *= 1e200                # numerators above 2**500
    for v in (a, b, c, f):             # every operand below 2**-500
        v[:, 100] *= 1e-200
    f[nk - 1, 130] = 0.0               # a zero numerator at the top
    c[nk - 1, :] = 0.0                 # the top row's r (its w2 is never used)
    f[5, ncol - 1] = 0.0
    b[30, 200 % ncol] *= 1e170         # one huge pivot in the middle
    return [np.asfortranarray(v) for v in (a, b, c, f)]


def _planes(torch, arrs, nk, ld):
    buf = torch.zeros((len(arrs), nk, ld), dtype=torch.float64, device="cuda")
    for i, v in enumerate(arrs):
        buf[i, :, :v.shape[1]] = torch.from_numpy(np.ascontiguousarray(v))
    return buf


@pytest.mark.parametrize("ncol,pad", [(1500, 0), (1500, 5), (17000, 0)],
                         ids=["tile", "tile_odd_ld", "global"])
@pytest.mark.parametrize("top", [0, 1])
def test_thomas_walk_is_the_oracle_solve(cuda, pkg, orc, ncol, pad, top):
    torch = cuda
    nk = 57
    K = nk - 1 if top == 1 else nk
    ld = ncol + pad
    a, b, c, f = _planted(pkg, nk, ncol, 31 + top)
    x0 = np.full((nk, ncol), -7.0, order="F")
    buf = _planes(torch, [a, b, c, f, x0], nk, ld)
    st = torch.zeros(1, dtype=torch.int32, device="cuda")
    pkg.selftest_walk(0, buf, nk, K, top, ncol, ld, st)
    torch.cuda.synchronize()
    assert int(st.item()) == pkg.TG_OK
    got = buf[4, :, :ncol].cpu().numpy()
    want = orc.trsolv_ng(a, b, c, f, K)
    assert np.array_equal(got[:K], want[:K])
    if top == 1:
        assert np.array_equal(got[K], want[K - 1] * want[K - 1] / want[K - 2])
    else:
        assert np.all(got[K:] == -7.0)


def _factor_ieee(p, q, r):
    """w1, 1/w1, w2 of every level with IEEE operations, level by level."""
    K = p.shape[0]
    w1, y1, w2 = (np.empty_like(p) for _ in range(3))
    for k in range(K):
        w1[k] = q[k] if k == 0 else q[k] - p[k] * w2[k - 1]
        y1[k] = 1.0 / w1[k]
        w2[k] = r[k] / w1[k]
    return w1, y1, w2


@pytest.mark.parametrize("ncol", [1500, 17000], ids=["tile", "global"])
def test_oplus_factor_pass_is_the_ieee_recurrence(cuda, pkg, ncol):
    torch = cuda
    nk = 57
    K = nk - 1
    ld = ncol + 3
    a, b, c, _ = _planted(pkg, K, ncol, 41)
    n = pkg.oplus_ng_factor_doubles(nk, ld)
    fac = torch.full((n,), 5.0, dtype=torch.float64, device="cuda")
    planes = fac.view(-1, nk, ld)
    for i, v in ((6, a), (7, b), (8, c)):
        planes[i, :K, :ncol] = torch.from_numpy(np.ascontiguousarray(v))
    st = torch.zeros(1, dtype=torch.int32, device="cuda")
    pkg.selftest_walk(1, fac, nk, K, 1, ncol, ld, st)
    torch.cuda.synchronize()
    assert int(st.item()) == pkg.TG_OK
    w1, y1, w2 = _factor_ieee(a, b, c)
    assert np.array_equal(planes[10, :K, :ncol].cpu().numpy(), w1)
    assert np.array_equal(planes[11, :K, :ncol].cpu().numpy(), y1)
    assert np.array_equal(planes[12, :K - 1, :ncol].cpu().numpy(), w2[:K - 1])


@pytest.mark.parametrize("ncol", [1500, 17000], ids=["tile", "global"])
def test_walks_report_a_zero_pivot(cuda, pkg, ncol):
    torch = cuda
    nk = 57
    a, b, c, f = (np.array(v) for v in pkg.synth.scalar_system(nk, ncol, 0.25, 51))
    a[12, 9] = b[12, 9] = 0.0          # w1 = 0 - 0*w2 at level 12 of one column
    buf = _planes(torch, [a, b, c, f, np.zeros((nk, ncol))], nk, ncol)
    st = torch.zeros(1, dtype=torch.int32, device="cuda")
    pkg.selftest_walk(0, buf, nk, nk, 0, ncol, ncol, st)
    torch.cuda.synchronize()
    assert int(st.item()) == pkg.TG_EPIVOT
    fac = torch.zeros((pkg.oplus_ng_factor_doubles(nk, ncol),), dtype=torch.float64, device="cuda")
    planes = fac.view(-1, nk, ncol)
    for i, v in ((6, a), (7, b), (8, c)):
        planes[i, :nk - 1] = torch.from_numpy(np.ascontiguousarray(v[:nk - 1]))
    st.zero_()
    pkg.selftest_walk(1, fac, nk, nk - 1, 1, ncol, ncol, st)
    torch.cuda.synchronize()
    assert int(st.item()) == pkg.TG_EPIVOT
