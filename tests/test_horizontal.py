"""Horizontal operators advec_ng (src/advec_ng.F90) and smooth_ng
(src/smooth_ng.F90) on a nest held as one subdomain: the oracle against an
independent numpy transcription and analytic properties, and the CUDA entries
(host and device forms) against the oracle, bit for bit."""
import numpy as np
import pytest

from conftest import golden

RE_INV = 1.0 / 6.37122e8   # 1/re, re in cm
SHAPIRO = 3.0e-2


def nest_inputs(nk, nlon, nlat, seed, dlon_deg=0.625, dlat_deg=0.625, lat0_deg=20.0):
    """Seeded fields of one nest: f and the winds (nk, nlon+4, nlat+4), racs
    = 1/(re cos(lat)) per latitude row, the grid spacings in radians."""
    rng = np.random.default_rng(seed)
    shape = (nk, nlon + 4, nlat + 4)
    lon = np.arange(nlon + 4)[None, :, None]
    lat = np.arange(nlat + 4)[None, None, :]
    lev = np.arange(nk)[:, None, None]
    f = (800.0 + 50.0 * np.sin(0.3 * lon + 0.1 * lev) * np.cos(0.2 * lat) + rng.normal(0.0, 2.0, shape))
    un = rng.uniform(-1.0e4, 1.0e4, shape)
    vn = rng.uniform(-1.0e4, 1.0e4, shape)
    latdeg = lat0_deg + dlat_deg * (np.arange(nlat + 4) - 2)
    racs = 1.0 / (6.37122e8 * np.cos(np.radians(latdeg)))
    return (np.asfortranarray(f), np.asfortranarray(un), np.asfortranarray(vn), racs,
            np.radians(dlon_deg), np.radians(dlat_deg))


def _shift(a, d, axis):
    """a[t + d] along axis (only read where t + d is in range)."""
    return np.roll(a, -d, axis=axis)


def np_df(f, order, axis):
    n = f.shape[axis]
    idx = np.arange(n).reshape([-1 if ax == axis else 1 for ax in range(f.ndim)])
    out = (_shift(f, order, axis) - _shift(f, -order, axis)) / float(2 * order)
    if order == 2:
        near = (_shift(f, 1, axis) - _shift(f, -1, axis)) / 2.0
        out = np.where((idx == 1) | (idx == n - 2), near, out)
    out = np.where(idx == 0, _shift(f, 1, axis) - f, out)
    out = np.where(idx == n - 1, f - _shift(f, -1, axis), out)
    return out


def np_fm(f, order, axis):
    n = f.shape[axis]
    idx = np.arange(n).reshape([-1 if ax == axis else 1 for ax in range(f.ndim)])
    out = (_shift(f, order, axis) + _shift(f, -order, axis)) / 2.0
    if order == 2:
        near = (_shift(f, 1, axis) + _shift(f, -1, axis)) / 2.0
        out = np.where((idx == 1) | (idx == n - 2), near, out)
    return np.where((idx == 0) | (idx == n - 1), f, out)


def np_advec(f, un, vn, racs, dlamda, dphi, re_inv):
    nlond, nlatd = f.shape[1], f.shape[2]
    d1, d2, m1, m2 = np_df(f, 1, 1), np_df(f, 2, 1), np_fm(un, 1, 1), np_fm(un, 2, 1)
    wk1 = d1 * 2. * 2. / 3. * m1 - d2 * 4. / 12. * m2
    edge = np.zeros(nlond, bool)
    edge[[0, 1, nlond - 2, nlond - 1]] = True
    wk1[:, edge, :] = (d1 * m1)[:, edge, :]
    wk1 = wk1 * racs[None, None, :]
    d1, d2, m1, m2 = np_df(f, 1, 2), np_df(f, 2, 2), np_fm(vn, 1, 2), np_fm(vn, 2, 2)
    wk2 = d1 * 2. * 2. / 3. * m1 - d2 * 4. / 12. * m2
    edge = np.zeros(nlatd, bool)
    edge[[0, 1, nlatd - 2, nlatd - 1]] = True
    wk2[:, :, edge] = (d1 * m1)[:, :, edge]
    return wk1 / dlamda + wk2 * re_inv / dphi


def np_smooth(fin, shapiro):
    def one(x, axis):
        n = x.shape[axis]
        idx = np.arange(n).reshape([-1 if ax == axis else 1 for ax in range(x.ndim)])
        m1, m2 = np_fm(x, 1, axis), np_fm(x, 2, axis)
        y = x - shapiro * (2. * m2 - 8. * m1 + 6. * x)
        y = np.where((idx == 1) | (idx == n - 2), x - shapiro * (-8. * m1 + 8. * x), y)
        return np.where((idx == 0) | (idx == n - 1), x, y)
    return one(one(fin, 2), 1)


def same_bits(a, b):
    return np.array_equal(np.asarray(a).view(np.int64), np.asarray(b).view(np.int64))


SIZES = [(57, 12, 9), (29, 1, 1), (3, 6, 2), (57, 97, 65)]


@pytest.mark.parametrize("nk,nlon,nlat", SIZES)
def test_oracle_advec_matches_numpy(orc, nk, nlon, nlat):
    f, un, vn, racs, dlam, dphi = nest_inputs(nk, nlon, nlat, 3 + nlon)
    got = orc.advec_ng(f, un, vn, racs, dlam, dphi, RE_INV)
    assert same_bits(got, np_advec(f, un, vn, racs, dlam, dphi, RE_INV))


@pytest.mark.parametrize("nk,nlon,nlat", SIZES)
def test_oracle_smooth_matches_numpy(orc, nk, nlon, nlat):
    f = nest_inputs(nk, nlon, nlat, 7 + nlat)[0]
    assert same_bits(orc.smooth_ng(f, SHAPIRO), np_smooth(f, SHAPIRO))


def test_oracle_properties(orc):
    """A constant field is advected to zero and left unchanged by the
    filter; a field linear in longitude gives u*slope*racs/dlamda in the
    interior for a wind constant along longitude (the fourth-order weights
    4/3 and -1/3 sum to one)."""
    nk, nlon, nlat = 5, 10, 7
    f, un, vn, racs, dlam, dphi = nest_inputs(nk, nlon, nlat, 1)
    un = np.asfortranarray(np.broadcast_to(un[:, :1, :], un.shape).copy())
    c = np.full_like(f, 273.25, order="F")
    assert np.all(orc.advec_ng(c, un, vn, racs, dlam, dphi, RE_INV) == 0.0)
    assert np.array_equal(orc.smooth_ng(c, SHAPIRO), c)
    slope = 0.75
    lin = np.asfortranarray(np.broadcast_to(slope * np.arange(nlon + 4)[None, :, None], f.shape).copy())
    h = orc.advec_ng(lin, un, vn, racs, dlam, dphi, RE_INV)
    want = un * slope * racs[None, None, :] / dlam
    inner = (slice(None), slice(2, nlon + 2), slice(None))
    assert np.allclose(h[inner], want[inner], rtol=1e-13, atol=0.0)


def _gpu_fields(torch, arrays, ld):
    """(nk, nlond, nlatd) Fortran arrays -> level-major (nk, ld) CUDA tensors
    with the column index i + nlond*j, padding filled with a marker."""
    out = []
    for a in arrays:
        nk = a.shape[0]
        ncol = a.shape[1] * a.shape[2]
        t = torch.full((nk, ld), -5.5, dtype=torch.float64, device="cuda")
        t[:, :ncol] = torch.from_numpy(np.ascontiguousarray(a.reshape(nk, ncol, order="F")))
        out.append(t)
    return out


@pytest.mark.gpu
@pytest.mark.parametrize("nk,nlon,nlat", SIZES + [(57, 193, 129)])
def test_advec_smooth_host_bit_exact(cuda, pkg, orc, nk, nlon, nlat):
    f, un, vn, racs, dlam, dphi = nest_inputs(nk, nlon, nlat, 11 + nk)
    h = np.zeros_like(f, order="F")
    assert pkg.advec_ng(f, un, vn, racs, dlam, dphi, RE_INV, h) == pkg.TG_OK
    assert same_bits(h, orc.advec_ng(f, un, vn, racs, dlam, dphi, RE_INV))
    s = np.zeros_like(f, order="F")
    assert pkg.smooth_ng(f, SHAPIRO, s) == pkg.TG_OK
    assert same_bits(s, orc.smooth_ng(f, SHAPIRO))


@pytest.mark.gpu
@pytest.mark.parametrize("nk,nlon,nlat", [(57, 97, 65), (29, 1, 1)])
def test_advec_smooth_device_level_major(cuda, pkg, orc, nk, nlon, nlat):
    torch = cuda
    f, un, vn, racs, dlam, dphi = nest_inputs(nk, nlon, nlat, 5)
    ncol = (nlon + 4) * (nlat + 4)
    ld = pkg.batch.pad_ld(ncol)
    df, dun, dvn, dh, ds = _gpu_fields(torch, [f, un, vn, f, f], ld)
    dr = torch.from_numpy(racs).cuda()
    assert pkg.advec_ng_dev(df, dun, dvn, dr, dlam, dphi, RE_INV, dh, nk, nlon, nlat, ld) == pkg.TG_OK
    assert pkg.smooth_ng_dev(df, SHAPIRO, ds, nk, nlon, nlat, ld) == pkg.TG_OK
    torch.cuda.synchronize()
    want_h = orc.advec_ng(f, un, vn, racs, dlam, dphi, RE_INV).reshape(nk, ncol, order="F")
    want_s = orc.smooth_ng(f, SHAPIRO).reshape(nk, ncol, order="F")
    assert same_bits(dh[:, :ncol].cpu().numpy(), want_h)
    assert same_bits(ds[:, :ncol].cpu().numpy(), want_s)
    assert bool((dh[:, ncol:] == -5.5).all()) and bool((ds[:, ncol:] == -5.5).all())


def test_horizontal_rejects_bad_arguments(pkg):
    """Argument checks run before any device call, so they hold without a GPU."""
    a = np.zeros((3, 5, 5), order="F")
    r = np.zeros(5)
    with pytest.raises(pkg.TgError):
        pkg.advec_ng(a, a, a, r, 0.01, 0.01, RE_INV, a)          # output aliases an input
    with pytest.raises(pkg.TgError):
        pkg.smooth_ng(a, SHAPIRO, a)
    L = pkg.colsolve.lib()
    assert L.tg_smooth_ng_dev(8, SHAPIRO, 16, 3, 0, 1, 64, None) == pkg.TG_EINVAL       # nlon < 1
    assert L.tg_smooth_ng_dev(8, SHAPIRO, 16, 3, 1, 1, 20, None) == pkg.TG_EINVAL       # ld < 25 columns
    assert L.tg_advec_ng_dev(8, 16, 24, 32, 0.01, 0.01, RE_INV, 40, 70000, 1, 1, 64, None) == pkg.TG_EINVAL


def _kat():
    g = golden("kat_horizontal.npz")
    return {k: g[k] for k in g.files}


def test_oracle_known_answers(orc):
    """Exact answers computed in rational arithmetic (tests/golden/make_golden.py)."""
    g = _kat()
    h = orc.advec_ng(g["f"], g["un"], g["vn"], g["racs"], float(g["dlamda"]), float(g["dphi"]), float(g["re_inv"]))
    assert np.array_equal(h, g["hadvec"])
    assert np.array_equal(orc.smooth_ng(g["f"], float(g["shapiro"])), g["fout"])


@pytest.mark.gpu
def test_known_answers_on_gpu(cuda, pkg):
    g = _kat()
    h = np.zeros_like(g["f"], order="F")
    assert pkg.advec_ng(g["f"], g["un"], g["vn"], g["racs"], float(g["dlamda"]), float(g["dphi"]),
                        float(g["re_inv"]), h) == pkg.TG_OK
    assert np.array_equal(h, g["hadvec"])
    s = np.zeros_like(g["f"], order="F")
    assert pkg.smooth_ng(g["f"], float(g["shapiro"]), s) == pkg.TG_OK
    assert np.array_equal(s, g["fout"])


def test_python_shape_checks(pkg):
    a = np.zeros((3, 5, 5), order="F")
    with pytest.raises(ValueError):
        pkg.advec_ng(a, a, np.zeros((3, 5, 6), order="F"), np.zeros(5), 0.01, 0.01, RE_INV,
                     np.zeros((3, 5, 5), order="F"))
    with pytest.raises(ValueError):
        pkg.advec_ng(a, a, a, np.zeros(4), 0.01, 0.01, RE_INV, np.zeros((3, 5, 5), order="F"))
    with pytest.raises(ValueError):
        pkg.smooth_ng(a, SHAPIRO, np.zeros((3, 5, 4), order="F"))
    with pytest.raises(ValueError):
        pkg.time_filter_ng(0, a, np.zeros((3, 5), order="F"), 0.95, 0.025, np.zeros((3, 5, 5), order="F"),
                           np.zeros((3, 5, 5), order="F"))
