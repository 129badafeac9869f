"""Scalar tridiagonal solves on the GPU through the C ABI, against the oracle.

FP64 results must be bit-identical to the oracle (the reference's arithmetic
in the reference's order); the FP32+refinement path must be within 1e-10
relative (normwise per field) of it."""
import numpy as np
import pytest

from conftest import golden

pytestmark = pytest.mark.gpu


def rel_err(x, ref):
    return np.max(np.abs(x - ref)) / np.max(np.abs(ref))


def system(pkg, cfg, ncol, seed=0):
    wl = pkg.synth.workload(cfg)
    g = wl.grids[0]
    return pkg.synth.scalar_system(g.nk, ncol, g.dz, 100 + seed, wl.d0_range, wl.loss, wl.d_span), g.nk


@pytest.mark.parametrize("cfg,ncol", [(0, 2592), (1, 3001), (2, 777)])
def test_trsolv_ng_bit_exact(cuda, pkg, orc, cfg, ncol):
    (a, b, c, f), nk = system(pkg, cfg, ncol)
    x = np.zeros_like(a, order="F")
    assert pkg.trsolv_ng(a, b, c, f, x, nk) == pkg.TG_OK
    assert np.array_equal(x, orc.trsolv_ng(a, b, c, f, nk))


@pytest.mark.parametrize("nk,k2,ncol", [(1, 1, 5), (2, 2, 1), (3, 3, 31), (3, 2, 33), (57, 56, 1025), (113, 113, 63)])
def test_trsolv_ng_edges_and_k2(cuda, pkg, orc, nk, k2, ncol):
    rng = np.random.default_rng(nk * 1000 + ncol)
    a = np.asfortranarray(-rng.uniform(0.1, 1, (nk, ncol)))
    c = np.asfortranarray(-rng.uniform(0.1, 1, (nk, ncol)))
    b = np.asfortranarray(2.5 + rng.uniform(0, 1, (nk, ncol)))
    f = np.asfortranarray(rng.uniform(-1, 1, (nk, ncol)))
    x = np.full((nk, ncol), 123.5, order="F")
    assert pkg.trsolv_ng(a, b, c, f, x, k2) == pkg.TG_OK
    ref = orc.trsolv_ng(a, b, c, f, k2)
    assert np.array_equal(x[:k2], ref[:k2])
    assert np.all(x[k2:] == 123.5)  # rows above k2 are not written


def test_trsolv_ng_golden(cuda, pkg):
    g = golden("pin_trsolv_ng_29.npz")
    x = np.zeros_like(g["a"], order="F")
    pkg.trsolv_ng(g["a"], g["b"], g["c"], g["f"], x, 29)
    assert np.array_equal(x, g["x_nk"])
    kat = golden("kat_scalar.npz")
    for nk in (2, 3, 5, 29, 57):
        a, b, c, f, xs = (kat[f"nk{nk}_{k}"] for k in "abcfx")
        x = np.zeros_like(a, order="F")
        pkg.trsolv_ng(a, b, c, f, x, nk)
        assert np.max(np.abs(x - xs)) <= 1e-13 * np.max(np.abs(xs))


@pytest.mark.parametrize("lon0,lon1,k1,k2", [(1, 76, 1, 56), (3, 40, 1, 57), (20, 76, 1, 57), (1, 76, 5, 50)])
def test_trsolv_slab(cuda, pkg, orc, lon0, lon1, k1, k2):
    lonmax, nlev = 76, 57
    (a, b, c, f), _ = system(pkg, 1, lon1 - lon0 + 1, seed=lon0)
    x = np.full(a.shape, -9.0, order="F")
    assert pkg.trsolv(a, b, c, f, x, 1, nlev, k1, k2, lon0, lon1, lonmax, 17, 0) == pkg.TG_OK
    ref = orc.trsolv(a, b, c, f, np.full(a.shape, -9.0, order="F"), 1, nlev, k1, k2, lon0, lon1, lonmax)
    assert np.array_equal(x, ref)


def test_nonfinite_solution_status_and_values(cuda, pkg, orc):
    """Finite pivots but an inf or NaN right-hand side: the columns' x turn
    non-finite from that level down (also through a zero w2), the call
    reports TG_ENONFINITE and the values match the oracle's."""
    (a, b, c, f), nk = system(pkg, 0, 96)
    c = c.copy(order="F")
    f = f.copy(order="F")
    f[5, 7] = np.inf
    f[15, 12] = np.nan
    f[20, 33] = -np.inf
    c[19, 33] = 0.0        # w2 = 0 just below the inf level of column 33
    x = np.zeros_like(a, order="F")
    assert pkg.trsolv_ng(a, b, c, f, x, nk) == pkg.TG_ENONFINITE
    ref = orc.trsolv_ng(a, b, c, f, nk)
    assert np.array_equal(x, ref, equal_nan=True)
    assert not np.isfinite(x[0, [7, 12, 33]]).any()
    assert np.isfinite(np.delete(x, [7, 12, 33], axis=1)).all()


def test_zero_pivot_status_and_values(cuda, pkg, orc):
    (a, b, c, f), nk = system(pkg, 0, 64)
    b = b.copy(order="F")
    b[0, 5] = 0.0          # zero pivot
    b[3, 9] = np.nan       # non-finite pivot
    x = np.zeros_like(a, order="F")
    assert pkg.trsolv_ng(a, b, c, f, x, nk) == pkg.TG_EPIVOT
    ref = orc.trsolv_ng(a, b, c, f, nk)
    assert np.array_equal(x, ref, equal_nan=True)
    # the library stays usable after a flagged call
    (a, b, c, f), nk = system(pkg, 0, 64, seed=3)
    assert pkg.trsolv_ng(a, b, c, f, x, nk) == pkg.TG_OK
    assert np.array_equal(x, orc.trsolv_ng(a, b, c, f, nk))


@pytest.mark.parametrize("layout", ["level", "column"])
def test_device_entry(cuda, pkg, orc, layout):
    torch = cuda
    (a, b, c, f), nk = system(pkg, 1, 1000)
    ref = orc.trsolv_ng(a, b, c, f, nk)
    st = torch.zeros(1, dtype=torch.int32, device="cuda")
    if layout == "level":
        ld = 1000 + 24
        ta, tb, tc, tf = (pkg.batch.level_scalar(v, ld, "cuda") for v in (a, b, c, f))
        tx = torch.zeros((nk, ld), dtype=torch.float64, device="cuda")
        pkg.trsolv_dev(ta, tb, tc, tf, tx, nk, nk, 1000, pkg.TG_LAYOUT_LEVEL, ld, status=st)
        x = pkg.batch.from_level_scalar(tx, 1000)
    else:
        ta, tb, tc, tf = (torch.from_numpy(np.ascontiguousarray(v.T)).cuda() for v in (a, b, c, f))
        tx = torch.zeros_like(ta)
        pkg.trsolv_dev(ta, tb, tc, tf, tx, nk, nk, 1000, pkg.TG_LAYOUT_COLUMN, 0, status=st)
        x = np.asfortranarray(tx.cpu().numpy().T)
    torch.cuda.synchronize()
    assert int(st.item()) == pkg.TG_OK
    assert np.array_equal(x, ref)


def test_two_columns_per_thread(cuda, pkg, orc):
    torch = cuda
    cs = pkg.colsolve
    (a, b, c, f), nk = system(pkg, 1, 777)
    ref = orc.trsolv_ng(a, b, c, f, nk)
    ld = 800
    ta, tb, tc, tf = (pkg.batch.level_scalar(v, ld, "cuda") for v in (a, b, c, f))
    tx = torch.zeros((nk, ld), dtype=torch.float64, device="cuda")
    cs.set_pipeline(cs.TG_KIND_SCALAR, cs.TG_PREC_F64, 0)
    cs.set_scratch_global(cs.TG_KIND_SCALAR, cs.TG_PREC_F64, 0)
    cs.set_tile(cs.TG_KIND_SCALAR, cs.TG_PREC_F64, 128, 2)
    try:
        pkg.trsolv_dev(ta, tb, tc, tf, tx, nk, nk, 777, pkg.TG_LAYOUT_LEVEL, ld)
        torch.cuda.synchronize()
    finally:
        cs.set_tile(cs.TG_KIND_SCALAR, cs.TG_PREC_F64, 0, 0)
        cs.set_scratch_global(cs.TG_KIND_SCALAR, cs.TG_PREC_F64, -1)
        cs.set_pipeline(cs.TG_KIND_SCALAR, cs.TG_PREC_F64, -1)
    assert np.array_equal(pkg.batch.from_level_scalar(tx, 777), ref)
    assert torch.all(tx[:, 777:] == 0)  # padding columns are not written


@pytest.mark.parametrize("cfg", [0, 1, 2])
def test_refine_accuracy(cuda, pkg, orc, cfg):
    torch = cuda
    (a, b, c, f), nk = system(pkg, cfg, 2000, seed=7)
    ref = orc.trsolv_ng(a, b, c, f, nk)
    ld = 2016
    ta, tb, tc, tf = (pkg.batch.level_scalar(v, ld, "cuda") for v in (a, b, c, f))
    tx = torch.zeros((nk, ld), dtype=torch.float64, device="cuda")
    st = torch.zeros(1, dtype=torch.int32, device="cuda")
    pkg.trsolv_dev(ta, tb, tc, tf, tx, nk, nk, 2000, pkg.TG_LAYOUT_LEVEL, ld, pkg.TG_PREC_F32_REFINE, status=st)
    torch.cuda.synchronize()
    x = pkg.batch.from_level_scalar(tx, 2000)
    assert rel_err(x, ref) <= 1e-10
    assert int(st.item()) in (pkg.TG_OK, pkg.TG_ENOCONV)


def test_division_routine_matches_ieee(cuda, pkg):
    """The kernels divide by a shared correctly rounded reciprocal with
    Markstein's correction; every quotient must equal IEEE a/b exactly."""
    torch = cuda
    rng = np.random.default_rng(99)
    n = 1 << 21
    a = rng.standard_normal(n) * np.exp2(rng.integers(-60, 60, n))
    b = rng.standard_normal(n) * np.exp2(rng.integers(-60, 60, n))
    # wide exponents, near-equal operands, exact quotients and edge values
    a[:4096] = rng.uniform(0.5, 1.0, 4096) * np.exp2(rng.integers(-1000, 1000, 4096))
    b[:4096] = rng.uniform(0.5, 1.0, 4096) * np.exp2(rng.integers(-1000, 1000, 4096))
    a[4096:8192] = b[4096:8192] * rng.integers(-1000, 1000, 4096)
    a[8192:8192 + 16] = [0.0, -0.0, np.inf, -np.inf, np.nan, 1e-310, 5e-324, 1e308, 1.0, 3.0, 1.0, -7.0, 2.0, 1e-300, 1e300, 0.0]
    b[8192:8192 + 16] = [3.0, 3.0, 2.0, 2.0, 1.0, 3.0, 7.0, 1e-10, 0.0, -0.0, np.inf, 1e-310, 5e-324, 1e300, 1e-300, np.nan]
    ta, tb = torch.from_numpy(a).cuda(), torch.from_numpy(b).cuda()
    tq = torch.empty_like(ta)
    pkg.selftest_division(ta, tb, tq)
    torch.cuda.synchronize()
    q = tq.cpu().numpy()
    with np.errstate(all="ignore"):
        ref = a / b
    same = (q.view(np.int64) == ref.view(np.int64)) | (np.isnan(q) & np.isnan(ref))
    assert same.all(), (a[~same][:5], b[~same][:5], q[~same][:5], ref[~same][:5])


def test_trsolv_deferred_latitude_scan_bit_exact(cuda, pkg, orc):
    """The global grid's latitude scan as dt.F runs it (one work array per
    latitude, reused for the next), with every trsolv call deferred and one
    flush: each latitude's x equals tg_trsolv's and the oracle's bit for bit.
    Slabs of two row counts (k2 = lev1-1 and lev1) and a partial-longitude
    slab make three runs in the flush."""
    nlev, lonmax, nlat = 57, 148, 72
    tn_upd = np.full((nlev, lonmax, nlat), -9.0, order="F")
    refs = {}
    work = [np.zeros((nlev, lonmax), order="F") for _ in range(4)]
    for lat in range(nlat):
        (a, b, c, f), _ = system(pkg, 1, lonmax, seed=500 + lat)
        for w, v in zip(work, (a, b, c, f)):
            w[...] = v                    # the scan's reused work arrays
        k2 = nlev - 1 if lat % 3 else nlev
        lon0, lon1 = (1, lonmax) if lat != 5 else (3, 80)
        x = tn_upd[:, lon0 - 1:lon1, lat]
        args = (1, nlev, 1, k2, lon0, lon1, lonmax)
        sl = [w[:, lon0 - 1:lon1] for w in work]
        sl = [np.asfortranarray(v) for v in sl]
        pkg.trsolv_defer(*sl, x, *args)
        refs[lat] = orc.trsolv(*sl, np.full(x.shape, -9.0, order="F"), *args)
        for w in work:
            w[...] = np.nan               # the caller reuses its arrays at once
    assert pkg.trsolv_flush() == pkg.TG_OK
    for lat, ref in refs.items():
        lon0, lon1 = (1, lonmax) if lat != 5 else (3, 80)
        assert np.array_equal(tn_upd[:, lon0 - 1:lon1, lat], ref), lat
    # an empty flush is a no-op
    assert pkg.trsolv_flush() == pkg.TG_OK
