"""The polar ring filter (src/ringfilter.F:1-111) as filter_o2o
(src/comp.F:1065-1145) applies it to the whole global grid: the oracle
against an independent numpy transcription of the Fortran statements, bit
for bit; the GPU kernel against the oracle, bit for bit."""
import math

import numpy as np
import pytest


def ringfilter_numpy(f, order, poly, chunks, dlamda):
    """ringfilter.F transcribed with numpy over the levels; sums run in
    longitude order (a loop), trigonometry from the C library (math)."""
    f = np.array(f, dtype=np.float64, order="F", copy=True)
    nk, nlonp4, nlat = f.shape
    nlon = nlonp4 - 4
    nf = len(chunks)
    for lat in range(1, nlat + 1):
        nchnk = chunks[lat - 1] if lat <= nf else chunks[nlat - lat] if lat >= nlat - nf + 1 else 0
        if nchnk == 0:
            continue
        w = f[:, 2:nlon + 2, lat - 1].T.copy()          # (nlon, nk)
        a0 = np.zeros(nk)
        for i in range(nlon):
            a0 = a0 + w[i]
        a0 = a0 / nlon
        a, b = np.zeros((order, nk)), np.zeros((order, nk))
        for i in range(1, nlon + 1):
            ang = i * dlamda
            for m in range(1, order + 1):
                a[m - 1] = a[m - 1] + w[i - 1] * math.cos(m * ang)
                b[m - 1] = b[m - 1] + w[i - 1] * math.sin(m * ang)
        a = 2. * a / nlon
        b = 2. * b / nlon
        wm = np.empty_like(w)
        for i in range(1, nlon + 1):
            ang = i * dlamda
            wm[i - 1] = a0
            for m in range(1, order + 1):
                wm[i - 1] = wm[i - 1] + a[m - 1] * math.cos(m * ang) + b[m - 1] * math.sin(m * ang)
        fx = w - wm
        n = nlon // nchnk
        avg = np.empty((nchnk, nk))
        for c in range(nchnk):
            s = np.zeros(nk)
            for i in range(c * n, (c + 1) * n):
                s = s + fx[i]
            avg[c] = s / n
        for ic in range(1, nchnk + 1):
            im2 = ic - 2 + (nchnk if ic - 2 <= 0 else 0)
            im1 = ic - 1 + (nchnk if ic - 1 <= 0 else 0)
            ip1 = ic + 1 - (nchnk if ic + 1 >= nchnk + 1 else 0)
            ip2 = ic + 2 - (nchnk if ic + 2 >= nchnk + 1 else 0)
            left = (-avg[im2 - 1] + 7. * avg[im1 - 1] + 7. * avg[ic - 1] - avg[ip1 - 1]) / 12.
            right = (-avg[im1 - 1] + 7. * avg[ic - 1] + 7. * avg[ip1 - 1] - avg[ip2 - 1]) / 12.
            fa = (left + right - 2. * avg[ic - 1]) / float(n ** 2)
            fb = (3. * avg[ic - 1] - 2. * left - right) / n
            for m in range(1, n + 1):
                if poly:
                    fx[(ic - 1) * n + m - 1] = fa * (3. * m ** 2 - 3. * m + 1.) + fb * (2. * m - 1.) + left
                else:
                    fx[(ic - 1) * n + m - 1] = (left * (n - m) + right * m) / n
        w = fx + wm
        f[:, 2:nlon + 2, lat - 1] = w.T
        f[:, 0:2, lat - 1] = w[nlon - 2:nlon].T
        f[:, nlon + 2:nlon + 4, lat - 1] = w[0:2].T
    return f


CASES = [(72, 36, 29, 1, 0), (144, 72, 57, 3, 0), (144, 72, 5, 3, 1), (288, 144, 3, 1, 0)]


@pytest.mark.parametrize("nlon,nlat,nk,order,poly", CASES)
def test_oracle_matches_transcription(pkg, orc, nlon, nlat, nk, order, poly):
    f = pkg.synth.ring_field(nk, nlon, nlat, 7 + nlon + order)
    chunks = pkg.synth.RING_CHUNKS[(nlon, nlat)]
    dl = 2.0 * (4.0 * math.atan(1.0)) / nlon
    got = orc.ringfilter(f, order, poly, chunks, dl)
    want = ringfilter_numpy(f, order, poly, chunks, dl)
    assert np.array_equal(got, want)
    # polar rows change, the rows between the filtered bands do not
    nf = len(chunks)
    assert not np.array_equal(got[:, :, 0], f[:, :, 0])
    if nlat > 2 * nf:
        assert np.array_equal(got[:, :, nf:nlat - nf], f[:, :, nf:nlat - nf])


def test_oracle_filter_removes_grid_noise_and_keeps_the_mean(pkg, orc):
    """With one chunk per grid point the linear reconstruction only
    redistributes within the chunk ring: each filtered row keeps its zonal
    mean, and the first filtered row loses most of its grid-scale noise."""
    nlon, nlat, nk = 144, 72, 4
    f = pkg.synth.ring_field(nk, nlon, nlat, 3)
    chunks = pkg.synth.RING_CHUNKS[(nlon, nlat)]
    g = orc.ringfilter(f, 1, 0, chunks, 2 * math.pi / nlon)
    for lat in (0, 5, nlat - 1):
        assert np.allclose(g[:, 2:nlon + 2, lat].mean(axis=1), f[:, 2:nlon + 2, lat].mean(axis=1), rtol=1e-13)
    rough = lambda x: np.abs(np.diff(x[:, 2:nlon + 2, 0], axis=1)).mean()  # noqa: E731
    assert rough(g) < 0.5 * rough(f)


def test_oracle_rejects_order_at_nlon(pkg, orc):
    f = pkg.synth.ring_field(2, 72, 36, 1)
    with pytest.raises(ValueError):
        orc.ringfilter(f, 72, 0, pkg.synth.RING_CHUNKS[(72, 36)], 2 * math.pi / 72)


@pytest.mark.gpu
@pytest.mark.parametrize("nlon,nlat,nk,order,poly", CASES + [(576, 288, 113, 1, 0), (576, 288, 7, 3, 1)])
def test_ringfilter_host_bit_exact(cuda, pkg, orc, nlon, nlat, nk, order, poly):
    f = pkg.synth.ring_field(nk, nlon, nlat, 11 + nlon + order)
    chunks = pkg.synth.RING_CHUNKS[(nlon, nlat)]
    dl = 2.0 * (4.0 * math.atan(1.0)) / nlon
    want = orc.ringfilter(f, order, poly, chunks, dl)
    got = f.copy(order="F")
    if order == 1 and not poly:
        pkg.filter_o2o(got, chunks, dl)
    else:
        pkg.ringfilter(got, order, poly, chunks, dl)
    assert np.array_equal(got, want)


@pytest.mark.gpu
def test_ringfilter_device_levels_and_both_orders(cuda, pkg, orc):
    """Level-major planes on the caller's stream; two orders one after the
    other (two cos/sin tables), O2, O and He as filter_o2o filters them."""
    torch = cuda
    nlon, nlat, nk = 144, 72, 57
    chunks = pkg.synth.RING_CHUNKS[(nlon, nlat)]
    dl = 2.0 * (4.0 * math.atan(1.0)) / nlon
    ncol = (nlon + 4) * nlat
    ld = pkg.batch.pad_ld(ncol)
    for order, poly, seed in ((1, 0, 1), (3, 0, 2), (1, 0, 3), (3, 1, 4)):
        f = pkg.synth.ring_field(nk, nlon, nlat, seed)
        t = pkg.batch.level_scalar(f.reshape(nk, ncol, order="F"), ld, "cuda")
        stream = torch.cuda.Stream()
        pkg.ringfilter_dev(t, nk, nlon, nlat, order, poly, chunks, dl, ld, stream=stream)
        stream.synchronize()
        got = pkg.batch.from_level_scalar(t, ncol).reshape(nk, nlon + 4, nlat, order="F")
        assert np.array_equal(got, orc.ringfilter(f, order, poly, chunks, dl))


def test_ringfilter_rejects_bad_arguments(pkg):
    f = np.zeros((3, 76, 36), order="F")
    ch = pkg.synth.RING_CHUNKS[(72, 36)]
    with pytest.raises(pkg.TgError):
        pkg.ringfilter(f, 72, 0, ch, 0.1)            # order >= nlon: the reference shuts down
    with pytest.raises(pkg.TgError):
        pkg.ringfilter(f, 16, 0, ch, 0.1)            # more modes than the kernel keeps
    with pytest.raises(pkg.TgError):
        pkg.ringfilter(f, 1, 0, (3, 2, 18), 0.1)     # fewer than 3 chunks


def test_oracle_matches_golden_pin(orc):
    """The oracle's filter of the committed field, bit for bit
    (tests/golden/pin_ringfilter.npz, made by tests/golden/make_golden.py)."""
    from conftest import golden
    g = golden("pin_ringfilter.npz")
    dl = float(g["dlamda"])
    assert np.array_equal(orc.ringfilter(g["f"], 1, 0, g["chunks"], dl), g["o1"])
    assert np.array_equal(orc.ringfilter(g["f"], 3, 0, g["chunks"], dl), g["o3"])
    assert np.array_equal(orc.ringfilter(g["f"], 3, 1, g["chunks"], dl), g["o3poly"])


@pytest.mark.gpu
def test_ringfilter_matches_golden_pin(cuda, pkg):
    from conftest import golden
    g = golden("pin_ringfilter.npz")
    dl = float(g["dlamda"])
    for key, order, poly in (("o1", 1, 0), ("o3", 3, 0), ("o3poly", 3, 1)):
        got = np.array(g["f"], order="F", copy=True)
        pkg.ringfilter(got, order, poly, g["chunks"], dl)
        assert np.array_equal(got, g[key]), key
