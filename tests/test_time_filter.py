"""Post-solve time filter and floor of dt_ng (src/dt_ng.F90:208-213), minor_ng
(src/minor_ng.F90:234-237) and oplus_ng (src/oplus_ng.F90:337-340): the
oracle against an independent numpy transcription, and the CUDA entries
(host and device forms) against the oracle, bit for bit."""
import numpy as np
import pytest

# dtsmooth of the reference's time filter and dtsmooth_div2 = (1 - dtsmooth)/2
DTSMOOTH = 0.95
DTSMOOTH_DIV2 = 0.5 * (1.0 - DTSMOOTH)
FLOORS = {0: 100.0, 1: 1.e-12, 2: 0.0}
SCALE = {0: 800.0, 1: 1.e-9, 2: 1.e5}  # Tn in K, minor mixing ratio, O+ in cm^-3


def inputs(which, nk, ncol, seed):
    """Seeded fields around the routine's typical magnitude, with values
    below, at and above the floor and the IEEE special cases the floor meets."""
    rng = np.random.default_rng(seed)
    s = SCALE[which]
    cur = np.asfortranarray(s * rng.uniform(0.05, 2.0, (nk, ncol)))
    prev = np.asfortranarray(cur * rng.uniform(0.9, 1.1, (nk, ncol)))
    upd = np.asfortranarray(cur * rng.uniform(0.8, 1.2, (nk, ncol)))
    fl = FLOORS[which]
    flat = upd.reshape(-1, order="F")
    n = flat.size
    specials = [fl, -fl, 0.0, -0.0, np.nan, np.inf, -np.inf, 5e-324, -5e-324, np.nextafter(fl, np.inf),
                np.nextafter(fl, -np.inf), -1.0, -s]
    idx = rng.choice(n, size=min(n, 8 * len(specials)), replace=False)
    for j, i in enumerate(idx):
        flat[i] = specials[j % len(specials)]
    # a filtered value that lands below the floor
    if n > len(idx):
        k = int(rng.integers(0, n))
        prev.reshape(-1, order="F")[k] = -3.0 * s
    return cur, prev, upd


def numpy_filter(which, cur, prev, upd):
    fl = FLOORS[which]
    if which == 0:
        nm = DTSMOOTH_DIV2 * (prev + upd) + DTSMOOTH * cur
    else:
        nm = DTSMOOTH * cur + DTSMOOTH_DIV2 * (prev + upd)
    u = np.where(upd > fl, upd, fl)
    if which != 0:
        nm = np.where(nm > fl, nm, fl)
    return u, nm


def same_bits(a, b):
    return np.array_equal(np.asarray(a).view(np.int64), np.asarray(b).view(np.int64))


@pytest.mark.parametrize("which", [0, 1, 2])
@pytest.mark.parametrize("nk,ncol", [(57, 300), (29, 64), (1, 1)])
def test_oracle_matches_numpy_transcription(orc, which, nk, ncol):
    cur, prev, upd = inputs(which, nk, ncol, 11 + which + nk)
    got_u, got_nm = orc.time_filter_ng(which, cur, prev, upd, DTSMOOTH, DTSMOOTH_DIV2)
    want_u, want_nm = numpy_filter(which, cur, prev, upd)
    with np.errstate(invalid="ignore"):
        assert same_bits(got_u, want_u)
        assert same_bits(got_nm, want_nm)


def test_oracle_floor_semantics(orc):
    """NaN and -0.0 go to the floor (x > floor is false for both); the dt
    filter leaves the filtered field unfloored."""
    cur = np.zeros((3, 1), order="F")
    prev = np.zeros((3, 1), order="F")
    upd = np.asfortranarray([[np.nan], [-0.0], [50.0]])
    u, nm = orc.time_filter_ng(2, cur, prev, upd, DTSMOOTH, DTSMOOTH_DIV2)
    assert same_bits(u[:, 0], np.array([0.0, 0.0, 50.0]))
    assert same_bits(nm[:, 0], np.array([0.0, 0.0, DTSMOOTH_DIV2 * 50.0]))
    u, nm = orc.time_filter_ng(0, cur, prev, upd, DTSMOOTH, DTSMOOTH_DIV2)
    assert same_bits(u[:, 0], np.array([100.0, 100.0, 100.0]))
    assert np.isnan(nm[0, 0]) and same_bits(nm[1:, 0], np.array([0.0, DTSMOOTH_DIV2 * 50.0]))


@pytest.mark.gpu
@pytest.mark.parametrize("which", [0, 1, 2])
@pytest.mark.parametrize("nk,ncol", [(57, 3001), (29, 2592), (113, 7), (1, 1)])
def test_time_filter_host_bit_exact(cuda, pkg, orc, which, nk, ncol):
    cur, prev, upd = inputs(which, nk, ncol, 5 + which + nk)
    want_u, want_nm = orc.time_filter_ng(which, cur, prev, upd, DTSMOOTH, DTSMOOTH_DIV2)
    u = upd.copy(order="F")
    nm = np.zeros_like(u, order="F")
    assert pkg.time_filter_ng(which, cur, prev, DTSMOOTH, DTSMOOTH_DIV2, u, nm) == pkg.TG_OK
    assert same_bits(u, want_u)
    assert same_bits(nm, want_nm)


@pytest.mark.gpu
@pytest.mark.parametrize("which", [0, 1, 2])
def test_time_filter_device_level_major_in_place(cuda, pkg, orc, which):
    """Level-major (nk, ld) device fields; the filtered field overwrites prev
    in place and the padding past ncol is left untouched."""
    torch = cuda
    nk, ncol = 57, 1000
    ld = pkg.batch.pad_ld(ncol)
    cur, prev, upd = inputs(which, nk, ncol, 40 + which)
    want_u, want_nm = orc.time_filter_ng(which, cur, prev, upd, DTSMOOTH, DTSMOOTH_DIV2)

    def dev(a):
        t = torch.full((nk, ld), 7.25, dtype=torch.float64, device="cuda")
        t[:, :ncol] = torch.from_numpy(np.ascontiguousarray(a))
        return t

    c, p, u = dev(cur), dev(prev), dev(upd)
    assert pkg.time_filter_ng_dev(which, c, p, DTSMOOTH, DTSMOOTH_DIV2, u, p, nk, ncol, ld) == pkg.TG_OK
    torch.cuda.synchronize()
    assert same_bits(u[:, :ncol].cpu().numpy(), want_u)
    assert same_bits(p[:, :ncol].cpu().numpy(), want_nm)
    assert bool((u[:, ncol:] == 7.25).all()) and bool((p[:, ncol:] == 7.25).all())


def test_time_filter_rejects_bad_arguments(pkg):
    """Argument checks run before any device call, so they hold without a GPU."""
    a = np.zeros((3, 4), order="F")
    b = np.zeros((3, 4), order="F")
    c = np.zeros((3, 4), order="F")
    for which, cur, upd, nm in ((3, a, b, c), (-1, a, b, c), (0, a, b, b), (1, b, b, c)):
        with pytest.raises(pkg.TgError) as e:
            pkg.time_filter_ng(which, cur, a, DTSMOOTH, DTSMOOTH_DIV2, upd, nm)
        assert e.value.status == pkg.TG_EINVAL
    L = pkg.colsolve.lib()
    assert L.tg_time_filter_ng_dev(0, 8, 8, DTSMOOTH, DTSMOOTH_DIV2, 70000, 4, 4, 16, 24, None) == pkg.TG_EINVAL
    assert L.tg_time_filter_ng_dev(0, 8, 8, DTSMOOTH, DTSMOOTH_DIV2, 3, 4, 2, 16, 24, None) == pkg.TG_EINVAL
