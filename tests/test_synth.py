"""Synthetic workloads: shapes, sizes and the value laws of the benchmark
configurations."""
import numpy as np
import pytest


def test_nest_geometry(pkg):
    wl = pkg.synth.workload(3)
    dims = [(g.nlon, g.nlat, g.ncol, g.nsub) for g in wl.grids]
    assert dims == [(144, 72, 10368, 1), (97, 65, 101 * 69, 4), (65, 49, 69 * 53, 32), (52, 33, 56 * 37, 512)]
    interior = sum(g.nlon * g.nlat * g.nsub for g in wl.grids)
    assert interior == 1016100
    assert sum(g.ncol * g.nsub for g in wl.grids) == 1216132


def test_unknowns_and_bytes(pkg):
    wl = pkg.synth.workload(1)
    assert wl.unknowns_per_step() == 10368 * 513
    assert abs(wl.bytes_per_step() / 1e9 - 0.241) < 0.002
    wl3 = pkg.synth.workload(1)
    wl3.block = 3
    assert wl3.unknowns_per_step() == 10368 * 570
    assert abs(wl3.bytes_per_step() / 1e9 - 0.321) < 0.002
    assert pkg.synth.workload(0).unknowns_per_step() == 75168
    w2 = pkg.synth.workload(2)
    assert w2.grids[0].ncol == 41472 and w2.grids[0].nk == 113


def test_scalar_law(pkg):
    a, b, c, f = pkg.synth.scalar_system(29, 100, 0.5, 1)
    assert a.flags.f_contiguous and a.shape == (29, 100)
    assert np.all(a[0] == 0) and np.all(c[0] == 0) and np.all(b[0] == 1)
    assert np.all(a[-1] == -1) and np.all(b[-1] == 1) and np.all(c[-1] == 0) and np.all(f[-1] == 0)
    inner = slice(1, -1)
    assert np.all(np.abs(b[inner]) - np.abs(a[inner]) - np.abs(c[inner]) >= 1 / 60 - 1e-12)
    a2, *_ = pkg.synth.scalar_system(29, 100, 0.5, 1)
    assert np.array_equal(a, a2)


@pytest.mark.parametrize("B", [2, 3])
def test_block_law_dominance(pkg, B):
    P, Q, R, f = pkg.synth.block_system(B, 57, 50, 0.25, 4)
    for k in range(1, 56):
        for i in range(B):
            off = np.abs(P[i, :, k]).sum(0) + np.abs(R[i, :, k]).sum(0) + np.abs(Q[i, :, k]).sum(0) - np.abs(Q[i, i, k])
            assert np.all(np.abs(Q[i, i, k]) - off > 0)
