"""Pins the CPU oracle (a restatement of src/trsolv_ng.F90, src/trsolv.F,
src/comp_ng.F90:166-332, src/duv.F:801-908, src/matutil.F90) against
independent answers: exact integer known-answer systems, closed forms, LAPACK
and a long-double restatement.  The reference itself cannot run here (no
Fortran compiler) and ships no test vectors, so these are the pins."""
import numpy as np
import pytest
import scipy.linalg as sl

from conftest import golden


def banded_solve(a, b, c, f, k2):
    n = k2
    ab = np.zeros((3, n))
    ab[0, 1:] = c[: n - 1]
    ab[1] = b[:n]
    ab[2, :-1] = a[1:n]
    return sl.solve_banded((1, 1), ab, f[:n])


def block_dense(P, Q, R, f, k2, col):
    B = f.shape[0]
    n = B * k2
    A = np.zeros((n, n))
    for k in range(k2):
        A[B * k:B * k + B, B * k:B * k + B] = Q[:, :, k, col]
        if k > 0:
            A[B * k:B * k + B, B * (k - 1):B * k] = P[:, :, k, col]
        if k < k2 - 1:
            A[B * k:B * k + B, B * (k + 1):B * (k + 2)] = R[:, :, k, col]
    return np.linalg.solve(A, f[:, :k2, col].T.reshape(-1)).reshape(k2, B).T


@pytest.mark.parametrize("nk", [2, 3, 5, 29, 57])
def test_scalar_known_answer(orc, nk):
    g = golden("kat_scalar.npz")
    a, b, c, f, xs = (g[f"nk{nk}_{k}"] for k in "abcfx")
    x = orc.trsolv_ng(a, b, c, f, nk)
    assert np.max(np.abs(x - xs)) <= 1e-13 * np.max(np.abs(xs))


@pytest.mark.parametrize("B", [2, 3])
@pytest.mark.parametrize("nk", [2, 3, 29])
def test_block_known_answer(orc, B, nk):
    g = golden(f"kat_block{B}.npz")
    P, Q, R, f, us = (g[f"nk{nk}_{k}"] for k in ("P", "Q", "R", "f", "u"))
    u = orc.blksolve(P, Q, R, f, nk)
    assert np.max(np.abs(u - us)) <= 1e-12 * np.max(np.abs(us))
    ul = orc.blksolve(P, Q, R, f, nk, long_double=True)
    assert np.max(np.abs(ul - us)) <= 1e-15 * np.max(np.abs(us))


@pytest.mark.parametrize("n", [2, 3, 17, 57, 113])
def test_scalar_laplacian_eigenvector(orc, n):
    # tridiag(-1, 2, -1) x = lambda x for x_k = sin(pi j k/(n+1)) (closed form)
    j = max(1, n // 3)
    k = np.arange(1, n + 1)
    xs = np.sin(np.pi * j * k / (n + 1))
    lam = 2.0 - 2.0 * np.cos(np.pi * j / (n + 1))
    a = np.full((n, 1), -1.0, order="F")
    c = np.full((n, 1), -1.0, order="F")
    b = np.full((n, 1), 2.0, order="F")
    f = np.asfortranarray((lam * xs)[:, None])
    x = orc.trsolv_ng(a, b, c, f, n)
    assert np.max(np.abs(x[:, 0] - xs)) <= 1e-13 * n * n


@pytest.mark.parametrize("cfg", [0, 1, 2])
def test_scalar_vs_lapack_and_long_double(orc, pkg, cfg):
    wl = pkg.synth.workload(cfg)
    gr = wl.grids[0]
    a, b, c, f = pkg.synth.scalar_system(gr.nk, 37, gr.dz, 5 + cfg, wl.d0_range, wl.loss, wl.d_span)
    x = orc.trsolv_ng(a, b, c, f, gr.nk, nthreads=2)
    xl = orc.trsolv_ng(a, b, c, f, gr.nk, long_double=True)
    for col in range(a.shape[1]):
        xs = banded_solve(a[:, col], b[:, col], c[:, col], f[:, col], gr.nk)
        assert np.max(np.abs(x[:, col] - xs)) <= 1e-12 * np.max(np.abs(xs))
    assert np.max(np.abs(x - xl)) <= 1e-12 * np.max(np.abs(xl))


@pytest.mark.parametrize("B", [2, 3])
def test_block_vs_dense(orc, pkg, B):
    P, Q, R, f = pkg.synth.block_system(B, 29, 9, 0.5, 77)
    u = orc.blksolve(P, Q, R, f, 29)
    for col in range(9):
        us = block_dense(P, Q, R, f, 29, col)
        assert np.max(np.abs(u[:, :, col] - us)) <= 1e-12 * np.max(np.abs(us))


def test_scalar_k2_leaves_rows_untouched(orc, pkg):
    a, b, c, f = pkg.synth.scalar_system(29, 11, 0.5, 3)
    x0 = np.full(a.shape, 7.25, order="F")
    x = orc.trsolv_ng(a, b, c, f, 20, x=x0)
    assert np.all(x[20:] == 7.25)
    for col in range(11):
        xs = banded_solve(a[:, col], b[:, col], c[:, col], f[:, col], 20)
        assert np.max(np.abs(x[:20, col] - xs)) <= 1e-12 * np.max(np.abs(xs))


def test_trsolv_periodic_skip(orc, pkg):
    # lon0=1 and lon1=lonmax: columns 1,2 and lonmax-1,lonmax are skipped
    nlev, lonmax = 29, 12
    a, b, c, f = pkg.synth.scalar_system(nlev, lonmax, 0.5, 9)
    x0 = np.full(a.shape, -1.0, order="F")
    x = orc.trsolv(a, b, c, f, x0, 1, nlev, 1, nlev - 1, 1, lonmax, lonmax)
    assert np.all(x[:, :2] == -1.0) and np.all(x[:, -2:] == -1.0)
    assert np.all(x[-1] == -1.0)
    ref = orc.trsolv_ng(a[:, 2:-2], b[:, 2:-2], c[:, 2:-2], f[:, 2:-2], nlev - 1)
    assert np.array_equal(x[: nlev - 1, 2:-2], ref[: nlev - 1])
    # an interior slab (lon0 > 1, lon1 < lonmax) solves every column
    x = orc.trsolv(a[:, 3:7], b[:, 3:7], c[:, 3:7], f[:, 3:7], np.zeros((nlev, 4), order="F"),
                   1, nlev, 1, nlev, 4, 7, lonmax)
    assert np.array_equal(x, orc.trsolv_ng(a[:, 3:7], b[:, 3:7], c[:, 3:7], f[:, 3:7], nlev))


def test_blktri_matches_block_solver_and_skips_periodic(orc, pkg):
    P, Q, R, f = pkg.synth.block_system(2, 29, 10, 0.5, 21)
    x0 = np.full(f.shape, 3.0, order="F")
    x = orc.blktri(P, Q, R, f, x0, 1, 29, 1, 10, 10)
    assert np.all(x[:, :, :2] == 3.0) and np.all(x[:, :, -2:] == 3.0)
    assert np.all(x[:, -1] == 3.0)
    ref = orc.blksolve(P[..., 2:-2], Q[..., 2:-2], R[..., 2:-2], f[..., 2:-2], 28)
    assert np.array_equal(x[:, :28, 2:-2], ref[:, :28])


def test_matinv(orc):
    rng = np.random.default_rng(0)
    for _ in range(20):
        A = rng.normal(size=(3, 3)) + 3 * np.eye(3)
        assert np.allclose(orc.matinv3(A), np.linalg.inv(A), rtol=1e-13, atol=1e-14)
        A2 = rng.normal(size=(2, 2)) + 3 * np.eye(2)
        assert np.allclose(orc.matinv2(A2), np.linalg.inv(A2), rtol=1e-13, atol=1e-14)


def test_block_ubc_row(orc, pkg):
    # comp_ng.F90:328-332: u(nk) = ratio*u(nk-1) + add
    P, Q, R, f = pkg.synth.block_system(3, 12, 5, 0.5, 2)
    rng = np.random.default_rng(2)
    ratio = np.asfortranarray(rng.uniform(0.5, 1.5, (3, 5)))
    add = np.asfortranarray(rng.uniform(-1, 1, (3, 5)))
    u = orc.blksolve(P, Q, R, f, 11, ubc_ratio=ratio, ubc_add=add)
    assert np.array_equal(u[:, 11], ratio * u[:, 10] + add)
    u2 = orc.blksolve(P, Q, R, f, 11, ubc_ratio=ratio)
    assert np.array_equal(u2[:, 11], ratio * u2[:, 10])


def test_oracle_bitwise_pins(orc):
    g = golden("pin_trsolv_ng_29.npz")
    assert np.array_equal(orc.trsolv_ng(g["a"], g["b"], g["c"], g["f"], 29), g["x_nk"])
    x = orc.trsolv_ng(g["a"], g["b"], g["c"], g["f"], 28)
    assert np.array_equal(x[:28], g["x_k2"][:28])
    g = golden("pin_block3_57.npz")
    u = orc.blksolve(g["P"], g["Q"], g["R"], g["f"], 56, ubc_ratio=g["ratio"], ubc_add=g["add"])
    assert np.array_equal(u, g["u"])
    g = golden("pin_block2_29.npz")
    assert np.array_equal(orc.blksolve(g["P"], g["Q"], g["R"], g["f"], 29), g["u"])


def test_zero_pivot_propagates_like_reference(orc):
    # the reference has no pivot check: b(1) = 0 yields Inf/NaN, not an error
    a = np.asfortranarray(np.full((5, 2), -1.0))
    b = np.asfortranarray(np.full((5, 2), 3.0))
    c = a.copy(order="F")
    f = np.asfortranarray(np.ones((5, 2)))
    b[0, 1] = 0.0
    x = orc.trsolv_ng(a, b, c, f, 5)
    assert np.all(np.isfinite(x[:, 0]))
    assert not np.all(np.isfinite(x[:, 1]))
