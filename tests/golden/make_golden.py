"""Generates the committed golden fixtures under tests/golden/.

kat_*.npz    known-answer tests: integer-valued, diagonally dominant systems
             with an integer solution x*; f = A x* is formed in exact integer
             arithmetic, so x* is the exact answer independently of any
             solver (the reference ships no golden vectors for this path).
pin_*.npz    bitwise pins of the oracle on small seeded synthetic inputs, so a
             change of the oracle's arithmetic is noticed (pin_ringfilter:
             the polar ring filter of ringfilter.F, orders 1 and 3, linear and
             polynomial reconstruction, on the 5 deg global grid).
kat_horizontal.npz  known answers of advec_ng and smooth_ng (src/advec_ng.F90,
             src/smooth_ng.F90, src/dffm_ng.F90) on a small nest: fields that
             are multiples of 3, integer winds and power-of-two
             spacings and factors keep every intermediate an exactly
             representable dyadic rational, so the answers are computed in
             exact rational arithmetic, independently of floating point.

Run from the repository root:  python tests/golden/make_golden.py [name ...]
(no names: every fixture; otherwise only the named files, e.g. kat_horizontal).
"""
from fractions import Fraction
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
import __graft_entry__ as ge  # noqa: E402


def kat_scalar(rng, nk, ncol):
    a = -rng.integers(1, 4, size=(nk, ncol)).astype(np.int64)
    c = -rng.integers(1, 4, size=(nk, ncol)).astype(np.int64)
    a[0] = 0
    c[-1] = 0
    b = -a - c + rng.integers(1, 5, size=(nk, ncol))
    x = rng.integers(-50, 51, size=(nk, ncol)).astype(np.int64)
    f = b * x
    f[1:] += a[1:] * x[:-1]
    f[:-1] += c[:-1] * x[1:]
    return {k: np.asfortranarray(v.astype(np.float64)) for k, v in dict(a=a, b=b, c=c, f=f, x=x).items()}


def kat_block(rng, B, nk, ncol):
    P = rng.integers(-2, 3, size=(B, B, nk, ncol)).astype(np.int64)
    Q = rng.integers(-2, 3, size=(B, B, nk, ncol)).astype(np.int64)
    R = rng.integers(-2, 3, size=(B, B, nk, ncol)).astype(np.int64)
    P[:, :, 0] = 0
    R[:, :, -1] = 0
    for i in range(B):
        off = np.abs(P[i]).sum(0) + np.abs(R[i]).sum(0) + np.abs(Q[i]).sum(0) - np.abs(Q[i, i])
        Q[i, i] = off + rng.integers(1, 4, size=(nk, ncol))
    u = rng.integers(-20, 21, size=(B, nk, ncol)).astype(np.int64)
    f = np.einsum("ijkc,jkc->ikc", Q, u)
    f[:, 1:] += np.einsum("ijkc,jkc->ikc", P[:, :, 1:], u[:, :-1])
    f[:, :-1] += np.einsum("ijkc,jkc->ikc", R[:, :, :-1], u[:, 1:])
    return {k: np.asfortranarray(v.astype(np.float64)) for k, v in dict(P=P, Q=Q, R=R, f=f, u=u).items()}


def _fm(v, t, n, order):
    """fm_3d along one axis in exact arithmetic; v(d) is the value d points away."""
    if t == 0 or t == n - 1:
        return v(0)
    d = 1 if (order == 2 and t in (1, n - 2)) else order
    return (v(d) + v(-d)) / 2


def _df(v, t, n, order):
    """df_3d along one axis in exact arithmetic."""
    if t == 0:
        return v(1) - v(0)
    if t == n - 1:
        return v(0) - v(-1)
    if order == 2 and t in (1, n - 2):
        return (v(1) - v(-1)) / 2
    return (v(order) - v(-order)) / (2 * order)


def kat_horizontal(rng, nk=3, nlon=7, nlat=5):
    """advec_ng and smooth_ng on a single-subdomain nest, exact answers."""
    nx, ny = nlon + 4, nlat + 4
    f = 3 * rng.integers(-40, 41, size=(nk, nx, ny))
    un = rng.integers(-9, 10, size=(nk, nx, ny))
    vn = rng.integers(-9, 10, size=(nk, nx, ny))
    racs = rng.integers(1, 16, size=ny)
    racs_q = [Fraction(int(r), 1024) for r in racs]
    dlamda, dphi, re_inv, shapiro = Fraction(1, 64), Fraction(1, 32), Fraction(1, 1024), Fraction(1, 32)
    F = lambda a: [[[Fraction(int(a[k, i, j])) for j in range(ny)] for i in range(nx)] for k in range(nk)]  # noqa: E731
    fq, uq, vq = F(f), F(un), F(vn)
    had = np.zeros((nk, nx, ny))
    fout = np.zeros((nk, nx, ny))

    def exact(x):
        y = float(x)
        assert Fraction(y) == x, "a known answer is not representable"
        return y

    for k in range(nk):
        for i in range(nx):
            for j in range(ny):
                def term(a, b, t, n, along_lon):
                    va = (lambda d: a[k][i + d][j]) if along_lon else (lambda d: a[k][i][j + d])
                    vb = (lambda d: b[k][i + d][j]) if along_lon else (lambda d: b[k][i][j + d])
                    d1, m1 = _df(va, t, n, 1), _fm(vb, t, n, 1)
                    if t <= 1 or t >= n - 2:
                        return d1 * m1
                    d2, m2 = _df(va, t, n, 2), _fm(vb, t, n, 2)
                    return d1 * 2 * 2 / 3 * m1 - d2 * 4 / 12 * m2
                wk1 = term(fq, uq, i, nx, True) * racs_q[j]
                wk2 = term(fq, vq, j, ny, False)
                had[k, i, j] = exact(wk1 / dlamda + wk2 * re_inv / dphi)
        # smooth_ng: the lat pass, then the lon pass on its result
        def shap(v, t, n):
            x = v(0)
            if t == 0 or t == n - 1:
                return x
            m1 = _fm(v, t, n, 1)
            if t in (1, n - 2):
                return x - shapiro * (-8 * m1 + 8 * x)
            return x - shapiro * (2 * _fm(v, t, n, 2) - 8 * m1 + 6 * x)
        tmp = [[shap(lambda d: fq[k][i][j + d], j, ny) for j in range(ny)] for i in range(nx)]
        for i in range(nx):
            for j in range(ny):
                fout[k, i, j] = exact(shap(lambda d: tmp[i + d][j], i, nx))
    return dict(f=np.asfortranarray(f.astype(np.float64)), un=np.asfortranarray(un.astype(np.float64)),
                vn=np.asfortranarray(vn.astype(np.float64)), racs=racs.astype(np.float64) / 1024,
                dlamda=float(dlamda), dphi=float(dphi), re_inv=float(re_inv), shapiro=float(shapiro),
                hadvec=np.asfortranarray(had), fout=np.asfortranarray(fout))


def pin_ringfilter():
    orc = ge.load_oracle()
    pkg = ge.load_package()
    f = pkg.synth.ring_field(2, 72, 36, pkg.synth.SEED_BASE + 7)
    chunks = np.asarray(pkg.synth.RING_CHUNKS[(72, 36)], dtype=np.int32)
    dl = 2.0 * (4.0 * np.arctan(1.0)) / 72
    return dict(f=f, chunks=chunks, dlamda=np.float64(dl), o1=orc.ringfilter(f, 1, 0, chunks, dl),
                o3=orc.ringfilter(f, 3, 0, chunks, dl), o3poly=orc.ringfilter(f, 3, 1, chunks, dl))


def main(names=()):
    if names:
        if "kat_horizontal" in names:
            np.savez_compressed(os.path.join(HERE, "kat_horizontal.npz"),
                                **kat_horizontal(np.random.default_rng(20261204)))
        if "pin_ringfilter" in names:
            np.savez_compressed(os.path.join(HERE, "pin_ringfilter.npz"), **pin_ringfilter())
        return
    np.savez_compressed(os.path.join(HERE, "pin_ringfilter.npz"), **pin_ringfilter())
    np.savez_compressed(os.path.join(HERE, "kat_horizontal.npz"), **kat_horizontal(np.random.default_rng(20261204)))
    rng = np.random.default_rng(20261203)
    out = {}
    for nk in (2, 3, 5, 29, 57):
        for k, v in kat_scalar(rng, nk, 33).items():
            out[f"nk{nk}_{k}"] = v
    np.savez_compressed(os.path.join(HERE, "kat_scalar.npz"), **out)
    for B in (2, 3):
        out = {}
        for nk in (2, 3, 29):
            for k, v in kat_block(rng, B, nk, 17).items():
                out[f"nk{nk}_{k}"] = v
        np.savez_compressed(os.path.join(HERE, f"kat_block{B}.npz"), **out)

    orc = ge.load_oracle()
    pkg = ge.load_package()
    a, b, c, f = pkg.synth.scalar_system(29, 64, 0.5, pkg.synth.SEED_BASE)
    np.savez_compressed(os.path.join(HERE, "pin_trsolv_ng_29.npz"), a=a, b=b, c=c, f=f,
                        x_nk=orc.trsolv_ng(a, b, c, f, 29), x_k2=orc.trsolv_ng(a, b, c, f, 28))
    P, Q, R, g = pkg.synth.block_system(3, 57, 16, 0.25, pkg.synth.SEED_BASE + 3)
    ratio = np.asfortranarray(np.random.default_rng(3).uniform(0.5, 1.5, (3, 16)))
    add = np.asfortranarray(np.random.default_rng(4).uniform(-1e-3, 1e-3, (3, 16)))
    np.savez_compressed(os.path.join(HERE, "pin_block3_57.npz"), P=P, Q=Q, R=R, f=g, ratio=ratio, add=add,
                        u=orc.blksolve(P, Q, R, g, 56, ubc_ratio=ratio, ubc_add=add))
    P, Q, R, g = pkg.synth.block_system(2, 29, 16, 0.5, pkg.synth.SEED_BASE + 2)
    np.savez_compressed(os.path.join(HERE, "pin_block2_29.npz"), P=P, Q=Q, R=R, f=g,
                        u=orc.blksolve(P, Q, R, g, 29))


if __name__ == "__main__":
    main(tuple(sys.argv[1:]))
