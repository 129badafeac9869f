"""Generates the committed golden fixtures under tests/golden/.

kat_*.npz    known-answer tests: integer-valued, diagonally dominant systems
             with an integer solution x*; f = A x* is formed in exact integer
             arithmetic, so x* is the exact answer independently of any
             solver (the reference ships no golden vectors for this path).
pin_*.npz    bitwise pins of the oracle on small seeded synthetic inputs, so a
             change of the oracle's arithmetic is noticed.

Run from the repository root:  python tests/golden/make_golden.py
"""
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


def main():
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
    main()
