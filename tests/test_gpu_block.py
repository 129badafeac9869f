"""Block-tridiagonal solves (3x3 comp_ng O2/O/He, 2x2 blktri) on the GPU
through the C ABI, against the oracle (bit-exact in FP64)."""
import numpy as np
import pytest

from conftest import golden

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("B,nk,ncol", [(3, 57, 1500), (2, 57, 1500), (3, 113, 301), (2, 29, 2592), (3, 2, 7), (3, 3, 33)])
def test_comp_blksolve_bit_exact(cuda, pkg, orc, B, nk, ncol):
    P, Q, R, f = pkg.synth.block_system(B, nk, ncol, 14.0 / (nk - 1), 31 + nk)
    rng = np.random.default_rng(B + nk)
    ratio = np.asfortranarray(rng.uniform(0.5, 1.5, (B, ncol)))
    add = np.asfortranarray(rng.uniform(-1e-3, 1e-3, (B, ncol)))
    u = np.zeros_like(f, order="F")
    assert pkg.comp_blksolve_ng(P, Q, R, f, u, ratio, add) == pkg.TG_OK
    assert np.array_equal(u, orc.blksolve(P, Q, R, f, nk - 1, ubc_ratio=ratio, ubc_add=add))
    u2 = np.full(f.shape, 5.0, order="F")
    assert pkg.comp_blksolve_ng(P, Q, R, f, u2) == pkg.TG_OK
    ref = orc.blksolve(P, Q, R, f, nk - 1)
    assert np.array_equal(u2[:, : nk - 1], ref[:, : nk - 1])
    assert np.all(u2[:, nk - 1] == 5.0)


def test_block_golden(cuda, pkg):
    g = golden("pin_block3_57.npz")
    u = np.zeros_like(g["f"], order="F")
    pkg.comp_blksolve_ng(g["P"], g["Q"], g["R"], g["f"], u, g["ratio"], g["add"])
    assert np.array_equal(u, g["u"])
    for B in (2, 3):
        kat = golden(f"kat_block{B}.npz")
        for nk in (2, 3, 29):
            P, Q, R, f, us = (kat[f"nk{nk}_{k}"] for k in ("P", "Q", "R", "f", "u"))
            # rows 1..nk solved through the device entry (column layout)
            import torch
            t = [torch.from_numpy(np.ascontiguousarray(np.ravel(v, order="F"))).cuda() for v in (P, Q, R, f)]
            tu = torch.zeros_like(t[3])
            pkg.blksolve_dev(B, *t, tu, nk, nk, f.shape[2], layout=pkg.TG_LAYOUT_COLUMN, ld=0)
            torch.cuda.synchronize()
            u = tu.cpu().numpy().reshape(f.shape, order="F")
            assert np.max(np.abs(u - us)) <= 1e-12 * np.max(np.abs(us))


@pytest.mark.parametrize("lon0,lon1", [(1, 40), (3, 30), (5, 40)])
def test_blktri_slab(cuda, pkg, orc, lon0, lon1):
    nlonp4, nlev = 40, 29
    ncol = lon1 - lon0 + 1
    P, Q, R, f = pkg.synth.block_system(2, nlev, ncol, 0.5, lon0)
    x = np.full(f.shape, 2.0, order="F")
    assert pkg.blktri(P, Q, R, f, None, None, None, x, 1, nlev, lon0, lon1, nlonp4) == pkg.TG_OK
    ref = orc.blktri(P, Q, R, f, np.full(f.shape, 2.0, order="F"), 1, nlev, lon0, lon1, nlonp4)
    assert np.array_equal(x, ref)


@pytest.mark.parametrize("B", [2, 3])
def test_block_level_layout_and_refine(cuda, pkg, orc, B):
    torch = cuda
    nk, ncol, ld = 57, 1200, 1216
    P, Q, R, f = pkg.synth.block_system(B, nk, ncol, 0.25, 90 + B)
    ref = orc.blksolve(P, Q, R, f, nk)
    tP, tQ, tR = (pkg.batch.level_matrix(v, ld, "cuda") for v in (P, Q, R))
    tf = pkg.batch.level_vector(f, ld, "cuda")
    for prec in (pkg.TG_PREC_F64, pkg.TG_PREC_F32_REFINE):
        tu = torch.zeros_like(tf)
        st = torch.zeros(1, dtype=torch.int32, device="cuda")
        pkg.blksolve_dev(B, tP, tQ, tR, tf, tu, nk, nk, ncol, layout=pkg.TG_LAYOUT_LEVEL, ld=ld, precision=prec,
                         status=st)
        torch.cuda.synchronize()
        u = pkg.batch.from_level_vector(tu, ncol)
        if prec == pkg.TG_PREC_F64:
            assert np.array_equal(u, ref)
            assert int(st.item()) == pkg.TG_OK
        else:
            assert np.max(np.abs(u - ref)) / np.max(np.abs(ref)) <= 1e-10
            assert int(st.item()) in (pkg.TG_OK, pkg.TG_ENOCONV)


def test_singular_block_flagged(cuda, pkg, orc):
    P, Q, R, f = pkg.synth.block_system(3, 12, 40, 0.5, 5)
    Q = Q.copy(order="F")
    Q[:, :, 0, 7] = 0.0   # the first row's pivot block is Q itself
    u = np.zeros_like(f, order="F")
    assert pkg.comp_blksolve_ng(P, Q, R, f, u) == pkg.TG_EPIVOT
    assert np.array_equal(u[:, :11], orc.blksolve(P, Q, R, f, 11)[:, :11], equal_nan=True)


def test_solve_host_mixed_batch(cuda, pkg, orc):
    """tg_solve_host: scalar and block systems of one stage in one pipelined call."""
    systems, refs = [], []
    for i, (nk, ncol) in enumerate(((57, 10368), (57, 3001), (29, 777))):
        a, b, c, f = pkg.synth.scalar_system(nk, ncol, 14.0 / (nk - 1), 500 + i)
        x = np.zeros_like(a, order="F")
        systems.append(dict(kind=pkg.TG_KIND_SCALAR, a=a, b=b, c=c, f=f, x=x, k2=nk - (i % 2)))
        refs.append(orc.trsolv_ng(a, b, c, f, nk - (i % 2)))
    for B in (2, 3):
        P, Q, R, f = pkg.synth.block_system(B, 57, 2000, 0.25, 600 + B)
        ratio = np.asfortranarray(np.random.default_rng(B).uniform(0.5, 1.5, (B, 2000)))
        u = np.zeros_like(f, order="F")
        systems.append(dict(kind=B, a=P, b=Q, c=R, f=f, x=u, k2=56, ubc_ratio=ratio))
        refs.append(orc.blksolve(P, Q, R, f, 56, ubc_ratio=ratio))
    assert pkg.solve_host(systems) == pkg.TG_OK
    for q, ref in zip(systems, refs):
        k2 = q["k2"]
        if q["kind"] == pkg.TG_KIND_SCALAR:
            assert np.array_equal(q["x"][:k2], ref[:k2])
        else:
            assert np.array_equal(q["x"][:, :k2 + 1], ref[:, :k2 + 1])


@pytest.mark.parametrize("chunk_kb,streams", [(1024, 1), (4096, 3), (65536, 8)])
def test_solve_host_chunking_keeps_bits(cuda, pkg, orc, chunk_kb, streams):
    """Any column-chunk size and stream count of the host pipeline gives the
    oracle's bits (the chunks are independent column batches)."""
    systems, refs = [], []
    for i, (nk, ncol) in enumerate(((57, 5000), (29, 777))):
        a, b, c, f = pkg.synth.scalar_system(nk, ncol, 14.0 / (nk - 1), 700 + i)
        x = np.zeros_like(a, order="F")
        systems.append(dict(kind=pkg.TG_KIND_SCALAR, a=a, b=b, c=c, f=f, x=x, k2=nk))
        refs.append(orc.trsolv_ng(a, b, c, f, nk))
    P, Q, R, f = pkg.synth.block_system(2, 57, 1500, 0.25, 702)
    u = np.zeros_like(f, order="F")
    systems.append(dict(kind=2, a=P, b=Q, c=R, f=f, x=u, k2=57))
    refs.append(orc.blksolve(P, Q, R, f, 57))
    pkg.set_host_pipeline(chunk_kb, streams)
    try:
        assert pkg.solve_host(systems) == pkg.TG_OK
    finally:
        pkg.set_host_pipeline(0, 0)
    for q, ref in zip(systems, refs):
        assert np.array_equal(q["x"], ref)


@pytest.mark.parametrize("chunk_kb,streams", [(0, 0), (1024, 2)])
def test_solve_host_arena_keeps_bits(cuda, pkg, orc, chunk_kb, streams):
    """Systems whose arrays lie side by side in one page-locked arena (the
    input copies of consecutive chunks then merge into one per run), with
    small gaps and one system outside the arena, give the oracle's bits."""
    torch = cuda
    shapes = [(57, 2072), (57, 2072), (29, 777), (57, 3001)]
    nbytes = sum(5 * nk * ncol * 8 + 5 * 64 for nk, ncol in shapes) + 4096
    arena = torch.empty(nbytes, dtype=torch.uint8, pin_memory=True).numpy()
    off = 0
    systems, refs = [], []

    def take(shape):
        nonlocal off
        v = np.ndarray(shape, dtype=np.float64, buffer=arena, offset=off, order="F")
        off += int(np.prod(shape)) * 8 + 64          # a 64-byte gap after every array
        return v

    for i, (nk, ncol) in enumerate(shapes):
        a, b, c, f = pkg.synth.scalar_system(nk, ncol, 14.0 / (nk - 1), 800 + i)
        if i == 3:            # outside the arena: separate host arrays
            arrs = [a, b, c, f, np.zeros_like(a, order="F")]
        else:
            arrs = [take((nk, ncol)) for _ in range(5)]
            for v, w in zip(arrs, (a, b, c, f)):
                np.copyto(v, w)
            arrs[4][...] = 0.0
        systems.append(dict(kind=pkg.TG_KIND_SCALAR, a=arrs[0], b=arrs[1], c=arrs[2], f=arrs[3], x=arrs[4],
                            k2=nk - (i % 2)))
        refs.append(orc.trsolv_ng(a, b, c, f, nk - (i % 2)))
    pkg.set_host_pipeline(chunk_kb, streams)
    try:
        assert pkg.solve_host(systems) == pkg.TG_OK
    finally:
        pkg.set_host_pipeline(0, 0)
    for q, ref in zip(systems, refs):
        k2 = q["k2"]
        assert np.array_equal(q["x"][:k2], ref[:k2])


@pytest.mark.parametrize("chunk_kb,streams", [(0, 0), (1024, 2), (300, 3)])
def test_solve_host_arena_strided_copies_keep_bits(cuda, pkg, orc, chunk_kb, streams):
    """Systems of one shape side by side in a page-locked arena, each followed
    by its solution array (their inputs cross the link as strided copies
    that skip the solutions), scalar and 2x2 block, give the oracle's bits;
    the solution arrays between the inputs are left as the solve wrote them."""
    torch = cuda
    nk, ncol, B = 57, 1000, 2
    shapes = [("s", (nk, ncol))] * 6 + [("b", None)] * 3
    blk = [(B, B, nk, ncol)] * 3 + [(B, nk, ncol)] * 2
    nbytes = sum(5 * nk * ncol * 8 + 5 * 256 for _ in range(6)) + 3 * sum(int(np.prod(s)) * 8 + 256 for s in blk)
    arena = torch.empty(nbytes + 4096, dtype=torch.uint8, pin_memory=True).numpy()
    off = 0

    def take(shape):
        nonlocal off
        v = np.ndarray(shape, dtype=np.float64, buffer=arena, offset=off, order="F")
        off += (int(np.prod(shape)) * 8 + 255) // 256 * 256
        return v

    systems, refs = [], []
    for i, (kind, shp) in enumerate(shapes):
        if kind == "s":
            src = pkg.synth.scalar_system(nk, ncol, 0.25, 900 + i)
            arrs = [take(shp) for _ in range(5)]
        else:
            src = pkg.synth.block_system(B, nk, ncol, 0.25, 900 + i)
            arrs = [take(s) for s in blk]
        for v, w in zip(arrs, src):
            np.copyto(v, w)
        arrs[4][...] = np.nan        # the solve overwrites every solution value
        if kind == "s":
            systems.append(dict(kind=pkg.TG_KIND_SCALAR, a=arrs[0], b=arrs[1], c=arrs[2], f=arrs[3], x=arrs[4],
                                k2=nk))
            refs.append(orc.trsolv_ng(*src, nk))
        else:
            systems.append(dict(kind=B, a=arrs[0], b=arrs[1], c=arrs[2], f=arrs[3], x=arrs[4], k2=nk))
            refs.append(orc.blksolve(*src, nk))
    pkg.set_host_pipeline(chunk_kb, streams)
    try:
        assert pkg.solve_host(systems) == pkg.TG_OK
    finally:
        pkg.set_host_pipeline(0, 0)
    for q, ref in zip(systems, refs):
        assert np.array_equal(q["x"], ref)
