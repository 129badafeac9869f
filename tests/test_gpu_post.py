"""The post-solve steps of dt_ng, minor_ng and oplus_ng (lateral-boundary
overwrite, time filter, floors: src/dt_ng.F90:201-213,
src/minor_ng.F90:226-237, src/oplus_ng.F90:330-340) fused into the solve's
back sweep give, bit for bit, what the separate steps give: the device solve,
the caller's overwrite of the flagged columns, then tg_time_filter_ng_dev."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _level(pkg, torch, F, nk, ncol, one_d, ld=None):
    ld = pkg.batch.pad_ld(ncol) if ld is None else ld
    dev = {}
    for k, v in F.items():
        if k == "fs":
            continue
        if v.ndim == 2:
            dev[k] = pkg.batch.level_scalar(v, ld, "cuda")
        elif k in one_d:
            dev[k] = torch.from_numpy(np.ascontiguousarray(v)).cuda()
        else:
            t = torch.zeros(ld, dtype=torch.float64, device="cuda")
            t[:ncol] = torch.from_numpy(v)
            dev[k] = t
    return dev, ld


def _post_inputs(torch, cur, nk, ncol, ld, seed, lo, hi, alias):
    g = torch.Generator(device="cuda").manual_seed(seed)
    prev = cur * (1.0 + 0.05 * (torch.rand((nk, ld), dtype=torch.float64, device="cuda", generator=g) - 0.5))
    bnd = torch.rand((nk, ld), dtype=torch.float64, device="cuda", generator=g) * (hi - lo) + lo
    # the ghost ring of a nest held as one subdomain, plus scattered columns
    mask = torch.zeros(ld, dtype=torch.uint8, device="cuda")
    mask[:ncol:7] = 1
    mask[:64] = 1
    nm = prev.clone() if alias else torch.full((nk, ld), -3.0, dtype=torch.float64, device="cuda")
    return prev, bnd, mask, nm


def _separate(pkg, torch, which, x, cur, prev, bnd, mask, ds, ds2, nk, ncol, ld):
    m = mask.bool()
    x[:, m] = bnd[:, m]
    nm = torch.empty_like(x)
    pkg.time_filter_ng_dev(which, cur, prev, ds, ds2, x, nm, nk, ncol, ld)
    torch.cuda.synchronize()
    return x, nm


@pytest.mark.parametrize("alias", [False, True], ids=["nm_separate", "nm_is_prev"])
def test_dt_post_fused(cuda, pkg, alias):
    torch = cuda
    nk, ncol, dz = 57, 3001, 0.25
    F, C = pkg.synth.dt_inputs(nk, ncol, dz, 5)
    dev, ld = _level(pkg, torch, F, nk, ncol, ("expz", "dift"))
    cur = dev["tn"]
    prev, bnd, mask, nm = _post_inputs(torch, cur, nk, ncol, ld, 1, 50.0, 1500.0, alias)
    prev0 = prev.clone()
    ds, ds2 = 0.95, 0.025
    x = torch.zeros((nk, ld), dtype=torch.float64, device="cuda")
    pkg.dt_ng_dev(dev, C, x, nk, ncol, ld)
    want_x, want_nm = _separate(pkg, torch, pkg.TG_FILTER_DT, x, cur, prev0, bnd, mask, ds, ds2, nk, ncol, ld)
    y = torch.zeros((nk, ld), dtype=torch.float64, device="cuda")
    st = torch.zeros(1, dtype=torch.int32, device="cuda")
    post = dict(cur=cur, prev=nm if alias else prev, nm_upd=nm, bnd_mask=mask, bnd=bnd, dtsmooth=ds, dtsmooth_div2=ds2)
    pkg.dt_ng_post_dev(dev, C, y, nk, ncol, ld, post, status=st)
    torch.cuda.synchronize()
    assert int(st.item()) == pkg.TG_OK
    assert torch.equal(y[:, :ncol], want_x[:, :ncol])
    assert torch.equal(nm[:, :ncol], want_nm[:, :ncol])
    assert bool((y[:, :ncol] >= 100.0).all())


def test_minor_post_fused(cuda, pkg):
    torch = cuda
    nk, ncol, dz = 57, 2000, 0.25
    F, C = pkg.synth.minor_inputs(nk, ncol, dz, 6)
    dev, ld = _level(pkg, torch, F, nk, ncol, ("expz", "difk"))
    cur = pkg.batch.level_scalar(np.asfortranarray(np.abs(F["ftm1_smooth"])), ld, "cuda")
    prev, bnd, mask, nm = _post_inputs(torch, cur, nk, ncol, ld, 2, -1e-9, 1e-5, False)
    ds, ds2 = 0.9, 0.05
    x = torch.zeros((nk, ld), dtype=torch.float64, device="cuda")
    pkg.minor_ng_dev(dev, C, x, nk, ncol, ld)
    want_x, want_nm = _separate(pkg, torch, pkg.TG_FILTER_MINOR, x, cur, prev, bnd, mask, ds, ds2, nk, ncol, ld)
    y = torch.zeros((nk, ld), dtype=torch.float64, device="cuda")
    post = dict(cur=cur, prev=prev, nm_upd=nm, bnd_mask=mask, bnd=bnd, dtsmooth=ds, dtsmooth_div2=ds2)
    for mode in (1, 0):   # both forms of the minor solve carry the epilogue
        pkg.set_assembly_mode(mode)
        try:
            y.zero_()
            nm.fill_(-3.0)
            pkg.minor_ng_post_dev(dev, C, y, nk, ncol, ld, post)
            torch.cuda.synchronize()
        finally:
            pkg.set_assembly_mode(-1)
        assert torch.equal(y[:, :ncol], want_x[:, :ncol]), mode
        assert torch.equal(nm[:, :ncol], want_nm[:, :ncol]), mode


def test_oplus_post_fused_without_mask(cuda, pkg):
    torch = cuda
    nk, ncol, dz = 57, 1500, 0.25
    F, C = pkg.synth.oplus_inputs(nk, ncol, dz, 7)
    dev, ld = _level(pkg, torch, F, nk, ncol, ("zpint",))
    cur = dev["op"] if "op" in dev else pkg.batch.level_scalar(np.asfortranarray(F["ne"]), ld, "cuda")
    prev, bnd, mask, nm = _post_inputs(torch, cur, nk, ncol, ld, 3, 0.0, 1e6, False)
    ds, ds2 = 0.9, 0.05
    outs = [torch.zeros((nk, ld), dtype=torch.float64, device="cuda") for _ in range(3)]
    pkg.oplus_ng_dev(dev, C, outs[0], outs[1], outs[2], nk, ncol, ld)
    x = outs[0]
    nm_want = torch.empty_like(x)
    pkg.time_filter_ng_dev(pkg.TG_FILTER_OPLUS, cur, prev, ds, ds2, x, nm_want, nk, ncol, ld)
    torch.cuda.synchronize()
    y = [torch.zeros((nk, ld), dtype=torch.float64, device="cuda") for _ in range(3)]
    post = dict(cur=cur, prev=prev, nm_upd=nm, dtsmooth=ds, dtsmooth_div2=ds2)
    pkg.oplus_ng_post_dev(dev, C, y[0], y[1], y[2], nk, ncol, ld, post)
    torch.cuda.synchronize()
    assert torch.equal(y[0][:, :ncol], x[:, :ncol])
    assert torch.equal(nm[:, :ncol], nm_want[:, :ncol])
    assert torch.equal(y[1][:, :ncol], outs[1][:, :ncol])


@pytest.mark.parametrize("ncol,odd_ld", [(1500, False), (1500, True), (17000, False)],
                         ids=["tile_bulk_rows", "tile_odd_ld", "global_reads"])
def test_three_pass_gives_the_two_pass_bits(cuda, pkg, ncol, odd_ld):
    """Assembly mode 2 (rows formed one thread per level and column, then the
    recurrence alone) gives the bits of mode 1, with and without the fused
    post-solve steps, for dt_ng, minor_ng and oplus_ng: with the column tile
    in shared memory (bulk row copies, or 8-byte copies when the column stride
    leaves the rows unaligned) and on larger launches."""
    torch = cuda
    nk, dz = 57, 0.25
    lds = ncol + 5 if odd_ld else None
    cases = []
    F, C = pkg.synth.dt_inputs(nk, ncol, dz, 21)
    dev, ld = _level(pkg, torch, F, nk, ncol, ("expz", "dift"), lds)
    cases.append(("dt", dev, C, dev["tn"], pkg.dt_ng_dev, pkg.dt_ng_post_dev, 50.0, 1500.0))
    F, C = pkg.synth.minor_inputs(nk, ncol, dz, 22)
    dev, ld = _level(pkg, torch, F, nk, ncol, ("expz", "difk"), lds)
    cur = pkg.batch.level_scalar(np.asfortranarray(np.abs(F["ftm1_smooth"])), ld, "cuda")
    cases.append(("minor", dev, C, cur, pkg.minor_ng_dev, pkg.minor_ng_post_dev, -1e-9, 1e-5))
    F, C = pkg.synth.oplus_inputs(nk, ncol, dz, 23)
    dev, ld = _level(pkg, torch, F, nk, ncol, ("zpint",), lds)
    cases.append(("oplus", dev, C, dev["op"], None, None, 0.0, 1e6))
    z = lambda: torch.zeros((nk, ld), dtype=torch.float64, device="cuda")  # noqa: E731
    for name, dev, C, cur, plain, fused, lo, hi in cases:
        prev, bnd, mask, _ = _post_inputs(torch, cur, nk, ncol, ld, 9, lo, hi, False)
        got = {}
        for mode in (1, 2):
            pkg.set_assembly_mode(mode)
            try:
                st = torch.zeros(1, dtype=torch.int32, device="cuda")
                nm = torch.full((nk, ld), -3.0, dtype=torch.float64, device="cuda")
                post = dict(cur=cur, prev=prev, nm_upd=nm, bnd_mask=mask, bnd=bnd, dtsmooth=0.9, dtsmooth_div2=0.05)
                if name == "oplus":
                    a, b = [z() for _ in range(3)], [z() for _ in range(3)]
                    pkg.oplus_ng_dev(dev, C, a[0], a[1], a[2], nk, ncol, ld, status=st)
                    pkg.oplus_ng_post_dev(dev, C, b[0], b[1], b[2], nk, ncol, ld, post)
                    outs = a + b
                else:
                    a, b = z(), z()
                    plain(dev, C, a, nk, ncol, ld, status=st)
                    fused(dev, C, b, nk, ncol, ld, post)
                    outs = [a, b]
                torch.cuda.synchronize()
                assert int(st.item()) == pkg.TG_OK, (name, mode)
                got[mode] = [o[:, :ncol].clone() for o in outs] + [nm[:, :ncol].clone()]
            finally:
                pkg.set_assembly_mode(-1)
        for i, (u, v) in enumerate(zip(got[1], got[2])):
            assert torch.equal(u, v), (name, i)


@pytest.mark.parametrize("ncol,calc_helium", [(1500, 1), (1500, 0), (17000, 1)])
def test_comp_three_pass_gives_the_two_pass_bits(cuda, pkg, ncol, calc_helium):
    """comp_ng in assembly mode 2 (the 30 row planes formed level-parallel,
    then the block recurrence alone) gives mode 1's solution and system."""
    torch = cuda
    nk, dz = 57, 0.25
    F, C = pkg.synth.comp_inputs(nk, ncol, dz, 31, calc_helium=calc_helium)
    ld = pkg.batch.pad_ld(ncol)
    grid = type("G", (), dict(nk=nk, ncol=ncol, ld=ld))()
    dev = pkg.dynamics._dev_fields(F, grid, ("expz", "difk"), "cuda")
    got = {}
    for mode in (1, 2):
        pkg.set_assembly_mode(mode)
        try:
            out = torch.zeros((3, nk, ld), dtype=torch.float64, device="cuda")
            so = torch.zeros((30, nk, ld), dtype=torch.float64, device="cuda")
            st = torch.zeros(1, dtype=torch.int32, device="cuda")
            pkg.comp_ng_dev(dev, C, out, nk, ncol, ld, system_out=so, status=st)
            torch.cuda.synchronize()
            assert int(st.item()) == pkg.TG_OK
            got[mode] = (out[..., :ncol].clone(), so[:, :nk - 1, :ncol].clone())
        finally:
            pkg.set_assembly_mode(-1)
    assert torch.equal(got[1][0], got[2][0])
    assert torch.equal(got[1][1], got[2][1])


@pytest.mark.parametrize("ncol,odd_ld", [(1500, False), (1500, True), (17000, False)],
                         ids=["tile_bulk_rows", "tile_odd_ld", "global_reads"])
def test_oplus_factor_and_solve_give_the_full_step_bits(cuda, pkg, ncol, odd_ld):
    """The O+ sub-cycle: the rows and pivots formed once, then three sub-steps
    with new explicit_h, optm1_smooth2 and op each, with and without the
    post-solve steps, give tg_oplus_ng_dev / tg_oplus_ng_post_dev's bits."""
    torch = cuda
    nk, dz = 57, 0.25
    F, C = pkg.synth.oplus_inputs(nk, ncol, dz, 41, nstep_sub=3)
    dev, ld = _level(pkg, torch, F, nk, ncol, ("zpint",), ncol + 5 if odd_ld else None)
    z = lambda: torch.zeros((nk, ld), dtype=torch.float64, device="cuda")  # noqa: E731
    factor = torch.zeros(pkg.oplus_ng_factor_doubles(nk, ld), dtype=torch.float64, device="cuda")
    x2p, x2d = z(), z()
    st = torch.zeros(1, dtype=torch.int32, device="cuda")
    pkg.oplus_ng_factor_dev(dev, C, x2p, x2d, factor, nk, ncol, ld, status=st)
    torch.cuda.synchronize()
    assert int(st.item()) == pkg.TG_OK
    g = torch.Generator(device="cuda").manual_seed(5)
    op = dev["op"]
    for sub in range(3):
        d = dict(dev, op=op)
        d["explicit_h"] = dev["explicit_h"] * (1.0 + 0.1 * torch.rand((nk, ld), dtype=torch.float64, device="cuda",
                                                                          generator=g))
        d["optm1_smooth2"] = op * (0.99 + 0.02 * torch.rand((nk, ld), dtype=torch.float64, device="cuda", generator=g))
        prev, bnd, mask, _ = _post_inputs(torch, op, nk, ncol, ld, 10 + sub, 0.0, 1e6, False)
        want = [z() for _ in range(3)]
        pkg.oplus_ng_dev(d, C, want[0], want[1], want[2], nk, ncol, ld)
        got = z()
        pkg.oplus_ng_solve_dev(d, C, factor, got, nk, ncol, ld, status=st)
        nm_w, nm_g = z(), z()
        post_w = dict(cur=op, prev=prev, nm_upd=nm_w, bnd_mask=mask, bnd=bnd, dtsmooth=0.9, dtsmooth_div2=0.05)
        post_g = dict(post_w, nm_upd=nm_g)
        want_p = [z() for _ in range(3)]
        pkg.oplus_ng_post_dev(d, C, want_p[0], want_p[1], want_p[2], nk, ncol, ld, post_w)
        got_p = z()
        pkg.oplus_ng_solve_dev(d, C, factor, got_p, nk, ncol, ld, post=post_g, status=st)
        torch.cuda.synchronize()
        assert int(st.item()) == pkg.TG_OK
        assert torch.equal(got[:, :ncol], want[0][:, :ncol]), sub
        assert torch.equal(got_p[:, :ncol], want_p[0][:, :ncol]), sub
        assert torch.equal(nm_g[:, :ncol], nm_w[:, :ncol]), sub
        assert torch.equal(x2p[:, :ncol], want[1][:, :ncol]) and torch.equal(x2d[:, :ncol], want[2][:, :ncol])
        op = got_p


@pytest.mark.parametrize("ncol,pad,et,eh", [(1500, 0, 1, 0), (1500, 5, 0, 6), (17000, 0, 1, 6)],
                         ids=["tile", "tile_odd_ld", "above_tile_limit"])
def test_settei_three_pass_gives_the_two_pass_bits(cuda, pkg, ncol, pad, et, eh):
    """settei_ng in assembly mode 2 (rows formed one thread per level and
    column, the Thomas walk alone, Te and Ti formed level-parallel) gives
    mode 1's Te, Ti, qtotal and system bit for bit."""
    torch = cuda
    nk, dz = 57, 0.25
    F, C, qt = pkg.synth.settei_inputs(nk, ncol, dz, 61, et=et, electron_heating=eh)
    ld = ncol + pad
    dev = {}
    for k, v in F.items():
        t = torch.zeros((nk, ld) if v.ndim == 2 else (ld,), dtype=torch.float64, device="cuda")
        if v.ndim == 2:
            t[:, :ncol] = torch.from_numpy(np.ascontiguousarray(v))
        else:
            t[:ncol] = torch.from_numpy(v)
        dev[k] = t
    q0 = torch.zeros((nk, ld), dtype=torch.float64, device="cuda")
    q0[:, :ncol] = torch.from_numpy(np.ascontiguousarray(qt))
    got = {}
    for mode in (1, 2):
        pkg.set_assembly_mode(mode)
        try:
            te, ti = (torch.full((nk, ld), -1.0, dtype=torch.float64, device="cuda") for _ in range(2))
            q2 = q0.clone()
            so = torch.zeros((4, nk, ld), dtype=torch.float64, device="cuda")
            st = torch.zeros(1, dtype=torch.int32, device="cuda")
            pkg.settei_ng_dev(dev, C, te, ti, q2, nk, ncol, ld, system_out=so, status=st)
            torch.cuda.synchronize()
            assert int(st.item()) == pkg.TG_OK
            got[mode] = [v[..., :ncol].clone() for v in (te, ti, q2)] + [so[:, :nk - 1, :ncol].clone()]
        finally:
            pkg.set_assembly_mode(-1)
    for i, (u, v) in enumerate(zip(got[1], got[2])):
        assert torch.equal(u, v), i
