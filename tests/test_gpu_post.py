"""The post-solve steps of dt_ng, minor_ng and oplus_ng (lateral-boundary
overwrite, time filter, floors: src/dt_ng.F90:201-213,
src/minor_ng.F90:226-237, src/oplus_ng.F90:330-340) fused into the solve's
back sweep give, bit for bit, what the separate steps give: the device solve,
the caller's overwrite of the flagged columns, then tg_time_filter_ng_dev."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _level(pkg, torch, F, nk, ncol, one_d):
    ld = pkg.batch.pad_ld(ncol)
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
