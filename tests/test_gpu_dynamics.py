"""One dynamics_ng step of column routines on the device (the package's
DynamicsStep: horizontal inputs, fused assembly + solve + post-solve steps,
the O+ sub-cycle, settei_ng's qtotal feeding dt_ng, the ring filter on the
global grid) against the same sequence of oracle routines on the CPU; and
the device entries on several streams at once."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

# Relative error (max |gpu - oracle| / max |oracle|) allowed per result.  The
# routines' own tests hold: dt_ng, advec_ng, smooth_ng, comp_ng's post steps
# and the ring filter bit-exact or to 1e-15; minor_ng 3e-13; comp_ng 1e-12;
# settei_ng 5e-14 (device exp/log/pow); oplus_ng 2e-11 per sub-step.  In the
# step dt_ng reads settei_ng's qtotal, and each O+ sub-step reads the last.
TOL = {"tn_upd": 1e-12, "tn_nm_upd": 1e-12, "te": 5e-14, "ti": 5e-14, "qtotal": 5e-14,
       "op": 1e-10, "optm1": 1e-10, "xiop2p": 1e-10, "xiop2d": 1e-10,
       "o2_upd": 1e-12, "o1_upd": 1e-12, "he_upd": 1e-12, "o2nm_upd": 1e-12, "o1nm_upd": 1e-12, "henm_upd": 1e-12}
MINOR_TOL = 1e-12


def _rel(got, want):
    want = np.asarray(want)
    m = np.abs(want).max()
    return float(np.abs(got - want).max() / (m if m > 0 else 1.0))


def _compare(pkg, step, want, ncol):
    errs = {}
    for name, t in step.outputs().items():
        got = pkg.batch.from_level_scalar(t, ncol)
        assert np.all(np.isfinite(got)), name
        errs[name] = _rel(got, want[name])
    for name, e in errs.items():
        tol = TOL.get(name, MINOR_TOL)
        assert e <= tol, (name, e, tol, errs)
    return errs


@pytest.mark.parametrize("mode", ["serial", "fan_out", "graph"])
def test_dynamics_step_matches_oracle(cuda, pkg, orc, mode):
    torch = cuda
    dyn = pkg.dynamics
    grid = dyn.Grid(57, 20, 12, 0.25, lat0_deg=20.0, dlat_deg=2.5)
    h = dyn.synthetic_inputs(grid, 5, nstep_sub=4)
    want = dyn.host_step(orc, grid, h)
    step = dyn.DynamicsStep(grid, h, fan_out=(mode != "serial"))
    st = torch.cuda.Stream()
    if mode == "graph":
        step.capture(st)
        st.synchronize()
        for o in step.outputs().values():
            o.fill_(-1.0)
        torch.cuda.synchronize()
        step.replay(st)
    else:
        step.issue(st)
    st.synchronize()
    _compare(pkg, step, want, grid.ncol)


def test_dynamics_step_global_grid_with_ring_filter(cuda, pkg, orc):
    """The 5-degree global grid (72 x 36): filter_o2o between comp_ng's solve
    and its post-solve steps, repeated graph replays giving the same bits."""
    torch = cuda
    dyn = pkg.dynamics
    grid = dyn.Grid(29, 72, 36, 0.5)
    ring = pkg.synth.RING_CHUNKS[(72, 36)]
    h = dyn.synthetic_inputs(grid, 11, nstep_sub=2)
    want = dyn.host_step(orc, grid, h, ring=ring)
    step = dyn.DynamicsStep(grid, h, ring=ring)
    st = torch.cuda.Stream()
    step.capture(st)
    step.replay(st)
    st.synchronize()
    first = {k: v.clone() for k, v in step.outputs().items()}
    _compare(pkg, step, want, grid.ncol)
    for _ in range(3):
        step.replay(st)
    st.synchronize()
    for k, v in step.outputs().items():
        assert torch.equal(v, first[k]), k


def test_host_entries_step_matches_oracle(cuda, pkg, orc):
    """The same step through the host-pointer entries, routine by routine
    (the drop-in a model makes without keeping fields on the device)."""
    dyn = pkg.dynamics
    grid = dyn.Grid(57, 20, 12, 0.25, lat0_deg=20.0, dlat_deg=2.5)
    h = dyn.synthetic_inputs(grid, 7, nstep_sub=3)
    want = dyn.host_step(orc, grid, h)
    got = dyn.host_step(dyn.HostEntries(), grid, h)
    for name, w in want.items():
        assert _rel(got[name], w) <= TOL.get(name, MINOR_TOL), name


def test_device_entries_on_concurrent_streams(cuda, pkg):
    """Fused routines issued on two streams at once (each stream has its own
    scratch and status word) give the bits each gives alone."""
    torch = cuda
    nk, ncol, dz = 57, 20000, 0.25
    ld = pkg.batch.pad_ld(ncol)
    dyn = pkg.dynamics
    grid = type("G", (), dict(nk=nk, ncol=ncol, ld=ld))()
    Fc, Cc = pkg.synth.comp_inputs(nk, ncol, dz, 3)
    Fm, Cm = pkg.synth.minor_inputs(nk, ncol, dz, 4)
    Fs, Cs, qt = pkg.synth.settei_inputs(nk, ncol, dz, 6)
    dc = dyn._dev_fields(Fc, grid, ("expz", "difk"), "cuda")
    dm = dyn._dev_fields(Fm, grid, ("expz", "difk"), "cuda")
    dset = dyn._dev_fields(Fs, grid, (), "cuda")
    qd = pkg.batch.level_scalar(qt, ld, "cuda")

    def run(streams):
        oc = torch.zeros((3, nk, ld), dtype=torch.float64, device="cuda")
        om = torch.zeros((nk, ld), dtype=torch.float64, device="cuda")
        te, ti = (torch.zeros((nk, ld), dtype=torch.float64, device="cuda") for _ in range(2))
        q = qd.clone()
        sts = [torch.zeros(1, dtype=torch.int32, device="cuda") for _ in range(3)]
        torch.cuda.synchronize()
        for _ in range(3):     # repeated, so that the streams' work overlaps
            pkg.comp_ng_dev(dc, Cc, oc, nk, ncol, ld, status=sts[0], stream=streams[0])
            pkg.minor_ng_dev(dm, Cm, om, nk, ncol, ld, status=sts[1], stream=streams[1])
            with torch.cuda.stream(streams[2]):
                q.copy_(qd)
            pkg.settei_ng_dev(dset, Cs, te, ti, q, nk, ncol, ld, status=sts[2], stream=streams[2])
        torch.cuda.synchronize()
        assert all(int(s.item()) == pkg.TG_OK for s in sts)
        return oc, om, te, ti, q

    one = torch.cuda.Stream()
    alone = run([one, one, one])
    three = [torch.cuda.Stream() for _ in range(3)]
    together = run(three)
    for a, b in zip(alone, together):
        assert torch.equal(a, b)
