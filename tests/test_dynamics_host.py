"""Host-side pieces of the device dynamics step: the lateral-boundary ring,
the seeded inputs and their layout (no device needed)."""
import numpy as np


def test_boundary_mask_is_the_outermost_ghost_ring(pkg):
    g = pkg.dynamics.Grid(57, 20, 12, 0.25)
    m = g.boundary_mask().reshape(g.nlat + 4, g.nlon + 4)
    assert m.sum() == 2 * (g.nlon + 4) + 2 * (g.nlat + 4) - 4
    assert m[0].all() and m[-1].all() and m[:, 0].all() and m[:, -1].all()
    assert not m[1:-1, 1:-1].any()
    assert g.ncol == (g.nlon + 4) * (g.nlat + 4) and g.ld % 32 == 0 and g.ld >= g.ncol
    assert g.racs.shape == (g.nlat + 4,) and np.all(g.racs > 0)


def test_synthetic_inputs_shapes_and_seeding(pkg):
    dyn = pkg.dynamics
    g = dyn.Grid(29, 8, 6, 0.5)
    a, b = dyn.synthetic_inputs(g, 3, nstep_sub=2), dyn.synthetic_inputs(g, 3, nstep_sub=2)
    c = dyn.synthetic_inputs(g, 4, nstep_sub=2)
    shape = (g.nk, g.ncol)
    assert [m["name"] for m in a["minor"]] == list(dyn.MINOR_SPECIES)
    assert a["oplus"]["C"]["nstep_sub"] == 2
    for arr in (a["dt"]["tn_nm"], a["dt"]["bnd"], a["oplus"]["optm1"], a["comp"]["o2_nm"], a["comp"]["he_bnd"],
                a["settei"]["qtotal"], a["minor"][0]["fcomp"], a["winds"]["un"]):
        assert arr.shape == shape and arr.flags.f_contiguous and np.all(np.isfinite(arr))
    assert np.array_equal(a["dt"]["tn_nm"], b["dt"]["tn_nm"])
    assert not np.array_equal(a["dt"]["tn_nm"], c["dt"]["tn_nm"])
    # the time levels the filters combine stay close, as in the model
    assert np.allclose(a["dt"]["tn_nm"], a["dt"]["F"]["tn"], rtol=0.011)
    assert np.all(a["comp"]["zpmid"][1:] > a["comp"]["zpmid"][:-1])
