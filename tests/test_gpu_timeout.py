"""The bounded waits of the bulk-copy ring kernels give up with TG_ETIMEOUT
instead of hanging.  The test runs the same wait on an mbarrier that nothing
completes (a flag nothing sets), with a short poll limit, checks the status,
and checks that the library still solves bit-exactly afterwards."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("polls", [1, 1000])
def test_wait_runs_out_and_reports_timeout(cuda, pkg, orc, polls):
    torch = cuda
    st = torch.full((1,), -1, dtype=torch.int32, device="cuda")
    assert pkg.selftest_wait(polls, st) == pkg.TG_OK
    torch.cuda.synchronize()
    assert int(st.item()) == pkg.TG_ETIMEOUT
    # the context is intact: a ring-kernel solve afterwards is bit-exact
    a, b, c, f = pkg.synth.scalar_system(57, 700, 0.25, 3)
    x = np.zeros_like(a, order="F")
    assert pkg.trsolv_ng(a, b, c, f, x, 56) == pkg.TG_OK
    assert np.array_equal(x[:56], orc.trsolv_ng(a, b, c, f, 56)[:56])


def test_wait_rejects_unbounded_limits(pkg):
    import ctypes
    st = ctypes.c_int(0)
    with pytest.raises(pkg.colsolve.TgError):
        pkg.selftest_wait(0, ctypes.addressof(st))
