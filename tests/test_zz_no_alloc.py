"""The allocation-free block solve, tg_blksolve_dev_noalloc.

It is for callers that cannot allocate device memory: a model that hands its
whole device-memory budget to its own pool at start-up, or a time loop that
must not be stalled by the device-wide synchronisation that freeing an
outgrown buffer implies.  Its scratch is a fixed array inside the library, so
it must give exactly the numbers of the regular device entry
(tg_blksolve_dev, level-major, FP64) on two calls in a row, and the second
call must not see the first call's status.

This file is collected last on purpose, so that a run stopping at the first
failure has already run every other test."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def level_inputs(pkg, torch, B, nk, ncol, seed):
    P, Q, R, f = pkg.synth.block_system(B, nk, ncol, 14.0 / (nk - 1), seed)
    rng = np.random.default_rng(seed)
    ratio = np.asfortranarray(rng.uniform(0.5, 1.5, (B, ncol)))
    add = np.asfortranarray(rng.uniform(-1e-3, 1e-3, (B, ncol)))
    ld = pkg.batch.pad_ld(ncol)
    t = dict(P=pkg.batch.level_matrix(P, ld, "cuda"), Q=pkg.batch.level_matrix(Q, ld, "cuda"),
             R=pkg.batch.level_matrix(R, ld, "cuda"), f=pkg.batch.level_vector(f, ld, "cuda"))
    for name, v in (("ratio", ratio), ("add", add)):
        tv = torch.zeros((B, ld), dtype=torch.float64, device="cuda")
        tv[:, :ncol] = torch.from_numpy(v)
        t[name] = tv
    return t, ld


def test_noalloc_matches_regular_entry_on_two_calls(cuda, pkg):
    torch = cuda
    cs = pkg.colsolve
    cases = [(3, 57, 3001, 11), (2, 57, 2500, 12)]
    inputs = [level_inputs(pkg, torch, *c) for c in cases]
    # first call: one singular first-row block, so its status is TG_EPIVOT
    inputs[0][0]["Q"][0, :, :, 5] = 0.0
    outs, stats = [], []
    for (B, nk, ncol, _), (t, ld) in zip(cases, inputs):
        u = torch.full_like(t["f"], 7.0)
        st = torch.zeros(1, dtype=torch.int32, device="cuda")
        cs.blksolve_dev_noalloc(B, t["P"], t["Q"], t["R"], t["f"], u, nk, nk - 1, ncol,
                                ubc_ratio=t["ratio"], ubc_add=t["add"], ld=ld, status=st)
        outs.append(u)
        stats.append(st)
    torch.cuda.synchronize()
    assert [int(s.item()) for s in stats] == [cs.TG_EPIVOT, cs.TG_OK]
    for (B, nk, ncol, _), (t, ld), u in zip(cases, inputs, outs):
        ref = torch.full_like(t["f"], 7.0)
        cs.blksolve_dev(B, t["P"], t["Q"], t["R"], t["f"], ref, nk, nk - 1, ncol, ubc_ratio=t["ratio"],
                        ubc_add=t["add"], layout=cs.TG_LAYOUT_LEVEL, ld=ld, precision=cs.TG_PREC_F64)
        torch.cuda.synchronize()
        assert torch.equal(torch.nan_to_num(u, nan=-1.0), torch.nan_to_num(ref, nan=-1.0))


def test_noalloc_rejects_oversized_columns(cuda, pkg):
    cs = pkg.colsolve
    torch = cuda
    nk = 4000
    buf = torch.zeros(8, dtype=torch.float64, device="cuda")
    with pytest.raises(cs.TgError, match="exceeds the fixed scratch"):
        cs.blksolve_dev_noalloc(3, buf, buf, buf, buf, buf, nk, nk, 1, ld=1)


NO_ALLOC_PROBE = r"""
import sys
import numpy as np
import torch
sys.path.insert(0, sys.argv[1])
import __graft_entry__ as ge
torch.cuda.set_device(0)
pkg = ge.load_package()
cs = pkg.colsolve


def inputs(B, nk, ncol, seed):
    P, Q, R, f = pkg.synth.block_system(B, nk, ncol, 14.0 / (nk - 1), seed)
    ld = pkg.batch.pad_ld(ncol)
    t = [pkg.batch.level_matrix(v, ld, "cuda") for v in (P, Q, R)] + [pkg.batch.level_vector(f, ld, "cuda")]
    return t, torch.zeros_like(t[3]), ld


small, u0, ld0 = inputs(3, 57, 500, 1)
big, u1, ld1 = inputs(3, 113, 60000, 2)
st = torch.zeros(2, dtype=torch.int32, device="cuda")
torch.cuda.synchronize()
# the first call loads the library's kernels and its fixed array
cs.blksolve_dev_noalloc(3, *small, u0, 57, 57, 500, ld=ld0, status=st[0:1])
torch.cuda.synchronize()
free0 = torch.cuda.mem_get_info()[0]
# a larger second call: the regular entry would grow its scratch here
cs.blksolve_dev_noalloc(3, *big, u1, 113, 113, 60000, ld=ld1, status=st[1:2])
torch.cuda.synchronize()
free1 = torch.cuda.mem_get_info()[0]
print("free", free0, free1, "status", st.tolist())
assert st.tolist() == [0, 0]
assert free1 == free0, (free0, free1)
"""


def test_noalloc_leaves_free_device_memory_unchanged(cuda, pkg):
    """In a fresh process whose first library call is this entry: a second,
    larger call leaves the device's free memory exactly as it was (the
    regular entry would have grown its scratch buffer for it)."""
    import os
    import subprocess
    import sys
    from conftest import ROOT
    r = subprocess.run([sys.executable, "-c", NO_ALLOC_PROBE, ROOT], capture_output=True, text=True, timeout=600,
                       env=dict(os.environ, CUDA_MODULE_LOADING="LAZY"))
    assert r.returncode == 0, r.stdout + r.stderr
    assert "free" in r.stdout
