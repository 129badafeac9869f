"""The C-ABI library loads and exports every symbol include/tg_colsolve.h
declares; host-only calls validate their arguments.  No GPU work here."""
import os
import re

import pytest

from conftest import ROOT


def header_functions():
    txt = open(os.path.join(ROOT, "include", "tg_colsolve.h")).read()
    return sorted(set(re.findall(r"^\s*(?:int|long|const char \*)\s*(tg_\w+)\s*\(", txt, re.M)))


def test_header_lists_every_export(pkg):
    assert header_functions() == sorted(pkg.colsolve.EXPORTS)


def test_library_exports_all_symbols(pkg):
    L = pkg.colsolve.lib()
    for name in header_functions():
        assert hasattr(L, name), name


def test_kernel_arch_without_device(pkg):
    """The architecture query needs a device; without one it says so."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("checks the no-device path")
    with pytest.raises(pkg.TgError) as e:
        pkg.colsolve.kernel_arch()
    assert e.value.status == pkg.TG_ENODEV


@pytest.mark.gpu
def test_library_runs_sm100a_code(cuda, pkg):
    """The kernels the device loads are the library's sm_100a build."""
    assert pkg.colsolve.kernel_arch() == 100


def test_version_and_host_validation(pkg):
    cs = pkg.colsolve
    assert "sm_100a" in cs.version()
    with pytest.raises(cs.TgError):
        cs.set_refine(0, 1e-10)
    with pytest.raises(cs.TgError):
        cs.set_refine(3, 2.0)
    cs.set_refine(3, 1e-11)
    with pytest.raises(cs.TgError):
        cs.set_tile(cs.TG_KIND_SCALAR, cs.TG_PREC_F64, 48, 1)
    with pytest.raises(cs.TgError):
        cs.set_tile(cs.TG_KIND_BLOCK3, cs.TG_PREC_F64, 64, 2)
    cs.set_tile(cs.TG_KIND_SCALAR, cs.TG_PREC_F64, 0, 0)


def test_python_argument_checks(pkg):
    import numpy as np
    cs = pkg.colsolve
    a = np.zeros((5, 3))  # C order: rejected before any device call
    with pytest.raises(TypeError):
        cs.trsolv_ng(a, a, a, a, a, 5)
    af = np.zeros((5, 3), order="F")
    with pytest.raises(ValueError):
        cs.trsolv_ng(af, af, af, af, np.zeros((4, 3), order="F"), 5)


def test_bad_arguments_rejected_without_device(pkg):
    import ctypes
    L = pkg.colsolve.lib()
    # null pointers / k2 > nk are rejected before the library touches CUDA
    assert L.tg_trsolv_ng(None, None, None, None, None, 5, 5, 3) == pkg.TG_EINVAL
    buf = (ctypes.c_double * 15)()
    p = ctypes.cast(buf, ctypes.c_void_p)
    assert L.tg_trsolv_ng(p, p, p, p, p, 5, 6, 3) == pkg.TG_EINVAL
    assert L.tg_comp_blksolve_ng(4, p, p, p, p, None, None, p, 5, 1) == pkg.TG_EINVAL
    assert L.tg_plan_create(None, 1, 0, None) == pkg.TG_EINVAL
    # the walk test entry: an unknown walk, a stride below the columns, a
    # missing status word, an O+ factor pass on fewer than 3 levels
    st = ctypes.cast((ctypes.c_int * 1)(), ctypes.c_void_p)
    assert L.tg_selftest_walk(2, p, 3, 3, 0, 2, 2, st, None) == pkg.TG_EINVAL
    assert L.tg_selftest_walk(0, p, 3, 3, 0, 4, 2, st, None) == pkg.TG_EINVAL
    assert L.tg_selftest_walk(0, p, 3, 3, 0, 2, 2, None, None) == pkg.TG_EINVAL
    assert L.tg_selftest_walk(1, p, 2, 1, 1, 2, 2, st, None) == pkg.TG_EINVAL


def test_tuning_entries_validate_without_device(pkg):
    """Tuning entries reject out-of-range values and accept their resets
    without touching CUDA."""
    L = pkg.colsolve.lib()
    assert L.tg_set_host_pipeline(0, 9) == pkg.TG_EINVAL   # at most 8 streams
    assert L.tg_set_host_pipeline(2048, 4) == pkg.TG_OK
    assert L.tg_set_host_pipeline(0, 0) == pkg.TG_OK       # defaults back
    assert L.tg_set_kind_overlap(0) == pkg.TG_OK
    assert L.tg_set_kind_overlap(-1) == pkg.TG_OK
    assert L.tg_set_scalar_scratch_budget(0.0) == pkg.TG_OK
    assert L.tg_set_pipeline(pkg.TG_KIND_SCALAR, pkg.TG_PREC_F32_REFINE, 8, 1) == pkg.TG_EINVAL
    assert L.tg_set_pipeline(pkg.TG_KIND_BLOCK2, pkg.TG_PREC_F32_REFINE, 3, 1) == pkg.TG_EINVAL
    assert L.tg_set_pipeline(pkg.TG_KIND_SCALAR, pkg.TG_PREC_F32_REFINE, -1, 0) == pkg.TG_OK


def header_arity():
    """Number of parameters of each declared entry point."""
    txt = open(os.path.join(ROOT, "include", "tg_colsolve.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    out = {}
    for m in re.finditer(r"^\s*(?:int|const char \*)\s*(tg_\w+)\s*\(([^;]*?)\)\s*;", txt, re.M | re.S):
        params = m.group(2).strip()
        out[m.group(1)] = 0 if params in ("", "void") else params.count(",") + 1
    return out


def test_fortran_binding_matches_header():
    """The ISO_C_BINDING module (not compilable here: no Fortran compiler)
    binds only exported names, each with the header's parameter count."""
    src = open(os.path.join(ROOT, "tiegcm3.0_ng_b200", "fortran", "tg_colsolve_mod.F90")).read()
    src = re.sub(r"!.*", "", src)
    src = re.sub(r"&\s*\n\s*", " ", src)
    arity = header_arity()
    found = re.findall(r"function\s+(\w+)\s*\(([^)]*)\)\s*bind\(C,\s*name=\"(\w+)\"\)", src, re.I)
    assert len(found) >= 15
    for fname, args, cname in found:
        assert fname == cname, (fname, cname)
        assert cname in arity, cname
        nargs = 0 if not args.strip() else args.count(",") + 1
        assert nargs == arity[cname], (cname, nargs, arity[cname])


def test_host_wrappers_check_field_sizes(pkg):
    """The fused host wrappers accept the benchmark's field shapes (the call
    then stops at the missing device) and reject a short field before any C
    call reads it."""
    import numpy as np
    import torch
    if torch.cuda.is_available():
        pytest.skip("checks the no-device path")
    nk, ncol, dz = 5, 12, 0.5
    z = lambda: np.zeros((nk, ncol), order="F")  # noqa: E731
    calls = {
        "dt": (pkg.synth.dt_inputs(nk, ncol, dz, 1), lambda F, C: pkg.dt_ng(F, C, z()), "tlbc"),
        "minor": (pkg.synth.minor_inputs(nk, ncol, dz, 1), lambda F, C: pkg.minor_ng(F, C, z()), "fubc"),
        "comp": (pkg.synth.comp_inputs(nk, ncol, dz, 1), lambda F, C: pkg.comp_ng(F, C, z(), z(), z()), "difk"),
        "oplus": (pkg.synth.oplus_inputs(nk, ncol, dz, 1), lambda F, C: pkg.oplus_ng(F, C, z(), z(), z()), "zpint"),
    }
    for name, ((F, C), call, short) in calls.items():
        with pytest.raises(pkg.TgError) as e:
            call(F, C)
        assert e.value.status == pkg.TG_ENODEV, name
        F = dict(F)
        F[short] = np.asarray(F[short])[:-1].copy()
        with pytest.raises(ValueError):
            call(F, C)
    F, C, qt = pkg.synth.settei_inputs(nk, ncol, dz, 1)
    with pytest.raises(pkg.TgError):
        pkg.settei_ng(F, C, z(), z(), qt.copy(order="F"))
    with pytest.raises(ValueError):
        pkg.settei_ng(F, C, z(), z(), np.zeros((nk, ncol - 1), order="F"))


def _run_c_caller(pkg, tmp_path):
    import shutil
    import subprocess
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    libdir = os.path.dirname(pkg.colsolve.LIB_PATH)
    exe = str(tmp_path / "abi_check")
    subprocess.run([cc, "-O0", "-std=c11", "-ffp-contract=off", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "c", "abi_check.c"), "-o", exe, "-L", libdir, "-ltg_colsolve",
                    f"-Wl,-rpath,{libdir}", "-lm"], check=True)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    return r.stdout


def test_plain_c_caller(pkg, tmp_path):
    """tests/c/abi_check.c: the header and library used from C alone."""
    assert _run_c_caller(pkg, tmp_path).startswith("abi_check: ok")


@pytest.mark.gpu
def test_plain_c_caller_solves_on_the_device(cuda, pkg, tmp_path):
    """The C caller's device branch: a solve, the architecture query and a
    deferred latitude slab, from C with no Python in the process."""
    assert _run_c_caller(pkg, tmp_path).startswith("abi_check: ok (solved on the device)")
