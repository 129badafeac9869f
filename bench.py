#!/usr/bin/env python
"""Column unknowns solved per second for the TIE-GCM NG vertical column solves
on one B200 (or N, one process each, weak scaling).

One step = every system of one outer step of the workload.  By default that
is the nested batch the performance target is quoted on: the 2.5 deg global
grid (144 x 72 columns) plus three nest levels (0.625, 0.3125 and 0.15625 deg
boxes with their ghost columns, 4, 8 and 16 sub-cycles each, so 4, 32 and 512
sub-steps per outer step), 57 levels, seven scalar tridiagonal systems plus
one 2x2 block-tridiagonal system per column and sub-step: 1.22 M column
steps, 624 M unknowns, 23.4 GB of coefficients per step, all sub-steps in
one persistent launch per system kind, the step replayed from one CUDA graph.
Inputs are seeded synthetic coefficients with the benchmark's value laws,
generated on the device; they exceed the 126 MB L2 many times over, so no
L2 flush is needed between steps.  --config 1 selects the global grid alone.

  value   FP64 path (bit-identical to the reference arithmetic), device-
          resident plan (unknowns/s); the FP32-sweep + FP64-refinement path is
          reported beside it ("refine") with its ratio to FP64 and its error
          against the FP64 solution.
  e2e     the same solves through the C-ABI (tg_solve_host) with pinned host
          buffers in the reference's Fortran layout, host<->device copies
          inside the timed region, on the workload's global grid (one
          sub-step; the per-unknown rate is the metric).
  roofline  the dominant kernel (scalar solve) against the measured HBM copy
          bandwidth, algorithmic bytes = 40 B per scalar unknown.
  assembly  the fused assembly + solve kernels (dt_ng, minor_ng, comp_ng,
          settei_ng, oplus_ng) on 4 copies of the global grid.
  horizontal  advec_ng, smooth_ng and the dt_ng post-solve time filter on the
          576 x 288 x 113 grid held as one subdomain.
  cpu_baseline  the oracle port (C, OpenMP, all host threads) on full steps of
          the global grid.

--impl reference times the reference algorithm on the host cores (the oracle
port: the reference is Fortran and no Fortran compiler exists here).
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
import __graft_entry__ as ge  # noqa: E402

FALLBACK_HBM_GBS = 6650.0


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=50)
    p.add_argument("--warmup", type=int, default=5)
    p.add_argument("--impl", choices=["ours", "reference"], default="ours")
    p.add_argument("--config", type=int, default=3,
                   help="workload index 0..4 (default 3: 2.5 deg global grid + 3 nests, all sub-steps)")
    p.add_argument("--block", type=int, default=2, help="block size of the block system (2: O2/O, 3: O2/O/He)")
    p.add_argument("--max-sub", type=int, default=None, help="cap nest sub-steps (nested workloads)")
    p.add_argument("--skip-e2e", action="store_true")
    p.add_argument("--skip-cpu", action="store_true")
    p.add_argument("--cpu-seconds", type=float, default=10.0)
    p.add_argument("--e2e-steps", type=int, default=5)
    p.add_argument("--profile", default=None,
                   help="run only one kind's plan for a profiler: KIND:PREC[:VARIANT], KIND scalar|block, "
                        "PREC f64|refine, VARIANT reg:CPB:CPT[:PF], regg:CPB:1[:PF], ring[g]:DEPTH[:WARPS] "
                        "(default: library default); or dt / minor / comp / settei / oplus for the fused assembly+solve kernels, "
                        "advec / smooth / filter for the horizontal operators and the time filter; "
                        "dynamics:N for one dynamics step of grid N, serial on one stream")
    p.add_argument("--skip-assembly", action="store_true")
    p.add_argument("--tune", action="store_true",
                   help="run the autotuner over this workload's segments first and record its choices in the "
                        "package's tuning cache (tiegcm3.0_ng_b200/tuned_b200.json)")
    p.add_argument("--no-tuned", action="store_true", help="ignore the package's tuning cache (library defaults)")
    return p.parse_args()


def measured_peak():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as fh:
            return float(json.load(fh)["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


def traffic_from_profiles(kernel, workload):
    """Per-launch DRAM bytes of a kernel from the committed ncu summary, if any
    (a line 'traffic_bytes_per_launch <kernel> <workload> <bytes>')."""
    d = os.path.join(ROOT, "profiles")
    if not os.path.isdir(d):
        return None
    for name in sorted(os.listdir(d)):
        if not name.endswith((".md", ".txt")):
            continue
        with open(os.path.join(d, name)) as fh:
            for line in fh:
                parts = line.strip().strip("`").split()
                if len(parts) == 4 and parts[0] == "traffic_bytes_per_launch" and parts[1] == kernel and parts[2] == workload:
                    return float(parts[3])
    return None


class Clocks:
    """nvidia-smi sampling of SM clock and throttle reasons (200 ms)."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.fh, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"], "samples": 0}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.fh.close()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        with open(self.path) as fh:
            for line in fh:
                p = [v.strip() for v in line.split(",")]
                if len(p) < 9:
                    continue
                try:
                    sm.append(float(p[1]))
                    smax = float(p[2])
                except ValueError:
                    continue
                for n, v in zip(names, p[5:9]):
                    if v.lower() == "active":
                        reasons.add(n)
        os.unlink(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


METRIC = "column unknowns/s (FP64 path; FP32+FP64-refine path beside it, <=1e-10 rel err)"


def host_inputs(pkg, wl, grid, seed_offset=0):
    """numpy (Fortran layout) inputs of one column step of one grid."""
    scal, blk = pkg.synth.column_step(wl, grid, sub=seed_offset)
    return scal, blk


def nsub_of(g, max_sub):
    return g.nsub if max_sub is None else min(g.nsub, max_sub)


def workload_config(pkg, wl, max_sub):
    """The `config` object of both arms' JSON lines: the workload's grids,
    systems and sizes, computed from its definition alone, so that the two
    arms describe the same work identically."""
    B = wl.block
    nsys = wl.n_scalar + (1 if B else 0)
    unknowns = segments = nbytes = 0
    for g in wl.grids:
        n = nsub_of(g, max_sub)
        unknowns += n * g.ncol * g.nk * (wl.n_scalar + (B or 0))
        segments += n * nsys
        nbytes += n * pkg.batch.pad_ld(g.ncol) * g.nk * 8 * (4 * wl.n_scalar + ((3 * B * B + B) if B else 0))
    return {"workload": wl.name, "grids": [(g.name, g.nlon, g.nlat, g.nk, nsub_of(g, max_sub)) for g in wl.grids],
            "systems_per_column": nsys, "block": B, "unknowns_per_step": unknowns, "segments": segments,
            "l2": f"inputs {nbytes / 1e9:.3f} GB per step > 126 MB L2 (no flush needed)",
            "parallelism": "columns sharded over the ranks (contiguous column ranges, balanced by unknowns)"}


def job_shapes(wl, g):
    """Fortran-layout shapes of the arrays of one grid sub-step: per scalar
    system a, b, c, f, x (nk, ncol); the block system P, Q, R (B, B, nk, ncol)
    and f, u (B, nk, ncol)."""
    shp = [[(g.nk, g.ncol)] * 5 for _ in range(wl.n_scalar)]
    if wl.block:
        B = wl.block
        shp.append([(B, B, g.nk, g.ncol)] * 3 + [(B, g.nk, g.ncol)] * 2)
    return shp


class HostWorkload:
    """Every system of one outer step of a workload (or of the given grid
    sub-steps) in host memory, in the reference's Fortran layout, with
    preallocated solutions.  Generated by the same seeded law as the device
    workload (synth.column_step per grid and sub-step), in parallel host
    threads.  With pinned=True all arrays live in one page-locked arena, as a
    host model's buffers registered for fast copies would."""

    def __init__(self, pkg, wl, max_sub=None, threads=8, jobs=None, pinned=False):
        from concurrent.futures import ThreadPoolExecutor
        if jobs is None:
            jobs = [(g, sub) for g in wl.grids for sub in range(nsub_of(g, max_sub))]
        self.jobs = [(g.name, sub) for g, sub in jobs]
        self.arena = None
        offs, off = [], 0
        for g, _ in jobs:
            o = []
            for sysshp in job_shapes(wl, g):
                oo = []
                for shp in sysshp:
                    oo.append(off)
                    off += (int(np.prod(shp)) * 8 + 255) // 256 * 256
                o.append(oo)
            offs.append(o)
        if pinned:
            import torch
            self.arena = torch.empty(max(off, 1), dtype=torch.uint8, pin_memory=True)
            buf = self.arena.numpy()
        else:
            buf = np.empty(max(off, 1), dtype=np.uint8)

        def view(o, shp):
            return np.ndarray(shp, dtype=np.float64, buffer=buf, offset=o, order="F")

        def make(i):
            g, sub = jobs[i]
            scal, blk = pkg.synth.column_step(wl, g, sub=sub)
            out = []
            for arrs, shps, oo in zip(list(scal) + ([blk] if blk is not None else []), job_shapes(wl, g), offs[i]):
                vs = [view(o, shp) for o, shp in zip(oo, shps)]
                for v, a in zip(vs, arrs):
                    np.copyto(v, a)
                vs[4][...] = 0.0
                out.append(tuple(vs))
            return out

        with ThreadPoolExecutor(max(1, threads)) as ex:
            per_job = list(ex.map(make, range(len(jobs))))
        self.scal, self.blk = [], []
        for systems in per_job:
            for t in systems:
                (self.scal if t[0].ndim == 2 else self.blk).append(t)

    def unknowns(self):
        return sum(a.size for (a, *_r) in self.scal) + sum(t[3].size for t in self.blk)

    def input_bytes(self):
        return sum(sum(v.nbytes for v in t[:4]) for t in self.scal + self.blk)

    def step(self, orc, nthreads):
        """One outer step through the oracle port (the reference's FP64
        arithmetic), OpenMP over the columns of each system."""
        for (a, b, c, f, x) in self.scal:
            orc.trsolv_ng(a, b, c, f, a.shape[0], x=x, nthreads=nthreads)
        for (P, Q, R, f, u) in self.blk:
            orc.blksolve(P, Q, R, f, f.shape[1], u=u, nthreads=nthreads)


def time_host_steps(orc, hw, nthreads, steps=None, seconds=None, warmup=1):
    for _ in range(warmup):
        hw.step(orc, nthreads)
    t0 = time.perf_counter()
    n = 0
    while True:
        hw.step(orc, nthreads)
        n += 1
        el = time.perf_counter() - t0
        if steps is not None and n >= steps:
            break
        if seconds is not None and el >= seconds:
            break
    return el / n, n


def host_memory_available():
    try:
        import psutil
        return psutil.virtual_memory().available
    except Exception:
        return None


def run_reference(args):
    """The reference's CPU implementation of the path on this host's cores:
    the oracle port (the reference is Fortran and no Fortran compiler exists
    here), timed on every system of the same workload and config as the
    GPU arm, rank 0 alone."""
    world, rank, _ = dist_setup(args)
    if rank != 0:
        return 0
    pkg = ge.load_package()
    orc = ge.load_oracle()
    wl = pkg.synth.workload(args.config)
    if wl.block:
        wl.block = args.block
    nthreads = orc.max_threads()
    cfg = workload_config(pkg, wl, args.max_sub)
    need = 1.3 * sum(nsub_of(g, args.max_sub) * g.ncol * g.nk * 8 * (5 * wl.n_scalar + ((3 * wl.block ** 2 + 2 * wl.block) if wl.block else 0))
                     for g in wl.grids)
    avail = host_memory_available()
    if avail is None or need < 0.6 * avail:
        hw = HostWorkload(pkg, wl, args.max_sub, threads=nthreads)
        sample = (f"every system of every grid and sub-step of the workload ({len(hw.jobs)} grid sub-steps, "
                  f"{hw.unknowns()} unknowns, {hw.input_bytes() / 1e9:.1f} GB of coefficients) per step")
    else:
        # not enough host memory for the whole step: one sub-step of each grid
        hw = HostWorkload(pkg, wl, threads=nthreads, jobs=[(g, 0) for g in wl.grids])
        sample = (f"one sub-step of each grid per step ({hw.unknowns()} unknowns; the whole step needs "
                  f"{need / 1e9:.0f} GB of host memory, {avail / 1e9:.0f} GB available)")
    dt, n = time_host_steps(orc, hw, nthreads, steps=args.steps, warmup=args.warmup)
    value = hw.unknowns() / dt
    out = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "unknowns/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt * 1e3,
        "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded, generated on the host)", "config": cfg,
        "cpu_baseline": {"value": value, "unit": "unknowns/s", "cores": nthreads, "kind": "port",
                         "sample": sample + ", oracle C port (-O2 -ffp-contract=off), OpenMP over columns"},
        "e2e": {"value": value, "unit": "unknowns/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": "reference algorithm restated in C (oracle port); the reference is Fortran and no Fortran "
                "compiler is available",
    }
    print(json.dumps(out))
    return 0


ASSEMBLY_REPLICAS = 4    # grid copies per assembly launch: inputs > L2


def assembly_setup(pkg, wl, which, dev, replicas=ASSEMBLY_REPLICAS):
    """Device inputs of one fused assembly+solve routine (dt_ng or minor_ng)
    over `replicas` copies of the workload's first grid, level-major.
    Returns (launch(stream), columns, algorithmic bytes per launch)."""
    import torch
    grid = wl.grids[0]
    nk, ncol, dz = grid.nk, grid.ncol * replicas, grid.dz
    nout = 1
    if which == "dt":
        F, C = pkg.synth.dt_inputs(nk, ncol, dz, 101)
        one_d, n2d, n3d = ("expz", "dift"), len(pkg.synth.DT_2D), len(pkg.synth.DT_FIELDS)
    elif which == "minor":
        F, C = pkg.synth.minor_inputs(nk, ncol, dz, 103)
        one_d, n2d, n3d = ("expz", "difk"), len(pkg.synth.MINOR_2D), len(pkg.synth.MINOR_FIELDS)
    elif which == "comp":
        F, C = pkg.synth.comp_inputs(nk, ncol, dz, 107)
        one_d, n2d, n3d = ("expz", "difk"), len(pkg.synth.COMP_2D), len(pkg.synth.COMP_FIELDS) + 12
        nout = 3
    elif which == "oplus":
        F, C = pkg.synth.oplus_inputs(nk, ncol, dz, 113)
        # 27 fields read; opout, xiop2p, xiop2d written (Fe, Fn not requested)
        one_d, n2d, n3d = ("zpint",), len(pkg.synth.OPLUS_2D), len(pkg.synth.OPLUS_FIELDS)
        nout = 3
    else:
        F, C, qt = pkg.synth.settei_inputs(nk, ncol, dz, 109)
        # 27 fields and qtotal read; te, ti and qtotal written
        one_d, n2d, n3d = (), len(pkg.synth.SETTEI_2D), len(pkg.synth.SETTEI_FIELDS) + 1
        nout = 3
    ld = pkg.batch.pad_ld(ncol)
    d = {}
    for k, v in F.items():
        if k == "fs":
            fs = np.asarray(v).reshape(12, ncol, nk)
            t = torch.zeros((12, nk, ld), dtype=torch.float64, device=dev)
            for s_ in range(12):
                t[s_, :, :ncol] = torch.from_numpy(np.ascontiguousarray(fs[s_].T)).to(dev)
            d[k] = t
        elif v.ndim == 2:
            d[k] = pkg.batch.level_scalar(v, ld, dev)
        elif k in one_d:
            d[k] = torch.from_numpy(np.ascontiguousarray(v)).to(dev)
        else:
            t = torch.zeros(ld, dtype=torch.float64, device=dev)
            t[:ncol] = torch.from_numpy(v)
            d[k] = t
    out = torch.zeros((nout, nk, ld), dtype=torch.float64, device=dev)
    # 3-D fields read + the solution written, 2-D and 1-D inputs read
    nbytes = 8 * ((n3d + nout) * nk * ncol + n2d * ncol + len(one_d) * nk)
    if which == "oplus":
        def launch(stream):
            pkg.oplus_ng_dev(d, C, out[0], out[1], out[2], nk, ncol, ld, stream=stream)
        return launch, ncol, nbytes
    if which == "settei":
        qtd = pkg.batch.level_scalar(qt, ld, dev)

        def launch(stream):
            pkg.settei_ng_dev(d, C, out[0], out[1], qtd, nk, ncol, ld, stream=stream)
        return launch, ncol, nbytes
    fn = {"dt": pkg.dt_ng_dev, "minor": pkg.minor_ng_dev, "comp": pkg.comp_ng_dev}[which]

    def launch(stream):
        fn(d, C, out, nk, ncol, ld, stream=stream)
    return launch, ncol, nbytes


HORIZ_GRID = (113, 576, 288)   # levels, lon, lat: the 0.625-degree global grid, inputs > L2
HORIZ_TAG = "576x288x113"
EARTH_RADIUS_CM = 6.37122e8


def horizontal_setup(pkg, which, dev):
    """Device inputs of advec_ng, smooth_ng or the dt_ng time filter on the
    576x288x113 grid held as one subdomain (level-major planes).  Returns
    (launch(stream), points, algorithmic bytes per launch)."""
    import torch
    nk, nlon, nlat = HORIZ_GRID
    ncol = (nlon + 4) * (nlat + 4)
    ld = pkg.batch.pad_ld(ncol)
    g = torch.Generator(device=dev).manual_seed(211)

    def field(lo, hi):
        return torch.rand((nk, ld), dtype=torch.float64, device=dev, generator=g) * (hi - lo) + lo

    dlat = np.radians(180.0 / nlat)
    dlon = np.radians(360.0 / nlon)
    if which == "advec":
        f, un, vn = field(150.0, 2000.0), field(-1.0e4, 1.0e4), field(-1.0e4, 1.0e4)
        lat = -np.pi / 2 + dlat * (np.arange(nlat + 4) - 1.5)
        racs = torch.from_numpy(1.0 / (EARTH_RADIUS_CM * np.maximum(np.cos(lat), 1e-3))).to(dev)
        out = torch.empty_like(f)

        def launch(stream):
            pkg.advec_ng_dev(f, un, vn, racs, dlon, dlat, 1.0 / EARTH_RADIUS_CM, out, nk, nlon, nlat, ld,
                             stream=stream)
        return launch, nk * ncol, 8 * (4 * nk * ncol + nlat + 4)
    if which == "smooth":
        fin = field(150.0, 2000.0)
        out = torch.empty_like(fin)

        def launch(stream):
            pkg.smooth_ng_dev(fin, 0.03, out, nk, nlon, nlat, ld, stream=stream)
        return launch, nk * ncol, 16 * nk * ncol
    if which == "ring":
        # filter_o2o's order-1 ring filter over the 576 x 288 global grid
        # (the model's 0.625 deg chunk table: 80 polar latitudes filtered)
        ncg = (nlon + 4) * nlat
        ldg = pkg.batch.pad_ld(ncg)
        chunks = pkg.synth.RING_CHUNKS[(nlon, nlat)]
        f = torch.rand((nk, ldg), dtype=torch.float64, device=dev, generator=g) * 0.25 + 0.05
        dl = 2.0 * (4.0 * np.arctan(1.0)) / nlon
        rows = 2 * len(chunks) * nk

        def launch(stream):
            pkg.ringfilter_dev(f, nk, nlon, nlat, 1, 0, chunks, dl, ldg, stream=stream)
        # each filtered row: nlon+4 values read and written
        return launch, rows * (nlon + 4), 16 * rows * (nlon + 4)
    cur, prev, upd = field(150.0, 2000.0), field(150.0, 2000.0), field(50.0, 2000.0)
    nm = torch.empty_like(cur)

    def launch(stream):
        pkg.time_filter_ng_dev(pkg.TG_FILTER_DT, cur, prev, 0.95, 0.025, upd, nm, nk, ncol, ld, stream=stream)
    return launch, nk * ncol, 40 * nk * ncol


def dynamics_leg(pkg, wl, steps, warmup, stream, max_over_ranks, barrier, cpu=True):
    """One dynamics_ng step of the column routines on each grid of the
    workload (the global grid with the polar ring filter, each nest held as
    one subdomain; 10 O+ sub-steps): device-resident, serial on one stream,
    fanned out over five streams, and as one CUDA graph; the same step through
    the host-pointer entries routine by routine, and the oracle's routines on
    one host core.  The model's outer step takes nsub steps of each grid one
    after the other (each nest step starts from the last), so its column
    physics costs the sum over grids of nsub x the graph's time."""
    import torch
    dyn = pkg.dynamics
    orc = ge.load_oracle() if cpu else None
    out = {}
    model_ms = 0.0
    for gi, g in enumerate(wl.grids):
        if (g.nlon + 4) * (g.nlat + 4) * g.nk > 4_000_000:
            # ~200 level-major fields per step: host generation of the inputs would dominate the run
            out[g.name] = {"grid": f"{g.name} {g.nlon}x{g.nlat}x{g.nk}", "skipped": "more than 4 M points per field"}
            continue
        ring = pkg.synth.RING_CHUNKS.get((g.nlon, g.nlat)) if gi == 0 else None
        if gi == 0:
            grid = dyn.Grid(g.nk, g.nlon, g.nlat, g.dz)
        else:
            # a regional nest: latitude rows 2.5 deg / 2**gi apart from 20 N
            grid = dyn.Grid(g.nk, g.nlon, g.nlat, g.dz, lat0_deg=20.0, dlat_deg=2.5 / 2 ** gi,
                            shapiro=0.03)
        h = dyn.synthetic_inputs(grid, 17 + gi, nstep_sub=10)
        rec = {"grid": f"{g.name} {g.nlon}x{g.nlat}x{g.nk}", "columns": grid.ncol, "levels": grid.nk,
               "nsub_per_outer_step": g.nsub, "o_plus_sub_steps": 10, "ring_filter": ring is not None}

        def timed(fn):
            for _ in range(warmup):
                fn()
            stream.synchronize()
            barrier()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(steps):
                fn()
            e1.record(stream)
            e1.synchronize()
            return max_over_ranks(e0.elapsed_time(e1) / steps)

        serial = dyn.DynamicsStep(grid, h, ring=ring, fan_out=False)
        rec["ms_serial"] = timed(lambda: serial.issue(stream))
        del serial
        fan = dyn.DynamicsStep(grid, h, ring=ring, fan_out=True)
        rec["ms_fan_out"] = timed(lambda: fan.issue(stream))
        fan.capture(stream)
        rec["ms_graph"] = timed(lambda: fan.replay(stream))
        nbytes = fan.bytes_per_step()
        pk, _ = measured_peak()
        ach = nbytes / (rec["ms_graph"] * 1e-3) / 1e9
        rec["algorithmic_bytes_per_step"] = nbytes
        rec["roofline"] = {"bound": "hbm", "achieved": ach, "peak": pk, "unit": "GB/s", "frac": ach / pk}
        del fan
        torch.cuda.synchronize()
        # the same step through the host-pointer entries (wall clock, synchronous calls)
        if gi <= 1:
            host = dyn.HostEntries()
            dyn.host_step(host, grid, h, ring)
            n, t0 = 0, time.perf_counter()
            while n < 2 or (n < 10 and time.perf_counter() - t0 < 2.0):
                dyn.host_step(host, grid, h, ring)
                n += 1
            rec["ms_host_entries"] = (time.perf_counter() - t0) / n * 1e3
            if orc is not None:
                n, t0 = 0, time.perf_counter()
                while n < 1 or (n < 5 and time.perf_counter() - t0 < 3.0):
                    dyn.host_step(orc, grid, h, ring)
                    n += 1
                rec["ms_oracle_one_core"] = (time.perf_counter() - t0) / n * 1e3
        model_ms += g.nsub * rec["ms_graph"]
        out[g.name] = rec
        torch.cuda.empty_cache()
    if not any("skipped" in r for r in out.values()):
        out["outer_step_column_physics_ms"] = model_ms
    out["outer_step_note"] = ("sum over grids of nsub x the graph's time: the column routines of one global step with "
                              "every nest sub-step in sequence")
    return out


def run_profile(args):
    """Executes one kind's plan --warmup + --steps times (for ncu captures)."""
    import torch
    pkg = ge.load_package()
    if args.profile.startswith("dynamics:"):
        # one dynamics step of grid N of the workload, serial on one stream
        dyn = pkg.dynamics
        wl = pkg.synth.workload(args.config)
        gi = int(args.profile.split(":")[1])
        g = wl.grids[gi]
        grid = (dyn.Grid(g.nk, g.nlon, g.nlat, g.dz) if gi == 0 else
                dyn.Grid(g.nk, g.nlon, g.nlat, g.dz, lat0_deg=20.0, dlat_deg=2.5 / 2 ** gi))
        ring = pkg.synth.RING_CHUNKS.get((g.nlon, g.nlat)) if gi == 0 else None
        step = dyn.DynamicsStep(grid, dyn.synthetic_inputs(grid, 17 + gi, nstep_sub=10), ring=ring, fan_out=False)
        stream = torch.cuda.Stream()
        for _ in range(args.warmup + args.steps):
            step.issue(stream)
        stream.synchronize()
        print(json.dumps({"profile": args.profile, "grid": g.name, "columns": grid.ncol, "steps": args.steps}))
        return 0
    if args.profile in ("dt", "minor", "comp", "settei", "oplus", "advec", "smooth", "filter", "ring"):
        wl = pkg.synth.workload(args.config)
        if args.profile in ("advec", "smooth", "filter", "ring"):
            launch, ncol, nbytes = horizontal_setup(pkg, args.profile, "cuda")
        else:
            launch, ncol, nbytes = assembly_setup(pkg, wl, args.profile, "cuda")
        stream = torch.cuda.Stream()
        for _ in range(args.warmup):
            launch(stream)
        stream.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            launch(stream)
        e1.record(stream)
        e1.synchronize()
        ms = e0.elapsed_time(e1) / args.steps
        print(json.dumps({"profile": args.profile, "workload": wl.name, "columns": ncol, "ms_per_launch": ms,
                          "algorithmic_bytes": nbytes, "GBps": nbytes / ms / 1e6}))
        return 0
    cs = pkg.colsolve
    from tiegcm_ng_b200 import autotune
    parts = args.profile.split(":")
    wl = pkg.synth.workload(args.config)
    if wl.block:
        wl.block = args.block
    kind = cs.TG_KIND_SCALAR if parts[0] == "scalar" else wl.block
    prec = cs.TG_PREC_F64 if parts[1] == "f64" else cs.TG_PREC_F32_REFINE
    if len(parts) > 2:
        v = parts[2]
        cand = (v, int(parts[3]), int(parts[4]) if len(parts) > 4 else 4, 4) if v in ("ring", "ringg", "rows", "ring16", "ring8") or v.startswith(("chunk", "res")) else \
            (v, int(parts[3]), int(parts[4]), int(parts[5]) if len(parts) > 5 else 4)
        autotune.apply(kind, prec, cand)
    dw = pkg.batch.DeviceWorkload(wl, "cuda", max_sub=args.max_sub)
    segs = dw.segments((kind,))
    plan = pkg.Plan(segs, prec)
    print(plan.describe(), file=sys.stderr)
    stream = torch.cuda.Stream()
    for _ in range(args.warmup):
        plan.execute(stream)
    stream.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        plan.execute(stream)
    e1.record(stream)
    e1.synchronize()
    ms = e0.elapsed_time(e1) / args.steps
    rc, _ = plan.status()
    print(json.dumps({"profile": args.profile, "workload": wl.name, "block": wl.block, "ms_per_launch": ms,
                      "algorithmic_bytes": dw.algorithmic_bytes((kind,)), "unknowns": dw.unknowns((kind,)),
                      "GBps": dw.algorithmic_bytes((kind,)) / ms / 1e6, "status": cs.STATUS_NAMES[rc]}))
    plan.close()
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    if args.profile:
        return run_profile(args)
    import torch
    import torch.distributed as dist

    world, rank, local = dist_setup(args)
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=dev)
    pkg = ge.load_package()
    cs = pkg.colsolve
    wl = pkg.synth.workload(args.config)
    if wl.block:
        wl.block = args.block

    # one workload, the same on every rank; each rank solves its share of the
    # columns (contiguous ranges of the flattened column space, balanced by
    # unknowns, cut on 32-column tiles): no data-path collective
    dw = pkg.batch.DeviceWorkload(wl, dev, seed=pkg.synth.SEED_BASE, max_sub=args.max_sub)
    segs = pkg.batch.shard_segments(dw.segments(), world, rank)
    scal_segs = [s for s in segs if s["kind"] == cs.TG_KIND_SCALAR]
    blk_segs = [s for s in segs if s["kind"] != cs.TG_KIND_SCALAR]
    unknowns = dw.unknowns()                       # the whole job's, over all ranks
    stream = torch.cuda.Stream(device=dev)
    from tiegcm_ng_b200 import autotune
    tuning = None
    if args.tune:
        res = autotune.tune(segs, cache=autotune.PACKAGED, reps=5)
        tuning = {"tuned_now": {f"kind{k}_prec{p}": [list(v[0]), v[1]] for (k, p), v in res.items()
                                if k != "combined"}}
        for (k, p), (best, ms, times) in sorted((kv for kv in res.items() if kv[0][0] != "combined"),
                                                key=lambda kv: kv[0]):
            print(f"autotune kind {k} prec {p}: best {best} {ms:.4f} ms; " +
                  ", ".join(f"{c}: {t:.4f}" for c, t in sorted(times.items(), key=lambda ct: ct[1])),
                  file=sys.stderr)
    elif not args.no_tuned:
        found = autotune.load(segs, cache=autotune.PACKAGED)
        tuning = {"applied_from_cache": [list(f) for f in found]} if found else {"applied_from_cache": []}

    def make(seglist, prec):
        p = pkg.Plan(seglist, prec)
        p.capture_graph(stream)
        return p

    def barrier():
        if world > 1:
            dist.barrier()

    def max_over_ranks(v):
        if world == 1:
            return v
        t = torch.tensor([v], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    def time_plan(plan, steps, warmup):
        for _ in range(warmup):
            plan.execute(stream)
        stream.synchronize()
        barrier()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            plan.execute(stream)
        e1.record(stream)
        e1.synchronize()
        ms = e0.elapsed_time(e1) / steps
        barrier()
        torch.cuda.synchronize()
        return max_over_ranks(ms)

    results = {}
    plans = {}
    for prec, name in ((cs.TG_PREC_F64, "fp64"), (cs.TG_PREC_F32_REFINE, "refine")):
        plans[name] = make(segs, prec)
        plans[name + "_scalar"] = make(scal_segs, prec)
        if blk_segs:
            plans[name + "_block"] = make(blk_segs, prec)

    # correctness of the refined solution against the FP64 (bit-exact) one
    plans["fp64"].execute(stream)
    stream.synchronize()
    ref = [s["x"].clone() for s in segs]
    plans["refine"].execute(stream)
    stream.synchronize()
    rc_ref, _ = plans["refine"].status()
    hist = plans["refine"].sweep_histogram(8)
    max_rel = 0.0
    for s, r in zip(segs, ref):
        n = s["ncol"]
        d = (s["x"][..., :n] - r[..., :n]).abs().max().item()
        m = r[..., :n].abs().max().item()
        max_rel = max(max_rel, d / m if m > 0 else d)
    rc64, _ = plans["fp64"].status()
    del ref

    clocks = Clocks(torch.cuda.current_device() if "CUDA_VISIBLE_DEVICES" not in os.environ else local)
    clocks.start()
    # untimed pre-heat so that clocks settle and the sampler sees the load
    t_end = time.time() + 1.0
    while time.time() < t_end:
        for _ in range(20):
            plans["fp64"].execute(stream)
        stream.synchronize()
    for name in ("fp64", "refine"):
        results[name] = time_plan(plans[name], args.steps, args.warmup)
    clk = clocks.stop()
    for name in ("refine_scalar", "fp64_scalar", "refine_block", "fp64_block"):
        if name in plans:
            results[name] = time_plan(plans[name], args.steps, args.warmup)

    # ---- fused assembly + solve routines (dt_ng, minor_ng), device-resident
    assembly = None
    if not args.skip_assembly:
        assembly = {}
        # the kernels each routine runs at this size (41472 columns) in the
        # default assembly form: three passes, comp_ng two above 16384 columns
        for which, kern in (("dt", "k_dt_coefs+k_thomas_post_ring"),
                            ("minor", "k_minor_levels+k_minor_coefs+k_thomas_post_ring"),
                            ("comp", "k_comp_levels+k_comp_rows"),
                            ("settei", "k_settei_levels+k_settei_coefs+k_thomas_post_ring+k_settei_post"),
                            ("oplus", "k_oplus_levels+k_oplus_coefs+k_thomas_post_ring")):
            launch, ncol_a, nbytes = assembly_setup(pkg, wl, which, dev)
            for _ in range(args.warmup):
                launch(stream)
            stream.synchronize()
            barrier()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(args.steps):
                launch(stream)
            e1.record(stream)
            e1.synchronize()
            ms = max_over_ranks(e0.elapsed_time(e1) / args.steps)
            pk, _ = measured_peak()
            ach = nbytes / (ms * 1e-3) / 1e9
            assembly[which + "_ng"] = {
                "kernel": kern, "columns": ncol_a, "levels": wl.grids[0].nk, "ms_per_launch": ms,
                "columns_per_s": world * ncol_a / (ms * 1e-3), "algorithmic_bytes_per_launch": nbytes,
                "roofline": {"bound": "hbm", "achieved": ach, "peak": pk, "unit": "GB/s", "frac": ach / pk,
                             "traffic": traffic_from_profiles(kern, f"{wl.name}_x{ASSEMBLY_REPLICAS}")},
                "inputs": f"{ASSEMBLY_REPLICAS} copies of the {wl.grids[0].name} grid, {nbytes / 1e6:.0f} MB > L2"}
            del launch
        torch.cuda.empty_cache()

    # ---- horizontal operators and the post-solve time filter, device-resident
    horizontal = None
    if not args.skip_assembly:
        horizontal = {}
        for which, name, kern in (("advec", "advec_ng", "k_advec_ng"), ("smooth", "smooth_ng", "k_smooth_ng"),
                                  ("filter", "time_filter_ng", "k_time_filter"), ("ring", "filter_o2o", "k_ringfilter")):
            launch, npts, nbytes = horizontal_setup(pkg, which, dev)
            for _ in range(args.warmup):
                launch(stream)
            stream.synchronize()
            barrier()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(args.steps):
                launch(stream)
            e1.record(stream)
            e1.synchronize()
            ms = max_over_ranks(e0.elapsed_time(e1) / args.steps)
            pk, _ = measured_peak()
            ach = nbytes / (ms * 1e-3) / 1e9
            horizontal[name] = {
                "kernel": kern, "points": npts, "ms_per_launch": ms, "points_per_s": world * npts / (ms * 1e-3),
                "algorithmic_bytes_per_launch": nbytes,
                "roofline": {"bound": "hbm", "achieved": ach, "peak": pk, "unit": "GB/s", "frac": ach / pk,
                             "traffic": traffic_from_profiles(kern, HORIZ_TAG)},
                "inputs": (f"the {HORIZ_TAG} grid held as one subdomain, {nbytes / 1e6:.0f} MB > L2" if which != "ring"
                           else f"the polar rows of the 576 x 288 x 113 global grid, {nbytes / 1e6:.0f} MB, filtered "
                                f"in place launch after launch (L2-resident)")}
            del launch
        torch.cuda.empty_cache()

    # ---- one dynamics_ng step of the column routines per grid, device-resident
    dynamics = None
    if not args.skip_assembly and wl.grids[0].nk >= 3 and len(wl.grids) > 1:
        dynamics = dynamics_leg(pkg, wl, args.steps, args.warmup, stream, max_over_ranks, barrier,
                                cpu=(rank == 0 and not args.skip_cpu))

    peak, peak_kind = measured_peak()
    bytes_scalar = pkg.batch.segment_bytes(scal_segs)          # this rank's share
    wl_tag = f"{wl.name}_B{wl.block}"

    def roofline(name, kernel):
        kernel = plans[name + "_scalar"].describe().split(" ")[0]
        ms = results[name + "_scalar"]
        ach = bytes_scalar / (ms * 1e-3) / 1e9
        tr = traffic_from_profiles(kernel, wl_tag)
        return {"bound": "hbm", "kernel": kernel, "achieved": ach, "peak": peak, "unit": "GB/s", "frac": ach / peak,
                "traffic": tr, "algorithmic_bytes_per_launch": bytes_scalar, "ms_per_launch": ms,
                "peak_source": f"{peak_kind} hbm_gbs (MEASURED_PEAKS.json)" if peak_kind == "measured" else "fallback 6.65 TB/s"}

    # the whole job's unknowns over the slowest rank's time
    vref = unknowns / (results["refine"] * 1e-3)
    value = unknowns / (results["fp64"] * 1e-3)
    launches_per_step = plans["refine"].launches

    # ---- end to end through the host-pointer C ABI: this rank's share of the
    # workload's systems in pinned host memory (Fortran layout), one
    # tg_solve_host call per step, copies in and out inside the timed region
    e2e = None
    cpu = None
    jobs_all = [(g, sub) for g in wl.grids for sub in range(nsub_of(g, args.max_sub))]
    nsys = wl.n_scalar + (1 if wl.block else 0)
    if not args.skip_e2e:
        seg_all = dw.segments()
        mine = pkg.batch.shard_columns([t["ncol"] for t in seg_all],
                                       [(1 if t["kind"] == cs.TG_KIND_SCALAR else t["kind"]) * t["k2"] for t in seg_all],
                                       world, rank, 32)
        need = sum(sum(int(np.prod(shp)) * 8 for sysshp in job_shapes(wl, g) for shp in sysshp) for g, _ in jobs_all)
        avail = host_memory_available()
        # each rank holds only the grid sub-steps its share touches: about
        # `need` over all ranks together
        whole = avail is None or need < 0.5 * avail
        if whole:
            jidx = sorted({i // nsys for i, _, _ in mine})
            hw = HostWorkload(pkg, wl, jobs=[jobs_all[j] for j in jidx], threads=os.cpu_count() or 8, pinned=True)
            pos = {j: n for n, j in enumerate(jidx)}
            flat = []
            for n in range(len(jidx)):   # systems of each job in segment order
                flat += hw.scal[n * wl.n_scalar:(n + 1) * wl.n_scalar] + ([hw.blk[n]] if wl.block else [])
            shares = [(flat[pos[i // nsys] * nsys + i % nsys], c0, c1) for i, c0, c1 in mine]
            what = "this rank's share of every system of the workload"
        else:
            # not enough host memory: one sub-step of each grid, whole columns
            hw = HostWorkload(pkg, wl, jobs=[(g, 0) for g in wl.grids], threads=os.cpu_count() or 8, pinned=True)
            flat = []
            for n in range(len(wl.grids)):
                flat += hw.scal[n * wl.n_scalar:(n + 1) * wl.n_scalar] + ([hw.blk[n]] if wl.block else [])
            shares = [(t, 0, t[0].shape[-1]) for t in flat]
            what = (f"one sub-step of each grid (the whole step needs {need / 1e9:.0f} GB of pinned host "
                    f"memory, {avail / 1e9:.0f} GB available)")
        systems = []
        h2d = d2h = e2e_unk = 0
        for t, c0, c1 in shares:
            v = [a[..., c0:c1] for a in t]
            if v[0].ndim == 2:
                systems.append(dict(kind=cs.TG_KIND_SCALAR, a=v[0], b=v[1], c=v[2], f=v[3], x=v[4], k2=v[0].shape[0]))
            else:
                systems.append(dict(kind=wl.block, a=v[0], b=v[1], c=v[2], f=v[3], x=v[4], k2=v[3].shape[1]))
            h2d += sum(a.nbytes for a in v[:4])
            d2h += v[4].nbytes
            e2e_unk += v[4].size

        def e2e_step():            # one pipelined C-ABI call for the whole step
            cs.solve_host(systems)

        def time_host(fn, steps):
            for _ in range(max(1, min(args.warmup, 2))):
                fn()
            torch.cuda.synchronize()
            barrier()
            t0 = time.perf_counter()
            for _ in range(steps):
                fn()
            torch.cuda.synchronize()
            return max_over_ranks((time.perf_counter() - t0) / steps)
        dt = time_host(e2e_step, args.e2e_steps)
        e2e = {"value": (unknowns if whole else world * e2e_unk) / dt, "unit": "unknowns/s",
               "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h), "ms_per_step": dt * 1e3,
               "steps": args.e2e_steps, "systems_per_call": len(systems),
               "path": f"tg_solve_host, {what} in one call per step, pinned host Fortran-layout arrays, FP64",
               "timer": "host wall clock around synchronous C-ABI calls, max over ranks"}
        # the per-routine drop-ins on the global grid (tg_trsolv_ng per scalar
        # system, tg_blksolve for the block system), one call per system
        if world == 1:
            g0 = flat[:nsys]

            def e2e_percall():
                for t in g0:
                    if t[0].ndim == 2:
                        cs.trsolv_ng(t[0], t[1], t[2], t[3], t[4], t[0].shape[0])
                    else:
                        cs.blksolve(t[0], t[1], t[2], t[3], t[4], t[3].shape[1])
            dt_pc = time_host(e2e_percall, 5)
            unk_pc = sum(t[4].size for t in g0)
            e2e["per_call_drop_ins"] = {"value": unk_pc / dt_pc, "ms_per_step": dt_pc * 1e3,
                                        "path": f"tg_trsolv_ng x{wl.n_scalar} + tg_blksolve on one sub-step of "
                                                f"{wl.grids[0].name}"}
        # the global grid's latitude scan (src/dt.F:126-330): one trsolv per
        # latitude slab of nlon+4 columns, as calls and deferred to one flush
        if world == 1:
            g = wl.grids[0]
            lonmax, nlat, nk = g.nlon + 4, g.nlat, g.nk
            a, b, c, f = pkg.synth.scalar_system(nk, lonmax * nlat, g.dz, 4242, wl.d0_range, wl.loss, wl.d_span)
            shp = (nk, lonmax, nlat)
            a, b, c, f = (np.asfortranarray(v.reshape(shp, order="F")) for v in (a, b, c, f))
            xs = np.zeros(shp, order="F")
            work = [np.zeros((nk, lonmax), order="F") for _ in range(4)]
            scan_args = (1, nk, 1, nk - 1, 1, lonmax, lonmax)

            def scan(defer):
                for lat in range(nlat):
                    for w, v in zip(work, (a, b, c, f)):
                        w[...] = v[:, :, lat]          # the scan's per-latitude work arrays
                    if defer:
                        cs.trsolv_defer(*work, xs[:, :, lat], *scan_args)
                    else:
                        cs.trsolv(*work, xs[:, :, lat], *scan_args)
                if defer:
                    cs.trsolv_flush()
            t_slab = time_host(lambda: scan(False), 5)
            x_slab = xs.copy()
            t_defer = time_host(lambda: scan(True), 5)
            e2e["per_latitude"] = {"per_slab_ms": t_slab * 1e3, "deferred_ms": t_defer * 1e3,
                                   "same_bits": bool(np.array_equal(x_slab, xs)),
                                   "scan": f"{nlat} latitude slabs of {lonmax} x {nk} (one scalar system of "
                                           f"{g.name}), tg_trsolv per slab vs tg_trsolv_defer + one "
                                           f"tg_trsolv_flush, host wall clock"}
        # the link this path is bound by: pinned host<->device copy bandwidth
        nb = min(h2d, 1 << 30) // 8
        hbuf = torch.empty(nb, dtype=torch.float64, pin_memory=True)
        dbuf = torch.empty(nb, dtype=torch.float64, device=dev)
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
        cstream = torch.cuda.Stream(device=dev)
        with torch.cuda.stream(cstream):
            dbuf.copy_(hbuf, non_blocking=True)
            ev[0].record(cstream)
            dbuf.copy_(hbuf, non_blocking=True)
            ev[1].record(cstream)
            hbuf.copy_(dbuf, non_blocking=True)
            ev[2].record(cstream)
        cstream.synchronize()
        h2d_gbs = nb * 8 / (ev[0].elapsed_time(ev[1]) * 1e-3) / 1e9
        d2h_gbs = nb * 8 / (ev[1].elapsed_time(ev[2]) * 1e-3) / 1e9
        e2e["link"] = {"h2d_GBps": h2d_gbs, "d2h_GBps": d2h_gbs, "h2d_bound_ms_per_step": h2d / h2d_gbs / 1e6}
        del hbuf, dbuf, systems, shares, flat, hw

    if rank == 0 and not args.skip_cpu and world == 1:
        # the oracle port on a bounded sample of the same workload: one
        # sub-step of each grid, repeated for --cpu-seconds
        orc = ge.load_oracle()
        nthr = orc.max_threads()
        hs = HostWorkload(pkg, wl, jobs=[(g, 0) for g in wl.grids], threads=nthr)
        dt, n = time_host_steps(orc, hs, nthr, seconds=args.cpu_seconds)
        cpu = {"value": hs.unknowns() / dt, "unit": "unknowns/s", "cores": nthr, "kind": "port",
               "sample": f"{n} passes over one sub-step of each grid of the workload ({hs.unknowns()} unknowns, "
                         f"{len(wl.grids)} grids x {nsys} systems), oracle C port (-O2 -ffp-contract=off), OpenMP"}
        del hs

    if rank == 0:
        out = {
            "metric": METRIC,
            "value": value, "unit": "unknowns/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": results["fp64"], "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic (seeded, generated on device)",
            "config": workload_config(pkg, wl, args.max_sub),
            "roofline": roofline("fp64", "k_scalar_f64"),
            "kernels": {k: plans[k].describe() for k in ("fp64", "refine")},
            "tuning": tuning,
            "fp64": {"value": value, "ms_per_step": results["fp64"], "status": cs.STATUS_NAMES[rc64]},
            "refine": {"value": vref, "ms_per_step": results["refine"], "refine_over_fp64": vref / value,
                       "max_rel_err_vs_fp64": max_rel, "sweep_histogram": hist, "status": cs.STATUS_NAMES[rc_ref],
                       "dtype": "f32 sweeps + f64 residual/update (f64 I/O)",
                       "roofline": roofline("refine", "k_scalar_refine")},
            "kernel_ms": {k: v for k, v in results.items()},
            "assembly": assembly,
            "horizontal": horizontal,
            "dynamics": dynamics,
            "cpu_baseline": cpu,
            "e2e": e2e,
            "clocks": clk,
            "gpu_launches": args.steps * launches_per_step,
        }
        print(json.dumps(out))
    for p in plans.values():
        p.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
