"""Autotuner for the column-solve kernels.

For each system kind (scalar, 2x2 block, 3x3 block) and precision it times
every launch shape on the actual segments (a plan of just that kind, replayed
from a CUDA graph, CUDA-event timed) and keeps the fastest:

  FP64      register-prefetch kernel: columns per block x columns per thread x
            prefetch depth, w2 scratch in shared memory ("reg") or global
            memory ("regg")
            bulk-copy ring kernel: staging depth 4, 8 or 16 levels, w2 in shared
            ("ring") or global ("ringg") memory; for block kinds also one lane
            per block row ("rows", depth 4 or 8) and 16 or 8 columns per warp
            ("ring16", "ring8"), and those rings with Gamma resident in shared
            memory ("ringsm", "ring16sm", "ring8sm"); for the scalar kind a ring of stages holding 2, 4
            or 8 levels each ("chunk2", "chunk4", "chunk8"), and the same ring with
            the sweep's w2 ("res1cL") or w2 and w3 ("res2cL") resident in
            shared memory, L levels per stage
  FP32+ref  columns per block x prefetch depth; scalar kind also the
            bulk-copy refinement ring of 2, 3 or 4 stages ("ring") and the
            whole tile held in shared memory ("tile")

Results are cached in a JSON file keyed by GPU name, kind, precision, level
count and a column-count bucket, and applied with tg_set_tile /
tg_set_pipeline before plans are built.
"""
import json
import math
import os

from . import colsolve as cs

CACHE_DEFAULT = os.path.join(os.path.expanduser("~"), ".cache", "tg_colsolve_tune.json")
# choices tuned on a B200 for the benchmark workloads, shipped with the package
PACKAGED = os.path.join(os.path.dirname(os.path.abspath(__file__)), "tuned_b200.json")

SCALAR_F64 = [("reg", 128, 1, 4), ("reg", 256, 1, 4), ("reg", 128, 1, 8), ("reg", 256, 1, 8), ("reg", 64, 1, 16),
              ("reg", 128, 1, 16), ("reg", 128, 2, 4), ("reg", 256, 2, 4), ("reg", 128, 2, 8),
              ("regg", 256, 1, 4), ("regg", 128, 1, 8), ("regg", 128, 1, 16),
              ("ring", 4, 4, 4), ("ring", 8, 4, 4), ("ring", 4, 2, 4),
              ("ringg", 4, 1, 4), ("ringg", 8, 1, 4), ("ringg", 4, 2, 4), ("ringg", 4, 4, 4), ("ringg", 4, 8, 4),
              ("chunk2", 4, 1, 4), ("chunk4", 2, 1, 4), ("chunk4", 3, 1, 4), ("chunk4", 4, 1, 4), ("chunk8", 2, 1, 4),
              ("chunk4", 2, 2, 4),
              ("res1c4", 2, 1, 4), ("res1c4", 3, 1, 4), ("res1c4", 4, 1, 4), ("res1c2", 4, 1, 4),
              ("res2c4", 2, 1, 4), ("res2c4", 3, 1, 4), ("res2c4", 4, 1, 4), ("res2c2", 4, 1, 4), ("res2c4", 2, 2, 4)]
BLOCK_F64 = [("reg", 32, 1, 4), ("reg", 64, 1, 4), ("reg", 128, 1, 4), ("reg", 96, 1, 4),
             ("ring", 4, 4, 4), ("ring", 8, 4, 4), ("ring", 4, 2, 4), ("ring", 8, 2, 4), ("ring", 16, 2, 4),
             ("ring", 4, 1, 4), ("ring16", 4, 1, 4), ("ring16", 8, 1, 4), ("ring16", 4, 2, 4), ("ring8", 4, 1, 4),
             ("ring8", 8, 1, 4), ("ring8", 4, 2, 4), ("rows", 4, 1, 4), ("rows", 4, 2, 4), ("rows", 8, 1, 4),
             ("ringsm", 4, 1, 4), ("ring16sm", 4, 1, 4), ("ring16sm", 8, 1, 4), ("ring8sm", 4, 1, 4),
             ("ring8sm", 8, 1, 4)]
SCALAR_REF = [("reg", 64, 1, 4), ("reg", 128, 1, 4), ("reg", 256, 1, 4), ("reg", 128, 1, 8), ("reg", 64, 1, 8),
              ("ring", 2, 1, 4), ("ring", 3, 1, 4), ("ring", 4, 1, 4), ("ring", 2, 2, 4), ("tile", 2, 1, 4)]
BLOCK_REF = [("reg", 32, 1, 4), ("reg", 64, 1, 4), ("reg", 128, 1, 4), ("ring", 4, 1, 4), ("ring", 8, 1, 4),
             ("ring", 4, 2, 4)]


def candidates(kind, precision):
    if precision == cs.TG_PREC_F64:
        return SCALAR_F64 if kind == cs.TG_KIND_SCALAR else BLOCK_F64
    return SCALAR_REF if kind == cs.TG_KIND_SCALAR else BLOCK_REF


def apply(kind, precision, cand):
    v, p1, p2 = cand[:3]
    pf = cand[3] if len(cand) > 3 else 4
    scalar64 = kind == cs.TG_KIND_SCALAR and precision == cs.TG_PREC_F64
    if kind == cs.TG_KIND_SCALAR:
        cs.set_prefetch(kind, precision, pf)
        if precision != cs.TG_PREC_F64:
            cs.set_column_residency(kind, precision, 1 if v == "tile" else 0)
        if precision == cs.TG_PREC_F64:
            levels = int(v[5:]) if v.startswith("chunk") else int(v[5:]) if v.startswith("res") else 1
            cs.set_stage_levels(kind, precision, levels)
            cs.set_column_residency(kind, precision, int(v[3]) if v.startswith("res") else 0)
    elif precision == cs.TG_PREC_F64:
        cs.set_block_rows(kind, 1 if v == "rows" else 0)
        cs.set_block_width(kind, {"ring16": 16, "ring8": 8, "ring16sm": 16, "ring8sm": 8}.get(v, 32))
        cs.set_column_residency(kind, precision, 1 if v.endswith("sm") else 0)
    if v in ("ring", "ringg", "rows", "ring16", "ring8", "tile") or v.startswith(("chunk", "res", "ring")):
        cs.set_pipeline(kind, precision, p1, p2)    # ring depth, warps per CTA
    else:
        cs.set_pipeline(kind, precision, 0)
        cs.set_tile(kind, precision, p1, p2)
    if scalar64:
        cs.set_scratch_global(kind, precision, 1 if v in ("regg", "ringg") or v.startswith(("chunk", "res")) else 0)


def reset(kind, precision):
    cs.set_tile(kind, precision, 0, 0)
    cs.set_pipeline(kind, precision, -1, 0)
    if kind == cs.TG_KIND_SCALAR:
        cs.set_prefetch(kind, precision, -1)
    if kind == cs.TG_KIND_SCALAR and precision != cs.TG_PREC_F64:
        cs.set_column_residency(kind, precision, -1)
    if kind == cs.TG_KIND_SCALAR and precision == cs.TG_PREC_F64:
        cs.set_scratch_global(kind, precision, -1)
        cs.set_stage_levels(kind, precision, 0)
        cs.set_column_residency(kind, precision, -1)
    if kind != cs.TG_KIND_SCALAR and precision == cs.TG_PREC_F64:
        cs.set_block_rows(kind, -1)
        cs.set_block_width(kind, 0)
        cs.set_column_residency(kind, precision, -1)


def key(gpu, kind, precision, nk, ncol):
    return f"{gpu}|kind{kind}|prec{precision}|nk{nk}|ncol2^{int(math.log2(max(ncol, 1)))}"


def time_segments(segments, precision, stream, reps=20, warmup=3):
    import torch
    plan = cs.Plan(segments, precision)
    try:
        plan.capture_graph(stream)
        for _ in range(warmup):
            plan.execute(stream)
        stream.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(reps):
            plan.execute(stream)
        e1.record(stream)
        e1.synchronize()
        rc, _ = plan.status()
        if rc not in (cs.TG_OK, cs.TG_ENOCONV):
            return math.inf
        return e0.elapsed_time(e1) / reps
    finally:
        plan.close()


def tune(segments, kinds=None, precisions=(cs.TG_PREC_F64, cs.TG_PREC_F32_REFINE), cache=CACHE_DEFAULT,
         reps=20, verbose=False):
    """Times every candidate per kind/precision on `segments` (plan dicts),
    applies the fastest and records it in the cache.  Returns
    {(kind, precision): (best_candidate, best_ms, {candidate: ms})}."""
    import torch
    gpu = torch.cuda.get_device_name()
    stream = torch.cuda.Stream()
    db = {}
    if cache and os.path.exists(cache):
        with open(cache) as fh:
            db = json.load(fh)
    out = {}
    kinds = kinds or sorted({s["kind"] for s in segments})
    for kind in kinds:
        segs = [s for s in segments if s["kind"] == kind]
        if not segs:
            continue
        nk = max(s["k2"] for s in segs)
        ncol = sum(s["ncol"] for s in segs)
        for prec in precisions:
            times = {}
            for cand in candidates(kind, prec):
                apply(kind, prec, cand)
                try:
                    times[cand] = time_segments(segs, prec, stream, reps=reps)
                except cs.TgError:
                    times[cand] = math.inf
                if verbose:
                    print(f"kind {kind} prec {prec} {cand}: {times[cand]:.4f} ms", flush=True)
            best = min(times, key=times.get)
            apply(kind, prec, best)
            out[(kind, prec)] = (best, times[best], times)
            db[key(gpu, kind, prec, nk, ncol)] = {"candidate": list(best), "ms": times[best]}
    # The kinds of one plan run concurrently (scalar beside block), so the
    # fastest shape of each alone may not be the fastest pair: time the best
    # few of each kind together on the whole plan.
    if len(kinds) > 1:
        for prec in precisions:
            tops = []
            for kind in kinds:
                if (kind, prec) not in out:
                    continue
                times = out[(kind, prec)][2]
                tops.append((kind, sorted(times, key=times.get)[:3]))
            if len(tops) < 2:
                continue
            import itertools
            best, best_ms = None, math.inf
            for combo in itertools.product(*[c for _, c in tops]):
                for (kind, _), cand in zip(tops, combo):
                    apply(kind, prec, cand)
                try:
                    ms = time_segments(segments, prec, stream, reps=reps)
                except cs.TgError:
                    ms = math.inf
                if verbose:
                    print(f"combined prec {prec} {combo}: {ms:.4f} ms", flush=True)
                if ms < best_ms:
                    best, best_ms = combo, ms
            for (kind, _), cand in zip(tops, best):
                apply(kind, prec, cand)
                segs = [s for s in segments if s["kind"] == kind]
                db[key(gpu, kind, prec, max(s["k2"] for s in segs), sum(s["ncol"] for s in segs))] = {
                    "candidate": list(cand), "ms": out[(kind, prec)][2][cand], "combined_ms": best_ms}
                out[(kind, prec)] = (cand, out[(kind, prec)][2][cand], out[(kind, prec)][2])
            out[("combined", prec)] = (best, best_ms, {})
    if cache:
        os.makedirs(os.path.dirname(cache), exist_ok=True)
        with open(cache, "w") as fh:
            json.dump(db, fh, indent=1)
    return out


def load(segments, cache=CACHE_DEFAULT):
    """Applies cached choices for these segments; returns the kinds found."""
    import torch
    if not cache or not os.path.exists(cache):
        return []
    with open(cache) as fh:
        db = json.load(fh)
    gpu = torch.cuda.get_device_name()
    found = []
    for kind in sorted({s["kind"] for s in segments}):
        segs = [s for s in segments if s["kind"] == kind]
        nk = max(s["k2"] for s in segs)
        ncol = sum(s["ncol"] for s in segs)
        for prec in (cs.TG_PREC_F64, cs.TG_PREC_F32_REFINE):
            rec = db.get(key(gpu, kind, prec, nk, ncol))
            if rec:
                apply(kind, prec, tuple(rec["candidate"]))
                found.append((kind, prec))
    return found
