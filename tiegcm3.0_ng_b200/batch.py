"""Batched (plan) layout helpers and device-resident synthetic workloads.

Plan layout (level-major, column index fastest, column stride ld):
  scalar (k, col)          -> k*ld + col                 torch shape (nk, ld)
  block matrix (i,j,k,col) -> ((k*B + j)*B + i)*ld + col torch shape (nk, B, B, ld) [k, j, i, col]
  block vector (i,k,col)   -> (k*B + i)*ld + col         torch shape (nk, B, ld)    [k, i, col]
  ubc (i,col)              -> i*ld + col                 torch shape (B, ld)
"""
import math

import numpy as np

from . import synth
from .colsolve import TG_KIND_SCALAR


def pad_ld(ncol, align=32):
    return (ncol + align - 1) // align * align


# ---- numpy Fortran layout <-> torch plan layout ---------------------------
def level_scalar(a, ld, device):
    import torch
    nk, ncol = a.shape[0], a.size // a.shape[0]
    t = torch.zeros((nk, ld), dtype=torch.float64, device=device)
    t[:, :ncol] = torch.from_numpy(np.ascontiguousarray(a.reshape(nk, ncol, order="F")))
    return t


def level_matrix(P, ld, device):
    import torch
    B, nk = P.shape[0], P.shape[2]
    ncol = P.size // (B * B * nk)
    t = torch.zeros((nk, B, B, ld), dtype=torch.float64, device=device)
    t[..., :ncol] = torch.from_numpy(np.ascontiguousarray(np.transpose(P.reshape(B, B, nk, ncol, order="F"), (2, 1, 0, 3))))
    return t


def level_vector(f, ld, device):
    import torch
    B, nk = f.shape[0], f.shape[1]
    ncol = f.size // (B * nk)
    t = torch.zeros((nk, B, ld), dtype=torch.float64, device=device)
    t[..., :ncol] = torch.from_numpy(np.ascontiguousarray(np.transpose(f.reshape(B, nk, ncol, order="F"), (1, 0, 2))))
    return t


def from_level_scalar(t, ncol):
    return np.asfortranarray(t[:, :ncol].cpu().numpy())


def from_level_vector(t, ncol):
    return np.asfortranarray(np.transpose(t[..., :ncol].cpu().numpy(), (1, 0, 2)))


# ---- device-side generation of the synthetic law ----------------------------
def _diffusion_dev(torch, gen, nk, ncol, ld, dz, d0_range, d_span, device):
    k = torch.arange(nk, dtype=torch.float64, device=device)[:, None]
    if d_span is None:
        d0 = torch.empty((1, ld), dtype=torch.float64, device=device).uniform_(d0_range[0], d0_range[1], generator=gen)
        prof = d0 * torch.exp(k * dz)
    else:
        lo, hi = math.log(d_span[0]), math.log(d_span[1])
        e0 = torch.empty((1, ld), dtype=torch.float64, device=device).uniform_(lo, lo + 0.25 * (hi - lo), generator=gen)
        e1 = torch.empty((1, ld), dtype=torch.float64, device=device).uniform_(hi - 0.25 * (hi - lo), hi, generator=gen)
        prof = torch.exp(e0 + (e1 - e0) * k / max(nk - 1, 1))
    ln = torch.empty((nk, ld), dtype=torch.float64, device=device).log_normal_(0.0, 0.3, generator=gen)
    return prof * ln


def _loss_dev(torch, gen, shape, loss, device):
    kind, p0, p1 = loss
    t = torch.empty(shape, dtype=torch.float64, device=device)
    return t.uniform_(p0, p1, generator=gen) if kind == "uniform" else t.log_normal_(p0, p1, generator=gen)


def gen_scalar_device(nk, ncol, ld, dz, gen, d0_range, loss, d_span, device):
    """The scalar law of synth.scalar_system, drawn with a torch generator
    on the device, in plan layout; padding columns hold a benign identity row."""
    import torch
    D = _diffusion_dev(torch, gen, nk, ncol, ld, dz, d0_range, d_span, device)
    a = -D / dz**2
    L = _loss_dev(torch, gen, (nk, ld), loss, device)
    b = 1.0 / synth.DT - 2.0 * a + L
    c = a.clone()
    f = torch.empty((nk, ld), dtype=torch.float64, device=device).uniform_(0.0, 1.0, generator=gen)
    a[0] = 0.0
    c[0] = 0.0
    b[0] = 1.0
    a[-1] = -1.0
    b[-1] = 1.0
    c[-1] = 0.0
    f[-1] = 0.0
    return a, b, c, f


def gen_block_device(B, nk, ncol, ld, dz, gen, d0_range, loss, d_span, device, coupling=0.2):
    """The block law of synth.block_system on the device, plan layout."""
    import torch
    P = torch.zeros((nk, B, B, ld), dtype=torch.float64, device=device)  # [k, j, i, col]
    Q = torch.zeros_like(P)
    R = torch.zeros_like(P)
    for i in range(B):
        a = -_diffusion_dev(torch, gen, nk, ncol, ld, dz, d0_range, d_span, device) / dz**2
        L = _loss_dev(torch, gen, (nk, ld), loss, device)
        P[:, i, i] = a
        R[:, i, i] = a
        Q[:, i, i] = 1.0 / synth.DT - 2.0 * a + L
    for M in (P, Q, R):
        for i in range(B):
            for j in range(B):
                if i != j:
                    u = torch.empty((nk, ld), dtype=torch.float64, device=device).uniform_(-coupling, coupling, generator=gen)
                    M[:, j, i] = u * M[:, i, i]
    for i in range(B):
        off = sum(M[:, j, i].abs() for M in (P, Q, R) for j in range(B)) - P[:, i, i].abs() - R[:, i, i].abs() - Q[:, i, i].abs()
        Q[:, i, i] += off
    f = torch.empty((nk, B, ld), dtype=torch.float64, device=device).uniform_(0.0, 1.0, generator=gen)
    P[0] = 0.0
    R[0] = 0.0
    Q[0] = 0.0
    P[-1] = 0.0
    Q[-1] = 0.0
    R[-1] = 0.0
    for i in range(B):
        Q[0, i, i] = 1.0
        P[-1, i, i] = -1.0
        Q[-1, i, i] = 1.0
    f[-1] = 0.0
    return P, Q, R, f


class DeviceWorkload:
    """Every system of one outer step of a workload, resident on the device
    in plan layout: for each grid and sub-step, the workload's scalar systems
    and (if any) its block system.  segments() gives the Plan segment list."""

    def __init__(self, wl, device="cuda", seed=synth.SEED_BASE, grids=None, max_sub=None):
        import torch
        self.wl = wl
        self.items = []
        gen = torch.Generator(device=device)
        gen.manual_seed(seed)
        for g in (grids or wl.grids):
            nsub = g.nsub if max_sub is None else min(g.nsub, max_sub)
            ld = pad_ld(g.ncol)
            for sub in range(nsub):
                for s in range(wl.n_scalar):
                    a, b, c, f = gen_scalar_device(g.nk, g.ncol, ld, g.dz, gen, wl.d0_range, wl.loss, wl.d_span, device)
                    x = torch.zeros((g.nk, ld), dtype=torch.float64, device=device)
                    self.items.append(dict(kind=TG_KIND_SCALAR, nk=g.nk, k2=g.nk, ncol=g.ncol, ld=ld,
                                           a=a, b=b, c=c, f=f, x=x, grid=g.name, sub=sub))
                if wl.block:
                    P, Q, R, f = gen_block_device(wl.block, g.nk, g.ncol, ld, g.dz, gen, wl.d0_range, wl.loss,
                                                  wl.d_span, device)
                    u = torch.zeros((g.nk, wl.block, ld), dtype=torch.float64, device=device)
                    self.items.append(dict(kind=wl.block, nk=g.nk, k2=g.nk, ncol=g.ncol, ld=ld,
                                           a=P, b=Q, c=R, f=f, x=u, grid=g.name, sub=sub))

    def segments(self, kinds=None):
        return [it for it in self.items if kinds is None or it["kind"] in kinds]

    def unknowns(self, kinds=None):
        return segment_unknowns(self.segments(kinds))

    def algorithmic_bytes(self, kinds=None):
        return segment_bytes(self.segments(kinds))

    def input_bytes(self):
        n = 0
        for it in self.items:
            for k in ("a", "b", "c", "f"):
                n += it[k].numel() * 8
        return n


def segment_unknowns(segs):
    """Unknowns solved by a list of plan segments: B*k2 per column."""
    n = 0
    for it in segs:
        B = 1 if it["kind"] == TG_KIND_SCALAR else it["kind"]
        n += B * it["k2"] * it["ncol"]
    return n


def segment_bytes(segs):
    """FP64 I/O contract bytes of a list of plan segments: 40 B per scalar
    unknown; (3B^2+2B)*8 B per B x B block row."""
    n = 0
    for it in segs:
        if it["kind"] == TG_KIND_SCALAR:
            n += 40 * it["k2"] * it["ncol"]
        else:
            B = it["kind"]
            n += (3 * B * B + 2 * B) * 8 * it["k2"] * it["ncol"]
    return n


# ---- sharding across GPUs -------------------------------------------------------
def shard_columns(ncols, weights, world, rank, align=1):
    """Contiguous share of the flattened column space for one rank.

    Segment i has ncols[i] columns of weight weights[i] (unknowns per column:
    B*k2).  The concatenated columns are cut at multiples of total/world in
    weight, so every column goes to exactly one rank and the ranks' unknowns
    differ by at most one column's weight (align columns' weight when a cut
    inside a segment is rounded up to a multiple of align columns, which
    keeps each share's first column on a tile boundary).  Returns
    [(segment, c0, c1), ...]."""
    total = sum(n * w for n, w in zip(ncols, weights))
    lo = total * rank // world
    hi = total * (rank + 1) // world
    out = []
    start = 0

    def cut(pos, seg_lo, n, w):
        # a column belongs to the rank whose range holds its first unknown;
        # both neighbours of a cut compute it from the same position
        c = -(-(pos - seg_lo) // w)
        return min(n, -(-c // align) * align)

    for i, (n, w) in enumerate(zip(ncols, weights)):
        seg_lo, seg_hi = start, start + n * w
        a, b = max(lo, seg_lo), min(hi, seg_hi)
        if a < b:
            c0 = cut(a, seg_lo, n, w)
            c1 = cut(b, seg_lo, n, w)
            if c1 > c0:
                out.append((i, c0, c1))
        start = seg_hi
    return out


def shard_segments(segments, world, rank, align=32):
    """Plan segments restricted to this rank's columns (views, no copies).
    Cuts inside a segment fall on multiples of `align` columns, so a share
    starts on a 32-column tile with 16-byte aligned rows and keeps the
    bulk-copy kernels."""
    ncols = [s["ncol"] for s in segments]
    weights = [(1 if s["kind"] == TG_KIND_SCALAR else s["kind"]) * s["k2"] for s in segments]
    out = []
    for i, c0, c1 in shard_columns(ncols, weights, world, rank, align):
        s = dict(segments[i])
        for k in ("a", "b", "c", "f", "x", "ubc_ratio", "ubc_add"):
            if s.get(k) is not None:
                s[k] = s[k][..., c0:c1]
        s["ncol"] = c1 - c0
        s["col0"] = c0
        out.append(s)
    return out
