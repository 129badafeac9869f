"""Seeded synthetic column systems with the shapes and value laws of the
benchmark workloads (no model data is available offline).

Scalar law, per system and column, levels k = 0..nk-1 (dz the level spacing):
    D_k = D0 * exp(k*dz) * LogNormal(0, 0.3)
    a_k = c_k = -D_k / dz**2
    b_k = 1/dt - a_k - c_k + L_k,   dt = 60 s
    rhs_k ~ U(0, 1)
with a Dirichlet bottom row (a=c=0, b=1, rhs=x_bot ~ U(0,1)) and a zero-flux
top row (a=-1, b=1, c=0, rhs=0).  exp(k*dz) is exp(z_k - z_bot): on the 5 deg
grid (dz = 0.5) it is exp(0.5k); finer grids keep the same altitude profile
(14 scale heights between the model's zibot=-7 and zitop=7).

Block law (B = 2 for the O2/O pair, 3 for O2/O/He): the diagonal of P, Q, R
is the scalar law of each component; every off-diagonal entry (i,j) of P, Q, R
is U(-0.2, 0.2) times the diagonal entry of row i of the same block; Q_ii is
then raised by the sum of the absolute off-diagonal couplings of row i so that
every block row stays strictly diagonally dominant by 1/dt + L_i.

Everything is FP64, seeded from numpy's PCG64.  Arrays come back in the
reference's Fortran layouts: scalar (nk, ncol), block matrices (B,B,nk,ncol),
block vectors (B,nk,ncol), all order='F' (level index fastest within a column).
"""
from dataclasses import dataclass, field

import numpy as np

DT = 60.0
SEED_BASE = 20261203

# Species order of the seven scalar systems and the block system of a column.
SCALAR_SYSTEMS = ("TN", "OPLUS", "N4S", "NO", "N2D", "AR", "HE")


@dataclass
class Grid:
    """One horizontal grid (global or a nest level) of columns."""
    name: str
    nlon: int
    nlat: int
    nk: int
    dz: float
    nsub: int = 1          # sub-steps of this grid per outer step
    ghost: int = 0         # ghost halo width on each side (nested grids: 2)

    @property
    def ncol(self):
        return (self.nlon + 2 * self.ghost) * (self.nlat + 2 * self.ghost)


@dataclass
class Workload:
    name: str
    grids: list
    n_scalar: int = 7
    block: int = 2                 # 0: no block system, else block size B
    d0_range: tuple = (1e-4, 1e-1)
    loss: tuple = ("lognormal", -6.0, 2.0)
    d_span: tuple = None           # (Dmin, Dmax): log-uniform bottom->top instead of exp(k dz)
    notes: str = ""
    extra: dict = field(default_factory=dict)

    def unknowns_per_step(self):
        n = 0
        for g in self.grids:
            per_col = self.n_scalar * g.nk + (self.block * g.nk if self.block else 0)
            n += per_col * g.ncol * g.nsub
        return n

    def bytes_per_step(self):
        """Algorithmic bytes of the FP64 I/O contract per outer step:
        scalar 40 B per unknown (a,b,c,f in, x out); B x B block rows
        (3*B*B + 2*B) * 8 B per block row."""
        n = 0
        for g in self.grids:
            s = self.n_scalar * g.nk * 40
            if self.block:
                B = self.block
                s += (3 * B * B + 2 * B) * 8 * g.nk
            n += s * g.ncol * g.nsub
        return n


def nest_dims(lat_span, lon_span, dres):
    """Nest interior size with the reference's truncation rule
    (src/advance.F:213-216: n = int(span/d + 1))."""
    return int(lon_span / dres + 1), int(lat_span / dres + 1)


def workload(config):
    """The five benchmark workloads by index (0..4)."""
    if config == 0:
        return Workload("5deg_trsolv_72x36x29", [Grid("global5", 72, 36, 29, 0.5)],
                        n_scalar=1, block=0, d0_range=(1e-3, 1e-2), loss=("uniform", 0.0, 1e-3))
    if config == 1:
        return Workload("2.5deg_column_step_144x72x57", [Grid("global2.5", 144, 72, 57, 0.25)])
    if config == 2:
        return Workload("1.25deg_144x288x113_widerange", [Grid("global1.25", 288, 144, 113, 0.125)],
                        d_span=(1e-5, 1e2))
    if config == 3:
        g = [Grid("global2.5", 144, 72, 57, 0.25)]
        sub = 1
        for i, (la, lo, d, n) in enumerate(((40, 60, 0.625, 4), (15, 20, 0.3125, 8), (5, 8, 0.15625, 16))):
            sub *= n
            nlon, nlat = nest_dims(la, lo, d)
            g.append(Grid(f"nest{i+1}", nlon, nlat, 57, 0.25, nsub=sub, ghost=2))
        return Workload("2.5deg_global_plus_3_nests", g)
    if config == 4:
        nlon, nlat = nest_dims(20, 30, 0.15625)
        return Workload("0.625deg_576x288x113_plus_nest",
                        [Grid("global0.625", 576, 288, 113, 0.125),
                         Grid("nest1", nlon, nlat, 113, 0.125, nsub=4, ghost=2)],
                        d_span=(1e-5, 1e2))
    raise ValueError(f"unknown workload {config}")


def _rng(seed):
    return np.random.Generator(np.random.PCG64(seed))


def _diffusion(rng, nk, ncol, dz, d0_range, d_span):
    k = np.arange(nk, dtype=np.float64)[:, None]
    if d_span is None:
        d0 = rng.uniform(d0_range[0], d0_range[1], size=(1, ncol))
        prof = d0 * np.exp(k * dz)
    else:
        lo, hi = np.log(d_span[0]), np.log(d_span[1])
        # log-uniform endpoints per column, bottom to top
        e0 = rng.uniform(lo, lo + 0.25 * (hi - lo), size=(1, ncol))
        e1 = rng.uniform(hi - 0.25 * (hi - lo), hi, size=(1, ncol))
        prof = np.exp(e0 + (e1 - e0) * k / max(nk - 1, 1))
    return prof * rng.lognormal(0.0, 0.3, size=(nk, ncol))


def _loss(rng, shape, loss):
    kind, p0, p1 = loss
    if kind == "uniform":
        return rng.uniform(p0, p1, size=shape)
    return rng.lognormal(p0, p1, size=shape)


def scalar_system(nk, ncol, dz, seed, d0_range=(1e-3, 1e-2), loss=("uniform", 0.0, 1e-3),
                  d_span=None, top_extra=0.0):
    """One scalar tridiagonal system per column: returns (a, b, c, f), each
    (nk, ncol) Fortran-ordered float64."""
    rng = _rng(seed)
    D = _diffusion(rng, nk, ncol, dz, d0_range, d_span)
    L = _loss(rng, (nk, ncol), loss)
    a = -D / dz**2
    c = a.copy()
    b = 1.0 / DT - a - c + L
    f = rng.uniform(0.0, 1.0, size=(nk, ncol))
    # Dirichlet bottom row
    a[0] = 0.0
    c[0] = 0.0
    b[0] = 1.0
    f[0] = rng.uniform(0.0, 1.0, size=ncol)
    # zero-flux top row
    a[-1] = -1.0
    b[-1] = 1.0 + top_extra
    c[-1] = 0.0
    f[-1] = 0.0
    return tuple(np.asfortranarray(v) for v in (a, b, c, f))


def block_system(B, nk, ncol, dz, seed, d0_range=(1e-4, 1e-1), loss=("lognormal", -6.0, 2.0),
                 d_span=None, coupling=0.2):
    """One B x B block-tridiagonal system per column: returns (P, Q, R, f)
    with P, Q, R (B,B,nk,ncol) and f (B,nk,ncol), Fortran-ordered float64."""
    rng = _rng(seed)
    P = np.zeros((B, B, nk, ncol))
    Q = np.zeros((B, B, nk, ncol))
    R = np.zeros((B, B, nk, ncol))
    for i in range(B):
        D = _diffusion(rng, nk, ncol, dz, d0_range, d_span)
        L = _loss(rng, (nk, ncol), loss)
        a = -D / dz**2
        P[i, i] = a
        R[i, i] = a
        Q[i, i] = 1.0 / DT - 2.0 * a + L
    for M in (P, Q, R):
        for i in range(B):
            for j in range(B):
                if i != j:
                    M[i, j] = rng.uniform(-coupling, coupling, size=(nk, ncol)) * M[i, i]
    off = np.zeros((B, nk, ncol))
    for i in range(B):
        s = np.abs(P[i]).sum(axis=0) - np.abs(P[i, i]) + np.abs(R[i]).sum(axis=0) - np.abs(R[i, i])
        s += np.abs(Q[i]).sum(axis=0) - np.abs(Q[i, i])
        off[i] = s
    for i in range(B):
        Q[i, i] += off[i]
    f = rng.uniform(0.0, 1.0, size=(B, nk, ncol))
    # Dirichlet bottom block row, zero-flux top block row
    P[:, :, 0] = 0.0
    R[:, :, 0] = 0.0
    Q[:, :, 0] = 0.0
    P[:, :, -1] = 0.0
    Q[:, :, -1] = 0.0
    R[:, :, -1] = 0.0
    for i in range(B):
        Q[i, i, 0] = 1.0
        P[i, i, -1] = -1.0
        Q[i, i, -1] = 1.0
    f[:, -1] = 0.0
    return tuple(np.asfortranarray(v) for v in (P, Q, R, f))


def column_step(wl, grid, sub=0, sys_count=None):
    """All systems of one grid's sub-step: returns (scalars, block) where
    scalars is a list of (a,b,c,f) and block is (P,Q,R,f) or None."""
    gi = [g.name for g in wl.grids].index(grid.name)
    base = SEED_BASE + 1000 * gi + 97 * sub
    ns = wl.n_scalar if sys_count is None else min(sys_count, wl.n_scalar)
    scal = [scalar_system(grid.nk, grid.ncol, grid.dz, base + s, wl.d0_range, wl.loss, wl.d_span)
            for s in range(ns)]
    blk = None
    if wl.block:
        blk = block_system(wl.block, grid.nk, grid.ncol, grid.dz, base + 50, wl.d0_range, wl.loss, wl.d_span)
    return scal, blk


# ---------------------------------------------------------------------------
# Physical inputs of the column assembly (dt_ng)
# ---------------------------------------------------------------------------
def level_constants(nk, dz, zibot=-7.0, dif0=5.0e-6, prndtl=1.0):
    """expz, expzmid, expzmid_inv, difk, dift of one grid, built by the
    recurrences of src/set_const_fields_ng.F90:50-60 (difk/dift start from the
    bottom-level background values of src/cons.F:244-249)."""
    expdz = np.exp(-dz)
    expz = np.empty(nk)
    difk = np.empty(nk)
    dift = np.empty(nk)
    expz[0] = np.exp(-zibot - .5 * dz)
    difk[0] = dif0
    dift[0] = dif0 / prndtl
    for k in range(1, nk):
        expz[k] = expz[k - 1] * expdz
        difk[k] = difk[k - 1] * expdz
        dift[k] = dift[k - 1] * expdz
    expzmid = np.exp(-.5 * dz)
    return dict(expz=expz, expzmid=expzmid, expzmid_inv=1. / expzmid, difk=difk, dift=dift)


DT_FIELDS = ("tn", "tnsmooth", "horadv", "un", "vn", "o1", "mbar", "xnmbar", "scht", "schti", "cp", "kt", "km",
             "hdt", "qji_tn", "cool_imp", "cool_exp", "w", "qtotal", "rkm12")
DT_2D = ("tlbc", "t_lbc", "ulbc", "vlbc")


def dt_inputs(nk, ncol, dz, seed, step=60.0):
    """Seeded physical fields of the dt_ng column assembly with the model's
    magnitudes (CGS units, as in the reference): Tn rising from ~200 K to
    ~1000 K, scale heights of 1e6-6e6 cm, specific heat ~1e7 erg/g/K, and so on.
    Returns (fields dict of (nk,ncol) / (ncol) / (nk) arrays, constants dict)."""
    rng = _rng(seed)
    z = np.linspace(0.0, 1.0, nk)[:, None]
    U = lambda lo, hi, shape=(nk, ncol): rng.uniform(lo, hi, size=shape)
    f = {}
    tn = 200.0 + 800.0 * z ** 0.7 * U(0.9, 1.1)
    f["tn"] = tn
    f["tnsmooth"] = tn * U(0.99, 1.01)
    f["horadv"] = U(-1e-3, 1e-3)
    f["un"] = U(-5e3, 5e3)
    f["vn"] = U(-5e3, 5e3)
    f["o1"] = 0.05 + 0.8 * z * U(0.9, 1.1)
    f["mbar"] = 28.0 - 12.0 * z * U(0.95, 1.05)
    f["xnmbar"] = 1e13 * np.exp(-10.0 * z) * U(0.5, 1.5)
    f["scht"] = 1e6 + 5e6 * z * U(0.9, 1.1)
    f["schti"] = f["scht"] * U(0.95, 1.05)
    f["cp"] = 1e7 * (1.0 + 0.5 * z) * U(0.95, 1.05)
    f["kt"] = 10.0 * tn ** 0.69 * U(0.9, 1.1)
    f["km"] = 3e-4 * tn ** 0.69 * U(0.9, 1.1)
    f["hdt"] = U(-1e-2, 1e-2)
    f["qji_tn"] = U(0.0, 1e-2)
    f["cool_imp"] = U(1e-6, 1e-4)
    f["cool_exp"] = U(-1e-3, 1e-3)
    f["w"] = U(-1e-4, 1e-4)
    f["qtotal"] = U(0.0, 5e-2) * (1.0 + z)
    f["rkm12"] = U(1e-33, 1e-32)
    for k in DT_FIELDS:
        f[k] = np.asfortranarray(f[k])
    f["tlbc"] = rng.uniform(190.0, 210.0, ncol)
    f["t_lbc"] = rng.uniform(190.0, 210.0, ncol)
    f["ulbc"] = rng.uniform(-1e3, 1e3, ncol)
    f["vlbc"] = rng.uniform(-1e3, 1e3, ncol)
    lc = level_constants(nk, dz)
    f["expz"], f["dift"] = lc["expz"], lc["dift"]
    c = dict(dz=dz, dtx2inv=1.0 / (2.0 * step), expzmid_inv=lc["expzmid_inv"], grav=870.0, p0=5.0e-4,
             avo=6.023e23, gask=8.314e7, tsurplus=5.11 * 1.602e-12, rmassinv_o1=1.0 / 16.0)
    return f, c


MINOR_FIELDS = ("tn", "o2", "o1", "he", "mbar", "barm", "xnmbar", "w", "ftm1_smooth", "hadvec", "sloss", "sprod")
MINOR_2D = ("tlbc", "flbc1", "flbc2", "flbc3", "fubc", "dfactor")


def minor_inputs(nk, ncol, dz, seed, step=60.0, rmx=30.0):
    """Seeded fields of the minor_ng column assembly with the model's
    magnitudes (CGS units): major-species mass mixing ratios O2 0.22 -> 0.01,
    O 0.05 -> 0.8, He 1e-5 -> 0.05, a minor species near 1e-7, and a lower
    boundary that mixes Robin (flbc1 != 0) and Dirichlet (flbc1 = 0) columns.
    Returns (fields dict of (nk,ncol) / (ncol) / (nk) arrays, constants dict)."""
    rng = _rng(seed)
    z = np.linspace(0.0, 1.0, nk)[:, None]
    U = lambda lo, hi, shape=(nk, ncol): rng.uniform(lo, hi, size=shape)
    f = {}
    f["tn"] = 200.0 + 800.0 * z ** 0.7 * U(0.9, 1.1)
    f["o2"] = (0.22 - 0.21 * z) * U(0.9, 1.1)
    f["o1"] = (0.05 + 0.75 * z) * U(0.9, 1.1)
    f["he"] = (1e-5 + 0.05 * z ** 2) * U(0.9, 1.1)
    f["mbar"] = 1.0 / (f["o2"] / 32.0 + f["o1"] / 16.0 + f["he"] / 4.0 +
                       (1.0 - f["o2"] - f["o1"] - f["he"]) / 28.0)
    f["barm"] = f["mbar"] * U(0.99, 1.01)
    f["xnmbar"] = 1e13 * np.exp(-10.0 * z) * U(0.5, 1.5)
    f["w"] = U(-1e-4, 1e-4)
    f["ftm1_smooth"] = 1e-7 * (1.0 + z) * U(0.5, 1.5)
    f["hadvec"] = U(-1e-12, 1e-12)
    f["sloss"] = U(1e-6, 1e-3)
    f["sprod"] = U(0.0, 1e-10) * f["xnmbar"] / rmx
    for k in MINOR_FIELDS:
        f[k] = np.asfortranarray(f[k])
    f["tlbc"] = rng.uniform(190.0, 210.0, ncol)
    f["flbc1"] = np.where(rng.uniform(size=ncol) < 0.5, 0.0, rng.uniform(0.5, 1.0, ncol))
    f["flbc2"] = rng.uniform(0.5, 1.5, ncol)
    f["flbc3"] = rng.uniform(-1e-7, 0.0, ncol)
    f["fubc"] = rng.uniform(0.0, 1e8, ncol)
    f["dfactor"] = rng.uniform(1.0, 2.0, ncol)
    lc = level_constants(nk, dz)
    f["expz"], f["difk"] = lc["expz"], lc["difk"]
    phix = np.array([rng.uniform(0.7, 1.0), rng.uniform(0.7, 1.0), rng.uniform(0.8, 1.1), rng.uniform(0.0, 0.2)])
    b = np.eye(3) * rng.uniform(0.6, 0.9, 3) + rng.uniform(-0.05, 0.05, (3, 3))
    c = dict(rmx=rmx, alfax=rng.uniform(-0.4, 0.0), phix=phix, dzp=dz, dtx2inv=1.0 / (2.0 * step),
             expzmid=lc["expzmid"], expzmid_inv=lc["expzmid_inv"],
             rmassinv_o2=1.0 / 32.0, rmassinv_o1=1.0 / 16.0, rmassinv_n2=1.0 / 28.0, rmassinv_he=1.0 / 4.0,
             rmass_o2=32.0, rmass_o1=16.0, rmass_he=4.0, rmass_n2=28.0, p0=5.0e-4, grav=870.0, avo=6.023e23,
             b=b, fb=rng.uniform(0.0, 0.02, 3))
    return f, c


COMP_FIELDS = ("tn", "o2", "o1", "he", "w", "mbar", "o2nm_smooth", "o1nm_smooth", "henm_smooth",
               "o2_advec", "o1_advec", "he_advec", "hdo2", "hdo1", "hdhe")
COMP_2D = ("tlbc", "flx_he", "dfactor")


def comp_inputs(nk, ncol, dz, seed, step=60.0, calc_helium=1):
    """Seeded fields of the comp_ng column step with the model's magnitudes:
    O2/O/He mass mixing ratios as in minor_inputs, production and a loss
    matrix fs(nk, ncol, 3, 0:3) (slab m*3+isp of a (12, ncol, nk) array,
    i.e. the reference's Fortran order), and an upper-boundary He flux.
    Returns (fields dict, constants dict)."""
    rng = _rng(seed)
    z = np.linspace(0.0, 1.0, nk)[:, None]
    U = lambda lo, hi, shape=(nk, ncol): rng.uniform(lo, hi, size=shape)
    f = {}
    f["tn"] = 200.0 + 800.0 * z ** 0.7 * U(0.9, 1.1)
    f["o2"] = (0.22 - 0.21 * z) * U(0.9, 1.1)
    f["o1"] = (0.05 + 0.75 * z) * U(0.9, 1.1)
    f["he"] = (1e-5 + 0.05 * z ** 2) * U(0.9, 1.1)
    f["mbar"] = 1.0 / (f["o2"] / 32.0 + f["o1"] / 16.0 + f["he"] / 4.0 +
                       (1.0 - f["o2"] - f["o1"] - f["he"]) / 28.0)
    f["w"] = U(-1e-4, 1e-4)
    for s in ("o2", "o1", "he"):
        f[s + "nm_smooth"] = f[s] * U(0.99, 1.01)
        f[s + "_advec"] = f[s] * U(-1e-6, 1e-6)
    f["hdo2"], f["hdo1"], f["hdhe"] = (U(-1e-9, 1e-9) for _ in range(3))
    for k in COMP_FIELDS:
        f[k] = np.asfortranarray(f[k])
    fs = np.empty((12, ncol, nk))
    fs[0:3] = rng.uniform(0.0, 1e-8, size=(3, ncol, nk))                 # production fs(:,:,isp,0)
    fs[3:12] = rng.uniform(-1e-6, 1e-6, size=(9, ncol, nk))              # loss fs(:,:,isp,m)
    for isp in range(3):
        fs[3 + isp * 3 + isp] = rng.uniform(1e-6, 1e-4, size=(ncol, nk))  # diagonal loss
    f["fs"] = fs
    f["tlbc"] = rng.uniform(190.0, 210.0, ncol)
    f["flx_he"] = rng.uniform(-1e-13, 1e-13, ncol)
    f["dfactor"] = rng.uniform(1.0, 2.0, ncol)
    lc = level_constants(nk, dz)
    f["expz"], f["difk"] = lc["expz"], lc["difk"]
    b = np.eye(3) * rng.uniform(0.6, 0.9, 3) + rng.uniform(-0.05, 0.05, (3, 3))
    c = dict(dz=dz, dtx2inv=1.0 / (2.0 * step), expzmid=lc["expzmid"], expzmid_inv=lc["expzmid_inv"],
             rmassinv_o2=1.0 / 32.0, rmassinv_o1=1.0 / 16.0, rmassinv_he=1.0 / 4.0, rmassinv_n2=1.0 / 28.0,
             rmass_o2=32.0, rmass_o1=16.0, rmass_he=4.0, p0=5.0e-4, grav=870.0, b=b, fb=rng.uniform(0.0, 0.02, 3),
             pshelb=0.1154e-5, calc_helium=calc_helium)
    return f, c


def comp_post_inputs(nk, ncol, dz, seed, zibot=-7.0):
    """Fields of the comp_ng post-solve steps: the current and previous
    O2/O/He, N2 number-density factors, level midpoints and a solution whose
    N2 drops below 0.01 in the upper levels of about half the columns."""
    rng = _rng(seed)
    z = np.linspace(0.0, 1.0, nk)[:, None]
    U = lambda lo, hi, shape=(nk, ncol): rng.uniform(lo, hi, size=shape)
    f = {}
    for pre in ("", "_nm", "_upd"):
        # N2 decays from 0.78 to 0.002-0.04 at the top; O2, He and O share the rest
        n2 = 0.78 * np.exp(-rng.uniform(3.0, 6.0, size=(1, ncol)) * z) * U(0.98, 1.02)
        rest = 1.0 - n2
        f["o2" + pre] = rest * (0.28 - 0.27 * z) * U(0.9, 1.1)
        f["he" + pre] = rest * (1e-5 + 0.1 * z ** 2) * U(0.5, 1.5)
        f["o1" + pre] = rest - f["o2" + pre] - f["he" + pre]
    f["xnmbar"] = 1e13 * np.exp(-10.0 * z) * U(0.5, 1.5)
    for k in list(f):
        f[k] = np.asfortranarray(f[k])
    f["zpmid"] = zibot + (np.arange(nk) + 0.5) * dz
    return f, dict(dz=dz, dtsmooth=0.95, dtsmooth_div2=0.5 * (1.0 - 0.95))


SETTEI_FIELDS = ("tn", "o2", "o1", "he", "n2", "ne", "te", "ti", "op", "o2p", "nplus", "n2p", "nop", "xnmbar",
                 "xnmbari", "scht", "schti", "qji_ti", "qop2p", "qop2d", "qo2p", "qop", "qn2p", "qnp", "qnop",
                 "Q1", "Q2")
SETTEI_2D = ("t_lbc", "chi", "rlatm", "dipmag", "qteaur")


def settei_inputs(nk, ncol, dz, seed, et=0, electron_heating=0):
    """Seeded fields of the settei_ng column step (CGS): neutral, electron and
    ion temperatures (Te >= Tn, a few columns with Te = Tn), species mixing
    ratios, ion and electron densities, ionisation rates and the solar zenith
    and magnetic latitude / dip angles spanning the branches of the
    upper-boundary flux.  Returns (fields dict, constants dict, qtotal)."""
    rng = _rng(seed)
    z = np.linspace(0.0, 1.0, nk)[:, None]
    U = lambda lo, hi, shape=(nk, ncol): rng.uniform(lo, hi, size=shape)
    f = {}
    tn = 200.0 + 800.0 * z ** 0.7 * U(0.9, 1.1)
    f["tn"] = tn
    te = tn + 2500.0 * z ** 1.5 * U(0.5, 1.5)
    te[:, :3] = tn[:, :3]                     # Te = Tn columns take the |Te-Tn| < del branch
    f["te"] = te
    f["ti"] = tn + 0.5 * (te - tn) * U(0.5, 1.0)
    f["o2"] = (0.22 - 0.21 * z) * U(0.9, 1.1)
    f["o1"] = (0.05 + 0.75 * z) * U(0.9, 1.1)
    f["he"] = (1e-5 + 0.05 * z ** 2) * U(0.9, 1.1)
    f["n2"] = np.maximum(1.0 - f["o2"] - f["o1"] - f["he"], 0.0)
    f["xnmbar"] = 1e13 * np.exp(-10.0 * z) * U(0.5, 1.5)
    f["xnmbari"] = f["xnmbar"] * U(0.95, 1.05)
    f["ne"] = 1e3 + 1e6 * np.exp(-((z - 0.6) / 0.25) ** 2) * U(0.5, 1.5)
    f["op"] = 0.8 * f["ne"] * z * U(0.9, 1.1)
    f["o2p"] = 0.1 * f["ne"] * (1.0 - z) * U(0.9, 1.1)
    f["nplus"] = 0.02 * f["ne"] * U(0.5, 1.5)
    f["n2p"] = 0.01 * f["ne"] * U(0.5, 1.5)
    f["nop"] = 0.1 * f["ne"] * (1.0 - z) * U(0.9, 1.1)
    f["scht"] = 1e6 + 5e6 * z * U(0.9, 1.1)
    f["schti"] = f["scht"] * U(0.95, 1.05)
    f["qji_ti"] = U(0.0, 1e-3)
    for k in ("qop2p", "qop2d", "qo2p", "qop", "qn2p", "qnp", "qnop"):
        f[k] = U(0.0, 1.0) * np.exp(-((z - 0.5) / 0.3) ** 2)
    f["Q1"] = U(0.0, 1e-11)
    f["Q2"] = U(-2e-12, 1e-11)
    for k in SETTEI_FIELDS:
        f[k] = np.asfortranarray(f[k])
    f["t_lbc"] = rng.uniform(190.0, 210.0, ncol)
    f["chi"] = rng.uniform(0.0, np.pi, ncol)               # crosses 80-100 deg and pi/2
    f["rlatm"] = rng.uniform(-np.pi / 2, np.pi / 2, ncol)  # all three branches of a
    f["dipmag"] = rng.uniform(-np.pi / 2, np.pi / 2, ncol)
    f["qteaur"] = rng.uniform(-1e8, 0.0, ncol)
    b = np.eye(3) * rng.uniform(0.6, 0.9, 3) + rng.uniform(-0.05, 0.05, (3, 3))
    c = dict(f107=rng.uniform(70.0, 300.0), dipmin=0.17, dz=dz, evergs=1.602e-12, avo=6.023e23, rmass_o1=16.0,
             rmassinv_o2=1.0 / 32.0, rmassinv_o1=1.0 / 16.0, rmassinv_he=1.0 / 4.0, rmassinv_n2=1.0 / 28.0,
             rmassinv_n4s=1.0 / 14.0, rmassinv_no=1.0 / 30.0, b=b, fb=rng.uniform(0.0, 0.02, 3), et=et,
             electron_heating=electron_heating)
    qtotal = np.asfortranarray(rng.uniform(0.0, 5e-2, (nk, ncol)))
    return f, c, qtotal


OPLUS_FIELDS = ("tn", "te", "ti", "o2", "o1", "n2", "he", "n2d", "ne", "u", "v", "w", "wi", "xnmbar", "scht",
                "qop2p", "qop2d", "qop", "rk1", "rk2", "rk19", "rk20", "rk25", "op", "optm1_smooth2", "explicit_h",
                "bdotdh_djbz")
OPLUS_2D = ("bx", "by", "bz", "dvb", "rlatm", "chi", "dipmag", "sndec", "csdec")


def oplus_inputs(nk, ncol, dz, seed, step=60.0, nstep_sub=10, opdiffcap=0.0):
    """Seeded fields of the oplus_ng vertical column step (CGS): neutral /
    ion / electron temperatures, composition, winds and ion drifts, O+ and
    its production, the temperature-dependent rate fields, the horizontal
    terms the host model supplies (explicit_h, bdotdh_djbz, dvb) and a
    magnetic field with |bz| >= 0.2.  Returns (fields dict, constants dict)."""
    rng = _rng(seed)
    z = np.linspace(0.0, 1.0, nk)[:, None]
    U = lambda lo, hi, shape=(nk, ncol): rng.uniform(lo, hi, size=shape)
    f = {}
    f["tn"] = 200.0 + 800.0 * z ** 0.7 * U(0.9, 1.1)
    f["te"] = f["tn"] + 2000.0 * z * U(0.5, 1.5)
    f["ti"] = f["tn"] + 0.5 * (f["te"] - f["tn"]) * U(0.5, 1.0)
    f["o2"] = (0.22 - 0.21 * z) * U(0.9, 1.1)
    f["o1"] = (0.05 + 0.75 * z) * U(0.9, 1.1)
    f["he"] = (1e-5 + 0.05 * z ** 2) * U(0.9, 1.1)
    f["n2"] = np.maximum(1.0 - f["o2"] - f["o1"] - f["he"], 1e-3)
    f["n2d"] = 1e-6 * U(0.5, 1.5)
    f["ne"] = 1e3 + 1e6 * np.exp(-((z - 0.6) / 0.25) ** 2) * U(0.5, 1.5)
    f["u"], f["v"] = U(-1e4, 1e4), U(-1e4, 1e4)
    f["w"], f["wi"] = U(-1e-4, 1e-4), U(-1e-4, 1e-4)
    f["xnmbar"] = 1e13 * np.exp(-10.0 * z) * U(0.5, 1.5)
    f["scht"] = 1e6 + 5e6 * z * U(0.9, 1.1)
    f["qop2p"], f["qop2d"], f["qop"] = (U(0.0, 10.0) * np.exp(-((z - 0.5) / 0.3) ** 2) + 1e-3 for _ in range(3))
    f["rk1"], f["rk2"] = U(1e-11, 3e-11), U(1e-12, 2e-12)
    f["rk19"], f["rk20"], f["rk25"] = U(1e-7, 2e-7), U(1e-7, 2e-7), U(1e-7, 2e-7)
    f["op"] = 0.8 * f["ne"] * z * U(0.9, 1.1) + 1.0
    f["optm1_smooth2"] = f["op"] * U(0.99, 1.01)
    f["explicit_h"] = f["op"] * U(-1e-4, 1e-4)
    f["bdotdh_djbz"] = U(-1e3, 1e3)
    for k in OPLUS_FIELDS:
        f[k] = np.asfortranarray(f[k])
    f["bx"], f["by"] = rng.uniform(-0.5, 0.5, ncol), rng.uniform(-0.5, 0.5, ncol)
    f["bz"] = rng.choice([-1.0, 1.0], ncol) * rng.uniform(0.2, 1.0, ncol)
    f["dvb"] = rng.uniform(-1e-9, 1e-9, ncol)
    f["rlatm"] = rng.uniform(-np.pi / 2, np.pi / 2, ncol)
    f["chi"] = rng.uniform(0.0, np.pi, ncol)
    f["dipmag"] = rng.uniform(-np.pi / 2, np.pi / 2, ncol)
    f["sndec"], f["csdec"] = rng.uniform(-0.2, 0.2, ncol), rng.uniform(0.9, 1.0, ncol)
    f["zpint"] = -7.0 + np.arange(nk) * dz
    c = dict(rmass_op=16.0, gask=8.314e7, grav=870.0, re=6.37122e8, rmassinv_o2=1 / 32., rmassinv_o1=1 / 16.,
             rmassinv_n2=1 / 28., rmassinv_n2d=1 / 14., rmassinv_he=1 / 4., rk10=1.3E-10, rk16=4.8E-10, rk17=1.0E-10,
             rk18=4.0E-10, rk21=0.047, rk22=0.171, rk23=8.E-10, rk24=5.0E-12, rk26=7.E-10, rk27=7.7E-5, colfac=1.5,
             opdiffcap=opdiffcap, dtx2inv=1.0 / (2.0 * step), dz=dz, dlev=dz, nstep_sub=nstep_sub)
    return f, c


# ---------------------------------------------------------------------------
# Global fields for the polar ring filter (ringfilter, filter_o2o)
# ---------------------------------------------------------------------------
# Chunk counts of the ring filter by latitude row from each pole, per global
# resolution (nlon, nlat): the model's constants (src/cons.F:331-355).
RING_CHUNKS = {
    (72, 36): (3, 9, 18, 36, 36),
    (144, 72): (3, 3, 9, 9, 18, 18, 36, 36, 72, 72),
    (288, 144): (3, 3, 3, 9, 9, 9, 18, 18, 18, 36, 36, 36, 72, 72, 72, 72, 144, 144, 144, 144, 144),
    (576, 288): (3, 3, 3, 3, 3, 9, 9, 9, 9, 9, 18, 18, 18, 18, 18, 18, 36, 36, 36, 36, 36, 36, 72, 72, 72, 72, 72,
                 72, 144, 144, 144, 144, 144, 144, 288, 288, 288, 288, 288, 288),
}


def ring_field(nk, nlon, nlat, seed, lo=0.05, hi=0.3):
    """A global mixing-ratio-like field (nk, nlon+4, nlat), Fortran order:
    a smooth zonal wave pattern plus grid-scale noise, with the two periodic
    longitude points on each side copied from the interior as the model
    keeps them."""
    rng = _rng(seed)
    lon = 2 * np.pi * np.arange(1, nlon + 1) / nlon
    lat = np.linspace(-np.pi / 2, np.pi / 2, nlat)
    k = np.arange(nk)[:, None, None]
    base = (0.5 * (lo + hi) + 0.25 * (hi - lo) * np.cos(lon)[None, :, None] * np.cos(lat)[None, None, :]
            * np.exp(-k / max(nk, 1)))
    noise = 0.1 * (hi - lo) * rng.standard_normal((nk, nlon, nlat))
    f = np.empty((nk, nlon + 4, nlat))
    f[:, 2:nlon + 2] = base + noise
    f[:, 0:2] = f[:, nlon:nlon + 2]
    f[:, nlon + 2:] = f[:, 2:4]
    return np.asfortranarray(f)
