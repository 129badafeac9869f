"""The column physics of one dynamics_ng step held on the device.

dynamics_ng (src/dynamics_ng.F90:98-232) runs, per nest and step, the
vertical column routines this package replaces, each after the horizontal
inputs it computes itself:

  oplus_ng x nstep_sub   smooth_ng(optm1), the O+ column step + lateral
                         hook + time filter (src/oplus_ng.F90:159, 125-340);
                         sub-step s reads what sub-step s-1 wrote; the rows
                         and pivots, the same in every sub-step, are formed
                         once (tg_oplus_ng_factor_dev) and each sub-step
                         solves from them (tg_oplus_ng_solve_dev)
  minor_ng x 4           N2D, N4S, NO, Ar (comp_n2d_ng ... comp_ar_ng):
                         smooth_ng(fcomp_tm1), advec_ng(fcomp), the column
                         step + lateral hook + time filter and floors
                         (src/minor_ng.F90:62-64, 60-237)
  settei_ng              Te, Ti; updates qtotal in place
                         (src/settei_ng.F90:60-261)
  dt_ng                  advec_ng(tn), smooth_ng(tn_nm), the column step
                         reading settei's qtotal + lateral hook + time filter
                         (src/dt_ng.F90:54-69, 57-213)
  comp_ng                advec_ng(o2, o1, he), smooth_ng(o2_nm, o1_nm,
                         he_nm), the O2/O/He block solve, the lateral hook
                         and the post-solve steps (src/comp_ng.F90:105-111,
                         74-457); on the global grid filter_o2o of the three
                         species between the solve and the time smoothing
                         (src/comp.F:929-934)

Every routine reads the step's input (itp) fields and writes new arrays, so
the only dependencies inside the step are the O+ sub-cycle and qtotal from
settei_ng to dt_ng.  DynamicsStep issues the routines through the
package's device entries on the caller's stream, or (fan_out) on four more
streams with those two dependencies as the only joins, and can capture the
whole step as one CUDA graph.  host_step runs the same step routine by
routine on host arrays (through this package's host-pointer entries, or
any set of routines of the same form).  The routines between these in dynamics_ng
(chemistry, heating, duv_ng's assembly, ...) are not part of this package:
their outputs are inputs here.

The grid is held as one subdomain, (nlon+4) x (nlat+4) ghost-inclusive
columns at index i + (nlon+4)*j, every field level-major (k*ld + col), as
tg_advec_ng_dev and tg_smooth_ng_dev define it.
"""
import numpy as np

from . import batch, colsolve as cs, synth

MINOR_SPECIES = ("n2d", "n4s", "no", "ar")
DTSMOOTH = 0.95                       # the model's dtsmooth; dtsmooth_div2 = (1 - dtsmooth) / 2
EARTH_RADIUS_CM = 6.37122e8


class Grid:
    """One grid held as a single subdomain: nk levels, nlon x nlat interior
    points with two ghost points on every side, the column stride ld and the
    horizontal constants of advec_ng/smooth_ng."""

    def __init__(self, nk, nlon, nlat, dz, lat0_deg=-90.0, dlat_deg=None, shapiro=0.03):
        self.nk, self.nlon, self.nlat, self.dz = nk, nlon, nlat, dz
        self.ncol = (nlon + 4) * (nlat + 4)
        self.ld = batch.pad_ld(self.ncol)
        self.dlamda = np.radians(360.0 / nlon)
        self.dphi = np.radians(180.0 / nlat if dlat_deg is None else dlat_deg)
        lat = np.radians(lat0_deg) + self.dphi * (np.arange(nlat + 4) - 1.5)
        self.racs = 1.0 / (EARTH_RADIUS_CM * np.maximum(np.cos(lat), 1e-3))
        self.re_inv = 1.0 / EARTH_RADIUS_CM
        self.shapiro = shapiro

    def boundary_mask(self):
        """The columns the lateral-boundary hooks overwrite: lon index -1 and
        nlon+2, lat index -1 and nlat+2 (the outermost ghost ring)."""
        m = np.zeros((self.nlat + 4, self.nlon + 4), dtype=np.uint8)
        m[0, :] = m[-1, :] = 1
        m[:, 0] = m[:, -1] = 1
        return m.reshape(-1)


def _dev_fields(F, grid, one_d, device):
    """A synthetic field dict on the device: 3-D (nk, ncol) fields level-major
    (nk, ld), 2-D (ncol) rows of ld, 1-D level profiles as they are; fs
    (12, ncol, nk) as 12 level-major slabs."""
    import torch
    nk, ncol, ld = grid.nk, grid.ncol, grid.ld
    out = {}
    for k, v in F.items():
        if k == "fs":
            fs = np.asarray(v).reshape(12, ncol, nk)
            t = torch.zeros((12, nk, ld), dtype=torch.float64, device=device)
            for s in range(12):
                t[s, :, :ncol] = torch.from_numpy(np.ascontiguousarray(fs[s].T))
            out[k] = t
        elif k in one_d:
            out[k] = torch.from_numpy(np.ascontiguousarray(v, dtype=np.float64)).to(device)
        elif np.ndim(v) == 2:
            out[k] = batch.level_scalar(np.asarray(v), ld, device)
        else:
            t = torch.zeros(ld, dtype=torch.float64, device=device)
            t[:ncol] = torch.from_numpy(np.asarray(v, dtype=np.float64))
            out[k] = t
    return out


def synthetic_inputs(grid, seed, nstep_sub=10):
    """Seeded host inputs of one step on `grid` with the model's magnitudes
    (the per-routine generators of synth), plus the fields each routine's
    horizontal steps start from: tn_nm, fcomp and fcomp_tm1 per minor
    species, optm1, o2_nm/o1_nm/he_nm, the lateral boundary values and the
    comp_ng post-step inputs.  Host (nk, ncol) Fortran arrays."""
    nk, ncol, dz = grid.nk, grid.ncol, grid.dz
    rng = np.random.default_rng(seed)
    U = lambda lo, hi: rng.uniform(lo, hi, size=(nk, ncol))  # noqa: E731
    F = lambda a: np.asfortranarray(a)  # noqa: E731
    h = {}
    Fd, Cd = synth.dt_inputs(nk, ncol, dz, seed + 1)
    h["dt"] = dict(F=Fd, C=Cd, tn_nm=F(Fd["tn"] * U(0.99, 1.01)), bnd=F(Fd["tn"] * U(0.98, 1.02)))
    h["minor"] = []
    for s, name in enumerate(MINOR_SPECIES):
        Fm, Cm = synth.minor_inputs(nk, ncol, dz, seed + 10 + s)
        tm1 = F(Fm["ftm1_smooth"].copy())
        h["minor"].append(dict(name=name, F=Fm, C=Cm, fcomp_tm1=tm1, fcomp=F(tm1 * U(0.98, 1.02)),
                               bnd=F(tm1 * U(0.95, 1.05))))
    Fs, Cs, qt = synth.settei_inputs(nk, ncol, dz, seed + 20)
    h["settei"] = dict(F=Fs, C=Cs, qtotal=qt)
    Fo, Co = synth.oplus_inputs(nk, ncol, dz, seed + 30, nstep_sub=nstep_sub)
    h["oplus"] = dict(F=Fo, C=Co, optm1=F(Fo["op"] * U(0.98, 1.02)), bnd=F(Fo["op"] * U(0.95, 1.05)))
    Fc, Cc = synth.comp_inputs(nk, ncol, dz, seed + 40)
    Fp, Cp = synth.comp_post_inputs(nk, ncol, dz, seed + 41)
    comp = dict(F=Fc, C=Cc, post_consts=Cp, xnmbar=Fp["xnmbar"], zpmid=Fp["zpmid"])
    for sp in ("o2", "o1", "he"):
        comp[sp + "_nm"] = F(Fc[sp] * U(0.99, 1.01))
        comp[sp + "_bnd"] = F(Fc[sp] * U(0.98, 1.02))
    h["comp"] = comp
    h["winds"] = dict(un=Fd["un"], vn=Fd["vn"])
    return h


class DynamicsStep:
    """One step of dynamics_ng's column routines on the device (see the
    module docstring).  `host` is what synthetic_inputs returns (or the same
    structure filled from the model's arrays); ring = (chunk_array) applies
    filter_o2o to O2, O and He as the global grid does.  The inputs are
    copied to the device once; every issue() recomputes the step from them
    into the output arrays, so repeated steps are identical."""

    def __init__(self, grid, host, ring=None, fan_out=True, device="cuda"):
        import torch
        self.grid, self.ring, self.fan_out, self.device = grid, ring, fan_out, device
        g, nk, ld = grid, grid.nk, grid.ld
        z = lambda: torch.zeros((nk, ld), dtype=torch.float64, device=device)  # noqa: E731
        lvl = lambda a: batch.level_scalar(np.asarray(a), ld, device)  # noqa: E731
        self.mask = torch.from_numpy(np.pad(g.boundary_mask(), (0, ld - g.ncol))).to(device)
        self.racs = torch.from_numpy(np.ascontiguousarray(g.racs)).to(device)
        self.un, self.vn = lvl(host["winds"]["un"]), lvl(host["winds"]["vn"])
        ds, ds2 = DTSMOOTH, 0.5 * (1.0 - DTSMOOTH)
        self.ds = (ds, ds2)
        # dt_ng: horadv and tnsmooth are written here; qtotal is settei's
        d = host["dt"]
        self.dt = dict(F=_dev_fields(d["F"], g, ("expz", "dift"), device), C=d["C"], tn_nm=lvl(d["tn_nm"]),
                       bnd=lvl(d["bnd"]), out=z(), nm=z())
        # settei_ng: qtotal is restored from qtotal0 at the start of the step
        s = host["settei"]
        self.settei = dict(F=_dev_fields(s["F"], g, (), device), C=s["C"], qtotal0=lvl(s["qtotal"]), qtotal=z(),
                           te=z(), ti=z())
        self.dt["F"]["qtotal"] = self.settei["qtotal"]
        # minor_ng x 4
        self.minor = []
        for m in host["minor"]:
            self.minor.append(dict(name=m["name"], F=_dev_fields(m["F"], g, ("expz", "difk"), device), C=m["C"],
                                   fcomp=lvl(m["fcomp"]), fcomp_tm1=lvl(m["fcomp_tm1"]), bnd=lvl(m["bnd"]),
                                   out=z(), nm=z()))
        # oplus_ng: sub-step s reads (op, optm1)[s] and writes [s + 1]
        o = host["oplus"]
        self.nstep_sub = int(o["C"]["nstep_sub"])
        Fo = _dev_fields(o["F"], g, ("zpint",), device)
        self.oplus = dict(F=Fo, C=o["C"], op0=Fo["op"], optm10=lvl(o["optm1"]), bnd=lvl(o["bnd"]),
                          op=[z(), z()], optm1=[z(), z()], xiop2p=z(), xiop2d=z(),
                          factor=torch.zeros(cs.oplus_ng_factor_doubles(nk, ld), dtype=torch.float64,
                                             device=device))
        # comp_ng + post-solve steps
        c = host["comp"]
        Fc = _dev_fields(c["F"], g, ("expz", "difk"), device)
        self.comp = dict(F=Fc, C=c["C"], pc=c["post_consts"], zpmid=torch.from_numpy(
            np.ascontiguousarray(c["zpmid"], dtype=np.float64)).to(device),
            post_in=dict(o2=Fc["o2"], o1=Fc["o1"], he=Fc["he"], o2_nm=lvl(c["o2_nm"]), o1_nm=lvl(c["o1_nm"]),
                         he_nm=lvl(c["he_nm"]), xnmbar=lvl(c["xnmbar"])),
            bnd=[lvl(c[sp + "_bnd"]) for sp in ("o2", "o1", "he")],
            out=torch.zeros((3, nk, ld), dtype=torch.float64, device=device),
            nm=torch.zeros((3, nk, ld), dtype=torch.float64, device=device))
        # the O+ sub-cycle is the step's longest chain: its stream gets the higher priority
        self.streams = ([torch.cuda.Stream(device=device, priority=-1)] +
                        [torch.cuda.Stream(device=device) for _ in range(3)]) if fan_out else []
        self.graph = None

    # ---- the routines, each on one stream --------------------------------
    def _advec(self, f, out, st):
        g = self.grid
        cs.advec_ng_dev(f, self.un, self.vn, self.racs, g.dlamda, g.dphi, g.re_inv, out, g.nk, g.nlon, g.nlat, g.ld,
                        stream=st)

    def _smooth(self, fin, out, st, shapiro=None):
        g = self.grid
        cs.smooth_ng_dev(fin, g.shapiro if shapiro is None else shapiro, out, g.nk, g.nlon, g.nlat, g.ld, stream=st)

    def _post(self, cur, prev, nm, bnd):
        return dict(cur=cur, prev=prev, nm_upd=nm, bnd_mask=self.mask, bnd=bnd, dtsmooth=self.ds[0],
                    dtsmooth_div2=self.ds[1])

    def _oplus(self, st):
        # the rows and pivots once (they do not change between sub-steps),
        # then each sub-step's smoothing and solve
        g, o = self.grid, self.oplus
        op, optm1 = o["op0"], o["optm10"]
        cs.oplus_ng_factor_dev(o["F"], o["C"], o["xiop2p"], o["xiop2d"], o["factor"], g.nk, g.ncol, g.ld, stream=st)
        for s in range(self.nstep_sub):
            nxt = s % 2
            self._smooth(optm1, o["F"]["optm1_smooth2"], st, g.shapiro / self.nstep_sub)
            F = dict(o["F"], op=op)
            cs.oplus_ng_solve_dev(F, o["C"], o["factor"], o["op"][nxt], g.nk, g.ncol, g.ld,
                                  self._post(op, optm1, o["optm1"][nxt], o["bnd"]), stream=st)
            op, optm1 = o["op"][nxt], o["optm1"][nxt]

    def _minor(self, m, st):
        g = self.grid
        self._smooth(m["fcomp_tm1"], m["F"]["ftm1_smooth"], st)
        self._advec(m["fcomp"], m["F"]["hadvec"], st)
        cs.minor_ng_post_dev(m["F"], m["C"], m["out"], g.nk, g.ncol, g.ld,
                             self._post(m["fcomp"], m["fcomp_tm1"], m["nm"], m["bnd"]), stream=st)

    def _settei_dt(self, st):
        g, s, d = self.grid, self.settei, self.dt
        self._advec(d["F"]["tn"], d["F"]["horadv"], st)
        self._smooth(d["tn_nm"], d["F"]["tnsmooth"], st)
        s["qtotal"].copy_(s["qtotal0"])
        cs.settei_ng_dev(s["F"], s["C"], s["te"], s["ti"], s["qtotal"], g.nk, g.ncol, g.ld, stream=st)
        cs.dt_ng_post_dev(d["F"], d["C"], d["out"], g.nk, g.ncol, g.ld,
                          self._post(d["F"]["tn"], d["tn_nm"], d["nm"], d["bnd"]), stream=st)

    def _comp(self, st):
        g, c = self.grid, self.comp
        F = c["F"]
        for sp in ("o2", "o1", "he"):
            self._advec(F[sp], F[sp + "_advec"], st)
            self._smooth(c["post_in"][sp + "_nm"], F[sp + "nm_smooth"], st)
        cs.comp_ng_dev(F, c["C"], c["out"], g.nk, g.ncol, g.ld, stream=st)
        if self.ring is not None:
            # filter_o2o on the interior latitudes: rows 2 .. nlat+1 of the subdomain
            off = 8 * 2 * (g.nlon + 4)
            for i in range(3):
                cs.ringfilter_dev(c["out"][i].data_ptr() + off, g.nk, g.nlon, g.nlat, 1, 0, self.ring, g.dlamda,
                                  g.ld, stream=st)
        cs.comp_post_ng_dev(c["post_in"], c["zpmid"], c["pc"], [c["out"][i] for i in range(3)],
                            [c["nm"][i] for i in range(3)], g.nk, g.ncol, g.ld, bnd_mask=self.mask, bnd=c["bnd"],
                            stream=st)

    def issue(self, stream):
        """Issues one step on `stream` (a torch.cuda.Stream); with fan_out the
        routines run on four more streams that fork from and join `stream`."""
        import torch
        if not self.fan_out:
            with torch.cuda.stream(stream):
                self._oplus(stream)
                for m in self.minor:
                    self._minor(m, stream)
                self._settei_dt(stream)
                self._comp(stream)
            return
        s_op, s_m0, s_m1, s_c = self.streams
        for s in self.streams:
            s.wait_stream(stream)
        with torch.cuda.stream(s_op):
            self._oplus(s_op)
        with torch.cuda.stream(s_m0):
            self._minor(self.minor[0], s_m0)
            self._minor(self.minor[1], s_m0)
        with torch.cuda.stream(s_m1):
            self._minor(self.minor[2], s_m1)
            self._minor(self.minor[3], s_m1)
        with torch.cuda.stream(s_c):
            self._comp(s_c)
        with torch.cuda.stream(stream):
            self._settei_dt(stream)
        for s in self.streams:
            stream.wait_stream(s)

    def capture(self, stream):
        """Records one step into a CUDA graph (after an eager step, which
        sizes the library's per-stream buffers); replay() then runs it."""
        import torch
        self.issue(stream)
        stream.synchronize()
        self.graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(self.graph, stream=stream, capture_error_mode="thread_local"):
            self.issue(stream)
        return self.graph

    def replay(self, stream):
        import torch
        with torch.cuda.stream(stream):
            self.graph.replay()

    def outputs(self):
        """The step's results on the device, by the reference's names."""
        o = self.oplus
        last = (self.nstep_sub - 1) % 2
        out = dict(tn_upd=self.dt["out"], tn_nm_upd=self.dt["nm"], te=self.settei["te"], ti=self.settei["ti"],
                   qtotal=self.settei["qtotal"], op=o["op"][last], optm1=o["optm1"][last], xiop2p=o["xiop2p"],
                   xiop2d=o["xiop2d"], o2_upd=self.comp["out"][0], o1_upd=self.comp["out"][1],
                   he_upd=self.comp["out"][2], o2nm_upd=self.comp["nm"][0], o1nm_upd=self.comp["nm"][1],
                   henm_upd=self.comp["nm"][2])
        for m in self.minor:
            out[m["name"] + "_upd"] = m["out"]
            out[m["name"] + "_nm_upd"] = m["nm"]
        return out

    def bytes_per_step(self):
        """Algorithmic device bytes of one step: every field each routine
        reads once and every array it writes once, 8 B per level and column
        (2-D rows 8 B per column; the level profiles and the boundary values
        of the outermost ring left out)."""
        g = self.grid
        lvl, row = 8 * g.nk * g.ncol, 8 * g.ncol
        n3 = lambda F: sum(1 for v in F.values() if v.dim() == 2 and v.shape[0] == g.nk)  # noqa: E731
        n2 = lambda F: sum(1 for v in F.values() if v.dim() == 1 and v.shape[0] == g.ld)  # noqa: E731
        n_adv = 1 + len(self.minor) + 3                 # advec: f, un, vn read, hadvec written
        n_smo = 1 + len(self.minor) + 3 + self.nstep_sub
        b = (4 * n_adv + 2 * n_smo) * lvl
        d, s, o, c = self.dt, self.settei, self.oplus, self.comp
        b += (n3(d["F"]) + 1 + 2) * lvl + n2(d["F"]) * row          # + tn_nm; tn_upd, tn_nm_upd
        b += (n3(s["F"]) + 1 + 3) * lvl + n2(s["F"]) * row          # + qtotal; te, ti, qtotal
        for m in self.minor:
            b += (n3(m["F"]) + 2 + 2) * lvl + n2(m["F"]) * row      # + fcomp, fcomp_tm1; out, nm
        b += self.nstep_sub * ((n3(o["F"]) + 1 + 4) * lvl + n2(o["F"]) * row)   # + optm1; 4 written
        b += (n3(c["F"]) + 12 + 3) * lvl + n2(c["F"]) * row         # fs slabs; O2, O, He
        b += (7 + 3 + 6) * lvl                                       # post: inputs, solution read, 6 written
        if self.ring is not None:
            b += 3 * 2 * 8 * g.nk * (g.nlon + 4) * 2 * len(self.ring)   # filtered rows read and written
        return b


def host_step(api, grid, h, ring=None):
    """The same step routine by routine on host (nk, ncol) arrays, in the
    reference's order: what a model calling the host-pointer drop-ins one
    routine at a time does.  `api` supplies the routines in the form
    returning new arrays (advec_ng, smooth_ng, time_filter_ng, oplus_ng,
    minor_ng, settei_ng, dt_ng, comp_ng, ringfilter, comp_post_ng and the
    FILTER_DT/_MINOR/_OPLUS codes): HostEntries(package) for this package's
    host entries.  Returns the results by the names DynamicsStep.outputs()
    uses."""
    nk, ncol = grid.nk, grid.ncol
    shp = (nk, grid.nlon + 4, grid.nlat + 4)
    to3 = lambda a: np.asfortranarray(np.asarray(a).reshape(shp, order="F"))  # noqa: E731
    back = lambda a: np.asfortranarray(np.asarray(a).reshape(nk, ncol, order="F"))  # noqa: E731
    un, vn = to3(h["winds"]["un"]), to3(h["winds"]["vn"])

    def adv(f):
        return back(api.advec_ng(to3(f), un, vn, grid.racs, grid.dlamda, grid.dphi, grid.re_inv))

    def smo(f, sh=grid.shapiro):
        return back(api.smooth_ng(to3(f), sh))

    mask = grid.boundary_mask().astype(bool)
    ds, ds2 = DTSMOOTH, 0.5 * (1.0 - DTSMOOTH)

    def post(which, x, cur, prev, bnd):
        x = np.array(x, order="F")
        x[:, mask] = bnd[:, mask]                 # the lateral-boundary hook
        return api.time_filter_ng(which, cur, prev, x, ds, ds2)

    out = {}
    o = h["oplus"]
    op, optm1 = o["F"]["op"], o["optm1"]
    nsub = int(o["C"]["nstep_sub"])
    for _ in range(nsub):
        F = dict(o["F"], op=op, optm1_smooth2=smo(optm1, grid.shapiro / nsub))
        opout, xi2p, xi2d = api.oplus_ng(F, o["C"])[:3]
        op, optm1 = post(api.FILTER_OPLUS, opout, op, optm1, o["bnd"])
    out.update(op=op, optm1=optm1, xiop2p=xi2p, xiop2d=xi2d)
    for m in h["minor"]:
        F = dict(m["F"], ftm1_smooth=smo(m["fcomp_tm1"]), hadvec=adv(m["fcomp"]))
        x, nm = post(api.FILTER_MINOR, api.minor_ng(F, m["C"]), m["fcomp"], m["fcomp_tm1"], m["bnd"])
        out[m["name"] + "_upd"], out[m["name"] + "_nm_upd"] = x, nm
    s = h["settei"]
    te, ti, qt = api.settei_ng(s["F"], s["C"], s["qtotal"])
    out.update(te=te, ti=ti, qtotal=qt)
    d = h["dt"]
    F = dict(d["F"], horadv=adv(d["F"]["tn"]), tnsmooth=smo(d["tn_nm"]), qtotal=qt)
    out["tn_upd"], out["tn_nm_upd"] = post(api.FILTER_DT, api.dt_ng(F, d["C"]), d["F"]["tn"], d["tn_nm"], d["bnd"])
    c = h["comp"]
    F = dict(c["F"])
    for sp in ("o2", "o1", "he"):
        F[sp + "_advec"] = adv(F[sp])
        F[sp + "nm_smooth"] = smo(c[sp + "_nm"])
    upd = [np.array(u, order="F") for u in api.comp_ng(F, c["C"])]
    if ring is not None:
        for i in range(3):
            f3 = to3(upd[i])
            inner = np.asfortranarray(f3[:, :, 2:grid.nlat + 2])
            f3[:, :, 2:grid.nlat + 2] = api.ringfilter(inner, 1, 0, ring, grid.dlamda)
            upd[i] = back(f3)
    for i, sp in enumerate(("o2", "o1", "he")):
        upd[i][:, mask] = c[sp + "_bnd"][:, mask]
    P = dict(o2=F["o2"], o1=F["o1"], he=F["he"], o2_nm=c["o2_nm"], o1_nm=c["o1_nm"], he_nm=c["he_nm"],
             xnmbar=c["xnmbar"], zpmid=c["zpmid"], o2_upd=upd[0], o1_upd=upd[1], he_upd=upd[2])
    for name, v in zip(("o2_upd", "o1_upd", "he_upd", "o2nm_upd", "o1nm_upd", "henm_upd"),
                       api.comp_post_ng(P, c["post_consts"])):
        out[name] = v
    return out


class HostEntries:
    """This package's host-pointer entries (synchronous, host arrays in and
    out, each call copying its inputs to the device and its results back)
    in the array-returning form host_step uses."""

    FILTER_DT, FILTER_MINOR, FILTER_OPLUS = cs.TG_FILTER_DT, cs.TG_FILTER_MINOR, cs.TG_FILTER_OPLUS

    @staticmethod
    def _z(a):
        return np.zeros(np.shape(a), order="F")

    def advec_ng(self, f, un, vn, racs, dlamda, dphi, re_inv):
        out = self._z(f)
        cs.advec_ng(f, un, vn, racs, dlamda, dphi, re_inv, out)
        return out

    def smooth_ng(self, fin, shapiro):
        out = self._z(fin)
        cs.smooth_ng(fin, shapiro, out)
        return out

    def time_filter_ng(self, which, cur, prev, upd, ds, ds2):
        upd, nm = np.array(upd, order="F"), self._z(upd)
        cs.time_filter_ng(which, cur, prev, ds, ds2, upd, nm)
        return upd, nm

    def oplus_ng(self, F, C):
        outs = [self._z(F["op"]) for _ in range(3)]
        cs.oplus_ng(F, C, *outs)
        return tuple(outs)

    def minor_ng(self, F, C):
        out = self._z(F["tn"])
        cs.minor_ng(F, C, out)
        return out

    def settei_ng(self, F, C, qtotal):
        te, ti, q = self._z(F["tn"]), self._z(F["tn"]), np.array(qtotal, order="F")
        cs.settei_ng(F, C, te, ti, q)
        return te, ti, q

    def dt_ng(self, F, C):
        out = self._z(F["tn"])
        cs.dt_ng(F, C, out)
        return out

    def comp_ng(self, F, C):
        outs = [self._z(F["tn"]) for _ in range(3)]
        cs.comp_ng(F, C, *outs)
        return tuple(outs)

    def ringfilter(self, f, order, poly, chunk_array, dlamda):
        f = np.array(f, order="F")
        cs.ringfilter(f, order, poly, chunk_array, dlamda)
        return f

    def comp_post_ng(self, P, C):
        upd = [np.array(P[k], order="F") for k in ("o2_upd", "o1_upd", "he_upd")]
        nm = [self._z(P["o2"]) for _ in range(3)]
        cs.comp_post_ng(P, C, upd, nm)
        return tuple(upd) + tuple(nm)
