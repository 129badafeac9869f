// oplus_ng (O+), the vertical part of src/oplus_ng.F90:88-307, as one kernel,
// one thread per column, in three passes over the levels:
//
//   1. level quantities: dj (with the optional cap), hdz, tp1, b.u, the loss
//      rate op_loss and the production op_prod, plus the outputs xiop2p,
//      xiop2d and (optionally) Fe, Fn.  The six quantities the rows need go
//      to a level-major scratch (6 * nk * ld doubles) that the next pass
//      re-reads while it is still in L2.
//   2. rows k = 0..nk-2: hdzi, tphdz0/1, djint, the diffusion / drift / wind
//      coefficients, both boundary folds and the chemistry, fed straight into
//      the Thomas forward sweep (w2 in shared memory, w3 parked in opout).
//   3. the back sweep and the top level opout(nk) = opout(nk-1)**2/opout(nk-2).
//
// Every operation is the reference's, in its order, with non-contracting FP64
// intrinsics.  log10, pow, sin and cos are the device library's, within a few
// ulp of the host C library's: the kernel agrees with the CPU restatement to
// a stated tolerance.
#include <cfloat>

#include "tg_internal.h"
#include "tg_arith.cuh"
#include "tg_stage.cuh"

namespace tg {
namespace {
__device__ __forceinline__ double xm(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double xa(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double xs(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double xd(double a, double b) { return __ddiv_rn(a, b); }

// scratch planes, level-major: the level quantities, then the rows of the
// three-pass form
// three-pass form, then the factorization the sub-step solves reuse (w1,
// 1/w1, w2 per row; the boundary terms of the right-hand side in rows 0 and 1
// of S_TB)
enum { S_DJ = 0, S_HDZ, S_TP1, S_BDOTU, S_OL, S_PROD, S_P, S_Q, S_R, S_EX, S_W1, S_Y1, S_W2, S_TB, S_N };

// interface value at j of a(j), a(j+1): .5*(a(j)+a(j+1)); at the top
// 1.5*a(nk)-.5*a(nk-1)
__device__ __forceinline__ double up(const double *p, int j, int nk, long ld, long col)
{
    if (j < nk - 1) return xm(.5, xa(__ldg(p + j * ld + col), __ldg(p + (j + 1) * ld + col)));
    return xs(xm(1.5, __ldg(p + (long)(nk - 1) * ld + col)), xm(.5, __ldg(p + (long)(nk - 2) * ld + col)));
}
}  // namespace

// Level quantities of level j of one column (oplus_ng.F90:112-169, 285-299):
// dj, hdz, tp1, b.u, op_loss and op_prod into the scratch planes, xiop2p,
// xiop2d and (if requested) Fe, Fn into the outputs.
__device__ __forceinline__ void oplus_level(const OplusFields &F, const OplusConsts &C, double *scr, double *xiop2p,
                                            double *xiop2d, double *Fe, double *Fn, int nk, long ld, long col, int j)
{
    auto at = [&](const double *p, int k) { return __ldg(p + k * ld + col); };
    auto S = [&](int e, int k) -> double & { return scr[(long)e * nk * ld + (long)k * ld + col]; };
    const double dz = C.dz;
    const double bx = __ldg(F.bx + col), by = __ldg(F.by + col), bz = __ldg(F.bz + col);
    const bool capped = !(fabs(xs(C.opdiffcap, 0.)) < 1e-9);
    const double sncs = Fe ? xm(sin(__ldg(F.dipmag + col)), cos(__ldg(F.dipmag + col))) : 0.;
    const double ogg = xd(xm(C.rmass_op, C.grav), C.gask);

    const double tn = at(F.tn, j), te = at(F.te, j), ti = at(F.ti, j), o2 = at(F.o2, j), o1 = at(F.o1, j),
                 n2 = at(F.n2, j), he = at(F.he, j), xn = at(F.xnmbar, j), hj = at(F.scht, j),
                 ne = at(F.ne, j);
    const double tr = xm(0.5, xa(tn, ti));
    const double lg = xs(1., xm(0.064, log10(tr)));
    double vni = xm(xm(18.1, o2), C.rmassinv_o2);
    vni = xa(vni, xm(xm(xm(xm(o1, C.rmassinv_o1), sqrt(tr)), xm(lg, lg)), C.colfac));
    vni = xa(vni, xm(xm(3.6, he), C.rmassinv_he));
    vni = xa(vni, xm(xm(18.6, n2), C.rmassinv_n2));
    double dj = xd(1.42E17, xm(xn, vni));
    vni = xm(xm(16., 3.53E-11), vni);
    if (capped) {
        const double cap = xd(C.opdiffcap, xa(1., pow(2., xs(__ldg(F.zpint + j), 6.))));
        dj = dj < cap ? dj : cap;
    }
    const double wni = up(F.w, j, nk, ld, col);
    S(S_DJ, j) = dj;
    S(S_HDZ, j) = xd(1., xm(hj, dz));
    S(S_TP1, j) = xm(0.5, xa(ti, te));
    S(S_BDOTU, j) = xa(xa(xm(bx, at(F.u, j)), xm(by, at(F.v, j))), xm(xm(hj, bz), wni));
    if (Fe) {
        auto tpop = [&](int i) { return xm(xa(at(F.te, i), at(F.ti, i)), at(F.op, i)); };
        double d;
        if (j == 0) d = xs(tpop(1), tpop(0));
        else if (j == nk - 1) d = xs(tpop(nk - 1), tpop(nk - 2));
        else if (j == nk - 2) d = xs(tpop(nk - 2), tpop(nk - 3));
        else d = xd(xs(tpop(j + 1), tpop(j - 1)), 2.);
        const double diffj = xa(xm(xd(1., xm(hj, C.dlev)), d), xm(ogg, at(F.op, j)));
        const double wd = xm(xm(vni, diffj), dj);
        Fe[j * ld + col] = xm(xm(wd, sncs), __ldg(F.sndec + col));
        Fn[j * ld + col] = xm(xm(wd, sncs), __ldg(F.csdec + col));
    }
    // chemistry (oplus_ng.F90:285-299)
    const double rk19 = at(F.rk19, j), rk20 = at(F.rk20, j), rk25 = at(F.rk25, j);
    const double den2p = xa(xa(xa(xm(xn, xa(xm(xm(xa(C.rk16, C.rk17), n2), C.rmassinv_n2),
                                            xm(xm(C.rk18, o1), C.rmassinv_o1))),
                                  xm(xa(rk19, rk20), ne)),
                               C.rk21),
                            C.rk22);
    const double x2p = xd(up(F.qop2p, j, nk, ld, col), den2p);
    const double den2d =
        xa(xa(xm(xn, xa(xa(xm(xm(C.rk23, n2), C.rmassinv_n2), xm(xm(C.rk24, o1), C.rmassinv_o1)),
                        xm(xm(C.rk26, o2), C.rmassinv_o2))),
              xm(rk25, ne)),
           C.rk27);
    const double x2d = xd(xa(up(F.qop2d, j, nk, ld, col), xm(xa(xm(rk20, ne), C.rk22), x2p)), den2d);
    xiop2p[j * ld + col] = x2p;
    xiop2d[j * ld + col] = x2d;
    S(S_OL, j) = xm(xn, xa(xa(xm(xm(at(F.rk1, j), o2), C.rmassinv_o2), xm(xm(at(F.rk2, j), n2), C.rmassinv_n2)),
                            xm(xm(C.rk10, at(F.n2d, j)), C.rmassinv_n2d)));
    double prod = xa(up(F.qop, j, nk, ld, col), xm(xa(xm(rk19, ne), C.rk21), x2p));
    prod = xa(prod, xm(xa(xm(rk25, ne), C.rk27), x2d));
    prod = xa(prod, xm(xm(xm(xa(xm(C.rk18, x2p), xm(C.rk24, x2d)), o1), C.rmassinv_o1), xn));
    S(S_PROD, j) = prod;
}

// Per-column constants of the rows: the top O+ flux (oplus_flux,
// oplus_ng.F90:88-99), b_z terms, g*m/(2R), the sub-step time factor and the
// upper-boundary ratios (:262-266).
struct OplusCol {
    double bz, opflux, dvbz, bz2, gmr, dtn, ubca, ubcb;
};

// Interface and half-level quantities of row j built from the level planes
// (oplus_ng.F90:209-254), as the reference forms them.
struct OplusRowsAt {
    const double *scr;
    long slab, ld, col;
    int nk;
    double gmr, dvbz, bz2;
    __device__ __forceinline__ double S(int e, int k) const { return scr[(long)e * slab + (long)k * ld + col]; }
    __device__ __forceinline__ double hdzi(int j) const
    {
        if (j == 0) return xs(xm(1.5, S(S_HDZ, 0)), xm(0.5, S(S_HDZ, 1)));
        if (j == nk - 1) return xs(xm(1.5, S(S_HDZ, nk - 2)), xm(0.5, S(S_HDZ, nk - 3)));
        return xm(0.5, xa(S(S_HDZ, j - 1), S(S_HDZ, j)));
    }
    __device__ __forceinline__ double tph1(int j) const
    {
        if (j == nk - 1) return xa(xm(xm(2., xs(xm(2., S(S_TP1, nk - 2)), S(S_TP1, nk - 3))), hdzi(nk - 1)), gmr);
        return xa(xm(xm(2., S(S_TP1, j)), hdzi(j)), gmr);
    }
    __device__ __forceinline__ double tph0(int j) const
    {
        if (j == 0) return xs(xm(xm(2., xs(xm(2., S(S_TP1, 0)), S(S_TP1, 1))), hdzi(0)), gmr);
        return xs(xm(xm(2., S(S_TP1, j - 1)), hdzi(j)), gmr);
    }
    __device__ __forceinline__ double djint(int j) const
    {
        if (j == 0) return xs(xm(1.5, S(S_DJ, 0)), xm(0.5, S(S_DJ, 1)));
        if (j == nk - 1) return xs(xm(1.5, S(S_DJ, nk - 2)), xm(0.5, S(S_DJ, nk - 3)));
        return xm(0.5, xa(S(S_DJ, j - 1), S(S_DJ, j)));
    }
};

__device__ __forceinline__ OplusCol oplus_col(const OplusFields &F, const OplusConsts &C, const OplusRowsAt &A)
{
    const long col = A.col;
    // pi = 4*atan(1) of the reference, correctly rounded
    const double pi = 3.141592653589793, rtd = 180. / pi;
    const double phid = 2.0e8, phin = -2.0e8, ppolar = 0.;
    OplusCol c;
    c.bz = __ldg(F.bz + col);
    {
        const double arl = fabs(__ldg(F.rlatm + col)), chi = __ldg(F.chi + col);
        double a = 0.;
        if (arl >= xd(pi, 4.5)) a = 1.;
        if (arl < xd(pi, 4.5) && arl > xd(pi, 18.)) a = xm(.5, xa(1., cos(xs(xm(arl, 6.), xd(xm(pi, 4.), 3.)))));
        if (arl <= xd(pi, 18.)) a = 0.;
        const double fed = xm(phid, a), fen = xm(phin, a);
        double opflux = chi >= xm(0.5, pi) ? fen : fed;
        const double cd = xm(chi, rtd);
        if (xm(xs(cd, 80.), xs(cd, 100.)) < 0.)
            opflux = xa(xm(.5, xa(fed, fen)), xm(xm(.5, xs(fed, fen)), cos(xd(xm(pi, xs(cd, 80.)), 20.))));
        if (arl >= xd(pi, 3.)) opflux = xa(opflux, ppolar);
        c.opflux = opflux;
    }
    c.dvbz = xd(__ldg(F.dvb + col), c.bz);
    c.bz2 = xm(c.bz, c.bz);
    c.gmr = xd(xm(C.grav, C.rmass_op), xm(2., C.gask));
    c.dtn = xm(C.dtx2inv, (double)C.nstep_sub);
    OplusRowsAt B = A;
    B.gmr = c.gmr;
    const int nk = A.nk;
    c.ubca = xm(xm(-c.bz2, B.djint(nk - 1)), B.tph1(nk - 1));
    c.ubcb = xm(xm(-c.bz2, B.djint(nk - 1)), B.tph0(nk - 1));
    return c;
}

// The diffusion, drift and wind parts of row k's coefficients (oplus_ng.F90:
// 255-282): {diffp, diffq, diffr, driftp, driftq, driftr, windp, windq, windr}.
__device__ __forceinline__ void oplus_parts(const OplusFields &F, const OplusConsts &C, const OplusRowsAt &A,
                                            const OplusCol &cc, int k, double (&pt)[9])
{
    const int nk = A.nk;
    const long ld = A.ld, col = A.col;
    auto at = [&](const double *pp, int kk) { return __ldg(pp + kk * ld + col); };
    const double bz = cc.bz;
    auto hdzmp = [&](int j, double sgn) {
        const double divbz = xa(cc.dvbz, xd(at(F.bdotdh_djbz, j), xm(A.S(S_DJ, j), cc.bz2)));
        const double h = A.S(S_HDZ, j);
        return xm(sgn > 0 ? xa(h, xm(0.5, divbz)) : xs(h, xm(0.5, divbz)), cc.bz2);
    };
    const double hdzm_k = hdzmp(k, -1.), hdzp_k = hdzmp(k, 1.);
    const double dji_k = A.djint(k), dji_1 = A.djint(k + 1);
    const double t0k = A.tph0(k), t1k = A.tph1(k), t01 = A.tph0(k + 1), t11 = A.tph1(k + 1);
    const double hdz_k = A.S(S_HDZ, k);
    pt[0] = xm(xm(hdzm_k, dji_k), t0k);
    pt[1] = -xa(xm(xm(hdzp_k, dji_1), t01), xm(xm(hdzm_k, dji_k), t1k));
    pt[2] = xm(xm(hdzp_k, dji_1), t11);
    const double wii = up(F.wi, k, nk, ld, col);
    pt[3] = xm(xm(wii, 0.5), hdz_k);
    pt[4] = xd(xm(-wii, 6.), C.re);
    pt[5] = xm(xm(-wii, 0.5), hdz_k);
    const double bu_k = A.S(S_BDOTU, k);
    pt[6] = k == 0 ? xm(xm(xm(bz, xs(xm(2., bu_k), A.S(S_BDOTU, 1))), 0.5), hdz_k)
                   : xm(xm(xm(bz, A.S(S_BDOTU, k - 1)), 0.5), hdz_k);
    pt[7] = xm(xm(-bu_k, cc.dvbz), bz);
    pt[8] = k == nk - 2 ? xm(xm(xm(bz, xs(xm(2., bu_k), A.S(S_BDOTU, k - 1 >= 0 ? k - 1 : 0))), 0.5), hdz_k)
                        : xm(xm(xm(-bz, A.S(S_BDOTU, k + 1)), 0.5), hdz_k);
}

// Row k (0..nk-2) of the O+ system: p, q, r and the right-hand side, with
// both boundary folds (oplus_ng.F90:255-303).
// t_top and t_bot receive the boundary terms the right-hand side takes at
// k = nk-2 and k = 0 (when given).
__device__ __forceinline__ void oplus_row(const OplusFields &F, const OplusConsts &C, const OplusRowsAt &A,
                                          const OplusCol &cc, int k, double &p, double &q, double &r, double &ex,
                                          double *t_top = nullptr, double *t_bot = nullptr)
{
    const int nk = A.nk;
    const long ld = A.ld, col = A.col;
    auto at = [&](const double *pp, int kk) { return __ldg(pp + kk * ld + col); };
    double pt[9];
    oplus_parts(F, C, A, cc, k, pt);
    p = xa(xa(pt[0], pt[3]), pt[6]);
    q = xs(xa(xa(pt[1], pt[4]), pt[7]), cc.dtn);
    r = xa(xa(pt[2], pt[5]), pt[8]);
    ex = xs(at(F.explicit_h, k), xm(xm(at(F.optm1_smooth2, k), C.dtx2inv), (double)C.nstep_sub));
    if (k == nk - 2) {
        q = xa(q, xm(xd(cc.ubcb, cc.ubca), r));
        const double tt = xd(xm(cc.opflux, r), cc.ubca);
        if (t_top) *t_top = tt;
        ex = xs(ex, tt);
        r = 0.;
    }
    q = xs(q, A.S(S_OL, k));
    ex = xs(ex, A.S(S_PROD, k));
    if (k == 0) {
        q = xs(q, p);
        const double tb = xd(xm(xm(2., p), at(F.qop, 0)), xs(xm(1.5, A.S(S_OL, 0)), xm(0.5, A.S(S_OL, 1))));
        if (t_bot) *t_bot = tb;
        ex = xs(ex, tb);
        p = 0.;
    }
}

// Rows k = 0..nk-2 from the level planes, the forward sweep and the back
// sweep of one column (oplus_ng.F90:88-99, 209-307).
__device__ __forceinline__ void oplus_walk(const OplusFields &F, const OplusConsts &C, double *opout, const double *scr,
                                           double *w2s, int T, int nk, long ld, long col, double *sys_out,
                                           unsigned *status, const PostStep &post, int has_post, int pd)
{
    const long slab = (long)nk * ld;
    OplusRowsAt A{scr, slab, ld, col, nk, 0., 0., 0.};
    const OplusCol cc = oplus_col(F, C, A);
    A.gmr = cc.gmr;
    bool ok = true;
    double w1 = 0., y1 = 0., w3 = 0., rprev = 0.;
    // bring the lines row kk touches first (the planes at level kk+1, the
    // fields at kk) into L1, pd rows ahead of the row that computes
    auto pf_row = [&](int kk) {
        const long o1 = (long)kk * ld + col;
        if (kk + 1 < nk) {
#pragma unroll
            for (int e = 0; e < 4; ++e) pf_l1(scr + (long)e * slab + o1 + ld);
            pf_l1(F.wi + o1 + ld);
        }
        pf_l1(F.bdotdh_djbz + o1);
        pf_l1(F.explicit_h + o1);
        pf_l1(F.optm1_smooth2 + o1);
        pf_l1(scr + (long)S_OL * slab + o1);
        pf_l1(scr + (long)S_PROD * slab + o1);
    };
    for (int kk = 1; kk < pd && kk < nk - 1; ++kk) pf_row(kk);
    for (int k = 0; k < nk - 1; ++k) {
        if (k + pd < nk - 1) pf_row(k + pd);
        double p, q, r, ex;
        oplus_row(F, C, A, cc, k, p, q, r, ex);
        if (sys_out) {
            const long o = (long)k * ld + col;
            sys_out[o] = p;
            sys_out[slab + o] = q;
            sys_out[2 * slab + o] = r;
            sys_out[3 * slab + o] = ex;
        }
        if (k == 0) {
            w1 = q;
            y1 = __drcp_rn(w1);
            w3 = qdiv(ex, w1, y1);
        } else {
            const double w2 = qdiv(rprev, w1, y1);
            w2s[(long)(k - 1) * T] = w2;
            w1 = xs(q, xm(p, w2));
            y1 = __drcp_rn(w1);
            w3 = qdiv(xs(ex, xm(p, w3)), w1, y1);
        }
        ok = ok && fabs(w1) <= DBL_MAX && w1 != 0.0;
        opout[(long)k * ld + col] = w3;
        rprev = r;
    }
    // ---- pass 3: back sweep and the top level (oplus_ng.F90:305-307)
    // with has_post every row goes through the post-solve steps (:330-340),
    // the top row computed from the unfiltered values first
    const int K = nk - 1;
    const bool bcol = has_post && post.bnd_mask && post.bnd_mask[col];
    double xn = w3, xtop = w3;
    bool fin = fabs(xn) <= DBL_MAX;
    double park = K >= 2 ? opout[(long)(K - 2) * ld + col] : 0.;
    for (int kk = K - 3; kk > K - 2 - pd && kk >= 0; --kk) post_prefetch(post, has_post, bcol, opout, (long)kk * ld + col);
    for (int k = K - 2; k >= 0; --k) {
        if (k - pd >= 0) post_prefetch(post, has_post, bcol, opout, (long)(k - pd) * ld + col);
        const double wk = park;
        if (k >= 1) park = opout[(long)(k - 1) * ld + col];
        xn = xs(wk, xm(w2s[(long)k * T], xn));
        fin = fin && fabs(xn) <= DBL_MAX;
        post_store(post, has_post, bcol, opout, (long)k * ld + col, xn);
        if (k == K - 2) {
            post_store(post, has_post, bcol, opout, (long)K * ld + col, xd(xm(xtop, xtop), xn));
            if (has_post) post_store(post, true, bcol, opout, (long)(K - 1) * ld + col, xtop);
        }
    }
    if (status && (!ok || !fin)) atomicOr(status, (ok ? 0u : FLAG_PIVOT) | (fin ? 0u : FLAG_NONFINITE));
}

__global__ void __launch_bounds__(128) k_oplus_ng(OplusFields F, OplusConsts C, double *opout, double *xiop2p,
                                                  double *xiop2d, double *Fe, double *Fn, double *scr, int nk,
                                                  int ncol, long ld, double *sys_out, unsigned *status,
                                                  PostStep post, int has_post, int pd)
{
    extern __shared__ double smem_op[];
    const long col = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (col >= ncol) return;
    for (int j = 0; j < nk; ++j) oplus_level(F, C, scr, xiop2p, xiop2d, Fe, Fn, nk, ld, col, j);
    oplus_walk(F, C, opout, scr, smem_op + threadIdx.x, blockDim.x, nk, ld, col, sys_out, status, post, has_post, pd);
}

// Two-pass form: the level quantities with one thread per (level, column),
// then the column walk.
__global__ void __launch_bounds__(128) k_oplus_levels(OplusFields F, OplusConsts C, double *xiop2p, double *xiop2d,
                                                      double *Fe, double *Fn, double *scr, int nk, int ncol, long ld)
{
    const long col = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (col >= ncol) return;
    const int j = blockIdx.y;
    {
        // every line level j reads, requested into L1 at once: the reads sit
        // between log10, sqrt, pow and divisions and would otherwise wait
        // one at a time
        const long o = (long)j * ld + col;
        const double *lvl[] = {F.tn, F.te, F.ti, F.o2, F.o1, F.n2, F.he, F.xnmbar, F.scht, F.ne, F.u, F.v,
                               F.rk19, F.rk20, F.rk25, F.rk1, F.rk2, F.n2d, F.w, F.qop2p, F.qop2d, F.qop};
#pragma unroll
        for (int i = 0; i < 22; ++i) pf_l1(lvl[i] + o);
        if (j + 1 < nk) {
            pf_l1(F.w + o + ld);
            pf_l1(F.qop2p + o + ld);
            pf_l1(F.qop2d + o + ld);
            pf_l1(F.qop + o + ld);
        }
    }
    oplus_level(F, C, scr, xiop2p, xiop2d, Fe, Fn, nk, ld, col, j);
}

__global__ void __launch_bounds__(128) k_oplus_rows(OplusFields F, OplusConsts C, double *opout, const double *scr,
                                                    int nk, int ncol, long ld, double *sys_out, unsigned *status,
                                                    PostStep post, int has_post, int pd)
{
    extern __shared__ double smem_or[];
    const long col = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (col >= ncol) return;
    oplus_walk(F, C, opout, scr, smem_or + threadIdx.x, blockDim.x, nk, ld, col, sys_out, status, post, has_post, pd);
}

// Three-pass form, pass 2: row k of every column, one thread per (row, column).
// A block covers kCoefCols columns x kCoefRows rows; the column quantities
// (oplus_col: the O+ flux boundary with its cosine, the upper-boundary
// coefficients, several divisions) are formed once per column and block by
// the block's first row of threads and shared.
constexpr int kCoefCols = 32, kCoefRows = 8;
dim3 coef_grid(int nk, int ncol)
{
    return dim3((unsigned)((ncol + kCoefCols - 1) / kCoefCols), (unsigned)((nk - 1 + kCoefRows - 1) / kCoefRows));
}
__global__ void __launch_bounds__(kCoefCols * kCoefRows) k_oplus_coefs(OplusFields F, OplusConsts C, double *scr,
                                                                       int nk, int ncol, long ld, double *sys_out)
{
    __shared__ OplusCol col_q[kCoefCols];
    const long col = (long)blockIdx.x * kCoefCols + threadIdx.x;
    const int k = blockIdx.y * kCoefRows + threadIdx.y;
    const long slab = (long)nk * ld, o = (long)k * ld + col;
    OplusRowsAt A{scr, slab, ld, col, nk, 0., 0., 0.};
    // every line row k reads, requested into L1 at once: the loads below
    // sit between divisions and would otherwise wait one at a time
    if (col < ncol && k < nk - 1) {
        const int km = k > 0 ? k - 1 : 0;
        for (int e = S_DJ; e <= S_PROD; ++e)
#pragma unroll
            for (int j = 0; j < 3; ++j) pf_l1(scr + (long)e * slab + (long)(km + j) * ld + col);
        pf_l1(F.bdotdh_djbz + o);
        pf_l1(F.bdotdh_djbz + o + ld);
        pf_l1(F.wi + o);
        pf_l1(F.wi + o + ld);
        pf_l1(F.explicit_h + o);
        pf_l1(F.optm1_smooth2 + o);
    }
    if (threadIdx.y == 0 && col < ncol) col_q[threadIdx.x] = oplus_col(F, C, A);
    __syncthreads();
    if (col >= ncol || k >= nk - 1) return;
    const OplusCol cc = col_q[threadIdx.x];
    A.gmr = cc.gmr;
    double p, q, r, ex, t_top = 0., t_bot = 0.;
    oplus_row(F, C, A, cc, k, p, q, r, ex, &t_top, &t_bot);
    if (k == nk - 2) scr[S_TB * slab + col] = t_top;
    if (k == 0) scr[S_TB * slab + ld + col] = t_bot;
    scr[S_P * slab + o] = p;
    scr[S_Q * slab + o] = q;
    scr[S_R * slab + o] = r;
    scr[S_EX * slab + o] = ex;
    if (sys_out) {
        sys_out[o] = p;
        sys_out[slab + o] = q;
        sys_out[2 * slab + o] = r;
        sys_out[3 * slab + o] = ex;
    }
}

// ---- the O+ sub-cycle: factor once, solve every sub-step -------------------
// Within one model step oplus_ng runs nstep_sub times (dynamics_ng.F90:103-
// 117) on the same fields; only op, optm1 (smoothed into optm1_smooth2) and
// the horizontal terms (explicit_h) change, and they enter the right-hand
// side alone.  The rows p, q, r and the forward elimination's w1, 1/w1 and w2
// are therefore the same in every sub-step: the factor pass forms them once,
// and each sub-step's solve runs the remaining recurrence w3 = (ex - p*w3)/w1
// (qdiv with the stored reciprocal) and the back sweep.  The operations and
// their order are those of the full walk, so the bits are too.

// Pass 3 of the factorization: w1, 1/w1 and w2 of every row, one column per
// thread.
__global__ void __launch_bounds__(32) k_oplus_factor(double *scr, int nk, int ncol, long ld, unsigned *status, int pd)
{
    const long col = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (col >= ncol) return;
    const long slab = (long)nk * ld;
    const int K = nk - 1;
    const double *P = scr + S_P * slab, *Q = scr + S_Q * slab, *R = scr + S_R * slab;
    double *W1 = scr + S_W1 * slab, *Y1 = scr + S_Y1 * slab, *W2 = scr + S_W2 * slab;
    auto pf_row = [&](int k) {
        const long o = (long)k * ld + col;
        pf_l1(P + o);
        pf_l1(Q + o);
        pf_l1(R + o);
    };
    for (int kk = 1; kk < pd && kk < K; ++kk) pf_row(kk);
    bool ok = true;
    double w1 = 0., y1 = 0., rprev = 0.;
    for (int k = 0; k < K; ++k) {
        if (k + pd < K) pf_row(k + pd);
        const long o = (long)k * ld + col;
        const double q = Q[o];
        if (k == 0) {
            w1 = q;
        } else {
            const double w2 = qdiv(rprev, w1, y1);
            W2[o - ld] = w2;
            w1 = xs(q, xm(P[o], w2));
        }
        y1 = __drcp_rn(w1);
        ok = ok && fabs(w1) <= DBL_MAX && w1 != 0.0;
        W1[o] = w1;
        Y1[o] = y1;
        rprev = R[o];
    }
    if (status && !ok) atomicOr(status, FLAG_PIVOT);
}

// The same pass for launches of few columns.  The kTileWarps warps of a
// block share one 32-column tile: together they copy the p, q, r rows of
// every level into shared memory (cp.async, every copy in flight, each warp
// a quarter of the levels); warp 0 alone runs the recurrence there, leaving
// 1/w1 where p(k) was, w1 where q(k) was and w2 where r(k-1) was; then all
// warps store the three planes, each its quarter of the levels.
constexpr int kTileWarps = 4;
__global__ void __launch_bounds__(32 * kTileWarps) k_oplus_factor_tile(double *scr, int nk, int ncol, long ld,
                                                                       unsigned *status)
{
    extern __shared__ double factor_tile[];
    const int T = 32, t = threadIdx.x & 31, w = threadIdx.x >> 5, NW = kTileWarps, K = nk - 1;
    const long col = (long)blockIdx.x * T + t, slab = (long)nk * ld;
    const bool live = col < ncol;
    double *sp = factor_tile, *sq = sp + (long)K * T, *sr = sq + (long)K * T;
    if (live)
        for (int k = w; k < K; k += NW) {
            const long o = (long)k * ld + col;
            const int s = k * T + t;
            cp_async8(sp + s, scr + S_P * slab + o);
            cp_async8(sq + s, scr + S_Q * slab + o);
            cp_async8(sr + s, scr + S_R * slab + o);
        }
    cp_async_commit();
    cp_async_wait<0>();
    __syncthreads();
    if (w == 0 && live) {
        // Level k forms the next level's w2 = r(k)/w1(k) and keeps it where
        // r(k) was.  The chain is the recurrence alone: quotients by
        // Markstein's sequence without a branch, operands read one level
        // ahead; from the first level whose operands leave the sequence's
        // safe range (stores stop there) the levels are walked again with
        // the IEEE fallback (qdiv1).
        bool ok = true;
        int bad = K;
        double w1 = 0., y1 = 0., w2 = 0.;
        auto level = [&](int k, double p, double q, double r, bool top_level) {
            w1 = k == 0 ? q : xs(q, xm(p, w2));
            y1 = __drcp_rn(w1);
            ok = ok && (bad < K || finite_nz(w1));
            const unsigned d = max(exp_dist(w1), top_level ? 0u : exp_dist(r));
            bad = d >= kExpSpan && bad == K ? k : bad;
            w2 = div_markstein(r, w1, y1);
            if (bad > k) {
                sq[k * T + t] = w1;
                sp[k * T + t] = y1;
                sr[k * T + t] = w2;
            }
        };
        double pn = sp[t], qn = sq[t], rn = sr[t];
        for (int k = 0; k < K - 1; ++k) {
            const int s = k * T + t;
            const double p = pn, q = qn, r = rn;
            pn = sp[s + T];
            qn = sq[s + T];
            rn = sr[s + T];
            level(k, p, q, r, false);
        }
        level(K - 1, pn, qn, rn, true);
        if (bad < K) {
            w2 = bad > 0 ? sr[(bad - 1) * T + t] : 0.;
            for (int k = bad; k < K; ++k) {
                const int s = k * T + t;
                w1 = k == 0 ? sq[s] : xs(sq[s], xm(sp[s], w2));
                y1 = __drcp_rn(w1);
                w2 = k + 1 < K ? qdiv1(sr[s], w1, y1) : 0.;
                ok = ok && finite_nz(w1);
                sq[s] = w1;
                sp[s] = y1;
                sr[s] = w2;
            }
        }
        if (status && !ok) atomicOr(status, FLAG_PIVOT);
    }
    __syncthreads();
    if (!live) return;
    double *W1 = scr + S_W1 * slab, *Y1 = scr + S_Y1 * slab, *W2 = scr + S_W2 * slab;
    for (int k = w; k < K; k += NW) {
        const long o = (long)k * ld + col;
        const int s = k * T + t;
        W1[o] = sq[s];
        Y1[o] = sp[s];
        if (k < K - 1) W2[o] = sr[s];
    }
}

// One sub-step's solve with the column tile in shared memory, the
// kTileWarps warps of a block on one 32-column tile: together they copy p,
// w1, 1/w1, w2 and the three right-hand-side inputs of every level (and the
// post-step inputs) at once (cp.async); warp 0 alone forms each level's ex
// as oplus_row forms it and runs the forward recurrence and the back sweep;
// all warps store the rows through the post-solve steps.
__global__ void __launch_bounds__(32 * kTileWarps) k_oplus_solve_tile(OplusFields F, OplusConsts C, const double *scr,
                                                                      double *opout, int nk, int ncol, long ld,
                                                                      unsigned *status, PostStep post, int has_post)
{
    extern __shared__ double solve_tile[];
    const int T = 32, t = threadIdx.x & 31, w = threadIdx.x >> 5, NW = kTileWarps, K = nk - 1;
    const long col = (long)blockIdx.x * T + t, slab = (long)nk * ld;
    const bool live = col < ncol;
    // ex, then the solution, in som: nk rows (the top row's extrapolation too)
    double *sp = solve_tile, *sw1 = sp + (long)K * T, *sy1 = sw1 + (long)K * T, *sw2 = sy1 + (long)K * T;
    double *sxh = sw2 + (long)K * T, *som = sxh + (long)K * T, *spr = som + (long)nk * T;
    // with the post-solve steps, prev and cur of the nk stored rows come in too
    double *sprev = spr + (long)K * T, *scur = sprev + (long)nk * T;
    if (live) {
        for (int k = w; k < K; k += NW) {
            const long o = (long)k * ld + col;
            const int s = k * T + t;
            cp_async8(sp + s, scr + S_P * slab + o);
            cp_async8(sw1 + s, scr + S_W1 * slab + o);
            cp_async8(sy1 + s, scr + S_Y1 * slab + o);
            cp_async8(sw2 + s, scr + S_W2 * slab + o);
            cp_async8(sxh + s, F.explicit_h + o);
            cp_async8(som + s, F.optm1_smooth2 + o);
            cp_async8(spr + s, scr + S_PROD * slab + o);
        }
        if (has_post)
            for (int k = w; k < nk; k += NW) {
                const long o = (long)k * ld + col;
                cp_async8(sprev + k * T + t, post.prev + o);
                cp_async8(scur + k * T + t, post.cur + o);
            }
    }
    const double t_top = w == 0 && live ? scr[S_TB * slab + col] : 0.;
    const double t_bot = w == 0 && live ? scr[S_TB * slab + ld + col] : 0.;
    cp_async_commit();
    cp_async_wait<0>();
    __syncthreads();
    if (w == 0 && live) {
        // ex formed as oplus_row forms it, then the recurrence; each level's
        // operands read one level ahead, so the ex arithmetic stays off the
        // recurrence's chain
        // quotients by Markstein's sequence without a branch; from the first
        // level whose operands leave its safe range (stores stop there) the
        // levels are walked again with the IEEE fallback (qdiv1)
        double w3 = 0.;
        int bad = K;
        auto ex_of = [&](int k, double xh, double om, double pr) {
            double ex = xs(xh, xm(xm(om, C.dtx2inv), (double)C.nstep_sub));
            if (k == nk - 2) ex = xs(ex, t_top);
            ex = xs(ex, pr);
            if (k == 0) ex = xs(ex, t_bot);
            return ex;
        };
        auto level = [&](int k, double ex, double p, double w1, double y1) {
            const double num = k == 0 ? ex : xs(ex, xm(p, w3));
            const unsigned d = max(exp_dist(num), exp_dist(w1));
            bad = d >= kExpSpan && bad == K ? k : bad;
            w3 = div_markstein(num, w1, y1);
            if (bad > k) som[k * T + t] = w3;
        };
        double xhn = sxh[t], omn = som[t], prn = spr[t], pn = sp[t], w1n = sw1[t], y1n = sy1[t];
        for (int k = 0; k < K - 1; ++k) {
            const int s = k * T + t;
            const double xh = xhn, om = omn, pr = prn, p = pn, w1 = w1n, y1 = y1n;
            xhn = sxh[s + T];
            omn = som[s + T];
            prn = spr[s + T];
            pn = sp[s + T];
            w1n = sw1[s + T];
            y1n = sy1[s + T];
            level(k, ex_of(k, xh, om, pr), p, w1, y1);
        }
        level(K - 1, ex_of(K - 1, xhn, omn, prn), pn, w1n, y1n);
        if (bad < K) {
            w3 = bad > 0 ? som[(bad - 1) * T + t] : 0.;
            for (int k = bad; k < K; ++k) {
                const int s = k * T + t;
                const double ex = ex_of(k, sxh[s], som[s], spr[s]);
                w3 = qdiv1(k == 0 ? ex : xs(ex, xm(sp[s], w3)), sw1[s], sy1[s]);
                som[s] = w3;
            }
        }
        const double xtop = w3;
        back_sweep(som, sw2, K, t, w3);
        // x(k) = w3 - w2*x(k+1) carries a non-finite value down to x(0)
        const bool fin = finite(som[t]) && finite(xtop);
        // opout(nk) = opout(nk-1)**2/opout(nk-2) from the unfiltered values (oplus_ng.F90:307)
        som[K * T + t] = xd(xm(xtop, xtop), som[(K - 2) * T + t]);
        if (status && !fin) atomicOr(status, FLAG_NONFINITE);
    }
    __syncthreads();
    if (!live) return;
    if (has_post) {
        const bool bcol = post.bnd_mask && post.bnd_mask[col];
        for (int k = w; k < nk; k += NW)
            post_store_v(post, bcol, opout, (long)k * ld + col, som[k * T + t], sprev[k * T + t], scur[k * T + t]);
    } else {
        for (int k = w; k < nk; k += NW) opout[(long)k * ld + col] = som[k * T + t];
    }
}

constexpr int kSolveThreads = 32;
// The same solve reading the rows from global memory (launches too large for
// the shared-memory tile), pd levels requested ahead.
__global__ void __launch_bounds__(kSolveThreads) k_oplus_solve(OplusFields F, OplusConsts C, const double *scr,
                                                               double *opout, int nk, int ncol, long ld,
                                                               unsigned *status, PostStep post, int has_post, int pd)
{
    const long col = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (col >= ncol) return;
    const int K = nk - 1;
    const long slab = (long)nk * ld;
    auto pf_row = [&](int k) {
        const long o = (long)k * ld + col;
        pf_l1(scr + S_P * slab + o);
        pf_l1(scr + S_W1 * slab + o);
        pf_l1(scr + S_Y1 * slab + o);
        pf_l1(F.explicit_h + o);
        pf_l1(F.optm1_smooth2 + o);
        pf_l1(scr + S_PROD * slab + o);
    };
    for (int kk = 1; kk < pd && kk < K; ++kk) pf_row(kk);
    const double t_top = scr[S_TB * slab + col], t_bot = scr[S_TB * slab + ld + col];
    double w3 = 0.;
    for (int k = 0; k < K; ++k) {
        if (k + pd < K) pf_row(k + pd);
        const long o = (long)k * ld + col;
        double ex = xs(F.explicit_h[o], xm(xm(F.optm1_smooth2[o], C.dtx2inv), (double)C.nstep_sub));
        if (k == nk - 2) ex = xs(ex, t_top);
        ex = xs(ex, scr[S_PROD * slab + o]);
        if (k == 0) {
            ex = xs(ex, t_bot);
            w3 = qdiv(ex, scr[S_W1 * slab + o], scr[S_Y1 * slab + o]);
        } else {
            w3 = qdiv(xs(ex, xm(scr[S_P * slab + o], w3)), scr[S_W1 * slab + o], scr[S_Y1 * slab + o]);
        }
        opout[o] = w3;
    }
    const bool bcol = has_post && post.bnd_mask && post.bnd_mask[col];
    double xn = w3;
    const double xtop = w3;
    bool fin = fabs(xn) <= DBL_MAX;
    double park = K >= 2 ? opout[(long)(K - 2) * ld + col] : 0.;
    for (int k = K - 2; k >= 0; --k) {
        if (k - pd >= 0) post_prefetch(post, has_post, bcol, opout, (long)(k - pd) * ld + col);
        const double wk = park;
        if (k >= 1) park = opout[(long)(k - 1) * ld + col];
        xn = xs(wk, xm(scr[S_W2 * slab + (long)k * ld + col], xn));
        fin = fin && fabs(xn) <= DBL_MAX;
        post_store(post, has_post, bcol, opout, (long)k * ld + col, xn);
        if (k == K - 2) {
            post_store(post, has_post, bcol, opout, (long)K * ld + col, xd(xm(xtop, xtop), xn));
            if (has_post) post_store(post, true, bcol, opout, (long)(K - 1) * ld + col, xtop);
        }
    }
    if (status && !fin) atomicOr(status, FLAG_NONFINITE);
}

// ---- oplus_ng's history diagnostics (oplus_ng.F90:309-330) ----------------
// Of the solution x (rows 1..nk, the top included, before the lateral
// overwrite and the post steps), one thread per (level, column): DOPDT,
// OP_PROD, OP_LOSS (= -op_loss*x), and on levels 2..nk-1 (1-based; 0 on the
// others, which the reference leaves unset) OP_DIFF, OP_DRIFT, OP_WIND: the
// horizontal term (diffexp, -vdotn_h, -bdotdh_bvel; 0 when not given) plus
// the vertical part's coefficients times x at k-1, k, k+1.
__global__ void __launch_bounds__(128) k_oplus_diag_ng(OplusFields F, OplusConsts C, const double *scr,
                                                       const double *x, const double *diffexp, const double *vdotn_h,
                                                       const double *bdotdh_bvel, int nk, int ncol, long ld,
                                                       double *diag)
{
    const long col = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (col >= ncol) return;
    const int k = blockIdx.y;
    const long slab = (long)nk * ld, o = (long)k * ld + col;
    auto D = [&](int n) -> double & { return diag[(long)n * slab + o]; };
    const double xk = __ldg(x + o);
    D(0) = xm(xm(xs(xk, __ldg(F.optm1_smooth2 + o)), C.dtx2inv), (double)C.nstep_sub);
    D(1) = scr[S_PROD * slab + o];
    D(2) = -xm(scr[S_OL * slab + o], xk);
    if (k == 0 || k == nk - 1) {
        D(3) = D(4) = D(5) = 0.0;
        return;
    }
    OplusRowsAt A{scr, slab, ld, col, nk, 0., 0., 0.};
    const OplusCol cc = oplus_col(F, C, A);
    A.gmr = cc.gmr;
    double pt[9];
    oplus_parts(F, C, A, cc, k, pt);
    const double xm1 = __ldg(x + o - ld), xp1 = __ldg(x + o + ld);
    const double *h3[3] = {diffexp, vdotn_h, bdotdh_bvel};
#pragma unroll
    for (int n = 0; n < 3; ++n) {
        const double hz = h3[n] ? __ldg(h3[n] + o) : 0.0;
        D(3 + n) = xa(xa(xa(n == 0 ? hz : -hz, xm(pt[3 * n], xm1)), xm(pt[3 * n + 1], xk)), xm(pt[3 * n + 2], xp1));
    }
}

cudaError_t launch_oplus_diag_ng(const OplusFields &F, const OplusConsts &C, const double *x, const double *diffexp,
                                 const double *vdotn_h, const double *bdotdh_bvel, int nk, int ncol, long ld,
                                 double *diag, double *scratch, cudaStream_t st)
{
    if (ncol <= 0) return cudaSuccess;
    if (nk < 3) return cudaErrorInvalidValue;
    const long slab = (long)nk * ld;
    // the level planes; the ion rates it also writes go to unused scratch planes
    k_oplus_levels<<<dim3((ncol + 127) / 128, nk), 128, 0, st>>>(F, C, scratch + S_W1 * slab, scratch + S_Y1 * slab,
                                                                 nullptr, nullptr, scratch, nk, ncol, ld);
    k_oplus_diag_ng<<<dim3((ncol + 127) / 128, nk), 128, 0, st>>>(F, C, scratch, x, diffexp, vdotn_h, bdotdh_bvel,
                                                                  nk, ncol, ld, diag);
    return cudaGetLastError();
}

cudaError_t launch_oplus_factor(const OplusFields &F, const OplusConsts &C, double *xiop2p, double *xiop2d,
                                double *factor, int nk, int ncol, long ld, unsigned *status, cudaStream_t st)
{
    if (ncol <= 0) return cudaSuccess;
    if (nk < 3) return cudaErrorInvalidValue;
    k_oplus_levels<<<dim3((ncol + 127) / 128, nk), 128, 0, st>>>(F, C, xiop2p, xiop2d, nullptr, nullptr, factor, nk,
                                                                 ncol, ld);
    k_oplus_coefs<<<coef_grid(nk, ncol), dim3(kCoefCols, kCoefRows), 0, st>>>(F, C, factor, nk, ncol, ld, nullptr);
    return launch_oplus_factor_pass(factor, nk, ncol, ld, status, st);
}

cudaError_t launch_oplus_factor_pass(double *factor, int nk, int ncol, long ld, unsigned *status, cudaStream_t st)
{
    if (ncol <= 0) return cudaSuccess;
    if (nk < 3) return cudaErrorInvalidValue;
    const size_t tile = (size_t)32 * 3 * (nk - 1) * sizeof(double);
    if (ncol <= kSmallWalkColumns && tile <= (size_t)smem_optin()) {
        once_per_device([] {
            cudaFuncSetAttribute(k_oplus_factor_tile, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_optin());
        });
        k_oplus_factor_tile<<<(ncol + 31) / 32, 32 * kTileWarps, tile, st>>>(factor, nk, ncol, ld, status);
    } else {
        k_oplus_factor<<<(ncol + 31) / 32, 32, 0, st>>>(factor, nk, ncol, ld, status, walk_prefetch(ncol));
    }
    return cudaGetLastError();
}

cudaError_t launch_oplus_solve(const OplusFields &F, const OplusConsts &C, const double *factor, double *opout, int nk,
                               int ncol, long ld, unsigned *status, cudaStream_t st, const PostStep *post)
{
    if (ncol <= 0) return cudaSuccess;
    if (nk < 3) return cudaErrorInvalidValue;
    const PostStep pv = post ? *post : PostStep{};
    const int hp = post != nullptr;
    const size_t tile = (size_t)32 * (7 * (nk - 1) + 1 + (post ? 2 * nk : 0)) * sizeof(double);
    const int T = kSolveThreads;
    if (ncol <= kSmallWalkColumns && tile <= (size_t)smem_optin()) {
        once_per_device([] {
            cudaFuncSetAttribute(k_oplus_solve_tile, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_optin());
        });
        k_oplus_solve_tile<<<(ncol + 31) / 32, 32 * kTileWarps, tile, st>>>(F, C, factor, opout, nk, ncol, ld, status,
                                                                            pv, hp);
    } else {
        k_oplus_solve<<<(ncol + T - 1) / T, T, 0, st>>>(F, C, factor, opout, nk, ncol, ld, status, pv, hp,
                                                        walk_prefetch(ncol));
    }
    return cudaGetLastError();
}

cudaError_t launch_oplus_ng(const OplusFields &F, const OplusConsts &C, double *opout, double *xiop2p,
                            double *xiop2d, double *Fe, double *Fn, double *scratch, int nk, int ncol, long ld,
                            double *sys_out, unsigned *status, cudaStream_t st, const PostStep *post)
{
    const PostStep pv = post ? *post : PostStep{};
    const int hp = post != nullptr;
    if (ncol <= 0) return cudaSuccess;
    if (nk < 3) return cudaErrorInvalidValue;
    const int optin = smem_optin();
    once_per_device([optin] {
        cudaFuncSetAttribute(k_oplus_ng, cudaFuncAttributeMaxDynamicSharedMemorySize, optin);
        cudaFuncSetAttribute(k_oplus_rows, cudaFuncAttributeMaxDynamicSharedMemorySize, optin);
    });
    int T = 128;
    const size_t per = (size_t)(nk - 1) * sizeof(double);
    while (T > 32 && (size_t)T * per > (size_t)optin) T /= 2;
    if ((size_t)T * per > (size_t)optin) return cudaErrorInvalidValue;
    const int pd = walk_prefetch(ncol);
    if (assembly_mode() == 2) {
        const long slab = (long)nk * ld;
        k_oplus_levels<<<dim3((ncol + 127) / 128, nk), 128, 0, st>>>(F, C, xiop2p, xiop2d, Fe, Fn, scratch, nk, ncol,
                                                                     ld);
        k_oplus_coefs<<<coef_grid(nk, ncol), dim3(kCoefCols, kCoefRows), 0, st>>>(F, C, scratch, nk, ncol, ld,
                                                                                  sys_out);
        return launch_thomas_post(scratch + S_P * slab, scratch + S_Q * slab, scratch + S_R * slab,
                                  scratch + S_EX * slab, opout, nk, nk - 1, 1, ncol, ld, status, post, st);
    }
    if (assembly_mode() >= 1) {
        k_oplus_levels<<<dim3((ncol + 127) / 128, nk), 128, 0, st>>>(F, C, xiop2p, xiop2d, Fe, Fn, scratch, nk, ncol,
                                                                     ld);
        k_oplus_rows<<<(ncol + T - 1) / T, T, (size_t)T * per, st>>>(F, C, opout, scratch, nk, ncol, ld, sys_out,
                                                                     status, pv, hp, pd);
        return cudaGetLastError();
    }
    k_oplus_ng<<<(ncol + T - 1) / T, T, (size_t)T * per, st>>>(F, C, opout, xiop2p, xiop2d, Fe, Fn, scratch, nk, ncol,
                                                               ld, sys_out, status, pv, hp, pd);
    return cudaGetLastError();
}

int oplus_scratch_planes() { return S_N; }
}  // namespace tg
