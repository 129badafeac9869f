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

namespace tg {
namespace {
__device__ __forceinline__ double xm(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double xa(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double xs(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double xd(double a, double b) { return __ddiv_rn(a, b); }

// scratch planes, level-major
enum { S_DJ = 0, S_HDZ, S_TP1, S_BDOTU, S_OL, S_PROD, S_N };

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

// Rows k = 0..nk-2 from the level planes, the forward sweep and the back
// sweep of one column (oplus_ng.F90:88-99, 209-307).
__device__ __forceinline__ void oplus_walk(const OplusFields &F, const OplusConsts &C, double *opout, const double *scr,
                                           double *w2s, int T, int nk, long ld, long col, double *sys_out,
                                           unsigned *status, const PostStep &post, int has_post)
{
    const long slab = (long)nk * ld;
    auto at = [&](const double *p, int k) { return __ldg(p + k * ld + col); };
    auto S = [&](int e, int k) { return scr[(long)e * slab + (long)k * ld + col]; };
    // pi = 4*atan(1) of the reference, correctly rounded
    const double pi = 3.141592653589793, rtd = 180. / pi;
    const double phid = 2.0e8, phin = -2.0e8, ppolar = 0.;
    const double bz = __ldg(F.bz + col);
    // oplus_flux (oplus_ng.F90:88-99)
    double opflux;
    {
        const double arl = fabs(__ldg(F.rlatm + col)), chi = __ldg(F.chi + col);
        double a = 0.;
        if (arl >= xd(pi, 4.5)) a = 1.;
        if (arl < xd(pi, 4.5) && arl > xd(pi, 18.)) a = xm(.5, xa(1., cos(xs(xm(arl, 6.), xd(xm(pi, 4.), 3.)))));
        if (arl <= xd(pi, 18.)) a = 0.;
        const double fed = xm(phid, a), fen = xm(phin, a);
        opflux = chi >= xm(0.5, pi) ? fen : fed;
        const double cd = xm(chi, rtd);
        if (xm(xs(cd, 80.), xs(cd, 100.)) < 0.)
            opflux = xa(xm(.5, xa(fed, fen)), xm(xm(.5, xs(fed, fen)), cos(xd(xm(pi, xs(cd, 80.)), 20.))));
        if (arl >= xd(pi, 3.)) opflux = xa(opflux, ppolar);
    }
    // ---- pass 2: rows and the forward sweep (oplus_ng.F90:209-303)
    const double dvbz = xd(__ldg(F.dvb + col), bz), bz2 = xm(bz, bz);
    const double gmr = xd(xm(C.grav, C.rmass_op), xm(2., C.gask));
    const double dtn = xm(C.dtx2inv, (double)C.nstep_sub);
    auto hdzi = [&](int j) {
        if (j == 0) return xs(xm(1.5, S(S_HDZ, 0)), xm(0.5, S(S_HDZ, 1)));
        if (j == nk - 1) return xs(xm(1.5, S(S_HDZ, nk - 2)), xm(0.5, S(S_HDZ, nk - 3)));
        return xm(0.5, xa(S(S_HDZ, j - 1), S(S_HDZ, j)));
    };
    auto tph1 = [&](int j) {
        if (j == nk - 1) return xa(xm(xm(2., xs(xm(2., S(S_TP1, nk - 2)), S(S_TP1, nk - 3))), hdzi(nk - 1)), gmr);
        return xa(xm(xm(2., S(S_TP1, j)), hdzi(j)), gmr);
    };
    auto tph0 = [&](int j) {
        if (j == 0) return xs(xm(xm(2., xs(xm(2., S(S_TP1, 0)), S(S_TP1, 1))), hdzi(0)), gmr);
        return xs(xm(xm(2., S(S_TP1, j - 1)), hdzi(j)), gmr);
    };
    auto djint = [&](int j) {
        if (j == 0) return xs(xm(1.5, S(S_DJ, 0)), xm(0.5, S(S_DJ, 1)));
        if (j == nk - 1) return xs(xm(1.5, S(S_DJ, nk - 2)), xm(0.5, S(S_DJ, nk - 3)));
        return xm(0.5, xa(S(S_DJ, j - 1), S(S_DJ, j)));
    };
    auto hdzmp = [&](int j, double sgn) {
        const double divbz = xa(dvbz, xd(at(F.bdotdh_djbz, j), xm(S(S_DJ, j), bz2)));
        const double h = S(S_HDZ, j);
        return xm(sgn > 0 ? xa(h, xm(0.5, divbz)) : xs(h, xm(0.5, divbz)), bz2);
    };
    const double ubca = xm(xm(-bz2, djint(nk - 1)), tph1(nk - 1));
    const double ubcb = xm(xm(-bz2, djint(nk - 1)), tph0(nk - 1));
    bool ok = true;
    double w1 = 0., y1 = 0., w3 = 0., rprev = 0.;
    // bring the lines row k+1 touches first (the planes at level k+2, the
    // fields at k+1) into L1 while row k computes
    auto pf = [&](const double *p) { asm volatile("prefetch.global.L1 [%0];" ::"l"(p)); };
    for (int k = 0; k < nk - 1; ++k) {
        if (k + 1 < nk - 1) {
            const long o1 = (long)(k + 1) * ld + col;
            if (k + 2 < nk) {
#pragma unroll
                for (int e = 0; e < 4; ++e) pf(scr + (long)e * slab + o1 + ld);
                pf(F.wi + o1 + ld);
            }
            pf(F.bdotdh_djbz + o1);
            pf(F.explicit_h + o1);
            pf(F.optm1_smooth2 + o1);
            pf(scr + (long)S_OL * slab + o1);
            pf(scr + (long)S_PROD * slab + o1);
        }
        const double hdzm_k = hdzmp(k, -1.), hdzp_k = hdzmp(k, 1.);
        const double dji_k = djint(k), dji_1 = djint(k + 1);
        const double t0k = tph0(k), t1k = tph1(k), t01 = tph0(k + 1), t11 = tph1(k + 1);
        const double hdz_k = S(S_HDZ, k);
        const double diffp = xm(xm(hdzm_k, dji_k), t0k);
        const double diffq = -xa(xm(xm(hdzp_k, dji_1), t01), xm(xm(hdzm_k, dji_k), t1k));
        const double diffr = xm(xm(hdzp_k, dji_1), t11);
        const double wii = up(F.wi, k, nk, ld, col);
        const double driftp = xm(xm(wii, 0.5), hdz_k);
        const double driftq = xd(xm(-wii, 6.), C.re);
        const double driftr = xm(xm(-wii, 0.5), hdz_k);
        const double bu_k = S(S_BDOTU, k);
        const double windp = k == 0 ? xm(xm(xm(bz, xs(xm(2., bu_k), S(S_BDOTU, 1))), 0.5), hdz_k)
                                    : xm(xm(xm(bz, S(S_BDOTU, k - 1)), 0.5), hdz_k);
        const double windq = xm(xm(-bu_k, dvbz), bz);
        const double windr = k == nk - 2 ? xm(xm(xm(bz, xs(xm(2., bu_k), S(S_BDOTU, k - 1 >= 0 ? k - 1 : 0))), 0.5), hdz_k)
                                         : xm(xm(xm(-bz, S(S_BDOTU, k + 1)), 0.5), hdz_k);
        double p = xa(xa(diffp, driftp), windp);
        double q = xs(xa(xa(diffq, driftq), windq), dtn);
        double r = xa(xa(diffr, driftr), windr);
        double ex = xs(at(F.explicit_h, k), xm(xm(at(F.optm1_smooth2, k), C.dtx2inv), (double)C.nstep_sub));
        if (k == nk - 2) {
            q = xa(q, xm(xd(ubcb, ubca), r));
            ex = xs(ex, xd(xm(opflux, r), ubca));
            r = 0.;
        }
        q = xs(q, S(S_OL, k));
        ex = xs(ex, S(S_PROD, k));
        if (k == 0) {
            q = xs(q, p);
            ex = xs(ex, xd(xm(xm(2., p), at(F.qop, 0)), xs(xm(1.5, S(S_OL, 0)), xm(0.5, S(S_OL, 1)))));
            p = 0.;
        }
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
    for (int k = K - 2; k >= 0; --k) {
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
                                                  PostStep post, int has_post)
{
    extern __shared__ double smem_op[];
    const long col = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (col >= ncol) return;
    for (int j = 0; j < nk; ++j) oplus_level(F, C, scr, xiop2p, xiop2d, Fe, Fn, nk, ld, col, j);
    oplus_walk(F, C, opout, scr, smem_op + threadIdx.x, blockDim.x, nk, ld, col, sys_out, status, post, has_post);
}

// Two-pass form: the level quantities with one thread per (level, column),
// then the column walk.
__global__ void __launch_bounds__(128) k_oplus_levels(OplusFields F, OplusConsts C, double *xiop2p, double *xiop2d,
                                                      double *Fe, double *Fn, double *scr, int nk, int ncol, long ld)
{
    const long col = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (col >= ncol) return;
    oplus_level(F, C, scr, xiop2p, xiop2d, Fe, Fn, nk, ld, col, blockIdx.y);
}

__global__ void __launch_bounds__(128) k_oplus_rows(OplusFields F, OplusConsts C, double *opout, const double *scr,
                                                    int nk, int ncol, long ld, double *sys_out, unsigned *status,
                                                    PostStep post, int has_post)
{
    extern __shared__ double smem_or[];
    const long col = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (col >= ncol) return;
    oplus_walk(F, C, opout, scr, smem_or + threadIdx.x, blockDim.x, nk, ld, col, sys_out, status, post, has_post);
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
    if (assembly_mode() == 1) {
        k_oplus_levels<<<dim3((ncol + 127) / 128, nk), 128, 0, st>>>(F, C, xiop2p, xiop2d, Fe, Fn, scratch, nk, ncol,
                                                                     ld);
        k_oplus_rows<<<(ncol + T - 1) / T, T, (size_t)T * per, st>>>(F, C, opout, scratch, nk, ncol, ld, sys_out,
                                                                     status, pv, hp);
        return cudaGetLastError();
    }
    k_oplus_ng<<<(ncol + T - 1) / T, T, (size_t)T * per, st>>>(F, C, opout, xiop2p, xiop2d, Fe, Fn, scratch, nk, ncol,
                                                               ld, sys_out, status, pv, hp);
    return cudaGetLastError();
}

int oplus_scratch_planes() { return S_N; }
}  // namespace tg
