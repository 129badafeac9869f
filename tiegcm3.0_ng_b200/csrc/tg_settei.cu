// settei_ng (electron and ion temperatures), src/settei_ng.F90:60-261, as one
// fused kernel: the routine is column-local from its first statement to its
// last, so one thread per column assembles the conduction system in Te^3.5,
// solves it and finishes Te and Ti without any intermediate touching memory
// except the Thomas w2 (shared memory) and two parked values per level.
//
// Row k (k = 0..nk-2) needs the interface quantities (te_int, the interface
// number densities, tek0) of levels k and k+1, and the heating / cooling of
// level k, which in turn reads levels k and k+1 (qtot, root_ne).  A thread
// keeps a window of levels k-1..k+1.  During the forward sweep w3 is parked
// in te_out and loss_ei in ti_out; loss_in sits in shared memory next to w2.
// The back sweep turns x = Te^3.5 into Te, extrapolates the top level and
// forms Ti.
//
// Every operation is the reference's, in its order, with non-contracting FP64
// intrinsics.  The transcendental functions (pow, exp, log, sin, cos) are the
// device library's, within a few ulp of the host C library's, so the kernel
// agrees with the CPU restatement to a stated tolerance, not bit for bit.
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
// max as the CPU restatement writes it (a > b ? a : b)
__device__ __forceinline__ double dmax(double a, double b) { return a > b ? a : b; }

// Fields of one level that the window carries.
struct Lev {
    double te, tn, o2, o1, he, n2;
};

__device__ __forceinline__ Lev load_lev(const SetteiFields &F, long o)
{
    Lev L;
    L.te = __ldg(F.te + o);
    L.tn = __ldg(F.tn + o);
    L.o2 = __ldg(F.o2 + o);
    L.o1 = __ldg(F.o1 + o);
    L.he = __ldg(F.he + o);
    L.n2 = __ldg(F.n2 + o);
    return L;
}

// tek0/h_int of an interface from its raw averages (settei_ng.F90:116-139)
struct Iface {
    double tek0, th, tn_int;
};

__device__ __forceinline__ Iface iface(const SetteiConsts &C, double te_int, double o2n, double o1n, double hen,
                                       double n2n, double tn_int, double xnmbari, double ne, double h_int)
{
    n2n = dmax(n2n, 0.);
    o2n = xm(xm(xnmbari, o2n), C.rmassinv_o2);
    o1n = xm(xm(xnmbari, o1n), C.rmassinv_o1);
    hen = xm(xm(xnmbari, hen), C.rmassinv_he);
    n2n = xm(xm(xnmbari, n2n), C.rmassinv_n2);
    const double rt = sqrt(te_int);
    double s = xm(xa(2.20e-16, xm(7.92e-18, rt)), o2n);
    s = xa(s, xm(xm(1.10e-16, xa(1.0, xm(5.7e-4, te_int))), o1n));
    s = xa(s, xm(5.60e-16, hen));
    s = xa(s, xm(xm(xs(2.82e-17, xm(3.41e-21, te_int)), rt), n2n));
    const double X = xm(xd(xm(3.22e4, xm(te_int, te_int)), ne), s);
    Iface I;
    I.tek0 = xm(xd(7.5e5, xa(1.0, X)), C.evergs);
    I.th = xd(I.tek0, h_int);
    I.tn_int = tn_int;
    return I;
}

__device__ __forceinline__ double qsum(const SetteiFields &F, long o)
{
    double s = xa(__ldg(F.qo2p + o), __ldg(F.qop + o));
    s = xa(s, __ldg(F.qn2p + o));
    s = xa(s, __ldg(F.qnop + o));
    s = xa(s, __ldg(F.qnp + o));
    s = xa(s, __ldg(F.qop2d + o));
    s = xa(s, __ldg(F.qop2p + o));
    return dmax(s, 1.e-20);
}
}  // namespace

namespace {
// Heating, cooling and exchange of one level (settei_ng.F90:157-246).
struct Loss {
    double dq;      // subtracted from q: (loss_en+loss_ei)/te**2.5
    double qe_h;    // qe*qtot*evergs, subtracted from rhs first
    double et_h;    // (Q1+Q2)*10 when et
    double len_tn;  // loss_en*tn
    double lei_ti;  // loss_ei*ti
    double lei, lin, q_eni;
};

__device__ __forceinline__ Loss level_loss(const SetteiFields &F, const SetteiConsts &C, long o, const Lev &L,
                                           double rne_raw, double qtot)
{
    const double del = 1.e-6, alam = 0.0069, ad = 0.0091, sd = 2.3e-11, ev = C.evergs;
    const double xn = __ldg(F.xnmbar + o), ti = __ldg(F.ti + o);
    const double rne = sqrt(dmax(rne_raw, 1.e4));
    const double o2n = xm(xm(xn, L.o2), C.rmassinv_o2);
    const double o1n = xm(xm(xn, L.o1), C.rmassinv_o1);
    const double hen = xm(xm(xn, L.he), C.rmassinv_he);
    const double n2n = xm(xm(xn, L.n2), C.rmassinv_n2);
    double qe;
    if (C.electron_heating == 6) {
        qe = log(xd(rne, xa(xa(o2n, n2n), o1n)));
        double t = xs(xm(-1.249e-5, qe), 5.755e-4);
        t = xs(xm(t, qe), 9.346e-3);
        t = xs(xm(t, qe), 5.900e-2);
        t = xs(xm(t, qe), 4.392e-2);
        t = xa(xm(t, qe), 1.056);
        t = xa(xm(t, qe), 5.342);
        qe = exp(t);
    } else {
        qe = log(xd(rne, xa(xa(o2n, n2n), xm(0.1, o1n))));
        double t = xa(xm(0.001996, qe), 0.08034);
        t = xa(xm(t, qe), 1.166);
        t = xa(xm(t, qe), 6.941);
        t = xa(xm(t, qe), 12.75);
        qe = exp(-t);
    }
    Loss R;
    R.qe_h = xm(xm(qe, qtot), ev);
    R.et_h = C.et ? xm(xa(__ldg(F.Q1 + o), __ldg(F.Q2 + o)), 10.0) : 0.0;
    const double te = L.te, tn = L.tn, rt = sqrt(te);
    double coll = te >= 1000. ? xm(2.e-7, exp(xd(-4605.2, te))) : xm(5.71e-8, exp(xd(-3352.6, te)));
    if (te > 2000.) coll = xm(xm(2.53e-6, rt), exp(xd(-17620., te)));
    double l2v;
    if (fabs(xs(te, tn)) < del) l2v = xd(3200., xm(tn, tn));
    else l2v = xm(xd(1., xs(te, tn)), xs(1., exp(xd(xm(-3200., xs(te, tn)), xm(te, tn)))));
    l2v = xm(xm(1.3e-4, l2v), coll);
    const double leo2 = xm(o2n, xa(xa(xm(xm(1.21e-18, xa(1., xm(3.6e-2, rt))), rt), xd(6.9e-14, rt)),
                                   xm(3.125e-21, xm(te, te))));
    const double leo1d = 0.;
    const double leo1 = xm(o1n, xa(xm(xm(7.9e-19, xa(1., xm(5.7e-4, te))), rt),
                                   xm(xd(xm(3.4e-12, xs(1., xm(7.e-5, te))), tn), xa(xd(150., te), 0.4))));
    const double lehe = xm(xm(hen, 2.46e-17), rt);
    const double len2 = xm(n2n, xa(xa(xm(xm(1.77E-19, xs(1., xm(1.21E-4, te))), te), xd(2.9e-14, rt)), l2v));
    double len = xa(xa(xa(leo2, leo1), lehe), len2);
    if (C.et && te > 500.0 && __ldg(F.Q2 + o) > 0.0) len = xm(len, exp(xm(-7.54E-4, xs(te, 500.0))));
    const double lxen = xm(xm(xa(len, xm(xm(o1n, xs(1., xd(alam, xa(ad, xm(sd, n2n))))), leo1d)), rne), ev);
    len = xm(xm(xa(len, xm(o1n, leo1d)), rne), ev);
    double ions = xm(__ldg(F.op + o), C.rmassinv_o1);
    ions = xa(ions, xm(__ldg(F.o2p + o), C.rmassinv_o2));
    ions = xa(ions, xm(__ldg(F.nplus + o), C.rmassinv_n4s));
    ions = xa(ions, xm(__ldg(F.n2p + o), C.rmassinv_n2));
    ions = xa(ions, xm(__ldg(F.nop + o), C.rmassinv_no));
    const double lei = xm(xm(xm(xm(xd(xm(3.2e-8, rne), xm(rt, te)), 15.), ev), C.rmass_o1), ions);
    const double rtn = sqrt(xm(2.0, tn));
    const double op = __ldg(F.op + o), o2p = __ldg(F.o2p + o), npl = __ldg(F.nplus + o), n2p = __ldg(F.n2p + o),
                 nop = __ldg(F.nop + o);
    double s = xm(op, xa(xa(xa(xm(5.8, o2n), xm(xm(0.21, o1n), rtn)), xm(2.8, hen)), xm(6.6, n2n)));
    s = xa(s, xm(o2p, xa(xa(xa(xm(xm(0.14, o2n), rtn), xm(4.36, o1n)), xm(1.63, hen)), xm(5.81, n2n))));
    s = xa(s, xm(npl, xa(xa(xa(xm(5.84, o2n), xm(5.84, o1n)), xm(3.05, hen)), xm(6.56, n2n))));
    s = xa(s, xm(n2p, xa(xa(xa(xm(5.54, o2n), xm(4.65, o1n)), xm(1.82, hen)), xm(xm(0.27, n2n), rtn))));
    s = xa(s, xm(nop, xa(xa(xa(xm(5.45, o2n), xm(4.5, o1n)), xm(1.72, hen)), xm(5.92, n2n))));
    const double lin = xm(xm(1e-14, ev), s);
    R.dq = xd(xa(len, lei), pow(te, 2.5));
    R.len_tn = xm(len, tn);
    R.lei_ti = xm(lei, ti);
    R.lei = lei;
    R.lin = lin;
    const double qi = xm(lei, dmax(xs(te, ti), 0.));
    R.q_eni = xd(xm(xa(xm(lxen, xs(te, tn)), qi), C.avo), xn);
    return R;
}
}  // namespace

__global__ void __launch_bounds__(128) k_settei_ng(SetteiFields F, SetteiConsts C, double *te_out, double *ti_out,
                                                   double *qtotal, int nk, int ncol, long ld, double *sys_out,
                                                   unsigned *status)
{
    extern __shared__ double smem_te[];
    const long col = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (col >= ncol) return;
    const int T = blockDim.x;
    double *w2s = smem_te + threadIdx.x;                     // w2, levels 0..nk-2
    double *lins = smem_te + (long)T * (nk - 1) + threadIdx.x;   // loss_in, levels 0..nk-1
    const long slab = (long)nk * ld;
    // pi = 4*atan(1) of the reference, correctly rounded
    const double pi = 3.141592653589793, rtd = 180.0 / pi, ev = C.evergs, dz = C.dz;
    const double fpolar = -3.0e+9;
    // fe: the upper-boundary heat flux (settei_ng.F90:62-87)
    double fe;
    {
        const double f107te = C.f107 < 235. ? C.f107 : 235.;
        const double arl = fabs(__ldg(F.rlatm + col)), chi = __ldg(F.chi + col), qa = __ldg(F.qteaur + col);
        double a = 0.;
        if (arl >= xd(pi, 4.5)) a = 1.;
        if (arl < xd(pi, 4.5) && arl > xd(pi, 18.)) a = xm(.5, xa(1., cos(xs(xm(arl, 6.), xd(xm(pi, 4.), 3.)))));
        if (arl <= xd(pi, 18.)) a = 0.;
        double fed = xm(xm(-9.0e+7, f107te), a);
        double fen = xd(fed, 2.);
        fed = xa(fed, qa);
        fen = xa(fen, qa);
        fe = chi >= xm(.5, pi) ? fen : fed;
        const double cd = xm(chi, rtd);
        if (xm(xs(cd, 80.), xs(cd, 100.)) >= 0.) fe = xm(fe, ev);
        else
            fe = xm(xa(xm(.5, xa(fed, fen)), xm(xm(.5, xs(fed, fen)), cos(xd(xm(pi, xs(cd, 80.)), 20.)))), ev);
        if (arl >= xd(pi, 3.)) fe = xa(fe, xm(fpolar, ev));
    }
    double sindip;
    {
        const double dm = fabs(__ldg(F.dipmag + col));
        const double s = sin(dm > C.dipmin ? dm : C.dipmin);
        sindip = dmax(xm(s, s), .10);
    }
    const double t_lbc = __ldg(F.t_lbc + col);
    auto at = [&](const double *p, int k) { return __ldg(p + k * ld + col); };
    // window of levels k-1, k, k+1
    Lev Lm = {}, L0 = load_lev(F, col), Lp = load_lev(F, ld + col);
    // interface 0 (settei_ng.F90:98-103)
    Iface I0;
    {
        const double *b = C.b, *fb = C.fb;
        const double te_int = dmax(xs(xm(1.5, L0.te), xm(.5, Lp.te)), t_lbc);
        const double o2n = xm(.5, xa(xa(xa(fb[0], xm(xa(b[0], 1.), L0.o2)), xm(b[3], L0.o1)), xm(b[6], L0.he)));
        const double o1n = xm(.5, xa(xa(xa(fb[0], xm(b[0], L0.o2)), xm(xa(b[3], 1.), L0.o1)), xm(b[6], L0.he)));
        const double hen = xm(.5, xa(xa(xa(fb[0], xm(b[0], L0.o2)), xm(b[3], L0.o1)), xm(xa(b[6], 1.), L0.he)));
        const double n2n = dmax(xs(xs(xs(1., o2n), o1n), hen), 0.);
        I0 = iface(C, te_int, o2n, o1n, hen, n2n, t_lbc, at(F.xnmbari, 0), at(F.ne, 0), at(F.schti, 0));
    }
    double qs0 = qsum(F, col), qs1 = qsum(F, ld + col);
    double ne0 = at(F.ne, 0), ne1 = at(F.ne, 1);
    double qe_m1 = 0.;                    // q_eni of level k-1
    double w1 = 0., w3 = 0., rprev = 0.;
    bool ok = true;
    for (int k = 0; k < nk; ++k) {
        const long o = (long)k * ld + col;
        // level-k heating and losses (needs levels k and k+1)
        const double qtot = k < nk - 1 ? sqrt(xm(qs0, qs1)) : 0.;
        const double rne_raw = k < nk - 1 ? xm(ne0, ne1) : xd(xm(xm(ne0, ne0), ne0), ne1);
        const Loss R = level_loss(F, C, o, L0, rne_raw, qtot);
        ti_out[o] = R.lei;     // parked until the back sweep
        lins[(long)k * T] = R.lin;
        // qtotal += q_eni at the interfaces (settei_ng.F90:248-254)
        if (k == 1) qtotal[col] = xa(qtotal[col], xs(xm(1.5, qe_m1), xm(0.5, R.q_eni)));
        if (k >= 1 && k <= nk - 2) qtotal[o] = xa(qtotal[o], xm(.5, xa(qe_m1, R.q_eni)));
        if (k == nk - 2) {
            const double qe_prev = k >= 1 ? qe_m1 : 0.;
            qtotal[(long)(nk - 1) * ld + col] = xa(qtotal[(long)(nk - 1) * ld + col], xs(xm(1.5, R.q_eni), xm(0.5, qe_prev)));
        }
        if (k <= nk - 2) {
            // interface k+1 (settei_ng.F90:89-112)
            Iface I1;
            if (k + 1 < nk - 1) {
                I1 = iface(C, xm(.5, xa(Lp.te, L0.te)), xm(.5, xa(Lp.o2, L0.o2)), xm(.5, xa(Lp.o1, L0.o1)),
                           xm(.5, xa(Lp.he, L0.he)), xm(.5, xa(Lp.n2, L0.n2)), xm(.5, xa(Lp.tn, L0.tn)),
                           at(F.xnmbari, k + 1), at(F.ne, k + 1), at(F.schti, k + 1));
            } else {
                // top interface: te_int and tn_int extrapolated from levels nk-2, nk-3
                const double te_im = k >= 1 ? Lm.te : 0., tn_im = k >= 1 ? Lm.tn : 0.;
                I1 = iface(C, xs(xm(1.5, L0.te), xm(.5, te_im)), xm(.5, xa(Lp.o2, L0.o2)), xm(.5, xa(Lp.o1, L0.o1)),
                           xm(.5, xa(Lp.he, L0.he)), xm(.5, xa(Lp.n2, L0.n2)), xs(xm(1.5, L0.tn), xm(.5, tn_im)),
                           at(F.xnmbari, k + 1), at(F.ne, k + 1), at(F.schti, k + 1));
            }
            // row k (settei_ng.F90:131-155, 183, 240-242)
            const double pb = xm(xd(xd(2., 7.), xm(at(F.scht, k), xm(dz, dz))), sindip);
            double r = xm(pb, I1.th);
            double p = xm(pb, I0.th);
            double q = -xa(p, r);
            double rhs = 0.;
            if (k == 0) {
                q = xs(q, p);
                rhs = xs(rhs, xm(xm(2., p), pow(I0.tn_int, 3.5)));
                p = 0.;
            }
            if (k == nk - 2) {
                q = xa(q, r);
                rhs = xa(rhs, xd(xm(xm(xm(xm(r, dz), 3.5), at(F.schti, nk - 1)), fe), I1.tek0));
                r = 0.;
            }
            rhs = xs(rhs, R.qe_h);
            if (C.et) rhs = xs(rhs, R.et_h);
            q = xs(q, R.dq);
            rhs = xs(xs(rhs, R.len_tn), R.lei_ti);
            if (sys_out) {
                sys_out[o] = p;
                sys_out[slab + o] = q;
                sys_out[2 * slab + o] = r;
                sys_out[3 * slab + o] = rhs;
            }
            // Thomas forward (trsolv_ng.F90:14-22), k2 = nk-1
            if (k == 0) {
                w1 = q;
                w3 = xd(rhs, w1);
            } else {
                const double w2 = xd(rprev, w1);
                w2s[(long)(k - 1) * T] = w2;
                w1 = xs(q, xm(p, w2));
                w3 = xd(xs(rhs, xm(p, w3)), w1);
            }
            ok = ok && fabs(w1) <= DBL_MAX && w1 != 0.0;
            te_out[o] = w3;
            rprev = r;
            I0 = I1;
        }
        // slide the window
        qe_m1 = R.q_eni;
        Lm = L0;
        L0 = Lp;
        qs0 = qs1;
        ne0 = ne1;
        if (k + 2 < nk) {
            Lp = load_lev(F, (long)(k + 2) * ld + col);
            qs1 = qsum(F, (long)(k + 2) * ld + col);
            ne1 = at(F.ne, k + 2);
        } else {
            ne1 = at(F.ne, nk - 2);   // the top level's root_ne divides by ne(nk-1)
        }
    }
    // back sweep, x = Te^3.5 -> Te, top level, Ti (settei_ng.F90:256-261)
    const int K = nk - 1;
    double xn = w3;
    double tk = pow(xn, xd(2., 7.));
    double t_top1 = tk, t_top2 = 0.;
    bool fin = fabs(xn) <= DBL_MAX;
    auto finish = [&](int k, double t) {
        const long o = (long)k * ld + col;
        const double tn = at(F.tn, k);
        const double te = dmax(t, tn);
        const double lei = ti_out[o], lin = lins[(long)k * T];
        te_out[o] = te;
        const double num = xa(xa(xd(xm(at(F.qji_ti, k), at(F.xnmbar, k)), C.avo), xm(lei, te)), xm(lin, tn));
        ti_out[o] = dmax(xd(num, xa(lei, lin)), tn);
    };
    finish(K - 1, tk);
    for (int k = K - 2; k >= 0; --k) {
        xn = xs(te_out[(long)k * ld + col], xm(w2s[(long)k * T], xn));
        fin = fin && fabs(xn) <= DBL_MAX;
        tk = pow(xn, xd(2., 7.));
        if (k == K - 2) t_top2 = tk;
        finish(k, tk);
    }
    finish(K, xd(xm(t_top1, t_top1), t_top2));
    if (status && (!ok || !fin)) atomicOr(status, (ok ? 0u : FLAG_PIVOT) | (fin ? 0u : FLAG_NONFINITE));
}

// ---------------------------------------------------------------------------
// settei_ng in two passes.  Everything expensive (the conductivity tek0 of
// each interface and the heating / cooling / exchange rates of each level,
// with their exp, log and pow) is independent across levels: the first
// kernel computes it with one thread per (level, column) into 10 level-major
// planes; the second walks each column once, forming the rows from the
// planes, solving and finishing Te, Ti and qtotal.  Same operations as
// k_settei_ng.
// ---------------------------------------------------------------------------
namespace {
enum { P_TEK0 = 0, P_TH, P_DQ, P_QE, P_ET, P_LENTN, P_LEITI, P_LEI, P_LIN, P_QENI, P_N };
constexpr int kSetteiStaged = 9;   // values per level staged by the row walk

__device__ __forceinline__ double settei_fe(const SetteiFields &F, const SetteiConsts &C, long col)
{
    const double pi = 3.141592653589793, rtd = 180.0 / pi, ev = C.evergs, fpolar = -3.0e+9;
    const double f107te = C.f107 < 235. ? C.f107 : 235.;
    const double arl = fabs(__ldg(F.rlatm + col)), chi = __ldg(F.chi + col), qa = __ldg(F.qteaur + col);
    double a = 0.;
    if (arl >= xd(pi, 4.5)) a = 1.;
    if (arl < xd(pi, 4.5) && arl > xd(pi, 18.)) a = xm(.5, xa(1., cos(xs(xm(arl, 6.), xd(xm(pi, 4.), 3.)))));
    if (arl <= xd(pi, 18.)) a = 0.;
    double fed = xm(xm(-9.0e+7, f107te), a);
    double fen = xd(fed, 2.);
    fed = xa(fed, qa);
    fen = xa(fen, qa);
    double fe = chi >= xm(.5, pi) ? fen : fed;
    const double cd = xm(chi, rtd);
    if (xm(xs(cd, 80.), xs(cd, 100.)) >= 0.) fe = xm(fe, ev);
    else fe = xm(xa(xm(.5, xa(fed, fen)), xm(xm(.5, xs(fed, fen)), cos(xd(xm(pi, xs(cd, 80.)), 20.)))), ev);
    if (arl >= xd(pi, 3.)) fe = xa(fe, xm(fpolar, ev));
    return fe;
}
}  // namespace

__global__ void __launch_bounds__(128) k_settei_levels(SetteiFields F, SetteiConsts C, double *lv, int nk, int ncol,
                                                       long ld)
{
    const long col = (long)blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y;
    if (col >= ncol) return;
    auto at = [&](const double *p, int k) { return __ldg(p + k * ld + col); };
    const long o = (long)j * ld + col;
    const Lev L = load_lev(F, o);
    // interface j (settei_ng.F90:89-139)
    Iface I;
    if (j == 0) {
        const double *b = C.b, *fb = C.fb, t_lbc = __ldg(F.t_lbc + col);
        const Lev L1 = load_lev(F, ld + col);
        const double te_int = dmax(xs(xm(1.5, L.te), xm(.5, L1.te)), t_lbc);
        const double o2n = xm(.5, xa(xa(xa(fb[0], xm(xa(b[0], 1.), L.o2)), xm(b[3], L.o1)), xm(b[6], L.he)));
        const double o1n = xm(.5, xa(xa(xa(fb[0], xm(b[0], L.o2)), xm(xa(b[3], 1.), L.o1)), xm(b[6], L.he)));
        const double hen = xm(.5, xa(xa(xa(fb[0], xm(b[0], L.o2)), xm(b[3], L.o1)), xm(xa(b[6], 1.), L.he)));
        const double n2n = dmax(xs(xs(xs(1., o2n), o1n), hen), 0.);
        I = iface(C, te_int, o2n, o1n, hen, n2n, t_lbc, at(F.xnmbari, 0), at(F.ne, 0), at(F.schti, 0));
    } else {
        const Lev Lm = load_lev(F, o - ld);
        double te_int, tn_int;
        if (j == nk - 1) {
            const Lev Lmm = load_lev(F, o - 2 * ld);
            te_int = xs(xm(1.5, Lm.te), xm(.5, Lmm.te));
            tn_int = xs(xm(1.5, Lm.tn), xm(.5, Lmm.tn));
        } else {
            te_int = xm(.5, xa(L.te, Lm.te));
            tn_int = xm(.5, xa(L.tn, Lm.tn));
        }
        I = iface(C, te_int, xm(.5, xa(L.o2, Lm.o2)), xm(.5, xa(L.o1, Lm.o1)), xm(.5, xa(L.he, Lm.he)),
                  xm(.5, xa(L.n2, Lm.n2)), tn_int, at(F.xnmbari, j), at(F.ne, j), at(F.schti, j));
    }
    // heating, cooling and exchange of level j (settei_ng.F90:157-246)
    const double ne0 = at(F.ne, j);
    double qtot, rne_raw;
    if (j < nk - 1) {
        qtot = sqrt(xm(qsum(F, o), qsum(F, o + ld)));
        rne_raw = xm(ne0, at(F.ne, j + 1));
    } else {
        qtot = 0.;
        rne_raw = xd(xm(xm(ne0, ne0), ne0), at(F.ne, nk - 2));
    }
    const Loss R = level_loss(F, C, o, L, rne_raw, qtot);
    const long slab = (long)nk * ld;
    lv[P_TEK0 * slab + o] = I.tek0;
    lv[P_TH * slab + o] = I.th;
    lv[P_DQ * slab + o] = R.dq;
    lv[P_QE * slab + o] = R.qe_h;
    lv[P_ET * slab + o] = R.et_h;
    lv[P_LENTN * slab + o] = R.len_tn;
    lv[P_LEITI * slab + o] = R.lei_ti;
    lv[P_LEI * slab + o] = R.lei;
    lv[P_LIN * slab + o] = R.lin;
    lv[P_QENI * slab + o] = R.q_eni;
}

// The column walk over the level planes.  Its per-level reads are staged
// one iteration ahead (Stage): the forward sweep's nine values of level k+1
// while level k computes, then the post steps' five values likewise.  The
// two divisions of a level share the divisor w1: one correctly rounded
// reciprocal and Markstein's correction (qdiv), the same bits as IEEE a/b.
__global__ void __launch_bounds__(128) k_settei_rows(SetteiFields F, SetteiConsts C, const double *lv, double *te_out,
                                                     double *ti_out, double *qtotal, int nk, int ncol, long ld,
                                                     double *sys_out, unsigned *status, int pd)
{
    extern __shared__ double smem_tr[];
    const long col = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (col >= ncol) return;
    const int T = blockDim.x;
    double *w2s = smem_tr + threadIdx.x;
    Stage<kSetteiStaged> sg{smem_tr + (long)(nk - 1) * T + threadIdx.x, T};
    const long slab = (long)nk * ld;
    auto at = [&](const double *p, int k) { return __ldg(p + k * ld + col); };
    auto pl = [&](int e, int k) { return __ldg(lv + e * slab + (long)k * ld + col); };
    const double dz = C.dz, fe = settei_fe(F, C, col);
    double sindip;
    {
        const double dm = fabs(__ldg(F.dipmag + col));
        const double sn = sin(dm > C.dipmin ? dm : C.dipmin);
        sindip = dmax(xm(sn, sn), .10);
    }
    const double t_lbc = __ldg(F.t_lbc + col);
    // forward reads of level k into buffer b: 0 q_eni, 1 qtotal, 2 th(k+1),
    // 3 scht, 4 qe, 5 et, 6 dq, 7 len_tn, 8 lei_ti
    auto reads = [&](int k, auto &&fn) {
        const long o = (long)k * ld + col;
        fn(0, lv + P_QENI * slab + o);
        if (k >= 1 && k <= nk - 2) fn(1, qtotal + o);
        if (k <= nk - 2) {
            fn(2, lv + P_TH * slab + o + ld);
            fn(3, F.scht + o);
            fn(4, lv + P_QE * slab + o);
            if (C.et) fn(5, lv + P_ET * slab + o);
            fn(6, lv + P_DQ * slab + o);
            fn(7, lv + P_LENTN * slab + o);
            fn(8, lv + P_LEITI * slab + o);
        }
    };
    auto issue = [&](int k, int b) { reads(k, [&](int v, const double *src) { sg.copy(b, v, src); }); };
    auto prefetch = [&](int k) { reads(k, [](int, const double *src) { pf_l1(src); }); };
    double qe_m1 = 0., w1 = 0., y1 = 0., w3 = 0., rprev = 0.;
    double th_k = pl(P_TH, 0);
    bool ok = true;
    issue(0, 0);
    sg.commit();
    for (int kk = 2; kk < pd + 1 && kk < nk; ++kk) prefetch(kk);
    for (int k = 0; k < nk; ++k) {
        if (pd > 1 && k + 1 + pd < nk) prefetch(k + 1 + pd);
        if (k + 1 < nk) issue(k + 1, (k + 1) & 1);
        sg.commit();
        sg.wait_prev();
        const int b = k & 1;
        const long o = (long)k * ld + col;
        const double q_eni = sg.at(b, 0);
        // qtotal += q_eni at the interfaces (settei_ng.F90:248-254)
        if (k == 1) qtotal[col] = xa(qtotal[col], xs(xm(1.5, qe_m1), xm(0.5, q_eni)));
        if (k >= 1 && k <= nk - 2) qtotal[o] = xa(sg.at(b, 1), xm(.5, xa(qe_m1, q_eni)));
        if (k == nk - 2) {
            const double qe_prev = k >= 1 ? qe_m1 : 0.;
            qtotal[(long)(nk - 1) * ld + col] = xa(qtotal[(long)(nk - 1) * ld + col], xs(xm(1.5, q_eni), xm(0.5, qe_prev)));
        }
        if (k <= nk - 2) {
            const double th_1 = sg.at(b, 2);
            const double pb = xm(xd(xd(2., 7.), xm(sg.at(b, 3), xm(dz, dz))), sindip);
            double r = xm(pb, th_1);
            double p = xm(pb, th_k);
            double q = -xa(p, r);
            double rhs = 0.;
            if (k == 0) {
                q = xs(q, p);
                rhs = xs(rhs, xm(xm(2., p), pow(t_lbc, 3.5)));
                p = 0.;
            }
            if (k == nk - 2) {
                q = xa(q, r);
                rhs = xa(rhs, xd(xm(xm(xm(xm(r, dz), 3.5), at(F.schti, nk - 1)), fe), pl(P_TEK0, nk - 1)));
                r = 0.;
            }
            rhs = xs(rhs, sg.at(b, 4));
            if (C.et) rhs = xs(rhs, sg.at(b, 5));
            q = xs(q, sg.at(b, 6));
            rhs = xs(xs(rhs, sg.at(b, 7)), sg.at(b, 8));
            if (sys_out) {
                sys_out[o] = p;
                sys_out[slab + o] = q;
                sys_out[2 * slab + o] = r;
                sys_out[3 * slab + o] = rhs;
            }
            if (k == 0) {
                w1 = q;
                y1 = __drcp_rn(w1);
                w3 = qdiv(rhs, w1, y1);
            } else {
                const double w2 = qdiv(rprev, w1, y1);
                w2s[(long)(k - 1) * T] = w2;
                w1 = xs(q, xm(p, w2));
                y1 = __drcp_rn(w1);
                w3 = qdiv(xs(rhs, xm(p, w3)), w1, y1);
            }
            ok = ok && fabs(w1) <= DBL_MAX && w1 != 0.0;
            te_out[o] = w3;
            rprev = r;
            th_k = th_1;
        }
        qe_m1 = q_eni;
    }
    // back substitution and post steps over the levels K-1, K-2, ..., 0, K
    // (call i treats level lev(i)); te_out holds w3 until a level is final
    const int K = nk - 1;
    auto lev = [&](int i) { return i < K ? K - 1 - i : K; };
    auto reads_b = [&](int i, auto &&fn) {
        const long o = (long)lev(i) * ld + col;
        fn(0, F.tn + o);
        fn(1, lv + P_LEI * slab + o);
        fn(2, lv + P_LIN * slab + o);
        fn(3, F.qji_ti + o);
        fn(4, F.xnmbar + o);
    };
    auto issue_b = [&](int i, int b) { reads_b(i, [&](int v, const double *src) { sg.copy(b, v, src); }); };
    // with the parked forward result of the level after
    auto prefetch_b = [&](int i) {
        reads_b(i, [](int, const double *src) { pf_l1(src); });
        if (lev(i) >= 1 && i < K) pf_l1(te_out + (long)(lev(i) - 1) * ld + col);
    };
    double xn = w3;
    double tk = pow(xn, xd(2., 7.));
    double t_top1 = tk, t_top2 = 0.;
    bool fin = fabs(xn) <= DBL_MAX;
    double park = K >= 2 ? te_out[(long)(K - 2) * ld + col] : 0.;
    issue_b(0, 0);
    sg.commit();
    for (int ii = 2; ii < pd + 1 && ii <= K; ++ii) prefetch_b(ii);
    for (int i = 0; i <= K; ++i) {
        if (pd > 1 && i + 1 + pd <= K) prefetch_b(i + 1 + pd);
        if (i + 1 <= K) issue_b(i + 1, (i + 1) & 1);
        sg.commit();
        sg.wait_prev();
        const int b = i & 1, k = lev(i);
        double t;
        if (i == 0) {
            t = tk;
        } else if (i < K) {
            const double wk = park;
            if (k >= 1) park = te_out[(long)(k - 1) * ld + col];
            xn = xs(wk, xm(w2s[(long)k * T], xn));
            fin = fin && fabs(xn) <= DBL_MAX;
            tk = pow(xn, xd(2., 7.));
            if (k == K - 2) t_top2 = tk;
            t = tk;
        } else {
            t = xd(xm(t_top1, t_top1), t_top2);
        }
        const long o = (long)k * ld + col;
        const double tn = sg.at(b, 0);
        const double te = dmax(t, tn);
        const double lei = sg.at(b, 1), lin = sg.at(b, 2);
        te_out[o] = te;
        const double num = xa(xa(xd(xm(sg.at(b, 3), sg.at(b, 4)), C.avo), xm(lei, te)), xm(lin, tn));
        ti_out[o] = dmax(xd(num, xa(lei, lin)), tn);
    }
    if (status && (!ok || !fin)) atomicOr(status, (ok ? 0u : FLAG_PIVOT) | (fin ? 0u : FLAG_NONFINITE));
}

// ---------------------------------------------------------------------------
// settei_ng in three passes (the default), so that the column walk is the
// recurrence alone instead of forming its rows and raising every solved
// level to the 2/7 power level by level.  After k_settei_levels:
//   k_settei_coefs: one thread per (level, column) forms row k (p, q, r and
//     rhs, as the walk forms them) into four planes and adds q_eni to qtotal
//     at the interfaces;
//   the Thomas walk of the assembly routines (launch_thomas_post) solves the
//     rows 0..nk-2 for x = Te^3.5 into a scratch plane;
//   k_settei_post: one thread per (level, column) turns x into Te, the top
//     level from its two neighbours, and forms Ti.
// The same operations on the same operands as k_settei_rows: the same bits.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(128) k_settei_coefs(SetteiFields F, SetteiConsts C, const double *lv,
                                                      double *rows, double *qtotal, int nk, int ncol, long ld,
                                                      double *sys_out)
{
    const long col = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (col >= ncol) return;
    const int k = blockIdx.y;
    const long slab = (long)nk * ld, o = (long)k * ld + col;
    auto pl = [&](int e, int kk) { return __ldg(lv + e * slab + (long)kk * ld + col); };
    {
        // every line the row reads, requested into L1 at once
        const int km = k > 0 ? k - 1 : 0, kp = k + 1 < nk ? k + 1 : nk - 1;
        pf_l1(lv + P_QENI * slab + (long)km * ld + col);
        pf_l1(lv + P_QENI * slab + o);
        pf_l1(lv + P_QENI * slab + (long)kp * ld + col);
        pf_l1(lv + P_TH * slab + (long)kp * ld + col);
#pragma unroll
        for (int e = P_TH; e <= P_LEITI; ++e) pf_l1(lv + e * slab + o);
        pf_l1(qtotal + o);
        pf_l1(F.scht + o);
    }
    // qtotal += q_eni at the interfaces (settei_ng.F90:248-254); level k
    // reads and writes only its own qtotal
    const double qe_k = pl(P_QENI, k);
    if (k == 0)
        qtotal[o] = xa(qtotal[o], xs(xm(1.5, qe_k), xm(0.5, pl(P_QENI, 1))));
    else if (k <= nk - 2)
        qtotal[o] = xa(qtotal[o], xm(.5, xa(pl(P_QENI, k - 1), qe_k)));
    else
        qtotal[o] = xa(qtotal[o], xs(xm(1.5, pl(P_QENI, nk - 2)), xm(0.5, nk >= 3 ? pl(P_QENI, nk - 3) : 0.)));
    if (k > nk - 2) return;
    const double dz = C.dz;
    double sindip;
    {
        const double dm = fabs(__ldg(F.dipmag + col));
        const double sn = sin(dm > C.dipmin ? dm : C.dipmin);
        sindip = dmax(xm(sn, sn), .10);
    }
    const double pb = xm(xd(xd(2., 7.), xm(__ldg(F.scht + o), xm(dz, dz))), sindip);
    double r = xm(pb, pl(P_TH, k + 1));
    double p = xm(pb, pl(P_TH, k));
    double q = -xa(p, r);
    double rhs = 0.;
    if (k == 0) {
        q = xs(q, p);
        rhs = xs(rhs, xm(xm(2., p), pow(__ldg(F.t_lbc + col), 3.5)));
        p = 0.;
    }
    if (k == nk - 2) {
        q = xa(q, r);
        rhs = xa(rhs, xd(xm(xm(xm(xm(r, dz), 3.5), __ldg(F.schti + (long)(nk - 1) * ld + col)), settei_fe(F, C, col)),
                         pl(P_TEK0, nk - 1)));
        r = 0.;
    }
    rhs = xs(rhs, pl(P_QE, k));
    if (C.et) rhs = xs(rhs, pl(P_ET, k));
    q = xs(q, pl(P_DQ, k));
    rhs = xs(xs(rhs, pl(P_LENTN, k)), pl(P_LEITI, k));
    rows[o] = p;
    rows[slab + o] = q;
    rows[2 * slab + o] = r;
    rows[3 * slab + o] = rhs;
    if (sys_out) {
        sys_out[o] = p;
        sys_out[slab + o] = q;
        sys_out[2 * slab + o] = r;
        sys_out[3 * slab + o] = rhs;
    }
}

__global__ void __launch_bounds__(128) k_settei_post(SetteiFields F, SetteiConsts C, const double *lv, const double *x,
                                                     double *te_out, double *ti_out, int nk, int ncol, long ld)
{
    const long col = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (col >= ncol) return;
    const int k = blockIdx.y, K = nk - 1;
    const long slab = (long)nk * ld, o = (long)k * ld + col;
    const double e27 = xd(2., 7.);
    double t;
    if (k < K) {
        t = pow(x[o], e27);
    } else {
        // te(nk) = te(nk-1)**2/te(nk-2) from the unfloored values
        const double t1 = pow(x[(long)(K - 1) * ld + col], e27), t2 = pow(x[(long)(K - 2) * ld + col], e27);
        t = xd(xm(t1, t1), t2);
    }
    const double tn = __ldg(F.tn + o);
    const double te = dmax(t, tn);
    const double lei = __ldg(lv + P_LEI * slab + o), lin = __ldg(lv + P_LIN * slab + o);
    te_out[o] = te;
    const double num = xa(xa(xd(xm(__ldg(F.qji_ti + o), __ldg(F.xnmbar + o)), C.avo), xm(lei, te)), xm(lin, tn));
    ti_out[o] = dmax(xd(num, xa(lei, lin)), tn);
}

// the level planes, then (three-pass form) the four row planes and x
size_t settei_scratch_doubles(int nk, long ld) { return (size_t)(P_N + 5) * nk * ld; }

cudaError_t launch_settei_ng(const SetteiFields &F, const SetteiConsts &C, double *te_out, double *ti_out,
                             double *qtotal, int nk, int ncol, long ld, double *sys_out, unsigned *status,
                             cudaStream_t st, double *scratch)
{
    if (ncol <= 0) return cudaSuccess;
    if (nk < 3) return cudaErrorInvalidValue;
    const int optin = smem_optin();
    once_per_device([optin] {
        cudaFuncSetAttribute(k_settei_ng, cudaFuncAttributeMaxDynamicSharedMemorySize, optin);
        cudaFuncSetAttribute(k_settei_rows, cudaFuncAttributeMaxDynamicSharedMemorySize, optin);
    });
    // w2 (nk-1) and loss_in (nk) per column in shared memory
    int T = 128;
    const size_t per = (size_t)(2 * nk - 1) * sizeof(double);
    while (T > 32 && (size_t)T * per > (size_t)optin) T /= 2;
    if ((size_t)T * per > (size_t)optin) return cudaErrorInvalidValue;
    // three-pass (on 41472 columns 271 against 280 us for the two-pass walk)
    if (scratch && assembly_mode() == 2) {
        const long slab = (long)nk * ld;
        double *rows = scratch + P_N * slab, *x = rows + 4 * slab;
        const dim3 grid((ncol + 127) / 128, nk);
        k_settei_levels<<<grid, 128, 0, st>>>(F, C, scratch, nk, ncol, ld);
        k_settei_coefs<<<grid, 128, 0, st>>>(F, C, scratch, rows, qtotal, nk, ncol, ld, sys_out);
        cudaError_t e = launch_thomas_post(rows, rows + slab, rows + 2 * slab, rows + 3 * slab, x, nk, nk - 1, 0, ncol,
                                           ld, status, nullptr, st);
        if (e != cudaSuccess) return e;
        k_settei_post<<<grid, 128, 0, st>>>(F, C, scratch, x, te_out, ti_out, nk, ncol, ld);
        return cudaGetLastError();
    }
    if (scratch && assembly_mode() >= 1) {
        int T2 = 128;
        const size_t per2 = (size_t)(nk - 1) * sizeof(double) + Stage<kSetteiStaged>::bytes_per_thread;
        while (T2 > 32 && (size_t)T2 * per2 > (size_t)optin) T2 /= 2;
        k_settei_levels<<<dim3((ncol + 127) / 128, nk), 128, 0, st>>>(F, C, scratch, nk, ncol, ld);
        k_settei_rows<<<(ncol + T2 - 1) / T2, T2, (size_t)T2 * per2, st>>>(F, C, scratch, te_out, ti_out, qtotal, nk,
                                                                           ncol, ld, sys_out, status,
                                                                           walk_prefetch(ncol));
        return cudaGetLastError();
    }
    k_settei_ng<<<(ncol + T - 1) / T, T, (size_t)T * per, st>>>(F, C, te_out, ti_out, qtotal, nk, ncol, ld, sys_out,
                                                                status);
    return cudaGetLastError();
}
}  // namespace tg
