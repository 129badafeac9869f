// Column assembly fused with the solve: dt_ng (neutral temperature).
//
// One thread per column walks the levels once.  At row k it forms the
// tridiagonal row p(k), q(k), r(k), rhs(k) of src/dt_ng.F90:57-163 from the
// physical fields of levels k-1, k, k+1 (kept in a sliding register window),
// applies the lower-boundary fold, and feeds the row straight into the Thomas
// forward sweep (src/trsolv_ng.F90:14-22); the coefficients never touch
// memory.  The back sweep and the top-level extrapolation tn(nk) =
// tn(nk-1)**2/tn(nk-2) (dt_ng.F90:167) follow.  Every operation is the
// reference's, in its order, with non-contracting FP64 intrinsics, so the
// result is bit-identical to the CPU restatement.
//
// Layout: level-major, field(k, col) at k*ld + col; 2-D fields at col; the
// level constants expz and dift at k.
#include <cfloat>

#include "tg_internal.h"

namespace tg {

namespace {
__device__ __forceinline__ double xm(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double xa(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double xs(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double xd(double a, double b) { return __ddiv_rn(a, b); }
__device__ __forceinline__ bool fin_nz(double w) { return fabs(w) <= DBL_MAX && w != 0.0; }

// g(k) and f(k) of dt_ng.F90:126-148 for one level.
struct GF {
    double g, f;
};
__device__ __forceinline__ GF dt_gf(const DtConsts &C, double h, double cp, double kt, double tni, double expz,
                                    double dift)
{
    double rho = xd(xm(C.p0, C.expzmid_inv), xm(h, C.grav));
    rho = xm(rho, expz);
    double gpart = xm(xm(xm(h, h), rho), cp);
    gpart = xm(gpart, dift);
    GF r;
    r.g = xd(xm(C.grav, xa(kt, gpart)), xm(xm(C.p0, h), xm(C.dz, C.dz)));
    const double ff = xd(xm(xm(xm(C.grav, C.grav), xm(h, h)), rho), xm(xm(xm(tni, C.p0), 2.0), C.dz));
    r.f = xm(ff, dift);
    return r;
}
}  // namespace

__global__ void __launch_bounds__(128) k_dt_ng(DtFields F, DtConsts C, double *tn_upd, int nk, int ncol, long ld,
                                               double *sys_out, unsigned *status)
{
    extern __shared__ double smem_dt[];
    const long col = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (col >= ncol) return;
    double *w2s = smem_dt + threadIdx.x;
    const int T = blockDim.x;
    auto at = [&](const double *p, int k) { return __ldg(p + k * ld + col); };
    const double dz = C.dz;
    const double tlbc_prev = __ldg(F.tlbc + col), tlbc_cur = __ldg(F.t_lbc + col);
    const double ulbc = __ldg(F.ulbc + col), vlbc = __ldg(F.vlbc + col);
    const int K = nk - 1;   // rows 0..K-1 are solved

    // window: level k-1, k, k+1 values
    double tn_m = 0.0, tn_0 = at(F.tn, 0), tn_p = at(F.tn, 1);
    double un_m = 0.0, un_0 = at(F.un, 0), un_p = at(F.un, 1);
    double vn_m = 0.0, vn_0 = at(F.vn, 0), vn_p = at(F.vn, 1);
    double w_0 = at(F.w, 0), w_p = at(F.w, 1);
    double cp_0 = at(F.cp, 0), cp_p = at(F.cp, 1);
    double km_0 = at(F.km, 0), km_p = at(F.km, 1);
    double qt_0 = at(F.qtotal, 0), qt_p = at(F.qtotal, 1);
    // vertical advection terms vad0(k) before averaging (dt_ng.F90:57-61)
    double v0_0 = xm(xm(xs(tn_0, tlbc_cur), w_0), 2.0);
    // g, f of level 0 (tni(1) = tlbc, the previous lower boundary)
    GF gf0 = dt_gf(C, at(F.schti, 0), cp_0, at(F.kt, 0), tlbc_prev, __ldg(F.expz), __ldg(F.dift));
    double dudz_prev = 0.0, dvdz_prev = 0.0;

    bool ok = true;
    double w1 = 0.0, w3 = 0.0, rprev = 0.0;
    for (int k = 0; k < K; ++k) {
        const double expz = __ldg(F.expz + k), expz_p = __ldg(F.expz + k + 1);
        // level k+1 quantities
        const double v0_p = (k + 1 <= nk - 2) ? xm(xs(tn_p, tn_0), w_p) : 0.0;
        const double tni_p = (k + 1 <= nk - 2) ? xm(0.5, xa(tn_0, tn_p)) : tn_0;
        const GF gfp = dt_gf(C, at(F.schti, k + 1), cp_p, at(F.kt, k + 1), tni_p, expz_p, __ldg(F.dift + k + 1));
        // tridiagonal row (dt_ng.F90:141-148)
        double p = xs(gf0.g, gf0.f);
        double q, r;
        if (k < K - 1) {
            q = -xa(xa(xs(gfp.g, gfp.f), gf0.g), gf0.f);
            r = xa(gfp.g, gfp.f);
        } else {
            q = xs(-gf0.g, gf0.f);
            r = 0.0;
        }
        // vertical advection, averaged and scaled (:62-66)
        const double vad = xd(xm(xa(v0_0, v0_p), 0.5), dz);
        const double cpi = xm(0.5, xa(cp_0, cp_p));
        const double kmi = xm(0.5, xa(km_0, km_p));
        const double wi = xm(0.5, xa(w_0, w_p));
        // wind shear (:86-95)
        double dudz, dvdz;
        if (k == 0) {
            dudz = xd(xs(xa(un_0, xm(1.0 / 3.0, un_p)), xm(4.0 / 3.0, ulbc)), dz);
            dvdz = xd(xs(xa(vn_0, xm(1.0 / 3.0, vn_p)), xm(4.0 / 3.0, vlbc)), dz);
        } else if (k <= nk - 3) {
            dudz = xd(xs(un_p, un_m), xm(2.0, dz));
            dvdz = xd(xs(vn_p, vn_m), xm(2.0, dz));
        } else {
            dudz = xd(dudz_prev, 3.0);
            dvdz = xd(dvdz_prev, 3.0);
        }
        const double qsolar = xm(0.5, xa(qt_0, qt_p));
        // heating and right-hand side (:81-84, :97-118, :150-157)
        const double advec = xa(at(F.horadv, k), vad);
        double cptn = xm(cpi, xs(advec, xm(C.dtx2inv, at(F.tnsmooth, k))));
        cptn = xm(cptn, expz);
        const double mbar = at(F.mbar, k);
        const double xo = xm(xm(at(F.xnmbar, k), at(F.o1, k)), C.rmassinv_o1);
        const double qrecomb = xd(xm(xm(xm(C.tsurplus, at(F.rkm12, k)), xm(xo, xo)), C.avo), mbar);
        double qm = xm(xd(xm(C.grav, kmi), xm(C.p0, at(F.scht, k))), xa(xm(dudz, dudz), xm(dvdz, dvdz)));
        qm = xd(qm, expz);
        const double th = xa(xa(xa(xa(qsolar, at(F.hdt, k)), qrecomb), at(F.qji_tn, k)), qm);
        cptn = xs(cptn, xm(th, expz));
        double rhs = xa(cptn, at(F.cool_exp, k));
        const double qpart = xa(xm(cpi, xa(C.dtx2inv, at(F.cool_imp, k))), xd(xm(wi, C.gask), mbar));
        q = xs(q, xm(qpart, expz));
        if (k == 0) {   // lower boundary fold (:159-163)
            q = xs(q, p);
            rhs = xs(rhs, xm(xm(2.0, p), tlbc_cur));
            p = 0.0;
        }
        if (sys_out) {
            const long n = (long)nk * ld;
            sys_out[k * ld + col] = p;
            sys_out[n + k * ld + col] = q;
            sys_out[2 * n + k * ld + col] = r;
            sys_out[3 * n + k * ld + col] = rhs;
        }
        // Thomas forward step (trsolv_ng.F90:14-22), a=p, b=q, c(k-1)=r(k-1), f=rhs
        if (k == 0) {
            w1 = q;
            w3 = xd(rhs, w1);
        } else {
            const double w2 = xd(rprev, w1);
            w2s[(k - 1) * T] = w2;
            w1 = xs(q, xm(p, w2));
            w3 = xd(xs(rhs, xm(p, w3)), w1);
        }
        ok = ok && fin_nz(w1);
        tn_upd[k * ld + col] = w3;
        rprev = r;
        // slide the window
        dudz_prev = dudz;
        dvdz_prev = dvdz;
        gf0 = gfp;
        v0_0 = v0_p;
        tn_m = tn_0; tn_0 = tn_p;
        un_m = un_0; un_0 = un_p;
        vn_m = vn_0; vn_0 = vn_p;
        w_0 = w_p; cp_0 = cp_p; km_0 = km_p; qt_0 = qt_p;
        if (k + 2 < nk) {
            tn_p = at(F.tn, k + 2);
            un_p = at(F.un, k + 2);
            vn_p = at(F.vn, k + 2);
            w_p = at(F.w, k + 2);
            cp_p = at(F.cp, k + 2);
            km_p = at(F.km, k + 2);
            qt_p = at(F.qtotal, k + 2);
        }
    }
    (void)tn_m;
    // back sweep (trsolv_ng.F90:23-26), then tn(nk) = tn(nk-1)**2/tn(nk-2)
    double xn = w3, xprev = w3;
    bool fin = fabs(xn) <= DBL_MAX;
    for (int k = K - 2; k >= 0; --k) {
        xprev = xn;
        xn = xs(tn_upd[k * ld + col], xm(w2s[k * T], xn));
        fin = fin && fabs(xn) <= DBL_MAX;
        tn_upd[k * ld + col] = xn;
        if (k == K - 2) {
            // xprev = x(K-1), xn = x(K-2): the two top solved rows
            tn_upd[(long)K * ld + col] = xd(xm(xprev, xprev), xn);
        }
    }
    if (status && (!ok || !fin)) atomicOr(status, (ok ? 0u : FLAG_PIVOT) | (fin ? 0u : FLAG_NONFINITE));
}

cudaError_t launch_dt_ng(const DtFields &F, const DtConsts &C, double *tn_upd, int nk, int ncol, long ld,
                         double *sys_out, unsigned *status, cudaStream_t st)
{
    if (ncol <= 0) return cudaSuccess;
    const int T = 128;
    const size_t smem = (size_t)T * (nk - 2 > 0 ? nk - 2 : 1) * sizeof(double);
    static bool attr = false;
    if (!attr) {
        int dev = 0, optin = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
        cudaFuncSetAttribute(k_dt_ng, cudaFuncAttributeMaxDynamicSharedMemorySize, optin - 1024);
        attr = true;
    }
    k_dt_ng<<<(ncol + T - 1) / T, T, smem, st>>>(F, C, tn_upd, nk, ncol, ld, sys_out, status);
    return cudaGetLastError();
}

}  // namespace tg
