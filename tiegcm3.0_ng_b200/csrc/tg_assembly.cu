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
#include <atomic>
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

// Per-level reads are staged one iteration ahead (Stage): the 13 fields of
// row k and the level-(k+2) window while row k-1 computes.  The two divisions
// of a row share the divisor w1 (qdiv: one correctly rounded reciprocal, the
// same bits as IEEE a/b).
constexpr int kDtStaged = 20;
__global__ void __launch_bounds__(128) k_dt_ng(DtFields F, DtConsts C, double *tn_upd, int nk, int ncol, long ld,
                                               double *sys_out, unsigned *status, PostStep post, int has_post, int pd)
{
    extern __shared__ double smem_dt[];
    const long col = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (col >= ncol) return;
    double *w2s = smem_dt + threadIdx.x;
    const int T = blockDim.x;
    Stage<kDtStaged> sg{smem_dt + (long)(nk - 2 > 0 ? nk - 2 : 1) * T + threadIdx.x, T};
    auto at = [&](const double *p, int k) { return __ldg(p + k * ld + col); };
    const double dz = C.dz;
    const double tlbc_prev = __ldg(F.tlbc + col), tlbc_cur = __ldg(F.t_lbc + col);
    const double ulbc = __ldg(F.ulbc + col), vlbc = __ldg(F.vlbc + col);
    const int K = nk - 1;   // rows 0..K-1 are solved

    // window: level k-1, k, k+1 values
    double tn_0 = at(F.tn, 0), tn_p = at(F.tn, 1);
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

    // reads of row k into buffer b: 0 schti(k+1), 1 kt(k+1), 2 horadv, 3
    // tnsmooth, 4 mbar, 5 xnmbar, 6 o1, 7 rkm12, 8 scht, 9 hdt, 10 qji_tn, 11
    // cool_exp, 12 cool_imp; 13..19 tn, un, vn, w, cp, km, qtotal of level k+2
    auto reads = [&](int k, auto &&fn) {
        const long o = (long)k * ld + col;
        fn(0, F.schti + o + ld);
        fn(1, F.kt + o + ld);
        fn(2, F.horadv + o);
        fn(3, F.tnsmooth + o);
        fn(4, F.mbar + o);
        fn(5, F.xnmbar + o);
        fn(6, F.o1 + o);
        fn(7, F.rkm12 + o);
        fn(8, F.scht + o);
        fn(9, F.hdt + o);
        fn(10, F.qji_tn + o);
        fn(11, F.cool_exp + o);
        fn(12, F.cool_imp + o);
        if (k + 2 < nk) {
            const long o2 = o + 2 * ld;
            fn(13, F.tn + o2);
            fn(14, F.un + o2);
            fn(15, F.vn + o2);
            fn(16, F.w + o2);
            fn(17, F.cp + o2);
            fn(18, F.km + o2);
            fn(19, F.qtotal + o2);
        }
    };
    auto issue = [&](int k, int b) { reads(k, [&](int v, const double *src) { sg.copy(b, v, src); }); };
    auto prefetch = [&](int k) { reads(k, [](int, const double *src) { pf_l1(src); }); };
    bool ok = true;
    double w1 = 0.0, y1 = 0.0, w3 = 0.0, rprev = 0.0;
    issue(0, 0);
    sg.commit();
    for (int kk = 2; kk < pd + 1 && kk < K; ++kk) prefetch(kk);
    for (int k = 0; k < K; ++k) {
        if (pd > 1 && k + 1 + pd < K) prefetch(k + 1 + pd);
        if (k + 1 < K) issue(k + 1, (k + 1) & 1);
        sg.commit();
        sg.wait_prev();
        const int b = k & 1;
        const double expz = __ldg(F.expz + k), expz_p = __ldg(F.expz + k + 1);
        // level k+1 quantities
        const double v0_p = (k + 1 <= nk - 2) ? xm(xs(tn_p, tn_0), w_p) : 0.0;
        const double tni_p = (k + 1 <= nk - 2) ? xm(0.5, xa(tn_0, tn_p)) : tn_0;
        const GF gfp = dt_gf(C, sg.at(b, 0), cp_p, sg.at(b, 1), tni_p, expz_p, __ldg(F.dift + k + 1));
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
        const double advec = xa(sg.at(b, 2), vad);
        double cptn = xm(cpi, xs(advec, xm(C.dtx2inv, sg.at(b, 3))));
        cptn = xm(cptn, expz);
        const double mbar = sg.at(b, 4);
        const double xo = xm(xm(sg.at(b, 5), sg.at(b, 6)), C.rmassinv_o1);
        const double qrecomb = xd(xm(xm(xm(C.tsurplus, sg.at(b, 7)), xm(xo, xo)), C.avo), mbar);
        double qm = xm(xd(xm(C.grav, kmi), xm(C.p0, sg.at(b, 8))), xa(xm(dudz, dudz), xm(dvdz, dvdz)));
        qm = xd(qm, expz);
        const double th = xa(xa(xa(xa(qsolar, sg.at(b, 9)), qrecomb), sg.at(b, 10)), qm);
        cptn = xs(cptn, xm(th, expz));
        double rhs = xa(cptn, sg.at(b, 11));
        const double qpart = xa(xm(cpi, xa(C.dtx2inv, sg.at(b, 12))), xd(xm(wi, C.gask), mbar));
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
            y1 = __drcp_rn(w1);
            w3 = qdiv(rhs, w1, y1);
        } else {
            const double w2 = qdiv(rprev, w1, y1);
            w2s[(k - 1) * T] = w2;
            w1 = xs(q, xm(p, w2));
            y1 = __drcp_rn(w1);
            w3 = qdiv(xs(rhs, xm(p, w3)), w1, y1);
        }
        ok = ok && fin_nz(w1);
        tn_upd[k * ld + col] = w3;
        rprev = r;
        // slide the window
        dudz_prev = dudz;
        dvdz_prev = dvdz;
        gf0 = gfp;
        v0_0 = v0_p;
        tn_0 = tn_p;
        un_m = un_0; un_0 = un_p;
        vn_m = vn_0; vn_0 = vn_p;
        w_0 = w_p; cp_0 = cp_p; km_0 = km_p; qt_0 = qt_p;
        if (k + 2 < nk) {
            tn_p = sg.at(b, 13);
            un_p = sg.at(b, 14);
            vn_p = sg.at(b, 15);
            w_p = sg.at(b, 16);
            cp_p = sg.at(b, 17);
            km_p = sg.at(b, 18);
            qt_p = sg.at(b, 19);
        }
    }
    // back sweep (trsolv_ng.F90:23-26), then tn(nk) = tn(nk-1)**2/tn(nk-2);
    // with has_post every row is stored through the post-solve steps
    // (:201-213), the top row computed from the unfiltered values first
    const bool bcol = has_post && post.bnd_mask && post.bnd_mask[col];
    double xn = w3, xprev = w3;
    bool fin = fabs(xn) <= DBL_MAX;
    double park = K >= 2 ? tn_upd[(K - 2) * ld + col] : 0.0;
    for (int kk = K - 3; kk > K - 2 - pd && kk >= 0; --kk) post_prefetch(post, has_post, bcol, tn_upd, (long)kk * ld + col);
    for (int k = K - 2; k >= 0; --k) {
        if (k - pd >= 0) post_prefetch(post, has_post, bcol, tn_upd, (long)(k - pd) * ld + col);
        xprev = xn;
        const double wk = park;
        if (k >= 1) park = tn_upd[(k - 1) * ld + col];
        xn = xs(wk, xm(w2s[k * T], xn));
        fin = fin && fabs(xn) <= DBL_MAX;
        post_store(post, has_post, bcol, tn_upd, k * ld + col, xn);
        if (k == K - 2) {
            // xprev = x(K-1), xn = x(K-2): the two top solved rows
            post_store(post, has_post, bcol, tn_upd, (long)K * ld + col, xd(xm(xprev, xprev), xn));
            if (has_post) post_store(post, true, bcol, tn_upd, (long)(K - 1) * ld + col, xprev);
        }
    }
    if (status && (!ok || !fin)) atomicOr(status, (ok ? 0u : FLAG_PIVOT) | (fin ? 0u : FLAG_NONFINITE));
}

// Three-pass form of dt_ng: row k (0..nk-2) of every column, one thread per
// (row, column), from the fields of levels k-1..k+1 read directly: the same
// operations as k_dt_ng's walk, which keeps those levels in a sliding window.
namespace {
// g, f of level j: tni(0) is the previous lower boundary, tni(j) the
// interface mean of tn(j-1), tn(j) up to nk-2 and tn(j-1) above
__device__ __forceinline__ GF dt_gf_at(const DtFields &F, const DtConsts &C, int j, int nk, long ld, long col)
{
    auto at = [&](const double *p, int k) { return __ldg(p + k * ld + col); };
    double tni;
    if (j == 0) tni = __ldg(F.tlbc + col);
    else if (j <= nk - 2) tni = xm(0.5, xa(at(F.tn, j - 1), at(F.tn, j)));
    else tni = at(F.tn, j - 1);
    return dt_gf(C, at(F.schti, j), at(F.cp, j), at(F.kt, j), tni, __ldg(F.expz + j), __ldg(F.dift + j));
}
// vertical advection term of level j before averaging (dt_ng.F90:57-61)
__device__ __forceinline__ double dt_v0(const DtFields &F, int j, int nk, long ld, long col)
{
    auto at = [&](const double *p, int k) { return __ldg(p + k * ld + col); };
    if (j == 0) return xm(xm(xs(at(F.tn, 0), __ldg(F.t_lbc + col)), at(F.w, 0)), 2.0);
    if (j <= nk - 2) return xm(xs(at(F.tn, j), at(F.tn, j - 1)), at(F.w, j));
    return 0.0;
}
// wind shear of row k (dt_ng.F90:86-95); the top rows divide the row below by 3
__device__ __forceinline__ void dt_shear_at(const DtFields &F, const DtConsts &C, int k, int nk, long ld, long col,
                                            double &dudz, double &dvdz)
{
    auto at = [&](const double *p, int kk) { return __ldg(p + kk * ld + col); };
    const double dz = C.dz;
    const int kc = k <= nk - 3 ? k : nk - 3;
    if (kc <= 0) {
        dudz = xd(xs(xa(at(F.un, 0), xm(1.0 / 3.0, at(F.un, 1))), xm(4.0 / 3.0, __ldg(F.ulbc + col))), dz);
        dvdz = xd(xs(xa(at(F.vn, 0), xm(1.0 / 3.0, at(F.vn, 1))), xm(4.0 / 3.0, __ldg(F.vlbc + col))), dz);
    } else {
        dudz = xd(xs(at(F.un, kc + 1), at(F.un, kc - 1)), xm(2.0, dz));
        dvdz = xd(xs(at(F.vn, kc + 1), at(F.vn, kc - 1)), xm(2.0, dz));
    }
    for (int kk = kc + 1; kk <= k; ++kk) {
        dudz = xd(dudz, 3.0);
        dvdz = xd(dvdz, 3.0);
    }
}
}  // namespace

__global__ void __launch_bounds__(128) k_dt_coefs(DtFields F, DtConsts C, double *pqrf, int nk, int ncol, long ld,
                                                  double *sys_out)
{
    const long col = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (col >= ncol) return;
    const int k = blockIdx.y, K = nk - 1;
    auto at = [&](const double *p, int kk) { return __ldg(p + kk * ld + col); };
    {
        // every line the row reads, requested into L1 at once: the reads
        // below sit between divisions and would otherwise wait one at a time
        const int km = k > 0 ? k - 1 : 0;
        const long o = (long)k * ld + col;
        for (int j = km; j <= k + 1; ++j) {
            const long oj = (long)j * ld + col;
            pf_l1(F.tn + oj);
            pf_l1(F.un + oj);
            pf_l1(F.vn + oj);
        }
        const double *pair[] = {F.schti, F.cp, F.kt, F.w, F.km, F.qtotal};
#pragma unroll
        for (int i = 0; i < 6; ++i) {
            pf_l1(pair[i] + o);
            pf_l1(pair[i] + o + ld);
        }
        const double *one[] = {F.horadv, F.tnsmooth, F.mbar, F.xnmbar, F.o1, F.rkm12, F.scht, F.hdt, F.qji_tn,
                               F.cool_exp, F.cool_imp};
#pragma unroll
        for (int i = 0; i < 11; ++i) pf_l1(one[i] + o);
    }
    const double dz = C.dz;
    const double expz = __ldg(F.expz + k);
    const GF gf0 = dt_gf_at(F, C, k, nk, ld, col), gfp = dt_gf_at(F, C, k + 1, nk, ld, col);
    double p = xs(gf0.g, gf0.f);
    double q, r;
    if (k < K - 1) {
        q = -xa(xa(xs(gfp.g, gfp.f), gf0.g), gf0.f);
        r = xa(gfp.g, gfp.f);
    } else {
        q = xs(-gf0.g, gf0.f);
        r = 0.0;
    }
    const double vad = xd(xm(xa(dt_v0(F, k, nk, ld, col), dt_v0(F, k + 1, nk, ld, col)), 0.5), dz);
    const double cp_0 = at(F.cp, k), cp_p = at(F.cp, k + 1);
    const double cpi = xm(0.5, xa(cp_0, cp_p));
    const double kmi = xm(0.5, xa(at(F.km, k), at(F.km, k + 1)));
    const double wi = xm(0.5, xa(at(F.w, k), at(F.w, k + 1)));
    double dudz, dvdz;
    dt_shear_at(F, C, k, nk, ld, col, dudz, dvdz);
    const double qsolar = xm(0.5, xa(at(F.qtotal, k), at(F.qtotal, k + 1)));
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
        rhs = xs(rhs, xm(xm(2.0, p), __ldg(F.t_lbc + col)));
        p = 0.0;
    }
    const long slab = (long)nk * ld, o = (long)k * ld + col;
    pqrf[o] = p;
    pqrf[slab + o] = q;
    pqrf[2 * slab + o] = r;
    pqrf[3 * slab + o] = rhs;
    if (sys_out) {
        sys_out[o] = p;
        sys_out[slab + o] = q;
        sys_out[2 * slab + o] = r;
        sys_out[3 * slab + o] = rhs;
    }
}

int dt_scratch_planes() { return 4; }

cudaError_t launch_dt_ng(const DtFields &F, const DtConsts &C, double *tn_upd, int nk, int ncol, long ld,
                         double *sys_out, unsigned *status, cudaStream_t st, const PostStep *post, double *scratch)
{
    if (ncol <= 0) return cudaSuccess;
    // three-pass: the rows level-parallel, then the Thomas walk alone (on
    // 41472 columns 143 against 151 us for the fused walk)
    if (scratch && assembly_mode() == 2 && nk >= 3) {
        const long slab = (long)nk * ld;
        k_dt_coefs<<<dim3((ncol + 127) / 128, nk - 1), 128, 0, st>>>(F, C, scratch, nk, ncol, ld, sys_out);
        return launch_thomas_post(scratch, scratch + slab, scratch + 2 * slab, scratch + 3 * slab, tn_upd, nk, nk - 1,
                                  1, ncol, ld, status, post, st);
    }
    // one warp per block keeps a wave of small blocks resident despite the
    // per-thread shared memory (w2 column + staged reads)
    const int T = 32;
    const size_t smem = (size_t)T * ((nk - 2 > 0 ? nk - 2 : 1) * sizeof(double) + Stage<kDtStaged>::bytes_per_thread);
    once_per_device([] { cudaFuncSetAttribute(k_dt_ng, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_optin() - 1024); });
    k_dt_ng<<<(ncol + T - 1) / T, T, smem, st>>>(F, C, tn_upd, nk, ncol, ld, sys_out, status,
                                                  post ? *post : PostStep{}, post != nullptr, walk_prefetch(ncol));
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// dt_ng's history diagnostics (src/dt_ng.F90:169-191, and the density of
// :133) from the fields and the solution x (rows 1..nk, before the lateral
// overwrite): 12 level-major planes DTDT, DT_SOLAR, DT_HORDIF, DT_RECOMB,
// DT_JOULE, DT_MOLDIF, DT_COOL, DT_HORADV, DT_VERADV, DT_ADIA, DT_CONDUCT,
// DEN, the values the reference hands to addfld.  One thread per (level,
// column): every term of level k needs only levels k-1..k+1 (the wind shear
// of the top two levels comes from level nk-3's), so no column walk is
// needed.  Same operations in the same order as the reference: bit-identical.
// ---------------------------------------------------------------------------
namespace {
__device__ __forceinline__ double dt_vad0(const DtFields &F, int j, int nk, long ld, long col)
{
    if (j == 0) return xm(xm(xs(__ldg(F.tn + col), __ldg(F.t_lbc + col)), __ldg(F.w + col)), 2.0);
    if (j >= nk - 1) return 0.0;
    return xm(xs(__ldg(F.tn + (long)j * ld + col), __ldg(F.tn + (long)(j - 1) * ld + col)),
              __ldg(F.w + (long)j * ld + col));
}
// .5*(v(k)+v(k+1)), the top level extrapolated as 1.5*v(nk)-.5*v(nk-1)
__device__ __forceinline__ double dt_iface(const double *v, int k, int nk, long ld, long col)
{
    if (k < nk - 1) return xm(0.5, xa(__ldg(v + (long)k * ld + col), __ldg(v + (long)(k + 1) * ld + col)));
    return xs(xm(1.5, __ldg(v + (long)(nk - 1) * ld + col)), xm(0.5, __ldg(v + (long)(nk - 2) * ld + col)));
}
__device__ __forceinline__ double dt_shear(const double *v, const double *vlbc, const DtConsts &C, int k, int nk,
                                           long ld, long col)
{
    auto at = [&](int j) { return __ldg(v + (long)j * ld + col); };
    auto base = [&](int j) {   // the levels the reference computes directly
        if (j == 0) return xd(xs(xa(at(0), xm(1.0 / 3.0, at(1))), xm(4.0 / 3.0, __ldg(vlbc + col))), C.dz);
        return xd(xs(at(j + 1), at(j - 1)), xm(2.0, C.dz));
    };
    if (k <= nk - 3) return base(k);
    const double d = xd(base(nk - 3), 3.0);   // level nk-2
    return k == nk - 2 ? d : xd(d, 3.0);
}
__device__ __forceinline__ double dt_tni(const DtFields &F, int j, int nk, long ld, long col)
{
    if (j == 0) return __ldg(F.tlbc + col);
    if (j == nk - 1) return __ldg(F.tn + (long)(nk - 2) * ld + col);
    return xm(0.5, xa(__ldg(F.tn + (long)(j - 1) * ld + col), __ldg(F.tn + (long)j * ld + col)));
}
}  // namespace

__global__ void __launch_bounds__(256) k_dt_diag_ng(DtFields F, DtConsts C, const double *x, int nk, int ncol, long ld,
                                                    double *diag)
{
    const long col = (long)blockIdx.x * blockDim.x + threadIdx.x;
    const int k = blockIdx.y;
    if (col >= ncol) return;
    const long o = (long)k * ld + col, slab = (long)nk * ld;
    auto at = [&](const double *p) { return __ldg(p + o); };
    const double xk = x[o];
    const double expz = __ldg(F.expz + k);
    const double vad = k < nk - 1 ? xd(xm(xa(dt_vad0(F, k, nk, ld, col), dt_vad0(F, k + 1, nk, ld, col)), 0.5), C.dz)
                                  : xd(0.0, C.dz);
    const double cpi = dt_iface(F.cp, k, nk, ld, col), kmi = dt_iface(F.km, k, nk, ld, col);
    const double wi = dt_iface(F.w, k, nk, ld, col), qsolar = dt_iface(F.qtotal, k, nk, ld, col);
    const double dudz = dt_shear(F.un, F.ulbc, C, k, nk, ld, col), dvdz = dt_shear(F.vn, F.vlbc, C, k, nk, ld, col);
    // density (:126-133)
    const double h = at(F.schti);
    double rho = xd(xm(C.p0, C.expzmid_inv), xm(h, C.grav));
    rho = xm(rho, expz);
    const double mbar = at(F.mbar);
    const double xo = xm(xm(at(F.xnmbar), at(F.o1)), C.rmassinv_o1);
    const double qrecomb = xd(xm(xm(xm(C.tsurplus, at(F.rkm12)), xm(xo, xo)), C.avo), mbar);
    double qm = xm(xd(xm(C.grav, kmi), xm(C.p0, at(F.scht))), xa(xm(dudz, dudz), xm(dvdz, dvdz)));
    qm = xd(qm, expz);
    double *d = diag + o;
    d[0] = xm(C.dtx2inv, xs(xk, at(F.tnsmooth)));
    d[slab] = xd(qsolar, cpi);
    d[2 * slab] = xd(at(F.hdt), cpi);
    d[3 * slab] = xd(qrecomb, cpi);
    d[4 * slab] = xd(at(F.qji_tn), cpi);
    d[5 * slab] = xd(qm, cpi);
    const double cool_exp = xd(xd(at(F.cool_exp), cpi), expz);
    d[6 * slab] = xs(-cool_exp, xm(at(F.cool_imp), xk));
    d[7 * slab] = -at(F.horadv);
    d[8 * slab] = -vad;
    d[9 * slab] = -xm(xd(xm(wi, C.gask), xm(cpi, mbar)), xk);
    // conductive heating (:181-186), rows 2..nk-1
    double cond = 0.0;
    if (k >= 1 && k <= nk - 2) {
        const GF g0 = dt_gf(C, h, at(F.cp), at(F.kt), dt_tni(F, k, nk, ld, col), expz, __ldg(F.dift + k));
        const long o1 = o + ld;
        const GF g1 = dt_gf(C, __ldg(F.schti + o1), __ldg(F.cp + o1), __ldg(F.kt + o1), dt_tni(F, k + 1, nk, ld, col),
                            __ldg(F.expz + k + 1), __ldg(F.dift + k + 1));
        const double t = xa(xs(xm(xs(g0.g, g0.f), x[o - ld]), xm(xa(xa(xs(g1.g, g1.f), g0.g), g0.f), xk)),
                            xm(xa(g1.g, g1.f), x[o1]));
        cond = xm(xd(1.0, expz), t);
    }
    d[10 * slab] = xd(cond, cpi);
    d[11 * slab] = rho;
}

cudaError_t launch_dt_diag_ng(const DtFields &F, const DtConsts &C, const double *x, int nk, int ncol, long ld,
                              double *diag, cudaStream_t st)
{
    if (ncol <= 0) return cudaSuccess;
    k_dt_diag_ng<<<dim3((ncol + 255) / 256, nk), 256, 0, st>>>(F, C, x, nk, ncol, ld, diag);
    return cudaGetLastError();
}

}  // namespace tg

// ===========================================================================
// minor_ng (N4S, NO, N2D, Ar): src/minor_ng.F90:60-200, fused with the solve.
// Row k of the system needs the level quantities ax, thdiff and dmdz/barm of
// levels k and k+1; level j's quantities need tni of j-1..j+1, the interface
// mixing ratios of levels j-1 and j, and the inverse of the 3x3 matrix alfa of
// level j.  A thread carries level k's quantities from the previous row and
// computes level k+1's.  The fractional powers (tni/t00)**(1.75-ss) and
// (t00/tni)**0.25 use the device pow (within 2 ulp of the host library's), so
// this kernel matches the CPU restatement to a stated tolerance, not bitwise.
// ===========================================================================
namespace tg {
namespace {
__device__ __constant__ double kMPhi[3][4] = {{0., 1.35, 2.16, 1.11}, {0.673, 0., 1.616, 0.769}, {0.270, 0.404, 0., 0.322}};
__device__ __constant__ double kMSs[3] = {1.710, 1.749, 1.718};

__device__ __forceinline__ void inv3_ieee(const double (&A)[9], double (&W)[9])
{
    // matdet3 / matadj3 / matinv3 (src/matutil.F90)
#define a_(i, j) A[((i) - 1) + 3 * ((j) - 1)]
#define w_(i, j) W[((i) - 1) + 3 * ((j) - 1)]
    double d = xm(xm(a_(1, 1), a_(2, 2)), a_(3, 3));
    d = xs(d, xm(xm(a_(1, 1), a_(2, 3)), a_(3, 2)));
    d = xs(d, xm(xm(a_(1, 2), a_(2, 1)), a_(3, 3)));
    d = xa(d, xm(xm(a_(1, 2), a_(2, 3)), a_(3, 1)));
    d = xa(d, xm(xm(a_(1, 3), a_(2, 1)), a_(3, 2)));
    d = xs(d, xm(xm(a_(1, 3), a_(2, 2)), a_(3, 1)));
    w_(1, 1) = xs(xm(a_(2, 2), a_(3, 3)), xm(a_(2, 3), a_(3, 2)));
    w_(2, 1) = -xs(xm(a_(2, 1), a_(3, 3)), xm(a_(2, 3), a_(3, 1)));
    w_(3, 1) = xs(xm(a_(2, 1), a_(3, 2)), xm(a_(2, 2), a_(3, 1)));
    w_(1, 2) = -xs(xm(a_(1, 2), a_(3, 3)), xm(a_(1, 3), a_(3, 2)));
    w_(2, 2) = xs(xm(a_(1, 1), a_(3, 3)), xm(a_(1, 3), a_(3, 1)));
    w_(3, 2) = -xs(xm(a_(1, 1), a_(3, 2)), xm(a_(1, 2), a_(3, 1)));
    w_(1, 3) = xs(xm(a_(1, 2), a_(2, 3)), xm(a_(1, 3), a_(2, 2)));
    w_(2, 3) = -xs(xm(a_(1, 1), a_(2, 3)), xm(a_(1, 3), a_(2, 1)));
    w_(3, 3) = xs(xm(a_(1, 1), a_(2, 2)), xm(a_(1, 2), a_(2, 1)));
#undef a_
#undef w_
    // the nine quotients share the divisor: correctly rounded, bit-identical
    // to IEEE division (qdiv)
    const double y = __drcp_rn(d);
    const bool ds = exp_safe(d);
    unsigned dm = exp_dist(d);
#pragma unroll
    for (int e = 0; e < 9; ++e) dm = max(dm, exp_dist(W[e]));
    if (dm < kExpSpan) {   // pivot and all nine numerators in range: one test
#pragma unroll
        for (int e = 0; e < 9; ++e) W[e] = div_markstein(W[e], d, y);
        return;
    }
#pragma unroll
    for (int e = 0; e < 9; ++e) W[e] = qdiv_pivot(W[e], d, y, ds);
}

struct MinorLevel {
    double ax, thdiff, dmdzs;   // dmdz/barm
};

// Raw interface quantities of level j (minor_ng.F90:77-96).
struct MinorIface {
    double pso1, pso2, pshe, do1dz, do2dz, dhedz, dmdz;
};

__device__ __forceinline__ MinorIface minor_iface(const MinorConsts &C, double o1, double o1m, double o2, double o2m,
                                                  double he, double hem, double mb, double mbm)
{
    MinorIface r;
    r.dmdz = xd(xs(mb, mbm), C.dzp);
    r.pso1 = xm(0.5, xa(o1, o1m));
    r.pso2 = xm(0.5, xa(o2, o2m));
    r.pshe = xm(0.5, xa(he, hem));
    r.do1dz = xd(xs(o1, o1m), C.dzp);
    r.do2dz = xd(xs(o2, o2m), C.dzp);
    r.dhedz = xd(xs(he, hem), C.dzp);
    return r;
}

// The diffusion powers of a level from one logarithm: (tni/t00)**(1.75-ss)
// of the three species and (t00/tni)**0.25, as exp(y*ln(tni/t00)).  With
// |y*ln(tni/t00)| below 1 the argument's rounding adds about 2 ulp to exp's
// own error, within the tolerance the device pow already needs against the
// host library (the reference writes these as ** powers).
__device__ __forceinline__ void diffusion_powers(double tni, double (&df)[3], double &p25)
{
    const double lx = log(xd(tni, 273.0));
#pragma unroll
    for (int n = 0; n < 3; ++n) df[n] = exp(xm(xs(1.75, kMSs[n]), lx));
    p25 = exp(xm(-0.25, lx));
}

// ax, thdiff, dmdz/barm of level j (minor_ng.F90:100-153).
__device__ __forceinline__ MinorLevel minor_level(const MinorConsts &C, const MinorIface &I, double barm, double tni,
                                                  double dtnidz)
{
    const double tau = 1.86e+3;
    double df[3], p25;
    diffusion_powers(tni, df, p25);
#define PH(i, j) kMPhi[(i) - 1][(j) - 1]
    double A[9], W[9];
    A[0] = -xa(xa(PH(1, 4), xm(xs(PH(1, 2), PH(1, 4)), I.pso1)), xm(xs(xm(df[0], PH(1, 3)), PH(1, 4)), I.pshe));
    A[4] = -xa(xa(PH(2, 4), xm(xs(PH(2, 1), PH(2, 4)), I.pso2)), xm(xs(xm(df[1], PH(2, 3)), PH(2, 4)), I.pshe));
    A[8] = -xa(xa(xm(df[2], PH(3, 4)), xm(xs(xm(df[0], PH(3, 1)), xm(df[2], PH(3, 4))), I.pso2)),
               xm(xs(xm(df[1], PH(3, 2)), xm(df[2], PH(3, 4))), I.pso1));
    A[3] = xm(xs(PH(1, 2), PH(1, 4)), I.pso2);                          // (1,2)
    A[6] = xm(xs(xm(df[0], PH(1, 3)), PH(1, 4)), I.pso2);               // (1,3)
    A[1] = xm(xs(PH(2, 1), PH(2, 4)), I.pso1);                          // (2,1)
    A[7] = xm(xs(xm(df[1], PH(2, 3)), PH(2, 4)), I.pso1);               // (2,3)
    A[2] = xm(xs(xm(df[0], PH(3, 1)), xm(df[2], PH(3, 4))), I.pshe);     // (3,1)
    A[5] = xm(xs(xm(df[1], PH(3, 2)), xm(df[2], PH(3, 4))), I.pshe);     // (3,2)
#undef PH
    inv3_ieee(A, W);
    const double s0 = xs(C.phix[0], C.phix[3]), s1 = xs(C.phix[1], C.phix[3]), s2 = xs(C.phix[2], C.phix[3]);
    // salfax . invalfa(:,n)
    const double sa1 = xa(xa(xm(s0, W[0]), xm(s1, W[1])), xm(s2, W[2]));
    const double sa2 = xa(xa(xm(s0, W[3]), xm(s1, W[4])), xm(s2, W[5]));
    const double sa3 = xa(xa(xm(s0, W[6]), xm(s1, W[7])), xm(s2, W[8]));
    double ex = xs(1.0, xd(xa(C.rmx, I.dmdz), barm));
    ex = xa(ex, xm(sa1, xs(I.do2dz, xm(xs(1.0, xd(xa(C.rmass_o2, I.dmdz), barm)), I.pso2))));
    ex = xa(ex, xm(sa2, xs(I.do1dz, xm(xs(1.0, xd(xa(C.rmass_o1, I.dmdz), barm)), I.pso1))));
    ex = xa(ex, xm(sa3, xs(I.dhedz, xm(xs(1.0, xd(xa(C.rmass_he, I.dmdz), barm)), I.pshe))));
    MinorLevel L;
    L.dmdzs = xd(I.dmdz, barm);
    const double den = xa(xa(xa(C.phix[2], xm(s0, I.pso2)), xm(s1, I.pso1)), xm(s2, I.pshe));
    L.ax = -xd(xm(xd(barm, xm(tau, C.rmass_n2)), p25), den);
    L.thdiff = xs(ex, xd(xm(C.alfax, dtnidz), xm(C.dzp, tni)));
    return L;
}
}  // namespace

__global__ void __launch_bounds__(128) k_minor_ng(MinorFields F, MinorConsts C, double *out, int nk, int ncol, long ld,
                                                  double *sys_out, unsigned *status, PostStep post, int has_post)
{
    extern __shared__ double smem_mn[];
    const long col = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (col >= ncol) return;
    double *w2s = smem_mn + threadIdx.x;
    const int T = blockDim.x;
    auto at = [&](const double *p, int k) { return __ldg(p + k * ld + col); };
    const double dzp = C.dzp;
    // lower-boundary mixing ratios and mean mass (:72-75)
    const double o2_0 = at(F.o2, 0), o1_0 = at(F.o1, 0), he_0 = at(F.he, 0), mb_0 = at(F.mbar, 0);
    const double bo2 = xa(xa(xa(xm(C.b[0], o2_0), xm(C.b[3], o1_0)), xm(C.b[6], he_0)), C.fb[0]);
    const double bo1 = xa(xa(xa(xm(C.b[1], o2_0), xm(C.b[4], o1_0)), xm(C.b[7], he_0)), C.fb[1]);
    const double bhe = xa(xa(xa(xm(C.b[2], o2_0), xm(C.b[5], o1_0)), xm(C.b[8], he_0)), C.fb[2]);
    const double xmbari =
        xd(1.0, xa(xa(xa(xm(bo2, C.rmassinv_o2), xm(bo1, C.rmassinv_o1)),
                      xm(xs(xs(xs(1.0, bo2), bo1), bhe), C.rmassinv_n2)),
                   xm(bhe, C.rmassinv_he)));
    // tni(j) for j = 0..nk-1: tni(0) = tlbc, tni(nk-1) = tn(nk-2), else .5*(tn(j)+tn(j-1))
    const double tlbc = __ldg(F.tlbc + col);
    double tn_a = at(F.tn, 0), tn_b = nk > 1 ? at(F.tn, 1) : 0.0;   // tn(j), tn(j+1) while computing tni(j+1)
    auto tni_of = [&](int j, double tnj, double tnjm1) { return j == 0 ? tlbc : (j == nk - 1 ? tnjm1 : xm(0.5, xa(tnj, tnjm1))); };
    double tni_m = 0.0, tni_0 = tlbc, tni_p = tni_of(1, tn_b, tn_a);
    // level 0 interface values
    MinorIface I0;
    I0.dmdz = xd(xs(mb_0, xmbari), dzp);
    I0.pso1 = xm(0.5, xa(bo1, o1_0));
    I0.pso2 = xm(0.5, xa(bo2, o2_0));
    I0.pshe = xm(0.5, xa(bhe, he_0));
    I0.do1dz = xd(xs(o1_0, bo1), dzp);
    I0.do2dz = xd(xs(o2_0, bo2), dzp);
    I0.dhedz = xd(xs(he_0, bhe), dzp);
    auto dtnidz_of = [&](int j, double tm, double t0, double tp) {
        return j == 0 ? xs(tp, t0) : (j == nk - 1 ? xs(t0, tm) : xd(xs(tp, tm), 2.0));
    };
    MinorLevel L0 = minor_level(C, I0, at(F.barm, 0), tni_0, dtnidz_of(0, tni_m, tni_0, tni_p));
    double o1_p = o1_0, o2_p = o2_0, he_p = he_0, mb_p = mb_0;   // level values of the previous level
    const double dfac = __ldg(F.dfactor + col);
    const double rdz = xd(1.0, dzp);
    bool ok = true;
    double w1 = 0.0, w3 = 0.0, rprev = 0.0;
    for (int k = 0; k < nk; ++k) {
        double p, q, r, f;
        const double expz = __ldg(F.expz + k);
        const double sp = xd(xm(at(F.sprod, k), C.rmx), at(F.xnmbar, k));
        f = xa(xs(xm(at(F.ftm1_smooth, k), C.dtx2inv), at(F.hadvec, k)), sp);
        f = xm(f, expz);
        MinorLevel L1 = L0;
        if (k < nk - 1) {
            // level k+1 quantities
            const double o1k = at(F.o1, k + 1), o2k = at(F.o2, k + 1), hek = at(F.he, k + 1), mbk = at(F.mbar, k + 1);
            const MinorIface I1 = minor_iface(C, o1k, o1_p, o2k, o2_p, hek, he_p, mbk, mb_p);
            o1_p = o1k; o2_p = o2k; he_p = hek; mb_p = mbk;
            // tni of k+2 for dtnidz(k+1)
            double tni_pp = 0.0;
            if (k + 2 <= nk - 1) {
                const double tn_c = at(F.tn, k + 2);
                tni_pp = tni_of(k + 2, tn_c, tn_b);
                tn_a = tn_b;
                tn_b = tn_c;
            }
            L1 = minor_level(C, I1, at(F.barm, k + 1), tni_p, dtnidz_of(k + 1, tni_0, tni_p, tni_pp));
            tni_m = tni_0;
            tni_0 = tni_p;
            tni_p = tni_pp;
            // row k (:161-184)
            const double difk0 = __ldg(F.difk + k), difk1 = __ldg(F.difk + k + 1);
            const double molp = xm(L0.ax, xa(rdz, xm(0.5, L0.thdiff)));
            const double molr = xm(L1.ax, xs(rdz, xm(0.5, L1.thdiff)));
            const double molq = xa(xm(L0.ax, xs(rdz, xm(0.5, L0.thdiff))), xm(L1.ax, xa(rdz, xm(0.5, L1.thdiff))));
            const double eddyp = xm(xm(C.expzmid_inv, difk0), xs(rdz, xm(0.5, L0.dmdzs)));
            const double eddyr = xm(xm(C.expzmid, difk1), xa(rdz, xm(0.5, L1.dmdzs)));
            const double eddyq = xa(xm(xm(C.expzmid_inv, difk0), xa(rdz, xm(0.5, L0.dmdzs))),
                                    xm(xm(C.expzmid, difk1), xs(rdz, xm(0.5, L1.dmdzs))));
            const double wk = at(F.w, k), wk1 = at(F.w, k + 1);
            const double wi = xm(0.5, xa(wk, wk1));
            p = xs(xd(molp, dzp), xd(xm(expz, xa(xm(eddyp, dfac), xm(0.5, wi))), dzp));
            r = xs(xd(molr, dzp), xd(xm(expz, xs(xm(eddyr, dfac), xm(0.5, wi))), dzp));
            q = xa(-xd(molq, dzp), xm(expz, xs(xa(xd(xm(eddyq, dfac), dzp), C.dtx2inv), at(F.sloss, k))));
            if (k == 0) {   // lower boundary (:191-193)
                const double l1 = __ldg(F.flbc1 + col), l2 = __ldg(F.flbc2 + col), l3 = __ldg(F.flbc3 + col);
                const double den = xs(l1, xm(xm(0.5, l2), dzp));
                q = xa(q, xd(xm(p, xa(l1, xm(xm(0.5, l2), dzp))), den));
                f = xs(f, xd(xm(xm(p, l3), dzp), den));
                p = 0.0;
            }
        } else {   // top row (:195-198)
            p = xa(1.0, xm(xm(0.5, dzp), L0.thdiff));
            q = xs(p, 2.0);
            r = 0.0;
            f = -xd(xm(xm(xm(C.grav, C.rmx), __ldg(F.fubc + col)), dzp), xm(xm(C.p0, L0.ax), C.avo));
        }
        if (sys_out) {
            const long n = (long)nk * ld;
            sys_out[k * ld + col] = p;
            sys_out[n + k * ld + col] = q;
            sys_out[2 * n + k * ld + col] = r;
            sys_out[3 * n + k * ld + col] = f;
        }
        // Thomas forward step
        if (k == 0) {
            w1 = q;
            w3 = xd(f, w1);
        } else {
            const double w2 = xd(rprev, w1);
            w2s[(k - 1) * T] = w2;
            w1 = xs(q, xm(p, w2));
            w3 = xd(xs(f, xm(p, w3)), w1);
        }
        ok = ok && fin_nz(w1);
        out[k * ld + col] = w3;
        rprev = r;
        L0 = L1;
    }
    (void)tn_a;
    (void)tni_m;
    // back sweep; with has_post every row goes through the post-solve steps
    // (:226-237), the top row's unfiltered value first
    const bool bcol = has_post && post.bnd_mask && post.bnd_mask[col];
    double xn = w3;
    bool fin = fabs(xn) <= DBL_MAX;
    if (has_post) post_store(post, true, bcol, out, (long)(nk - 1) * ld + col, xn);
    for (int k = nk - 2; k >= 0; --k) {
        xn = xs(out[k * ld + col], xm(w2s[k * T], xn));
        fin = fin && fabs(xn) <= DBL_MAX;
        post_store(post, has_post, bcol, out, k * ld + col, xn);
    }
    if (status && (!ok || !fin)) atomicOr(status, (ok ? 0u : FLAG_PIVOT) | (fin ? 0u : FLAG_NONFINITE));
}

// ---------------------------------------------------------------------------
// minor_ng in two passes.  The level quantities (ax, thdiff, dmdz/barm: four
// fractional powers and a 3x3 inverse per level) are independent across
// levels, so the first kernel computes them with one thread per (level,
// column), i.e. nk times the parallelism of the column walk, into a 3-plane
// level-major buffer; the second walks each column once, forming the rows
// from those planes and solving.  Same operations as k_minor_ng.
// ---------------------------------------------------------------------------
__device__ __forceinline__ double minor_tni(const MinorFields &F, int j, int nk, long ld, long col, double tlbc)
{
    if (j == 0) return tlbc;
    if (j == nk - 1) return __ldg(F.tn + (long)(nk - 2) * ld + col);
    return xm(0.5, xa(__ldg(F.tn + (long)j * ld + col), __ldg(F.tn + (long)(j - 1) * ld + col)));
}

// ax, thdiff, dmdz/barm of level j of one column (minor_ng.F90:72-153).
__device__ __forceinline__ MinorLevel minor_level_at(const MinorFields &F, const MinorConsts &C, int j, int nk, long ld,
                                                     long col)
{
    auto at = [&](const double *p, int k) { return __ldg(p + k * ld + col); };
    const double dzp = C.dzp, tlbc = __ldg(F.tlbc + col);
    MinorIface I;
    if (j == 0) {
        const double o2_0 = at(F.o2, 0), o1_0 = at(F.o1, 0), he_0 = at(F.he, 0), mb_0 = at(F.mbar, 0);
        const double bo2 = xa(xa(xa(xm(C.b[0], o2_0), xm(C.b[3], o1_0)), xm(C.b[6], he_0)), C.fb[0]);
        const double bo1 = xa(xa(xa(xm(C.b[1], o2_0), xm(C.b[4], o1_0)), xm(C.b[7], he_0)), C.fb[1]);
        const double bhe = xa(xa(xa(xm(C.b[2], o2_0), xm(C.b[5], o1_0)), xm(C.b[8], he_0)), C.fb[2]);
        const double xmbari =
            xd(1.0, xa(xa(xa(xm(bo2, C.rmassinv_o2), xm(bo1, C.rmassinv_o1)),
                          xm(xs(xs(xs(1.0, bo2), bo1), bhe), C.rmassinv_n2)),
                       xm(bhe, C.rmassinv_he)));
        I.dmdz = xd(xs(mb_0, xmbari), dzp);
        I.pso1 = xm(0.5, xa(bo1, o1_0));
        I.pso2 = xm(0.5, xa(bo2, o2_0));
        I.pshe = xm(0.5, xa(bhe, he_0));
        I.do1dz = xd(xs(o1_0, bo1), dzp);
        I.do2dz = xd(xs(o2_0, bo2), dzp);
        I.dhedz = xd(xs(he_0, bhe), dzp);
    } else {
        I = minor_iface(C, at(F.o1, j), at(F.o1, j - 1), at(F.o2, j), at(F.o2, j - 1), at(F.he, j), at(F.he, j - 1),
                        at(F.mbar, j), at(F.mbar, j - 1));
    }
    const double t0 = minor_tni(F, j, nk, ld, col, tlbc);
    double dt;
    if (j == 0) dt = xs(minor_tni(F, 1, nk, ld, col, tlbc), t0);
    else if (j == nk - 1) dt = xs(t0, minor_tni(F, nk - 2, nk, ld, col, tlbc));
    else dt = xd(xs(minor_tni(F, j + 1, nk, ld, col, tlbc), minor_tni(F, j - 1, nk, ld, col, tlbc)), 2.0);
    return minor_level(C, I, at(F.barm, j), t0, dt);
}

__global__ void __launch_bounds__(128) k_minor_levels(MinorFields F, MinorConsts C, double *lv, int nk, int ncol,
                                                      long ld)
{
    const long col = (long)blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y;
    if (col >= ncol) return;
    const MinorLevel L = minor_level_at(F, C, j, nk, ld, col);
    const long slab = (long)nk * ld;
    lv[(long)j * ld + col] = L.ax;
    lv[slab + (long)j * ld + col] = L.thdiff;
    lv[2 * slab + (long)j * ld + col] = L.dmdzs;
}

// Row k of minor_ng's system (minor_ng.F90:150-198): from the level planes
// of levels k and k+1 and the fields of level k; the lower-boundary fold at
// k = 0 and the upper-boundary row at k = nk-1.
struct MinorRowIn {
    double sprod, xnmbar, ftm1, hadvec, sloss, w0, w1;
    MinorLevel L0, L1;
};
__device__ __forceinline__ void minor_row(const MinorFields &F, const MinorConsts &C, long col, int k, int nk,
                                          double dfac, const MinorRowIn &in, double &p, double &q, double &r,
                                          double &f)
{
    const double dzp = C.dzp, rdz = xd(1.0, dzp);
    const MinorLevel &L0 = in.L0, &L1 = in.L1;
    const double expz = __ldg(F.expz + k);
    const double sp = xd(xm(in.sprod, C.rmx), in.xnmbar);
    f = xa(xs(xm(in.ftm1, C.dtx2inv), in.hadvec), sp);
    f = xm(f, expz);
    if (k < nk - 1) {
        const double difk0 = __ldg(F.difk + k), difk1 = __ldg(F.difk + k + 1);
        const double molp = xm(L0.ax, xa(rdz, xm(0.5, L0.thdiff)));
        const double molr = xm(L1.ax, xs(rdz, xm(0.5, L1.thdiff)));
        const double molq = xa(xm(L0.ax, xs(rdz, xm(0.5, L0.thdiff))), xm(L1.ax, xa(rdz, xm(0.5, L1.thdiff))));
        const double eddyp = xm(xm(C.expzmid_inv, difk0), xs(rdz, xm(0.5, L0.dmdzs)));
        const double eddyr = xm(xm(C.expzmid, difk1), xa(rdz, xm(0.5, L1.dmdzs)));
        const double eddyq = xa(xm(xm(C.expzmid_inv, difk0), xa(rdz, xm(0.5, L0.dmdzs))),
                                xm(xm(C.expzmid, difk1), xs(rdz, xm(0.5, L1.dmdzs))));
        const double wi = xm(0.5, xa(in.w0, in.w1));
        p = xs(xd(molp, dzp), xd(xm(expz, xa(xm(eddyp, dfac), xm(0.5, wi))), dzp));
        r = xs(xd(molr, dzp), xd(xm(expz, xs(xm(eddyr, dfac), xm(0.5, wi))), dzp));
        q = xa(-xd(molq, dzp), xm(expz, xs(xa(xd(xm(eddyq, dfac), dzp), C.dtx2inv), in.sloss)));
        if (k == 0) {
            const double l1 = __ldg(F.flbc1 + col), l2 = __ldg(F.flbc2 + col), l3 = __ldg(F.flbc3 + col);
            const double den = xs(l1, xm(xm(0.5, l2), dzp));
            q = xa(q, xd(xm(p, xa(l1, xm(xm(0.5, l2), dzp))), den));
            f = xs(f, xd(xm(xm(p, l3), dzp), den));
            p = 0.0;
        }
    } else {
        p = xa(1.0, xm(xm(0.5, dzp), L0.thdiff));
        q = xs(p, 2.0);
        r = 0.0;
        f = -xd(xm(xm(xm(C.grav, C.rmx), __ldg(F.fubc + col)), dzp), xm(xm(C.p0, L0.ax), C.avo));
    }
}

// Three-pass form, pass 2: row k of every column, one thread per (row,
// column), into the planes pqrf (p, q, r, f, each nk*ld).
__global__ void __launch_bounds__(128) k_minor_coefs(MinorFields F, MinorConsts C, const double *lv, double *pqrf,
                                                     int nk, int ncol, long ld, double *sys_out)
{
    const long col = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (col >= ncol) return;
    const int k = blockIdx.y;
    const long slab = (long)nk * ld, o = (long)k * ld + col;
    {
        // every line the row reads, requested into L1 at once
        const long op = k < nk - 1 ? o + ld : o;
        const double *one[] = {F.sprod, F.xnmbar, F.ftm1_smooth, F.hadvec, F.sloss, F.w};
#pragma unroll
        for (int i = 0; i < 6; ++i) pf_l1(one[i] + o);
        pf_l1(F.w + op);
#pragma unroll
        for (int e = 0; e < 3; ++e) {
            pf_l1(lv + e * slab + o);
            pf_l1(lv + e * slab + op);
        }
    }
    MinorRowIn in;
    in.sprod = __ldg(F.sprod + o);
    in.xnmbar = __ldg(F.xnmbar + o);
    in.ftm1 = __ldg(F.ftm1_smooth + o);
    in.hadvec = __ldg(F.hadvec + o);
    in.L0.ax = __ldg(lv + o);
    in.L0.thdiff = __ldg(lv + slab + o);
    in.L0.dmdzs = __ldg(lv + 2 * slab + o);
    in.L1 = in.L0;
    in.sloss = in.w0 = in.w1 = 0.0;
    if (k < nk - 1) {
        in.sloss = __ldg(F.sloss + o);
        in.w0 = __ldg(F.w + o);
        in.w1 = __ldg(F.w + o + ld);
        in.L1.ax = __ldg(lv + o + ld);
        in.L1.thdiff = __ldg(lv + slab + o + ld);
        in.L1.dmdzs = __ldg(lv + 2 * slab + o + ld);
    }
    double p, q, r, f;
    minor_row(F, C, col, k, nk, __ldg(F.dfactor + col), in, p, q, r, f);
    pqrf[o] = p;
    pqrf[slab + o] = q;
    pqrf[2 * slab + o] = r;
    pqrf[3 * slab + o] = f;
    if (sys_out) {
        sys_out[o] = p;
        sys_out[slab + o] = q;
        sys_out[2 * slab + o] = r;
        sys_out[3 * slab + o] = f;
    }
}

// The column walk over the level planes.  Its eleven per-level reads are
// staged one iteration ahead (Stage); the back sweep re-reads the parked w3
// one level ahead.  The two divisions of a level share the divisor w1
// (qdiv: one correctly rounded reciprocal, the same bits as IEEE a/b).
constexpr int kMinorStaged = 11;
__global__ void __launch_bounds__(128) k_minor_rows(MinorFields F, MinorConsts C, const double *lv, double *out,
                                                    int nk, int ncol, long ld, double *sys_out, unsigned *status,
                                                    PostStep post, int has_post, int pd)
{
    extern __shared__ double smem_mr[];
    const long col = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (col >= ncol) return;
    double *w2s = smem_mr + threadIdx.x;
    const int T = blockDim.x;
    Stage<kMinorStaged> sg{smem_mr + (long)(nk > 1 ? nk - 1 : 1) * T + threadIdx.x, T};
    const long slab = (long)nk * ld;
    // reads of level k into buffer b: 0 sprod, 1 xnmbar, 2 ftm1_smooth,
    // 3 hadvec, 4 sloss, 5 w(k), 6 w(k+1), 7..9 planes of level k+1;
    // fn(value index, address)
    auto reads = [&](int k, auto &&fn) {
        const long o = (long)k * ld + col;
        fn(0, F.sprod + o);
        fn(1, F.xnmbar + o);
        fn(2, F.ftm1_smooth + o);
        fn(3, F.hadvec + o);
        if (k < nk - 1) {
            fn(4, F.sloss + o);
            fn(5, F.w + o);
            fn(6, F.w + o + ld);
            fn(7, lv + o + ld);
            fn(8, lv + slab + o + ld);
            fn(9, lv + 2 * slab + o + ld);
        }
    };
    auto issue = [&](int k, int b) { reads(k, [&](int v, const double *src) { sg.copy(b, v, src); }); };
    auto prefetch = [&](int k) { reads(k, [](int, const double *src) { pf_l1(src); }); };
    const double dfac = __ldg(F.dfactor + col);
    MinorLevel L0;
    L0.ax = __ldg(lv + col);
    L0.thdiff = __ldg(lv + slab + col);
    L0.dmdzs = __ldg(lv + 2 * slab + col);
    bool ok = true;
    double w1 = 0.0, y1 = 0.0, w3 = 0.0, rprev = 0.0;
    issue(0, 0);
    sg.commit();
    for (int kk = 2; kk < pd + 1 && kk < nk; ++kk) prefetch(kk);
    for (int k = 0; k < nk; ++k) {
        if (pd > 1 && k + 1 + pd < nk) prefetch(k + 1 + pd);
        if (k + 1 < nk) issue(k + 1, (k + 1) & 1);
        sg.commit();
        sg.wait_prev();
        const int b = k & 1;
        MinorRowIn in;
        in.sloss = in.w0 = in.w1 = 0.0;
        in.sprod = sg.at(b, 0);
        in.xnmbar = sg.at(b, 1);
        in.ftm1 = sg.at(b, 2);
        in.hadvec = sg.at(b, 3);
        in.L0 = L0;
        in.L1 = L0;
        if (k < nk - 1) {
            in.sloss = sg.at(b, 4);
            in.w0 = sg.at(b, 5);
            in.w1 = sg.at(b, 6);
            in.L1.ax = sg.at(b, 7);
            in.L1.thdiff = sg.at(b, 8);
            in.L1.dmdzs = sg.at(b, 9);
        }
        double p, q, r, f;
        minor_row(F, C, col, k, nk, dfac, in, p, q, r, f);
        const MinorLevel L1 = in.L1;
        if (sys_out) {
            sys_out[k * ld + col] = p;
            sys_out[slab + k * ld + col] = q;
            sys_out[2 * slab + k * ld + col] = r;
            sys_out[3 * slab + k * ld + col] = f;
        }
        if (k == 0) {
            w1 = q;
            y1 = __drcp_rn(w1);
            w3 = qdiv(f, w1, y1);
        } else {
            const double w2 = qdiv(rprev, w1, y1);
            w2s[(k - 1) * T] = w2;
            w1 = xs(q, xm(p, w2));
            y1 = __drcp_rn(w1);
            w3 = qdiv(xs(f, xm(p, w3)), w1, y1);
        }
        ok = ok && fin_nz(w1);
        out[k * ld + col] = w3;
        rprev = r;
        L0 = L1;
    }
    const bool bcol = has_post && post.bnd_mask && post.bnd_mask[col];
    double xn = w3;
    bool fin = fabs(xn) <= DBL_MAX;
    double park = nk >= 2 ? out[(nk - 2) * ld + col] : 0.0;
    if (has_post) post_store(post, true, bcol, out, (long)(nk - 1) * ld + col, xn);
    for (int kk = nk - 3; kk > nk - 2 - pd && kk >= 0; --kk) post_prefetch(post, has_post, bcol, out, (long)kk * ld + col);
    for (int k = nk - 2; k >= 0; --k) {
        if (k - pd >= 0) post_prefetch(post, has_post, bcol, out, (long)(k - pd) * ld + col);
        const double wk = park;
        if (k >= 1) park = out[(k - 1) * ld + col];
        xn = xs(wk, xm(w2s[k * T], xn));
        fin = fin && fabs(xn) <= DBL_MAX;
        post_store(post, has_post, bcol, out, k * ld + col, xn);
    }
    if (status && (!ok || !fin)) atomicOr(status, (ok ? 0u : FLAG_PIVOT) | (fin ? 0u : FLAG_NONFINITE));
}

static std::atomic<int> g_assembly_mode{2};
int assembly_mode() { return g_assembly_mode.load(); }
void set_assembly_mode(int m) { g_assembly_mode.store(m < 0 ? 2 : (m > 2 ? 2 : m)); }

// level planes (ax, thdiff, dmdz/barm) and the rows p, q, r, f
int minor_scratch_planes() { return 7; }

static std::atomic<int> g_walk_prefetch{-1};
int walk_prefetch(long ncol)
{
    const int v = g_walk_prefetch.load();
    if (v >= 1) return v;
    return ncol <= kSmallWalkColumns ? 8 : 1;
}
void set_walk_prefetch(int levels) { g_walk_prefetch.store(levels < 1 ? -1 : (levels > 32 ? 32 : levels)); }

cudaError_t launch_minor_ng(const MinorFields &F, const MinorConsts &C, double *out, int nk, int ncol, long ld,
                            double *sys_out, unsigned *status, cudaStream_t st, double *scratch, const PostStep *post)
{
    const PostStep pv = post ? *post : PostStep{};
    const int hp = post != nullptr;
    if (ncol <= 0) return cudaSuccess;
    const int optin = smem_optin();
    once_per_device([optin] {
        cudaFuncSetAttribute(k_minor_ng, cudaFuncAttributeMaxDynamicSharedMemorySize, optin);
        cudaFuncSetAttribute(k_minor_rows, cudaFuncAttributeMaxDynamicSharedMemorySize, optin);
    });
    // w2 of the forward sweep lives in shared memory, one column per thread:
    // shrink the block until the column fits (nk <= ~220 at 128 threads).
    int T = 128;
    while (T > 32 && (size_t)T * (nk - 1) * sizeof(double) > (size_t)optin) T /= 2;
    const size_t smem = (size_t)T * (nk - 1 > 0 ? nk - 1 : 1) * sizeof(double);
    if (smem > (size_t)optin) return cudaErrorInvalidValue;
    if (scratch && assembly_mode() == 2) {
        const long slab = (long)nk * ld;
        double *pqrf = scratch + 3 * slab;
        k_minor_levels<<<dim3((ncol + 127) / 128, nk), 128, 0, st>>>(F, C, scratch, nk, ncol, ld);
        k_minor_coefs<<<dim3((ncol + 127) / 128, nk), 128, 0, st>>>(F, C, scratch, pqrf, nk, ncol, ld, sys_out);
        return launch_thomas_post(pqrf, pqrf + slab, pqrf + 2 * slab, pqrf + 3 * slab, out, nk, nk, 0, ncol, ld,
                                  status, post, st);
    }
    if (scratch && assembly_mode() >= 1) {
        // the row walk also holds its staged reads in shared memory
        const size_t per_r = (size_t)(nk - 1 > 0 ? nk - 1 : 1) * sizeof(double) + Stage<kMinorStaged>::bytes_per_thread;
        int TR = 128;
        while (TR > 32 && (size_t)TR * per_r > (size_t)optin) TR /= 2;
        if ((size_t)TR * per_r > (size_t)optin) return cudaErrorInvalidValue;
        k_minor_levels<<<dim3((ncol + 127) / 128, nk), 128, 0, st>>>(F, C, scratch, nk, ncol, ld);
        k_minor_rows<<<(ncol + TR - 1) / TR, TR, (size_t)TR * per_r, st>>>(F, C, scratch, out, nk, ncol, ld, sys_out,
                                                                          status, pv, hp, walk_prefetch(ncol));
        return cudaGetLastError();
    }
    k_minor_ng<<<(ncol + T - 1) / T, T, smem, st>>>(F, C, out, nk, ncol, ld, sys_out, status, pv, hp);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// minor_ng's history diagnostics (src/minor_ng.F90:202-224) from the fields
// and the solution x (before the lateral overwrite and the floor): 7
// level-major planes D<name>DT, <name>_PROD, <name>_LOSS, <name>_MOLDIF,
// <name>_EDDYDIF, -<name>_VERADV, -<name>_HORADV, the values the reference
// hands to addfld (MOLDIF, EDDYDIF and VERADV rows 1 and nk, which the
// reference leaves unset, are 0).  One thread per (level, column); the level
// quantities ax, thdiff, dmdz/barm of levels k and k+1 come from the same
// device code as the solve (its fractional powers within a few ulp of the
// host library's), everything else is bit-identical.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(128) k_minor_diag_ng(MinorFields F, MinorConsts C, const double *x, int nk, int ncol,
                                                       long ld, double *diag)
{
    const long col = (long)blockIdx.x * blockDim.x + threadIdx.x;
    const int k = blockIdx.y;
    if (col >= ncol) return;
    const long o = (long)k * ld + col, slab = (long)nk * ld;
    const double xk = x[o], dzp = C.dzp;
    double *d = diag + o;
    d[0] = xm(C.dtx2inv, xs(xk, __ldg(F.ftm1_smooth + o)));
    d[slab] = xd(xm(__ldg(F.sprod + o), C.rmx), __ldg(F.xnmbar + o));
    d[2 * slab] = xm(__ldg(F.sloss + o), xk);
    d[6 * slab] = -__ldg(F.hadvec + o);
    double mol = 0.0, eddy = 0.0, vadv = 0.0;
    if (k >= 1 && k <= nk - 2) {
        const MinorLevel L0 = minor_level_at(F, C, k, nk, ld, col), L1 = minor_level_at(F, C, k + 1, nk, ld, col);
        const double rdz = xd(1.0, dzp);
        const double molp = xm(L0.ax, xa(rdz, xm(0.5, L0.thdiff)));
        const double molr = xm(L1.ax, xs(rdz, xm(0.5, L1.thdiff)));
        const double molq = xa(xm(L0.ax, xs(rdz, xm(0.5, L0.thdiff))), xm(L1.ax, xa(rdz, xm(0.5, L1.thdiff))));
        const double dk = __ldg(F.difk + k), dk1 = __ldg(F.difk + k + 1);
        const double eddyp = xm(xm(C.expzmid_inv, dk), xs(rdz, xm(0.5, L0.dmdzs)));
        const double eddyr = xm(xm(C.expzmid, dk1), xa(rdz, xm(0.5, L1.dmdzs)));
        const double eddyq = xa(xm(xm(C.expzmid_inv, dk), xa(rdz, xm(0.5, L0.dmdzs))),
                                xm(xm(C.expzmid, dk1), xs(rdz, xm(0.5, L1.dmdzs))));
        const double xm1 = x[o - ld], xp1 = x[o + ld];
        mol = -xm(xd(xd(1.0, __ldg(F.expz + k)), dzp), xa(xs(xm(molp, xm1), xm(molq, xk)), xm(molr, xp1)));
        eddy = xm(rdz, xa(xs(xm(eddyp, xm1), xm(eddyq, xk)), xm(eddyr, xp1)));
        const double wi = xm(0.5, xa(__ldg(F.w + o), __ldg(F.w + o + ld)));
        vadv = -xm(xd(wi, xm(2.0, dzp)), xs(xp1, xm1));
    }
    d[3 * slab] = mol;
    d[4 * slab] = xm(eddy, __ldg(F.dfactor + col));
    d[5 * slab] = vadv;
}

cudaError_t launch_minor_diag_ng(const MinorFields &F, const MinorConsts &C, const double *x, int nk, int ncol, long ld,
                                 double *diag, cudaStream_t st)
{
    if (ncol <= 0) return cudaSuccess;
    k_minor_diag_ng<<<dim3((ncol + 127) / 128, nk), 128, 0, st>>>(F, C, x, nk, ncol, ld, diag);
    return cudaGetLastError();
}

}  // namespace tg

// ===========================================================================
// comp_ng (O2, O, He): src/comp_ng.F90:74-332, assembly fused with the 3x3
// block solve.  Row k needs ep and ak = inv(alpha)*wks1 of levels k and k+1
// and the interface averages of level k+1; a thread carries level k from the
// previous row.  The forward sweep keeps Gamma_{k+1} (9) and z_{k+1} (3) of
// every row in a level-major global scratch (L2-resident for the back sweep).
// The fractional powers use the device pow, as in minor_ng: the kernel agrees
// with the CPU restatement to a stated tolerance.
// ===========================================================================
namespace tg {
namespace {
struct CompLevel {
    double ep[3], ak[9], wks4, a22, a33, a23, a32;
};

// ep, alpha, ak and wks4 of one level (comp_ng.F90:128-166, 176-211)
__device__ __forceinline__ void comp_level(const CompConsts &C, double o2i, double o1i, double hei, double embari,
                                           double tni, double dembardz, double dtndz, bool thermal, CompLevel &L)
{
    const double tau = 1.86e+3, thdiffalpha = -0.38;
    double df[3], p25;
    diffusion_powers(tni, df, p25);
    const double rinv = xd(1.0, embari);
    L.ep[0] = xs(1.0, xm(rinv, xa(C.rmass_o2, dembardz)));
    L.ep[1] = xs(1.0, xm(rinv, xa(C.rmass_o1, dembardz)));
    L.ep[2] = xs(1.0, xm(rinv, xa(C.rmass_he, dembardz)));
    if (thermal) L.ep[2] = xs(L.ep[2], xd(xm(thdiffalpha, dtndz), tni));
#define PH(i, j) kMPhi[(i) - 1][(j) - 1]
    double A[9], W[9];
    A[0] = -xa(xa(PH(1, 4), xm(xs(PH(1, 2), PH(1, 4)), o1i)), xm(xs(xm(df[0], PH(1, 3)), PH(1, 4)), hei));
    A[4] = -xa(xa(PH(2, 4), xm(xs(PH(2, 1), PH(2, 4)), o2i)), xm(xs(xm(df[1], PH(2, 3)), PH(2, 4)), hei));
    A[8] = -xa(xa(xm(df[2], PH(3, 4)), xm(xs(xm(df[0], PH(3, 1)), xm(df[2], PH(3, 4))), o2i)),
               xm(xs(xm(df[1], PH(3, 2)), xm(df[2], PH(3, 4))), o1i));
    A[3] = xm(xs(PH(1, 2), PH(1, 4)), o2i);                          // (1,2)
    A[6] = xm(xs(xm(df[0], PH(1, 3)), PH(1, 4)), o2i);               // (1,3)
    A[1] = xm(xs(PH(2, 1), PH(2, 4)), o1i);                          // (2,1)
    A[7] = xm(xs(xm(df[1], PH(2, 3)), PH(2, 4)), o1i);               // (2,3)
    A[2] = xm(xs(xm(df[0], PH(3, 1)), xm(df[2], PH(3, 4))), hei);     // (3,1)
    A[5] = xm(xs(xm(df[1], PH(3, 2)), xm(df[2], PH(3, 4))), hei);     // (3,2)
#undef PH
    L.a22 = A[4];
    L.a33 = A[8];
    L.a23 = A[7];
    L.a32 = A[5];
    inv3_ieee(A, W);
    const double wks1 = xd(xm(xm(embari, C.rmassinv_n2), p25), tau);
#pragma unroll
    for (int e = 0; e < 9; ++e) L.ak[e] = xm(W[e], wks1);
    L.wks4 = xd(dembardz, xm(embari, 2.0));
}
}  // namespace
}  // namespace tg

namespace tg {
// Row k of the comp_ng block system (comp_ng.F90:213-279): P, Q, R and f
// from the level quantities of levels k (Lk) and k+1 (Lp) and the fields of
// level k (through Src), with both boundary folds; flx00 is set at the top row.
template <class Src>
__device__ __forceinline__ void comp_row(const CompFields &F, const CompConsts &C, const Src &src, const CompLevel &Lk,
                                         const CompLevel &Lp, int k, int nk, long ld, long col, double dfac,
                                         double flx_he, double (&P)[9], double (&Q)[9], double (&R)[9],
                                         double (&f)[3], double &flx00)
{
    auto at = [&](const double *p, int kk) { return __ldg(p + kk * ld + col); };
    const double tau = 1.86e+3, t00 = 273.;
    const double dz = C.dz, rdz = xd(1.0, dz);
    const double wi = xm(0.5, xa(src.w(k), src.w1(k)));
    const double difk0 = __ldg(F.difk + k), difk1 = __ldg(F.difk + k + 1), ez = __ldg(F.expz + k);
    // mol / eddy coefficients and the rows (comp_ng.F90:213-244)
    const double eddyp = xm(xm(C.expzmid_inv, difk0), xs(rdz, Lk.wks4));
    const double eddyr = xm(xm(C.expzmid, difk1), xa(rdz, Lp.wks4));
    const double eddyq =
        xa(xm(xm(C.expzmid_inv, difk0), xa(rdz, Lk.wks4)), xm(xm(C.expzmid, difk1), xs(rdz, Lp.wks4)));
    const double ezdz = xd(ez, dz);
    const double tp = xm(ezdz, xa(xm(eddyp, dfac), xm(0.5, wi)));
    const double tr = xm(ezdz, xs(xm(eddyr, dfac), xm(0.5, wi)));
    const double tq = xm(ez, xa(xd(xm(eddyq, dfac), dz), C.dtx2inv));
#pragma unroll
    for (int m = 0; m < 3; ++m) {
        const double hk = xd(Lk.ep[m], 2.0), hp = xd(Lp.ep[m], 2.0);
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            const int e = i + 3 * m;
            const double molp = xm(Lk.ak[e], xa(rdz, hk));
            const double molr = xm(Lp.ak[e], xs(rdz, hp));
            const double molq = xa(xm(Lk.ak[e], xs(rdz, hk)), xm(Lp.ak[e], xa(rdz, hp)));
            const double fsl = xm(ez, src.fs((m + 1) * 3 + i, k));
            P[e] = i == m ? xs(xd(molp, dz), tp) : xd(molp, dz);
            R[e] = i == m ? xs(xd(molr, dz), tr) : xd(molr, dz);
            Q[e] = i == m ? xs(xa(-xd(molq, dz), tq), fsl) : xs(-xd(molq, dz), fsl);
        }
    }
#pragma unroll
    for (int i = 0; i < 3; ++i)
        f[i] = xm(ez, xa(xs(xm(src.nms(i, k), C.dtx2inv), xs(src.adv(i, k), src.fs(i, k))), src.hd(i, k)));
    if (k == 0) {
        // lower boundary b(3,3), fb(3) (comp_ng.F90:246-258)
#pragma unroll
        for (int m = 0; m < 3; ++m)
#pragma unroll
            for (int n = 0; n < 3; ++n)
#pragma unroll
                for (int i = 0; i < 3; ++i) Q[i + 3 * m] = xa(Q[i + 3 * m], xm(P[i + 3 * n], C.b[n + 3 * m]));
#pragma unroll
        for (int m = 0; m < 3; ++m)
#pragma unroll
            for (int i = 0; i < 3; ++i) f[i] = xs(f[i], xm(P[i + 3 * m], C.fb[m]));
#pragma unroll
        for (int e = 0; e < 9; ++e) P[e] = 0.0;
    } else if (k == nk - 2) {
        // upper boundary with the He escape flux (comp_ng.F90:259-279)
#pragma unroll
        for (int m = 0; m < 3; ++m) {
            const double h = xm(xm(0.5, Lp.ep[m]), dz);
            const double ratio = xd(xa(1.0, h), xs(1.0, h));
#pragma unroll
            for (int i = 0; i < 3; ++i) Q[i + 3 * m] = xa(Q[i + 3 * m], xm(ratio, R[i + 3 * m]));
        }
        // embari and tn of level k (k = nk-2 >= 1)
        const double embari_k = xm(0.5, xa(at(F.mbar, k - 1), at(F.mbar, k)));
        flx00 = xd(xm(xm(xm(embari_k, C.rmassinv_n2), C.p0), pow(xd(t00, at(F.tn, k)), 0.25)), xm(tau, C.grav));
        const double d2 = xm(flx00, xs(rdz, xm(0.5, Lp.ep[1]))), d3 = xm(flx00, xs(rdz, xm(0.5, Lp.ep[2])));
#pragma unroll
        for (int i = 0; i < 3; ++i)
            f[i] = xs(xs(f[i], xd(xm(xm(R[i + 3], xs(Lp.a23, Lp.a22)), flx_he), d2)),
                      xd(xm(xm(R[i + 6], xs(Lp.a33, Lp.a32)), flx_he), d3));
#pragma unroll
        for (int e = 0; e < 9; ++e) R[e] = 0.0;
    }
}

// The block forward step of row k (comp_ng.F90:280-314): Q' = Q - P Gamma_k,
// W = Q'^-1, z_(k+1) = W (f - P z_k), Gamma_(k+1) = W R, the last two into the
// scratch rows of level k+1.
__device__ __forceinline__ void comp_forward(const double (&P)[9], double (&Q)[9], const double (&R)[9],
                                             const double (&f)[3], int k, int nk, long ld, long col, double *scr,
                                             double (&G)[9], double (&z)[3], bool &ok)
{
    double W[9], v[3];
    if (k > 0) {
#pragma unroll
        for (int m = 0; m < 3; ++m)
#pragma unroll
            for (int n = 0; n < 3; ++n)
#pragma unroll
                for (int i = 0; i < 3; ++i) Q[i + 3 * m] = xs(Q[i + 3 * m], xm(P[i + 3 * n], G[n + 3 * m]));
    }
    inv3_ieee(Q, W);
#pragma unroll
    for (int e = 0; e < 9; ++e) ok = ok && fabs(W[e]) <= DBL_MAX;
#pragma unroll
    for (int i = 0; i < 3; ++i) v[i] = f[i];
    if (k > 0) {
#pragma unroll
        for (int m = 0; m < 3; ++m)
#pragma unroll
            for (int i = 0; i < 3; ++i) v[i] = xs(v[i], xm(P[i + 3 * m], z[m]));
    }
#pragma unroll
    for (int i = 0; i < 3; ++i) z[i] = xa(xa(xm(W[i], v[0]), xm(W[i + 3], v[1])), xm(W[i + 6], v[2]));
    if (k < nk - 2) {
#pragma unroll
        for (int m = 0; m < 3; ++m)
#pragma unroll
            for (int i = 0; i < 3; ++i)
                G[i + 3 * m] = xa(xa(xm(W[i], R[3 * m]), xm(W[i + 3], R[1 + 3 * m])), xm(W[i + 6], R[2 + 3 * m]));
        double *sg = scr + (long)(k + 1) * 12 * ld + col;
#pragma unroll
        for (int e = 0; e < 9; ++e) sg[(long)e * ld] = G[e];
#pragma unroll
        for (int i = 0; i < 3; ++i) sg[(long)(9 + i) * ld] = z[i];
    }
}

// The back sweep (comp_ng.F90:317-324) from the scratch rows, the top level
// with the He escape flux (:326-332) and calc_helium = 0's fixed He.
// One level of the back sweep: x(k) = z(k+1) - Gamma(k+1) x(k+1), stored.
__device__ __forceinline__ void comp_back_level(const double (&g)[9], const double (&zk)[3], double (&x)[3], bool &fin,
                                                double *out, long slab, long o)
{
    double xn[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) xn[i] = xs(xs(xs(zk[i], xm(g[i], x[0])), xm(g[i + 3], x[1])), xm(g[i + 6], x[2]));
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        x[i] = xn[i];
        fin = fin && fabs(x[i]) <= DBL_MAX;
        out[(long)i * slab + o] = x[i];
    }
}

// The top level (comp_ng.F90:326-332) from xb = x(nk-2), calc_helium = 0's
// fixed He, and the status.
__device__ __forceinline__ void comp_top(const CompConsts &C, const CompLevel &Lp, double flx00, double flx_he,
                                         const double (&xb)[3], bool ok, bool fin, double *out, int nk, long ld,
                                         long col, unsigned *status)
{
    const long slab = (long)nk * ld;
    const double dz = C.dz, rdz = xd(1.0, dz);
    double top[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        const double h = xm(xm(0.5, Lp.ep[i]), dz);
        top[i] = xm(xd(xa(1.0, h), xs(1.0, h)), xb[i]);
    }
    top[1] = xa(top[1], xd(xm(xs(Lp.a23, Lp.a22), flx_he), xm(flx00, xs(rdz, xm(0.5, Lp.ep[1])))));
    top[2] = xa(top[2], xd(xm(xs(Lp.a33, Lp.a32), flx_he), xm(flx00, xs(rdz, xm(0.5, Lp.ep[2])))));
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        fin = fin && fabs(top[i]) <= DBL_MAX;
        out[(long)i * slab + (long)(nk - 1) * ld + col] = top[i];
    }
    if (!C.calc_helium)
        for (int k = 0; k < nk; ++k) out[2 * slab + (long)k * ld + col] = C.pshelb;
    if (!ok || !fin) atomicOr(status, (ok ? 0u : FLAG_PIVOT) | (fin ? 0u : FLAG_NONFINITE));
}

__device__ __forceinline__ void comp_back(const CompConsts &C, const CompLevel &Lp, double flx00, double flx_he,
                                          const double (&z)[3], bool ok, double *out, const double *scr, int nk,
                                          long ld, long col, unsigned *status, int pd)
{
    const long slab = (long)nk * ld;
    // back sweep (comp_ng.F90:317-324); x(nk-1) = z_{nk-1}
    bool fin = true;
    double x[3], xb[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        x[i] = z[i];
        xb[i] = z[i];
        out[(long)i * slab + (long)(nk - 2) * ld + col] = x[i];
        fin = fin && fabs(x[i]) <= DBL_MAX;
    }
    // the Gamma/z rows of level kk+1, requested pd levels ahead of their use
    auto pf_gz = [&](int kk) {
        const double *sg = scr + (long)(kk + 1) * 12 * ld + col;
#pragma unroll
        for (int e = 0; e < 12; ++e) pf_l1(sg + (long)e * ld);
    };
    for (int kk = nk - 4; kk > nk - 3 - pd && kk >= 0; --kk) pf_gz(kk);
    for (int k = nk - 3; k >= 0; --k) {
        if (k - pd >= 0) pf_gz(k - pd);
        const double *sg = scr + (long)(k + 1) * 12 * ld + col;
        double g[9], zk[3];
#pragma unroll
        for (int e = 0; e < 9; ++e) g[e] = sg[(long)e * ld];
#pragma unroll
        for (int i = 0; i < 3; ++i) zk[i] = sg[(long)(9 + i) * ld];
        comp_back_level(g, zk, x, fin, out, slab, (long)k * ld + col);
    }
    comp_top(C, Lp, flx00, flx_he, xb, ok, fin, out, nk, ld, col, status);
}

// One column of comp_ng's rows and block solve (comp_ng.F90:170-332).  The
// level quantities (ep, ak, wks4 and, at the top, the alpha entries of the
// He-flux condition) come from Src: computed on the fly from the fields
// (CompFusedSrc) or read from planes a level-parallel kernel wrote
// (CompPlaneSrc).  first(L) gives level 0, next(k, L) level k+1, in order.
template <class Src>
__device__ __forceinline__ void comp_walk(const CompFields &F, const CompConsts &C, Src &src, double *out,
                                          double *scr, int nk, long ld, long col, double *sys_out, unsigned *status,
                                          int pd = 1)
{
    const long slab = (long)nk * ld;
    const double dfac = __ldg(F.dfactor + col);
    const double flx_he = C.calc_helium ? __ldg(F.flx_he + col) : 0.0;
    CompLevel Lk, Lp;
    src.first(Lp);
    double G[9], z[3];
#pragma unroll
    for (int e = 0; e < 9; ++e) G[e] = 0.0;
#pragma unroll
    for (int i = 0; i < 3; ++i) z[i] = 0.0;
    bool ok = true;
    double flx00 = 1.0;
    for (int k = 0; k < nk - 1; ++k) {
        src.begin(k);
        Lk = Lp;
        src.next(k, Lp);
        double P[9], Q[9], R[9], f[3];
        comp_row(F, C, src, Lk, Lp, k, nk, ld, col, dfac, flx_he, P, Q, R, f, flx00);
        if (sys_out) {
            double *so = sys_out + (long)k * ld + col;
#pragma unroll
            for (int e = 0; e < 9; ++e) {
                so[(long)e * slab] = P[e];
                so[(long)(9 + e) * slab] = Q[e];
                so[(long)(18 + e) * slab] = R[e];
            }
#pragma unroll
            for (int i = 0; i < 3; ++i) so[(long)(27 + i) * slab] = f[i];
        }
        comp_forward(P, Q, R, f, k, nk, ld, col, scr, G, z, ok);
    }
    comp_back(C, Lp, flx00, flx_he, z, ok, out, scr, nk, ld, col, status, pd);
}

// Per-level field reads of comp_walk straight from global memory.
struct CompFieldReads {
    const CompFields &F;
    long ld, col;
    int nk;
    __device__ __forceinline__ double fat(const double *p, int k) const { return __ldg(p + k * ld + col); }
    __device__ __forceinline__ void begin(int) {}
    __device__ __forceinline__ double w(int k) const { return fat(F.w, k); }
    __device__ __forceinline__ double w1(int k) const { return fat(F.w, k + 1); }
    __device__ __forceinline__ double fs(int r, int k) const { return fat(F.fs + (long)r * nk * ld, k); }
    __device__ __forceinline__ double nms(int i, int k) const
    {
        return fat(i == 0 ? F.o2nm_smooth : i == 1 ? F.o1nm_smooth : F.henm_smooth, k);
    }
    __device__ __forceinline__ double adv(int i, int k) const
    {
        return fat(i == 0 ? F.o2_advec : i == 1 ? F.o1_advec : F.he_advec, k);
    }
    __device__ __forceinline__ double hd(int i, int k) const { return fat(i == 0 ? F.hdo2 : i == 1 ? F.hdo1 : F.hdhe, k); }
};

// Level quantities computed from the fields with a window of two levels.
struct CompFusedSrc : CompFieldReads {
    const CompConsts &C;
    double o2_0, o1_0, he_0, mb_0, tn_0;
    __device__ __forceinline__ double at(const double *p, int k) const { return __ldg(p + k * ld + col); }
    __device__ __forceinline__ void first(CompLevel &L)
    {
        // lower-boundary mixing ratios and level 1 (comp_ng.F90:74-96, 128-166)
        const double dz = C.dz, tlbc = __ldg(F.tlbc + col);
        o2_0 = at(F.o2, 0);
        o1_0 = at(F.o1, 0);
        he_0 = at(F.he, 0);
        mb_0 = at(F.mbar, 0);
        tn_0 = at(F.tn, 0);
        double ps0[3];
#pragma unroll
        for (int i = 0; i < 3; ++i)
            ps0[i] = xa(xa(xa(xm(C.b[i], o2_0), xm(C.b[i + 3], o1_0)), xm(C.b[i + 6], he_0)), C.fb[i]);
        const double embar0 =
            xd(1.0, xa(xa(xa(xm(ps0[0], C.rmassinv_o2), xm(ps0[1], C.rmassinv_o1)), xm(ps0[2], C.rmassinv_he)),
                       xm(xs(xs(xs(1.0, ps0[0]), ps0[1]), ps0[2]), C.rmassinv_n2)));
        comp_level(C, xm(0.5, xa(ps0[0], o2_0)), xm(0.5, xa(ps0[1], o1_0)), xm(0.5, xa(ps0[2], he_0)),
                   xm(0.5, xa(embar0, mb_0)), tlbc, xd(xs(mb_0, embar0), dz), xd(xm(xs(tn_0, tlbc), 2.0), dz), true, L);
    }
    __device__ __forceinline__ void next(int k, CompLevel &L)
    {
        const double dz = C.dz;
        const double o2_1 = at(F.o2, k + 1), o1_1 = at(F.o1, k + 1), he_1 = at(F.he, k + 1), mb_1 = at(F.mbar, k + 1),
                     tn_1 = at(F.tn, k + 1);
        comp_level(C, xm(0.5, xa(o2_0, o2_1)), xm(0.5, xa(o1_0, o1_1)), xm(0.5, xa(he_0, he_1)),
                   xm(0.5, xa(mb_0, mb_1)), xm(0.5, xa(tn_0, tn_1)), xd(xs(mb_1, mb_0), dz), xd(xs(tn_1, tn_0), dz),
                   k + 1 != nk - 1, L);
        o2_0 = o2_1;
        o1_0 = o1_1;
        he_0 = he_1;
        mb_0 = mb_1;
        tn_0 = tn_1;
    }
};

__global__ void __launch_bounds__(128) k_comp_ng(CompFields F, CompConsts C, double *out, double *scr, int nk, int ncol,
                                                 long ld, double *sys_out, unsigned *status)
{
    const long col = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (col >= ncol) return;
    CompFusedSrc src{{F, ld, col, nk}, C};
    comp_walk(F, C, src, out, scr, nk, ld, col, sys_out, status);
}

// Planes of the level-parallel pass: ep (3), ak (9), wks4 at (e*nk + j)*ld +
// col; the top level's a22, a33, a23, a32 in 4 rows of ld after them.
constexpr int kCompPlanes = 13;

__global__ void __launch_bounds__(128) k_comp_levels(CompFields F, CompConsts C, double *lv, int nk, int ncol, long ld)
{
    const long col = (long)blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y;
    if (col >= ncol) return;
    CompLevel L;
    if (j == 0) {
        CompFusedSrc src{{F, ld, col, nk}, C};
        src.first(L);
    } else {
        auto at = [&](const double *p, int k) { return __ldg(p + k * ld + col); };
        const double dz = C.dz;
        const double mb0 = at(F.mbar, j - 1), mb1 = at(F.mbar, j), tn0 = at(F.tn, j - 1), tn1 = at(F.tn, j);
        comp_level(C, xm(0.5, xa(at(F.o2, j - 1), at(F.o2, j))), xm(0.5, xa(at(F.o1, j - 1), at(F.o1, j))),
                   xm(0.5, xa(at(F.he, j - 1), at(F.he, j))), xm(0.5, xa(mb0, mb1)), xm(0.5, xa(tn0, tn1)),
                   xd(xs(mb1, mb0), dz), xd(xs(tn1, tn0), dz), j != nk - 1, L);
    }
    const long slab = (long)nk * ld, o = (long)j * ld + col;
#pragma unroll
    for (int i = 0; i < 3; ++i) lv[i * slab + o] = L.ep[i];
#pragma unroll
    for (int e = 0; e < 9; ++e) lv[(3 + e) * slab + o] = L.ak[e];
    lv[12 * slab + o] = L.wks4;
    if (j == nk - 1) {
        double *top = lv + kCompPlanes * slab;
        top[col] = L.a22;
        top[ld + col] = L.a33;
        top[2 * ld + col] = L.a23;
        top[3 * ld + col] = L.a32;
    }
}

// Level quantities read back from the planes.
struct CompPlaneSrc : CompFieldReads {
    const double *lv;
    __device__ __forceinline__ void load(int j, CompLevel &L) const
    {
        const long slab = (long)nk * ld, o = (long)j * ld + col;
#pragma unroll
        for (int i = 0; i < 3; ++i) L.ep[i] = __ldg(lv + i * slab + o);
#pragma unroll
        for (int e = 0; e < 9; ++e) L.ak[e] = __ldg(lv + (3 + e) * slab + o);
        L.wks4 = __ldg(lv + 12 * slab + o);
        if (j == nk - 1) {
            const double *top = lv + kCompPlanes * slab;
            L.a22 = __ldg(top + col);
            L.a33 = __ldg(top + ld + col);
            L.a23 = __ldg(top + 2 * ld + col);
            L.a32 = __ldg(top + 3 * ld + col);
        } else {
            L.a22 = L.a33 = L.a23 = L.a32 = 0.0;
        }
    }
    __device__ __forceinline__ void first(CompLevel &L) { load(0, L); }
    __device__ __forceinline__ void next(int k, CompLevel &L) { load(k + 1, L); }
};

// The plane source with every per-level read of the walk staged one
// iteration ahead: while iteration k computes, asynchronous 8-byte copies
// bring the 36 values iteration k+1 reads (the 13 planes of level k+2, w at
// k+1 and k+2, the 12 fs rows, nm, advec and hd of the three species at k+1)
// into a two-buffer shared-memory array [buffer][value][thread].  Each thread
// reads only what it copied itself, so no block barrier is needed.
struct CompStagedSrc : CompPlaneSrc {
    static constexpr int NS = 36;
    double *sm;   // this thread's column of the block's slot array
    int T;        // threads per block (row stride of the slot array)
    int cur;
    int pd;       // levels ahead whose reads are requested into L1
    __device__ __forceinline__ double &slot(int b, int v) const { return sm[(long)(b * NS + v) * T]; }
    __device__ __forceinline__ void issue(int k, int b)
    {
        const long slab = (long)nk * ld, o = (long)k * ld + col;
#pragma unroll
        for (int v = 0; v < kCompPlanes; ++v) cp_async8(&slot(b, v), lv + v * slab + o + ld);
        cp_async8(&slot(b, 13), F.w + o);
        cp_async8(&slot(b, 14), F.w + o + ld);
#pragma unroll
        for (int r = 0; r < 12; ++r) cp_async8(&slot(b, 15 + r), F.fs + r * slab + o);
        cp_async8(&slot(b, 27), F.o2nm_smooth + o);
        cp_async8(&slot(b, 28), F.o1nm_smooth + o);
        cp_async8(&slot(b, 29), F.henm_smooth + o);
        cp_async8(&slot(b, 30), F.o2_advec + o);
        cp_async8(&slot(b, 31), F.o1_advec + o);
        cp_async8(&slot(b, 32), F.he_advec + o);
        cp_async8(&slot(b, 33), F.hdo2 + o);
        cp_async8(&slot(b, 34), F.hdo1 + o);
        cp_async8(&slot(b, 35), F.hdhe + o);
    }
    // the lines issue(k) copies, requested into L1 ahead of the copies
    __device__ __forceinline__ void prefetch(int k) const
    {
        const long slab = (long)nk * ld, o = (long)k * ld + col;
#pragma unroll
        for (int v = 0; v < kCompPlanes; ++v) pf_l1(lv + v * slab + o + ld);
        pf_l1(F.w + o);
        pf_l1(F.w + o + ld);
#pragma unroll
        for (int r = 0; r < 12; ++r) pf_l1(F.fs + r * slab + o);
        pf_l1(F.o2nm_smooth + o);
        pf_l1(F.o1nm_smooth + o);
        pf_l1(F.henm_smooth + o);
        pf_l1(F.o2_advec + o);
        pf_l1(F.o1_advec + o);
        pf_l1(F.he_advec + o);
        pf_l1(F.hdo2 + o);
        pf_l1(F.hdo1 + o);
        pf_l1(F.hdhe + o);
    }
    __device__ __forceinline__ void first(CompLevel &L)
    {
        load(0, L);
        issue(0, 0);
        cp_async_commit();
        for (int kk = 2; kk < pd + 1 && kk < nk - 1; ++kk) prefetch(kk);
    }
    // iteration k: start the copies of iteration k+1, wait for those of k
    __device__ __forceinline__ void begin(int k)
    {
        if (k + 1 + pd < nk - 1 && pd > 1) prefetch(k + 1 + pd);
        if (k + 1 < nk - 1) issue(k + 1, (k + 1) & 1);
        cp_async_commit();
        cp_async_wait<1>();
        cur = k & 1;
    }
    __device__ __forceinline__ void next(int k, CompLevel &L) const
    {
#pragma unroll
        for (int i = 0; i < 3; ++i) L.ep[i] = slot(cur, i);
#pragma unroll
        for (int e = 0; e < 9; ++e) L.ak[e] = slot(cur, 3 + e);
        L.wks4 = slot(cur, 12);
        if (k + 1 == nk - 1) {
            const double *top = lv + kCompPlanes * (long)nk * ld;
            L.a22 = __ldg(top + col);
            L.a33 = __ldg(top + ld + col);
            L.a23 = __ldg(top + 2 * ld + col);
            L.a32 = __ldg(top + 3 * ld + col);
        } else {
            L.a22 = L.a33 = L.a23 = L.a32 = 0.0;
        }
    }
    __device__ __forceinline__ double w(int) const { return slot(cur, 13); }
    __device__ __forceinline__ double w1(int) const { return slot(cur, 14); }
    __device__ __forceinline__ double fs(int r, int) const { return slot(cur, 15 + r); }
    __device__ __forceinline__ double nms(int i, int) const { return slot(cur, 27 + i); }
    __device__ __forceinline__ double adv(int i, int) const { return slot(cur, 30 + i); }
    __device__ __forceinline__ double hd(int i, int) const { return slot(cur, 33 + i); }
};

constexpr int kCompRowThreads = 64;

__global__ void __launch_bounds__(kCompRowThreads, 5) k_comp_rows(CompFields F, CompConsts C, const double *lv,
                                                               double *out, double *scr, int nk, int ncol, long ld,
                                                               double *sys_out, unsigned *status, int pd)
{
    extern __shared__ double comp_slots[];
    const long col = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (col >= ncol) return;
    CompStagedSrc src{{{F, ld, col, nk}, lv}, comp_slots + threadIdx.x, (int)blockDim.x, 0, pd};
    comp_walk(F, C, src, out, scr, nk, ld, col, sys_out, status, pd);
}

// Three-pass form, pass 2: row k of every column, one thread per (row,
// column), into 30 row planes (P, Q, R by entry i + 3m, then f); the top row
// also leaves flx00 in its column's slot.
__global__ void __launch_bounds__(128) k_comp_coefs(CompFields F, CompConsts C, const double *lv, double *rows,
                                                    double *flx00_row, int nk, int ncol, long ld, double *sys_out)
{
    const long col = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (col >= ncol) return;
    const int k = blockIdx.y;
    const long slab = (long)nk * ld, o = (long)k * ld + col;
    CompPlaneSrc src{{F, ld, col, nk}, lv};
    CompLevel Lk, Lp;
    src.load(k, Lk);
    src.load(k + 1, Lp);
    double P[9], Q[9], R[9], f[3], flx00 = 1.0;
    comp_row(F, C, src, Lk, Lp, k, nk, ld, col, __ldg(F.dfactor + col),
             C.calc_helium ? __ldg(F.flx_he + col) : 0.0, P, Q, R, f, flx00);
#pragma unroll
    for (int e = 0; e < 9; ++e) {
        rows[(long)e * slab + o] = P[e];
        rows[(long)(9 + e) * slab + o] = Q[e];
        rows[(long)(18 + e) * slab + o] = R[e];
    }
#pragma unroll
    for (int i = 0; i < 3; ++i) rows[(long)(27 + i) * slab + o] = f[i];
    if (k == nk - 2) flx00_row[col] = flx00;
    if (sys_out) {
        double *so = sys_out + o;
#pragma unroll
        for (int e = 0; e < 9; ++e) {
            so[(long)e * slab] = P[e];
            so[(long)(9 + e) * slab] = Q[e];
            so[(long)(18 + e) * slab] = R[e];
        }
#pragma unroll
        for (int i = 0; i < 3; ++i) so[(long)(27 + i) * slab] = f[i];
    }
}

// Three-pass form, pass 3: the block recurrence over the row planes, on a
// 16-column tile per block of kCompTileWarps warps.  The 30 row planes
// stream through a two-buffer shared-memory ring, kCompChunk levels per
// buffer: all warps copy the next
// chunk (cp.async) while warp 0 runs the recurrence over this one.  Gamma
// and z of every level go to the global scratch (L2) and come back through
// the same ring, top down, for the back sweep.  Same arithmetic
// (comp_forward, comp_back_level, comp_top), same bits.
constexpr int kCompTileCols = 16, kCompChunk = 8, kCompTileWarps = 4;
constexpr size_t kCompTileBytes = sizeof(double) * 2 * kCompChunk * 30 * kCompTileCols;
__global__ void __launch_bounds__(32 * kCompTileWarps) k_comp_walk_tile(CompFields F, CompConsts C, const double *lv,
                                                                        const double *rows, const double *flx00_row,
                                                                        double *out, double *scr, int nk, int ncol,
                                                                        long ld, unsigned *status)
{
    extern __shared__ double comp_tile[];
    constexpr int TC = kCompTileCols, L = kCompChunk, NT = 32 * kCompTileWarps;
    double *ring = comp_tile;
    const int tid = threadIdx.x, w = tid >> 5, lane = tid & 31;
    const long col0 = (long)blockIdx.x * TC, col = col0 + lane;
    const long slab = (long)nk * ld;
    const int K = nk - 1, nch = (K + L - 1) / L;
    // chunk c (levels c*L .. c*L+L-1 below K) into buffer c & 1, laid out
    // [level][plane][column]
    auto load = [&](int c) {
        const int k0 = c * L, nl = K - k0 < L ? K - k0 : L;
        double *buf = ring + (c & 1) * L * 30 * TC;
        for (int i = tid; i < nl * 30 * TC; i += NT) {
            const int j = i % TC, lv30 = i / TC, l = lv30 / 30, v = lv30 - 30 * l;
            if (col0 + j < ncol) cp_async8(buf + i, rows + (long)v * slab + (long)(k0 + l) * ld + col0 + j);
        }
        cp_async_commit();
    };
    const bool walker = w == 0 && lane < TC && col < ncol;
    double G[9], z[3];
#pragma unroll
    for (int e = 0; e < 9; ++e) G[e] = 0.0;
#pragma unroll
    for (int i = 0; i < 3; ++i) z[i] = 0.0;
    bool ok = true;
    load(0);
    for (int c = 0; c < nch; ++c) {
        if (c + 1 < nch) load(c + 1);
        else cp_async_commit();
        cp_async_wait<1>();
        __syncthreads();
        if (walker) {
            const double *buf = ring + (c & 1) * L * 30 * TC + lane;
            const int k0 = c * L, nl = K - k0 < L ? K - k0 : L;
            for (int l = 0; l < nl; ++l) {
                const double *r = buf + l * 30 * TC;
                double P[9], Q[9], R[9], f[3];
#pragma unroll
                for (int e = 0; e < 9; ++e) {
                    P[e] = r[e * TC];
                    Q[e] = r[(9 + e) * TC];
                    R[e] = r[(18 + e) * TC];
                }
#pragma unroll
                for (int i = 0; i < 3; ++i) f[i] = r[(27 + i) * TC];
                comp_forward(P, Q, R, f, k0 + l, nk, ld, col, scr, G, z, ok);
            }
        }
        __syncthreads();
    }
    // back sweep (comp_ng.F90:317-324): level k from the Gamma/z row k+1,
    // k = nk-3 .. 0, chunk d holding levels kh(d) - l, l < L
    const int KB = nk - 2, nb = (KB + L - 1) / L;
    auto load_b = [&](int d) {
        const int kh = nk - 3 - d * L, nl = KB - d * L < L ? KB - d * L : L;
        double *buf = ring + (d & 1) * L * 30 * TC;
        for (int i = tid; i < nl * 12 * TC; i += NT) {
            const int j = i % TC, le = i / TC, l = le / 12, e = le - 12 * l;
            if (col0 + j < ncol) cp_async8(buf + i, scr + (long)(kh - l + 1) * 12 * ld + (long)e * ld + col0 + j);
        }
        cp_async_commit();
    };
    bool fin = true;
    double x[3], xb[3];
    if (walker)
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            x[i] = xb[i] = z[i];
            out[(long)i * slab + (long)(nk - 2) * ld + col] = x[i];
            fin = fin && fabs(x[i]) <= DBL_MAX;
        }
    load_b(0);
    for (int d = 0; d < nb; ++d) {
        if (d + 1 < nb) load_b(d + 1);
        else cp_async_commit();
        cp_async_wait<1>();
        __syncthreads();
        if (walker) {
            const double *buf = ring + (d & 1) * L * 30 * TC + lane;
            const int kh = nk - 3 - d * L, nl = KB - d * L < L ? KB - d * L : L;
            for (int l = 0; l < nl; ++l) {
                double g[9], zk[3];
#pragma unroll
                for (int e = 0; e < 9; ++e) g[e] = buf[(l * 12 + e) * TC];
#pragma unroll
                for (int i = 0; i < 3; ++i) zk[i] = buf[(l * 12 + 9 + i) * TC];
                comp_back_level(g, zk, x, fin, out, slab, (long)(kh - l) * ld + col);
            }
        }
        __syncthreads();
    }
    if (!walker) return;
    CompPlaneSrc src{{F, ld, col, nk}, lv};
    CompLevel Lp;
    src.load(nk - 1, Lp);
    comp_top(C, Lp, flx00_row[col], C.calc_helium ? __ldg(F.flx_he + col) : 0.0, xb, ok, fin, out, nk, ld, col,
             status);
}

// ---------------------------------------------------------------------------
// comp_ng's history diagnostics (src/comp_ng.F90:334-380) from the fields and
// the solution x (three level-major planes O2, O, He, before the lateral
// overwrite and the post steps): 24 planes in the order of the addfld calls,
// D<sp>DT, <sp>_PROD, _LOSS, _HORDIF, _MOLDIF, _EDDYDIF, -_VERADV, -_HORADV
// for sp = O2, O1, HE.  loss and moldif are summed over their fourth index,
// the row's species, from 0 (sum(..., dim=4)); MOLDIF, EDDYDIF and VERADV,
// which the reference leaves unset on the first and top levels, are 0 there.
// One thread per (level, column); ep, ak and wks4 of levels k and k+1 from
// the planes k_comp_levels wrote (its fractional powers within a few ulp of
// the host library's: MOLDIF and EDDYDIF to a tolerance), everything else
// bit-identical.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(128) k_comp_diag_ng(CompFields F, CompConsts C, const double *lv, const double *x,
                                                      int nk, int ncol, long ld, double *diag)
{
    const long col = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (col >= ncol) return;
    const int k = blockIdx.y;
    const long slab = (long)nk * ld, o = (long)k * ld + col;
    const double dz = C.dz, rdz = xd(1.0, dz);
    auto X = [&](int i, int kk) { return __ldg(x + i * slab + (long)kk * ld + col); };
    auto D = [&](int n) -> double & { return diag[(long)n * slab + o]; };
    const double *nms[3] = {F.o2nm_smooth, F.o1nm_smooth, F.henm_smooth};
    const double *adv[3] = {F.o2_advec, F.o1_advec, F.he_advec};
    const double *hd[3] = {F.hdo2, F.hdo1, F.hdhe};
    double xk[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        xk[i] = X(i, k);
        D(i) = xm(C.dtx2inv, xs(xk[i], __ldg(nms[i] + o)));
        D(3 + i) = __ldg(F.fs + (long)i * slab + o);
        D(9 + i) = __ldg(hd[i] + o);
        D(21 + i) = -__ldg(adv[i] + o);
    }
#pragma unroll
    for (int m = 0; m < 3; ++m) {
        double s = 0.0;
#pragma unroll
        for (int i = 0; i < 3; ++i) s = xa(s, xm(__ldg(F.fs + (long)((m + 1) * 3 + i) * slab + o), xk[m]));
        D(6 + m) = s;
    }
    if (k == 0 || k == nk - 1) {
#pragma unroll
        for (int i = 0; i < 3; ++i) D(12 + i) = D(15 + i) = D(18 + i) = 0.0;
        return;
    }
    CompPlaneSrc src{{F, ld, col, nk}, lv};
    CompLevel Lk, Lp;
    src.load(k, Lk);
    src.load(k + 1, Lp);
    const double difk0 = __ldg(F.difk + k), difk1 = __ldg(F.difk + k + 1);
    const double eddyp = xm(xm(C.expzmid_inv, difk0), xs(rdz, Lk.wks4));
    const double eddyr = xm(xm(C.expzmid, difk1), xa(rdz, Lp.wks4));
    const double eddyq =
        xa(xm(xm(C.expzmid_inv, difk0), xa(rdz, Lk.wks4)), xm(xm(C.expzmid, difk1), xs(rdz, Lp.wks4)));
    const double emd = xd(xd(1.0, __ldg(F.expz + k)), dz);
    double xm1[3], xp1[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        xm1[i] = X(i, k - 1);
        xp1[i] = X(i, k + 1);
    }
#pragma unroll
    for (int m = 0; m < 3; ++m) {
        const double hk = xd(Lk.ep[m], 2.0), hp = xd(Lp.ep[m], 2.0);
        double s = 0.0;
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            const int e = i + 3 * m;
            const double molp = xm(Lk.ak[e], xa(rdz, hk));
            const double molr = xm(Lp.ak[e], xs(rdz, hp));
            const double molq = xa(xm(Lk.ak[e], xs(rdz, hk)), xm(Lp.ak[e], xa(rdz, hp)));
            s = xa(s, -xm(emd, xa(xs(xm(molp, xm1[m]), xm(molq, xk[m])), xm(molr, xp1[m]))));
        }
        D(12 + m) = s;
    }
    const double dfac = __ldg(F.dfactor + col);
    const double wi = xm(0.5, xa(__ldg(F.w + o), __ldg(F.w + o + ld)));
    const double wdz = xd(wi, xm(2.0, dz));
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        D(15 + i) = xm(xm(rdz, xa(xs(xm(eddyp, xm1[i]), xm(eddyq, xk[i])), xm(eddyr, xp1[i]))), dfac);
        D(18 + i) = -xm(wdz, xs(xp1[i], xm1[i]));
    }
}

cudaError_t launch_comp_diag_ng(const CompFields &F, const CompConsts &C, const double *x, int nk, int ncol, long ld,
                                double *diag, double *scratch, cudaStream_t st)
{
    if (ncol <= 0) return cudaSuccess;
    if (nk < 3) return cudaErrorInvalidValue;
    const int T = 128;
    double *lv = scratch + 12 * (long)nk * ld;
    k_comp_levels<<<dim3((ncol + T - 1) / T, nk), T, 0, st>>>(F, C, lv, nk, ncol, ld);
    k_comp_diag_ng<<<dim3((ncol + T - 1) / T, nk), T, 0, st>>>(F, C, lv, x, nk, ncol, ld, diag);
    return cudaGetLastError();
}

cudaError_t launch_comp_ng(const CompFields &F, const CompConsts &C, double *out, double *scratch, int nk, int ncol,
                           long ld, double *sys_out, unsigned *status, cudaStream_t st)
{
    if (ncol <= 0) return cudaSuccess;
    if (nk < 3) return cudaErrorInvalidValue;
    const int T = 128;
    // the 30 row planes cost more traffic than they save above a few thousand
    // columns per SM-wave (41472 columns: 625 against 449 us)
    if (assembly_mode() == 2 && ncol <= kSmallWalkColumns) {
        const long slab = (long)nk * ld;
        double *lv = scratch + 12 * slab;                   // after the Gamma/z scratch
        double *flx00_row = lv + kCompPlanes * slab + 4 * ld;
        double *rows = flx00_row + ld;
        k_comp_levels<<<dim3((ncol + T - 1) / T, nk), T, 0, st>>>(F, C, lv, nk, ncol, ld);
        k_comp_coefs<<<dim3((ncol + T - 1) / T, nk - 1), T, 0, st>>>(F, C, lv, rows, flx00_row, nk, ncol, ld, sys_out);
        once_per_device([] {
            cudaFuncSetAttribute(k_comp_walk_tile, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kCompTileBytes);
        });
        k_comp_walk_tile<<<(ncol + kCompTileCols - 1) / kCompTileCols, 32 * kCompTileWarps, kCompTileBytes, st>>>(
            F, C, lv, rows, flx00_row, out, scratch, nk, ncol, ld, status);
        return cudaGetLastError();
    }
    if (assembly_mode() >= 1) {
        double *lv = scratch + 12 * (long)nk * ld;   // after the Gamma/z scratch
        k_comp_levels<<<dim3((ncol + T - 1) / T, nk), T, 0, st>>>(F, C, lv, nk, ncol, ld);
        const int TR = kCompRowThreads;
        k_comp_rows<<<(ncol + TR - 1) / TR, TR, 2 * CompStagedSrc::NS * TR * sizeof(double), st>>>(
            F, C, lv, out, scratch, nk, ncol, ld, sys_out, status, walk_prefetch(ncol));
        return cudaGetLastError();
    }
    k_comp_ng<<<(ncol + T - 1) / T, T, 0, st>>>(F, C, out, scratch, nk, ncol, ld, sys_out, status);
    return cudaGetLastError();
}

// Gamma/z (12 planes), the level planes and their 4 top rows, then (three-pass
// form) the flx00 row and the 30 row planes
size_t comp_scratch_doubles(int nk, long ld) { return (size_t)(12 + kCompPlanes + 30) * nk * ld + 5 * (size_t)ld; }
}  // namespace tg

// comp_ng post-solve steps (src/comp_ng.F90:394-457): the lateral-boundary
// overwrite of the columns flagged in bmask (when given), the time filter,
// the N2 extrapolation, floors and normalisation.  A block takes 32 columns
// with sixteen warps (about four levels each, so that few-column launches
// do not wait on a long run of levels per warp); a warp works on the 32
// columns of one level at a time, so
// every phase runs over all levels at once: the overwrite, the search for the
// first level with N2 < 0.01 (the least level any warp finds), the
// extrapolation constants (one thread per column), then the per-level steps.
// The N2 extrapolation uses the device log/exp, so it agrees with the CPU
// restatement to a tolerance in the extrapolated levels.
namespace tg {
constexpr int kPostCols = 32, kPostWarps = 16;

__global__ void __launch_bounds__(kPostCols * kPostWarps) k_comp_post_ng(
    const double *o2, const double *o1, const double *he, const double *o2_nm, const double *o1_nm,
    const double *he_nm, const double *xnmbar, const double *zpmid, double dz, double ds, double ds2, int nk, int ncol,
    long ld, double *o2u, double *o1u, double *heu, double *o2n, double *o1n, double *hen, const unsigned char *bmask,
    const double *b2, const double *b1, const double *bh)
{
    __shared__ int ktop_s[kPostCols];
    __shared__ double n2top_s[kPostCols], dn2dz_s[kPostCols], zmtop_s[kPostCols];
    const int c = threadIdx.x % kPostCols, w = threadIdx.x / kPostCols;
    const long col = (long)blockIdx.x * kPostCols + c;
    const bool live = col < ncol;
    const double small = 1.e-9;
    if (w == 0) ktop_s[c] = nk;
    // the Dirichlet lateral-boundary hook (comp_ng.F90:394-413)
    if (live && bmask && bmask[col])
        for (int k = w; k < nk; k += kPostWarps) {
            const long o = (long)k * ld + col;
            o2u[o] = b2[o];
            o1u[o] = b1[o];
            heu[o] = bh[o];
        }
    __syncthreads();
    // first level with N2 < 0.01 (comp_ng.F90:425-429)
    if (live)
        for (int k = w; k < nk; k += kPostWarps) {
            const long o = (long)k * ld + col;
            if (xs(xs(xs(1.0, o2u[o]), o1u[o]), heu[o]) < 0.01) {
                atomicMin(&ktop_s[c], k);
                break;
            }
        }
    __syncthreads();
    if (w == 0 && live) {
        const int ktop = ktop_s[c];
        double n2top = 0.0, dn2dz = 0.0, zmtop = 0.0;
        if (ktop > 0 && ktop < nk - 1) {
            const long o = (long)ktop * ld + col, om = o - ld;
            zmtop = zpmid[ktop];
            n2top = log(xm(xs(xs(xs(1.0, o2u[o]), o1u[o]), heu[o]), xnmbar[o]));
            const double n2top1 = log(xm(xs(xs(xs(1.0, o2u[om]), o1u[om]), heu[om]), xnmbar[om]));
            dn2dz = xd(xs(n2top, n2top1), dz);
        }
        n2top_s[c] = n2top;
        dn2dz_s[c] = dn2dz;
        zmtop_s[c] = zmtop;
    }
    __syncthreads();
    if (!live) return;
    const int ktop = ktop_s[c];
    const bool extrap = ktop > 0 && ktop < nk - 1;
    const double n2top = n2top_s[c], dn2dz = dn2dz_s[c], zmtop = zmtop_s[c];
    for (int k = w; k < nk; k += kPostWarps) {
        const long o = (long)k * ld + col;
        const double a0 = o2u[o], b0 = o1u[o], c0 = heu[o];
        const double an = xa(xm(ds2, xa(o2_nm[o], a0)), xm(ds, o2[o]));
        const double bn = xa(xm(ds2, xa(o1_nm[o], b0)), xm(ds, o1[o]));
        const double cn = xa(xm(ds2, xa(he_nm[o], c0)), xm(ds, he[o]));
        double n2 = xs(xs(xs(1.0, a0), b0), c0);
        if (extrap && k > ktop) n2 = xd(exp(xa(n2top, xm(dn2dz, xs(zpmid[k], zmtop)))), xnmbar[o]);
        const double n2nm = xs(xs(xs(1.0, an), bn), cn);
        double a = fmax(a0, small), b = fmax(b0, small), cc = fmax(c0, small), d = fmax(n2, small);
        // the three quotients by one sum share a correctly rounded reciprocal
        double s = xa(xa(xa(a, b), cc), d), y = __drcp_rn(s);
        o2u[o] = qdiv(a, s, y);
        o1u[o] = qdiv(b, s, y);
        heu[o] = qdiv(cc, s, y);
        a = fmax(an, small);
        b = fmax(bn, small);
        cc = fmax(cn, small);
        d = fmax(n2nm, small);
        s = xa(xa(xa(a, b), cc), d);
        y = __drcp_rn(s);
        o2n[o] = qdiv(a, s, y);
        o1n[o] = qdiv(b, s, y);
        hen[o] = qdiv(cc, s, y);
    }
}

cudaError_t launch_comp_post_ng(const double *const *in7, const double *zpmid, double dz, double dtsmooth,
                                double dtsmooth_div2, int nk, int ncol, long ld, double *const *upd6, cudaStream_t st,
                                const unsigned char *bnd_mask, const double *const *bnd3)
{
    if (ncol <= 0) return cudaSuccess;
    k_comp_post_ng<<<(ncol + kPostCols - 1) / kPostCols, kPostCols * kPostWarps, 0, st>>>(
        in7[0], in7[1], in7[2], in7[3], in7[4], in7[5], in7[6], zpmid, dz, dtsmooth, dtsmooth_div2, nk, ncol, ld,
        upd6[0], upd6[1], upd6[2], upd6[3], upd6[4], upd6[5], bnd_mask, bnd_mask ? bnd3[0] : nullptr,
        bnd_mask ? bnd3[1] : nullptr, bnd_mask ? bnd3[2] : nullptr);
    return cudaGetLastError();
}

// The post-solve time filter and floor that dt_ng (src/dt_ng.F90:208-213),
// minor_ng (src/minor_ng.F90:234-237) and oplus_ng (src/oplus_ng.F90:337-340)
// apply once the lateral-boundary columns are written:
//   nm = dtsmooth_div2*(prev + upd) + dtsmooth*cur,  upd = max(upd, fl)
// and, for minor_ng and oplus_ng, nm = max(nm, fl).  Element-wise, so one
// thread per element of rows of len elements at stride ld; nm may alias prev
// or cur (each element is read before it is written by the same thread).
// A floor keeps x when x > fl and gives fl otherwise, NaN included.
template <bool FloorNm>
__global__ void __launch_bounds__(256) k_time_filter(const double *cur, const double *prev, double ds, double ds2,
                                                     double fl, long len, long ld, double *upd, double *nm)
{
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= len) return;
    const long o = (long)blockIdx.y * ld + i;
    const double u = upd[o];
    const double n = xa(xm(ds2, xa(prev[o], u)), xm(ds, cur[o]));
    upd[o] = u > fl ? u : fl;
    nm[o] = (!FloorNm || n > fl) ? n : fl;
}

cudaError_t launch_time_filter(int which, const double *cur, const double *prev, double dtsmooth,
                               double dtsmooth_div2, int rows, long len, long ld, double *upd, double *nm,
                               cudaStream_t st)
{
    if (rows <= 0 || len <= 0) return cudaSuccess;
    const int T = 256;
    const dim3 grid((unsigned)((len + T - 1) / T), (unsigned)rows);
    if (which == TG_FILTER_DT)
        k_time_filter<false><<<grid, T, 0, st>>>(cur, prev, dtsmooth, dtsmooth_div2, 100.0, len, ld, upd, nm);
    else
        k_time_filter<true><<<grid, T, 0, st>>>(cur, prev, dtsmooth, dtsmooth_div2,
                                                which == TG_FILTER_MINOR ? 1.e-12 : 0.0, len, ld, upd, nm);
    return cudaGetLastError();
}
}  // namespace tg
