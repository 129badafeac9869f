// Column-solve kernels for sm_100a.
//
// Data layout on the device is level-major ("L layout"): element (k, col) of
// a scalar array at k*ld + col, so the 32 columns of a warp read 256
// contiguous bytes per level and every level's load is coalesced.  One thread
// solves one column (or two adjacent columns with 128-bit loads), walking the
// levels sequentially; columns are independent.
//
// FP64 kernels reproduce the reference arithmetic bit for bit: every
// multiply, add and subtract uses the non-contracting __dmul_rn/__dadd_rn/
// __dsub_rn intrinsics and divisions are IEEE (__ddiv_rn), in the reference's
// operation order (src/trsolv_ng.F90:14-26, src/comp_ng.F90:281-332,
// src/matutil.F90:25-27,63-71,116).
#include <cfloat>
#include <cstdio>

#include "tg_internal.h"

namespace tg {

// ---------------------------------------------------------------------------
// Arithmetic and memory helpers
// ---------------------------------------------------------------------------
__device__ __forceinline__ double xmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double xsub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double xadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double xdiv(double a, double b) { return __ddiv_rn(a, b); }
__device__ __forceinline__ bool finite_nz(double w) { return fabs(w) <= DBL_MAX && w != 0.0; }
__device__ __forceinline__ bool finite(double w) { return fabs(w) <= DBL_MAX; }

// Streaming read of coefficients used once (evict-first in L1/L2).
template <int N>
__device__ __forceinline__ void ld_stream(const double *p, double (&v)[N]);
template <>
__device__ __forceinline__ void ld_stream<1>(const double *p, double (&v)[1]) { v[0] = __ldcs(p); }
template <>
__device__ __forceinline__ void ld_stream<2>(const double *p, double (&v)[2])
{
    double2 t = __ldcs(reinterpret_cast<const double2 *>(p));
    v[0] = t.x;
    v[1] = t.y;
}
// Read-only read that should stay in L2 for a later re-read.
template <int N>
__device__ __forceinline__ void ld_keep(const double *p, double (&v)[N]);
template <>
__device__ __forceinline__ void ld_keep<1>(const double *p, double (&v)[1]) { v[0] = __ldg(p); }
template <>
__device__ __forceinline__ void ld_keep<2>(const double *p, double (&v)[2])
{
    double2 t = __ldg(reinterpret_cast<const double2 *>(p));
    v[0] = t.x;
    v[1] = t.y;
}
// Coherent read of data this thread wrote earlier in the same launch.
template <int N>
__device__ __forceinline__ void ld_rw(const double *p, double (&v)[N]);
template <>
__device__ __forceinline__ void ld_rw<1>(const double *p, double (&v)[1]) { v[0] = *p; }
template <>
__device__ __forceinline__ void ld_rw<2>(const double *p, double (&v)[2])
{
    double2 t = *reinterpret_cast<const double2 *>(p);
    v[0] = t.x;
    v[1] = t.y;
}
// Store of nvalid (<= N) adjacent columns.
template <int N>
__device__ __forceinline__ void st_cols(double *p, const double (&v)[N], int nvalid);
template <>
__device__ __forceinline__ void st_cols<1>(double *p, const double (&v)[1], int) { *p = v[0]; }
template <>
__device__ __forceinline__ void st_cols<2>(double *p, const double (&v)[2], int nvalid)
{
    if (nvalid == 2)
        *reinterpret_cast<double2 *>(p) = make_double2(v[0], v[1]);
    else
        *p = v[0];
}

// Segment of flattened tile t (tile0 is a prefix sum over segments).
__device__ __forceinline__ int find_seg(const SegTable &tab, int t)
{
    int lo = 0, hi = tab.nseg - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (__ldg(&tab.segs[mid].tile0) <= t)
            lo = mid;
        else
            hi = mid - 1;
    }
    return lo;
}

__device__ __forceinline__ void report(unsigned *status, int idx, unsigned flags)
{
    if (flags && status) atomicOr(status + idx, flags);
}

// ---------------------------------------------------------------------------
// Scalar Thomas, FP64, bit-exact (trsolv_ng.F90:14-26).
//
// Forward: w2(k-1) = c(k-1)/w1(k-1); w1(k) = b(k)-a(k)*w2(k-1);
//          w3(k) = (f(k)-a(k)*w3(k-1))/w1(k).
// w2 goes to this thread's shared-memory slots; w3 is parked in x (the line
// stays in L2 until the back sweep reads and overwrites it), so only 8 bytes
// of shared memory per level and column are needed.
// Back:    x(k) = w3(k) - w2(k)*x(k+1).
// Coefficient loads run PF levels ahead in a register ring.
// ---------------------------------------------------------------------------
template <int CPT, int PF>
__device__ __forceinline__ unsigned thomas_f64_cols(const Seg &s, long col, double *w2s, int sstride,
                                                    int nvalid)
{
    const long ld = s.ld;
    const int k2 = s.k2;
    const double *__restrict__ pa = s.a + col;
    const double *__restrict__ pb = s.b + col;
    const double *__restrict__ pc = s.c + col;
    const double *__restrict__ pf = s.f + col;
    double *__restrict__ px = s.x + col;

    bool ok = true;
    double w1[CPT], w3[CPT], cprev[CPT];
    {
        double b0[CPT], f0[CPT];
        ld_stream<CPT>(pb, b0);
        ld_stream<CPT>(pf, f0);
        ld_stream<CPT>(pc, cprev);
#pragma unroll
        for (int j = 0; j < CPT; ++j) {
            w1[j] = b0[j];
            w3[j] = xdiv(f0[j], w1[j]);
            if (j < nvalid) ok = ok && finite_nz(w1[j]);
        }
        st_cols<CPT>(px, w3, nvalid);
    }

    double ra[PF][CPT], rb[PF][CPT], rc[PF][CPT], rf[PF][CPT];
#pragma unroll
    for (int u = 0; u < PF; ++u) {
        const int k = 1 + u;
        if (k < k2) {
            ld_stream<CPT>(pa + k * ld, ra[u]);
            ld_stream<CPT>(pb + k * ld, rb[u]);
            ld_stream<CPT>(pc + k * ld, rc[u]);
            ld_stream<CPT>(pf + k * ld, rf[u]);
        }
    }
    for (int kb = 1; kb < k2; kb += PF) {
#pragma unroll
        for (int u = 0; u < PF; ++u) {
            const int k = kb + u;
            if (k < k2) {
                double w2[CPT];
#pragma unroll
                for (int j = 0; j < CPT; ++j) {
                    w2[j] = xdiv(cprev[j], w1[j]);
                    w1[j] = xsub(rb[u][j], xmul(ra[u][j], w2[j]));
                    w3[j] = xdiv(xsub(rf[u][j], xmul(ra[u][j], w3[j])), w1[j]);
                    if (j < nvalid) ok = ok && finite_nz(w1[j]);
                    cprev[j] = rc[u][j];
                }
                if (CPT == 2)
                    *reinterpret_cast<double2 *>(w2s + (k - 1) * sstride) = make_double2(w2[0], w2[CPT - 1]);
                else
                    w2s[(k - 1) * sstride] = w2[0];
                st_cols<CPT>(px + k * ld, w3, nvalid);
                const int kn = k + PF;
                if (kn < k2) {
                    ld_stream<CPT>(pa + kn * ld, ra[u]);
                    ld_stream<CPT>(pb + kn * ld, rb[u]);
                    ld_stream<CPT>(pc + kn * ld, rc[u]);
                    ld_stream<CPT>(pf + kn * ld, rf[u]);
                }
            }
        }
    }

    // Back substitution; w3(k) is re-read from x PF levels ahead.
    bool fin = true;
    double xn[CPT];
#pragma unroll
    for (int j = 0; j < CPT; ++j) {
        xn[j] = w3[j];
        if (j < nvalid) fin = fin && finite(xn[j]);
    }
    double rw[PF][CPT];
#pragma unroll
    for (int u = 0; u < PF; ++u) {
        const int k = k2 - 2 - u;
        if (k >= 0) ld_rw<CPT>(px + k * ld, rw[u]);
    }
    for (int kb = k2 - 2; kb >= 0; kb -= PF) {
#pragma unroll
        for (int u = 0; u < PF; ++u) {
            const int k = kb - u;
            if (k >= 0) {
                double w2[CPT];
                if (CPT == 2) {
                    double2 t = *reinterpret_cast<const double2 *>(w2s + k * sstride);
                    w2[0] = t.x;
                    w2[CPT - 1] = t.y;
                } else {
                    w2[0] = w2s[k * sstride];
                }
#pragma unroll
                for (int j = 0; j < CPT; ++j) {
                    xn[j] = xsub(rw[u][j], xmul(w2[j], xn[j]));
                    if (j < nvalid) fin = fin && finite(xn[j]);
                }
                const int kn = k - PF;
                if (kn >= 0) ld_rw<CPT>(px + kn * ld, rw[u]);
                st_cols<CPT>(px + k * ld, xn, nvalid);
            }
        }
    }
    return (ok ? 0u : FLAG_PIVOT) | (fin ? 0u : FLAG_NONFINITE);
}

template <int CPT, int PF>
__global__ void __launch_bounds__(256) k_scalar_f64(SegTable tab, unsigned *status)
{
    extern __shared__ double smem_d[];
    const int cpb = blockDim.x * CPT;
    double *w2s = smem_d + threadIdx.x * CPT;
    for (int t = blockIdx.x; t < tab.ntiles; t += gridDim.x) {
        const Seg s = tab.segs ? tab.segs[find_seg(tab, t)] : tab.one;
        const long col = (long)(t - s.tile0) * cpb + (long)threadIdx.x * CPT;
        const long left = (long)s.ncol - col;
        if (left > 0) {
            const int nvalid = left < CPT ? (int)left : CPT;
            report(status, s.status_idx, thomas_f64_cols<CPT, PF>(s, col, w2s, cpb, nvalid));
        }
    }
}

// ---------------------------------------------------------------------------
// Scalar Thomas, FP32 sweeps + FP64 iterative refinement.
//
// Sweep 0 factors A in FP32 (w2 = c/w1 and 1/w1 kept in shared memory) and
// solves; every later sweep forms the FP64 residual r = f - A x from the FP64
// coefficients (re-read, normally from L2) and solves A d = r with the FP32
// factors, x += d in FP64.  A column stops when max|d| <= tol*max|x|; if the
// cap is reached it is re-solved with the bit-exact FP64 sweep (shared-memory
// slots reused for w2) and flagged FLAG_NOCONV.
// Shared memory per thread: three float planes (w2, 1/w1, y) of k2 levels.
// ---------------------------------------------------------------------------
template <int PF>
__device__ __forceinline__ unsigned thomas_refine_col(const Seg &s, long col, float *sw2, float *sri,
                                                      float *sy, int T, Refine rf, int &sweeps)
{
    const long ld = s.ld;
    const int k2 = s.k2;
    const double *__restrict__ pa = s.a + col;
    const double *__restrict__ pb = s.b + col;
    const double *__restrict__ pc = s.c + col;
    const double *__restrict__ pf = s.f + col;
    double *__restrict__ px = s.x + col;
    bool ok = true;

    // ---- sweep 0: FP32 factor + solve
    {
        float w1 = 0.f, ri = 0.f, y = 0.f, cprev = 0.f;
        double ra[PF], rb[PF], rc[PF], rfv[PF];
#pragma unroll
        for (int u = 0; u < PF; ++u)
            if (u < k2) {
                ra[u] = __ldg(pa + u * ld);
                rb[u] = __ldg(pb + u * ld);
                rc[u] = __ldg(pc + u * ld);
                rfv[u] = __ldg(pf + u * ld);
            }
        for (int kb = 0; kb < k2; kb += PF) {
#pragma unroll
            for (int u = 0; u < PF; ++u) {
                const int k = kb + u;
                if (k < k2) {
                    const float af = (float)ra[u], bf = (float)rb[u], ff = (float)rfv[u];
                    if (k == 0) {
                        w1 = bf;
                        ri = __frcp_rn(w1);
                        y = ff * ri;
                    } else {
                        const float w2 = cprev * ri;
                        sw2[(k - 1) * T] = w2;
                        w1 = bf - af * w2;
                        ri = __frcp_rn(w1);
                        y = (ff - af * y) * ri;
                    }
                    ok = ok && (fabsf(w1) <= FLT_MAX) && (w1 != 0.f);
                    sri[k * T] = ri;
                    sy[k * T] = y;
                    cprev = (float)rc[u];
                    const int kn = k + PF;
                    if (kn < k2) {
                        ra[u] = __ldg(pa + kn * ld);
                        rb[u] = __ldg(pb + kn * ld);
                        rc[u] = __ldg(pc + kn * ld);
                        rfv[u] = __ldg(pf + kn * ld);
                    }
                }
            }
        }
        float xk = y;
        px[(k2 - 1) * ld] = (double)xk;
        for (int k = k2 - 2; k >= 0; --k) {
            xk = sy[k * T] - sw2[k * T] * xk;
            px[k * ld] = (double)xk;
        }
    }

    // ---- refinement sweeps
    bool conv = false;
    int sw = 0;
    if (ok) {
        for (sw = 1; sw <= rf.max_sweeps; ++sw) {
            double xm1 = 0.0, x0 = px[0];
            float y = 0.f;
            double ra[PF], rb[PF], rc[PF], rfv[PF];
#pragma unroll
            for (int u = 0; u < PF; ++u)
                if (u < k2) {
                    ra[u] = __ldg(pa + u * ld);
                    rb[u] = __ldg(pb + u * ld);
                    rc[u] = __ldg(pc + u * ld);
                    rfv[u] = __ldg(pf + u * ld);
                }
            for (int kb = 0; kb < k2; kb += PF) {
#pragma unroll
                for (int u = 0; u < PF; ++u) {
                    const int k = kb + u;
                    if (k < k2) {
                        const double xp1 = (k + 1 < k2) ? px[(k + 1) * ld] : 0.0;
                        double r = fma(-rb[u], x0, rfv[u]);
                        if (k > 0) r = fma(-ra[u], xm1, r);
                        if (k + 1 < k2) r = fma(-rc[u], xp1, r);
                        const float rr = (float)r;
                        y = (k == 0) ? rr * sri[0] : (rr - (float)ra[u] * y) * sri[k * T];
                        sy[k * T] = y;
                        xm1 = x0;
                        x0 = xp1;
                        const int kn = k + PF;
                        if (kn < k2) {
                            ra[u] = __ldg(pa + kn * ld);
                            rb[u] = __ldg(pb + kn * ld);
                            rc[u] = __ldg(pc + kn * ld);
                            rfv[u] = __ldg(pf + kn * ld);
                        }
                    }
                }
            }
            float d = y;
            double xv = px[(k2 - 1) * ld] + (double)d;
            px[(k2 - 1) * ld] = xv;
            double dmax = fabs((double)d), xmax = fabs(xv);
            for (int k = k2 - 2; k >= 0; --k) {
                d = sy[k * T] - sw2[k * T] * d;
                xv = px[k * ld] + (double)d;
                px[k * ld] = xv;
                dmax = fmax(dmax, fabs((double)d));
                xmax = fmax(xmax, fabs(xv));
            }
            if (!(xmax <= DBL_MAX) || !(dmax <= DBL_MAX)) break;
            if (dmax <= rf.rel_tol * xmax) {
                conv = true;
                break;
            }
        }
    }
    sweeps = conv ? sw : rf.max_sweeps + 1;
    if (conv) return 0u;

    // ---- fallback: bit-exact FP64 re-solve; w2 kept as two 32-bit halves in
    // this thread's (sw2, sri) slots, w3 parked in x.
    bool okd = true, fin = true;
    double w1 = __ldg(pb), w3 = xdiv(__ldg(pf), w1);
    okd = finite_nz(w1);
    px[0] = w3;
    double cprev = __ldg(pc);
    for (int k = 1; k < k2; ++k) {
        const double ak = __ldg(pa + k * ld), bk = __ldg(pb + k * ld), fk = __ldg(pf + k * ld);
        const double w2 = xdiv(cprev, w1);
        sw2[(k - 1) * T] = __int_as_float(__double2hiint(w2));
        sri[(k - 1) * T] = __int_as_float(__double2loint(w2));
        w1 = xsub(bk, xmul(ak, w2));
        w3 = xdiv(xsub(fk, xmul(ak, w3)), w1);
        okd = okd && finite_nz(w1);
        px[k * ld] = w3;
        cprev = __ldg(pc + k * ld);
    }
    double xn = w3;
    fin = finite(xn);
    for (int k = k2 - 2; k >= 0; --k) {
        const double w2 = __hiloint2double(__float_as_int(sw2[k * T]), __float_as_int(sri[k * T]));
        xn = xsub(px[k * ld], xmul(w2, xn));
        fin = fin && finite(xn);
        px[k * ld] = xn;
    }
    return FLAG_NOCONV | (okd ? 0u : FLAG_PIVOT) | (fin ? 0u : FLAG_NONFINITE);
}


template <int PF>
__global__ void __launch_bounds__(256) k_scalar_refine(SegTable tab, Refine rf, unsigned *status,
                                                       unsigned long long *hist)
{
    extern __shared__ float smem_f[];
    __shared__ unsigned long long shist[kMaxSweepBins];
    const int T = blockDim.x;
    if (threadIdx.x < kMaxSweepBins) shist[threadIdx.x] = 0ull;
    __syncthreads();
    const long plane = (long)T * tab.k2max;
    float *sw2 = smem_f + threadIdx.x;
    float *sri = sw2 + plane;
    float *sy = sri + plane;
    for (int t = blockIdx.x; t < tab.ntiles; t += gridDim.x) {
        const Seg s = tab.segs ? tab.segs[find_seg(tab, t)] : tab.one;
        const long col = (long)(t - s.tile0) * T + threadIdx.x;
        if (col < s.ncol) {
            int sweeps = 0;
            report(status, s.status_idx, thomas_refine_col<PF>(s, col, sw2, sri, sy, T, rf, sweeps));
            atomicAdd(&shist[min(sweeps, kMaxSweepBins - 1)], 1ull);
        }
    }
    __syncthreads();
    if (hist && threadIdx.x < kMaxSweepBins && shist[threadIdx.x])
        atomicAdd(hist + threadIdx.x, shist[threadIdx.x]);
}

// ---------------------------------------------------------------------------
// Small-matrix inverse, adjugate / determinant without pivoting, exactly as
// matdet2/matadj2/matinv2 and matdet3/matadj3/matinv3 (src/matutil.F90).
// Column-major: A(i,j) = A[(i-1) + B*(j-1)].  Returns false for a zero or
// non-finite determinant.
// ---------------------------------------------------------------------------
template <int B>
__device__ __forceinline__ bool inv_exact(const double (&A)[B * B], double (&W)[B * B]);

template <>
__device__ __forceinline__ bool inv_exact<2>(const double (&A)[4], double (&W)[4])
{
    const double d = xsub(xmul(A[0], A[3]), xmul(A[2], A[1]));
    W[0] = xdiv(A[3], d);
    W[1] = xdiv(-A[1], d);
    W[2] = xdiv(-A[2], d);
    W[3] = xdiv(A[0], d);
    return finite_nz(d);
}

template <>
__device__ __forceinline__ bool inv_exact<3>(const double (&A)[9], double (&W)[9])
{
#define a_(i, j) A[((i) - 1) + 3 * ((j) - 1)]
#define w_(i, j) W[((i) - 1) + 3 * ((j) - 1)]
    double d = xmul(xmul(a_(1, 1), a_(2, 2)), a_(3, 3));
    d = xsub(d, xmul(xmul(a_(1, 1), a_(2, 3)), a_(3, 2)));
    d = xsub(d, xmul(xmul(a_(1, 2), a_(2, 1)), a_(3, 3)));
    d = xadd(d, xmul(xmul(a_(1, 2), a_(2, 3)), a_(3, 1)));
    d = xadd(d, xmul(xmul(a_(1, 3), a_(2, 1)), a_(3, 2)));
    d = xsub(d, xmul(xmul(a_(1, 3), a_(2, 2)), a_(3, 1)));
    w_(1, 1) = xsub(xmul(a_(2, 2), a_(3, 3)), xmul(a_(2, 3), a_(3, 2)));
    w_(2, 1) = -xsub(xmul(a_(2, 1), a_(3, 3)), xmul(a_(2, 3), a_(3, 1)));
    w_(3, 1) = xsub(xmul(a_(2, 1), a_(3, 2)), xmul(a_(2, 2), a_(3, 1)));
    w_(1, 2) = -xsub(xmul(a_(1, 2), a_(3, 3)), xmul(a_(1, 3), a_(3, 2)));
    w_(2, 2) = xsub(xmul(a_(1, 1), a_(3, 3)), xmul(a_(1, 3), a_(3, 1)));
    w_(3, 2) = -xsub(xmul(a_(1, 1), a_(3, 2)), xmul(a_(1, 2), a_(3, 1)));
    w_(1, 3) = xsub(xmul(a_(1, 2), a_(2, 3)), xmul(a_(1, 3), a_(2, 2)));
    w_(2, 3) = -xsub(xmul(a_(1, 1), a_(2, 3)), xmul(a_(1, 3), a_(2, 1)));
    w_(3, 3) = xsub(xmul(a_(1, 1), a_(2, 2)), xmul(a_(1, 2), a_(2, 1)));
#undef a_
#undef w_
#pragma unroll
    for (int e = 0; e < 9; ++e) W[e] = xdiv(W[e], d);
    return finite_nz(d);
}

// Loads the blocks of level k: P (if wantP), Q, R (if wantR), f.
template <int B>
__device__ __forceinline__ void blk_load(const double *pP, const double *pQ, const double *pR,
                                         const double *pF, long ld, int k, bool wantP, bool wantR,
                                         double (&P)[B * B], double (&Q)[B * B], double (&R)[B * B],
                                         double (&F)[B])
{
    constexpr int BB = B * B;
    const long om = (long)k * BB * ld, ov = (long)k * B * ld;
#pragma unroll
    for (int e = 0; e < BB; ++e) {
        P[e] = wantP ? __ldcs(pP + om + e * ld) : 0.0;
        Q[e] = __ldcs(pQ + om + e * ld);
        R[e] = wantR ? __ldcs(pR + om + e * ld) : 0.0;
    }
#pragma unroll
    for (int i = 0; i < B; ++i) F[i] = __ldcs(pF + ov + i * ld);
}

// ---------------------------------------------------------------------------
// Block-tridiagonal Thomas, FP64, bit-exact (comp_ng.F90:281-332; the same
// operations as duv.F blktri for B = 2).  Per row k (0-based):
//   Q' = Q_k - P_k G_k ; W = inv(Q') ; G_{k+1} = W R_k ; z_{k+1} = W (f_k - P_k z_k)
// z_{k+1} is parked in u(row k); G_{k+1} goes to this thread's global
// scratch slots (element (k, e) at gam[(k*B*B + e)*gs]), sized so the
// resident working set stays in L2.  Back: u_k = z_{k+1} - G_{k+1} u_{k+1}.
// ---------------------------------------------------------------------------
template <int B>
__device__ __forceinline__ unsigned blk_f64_col(const Seg &s, long col, double *gam, long gs)
{
    constexpr int BB = B * B;
    const long ld = s.ld;
    const int k2 = s.k2;
    const double *pP = s.a + col, *pQ = s.b + col, *pR = s.c + col, *pF = s.f + col;
    double *pU = s.x + col;

    bool ok = true;
    double G[BB], z[B];
    double P[BB], Q[BB], R[BB], F[B];
    double nP[BB], nQ[BB], nR[BB], nF[B];
    blk_load<B>(pP, pQ, pR, pF, ld, 0, false, k2 > 1, P, Q, R, F);
    if (k2 > 1) blk_load<B>(pP, pQ, pR, pF, ld, 1, true, k2 > 2, nP, nQ, nR, nF);
    for (int k = 0; k < k2; ++k) {
        double Qp[BB], W[BB], v[B];
        if (k == 0) {
#pragma unroll
            for (int e = 0; e < BB; ++e) Qp[e] = Q[e];
#pragma unroll
            for (int i = 0; i < B; ++i) v[i] = F[i];
        } else {
#pragma unroll
            for (int m = 0; m < B; ++m)
#pragma unroll
                for (int i = 0; i < B; ++i) {
                    double q = Q[i + B * m];
#pragma unroll
                    for (int n = 0; n < B; ++n) q = xsub(q, xmul(P[i + B * n], G[n + B * m]));
                    Qp[i + B * m] = q;
                }
#pragma unroll
            for (int i = 0; i < B; ++i) {
                double t = F[i];
#pragma unroll
                for (int m = 0; m < B; ++m) t = xsub(t, xmul(P[i + B * m], z[m]));
                v[i] = t;
            }
        }
        ok = inv_exact<B>(Qp, W) && ok;
#pragma unroll
        for (int i = 0; i < B; ++i) {
            double t = xmul(W[i], v[0]);
#pragma unroll
            for (int m = 1; m < B; ++m) t = xadd(t, xmul(W[i + B * m], v[m]));
            z[i] = t;
            pU[((long)k * B + i) * ld] = t;
        }
        if (k < k2 - 1) {
#pragma unroll
            for (int m = 0; m < B; ++m)
#pragma unroll
                for (int i = 0; i < B; ++i) {
                    double g = xmul(W[i], R[B * m]);
#pragma unroll
                    for (int n = 1; n < B; ++n) g = xadd(g, xmul(W[i + B * n], R[n + B * m]));
                    G[i + B * m] = g;
                    gam[((long)k * BB + i + B * m) * gs] = g;
                }
        }
        if (k + 1 < k2) {
#pragma unroll
            for (int e = 0; e < BB; ++e) {
                P[e] = nP[e];
                Q[e] = nQ[e];
                R[e] = nR[e];
            }
#pragma unroll
            for (int i = 0; i < B; ++i) F[i] = nF[i];
            if (k + 2 < k2) blk_load<B>(pP, pQ, pR, pF, ld, k + 2, true, k + 2 < k2 - 1, nP, nQ, nR, nF);
        }
    }

    bool fin = true;
    double un[B], top[B];
#pragma unroll
    for (int i = 0; i < B; ++i) {
        un[i] = z[i];
        top[i] = z[i];
        fin = fin && finite(z[i]);
    }
    for (int k = k2 - 2; k >= 0; --k) {
        double zk[B], Gk[BB], nu[B];
#pragma unroll
        for (int i = 0; i < B; ++i) zk[i] = pU[((long)k * B + i) * ld];
#pragma unroll
        for (int e = 0; e < BB; ++e) Gk[e] = gam[((long)k * BB + e) * gs];
#pragma unroll
        for (int i = 0; i < B; ++i) {
            double t = zk[i];
#pragma unroll
            for (int m = 0; m < B; ++m) t = xsub(t, xmul(Gk[i + B * m], un[m]));
            nu[i] = t;
            fin = fin && finite(t);
        }
#pragma unroll
        for (int i = 0; i < B; ++i) {
            un[i] = nu[i];
            pU[((long)k * B + i) * ld] = nu[i];
        }
    }
    if (s.ubc_ratio) {
#pragma unroll
        for (int i = 0; i < B; ++i) {
            double t = xmul(__ldg(s.ubc_ratio + i * ld + col), top[i]);
            if (s.ubc_add) t = xadd(t, __ldg(s.ubc_add + i * ld + col));
            fin = fin && finite(t);
            pU[((long)k2 * B + i) * ld] = t;
        }
    }
    return (ok ? 0u : FLAG_PIVOT) | (fin ? 0u : FLAG_NONFINITE);
}

template <int B>
__global__ void __launch_bounds__(128) k_block_f64(SegTable tab, double *scratch, unsigned *status)
{
    const long gs = (long)gridDim.x * blockDim.x;
    double *gam = scratch + (long)blockIdx.x * blockDim.x + threadIdx.x;
    for (int t = blockIdx.x; t < tab.ntiles; t += gridDim.x) {
        const Seg s = tab.segs ? tab.segs[find_seg(tab, t)] : tab.one;
        const long col = (long)(t - s.tile0) * blockDim.x + threadIdx.x;
        if (col < s.ncol) report(status, s.status_idx, blk_f64_col<B>(s, col, gam, gs));
    }
}

// ---------------------------------------------------------------------------
// Block-tridiagonal, FP32 Gamma/z sweeps + FP64 iterative refinement.
// Pivot blocks Q' = Q - P G and their inverses W stay in FP64; W and
// G_{k+1} = W R are kept in FP32 in the thread's scratch slots together with
// the FP32 forward vector of the current correction sweep:
//   level k: W (B*B floats) | G_{k+1} (B*B floats) | z_{k+1} (B floats).
// Refinement sweeps form r = f - P u_{k-1} - Q u_k - R u_{k+1} in FP64 and
// solve the correction with the FP32 factors.  Non-converged columns are
// re-solved with the bit-exact FP64 sweep (its G kept as float pairs).
// ---------------------------------------------------------------------------
template <int B>
__device__ __forceinline__ unsigned blk_refine_col(const Seg &s, long col, float *scr, long gs,
                                                   Refine rf, int &sweeps)
{
    constexpr int BB = B * B, NS = 2 * BB + B;
    const long ld = s.ld;
    const int k2 = s.k2;
    const double *pP = s.a + col, *pQ = s.b + col, *pR = s.c + col, *pF = s.f + col;
    double *pU = s.x + col;
    auto S = [&](int k, int e) -> float & { return scr[((long)k * NS + e) * gs]; };

    bool ok = true;
    // ---- sweep 0
    {
        float G[BB], z[B];
        for (int k = 0; k < k2; ++k) {
            double P[BB], Q[BB], R[BB], F[B];
            const long om = (long)k * BB * ld, ov = (long)k * B * ld;
#pragma unroll
            for (int e = 0; e < BB; ++e) {
                P[e] = k > 0 ? __ldg(pP + om + e * ld) : 0.0;
                Q[e] = __ldg(pQ + om + e * ld);
                R[e] = k < k2 - 1 ? __ldg(pR + om + e * ld) : 0.0;
            }
#pragma unroll
            for (int i = 0; i < B; ++i) F[i] = __ldg(pF + ov + i * ld);
            double Qp[BB], W[BB];
#pragma unroll
            for (int m = 0; m < B; ++m)
#pragma unroll
                for (int i = 0; i < B; ++i) {
                    double q = Q[i + B * m];
                    if (k > 0)
#pragma unroll
                        for (int n = 0; n < B; ++n) q = fma(-P[i + B * n], (double)G[n + B * m], q);
                    Qp[i + B * m] = q;
                }
            ok = inv_exact<B>(Qp, W) && ok;
            float W32[BB], v[B];
#pragma unroll
            for (int e = 0; e < BB; ++e) {
                W32[e] = (float)W[e];
                S(k, e) = W32[e];
            }
#pragma unroll
            for (int i = 0; i < B; ++i) {
                float t = (float)F[i];
                if (k > 0)
#pragma unroll
                    for (int m = 0; m < B; ++m) t = fmaf(-(float)P[i + B * m], z[m], t);
                v[i] = t;
            }
#pragma unroll
            for (int i = 0; i < B; ++i) {
                float t = 0.f;
#pragma unroll
                for (int m = 0; m < B; ++m) t = fmaf(W32[i + B * m], v[m], t);
                z[i] = t;
                S(k, 2 * BB + i) = t;
            }
#pragma unroll
            for (int m = 0; m < B; ++m)
#pragma unroll
                for (int i = 0; i < B; ++i) {
                    float g = 0.f;
                    if (k < k2 - 1)
#pragma unroll
                        for (int n = 0; n < B; ++n) g = fmaf(W32[i + B * n], (float)R[n + B * m], g);
                    G[i + B * m] = g;
                    S(k, BB + i + B * m) = g;
                }
        }
        float un[B];
#pragma unroll
        for (int i = 0; i < B; ++i) {
            un[i] = z[i];
            pU[((long)(k2 - 1) * B + i) * ld] = (double)z[i];
        }
        for (int k = k2 - 2; k >= 0; --k) {
            float nu[B];
#pragma unroll
            for (int i = 0; i < B; ++i) {
                float t = S(k, 2 * BB + i);
#pragma unroll
                for (int m = 0; m < B; ++m) t = fmaf(-S(k, BB + i + B * m), un[m], t);
                nu[i] = t;
            }
#pragma unroll
            for (int i = 0; i < B; ++i) {
                un[i] = nu[i];
                pU[((long)k * B + i) * ld] = (double)nu[i];
            }
        }
    }

    // ---- refinement sweeps
    bool conv = false;
    int sw = 0;
    if (ok) {
        for (sw = 1; sw <= rf.max_sweeps; ++sw) {
            double um[B], u0[B];
            float zc[B];
#pragma unroll
            for (int i = 0; i < B; ++i) {
                um[i] = 0.0;
                u0[i] = pU[i * ld];
                zc[i] = 0.f;
            }
            for (int k = 0; k < k2; ++k) {
                const long om = (long)k * BB * ld, ov = (long)k * B * ld;
                double up[B], r[B];
#pragma unroll
                for (int i = 0; i < B; ++i) {
                    up[i] = (k + 1 < k2) ? pU[((long)(k + 1) * B + i) * ld] : 0.0;
                    r[i] = __ldg(pF + ov + i * ld);
                }
                float P32[BB];
#pragma unroll
                for (int e = 0; e < BB; ++e) {
                    const int i = e % B, m = e / B;
                    const double q = __ldg(pQ + om + e * ld);
                    r[i] = fma(-q, u0[m], r[i]);
                    double p = 0.0;
                    if (k > 0) {
                        p = __ldg(pP + om + e * ld);
                        r[i] = fma(-p, um[m], r[i]);
                    }
                    P32[e] = (float)p;
                    if (k + 1 < k2) r[i] = fma(-__ldg(pR + om + e * ld), up[m], r[i]);
                }
                float v[B];
#pragma unroll
                for (int i = 0; i < B; ++i) {
                    float t = (float)r[i];
#pragma unroll
                    for (int m = 0; m < B; ++m) t = fmaf(-P32[i + B * m], zc[m], t);
                    v[i] = t;
                }
#pragma unroll
                for (int i = 0; i < B; ++i) {
                    float t = 0.f;
#pragma unroll
                    for (int m = 0; m < B; ++m) t = fmaf(S(k, i + B * m), v[m], t);
                    zc[i] = t;
                    S(k, 2 * BB + i) = t;
                }
#pragma unroll
                for (int i = 0; i < B; ++i) {
                    um[i] = u0[i];
                    u0[i] = up[i];
                }
            }
            double dmax = 0.0, xmax = 0.0;
            float dn[B];
#pragma unroll
            for (int i = 0; i < B; ++i) {
                dn[i] = zc[i];
                double* p = pU + ((long)(k2 - 1) * B + i) * ld;
                const double xv = *p + (double)dn[i];
                *p = xv;
                dmax = fmax(dmax, fabs((double)dn[i]));
                xmax = fmax(xmax, fabs(xv));
            }
            for (int k = k2 - 2; k >= 0; --k) {
                float nd[B];
#pragma unroll
                for (int i = 0; i < B; ++i) {
                    float t = S(k, 2 * BB + i);
#pragma unroll
                    for (int m = 0; m < B; ++m) t = fmaf(-S(k, BB + i + B * m), dn[m], t);
                    nd[i] = t;
                }
#pragma unroll
                for (int i = 0; i < B; ++i) {
                    dn[i] = nd[i];
                    double* p = pU + ((long)k * B + i) * ld;
                    const double xv = *p + (double)nd[i];
                    *p = xv;
                    dmax = fmax(dmax, fabs((double)nd[i]));
                    xmax = fmax(xmax, fabs(xv));
                }
            }
            if (!(xmax <= DBL_MAX) || !(dmax <= DBL_MAX)) break;
            if (dmax <= rf.rel_tol * xmax) {
                conv = true;
                break;
            }
        }
    }
    sweeps = conv ? sw : rf.max_sweeps + 1;
    unsigned flags = 0u;
    if (!conv) {
        // ---- fallback: bit-exact FP64 solve, G kept as (hi, lo) float pairs.
        flags |= FLAG_NOCONV;
        bool okd = true, fin = true;
        double G[BB], z[B];
        for (int k = 0; k < k2; ++k) {
            double P[BB], Q[BB], R[BB], F[B];
            blk_load<B>(pP, pQ, pR, pF, ld, k, k > 0, k < k2 - 1, P, Q, R, F);
            double Qp[BB], W[BB], v[B];
#pragma unroll
            for (int m = 0; m < B; ++m)
#pragma unroll
                for (int i = 0; i < B; ++i) {
                    double q = Q[i + B * m];
                    if (k > 0)
#pragma unroll
                        for (int n = 0; n < B; ++n) q = xsub(q, xmul(P[i + B * n], G[n + B * m]));
                    Qp[i + B * m] = q;
                }
#pragma unroll
            for (int i = 0; i < B; ++i) {
                double t = F[i];
                if (k > 0)
#pragma unroll
                    for (int m = 0; m < B; ++m) t = xsub(t, xmul(P[i + B * m], z[m]));
                v[i] = t;
            }
            okd = inv_exact<B>(Qp, W) && okd;
#pragma unroll
            for (int i = 0; i < B; ++i) {
                double t = xmul(W[i], v[0]);
#pragma unroll
                for (int m = 1; m < B; ++m) t = xadd(t, xmul(W[i + B * m], v[m]));
                z[i] = t;
                pU[((long)k * B + i) * ld] = t;
            }
            if (k < k2 - 1) {
#pragma unroll
                for (int m = 0; m < B; ++m)
#pragma unroll
                    for (int i = 0; i < B; ++i) {
                        double g = xmul(W[i], R[B * m]);
#pragma unroll
                        for (int n = 1; n < B; ++n) g = xadd(g, xmul(W[i + B * n], R[n + B * m]));
                        G[i + B * m] = g;
                        S(k, 2 * (i + B * m)) = __int_as_float(__double2hiint(g));
                        S(k, 2 * (i + B * m) + 1) = __int_as_float(__double2loint(g));
                    }
            }
        }
        double un[B];
#pragma unroll
        for (int i = 0; i < B; ++i) {
            un[i] = z[i];
            fin = fin && finite(z[i]);
        }
        for (int k = k2 - 2; k >= 0; --k) {
            double nu[B];
#pragma unroll
            for (int i = 0; i < B; ++i) {
                double t = pU[((long)k * B + i) * ld];
#pragma unroll
                for (int m = 0; m < B; ++m) {
                    const int e = i + B * m;
                    const double g = __hiloint2double(__float_as_int(S(k, 2 * e)), __float_as_int(S(k, 2 * e + 1)));
                    t = xsub(t, xmul(g, un[m]));
                }
                nu[i] = t;
                fin = fin && finite(t);
            }
#pragma unroll
            for (int i = 0; i < B; ++i) {
                un[i] = nu[i];
                pU[((long)k * B + i) * ld] = nu[i];
            }
        }
        flags |= (okd ? 0u : FLAG_PIVOT) | (fin ? 0u : FLAG_NONFINITE);
    } else if (!ok) {
        flags |= FLAG_PIVOT;
    }
    if (s.ubc_ratio) {
        bool fin = true;
#pragma unroll
        for (int i = 0; i < B; ++i) {
            const double top = pU[((long)(k2 - 1) * B + i) * ld];
            double t = xmul(__ldg(s.ubc_ratio + i * ld + col), top);
            if (s.ubc_add) t = xadd(t, __ldg(s.ubc_add + i * ld + col));
            fin = fin && finite(t);
            pU[((long)k2 * B + i) * ld] = t;
        }
        if (!fin) flags |= FLAG_NONFINITE;
    }
    return flags;
}

template <int B>
__global__ void __launch_bounds__(128) k_block_refine(SegTable tab, Refine rf, float *scratch,
                                                      unsigned *status, unsigned long long *hist)
{
    __shared__ unsigned long long shist[kMaxSweepBins];
    if (threadIdx.x < kMaxSweepBins) shist[threadIdx.x] = 0ull;
    __syncthreads();
    const long gs = (long)gridDim.x * blockDim.x;
    float *scr = scratch + (long)blockIdx.x * blockDim.x + threadIdx.x;
    for (int t = blockIdx.x; t < tab.ntiles; t += gridDim.x) {
        const Seg s = tab.segs ? tab.segs[find_seg(tab, t)] : tab.one;
        const long col = (long)(t - s.tile0) * blockDim.x + threadIdx.x;
        if (col < s.ncol) {
            int sweeps = 0;
            report(status, s.status_idx, blk_refine_col<B>(s, col, scr, gs, rf, sweeps));
            atomicAdd(&shist[min(sweeps, kMaxSweepBins - 1)], 1ull);
        }
    }
    __syncthreads();
    if (hist && threadIdx.x < kMaxSweepBins && shist[threadIdx.x])
        atomicAdd(hist + threadIdx.x, shist[threadIdx.x]);
}

// ---------------------------------------------------------------------------
// Relayout between the Fortran column layout and the level-major layout,
// 32x32 tiles through shared memory (padded to avoid bank conflicts).
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_col_to_level(const double *__restrict__ in, long in_ld,
                                                      double *__restrict__ out, long out_ld, long nrows,
                                                      long ncols)
{
    __shared__ double tile[32][33];
    const long nrt = (nrows + 31) / 32, nct = (ncols + 31) / 32;
    for (long bt = blockIdx.x; bt < nrt * nct; bt += gridDim.x) {
        const long r0 = (bt % nrt) * 32, c0 = (bt / nrt) * 32;
        for (int j = threadIdx.y; j < 32; j += 8) {
            const long c = c0 + j, r = r0 + threadIdx.x;
            if (c < ncols && r < nrows) tile[j][threadIdx.x] = __ldcs(in + r + in_ld * c);
        }
        __syncthreads();
        for (int j = threadIdx.y; j < 32; j += 8) {
            const long r = r0 + j, c = c0 + threadIdx.x;
            if (r < nrows && c < ncols) out[r * out_ld + c] = tile[threadIdx.x][j];
        }
        __syncthreads();
    }
}

__global__ void __launch_bounds__(256) k_level_to_col(const double *__restrict__ in, long in_ld,
                                                      double *__restrict__ out, long out_ld, long nrows,
                                                      long ncols)
{
    __shared__ double tile[32][33];
    const long nrt = (nrows + 31) / 32, nct = (ncols + 31) / 32;
    for (long bt = blockIdx.x; bt < nrt * nct; bt += gridDim.x) {
        const long r0 = (bt % nrt) * 32, c0 = (bt / nrt) * 32;
        for (int j = threadIdx.y; j < 32; j += 8) {
            const long r = r0 + j, c = c0 + threadIdx.x;
            if (r < nrows && c < ncols) tile[j][threadIdx.x] = __ldcs(in + r * in_ld + c);
        }
        __syncthreads();
        for (int j = threadIdx.y; j < 32; j += 8) {
            const long c = c0 + j, r = r0 + threadIdx.x;
            if (c < ncols && r < nrows) out[r + out_ld * c] = tile[threadIdx.x][j];
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// Launch shapes and launchers
// ---------------------------------------------------------------------------
namespace {
constexpr int kPF = 4;
struct TileCfg {
    int cpb, cpt;
};
// [kind index: scalar, block2, block3][precision]
TileCfg g_tile[3][2] = {{{128, 1}, {128, 1}}, {{64, 1}, {64, 1}}, {{64, 1}, {64, 1}}};
const TileCfg kDefaultTile[3][2] = {{{128, 1}, {128, 1}}, {{64, 1}, {64, 1}}, {{64, 1}, {64, 1}}};
int kind_index(int kind) { return kind == TG_KIND_SCALAR ? 0 : (kind == TG_KIND_BLOCK2 ? 1 : 2); }
int g_num_sms = -1;
int g_smem_optin = -1;

int num_sms()
{
    if (g_num_sms < 0) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&g_num_sms, cudaDevAttrMultiProcessorCount, dev);
        cudaDeviceGetAttribute(&g_smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
        // every kernel that takes dynamic shared memory may use up to the
        // opt-in limit (minus its static shared memory)
        const int lim = g_smem_optin - 1024;
        cudaFuncSetAttribute(k_scalar_f64<1, kPF>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
        cudaFuncSetAttribute(k_scalar_f64<2, kPF>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
        cudaFuncSetAttribute(k_scalar_refine<kPF>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
    }
    return g_num_sms;
}

template <typename K>
cudaError_t occupancy(K kernel, int threads, size_t smem, int *per_sm)
{
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(per_sm, kernel, threads, smem);
}

// Resident threads per SM allowed for the block kernels: their Gamma scratch
// (k2 * B*B doubles per resident thread) should stay well inside L2.
constexpr double kBlockScratchBudget = 48.0 * 1024 * 1024;
}  // namespace

int cols_per_block(int kind, int precision)
{
    const TileCfg &t = g_tile[kind_index(kind)][precision ? 1 : 0];
    return t.cpb;
}
int cols_per_thread(int kind, int precision) { return g_tile[kind_index(kind)][precision ? 1 : 0].cpt; }
void set_tile(int kind, int precision, int cpb, int cpt)
{
    TileCfg &t = g_tile[kind_index(kind)][precision ? 1 : 0];
    const TileCfg &d = kDefaultTile[kind_index(kind)][precision ? 1 : 0];
    t.cpb = cpb > 0 ? cpb : d.cpb;
    t.cpt = cpt > 0 ? cpt : d.cpt;
    if (kind != TG_KIND_SCALAR || precision) t.cpt = 1;
}

size_t scalar_smem_bytes(int precision, int threads, int cpt, int k2max)
{
    if (precision == TG_PREC_F64) return (size_t)threads * cpt * (size_t)(k2max > 1 ? k2max - 1 : 1) * 8;
    return (size_t)threads * 3 * (size_t)k2max * 4;
}

size_t block_scratch_bytes(int B, int precision, long slots, int k2max)
{
    if (precision == TG_PREC_F64) return (size_t)slots * B * B * (size_t)k2max * 8;
    return (size_t)slots * (2 * B * B + B) * (size_t)k2max * 4;
}

cudaError_t plan_shape(int kind, int precision, int k2max, int ntiles, Shape *sh)
{
    const int nsm = num_sms();
    const TileCfg &t = g_tile[kind_index(kind)][precision ? 1 : 0];
    int per_sm = 0;
    cudaError_t e = cudaSuccess;
    sh->cpt = t.cpt;
    sh->threads = t.cpb / t.cpt;
    if (kind == TG_KIND_SCALAR) {
        sh->smem = scalar_smem_bytes(precision, sh->threads, sh->cpt, k2max);
        if (sh->smem > (size_t)(g_smem_optin - 1024)) return cudaErrorInvalidConfiguration;
        if (precision == TG_PREC_F64)
            e = sh->cpt == 2 ? occupancy(k_scalar_f64<2, kPF>, sh->threads, sh->smem, &per_sm)
                             : occupancy(k_scalar_f64<1, kPF>, sh->threads, sh->smem, &per_sm);
        else
            e = occupancy(k_scalar_refine<kPF>, sh->threads, sh->smem, &per_sm);
    } else {
        const int B = kind;
        sh->smem = 0;
        if (precision == TG_PREC_F64)
            e = B == 2 ? occupancy(k_block_f64<2>, sh->threads, 0, &per_sm)
                       : occupancy(k_block_f64<3>, sh->threads, 0, &per_sm);
        else
            e = B == 2 ? occupancy(k_block_refine<2>, sh->threads, 0, &per_sm)
                       : occupancy(k_block_refine<3>, sh->threads, 0, &per_sm);
        if (e == cudaSuccess) {
            const double per_thread = (double)block_scratch_bytes(B, precision, 1, k2max);
            const int cap = (int)(kBlockScratchBudget / (per_thread * sh->threads * nsm));
            per_sm = per_sm < cap ? per_sm : (cap > 0 ? cap : 1);
        }
    }
    if (e != cudaSuccess) return e;
    if (per_sm < 1) return cudaErrorInvalidConfiguration;
    long blocks = (long)per_sm * nsm;
    if (blocks > ntiles) blocks = ntiles;
    sh->blocks = (int)(blocks > 0 ? blocks : 1);
    return cudaSuccess;
}

cudaError_t launch_scalar(const SegTable &tab, int precision, const Shape &sh, Refine rf,
                          unsigned *status, unsigned long long *hist, cudaStream_t st)
{
    if (tab.ntiles <= 0) return cudaSuccess;
    if (precision == TG_PREC_F64) {
        if (sh.cpt == 2)
            k_scalar_f64<2, kPF><<<sh.blocks, sh.threads, sh.smem, st>>>(tab, status);
        else
            k_scalar_f64<1, kPF><<<sh.blocks, sh.threads, sh.smem, st>>>(tab, status);
    } else {
        k_scalar_refine<kPF><<<sh.blocks, sh.threads, sh.smem, st>>>(tab, rf, status, hist);
    }
    return cudaGetLastError();
}

cudaError_t launch_block(const SegTable &tab, int B, int precision, const Shape &sh, Refine rf,
                         double *scratch, unsigned *status, unsigned long long *hist, cudaStream_t st)
{
    if (tab.ntiles <= 0) return cudaSuccess;
    if (precision == TG_PREC_F64) {
        if (B == 2)
            k_block_f64<2><<<sh.blocks, sh.threads, 0, st>>>(tab, scratch, status);
        else
            k_block_f64<3><<<sh.blocks, sh.threads, 0, st>>>(tab, scratch, status);
    } else {
        float *fs = reinterpret_cast<float *>(scratch);
        if (B == 2)
            k_block_refine<2><<<sh.blocks, sh.threads, 0, st>>>(tab, rf, fs, status, hist);
        else
            k_block_refine<3><<<sh.blocks, sh.threads, 0, st>>>(tab, rf, fs, status, hist);
    }
    return cudaGetLastError();
}

static int relayout_blocks(long nrows, long ncols)
{
    const long tiles = ((nrows + 31) / 32) * ((ncols + 31) / 32);
    const long cap = (long)num_sms() * 8;
    return (int)(tiles < cap ? (tiles > 0 ? tiles : 1) : cap);
}

cudaError_t launch_col_to_level(const double *in, long in_ld, double *out, long out_ld, long nrows,
                                long ncols, cudaStream_t st)
{
    if (nrows <= 0 || ncols <= 0) return cudaSuccess;
    k_col_to_level<<<relayout_blocks(nrows, ncols), dim3(32, 8), 0, st>>>(in, in_ld, out, out_ld, nrows, ncols);
    return cudaGetLastError();
}

cudaError_t launch_level_to_col(const double *in, long in_ld, double *out, long out_ld, long nrows,
                                long ncols, cudaStream_t st)
{
    if (nrows <= 0 || ncols <= 0) return cudaSuccess;
    k_level_to_col<<<relayout_blocks(nrows, ncols), dim3(32, 8), 0, st>>>(in, in_ld, out, out_ld, nrows, ncols);
    return cudaGetLastError();
}

}  // namespace tg
