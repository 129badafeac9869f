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
#include <atomic>
#include <mutex>

#include "tg_internal.h"
#include "tg_arith.cuh"
#include "tg_bulk.cuh"

namespace tg {

// ---------------------------------------------------------------------------
// Arithmetic and memory helpers
// ---------------------------------------------------------------------------
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

// L2 eviction-priority policies (createpolicy): the coefficient streams are
// read once (evict-first); the sweep's own scratch (w2, and w3 parked in x)
// is re-read by the back sweep and should stay in L2 (evict-last).  With
// hints off both are evict-normal.
__device__ __forceinline__ unsigned long long l2_policy(int hints, bool keep)
{
    unsigned long long p;
    if (!hints)
        asm volatile("createpolicy.fractional.L2::evict_normal.b64 %0, 1.0;" : "=l"(p));
    else if (keep)
        asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
    else
        asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
    return p;
}
// Coefficient fills of the refinement kernels, which read a, b, c, f (P, Q,
// R, f) once per sweep: hints 2 and 3 keep them in L2 between the sweeps
// (evict-normal, evict-last) instead of marking them evict-first.
__device__ __forceinline__ unsigned long long refine_fill_policy(int hints)
{
    unsigned long long p;
    if (hints == 2)
        asm volatile("createpolicy.fractional.L2::evict_normal.b64 %0, 1.0;" : "=l"(p));
    else if (hints == 3)
        asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
    else
        p = l2_policy(hints, false);
    return p;
}
__device__ __forceinline__ void bulk_load_hint(void *dst, const void *src, uint32_t bytes, unsigned long long *bar,
                                               unsigned long long pol)
{
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint [%0], [%1], %2, [%3], %4;" ::"r"(
            smem_addr(dst)),
        "l"(src), "r"(bytes), "r"(smem_addr(bar)), "l"(pol)
        : "memory");
}
__device__ __forceinline__ void st_hint(double *p, double v, unsigned long long pol)
{
    asm volatile("st.global.L2::cache_hint.f64 [%0], %1, %2;" ::"l"(p), "d"(v), "l"(pol) : "memory");
}
__device__ __forceinline__ double ld_hint(const double *p, unsigned long long pol)
{
    double v;
    asm volatile("ld.global.L2::cache_hint.f64 %0, [%1], %2;" : "=d"(v) : "l"(p), "l"(pol) : "memory");
    return v;
}
// Stage ring of a single-warp CTA: level k of NE arrays (W columns x 8 B
// each) lands in stage (q % D), q the running level counter of the CTA.
template <int NE, int D, int W = 32>
struct Ring {
    double *buf;                 // D * NE * W doubles
    unsigned long long *bar;     // D mbarriers
    unsigned long long pol;      // L2 policy of the fills
    __device__ __forceinline__ void init(int lane)
    {
        if (lane == 0) {
#pragma unroll 1
            for (int s = 0; s < D; ++s) mbar_init(&bar[s], 1);
            fence_mbar_init();
        }
        __syncwarp();
    }
    // All lanes call; lanes e < NE issue entry e from src[e].
    __device__ __forceinline__ void issue(unsigned q, const double *src_e, int lane)
    {
        const int st = (int)(q % D);
        if (lane == 0) mbar_expect(&bar[st], NE * W * 8u);
        __syncwarp();
        if (lane < NE) bulk_load_hint(buf + (st * NE + lane) * W, src_e, W * 8u, &bar[st], pol);
    }
    __device__ __forceinline__ bool wait(unsigned q) { return mbar_wait_warp(&bar[q % D], (q / D) & 1u); }
    __device__ __forceinline__ double at(unsigned q, int e, int c) const
    {
        return buf[((int)(q % D) * NE + e) * W + c];
    }
    // After a timeout: bounded wait for the fills still in flight (q0..q1-1).
    __device__ __forceinline__ void drain(unsigned q0, unsigned q1)
    {
#pragma unroll 1
        for (unsigned q = q0; q < q1; ++q) mbar_wait_warp(&bar[q % D], (q / D) & 1u);
    }
};

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
    double w1[CPT], y1[CPT], w3[CPT], cprev[CPT];   // y1 = RN(1/w1)
    {
        double b0[CPT], f0[CPT];
        ld_stream<CPT>(pb, b0);
        ld_stream<CPT>(pf, f0);
        ld_stream<CPT>(pc, cprev);
#pragma unroll
        for (int j = 0; j < CPT; ++j) {
            w1[j] = b0[j];
            y1[j] = __drcp_rn(w1[j]);
            w3[j] = qdiv(f0[j], w1[j], y1[j]);
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
                    w2[j] = qdiv(cprev[j], w1[j], y1[j]);
                    w1[j] = xsub(rb[u][j], xmul(ra[u][j], w2[j]));
                    y1[j] = __drcp_rn(w1[j]);
                    w3[j] = qdiv(xsub(rf[u][j], xmul(ra[u][j], w3[j])), w1[j], y1[j]);
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

// Same sweep with w2 in a global scratch buffer instead of shared memory
// (element (k, slot) at scratch[k*S + slot], S resident threads): no shared
// memory limits residency, so a grid of register-limited size keeps every
// column of a batch in flight at once; the scratch lines stay in L2 between
// the forward and back sweeps.
template <int PF>
__global__ void __launch_bounds__(256) k_scalar_f64_g(SegTable tab, double *scratch, unsigned *status)
{
    const long S = (long)gridDim.x * blockDim.x;
    double *w2s = scratch + (long)blockIdx.x * blockDim.x + threadIdx.x;
    for (int t = blockIdx.x; t < tab.ntiles; t += gridDim.x) {
        const Seg s = tab.segs ? tab.segs[find_seg(tab, t)] : tab.one;
        const long col = (long)(t - s.tile0) * blockDim.x + threadIdx.x;
        if (col < s.ncol) report(status, s.status_idx, thomas_f64_cols<1, PF>(s, col, w2s, (int)S, 1));
    }
}

// ---------------------------------------------------------------------------
// Scalar Thomas, FP64, bit-exact, coefficients staged by bulk copies.
//
// One warp per CTA solves 32 adjacent columns.  a, b, c, f of level k arrive
// in a D-stage shared-memory ring (4 x 256 B per level), refilled D levels
// ahead, so a warp keeps 4*D*256 bytes of loads in flight without spending
// registers.  w2 goes to shared memory ([k][lane]), w3 is parked in x.
// Requires ld % 32 == 0 and 16-byte aligned array bases (checked on the host).
// With W2G, w2 goes to a global scratch slot (element k at w2s[k*S], S the
// resident lanes) instead of shared memory, so shared memory holds only the
// ring and every column of a batch can be resident at once.
// ---------------------------------------------------------------------------
template <int D, bool W2G>
__global__ void __launch_bounds__(256) k_scalar_f64_ring(SegTable tab, double *scratch, unsigned *status)
{
    constexpr int NE = 4;
    __shared__ __align__(8) unsigned long long bars[8 * D];
    extern __shared__ __align__(128) double smem_r[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    // each warp of the CTA is independent: its own ring, barriers and tiles
    const long per_warp = (long)D * NE * 32 + (W2G ? 0 : (long)32 * (tab.k2max > 1 ? tab.k2max - 1 : 1));
    double *mine = smem_r + warp * per_warp;
    Ring<NE, D> ring{mine, bars + warp * D, l2_policy(tab.hints, false)};
    const unsigned long long keep = l2_policy(tab.hints, true);
    const long ws = W2G ? (long)gridDim.x * blockDim.x : 32;
    double *w2s = W2G ? scratch + (long)blockIdx.x * blockDim.x + threadIdx.x : mine + D * NE * 32 + lane;
    ring.init(lane);
    unsigned q = 0;
    for (int t = blockIdx.x * nwarps + warp; t < tab.ntiles; t += gridDim.x * nwarps) {
        const Seg s = tab.segs ? tab.segs[find_seg(tab, t)] : tab.one;
        const long col0 = (long)(t - s.tile0) * 32;
        const long ld = s.ld;
        const int k2 = s.k2;
        const bool valid = col0 + lane < s.ncol;
        const double *src = (lane == 0 ? s.a : lane == 1 ? s.b : lane == 2 ? s.c : s.f) + col0;
        double *px = s.x + col0 + lane;
        const int pre = k2 < D ? k2 : D;
        for (int j = 0; j < pre; ++j) ring.issue(q + j, src + j * ld, lane);
        bool ok = true, fin = true;
        double w1 = 0.0, y1 = 0.0, w3 = 0.0, cprev = 0.0;
        for (int k = 0; k < k2; ++k) {
            const unsigned qk = q + k;
            if (!ring.wait(qk)) {
                ring.drain(qk, q + (k + D < k2 ? k + D : k2));
                if (lane == 0) report(status, s.status_idx, FLAG_TIMEOUT);
                return;
            }
            const double ak = ring.at(qk, 0, lane), bk = ring.at(qk, 1, lane), ck = ring.at(qk, 2, lane),
                         fk = ring.at(qk, 3, lane);
            __syncwarp();
            fence_proxy_async();
            if (k + D < k2) ring.issue(qk + D, src + (k + D) * ld, lane);
            if (valid) {
                if (k == 0) {
                    w1 = bk;
                    y1 = __drcp_rn(w1);
                    w3 = qdiv(fk, w1, y1);
                } else {
                    const double w2 = qdiv(cprev, w1, y1);
                    if (W2G) st_hint(&w2s[(k - 1) * ws], w2, keep);
                    else w2s[(k - 1) * ws] = w2;
                    w1 = xsub(bk, xmul(ak, w2));
                    y1 = __drcp_rn(w1);
                    w3 = qdiv(xsub(fk, xmul(ak, w3)), w1, y1);
                }
                ok = ok && finite_nz(w1);
                cprev = ck;
                st_hint(&px[k * ld], w3, keep);
            }
        }
        q += k2;
        if (valid) {
            // back sweep; w3 (in x) and w2 of the next 4 levels in flight
            double xn = w3;
            fin = finite(xn);
            double rw[4], r2[4];
#pragma unroll
            for (int u = 0; u < 4; ++u)
                if (k2 - 2 - u >= 0) {
                    rw[u] = px[(k2 - 2 - u) * ld];
                    r2[u] = w2s[(k2 - 2 - u) * ws];
                }
            for (int kb = k2 - 2; kb >= 0; kb -= 4) {
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    const int k = kb - u;
                    if (k >= 0) {
                        xn = xsub(rw[u], xmul(r2[u], xn));
                        fin = fin && finite(xn);
                        if (k - 4 >= 0) {
                            rw[u] = px[(k - 4) * ld];
                            r2[u] = w2s[(k - 4) * ws];
                        }
                        px[k * ld] = xn;
                    }
                }
            }
            report(status, s.status_idx, (ok ? 0u : FLAG_PIVOT) | (fin ? 0u : FLAG_NONFINITE));
        }
    }
}

// ---------------------------------------------------------------------------
// Scalar Thomas, FP64, bulk-copy ring of chunks: each of C stages holds L
// consecutive levels of the four coefficient arrays (4L copies of 256 B), so
// the mbarrier wait, proxy fence and copy issue happen once per L levels
// instead of once per level.  w2 in the L2 scratch slot of the lane, w3
// parked in x, as in k_scalar_f64_ring; same arithmetic, same bits.
// ---------------------------------------------------------------------------
template <int C, int L>
__global__ void __launch_bounds__(256) k_scalar_f64_chunk(SegTable tab, double *scratch, unsigned *status)
{
    constexpr int NE = 4 * L;
    static_assert(NE <= 32, "one copy per lane");
    __shared__ __align__(8) unsigned long long bars[8 * C];
    extern __shared__ __align__(128) double smem_r[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    double *buf = smem_r + (long)warp * C * NE * 32;
    unsigned long long *bar = bars + warp * C;
    const unsigned long long pol = l2_policy(tab.hints, false), keep = l2_policy(tab.hints, true);
    const long ws = (long)gridDim.x * blockDim.x;
    double *w2s = scratch + (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (lane == 0) {
#pragma unroll 1
        for (int i = 0; i < C; ++i) mbar_init(&bar[i], 1);
        fence_mbar_init();
    }
    __syncwarp();
    unsigned q = 0;
    for (int t = blockIdx.x * nwarps + warp; t < tab.ntiles; t += gridDim.x * nwarps) {
        const Seg s = tab.segs ? tab.segs[find_seg(tab, t)] : tab.one;
        const long col0 = (long)(t - s.tile0) * 32;
        const long ld = s.ld;
        const int k2 = s.k2;
        const bool valid = col0 + lane < s.ncol;
        const int arr = lane & 3;
        const double *src = (arr == 0 ? s.a : arr == 1 ? s.b : arr == 2 ? s.c : s.f) + col0 + (long)(lane >> 2) * ld;
        double *px = s.x + col0 + lane;
        const int nch = (k2 + L - 1) / L;
        // chunk j: levels j*L .. j*L+L-1 (those < k2) into stage (q + j) % C
        auto issue = [&](unsigned qc, int j) {
            const int st = (int)(qc % C), l0 = j * L;
            const int nl = k2 - l0 < L ? k2 - l0 : L;
            if (lane == 0) mbar_expect(&bar[st], (uint32_t)(4 * nl * 256));
            __syncwarp();
            if (lane < 4 * nl) bulk_load_hint(buf + (st * NE + lane) * 32, src + (long)l0 * ld, 256u, &bar[st], pol);
        };
        const int pre = nch < C ? nch : C;
        for (int j = 0; j < pre; ++j) issue(q + j, j);
        bool ok = true, fin = true;
        double w1 = 0.0, y1 = 0.0, w3 = 0.0, w2 = 0.0;   // w2: the next level's, from this pivot
        for (int j = 0; j < nch; ++j) {
            const unsigned qc = q + j;
            if (!mbar_wait_warp(&bar[qc % C], (qc / C) & 1u)) {
                const unsigned qe = q + (j + C < nch ? j + C : nch);
#pragma unroll 1
                for (unsigned r = qc; r < qe; ++r) mbar_wait_warp(&bar[r % C], (r / C) & 1u);
                if (lane == 0) report(status, s.status_idx, FLAG_TIMEOUT);
                return;
            }
            // the stage is read in place and handed back to the copy engine
            // after the L levels are done (registers stay low: more warps/SM)
            const double *stg = buf + (int)(qc % C) * NE * 32 + lane;
            // Level k from stage row l.  Both divisions by the pivot w1(k) are
            // done here: w3(k) = (f - a*w3(k-1))/w1(k) and the next level's
            // w2 = c(k)/w1(k) (the same operands as the reference's, so the
            // same correctly rounded quotients), under one range test.
            auto step = [&](int l, int k, bool first, bool last) {
                const double ak = stg[(4 * l + 0) * 32], bk = stg[(4 * l + 1) * 32], fk = stg[(4 * l + 3) * 32],
                             ck = stg[(4 * l + 2) * 32];
                w1 = first ? bk : xsub(bk, xmul(ak, w2));
                y1 = __drcp_rn(w1);
                const double num = first ? fk : xsub(fk, xmul(ak, w3));
                if (max(exp_dist(w1), max(exp_dist(num), exp_dist(ck))) < kExpSpan) {
                    w3 = div_markstein(num, w1, y1);
                    w2 = div_markstein(ck, w1, y1);
                } else {
                    const bool w1s = exp_safe(w1);
                    w3 = qdiv_pivot(num, w1, y1, w1s);
                    w2 = qdiv_pivot(ck, w1, y1, w1s);
                    // a pivot in the safe range is finite and nonzero
                    if (!w1s) ok = ok && finite_nz(w1);
                }
                if (!last) st_hint(&w2s[k * ws], w2, keep);
                st_hint(&px[k * ld], w3, keep);
            };
            if (valid) {
                if (j > 0 && (j + 1) * L < k2) {   // a full chunk, neither level 0 nor the top
#pragma unroll
                    for (int l = 0; l < L; ++l) step(l, j * L + l, false, false);
                } else {
#pragma unroll
                    for (int l = 0; l < L; ++l) {
                        const int k = j * L + l;
                        if (k < k2) step(l, k, k == 0, k + 1 == k2);
                    }
                }
            }
            __syncwarp();
            fence_proxy_async();
            if (j + C < nch) issue(qc + C, j + C);
        }
        q += nch;
        if (valid) {
            // A non-finite x(k+1) makes x(k) = w3 - w2*x(k+1) non-finite (inf
            // or NaN), down to x(0): x(0) finite <=> every x finite.
            double xn = w3;
            double rw[4], r2[4];
#pragma unroll
            for (int u = 0; u < 4; ++u)
                if (k2 - 2 - u >= 0) {
                    rw[u] = px[(k2 - 2 - u) * ld];
                    r2[u] = w2s[(k2 - 2 - u) * ws];
                }
            int kb = k2 - 2;
            for (; kb - 7 >= 0; kb -= 4) {   // four levels and their refills all in range
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    const int k = kb - u;
                    xn = xsub(rw[u], xmul(r2[u], xn));
                    rw[u] = px[(k - 4) * ld];
                    r2[u] = w2s[(k - 4) * ws];
                    px[k * ld] = xn;
                }
            }
            for (; kb >= 0; kb -= 4) {
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    const int k = kb - u;
                    if (k >= 0) {
                        xn = xsub(rw[u], xmul(r2[u], xn));
                        if (k - 4 >= 0) {
                            rw[u] = px[(k - 4) * ld];
                            r2[u] = w2s[(k - 4) * ws];
                        }
                        px[k * ld] = xn;
                    }
                }
            }
            fin = finite(xn);
            report(status, s.status_idx, (ok ? 0u : FLAG_PIVOT) | (fin ? 0u : FLAG_NONFINITE));
        }
    }
}

// ---------------------------------------------------------------------------
// Scalar Thomas, FP64, chunked bulk-copy ring with the column's sweep
// quantities resident in shared memory.  w2(k) of the warp's 32 columns for
// every level (and, with W3S, w3(k) too) stay in this warp's slice of shared
// memory from the forward sweep to the back sweep, so DRAM sees a, b, c, f
// read once and x written once; k_scalar_f64_chunk sends w2 to an L2 scratch
// slot and parks w3 in x, and part of that spills to DRAM when L2 is busy.
// Without W3S, w3 is still parked in x (an L2 line written and re-read), which
// halves the shared memory per warp: more warps per SM, more copies in flight.
// The first chunks of the warp's next tile are requested before its back
// sweep, so the copy engine keeps streaming while the warp substitutes.
// Same arithmetic and operation order as k_scalar_f64_chunk: same bits.
// Shared memory per warp: C*4L ring rows + (k2max-1) w2 rows (+ as many w3
// rows with W3S; the top level's w3 stays in a register), 256 B each.
// ---------------------------------------------------------------------------
__host__ __device__ constexpr long res_rows(int C, int L, int k2max, bool w3s)
{
    return (long)C * 4 * L + (long)(k2max > 1 ? k2max - 1 : 1) * (w3s ? 2 : 1);
}

template <int C, int L>
__device__ __forceinline__ void chunk_issue(double *buf, unsigned long long *bar, const double *src, long ld, int k2,
                                            unsigned qc, int j, int lane, unsigned long long pol)
{
    const int st = (int)(qc % C), l0 = j * L;
    const int nl = k2 - l0 < L ? k2 - l0 : L;
    if (lane == 0) mbar_expect(&bar[st], (uint32_t)(4 * nl * 256));
    __syncwarp();
    if (lane < 4 * nl) bulk_load_hint(buf + (st * 4 * L + lane) * 32, src + (long)l0 * ld, 256u, &bar[st], pol);
}

template <int C, int L, bool W3S>
__global__ void __launch_bounds__(256) k_scalar_f64_res(SegTable tab, unsigned *status)
{
    constexpr int NE = 4 * L;
    static_assert(NE <= 32, "one copy per lane");
    __shared__ __align__(8) unsigned long long bars[8 * C];
    extern __shared__ __align__(128) double smem_r[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    const int K = tab.k2max;
    double *buf = smem_r + (long)warp * res_rows(C, L, K, W3S) * 32;
    double *w2c = buf + C * NE * 32 + lane;                      // w2(k) at w2c[k*32]
    double *w3c = w2c + (long)(K > 1 ? K - 1 : 1) * 32;          // w3(k) at w3c[k*32] (W3S)
    unsigned long long *bar = bars + warp * C;
    const unsigned long long pol = l2_policy(tab.hints, false), keep = l2_policy(tab.hints, true);
    if (lane == 0) {
#pragma unroll 1
        for (int i = 0; i < C; ++i) mbar_init(&bar[i], 1);
        fence_mbar_init();
    }
    __syncwarp();
    const int arr = lane & 3;
    // this lane's copy source (row lane/4 of array lane%4) of tile t of segment s
    auto source = [&](const Seg &s, int t) -> const double * {
        return (arr == 0 ? s.a : arr == 1 ? s.b : arr == 2 ? s.c : s.f) + (long)(t - s.tile0) * 32 +
               (long)(lane >> 2) * s.ld;
    };
    const int tstride = gridDim.x * nwarps;
    unsigned q = 0;
    int issued = 0;   // chunks of the current tile requested during the previous tile
    for (int t = blockIdx.x * nwarps + warp; t < tab.ntiles; t += tstride) {
        const Seg s = tab.segs ? tab.segs[find_seg(tab, t)] : tab.one;
        const long col0 = (long)(t - s.tile0) * 32;
        const long ld = s.ld;
        const int k2 = s.k2;
        const bool valid = col0 + lane < s.ncol;
        const double *src = source(s, t);
        double *px = s.x + col0 + lane;
        const int nch = (k2 + L - 1) / L;
        const int pre = nch < C ? nch : C;
        for (int j = issued; j < pre; ++j) chunk_issue<C, L>(buf, bar, src, ld, k2, q + j, j, lane, pol);
        bool ok = true;
        double w1 = 0.0, y1 = 0.0, w3 = 0.0, w2 = 0.0;   // w2: the next level's, from this pivot
        for (int j = 0; j < nch; ++j) {
            const unsigned qc = q + j;
            if (!mbar_wait_warp(&bar[qc % C], (qc / C) & 1u)) {
                const unsigned qe = q + (j + C < nch ? j + C : nch);
#pragma unroll 1
                for (unsigned r = qc; r < qe; ++r) mbar_wait_warp(&bar[r % C], (r / C) & 1u);
                if (lane == 0) report(status, s.status_idx, FLAG_TIMEOUT);
                return;
            }
            const double *stg = buf + (int)(qc % C) * NE * 32 + lane;
            // level k from stage row l: both divisions by the pivot w1(k)
            // under one range test, as in k_scalar_f64_chunk
            auto step = [&](int l, int k, bool first, bool last) {
                const double ak = stg[(4 * l + 0) * 32], bk = stg[(4 * l + 1) * 32], fk = stg[(4 * l + 3) * 32],
                             ck = stg[(4 * l + 2) * 32];
                w1 = first ? bk : xsub(bk, xmul(ak, w2));
                y1 = __drcp_rn(w1);
                const double num = first ? fk : xsub(fk, xmul(ak, w3));
                if (max(exp_dist(w1), max(exp_dist(num), exp_dist(ck))) < kExpSpan) {
                    w3 = div_markstein(num, w1, y1);
                    w2 = div_markstein(ck, w1, y1);
                } else {
                    const bool w1s = exp_safe(w1);
                    w3 = qdiv_pivot(num, w1, y1, w1s);
                    w2 = qdiv_pivot(ck, w1, y1, w1s);
                    if (!w1s) ok = ok && finite_nz(w1);
                }
                if (!last) w2c[k * 32] = w2;
                if (W3S) {
                    if (!last) w3c[k * 32] = w3;
                } else {
                    st_hint(&px[k * ld], w3, keep);
                }
            };
            if (valid) {
                if (j > 0 && (j + 1) * L < k2) {   // a full chunk, neither level 0 nor the top
#pragma unroll
                    for (int l = 0; l < L; ++l) step(l, j * L + l, false, false);
                } else {
#pragma unroll
                    for (int l = 0; l < L; ++l) {
                        const int k = j * L + l;
                        if (k < k2) step(l, k, k == 0, k + 1 == k2);
                    }
                }
            }
            __syncwarp();
            fence_proxy_async();
            if (j + C < nch) chunk_issue<C, L>(buf, bar, src, ld, k2, qc + C, j + C, lane, pol);
        }
        q += nch;
        // the ring is free: request the next tile's first chunks before the
        // back sweep, which needs only the resident rows
        issued = 0;
        {
            const int tn = t + tstride;
            if (tn < tab.ntiles) {
                const Seg sn = tab.segs ? tab.segs[find_seg(tab, tn)] : tab.one;
                const int nchn = (sn.k2 + L - 1) / L;
                issued = nchn < C ? nchn : C;
                const double *srcn = source(sn, tn);
                for (int j = 0; j < issued; ++j) chunk_issue<C, L>(buf, bar, srcn, sn.ld, sn.k2, q + j, j, lane, pol);
            }
        }
        if (valid) {
            // x(k2-1) = w3(k2-1); a non-finite x(k+1) makes every lower x
            // non-finite, so x(0) finite <=> every x finite
            double xn = w3;
            if (W3S) {
                px[(k2 - 1) * ld] = xn;
#pragma unroll 4
                for (int k = k2 - 2; k >= 0; --k) {
                    xn = xsub(w3c[k * 32], xmul(w2c[k * 32], xn));
                    px[k * ld] = xn;
                }
            } else {
                double rw[4];
#pragma unroll
                for (int u = 0; u < 4; ++u)
                    if (k2 - 2 - u >= 0) rw[u] = px[(k2 - 2 - u) * ld];
                int kb = k2 - 2;
                for (; kb - 7 >= 0; kb -= 4) {   // four levels and their refills all in range
#pragma unroll
                    for (int u = 0; u < 4; ++u) {
                        const int k = kb - u;
                        xn = xsub(rw[u], xmul(w2c[k * 32], xn));
                        rw[u] = px[(k - 4) * ld];
                        px[k * ld] = xn;
                    }
                }
                for (; kb >= 0; kb -= 4) {
#pragma unroll
                    for (int u = 0; u < 4; ++u) {
                        const int k = kb - u;
                        if (k >= 0) {
                            xn = xsub(rw[u], xmul(w2c[k * 32], xn));
                            if (k - 4 >= 0) rw[u] = px[(k - 4) * ld];
                            px[k * ld] = xn;
                        }
                    }
                }
            }
            const bool fin = finite(xn);
            report(status, s.status_idx, (ok ? 0u : FLAG_PIVOT) | (fin ? 0u : FLAG_NONFINITE));
        }
        __syncwarp();
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
// Stopping rule of the refinement sweeps.  dmax = max|d| of this sweep's
// correction, xmax = max|x| after it, dprev = max|d| of the previous
// correction; for the first correction, max|x| of the FP32 sweep-0 solution
// (sweep 0 is the correction from x = 0).  Each sweep shrinks the error by a
// factor rho, estimated as dmax/dprev; the error left after applying d is
// then about dmax*rho/(1-rho).  A column stops when that estimate, or the
// correction itself, is below rel_tol*xmax.  The first estimate (from the
// sweep-0 solution rather than a correction) is the coarser one and must
// clear the tolerance by a factor 16.  With well-conditioned columns (rho
// near the FP32 rounding level) one correction suffices.
__device__ __forceinline__ bool refine_done(double dmax, double xmax, double dprev, double tol, bool first)
{
    if (dmax <= tol * xmax) return true;
    if (dprev > 0.0) {
        const double rho = dmax / dprev;
        const double margin = first ? 16.0 : 1.0;
        if (rho < 0.5 && margin * dmax * rho <= (1.0 - rho) * tol * xmax) return true;
    }
    return false;
}

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
    double xmax0 = 0.0;

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
        float xk = y, xm = fabsf(y);
        px[(k2 - 1) * ld] = (double)xk;
        for (int k = k2 - 2; k >= 0; --k) {
            xk = sy[k * T] - sw2[k * T] * xk;
            xm = fmaxf(xm, fabsf(xk));
            px[k * ld] = (double)xk;
        }
        xmax0 = (double)xm;
    }

    // ---- refinement sweeps
    bool conv = false;
    int sw = 0;
    double dprev = xmax0;
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
            if (refine_done(dmax, xmax, dprev, rf.rel_tol, sw == 1)) {
                conv = true;
                break;
            }
            dprev = dmax;
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
// Scalar Thomas, FP32 sweeps + FP64 refinement, coefficients staged by the
// bulk-copy ring (one warp per 32 columns, its own ring and barriers).
//
// Sweep 0 reads a, b, c, f rows through the ring (4L copies of 256 B per
// stage of L levels), factors in FP32 and solves.  The FP32 factors (w2,
// 1/w1) and the forward result y go to three float planes of a global
// scratch slot per resident lane ([plane][level][slot], kept in L2 by
// eviction hints), so shared memory holds only the ring.  Each correction
// sweep streams a, b, c, f, the x rows one level above and the 1/w1 rows
// (5L copies of 256 B and L of 128 B per stage), forms the FP64 residual,
// eliminates with the FP32 factors and back-substitutes x += d.  Stopping
// rule, cap, bit-exact FP64 fallback and flags as in k_scalar_refine.
// x and 1/w1 rows written by this warp's generic stores are read back by bulk
// copies: a proxy fence orders the two before each correction sweep.
// Requires ld % 32 == 0 and 16-byte aligned a, b, c, f, x.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void fence_proxy_async_global()
{
    asm volatile("fence.proxy.async.global;" ::: "memory");
}
__device__ __forceinline__ void st_hint_f(float *p, float v, unsigned long long pol)
{
    asm volatile("st.global.L2::cache_hint.f32 [%0], %1, %2;" ::"l"(p), "f"(v), "l"(pol) : "memory");
}

constexpr int kRefineStageLevels = 4;   // levels per ring stage of the refinement ring

template <int C>
__global__ void __launch_bounds__(256) k_scalar_refine_ring(SegTable tab, Refine rf, float *scratch, unsigned *status,
                                                            unsigned long long *hist)
{
    constexpr int L = kRefineStageLevels, NC = 4 * L, NE = 5 * L;
    constexpr int SD = NE * 32 + L * 16;   // doubles per stage: NE double rows, L float rows
    static_assert(NE + L <= 32, "one copy per lane");
    __shared__ __align__(8) unsigned long long bars[8 * C];
    extern __shared__ __align__(128) double smem_r[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    const long K = tab.k2max;
    double *buf = smem_r + (long)warp * C * SD;
    const long S = (long)gridDim.x * blockDim.x;            // slots: level stride of a plane
    const long slot0 = (long)blockIdx.x * blockDim.x + warp * 32;
    float *gw2 = scratch + slot0 + lane;                    // plane 0: w2(k)
    float *gri = gw2 + K * S;                               // plane 1: 1/w1(k)
    float *gy = gri + K * S;                                // plane 2: y(k)
    const float *rirow = scratch + K * S + slot0;           // row k of plane 1 for this warp
    unsigned long long *bar = bars + warp * C;
    const unsigned long long pol = refine_fill_policy(tab.hints), keep = l2_policy(tab.hints, true);
    if (lane == 0) {
#pragma unroll 1
        for (int i = 0; i < C; ++i) mbar_init(&bar[i], 1);
        fence_mbar_init();
    }
    __syncwarp();
    unsigned long long hl[kMaxSweepBins];
#pragma unroll
    for (int i = 0; i < kMaxSweepBins; ++i) hl[i] = 0ull;
    unsigned q = 0;
    for (int t = blockIdx.x * nwarps + warp; t < tab.ntiles; t += gridDim.x * nwarps) {
        const Seg s = tab.segs ? tab.segs[find_seg(tab, t)] : tab.one;
        const long col0 = (long)(t - s.tile0) * 32;
        const long ld = s.ld;
        const int k2 = s.k2;
        const bool valid = col0 + lane < s.ncol;
        double *px = s.x + col0 + lane;
        const int nch = (k2 + L - 1) / L;
        // lanes 0..4L-1: row (level lane/4) of array lane%4; lanes 4L..5L-1:
        // x row (lane - 4L + 1) above the chunk's first level; lanes
        // 5L..6L-1: 1/w1 row (lane - 5L)
        const int arr = lane & 3;
        const double *src = lane < NC ? (arr == 0 ? s.a : arr == 1 ? s.b : arr == 2 ? s.c : s.f) + col0 +
                                            (long)(lane >> 2) * ld
                                      : s.x + col0 + (long)(lane - NC + 1) * ld;
        auto issue = [&](unsigned qc, int j, bool corr) {
            const int st = (int)(qc % C), l0 = j * L;
            const int nl = k2 - l0 < L ? k2 - l0 : L;
            const int nx = corr ? (k2 - 1 - l0 < L ? k2 - 1 - l0 : L) : 0;
            if (lane == 0) mbar_expect(&bar[st], (uint32_t)(4 * nl + nx) * 256u + (corr ? (uint32_t)nl * 128u : 0u));
            __syncwarp();
            double *stg = buf + (long)st * SD;
            if (lane < NC) {
                if ((lane >> 2) < nl) bulk_load_hint(stg + lane * 32, src + (long)l0 * ld, 256u, &bar[st], pol);
            } else if (lane < NE) {
                if (lane - NC < nx) bulk_load_hint(stg + lane * 32, src + (long)l0 * ld, 256u, &bar[st], pol);
            } else if (lane < NE + L) {
                const int i = lane - NE;
                if (corr && i < nl)
                    bulk_load_hint(stg + NE * 32 + i * 16, rirow + (long)(l0 + i) * S, 128u, &bar[st], keep);
            }
        };
        // bounded wait for chunk j; on timeout drain the fills in flight
        auto wait = [&](unsigned q0, int j, int n) -> bool {
            const unsigned qc = q0 + j;
            if (mbar_wait_warp(&bar[qc % C], (qc / C) & 1u)) return true;
            const unsigned qe = q0 + (j + C < n ? j + C : n);
#pragma unroll 1
            for (unsigned r = qc; r < qe; ++r) mbar_wait_warp(&bar[r % C], (r / C) & 1u);
            if (lane == 0) report(status, s.status_idx, FLAG_TIMEOUT);
            return false;
        };

        // ---- sweep 0: FP32 factor + solve
        bool ok = true;
        float xm0 = 0.f;
        {
            const int pre = nch < C ? nch : C;
            for (int j = 0; j < pre; ++j) issue(q + j, j, false);
            float w1 = 0.f, ri = 0.f, y = 0.f, cprev = 0.f;
            for (int j = 0; j < nch; ++j) {
                if (!wait(q, j, nch)) return;
                const double *stg = buf + (long)((q + j) % C) * SD + lane;
                auto step0 = [&](int l, int k, bool first) {
                    const float af = (float)stg[(4 * l) * 32], bf = (float)stg[(4 * l + 1) * 32],
                                ff = (float)stg[(4 * l + 3) * 32];
                    if (first) {
                        w1 = bf;
                        ri = __frcp_rn(w1);
                        y = ff * ri;
                    } else {
                        const float w2 = cprev * ri;
                        st_hint_f(&gw2[(k - 1) * S], w2, keep);
                        w1 = bf - af * w2;
                        ri = __frcp_rn(w1);
                        y = (ff - af * y) * ri;
                    }
                    ok = ok && (fabsf(w1) <= FLT_MAX) && (w1 != 0.f);
                    st_hint_f(&gri[k * S], ri, keep);
                    st_hint_f(&gy[k * S], y, keep);
                    cprev = (float)stg[(4 * l + 2) * 32];
                };
                if (valid) {
                    if (j > 0 && (j + 1) * L <= k2) {   // a full chunk past level 0: no per-level tests
#pragma unroll
                        for (int l = 0; l < L; ++l) step0(l, j * L + l, false);
                    } else {
#pragma unroll
                        for (int l = 0; l < L; ++l)
                            if (j * L + l < k2) step0(l, j * L + l, j * L + l == 0);
                    }
                }
                __syncwarp();
                fence_proxy_async();
                if (j + C < nch) issue(q + j + C, j + C, false);
            }
            q += nch;
            if (valid) {
                // back substitution; y and w2 re-read 4 levels ahead
                float xk = y;
                xm0 = fabsf(y);
                px[(k2 - 1) * ld] = (double)xk;
                float ry[4], rw[4];
#pragma unroll
                for (int u = 0; u < 4; ++u)
                    if (k2 - 2 - u >= 0) {
                        ry[u] = gy[(k2 - 2 - u) * S];
                        rw[u] = gw2[(k2 - 2 - u) * S];
                    }
                for (int kb = k2 - 2; kb >= 0; kb -= 4) {
#pragma unroll
                    for (int u = 0; u < 4; ++u) {
                        const int k = kb - u;
                        if (k >= 0) {
                            xk = ry[u] - rw[u] * xk;
                            if (k - 4 >= 0) {
                                ry[u] = gy[(k - 4) * S];
                                rw[u] = gw2[(k - 4) * S];
                            }
                            xm0 = fmaxf(xm0, fabsf(xk));
                            st_hint(&px[k * ld], (double)xk, keep);
                        }
                    }
                }
            }
        }

        // ---- correction sweeps (the warp streams while any lane is active)
        bool active = valid && ok, conv = false;
        int sw = 0, taken = rf.max_sweeps + 1;   // sweep of convergence, else cap + 1
        double dprev = (double)xm0;
        for (sw = 1; sw <= rf.max_sweeps && __any_sync(0xffffffffu, active); ++sw) {
            fence_proxy_async_global();
            __syncwarp();
            const int pre = nch < C ? nch : C;
            for (int j = 0; j < pre; ++j) issue(q + j, j, true);
            double xm1 = 0.0, x0 = active ? px[0] : 0.0;
            float y = 0.f;
            for (int j = 0; j < nch; ++j) {
                if (!wait(q, j, nch)) return;
                const double *stg = buf + (long)((q + j) % C) * SD + lane;
                const float *stf = reinterpret_cast<const float *>(buf + (long)((q + j) % C) * SD + NE * 32) + lane;
                // level k from stage row l; `first` for level 0, `last` for k2-1
                auto step = [&](int l, int k, bool first, bool last) {
                    const double xp1 = last ? 0.0 : stg[(NC + l) * 32];
                    if (active) {
                        const double ak = stg[(4 * l) * 32];
                        double r = fma(-stg[(4 * l + 1) * 32], x0, stg[(4 * l + 3) * 32]);
                        if (!first) r = fma(-ak, xm1, r);
                        if (!last) r = fma(-stg[(4 * l + 2) * 32], xp1, r);
                        const float rr = (float)r, rik = stf[l * 32];
                        y = first ? rr * rik : (rr - (float)ak * y) * rik;
                        st_hint_f(&gy[k * S], y, keep);
                    }
                    xm1 = x0;
                    x0 = xp1;
                };
                if (j > 0 && (j + 1) * L < k2) {   // a full chunk, neither level 0 nor the top
#pragma unroll
                    for (int l = 0; l < L; ++l) step(l, j * L + l, false, false);
                } else {
#pragma unroll
                    for (int l = 0; l < L; ++l) {
                        const int k = j * L + l;
                        if (k < k2) step(l, k, k == 0, k + 1 == k2);
                    }
                }
                __syncwarp();
                fence_proxy_async();
                if (j + C < nch) issue(q + j + C, j + C, true);
            }
            q += nch;
            if (active) {
                // back substitution, x += d; x(k2-1) is in xm1; x, y and w2
                // of lower levels re-read 4 levels ahead
                float d = y;
                double xv = xm1 + (double)d;
                st_hint(&px[(k2 - 1) * ld], xv, keep);
                double dmax = fabs((double)d), xmax = fabs(xv);
                double rx[4];
                float ry[4], rw[4];
#pragma unroll
                for (int u = 0; u < 4; ++u)
                    if (k2 - 2 - u >= 0) {
                        rx[u] = px[(k2 - 2 - u) * ld];
                        ry[u] = gy[(k2 - 2 - u) * S];
                        rw[u] = gw2[(k2 - 2 - u) * S];
                    }
                for (int kb = k2 - 2; kb >= 0; kb -= 4) {
#pragma unroll
                    for (int u = 0; u < 4; ++u) {
                        const int k = kb - u;
                        if (k >= 0) {
                            d = ry[u] - rw[u] * d;
                            xv = rx[u] + (double)d;
                            if (k - 4 >= 0) {
                                rx[u] = px[(k - 4) * ld];
                                ry[u] = gy[(k - 4) * S];
                                rw[u] = gw2[(k - 4) * S];
                            }
                            st_hint(&px[k * ld], xv, keep);
                            dmax = fmax(dmax, fabs((double)d));
                            xmax = fmax(xmax, fabs(xv));
                        }
                    }
                }
                if (!(xmax <= DBL_MAX) || !(dmax <= DBL_MAX)) {
                    active = false;
                } else if (refine_done(dmax, xmax, dprev, rf.rel_tol, sw == 1)) {
                    conv = true;
                    active = false;
                    taken = sw;
                } else {
                    dprev = dmax;
                }
            }
        }
        unsigned flags = 0u;
        if (valid && !conv) {
            // ---- fallback: bit-exact FP64 re-solve; w2 as two 32-bit halves
            // in this lane's w2 and 1/w1 plane slots, w3 parked in x
            const double *pa = s.a + col0 + lane, *pb = s.b + col0 + lane, *pc = s.c + col0 + lane,
                         *pf = s.f + col0 + lane;
            bool okd = true, fin = true;
            double w1 = pb[0], w3 = xdiv(pf[0], w1);
            okd = finite_nz(w1);
            px[0] = w3;
            double cprev = pc[0];
            for (int k = 1; k < k2; ++k) {
                const double ak = pa[k * ld], bk = pb[k * ld], fk = pf[k * ld];
                const double w2 = xdiv(cprev, w1);
                gw2[(k - 1) * S] = __int_as_float(__double2hiint(w2));
                gri[(k - 1) * S] = __int_as_float(__double2loint(w2));
                w1 = xsub(bk, xmul(ak, w2));
                w3 = xdiv(xsub(fk, xmul(ak, w3)), w1);
                okd = okd && finite_nz(w1);
                px[k * ld] = w3;
                cprev = pc[k * ld];
            }
            double xn = w3;
            fin = finite(xn);
            for (int k = k2 - 2; k >= 0; --k) {
                const double w2 = __hiloint2double(__float_as_int(gw2[k * S]), __float_as_int(gri[k * S]));
                xn = xsub(px[k * ld], xmul(w2, xn));
                fin = fin && finite(xn);
                px[k * ld] = xn;
            }
            flags = FLAG_NOCONV | (okd ? 0u : FLAG_PIVOT) | (fin ? 0u : FLAG_NONFINITE);
        }
        if (valid) report(status, s.status_idx, flags);
        const int bin = taken < kMaxSweepBins - 1 ? taken : kMaxSweepBins - 1;
#pragma unroll
        for (int i = 0; i < kMaxSweepBins; ++i) hl[i] += __popc(__ballot_sync(0xffffffffu, valid && bin == i));
    }
    if (hist && lane == 0)
#pragma unroll
        for (int i = 0; i < kMaxSweepBins; ++i)
            if (hl[i]) atomicAdd(hist + i, hl[i]);
}

// ---------------------------------------------------------------------------
// Scalar refinement with the whole tile on chip: the FP64 a, b, c, f of the
// warp's 32 columns for every level arrive once (one mbarrier transaction of
// 4*k2 bulk copies), and sweep 0, every residual, every correction and an
// FP64 fallback run from shared memory, with x (FP64) and the FP32 factors
// beside them; x goes to HBM once.  DRAM sees 40 B per unknown, at the price
// of (5 doubles + 3 floats) per level and column of shared memory: 95 KB per
// warp at 57 levels, two warps per SM.  Same stopping rule and FP64 fallback
// as k_scalar_refine_ring.
// ---------------------------------------------------------------------------
constexpr int kRefineTileBytesPerLevel = 32 * (5 * 8 + 3 * 4);

__global__ void __launch_bounds__(32) k_scalar_refine_tile(SegTable tab, Refine rf, unsigned *status,
                                                           unsigned long long *hist)
{
    extern __shared__ __align__(128) double smem_t[];
    __shared__ __align__(8) unsigned long long bar;
    const int lane = threadIdx.x;
    const long K = tab.k2max;
    double *A = smem_t;                                  // plane p (a, b, c, f) row k at (p*K + k)*32
    double *X = A + 4 * K * 32;                          // x(k) at k*32
    float *W2 = reinterpret_cast<float *>(X + K * 32);   // w2(k), 1/w1(k), y(k) at k*32
    float *RI = W2 + K * 32;
    float *Y = RI + K * 32;
    const unsigned long long pol = l2_policy(tab.hints, false);
    if (lane == 0) {
        mbar_init(&bar, 1);
        fence_mbar_init();
    }
    __syncwarp();
    unsigned long long hl[kMaxSweepBins];
#pragma unroll
    for (int i = 0; i < kMaxSweepBins; ++i) hl[i] = 0ull;
    unsigned phase = 0;
    for (int t = blockIdx.x; t < tab.ntiles; t += gridDim.x) {
        const Seg s = tab.segs ? tab.segs[find_seg(tab, t)] : tab.one;
        const long col0 = (long)(t - s.tile0) * 32;
        const long ld = s.ld;
        const int k2 = s.k2;
        const bool valid = col0 + lane < s.ncol;
        // the tile's 4*k2 rows of 256 B, one transaction
        if (lane == 0) mbar_expect(&bar, (uint32_t)(4 * k2 * 256));
        __syncwarp();
        for (int r = lane; r < 4 * k2; r += 32) {
            const int p = r & 3, k = r >> 2;
            const double *src = (p == 0 ? s.a : p == 1 ? s.b : p == 2 ? s.c : s.f) + (long)k * ld + col0;
            bulk_load_hint(A + ((long)p * K + k) * 32, src, 256u, &bar, pol);
        }
        if (!mbar_wait_warp(&bar, phase)) {
            mbar_wait_warp(&bar, phase);
            if (lane == 0) report(status, s.status_idx, FLAG_TIMEOUT);
            return;
        }
        phase ^= 1u;
        const double *pa = A + lane, *pb = A + K * 32 + lane, *pc = A + 2 * K * 32 + lane, *pf = A + 3 * K * 32 + lane;
        double *px = X + lane;
        float *pw2 = W2 + lane, *pri = RI + lane, *py = Y + lane;
        // ---- sweep 0: FP32 factor and solve
        bool ok = true;
        float xm0 = 0.f;
        if (valid) {
            float w1 = (float)pb[0], ri = __frcp_rn(w1), y = (float)pf[0] * ri;
            ok = (fabsf(w1) <= FLT_MAX) && (w1 != 0.f);
            pri[0] = ri;
            py[0] = y;
            for (int k = 1; k < k2; ++k) {
                const float af = (float)pa[k * 32];
                const float w2 = (float)pc[(k - 1) * 32] * ri;
                pw2[(k - 1) * 32] = w2;
                w1 = (float)pb[k * 32] - af * w2;
                ri = __frcp_rn(w1);
                y = ((float)pf[k * 32] - af * y) * ri;
                ok = ok && (fabsf(w1) <= FLT_MAX) && (w1 != 0.f);
                pri[k * 32] = ri;
                py[k * 32] = y;
            }
            float xk = y;
            xm0 = fabsf(xk);
            px[(k2 - 1) * 32] = (double)xk;
            for (int k = k2 - 2; k >= 0; --k) {
                xk = py[k * 32] - pw2[k * 32] * xk;
                xm0 = fmaxf(xm0, fabsf(xk));
                px[k * 32] = (double)xk;
            }
        }
        // ---- corrections: FP64 residual from the tile, FP32 solve, x += d
        bool active = valid && ok, conv = false;
        int taken = rf.max_sweeps + 1;
        double dprev = (double)xm0;
        for (int sw = 1; sw <= rf.max_sweeps && active; ++sw) {
            double xm1 = 0.0, x0 = px[0];
            float y = 0.f;
            for (int k = 0; k < k2; ++k) {
                const double xp1 = k + 1 < k2 ? px[(k + 1) * 32] : 0.0;
                const double ak = pa[k * 32];
                double r = fma(-pb[k * 32], x0, pf[k * 32]);
                if (k > 0) r = fma(-ak, xm1, r);
                if (k + 1 < k2) r = fma(-pc[k * 32], xp1, r);
                const float rr = (float)r;
                y = k == 0 ? rr * pri[0] : (rr - (float)ak * y) * pri[k * 32];
                py[k * 32] = y;
                xm1 = x0;
                x0 = xp1;
            }
            float d = y;
            double xv = px[(k2 - 1) * 32] + (double)d;
            px[(k2 - 1) * 32] = xv;
            double dmax = fabs((double)d), xmax = fabs(xv);
            for (int k = k2 - 2; k >= 0; --k) {
                d = py[k * 32] - pw2[k * 32] * d;
                xv = px[k * 32] + (double)d;
                px[k * 32] = xv;
                dmax = fmax(dmax, fabs((double)d));
                xmax = fmax(xmax, fabs(xv));
            }
            if (!(xmax <= DBL_MAX) || !(dmax <= DBL_MAX)) {
                active = false;
            } else if (refine_done(dmax, xmax, dprev, rf.rel_tol, sw == 1)) {
                conv = true;
                active = false;
                taken = sw;
            } else {
                dprev = dmax;
            }
        }
        unsigned flags = 0u;
        if (valid && !conv) {
            // FP64 re-solve from the tile (bit-exact; w3 in x, w2 in the two
            // float planes' halves)
            bool okd = true;
            double w1 = pb[0], w3 = xdiv(pf[0], w1);
            okd = finite_nz(w1);
            px[0] = w3;
            for (int k = 1; k < k2; ++k) {
                const double ak = pa[k * 32];
                const double w2 = xdiv(pc[(k - 1) * 32], w1);
                pw2[(k - 1) * 32] = __int_as_float(__double2hiint(w2));
                pri[(k - 1) * 32] = __int_as_float(__double2loint(w2));
                w1 = xsub(pb[k * 32], xmul(ak, w2));
                w3 = xdiv(xsub(pf[k * 32], xmul(ak, w3)), w1);
                okd = okd && finite_nz(w1);
                px[k * 32] = w3;
            }
            double xn = w3;
            bool fin = finite(xn);
            for (int k = k2 - 2; k >= 0; --k) {
                const double w2 = __hiloint2double(__float_as_int(pw2[k * 32]), __float_as_int(pri[k * 32]));
                xn = xsub(px[k * 32], xmul(w2, xn));
                fin = fin && finite(xn);
                px[k * 32] = xn;
            }
            flags = FLAG_NOCONV | (okd ? 0u : FLAG_PIVOT) | (fin ? 0u : FLAG_NONFINITE);
        }
        if (valid) {
            double *gx = s.x + col0 + lane;
            for (int k = 0; k < k2; ++k) gx[k * ld] = px[k * 32];
            report(status, s.status_idx, flags);
        }
        const int bin = taken < kMaxSweepBins - 1 ? taken : kMaxSweepBins - 1;
#pragma unroll
        for (int i = 0; i < kMaxSweepBins; ++i) hl[i] += __popc(__ballot_sync(0xffffffffu, valid && bin == i));
        // every lane is done with the tile before the next one's copies land
        __syncwarp();
        fence_proxy_async();
    }
    if (hist && lane == 0)
#pragma unroll
        for (int i = 0; i < kMaxSweepBins; ++i)
            if (hl[i]) atomicAdd(hist + i, hl[i]);
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
    const double y = __drcp_rn(d);
    const bool ds = exp_safe(d);
    // one range test for the pivot and all four numerators (a sign does not
    // change the exponent); any out of range: each division on its own
    if (max(max(exp_dist(d), exp_dist(A[0])), max(max(exp_dist(A[1]), exp_dist(A[2])), exp_dist(A[3]))) < kExpSpan) {
        W[0] = div_markstein(A[3], d, y);
        W[1] = div_markstein(-A[1], d, y);
        W[2] = div_markstein(-A[2], d, y);
        W[3] = div_markstein(A[0], d, y);
        return true;
    }
    W[0] = qdiv_pivot(A[3], d, y, ds);
    W[1] = qdiv_pivot(-A[1], d, y, ds);
    W[2] = qdiv_pivot(-A[2], d, y, ds);
    W[3] = qdiv_pivot(A[0], d, y, ds);
    return ds || finite_nz(d);
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
    const double y = __drcp_rn(d);
    const bool ds = exp_safe(d);
    unsigned dm = exp_dist(d);
#pragma unroll
    for (int e = 0; e < 9; ++e) dm = max(dm, exp_dist(W[e]));
    if (dm < kExpSpan) {   // pivot and all nine numerators in range: one test
#pragma unroll
        for (int e = 0; e < 9; ++e) W[e] = div_markstein(W[e], d, y);
        return true;
    }
#pragma unroll
    for (int e = 0; e < 9; ++e) W[e] = qdiv_pivot(W[e], d, y, ds);
    return ds || finite_nz(d);
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
// Back sweep u_k = z_{k+1} - Gamma_{k+1} u_{k+1} for k = k2-2..0 (z parked in
// u, Gamma in the scratch slots), keeping the loads of the next BPF levels in
// flight: every level's operands come from L2, so an unprefetched sweep would
// wait a full L2 round trip per level.  un holds u_{k2-1} on entry.
template <int B>
__device__ __forceinline__ bool blk_back(double *pU, long ld, const double *gam, long gs, int k2, double (&un)[B])
{
    constexpr int BB = B * B, BPF = B == 2 ? 4 : 2;
    bool fin = true;
    double rz[BPF][B], rg[BPF][BB];
    // level k of u (z parked there) and of Gamma; rows BPF levels apart
    const long su = (long)B * ld, sg = (long)BB * gs;
#pragma unroll
    for (int u = 0; u < BPF; ++u) {
        const int k = k2 - 2 - u;
        if (k >= 0) {
#pragma unroll
            for (int i = 0; i < B; ++i) rz[u][i] = pU[k * su + i * ld];
#pragma unroll
            for (int e = 0; e < BB; ++e) rg[u][e] = gam[k * sg + e * gs];
        }
    }
    double *uk = pU + (long)(k2 - 2) * su;
    const double *gn = gam + (long)(k2 - 2 - BPF) * sg;   // refill rows: level k - BPF
    for (int kb = k2 - 2; kb >= 0; kb -= BPF) {
#pragma unroll
        for (int u = 0; u < BPF; ++u) {
            const int k = kb - u;
            if (k >= 0) {
                double nu[B];
#pragma unroll
                for (int i = 0; i < B; ++i) {
                    double t = rz[u][i];
#pragma unroll
                    for (int m = 0; m < B; ++m) t = xsub(t, xmul(rg[u][i + B * m], un[m]));
                    nu[i] = t;
                    fin = fin && finite(t);
                }
                if (k - BPF >= 0) {
                    const double *un_src = uk - BPF * su;
#pragma unroll
                    for (int i = 0; i < B; ++i) rz[u][i] = un_src[i * ld];
#pragma unroll
                    for (int e = 0; e < BB; ++e) rg[u][e] = gn[e * gs];
                }
#pragma unroll
                for (int i = 0; i < B; ++i) {
                    un[i] = nu[i];
                    uk[i * ld] = nu[i];
                }
                uk -= su;
                gn -= sg;
            }
        }
    }
    return fin;
}

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
    fin = blk_back<B>(pU, ld, gam, gs, k2, un) && fin;
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
// Block-tridiagonal Thomas, FP64, bit-exact, coefficients staged by bulk
// copies: one warp per CTA, 32 columns; the 3*B*B + B entries of a level
// (P, Q, R, f) arrive in a D-stage shared-memory ring, one 256-byte copy per
// entry issued by one lane.  Same arithmetic as blk_f64_col.
// ---------------------------------------------------------------------------
// With GSM, Gamma of the warp's columns stays in the warp's slice of shared
// memory for every level (k2max-1 rows of B*B*W doubles after the ring)
// instead of an L2 scratch slot, so DRAM sees P, Q, R, f read once and u
// written once (z is still parked in u, a small L2 footprint); and the next
// tile's first D levels are requested before the back sweep, which needs only
// Gamma and the parked z.  Same arithmetic, same bits.
template <int B, int D, int W, bool GSM = false>
__global__ void __launch_bounds__(256) k_block_f64_ring(SegTable tab, double *scratch, unsigned *status)
{
    // W < 32: a warp covers W columns (lanes >= W idle), so that more warps
    // share the SM's issue slots when there are few columns
    constexpr int BB = B * B, NE = 3 * BB + B, NSUB = 32 / W;
    __shared__ __align__(8) unsigned long long bars[8 * D];
    extern __shared__ __align__(128) double smem_b[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    const int cl = lane & (W - 1);            // column of this lane within the tile (idle lanes alias)
    const long gsm_rows = GSM ? (long)(tab.k2max > 1 ? tab.k2max - 1 : 1) * BB : 0;
    double *wbase = smem_b + (long)warp * (D * NE * W + gsm_rows * W);
    Ring<NE, D, W> ring{wbase, bars + warp * D, l2_policy(tab.hints, false)};
    const unsigned long long keep = l2_policy(tab.hints, true);
    ring.init(lane);
    const long gs = GSM ? (long)W : (long)gridDim.x * nwarps * W;
    double *gam = GSM ? wbase + D * NE * W + cl : scratch + ((long)blockIdx.x * nwarps + warp) * W + cl;
    // this lane's copy source (entry `lane` of level 0) of the tile at col0
    // of segment s, and its level stride
    auto source = [&](const Seg &s, long col0, long &lstride) -> const double * {
        const long ld = s.ld;
        lstride = 0;
        if (lane < BB) {
            lstride = BB * ld;
            return s.a + col0 + lane * ld;
        }
        if (lane < 2 * BB) {
            lstride = BB * ld;
            return s.b + col0 + (lane - BB) * ld;
        }
        if (lane < 3 * BB) {
            lstride = BB * ld;
            return s.c + col0 + (lane - 2 * BB) * ld;
        }
        if (lane < NE) {
            lstride = B * ld;
            return s.f + col0 + (lane - 3 * BB) * ld;
        }
        return s.a + col0;
    };
    const int vstride = gridDim.x * nwarps;
    unsigned q = 0;
    int pref_vt = -1;   // a tile whose first levels were requested during the previous one
    for (int vt = blockIdx.x * nwarps + warp; vt < tab.ntiles * NSUB; vt += vstride) {
        const int t = vt / NSUB;
        const Seg s = tab.segs ? tab.segs[find_seg(tab, t)] : tab.one;
        const long col0 = (long)(t - s.tile0) * 32 + (long)(vt % NSUB) * W;
        if (col0 >= s.ncol) continue;        // uniform across the warp
        const long ld = s.ld;
        const int k2 = s.k2;
        const bool valid = lane < W && col0 + lane < s.ncol;
        // entry e of level k: P/Q/R element e at (k*BB + e)*ld, f component at (k*B + i)*ld
        long lstride = 0;
        const double *src = source(s, col0, lstride);
        double *pU = s.x + col0 + cl;
        const int pre = k2 < D ? k2 : D;
        if (pref_vt != vt)
            for (int j = 0; j < pre; ++j) ring.issue(q + j, src + j * lstride, lane);
        pref_vt = -1;
        bool ok = true;
        double G[BB], z[B];
        double *pUk = pU, *gk = gam;   // level k of the parked z and of Gamma
        for (int k = 0; k < k2; ++k, pUk += B * ld, gk += BB * gs) {
            const unsigned qk = q + k;
            if (!ring.wait(qk)) {
                ring.drain(qk, q + (k + D < k2 ? k + D : k2));
                if (lane == 0) report(status, s.status_idx, FLAG_TIMEOUT);
                return;
            }
            double P[BB], Q[BB], R[BB], F[B];
#pragma unroll
            for (int e = 0; e < BB; ++e) {
                P[e] = ring.at(qk, e, cl);
                Q[e] = ring.at(qk, BB + e, cl);
                R[e] = ring.at(qk, 2 * BB + e, cl);
            }
#pragma unroll
            for (int i = 0; i < B; ++i) F[i] = ring.at(qk, 3 * BB + i, cl);
            __syncwarp();
            fence_proxy_async();
            if (k + D < k2) ring.issue(qk + D, src + (k + D) * lstride, lane);
            if (!valid) continue;
            double Qp[BB], Wi[BB], v[B];
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
                        double qv = Q[i + B * m];
#pragma unroll
                        for (int n = 0; n < B; ++n) qv = xsub(qv, xmul(P[i + B * n], G[n + B * m]));
                        Qp[i + B * m] = qv;
                    }
#pragma unroll
                for (int i = 0; i < B; ++i) {
                    double tv = F[i];
#pragma unroll
                    for (int m = 0; m < B; ++m) tv = xsub(tv, xmul(P[i + B * m], z[m]));
                    v[i] = tv;
                }
            }
            ok = inv_exact<B>(Qp, Wi) && ok;
#pragma unroll
            for (int i = 0; i < B; ++i) {
                double tv = xmul(Wi[i], v[0]);
#pragma unroll
                for (int m = 1; m < B; ++m) tv = xadd(tv, xmul(Wi[i + B * m], v[m]));
                z[i] = tv;
                st_hint(&pUk[(long)i * ld], tv, keep);
            }
            if (k < k2 - 1) {
#pragma unroll
                for (int m = 0; m < B; ++m)
#pragma unroll
                    for (int i = 0; i < B; ++i) {
                        double g = xmul(Wi[i], R[B * m]);
#pragma unroll
                        for (int n = 1; n < B; ++n) g = xadd(g, xmul(Wi[i + B * n], R[n + B * m]));
                        G[i + B * m] = g;
                        if (GSM)
                            gk[(long)(i + B * m) * gs] = g;
                        else
                            st_hint(&gk[(long)(i + B * m) * gs], g, keep);
                    }
            }
        }
        q += k2;
        if (GSM) {
            // the ring is free: request the next tile's first levels before
            // the back sweep (only when that tile is one this warp solves)
            const int vn = vt + vstride;
            if (vn < tab.ntiles * NSUB) {
                const int tn = vn / NSUB;
                const Seg sn = tab.segs ? tab.segs[find_seg(tab, tn)] : tab.one;
                const long c0n = (long)(tn - sn.tile0) * 32 + (long)(vn % NSUB) * W;
                if (c0n < sn.ncol) {
                    long lsn = 0;
                    const double *srcn = source(sn, c0n, lsn);
                    const int pren = sn.k2 < D ? sn.k2 : D;
                    for (int j = 0; j < pren; ++j) ring.issue(q + j, srcn + j * lsn, lane);
                    pref_vt = vn;
                }
            }
        }
        if (!valid) continue;
        bool fin = true;
        double un[B], top[B];
#pragma unroll
        for (int i = 0; i < B; ++i) {
            un[i] = z[i];
            top[i] = z[i];
            fin = fin && finite(z[i]);
        }
        fin = blk_back<B>(pU, ld, gam, gs, k2, un) && fin;
        if (s.ubc_ratio) {
#pragma unroll
            for (int i = 0; i < B; ++i) {
                double tv = xmul(__ldg(s.ubc_ratio + i * ld + col0 + cl), top[i]);
                if (s.ubc_add) tv = xadd(tv, __ldg(s.ubc_add + i * ld + col0 + cl));
                fin = fin && finite(tv);
                pU[((long)k2 * B + i) * ld] = tv;
            }
        }
        report(status, s.status_idx, (ok ? 0u : FLAG_PIVOT) | (fin ? 0u : FLAG_NONFINITE));
    }
}

// ---------------------------------------------------------------------------
// Block-tridiagonal Thomas, FP64, bit-exact, one lane per block row.  The
// block recurrence of a single column is a long chain of dependent FP64
// operations (about 400 warp instructions per level for B = 2 with one lane
// per column), and a 2.5 deg grid has only ~2 such warps per SM, so the
// single-lane kernel runs at the latency of that chain.  Here the B rows of a
// column go to B lanes of a group of G lanes (G = 2 for B = 2, 4 for B = 3
// with one helper lane), a warp covers 32/G columns, and each lane computes
// its row of Q' = Q - P Gamma, of W = inv(Q') (the determinant and cofactors
// redundantly, its own B divisions), of z and of Gamma; whole rows, blocks
// and vectors are exchanged by shuffles within the group.  Every element is
// formed by the same operations in the same order as blk_f64_col, so the
// result is bit-identical.  Coefficients arrive through the bulk-copy ring
// (entries of 32/G columns), Gamma goes to the column's L2 scratch slot, z is
// parked in u.
// ---------------------------------------------------------------------------
template <int B, int D>
__global__ void __launch_bounds__(256) k_block_f64_rows(SegTable tab, double *scratch, unsigned *status)
{
    constexpr int BB = B * B, NE = 3 * BB + B, G = B == 2 ? 2 : 4, W = 32 / G;
    constexpr unsigned FULL = 0xffffffffu;
    __shared__ __align__(8) unsigned long long bars[8 * D];
    extern __shared__ __align__(128) double smem_b[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    const int c = lane / G, ri = lane % G, base = lane - ri;
    const int i = ri < B ? ri : B - 1;       // the helper lane of B = 3 mirrors row B-1
    const bool row_lane = ri < B;
    const unsigned gmask = ((1u << G) - 1u) << base;
    Ring<NE, D, W> ring{smem_b + (long)warp * D * NE * W, bars + warp * D, l2_policy(tab.hints, false)};
    const unsigned long long keep = l2_policy(tab.hints, true);
    ring.init(lane);
    const long gs = (long)gridDim.x * nwarps * W;
    double *gam = scratch + ((long)blockIdx.x * nwarps + warp) * W + c;
    unsigned q = 0;
    const int nvt = tab.ntiles * G;          // sub-tiles of W columns
    for (int vt = blockIdx.x * nwarps + warp; vt < nvt; vt += gridDim.x * nwarps) {
        const int t = vt / G, sub = vt % G;
        const Seg s = tab.segs ? tab.segs[find_seg(tab, t)] : tab.one;
        const long col0 = (long)(t - s.tile0) * 32 + (long)sub * W;
        if (col0 >= s.ncol) continue;        // uniform across the warp
        const long ld = s.ld;
        const int k2 = s.k2;
        const bool valid = col0 + c < s.ncol;
        const double *src = s.a + col0;
        long lstride = 0;
        if (lane < BB) {
            src = s.a + col0 + lane * ld;
            lstride = BB * ld;
        } else if (lane < 2 * BB) {
            src = s.b + col0 + (lane - BB) * ld;
            lstride = BB * ld;
        } else if (lane < 3 * BB) {
            src = s.c + col0 + (lane - 2 * BB) * ld;
            lstride = BB * ld;
        } else if (lane < NE) {
            src = s.f + col0 + (lane - 3 * BB) * ld;
            lstride = B * ld;
        }
        double *pU = s.x + col0 + c;
        const int pre = k2 < D ? k2 : D;
        for (int j = 0; j < pre; ++j) ring.issue(q + j, src + j * lstride, lane);
        bool ok = true;
        double Gf[BB], z[B];
        for (int k = 0; k < k2; ++k) {
            const unsigned qk = q + k;
            if (!ring.wait(qk)) {
                ring.drain(qk, q + (k + D < k2 ? k + D : k2));
                if (lane == 0) report(status, s.status_idx, FLAG_TIMEOUT);
                return;
            }
            double P[B], Qr[B], R[BB], fi;
#pragma unroll
            for (int n = 0; n < B; ++n) {
                P[n] = ring.at(qk, i + B * n, c);
                Qr[n] = ring.at(qk, BB + i + B * n, c);
            }
#pragma unroll
            for (int e = 0; e < BB; ++e) R[e] = ring.at(qk, 2 * BB + e, c);
            fi = ring.at(qk, 3 * BB + i, c);
            __syncwarp();
            fence_proxy_async();
            if (k + D < k2) ring.issue(qk + D, src + (k + D) * lstride, lane);
            // row i of Q' = Q - P Gamma, then the whole Q' of the column
            double Qp[B];
#pragma unroll
            for (int m = 0; m < B; ++m) {
                double qv = Qr[m];
                if (k > 0) {
#pragma unroll
                    for (int n = 0; n < B; ++n) qv = xsub(qv, xmul(P[n], Gf[n + B * m]));
                }
                Qp[m] = qv;
            }
            double A[BB];
#pragma unroll
            for (int n = 0; n < B; ++n)
#pragma unroll
                for (int m = 0; m < B; ++m) A[n + B * m] = __shfl_sync(FULL, Qp[m], base + n);
            // row i of W = inv(Q') (inv_exact's operations)
            double d, Wn[B];
            if (B == 2) {
                d = xsub(xmul(A[0], A[3]), xmul(A[2], A[1]));
                Wn[0] = i == 0 ? A[3] : -A[1];
                Wn[1] = i == 0 ? -A[2] : A[0];
            } else {
#define a_(r, q2) A[((r) - 1) + 3 * ((q2) - 1)]
                d = xmul(xmul(a_(1, 1), a_(2, 2)), a_(3, 3));
                d = xsub(d, xmul(xmul(a_(1, 1), a_(2, 3)), a_(3, 2)));
                d = xsub(d, xmul(xmul(a_(1, 2), a_(2, 1)), a_(3, 3)));
                d = xadd(d, xmul(xmul(a_(1, 2), a_(2, 3)), a_(3, 1)));
                d = xadd(d, xmul(xmul(a_(1, 3), a_(2, 1)), a_(3, 2)));
                d = xsub(d, xmul(xmul(a_(1, 3), a_(2, 2)), a_(3, 1)));
                double w[9];
                w[0] = xsub(xmul(a_(2, 2), a_(3, 3)), xmul(a_(2, 3), a_(3, 2)));
                w[1] = -xsub(xmul(a_(2, 1), a_(3, 3)), xmul(a_(2, 3), a_(3, 1)));
                w[2] = xsub(xmul(a_(2, 1), a_(3, 2)), xmul(a_(2, 2), a_(3, 1)));
                w[3] = -xsub(xmul(a_(1, 2), a_(3, 3)), xmul(a_(1, 3), a_(3, 2)));
                w[4] = xsub(xmul(a_(1, 1), a_(3, 3)), xmul(a_(1, 3), a_(3, 1)));
                w[5] = -xsub(xmul(a_(1, 1), a_(3, 2)), xmul(a_(1, 2), a_(3, 1)));
                w[6] = xsub(xmul(a_(1, 2), a_(2, 3)), xmul(a_(1, 3), a_(2, 2)));
                w[7] = -xsub(xmul(a_(1, 1), a_(2, 3)), xmul(a_(1, 3), a_(2, 1)));
                w[8] = xsub(xmul(a_(1, 1), a_(2, 2)), xmul(a_(1, 2), a_(2, 1)));
#undef a_
#pragma unroll
                for (int m = 0; m < B; ++m) Wn[m] = i == 0 ? w[3 * m] : (i == 1 ? w[1 + 3 * m] : w[2 + 3 * m]);
            }
            const double y = __drcp_rn(d);
            double Wr[B];
#pragma unroll
            for (int m = 0; m < B; ++m) Wr[m] = qdiv(Wn[m], d, y);
            ok = finite_nz(d) && ok;
            // v = f - P z (row i), z' = W v (row i), then the whole z'
            double vi = fi;
            if (k > 0) {
#pragma unroll
                for (int m = 0; m < B; ++m) vi = xsub(vi, xmul(P[m], z[m]));
            }
            double v[B];
#pragma unroll
            for (int n = 0; n < B; ++n) v[n] = __shfl_sync(FULL, vi, base + n);
            double zi = xmul(Wr[0], v[0]);
#pragma unroll
            for (int m = 1; m < B; ++m) zi = xadd(zi, xmul(Wr[m], v[m]));
#pragma unroll
            for (int n = 0; n < B; ++n) z[n] = __shfl_sync(FULL, zi, base + n);
            if (valid && row_lane) st_hint(&pU[((long)k * B + i) * ld], zi, keep);
            if (k < k2 - 1) {
                double Gr[B];
#pragma unroll
                for (int m = 0; m < B; ++m) {
                    double g = xmul(Wr[0], R[B * m]);
#pragma unroll
                    for (int n = 1; n < B; ++n) g = xadd(g, xmul(Wr[n], R[n + B * m]));
                    Gr[m] = g;
                    if (valid && row_lane) st_hint(&gam[((long)k * BB + i + B * m) * gs], g, keep);
                }
#pragma unroll
                for (int n = 0; n < B; ++n)
#pragma unroll
                    for (int m = 0; m < B; ++m) Gf[n + B * m] = __shfl_sync(FULL, Gr[m], base + n);
            }
        }
        q += k2;
        // back sweep u_k = z_{k+1} - Gamma_{k+1} u_{k+1}, row i per lane;
        // the loads of the next BPF levels stay in flight
        constexpr int BPF = 4;
        bool fin = true;
        double un[B];
#pragma unroll
        for (int m = 0; m < B; ++m) un[m] = z[m];
        const double top = z[i];
        fin = fabs(top) <= DBL_MAX;
        double rz[BPF], rg[BPF][B];
#pragma unroll
        for (int u = 0; u < BPF; ++u) {
            const int k = k2 - 2 - u;
            if (k >= 0 && valid) {
                rz[u] = pU[((long)k * B + i) * ld];
#pragma unroll
                for (int m = 0; m < B; ++m) rg[u][m] = gam[((long)k * BB + i + B * m) * gs];
            } else {
                rz[u] = 0.0;
#pragma unroll
                for (int m = 0; m < B; ++m) rg[u][m] = 0.0;
            }
        }
        for (int kb = k2 - 2; kb >= 0; kb -= BPF) {
#pragma unroll
            for (int u = 0; u < BPF; ++u) {
                const int k = kb - u;
                if (k >= 0) {
                    double t = rz[u];
#pragma unroll
                    for (int m = 0; m < B; ++m) t = xsub(t, xmul(rg[u][m], un[m]));
                    fin = fin && fabs(t) <= DBL_MAX;
                    const int kn = k - BPF;
                    if (kn >= 0 && valid) {
                        rz[u] = pU[((long)kn * B + i) * ld];
#pragma unroll
                        for (int m = 0; m < B; ++m) rg[u][m] = gam[((long)kn * BB + i + B * m) * gs];
                    }
#pragma unroll
                    for (int n = 0; n < B; ++n) un[n] = __shfl_sync(FULL, t, base + n);
                    if (valid && row_lane) pU[((long)k * B + i) * ld] = t;
                }
            }
        }
        if (s.ubc_ratio && valid) {
            double tv = xmul(__ldg(s.ubc_ratio + i * ld + col0 + c), top);
            if (s.ubc_add) tv = xadd(tv, __ldg(s.ubc_add + i * ld + col0 + c));
            fin = fin && fabs(tv) <= DBL_MAX;
            if (row_lane) pU[((long)k2 * B + i) * ld] = tv;
        }
        const unsigned bad = __ballot_sync(FULL, !(fin || !row_lane)) & gmask;
        if (valid && ri == 0) report(status, s.status_idx, (ok ? 0u : FLAG_PIVOT) | (bad ? FLAG_NONFINITE : 0u));
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
                                                   Refine rf, int &sweeps, unsigned long long keep)
{
    constexpr int BB = B * B, NS = 2 * BB + B;
    const long ld = s.ld;
    const int k2 = s.k2;
    const double *pP = s.a + col, *pQ = s.b + col, *pR = s.c + col, *pF = s.f + col;
    double *pU = s.x + col;
    auto S = [&](int k, int e) -> float & { return scr[((long)k * NS + e) * gs]; };

    bool ok = true;
    double xmax0 = 0.0;
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
                st_hint_f(&S(k, e), W32[e], keep);
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
                st_hint_f(&S(k, 2 * BB + i), t, keep);
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
                    st_hint_f(&S(k, BB + i + B * m), g, keep);
                }
        }
        float un[B], xm = 0.f;
#pragma unroll
        for (int i = 0; i < B; ++i) {
            un[i] = z[i];
            xm = fmaxf(xm, fabsf(z[i]));
            st_hint(&pU[((long)(k2 - 1) * B + i) * ld], (double)z[i], keep);
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
                xm = fmaxf(xm, fabsf(nu[i]));
                st_hint(&pU[((long)k * B + i) * ld], (double)nu[i], keep);
            }
        }
        xmax0 = (double)xm;
    }

    // ---- refinement sweeps
    bool conv = false;
    int sw = 0;
    double dprev = xmax0;
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
                    st_hint_f(&S(k, 2 * BB + i), t, keep);
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
            if (refine_done(dmax, xmax, dprev, rf.rel_tol, sw == 1)) {
                conv = true;
                break;
            }
            dprev = dmax;
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

// ---------------------------------------------------------------------------
// Block-tridiagonal FP32 sweeps + FP64 refinement with the coefficients
// staged by the bulk-copy ring: one warp per 32 columns, a D-level ring of
// the 3*B*B + B coefficient rows per level (and, in the correction sweeps,
// the B rows of u one level above), one 256-byte copy per row.  Same
// arithmetic, planes, stopping rule, fallback and flags as blk_refine_col;
// the FP32 planes W | G | z of level k sit at (k*NS + e)*gs of the lane's
// scratch slot.  u rows written by this warp's generic stores are read back
// by bulk copies: a proxy fence orders the two before each correction sweep.
// Requires ld % 32 == 0 and 16-byte aligned P, Q, R, f, u.
// ---------------------------------------------------------------------------
template <int B, int D>
__global__ void __launch_bounds__(256) k_block_refine_ring(SegTable tab, Refine rf, float *scratch, unsigned *status,
                                                           unsigned long long *hist)
{
    constexpr int BB = B * B, NE = 3 * BB + B, NX = NE + B, NS = 2 * BB + B;
    static_assert(NX <= 32, "one copy per lane");
    __shared__ __align__(8) unsigned long long bars[8 * D];
    extern __shared__ __align__(128) double smem_b[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    double *buf = smem_b + (long)warp * D * NX * 32;
    unsigned long long *bar = bars + warp * D;
    const unsigned long long pol = refine_fill_policy(tab.hints), keep = l2_policy(tab.hints, true);
    const long gs = (long)gridDim.x * blockDim.x;
    float *scr = scratch + (long)blockIdx.x * blockDim.x + threadIdx.x;
    auto S = [&](int k, int e) -> float & { return scr[((long)k * NS + e) * gs]; };
    if (lane == 0) {
#pragma unroll 1
        for (int i = 0; i < D; ++i) mbar_init(&bar[i], 1);
        fence_mbar_init();
    }
    __syncwarp();
    unsigned long long hl[kMaxSweepBins];
#pragma unroll
    for (int i = 0; i < kMaxSweepBins; ++i) hl[i] = 0ull;
    unsigned q = 0;
    for (int t = blockIdx.x * nwarps + warp; t < tab.ntiles; t += gridDim.x * nwarps) {
        const Seg s = tab.segs ? tab.segs[find_seg(tab, t)] : tab.one;
        const long col0 = (long)(t - s.tile0) * 32;
        const long ld = s.ld;
        const int k2 = s.k2;
        const bool valid = col0 + lane < s.ncol;
        // row e of level k: P/Q/R element e at (k*BB + e)*ld, f and u
        // component i at (k*B + i)*ld; lanes NE.. copy u of level k+1
        const double *src = s.a + col0;
        long lstride = 0;
        if (lane < BB) {
            src = s.a + col0 + lane * ld;
            lstride = BB * ld;
        } else if (lane < 2 * BB) {
            src = s.b + col0 + (lane - BB) * ld;
            lstride = BB * ld;
        } else if (lane < 3 * BB) {
            src = s.c + col0 + (lane - 2 * BB) * ld;
            lstride = BB * ld;
        } else if (lane < NE) {
            src = s.f + col0 + (lane - 3 * BB) * ld;
            lstride = B * ld;
        } else if (lane < NX) {
            src = s.x + col0 + (lane - NE + B) * ld;
            lstride = B * ld;
        }
        double *pU = s.x + col0 + lane;
        auto issue = [&](unsigned qk, int k, bool withu) {
            const int st = (int)(qk % D);
            const bool u = withu && k + 1 < k2;
            if (lane == 0) mbar_expect(&bar[st], (uint32_t)(NE + (u ? B : 0)) * 256u);
            __syncwarp();
            if (lane < NE || (u && lane < NX))
                bulk_load_hint(buf + (st * NX + lane) * 32, src + (long)k * lstride, 256u, &bar[st], pol);
        };
        auto wait = [&](unsigned q0, int k) -> bool {
            const unsigned qk = q0 + k;
            if (mbar_wait_warp(&bar[qk % D], (qk / D) & 1u)) return true;
            const unsigned qe = q0 + (k + D < k2 ? k + D : k2);
#pragma unroll 1
            for (unsigned r = qk; r < qe; ++r) mbar_wait_warp(&bar[r % D], (r / D) & 1u);
            if (lane == 0) report(status, s.status_idx, FLAG_TIMEOUT);
            return false;
        };
        auto at = [&](unsigned qk, int e) { return buf[((int)(qk % D) * NX + e) * 32 + lane]; };

        // ---- sweep 0: FP64 pivots and inverses, FP32 planes and sweeps
        bool ok = true;
        float xm = 0.f;
        {
            const int pre = k2 < D ? k2 : D;
            for (int j = 0; j < pre; ++j) issue(q + j, j, false);
            float G[BB], z[B];
#pragma unroll
            for (int e = 0; e < BB; ++e) G[e] = 0.f;
#pragma unroll
            for (int i = 0; i < B; ++i) z[i] = 0.f;
            for (int k = 0; k < k2; ++k) {
                const unsigned qk = q + k;
                if (!wait(q, k)) return;
                double P[BB], Q[BB], R[BB], F[B];
#pragma unroll
                for (int e = 0; e < BB; ++e) {
                    P[e] = k > 0 ? at(qk, e) : 0.0;
                    Q[e] = at(qk, BB + e);
                    R[e] = k < k2 - 1 ? at(qk, 2 * BB + e) : 0.0;
                }
#pragma unroll
                for (int i = 0; i < B; ++i) F[i] = at(qk, 3 * BB + i);
                __syncwarp();
                fence_proxy_async();
                if (k + D < k2) issue(qk + D, k + D, false);
                if (!valid) continue;
                double Qp[BB], W[BB];
#pragma unroll
                for (int m = 0; m < B; ++m)
#pragma unroll
                    for (int i = 0; i < B; ++i) {
                        double qv = Q[i + B * m];
                        if (k > 0)
#pragma unroll
                            for (int n = 0; n < B; ++n) qv = fma(-P[i + B * n], (double)G[n + B * m], qv);
                        Qp[i + B * m] = qv;
                    }
                ok = inv_exact<B>(Qp, W) && ok;
                float W32[BB], v[B];
#pragma unroll
                for (int e = 0; e < BB; ++e) {
                    W32[e] = (float)W[e];
                    st_hint_f(&S(k, e), W32[e], keep);
                }
#pragma unroll
                for (int i = 0; i < B; ++i) {
                    float tv = (float)F[i];
                    if (k > 0)
#pragma unroll
                        for (int m = 0; m < B; ++m) tv = fmaf(-(float)P[i + B * m], z[m], tv);
                    v[i] = tv;
                }
#pragma unroll
                for (int i = 0; i < B; ++i) {
                    float tv = 0.f;
#pragma unroll
                    for (int m = 0; m < B; ++m) tv = fmaf(W32[i + B * m], v[m], tv);
                    z[i] = tv;
                    st_hint_f(&S(k, 2 * BB + i), tv, keep);
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
                        st_hint_f(&S(k, BB + i + B * m), g, keep);
                    }
            }
            q += k2;
            if (valid) {
                float un[B];
#pragma unroll
                for (int i = 0; i < B; ++i) {
                    un[i] = z[i];
                    xm = fmaxf(xm, fabsf(z[i]));
                    st_hint(&pU[((long)(k2 - 1) * B + i) * ld], (double)z[i], keep);
                }
                for (int k = k2 - 2; k >= 0; --k) {
                    float nu[B];
#pragma unroll
                    for (int i = 0; i < B; ++i) {
                        float tv = S(k, 2 * BB + i);
#pragma unroll
                        for (int m = 0; m < B; ++m) tv = fmaf(-S(k, BB + i + B * m), un[m], tv);
                        nu[i] = tv;
                    }
#pragma unroll
                    for (int i = 0; i < B; ++i) {
                        un[i] = nu[i];
                        xm = fmaxf(xm, fabsf(nu[i]));
                        st_hint(&pU[((long)k * B + i) * ld], (double)nu[i], keep);
                    }
                }
            }
        }

        // ---- correction sweeps (the warp streams while any lane is active)
        bool active = valid && ok, conv = false;
        int sw = 0, taken = rf.max_sweeps + 1;
        double dprev = (double)xm;
        for (sw = 1; sw <= rf.max_sweeps && __any_sync(0xffffffffu, active); ++sw) {
            fence_proxy_async_global();
            __syncwarp();
            const int pre = k2 < D ? k2 : D;
            for (int j = 0; j < pre; ++j) issue(q + j, j, true);
            double um[B], u0[B];
            float zc[B];
#pragma unroll
            for (int i = 0; i < B; ++i) {
                um[i] = 0.0;
                u0[i] = active ? pU[i * ld] : 0.0;
                zc[i] = 0.f;
            }
            for (int k = 0; k < k2; ++k) {
                const unsigned qk = q + k;
                if (!wait(q, k)) return;
                double up[B], r[B];
#pragma unroll
                for (int i = 0; i < B; ++i) {
                    up[i] = k + 1 < k2 ? at(qk, NE + i) : 0.0;
                    r[i] = at(qk, 3 * BB + i);
                }
                float P32[BB];
#pragma unroll
                for (int e = 0; e < BB; ++e) {
                    const int i = e % B, m = e / B;
                    r[i] = fma(-at(qk, BB + e), u0[m], r[i]);
                    double p = 0.0;
                    if (k > 0) {
                        p = at(qk, e);
                        r[i] = fma(-p, um[m], r[i]);
                    }
                    P32[e] = (float)p;
                    if (k + 1 < k2) r[i] = fma(-at(qk, 2 * BB + e), up[m], r[i]);
                }
                __syncwarp();
                fence_proxy_async();
                if (k + D < k2) issue(qk + D, k + D, true);
                if (active) {
                    float v[B];
#pragma unroll
                    for (int i = 0; i < B; ++i) {
                        float tv = (float)r[i];
#pragma unroll
                        for (int m = 0; m < B; ++m) tv = fmaf(-P32[i + B * m], zc[m], tv);
                        v[i] = tv;
                    }
#pragma unroll
                    for (int i = 0; i < B; ++i) {
                        float tv = 0.f;
#pragma unroll
                        for (int m = 0; m < B; ++m) tv = fmaf(S(k, i + B * m), v[m], tv);
                        zc[i] = tv;
                        st_hint_f(&S(k, 2 * BB + i), tv, keep);
                    }
                }
#pragma unroll
                for (int i = 0; i < B; ++i) {
                    um[i] = u0[i];
                    u0[i] = up[i];
                }
            }
            q += k2;
            if (active) {
                double dmax = 0.0, xmax = 0.0;
                float dn[B];
#pragma unroll
                for (int i = 0; i < B; ++i) {
                    dn[i] = zc[i];
                    const double xv = um[i] + (double)dn[i];   // um holds u(k2-1)
                    st_hint(&pU[((long)(k2 - 1) * B + i) * ld], xv, keep);
                    dmax = fmax(dmax, fabs((double)dn[i]));
                    xmax = fmax(xmax, fabs(xv));
                }
                for (int k = k2 - 2; k >= 0; --k) {
                    float nd[B];
#pragma unroll
                    for (int i = 0; i < B; ++i) {
                        float tv = S(k, 2 * BB + i);
#pragma unroll
                        for (int m = 0; m < B; ++m) tv = fmaf(-S(k, BB + i + B * m), dn[m], tv);
                        nd[i] = tv;
                    }
#pragma unroll
                    for (int i = 0; i < B; ++i) {
                        dn[i] = nd[i];
                        double *p = pU + ((long)k * B + i) * ld;
                        const double xv = *p + (double)nd[i];
                        st_hint(p, xv, keep);
                        dmax = fmax(dmax, fabs((double)nd[i]));
                        xmax = fmax(xmax, fabs(xv));
                    }
                }
                if (!(xmax <= DBL_MAX) || !(dmax <= DBL_MAX)) {
                    active = false;
                } else if (refine_done(dmax, xmax, dprev, rf.rel_tol, sw == 1)) {
                    conv = true;
                    active = false;
                    taken = sw;
                } else {
                    dprev = dmax;
                }
            }
        }
        unsigned flags = 0u;
        if (valid && !conv) {
            // ---- fallback: bit-exact FP64 solve, G kept as (hi, lo) float pairs
            const double *pP = s.a + col0 + lane, *pQ = s.b + col0 + lane, *pR = s.c + col0 + lane,
                         *pF = s.f + col0 + lane;
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
                        double qv = Q[i + B * m];
                        if (k > 0)
#pragma unroll
                            for (int n = 0; n < B; ++n) qv = xsub(qv, xmul(P[i + B * n], G[n + B * m]));
                        Qp[i + B * m] = qv;
                    }
#pragma unroll
                for (int i = 0; i < B; ++i) {
                    double tv = F[i];
                    if (k > 0)
#pragma unroll
                        for (int m = 0; m < B; ++m) tv = xsub(tv, xmul(P[i + B * m], z[m]));
                    v[i] = tv;
                }
                okd = inv_exact<B>(Qp, W) && okd;
#pragma unroll
                for (int i = 0; i < B; ++i) {
                    double tv = xmul(W[i], v[0]);
#pragma unroll
                    for (int m = 1; m < B; ++m) tv = xadd(tv, xmul(W[i + B * m], v[m]));
                    z[i] = tv;
                    pU[((long)k * B + i) * ld] = tv;
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
                    double tv = pU[((long)k * B + i) * ld];
#pragma unroll
                    for (int m = 0; m < B; ++m) {
                        const int e = i + B * m;
                        const double g = __hiloint2double(__float_as_int(S(k, 2 * e)), __float_as_int(S(k, 2 * e + 1)));
                        tv = xsub(tv, xmul(g, un[m]));
                    }
                    nu[i] = tv;
                    fin = fin && finite(tv);
                }
#pragma unroll
                for (int i = 0; i < B; ++i) {
                    un[i] = nu[i];
                    pU[((long)k * B + i) * ld] = nu[i];
                }
            }
            flags |= (okd ? 0u : FLAG_PIVOT) | (fin ? 0u : FLAG_NONFINITE);
        } else if (valid && !ok) {
            flags |= FLAG_PIVOT;
        }
        if (valid && s.ubc_ratio) {
            bool fin = true;
#pragma unroll
            for (int i = 0; i < B; ++i) {
                const double top = pU[((long)(k2 - 1) * B + i) * ld];
                double tv = xmul(__ldg(s.ubc_ratio + i * ld + col0 + lane), top);
                if (s.ubc_add) tv = xadd(tv, __ldg(s.ubc_add + i * ld + col0 + lane));
                fin = fin && finite(tv);
                pU[((long)k2 * B + i) * ld] = tv;
            }
            if (!fin) flags |= FLAG_NONFINITE;
        }
        if (valid) report(status, s.status_idx, flags);
        const int bin = taken < kMaxSweepBins - 1 ? taken : kMaxSweepBins - 1;
#pragma unroll
        for (int i = 0; i < kMaxSweepBins; ++i) hl[i] += __popc(__ballot_sync(0xffffffffu, valid && bin == i));
    }
    if (hist && lane == 0)
#pragma unroll
        for (int i = 0; i < kMaxSweepBins; ++i)
            if (hl[i]) atomicAdd(hist + i, hl[i]);
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
    // the FP32 planes and u are re-read by the next sweep: keep them in L2
    const unsigned long long keep = l2_policy(tab.hints, true);
    for (int t = blockIdx.x; t < tab.ntiles; t += gridDim.x) {
        const Seg s = tab.segs ? tab.segs[find_seg(tab, t)] : tab.one;
        const long col = (long)(t - s.tile0) * blockDim.x + threadIdx.x;
        if (col < s.ncol) {
            int sweeps = 0;
            report(status, s.status_idx, blk_refine_col<B>(s, col, scr, gs, rf, sweeps, keep));
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

// Up to four arrays relaid in one launch (blockIdx.y = array), each with its
// own row count and input column stride; output column stride shared.
__global__ void __launch_bounds__(256) k_col_to_level_multi(Relayout r)
{
    __shared__ double tile[32][33];
    const int a = blockIdx.y;
    const double *__restrict__ in = r.in[a];
    double *__restrict__ out = r.out[a];
    const long nrows = r.nrows[a], in_ld = r.in_ld[a], out_ld = r.out_ld, ncols = r.ncols;
    const long nrt = (nrows + 31) / 32, nct = (ncols + 31) / 32;
    for (long bt = blockIdx.x; bt < nrt * nct; bt += gridDim.x) {
        const long r0 = (bt % nrt) * 32, c0 = (bt / nrt) * 32;
        for (int j = threadIdx.y; j < 32; j += 8) {
            const long c = c0 + j, rr = r0 + threadIdx.x;
            if (c < ncols && rr < nrows) tile[j][threadIdx.x] = __ldcs(in + rr + in_ld * c);
        }
        __syncthreads();
        for (int j = threadIdx.y; j < 32; j += 8) {
            const long rr = r0 + j, c = c0 + threadIdx.x;
            if (rr < nrows && c < ncols) out[rr * out_ld + c] = tile[threadIdx.x][j];
        }
        __syncthreads();
    }
}

// Division self-test: q[i] = a[i]/b[i] through qdiv (Markstein where safe).
__global__ void k_selftest_division(const double *a, const double *b, double *q, long n)
{
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
        q[i] = qdiv(a[i], b[i], __drcp_rn(b[i]));
}

// The ring kernels' bounded wait, run on an mbarrier that nothing arrives
// at: after `polls` polls the warp gives up and reports FLAG_TIMEOUT, as a
// ring kernel does when a bulk copy never lands.  Exercises the timeout path
// without a stuck copy.
__global__ void __launch_bounds__(32) k_selftest_wait(unsigned polls, unsigned *status)
{
    __shared__ __align__(8) unsigned long long bar;
    const int lane = threadIdx.x & 31;
    if (lane == 0) {
        mbar_init(&bar, 1);
        fence_mbar_init();
    }
    __syncwarp();
    const bool ok = mbar_wait_warp(&bar, 0u, polls);
    if (lane == 0 && !ok) atomicOr(status, FLAG_TIMEOUT);
}

cudaError_t launch_selftest_wait(unsigned polls, unsigned *status, cudaStream_t st)
{
    k_selftest_wait<<<1, 32, 0, st>>>(polls, status);
    return cudaGetLastError();
}

cudaError_t launch_selftest_division(const double *a, const double *b, double *q, long n, cudaStream_t st)
{
    if (n <= 0) return cudaSuccess;
    k_selftest_division<<<1184, 256, 0, st>>>(a, b, q, n);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Launch shapes and launchers
// ---------------------------------------------------------------------------
namespace {
struct TileCfg {
    int cpb, cpt, stages;  // register kernel: columns per block / per thread; ring depth (0: no ring)
    int w2g;               // scalar register kernel: w2 in global scratch instead of shared memory
    int pf;                // scalar register kernels: levels of coefficient loads in flight per column
    int wpb;               // ring kernels: independent warps (32-column tiles) per CTA
    int rows;              // block ring kernels: one lane per block row (k_block_f64_rows)
    int bw;                // block ring kernels: columns per warp (32, 16 or 8)
    int lps;               // scalar FP64 ring: levels per stage (1: k_scalar_f64_ring, >1: k_scalar_f64_chunk)
    int res;               // scalar FP64 chunked ring: 0 scratch in L2 (k_scalar_f64_chunk), 1 w2 resident in
                           // shared memory, w3 parked in x, 2 w2 and w3 resident (k_scalar_f64_res)
};
// [kind index: scalar, block2, block3][precision]
// Defaults: the fastest shapes on a B200 (autotune.py sweeps of the 2.5 deg
// column step, 10368 x 57, and of the nested 2.5 deg + 3-nest batch): scalar
// FP64 chunked bulk-copy ring of 2 stages x 4 levels, one warp per CTA, w2 in
// global scratch; 2x2 and 3x3 block rings of depth 4, one warp per CTA (the
// 3x3 ring beat the 128-thread register kernel on the nested batch with
// 3x3 blocks, 2.14 against 2.32 ms); scalar refinement ring of 2 stages and
// 2x2 block refinement ring of depth 4, one warp per CTA each; 3x3 block
// refinement register kernel of 128 threads.
const TileCfg kDefaultTile[3][2] = {{{256, 1, 2, 1, 4, 1, 0, 32, 4, 0}, {64, 1, 2, 0, 8, 1, 0, 32, 1, 0}},
                                     {{64, 1, 4, 0, 4, 1, 0, 32, 1, 0}, {64, 1, 4, 0, 4, 1, 0, 32, 1, 0}},
                                     {{128, 1, 4, 0, 4, 1, 0, 32, 1, 0}, {128, 1, 0, 0, 4, 4, 0, 32, 1, 0}}};
TileCfg g_tile[3][2] = {{{256, 1, 2, 1, 4, 1, 0, 32, 4, 0}, {64, 1, 2, 0, 8, 1, 0, 32, 1, 0}},
                        {{64, 1, 4, 0, 4, 1, 0, 32, 1, 0}, {64, 1, 4, 0, 4, 1, 0, 32, 1, 0}},
                        {{128, 1, 4, 0, 4, 1, 0, 32, 1, 0}, {128, 1, 0, 0, 4, 4, 0, 32, 1, 0}}};
int kind_index(int kind) { return kind == TG_KIND_SCALAR ? 0 : (kind == TG_KIND_BLOCK2 ? 1 : 2); }
constexpr int kMaxDevIdx = 64;
int g_num_sms[kMaxDevIdx] = {};
int g_carveout = cudaSharedmemCarveoutMaxShared;   // percent of the unified L1/shared store
int g_smem_optin[kMaxDevIdx] = {};

// Register-prefetch scalar kernels by (columns per thread, prefetch depth).
template <typename F>
cudaError_t with_scalar_reg(int cpt, int pf, F f)
{
    if (cpt == 2) {
        switch (pf) {
        case 4: return f(k_scalar_f64<2, 4>);
        case 8: return f(k_scalar_f64<2, 8>);
        default: return cudaErrorInvalidValue;
        }
    }
    switch (pf) {
    case 4: return f(k_scalar_f64<1, 4>);
    case 8: return f(k_scalar_f64<1, 8>);
    case 16: return f(k_scalar_f64<1, 16>);
    default: return cudaErrorInvalidValue;
    }
}
template <typename F>
cudaError_t with_scalar_g(int pf, F f)
{
    switch (pf) {
    case 4: return f(k_scalar_f64_g<4>);
    case 8: return f(k_scalar_f64_g<8>);
    case 16: return f(k_scalar_f64_g<16>);
    default: return cudaErrorInvalidValue;
    }
}
template <typename F>
cudaError_t with_scalar_refine(int pf, F f)
{
    switch (pf) {
    case 4: return f(k_scalar_refine<4>);
    case 8: return f(k_scalar_refine<8>);
    case 16: return f(k_scalar_refine<16>);
    default: return cudaErrorInvalidValue;
    }
}

// Scalar refinement ring kernels by stage count.
template <typename F>
cudaError_t with_scalar_refine_ring(int C, F f)
{
    switch (C) {
    case 2: return f(k_scalar_refine_ring<2>);
    case 3: return f(k_scalar_refine_ring<3>);
    case 4: return f(k_scalar_refine_ring<4>);
    default: return cudaErrorInvalidValue;
    }
}

template <typename F>
cudaError_t with_scalar_ring(int D, int w2g, F f)
{
    if (w2g) {
        switch (D) {
        case 4: return f(k_scalar_f64_ring<4, true>);
        case 8: return f(k_scalar_f64_ring<8, true>);
        case 16: return f(k_scalar_f64_ring<16, true>);
        default: return cudaErrorInvalidValue;
        }
    }
    switch (D) {
    case 4: return f(k_scalar_f64_ring<4, false>);
    case 8: return f(k_scalar_f64_ring<8, false>);
    case 16: return f(k_scalar_f64_ring<16, false>);
    default: return cudaErrorInvalidValue;
    }
}
template <typename F>
cudaError_t with_scalar_chunk(int C, int L, F f)
{
#define TG_CHUNK(c, l) \
    if (C == c && L == l) return f(k_scalar_f64_chunk<c, l>);
    TG_CHUNK(2, 2) TG_CHUNK(3, 2) TG_CHUNK(4, 2) TG_CHUNK(2, 4) TG_CHUNK(3, 4) TG_CHUNK(4, 4) TG_CHUNK(2, 8)
#undef TG_CHUNK
    return cudaErrorInvalidValue;
}
// Shared-memory-resident scalar kernels by (stages, levels per stage, w3 resident).
template <typename F>
cudaError_t with_scalar_res(int C, int L, int w3s, F f)
{
#define TG_RES(c, l)                                                 \
    if (C == c && L == l) {                                          \
        if (w3s) return f(k_scalar_f64_res<c, l, true>);             \
        return f(k_scalar_f64_res<c, l, false>);                     \
    }
    TG_RES(2, 2) TG_RES(3, 2) TG_RES(4, 2) TG_RES(2, 4) TG_RES(3, 4) TG_RES(4, 4)
#undef TG_RES
    return cudaErrorInvalidValue;
}
template <typename F>
cudaError_t with_block_ring(int B, int D, int W, F f)
{
#define TG_RING(b, d, w) \
    if (B == b && D == d && W == w) return f(k_block_f64_ring<b, d, w>);
    TG_RING(2, 4, 32) TG_RING(2, 8, 32) TG_RING(2, 16, 32) TG_RING(2, 4, 16) TG_RING(2, 8, 16) TG_RING(2, 4, 8)
    TG_RING(2, 8, 8) TG_RING(3, 4, 32) TG_RING(3, 8, 32) TG_RING(3, 16, 32) TG_RING(3, 4, 16) TG_RING(3, 8, 16)
    TG_RING(3, 4, 8) TG_RING(3, 8, 8)
#undef TG_RING
    return cudaErrorInvalidValue;
}

// Block ring kernels with Gamma resident in shared memory.
template <typename F>
cudaError_t with_block_ring_gsm(int B, int D, int W, F f)
{
#define TG_RING_GSM(b, d, w) \
    if (B == b && D == d && W == w) return f(k_block_f64_ring<b, d, w, true>);
    TG_RING_GSM(2, 4, 32) TG_RING_GSM(2, 4, 16) TG_RING_GSM(2, 8, 16) TG_RING_GSM(2, 4, 8) TG_RING_GSM(2, 8, 8)
    TG_RING_GSM(3, 4, 16) TG_RING_GSM(3, 4, 8) TG_RING_GSM(3, 8, 8)
#undef TG_RING_GSM
    return cudaErrorInvalidValue;
}

// Block refinement ring kernels (2x2 blocks) by ring depth.
template <typename F>
cudaError_t with_block_refine_ring(int B, int D, F f)
{
    if (B != 2) return cudaErrorInvalidValue;
    switch (D) {
    case 4: return f(k_block_refine_ring<2, 4>);
    case 8: return f(k_block_refine_ring<2, 8>);
    default: return cudaErrorInvalidValue;
    }
}

template <typename F>
cudaError_t with_block_rows(int B, int D, F f)
{
    if (B == 2) {
        switch (D) {
        case 4: return f(k_block_f64_rows<2, 4>);
        case 8: return f(k_block_f64_rows<2, 8>);
        default: return cudaErrorInvalidValue;
        }
    }
    switch (D) {
    case 4: return f(k_block_f64_rows<3, 4>);
    case 8: return f(k_block_f64_rows<3, 8>);
    default: return cudaErrorInvalidValue;
    }
}

template <typename K>
void allow_smem(K k, int lim)
{
    cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
    // the rings live in shared memory and the coefficient streams bypass L1:
    // prefer the largest shared-memory carveout so that more warps fit per SM
    cudaFuncSetAttribute(k, cudaFuncAttributePreferredSharedMemoryCarveout, g_carveout);
}

// SM count and opt-in shared memory per device; the first call on a device
// also lets every kernel that takes dynamic shared memory use up to the
// opt-in limit (minus its static shared memory).
int device_index()
{
    int d = 0;
    cudaGetDevice(&d);
    return d >= 0 && d < kMaxDevIdx ? d : 0;
}
void device_init()
{
    once_per_device([] {
        const int d = device_index();
        cudaDeviceGetAttribute(&g_num_sms[d], cudaDevAttrMultiProcessorCount, d);
        cudaDeviceGetAttribute(&g_smem_optin[d], cudaDevAttrMaxSharedMemoryPerBlockOptin, d);
        const int lim = g_smem_optin[d] - 1024;
        for (int pf : {4, 8, 16}) {
            with_scalar_reg(1, pf, [&](auto k) { allow_smem(k, lim); return cudaSuccess; });
            with_scalar_reg(2, pf, [&](auto k) { allow_smem(k, lim); return cudaSuccess; });
            with_scalar_refine(pf, [&](auto k) { allow_smem(k, lim); return cudaSuccess; });
        }
        for (int d : {4, 8, 16})
            for (int g : {0, 1}) with_scalar_ring(d, g, [&](auto k) { allow_smem(k, lim); return cudaSuccess; });
        for (int c : {2, 3, 4}) with_scalar_refine_ring(c, [&](auto k) { allow_smem(k, lim); return cudaSuccess; });
        allow_smem(k_scalar_refine_tile, lim);
        for (int dd : {4, 8}) with_block_refine_ring(2, dd, [&](auto k) { allow_smem(k, lim); return cudaSuccess; });
        for (int c : {2, 3, 4})
            for (int l : {2, 4, 8}) with_scalar_chunk(c, l, [&](auto k) { allow_smem(k, lim); return cudaSuccess; });
        for (int c : {2, 3, 4})
            for (int l : {2, 4})
                for (int w : {0, 1}) with_scalar_res(c, l, w, [&](auto k) { allow_smem(k, lim); return cudaSuccess; });
        for (int b : {2, 3})
            for (int d : {4, 8, 16})
                for (int w : {32, 16, 8}) {
                    with_block_ring(b, d, w, [&](auto k) { allow_smem(k, lim); return cudaSuccess; });
                    with_block_ring_gsm(b, d, w, [&](auto k) { allow_smem(k, lim); return cudaSuccess; });
                }
        for (int d : {4, 8})
            for (int b : {2, 3}) with_block_rows(b, d, [&](auto k) { allow_smem(k, lim); return cudaSuccess; });
    });
}
int num_sms()
{
    device_init();
    return g_num_sms[device_index()];
}
}  // namespace
int smem_optin()
{
    device_init();
    return g_smem_optin[device_index()];
}
namespace {

// Occupancy queries are cached per (kernel, threads, shared memory): the host
// drop-ins shape one launch per column chunk, and the query is host time on
// the path that feeds the copy engines.
struct OccKey {
    const void *k;
    int threads;
    size_t smem;
    int per_sm;
};
OccKey g_occ[64];
int g_nocc = 0;
std::mutex g_occ_mu;

template <typename K>
cudaError_t occupancy(K kernel, int threads, size_t smem, int *per_sm)
{
    const void *kp = reinterpret_cast<const void *>(kernel);
    {
        std::lock_guard<std::mutex> lk(g_occ_mu);
        for (int i = 0; i < g_nocc; ++i)
            if (g_occ[i].k == kp && g_occ[i].threads == threads && g_occ[i].smem == smem) {
                *per_sm = g_occ[i].per_sm;
                return cudaSuccess;
            }
    }
    cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(per_sm, kernel, threads, smem);
    if (e == cudaSuccess) {
        std::lock_guard<std::mutex> lk(g_occ_mu);
        if (g_nocc < 64) g_occ[g_nocc++] = OccKey{kp, threads, smem, *per_sm};
    }
    return e;
}

// Resident threads allowed for the block kernels: their Gamma scratch (k2 *
// B*B doubles per resident thread) of all of them within this budget.  160 MB
// lets more columns into flight than L2 holds, and that wins: 3x3 blocks on
// the nested batch took 2.15 ms at 96 MB and 1.72 ms at 128 and 192 MB (2x2
// blocks are occupancy-bound from 128 MB on: 2.19 -> 2.17 ms).
constexpr double kBlockBudgetMB = 160.0;
double g_block_scratch_budget = kBlockBudgetMB * 1024 * 1024;
// Scalar ring kernels: L2 bytes of w2 scratch and parked w3 of all resident
// columns.  Past the L2's capacity the back sweep's re-reads go to DRAM.
constexpr double kScalarBudgetMB = 128.0;
double g_scalar_scratch_budget = kScalarBudgetMB * 1024 * 1024;
std::atomic<int> g_kind_overlap{-1};
}  // namespace

int prefetch_depth(int kind, int precision) { return g_tile[kind_index(kind)][precision ? 1 : 0].pf; }
void set_prefetch(int kind, int precision, int pf)
{
    TileCfg &t = g_tile[kind_index(kind)][precision ? 1 : 0];
    t.pf = pf > 0 ? pf : kDefaultTile[kind_index(kind)][precision ? 1 : 0].pf;
}

void tile_for(int kind, int precision, bool ring_ok, int *cpb, int *cpt, int *stages, int *w2g)
{
    const TileCfg &t = g_tile[kind_index(kind)][precision ? 1 : 0];
    *w2g = 0;
    if ((precision == TG_PREC_F64 || kind != TG_KIND_BLOCK3) && t.stages > 0 && ring_ok) {
        *cpb = 32;
        *cpt = 1;
        *stages = t.stages;
        *w2g = kind == TG_KIND_SCALAR ? t.w2g : 0;
    } else {
        *cpb = t.cpb;
        *cpt = t.cpt;
        *stages = 0;
        if (kind == TG_KIND_SCALAR && precision == TG_PREC_F64 && t.w2g) {
            *w2g = 1;
            *cpb = t.cpb / t.cpt;
            *cpt = 1;
        }
    }
}

void set_w2g(int kind, int precision, int on)
{
    TileCfg &t = g_tile[kind_index(kind)][precision ? 1 : 0];
    t.w2g = on >= 0 ? on : kDefaultTile[kind_index(kind)][precision ? 1 : 0].w2g;
}

size_t scalar_scratch_bytes(long slots, int k2max) { return (size_t)slots * (size_t)(k2max > 1 ? k2max - 1 : 1) * 8; }
size_t refine_scratch_bytes(long slots, int k2max) { return (size_t)slots * 3 * (size_t)k2max * 4; }

int cols_per_block(int kind, int precision) { return g_tile[kind_index(kind)][precision ? 1 : 0].cpb; }
int cols_per_thread(int kind, int precision) { return g_tile[kind_index(kind)][precision ? 1 : 0].cpt; }
void set_tile(int kind, int precision, int cpb, int cpt)
{
    TileCfg &t = g_tile[kind_index(kind)][precision ? 1 : 0];
    const TileCfg &d = kDefaultTile[kind_index(kind)][precision ? 1 : 0];
    t.cpb = cpb > 0 ? cpb : d.cpb;
    t.cpt = cpt > 0 ? cpt : d.cpt;
    if (kind != TG_KIND_SCALAR || precision) t.cpt = 1;
}
void set_stages(int kind, int precision, int stages, int wpb)
{
    TileCfg &t = g_tile[kind_index(kind)][precision ? 1 : 0];
    const TileCfg &d = kDefaultTile[kind_index(kind)][precision ? 1 : 0];
    t.stages = stages >= 0 ? stages : d.stages;
    t.wpb = wpb > 0 ? wpb : d.wpb;
}
int ring_warps(int kind, int precision) { return g_tile[kind_index(kind)][precision ? 1 : 0].wpb; }
void set_block_rows(int kind, int on)
{
    if (kind == TG_KIND_SCALAR) return;
    TileCfg &t = g_tile[kind_index(kind)][0];
    t.rows = on < 0 ? kDefaultTile[kind_index(kind)][0].rows : (on ? 1 : 0);
}
void set_block_scratch_budget(double mb) { g_block_scratch_budget = (mb > 0 ? mb : kBlockBudgetMB) * 1024 * 1024; }
void set_scalar_scratch_budget(double mb)
{
    g_scalar_scratch_budget = (mb > 0 ? mb : kScalarBudgetMB) * 1024 * 1024;
}
void set_kind_overlap(int mode) { g_kind_overlap.store(mode == 0 || mode == 1 ? mode : -1); }
int kind_overlap() { return g_kind_overlap.load(); }
void set_column_residency(int kind, int precision, int mode)
{
    if (precision != TG_PREC_F64) {   // scalar refinement: 1 the whole tile on chip
        if (kind != TG_KIND_SCALAR) return;
        g_tile[0][1].res = mode >= 0 && mode <= 2 ? (mode ? 1 : 0) : kDefaultTile[0][1].res;
        return;
    }
    TileCfg &t = g_tile[kind_index(kind)][0];
    const int def = kDefaultTile[kind_index(kind)][0].res;
    if (kind == TG_KIND_SCALAR) t.res = mode >= 0 && mode <= 2 ? mode : def;
    else t.res = mode >= 0 && mode <= 2 ? (mode ? 1 : 0) : def;
}
int column_residency() { return g_tile[0][0].res; }
void set_stage_levels(int kind, int precision, int l)
{
    if (kind != TG_KIND_SCALAR || precision != TG_PREC_F64) return;
    TileCfg &t = g_tile[0][0];
    t.lps = (l == 1 || l == 2 || l == 4 || l == 8) ? l : kDefaultTile[0][0].lps;
}
void set_block_width(int kind, int w)
{
    if (kind == TG_KIND_SCALAR) return;
    TileCfg &t = g_tile[kind_index(kind)][0];
    t.bw = (w == 8 || w == 16 || w == 32) ? w : kDefaultTile[kind_index(kind)][0].bw;
}
static int block_width(int kind, int precision)
{
    return kind != TG_KIND_SCALAR && precision == TG_PREC_F64 ? g_tile[kind_index(kind)][0].bw : 32;
}
static int block_rows(int kind, int precision)
{
    return kind != TG_KIND_SCALAR && precision == TG_PREC_F64 && g_tile[kind_index(kind)][0].rows;
}
// lanes per column of the row kernel
static int rows_group(int B) { return B == 2 ? 2 : 4; }

size_t scalar_smem_bytes(int precision, int threads, int cpt, int k2max, int stages, int w2g, int lps)
{
    const size_t lev = (size_t)(k2max > 1 ? k2max - 1 : 1);
    if (stages > 0 && precision != TG_PREC_F64)   // refinement ring: 5L double rows + L float rows per stage
        return (size_t)threads / 32 * stages * (5 * kRefineStageLevels * 32 + kRefineStageLevels * 16) * 8;
    if (stages > 0 && lps > 1) return (size_t)threads / 32 * stages * 4 * lps * 32 * 8;
    if (stages > 0) return (size_t)threads / 32 * ((size_t)stages * 4 * 32 * 8 + (w2g ? 0 : 32 * lev * 8));
    if (w2g) return 0;
    if (precision == TG_PREC_F64) return (size_t)threads * cpt * lev * 8;
    return (size_t)threads * 3 * (size_t)k2max * 4;
}

size_t block_smem_bytes(int B, int stages, int threads, int rows, int bw, int precision)
{
    if (precision != TG_PREC_F64)   // refinement ring: P, Q, R, f and u rows per level
        return stages > 0 ? (size_t)threads / 32 * stages * (3 * B * B + 2 * B) * 32 * 8 : 0;
    const int w = rows ? 32 / rows_group(B) : bw;
    return stages > 0 ? (size_t)threads / 32 * stages * (3 * B * B + B) * w * 8 : 0;
}

size_t block_scratch_bytes(int B, int precision, long slots, int k2max)
{
    if (precision == TG_PREC_F64) return (size_t)slots * B * B * (size_t)k2max * 8;
    return (size_t)slots * (2 * B * B + B) * (size_t)k2max * 4;
}

cudaError_t plan_shape(int kind, int precision, int k2max, int ntiles, int cpb, int cpt, int stages, int w2g,
                       Shape *sh)
{
    const int nsm = num_sms();
    int per_sm = 0;
    cudaError_t e = cudaSuccess;
    sh->cpt = cpt;
    sh->threads = stages > 0 ? 32 * ring_warps(kind, precision) : cpb / cpt;
    sh->stages = stages;
    sh->w2g = w2g;
    sh->pf = prefetch_depth(kind, precision);
    sh->rows = stages > 0 ? block_rows(kind, precision) : 0;
    sh->bw = stages > 0 && kind != TG_KIND_SCALAR && !sh->rows ? block_width(kind, precision) : 32;
    // chunked scalar ring: w2 in global scratch, C = stages chunks of lps levels
    sh->lps = stages > 0 && kind == TG_KIND_SCALAR && precision == TG_PREC_F64 && w2g ? g_tile[0][0].lps : 1;
    if (kind == TG_KIND_SCALAR && precision != TG_PREC_F64 && stages > 0)   // refinement ring: 2..4 stages
        stages = sh->stages = stages < 2 ? 2 : (stages > 4 ? 4 : stages);
    // refinement with the whole tile on chip (k_scalar_refine_tile)
    const bool refine_tile = kind == TG_KIND_SCALAR && precision != TG_PREC_F64 && stages > 0 && g_tile[0][1].res > 0 &&
                             (size_t)k2max * kRefineTileBytesPerLevel <= (size_t)(smem_optin() - 1024);
    if (kind == TG_KIND_BLOCK2 && precision != TG_PREC_F64 && stages > 0)   // block refinement ring: 4 or 8 levels
        stages = sh->stages = stages > 4 ? 8 : 4;
    // shared-memory-resident scalar kernel (k_scalar_f64_res): chunked ring of
    // 2..4 stages of 2 or 4 levels, w2 (and w3) on chip, no global scratch
    sh->res = 0;
    if (kind == TG_KIND_SCALAR && precision == TG_PREC_F64 && stages > 0 && g_tile[0][0].res > 0) {
        sh->res = g_tile[0][0].res;
        sh->lps = g_tile[0][0].lps == 2 ? 2 : 4;
        sh->w2g = 0;
        stages = sh->stages = stages < 2 ? 2 : (stages > 4 ? 4 : stages);
    }
    if (sh->lps > 1 && stages > 4) stages = sh->stages = 4;
    if (sh->lps > 1 && sh->lps * stages > 16) stages = sh->stages = 2;
    if (sh->lps == 1 && stages > 0 && stages < 4 && precision == TG_PREC_F64)
        stages = sh->stages = 4;   // per-level rings: depth 4, 8, 16
    if (sh->bw < 32 && stages > 8) stages = sh->stages = 8;
    // block kinds: Gamma resident in shared memory (k_block_f64_ring<..., true>)
    if (kind != TG_KIND_SCALAR && precision == TG_PREC_F64 && stages > 0 && !sh->rows &&
        g_tile[kind_index(kind)][0].res > 0) {
        sh->res = 1;
        if (stages > 8) stages = sh->stages = 8;
        if (with_block_ring_gsm(kind, stages, sh->bw, [](auto) { return cudaSuccess; }) != cudaSuccess) sh->res = 0;
    }
    if (sh->rows && stages > 8) stages = sh->stages = 8;
    if (kind == TG_KIND_SCALAR && sh->cpt == 2 && sh->pf > 8) sh->pf = 8;
    if (stages > 0) {
        // a ring that does not fit in shared memory falls back to the
        // register-prefetch kernel with the same 32-column tile
        if (sh->res && (size_t)sh->threads / 32 * res_rows(stages, sh->lps, k2max, sh->res == 2) * 256 >
                           (size_t)(smem_optin() - 1024)) {
            // columns too tall to stay on chip: the chunked ring with L2 scratch
            sh->res = 0;
            sh->w2g = w2g = 1;
        }
        size_t need = kind == TG_KIND_SCALAR ? scalar_smem_bytes(precision, sh->threads, 1, k2max, stages, w2g, sh->lps)
                                             : block_smem_bytes(kind, stages, sh->threads, sh->rows, sh->bw, precision);
        if (kind != TG_KIND_SCALAR && sh->res) {
            const size_t gam = (size_t)sh->threads / 32 * (size_t)(k2max > 1 ? k2max - 1 : 1) * kind * kind * sh->bw * 8;
            if (need + gam > (size_t)(smem_optin() - 1024)) sh->res = 0;   // too tall: Gamma in L2
            else need += gam;
        }
        if (!sh->res && need > (size_t)(smem_optin() - 1024)) {
            stages = 0;
            sh->stages = 0;
            sh->threads = 32;
            sh->cpt = 1;
            sh->rows = 0;
            sh->bw = 32;
            sh->lps = 1;
        }
    }
    if (refine_tile) {
        sh->res = 3;
        sh->threads = 32;
        sh->smem = (size_t)k2max * kRefineTileBytesPerLevel;
        e = occupancy(k_scalar_refine_tile, 32, sh->smem, &per_sm);
    } else if (kind == TG_KIND_SCALAR) {
        sh->smem = sh->res ? (size_t)sh->threads / 32 * res_rows(stages, sh->lps, k2max, sh->res == 2) * 256
                           : scalar_smem_bytes(precision, sh->threads, sh->cpt, k2max, stages, w2g, sh->lps);
        if (sh->smem > (size_t)(smem_optin() - 1024)) return cudaErrorInvalidConfiguration;
        auto occ = [&](auto k) { return occupancy(k, sh->threads, sh->smem, &per_sm); };
        if (sh->res)
            e = with_scalar_res(stages, sh->lps, sh->res == 2, occ);
        else if (stages > 0 && precision != TG_PREC_F64)
            e = with_scalar_refine_ring(stages, occ);
        else if (stages > 0 && sh->lps > 1)
            e = with_scalar_chunk(stages, sh->lps, occ);
        else if (stages > 0)
            e = with_scalar_ring(stages, w2g, [&](auto k) { return occupancy(k, sh->threads, sh->smem, &per_sm); });
        else if (w2g)
            e = with_scalar_g(sh->pf, occ);
        else if (precision == TG_PREC_F64)
            e = with_scalar_reg(sh->cpt, sh->pf, occ);
        else
            e = with_scalar_refine(sh->pf, occ);
    } else {
        const int B = kind;
        sh->smem = block_smem_bytes(B, stages, sh->threads, sh->rows, sh->bw, precision);
        if (sh->res)
            sh->smem += (size_t)sh->threads / 32 * (size_t)(k2max > 1 ? k2max - 1 : 1) * B * B * sh->bw * 8;
        if (sh->smem > (size_t)(smem_optin() - 1024)) return cudaErrorInvalidConfiguration;
        if (sh->res)
            e = with_block_ring_gsm(B, stages, sh->bw, [&](auto k) { return occupancy(k, sh->threads, sh->smem, &per_sm); });
        else if (stages > 0 && precision != TG_PREC_F64)
            e = with_block_refine_ring(B, stages, [&](auto k) { return occupancy(k, sh->threads, sh->smem, &per_sm); });
        else if (stages > 0 && sh->rows)
            e = with_block_rows(B, stages, [&](auto k) { return occupancy(k, sh->threads, sh->smem, &per_sm); });
        else if (stages > 0)
            e = with_block_ring(B, stages, sh->bw,
                                [&](auto k) { return occupancy(k, sh->threads, sh->smem, &per_sm); });
        else if (precision == TG_PREC_F64)
            e = B == 2 ? occupancy(k_block_f64<2>, sh->threads, 0, &per_sm)
                       : occupancy(k_block_f64<3>, sh->threads, 0, &per_sm);
        else
            e = B == 2 ? occupancy(k_block_refine<2>, sh->threads, 0, &per_sm)
                       : occupancy(k_block_refine<3>, sh->threads, 0, &per_sm);
    }
    if (e != cudaSuccess) return e;
    if (per_sm < 1) return cudaErrorInvalidConfiguration;
    long blocks = (long)per_sm * nsm;
    if (kind != TG_KIND_SCALAR && precision == TG_PREC_F64 && !sh->res) {
        // keep the Gamma scratch of all resident blocks within the L2 budget
        // (a cap on the total, not per SM, so that a grid that fits in one
        // wave is not split into two).  The block refinement kernel is not
        // capped: its loads are latency-bound, and more columns in flight
        // win over the planes' L2 spill (6.2 vs 7.4 ms on the nested batch).
        const double per_thread = (double)block_scratch_bytes(kind, precision, 1, k2max);
        const long cap = (long)(g_block_scratch_budget / (per_thread * sh->threads));
        if (blocks > cap) blocks = cap > 0 ? cap : 1;
    } else if (stages > 0 && sh->res != 2 && sh->res != 3) {
        // ring kernels: w2 scratch plus the w3 parked in x, 8 B each per level
        // and column (refinement: three float planes plus x; w2 on chip: the
        // parked w3 alone), of every resident column within the L2 budget
        // (refinement with hints 2 or 3 keeps its FP64 coefficients in L2
        // between the sweeps: their 32 B per level count too)
        const double per_col = sh->res == 1 ? (double)k2max * 8.0
                               : precision == TG_PREC_F64 ? (double)(2 * k2max - 1) * 8.0
                                                          : (double)k2max * (cache_hints() >= 2 ? 52.0 : 20.0);
        const long cap = (long)(g_scalar_scratch_budget / (per_col * sh->threads * sh->cpt));
        if (blocks > cap) blocks = cap > 0 ? cap : 1;
    }
    const long vt = sh->rows ? (long)ntiles * rows_group(kind)
                             : (kind != TG_KIND_SCALAR ? (long)ntiles * (32 / sh->bw) : ntiles);   // warp tiles
    const long units = stages > 0 ? (vt + sh->threads / 32 - 1) / (sh->threads / 32) : ntiles;
    sh->one_wave = blocks >= units;
    if (blocks > units) blocks = units;
    sh->blocks = (int)(blocks > 0 ? blocks : 1);
    return cudaSuccess;
}

static std::atomic<int> g_cache_hints{1};
int cache_hints() { return g_cache_hints.load(); }
void set_cache_hints(int on) { g_cache_hints.store(on < 0 || on > 3 ? 1 : on); }

cudaError_t launch_scalar(const SegTable &tab, int precision, const Shape &sh, Refine rf, double *scratch,
                          unsigned *status, unsigned long long *hist, cudaStream_t st)
{
    if (tab.ntiles <= 0) return cudaSuccess;
    cudaError_t e = cudaSuccess;
    if (precision != TG_PREC_F64 && sh.res == 3) {
        SegTable t = tab;
        t.hints = cache_hints();
        k_scalar_refine_tile<<<sh.blocks, 32, sh.smem, st>>>(t, rf, status, hist);
    } else if (precision != TG_PREC_F64 && sh.stages > 0) {
        SegTable t = tab;
        t.hints = cache_hints();
        e = with_scalar_refine_ring(sh.stages, [&](auto k) {
            k<<<sh.blocks, sh.threads, sh.smem, st>>>(t, rf, reinterpret_cast<float *>(scratch), status, hist);
            return cudaSuccess;
        });
    } else if (precision == TG_PREC_F64 && sh.stages > 0 && sh.res > 0) {
        SegTable t = tab;
        t.hints = cache_hints();
        e = with_scalar_res(sh.stages, sh.lps, sh.res == 2, [&](auto k) {
            k<<<sh.blocks, sh.threads, sh.smem, st>>>(t, status);
            return cudaSuccess;
        });
    } else if (precision == TG_PREC_F64 && sh.stages > 0 && sh.lps > 1) {
        SegTable t = tab;
        t.hints = cache_hints();
        e = with_scalar_chunk(sh.stages, sh.lps, [&](auto k) {
            k<<<sh.blocks, sh.threads, sh.smem, st>>>(t, scratch, status);
            return cudaSuccess;
        });
    } else if (precision == TG_PREC_F64 && sh.stages > 0) {
        SegTable t = tab;
        t.hints = cache_hints();
        e = with_scalar_ring(sh.stages, sh.w2g, [&](auto k) {
            k<<<sh.blocks, sh.threads, sh.smem, st>>>(t, scratch, status);
            return cudaSuccess;
        });
    } else if (precision == TG_PREC_F64 && sh.w2g) {
        e = with_scalar_g(sh.pf, [&](auto k) {
            k<<<sh.blocks, sh.threads, 0, st>>>(tab, scratch, status);
            return cudaSuccess;
        });
    } else if (precision == TG_PREC_F64) {
        e = with_scalar_reg(sh.cpt, sh.pf, [&](auto k) {
            k<<<sh.blocks, sh.threads, sh.smem, st>>>(tab, status);
            return cudaSuccess;
        });
    } else {
        e = with_scalar_refine(sh.pf, [&](auto k) {
            k<<<sh.blocks, sh.threads, sh.smem, st>>>(tab, rf, status, hist);
            return cudaSuccess;
        });
    }
    if (e != cudaSuccess) return e;
    return cudaGetLastError();
}

cudaError_t launch_block(const SegTable &tab, int B, int precision, const Shape &sh, Refine rf,
                         double *scratch, unsigned *status, unsigned long long *hist, cudaStream_t st)
{
    if (tab.ntiles <= 0) return cudaSuccess;
    if (precision != TG_PREC_F64 && sh.stages > 0) {
        SegTable t = tab;
        t.hints = cache_hints();
        cudaError_t e = with_block_refine_ring(B, sh.stages, [&](auto k) {
            k<<<sh.blocks, sh.threads, sh.smem, st>>>(t, rf, reinterpret_cast<float *>(scratch), status, hist);
            return cudaSuccess;
        });
        if (e != cudaSuccess) return e;
    } else if (precision == TG_PREC_F64 && sh.stages > 0 && sh.res) {
        SegTable t = tab;
        t.hints = cache_hints();
        cudaError_t e = with_block_ring_gsm(B, sh.stages, sh.bw, [&](auto k) {
            k<<<sh.blocks, sh.threads, sh.smem, st>>>(t, scratch, status);
            return cudaSuccess;
        });
        if (e != cudaSuccess) return e;
    } else if (precision == TG_PREC_F64 && sh.stages > 0 && sh.rows) {
        SegTable t = tab;
        t.hints = cache_hints();
        cudaError_t e = with_block_rows(B, sh.stages, [&](auto k) {
            k<<<sh.blocks, sh.threads, sh.smem, st>>>(t, scratch, status);
            return cudaSuccess;
        });
        if (e != cudaSuccess) return e;
    } else if (precision == TG_PREC_F64 && sh.stages > 0) {
        SegTable t = tab;
        t.hints = cache_hints();
        cudaError_t e = with_block_ring(B, sh.stages, sh.bw, [&](auto k) {
            k<<<sh.blocks, sh.threads, sh.smem, st>>>(t, scratch, status);
            return cudaSuccess;
        });
        if (e != cudaSuccess) return e;
    } else if (precision == TG_PREC_F64) {
        if (B == 2)
            k_block_f64<2><<<sh.blocks, sh.threads, 0, st>>>(tab, scratch, status);
        else
            k_block_f64<3><<<sh.blocks, sh.threads, 0, st>>>(tab, scratch, status);
    } else {
        float *fs = reinterpret_cast<float *>(scratch);
        SegTable t = tab;
        t.hints = cache_hints();
        if (B == 2)
            k_block_refine<2><<<sh.blocks, sh.threads, 0, st>>>(t, rf, fs, status, hist);
        else
            k_block_refine<3><<<sh.blocks, sh.threads, 0, st>>>(t, rf, fs, status, hist);
    }
    return cudaGetLastError();
}

cudaError_t kernel_binary_version(int *v)
{
    cudaFuncAttributes attr{};
    const cudaError_t e = cudaFuncGetAttributes(&attr, k_col_to_level);
    if (e == cudaSuccess) *v = attr.binaryVersion;
    return e;
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

cudaError_t launch_col_to_level_multi(const Relayout &r, cudaStream_t st)
{
    long tiles = 0;
    for (int a = 0; a < r.n; ++a) {
        const long t = ((r.nrows[a] + 31) / 32) * ((r.ncols + 31) / 32);
        tiles = t > tiles ? t : tiles;
    }
    if (tiles <= 0 || r.n <= 0) return cudaSuccess;
    const long cap = (long)num_sms() * 4;
    const int bx = (int)(tiles < cap ? tiles : cap);
    k_col_to_level_multi<<<dim3(bx, r.n), dim3(32, 8), 0, st>>>(r);
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
