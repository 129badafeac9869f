// The column walk of the three-pass assembly routines: the Thomas solve
// (src/trsolv_ng.F90:14-26) of rows already formed by a level-parallel pass,
// stored through the routines' post-solve steps.
//
// In the two-pass form each walk forms its rows as it goes (hundreds of
// dependent instructions per level, one thread per column); with few columns
// per SM every level then waits on its own instruction latencies.  Here the
// rows come from planes p, q, r, f (level-major, k*ld + col) that one thread
// per (level, column) wrote, so a walk level is the recurrence alone: two
// divisions sharing one correctly rounded reciprocal (qdiv), a product and a
// difference, with the planes requested pd levels ahead.
//
//   top = 0 (minor_ng): rows 0..K-1 with K = nk, no extrapolation;
//   top = 1 (dt_ng, oplus_ng): rows 0..K-1 with K = nk-1 and
//         x(nk-1) = x(nk-2)**2/x(nk-3) from the unfiltered values
//         (dt_ng.F90:167, oplus_ng.F90:307).
// With a PostStep every row is stored through post_store: the lateral
// boundary overwrite, the time filter and the floors.  Same operations in the
// same order as the fused walks, so the same bits.
#include <cfloat>

#include "tg_internal.h"
#include "tg_arith.cuh"
#include "tg_stage.cuh"

namespace tg {
namespace {
__device__ __forceinline__ double xm(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double xs(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double xd(double a, double b) { return __ddiv_rn(a, b); }

constexpr int kWalkThreads = 32;   // one warp per block: the walk's columns spread over every SM

__global__ void __launch_bounds__(kWalkThreads) k_thomas_post(const double *P, const double *Q, const double *R,
                                                              const double *Fv, double *x, int nk, int K, int top,
                                                              int ncol, long ld, unsigned *status, PostStep post,
                                                              int has_post, int pd)
{
    extern __shared__ double w2_walk[];
    const long col = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (col >= ncol) return;
    const int T = blockDim.x;
    double *w2s = w2_walk + threadIdx.x;
    auto pf_row = [&](int k) {
        const long o = (long)k * ld + col;
        pf_l1(P + o);
        pf_l1(Q + o);
        pf_l1(R + o);
        pf_l1(Fv + o);
    };
    for (int kk = 1; kk < pd && kk < K; ++kk) pf_row(kk);
    bool ok = true;
    double w1 = 0.0, y1 = 0.0, w3 = 0.0, rprev = 0.0;
    for (int k = 0; k < K; ++k) {
        if (k + pd < K) pf_row(k + pd);
        const long o = (long)k * ld + col;
        const double p = P[o], q = Q[o], r = R[o], f = Fv[o];
        if (k == 0) {
            w1 = q;
            y1 = __drcp_rn(w1);
            w3 = qdiv(f, w1, y1);
        } else {
            const double w2 = qdiv(rprev, w1, y1);
            w2s[(long)(k - 1) * T] = w2;
            w1 = xs(q, xm(p, w2));
            y1 = __drcp_rn(w1);
            w3 = qdiv(xs(f, xm(p, w3)), w1, y1);
        }
        ok = ok && fabs(w1) <= DBL_MAX && w1 != 0.0;
        x[o] = w3;
        rprev = r;
    }
    const bool bcol = has_post && post.bnd_mask && post.bnd_mask[col];
    double xn = w3;
    const double xtop = w3;
    bool fin = fabs(xn) <= DBL_MAX;
    double park = K >= 2 ? x[(long)(K - 2) * ld + col] : 0.0;
    if (top == 0 && has_post) post_store(post, true, bcol, x, (long)(K - 1) * ld + col, xn);
    for (int kk = K - 3; kk > K - 2 - pd && kk >= 0; --kk) post_prefetch(post, has_post, bcol, x, (long)kk * ld + col);
    for (int k = K - 2; k >= 0; --k) {
        if (k - pd >= 0) post_prefetch(post, has_post, bcol, x, (long)(k - pd) * ld + col);
        const double wk = park;
        if (k >= 1) park = x[(long)(k - 1) * ld + col];
        xn = xs(wk, xm(w2s[(long)k * T], xn));
        fin = fin && fabs(xn) <= DBL_MAX;
        post_store(post, has_post, bcol, x, (long)k * ld + col, xn);
        if (top == 1 && k == K - 2) {
            // xtop = x(K-1), xn = x(K-2): the two top solved rows
            post_store(post, has_post, bcol, x, (long)K * ld + col, xd(xm(xtop, xtop), xn));
            if (has_post) post_store(post, true, bcol, x, (long)(K - 1) * ld + col, xtop);
        }
    }
    if (status && (!ok || !fin)) atomicOr(status, (ok ? 0u : FLAG_PIVOT) | (fin ? 0u : FLAG_NONFINITE));
}
// The same walk with the column tile held in shared memory, for launches of
// few columns.  The kTileWarps warps of a block share one 32-column tile:
// together they copy the p, q, r, f rows of every level (cp.async, every
// copy in flight at once, each warp a quarter of the levels), then warp 0
// alone runs the recurrence from shared memory, keeping the next level's
// w2 = r(k)/w1(k) where r(k) was and the parked w3, then the solution, where
// q(k) was; finally all warps
// store the rows through the post-solve steps, each its quarter of the
// levels.  The per-column serial part is the recurrence alone.
constexpr int kTileWarps = 4;
__global__ void __launch_bounds__(32 * kTileWarps) k_thomas_post_tile(const double *P, const double *Q,
                                                                      const double *R, const double *Fv, double *x,
                                                                      int nk, int K, int top, int ncol, long ld,
                                                                      unsigned *status, PostStep post, int has_post)
{
    extern __shared__ double tile_walk[];
    const int T = 32, t = threadIdx.x & 31, w = threadIdx.x >> 5, NW = kTileWarps;
    const long col = (long)blockIdx.x * T + t;
    const bool live = col < ncol;
    // with the post-solve steps, prev and cur of every stored row (K, and the
    // top row for top = 1) come in with the rows; q holds the KS solved rows
    const int KS = top == 1 ? K + 1 : K;
    double *sp = tile_walk, *sq = sp + (long)K * T, *sr = sq + (long)KS * T, *sf = sr + (long)K * T;
    double *sprev = sf + (long)K * T, *scur = sprev + (long)KS * T;
    if (live) {
        for (int k = w; k < K; k += NW) {
            const long o = (long)k * ld + col;
            const int s = k * T + t;
            cp_async8(sp + s, P + o);
            cp_async8(sq + s, Q + o);
            cp_async8(sr + s, R + o);
            cp_async8(sf + s, Fv + o);
        }
        if (has_post)
            for (int k = w; k < KS; k += NW) {
                const long o = (long)k * ld + col;
                cp_async8(sprev + k * T + t, post.prev + o);
                cp_async8(scur + k * T + t, post.cur + o);
            }
    }
    cp_async_commit();
    cp_async_wait<0>();
    __syncthreads();
    if (w == 0 && live) {
        // Level k divides by its pivot w1(k) twice: w3(k) and the next
        // level's w2 = r(k)/w1(k) (the reference's operands, so the same
        // quotients), kept where r(k) was.  The walk's chain is the
        // recurrence alone: every quotient by Markstein's sequence, no
        // branch, each level's operands read one level ahead.  A level whose
        // operands leave the sequence's safe range (zeros, non-finite or
        // extreme values) stops the stores; the levels from the first such
        // one are then walked again with the IEEE fallback (qdiv2, qdiv1).
        bool ok = true;
        int bad = K;
        double w1 = 0.0, y1 = 0.0, w2 = 0.0, w3 = 0.0;
        auto level = [&](int k, double p, double q, double r, double f, bool top_level) {
            w1 = k == 0 ? q : xs(q, xm(p, w2));
            y1 = __drcp_rn(w1);
            const double num = k == 0 ? f : xs(f, xm(p, w3));
            ok = ok && (bad < K || finite_nz(w1));
            const unsigned d = max(exp_dist(w1), max(exp_dist(num), top_level ? 0u : exp_dist(r)));
            bad = d >= kExpSpan && bad == K ? k : bad;
            w3 = div_markstein(num, w1, y1);
            w2 = div_markstein(r, w1, y1);
            if (bad > k) {
                sr[k * T + t] = w2;
                sq[k * T + t] = w3;
            }
        };
        double pn = sp[t], qn = sq[t], rn = sr[t], fn = sf[t];
        for (int k = 0; k < K - 1; ++k) {
            const int s = k * T + t;
            const double p = pn, q = qn, r = rn, f = fn;
            pn = sp[s + T];
            qn = sq[s + T];
            rn = sr[s + T];
            fn = sf[s + T];
            level(k, p, q, r, f, false);
        }
        level(K - 1, pn, qn, rn, fn, true);
        if (bad < K) {
            w2 = bad > 0 ? sr[(bad - 1) * T + t] : 0.0;
            w3 = bad > 0 ? sq[(bad - 1) * T + t] : 0.0;
            for (int k = bad; k < K; ++k) {
                const int s = k * T + t;
                const double p = sp[s], q = sq[s], f = sf[s];
                w1 = k == 0 ? q : xs(q, xm(p, w2));
                y1 = __drcp_rn(w1);
                const double num = k == 0 ? f : xs(f, xm(p, w3));
                if (k + 1 < K) {
                    qdiv2(num, sr[s], w1, y1, w3, w2);
                    sr[s] = w2;
                } else {
                    w3 = qdiv1(num, w1, y1);
                }
                ok = ok && finite_nz(w1);
                sq[s] = w3;
            }
        }
        const double xtop = w3;
        back_sweep(sq, sr, K, t, w3);
        // x(k) = w3 - w2*x(k+1) carries a non-finite value down to x(0)
        const bool fin = finite(sq[t]) && finite(xtop);
        // x(nk-1) = x(nk-2)**2/x(nk-3) from the unfiltered values
        if (top == 1) sq[K * T + t] = xd(xm(xtop, xtop), sq[(K - 2) * T + t]);
        if (status && (!ok || !fin)) atomicOr(status, (ok ? 0u : FLAG_PIVOT) | (fin ? 0u : FLAG_NONFINITE));
    }
    __syncthreads();
    if (!live) return;
    if (has_post) {
        const bool bcol = post.bnd_mask && post.bnd_mask[col];
        for (int k = w; k < KS; k += NW)
            post_store_v(post, bcol, x, (long)k * ld + col, sq[k * T + t], sprev[k * T + t], scur[k * T + t]);
    } else {
        for (int k = w; k < KS; k += NW) x[(long)k * ld + col] = sq[k * T + t];
    }
}

// The walk for launches above the tile limit, one warp per 32-column block:
// each lane's rows of p, q, r, f stream through a two-buffer shared-memory
// ring of kRingLevels levels, the copies of the next chunk in flight while
// this one is walked (a lane reads only what it copied itself: no barrier).
// w2 of every level stays in shared memory, w3 is parked in x; the main loop
// is branch-free Markstein with the IEEE re-walk from the first out-of-range
// level (from the planes in global memory), as in the tile walk.  The back
// sweep leaves the solution in shared memory where w2 was, and the stores
// through the post steps go out last.
constexpr int kRingLevels = 4;
__global__ void __launch_bounds__(32) k_thomas_post_ring(const double *P, const double *Q, const double *R,
                                                         const double *Fv, double *x, int nk, int K, int top,
                                                         int ncol, long ld, unsigned *status, PostStep post,
                                                         int has_post)
{
    extern __shared__ double ring_walk[];
    const int T = 32, t = threadIdx.x, L = kRingLevels;
    const long col = (long)blockIdx.x * T + t;
    if (col >= ncol) return;
    const int KS = top == 1 ? K + 1 : K, nch = (K + L - 1) / L;
    double *rb = ring_walk, *sw = ring_walk + 2 * L * 4 * T;   // ring [2][L][4][32]; w2, then x: KS rows
    const double *src[4] = {P, Q, R, Fv};
    auto load = [&](int c) {
        const int k0 = c * L, nl = K - k0 < L ? K - k0 : L;
        double *buf = rb + (c & 1) * L * 4 * T + t;
        for (int l = 0; l < nl; ++l)
#pragma unroll
            for (int v = 0; v < 4; ++v) cp_async8(buf + (l * 4 + v) * T, src[v] + (long)(k0 + l) * ld + col);
        cp_async_commit();
    };
    bool ok = true;
    int bad = K;
    double w1 = 0.0, y1 = 0.0, w2 = 0.0, w3 = 0.0;
    load(0);
    for (int c = 0; c < nch; ++c) {
        if (c + 1 < nch) load(c + 1);
        else cp_async_commit();
        cp_async_wait<1>();
        const double *buf = rb + (c & 1) * L * 4 * T + t;
        const int k0 = c * L, nl = K - k0 < L ? K - k0 : L;
        for (int l = 0; l < nl; ++l) {
            const int k = k0 + l;
            const double p = buf[(l * 4) * T], q = buf[(l * 4 + 1) * T], r = buf[(l * 4 + 2) * T],
                         f = buf[(l * 4 + 3) * T];
            w1 = k == 0 ? q : xs(q, xm(p, w2));
            y1 = __drcp_rn(w1);
            const double num = k == 0 ? f : xs(f, xm(p, w3));
            ok = ok && (bad < K || finite_nz(w1));
            const unsigned d = max(exp_dist(w1), max(exp_dist(num), k + 1 == K ? 0u : exp_dist(r)));
            bad = d >= kExpSpan && bad == K ? k : bad;
            w3 = div_markstein(num, w1, y1);
            w2 = div_markstein(r, w1, y1);
            if (bad > k) {
                sw[k * T + t] = w2;
                x[(long)k * ld + col] = w3;
            }
        }
    }
    if (bad < K) {
        // from the first out-of-range level, the divisions with their IEEE
        // fallback, the rows read again from the planes
        w2 = bad > 0 ? sw[(bad - 1) * T + t] : 0.0;
        w3 = bad > 0 ? x[(long)(bad - 1) * ld + col] : 0.0;
        for (int k = bad; k < K; ++k) {
            const long o = (long)k * ld + col;
            const double p = P[o], q = Q[o], f = Fv[o];
            w1 = k == 0 ? q : xs(q, xm(p, w2));
            y1 = __drcp_rn(w1);
            const double num = k == 0 ? f : xs(f, xm(p, w3));
            if (k + 1 < K) qdiv2(num, R[o], w1, y1, w3, w2);
            else w3 = qdiv1(num, w1, y1);
            ok = ok && finite_nz(w1);
            sw[k * T + t] = w2;
            x[o] = w3;
        }
    }
    // back sweep: x(k) = w3(k) - w2(k)*x(k+1), w3 from x four levels ahead
    const double xtop = w3;
    double xn = xtop, rw[4] = {0., 0., 0., 0.};
#pragma unroll
    for (int u = 0; u < 4; ++u)
        if (K - 2 - u >= 0) rw[u] = x[(long)(K - 2 - u) * ld + col];
    sw[(K - 1) * T + t] = xtop;
    int kb = K - 2;
    for (; kb - 7 >= 0; kb -= 4) {
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int k = kb - u;
            xn = xs(rw[u], xm(sw[k * T + t], xn));
            rw[u] = x[(long)(k - 4) * ld + col];
            sw[k * T + t] = xn;
        }
    }
    for (; kb >= 0; kb -= 4) {
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int k = kb - u;
            if (k >= 0) {
                xn = xs(rw[u], xm(sw[k * T + t], xn));
                if (k - 4 >= 0) rw[u] = x[(long)(k - 4) * ld + col];
                sw[k * T + t] = xn;
            }
        }
    }
    // x(k) = w3 - w2*x(k+1) carries a non-finite value down to x(0)
    const bool fin = finite(sw[t]) && finite(xtop);
    // x(nk-1) = x(nk-2)**2/x(nk-3) from the unfiltered values
    if (top == 1) sw[K * T + t] = xd(xm(xtop, xtop), sw[(K - 2) * T + t]);
    if (status && (!ok || !fin)) atomicOr(status, (ok ? 0u : FLAG_PIVOT) | (fin ? 0u : FLAG_NONFINITE));
    if (has_post) {
        const bool bcol = post.bnd_mask && post.bnd_mask[col];
        for (int k = 0; k < KS; ++k) post_store(post, true, bcol, x, (long)k * ld + col, sw[k * T + t]);
    } else {
        for (int k = 0; k < KS; ++k) x[(long)k * ld + col] = sw[k * T + t];
    }
}
}  // namespace

cudaError_t launch_thomas_post(const double *p, const double *q, const double *r, const double *f, double *x, int nk,
                               int K, int top, int ncol, long ld, unsigned *status, const PostStep *post,
                               cudaStream_t st)
{
    if (ncol <= 0) return cudaSuccess;
    if (K < 1 || K > nk || (top == 1 && (K != nk - 1 || K < 2))) return cudaErrorInvalidValue;
    const int KS = top == 1 ? K + 1 : K;
    const size_t tile = (size_t)32 * (3 * K + KS + (post ? 2 * KS : 0)) * sizeof(double);
    if (ncol <= kSmallWalkColumns && tile <= (size_t)smem_optin()) {
        once_per_device([] {
            cudaFuncSetAttribute(k_thomas_post_tile, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_optin());
        });
        k_thomas_post_tile<<<(ncol + 31) / 32, 32 * kTileWarps, tile, st>>>(
            p, q, r, f, x, nk, K, top, ncol, ld, status, post ? *post : PostStep{}, post != nullptr);
        return cudaGetLastError();
    }
    const size_t ring = (size_t)32 * (2 * kRingLevels * 4 + KS) * sizeof(double);
    if (ring <= (size_t)smem_optin()) {
        once_per_device([] {
            cudaFuncSetAttribute(k_thomas_post_ring, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_optin());
        });
        k_thomas_post_ring<<<(ncol + 31) / 32, 32, ring, st>>>(p, q, r, f, x, nk, K, top, ncol, ld, status,
                                                               post ? *post : PostStep{}, post != nullptr);
        return cudaGetLastError();
    }
    const size_t smem = (size_t)kWalkThreads * (K > 1 ? K - 1 : 1) * sizeof(double);
    once_per_device([] { cudaFuncSetAttribute(k_thomas_post, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_optin()); });
    if (smem > (size_t)smem_optin()) return cudaErrorInvalidValue;
    k_thomas_post<<<(ncol + kWalkThreads - 1) / kWalkThreads, kWalkThreads, smem, st>>>(
        p, q, r, f, x, nk, K, top, ncol, ld, status, post ? *post : PostStep{}, post != nullptr,
        walk_prefetch(ncol));
    return cudaGetLastError();
}
}  // namespace tg
