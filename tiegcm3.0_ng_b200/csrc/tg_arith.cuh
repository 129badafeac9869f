// Exact FP64 arithmetic helpers shared by the solver and assembly kernels.
#pragma once
#include <cfloat>
#include <cuda_runtime.h>

namespace tg {

__device__ __forceinline__ double xmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double xsub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double xadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double xdiv(double a, double b) { return __ddiv_rn(a, b); }
__device__ __forceinline__ bool finite_nz(double w) { return fabs(w) <= DBL_MAX && w != 0.0; }
__device__ __forceinline__ bool finite(double w) { return fabs(w) <= DBL_MAX; }

// Correctly rounded quotients that share a divisor.  y = __drcp_rn(b) is the
// correctly rounded reciprocal; q0 = RN(a*y) is within ~2 ulp of a/b, one
// FMA correction q1 = RN(q0 + RN(a - b*q0)*y) brings it within 1 ulp, and
// Markstein's theorem (P. Markstein, IBM J. Res. Dev. 34(1), 1990; Muller et
// al., Handbook of Floating-Point Arithmetic, Thm. 5.8) makes the second
// correction RN(q1 + (a - b*q1)*y) equal to RN(a/b), provided nothing
// underflows or overflows.  div_safe() keeps a, b (and hence a/b and the
// residuals) well inside the normal range; other operands, zeros included
// (whose quotient's sign the correction steps would not keep), take IEEE
// division.
// The result is therefore bit-identical to a/b; tg_selftest_division checks
// it against the hardware division.
__device__ __forceinline__ bool div_safe(double a, double b)
{
    const double lo = 0x1p-500, hi = 0x1p500;
    const double fa = fabs(a), fb = fabs(b);
    return fb >= lo && fb <= hi && fa >= lo && fa <= hi;
}
__device__ __forceinline__ double div_markstein(double a, double b, double y)
{
    double q = __dmul_rn(a, y);
    double r = __fma_rn(-b, q, a);
    q = __fma_rn(r, y, q);
    r = __fma_rn(-b, q, a);
    return __fma_rn(r, y, q);
}
// a/b, correctly rounded, given y = __drcp_rn(b).
__device__ __forceinline__ double qdiv(double a, double b, double y)
{
    return div_safe(a, b) ? div_markstein(a, b, y) : __ddiv_rn(a, b);
}

// |v| in [2^-500, 2^500) from the exponent bits alone (biased exponent
// 523..1522): integer operations, a subset of div_safe's range.
__device__ __forceinline__ bool exp_safe(double v)
{
    const unsigned e2 = (unsigned)__double2hiint(v) * 2u - (523u << 21);   // sign bit shifted out
    return e2 < (1000u << 21);
}
// exp_safe's biased-exponent distance, combined over several values with max:
// all are safe when the maximum is below kExpSpan.
constexpr unsigned kExpSpan = 1000u << 21;
__device__ __forceinline__ unsigned exp_dist(double v) { return (unsigned)__double2hiint(v) * 2u - (523u << 21); }
// a/b, correctly rounded, given y = __drcp_rn(b) and b_safe = exp_safe(b),
// which a recurrence computes once for the two divisions by the same pivot.
__device__ __forceinline__ double qdiv_pivot(double a, double b, double y, bool b_safe)
{
    return b_safe && exp_safe(a) ? div_markstein(a, b, y) : __ddiv_rn(a, b);
}

// a/b, correctly rounded, given y = __drcp_rn(b): one exponent-range test
// (integer operations) for both operands, a subset of div_safe's range.
__device__ __forceinline__ double qdiv1(double a, double b, double y)
{
    return max(exp_dist(a), exp_dist(b)) < kExpSpan ? div_markstein(a, b, y) : __ddiv_rn(a, b);
}
// Both quotients by one pivot, qa = a/b and qc = c/b, correctly rounded,
// given y = __drcp_rn(b), under one exponent-range test for the three
// operands (a recurrence's w3 and next w2).
__device__ __forceinline__ void qdiv2(double a, double c, double b, double y, double &qa, double &qc)
{
    if (max(exp_dist(b), max(exp_dist(a), exp_dist(c))) < kExpSpan) {
        qa = div_markstein(a, b, y);
        qc = div_markstein(c, b, y);
    } else {
        const bool bs = exp_safe(b);
        qa = qdiv_pivot(a, b, y, bs);
        qc = qdiv_pivot(c, b, y, bs);
    }
}

// A hint that brings the line holding p into L1 (no register, no wait).
__device__ __forceinline__ void pf_l1(const void *p) { asm volatile("prefetch.global.L1 [%0];" ::"l"(p)); }

// The reads of post_store at index o, requested ahead of the store.
template <class P>
__device__ __forceinline__ void post_prefetch(const P &post, bool on, bool bcol, const double *out, long o)
{
    pf_l1(out + o);
    if (!on) return;
    pf_l1(post.prev + o);
    pf_l1(post.cur + o);
    if (bcol) pf_l1(post.bnd + o);
}

// The store of solution row o with the post-solve steps when `on`: a flagged
// lateral-boundary column takes its boundary value, the previous-step field
// is filtered, nm = ds2*(prev + x) + ds*cur, and both are floored (a floor
// keeps v when v > floor, NaN included otherwise).  The same operations as
// the reference's statements and as tg_time_filter_ng.
// post_store with the previous- and current-step values already read (the
// shared-memory tile walks copy them in with the rows).
template <class P>
__device__ __forceinline__ void post_store_v(const P &post, bool bcol, double *out, long o, double x, double prev,
                                             double cur)
{
    if (bcol) x = __ldg(post.bnd + o);
    const double n = __dadd_rn(__dmul_rn(post.ds2, __dadd_rn(prev, x)), __dmul_rn(post.ds, cur));
    post.nm[o] = (!post.floor_nm || n > post.floor) ? n : post.floor;
    out[o] = x > post.floor ? x : post.floor;
}

template <class P>
__device__ __forceinline__ void post_store(const P &post, bool on, bool bcol, double *out, long o, double x)
{
    if (!on) {
        out[o] = x;
        return;
    }
    if (bcol) x = __ldg(post.bnd + o);
    // plain loads: nm may alias prev or cur
    const double n = __dadd_rn(__dmul_rn(post.ds2, __dadd_rn(post.prev[o], x)), __dmul_rn(post.ds, post.cur[o]));
    post.nm[o] = (!post.floor_nm || n > post.floor) ? n : post.floor;
    out[o] = x > post.floor ? x : post.floor;
}

}  // namespace tg
