// Per-thread software pipelining of a column walk's reads: while iteration k
// computes, asynchronous 8-byte copies (cp.async) bring the values iteration
// k+1 will read into a two-buffer shared-memory array [buffer][value][thread].
// Each thread reads only what it copied itself, so no block barrier is needed.
#pragma once
#include <cuda_runtime.h>

namespace tg {

// One asynchronous 8-byte copy global -> shared, and the group operations.
__device__ __forceinline__ void cp_async8(double *dst, const double *src)
{
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"((unsigned)__cvta_generic_to_shared(dst)), "l"(src)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

// Back sweep of a 32-column tile held in shared memory (rows of 32):
// x(k) = w3(k) - w2(k)*x(k+1) for k = K-2 .. 0 from x(K-1) = xtop, the w3
// rows in sx (overwritten by x), the w2 rows in sw2.  The operands of the
// next four levels are read ahead into registers, off the chain, and the
// main loop runs without per-level guards (one level's chain: a product and
// a difference).
__device__ __forceinline__ void back_sweep(double *sx, const double *sw2, int K, int t, double xtop)
{
    double xn = xtop, rw[4] = {0., 0., 0., 0.}, r2[4] = {0., 0., 0., 0.};
#pragma unroll
    for (int u = 0; u < 4; ++u)
        if (K - 2 - u >= 0) {
            rw[u] = sx[(K - 2 - u) * 32 + t];
            r2[u] = sw2[(K - 2 - u) * 32 + t];
        }
    int kb = K - 2;
    for (; kb - 7 >= 0; kb -= 4) {   // four levels and their read-ahead all in range
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int k = kb - u;
            xn = __dsub_rn(rw[u], __dmul_rn(r2[u], xn));
            rw[u] = sx[(k - 4) * 32 + t];
            r2[u] = sw2[(k - 4) * 32 + t];
            sx[k * 32 + t] = xn;
        }
    }
    for (; kb >= 0; kb -= 4) {
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int k = kb - u;
            if (k >= 0) {
                xn = __dsub_rn(rw[u], __dmul_rn(r2[u], xn));
                if (k - 4 >= 0) {
                    rw[u] = sx[(k - 4) * 32 + t];
                    r2[u] = sw2[(k - 4) * 32 + t];
                }
                sx[k * 32 + t] = xn;
            }
        }
    }
}

template <int NV>
struct Stage {
    double *sm;   // this thread's column of the block's array (base + threadIdx.x)
    int T;        // threads per block: the array's row stride
    __device__ __forceinline__ double &at(int b, int v) const { return sm[(long)(b * NV + v) * T]; }
    __device__ __forceinline__ void copy(int b, int v, const double *src) const
    {
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"((unsigned)__cvta_generic_to_shared(&at(b, v))),
                     "l"(src)
                     : "memory");
    }
    __device__ __forceinline__ static void commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
    // every group but the most recent one has landed
    __device__ __forceinline__ static void wait_prev() { asm volatile("cp.async.wait_group 1;" ::: "memory"); }
    __device__ __forceinline__ static void wait_all() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }
    static constexpr size_t bytes_per_thread = 2 * NV * sizeof(double);
};

}  // namespace tg
