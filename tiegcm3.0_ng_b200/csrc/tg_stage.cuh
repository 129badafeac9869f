// Per-thread software pipelining of a column walk's reads: while iteration k
// computes, asynchronous 8-byte copies (cp.async) bring the values iteration
// k+1 will read into a two-buffer shared-memory array [buffer][value][thread].
// Each thread reads only what it copied itself, so no block barrier is needed.
#pragma once
#include <cuda_runtime.h>

namespace tg {

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
