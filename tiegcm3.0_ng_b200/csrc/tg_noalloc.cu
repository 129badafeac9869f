// tg_blksolve_dev_noalloc: the FP64 block-tridiagonal solve for callers that
// cannot allocate device memory.
//
// The regular device entry (tg_blksolve_dev) grows a library-owned scratch
// buffer with cudaMalloc on demand, and cudaFree of an outgrown buffer
// synchronises the whole device.  Some callers cannot accept either:
//   - a model running under a fixed, pre-reserved device-memory budget (all
//     of the GPU handed to one pool at start-up), where a later cudaMalloc
//     fails or steals memory from the pool;
//   - a time loop that shares the GPU with other work in flight and must
//     not be stalled by the implicit device synchronisation of cudaFree.
// This entry point allocates nothing.  Its scratch (the Gamma blocks of the
// block Thomas sweep, B*B doubles per level per resident thread) lives in the
// fixed array below, which every GPU that loads the library holds until the
// process exits.  The caller still passes the inputs and outputs.
#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdio>
#include <mutex>

#include "tg_internal.h"

namespace {

// 16 MiB of FP64 scratch, plus one status word.
constexpr long kScratchDoubles = (16l << 20) / (long)sizeof(double);
static __device__ __align__(256) double g_noalloc_scratch[kScratchDoubles];
static __device__ __align__(256) unsigned g_noalloc_flags[1];
// Columns per thread block of this entry's launches: fixed, so that its
// limit (B*B*k2*kTileColumns <= kScratchDoubles) does not depend on the
// tuning entries.
constexpr int kTileColumns = 64;

// Device addresses of the two arrays, looked up once per device and context.
// The names above are host-side stand-ins in host code, never device
// addresses.  A device reset (cudaDeviceReset) destroys the context and the
// module; the next context may load the array elsewhere, so the cached
// addresses are tied to the unique id of the context they were looked up in.
struct DevPtrs {
    bool ready = false;
    unsigned long long ctx_id = 0;
    double *scratch = nullptr;
    unsigned *flags = nullptr;
};
constexpr int kMaxDev = 64;
DevPtrs g_ptrs[kMaxDev];
std::mutex g_mu;

// Unique id of the calling thread's current context (driver entries reached
// through the runtime, so the library needs no link to libcuda); 0 when none
// is current or the driver cannot say.
unsigned long long current_ctx_id()
{
    typedef CUresult (*GetCurrent)(CUcontext *);
    typedef CUresult (*GetId)(CUcontext, unsigned long long *);
    static GetCurrent get_current = nullptr;
    static GetId get_id = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void *fn = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", &fn, 12000, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_current = (GetCurrent)fn;
        fn = nullptr;
        if (cudaGetDriverEntryPointByVersion("cuCtxGetId", &fn, 12000, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_id = (GetId)fn;
        cudaGetLastError();
    });
    CUcontext ctx = nullptr;
    unsigned long long id = 0;
    if (!get_current || !get_id || get_current(&ctx) != CUDA_SUCCESS || !ctx || get_id(ctx, &id) != CUDA_SUCCESS)
        return 0;
    return id;
}

int device_ptrs(DevPtrs *out)
{
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess || dev < 0 || dev >= kMaxDev) {
        tg::record_error("tg_blksolve_dev_noalloc: no usable CUDA device");
        return TG_ENODEV;
    }
    std::lock_guard<std::mutex> lk(g_mu);
    DevPtrs &p = g_ptrs[dev];
    // a context other than the one of the cached addresses (or none yet,
    // before the first runtime call on this device): look them up again;
    // the lookup makes the device's primary context current
    if (p.ready && (p.ctx_id == 0 || current_ctx_id() != p.ctx_id)) p.ready = false;
    if (!p.ready) {
        e = cudaGetSymbolAddress((void **)&p.scratch, g_noalloc_scratch);
        if (e != cudaSuccess) {
            char msg[256];
            snprintf(msg, sizeof msg, "tg_blksolve_dev_noalloc: cudaGetSymbolAddress(scratch) failed: %s",
                     cudaGetErrorString(e));
            tg::record_error(msg);
            return TG_ECUDA;
        }
        e = cudaGetSymbolAddress((void **)&p.flags, g_noalloc_flags);
        if (e != cudaSuccess) {
            char msg[256];
            snprintf(msg, sizeof msg, "tg_blksolve_dev_noalloc: cudaGetSymbolAddress(flags) failed: %s",
                     cudaGetErrorString(e));
            tg::record_error(msg);
            return TG_ECUDA;
        }
        p.ctx_id = current_ctx_id();
        p.ready = true;
    }
    *out = p;
    return TG_OK;
}

__global__ void k_noalloc_status(const unsigned *flags, int *out)
{
    const unsigned f = *flags;
    *out = (f & tg::FLAG_TIMEOUT) ? TG_ETIMEOUT : (f & tg::FLAG_PIVOT) ? TG_EPIVOT : (f & tg::FLAG_NONFINITE) ? TG_ENONFINITE : TG_OK;
}

}  // namespace

extern "C" __attribute__((visibility("default"))) int tg_blksolve_dev_noalloc(
    int B, const double *P, const double *Q, const double *R, const double *f, const double *ubc_ratio,
    const double *ubc_add, double *u, int nk, int k2, int ncol, long ld, int *status_dev, void *stream)
{
    if ((B != 2 && B != 3) || !P || !Q || !R || !f || !u || nk < 1 || k2 < 1 || k2 > nk || ncol < 0 ||
        ld < ncol || (ubc_ratio && k2 >= nk)) {
        tg::record_error("tg_blksolve_dev_noalloc: bad arguments");
        return TG_EINVAL;
    }
    // Each resident thread needs B*B*k2 doubles; at least one thread block
    // must fit in the fixed scratch.
    const int threads = kTileColumns;
    const long per_thread = (long)B * B * k2;
    const long max_slots = kScratchDoubles / per_thread;
    if (max_slots < threads) {
        char msg[256];
        snprintf(msg, sizeof msg,
                 "tg_blksolve_dev_noalloc: B*B*k2 = %ld doubles per column exceeds the fixed scratch "
                 "(%ld doubles for %d threads: k2 <= %ld for B = %d)",
                 per_thread, kScratchDoubles, threads, kScratchDoubles / ((long)B * B * threads), B);
        tg::record_error(msg);
        return TG_EINVAL;
    }
    DevPtrs p;
    int rc = device_ptrs(&p);
    if (rc) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    cudaError_t e = cudaMemsetAsync(p.flags, 0, sizeof(unsigned), st);
    if (e == cudaSuccess && ncol > 0) {
        tg::Seg seg{};
        seg.a = P;
        seg.b = Q;
        seg.c = R;
        seg.f = f;
        seg.x = u;
        seg.ubc_ratio = ubc_ratio;
        seg.ubc_add = ubc_ratio ? ubc_add : nullptr;
        seg.ld = ld;
        seg.nk = nk;
        seg.k2 = k2;
        seg.ncol = ncol;
        seg.kind = B;
        tg::SegTable tab{};
        tab.segs = nullptr;
        tab.nseg = 1;
        tab.ntiles = (ncol + threads - 1) / threads;
        tab.k2max = k2;
        tab.one = seg;
        tg::Shape sh{};
        e = tg::plan_shape(B, TG_PREC_F64, k2, tab.ntiles, threads, 1, 0, 0, &sh);
        if (e == cudaSuccess) {
            const long cap_blocks = max_slots / threads;
            if (sh.blocks > cap_blocks) sh.blocks = (int)cap_blocks;
            e = tg::launch_block(tab, B, TG_PREC_F64, sh, tg::Refine{1, 0.5}, p.scratch, p.flags, nullptr, st);
        }
    }
    if (e == cudaSuccess && status_dev) {
        k_noalloc_status<<<1, 1, 0, st>>>(p.flags, status_dev);
        e = cudaGetLastError();
    }
    if (e != cudaSuccess) {
        char msg[256];
        snprintf(msg, sizeof msg, "tg_blksolve_dev_noalloc: %s", cudaGetErrorString(e));
        tg::record_error(msg);
        return TG_ECUDA;
    }
    return TG_OK;
}
