// C ABI of the column solvers (include/tg_colsolve.h).
//
// Host-pointer drop-ins copy the reference's Fortran-layout arrays to the
// device in column chunks on two streams (host->device copy of chunk j+1
// overlaps the relayout + solve + device->host copy of chunk j), relayout
// them to the level-major layout the kernels want, solve, and copy back only
// the rows the reference writes.  Device-pointer entries and plans run on the
// caller's stream.
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <atomic>
#include <mutex>
#include <string>
#include <new>
#include <vector>

#include "tg_internal.h"

using namespace tg;

namespace {

thread_local char g_err[512] = "";

void set_err(const char *fmt, ...)
{
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof g_err, fmt, ap);
    va_end(ap);
}

#define TG_CUDA(call)                                                                             \
    do {                                                                                          \
        cudaError_t e_ = (call);                                                                  \
        if (e_ != cudaSuccess) {                                                                  \
            set_err("%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, __LINE__); \
            return TG_ECUDA;                                                                      \
        }                                                                                         \
    } while (0)

Refine g_refine = {3, 1e-11};
int g_host_precision = TG_PREC_F64;

struct Buf {
    void *p = nullptr;
    size_t n = 0;
};

// Per-device work buffers and streams, created on first use.  The host
// drop-ins pipeline column chunks over up to kSlots streams (g_host_slots in
// use, 4 by default: on the nested workload's 4392 systems 3 took 532 ms and
// 4, 6 or 8 took 514 ms), each with its own buffers.
constexpr int kSlots = 8;
constexpr int kHostSlotsDefault = 4;
std::atomic<int> g_host_slots{kHostSlotsDefault};
std::atomic<long> g_host_chunk_bytes{0};   // 0: chosen per call
// Device workspace of the stream-ordered (_dev) entries, one per caller
// stream: entries issued on different streams may run at the same time, so
// each stream's work gets its own scratch, relayout buffers, status word and
// sweep histogram.  Work on one stream is ordered, so it can share them.
struct StreamWs {
    cudaStream_t key = nullptr;
    bool used = false;
    unsigned long long tick = 0;   // last use, for eviction
    Buf lvl[7];                    // level-major relayout of column-layout solves
    Buf scratch;                   // kernel scratch (Gamma, planes, w2)
    unsigned *flags = nullptr;     // device status word
    unsigned long long *hist = nullptr;   // device, kMaxSweepBins
};
constexpr int kStreamWs = 16;

struct DevCtx {
    int dev = -1;
    std::mutex mu;
    cudaStream_t st[kSlots] = {};
    Buf colbuf[kSlots][5];   // Fortran-layout staging: 4 inputs + output, per slot
    Buf lvlbuf[kSlots][7];   // level-major arrays: a,b,c,f,x,ubc_ratio,ubc_add, per slot
    Buf scratch[kSlots];     // block-kernel scratch, per slot
    Buf span[kSlots];        // one host region's inputs copied at once (coalesced runs), per slot
    unsigned *flags = nullptr;           // device, one word per slot
    unsigned *flags_host = nullptr;      // pinned, one word per slot
    unsigned long long *hist = nullptr;  // device, kMaxSweepBins
    StreamWs ws[kStreamWs];              // per caller stream, see StreamWs
    unsigned long long ws_tick = 0;
};

constexpr int kMaxDev = 64;
DevCtx *g_ctx[kMaxDev] = {};
std::mutex g_ctx_mu;

int get_ctx(DevCtx **out)
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) {
        int n = 0;
        if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
            set_err("no CUDA device available");
            return TG_ENODEV;
        }
        set_err("cudaGetDevice failed: %s", cudaGetErrorString(e));
        return TG_ECUDA;
    }
    if (dev < 0 || dev >= kMaxDev) {
        set_err("device index %d out of range", dev);
        return TG_ENODEV;
    }
    std::lock_guard<std::mutex> lk(g_ctx_mu);
    if (!g_ctx[dev]) {
        DevCtx *c = new (std::nothrow) DevCtx;
        if (!c) return TG_ENOMEM;
        c->dev = dev;
        for (int i = 0; i < kSlots; ++i) TG_CUDA(cudaStreamCreateWithFlags(&c->st[i], cudaStreamNonBlocking));
        TG_CUDA(cudaMalloc(&c->flags, kSlots * sizeof(unsigned)));
        TG_CUDA(cudaMallocHost(&c->flags_host, kSlots * sizeof(unsigned)));
        TG_CUDA(cudaMalloc(&c->hist, kMaxSweepBins * sizeof(unsigned long long)));
        g_ctx[dev] = c;
    }
    *out = g_ctx[dev];
    return TG_OK;
}

// Grows a device buffer; the device is synchronised before an old buffer is
// freed, since queued work may still use it.
int grow(Buf &b, size_t bytes)
{
    if (bytes <= b.n) return TG_OK;
    if (b.p) {
        TG_CUDA(cudaDeviceSynchronize());
        TG_CUDA(cudaFree(b.p));
        b.p = nullptr;
        b.n = 0;
    }
    bytes = (bytes + 4095) & ~(size_t)4095;
    cudaError_t e = cudaMalloc(&b.p, bytes);
    if (e != cudaSuccess) {
        cudaGetLastError();
        set_err("cudaMalloc(%zu) failed: %s", bytes, cudaGetErrorString(e));
        return TG_ENOMEM;
    }
    b.n = bytes;
    return TG_OK;
}

// The workspace of caller stream st (the caller holds c->mu).  A stream
// seen for the first time takes a free entry; with all kStreamWs taken, the
// least recently used one is drained (device synchronised) and reassigned.
int stream_ws(DevCtx *c, cudaStream_t st, StreamWs **out)
{
    StreamWs *hit = nullptr, *free_ws = nullptr, *lru = nullptr;
    for (StreamWs &w : c->ws) {
        if (w.used && w.key == st) {
            hit = &w;
            break;
        }
        if (!w.used && !free_ws) free_ws = &w;
        if (w.used && (!lru || w.tick < lru->tick)) lru = &w;
    }
    if (!hit) {
        hit = free_ws;
        if (!hit) {
            // another stream's queued work may still use these buffers
            TG_CUDA(cudaDeviceSynchronize());
            hit = lru;
            for (Buf &b : hit->lvl)
                if (b.p) {
                    TG_CUDA(cudaFree(b.p));
                    b = Buf{};
                }
            if (hit->scratch.p) {
                TG_CUDA(cudaFree(hit->scratch.p));
                hit->scratch = Buf{};
            }
        }
        if (!hit->flags) TG_CUDA(cudaMalloc(&hit->flags, sizeof(unsigned)));
        if (!hit->hist) TG_CUDA(cudaMalloc(&hit->hist, kMaxSweepBins * sizeof(unsigned long long)));
        hit->key = st;
        hit->used = true;
    }
    hit->tick = ++c->ws_tick;
    *out = hit;
    return TG_OK;
}

int flags_to_status(unsigned f)
{
    if (f & FLAG_TIMEOUT) return TG_ETIMEOUT;
    if (f & FLAG_PIVOT) return TG_EPIVOT;
    if (f & FLAG_NONFINITE) return TG_ENONFINITE;
    if (f & FLAG_NOCONV) return TG_ENOCONV;
    return TG_OK;
}

__global__ void k_finish_status(const unsigned *flags, int *out)
{
    const unsigned f = *flags;
    *out = (f & FLAG_TIMEOUT) ? TG_ETIMEOUT : (f & FLAG_PIVOT) ? TG_EPIVOT : (f & FLAG_NONFINITE) ? TG_ENONFINITE : (f & FLAG_NOCONV) ? TG_ENOCONV : TG_OK;
}

long round_up(long v, long m) { return (v + m - 1) / m * m; }

bool aligned16(const void *p) { return ((uintptr_t)p & 15u) == 0; }

// One level-major solve of a single segment on stream st.
bool ring_ok_seg(const Seg &s)
{
    return s.ld % 32 == 0 && aligned16(s.a) && aligned16(s.b) && aligned16(s.c) && aligned16(s.f);
}
// The refinement ring also reads x rows by bulk copies.
bool ring_ok_for(const Seg &s, int precision)
{
    return ring_ok_seg(s) && (precision == TG_PREC_F64 || aligned16(s.x));
}
bool cpt2_ok_seg(const Seg &s)
{
    return s.ld % 2 == 0 && aligned16(s.a) && aligned16(s.b) && aligned16(s.c) && aligned16(s.f) && aligned16(s.x);
}

int solve_level(Buf &scratch, unsigned long long *hist, int kind, int precision, Seg seg, unsigned *flags,
                cudaStream_t st)
{
    const int B = kind == TG_KIND_SCALAR ? 1 : kind;
    int cpb = 0, cpt = 1, stages = 0, w2g = 0;
    tile_for(kind, precision, ring_ok_for(seg, precision), &cpb, &cpt, &stages, &w2g);
    if (cpt == 2 && !cpt2_ok_seg(seg)) {
        cpb /= 2;
        cpt = 1;
    }
    SegTable tab{};
    tab.segs = nullptr;
    tab.nseg = 1;
    tab.ntiles = (int)((seg.ncol + cpb - 1) / cpb);
    tab.k2max = seg.k2;
    seg.tile0 = 0;
    seg.status_idx = 0;
    tab.one = seg;
    Shape sh{};
    cudaError_t e = plan_shape(kind, precision, seg.k2, tab.ntiles, cpb, cpt, stages, w2g, &sh);
    if (e != cudaSuccess) {
        set_err("no launch shape for kind %d k2 %d: %s", kind, seg.k2, cudaGetErrorString(e));
        return TG_EINVAL;
    }
    if (kind == TG_KIND_SCALAR) {
        double *scr = nullptr;
        const bool ring_refine = precision != TG_PREC_F64 && sh.stages > 0;
        if (sh.w2g || ring_refine) {
            const long slots = (long)sh.blocks * sh.threads;
            int rc = grow(scratch, ring_refine ? refine_scratch_bytes(slots, seg.k2) : scalar_scratch_bytes(slots, seg.k2));
            if (rc) return rc;
            scr = (double *)scratch.p;
        }
        TG_CUDA(launch_scalar(tab, precision, sh, g_refine, scr, flags, hist, st));
    } else {
        const size_t need = block_scratch_bytes(B, precision, (long)sh.blocks * sh.threads, seg.k2);
        int rc = grow(scratch, need);
        if (rc) return rc;
        TG_CUDA(launch_block(tab, B, precision, sh, g_refine, (double *)scratch.p, flags, hist, st));
    }
    return TG_OK;
}

// Host arrays in Fortran layout -> solve -> host x, for a list of systems.
//   B = 1 (scalar) or 2/3 (block); m[3], v (vectors) point at row 0 of the
//   solve in column 0; colstride = elements between columns of a vector
//   array (matrices: B*colstride); k2 rows are solved; ubc arrays (B, ncol).
// Every system is cut into column chunks of about 4 MB of input, and all
// chunks of all systems are pipelined over kSlots streams: while a chunk is
// relaid, solved and copied back on its stream, the next chunks' host->device
// copies are already queued on the others.  One synchronisation at the end.
struct HostSys {
    int kind;
    const double *m[3];
    const double *v;
    double *x;
    long colstride;
    int k2;
    long ncol;
    const double *ubc_ratio, *ubc_add;
};

struct HostPlan {
    int B;
    long mrows, vrows, orows, mstride, chunk;
};

// Input bytes of one system in the host (Fortran) layout.
long host_bytes(const HostSys &h)
{
    const long B = h.kind == TG_KIND_SCALAR ? 1 : h.kind;
    return (3 * B * B + B) * (long)h.k2 * h.ncol * 8;
}

// Column chunk size of a call: every chunk costs a fixed few tens of
// microseconds (copies, relayouts, a solve launch whose columns are too few
// to fill the GPU), so large calls use large chunks; about six chunks per
// call keep the copy-in of the next chunk overlapping the solve of this one.
// Whether [lo, hi) lies in one page-locked host allocation (the driver's
// range attributes of the allocation holding lo); a copy of that region then
// reads only the caller's registered memory.  False when the query is not
// available or says otherwise.
bool pinned_region(const char *lo, const char *hi)
{
    typedef CUresult (*GetAttr)(void *, CUpointer_attribute, CUdeviceptr);
    static GetAttr get_attr = [] {
        void *fn = nullptr;
        cudaDriverEntryPointQueryResult q;
        GetAttr g = nullptr;
        if (cudaGetDriverEntryPointByVersion("cuPointerGetAttribute", &fn, 12000, cudaEnableDefault, &q) ==
                cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            g = (GetAttr)fn;
        cudaGetLastError();
        return g;
    }();
    if (!get_attr || hi <= lo) return false;
    unsigned int type = 0;
    CUdeviceptr start = 0;
    size_t size = 0;
    const CUdeviceptr p = (CUdeviceptr)(uintptr_t)lo;
    if (get_attr(&type, CU_POINTER_ATTRIBUTE_MEMORY_TYPE, p) != CUDA_SUCCESS || type != CU_MEMORYTYPE_HOST) return false;
    if (get_attr(&start, CU_POINTER_ATTRIBUTE_RANGE_START_ADDR, p) != CUDA_SUCCESS ||
        get_attr(&size, CU_POINTER_ATTRIBUTE_RANGE_SIZE, p) != CUDA_SUCCESS)
        return false;
    return (uintptr_t)lo >= (uintptr_t)start && (uintptr_t)hi <= (uintptr_t)start + size;
}

long host_chunk_bytes(const HostSys *sys, int nsys)
{
    const long set = g_host_chunk_bytes.load();
    if (set > 0) return set;
    long total = 0;
    for (int i = 0; i < nsys; ++i) total += host_bytes(sys[i]);
    return std::max(4l << 20, std::min(64l << 20, total / 6));
}

HostPlan host_plan(const HostSys &h, long chunk_bytes)
{
    HostPlan p;
    p.B = h.kind == TG_KIND_SCALAR ? 1 : h.kind;
    p.mrows = (long)p.B * p.B * h.k2;
    p.vrows = (long)p.B * h.k2;
    p.orows = (long)p.B * (h.k2 + (h.ubc_ratio ? 1 : 0));
    p.mstride = (long)p.B * h.colstride;
    const long in_per_col = (3 * p.mrows + p.vrows) * 8;
    long nchunks = (in_per_col * h.ncol + chunk_bytes - 1) / chunk_bytes;
    nchunks = std::max<long>(1, std::min<long>(nchunks, 64));
    p.chunk = round_up((h.ncol + nchunks - 1) / nchunks, 32);
    return p;
}

int host_solve_many(const HostSys *sys, int nsys, int precision)
{
    DevCtx *c = nullptr;
    int rc = get_ctx(&c);
    if (rc) return rc;
    std::lock_guard<std::mutex> lk(c->mu);
    TG_CUDA(cudaSetDevice(c->dev));
    std::vector<HostPlan> plans(nsys);
    long need_m = 0, need_v = 0, need_o = 0, need_u = 0, total_chunks = 0;
    const long chunk_bytes = host_chunk_bytes(sys, nsys);
    for (int i = 0; i < nsys; ++i) {
        plans[i] = host_plan(sys[i], chunk_bytes);
        const HostPlan &p = plans[i];
        need_m = std::max(need_m, p.mrows * p.chunk);
        need_v = std::max(need_v, p.vrows * p.chunk);
        need_o = std::max(need_o, std::max<long>(p.orows, 2l * p.B) * p.chunk);
        if (sys[i].ubc_ratio) need_u = std::max(need_u, (long)p.B * p.chunk);
        total_chunks += (sys[i].ncol + p.chunk - 1) / p.chunk;
    }
    if (total_chunks == 0) return TG_OK;
    const int nslots = (int)std::min<long>(g_host_slots.load(), total_chunks);
    for (int s = 0; s < nslots; ++s) {
        for (int i = 0; i < 3; ++i)
            if ((rc = grow(c->colbuf[s][i], sizeof(double) * need_m))) return rc;
        if ((rc = grow(c->colbuf[s][3], sizeof(double) * need_v))) return rc;
        if ((rc = grow(c->colbuf[s][4], sizeof(double) * need_o))) return rc;
        for (int i = 0; i < 3; ++i)
            if ((rc = grow(c->lvlbuf[s][i], sizeof(double) * need_m))) return rc;
        if ((rc = grow(c->lvlbuf[s][3], sizeof(double) * need_v))) return rc;
        if ((rc = grow(c->lvlbuf[s][4], sizeof(double) * need_o))) return rc;
        if (need_u) {
            if ((rc = grow(c->lvlbuf[s][5], sizeof(double) * need_u))) return rc;
            if ((rc = grow(c->lvlbuf[s][6], sizeof(double) * need_u))) return rc;
        }
        TG_CUDA(cudaMemsetAsync(c->flags + s, 0, sizeof(unsigned), c->st[s]));
    }
    // The chunks in issue order, each with the host ranges of its inputs.
    // Consecutive chunks whose inputs lie in one page-locked region (a caller
    // that keeps its systems' arrays side by side, as in one registered
    // arena) form a run: a device buffer mirrors the region, and the inputs
    // cross the link in few large copies instead of one per array (~1 MB
    // copies move ~20% fewer bytes per second on this part).  Only the
    // inputs are copied: ranges that touch merge into one copy, and equal
    // ranges at a fixed pitch (systems of one shape, each followed by its
    // solution array) into one strided copy.
    struct Piece {
        const char *lo, *hi;
    };
    struct ChunkRef {
        int si;
        long c0, nc;
        const char *lo, *hi;   // region of the chunk's inputs (flat: each a single range)
        bool flat;
        int npc;
        Piece pc[6];
    };
    std::vector<ChunkRef> chunks;
    chunks.reserve(total_chunks);
    for (int si = 0; si < nsys; ++si) {
        const HostSys &h = sys[si];
        const HostPlan &p = plans[si];
        for (long c0 = 0; c0 < h.ncol; c0 += p.chunk) {
            const long nc = std::min(p.chunk, h.ncol - c0);
            ChunkRef ch{si, c0, nc, nullptr, nullptr, true, 0, {}};
            auto add = [&](const double *base, long rows, long stride) {
                if (rows != stride) {
                    ch.flat = false;
                    return;
                }
                const char *a = (const char *)(base + c0 * stride), *b = a + sizeof(double) * rows * nc;
                ch.lo = ch.lo && ch.lo < a ? ch.lo : a;
                ch.hi = ch.hi && ch.hi > b ? ch.hi : b;
                ch.pc[ch.npc++] = Piece{a, b};
            };
            for (int i = 0; i < 3; ++i) add(h.m[i], p.mrows, p.mstride);
            add(h.v, p.vrows, h.colstride);
            if (h.ubc_ratio) add(h.ubc_ratio, p.B, p.B);
            if (h.ubc_ratio && h.ubc_add) add(h.ubc_add, p.B, p.B);
            chunks.push_back(ch);
        }
    }
    struct Run {
        size_t j0, j1;
        const char *lo;
        long bytes;   // the region the device buffer mirrors (0: per-array copies)
    };
    std::vector<Run> runs;
    long max_span = 0;
    const long run_cap = std::max(chunk_bytes, 8l << 20);
    for (size_t j = 0; j < chunks.size();) {
        Run r{j, j + 1, chunks[j].lo, 0};
        if (chunks[j].flat) {
            const char *lo = chunks[j].lo, *hi = chunks[j].hi;
            while (r.j1 < chunks.size() && chunks[r.j1].flat) {
                const ChunkRef &n = chunks[r.j1];
                const char *l2 = std::min(lo, n.lo), *h2 = std::max(hi, n.hi);
                if (h2 - l2 > run_cap) break;
                lo = l2;
                hi = h2;
                ++r.j1;
            }
            if (hi - lo <= run_cap && pinned_region(lo, hi)) {
                r.lo = lo;
                r.bytes = hi - lo;
                max_span = std::max(max_span, r.bytes);
            }
        }
        runs.push_back(r);
        j = r.j1;
    }
    // The copies of a run's inputs: the pieces in address order, merged where
    // they touch (gaps of alignment padding included), then equal pieces at
    // one pitch grouped into a strided copy.
    std::vector<Piece> pieces;
    auto copy_run = [&](const Run &run, char *dspan, cudaStream_t st) -> cudaError_t {
        pieces.clear();
        for (size_t jj = run.j0; jj < run.j1; ++jj)
            for (int i = 0; i < chunks[jj].npc; ++i) pieces.push_back(chunks[jj].pc[i]);
        std::sort(pieces.begin(), pieces.end(), [](const Piece &a, const Piece &b) { return a.lo < b.lo; });
        size_t n = 0;
        for (const Piece &q : pieces) {
            if (n > 0 && q.lo <= pieces[n - 1].hi + 4096) {
                pieces[n - 1].hi = std::max(pieces[n - 1].hi, q.hi);
            } else {
                pieces[n++] = q;
            }
        }
        for (size_t i = 0; i < n;) {
            const long w = pieces[i].hi - pieces[i].lo;
            size_t e = i + 1;
            const long pitch = e < n ? pieces[e].lo - pieces[i].lo : 0;
            while (e < n && pieces[e].hi - pieces[e].lo == w && pieces[e].lo - pieces[e - 1].lo == pitch) ++e;
            char *d = dspan + (pieces[i].lo - run.lo);
            cudaError_t err = e - i > 1 ? cudaMemcpy2DAsync(d, pitch, pieces[i].lo, pitch, w, e - i,
                                                            cudaMemcpyHostToDevice, st)
                                        : cudaMemcpyAsync(d, pieces[i].lo, w, cudaMemcpyHostToDevice, st);
            if (err != cudaSuccess) return err;
            i = e;
        }
        return cudaSuccess;
    };
    if (max_span > 0)
        for (int s = 0; s < nslots; ++s)
            if ((rc = grow(c->span[s], (size_t)max_span))) return rc;
    for (size_t ri = 0; ri < runs.size(); ++ri) {
        const Run &run = runs[ri];
        const int s = (int)(ri % nslots);
        cudaStream_t st = c->st[s];
        const char *dspan = (const char *)c->span[s].p;
        if (run.bytes > 0) TG_CUDA(copy_run(run, (char *)c->span[s].p, st));
        // where a run's host array landed on the device
        auto in_span = [&](const double *host) { return (const double *)(dspan + ((const char *)host - run.lo)); };
        for (size_t jj = run.j0; jj < run.j1; ++jj) {
            const ChunkRef &ch = chunks[jj];
            const HostSys &h = sys[ch.si];
            const HostPlan &p = plans[ch.si];
            const int B = p.B;
            const long ld = p.chunk, c0 = ch.c0, nc = ch.nc;
            double *lv[7];
            for (int i = 0; i < 7; ++i) lv[i] = (double *)c->lvlbuf[s][i].p;
            Relayout r{};
            r.out_ld = ld;
            r.ncols = nc;
            r.n = 4;
            for (int i = 0; i < 4; ++i) {
                const double *src = i < 3 ? h.m[i] : h.v;
                const long rows = i < 3 ? p.mrows : p.vrows, stride = i < 3 ? p.mstride : h.colstride;
                if (run.bytes > 0) {
                    r.in[i] = in_span(src + c0 * stride);
                } else {
                    double *cb = (double *)c->colbuf[s][i].p;
                    if (rows == stride)
                        TG_CUDA(cudaMemcpyAsync(cb, src + c0 * stride, sizeof(double) * rows * nc,
                                                cudaMemcpyHostToDevice, st));
                    else
                        TG_CUDA(cudaMemcpy2DAsync(cb, sizeof(double) * rows, src + c0 * stride,
                                                  sizeof(double) * stride, sizeof(double) * rows, nc,
                                                  cudaMemcpyHostToDevice, st));
                    r.in[i] = cb;
                }
                r.out[i] = lv[i];
                r.in_ld[i] = rows;
                r.nrows[i] = rows;
            }
            TG_CUDA(launch_col_to_level_multi(r, st));
            if (h.ubc_ratio) {
                double *cb = (double *)c->colbuf[s][4].p;
                Relayout u{};
                u.out_ld = ld;
                u.ncols = nc;
                u.n = h.ubc_add ? 2 : 1;
                if (run.bytes > 0) {
                    u.in[0] = in_span(h.ubc_ratio + c0 * B);
                } else {
                    TG_CUDA(cudaMemcpyAsync(cb, h.ubc_ratio + c0 * B, sizeof(double) * B * nc,
                                            cudaMemcpyHostToDevice, st));
                    u.in[0] = cb;
                }
                u.out[0] = lv[5];
                u.in_ld[0] = B;
                u.nrows[0] = B;
                if (h.ubc_add) {
                    if (run.bytes > 0) {
                        u.in[1] = in_span(h.ubc_add + c0 * B);
                    } else {
                        TG_CUDA(cudaMemcpyAsync(cb + B * p.chunk, h.ubc_add + c0 * B, sizeof(double) * B * nc,
                                                cudaMemcpyHostToDevice, st));
                        u.in[1] = cb + B * p.chunk;
                    }
                    u.out[1] = lv[6];
                    u.in_ld[1] = B;
                    u.nrows[1] = B;
                }
                TG_CUDA(launch_col_to_level_multi(u, st));
            }
            Seg seg{};
            seg.a = lv[0];
            seg.b = lv[1];
            seg.c = lv[2];
            seg.f = lv[3];
            seg.x = lv[4];
            seg.ubc_ratio = h.ubc_ratio ? lv[5] : nullptr;
            seg.ubc_add = (h.ubc_ratio && h.ubc_add) ? lv[6] : nullptr;
            seg.ld = ld;
            seg.nk = h.k2 + (h.ubc_ratio ? 1 : 0);
            seg.k2 = h.k2;
            seg.ncol = (int)nc;
            seg.kind = h.kind;
            if ((rc = solve_level(c->scratch[s], c->hist, h.kind, precision, seg, c->flags + s, st))) return rc;
            double *ob = (double *)c->colbuf[s][4].p;
            TG_CUDA(launch_level_to_col(lv[4], ld, ob, p.orows, p.orows, nc, st));
            if (p.orows == h.colstride)
                TG_CUDA(cudaMemcpyAsync(h.x + c0 * h.colstride, ob, sizeof(double) * p.orows * nc,
                                        cudaMemcpyDeviceToHost, st));
            else
                TG_CUDA(cudaMemcpy2DAsync(h.x + c0 * h.colstride, sizeof(double) * h.colstride, ob,
                                          sizeof(double) * p.orows, sizeof(double) * p.orows, nc,
                                          cudaMemcpyDeviceToHost, st));
        }
    }
    for (int s = 0; s < nslots; ++s) TG_CUDA(cudaStreamSynchronize(c->st[s]));
    TG_CUDA(cudaMemcpy(c->flags_host, c->flags, nslots * sizeof(unsigned), cudaMemcpyDeviceToHost));
    unsigned all = 0;
    for (int s = 0; s < nslots; ++s) all |= c->flags_host[s];
    return flags_to_status(all);
}

int host_solve(int kind, const double *const m[3], const double *v, double *x, long colstride, int k2,
               long ncol, const double *ubc_ratio, const double *ubc_add, int precision)
{
    HostSys h{kind, {m[0], m[1], m[2]}, v, x, colstride, k2, ncol, ubc_ratio, ubc_add};
    return host_solve_many(&h, 1, precision);
}

bool bad_prec(int p) { return p != TG_PREC_F64 && p != TG_PREC_F32_REFINE; }

}  // namespace

void tg::record_error(const char *msg) { set_err("%s", msg); }

// ===========================================================================
// Public entry points
// ===========================================================================
extern "C" {

__attribute__((visibility("default"))) const char *tg_version(void) { return "tg_colsolve 0.1.0 sm_100a"; }

__attribute__((visibility("default"))) int tg_kernel_arch(int *arch)
{
    if (!arch) {
        set_err("tg_kernel_arch: null argument");
        return TG_EINVAL;
    }
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
        cudaGetLastError();
        set_err("no CUDA device available");
        return TG_ENODEV;
    }
    TG_CUDA(kernel_binary_version(arch));
    return TG_OK;
}

__attribute__((visibility("default"))) const char *tg_last_error(void) { return g_err; }

__attribute__((visibility("default"))) int tg_set_refine(int max_sweeps, double rel_tol)
{
    if (max_sweeps < 1 || max_sweeps > kMaxSweepBins - 2 || !(rel_tol > 0.0) || !(rel_tol < 1.0)) {
        set_err("tg_set_refine: max_sweeps must be 1..%d and 0 < rel_tol < 1", kMaxSweepBins - 2);
        return TG_EINVAL;
    }
    g_refine.max_sweeps = max_sweeps;
    g_refine.rel_tol = rel_tol;
    return TG_OK;
}

__attribute__((visibility("default"))) int tg_set_pipeline(int kind, int precision, int stages, int warps)
{
    if ((kind != TG_KIND_SCALAR && kind != TG_KIND_BLOCK2 && kind != TG_KIND_BLOCK3) || bad_prec(precision) ||
        (stages != -1 && stages != 0 && stages != 2 && stages != 3 && stages != 4 && stages != 8 && stages != 16) ||
        (stages > 0 && precision != TG_PREC_F64 &&
         !(kind == TG_KIND_SCALAR && stages <= 4) && !(kind == TG_KIND_BLOCK2 && (stages == 4 || stages == 8))) ||
        warps < 0 || warps > 8) {
        set_err("tg_set_pipeline: stages must be 0, 2, 3, 4, 8 or 16 (FP64; refinement: scalar 2..4, 2x2 4 or 8) or -1; "
                "warps 0..8");
        return TG_EINVAL;
    }
    set_stages(kind, precision, stages, warps);
    return TG_OK;
}

__attribute__((visibility("default"))) int tg_set_prefetch(int kind, int precision, int levels)
{
    if (kind != TG_KIND_SCALAR || bad_prec(precision) || (levels != -1 && levels != 4 && levels != 8 && levels != 16)) {
        set_err("tg_set_prefetch: scalar kind only, levels 4, 8, 16 or -1");
        return TG_EINVAL;
    }
    set_prefetch(kind, precision, levels);
    return TG_OK;
}

__attribute__((visibility("default"))) int tg_set_scratch_global(int kind, int precision, int on)
{
    if (kind != TG_KIND_SCALAR || precision != TG_PREC_F64 || on < -1 || on > 1) {
        set_err("tg_set_scratch_global: only the scalar FP64 kernel, on = 0, 1 or -1");
        return TG_EINVAL;
    }
    set_w2g(kind, precision, on);
    return TG_OK;
}

__attribute__((visibility("default"))) int tg_selftest_division(const double *a, const double *b, double *q,
                                                                long n, void *stream)
{
    if (!a || !b || !q || n < 0) {
        set_err("tg_selftest_division: bad arguments");
        return TG_EINVAL;
    }
    TG_CUDA(launch_selftest_division(a, b, q, n, (cudaStream_t)stream));
    return TG_OK;
}

__attribute__((visibility("default"))) int tg_set_host_precision(int precision)
{
    if (bad_prec(precision)) {
        set_err("tg_set_host_precision: unknown precision %d", precision);
        return TG_EINVAL;
    }
    g_host_precision = precision;
    return TG_OK;
}

__attribute__((visibility("default"))) int tg_set_tile(int kind, int precision, int cols_per_block_,
                                                       int cols_per_thread_)
{
    if ((kind != TG_KIND_SCALAR && kind != TG_KIND_BLOCK2 && kind != TG_KIND_BLOCK3) || bad_prec(precision)) {
        set_err("tg_set_tile: bad kind or precision");
        return TG_EINVAL;
    }
    if (cols_per_block_ != 0 || cols_per_thread_ != 0) {
        const int cpt = cols_per_thread_ ? cols_per_thread_ : 1;
        const int maxthr = kind == TG_KIND_SCALAR ? 256 : 128;
        if ((cpt != 1 && cpt != 2) || (cpt == 2 && (kind != TG_KIND_SCALAR || precision != TG_PREC_F64)) ||
            cols_per_block_ < 32 || cols_per_block_ > 512 || cols_per_block_ % 32 ||
            cols_per_block_ / cpt > maxthr || (cols_per_block_ / cpt) % 32) {
            set_err("tg_set_tile: unsupported shape cpb=%d cpt=%d", cols_per_block_, cols_per_thread_);
            return TG_EINVAL;
        }
    }
    set_tile(kind, precision, cols_per_block_, cols_per_thread_);
    return TG_OK;
}

__attribute__((visibility("default"))) int tg_solve_host(const tg_host_system *sys, int nsys)
{
    if (nsys < 0 || (nsys > 0 && !sys)) {
        set_err("tg_solve_host: bad arguments");
        return TG_EINVAL;
    }
    std::vector<HostSys> hs;
    hs.reserve(nsys);
    for (int i = 0; i < nsys; ++i) {
        const tg_host_system &q = sys[i];
        const bool blk = q.kind == TG_KIND_BLOCK2 || q.kind == TG_KIND_BLOCK3;
        if ((q.kind != TG_KIND_SCALAR && !blk) || !q.a || !q.b || !q.c || !q.f || !q.x || q.nk < 1 || q.k2 < 1 ||
            q.k2 > q.nk || q.ncol < 0 || (blk && q.ubc_ratio && q.k2 >= q.nk)) {
            set_err("tg_solve_host: system %d invalid", i);
            return TG_EINVAL;
        }
        if (q.ncol == 0) continue;
        const int B = blk ? q.kind : 1;
        hs.push_back(HostSys{q.kind, {q.a, q.b, q.c}, q.f, q.x, (long)B * q.nk, q.k2, q.ncol,
                             blk ? q.ubc_ratio : nullptr, blk && q.ubc_ratio ? q.ubc_add : nullptr});
    }
    if (hs.empty()) return TG_OK;
    return host_solve_many(hs.data(), (int)hs.size(), g_host_precision);
}

__attribute__((visibility("default"))) int tg_trsolv_ng(const double *a, const double *b, const double *c,
                                                        const double *f, double *x, int nk, int k2, int ncol)
{
    if (!a || !b || !c || !f || !x || nk < 1 || k2 < 1 || k2 > nk || ncol < 0) {
        set_err("tg_trsolv_ng: bad arguments (nk=%d k2=%d ncol=%d)", nk, k2, ncol);
        return TG_EINVAL;
    }
    if (ncol == 0) return TG_OK;
    const double *m[3] = {a, b, c};
    return host_solve(TG_KIND_SCALAR, m, f, x, nk, k2, ncol, nullptr, nullptr, g_host_precision);
}

__attribute__((visibility("default"))) int tg_trsolv(const double *a, const double *b, const double *c,
                                                     const double *f, double *x, int lev0, int lev1, int k1,
                                                     int k2, int lon0, int lon1, int lonmax)
{
    const int nlev = lev1 - lev0 + 1;
    if (!a || !b || !c || !f || !x || nlev < 1 || k1 < lev0 || k2 > lev1 || k2 < k1 || lon1 < lon0) {
        set_err("tg_trsolv: bad arguments");
        return TG_EINVAL;
    }
    const int lonbeg = lon0 == 1 ? 3 : lon0;
    const int lonend = lon1 == lonmax ? lon1 - 2 : lon1;
    if (lonend < lonbeg) return TG_OK;
    const size_t off = (size_t)nlev * (lonbeg - lon0) + (k1 - lev0);
    const double *m[3] = {a + off, b + off, c + off};
    return host_solve(TG_KIND_SCALAR, m, f + off, x + off, nlev, k2 - k1 + 1, lonend - lonbeg + 1, nullptr,
                      nullptr, g_host_precision);
}

}  // extern "C"

// Deferred latitude slabs (tg_trsolv_defer, tg_trsolv_flush).  The global
// callers of trsolv assemble each latitude into work arrays they reuse for
// the next one, so a slab is copied when it is queued: rows k1..k2 of the
// solved columns of a, b, c, f go to page-locked staging, one region per
// array, slab after slab; each slab's columns are then nrows-long contiguous
// columns, and consecutive slabs of equal nrows form one (nrows, sum ncol)
// system.  The flush solves every run in one batched host call and copies the
// solutions to each slab's x.  One queue per process, guarded by a mutex.
namespace {
struct DeferSlab {
    double *x;        // row k1 of the first solved column of the caller's x
    long xstride;     // elements between the caller's columns (lev1-lev0+1)
    int nrows;        // k2-k1+1
    long ncol;
    size_t off;       // first element in each staging region
};
struct DeferQueue {
    std::mutex mu;
    std::vector<DeferSlab> slabs;
    double *in = nullptr;    // page-locked: regions a, b, c, f of cap elements each
    double *out = nullptr;   // page-locked: cap elements
    size_t cap = 0, used = 0;
};
DeferQueue g_defer;

int defer_reserve(DeferQueue &q, size_t need)
{
    if (need <= q.cap) return TG_OK;
    size_t cap = std::max(need, std::max(2 * q.cap, (size_t)1 << 20));
    double *in = nullptr, *out = nullptr;
    if (cudaHostAlloc((void **)&in, sizeof(double) * 4 * cap, cudaHostAllocPortable) != cudaSuccess ||
        cudaHostAlloc((void **)&out, sizeof(double) * cap, cudaHostAllocPortable) != cudaSuccess) {
        cudaGetLastError();
        if (in) cudaFreeHost(in);
        set_err("tg_trsolv_defer: page-locked staging of %zu MB not available", sizeof(double) * 5 * cap >> 20);
        return TG_ENOMEM;
    }
    for (int r = 0; r < 4 && q.used; ++r) memcpy(in + r * cap, q.in + r * q.cap, sizeof(double) * q.used);
    if (q.in) cudaFreeHost(q.in);
    if (q.out) cudaFreeHost(q.out);
    q.in = in;
    q.out = out;
    q.cap = cap;
    return TG_OK;
}
}  // namespace

extern "C" {

__attribute__((visibility("default"))) int tg_trsolv_defer(const double *a, const double *b, const double *c,
                                                           const double *f, double *x, int lev0, int lev1, int k1,
                                                           int k2, int lon0, int lon1, int lonmax)
{
    const int nlev = lev1 - lev0 + 1;
    if (!a || !b || !c || !f || !x || nlev < 1 || k1 < lev0 || k2 > lev1 || k2 < k1 || lon1 < lon0) {
        set_err("tg_trsolv_defer: bad arguments");
        return TG_EINVAL;
    }
    const int lonbeg = lon0 == 1 ? 3 : lon0;
    const int lonend = lon1 == lonmax ? lon1 - 2 : lon1;
    if (lonend < lonbeg) return TG_OK;
    const int nrows = k2 - k1 + 1;
    const long ncol = lonend - lonbeg + 1;
    const size_t off0 = (size_t)nlev * (lonbeg - lon0) + (k1 - lev0);
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) {
        cudaGetLastError();
        set_err("no CUDA device available");
        return TG_ENODEV;
    }
    std::lock_guard<std::mutex> lk(g_defer.mu);
    int rc = defer_reserve(g_defer, g_defer.used + (size_t)nrows * ncol);
    if (rc) return rc;
    const double *src[4] = {a, b, c, f};
    for (int r = 0; r < 4; ++r) {
        double *dst = g_defer.in + r * g_defer.cap + g_defer.used;
        for (long i = 0; i < ncol; ++i)
            memcpy(dst + i * nrows, src[r] + off0 + (size_t)nlev * i, sizeof(double) * nrows);
    }
    g_defer.slabs.push_back(DeferSlab{x + off0, nlev, nrows, ncol, g_defer.used});
    g_defer.used += (size_t)nrows * ncol;
    return TG_OK;
}

__attribute__((visibility("default"))) int tg_trsolv_flush(void)
{
    std::lock_guard<std::mutex> lk(g_defer.mu);
    DeferQueue &q = g_defer;
    if (q.slabs.empty()) return TG_OK;
    std::vector<HostSys> hs;
    for (size_t i = 0; i < q.slabs.size();) {
        size_t j = i;
        long ncol = 0;
        while (j < q.slabs.size() && q.slabs[j].nrows == q.slabs[i].nrows) ncol += q.slabs[j++].ncol;
        const size_t o = q.slabs[i].off;
        hs.push_back(HostSys{TG_KIND_SCALAR, {q.in + o, q.in + q.cap + o, q.in + 2 * q.cap + o}, q.in + 3 * q.cap + o,
                             q.out + o, (long)q.slabs[i].nrows, q.slabs[i].nrows, ncol, nullptr, nullptr});
        i = j;
    }
    const int rc = host_solve_many(hs.data(), (int)hs.size(), g_host_precision);
    const bool numeric = rc == TG_OK || rc == TG_EPIVOT || rc == TG_ENONFINITE || rc == TG_ENOCONV;
    if (numeric)
        for (const DeferSlab &d : q.slabs)
            for (long i = 0; i < d.ncol; ++i)
                memcpy(d.x + d.xstride * i, q.out + d.off + (size_t)d.nrows * i, sizeof(double) * d.nrows);
    q.slabs.clear();
    q.used = 0;
    return rc;
}

__attribute__((visibility("default"))) int tg_blktri(const double *a, const double *b, const double *c,
                                                     const double *f, double *x, int lev0, int lev1, int lon0,
                                                     int lon1, int nlonp4)
{
    const int nlev = lev1 - lev0 + 1;
    if (!a || !b || !c || !f || !x || nlev < 2 || lon1 < lon0) {
        set_err("tg_blktri: bad arguments");
        return TG_EINVAL;
    }
    const int lonbeg = lon0 == 1 ? 3 : lon0;
    const int lonend = lon1 == nlonp4 ? nlonp4 - 2 : lon1;
    if (lonend < lonbeg) return TG_OK;
    const size_t om = (size_t)4 * nlev * (lonbeg - lon0), ov = (size_t)2 * nlev * (lonbeg - lon0);
    const double *m[3] = {a + om, b + om, c + om};
    return host_solve(TG_KIND_BLOCK2, m, f + ov, x + ov, 2l * nlev, nlev - 1, lonend - lonbeg + 1, nullptr,
                      nullptr, g_host_precision);
}

__attribute__((visibility("default"))) int tg_blksolve(int B, const double *P, const double *Q,
                                                       const double *R, const double *f,
                                                       const double *ubc_ratio, const double *ubc_add, double *u,
                                                       int nk, int k2, int ncol)
{
    if ((B != 2 && B != 3) || !P || !Q || !R || !f || !u || nk < 1 || k2 < 1 || k2 > nk || ncol < 0 ||
        (ubc_ratio && k2 >= nk)) {
        set_err("tg_blksolve: bad arguments (B=%d nk=%d k2=%d ncol=%d)", B, nk, k2, ncol);
        return TG_EINVAL;
    }
    if (ncol == 0) return TG_OK;
    const double *m[3] = {P, Q, R};
    return host_solve(B, m, f, u, (long)B * nk, k2, ncol, ubc_ratio, ubc_add, g_host_precision);
}

__attribute__((visibility("default"))) int tg_comp_blksolve_ng(int B, const double *P, const double *Q,
                                                               const double *R, const double *f,
                                                               const double *ubc_ratio, const double *ubc_add,
                                                               double *u, int nk, int ncol)
{
    if (nk < 2) {
        set_err("tg_comp_blksolve_ng: nk must be >= 2");
        return TG_EINVAL;
    }
    return tg_blksolve(B, P, Q, R, f, ubc_ratio, ubc_add, u, nk, nk - 1, ncol);
}

static int dev_solve(int kind, const double *a, const double *b, const double *c, const double *f,
                     const double *ubc_ratio, const double *ubc_add, double *x, int nk, int k2, int ncol,
                     int layout, long ld, int precision, int *status_dev, void *stream)
{
    const int B = kind == TG_KIND_SCALAR ? 1 : kind;
    cudaStream_t st = (cudaStream_t)stream;
    if (!a || !b || !c || !f || !x || nk < 1 || k2 < 1 || k2 > nk || ncol < 0 || bad_prec(precision) ||
        (layout != TG_LAYOUT_COLUMN && layout != TG_LAYOUT_LEVEL) || (layout == TG_LAYOUT_LEVEL && ld < ncol) ||
        (ubc_ratio && k2 >= nk)) {
        set_err("device solve: bad arguments (nk=%d k2=%d ncol=%d layout=%d ld=%ld)", nk, k2, ncol, layout, ld);
        return TG_EINVAL;
    }
    DevCtx *cx = nullptr;
    int rc = get_ctx(&cx);
    if (rc) return rc;
    std::lock_guard<std::mutex> lk(cx->mu);
    StreamWs *ws = nullptr;
    if ((rc = stream_ws(cx, st, &ws))) return rc;
    unsigned *flags = ws->flags;
    TG_CUDA(cudaMemsetAsync(flags, 0, sizeof(unsigned), st));
    if (precision != TG_PREC_F64)
        TG_CUDA(cudaMemsetAsync(ws->hist, 0, kMaxSweepBins * sizeof(unsigned long long), st));
    if (ncol > 0) {
        Seg seg{};
        seg.nk = nk;
        seg.k2 = k2;
        seg.ncol = ncol;
        seg.kind = kind;
        const long orows = (long)B * (k2 + (ubc_ratio ? 1 : 0));
        if (layout == TG_LAYOUT_LEVEL) {
            seg.a = a; seg.b = b; seg.c = c; seg.f = f; seg.x = x;
            seg.ubc_ratio = ubc_ratio;
            seg.ubc_add = ubc_ratio ? ubc_add : nullptr;
            seg.ld = ld;
            if ((rc = solve_level(ws->scratch, ws->hist, kind, precision, seg, flags, st))) return rc;
        } else {
            const long mrows = (long)B * B * k2, vrows = (long)B * k2;
            const long lld = round_up(ncol, 32);
            for (int i = 0; i < 3; ++i)
                if ((rc = grow(ws->lvl[i], sizeof(double) * mrows * lld))) return rc;
            if ((rc = grow(ws->lvl[3], sizeof(double) * vrows * lld))) return rc;
            if ((rc = grow(ws->lvl[4], sizeof(double) * orows * lld))) return rc;
            if (ubc_ratio) {
                if ((rc = grow(ws->lvl[5], sizeof(double) * B * lld))) return rc;
                if ((rc = grow(ws->lvl[6], sizeof(double) * B * lld))) return rc;
            }
            double *lv[7];
            for (int i = 0; i < 7; ++i) lv[i] = (double *)ws->lvl[i].p;
            const double *src[3] = {a, b, c};
            for (int i = 0; i < 3; ++i) TG_CUDA(launch_col_to_level(src[i], (long)B * B * nk, lv[i], lld, mrows, ncol, st));
            TG_CUDA(launch_col_to_level(f, (long)B * nk, lv[3], lld, vrows, ncol, st));
            if (ubc_ratio) {
                TG_CUDA(launch_col_to_level(ubc_ratio, B, lv[5], lld, B, ncol, st));
                if (ubc_add) TG_CUDA(launch_col_to_level(ubc_add, B, lv[6], lld, B, ncol, st));
            }
            seg.a = lv[0]; seg.b = lv[1]; seg.c = lv[2]; seg.f = lv[3]; seg.x = lv[4];
            seg.ubc_ratio = ubc_ratio ? lv[5] : nullptr;
            seg.ubc_add = (ubc_ratio && ubc_add) ? lv[6] : nullptr;
            seg.ld = lld;
            seg.nk = k2 + (ubc_ratio ? 1 : 0);
            if ((rc = solve_level(ws->scratch, ws->hist, kind, precision, seg, flags, st))) return rc;
            TG_CUDA(launch_level_to_col(lv[4], lld, x, (long)B * nk, orows, ncol, st));
        }
    }
    if (status_dev) {
        k_finish_status<<<1, 1, 0, st>>>(flags, status_dev);
        TG_CUDA(cudaGetLastError());
    }
    return TG_OK;
}

__attribute__((visibility("default"))) int tg_dt_ng_dev(const tg_dt_fields *F, const tg_dt_consts *C,
                                                        double *tn_upd, int nk, int ncol, long ld, double *system_out,
                                                        int *status_dev, void *stream)
{
    if (!F || !C || !tn_upd || nk < 3 || ncol < 0 || ld < ncol) {
        set_err("tg_dt_ng_dev: bad arguments (nk=%d ncol=%d ld=%ld)", nk, ncol, ld);
        return TG_EINVAL;
    }
    const double *const ptrs[] = {F->tn, F->tnsmooth, F->horadv, F->un, F->vn, F->o1, F->mbar, F->xnmbar,
                                  F->scht, F->schti, F->cp, F->kt, F->km, F->hdt, F->qji_tn, F->cool_imp,
                                  F->cool_exp, F->w, F->qtotal, F->rkm12, F->tlbc, F->t_lbc, F->ulbc, F->vlbc,
                                  F->expz, F->dift};
    for (const double *p : ptrs)
        if (!p) {
            set_err("tg_dt_ng_dev: a field pointer is NULL");
            return TG_EINVAL;
        }
    DevCtx *cx = nullptr;
    int rc = get_ctx(&cx);
    if (rc) return rc;
    std::lock_guard<std::mutex> lk(cx->mu);
    cudaStream_t st = (cudaStream_t)stream;
    StreamWs *ws = nullptr;
    if ((rc = stream_ws(cx, st, &ws))) return rc;
    TG_CUDA(cudaMemsetAsync(ws->flags, 0, sizeof(unsigned), st));
    if ((rc = grow(ws->scratch, sizeof(double) * dt_scratch_planes() * (size_t)nk * (size_t)(ld > 0 ? ld : 1))))
        return rc;
    TG_CUDA(launch_dt_ng(*F, *C, tn_upd, nk, ncol, ld, system_out, ws->flags, st, nullptr, (double *)ws->scratch.p));
    if (status_dev) {
        k_finish_status<<<1, 1, 0, st>>>(ws->flags, status_dev);
        TG_CUDA(cudaGetLastError());
    }
    return TG_OK;
}

__attribute__((visibility("default"))) int tg_dt_ng(const tg_dt_fields *F, const tg_dt_consts *C, double *tn_upd,
                                                    int nk, int ncol)
{
    if (!F || !C || !tn_upd || nk < 3 || ncol < 0) {
        set_err("tg_dt_ng: bad arguments (nk=%d ncol=%d)", nk, ncol);
        return TG_EINVAL;
    }
    if (ncol == 0) return TG_OK;
    const double *const f3[20] = {F->tn, F->tnsmooth, F->horadv, F->un, F->vn, F->o1, F->mbar, F->xnmbar,
                                  F->scht, F->schti, F->cp, F->kt, F->km, F->hdt, F->qji_tn, F->cool_imp,
                                  F->cool_exp, F->w, F->qtotal, F->rkm12};
    const double *const f2[4] = {F->tlbc, F->t_lbc, F->ulbc, F->vlbc};
    for (const double *p : f3)
        if (!p) return set_err("tg_dt_ng: a field pointer is NULL"), TG_EINVAL;
    for (const double *p : f2)
        if (!p) return set_err("tg_dt_ng: a field pointer is NULL"), TG_EINVAL;
    if (!F->expz || !F->dift) return set_err("tg_dt_ng: expz/dift NULL"), TG_EINVAL;
    DevCtx *c = nullptr;
    int rc = get_ctx(&c);
    if (rc) return rc;
    std::lock_guard<std::mutex> lk(c->mu);
    TG_CUDA(cudaSetDevice(c->dev));
    const long ld = round_up(ncol, 32);
    const size_t lvl = (size_t)nk * ld, colsz = (size_t)nk * ncol;
    // one buffer: 20 level-major 3-D fields, the output, 4 2-D fields, expz, dift; one staging buffer
    if ((rc = grow(c->lvlbuf[0][0], sizeof(double) * (21 * lvl + 4 * (size_t)ld + 2 * (size_t)nk)))) return rc;
    if ((rc = grow(c->colbuf[0][0], sizeof(double) * colsz))) return rc;
    double *base = (double *)c->lvlbuf[0][0].p, *stage = (double *)c->colbuf[0][0].p;
    cudaStream_t st = c->st[0];
    tg_dt_fields D;
    const double **dst3[20] = {&D.tn, &D.tnsmooth, &D.horadv, &D.un, &D.vn, &D.o1, &D.mbar, &D.xnmbar, &D.scht,
                               &D.schti, &D.cp, &D.kt, &D.km, &D.hdt, &D.qji_tn, &D.cool_imp, &D.cool_exp, &D.w,
                               &D.qtotal, &D.rkm12};
    for (int i = 0; i < 20; ++i) {
        double *d = base + i * lvl;
        TG_CUDA(cudaMemcpyAsync(stage, f3[i], sizeof(double) * colsz, cudaMemcpyHostToDevice, st));
        TG_CUDA(launch_col_to_level(stage, nk, d, ld, nk, ncol, st));
        *dst3[i] = d;
    }
    double *out = base + 20 * lvl, *two = base + 21 * lvl, *one = two + 4 * ld;
    const double **dst2[4] = {&D.tlbc, &D.t_lbc, &D.ulbc, &D.vlbc};
    for (int i = 0; i < 4; ++i) {
        TG_CUDA(cudaMemcpyAsync(two + i * ld, f2[i], sizeof(double) * ncol, cudaMemcpyHostToDevice, st));
        *dst2[i] = two + i * ld;
    }
    TG_CUDA(cudaMemcpyAsync(one, F->expz, sizeof(double) * nk, cudaMemcpyHostToDevice, st));
    TG_CUDA(cudaMemcpyAsync(one + nk, F->dift, sizeof(double) * nk, cudaMemcpyHostToDevice, st));
    D.expz = one;
    D.dift = one + nk;
    if ((rc = grow(c->scratch[0], sizeof(double) * dt_scratch_planes() * lvl))) return rc;
    TG_CUDA(cudaMemsetAsync(c->flags, 0, sizeof(unsigned), st));
    TG_CUDA(launch_dt_ng(D, *C, out, nk, ncol, ld, nullptr, c->flags, st, nullptr, (double *)c->scratch[0].p));
    TG_CUDA(launch_level_to_col(out, ld, stage, nk, nk, ncol, st));
    TG_CUDA(cudaMemcpyAsync(tn_upd, stage, sizeof(double) * colsz, cudaMemcpyDeviceToHost, st));
    TG_CUDA(cudaStreamSynchronize(st));
    TG_CUDA(cudaMemcpy(c->flags_host, c->flags, sizeof(unsigned), cudaMemcpyDeviceToHost));
    return flags_to_status(c->flags_host[0]);
}

__attribute__((visibility("default"))) int tg_minor_ng_dev(const tg_minor_fields *F, const tg_minor_consts *C,
                                                           double *out, int nk, int ncol, long ld, double *system_out,
                                                           int *status_dev, void *stream)
{
    if (!F || !C || !out || nk < 3 || ncol < 0 || ld < ncol) {
        set_err("tg_minor_ng_dev: bad arguments (nk=%d ncol=%d ld=%ld)", nk, ncol, ld);
        return TG_EINVAL;
    }
    const double *const ptrs[] = {F->tn, F->o2, F->o1, F->he, F->mbar, F->barm, F->xnmbar, F->w, F->ftm1_smooth,
                                  F->hadvec, F->sloss, F->sprod, F->tlbc, F->flbc1, F->flbc2, F->flbc3, F->fubc,
                                  F->dfactor, F->expz, F->difk};
    for (const double *p : ptrs)
        if (!p) return set_err("tg_minor_ng_dev: a field pointer is NULL"), TG_EINVAL;
    DevCtx *cx = nullptr;
    int rc = get_ctx(&cx);
    if (rc) return rc;
    std::lock_guard<std::mutex> lk(cx->mu);
    cudaStream_t st = (cudaStream_t)stream;
    StreamWs *ws = nullptr;
    if ((rc = stream_ws(cx, st, &ws))) return rc;
    if ((rc = grow(ws->scratch, sizeof(double) * minor_scratch_planes() * (size_t)nk * (size_t)(ld > 0 ? ld : 1)))) return rc;
    TG_CUDA(cudaMemsetAsync(ws->flags, 0, sizeof(unsigned), st));
    TG_CUDA(launch_minor_ng(*F, *C, out, nk, ncol, ld, system_out, ws->flags, st, (double *)ws->scratch.p));
    if (status_dev) {
        k_finish_status<<<1, 1, 0, st>>>(ws->flags, status_dev);
        TG_CUDA(cudaGetLastError());
    }
    return TG_OK;
}

__attribute__((visibility("default"))) int tg_minor_ng(const tg_minor_fields *F, const tg_minor_consts *C,
                                                       double *out, int nk, int ncol)
{
    if (!F || !C || !out || nk < 3 || ncol < 0) {
        set_err("tg_minor_ng: bad arguments (nk=%d ncol=%d)", nk, ncol);
        return TG_EINVAL;
    }
    if (ncol == 0) return TG_OK;
    const double *const f3[12] = {F->tn, F->o2, F->o1, F->he, F->mbar, F->barm, F->xnmbar, F->w, F->ftm1_smooth,
                                  F->hadvec, F->sloss, F->sprod};
    const double *const f2[6] = {F->tlbc, F->flbc1, F->flbc2, F->flbc3, F->fubc, F->dfactor};
    for (const double *p : f3)
        if (!p) return set_err("tg_minor_ng: a field pointer is NULL"), TG_EINVAL;
    for (const double *p : f2)
        if (!p) return set_err("tg_minor_ng: a field pointer is NULL"), TG_EINVAL;
    if (!F->expz || !F->difk) return set_err("tg_minor_ng: expz/difk NULL"), TG_EINVAL;
    DevCtx *c = nullptr;
    int rc = get_ctx(&c);
    if (rc) return rc;
    std::lock_guard<std::mutex> lk(c->mu);
    TG_CUDA(cudaSetDevice(c->dev));
    const long ld = round_up(ncol, 32);
    const size_t lvl = (size_t)nk * ld, colsz = (size_t)nk * ncol;
    if ((rc = grow(c->lvlbuf[0][0], sizeof(double) * (13 * lvl + 6 * (size_t)ld + 2 * (size_t)nk)))) return rc;
    if ((rc = grow(c->colbuf[0][0], sizeof(double) * colsz))) return rc;
    double *base = (double *)c->lvlbuf[0][0].p, *stage = (double *)c->colbuf[0][0].p;
    cudaStream_t st = c->st[0];
    tg_minor_fields D;
    const double **dst3[12] = {&D.tn, &D.o2, &D.o1, &D.he, &D.mbar, &D.barm, &D.xnmbar, &D.w, &D.ftm1_smooth,
                               &D.hadvec, &D.sloss, &D.sprod};
    for (int i = 0; i < 12; ++i) {
        double *d = base + i * lvl;
        TG_CUDA(cudaMemcpyAsync(stage, f3[i], sizeof(double) * colsz, cudaMemcpyHostToDevice, st));
        TG_CUDA(launch_col_to_level(stage, nk, d, ld, nk, ncol, st));
        *dst3[i] = d;
    }
    double *out_l = base + 12 * lvl, *two = base + 13 * lvl, *one = two + 6 * ld;
    const double **dst2[6] = {&D.tlbc, &D.flbc1, &D.flbc2, &D.flbc3, &D.fubc, &D.dfactor};
    for (int i = 0; i < 6; ++i) {
        TG_CUDA(cudaMemcpyAsync(two + i * ld, f2[i], sizeof(double) * ncol, cudaMemcpyHostToDevice, st));
        *dst2[i] = two + i * ld;
    }
    TG_CUDA(cudaMemcpyAsync(one, F->expz, sizeof(double) * nk, cudaMemcpyHostToDevice, st));
    TG_CUDA(cudaMemcpyAsync(one + nk, F->difk, sizeof(double) * nk, cudaMemcpyHostToDevice, st));
    D.expz = one;
    D.difk = one + nk;
    TG_CUDA(cudaMemsetAsync(c->flags, 0, sizeof(unsigned), st));
    if ((rc = grow(c->scratch[0], sizeof(double) * minor_scratch_planes() * lvl))) return rc;
    TG_CUDA(launch_minor_ng(D, *C, out_l, nk, ncol, ld, nullptr, c->flags, st, (double *)c->scratch[0].p));
    TG_CUDA(launch_level_to_col(out_l, ld, stage, nk, nk, ncol, st));
    TG_CUDA(cudaMemcpyAsync(out, stage, sizeof(double) * colsz, cudaMemcpyDeviceToHost, st));
    TG_CUDA(cudaStreamSynchronize(st));
    TG_CUDA(cudaMemcpy(c->flags_host, c->flags, sizeof(unsigned), cudaMemcpyDeviceToHost));
    return flags_to_status(c->flags_host[0]);
}

// ---- history diagnostics of dt_ng and minor_ng (the addfld fields) --------
// Host forms: the fields and the solution in the Fortran layout, relaid out to
// level-major planes; diag receives nd slabs of (nk, ncol).
namespace {
struct Upload {
    double *base, *stage;
    long ld;
    size_t lvl, colsz;
    cudaStream_t st;
};
int upload3(const Upload &u, int nk, long ncol, const double *src, int i, const double **dst)
{
    double *d = u.base + (size_t)i * u.lvl;
    TG_CUDA(cudaMemcpyAsync(u.stage, src, sizeof(double) * u.colsz, cudaMemcpyHostToDevice, u.st));
    TG_CUDA(launch_col_to_level(u.stage, nk, d, u.ld, nk, ncol, u.st));
    *dst = d;
    return TG_OK;
}
int download3(const Upload &u, int nk, long ncol, const double *planes, int nd, double *diag)
{
    for (int i = 0; i < nd; ++i) {
        TG_CUDA(launch_level_to_col(planes + (size_t)i * u.lvl, u.ld, u.stage, nk, nk, ncol, u.st));
        TG_CUDA(cudaMemcpyAsync(diag + (size_t)i * u.colsz, u.stage, sizeof(double) * u.colsz, cudaMemcpyDeviceToHost,
                                u.st));
    }
    TG_CUDA(cudaStreamSynchronize(u.st));
    return TG_OK;
}
}  // namespace

__attribute__((visibility("default"))) int tg_dt_diag_ng_dev(const tg_dt_fields *F, const tg_dt_consts *C,
                                                             const double *tn_upd, double *diag, int nk, int ncol,
                                                             long ld, void *stream)
{
    if (!F || !C || !tn_upd || !diag || nk < 3 || ncol < 0 || ld < ncol) {
        set_err("tg_dt_diag_ng_dev: bad arguments (nk=%d ncol=%d ld=%ld)", nk, ncol, ld);
        return TG_EINVAL;
    }
    TG_CUDA(launch_dt_diag_ng(*F, *C, tn_upd, nk, ncol, ld, diag, (cudaStream_t)stream));
    return TG_OK;
}

__attribute__((visibility("default"))) int tg_minor_diag_ng_dev(const tg_minor_fields *F, const tg_minor_consts *C,
                                                                const double *fcomp_out, double *diag, int nk,
                                                                int ncol, long ld, void *stream)
{
    if (!F || !C || !fcomp_out || !diag || nk < 3 || ncol < 0 || ld < ncol) {
        set_err("tg_minor_diag_ng_dev: bad arguments (nk=%d ncol=%d ld=%ld)", nk, ncol, ld);
        return TG_EINVAL;
    }
    TG_CUDA(launch_minor_diag_ng(*F, *C, fcomp_out, nk, ncol, ld, diag, (cudaStream_t)stream));
    return TG_OK;
}

__attribute__((visibility("default"))) int tg_dt_diag_ng(const tg_dt_fields *F, const tg_dt_consts *C,
                                                         const double *tn_upd, double *diag, int nk, int ncol)
{
    if (!F || !C || !tn_upd || !diag || nk < 3 || ncol < 0) {
        set_err("tg_dt_diag_ng: bad arguments (nk=%d ncol=%d)", nk, ncol);
        return TG_EINVAL;
    }
    if (ncol == 0) return TG_OK;
    const double *const f3[21] = {F->tn, F->tnsmooth, F->horadv, F->un, F->vn, F->o1, F->mbar, F->xnmbar,
                                  F->scht, F->schti, F->cp, F->kt, F->km, F->hdt, F->qji_tn, F->cool_imp,
                                  F->cool_exp, F->w, F->qtotal, F->rkm12, tn_upd};
    const double *const f2[4] = {F->tlbc, F->t_lbc, F->ulbc, F->vlbc};
    for (const double *p : f3)
        if (!p) return set_err("tg_dt_diag_ng: a field pointer is NULL"), TG_EINVAL;
    for (const double *p : f2)
        if (!p) return set_err("tg_dt_diag_ng: a field pointer is NULL"), TG_EINVAL;
    if (!F->expz || !F->dift) return set_err("tg_dt_diag_ng: expz/dift NULL"), TG_EINVAL;
    DevCtx *c = nullptr;
    int rc = get_ctx(&c);
    if (rc) return rc;
    std::lock_guard<std::mutex> lk(c->mu);
    TG_CUDA(cudaSetDevice(c->dev));
    const long ld = round_up(ncol, 32);
    Upload u{nullptr, nullptr, ld, (size_t)nk * ld, (size_t)nk * ncol, c->st[0]};
    if ((rc = grow(c->lvlbuf[0][0], sizeof(double) * (33 * u.lvl + 4 * (size_t)ld + 2 * (size_t)nk)))) return rc;
    if ((rc = grow(c->colbuf[0][0], sizeof(double) * u.colsz))) return rc;
    u.base = (double *)c->lvlbuf[0][0].p;
    u.stage = (double *)c->colbuf[0][0].p;
    tg_dt_fields D;
    const double *x = nullptr;
    const double **dst3[21] = {&D.tn, &D.tnsmooth, &D.horadv, &D.un, &D.vn, &D.o1, &D.mbar, &D.xnmbar, &D.scht,
                               &D.schti, &D.cp, &D.kt, &D.km, &D.hdt, &D.qji_tn, &D.cool_imp, &D.cool_exp, &D.w,
                               &D.qtotal, &D.rkm12, &x};
    for (int i = 0; i < 21; ++i)
        if ((rc = upload3(u, nk, ncol, f3[i], i, dst3[i]))) return rc;
    double *planes = u.base + 21 * u.lvl, *two = u.base + 33 * u.lvl, *one = two + 4 * ld;
    const double **dst2[4] = {&D.tlbc, &D.t_lbc, &D.ulbc, &D.vlbc};
    for (int i = 0; i < 4; ++i) {
        TG_CUDA(cudaMemcpyAsync(two + i * ld, f2[i], sizeof(double) * ncol, cudaMemcpyHostToDevice, u.st));
        *dst2[i] = two + i * ld;
    }
    TG_CUDA(cudaMemcpyAsync(one, F->expz, sizeof(double) * nk, cudaMemcpyHostToDevice, u.st));
    TG_CUDA(cudaMemcpyAsync(one + nk, F->dift, sizeof(double) * nk, cudaMemcpyHostToDevice, u.st));
    D.expz = one;
    D.dift = one + nk;
    TG_CUDA(launch_dt_diag_ng(D, *C, x, nk, ncol, ld, planes, u.st));
    return download3(u, nk, ncol, planes, 12, diag);
}

__attribute__((visibility("default"))) int tg_minor_diag_ng(const tg_minor_fields *F, const tg_minor_consts *C,
                                                            const double *fcomp_out, double *diag, int nk, int ncol)
{
    if (!F || !C || !fcomp_out || !diag || nk < 3 || ncol < 0) {
        set_err("tg_minor_diag_ng: bad arguments (nk=%d ncol=%d)", nk, ncol);
        return TG_EINVAL;
    }
    if (ncol == 0) return TG_OK;
    const double *const f3[13] = {F->tn, F->o2, F->o1, F->he, F->mbar, F->barm, F->xnmbar, F->w, F->ftm1_smooth,
                                  F->hadvec, F->sloss, F->sprod, fcomp_out};
    const double *const f2[6] = {F->tlbc, F->flbc1, F->flbc2, F->flbc3, F->fubc, F->dfactor};
    for (const double *p : f3)
        if (!p) return set_err("tg_minor_diag_ng: a field pointer is NULL"), TG_EINVAL;
    for (const double *p : f2)
        if (!p) return set_err("tg_minor_diag_ng: a field pointer is NULL"), TG_EINVAL;
    if (!F->expz || !F->difk) return set_err("tg_minor_diag_ng: expz/difk NULL"), TG_EINVAL;
    DevCtx *c = nullptr;
    int rc = get_ctx(&c);
    if (rc) return rc;
    std::lock_guard<std::mutex> lk(c->mu);
    TG_CUDA(cudaSetDevice(c->dev));
    const long ld = round_up(ncol, 32);
    Upload u{nullptr, nullptr, ld, (size_t)nk * ld, (size_t)nk * ncol, c->st[0]};
    if ((rc = grow(c->lvlbuf[0][0], sizeof(double) * (20 * u.lvl + 6 * (size_t)ld + 2 * (size_t)nk)))) return rc;
    if ((rc = grow(c->colbuf[0][0], sizeof(double) * u.colsz))) return rc;
    u.base = (double *)c->lvlbuf[0][0].p;
    u.stage = (double *)c->colbuf[0][0].p;
    tg_minor_fields D;
    const double *x = nullptr;
    const double **dst3[13] = {&D.tn, &D.o2, &D.o1, &D.he, &D.mbar, &D.barm, &D.xnmbar, &D.w, &D.ftm1_smooth,
                               &D.hadvec, &D.sloss, &D.sprod, &x};
    for (int i = 0; i < 13; ++i)
        if ((rc = upload3(u, nk, ncol, f3[i], i, dst3[i]))) return rc;
    double *planes = u.base + 13 * u.lvl, *two = u.base + 20 * u.lvl, *one = two + 6 * ld;
    const double **dst2[6] = {&D.tlbc, &D.flbc1, &D.flbc2, &D.flbc3, &D.fubc, &D.dfactor};
    for (int i = 0; i < 6; ++i) {
        TG_CUDA(cudaMemcpyAsync(two + i * ld, f2[i], sizeof(double) * ncol, cudaMemcpyHostToDevice, u.st));
        *dst2[i] = two + i * ld;
    }
    TG_CUDA(cudaMemcpyAsync(one, F->expz, sizeof(double) * nk, cudaMemcpyHostToDevice, u.st));
    TG_CUDA(cudaMemcpyAsync(one + nk, F->difk, sizeof(double) * nk, cudaMemcpyHostToDevice, u.st));
    D.expz = one;
    D.difk = one + nk;
    TG_CUDA(launch_minor_diag_ng(D, *C, x, nk, ncol, ld, planes, u.st));
    return download3(u, nk, ncol, planes, 7, diag);
}

// ---- the post-solve steps fused into the back sweep -------------------------
static bool post_ok(const char *who, const tg_post_step *P)
{
    if (!P || !P->cur || !P->prev || !P->nm_upd || (!P->bnd_mask) != (!P->bnd)) {
        set_err("%s: bad post-step arguments (cur, prev, nm_upd needed; bnd_mask and bnd both or neither)", who);
        return false;
    }
    return true;
}
static PostStep post_of(const tg_post_step *P, double floor, int floor_nm)
{
    return PostStep{P->cur, P->prev, P->nm_upd, P->bnd_mask, P->bnd, P->dtsmooth, P->dtsmooth_div2, floor, floor_nm};
}

__attribute__((visibility("default"))) int tg_dt_ng_post_dev(const tg_dt_fields *F, const tg_dt_consts *C,
                                                             double *tn_upd, int nk, int ncol, long ld,
                                                             const tg_post_step *P, int *status_dev, void *stream)
{
    if (!F || !C || !tn_upd || nk < 3 || ncol < 0 || ld < ncol || !post_ok("tg_dt_ng_post_dev", P)) {
        if (!P || P->cur) set_err("tg_dt_ng_post_dev: bad arguments (nk=%d ncol=%d ld=%ld)", nk, ncol, ld);
        return TG_EINVAL;
    }
    DevCtx *cx = nullptr;
    int rc = get_ctx(&cx);
    if (rc) return rc;
    std::lock_guard<std::mutex> lk(cx->mu);
    cudaStream_t st = (cudaStream_t)stream;
    StreamWs *ws = nullptr;
    if ((rc = stream_ws(cx, st, &ws))) return rc;
    const PostStep post = post_of(P, 100.0, 0);
    TG_CUDA(cudaMemsetAsync(ws->flags, 0, sizeof(unsigned), st));
    if ((rc = grow(ws->scratch, sizeof(double) * dt_scratch_planes() * (size_t)nk * (size_t)(ld > 0 ? ld : 1))))
        return rc;
    TG_CUDA(launch_dt_ng(*F, *C, tn_upd, nk, ncol, ld, nullptr, ws->flags, st, &post, (double *)ws->scratch.p));
    if (status_dev) {
        k_finish_status<<<1, 1, 0, st>>>(ws->flags, status_dev);
        TG_CUDA(cudaGetLastError());
    }
    return TG_OK;
}

__attribute__((visibility("default"))) int tg_minor_ng_post_dev(const tg_minor_fields *F, const tg_minor_consts *C,
                                                                double *fcomp_out, int nk, int ncol, long ld,
                                                                const tg_post_step *P, int *status_dev, void *stream)
{
    if (!F || !C || !fcomp_out || nk < 3 || ncol < 0 || ld < ncol || !post_ok("tg_minor_ng_post_dev", P)) {
        if (!P || P->cur) set_err("tg_minor_ng_post_dev: bad arguments (nk=%d ncol=%d ld=%ld)", nk, ncol, ld);
        return TG_EINVAL;
    }
    DevCtx *cx = nullptr;
    int rc = get_ctx(&cx);
    if (rc) return rc;
    std::lock_guard<std::mutex> lk(cx->mu);
    cudaStream_t st = (cudaStream_t)stream;
    StreamWs *ws = nullptr;
    if ((rc = stream_ws(cx, st, &ws))) return rc;
    if ((rc = grow(ws->scratch, sizeof(double) * minor_scratch_planes() * (size_t)nk * (size_t)(ld > 0 ? ld : 1)))) return rc;
    const PostStep post = post_of(P, 1.e-12, 1);
    TG_CUDA(cudaMemsetAsync(ws->flags, 0, sizeof(unsigned), st));
    TG_CUDA(launch_minor_ng(*F, *C, fcomp_out, nk, ncol, ld, nullptr, ws->flags, st, (double *)ws->scratch.p,
                            &post));
    if (status_dev) {
        k_finish_status<<<1, 1, 0, st>>>(ws->flags, status_dev);
        TG_CUDA(cudaGetLastError());
    }
    return TG_OK;
}

static bool comp_fields_ok(const tg_comp_fields *F)
{
    const double *const p[] = {F->tn, F->o2, F->o1, F->he, F->w, F->mbar, F->o2nm_smooth, F->o1nm_smooth,
                               F->henm_smooth, F->o2_advec, F->o1_advec, F->he_advec, F->hdo2, F->hdo1, F->hdhe,
                               F->fs, F->tlbc, F->flx_he, F->dfactor, F->expz, F->difk};
    for (const double *q : p)
        if (!q) return false;
    return true;
}

__attribute__((visibility("default"))) int tg_comp_ng_dev(const tg_comp_fields *F, const tg_comp_consts *C,
                                                          double *out, int nk, int ncol, long ld, double *system_out,
                                                          int *status_dev, void *stream)
{
    if (!F || !C || !out || nk < 3 || ncol < 0 || ld < ncol || !comp_fields_ok(F)) {
        set_err("tg_comp_ng_dev: bad arguments (nk=%d ncol=%d ld=%ld)", nk, ncol, ld);
        return TG_EINVAL;
    }
    DevCtx *cx = nullptr;
    int rc = get_ctx(&cx);
    if (rc) return rc;
    std::lock_guard<std::mutex> lk(cx->mu);
    cudaStream_t st = (cudaStream_t)stream;
    StreamWs *ws = nullptr;
    if ((rc = stream_ws(cx, st, &ws))) return rc;
    if ((rc = grow(ws->scratch, sizeof(double) * comp_scratch_doubles(nk, ld > 0 ? ld : 1)))) return rc;
    TG_CUDA(cudaMemsetAsync(ws->flags, 0, sizeof(unsigned), st));
    TG_CUDA(launch_comp_ng(*F, *C, out, (double *)ws->scratch.p, nk, ncol, ld, system_out, ws->flags, st));
    if (status_dev) {
        k_finish_status<<<1, 1, 0, st>>>(ws->flags, status_dev);
        TG_CUDA(cudaGetLastError());
    }
    return TG_OK;
}

__attribute__((visibility("default"))) int tg_comp_diag_ng_dev(const tg_comp_fields *F, const tg_comp_consts *C,
                                                               const double *upd, double *diag, int nk, int ncol,
                                                               long ld, void *stream)
{
    if (!F || !C || !upd || !diag || nk < 3 || ncol < 0 || ld < ncol || !comp_fields_ok(F)) {
        set_err("tg_comp_diag_ng_dev: bad arguments (nk=%d ncol=%d ld=%ld)", nk, ncol, ld);
        return TG_EINVAL;
    }
    DevCtx *cx = nullptr;
    int rc = get_ctx(&cx);
    if (rc) return rc;
    std::lock_guard<std::mutex> lk(cx->mu);
    cudaStream_t st = (cudaStream_t)stream;
    StreamWs *ws = nullptr;
    if ((rc = stream_ws(cx, st, &ws))) return rc;
    if ((rc = grow(ws->scratch, sizeof(double) * comp_scratch_doubles(nk, ld > 0 ? ld : 1)))) return rc;
    TG_CUDA(launch_comp_diag_ng(*F, *C, upd, nk, ncol, ld, diag, (double *)ws->scratch.p, st));
    return TG_OK;
}

__attribute__((visibility("default"))) int tg_comp_diag_ng(const tg_comp_fields *F, const tg_comp_consts *C,
                                                           const double *o2_upd, const double *o1_upd,
                                                           const double *he_upd, double *diag, int nk, int ncol)
{
    if (!F || !C || !o2_upd || !o1_upd || !he_upd || !diag || nk < 3 || ncol < 0 || !comp_fields_ok(F)) {
        set_err("tg_comp_diag_ng: bad arguments (nk=%d ncol=%d)", nk, ncol);
        return TG_EINVAL;
    }
    if (ncol == 0) return TG_OK;
    DevCtx *c = nullptr;
    int rc = get_ctx(&c);
    if (rc) return rc;
    std::lock_guard<std::mutex> lk(c->mu);
    TG_CUDA(cudaSetDevice(c->dev));
    const long ld = round_up(ncol, 32);
    Upload u{nullptr, nullptr, ld, (size_t)nk * ld, (size_t)nk * ncol, c->st[0]};
    // 15 fields, 12 fs slabs and the 3 solution planes, then 24 diagnostic planes, 3 rows, 2 profiles
    if ((rc = grow(c->lvlbuf[0][0], sizeof(double) * (54 * u.lvl + 3 * (size_t)ld + 2 * (size_t)nk)))) return rc;
    if ((rc = grow(c->colbuf[0][0], sizeof(double) * u.colsz))) return rc;
    if ((rc = grow(c->scratch[0], sizeof(double) * comp_scratch_doubles(nk, ld)))) return rc;
    u.base = (double *)c->lvlbuf[0][0].p;
    u.stage = (double *)c->colbuf[0][0].p;
    tg_comp_fields D;
    const double *src3[15] = {F->tn, F->o2, F->o1, F->he, F->w, F->mbar, F->o2nm_smooth, F->o1nm_smooth,
                              F->henm_smooth, F->o2_advec, F->o1_advec, F->he_advec, F->hdo2, F->hdo1, F->hdhe};
    const double **dst3[15] = {&D.tn, &D.o2, &D.o1, &D.he, &D.w, &D.mbar, &D.o2nm_smooth, &D.o1nm_smooth,
                               &D.henm_smooth, &D.o2_advec, &D.o1_advec, &D.he_advec, &D.hdo2, &D.hdo1, &D.hdhe};
    for (int i = 0; i < 15; ++i)
        if ((rc = upload3(u, nk, ncol, src3[i], i, dst3[i]))) return rc;
    const double *ignored = nullptr;
    for (int i = 0; i < 12; ++i)
        if ((rc = upload3(u, nk, ncol, F->fs + (size_t)i * u.colsz, 15 + i, &ignored))) return rc;
    D.fs = u.base + 15 * u.lvl;
    const double *x3[3] = {o2_upd, o1_upd, he_upd};
    for (int i = 0; i < 3; ++i)
        if ((rc = upload3(u, nk, ncol, x3[i], 27 + i, &ignored))) return rc;
    double *planes = u.base + 30 * u.lvl, *two = u.base + 54 * u.lvl, *one = two + 3 * ld;
    const double *src2[3] = {F->tlbc, F->flx_he, F->dfactor};
    const double **dst2[3] = {&D.tlbc, &D.flx_he, &D.dfactor};
    for (int i = 0; i < 3; ++i) {
        TG_CUDA(cudaMemcpyAsync(two + i * ld, src2[i], sizeof(double) * ncol, cudaMemcpyHostToDevice, u.st));
        *dst2[i] = two + i * ld;
    }
    TG_CUDA(cudaMemcpyAsync(one, F->expz, sizeof(double) * nk, cudaMemcpyHostToDevice, u.st));
    TG_CUDA(cudaMemcpyAsync(one + nk, F->difk, sizeof(double) * nk, cudaMemcpyHostToDevice, u.st));
    D.expz = one;
    D.difk = one + nk;
    TG_CUDA(launch_comp_diag_ng(D, *C, u.base + 27 * u.lvl, nk, ncol, ld, planes, (double *)c->scratch[0].p, u.st));
    return download3(u, nk, ncol, planes, 24, diag);
}

__attribute__((visibility("default"))) int tg_comp_ng(const tg_comp_fields *F, const tg_comp_consts *C,
                                                      double *o2_upd, double *o1_upd, double *he_upd, int nk,
                                                      int ncol)
{
    if (!F || !C || !o2_upd || !o1_upd || !he_upd || nk < 3 || ncol < 0 || !comp_fields_ok(F)) {
        set_err("tg_comp_ng: bad arguments (nk=%d ncol=%d)", nk, ncol);
        return TG_EINVAL;
    }
    if (ncol == 0) return TG_OK;
    DevCtx *c = nullptr;
    int rc = get_ctx(&c);
    if (rc) return rc;
    std::lock_guard<std::mutex> lk(c->mu);
    TG_CUDA(cudaSetDevice(c->dev));
    const long ld = round_up(ncol, 32);
    const size_t lvl = (size_t)nk * ld, colsz = (size_t)nk * ncol;
    // 15 fields + 12 fs slabs + 3 outputs, level-major; 3 2-D rows; 2 level profiles
    if ((rc = grow(c->lvlbuf[0][0], sizeof(double) * (30 * lvl + 3 * (size_t)ld + 2 * (size_t)nk)))) return rc;
    if ((rc = grow(c->colbuf[0][0], sizeof(double) * colsz))) return rc;
    if ((rc = grow(c->scratch[0], sizeof(double) * comp_scratch_doubles(nk, ld)))) return rc;
    double *base = (double *)c->lvlbuf[0][0].p, *stage = (double *)c->colbuf[0][0].p;
    cudaStream_t st = c->st[0];
    tg_comp_fields D;
    const double *src3[15] = {F->tn, F->o2, F->o1, F->he, F->w, F->mbar, F->o2nm_smooth, F->o1nm_smooth,
                              F->henm_smooth, F->o2_advec, F->o1_advec, F->he_advec, F->hdo2, F->hdo1, F->hdhe};
    const double **dst3[15] = {&D.tn, &D.o2, &D.o1, &D.he, &D.w, &D.mbar, &D.o2nm_smooth, &D.o1nm_smooth,
                               &D.henm_smooth, &D.o2_advec, &D.o1_advec, &D.he_advec, &D.hdo2, &D.hdo1, &D.hdhe};
    for (int i = 0; i < 27; ++i) {
        const double *h = i < 15 ? src3[i] : F->fs + (size_t)(i - 15) * colsz;
        double *d = base + i * lvl;
        TG_CUDA(cudaMemcpyAsync(stage, h, sizeof(double) * colsz, cudaMemcpyHostToDevice, st));
        TG_CUDA(launch_col_to_level(stage, nk, d, ld, nk, ncol, st));
        if (i < 15) *dst3[i] = d;
    }
    D.fs = base + 15 * lvl;
    double *out_l = base + 27 * lvl, *two = base + 30 * lvl, *one = two + 3 * ld;
    const double *src2[3] = {F->tlbc, F->flx_he, F->dfactor};
    const double **dst2[3] = {&D.tlbc, &D.flx_he, &D.dfactor};
    for (int i = 0; i < 3; ++i) {
        TG_CUDA(cudaMemcpyAsync(two + i * ld, src2[i], sizeof(double) * ncol, cudaMemcpyHostToDevice, st));
        *dst2[i] = two + i * ld;
    }
    TG_CUDA(cudaMemcpyAsync(one, F->expz, sizeof(double) * nk, cudaMemcpyHostToDevice, st));
    TG_CUDA(cudaMemcpyAsync(one + nk, F->difk, sizeof(double) * nk, cudaMemcpyHostToDevice, st));
    D.expz = one;
    D.difk = one + nk;
    TG_CUDA(cudaMemsetAsync(c->flags, 0, sizeof(unsigned), st));
    TG_CUDA(launch_comp_ng(D, *C, out_l, (double *)c->scratch[0].p, nk, ncol, ld, nullptr, c->flags, st));
    double *hout[3] = {o2_upd, o1_upd, he_upd};
    for (int i = 0; i < 3; ++i) {
        TG_CUDA(launch_level_to_col(out_l + i * lvl, ld, stage, nk, nk, ncol, st));
        TG_CUDA(cudaMemcpyAsync(hout[i], stage, sizeof(double) * colsz, cudaMemcpyDeviceToHost, st));
        // the staging buffer is reused by the next species
        TG_CUDA(cudaStreamSynchronize(st));
    }
    TG_CUDA(cudaMemcpy(c->flags_host, c->flags, sizeof(unsigned), cudaMemcpyDeviceToHost));
    return flags_to_status(c->flags_host[0]);
}

__attribute__((visibility("default"))) int tg_comp_post_ng(const double *o2, const double *o1, const double *he,
                                                           const double *o2_nm, const double *o1_nm,
                                                           const double *he_nm, const double *xnmbar,
                                                           const double *zpmid, double dz, double dtsmooth,
                                                           double dtsmooth_div2, int nk, int ncol, double *o2_upd,
                                                           double *o1_upd, double *he_upd, double *o2nm_upd,
                                                           double *o1nm_upd, double *henm_upd)
{
    const double *in7[7] = {o2, o1, he, o2_nm, o1_nm, he_nm, xnmbar};
    double *io6[6] = {o2_upd, o1_upd, he_upd, o2nm_upd, o1nm_upd, henm_upd};
    bool ok = zpmid && nk >= 1 && ncol >= 0;
    for (const double *p : in7) ok = ok && p;
    for (double *p : io6) ok = ok && p;
    if (!ok) {
        set_err("tg_comp_post_ng: bad arguments (nk=%d ncol=%d)", nk, ncol);
        return TG_EINVAL;
    }
    if (ncol == 0) return TG_OK;
    DevCtx *c = nullptr;
    int rc = get_ctx(&c);
    if (rc) return rc;
    std::lock_guard<std::mutex> lk(c->mu);
    TG_CUDA(cudaSetDevice(c->dev));
    const long ld = round_up(ncol, 32);
    const size_t lvl = (size_t)nk * ld, colsz = (size_t)nk * ncol;
    if ((rc = grow(c->lvlbuf[0][0], sizeof(double) * (13 * lvl + (size_t)nk)))) return rc;
    if ((rc = grow(c->colbuf[0][0], sizeof(double) * colsz))) return rc;
    double *base = (double *)c->lvlbuf[0][0].p, *stage = (double *)c->colbuf[0][0].p;
    cudaStream_t st = c->st[0];
    const double *din[7];
    double *dio[6];
    for (int i = 0; i < 10; ++i) {
        const double *h = i < 7 ? in7[i] : io6[i - 7];
        double *d = base + i * lvl;
        TG_CUDA(cudaMemcpyAsync(stage, h, sizeof(double) * colsz, cudaMemcpyHostToDevice, st));
        TG_CUDA(launch_col_to_level(stage, nk, d, ld, nk, ncol, st));
        if (i < 7) din[i] = d;
        else dio[i - 7] = d;
    }
    for (int i = 3; i < 6; ++i) dio[i] = base + (10 + i - 3) * lvl;
    double *zp = base + 13 * lvl;
    TG_CUDA(cudaMemcpyAsync(zp, zpmid, sizeof(double) * nk, cudaMemcpyHostToDevice, st));
    TG_CUDA(launch_comp_post_ng(din, zp, dz, dtsmooth, dtsmooth_div2, nk, ncol, ld, dio, st));
    for (int i = 0; i < 6; ++i) {
        TG_CUDA(launch_level_to_col(dio[i], ld, stage, nk, nk, ncol, st));
        TG_CUDA(cudaMemcpyAsync(io6[i], stage, sizeof(double) * colsz, cudaMemcpyDeviceToHost, st));
        TG_CUDA(cudaStreamSynchronize(st));
    }
    return TG_OK;
}

__attribute__((visibility("default"))) int tg_comp_post_ng_dev(const double *o2, const double *o1, const double *he,
                                                               const double *o2_nm, const double *o1_nm,
                                                               const double *he_nm, const double *xnmbar,
                                                               const double *zpmid, double dz, double dtsmooth,
                                                               double dtsmooth_div2, int nk, int ncol, long ld,
                                                               double *o2_upd, double *o1_upd, double *he_upd,
                                                               double *o2nm_upd, double *o1nm_upd, double *henm_upd,
                                                               const unsigned char *bnd_mask, const double *o2_bnd,
                                                               const double *o1_bnd, const double *he_bnd,
                                                               void *stream)
{
    const double *in7[7] = {o2, o1, he, o2_nm, o1_nm, he_nm, xnmbar};
    double *io6[6] = {o2_upd, o1_upd, he_upd, o2nm_upd, o1nm_upd, henm_upd};
    const double *bnd3[3] = {o2_bnd, o1_bnd, he_bnd};
    bool ok = zpmid && nk >= 1 && nk <= 65535 && ncol >= 0 && ld >= ncol &&
              (!bnd_mask || (o2_bnd && o1_bnd && he_bnd));
    for (const double *p : in7) ok = ok && p;
    for (double *p : io6) ok = ok && p;
    if (!ok) {
        set_err("tg_comp_post_ng_dev: bad arguments (nk=%d ncol=%d ld=%ld)", nk, ncol, ld);
        return TG_EINVAL;
    }
    TG_CUDA(launch_comp_post_ng(in7, zpmid, dz, dtsmooth, dtsmooth_div2, nk, ncol, ld, io6, (cudaStream_t)stream,
                                bnd_mask, bnd3));
    return TG_OK;
}

static bool horiz_args_ok(const char *who, int nk, int nlon, int nlat, long ld, bool ld_given)
{
    const long ncol = (long)(nlon + 4) * (nlat + 4);
    const bool ok = nk >= 1 && nk <= 65535 && nlon >= 1 && nlat >= 1 && nlon <= (1 << 24) && nlat <= 500000 &&
                    (!ld_given || ld >= ncol);
    if (!ok) set_err("%s: bad arguments (nk=%d nlon=%d nlat=%d ld=%ld)", who, nk, nlon, nlat, ld);
    return ok;
}

__attribute__((visibility("default"))) int tg_advec_ng_dev(const double *f, const double *un, const double *vn,
                                                           const double *racs, double dlamda, double dphi,
                                                           double re_inv, double *hadvec, int nk, int nlon,
                                                           int nlat, long ld, void *stream)
{
    if (!f || !un || !vn || !racs || !hadvec || hadvec == f || hadvec == un || hadvec == vn) {
        set_err("tg_advec_ng_dev: a pointer is NULL or hadvec aliases an input");
        return TG_EINVAL;
    }
    if (!horiz_args_ok("tg_advec_ng_dev", nk, nlon, nlat, ld, true)) return TG_EINVAL;
    TG_CUDA(launch_advec_ng(f, un, vn, racs, dlamda, dphi, re_inv, nk, nlon, nlat, ld, hadvec,
                            (cudaStream_t)stream));
    return TG_OK;
}

__attribute__((visibility("default"))) int tg_smooth_ng_dev(const double *fin, double shapiro, double *fout, int nk,
                                                            int nlon, int nlat, long ld, void *stream)
{
    if (!fin || !fout || fin == fout) {
        set_err("tg_smooth_ng_dev: a pointer is NULL or fout is fin");
        return TG_EINVAL;
    }
    if (!horiz_args_ok("tg_smooth_ng_dev", nk, nlon, nlat, ld, true)) return TG_EINVAL;
    TG_CUDA(launch_smooth_ng(fin, shapiro, nk, nlon, nlat, ld, fout, (cudaStream_t)stream));
    return TG_OK;
}

// The polar ring filter: the latitudes it changes and their chunk counts
// (src/ringfilter.F:24-33), checked against the filter's limits.
static bool ring_rows(const char *who, int nk, int nlon, int nlat, int order, const int *chunk_array,
                      int nlat_filter, RingRows *rows)
{
    if (nk < 1 || nk > 65535 || nlon < 1 || nlon > (1 << 20) || nlat < 1 || nlat > 500000 || order < 1 ||
        order > kMaxRingOrder || order >= nlon || nlat_filter < 0 || (nlat_filter > 0 && !chunk_array) ||
        ringfilter_smem_bytes(nlon) > (size_t)(200 * 1024)) {
        set_err("%s: bad arguments (nk=%d nlon=%d nlat=%d order=%d nlat_filter=%d; order must be 1..%d and below "
                "nlon)", who, nk, nlon, nlat, order, nlat_filter, kMaxRingOrder);
        return false;
    }
    rows->n = 0;
    for (int lat = 1; lat <= nlat; ++lat) {
        int nchnk = 0;
        if (lat <= nlat_filter) nchnk = chunk_array[lat - 1];
        else if (lat >= nlat - nlat_filter + 1) nchnk = chunk_array[nlat - lat];
        if (nchnk == 0) continue;
        if (nchnk < 3 || nchnk > nlon || rows->n == kMaxRingRows) {
            set_err("%s: latitude %d: %d chunks (3..nlon allowed, at most %d filtered latitudes)", who, lat, nchnk,
                    kMaxRingRows);
            return false;
        }
        rows->lat[rows->n] = lat - 1;
        rows->nchnk[rows->n] = nchnk;
        ++rows->n;
    }
    return true;
}

__attribute__((visibility("default"))) int tg_ringfilter_dev(double *f, int nk, int nlon, int nlat, int order,
                                                             int poly, const int *chunk_array, int nlat_filter,
                                                             double dlamda, long ld, void *stream)
{
    RingRows rows;
    if (!f || !ring_rows("tg_ringfilter_dev", nk, nlon, nlat, order, chunk_array, nlat_filter, &rows))
        return TG_EINVAL;
    if (ld < (long)(nlon + 4) * nlat) {
        set_err("tg_ringfilter_dev: ld %ld below (nlon+4)*nlat", ld);
        return TG_EINVAL;
    }
    TG_CUDA(launch_ringfilter(rows, f, ld, nk, nlon, order, poly ? 1 : 0, dlamda, (cudaStream_t)stream));
    return TG_OK;
}

__attribute__((visibility("default"))) int tg_ringfilter(double *f, int nk, int nlon, int nlat, int order, int poly,
                                                         const int *chunk_array, int nlat_filter, double dlamda)
{
    RingRows rows;
    if (!f || !ring_rows("tg_ringfilter", nk, nlon, nlat, order, chunk_array, nlat_filter, &rows)) return TG_EINVAL;
    if (rows.n == 0) return TG_OK;
    DevCtx *c = nullptr;
    int rc = get_ctx(&c);
    if (rc) return rc;
    std::lock_guard<std::mutex> lk(c->mu);
    TG_CUDA(cudaSetDevice(c->dev));
    const long ncol = (long)(nlon + 4) * nlat, ld = round_up(ncol, 32);
    const size_t colsz = (size_t)nk * ncol;
    if ((rc = grow(c->lvlbuf[0][0], sizeof(double) * (size_t)nk * ld))) return rc;
    if ((rc = grow(c->colbuf[0][0], sizeof(double) * colsz))) return rc;
    double *lvl = (double *)c->lvlbuf[0][0].p, *stage = (double *)c->colbuf[0][0].p;
    cudaStream_t st = c->st[0];
    TG_CUDA(cudaMemcpyAsync(stage, f, sizeof(double) * colsz, cudaMemcpyHostToDevice, st));
    TG_CUDA(launch_col_to_level(stage, nk, lvl, ld, nk, ncol, st));
    TG_CUDA(launch_ringfilter(rows, lvl, ld, nk, nlon, order, poly ? 1 : 0, dlamda, st));
    TG_CUDA(launch_level_to_col(lvl, ld, stage, nk, nk, ncol, st));
    TG_CUDA(cudaMemcpyAsync(f, stage, sizeof(double) * colsz, cudaMemcpyDeviceToHost, st));
    TG_CUDA(cudaStreamSynchronize(st));
    return TG_OK;
}

__attribute__((visibility("default"))) int tg_filter_o2o(double *fout, int nk, int nlon, int nlat,
                                                         const int *chunk_array, int nlat_filter, double dlamda)
{
    return tg_ringfilter(fout, nk, nlon, nlat, 1, 0, chunk_array, nlat_filter, dlamda);
}

// Host forms: the (nk, nlon+4, nlat+4) Fortran arrays are (nk, ncol) column
// arrays, relaid out to level-major planes for the kernels and back.
__attribute__((visibility("default"))) int tg_advec_ng(const double *f, const double *un, const double *vn,
                                                       const double *racs, double dlamda, double dphi,
                                                       double re_inv, int nk, int nlon, int nlat, double *hadvec)
{
    if (!f || !un || !vn || !racs || !hadvec || hadvec == f || hadvec == un || hadvec == vn) {
        set_err("tg_advec_ng: a pointer is NULL or hadvec aliases an input");
        return TG_EINVAL;
    }
    if (!horiz_args_ok("tg_advec_ng", nk, nlon, nlat, 0, false)) return TG_EINVAL;
    DevCtx *c = nullptr;
    int rc = get_ctx(&c);
    if (rc) return rc;
    std::lock_guard<std::mutex> lk(c->mu);
    TG_CUDA(cudaSetDevice(c->dev));
    const long ncol = (long)(nlon + 4) * (nlat + 4), ld = round_up(ncol, 32);
    const size_t lvl = (size_t)nk * ld, colsz = (size_t)nk * ncol;
    if ((rc = grow(c->lvlbuf[0][0], sizeof(double) * (4 * lvl + (size_t)(nlat + 4))))) return rc;
    if ((rc = grow(c->colbuf[0][0], sizeof(double) * colsz))) return rc;
    double *base = (double *)c->lvlbuf[0][0].p, *stage = (double *)c->colbuf[0][0].p;
    cudaStream_t st = c->st[0];
    const double *in3[3] = {f, un, vn};
    for (int i = 0; i < 3; ++i) {
        TG_CUDA(cudaMemcpyAsync(stage, in3[i], sizeof(double) * colsz, cudaMemcpyHostToDevice, st));
        TG_CUDA(launch_col_to_level(stage, nk, base + i * lvl, ld, nk, ncol, st));
    }
    double *out = base + 3 * lvl, *dr = base + 4 * lvl;
    TG_CUDA(cudaMemcpyAsync(dr, racs, sizeof(double) * (nlat + 4), cudaMemcpyHostToDevice, st));
    TG_CUDA(launch_advec_ng(base, base + lvl, base + 2 * lvl, dr, dlamda, dphi, re_inv, nk, nlon, nlat, ld, out, st));
    TG_CUDA(launch_level_to_col(out, ld, stage, nk, nk, ncol, st));
    TG_CUDA(cudaMemcpyAsync(hadvec, stage, sizeof(double) * colsz, cudaMemcpyDeviceToHost, st));
    TG_CUDA(cudaStreamSynchronize(st));
    return TG_OK;
}

__attribute__((visibility("default"))) int tg_smooth_ng(const double *fin, double shapiro, int nk, int nlon, int nlat,
                                                        double *fout)
{
    if (!fin || !fout || fin == fout) {
        set_err("tg_smooth_ng: a pointer is NULL or fout is fin");
        return TG_EINVAL;
    }
    if (!horiz_args_ok("tg_smooth_ng", nk, nlon, nlat, 0, false)) return TG_EINVAL;
    DevCtx *c = nullptr;
    int rc = get_ctx(&c);
    if (rc) return rc;
    std::lock_guard<std::mutex> lk(c->mu);
    TG_CUDA(cudaSetDevice(c->dev));
    const long ncol = (long)(nlon + 4) * (nlat + 4), ld = round_up(ncol, 32);
    const size_t lvl = (size_t)nk * ld, colsz = (size_t)nk * ncol;
    if ((rc = grow(c->lvlbuf[0][0], sizeof(double) * 2 * lvl))) return rc;
    if ((rc = grow(c->colbuf[0][0], sizeof(double) * colsz))) return rc;
    double *base = (double *)c->lvlbuf[0][0].p, *stage = (double *)c->colbuf[0][0].p;
    cudaStream_t st = c->st[0];
    TG_CUDA(cudaMemcpyAsync(stage, fin, sizeof(double) * colsz, cudaMemcpyHostToDevice, st));
    TG_CUDA(launch_col_to_level(stage, nk, base, ld, nk, ncol, st));
    TG_CUDA(launch_smooth_ng(base, shapiro, nk, nlon, nlat, ld, base + lvl, st));
    TG_CUDA(launch_level_to_col(base + lvl, ld, stage, nk, nk, ncol, st));
    TG_CUDA(cudaMemcpyAsync(fout, stage, sizeof(double) * colsz, cudaMemcpyDeviceToHost, st));
    TG_CUDA(cudaStreamSynchronize(st));
    return TG_OK;
}

static bool time_filter_args_ok(const char *who, int which, const double *cur, const double *prev, int nk, int ncol,
                                const double *upd, const double *nm)
{
    const bool ok = which >= TG_FILTER_DT && which <= TG_FILTER_OPLUS && cur && prev && upd && nm && upd != nm &&
                    upd != cur && upd != prev && nk >= 1 && ncol >= 0;
    if (!ok) set_err("%s: bad arguments (which=%d nk=%d ncol=%d)", who, which, nk, ncol);
    return ok;
}

__attribute__((visibility("default"))) int tg_time_filter_ng_dev(int which, const double *cur, const double *prev,
                                                                 double dtsmooth, double dtsmooth_div2, int nk,
                                                                 int ncol, long ld, double *upd, double *nm_upd,
                                                                 void *stream)
{
    if (!time_filter_args_ok("tg_time_filter_ng_dev", which, cur, prev, nk, ncol, upd, nm_upd)) return TG_EINVAL;
    if (ld < ncol || nk > 65535) {
        set_err("tg_time_filter_ng_dev: bad arguments (nk=%d ncol=%d ld=%ld)", nk, ncol, ld);
        return TG_EINVAL;
    }
    TG_CUDA(launch_time_filter(which, cur, prev, dtsmooth, dtsmooth_div2, nk, ncol, ld, upd, nm_upd,
                               (cudaStream_t)stream));
    return TG_OK;
}

__attribute__((visibility("default"))) int tg_time_filter_ng(int which, const double *cur, const double *prev,
                                                             double dtsmooth, double dtsmooth_div2, int nk, int ncol,
                                                             double *upd, double *nm_upd)
{
    if (!time_filter_args_ok("tg_time_filter_ng", which, cur, prev, nk, ncol, upd, nm_upd)) return TG_EINVAL;
    if (ncol == 0) return TG_OK;
    DevCtx *c = nullptr;
    int rc = get_ctx(&c);
    if (rc) return rc;
    std::lock_guard<std::mutex> lk(c->mu);
    TG_CUDA(cudaSetDevice(c->dev));
    // element-wise, so the Fortran (nk, ncol) arrays are one row of nk*ncol
    const size_t n = (size_t)nk * ncol, bytes = sizeof(double) * n;
    if ((rc = grow(c->lvlbuf[0][0], 4 * bytes))) return rc;
    double *d = (double *)c->lvlbuf[0][0].p;
    cudaStream_t st = c->st[0];
    TG_CUDA(cudaMemcpyAsync(d, cur, bytes, cudaMemcpyHostToDevice, st));
    TG_CUDA(cudaMemcpyAsync(d + n, prev, bytes, cudaMemcpyHostToDevice, st));
    TG_CUDA(cudaMemcpyAsync(d + 2 * n, upd, bytes, cudaMemcpyHostToDevice, st));
    TG_CUDA(launch_time_filter(which, d, d + n, dtsmooth, dtsmooth_div2, 1, (long)n, (long)n, d + 2 * n, d + 3 * n,
                               st));
    TG_CUDA(cudaMemcpyAsync(upd, d + 2 * n, bytes, cudaMemcpyDeviceToHost, st));
    TG_CUDA(cudaMemcpyAsync(nm_upd, d + 3 * n, bytes, cudaMemcpyDeviceToHost, st));
    TG_CUDA(cudaStreamSynchronize(st));
    return TG_OK;
}

static bool settei_fields_ok(const tg_settei_fields *F)
{
    const double *const *p = &F->tn;
    for (int i = 0; i < 32; ++i)
        if (!p[i]) return false;
    return true;
}

__attribute__((visibility("default"))) int tg_settei_ng_dev(const tg_settei_fields *F, const tg_settei_consts *C,
                                                            double *te_out, double *ti_out, double *qtotal, int nk,
                                                            int ncol, long ld, double *system_out, int *status_dev,
                                                            void *stream)
{
    if (!F || !C || !te_out || !ti_out || !qtotal || nk < 3 || ncol < 0 || ld < ncol || !settei_fields_ok(F)) {
        set_err("tg_settei_ng_dev: bad arguments (nk=%d ncol=%d ld=%ld)", nk, ncol, ld);
        return TG_EINVAL;
    }
    DevCtx *cx = nullptr;
    int rc = get_ctx(&cx);
    if (rc) return rc;
    std::lock_guard<std::mutex> lk(cx->mu);
    cudaStream_t st = (cudaStream_t)stream;
    StreamWs *ws = nullptr;
    if ((rc = stream_ws(cx, st, &ws))) return rc;
    if ((rc = grow(ws->scratch, sizeof(double) * settei_scratch_doubles(nk, ld > 0 ? ld : 1)))) return rc;
    TG_CUDA(cudaMemsetAsync(ws->flags, 0, sizeof(unsigned), st));
    TG_CUDA(launch_settei_ng(*F, *C, te_out, ti_out, qtotal, nk, ncol, ld, system_out, ws->flags, st,
                             (double *)ws->scratch.p));
    if (status_dev) {
        k_finish_status<<<1, 1, 0, st>>>(ws->flags, status_dev);
        TG_CUDA(cudaGetLastError());
    }
    return TG_OK;
}

__attribute__((visibility("default"))) int tg_settei_ng(const tg_settei_fields *F, const tg_settei_consts *C,
                                                        double *te_out, double *ti_out, double *qtotal, int nk,
                                                        int ncol)
{
    if (!F || !C || !te_out || !ti_out || !qtotal || nk < 3 || ncol < 0 || !settei_fields_ok(F)) {
        set_err("tg_settei_ng: bad arguments (nk=%d ncol=%d)", nk, ncol);
        return TG_EINVAL;
    }
    if (ncol == 0) return TG_OK;
    DevCtx *c = nullptr;
    int rc = get_ctx(&c);
    if (rc) return rc;
    std::lock_guard<std::mutex> lk(c->mu);
    TG_CUDA(cudaSetDevice(c->dev));
    const long ld = round_up(ncol, 32);
    const size_t lvl = (size_t)nk * ld, colsz = (size_t)nk * ncol;
    // 27 fields + qtotal + te_out + ti_out level-major; 5 2-D rows
    if ((rc = grow(c->lvlbuf[0][0], sizeof(double) * (30 * lvl + 5 * (size_t)ld)))) return rc;
    if ((rc = grow(c->colbuf[0][0], sizeof(double) * colsz))) return rc;
    double *base = (double *)c->lvlbuf[0][0].p, *stage = (double *)c->colbuf[0][0].p;
    cudaStream_t st = c->st[0];
    tg_settei_fields D;
    const double *const *src = &F->tn;
    const double **dst = &D.tn;
    for (int i = 0; i < 28; ++i) {
        const double *h = i < 27 ? src[i] : qtotal;
        double *d = base + i * lvl;
        TG_CUDA(cudaMemcpyAsync(stage, h, sizeof(double) * colsz, cudaMemcpyHostToDevice, st));
        TG_CUDA(launch_col_to_level(stage, nk, d, ld, nk, ncol, st));
        if (i < 27) dst[i] = d;
    }
    double *qt = base + 27 * lvl, *te_l = base + 28 * lvl, *ti_l = base + 29 * lvl, *two = base + 30 * lvl;
    for (int i = 0; i < 5; ++i) {
        TG_CUDA(cudaMemcpyAsync(two + i * ld, src[27 + i], sizeof(double) * ncol, cudaMemcpyHostToDevice, st));
        dst[27 + i] = two + i * ld;
    }
    TG_CUDA(cudaMemsetAsync(c->flags, 0, sizeof(unsigned), st));
    if ((rc = grow(c->scratch[0], sizeof(double) * settei_scratch_doubles(nk, ld)))) return rc;
    TG_CUDA(launch_settei_ng(D, *C, te_l, ti_l, qt, nk, ncol, ld, nullptr, c->flags, st, (double *)c->scratch[0].p));
    double *hout[3] = {te_out, ti_out, qtotal};
    double *dout[3] = {te_l, ti_l, qt};
    for (int i = 0; i < 3; ++i) {
        TG_CUDA(launch_level_to_col(dout[i], ld, stage, nk, nk, ncol, st));
        TG_CUDA(cudaMemcpyAsync(hout[i], stage, sizeof(double) * colsz, cudaMemcpyDeviceToHost, st));
        TG_CUDA(cudaStreamSynchronize(st));
    }
    TG_CUDA(cudaMemcpy(c->flags_host, c->flags, sizeof(unsigned), cudaMemcpyDeviceToHost));
    return flags_to_status(c->flags_host[0]);
}

static bool oplus_fields_ok(const tg_oplus_fields *F)
{
    const double *const *p = &F->tn;
    for (int i = 0; i < 37; ++i)
        if (!p[i]) return false;
    return true;
}

__attribute__((visibility("default"))) int tg_oplus_ng_dev(const tg_oplus_fields *F, const tg_oplus_consts *C,
                                                           double *opout, double *xiop2p, double *xiop2d, double *Fe,
                                                           double *Fn, int nk, int ncol, long ld, double *system_out,
                                                           int *status_dev, void *stream)
{
    if (!F || !C || !opout || !xiop2p || !xiop2d || (!Fe) != (!Fn) || nk < 3 || ncol < 0 || ld < ncol ||
        !oplus_fields_ok(F)) {
        set_err("tg_oplus_ng_dev: bad arguments (nk=%d ncol=%d ld=%ld)", nk, ncol, ld);
        return TG_EINVAL;
    }
    DevCtx *cx = nullptr;
    int rc = get_ctx(&cx);
    if (rc) return rc;
    std::lock_guard<std::mutex> lk(cx->mu);
    cudaStream_t st = (cudaStream_t)stream;
    StreamWs *ws = nullptr;
    if ((rc = stream_ws(cx, st, &ws))) return rc;
    const size_t sbytes = sizeof(double) * oplus_scratch_planes() * (size_t)nk * (size_t)(ld > 0 ? ld : 1);
    if ((rc = grow(ws->scratch, sbytes))) return rc;
    TG_CUDA(cudaMemsetAsync(ws->flags, 0, sizeof(unsigned), st));
    TG_CUDA(launch_oplus_ng(*F, *C, opout, xiop2p, xiop2d, Fe, Fn, (double *)ws->scratch.p, nk, ncol, ld,
                            system_out, ws->flags, st));
    if (status_dev) {
        k_finish_status<<<1, 1, 0, st>>>(ws->flags, status_dev);
        TG_CUDA(cudaGetLastError());
    }
    return TG_OK;
}

__attribute__((visibility("default"))) int tg_oplus_ng_post_dev(const tg_oplus_fields *F, const tg_oplus_consts *C,
                                                                double *opout, double *xiop2p, double *xiop2d,
                                                                double *Fe, double *Fn, int nk, int ncol, long ld,
                                                                const tg_post_step *P, int *status_dev, void *stream)
{
    if (!F || !C || !opout || !xiop2p || !xiop2d || (!Fe) != (!Fn) || nk < 3 || ncol < 0 || ld < ncol ||
        !oplus_fields_ok(F) || !post_ok("tg_oplus_ng_post_dev", P)) {
        if (!P || P->cur) set_err("tg_oplus_ng_post_dev: bad arguments (nk=%d ncol=%d ld=%ld)", nk, ncol, ld);
        return TG_EINVAL;
    }
    DevCtx *cx = nullptr;
    int rc = get_ctx(&cx);
    if (rc) return rc;
    std::lock_guard<std::mutex> lk(cx->mu);
    cudaStream_t st = (cudaStream_t)stream;
    StreamWs *ws = nullptr;
    if ((rc = stream_ws(cx, st, &ws))) return rc;
    const size_t sbytes = sizeof(double) * oplus_scratch_planes() * (size_t)nk * (size_t)(ld > 0 ? ld : 1);
    if ((rc = grow(ws->scratch, sbytes))) return rc;
    const PostStep post = post_of(P, 0.0, 1);
    TG_CUDA(cudaMemsetAsync(ws->flags, 0, sizeof(unsigned), st));
    TG_CUDA(launch_oplus_ng(*F, *C, opout, xiop2p, xiop2d, Fe, Fn, (double *)ws->scratch.p, nk, ncol, ld, nullptr,
                            ws->flags, st, &post));
    if (status_dev) {
        k_finish_status<<<1, 1, 0, st>>>(ws->flags, status_dev);
        TG_CUDA(cudaGetLastError());
    }
    return TG_OK;
}

__attribute__((visibility("default"))) long tg_oplus_ng_factor_doubles(int nk, long ld)
{
    return nk < 3 || ld < 1 ? 0 : (long)oplus_scratch_planes() * nk * ld;
}

__attribute__((visibility("default"))) int tg_oplus_ng_factor_dev(const tg_oplus_fields *F, const tg_oplus_consts *C,
                                                                  double *xiop2p, double *xiop2d, double *factor,
                                                                  int nk, int ncol, long ld, int *status_dev,
                                                                  void *stream)
{
    if (!F || !C || !xiop2p || !xiop2d || !factor || nk < 3 || ncol < 0 || ld < ncol || !oplus_fields_ok(F)) {
        set_err("tg_oplus_ng_factor_dev: bad arguments (nk=%d ncol=%d ld=%ld)", nk, ncol, ld);
        return TG_EINVAL;
    }
    DevCtx *cx = nullptr;
    int rc = get_ctx(&cx);
    if (rc) return rc;
    std::lock_guard<std::mutex> lk(cx->mu);
    cudaStream_t st = (cudaStream_t)stream;
    StreamWs *ws = nullptr;
    if ((rc = stream_ws(cx, st, &ws))) return rc;
    TG_CUDA(cudaMemsetAsync(ws->flags, 0, sizeof(unsigned), st));
    TG_CUDA(launch_oplus_factor(*F, *C, xiop2p, xiop2d, factor, nk, ncol, ld, ws->flags, st));
    if (status_dev) {
        k_finish_status<<<1, 1, 0, st>>>(ws->flags, status_dev);
        TG_CUDA(cudaGetLastError());
    }
    return TG_OK;
}

__attribute__((visibility("default"))) int tg_oplus_ng_solve_dev(const tg_oplus_fields *F, const tg_oplus_consts *C,
                                                                 const double *factor, double *opout, int nk,
                                                                 int ncol, long ld, const tg_post_step *P,
                                                                 int *status_dev, void *stream)
{
    if (!F || !C || !factor || !opout || nk < 3 || ncol < 0 || ld < ncol || !oplus_fields_ok(F) ||
        (P && !post_ok("tg_oplus_ng_solve_dev", P))) {
        if (!P || P->cur) set_err("tg_oplus_ng_solve_dev: bad arguments (nk=%d ncol=%d ld=%ld)", nk, ncol, ld);
        return TG_EINVAL;
    }
    DevCtx *cx = nullptr;
    int rc = get_ctx(&cx);
    if (rc) return rc;
    std::lock_guard<std::mutex> lk(cx->mu);
    cudaStream_t st = (cudaStream_t)stream;
    StreamWs *ws = nullptr;
    if ((rc = stream_ws(cx, st, &ws))) return rc;
    TG_CUDA(cudaMemsetAsync(ws->flags, 0, sizeof(unsigned), st));
    if (P) {
        const PostStep post = post_of(P, 0.0, 1);
        TG_CUDA(launch_oplus_solve(*F, *C, factor, opout, nk, ncol, ld, ws->flags, st, &post));
    } else {
        TG_CUDA(launch_oplus_solve(*F, *C, factor, opout, nk, ncol, ld, ws->flags, st, nullptr));
    }
    if (status_dev) {
        k_finish_status<<<1, 1, 0, st>>>(ws->flags, status_dev);
        TG_CUDA(cudaGetLastError());
    }
    return TG_OK;
}

__attribute__((visibility("default"))) int tg_oplus_diag_ng_dev(const tg_oplus_fields *F, const tg_oplus_consts *C,
                                                                const double *opout, const double *diffexp,
                                                                const double *vdotn_h, const double *bdotdh_bvel,
                                                                double *diag, int nk, int ncol, long ld, void *stream)
{
    if (!F || !C || !opout || !diag || nk < 3 || ncol < 0 || ld < ncol || !oplus_fields_ok(F)) {
        set_err("tg_oplus_diag_ng_dev: bad arguments (nk=%d ncol=%d ld=%ld)", nk, ncol, ld);
        return TG_EINVAL;
    }
    DevCtx *cx = nullptr;
    int rc = get_ctx(&cx);
    if (rc) return rc;
    std::lock_guard<std::mutex> lk(cx->mu);
    cudaStream_t st = (cudaStream_t)stream;
    StreamWs *ws = nullptr;
    if ((rc = stream_ws(cx, st, &ws))) return rc;
    const size_t sbytes = sizeof(double) * oplus_scratch_planes() * (size_t)nk * (size_t)(ld > 0 ? ld : 1);
    if ((rc = grow(ws->scratch, sbytes))) return rc;
    TG_CUDA(launch_oplus_diag_ng(*F, *C, opout, diffexp, vdotn_h, bdotdh_bvel, nk, ncol, ld, diag,
                                 (double *)ws->scratch.p, st));
    return TG_OK;
}

__attribute__((visibility("default"))) int tg_oplus_diag_ng(const tg_oplus_fields *F, const tg_oplus_consts *C,
                                                            const double *opout, const double *diffexp,
                                                            const double *vdotn_h, const double *bdotdh_bvel,
                                                            double *diag, int nk, int ncol)
{
    if (!F || !C || !opout || !diag || nk < 3 || ncol < 0 || !oplus_fields_ok(F)) {
        set_err("tg_oplus_diag_ng: bad arguments (nk=%d ncol=%d)", nk, ncol);
        return TG_EINVAL;
    }
    if (ncol == 0) return TG_OK;
    DevCtx *c = nullptr;
    int rc = get_ctx(&c);
    if (rc) return rc;
    std::lock_guard<std::mutex> lk(c->mu);
    TG_CUDA(cudaSetDevice(c->dev));
    const long ld = round_up(ncol, 32);
    Upload u{nullptr, nullptr, ld, (size_t)nk * ld, (size_t)nk * ncol, c->st[0]};
    // 27 fields, the solution and 3 horizontal terms, then 6 diagnostic planes, 9 rows, zpint
    if ((rc = grow(c->lvlbuf[0][0], sizeof(double) * (37 * u.lvl + 9 * (size_t)ld + (size_t)nk)))) return rc;
    if ((rc = grow(c->colbuf[0][0], sizeof(double) * u.colsz))) return rc;
    if ((rc = grow(c->scratch[0], sizeof(double) * oplus_scratch_planes() * u.lvl))) return rc;
    u.base = (double *)c->lvlbuf[0][0].p;
    u.stage = (double *)c->colbuf[0][0].p;
    tg_oplus_fields D;
    const double *const *src = &F->tn;
    const double **dst = &D.tn;
    for (int i = 0; i < 27; ++i)
        if ((rc = upload3(u, nk, ncol, src[i], i, &dst[i]))) return rc;
    const double *x = nullptr, *h[3] = {nullptr, nullptr, nullptr};
    if ((rc = upload3(u, nk, ncol, opout, 27, &x))) return rc;
    const double *hin[3] = {diffexp, vdotn_h, bdotdh_bvel};
    for (int i = 0; i < 3; ++i)
        if (hin[i] && (rc = upload3(u, nk, ncol, hin[i], 28 + i, &h[i]))) return rc;
    double *planes = u.base + 31 * u.lvl, *two = u.base + 37 * u.lvl, *zp = two + 9 * ld;
    for (int i = 0; i < 9; ++i) {
        TG_CUDA(cudaMemcpyAsync(two + i * ld, src[27 + i], sizeof(double) * ncol, cudaMemcpyHostToDevice, u.st));
        dst[27 + i] = two + i * ld;
    }
    TG_CUDA(cudaMemcpyAsync(zp, F->zpint, sizeof(double) * nk, cudaMemcpyHostToDevice, u.st));
    D.zpint = zp;
    TG_CUDA(launch_oplus_diag_ng(D, *C, x, h[0], h[1], h[2], nk, ncol, ld, planes, (double *)c->scratch[0].p, u.st));
    return download3(u, nk, ncol, planes, 6, diag);
}

__attribute__((visibility("default"))) int tg_oplus_ng(const tg_oplus_fields *F, const tg_oplus_consts *C,
                                                       double *opout, double *xiop2p, double *xiop2d, double *Fe,
                                                       double *Fn, int nk, int ncol)
{
    if (!F || !C || !opout || !xiop2p || !xiop2d || (!Fe) != (!Fn) || nk < 3 || ncol < 0 || !oplus_fields_ok(F)) {
        set_err("tg_oplus_ng: bad arguments (nk=%d ncol=%d)", nk, ncol);
        return TG_EINVAL;
    }
    if (ncol == 0) return TG_OK;
    DevCtx *c = nullptr;
    int rc = get_ctx(&c);
    if (rc) return rc;
    std::lock_guard<std::mutex> lk(c->mu);
    TG_CUDA(cudaSetDevice(c->dev));
    const long ld = round_up(ncol, 32);
    const size_t lvl = (size_t)nk * ld, colsz = (size_t)nk * ncol;
    const int nout = Fe ? 5 : 3;
    // 27 fields + outputs level-major; 9 2-D rows; zpint
    if ((rc = grow(c->lvlbuf[0][0], sizeof(double) * ((27 + nout) * lvl + 9 * (size_t)ld + (size_t)nk)))) return rc;
    if ((rc = grow(c->colbuf[0][0], sizeof(double) * colsz))) return rc;
    if ((rc = grow(c->scratch[0], sizeof(double) * oplus_scratch_planes() * lvl))) return rc;
    double *base = (double *)c->lvlbuf[0][0].p, *stage = (double *)c->colbuf[0][0].p;
    cudaStream_t st = c->st[0];
    tg_oplus_fields D;
    const double *const *src = &F->tn;
    const double **dst = &D.tn;
    for (int i = 0; i < 27; ++i) {
        double *d = base + i * lvl;
        TG_CUDA(cudaMemcpyAsync(stage, src[i], sizeof(double) * colsz, cudaMemcpyHostToDevice, st));
        TG_CUDA(launch_col_to_level(stage, nk, d, ld, nk, ncol, st));
        dst[i] = d;
    }
    double *outs = base + 27 * lvl, *two = outs + nout * lvl, *zp = two + 9 * ld;
    for (int i = 0; i < 9; ++i) {
        TG_CUDA(cudaMemcpyAsync(two + i * ld, src[27 + i], sizeof(double) * ncol, cudaMemcpyHostToDevice, st));
        dst[27 + i] = two + i * ld;
    }
    TG_CUDA(cudaMemcpyAsync(zp, F->zpint, sizeof(double) * nk, cudaMemcpyHostToDevice, st));
    D.zpint = zp;
    double *dout[5];
    for (int i = 0; i < nout; ++i) dout[i] = outs + i * lvl;
    TG_CUDA(cudaMemsetAsync(c->flags, 0, sizeof(unsigned), st));
    TG_CUDA(launch_oplus_ng(D, *C, dout[0], dout[1], dout[2], Fe ? dout[3] : nullptr, Fe ? dout[4] : nullptr,
                            (double *)c->scratch[0].p, nk, ncol, ld, nullptr, c->flags, st));
    double *hout[5] = {opout, xiop2p, xiop2d, Fe, Fn};
    for (int i = 0; i < nout; ++i) {
        TG_CUDA(launch_level_to_col(dout[i], ld, stage, nk, nk, ncol, st));
        TG_CUDA(cudaMemcpyAsync(hout[i], stage, sizeof(double) * colsz, cudaMemcpyDeviceToHost, st));
        TG_CUDA(cudaStreamSynchronize(st));
    }
    TG_CUDA(cudaMemcpy(c->flags_host, c->flags, sizeof(unsigned), cudaMemcpyDeviceToHost));
    return flags_to_status(c->flags_host[0]);
}

__attribute__((visibility("default"))) int tg_trsolv_dev(const double *a, const double *b, const double *c,
                                                         const double *f, double *x, int nk, int k2, int ncol,
                                                         int layout, long ld, int precision, int *status_dev,
                                                         void *stream)
{
    return dev_solve(TG_KIND_SCALAR, a, b, c, f, nullptr, nullptr, x, nk, k2, ncol, layout, ld, precision,
                     status_dev, stream);
}

__attribute__((visibility("default"))) int tg_blksolve_dev(int B, const double *P, const double *Q,
                                                           const double *R, const double *f,
                                                           const double *ubc_ratio, const double *ubc_add,
                                                           double *u, int nk, int k2, int ncol, int layout,
                                                           long ld, int precision, int *status_dev, void *stream)
{
    if (B != 2 && B != 3) {
        set_err("tg_blksolve_dev: B must be 2 or 3");
        return TG_EINVAL;
    }
    return dev_solve(B, P, Q, R, f, ubc_ratio, ubc_add, u, nk, k2, ncol, layout, ld, precision, status_dev,
                     stream);
}

}  // extern "C"

// ===========================================================================
// Plans
// ===========================================================================
struct tg_plan {
    int dev = 0;
    int precision = 0;
    int nseg = 0;
    struct Group {
        int kind = 0;
        int nseg = 0;
        int ntiles = 0;
        int k2max = 0;
        Seg *d_segs = nullptr;
        Shape shape{};
        void *scratch = nullptr;
    } groups[3];
    unsigned *d_flags = nullptr;
    int *d_status = nullptr;
    unsigned long long *d_hist = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    cudaStream_t graph_stream = nullptr;
    cudaStream_t side = nullptr;            // block kinds run here, beside the scalar kind
    cudaEvent_t fork = nullptr, join = nullptr;
    int launches = 0;
    bool side_by_side = false;              // block kinds on `side` beside the scalar kind
};

namespace {
int plan_launch_group(tg_plan *p, tg_plan::Group &g, cudaStream_t st)
{
    SegTable tab{};
    tab.segs = g.d_segs;
    tab.nseg = g.nseg;
    tab.ntiles = g.ntiles;
    tab.k2max = g.k2max;
    if (g.kind == TG_KIND_SCALAR)
        TG_CUDA(launch_scalar(tab, p->precision, g.shape, g_refine, (double *)g.scratch, p->d_flags, p->d_hist, st));
    else
        TG_CUDA(launch_block(tab, g.kind, p->precision, g.shape, g_refine, (double *)g.scratch, p->d_flags, p->d_hist,
                             st));
    return TG_OK;
}

// When every kind's tiles fit in one resident wave the kernels are latency-
// bound (few columns, long per-level dependency chains), so the block groups
// run on a side stream forked from st and joined back: in a captured graph
// they are parallel branches and the kernels share the GPU.  Larger batches
// run the kinds one after the other: each kind's grid is sized so that its
// sweep scratch fits in L2, and two such grids side by side would not.
int plan_enqueue(tg_plan *p, cudaStream_t st)
{
    TG_CUDA(cudaMemsetAsync(p->d_flags, 0, sizeof(unsigned) * p->nseg, st));
    if (p->precision != TG_PREC_F64)
        TG_CUDA(cudaMemsetAsync(p->d_hist, 0, kMaxSweepBins * sizeof(unsigned long long), st));
    int rc;
    if (!p->side_by_side) {
        for (auto &g : p->groups)
            if (g.nseg > 0 && (rc = plan_launch_group(p, g, st))) return rc;
        return TG_OK;
    }
    TG_CUDA(cudaEventRecord(p->fork, st));
    TG_CUDA(cudaStreamWaitEvent(p->side, p->fork, 0));
    for (int gi = 1; gi < 3; ++gi)
        if (p->groups[gi].nseg > 0 && (rc = plan_launch_group(p, p->groups[gi], p->side))) return rc;
    if ((rc = plan_launch_group(p, p->groups[0], st))) return rc;
    TG_CUDA(cudaEventRecord(p->join, p->side));
    TG_CUDA(cudaStreamWaitEvent(st, p->join, 0));
    return TG_OK;
}

void plan_free(tg_plan *p)
{
    if (!p) return;
    if (p->exec) cudaGraphExecDestroy(p->exec);
    if (p->graph) cudaGraphDestroy(p->graph);
    for (auto &g : p->groups) {
        if (g.d_segs) cudaFree(g.d_segs);
        if (g.scratch) cudaFree(g.scratch);
    }
    if (p->d_flags) cudaFree(p->d_flags);
    if (p->d_status) cudaFree(p->d_status);
    if (p->d_hist) cudaFree(p->d_hist);
    if (p->fork) cudaEventDestroy(p->fork);
    if (p->join) cudaEventDestroy(p->join);
    if (p->side) cudaStreamDestroy(p->side);
    delete p;
}
}  // namespace

extern "C" {

__attribute__((visibility("default"))) int tg_plan_create(const tg_segment *segs, int nseg, int precision,
                                                          tg_plan **out)
{
    if (!out || (!segs && nseg > 0) || nseg < 0 || bad_prec(precision)) {
        set_err("tg_plan_create: bad arguments");
        return TG_EINVAL;
    }
    *out = nullptr;
    for (int i = 0; i < nseg; ++i) {
        const tg_segment &s = segs[i];
        const bool blk = s.kind == TG_KIND_BLOCK2 || s.kind == TG_KIND_BLOCK3;
        if ((s.kind != TG_KIND_SCALAR && !blk) || s.nk < 1 || s.k2 < 1 || s.k2 > s.nk || s.ncol < 0 ||
            s.ld < s.ncol || !s.a || !s.b || !s.c || !s.f || !s.x || (blk && s.ubc_ratio && s.k2 >= s.nk)) {
            set_err("tg_plan_create: segment %d invalid", i);
            return TG_EINVAL;
        }
    }
    DevCtx *cx = nullptr;
    int rc = get_ctx(&cx);
    if (rc) return rc;
    tg_plan *p = new (std::nothrow) tg_plan;
    if (!p) return TG_ENOMEM;
    p->dev = cx->dev;
    p->precision = precision;
    p->nseg = nseg;
    const int kinds[3] = {TG_KIND_SCALAR, TG_KIND_BLOCK2, TG_KIND_BLOCK3};
    for (int gi = 0; gi < 3; ++gi) {
        auto &g = p->groups[gi];
        g.kind = kinds[gi];
        std::vector<Seg> hs;
        bool ring_ok = true, cpt2_ok = true;
        for (int i = 0; i < nseg; ++i) {
            const tg_segment &s = segs[i];
            if (s.kind != g.kind || s.ncol == 0) continue;
            Seg d{};
            d.a = s.a; d.b = s.b; d.c = s.c; d.f = s.f; d.x = s.x;
            d.ubc_ratio = g.kind == TG_KIND_SCALAR ? nullptr : s.ubc_ratio;
            d.ubc_add = d.ubc_ratio ? s.ubc_add : nullptr;
            d.ld = s.ld; d.nk = s.nk; d.k2 = s.k2; d.ncol = s.ncol; d.kind = s.kind;
            d.status_idx = i;
            ring_ok = ring_ok && ring_ok_for(d, precision);
            cpt2_ok = cpt2_ok && cpt2_ok_seg(d);
            hs.push_back(d);
            g.k2max = std::max(g.k2max, s.k2);
        }
        if (hs.empty()) continue;
        int cpb = 0, cpt = 1, stages = 0, w2g = 0;
        tile_for(g.kind, precision, ring_ok, &cpb, &cpt, &stages, &w2g);
        if (cpt == 2 && !cpt2_ok) {
            cpb /= 2;
            cpt = 1;
        }
        long tiles = 0;
        for (auto &d : hs) {
            d.tile0 = (int)tiles;
            tiles += (d.ncol + cpb - 1) / cpb;
        }
        if (tiles > 0x7fffffffL) {
            plan_free(p);
            set_err("tg_plan_create: too many tiles");
            return TG_EINVAL;
        }
        g.nseg = (int)hs.size();
        g.ntiles = (int)tiles;
        cudaError_t e = plan_shape(g.kind, precision, g.k2max, g.ntiles, cpb, cpt, stages, w2g, &g.shape);
        if (e != cudaSuccess) {
            plan_free(p);
            set_err("tg_plan_create: no launch shape: %s", cudaGetErrorString(e));
            return TG_EINVAL;
        }
        if (cudaMalloc(&g.d_segs, sizeof(Seg) * hs.size()) != cudaSuccess ||
            cudaMemcpy(g.d_segs, hs.data(), sizeof(Seg) * hs.size(), cudaMemcpyHostToDevice) != cudaSuccess) {
            cudaGetLastError();
            plan_free(p);
            set_err("tg_plan_create: segment table upload failed");
            return TG_ENOMEM;
        }
        p->launches += 1;
    }
    // Kinds side by side (the latency-bound regime, every kind in one wave):
    // the FP64 scalar grid is halved, each warp taking two tiles.  The scalar kind
    // then still finishes inside the block kinds' time, and the block warps,
    // the long pole, get more of the SMs' issue slots (2.5 deg grid, 10368
    // columns: 84 -> 78 us).  Decided here, with the overlap setting of the
    // plan's creation.
    {
        auto &g0 = p->groups[0];
        bool split = g0.nseg > 0 && (p->groups[1].nseg > 0 || p->groups[2].nseg > 0);
        const int overlap = kind_overlap();
        if (overlap == 0) split = false;
        if (overlap < 0)
            for (const auto &g : p->groups)
                if (g.nseg > 0 && !g.shape.one_wave) split = false;
        p->side_by_side = split;
        if (split && precision == TG_PREC_F64 && g0.shape.stages > 0 && g0.shape.blocks > 1)
            g0.shape.blocks = (g0.shape.blocks + 1) / 2;
    }
    for (auto &g : p->groups) {
        if (!g.nseg) continue;
        const bool ring_refine = g.kind == TG_KIND_SCALAR && precision != TG_PREC_F64 && g.shape.stages > 0;
        if (g.kind != TG_KIND_SCALAR || g.shape.w2g || ring_refine) {
            const long slots = (long)g.shape.blocks * g.shape.threads;
            const size_t need = ring_refine ? refine_scratch_bytes(slots, g.k2max)
                                : g.kind == TG_KIND_SCALAR ? scalar_scratch_bytes(slots, g.k2max)
                                                           : block_scratch_bytes(g.kind, precision, slots, g.k2max);
            if (cudaMalloc(&g.scratch, need) != cudaSuccess) {
                cudaGetLastError();
                plan_free(p);
                set_err("tg_plan_create: scratch allocation failed");
                return TG_ENOMEM;
            }
        }
    }
    if (cudaStreamCreateWithFlags(&p->side, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&p->fork, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&p->join, cudaEventDisableTiming) != cudaSuccess ||
        cudaMalloc(&p->d_flags, sizeof(unsigned) * std::max(nseg, 1)) != cudaSuccess ||
        cudaMalloc(&p->d_status, sizeof(int) * std::max(nseg, 1)) != cudaSuccess ||
        cudaMalloc(&p->d_hist, kMaxSweepBins * sizeof(unsigned long long)) != cudaSuccess ||
        cudaMemset(p->d_flags, 0, sizeof(unsigned) * std::max(nseg, 1)) != cudaSuccess ||
        cudaMemset(p->d_hist, 0, kMaxSweepBins * sizeof(unsigned long long)) != cudaSuccess) {
        cudaGetLastError();
        plan_free(p);
        set_err("tg_plan_create: allocation failed");
        return TG_ENOMEM;
    }
    *out = p;
    return TG_OK;
}

__attribute__((visibility("default"))) int tg_plan_execute(tg_plan *p, void *stream)
{
    if (!p) {
        set_err("tg_plan_execute: null plan");
        return TG_EINVAL;
    }
    cudaStream_t st = (cudaStream_t)stream;
    if (p->exec) {
        TG_CUDA(cudaGraphLaunch(p->exec, st));
        return TG_OK;
    }
    return plan_enqueue(p, st);
}

__attribute__((visibility("default"))) int tg_plan_capture_graph(tg_plan *p, void *stream)
{
    if (!p || !stream) {
        set_err("tg_plan_capture_graph: needs a plan and a non-default stream");
        return TG_EINVAL;
    }
    cudaStream_t st = (cudaStream_t)stream;
    if (p->exec) {
        cudaGraphExecDestroy(p->exec);
        p->exec = nullptr;
    }
    if (p->graph) {
        cudaGraphDestroy(p->graph);
        p->graph = nullptr;
    }
    TG_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    int rc = plan_enqueue(p, st);
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamEndCapture(st, &g);
    if (rc) {
        if (g) cudaGraphDestroy(g);
        return rc;
    }
    if (e != cudaSuccess) {
        set_err("graph capture failed: %s", cudaGetErrorString(e));
        return TG_ECUDA;
    }
    p->graph = g;
    TG_CUDA(cudaGraphInstantiate(&p->exec, g, 0));
    p->graph_stream = st;
    return TG_OK;
}

__attribute__((visibility("default"))) int tg_plan_status(tg_plan *p, int *per_segment_status)
{
    if (!p) {
        set_err("tg_plan_status: null plan");
        return TG_EINVAL;
    }
    TG_CUDA(cudaDeviceSynchronize());
    std::vector<unsigned> f(std::max(p->nseg, 1));
    TG_CUDA(cudaMemcpy(f.data(), p->d_flags, sizeof(unsigned) * p->nseg, cudaMemcpyDeviceToHost));
    unsigned all = 0;
    for (int i = 0; i < p->nseg; ++i) {
        if (per_segment_status) per_segment_status[i] = flags_to_status(f[i]);
        all |= f[i];
    }
    return flags_to_status(all);
}

__attribute__((visibility("default"))) int tg_plan_launches(const tg_plan *p) { return p ? p->launches : 0; }

__attribute__((visibility("default"))) int tg_selftest_wait(unsigned polls, int *status_dev, void *stream)
{
    if (!status_dev || polls < 1 || polls > (1u << 22)) {
        set_err("tg_selftest_wait: bad arguments (polls=%u)", polls);
        return TG_EINVAL;
    }
    DevCtx *cx = nullptr;
    int rc = get_ctx(&cx);
    if (rc) return rc;
    std::lock_guard<std::mutex> lk(cx->mu);
    cudaStream_t st = (cudaStream_t)stream;
    StreamWs *ws = nullptr;
    if ((rc = stream_ws(cx, st, &ws))) return rc;
    TG_CUDA(cudaMemsetAsync(ws->flags, 0, sizeof(unsigned), st));
    TG_CUDA(launch_selftest_wait(polls, ws->flags, st));
    k_finish_status<<<1, 1, 0, st>>>(ws->flags, status_dev);
    TG_CUDA(cudaGetLastError());
    return TG_OK;
}

__attribute__((visibility("default"))) int tg_selftest_walk(int which, double *buf, int nk, int K, int top, int ncol,
                                                            long ld, int *status_dev, void *stream)
{
    if (!buf || !status_dev || (which != 0 && which != 1) || nk < 1 || ncol < 0 || ld < ncol ||
        (which == 1 && nk < 3)) {
        set_err("tg_selftest_walk: bad arguments (which=%d nk=%d ncol=%d ld=%ld)", which, nk, ncol, ld);
        return TG_EINVAL;
    }
    DevCtx *cx = nullptr;
    int rc = get_ctx(&cx);
    if (rc) return rc;
    std::lock_guard<std::mutex> lk(cx->mu);
    cudaStream_t st = (cudaStream_t)stream;
    StreamWs *ws = nullptr;
    if ((rc = stream_ws(cx, st, &ws))) return rc;
    TG_CUDA(cudaMemsetAsync(ws->flags, 0, sizeof(unsigned), st));
    const long slab = (long)nk * ld;
    cudaError_t e = which == 0 ? launch_thomas_post(buf, buf + slab, buf + 2 * slab, buf + 3 * slab, buf + 4 * slab,
                                                    nk, K, top, ncol, ld, ws->flags, nullptr, st)
                               : launch_oplus_factor_pass(buf, nk, ncol, ld, ws->flags, st);
    if (e == cudaErrorInvalidValue) {
        set_err("tg_selftest_walk: unsupported rows (K=%d top=%d nk=%d)", K, top, nk);
        return TG_EINVAL;
    }
    TG_CUDA(e);
    k_finish_status<<<1, 1, 0, st>>>(ws->flags, status_dev);
    TG_CUDA(cudaGetLastError());
    return TG_OK;
}

__attribute__((visibility("default"))) int tg_set_block_rows(int kind, int on)
{
    if (kind != TG_KIND_BLOCK2 && kind != TG_KIND_BLOCK3) {
        set_err("tg_set_block_rows: kind must be TG_KIND_BLOCK2 or TG_KIND_BLOCK3");
        return TG_EINVAL;
    }
    tg::set_block_rows(kind, on);
    return TG_OK;
}

__attribute__((visibility("default"))) int tg_set_block_width(int kind, int width)
{
    if (kind != TG_KIND_BLOCK2 && kind != TG_KIND_BLOCK3) {
        set_err("tg_set_block_width: kind must be TG_KIND_BLOCK2 or TG_KIND_BLOCK3");
        return TG_EINVAL;
    }
    tg::set_block_width(kind, width);
    return TG_OK;
}

__attribute__((visibility("default"))) int tg_set_stage_levels(int kind, int precision, int levels)
{
    if (kind != TG_KIND_SCALAR || precision != TG_PREC_F64) {
        set_err("tg_set_stage_levels: applies to TG_KIND_SCALAR, TG_PREC_F64");
        return TG_EINVAL;
    }
    tg::set_stage_levels(kind, precision, levels);
    return TG_OK;
}

__attribute__((visibility("default"))) int tg_set_column_residency(int kind, int precision, int mode)
{
    if ((kind != TG_KIND_SCALAR && kind != TG_KIND_BLOCK2 && kind != TG_KIND_BLOCK3) || bad_prec(precision) ||
        (precision != TG_PREC_F64 && kind != TG_KIND_SCALAR) || mode > 2) {
        set_err("tg_set_column_residency: FP64 kinds or the scalar refinement, mode 0, 1, 2 or -1");
        return TG_EINVAL;
    }
    tg::set_column_residency(kind, precision, mode);
    return TG_OK;
}

__attribute__((visibility("default"))) int tg_set_scalar_scratch_budget(double megabytes)
{
    tg::set_scalar_scratch_budget(megabytes);
    return TG_OK;
}

__attribute__((visibility("default"))) int tg_set_kind_overlap(int mode)
{
    tg::set_kind_overlap(mode);
    return TG_OK;
}

__attribute__((visibility("default"))) int tg_set_host_pipeline(int chunk_kb, int streams)
{
    if (streams > kSlots) {
        set_err("tg_set_host_pipeline: at most %d streams", kSlots);
        return TG_EINVAL;
    }
    g_host_chunk_bytes.store(chunk_kb > 0 ? (long)chunk_kb << 10 : 0);
    g_host_slots.store(streams > 0 ? streams : kHostSlotsDefault);
    return TG_OK;
}

__attribute__((visibility("default"))) int tg_set_block_scratch_budget(double megabytes)
{
    tg::set_block_scratch_budget(megabytes);
    return TG_OK;
}

__attribute__((visibility("default"))) int tg_set_assembly_mode(int mode)
{
    if (mode < -1 || mode > 2) {
        set_err("tg_set_assembly_mode: mode must be 0, 1, 2 or -1");
        return TG_EINVAL;
    }
    tg::set_assembly_mode(mode);
    return TG_OK;
}

__attribute__((visibility("default"))) int tg_set_walk_prefetch(int levels)
{
    if (levels < -1 || levels == 0 || levels > 32) {
        set_err("tg_set_walk_prefetch: levels must be 1..32 or -1");
        return TG_EINVAL;
    }
    tg::set_walk_prefetch(levels);
    return TG_OK;
}

__attribute__((visibility("default"))) int tg_set_cache_hints(int on)
{
    tg::set_cache_hints(on);
    return TG_OK;
}

__attribute__((visibility("default"))) int tg_plan_describe(const tg_plan *p, char *buf, int n)
{
    if (!p || !buf || n < 1) {
        set_err("tg_plan_describe: bad arguments");
        return TG_EINVAL;
    }
    std::string out;
    const bool f64 = p->precision == TG_PREC_F64;
    for (const tg_plan::Group &g : p->groups) {
        if (!g.nseg) continue;
        const Shape &h = g.shape;
        char name[96];
        if (g.kind == TG_KIND_SCALAR) {
            if (!f64 && h.res == 3) snprintf(name, sizeof name, "k_scalar_refine_tile");
            else if (!f64 && h.stages) snprintf(name, sizeof name, "k_scalar_refine_ring<%d>", h.stages);
            else if (!f64) snprintf(name, sizeof name, "k_scalar_refine<%d>", h.pf);
            else if (h.stages && h.res) snprintf(name, sizeof name, "k_scalar_f64_res<%d,%d,%d>", h.stages, h.lps, h.res == 2);
            else if (h.stages && h.lps > 1) snprintf(name, sizeof name, "k_scalar_f64_chunk<%d,%d>", h.stages, h.lps);
            else if (h.stages) snprintf(name, sizeof name, "k_scalar_f64_ring<%d,%d>", h.stages, h.w2g);
            else if (h.w2g) snprintf(name, sizeof name, "k_scalar_f64_g<%d>", h.pf);
            else snprintf(name, sizeof name, "k_scalar_f64<%d,%d>", h.cpt, h.pf);
        } else {
            if (!f64 && h.stages) snprintf(name, sizeof name, "k_block_refine_ring<%d,%d>", g.kind, h.stages);
            else if (!f64) snprintf(name, sizeof name, "k_block_refine<%d>", g.kind);
            else if (h.stages && h.rows) snprintf(name, sizeof name, "k_block_f64_rows<%d,%d>", g.kind, h.stages);
            else if (h.stages && h.res) snprintf(name, sizeof name, "k_block_f64_ring<%d,%d,%d,1>", g.kind, h.stages, h.bw);
            else if (h.stages) snprintf(name, sizeof name, "k_block_f64_ring<%d,%d,%d>", g.kind, h.stages, h.bw);
            else snprintf(name, sizeof name, "k_block_f64<%d>", g.kind);
        }
        char line[256];
        snprintf(line, sizeof line, "%s%s kind=%d threads=%d blocks=%d smem=%zu tiles=%d k2max=%d",
                 out.empty() ? "" : "; ", name, g.kind, h.threads, h.blocks, h.smem, g.ntiles, g.k2max);
        out += line;
    }
    snprintf(buf, (size_t)n, "%s", out.c_str());
    return (int)out.size() < n ? TG_OK : TG_EINVAL;
}

__attribute__((visibility("default"))) int tg_plan_sweep_histogram(tg_plan *p, long *hist, int nbins)
{
    if (!p || !hist || nbins < 1) {
        set_err("tg_plan_sweep_histogram: bad arguments");
        return TG_EINVAL;
    }
    unsigned long long h[kMaxSweepBins];
    if (cudaDeviceSynchronize() != cudaSuccess ||
        cudaMemcpy(h, p->d_hist, sizeof h, cudaMemcpyDeviceToHost) != cudaSuccess) {
        set_err("tg_plan_sweep_histogram: copy failed");
        return -TG_ECUDA;
    }
    const int n = std::min(nbins, kMaxSweepBins);
    for (int i = 0; i < n; ++i) hist[i] = (long)h[i];
    for (int i = n; i < kMaxSweepBins; ++i) hist[n - 1] += (long)h[i];
    return n;
}

__attribute__((visibility("default"))) int tg_plan_destroy(tg_plan *p)
{
    if (!p) return TG_OK;
    cudaDeviceSynchronize();
    plan_free(p);
    return TG_OK;
}

__attribute__((visibility("default"))) int tg_release_buffers(void)
{
    std::lock_guard<std::mutex> lk(g_ctx_mu);
    for (int d = 0; d < kMaxDev; ++d) {
        DevCtx *c = g_ctx[d];
        if (!c) continue;
        std::lock_guard<std::mutex> lk2(c->mu);
        int cur = 0;
        cudaGetDevice(&cur);
        cudaSetDevice(d);
        cudaDeviceSynchronize();
        for (int s = 0; s < kSlots; ++s) {
            for (auto &b : c->colbuf[s])
                if (b.p) cudaFree(b.p);
            for (auto &b : c->lvlbuf[s])
                if (b.p) cudaFree(b.p);
            if (c->scratch[s].p) cudaFree(c->scratch[s].p);
            if (c->span[s].p) cudaFree(c->span[s].p);
            if (c->st[s]) cudaStreamDestroy(c->st[s]);
        }
        for (StreamWs &w : c->ws) {
            for (auto &b : w.lvl)
                if (b.p) cudaFree(b.p);
            if (w.scratch.p) cudaFree(w.scratch.p);
            if (w.flags) cudaFree(w.flags);
            if (w.hist) cudaFree(w.hist);
        }
        if (c->flags) cudaFree(c->flags);
        if (c->flags_host) cudaFreeHost(c->flags_host);
        if (c->hist) cudaFree(c->hist);
        cudaSetDevice(cur);
        delete c;
        g_ctx[d] = nullptr;
    }
    return TG_OK;
}

}  // extern "C"
