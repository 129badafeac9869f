// Internal declarations shared by the kernels (tg_kernels.cu) and the C ABI
// (tg_api.cu).  Nothing here is part of the public interface.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <mutex>

#include "tg_colsolve.h"

namespace tg {

// Kernel attributes (the dynamic shared-memory opt-in) belong to the device
// context: runs f the first time it is reached with device d current, once
// per device and call site, safe against concurrent first calls.
template <class F>
inline void once_per_device(F &&f)
{
    static std::mutex mu;
    static bool done[64] = {};
    int d = 0;
    if (cudaGetDevice(&d) != cudaSuccess || d < 0 || d >= 64) {
        f();
        return;
    }
    std::lock_guard<std::mutex> lk(mu);
    if (!done[d]) {
        f();
        done[d] = true;
    }
}
// Opt-in shared memory per block of the current device (bytes).
int smem_optin();

// Per-segment status bits written by the kernels (atomicOr into a device word).
enum : unsigned {
    FLAG_PIVOT = 1u,      // zero or non-finite pivot / block determinant
    FLAG_NONFINITE = 2u,  // non-finite solution value
    FLAG_NOCONV = 4u,     // refinement hit the sweep cap (column re-solved in FP64)
    FLAG_TIMEOUT = 8u,    // a bounded wait on an asynchronous copy gave up
};

// Maximum refinement sweeps tracked by the histogram (bins 0..kMaxSweepBins-1).
constexpr int kMaxSweepBins = 8;

// Device-side description of one batch of independent systems in level-major
// layout (column index fastest, column stride ld).  For block kinds a/b/c
// hold P/Q/R and x holds u.
struct Seg {
    const double *a, *b, *c, *f;
    double *x;
    const double *ubc_ratio, *ubc_add;
    long ld;
    int nk, k2, ncol, kind;
    int tile0;        // first tile of this segment in the flattened tile space
    int status_idx;   // index into the per-segment status array
};

// Flattened tile table: tile t belongs to the segment s with
// segs[s].tile0 <= t < segs[s+1].tile0 (tile0 is a prefix sum).  When segs is
// null the single segment `one` is used.
struct SegTable {
    const Seg *segs;
    int nseg;
    int ntiles;
    int k2max;        // largest k2 of any segment (sizes per-thread scratch)
    Seg one;
    int hints;        // L2 policy hints: inputs evict-first, sweep scratch evict-last
};

struct Refine {
    int max_sweeps;
    double rel_tol;
};

// Launch shape.
struct Shape {
    int threads;        // threads per block
    int cpt;            // columns per thread (1 or 2)
    int blocks;         // persistent grid size
    int stages;         // bulk-copy ring depth (0: register-prefetch kernel)
    int w2g;            // scalar register kernel with w2 in global scratch
    int pf;             // scalar register kernels: prefetch depth in levels
    size_t smem;        // dynamic shared memory bytes
    int rows;           // block ring kernel with one lane per block row
    int bw;             // block ring kernel: columns per warp (32, 16, 8)
    int lps;            // scalar FP64 ring: levels per stage (>1: chunked ring kernel)
    int res;            // scalar FP64 chunked ring: 1 w2 in shared memory (w3 parked in x), 2 w2 and w3 in
                        // shared memory (k_scalar_f64_res); 0 L2 scratch (k_scalar_f64_chunk)
    int one_wave;       // the grid holds every tile at once (no grid-stride second pass)
};

// Register-prefetch kernel shape of a kind/precision (tg_set_tile).
int cols_per_block(int kind, int precision);
int cols_per_thread(int kind, int precision);
void set_tile(int kind, int precision, int cpb, int cpt);
// Bulk-copy ring depth of a kind/precision (tg_set_pipeline); 0 disables.
// wpb: independent warps per CTA of the ring kernels (0 keeps the default).
void set_stages(int kind, int precision, int stages, int wpb);
int ring_warps(int kind, int precision);
// Effective tile of a launch: the ring kernel (32 columns per warp-CTA)
// when configured and ring_ok (ld % 32 == 0, 16-byte aligned bases), else
// the register-prefetch kernel.
void tile_for(int kind, int precision, bool ring_ok, int *cpb, int *cpt, int *stages, int *w2g);
// Levels of coefficient loads the scalar register kernels keep in flight
// (4, 8 or 16; 2-column threads at most 8).
int prefetch_depth(int kind, int precision);
void set_prefetch(int kind, int precision, int pf);
// Scalar FP64 register kernel keeps w2 in global scratch (1) or shared
// memory (0); -1 restores the default.
void set_w2g(int kind, int precision, int on);
// Global scratch (bytes) of the scalar kernel with w2 in global memory.
size_t scalar_scratch_bytes(long slots, int k2max);
// Global scratch (bytes) of the scalar refinement ring: three float planes.
size_t refine_scratch_bytes(long slots, int k2max);

// Shared memory / scratch needs of a kernel for the largest k2 it will see.
size_t scalar_smem_bytes(int precision, int threads, int cpt, int k2max, int stages, int w2g, int lps);
size_t block_smem_bytes(int B, int stages, int threads, int rows, int bw, int precision);
// Global scratch (bytes) of a block kernel with `slots` resident threads.
size_t block_scratch_bytes(int B, int precision, long slots, int k2max);

// Computes the persistent grid for a launch on the current device, limited
// to ntiles.
cudaError_t plan_shape(int kind, int precision, int k2max, int ntiles, int cpb, int cpt, int stages, int w2g,
                       Shape *shape);

// Solve launches (level-major).  status: per-segment device status words.
// hist: device histogram of refinement sweeps (kMaxSweepBins longs), may be null.
cudaError_t launch_scalar(const SegTable &tab, int precision, const Shape &sh, Refine rf, double *scratch,
                          unsigned *status, unsigned long long *hist, cudaStream_t st);
// q[i] = a[i]/b[i] through the kernels' division (test entry).
cudaError_t launch_selftest_division(const double *a, const double *b, double *q, long n, cudaStream_t st);
cudaError_t launch_block(const SegTable &tab, int B, int precision, const Shape &sh, Refine rf,
                         double *scratch, unsigned *status, unsigned long long *hist,
                         cudaStream_t st);

// 2-D relayout between the Fortran column layout and the level-major layout.
// in(r, col) at in[r + in_ld*col] -> out[r*out_ld + col], r < nrows.
cudaError_t launch_col_to_level(const double *in, long in_ld, double *out, long out_ld,
                                long nrows, long ncols, cudaStream_t st);
// Up to four column->level relayouts in one launch.
struct Relayout {
    const double *in[4];
    double *out[4];
    long in_ld[4];
    long nrows[4];
    long out_ld;
    long ncols;
    int n;
};
cudaError_t launch_col_to_level_multi(const Relayout &r, cudaStream_t st);
// in[r*in_ld + col] -> out(r, col) at out[r + out_ld*col], r < nrows.
cudaError_t launch_level_to_col(const double *in, long in_ld, double *out, long out_ld,
                                long nrows, long ncols, cudaStream_t st);

// The post-solve steps of dt_ng, minor_ng and oplus_ng (src/dt_ng.F90:201-213,
// src/minor_ng.F90:226-237, src/oplus_ng.F90:330-340) done at the back sweep's
// stores: the lateral-boundary overwrite of the flagged columns, the time
// filter of the previous-step field and the floors.  Level-major planes.
struct PostStep {
    const double *cur, *prev;        // the field at this step and at the previous one
    double *nm;                      // receives the filtered previous-step field (may alias prev or cur)
    const unsigned char *bnd_mask;   // (ncol) nonzero: a lateral-boundary column, or null for none
    const double *bnd;               // the boundary values of those columns
    double ds, ds2, floor;           // dtsmooth, dtsmooth_div2, the floor
    int floor_nm;                    // the filtered field is floored too
};

// dt_ng fused assembly + solve (tg_assembly.cu).
typedef tg_dt_fields DtFields;
typedef tg_dt_consts DtConsts;
// scratch (dt_scratch_planes() planes of nk*ld) is used by the three-pass
// form only; without it the fused walk runs.
cudaError_t launch_dt_ng(const DtFields &F, const DtConsts &C, double *tn_upd, int nk, int ncol, long ld,
                         double *sys_out, unsigned *status, cudaStream_t st, const PostStep *post = nullptr,
                         double *scratch = nullptr);
int dt_scratch_planes();

// dt_ng's 12 history diagnostics of a solution x: level-major planes of nk*ld
cudaError_t launch_dt_diag_ng(const DtFields &F, const DtConsts &C, const double *x, int nk, int ncol, long ld,
                              double *diag, cudaStream_t st);

typedef tg_minor_fields MinorFields;
typedef tg_minor_consts MinorConsts;
// scratch (3 * nk * ld doubles, may be NULL): the level-quantity planes of the
// two-pass form, used when assembly_mode() is 1
cudaError_t launch_minor_ng(const MinorFields &F, const MinorConsts &C, double *out, int nk, int ncol, long ld,
                            double *sys_out, unsigned *status, cudaStream_t st, double *scratch,
                            const PostStep *post = nullptr);
// Assembly kernels: 1 (default) two-pass (level-parallel level quantities,
// then the column walk) where built, 0 the single fused column walk.
// 0 one fused column walk, 1 two passes (level quantities, then a walk that
// forms the rows), 2 three passes (the rows too are formed one thread per
// level and column; the walk is the recurrence alone) where built
int assembly_mode();
void set_assembly_mode(int m);
// The walk of the three-pass form (tg_walk.cu): rows 0..K-1 of the p, q, r, f
// planes into x; top 0: K = nk; top 1: K = nk-1 and x(nk-1) =
// x(nk-2)**2/x(nk-3); stored through post when given.
cudaError_t launch_thomas_post(const double *p, const double *q, const double *r, const double *f, double *x, int nk,
                               int K, int top, int ncol, long ld, unsigned *status, const PostStep *post,
                               cudaStream_t st);
// Levels a column walk of the assembly kernels prefetches ahead of the level
// it computes, for a launch over ncol columns: few columns leave few warps
// per SM, and each level of the walk then waits out a memory latency unless
// its reads were requested several levels earlier.  set_walk_prefetch(n):
// n >= 1 fixed, -1 automatic (8 up to kSmallWalkColumns columns, else 1).
constexpr int kSmallWalkColumns = 16384;
// level-major planes of nk*ld doubles the minor_ng scratch holds
int minor_scratch_planes();
int walk_prefetch(long ncol);
void set_walk_prefetch(int levels);

// minor_ng's 7 history diagnostics of a solution x: level-major planes of nk*ld
cudaError_t launch_minor_diag_ng(const MinorFields &F, const MinorConsts &C, const double *x, int nk, int ncol,
                                 long ld, double *diag, cudaStream_t st);

typedef tg_comp_fields CompFields;
typedef tg_comp_consts CompConsts;
// scratch: comp_scratch_doubles(nk, ld) doubles (the block solve's Gamma/z and,
// in the two-pass form, the level planes)
cudaError_t launch_comp_ng(const CompFields &F, const CompConsts &C, double *out, double *scratch, int nk, int ncol,
                           long ld, double *sys_out, unsigned *status, cudaStream_t st);
// comp_ng's 24 history diagnostics of the solution x (3 planes); scratch as
// for launch_comp_ng.
cudaError_t launch_comp_diag_ng(const CompFields &F, const CompConsts &C, const double *x, int nk, int ncol, long ld,
                                double *diag, double *scratch, cudaStream_t st);
size_t comp_scratch_doubles(int nk, long ld);
// bnd_mask (per column, nonzero = lateral boundary) and bnd3 (o2, o1, he
// boundary values) are optional: the overwrite the caller otherwise makes.
cudaError_t launch_comp_post_ng(const double *const *in7, const double *zpmid, double dz, double dtsmooth,
                                double dtsmooth_div2, int nk, int ncol, long ld, double *const *upd6,
                                cudaStream_t st, const unsigned char *bnd_mask = nullptr,
                                const double *const *bnd3 = nullptr);
// advec_ng / smooth_ng on one nest held as a single subdomain (tg_horiz.cu):
// level-major planes (k, i, j) at k*ld + i + (nlon+4)*j
cudaError_t launch_advec_ng(const double *f, const double *un, const double *vn, const double *racs, double dlamda,
                            double dphi, double re_inv, int nk, int nlon, int nlat, long ld, double *hadvec,
                            cudaStream_t st);
cudaError_t launch_smooth_ng(const double *fin, double shapiro, int nk, int nlon, int nlat, long ld, double *fout,
                             cudaStream_t st);
// post-solve time filter and floor of dt_ng / minor_ng / oplus_ng (which =
// TG_FILTER_*) over rows of len elements at stride ld
cudaError_t launch_time_filter(int which, const double *cur, const double *prev, double dtsmooth,
                               double dtsmooth_div2, int rows, long len, long ld, double *upd, double *nm,
                               cudaStream_t st);

typedef tg_settei_fields SetteiFields;
typedef tg_settei_consts SetteiConsts;
// scratch (settei_scratch_doubles(nk, ld) doubles, may be NULL): the level
// planes of the two-pass form, used when assembly_mode() is 1
cudaError_t launch_settei_ng(const SetteiFields &F, const SetteiConsts &C, double *te_out, double *ti_out,
                             double *qtotal, int nk, int ncol, long ld, double *sys_out, unsigned *status,
                             cudaStream_t st, double *scratch);
size_t settei_scratch_doubles(int nk, long ld);

typedef tg_oplus_fields OplusFields;
typedef tg_oplus_consts OplusConsts;
cudaError_t launch_oplus_ng(const OplusFields &F, const OplusConsts &C, double *opout, double *xiop2p,
                            double *xiop2d, double *Fe, double *Fn, double *scratch, int nk, int ncol, long ld,
                            double *sys_out, unsigned *status, cudaStream_t st, const PostStep *post = nullptr);
// The O+ sub-cycle (tg_oplus.cu): the factorization of one step's rows into
// `factor` (oplus_scratch_planes() planes of nk*ld), then one sub-step's
// solve from it with that sub-step's optm1_smooth2 and explicit_h.
cudaError_t launch_oplus_factor(const OplusFields &F, const OplusConsts &C, double *xiop2p, double *xiop2d,
                                double *factor, int nk, int ncol, long ld, unsigned *status, cudaStream_t st);
// oplus_ng's 6 history diagnostics of the solution x; the horizontal terms
// may be NULL; scratch of oplus_scratch_planes() planes.
cudaError_t launch_oplus_diag_ng(const OplusFields &F, const OplusConsts &C, const double *x, const double *diffexp,
                                 const double *vdotn_h, const double *bdotdh_bvel, int nk, int ncol, long ld,
                                 double *diag, double *scratch, cudaStream_t st);
// The factor pass alone (w1, 1/w1, w2 from the p, q, r planes of a factor
// buffer the level and row passes filled).
cudaError_t launch_oplus_factor_pass(double *factor, int nk, int ncol, long ld, unsigned *status, cudaStream_t st);
cudaError_t launch_oplus_solve(const OplusFields &F, const OplusConsts &C, const double *factor, double *opout, int nk,
                               int ncol, long ld, unsigned *status, cudaStream_t st, const PostStep *post = nullptr);
int oplus_scratch_planes();   // level-major scratch planes of launch_oplus_ng (each nk*ld doubles)

// Polar ring filter (tg_filter.cu): the latitudes it filters, with their
// chunk counts; planes (k, i + (nlon+4)*j) at stride ld.
constexpr int kMaxRingRows = 128;    // filtered latitudes (both polar bands)
constexpr int kMaxRingOrder = 15;    // Fourier modes kept as the mean
struct RingRows {
    int n;
    int lat[kMaxRingRows];     // 0-based latitude index
    int nchnk[kMaxRingRows];   // chunks of that latitude
};
size_t ringfilter_smem_bytes(int nlon);
cudaError_t launch_ringfilter(const RingRows &rows, double *f, long ld, int nk, int nlon, int order, int poly,
                              double dlamda, cudaStream_t st);

cudaError_t launch_selftest_wait(unsigned polls, unsigned *status, cudaStream_t st);
// binaryVersion of the library's kernels as loaded on the current device
// (major*10 + minor of the SASS target: 100 for sm_100a).
cudaError_t kernel_binary_version(int *v);

// Block kinds: the bulk-copy ring kernel with one lane per block row
// (tg_set_block_rows); 1 on, 0 off, -1 default.
void set_block_rows(int kind, int on);
// Block kinds: columns per warp of the bulk-copy ring kernel (32, 16 or 8;
// other values restore the default).
void set_block_width(int kind, int w);
// Scalar FP64 ring with w2 in global scratch: levels per ring stage (1, 2, 4,
// 8; other values restore the default).
void set_stage_levels(int kind, int precision, int l);
// Scalar FP64 chunked ring: where the sweep's w2/w3 live between the forward
// and back sweeps (0 L2 scratch, 1 w2 in shared memory, 2 w2 and w3 in shared
// memory; other values restore the default).
void set_column_residency(int kind, int precision, int mode);
int column_residency();
// L2 budget (MB) for the Gamma scratch of all resident block-kernel warps;
// <= 0 restores the default 96 MB.
void set_block_scratch_budget(double mb);
void set_scalar_scratch_budget(double mb);
// Kinds of one plan: 1 concurrently (block kinds on a side stream), 0 one
// after the other, -1 concurrently only when every kind fits in one wave.
void set_kind_overlap(int mode);
int kind_overlap();

// L2 cache-policy hints of the bulk-copy ring kernels (tg_set_cache_hints).
int cache_hints();
void set_cache_hints(int on);

// Records the message tg_last_error() returns on this thread.
void record_error(const char *msg);

}  // namespace tg
