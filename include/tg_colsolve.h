/*
 * tg_colsolve.h -- C ABI of the B200 vertical column solvers for TIE-GCM NG.
 *
 * The library (libtg_colsolve.so) replaces the reference's vertical implicit
 * column solves:
 *   - the scalar tridiagonal Thomas solve trsolv / trsolv_ng, used by dt,
 *     minor (N4S, NO, N2D, Ar), oplus and settei;
 *   - the block-tridiagonal solves: the 3x3 O2/O/He system inline in
 *     comp / comp_ng and the 2x2 U/V system blktri in duv.
 *
 * Conventions
 *   - FP64 everywhere in the interface ("real" is promoted to 8 bytes in the
 *     reference builds).
 *   - Arrays are the reference's column-major (Fortran) arrays passed by
 *     address, unless a layout argument says otherwise:
 *       scalar          (nk, ncol)         element (k,col)     at k + nk*col
 *       block matrices  (B, B, nk, ncol)   element (i,j,k,col) at i + B*j + B*B*(k + nk*col)
 *       block vectors   (B, nk, ncol)      element (i,k,col)   at i + B*(k + nk*col)
 *     Row arguments (k1, k2, lev0, lev1 ...) are 1-based, as in the reference.
 *   - Host-pointer entry points are synchronous, like the Fortran routines
 *     they replace.  Device-pointer entry points (suffix _dev) are
 *     stream-ordered and do not synchronise.  Each caller stream has its own
 *     device work buffers and status word, so _dev calls on different
 *     streams may run at the same time (up to 16 streams at once; a 17th
 *     stream drains the device and takes the least recently used stream's
 *     buffers).  A stream's first call, and a call that needs larger buffers
 *     than the stream had, allocate and synchronise: make those calls once
 *     before capturing the calls into a CUDA graph.
 *   - Every entry point returns a tg_status.  The reference has no error
 *     return (a zero pivot silently yields Inf/NaN); the solves here produce
 *     the same numbers in that case and additionally report TG_EPIVOT.
 *   - The caller owns all arrays.  The library keeps device mirrors and work
 *     buffers per device, reused across calls and released by
 *     tg_release_buffers() or at process exit.  Calls from several host
 *     threads are serialised per device.
 *   - Precision: TG_PREC_F64 reproduces the reference's FP64 arithmetic bit
 *     for bit (same operation order, no FMA contraction, IEEE division).
 *     TG_PREC_F32_REFINE runs the Thomas sweeps in FP32 and corrects with
 *     FP64 residuals (iterative refinement) to a relative correction below
 *     tg_set_refine(); columns that do not converge are re-solved in FP64 on
 *     the GPU.
 */
#ifndef TG_COLSOLVE_H
#define TG_COLSOLVE_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
typedef enum {
    TG_OK = 0,
    TG_EINVAL = 1,      /* an argument is out of range or a pointer is NULL   */
    TG_EPIVOT = 2,      /* a pivot (w1, or a block determinant) was zero or    */
                        /* non-finite in at least one column                   */
    TG_ENONFINITE = 3,  /* a solution value is non-finite                      */
    TG_ENOCONV = 4,     /* FP32 refinement did not converge in the sweep cap   */
                        /* for some column (that column was re-solved in FP64) */
    TG_ETIMEOUT = 5,    /* a bounded device wait gave up                       */
    TG_ECUDA = 6,       /* a CUDA runtime call failed                          */
    TG_ENOMEM = 7,      /* device or pinned memory allocation failed           */
    TG_ENODEV = 8       /* no CUDA device is available                         */
} tg_status;

typedef enum {
    TG_PREC_F64 = 0,         /* FP64 throughout: the drop-in                  */
    TG_PREC_F32_REFINE = 1   /* FP32 sweeps + FP64 iterative refinement       */
} tg_precision;

typedef enum {
    TG_LAYOUT_COLUMN = 0,    /* Fortran layout: level index fastest           */
    TG_LAYOUT_LEVEL = 1      /* level-major: column index fastest, column     */
                             /* stride ld >= ncol (see tg_segment)            */
} tg_layout;

typedef enum {
    TG_KIND_SCALAR = 0,      /* tridiagonal, a/b/c/f -> x                      */
    TG_KIND_BLOCK2 = 2,      /* 2x2 block tridiagonal, P/Q/R/f -> u            */
    TG_KIND_BLOCK3 = 3       /* 3x3 block tridiagonal, P/Q/R/f -> u            */
} tg_kind;

/* ---- drop-in replacements, host pointers, synchronous -------------------- */

/* trsolv (src/trsolv.F:2-107): one latitude slab of the global grid.
 * a,b,c,f,x are (lev0:lev1, lon0:lon1).  Solves rows k1..k2 of every column
 * except the periodic points 1,2 and lonmax-1,lonmax when the slab touches
 * them (trsolv.F:32-35).  Elements of x outside rows k1..k2 or in skipped
 * columns are not written.  The reference reads w1(k1) after initialising
 * w1(lev0); every caller passes k1 == lev0, and here w1(k1) = b(k1).
 * The reference's lat and idebug arguments only feed its debug output. */
int tg_trsolv(const double *a, const double *b, const double *c, const double *f,
              double *x, int lev0, int lev1, int k1, int k2, int lon0, int lon1,
              int lonmax);

/* trsolv_ng (src/trsolv_ng.F90:1-28): all ncol = (lond1-lond0+1)*(latd1-latd0+1)
 * ghost-inclusive columns of a nest level, arrays (nk, ncol).  Rows 1..k2
 * are solved; rows k2+1..nk of x are not written. */
int tg_trsolv_ng(const double *a, const double *b, const double *c, const double *f,
                 double *x, int nk, int k2, int ncol);

/* blktri (src/duv.F:801-908): 2x2 block solve on one slab, a,b,c are
 * (2,2,lev0:lev1,lon0:lon1) and f,x are (2,lev0:lev1,lon0:lon1).  Solves
 * rows lev0..lev1-1, skipping the periodic columns as duv.F:102-105 does with
 * nlonp4.  The reference's beta, gamma and y arguments are work arrays its
 * callers never read; they are not produced. */
/* Deferred form of tg_trsolv for the global grid's latitude scans
 * (src/dt.F:126-330, src/minor.F:491, src/oplus.F:840, src/settei.F:651),
 * which call trsolv once per latitude slab of ~nlon columns: too few to pay
 * for a host->device copy, a launch and a device->host copy each.
 * tg_trsolv_defer takes tg_trsolv's arguments and semantics (rows k1..k2,
 * periodic columns skipped) but only queues the slab: it copies the solved
 * rows and columns of a, b, c, f at once (the caller may reuse them for the
 * next latitude) and remembers x.  tg_trsolv_flush solves every queued slab
 * in one batched host call (runs of slabs with equal k2-k1+1 form one system)
 * and writes each slab's rows k1..k2 into its x; x must stay valid and
 * unread until then.  Same bits as tg_trsolv.  The flush returns the first
 * status; on a numerical status the x values are written as the reference
 * would compute them.  One queue per process, safe from several threads; the
 * flush runs on the calling thread's current device. */
int tg_trsolv_defer(const double *a, const double *b, const double *c, const double *f, double *x,
                    int lev0, int lev1, int k1, int k2, int lon0, int lon1, int lonmax);
int tg_trsolv_flush(void);

int tg_blktri(const double *a, const double *b, const double *c, const double *f,
              double *x, int lev0, int lev1, int lon0, int lon1, int nlonp4);

/* The comp_ng 3x3 O2/O/He block solve (src/comp_ng.F90:166-332), extracted
 * into a call: P,Q,R are the per-level pk,qk,rk blocks (3,3,nk,ncol) with
 * the LBC/UBC folds already applied, f is fk (3,nk,ncol).  Rows 1..nk-1 are
 * solved and row nk is set from the upper boundary as comp_ng.F90:328-332
 * does:  u(i,nk) = ubc_ratio(i)*u(i,nk-1) + ubc_add(i), with ubc_ratio and
 * ubc_add (3,ncol) (ubc_add may be NULL for zero).  B = 2 gives the same
 * solve for 2x2 blocks. */
int tg_comp_blksolve_ng(int B, const double *P, const double *Q, const double *R,
                        const double *f, const double *ubc_ratio, const double *ubc_add,
                        double *u, int nk, int ncol);

/* General host-pointer block solve: P,Q,R (B,B,nk,ncol), f,u (B,nk,ncol),
 * rows 1..k2 solved; if ubc_ratio (B,ncol) is given (k2 < nk), row k2+1 is
 * set as in tg_comp_blksolve_ng.  tg_comp_blksolve_ng(B,...,nk,ncol) is
 * tg_blksolve(B,...,nk,nk-1,ncol), and duv's blktri is the B = 2 case with
 * k2 = nlev-1. */
int tg_blksolve(int B, const double *P, const double *Q, const double *R, const double *f,
                const double *ubc_ratio, const double *ubc_add, double *u, int nk, int k2,
                int ncol);

/* Many independent systems of one model stage in one call (host arrays,
 * Fortran layout, synchronous): e.g. the scalar species of a step together
 * with the major-species block system.  The host<->device copies of all
 * systems are pipelined together, so the call costs about the transfer time
 * of its bytes rather than the sum of per-system calls.  Scalar systems take
 * a,b,c,f,x as in tg_trsolv_ng; block systems (kind 2 or 3) P,Q,R in a,b,c
 * and u in x, as in tg_blksolve. */
typedef struct {
    int kind;               /* tg_kind                                        */
    int nk, k2, ncol;       /* levels, rows solved, columns                   */
    const double *a, *b, *c, *f;
    double *x;
    const double *ubc_ratio, *ubc_add;   /* block only, optional               */
} tg_host_system;

int tg_solve_host(const tg_host_system *sys, int nsys);

/* ---- device-pointer entry points, stream-ordered ----------------------------
 * Pointers are device memory.  layout selects TG_LAYOUT_COLUMN (ld ignored)
 * or TG_LAYOUT_LEVEL (ld = column stride in elements, ld >= ncol).  stream is
 * a cudaStream_t (NULL = legacy default stream).  status_dev, if not NULL,
 * is a device int that receives TG_OK or the first error status; the call
 * itself only reports argument and launch errors. */
int tg_trsolv_dev(const double *a, const double *b, const double *c, const double *f,
                  double *x, int nk, int k2, int ncol, int layout, long ld,
                  int precision, int *status_dev, void *stream);

int tg_blksolve_dev(int B, const double *P, const double *Q, const double *R,
                    const double *f, const double *ubc_ratio, const double *ubc_add,
                    double *u, int nk, int k2, int ncol, int layout, long ld,
                    int precision, int *status_dev, void *stream);

/* Allocation-free variant of tg_blksolve_dev (no counterpart in the reference).
 * For callers that cannot allocate device memory: a model that reserves its
 * whole device-memory budget up front, or a time loop that must not be
 * stalled by the device synchronisation cudaFree implies.  FP64 only,
 * TG_LAYOUT_LEVEL only; results are bit-identical to tg_blksolve_dev.
 * The scratch is a fixed 16 MiB array (2^21 doubles) in the library's device
 * image, held by every GPU that loads the library until the process exits.
 * Limit: each resident thread needs B*B*k2 doubles and one 64-column thread
 * block (a fixed tile, whatever tg_set_tile says) must fit:
 * B*B*k2*64 <= 2^21, so k2 <= 3640 for B = 3 and k2 <= 8192 for B = 2;
 * larger k2 returns TG_EINVAL.  The first call on a device (and the first
 * after a device reset) looks up the array's device address
 * (cudaGetSymbolAddress); make that first call before any stream capture.
 * All calls share the array: calls that overlap on the GPU (e.g. on two
 * streams) race and must not be issued concurrently. */
int tg_blksolve_dev_noalloc(int B, const double *P, const double *Q, const double *R,
                            const double *f, const double *ubc_ratio, const double *ubc_add,
                            double *u, int nk, int k2, int ncol, long ld, int *status_dev,
                            void *stream);

/* ---- fused column assembly + solve ------------------------------------------
 * dt_ng's vertical column step (src/dt_ng.F90:57-167): the neutral-
 * temperature coefficients p, q, r, rhs are assembled per column from the
 * physical fields and solved (rows 1..nk-1, trsolv_ng), and row nk is set to
 * tn(nk-1)**2/tn(nk-2).  The horizontal operators stay in the host model:
 * horadv = advec_ng(tn) and tnsmooth = smooth_ng(tn_nm) are inputs.
 * tlbc is the previous step's lower-boundary Tn (the routine's tlbc
 * argument), t_lbc the current one.  3-D fields (nk, ncol); 2-D (ncol);
 * expz, dift (nk).  nk >= 3.  Results are bit-identical to the reference's
 * FP64 arithmetic. */
typedef struct {
    const double *tn, *tnsmooth, *horadv, *un, *vn, *o1, *mbar, *xnmbar, *scht, *schti, *cp, *kt,
        *km, *hdt, *qji_tn, *cool_imp, *cool_exp, *w, *qtotal, *rkm12;
    const double *tlbc, *t_lbc, *ulbc, *vlbc;
    const double *expz, *dift;
} tg_dt_fields;

typedef struct {
    double dz, dtx2inv, expzmid_inv, grav, p0, avo, gask, tsurplus, rmassinv_o1;
} tg_dt_consts;

/* Host arrays in the Fortran layout, synchronous. */
int tg_dt_ng(const tg_dt_fields *F, const tg_dt_consts *C, double *tn_upd, int nk, int ncol);
/* Device arrays, level-major (3-D field (k,col) at k*ld + col).  If
 * system_out is not NULL it receives the assembled rows 1..nk-1 (after the
 * lower-boundary fold) as four level-major planes p, q, r, rhs of nk*ld each. */
int tg_dt_ng_dev(const tg_dt_fields *F, const tg_dt_consts *C, double *tn_upd, int nk, int ncol, long ld,
                 double *system_out, int *status_dev, void *stream);

/* minor_ng's vertical column step (src/minor_ng.F90:60-200), used for the
 * minor species N4S, NO, N2D and Ar: the coefficients are assembled per
 * column (a 3x3 diffusion matrix alfa is inverted per level) and solved for
 * rows 1..nk.  The horizontal operators stay in the host model: hadvec =
 * advec_ng(fcomp) and ftm1_smooth = smooth_ng(fcomp_tm1) are inputs, and
 * dfactor is the per-column latitude factor of minor_ng.F90:146-155.  b (3x3,
 * column-major) and fb (3) are the lbc module's lower-boundary relation,
 * phix/alfax/rmx the species parameters.  3-D fields (nk, ncol); 2-D (ncol);
 * expz, difk (nk).  The fractional powers use the device pow, so results
 * agree with the reference arithmetic to ~1e-13 relative, not bit for bit. */
typedef struct {
    const double *tn, *o2, *o1, *he, *mbar, *barm, *xnmbar, *w, *ftm1_smooth, *hadvec, *sloss, *sprod;
    const double *tlbc, *flbc1, *flbc2, *flbc3, *fubc, *dfactor;
    const double *expz, *difk;
} tg_minor_fields;

typedef struct {
    double rmx, alfax, phix[4], dzp, dtx2inv, expzmid, expzmid_inv;
    double rmassinv_o2, rmassinv_o1, rmassinv_n2, rmassinv_he;
    double rmass_o2, rmass_o1, rmass_he, rmass_n2, p0, grav, avo;
    double b[9], fb[3];
} tg_minor_consts;

int tg_minor_ng(const tg_minor_fields *F, const tg_minor_consts *C, double *fcomp_out, int nk, int ncol);
int tg_minor_ng_dev(const tg_minor_fields *F, const tg_minor_consts *C, double *fcomp_out, int nk, int ncol,
                    long ld, double *system_out, int *status_dev, void *stream);

/* History diagnostics of dt_ng (src/dt_ng.F90:169-191) and minor_ng
 * (src/minor_ng.F90:202-224): the fields the reference passes to addfld,
 * computed from the routine's fields and its solution (tn_upd / fcomp_out
 * rows 1..nk as the solve returns them, before the lateral-boundary
 * overwrite).  dt_ng: 12 slabs DTDT, DT_SOLAR, DT_HORDIF, DT_RECOMB,
 * DT_JOULE, DT_MOLDIF, DT_COOL, DT_HORADV (= -horadv), DT_VERADV (= -the
 * vertical advection), DT_ADIA, DT_CONDUCT (rows 1 and nk zero), DEN (the
 * density of :133); bit-identical to the reference arithmetic.  minor_ng: 7
 * slabs D<name>DT, <name>_PROD, <name>_LOSS, <name>_MOLDIF, <name>_EDDYDIF,
 * -<name>_VERADV, -<name>_HORADV (MOLDIF, EDDYDIF, VERADV rows 1 and nk
 * zero); MOLDIF and EDDYDIF use the device's fractional powers like
 * tg_minor_ng (within ~1e-13 relative), the others are bit-identical.
 * Host forms: fields as for tg_dt_ng / tg_minor_ng, diag (nk, ncol, nd) in
 * the Fortran layout.  Device forms: level-major planes, diag nd planes of
 * nk*ld, on the caller's stream. */
int tg_dt_diag_ng(const tg_dt_fields *F, const tg_dt_consts *C, const double *tn_upd, double *diag, int nk,
                  int ncol);
int tg_dt_diag_ng_dev(const tg_dt_fields *F, const tg_dt_consts *C, const double *tn_upd, double *diag, int nk,
                      int ncol, long ld, void *stream);
int tg_minor_diag_ng(const tg_minor_fields *F, const tg_minor_consts *C, const double *fcomp_out, double *diag,
                     int nk, int ncol);
int tg_minor_diag_ng_dev(const tg_minor_fields *F, const tg_minor_consts *C, const double *fcomp_out, double *diag,
                         int nk, int ncol, long ld, void *stream);

/* comp_ng's major-species column step (src/comp_ng.F90:74-332): O2, O and He
 * from the 3x3 block-tridiagonal diffusion system, assembled per column and
 * solved for rows 1..nk-1, with the top level from the upper boundary (He
 * escape flux flx_he).  Horizontal operators stay in the host model: the
 * *_advec fields are advec_ng of the species, *nm_smooth smooth_ng of the
 * previous step, hdo2/hdo1/hdhe the horizontal diffusion.  fs is the
 * reference's fs(nk, ncol, 3, 0:3): 12 slabs (nk, ncol), slab m*3+isp, m = 0
 * production, 1..3 the loss matrix.  b, fb: the lbc module's lower-boundary
 * relation.  calc_helium = 0 takes flx_he as 0 and returns He = pshelb
 * (comp_ng.F90:72,386-389).  Outputs o2/o1/he_upd before the time filter;
 * tg_comp_post_ng applies the post-solve steps (:415-457) after the caller
 * has written its lateral-boundary columns. */
typedef struct {
    const double *tn, *o2, *o1, *he, *w, *mbar, *o2nm_smooth, *o1nm_smooth, *henm_smooth;
    const double *o2_advec, *o1_advec, *he_advec, *hdo2, *hdo1, *hdhe, *fs;
    const double *tlbc, *flx_he, *dfactor;
    const double *expz, *difk;
} tg_comp_fields;

typedef struct {
    double dz, dtx2inv, expzmid, expzmid_inv;
    double rmassinv_o2, rmassinv_o1, rmassinv_he, rmassinv_n2;
    double rmass_o2, rmass_o1, rmass_he, p0, grav;
    double b[9], fb[3];
    double pshelb;
    int calc_helium;
} tg_comp_consts;

int tg_comp_ng(const tg_comp_fields *F, const tg_comp_consts *C, double *o2_upd, double *o1_upd, double *he_upd,
               int nk, int ncol);
/* Device form: level-major (k*ld + col) fields, fs 12 slabs of nk*ld; out
 * receives 3 slabs (O2, O, He) of nk*ld; system_out (may be NULL) 30 slabs
 * of nk*ld: P(i,m) at slab i+3m, Q at 9+i+3m, R at 18+i+3m, f at 27+i. */
int tg_comp_ng_dev(const tg_comp_fields *F, const tg_comp_consts *C, double *out, int nk, int ncol, long ld,
                   double *system_out, int *status_dev, void *stream);
/* comp_ng's history diagnostics (src/comp_ng.F90:334-380): the 24 fields the
 * reference passes to addfld, from the fields and the solution (o2/o1/he_upd
 * as tg_comp_ng returns them, before the lateral-boundary overwrite and the
 * post steps), in the order of the calls: DO2DT, DO1DT, DHEDT, O2/O1/HE_PROD,
 * O2/O1/HE_LOSS, O2/O1/HE_HORDIF, O2/O1/HE_MOLDIF, O2/O1/HE_EDDYDIF,
 * -O2/O1/HE_VERADV, -O2/O1/HE_HORADV.  LOSS and MOLDIF are summed over the
 * fourth index of loss(k,i,j,isp,m) and moldif, the row's species, as the
 * reference's sum(., dim=4) does; MOLDIF, EDDYDIF and VERADV, which the
 * reference leaves unset on the first and top levels, are 0 there.  MOLDIF
 * and EDDYDIF use the device's fractional powers like tg_comp_ng (within
 * ~1e-13 relative); the others are bit-identical.  With calc_helium = 0
 * the reference's He planes use the solved He, which tg_comp_ng replaces by
 * pshelb before returning it: their values here are those of the He passed.
 * Host form: diag (nk, ncol, 24) in the Fortran layout.  Device form: upd the three level-major
 * planes (as tg_comp_ng_dev writes them), diag 24 planes of nk*ld, on the
 * caller's stream. */
int tg_comp_diag_ng(const tg_comp_fields *F, const tg_comp_consts *C, const double *o2_upd, const double *o1_upd,
                    const double *he_upd, double *diag, int nk, int ncol);
int tg_comp_diag_ng_dev(const tg_comp_fields *F, const tg_comp_consts *C, const double *upd, double *diag, int nk,
                        int ncol, long ld, void *stream);

/* comp_ng's post-solve steps per column (src/comp_ng.F90:415-457): time
 * filter, N2 = 1-O2-O-He with the exponential extrapolation above the first
 * level where N2 < 0.01, the floor at 1e-9 and the normalisation.  o2/o1/he
 * are the current-step fields, *_nm the previous step; o2/o1/he_upd are
 * updated in place, *nm_upd receive the filtered fields.  Host arrays (nk,
 * ncol); zpmid (nk) the level midpoints.  A column whose N2 is below 0.01 at
 * level 1 is left without extrapolation (the reference reads level 0 there). */
int tg_comp_post_ng(const double *o2, const double *o1, const double *he, const double *o2_nm, const double *o1_nm,
                    const double *he_nm, const double *xnmbar, const double *zpmid, double dz, double dtsmooth,
                    double dtsmooth_div2, int nk, int ncol, double *o2_upd, double *o1_upd, double *he_upd,
                    double *o2nm_upd, double *o1nm_upd, double *henm_upd);
/* Device form: level-major (k*ld + col) device arrays, zpmid a device array
 * (nk), stream-ordered.  o2_upd/o1_upd/he_upd hold comp_ng's solution on
 * entry (e.g. the three planes tg_comp_ng_dev wrote) and are updated in
 * place; each nm_upd may be the same array as its species' *_nm or current
 * field (every value is read before its own index is written).  With
 * bnd_mask (ncol bytes, nonzero = a lateral-boundary column) the flagged
 * columns of o2/o1/he_upd first take o2_bnd/o1_bnd/he_bnd (level-major, like
 * the fields): the Dirichlet hook of src/comp_ng.F90:394-413.  bnd_mask and
 * the three bnd arrays NULL: no overwrite. */
int tg_comp_post_ng_dev(const double *o2, const double *o1, const double *he, const double *o2_nm,
                        const double *o1_nm, const double *he_nm, const double *xnmbar, const double *zpmid,
                        double dz, double dtsmooth, double dtsmooth_div2, int nk, int ncol, long ld,
                        double *o2_upd, double *o1_upd, double *he_upd, double *o2nm_upd, double *o1nm_upd,
                        double *henm_upd, const unsigned char *bnd_mask, const double *o2_bnd,
                        const double *o1_bnd, const double *he_bnd, void *stream);

/* The post-solve time filter and floor of the scalar routines, applied after
 * the caller has written its lateral-boundary columns:
 *   TG_FILTER_DT    src/dt_ng.F90:208-213     tn_nm_upd = dtsmooth_div2*(tn_nm+tn_upd) + dtsmooth*tn,
 *                                             tn_upd = max(tn_upd, 100.)
 *   TG_FILTER_MINOR src/minor_ng.F90:234-237  fcomp_tm1_out = dtsmooth*fcomp + dtsmooth_div2*(fcomp_tm1+fcomp_out),
 *                                             both floored at 1e-12
 *   TG_FILTER_OPLUS src/oplus_ng.F90:337-340  optm1out = dtsmooth*op + dtsmooth_div2*(optm1+opout),
 *                                             both floored at 0
 * cur is the field at the current step (tn, fcomp, op), prev the previous
 * step (tn_nm, fcomp_tm1, optm1); upd (tn_upd, fcomp_out, opout) is read and
 * floored in place and nm_upd receives the filtered field.  nm_upd may be
 * the same array as prev or cur.  A floor keeps x when x > floor and gives
 * the floor otherwise (NaN included, as tg_comp_post_ng does).  Results are
 * bit-identical to the reference's FP64 arithmetic (no fused multiply-add).
 * Host arrays (nk, ncol), synchronous. */
#define TG_FILTER_DT 0
#define TG_FILTER_MINOR 1
#define TG_FILTER_OPLUS 2
int tg_time_filter_ng(int which, const double *cur, const double *prev, double dtsmooth, double dtsmooth_div2,
                      int nk, int ncol, double *upd, double *nm_upd);
/* ---- horizontal operators feeding the assembly -------------------------------
 * advec_ng (src/advec_ng.F90:1-52) and smooth_ng (src/smooth_ng.F90:1-42)
 * with their difference and mean helpers (src/dffm_ng.F90), for a nest held
 * as one subdomain: arrays (nk, nlon+4, nlat+4) over the ghost-inclusive
 * lond0:lond1 x latd0:latd1, every lateral edge a boundary (is_bndry all
 * true, the one-task decomposition of src/fields_ng.F90:143-147), so the
 * halo exchanges of src/sync_ng.F90 have nothing to exchange.
 *   tg_advec_ng:  hadvec from f, the winds un, vn (the itp level of the
 *                 model's fields), racs (nlat+4) per latitude, dlamda, dphi
 *                 and re_inv = 1/re.
 *   tg_smooth_ng: fout = the Shapiro filter of fin, in lat then lon.
 * Results are bit-identical to the reference's FP64 arithmetic.  Outputs
 * must not alias inputs.  nk <= 65535, nlat <= 500000. */
int tg_advec_ng(const double *f, const double *un, const double *vn, const double *racs, double dlamda,
                double dphi, double re_inv, int nk, int nlon, int nlat, double *hadvec);
int tg_smooth_ng(const double *fin, double shapiro, int nk, int nlon, int nlat, double *fout);
/* Device forms: level-major planes, (k, i, j) at k*ld + i + (nlon+4)*j with
 * ld >= (nlon+4)*(nlat+4) (the column index of the other device entries);
 * racs a device array (nlat+4); stream-ordered. */
int tg_advec_ng_dev(const double *f, const double *un, const double *vn, const double *racs, double dlamda,
                    double dphi, double re_inv, double *hadvec, int nk, int nlon, int nlat, long ld,
                    void *stream);
int tg_smooth_ng_dev(const double *fin, double shapiro, double *fout, int nk, int nlon, int nlat, long ld,
                     void *stream);

/* Device arrays, level-major (k*ld + col), stream-ordered; nk <= 65535. */
int tg_time_filter_ng_dev(int which, const double *cur, const double *prev, double dtsmooth,
                          double dtsmooth_div2, int nk, int ncol, long ld, double *upd, double *nm_upd,
                          void *stream);

/* The same post-solve steps fused into the solve: the fused assembly + solve
 * of dt_ng, minor_ng or oplus_ng (as tg_*_ng_dev) stores every solution row
 * through them, so the solution is written once, already filtered.  In the
 * reference's order: the top row (dt_ng, oplus_ng) from the unfiltered
 * values; then the lateral-boundary overwrite (src/dt_ng.F90:201-206,
 * src/minor_ng.F90:226-232, src/oplus_ng.F90:330-335), which here takes the
 * columns flagged in bnd_mask (ncol bytes, nonzero = a boundary column) from
 * bnd (level-major, the values the caller's lon_b/lat_b give those columns;
 * bnd_mask and bnd both NULL when there is none); then the time filter into
 * nm_upd and the floors of TG_FILTER_DT / MINOR / OPLUS.  nm_upd may alias
 * prev or cur.  Results are the separate solve, overwrite and
 * tg_time_filter_ng_dev's, bit for bit (to the routine's tolerance for
 * minor_ng and oplus_ng, whose solves carry the device's fractional powers).
 * The history diagnostics (tg_dt_diag_ng_dev, tg_minor_diag_ng_dev) need the
 * unfiltered solution: callers that write them use the separate steps.
 * Device arrays, level-major, stream-ordered. */
typedef struct {
    const double *cur;              /* tn, fcomp, op: the field at this step        */
    const double *prev;             /* tn_nm, fcomp_tm1, optm1: the previous step   */
    double *nm_upd;                 /* tn_nm_upd, fcomp_tm1_out, optm1out            */
    const unsigned char *bnd_mask;  /* per column: nonzero for a lateral boundary   */
    const double *bnd;              /* boundary values of the flagged columns       */
    double dtsmooth, dtsmooth_div2;
} tg_post_step;
int tg_dt_ng_post_dev(const tg_dt_fields *F, const tg_dt_consts *C, double *tn_upd, int nk, int ncol, long ld,
                      const tg_post_step *P, int *status_dev, void *stream);
int tg_minor_ng_post_dev(const tg_minor_fields *F, const tg_minor_consts *C, double *fcomp_out, int nk, int ncol,
                         long ld, const tg_post_step *P, int *status_dev, void *stream);
/* tg_oplus_ng_post_dev follows tg_oplus_ng_dev below. */

/* ---- polar ring filter ------------------------------------------------------
 * ringfilter (src/ringfilter.F:1-111) over every latitude of a global field
 * held whole on one device, as filter_o2o (src/comp.F:1065-1145) and the
 * global dt, oplus, minor and duv filters apply it once the longitudes are
 * gathered (here no gather is needed).  f is (nk, nlon+4, nlat) in the
 * reference's layout, longitude index 1..nlon+4 with the interior at
 * 3..nlon+2 and two periodic points each side, filtered in place.
 * Latitudes within nlat_filter rows of a pole take chunk_array's chunk count
 * (cons_module's chunk_array, src/cons.F:331-355); the others are unchanged.
 * order: Fourier modes kept as the mean, 1..15 and below nlon (filter_o2o 1,
 * the others 3); poly: 1 for OPLUS's piecewise polynomial reconstruction, 0
 * the piecewise linear one.  Bit-identical to the reference arithmetic with
 * sums in longitude order.  The first call with a given (nlon, order,
 * dlamda) on a device uploads a cos/sin table (synchronously). */
int tg_ringfilter(double *f, int nk, int nlon, int nlat, int order, int poly, const int *chunk_array,
                  int nlat_filter, double dlamda);
/* filter_o2o's filter of one species (src/comp.F:1065-1145): tg_ringfilter
 * with order 1, linear reconstruction. */
int tg_filter_o2o(double *fout, int nk, int nlon, int nlat, const int *chunk_array, int nlat_filter,
                  double dlamda);
/* Device form: level-major planes, element (k, i, j) at k*ld + i + (nlon+4)*j
 * (i, j 0-based), on the caller's stream. */
int tg_ringfilter_dev(double *f, int nk, int nlon, int nlat, int order, int poly, const int *chunk_array,
                      int nlat_filter, double dlamda, long ld, void *stream);

/* settei_ng's electron and ion temperature step (src/settei_ng.F90:60-261):
 * the whole routine is column-local, so it is one fused kernel: the heat-flux
 * boundary fe, thermal conductivity, the conduction rows in Te^3.5, heating,
 * cooling and exchange rates, the solve of rows 1..nk-1, Te = x^(2/7) with the
 * top level, and Ti.  qtotal is read and updated (qtotal += q_eni at the
 * interfaces, :248-254).  3-D fields (nk, ncol), 2-D (ncol).  b, fb: the lbc
 * module's lower-boundary relation; et and electron_heating: the input
 * switches of the reference; dipmin the grid's minimum dip. */
typedef struct {
    const double *tn, *o2, *o1, *he, *n2, *ne, *te, *ti, *op, *o2p, *nplus, *n2p, *nop, *xnmbar, *xnmbari, *scht;
    const double *schti, *qji_ti, *qop2p, *qop2d, *qo2p, *qop, *qn2p, *qnp, *qnop, *Q1, *Q2;
    const double *t_lbc, *chi, *rlatm, *dipmag, *qteaur;
} tg_settei_fields;

typedef struct {
    double f107, dipmin, dz, evergs, avo, rmass_o1;
    double rmassinv_o2, rmassinv_o1, rmassinv_he, rmassinv_n2, rmassinv_n4s, rmassinv_no;
    double b[9], fb[3];
    int et, electron_heating;
} tg_settei_consts;

int tg_settei_ng(const tg_settei_fields *F, const tg_settei_consts *C, double *te_out, double *ti_out,
                 double *qtotal, int nk, int ncol);
/* Device form: level-major (k*ld + col) arrays; system_out (may be NULL)
 * 4 slabs (p, q, r, rhs) of nk*ld, rows 1..nk-1. */
int tg_settei_ng_dev(const tg_settei_fields *F, const tg_settei_consts *C, double *te_out, double *ti_out,
                     double *qtotal, int nk, int ncol, long ld, double *system_out, int *status_dev, void *stream);

/* oplus_ng's O+ column step, vertical part (src/oplus_ng.F90:88-307): the
 * diffusion, drift and wind rows, chemistry, both boundaries, the solve of
 * rows 1..nk-1 and the top level.  The terms built from horizontal
 * derivatives come from the host model as inputs, exactly as the reference
 * computes them: explicit_h = -explic*diffexp + vdotn_h + bdotdh_bvel
 * (:178-207), bdotdh_djbz = bdotdh(dj*bz) (:234), dvb = (div b + 2 bz)/re
 * before its division by bz (:101-107), optm1_smooth2 = smooth_ng(optm1)
 * (:162).  Outputs opout (before the lateral-boundary overwrite, the time
 * filter and the clamp of :332-340, which stay with the caller), xiop2p,
 * xiop2d (:285-288); Fe, Fn (:164-169) may be NULL.  The diffusion cap
 * applies when |opdiffcap| >= 1e-9 (isclose of src/util.F:1384). */
typedef struct {
    const double *tn, *te, *ti, *o2, *o1, *n2, *he, *n2d, *ne, *u, *v, *w, *wi, *xnmbar, *scht, *qop2p, *qop2d;
    const double *qop, *rk1, *rk2, *rk19, *rk20, *rk25, *op, *optm1_smooth2, *explicit_h, *bdotdh_djbz;
    const double *bx, *by, *bz, *dvb, *rlatm, *chi, *dipmag, *sndec, *csdec;
    const double *zpint;
} tg_oplus_fields;

typedef struct {
    double rmass_op, gask, grav, re, rmassinv_o2, rmassinv_o1, rmassinv_n2, rmassinv_n2d, rmassinv_he;
    double rk10, rk16, rk17, rk18, rk21, rk22, rk23, rk24, rk26, rk27;
    double colfac, opdiffcap, dtx2inv, dz, dlev;
    int nstep_sub;
} tg_oplus_consts;

int tg_oplus_ng(const tg_oplus_fields *F, const tg_oplus_consts *C, double *opout, double *xiop2p, double *xiop2d,
                double *Fe, double *Fn, int nk, int ncol);
/* Device form: level-major (k*ld + col) arrays, zpint (nk); system_out (may
 * be NULL) 4 slabs (p, q, r, explicit) of nk*ld, rows 1..nk-1. */
int tg_oplus_ng_dev(const tg_oplus_fields *F, const tg_oplus_consts *C, double *opout, double *xiop2p,
                    double *xiop2d, double *Fe, double *Fn, int nk, int ncol, long ld, double *system_out,
                    int *status_dev, void *stream);
/* oplus_ng with the post-solve steps fused (see tg_post_step above). */
int tg_oplus_ng_post_dev(const tg_oplus_fields *F, const tg_oplus_consts *C, double *opout, double *xiop2p,
                         double *xiop2d, double *Fe, double *Fn, int nk, int ncol, long ld, const tg_post_step *P,
                         int *status_dev, void *stream);

/* The O+ sub-cycle (src/dynamics_ng.F90:103-117): oplus_ng runs nstep_sub
 * times on the same fields, and only op, optm1 (hence optm1_smooth2) and the
 * horizontal terms explicit_h change from one sub-step to the next.  They
 * enter the right-hand side alone, so the rows p, q, r and the forward
 * elimination's pivots are the same in every sub-step:
 *   tg_oplus_ng_factor_dev  forms them once per step into `factor` (device
 *                           memory of tg_oplus_ng_factor_doubles(nk, ld)
 *                           doubles, owned by the caller), with xiop2p and
 *                           xiop2d; status TG_EPIVOT for a zero pivot;
 *   tg_oplus_ng_solve_dev   one sub-step: opout from the factor and F's
 *                           current explicit_h and optm1_smooth2 (the other
 *                           fields must be those the factor was formed from),
 *                           with the post-solve steps when P is not NULL.
 * Each sub-step's opout is bit-identical to tg_oplus_ng_dev /
 * tg_oplus_ng_post_dev on the same fields. */
long tg_oplus_ng_factor_doubles(int nk, long ld);
/* oplus_ng's history diagnostics (src/oplus_ng.F90:309-330): 6 fields DOPDT,
 * OP_PROD, OP_LOSS (= -op_loss*opout), OP_DIFF, OP_DRIFT, OP_WIND of the
 * solution opout (rows 1..nk, the top level included, before the lateral
 * overwrite and the post steps).  The three sums add the horizontal terms
 * the host model computes in the routine's horizontal part (diffexp,
 * vdotn_h, bdotdh_bvel: each may be NULL, taken as 0, and the sum then holds
 * the vertical part alone) and are defined on levels 2..nk-1; the reference
 * leaves the first and top levels unset, here they are 0.  OP_DIFF carries
 * the device's log10 and pow through dj (within ~1e-13 relative, like
 * tg_oplus_ng); the others are bit-identical.  Host form: diag (nk, ncol, 6)
 * in the Fortran layout; device form: 6 planes of nk*ld on the caller's
 * stream. */
int tg_oplus_diag_ng(const tg_oplus_fields *F, const tg_oplus_consts *C, const double *opout, const double *diffexp,
                     const double *vdotn_h, const double *bdotdh_bvel, double *diag, int nk, int ncol);
int tg_oplus_diag_ng_dev(const tg_oplus_fields *F, const tg_oplus_consts *C, const double *opout,
                         const double *diffexp, const double *vdotn_h, const double *bdotdh_bvel, double *diag,
                         int nk, int ncol, long ld, void *stream);
int tg_oplus_ng_factor_dev(const tg_oplus_fields *F, const tg_oplus_consts *C, double *xiop2p, double *xiop2d,
                           double *factor, int nk, int ncol, long ld, int *status_dev, void *stream);
int tg_oplus_ng_solve_dev(const tg_oplus_fields *F, const tg_oplus_consts *C, const double *factor, double *opout,
                          int nk, int ncol, long ld, const tg_post_step *P, int *status_dev, void *stream);

/* ---- batched, GPU-resident plans ---------------------------------------------
 * A plan solves many independent systems ("segments": any mix of grids, nest
 * levels, sub-steps and species) in one persistent launch per system kind,
 * driven by a flattened table of column tiles.  Segment arrays are device
 * memory in TG_LAYOUT_LEVEL with column stride ld:
 *   scalar  a,b,c,f,x   element (k,col)     at k*ld + col
 *   block   P,Q,R       element (i,j,k,col) at ((k*B + j)*B + i)*ld + col
 *           f,u         element (i,k,col)   at (k*B + i)*ld + col
 *           ubc_ratio, ubc_add (optional)   at i*ld + col
 * For block segments a,b,c carry P,Q,R and x carries u. */
typedef struct {
    int kind;              /* tg_kind                                        */
    int nk;                /* levels per column (array extent)               */
    int k2;                /* rows 1..k2 are solved                          */
    int ncol;              /* columns                                        */
    long ld;               /* column stride, >= ncol                         */
    const double *a, *b, *c, *f;
    double *x;
    const double *ubc_ratio, *ubc_add;   /* block only; NULL for none        */
} tg_segment;

typedef struct tg_plan tg_plan;

/* Copies the segment table; the arrays themselves are referenced, not
 * copied, and must stay valid while the plan is executed. */
int tg_plan_create(const tg_segment *segs, int nseg, int precision, tg_plan **plan);
/* Enqueues the solve of every segment on stream (cudaStream_t). */
int tg_plan_execute(tg_plan *plan, void *stream);
/* Records one tg_plan_execute into a CUDA graph and replays it from then on
 * (the stream must be the one used by later executes). */
int tg_plan_capture_graph(tg_plan *plan, void *stream);
/* Waits for the plan's work and copies one tg_status per segment. */
int tg_plan_status(tg_plan *plan, int *per_segment_status);
/* Number of kernel launches one tg_plan_execute issues. */
int tg_plan_launches(const tg_plan *plan);
/* The kernel each group of the plan launches, with its launch shape, as
 * "k_scalar_f64_ring<4,1> kind=0 threads=32 blocks=...; ..." (for logs and
 * profiler filters).  TG_EINVAL when n is too small (output truncated). */
int tg_plan_describe(const tg_plan *plan, char *buf, int n);
/* Refinement sweep histogram of the last execute: hist[s] = columns that
 * needed s sweeps (s = 0..nbins-1; the last bin also counts the FP64
 * re-solves).  Returns the number of bins written. */
int tg_plan_sweep_histogram(tg_plan *plan, long *hist, int nbins);
int tg_plan_destroy(tg_plan *plan);

/* ---- tuning, configuration, housekeeping ------------------------------------ */

/* Tuning entries (tg_set_*) change process-wide settings that plans and
 * calls read when they are created or launched: set them before other threads
 * create plans or call the solvers.
 *
 * Mixed-precision refinement: at most max_sweeps FP64 residual sweeps per
 * column (defaults 3 and 1e-11).  A column stops when its correction, or the
 * error left after it as estimated from the contraction of successive
 * corrections (the FP32 sweep-0 solution counting as the first, with a
 * 16-fold margin), is below rel_tol * max|x|. */
int tg_set_refine(int max_sweeps, double rel_tol);
/* Precision of the host-pointer drop-ins (tg_trsolv, tg_trsolv_ng, tg_blktri,
 * tg_comp_blksolve_ng, tg_blksolve), which keep the reference's signatures
 * and therefore have no precision argument.  Default TG_PREC_F64. */
int tg_set_host_precision(int precision);
/* Launch shape of a kind/precision: columns per thread block (32..512, a
 * multiple of 32) and columns per thread (1 or 2); 0 restores the default. */
int tg_set_tile(int kind, int precision, int cols_per_block, int cols_per_thread);
/* Coefficient staging of the FP64 kernels of a kind: 0 = register-prefetch
 * kernel (shape from tg_set_tile); 4, 8 or 16 = depth in levels of the
 * shared-memory ring that bulk asynchronous copies fill ahead of the sweep
 * (one warp per 32 columns, `warps` independent warps per CTA, 1..8, 0 the
 * default count; used when the level-major column stride is a multiple
 * of 32 and the arrays are 16-byte aligned, otherwise the register-prefetch
 * kernel runs); -1 restores the default.  Scalar kind, TG_PREC_F32_REFINE:
 * 2..4 = stages of 4 levels of the refinement ring (x 16-byte aligned too),
 * 0 = register-prefetch refinement kernel. */
int tg_set_pipeline(int kind, int precision, int stages, int warps);
/* Depth (levels) of the register prefetch of the scalar kernels' coefficient
 * loads: 4, 8 or 16 (kind TG_KIND_SCALAR, either precision); -1 restores the
 * default.  Deeper prefetch keeps more bytes in flight per column at the cost
 * of registers. */
int tg_set_prefetch(int kind, int precision, int levels);
/* Where the scalar FP64 register-prefetch kernel keeps its forward-sweep
 * quotients w2: 0 = shared memory (limits residency to ~8 B x nk per column
 * of shared memory), 1 = a library-owned global scratch that stays in L2
 * (residency then limited only by registers); -1 restores the default.
 * Only kind TG_KIND_SCALAR with TG_PREC_F64. */
int tg_set_scratch_global(int kind, int precision, int on);
/* L2 eviction-priority hints of the bulk-copy (ring) kernels: coefficient
 * streams evict-first, the sweep's scratch and parked w3 evict-last.
 * on: 1 (default), 0 off, -1 back to the default; 2 and 3 as 1, except that
 * the refinement kernels' coefficient fills, which every sweep reads again,
 * are evict-normal (2) or evict-last (3). */
int tg_set_cache_hints(int on);

/* FP64 block kinds with a bulk-copy ring: one lane per block row (B lanes per
 * column, whole blocks exchanged by warp shuffles) instead of one lane per
 * column.  Same arithmetic, bit-identical results.  on: 1, 0, -1 default. */
int tg_set_block_rows(int kind, int on);

/* FP64 block kinds with a bulk-copy ring: columns per warp, 32 (default), 16
 * or 8 (other values restore the default).  Fewer columns per warp means more
 * warps for the same columns, which helps when a grid has too few columns to
 * hide the latency of the block recurrence.  Same arithmetic, same bits. */
int tg_set_block_width(int kind, int width);

/* Scalar FP64 bulk-copy ring with w2 in global scratch: levels per ring stage
 * (1, 2, 4 or 8; other values restore the default).  With L > 1 one mbarrier
 * wait and one round of copies serve L levels; the ring depth set by
 * tg_set_pipeline then counts stages of L levels (2, 3 or 4). */
int tg_set_stage_levels(int kind, int precision, int levels);

/* Where the FP64 bulk-copy ring kernels keep the forward sweep's quantities
 * until the back sweep reads them.  Scalar kind (chunked ring): 0 w2 in an L2
 * scratch slot per resident lane, w3 parked in x (k_scalar_f64_chunk); 1 w2
 * in the warp's shared memory, w3 parked in x; 2 both in shared memory
 * (k_scalar_f64_res).  Block kinds: 0 Gamma in an L2 scratch slot, 1 or 2
 * Gamma in the warp's shared memory (k_block_f64_ring<..., 1>).  Scalar
 * refinement (TG_PREC_F32_REFINE): 1 the warp's whole 32-column tile (FP64
 * a, b, c, f, x and the FP32 factors) in shared memory, so the coefficients
 * are read once for all sweeps (k_scalar_refine_tile).  On chip,
 * DRAM sees the coefficients read once, at the cost of fewer warps per SM.
 * -1 restores the default.  Columns too tall for shared memory take mode 0.
 * Same arithmetic, same bits. */
int tg_set_column_residency(int kind, int precision, int mode);

/* Fused assembly routines: 2 (default) three passes where built (dt_ng,
 * minor_ng, oplus_ng, settei_ng, and comp_ng on launches of up to 16384
 * columns): the level quantities and then the rows with one thread per
 * (level, column), then a column walk that is the recurrence alone (and
 * settei_ng's Te, Ti level-parallel again); 1 two passes, the level
 * quantities then a walk that forms the rows as it goes (comp_ng above
 * 16384 columns in mode 2 too); 0 one fused column walk.  Same operations,
 * same results. */
int tg_set_assembly_mode(int mode);

/* Fused assembly routines: how many levels ahead their column walks request
 * the reads of a level (n >= 1), or -1 (default) for automatic: 8 levels for
 * launches of up to 16384 columns, where few warps per SM leave every level
 * waiting on memory otherwise, 1 above.  Same results. */
int tg_set_walk_prefetch(int levels);

/* Block kinds, FP64: the budget for the Gamma scratch of all resident warps
 * of the block kernels, in MB (default 160; <= 0 restores it).  It caps
 * how many columns are in flight at once on large batches (the refinement
 * kernel is not capped). */
int tg_set_block_scratch_budget(double megabytes);

/* Scalar kind, FP64 ring kernels: the L2 budget for the w2 scratch and the
 * parked forward-sweep results (16 B per level and column) of all resident
 * columns, in MB (default 128; <= 0 restores it).  It caps how many columns
 * are in flight at once on large batches. */
int tg_set_scalar_scratch_budget(double megabytes);

/* How the kinds of one plan share the GPU, read when a plan is created: 1 the
 * block kinds run on a side stream beside the scalar kind (whose FP64 grid is
 * then halved, leaving the block warps, the long pole, more issue slots), 0
 * one kind after the other, any other value (default) side by side only when
 * every kind's tiles fit in one resident wave.  Same results either way. */
int tg_set_kind_overlap(int mode);

/* Host-array entries (tg_solve_host and the per-routine drop-ins): the input
 * bytes per pipelined column chunk, in KiB, and the number of streams the
 * chunks rotate over (1..8); <= 0 restores the defaults (streams 4; chunks of
 * a sixth of the call's input bytes, kept within 4..64 MiB).  Consecutive
 * chunks whose input arrays lie in one page-locked allocation, within a
 * region of up to max(chunk, 8 MiB) bytes, form a run whose inputs cross the
 * link in few copies instead of one per array: inputs that touch (gaps of up
 * to 4 KiB) in one copy, equal inputs at one pitch (systems of one shape,
 * each with its solution array between them) in one strided copy; nothing
 * but inputs and those small gaps is copied. */
int tg_set_host_pipeline(int chunk_kb, int streams);

/* Runs the ring kernels' bounded mbarrier wait on a barrier that nothing
 * completes, giving up after `polls` polls (1..2^22): *status_dev receives
 * TG_ETIMEOUT, as a solve does when a bulk copy never lands.  Tests the
 * timeout path without a stuck copy or a fault. */
int tg_selftest_wait(unsigned polls, int *status_dev, void *stream);
/* Test entry: q[i] = a[i]/b[i] (device arrays, n elements) computed by the
 * kernels' division routine (Markstein's correction of the correctly rounded
 * reciprocal, IEEE division outside its safe range); must equal IEEE a/b. */
int tg_selftest_division(const double *a, const double *b, double *q, long n, void *stream);
/* Test entry: one column walk of the assembly routines on rows the caller
 * formed, level-major (k*ld + col) device planes of nk*ld doubles.
 *   which 0: the Thomas walk of the three-pass routines: buf holds five
 *            planes p, q, r, f, x; rows 0..K-1 are solved into x (top = 1:
 *            K = nk-1 and x(nk-1) = x(nk-2)**2/x(nk-3)).
 *   which 1: oplus_ng's factor pass: buf is a factor buffer of
 *            tg_oplus_ng_factor_doubles(nk, ld) doubles whose p, q, r planes
 *            (planes 6, 7, 8 of nk*ld; rows 0..nk-2) the caller filled; the
 *            pass writes w1 (plane 10), 1/w1 (plane 11) and w2 (plane 12,
 *            rows 0..nk-3).
 * Launches of up to 16384 columns take the shared-memory tile walks, larger
 * ones the walks that read global memory; both give the same bits.
 * *status_dev receives the walk's status (TG_EPIVOT, TG_ENONFINITE). */
int tg_selftest_walk(int which, double *buf, int nk, int K, int top, int ncol, long ld, int *status_dev,
                     void *stream);
/* Frees the per-device mirrors, work buffers and streams. */
int tg_release_buffers(void);
/* Library version, e.g. "tg_colsolve 0.1.0 sm_100a". */
const char *tg_version(void);
/* The SASS target the library's kernels run as on the current device, as
 * major*10 + minor (100 for sm_100a); TG_ENODEV without a device. */
int tg_kernel_arch(int *arch);
/* Message of the last failing call on this thread. */
const char *tg_last_error(void);

#ifdef __cplusplus
}
#endif
#endif /* TG_COLSOLVE_H */
