// Horizontal operators that feed the column assembly: advec_ng
// (src/advec_ng.F90) and smooth_ng (src/smooth_ng.F90), over one nest held as
// a single subdomain.  Every lateral edge is then a boundary (is_bndry all
// true, src/fields_ng.F90:143-147) and the halo syncs of src/sync_ng.F90
// exchange nothing, so the operators are plain stencils over the
// ghost-inclusive (nlon+4) x (nlat+4) plane of each level.
//
// Layout: level-major planes, (k, i, j) at k*ld + i + nlond*j with
// nlond = nlon+4, i.e. the column index of the other device entries.  One
// thread per point; a block covers 32 longitudes x 8 latitudes of one level
// (blockIdx.z), so the lat neighbours are rows that the block's other warps
// bring into L1.
//
// Arithmetic follows the reference's operation order with separately rounded
// operations.  Divisions by 2 and 4 are written as multiplications by 0.5
// and 0.25 (the same correctly rounded number); divisions by 3, 12, dlamda
// and dphi are correctly rounded (qdiv with the reciprocal from the host).
#include "tg_internal.h"
#include "tg_arith.cuh"

namespace tg {
namespace {

constexpr int kTx = 32, kTy = 8;

// a point's index along one axis, the axis extent and the element stride
struct Axis {
    int t, n;
    long s;
};

// fm_3d (src/dffm_ng.F90:166-205): the centred mean over +-O points, the
// input itself on the edge rows, the +-1 mean on the rows next to them (O=2).
template <int O>
__device__ __forceinline__ double fm_at(const double *p, Axis a)
{
    if (a.t == 0 || a.t == a.n - 1) return __ldg(p);
    const long d = (O == 2 && (a.t == 1 || a.t == a.n - 2)) ? a.s : O * a.s;
    return xmul(xadd(__ldg(p + d), __ldg(p - d)), 0.5);
}

// df_3d (src/dffm_ng.F90:66-110): the centred difference over 2*O spacings,
// one-sided on the edge rows, over 2 spacings on the rows next to them (O=2).
template <int O>
__device__ __forceinline__ double df_at(const double *p, Axis a)
{
    if (a.t == 0) return xsub(__ldg(p + a.s), __ldg(p));
    if (a.t == a.n - 1) return xsub(__ldg(p), __ldg(p - a.s));
    if (O == 2 && (a.t == 1 || a.t == a.n - 2)) return xmul(xsub(__ldg(p + a.s), __ldg(p - a.s)), 0.5);
    return xmul(xsub(__ldg(p + O * a.s), __ldg(p - O * a.s)), O == 1 ? 0.5 : 0.25);
}

struct AdvecRcp {
    double r3, r12, rlam, rphi;  // correctly rounded 1/3, 1/12, 1/dlamda, 1/dphi
};

// One direction of advec_ng (:33-37 lon, :44-48 lat): the fourth-order term
// dfdx1*2*2/3*ubar1 - dfdx2*4/12*ubar2, and dfdx1*ubar1 on the two ghost
// rows of a boundary side.  (d*2)*2 is d*4 exactly.
__device__ __forceinline__ double advec_dir(const double *f, const double *u, Axis a, const AdvecRcp &rc)
{
    const double d1 = df_at<1>(f, a), m1 = fm_at<1>(u, a);
    if (a.t <= 1 || a.t >= a.n - 2) return xmul(d1, m1);
    const double d2 = df_at<2>(f, a), m2 = fm_at<2>(u, a);
    const double lhs = xmul(qdiv(xmul(d1, 4.0), 3.0, rc.r3), m1);
    const double rhs = xmul(qdiv(xmul(d2, 4.0), 12.0, rc.r12), m2);
    return xsub(lhs, rhs);
}

__global__ void __launch_bounds__(kTx * kTy) k_advec_ng(const double *f, const double *un, const double *vn,
                                                       const double *racs, double dlamda, double dphi,
                                                       double re_inv, AdvecRcp rc, int nlond, int nlatd, long ld,
                                                       double *hadvec)
{
    const int i = blockIdx.x * kTx + threadIdx.x, j = blockIdx.y * kTy + threadIdx.y;
    if (i >= nlond || j >= nlatd) return;
    const long o = (long)blockIdx.z * ld + i + (long)nlond * j;
    const double wk1 = xmul(advec_dir(f + o, un + o, Axis{i, nlond, 1}, rc), __ldg(racs + j));
    const double wk2 = advec_dir(f + o, vn + o, Axis{j, nlatd, nlond}, rc);
    // hadvec = wk1/dlamda + wk2*re_inv/dphi (:50)
    hadvec[o] = xadd(qdiv(wk1, dlamda, rc.rlam), qdiv(xmul(wk2, re_inv), dphi, rc.rphi));
}

// One Shapiro pass of smooth_ng along an axis (lat :18-29, lon :31-42):
// x - sh*(2*fm2 - 8*fm1 + 6*x) inside, x - sh*(-8*fm1 + 8*x) one row in from
// a boundary (written 8*x - 8*fm1, the same rounded number), x on the
// outermost ghost row.
template <class Load>
__device__ __forceinline__ double shapiro_at(Load ld, int t, int n, double sh)
{
    const double x = ld(0);
    if (t == 0 || t == n - 1) return x;
    const double m1 = xmul(xadd(ld(1), ld(-1)), 0.5);
    if (t == 1 || t == n - 2) return xsub(x, xmul(sh, xsub(xmul(8.0, x), xmul(8.0, m1))));
    const double m2 = xmul(xadd(ld(2), ld(-2)), 0.5);
    return xsub(x, xmul(sh, xadd(xsub(xmul(2.0, m2), xmul(8.0, m1)), xmul(6.0, x))));
}

// The lat pass lands in a shared tile of the block's 8 rows x (32 + 4)
// longitudes (the lon pass needs +-2 neighbours), then the lon pass reads it.
__global__ void __launch_bounds__(kTx * kTy) k_smooth_ng(const double *fin, double sh, int nlond, int nlatd,
                                                        long ld, double *fout)
{
    __shared__ double ft[kTy][kTx + 4 + 1];
    const int i0 = blockIdx.x * kTx, j = blockIdx.y * kTy + threadIdx.y;
    const double *plane = fin + (long)blockIdx.z * ld;
    if (j < nlatd) {
        for (int c = threadIdx.x; c < kTx + 4; c += kTx) {
            const int i = i0 - 2 + c;
            if (i < 0 || i >= nlond) continue;
            const double *p = plane + i + (long)nlond * j;
            ft[threadIdx.y][c] = shapiro_at([&](int d) { return __ldg(p + (long)d * nlond); }, j, nlatd, sh);
        }
    }
    __syncthreads();
    const int i = i0 + threadIdx.x;
    if (i >= nlond || j >= nlatd) return;
    const double *row = &ft[threadIdx.y][threadIdx.x + 2];
    fout[(long)blockIdx.z * ld + i + (long)nlond * j] = shapiro_at([&](int d) { return row[d]; }, i, nlond, sh);
}

dim3 plane_grid(int nk, int nlond, int nlatd)
{
    return dim3((unsigned)((nlond + kTx - 1) / kTx), (unsigned)((nlatd + kTy - 1) / kTy), (unsigned)nk);
}

}  // namespace

cudaError_t launch_advec_ng(const double *f, const double *un, const double *vn, const double *racs, double dlamda,
                            double dphi, double re_inv, int nk, int nlon, int nlat, long ld, double *hadvec,
                            cudaStream_t st)
{
    const int nlond = nlon + 4, nlatd = nlat + 4;
    // host IEEE division: the correctly rounded reciprocals the Markstein step needs
    const AdvecRcp rc{1.0 / 3.0, 1.0 / 12.0, 1.0 / dlamda, 1.0 / dphi};
    k_advec_ng<<<plane_grid(nk, nlond, nlatd), dim3(kTx, kTy), 0, st>>>(f, un, vn, racs, dlamda, dphi, re_inv, rc,
                                                                        nlond, nlatd, ld, hadvec);
    return cudaGetLastError();
}

cudaError_t launch_smooth_ng(const double *fin, double shapiro, int nk, int nlon, int nlat, long ld, double *fout,
                             cudaStream_t st)
{
    const int nlond = nlon + 4, nlatd = nlat + 4;
    k_smooth_ng<<<plane_grid(nk, nlond, nlatd), dim3(kTx, kTy), 0, st>>>(fin, shapiro, nlond, nlatd, ld, fout);
    return cudaGetLastError();
}

}  // namespace tg
