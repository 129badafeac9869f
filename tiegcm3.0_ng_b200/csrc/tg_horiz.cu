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
#include <cmath>

#include "tg_internal.h"
#include "tg_arith.cuh"

namespace tg {
namespace {

constexpr int kTx = 32, kTy = 8;

struct AdvecRcp {
    double r3, r12, rlam, rphi;  // correctly rounded 1/3, 1/12, 1/dlamda, 1/dphi
    int lam_safe, phi_safe;      // dlamda, dphi inside the Markstein range
};

// a/b correctly rounded, y the reciprocal of b, b known to be in range
__device__ __forceinline__ double qdiv_by(double a, double b, double y, bool b_safe)
{
    return b_safe && exp_safe(a) ? div_markstein(a, b, y) : __ddiv_rn(a, b);
}

// One direction of advec_ng (:33-37 lon, :44-48 lat) at index t of an axis
// of n points with element stride s (p: the field, u: the wind, both at the
// point).  df_3d and fm_3d (src/dffm_ng.F90:66-110, :166-205) of order 1 are
// (p[+1]-p[-1])/2 and (u[+1]+u[-1])/2 inside, and on the edge rows the
// one-sided difference and the value itself; with the neighbour indices
// clamped into the axis, p[+1]-p[-1] is the one-sided difference there.  The
// term is dfdx1*2*2/3*ubar1 - dfdx2*4/12*ubar2 on rows 2..n-3 (where the
// order-2 helpers take their centred form) and dfdx1*ubar1 on the two ghost
// rows of each boundary side.  (d*2)*2 is d*4 exactly; x/2 and x/4 are the
// same numbers as x*0.5 and x*0.25.
__device__ __forceinline__ double advec_dir(const double *p, const double *u, int t, int n, int s,
                                            const AdvecRcp &rc)
{
    const int dm = t > 0 ? -s : 0, dp = t < n - 1 ? s : 0;
    const bool edge = t == 0 || t == n - 1;
    const double dif = xsub(__ldg(p + dp), __ldg(p + dm));
    const double d1 = edge ? dif : xmul(dif, 0.5);
    const double m1 = edge ? __ldg(u) : xmul(xadd(__ldg(u + dp), __ldg(u + dm)), 0.5);
    if (t <= 1 || t >= n - 2) return xmul(d1, m1);
    const double d2 = xmul(xsub(__ldg(p + 2 * s), __ldg(p - 2 * s)), 0.25);
    const double m2 = xmul(xadd(__ldg(u + 2 * s), __ldg(u - 2 * s)), 0.5);
    const double lhs = xmul(qdiv_by(xmul(d1, 4.0), 3.0, rc.r3, true), m1);
    const double rhs = xmul(qdiv_by(xmul(d2, 4.0), 12.0, rc.r12, true), m2);
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
    const double wk1 = xmul(advec_dir(f + o, un + o, i, nlond, 1, rc), __ldg(racs + j));
    const double wk2 = advec_dir(f + o, vn + o, j, nlatd, nlond, rc);
    // hadvec = wk1/dlamda + wk2*re_inv/dphi (:50)
    hadvec[o] = xadd(qdiv_by(wk1, dlamda, rc.rlam, rc.lam_safe), qdiv_by(xmul(wk2, re_inv), dphi, rc.rphi, rc.phi_safe));
}

// One Shapiro pass of smooth_ng along an axis (lat :18-29, lon :31-42) at
// index t of n points, stride s: x - sh*(2*fm2 - 8*fm1 + 6*x) inside,
// x - sh*(-8*fm1 + 8*x) one row in from a boundary (written 8*x - 8*fm1,
// the same rounded number), x on the outermost ghost row.  Where they are
// used, fm1 and fm2 are the plain +-1 and +-2 means.
__device__ __forceinline__ double shapiro_at(const double *p, int t, int n, int s, double sh)
{
    const double x = p[0];
    if (t == 0 || t == n - 1) return x;
    const double m1 = xmul(xadd(p[s], p[-s]), 0.5);
    if (t == 1 || t == n - 2) return xsub(x, xmul(sh, xsub(xmul(8.0, x), xmul(8.0, m1))));
    const double m2 = xmul(xadd(p[2 * s], p[-2 * s]), 0.5);
    return xsub(x, xmul(sh, xadd(xsub(xmul(2.0, m2), xmul(8.0, m1)), xmul(6.0, x))));
}

// The lat pass lands in a shared tile of the block's 8 rows x (32 + 4)
// longitudes (the lon pass needs +-2 neighbours): its 288 points are dealt
// to the 256 threads in order, so only one warp takes a second point.  Then
// the lon pass reads the tile.
__global__ void __launch_bounds__(kTx * kTy) k_smooth_ng(const double *fin, double sh, int nlond, int nlatd,
                                                        long ld, double *fout)
{
    constexpr int W = kTx + 4;
    __shared__ double ft[kTy][W + 1];
    const int i0 = blockIdx.x * kTx, j0 = blockIdx.y * kTy;
    const double *plane = fin + (long)blockIdx.z * ld;
    for (int q = threadIdx.y * kTx + threadIdx.x; q < W * kTy; q += kTx * kTy) {
        const int r = q / W, c = q - r * W;
        const int i = i0 - 2 + c, j = j0 + r;
        if (i < 0 || i >= nlond || j >= nlatd) continue;
        ft[r][c] = shapiro_at(plane + i + (long)nlond * j, j, nlatd, nlond, sh);
    }
    __syncthreads();
    const int i = i0 + threadIdx.x, j = j0 + threadIdx.y;
    if (i >= nlond || j >= nlatd) return;
    // every longitude the lon pass reads (i-2..i+2 where used) is in the tile
    fout[(long)blockIdx.z * ld + i + (long)nlond * j] = shapiro_at(&ft[threadIdx.y][threadIdx.x + 2], i, nlond, 1, sh);
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
    auto in_range = [](double b) { return std::fabs(b) >= 0x1p-500 && std::fabs(b) < 0x1p500; };
    const AdvecRcp rc{1.0 / 3.0, 1.0 / 12.0, 1.0 / dlamda, 1.0 / dphi, in_range(dlamda), in_range(dphi)};
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
