// The polar ring filter (src/ringfilter.F:1-111) on the whole global grid
// held on one device, as filter_o2o (src/comp.F:1065-1145) applies it after
// gathering the longitudes: on one GPU the longitude gather is a read of the
// row, so there is no MPI step.
//
// Layout: level-major planes, element (k, i, j) at k*ld + i + (nlon+4)*j,
// i = 0..nlon+3 the longitude (interior 2..nlon+1, two periodic points on
// each side), j = 0..nlat-1 the latitude.
//
// One warp per (filtered latitude, level) row of nlon values.  The row is
// read into shared memory once (coalesced: consecutive longitudes are
// consecutive addresses).  Every sum runs in longitude order, as the
// reference's loops do: the 2*order+1 Fourier sums are independent chains,
// one lane each; the chunk means are one lane per chunk; the reconstruction
// and the write-back are one lane per longitude.  The cos/sin values come
// from a table the host fills with the C library's cos and sin of the same
// arguments (m * (i * dlamda)), and every product and sum is rounded on its
// own (no FMA contraction), so the result is bit-identical to the reference
// arithmetic.
#include <cuda_runtime.h>

#include <cmath>
#include <mutex>
#include <vector>

#include "tg_internal.h"
#include "tg_arith.cuh"

namespace tg {

namespace {

constexpr int kRowsPerBlock = 4;

__global__ void __launch_bounds__(32 * kRowsPerBlock) k_ringfilter(RingRows rows, double *f, long ld, int nk,
                                                                   int nlon, int order, int poly,
                                                                   const double *cs, const double *sn)
{
    extern __shared__ __align__(16) double smem_rf[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const long r = (long)blockIdx.x * kRowsPerBlock + warp;
    if (r >= (long)rows.n * nk) return;
    const int slot = (int)(r / nk), k = (int)(r % nk);
    const int j = rows.lat[slot], nchnk = rows.nchnk[slot];
    const int nlonp4 = nlon + 4;
    // per warp: w (becomes fx), wm, avg (nlon each), series coefficients
    double *w = smem_rf + (long)warp * (3 * nlon + 2 * kMaxRingOrder + 1);
    double *wm = w + nlon, *avg = wm + nlon, *coef = avg + nlon;   // coef: a0, a(1..order), b(1..order)
    double *row = f + (long)k * ld + (long)nlonp4 * j;
    for (int i = lane; i < nlon; i += 32) w[i] = row[i + 2];
    __syncwarp();
    // the Fourier sums: lane 0 the mean, lanes 1..order a(m), the next
    // order lanes b(m), each over i = 1..nlon in order
    if (lane <= 2 * order) {
        double s = 0.0;
        if (lane == 0) {
            for (int i = 0; i < nlon; ++i) s = xadd(s, w[i]);
            s = xdiv(s, (double)nlon);
        } else {
            const double *tab = lane <= order ? cs + (long)(lane - 1) * nlon : sn + (long)(lane - order - 1) * nlon;
            for (int i = 0; i < nlon; ++i) s = xadd(s, xmul(w[i], tab[i]));
            s = xdiv(xmul(2.0, s), (double)nlon);
        }
        coef[lane] = s;
    }
    __syncwarp();
    // the series as the mean, and the deviation (kept in w)
    const double a0 = coef[0];
    for (int i = lane; i < nlon; i += 32) {
        double v = a0;
        for (int m = 0; m < order; ++m)
            v = xadd(xadd(v, xmul(coef[1 + m], cs[(long)m * nlon + i])), xmul(coef[1 + order + m], sn[(long)m * nlon + i]));
        wm[i] = v;
        w[i] = xsub(w[i], v);
    }
    __syncwarp();
    // chunk means, one lane per chunk
    const int n = nlon / nchnk;
    for (int c = lane; c < nchnk; c += 32) {
        double s = 0.0;
        for (int i = c * n; i < (c + 1) * n; ++i) s = xadd(s, w[i]);
        avg[c] = xdiv(s, (double)n);
    }
    __syncwarp();
    // reconstruction within each chunk from its neighbours' means
    // (periodic in longitude), then the full field and the periodic points
    for (int i = lane; i < nlon; i += 32) {
        double x = w[i];
        const int c = i / n;
        if (c < nchnk) {
            const int m = i - c * n + 1;
            const int im2 = (c - 2 + 2 * nchnk) % nchnk, im1 = (c - 1 + nchnk) % nchnk, ip1 = (c + 1) % nchnk,
                      ip2 = (c + 2) % nchnk;
            const double av = avg[c];
            const double left = xdiv(xsub(xadd(xadd(-avg[im2], xmul(7.0, avg[im1])), xmul(7.0, av)), avg[ip1]), 12.0);
            const double right = xdiv(xsub(xadd(xadd(-avg[im1], xmul(7.0, av)), xmul(7.0, avg[ip1])), avg[ip2]), 12.0);
            if (poly) {
                const double fa = xdiv(xsub(xadd(left, right), xmul(2.0, av)), (double)(n * n));
                const double fb = xdiv(xsub(xsub(xmul(3.0, av), xmul(2.0, left)), right), (double)n);
                const double p = xadd(xsub(xmul(3.0, (double)(m * m)), xmul(3.0, (double)m)), 1.0);
                x = xadd(xadd(xmul(fa, p), xmul(fb, xsub(xmul(2.0, (double)m), 1.0))), left);
            } else {
                x = xdiv(xadd(xmul(left, (double)(n - m)), xmul(right, (double)m)), (double)n);
            }
        }
        w[i] = xadd(x, wm[i]);
        row[i + 2] = w[i];
    }
    __syncwarp();
    if (lane == 0) {
        row[0] = w[nlon - 2];
        row[1] = w[nlon - 1];
        row[nlon + 2] = w[0];
        row[nlon + 3] = w[1];
    }
}

// cos(m*(i*dlamda)) and sin(...) for m = 1..order, i = 1..nlon, computed on
// the host with the C library.  One table per (device, nlon, order, dlamda)
// asked for, built on first use (a synchronous upload) and kept until the
// process exits: the model filters a handful of fields with two orders.
struct TrigTable {
    int dev, nlon, order;
    double dlamda;
    double *d;   // cos rows then sin rows
};
std::vector<TrigTable> g_trig;
std::mutex g_trig_mu;

cudaError_t trig_table(int nlon, int order, double dlamda, const double **cs, const double **sn)
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    std::lock_guard<std::mutex> lk(g_trig_mu);
    for (const TrigTable &t : g_trig)
        if (t.dev == dev && t.nlon == nlon && t.order == order && t.dlamda == dlamda) {
            *cs = t.d;
            *sn = t.d + (size_t)order * nlon;
            return cudaSuccess;
        }
    std::vector<double> h(2 * (size_t)order * nlon);
    for (int m = 1; m <= order; ++m)
        for (int i = 1; i <= nlon; ++i) {
            const double ang = i * dlamda;
            h[(size_t)(m - 1) * nlon + (i - 1)] = std::cos(m * ang);
            h[((size_t)order + m - 1) * nlon + (i - 1)] = std::sin(m * ang);
        }
    TrigTable t{dev, nlon, order, dlamda, nullptr};
    if ((e = cudaMalloc(&t.d, sizeof(double) * h.size())) != cudaSuccess) return e;
    if ((e = cudaMemcpy(t.d, h.data(), sizeof(double) * h.size(), cudaMemcpyHostToDevice)) != cudaSuccess) {
        cudaFree(t.d);
        return e;
    }
    g_trig.push_back(t);
    *cs = t.d;
    *sn = t.d + (size_t)order * nlon;
    return cudaSuccess;
}

}  // namespace

size_t ringfilter_smem_bytes(int nlon) { return sizeof(double) * kRowsPerBlock * (3 * (size_t)nlon + 2 * kMaxRingOrder + 1); }

cudaError_t launch_ringfilter(const RingRows &rows, double *f, long ld, int nk, int nlon, int order, int poly,
                              double dlamda, cudaStream_t st)
{
    if (rows.n <= 0 || nk <= 0) return cudaSuccess;
    const double *cs = nullptr, *sn = nullptr;
    cudaError_t e = trig_table(nlon, order, dlamda, &cs, &sn);
    if (e != cudaSuccess) return e;
    const size_t smem = ringfilter_smem_bytes(nlon);
    if (smem > (size_t)(smem_optin() - 1024)) return cudaErrorInvalidValue;
    once_per_device(
        [] { cudaFuncSetAttribute(k_ringfilter, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_optin() - 1024); });
    const long nrows = (long)rows.n * nk;
    const int blocks = (int)((nrows + kRowsPerBlock - 1) / kRowsPerBlock);
    k_ringfilter<<<blocks, 32 * kRowsPerBlock, smem, st>>>(rows, f, ld, nk, nlon, order, poly, cs, sn);
    return cudaGetLastError();
}

}  // namespace tg
