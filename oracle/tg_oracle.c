/*
 * CPU oracle for the TIE-GCM NG vertical column solves.
 *
 * TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and the
 * cpu_baseline / --impl reference legs of bench.py load this library, and only
 * as the checker or the timed CPU baseline.  The product (the CUDA C-ABI
 * library) never links or calls it.
 *
 * Parity status: the reference is Fortran and no Fortran compiler exists in
 * this image, and the reference ships no tests, golden vectors or fixtures for
 * this path.  Parity of this restatement against the reference itself is
 * therefore UNPINNED; it is pinned instead against independent solvers (LAPACK
 * banded / dense solves), manufactured solutions and a long-double restatement
 * (tests/test_oracle.py, tests/golden/).
 *
 * Every routine restates the reference's arithmetic in the reference's own
 * operation order (separate multiply, subtract and IEEE divide; build with
 * -ffp-contract=off so no FMA is formed), so that a GPU kernel that uses the
 * same order and non-contracting intrinsics reproduces it bit for bit.
 *
 * Layouts (all column-major like the Fortran caller):
 *   scalar arrays   (nk, ncol)        element (k,col)   at k + nk*col
 *   block  matrices (B, B, nk, ncol)  element (i,j,k,col) at i + B*j + B*B*k + B*B*nk*col
 *   block  vectors  (B, nk, ncol)     element (i,k,col)   at i + B*k + B*nk*col
 * Row indices in the argument lists (k2, k1, lev0 ...) are 1-based as in the
 * reference.
 */
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define ORACLE_API __attribute__((visibility("default")))

/* ------------------------------------------------------------------------ */
/* Scalar Thomas solve, trsolv_ng semantics (src/trsolv_ng.F90:14-26).       */
/* ------------------------------------------------------------------------ */

/* One column.  w holds 3*k2 doubles of work (w1, w2, w3 of the reference). */
static void thomas_column(const double *a, const double *b, const double *c,
                          const double *f, double *x, int k2, double *w)
{
    double *w1 = w, *w2 = w + k2, *w3 = w + 2 * k2;
    int k;
    /* w1(1) = b(1)                                   trsolv_ng.F90:14 */
    w1[0] = b[0];
    /* w2(k-1) = c(k-1)/w1(k-1); w1(k) = b(k)-a(k)*w2(k-1)   :15-18 */
    for (k = 1; k < k2; ++k) {
        w2[k - 1] = c[k - 1] / w1[k - 1];
        w1[k] = b[k] - a[k] * w2[k - 1];
    }
    /* w3(1) = f(1)/w1(1)                                     :19 */
    w3[0] = f[0] / w1[0];
    /* w3(k) = (f(k)-a(k)*w3(k-1))/w1(k)                      :20-22 */
    for (k = 1; k < k2; ++k)
        w3[k] = (f[k] - a[k] * w3[k - 1]) / w1[k];
    /* x(k2) = w3(k2); x(k) = w3(k)-w2(k)*x(k+1)              :23-26 */
    x[k2 - 1] = w3[k2 - 1];
    for (k = k2 - 2; k >= 0; --k)
        x[k] = w3[k] - w2[k] * x[k + 1];
}

/* trsolv_ng(a,b,c,f,x,k2,i_ng) over ncol columns of leading dimension nk.
 * Rows k2+1..nk of x are not written (the reference leaves them undefined). */
ORACLE_API void oracle_trsolv_ng(const double *a, const double *b, const double *c,
                                 const double *f, double *x, int nk, int k2,
                                 long ncol, int nthreads)
{
    if (k2 < 1 || k2 > nk || ncol <= 0) return;
    if (nthreads < 1) nthreads = 1;
#pragma omp parallel num_threads(nthreads)
    {
        double *w = (double *)malloc(sizeof(double) * 3 * (size_t)k2);
        long col;
#pragma omp for schedule(static)
        for (col = 0; col < ncol; ++col) {
            size_t o = (size_t)nk * (size_t)col;
            thomas_column(a + o, b + o, c + o, f + o, x + o, k2, w);
        }
        free(w);
    }
}

/* Same algorithm in long double (x87 extended) rounded to double at the end:
 * the "truth" used for error budgets, not a parity target. */
ORACLE_API void oracle_trsolv_ng_ld(const double *a, const double *b, const double *c,
                                    const double *f, double *x, int nk, int k2,
                                    long ncol)
{
    long double *w1, *w2, *w3, *xx;
    long col;
    int k;
    if (k2 < 1 || k2 > nk || ncol <= 0) return;
    w1 = (long double *)malloc(sizeof(long double) * 4 * (size_t)k2);
    w2 = w1 + k2; w3 = w2 + k2; xx = w3 + k2;
    for (col = 0; col < ncol; ++col) {
        size_t o = (size_t)nk * (size_t)col;
        const double *A = a + o, *B = b + o, *C = c + o, *F = f + o;
        w1[0] = B[0];
        for (k = 1; k < k2; ++k) {
            w2[k - 1] = (long double)C[k - 1] / w1[k - 1];
            w1[k] = (long double)B[k] - (long double)A[k] * w2[k - 1];
        }
        w3[0] = (long double)F[0] / w1[0];
        for (k = 1; k < k2; ++k)
            w3[k] = ((long double)F[k] - (long double)A[k] * w3[k - 1]) / w1[k];
        xx[k2 - 1] = w3[k2 - 1];
        for (k = k2 - 2; k >= 0; --k) xx[k] = w3[k] - w2[k] * xx[k + 1];
        for (k = 0; k < k2; ++k) x[o + k] = (double)xx[k];
    }
    free(w1);
}

/* ------------------------------------------------------------------------ */
/* trsolv (global grid, one latitude slab), src/trsolv.F:2-101.              */
/* Arrays are (lev0:lev1, lon0:lon1).  Columns 1,2 and lonmax-1,lonmax are    */
/* skipped when the slab touches the periodic edges (trsolv.F:32-35).  The    */
/* reference initialises w1(lev0) (trsolv.F:38-40) and then reads w1(k1);    */
/* every caller passes k1 == lev0, the only case it defines.  Here w1(k1) =   */
/* b(k1), which coincides with it whenever k1 == lev0.                        */
/* ------------------------------------------------------------------------ */
ORACLE_API void oracle_trsolv(const double *a, const double *b, const double *c,
                              const double *f, double *x, int lev0, int lev1, int k1,
                              int k2, int lon0, int lon1, int lonmax)
{
    int nlev = lev1 - lev0 + 1, lonbeg = lon0, lonend = lon1, i, n;
    double *w;
    if (nlev < 1 || k1 < lev0 || k2 > lev1 || k2 < k1) return;
    if (lon0 == 1) lonbeg = 3;
    if (lon1 == lonmax) lonend = lon1 - 2;
    n = k2 - k1 + 1;
    w = (double *)malloc(sizeof(double) * 3 * (size_t)n);
    for (i = lonbeg; i <= lonend; ++i) {
        size_t o = (size_t)nlev * (size_t)(i - lon0) + (size_t)(k1 - lev0);
        thomas_column(a + o, b + o, c + o, f + o, x + o, n, w);
    }
    free(w);
}

/* ------------------------------------------------------------------------ */
/* Small-matrix inverses, src/matutil.F90:9-118 (adjugate / determinant, no   */
/* pivoting).  Column-major: A(i,j) = A[(i-1) + n*(j-1)].                    */
/* ------------------------------------------------------------------------ */
#define M3(A, i, j) (A)[((i) - 1) + 3 * ((j) - 1)]
#define M2(A, i, j) (A)[((i) - 1) + 2 * ((j) - 1)]

ORACLE_API void oracle_matinv3(const double *A, double *Bo)
{
    /* matdet3, matutil.F90:25-27, evaluated left to right */
    double d = M3(A,1,1)*M3(A,2,2)*M3(A,3,3) - M3(A,1,1)*M3(A,2,3)*M3(A,3,2)
             - M3(A,1,2)*M3(A,2,1)*M3(A,3,3) + M3(A,1,2)*M3(A,2,3)*M3(A,3,1)
             + M3(A,1,3)*M3(A,2,1)*M3(A,3,2) - M3(A,1,3)*M3(A,2,2)*M3(A,3,1);
    double adj[9];
    /* matadj3, matutil.F90:63-71 */
    M3(adj,1,1) =  (M3(A,2,2)*M3(A,3,3) - M3(A,2,3)*M3(A,3,2));
    M3(adj,2,1) = -(M3(A,2,1)*M3(A,3,3) - M3(A,2,3)*M3(A,3,1));
    M3(adj,3,1) =  (M3(A,2,1)*M3(A,3,2) - M3(A,2,2)*M3(A,3,1));
    M3(adj,1,2) = -(M3(A,1,2)*M3(A,3,3) - M3(A,1,3)*M3(A,3,2));
    M3(adj,2,2) =  (M3(A,1,1)*M3(A,3,3) - M3(A,1,3)*M3(A,3,1));
    M3(adj,3,2) = -(M3(A,1,1)*M3(A,3,2) - M3(A,1,2)*M3(A,3,1));
    M3(adj,1,3) =  (M3(A,1,2)*M3(A,2,3) - M3(A,1,3)*M3(A,2,2));
    M3(adj,2,3) = -(M3(A,1,1)*M3(A,2,3) - M3(A,1,3)*M3(A,2,1));
    M3(adj,3,3) =  (M3(A,1,1)*M3(A,2,2) - M3(A,1,2)*M3(A,2,1));
    /* matinv3 = matadj3/matdet3, matutil.F90:116 */
    for (int e = 0; e < 9; ++e) Bo[e] = adj[e] / d;
}

ORACLE_API void oracle_matinv2(const double *A, double *Bo)
{
    /* matdet2 / matadj2 / matinv2, matutil.F90:15,50-53,106 */
    double d = M2(A,1,1)*M2(A,2,2) - M2(A,1,2)*M2(A,2,1);
    M2(Bo,1,1) =  M2(A,2,2) / d;
    M2(Bo,2,1) = -M2(A,2,1) / d;
    M2(Bo,1,2) = -M2(A,1,2) / d;
    M2(Bo,2,2) =  M2(A,1,1) / d;
}

/* ------------------------------------------------------------------------ */
/* Block-tridiagonal Thomas solve, B = 2 or 3.                               */
/*                                                                          */
/* Follows the comp_ng forward sweep (src/comp_ng.F90:281-314): with Gamma_1 */
/* = 0 and z_1 = 0, for rows k = 1..k2                                      */
/*   Q'      = Q_k - P_k Gamma_k            (n summed left to right, :281-287) */
/*   W       = inv(Q')                      (matinv3/matinv2, :289-293)      */
/*   Gamma'  = W R_k                        (:296-306)                       */
/*   z'      = W (f_k - P_k z_k)            (:295-313)                       */
/* and the back sweep u_k = z_{k+1} - Gamma_{k+1} u_{k+1} (:317-326).  The    */
/* duv.F blktri 2x2 solver (src/duv.F:801-908) performs the same operations   */
/* in the same order (its GAMMA(K) = B - A GAMMA(K-1), BETA = adj/det,        */
/* Y = BETA (F - A Y)), so B = 2 reproduces blktri.                           */
/* P of row 1 and R of row k2 are not referenced: the callers zero them       */
/* (comp_ng.F90:258,278; duv.F:336-339) and blktri never reads them.          */
/* If ubc_ratio is given, row k2+1 is filled as in comp_ng.F90:328-332:       */
/*   u(k2+1,i) = ubc_ratio(i,col)*u(k2,i) + ubc_add(i,col)   (ubc_add may be  */
/*   NULL, meaning zero).  ubc arrays are (B, ncol).                          */
/* ------------------------------------------------------------------------ */
static void blk_inv(int B, const double *A, double *W)
{
    if (B == 3) oracle_matinv3(A, W);
    else oracle_matinv2(A, W);
}

static void blk_column(int B, const double *P, const double *Q, const double *R,
                       const double *f, double *u, int nk, int k2,
                       const double *ratio, const double *add, double *G, double *Z)
{
    /* G: (B,B,k2+1) Gamma_1..Gamma_{k2+1}; Z: (B,k2+1) z_1..z_{k2+1} */
    int BB = B * B, k, i, m, n;
    double Qp[9], W[9], v[3];
    (void)nk;
    for (k = 0; k < k2; ++k) {
        const double *Pk = P + BB * k, *Qk = Q + BB * k, *Rk = R + BB * k, *fk = f + B * k;
        const double *Gk = G + BB * k, *zk = Z + B * k;
        double *Gn = G + BB * (k + 1), *zn = Z + B * (k + 1);
        for (m = 0; m < B; ++m)
            for (i = 0; i < B; ++i) {
                double q = Qk[i + B * m];
                if (k > 0)
                    for (n = 0; n < B; ++n) q = q - Pk[i + B * n] * Gk[n + B * m];
                Qp[i + B * m] = q;
            }
        blk_inv(B, Qp, W);
        for (i = 0; i < B; ++i) {
            double t = fk[i];
            if (k > 0)
                for (m = 0; m < B; ++m) t = t - Pk[i + B * m] * zk[m];
            v[i] = t;
        }
        for (m = 0; m < B; ++m)
            for (i = 0; i < B; ++i) {
                double g = 0.0;
                if (k < k2 - 1) {
                    g = W[i] * Rk[0 + B * m];
                    for (n = 1; n < B; ++n) g = g + W[i + B * n] * Rk[n + B * m];
                }
                Gn[i + B * m] = g;
            }
        for (i = 0; i < B; ++i) {
            double t = W[i] * v[0];
            for (m = 1; m < B; ++m) t = t + W[i + B * m] * v[m];
            zn[i] = t;
        }
    }
    /* back sweep */
    for (i = 0; i < B; ++i) u[i + B * (k2 - 1)] = Z[i + B * k2];
    for (k = k2 - 2; k >= 0; --k) {
        const double *Gn = G + BB * (k + 1), *zn = Z + B * (k + 1);
        for (i = 0; i < B; ++i) {
            double t = zn[i];
            for (m = 0; m < B; ++m) t = t - Gn[i + B * m] * u[m + B * (k + 1)];
            u[i + B * k] = t;
        }
    }
    if (ratio) {
        for (i = 0; i < B; ++i) {
            double t = ratio[i] * u[i + B * (k2 - 1)];
            if (add) t = t + add[i];
            u[i + B * k2] = t;
        }
    }
}

ORACLE_API void oracle_blksolve(int B, const double *P, const double *Q, const double *R,
                                const double *f, double *u, int nk, int k2, long ncol,
                                const double *ubc_ratio, const double *ubc_add,
                                int nthreads)
{
    if ((B != 2 && B != 3) || k2 < 1 || k2 > nk || ncol <= 0) return;
    if (ubc_ratio && k2 >= nk) return;
    if (nthreads < 1) nthreads = 1;
#pragma omp parallel num_threads(nthreads)
    {
        double *G = (double *)malloc(sizeof(double) * (size_t)(B * B + B) * (size_t)(k2 + 1));
        double *Z = G + (size_t)B * B * (size_t)(k2 + 1);
        long col;
#pragma omp for schedule(static)
        for (col = 0; col < ncol; ++col) {
            size_t om = (size_t)B * B * nk * (size_t)col, ov = (size_t)B * nk * (size_t)col;
            blk_column(B, P + om, Q + om, R + om, f + ov, u + ov, nk, k2,
                       ubc_ratio ? ubc_ratio + (size_t)B * col : NULL,
                       ubc_add ? ubc_add + (size_t)B * col : NULL, G, Z);
        }
        free(G);
    }
}

/* blktri (src/duv.F:801-908): 2x2 blocks over rows lev0..lev1-1 of a slab
 * (2,2,lev0:lev1,lon0:lon1), periodic columns skipped as in duv.F:102-105
 * with nlonp4 the padded longitude count.  Only x is produced; the
 * reference's beta, gamma and y are its work arrays. */
ORACLE_API void oracle_blktri(const double *a, const double *b, const double *c,
                              const double *f, double *x, int lev0, int lev1, int lon0,
                              int lon1, int nlonp4)
{
    int nlev = lev1 - lev0 + 1, lonbeg = lon0, lonend = lon1, i;
    int k2 = nlev - 1;
    double *G, *Z;
    if (k2 < 1) return;
    if (lon0 == 1) lonbeg = 3;
    if (lon1 == nlonp4) lonend = nlonp4 - 2;
    G = (double *)malloc(sizeof(double) * 6 * (size_t)(k2 + 1));
    Z = G + 4 * (size_t)(k2 + 1);
    for (i = lonbeg; i <= lonend; ++i) {
        size_t om = (size_t)4 * nlev * (size_t)(i - lon0), ov = (size_t)2 * nlev * (size_t)(i - lon0);
        blk_column(2, a + om, b + om, c + om, f + ov, x + ov, nlev, k2, NULL, NULL, G, Z);
    }
    free(G);
}

/* Long-double block solve (same algorithm, extended precision): error-budget
 * truth for the block kernels. */
static void blk_inv_ld(int B, const long double *A, long double *W)
{
    if (B == 3) {
#define L3(X, i, j) (X)[((i) - 1) + 3 * ((j) - 1)]
        long double d = L3(A,1,1)*L3(A,2,2)*L3(A,3,3) - L3(A,1,1)*L3(A,2,3)*L3(A,3,2)
                      - L3(A,1,2)*L3(A,2,1)*L3(A,3,3) + L3(A,1,2)*L3(A,2,3)*L3(A,3,1)
                      + L3(A,1,3)*L3(A,2,1)*L3(A,3,2) - L3(A,1,3)*L3(A,2,2)*L3(A,3,1);
        L3(W,1,1) =  (L3(A,2,2)*L3(A,3,3) - L3(A,2,3)*L3(A,3,2)) / d;
        L3(W,2,1) = -(L3(A,2,1)*L3(A,3,3) - L3(A,2,3)*L3(A,3,1)) / d;
        L3(W,3,1) =  (L3(A,2,1)*L3(A,3,2) - L3(A,2,2)*L3(A,3,1)) / d;
        L3(W,1,2) = -(L3(A,1,2)*L3(A,3,3) - L3(A,1,3)*L3(A,3,2)) / d;
        L3(W,2,2) =  (L3(A,1,1)*L3(A,3,3) - L3(A,1,3)*L3(A,3,1)) / d;
        L3(W,3,2) = -(L3(A,1,1)*L3(A,3,2) - L3(A,1,2)*L3(A,3,1)) / d;
        L3(W,1,3) =  (L3(A,1,2)*L3(A,2,3) - L3(A,1,3)*L3(A,2,2)) / d;
        L3(W,2,3) = -(L3(A,1,1)*L3(A,2,3) - L3(A,1,3)*L3(A,2,1)) / d;
        L3(W,3,3) =  (L3(A,1,1)*L3(A,2,2) - L3(A,1,2)*L3(A,2,1)) / d;
#undef L3
    } else {
        long double d = A[0] * A[3] - A[2] * A[1];
        W[0] = A[3] / d; W[1] = -A[1] / d; W[2] = -A[2] / d; W[3] = A[0] / d;
    }
}

ORACLE_API void oracle_blksolve_ld(int B, const double *P, const double *Q, const double *R,
                                   const double *f, double *u, int nk, int k2, long ncol,
                                   const double *ubc_ratio, const double *ubc_add)
{
    int BB = B * B;
    long col;
    long double *G, *Z, *U;
    if ((B != 2 && B != 3) || k2 < 1 || k2 > nk || ncol <= 0) return;
    if (ubc_ratio && k2 >= nk) return;
    G = (long double *)malloc(sizeof(long double) * (size_t)(BB + 2 * B) * (size_t)(k2 + 2));
    Z = G + (size_t)BB * (k2 + 2);
    U = Z + (size_t)B * (k2 + 2);
    for (col = 0; col < ncol; ++col) {
        size_t om = (size_t)BB * nk * (size_t)col, ov = (size_t)B * nk * (size_t)col;
        const double *Pc = P + om, *Qc = Q + om, *Rc = R + om, *fc = f + ov;
        long double Qp[9], W[9], v[3];
        int k, i, m, n;
        for (k = 0; k < k2; ++k) {
            const long double *Gk = G + BB * k, *zk = Z + B * k;
            long double *Gn = G + BB * (k + 1), *zn = Z + B * (k + 1);
            for (m = 0; m < B; ++m)
                for (i = 0; i < B; ++i) {
                    long double q = Qc[BB * k + i + B * m];
                    if (k > 0)
                        for (n = 0; n < B; ++n) q -= (long double)Pc[BB * k + i + B * n] * Gk[n + B * m];
                    Qp[i + B * m] = q;
                }
            blk_inv_ld(B, Qp, W);
            for (i = 0; i < B; ++i) {
                long double t = fc[B * k + i];
                if (k > 0)
                    for (m = 0; m < B; ++m) t -= (long double)Pc[BB * k + i + B * m] * zk[m];
                v[i] = t;
            }
            for (m = 0; m < B; ++m)
                for (i = 0; i < B; ++i) {
                    long double g = 0.0L;
                    if (k < k2 - 1)
                        for (n = 0; n < B; ++n) g += W[i + B * n] * (long double)Rc[BB * k + n + B * m];
                    Gn[i + B * m] = g;
                }
            for (i = 0; i < B; ++i) {
                long double t = 0.0L;
                for (m = 0; m < B; ++m) t += W[i + B * m] * v[m];
                zn[i] = t;
            }
        }
        for (i = 0; i < B; ++i) U[i + B * (k2 - 1)] = Z[i + B * k2];
        for (k = k2 - 2; k >= 0; --k)
            for (i = 0; i < B; ++i) {
                long double t = Z[i + B * (k + 1)];
                for (m = 0; m < B; ++m) t -= G[BB * (k + 1) + i + B * m] * U[m + B * (k + 1)];
                U[i + B * k] = t;
            }
        for (k = 0; k < k2; ++k)
            for (i = 0; i < B; ++i) u[ov + i + B * k] = (double)U[i + B * k];
        if (ubc_ratio)
            for (i = 0; i < B; ++i) {
                long double t = (long double)ubc_ratio[B * col + i] * U[i + B * (k2 - 1)];
                if (ubc_add) t += ubc_add[B * col + i];
                u[ov + i + B * k2] = (double)t;
            }
    }
    free(G);
}

ORACLE_API int oracle_max_threads(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

/* ------------------------------------------------------------------------ */
/* dt_ng neutral-temperature column assembly + solve (src/dt_ng.F90:57-167). */
/* Fields are (nk, ncol); 2-D fields (ncol); expz, dift (nk).  The outputs   */
/* of the horizontal operators (horadv = advec_ng(tn), tnsmooth =            */
/* smooth_ng(tn_nm)) are inputs.  tlbc is the previous step's lower-boundary  */
/* Tn (the routine's tlbc argument, dt_ng.F90:126), t_lbc the current one.   */
/* p, q, r, rhs (may be NULL) receive rows 1..nk-1 of the assembled system  */
/* after the LBC fold; tn_upd rows 1..nk (row nk from dt_ng.F90:167).        */
/* ------------------------------------------------------------------------ */
typedef struct {
    double dz, dtx2inv, expzmid_inv, grav, p0, avo, gask, tsurplus, rmassinv_o1;
} oracle_dt_consts;

typedef struct {
    const double *tn, *tnsmooth, *horadv, *un, *vn, *o1, *mbar, *xnmbar, *scht, *schti, *cp, *kt, *km,
        *hdt, *qji_tn, *cool_imp, *cool_exp, *w, *qtotal, *rkm12;   /* (nk, ncol) */
    const double *tlbc, *t_lbc, *ulbc, *vlbc;                          /* (ncol)     */
    const double *expz, *dift;                                         /* (nk)       */
} oracle_dt_fields;

ORACLE_API void oracle_dt_ng(const oracle_dt_fields *F, const oracle_dt_consts *C, int nk, long ncol,
                             double *p_out, double *q_out, double *r_out, double *rhs_out, double *tn_upd)
{
    double *w = (double *)malloc(sizeof(double) * 17 * (size_t)nk);
    double *vad = w, *cpi = w + nk, *kmi = w + 2 * nk, *wi = w + 3 * nk, *dudz = w + 4 * nk,
           *dvdz = w + 5 * nk, *qsolar = w + 6 * nk, *tni = w + 7 * nk, *g = w + 8 * nk, *f = w + 9 * nk,
           *p = w + 10 * nk, *q = w + 11 * nk, *r = w + 12 * nk, *rhs = w + 13 * nk, *ws = w + 14 * nk;
    const double dz = C->dz, dtx2inv = C->dtx2inv;
    long col;
    int k;
    for (col = 0; col < ncol; ++col) {
        const size_t o = (size_t)nk * col;
        const double *tn = F->tn + o, *ww = F->w + o, *cp = F->cp + o, *km = F->km + o, *un = F->un + o,
                     *vn = F->vn + o, *qt = F->qtotal + o;
        /* vertical advection (dt_ng.F90:57-64) */
        vad[0] = (tn[0] - F->t_lbc[col]) * ww[0] * 2.;
        vad[nk - 1] = 0.;
        for (k = 1; k < nk - 1; ++k) vad[k] = (tn[k] - tn[k - 1]) * ww[k];
        for (k = 0; k < nk - 1; ++k) vad[k] = (vad[k] + vad[k + 1]) * .5;
        for (k = 0; k < nk; ++k) vad[k] = vad[k] / dz;
        /* interface averages (:72-79) */
        for (k = 0; k < nk - 1; ++k) {
            cpi[k] = .5 * (cp[k] + cp[k + 1]);
            kmi[k] = .5 * (km[k] + km[k + 1]);
            wi[k] = .5 * (ww[k] + ww[k + 1]);
        }
        cpi[nk - 1] = 1.5 * cp[nk - 1] - .5 * cp[nk - 2];
        kmi[nk - 1] = 1.5 * km[nk - 1] - .5 * km[nk - 2];
        wi[nk - 1] = 1.5 * ww[nk - 1] - .5 * ww[nk - 2];
        /* wind shear (:86-95) */
        for (k = 1; k < nk - 2; ++k) {
            dudz[k] = (un[k + 1] - un[k - 1]) / (2. * dz);
            dvdz[k] = (vn[k + 1] - vn[k - 1]) / (2. * dz);
        }
        dudz[0] = (un[0] + 1. / 3. * un[1] - 4. / 3. * F->ulbc[col]) / dz;
        dvdz[0] = (vn[0] + 1. / 3. * vn[1] - 4. / 3. * F->vlbc[col]) / dz;
        dudz[nk - 2] = dudz[nk - 3] / 3.;
        dvdz[nk - 2] = dvdz[nk - 3] / 3.;
        dudz[nk - 1] = dudz[nk - 2] / 3.;
        dvdz[nk - 1] = dvdz[nk - 2] / 3.;
        for (k = 0; k < nk - 1; ++k) qsolar[k] = .5 * (qt[k] + qt[k + 1]);
        qsolar[nk - 1] = 1.5 * qt[nk - 1] - .5 * qt[nk - 2];
        /* tni (:120-124), conductivity terms (:126-148) */
        for (k = 1; k < nk - 1; ++k) tni[k] = .5 * (tn[k - 1] + tn[k]);
        tni[0] = F->tlbc[col];
        tni[nk - 1] = tn[nk - 2];
        for (k = 0; k < nk; ++k) {
            const double h = F->schti[o + k];
            double rho = C->p0 * C->expzmid_inv / (h * C->grav);
            rho = rho * F->expz[k];
            double gpart = h * h * rho * cp[k];
            gpart = gpart * F->dift[k];
            g[k] = C->grav * (F->kt[o + k] + gpart) / (C->p0 * h * (dz * dz));
            double ff = C->grav * C->grav * (h * h) * rho / (tni[k] * C->p0 * 2. * dz);
            f[k] = ff * F->dift[k];
        }
        for (k = 0; k < nk - 1; ++k) {
            p[k] = g[k] - f[k];
            q[k] = -(g[k + 1] - f[k + 1] + g[k] + f[k]);
            r[k] = g[k + 1] + f[k + 1];
        }
        q[nk - 2] = -g[nk - 2] - f[nk - 2];
        r[nk - 2] = 0.;
        /* right-hand side and implicit part (:81-84, :97-118, :150-163) */
        for (k = 0; k < nk - 1; ++k) {
            const size_t i = o + k;
            const double advec = F->horadv[i] + vad[k];
            double cptn = cpi[k] * (advec - dtx2inv * F->tnsmooth[i]);
            cptn = cptn * F->expz[k];
            const double x = F->xnmbar[i] * F->o1[i] * C->rmassinv_o1;
            const double qrecomb = C->tsurplus * F->rkm12[i] * (x * x) * C->avo / F->mbar[i];
            double qm = C->grav * kmi[k] / (C->p0 * F->scht[i]) * (dudz[k] * dudz[k] + dvdz[k] * dvdz[k]);
            qm = qm / F->expz[k];
            const double th = qsolar[k] + F->hdt[i] + qrecomb + F->qji_tn[i] + qm;
            cptn = cptn - th * F->expz[k];
            rhs[k] = cptn + F->cool_exp[i];
            const double qpart = cpi[k] * (dtx2inv + F->cool_imp[i]) + wi[k] * C->gask / F->mbar[i];
            q[k] = q[k] - qpart * F->expz[k];
        }
        q[0] = q[0] - p[0];
        rhs[0] = rhs[0] - 2. * p[0] * F->t_lbc[col];
        p[0] = 0.;
        if (p_out)
            for (k = 0; k < nk - 1; ++k) {
                p_out[o + k] = p[k];
                q_out[o + k] = q[k];
                r_out[o + k] = r[k];
                rhs_out[o + k] = rhs[k];
            }
        /* trsolv_ng(p,q,r,rhs,tn_upd,nk-1) and the top row (:165-167) */
        thomas_column(p, q, r, rhs, tn_upd + o, nk - 1, ws);
        tn_upd[o + nk - 1] = tn_upd[o + nk - 2] * tn_upd[o + nk - 2] / tn_upd[o + nk - 3];
    }
    free(w);
}

/* ------------------------------------------------------------------------ */
/* dt_ng's history diagnostics (src/dt_ng.F90:169-191 and DEN at :133), from */
/* the fields of oracle_dt_ng and its solution tn_upd (rows 1..nk, before   */
/* the lateral-boundary overwrite, as the reference writes them).  diag     */
/* receives 12 slabs of (nk, ncol): DTDT, DT_SOLAR, DT_HORDIF, DT_RECOMB,    */
/* DT_JOULE, DT_MOLDIF, DT_COOL, DT_HORADV, DT_VERADV, DT_ADIA, DT_CONDUCT,  */
/* DEN.  DT_CONDUCT rows 1 and nk are left unset by the reference (a local   */
/* array); they are 0 here.                                                  */
/* ------------------------------------------------------------------------ */
ORACLE_API void oracle_dt_diag_ng(const oracle_dt_fields *F, const oracle_dt_consts *C, int nk, long ncol,
                                  const double *tn_upd, double *diag)
{
    double *w = (double *)malloc(sizeof(double) * 10 * (size_t)nk);
    double *vad = w, *cpi = w + nk, *kmi = w + 2 * nk, *wi = w + 3 * nk, *dudz = w + 4 * nk,
           *dvdz = w + 5 * nk, *qsolar = w + 6 * nk, *tni = w + 7 * nk, *g = w + 8 * nk, *f = w + 9 * nk;
    const double dz = C->dz;
    const size_t slab = (size_t)nk * ncol;
    long col;
    int k;
    for (col = 0; col < ncol; ++col) {
        const size_t o = (size_t)nk * col;
        const double *tn = F->tn + o, *ww = F->w + o, *cp = F->cp + o, *km = F->km + o, *un = F->un + o,
                     *vn = F->vn + o, *qt = F->qtotal + o, *x = tn_upd + o;
        double *d[12];
        for (k = 0; k < 12; ++k) d[k] = diag + k * slab + o;
        /* the intermediates, as oracle_dt_ng forms them (:57-148) */
        vad[0] = (tn[0] - F->t_lbc[col]) * ww[0] * 2.;
        vad[nk - 1] = 0.;
        for (k = 1; k < nk - 1; ++k) vad[k] = (tn[k] - tn[k - 1]) * ww[k];
        for (k = 0; k < nk - 1; ++k) vad[k] = (vad[k] + vad[k + 1]) * .5;
        for (k = 0; k < nk; ++k) vad[k] = vad[k] / dz;
        for (k = 0; k < nk - 1; ++k) {
            cpi[k] = .5 * (cp[k] + cp[k + 1]);
            kmi[k] = .5 * (km[k] + km[k + 1]);
            wi[k] = .5 * (ww[k] + ww[k + 1]);
        }
        cpi[nk - 1] = 1.5 * cp[nk - 1] - .5 * cp[nk - 2];
        kmi[nk - 1] = 1.5 * km[nk - 1] - .5 * km[nk - 2];
        wi[nk - 1] = 1.5 * ww[nk - 1] - .5 * ww[nk - 2];
        for (k = 1; k < nk - 2; ++k) {
            dudz[k] = (un[k + 1] - un[k - 1]) / (2. * dz);
            dvdz[k] = (vn[k + 1] - vn[k - 1]) / (2. * dz);
        }
        dudz[0] = (un[0] + 1. / 3. * un[1] - 4. / 3. * F->ulbc[col]) / dz;
        dvdz[0] = (vn[0] + 1. / 3. * vn[1] - 4. / 3. * F->vlbc[col]) / dz;
        dudz[nk - 2] = dudz[nk - 3] / 3.;
        dvdz[nk - 2] = dvdz[nk - 3] / 3.;
        dudz[nk - 1] = dudz[nk - 2] / 3.;
        dvdz[nk - 1] = dvdz[nk - 2] / 3.;
        for (k = 0; k < nk - 1; ++k) qsolar[k] = .5 * (qt[k] + qt[k + 1]);
        qsolar[nk - 1] = 1.5 * qt[nk - 1] - .5 * qt[nk - 2];
        for (k = 1; k < nk - 1; ++k) tni[k] = .5 * (tn[k - 1] + tn[k]);
        tni[0] = F->tlbc[col];
        tni[nk - 1] = tn[nk - 2];
        for (k = 0; k < nk; ++k) {
            const size_t i = o + k;
            const double h = F->schti[i];
            double rho = C->p0 * C->expzmid_inv / (h * C->grav);
            rho = rho * F->expz[k];
            double gpart = h * h * rho * cp[k];
            gpart = gpart * F->dift[k];
            g[k] = C->grav * (F->kt[i] + gpart) / (C->p0 * h * (dz * dz));
            double ff = C->grav * C->grav * (h * h) * rho / (tni[k] * C->p0 * 2. * dz);
            f[k] = ff * F->dift[k];
            const double xo = F->xnmbar[i] * F->o1[i] * C->rmassinv_o1;
            const double qrecomb = C->tsurplus * F->rkm12[i] * (xo * xo) * C->avo / F->mbar[i];
            double qm = C->grav * kmi[k] / (C->p0 * F->scht[i]) * (dudz[k] * dudz[k] + dvdz[k] * dvdz[k]);
            qm = qm / F->expz[k];
            /* :169-180 */
            d[0][k] = C->dtx2inv * (x[k] - F->tnsmooth[i]);
            d[1][k] = qsolar[k] / cpi[k];
            d[2][k] = F->hdt[i] / cpi[k];
            d[3][k] = qrecomb / cpi[k];
            d[4][k] = F->qji_tn[i] / cpi[k];
            d[5][k] = qm / cpi[k];
            double cool_exp = F->cool_exp[i] / cpi[k];
            cool_exp = cool_exp / F->expz[k];
            d[6][k] = -cool_exp - F->cool_imp[i] * x[k];
            d[7][k] = -F->horadv[i];
            d[8][k] = -vad[k];
            d[9][k] = -(wi[k] * C->gask / (cpi[k] * F->mbar[i]) * x[k]);
            d[11][k] = rho;
        }
        /* DT_CONDUCT (:181-186) */
        d[10][0] = 0.;
        d[10][nk - 1] = 0.;
        for (k = 1; k < nk - 1; ++k) {
            const double t = (g[k] - f[k]) * x[k - 1] - (g[k + 1] - f[k + 1] + g[k] + f[k]) * x[k] +
                             (g[k + 1] + f[k + 1]) * x[k + 1];
            d[10][k] = 1. / F->expz[k] * t;
        }
        for (k = 0; k < nk; ++k) d[10][k] = d[10][k] / cpi[k];
    }
    free(w);
}

/* ------------------------------------------------------------------------ */
/* minor_ng minor-species column assembly + solve (src/minor_ng.F90:60-200), */
/* used for N4S, NO, N2D and Ar.  Fields (nk, ncol); 2-D (ncol); expz, difk  */
/* (nk).  hadvec = advec_ng(fcomp) and ftm1_smooth = smooth_ng(fcomp_tm1)    */
/* are inputs (horizontal operators), dfactor the latitude factor of         */
/* minor_ng.F90:146-155 per column.  b (3x3, column-major) and fb (3) are the */
/* lower-boundary relation of the lbc module.  p,q,r,f (may be NULL) receive */
/* rows 1..nk after the boundary folds; fcomp_out rows 1..nk (k2 = nk).       */
/* ------------------------------------------------------------------------ */
#include <math.h>

typedef struct {
    const double *tn, *o2, *o1, *he, *mbar, *barm, *xnmbar, *w, *ftm1_smooth, *hadvec, *sloss, *sprod;
    const double *tlbc, *flbc1, *flbc2, *flbc3, *fubc, *dfactor;
    const double *expz, *difk;
} oracle_minor_fields;

typedef struct {
    double rmx, alfax, phix[4], dzp, dtx2inv, expzmid, expzmid_inv;
    double rmassinv_o2, rmassinv_o1, rmassinv_n2, rmassinv_he;
    double rmass_o2, rmass_o1, rmass_he, rmass_n2, p0, grav, avo;
    double b[9], fb[3];
} oracle_minor_consts;

/* phi(3,4) and ss(3) of minor_ng.F90:25-28 (column-major phi(i,j) = PHI[i-1][j-1]) */
static const double MPHI[3][4] = {{0., 1.35, 2.16, 1.11}, {0.673, 0., 1.616, 0.769}, {0.270, 0.404, 0., 0.322}};
static const double MSS[3] = {1.710, 1.749, 1.718};

/* Per-column terms of minor_ng's rows (:72-159): after the call ax, thdiff,
 * dmdz (divided by barm) and wi hold their values for levels 0..nk-1.  w
 * holds 15*nk doubles of work, the first four blocks being those arrays. */
static void minor_terms(const oracle_minor_fields *F, const oracle_minor_consts *C, int nk, long col,
                        const double *salfax, double *w)
{
    const double tau = 1.86e+3, t00 = 273.;
    const double dzp = C->dzp;
    double *ax = w, *thdiff = w + nk, *dmdz = w + 2 * nk, *wi = w + 3 * nk, *pso1 = w + 4 * nk,
           *pso2 = w + 5 * nk, *pshe = w + 6 * nk, *do1dz = w + 7 * nk, *do2dz = w + 8 * nk, *dhedz = w + 9 * nk,
           *tni = w + 10 * nk, *sa1 = w + 11 * nk, *sa2 = w + 12 * nk, *sa3 = w + 13 * nk, *ex = w + 14 * nk;
    const size_t o = (size_t)nk * col;
    const double *tn = F->tn + o, *o2 = F->o2 + o, *o1 = F->o1 + o, *he = F->he + o, *mbar = F->mbar + o,
                 *barm = F->barm + o, *ww = F->w + o;
    int k, n;
    /* lower-boundary mixing ratios (:72-75) */
    const double bo2 = C->b[0] * o2[0] + C->b[3] * o1[0] + C->b[6] * he[0] + C->fb[0];
    const double bo1 = C->b[1] * o2[0] + C->b[4] * o1[0] + C->b[7] * he[0] + C->fb[1];
    const double bhe = C->b[2] * o2[0] + C->b[5] * o1[0] + C->b[8] * he[0] + C->fb[2];
    const double xmbari = 1. / (bo2 * C->rmassinv_o2 + bo1 * C->rmassinv_o1 +
                                (1. - bo2 - bo1 - bhe) * C->rmassinv_n2 + bhe * C->rmassinv_he);
    /* interface quantities (:77-96) */
    dmdz[0] = (mbar[0] - xmbari) / dzp;
    pso1[0] = .5 * (bo1 + o1[0]);
    pso2[0] = .5 * (bo2 + o2[0]);
    pshe[0] = .5 * (bhe + he[0]);
    do1dz[0] = (o1[0] - bo1) / dzp;
    do2dz[0] = (o2[0] - bo2) / dzp;
    dhedz[0] = (he[0] - bhe) / dzp;
    for (k = 1; k < nk; ++k) {
        dmdz[k] = (mbar[k] - mbar[k - 1]) / dzp;
        pso1[k] = .5 * (o1[k] + o1[k - 1]);
        pso2[k] = .5 * (o2[k] + o2[k - 1]);
        pshe[k] = .5 * (he[k] + he[k - 1]);
        do1dz[k] = (o1[k] - o1[k - 1]) / dzp;
        do2dz[k] = (o2[k] - o2[k - 1]) / dzp;
        dhedz[k] = (he[k] - he[k - 1]) / dzp;
    }
    tni[0] = F->tlbc[col];
    tni[nk - 1] = tn[nk - 2];
    for (k = 1; k < nk - 1; ++k) tni[k] = .5 * (tn[k] + tn[k - 1]);
    /* alfa matrix, its inverse, salfax . invalfa(:,n) (:100-133) */
    for (k = 0; k < nk; ++k) {
        double df[3], A[9], Ai[9];
        for (n = 0; n < 3; ++n) df[n] = pow(tni[k] / t00, 1.75 - MSS[n]);
#define PH(i, j) MPHI[(i) - 1][(j) - 1]
        M3(A, 1, 1) = -(PH(1, 4) + (PH(1, 2) - PH(1, 4)) * pso1[k] + (df[0] * PH(1, 3) - PH(1, 4)) * pshe[k]);
        M3(A, 2, 2) = -(PH(2, 4) + (PH(2, 1) - PH(2, 4)) * pso2[k] + (df[1] * PH(2, 3) - PH(2, 4)) * pshe[k]);
        M3(A, 3, 3) = -(df[2] * PH(3, 4) + (df[0] * PH(3, 1) - df[2] * PH(3, 4)) * pso2[k] +
                       (df[1] * PH(3, 2) - df[2] * PH(3, 4)) * pso1[k]);
        M3(A, 1, 2) = (PH(1, 2) - PH(1, 4)) * pso2[k];
        M3(A, 1, 3) = (df[0] * PH(1, 3) - PH(1, 4)) * pso2[k];
        M3(A, 2, 1) = (PH(2, 1) - PH(2, 4)) * pso1[k];
        M3(A, 2, 3) = (df[1] * PH(2, 3) - PH(2, 4)) * pso1[k];
        M3(A, 3, 1) = (df[0] * PH(3, 1) - df[2] * PH(3, 4)) * pshe[k];
        M3(A, 3, 2) = (df[1] * PH(3, 2) - df[2] * PH(3, 4)) * pshe[k];
        oracle_matinv3(A, Ai);
        sa1[k] = salfax[0] * M3(Ai, 1, 1) + salfax[1] * M3(Ai, 2, 1) + salfax[2] * M3(Ai, 3, 1);
        sa2[k] = salfax[0] * M3(Ai, 1, 2) + salfax[1] * M3(Ai, 2, 2) + salfax[2] * M3(Ai, 3, 2);
        sa3[k] = salfax[0] * M3(Ai, 1, 3) + salfax[1] * M3(Ai, 2, 3) + salfax[2] * M3(Ai, 3, 3);
    }
    /* ex, ax, thdiff (:135-153) */
    for (k = 0; k < nk; ++k) {
        ex[k] = 1. - (C->rmx + dmdz[k]) / barm[k] +
                sa1[k] * (do2dz[k] - (1. - (C->rmass_o2 + dmdz[k]) / barm[k]) * pso2[k]) +
                sa2[k] * (do1dz[k] - (1. - (C->rmass_o1 + dmdz[k]) / barm[k]) * pso1[k]) +
                sa3[k] * (dhedz[k] - (1. - (C->rmass_he + dmdz[k]) / barm[k]) * pshe[k]);
        dmdz[k] = dmdz[k] / barm[k];
        ax[k] = -(barm[k] / (tau * C->rmass_n2) * pow(t00 / tni[k], 0.25) /
                  (C->phix[2] + salfax[0] * pso2[k] + salfax[1] * pso1[k] + salfax[2] * pshe[k]));
    }
    for (k = 0; k < nk; ++k) {
        double dt;
        if (k == 0) dt = tni[1] - tni[0];
        else if (k == nk - 1) dt = tni[nk - 1] - tni[nk - 2];
        else dt = (tni[k + 1] - tni[k - 1]) / 2.;
        thdiff[k] = ex[k] - C->alfax * dt / (dzp * tni[k]);
    }
    for (k = 0; k < nk - 1; ++k) wi[k] = .5 * (ww[k] + ww[k + 1]);
    wi[nk - 1] = 1.5 * ww[nk - 1] - .5 * ww[nk - 2];
}

/* minor_ng's history diagnostics (src/minor_ng.F90:202-224) from the      */
/* fields of oracle_minor_ng and its solution fcomp_out (before the lateral */
/* overwrite).  diag receives 7 slabs of (nk, ncol): DPDT, PROD (s0prod),   */
/* LOSS, MOLDIF, EDDYDIF (times dfactor), -VERADV and -HORADV, the values    */
/* the reference passes to addfld.  MOLDIF, EDDYDIF and VERADV rows 1 and nk */
/* are left unset by the reference (local arrays); they are 0 here.          */
ORACLE_API void oracle_minor_diag_ng(const oracle_minor_fields *F, const oracle_minor_consts *C, int nk, long ncol,
                                     const double *fcomp_out, double *diag)
{
    const double dzp = C->dzp;
    double salfax[3];
    double *w = (double *)malloc(sizeof(double) * 15 * (size_t)nk);
    const double *ax = w, *thdiff = w + nk, *dmdz = w + 2 * nk, *wi = w + 3 * nk;
    const size_t slab = (size_t)nk * ncol;
    long col;
    int k, n;
    for (n = 0; n < 3; ++n) salfax[n] = C->phix[n] - C->phix[3];
    for (col = 0; col < ncol; ++col) {
        const size_t o = (size_t)nk * col;
        const double *x = fcomp_out + o;
        double *d[7];
        for (n = 0; n < 7; ++n) d[n] = diag + n * slab + o;
        minor_terms(F, C, nk, col, salfax, w);
        for (k = 0; k < nk; ++k) {
            d[0][k] = C->dtx2inv * (x[k] - F->ftm1_smooth[o + k]);
            d[1][k] = F->sprod[o + k] * C->rmx / F->xnmbar[o + k];
            d[2][k] = F->sloss[o + k] * x[k];
            d[3][k] = d[4][k] = d[5][k] = 0.;
            d[6][k] = -F->hadvec[o + k];
        }
        for (k = 1; k < nk - 1; ++k) {
            const double molp = ax[k] * (1. / dzp + .5 * thdiff[k]);
            const double molr = ax[k + 1] * (1. / dzp - .5 * thdiff[k + 1]);
            const double molq = ax[k] * (1. / dzp - .5 * thdiff[k]) + ax[k + 1] * (1. / dzp + .5 * thdiff[k + 1]);
            const double eddyp = C->expzmid_inv * F->difk[k] * (1. / dzp - .5 * dmdz[k]);
            const double eddyr = C->expzmid * F->difk[k + 1] * (1. / dzp + .5 * dmdz[k + 1]);
            const double eddyq = C->expzmid_inv * F->difk[k] * (1. / dzp + .5 * dmdz[k]) +
                                 C->expzmid * F->difk[k + 1] * (1. / dzp - .5 * dmdz[k + 1]);
            d[3][k] = -(1. / F->expz[k] / dzp * (molp * x[k - 1] - molq * x[k] + molr * x[k + 1]));
            d[4][k] = 1. / dzp * (eddyp * x[k - 1] - eddyq * x[k] + eddyr * x[k + 1]);
            d[5][k] = -(wi[k] / (2. * dzp) * (x[k + 1] - x[k - 1]));
        }
        for (k = 0; k < nk; ++k) d[4][k] = d[4][k] * F->dfactor[col];
    }
    free(w);
}

ORACLE_API void oracle_minor_ng(const oracle_minor_fields *F, const oracle_minor_consts *C, int nk, long ncol,
                                double *p_out, double *q_out, double *r_out, double *f_out, double *fcomp_out)
{
    const double dzp = C->dzp;
    double salfax[3];
    double *w = (double *)malloc(sizeof(double) * 24 * (size_t)nk);
    double *ax = w, *thdiff = w + nk, *dmdz = w + 2 * nk, *wi = w + 3 * nk, *p = w + 15 * nk, *q = w + 16 * nk,
           *r = w + 17 * nk, *f = w + 18 * nk, *ws = w + 19 * nk;
    long col;
    int k, n;
    for (n = 0; n < 3; ++n) salfax[n] = C->phix[n] - C->phix[3];
    for (col = 0; col < ncol; ++col) {
        const size_t o = (size_t)nk * col;
        minor_terms(F, C, nk, col, salfax, w);
        /* p, q, r, f (:161-198) */
        const double dfac = F->dfactor[col];
        for (k = 0; k < nk - 1; ++k) {
            const double molp = ax[k] * (1. / dzp + .5 * thdiff[k]);
            const double molr = ax[k + 1] * (1. / dzp - .5 * thdiff[k + 1]);
            const double molq = ax[k] * (1. / dzp - .5 * thdiff[k]) + ax[k + 1] * (1. / dzp + .5 * thdiff[k + 1]);
            const double eddyp = C->expzmid_inv * F->difk[k] * (1. / dzp - .5 * dmdz[k]);
            const double eddyr = C->expzmid * F->difk[k + 1] * (1. / dzp + .5 * dmdz[k + 1]);
            const double eddyq = C->expzmid_inv * F->difk[k] * (1. / dzp + .5 * dmdz[k]) +
                                 C->expzmid * F->difk[k + 1] * (1. / dzp - .5 * dmdz[k + 1]);
            p[k] = molp / dzp - F->expz[k] * (eddyp * dfac + .5 * wi[k]) / dzp;
            r[k] = molr / dzp - F->expz[k] * (eddyr * dfac - .5 * wi[k]) / dzp;
            q[k] = -molq / dzp + F->expz[k] * (eddyq * dfac / dzp + C->dtx2inv - F->sloss[o + k]);
        }
        for (k = 0; k < nk; ++k) {
            const double s0prod = F->sprod[o + k] * C->rmx / F->xnmbar[o + k];
            f[k] = F->ftm1_smooth[o + k] * C->dtx2inv - F->hadvec[o + k] + s0prod;
            f[k] = f[k] * F->expz[k];
        }
        {
            const double l1 = F->flbc1[col], l2 = F->flbc2[col], l3 = F->flbc3[col];
            q[0] = q[0] + p[0] * (l1 + .5 * l2 * dzp) / (l1 - .5 * l2 * dzp);
            f[0] = f[0] - p[0] * l3 * dzp / (l1 - .5 * l2 * dzp);
            p[0] = 0.;
        }
        p[nk - 1] = 1. + .5 * dzp * thdiff[nk - 1];
        q[nk - 1] = p[nk - 1] - 2.;
        r[nk - 1] = 0.;
        f[nk - 1] = -C->grav * C->rmx * F->fubc[col] * dzp / (C->p0 * ax[nk - 1] * C->avo);
        if (p_out)
            for (k = 0; k < nk; ++k) {
                p_out[o + k] = p[k];
                q_out[o + k] = q[k];
                r_out[o + k] = r[k];
                f_out[o + k] = f[k];
            }
        thomas_column(p, q, r, f, fcomp_out + o, nk, ws);
    }
    free(w);
}

/* ------------------------------------------------------------------------ */
/* comp_ng major-species column step (src/comp_ng.F90:74-332): O2, O and He */
/* mass mixing ratios from the 3x3 block-tridiagonal diffusion system.      */
/* Fields (nk, ncol); fs is fs(nk, ncol, 3, 0:3) of the reference, i.e. 12  */
/* slabs (nk, ncol) with slab index m*3+isp; 2-D (ncol); expz, difk (nk).    */
/* o2/o1/he_advec = advec_ng(o2/o1/he), o2/o1/henm_smooth = smooth_ng(..nm) */
/* and hdo2/hdo1/hdhe are inputs (horizontal operators), dfactor the        */
/* latitude factor of comp_ng.F90:117-126.  Outputs upd (o2, o1, he) rows   */
/* 1..nk before the time filter (he_upd = pshelb when calc_helium is 0);    */
/* P,Q,R (3,3,nk,ncol), f (3,nk,ncol) and                                   */
/* ubc (6,ncol: ratio(3), add(3)) may be NULL and receive the system the    */
/* block solve sees, rows 1..nk-1, after the boundary folds.                */
/* ------------------------------------------------------------------------ */
typedef struct {
    const double *tn, *o2, *o1, *he, *w, *mbar, *o2nm_smooth, *o1nm_smooth, *henm_smooth;
    const double *o2_advec, *o1_advec, *he_advec, *hdo2, *hdo1, *hdhe, *fs;
    const double *tlbc, *flx_he, *dfactor;
    const double *expz, *difk;
} oracle_comp_fields;

typedef struct {
    double dz, dtx2inv, expzmid, expzmid_inv;
    double rmassinv_o2, rmassinv_o1, rmassinv_he, rmassinv_n2;
    double rmass_o2, rmass_o1, rmass_he, p0, grav;
    double b[9], fb[3];
    double pshelb;     /* He mixing ratio held when calc_helium is 0 */
    int calc_helium;   /* 0: flx_he is taken as 0 and he_upd = pshelb (comp_ng.F90:72,386-389) */
} oracle_comp_consts;

/* ep, alpha, ak = matinv3(alpha)*wks1 and wks4 of one level (comp_ng.F90:128-166, 176-211) */
static void comp_level(const oracle_comp_consts *C, double o2i, double o1i, double hei, double embari,
                       double tni, double dembardz, double dtndz, int he_thermal, double ep[3],
                       double A[9], double ak[9], double *wks4)
{
    const double tau = 1.86e+3, thdiffalpha = -0.38, t00 = 273.;
    double df[3], Ai[9], wks1;
    int n, e;
    for (n = 0; n < 3; ++n) df[n] = pow(tni / t00, 1.75 - MSS[n]);
    ep[0] = 1. - 1. / embari * (C->rmass_o2 + dembardz);
    ep[1] = 1. - 1. / embari * (C->rmass_o1 + dembardz);
    ep[2] = 1. - 1. / embari * (C->rmass_he + dembardz);
    if (he_thermal) ep[2] = ep[2] - thdiffalpha * dtndz / tni;
    M3(A, 1, 1) = -(PH(1, 4) + (PH(1, 2) - PH(1, 4)) * o1i + (df[0] * PH(1, 3) - PH(1, 4)) * hei);
    M3(A, 2, 2) = -(PH(2, 4) + (PH(2, 1) - PH(2, 4)) * o2i + (df[1] * PH(2, 3) - PH(2, 4)) * hei);
    M3(A, 3, 3) = -(df[2] * PH(3, 4) + (df[0] * PH(3, 1) - df[2] * PH(3, 4)) * o2i +
                   (df[1] * PH(3, 2) - df[2] * PH(3, 4)) * o1i);
    M3(A, 1, 2) = (PH(1, 2) - PH(1, 4)) * o2i;
    M3(A, 1, 3) = (df[0] * PH(1, 3) - PH(1, 4)) * o2i;
    M3(A, 2, 1) = (PH(2, 1) - PH(2, 4)) * o1i;
    M3(A, 2, 3) = (df[1] * PH(2, 3) - PH(2, 4)) * o1i;
    M3(A, 3, 1) = (df[0] * PH(3, 1) - df[2] * PH(3, 4)) * hei;
    M3(A, 3, 2) = (df[1] * PH(3, 2) - df[2] * PH(3, 4)) * hei;
    oracle_matinv3(A, Ai);
    wks1 = embari * C->rmassinv_n2 * pow(t00 / tni, 0.25) / tau;
    for (e = 0; e < 9; ++e) ak[e] = Ai[e] * wks1;
    *wks4 = dembardz / (embari * 2.);
}

ORACLE_API void oracle_comp_ng(const oracle_comp_fields *F, const oracle_comp_consts *C, int nk, long ncol,
                               double *o2_upd, double *o1_upd, double *he_upd, double *P_out, double *Q_out,
                               double *R_out, double *f_out, double *ubc_out)
{
    const double tau = 1.86e+3, t00 = 273.;
    const double dz = C->dz;
    double *w = (double *)malloc(sizeof(double) * (8 + 12 + 3) * (size_t)nk);
    long col;
    if (nk < 3) { free(w); return; }
    for (col = 0; col < ncol; ++col) {
        const size_t o = (size_t)nk * col, slab = (size_t)nk * ncol;
        const double *tn = F->tn + o, *o2 = F->o2 + o, *o1 = F->o1 + o, *he = F->he + o, *mbar = F->mbar + o,
                     *ww = F->w + o;
        const double *nms[3] = {F->o2nm_smooth + o, F->o1nm_smooth + o, F->henm_smooth + o};
        const double *adv[3] = {F->o2_advec + o, F->o1_advec + o, F->he_advec + o};
        const double *hd[3] = {F->hdo2 + o, F->hdo1 + o, F->hdhe + o};
        double *o2i = w, *o1i = w + nk, *hei = w + 2 * nk, *embari = w + 3 * nk, *tni = w + 4 * nk,
               *dembardz = w + 5 * nk, *dtndz = w + 6 * nk, *wi = w + 7 * nk, *G = w + 8 * nk;
        double ps0[3], embar0, ep_km[3], ep_kp[3], A[9], ak_km[9], ak_kp[9], wks3, wks4;
        double a22 = 0., a33 = 0., a23 = 0., a32 = 0., flx00 = 1.;
        double upd[3][2];
        const double flx_he = C->calc_helium ? F->flx_he[col] : 0.;
        int k, i, m, n;
        /* lower-boundary mixing ratios and interface quantities (:74-102) */
        for (i = 0; i < 3; ++i)
            ps0[i] = C->b[i] * o2[0] + C->b[i + 3] * o1[0] + C->b[i + 6] * he[0] + C->fb[i];
        embar0 = 1. / (ps0[0] * C->rmassinv_o2 + ps0[1] * C->rmassinv_o1 + ps0[2] * C->rmassinv_he +
                       (1. - ps0[0] - ps0[1] - ps0[2]) * C->rmassinv_n2);
        o2i[0] = .5 * (ps0[0] + o2[0]);
        o1i[0] = .5 * (ps0[1] + o1[0]);
        hei[0] = .5 * (ps0[2] + he[0]);
        embari[0] = .5 * (embar0 + mbar[0]);
        tni[0] = F->tlbc[col];
        dembardz[0] = mbar[0] - embar0;
        dtndz[0] = (tn[0] - F->tlbc[col]) * 2;
        for (k = 1; k < nk; ++k) {
            o2i[k] = .5 * (o2[k - 1] + o2[k]);
            o1i[k] = .5 * (o1[k - 1] + o1[k]);
            hei[k] = .5 * (he[k - 1] + he[k]);
            embari[k] = .5 * (mbar[k - 1] + mbar[k]);
            tni[k] = .5 * (tn[k - 1] + tn[k]);
            dembardz[k] = mbar[k] - mbar[k - 1];
            dtndz[k] = tn[k] - tn[k - 1];
        }
        for (k = 0; k < nk; ++k) {
            dembardz[k] = dembardz[k] / dz;
            dtndz[k] = dtndz[k] / dz;
        }
        for (k = 0; k < nk - 1; ++k) wi[k] = .5 * (ww[k] + ww[k + 1]);
        wi[nk - 1] = 1.5 * ww[nk - 1] - .5 * ww[nk - 2];
        /* level 1 (:128-166) */
        comp_level(C, o2i[0], o1i[0], hei[0], embari[0], tni[0], dembardz[0], dtndz[0], 1, ep_kp, A, ak_kp, &wks4);
        for (i = 0; i < 12; ++i) G[i] = 0.;
        const double dfac = F->dfactor[col];
        /* rows 1..nk-1: assembly (:176-278) and block forward sweep (:280-314) */
        for (k = 0; k < nk - 1; ++k) {
            double Pk[9], Qk[9], Rk[9], fk[3], W[9], v[3];
            for (i = 0; i < 3; ++i) ep_km[i] = ep_kp[i];
            for (i = 0; i < 9; ++i) ak_km[i] = ak_kp[i];
            wks3 = wks4;
            comp_level(C, o2i[k + 1], o1i[k + 1], hei[k + 1], embari[k + 1], tni[k + 1], dembardz[k + 1],
                       dtndz[k + 1], k + 1 != nk - 1, ep_kp, A, ak_kp, &wks4);
            const double eddyp = C->expzmid_inv * F->difk[k] * (1. / dz - wks3);
            const double eddyr = C->expzmid * F->difk[k + 1] * (1. / dz + wks4);
            const double eddyq = C->expzmid_inv * F->difk[k] * (1. / dz + wks3) +
                                 C->expzmid * F->difk[k + 1] * (1. / dz - wks4);
            const double ez = F->expz[k];
            for (m = 0; m < 3; ++m)
                for (i = 0; i < 3; ++i) {
                    const double delta = i == m ? 1. : 0.;
                    const double molp = ak_km[i + 3 * m] * (1. / dz + ep_km[m] / 2.);
                    const double molr = ak_kp[i + 3 * m] * (1. / dz - ep_kp[m] / 2.);
                    const double molq = ak_km[i + 3 * m] * (1. / dz - ep_km[m] / 2.) +
                                        ak_kp[i + 3 * m] * (1. / dz + ep_kp[m] / 2.);
                    Pk[i + 3 * m] = molp / dz - ez * delta / dz * (eddyp * dfac + .5 * wi[k]);
                    Rk[i + 3 * m] = molr / dz - ez * delta / dz * (eddyr * dfac - .5 * wi[k]);
                    Qk[i + 3 * m] = -molq / dz + ez * delta * (eddyq * dfac / dz + C->dtx2inv) -
                                    ez * F->fs[(size_t)(m + 1) * 3 * slab + (size_t)i * slab + o + k];
                }
            for (i = 0; i < 3; ++i)
                fk[i] = ez * (nms[i][k] * C->dtx2inv - (adv[i][k] - F->fs[(size_t)i * slab + o + k]) + hd[i][k]);
            if (k == 0) {
                for (m = 0; m < 3; ++m)
                    for (n = 0; n < 3; ++n)
                        for (i = 0; i < 3; ++i) Qk[i + 3 * m] = Qk[i + 3 * m] + Pk[i + 3 * n] * C->b[n + 3 * m];
                for (m = 0; m < 3; ++m)
                    for (i = 0; i < 3; ++i) fk[i] = fk[i] - Pk[i + 3 * m] * C->fb[m];
                for (i = 0; i < 9; ++i) Pk[i] = 0.;
            } else if (k == nk - 2) {
                for (m = 0; m < 3; ++m)
                    for (i = 0; i < 3; ++i)
                        Qk[i + 3 * m] = Qk[i + 3 * m] +
                                        (1. + .5 * ep_kp[m] * dz) / (1. - .5 * ep_kp[m] * dz) * Rk[i + 3 * m];
                a22 = M3(A, 2, 2);
                a33 = M3(A, 3, 3);
                a23 = M3(A, 2, 3);
                a32 = M3(A, 3, 2);
                flx00 = embari[k] * C->rmassinv_n2 * C->p0 * pow(t00 / tn[k], 0.25) / (tau * C->grav);
                for (i = 0; i < 3; ++i)
                    fk[i] = fk[i] - Rk[i + 3] * (a23 - a22) * flx_he / (flx00 * (1. / dz - 0.5 * ep_kp[1])) -
                            Rk[i + 6] * (a33 - a32) * flx_he / (flx00 * (1. / dz - 0.5 * ep_kp[2]));
                for (i = 0; i < 9; ++i) Rk[i] = 0.;
            }
            if (P_out) {
                const size_t om = (size_t)9 * nk * col + 9 * (size_t)k, ov = (size_t)3 * nk * col + 3 * (size_t)k;
                for (i = 0; i < 9; ++i) {
                    P_out[om + i] = Pk[i];
                    Q_out[om + i] = Qk[i];
                    R_out[om + i] = Rk[i];
                }
                for (i = 0; i < 3; ++i) f_out[ov + i] = fk[i];
            }
            {
                const double *Gk = G + 12 * k;
                double *Gn = G + 12 * (k + 1);
                for (m = 0; m < 3; ++m)
                    for (n = 0; n < 3; ++n)
                        for (i = 0; i < 3; ++i) Qk[i + 3 * m] = Qk[i + 3 * m] - Pk[i + 3 * n] * Gk[n + 3 * m];
                oracle_matinv3(Qk, W);
                for (i = 0; i < 3; ++i) v[i] = fk[i];
                for (m = 0; m < 3; ++m) {
                    for (i = 0; i < 3; ++i) v[i] = v[i] - Pk[i + 3 * m] * Gk[9 + m];
                }
                for (i = 0; i < 12; ++i) Gn[i] = 0.;
                for (m = 0; m < 3; ++m)
                    for (n = 0; n < 3; ++n)
                        for (i = 0; i < 3; ++i) Gn[i + 3 * m] = Gn[i + 3 * m] + W[i + 3 * n] * Rk[n + 3 * m];
                for (m = 0; m < 3; ++m)
                    for (i = 0; i < 3; ++i) Gn[9 + i] = Gn[9 + i] + W[i + 3 * m] * v[m];
            }
        }
        /* back sweep (:317-324) */
        {
            double *x[3] = {o2_upd + o, o1_upd + o, he_upd + o};
            for (i = 0; i < 3; ++i) x[i][nk - 1] = 0.;
            for (k = nk - 2; k >= 0; --k) {
                const double *Gn = G + 12 * (k + 1);
                for (i = 0; i < 3; ++i) upd[i][0] = Gn[9 + i];
                for (i = 0; i < 3; ++i)
                    for (m = 0; m < 3; ++m) upd[i][0] = upd[i][0] - Gn[i + 3 * m] * x[m][k + 1];
                for (i = 0; i < 3; ++i) x[i][k] = upd[i][0];
            }
            /* upper boundary (:326-332) */
            double ratio[3], add[3] = {0., 0., 0.};
            for (i = 0; i < 3; ++i) {
                ratio[i] = (1. + .5 * ep_kp[i] * dz) / (1. - .5 * ep_kp[i] * dz);
                x[i][nk - 1] = ratio[i] * x[i][nk - 2];
            }
            add[1] = (a23 - a22) * flx_he / (flx00 * (1. / dz - 0.5 * ep_kp[1]));
            add[2] = (a33 - a32) * flx_he / (flx00 * (1. / dz - 0.5 * ep_kp[2]));
            x[1][nk - 1] = x[1][nk - 1] + add[1];
            x[2][nk - 1] = x[2][nk - 1] + add[2];
            if (ubc_out)
                for (i = 0; i < 3; ++i) {
                    ubc_out[6 * col + i] = ratio[i];
                    ubc_out[6 * col + 3 + i] = add[i];
                }
            if (!C->calc_helium)
                for (k = 0; k < nk; ++k) x[2][k] = C->pshelb;
        }
    }
    free(w);
}

/* comp_ng post-solve steps per column (src/comp_ng.F90:415-457): the time  */
/* filter, N2 = 1 - O2 - O - He with the exponential extrapolation above the */
/* level where N2 < 0.01, the floor at 1e-9 and the normalisation.  o2/o1/he */
/* are the fields at the current step (itp), o2/o1/he_nm the previous one;    */
/* upd arrays (in: solution, lateral-boundary columns already overwritten)   */
/* receive the final mixing ratios, *nm_upd the filtered ones.  A column    */
/* whose N2 drops below 0.01 at level 1 is left without extrapolation (the  */
/* reference would read level 0 there).                                      */
/* comp_ng's history diagnostics (comp_ng.F90:334-380) of a solution upd =
 * (o2, o1, he) before the lateral overwrite and the post steps: 24 planes
 * (nk, ncol) in the order of the addfld calls,
 *   DO2DT DO1DT DHEDT, O2/O1/HE_PROD, _LOSS, _HORDIF, _MOLDIF, _EDDYDIF,
 *   -_VERADV, -_HORADV.
 * loss and moldif are summed over their fourth index, the species the row
 * belongs to (sum(loss, dim=4), sum(moldif, dim=4)), so X_LOSS and X_MOLDIF
 * are indexed by the species the solution value belongs to.  MOLDIF,
 * EDDYDIF and VERADV are defined on levels 2..nk-1 (1-based); the reference
 * leaves the others unset, here they are 0. */
ORACLE_API void oracle_comp_diag_ng(const oracle_comp_fields *F, const oracle_comp_consts *C, int nk, long ncol,
                                    const double *o2_upd, const double *o1_upd, const double *he_upd, double *diag)
{
    const double dz = C->dz;
    double *w = (double *)malloc(sizeof(double) * (8 + 14 * 2) * (size_t)nk);
    long col;
    if (nk < 3) { free(w); return; }
    const size_t slab = (size_t)nk * ncol;
    for (col = 0; col < ncol; ++col) {
        const size_t o = (size_t)nk * col;
        const double *tn = F->tn + o, *o2 = F->o2 + o, *o1 = F->o1 + o, *he = F->he + o, *mbar = F->mbar + o,
                     *ww = F->w + o;
        const double *nms[3] = {F->o2nm_smooth + o, F->o1nm_smooth + o, F->henm_smooth + o};
        const double *adv[3] = {F->o2_advec + o, F->o1_advec + o, F->he_advec + o};
        const double *hd[3] = {F->hdo2 + o, F->hdo1 + o, F->hdhe + o};
        const double *x[3] = {o2_upd + o, o1_upd + o, he_upd + o};
        double *o2i = w, *o1i = w + nk, *hei = w + 2 * nk, *embari = w + 3 * nk, *tni = w + 4 * nk,
               *dembardz = w + 5 * nk, *dtndz = w + 6 * nk, *wi = w + 7 * nk;
        /* per level: ep (3), ak (9), wks4 */
        double *lev = w + 8 * nk;
        double ps0[3], embar0, A[9];
        double *d[24];
        int k, i, m, n;
        for (n = 0; n < 24; ++n) d[n] = diag + n * slab + o;
        for (i = 0; i < 3; ++i)
            ps0[i] = C->b[i] * o2[0] + C->b[i + 3] * o1[0] + C->b[i + 6] * he[0] + C->fb[i];
        embar0 = 1. / (ps0[0] * C->rmassinv_o2 + ps0[1] * C->rmassinv_o1 + ps0[2] * C->rmassinv_he +
                       (1. - ps0[0] - ps0[1] - ps0[2]) * C->rmassinv_n2);
        o2i[0] = .5 * (ps0[0] + o2[0]);
        o1i[0] = .5 * (ps0[1] + o1[0]);
        hei[0] = .5 * (ps0[2] + he[0]);
        embari[0] = .5 * (embar0 + mbar[0]);
        tni[0] = F->tlbc[col];
        dembardz[0] = mbar[0] - embar0;
        dtndz[0] = (tn[0] - F->tlbc[col]) * 2;
        for (k = 1; k < nk; ++k) {
            o2i[k] = .5 * (o2[k - 1] + o2[k]);
            o1i[k] = .5 * (o1[k - 1] + o1[k]);
            hei[k] = .5 * (he[k - 1] + he[k]);
            embari[k] = .5 * (mbar[k - 1] + mbar[k]);
            tni[k] = .5 * (tn[k - 1] + tn[k]);
            dembardz[k] = mbar[k] - mbar[k - 1];
            dtndz[k] = tn[k] - tn[k - 1];
        }
        for (k = 0; k < nk; ++k) {
            dembardz[k] = dembardz[k] / dz;
            dtndz[k] = dtndz[k] / dz;
        }
        for (k = 0; k < nk - 1; ++k) wi[k] = .5 * (ww[k] + ww[k + 1]);
        wi[nk - 1] = 1.5 * ww[nk - 1] - .5 * ww[nk - 2];
        /* level quantities (:128-211); the top level has no thermal diffusion term */
        for (k = 0; k < nk; ++k) {
            double *L = lev + 13 * (size_t)k;
            comp_level(C, o2i[k], o1i[k], hei[k], embari[k], tni[k], dembardz[k], dtndz[k], k != nk - 1, L, A,
                       L + 3, L + 12);
        }
        for (k = 0; k < nk; ++k) {
            for (i = 0; i < 3; ++i) {
                d[i][k] = C->dtx2inv * (x[i][k] - nms[i][k]);
                d[3 + i][k] = F->fs[(size_t)i * slab + o + k];
                d[9 + i][k] = hd[i][k];
                d[21 + i][k] = -adv[i][k];
            }
            /* loss_sum(m) = sum over isp of fs(isp, m) * upd(m), accumulated from 0 as SUM does */
            for (m = 0; m < 3; ++m) {
                double s = 0.;
                for (i = 0; i < 3; ++i) s = s + F->fs[(size_t)(m + 1) * 3 * slab + (size_t)i * slab + o + k] * x[m][k];
                d[6 + m][k] = s;
            }
            for (i = 0; i < 3; ++i) d[12 + i][k] = d[15 + i][k] = d[18 + i][k] = 0.;
        }
        for (k = 1; k < nk - 1; ++k) {
            /* row k's coefficients: levels k (km) and k+1 (kp) */
            const double *Lk = lev + 13 * (size_t)k, *Lp = lev + 13 * (size_t)(k + 1);
            const double wks3 = Lk[12], wks4 = Lp[12];
            const double eddyp = C->expzmid_inv * F->difk[k] * (1. / dz - wks3);
            const double eddyr = C->expzmid * F->difk[k + 1] * (1. / dz + wks4);
            const double eddyq = C->expzmid_inv * F->difk[k] * (1. / dz + wks3) +
                                 C->expzmid * F->difk[k + 1] * (1. / dz - wks4);
            for (m = 0; m < 3; ++m) {
                double s = 0.;
                for (i = 0; i < 3; ++i) {
                    const double molp = Lk[3 + i + 3 * m] * (1. / dz + Lk[m] / 2.);
                    const double molr = Lp[3 + i + 3 * m] * (1. / dz - Lp[m] / 2.);
                    const double molq = Lk[3 + i + 3 * m] * (1. / dz - Lk[m] / 2.) +
                                        Lp[3 + i + 3 * m] * (1. / dz + Lp[m] / 2.);
                    s = s + -(1. / F->expz[k] / dz * (molp * x[m][k - 1] - molq * x[m][k] + molr * x[m][k + 1]));
                }
                d[12 + m][k] = s;
            }
            for (i = 0; i < 3; ++i) {
                d[15 + i][k] = 1. / dz * (eddyp * x[i][k - 1] - eddyq * x[i][k] + eddyr * x[i][k + 1]);
                d[18 + i][k] = -(wi[k] / (2. * dz) * (x[i][k + 1] - x[i][k - 1]));
            }
        }
        for (k = 0; k < nk; ++k)
            for (i = 0; i < 3; ++i) d[15 + i][k] = d[15 + i][k] * F->dfactor[col];
    }
    free(w);
}

ORACLE_API void oracle_comp_post_ng(const double *o2, const double *o1, const double *he, const double *o2_nm,
                                    const double *o1_nm, const double *he_nm, const double *xnmbar,
                                    const double *zpmid, double dz, double dtsmooth, double dtsmooth_div2,
                                    int nk, long ncol, double *o2_upd,
                                    double *o1_upd, double *he_upd, double *o2nm_upd, double *o1nm_upd,
                                    double *henm_upd)
{
    const double small = 1.e-9;
    double *n2 = (double *)malloc(sizeof(double) * 2 * (size_t)nk), *n2nm = n2 + nk;
    long col;
    for (col = 0; col < ncol; ++col) {
        const size_t o = (size_t)nk * col;
        int k, ktop;
        for (k = 0; k < nk; ++k) {
            o2nm_upd[o + k] = dtsmooth_div2 * (o2_nm[o + k] + o2_upd[o + k]) + dtsmooth * o2[o + k];
            o1nm_upd[o + k] = dtsmooth_div2 * (o1_nm[o + k] + o1_upd[o + k]) + dtsmooth * o1[o + k];
            henm_upd[o + k] = dtsmooth_div2 * (he_nm[o + k] + he_upd[o + k]) + dtsmooth * he[o + k];
        }
        for (k = 0; k < nk; ++k) {
            n2[k] = 1. - o2_upd[o + k] - o1_upd[o + k] - he_upd[o + k];
            n2nm[k] = 1. - o2nm_upd[o + k] - o1nm_upd[o + k] - henm_upd[o + k];
        }
        for (ktop = 0; ktop < nk; ++ktop)
            if (n2[ktop] < 0.01) break;
        if (ktop < nk - 1 && ktop > 0) {
            const double zmtop = zpmid[ktop];
            const double n2top = log(n2[ktop] * xnmbar[o + ktop]);
            const double n2top1 = log(n2[ktop - 1] * xnmbar[o + ktop - 1]);
            const double dn2dz = (n2top - n2top1) / dz;
            for (k = ktop + 1; k < nk; ++k) n2[k] = exp(n2top + dn2dz * (zpmid[k] - zmtop)) / xnmbar[o + k];
        }
        for (k = 0; k < nk; ++k) {
            double a = o2_upd[o + k] > small ? o2_upd[o + k] : small;
            double b = o1_upd[o + k] > small ? o1_upd[o + k] : small;
            double c = he_upd[o + k] > small ? he_upd[o + k] : small;
            double d = n2[k] > small ? n2[k] : small;
            double s = a + b + c + d;
            o2_upd[o + k] = a / s;
            o1_upd[o + k] = b / s;
            he_upd[o + k] = c / s;
            a = o2nm_upd[o + k] > small ? o2nm_upd[o + k] : small;
            b = o1nm_upd[o + k] > small ? o1nm_upd[o + k] : small;
            c = henm_upd[o + k] > small ? henm_upd[o + k] : small;
            d = n2nm[k] > small ? n2nm[k] : small;
            s = a + b + c + d;
            o2nm_upd[o + k] = a / s;
            o1nm_upd[o + k] = b / s;
            henm_upd[o + k] = c / s;
        }
    }
    free(n2);
}

/* Post-solve time filter and floor of dt_ng (src/dt_ng.F90:208-213,        */
/* which 0: floor 100 on upd only), minor_ng (src/minor_ng.F90:234-237,     */
/* which 1: floor small = 1e-12 on both) and oplus_ng                        */
/* (src/oplus_ng.F90:337-340, which 2: floor 0 on both).  upd is read and   */
/* floored in place, nm receives the filtered field.  Element-wise, so n =  */
/* nk*ncol elements in any layout.  The floor keeps x when x > fl, as the   */
/* comp_ng restatement above does.                                           */
ORACLE_API void oracle_time_filter_ng(int which, const double *cur, const double *prev, double dtsmooth,
                                      double dtsmooth_div2, long n, double *upd, double *nm)
{
    const double fl = which == 0 ? 100. : which == 1 ? 1.e-12 : 0.;
    long i;
    for (i = 0; i < n; ++i) {
        const double u = upd[i];
        /* dt_ng writes dtsmooth_div2*(tn_nm+tn_upd)+dtsmooth*tn, the other two */
        /* dtsmooth*cur+dtsmooth_div2*(prev+upd): the same two rounded terms    */
        /* summed, and IEEE addition is commutative.                            */
        const double v = which == 0 ? dtsmooth_div2 * (prev[i] + u) + dtsmooth * cur[i]
                                    : dtsmooth * cur[i] + dtsmooth_div2 * (prev[i] + u);
        upd[i] = u > fl ? u : fl;
        nm[i] = (which == 0 || v > fl) ? v : fl;
    }
}

/* ------------------------------------------------------------------------ */
/* settei_ng electron / ion temperature column step (src/settei_ng.F90:     */
/* 60-261): the whole routine is column-local.  Fields (nk, ncol), 2-D      */
/* (ncol).  qtotal is read and updated (qtotal += q_eni_i, :254).  te_out   */
/* and ti_out receive the new Te and Ti; p,q,r,rhs (may be NULL) the system */
/* rows 1..nk-1 after the boundary folds.                                   */
/* ------------------------------------------------------------------------ */
typedef struct {
    const double *tn, *o2, *o1, *he, *n2, *ne, *te, *ti, *op, *o2p, *nplus, *n2p, *nop, *xnmbar, *xnmbari, *scht,
        *schti, *qji_ti, *qop2p, *qop2d, *qo2p, *qop, *qn2p, *qnp, *qnop, *Q1, *Q2;
    const double *t_lbc, *chi, *rlatm, *dipmag, *qteaur;
} oracle_settei_fields;

typedef struct {
    double f107, dipmin, dz, evergs, avo, rmass_o1;
    double rmassinv_o2, rmassinv_o1, rmassinv_he, rmassinv_n2, rmassinv_n4s, rmassinv_no;
    double b[9], fb[3];
    int et, electron_heating;
} oracle_settei_consts;

static double omax(double a, double b) { return a > b ? a : b; }
static double omin(double a, double b) { return a < b ? a : b; }

ORACLE_API void oracle_settei_ng(const oracle_settei_fields *F, const oracle_settei_consts *C, int nk, long ncol,
                                 double *te_out, double *ti_out, double *qtotal, double *p_out, double *q_out,
                                 double *r_out, double *rhs_out)
{
    const double fpolar = -3.0e+9, del = 1.e-6, alam = 0.0069, ad = 0.0091, sd = 2.3e-11;
    const double pi = 4.0 * atan(1.0), rtd = 180.0 / pi, dz = C->dz, ev = C->evergs;
    const double *b = C->b, *fb = C->fb;
    double *w = (double *)malloc(sizeof(double) * 21 * (size_t)nk);
    long col;
    if (nk < 3) { free(w); return; }
    for (col = 0; col < ncol; ++col) {
        const size_t o = (size_t)nk * col;
        const double *tn = F->tn + o, *o2 = F->o2 + o, *o1 = F->o1 + o, *he = F->he + o, *n2 = F->n2 + o,
                     *ne = F->ne + o, *te = F->te + o, *ti = F->ti + o, *xnmbar = F->xnmbar + o,
                     *xnmbari = F->xnmbari + o, *hmid = F->scht + o, *hint = F->schti + o;
        double *te_int = w, *o2n = w + nk, *o1n = w + 2 * nk, *hen = w + 3 * nk, *n2n = w + 4 * nk,
               *tn_int = w + 5 * nk, *tek0 = w + 6 * nk, *p = w + 7 * nk, *q = w + 8 * nk, *r = w + 9 * nk,
               *rhs = w + 10 * nk, *th = w + 11 * nk, *qtot = w + 12 * nk, *rne = w + 13 * nk,
               *loss_ei = w + 14 * nk, *loss_in = w + 15 * nk, *q_eni = w + 16 * nk, *ws = w + 17 * nk,
               *x = w + 20 * nk;
        int k;
        /* fe: the upper-boundary heat flux (:62-87) */
        const double f107te = omin(C->f107, 235.);
        const double arl = fabs(F->rlatm[col]), chi = F->chi[col];
        double a = 0., fed, fen, fe;
        if (arl >= pi / 4.5) a = 1.;
        if (arl < pi / 4.5 && arl > pi / 18) a = .5 * (1. + cos(arl * 6. - pi * 4. / 3.));
        if (arl <= pi / 18) a = 0.;
        fed = -9.0e+7 * f107te * a;
        fen = fed / 2.;
        fed = fed + F->qteaur[col];
        fen = fen + F->qteaur[col];
        fe = chi >= .5 * pi ? fen : fed;
        if ((chi * rtd - 80.) * (chi * rtd - 100.) >= 0.) fe = fe * ev;
        else fe = (.5 * (fed + fen) + .5 * (fed - fen) * cos(pi * (chi * rtd - 80.) / 20.)) * ev;
        if (arl >= pi / 3.) fe = fe + fpolar * ev;
        /* interface quantities (:89-120) */
        for (k = 1; k < nk - 1; ++k) {
            te_int[k] = .5 * (te[k] + te[k - 1]);
            o2n[k] = .5 * (o2[k] + o2[k - 1]);
            o1n[k] = .5 * (o1[k] + o1[k - 1]);
            hen[k] = .5 * (he[k] + he[k - 1]);
            n2n[k] = .5 * (n2[k] + n2[k - 1]);
            tn_int[k] = .5 * (tn[k] + tn[k - 1]);
        }
        te_int[0] = omax(1.5 * te[0] - .5 * te[1], F->t_lbc[col]);
        o2n[0] = .5 * (fb[0] + (b[0] + 1.) * o2[0] + b[3] * o1[0] + b[6] * he[0]);
        o1n[0] = .5 * (fb[0] + b[0] * o2[0] + (b[3] + 1.) * o1[0] + b[6] * he[0]);
        hen[0] = .5 * (fb[0] + b[0] * o2[0] + b[3] * o1[0] + (b[6] + 1.) * he[0]);
        n2n[0] = omax(1. - o2n[0] - o1n[0] - hen[0], 0.);
        tn_int[0] = F->t_lbc[col];
        te_int[nk - 1] = 1.5 * te[nk - 2] - .5 * te[nk - 3];
        o2n[nk - 1] = .5 * (o2[nk - 1] + o2[nk - 2]);
        o1n[nk - 1] = .5 * (o1[nk - 1] + o1[nk - 2]);
        hen[nk - 1] = .5 * (he[nk - 1] + he[nk - 2]);
        n2n[nk - 1] = .5 * (n2[nk - 1] + n2[nk - 2]);
        tn_int[nk - 1] = 1.5 * tn[nk - 2] - .5 * tn[nk - 3];
        for (k = 0; k < nk; ++k) {
            n2n[k] = omax(n2n[k], 0.);
            o2n[k] = xnmbari[k] * o2n[k] * C->rmassinv_o2;
            o1n[k] = xnmbari[k] * o1n[k] * C->rmassinv_o1;
            hen[k] = xnmbari[k] * hen[k] * C->rmassinv_he;
            n2n[k] = xnmbari[k] * n2n[k] * C->rmassinv_n2;
        }
        /* thermal conductivity and the conduction rows (:122-155) */
        {
            const double sd_ = sin(omax(fabs(F->dipmag[col]), C->dipmin));
            const double sindip = omax(sd_ * sd_, .10);
            for (k = 0; k < nk; ++k) {
                const double rt = sqrt(te_int[k]);
                tek0[k] = 7.5e5 /
                          (1. + 3.22e4 * (te_int[k] * te_int[k]) / ne[k] *
                                    ((2.20e-16 + 7.92e-18 * rt) * o2n[k] + 1.10e-16 * (1. + 5.7e-4 * te_int[k]) * o1n[k] +
                                     5.60e-16 * hen[k] + (2.82e-17 - 3.41e-21 * te_int[k]) * rt * n2n[k])) *
                          ev;
                p[k] = 2. / 7. / (hmid[k] * (dz * dz));
                p[k] = p[k] * sindip;
                th[k] = tek0[k] / hint[k];
            }
            for (k = 0; k < nk; ++k) {
                const double th1 = k < nk - 1 ? th[k + 1] : 2. * th[nk - 1] - th[nk - 2];
                r[k] = p[k] * th1;
                p[k] = p[k] * th[k];
                q[k] = -(p[k] + r[k]);
                rhs[k] = 0.;
            }
            q[0] = q[0] - p[0];
            rhs[0] = rhs[0] - 2. * p[0] * pow(tn_int[0], 3.5);
            p[0] = 0.;
            q[nk - 2] = q[nk - 2] + r[nk - 2];
            rhs[nk - 2] = rhs[nk - 2] + r[nk - 2] * dz * 3.5 * hint[nk - 1] * fe / tek0[nk - 1];
            r[nk - 2] = 0.;
        }
        /* heating (:157-186) */
        for (k = 0; k < nk; ++k)
            qtot[k] = omax(F->qo2p[o + k] + F->qop[o + k] + F->qn2p[o + k] + F->qnop[o + k] + F->qnp[o + k] +
                               F->qop2d[o + k] + F->qop2p[o + k],
                           1.e-20);
        for (k = 0; k < nk - 1; ++k) qtot[k] = sqrt(qtot[k] * qtot[k + 1]);
        qtot[nk - 1] = 0.;
        for (k = 0; k < nk - 1; ++k) rne[k] = ne[k] * ne[k + 1];
        rne[nk - 1] = ne[nk - 1] * ne[nk - 1] * ne[nk - 1] / ne[nk - 2];
        for (k = 0; k < nk; ++k) {
            rne[k] = sqrt(omax(rne[k], 1.e4));
            o2n[k] = xnmbar[k] * o2[k] * C->rmassinv_o2;
            o1n[k] = xnmbar[k] * o1[k] * C->rmassinv_o1;
            hen[k] = xnmbar[k] * he[k] * C->rmassinv_he;
            n2n[k] = xnmbar[k] * n2[k] * C->rmassinv_n2;
            double qe;
            if (C->electron_heating == 6) {
                qe = log(rne[k] / (o2n[k] + n2n[k] + o1n[k]));
                qe = exp(((((((-1.249e-5 * qe - 5.755e-4) * qe - 9.346e-3) * qe - 5.900e-2) * qe - 4.392e-2) * qe +
                           1.056) * qe + 5.342));
            } else {
                qe = log(rne[k] / (o2n[k] + n2n[k] + 0.1 * o1n[k]));
                qe = exp(-((((0.001996 * qe + 0.08034) * qe + 1.166) * qe + 6.941) * qe + 12.75));
            }
            rhs[k] = rhs[k] - qe * qtot[k] * ev;
            if (C->et) rhs[k] = rhs[k] - (F->Q1[o + k] + F->Q2[o + k]) * 10.0;
        }
        /* electron cooling, electron-ion and ion-neutral exchange (:188-246) */
        for (k = 0; k < nk; ++k) {
            const double tek = te[k], tnk = tn[k], rt = sqrt(tek);
            double coll, l2v, leo2, leo1, lehe, len2, len, lxen;
            const double leo1d = 0.;
            if (tek >= 1000.) coll = 2.e-7 * exp(-4605.2 / tek);
            else coll = 5.71e-8 * exp(-3352.6 / tek);
            if (tek > 2000.) coll = 2.53e-6 * rt * exp(-17620. / tek);
            if (fabs(tek - tnk) < del) l2v = 3200. / (tnk * tnk);
            else l2v = 1. / (tek - tnk) * (1. - exp(-3200. * (tek - tnk) / (tek * tnk)));
            l2v = 1.3e-4 * l2v * coll;
            leo2 = o2n[k] * (1.21e-18 * (1. + 3.6e-2 * rt) * rt + 6.9e-14 / rt + 3.125e-21 * (tek * tek));
            leo1 = o1n[k] * (7.9e-19 * (1. + 5.7e-4 * tek) * rt + 3.4e-12 * (1. - 7.e-5 * tek) / tnk * (150. / tek + 0.4));
            lehe = hen[k] * 2.46e-17 * rt;
            len2 = n2n[k] * (1.77E-19 * (1. - 1.21E-4 * tek) * tek + 2.9e-14 / rt + l2v);
            len = leo2 + leo1 + lehe + len2;
            if (C->et && tek > 500.0 && F->Q2[o + k] > 0.0) len = len * exp(-7.54E-4 * (tek - 500.0));
            lxen = (len + o1n[k] * (1. - alam / (ad + sd * n2n[k])) * leo1d) * rne[k] * ev;
            len = (len + o1n[k] * leo1d) * rne[k] * ev;
            loss_ei[k] = 3.2e-8 * rne[k] / (rt * tek) * 15. * ev * C->rmass_o1 *
                         (F->op[o + k] * C->rmassinv_o1 + F->o2p[o + k] * C->rmassinv_o2 +
                          F->nplus[o + k] * C->rmassinv_n4s + F->n2p[o + k] * C->rmassinv_n2 +
                          F->nop[o + k] * C->rmassinv_no);
            const double rtn = sqrt(2 * tnk);
            loss_in[k] = 1e-14 * ev *
                         (F->op[o + k] * (5.8 * o2n[k] + 0.21 * o1n[k] * rtn + 2.8 * hen[k] + 6.6 * n2n[k]) +
                          F->o2p[o + k] * (0.14 * o2n[k] * rtn + 4.36 * o1n[k] + 1.63 * hen[k] + 5.81 * n2n[k]) +
                          F->nplus[o + k] * (5.84 * o2n[k] + 5.84 * o1n[k] + 3.05 * hen[k] + 6.56 * n2n[k]) +
                          F->n2p[o + k] * (5.54 * o2n[k] + 4.65 * o1n[k] + 1.82 * hen[k] + 0.27 * n2n[k] * rtn) +
                          F->nop[o + k] * (5.45 * o2n[k] + 4.5 * o1n[k] + 1.72 * hen[k] + 5.92 * n2n[k]));
            q[k] = q[k] - (len + loss_ei[k]) / pow(tek, 2.5);
            rhs[k] = rhs[k] - len * tnk - loss_ei[k] * ti[k];
            q_eni[k] = loss_ei[k] * omax(tek - ti[k], 0.);
            q_eni[k] = (lxen * (tek - tnk) + q_eni[k]) * C->avo / xnmbar[k];
        }
        /* qtotal += q_eni at interfaces (:248-254) */
        for (k = 1; k < nk - 1; ++k) qtotal[o + k] = qtotal[o + k] + .5 * (q_eni[k - 1] + q_eni[k]);
        {
            const double q0 = 1.5 * q_eni[0] - 0.5 * q_eni[1], qn = 1.5 * q_eni[nk - 2] - 0.5 * q_eni[nk - 3];
            qtotal[o] = qtotal[o] + q0;
            qtotal[o + nk - 1] = qtotal[o + nk - 1] + qn;
        }
        if (p_out)
            for (k = 0; k < nk; ++k) {
                p_out[o + k] = p[k];
                q_out[o + k] = q[k];
                r_out[o + k] = r[k];
                rhs_out[o + k] = rhs[k];
            }
        /* solve rows 1..nk-1, Te = (Te^3.5)^(2/7), top level, Ti (:256-261) */
        thomas_column(p, q, r, rhs, x, nk - 1, ws);
        for (k = 0; k < nk - 1; ++k) x[k] = pow(x[k], 2. / 7.);
        x[nk - 1] = x[nk - 2] * x[nk - 2] / x[nk - 3];
        for (k = 0; k < nk; ++k) {
            const double t = omax(x[k], tn[k]);
            te_out[o + k] = t;
            ti_out[o + k] = omax((F->qji_ti[o + k] * xnmbar[k] / C->avo + loss_ei[k] * t + loss_in[k] * tn[k]) /
                                     (loss_ei[k] + loss_in[k]),
                                 tn[k]);
        }
    }
    free(w);
}

/* ------------------------------------------------------------------------ */
/* oplus_ng O+ column step, vertical part (src/oplus_ng.F90:125-303).       */
/* The terms that need horizontal derivatives are inputs, computed by the   */
/* host model as the reference does: explicit_h = -explic*diffexp +         */
/* vdotn_h + bdotdh_bvel (:178-207), bdotdh_djbz = bdotdh(dj*bz) (:234),    */
/* dvb = (div b + 2 bz)/re before its division by bz (:101-107), and        */
/* optm1_smooth2 = smooth_ng(optm1) (:162).  Fields (nk, ncol); 2-D (ncol); */
/* zpint (nk).  Outputs: opout rows 1..nk (the top from :307), xiop2p,      */
/* xiop2d (:285-288); Fe, Fn (:164-169) and the system p,q,r,explicit rows   */
/* 1..nk-1 may be NULL.  opout is before the lateral-boundary overwrite,    */
/* the time filter and the max(.,0) of :332-340, which the caller applies.   */
/* ------------------------------------------------------------------------ */
typedef struct {
    const double *tn, *te, *ti, *o2, *o1, *n2, *he, *n2d, *ne, *u, *v, *w, *wi, *xnmbar, *scht, *qop2p, *qop2d,
        *qop, *rk1, *rk2, *rk19, *rk20, *rk25, *op, *optm1_smooth2, *explicit_h, *bdotdh_djbz;
    const double *bx, *by, *bz, *dvb, *rlatm, *chi, *dipmag, *sndec, *csdec;
    const double *zpint;
} oracle_oplus_fields;

typedef struct {
    double rmass_op, gask, grav, re, rmassinv_o2, rmassinv_o1, rmassinv_n2, rmassinv_n2d, rmassinv_he;
    double rk10, rk16, rk17, rk18, rk21, rk22, rk23, rk24, rk26, rk27;
    double colfac, opdiffcap, dtx2inv, dz, dlev;
    int nstep_sub;
} oracle_oplus_consts;

/* The O+ column step, and (diag not NULL) instead of the solve the history
 * diagnostics of a given solution xsol (oplus_ng.F90:309-330) with the
 * horizontal terms h3 = diffexp, vdotn_h, bdotdh_bvel (each may be NULL: 0). */
static void oplus_core(const oracle_oplus_fields *F, const oracle_oplus_consts *C, int nk, long ncol, double *opout,
                       double *xiop2p, double *xiop2d, double *Fe, double *Fn, double *p_out, double *q_out,
                       double *r_out, double *f_out, const double *xsol, const double *const *h3, double *diag)
{
    const double explic = 1., phid = 2.0e8, phin = -2.0e8, ppolar = 0.;
    const double pi = 4.0 * atan(1.0), rtd = 180.0 / pi, dz = C->dz;
    double *w = (double *)malloc(sizeof(double) * 34 * (size_t)nk);
    long col;
    (void)explic;
    if (nk < 3) { free(w); return; }
    for (col = 0; col < ncol; ++col) {
        const size_t o = (size_t)nk * col;
#define FL(name) (F->name + o)
        const double *tn = FL(tn), *te = FL(te), *ti = FL(ti), *o2 = FL(o2), *o1 = FL(o1), *n2 = FL(n2),
                     *he = FL(he), *n2d = FL(n2d), *ne = FL(ne), *uu = FL(u), *vv = FL(v), *ww = FL(w),
                     *wiw = FL(wi), *xnmbar = FL(xnmbar), *hj = FL(scht), *qop = FL(qop), *op = FL(op);
        double *dj = w, *bdotu = w + nk, *hdz = w + 2 * nk, *hdzi = w + 3 * nk, *tp1 = w + 4 * nk,
               *tph1 = w + 5 * nk, *tph0 = w + 6 * nk, *djint = w + 7 * nk, *hdzm = w + 8 * nk, *hdzp = w + 9 * nk,
               *p = w + 10 * nk, *q = w + 11 * nk, *r = w + 12 * nk, *ex = w + 13 * nk, *ol = w + 14 * nk,
               *wni = w + 15 * nk, *wii = w + 16 * nk, *vni = w + 17 * nk, *tpop = w + 18 * nk, *ws = w + 19 * nk,
               *x = w + 22 * nk, *part = w + 24 * nk, *prodv = w + 33 * nk;
        const double bx = F->bx[col], by = F->by[col], bz = F->bz[col];
        int k;
        /* oplus_flux (:88-99) */
        const double arl = fabs(F->rlatm[col]), chi = F->chi[col];
        double a = 0., opflux;
        if (arl >= pi / 4.5) a = 1.;
        if (arl < pi / 4.5 && arl > pi / 18) a = .5 * (1. + cos(arl * 6. - pi * 4. / 3.));
        if (arl <= pi / 18) a = 0.;
        {
            const double fed = phid * a, fen = phin * a;
            opflux = chi >= 0.5 * pi ? fen : fed;
            if ((chi * rtd - 80.) * (chi * rtd - 100.) < 0.)
                opflux = .5 * (fed + fen) + .5 * (fed - fen) * cos(pi * (chi * rtd - 80.) / 20.);
            if (arl >= pi / 3.) opflux = opflux + ppolar;
        }
        /* interface winds (:112-123) */
        for (k = 0; k < nk - 1; ++k) {
            wni[k] = .5 * (ww[k] + ww[k + 1]);
            wii[k] = .5 * (wiw[k] + wiw[k + 1]);
        }
        wni[nk - 1] = 1.5 * ww[nk - 1] - .5 * ww[nk - 2];
        wii[nk - 1] = 1.5 * wiw[nk - 1] - .5 * wiw[nk - 2];
        /* rrk: collision frequency and diffusion coefficient (:125-135) */
        for (k = 0; k < nk; ++k) {
            const double tr = 0.5 * (tn[k] + ti[k]);
            const double lg = 1. - 0.064 * log10(tr);
            vni[k] = 18.1 * o2[k] * C->rmassinv_o2 + o1[k] * C->rmassinv_o1 * sqrt(tr) * (lg * lg) * C->colfac +
                     3.6 * he[k] * C->rmassinv_he + 18.6 * n2[k] * C->rmassinv_n2;
            dj[k] = 1.42E17 / (xnmbar[k] * vni[k]);
            vni[k] = 16 * 3.53E-11 * vni[k];
            if (!(fabs(C->opdiffcap - 0.) < 1e-9)) {
                const double cap = C->opdiffcap / (1 + pow(2., F->zpint[k] - 6));
                dj[k] = dj[k] < cap ? dj[k] : cap;
            }
            bdotu[k] = bx * uu[k] + by * vv[k] + hj[k] * bz * wni[k];
            tpop[k] = (te[k] + ti[k]) * op[k];
        }
        /* Fe, Fn (:151-169) */
        if (Fe) {
            const double sncs = sin(F->dipmag[col]) * cos(F->dipmag[col]);
            for (k = 0; k < nk; ++k) {
                double d;
                if (k == 0) d = tpop[1] - tpop[0];
                else if (k == nk - 1) d = tpop[nk - 1] - tpop[nk - 2];
                else if (k == nk - 2) d = tpop[nk - 2] - tpop[nk - 3];
                else d = (tpop[k + 1] - tpop[k - 1]) / 2.;
                const double diffj = 1. / (hj[k] * C->dlev) * d + C->rmass_op * C->grav / C->gask * op[k];
                const double wd = vni[k] * diffj * dj[k];
                Fe[o + k] = wd * sncs * F->sndec[col];
                Fn[o + k] = wd * sncs * F->csdec[col];
            }
        }
        /* vertical coefficients (:209-262) */
        const double dvbz = F->dvb[col] / bz;
        const double gmr = C->grav * C->rmass_op / (2. * C->gask);
        for (k = 0; k < nk; ++k) {
            hdz[k] = 1. / (hj[k] * dz);
            tp1[k] = 0.5 * (ti[k] + te[k]);
        }
        for (k = 1; k < nk - 1; ++k) hdzi[k] = 0.5 * (hdz[k - 1] + hdz[k]);
        hdzi[0] = 1.5 * hdz[0] - 0.5 * hdz[1];
        hdzi[nk - 1] = 1.5 * hdz[nk - 2] - 0.5 * hdz[nk - 3];
        for (k = 0; k < nk; ++k) tph1[k] = 2. * tp1[k] * hdzi[k] + gmr;
        for (k = 1; k < nk; ++k) tph0[k] = 2. * tp1[k - 1] * hdzi[k] - gmr;
        tph1[nk - 1] = 2. * (2. * tp1[nk - 2] - tp1[nk - 3]) * hdzi[nk - 1] + gmr;
        tph0[0] = 2. * (2. * tp1[0] - tp1[1]) * hdzi[0] - gmr;
        for (k = 1; k < nk - 1; ++k) djint[k] = 0.5 * (dj[k - 1] + dj[k]);
        djint[0] = 1.5 * dj[0] - 0.5 * dj[1];
        djint[nk - 1] = 1.5 * dj[nk - 2] - 0.5 * dj[nk - 3];
        for (k = 0; k < nk; ++k) {
            const double divbz = dvbz + F->bdotdh_djbz[o + k] / (dj[k] * (bz * bz));
            hdzm[k] = (hdz[k] - 0.5 * divbz) * (bz * bz);
            hdzp[k] = (hdz[k] + 0.5 * divbz) * (bz * bz);
            ex[k] = F->explicit_h[o + k] - F->optm1_smooth2[o + k] * C->dtx2inv * C->nstep_sub;
        }
        for (k = 0; k < nk - 1; ++k) {
            const double diffp = hdzm[k] * djint[k] * tph0[k];
            const double diffq = -(hdzp[k] * djint[k + 1] * tph0[k + 1] + hdzm[k] * djint[k] * tph1[k]);
            const double diffr = hdzp[k] * djint[k + 1] * tph1[k + 1];
            const double driftp = wii[k] * 0.5 * hdz[k], driftq = -wii[k] * 6. / C->re, driftr = -wii[k] * 0.5 * hdz[k];
            double windp, windq, windr;
            if (k == 0) windp = bz * (2. * bdotu[0] - bdotu[1]) * 0.5 * hdz[0];
            else windp = bz * bdotu[k - 1] * 0.5 * hdz[k];
            windq = -bdotu[k] * dvbz * bz;
            if (k == nk - 2) windr = bz * (2. * bdotu[nk - 2] - bdotu[nk - 3]) * 0.5 * hdz[nk - 2];
            else windr = -bz * bdotu[k + 1] * 0.5 * hdz[k];
            {
                const double pt[9] = {diffp, diffq, diffr, driftp, driftq, driftr, windp, windq, windr};
                int e;
                for (e = 0; e < 9; ++e) part[e * nk + k] = pt[e];
            }
            p[k] = diffp + driftp + windp;
            q[k] = diffq + driftq + windq - C->dtx2inv * C->nstep_sub;
            r[k] = diffr + driftr + windr;
        }
        {
            const double ubcb = -(bz * bz) * djint[nk - 1] * tph0[nk - 1];
            const double ubca = -(bz * bz) * djint[nk - 1] * tph1[nk - 1];
            q[nk - 2] = q[nk - 2] + ubcb / ubca * r[nk - 2];
            ex[nk - 2] = ex[nk - 2] - opflux * r[nk - 2] / ubca;
            r[nk - 2] = 0.;
        }
        /* chemistry (:285-299) */
        for (k = 0; k < nk; ++k) {
            const double q2pi = k < nk - 1 ? .5 * (F->qop2p[o + k] + F->qop2p[o + k + 1])
                                           : 1.5 * F->qop2p[o + nk - 1] - .5 * F->qop2p[o + nk - 2];
            const double q2di = k < nk - 1 ? .5 * (F->qop2d[o + k] + F->qop2d[o + k + 1])
                                           : 1.5 * F->qop2d[o + nk - 1] - .5 * F->qop2d[o + nk - 2];
            const double qopi = k < nk - 1 ? .5 * (qop[k] + qop[k + 1]) : 1.5 * qop[nk - 1] - .5 * qop[nk - 2];
            const double rk19 = F->rk19[o + k], rk20 = F->rk20[o + k], rk25 = F->rk25[o + k];
            const double x2p = q2pi / (xnmbar[k] * ((C->rk16 + C->rk17) * n2[k] * C->rmassinv_n2 +
                                                   C->rk18 * o1[k] * C->rmassinv_o1) +
                                       (rk19 + rk20) * ne[k] + C->rk21 + C->rk22);
            const double x2d = (q2di + (rk20 * ne[k] + C->rk22) * x2p) /
                               (xnmbar[k] * (C->rk23 * n2[k] * C->rmassinv_n2 + C->rk24 * o1[k] * C->rmassinv_o1 +
                                             C->rk26 * o2[k] * C->rmassinv_o2) +
                                rk25 * ne[k] + C->rk27);
            if (xiop2p) xiop2p[o + k] = x2p;
            if (xiop2d) xiop2d[o + k] = x2d;
            ol[k] = xnmbar[k] * (F->rk1[o + k] * o2[k] * C->rmassinv_o2 + F->rk2[o + k] * n2[k] * C->rmassinv_n2 +
                                 C->rk10 * n2d[k] * C->rmassinv_n2d);
            if (k < nk - 1) q[k] = q[k] - ol[k];
            const double prod = qopi + (rk19 * ne[k] + C->rk21) * x2p + (rk25 * ne[k] + C->rk27) * x2d +
                                (C->rk18 * x2p + C->rk24 * x2d) * o1[k] * C->rmassinv_o1 * xnmbar[k];
            ex[k] = ex[k] - prod;
            prodv[k] = prod;
        }
        if (diag) {
            /* dopdt, op_prod, -op_loss_out, diffsum, driftsum, windsum (:309-330) */
            const double *xs = xsol + o;
            const size_t slab = (size_t)nk * ncol;
            double *d[6];
            int n;
            for (n = 0; n < 6; ++n) d[n] = diag + n * slab + o;
            for (k = 0; k < nk; ++k) {
                d[0][k] = (xs[k] - F->optm1_smooth2[o + k]) * C->dtx2inv * C->nstep_sub;
                d[1][k] = prodv[k];
                d[2][k] = -(ol[k] * xs[k]);
                d[3][k] = d[4][k] = d[5][k] = 0.;
            }
            for (k = 1; k < nk - 1; ++k)
                for (n = 0; n < 3; ++n) {
                    const double hz = h3 && h3[n] ? h3[n][o + k] : 0.;
                    const double *pt = part + 3 * n * nk;
                    d[3 + n][k] = (n == 0 ? hz : -hz) + pt[k] * xs[k - 1] + pt[nk + k] * xs[k] + pt[2 * nk + k] * xs[k + 1];
                }
            continue;
        }
        /* lower boundary (:301-303) */
        q[0] = q[0] - p[0];
        ex[0] = ex[0] - 2. * p[0] * qop[0] / (1.5 * ol[0] - 0.5 * ol[1]);
        p[0] = 0.;
        if (p_out)
            for (k = 0; k < nk - 1; ++k) {
                p_out[o + k] = p[k];
                q_out[o + k] = q[k];
                r_out[o + k] = r[k];
                f_out[o + k] = ex[k];
            }
        /* solve rows 1..nk-1 and the top level (:305-307) */
        thomas_column(p, q, r, ex, x, nk - 1, ws);
        for (k = 0; k < nk - 1; ++k) opout[o + k] = x[k];
        opout[o + nk - 1] = x[nk - 2] * x[nk - 2] / x[nk - 3];
#undef FL
    }
    free(w);
}

ORACLE_API void oracle_oplus_ng(const oracle_oplus_fields *F, const oracle_oplus_consts *C, int nk, long ncol,
                                double *opout, double *xiop2p, double *xiop2d, double *Fe, double *Fn,
                                double *p_out, double *q_out, double *r_out, double *f_out)
{
    oplus_core(F, C, nk, ncol, opout, xiop2p, xiop2d, Fe, Fn, p_out, q_out, r_out, f_out, NULL, NULL, NULL);
}

/* oplus_ng's history diagnostics (oplus_ng.F90:309-330) of the solution
 * opout (rows 1..nk, the top included, before the lateral overwrite and the
 * post steps): 6 planes (nk, ncol) DOPDT, OP_PROD, OP_LOSS (= -op_loss*opout),
 * OP_DIFF, OP_DRIFT, OP_WIND.  The last three add the horizontal terms
 * diffexp, -vdotn_h, -bdotdh_bvel the host model computes (NULL: 0) to the
 * vertical parts, on levels 2..nk-1 (1-based); the reference leaves the
 * first and top levels unset, here they are 0. */
ORACLE_API void oracle_oplus_diag_ng(const oracle_oplus_fields *F, const oracle_oplus_consts *C, int nk, long ncol,
                                     const double *opout, const double *diffexp, const double *vdotn_h,
                                     const double *bdotdh_bvel, double *diag)
{
    const double *h3[3] = {diffexp, vdotn_h, bdotdh_bvel};
    oplus_core(F, C, nk, ncol, NULL, NULL, NULL, NULL, NULL, NULL, NULL, NULL, NULL, opout, h3, diag);
}

/* ------------------------------------------------------------------------ */
/* Horizontal operators of one nest held as a single subdomain: arrays       */
/* (nk, nlon+4, nlat+4) over the ghost-inclusive lond0:lond1 x latd0:latd1, */
/* every lateral edge a boundary (is_bndry all true, the one-task           */
/* decomposition of src/fields_ng.F90:143-147), so the halo syncs of        */
/* src/sync_ng.F90 exchange nothing.                                         */
/* ------------------------------------------------------------------------ */

/* df_3d (src/dffm_ng.F90:66-110) along lon (dir 0) or lat (dir 1), order   */
/* 1 or 2: centred differences over 2*order spacings, one-sided at the      */
/* edges.                                                                    */
static void hz_df(const double *f, double *df, int order, int dir, int nk, int nlond, int nlatd)
{
    const long s = dir == 0 ? nk : (long)nk * nlond;
    const int n = dir == 0 ? nlond : nlatd;
    int k, i, j;
    for (j = 0; j < nlatd; ++j)
        for (i = 0; i < nlond; ++i)
            for (k = 0; k < nk; ++k) {
                const long o = k + (long)nk * (i + (long)nlond * j);
                const int t = dir == 0 ? i : j;
                if (t == 0) df[o] = f[o + s] - f[o];
                else if (t == n - 1) df[o] = f[o] - f[o - s];
                else if (order == 2 && (t == 1 || t == n - 2)) df[o] = (f[o + s] - f[o - s]) / 2.;
                else df[o] = (f[o + order * s] - f[o - order * s]) / (double)(order * 2);
            }
}

/* fm_3d (src/dffm_ng.F90:166-205): centred means, the input at the edges. */
static void hz_fm(const double *f, double *fm, int order, int dir, int nk, int nlond, int nlatd)
{
    const long s = dir == 0 ? nk : (long)nk * nlond;
    const int n = dir == 0 ? nlond : nlatd;
    int k, i, j;
    for (j = 0; j < nlatd; ++j)
        for (i = 0; i < nlond; ++i)
            for (k = 0; k < nk; ++k) {
                const long o = k + (long)nk * (i + (long)nlond * j);
                const int t = dir == 0 ? i : j;
                if (t == 0 || t == n - 1) fm[o] = f[o];
                else if (order == 2 && (t == 1 || t == n - 2)) fm[o] = (f[o + s] + f[o - s]) / 2.;
                else fm[o] = (f[o + order * s] + f[o - order * s]) / 2.;
            }
}

/* advec_ng (src/advec_ng.F90:1-52): hadvec = wk1/dlamda + wk2*re_inv/dphi  */
/* with the fourth-order lon and lat advection terms; on the two ghost rows */
/* of each boundary side the second-order term alone (:36-37, :47-48).      */
/* racs (nlat+4) per latitude.                                              */
ORACLE_API void oracle_advec_ng(const double *f, const double *un, const double *vn, const double *racs,
                                double dlamda, double dphi, double re_inv, int nk, int nlon, int nlat,
                                double *hadvec)
{
    const int nlond = nlon + 4, nlatd = nlat + 4;
    const size_t n = (size_t)nk * nlond * nlatd;
    double *w = (double *)malloc(sizeof(double) * 4 * n);
    double *m1 = w, *m2 = w + n, *d1 = w + 2 * n, *d2 = w + 3 * n;
    int k, i, j;
    /* wk1 into hadvec */
    hz_fm(un, m1, 1, 0, nk, nlond, nlatd);
    hz_fm(un, m2, 2, 0, nk, nlond, nlatd);
    hz_df(f, d1, 1, 0, nk, nlond, nlatd);
    hz_df(f, d2, 2, 0, nk, nlond, nlatd);
    for (j = 0; j < nlatd; ++j)
        for (i = 0; i < nlond; ++i)
            for (k = 0; k < nk; ++k) {
                const long o = k + (long)nk * (i + (long)nlond * j);
                double v = d1[o] * 2. * 2. / 3. * m1[o] - d2[o] * 4. / 12. * m2[o];
                if (i <= 1 || i >= nlond - 2) v = d1[o] * m1[o];
                hadvec[o] = v * racs[j];
            }
    /* wk2, combined */
    hz_fm(vn, m1, 1, 1, nk, nlond, nlatd);
    hz_fm(vn, m2, 2, 1, nk, nlond, nlatd);
    hz_df(f, d1, 1, 1, nk, nlond, nlatd);
    hz_df(f, d2, 2, 1, nk, nlond, nlatd);
    for (j = 0; j < nlatd; ++j)
        for (i = 0; i < nlond; ++i)
            for (k = 0; k < nk; ++k) {
                const long o = k + (long)nk * (i + (long)nlond * j);
                double v = d1[o] * 2. * 2. / 3. * m1[o] - d2[o] * 4. / 12. * m2[o];
                if (j <= 1 || j >= nlatd - 2) v = d1[o] * m1[o];
                hadvec[o] = hadvec[o] / dlamda + v * re_inv / dphi;
            }
    free(w);
}

/* smooth_ng (src/smooth_ng.F90:1-42): the Shapiro filter in lat, then in   */
/* lon, each with the 3-point form one row in from a boundary and the input */
/* kept on the outermost ghost row.                                          */
ORACLE_API void oracle_smooth_ng(const double *fin, double shapiro, int nk, int nlon, int nlat, double *fout)
{
    const int nlond = nlon + 4, nlatd = nlat + 4;
    const size_t n = (size_t)nk * nlond * nlatd;
    double *w = (double *)malloc(sizeof(double) * 3 * n);
    double *m1 = w, *m2 = w + n, *ft = w + 2 * n;
    int k, i, j;
    hz_fm(fin, m1, 1, 1, nk, nlond, nlatd);
    hz_fm(fin, m2, 2, 1, nk, nlond, nlatd);
    for (j = 0; j < nlatd; ++j)
        for (i = 0; i < nlond; ++i)
            for (k = 0; k < nk; ++k) {
                const long o = k + (long)nk * (i + (long)nlond * j);
                if (j == 0 || j == nlatd - 1) ft[o] = fin[o];
                else if (j == 1 || j == nlatd - 2) ft[o] = fin[o] - shapiro * (-8. * m1[o] + 8. * fin[o]);
                else ft[o] = fin[o] - shapiro * (2. * m2[o] - 8. * m1[o] + 6. * fin[o]);
            }
    hz_fm(ft, m1, 1, 0, nk, nlond, nlatd);
    hz_fm(ft, m2, 2, 0, nk, nlond, nlatd);
    for (j = 0; j < nlatd; ++j)
        for (i = 0; i < nlond; ++i)
            for (k = 0; k < nk; ++k) {
                const long o = k + (long)nk * (i + (long)nlond * j);
                if (i == 0 || i == nlond - 1) fout[o] = ft[o];
                else if (i == 1 || i == nlond - 2) fout[o] = ft[o] - shapiro * (-8. * m1[o] + 8. * ft[o]);
                else fout[o] = ft[o] - shapiro * (2. * m2[o] - 8. * m1[o] + 6. * ft[o]);
            }
    free(w);
}

/* ------------------------------------------------------------------------ */
/* ringfilter (src/ringfilter.F:1-111) over every latitude of a global      */
/* field held whole, as filter_o2o (src/comp.F:1065-1145) runs it once the  */
/* longitudes are gathered, without the MPI gather and scatter.  f is       */
/* (nk, nlon+4, nlat), longitude index 1..nlon+4 with the interior at       */
/* 3..nlon+2 and two periodic points on each side, filtered in place.       */
/* Latitude lat (1..nlat) within nlat_filter rows of a pole takes           */
/* chunk_array's chunk count (src/cons.F:331-355, :25-29 of ringfilter.F);  */
/* the others are left as they are.  order: Fourier modes kept as the mean  */
/* (1 for O2O, 3 for TN and the others); poly: 1 for the piecewise          */
/* polynomial reconstruction of OPLUS (:84-89), 0 the piecewise linear one  */
/* (:91-94).  Returns 1 (and filters nothing) when order >= nlon, where the */
/* reference shuts down.  Sums run in index order, as a loop does.          */
/* ------------------------------------------------------------------------ */
ORACLE_API int oracle_ringfilter(double *f, int nk, int nlon, int nlat, int order, int poly,
                                 const int *chunk_array, int nlat_filter, double dlamda)
{
    const int nlonp4 = nlon + 4;
    int lat, k, i, m, ichnk;
    if (order >= nlon) return 1;
    double *w = (double *)malloc(sizeof(double) * (size_t)(4 * nlon + 2 * order + 2));
    double *wm = w + nlon, *fx = wm + nlon, *avg = fx + nlon, *a = avg + nlon, *b = a + order;
    for (lat = 1; lat <= nlat; ++lat) {
        int nchnk = 0;
        if (lat <= nlat_filter) nchnk = chunk_array[lat - 1];
        else if (lat >= nlat - nlat_filter + 1) nchnk = chunk_array[nlat - lat];
        if (nchnk == 0) continue;
        for (k = 0; k < nk; ++k) {
            /* f(k, i, lat) for the 1-based longitude index i */
            double *row = f + k + (size_t)nk * (size_t)nlonp4 * (size_t)(lat - 1);
#define RF(i) row[(size_t)nk * (size_t)((i) - 1)]
            for (i = 1; i <= nlon; ++i) w[i - 1] = RF(i + 2);
            /* Fourier series to order `order` (:41-52) */
            double a0 = 0.;
            for (i = 0; i < nlon; ++i) a0 = a0 + w[i];
            a0 = a0 / nlon;
            for (m = 0; m < order; ++m) a[m] = b[m] = 0.;
            for (i = 1; i <= nlon; ++i) {
                const double ang = i * dlamda;
                for (m = 1; m <= order; ++m) {
                    a[m - 1] = a[m - 1] + w[i - 1] * cos(m * ang);
                    b[m - 1] = b[m - 1] + w[i - 1] * sin(m * ang);
                }
            }
            for (m = 0; m < order; ++m) {
                a[m] = 2. * a[m] / nlon;
                b[m] = 2. * b[m] / nlon;
            }
            /* the series as the mean (:55-61), the deviation (:64) */
            for (i = 1; i <= nlon; ++i) {
                const double ang = i * dlamda;
                double v = a0;
                for (m = 1; m <= order; ++m) v = v + a[m - 1] * cos(m * ang) + b[m - 1] * sin(m * ang);
                wm[i - 1] = v;
                fx[i - 1] = w[i - 1] - v;
            }
            /* chunk means (:67-71) and the reconstruction (:73-96) */
            const int n = nlon / nchnk;
            for (ichnk = 1; ichnk <= nchnk; ++ichnk) {
                double s = 0.;
                for (i = (ichnk - 1) * n; i < ichnk * n; ++i) s = s + fx[i];
                avg[ichnk - 1] = s / n;
            }
            for (ichnk = 1; ichnk <= nchnk; ++ichnk) {
                int im2 = ichnk - 2, im1 = ichnk - 1, ip1 = ichnk + 1, ip2 = ichnk + 2;
                if (im2 <= 0) im2 += nchnk;
                if (im1 <= 0) im1 += nchnk;
                if (ip1 >= nchnk + 1) ip1 -= nchnk;
                if (ip2 >= nchnk + 1) ip2 -= nchnk;
                const double av = avg[ichnk - 1];
                const double left = (-avg[im2 - 1] + 7. * avg[im1 - 1] + 7. * av - avg[ip1 - 1]) / 12.;
                const double right = (-avg[im1 - 1] + 7. * av + 7. * avg[ip1 - 1] - avg[ip2 - 1]) / 12.;
                const double fa = (left + right - 2. * av) / (double)(n * n);
                const double fb = (3. * av - 2. * left - right) / n;
                for (m = 1; m <= n; ++m) {
                    double *x = fx + (ichnk - 1) * n + m - 1;
                    if (poly)
                        *x = fa * (3. * (double)(m * m) - 3. * m + 1.) + fb * (2. * m - 1.) + left;
                    else
                        *x = (left * (n - m) + right * m) / n;
                }
            }
            /* the full field and its periodic points (:99-104) */
            for (i = 1; i <= nlon; ++i) RF(i + 2) = fx[i - 1] + wm[i - 1];
            RF(1) = RF(nlon + 1);
            RF(2) = RF(nlon + 2);
            RF(nlon + 3) = RF(3);
            RF(nlon + 4) = RF(4);
#undef RF
        }
    }
    free(w);
    return 0;
}
