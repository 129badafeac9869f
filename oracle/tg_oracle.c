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
