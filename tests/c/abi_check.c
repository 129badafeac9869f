/*
 * A plain C caller of libtg_colsolve.so: includes include/tg_colsolve.h,
 * links the library with no Python or torch in the process, and checks the
 * host-side behaviour of the ABI that needs no GPU (version string, argument
 * validation, the error message).  With a device present it also solves one
 * small tridiagonal system and checks it against the Thomas recurrence.
 * Exit status 0 on success.
 */
#include <math.h>
#include <stdio.h>
#include <string.h>

#include "tg_colsolve.h"

#define CHECK(cond)                                                        \
    do {                                                                   \
        if (!(cond)) {                                                     \
            fprintf(stderr, "check failed at line %d: %s\n", __LINE__, #cond); \
            return 1;                                                      \
        }                                                                  \
    } while (0)

int main(void)
{
    double a[4] = {0, -1, -1, -1}, b[4] = {4, 4, 4, 4}, c[4] = {-1, -1, -1, 0}, f[4] = {3, 2, 2, 3}, x[4] = {0};
    CHECK(strncmp(tg_version(), "tg_colsolve", 11) == 0);
    /* argument errors are reported before any device call */
    CHECK(tg_trsolv_ng(a, b, c, f, x, 4, 5, 1) == TG_EINVAL);   /* k2 > nk */
    CHECK(strlen(tg_last_error()) > 0);
    CHECK(tg_trsolv_ng(NULL, b, c, f, x, 4, 4, 1) == TG_EINVAL);
    CHECK(tg_blksolve(4, a, b, c, f, NULL, NULL, x, 4, 4, 1) == TG_EINVAL);   /* B not 2 or 3 */
    CHECK(tg_time_filter_ng(7, a, b, 0.95, 0.025, 4, 1, c, f) == TG_EINVAL);
    CHECK(tg_smooth_ng(a, 0.03, 1, 0, 1, x) == TG_EINVAL);                    /* nlon < 1 */
    CHECK(tg_set_refine(0, 1e-11) == TG_EINVAL);

    int rc = tg_trsolv_ng(a, b, c, f, x, 4, 4, 1);
    if (rc == TG_ENODEV) {
        printf("abi_check: ok (no device)\n");
        return 0;
    }
    CHECK(rc == TG_OK);
    /* the same recurrence on the host, in the reference's operation order */
    double w1[4], w2[4], w3[4], y[4];
    w1[0] = b[0];
    w3[0] = f[0] / w1[0];
    for (int k = 1; k < 4; ++k) {
        w2[k - 1] = c[k - 1] / w1[k - 1];
        w1[k] = b[k] - a[k] * w2[k - 1];
        w3[k] = (f[k] - a[k] * w3[k - 1]) / w1[k];
    }
    y[3] = w3[3];
    for (int k = 2; k >= 0; --k) y[k] = w3[k] - w2[k] * y[k + 1];
    for (int k = 0; k < 4; ++k) CHECK(x[k] == y[k]);
    /* the kernels run as the library's sm_100a build */
    int arch = 0;
    CHECK(tg_kernel_arch(&arch) == TG_OK && arch == 100);
    /* the same system as a latitude slab with the periodic columns around it
     * (lon0 = 1, lon1 = lonmax = 5: columns 1, 2, 4, 5 are skipped), queued
     * and flushed; the work arrays are overwritten before the flush */
    double sa[20], sb[20], sc[20], sf[20], sx[20];
    for (int i = 0; i < 5; ++i)
        for (int k = 0; k < 4; ++k) {
            sa[4 * i + k] = a[k];
            sb[4 * i + k] = b[k];
            sc[4 * i + k] = c[k];
            sf[4 * i + k] = f[k];
            sx[4 * i + k] = -1.0;
        }
    CHECK(tg_trsolv_defer(sa, sb, sc, sf, sx, 1, 4, 1, 4, 1, 5, 5) == TG_OK);
    for (int i = 0; i < 20; ++i) sa[i] = sb[i] = sc[i] = sf[i] = NAN;
    CHECK(tg_trsolv_flush() == TG_OK);
    for (int k = 0; k < 4; ++k) CHECK(sx[8 + k] == y[k]);
    for (int i = 0; i < 5; ++i)
        if (i != 2)
            for (int k = 0; k < 4; ++k) CHECK(sx[4 * i + k] == -1.0);
    printf("abi_check: ok (solved on the device)\n");
    return 0;
}
