/*
 * Oracle (test infrastructure only): C restatement of the reference's host
 * matrix generator, include/gen.h:23-38 (generateRandomSymmetricPositiveDefiniteMatrix).
 *
 * Algorithm, as the reference states it: seed glibc rand() with 420; fill the
 * upper triangle of a row-major n x n array, row by row, with rand()/RAND_MAX;
 * mirror it into the lower triangle; add n to every diagonal entry.  The result
 * is symmetric, so row-major and column-major storage coincide.
 *
 * Only tests, the smoke check and the CPU baseline of the bench load this file.
 */
#include <stdlib.h>
#include <stddef.h>

void oracle_ref_spd(double *a, size_t n)
{
    srand(420);
    for (size_t r = 0; r < n; ++r)
        for (size_t c = r; c < n; ++c)
            a[r * n + c] = (double)rand() / (double)RAND_MAX;
    for (size_t r = 0; r < n; ++r)
        for (size_t c = 0; c < r; ++c)
            a[r * n + c] = a[c * n + r];
    for (size_t r = 0; r < n; ++r)
        a[r * n + r] += (double)n;
}

/* Plain triple-loop residual of the reference's verifier, include/verify.h:31-70
 * (LU) and :91-128 (Cholesky): sum over all entries of |A - L*U| where L and U
 * are taken from the in-place column-major factor F (L unit lower for LU).
 * Loop order follows the reference (i, j, k accumulation of L[i,k]*U[k,j]). */
double oracle_ref_verify_lu(const double *a, const double *f, size_t n)
{
    double err = 0.0;
    for (size_t i = 0; i < n; ++i) {
        for (size_t j = 0; j < n; ++j) {
            double s = 0.0;
            for (size_t k = 0; k < n; ++k) {
                double l = (k < i) ? f[i + k * n] : (k == i ? 1.0 : 0.0);
                double u = (k <= j) ? f[k + j * n] : 0.0;
                s += l * u;
            }
            double d = a[i * n + j] - s;
            err += d < 0 ? -d : d;
        }
    }
    return err;
}

double oracle_ref_verify_chol(const double *a, const double *f, size_t n)
{
    double err = 0.0;
    for (size_t i = 0; i < n; ++i) {
        for (size_t j = 0; j < n; ++j) {
            double s = 0.0;
            for (size_t k = 0; k < n; ++k) {
                double l = (k <= i) ? f[i + k * n] : 0.0;      /* L[i,k] */
                double lt = (k <= j) ? f[j + k * n] : 0.0;     /* L^T[k,j] = L[j,k] */
                s += l * lt;
            }
            double d = a[i * n + j] - s;
            err += d < 0 ? -d : d;
        }
    }
    return err;
}
