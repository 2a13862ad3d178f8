// Test infrastructure (oracle side): a wrapper around the reference's include/verify.h for
// the reference's own lu_mustard / cholesky_mustard drivers built by oracle/ref/Makefile.
//
// It sits earlier on the include path than the reference's include/ directory, renames the
// four verification functions of include/verify.h:17-129, pulls the real header in with
// #include_next (so nothing of it is copied) and puts thin wrappers in their place:
//
//   - MTD_REF_DUMP=<path>: the factor exactly as the driver copied it off the device
//     (column-major, n*n doubles, before the clean-up step) is written to <path>, for the
//     parity tests that compare this repository's factors with the reference's;
//   - n <= MTD_REF_VERIFY_MAX (default 2048): the reference's own O(n^3) verification runs
//     unchanged (its "error = " line and pass flag);
//   - larger n: an O(n^2) probe residual ||A X - L (U X)||_F / ||A X||_F over 8 random
//     columns replaces it, printed as "probe_residual = ", passing below 1e-14.
//
// The drivers call clean...Result on the factor right before verify...Decomposition; the
// wrappers keep that order.
#pragma once

#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <vector>

#define cleanCusolverLUDecompositionResult mtd_reference_clean_lu
#define verifyLUDecomposition mtd_reference_verify_lu
#define cleanCusolverCholeskyDecompositionResult mtd_reference_clean_chol
#define verifyCholeskyDecomposition mtd_reference_verify_chol
#include_next <verify.h>
#undef cleanCusolverLUDecompositionResult
#undef verifyLUDecomposition
#undef cleanCusolverCholeskyDecompositionResult
#undef verifyCholeskyDecomposition

namespace mtd_shim {

inline long verify_max() {
    const char *s = std::getenv("MTD_REF_VERIFY_MAX");
    return s ? std::atol(s) : 2048;
}

inline void dump(const double *f, int n) {
    const char *path = std::getenv("MTD_REF_DUMP");
    if (!path) return;
    FILE *fp = std::fopen(path, "wb");
    if (!fp) {
        std::fprintf(stderr, "MTD_REF_DUMP: cannot open %s\n", path);
        return;
    }
    const size_t count = size_t(n) * size_t(n);
    const size_t wrote = std::fwrite(f, sizeof(double), count, fp);
    std::fclose(fp);
    if (wrote != count) std::fprintf(stderr, "MTD_REF_DUMP: short write to %s\n", path);
}

// Raw (column-major, in-place) factor of the last clean call, kept for the probe residual.
inline std::vector<double> &raw() {
    static std::vector<double> r;
    return r;
}

// ||A X - L (U X)||_F / ||A X||_F, X = 8 columns of a fixed xorshift sequence in [-1, 1).
// A is the driver's input (symmetric, so its row- and column-major forms agree); f is the
// raw in-place factor: LU -> unit-lower L below the diagonal and U on and above it;
// Cholesky -> L in the lower triangle (upper triangle ignored).
inline double probe_residual(const double *a, const double *f, int n, bool lu) {
    const int P = 8;
    const size_t N = size_t(n);
    std::vector<double> x(N * P), y(N * P, 0.0), ax(N * P, 0.0), t(N * P, 0.0);
    uint64_t s = 0x9E3779B97F4A7C15ull;
    for (auto &v : x) {
        s ^= s << 13;
        s ^= s >> 7;
        s ^= s << 17;
        v = double(s >> 11) * (2.0 / 9007199254740992.0) - 1.0;
    }
    for (size_t j = 0; j < N; ++j)  // A X, column j of A
        for (int p = 0; p < P; ++p) {
            const double xv = x[j + p * N];
            const double *col = a + j * N;
            double *o = &ax[p * N];
            for (size_t i = 0; i < N; ++i) o[i] += col[i] * xv;
        }
    // t = U X (LU: upper triangle incl. diagonal; Cholesky: L^T X)
    for (size_t j = 0; j < N; ++j) {
        const double *col = f + j * N;
        for (int p = 0; p < P; ++p) {
            if (lu) {
                const double xv = x[j + p * N];
                double *o = &t[p * N];
                for (size_t i = 0; i <= j; ++i) o[i] += col[i] * xv;
            } else {
                double acc = 0.0;
                const double *xp = &x[p * N];
                for (size_t i = j; i < N; ++i) acc += col[i] * xp[i];
                t[j + p * N] = acc;
            }
        }
    }
    // y = L t (LU: unit lower; Cholesky: lower incl. diagonal)
    for (size_t j = 0; j < N; ++j) {
        const double *col = f + j * N;
        for (int p = 0; p < P; ++p) {
            const double tv = t[j + p * N];
            double *o = &y[p * N];
            if (lu) {
                o[j] += tv;
                for (size_t i = j + 1; i < N; ++i) o[i] += col[i] * tv;
            } else {
                for (size_t i = j; i < N; ++i) o[i] += col[i] * tv;
            }
        }
    }
    double num = 0.0, den = 0.0;
    for (size_t i = 0; i < N * P; ++i) {
        const double d = ax[i] - y[i];
        num += d * d;
        den += ax[i] * ax[i];
    }
    return std::sqrt(num / den);
}

inline bool report_probe(const double *a, int n, bool lu) {
    const double r = probe_residual(a, raw().data(), n, lu);
    std::printf("probe_residual = %.3e\n", r);
    return r < 1e-14;
}

}  // namespace mtd_shim

inline void cleanCusolverLUDecompositionResult(double *L, double *U, const int n) {
    mtd_shim::dump(L, n);
    if (n <= mtd_shim::verify_max()) {
        mtd_reference_clean_lu(L, U, n);
        return;
    }
    mtd_shim::raw().assign(L, L + size_t(n) * size_t(n));
}

inline bool verifyLUDecomposition(double *A, double *L, double *U, const int n, bool verbose = false) {
    if (n <= mtd_shim::verify_max()) return mtd_reference_verify_lu(A, L, U, n, verbose);
    return mtd_shim::report_probe(A, n, true);
}

inline void cleanCusolverCholeskyDecompositionResult(double *L, const int n) {
    mtd_shim::dump(L, n);
    if (n <= mtd_shim::verify_max()) {
        mtd_reference_clean_chol(L, n);
        return;
    }
    mtd_shim::raw().assign(L, L + size_t(n) * size_t(n));
}

inline bool verifyCholeskyDecomposition(double *A, double *L, const int n, bool verbose = false) {
    if (n <= mtd_shim::verify_max()) return mtd_reference_verify_chol(A, L, n, verbose);
    return mtd_shim::report_probe(A, n, false);
}
