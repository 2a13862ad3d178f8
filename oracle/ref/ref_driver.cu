// Oracle pin (test infrastructure): a tiny driver around the reference's own host
// generator and verifier, compiled from the reference's headers where they lie
// (include/gen.h:23-38, include/verify.h:17-129).  It runs on the CPU only.
//
//   ref_driver gen <n> <out.bin>                 row-major n*n doubles from the generator
//   ref_driver verify_lu|verify_chol <n> <A.bin> <F.bin>
//       A: the generator's row-major matrix; F: column-major in-place factor.
//       Prints the reference's "error = %.6f" line and "pass=<0|1>".
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>

#include "gen.h"
#include "verify.h"

static bool read_all(const char *path, double *buf, size_t count) {
    FILE *f = fopen(path, "rb");
    if (!f) return false;
    size_t got = fread(buf, sizeof(double), count, f);
    fclose(f);
    return got == count;
}

int main(int argc, char **argv) {
    if (argc < 4) {
        fprintf(stderr, "usage: ref_driver gen|verify_lu|verify_chol n files...\n");
        return 2;
    }
    std::string mode = argv[1];
    const int n = atoi(argv[2]);
    const size_t nn = size_t(n) * size_t(n);
    if (mode == "gen") {
        double *a = (double *)calloc(nn, sizeof(double));
        generateRandomSymmetricPositiveDefiniteMatrix(a, n);
        FILE *f = fopen(argv[3], "wb");
        if (!f) return 3;
        fwrite(a, sizeof(double), nn, f);
        fclose(f);
        free(a);
        return 0;
    }
    if (argc < 5) return 2;
    double *a = (double *)calloc(nn, sizeof(double));
    double *l = (double *)calloc(nn, sizeof(double));
    double *u = (double *)calloc(nn, sizeof(double));  // zero-filled, as large mallocs are
    if (!read_all(argv[3], a, nn) || !read_all(argv[4], l, nn)) return 3;
    bool pass;
    if (mode == "verify_lu") {
        cleanCusolverLUDecompositionResult(l, u, n);
        pass = verifyLUDecomposition(a, l, u, n);
    } else if (mode == "verify_chol") {
        cleanCusolverCholeskyDecompositionResult(l, n);
        pass = verifyCholeskyDecomposition(a, l, n);
    } else {
        return 2;
    }
    printf("pass=%d\n", pass ? 1 : 0);
    free(a);
    free(l);
    free(u);
    return 0;
}
