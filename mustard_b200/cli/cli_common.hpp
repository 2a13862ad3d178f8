// Shared command line and driver loop of lu_mustard / cholesky_mustard.
//
// Flags follow the reference (include/cli.h:21-97, README.md:185-216): -n/-N, -t/-T,
// --tiled, --subgraph, -r/--runs, --verify, --dot, -v/--verbose, --sm, --ws; values as
// `-n=600` or `-n 600`.  The reference requires N % T == 0 (include/cli.h:80-83) and so
// does this driver for -t; `--tile=B` instead sets the tile edge directly and allows a
// ragged last tile.  Extra: --gen=ref|uniform|spd (input; default the reference's
// generator, include/gen.h:23-38), --seed, --timeout (seconds for device-side waits).
//
// Modes: --subgraph runs the persistent device scheduler (the reference's Mustard
// mode); --tiled launches the same tile kernels as one host-launched CUDA graph whose
// edges are the task dependencies (the reference's cudaGraph mode); with neither flag
// the whole matrix is one task graph with an automatically chosen tile edge (the
// reference's single-call mode makes one cuSOLVER call).
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <random>
#include <string>
#include <vector>

#include "mustard_b200.hpp"

namespace mtdcli {

struct Config {
    long long n = 15;
    long long t = 5;
    long long tile = 0;  // --tile, 0 = N / T
    bool tiled = false, subgraph = false, verify = false, dot = false, verbose = false, help = false;
    int runs = 1;
    int sm = 20;
    int ws = 256;
    std::string gen = "ref";
    unsigned long long seed = 2024;
    double timeout = 10.0;
};

inline bool parse_value(const std::string &s, long long &out) {
    char *end = nullptr;
    const long long v = std::strtoll(s.c_str(), &end, 10);
    if (end == s.c_str() || *end) return false;
    out = v;
    return true;
}

inline void usage(const char *prog, const char *what) {
    std::fprintf(stderr,
                 "Usage: %s [options]\n\n  %s decomposition on one B200 through the persistent task-graph scheduler.\n\n"
                 "  Mode (pick one; default is single-kernel if none given):\n"
                 "    --tiled              Tiled execution (one host-launched CUDA graph of tile kernels)\n"
                 "    --subgraph           Device-scheduled execution (persistent scheduler)\n\n"
                 "  Common options:\n"
                 "    -n, -N=<int>         Matrix dimension N                       [default: 15]\n"
                 "    -t, -T=<int>         Number of tiles (N must be divisible)    [default: 5]\n"
                 "    --tile=<int>         Tile edge B (last tile may be ragged; overrides -t)\n"
                 "    --sm, --smLimit=<int> accepted for compatibility (the scheduler uses every SM)\n"
                 "    --ws, --workspace=<int> accepted for compatibility (no library workspaces)\n"
                 "    -r, --runs=<int>     Number of timing runs                    [default: 1]\n"
                 "    -v, --verbose        Enable verbose output\n"
                 "    --verify             Verify result correctness\n"
                 "    --dot                Dump the task graph in DOT format (graph.dot)\n"
                 "    --gen=ref|uniform|spd  Input generator                         [default: ref]\n"
                 "    --seed=<int>         Seed of the uniform / spd generators\n"
                 "    --timeout=<sec>      Limit on any device-side wait            [default: 10]\n\n"
                 "  Examples:\n    %s -n=600 -t=2 --subgraph --verify\n    %s -n=24000 --tile=512 --subgraph -r=5\n",
                 prog, what, prog, prog);
}

// Returns false (after printing why) when the arguments are invalid.
inline bool parse(int argc, char **argv, Config &c) {
    std::vector<std::string> args(argv + 1, argv + argc);
    for (size_t i = 0; i < args.size(); ++i) {
        std::string a = args[i];
        std::string key = a, val;
        bool has_val = false;
        const size_t eq = a.find('=');
        if (eq != std::string::npos) {
            key = a.substr(0, eq);
            val = a.substr(eq + 1);
            has_val = true;
        }
        while (!key.empty() && key[0] == '-') key.erase(0, 1);
        auto need = [&](long long &dst, const char *what) {
            if (!has_val) {
                if (i + 1 >= args.size()) {
                    std::fprintf(stderr, "Error: Must provide a valid %s value!\n", what);
                    return false;
                }
                val = args[++i];
            }
            if (!parse_value(val, dst)) {
                std::fprintf(stderr, "Error: Must provide a valid %s value! Got '%s'\n", what, val.c_str());
                return false;
            }
            return true;
        };
        long long v = 0;
        if (key == "h" || key == "help") c.help = true;
        else if (key == "n" || key == "N") { if (!need(c.n, "N")) return false; }
        else if (key == "t" || key == "T") { if (!need(c.t, "T")) return false; }
        else if (key == "tile") { if (!need(c.tile, "tile")) return false; }
        else if (key == "r" || key == "R" || key == "run" || key == "runs") {
            if (!need(v, "number of runs") || v < 1) { std::fprintf(stderr, "Error: Must provide a valid number of runs!\n"); return false; }
            c.runs = static_cast<int>(v);
        } else if (key == "sm" || key == "SM" || key == "smLimit") {
            if (!need(v, "SM Limit") || v < 1) return false;
            c.sm = static_cast<int>(v);
        } else if (key == "ws" || key == "w" || key == "W" || key == "workspace") {
            if (!need(v, "workspace") || v < 1 || v > 1024 * 1024) return false;
            c.ws = static_cast<int>(v);
        } else if (key == "seed") {
            if (!need(v, "seed")) return false;
            c.seed = static_cast<unsigned long long>(v);
        } else if (key == "timeout") {
            if (!has_val && i + 1 < args.size()) val = args[++i];
            c.timeout = std::atof(val.c_str());
        } else if (key == "gen") {
            if (!has_val && i + 1 < args.size()) val = args[++i];
            c.gen = val;
        } else if (key == "tiled") c.tiled = true;
        else if (key == "subgraph") c.subgraph = true;
        else if (key == "verify") c.verify = true;
        else if (key == "dot") c.dot = true;
        else if (key == "v" || key == "verbose") c.verbose = true;
        else {
            std::fprintf(stderr, "Error: unknown option '%s'\n", a.c_str());
            return false;
        }
    }
    if (c.help) return false;
    if (c.n < 1 || c.t < 1) {
        std::fprintf(stderr, "Error: N and T must be positive\n");
        return false;
    }
    if (c.tile == 0 && c.n % c.t > 0) {
        std::fprintf(stderr, "Error: N must be divisible by T! Got 'N=%lld & T=%lld'\n", c.n, c.t);
        return false;
    }
    if (c.gen != "ref" && c.gen != "uniform" && c.gen != "spd") {
        std::fprintf(stderr, "Error: --gen must be ref, uniform or spd\n");
        return false;
    }
    return true;
}

inline void cuda_check(cudaError_t e, const char *what) {
    if (e != cudaSuccess) {
        std::fprintf(stderr, "CUDA error in %s: %s\n", what, cudaGetErrorString(e));
        std::exit(EXIT_FAILURE);
    }
}

// Column-major host input.
inline std::vector<double> make_input(const Config &c, bool lu) {
    const size_t n = static_cast<size_t>(c.n);
    std::vector<double> a(n * n);
    if (c.gen == "ref") {
        mustard_b200::check(mtd_generate_reference_host(a.data(), c.n));  // symmetric
        return a;
    }
    double *d = nullptr;
    cuda_check(cudaMalloc(&d, n * n * sizeof(double)), "cudaMalloc");
    mustard_b200::check(mtd_generate(d, c.n, c.n, c.gen == "uniform" ? MTD_GEN_UNIFORM_DIAG : MTD_GEN_SPD,
                                     c.seed, 1.0, nullptr));
    cuda_check(cudaMemcpy(a.data(), d, n * n * sizeof(double), cudaMemcpyDeviceToHost), "cudaMemcpy");
    cuda_check(cudaFree(d), "cudaFree");
    (void)lu;
    return a;
}

// The reference's verifier (include/verify.h:31-70 / :91-128): sum over all entries of
// |A - L U| (|A - L L^T|), passing at <= 1e-6 -- a plain O(n^3) loop, run here for
// n <= 2048.  For every n a normwise residual ||(A - LU) X||_F / ||A X||_F over 8
// random probe vectors is printed as well; above 2048 it decides the pass (<= 1e-12).
inline bool verify(const std::vector<double> &a, const std::vector<double> &f, long long nn, bool lu) {
    const size_t n = static_cast<size_t>(nn);
    auto L = [&](size_t i, size_t k) -> double {  // unit lower for LU
        if (lu) return k < i ? f[i + k * n] : (k == i ? 1.0 : 0.0);
        return k <= i ? f[i + k * n] : 0.0;
    };
    auto U = [&](size_t k, size_t j) -> double {  // U for LU, L^T for Cholesky
        if (lu) return k <= j ? f[k + j * n] : 0.0;
        return k <= j ? f[j + k * n] : 0.0;
    };
    // probe residual
    const int P = 8;
    std::mt19937_64 rng(7);
    std::normal_distribution<double> nd;
    std::vector<double> x(n * P), ux(n * P, 0.0), r(n * P, 0.0), ax(n * P, 0.0);
    for (auto &v : x) v = nd(rng);
    for (int p = 0; p < P; ++p) {
        for (size_t j = 0; j < n; ++j) {
            const double xj = x[j + p * n];
            for (size_t i = 0; i < n; ++i) ax[i + p * n] += a[i + j * n] * xj;
            for (size_t k = 0; k <= j; ++k) ux[k + p * n] += U(k, j) * xj;
        }
        for (size_t k = 0; k < n; ++k) {
            const double uk = ux[k + p * n];
            for (size_t i = k; i < n; ++i) r[i + p * n] += L(i, k) * uk;
        }
    }
    double num = 0.0, den = 0.0;
    for (size_t i = 0; i < n * P; ++i) {
        num += (ax[i] - r[i]) * (ax[i] - r[i]);
        den += ax[i] * ax[i];
    }
    const double resid = std::sqrt(num / den);
    std::printf("normwise residual (8 probes) = %.3e\n", resid);
    if (n > 2048) return resid <= 1e-12;
    double err = 0.0;
    for (size_t i = 0; i < n; ++i)
        for (size_t j = 0; j < n; ++j) {
            double s = 0.0;
            for (size_t k = 0; k < n; ++k) s += L(i, k) * U(k, j);
            err += std::fabs(a[i * n + j] - s);  // the reference indexes A row-major (A symmetric there)
        }
    std::printf("error = %.6f\n", err);
    return err <= 1e-6;
}

inline void write_dot(mustard_b200::TiledGraphCreator &g, const char *path) {
    FILE *f = std::fopen(path, "w");
    if (!f) return;
    std::fprintf(f, "digraph tasks {\n");
    for (size_t t = 0; t < g.subgraphDependencies.size(); ++t)
        for (int d : g.subgraphDependencies[t]) std::fprintf(f, "  %d -> %zu;\n", d, t);
    std::fprintf(f, "}\n");
    std::fclose(f);
}

// Shared main body; kind = MTD_KIND_LU or MTD_KIND_CHOLESKY.
inline int run_main(int argc, char **argv, int kind, const char *what) {
    Config c;
    if (!parse(argc, argv, c)) {
        usage(argv[0], what);
        return 1;
    }
    const bool lu = kind == MTD_KIND_LU;
    long long B;
    const char *mode;
    if (c.tiled || c.subgraph) {
        B = c.tile > 0 ? c.tile : c.n / c.t;
        mode = c.tiled ? "TILED" : "SUBGRAPH";
    } else {
        B = c.tile > 0 ? c.tile : std::min<long long>(c.n, 512);  // auto tile edge
        mode = "Single-kernel";
    }
    if (B < 1 || B > c.n) {
        std::fprintf(stderr, "Error: invalid tile edge %lld\n", B);
        return 1;
    }
    const long long T = (c.n + B - 1) / B;
    std::printf("%s with N=%lld (%lld of %lldx%lld tiles)\n", mode, c.n, T, B, B);
    int sms = 0;
    cuda_check(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, 0), "device query");
    std::printf("Persistent CTAs = %d (one per SM)\n", sms);

    std::vector<double> a = make_input(c, lu);
    const size_t bytes = size_t(c.n) * size_t(c.n) * sizeof(double);
    double *d = nullptr;
    cuda_check(cudaMalloc(&d, bytes), "cudaMalloc");
    cudaStream_t s;
    cuda_check(cudaStreamCreate(&s), "cudaStreamCreate");
    cudaEvent_t e0, e1;
    cuda_check(cudaEventCreate(&e0), "event");
    cuda_check(cudaEventCreate(&e1), "event");

    double total = 0.0;
    int status = 0;
    try {
        mustard_b200::TiledGraphCreator g(kind, c.n, B);
        g.buildTiled();
        if (c.verbose) {
            std::printf("totalNodes=%d\n", g.numTasks());
            g.printDeps();
        }
        if (c.dot) write_dot(g, "./graph.dot");
        g.setTimeout(c.timeout);
        g.finalize();
        for (int r = 0; r < c.runs; ++r) {
            cuda_check(cudaMemcpy(d, a.data(), bytes, cudaMemcpyHostToDevice), "cudaMemcpy");
            cuda_check(cudaEventRecord(e0, s), "event");
            int info = 0;
            const int rc = c.tiled ? mtd_run_graph(g.handle(), d, c.n, s, nullptr) : mtd_run(g.handle(), d, c.n, s, nullptr);
            mustard_b200::check(rc);
            cuda_check(cudaEventRecord(e1, s), "event");
            cuda_check(cudaStreamSynchronize(s), "cudaStreamSynchronize");
            mustard_b200::check(mtd_graph_status(g.handle(), &info), info);
            float ms = 0.f;
            cuda_check(cudaEventElapsedTime(&ms, e0, e1), "event");
            std::printf("device %d | %d run | time (s): %4.4f\n", 0, r, ms * 1e-3);
            total += ms * 1e-3;
        }
    } catch (const mustard_b200::Error &err) {
        std::fprintf(stderr, "mustard_b200 error: %s\n", err.what());
        status = 2;
    }
    if (status == 0 && c.verify) {
        std::vector<double> f(a.size());
        cuda_check(cudaMemcpy(f.data(), d, bytes, cudaMemcpyDeviceToHost), "cudaMemcpy");
        std::printf("Result passes verification: %d\n", verify(a, f, c.n, lu) ? 1 : 0);
    }
    std::printf("Total time used (s): %4.4f\n", total);
    const double flops = lu ? 2.0 * double(c.n) * c.n * c.n / 3.0 : double(c.n) * c.n * c.n / 3.0;
    if (total > 0) std::printf("TFLOP/s (mean over runs): %.3f\n", flops * c.runs / total / 1e12);
    cudaFree(d);
    cudaStreamDestroy(s);
    return status;
}

}  // namespace mtdcli
