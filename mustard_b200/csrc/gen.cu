// Input generators and the FP64 tensor-core rate probe.
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdlib>

#include "../../include/mustard_b200.h"
#include "tile_ops.cuh"

using namespace mtd;

namespace {

// Entry idx (column-major index with leading dimension n) of stream `seed`: a SplitMix64
// finaliser of seed * 0x9E3779B97F4A7C15 + (idx + 1) * 0xD1B54A32D192ED03, top 53 bits
// scaled to [0, 1), mapped to [-1, 1).  The test oracle computes the same bits.
__device__ __forceinline__ double uniform_pm1(uint64_t seed, uint64_t idx) {
    uint64_t z = seed * 0x9E3779B97F4A7C15ull + (idx + 1) * 0xD1B54A32D192ED03ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z ^= z >> 31;
    const double u = static_cast<double>(z >> 11) * (1.0 / 9007199254740992.0);
    return 2.0 * u - 1.0;
}

__global__ void uniform_kernel(double *a, int64_t n, int64_t lda, uint64_t seed, double diag_add) {
    const int64_t total = n * n;
    const int64_t stride = int64_t(gridDim.x) * blockDim.x;
    for (int64_t idx = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; idx < total; idx += stride) {
        const int64_t i = idx % n, j = idx / n;
        double v = uniform_pm1(seed, static_cast<uint64_t>(idx));
        if (i == j) v += diag_add;
        a[i + j * lda] = v;
    }
}

// C = B B^T / n + alpha I, one 128 x 128 output block per CTA (B: n x n, ld n).
__global__ void __launch_bounds__(kThreads, 1) spd_kernel(double *c, int64_t ldc, const double *b, int64_t n,
                                                          double alpha) {
    extern __shared__ __align__(128) double smem[];
    using M = GemmMma<kBNContig, 2>;
    const int r0 = blockIdx.x * kGemmTile, c0 = blockIdx.y * kGemmTile;
    const int mm = static_cast<int>(n - r0 < kGemmTile ? n - r0 : kGemmTile);
    const int nn = static_cast<int>(n - c0 < kGemmTile ? n - c0 : kGemmTile);
    M m;
    m.zero();
    m.run(smem, b + r0, n, b + c0, n, mm, nn, static_cast<int>(n));
    const double dn = static_cast<double>(n);
    m.for_each(mm, nn, [&](int r, int cc, double v) {
        double x = v / dn;
        if (r + r0 == cc + c0) x += alpha;
        c[(r + r0) + int64_t(cc + c0) * ldc] = x;
    });
}

__global__ void dmma_probe_kernel(double *out, int iters) {
    double acc[8][4];
    double a[4], b[2];
    for (int i = 0; i < 4; ++i) a[i] = 1e-3 * (threadIdx.x + i);
    for (int i = 0; i < 2; ++i) b[i] = 1e-3 * (threadIdx.x - i);
    for (int s = 0; s < 8; ++s)
        for (int v = 0; v < 4; ++v) acc[s][v] = 0.0;
    for (int it = 0; it < iters; ++it) {
#pragma unroll
        for (int s = 0; s < 8; ++s) dmma_16x8x8(acc[s], a, b);
    }
    double t = 0.0;
    for (int s = 0; s < 8; ++s)
        for (int v = 0; v < 4; ++v) t += acc[s][v];
    out[blockIdx.x * blockDim.x + threadIdx.x] = t;
}

}  // namespace

extern "C" {

int mtd_generate(double *dA, int64_t n, int64_t lda, int which, uint64_t seed, double alpha, void *stream) {
    if (!dA || n <= 0 || lda < n) return MTD_ERR_INVALID_ARG;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (which == MTD_GEN_UNIFORM_DIAG) {
        uniform_kernel<<<4096, 256, 0, s>>>(dA, n, lda, seed, static_cast<double>(n));
        return cudaGetLastError() == cudaSuccess ? MTD_OK : MTD_ERR_CUDA;
    }
    if (which != MTD_GEN_SPD) return MTD_ERR_INVALID_ARG;
    if (n % 2 != 0 || lda % 2 != 0 || reinterpret_cast<uintptr_t>(dA) % 16 != 0) return MTD_ERR_INVALID_ARG;
    double *b = nullptr;
    if (cudaMalloc(&b, size_t(n) * size_t(n) * sizeof(double)) != cudaSuccess) {
        cudaGetLastError();
        return MTD_ERR_OUT_OF_MEMORY;
    }
    uniform_kernel<<<4096, 256, 0, s>>>(b, n, n, seed, 0.0);
    constexpr int smem = GemmMma<kBNContig, 2>::SMEM_BYTES;
    cudaFuncSetAttribute(spd_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    const dim3 grid(static_cast<unsigned>((n + kGemmTile - 1) / kGemmTile),
                    static_cast<unsigned>((n + kGemmTile - 1) / kGemmTile));
    spd_kernel<<<grid, kThreads, smem, s>>>(dA, lda, b, n, alpha);
    int rc = cudaGetLastError() == cudaSuccess ? MTD_OK : MTD_ERR_CUDA;
    if (cudaStreamSynchronize(s) != cudaSuccess) rc = MTD_ERR_CUDA;
    cudaFree(b);
    return rc;
}

int mtd_generate_reference_host(double *hA, int64_t n) {
    // include/gen.h:23-38: srand(420); upper triangle (row-major) of rand()/RAND_MAX,
    // mirrored into the lower triangle; n added to the diagonal.
    if (!hA || n <= 0) return MTD_ERR_INVALID_ARG;
    const size_t N = static_cast<size_t>(n);
    srand(420);
    for (size_t r = 0; r < N; ++r)
        for (size_t c = r; c < N; ++c) hA[r * N + c] = static_cast<double>(rand()) / static_cast<double>(RAND_MAX);
    for (size_t r = 0; r < N; ++r)
        for (size_t c = 0; c < r; ++c) hA[r * N + c] = hA[c * N + r];
    for (size_t r = 0; r < N; ++r) hA[r * N + r] += static_cast<double>(n);
    return MTD_OK;
}

int mtd_probe_fp64_peak(double *tflops_out) {
    if (!tflops_out) return MTD_ERR_INVALID_ARG;
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return MTD_ERR_NO_DEVICE;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return MTD_ERR_NO_DEVICE;
    const int blocks = sms * 4, threads = 256, iters = 4000;
    double *out = nullptr;
    if (cudaMalloc(&out, sizeof(double) * blocks * threads) != cudaSuccess) return MTD_ERR_OUT_OF_MEMORY;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    dmma_probe_kernel<<<blocks, threads>>>(out, iters);  // warm-up
    cudaEventRecord(e0);
    dmma_probe_kernel<<<blocks, threads>>>(out, iters);
    cudaEventRecord(e1);
    int rc = cudaEventSynchronize(e1) == cudaSuccess ? MTD_OK : MTD_ERR_CUDA;
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    const double flops = 2.0 * 16 * 8 * 8 * 8.0 * iters * (double(blocks) * threads / 32.0);
    *tflops_out = rc == MTD_OK && ms > 0 ? flops / (ms * 1e-3) / 1e12 : 0.0;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(out);
    return rc;
}

}  // extern "C"
