// DMMA probe: where the FP64 engine's k-loop can lose against the register-only peak.
//   reg  : W warps per SM, ACC independent accumulators per warp, register operands only
//   lds  : the engine's fragment loads from padded shared memory every k8 step (no barrier)
//   lds + barrier : the same with a CTA barrier every 32-deep slice
// All accesses stay inside the staged slice; prints TFLOP/s per variant.
#include <cstdio>
#include <cuda_runtime.h>

__device__ __forceinline__ void dmma(double (&d)[4], const double (&a)[4], const double (&b)[2]) {
    asm volatile("mma.sync.aligned.m16n8k8.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};\n"
                 : "+d"(d[0]), "+d"(d[1]), "+d"(d[2]), "+d"(d[3])
                 : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(b[0]), "d"(b[1]));
}

template <int ACC>
__global__ void reg_kernel(double *out, int iters) {
    double acc[ACC][4];
    double a[4], b[2];
    for (int i = 0; i < 4; ++i) a[i] = 1e-3 * (threadIdx.x + i);
    for (int i = 0; i < 2; ++i) b[i] = 1e-3 * (threadIdx.x - i);
    for (int s = 0; s < ACC; ++s)
        for (int v = 0; v < 4; ++v) acc[s][v] = 0.0;
    for (int it = 0; it < iters; ++it) {
#pragma unroll
        for (int s = 0; s < ACC; ++s) dmma(acc[s], a, b);
    }
    double t = 0;
    for (int s = 0; s < ACC; ++s)
        for (int v = 0; v < 4; ++v) t += acc[s][v];
    out[blockIdx.x * blockDim.x + threadIdx.x] = t;
}

// engine shape: 16 warps as 4 x 4, warp tile 32 x 32 (FM=2, FN=4), A staged [k][m] LDA=132,
// B staged [k][n] LDB=132, BK=32 slice re-read every iteration (no global traffic)
template <int FM, int FN, int WARPS_M, int WARPS_N, bool BAR>
__global__ void lds_kernel(double *out, int iters) {
    extern __shared__ double sm[];
    constexpr int BM = FM * 16 * WARPS_M, BN = FN * 8 * WARPS_N, BK = 32, LDA = BM + 4, LDB = BN + 4;
    double *As = sm, *Bs = sm + BK * LDA;
    for (int i = threadIdx.x; i < BK * (LDA + LDB); i += blockDim.x) sm[i] = 1e-3 * (i % 97);
    __syncthreads();
    double acc[FM][FN][4];
    for (int i = 0; i < FM; ++i)
        for (int j = 0; j < FN; ++j)
            for (int v = 0; v < 4; ++v) acc[i][j][v] = 0.0;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int wm0 = (warp / WARPS_N) * FM * 16, wn0 = (warp % WARPS_N) * FN * 8;
    const int g = lane >> 2, t = lane & 3;
    for (int it = 0; it < iters; ++it) {
#pragma unroll
        for (int ks = 0; ks < BK; ks += 8) {
            double bf[FN][2];
#pragma unroll
            for (int j = 0; j < FN; ++j) {
                const int n = wn0 + j * 8 + g;
                bf[j][0] = Bs[(ks + t) * LDB + n];
                bf[j][1] = Bs[(ks + t + 4) * LDB + n];
            }
#pragma unroll
            for (int i = 0; i < FM; ++i) {
                const int m = wm0 + i * 16 + g;
                double af[4];
                af[0] = As[(ks + t) * LDA + m];
                af[1] = As[(ks + t) * LDA + m + 8];
                af[2] = As[(ks + t + 4) * LDA + m];
                af[3] = As[(ks + t + 4) * LDA + m + 8];
#pragma unroll
                for (int j = 0; j < FN; ++j) dmma(acc[i][j], af, bf[j]);
            }
        }
        if (BAR) __syncthreads();
    }
    double s = 0;
    for (int i = 0; i < FM; ++i)
        for (int j = 0; j < FN; ++j)
            for (int v = 0; v < 4; ++v) s += acc[i][j][v];
    out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

template <typename K>
float time_kernel(K kern, int blocks, int threads, int smem, double *out, int iters) {
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    kern<<<blocks, threads, smem>>>(out, iters);
    cudaEventRecord(e0);
    kern<<<blocks, threads, smem>>>(out, iters);
    cudaEventRecord(e1);
    cudaEventSynchronize(e1);
    float ms;
    cudaEventElapsedTime(&ms, e0, e1);
    return ms;
}

int main() {
    int sms;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, 0);
    double *out;
    cudaMalloc(&out, sizeof(double) * sms * 4 * 1024);
    const double mma_flops = 2.0 * 16 * 8 * 8;
    auto report = [&](const char *name, float ms, double mmas_per_warp_iter, int warps_total, int iters) {
        const double fl = mma_flops * mmas_per_warp_iter * iters * warps_total;
        printf("%-40s %8.3f ms  %6.2f TFLOP/s\n", name, ms, fl / (ms * 1e-3) / 1e12);
    };
    const int it = 4000;
    // register-only: warps per SM = blocks/SM * threads/32
    report("reg 8 acc, 32 warps/SM (4 blk x 256)", time_kernel(reg_kernel<8>, sms * 4, 256, 0, out, it), 8, sms * 32, it);
    report("reg 8 acc, 16 warps/SM (1 blk x 512)", time_kernel(reg_kernel<8>, sms, 512, 0, out, it), 8, sms * 16, it);
    report("reg 16 acc, 8 warps/SM", time_kernel(reg_kernel<16>, sms, 256, 0, out, it), 16, sms * 8, it);
    report("reg 16 acc, 4 warps/SM", time_kernel(reg_kernel<16>, sms, 128, 0, out, it), 16, sms * 4, it);
    report("reg 8 acc, 8 warps/SM", time_kernel(reg_kernel<8>, sms, 256, 0, out, it), 8, sms * 8, it);
    report("reg 4 acc, 16 warps/SM", time_kernel(reg_kernel<4>, sms, 512, 0, out, it * 2), 4, sms * 16, it * 2);
    const int li = 2000;
    {
        constexpr int smem = 32 * (132 + 132) * 8;
        auto k = lds_kernel<2, 4, 4, 4, false>;
        cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        report("lds 16w 32x32 (engine) no barrier", time_kernel(k, sms, 512, smem, out, li), 32, sms * 16, li);
        auto kb = lds_kernel<2, 4, 4, 4, true>;
        cudaFuncSetAttribute(kb, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        report("lds 16w 32x32 (engine) barrier/slice", time_kernel(kb, sms, 512, smem, out, li), 32, sms * 16, li);
    }
    {
        constexpr int smem = 32 * (132 + 132) * 8;
        auto k = lds_kernel<4, 4, 2, 4, false>;  // 8 warps, warp tile 64 x 32
        cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        report("lds 8w 64x32 no barrier", time_kernel(k, sms, 256, smem, out, li), 64, sms * 8, li);
        auto kb = lds_kernel<4, 4, 2, 4, true>;
        cudaFuncSetAttribute(kb, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        report("lds 8w 64x32 barrier/slice", time_kernel(kb, sms, 256, smem, out, li), 64, sms * 8, li);
    }
    cudaError_t e = cudaGetLastError();
    printf("status: %s\n", cudaGetErrorString(e));
    return e == cudaSuccess ? 0 : 1;
}
