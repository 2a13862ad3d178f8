// The launches of the batched factor-and-solve (mtd_batch_factor_solve) and of the pivoted
// LU (mtd_lupiv): the persistent kernel's instances that also run their own tasks
// (scheduler.cuh, SOLVE = true), in their own translation unit so the factorisation-only
// instances in runtime.cu stay as they are.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <mutex>

#include "../../include/mustard_b200.h"
#include "scheduler.cuh"

namespace mtd {

namespace {

template <int VEC, typename T, int SPLIT, int OPS = kOpsAll>
bool allow_smem(int bytes) {
    return cudaFuncSetAttribute(persistent_kernel<VEC, T, SPLIT, false, false, true, OPS>,
                                cudaFuncAttributeMaxDynamicSharedMemorySize, bytes) == cudaSuccess;
}

// Opt the instances into the tile operations' shared memory, once per device.
int solve_smem_setup(int device) {
    static std::atomic<bool> done[64];
    static std::mutex mu;
    if (device < 0 || device >= 64) return MTD_ERR_INVALID_ARG;
    if (done[device].load(std::memory_order_acquire)) return MTD_OK;
    std::lock_guard<std::mutex> lock(mu);
    if (!done[device].load(std::memory_order_relaxed)) {
        const int bytes = kOpSmemBytes();
        const bool ok = allow_smem<2, double, 1>(bytes) && allow_smem<1, double, 1>(bytes) &&
                        allow_smem<2, double, 1, kOpsCholesky>(bytes) && allow_smem<2, double, 1, kOpsLu>(bytes) &&
                        allow_smem<2, float, 1>(bytes) && allow_smem<1, float, 1>(bytes) &&
                        allow_smem<2, float, 3>(bytes) && allow_smem<1, float, 3>(bytes);
        if (!ok) return MTD_ERR_CUDA;
        done[device].store(true, std::memory_order_release);
    }
    return MTD_OK;
}

}  // namespace

// Dynamic shared memory of the persistent kernel (what a pivoted panel item may use).
int ext_op_smem_bytes() { return kOpSmemBytes(); }

// Reset the run's counters and queues, seed the roots, and launch the SOLVE instance for the
// batch's precision (prec) and operand alignment (vec2) on `grid` CTAs.
int launch_run_solve(const RunArgs &a, const int *deps_init, const int *roots, int n_roots, long long total_items,
                     int prec, bool vec2, int grid, cudaStream_t s) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return MTD_ERR_NO_DEVICE;
    const int rc = solve_smem_setup(dev);
    if (rc) return rc;
    const int reset_blocks = static_cast<int>(std::min<long long>(
        1024, std::max<long long>(1, (std::max<long long>(total_items, a.n_tasks) + kThreads - 1) / kThreads)));
    reset_kernel<<<reset_blocks, kThreads, 0, s>>>(a, deps_init);
    seed_kernel<<<1, kSeedThreads, 0, s>>>(a, roots, n_roots);
    const int bytes = kOpSmemBytes();
    if (prec == MTD_PREC_FP64) {
        // the batched factor-and-solve (Cholesky) and the pivoted LU run instances compiled with
        // their own operations only
        if (vec2 && a.opset == kOpsCholesky)
            persistent_kernel<2, double, 1, false, false, true, kOpsCholesky><<<grid, kThreads, bytes, s>>>(a);
        else if (vec2 && a.opset == kOpsLu)
            persistent_kernel<2, double, 1, false, false, true, kOpsLu><<<grid, kThreads, bytes, s>>>(a);
        else if (vec2) persistent_kernel<2, double, 1, false, false, true><<<grid, kThreads, bytes, s>>>(a);
        else persistent_kernel<1, double, 1, false, false, true><<<grid, kThreads, bytes, s>>>(a);
    } else if (prec == MTD_PREC_FP32) {
        if (vec2) persistent_kernel<2, float, 3, false, false, true><<<grid, kThreads, bytes, s>>>(a);
        else persistent_kernel<1, float, 3, false, false, true><<<grid, kThreads, bytes, s>>>(a);
    } else {
        if (vec2) persistent_kernel<2, float, 1, false, false, true><<<grid, kThreads, bytes, s>>>(a);
        else persistent_kernel<1, float, 1, false, false, true><<<grid, kThreads, bytes, s>>>(a);
    }
    return cudaGetLastError() == cudaSuccess ? MTD_OK : MTD_ERR_CUDA;
}

}  // namespace mtd
