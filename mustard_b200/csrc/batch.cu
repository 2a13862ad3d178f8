// Batched factorisations and solves: many independent SPD matrices of different sizes
// run as ONE merged task graph on the persistent scheduler (one launch: graph-capturable),
// then solved with per-matrix triangular solves, in FP64 or in low precision with FP64
// iterative refinement.  No counterpart in the reference.
//
// Each matrix gets the reference's tiled Cholesky DAG for its own tile edge (chosen per
// size by the caller or by mtd_batch_autotune), lowered with nested diagonal
// factorisations, and the DAGs are concatenated with every task tagged by its matrix.  A
// bad pivot records LAPACK-style info for that matrix only; the rest of the batch runs on.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <map>
#include <new>
#include <vector>

#include "../../include/mustard_b200.h"
#include "batch_ops.cuh"
#include "dag.hpp"
#include "device_types.hpp"

namespace mtd {
int launch_run(const RunArgs &a, const int *deps_init, const int *roots, int n_roots, long long total_items,
               int prec, bool vec2, int grid, cudaStream_t s, bool adjoint);
int launch_run_solve(const RunArgs &a, const int *deps_init, const int *roots, int n_roots, long long total_items,
                     int prec, bool vec2, int grid, cudaStream_t s);
}
using namespace mtd;

namespace {

constexpr int kSB = bsolve::kSB;
constexpr int kMaxRhs = bsolve::kMaxRhs;
constexpr int kBT = 256;       // threads of the standalone batched solve kernels
constexpr int kInfoOk = 0x7f7f7f7f;  // per-matrix info sentinel (bytes 0x7f): no bad pivot
using bsolve::kOnD;
using bsolve::kOnR;
using bsolve::kOnX;

// The standalone solve kernels, one CTA per matrix (batch_ops.cuh holds their bodies, which
// the solve tasks of the factor-and-solve launch share).  A refinement step skips the
// matrices that have converged (`done`: berr[m] <= tol), as a solve task stops refining its
// own matrix, so both paths apply the same steps to every matrix.
struct Skip {
    const double *berr;  // nullptr: skip nothing
    double tol;
    __device__ bool operator()() const { return berr && berr[blockIdx.x] <= tol; }
};

// (2 CTAs per SM: the FP64 blocks fill the shared memory; more float CTAs would spill)
template <typename T>
__global__ void __launch_bounds__(kBT, 2) batch_trsv_kernel(const SolveMat *mats, const T *ws, int target, Skip done) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    if (done()) return;
    bsolve::trsv<T, kBT>(bsolve::Grp{int(threadIdx.x), 0}, mats[blockIdx.x], ws, target, bsolve::Smem{smem_raw});
}

// r = b - A_sym x and the matrix's backward error into berr[m]; the first call of a solve
// (want_anorm) also computes ||A_sym||_inf into anorm[m], which later calls read.
__global__ void __launch_bounds__(kBT, 2) batch_residual_kernel(const SolveMat *mats, double *anorm, double *berr,
                                                                int want_anorm, Skip done) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    if (done()) return;  // converged before the last step: x and berr[m] stand
    const double be = bsolve::residual<kBT>(bsolve::Grp{int(threadIdx.x), 0}, mats[blockIdx.x], anorm + blockIdx.x,
                                            want_anorm != 0, bsolve::Smem{smem_raw});
    if (threadIdx.x == 0) berr[blockIdx.x] = be;
}

// r = b and its backward error, for x = 0 (the first step of a low-precision solve).
__global__ void __launch_bounds__(kBT) batch_residual_zero_kernel(const SolveMat *mats, double *berr) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const double be = bsolve::residual_of_zero<kBT>(bsolve::Grp{int(threadIdx.x), 0}, mats[blockIdx.x],
                                                    bsolve::Smem{smem_raw});
    if (threadIdx.x == 0) berr[blockIdx.x] = be;
}

// d = r / max|r| per column (rounded to T), or x += max|r| * d.
template <typename T>
__global__ void __launch_bounds__(kBT) batch_scale_kernel(const SolveMat *mats, double *colscale, bool to_low, Skip done) {
    __shared__ double red[kBT / 32];
    if (done()) return;
    double *scale = colscale + int64_t(blockIdx.x) * kMaxRhs;
    if (to_low)
        bsolve::scale_to_low<T, kBT>(bsolve::Grp{int(threadIdx.x), 0}, mats[blockIdx.x], scale, red);
    else
        bsolve::add_scaled<T, kBT>(bsolve::Grp{int(threadIdx.x), 0}, mats[blockIdx.x], scale);
}

// x += r (FP64 correction).
__global__ void __launch_bounds__(kBT) batch_add_kernel(const SolveMat *mats, Skip done) {
    if (!done()) bsolve::add_r<kBT>(bsolve::Grp{int(threadIdx.x), 0}, mats[blockIdx.x]);
}

// X = B (columns), or X = 0.
__global__ void __launch_bounds__(kBT) batch_copy_rhs_kernel(const SolveMat *mats, bool zero) {
    bsolve::copy_rhs<kBT>(bsolve::Grp{int(threadIdx.x), 0}, mats[blockIdx.x], zero);
}

// F = lower triangle of A (+ shift on the diagonal), as float; grid (column strips, count).
__global__ void __launch_bounds__(kBT) batch_convert_kernel(const SolveMat *mats, double shift) {
    const SolveMat &sm = mats[blockIdx.y];
    for (int c0 = blockIdx.x * kConvertCols; c0 < sm.n; c0 += gridDim.x * kConvertCols)
        bsolve::convert<float, kBT>(bsolve::Grp{int(threadIdx.x), 0}, sm.a, sm.lda,
                                    static_cast<float *>(const_cast<void *>(sm.f)), sm.ldf, sm.n, shift, c0,
                                    min(sm.n, c0 + kConvertCols));
}

template <typename T>
int dalloc(T **p, size_t count) {
    if (cudaMalloc(reinterpret_cast<void **>(p), std::max<size_t>(count, 1) * sizeof(T)) != cudaSuccess) {
        cudaGetLastError();
        *p = nullptr;
        return MTD_ERR_OUT_OF_MEMORY;
    }
    return MTD_OK;
}

}  // namespace

struct mtd_batch {
    int count = 0;
    int prec = MTD_PREC_FP64;
    int sms = 148;
    std::vector<int64_t> n, tile, ws_off, ws_ld, rhs_off;
    std::vector<int> nest;
    int n_dev = 0, n_roots = 0;
    long long total_items = 0;
    long long qcap[kNumQueues] = {0, 0};
    DevTask *d_tasks = nullptr;
    int *d_succ = nullptr, *d_deps_init = nullptr, *d_deps = nullptr, *d_items_left = nullptr, *d_roots = nullptr;
    unsigned long long *d_queue[kNumQueues] = {nullptr, nullptr};
    QueueCtl *d_qctl = nullptr;
    RunCtl *d_ctl = nullptr;
    RunCtl *h_ctl = nullptr;       // pinned
    unsigned char *d_ws = nullptr;
    BatchMat *d_mats = nullptr;
    BatchMat *h_mats = nullptr;    // pinned staging of the per-run table
    int *d_info = nullptr;
    unsigned long long *d_done = nullptr;
    cudaStream_t last_stream = nullptr;
    bool pending = false;
    // solve state
    SolveMat *d_solve = nullptr, *h_solve = nullptr;  // pinned staging
    double *d_r = nullptr, *d_anorm = nullptr, *d_berr = nullptr, *d_scale = nullptr;
    double *h_berr = nullptr;      // pinned
    void *d_low = nullptr;
    int64_t rhs_total = 0;
    // the merged factor DAG on the host (the factor-and-solve tables extend it), each matrix's
    // roots and task range, and the CTA-to-task schedule (MTD_BATCH_ORDER_* | SOLVE_LATE)
    std::vector<DevTask> h_tasks;
    std::vector<int> h_succ, h_deps_init, first_task;
    std::vector<std::vector<int>> roots_of;
    int schedule = MTD_BATCH_ORDER_INPUT;
    int last_tasks = 0;            // tasks of the last launch (factor or factor-and-solve)
    // factor-and-solve launch: its tables (built at first use for the current schedule) and
    // its per-matrix outcomes
    int fs_convert = -1;           // the tables hold conversion tasks (1) or not (0); -1: not built
    int fs_tasks = 0, fs_roots = 0;
    long long fs_qcap[kNumQueues] = {0, 0, 0};
    DevTask *d_fs_tasks = nullptr;
    int *d_fs_succ = nullptr, *d_fs_deps_init = nullptr, *d_fs_deps = nullptr, *d_fs_items_left = nullptr,
        *d_fs_roots = nullptr;
    unsigned long long *d_fs_queue[kNumQueues] = {nullptr, nullptr, nullptr};
    double *d_fs_berr = nullptr;
    int *d_fs_iters = nullptr;
    double fs_tol = 0.0;
    bool fs_pending = false;
};

namespace {

size_t batch_elem(const mtd_batch *b) { return b->prec == MTD_PREC_FP64 ? sizeof(double) : sizeof(float); }

void release(mtd_batch *b) {
    cudaFree(b->d_tasks);
    cudaFree(b->d_succ);
    cudaFree(b->d_deps_init);
    cudaFree(b->d_deps);
    cudaFree(b->d_items_left);
    cudaFree(b->d_roots);
    for (int q = 0; q < kNumQueues; ++q) cudaFree(b->d_queue[q]);
    cudaFree(b->d_qctl);
    cudaFree(b->d_ctl);
    if (b->h_ctl) cudaFreeHost(b->h_ctl);
    cudaFree(b->d_ws);
    cudaFree(b->d_mats);
    if (b->h_mats) cudaFreeHost(b->h_mats);
    cudaFree(b->d_info);
    cudaFree(b->d_done);
    cudaFree(b->d_solve);
    if (b->h_solve) cudaFreeHost(b->h_solve);
    cudaFree(b->d_r);
    cudaFree(b->d_anorm);
    cudaFree(b->d_berr);
    cudaFree(b->d_scale);
    if (b->h_berr) cudaFreeHost(b->h_berr);
    cudaFree(b->d_low);
    cudaFree(b->d_fs_berr);
    cudaFree(b->d_fs_iters);
}

// The factor-and-solve tables (rebuilt when the schedule changes).
void release_fs(mtd_batch *b) {
    cudaFree(b->d_fs_tasks);
    cudaFree(b->d_fs_succ);
    cudaFree(b->d_fs_deps_init);
    cudaFree(b->d_fs_deps);
    cudaFree(b->d_fs_items_left);
    cudaFree(b->d_fs_roots);
    for (int q = 0; q < kNumQueues; ++q) cudaFree(b->d_fs_queue[q]);
    b->d_fs_tasks = nullptr;
    b->d_fs_succ = b->d_fs_deps_init = b->d_fs_deps = b->d_fs_items_left = b->d_fs_roots = nullptr;
    for (int q = 0; q < kNumQueues; ++q) b->d_fs_queue[q] = nullptr;
    b->fs_convert = -1;
}

// The matrices in the order their first tasks enter the queues under the batch's schedule.
std::vector<int> schedule_order(const mtd_batch *b) {
    std::vector<int> order(b->count);
    for (int m = 0; m < b->count; ++m) order[m] = m;
    const int o = b->schedule & 3;
    if (o == MTD_BATCH_ORDER_LARGEST_FIRST)
        std::stable_sort(order.begin(), order.end(), [b](int x, int y) { return b->n[x] > b->n[y]; });
    else if (o == MTD_BATCH_ORDER_SMALLEST_FIRST)
        std::stable_sort(order.begin(), order.end(), [b](int x, int y) { return b->n[x] < b->n[y]; });
    return order;
}

// The factor launch's root list in schedule order.
std::vector<int> scheduled_roots(const mtd_batch *b) {
    std::vector<int> roots;
    for (int m : schedule_order(b))
        for (int r : b->roots_of[m]) roots.push_back(r);
    return roots;
}

// The factor-and-solve task graph: the merged factor DAG, a solve task per matrix after its
// sinks (queue 0, or queue 2 with MTD_BATCH_SOLVE_LATE) and, with `convert`, a conversion
// task per matrix (queue 0) before its roots, which become the launch's roots in schedule
// order.  Uploaded into the batch's fs tables.
int build_fs(mtd_batch *b, bool convert) {
    release_fs(b);
    const int count = b->count;
    std::vector<DevTask> t = b->h_tasks;
    std::vector<int> succ = b->h_succ, deps = b->h_deps_init, roots;
    const int solve_queue = (b->schedule & MTD_BATCH_SOLVE_LATE) ? kNumQueues - 1 : 0;
    const bool pairs = (b->schedule & MTD_BATCH_SOLVE_PAIRS) != 0;
    const std::vector<int> order = schedule_order(b);
    // solve tasks: one per matrix, or one per two matrices adjacent in the schedule order
    std::vector<int> solve_of(count);
    for (size_t q = 0; q < order.size(); q += pairs ? 2 : 1) {
        DevTask s{};
        s.op = kOpBatchSolve;
        s.queue = solve_queue;
        s.n_items = 1;
        s.mat = order[q];
        s.pad = (pairs && q + 1 < order.size()) ? order[q + 1] : -1;
        s.m = s.n = static_cast<int32_t>(b->n[s.mat]);
        const int idx = static_cast<int>(t.size());
        t.push_back(s);
        solve_of[s.mat] = idx;
        if (s.pad >= 0) solve_of[s.pad] = idx;
    }
    deps.resize(t.size(), 0);
    for (int m = 0; m < count; ++m) {
        for (int i = b->first_task[m]; i < b->first_task[m + 1]; ++i)
            if (t[i].succ_count == 0) {  // a sink of matrix m: its solve follows it
                t[i].succ_begin = static_cast<int32_t>(succ.size());
                t[i].succ_count = 1;
                succ.push_back(solve_of[m]);
                ++deps[solve_of[m]];
            }
    }
    const int first_convert = static_cast<int>(t.size());
    if (convert) {
        t.resize(first_convert + count);
        deps.resize(t.size(), 0);
    }
    for (int m : order) {
        if (!convert) {
            for (int r : b->roots_of[m]) roots.push_back(r);
            continue;
        }
        const int c = first_convert + m;
        DevTask d{};
        d.op = kOpBatchConvert;
        d.queue = 0;
        d.n_items = static_cast<int32_t>((b->n[m] + kConvertCols - 1) / kConvertCols);
        d.m = d.n = static_cast<int32_t>(b->n[m]);
        d.mat = m;
        d.succ_begin = static_cast<int32_t>(succ.size());
        d.succ_count = static_cast<int32_t>(b->roots_of[m].size());
        for (int r : b->roots_of[m]) {
            succ.push_back(r);
            deps[r] = 1;
        }
        t[c] = d;
        roots.push_back(c);
    }
    long long qcap[kNumQueues] = {0, 0, 0};
    for (const DevTask &d : t) qcap[d.queue] += d.n_items;
    int rc = dalloc(&b->d_fs_tasks, t.size());
    if (!rc) rc = dalloc(&b->d_fs_succ, succ.size());
    if (!rc) rc = dalloc(&b->d_fs_deps_init, t.size());
    if (!rc) rc = dalloc(&b->d_fs_deps, t.size());
    if (!rc) rc = dalloc(&b->d_fs_items_left, t.size());
    if (!rc) rc = dalloc(&b->d_fs_roots, roots.size());
    for (int q = 0; q < kNumQueues && !rc; ++q) rc = dalloc(&b->d_fs_queue[q], size_t(qcap[q]));
    if (!rc && (cudaMemcpy(b->d_fs_tasks, t.data(), t.size() * sizeof(DevTask), cudaMemcpyHostToDevice) != cudaSuccess ||
                cudaMemcpy(b->d_fs_succ, succ.data(), succ.size() * sizeof(int), cudaMemcpyHostToDevice) != cudaSuccess ||
                cudaMemcpy(b->d_fs_deps_init, deps.data(), deps.size() * sizeof(int), cudaMemcpyHostToDevice) !=
                    cudaSuccess ||
                cudaMemcpy(b->d_fs_roots, roots.data(), roots.size() * sizeof(int), cudaMemcpyHostToDevice) !=
                    cudaSuccess))
        rc = MTD_ERR_CUDA;
    if (rc) {
        release_fs(b);
        return rc;
    }
    b->fs_tasks = static_cast<int>(t.size());
    b->fs_roots = static_cast<int>(roots.size());
    for (int q = 0; q < kNumQueues; ++q) b->fs_qcap[q] = qcap[q];
    b->fs_convert = convert ? 1 : 0;
    return MTD_OK;
}

// Pinned staging, device table and scratch of the batched solves (allocated at first use).
int ensure_solve_buffers(mtd_batch *b) {
    const int count = b->count;
    if (!b->h_solve && cudaMallocHost(reinterpret_cast<void **>(&b->h_solve), count * sizeof(SolveMat)) != cudaSuccess)
        return MTD_ERR_OUT_OF_MEMORY;
    if (!b->h_berr && cudaMallocHost(reinterpret_cast<void **>(&b->h_berr), count * sizeof(double)) != cudaSuccess)
        return MTD_ERR_OUT_OF_MEMORY;
    int rc = MTD_OK;
    if (!b->d_solve) rc = dalloc(&b->d_solve, count);
    if (!rc && !b->d_r) rc = dalloc(&b->d_r, size_t(b->rhs_total));
    if (!rc && !b->d_anorm) rc = dalloc(&b->d_anorm, count);
    if (!rc && !b->d_berr) rc = dalloc(&b->d_berr, count);
    if (!rc && !b->d_scale) rc = dalloc(&b->d_scale, size_t(count) * kMaxRhs);
    if (!rc && !b->d_low && cudaMalloc(&b->d_low, size_t(b->rhs_total) * sizeof(float)) != cudaSuccess)
        rc = MTD_ERR_OUT_OF_MEMORY;
    if (!rc && !b->d_fs_berr) rc = dalloc(&b->d_fs_berr, count);
    if (!rc && !b->d_fs_iters) rc = dalloc(&b->d_fs_iters, count);
    return rc;
}

// Validate a solve's arguments and stage its per-matrix table (SolveMat) in pinned memory.
int stage_solve(mtd_batch *b, const double *const *dA, const int64_t *lda, void *const *dF, const int64_t *ldf,
                const double *const *dB, const int64_t *ldb, double *const *dX, const int64_t *ldx, const int *nrhs) {
    for (int m = 0; m < b->count; ++m) {
        if (!dF[m] || !dB[m] || !dX[m] || nrhs[m] < 1 || nrhs[m] > kMaxRhs || ldb[m] < b->n[m] ||
            ldx[m] < b->n[m] || ldf[m] < b->n[m])
            return MTD_ERR_INVALID_ARG;
        if (dA && (!dA[m] || lda[m] < b->n[m])) return MTD_ERR_INVALID_ARG;
        SolveMat &sm = b->h_solve[m];
        sm.a = dA ? dA[m] : nullptr;
        sm.lda = dA ? lda[m] : 0;
        sm.f = dF[m];
        sm.ldf = ldf[m];
        sm.ws_off = b->ws_off[m];
        sm.ws_ld = b->ws_ld[m];
        sm.b = dB[m];
        sm.ldb = ldb[m];
        sm.x = dX[m];
        sm.ldx = ldx[m];
        sm.r = b->d_r + b->rhs_off[m];
        sm.d = static_cast<float *>(b->d_low) + b->rhs_off[m];
        sm.n = static_cast<int>(b->n[m]);
        sm.nrhs = nrhs[m];
    }
    return MTD_OK;
}

// Stage the per-run matrix table (dA[m] factored in place) and reset the per-matrix info
// and completion stamps, on stream s; *vec2: every matrix allows 16-byte operand loads.
int stage_factor(mtd_batch *b, void *const *dA, const int64_t *lda, cudaStream_t s, bool *vec2) {
    const int64_t epc = 16 / static_cast<int64_t>(batch_elem(b));
    *vec2 = true;
    for (int m = 0; m < b->count; ++m) {
        if (!dA[m] || lda[m] < b->n[m]) return MTD_ERR_INVALID_ARG;
        b->h_mats[m] = BatchMat{dA[m], lda[m], b->ws_off[m], b->ws_ld[m]};
        *vec2 = *vec2 && reinterpret_cast<uintptr_t>(dA[m]) % 16 == 0 && lda[m] % epc == 0 && b->n[m] % epc == 0 &&
                b->tile[m] % epc == 0;
    }
    if (cudaMemcpyAsync(b->d_mats, b->h_mats, b->count * sizeof(BatchMat), cudaMemcpyHostToDevice, s) != cudaSuccess ||
        cudaMemsetAsync(b->d_info, 0x7f, b->count * sizeof(int), s) != cudaSuccess ||
        cudaMemsetAsync(b->d_done, 0, b->count * sizeof(unsigned long long), s) != cudaSuccess)
        return MTD_ERR_CUDA;
    return MTD_OK;
}

// The run arguments every batched launch shares (the task tables are the caller's).
RunArgs batch_args(const mtd_batch *b) {
    RunArgs a{};
    a.opset = kOpsCholesky;  // every matrix's graph is a tiled Cholesky (+ its solve tasks)
    a.qctl = b->d_qctl;
    a.ctl = b->d_ctl;
    a.ws_lower = b->d_ws;
    a.ws_upper = nullptr;
    a.timeout_ns = 10ull * 1000000000ull;
    a.mats = b->d_mats;
    a.mat_info = b->d_info;
    a.mat_done_ns = b->d_done;
    return a;
}

// Default tile for a size when the caller gives none: one tile up to 512 (its diagonal
// factorisation nested at 128), 512-wide tiles above.
int64_t default_tile(int64_t n) { return n <= 512 ? n : 512; }

}  // namespace

extern "C" {

int mtd_batch_create(mtd_batch **out, int count, const int64_t *n, const int64_t *tile, const int *nest, int prec) {
    if (!out) return MTD_ERR_INVALID_ARG;
    *out = nullptr;
    if (count <= 0 || !n || (prec != MTD_PREC_FP64 && prec != MTD_PREC_TF32 && prec != MTD_PREC_FP32))
        return MTD_ERR_INVALID_ARG;
    mtd_batch *b = new (std::nothrow) mtd_batch();
    if (!b) return MTD_ERR_OUT_OF_MEMORY;
    b->count = count;
    b->prec = prec;
    int dev = 0;
    cudaGetDevice(&dev);
    int major = 0;
    cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev);
    if (major != 10) {
        delete b;
        return MTD_ERR_NO_DEVICE;
    }
    cudaDeviceGetAttribute(&b->sms, cudaDevAttrMultiProcessorCount, dev);

    std::vector<DevTask> tasks;
    std::vector<int> succ, deps_init, roots;
    int64_t ws_total = 0, rhs_total = 0;
    int rc = MTD_OK;
    for (int m = 0; m < count && !rc; ++m) {
        const int64_t nm = n[m];
        const int64_t tm = tile ? tile[m] : default_tile(nm);
        const int km = nest ? nest[m] : (nm > kNestTile ? kNestTile : 0);
        if (nm <= 0 || nm > (int64_t(1) << 20) || tm <= 0 || tm > nm || (tm != nm && tm % kSB != 0) || km < 0 ||
            km % kSB != 0) {
            rc = MTD_ERR_INVALID_ARG;
            break;
        }
        b->n.push_back(nm);
        b->tile.push_back(tm);
        b->nest.push_back(km);
        Dag dag(MTD_KIND_CHOLESKY, nm, tm);
        rc = dag.build_reference_order();
        Lowered low;
        if (!rc) rc = dag.lower(km, low);
        if (rc) break;
        const int base = static_cast<int>(tasks.size());
        const int sbase = static_cast<int>(succ.size());
        b->first_task.push_back(base);
        b->roots_of.emplace_back();
        for (size_t t = 0; t < low.tasks.size(); ++t) {
            DevTask d = low.tasks[t];
            d.mat = m;
            d.succ_begin += sbase;
            tasks.push_back(d);
            deps_init.push_back(static_cast<int>(low.preds[t].size()));
            if (low.preds[t].empty()) {
                roots.push_back(base + static_cast<int>(t));
                b->roots_of.back().push_back(base + static_cast<int>(t));
            }
        }
        for (int s : low.succ) succ.push_back(s + base);
        for (int q = 0; q < kNumQueues; ++q) b->qcap[q] += low.queue_cap[q];
        const int64_t wld = (nm + 3) & ~int64_t(3);
        b->ws_off.push_back(ws_total);
        b->ws_ld.push_back(wld);
        ws_total += wld * kSB;
        b->rhs_off.push_back(rhs_total);
        rhs_total += nm * kMaxRhs;
    }
    if (!rc && roots.empty()) rc = MTD_ERR_BAD_DAG;
    b->n_dev = static_cast<int>(tasks.size());
    b->n_roots = static_cast<int>(roots.size());
    b->total_items = 0;
    for (int q = 0; q < kNumQueues; ++q) b->total_items += b->qcap[q];
    b->rhs_total = rhs_total;
    const int nt = b->n_dev;
    if (!rc) rc = dalloc(&b->d_tasks, nt);
    if (!rc) rc = dalloc(&b->d_succ, succ.size());
    if (!rc) rc = dalloc(&b->d_deps_init, nt);
    if (!rc) rc = dalloc(&b->d_deps, nt);
    if (!rc) rc = dalloc(&b->d_items_left, nt);
    if (!rc) rc = dalloc(&b->d_roots, roots.size());
    for (int q = 0; q < kNumQueues && !rc; ++q) rc = dalloc(&b->d_queue[q], size_t(b->qcap[q]));
    if (!rc) rc = dalloc(&b->d_qctl, kNumQueues);
    if (!rc) rc = dalloc(&b->d_ctl, 1);
    if (!rc) rc = dalloc(&b->d_ws, size_t(ws_total) * batch_elem(b));
    if (!rc) rc = dalloc(&b->d_mats, count);
    if (!rc) rc = dalloc(&b->d_info, count);
    if (!rc) rc = dalloc(&b->d_done, count);
    if (!rc && cudaMallocHost(reinterpret_cast<void **>(&b->h_ctl), sizeof(RunCtl)) != cudaSuccess) rc = MTD_ERR_OUT_OF_MEMORY;
    if (!rc && cudaMallocHost(reinterpret_cast<void **>(&b->h_mats), count * sizeof(BatchMat)) != cudaSuccess)
        rc = MTD_ERR_OUT_OF_MEMORY;
    if (!rc) {
        bool ok = cudaMemcpy(b->d_tasks, tasks.data(), nt * sizeof(DevTask), cudaMemcpyHostToDevice) == cudaSuccess;
        ok = ok && (succ.empty() ||
                    cudaMemcpy(b->d_succ, succ.data(), succ.size() * sizeof(int), cudaMemcpyHostToDevice) == cudaSuccess);
        ok = ok && cudaMemcpy(b->d_deps_init, deps_init.data(), nt * sizeof(int), cudaMemcpyHostToDevice) == cudaSuccess;
        ok = ok && cudaMemcpy(b->d_roots, roots.data(), roots.size() * sizeof(int), cudaMemcpyHostToDevice) == cudaSuccess;
        ok = ok && cudaMemset(b->d_ctl, 0, sizeof(RunCtl)) == cudaSuccess;
        if (!ok) rc = MTD_ERR_CUDA;
    }
    if (rc) {
        release(b);
        delete b;
        return rc;
    }
    std::memset(b->h_ctl, 0, sizeof(RunCtl));
    b->first_task.push_back(b->n_dev);
    b->h_tasks = std::move(tasks);
    b->h_succ = std::move(succ);
    b->h_deps_init = std::move(deps_init);
    *out = b;
    return MTD_OK;
}

int mtd_batch_num_tasks(const mtd_batch *b) { return b ? b->n_dev : -MTD_ERR_INVALID_ARG; }

int mtd_batch_set_schedule(mtd_batch *b, int schedule) {
    if (!b || schedule < 0 || (schedule & ~(3 | MTD_BATCH_SOLVE_LATE | MTD_BATCH_SOLVE_PAIRS)) ||
        (schedule & 3) > MTD_BATCH_ORDER_SMALLEST_FIRST)
        return MTD_ERR_INVALID_ARG;
    if (schedule == b->schedule) return MTD_OK;
    if ((b->pending || b->fs_pending) && b->last_stream && cudaStreamSynchronize(b->last_stream) != cudaSuccess)
        return MTD_ERR_CUDA;
    b->schedule = schedule;
    const std::vector<int> roots = scheduled_roots(b);
    if (cudaMemcpy(b->d_roots, roots.data(), roots.size() * sizeof(int), cudaMemcpyHostToDevice) != cudaSuccess)
        return MTD_ERR_CUDA;
    // factor-and-solve tables already built are rebuilt now, so the next launch allocates
    // nothing (it may be under CUDA-graph capture)
    return b->fs_convert >= 0 ? build_fs(b, b->fs_convert == 1) : MTD_OK;
}

int mtd_batch_get_schedule(const mtd_batch *b) { return b ? b->schedule : -MTD_ERR_INVALID_ARG; }

int mtd_batch_factor(mtd_batch *b, void *const *dA, const int64_t *lda, void *stream) {
    if (!b || !dA || !lda) return MTD_ERR_INVALID_ARG;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    bool vec2 = true;
    int rc = stage_factor(b, dA, lda, s, &vec2);
    if (rc) return rc;
    RunArgs a = batch_args(b);
    a.n_tasks = b->n_dev;
    a.tasks = b->d_tasks;
    a.succ = b->d_succ;
    a.deps = b->d_deps;
    a.items_left = b->d_items_left;
    for (int q = 0; q < kNumQueues; ++q) {
        a.queue[q] = b->d_queue[q];
        a.queue_cap[q] = b->qcap[q];
    }
    rc = launch_run(a, b->d_deps_init, b->d_roots, b->n_roots, b->total_items, b->prec, vec2, b->sms, s, false);
    if (rc) return rc;
    if (cudaMemcpyAsync(b->h_ctl, b->d_ctl, sizeof(RunCtl), cudaMemcpyDeviceToHost, s) != cudaSuccess) return MTD_ERR_CUDA;
    b->last_stream = s;
    b->last_tasks = b->n_dev;
    b->pending = true;
    b->fs_pending = false;
    return MTD_OK;
}

int mtd_batch_status(mtd_batch *b, int *info, double *latency_ms) {
    if (!b) return MTD_ERR_INVALID_ARG;
    if (!b->pending) return MTD_ERR_STATE;
    if (cudaStreamSynchronize(b->last_stream) != cudaSuccess) return MTD_ERR_CUDA;
    if (info) {
        if (cudaMemcpy(info, b->d_info, b->count * sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess) return MTD_ERR_CUDA;
        for (int m = 0; m < b->count; ++m)
            if (info[m] == kInfoOk) info[m] = 0;
    }
    if (latency_ms) {
        std::vector<unsigned long long> done(b->count);
        if (cudaMemcpy(done.data(), b->d_done, b->count * sizeof(unsigned long long), cudaMemcpyDeviceToHost) !=
            cudaSuccess)
            return MTD_ERR_CUDA;
        for (int m = 0; m < b->count; ++m)
            latency_ms[m] = done[m] > b->h_ctl->start_ns ? double(done[m] - b->h_ctl->start_ns) * 1e-6 : -1.0;
    }
    if (b->h_ctl->error) return b->h_ctl->error;
    if (b->h_ctl->tasks_done != b->last_tasks) return MTD_ERR_TIMEOUT;
    return MTD_OK;
}

int mtd_batch_solve(mtd_batch *b, const double *const *dA, const int64_t *lda, void *const *dF, const int64_t *ldf,
                    const double *const *dB, const int64_t *ldb, double *const *dX, const int64_t *ldx,
                    const int *nrhs, int method, double tol, int max_iter, void *stream, mtd_batch_solve_stats *stats) {
    if (!b || !dF || !ldf || !dB || !ldb || !dX || !ldx || !nrhs || max_iter < 0) return MTD_ERR_INVALID_ARG;
    if (method != MTD_REFINE_NONE && method != MTD_REFINE_IR) return MTD_ERR_INVALID_ARG;
    const bool low = b->prec != MTD_PREC_FP64;
    if ((method == MTD_REFINE_IR || low) && (!dA || !lda)) return MTD_ERR_INVALID_ARG;
    if (low && method == MTD_REFINE_NONE) return MTD_ERR_INVALID_ARG;  // a low-precision factor needs refinement
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const int count = b->count;
    int rc = ensure_solve_buffers(b);
    if (!rc) rc = stage_solve(b, dA, lda, dF, ldf, dB, ldb, dX, ldx, nrhs);
    if (rc) return rc;
    const auto t0 = std::chrono::steady_clock::now();
    if (cudaMemcpyAsync(b->d_solve, b->h_solve, count * sizeof(SolveMat), cudaMemcpyHostToDevice, s) != cudaSuccess)
        return MTD_ERR_CUDA;
    const size_t smem = bsolve::smem_bytes<kBT>(), smem64 = bsolve::trsv_bytes<double>(),
                 smem32 = bsolve::trsv_bytes<float>();
    if (cudaFuncSetAttribute(batch_trsv_kernel<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem64)) !=
            cudaSuccess ||
        cudaFuncSetAttribute(batch_trsv_kernel<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem32)) !=
            cudaSuccess ||
        cudaFuncSetAttribute(batch_residual_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)) !=
            cudaSuccess ||
        cudaFuncSetAttribute(batch_residual_zero_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)) !=
            cudaSuccess)
        return MTD_ERR_CUDA;
    const double *ws64 = reinterpret_cast<const double *>(b->d_ws);
    const float *ws32 = reinterpret_cast<const float *>(b->d_ws);
    mtd_batch_solve_stats st{};
    double worst = -1.0;
    if (!low) {  // one FP64 solve: x = (L L^T)^-1 b
        batch_copy_rhs_kernel<<<count, kBT, 0, s>>>(b->d_solve, false);
        batch_trsv_kernel<double><<<count, kBT, smem64, s>>>(b->d_solve, ws64, kOnX, Skip{nullptr, 0.0});
        st.iterations = 1;
    } else {
        batch_copy_rhs_kernel<<<count, kBT, 0, s>>>(b->d_solve, true);  // x = 0
    }
    if (dA) {
        for (int it = 0;; ++it) {
            if (low && it == 0)  // x = 0: the residual is b itself
                batch_residual_zero_kernel<<<count, kBT, smem, s>>>(b->d_solve, b->d_berr);
            else
                batch_residual_kernel<<<count, kBT, smem, s>>>(b->d_solve, b->d_anorm, b->d_berr, it == (low ? 1 : 0),
                                                               Skip{(it > 1 || (it > 0 && !low)) ? b->d_berr : nullptr,
                                                                    tol});
            if (cudaMemcpyAsync(b->h_berr, b->d_berr, count * sizeof(double), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
                cudaStreamSynchronize(s) != cudaSuccess)
                return MTD_ERR_CUDA;
            worst = 0.0;
            int done = 0;
            for (int m = 0; m < count; ++m) {
                worst = std::max(worst, b->h_berr[m]);
                done += b->h_berr[m] <= tol;
            }
            st.converged_count = done;
            if (method == MTD_REFINE_NONE) break;
            if ((it > 0 || !low) && done == count) break;
            if (it >= max_iter) break;
            // matrices already at tol keep their x (from the second residual on for a
            // low-precision factor, whose first residual is of x = 0)
            const Skip at_tol{(it > 0 || !low) ? b->d_berr : nullptr, tol};
            if (low) {  // x += M^-1 r through the low-precision factor
                batch_scale_kernel<float><<<count, kBT, 0, s>>>(b->d_solve, b->d_scale, true, at_tol);
                batch_trsv_kernel<float><<<count, kBT, smem32, s>>>(b->d_solve, ws32, kOnD, at_tol);
                batch_scale_kernel<float><<<count, kBT, 0, s>>>(b->d_solve, b->d_scale, false, at_tol);
            } else {    // x += (L L^T)^-1 r in FP64
                batch_trsv_kernel<double><<<count, kBT, smem64, s>>>(b->d_solve, ws64, kOnR, at_tol);
                batch_add_kernel<<<count, kBT, 0, s>>>(b->d_solve, at_tol);
            }
            st.iterations = it + 1 + (low ? 0 : 1);  // + the first FP64 solve
        }
    }
    if (cudaStreamSynchronize(s) != cudaSuccess || cudaGetLastError() != cudaSuccess) return MTD_ERR_CUDA;
    st.max_backward_error = worst;
    st.solve_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    if (stats) *stats = st;
    return rc;
}

int mtd_batch_factor_solve(mtd_batch *b, void *const *dF, const int64_t *ldf, const double *const *dA,
                           const int64_t *lda, const double *const *dB, const int64_t *ldb, double *const *dX,
                           const int64_t *ldx, const int *nrhs, int method, double tol, int max_iter, double shift,
                           void *stream) {
    if (!b || !dF || !ldf || !dB || !ldb || !dX || !ldx || !nrhs || max_iter < 0) return MTD_ERR_INVALID_ARG;
    if (method != MTD_REFINE_NONE && method != MTD_REFINE_IR) return MTD_ERR_INVALID_ARG;
    const bool low = b->prec != MTD_PREC_FP64;
    if ((method == MTD_REFINE_IR || low) && (!dA || !lda)) return MTD_ERR_INVALID_ARG;
    if (low && method == MTD_REFINE_NONE) return MTD_ERR_INVALID_ARG;  // a low-precision factor needs refinement
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    int rc = ensure_solve_buffers(b);
    if (!rc) rc = stage_solve(b, dA, lda, dF, ldf, dB, ldb, dX, ldx, nrhs);
    if (!rc && b->fs_convert != (low ? 1 : 0)) rc = build_fs(b, low);
    bool vec2 = true;
    if (!rc) rc = stage_factor(b, dF, ldf, s, &vec2);
    if (rc) return rc;
    if (cudaMemcpyAsync(b->d_solve, b->h_solve, b->count * sizeof(SolveMat), cudaMemcpyHostToDevice, s) !=
            cudaSuccess ||
        cudaMemsetAsync(b->d_fs_berr, 0xff, b->count * sizeof(double), s) != cudaSuccess ||  // NaN: not solved
        cudaMemsetAsync(b->d_fs_iters, 0, b->count * sizeof(int), s) != cudaSuccess)
        return MTD_ERR_CUDA;
    RunArgs a = batch_args(b);
    a.n_tasks = b->fs_tasks;
    a.tasks = b->d_fs_tasks;
    a.succ = b->d_fs_succ;
    a.deps = b->d_fs_deps;
    a.items_left = b->d_fs_items_left;
    long long items = 0;
    for (int q = 0; q < kNumQueues; ++q) {
        a.queue[q] = b->d_fs_queue[q];
        a.queue_cap[q] = b->fs_qcap[q];
        items += b->fs_qcap[q];
    }
    a.solve = b->d_solve;
    a.solve_berr = b->d_fs_berr;
    a.solve_iters = b->d_fs_iters;
    a.solve_tol = tol;
    a.solve_shift = shift;
    a.solve_method = method;
    a.solve_max_iter = max_iter;
    rc = launch_run_solve(a, b->d_fs_deps_init, b->d_fs_roots, b->fs_roots, items, b->prec, vec2, b->sms, s);
    if (rc) return rc;
    if (cudaMemcpyAsync(b->h_ctl, b->d_ctl, sizeof(RunCtl), cudaMemcpyDeviceToHost, s) != cudaSuccess) return MTD_ERR_CUDA;
    b->last_stream = s;
    b->last_tasks = b->fs_tasks;
    b->fs_tol = tol;
    b->pending = true;
    b->fs_pending = true;
    return MTD_OK;
}

int mtd_batch_solve_status(mtd_batch *b, int *info, double *latency_ms, double *berr, int *iterations,
                           mtd_batch_solve_stats *stats) {
    if (!b) return MTD_ERR_INVALID_ARG;
    if (!b->fs_pending) return MTD_ERR_STATE;
    const int count = b->count;
    std::vector<double> lat(count), be(count);
    std::vector<int> it(count);
    const int rc = mtd_batch_status(b, info, lat.data());
    if (rc == MTD_ERR_CUDA) return rc;
    if (cudaMemcpy(be.data(), b->d_fs_berr, count * sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess ||
        cudaMemcpy(it.data(), b->d_fs_iters, count * sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess)
        return MTD_ERR_CUDA;
    if (latency_ms) std::copy(lat.begin(), lat.end(), latency_ms);
    if (berr) std::copy(be.begin(), be.end(), berr);
    if (iterations) std::copy(it.begin(), it.end(), iterations);
    if (stats) {
        mtd_batch_solve_stats st{};
        st.max_backward_error = -1.0;
        double span = 0.0;
        for (int m = 0; m < count; ++m) {
            st.iterations = std::max(st.iterations, it[m]);
            if (be[m] == be[m]) {  // not NaN: solved
                st.max_backward_error = std::max(st.max_backward_error, be[m]);
                st.converged_count += be[m] >= 0.0 && be[m] <= b->fs_tol;
            }
            span = std::max(span, lat[m]);
        }
        st.solve_ms = span;
        *stats = st;
    }
    return rc;
}

int mtd_batch_tune_schedule(mtd_batch *b, void *const *dF, const int64_t *ldf, const void *const *dSrc,
                            const int64_t *ldsrc, const double *const *dA, const int64_t *lda, const double *const *dB,
                            const int64_t *ldb, double *const *dX, const int64_t *ldx, const int *nrhs, int method,
                            double tol, int max_iter, double shift, int reps, int *best, double *ms, void *stream) {
    if (!b || !dF || !ldf || reps < 1) return MTD_ERR_INVALID_ARG;
    const bool low = b->prec != MTD_PREC_FP64;
    if (!low && (!dSrc || !ldsrc)) return MTD_ERR_INVALID_ARG;  // FP64 factors overwrite their inputs
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const size_t es = batch_elem(b);
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) return MTD_ERR_CUDA;
    int rc = MTD_OK, winner = b->schedule;
    double best_ms = 1e300;
    for (int c = 0; c < MTD_BATCH_NUM_SCHEDULES && !rc; ++c) {
        const int sched = (c % 6 / 2) | (c % 2 ? MTD_BATCH_SOLVE_LATE : 0) | (c >= 6 ? MTD_BATCH_SOLVE_PAIRS : 0);
        rc = mtd_batch_set_schedule(b, sched);
        double cand = 1e300;
        for (int rep = 0; rep <= reps && !rc; ++rep) {  // rep 0 is untimed
            if (dSrc)
                for (int m = 0; m < b->count && !rc; ++m)
                    if (cudaMemcpy2DAsync(dF[m], ldf[m] * es, dSrc[m], ldsrc[m] * es, b->n[m] * es, b->n[m],
                                          cudaMemcpyDeviceToDevice, s) != cudaSuccess)
                        rc = MTD_ERR_CUDA;
            if (!rc && cudaEventRecord(e0, s) != cudaSuccess) rc = MTD_ERR_CUDA;
            if (!rc) rc = mtd_batch_factor_solve(b, dF, ldf, dA, lda, dB, ldb, dX, ldx, nrhs, method, tol, max_iter, shift, s);
            if (!rc && cudaEventRecord(e1, s) != cudaSuccess) rc = MTD_ERR_CUDA;
            if (!rc) rc = mtd_batch_solve_status(b, nullptr, nullptr, nullptr, nullptr, nullptr);
            float t = 0.f;
            if (!rc && cudaEventElapsedTime(&t, e0, e1) != cudaSuccess) rc = MTD_ERR_CUDA;
            if (!rc && rep > 0) cand = std::min(cand, double(t));
        }
        if (ms) ms[c] = rc ? -1.0 : cand;
        if (!rc && cand < best_ms) {
            best_ms = cand;
            winner = sched;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc) return rc;
    rc = mtd_batch_set_schedule(b, winner);
    if (best) *best = winner;
    return rc;
}

int mtd_batch_convert(mtd_batch *b, const double *const *dA, const int64_t *lda, void *const *dF, const int64_t *ldf,
                      double shift, void *stream) {
    if (!b || !dA || !lda || !dF || !ldf || b->prec == MTD_PREC_FP64) return MTD_ERR_INVALID_ARG;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (!b->h_solve) {
        if (cudaMallocHost(reinterpret_cast<void **>(&b->h_solve), b->count * sizeof(SolveMat)) != cudaSuccess)
            return MTD_ERR_OUT_OF_MEMORY;
        if (dalloc(&b->d_solve, b->count)) return MTD_ERR_OUT_OF_MEMORY;
    }
    for (int m = 0; m < b->count; ++m) {
        if (lda[m] < b->n[m] || ldf[m] < b->n[m]) return MTD_ERR_INVALID_ARG;
        SolveMat sm{};
        sm.a = dA[m];
        sm.lda = lda[m];
        sm.f = dF[m];
        sm.ldf = ldf[m];
        sm.n = static_cast<int>(b->n[m]);
        b->h_solve[m] = sm;
    }
    if (cudaMemcpyAsync(b->d_solve, b->h_solve, b->count * sizeof(SolveMat), cudaMemcpyHostToDevice, s) != cudaSuccess)
        return MTD_ERR_CUDA;
    batch_convert_kernel<<<dim3(8, b->count), kBT, 0, s>>>(b->d_solve, shift);
    // the staging buffer is reused by the next call: wait until the copy has been consumed
    if (cudaStreamSynchronize(s) != cudaSuccess) return MTD_ERR_CUDA;
    return cudaGetLastError() == cudaSuccess ? MTD_OK : MTD_ERR_CUDA;
}

int mtd_batch_destroy(mtd_batch *b) {
    if (!b) return MTD_ERR_INVALID_ARG;
    if (b->pending && b->last_stream) cudaStreamSynchronize(b->last_stream);
    cudaDeviceSynchronize();
    release_fs(b);
    release(b);
    delete b;
    return MTD_OK;
}

}  // extern "C"

namespace {

__global__ void to_float_kernel(const double *x, float *y, int64_t count) {
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < count; i += int64_t(gridDim.x) * blockDim.x)
        y[i] = static_cast<float>(x[i]);
}

// Trial settings for matrices of size n: one tile (tile = n), or tiles of 128 .. 512
// elements; each with no nesting or with 64- / 128-element nested diagonal factorisations.
std::vector<std::pair<int64_t, int>> tune_candidates(int64_t n) {
    std::vector<int64_t> tiles{n};
    for (int64_t t : {128, 256, 384, 512})
        if (t < n) tiles.push_back(t);
    std::vector<std::pair<int64_t, int>> out;
    for (int64_t t : tiles) {
        out.push_back({t, 0});
        for (int nest : {64, 128})
            if (nest < t) out.push_back({t, nest});
    }
    return out;
}

}  // namespace

extern "C" {

int mtd_batch_autotune(int count, const int64_t *n, int prec, int64_t *tile_out, int *nest_out, double *trial_ms,
                       void *stream) {
    if (count <= 0 || !n || !tile_out || !nest_out ||
        (prec != MTD_PREC_FP64 && prec != MTD_PREC_TF32 && prec != MTD_PREC_FP32))
        return MTD_ERR_INVALID_ARG;
    for (int m = 0; m < count; ++m)
        if (n[m] <= 0 || n[m] > (int64_t(1) << 20)) return MTD_ERR_INVALID_ARG;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const auto t0 = std::chrono::steady_clock::now();
    std::map<int64_t, int> per_size;
    for (int m = 0; m < count; ++m) ++per_size[n[m]];
    const size_t es = prec == MTD_PREC_FP64 ? sizeof(double) : sizeof(float);
    std::map<int64_t, std::pair<int64_t, int>> choice;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) return MTD_ERR_CUDA;
    int rc = MTD_OK;
    for (const auto &kv : per_size) {
        if (rc) break;
        const int64_t sz = kv.first;
        // a trial batch as large as this size's share of the batch (so the trial sees the
        // parallelism the real batch offers), capped at ~2^38 / 3 flop so it stays milliseconds
        const int k = std::max(1, std::min(kv.second, static_cast<int>(std::max<int64_t>(4, (int64_t(1) << 38) /
                                                                                         (sz * sz * sz)))));
        const size_t elems = size_t(k) * size_t(sz) * size_t(sz);
        double *src = nullptr;
        void *work = nullptr;
        float *src32 = nullptr;
        if (dalloc(&src, elems) || cudaMalloc(&work, std::max<size_t>(elems * es, 1)) != cudaSuccess ||
            (prec != MTD_PREC_FP64 && dalloc(&src32, elems))) {
            cudaFree(src);
            cudaFree(work);
            rc = MTD_ERR_OUT_OF_MEMORY;
            break;
        }
        for (int i = 0; i < k && !rc; ++i)
            rc = mtd_generate(src + size_t(i) * sz * sz, sz, sz, MTD_GEN_SPD, 0x5eed + uint64_t(i), 1.0, s);
        if (!rc && src32) to_float_kernel<<<1024, 256, 0, s>>>(src, src32, static_cast<int64_t>(elems));
        const void *pristine = src32 ? static_cast<const void *>(src32) : static_cast<const void *>(src);
        std::vector<void *> ptrs(k);
        std::vector<int64_t> lds(k, sz), sizes(k, sz), tiles(k);
        std::vector<int> nests(k);
        for (int i = 0; i < k; ++i) ptrs[i] = static_cast<unsigned char *>(work) + size_t(i) * sz * sz * es;
        double best_ms = 1e300;
        std::pair<int64_t, int> best{std::min<int64_t>(sz, 512), sz > kNestTile ? kNestTile : 0};
        for (const auto &cand : tune_candidates(sz)) {
            if (rc) break;
            std::fill(tiles.begin(), tiles.end(), cand.first);
            std::fill(nests.begin(), nests.end(), cand.second);
            mtd_batch *b = nullptr;
            rc = mtd_batch_create(&b, k, sizes.data(), tiles.data(), nests.data(), prec);
            if (rc) break;
            double ms_min = 1e300;
            for (int rep = 0; rep < 2 && !rc; ++rep) {  // the first run warms up
                if (cudaMemcpyAsync(work, pristine, elems * es, cudaMemcpyDeviceToDevice, s) != cudaSuccess ||
                    cudaEventRecord(e0, s) != cudaSuccess) {
                    rc = MTD_ERR_CUDA;
                    break;
                }
                rc = mtd_batch_factor(b, ptrs.data(), lds.data(), s);
                if (!rc && cudaEventRecord(e1, s) != cudaSuccess) rc = MTD_ERR_CUDA;
                if (!rc) rc = mtd_batch_status(b, nullptr, nullptr);
                float ms = 0.f;
                if (!rc && cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess) rc = MTD_ERR_CUDA;
                if (!rc && rep > 0) ms_min = std::min(ms_min, double(ms));
            }
            mtd_batch_destroy(b);
            if (!rc && ms_min < best_ms) {
                best_ms = ms_min;
                best = cand;
            }
        }
        choice[sz] = best;
        cudaFree(src);
        cudaFree(work);
        cudaFree(src32);
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc) return rc;
    for (int m = 0; m < count; ++m) {
        tile_out[m] = choice[n[m]].first;
        nest_out[m] = choice[n[m]].second;
    }
    if (trial_ms) *trial_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    return MTD_OK;
}

}  // extern "C"
