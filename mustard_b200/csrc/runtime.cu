// C ABI implementation: graph lifetime, device upload, runs, statistics.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <new>
#include <vector>

#include "../../include/mustard_b200.h"
#include "dag.hpp"
#include "scheduler.cuh"

using namespace mtd;

// Device scratch of mtd_factor_noalloc: task table, successor lists, counters, ready
// queues, control block and inverse workspaces of one factorisation, carved from this
// one array at 256-byte boundaries.  Its size and the limits below are fixed; every GPU
// that loads the library holds the array until the process exits.
constexpr size_t kNoAllocBytes = size_t(24) << 20;
constexpr int64_t kNoAllocMaxN = 16384;
constexpr int kNoAllocMaxTasks = 32768;
constexpr int kNoAllocMaxEdges = 131072;
constexpr long long kNoAllocMaxItems = 262144;
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

struct mtd_graph {
    Dag dag;
    bool finalized = false;
    int device = 0;
    int num_sms = 0;
    bool trace = false;
    double timeout_s = 10.0;
    int nest = kNestTile;
    // FP64 GEMM / SYRK items fed by TMA (tma64.cuh) when the geometry allows and the
    // environment variable MTD_TMA64=1 is set when the graph is finalised; by default they run
    // on the cp.async engine, which measured faster on B200 (the TMA engine's swizzled
    // fragment addressing costs more issue slots than the copies it saves)
    bool use_tma64 = false;
    int opset = kOpsAll;  // operation family of the lowered tasks (the FP64 kernel instance)
    int prec = MTD_PREC_FP64;  // element type of the matrix runs factor
    unsigned short *d_bf16 = nullptr;  // MTD_PREC_BF16: BF16 copy of the panels (bf16_ld x n)
    int64_t bf16_ld = 0;
    float *d_lo = nullptr;  // MTD_PREC_FP32: low parts of the panels (lo_ld x n)
    int64_t lo_ld = 0;
    Lowered low;   // device form, kept for the CUDA-graph executor and item queries
    int n_dev = 0;

    DevTask *d_tasks = nullptr;
    int *d_succ = nullptr;
    int *d_deps_init = nullptr;
    int *d_deps = nullptr;
    int *d_items_left = nullptr;
    int *d_roots = nullptr;
    int n_roots = 0;
    unsigned long long *d_queue[kNumQueues] = {nullptr, nullptr};
    long long queue_cap[kNumQueues] = {0, 0};
    QueueCtl *d_qctl = nullptr;
    RunCtl *d_ctl = nullptr;
    RunCtl *h_ctl = nullptr;  // pinned copy of the control block, filled at the end of a run
    unsigned char *d_ws_lower = nullptr;  // inverse workspaces, elements of the run's type
    unsigned char *d_ws_upper = nullptr;
    unsigned long long *d_trace = nullptr;
    long long trace_cap = 0;
    long long total_items = 0;

    cudaStream_t last_stream = nullptr;
    bool run_pending = false;
    bool last_was_graph = false;
    int last_grid = 0;

    // Host-launched CUDA-graph executor (built on first use for a given matrix).
    cudaGraph_t cgraph = nullptr;
    cudaGraphExec_t cexec = nullptr;
    double *cgraph_a = nullptr;
    int64_t cgraph_lda = 0;

    mtd_graph(int kind, int64_t n, int64_t tile) : dag(kind, n, tile) {}
};

namespace {

// Once per device and vector width: the kernels' dynamic shared-memory limits.  Runs on
// different graphs may start from several host threads at once.
template <int VEC>
int smem_setup(int device) {
    static std::atomic<bool> done[64];
    static std::mutex mu;
    if (device < 0 || device >= 64) return MTD_ERR_INVALID_ARG;
    if (done[device].load(std::memory_order_acquire)) return MTD_OK;
    std::lock_guard<std::mutex> lock(mu);
    if (!done[device].load(std::memory_order_relaxed)) {
        const int bytes = kOpSmemBytes();
        if (cudaFuncSetAttribute(persistent_kernel<VEC, double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 bytes) != cudaSuccess ||
            cudaFuncSetAttribute(persistent_kernel<VEC, float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 bytes) != cudaSuccess ||
            cudaFuncSetAttribute(persistent_kernel<VEC, float, 3>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 bytes) != cudaSuccess ||
            cudaFuncSetAttribute(task_kernel<VEC, double>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes) !=
                cudaSuccess ||
            cudaFuncSetAttribute(persistent_kernel<VEC, double, 1, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 bytes) != cudaSuccess ||
            cudaFuncSetAttribute(persistent_kernel<VEC, float, 3, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 bytes) != cudaSuccess ||
            cudaFuncSetAttribute(persistent_kernel<VEC, double, 1, false, true>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, bytes) != cudaSuccess)
            return MTD_ERR_CUDA;
        if constexpr (VEC == 2) {
            if (cudaFuncSetAttribute(persistent_kernel<2, double, 1, false, false, false, kOpsCholesky>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, bytes) != cudaSuccess ||
                cudaFuncSetAttribute(persistent_kernel<2, double, 1, false, false, false, kOpsLu>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, bytes) != cudaSuccess)
                return MTD_ERR_CUDA;
        }
        done[device].store(true, std::memory_order_release);
    }
    return MTD_OK;
}

// Leading dimension of the inverse workspace of an n x n factorisation: n rounded up to a
// multiple of 4 so every 64-column block starts on a 16-byte boundary for either element
// size.  Every entry point that lays out a workspace uses this one rule.
int64_t ws_ld_for(int64_t n) { return (n + 3) & ~int64_t(3); }
int64_t ws_ld(const mtd_graph *g) { return ws_ld_for(g->dag.n()); }

// The operation family of a lowered task list (joins belong to every family).
int opset_of(const std::vector<DevTask> &tasks) {
    bool chol = true, lu = true;
    for (const auto &t : tasks) {
        if (t.op == kOpJoin) continue;
        const bool c = t.op == MTD_OP_POTRF || t.op == MTD_OP_TRSM_RLT || t.op == MTD_OP_SYRK_LN || t.op == MTD_OP_GEMM_NT;
        const bool l = t.op == MTD_OP_GETRF || t.op == MTD_OP_TRSM_LLNU || t.op == MTD_OP_TRSM_RUN || t.op == MTD_OP_GEMM_NN;
        chol = chol && c;
        lu = lu && l;
    }
    return chol ? kOpsCholesky : lu ? kOpsLu : kOpsAll;
}


size_t elem_size(const mtd_graph *g) { return g->prec == MTD_PREC_FP64 ? sizeof(double) : sizeof(float); }

// 16-byte copies need 16-byte aligned bases and leading dimensions and extents that are
// whole 16-byte chunks of elements.
bool use_vec2(const mtd_graph *g, const void *dA, int64_t lda) {
    const int64_t epc = 16 / static_cast<int64_t>(elem_size(g));
    return (reinterpret_cast<uintptr_t>(dA) % 16 == 0) && (lda % epc == 0) && (g->dag.unit() % epc == 0) &&
           (g->dag.n() % epc == 0);
}

RunArgs make_args(const mtd_graph *g, void *dA, int64_t lda) {
    RunArgs a{};
    a.a = dA;
    a.lda = lda;
    a.n_tasks = g->n_dev;
    a.tasks = g->d_tasks;
    a.succ = g->d_succ;
    a.deps = g->d_deps;
    a.items_left = g->d_items_left;
    for (int q = 0; q < kNumQueues; ++q) {
        a.queue[q] = g->d_queue[q];
        a.queue_cap[q] = g->queue_cap[q];
    }
    a.qctl = g->d_qctl;
    a.ctl = g->d_ctl;
    a.ws_lower = g->d_ws_lower;
    a.ws_upper = g->d_ws_upper;
    a.ws_ld = ws_ld(g);
    a.trace = g->d_trace;
    a.trace_cap = g->trace_cap;
    a.timeout_ns = static_cast<unsigned long long>(g->timeout_s * 1e9);
    a.bf16 = g->d_bf16;
    a.bf16_ld = g->bf16_ld;
    return a;
}

void release_cgraph(mtd_graph *g) {
    if (g->cexec) cudaGraphExecDestroy(g->cexec);
    if (g->cgraph) cudaGraphDestroy(g->cgraph);
    g->cexec = nullptr;
    g->cgraph = nullptr;
    g->cgraph_a = nullptr;
}

// One kernel node per task (grid = its work items) with the task's predecessors as
// node dependencies, after a node that clears the error word.
int build_cgraph(mtd_graph *g, double *dA, int64_t lda) {
    release_cgraph(g);
    const RunArgs a = make_args(g, dA, lda);
    const bool vec2 = use_vec2(g, dA, lda);
    if (cudaGraphCreate(&g->cgraph, 0) != cudaSuccess) return MTD_ERR_CUDA;
    cudaGraphNode_t reset;
    {
        cudaKernelNodeParams kp{};
        void *args[] = {const_cast<RunArgs *>(&a)};
        kp.func = reinterpret_cast<void *>(reset_ctl_kernel);
        kp.gridDim = dim3(1);
        kp.blockDim = dim3(32);
        kp.kernelParams = args;
        if (cudaGraphAddKernelNode(&reset, g->cgraph, nullptr, 0, &kp) != cudaSuccess) return MTD_ERR_CUDA;
    }
    const int nt = g->n_dev;
    std::vector<cudaGraphNode_t> nodes(nt);
    std::vector<cudaGraphNode_t> deps;
    for (int t = 0; t < nt; ++t) {
        deps.clear();
        for (int d : g->low.preds[t]) deps.push_back(nodes[d]);
        if (deps.empty()) deps.push_back(reset);
        const int items = g->low.tasks[t].n_items;
        if (items == 0) {
            if (cudaGraphAddEmptyNode(&nodes[t], g->cgraph, deps.data(), deps.size()) != cudaSuccess)
                return MTD_ERR_CUDA;
            continue;
        }
        int task = t;
        void *args[] = {const_cast<RunArgs *>(&a), &task};
        cudaKernelNodeParams kp{};
        kp.func = vec2 ? reinterpret_cast<void *>(task_kernel<2, double>)
                       : reinterpret_cast<void *>(task_kernel<1, double>);
        kp.gridDim = dim3(static_cast<unsigned>(items));
        kp.blockDim = dim3(kThreads);
        kp.sharedMemBytes = kOpSmemBytes();
        kp.kernelParams = args;
        if (cudaGraphAddKernelNode(&nodes[t], g->cgraph, deps.data(), deps.size(), &kp) != cudaSuccess)
            return MTD_ERR_CUDA;
    }
    if (cudaGraphInstantiate(&g->cexec, g->cgraph, 0) != cudaSuccess) return MTD_ERR_CUDA;
    g->cgraph_a = dA;
    g->cgraph_lda = lda;
    return MTD_OK;
}

int check_device(int *device, int *num_sms) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return MTD_ERR_NO_DEVICE;
    int major = 0;
    if (cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev) != cudaSuccess)
        return MTD_ERR_NO_DEVICE;
    if (major != 10) return MTD_ERR_NO_DEVICE;  // built for sm_100a only
    if (cudaDeviceGetAttribute(num_sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
        return MTD_ERR_NO_DEVICE;
    *device = dev;
    return MTD_OK;
}

template <typename T>
int dev_alloc(T **p, size_t count) {
    if (count == 0) count = 1;
    if (cudaMalloc(reinterpret_cast<void **>(p), count * sizeof(T)) != cudaSuccess) {
        cudaGetLastError();
        *p = nullptr;
        return MTD_ERR_OUT_OF_MEMORY;
    }
    return MTD_OK;
}

void release_device(mtd_graph *g) {
    cudaFree(g->d_tasks);
    cudaFree(g->d_succ);
    cudaFree(g->d_deps_init);
    cudaFree(g->d_deps);
    cudaFree(g->d_items_left);
    cudaFree(g->d_roots);
    for (int q = 0; q < kNumQueues; ++q) cudaFree(g->d_queue[q]);
    cudaFree(g->d_qctl);
    cudaFree(g->d_ctl);
    if (g->h_ctl) cudaFreeHost(g->h_ctl);
    cudaFree(g->d_ws_lower);
    cudaFree(g->d_bf16);
    g->d_bf16 = nullptr;
    cudaFree(g->d_lo);
    g->d_lo = nullptr;
    cudaFree(g->d_ws_upper);
    cudaFree(g->d_trace);
}

}  // namespace

extern "C" {

int mtd_abi_version(void) { return MTD_ABI_VERSION; }

const char *mtd_strerror(int status) {
    switch (status) {
    case MTD_OK: return "ok";
    case MTD_ERR_INVALID_ARG: return "invalid argument";
    case MTD_ERR_STATE: return "call out of order for this graph";
    case MTD_ERR_CUDA: return "CUDA runtime error";
    case MTD_ERR_TIMEOUT: return "device-side wait exceeded its time limit";
    case MTD_ERR_NOT_POSITIVE_DEFINITE: return "matrix is not positive definite (see info)";
    case MTD_ERR_SINGULAR: return "zero pivot in LU without pivoting (see info)";
    case MTD_ERR_BAD_DAG: return "task graph cannot be executed";
    case MTD_ERR_NO_DEVICE: return "no sm_100 CUDA device";
    case MTD_ERR_OUT_OF_MEMORY: return "device allocation failed";
    case MTD_ERR_QUEUE: return "ready-queue overflow";
    case MTD_ERR_TOO_LARGE: return "problem exceeds the fixed scratch of mtd_factor_noalloc";
    default: return "unknown status";
    }
}

int mtd_graph_create(mtd_graph **out, int kind, int64_t n, int64_t tile) {
    if (!out) return MTD_ERR_INVALID_ARG;
    *out = nullptr;
    if (kind < MTD_KIND_LU || kind > MTD_KIND_CUSTOM) return MTD_ERR_INVALID_ARG;
    if (n <= 0 || tile <= 0 || tile > n) return MTD_ERR_INVALID_ARG;
    if (n > (int64_t(1) << 31) - 1) return MTD_ERR_INVALID_ARG;
    if ((n + tile - 1) / tile > 4096) return MTD_ERR_INVALID_ARG;
    mtd_graph *g = new (std::nothrow) mtd_graph(kind, n, tile);
    if (!g) return MTD_ERR_OUT_OF_MEMORY;
    *out = g;
    return MTD_OK;
}

int mtd_graph_add_task(mtd_graph *g, int op, int wi, int wj, const int *reads, int nreads) {
    if (!g) return -MTD_ERR_INVALID_ARG;
    if (g->finalized) return -MTD_ERR_STATE;
    return g->dag.add_task(op, wi, wj, reads, nreads);
}

int mtd_graph_build_tiled(mtd_graph *g) {
    if (!g) return MTD_ERR_INVALID_ARG;
    if (g->finalized || g->dag.num_tasks() != 0) return MTD_ERR_STATE;
    return g->dag.build_reference_order();
}

int mtd_graph_num_tasks(const mtd_graph *g) { return g ? g->dag.num_tasks() : -MTD_ERR_INVALID_ARG; }

int mtd_graph_get_deps(const mtd_graph *g, int task, int *out, int cap) {
    if (!g || task < 0 || task >= g->dag.num_tasks() || cap < 0 || (cap > 0 && !out)) return -MTD_ERR_INVALID_ARG;
    const auto &d = g->dag.deps(task);
    for (int i = 0; i < cap && i < static_cast<int>(d.size()); ++i) out[i] = d[i];
    return static_cast<int>(d.size());
}

int mtd_graph_task_info(const mtd_graph *g, int task, int *op_out, int *wi_out, int *wj_out, int *reads_out,
                        int cap) {
    if (!g || task < 0 || task >= g->dag.num_tasks() || cap < 0 || (cap > 0 && !reads_out)) return -MTD_ERR_INVALID_ARG;
    const HostTask &t = g->dag.task(task);
    if (op_out) *op_out = t.op;
    if (wi_out) *wi_out = t.write.first;
    if (wj_out) *wj_out = t.write.second;
    const int nr = static_cast<int>(t.reads.size());
    for (int r = 0; r < nr && r < cap; ++r) {
        reads_out[2 * r] = t.reads[r].first;
        reads_out[2 * r + 1] = t.reads[r].second;
    }
    return nr;
}

int mtd_graph_num_device_tasks(const mtd_graph *g) { return g ? (g->finalized ? g->n_dev : 0) : -MTD_ERR_INVALID_ARG; }

int mtd_graph_task_items(const mtd_graph *g, int task) {
    if (!g || task < 0 || task >= g->dag.num_tasks()) return -MTD_ERR_INVALID_ARG;
    return g->finalized ? g->low.host_items[task] : 0;
}

int mtd_graph_device_task_op(const mtd_graph *g, int task) {
    if (!g || !g->finalized || task < 0 || task >= static_cast<int>(g->low.tasks.size())) return -MTD_ERR_INVALID_ARG;
    return g->low.tasks[task].op;
}

int mtd_graph_device_task_deps(const mtd_graph *g, int task, int *out, int cap) {
    if (!g || !g->finalized || task < 0 || task >= static_cast<int>(g->low.tasks.size()) || cap < 0 ||
        (cap > 0 && !out))
        return -MTD_ERR_INVALID_ARG;
    const auto &d = g->low.preds[task];
    for (int i = 0; i < cap && i < static_cast<int>(d.size()); ++i) out[i] = d[i];
    return static_cast<int>(d.size());
}

int mtd_graph_set_trace(mtd_graph *g, int enable) {
    if (!g) return MTD_ERR_INVALID_ARG;
    if (g->finalized) return MTD_ERR_STATE;
    g->trace = enable != 0;
    return MTD_OK;
}

int mtd_graph_set_nest(mtd_graph *g, int nest) {
    if (!g || nest < 0 || nest % kNB != 0) return MTD_ERR_INVALID_ARG;
    if (g->finalized) return MTD_ERR_STATE;
    g->nest = nest;
    return MTD_OK;
}

int mtd_graph_set_tile_edges(mtd_graph *g, const int64_t *edges, int count) {
    if (!g || !edges || count < 2) return MTD_ERR_INVALID_ARG;
    if (g->finalized) return MTD_ERR_STATE;
    return g->dag.set_edges(std::vector<int64_t>(edges, edges + count));
}

int mtd_graph_set_timeout(mtd_graph *g, double seconds) {
    if (!g || !(seconds > 0.0) || seconds > 3600.0) return MTD_ERR_INVALID_ARG;
    g->timeout_s = seconds;
    return MTD_OK;
}

int mtd_graph_finalize(mtd_graph *g) {
    if (!g) return MTD_ERR_INVALID_ARG;
    if (g->finalized) return MTD_ERR_STATE;
    if (g->dag.num_tasks() == 0) return MTD_ERR_BAD_DAG;
    int rc = check_device(&g->device, &g->num_sms);
    if (rc) return rc;

    rc = g->dag.lower(g->nest, g->low);
    if (rc) return rc;
    {
        const char *e = std::getenv("MTD_TMA64");
        g->use_tma64 = e && e[0] == '1';
    }
    const std::vector<DevTask> &tasks = g->low.tasks;
    const std::vector<int> &succ = g->low.succ;
    const int64_t *cap = g->low.queue_cap;
    const int nt = static_cast<int>(tasks.size());
    std::vector<int> preds(nt), roots;
    for (int t = 0; t < nt; ++t) {
        preds[t] = static_cast<int>(g->low.preds[t].size());
        if (preds[t] == 0) roots.push_back(t);
    }
    if (roots.empty()) return MTD_ERR_BAD_DAG;
    g->n_dev = nt;
    g->opset = opset_of(tasks);
    const size_t ws = size_t(ws_ld(g)) * kNB * elem_size(g);  // bytes
    g->total_items = 0;
    for (int q = 0; q < kNumQueues; ++q) {
        g->queue_cap[q] = cap[q];
        g->total_items += cap[q];
    }
    g->trace_cap = g->trace ? g->total_items : 0;
    bool needs_upper = false;
    for (const auto &t : tasks)
        if (t.op == MTD_OP_GETRF) needs_upper = true;
    if (g->prec != MTD_PREC_FP64) {
        // the low-precision factor is Cholesky-only
        for (const auto &t : tasks)
            if (t.op != MTD_OP_POTRF && t.op != MTD_OP_TRSM_RLT && t.op != MTD_OP_SYRK_LN && t.op != MTD_OP_GEMM_NT &&
                t.op != kOpJoin)
                return MTD_ERR_INVALID_ARG;
    }

    rc = MTD_OK;
    rc = rc ? rc : dev_alloc(&g->d_tasks, nt);
    rc = rc ? rc : dev_alloc(&g->d_succ, succ.size());
    rc = rc ? rc : dev_alloc(&g->d_deps_init, nt);
    rc = rc ? rc : dev_alloc(&g->d_deps, nt);
    rc = rc ? rc : dev_alloc(&g->d_items_left, nt);
    rc = rc ? rc : dev_alloc(&g->d_roots, roots.size());
    for (int q = 0; q < kNumQueues; ++q) rc = rc ? rc : dev_alloc(&g->d_queue[q], size_t(cap[q]));
    rc = rc ? rc : dev_alloc(&g->d_qctl, kNumQueues);
    rc = rc ? rc : dev_alloc(&g->d_ctl, 1);
    rc = rc ? rc : dev_alloc(&g->d_ws_lower, ws);
    if (needs_upper) rc = rc ? rc : dev_alloc(&g->d_ws_upper, ws);
    if (g->prec == MTD_PREC_BF16) {
        g->bf16_ld = (g->dag.n() + 63) & ~int64_t(63);
        rc = rc ? rc : dev_alloc(&g->d_bf16, size_t(g->bf16_ld) * size_t(g->dag.n()));
    }
    // FP32-accurate runs whose updates can take the three-pass tcgen05 path: the panels' low
    // parts (the TMA boxes start on 32-row atoms, so n, the tile and the nested sub-tile are
    // multiples of 32)
    if (g->prec == MTD_PREC_FP32 && g->dag.n() % 32 == 0 && g->dag.unit() % 32 == 0 && g->nest % 32 == 0) {
        g->lo_ld = (g->dag.n() + 63) & ~int64_t(63);
        rc = rc ? rc : dev_alloc(&g->d_lo, size_t(g->lo_ld) * size_t(g->dag.n()));
    }
    if (g->trace) rc = rc ? rc : dev_alloc(&g->d_trace, size_t(4 * g->trace_cap));
    if (!rc && cudaMallocHost(reinterpret_cast<void **>(&g->h_ctl), sizeof(RunCtl)) != cudaSuccess) {
        g->h_ctl = nullptr;
        rc = MTD_ERR_OUT_OF_MEMORY;
    }
    if (!rc) {
        bool ok = cudaMemcpy(g->d_tasks, tasks.data(), nt * sizeof(DevTask), cudaMemcpyHostToDevice) == cudaSuccess;
        ok = ok && (succ.empty() ||
                    cudaMemcpy(g->d_succ, succ.data(), succ.size() * sizeof(int), cudaMemcpyHostToDevice) == cudaSuccess);
        ok = ok && cudaMemcpy(g->d_deps_init, preds.data(), nt * sizeof(int), cudaMemcpyHostToDevice) == cudaSuccess;
        ok = ok && cudaMemcpy(g->d_roots, roots.data(), roots.size() * sizeof(int), cudaMemcpyHostToDevice) == cudaSuccess;
        ok = ok && cudaMemset(g->d_ws_lower, 0, ws) == cudaSuccess;
        if (needs_upper) ok = ok && cudaMemset(g->d_ws_upper, 0, ws) == cudaSuccess;
        // rows past n of the copy's last atom are read by TMA and multiplied into rows the
        // epilogue never stores; keep them finite
        if (g->d_bf16)
            ok = ok && cudaMemset(g->d_bf16, 0, size_t(g->bf16_ld) * size_t(g->dag.n()) * 2) == cudaSuccess;
        if (g->d_lo)  // rows past n of the last atom are read by TMA; keep them finite
            ok = ok && cudaMemset(g->d_lo, 0, size_t(g->lo_ld) * size_t(g->dag.n()) * sizeof(float)) == cudaSuccess;
        ok = ok && cudaMemset(g->d_ctl, 0, sizeof(RunCtl)) == cudaSuccess;
        if (!ok) rc = MTD_ERR_CUDA;
    }
    if (!rc) rc = smem_setup<2>(g->device);
    if (!rc) rc = smem_setup<1>(g->device);
    if (rc) {
        release_device(g);
        g->d_tasks = nullptr;
        return rc;
    }
    std::memset(g->h_ctl, 0, sizeof(RunCtl));
    g->n_roots = static_cast<int>(roots.size());
    g->finalized = true;
    return MTD_OK;
}

}  // extern "C"

namespace mtd {

// TMA tensor map of an FP32 n x n column-major matrix (ld elements) for the tcgen05 GEMM /
// SYRK items: 128-byte swizzle with 32-byte atoms (the layout the TF32 MMA reads for MN-major
// operands), zero fill past the matrix.  With n a multiple of 32 the map is 3D (32 rows of an
// atom, columns, atoms 128 bytes apart; box 32 x 64 x 4), so one load fetches a whole
// 128-row operand slice; otherwise 2D (rows, columns; box 32 x 64).  The driver entry point
// is looked up once; without it (or on an encoding error) the run keeps its cp.async path.
// The driver's tensor-map encoder, looked up once (nullptr if the driver has none).
PFN_cuTensorMapEncodeTiled_v12000 tmap_encoder() {
    static PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        cudaDriverEntryPointQueryResult q;
        void *fn = nullptr;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
    });
    return encode;
}

void encode_tmap(RunArgs &a, void *dA, int64_t n, int64_t ld) {
    static_assert(sizeof(CUtensorMap) == sizeof(a.tmap), "tensor map storage");
    const PFN_cuTensorMapEncodeTiled_v12000 encode = tmap_encoder();
    a.tma = tc::kTmaNone;
    if (!encode) return;
    CUtensorMap map;
    CUresult r;
    if (n % 32 == 0) {
        const cuuint64_t dims[3] = {32, cuuint64_t(n), cuuint64_t(n / 32)};
        const cuuint64_t strides[2] = {cuuint64_t(ld) * sizeof(float), 32 * sizeof(float)};
        const cuuint32_t box[3] = {32, tc::kTmaBK, 4}, elem[3] = {1, 1, 1};
        r = encode(&map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, dA, dims, strides, box, elem, CU_TENSOR_MAP_INTERLEAVE_NONE,
                   CU_TENSOR_MAP_SWIZZLE_128B_ATOM_32B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                   CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    } else {
        const cuuint64_t dims[2] = {cuuint64_t(n), cuuint64_t(n)};
        const cuuint64_t strides[1] = {cuuint64_t(ld) * sizeof(float)};
        const cuuint32_t box[2] = {32, tc::kTmaBK}, elem[2] = {1, 1};
        r = encode(&map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, dA, dims, strides, box, elem, CU_TENSOR_MAP_INTERLEAVE_NONE,
                   CU_TENSOR_MAP_SWIZZLE_128B_ATOM_32B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                   CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    }
    if (r != CUDA_SUCCESS) return;
    std::memcpy(a.tmap, &map, sizeof(map));
    a.tma = n % 32 == 0 ? tc::kTmaMap3D : tc::kTmaMap2D;
}

// TMA tensor map of the BF16 copy of the panels (column-major, leading dimension ld, a
// multiple of 64) for the BF16 GEMM / SYRK items: 3D (64 rows of an atom, columns, atoms
// 128 bytes apart), box 64 x 128 x 2 (a 128-row x 128-column operand slice per load),
// 128-byte swizzle -- the MN-major layout tcgen05 kind::f16 reads with 64-element atoms.
// Rows past n (the last atom's padding) hold zeros.  Without the encoder, or on an encoding
// error, the run keeps the TF32 path for every update.
void encode_tmap_bf16(RunArgs &a, void *d16, int64_t n, int64_t ld) {
    static_assert(sizeof(CUtensorMap) == sizeof(a.tmap_bf16), "tensor map storage");
    const PFN_cuTensorMapEncodeTiled_v12000 encode = tmap_encoder();
    a.tma_bf16 = 0;
    if (!encode || !d16 || ld % 64 != 0) return;
    const cuuint64_t dims[3] = {64, cuuint64_t(n), cuuint64_t(ld / 64)};
    const cuuint64_t strides[2] = {cuuint64_t(ld) * 2, 128};
    const cuuint32_t box[3] = {64, tc::kBfBK, 2}, elem[3] = {1, 1, 1};
    CUtensorMap map;
    if (encode(&map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 3, d16, dims, strides, box, elem, CU_TENSOR_MAP_INTERLEAVE_NONE,
               CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
        return;
    std::memcpy(a.tmap_bf16, &map, sizeof(map));
    a.tma_bf16 = 1;
}

// 3D TMA map of an FP32 n x n column-major matrix (ld elements; n a multiple of 32): 32 rows of
// an atom, columns, atoms 128 bytes apart; box 32 x bk x 4 (a 128-row operand slice per load);
// 128-byte swizzle with 32-byte atoms, zero fill past the matrix.  False without the encoder or
// on an encoding error.
bool encode_f32_3d(unsigned char *storage, void *ptr, int64_t n, int64_t ld, int bk) {
    const PFN_cuTensorMapEncodeTiled_v12000 encode = tmap_encoder();
    if (!encode || n % 32 != 0 || ld % 4 != 0) return false;
    CUtensorMap map;
    const cuuint64_t dims[3] = {32, cuuint64_t(n), cuuint64_t(n / 32)};
    const cuuint64_t strides[2] = {cuuint64_t(ld) * sizeof(float), 32 * sizeof(float)};
    const cuuint32_t box[3] = {32, cuuint32_t(bk), 4}, elem[3] = {1, 1, 1};
    if (encode(&map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, ptr, dims, strides, box, elem, CU_TENSOR_MAP_INTERLEAVE_NONE,
               CU_TENSOR_MAP_SWIZZLE_128B_ATOM_32B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
        return false;
    std::memcpy(storage, &map, sizeof(map));
    return true;
}

// TMA tensor maps of an FP64 n x n column-major matrix (ld elements) for the FP64 GEMM /
// SYRK items (tma64.cuh): 3D {16 rows of an atom, columns, atoms} with box {16, 16, 8} for
// m- / n-contiguous operands, 2D {rows, columns} with box {16, 128} for the k-contiguous
// operand of GEMM_NN; 128-byte swizzle, zero fill past the matrix.  Needs n a multiple of
// 16 (whole atoms) and 16-byte aligned columns; without the encoder, or on an encoding
// error, the run keeps the cp.async engine for every item.
void encode_tmap64(RunArgs &a, void *dA, int64_t n, int64_t ld) {
    static_assert(sizeof(CUtensorMap) == sizeof(a.tmap64_mn), "tensor map storage");
    const PFN_cuTensorMapEncodeTiled_v12000 encode = tmap_encoder();
    a.tma64 = 0;
    if (!encode || n % 16 != 0 || ld % 2 != 0 || reinterpret_cast<uintptr_t>(dA) % 16 != 0) return;
    CUtensorMap mn, kc;
    const cuuint64_t dims3[3] = {16, cuuint64_t(n), cuuint64_t(n / 16)};
    const cuuint64_t strides3[2] = {cuuint64_t(ld) * sizeof(double), 16 * sizeof(double)};
    const cuuint32_t box3[3] = {16, cuuint32_t(t64::kBK), 8}, elem3[3] = {1, 1, 1};
    if (encode(&mn, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, dA, dims3, strides3, box3, elem3, CU_TENSOR_MAP_INTERLEAVE_NONE,
               CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
        return;
    const cuuint64_t dims2[2] = {cuuint64_t(n), cuuint64_t(n)};
    const cuuint64_t strides2[1] = {cuuint64_t(ld) * sizeof(double)};
    const cuuint32_t box2[2] = {16, 128}, elem2[2] = {1, 1};
    if (encode(&kc, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 2, dA, dims2, strides2, box2, elem2, CU_TENSOR_MAP_INTERLEAVE_NONE,
               CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
        return;
    std::memcpy(a.tmap64_mn, &mn, sizeof(mn));
    std::memcpy(a.tmap64_k, &kc, sizeof(kc));
    a.tma64 = 1;
}

// Reset, seed and launch one persistent run (shared by graphs, batches and the
// no-allocation entry point's sibling paths).  Stream-ordered; no host synchronisation.
int launch_run(const RunArgs &a, const int *deps_init, const int *roots, int n_roots, long long total_items,
               int prec, bool vec2, int grid, cudaStream_t s, bool adjoint) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return MTD_ERR_NO_DEVICE;
    int rc = smem_setup<2>(dev);
    if (!rc) rc = smem_setup<1>(dev);
    if (rc) return rc;
    const int reset_blocks = static_cast<int>(std::min<long long>(
        1024, std::max<long long>(1, (std::max<long long>(total_items, a.n_tasks) + kThreads - 1) / kThreads)));
    reset_kernel<<<reset_blocks, kThreads, 0, s>>>(a, deps_init);
    seed_kernel<<<1, kSeedThreads, 0, s>>>(a, roots, n_roots);
    const int bytes = kOpSmemBytes();
    const bool fp64 = prec == MTD_PREC_FP64;
    const bool x3 = prec == MTD_PREC_FP32;
    if (adjoint) {  // FP64, or FP32 with split-TF32 (FP32-accurate) products
        if (fp64 && vec2) persistent_kernel<2, double, 1, true><<<grid, kThreads, bytes, s>>>(a);
        else if (fp64) persistent_kernel<1, double, 1, true><<<grid, kThreads, bytes, s>>>(a);
        else if (vec2) persistent_kernel<2, float, 3, true><<<grid, kThreads, bytes, s>>>(a);
        else persistent_kernel<1, float, 3, true><<<grid, kThreads, bytes, s>>>(a);
        return cudaGetLastError() == cudaSuccess ? MTD_OK : MTD_ERR_CUDA;
    }
    if (fp64 && vec2 && a.tma64) persistent_kernel<2, double, 1, false, true><<<grid, kThreads, bytes, s>>>(a);
    else if (fp64 && vec2 && a.opset == kOpsCholesky)
        persistent_kernel<2, double, 1, false, false, false, kOpsCholesky><<<grid, kThreads, bytes, s>>>(a);
    else if (fp64 && vec2 && a.opset == kOpsLu)
        persistent_kernel<2, double, 1, false, false, false, kOpsLu><<<grid, kThreads, bytes, s>>>(a);
    else if (fp64 && vec2) persistent_kernel<2, double><<<grid, kThreads, bytes, s>>>(a);
    else if (fp64) persistent_kernel<1, double><<<grid, kThreads, bytes, s>>>(a);
    else if (x3 && vec2) persistent_kernel<2, float, 3><<<grid, kThreads, bytes, s>>>(a);
    else if (x3) persistent_kernel<1, float, 3><<<grid, kThreads, bytes, s>>>(a);
    else if (vec2) persistent_kernel<2, float><<<grid, kThreads, bytes, s>>>(a);
    else persistent_kernel<1, float><<<grid, kThreads, bytes, s>>>(a);
    return cudaGetLastError() == cudaSuccess ? MTD_OK : MTD_ERR_CUDA;
}

}  // namespace mtd

static int run_persistent(mtd_graph *g, void *dA, int64_t lda, void *stream, int *info_out) {
    if (!g || !dA) return MTD_ERR_INVALID_ARG;
    if (!g->finalized) return MTD_ERR_STATE;
    if (lda < g->dag.n()) return MTD_ERR_INVALID_ARG;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev != g->device) return MTD_ERR_STATE;
    cudaStream_t s = static_cast<cudaStream_t>(stream);

    RunArgs a = make_args(g, dA, lda);
    const bool vec2 = use_vec2(g, dA, lda);
    // TF32 runs feed their tcgen05 GEMM items with TMA when every item's rows start on a
    // 32-row atom (tile and nested sub-tile edges multiples of 32); updates whose depth is
    // not a whole number of 64-column stages use the cp.async path
    const bool tf32_items = g->prec == MTD_PREC_TF32 || g->prec == MTD_PREC_BF16;
    if (tf32_items && vec2 && g->dag.unit() % 32 == 0 && g->nest % 32 == 0) mtd::encode_tmap(a, dA, g->dag.n(), lda);
    // BF16 updates read the BF16 copy by TMA when every item's rows start on a 64-row atom;
    // the others keep the TF32 path on the FP32 matrix
    if (g->prec == MTD_PREC_BF16 && vec2 && g->dag.unit() % 64 == 0 && g->nest % 64 == 0)
        mtd::encode_tmap_bf16(a, g->d_bf16, g->dag.n(), g->bf16_ld);
    // FP32-accurate runs: the three-pass tcgen05 updates read the matrix and its low parts by
    // TMA (boxes of 32-deep slices); the TRSM items write the low parts only then
    if (g->prec == MTD_PREC_FP32 && g->d_lo && vec2 && g->dag.n() % 32 == 0 &&
        mtd::encode_f32_3d(a.tmap, dA, g->dag.n(), lda, tc::kX3BK) &&
        mtd::encode_f32_3d(a.tmap_lo, g->d_lo, g->dag.n(), g->lo_ld, tc::kX3BK)) {
        a.tma = tc::kTmaMap3D;
        a.lo = g->d_lo;
        a.lo_ld = g->lo_ld;
        a.tma_lo = 1;
    }
    // FP64 GEMM / SYRK items read their operands by TMA when every operand block starts on a
    // 16-row atom (tile and nested sub-tile edges multiples of 16)
    if (g->prec == MTD_PREC_FP64 && vec2 && g->dag.unit() % 16 == 0 && g->nest % 16 == 0 && g->use_tma64)
        mtd::encode_tmap64(a, dA, g->dag.n(), lda);
    const int grid = g->num_sms;
    g->last_grid = grid;
    a.opset = g->opset;
    const int rc = launch_run(a, g->d_deps_init, g->d_roots, g->n_roots, g->total_items, g->prec, vec2, grid, s,
                              false);
    if (rc) return rc;
    if (cudaMemcpyAsync(g->h_ctl, g->d_ctl, sizeof(RunCtl), cudaMemcpyDeviceToHost, s) != cudaSuccess)
        return MTD_ERR_CUDA;
    g->last_stream = s;
    g->run_pending = true;
    g->last_was_graph = false;
    if (info_out) return mtd_graph_status(g, info_out);
    return MTD_OK;
}

extern "C" {

int mtd_run(mtd_graph *g, double *dA, int64_t lda, void *stream, int *info_out) {
    if (g && g->prec != MTD_PREC_FP64) return MTD_ERR_STATE;
    return run_persistent(g, dA, lda, stream, info_out);
}

int mtd_run_f32(mtd_graph *g, float *dA, int64_t lda, void *stream, int *info_out) {
    if (g && g->prec == MTD_PREC_FP64) return MTD_ERR_STATE;
    return run_persistent(g, dA, lda, stream, info_out);
}

int mtd_graph_set_precision(mtd_graph *g, int prec) {
    if (!g || (prec != MTD_PREC_FP64 && prec != MTD_PREC_TF32 && prec != MTD_PREC_FP32 && prec != MTD_PREC_BF16))
        return MTD_ERR_INVALID_ARG;
    if (g->finalized) return MTD_ERR_STATE;
    g->prec = prec;
    return MTD_OK;
}

int mtd_run_graph(mtd_graph *g, double *dA, int64_t lda, void *stream, int *info_out) {
    if (!g || !dA) return MTD_ERR_INVALID_ARG;
    if (g->prec != MTD_PREC_FP64) return MTD_ERR_STATE;
    if (!g->finalized) return MTD_ERR_STATE;
    if (lda < g->dag.n()) return MTD_ERR_INVALID_ARG;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev != g->device) return MTD_ERR_STATE;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (!g->cexec || g->cgraph_a != dA || g->cgraph_lda != lda) {
        const int rc = build_cgraph(g, dA, lda);
        if (rc) {
            release_cgraph(g);
            return rc;
        }
    }
    if (cudaGraphLaunch(g->cexec, s) != cudaSuccess) return MTD_ERR_CUDA;
    if (cudaMemcpyAsync(g->h_ctl, g->d_ctl, sizeof(RunCtl), cudaMemcpyDeviceToHost, s) != cudaSuccess)
        return MTD_ERR_CUDA;
    g->last_stream = s;
    g->run_pending = true;
    g->last_was_graph = true;
    g->last_grid = 0;
    if (info_out) return mtd_graph_status(g, info_out);
    return MTD_OK;
}

int mtd_graph_status(mtd_graph *g, int *info_out) {
    if (!g) return MTD_ERR_INVALID_ARG;
    if (info_out) *info_out = 0;
    if (!g->run_pending) return MTD_ERR_STATE;
    if (cudaStreamSynchronize(g->last_stream) != cudaSuccess) return MTD_ERR_CUDA;
    const RunCtl &c = *g->h_ctl;
    if (info_out) *info_out = (c.error != 0 && c.info != 0x7fffffff) ? c.info : 0;
    if (c.error) return c.error;
    if (!g->last_was_graph && c.tasks_done != g->n_dev) return MTD_ERR_TIMEOUT;
    return MTD_OK;
}

int mtd_graph_last_stats(mtd_graph *g, mtd_run_stats *out) {
    if (!g || !out) return MTD_ERR_INVALID_ARG;
    if (!g->run_pending) return MTD_ERR_STATE;
    if (cudaStreamSynchronize(g->last_stream) != cudaSuccess) return MTD_ERR_CUDA;
    out->tasks = g->h_ctl->tasks_done;
    out->items = static_cast<int64_t>(g->h_ctl->items_done);
    out->ctas = g->last_grid;
    out->busy_fraction = -1.0;
    out->span_ms = -1.0;
    if (g->trace && g->d_trace) {
        const long long n = std::min<long long>(static_cast<long long>(g->h_ctl->items_done), g->trace_cap);
        std::vector<unsigned long long> rec(size_t(4 * std::max<long long>(n, 1)));
        if (n > 0 && cudaMemcpy(rec.data(), g->d_trace, size_t(4 * n) * sizeof(unsigned long long),
                                cudaMemcpyDeviceToHost) != cudaSuccess)
            return MTD_ERR_CUDA;
        if (n > 0) {
            unsigned long long lo = ~0ull, hi = 0;
            double busy = 0.0;
            for (long long i = 0; i < n; ++i) {
                lo = std::min(lo, rec[4 * i]);
                hi = std::max(hi, rec[4 * i + 1]);
                busy += double(rec[4 * i + 1] - rec[4 * i]);
            }
            const double span = double(hi - lo);
            out->span_ms = span * 1e-6;
            out->busy_fraction = span > 0 ? busy / (span * g->last_grid) : 0.0;
        }
    }
    return MTD_OK;
}

// Raw trace of the last run: 4 words per work item (start ns, end ns, SM id,
// task << 32 | item).  Returns the number of records copied.
long long mtd_graph_copy_trace(mtd_graph *g, unsigned long long *out, long long cap_records) {
    if (!g || !out || cap_records < 0) return -MTD_ERR_INVALID_ARG;
    if (!g->trace || !g->run_pending) return -MTD_ERR_STATE;
    if (cudaStreamSynchronize(g->last_stream) != cudaSuccess) return -MTD_ERR_CUDA;
    const long long n = std::min(std::min<long long>(static_cast<long long>(g->h_ctl->items_done), g->trace_cap), cap_records);
    if (n > 0 && cudaMemcpy(out, g->d_trace, size_t(4 * n) * sizeof(unsigned long long), cudaMemcpyDeviceToHost) !=
                     cudaSuccess)
        return -MTD_ERR_CUDA;
    return n;
}

int mtd_graph_destroy(mtd_graph *g) {
    if (!g) return MTD_ERR_INVALID_ARG;
    if (g->run_pending && g->last_stream != nullptr) cudaStreamSynchronize(g->last_stream);
    else if (g->run_pending) cudaDeviceSynchronize();
    release_cgraph(g);
    if (g->finalized) release_device(g);
    delete g;
    return MTD_OK;
}

static int tiled_driver(int kind, double *dA, int64_t n, int64_t lda, int64_t tile, void *stream, int *info_out) {
    mtd_graph *g = nullptr;
    int rc = mtd_graph_create(&g, kind, n, tile);
    if (rc) return rc;
    rc = mtd_graph_build_tiled(g);
    if (!rc) rc = mtd_graph_finalize(g);
    int info = 0;
    if (!rc) rc = mtd_run(g, dA, lda, stream, &info);
    if (info_out) *info_out = info;
    mtd_graph_destroy(g);
    return rc;
}

int mtd_tiled_cholesky(double *dA, int64_t n, int64_t lda, int64_t tile, void *stream, int *info_out) {
    return tiled_driver(MTD_KIND_CHOLESKY, dA, n, lda, tile, stream, info_out);
}

int mtd_tiled_lu(double *dA, int64_t n, int64_t lda, int64_t tile, void *stream, int *info_out) {
    return tiled_driver(MTD_KIND_LU, dA, n, lda, tile, stream, info_out);
}

}  // extern "C"

namespace {

// Per-device set-up of mtd_factor_noalloc, done by the first call on each device: in host
// code the array's name is only a host-side stand-in, so its device address comes from
// cudaGetSymbolAddress with that device current.
int noalloc_scratch(int device, unsigned char **out) {
    static std::mutex mu;
    static unsigned char *addr[64] = {nullptr};
    if (device < 0 || device >= 64) return MTD_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> lock(mu);
    if (!addr[device]) {
        void *p = nullptr;
        if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || p == nullptr) {
            cudaGetLastError();
            return MTD_ERR_CUDA;
        }
        addr[device] = static_cast<unsigned char *>(p);
    }
    int rc = smem_setup<2>(device);
    if (!rc) rc = smem_setup<1>(device);
    if (rc) return rc;
    *out = addr[device];
    return MTD_OK;
}

// Bump allocation inside the fixed scratch (256-byte aligned pieces).
struct ScratchCarver {
    unsigned char *base;
    size_t used = 0;
    template <typename T>
    T *take(size_t count) {
        used = (used + 255) & ~size_t(255);
        T *p = reinterpret_cast<T *>(base + used);
        used += (count ? count : 1) * sizeof(T);
        return p;
    }
};

}  // namespace

extern "C" int mtd_factor_noalloc(int kind, double *dA, int64_t n, int64_t lda, int64_t tile, void *stream,
                                  int *info_out) {
    if (info_out) *info_out = 0;
    if (kind != MTD_KIND_LU && kind != MTD_KIND_CHOLESKY) return MTD_ERR_INVALID_ARG;
    if (!dA || n <= 0 || tile <= 0 || tile > n || lda < n) return MTD_ERR_INVALID_ARG;
    if (n > kNoAllocMaxN) return MTD_ERR_TOO_LARGE;
    // Every host task becomes at least one device task: reject a tile so small that the
    // task list alone exceeds the task table before building anything (the count is cubic
    // in the tile count).
    if (Dag::reference_task_count(kind, (n + tile - 1) / tile) > kNoAllocMaxTasks) return MTD_ERR_TOO_LARGE;

    // The task graph: host memory only.
    Dag dag(kind, n, tile);
    int rc = dag.build_reference_order();
    if (rc) return rc;
    Lowered low;
    rc = dag.lower(kNestTile, low);
    if (rc) return rc;
    const int nt = static_cast<int>(low.tasks.size());
    long long items = 0;
    for (int q = 0; q < kNumQueues; ++q) items += low.queue_cap[q];
    if (nt > kNoAllocMaxTasks || static_cast<long long>(low.succ.size()) > kNoAllocMaxEdges ||
        items > kNoAllocMaxItems)
        return MTD_ERR_TOO_LARGE;
    std::vector<int> deps_init(nt), roots;
    for (int t = 0; t < nt; ++t) {
        deps_init[t] = static_cast<int>(low.preds[t].size());
        if (deps_init[t] == 0) roots.push_back(t);
    }
    if (roots.empty()) return MTD_ERR_BAD_DAG;

    int device = 0, sms = 0;
    rc = check_device(&device, &sms);
    if (rc) return rc;
    unsigned char *scratch = nullptr;
    rc = noalloc_scratch(device, &scratch);
    if (rc) return rc;

    const int64_t wld = ws_ld_for(n);
    ScratchCarver sc{scratch};
    RunArgs a{};
    DevTask *d_tasks = sc.take<DevTask>(nt);
    int *d_succ = sc.take<int>(low.succ.size());
    int *d_deps_init = sc.take<int>(nt);
    int *d_roots = sc.take<int>(roots.size());
    a.deps = sc.take<int>(nt);
    a.items_left = sc.take<int>(nt);
    for (int q = 0; q < kNumQueues; ++q) {
        a.queue[q] = sc.take<unsigned long long>(size_t(low.queue_cap[q]));
        a.queue_cap[q] = low.queue_cap[q];
    }
    a.qctl = sc.take<QueueCtl>(kNumQueues);
    a.ctl = sc.take<RunCtl>(1);
    a.ws_lower = sc.take<double>(size_t(wld) * kNB);
    a.ws_upper = kind == MTD_KIND_LU ? sc.take<double>(size_t(wld) * kNB) : nullptr;
    if (sc.used > kNoAllocBytes) return MTD_ERR_TOO_LARGE;
    a.a = dA;
    a.lda = lda;
    a.n_tasks = nt;
    a.tasks = d_tasks;
    a.succ = d_succ;
    a.ws_ld = wld;
    a.trace = nullptr;
    a.trace_cap = 0;
    a.timeout_ns = 10ull * 1000000000ull;

    cudaStream_t s = static_cast<cudaStream_t>(stream);
    bool ok = cudaMemcpyAsync(d_tasks, low.tasks.data(), nt * sizeof(DevTask), cudaMemcpyHostToDevice, s) ==
              cudaSuccess;
    ok = ok && (low.succ.empty() || cudaMemcpyAsync(d_succ, low.succ.data(), low.succ.size() * sizeof(int),
                                                    cudaMemcpyHostToDevice, s) == cudaSuccess);
    ok = ok && cudaMemcpyAsync(d_deps_init, deps_init.data(), nt * sizeof(int), cudaMemcpyHostToDevice, s) ==
                   cudaSuccess;
    ok = ok && cudaMemcpyAsync(d_roots, roots.data(), roots.size() * sizeof(int), cudaMemcpyHostToDevice, s) ==
                   cudaSuccess;
    if (!ok) return MTD_ERR_CUDA;
    // reset_kernel zeroes the counters and control block and empties the queues, so
    // nothing left in the array by an earlier call leaks into this one; the inverse
    // workspace is always written by a diagonal factorisation before it is read.
    const bool vec2 = (reinterpret_cast<uintptr_t>(dA) % 16 == 0) && (lda % 2 == 0) && (tile % 2 == 0) &&
                      (n % 2 == 0);
    const int reset_blocks =
        static_cast<int>(std::min<long long>(1024, (std::max<long long>(items, nt) + kThreads - 1) / kThreads));
    reset_kernel<<<std::max(reset_blocks, 1), kThreads, 0, s>>>(a, d_deps_init);
    seed_kernel<<<1, kSeedThreads, 0, s>>>(a, d_roots, static_cast<int>(roots.size()));
    const int opset = opset_of(low.tasks);
    if (vec2 && opset == kOpsCholesky)
        persistent_kernel<2, double, 1, false, false, false, kOpsCholesky><<<sms, kThreads, kOpSmemBytes(), s>>>(a);
    else if (vec2 && opset == kOpsLu)
        persistent_kernel<2, double, 1, false, false, false, kOpsLu><<<sms, kThreads, kOpSmemBytes(), s>>>(a);
    else if (vec2) persistent_kernel<2, double><<<sms, kThreads, kOpSmemBytes(), s>>>(a);
    else persistent_kernel<1, double><<<sms, kThreads, kOpSmemBytes(), s>>>(a);
    if (cudaGetLastError() != cudaSuccess) return MTD_ERR_CUDA;
    RunCtl c;
    if (cudaMemcpyAsync(&c, a.ctl, sizeof(RunCtl), cudaMemcpyDeviceToHost, s) != cudaSuccess) return MTD_ERR_CUDA;
    if (cudaStreamSynchronize(s) != cudaSuccess) return MTD_ERR_CUDA;
    if (info_out) *info_out = (c.error != 0 && c.info != 0x7fffffff) ? c.info : 0;
    if (c.error) return c.error;
    if (c.tasks_done != nt) return MTD_ERR_TIMEOUT;
    return MTD_OK;
}

// Internal accessors for the solver (mustard_b200/csrc/solver.cu): the inverse diagonal
// blocks a finalised graph's last run left in its workspace.
namespace mtd {
void *graph_ws_lower(mtd_graph *g) { return g ? g->d_ws_lower : nullptr; }
int64_t graph_ws_ld(mtd_graph *g) { return g ? ws_ld(g) : 0; }
}  // namespace mtd
