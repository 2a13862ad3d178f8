// Blocked Cholesky adjoint on the persistent scheduler.
//
// No counterpart in the reference.  The reverse sweep of the tiled Cholesky (operations in
// adjoint_ops.cuh) becomes a task graph over the same tiles, built here with explicit
// read / write sets per task (last-writer, write-after-read and write-after-write edges);
// the graphs of many matrices are concatenated into one launch, each task tagged with its
// matrix's entries in the run's matrix table.  The inverses of L's 64 x 64 diagonal
// blocks, which the reverse triangular solves and the diagonal adjoints use, are computed
// from L by a small kernel in front of the sweep, so the adjoint needs only L and Lbar
// (whether L was kept from the forward pass or recomputed).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <map>
#include <new>
#include <vector>

#include "../../include/mustard_b200.h"
#include "device_types.hpp"
#include "tile_ops.cuh"

namespace mtd {
int launch_run(const RunArgs &a, const int *deps_init, const int *roots, int n_roots, long long total_items,
               int prec, bool vec2, int grid, cudaStream_t s, bool adjoint);
}
using namespace mtd;

struct mtd_adjoint {
    int count = 0;
    int prec = MTD_PREC_FP64;
    int sms = 148;
    std::vector<int64_t> n, tile, ws_off, ws_ld, y_off, y_ld;
    int64_t max_blocks = 0;  // 64-row diagonal blocks of the largest matrix
    int n_dev = 0, n_roots = 0;
    long long total_items = 0;
    long long qcap[kNumQueues] = {0, 0};
    DevTask *d_tasks = nullptr;
    int *d_succ = nullptr, *d_deps_init = nullptr, *d_deps = nullptr, *d_items_left = nullptr, *d_roots = nullptr;
    unsigned long long *d_queue[kNumQueues] = {nullptr, nullptr};
    QueueCtl *d_qctl = nullptr;
    RunCtl *d_ctl = nullptr;
    RunCtl *h_ctl = nullptr;     // pinned
    unsigned char *d_ws = nullptr;
    unsigned char *d_y = nullptr;
    BatchMat *d_mats = nullptr;  // 3 per matrix: adjoint, factor, Y
    BatchMat *h_mats = nullptr;  // pinned staging
    int *d_info = nullptr;
    unsigned long long *d_done = nullptr;
    unsigned long long *d_trace = nullptr;  // per-item records when tracing (4 words each)
    std::vector<int> task_op;               // op of each device task (for trace readers)
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    cudaStream_t last_stream = nullptr;
    bool pending = false;
};

namespace {

constexpr int kInvThreads = 256;

size_t adj_elem(const mtd_adjoint *a) { return a->prec == MTD_PREC_FP64 ? sizeof(double) : sizeof(float); }

// W = inverse of each 64 x 64 diagonal block of L, for every matrix (grid (blocks, count)).
template <typename T>
__global__ void __launch_bounds__(kInvThreads) adjoint_inverse_kernel(const BatchMat *mats, T *ws) {
    __shared__ T X[kNB * kDiagLd];
    const BatchMat &lm = mats[3 * blockIdx.y + 1];
    const BatchMat &ym = mats[3 * blockIdx.y + 2];
    const int64_t r0 = int64_t(blockIdx.x) * kNB;
    const int64_t n = ym.ws_ld;  // the Y entry carries n in its ws_ld slot
    if (r0 >= n) return;
    const int jn = static_cast<int>(min(int64_t(kNB), n - r0));
    const T *L = static_cast<const T *>(lm.a) + r0 + r0 * lm.lda;
    const int64_t ldl = lm.lda;
    lower_inverse<false>(jn, [&](int i, int l) { return L[i + int64_t(l) * ldl]; }, X);
    T *W = ws + lm.ws_off + r0;
    for (int e = threadIdx.x; e < kNB * kNB; e += kInvThreads) {
        const int r = e % kNB, c = e / kNB;
        if (r < jn) W[r + int64_t(c) * lm.ws_ld] = c < jn ? X[r + c * kDiagLd] : T(0);
    }
}

// Read / write sets of the adjoint's tasks: tiles (i, j), i >= j, of the adjoint, and the
// Y block of diagonal tile j as key (-1 - j, 0).  The factor is read-only and needs none.
using Key = std::pair<int, int>;

struct GraphBuilder {
    std::vector<DevTask> tasks;
    std::vector<std::vector<int>> preds;
    std::map<Key, int> last_writer;
    std::map<Key, std::vector<int>> readers;

    int add(const DevTask &d, const std::vector<Key> &reads, const std::vector<Key> &writes) {
        const int id = static_cast<int>(tasks.size());
        std::vector<int> dep;
        for (const Key &k : reads) {
            auto it = last_writer.find(k);
            if (it != last_writer.end()) dep.push_back(it->second);
        }
        for (const Key &k : writes) {
            auto it = last_writer.find(k);
            if (it != last_writer.end()) dep.push_back(it->second);
            auto rd = readers.find(k);
            if (rd != readers.end())
                for (int r : rd->second) dep.push_back(r);
        }
        std::sort(dep.begin(), dep.end());
        dep.erase(std::unique(dep.begin(), dep.end()), dep.end());
        dep.erase(std::remove(dep.begin(), dep.end(), id), dep.end());
        for (const Key &k : reads) readers[k].push_back(id);
        for (const Key &k : writes) {
            last_writer[k] = id;
            readers[k].clear();
        }
        tasks.push_back(d);
        preds.push_back(dep);
        return id;
    }
};

int64_t cdiv(int64_t a, int64_t b) { return (a + b - 1) / b; }

DevTask adj_task(int op, int queue, int64_t cr, int64_t cc, int64_t ar, int64_t ac, int64_t br, int64_t bc, int64_t m,
                 int64_t n, int64_t k, int pad, int mat) {
    DevTask d{};
    d.op = op;
    d.queue = queue;
    d.cr = static_cast<int32_t>(cr);
    d.cc = static_cast<int32_t>(cc);
    d.ar = static_cast<int32_t>(ar);
    d.ac = static_cast<int32_t>(ac);
    d.br = static_cast<int32_t>(br);
    d.bc = static_cast<int32_t>(bc);
    d.m = static_cast<int32_t>(m);
    d.n = static_cast<int32_t>(n);
    d.k = static_cast<int32_t>(k);
    d.pad = pad;
    d.mat = mat;
    switch (op) {
    case kOpAdjTrsm: d.n_items = static_cast<int32_t>(cdiv(m, kPanelRows)); break;
    case kOpAdjPotrf: d.n_items = 1; break;
    default: d.n_items = static_cast<int32_t>(cdiv(m, kGemmTile) * cdiv(n, kGemmTile)); break;
    }
    return d;
}

// The reverse sweep of one n x n matrix with tile t (block columns j = nb-1 .. 0).
void build_matrix(GraphBuilder &g, int64_t n, int64_t t, int mat) {
    const int nb = static_cast<int>(cdiv(n, t));
    auto ext = [&](int i) { return std::min<int64_t>(t, n - int64_t(i) * t); };
    for (int j = nb - 1; j >= 0; --j) {
        const int64_t jt = int64_t(j) * t, ej = ext(j), lo = jt + ej, below = n - lo;
        std::vector<Key> colj;
        for (int i = j + 1; i < nb; ++i) colj.push_back({i, j});
        if (below > 0) {
            g.add(adj_task(kOpAdjTrsm, 0, lo, jt, jt, jt, 0, 0, below, ej, 0, 0, mat), colj, colj);
            std::vector<Key> rd = colj;
            rd.push_back({j, j});
            g.add(adj_task(kOpAdjGemmTN, 0, jt, jt, lo, jt, lo, jt, ej, ej, below, 1, mat), rd, {{j, j}});
        }
        g.add(adj_task(kOpAdjPotrf, 0, jt, jt, jt, jt, 0, 0, ej, ej, ej, 0, mat), {{j, j}}, {{j, j}, {-1 - j, 0}});
        for (int k = 0; k < j; ++k) {
            const int64_t kt = int64_t(k) * t, ek = ext(k);
            const int q = k == j - 1 ? 0 : 1;  // updates of the next block column: critical path
            if (below > 0) {
                std::vector<Key> colk, rd = colj;
                for (int i = j + 1; i < nb; ++i) colk.push_back({i, k});
                rd.insert(rd.end(), colk.begin(), colk.end());
                g.add(adj_task(kOpAdjGemmNN, q, lo, kt, lo, jt, jt, kt, below, ek, ej, 0, mat), rd, colk);
                std::vector<Key> rd2 = colj;
                rd2.push_back({j, k});
                g.add(adj_task(kOpAdjGemmTN, q, jt, kt, lo, jt, lo, kt, ej, ek, below, 0, mat), rd2, {{j, k}});
            }
            g.add(adj_task(kOpAdjGemmNN, q, jt, kt, jt, 0, jt, kt, ej, ek, ej, 2, mat), {{-1 - j, 0}, {j, k}},
                  {{j, k}});
        }
    }
}

template <typename P>
int dalloc(P **p, size_t count) {
    if (cudaMalloc(reinterpret_cast<void **>(p), std::max<size_t>(count, 1) * sizeof(P)) != cudaSuccess) {
        *p = nullptr;
        return MTD_ERR_OUT_OF_MEMORY;
    }
    return MTD_OK;
}

void release(mtd_adjoint *a) {
    cudaFree(a->d_tasks);
    cudaFree(a->d_succ);
    cudaFree(a->d_deps_init);
    cudaFree(a->d_deps);
    cudaFree(a->d_items_left);
    cudaFree(a->d_roots);
    for (int q = 0; q < kNumQueues; ++q) cudaFree(a->d_queue[q]);
    cudaFree(a->d_qctl);
    cudaFree(a->d_ctl);
    cudaFree(a->d_ws);
    cudaFree(a->d_y);
    cudaFree(a->d_mats);
    cudaFree(a->d_info);
    cudaFree(a->d_done);
    cudaFree(a->d_trace);
    if (a->h_ctl) cudaFreeHost(a->h_ctl);
    if (a->h_mats) cudaFreeHost(a->h_mats);
    if (a->ev0) cudaEventDestroy(a->ev0);
    if (a->ev1) cudaEventDestroy(a->ev1);
}

}  // namespace

extern "C" {

int mtd_adjoint_create(mtd_adjoint **out, int count, const int64_t *n, int64_t tile, int prec) {
    if (!out) return MTD_ERR_INVALID_ARG;
    *out = nullptr;
    if (count <= 0 || !n || (tile != 64 && tile != 128 && tile != 256) ||
        (prec != MTD_PREC_FP64 && prec != MTD_PREC_FP32))
        return MTD_ERR_INVALID_ARG;
    int dev = 0, major = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return MTD_ERR_NO_DEVICE;
    cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev);
    if (major != 10) return MTD_ERR_NO_DEVICE;
    mtd_adjoint *a = new (std::nothrow) mtd_adjoint();
    if (!a) return MTD_ERR_OUT_OF_MEMORY;
    a->count = count;
    a->prec = prec;
    cudaDeviceGetAttribute(&a->sms, cudaDevAttrMultiProcessorCount, dev);
    GraphBuilder g;
    int64_t ws_total = 0, y_total = 0;
    int rc = MTD_OK;
    for (int m = 0; m < count; ++m) {
        const int64_t nm = n[m];
        if (nm <= 0 || nm > (int64_t(1) << 20)) {
            rc = MTD_ERR_INVALID_ARG;
            break;
        }
        const int64_t ld = (nm + 3) & ~int64_t(3);
        a->n.push_back(nm);
        a->tile.push_back(std::min<int64_t>(tile, nm));
        a->ws_off.push_back(ws_total);
        a->ws_ld.push_back(ld);
        ws_total += ld * kNB;
        a->y_off.push_back(y_total);
        a->y_ld.push_back(ld);
        y_total += ld * tile;
        a->max_blocks = std::max(a->max_blocks, cdiv(nm, kNB));
        GraphBuilder one;  // tile keys are per matrix: the matrices share no dependency
        build_matrix(one, nm, tile, 3 * m);
        const int base = static_cast<int>(g.tasks.size());
        for (size_t t = 0; t < one.tasks.size(); ++t) {
            g.tasks.push_back(one.tasks[t]);
            std::vector<int> p = one.preds[t];
            for (int &x : p) x += base;
            g.preds.push_back(std::move(p));
        }
    }
    const int nt = static_cast<int>(g.tasks.size());
    std::vector<int> succ, deps_init(nt), roots;
    if (!rc) {
        std::vector<std::vector<int>> succs(nt);
        for (int t = 0; t < nt; ++t) {
            deps_init[t] = static_cast<int>(g.preds[t].size());
            if (g.preds[t].empty()) roots.push_back(t);
            for (int p : g.preds[t]) succs[p].push_back(t);
        }
        for (int t = 0; t < nt; ++t) {
            g.tasks[t].succ_begin = static_cast<int32_t>(succ.size());
            g.tasks[t].succ_count = static_cast<int32_t>(succs[t].size());
            succ.insert(succ.end(), succs[t].begin(), succs[t].end());
            a->qcap[g.tasks[t].queue] += g.tasks[t].n_items;
        }
        if (roots.empty()) rc = MTD_ERR_BAD_DAG;
    }
    a->n_dev = nt;
    a->n_roots = static_cast<int>(roots.size());
    a->total_items = a->qcap[0] + a->qcap[1];
    for (const DevTask &d : g.tasks) a->task_op.push_back(d.op);
    if (!rc) rc = dalloc(&a->d_tasks, nt);
    if (!rc) rc = dalloc(&a->d_succ, succ.size());
    if (!rc) rc = dalloc(&a->d_deps_init, nt);
    if (!rc) rc = dalloc(&a->d_deps, nt);
    if (!rc) rc = dalloc(&a->d_items_left, nt);
    if (!rc) rc = dalloc(&a->d_roots, roots.size());
    for (int q = 0; q < kNumQueues && !rc; ++q) rc = dalloc(&a->d_queue[q], size_t(a->qcap[q]));
    if (!rc) rc = dalloc(&a->d_qctl, kNumQueues);
    if (!rc) rc = dalloc(&a->d_ctl, 1);
    if (!rc) rc = dalloc(&a->d_ws, size_t(ws_total) * adj_elem(a));
    if (!rc) rc = dalloc(&a->d_y, size_t(y_total) * adj_elem(a));
    if (!rc) rc = dalloc(&a->d_mats, size_t(3) * count);
    if (!rc) rc = dalloc(&a->d_info, size_t(3) * count);
    if (!rc) rc = dalloc(&a->d_done, size_t(3) * count);
    if (!rc && cudaMallocHost(reinterpret_cast<void **>(&a->h_ctl), sizeof(RunCtl)) != cudaSuccess)
        rc = MTD_ERR_OUT_OF_MEMORY;
    if (!rc && cudaMallocHost(reinterpret_cast<void **>(&a->h_mats), 3 * count * sizeof(BatchMat)) != cudaSuccess)
        rc = MTD_ERR_OUT_OF_MEMORY;
    if (!rc && (cudaEventCreate(&a->ev0) != cudaSuccess || cudaEventCreate(&a->ev1) != cudaSuccess)) rc = MTD_ERR_CUDA;
    if (!rc) {
        bool ok = cudaMemcpy(a->d_tasks, g.tasks.data(), nt * sizeof(DevTask), cudaMemcpyHostToDevice) == cudaSuccess;
        ok = ok && (succ.empty() ||
                    cudaMemcpy(a->d_succ, succ.data(), succ.size() * sizeof(int), cudaMemcpyHostToDevice) == cudaSuccess);
        ok = ok && cudaMemcpy(a->d_deps_init, deps_init.data(), nt * sizeof(int), cudaMemcpyHostToDevice) == cudaSuccess;
        ok = ok && cudaMemcpy(a->d_roots, roots.data(), roots.size() * sizeof(int), cudaMemcpyHostToDevice) == cudaSuccess;
        ok = ok && cudaMemset(a->d_ctl, 0, sizeof(RunCtl)) == cudaSuccess;
        ok = ok && cudaMemset(a->d_y, 0, size_t(y_total) * adj_elem(a)) == cudaSuccess;
        if (!ok) rc = MTD_ERR_CUDA;
    }
    if (rc) {
        release(a);
        delete a;
        return rc;
    }
    std::memset(a->h_ctl, 0, sizeof(RunCtl));
    *out = a;
    return MTD_OK;
}

int mtd_adjoint_num_tasks(const mtd_adjoint *a) { return a ? a->n_dev : -MTD_ERR_INVALID_ARG; }

int mtd_adjoint_run(mtd_adjoint *a, void *const *dL, const int64_t *ldl, void *const *dLbar, const int64_t *ldlb,
                    void *stream) {
    if (!a || !dL || !ldl || !dLbar || !ldlb) return MTD_ERR_INVALID_ARG;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const size_t es = adj_elem(a);
    const int64_t epc = 16 / static_cast<int64_t>(es);
    bool vec2 = true;
    for (int m = 0; m < a->count; ++m) {
        if (!dL[m] || !dLbar[m] || ldl[m] < a->n[m] || ldlb[m] < a->n[m] || dL[m] == dLbar[m])
            return MTD_ERR_INVALID_ARG;
        void *y = a->d_y + size_t(a->y_off[m]) * es;
        a->h_mats[3 * m] = BatchMat{dLbar[m], ldlb[m], a->ws_off[m], a->ws_ld[m]};
        a->h_mats[3 * m + 1] = BatchMat{dL[m], ldl[m], a->ws_off[m], a->ws_ld[m]};
        a->h_mats[3 * m + 2] = BatchMat{y, a->y_ld[m], a->ws_off[m], a->n[m]};
        vec2 = vec2 && reinterpret_cast<uintptr_t>(dL[m]) % 16 == 0 && reinterpret_cast<uintptr_t>(dLbar[m]) % 16 == 0 &&
               ldl[m] % epc == 0 && ldlb[m] % epc == 0 && a->n[m] % epc == 0 && a->tile[m] % epc == 0;
    }
    if (cudaMemcpyAsync(a->d_mats, a->h_mats, 3 * a->count * sizeof(BatchMat), cudaMemcpyHostToDevice, s) !=
            cudaSuccess ||
        cudaMemsetAsync(a->d_done, 0, 3 * a->count * sizeof(unsigned long long), s) != cudaSuccess ||
        cudaEventRecord(a->ev0, s) != cudaSuccess)
        return MTD_ERR_CUDA;
    const dim3 ig(static_cast<unsigned>(a->max_blocks), static_cast<unsigned>(a->count));
    if (a->prec == MTD_PREC_FP64)
        adjoint_inverse_kernel<double><<<ig, kInvThreads, 0, s>>>(a->d_mats, reinterpret_cast<double *>(a->d_ws));
    else
        adjoint_inverse_kernel<float><<<ig, kInvThreads, 0, s>>>(a->d_mats, reinterpret_cast<float *>(a->d_ws));
    if (cudaGetLastError() != cudaSuccess) return MTD_ERR_CUDA;
    RunArgs r{};
    r.n_tasks = a->n_dev;
    r.tasks = a->d_tasks;
    r.succ = a->d_succ;
    r.deps = a->d_deps;
    r.items_left = a->d_items_left;
    for (int q = 0; q < kNumQueues; ++q) {
        r.queue[q] = a->d_queue[q];
        r.queue_cap[q] = a->qcap[q];
    }
    r.qctl = a->d_qctl;
    r.ctl = a->d_ctl;
    r.ws_lower = a->d_ws;
    r.ws_upper = nullptr;
    r.timeout_ns = 10ull * 1000000000ull;
    r.mats = a->d_mats;
    r.mat_info = a->d_info;
    r.mat_done_ns = a->d_done;
    r.trace = a->d_trace;
    r.trace_cap = a->d_trace ? a->total_items : 0;
    int rc = launch_run(r, a->d_deps_init, a->d_roots, a->n_roots, a->total_items, a->prec, vec2, a->sms, s, true);
    if (rc) return rc;
    if (cudaEventRecord(a->ev1, s) != cudaSuccess ||
        cudaMemcpyAsync(a->h_ctl, a->d_ctl, sizeof(RunCtl), cudaMemcpyDeviceToHost, s) != cudaSuccess)
        return MTD_ERR_CUDA;
    a->last_stream = s;
    a->pending = true;
    return MTD_OK;
}

int mtd_adjoint_status(mtd_adjoint *a, double *elapsed_ms) {
    if (!a) return MTD_ERR_INVALID_ARG;
    if (!a->pending) return MTD_ERR_STATE;
    if (cudaStreamSynchronize(a->last_stream) != cudaSuccess) return MTD_ERR_CUDA;
    if (elapsed_ms) {
        float ms = 0.f;
        if (cudaEventElapsedTime(&ms, a->ev0, a->ev1) != cudaSuccess) return MTD_ERR_CUDA;
        *elapsed_ms = ms;
    }
    if (a->h_ctl->error) return a->h_ctl->error;
    if (a->h_ctl->tasks_done != a->n_dev) return MTD_ERR_TIMEOUT;
    return MTD_OK;
}

int mtd_adjoint_set_trace(mtd_adjoint *a, int enable) {
    if (!a) return MTD_ERR_INVALID_ARG;
    if (cudaDeviceSynchronize() != cudaSuccess) return MTD_ERR_CUDA;
    cudaFree(a->d_trace);
    a->d_trace = nullptr;
    if (enable) return dalloc(&a->d_trace, size_t(4) * size_t(a->total_items));
    return MTD_OK;
}

long long mtd_adjoint_copy_trace(mtd_adjoint *a, unsigned long long *out, long long cap_records) {
    if (!a || !out || cap_records < 0) return -MTD_ERR_INVALID_ARG;
    if (!a->d_trace) return -MTD_ERR_STATE;
    const long long n = std::min<long long>(cap_records, a->total_items);
    if (cudaMemcpy(out, a->d_trace, size_t(n) * 4 * sizeof(unsigned long long), cudaMemcpyDeviceToHost) != cudaSuccess)
        return -MTD_ERR_CUDA;
    return n;
}

int mtd_adjoint_task_op(const mtd_adjoint *a, int task) {
    if (!a || task < 0 || task >= a->n_dev) return -MTD_ERR_INVALID_ARG;
    return a->task_op[task];
}

int mtd_adjoint_destroy(mtd_adjoint *a) {
    if (!a) return MTD_ERR_INVALID_ARG;
    cudaDeviceSynchronize();
    release(a);
    delete a;
    return MTD_OK;
}

int mtd_cholesky_adjoint(int prec, void *dL, int64_t ldl, void *dLbar, int64_t ldlb, int64_t n, int64_t tile,
                         void *stream) {
    mtd_adjoint *a = nullptr;
    int rc = mtd_adjoint_create(&a, 1, &n, tile, prec);
    if (rc) return rc;
    rc = mtd_adjoint_run(a, &dL, &ldl, &dLbar, &ldlb, stream);
    if (!rc) rc = mtd_adjoint_status(a, nullptr);
    mtd_adjoint_destroy(a);
    return rc;
}

}  // extern "C"
