// Pivoted LU (LAPACK's dgetrf semantics: partial pivoting, ipiv 1-based) as a device-side
// task graph on the persistent scheduler.  No counterpart in the reference, which factors
// without pivoting.
//
// Right-looking over block columns of `tile` (T of them).  Step k:
//   PANEL(k)    the m x w panel at (k*tile, k*tile): P cooperating items (lupiv_ops.cuh)
//               choose, apply and record the panel's interchanges and factor it;
//   SWAP(k, j)  the panel's interchanges applied to block column j > k (rows >= k*tile);
//   TRSM(k, j)  U(k, j) = L_kk^-1 A(k, j) (unit lower);
//   GEMM(k, j)  A(k+1:, j) -= L(k+1:, k) U(k, j), one task per block column (its items are
//               128 x 128 output blocks), so the graph holds ~1.5 T^2 tasks.
// After the last panel, LSWAP(j) applies the interchanges of every later panel to block
// column j < T-1 (LAPACK applies them as it goes; the result is the same, and deferring
// them keeps them away from the updates that still read those columns).
// Priorities: the panel, and the swap / solve / update of the next block column, are on the
// critical path (queue 0); the column after it queue 1; the rest queue 2.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <new>
#include <vector>

#include "../../include/mustard_b200.h"
#include "device_types.hpp"

namespace mtd {
int launch_run_solve(const RunArgs &a, const int *deps_init, const int *roots, int n_roots, long long total_items,
                     int prec, bool vec2, int grid, cudaStream_t s);
int ext_op_smem_bytes();
}  // namespace mtd
using namespace mtd;

namespace {

constexpr int kGemmEdge = 128;   // output block of one GEMM work item
constexpr int kTrsmCols = 64;    // columns of one TRSM work item
constexpr int kSwapColsHost = 64;

template <typename T>
int dalloc(T **p, size_t count) {
    if (cudaMalloc(reinterpret_cast<void **>(p), std::max<size_t>(count, 1) * sizeof(T)) != cudaSuccess) {
        cudaGetLastError();
        *p = nullptr;
        return MTD_ERR_OUT_OF_MEMORY;
    }
    return MTD_OK;
}

int64_t ceil_div(int64_t a, int64_t b) { return (a + b - 1) / b; }

}  // namespace

struct mtd_lupiv {
    int64_t n = 0, tile = 0;
    int T = 0, sms = 148, device = 0;
    int n_tasks = 0, n_roots = 0, max_items = 0;
    long long qcap[kNumQueues] = {0, 0, 0};
    long long total_items = 0;
    DevTask *d_tasks = nullptr;
    int *d_succ = nullptr, *d_deps_init = nullptr, *d_deps = nullptr, *d_items_left = nullptr, *d_roots = nullptr;
    unsigned long long *d_queue[kNumQueues] = {nullptr, nullptr, nullptr};
    QueueCtl *d_qctl = nullptr;
    RunCtl *d_ctl = nullptr;
    RunCtl *h_ctl = nullptr;  // pinned
    double *d_ws = nullptr;
    int64_t ws_ld = 0;
    unsigned int *d_bar = nullptr;
    double *d_slots = nullptr;
    cudaStream_t last_stream = nullptr;
    bool pending = false;
};

namespace {

void release(mtd_lupiv *h) {
    cudaFree(h->d_tasks);
    cudaFree(h->d_succ);
    cudaFree(h->d_deps_init);
    cudaFree(h->d_deps);
    cudaFree(h->d_items_left);
    cudaFree(h->d_roots);
    for (int q = 0; q < kNumQueues; ++q) cudaFree(h->d_queue[q]);
    cudaFree(h->d_qctl);
    cudaFree(h->d_ctl);
    if (h->h_ctl) cudaFreeHost(h->h_ctl);
    cudaFree(h->d_ws);
    cudaFree(h->d_bar);
    cudaFree(h->d_slots);
}

struct Plan {
    std::vector<DevTask> tasks;
    std::vector<std::vector<int>> preds;
    int add(const DevTask &d, std::vector<int> pr) {
        tasks.push_back(d);
        preds.push_back(std::move(pr));
        return static_cast<int>(tasks.size()) - 1;
    }
};

DevTask make(int op, int queue, int n_items) {
    DevTask d{};
    d.op = op;
    d.queue = queue;
    d.n_items = n_items;
    return d;
}

}  // namespace

namespace mtd {

// Rows per panel item and items per panel for an m x w panel: the fewest items whose slabs
// fit the kernel's shared memory, never fewer rows than w (item 0 holds the diagonal tile);
// 0 if more than `grid` items would be needed.
int lupiv_panel_shape(int64_t m, int w, int smem_bytes, int grid, int *R_out) {
    const int64_t rmax = (smem_bytes - panel_piv_extra_bytes(w)) / (int64_t(w) * 8);
    if (rmax < std::min<int64_t>(m, w)) return 0;
    int64_t P = ceil_div(m, std::min(m, rmax));
    int64_t R = std::max(ceil_div(m, P), std::min<int64_t>(m, w));
    P = ceil_div(m, R);
    if (P > grid) return 0;
    *R_out = static_cast<int>(R);
    return static_cast<int>(P);
}

// The task graph above; false if some panel does not fit (n too large for the tile).
bool lupiv_plan(int64_t n, int64_t b, int smem_bytes, int grid, std::vector<DevTask> &tasks,
                std::vector<std::vector<int>> &preds, int *max_items) {
    const int T = static_cast<int>(ceil_div(n, b));
    auto ext = [&](int t) { return static_cast<int>(std::min<int64_t>(b, n - int64_t(t) * b)); };
    Plan pl;
    std::vector<int> gemm_prev(T, -1);  // GEMM(k-1, j): the last writer of block column j below row k*b
    int last_panel = -1;
    *max_items = 0;
    for (int k = 0; k < T; ++k) {
        const int64_t r0 = int64_t(k) * b, m = n - r0;
        const int w = ext(k);
        int R = 0;
        const int P = lupiv_panel_shape(m, w, smem_bytes, grid, &R);
        if (P == 0) return false;
        *max_items = std::max(*max_items, P);
        DevTask d = make(kOpPanelPiv, 0, P);
        d.cr = d.cc = static_cast<int32_t>(r0);
        d.m = static_cast<int32_t>(m);
        d.n = w;
        d.k = R;
        d.pad = k;
        std::vector<int> pp;
        if (gemm_prev[k] >= 0) pp.push_back(gemm_prev[k]);
        const int panel = pl.add(d, pp);
        last_panel = panel;
        for (int j = k + 1; j < T; ++j) {
            const int q = j == k + 1 ? 0 : (j == k + 2 ? 1 : 2);
            const int wj = ext(j);
            DevTask s = make(kOpLaswp, q, static_cast<int>(ceil_div(wj, kSwapColsHost)));
            s.cr = static_cast<int32_t>(r0);
            s.cc = static_cast<int32_t>(int64_t(j) * b);
            s.ar = static_cast<int32_t>(r0);
            s.k = w;
            s.m = static_cast<int32_t>(m);
            s.n = wj;
            std::vector<int> sp{panel};
            if (gemm_prev[j] >= 0) sp.push_back(gemm_prev[j]);
            const int swap = pl.add(s, sp);
            DevTask tr = make(MTD_OP_TRSM_LLNU, q, static_cast<int>(ceil_div(wj, kTrsmCols)));
            tr.cr = static_cast<int32_t>(r0);
            tr.cc = static_cast<int32_t>(int64_t(j) * b);
            tr.ar = tr.ac = static_cast<int32_t>(r0);
            tr.m = w;
            tr.n = wj;
            const int trsm = pl.add(tr, {swap, panel});
            const int64_t below = m - w;
            if (below > 0) {
                DevTask g = make(MTD_OP_GEMM_NN, q,
                                 static_cast<int>(ceil_div(below, kGemmEdge) * ceil_div(wj, kGemmEdge)));
                g.cr = g.ar = static_cast<int32_t>(r0 + w);
                g.cc = g.bc = static_cast<int32_t>(int64_t(j) * b);
                g.ac = g.br = static_cast<int32_t>(r0);
                g.m = static_cast<int32_t>(below);
                g.n = wj;
                g.k = w;
                gemm_prev[j] = pl.add(g, {trsm, panel, swap});
            } else {
                gemm_prev[j] = trsm;
            }
        }
    }
    for (int j = 0; j + 1 < T; ++j) {  // the later panels' interchanges, left of each panel
        const int64_t first = int64_t(j + 1) * b;
        const int wj = ext(j);
        DevTask s = make(kOpLaswp, kNumQueues - 1, static_cast<int>(ceil_div(wj, kSwapColsHost)));
        s.cr = static_cast<int32_t>(first);
        s.cc = static_cast<int32_t>(int64_t(j) * b);
        s.ar = static_cast<int32_t>(first);
        s.k = static_cast<int32_t>(n - first);
        s.m = static_cast<int32_t>(n - first);
        s.n = wj;
        pl.add(s, {last_panel});
    }
    tasks = std::move(pl.tasks);
    preds = std::move(pl.preds);
    return true;
}

}  // namespace mtd

extern "C" {

int mtd_lupiv_create(mtd_lupiv **out, int64_t n, int64_t tile) {
    if (!out) return MTD_ERR_INVALID_ARG;
    *out = nullptr;
    // item 0's slab holds the whole diagonal tile (tile x tile doubles), so tile <= 128
    if (n <= 0 || n > (int64_t(1) << 30) || (tile != 64 && tile != 128)) return MTD_ERR_INVALID_ARG;
    int dev = 0, major = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return MTD_ERR_NO_DEVICE;
    cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev);
    if (major != 10) return MTD_ERR_NO_DEVICE;
    mtd_lupiv *h = new (std::nothrow) mtd_lupiv();
    if (!h) return MTD_ERR_OUT_OF_MEMORY;
    h->n = n;
    h->tile = std::min(tile, n);
    h->T = static_cast<int>(ceil_div(n, h->tile));
    h->device = dev;
    cudaDeviceGetAttribute(&h->sms, cudaDevAttrMultiProcessorCount, dev);
    std::vector<DevTask> tasks;
    std::vector<std::vector<int>> preds;
    if (!lupiv_plan(n, h->tile, ext_op_smem_bytes(), h->sms, tasks, preds, &h->max_items)) {
        delete h;
        return MTD_ERR_INVALID_ARG;  // a panel would need more items than the GPU has SMs
    }
    const int nt = static_cast<int>(tasks.size());
    std::vector<std::vector<int>> succs(nt);
    std::vector<int> deps_init(nt), roots;
    for (int t = 0; t < nt; ++t) {
        deps_init[t] = static_cast<int>(preds[t].size());
        for (int p : preds[t]) succs[p].push_back(t);
        if (preds[t].empty()) roots.push_back(t);
    }
    std::vector<int> succ;
    for (int t = 0; t < nt; ++t) {
        tasks[t].succ_begin = static_cast<int32_t>(succ.size());
        tasks[t].succ_count = static_cast<int32_t>(succs[t].size());
        succ.insert(succ.end(), succs[t].begin(), succs[t].end());
        h->qcap[tasks[t].queue] += tasks[t].n_items;
    }
    h->n_tasks = nt;
    h->n_roots = static_cast<int>(roots.size());
    for (int q = 0; q < kNumQueues; ++q) h->total_items += h->qcap[q];
    h->ws_ld = (n + 3) & ~int64_t(3);
    int rc = dalloc(&h->d_tasks, nt);
    if (!rc) rc = dalloc(&h->d_succ, succ.size());
    if (!rc) rc = dalloc(&h->d_deps_init, nt);
    if (!rc) rc = dalloc(&h->d_deps, nt);
    if (!rc) rc = dalloc(&h->d_items_left, nt);
    if (!rc) rc = dalloc(&h->d_roots, roots.size());
    for (int q = 0; q < kNumQueues && !rc; ++q) rc = dalloc(&h->d_queue[q], size_t(h->qcap[q]));
    if (!rc) rc = dalloc(&h->d_qctl, kNumQueues);
    if (!rc) rc = dalloc(&h->d_ctl, 1);
    if (!rc) rc = dalloc(&h->d_ws, size_t(h->ws_ld) * kNB);
    if (!rc) rc = dalloc(&h->d_bar, h->T);
    if (!rc) rc = dalloc(&h->d_slots, size_t(2) * h->max_items * (h->tile + 2) + size_t(2) * h->tile);
    if (!rc && cudaMallocHost(reinterpret_cast<void **>(&h->h_ctl), sizeof(RunCtl)) != cudaSuccess)
        rc = MTD_ERR_OUT_OF_MEMORY;
    if (!rc &&
        (cudaMemcpy(h->d_tasks, tasks.data(), nt * sizeof(DevTask), cudaMemcpyHostToDevice) != cudaSuccess ||
         (!succ.empty() &&
          cudaMemcpy(h->d_succ, succ.data(), succ.size() * sizeof(int), cudaMemcpyHostToDevice) != cudaSuccess) ||
         cudaMemcpy(h->d_deps_init, deps_init.data(), nt * sizeof(int), cudaMemcpyHostToDevice) != cudaSuccess ||
         cudaMemcpy(h->d_roots, roots.data(), roots.size() * sizeof(int), cudaMemcpyHostToDevice) != cudaSuccess ||
         cudaMemset(h->d_ctl, 0, sizeof(RunCtl)) != cudaSuccess))
        rc = MTD_ERR_CUDA;
    if (rc) {
        release(h);
        delete h;
        return rc;
    }
    std::memset(h->h_ctl, 0, sizeof(RunCtl));
    *out = h;
    return MTD_OK;
}

int mtd_lupiv_num_tasks(const mtd_lupiv *h) { return h ? h->n_tasks : -MTD_ERR_INVALID_ARG; }

int mtd_lupiv_run(mtd_lupiv *h, double *dA, int64_t lda, int *d_ipiv, void *stream) {
    if (!h || !dA || !d_ipiv || lda < h->n) return MTD_ERR_INVALID_ARG;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev != h->device) return MTD_ERR_STATE;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    RunArgs a{};
    a.a = dA;
    a.lda = lda;
    a.n_tasks = h->n_tasks;
    a.tasks = h->d_tasks;
    a.succ = h->d_succ;
    a.deps = h->d_deps;
    a.items_left = h->d_items_left;
    for (int q = 0; q < kNumQueues; ++q) {
        a.queue[q] = h->d_queue[q];
        a.queue_cap[q] = h->qcap[q];
    }
    a.qctl = h->d_qctl;
    a.ctl = h->d_ctl;
    a.ws_lower = h->d_ws;
    a.ws_upper = nullptr;
    a.ws_ld = h->ws_ld;
    a.timeout_ns = 10ull * 1000000000ull;
    a.ipiv = d_ipiv;
    a.panel_bar = h->d_bar;
    a.n_panel_bar = h->T;
    a.panel_slots = h->d_slots;
    a.opset = kOpsLu;  // panel, interchange, TRSM_LLNU and GEMM_NN tasks
    const bool vec2 = reinterpret_cast<uintptr_t>(dA) % 16 == 0 && lda % 2 == 0 && h->n % 2 == 0 && h->tile % 2 == 0;
    const int rc = launch_run_solve(a, h->d_deps_init, h->d_roots, h->n_roots, h->total_items, MTD_PREC_FP64, vec2,
                                    h->sms, s);
    if (rc) return rc;
    if (cudaMemcpyAsync(h->h_ctl, h->d_ctl, sizeof(RunCtl), cudaMemcpyDeviceToHost, s) != cudaSuccess) return MTD_ERR_CUDA;
    h->last_stream = s;
    h->pending = true;
    return MTD_OK;
}

int mtd_lupiv_status(mtd_lupiv *h, int *info) {
    if (!h) return MTD_ERR_INVALID_ARG;
    if (info) *info = 0;
    if (!h->pending) return MTD_ERR_STATE;
    if (cudaStreamSynchronize(h->last_stream) != cudaSuccess) return MTD_ERR_CUDA;
    if (h->h_ctl->error) return h->h_ctl->error;
    if (h->h_ctl->tasks_done != h->n_tasks) return MTD_ERR_TIMEOUT;
    if (info && h->h_ctl->info != 0x7fffffff) *info = h->h_ctl->info;
    return MTD_OK;
}

int mtd_lupiv_destroy(mtd_lupiv *h) {
    if (!h) return MTD_ERR_INVALID_ARG;
    if (h->pending && h->last_stream) cudaStreamSynchronize(h->last_stream);
    release(h);
    delete h;
    return MTD_OK;
}

int mtd_lu_pivot(double *dA, int64_t n, int64_t lda, int64_t tile, int *d_ipiv, void *stream, int *info) {
    mtd_lupiv *h = nullptr;
    int rc = mtd_lupiv_create(&h, n, tile);
    if (rc) return rc;
    rc = mtd_lupiv_run(h, dA, lda, d_ipiv, stream);
    if (!rc) rc = mtd_lupiv_status(h, info);
    mtd_lupiv_destroy(h);
    return rc;
}

}  // extern "C"
