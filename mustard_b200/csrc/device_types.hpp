// Plain structs shared by the host runtime and the device kernels.
#pragma once

#include <cstdint>

namespace mtd {

constexpr int kNumQueues = 2;   // 0: critical path (diagonal, panel, next-panel updates); 1: rest
constexpr int kThreads = 256;   // threads per persistent CTA
constexpr int kGemmTile = 128;  // output sub-tile edge of one GEMM / SYRK work item
constexpr int kPanelRows = 64;  // rows (or columns) of one TRSM work item
constexpr int kNB = 64;         // diagonal block edge inside POTRF / GETRF (and inverse blocks)

// One task of the DAG as the device sees it.
struct DevTask {
    int32_t op;
    int32_t queue;       // 0 or 1
    int32_t n_items;
    int32_t wi, wj;      // tile written
    int32_t ai, aj;      // first operand tile (triangular tile for TRSM)
    int32_t bi, bj;      // second operand tile (GEMM)
    int32_t succ_begin;  // successors are succ[succ_begin, succ_begin + succ_count)
    int32_t succ_count;
};

// Device-resident control block of one graph (one cache line per hot counter).
struct alignas(128) QueueCtl {
    unsigned long long head;   // next slot to claim
    char pad0[120];
    unsigned long long tail;   // slots reserved by producers
    char pad1[120];
};

struct alignas(128) RunCtl {
    int tasks_done;
    int error;      // first mtd_status raised on the device, 0 if none
    int info;       // LAPACK-style info (1-based global column), 0 if none
    int abort;      // set with error; every CTA polls it
    unsigned long long items_done;
    char pad[104];
};

// Everything the persistent kernel needs for one run (passed by value).
struct RunArgs {
    double *a;             // matrix, column-major
    int64_t lda;
    int64_t n;
    int64_t tile;
    int tiles;
    int n_tasks;
    const DevTask *tasks;
    const int *succ;
    int *deps;             // remaining predecessor counts (reset each run)
    int *items_left;       // remaining work items per task (reset each run)
    unsigned long long *queue[kNumQueues];
    long long queue_cap[kNumQueues];
    QueueCtl *qctl;        // kNumQueues entries
    RunCtl *ctl;
    double *ws_lower;      // per-step inverses of the diagonal blocks of L (tiles*tile*kNB)
    double *ws_upper;      // per-step inverses of the diagonal blocks of U (LU only)
    unsigned long long *trace;  // optional: 4 words per item (start, end, sm, task<<32|item)
    long long trace_cap;
    unsigned long long timeout_ns;
};

}  // namespace mtd
