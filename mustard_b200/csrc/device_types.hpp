// Plain structs shared by the host runtime and the device kernels.
#pragma once

#include <cstdint>

namespace mtd {

// Ready queues, popped in order: 0 critical path (diagonal factorisations, panel solves,
// diagonal-tile updates, updates of the next panel column); 1 updates of the two panel
// columns after it; 2 the other updates.
constexpr int kNumQueues = 3;
#ifndef MTD_THREADS
#define MTD_THREADS 512
#endif
constexpr int kThreads = MTD_THREADS;  // threads per persistent CTA
constexpr int kGemmTile = 128;  // output sub-tile edge of one GEMM / SYRK work item
constexpr int kPanelRows = 64;  // rows of one TRSM work item of the adjoint
// Rows (or columns) of one TRSM strip of the tiled factorisations: 64, or 128 (fewer, larger
// items whose updates run on the 128 x 128 update engine).
#ifndef MTD_TRSM_ROWS
#define MTD_TRSM_ROWS 64
#endif
constexpr int kTrsmRows = MTD_TRSM_ROWS;
static_assert(kTrsmRows == 64 || kTrsmRows == 128, "TRSM strips are 64 or 128 rows");
constexpr int kNB = 64;         // diagonal block edge inside POTRF / GETRF (and inverse blocks)
constexpr int kNestTile = 128;  // default sub-tile edge of a nested diagonal factorisation

// Device-side operation codes: the public mtd_op values plus a join (one no-op work item).
// Codes from kOpJoin up are the scheduler's own tasks; the batched factor-and-solve launch
// adds two (mtd_batch_factor_solve): a matrix's conversion to the factor's precision (its
// root) and its solve with refinement (its sink).
constexpr int kOpJoin = 100;
constexpr int kOpBatchSolve = 101;    // one item: solve (+ refine) one matrix of the batch
constexpr int kOpBatchConvert = 102;  // items = 128-column strips: F = lower(A) + shift I, as T
constexpr int kConvertCols = 128;
constexpr int kBatchInfoOk = 0x7f7f7f7f;  // per-matrix info of a batched run before any bad pivot
// Pivoted LU (mtd_lupiv): a panel factorisation with partial pivoting (P cooperating items)
// and the row interchanges of one block column.
constexpr int kOpPanelPiv = 103;
constexpr int kOpLaswp = 104;
// Shared memory a pivoted panel item needs besides its slab of w-wide rows: the pivot row
// and the previous row c (w doubles each) and the per-warp reduction scratch.
#ifdef __CUDACC__
__host__ __device__
#endif
constexpr int64_t panel_piv_extra_bytes(int w) {
    return int64_t(2 * w) * 8 + int64_t(kThreads / 32) * (8 + 4) + 64;
}

// Cholesky adjoint operations (device tasks of the reverse sweep; see adjoint_ops.cuh).
constexpr int kOpAdjTrsm = 20;    // C(m x n) := C * L^-1, L = n x n lower at (ar, ac) of the factor
constexpr int kOpAdjGemmNN = 21;  // C(m x n) -= A(m x k) * B(k x n); A in the adjoint (pad 0) or Y (pad 2), B in L
constexpr int kOpAdjGemmTN = 22;  // C(m x n) -= A^T * B, A stored k x m in the adjoint, B (k x n) in L;
                                  // pad & 1: lower triangle of C only
constexpr int kOpAdjPotrf = 23;   // diagonal tile (m x m) adjoint at (cr, cc); writes Y rows cr.., columns 0..m
#ifdef __CUDACC__
__host__ __device__
#endif
constexpr bool is_adjoint_op(int op) { return op >= kOpAdjTrsm && op <= kOpAdjPotrf; }

// One device task.  Geometry is in matrix elements (row, column origins of each block
// inside the column-major matrix), so a task can cover a whole tile or a sub-tile of a
// nested diagonal factorisation.
//   GEMM_NT  C(m x n) -= A(m x k) * B(n x k)^T
//   GEMM_NN  C(m x n) -= A(m x k) * B(k x n)
//   SYRK_LN  C(m x m) -= A(m x k) * A^T (lower)
//   TRSM_RLT X(m x n) = X * L^-T,  L = n x n at A's origin
//   TRSM_RUN X(m x n) = X * U^-1,  U = n x n at A's origin
//   TRSM_LLNU X(m x n) = L^-1 * X, L = m x m (unit) at A's origin
//   POTRF / GETRF: the m x m block at C's origin
// The inverse workspaces are indexed by absolute matrix row: the inverse of the kNB x kNB
// diagonal block whose first row is r sits at ws[r + c * ws_ld], c < kNB.
struct alignas(16) DevTask {
    int32_t op;
    int32_t queue;       // ready queue, 0 .. kNumQueues - 1
    int32_t n_items;     // >= 1 (a join has one no-op item)
    int32_t cr, cc;      // output block origin
    int32_t ar, ac;      // first operand (triangular block for TRSM)
    int32_t br, bc;      // second operand (GEMM)
    int32_t m, n, k;     // extents
    int32_t succ_begin;  // successors are succ[succ_begin, succ_begin + succ_count)
    int32_t succ_count;
    int32_t mat;         // matrix of a batched run (index into RunArgs::mats), else 0
    int32_t pad;
};
static_assert(sizeof(DevTask) == 64, "DevTask is read as four 16-byte words");

// Per-matrix arguments of the batched solves (standalone kernels and the solve tasks of
// the factor-and-solve launch).
struct SolveMat {
    const double *a;  // FP64 matrix (lower triangle read), for residuals
    int64_t lda;
    const void *f;    // factor (element type of the batch)
    int64_t ldf;
    int64_t ws_off, ws_ld;
    const double *b;
    int64_t ldb;
    double *x;
    int64_t ldx;
    double *r;        // residual scratch, n x nrhs (ld n)
    void *d;          // low-precision correction scratch, n x nrhs (ld n)
    int n, nrhs;
};

// One matrix of a batched run.
struct BatchMat {
    void *a;         // column-major matrix (element type of the run)
    int64_t lda;
    int64_t ws_off;  // this matrix's slice of the inverse workspaces (elements)
    int64_t ws_ld;
};

// Device-resident control block of one graph (one cache line per hot counter).
struct alignas(128) QueueCtl {
    unsigned long long head;   // next slot to claim
    char pad0[120];
    unsigned long long tail;   // slots reserved by producers
    char pad1[120];
    long long avail;           // items pushed and not yet claimed (transiently low while a
    char pad2[120];            // failed claim is being undone)
};

struct alignas(128) RunCtl {
    int tasks_done;
    int error;      // first mtd_status raised on the device, 0 if none
    int info;       // LAPACK-style info (1-based global column), 0 if none
    int abort;      // set with error; every CTA polls it
    unsigned long long items_done;
    unsigned long long start_ns;  // earliest %globaltimer at which a CTA started popping
    char pad[96];
};

// Everything the persistent kernel needs for one run (passed by value).
// Operation families a run's tasks use; FP64 runs whose tasks are all Cholesky (POTRF, TRSM_RLT,
// SYRK, GEMM_NT) or all LU (GETRF, TRSM_LLNU, TRSM_RUN, GEMM_NN) operations launch a kernel
// instance compiled with that family's operations only.
enum : int { kOpsAll = 0, kOpsCholesky = 1, kOpsLu = 2 };

struct RunArgs {
    void *a;               // matrix, column-major (double, or float for the low-precision factor)
    int64_t lda;
    int n_tasks;           // device tasks (including joins)
    const DevTask *tasks;
    const int *succ;
    int *deps;             // remaining predecessor counts (reset each run)
    int *items_left;       // remaining work items per task (reset each run)
    unsigned long long *queue[kNumQueues];
    long long queue_cap[kNumQueues];
    QueueCtl *qctl;        // kNumQueues entries
    RunCtl *ctl;
    void *ws_lower;        // inverses of the diagonal blocks of L (ws_ld x kNB, matrix type)
    void *ws_upper;        // inverses of the diagonal blocks of U (LU only)
    int64_t ws_ld;
    unsigned long long *trace;  // optional: 4 words per item (start, end, sm, task<<32|item)
    long long trace_cap;
    unsigned long long timeout_ns;
    // Batched runs only (mats == nullptr otherwise): per-matrix geometry, per-matrix
    // LAPACK-style info (INT_MAX = success), and the %globaltimer time at which each
    // matrix's last task finished (for per-matrix latency).
    const BatchMat *mats;
    int *mat_info;
    unsigned long long *mat_done_ns;
    // TF32 single-matrix runs: a TMA tensor map of the matrix (FP32, ld = lda, 128-byte /
    // 32-byte-atom swizzle) for the tcgen05 GEMM items; tma = 0 none, 1 a 2D map (box 32 x 64),
    // 2 a 3D map (32 rows of an atom, columns, atoms; box 32 x 64 x 4).  The kernel receives
    // RunArgs as a __grid_constant__ parameter, so the map's address is a valid TMA
    // descriptor address.
    int tma;
    alignas(64) unsigned char tmap[128];
    // BF16-update runs (MTD_PREC_BF16): the BF16 copy of the panels (column-major, leading
    // dimension bf16_ld, a multiple of 64) that TRSM items write and GEMM / SYRK items read,
    // and its TMA tensor map (3D: 64 rows of an atom, columns, atoms; box 64 x 128 x 2,
    // 128-byte swizzle) when tma_bf16 != 0.
    void *bf16;
    int64_t bf16_ld;
    int tma_bf16;
    alignas(64) unsigned char tmap_bf16[128];
    // FP64 single-matrix runs: TMA tensor maps of the matrix for the GEMM / SYRK items
    // (tma64.cuh) when tma64 != 0: a 3D map {16 rows of an atom, columns, atoms}, box
    // {16, 16, 8}, for m- and n-contiguous operands, and a 2D map {rows, columns}, box
    // {16, 128}, for the k-contiguous operand of GEMM_NN; both with the 128-byte swizzle.
    int tma64;
    alignas(64) unsigned char tmap64_mn[128];
    alignas(64) unsigned char tmap64_k[128];
    // FP32-accurate runs (MTD_PREC_FP32): the low parts of the panels that TRSM items write
    // (x minus x truncated to TF32, rounded to nearest TF32; column-major, leading dimension
    // lo_ld), read with the panels themselves by the three-pass tcgen05 updates; its TMA
    // tensor map (3D like `tmap`, box 32 x 32 x 4) when tma_lo != 0, `tmap` then holding the
    // matrix's map with the same box.
    void *lo;
    int64_t lo_ld;
    int tma_lo;
    alignas(64) unsigned char tmap_lo[128];
    // Batched factor-and-solve launches only (solve == nullptr otherwise): per-matrix solve
    // arguments, the refinement method (MTD_REFINE_*), its tolerance and step limit, the
    // diagonal shift of the conversion tasks, and per-matrix outcomes (backward error, -1 when
    // no FP64 matrix was given; solves applied).
    const SolveMat *solve;
    double *solve_berr;
    int *solve_iters;
    double solve_tol;
    double solve_shift;
    int solve_method;
    int solve_max_iter;
    // Pivoted LU runs only: the pivot vector (ipiv, 1-based rows as LAPACK's), one arrival
    // counter per panel (zeroed by the per-run reset) and the panel items' exchange slots.
    int *ipiv;
    unsigned int *panel_bar;
    int n_panel_bar;
    double *panel_slots;
    int opset;             // kOpsAll / kOpsCholesky / kOpsLu: the kernel instance the host launches
};

}  // namespace mtd
