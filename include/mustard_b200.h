/*
 * mustard_b200.h -- C ABI of the B200 (sm_100a) runtime for static tiled LU / Cholesky
 * task graphs.
 *
 * The reference (ParCoreLab/mustard) exposes a header-only C++ interface whose tasks are
 * captured cuBLAS/cuSOLVER calls: TiledGraphCreator (mustard/mustard.h:132-384), a
 * broker queue (mustard/broker_queue.h:13-147), and the device kernels kernel_scheduler,
 * kernel_dep_update and kernel_populate_queue (mustard/mustard.h:70-129).  Here a task is
 * structured data (operation, tile written, tiles read) and a single persistent kernel
 * pops ready work, runs hand-written FP64 tile kernels and resolves dependencies on the
 * device.  Every entry point returns an mtd_status; nothing here exits the process.
 *
 * Conventions
 *   - Matrices are FP64, column-major, leading dimension lda >= n.  Tile (i, j) covers
 *     rows [i*tile, min((i+1)*tile, n)) and columns [j*tile, min((j+1)*tile, n)), as in
 *     the reference's `matrix + i*B + j*B*N` (mustard/cholesky_mustard.cu:157-160).  The
 *     last tile row/column may be ragged (the reference requires tile | n).
 *   - The caller owns the matrix; a graph owns its device-side DAG, queues, counters and
 *     the per-step inverse workspace.
 *   - `stream` is a cudaStream_t passed as void* (0 = legacy default stream).
 *   - One host thread per graph; different graphs are independent.
 */
#ifndef MUSTARD_B200_H
#define MUSTARD_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define MTD_ABI_VERSION 1

typedef enum mtd_status {
    MTD_OK = 0,
    MTD_ERR_INVALID_ARG = 1,     /* bad argument (size, tile, op, pointer)              */
    MTD_ERR_STATE = 2,           /* call out of order (e.g. add_task after finalize)    */
    MTD_ERR_CUDA = 3,            /* a CUDA runtime call failed                          */
    MTD_ERR_TIMEOUT = 4,         /* a device-side wait ran past its limit               */
    MTD_ERR_NOT_POSITIVE_DEFINITE = 5, /* POTRF met a non-positive pivot; see info    */
    MTD_ERR_SINGULAR = 6,        /* GETRF (no pivoting) met a zero pivot; see info      */
    MTD_ERR_BAD_DAG = 7,         /* graph cannot be executed (see mtd_graph_finalize)   */
    MTD_ERR_NO_DEVICE = 8,       /* no CUDA device / not an sm_100 device               */
    MTD_ERR_OUT_OF_MEMORY = 9,   /* device allocation failed                            */
    MTD_ERR_QUEUE = 10,          /* ready-queue overflow (internal invariant broken)    */
    MTD_ERR_TOO_LARGE = 11       /* problem exceeds mtd_factor_noalloc's fixed scratch  */
} mtd_status;

typedef enum mtd_kind {
    MTD_KIND_LU = 0,             /* no-pivot LU, reference lu_mustard                   */
    MTD_KIND_CHOLESKY = 1,       /* lower Cholesky, reference cholesky_mustard          */
    MTD_KIND_CUSTOM = 2          /* tasks supplied one by one with mtd_graph_add_task   */
} mtd_kind;

/* Tile operations.  Each replaces one captured library call of the reference. */
typedef enum mtd_op {
    MTD_OP_POTRF = 0,     /* A(k,k) = chol(A(k,k)), lower         cholesky_mustard.cu:238   */
    MTD_OP_TRSM_RLT = 1,  /* A(i,k) = A(i,k) L(k,k)^-T            cholesky_mustard.cu:281   */
    MTD_OP_SYRK_LN = 2,   /* A(i,i) -= A(i,k) A(i,k)^T, lower     cholesky_mustard.cu:327   */
    MTD_OP_GEMM_NT = 3,   /* A(j,i) -= A(j,k) A(i,k)^T            cholesky_mustard.cu:376   */
    MTD_OP_GETRF = 4,     /* A(k,k) = L U, no pivoting            lu_mustard.cu:361         */
    MTD_OP_TRSM_LLNU = 5, /* A(k,i) = L(k,k)^-1 A(k,i), unit L    lu_mustard.cu:413         */
    MTD_OP_TRSM_RUN = 6,  /* A(i,k) = A(i,k) U(k,k)^-1            lu_mustard.cu:459         */
    MTD_OP_GEMM_NN = 7    /* A(i,j) -= A(i,k) A(k,j)              lu_mustard.cu:511         */
} mtd_op;

/* Arithmetic of a graph's runs. */
typedef enum mtd_precision {
    MTD_PREC_FP64 = 0,           /* FP64 matrix, FP64 tensor-core (DMMA) tiles: the reference's */
    MTD_PREC_TF32 = 1,           /* FP32 matrix, TF32 tensor-core products with FP32           */
                                 /* accumulation, FP32 diagonal blocks (Cholesky only); the    */
                                 /* low-precision factor of the mixed-precision solver         */
    MTD_PREC_FP32 = 2,           /* FP32 matrix, FP32-accurate products from three TF32 MMAs   */
                                 /* per product (split operands: hi*hi + hi*lo + lo*hi)        */
    MTD_PREC_BF16 = 3            /* FP32 matrix; the GEMM / SYRK updates take BF16 operands    */
                                 /* (FP32 accumulation) from a BF16 copy of the panels that    */
                                 /* the TRSMs write (the graph allocates it: 2 N^2 bytes);     */
                                 /* diagonal and panel work as MTD_PREC_TF32 (Cholesky only)   */
} mtd_precision;

typedef enum mtd_generator {
    MTD_GEN_UNIFORM_DIAG = 0,    /* U[-1,1) entries + n on the diagonal (LU input)      */
    MTD_GEN_SPD = 1              /* B B^T / n + alpha I, B = U[-1,1) (Cholesky input)   */
} mtd_generator;

typedef struct mtd_graph mtd_graph;

/* Per-run statistics, filled by mtd_graph_last_stats after a run completed. */
typedef struct mtd_run_stats {
    int64_t tasks;               /* tasks executed                                      */
    int64_t items;               /* work items executed                                 */
    int64_t ctas;                /* persistent CTAs launched                            */
    double busy_fraction;        /* sum of item durations / (ctas * kernel span); only  */
                                 /* valid when tracing was enabled, else -1             */
    double span_ms;              /* first item start to last item end (tracing), or -1  */
} mtd_run_stats;

/* ---- graph construction: replaces TiledGraphCreator (mustard/mustard.h:132-384) ---- */

/* Create an empty graph over an n x n matrix cut into tile x tile tiles.
 * Replaces the TiledGraphCreator constructor (mustard/mustard.h:139-146). */
int mtd_graph_create(mtd_graph **out, int kind, int64_t n, int64_t tile);

/* Record one task: operation `op` writing tile (wi, wj) and reading `nreads` tiles given
 * as (row, col) pairs in `reads` -- the arguments of the reference's
 * beginCaptureOperation(tileToWrite, {tilesToRead}) (mustard/mustard.h:148-167); the
 * operation replaces the library call captured between begin and endCaptureOperation.
 * Predecessors are inferred as in getSubgraphDependencies (mustard/mustard.h:279-296):
 * the last writer of every tile in reads + {write}, sorted and de-duplicated; a writer
 * additionally waits for earlier readers of the tile it overwrites.  Returns the task
 * index (>= 0) or a negative mtd_status. */
int mtd_graph_add_task(mtd_graph *g, int op, int wi, int wj, const int *reads, int nreads);

/* Tile rows (and columns) at the element edges edges[0] = 0 < edges[1] < ... <
 * edges[count - 1] = n instead of uniform `tile`-wide ones, e.g. a narrower first or last
 * tile (the reference's tiles are uniform).  Only before any task is recorded. */
int mtd_graph_set_tile_edges(mtd_graph *g, const int64_t *edges, int count);

/* Emit the reference's whole task list for the graph's kind, in its loop order
 * (cholesky_mustard.cu:224-395 or lu_mustard.cu:345-533).  MTD_ERR_INVALID_ARG when the
 * list would exceed 2^25 tasks (the count is cubic in the tile count). */
int mtd_graph_build_tiled(mtd_graph *g);

/* Number of tasks recorded so far. */
int mtd_graph_num_tasks(const mtd_graph *g);

/* Copy task `task`'s predecessor list (the reference's subgraphDependencies[task],
 * mustard/mustard.h:137) into out[0..cap); returns the full count or a negative status. */
int mtd_graph_get_deps(const mtd_graph *g, int task, int *out, int cap);

/* Task `task` as recorded: its operation (mtd_op), the tile it writes, and up to `cap` of
 * the tiles it reads as (row, col) pairs in reads_out[0..2*cap) -- the arguments of the
 * reference's beginCaptureOperation (mustard/mustard.h:148-167).  Returns the number of
 * tiles read or a negative status.  Used to plan how a graph's tasks and tiles are spread
 * over several GPUs (mustard_b200/distribution.py). */
int mtd_graph_task_info(const mtd_graph *g, int task, int *op_out, int *wi_out, int *wj_out, int *reads_out, int cap);

/* Number of device tasks after mtd_graph_finalize: the host tasks, with every nested
 * diagonal factorisation counted as its sub-tasks (0 before finalize). */
int mtd_graph_num_device_tasks(const mtd_graph *g);

/* Number of device work items task `task` is split into (0 before finalize). */
int mtd_graph_task_items(const mtd_graph *g, int task);

/* Operation (mtd_op; 100 for a zero-work join) of device task `task` after finalize, the
 * task index the trace records carry; a negative status otherwise. */
int mtd_graph_device_task_op(const mtd_graph *g, int task);

/* Copy device task `task`'s predecessor device tasks into out[0..cap) after finalize (for
 * critical-path analysis of traces); returns the full count or a negative status. */
int mtd_graph_device_task_deps(const mtd_graph *g, int task, int *out, int cap);

/* Validate and upload the DAG: predecessor counts (the reference's h_dependencies,
 * cholesky_mustard.cu:422-425), successor lists (what insertDependencyKernel wires,
 * mustard/mustard.h:197-211), work items, priorities, queues and workspace.  Replaces
 * the per-task graph instantiation and queue set-up of cholesky_mustard.cu:408-466. */
int mtd_graph_finalize(mtd_graph *g);

/* Enable (1) or disable (0) the per-item device trace used for busy-fraction stats. */
int mtd_graph_set_trace(mtd_graph *g, int enable);

/* Sub-tile edge for nested diagonal factorisations (a multiple of 64; 0 disables).  A
 * POTRF/GETRF task on a tile larger than this runs as a tiled factorisation of that tile
 * with sub-tiles of this edge, spread over many SMs -- as the reference nests a tiled
 * sub-LU when the tile exceeds MAX_TILE (lu_mustard.cu:133-254, :381-388).  Default 128.
 * Must be called before mtd_graph_finalize. */
int mtd_graph_set_nest(mtd_graph *g, int nest);

/* Upper bound (seconds) on any single device-side wait; default 10 s. */
int mtd_graph_set_timeout(mtd_graph *g, double seconds);

/* Run the graph on the device matrix dA (column-major, leading dimension lda).
 * Replaces the timed cudaGraphLaunch(schedulerExec, s) of cholesky_mustard.cu:474 /
 * lu_mustard.cu:609, plus the counter/queue reset of :479-485.  Stream-ordered.  If
 * info_out is non-NULL the call synchronises the stream and returns the run's status
 * with LAPACK-style info (1-based column of the first bad pivot, else 0); if NULL it
 * returns after enqueueing and mtd_graph_status reports the outcome later. */
int mtd_run(mtd_graph *g, double *dA, int64_t lda, void *stream, int *info_out);

/* The same tasks and tile kernels executed as one host-launched CUDA graph: one kernel
 * node per task (grid = its work items) whose node dependencies are the task's
 * predecessors, so the CUDA graph executor resolves the DAG.  Replaces the reference's
 * --tiled mode (mustard/mustard.h:155-159, :341-383; cholesky_mustard.cu:498-513).  The
 * CUDA graph is built on the first call for a given (dA, lda) and reused.  Same
 * status/info conventions as mtd_run. */
int mtd_run_graph(mtd_graph *g, double *dA, int64_t lda, void *stream, int *info_out);

/* Arithmetic of the graph's runs (mtd_precision); before mtd_graph_finalize.  Default
 * MTD_PREC_FP64.  MTD_PREC_TF32 accepts Cholesky tasks only and runs with mtd_run_f32. */
int mtd_graph_set_precision(mtd_graph *g, int prec);

/* mtd_run for a MTD_PREC_TF32 graph: factors the FP32 column-major matrix dA in place. */
int mtd_run_f32(mtd_graph *g, float *dA, int64_t lda, void *stream, int *info_out);

/* Synchronise with the last run and return its status (and info). */
int mtd_graph_status(mtd_graph *g, int *info_out);

/* Statistics of the last completed run. */
int mtd_graph_last_stats(mtd_graph *g, mtd_run_stats *out);

/* Raw per-item trace of the last run (tracing enabled): 4 words per work item -- start
 * and end %globaltimer ns, SM id, task << 32 | item.  Returns the number of records
 * copied into out (at most cap_records), or a negative status. */
long long mtd_graph_copy_trace(mtd_graph *g, unsigned long long *out, long long cap_records);

/* Release everything the graph owns (replaces queue.free_mem(), broker_queue.h:36-43). */
int mtd_graph_destroy(mtd_graph *g);

/* ---- one-call drivers: replace tiledCholesky / tiledLU (cholesky_mustard.cu:135,
 *      lu_mustard.cu:256) for a caller that owns the device matrix ---- */
int mtd_tiled_cholesky(double *dA, int64_t n, int64_t lda, int64_t tile, void *stream,
                       int *info_out);
int mtd_tiled_lu(double *dA, int64_t n, int64_t lda, int64_t tile, void *stream,
                 int *info_out);

/* ---- factorisation without any device allocation ----
 *
 * No counterpart in the reference.  Every other entry point gets its task table, ready
 * queues, counters and inverse workspace from cudaMalloc.  Some callers cannot do that:
 * applications whose device memory is owned entirely by a pool allocator (PyTorch's
 * caching allocator, RAPIDS RMM) that must not see raw allocations, and latency-critical
 * services that cannot afford an allocation, or its failure, on the request path.  This
 * entry point serves them: it runs the same tiled LU (kind
 * MTD_KIND_LU) or Cholesky (MTD_KIND_CHOLESKY) as mtd_tiled_lu / mtd_tiled_cholesky, but
 * all of its device scratch lives in one fixed, file-scope device array of 24 MiB inside
 * this library (every GPU that loads the library holds it until the process exits).  It
 * calls no cudaMalloc, cudaFree, cudaMallocHost or other allocating CUDA routine; the task
 * list is assembled in ordinary host memory and copied into the array.
 *
 * Limits: n <= 16384 and, for the chosen tile, at most 32768 device tasks, 131072
 * dependency edges and 262144 work items; larger problems return MTD_ERR_TOO_LARGE (a tile
 * so small that the task list alone is too long is rejected before the list is built).
 * The first call on a device looks up the array's device address (and sets the kernel's
 * shared-memory limit).
 * All calls share the one array: calls whose work overlaps on the GPU (different streams,
 * host threads, or graphs) race and corrupt each other's results; serialise them.  The
 * call copies the task list from ordinary (pageable) host memory into the array, waits
 * for its stream and returns the run's status, so it cannot be called while its stream
 * is being captured into a CUDA graph; info_out (may be NULL) receives LAPACK-style info
 * as with mtd_run. */
int mtd_factor_noalloc(int kind, double *dA, int64_t n, int64_t lda, int64_t tile, void *stream,
                       int *info_out);

/* ---- mixed-precision SPD solver (no counterpart in the reference) ----
 *
 * Factor A (FP64, lower triangle read) in the solver's precision on the task-graph
 * scheduler, then solve A X = B to FP64 accuracy: MTD_REFINE_IR adds corrections
 * M^-1 (B - A X) with M = L L^T the low-precision factor; MTD_REFINE_GMRES_IR solves each
 * correction equation with FP64 GMRES preconditioned by M (Carson & Higham 2017/2018);
 * MTD_REFINE_NONE is one solve with the factor.  Residuals and updates are FP64.  With
 * MTD_PREC_FP64 the same calls give the plain FP64 solve (the time-to-solution baseline).
 * The caller's A must stay unchanged on the device while the solver uses it. */
typedef enum mtd_refine {
    MTD_REFINE_NONE = 0,
    MTD_REFINE_IR = 1,
    MTD_REFINE_GMRES_IR = 2
} mtd_refine;

typedef struct mtd_solve_stats {
    int iterations;            /* refinement steps (corrections applied)                */
    int inner_iterations;      /* GMRES iterations summed over the steps                */
    int converged;             /* 1 when backward_error <= tol was reached              */
    double backward_error;     /* max over columns of ||b - A x||_inf /                 */
                               /*   (||A||_inf ||x||_inf + ||b||_inf), in FP64          */
    double factor_ms;          /* device time of the last mtd_solver_factor             */
    double solve_ms;           /* host wall time of this solve (includes its syncs)     */
} mtd_solve_stats;

typedef struct mtd_solver mtd_solver;

/* n x n systems; tile must be a multiple of 64; prec MTD_PREC_TF32, MTD_PREC_FP32,
 * MTD_PREC_BF16 (low-precision factors) or MTD_PREC_FP64 (the plain FP64 baseline). */
int mtd_solver_create(mtd_solver **out, int64_t n, int64_t tile, int prec);
/* Factor A + shift*I (shift >= 0; a diagonal shift keeps a low-precision factorisation of
 * an ill-conditioned matrix positive definite; refinement still solves with A itself). */
int mtd_solver_factor(mtd_solver *s, const double *dA, int64_t lda, double shift, void *stream, int *info_out);
/* Solve for nrhs <= 16 right-hand sides (GMRES-IR: nrhs = 1); stops at backward error
 * <= tol or after max_iter corrections. */
int mtd_solver_solve(mtd_solver *s, const double *dB, int64_t ldb, double *dX, int64_t ldx, int64_t nrhs, int method,
                     double tol, int max_iter, void *stream, mtd_solve_stats *stats);
int mtd_solver_destroy(mtd_solver *s);

/* ---- batched factorisations (no counterpart in the reference) ----
 *
 * `count` independent SPD matrices of sizes n[m] (each its own tile edge tile[m] -- equal
 * to n[m] or a multiple of 64 -- and nested sub-tile edge nest[m]; NULL arrays pick the
 * defaults or use mtd_batch_autotune's choice) factored as ONE merged task graph by one
 * persistent launch (stream-ordered, no host synchronisation: it can be captured into a
 * CUDA graph).  Element type per batch: MTD_PREC_FP64 (double matrices) or MTD_PREC_TF32 /
 * MTD_PREC_FP32 (float matrices, refined in FP64 by mtd_batch_solve).  A bad pivot in one
 * matrix records its info and the rest of the batch runs on. */
typedef struct mtd_batch mtd_batch;

typedef struct mtd_batch_solve_stats {
    int iterations;            /* solves applied: FP64 1 + corrections; low: corrections */
    int converged_count;       /* matrices whose backward error reached tol             */
    double max_backward_error; /* max over matrices and columns (FP64), -1 if not known */
    double solve_ms;           /* host wall time of the solve call                      */
} mtd_batch_solve_stats;

int mtd_batch_create(mtd_batch **out, int count, const int64_t *n, const int64_t *tile, const int *nest, int prec);
int mtd_batch_num_tasks(const mtd_batch *b);
/* Factor matrix m at dA[m] (device pointer; double or float per the batch) in place. */
int mtd_batch_factor(mtd_batch *b, void *const *dA, const int64_t *lda, void *stream);
/* Wait for the last factorisation; info[m] (nullable) = 0 or the 1-based column of the
 * first bad pivot; latency_ms[m] (nullable) = time from the launch's first work to the
 * completion of matrix m's last task (device %globaltimer). */
int mtd_batch_status(mtd_batch *b, int *info, double *latency_ms);
/* Low-precision batches: dF[m] = float(lower(dA[m]) + shift I), ready for factoring. */
int mtd_batch_convert(mtd_batch *b, const double *const *dA, const int64_t *lda, void *const *dF, const int64_t *ldf,
                      double shift, void *stream);
/* Solve A_m X_m = B_m with the factors dF[m] (nrhs[m] <= 16).  FP64 batches: one solve,
 * plus FP64 IR when method is MTD_REFINE_IR; low-precision batches: FP64 IR (required) to
 * backward error tol.  dA (the FP64 matrices) may be NULL only for an FP64 batch with
 * MTD_REFINE_NONE. */
int mtd_batch_solve(mtd_batch *b, const double *const *dA, const int64_t *lda, void *const *dF, const int64_t *ldf,
                    const double *const *dB, const int64_t *ldb, double *const *dX, const int64_t *ldx,
                    const int *nrhs, int method, double tol, int max_iter, void *stream, mtd_batch_solve_stats *stats);
/* Factor AND solve in ONE persistent launch (stream-ordered, no host synchronisation: it
 * can be captured into a CUDA graph).  The launch's task graph is the merged factorisation
 * DAG plus, per matrix, a solve task after its last factor task (one CTA: the whole solve
 * with its refinement steps, as mtd_batch_solve's launches do them) and, for low-precision
 * batches, a conversion task before its first (dF[m] = lower(dA[m]) + shift I, rounded to
 * float: dF needs no initialisation).  So one matrix's solve overlaps the other matrices'
 * factorisations.  FP64 batches factor dF[m] in place; dA (the FP64 matrices, for the
 * residuals) may then be NULL with MTD_REFINE_NONE.  Low-precision batches need dA and
 * MTD_REFINE_IR.  Results: mtd_batch_solve_status. */
int mtd_batch_factor_solve(mtd_batch *b, void *const *dF, const int64_t *ldf, const double *const *dA,
                           const int64_t *lda, const double *const *dB, const int64_t *ldb, double *const *dX,
                           const int64_t *ldx, const int *nrhs, int method, double tol, int max_iter, double shift,
                           void *stream);
/* Wait for the last mtd_batch_factor_solve.  Per matrix (each array nullable): info as
 * mtd_batch_status, latency_ms up to the end of its solve, berr = its normwise backward error
 * (max over its columns; -1 without dA; NaN if its factorisation failed), iterations = the
 * solves applied.  stats: max iterations, matrices with berr <= tol, the max berr, and
 * solve_ms = the launch's device time (first work to last matrix done). */
int mtd_batch_solve_status(mtd_batch *b, int *info, double *latency_ms, double *berr, int *iterations,
                           mtd_batch_solve_stats *stats);
/* CTA-to-task schedule of the batch's launches: the order in which the matrices' first
 * tasks enter the ready queues (MTD_BATCH_ORDER_*; the queues are FIFO, so it is the order
 * in which the 148 CTAs start the matrices), ORed with MTD_BATCH_SOLVE_LATE to queue the
 * solve tasks of mtd_batch_factor_solve behind all factor work instead of ahead of it, and
 * with MTD_BATCH_SOLVE_PAIRS to give each solve task two matrices adjacent in that order
 * (one per half of the CTA) instead of one (the whole CTA). */
enum {
    MTD_BATCH_ORDER_INPUT = 0,
    MTD_BATCH_ORDER_LARGEST_FIRST = 1,
    MTD_BATCH_ORDER_SMALLEST_FIRST = 2,
    MTD_BATCH_SOLVE_LATE = 4,
    MTD_BATCH_SOLVE_PAIRS = 8,
    MTD_BATCH_NUM_SCHEDULES = 12 /* candidates the schedule tuner times: 3 orders x 2 x 2 */
};
int mtd_batch_set_schedule(mtd_batch *b, int schedule);
int mtd_batch_get_schedule(const mtd_batch *b);
/* Schedule tuner: times mtd_batch_factor_solve (arguments as there) under each of the
 * MTD_BATCH_NUM_SCHEDULES schedules (candidate c = (c % 6 / 2) | (c % 2 ?
 * MTD_BATCH_SOLVE_LATE : 0) | (c >= 6 ? MTD_BATCH_SOLVE_PAIRS : 0)), `reps` timed launches
 * each after one untimed, and keeps the fastest (set on the batch and returned in *best).
 * FP64 batches factor in place, so before every launch the tuner restores dF[m] from
 * dSrc[m] (device copies, outside the timed region); dSrc may be NULL for low-precision
 * batches, whose conversion tasks rewrite dF.  ms (nullable, MTD_BATCH_NUM_SCHEDULES
 * entries): each candidate's best device time. */
int mtd_batch_tune_schedule(mtd_batch *b, void *const *dF, const int64_t *ldf, const void *const *dSrc,
                            const int64_t *ldsrc, const double *const *dA, const int64_t *lda, const double *const *dB,
                            const int64_t *ldb, double *const *dX, const int64_t *ldx, const int *nrhs, int method,
                            double tol, int max_iter, double shift, int reps, int *best, double *ms, void *stream);
int mtd_batch_destroy(mtd_batch *b);
/* Autotuner: picks tile[m] and nest[m] for a batch of sizes n[m] by timing, for each
 * distinct size, trial factorisations of that size's share of the batch (seeded SPD
 * matrices on this GPU) with each candidate tile (n itself, 128, 256, 384, 512) and nested
 * sub-tile (none, 64, 128), keeping the fastest.  trial_ms (nullable): wall time spent. */
int mtd_batch_autotune(int count, const int64_t *n, int prec, int64_t *tile_out, int *nest_out, double *trial_ms,
                       void *stream);

/* ---- LU with partial pivoting (no counterpart in the reference) ----
 *
 * LAPACK dgetrf's factorisation (P A = L U, row interchanges chosen by the largest |a| of
 * each column, the first such row on ties) as a device-side task graph of one persistent
 * launch: per block column of `tile` elements a panel task whose items (at most one per SM)
 * factor the panel together, the panel's row interchanges on the other block columns, a
 * unit-lower TRSM and a GEMM update.  tile: 64 or 128 (each item keeps its panel rows in
 * shared memory, ~213 rows of 128 at most, and one item per SM: n up to ~31,000 at tile 128;
 * MTD_ERR_INVALID_ARG beyond).  d_ipiv: n device
 * ints, LAPACK's 1-based ipiv on return.  A zero pivot does not stop the factorisation; the
 * status call reports the first one as info (1-based column), as dgetrf does. */
typedef struct mtd_lupiv mtd_lupiv;
int mtd_lupiv_create(mtd_lupiv **out, int64_t n, int64_t tile);
int mtd_lupiv_num_tasks(const mtd_lupiv *h);
/* Stream-ordered; wait with mtd_lupiv_status. */
int mtd_lupiv_run(mtd_lupiv *h, double *dA, int64_t lda, int *d_ipiv, void *stream);
int mtd_lupiv_status(mtd_lupiv *h, int *info);
int mtd_lupiv_destroy(mtd_lupiv *h);
/* One call: create, run, wait, destroy. */
int mtd_lu_pivot(double *dA, int64_t n, int64_t lda, int64_t tile, int *d_ipiv, void *stream, int *info);

/* ---- Cholesky adjoint (no counterpart in the reference) ----
 *
 * Reverse-mode derivative of A = L L^T: given the factor L and Lbar = dLoss/dL (lower
 * triangles), overwrite Lbar's lower triangle with Abar = dLoss/dA, the gradient with
 * respect to the lower triangle of A (all a Cholesky factorisation reads; the symmetric
 * gradient is (Abar + Abar^T) / 2 with the diagonal kept).  A reverse sweep over the tiled
 * factorisation's block columns (tile 64, 128 or 256) with its own TRSM / GEMM / diagonal-
 * adjoint tasks, run by the persistent scheduler; many matrices of different sizes go in
 * one merged task graph and one launch.  MTD_PREC_FP64: double matrices; MTD_PREC_FP32:
 * float matrices with FP32-accurate (split-TF32) tensor-core products.  L is only read (the
 * factor of a forward pass, or recomputed); the strict upper triangles are not touched. */
typedef struct mtd_adjoint mtd_adjoint;

int mtd_adjoint_create(mtd_adjoint **out, int count, const int64_t *n, int64_t tile, int prec);
int mtd_adjoint_num_tasks(const mtd_adjoint *a);
/* Stream-ordered; dL[m] and dLbar[m] are distinct device matrices of size n[m]. */
int mtd_adjoint_run(mtd_adjoint *a, void *const *dL, const int64_t *ldl, void *const *dLbar, const int64_t *ldlb,
                    void *stream);
/* Wait for the last run; elapsed_ms (nullable) = its device time. */
int mtd_adjoint_status(mtd_adjoint *a, double *elapsed_ms);
/* Per-work-item trace of the next runs (records as mtd_graph_copy_trace's: start ns, end
 * ns, SM, task << 32 | item); mtd_adjoint_task_op gives a task's operation (internal code:
 * 20 X L^-1, 21 C -= A B, 22 C -= A^T B, 23 diagonal-tile adjoint). */
int mtd_adjoint_set_trace(mtd_adjoint *a, int enable);
long long mtd_adjoint_copy_trace(mtd_adjoint *a, unsigned long long *out, long long cap_records);
int mtd_adjoint_task_op(const mtd_adjoint *a, int task);
int mtd_adjoint_destroy(mtd_adjoint *a);
/* One matrix, synchronous. */
int mtd_cholesky_adjoint(int prec, void *dL, int64_t ldl, void *dLbar, int64_t ldlb, int64_t n, int64_t tile,
                         void *stream);

/* ---- inputs: device generators (the reference builds its input on the host,
 *      include/gen.h:23-38; these make the seeded inputs of the benchmark shapes) ---- */
int mtd_generate(double *dA, int64_t n, int64_t lda, int which, uint64_t seed, double alpha,
                 void *stream);

/* Host generator identical to the reference's include/gen.h:23-38 (glibc srand(420),
 * rand()/RAND_MAX upper triangle, mirrored, +n diagonal); writes n*n doubles. */
int mtd_generate_reference_host(double *hA, int64_t n);

/* ---- measurement ---- */

/* Measure the device's FP64 tensor-core (DMMA) rate with a register-only loop; writes
 * TFLOP/s.  Used as the roofline denominator next to the datasheet figure. */
int mtd_probe_fp64_peak(double *tflops_out);

const char *mtd_strerror(int status);
int mtd_abi_version(void);

#ifdef __cplusplus
}
#endif
#endif /* MUSTARD_B200_H */
