// The persistent scheduler: one CTA per SM pops ready work items, runs the tile
// operation, and resolves dependencies on the device.
//
// It replaces, for one GPU, the reference's device runtime (mustard/mustard.h:57-129,
// mustard/broker_queue.h): the 1-thread kernel_scheduler that dequeues task ids and
// device-launches one CUDA graph per task, the per-edge kernel_dep_update nodes that
// decrement a successor's counter and enqueue it at zero, kernel_populate_queue, and the
// occupancy throttle.  Differences, by design:
//   - a task is split into independent work items (output sub-tiles / row strips) so all
//     148 SMs can share one tile operation;
//   - the dependency decrement is fused into the epilogue of a task's last work item;
//   - three ready queues (critical path first, then by distance to the panel) replace the
//     single FIFO ring;
//   - a queue is a bounded array of 64-bit slots (task << 32 | item); a producer reserves
//     slots with a fetch-and-add on `tail`, writes them, then adds their number to `avail`;
//     a consumer first takes one unit of `avail` (fetch-and-add, undone if it was not
//     positive) and only then a slot index from `head` (fetch-and-add), so it never claims
//     a slot nobody has reserved and no claim ever retries: with 148 CTAs popping short
//     items a compare-and-swap on `head` admits about one claim per L2 round trip, which
//     starved the tensor-core items; every slot is written once per run (capacity = that
//     queue's total items);
//   - every wait is bounded by a globaltimer deadline after which the CTA records
//     MTD_ERR_TIMEOUT, raises the abort flag and returns.
#pragma once

#include "device_types.hpp"
#include "adjoint_ops.cuh"
#include "batch_ops.cuh"
#include "lupiv_ops.cuh"
#include "sync_util.cuh"
#include "tcgen05.cuh"
#include "tile_ops.cuh"

namespace mtd {

// 1: the FP64 persistent loop completes an item on thread 32 while thread 0 claims the next.
#ifndef MTD_OVERLAP_FINISH
#define MTD_OVERLAP_FINISH 0
#endif

constexpr unsigned long long kEmptySlot = ~0ull;
enum { kCmdWork = 0, kCmdExit = 1, kCmdNone = 2 };

// Signed fetch-and-add on a queue's `avail` count (two's complement in 64 bits).
__device__ __forceinline__ long long add_avail(long long *c, long long v) {
    return static_cast<long long>(
        atomicAdd(reinterpret_cast<unsigned long long *>(c), static_cast<unsigned long long>(v)));
}

// One thread of a CTA: `task` has no predecessors left.  Push its work items.  Every task
// has at least one: a join (the stand-in of a nested factorisation with several sinks) has
// one no-op item, so a release never recurses and a chain of joins needs no stack.
__device__ __forceinline__ void release_task(const RunArgs &p, int task) {
    const int q = __ldg(&p.tasks[task].queue);
    const int n_items = __ldg(&p.tasks[task].n_items);
    const unsigned long long n = static_cast<unsigned long long>(n_items);
    const unsigned long long base = atomicAdd(&p.qctl[q].tail, n);
    if (n_items <= 0 || base + n > static_cast<unsigned long long>(p.queue_cap[q])) {
        report_error(p.ctl, MTD_ERR_QUEUE, 0);
        return;
    }
    volatile unsigned long long *slots = p.queue[q];
    for (unsigned long long i = 0; i < n; ++i) slots[base + i] = (static_cast<unsigned long long>(task) << 32) | i;
    __threadfence();  // the slots before the count that lets consumers claim them
    add_avail(&p.qctl[q].avail, static_cast<long long>(n));
}

// One thread of a CTA: one attempt to claim a work item.  The exit flags and every queue's
// count are read together (one round trip); a claim is then two fetch-and-adds and the slot
// read.  kCmdNone: nothing is ready right now.
__device__ __forceinline__ int claim_item(const RunArgs &p, int *task, int *item, unsigned long long t0) {
    const int abort = ld_volatile(&p.ctl->abort);
    const int done = ld_volatile(&p.ctl->tasks_done);
    long long avail[kNumQueues];
#pragma unroll
    for (int q = 0; q < kNumQueues; ++q)
        avail[q] = static_cast<long long>(ld_volatile(reinterpret_cast<const unsigned long long *>(&p.qctl[q].avail)));
    if (abort || done >= p.n_tasks) return kCmdExit;
    for (int q = 0; q < kNumQueues; ++q) {
        if (avail[q] <= 0) continue;
        if (add_avail(&p.qctl[q].avail, -1) <= 0) {  // taken meanwhile: give the unit back
            add_avail(&p.qctl[q].avail, 1);
            continue;
        }
        // one unit of avail = one pushed, unclaimed item, so this slot is reserved
        const unsigned long long h = atomicAdd(&p.qctl[q].head, 1ull);
        const unsigned long long *slot = p.queue[q] + h;
        unsigned long long v;
        while ((v = ld_volatile(slot)) == kEmptySlot) {
            if (global_ns() - t0 > p.timeout_ns) {
                report_error(p.ctl, MTD_ERR_TIMEOUT, 0);
                return kCmdExit;
            }
            __nanosleep(20);
        }
        __threadfence();
        *task = static_cast<int>(v >> 32);
        *item = static_cast<int>(v & 0xffffffffull);
        return kCmdWork;
    }
    return kCmdNone;
}

#if MTD_EARLY_CLAIM2
// The item an FP64 update claimed ahead (early_claim), for the persistent loop's next round.
struct EarlyClaim {
    int valid, task, item;
};
static __shared__ EarlyClaim g_early;

// Thread 0 of an FP64 update item, before its last k-slice: one attempt to claim the CTA's
// next item (kept in g_early).  Not inlined, so the claim's registers are not allocated in the
// update's k-loop.
static __device__ __noinline__ void early_claim(const RunArgs &p) {
    if (g_early.valid) return;
    int tk = 0, it = 0;
    if (claim_item(p, &tk, &it, global_ns()) == kCmdWork) {
        g_early.task = tk;
        g_early.item = it;
        g_early.valid = 1;
    }
}
#endif

// One thread of a CTA: claim one work item, waiting (bounded) while none is ready.
__device__ __forceinline__ int pop_item(const RunArgs &p, int *task, int *item) {
    const unsigned long long t0 = global_ns();
    unsigned int backoff = 32;
    while (true) {
        const int cmd = claim_item(p, task, item, t0);
        if (cmd != kCmdNone) return cmd;
        if (global_ns() - t0 > p.timeout_ns) {
            report_error(p.ctl, MTD_ERR_TIMEOUT, 0);
            return kCmdExit;
        }
        __nanosleep(backoff);
        if (backoff < 256) backoff *= 2;
    }
}

// One thread of a CTA, after the threads that wrote an item of `task` passed a barrier with it.
__device__ __forceinline__ void complete_item(const RunArgs &p, int task) {
    __threadfence();
    if (atomicSub(&p.items_left[task], 1) != 1) return;
    __threadfence();
    const int sb = __ldg(&p.tasks[task].succ_begin), sc = __ldg(&p.tasks[task].succ_count);
    for (int s = 0; s < sc; ++s) {
        const int succ = __ldg(&p.succ[sb + s]);
        if (atomicSub(&p.deps[succ], 1) == 1) release_task(p, succ);
    }
    // the last task of a batched matrix (its DAG's only sink) stamps the matrix's finish time
    if (sc == 0 && p.mat_done_ns) p.mat_done_ns[__ldg(&p.tasks[task].mat)] = global_ns();
    __threadfence();
    atomicAdd(&p.ctl->tasks_done, 1);
}

// One thread, once every thread that wrote the item's results has passed a barrier with it:
// complete the item (unless it failed), count it and, when tracing, record
// (start, end, SM, task << 32 | item).
__device__ __forceinline__ void finish_item(const RunArgs &p, int task, int item, unsigned long long t_start, bool ok) {
    if (ok) complete_item(p, task);
    if (!p.trace) {
        atomicAdd(&p.ctl->items_done, 1ull);  // result unused: no round trip
        return;
    }
    const long long slot = static_cast<long long>(atomicAdd(&p.ctl->items_done, 1ull));
    if (slot < p.trace_cap) {
        unsigned int smid;
        asm volatile("mov.u32 %0, %%smid;" : "=r"(smid));
        unsigned long long *rec = p.trace + 4 * slot;
        rec[0] = t_start;
        rec[1] = global_ns();
        rec[2] = smid;
        rec[3] = (static_cast<unsigned long long>(task) << 32) | static_cast<unsigned int>(item);
    }
}

// Element type of the matrix a run factors: double (the reference's FP64 arithmetic) or
// float (low-precision Cholesky factor of the mixed-precision solver: SPLIT = 1 TF32
// products, SPLIT = 3 FP32-accurate split-TF32 products).
// ADJ: the kernel instance that runs the Cholesky adjoint's task graphs (its operations
// only), so the factorisation kernels keep their own register allocation.
// The TF32 factorisation with 16-byte aligned operands runs its GEMM and SYRK items on the
// fifth-generation tensor cores (tcgen05, accumulator in TMEM); everything else on mma.sync.
template <int VEC, typename T, int SPLIT, bool ADJ>
constexpr bool uses_tcgen05() {
    return VEC == 2 && sizeof(T) == 4 && (SPLIT == 1 || SPLIT == 3) && !ADJ;
}

// One 128 x 128 output tile of C -= A B^T (GEMM_NT) or of the lower part of C -= A A^T
// (SYRK_LN): item -> output offset (r0, c0) inside the task's tile, extent mm x nn, the first
// row and column of its B panel, and whether it is a diagonal SYRK block.
struct UpdateGeom {
    int r0, c0, mm, nn, brow, bcol;
    bool lower;
};

__device__ __forceinline__ UpdateGeom update_geom(const DevTask &t, int item) {
    UpdateGeom g;
    if (t.op == MTD_OP_SYRK_LN) {
        int pb = 0;
        while ((pb + 1) * (pb + 2) / 2 <= item) ++pb;
        const int qb = item - pb * (pb + 1) / 2;
        g.r0 = pb * kGemmTile;
        g.c0 = qb * kGemmTile;
        g.mm = min(kGemmTile, t.m - g.r0);
        g.nn = min(kGemmTile, t.m - g.c0);
        g.lower = pb == qb;
        g.brow = t.ar + g.c0;
        g.bcol = t.ac;  // SYRK's B panel starts in the same column as A; GEMM_NT's may not
    } else {
        const int nbn = (t.n + kGemmTile - 1) / kGemmTile;
        g.r0 = (item / nbn) * kGemmTile;
        g.c0 = (item % nbn) * kGemmTile;
        g.mm = min(kGemmTile, t.m - g.r0);
        g.nn = min(kGemmTile, t.n - g.c0);
        g.lower = false;
        g.brow = t.br + g.c0;
        g.bcol = t.bc;
    }
    return g;
}

enum { kTcStaged = 0, kTcTmaTf32 = 1, kTcTmaBf16 = 2, kTcTmaX3 = 3 };

// How a GEMM_NT / SYRK_LN item runs on tcgen05: BF16 operands from the BF16 copy of the
// panels when the depth is whole 128-column stages and both operand slices start on 64-row
// atoms; TF32 operands by TMA from the matrix's tensor map when the depth is whole 64-column
// stages; otherwise staged by cp.async.
__device__ __forceinline__ int tc_path(const RunArgs &p, const DevTask &t, const UpdateGeom &g, bool tmap) {
    if (t.op != MTD_OP_GEMM_NT && t.op != MTD_OP_SYRK_LN) return kTcStaged;
    if (p.tma_lo)  // FP32-accurate runs: three passes, both operand slices on 32-row atoms
        return (t.k % tc::kX3BK == 0 && t.ac == g.bcol && (t.ar + g.r0) % 32 == 0 && g.brow % 32 == 0) ? kTcTmaX3
                                                                                                     : kTcStaged;
    if (p.tma_bf16 && t.k % tc::kBfBK == 0 && t.ac == g.bcol && (t.ar + g.r0) % 64 == 0 && g.brow % 64 == 0)
        return kTcTmaBf16;
    if (tmap && t.k % tc::kTmaBK == 0 && t.ac == g.bcol) return kTcTmaTf32;
    return kTcStaged;
}

// The 1024-byte aligned start of the tcgen05 stage buffers (the swizzled layouts want it).
__device__ __forceinline__ uint8_t *tc_stages(void *smem) {
    return reinterpret_cast<uint8_t *>((reinterpret_cast<uintptr_t>(smem) + 1023) & ~uintptr_t(1023));
}

// A GEMM_NT / SYRK_LN item with cp.async-staged operands on tcgen05, start to finish (the
// persistent loop runs the TMA items itself, with their C update deferred).
__device__ __forceinline__ int op_update_tc(const RunArgs &p, const MatCtx &m, const DevTask &t, int item, void *smem,
                                            tc::State *tcs) {
    const UpdateGeom g = update_geom(t, item);
    const float *B = at<float>(m, g.brow, g.bcol);
    float *C = at<float>(m, t.cr + g.r0, t.cc + g.c0);
    const bool ok = tc::gemm_nt<kThreads>(tcs, tc_stages(smem), at<float>(m, t.ar + g.r0, t.ac), m.lda, B, m.lda, g.mm,
                                          g.nn, t.k, C, m.lda, g.lower, 0, 0, p.timeout_ns);
    if (!ok) {
        if (threadIdx.x == 0) report_error(p.ctl, MTD_ERR_TIMEOUT, 0);
        return MTD_ERR_TIMEOUT;
    }
    return 0;
}

// The solve task of a batched factor-and-solve launch (after its matrices' factorisations):
// the whole solve with refinement of matrix t.mat on this CTA (batch_ops.cuh) or, when the
// task pairs two matrices (t.pad >= 0), of t.mat on threads 0-255 and of t.pad on threads
// 256-511, each half with its own named barrier and half of the shared memory.  A matrix
// whose factorisation met a bad pivot is not solved: its backward error and step count keep
// the values the launch reset them to.  Each group stamps its matrix's finish time.
template <typename T, int NT>
__device__ __forceinline__ void batch_solve_one(const RunArgs &p, int mat, bsolve::Grp g, unsigned char *smem) {
    if (ld_volatile(p.mat_info + mat) != kBatchInfoOk) return;
    double berr = -1.0;
    int iters = 0;
    bsolve::solve_refine<T, NT>(g, p.solve[mat], static_cast<const T *>(p.ws_lower), p.solve_method, p.solve_tol,
                                p.solve_max_iter, bsolve::Smem{smem}, &berr, &iters);
    if (g.tid == 0) {
        p.solve_berr[mat] = berr;
        p.solve_iters[mat] = iters;
        if (p.mat_done_ns) p.mat_done_ns[mat] = global_ns();
    }
}
// The two forms in their own functions, each with its own register allocation (the
// half-CTA form stages twice the elements per thread).
template <typename T>
__device__ __noinline__ void batch_solve_whole(const RunArgs &p, const DevTask &t, void *smem) {
    batch_solve_one<T, kThreads>(p, t.mat, bsolve::Grp{static_cast<int>(threadIdx.x), 0},
                                 static_cast<unsigned char *>(smem));
}
template <typename T>
__device__ __noinline__ void batch_solve_halves(const RunArgs &p, const DevTask &t, void *smem) {
    constexpr int kHalf = kThreads / 2;
    const int half = static_cast<int>(threadIdx.x) / kHalf;
    batch_solve_one<T, kHalf>(p, half ? t.pad : t.mat, bsolve::Grp{static_cast<int>(threadIdx.x) % kHalf, 3 + half},
                              static_cast<unsigned char *>(smem) + half * bsolve::smem_bytes<kHalf>());
}
template <typename T>
__device__ int op_batch_solve(const RunArgs &p, const DevTask &t, void *smem) {
    static_assert(bsolve::smem_bytes<kThreads>() <= size_t(kOpSmemBytes()) &&
                      2 * bsolve::smem_bytes<kThreads / 2>() <= size_t(kOpSmemBytes()),
                  "solve scratch fits the kernel's");
    if (t.pad >= 0) batch_solve_halves<T>(p, t, smem);
    else batch_solve_whole<T>(p, t, smem);
    return 0;
}

// One 128-column strip of a batched matrix's conversion to the factor's precision (the root
// of its DAG in a low-precision factor-and-solve launch): F = lower(A) + shift I.
template <typename T>
__device__ __noinline__ int op_batch_convert(const RunArgs &p, const DevTask &t, int item) {
    const SolveMat &sm = p.solve[t.mat];
    const BatchMat bm = p.mats[t.mat];
    const int c0 = item * kConvertCols;
    bsolve::convert<T, kThreads>(bsolve::Grp{static_cast<int>(threadIdx.x), 0}, sm.a, sm.lda, static_cast<T *>(bm.a),
                                 bm.lda, sm.n, p.solve_shift, c0, min(sm.n, c0 + kConvertCols));
    return 0;
}

// SOLVE: the instances of the batched factor-and-solve launch and of the pivoted LU, which
// also run their own tasks (solve, conversion; pivoted panel, row interchanges); the other
// instances carry none of that code.
template <int VEC, typename T, int SPLIT = 1, bool ADJ = false, bool SOLVE = false, int OPS = kOpsAll>
__device__ __forceinline__ int dispatch(const RunArgs &p, const DevTask &t, int item, void *smem,
                                        tc::State *tcs = nullptr, t64::State *s64 = nullptr) {
    if constexpr (SOLVE) {
        if constexpr (OPS != kOpsLu) {
            if (t.op == kOpBatchSolve) return op_batch_solve<T>(p, t, smem);
            if (t.op == kOpBatchConvert) return op_batch_convert<T>(p, t, item);
        }
        if constexpr (sizeof(T) == 8 && OPS != kOpsCholesky) {
            if (t.op == kOpPanelPiv) return op_panel_piv(p, mat_ctx<T>(p, t), t, item, smem);
            if (t.op == kOpLaswp) return op_laswp(p, mat_ctx<T>(p, t), t, item, smem);
        }
    }
    if (t.op == kOpJoin) return 0;  // a join's one item: nothing to compute
    if constexpr (ADJ) return dispatch_adjoint<T, VEC, SPLIT>(p, t, item, smem);
    const MatCtx m = mat_ctx<T>(p, t);
    // single-pass TF32 runs stage their other updates for tcgen05 too; FP32-accurate runs keep
    // them on the three-product mma.sync path
    if constexpr (uses_tcgen05<VEC, T, SPLIT, ADJ>() && SPLIT == 1)
        if (t.op == MTD_OP_GEMM_NT || t.op == MTD_OP_SYRK_LN) return op_update_tc(p, m, t, item, smem, tcs);
    if constexpr (sizeof(T) == 8) {
        if constexpr (OPS != kOpsLu) {
            switch (t.op) {
            case MTD_OP_POTRF: return op_potrf<T, VEC>(p, m, t, smem);
            case MTD_OP_TRSM_RLT: return op_trsm_rlt<T, VEC>(p, m, t, item, smem);
            case MTD_OP_SYRK_LN: return op_syrk_ln<T, VEC>(p, m, t, item, smem, s64);
            case MTD_OP_GEMM_NT: return op_gemm_nt<T, VEC>(p, m, t, item, smem, s64);
            default: break;
            }
        }
        if constexpr (OPS != kOpsCholesky) {
            switch (t.op) {
            case MTD_OP_GETRF: return op_getrf<VEC>(p, m, t, smem);
            case MTD_OP_TRSM_LLNU: return op_trsm_llnu<VEC>(p, m, t, item, smem);
            case MTD_OP_TRSM_RUN: return op_trsm_run<VEC>(p, m, t, item, smem);
            case MTD_OP_GEMM_NN: return op_gemm_nn<VEC>(p, m, t, item, smem, s64);
            default: break;
            }
        }
    } else {
        switch (t.op) {
        case MTD_OP_POTRF: return op_potrf<T, VEC, SPLIT>(p, m, t, smem);
        case MTD_OP_TRSM_RLT: return op_trsm_rlt<T, VEC, SPLIT>(p, m, t, item, smem);
        case MTD_OP_SYRK_LN: return op_syrk_ln<T, VEC, SPLIT>(p, m, t, item, smem);
        case MTD_OP_GEMM_NT: return op_gemm_nt<T, VEC, SPLIT>(p, m, t, item, smem);
        default: break;
        }
    }
    if (threadIdx.x == 0) report_error(p.ctl, MTD_ERR_INVALID_ARG, 0);
    return MTD_ERR_INVALID_ARG;
}

__device__ __forceinline__ void load_task(const RunArgs &p, int task, DevTask *t) {
    const int4 *src = reinterpret_cast<const int4 *>(p.tasks + task);
    int4 *dst = reinterpret_cast<int4 *>(t);
#pragma unroll
    for (int w = 0; w < int(sizeof(DevTask) / sizeof(int4)); ++w) dst[w] = __ldg(src + w);
}

// Named barrier 1 over the threads of warps 1 .. 15 (barrier 0 is __syncthreads).
__device__ __forceinline__ void sync_drain_warps() {
    asm volatile("bar.sync 1, %0;" ::"r"(kThreads - 32) : "memory");
}

// The persistent loop of the tcgen05 kernel (TF32 / BF16 Cholesky factor).  A TMA item
// (GEMM_NT / SYRK_LN with operands fetched by TMA) runs its loads and MMAs on thread 0 into
// one of the two TMEM accumulators while warps 1 .. 15 fetch its C values into registers;
// its C update is deferred to the top of the next iteration, where warps 1 .. 15 write it
// and thread 32 completes the item (releasing its successors) while thread 0 claims the
// next item.  So a TMA item's C reads overlap its own MMAs, and its C update and completion
// overlap the next claim.  The claim may wait: the pending item's completion never depends
// on thread 0.  The next TMA item writes the other accumulator.
// (Measured against the alternatives on one B200, Cholesky N = 32768, tile 1536: deferring
// the C update further, into the next item's MMAs, or starting those MMAs before the C
// update ends, streams GEMM items faster but completes them later, and the factorisation,
// which waits on its dependency chain, comes out slower.)
template <int VEC, typename T, int SPLIT, bool SOLVE = false>
__device__ __forceinline__ void persistent_loop_tc(const RunArgs &p, double *smem, tc::State &tcs) {
    __shared__ int s_cmd, s_task, s_item;
    __shared__ tc::Pending pend;
    __shared__ uint32_t s_buf;       // thread 0: the accumulator the next TMA item writes
    float cv[tc::kDrainChunks][16];  // warps 1 .. 15: the pending item's C values
    if (threadIdx.x == 0) {
        pend.valid = 0;
        s_buf = 0;
    }
    __syncthreads();
    while (true) {
        if (threadIdx.x == 0) {
            int tk = 0, it = 0;
            s_cmd = pop_item(p, &tk, &it);
            s_task = tk;
            s_item = it;
        } else if (threadIdx.x >= 32 && pend.valid) {
            tc::drain(pend, cv);
            sync_drain_warps();
            if (threadIdx.x == 32) finish_item(p, pend.task, pend.item, pend.t_start, true);
        }
        __syncthreads();
        const int cmd = s_cmd, task = s_task, item = s_item;
        if (cmd != kCmdWork) break;
        if (threadIdx.x == 0) pend.valid = 0;  // drained above; read again only after a barrier
        const unsigned long long t_start = p.trace ? global_ns() : 0ull;
        DevTask t;
        load_task(p, task, &t);
        const UpdateGeom g = update_geom(t, item);
        const int path = tc_path(p, t, g, p.tma != 0);
        if (path != kTcStaged) {
            const MatCtx m = mat_ctx<T>(p, t);
            float *C = at<float>(m, t.cr + g.r0, t.cc + g.c0);
            if (threadIdx.x == 0) {
                const uint32_t acc = tcs.taddr + tc::kAccCols * s_buf;
                // the tensor maps' addresses are taken on the kernel parameter itself
                const bool ok =
                    path == kTcTmaBf16
                        ? tc::mainloop_tma_bf16(&tcs, tc_stages(smem), p.tmap_bf16, t.ar + g.r0, g.brow, t.ac, t.k, acc,
                                                p.timeout_ns)
                    : path == kTcTmaX3
                        ? tc::mainloop_tma_x3(&tcs, tc_stages(smem), p.tmap, p.tmap_lo, t.ar + g.r0, g.brow, t.ac, t.k,
                                              acc, p.timeout_ns)
                        : tc::mainloop_tma(&tcs, tc_stages(smem), p.tmap, p.tma, t.ar + g.r0, g.brow, t.ac, t.k, acc,
                                           p.timeout_ns);
                if (ok) {
                    pend.C = C;
                    pend.ldc = m.lda;
                    pend.M = g.mm;
                    pend.N = g.nn;
                    pend.lower = g.lower ? 1 : 0;
                    pend.task = task;
                    pend.item = item;
                    pend.t_start = t_start;
                    pend.acc = acc;
                    pend.valid = 1;
                    s_buf ^= 1u;
                } else {
                    report_error(p.ctl, MTD_ERR_TIMEOUT, 0);
                }
            } else if (threadIdx.x >= 32) {
                tc::prefetch_c(C, m.lda, g.mm, g.nn, g.lower, cv);
            }
            __syncthreads();
            continue;
        }
        const int st = dispatch<VEC, T, SPLIT, false, SOLVE>(p, t, item, smem, &tcs);
        // nothing is pending here (drained above): redefining cv after the tile operation
        // frees its registers during it
#pragma unroll
        for (int c = 0; c < tc::kDrainChunks; ++c)
#pragma unroll
            for (int j = 0; j < 16; ++j) cv[c][j] = 0.f;
        __syncthreads();
        if (threadIdx.x == 0) finish_item(p, task, item, t_start, st == 0);
    }
}

// Named barrier 2 over warps 2 .. 15 (the warp-specialised loop's drain warps).
__device__ __forceinline__ void sync_ws_drain_warps() { asm volatile("bar.sync 2, %0;" ::"r"(kThreads - 64) : "memory"); }

// The persistent loop of the tcgen05 kernel on the warp-specialised pipeline (tcgen05.cuh,
// ws_*).  One item per round, taken from one of two claim slots:
//   - a TMA item (GEMM_NT / SYRK_LN with TMA operands): thread 0 loads its slices and then
//     tries once to claim the next item into the other slot (never waiting: this item
//     completes only in the next round, and the work a waiting claim would wait for may be
//     its successors); if nothing was ready, the next round starts with thread 0 waiting for
//     an item while warps 2 .. 15 complete this one; thread 32 issues its MMAs into accumulator
//     `buf`; warps 2 .. 15 first update C from the previous TMA item's accumulator (waiting on
//     its accf barrier; thread 64 then completes that item) and then prefetch this item's C.
//     The round ends when all three are done, so the previous item's C update and this
//     item's loads and MMAs overlap, and the next item's loads queue behind this item's MMAs;
//   - any other item: warps 2 .. 15 finish the pending TMA item first (its MMAs are then done,
//     so the ring's shared memory is free), then all threads run the item as the plain loop
//     does, and thread 0 completes it and claims the next.
// Every wait is bounded by the run's timeout; an expired wait raises the error (abort) and
// the loop drains what it has started before leaving.
template <int VEC, typename T, int SPLIT>
__device__ __forceinline__ void persistent_loop_ws(const RunArgs &p, double *smem, tc::State &tcs, tc::WsState &ws) {
    __shared__ int s_cmd[2], s_task[2], s_item[2];
    float cv[tc::kWsDrainChunks][16];  // warps 2 .. 15: the pending item's C values
    // warps 2 .. 15: the pending TMA item (its accumulator is being computed or is final)
    bool pv = false;
    float *pC = nullptr;
    int64_t pld = 0;
    int pM = 0, pN = 0, plower = 0, ptask = 0, pitem = 0, pbuf = 0;
    unsigned long long pt0 = 0;
    uint32_t uses0 = 0, uses1 = 0;  // items drained from each accumulator (accf parities)
    int buf = 0;
    const int warp = threadIdx.x >> 5;
    uint8_t *ring = tc_stages(smem);
    auto drain_pending = [&]() {  // warps 2 .. 15
        if (!pv) return;
        const uint32_t par = (pbuf ? uses1 : uses0) & 1u;
        const bool ok = tc::wait_bar(&ws.accf[pbuf], par, global_ns() + p.timeout_ns);
        if (pbuf) ++uses1;
        else ++uses0;
        if (ok) tc::ws_drain(tcs.taddr + tc::kAccCols * pbuf, pC, pld, pM, pN, plower != 0, cv);
        sync_ws_drain_warps();
        if (threadIdx.x == 64) {
            if (!ok) report_error(p.ctl, MTD_ERR_TIMEOUT, 0);
            finish_item(p, ptask, pitem, pt0, ok);
        }
        pv = false;
    };
    if (threadIdx.x == 0) s_cmd[0] = kCmdNone;
    __syncthreads();
    for (int r = 0;; ++r) {
        const int slot = r & 1;
        if (s_cmd[slot] == kCmdNone) {
            // nothing claimed yet: thread 0 waits for an item while warps 2 .. 15 complete the
            // pending one, which may be the item that releases the work it waits for
            if (threadIdx.x == 0) {
                int tk = 0, it = 0;
                s_cmd[slot] = pop_item(p, &tk, &it);
                s_task[slot] = tk;
                s_item[slot] = it;
            } else if (warp >= 2) {
                drain_pending();
            }
            __syncthreads();
        }
        const int cmd = s_cmd[slot], task = s_task[slot], item = s_item[slot];
        if (cmd != kCmdWork) {
            if (warp >= 2) drain_pending();
            break;
        }
        const unsigned long long t_start = p.trace ? global_ns() : 0ull;
        DevTask t;
        load_task(p, task, &t);
        const UpdateGeom g = update_geom(t, item);
        int path = tc_path(p, t, g, p.tma != 0);
        if (path == kTcTmaX3) path = kTcStaged;  // three-pass items run on the single-thread pipeline only
        if (path != kTcStaged) {
            const MatCtx m = mat_ctx<T>(p, t);
            float *C = at<float>(m, t.cr + g.r0, t.cc + g.c0);
            const int kind = path == kTcTmaBf16 ? tc::kWsBf16 : (p.tma == tc::kTmaMap3D ? tc::kWsTf32Map3D : tc::kWsTf32Map2D);
            if (threadIdx.x == 0) {
                const void *map = path == kTcTmaBf16 ? static_cast<const void *>(p.tmap_bf16) : static_cast<const void *>(p.tmap);
                if (!tc::ws_load(&ws, ring, map, kind, t.ar + g.r0, g.brow, t.ac, t.k, global_ns() + p.timeout_ns))
                    report_error(p.ctl, MTD_ERR_TIMEOUT, 0);
                // one attempt, never a wait: this item completes only in the next round, and
                // what a waiting claim would wait for may be its successors
                int tk = 0, it = 0;
                s_cmd[slot ^ 1] = claim_item(p, &tk, &it, global_ns());
                s_task[slot ^ 1] = tk;
                s_item[slot ^ 1] = it;
            } else if (threadIdx.x == 32) {
                if (!tc::ws_mma(&ws, ring, kind, t.k, tcs.taddr + tc::kAccCols * buf, buf, global_ns() + p.timeout_ns))
                    report_error(p.ctl, MTD_ERR_TIMEOUT, 0);
            } else if (warp >= 2) {
                drain_pending();
                tc::ws_prefetch_c(C, m.lda, g.mm, g.nn, g.lower, cv);
                pv = true;
                pC = C;
                pld = m.lda;
                pM = g.mm;
                pN = g.nn;
                plower = g.lower ? 1 : 0;
                ptask = task;
                pitem = item;
                pt0 = t_start;
                pbuf = buf;
            }
            buf ^= 1;
            __syncthreads();
            continue;
        }
        if (warp >= 2) drain_pending();
        __syncthreads();
        const int st = dispatch<VEC, T, SPLIT, false>(p, t, item, smem, &tcs);
        // nothing is pending here: redefining cv after the tile operation frees its registers
#pragma unroll
        for (int c = 0; c < tc::kWsDrainChunks; ++c)
#pragma unroll
            for (int j = 0; j < 16; ++j) cv[c][j] = 0.f;
        __syncthreads();
        if (threadIdx.x == 0) {
            finish_item(p, task, item, t_start, st == 0);
            int tk = 0, it = 0;
            s_cmd[slot ^ 1] = pop_item(p, &tk, &it);
            s_task[slot ^ 1] = tk;
            s_item[slot ^ 1] = it;
        }
        __syncthreads();
    }
    // leave nothing in flight: thread 0 waits (bounded) for loads no MMA consumed, thread 32
    // for its MMAs
    __syncthreads();
    if (threadIdx.x == 0) {
        const unsigned long long grace = global_ns() + 1000000ull;
        for (uint32_t g = ws.cons; g < ws.prod; ++g) tc::wait_bar(&ws.full[g % tc::kWsStages], (g / tc::kWsStages) & 1u, grace);
    } else if (threadIdx.x == 32) {
        tc::ws_quiesce(&ws, global_ns() + 1000000ull);
    }
}

// T64: the instance whose FP64 GEMM / SYRK items may read their operands by TMA (tma64.cuh,
// runs that carry the tensor maps); the other instances carry none of that code.
// SOLVE: the batched factor-and-solve launch's instances (see dispatch).
// OPS: the operation family the instance carries (kOpsAll: every operation).
template <int VEC, typename T, int SPLIT = 1, bool ADJ = false, bool T64 = false, bool SOLVE = false,
          int OPS = kOpsAll>
__global__ void __launch_bounds__(kThreads, 1) persistent_kernel(const __grid_constant__ RunArgs p) {
    extern __shared__ __align__(128) double smem[];
    constexpr bool kTc = uses_tcgen05<VEC, T, SPLIT, ADJ>();
    if (threadIdx.x == 0) atomicMin(&p.ctl->start_ns, global_ns());
    if constexpr (kTc) {
        __shared__ tc::State tcs;
        if (MTD_TC_WS && !SOLVE) {
            __shared__ tc::WsState ws;
            tc::ws_init(&ws);
            tc::init(&tcs);  // TMEM accumulators and the staged items' barriers; its barrier publishes ws
            persistent_loop_ws<VEC, T, SPLIT>(p, smem, tcs, ws);
        } else {
            tc::init(&tcs);  // TMEM accumulators and barriers, held for the whole run
            persistent_loop_tc<VEC, T, SPLIT, SOLVE>(p, smem, tcs);
        }
        tc::release(&tcs);
        return;
    } else {
        __shared__ int s_cmd, s_task, s_item;
        // FP64 factorisations: barriers of the TMA-fed GEMM / SYRK items (tma64.cuh), kept
        // for the whole run (the items use them only when the run carries tensor maps)
        __shared__ t64::State s64;
        constexpr bool kT64 = T64 && sizeof(T) == 8 && !ADJ;
        if constexpr (kT64) t64::init(&s64);
#if MTD_OVERLAP_FINISH
        // thread 32 completes the previous item (releasing its successors) while thread 0
        // claims the next one; a claim that waits for those successors ends when thread 32
        // has released them
        __shared__ int s_st;
        int prev_task = -1, prev_item = 0, prev_ok = 0;
        unsigned long long prev_start = 0ull;
        while (true) {
            if (threadIdx.x == 0) {
                int tk = 0, it = 0;
                s_cmd = pop_item(p, &tk, &it);
                s_task = tk;
                s_item = it;
            } else if (threadIdx.x == 32 && prev_task >= 0) {
                finish_item(p, prev_task, prev_item, prev_start, prev_ok != 0);
            }
            __syncthreads();
            const int cmd = s_cmd, task = s_task, item = s_item;
            if (cmd != kCmdWork) break;
            const unsigned long long t_start = p.trace ? global_ns() : 0ull;
            DevTask t;
            load_task(p, task, &t);
            const int st = dispatch<VEC, T, SPLIT, ADJ, SOLVE, OPS>(p, t, item, smem, nullptr, kT64 ? &s64 : nullptr);
            if (threadIdx.x == 0) s_st = st;
            __syncthreads();
            prev_task = task;
            prev_item = item;
            prev_start = t_start;
            prev_ok = s_st == 0;
        }
#else
#if MTD_EARLY_CLAIM2
        if (threadIdx.x == 0) g_early.valid = 0;
#endif
        while (true) {
            if (threadIdx.x == 0) {
                int tk = 0, it = 0;
#if MTD_EARLY_CLAIM2
                if (g_early.valid) {  // claimed during the previous item
                    s_cmd = kCmdWork;
                    tk = g_early.task;
                    it = g_early.item;
                    g_early.valid = 0;
                } else {
                    s_cmd = pop_item(p, &tk, &it);
                }
#else
                s_cmd = pop_item(p, &tk, &it);
#endif
                s_task = tk;
                s_item = it;
            }
            __syncthreads();
            const int cmd = s_cmd, task = s_task, item = s_item;
            if (cmd != kCmdWork) break;
            const unsigned long long t_start = p.trace ? global_ns() : 0ull;
            DevTask t;
            load_task(p, task, &t);
            const int st = dispatch<VEC, T, SPLIT, ADJ, SOLVE, OPS>(p, t, item, smem, nullptr, kT64 ? &s64 : nullptr);
            __syncthreads();
            if (threadIdx.x == 0) finish_item(p, task, item, t_start, st == 0);
        }
#endif
    }
}

// One task as an ordinary launch (grid = its work items): the node kernel of the
// host-launched CUDA-graph executor, the reference's --tiled mode
// (mustard/mustard.h:155-159, cholesky_mustard.cu:498-513).
template <int VEC, typename T>
__global__ void __launch_bounds__(kThreads, 1) task_kernel(const RunArgs p, int task) {
    extern __shared__ __align__(128) double smem[];
    if (ld_volatile(&p.ctl->abort)) return;
    const DevTask t = p.tasks[task];
    if (t.n_items > 0) dispatch<VEC, T>(p, t, static_cast<int>(blockIdx.x), smem);
}

static __global__ void reset_ctl_kernel(const RunArgs p) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        p.ctl->tasks_done = 0;
        p.ctl->error = 0;
        p.ctl->info = 0x7fffffff;
        p.ctl->abort = 0;
        p.ctl->items_done = 0;
        p.ctl->start_ns = ~0ull;
    }
}

// Per-run reset: counters from their initial values, queues empty.
static __global__ void reset_kernel(const RunArgs p, const int *deps_init) {
    const long long stride = static_cast<long long>(gridDim.x) * blockDim.x;
    const long long tid = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    for (long long i = tid; i < p.n_tasks; i += stride) {
        p.deps[i] = deps_init[i];
        p.items_left[i] = p.tasks[i].n_items;
    }
    for (long long i = tid; i < p.n_panel_bar; i += stride) p.panel_bar[i] = 0u;
    for (int q = 0; q < kNumQueues; ++q)
        for (long long i = tid; i < p.queue_cap[q]; i += stride) p.queue[q][i] = kEmptySlot;
    if (tid == 0) {
        for (int q = 0; q < kNumQueues; ++q) {
            p.qctl[q].head = 0;
            p.qctl[q].tail = 0;
            p.qctl[q].avail = 0;
        }
        p.ctl->tasks_done = 0;
        p.ctl->error = 0;
        p.ctl->info = 0x7fffffff;
        p.ctl->abort = 0;
        p.ctl->items_done = 0;
        p.ctl->start_ns = ~0ull;
    }
}

// Seed the queues with the tasks that have no predecessor (kernel_populate_queue,
// mustard/mustard.h:87-95), in root order within each queue.  One block: each thread takes a
// contiguous run of roots, a scan of the per-thread item counts gives every run its slots,
// and each queue's counters are published once at the end.  (A batched run seeds thousands
// of roots; pushing them one at a time, each behind a memory fence, took ~6 ms for 4096.)
constexpr int kSeedThreads = 1024;
static __global__ void __launch_bounds__(kSeedThreads) seed_kernel(const RunArgs p, const int *roots, int n_roots) {
    __shared__ long long cnt[kNumQueues][kSeedThreads];
    __shared__ long long total[kNumQueues];
    const int tid = threadIdx.x;
    const int per = (n_roots + kSeedThreads - 1) / kSeedThreads;
    const int r0 = min(n_roots, tid * per), r1 = min(n_roots, r0 + per);
    long long c[kNumQueues] = {};
    for (int r = r0; r < r1; ++r) {
        const int task = roots[r];
        c[p.tasks[task].queue] += p.tasks[task].n_items;
    }
#pragma unroll
    for (int q = 0; q < kNumQueues; ++q) cnt[q][tid] = c[q];
    __syncthreads();
    if (tid < kNumQueues) {  // exclusive scan of queue tid's counts
        long long run = 0;
        for (int i = 0; i < kSeedThreads; ++i) {
            const long long v = cnt[tid][i];
            cnt[tid][i] = run;
            run += v;
        }
        total[tid] = run;
    }
    __syncthreads();
    long long off[kNumQueues];
#pragma unroll
    for (int q = 0; q < kNumQueues; ++q) off[q] = cnt[q][tid];
    for (int r = r0; r < r1; ++r) {
        const int task = roots[r];
        const int q = p.tasks[task].queue, n = p.tasks[task].n_items;
        if (off[q] + n > p.queue_cap[q]) break;  // reported below
        for (int i = 0; i < n; ++i)
            p.queue[q][off[q] + i] = (static_cast<unsigned long long>(task) << 32) | static_cast<unsigned int>(i);
        off[q] += n;
    }
    __threadfence();  // the slots before the counts that let consumers claim them
    __syncthreads();
    if (tid == 0) {
        for (int q = 0; q < kNumQueues; ++q) {
            if (total[q] > p.queue_cap[q]) {
                report_error(p.ctl, MTD_ERR_QUEUE, 0);
                continue;
            }
            p.qctl[q].tail = static_cast<unsigned long long>(total[q]);
            add_avail(&p.qctl[q].avail, total[q]);
        }
        __threadfence();
    }
}

}  // namespace mtd
