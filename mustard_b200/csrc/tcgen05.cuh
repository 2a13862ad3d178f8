// Fifth-generation tensor cores (tcgen05) for the TF32 GEMM items of the low-precision
// factorisation: C(M x N) -= A(M x K) * B(N x K)^T with M, N <= 128, FP32 operands in HBM
// (column-major, A and B both MN-contiguous), FP32 accumulation in tensor memory (TMEM).
//
// Operands are staged by 16-byte cp.async pieces straight into the MN-major layout that
// 32-bit operands need (the "128-byte swizzle with 32-byte atoms" mode; with no swizzle a
// TF32 MN-major MMA reads zeros): atoms of 4 K-rows x 128 bytes (32 FP32 along MN), the
// 32-byte chunks of row r stored at chunk index (c ^ r); MN-adjacent atoms kAtomMN = 512
// bytes apart, K-adjacent atoms kAtomK = 2 KB apart.  Each piece is rounded to nearest TF32 in
// shared memory before the MMAs read it (the tensor core reads the TF32 part of each FP32
// bit pattern).  One thread issues tcgen05.mma (M = N = 128, K = 8 per instruction) for a
// stage and commits the group to that stage's mbarrier; the stage's buffer is refilled only
// after the barrier says the MMAs that read it are done.  The epilogue reads the accumulator
// with tcgen05.ld (warp w: TMEM lanes 32 (w % 4) .., columns 32 (w / 4) ..) and updates C.
// Items whose operands come by TMA (mainloop_tma, mainloop_tma_bf16) run their pipeline on
// thread 0 alone, into one of two accumulators; the scheduler defers their C update
// (prefetch_c during the MMAs, drain afterwards, both by warps 1 .. 15).
//
// Every mbarrier wait is bounded by a %globaltimer deadline; on expiry the caller's error
// word is set and the item ends (its result is then not used: the run reports the error).
#pragma once

#include <cstdint>

#include "device_types.hpp"

namespace mtd {
namespace tc {

constexpr int kM = 128, kN = 128;     // MMA shape (one CTA)
constexpr int kBK = 32;               // K per stage (4 MMAs of K = 8)
constexpr int kStages = 6;            // up to 5 stages (160 KB) in flight: items are bandwidth-bound
constexpr int kAtomMN = 512;          // bytes between MN-adjacent atoms (4 x 128-byte rows)
constexpr int kAtomK = 4 * kAtomMN;   // bytes between K-adjacent atoms (4 MN atoms cover 128)
constexpr int kOperandBytes = (kBK / 4) * kAtomK;    // 128 x 32 FP32 = 16 KB
constexpr int kStageBytes = 2 * kOperandBytes;       // A and B
constexpr int kSmemBytes = kStages * kStageBytes;    // 192 KB
// Two 128-column FP32 accumulators: the TMA items alternate between them, so one item's
// MMAs run while the previous item's accumulator is still being read out (see drain).
constexpr uint32_t kAccCols = 128;
constexpr uint32_t kTmemCols = 2 * kAccCols;

// Instruction descriptor: F32 accumulator, TF32 A and B, both MN-major, M = 128, N = 128.
constexpr uint32_t kIdescTf32 = (1u << 4) | (2u << 7) | (2u << 10) | (1u << 15) | (1u << 16) |
                                (uint32_t(kN >> 3) << 17) | (uint32_t(kM >> 4) << 24);

struct State {
    uint64_t mbar[kStages];  // MMAs reading stage s are done (tcgen05.commit)
    uint64_t full[kStages];  // stage s is loaded (TMA complete_tx)
    uint32_t taddr;          // TMEM base address (lane 0, first allocated column)
    uint32_t phases;         // bit s: parity of the next completion of mbar[s]
    uint32_t fphases;        // bit s: parity of the next completion of full[s]
};

__device__ __forceinline__ uint32_t smem_addr(const void *p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Shared-memory matrix descriptor for the swizzled MN-major layout: start address, leading
// byte offset (between MN atoms) and stride byte offset (between K atoms) in 16-byte units,
// descriptor version 1, layout type 1 (128-byte swizzle, 32-byte atoms).
__device__ __forceinline__ uint64_t make_desc(uint32_t saddr) {
    return uint64_t((saddr >> 4) & 0x3fff) | (uint64_t((kAtomMN >> 4) & 0x3fff) << 16) |
           (uint64_t((kAtomK >> 4) & 0x3fff) << 32) | (1ull << 46) | (1ull << 61);
}

// Byte offset in an operand stage of the 16-byte piece holding elements (mn .. mn+3, k):
// atom (mn / 32, k / 4), row k % 4, 32-byte chunk (mn % 32) / 8 swizzled with the row.
__device__ __forceinline__ int piece_offset(int mn, int k) {
    const int row = k & 3, cb = (mn & 31) * 4;  // byte column inside the 128-byte row
    const int chunk = ((cb >> 5) ^ row) & 3;
    return (mn >> 5) * kAtomMN + (k >> 2) * kAtomK + row * 128 + (chunk << 5) + (cb & 16);
}

__device__ __forceinline__ unsigned long long now_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Once per CTA, all threads: TMEM for the accumulator and the stage barriers.
__device__ __forceinline__ void init(State *st) {
    if (threadIdx.x < 32) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(&st->taddr)),
                     "r"(kTmemCols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
    }
    if (threadIdx.x == 0) {
        for (int s = 0; s < kStages; ++s) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(&st->mbar[s])), "r"(1));
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(&st->full[s])), "r"(1));
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        st->phases = 0;
        st->fphases = 0;
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

// Once per CTA, all threads, after the last use.
__device__ __forceinline__ void release(State *st) {
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (threadIdx.x < 32)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(st->taddr), "r"(kTmemCols));
}

// Wait for the completion of parity `parity` of the barrier; false on timeout.
__device__ __forceinline__ bool wait_bar(uint64_t *bar, uint32_t parity, unsigned long long deadline) {
    const uint32_t a = smem_addr(bar);
    for (unsigned it = 0;; ++it) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(a), "r"(parity)
            : "memory");
        if (done) return true;
        if ((it & 255) == 255 && now_ns() > deadline) return false;
    }
}

__device__ __forceinline__ void cp16(uint32_t dst, const void *src, int bytes) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(dst), "l"(src), "r"(bytes) : "memory");
}

// Pieces of a stage: e -> (operand, K atom, MN atom, row, piece in row); 32 consecutive e
// fill one 512-byte atom (conflict-free) from four 128-byte runs of consecutive columns.
constexpr int kPieces = 2 * (kBK / 4) * 4 * 4 * 8;  // operands x K atoms x MN atoms x rows x pieces
__device__ __forceinline__ void piece_of(int e, int &op, int &mn, int &k) {
    const int p8 = e & 7, r4 = (e >> 3) & 3, am = (e >> 5) & 3, ka = (e >> 7) & 7;
    op = e >> 10;
    mn = am * 32 + p8 * 4;
    k = ka * 4 + r4;
}

// Stage k-slice k0 of A (rows m < M) and B (rows n < N), thread-owned pieces e = tid + 512 i.
template <int THREADS>
__device__ __forceinline__ void load_stage(uint8_t *stage, const float *A, int64_t lda, const float *B, int64_t ldb,
                                           int M, int N, int K, int k0) {
    for (int e = threadIdx.x; e < kPieces; e += THREADS) {
        int op, r, kl;
        piece_of(e, op, r, kl);
        const int kk = k0 + kl;
        const int lim = op ? N : M;
        const int rows = kk < K ? min(4, max(0, lim - r)) : 0;
        const float *src = op ? B + r + int64_t(kk) * ldb : A + r + int64_t(kk) * lda;
        cp16(smem_addr(stage + op * kOperandBytes + piece_offset(r, kl)), rows ? src : (op ? B : A), rows * 4);
    }
}

// Round this thread's pieces of the stage to nearest TF32, in place.
template <int THREADS>
__device__ __forceinline__ void round_stage(uint8_t *stage) {
    for (int e = threadIdx.x; e < kPieces; e += THREADS) {
        int op, r, kl;
        piece_of(e, op, r, kl);
        float4 *p = reinterpret_cast<float4 *>(stage + op * kOperandBytes + piece_offset(r, kl));
        float4 v = *p;
        uint32_t x, y, z, w;
        asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(x) : "f"(v.x));
        asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(y) : "f"(v.y));
        asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(z) : "f"(v.z));
        asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(w) : "f"(v.w));
        *p = make_float4(__uint_as_float(x), __uint_as_float(y), __uint_as_float(z), __uint_as_float(w));
    }
}

// This thread's 32 elements of C in the epilogue's layout (row 32 (w % 4) + lane, columns
// 32 (w / 4) ..), loaded back to back so that their latencies overlap (elements outside
// the block, or above the diagonal with lower_only, read as 0 and are not written back).
__device__ __forceinline__ void load_c(float (&cv)[32], int M, int N, const float *C, int64_t ldc, bool lower_only,
                                       int r0, int c0) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int row = (warp & 3) * 32 + lane, col0 = (warp >> 2) * 32;
#pragma unroll
    for (int j = 0; j < 32; ++j) {
        const int col = col0 + j;
        const bool in = row < M && col < N && (!lower_only || row + r0 >= col + c0);
        cv[j] = in ? __ldcg(C + row + int64_t(col) * ldc) : 0.f;
    }
}

// C = cv - accumulator (all threads; warp w reads TMEM lanes 32 (w % 4) .. and columns
// 32 (w / 4) ..; cv from load_c), then release the accumulator for the next item.
__device__ __forceinline__ bool epilogue(State *st, bool ok, const float (&cv)[32], int M, int N, float *C,
                                         int64_t ldc, bool lower_only, int r0, int c0) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int row = (warp & 3) * 32 + lane, col0 = (warp >> 2) * 32;
    const uint32_t taddr = st->taddr + (uint32_t((warp & 3) * 32) << 16) + uint32_t(col0);
#pragma unroll
    for (int h = 0; h < 2; ++h) {  // two halves of 16 columns: fewer live registers
        uint32_t v[16];
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
            : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
              "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
            : "r"(taddr + 16 * h));
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
        if (ok && row < M) {
#pragma unroll
            for (int j = 0; j < 16; ++j) {
                const int col = col0 + 16 * h + j;
                if (col < N && (!lower_only || row + r0 >= col + c0))
                    C[row + int64_t(col) * ldc] = cv[16 * h + j] - __uint_as_float(v[j]);
            }
        }
    }
    // the next item's MMAs overwrite the accumulator only after every warp has read it
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    return ok;
}

// C -= A B^T over K, M, N <= 128 (C(r, c) with r + r0 >= c + c0 only, when lower_only).
// All THREADS threads of the CTA call it; `smem` holds kSmemBytes (1024-byte aligned).
// Returns false if a wait timed out.
template <int THREADS>
__device__ bool gemm_nt(State *st, uint8_t *smem, const float *A, int64_t lda, const float *B, int64_t ldb, int M,
                        int N, int K, float *C, int64_t ldc, bool lower_only, int r0, int c0,
                        unsigned long long timeout_ns) {
    static_assert(THREADS == 512, "epilogue: 16 warps cover 4 lane quarters x 4 column quarters of 128 x 128");
    const unsigned long long deadline = now_ns() + timeout_ns;
    const int nk = (K + kBK - 1) / kBK;
    uint32_t phases = st->phases;
    bool ok = true;
#pragma unroll
    for (int s = 0; s < kStages - 1; ++s) {
        if (s < nk) load_stage<THREADS>(smem + s * kStageBytes, A, lda, B, ldb, M, N, K, s * kBK);
        asm volatile("cp.async.commit_group;\n" ::: "memory");
    }
    for (int kt = 0; kt < nk; ++kt) {
        const int s = kt % kStages;
        uint8_t *stage = smem + s * kStageBytes;
        asm volatile("cp.async.wait_group %0;\n" ::"n"(kStages - 2) : "memory");
        round_stage<THREADS>(stage);
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        if (threadIdx.x == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const uint32_t a0 = smem_addr(stage), b0 = a0 + kOperandBytes;
#pragma unroll
            for (int g = 0; g < kBK / 8; ++g) {
                const uint64_t ad = make_desc(a0 + g * 2 * kAtomK), bd = make_desc(b0 + g * 2 * kAtomK);
                const uint32_t acc = (kt > 0 || g > 0) ? 1u : 0u;
                asm volatile(
                    "{\n\t.reg .pred p;\n\t"
                    "setp.ne.b32 p, %4, 0;\n\t"
                    "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}"
                    ::"r"(st->taddr), "l"(ad), "l"(bd), "r"(kIdescTf32), "r"(acc)
                    : "memory");
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                             smem_addr(&st->mbar[s]))
                         : "memory");
        }
        // refill the stage used by k-slice kt - 1 once its MMAs are done
        if (kt > 0) {
            const int sp = (kt - 1) % kStages;
            ok = ok && wait_bar(&st->mbar[sp], (phases >> sp) & 1u, deadline);
            phases ^= 1u << sp;
        }
        const int nxt = kt + kStages - 1;
        if (ok && nxt < nk) load_stage<THREADS>(smem + (nxt % kStages) * kStageBytes, A, lda, B, ldb, M, N, K, nxt * kBK);
        asm volatile("cp.async.commit_group;\n" ::: "memory");
    }
    {  // the accumulator is complete once the last k-slice's MMAs are
        const int sl = (nk - 1) % kStages;
        ok = ok && wait_bar(&st->mbar[sl], (phases >> sl) & 1u, deadline);
        phases ^= 1u << sl;
    }
    asm volatile("cp.async.wait_group 0;\n" ::: "memory");
    if (threadIdx.x == 0) st->phases = phases;
    float cv[32];
    load_c(cv, M, N, C, ldc, lower_only, r0, c0);
    return epilogue(st, ok, cv, M, N, C, ldc, lower_only, r0, c0);
}

__device__ __forceinline__ void tma_load_2d(uint32_t dst, const void *map, int x, int y, uint32_t bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
            dst),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(bar)
        : "memory");
}

__device__ __forceinline__ void tma_load_3d(uint32_t dst, const void *map, int x, int y, int z, uint32_t bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(
            dst),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(bar)
        : "memory");
}

// 1: TMA items run on the warp-specialised pipeline (thread 0 loads, thread 32 issues MMAs,
// warps 2 .. 15 drain accumulators; ws_* below), with 32-deep TF32 / 64-deep BF16 slices of
// 32 KB in a ring of six stages; 0 (default): the single-thread pipeline (mainloop_tma*) with
// 64-deep / 128-deep slices of 64 KB in three stages.  Measured on one B200 (Cholesky,
// N = 32768, tile 1536): TF32 factor 64.4 ms with the warp-specialised pipeline against
// 56.3 ms, BF16 59.9 against 49.1 ms -- the items are bound by the operand data rate per SM
// (~85 GB/s at depth 1536) and by per-item costs the single-thread loop already overlaps.
#ifndef MTD_TC_WS
#define MTD_TC_WS 0
#endif

// TMA pipeline geometry: kTmaBK-deep k-slices (A then B).  An operand slice is 4 MN atoms of
// 32 rows, each atom kTmaBK K-rows of 128 bytes, K-rows 128 bytes apart.
constexpr int kTmaBK = MTD_TC_WS ? 32 : 64;
constexpr int kTmaStages = 3;
constexpr int kTmaAtomBytes = 32 * kTmaBK * 4;                // 4 KB (8 KB at kTmaBK = 64)
constexpr int kTmaOperandBytes = 4 * kTmaAtomBytes;
constexpr int kTmaStageBytes = 2 * kTmaOperandBytes;
static_assert(kTmaStages * kTmaStageBytes <= kSmemBytes, "TMA stages fit the engine's shared memory");
static_assert(kTmaStages <= kStages, "TMA stages use the engine's barriers");
enum { kTmaNone = 0, kTmaMap2D = 1, kTmaMap3D = 2 };

// acc(128 x 128) = A B^T into the accumulator at TMEM address `acc`, both operands fetched by
// TMA from the FP32 matrix `map` describes, 128-byte swizzle with 32-byte atoms (an atom row k
// holds 32 consecutive MN elements of column k, its 32-byte chunks at c ^ (k % 4)).
// A = rows a_row .. a_row + 127, B = rows b_row .., columns k0 .. k0 + K - 1 (K a multiple
// of 64; a_row, b_row multiples of 32; rows past the matrix read as zero).  map_kind
// kTmaMap3D: dims (32 rows of an atom, columns, atoms), box 32 x 64 x 4, one load per
// operand and stage; kTmaMap2D: dims (rows, columns), box 32 x 64, four loads per operand
// and stage (the number of TMA instructions, not the bytes, limited the 32 x 32 boxes of
// the first design to ~25 GB/s per SM).  Thread 0 alone runs it: per stage one expect_tx
// and the loads on full[s], then, once the stage has landed, 8 MMAs committed to mbar[s]; a
// stage is reloaded after its MMAs are done.  On a true return every MMA has completed (the
// accumulator is final and every stage free); false if a wait timed out.  Operands must
// already be TF32 values (the tensor core truncates what it reads).
static __device__ bool mainloop_tma(State *st, uint8_t *smem, const void *map, int map_kind, int a_row, int b_row, int k0,
                             int K, uint32_t acc, unsigned long long timeout_ns) {
    bool ok = true;
    {
        const unsigned long long deadline = now_ns() + timeout_ns;
        const int nk = K / kTmaBK;
        uint32_t ph = st->phases, fph = st->fphases;
        // the operands were written by other CTAs with generic stores (released and acquired
        // through the scheduler's counters): order them before this thread's async-proxy loads
        asm volatile("fence.proxy.async.global;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // after generic use of the stages
        auto issue = [&](int s, int kt) {
            const uint32_t bar = smem_addr(&st->full[s]), base = smem_addr(smem + s * kTmaStageBytes);
            const int k = k0 + kt * kTmaBK;
            asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(kTmaStageBytes)
                         : "memory");
            if (map_kind == kTmaMap3D) {
                tma_load_3d(base, map, 0, k, a_row >> 5, bar);
                tma_load_3d(base + kTmaOperandBytes, map, 0, k, b_row >> 5, bar);
            } else {
                for (int i = 0; i < 4; ++i) {
                    tma_load_2d(base + i * kTmaAtomBytes, map, a_row + 32 * i, k, bar);
                    tma_load_2d(base + kTmaOperandBytes + i * kTmaAtomBytes, map, b_row + 32 * i, k, bar);
                }
            }
        };
        for (int s = 0; s < kTmaStages && s < nk; ++s) issue(s, s);
        for (int kt = 0; kt < nk && ok; ++kt) {
            const int s = kt % kTmaStages;
            ok = wait_bar(&st->full[s], (fph >> s) & 1u, deadline);
            fph ^= 1u << s;
            if (!ok) break;
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const uint32_t a0 = smem_addr(smem + s * kTmaStageBytes), b0 = a0 + kTmaOperandBytes;
#pragma unroll
            for (int g = 0; g < kTmaBK / 8; ++g) {
                // MN atoms kTmaAtomBytes apart, groups of 4 K-rows 512 bytes apart
                const uint64_t lead = uint64_t(kTmaAtomBytes >> 4) << 16, stride = uint64_t(512 >> 4) << 32;
                const uint64_t ad = uint64_t(((a0 + g * 1024) >> 4) & 0x3fff) | lead | stride | (1ull << 46) | (1ull << 61);
                const uint64_t bd = uint64_t(((b0 + g * 1024) >> 4) & 0x3fff) | lead | stride | (1ull << 46) | (1ull << 61);
                asm volatile(
                    "{\n\t.reg .pred p;\n\t"
                    "setp.ne.b32 p, %4, 0;\n\t"
                    "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}" ::"r"(acc),
                    "l"(ad), "l"(bd), "r"(kIdescTf32), "r"((kt > 0 || g > 0) ? 1u : 0u)
                    : "memory");
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                             smem_addr(&st->mbar[s]))
                         : "memory");
            // reload the stage of k-slice kt - 1 once its MMAs are done
            if (kt > 0 && kt - 1 + kTmaStages < nk) {
                const int sp = (kt - 1) % kTmaStages;
                ok = wait_bar(&st->mbar[sp], (ph >> sp) & 1u, deadline);
                ph ^= 1u << sp;
                if (ok) issue(sp, kt - 1 + kTmaStages);
            }
        }
        // consume the commits not waited above (the last kTmaStages k-slices, in order), so
        // the barriers' parities stay in step; the last one means the accumulator is complete
        for (int kt = nk > kTmaStages ? nk - kTmaStages : 0; kt < nk && ok; ++kt) {
            const int s = kt % kTmaStages;
            ok = wait_bar(&st->mbar[s], (ph >> s) & 1u, deadline);
            ph ^= 1u << s;
        }
        st->phases = ph;
        st->fphases = fph;
    }
    return ok;
}

// BF16 updates: C -= A B^T with BF16 operands read by TMA from the BF16 copy of the panels
// (`map`: 3D, 64-row atoms, box 64 x kBfBK x 2, 128-byte swizzle), tcgen05.mma kind::f16
// (BF16 x BF16, FP32 accumulation in TMEM, M = N = 128, K = 16 per instruction).  A stage is
// 128 MN rows x kBfBK columns per operand: two atoms of kBfBK rows x 128 bytes, 16 KB apart
// (LBO), 8-row groups 1 KB apart (SBO), layout type 2 (128-byte swizzle); this layout was
// checked bit-exact against a host product of the same BF16 values.  a_row, b_row multiples
// of 64, K a multiple of kBfBK; otherwise as mainloop_tma (thread 0 alone, into `acc`).
constexpr int kBfBK = MTD_TC_WS ? 64 : 128;
constexpr int kBfStages = 3;
constexpr int kBfAtomBytes = kBfBK * 128;                   // 64 BF16 x kBfBK rows
constexpr int kBfOperandBytes = 2 * kBfAtomBytes;
constexpr int kBfStageBytes = 2 * kBfOperandBytes;
static_assert(kBfStages * kBfStageBytes <= kSmemBytes, "BF16 stages fit the engine's shared memory");
static_assert(kBfStages <= kStages, "BF16 stages use the engine's barriers");
constexpr uint32_t kIdescBf16 = (1u << 4) | (1u << 7) | (1u << 10) | (1u << 15) | (1u << 16) |
                                (uint32_t(kN >> 3) << 17) | (uint32_t(kM >> 4) << 24);

static __device__ bool mainloop_tma_bf16(State *st, uint8_t *smem, const void *map, int a_row, int b_row, int k0, int K,
                                  uint32_t acc, unsigned long long timeout_ns) {
    bool ok = true;
    {
        const unsigned long long deadline = now_ns() + timeout_ns;
        const int nk = K / kBfBK;
        uint32_t ph = st->phases, fph = st->fphases;
        asm volatile("fence.proxy.async.global;" ::: "memory");  // see mainloop_tma
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        auto issue = [&](int s, int kt) {
            const uint32_t bar = smem_addr(&st->full[s]), base = smem_addr(smem + s * kBfStageBytes);
            const int k = k0 + kt * kBfBK;
            asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(kBfStageBytes)
                         : "memory");
            tma_load_3d(base, map, 0, k, a_row >> 6, bar);
            tma_load_3d(base + kBfOperandBytes, map, 0, k, b_row >> 6, bar);
        };
        for (int s = 0; s < kBfStages && s < nk; ++s) issue(s, s);
        for (int kt = 0; kt < nk && ok; ++kt) {
            const int s = kt % kBfStages;
            ok = wait_bar(&st->full[s], (fph >> s) & 1u, deadline);
            fph ^= 1u << s;
            if (!ok) break;
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const uint32_t a0 = smem_addr(smem + s * kBfStageBytes), b0 = a0 + kBfOperandBytes;
#pragma unroll
            for (int g = 0; g < kBfBK / 16; ++g) {
                const uint64_t lead = uint64_t(kBfAtomBytes >> 4) << 16, stride = uint64_t(1024 >> 4) << 32;
                const uint64_t ad = uint64_t(((a0 + g * 2048) >> 4) & 0x3fff) | lead | stride | (1ull << 46) | (2ull << 61);
                const uint64_t bd = uint64_t(((b0 + g * 2048) >> 4) & 0x3fff) | lead | stride | (1ull << 46) | (2ull << 61);
                asm volatile(
                    "{\n\t.reg .pred p;\n\t"
                    "setp.ne.b32 p, %4, 0;\n\t"
                    "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(acc),
                    "l"(ad), "l"(bd), "r"(kIdescBf16), "r"((kt > 0 || g > 0) ? 1u : 0u)
                    : "memory");
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                             smem_addr(&st->mbar[s]))
                         : "memory");
            if (kt > 0 && kt - 1 + kBfStages < nk) {
                const int sp = (kt - 1) % kBfStages;
                ok = wait_bar(&st->mbar[sp], (ph >> sp) & 1u, deadline);
                ph ^= 1u << sp;
                if (ok) issue(sp, kt - 1 + kBfStages);
            }
        }
        for (int kt = nk > kBfStages ? nk - kBfStages : 0; kt < nk && ok; ++kt) {
            const int s = kt % kBfStages;
            ok = wait_bar(&st->mbar[s], (ph >> s) & 1u, deadline);
            ph ^= 1u << s;
        }
        st->phases = ph;
        st->fphases = fph;
    }
    return ok;
}

// ---- warp-specialised pipeline ------------------------------------------------------------
//
// Thread 0 loads: one expect_tx and two (TF32 2D map: eight) TMA loads per slice into stage
// g % kWsStages of a ring that runs on across items (g counts the CTA's slices), waiting for a
// stage only while the MMAs of its previous slice are still reading it.  Thread 32 issues the
// MMAs of each slice once it has landed, commits them to the stage's `empty` barrier, and
// after the item's last slice commits to the accumulator's `accf` barrier.  Neither waits for
// the other's work beyond the stage hand-offs, so loads run up to six slices ahead of the
// MMAs and the MMA thread never waits for a reload.  Warps 2 .. 15 update C from the finished
// accumulator (one of two in TMEM) while the next item's slices stream in.
constexpr int kWsStages = 6;
constexpr int kWsStageBytes = 32768;
static_assert(kWsStages * kWsStageBytes <= kSmemBytes, "the ring fits the engine's shared memory");
static_assert(!MTD_TC_WS || (kTmaStageBytes == kWsStageBytes && kBfStageBytes == kWsStageBytes),
              "TF32 and BF16 slices share the ring");
enum { kWsTf32Map3D = 0, kWsTf32Map2D = 1, kWsBf16 = 2 };

struct WsState {
    uint64_t full[kWsStages];   // slice g landed (TMA complete_tx); parity (g / kWsStages) & 1
    uint64_t empty[kWsStages];  // MMAs of slice g done (tcgen05.commit)
    uint64_t accf[2];           // an item's last MMAs into accumulator b done
    uint64_t quiet;             // thread 32's last MMAs done, before the TMEM is freed
    uint32_t prod;              // slices loaded so far (thread 0)
    uint32_t cons;              // slices whose MMAs were issued (thread 32)
};

// Once per CTA (thread 0 initialises; the caller's barrier publishes it).
__device__ __forceinline__ void ws_init(WsState *w) {
    if (threadIdx.x == 0) {
        for (int s = 0; s < kWsStages; ++s) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(&w->full[s])), "r"(1));
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(&w->empty[s])), "r"(1));
        }
        for (int b = 0; b < 2; ++b)
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(&w->accf[b])), "r"(1));
        asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(&w->quiet)), "r"(1));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        w->prod = 0;
        w->cons = 0;
    }
}

__device__ __forceinline__ int ws_bk(int kind) { return kind == kWsBf16 ? kBfBK : kTmaBK; }

// Thread 0: load the item's K / bk slices (A rows a_row .., B rows b_row .., columns k0 ..).
// False if a wait for a free stage ran past the deadline.
static __device__ bool ws_load(WsState *w, uint8_t *ring, const void *map, int kind, int a_row, int b_row, int k0, int K,
                        unsigned long long deadline) {
    asm volatile("fence.proxy.async.global;" ::: "memory");       // operands other CTAs wrote
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // the ring's earlier generic use
    const int bk = ws_bk(kind), nk = K / bk;
    uint32_t g = w->prod;
    bool ok = true;
    for (int kt = 0; kt < nk; ++kt, ++g) {
        const int s = static_cast<int>(g % kWsStages);
        if (g >= uint32_t(kWsStages) && !wait_bar(&w->empty[s], ((g / kWsStages) - 1) & 1u, deadline)) {
            ok = false;
            break;
        }
        const uint32_t bar = smem_addr(&w->full[s]), base = smem_addr(ring + s * kWsStageBytes);
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(kWsStageBytes)
                     : "memory");
        const int k = k0 + kt * bk;
        if (kind == kWsBf16) {
            tma_load_3d(base, map, 0, k, a_row >> 6, bar);
            tma_load_3d(base + kWsStageBytes / 2, map, 0, k, b_row >> 6, bar);
        } else if (kind == kWsTf32Map3D) {
            tma_load_3d(base, map, 0, k, a_row >> 5, bar);
            tma_load_3d(base + kWsStageBytes / 2, map, 0, k, b_row >> 5, bar);
        } else {
            for (int i = 0; i < 4; ++i) {
                tma_load_2d(base + i * kTmaAtomBytes, map, a_row + 32 * i, k, bar);
                tma_load_2d(base + kWsStageBytes / 2 + i * kTmaAtomBytes, map, b_row + 32 * i, k, bar);
            }
        }
    }
    w->prod = g;
    return ok;
}

// Thread 32: acc(128 x 128) = A B^T over the item's slices as they land; commits each slice to
// its stage's `empty` barrier and the whole item to accf[buf].  False on a timed-out wait.
static __device__ bool ws_mma(WsState *w, uint8_t *ring, int kind, int K, uint32_t acc, int buf,
                       unsigned long long deadline) {
    const int bk = ws_bk(kind), nk = K / bk;
    uint32_t g = w->cons;
    bool ok = true;
    for (int kt = 0; kt < nk; ++kt, ++g) {
        const int s = static_cast<int>(g % kWsStages);
        if (!wait_bar(&w->full[s], (g / kWsStages) & 1u, deadline)) {
            ok = false;
            break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint32_t a0 = smem_addr(ring + s * kWsStageBytes), b0 = a0 + kWsStageBytes / 2;
        if (kind == kWsBf16) {
#pragma unroll
            for (int q = 0; q < kBfBK / 16; ++q) {
                const uint64_t lead = uint64_t(kBfAtomBytes >> 4) << 16, stride = uint64_t(1024 >> 4) << 32;
                const uint64_t ad = uint64_t(((a0 + q * 2048) >> 4) & 0x3fff) | lead | stride | (1ull << 46) | (2ull << 61);
                const uint64_t bd = uint64_t(((b0 + q * 2048) >> 4) & 0x3fff) | lead | stride | (1ull << 46) | (2ull << 61);
                asm volatile(
                    "{\n\t.reg .pred p;\n\t"
                    "setp.ne.b32 p, %4, 0;\n\t"
                    "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(acc),
                    "l"(ad), "l"(bd), "r"(kIdescBf16), "r"((kt > 0 || q > 0) ? 1u : 0u)
                    : "memory");
            }
        } else {
#pragma unroll
            for (int q = 0; q < kTmaBK / 8; ++q) {
                const uint64_t lead = uint64_t(kTmaAtomBytes >> 4) << 16, stride = uint64_t(512 >> 4) << 32;
                const uint64_t ad = uint64_t(((a0 + q * 1024) >> 4) & 0x3fff) | lead | stride | (1ull << 46) | (1ull << 61);
                const uint64_t bd = uint64_t(((b0 + q * 1024) >> 4) & 0x3fff) | lead | stride | (1ull << 46) | (1ull << 61);
                asm volatile(
                    "{\n\t.reg .pred p;\n\t"
                    "setp.ne.b32 p, %4, 0;\n\t"
                    "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}" ::"r"(acc),
                    "l"(ad), "l"(bd), "r"(kIdescTf32), "r"((kt > 0 || q > 0) ? 1u : 0u)
                    : "memory");
            }
        }
        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                         smem_addr(&w->empty[s]))
                     : "memory");
    }
    if (ok)
        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                         smem_addr(&w->accf[buf]))
                     : "memory");
    w->cons = g;
    return ok;
}

// Thread 32, once, before the CTA frees its TMEM: wait (bounded) until every MMA it issued
// has completed (they normally have: the last item was drained).
__device__ __forceinline__ void ws_quiesce(WsState *w, unsigned long long deadline) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                     smem_addr(&w->quiet))
                 : "memory");
    wait_bar(&w->quiet, 0u, deadline);
}

// The C update of a finished accumulator is shared by warps 2 .. 15.  Warp w covers TMEM lane
// quarter q = w % 4; the quarter's 8 chunks of 16 columns go to its warps among 2 .. 15 --
// three for q = 0, 1 (warps 4 + q, 8 + q, 12 + q), four for q = 2, 3 -- chunk rank + c * count.
constexpr int kWsDrainChunks = 3;
__host__ __device__ constexpr int ws_count(int q) { return q < 2 ? 3 : 4; }
__host__ __device__ constexpr int ws_rank(int warp) { return (warp & 3) < 2 ? (warp >> 2) - 1 : (warp >> 2); }
constexpr bool ws_drain_covers_once() {
    for (int q = 0; q < 4; ++q)
        for (int ch = 0; ch < kN / 16; ++ch) {
            int owners = 0;
            for (int w = 2; w < 16; ++w) {
                if ((w & 3) != q) continue;
                for (int c = 0; c < kWsDrainChunks; ++c)
                    if (ws_rank(w) + c * ws_count(q) == ch) ++owners;
            }
            if (owners != 1) return false;
        }
    for (int w = 2; w < 16; ++w)
        if (ws_rank(w) < 0 || ws_rank(w) >= ws_count(w & 3)) return false;
    return true;
}
static_assert(ws_drain_covers_once(), "warps 2 .. 15 cover the accumulator once");

// Warps 2 .. 15: this thread's C values of an item (row 32 q + lane of its chunks; 0 outside
// the block or above the diagonal), all loads issued back to back.
__device__ __forceinline__ void ws_prefetch_c(const float *C, int64_t ldc, int M, int N, bool lower,
                                              float (&cv)[kWsDrainChunks][16]) {
    const int warp = threadIdx.x >> 5, q = warp & 3, rank = ws_rank(warp), count = ws_count(q);
    const int row = q * 32 + (threadIdx.x & 31);
#pragma unroll
    for (int c = 0; c < kWsDrainChunks; ++c) {
        const int ch = rank + c * count;
#pragma unroll
        for (int j = 0; j < 16; ++j) {
            const int col = ch * 16 + j;
            const bool in = ch < kN / 16 && row < M && col < N && (!lower || row >= col);
            cv[c][j] = in ? __ldcg(C + row + int64_t(col) * ldc) : 0.f;
        }
    }
}

// Warps 2 .. 15, once accf[buf] says the item's MMAs are done: C = cv - accumulator.
__device__ __forceinline__ void ws_drain(uint32_t acc, float *C, int64_t ldc, int M, int N, bool lower,
                                         const float (&cv)[kWsDrainChunks][16]) {
    const int warp = threadIdx.x >> 5, q = warp & 3, rank = ws_rank(warp), count = ws_count(q);
    const int row = q * 32 + (threadIdx.x & 31);
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
#pragma unroll
    for (int c = 0; c < kWsDrainChunks; ++c) {
        const int ch = rank + c * count;
        if (ch >= kN / 16) break;  // warp-uniform
        uint32_t v[16];
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
            : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
              "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
            : "r"(acc + (uint32_t(q * 32) << 16) + uint32_t(ch * 16)));
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
        for (int j = 0; j < 16; ++j) {
            const int col = ch * 16 + j;
            if (row < M && col < N && (!lower || row >= col)) C[row + int64_t(col) * ldc] = cv[c][j] - __uint_as_float(v[j]);
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}

// FP32-accurate updates: C -= A B^T as A_h B_h^T + A_h B_l^T + A_l B_h^T, three TF32 passes
// (tcgen05.mma kind::tf32, FP32 accumulation in TMEM).  A_h, B_h are the panels as stored
// (full FP32 values: the tensor core reads their TF32 part, i.e. truncates them); A_l, B_l
// come from the low-part copy the TRSM items write (x - trunc(x), rounded to nearest TF32, so
// the tensor core reads it exactly).  A stage holds 32-deep slices of the four operands (16 KB
// each, the TF32 layout of mainloop_tma with 4 KB atoms): 64 KB, three stages; 4 x 3 MMAs.
// `map` / `map_lo`: 3D maps of the matrix and of the low copy, box 32 x 32 x 4.  a_row, b_row
// multiples of 32, K a multiple of 32; otherwise as mainloop_tma (thread 0 alone, into `acc`).
constexpr int kX3BK = 32;
constexpr int kX3Stages = 3;
constexpr int kX3AtomBytes = 32 * kX3BK * 4;              // 4 KB
constexpr int kX3OperandBytes = 4 * kX3AtomBytes;         // 16 KB
constexpr int kX3StageBytes = 4 * kX3OperandBytes;        // 64 KB
static_assert(kX3Stages * kX3StageBytes <= kSmemBytes, "three-pass stages fit the engine's shared memory");
static_assert(kX3Stages <= kStages, "three-pass stages use the engine's barriers");

static __device__ bool mainloop_tma_x3(State *st, uint8_t *smem, const void *map, const void *map_lo, int a_row, int b_row,
                                int k0, int K, uint32_t acc, unsigned long long timeout_ns) {
    bool ok = true;
    {
        const unsigned long long deadline = now_ns() + timeout_ns;
        const int nk = K / kX3BK;
        uint32_t ph = st->phases, fph = st->fphases;
        asm volatile("fence.proxy.async.global;" ::: "memory");  // see mainloop_tma
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        auto issue = [&](int s, int kt) {
            const uint32_t bar = smem_addr(&st->full[s]), base = smem_addr(smem + s * kX3StageBytes);
            const int k = k0 + kt * kX3BK;
            asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(kX3StageBytes)
                         : "memory");
            tma_load_3d(base, map, 0, k, a_row >> 5, bar);
            tma_load_3d(base + kX3OperandBytes, map, 0, k, b_row >> 5, bar);
            tma_load_3d(base + 2 * kX3OperandBytes, map_lo, 0, k, a_row >> 5, bar);
            tma_load_3d(base + 3 * kX3OperandBytes, map_lo, 0, k, b_row >> 5, bar);
        };
        for (int s = 0; s < kX3Stages && s < nk; ++s) issue(s, s);
        for (int kt = 0; kt < nk && ok; ++kt) {
            const int s = kt % kX3Stages;
            ok = wait_bar(&st->full[s], (fph >> s) & 1u, deadline);
            fph ^= 1u << s;
            if (!ok) break;
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const uint32_t ah0 = smem_addr(smem + s * kX3StageBytes), bh0 = ah0 + kX3OperandBytes,
                           al0 = ah0 + 2 * kX3OperandBytes, bl0 = ah0 + 3 * kX3OperandBytes;
            const uint64_t lead = uint64_t(kX3AtomBytes >> 4) << 16, stride = uint64_t(512 >> 4) << 32;
            auto desc = [&](uint32_t a) {
                return uint64_t((a >> 4) & 0x3fff) | lead | stride | (1ull << 46) | (1ull << 61);
            };
#pragma unroll
            for (int q = 0; q < kX3BK / 8; ++q) {
                const uint64_t ah = desc(ah0 + q * 1024), bh = desc(bh0 + q * 1024), al = desc(al0 + q * 1024),
                               bl = desc(bl0 + q * 1024);
                const uint32_t first = (kt > 0 || q > 0) ? 1u : 0u;
                asm volatile(
                    "{\n\t.reg .pred p, q;\n\t"
                    "setp.ne.b32 p, %6, 0;\n\t"
                    "setp.eq.b32 q, %6, %6;\n\t"
                    "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %5, p;\n\t"
                    "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %3, %5, q;\n\t"
                    "tcgen05.mma.cta_group::1.kind::tf32 [%0], %4, %2, %5, q;\n\t}" ::"r"(acc),
                    "l"(ah), "l"(bh), "l"(bl), "l"(al), "r"(kIdescTf32), "r"(first)
                    : "memory");
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                             smem_addr(&st->mbar[s]))
                         : "memory");
            if (kt > 0 && kt - 1 + kX3Stages < nk) {
                const int sp = (kt - 1) % kX3Stages;
                ok = wait_bar(&st->mbar[sp], (ph >> sp) & 1u, deadline);
                ph ^= 1u << sp;
                if (ok) issue(sp, kt - 1 + kX3Stages);
            }
        }
        for (int kt = nk > kX3Stages ? nk - kX3Stages : 0; kt < nk && ok; ++kt) {
            const int s = kt % kX3Stages;
            ok = wait_bar(&st->mbar[s], (ph >> s) & 1u, deadline);
            ph ^= 1u << s;
        }
        st->phases = ph;
        st->fphases = fph;
    }
    return ok;
}

// A TMA item whose accumulator is final but whose update of C is still to be done.
struct Pending {
    float *C;
    int64_t ldc;
    int M, N, lower;   // C(r, c) for r < M, c < N (and r >= c when lower)
    int task, item;
    unsigned long long t_start;
    uint32_t acc;      // TMEM address of its accumulator
    int valid;
};

// The C update of an item is shared by warps 1 .. 15 (warp 0 runs the pipelines).  A warp
// covers TMEM lane quarter q = warp % 4 (rows 32 q ..); the quarter's 8 chunks of 16 columns
// are dealt to the warps w = q (mod 4) of 1 .. 15 -- three for q = 0 (chunks first + 3 c),
// four otherwise (first + 4 c) -- so a warp holds at most 3 chunks.
constexpr int kDrainChunks = 3;
__host__ __device__ constexpr int drain_first(int warp) { return (warp & 3) == 0 ? (warp >> 2) - 1 : (warp >> 2); }
__host__ __device__ constexpr int drain_step(int warp) { return (warp & 3) == 0 ? 3 : 4; }
__device__ __forceinline__ void drain_share(int &q, int &first, int &step) {
    const int warp = threadIdx.x >> 5;
    q = warp & 3;
    first = drain_first(warp);
    step = drain_step(warp);
}
// Every (lane quarter, 16-column chunk) of the accumulator is written by exactly one of warps
// 1 .. 15, a warp of that quarter, within kDrainChunks chunks of its own.
constexpr bool drain_covers_once() {
    for (int q = 0; q < 4; ++q)
        for (int ch = 0; ch < kN / 16; ++ch) {
            int owners = 0;
            for (int w = 1; w < 16; ++w) {
                if ((w & 3) != q) continue;
                for (int c = 0; c < kDrainChunks; ++c)
                    if (drain_first(w) + c * drain_step(w) == ch) ++owners;
            }
            if (owners != 1) return false;
        }
    for (int w = 1; w < 16; ++w)  // and no warp has a chunk beyond the ones it holds
        if (drain_first(w) < 0 || drain_first(w) + kDrainChunks * drain_step(w) < kN / 16) return false;
    return true;
}
static_assert(drain_covers_once(), "the C update covers the accumulator once");

// Warps 1 .. 15, while thread 0 runs the item's loads and MMAs: this thread's C values of the
// item (row 32 q + lane of its chunks; 0 outside the block or above the diagonal), all
// loads issued back to back.
__device__ __forceinline__ void prefetch_c(const float *C, int64_t ldc, int M, int N, bool lower,
                                           float (&cv)[kDrainChunks][16]) {
    int q, first, step;
    drain_share(q, first, step);
    const int row = q * 32 + (threadIdx.x & 31);
#pragma unroll
    for (int c = 0; c < kDrainChunks; ++c) {
        const int ch = first + c * step;
#pragma unroll
        for (int j = 0; j < 16; ++j) {
            const int col = ch * 16 + j;
            const bool in = ch < kN / 16 && row < M && col < N && (!lower || row >= col);
            cv[c][j] = in ? __ldcg(C + row + int64_t(col) * ldc) : 0.f;
        }
    }
}

// Warps 1 .. 15, while thread 0 claims and starts the next item: C = cv - accumulator of `pd`
// (tcgen05.ld of each 16-column chunk, then its stores: one 128-byte line per warp and column).
__device__ __forceinline__ void drain(const Pending &pd, const float (&cv)[kDrainChunks][16]) {
    int q, first, step;
    drain_share(q, first, step);
    const int row = q * 32 + (threadIdx.x & 31);
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
#pragma unroll
    for (int c = 0; c < kDrainChunks; ++c) {
        const int ch = first + c * step;
        if (ch >= kN / 16) break;  // warp-uniform
        uint32_t v[16];
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
            : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
              "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
            : "r"(pd.acc + (uint32_t(q * 32) << 16) + uint32_t(ch * 16)));
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
        for (int j = 0; j < 16; ++j) {
            const int col = ch * 16 + j;
            if (row < pd.M && col < pd.N && (!pd.lower || row >= col))
                pd.C[row + int64_t(col) * pd.ldc] = cv[c][j] - __uint_as_float(v[j]);
        }
    }
    // the accumulator is written again (two TMA items later) only after a CTA barrier
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}

}  // namespace tc
}  // namespace mtd
