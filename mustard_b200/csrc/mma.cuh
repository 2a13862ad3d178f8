// Block-GEMM engine for one CTA on sm_100a, FP64 (DMMA) or FP32 storage with TF32 MMA.
//
// acc(BM x BN) += A(BM x K) * B(K x BN), operands read from global memory (L2) into a
// multi-stage shared-memory ring with cp.async.cg (16-byte, L1-bypassing: tiles written
// by other CTAs of the persistent kernel are never read from a stale L1 line), and
// multiplied on the tensor cores with warp-level MMA:
//   T = double: mma.sync.m16n8k8.f64 (DMMA).  sm_100a's tcgen05 MMA has no FP64 kind, so
//               DMMA is the FP64 tensor path on B200; a register-only probe measures it at
//               the same 37 TFLOP/s as the datasheet's FP64 figure.
//   T = float : mma.sync.m16n8k8.tf32 with FP32 accumulation (operands rounded to TF32
//               with cvt.rna); used by the low-precision factorisation of the mixed-
//               precision solver.
// Both shapes share one fragment layout: A (g, t), (g+8, t), (g, t+4), (g+8, t+4);
// B (k = t, n = g), (k = t+4, n = g); C (g, 2t), (g, 2t+1), (g+8, 2t), (g+8, 2t+1), with
// g = lane / 4 and t = lane % 4.
//
// Layouts (column-major global memory):
//   A(m, k) = A[m + k * lda]                                   ("m-contiguous")
//   B(k, n) = B[n + k * ldb]   when BL == kBNContig            (Cholesky: B = L(i,k)^T)
//   B(k, n) = B[k + n * ldb]   when BL == kBKContig            (LU:       B = U(k,j))
// Shared-memory rows are padded so every fragment load is bank-conflict-free: for 8-byte
// elements a half-warp touches 16 distinct bank pairs (row pad = 4 mod 16), for 4-byte
// elements a warp touches 32 distinct banks (row pad = 8 mod 32, 4 mod 32 for k-rows).
//
// VEC == 2: 16-byte copies; needs 16-byte aligned bases and leading dimensions and
// extents that are multiples of 16 bytes' worth of elements (the host checks).
// VEC == 1: element loads through registers, any shape.
#pragma once

#include <cuda_bf16.h>

#include <cstdint>

#include "device_types.hpp"
#include "sync_util.cuh"

namespace mtd {

// 1: BlockMmaT::run refills a stage right after the slice barrier, before that slice's
// compute; 0: after it.
#ifndef MTD_EARLY_ISSUE
#define MTD_EARLY_ISSUE 0
#endif
// 1: the GEMM / SYRK update items use BlockMmaT::run_sp (split-phase mbarrier
// synchronisation of the stage ring) instead of run (one CTA barrier per slice): measured on
// one B200 at N = 24000, tile 1536, LU 309.0 -> 297.9 ms, Cholesky 160.6 -> 153.5 ms.
#ifndef MTD_SPLIT_PHASE
#define MTD_SPLIT_PHASE 1
#endif
// 1: the TRSM strips' engines use run_sp too.
#ifndef MTD_SPLIT_PHASE_TRSM
#define MTD_SPLIT_PHASE_TRSM 0
#endif
// 1: BlockMmaT::run_sp_update keeps the C pointer, its leading dimension and the lower flag
// in shared memory during the k-loop.
#ifndef MTD_STAGE_C_PARK
#define MTD_STAGE_C_PARK 0
#endif

enum { kBNContig = 0, kBKContig = 1 };

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void cp_async16(void *dst, const void *src, bool valid) {
    const int bytes = valid ? 16 : 0;  // 0 source bytes: the 16 destination bytes are zero-filled
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(smem_u32(dst)), "l"(src),
                 "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

__device__ __forceinline__ double ld_cg(const double *p) { return __ldcg(p); }
__device__ __forceinline__ float ld_cg(const float *p) { return __ldcg(p); }

__device__ __forceinline__ void mma_16x8x8(double (&d)[4], const double (&a)[4], const double (&b)[2]) {
    asm volatile(
        "mma.sync.aligned.m16n8k8.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+d"(d[0]), "+d"(d[1]), "+d"(d[2]), "+d"(d[3])
        : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(b[0]), "d"(b[1]));
}
__device__ __forceinline__ void dmma_16x8x8(double (&d)[4], const double (&a)[4], const double (&b)[2]) {
    mma_16x8x8(d, a, b);
}

__device__ __forceinline__ uint32_t to_tf32(float x) {
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;\n" : "=r"(r) : "f"(x));
    return r;
}

// TF32 product with FP32 accumulation.  The operand bits go to the tensor core as they are:
// it reads the TF32 part (sign, exponent, top 10 mantissa bits).  The engine rounds each
// fragment element to nearest once, when it is read from shared memory (frag_round), so a
// fragment reused by several MMAs is converted once; rounding inside every MMA cost six
// conversions per MMA and left the FP32-storage GEMM issue-bound at a third of the peak.
__device__ __forceinline__ void mma_16x8x8(float (&d)[4], const float (&a)[4], const float (&b)[2]) {
    asm volatile(
        "mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(__float_as_uint(a[0])), "r"(__float_as_uint(a[1])), "r"(__float_as_uint(a[2])),
          "r"(__float_as_uint(a[3])), "r"(__float_as_uint(b[0])), "r"(__float_as_uint(b[1])));
}

// FP32-accurate products from TF32 tensor cores: each operand is split into a TF32 head
// (the top 19 bits, by masking) and the exact FP32 remainder (x = hi + lo), and
// d += lo_a*hi_b + hi_a*lo_b + hi_a*hi_b (lo*lo is below FP32 roundoff; the remainders
// enter the tensor core truncated to TF32, an error of ~2^-21 relative of a term that is
// itself 2^-10 of the product).  Three MMAs per product; accuracy close to FP32.
__device__ __forceinline__ void mma_16x8x8_x3(float (&d)[4], const float (&a)[4], const float (&b)[2]) {
    uint32_t ah[4], al[4], bh[2], bl[2];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        ah[i] = __float_as_uint(a[i]) & 0xffffe000u;
        al[i] = __float_as_uint(a[i] - __uint_as_float(ah[i]));
    }
#pragma unroll
    for (int i = 0; i < 2; ++i) {
        bh[i] = __float_as_uint(b[i]) & 0xffffe000u;
        bl[i] = __float_as_uint(b[i] - __uint_as_float(bh[i]));
    }
    asm volatile(
        "mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};\n"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(al[0]), "r"(al[1]), "r"(al[2]), "r"(al[3]), "r"(bh[0]), "r"(bh[1]));
    asm volatile(
        "mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};\n"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(ah[0]), "r"(ah[1]), "r"(ah[2]), "r"(ah[3]), "r"(bl[0]), "r"(bl[1]));
    asm volatile(
        "mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};\n"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(ah[0]), "r"(ah[1]), "r"(ah[2]), "r"(ah[3]), "r"(bh[0]), "r"(bh[1]));
}

// Fragment element as the tensor core should see it: FP64 unchanged; single TF32 products
// round to nearest TF32 (a truncated operand biases every product towards zero, and those
// errors add up linearly along a long update chain); the split mode keeps all FP32 bits.
template <int SPLIT>
__device__ __forceinline__ double frag_round(double x) {
    return x;
}
template <int SPLIT>
__device__ __forceinline__ float frag_round(float x) {
    if constexpr (SPLIT == 3) return x;
    else return __uint_as_float(to_tf32(x));
}

template <int SPLIT>
__device__ __forceinline__ void mma_op(double (&d)[4], const double (&a)[4], const double (&b)[2]) {
    mma_16x8x8(d, a, b);
}
template <int SPLIT>
__device__ __forceinline__ void mma_op(float (&d)[4], const float (&a)[4], const float (&b)[2]) {
    if constexpr (SPLIT == 3) mma_16x8x8_x3(d, a, b);
    else mma_16x8x8(d, a, b);
}

template <typename T>
struct SmemPad {
    static constexpr int a = sizeof(T) == 8 ? 4 : 8;  // rows of A and of n-contiguous B
    static constexpr int bk = 4;                        // rows of k-contiguous B
    static constexpr int a_mod = sizeof(T) == 8 ? 16 : 32;
};

// A operand layout: element (m, k) at A[m + k lda] (kAMContig, column-major A) or at
// A[k + m lda] (kAKContig: the transpose of a column-major block, for C -= X^T Y).
enum { kAMContig = 0, kAKContig = 1 };

template <typename T, int BM, int BN, int WARPS_M, int WARPS_N, int BL, int VEC, int STAGES = 3, int BK_ = 16,
          int SPLIT = 1, int AL = kAMContig>
struct BlockMmaT {
    static constexpr int BK = BK_;
    static constexpr int EPC = 16 / int(sizeof(T));  // elements per 16-byte copy
    static constexpr int WM = BM / WARPS_M;
    static constexpr int WN = BN / WARPS_N;
    static constexpr int FM = WM / 16;
    static constexpr int FN = WN / 8;
    // m-contiguous A is staged [k][m] (stride LDA); k-contiguous A is staged [m][k] with
    // the k-contiguous B padding, which keeps its fragment reads conflict-free the same way
    static constexpr int LDA = (AL == kAMContig) ? BM + SmemPad<T>::a : BK + SmemPad<T>::bk;
    static constexpr int LDB = (BL == kBNContig) ? BN + SmemPad<T>::a : BK + SmemPad<T>::bk;
    static constexpr int A_STAGE = (AL == kAMContig) ? BK * LDA : BM * LDA;
    static constexpr int B_STAGE = (BL == kBNContig) ? BK * LDB : BN * LDB;
    static constexpr int SMEM_ELEMS = STAGES * (A_STAGE + B_STAGE);
    static constexpr int SMEM_BYTES = SMEM_ELEMS * int(sizeof(T));
    static_assert(WARPS_M * WARPS_N * 32 == kThreads, "one warp tile per warp of the CTA");
    static_assert(FM >= 1 && FN >= 1 && WM % 16 == 0 && WN % 8 == 0, "warp tile");
    static_assert(AL != kAMContig || LDA % SmemPad<T>::a_mod == SmemPad<T>::a, "bank-conflict-free padding (A)");
    static_assert((LDA * int(sizeof(T))) % 16 == 0 && (LDB * int(sizeof(T))) % 16 == 0, "16-byte rows");
    static_assert(BK % 8 == 0 && BM % EPC == 0 && BN % EPC == 0 && BK % EPC == 0, "copy granularity");

    T acc[FM][FN][4];

    __device__ __forceinline__ void zero() {
#pragma unroll
        for (int i = 0; i < FM; ++i)
#pragma unroll
            for (int j = 0; j < FN; ++j)
#pragma unroll
                for (int v = 0; v < 4; ++v) acc[i][j][v] = T(0);
    }

    // ---- global -> shared stage loads ----
    __device__ __forceinline__ static void load_a(T *As, const T *A, int64_t lda, int M, int K, int k0) {
        const int tid = threadIdx.x;
        if constexpr (AL == kAKContig) {
            if (VEC == 2) {
                constexpr int CH = BM * (BK / EPC);
#pragma unroll
                for (int c = tid; c < CH; c += kThreads) {
                    const int m = c / (BK / EPC);
                    const int k = EPC * (c % (BK / EPC));
                    const int kk = k0 + k;
                    const bool ok = m < M && kk < K;
                    const T *src = ok ? A + kk + int64_t(m) * lda : A;
                    cp_async16(As + m * LDA + k, src, ok);
                }
            } else {
                constexpr int EL = BM * BK;
                for (int e = tid; e < EL; e += kThreads) {
                    const int m = e / BK;
                    const int k = e % BK;
                    const int kk = k0 + k;
                    As[m * LDA + k] = (m < M && kk < K) ? ld_cg(A + kk + int64_t(m) * lda) : T(0);
                }
            }
            return;
        }
        if (VEC == 2) {
            constexpr int CH = BK * (BM / EPC);
#pragma unroll
            for (int c = tid; c < CH; c += kThreads) {
                const int col = c / (BM / EPC);
                const int row = EPC * (c % (BM / EPC));
                const int kk = k0 + col;
                const bool ok = row < M && kk < K;
                const T *src = ok ? A + row + int64_t(kk) * lda : A;
                cp_async16(As + col * LDA + row, src, ok);
            }
        } else {
            constexpr int EL = BK * BM;
            for (int e = tid; e < EL; e += kThreads) {
                const int col = e / BM;
                const int row = e % BM;
                const int kk = k0 + col;
                As[col * LDA + row] = (row < M && kk < K) ? ld_cg(A + row + int64_t(kk) * lda) : T(0);
            }
        }
    }

    __device__ __forceinline__ static void load_b(T *Bs, const T *B, int64_t ldb, int N, int K, int k0) {
        const int tid = threadIdx.x;
        if (BL == kBNContig) {
            if (VEC == 2) {
                constexpr int CH = BK * (BN / EPC);
#pragma unroll
                for (int c = tid; c < CH; c += kThreads) {
                    const int col = c / (BN / EPC);
                    const int n = EPC * (c % (BN / EPC));
                    const int kk = k0 + col;
                    const bool ok = n < N && kk < K;
                    const T *src = ok ? B + n + int64_t(kk) * ldb : B;
                    cp_async16(Bs + col * LDB + n, src, ok);
                }
            } else {
                constexpr int EL = BK * BN;
                for (int e = tid; e < EL; e += kThreads) {
                    const int col = e / BN;
                    const int n = e % BN;
                    const int kk = k0 + col;
                    Bs[col * LDB + n] = (n < N && kk < K) ? ld_cg(B + n + int64_t(kk) * ldb) : T(0);
                }
            }
        } else {
            if (VEC == 2) {
                constexpr int CH = BN * (BK / EPC);
#pragma unroll
                for (int c = tid; c < CH; c += kThreads) {
                    const int n = c / (BK / EPC);
                    const int k = EPC * (c % (BK / EPC));
                    const int kk = k0 + k;
                    const bool ok = n < N && kk < K;
                    const T *src = ok ? B + kk + int64_t(n) * ldb : B;
                    cp_async16(Bs + n * LDB + k, src, ok);
                }
            } else {
                constexpr int EL = BN * BK;
                for (int e = tid; e < EL; e += kThreads) {
                    const int n = e / BK;
                    const int k = e % BK;
                    const int kk = k0 + k;
                    Bs[n * LDB + k] = (n < N && kk < K) ? ld_cg(B + kk + int64_t(n) * ldb) : T(0);
                }
            }
        }
    }

    __device__ __forceinline__ void compute_stage(const T *As, const T *Bs) {
        const int lane = threadIdx.x & 31;
        const int warp = threadIdx.x >> 5;
        const int wm0 = (warp / WARPS_N) * WM;
        const int wn0 = (warp % WARPS_N) * WN;
        const int g = lane >> 2;
        const int t = lane & 3;
#pragma unroll
        for (int ks = 0; ks < BK; ks += 8) {
            T bf[FN][2];
#pragma unroll
            for (int j = 0; j < FN; ++j) {
                const int n = wn0 + j * 8 + g;
                if (BL == kBNContig) {
                    bf[j][0] = frag_round<SPLIT>(Bs[(ks + t) * LDB + n]);
                    bf[j][1] = frag_round<SPLIT>(Bs[(ks + t + 4) * LDB + n]);
                } else {
                    bf[j][0] = frag_round<SPLIT>(Bs[n * LDB + ks + t]);
                    bf[j][1] = frag_round<SPLIT>(Bs[n * LDB + ks + t + 4]);
                }
            }
#pragma unroll
            for (int i = 0; i < FM; ++i) {
                const int m = wm0 + i * 16 + g;
                T af[4];
                if constexpr (AL == kAMContig) {
                    af[0] = frag_round<SPLIT>(As[(ks + t) * LDA + m]);
                    af[1] = frag_round<SPLIT>(As[(ks + t) * LDA + m + 8]);
                    af[2] = frag_round<SPLIT>(As[(ks + t + 4) * LDA + m]);
                    af[3] = frag_round<SPLIT>(As[(ks + t + 4) * LDA + m + 8]);
                } else {
                    af[0] = frag_round<SPLIT>(As[m * LDA + ks + t]);
                    af[1] = frag_round<SPLIT>(As[(m + 8) * LDA + ks + t]);
                    af[2] = frag_round<SPLIT>(As[m * LDA + ks + t + 4]);
                    af[3] = frag_round<SPLIT>(As[(m + 8) * LDA + ks + t + 4]);
                }
#pragma unroll
                for (int j = 0; j < FN; ++j) mma_op<SPLIT>(acc[i][j], af, bf[j]);
            }
        }
    }

    // acc += A(M x K) * B(K x N).  M <= BM, N <= BN; rows/columns beyond M/N and depth
    // beyond K are zero-filled.  All threads of the CTA must call; shared memory is free
    // again on return.
    __device__ __forceinline__ void run(void *smem_raw, const T *A, int64_t lda, const T *B, int64_t ldb, int M,
                                        int N, int K) {
        if (K <= 0) return;
        T *As = static_cast<T *>(smem_raw);
        T *Bs = As + STAGES * A_STAGE;
        const int ktiles = (K + BK - 1) / BK;
#pragma unroll
        for (int s = 0; s < STAGES - 1; ++s) {
            if (s < ktiles) {
                load_a(As + s * A_STAGE, A, lda, M, K, s * BK);
                load_b(Bs + s * B_STAGE, B, ldb, N, K, s * BK);
            }
            cp_async_commit();
        }
        for (int kt = 0; kt < ktiles; ++kt) {
            cp_async_wait<STAGES - 2>();
            __syncthreads();
            const int st = kt % STAGES;
#if MTD_EARLY_ISSUE
            // the stage slice kt + STAGES - 1 goes into was read in iteration kt - 1, which every
            // thread has finished (the barrier above): refill it before this slice's compute, so
            // the copies have STAGES - 1 compute phases to land
            {
                const int nk = kt + STAGES - 1;
                if (nk < ktiles) {
                    const int ns = nk % STAGES;
                    load_a(As + ns * A_STAGE, A, lda, M, K, nk * BK);
                    load_b(Bs + ns * B_STAGE, B, ldb, N, K, nk * BK);
                }
                cp_async_commit();
            }
            compute_stage(As + st * A_STAGE, Bs + st * B_STAGE);
#else
            compute_stage(As + st * A_STAGE, Bs + st * B_STAGE);
            const int nk = kt + STAGES - 1;
            if (nk < ktiles) {
                const int ns = nk % STAGES;
                load_a(As + ns * A_STAGE, A, lda, M, K, nk * BK);
                load_b(Bs + ns * B_STAGE, B, ldb, N, K, nk * BK);
            }
            cp_async_commit();
#endif
        }
        cp_async_wait<0>();
        __syncthreads();
    }

    // The k-loop of run with split-phase synchronisation.  Per stage a `full` mbarrier that
    // completes when every thread's copies of the slice have landed (each thread arrives with
    // cp.async.mbarrier.arrive.noinc after issuing them) and an `empty` one that completes when
    // every warp has read it (lane 0 arrives after the warp's compute).  A warp waits only for
    // the slice it reads and, before refilling a stage, for the warps still reading its
    // previous slice, so the warps drift up to a slice apart instead of draining the tensor
    // pipe at a CTA barrier every slice.  All threads must call.  Returns false if a wait ran
    // past ~1 s (in a correct run every copy lands and every warp arrives): the caller
    // reports a timeout.  Shared memory is free again on return.
#if MTD_EARLY_CLAIM2
    __device__ __forceinline__ bool run_sp(void *smem_raw, const T *A, int64_t lda, const T *B, int64_t ldb, int M,
                                           int N, int K) {
        return run_sp(smem_raw, A, lda, B, ldb, M, N, K, [] {});
    }
    template <typename OnLast>
    __device__ __forceinline__ bool run_sp(void *smem_raw, const T *A, int64_t lda, const T *B, int64_t ldb, int M,
                                           int N, int K, OnLast on_last) {
#else
    // end_sync false: no CTA barrier at the end, so each warp goes on to its own epilogue as
    // soon as its last slice is read; the caller then must pass a CTA barrier before shared
    // memory or these barriers are used again.
    __device__ __forceinline__ bool run_sp(void *smem_raw, const T *A, int64_t lda, const T *B, int64_t ldb, int M,
                                           int N, int K, bool end_sync = true) {
#endif
        __shared__ alignas(8) unsigned long long full[STAGES], empty[STAGES];
        if (K <= 0) return true;
        T *As = static_cast<T *>(smem_raw);
        T *Bs = As + STAGES * A_STAGE;
        const int ktiles = (K + BK - 1) / BK;
        if (threadIdx.x == 0) {
#pragma unroll
            for (int s = 0; s < STAGES; ++s) {
                asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(&full[s])), "r"(kThreads));
                asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(&empty[s])), "r"(kThreads / 32));
            }
            asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        }
        __syncthreads();
        const unsigned long long deadline = global_ns() + 1000000000ull;
        bool ok = true;
        auto wait = [&](unsigned long long *bar, uint32_t parity) {
            for (unsigned it = 0; ok; ++it) {
                uint32_t done;
                asm volatile(
                    "{\n\t.reg .pred p;\n\t"
                    "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                    "selp.u32 %0, 1, 0, p;\n\t}"
                    : "=r"(done)
                    : "r"(smem_u32(bar)), "r"(parity)
                    : "memory");
                if (done) return;
                if ((it & 63) == 63 && global_ns() > deadline) ok = false;
            }
        };
        auto fill = [&](int slice) {
            const int st = slice % STAGES;
            load_a(As + st * A_STAGE, A, lda, M, K, slice * BK);
            load_b(Bs + st * B_STAGE, B, ldb, N, K, slice * BK);
            asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];" ::"r"(smem_u32(&full[st])) : "memory");
        };
#pragma unroll
        for (int s = 0; s < STAGES - 1; ++s)
            if (s < ktiles) fill(s);
        for (int kt = 0; kt < ktiles; ++kt) {
            const int st = kt % STAGES;
            wait(&full[st], (kt / STAGES) & 1);
#if MTD_EARLY_CLAIM2
            if (kt == ktiles - 1 && threadIdx.x == 0) on_last();  // thread 0, before the last slice
#endif
            compute_stage(As + st * A_STAGE, Bs + st * B_STAGE);
            __syncwarp();
            if ((threadIdx.x & 31) == 0)
                asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(&empty[st])) : "memory");
            const int nk = kt + STAGES - 1;
            if (nk < ktiles) {
                if (kt >= 1) wait(&empty[nk % STAGES], ((kt - 1) / STAGES) & 1);  // slice kt - 1 read by all
                fill(nk);
            }
        }
        asm volatile("cp.async.wait_all;" ::: "memory");
#if MTD_EARLY_CLAIM2
        __syncthreads();
#else
        if (end_sync) __syncthreads();
#endif
        return ok;
    }

    // C block staging of run_sp_update: four chunks of BN / 4 columns, each [column][row] with
    // the A stage's padded row stride, in the A and B stages of the two slices before the last.
    static constexpr int kCCols = BN / 4;
    static constexpr int kCLd = BM + SmemPad<T>::a;
    static constexpr int kCPiecesPerCol = BM / EPC;                   // 16-byte copies per column
    static constexpr int kCColsPerPass = kThreads / kCPiecesPerCol;  // columns one pass of the CTA copies
    static constexpr bool kStageC = sizeof(T) == 8 && STAGES == 3 && AL == kAMContig && BN % 4 == 0 &&
                                    kCCols * kCLd <= A_STAGE && kCCols * kCLd <= B_STAGE &&
                                    kThreads % kCPiecesPerCol == 0 && kCCols % kCColsPerPass == 0 &&
                                    (kCLd * int(sizeof(T))) % 16 == 0;

    // C(r, c) -= A(M x K) * B(K x N) for r < M, c < N (with lower_only, only where r >= c): the
    // update items' k-loop and C update in one.  The split-phase k-loop of run_sp, except that
    // before computing the last slice every thread copies its share of the C block (cp.async)
    // into the stages the two slices before it used (once every warp has read them), so the
    // read half of the read-modify-write overlaps that slice's compute instead of following it;
    // each warp then subtracts its accumulators from the staged C and stores the result.  Needs
    // at least three slices, 16-byte aligned C columns and M a multiple of the copy width, else
    // it runs run_sp and sub_from.  Ends without a CTA barrier: the caller passes one before
    // shared memory or the barriers are used again.  Returns false if a wait ran past ~1 s.
    __device__ __forceinline__ bool run_sp_update(void *smem_raw, const T *A, int64_t lda, const T *B, int64_t ldb,
                                                  int M, int N, int K, T *C, int64_t ldc, bool lower_only) {
        const int ktiles = (K + BK - 1) / BK;
        if constexpr (kStageC) {
            if (ktiles >= 3 && VEC == 2 && M % EPC == 0 && ldc % EPC == 0 &&
                (reinterpret_cast<uintptr_t>(C) & 15) == 0)
                return run_sp_staged_c(smem_raw, A, lda, B, ldb, M, N, K, C, ldc, lower_only);
        }
#if MTD_EARLY_CLAIM2
        if (!run_sp(smem_raw, A, lda, B, ldb, M, N, K)) return false;
#else
        if (!run_sp(smem_raw, A, lda, B, ldb, M, N, K, false)) return false;
#endif
        sub_from(C, ldc, M, N, lower_only, 0, 0);
        return true;
    }

    __device__ __forceinline__ bool run_sp_staged_c(void *smem_raw, const T *A, int64_t lda, const T *B, int64_t ldb,
                                                    int M, int N, int K, T *C, int64_t ldc, bool lower_only) {
        __shared__ alignas(8) unsigned long long full[STAGES], empty[STAGES], cfull;
#if MTD_STAGE_C_PARK
        // C, ldc and lower wait in shared memory during the k-loop, out of its registers
        __shared__ T *park_c;
        __shared__ int64_t park_ldc;
        __shared__ int park_lower;
        if (threadIdx.x == 0) {
            park_c = C;
            park_ldc = ldc;
            park_lower = lower_only ? 1 : 0;
        }
#endif
        T *As = static_cast<T *>(smem_raw);
        T *Bs = As + STAGES * A_STAGE;
        const int ktiles = (K + BK - 1) / BK;  // >= 3
        if (threadIdx.x == 0) {
#pragma unroll
            for (int s = 0; s < STAGES; ++s) {
                asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(&full[s])), "r"(kThreads));
                asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(&empty[s])), "r"(kThreads / 32));
            }
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(&cfull)), "r"(kThreads));
            asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        }
        __syncthreads();
        const unsigned long long deadline = global_ns() + 1000000000ull;
        bool ok = true;
        auto wait = [&](unsigned long long *bar, uint32_t parity) {
            for (unsigned it = 0; ok; ++it) {
                uint32_t done;
                asm volatile(
                    "{\n\t.reg .pred p;\n\t"
                    "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                    "selp.u32 %0, 1, 0, p;\n\t}"
                    : "=r"(done)
                    : "r"(smem_u32(bar)), "r"(parity)
                    : "memory");
                if (done) return;
                if ((it & 63) == 63 && global_ns() > deadline) ok = false;
            }
        };
        auto fill = [&](int slice) {
            const int st = slice % STAGES;
            load_a(As + st * A_STAGE, A, lda, M, K, slice * BK);
            load_b(Bs + st * B_STAGE, B, ldb, N, K, slice * BK);
            asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];" ::"r"(smem_u32(&full[st])) : "memory");
        };
        // C chunk q: the A (q = 0, 1) or B (q = 2, 3) stage of slice ktiles - 2 (q even) or
        // ktiles - 3 (q odd)
        auto chunk = [&](int q) {
            const int s = (ktiles - 2 - (q & 1)) % STAGES;
            return q < 2 ? As + s * A_STAGE : Bs + s * B_STAGE;
        };
#pragma unroll
        for (int s = 0; s < STAGES - 1; ++s) fill(s);
        for (int kt = 0; kt < ktiles; ++kt) {
            const int st = kt % STAGES;
            wait(&full[st], (kt / STAGES) & 1);
            if (kt == ktiles - 1) {
#if MTD_STAGE_C_PARK
                C = *static_cast<T *volatile *>(&park_c);
                ldc = *static_cast<volatile int64_t *>(&park_ldc);
#endif
                // every warp has read slices kt - 1 and kt - 2: their stages take the C block
                wait(&empty[(kt - 1) % STAGES], ((kt - 1) / STAGES) & 1);
                wait(&empty[(kt - 2) % STAGES], ((kt - 2) / STAGES) & 1);
                const int r = EPC * (threadIdx.x % kCPiecesPerCol);
                const int c_in = threadIdx.x / kCPiecesPerCol;
#pragma unroll
                for (int u = 0; u < BN / kCColsPerPass; ++u) {
                    constexpr int kPassesPerChunk = kCCols / kCColsPerPass;
                    const int c = u * kCColsPerPass + c_in;
                    const bool in = r < M && c < N;
                    cp_async16(chunk(u / kPassesPerChunk) + (c - (u / kPassesPerChunk) * kCCols) * kCLd + r,
                               in ? C + r + int64_t(c) * ldc : C, in);
                }
                asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];" ::"r"(smem_u32(&cfull)) : "memory");
            }
            compute_stage(As + st * A_STAGE, Bs + st * B_STAGE);
            __syncwarp();
            if ((threadIdx.x & 31) == 0)
                asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(&empty[st])) : "memory");
            const int nk = kt + STAGES - 1;
            if (nk < ktiles) {
                if (kt >= 1) wait(&empty[nk % STAGES], ((kt - 1) / STAGES) & 1);  // slice kt - 1 read by all
                fill(nk);
            }
        }
        wait(&cfull, 0);
#if MTD_STAGE_C_PARK
        lower_only = *static_cast<volatile int *>(&park_lower) != 0;
#endif
        if (ok) {
            const int lane = threadIdx.x & 31;
            const int warp = threadIdx.x >> 5;
            const int wm0 = (warp / WARPS_N) * WM;
            const int wn0 = (warp % WARPS_N) * WN;
            const int g = lane >> 2;
            const int t = lane & 3;
#pragma unroll
            for (int i = 0; i < FM; ++i)
#pragma unroll
                for (int j = 0; j < FN; ++j)
#pragma unroll
                    for (int v = 0; v < 4; ++v) {
                        const int r = wm0 + i * 16 + g + ((v & 2) ? 8 : 0);
                        const int c = wn0 + j * 8 + 2 * t + (v & 1);
                        if (r < M && c < N && (!lower_only || r >= c)) {
                            const int q = c / kCCols;
                            C[r + int64_t(c) * ldc] = chunk(q)[(c - q * kCCols) * kCLd + r] - acc[i][j][v];
                        }
                    }
        }
        asm volatile("cp.async.wait_all;" ::: "memory");
        return ok;
    }

    // Visit every accumulator element inside the M x N block: f(row, col, value).
    template <typename F>
    __device__ __forceinline__ void for_each(int M, int N, F &&f) const {
        const int lane = threadIdx.x & 31;
        const int warp = threadIdx.x >> 5;
        const int wm0 = (warp / WARPS_N) * WM;
        const int wn0 = (warp % WARPS_N) * WN;
        const int g = lane >> 2;
        const int t = lane & 3;
#pragma unroll
        for (int i = 0; i < FM; ++i)
#pragma unroll
            for (int j = 0; j < FN; ++j)
#pragma unroll
                for (int v = 0; v < 4; ++v) {
                    const int r = wm0 + i * 16 + g + ((v & 2) ? 8 : 0);
                    const int c = wn0 + j * 8 + 2 * t + (v & 1);
                    if (r < M && c < N) f(r, c, acc[i][j][v]);
                }
    }

    // C(r, c) -= acc(r, c); with lower_only, only where (r + r0) >= (c + c0).  The loads of
    // one fragment row (FN x 4 elements) are issued together before any store, so their
    // latencies overlap (interleaved load / store pairs would wait for each load in turn).
    __device__ __forceinline__ void sub_from(T *C, int64_t ldc, int M, int N, bool lower_only = false, int r0 = 0,
                                             int c0 = 0) const {
        const int lane = threadIdx.x & 31;
        const int warp = threadIdx.x >> 5;
        const int wm0 = (warp / WARPS_N) * WM;
        const int wn0 = (warp % WARPS_N) * WN;
        const int g = lane >> 2;
        const int t = lane & 3;
#pragma unroll
        for (int i = 0; i < FM; ++i) {
            T cv[FN][4];
#pragma unroll
            for (int j = 0; j < FN; ++j)
#pragma unroll
                for (int v = 0; v < 4; ++v) {
                    const int r = wm0 + i * 16 + g + ((v & 2) ? 8 : 0);
                    const int c = wn0 + j * 8 + 2 * t + (v & 1);
                    const bool in = r < M && c < N && (!lower_only || r + r0 >= c + c0);
                    cv[j][v] = in ? ld_cg(C + r + int64_t(c) * ldc) : T(0);
                }
#pragma unroll
            for (int j = 0; j < FN; ++j)
#pragma unroll
                for (int v = 0; v < 4; ++v) {
                    const int r = wm0 + i * 16 + g + ((v & 2) ? 8 : 0);
                    const int c = wn0 + j * 8 + 2 * t + (v & 1);
                    if (r < M && c < N && (!lower_only || r + r0 >= c + c0))
                        C[r + int64_t(c) * ldc] = cv[j][v] - acc[i][j][v];
                }
        }
    }

    // S[idx(r, c)] = C(r, c) - acc(r, c) for r < M, c < N and 0 elsewhere in the BM x BN block;
    // S in shared memory at the offsets idx gives.  The loads of one fragment row are issued
    // together, as in sub_from.
    template <typename Idx>
    __device__ __forceinline__ void sub_to_smem(const T *C, int64_t ldc, int M, int N, T *S, Idx &&idx) const {
        const int lane = threadIdx.x & 31;
        const int warp = threadIdx.x >> 5;
        const int wm0 = (warp / WARPS_N) * WM;
        const int wn0 = (warp % WARPS_N) * WN;
        const int g = lane >> 2;
        const int t = lane & 3;
#pragma unroll
        for (int i = 0; i < FM; ++i) {
            T cv[FN][4];
#pragma unroll
            for (int j = 0; j < FN; ++j)
#pragma unroll
                for (int v = 0; v < 4; ++v) {
                    const int r = wm0 + i * 16 + g + ((v & 2) ? 8 : 0);
                    const int c = wn0 + j * 8 + 2 * t + (v & 1);
                    cv[j][v] = (r < M && c < N) ? ld_cg(C + r + int64_t(c) * ldc) : T(0);
                }
#pragma unroll
            for (int j = 0; j < FN; ++j)
#pragma unroll
                for (int v = 0; v < 4; ++v) {
                    const int r = wm0 + i * 16 + g + ((v & 2) ? 8 : 0);
                    const int c = wn0 + j * 8 + 2 * t + (v & 1);
                    S[idx(r, c)] = (r < M && c < N) ? cv[j][v] - acc[i][j][v] : T(0);
                }
        }
    }

    // C(r, c) = acc(r, c).
    __device__ __forceinline__ void store_to(T *C, int64_t ldc, int M, int N) const {
        for_each(M, N, [&](int r, int c, T v) { C[r + int64_t(c) * ldc] = v; });
    }

    // C(r, c) = acc(r, c) rounded to nearest BF16 (the copy BF16 updates read).
    __device__ __forceinline__ void store_bf16_to(__nv_bfloat16 *C, int64_t ldc, int M, int N) const {
        for_each(M, N, [&](int r, int c, T v) { C[r + int64_t(c) * ldc] = __float2bfloat16_rn(float(v)); });
    }

    // C(r, c) = the low part of acc(r, c) for three-pass TF32 products: v minus v truncated to
    // TF32 (the part a tensor core reading v's bits uses), rounded to nearest TF32.
    __device__ __forceinline__ void store_lo_to(float *C, int64_t ldc, int M, int N) const {
        for_each(M, N, [&](int r, int c, T v) {
            const float x = float(v);
            const float lo = x - __uint_as_float(__float_as_uint(x) & 0xffffe000u);
            C[r + int64_t(c) * ldc] = __uint_as_float(to_tf32(lo));
        });
    }

    // C(r, c) = acc(r, c) as the tensor cores of this mode read it: rounded to nearest TF32
    // for single TF32 products (so later products that truncate their operands see the
    // rounded value), unchanged for FP64 and split-TF32.
    __device__ __forceinline__ void store_rounded_to(T *C, int64_t ldc, int M, int N) const {
        for_each(M, N, [&](int r, int c, T v) { C[r + int64_t(c) * ldc] = frag_round<SPLIT>(v); });
    }
};

template <int BM, int BN, int WARPS_M, int WARPS_N, int BL, int VEC, int STAGES = 3, int BK_ = 16>
using BlockMma = BlockMmaT<double, BM, BN, WARPS_M, WARPS_N, BL, VEC, STAGES, BK_>;

}  // namespace mtd
