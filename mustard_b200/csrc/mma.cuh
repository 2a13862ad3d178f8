// FP64 block-GEMM engine for one CTA of 256 threads on sm_100a.
//
// acc(BM x BN) += A(BM x K) * B(K x BN), operands read from global memory (L2) into a
// multi-stage shared-memory ring with cp.async.cg (16-byte, L1-bypassing: tiles written
// by other CTAs of the persistent kernel are never read from a stale L1 line), and
// multiplied with the FP64 tensor-core instruction mma.sync.m16n8k8.f64.  sm_100a's
// tcgen05 MMA has no FP64 kind, so DMMA is the FP64 tensor path on B200; a register-only
// probe measures it at the same 37 TFLOP/s as the datasheet's FP64 figure.
//
// Layouts (column-major global memory):
//   A(m, k) = A[m + k * lda]                                   ("m-contiguous")
//   B(k, n) = B[n + k * ldb]   when BL == kBNContig            (Cholesky: B = L(i,k)^T)
//   B(k, n) = B[k + n * ldb]   when BL == kBKContig            (LU:       B = U(k,j))
// Shared-memory rows are padded to 4 (mod 16) doubles so every fragment load of a
// half-warp touches 16 distinct 8-byte bank pairs.
//
// VEC == 2: 16-byte copies; needs 16-byte aligned bases, even leading dimensions and
// even extents (the host checks).  VEC == 1: 8-byte loads through registers, any shape.
#pragma once

#include <cstdint>

#include "device_types.hpp"

namespace mtd {

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

__device__ __forceinline__ void dmma_16x8x8(double (&d)[4], const double (&a)[4], const double (&b)[2]) {
    asm volatile(
        "mma.sync.aligned.m16n8k8.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+d"(d[0]), "+d"(d[1]), "+d"(d[2]), "+d"(d[3])
        : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(b[0]), "d"(b[1]));
}

template <int BM, int BN, int WARPS_M, int WARPS_N, int BL, int VEC, int STAGES = 3, int BK_ = 16>
struct BlockMma {
    static constexpr int BK = BK_;
    static constexpr int WM = BM / WARPS_M;
    static constexpr int WN = BN / WARPS_N;
    static constexpr int FM = WM / 16;
    static constexpr int FN = WN / 8;
    static constexpr int LDA = BM + 4;
    static constexpr int LDB = (BL == kBNContig) ? BN + 4 : BK + 4;
    static constexpr int A_STAGE = BK * LDA;
    static constexpr int B_STAGE = (BL == kBNContig) ? BK * LDB : BN * LDB;
    static constexpr int SMEM_DOUBLES = STAGES * (A_STAGE + B_STAGE);
    static_assert(WARPS_M * WARPS_N * 32 == kThreads, "one warp tile per warp of the CTA");
    static_assert(FM >= 1 && FN >= 1 && WM % 16 == 0 && WN % 8 == 0, "warp tile");
    static_assert(LDA % 16 == 4 && LDB % 16 == 4, "bank-conflict-free padding");

    double acc[FM][FN][4];

    __device__ __forceinline__ void zero() {
#pragma unroll
        for (int i = 0; i < FM; ++i)
#pragma unroll
            for (int j = 0; j < FN; ++j)
#pragma unroll
                for (int v = 0; v < 4; ++v) acc[i][j][v] = 0.0;
    }

    // ---- global -> shared stage loads ----
    __device__ __forceinline__ static void load_a(double *As, const double *A, int64_t lda, int M, int K,
                                                  int k0) {
        const int tid = threadIdx.x;
        if (VEC == 2) {
            constexpr int CH = BK * (BM / 2);
#pragma unroll
            for (int c = tid; c < CH; c += kThreads) {
                const int col = c / (BM / 2);
                const int row = 2 * (c % (BM / 2));
                const int kk = k0 + col;
                const bool ok = row < M && kk < K;
                const double *src = ok ? A + row + int64_t(kk) * lda : A;
                cp_async16(As + col * LDA + row, src, ok);
            }
        } else {
            constexpr int EL = BK * BM;
            for (int e = tid; e < EL; e += kThreads) {
                const int col = e / BM;
                const int row = e % BM;
                const int kk = k0 + col;
                As[col * LDA + row] = (row < M && kk < K) ? ld_cg(A + row + int64_t(kk) * lda) : 0.0;
            }
        }
    }

    __device__ __forceinline__ static void load_b(double *Bs, const double *B, int64_t ldb, int N, int K,
                                                  int k0) {
        const int tid = threadIdx.x;
        if (BL == kBNContig) {
            if (VEC == 2) {
                constexpr int CH = BK * (BN / 2);
#pragma unroll
                for (int c = tid; c < CH; c += kThreads) {
                    const int col = c / (BN / 2);
                    const int n = 2 * (c % (BN / 2));
                    const int kk = k0 + col;
                    const bool ok = n < N && kk < K;
                    const double *src = ok ? B + n + int64_t(kk) * ldb : B;
                    cp_async16(Bs + col * LDB + n, src, ok);
                }
            } else {
                constexpr int EL = BK * BN;
                for (int e = tid; e < EL; e += kThreads) {
                    const int col = e / BN;
                    const int n = e % BN;
                    const int kk = k0 + col;
                    Bs[col * LDB + n] = (n < N && kk < K) ? ld_cg(B + n + int64_t(kk) * ldb) : 0.0;
                }
            }
        } else {
            if (VEC == 2) {
                constexpr int CH = BN * (BK / 2);
#pragma unroll
                for (int c = tid; c < CH; c += kThreads) {
                    const int n = c / (BK / 2);
                    const int k = 2 * (c % (BK / 2));
                    const int kk = k0 + k;
                    const bool ok = n < N && kk < K;
                    const double *src = ok ? B + kk + int64_t(n) * ldb : B;
                    cp_async16(Bs + n * LDB + k, src, ok);
                }
            } else {
                constexpr int EL = BN * BK;
                for (int e = tid; e < EL; e += kThreads) {
                    const int n = e / BK;
                    const int k = e % BK;
                    const int kk = k0 + k;
                    Bs[n * LDB + k] = (n < N && kk < K) ? ld_cg(B + kk + int64_t(n) * ldb) : 0.0;
                }
            }
        }
    }

    __device__ __forceinline__ void compute_stage(const double *As, const double *Bs) {
        const int lane = threadIdx.x & 31;
        const int warp = threadIdx.x >> 5;
        const int wm0 = (warp / WARPS_N) * WM;
        const int wn0 = (warp % WARPS_N) * WN;
        const int g = lane >> 2;
        const int t = lane & 3;
#pragma unroll
        for (int ks = 0; ks < BK; ks += 8) {
            double bf[FN][2];
#pragma unroll
            for (int j = 0; j < FN; ++j) {
                const int n = wn0 + j * 8 + g;
                if (BL == kBNContig) {
                    bf[j][0] = Bs[(ks + t) * LDB + n];
                    bf[j][1] = Bs[(ks + t + 4) * LDB + n];
                } else {
                    bf[j][0] = Bs[n * LDB + ks + t];
                    bf[j][1] = Bs[n * LDB + ks + t + 4];
                }
            }
#pragma unroll
            for (int i = 0; i < FM; ++i) {
                const int m = wm0 + i * 16 + g;
                double af[4];
                af[0] = As[(ks + t) * LDA + m];
                af[1] = As[(ks + t) * LDA + m + 8];
                af[2] = As[(ks + t + 4) * LDA + m];
                af[3] = As[(ks + t + 4) * LDA + m + 8];
#pragma unroll
                for (int j = 0; j < FN; ++j) dmma_16x8x8(acc[i][j], af, bf[j]);
            }
        }
    }

    // acc += A(M x K) * B(K x N).  M <= BM, N <= BN; rows/columns beyond M/N and depth
    // beyond K are zero-filled.  All 256 threads must call; shared memory is free again
    // on return.
    __device__ __forceinline__ void run(double *smem, const double *A, int64_t lda, const double *B,
                                        int64_t ldb, int M, int N, int K) {
        if (K <= 0) return;
        double *As = smem;
        double *Bs = smem + STAGES * A_STAGE;
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
            compute_stage(As + st * A_STAGE, Bs + st * B_STAGE);
            const int nk = kt + STAGES - 1;
            if (nk < ktiles) {
                const int ns = nk % STAGES;
                load_a(As + ns * A_STAGE, A, lda, M, K, nk * BK);
                load_b(Bs + ns * B_STAGE, B, ldb, N, K, nk * BK);
            }
            cp_async_commit();
        }
        cp_async_wait<0>();
        __syncthreads();
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

    // C(r, c) -= acc(r, c); with lower_only, only where (r + r0) >= (c + c0).
    __device__ __forceinline__ void sub_from(double *C, int64_t ldc, int M, int N, bool lower_only = false,
                                             int r0 = 0, int c0 = 0) const {
        for_each(M, N, [&](int r, int c, double v) {
            if (!lower_only || r + r0 >= c + c0) {
                double *p = C + r + int64_t(c) * ldc;
                *p = ld_cg(p) - v;
            }
        });
    }

    // C(r, c) = acc(r, c).
    __device__ __forceinline__ void store_to(double *C, int64_t ldc, int M, int N) const {
        for_each(M, N, [&](int r, int c, double v) { C[r + int64_t(c) * ldc] = v; });
    }
};

}  // namespace mtd
