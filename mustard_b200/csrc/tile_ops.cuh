// Tile operations executed by one persistent CTA per work item.
//
// Each operation replaces one captured cuBLAS / cuSOLVER call of the reference
// (mustard/cholesky_mustard.cu:238-387, mustard/lu_mustard.cu:361-522).  The dense
// updates are tensor-core block products (mma.cuh).  The diagonal factorisations are
// left-looking blocked algorithms with kNB-wide diagonal blocks factored in shared
// memory; while a block is in shared memory its triangular inverse is formed and left in
// the inverse workspace (indexed by the block's first matrix row), so every triangular
// solve -- inside the diagonal task and in the TRSM tasks that follow it -- becomes a
// block product as well.  Block geometry comes from the task (DevTask), in elements.
//
// The Cholesky operations are templated on the element type: double (FP64 DMMA, the
// reference's arithmetic) or float (FP32 storage, TF32 tensor-core products with FP32
// accumulation, FP32 diagonal blocks) for the low-precision factor of the mixed-precision
// solver.  The LU operations are FP64 only.
#pragma once

#include <type_traits>

#include "device_types.hpp"
#include "mma.cuh"
#include "tma64.cuh"
#include "../../include/mustard_b200.h"

namespace mtd {

constexpr int kDiagLd = kNB + 1;  // shared-memory leading dimension of a diagonal block

// Engine shapes.  GEMM / SYRK items: kGemmTile x kGemmTile output per CTA; panel work
// (TRSM strips, diagonal factorisations): 64 x 64 blocks.  Defaults measured best on B200
// at N = 24000 (512-thread CTAs, 4 x 4 warps of 32 x 32, 32-deep k-slices, 3 stages: 25.4 /
// 26.5 TFLOP/s Cholesky / LU at tile 768, against 22.2 / 23.8 for 256 threads and 16-deep
// slices, where only two warps per SM sub-partition could not hide the DMMA latencies).
#ifndef MTD_GEMM_WARPS_M
#define MTD_GEMM_WARPS_M 4
#endif
#ifndef MTD_GEMM_STAGES
#define MTD_GEMM_STAGES 3
#endif
#ifndef MTD_GEMM_BK
#define MTD_GEMM_BK 32
#endif
#ifndef MTD_PANEL_WARPS_M
#define MTD_PANEL_WARPS_M 4
#endif
// Panel engine (64 x 64 blocks: TRSM strips, updates inside diagonal factorisations):
// 4 stages of 32-deep k-slices.  Measured at N = 32768, tile 1536: TRSM item 598 -> 398 us
// (TF32) and 957 -> 886 us (FP64) against 3 stages of 16, whose ~24 KB in flight left each
// step waiting on L2 round trips; 5-6 stages or 64-deep slices gave nothing more.
#ifndef MTD_PANEL_STAGES
#define MTD_PANEL_STAGES 4
#endif
#ifndef MTD_PANEL_BK
#define MTD_PANEL_BK 32
#endif
constexpr int kGemmWarpsM = MTD_GEMM_WARPS_M;
constexpr int kGemmWarpsN = kThreads / 32 / kGemmWarpsM;
constexpr int kPanelWarpsM = MTD_PANEL_WARPS_M;
constexpr int kPanelWarpsN = kThreads / 32 / kPanelWarpsM;
template <int BL, int VEC, typename T = double, int SPLIT = 1>
using GemmMma =
    BlockMmaT<T, kGemmTile, kGemmTile, kGemmWarpsM, kGemmWarpsN, BL, VEC, MTD_GEMM_STAGES, MTD_GEMM_BK, SPLIT>;
template <int BL, int VEC, typename T = double, int SPLIT = 1>
using PanelMma = BlockMmaT<T, 64, 64, kPanelWarpsM, kPanelWarpsN, BL, VEC, MTD_PANEL_STAGES, MTD_PANEL_BK, SPLIT>;
// The TRSM strips' updates over two inverse blocks at a time (MTD_TRSM_WIDE=1): 64 x 128
// (row strips: TRSM_RLT, TRSM_RUN) and 128 x 64 (column strips: TRSM_LLNU) output blocks,
// one 16 x 32 warp tile per warp; half the steps, each with one engine fill and one C
// update.  Measured on one B200 (N = 24000, tile 1536): Cholesky 153.5 -> 151.3 ms, LU
// unchanged (297.8 / 297.6 ms).
#ifndef MTD_TRSM_WIDE
#define MTD_TRSM_WIDE 1
#endif
template <int BL, int VEC, typename T = double, int SPLIT = 1>
using WideMma = BlockMmaT<T, 64, 128, 4, kThreads / 32 / 4, BL, VEC, MTD_PANEL_STAGES, MTD_PANEL_BK, SPLIT>;
template <int VEC, int BL = kBKContig, typename T = double, int SPLIT = 1>
using TallMma = BlockMmaT<T, 128, 64, kThreads / 32 / 2, 2, BL, VEC, MTD_PANEL_STAGES, MTD_PANEL_BK, SPLIT>;
// The engines of one TRSM strip: its solve steps (kTrsmRows x 64 blocks: row strips; 64 x
// kTrsmRows: column strips) and its updates over two inverse blocks (kTrsmRows x 128 and
// 128 x kTrsmRows).  128-row strips run their updates on the 128 x 128 update engine.
template <int BL, int VEC, typename T = double, int SPLIT = 1>
using StripStep = std::conditional_t<kTrsmRows == 128, TallMma<VEC, BL, T, SPLIT>, PanelMma<BL, VEC, T, SPLIT>>;
template <int BL, int VEC, typename T = double, int SPLIT = 1>
using StripUpdate = std::conditional_t<kTrsmRows == 128, GemmMma<BL, VEC, T, SPLIT>, WideMma<BL, VEC, T, SPLIT>>;
template <int VEC>
using ColStripStep = std::conditional_t<kTrsmRows == 128, WideMma<kBKContig, VEC>, PanelMma<kBKContig, VEC>>;
template <int VEC>
using ColStripUpdate = std::conditional_t<kTrsmRows == 128, GemmMma<kBKContig, VEC>, TallMma<VEC>>;

// 1: the diagonal factorisations and the TRSM strips are separate (not inlined) functions, so
// the update items' paths of the persistent kernel are allocated without them.
#ifndef MTD_NOINLINE_PANEL_OPS
#define MTD_NOINLINE_PANEL_OPS 0
#endif
#if MTD_NOINLINE_PANEL_OPS
#define MTD_PANEL_OP_LINKAGE static __device__ __noinline__
#else
#define MTD_PANEL_OP_LINKAGE __device__
#endif

__device__ __forceinline__ void block_fence_sync() {
    __threadfence_block();
    __syncthreads();
}

// The matrix one task works on: the run's matrix, or in a batched run the task's own
// matrix (DevTask::mat), with its inverse workspace.
struct MatCtx {
    void *a;
    int64_t lda;
    void *wsl;
    void *wsu;
    int64_t wsld;
    int mat;  // -1 for a single-matrix run
};

template <typename T>
__device__ __forceinline__ MatCtx mat_ctx(const RunArgs &p, const DevTask &t) {
    if (p.mats == nullptr) return MatCtx{p.a, p.lda, p.ws_lower, p.ws_upper, p.ws_ld, -1};
    const BatchMat &bm = p.mats[t.mat];
    return MatCtx{bm.a, bm.lda, static_cast<T *>(p.ws_lower) + bm.ws_off,
                  p.ws_upper ? static_cast<T *>(p.ws_upper) + bm.ws_off : nullptr, bm.ws_ld, t.mat};
}

template <typename T>
__device__ __forceinline__ T *at(const MatCtx &m, int r, int c) {
    return static_cast<T *>(m.a) + r + int64_t(c) * m.lda;
}
template <typename T>
__device__ __forceinline__ T *ws_lo(const MatCtx &m) { return static_cast<T *>(m.wsl); }
template <typename T>
__device__ __forceinline__ T *ws_up(const MatCtx &m) { return static_cast<T *>(m.wsu); }

__device__ __forceinline__ void report_error(RunCtl *ctl, int code, int info) {
    if (info > 0) atomicMin(&ctl->info, info);
    atomicCAS(&ctl->error, 0, code);
    __threadfence();
    atomicExch(&ctl->abort, 1);
}

// A diagonal factorisation met a bad pivot (thread 0 reports).  A single-matrix run stops
// with the error; a batched run records LAPACK-style info for that matrix only and lets
// the task complete, so the other matrices of the batch finish (the failed matrix's
// factor is left partial, as LAPACK's batched routines leave it).  Returns the status the
// task ends with.
__device__ __forceinline__ int diag_failure(const RunArgs &p, const MatCtx &m, int code, int info) {
    if (m.mat < 0) {
        if (threadIdx.x == 0) report_error(p.ctl, code, info);
        return code;
    }
    if (threadIdx.x == 0) atomicMin(p.mat_info + m.mat, info);
    return 0;
}

// X = T^-1 for a jn x jn lower-triangular T read through tl(i, l) (i >= l); unit
// diagonal when UNIT.  Four lanes per column (64 columns); rows swept top-down.
template <bool UNIT, typename E, typename TL>
__device__ __forceinline__ void lower_inverse(int jn, TL tl, E *X) {
    const int c = threadIdx.x >> 2;
    const int q = threadIdx.x & 3;
    for (int i = 0; i < jn; ++i) {
        E part = E(0);
        if (c < i)
            for (int l = c + q; l < i; l += 4) part += tl(i, l) * X[l + c * kDiagLd];
        part += __shfl_xor_sync(0xffffffffu, part, 1);
        part += __shfl_xor_sync(0xffffffffu, part, 2);
        if (q == 0 && c < jn) {
            E v;
            if (c > i) v = E(0);
            else if (UNIT) v = (c == i) ? E(1) : -part;
            else v = (c == i) ? E(1) / tl(i, i) : -part / tl(i, i);
            X[i + c * kDiagLd] = v;
        }
        __syncwarp();
    }
    __syncthreads();
}

// Cholesky of the n x n diagonal block at Ad (n <= kSmallChol, lower; the strict upper
// triangle is never touched, as with LAPACK's uplo = 'L'), and the inverses of its kNB-row
// diagonal blocks to Wd (Wd[r + c * ldw], full kNB x kNB blocks with zeros above the
// diagonal).  The block is held in shared memory and factored in panels of PW columns
// (16 in FP64, 32 in FP32, so that a row of the panel fits in registers):
//   - warp 0 factors the panel's PW x PW diagonal block in registers (lane r holds row r;
//     column j is broadcast with shuffles: no block barrier inside the panel) with the
//     arithmetic of LAPACK's dpotf2 (l(r, j) = d(r, j) * (1 / sqrt(d(j, j))), then the
//     rank-1 update; the reciprocal square root is CUDA's rsqrt, within 1 ulp), and then
//     its inverse (lane c forms column c by forward substitution);
//   - the whole CTA computes the panel below it, P = A_panel X^T, and the trailing update
//     A -= P P^T (lower), each followed by one barrier.
// The kNB x kNB inverses are composed from the panel inverses by doubling:
// inv([La 0; L21 Lb]) = [Xa 0; -Xb (L21 Xa) Xb].
// (The first design synchronised the CTA three times per column and formed the inverse
// row by row: ~170 us for a 128 x 128 block, which made the chain of nested diagonal
// factorisations the critical path of the TF32 factor.)
constexpr int kSmallChol = 128;
constexpr int kSmallLd = kSmallChol + 1;
constexpr int kInvLd = kNB + 1;
template <typename T>
constexpr int chol_panel() {
    return sizeof(T) == 8 ? 16 : 32;
}
template <typename T>
constexpr int chol_small_smem_bytes() {
    // the block, the inverses of its two kNB-row diagonal blocks, a 2 x 32 x 33 scratch
    // product, 1 / L(r, r), the failure flag
    return int(sizeof(T)) * (kSmallChol * kSmallLd + 2 * kNB * kInvLd + 2 * 32 * 33 + kSmallChol + 1);
}

// Warp 0: Cholesky of the pw x pw block at S(p0, p0) (pw <= PW) in registers, L written
// back to S (lower part), 1 / L(r, r) to rdiag[r], and X = L^-1 to X (leading dimension
// kInvLd, lower part).  Returns the 0-based column of the first non-positive pivot, or -1.
template <typename T, int PW>
__device__ __forceinline__ int warp_chol(T *S, int p0, int pw, T *rdiag, T *X) {
    const int lane = threadIdx.x & 31;
    const unsigned full = 0xffffffffu;
    T a[PW];
#pragma unroll
    for (int c = 0; c < PW; ++c)
        a[c] = (lane < pw && c <= lane) ? S[(p0 + lane) + (p0 + c) * kSmallLd] : T(0);
    T myd = T(1), myrs = T(1);
    int bad = -1;
#pragma unroll
    for (int j = 0; j < PW; ++j) {
        if (j < pw && bad < 0) {
            const T d = __shfl_sync(full, a[j], j);
            if (!(d > T(0))) {  // also catches NaN; the same value in every lane
                bad = j;
            } else {
                const T rs = rsqrt(d);
                if (lane == j) {
                    myd = d;
                    myrs = rs;
                }
                const T l = a[j] * rs;  // l(lane, j) for lane > j
                a[j] = l;
#pragma unroll
                for (int c = j + 1; c < PW; ++c) {
                    const T lc = __shfl_sync(full, l, c);
                    a[c] -= l * lc;
                }
            }
        }
    }
    if (bad >= 0) return bad;
    // L back to S (the diagonal as sqrt of the pivot, formed once here, off the chain)
    if (lane < pw) {
#pragma unroll
        for (int c = 0; c < PW; ++c)
            if (c < lane) S[(p0 + lane) + (p0 + c) * kSmallLd] = a[c];
        S[(p0 + lane) + (p0 + lane) * kSmallLd] = sqrt(myd);
        rdiag[lane] = myrs;
    }
    __syncwarp();
    // X = L^-1: lane c forms column c, rows i >= c, by forward substitution in registers
    // (fully unrolled: the loads of L do not wait on the recurrence, which carries one
    // multiply-add per row: the newest x[i - 1] enters the sum last)
    T x[PW];
#pragma unroll
    for (int i = 0; i < PW; ++i) {
        if (i < pw) {
            T s0 = (i == lane) ? T(1) : T(0), s1 = T(0);
#pragma unroll
            for (int l = 0; l + 1 < i; ++l) {
                const T v = S[(p0 + i) + (p0 + l) * kSmallLd] * x[l];
                if (l & 1) s1 -= v;
                else s0 -= v;
            }
            if (i > 0) s0 -= S[(p0 + i) + (p0 + i - 1) * kSmallLd] * x[i - 1];
            x[i] = (s0 + s1) * rdiag[i];
        } else {
            x[i] = T(0);
        }
    }
    if (lane < pw) {
#pragma unroll
        for (int i = 0; i < PW; ++i)
            if (i >= lane && i < pw) X[i + lane * kInvLd] = x[i];
    }
    return -1;
}

// Not inlined: its register-heavy phases are allocated on their own, so they do not raise
// the register pressure (or cause spills) in the GEMM paths of the persistent kernel.
template <typename T>
__device__ __noinline__ int chol_small(const RunArgs &p, const MatCtx &m, T *Ad, int n, T *Wd, void *smem_raw,
                                      int info_base) {
    static_assert(kThreads == 512, "work split over 512 threads");
    static_assert(kNB == 64, "two kNB-row inverse blocks per 128-row block");
    constexpr int PW = chol_panel<T>();
    const int tid = threadIdx.x;
    T *S = static_cast<T *>(smem_raw);              // the block, then L (column-major, kSmallLd)
    T *XI = S + kSmallChol * kSmallLd;              // inverses of the kNB-row diagonal blocks
    T *T1 = XI + 2 * kNB * kInvLd;                  // scratch products of the composition
    T *rdiag = T1 + 2 * 32 * 33;                    // 1 / L(r, r)
    int *flag = reinterpret_cast<int *>(rdiag + kSmallChol);
    const int64_t lda = m.lda;
    // load the lower triangle: each batch of a thread's loads issues before its stores
    {
        constexpr int kPer = kSmallChol * kSmallChol / kThreads, kBatch = 8;  // 32 elements, 4 batches
        const int r = tid & (kSmallChol - 1);
#pragma unroll 1
        for (int h = 0; h < kPer / kBatch; ++h) {
            T v[kBatch];
#pragma unroll
            for (int i = 0; i < kBatch; ++i) {
                const int c = (tid + (h * kBatch + i) * kThreads) >> 7;
                v[i] = (r < n && c < n && r >= c) ? ld_cg(Ad + r + int64_t(c) * lda) : T(0);
            }
#pragma unroll
            for (int i = 0; i < kBatch; ++i) S[r + ((tid + (h * kBatch + i) * kThreads) >> 7) * kSmallLd] = v[i];
        }
    }
    if (tid == 0) *flag = -1;
    __syncthreads();
    for (int p0 = 0; p0 < n; p0 += PW) {
        const int pw = min(PW, n - p0);
        T *X = XI + (p0 / kNB) * kNB * kInvLd + (p0 % kNB) * (1 + kInvLd);  // panel inverse, kInvLd
        if (tid < 32) {
            const int bad = warp_chol<T, PW>(S, p0, pw, rdiag + p0, X);
            if (tid == 0 && bad >= 0) *flag = p0 + bad;
        }
        __syncthreads();
        const int bad = *flag;  // every thread reads the same flag
        if (bad >= 0) return diag_failure(p, m, MTD_ERR_NOT_POSITIVE_DEFINITE, info_base + bad + 1);
        const int q0 = p0 + pw, nr = n - q0;
        if (nr <= 0) break;
        // panel below: P(r, c) = sum_{l <= c} A(r, p0 + l) X(c, l), rows q0 .., four columns a unit
        {
            const int groups = (pw + 3) >> 2, units = nr * groups;
            T out[2][4];
#pragma unroll
            for (int k = 0; k < 2; ++k) {
                const int u = tid + k * kThreads;
                if (u >= units) continue;
                const int r = q0 + u % nr, c0 = 4 * (u / nr);
                T acc[4] = {T(0), T(0), T(0), T(0)};
#pragma unroll 2
                for (int l = 0; l < PW; ++l) {
                    if (l >= pw) break;
                    const T av = S[r + (p0 + l) * kSmallLd];
#pragma unroll
                    for (int q = 0; q < 4; ++q)
                        if (l <= c0 + q && c0 + q < pw) acc[q] += av * X[(c0 + q) + l * kInvLd];
                }
#pragma unroll
                for (int q = 0; q < 4; ++q) out[k][q] = acc[q];
            }
            __syncthreads();
#pragma unroll
            for (int k = 0; k < 2; ++k) {
                const int u = tid + k * kThreads;
                if (u >= units) continue;
                const int r = q0 + u % nr, c0 = 4 * (u / nr);
#pragma unroll
                for (int q = 0; q < 4; ++q)
                    if (c0 + q < pw) S[r + (p0 + c0 + q) * kSmallLd] = out[k][q];
            }
            __syncthreads();
        }
        // trailing update: A(r, c) -= sum_l P(r, l) P(c, l), r >= c >= q0, in 4 x 4 blocks
        {
            const int nb4 = (nr + 3) >> 2, blocks = nb4 * (nb4 + 1) / 2;
            if (tid < blocks) {
                int br = int((sqrtf(8.0f * float(tid) + 1.0f) - 1.0f) * 0.5f);
                while ((br + 1) * (br + 2) / 2 <= tid) ++br;
                while (br * (br + 1) / 2 > tid) --br;
                const int r0 = q0 + 4 * br, c0 = q0 + 4 * (tid - br * (br + 1) / 2);
                T acc[4][4];
#pragma unroll
                for (int i = 0; i < 4; ++i)
#pragma unroll
                    for (int q = 0; q < 4; ++q) acc[i][q] = T(0);
#pragma unroll 2
                for (int l = 0; l < PW; ++l) {
                    if (l >= pw) break;
                    T x[4], y[4];
#pragma unroll
                    for (int i = 0; i < 4; ++i) {
                        x[i] = S[min(r0 + i, kSmallChol - 1) + (p0 + l) * kSmallLd];
                        y[i] = S[min(c0 + i, kSmallChol - 1) + (p0 + l) * kSmallLd];
                    }
#pragma unroll
                    for (int i = 0; i < 4; ++i)
#pragma unroll
                        for (int q = 0; q < 4; ++q) acc[i][q] += x[i] * y[q];
                }
#pragma unroll
                for (int i = 0; i < 4; ++i)
#pragma unroll
                    for (int q = 0; q < 4; ++q) {
                        const int r = r0 + i, c = c0 + q;
                        if (r < n && c < n && r >= c) S[r + c * kSmallLd] -= acc[i][q];
                    }
            }
            __syncthreads();
        }
    }
    // L to the matrix
    for (int e = tid; e < n * kSmallChol; e += kThreads) {
        const int r = e & (kSmallChol - 1), c = e >> 7;
        if (r < n && r >= c) Ad[r + int64_t(c) * lda] = S[r + c * kSmallLd];
    }
    // kNB-row inverses by doubling: for each pair of adjacent h-blocks (a above b) inside a
    // kNB block, X21 = -Xb (L21 Xa); all pairs of a level at once, two barriers a level
    for (int h = PW; h < kNB; h *= 2) {
        const int pairs = kSmallChol / (2 * h);
        // T1 = L21 Xa  (hb x h per pair; Xa lower)
        for (int e = tid; e < pairs * h * h; e += kThreads) {
            const int pr = e / (h * h), r = e % h, c = (e / h) % h;
            const int g0 = pr * 2 * h, hb = min(h, n - g0 - h);  // rows of the lower half
            if (hb <= 0 || r >= hb) continue;
            const T *Xa = XI + (g0 / kNB) * kNB * kInvLd + (g0 % kNB) * (1 + kInvLd);
            T acc = T(0);
            for (int l = c; l < h; ++l) acc += S[(g0 + h + r) + (g0 + l) * kSmallLd] * Xa[l + c * kInvLd];
            T1[pr * h * (h + 1) + r + c * (h + 1)] = acc;
        }
        __syncthreads();
        // X21 = -Xb T1  (Xb lower), into the composed inverse
        for (int e = tid; e < pairs * h * h; e += kThreads) {
            const int pr = e / (h * h), r = e % h, c = (e / h) % h;
            const int g0 = pr * 2 * h, hb = min(h, n - g0 - h);
            if (hb <= 0 || r >= hb) continue;
            T *Xg = XI + (g0 / kNB) * kNB * kInvLd + (g0 % kNB) * (1 + kInvLd);  // the 2h block
            const T *Xb = Xg + h * (1 + kInvLd);
            T acc = T(0);
            for (int l = 0; l <= r; ++l) acc += Xb[r + l * kInvLd] * T1[pr * h * (h + 1) + l + c * (h + 1)];
            Xg[(h + r) + c * kInvLd] = -acc;
        }
        __syncthreads();
    }
    const int64_t ldw = m.wsld;
    for (int e = tid; e < n * kNB; e += kThreads) {
        const int r = e % n, c = e / n;
        const int b0 = (r / kNB) * kNB;
        if (c < min(kNB, n - b0)) Wd[r + int64_t(c) * ldw] = (r - b0 >= c) ? XI[(b0 / kNB) * kNB * kInvLd + (r - b0) + c * kInvLd] : T(0);
    }
    __syncthreads();
    return 0;
}

// No-pivot LU of the jn x jn diagonal block at Ad, in shared memory (what
// cusolverDnDgetrf computes with ipiv = NULL).  Writes L\U back, L^-1 (unit lower) to
// WLd and U^-1 (upper) to WUd.
__device__ __forceinline__ int factor_lu_diag(const RunArgs &p, const MatCtx &m, double *Ad, int jn, double *WLd, double *WUd,
                                              void *smem_raw, int info_base) {
    const int tid = threadIdx.x;
    double *D = static_cast<double *>(smem_raw);
    double *XL = D + kNB * kDiagLd;
    double *XU = D + 2 * kNB * kDiagLd;
    const int64_t lda = m.lda;
    for (int e = tid; e < jn * jn; e += kThreads) {
        const int r = e % jn, c = e / jn;
        D[r + c * kDiagLd] = ld_cg(Ad + r + int64_t(c) * lda);
    }
    __syncthreads();
    for (int j = 0; j < jn; ++j) {
        const double piv = D[j + j * kDiagLd];
        if (piv == 0.0) return diag_failure(p, m, MTD_ERR_SINGULAR, info_base + j + 1);
        const double rp = 1.0 / piv;
        for (int r = j + 1 + tid; r < jn; r += kThreads) D[r + j * kDiagLd] *= rp;
        __syncthreads();
        const int rest = jn - j - 1;
        for (int e = tid; e < rest * rest; e += kThreads) {
            const int r = j + 1 + e % rest, c = j + 1 + e / rest;
            D[r + c * kDiagLd] -= D[r + j * kDiagLd] * D[j + c * kDiagLd];
        }
        __syncthreads();
    }
    lower_inverse<true>(jn, [&](int i, int l) { return D[i + l * kDiagLd]; }, XL);
    // U^-1 = ((U^T)^-1)^T, and U^T is lower triangular.
    lower_inverse<false>(jn, [&](int i, int l) { return D[l + i * kDiagLd]; }, XU);
    const int64_t ldw = m.wsld;
    for (int e = tid; e < jn * jn; e += kThreads) {
        const int r = e % jn, c = e / jn;
        Ad[r + int64_t(c) * lda] = D[r + c * kDiagLd];
        WLd[r + int64_t(c) * ldw] = XL[r + c * kDiagLd];
        WUd[r + int64_t(c) * ldw] = XU[c + r * kDiagLd];
    }
    return 0;
}

// ---------------------------------------------------------------------------------
// POTRF: left-looking blocked Cholesky of the m x m diagonal block at (cr, cc), one CTA.
// ---------------------------------------------------------------------------------
template <typename T, int VEC, int SPLIT = 1>
MTD_PANEL_OP_LINKAGE int op_potrf(const RunArgs &p, const MatCtx &m, const DevTask &t, void *smem) {
    using Mn = PanelMma<kBNContig, VEC, T, SPLIT>;
    const int n = t.m;
    T *A = at<T>(m, t.cr, t.cc);
    T *W = ws_lo<T>(m) + t.cr;
    const int64_t lda = m.lda, ldw = m.wsld;
    if (n <= kSmallChol) {  // the whole block in shared memory
        const int st = chol_small<T>(p, m, A, n, W, smem, t.cc);
        block_fence_sync();
        return st;
    }
    for (int jb = 0; jb < n; jb += kNB) {
        const int jn = min(kNB, n - jb);
        if (jb > 0) {
            // A[jb:n, jb:jb+jn] -= A[jb:n, 0:jb] * A[jb:jb+jn, 0:jb]^T (lower part of the block)
            for (int r0 = jb; r0 < n; r0 += 64) {
                const int mm = min(64, n - r0);
                Mn e;
                e.zero();
                e.run(smem, A + r0, lda, A + jb, lda, mm, jn, jb);
                e.sub_from(A + r0 + int64_t(jb) * lda, lda, mm, jn, r0 == jb, 0, 0);
            }
            block_fence_sync();
        }
        const int st = chol_small<T>(p, m, A + jb + int64_t(jb) * lda, jn, W + jb, smem, t.cc + jb);
        if (st) return st;
        block_fence_sync();
        // A[jb+jn:n, jb:jb+jn] = A[jb+jn:n, jb:jb+jn] * L_jj^-T
        for (int r0 = jb + jn; r0 < n; r0 += 64) {
            const int mm = min(64, n - r0);
            Mn e;
            e.zero();
            e.run(smem, A + r0 + int64_t(jb) * lda, lda, W + jb, ldw, mm, jn, jn);
            e.store_to(A + r0 + int64_t(jb) * lda, lda, mm, jn);
        }
        block_fence_sync();
    }
    return 0;
}

// ---------------------------------------------------------------------------------
// GETRF without pivoting: left-looking (Crout) blocked LU of the m x m block, one CTA.
// ---------------------------------------------------------------------------------
template <int VEC>
MTD_PANEL_OP_LINKAGE int op_getrf(const RunArgs &p, const MatCtx &m, const DevTask &t, void *smem) {
    using Mk = PanelMma<kBKContig, VEC>;
    const int n = t.m;
    double *A = at<double>(m, t.cr, t.cc);
    double *WL = ws_lo<double>(m) + t.cr;
    double *WU = ws_up<double>(m) + t.cr;
    const int64_t lda = m.lda, ldw = m.wsld;
    for (int jb = 0; jb < n; jb += kNB) {
        const int jn = min(kNB, n - jb);
        if (jb > 0) {
            // block column: A[jb:n, jb:jb+jn] -= A[jb:n, 0:jb] * A[0:jb, jb:jb+jn]
            for (int r0 = jb; r0 < n; r0 += 64) {
                const int mm = min(64, n - r0);
                Mk e;
                e.zero();
                e.run(smem, A + r0, lda, A + int64_t(jb) * lda, lda, mm, jn, jb);
                e.sub_from(A + r0 + int64_t(jb) * lda, lda, mm, jn);
            }
            // block row: A[jb:jb+jn, jb+jn:n] -= A[jb:jb+jn, 0:jb] * A[0:jb, jb+jn:n]
            for (int c0 = jb + jn; c0 < n; c0 += 64) {
                const int nn = min(64, n - c0);
                Mk e;
                e.zero();
                e.run(smem, A + jb, lda, A + int64_t(c0) * lda, lda, jn, nn, jb);
                e.sub_from(A + jb + int64_t(c0) * lda, lda, jn, nn);
            }
            block_fence_sync();
        }
        const int st = factor_lu_diag(p, m, A + jb + int64_t(jb) * lda, jn, WL + jb, WU + jb, smem, t.cc + jb);
        if (st) return st;
        block_fence_sync();
        // L panel: A[jb+jn:n, jb:jb+jn] = A[...] * U_jj^-1
        for (int r0 = jb + jn; r0 < n; r0 += 64) {
            const int mm = min(64, n - r0);
            Mk e;
            e.zero();
            e.run(smem, A + r0 + int64_t(jb) * lda, lda, WU + jb, ldw, mm, jn, jn);
            e.store_to(A + r0 + int64_t(jb) * lda, lda, mm, jn);
        }
        // U row: A[jb:jb+jn, jb+jn:n] = L_jj^-1 * A[...]
        for (int c0 = jb + jn; c0 < n; c0 += 64) {
            const int nn = min(64, n - c0);
            Mk e;
            e.zero();
            e.run(smem, WL + jb, ldw, A + jb + int64_t(c0) * lda, lda, jn, nn, jn);
            e.store_to(A + jb + int64_t(c0) * lda, lda, jn, nn);
        }
        block_fence_sync();
    }
    return 0;
}

// ---------------------------------------------------------------------------------
// TRSM work items: kTrsmRows-row (or -column) strips of the block being solved,
// left-looking over the kNB-wide diagonal blocks of the triangular block.
// ---------------------------------------------------------------------------------

// An engine's k-loop: BlockMmaT::run, or its split-phase form (run_sp) when SP; false (after
// reporting MTD_ERR_TIMEOUT) if a wait of the latter expired.
template <bool SP, typename E, typename T>
__device__ __forceinline__ bool eng_run(const RunArgs &p, E &e, void *smem, const T *A, int64_t lda, const T *B,
                                        int64_t ldb, int M, int N, int K, bool end_sync = true) {
    if constexpr (SP) {
#if MTD_EARLY_CLAIM2
        const bool ran = e.run_sp(smem, A, lda, B, ldb, M, N, K);
#else
        const bool ran = e.run_sp(smem, A, lda, B, ldb, M, N, K, end_sync);
#endif
        if (!ran) {
            if (threadIdx.x == 0) report_error(p.ctl, MTD_ERR_TIMEOUT, 0);
            return false;
        }
    } else {
        e.run(smem, A, lda, B, ldb, M, N, K);
    }
    return true;
}
// 1: in the FP64 persistent loop, thread 0 of an update item makes one attempt to claim the
// CTA's next item before the item's last k-slice (scheduler.cuh, early_claim).
#ifndef MTD_EARLY_CLAIM2
#define MTD_EARLY_CLAIM2 0
#endif
#if MTD_EARLY_CLAIM2
static __device__ __noinline__ void early_claim(const RunArgs &p);
#endif

// 0: the update items' split-phase k-loop ends without a CTA barrier; each warp subtracts its
// accumulators from C as soon as it has read its last slice, and the persistent loop's barrier
// after the item is the first one every warp meets.  Measured on one B200 (ms, tile 1536, one
// call, base / this / base): LU N = 24000 298.2 / 296.5 / 297.8, Cholesky 152.0 / 151.5 /
// 151.9, GEMM-only N = 12288 4.83 / 4.81.
#ifndef MTD_UPDATE_END_SYNC
#define MTD_UPDATE_END_SYNC 0
#endif
// 1: FP64 update items copy their C block into shared memory during the last k-slice
// (BlockMmaT::run_sp_update) instead of reading it after the k-loop.  A traced GEMM-only run
// (N = 12288, tile 1536; probe timestamps after the k-loop and after the C update) put 8.8 us
// of a 228 us item in the C read-modify-write after the k-loop.  Measured with the kernel
// instances per operation family (ms, N = 24000, tile 1536, one call): Cholesky 152.7 ->
// 150.3 (GEMM_NT item 224.4 -> 222.0 us), GEMM-only N = 12288 4.81 -> 4.74; for the LU's
// GEMM_NN items the staged update measured slower (item 221.3 -> 223.0 us, LU 296.0 ->
// 297.5 ms), so they keep the plain C update (MTD_STAGE_C_NN=0).
#ifndef MTD_STAGE_C
#define MTD_STAGE_C 1
#endif
#ifndef MTD_STAGE_C_NN
#define MTD_STAGE_C_NN 0
#endif

// The update items' k-loop (MTD_SPLIT_PHASE) and the TRSM strips' (MTD_SPLIT_PHASE_TRSM).  The
// update items return straight to the persistent loop after their C update, which passes a CTA
// barrier before the next item touches shared memory.
template <typename E, typename T>
__device__ __forceinline__ bool gemm_run(const RunArgs &p, E &e, void *smem, const T *A, int64_t lda, const T *B,
                                         int64_t ldb, int M, int N, int K) {
#if MTD_EARLY_CLAIM2
    if constexpr (sizeof(T) == 8) {
        if (!e.run_sp(smem, A, lda, B, ldb, M, N, K, [&]() { early_claim(p); })) {
            if (threadIdx.x == 0) report_error(p.ctl, MTD_ERR_TIMEOUT, 0);
            return false;
        }
        return true;
    }
#endif
    return eng_run<MTD_SPLIT_PHASE != 0>(p, e, smem, A, lda, B, ldb, M, N, K, MTD_UPDATE_END_SYNC != 0);
}
// An update item's k-loop and C update: C -= A B (operand layouts as the engine's), lower
// triangle only when lower.  The split-phase engine stages C in shared memory during the last
// k-slice (BlockMmaT::run_sp_update); false (after reporting MTD_ERR_TIMEOUT) if a wait expired.
template <bool STAGED = true, typename E, typename T>
__device__ __forceinline__ bool update_run(const RunArgs &p, E &e, void *smem, const T *A, int64_t lda, const T *B,
                                           int64_t ldb, int M, int N, int K, T *C, int64_t ldc, bool lower) {
#if MTD_SPLIT_PHASE && !MTD_EARLY_CLAIM2 && MTD_STAGE_C
    if constexpr (STAGED) {
        if (!e.run_sp_update(smem, A, lda, B, ldb, M, N, K, C, ldc, lower)) {
            if (threadIdx.x == 0) report_error(p.ctl, MTD_ERR_TIMEOUT, 0);
            return false;
        }
        return true;
    }
#endif
    if (!gemm_run(p, e, smem, A, lda, B, ldb, M, N, K)) return false;
    e.sub_from(C, ldc, M, N, lower, 0, 0);
    return true;
}

template <typename E, typename T>
__device__ __forceinline__ bool trsm_run(const RunArgs &p, E &e, void *smem, const T *A, int64_t lda, const T *B,
                                         int64_t ldb, int M, int N, int K) {
    return eng_run<MTD_SPLIT_PHASE_TRSM != 0>(p, e, smem, A, lda, B, ldb, M, N, K);
}

// 1: the FP64 TRSM strips run each two-block step's solve products from shared memory (the
// step's 64 x 128 block and the step's three 64 x 64 operand blocks staged there once)
// instead of as three engine runs through global memory.
// Measured on one B200 (one call each; traced item medians, N = 24000, tile 1536):
// Cholesky TRSM_RLT items 842 -> 833 us, Cholesky 149.8 -> 149.0 ms.  The LU's strips
// (MTD_TRSM_FUSED_LU, off): TRSM_LLNU / TRSM_RUN items 848 / 843 -> 822 / 822 us, but its
// GEMM_NN items in the same kernel instance went 221.2 -> 223.9 us and the LU 295.4 -> 296.5 ms.
#ifndef MTD_TRSM_FUSED
#define MTD_TRSM_FUSED 1
#endif
#ifndef MTD_TRSM_FUSED_LU
#define MTD_TRSM_FUSED_LU 0
#endif
// 1: the fused strips are separate (not inlined) functions with their own register
// allocation, apart from the update items' paths.
#ifndef MTD_TRSM_FUSED_NOINLINE
#define MTD_TRSM_FUSED_NOINLINE 0
#endif
#if MTD_TRSM_FUSED_NOINLINE
#define MTD_TRSM_FUSED_LINKAGE static __device__ __noinline__
#else
#define MTD_TRSM_FUSED_LINKAGE __device__
#endif

// Leading dimension of the fused TRSM steps' shared-memory blocks: the 64 x 64 engine's padded
// rows, so its compute_stage reads them as staged slices.
constexpr int kStepLd = 64 + SmemPad<double>::a;

// dst[k * kStepLd + n] = src[n + k * lds] for n < rows, k < cols, zero elsewhere in 64 x 64
// (16-byte cp.async copies; rows even, src columns 16-byte aligned).  Completes at the
// caller's cp_async_wait.
__device__ __forceinline__ void stage_block64(double *dst, const double *src, int64_t lds, int rows, int cols) {
    static_assert((64 * 32) % kThreads == 0, "whole passes of the CTA");
#pragma unroll
    for (int u = 0; u < 64 * 32 / kThreads; ++u) {
        const int pc = threadIdx.x + u * kThreads;
        const int k = pc / 32, n = 2 * (pc % 32);
        const bool ok = k < cols && n < rows;
        cp_async16(dst + k * kStepLd + n, ok ? src + n + int64_t(k) * lds : src, ok);
    }
}

// X = X * L^-T for one 64-row strip, FP64 with 16-byte operands (op_trsm_rlt below): per step
// of two inverse blocks (jb .. jb + 128), the wide update from global memory, then
//   Y  = X(:, jb .. jb + 128) - update          (shared memory, SY)
//   X1 = Y1 W1^T;  Y2 -= X1 L21^T;  X2 = Y2 W2^T  (64 x 64 products from shared memory)
// with W1, L21, W2 staged by cp.async while Y is formed; X1 and X2 go to global memory.  The
// same products in the same order as the engine-run steps, so the same results.
template <int VEC>
MTD_TRSM_FUSED_LINKAGE int trsm_rlt_fused(const RunArgs &p, const MatCtx &m, const DevTask &t, int item, void *smem) {
    using Mw = WideMma<kBNContig, VEC>;
    using Ms = PanelMma<kBNContig, VEC>;
    const int r0 = item * kTrsmRows;
    const int mm = min(kTrsmRows, t.m - r0);
    const int nk = t.n;
    const int64_t lda = m.lda, ldw = m.wsld;
    double *X = at<double>(m, t.cr + r0, t.cc);
    const double *L = at<double>(m, t.ar, t.ac);
    const double *W = ws_lo<double>(m) + t.ar;
    double *SY = static_cast<double *>(smem);  // 128 columns
    double *SW1 = SY + 128 * kStepLd;
    double *SL21 = SW1 + 64 * kStepLd;
    double *SW2 = SL21 + 64 * kStepLd;
    for (int jb = 0; jb < nk; jb += 2 * kNB) {
        const int jw = min(2 * kNB, nk - jb);
        const int j1 = min(kNB, jw), j2 = jw - j1;
        {
            Mw e;
            e.zero();
            // X(:, jb .. jb + jw) -= X(:, 0 .. jb) L(jb .. jb + jw, 0 .. jb)^T; the run ends at a
            // CTA barrier, so its ring is free below
            if (jb > 0 && !trsm_run(p, e, smem, X, lda, L + jb, lda, mm, jw, jb)) return MTD_ERR_TIMEOUT;
            stage_block64(SW1, W + jb, ldw, j1, j1);
            if (j2 > 0) {
                stage_block64(SL21, L + (jb + kNB) + int64_t(jb) * lda, lda, j2, j1);
                stage_block64(SW2, W + jb + kNB, ldw, j2, j2);
            }
            cp_async_commit();
            e.sub_to_smem(X + int64_t(jb) * lda, lda, mm, jw, SY, [](int r, int c) { return r + c * kStepLd; });
        }
        cp_async_wait<0>();
        __syncthreads();
        {  // X1 = Y1 W1^T
            Ms e;
            e.zero();
            e.compute_stage(SY, SW1);
            e.compute_stage(SY + 32 * kStepLd, SW1 + 32 * kStepLd);
            __syncthreads();  // every warp has read Y1
            e.for_each(kNB, kNB, [&](int r, int c, double v) {
                SY[r + c * kStepLd] = v;
                if (r < mm && c < j1) X[r + int64_t(jb + c) * lda] = v;
            });
        }
        __syncthreads();
        if (j2 > 0) {
            {  // Y2 -= X1 L21^T (each thread updates its own elements of SY's second half)
                Ms e;
                e.zero();
                e.compute_stage(SY, SL21);
                e.compute_stage(SY + 32 * kStepLd, SL21 + 32 * kStepLd);
                e.for_each(kNB, kNB, [&](int r, int c, double v) { SY[r + (kNB + c) * kStepLd] -= v; });
            }
            __syncthreads();
            {  // X2 = Y2 W2^T
                Ms e;
                e.zero();
                e.compute_stage(SY + kNB * kStepLd, SW2);
                e.compute_stage(SY + (kNB + 32) * kStepLd, SW2 + 32 * kStepLd);
                e.for_each(kNB, kNB, [&](int r, int c, double v) {
                    if (r < mm && c < j2) X[r + int64_t(jb + kNB + c) * lda] = v;
                });
            }
        }
        block_fence_sync();
    }
    return 0;
}

// A k-contiguous 64 x 64 operand block as the 64 x 64 engine stages it: two 32-deep slices of
// kStepSliceB elements, dst[s * kStepSliceB + n * kStepLdK + kk] = src[(32 s + kk) + n * lds]
// for k = 32 s + kk < krows, n < cols, zero elsewhere (16-byte cp.async copies; krows even,
// src columns 16-byte aligned).  Completes at the caller's cp_async_wait.
constexpr int kStepLdK = 32 + SmemPad<double>::bk;
constexpr int kStepSliceB = 64 * kStepLdK;
__device__ __forceinline__ void stage_block64_k(double *dst, const double *src, int64_t lds, int krows, int cols) {
    static_assert((64 * 32) % kThreads == 0, "whole passes of the CTA");
#pragma unroll
    for (int u = 0; u < 64 * 32 / kThreads; ++u) {
        const int pc = threadIdx.x + u * kThreads;
        const int n = pc / 32, k = 2 * (pc % 32);  // k in 0 .. 63
        const bool ok = n < cols && k < krows;
        cp_async16(dst + (k / 32) * kStepSliceB + n * kStepLdK + (k % 32), ok ? src + k + int64_t(n) * lds : src, ok);
    }
}

// X = X * U^-1 for one 64-row strip, FP64 with 16-byte operands (op_trsm_run below): the fused
// steps of trsm_rlt_fused with U's blocks (k-contiguous B operands): X1 = Y1 W1,
// Y2 -= X1 U12, X2 = Y2 W2 (W = the inverses of U's diagonal blocks).
template <int VEC>
MTD_TRSM_FUSED_LINKAGE int trsm_run_fused(const RunArgs &p, const MatCtx &m, const DevTask &t, int item, void *smem) {
    using Mw = WideMma<kBKContig, VEC>;
    using Ms = PanelMma<kBKContig, VEC>;
    static_assert(Ms::LDB == kStepLdK && Ms::B_STAGE == kStepSliceB && Ms::LDA == kStepLd, "staged layouts");
    const int r0 = item * kTrsmRows;
    const int mm = min(kTrsmRows, t.m - r0);
    const int nk = t.n;
    const int64_t lda = m.lda, ldw = m.wsld;
    double *X = at<double>(m, t.cr + r0, t.cc);
    const double *U = at<double>(m, t.ar, t.ac);
    const double *W = ws_up<double>(m) + t.ar;
    double *SY = static_cast<double *>(smem);  // 128 columns
    double *SW1 = SY + 2 * kNB * kStepLd;
    double *SU12 = SW1 + 2 * kStepSliceB;
    double *SW2 = SU12 + 2 * kStepSliceB;
    for (int jb = 0; jb < nk; jb += 2 * kNB) {
        const int jw = min(2 * kNB, nk - jb);
        const int j1 = min(kNB, jw), j2 = jw - j1;
        {
            Mw e;
            e.zero();
            // X(:, jb .. jb + jw) -= X(:, 0 .. jb) U(0 .. jb, jb .. jb + jw)
            if (jb > 0 && !trsm_run(p, e, smem, X, lda, U + int64_t(jb) * lda, lda, mm, jw, jb)) return MTD_ERR_TIMEOUT;
            stage_block64_k(SW1, W + jb, ldw, j1, j1);
            if (j2 > 0) {
                stage_block64_k(SU12, U + jb + int64_t(jb + kNB) * lda, lda, j1, j2);
                stage_block64_k(SW2, W + jb + kNB, ldw, j2, j2);
            }
            cp_async_commit();
            e.sub_to_smem(X + int64_t(jb) * lda, lda, mm, jw, SY, [](int r, int c) { return r + c * kStepLd; });
        }
        cp_async_wait<0>();
        __syncthreads();
        {  // X1 = Y1 W1
            Ms e;
            e.zero();
            e.compute_stage(SY, SW1);
            e.compute_stage(SY + 32 * kStepLd, SW1 + kStepSliceB);
            __syncthreads();  // every warp has read Y1
            e.for_each(kNB, kNB, [&](int r, int c, double v) {
                SY[r + c * kStepLd] = v;
                if (r < mm && c < j1) X[r + int64_t(jb + c) * lda] = v;
            });
        }
        __syncthreads();
        if (j2 > 0) {
            {  // Y2 -= X1 U12
                Ms e;
                e.zero();
                e.compute_stage(SY, SU12);
                e.compute_stage(SY + 32 * kStepLd, SU12 + kStepSliceB);
                e.for_each(kNB, kNB, [&](int r, int c, double v) { SY[r + (kNB + c) * kStepLd] -= v; });
            }
            __syncthreads();
            {  // X2 = Y2 W2
                Ms e;
                e.zero();
                e.compute_stage(SY + kNB * kStepLd, SW2);
                e.compute_stage(SY + (kNB + 32) * kStepLd, SW2 + kStepSliceB);
                e.for_each(kNB, kNB, [&](int r, int c, double v) {
                    if (r < mm && c < j2) X[r + int64_t(jb + kNB + c) * lda] = v;
                });
            }
        }
        block_fence_sync();
    }
    return 0;
}

// X = L^-1 X, unit diagonal, for one 64-column strip, FP64 with 16-byte operands
// (op_trsm_llnu below): per step of two inverse blocks (rows jb .. jb + 128), the tall update
// from global memory, then Y = X(jb .. jb + 128, :) - update in shared memory as the 64 x 64
// engine's k-contiguous B slices (four 32-row slices), X1 = W1 Y1, Y2 -= L21 X1, X2 = W2 Y2
// with W1, L21, W2 staged as m-contiguous A blocks.
template <int VEC>
MTD_TRSM_FUSED_LINKAGE int trsm_llnu_fused(const RunArgs &p, const MatCtx &m, const DevTask &t, int item, void *smem) {
    using Mt = TallMma<VEC>;
    using Ms = PanelMma<kBKContig, VEC>;
    static_assert(Ms::LDB == kStepLdK && Ms::B_STAGE == kStepSliceB && Ms::LDA == kStepLd, "staged layouts");
    const int c0 = item * kTrsmRows;
    const int nc = min(kTrsmRows, t.n - c0);
    const int nk = t.m;
    const int64_t lda = m.lda, ldw = m.wsld;
    double *X = at<double>(m, t.cr, t.cc + c0);
    const double *L = at<double>(m, t.ar, t.ac);
    const double *W = ws_lo<double>(m) + t.ar;
    double *SY = static_cast<double *>(smem);  // 128 rows: four slices
    double *SW1 = SY + 4 * kStepSliceB;
    double *SL21 = SW1 + kNB * kStepLd;
    double *SW2 = SL21 + kNB * kStepLd;
    for (int jb = 0; jb < nk; jb += 2 * kNB) {
        const int jw = min(2 * kNB, nk - jb);
        const int j1 = min(kNB, jw), j2 = jw - j1;
        {
            Mt e;
            e.zero();
            // X(jb .. jb + jw, :) -= L(jb .. jb + jw, 0 .. jb) X(0 .. jb, :)
            if (jb > 0 && !trsm_run(p, e, smem, L + jb, lda, X, lda, jw, nc, jb)) return MTD_ERR_TIMEOUT;
            stage_block64(SW1, W + jb, ldw, j1, j1);
            if (j2 > 0) {
                stage_block64(SL21, L + (jb + kNB) + int64_t(jb) * lda, lda, j2, j1);
                stage_block64(SW2, W + jb + kNB, ldw, j2, j2);
            }
            cp_async_commit();
            e.sub_to_smem(X + jb, lda, jw, nc, SY,
                          [](int r, int c) { return (r / 32) * kStepSliceB + c * kStepLdK + (r % 32); });
        }
        cp_async_wait<0>();
        __syncthreads();
        {  // X1 = W1 Y1
            Ms e;
            e.zero();
            e.compute_stage(SW1, SY);
            e.compute_stage(SW1 + 32 * kStepLd, SY + kStepSliceB);
            __syncthreads();  // every warp has read Y1
            e.for_each(kNB, kNB, [&](int r, int c, double v) {
                SY[(r / 32) * kStepSliceB + c * kStepLdK + (r % 32)] = v;
                if (r < j1 && c < nc) X[jb + r + int64_t(c) * lda] = v;
            });
        }
        __syncthreads();
        if (j2 > 0) {
            {  // Y2 -= L21 X1
                Ms e;
                e.zero();
                e.compute_stage(SL21, SY);
                e.compute_stage(SL21 + 32 * kStepLd, SY + kStepSliceB);
                e.for_each(kNB, kNB, [&](int r, int c, double v) {
                    SY[(2 + r / 32) * kStepSliceB + c * kStepLdK + (r % 32)] -= v;
                });
            }
            __syncthreads();
            {  // X2 = W2 Y2
                Ms e;
                e.zero();
                e.compute_stage(SW2, SY + 2 * kStepSliceB);
                e.compute_stage(SW2 + 32 * kStepLd, SY + 3 * kStepSliceB);
                e.for_each(kNB, kNB, [&](int r, int c, double v) {
                    if (r < j2 && c < nc) X[jb + kNB + r + int64_t(c) * lda] = v;
                });
            }
        }
        block_fence_sync();
    }
    return 0;
}

// X = X * L^-T   (cublasDtrsm R, L, T, NonUnit; cholesky_mustard.cu:281)
template <typename T, int VEC, int SPLIT = 1>
MTD_PANEL_OP_LINKAGE int op_trsm_rlt(const RunArgs &p, const MatCtx &m, const DevTask &t, int item, void *smem) {
#if MTD_TRSM_FUSED && MTD_TRSM_WIDE
    if constexpr (sizeof(T) == 8 && VEC == 2 && kTrsmRows == 64 && kNB == 64)
        return trsm_rlt_fused<VEC>(p, m, t, item, smem);
#endif
    using Mn = StripStep<kBNContig, VEC, T, SPLIT>;
    const int r0 = item * kTrsmRows;
    const int mm = min(kTrsmRows, t.m - r0);
    const int nk = t.n;
    const int64_t lda = m.lda, ldw = m.wsld;
    T *X = at<T>(m, t.cr + r0, t.cc);
    const T *L = at<T>(m, t.ar, t.ac);
    const T *W = ws_lo<T>(m) + t.ar;
    // X(:, jb .. jb + jn) = X(:, jb .. jb + jn) W_jb^T (W_jb: the inverse of that diagonal block)
    auto solve_block = [&](int jb, int jn) {
        Mn e;
        e.zero();
        if (!trsm_run(p, e, smem, X + int64_t(jb) * lda, lda, W + jb, ldw, mm, jn, jn)) return false;
        e.store_rounded_to(X + int64_t(jb) * lda, lda, mm, jn);  // panel of L: an operand of the updates
        if constexpr (sizeof(T) == 4)
            if (p.bf16)  // BF16-update runs: the updates read the panel from its BF16 copy
                e.store_bf16_to(static_cast<__nv_bfloat16 *>(p.bf16) + (t.cr + r0) + int64_t(t.cc + jb) * p.bf16_ld,
                                p.bf16_ld, mm, jn);
        if constexpr (sizeof(T) == 4 && SPLIT == 3)
            if (p.lo)  // FP32-accurate runs: the three-pass updates read the panel's low part
                e.store_lo_to(static_cast<float *>(p.lo) + (t.cr + r0) + int64_t(t.cc + jb) * p.lo_ld, p.lo_ld, mm, jn);
        block_fence_sync();
        return true;
    };
#if MTD_TRSM_WIDE
    using Mw = StripUpdate<kBNContig, VEC, T, SPLIT>;
    for (int jb = 0; jb < nk; jb += 2 * kNB) {
        const int jw = min(2 * kNB, nk - jb);
        if (jb > 0) {  // X(:, jb .. jb + jw) -= X(:, 0 .. jb) L(jb .. jb + jw, 0 .. jb)^T
            Mw e;
            e.zero();
            if (!trsm_run(p, e, smem, X, lda, L + jb, lda, mm, jw, jb)) return MTD_ERR_TIMEOUT;
            e.sub_from(X + int64_t(jb) * lda, lda, mm, jw);
            block_fence_sync();
        }
        if (!solve_block(jb, min(kNB, jw))) return MTD_ERR_TIMEOUT;
        if (jw > kNB) {  // the second block's update by the first, then its solve
            Mn e;
            e.zero();
            if (!trsm_run(p, e, smem, X + int64_t(jb) * lda, lda, L + (jb + kNB) + int64_t(jb) * lda, lda, mm,
                          jw - kNB, kNB))
                return MTD_ERR_TIMEOUT;
            e.sub_from(X + int64_t(jb + kNB) * lda, lda, mm, jw - kNB);
            block_fence_sync();
            if (!solve_block(jb + kNB, jw - kNB)) return MTD_ERR_TIMEOUT;
        }
    }
#else
    for (int jb = 0; jb < nk; jb += kNB) {
        const int jn = min(kNB, nk - jb);
        if (jb > 0) {
            Mn e;
            e.zero();
            if (!trsm_run(p, e, smem, X, lda, L + jb, lda, mm, jn, jb)) return MTD_ERR_TIMEOUT;
            e.sub_from(X + int64_t(jb) * lda, lda, mm, jn);
            block_fence_sync();
        }
        if (!solve_block(jb, jn)) return MTD_ERR_TIMEOUT;
    }
#endif
    return 0;
}

// X = X * U^-1   (cublasDtrsm R, U, N, NonUnit; lu_mustard.cu:459)
template <int VEC>
MTD_PANEL_OP_LINKAGE int op_trsm_run(const RunArgs &p, const MatCtx &m, const DevTask &t, int item, void *smem) {
#if MTD_TRSM_FUSED_LU && MTD_TRSM_WIDE
    if constexpr (VEC == 2 && kTrsmRows == 64 && kNB == 64) return trsm_run_fused<VEC>(p, m, t, item, smem);
#endif
    using Mk = StripStep<kBKContig, VEC>;
    const int r0 = item * kTrsmRows;
    const int mm = min(kTrsmRows, t.m - r0);
    const int nk = t.n;
    const int64_t lda = m.lda, ldw = m.wsld;
    double *X = at<double>(m, t.cr + r0, t.cc);
    const double *U = at<double>(m, t.ar, t.ac);
    const double *W = ws_up<double>(m) + t.ar;
    auto solve_block = [&](int jb, int jn) {
        Mk e;
        e.zero();
        if (!trsm_run(p, e, smem, X + int64_t(jb) * lda, lda, W + jb, ldw, mm, jn, jn)) return false;
        e.store_to(X + int64_t(jb) * lda, lda, mm, jn);
        block_fence_sync();
        return true;
    };
#if MTD_TRSM_WIDE
    using Mw = StripUpdate<kBKContig, VEC>;
    for (int jb = 0; jb < nk; jb += 2 * kNB) {
        const int jw = min(2 * kNB, nk - jb);
        if (jb > 0) {  // X(:, jb .. jb + jw) -= X(:, 0 .. jb) U(0 .. jb, jb .. jb + jw)
            Mw e;
            e.zero();
            if (!trsm_run(p, e, smem, X, lda, U + int64_t(jb) * lda, lda, mm, jw, jb)) return MTD_ERR_TIMEOUT;
            e.sub_from(X + int64_t(jb) * lda, lda, mm, jw);
            block_fence_sync();
        }
        if (!solve_block(jb, min(kNB, jw))) return MTD_ERR_TIMEOUT;
        if (jw > kNB) {
            Mk e;
            e.zero();
            if (!trsm_run(p, e, smem, X + int64_t(jb) * lda, lda, U + jb + int64_t(jb + kNB) * lda, lda, mm,
                          jw - kNB, kNB))
                return MTD_ERR_TIMEOUT;
            e.sub_from(X + int64_t(jb + kNB) * lda, lda, mm, jw - kNB);
            block_fence_sync();
            if (!solve_block(jb + kNB, jw - kNB)) return MTD_ERR_TIMEOUT;
        }
    }
#else
    for (int jb = 0; jb < nk; jb += kNB) {
        const int jn = min(kNB, nk - jb);
        if (jb > 0) {
            Mk e;
            e.zero();
            if (!trsm_run(p, e, smem, X, lda, U + int64_t(jb) * lda, lda, mm, jn, jb)) return MTD_ERR_TIMEOUT;
            e.sub_from(X + int64_t(jb) * lda, lda, mm, jn);
            block_fence_sync();
        }
        if (!solve_block(jb, jn)) return MTD_ERR_TIMEOUT;
    }
#endif
    return 0;
}

// X = L^-1 * X, unit diagonal   (cublasDtrsm L, L, N, Unit; lu_mustard.cu:413)
template <int VEC>
MTD_PANEL_OP_LINKAGE int op_trsm_llnu(const RunArgs &p, const MatCtx &m, const DevTask &t, int item, void *smem) {
#if MTD_TRSM_FUSED_LU && MTD_TRSM_WIDE
    if constexpr (VEC == 2 && kTrsmRows == 64 && kNB == 64) return trsm_llnu_fused<VEC>(p, m, t, item, smem);
#endif
    using Mk = ColStripStep<VEC>;
    const int c0 = item * kTrsmRows;
    const int nc = min(kTrsmRows, t.n - c0);
    const int nk = t.m;
    const int64_t lda = m.lda, ldw = m.wsld;
    double *X = at<double>(m, t.cr, t.cc + c0);
    const double *L = at<double>(m, t.ar, t.ac);
    const double *W = ws_lo<double>(m) + t.ar;
    auto solve_block = [&](int jb, int jn) {
        Mk e;
        e.zero();
        if (!trsm_run(p, e, smem, W + jb, ldw, X + jb, lda, jn, nc, jn)) return false;
        e.store_to(X + jb, lda, jn, nc);
        block_fence_sync();
        return true;
    };
#if MTD_TRSM_WIDE
    using Mt = ColStripUpdate<VEC>;
    for (int jb = 0; jb < nk; jb += 2 * kNB) {
        const int jw = min(2 * kNB, nk - jb);
        if (jb > 0) {  // X(jb .. jb + jw, :) -= L(jb .. jb + jw, 0 .. jb) X(0 .. jb, :)
            Mt e;
            e.zero();
            if (!trsm_run(p, e, smem, L + jb, lda, X, lda, jw, nc, jb)) return MTD_ERR_TIMEOUT;
            e.sub_from(X + jb, lda, jw, nc);
            block_fence_sync();
        }
        if (!solve_block(jb, min(kNB, jw))) return MTD_ERR_TIMEOUT;
        if (jw > kNB) {
            Mk e;
            e.zero();
            if (!trsm_run(p, e, smem, L + (jb + kNB) + int64_t(jb) * lda, lda, X + jb, lda, jw - kNB, nc, kNB))
                return MTD_ERR_TIMEOUT;
            e.sub_from(X + jb + kNB, lda, jw - kNB, nc);
            block_fence_sync();
            if (!solve_block(jb + kNB, jw - kNB)) return MTD_ERR_TIMEOUT;
        }
    }
#else
    for (int jb = 0; jb < nk; jb += kNB) {
        const int jn = min(kNB, nk - jb);
        if (jb > 0) {
            Mk e;
            e.zero();
            if (!trsm_run(p, e, smem, L + jb, lda, X, lda, jn, nc, jb)) return MTD_ERR_TIMEOUT;
            e.sub_from(X + jb, lda, jn, nc);
            block_fence_sync();
        }
        if (!solve_block(jb, jn)) return MTD_ERR_TIMEOUT;
    }
#endif
    return 0;
}

// ---------------------------------------------------------------------------------
// Update work items: one kGemmTile x kGemmTile output block each.
// ---------------------------------------------------------------------------------

// FP64 update items whose operands come by TMA (tma64.cuh): the run carries the tensor maps
// (single-matrix FP64 runs of suitable geometry), the depth is whole k-slices and both
// operand blocks start on 16-row atoms.
__device__ __forceinline__ bool tma64_ok(const RunArgs &p, const t64::State *s64, int k, int a_row, int b_row) {
    return s64 != nullptr && p.tma64 != 0 && p.mats == nullptr && k % t64::kBK == 0 && (a_row & 15) == 0 &&
           (b_row & 15) == 0;
}

#ifndef MTD_T64_NOINLINE
#define MTD_T64_NOINLINE 1
#endif
#if MTD_T64_NOINLINE
#define MTD_T64_INLINE __noinline__
#else
#define MTD_T64_INLINE __forceinline__
#endif
template <int BL>
__device__ MTD_T64_INLINE int update_tma64(const RunArgs &p, t64::State *s64, void *smem, const t64::Coords &c, double *C,
                                         int64_t ldc,
                            int mm, int nn, bool lower) {
    t64::Engine<BL> e;
    e.zero();
    uint8_t *ring = reinterpret_cast<uint8_t *>((reinterpret_cast<uintptr_t>(smem) + 1023) & ~uintptr_t(1023));
    // the tensor maps' addresses are taken on the kernel parameter itself
    if (!e.run(s64, ring, p.tmap64_mn, p.tmap64_k, c, p.timeout_ns)) {
        if (threadIdx.x == 0) report_error(p.ctl, MTD_ERR_TIMEOUT, 0);
        return MTD_ERR_TIMEOUT;
    }
    e.sub_from(C, ldc, mm, nn, lower);
    return 0;
}

// C -= A B^T   (cublasGemmEx N, T; cholesky_mustard.cu:376)
template <typename T, int VEC, int SPLIT = 1>
__device__ int op_gemm_nt(const RunArgs &p, const MatCtx &m, const DevTask &t, int item, void *smem,
                          t64::State *s64 = nullptr) {
    using Mg = GemmMma<kBNContig, VEC, T, SPLIT>;
    const int nbn = (t.n + kGemmTile - 1) / kGemmTile;
    const int r0 = (item / nbn) * kGemmTile, c0 = (item % nbn) * kGemmTile;
    const int mm = min(kGemmTile, t.m - r0), nn = min(kGemmTile, t.n - c0);
    if constexpr (sizeof(T) == 8 && VEC == 2)
        if (tma64_ok(p, s64, t.k, t.ar + r0, t.br + c0))
            return update_tma64<kBNContig>(p, s64, smem, t64::Coords{t.ar + r0, t.ac, t.br + c0, t.bc, t.k},
                                           at<double>(m, t.cr + r0, t.cc + c0), m.lda, mm, nn, false);
    Mg e;
    e.zero();
    if (!update_run(p, e, smem, at<T>(m, t.ar + r0, t.ac), m.lda, at<T>(m, t.br + c0, t.bc), m.lda, mm, nn, t.k,
                    at<T>(m, t.cr + r0, t.cc + c0), m.lda, false))
        return MTD_ERR_TIMEOUT;
    return 0;
}

// C -= A B   (cublasGemmEx N, N; lu_mustard.cu:511)
template <int VEC>
__device__ int op_gemm_nn(const RunArgs &p, const MatCtx &m, const DevTask &t, int item, void *smem,
                          t64::State *s64 = nullptr) {
    using Mg = GemmMma<kBKContig, VEC>;
    const int nbn = (t.n + kGemmTile - 1) / kGemmTile;
    const int r0 = (item / nbn) * kGemmTile, c0 = (item % nbn) * kGemmTile;
    const int mm = min(kGemmTile, t.m - r0), nn = min(kGemmTile, t.n - c0);
    if constexpr (VEC == 2)
        if (tma64_ok(p, s64, t.k, t.ar + r0, t.br))  // B: k range from row br, columns bc + c0 ..
            return update_tma64<kBKContig>(p, s64, smem, t64::Coords{t.ar + r0, t.ac, t.br, t.bc + c0, t.k},
                                           at<double>(m, t.cr + r0, t.cc + c0), m.lda, mm, nn, false);
    Mg e;
    e.zero();
    if (!update_run<MTD_STAGE_C_NN != 0>(p, e, smem, at<double>(m, t.ar + r0, t.ac), m.lda,
                                         at<double>(m, t.br, t.bc + c0), m.lda, mm, nn, t.k,
                                         at<double>(m, t.cr + r0, t.cc + c0), m.lda, false))
        return MTD_ERR_TIMEOUT;
    return 0;
}

// C -= A A^T, lower triangle only   (cublasDsyrk L, N; cholesky_mustard.cu:327)
template <typename T, int VEC, int SPLIT = 1>
__device__ int op_syrk_ln(const RunArgs &p, const MatCtx &m, const DevTask &t, int item, void *smem,
                          t64::State *s64 = nullptr) {
    using Mg = GemmMma<kBNContig, VEC, T, SPLIT>;
    int pb = 0;
    while ((pb + 1) * (pb + 2) / 2 <= item) ++pb;
    const int qb = item - pb * (pb + 1) / 2;
    const int r0 = pb * kGemmTile, c0 = qb * kGemmTile;
    const int mm = min(kGemmTile, t.m - r0), nn = min(kGemmTile, t.m - c0);
    if constexpr (sizeof(T) == 8 && VEC == 2)
        if (tma64_ok(p, s64, t.k, t.ar + r0, t.ar + c0))
            return update_tma64<kBNContig>(p, s64, smem, t64::Coords{t.ar + r0, t.ac, t.ar + c0, t.ac, t.k},
                                           at<double>(m, t.cr + r0, t.cc + c0), m.lda, mm, nn, pb == qb);
    Mg e;
    e.zero();
    if (!update_run(p, e, smem, at<T>(m, t.ar + r0, t.ac), m.lda, at<T>(m, t.ar + c0, t.ac), m.lda, mm, nn, t.k,
                    at<T>(m, t.cr + r0, t.cc + c0), m.lda, pb == qb))
        return MTD_ERR_TIMEOUT;
    return 0;
}

// Shared memory (bytes) the largest operation needs.
constexpr int kOpSmemBytes() {
    constexpr int g1 = GemmMma<kBNContig, 2>::SMEM_BYTES;
    constexpr int g2 = GemmMma<kBKContig, 2>::SMEM_BYTES;
    // C -= A^T B of the Cholesky adjoint: both operands staged k-contiguous
    constexpr int g3 = BlockMmaT<double, kGemmTile, kGemmTile, kGemmWarpsM, kGemmWarpsN, kBKContig, 2, MTD_GEMM_STAGES,
                                 MTD_GEMM_BK, 1, kAKContig>::SMEM_BYTES;
    constexpr int diag = 5 * kNB * kDiagLd * 8;  // the adjoint's diagonal block: five 64 x 64 blocks
    constexpr int chol = chol_small_smem_bytes<double>();
    constexpr int pn = PanelMma<kBNContig, 2>::SMEM_BYTES > PanelMma<kBKContig, 2>::SMEM_BYTES
                           ? PanelMma<kBNContig, 2>::SMEM_BYTES
                           : PanelMma<kBKContig, 2>::SMEM_BYTES;
    static_assert(pn <= 227 * 1024, "panel engine stages fit shared memory");
#if MTD_TRSM_WIDE
    constexpr int w1 = WideMma<kBNContig, 2>::SMEM_BYTES > WideMma<kBKContig, 2>::SMEM_BYTES
                           ? WideMma<kBNContig, 2>::SMEM_BYTES
                           : WideMma<kBKContig, 2>::SMEM_BYTES;
    constexpr int w2 = w1 > TallMma<2>::SMEM_BYTES ? w1 : TallMma<2>::SMEM_BYTES;
    constexpr int w = w2 > TallMma<2, kBNContig>::SMEM_BYTES ? w2 : TallMma<2, kBNContig>::SMEM_BYTES;
    static_assert(w <= 227 * 1024, "wide TRSM engine stages fit shared memory");
#else
    constexpr int w = 0;
#endif
    constexpr int m12 = (g1 > g2 ? g1 : g2) > pn ? (g1 > g2 ? g1 : g2) : pn;
    constexpr int m3 = m12 > g3 ? m12 : g3;
    constexpr int m = m3 > w ? m3 : w;
    constexpr int d = diag > chol ? diag : chol;
    static_assert(t64::kSmemBytes <= (m > d ? m : d), "the FP64 TMA ring fits the engines' shared memory");
    return m > d ? m : d;
}
static_assert((2 * kNB + 3 * kNB) * kStepLd * int(sizeof(double)) <= kOpSmemBytes() &&
                  (2 * kNB * kStepLd + 6 * kStepSliceB) * int(sizeof(double)) <= kOpSmemBytes() &&
                  (4 * kStepSliceB + 3 * kNB * kStepLd) * int(sizeof(double)) <= kOpSmemBytes(),
              "a fused TRSM step's blocks fit the operations' shared memory");

}  // namespace mtd
