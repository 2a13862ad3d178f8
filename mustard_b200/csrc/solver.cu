// Mixed-precision SPD solver: low-precision tiled Cholesky + FP64 iterative refinement.
//
// No counterpart in the reference (it factors in FP64 only).  The factor runs on the same
// task graph and persistent scheduler as the FP64 path, in FP32 storage with TF32
// tensor-core products (MTD_PREC_TF32); accuracy is won back in FP64:
//   IR        x <- x + M^-1 (b - A x), M = L L^T the low-precision factor
//   GMRES-IR  each correction solves A d = r with GMRES in FP64 on the left-preconditioned
//             system M^-1 A d = M^-1 r (Carson & Higham, SIAM J. Sci. Comput. 39 (2017)
//             and 40 (2018)), which converges for condition numbers where plain IR does not
// The residual r = b - A x and the solution update are FP64 (A's lower triangle, read as
// a symmetric matrix).  Triangular solves with the factor are sync-free wavefront kernels
// over 64-row blocks that reuse the inverse diagonal blocks the factorisation left in its
// workspace, so each block step is a small matrix product.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <new>
#include <vector>

#include "../../include/mustard_b200.h"
#include "device_types.hpp"

namespace mtd {
void *graph_ws_lower(mtd_graph *g);
int64_t graph_ws_ld(mtd_graph *g);
}  // namespace mtd

namespace {

constexpr int kSB = 64;       // block edge of the triangular solves (= inverse block edge)
constexpr int kMaxRhs = 16;   // right-hand sides per solve call
constexpr int kSolveThreads = 256;

__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// ---- conversions and small reductions --------------------------------------------

// Lower triangle of A (+ shift on the diagonal) into B of element type T.
template <typename T>
__global__ void copy_lower_kernel(const double *A, int64_t lda, T *B, int64_t ldb, int64_t n, double shift) {
    const int64_t total = n * n;
    for (int64_t e = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; e < total; e += int64_t(gridDim.x) * blockDim.x) {
        const int64_t i = e % n, j = e / n;
        if (i < j) continue;
        double v = A[i + j * lda];
        if (i == j) v += shift;
        B[i + j * ldb] = static_cast<T>(v);
    }
}

__global__ void fill_kernel(double *x, int64_t n, double v) {
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
        x[i] = v;
}

// out[c] = max_i |X(i, c)| (as ordered bits of a non-negative double), c < nrhs.
__global__ void colmax_kernel(const double *X, int64_t ldx, int64_t n, int nrhs, unsigned long long *out) {
    const int c = blockIdx.y;
    double m = 0.0;
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
        m = fmax(m, fabs(X[i + c * ldx]));
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) atomicMax(out + c, static_cast<unsigned long long>(__double_as_longlong(m)));
}

// Y(:, c) = X(:, c) * s (+ Y when accumulate); s = scale[c] or 1 / scale[c].
template <typename TI, typename TO>
__global__ void scale_copy_kernel(const TI *X, int64_t ldx, TO *Y, int64_t ldy, int64_t n, int nrhs,
                                  const unsigned long long *scale, bool invert, bool accumulate) {
    const int c = blockIdx.y;
    double s = scale ? __longlong_as_double(static_cast<long long>(scale[c])) : 1.0;
    if (s == 0.0) s = 1.0;
    if (invert) s = 1.0 / s;
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
        const double v = static_cast<double>(X[i + c * ldx]) * s;
        if (accumulate) Y[i + c * ldy] = static_cast<TO>(static_cast<double>(Y[i + c * ldy]) + v);
        else Y[i + c * ldy] = static_cast<TO>(v);
    }
}

// ---- asynchronous element copies into shared memory --------------------------------

constexpr int kTS = kSB + 1;  // shared-memory stride of a staged 64 x 64 block (odd: no bank conflicts)

template <typename T>
__device__ __forceinline__ void cp_async_elem(T *dst, const T *src, bool valid) {
    const unsigned d = static_cast<unsigned>(__cvta_generic_to_shared(dst));
    const int bytes = valid ? int(sizeof(T)) : 0;  // 0 source bytes: the destination is zero-filled
    if constexpr (sizeof(T) == 8)
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(d), "l"(src), "r"(bytes) : "memory");
    else
        asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(d), "l"(src), "r"(bytes) : "memory");
}
// 16-byte asynchronous copy that reads only `bytes` (0..16) of the source and zero-fills
// the rest of the destination.
__device__ __forceinline__ void cp_async16_part(void *dst, const void *src, int bytes) {
    const unsigned d = static_cast<unsigned>(__cvta_generic_to_shared(dst));
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(d), "l"(src), "r"(bytes) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// ---- FP64 symmetric block product: Y += alpha * A_sym * X (A lower triangle) ------

// (I, J), I >= J, of the b-th 64 x 64 block of the lower triangle in row-major order.
__device__ __forceinline__ void lower_block_coords(int64_t b, int64_t &I, int64_t &J) {
    I = static_cast<int64_t>((sqrt(8.0 * double(b) + 1.0) - 1.0) / 2.0);
    while (I * (I + 1) / 2 > b) --I;
    while ((I + 1) * (I + 2) / 2 <= b) ++I;
    J = b - I * (I + 1) / 2;
}

// Each CTA streams a contiguous run of the lower triangle's 64 x 64 blocks (row-major, so a
// run covers long stretches of one block row) through a two-deep cp.async ring; every
// block of A is read once.  Thread (r, part) accumulates row r of block row I over a
// quarter of each block's columns in registers until the row's diagonal block (or the end
// of the run), then the four partials go to Y with one atomic per row.  A strictly lower
// block also contributes A(I, J)^T x_I to block row J: reduced in shared memory, one atomic
// per row of J.  ABS uses |A| (row sums of |A| give the infinity norm).  VEC stages A in
// 16-byte pieces (A 16-byte aligned, lda even), else one element per copy.
template <bool ABS, int NR, bool VEC>
__global__ void __launch_bounds__(kSolveThreads) symm_lower_kernel(const double *A, int64_t lda, int64_t n,
                                                                   const double *X, int64_t ldx, double *Y,
                                                                   int64_t ldy, int nrhs, double alpha) {
    constexpr int STAGES = 2;
    constexpr int kStr = VEC ? kSB + 2 : kTS;  // shared-memory stride of a staged block
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double *ring = reinterpret_cast<double *>(smem_raw);  // STAGES x [kSB][kStr], element (r, c) at c * kStr + r
    double *xs = ring + STAGES * kSB * kStr;              // STAGES x {x_J, x_I} x [NR][kSB]
    double *red = xs + STAGES * 2 * NR * kSB;             // [4][NR][kSB] column partials
    double *rred = red + 4 * NR * kSB;                    // [4][NR][kSB] row partials
    const int tid = threadIdx.x, r = tid % kSB, part = tid / kSB;
    const int64_t nb = (n + kSB - 1) / kSB;
    const int64_t total = nb * (nb + 1) / 2;
    const int64_t first = total * blockIdx.x / gridDim.x, last = total * (blockIdx.x + 1) / gridDim.x;
    if (first >= last) return;
    auto stage = [&](int64_t b) {
        if (b < last) {
            int64_t I, J;
            lower_block_coords(b, I, J);
            const int slot = static_cast<int>((b - first) % STAGES);
            const int ri = static_cast<int>(min(int64_t(kSB), n - I * kSB));
            const int cj = static_cast<int>(min(int64_t(kSB), n - J * kSB));
            const double *G = A + I * kSB + J * kSB * lda;
            double *T = ring + slot * kSB * kStr;
            if constexpr (VEC) {
                for (int e = tid; e < kSB * kSB / 2; e += kSolveThreads) {
                    const int rr = (e % (kSB / 2)) * 2, cc = e / (kSB / 2);
                    const int rows = cc < cj ? min(2, max(0, ri - rr)) : 0;
                    cp_async16_part(T + cc * kStr + rr, rows ? G + rr + int64_t(cc) * lda : G, rows * 8);
                }
            } else {
                for (int e = tid; e < kSB * kSB; e += kSolveThreads) {
                    const int rr = e % kSB, cc = e / kSB;
                    const bool ok = rr < ri && cc < cj;
                    cp_async_elem(T + cc * kStr + rr, ok ? G + rr + int64_t(cc) * lda : G, ok);
                }
            }
            double *xj = xs + slot * 2 * NR * kSB, *xi = xj + NR * kSB;
            for (int e = tid; e < NR * kSB; e += kSolveThreads) {
                const int q = e % kSB, c = e / kSB;
                const bool okj = q < cj && c < nrhs, oki = q < ri && c < nrhs;
                cp_async_elem(xj + e, okj ? X + (J * kSB + q) + int64_t(c) * ldx : X, okj);
                cp_async_elem(xi + e, oki ? X + (I * kSB + q) + int64_t(c) * ldx : X, oki);
            }
        }
        cp_async_commit();
    };
    double racc[NR];
#pragma unroll
    for (int k = 0; k < NR; ++k) racc[k] = 0.0;
    stage(first);
    for (int64_t b = first; b < last; ++b) {
        int64_t I, J;
        lower_block_coords(b, I, J);
        const int slot = static_cast<int>((b - first) % STAGES);
        cp_async_wait<STAGES - 2>();
        __syncthreads();  // block b landed; block b - 1's readers of its slot and of red are done
        stage(b + 1);
        const double *T = ring + slot * kSB * kStr;
        const double *xj = xs + slot * 2 * NR * kSB, *xi = xj + NR * kSB;
#pragma unroll
        for (int i = 0; i < kSB / 4; ++i) {
            const int c = part * (kSB / 4) + i;
            double a = (I != J || r >= c) ? T[c * kStr + r] : T[r * kStr + c];  // mirror inside the diagonal block
            if (ABS) a = fabs(a);
#pragma unroll
            for (int k = 0; k < NR; ++k) racc[k] += a * xj[k * kSB + c];
        }
        if (I != J) {
            double cacc[NR];
#pragma unroll
            for (int k = 0; k < NR; ++k) cacc[k] = 0.0;
#pragma unroll
            for (int i = 0; i < kSB / 4; ++i) {
                const int rr = part * (kSB / 4) + i;
                double a = T[r * kStr + rr];  // A(rr, r): row rr of block row I, column r of block row J
                if (ABS) a = fabs(a);
#pragma unroll
                for (int k = 0; k < NR; ++k) cacc[k] += a * xi[k * kSB + rr];
            }
#pragma unroll
            for (int k = 0; k < NR; ++k) red[(part * NR + k) * kSB + r] = cacc[k];
        }
        const bool row_end = J == I || b + 1 == last;
        if (row_end) {
#pragma unroll
            for (int k = 0; k < NR; ++k) {
                rred[(part * NR + k) * kSB + r] = racc[k];
                racc[k] = 0.0;
            }
        }
        if (I != J || row_end) __syncthreads();
        if (I != J) {
            const int cj = static_cast<int>(min(int64_t(kSB), n - J * kSB));
            for (int e = tid; e < NR * kSB; e += kSolveThreads) {
                const int q = e % kSB, k = e / kSB;
                if (q < cj && k < nrhs)
                    atomicAdd(Y + (J * kSB + q) + int64_t(k) * ldy,
                              alpha * (red[e] + red[NR * kSB + e] + red[2 * NR * kSB + e] + red[3 * NR * kSB + e]));
            }
        }
        if (row_end) {
            const int ri = static_cast<int>(min(int64_t(kSB), n - I * kSB));
            for (int e = tid; e < NR * kSB; e += kSolveThreads) {
                const int q = e % kSB, k = e / kSB;
                if (q < ri && k < nrhs)
                    atomicAdd(Y + (I * kSB + q) + int64_t(k) * ldy,
                              alpha * (rred[e] + rred[NR * kSB + e] + rred[2 * NR * kSB + e] + rred[3 * NR * kSB + e]));
            }
        }
    }
    cp_async_wait<0>();
}

template <int NR>
constexpr size_t symm_smem() {
    return (size_t(2) * kSB * (kSB + 2) + 2 * 2 * NR * kSB + 8 * NR * kSB) * sizeof(double);
}

// ---- wavefront triangular solves with the factor ---------------------------------

// Start the copy of the KB x KB block B into S, S[q * STRIDE + r] = B(r, q) = G[r + q ld],
// in 16-byte pieces along r (G, ld and STRIDE keep every piece 16-byte aligned); entries
// outside rv x qv are zero, and a piece that straddles row rv reads only the rows before it.
template <typename T, int KB, int STRIDE>
__device__ __forceinline__ void stage_block_v(T *S, const T *G, int64_t ld, int rv, int qv) {
    constexpr int kEpc = 16 / int(sizeof(T));
    constexpr int kPieces = KB / kEpc;
    for (int e = threadIdx.x; e < kPieces * KB; e += kSolveThreads) {
        const int r = (e % kPieces) * kEpc, q = e / kPieces;
        const int rows = q < qv ? min(kEpc, max(0, rv - r)) : 0;
        cp_async16_part(S + q * STRIDE + r, rows ? G + r + int64_t(q) * ld : G, rows * int(sizeof(T)));
    }
}

// WT(j) = W(j)^T for each KB x KB diagonal-block inverse (rows j KB.., columns 0..KB-1 of
// W and of WT), so that the backward sweeps stage W_j^T with contiguous column pieces too.
template <typename T, int KB>
__global__ void __launch_bounds__(kSolveThreads) transpose_blocks_kernel(const T *W, int64_t ldw, T *WT, int64_t ldt,
                                                                         int n) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T *tile = reinterpret_cast<T *>(smem_raw);  // [KB][KB + 1]
    const int64_t r0 = int64_t(blockIdx.x) * KB;
    const int rj = static_cast<int>(min(int64_t(KB), n - r0));
    for (int e = threadIdx.x; e < KB * KB; e += kSolveThreads) {
        const int r = e % KB, c = e / KB;
        tile[c * (KB + 1) + r] = (r < rj && c < rj) ? W[(r0 + r) + int64_t(c) * ldw] : T(0);
    }
    __syncthreads();
    for (int e = threadIdx.x; e < KB * KB; e += kSolveThreads) {
        const int r = e % KB, c = e / KB;
        if (r < rj) WT[(r0 + r) + int64_t(c) * ldt] = tile[r * (KB + 1) + c];
    }
}

// Copy the strictly lower 64 x 64 blocks of L into the upper triangle as L^T, so that the
// backward sweep reads L(k, j)^T = U(j, k) with the same contiguous column pieces as the
// forward sweep reads L(j, k).  Grid (J, I); blocks with I <= J return at once.
template <typename T>
__global__ void __launch_bounds__(kSolveThreads) upper_from_lower_kernel(T *F, int64_t ldf, int n) {
    __shared__ T tile[kSB][kSB + 1];
    const int J = blockIdx.x, I = blockIdx.y;
    if (I <= J) return;
    const int64_t r0 = int64_t(I) * kSB, c0 = int64_t(J) * kSB;
    const int ri = static_cast<int>(min(int64_t(kSB), n - r0));
    for (int e = threadIdx.x; e < kSB * kSB; e += kSolveThreads) {
        const int r = e % kSB, c = e / kSB;
        if (r < ri) tile[c][r] = F[(r0 + r) + (c0 + c) * ldf];
    }
    __syncthreads();
    for (int e = threadIdx.x; e < kSB * kSB; e += kSolveThreads) {
        const int c = e % kSB, r = e / kSB;  // element (c, r) of U: row c0 + c, column r0 + r
        if (r < ri) F[(c0 + c) + (r0 + r) * ldf] = tile[c][r];
    }
}

// V(J) = inverse of the 128 x 128 diagonal block J of L, from the inverses W1, W2 of its two
// 64 x 64 diagonal blocks (in W, rows of the block, columns 0..63):
//   inv([[L11, 0], [L21, L22]]) = [[W1, 0], [-W2 L21 W1, W2]].
// One CTA per block; entries past n are zero.
template <typename T>
__global__ void __launch_bounds__(kSolveThreads) inverse128_kernel(const T *L, int64_t ldl, const T *W, int64_t ldw,
                                                                   int n, T *V, int64_t ldv) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T *w1 = reinterpret_cast<T *>(smem_raw);  // [c][r] at c * kTS + r
    T *w2 = w1 + kSB * kTS;
    T *l21 = w2 + kSB * kTS;
    T *t = l21 + kSB * kTS;
    const int tid = threadIdx.x;
    const int64_t r0 = int64_t(blockIdx.x) * 128;
    const int h1 = static_cast<int>(min(int64_t(kSB), n - r0));
    const int h2 = static_cast<int>(max(int64_t(0), min(int64_t(kSB), n - r0 - kSB)));
    for (int e = tid; e < kSB * kSB; e += kSolveThreads) {
        const int a = e % kSB, c = e / kSB;
        w1[c * kTS + a] = (a < h1 && c < h1) ? W[(r0 + a) + int64_t(c) * ldw] : T(0);
        w2[c * kTS + a] = (a < h2 && c < h2) ? W[(r0 + kSB + a) + int64_t(c) * ldw] : T(0);
        l21[c * kTS + a] = (a < h2 && c < h1) ? L[(r0 + kSB + a) + (r0 + c) * ldl] : T(0);
    }
    __syncthreads();
    // t = L21 W1, then V21 = -W2 t; thread (a, quarter) makes 16 entries of row a
    const int a = tid % kSB, q0 = (tid / kSB) * (kSB / 4);
    T acc[kSB / 4];
#pragma unroll
    for (int i = 0; i < kSB / 4; ++i) acc[i] = T(0);
    for (int m = 0; m < kSB; ++m) {
        const T x = l21[m * kTS + a];
#pragma unroll
        for (int i = 0; i < kSB / 4; ++i) acc[i] += x * w1[(q0 + i) * kTS + m];
    }
#pragma unroll
    for (int i = 0; i < kSB / 4; ++i) t[(q0 + i) * kTS + a] = acc[i];
    __syncthreads();
#pragma unroll
    for (int i = 0; i < kSB / 4; ++i) acc[i] = T(0);
    for (int m = 0; m < kSB; ++m) {
        const T x = w2[m * kTS + a];
#pragma unroll
        for (int i = 0; i < kSB / 4; ++i) acc[i] -= x * t[(q0 + i) * kTS + m];
    }
    for (int e = tid; e < 128 * 128; e += kSolveThreads) {
        const int rr = e % 128, c = e / 128;
        if (rr >= kSB && c < kSB) continue;  // V21: written from acc below
        T v = T(0);
        if (rr < kSB && c < kSB) v = w1[c * kTS + rr];
        else if (rr >= kSB && c >= kSB) v = w2[(c - kSB) * kTS + rr - kSB];
        if (r0 + rr < n) V[(r0 + rr) + int64_t(c) * ldv] = v;
    }
#pragma unroll
    for (int i = 0; i < kSB / 4; ++i)
        if (r0 + kSB + a < n) V[(r0 + kSB + a) + int64_t(q0 + i) * ldv] = acc[i];
}

// ---- mailbox words: a 32-bit payload tagged with the epoch of the launch that wrote it ----
//
// A solved block is published as 64-bit words (payload in the low half, epoch in the high
// half), each written with one single-copy-atomic store.  A reader that sees the current
// epoch in a word has that word's payload: no flag, no fence and no second read.  A float
// takes one word, a double two (low and high halves of its bits).

__device__ __forceinline__ unsigned long long ld_relaxed(const unsigned long long *p) {
    unsigned long long v;
    asm volatile("ld.relaxed.gpu.global.b64 %0, [%1];\n" : "=l"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_relaxed(unsigned long long *p, unsigned long long v) {
    asm volatile("st.relaxed.gpu.global.b64 [%0], %1;\n" ::"l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ unsigned long long tag(unsigned payload, unsigned epoch) {
    return (static_cast<unsigned long long>(epoch) << 32) | payload;
}

template <typename T>
struct MailWords {
    static constexpr int kPerValue = sizeof(T) / 4;
};

template <typename T>
__device__ __forceinline__ void post_value(unsigned long long *box, int i, T v, unsigned epoch) {
    if constexpr (sizeof(T) == 4) {
        st_relaxed(box + i, tag(__float_as_uint(v), epoch));
    } else {
        const unsigned long long b = static_cast<unsigned long long>(__double_as_longlong(v));
        st_relaxed(box + 2 * i, tag(static_cast<unsigned>(b), epoch));
        st_relaxed(box + 2 * i + 1, tag(static_cast<unsigned>(b >> 32), epoch));
    }
}

// Warp-wide: copy the `count` values of mailbox `box` into y once every word carries
// `epoch` (returns 1), or give up when the shared error word is set or the kernel has run
// for timeout_ns (returns 0, recording MTD_ERR_TIMEOUT).  All 32 lanes must call.
template <typename T>
__device__ __forceinline__ int collect(const unsigned long long *box, int count, unsigned epoch, T *y, int *err,
                                       unsigned long long t0, unsigned long long timeout_ns) {
    const int lane = threadIdx.x & 31;
    constexpr int kW = MailWords<T>::kPerValue;
    for (unsigned it = 1;; ++it) {
        bool ok = true;
        for (int i = lane; i < count; i += 32) {
            if constexpr (kW == 1) {
                const unsigned long long w = ld_relaxed(box + i);
                ok &= static_cast<unsigned>(w >> 32) == epoch;
                y[i] = __uint_as_float(static_cast<unsigned>(w));
            } else {
                const unsigned long long lo = ld_relaxed(box + 2 * i), hi = ld_relaxed(box + 2 * i + 1);
                ok &= static_cast<unsigned>(lo >> 32) == epoch && static_cast<unsigned>(hi >> 32) == epoch;
                y[i] = __longlong_as_double(static_cast<long long>((hi << 32) | (lo & 0xffffffffull)));
            }
        }
        if (__all_sync(0xffffffffu, ok)) return 1;
        if ((it & 63) == 0) {
            int stop = 0;
            if (lane == 0) {
                if (*reinterpret_cast<volatile int *>(err) != 0) stop = 1;
                else if (global_ns() - t0 > timeout_ns) {
                    atomicCAS(err, 0, MTD_ERR_TIMEOUT);
                    stop = 1;
                }
            }
            if (__shfl_sync(0xffffffffu, stop, 0)) return 0;
        }
    }
}

// One warp's view of a mailbox of NV * 32 values, lane l holding values l + 32 m: load()
// issues the reads without waiting, so a poll can overlap other work; valid() / decode()
// use the words last loaded.
template <typename T, int NV>
struct MailPrefetch {
    static constexpr int kW = MailWords<T>::kPerValue;
    unsigned long long w[NV * kW];
    __device__ __forceinline__ void load(const unsigned long long *box, int lane) {
#pragma unroll
        for (int m = 0; m < NV; ++m) {
            const int i = lane + 32 * m;
            if constexpr (kW == 1) {
                w[m] = ld_relaxed(box + i);
            } else {
                w[2 * m] = ld_relaxed(box + 2 * i);
                w[2 * m + 1] = ld_relaxed(box + 2 * i + 1);
            }
        }
    }
    __device__ __forceinline__ bool valid(unsigned epoch) const {
        bool ok = true;
#pragma unroll
        for (int m = 0; m < NV * kW; ++m) ok &= static_cast<unsigned>(w[m] >> 32) == epoch;
        return ok;
    }
    __device__ __forceinline__ void decode(T *y, int lane) const {
#pragma unroll
        for (int m = 0; m < NV; ++m) {
            if constexpr (kW == 1)
                y[lane + 32 * m] = __uint_as_float(static_cast<unsigned>(w[m]));
            else
                y[lane + 32 * m] = __longlong_as_double(
                    static_cast<long long>((w[2 * m + 1] << 32) | (w[2 * m] & 0xffffffffull)));
        }
    }
};

// X <- L^-1 X (forward) or L^-T X (backward), L lower with the inverses of its KB x KB
// diagonal blocks in W.  One CTA per KB-row block j; a CTA takes its block from a ticket
// counter, so every block it waits for belongs to a CTA that started earlier (no CTA ever
// waits on one that may not be resident).  Each wait is bounded; a CTA that gives up or
// sees the shared error word set records MTD_ERR_TIMEOUT and returns.
//
// The coupling blocks L(j, k) (forward) or L(k, j)^T = U(j, k) (backward, from the copy of
// L^T in the factor's upper triangle) stream through a STAGES-deep ring of 16-byte
// cp.async pieces ahead of the wavefront, followed by W_j, so a CTA's only wait on the
// chain is for block k's mailbox.  Thread (r, part) keeps the partial sums of output row r over a
// share of each block's columns in registers for the whole sweep; warp 0 collects y_k
// from the mailbox, and a single barrier per block step publishes it with the staged tile.
// The last step reduces the partials and applies W_j (forward y_j = W_j acc, backward
// W_j^T acc), then posts y_j to block j's mailbox and to X.  The sweep is a chain of
// n / KB hand-offs, so larger blocks mean a shorter chain.
template <typename T, bool BACKWARD, int NR, int STAGES, int KB>
__global__ void __launch_bounds__(kSolveThreads) trsv_wavefront_kernel(
    const T *L, int64_t ldl, const T *W, int64_t ldw, int n, T *X, int64_t ldx, int nrhs, int *ticket,
    unsigned long long *mail, unsigned epoch, unsigned long long timeout_ns, int *err) {
    constexpr int kStride = KB + 16 / int(sizeof(T));  // rows of a staged block stay 16-byte aligned
    constexpr int kParts = kSolveThreads / KB;
    constexpr int kCols = KB / kParts;  // columns of a block per thread and step
    constexpr int kBoxWords = NR * KB * MailWords<T>::kPerValue;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T *ring = reinterpret_cast<T *>(smem_raw);  // STAGES x [KB][kStride]
    T *ys = ring + STAGES * KB * kStride;       // [2][NR][KB]        y_k, double-buffered
    T *red = ys + 2 * NR * KB;                  // [kParts][NR][KB]   partial sums at the end
    __shared__ int s_b, s_abort;
    const int tid = threadIdx.x, lane = tid & 31;
    const int r = tid % KB, part = tid / KB;
    const int nb = (n + KB - 1) / KB;
    if (tid == 0) {
        s_b = atomicAdd(ticket, 1);
        s_abort = 0;
    }
    __syncthreads();
    const int b = s_b;
    if (b >= nb) return;
    const int j = BACKWARD ? nb - 1 - b : b;
    const int rj = min(KB, n - j * KB);
    const int count = BACKWARD ? nb - 1 - j : j;
    // copy for step s: coupling block of step s < count, W_j at s == count, nothing after
    auto stage = [&](int s) {
        T *S = ring + (s % STAGES) * KB * kStride;
        if (s < count) {
            const int k = BACKWARD ? nb - 1 - s : s;
            const int rk = min(KB, n - k * KB);
            stage_block_v<T, KB, kStride>(S, L + int64_t(j) * KB + int64_t(k) * KB * ldl, ldl, rj, rk);
        } else if (s == count) {
            stage_block_v<T, KB, kStride>(S, W + int64_t(j) * KB, ldw, rj, rj);
        }
        cp_async_commit();
    };
    T acc[NR];
#pragma unroll
    for (int c = 0; c < NR; ++c)
        acc[c] = (part == 0 && r < rj && c < nrhs) ? X[(int64_t(j) * KB + r) + int64_t(c) * ldx] : T(0);
#pragma unroll
    for (int s = 0; s < STAGES - 1; ++s) stage(s);
    const unsigned long long t0 = global_ns();
    // Small mailboxes are read one step ahead by warp 0 (the loads fly while the CTA works
    // on the current step), so a step whose y_k is already posted costs no round trip.
    constexpr int kNV = NR * KB / 32;
    constexpr bool kAhead = kNV * MailWords<T>::kPerValue <= 8;
    MailPrefetch<T, kAhead ? kNV : 1> ahead;
    auto box_of = [&](int s) { return mail + int64_t(BACKWARD ? nb - 1 - s : s) * kBoxWords; };
    if constexpr (kAhead)
        if (tid < 32 && count > 0) ahead.load(box_of(0), lane);
    for (int s = 0; s < count; ++s) {
        T *yk = ys + (s & 1) * NR * KB;
        if (tid < 32) {
            bool ready = false;
            if constexpr (kAhead) {
                ready = __all_sync(0xffffffffu, ahead.valid(epoch));
                if (ready) ahead.decode(yk, lane);
            }
            if (!ready && !collect<T>(box_of(s), NR * KB, epoch, yk, err, t0, timeout_ns) && lane == 0)
                s_abort = 1;
        }
        cp_async_wait<STAGES - 2>();
        __syncthreads();
        if (s_abort) {
            cp_async_wait<0>();
            return;
        }
        if constexpr (kAhead)
            if (tid < 32 && s + 1 < count) ahead.load(box_of(s + 1), lane);
        stage(s + STAGES - 1);
        const T *S = ring + (s % STAGES) * KB * kStride;
#pragma unroll
        for (int i = 0; i < kCols; ++i) {
            const int q = part * kCols + i;
            const T l = S[q * kStride + r];
#pragma unroll
            for (int c = 0; c < NR; ++c) acc[c] -= l * yk[c * KB + q];
        }
    }
#pragma unroll
    for (int c = 0; c < NR; ++c) red[(part * NR + c) * KB + r] = acc[c];
    cp_async_wait<0>();
    __syncthreads();
    for (int e = tid; e < NR * KB; e += kSolveThreads) {
        T v = red[e];
#pragma unroll
        for (int p = 1; p < kParts; ++p) v += red[p * NR * KB + e];
        ys[e] = v;
    }
    __syncthreads();
    const T *Wt = ring + (count % STAGES) * KB * kStride;
    unsigned long long *box = mail + int64_t(j) * kBoxWords;
    for (int e = tid; e < NR * KB; e += kSolveThreads) {
        const int rr = e % KB, c = e / KB;
        T s = T(0);
#pragma unroll 16
        for (int q = 0; q < KB; ++q) s += Wt[q * kStride + rr] * ys[c * KB + q];
        // rows past n and columns past nrhs hold zeros: they are posted too, so readers
        // need no bounds of their own
        post_value(box, e, s, epoch);
        if (rr < rj && c < nrhs) X[(int64_t(j) * KB + rr) + int64_t(c) * ldx] = s;
    }
}

// Solve block edge: 128 for FP32 factors (inverse blocks built after the factorisation),
// 64 for FP64 (two 128 x 128 FP64 blocks would not fit shared memory twice over).
template <typename T>
constexpr int trsv_block() {
    return sizeof(T) == 8 ? 64 : 128;
}
template <typename T, int NR>
constexpr int trsv_stages() {
    return sizeof(T) == 8 ? 2 : (NR <= 4 ? 3 : 2);
}
template <typename T, int NR>
constexpr size_t trsv_smem() {
    constexpr int kb = trsv_block<T>();
    constexpr int stride = kb + 16 / int(sizeof(T));
    return (size_t(trsv_stages<T, NR>()) * kb * stride + (2 + kSolveThreads / kb) * NR * kb) * sizeof(T);
}

// ---- GMRES helpers (FP64 vectors) ------------------------------------------------

// out[i] = sum_r V(r, i) * w(r), i < m  (one block row per CTA column pass)
__global__ void multi_dot_kernel(const double *V, int64_t ldv, int m, const double *w, int64_t n, double *out) {
    __shared__ double part[kSolveThreads / 32];
    const int i = blockIdx.y;
    double s = 0.0;
    for (int64_t r = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; r < n; r += int64_t(gridDim.x) * blockDim.x)
        s += V[r + i * ldv] * w[r];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int k = 0; k < int(blockDim.x / 32); ++k) t += part[k];
        atomicAdd(out + i, t);
    }
    (void)m;
}

// w -= V(:, 0:m) * h
__global__ void multi_axpy_kernel(const double *V, int64_t ldv, int m, const double *h, double *w, int64_t n) {
    for (int64_t r = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; r < n; r += int64_t(gridDim.x) * blockDim.x) {
        double s = w[r];
        for (int i = 0; i < m; ++i) s -= V[r + i * ldv] * h[i];
        w[r] = s;
    }
}

// y = V(:, 0:m) * h (+ y when accumulate)
__global__ void combine_kernel(const double *V, int64_t ldv, int m, const double *h, double *y, int64_t n,
                               bool accumulate) {
    for (int64_t r = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; r < n; r += int64_t(gridDim.x) * blockDim.x) {
        double s = accumulate ? y[r] : 0.0;
        for (int i = 0; i < m; ++i) s += V[r + i * ldv] * h[i];
        y[r] = s;
    }
}

__global__ void scal_kernel(double *x, int64_t n, double a) {
    for (int64_t r = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; r < n; r += int64_t(gridDim.x) * blockDim.x)
        x[r] *= a;
}

double bits_to_double(unsigned long long b) {
    double d;
    std::memcpy(&d, &b, sizeof(d));
    return d;
}

}  // namespace

struct mtd_solver {
    int64_t n = 0, tile = 0;
    int prec = MTD_PREC_TF32;
    int sms = 148;
    mtd_graph *g = nullptr;
    void *fac = nullptr;      // factor storage (float or double), ld = ldf
    int64_t ldf = 0;
    const double *a = nullptr;  // caller's matrix (lower triangle read), for residuals
    int64_t lda = 0;
    double anorm = 0.0;
    double shift = 0.0;
    bool factored = false;
    double factor_ms = 0.0;
    // work (n x kMaxRhs unless noted)
    double *r = nullptr, *d64 = nullptr, *ones = nullptr;
    void *dlo = nullptr;      // low-precision solve vectors (factor's element type)
    unsigned long long *norms = nullptr;  // 4 x kMaxRhs ordered-bit maxima
    int *ticket = nullptr, *err = nullptr;
    unsigned long long *mail = nullptr;  // triangular-solve mailboxes: nb x 64 x kMaxRhs x 2 words
    float *inv128 = nullptr;             // FP32 factors: inverses of the 128 x 128 diagonal blocks (ldf x 128)
    void *inv_t = nullptr;               // transposes of the solve's diagonal-block inverses (ldf x block)
    unsigned epoch = 0;                  // tag of the current solve launch (0 never used)
    // GMRES (one right-hand side at a time)
    int gm_restart = 0;
    double *V = nullptr, *w = nullptr, *hbuf = nullptr;
};

namespace {

size_t fac_elem(const mtd_solver *s) { return s->prec == MTD_PREC_FP64 ? sizeof(double) : sizeof(float); }

dim3 vec_grid(int64_t n, int cols) {
    return dim3(static_cast<unsigned>(std::min<int64_t>(1024, (n + kSolveThreads - 1) / kSolveThreads)),
                static_cast<unsigned>(cols));
}

template <bool ABS, int NR>
int symm_launch(mtd_solver *s, const double *X, int64_t ldx, double *Y, int64_t ldy, int nrhs, double alpha,
                cudaStream_t st) {
    const bool vec = (reinterpret_cast<uintptr_t>(s->a) & 15) == 0 && (s->lda & 1) == 0;
    auto kern = vec ? symm_lower_kernel<ABS, NR, true> : symm_lower_kernel<ABS, NR, false>;
    constexpr size_t kSmem = symm_smem<NR>();
    int dev = 0, sms = 0, per_sm = 0;
    if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(kSmem)) != cudaSuccess ||
        cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kSolveThreads, kSmem) != cudaSuccess)
        return MTD_ERR_CUDA;
    const int64_t nb = (s->n + kSB - 1) / kSB;
    const int64_t blocks = std::min<int64_t>(nb * (nb + 1) / 2, int64_t(sms) * std::max(per_sm, 1));
    kern<<<static_cast<unsigned>(blocks), kSolveThreads, kSmem, st>>>(s->a, s->lda, s->n, X, ldx, Y, ldy, nrhs, alpha);
    return cudaGetLastError() == cudaSuccess ? MTD_OK : MTD_ERR_CUDA;
}

// Y += alpha * A X with A symmetric (lower triangle read); |A| when abs.
int symm(mtd_solver *s, const double *X, int64_t ldx, double *Y, int64_t ldy, int nrhs, double alpha, bool abs,
         cudaStream_t st) {
    if (abs) return symm_launch<true, 1>(s, X, ldx, Y, ldy, nrhs, alpha, st);  // nrhs is 1 here (a vector of ones)
    if (nrhs <= 1) return symm_launch<false, 1>(s, X, ldx, Y, ldy, nrhs, alpha, st);
    if (nrhs <= 4) return symm_launch<false, 4>(s, X, ldx, Y, ldy, nrhs, alpha, st);
    return symm_launch<false, kMaxRhs>(s, X, ldx, Y, ldy, nrhs, alpha, st);
}

template <typename T, bool BACKWARD, int NR>
int trsv_launch(mtd_solver *s, T *X, int64_t ldx, int nrhs, cudaStream_t st) {
    constexpr int kStages = trsv_stages<T, NR>();
    constexpr int kBlock = trsv_block<T>();
    constexpr size_t kSmem = trsv_smem<T, NR>();
    auto kern = trsv_wavefront_kernel<T, BACKWARD, NR, kStages, kBlock>;
    if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(kSmem)) != cudaSuccess)
        return MTD_ERR_CUDA;
    const void *w = BACKWARD ? s->inv_t : kBlock == kSB ? mtd::graph_ws_lower(s->g) : static_cast<const void *>(s->inv128);
    const T *W = static_cast<const T *>(w);
    const int64_t ldw = kBlock == kSB && !BACKWARD ? mtd::graph_ws_ld(s->g) : s->ldf;
    const int nb = static_cast<int>((s->n + kBlock - 1) / kBlock);
    const unsigned long long timeout = 10ull * 1000000000ull;
    if (cudaMemsetAsync(s->ticket, 0, sizeof(int), st) != cudaSuccess) return MTD_ERR_CUDA;
    if (++s->epoch == 0) ++s->epoch;  // the zeroed mailboxes carry epoch 0
    kern<<<nb, kSolveThreads, kSmem, st>>>(static_cast<const T *>(s->fac), s->ldf, W, ldw, static_cast<int>(s->n), X,
                                           ldx, nrhs, s->ticket, s->mail, s->epoch, timeout, s->err);
    return cudaGetLastError() == cudaSuccess ? MTD_OK : MTD_ERR_CUDA;
}

template <typename T, int NR>
int trsv_pair_nr(mtd_solver *s, T *X, int64_t ldx, int nrhs, cudaStream_t st) {
    int rc = trsv_launch<T, false, NR>(s, X, ldx, nrhs, st);
    return rc ? rc : trsv_launch<T, true, NR>(s, X, ldx, nrhs, st);
}

// X <- (L L^T)^-1 X; right-hand sides go in register-resident groups of 1, 4 or 16.
template <typename T>
int trsv_pair(mtd_solver *s, T *X, int64_t ldx, int nrhs, cudaStream_t st) {
    if (nrhs <= 1) return trsv_pair_nr<T, 1>(s, X, ldx, nrhs, st);
    if (nrhs <= 4) return trsv_pair_nr<T, 4>(s, X, ldx, nrhs, st);
    return trsv_pair_nr<T, kMaxRhs>(s, X, ldx, nrhs, st);
}

// D = M^-1 R (in FP64 columns), M = L L^T the factor.  R is not modified.
int apply_inverse(mtd_solver *s, const double *R, int64_t ldr, double *D, int64_t ldd, int nrhs, cudaStream_t st) {
    const int64_t n = s->n;
    if (s->prec == MTD_PREC_FP64) {
        if (cudaMemcpy2DAsync(D, ldd * sizeof(double), R, ldr * sizeof(double), n * sizeof(double), nrhs,
                              cudaMemcpyDeviceToDevice, st) != cudaSuccess)
            return MTD_ERR_CUDA;
        return trsv_pair<double>(s, D, ldd, nrhs, st);
    }
    // scale each column to max-norm 1 before rounding to FP32, solve, scale back
    unsigned long long *scale = s->norms + 3 * kMaxRhs;
    if (cudaMemsetAsync(scale, 0, kMaxRhs * sizeof(unsigned long long), st) != cudaSuccess) return MTD_ERR_CUDA;
    colmax_kernel<<<vec_grid(n, nrhs), kSolveThreads, 0, st>>>(R, ldr, n, nrhs, scale);
    float *lo = static_cast<float *>(s->dlo);
    scale_copy_kernel<double, float><<<vec_grid(n, nrhs), kSolveThreads, 0, st>>>(R, ldr, lo, n, n, nrhs, scale,
                                                                                   true, false);
    int rc = trsv_pair<float>(s, lo, n, nrhs, st);
    if (rc) return rc;
    scale_copy_kernel<float, double><<<vec_grid(n, nrhs), kSolveThreads, 0, st>>>(lo, n, D, ldd, n, nrhs, scale,
                                                                                   false, false);
    return cudaGetLastError() == cudaSuccess ? MTD_OK : MTD_ERR_CUDA;
}

// Normwise backward error per column: ||r||_inf / (||A||_inf ||x||_inf + ||b||_inf); returns the max.
int backward_error(mtd_solver *s, const double *X, int64_t ldx, const double *B, int64_t ldb, int nrhs,
                   cudaStream_t st, double *berr, double *per_col) {
    const int64_t n = s->n;
    // r = b - A x
    if (cudaMemcpy2DAsync(s->r, n * sizeof(double), B, ldb * sizeof(double), n * sizeof(double), nrhs,
                          cudaMemcpyDeviceToDevice, st) != cudaSuccess)
        return MTD_ERR_CUDA;
    int rc = symm(s, X, ldx, s->r, n, nrhs, -1.0, false, st);
    if (rc) return rc;
    if (cudaMemsetAsync(s->norms, 0, 3 * kMaxRhs * sizeof(unsigned long long), st) != cudaSuccess) return MTD_ERR_CUDA;
    colmax_kernel<<<vec_grid(n, nrhs), kSolveThreads, 0, st>>>(s->r, n, n, nrhs, s->norms);
    colmax_kernel<<<vec_grid(n, nrhs), kSolveThreads, 0, st>>>(X, ldx, n, nrhs, s->norms + kMaxRhs);
    colmax_kernel<<<vec_grid(n, nrhs), kSolveThreads, 0, st>>>(B, ldb, n, nrhs, s->norms + 2 * kMaxRhs);
    unsigned long long h[3 * kMaxRhs];
    if (cudaMemcpyAsync(h, s->norms, sizeof(h), cudaMemcpyDeviceToHost, st) != cudaSuccess) return MTD_ERR_CUDA;
    if (cudaStreamSynchronize(st) != cudaSuccess) return MTD_ERR_CUDA;
    int e = 0;
    if (cudaMemcpy(&e, s->err, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess) return MTD_ERR_CUDA;
    if (e) return e;
    double worst = 0.0;
    for (int c = 0; c < nrhs; ++c) {
        const double rn = bits_to_double(h[c]), xn = bits_to_double(h[kMaxRhs + c]), bn = bits_to_double(h[2 * kMaxRhs + c]);
        const double den = s->anorm * xn + bn;
        const double be = den > 0 ? rn / den : rn;
        if (per_col) per_col[c] = be;
        worst = std::max(worst, be);
    }
    *berr = worst;
    return MTD_OK;
}

void release(mtd_solver *s) {
    if (s->g) mtd_graph_destroy(s->g);
    cudaFree(s->fac);
    cudaFree(s->r);
    cudaFree(s->d64);
    cudaFree(s->ones);
    cudaFree(s->dlo);
    cudaFree(s->norms);
    cudaFree(s->ticket);
    cudaFree(s->mail);
    cudaFree(s->inv128);
    cudaFree(s->inv_t);
    cudaFree(s->err);
    cudaFree(s->V);
    cudaFree(s->w);
    cudaFree(s->hbuf);
}

template <typename T>
int alloc(T **p, size_t count) {
    if (cudaMalloc(reinterpret_cast<void **>(p), std::max<size_t>(count, 1) * sizeof(T)) != cudaSuccess) {
        cudaGetLastError();
        *p = nullptr;
        return MTD_ERR_OUT_OF_MEMORY;
    }
    return MTD_OK;
}

// GMRES(m) on M^-1 A d = M^-1 r for one column (FP64 Krylov basis, classical Gram-Schmidt
// applied twice, Givens rotations on the host).  Returns the inner iterations used.
int gmres_correction(mtd_solver *s, const double *r, double *d, double rel_tol, int max_inner, cudaStream_t st,
                     int *inner_out) {
    const int64_t n = s->n;
    const int m = s->gm_restart;
    double *V = s->V, *w = s->w;
    // v0 = M^-1 r / beta
    int rc = apply_inverse(s, r, n, V, n, 1, st);
    if (rc) return rc;
    auto norm2 = [&](const double *x, double *out) -> int {
        if (cudaMemsetAsync(s->hbuf, 0, sizeof(double), st) != cudaSuccess) return MTD_ERR_CUDA;
        multi_dot_kernel<<<dim3(vec_grid(n, 1).x, 1), kSolveThreads, 0, st>>>(x, n, 1, x, n, s->hbuf);
        double h = 0;
        if (cudaMemcpyAsync(&h, s->hbuf, sizeof(double), cudaMemcpyDeviceToHost, st) != cudaSuccess) return MTD_ERR_CUDA;
        if (cudaStreamSynchronize(st) != cudaSuccess) return MTD_ERR_CUDA;
        *out = std::sqrt(h);
        return MTD_OK;
    };
    double beta = 0;
    if ((rc = norm2(V, &beta))) return rc;
    if (beta == 0.0) {
        cudaMemsetAsync(d, 0, n * sizeof(double), st);
        *inner_out = 0;
        return MTD_OK;
    }
    scal_kernel<<<vec_grid(n, 1), kSolveThreads, 0, st>>>(V, n, 1.0 / beta);
    std::vector<double> H(size_t(m + 1) * m, 0.0), cs(m, 0.0), sn(m, 0.0), g(m + 1, 0.0);
    g[0] = beta;
    int k = 0;
    std::vector<double> hcol(m + 1);
    for (; k < m && k < max_inner; ++k) {
        // w = M^-1 (A v_k)
        if (cudaMemsetAsync(s->r + n, 0, n * sizeof(double), st) != cudaSuccess) return MTD_ERR_CUDA;
        double *av = s->r + n;  // column 1 of the residual buffer as scratch
        if ((rc = symm(s, V + k * n, n, av, n, 1, 1.0, false, st))) return rc;
        if ((rc = apply_inverse(s, av, n, w, n, 1, st))) return rc;
        // two passes of classical Gram-Schmidt against v_0..v_k
        std::fill(hcol.begin(), hcol.end(), 0.0);
        for (int pass = 0; pass < 2; ++pass) {
            if (cudaMemsetAsync(s->hbuf, 0, (k + 1) * sizeof(double), st) != cudaSuccess) return MTD_ERR_CUDA;
            multi_dot_kernel<<<dim3(vec_grid(n, 1).x, k + 1), kSolveThreads, 0, st>>>(V, n, k + 1, w, n, s->hbuf);
            multi_axpy_kernel<<<vec_grid(n, 1), kSolveThreads, 0, st>>>(V, n, k + 1, s->hbuf, w, n);
            std::vector<double> hh(k + 1);
            if (cudaMemcpyAsync(hh.data(), s->hbuf, (k + 1) * sizeof(double), cudaMemcpyDeviceToHost, st) != cudaSuccess)
                return MTD_ERR_CUDA;
            if (cudaStreamSynchronize(st) != cudaSuccess) return MTD_ERR_CUDA;
            for (int i = 0; i <= k; ++i) hcol[i] += hh[i];
        }
        double hn = 0;
        if ((rc = norm2(w, &hn))) return rc;
        hcol[k + 1] = hn;
        if (hn > 0) {
            if (cudaMemcpyAsync(V + (k + 1) * n, w, n * sizeof(double), cudaMemcpyDeviceToDevice, st) != cudaSuccess)
                return MTD_ERR_CUDA;
            scal_kernel<<<vec_grid(n, 1), kSolveThreads, 0, st>>>(V + (k + 1) * n, n, 1.0 / hn);
        }
        // apply previous rotations, then a new one
        for (int i = 0; i < k; ++i) {
            const double t = cs[i] * hcol[i] + sn[i] * hcol[i + 1];
            hcol[i + 1] = -sn[i] * hcol[i] + cs[i] * hcol[i + 1];
            hcol[i] = t;
        }
        const double den = std::hypot(hcol[k], hcol[k + 1]);
        cs[k] = den > 0 ? hcol[k] / den : 1.0;
        sn[k] = den > 0 ? hcol[k + 1] / den : 0.0;
        hcol[k] = den;
        hcol[k + 1] = 0.0;
        g[k + 1] = -sn[k] * g[k];
        g[k] = cs[k] * g[k];
        for (int i = 0; i <= k; ++i) H[i + size_t(k) * (m + 1)] = hcol[i];
        if (std::fabs(g[k + 1]) <= rel_tol * beta || hn == 0.0) {
            ++k;
            break;
        }
    }
    // y = H(0:k, 0:k)^-1 g(0:k); d = V(:, 0:k) y
    std::vector<double> y(k, 0.0);
    for (int i = k - 1; i >= 0; --i) {
        double t = g[i];
        for (int j = i + 1; j < k; ++j) t -= H[i + size_t(j) * (m + 1)] * y[j];
        y[i] = t / H[i + size_t(i) * (m + 1)];
    }
    if (cudaMemcpyAsync(s->hbuf, y.data(), std::max(k, 1) * sizeof(double), cudaMemcpyHostToDevice, st) != cudaSuccess)
        return MTD_ERR_CUDA;
    combine_kernel<<<vec_grid(n, 1), kSolveThreads, 0, st>>>(V, n, k, s->hbuf, d, n, false);
    *inner_out = k;
    return cudaGetLastError() == cudaSuccess ? MTD_OK : MTD_ERR_CUDA;
}

}  // namespace

extern "C" {

int mtd_solver_create(mtd_solver **out, int64_t n, int64_t tile, int prec) {
    if (!out) return MTD_ERR_INVALID_ARG;
    *out = nullptr;
    if (n <= 0 || tile <= 0 || tile > n || tile % kSB != 0 || n > (int64_t(1) << 30)) return MTD_ERR_INVALID_ARG;
    if (prec != MTD_PREC_FP64 && prec != MTD_PREC_TF32 && prec != MTD_PREC_FP32 && prec != MTD_PREC_BF16)
        return MTD_ERR_INVALID_ARG;
    mtd_solver *s = new (std::nothrow) mtd_solver();
    if (!s) return MTD_ERR_OUT_OF_MEMORY;
    s->n = n;
    s->tile = tile;
    s->prec = prec;
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&s->sms, cudaDevAttrMultiProcessorCount, dev);
    int rc = mtd_graph_create(&s->g, MTD_KIND_CHOLESKY, n, tile);
    if (!rc) rc = mtd_graph_build_tiled(s->g);
    if (!rc) rc = mtd_graph_set_precision(s->g, prec);
    if (!rc) rc = mtd_graph_finalize(s->g);
    s->ldf = (n + 3) & ~int64_t(3);
    const int nb = static_cast<int>((n + kSB - 1) / kSB);
    s->gm_restart = 50;
    if (!rc) rc = cudaMalloc(&s->fac, size_t(s->ldf) * size_t(n) * fac_elem(s)) == cudaSuccess ? MTD_OK : MTD_ERR_OUT_OF_MEMORY;
    if (!rc) rc = alloc(&s->r, size_t(n) * kMaxRhs);
    if (!rc) rc = alloc(&s->d64, size_t(n) * kMaxRhs);
    if (!rc) rc = alloc(&s->ones, size_t(n));
    if (!rc) rc = cudaMalloc(&s->dlo, size_t(n) * kMaxRhs * sizeof(float)) == cudaSuccess ? MTD_OK : MTD_ERR_OUT_OF_MEMORY;
    if (!rc) rc = alloc(&s->norms, 4 * kMaxRhs);
    if (!rc) rc = alloc(&s->ticket, 1);
    if (!rc) rc = alloc(&s->mail, size_t(nb) * kSB * kMaxRhs * 2);
    if (!rc && prec != MTD_PREC_FP64) rc = alloc(&s->inv128, size_t(s->ldf) * 128);
    if (!rc)  // 128 floats or 64 doubles per row: the same bytes
        rc = cudaMalloc(&s->inv_t, size_t(s->ldf) * 512) == cudaSuccess ? MTD_OK : MTD_ERR_OUT_OF_MEMORY;
    if (!rc) rc = alloc(&s->err, 1);
    if (!rc) rc = alloc(&s->V, size_t(n) * (s->gm_restart + 1));
    if (!rc) rc = alloc(&s->w, size_t(n));
    if (!rc) rc = alloc(&s->hbuf, s->gm_restart + 2);
    if (!rc) {
        cudaMemset(s->mail, 0, size_t(nb) * kSB * kMaxRhs * 2 * sizeof(unsigned long long));
        cudaMemset(s->err, 0, sizeof(int));
        fill_kernel<<<256, 256>>>(s->ones, n, 1.0);
        if (cudaDeviceSynchronize() != cudaSuccess) rc = MTD_ERR_CUDA;
    }
    if (rc) {
        release(s);
        delete s;
        return rc;
    }
    *out = s;
    return MTD_OK;
}

int mtd_solver_factor(mtd_solver *s, const double *dA, int64_t lda, double shift, void *stream, int *info_out) {
    if (info_out) *info_out = 0;
    if (!s || !dA || lda < s->n || shift < 0) return MTD_ERR_INVALID_ARG;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    s->a = dA;
    s->lda = lda;
    s->shift = shift;
    s->factored = false;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, st);
    const unsigned blocks = static_cast<unsigned>(std::min<int64_t>(65535, (s->n * s->n + 255) / 256));
    if (s->prec == MTD_PREC_FP64)
        copy_lower_kernel<double><<<blocks, 256, 0, st>>>(dA, lda, static_cast<double *>(s->fac), s->ldf, s->n, shift);
    else
        copy_lower_kernel<float><<<blocks, 256, 0, st>>>(dA, lda, static_cast<float *>(s->fac), s->ldf, s->n, shift);
    int info = 0;
    int rc = s->prec == MTD_PREC_FP64 ? mtd_run(s->g, static_cast<double *>(s->fac), s->ldf, stream, nullptr)
                                      : mtd_run_f32(s->g, static_cast<float *>(s->fac), s->ldf, stream, nullptr);
    cudaEventRecord(e1, st);
    if (!rc) rc = mtd_graph_status(s->g, &info);
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    s->factor_ms = ms;
    if (info_out) *info_out = info;
    if (rc) return rc;
    // L^T into the upper triangle for the backward sweeps
    const unsigned nb64 = static_cast<unsigned>((s->n + kSB - 1) / kSB);
    if (s->prec == MTD_PREC_FP64)
        upper_from_lower_kernel<double><<<dim3(nb64, nb64), kSolveThreads, 0, st>>>(static_cast<double *>(s->fac),
                                                                                  s->ldf, static_cast<int>(s->n));
    else
        upper_from_lower_kernel<float><<<dim3(nb64, nb64), kSolveThreads, 0, st>>>(static_cast<float *>(s->fac),
                                                                                 s->ldf, static_cast<int>(s->n));
    if (cudaGetLastError() != cudaSuccess) return MTD_ERR_CUDA;
    if (s->prec != MTD_PREC_FP64) {  // 128 x 128 inverse diagonal blocks for the triangular solves
        constexpr size_t kInvSmem = 4 * kSB * kTS * sizeof(float);
        if (cudaFuncSetAttribute(inverse128_kernel<float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 int(kInvSmem)) != cudaSuccess)
            return MTD_ERR_CUDA;
        inverse128_kernel<float><<<static_cast<unsigned>((s->n + 127) / 128), kSolveThreads, kInvSmem, st>>>(
            static_cast<const float *>(s->fac), s->ldf, static_cast<const float *>(mtd::graph_ws_lower(s->g)),
            mtd::graph_ws_ld(s->g), static_cast<int>(s->n), s->inv128, s->ldf);
        constexpr size_t kTrSmem = 128 * 129 * sizeof(float);
        if (cudaFuncSetAttribute(transpose_blocks_kernel<float, 128>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 int(kTrSmem)) != cudaSuccess)
            return MTD_ERR_CUDA;
        transpose_blocks_kernel<float, 128><<<static_cast<unsigned>((s->n + 127) / 128), kSolveThreads, kTrSmem, st>>>(
            s->inv128, s->ldf, static_cast<float *>(s->inv_t), s->ldf, static_cast<int>(s->n));
    } else {
        constexpr size_t kTrSmem = 64 * 65 * sizeof(double);
        if (cudaFuncSetAttribute(transpose_blocks_kernel<double, 64>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 int(kTrSmem)) != cudaSuccess)
            return MTD_ERR_CUDA;
        transpose_blocks_kernel<double, 64><<<nb64, kSolveThreads, kTrSmem, st>>>(
            static_cast<const double *>(mtd::graph_ws_lower(s->g)), mtd::graph_ws_ld(s->g),
            static_cast<double *>(s->inv_t), s->ldf, static_cast<int>(s->n));
    }
    if (cudaGetLastError() != cudaSuccess) return MTD_ERR_CUDA;
    // ||A||_inf of the symmetric matrix: max row sum of |A|
    if (cudaMemsetAsync(s->d64, 0, s->n * sizeof(double), st) != cudaSuccess) return MTD_ERR_CUDA;
    if ((rc = symm(s, s->ones, s->n, s->d64, s->n, 1, 1.0, true, st))) return rc;
    if (cudaMemsetAsync(s->norms, 0, sizeof(unsigned long long), st) != cudaSuccess) return MTD_ERR_CUDA;
    colmax_kernel<<<vec_grid(s->n, 1), kSolveThreads, 0, st>>>(s->d64, s->n, s->n, 1, s->norms);
    unsigned long long h = 0;
    if (cudaMemcpyAsync(&h, s->norms, sizeof(h), cudaMemcpyDeviceToHost, st) != cudaSuccess) return MTD_ERR_CUDA;
    if (cudaStreamSynchronize(st) != cudaSuccess) return MTD_ERR_CUDA;
    s->anorm = bits_to_double(h);
    s->factored = true;
    return MTD_OK;
}

int mtd_solver_solve(mtd_solver *s, const double *dB, int64_t ldb, double *dX, int64_t ldx, int64_t nrhs, int method,
                     double tol, int max_iter, void *stream, mtd_solve_stats *stats) {
    if (!s || !dB || !dX || ldb < s->n || ldx < s->n || nrhs < 1 || nrhs > kMaxRhs || max_iter < 0)
        return MTD_ERR_INVALID_ARG;
    if (method != MTD_REFINE_NONE && method != MTD_REFINE_IR && method != MTD_REFINE_GMRES_IR) return MTD_ERR_INVALID_ARG;
    if (method == MTD_REFINE_GMRES_IR && nrhs != 1) return MTD_ERR_INVALID_ARG;
    if (!s->factored) return MTD_ERR_STATE;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int64_t n = s->n;
    const int nr = static_cast<int>(nrhs);
    const auto t0 = std::chrono::steady_clock::now();
    mtd_solve_stats local{};
    local.factor_ms = s->factor_ms;
    int rc = cudaMemsetAsync(s->err, 0, sizeof(int), st) == cudaSuccess ? MTD_OK : MTD_ERR_CUDA;
    double berr = 0.0;
    if (method == MTD_REFINE_NONE) {
        rc = apply_inverse(s, dB, ldb, dX, ldx, nr, st);
        if (!rc) rc = backward_error(s, dX, ldx, dB, ldb, nr, st, &berr, nullptr);
        local.iterations = 1;
        local.converged = berr <= tol;
    } else {
        // x = 0, then x += correction until the backward error reaches tol
        if (cudaMemset2DAsync(dX, ldx * sizeof(double), 0, n * sizeof(double), nr, st) != cudaSuccess) rc = MTD_ERR_CUDA;
        int it = 0;
        while (!rc) {
            if (it == 0) {  // x = 0: r = b, backward error 1, no product with A needed
                berr = 1.0;
                if (cudaMemcpy2DAsync(s->r, n * sizeof(double), dB, ldb * sizeof(double), n * sizeof(double), nr,
                                      cudaMemcpyDeviceToDevice, st) != cudaSuccess)
                    rc = MTD_ERR_CUDA;
            } else {
                rc = backward_error(s, dX, ldx, dB, ldb, nr, st, &berr, nullptr);  // leaves r = b - A x in s->r
            }
            if (rc) break;
            if (it > 0 && berr <= tol) {
                local.converged = 1;
                break;
            }
            if (it >= max_iter) break;
            if (method == MTD_REFINE_IR) {
                rc = apply_inverse(s, s->r, n, s->d64, n, nr, st);
            } else {
                int inner = 0;
                rc = gmres_correction(s, s->r, s->d64, 1e-4, s->gm_restart, st, &inner);
                local.inner_iterations += inner;
            }
            if (rc) break;
            for (int c = 0; c < nr; ++c)
                combine_kernel<<<vec_grid(n, 1), kSolveThreads, 0, st>>>(s->d64 + c * n, n, 1, s->ones, dX + c * ldx, n,
                                                                         true);
            ++it;
        }
        local.iterations = it;
    }
    if (cudaStreamSynchronize(st) != cudaSuccess && !rc) rc = MTD_ERR_CUDA;
    local.backward_error = berr;
    local.solve_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    if (stats) *stats = local;
    return rc;
}

int mtd_solver_destroy(mtd_solver *s) {
    if (!s) return MTD_ERR_INVALID_ARG;
    cudaDeviceSynchronize();
    release(s);
    delete s;
    return MTD_OK;
}

}  // extern "C"
