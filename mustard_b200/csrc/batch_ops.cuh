// Batched solves, one CTA of NT threads per matrix: forward / backward substitution with the
// Cholesky factor and the inverses of its 64 x 64 diagonal blocks, the FP64 residual with
// the matrix's normwise backward error, the steps of iterative refinement, and the
// conversion of a matrix to the factor's precision.  The standalone solve kernels
// (batch.cu, 256 threads) and the solve / conversion tasks of the persistent
// factor-and-solve launch (scheduler.cuh, 512 threads) run this same code.
//
// Blocks stream through two shared-memory buffers: each thread loads its elements of block
// t + 1 into registers, the CTA multiplies with block t, and the registers are stored into
// the other buffer before the step's one barrier, so the loads of the next block are in
// flight during the product.  (The first solve kernels loaded every block element by element
// in dependent load / store loops: ~5 ms per launch for 4096 matrices of up to 1024.)  The
// 64 x 64 by 64 x nrhs block products run on the tensor cores, one 16 x 8 output tile per
// warp: FP64 DMMA (mma.sync.m16n8k8.f64) for the FP64 steps, and for the float solves the
// FP32-accurate three-pass TF32 product (mma.cuh): a scalar loop over a block reads two
// shared-memory operands per multiply-add and bound each step at ~2 us.
// The factor and its inverse blocks are read through L2 (ld.global.cg): inside the
// persistent launch other SMs wrote them during the same kernel, and L1 is not coherent
// across SMs.  Vectors this CTA wrote itself are read with plain loads after a barrier.
#pragma once

#include <cstdint>

#include "../../include/mustard_b200.h"
#include "device_types.hpp"
#include "mma.cuh"

namespace mtd {
namespace bsolve {

constexpr int kSB = 64;      // solve block (= inverse block edge)
constexpr int kMaxRhs = 16;  // right-hand sides per matrix
enum { kOnX = 0, kOnD = 1, kOnR = 2 };  // which vector block of SolveMat a solve overwrites

// Shared memory of one CTA: two [kSB][kLD] blocks, two [kMaxRhs][kLD] vector blocks and one
// [kMaxRhs][kLD] accumulator in the element type of the step (a float solve packs them into
// half the bytes), then, at the offsets of the FP64 layout, the reductions
// (3 x kMaxRhs x warps), kMaxRhs column scales and the matrix norm.  A row stride of
// 68 = 4 mod 16 elements makes the fragment reads of a half-warp (rows g = 0..3, columns
// t = 0..3) hit 16 distinct 8-byte bank pairs.
constexpr int kLD = kSB + 4;
constexpr int kBlkD = 2 * kSB * kLD;
constexpr int kVecD = 2 * kMaxRhs * kLD;
constexpr int kAccD = kMaxRhs * kLD;
template <int NT>
constexpr int red_doubles() { return 3 * kMaxRhs * (NT / 32); }
template <typename T>
constexpr size_t trsv_bytes() { return size_t(kBlkD + kVecD + kAccD) * sizeof(T); }
template <int NT>
constexpr size_t smem_bytes() { return size_t(kBlkD + kVecD + kAccD + red_doubles<NT>() + kMaxRhs + 2) * sizeof(double); }

struct Smem {
    unsigned char *base;
    template <typename T> __device__ T *blocks() const { return reinterpret_cast<T *>(base); }
    template <typename T> __device__ T *vecs() const { return reinterpret_cast<T *>(base) + kBlkD; }
    template <typename T> __device__ T *acc() const { return reinterpret_cast<T *>(base) + kBlkD + kVecD; }
    __device__ double *red() const { return reinterpret_cast<double *>(base) + kBlkD + kVecD + kAccD; }
    template <int NT> __device__ double *scale() const { return red() + red_doubles<NT>(); }
    template <int NT> __device__ double *norm() const { return scale<NT>() + kMaxRhs; }
};

template <typename T>
__device__ __forceinline__ T ldcg(const T *p) { return __ldcg(p); }

// The threads that run one matrix's steps: the whole CTA (bar = 0: __syncthreads), or a
// warp-aligned group of NT threads that meets at named barrier `bar` (two matrices per CTA).
struct Grp {
    int tid;  // thread index within the group
    int bar;
};
template <int NT>
__device__ __forceinline__ void gsync(const Grp &g) {
    if (g.bar == 0) gsync<NT>(g);
    else asm volatile("bar.sync %0, %1;" ::"r"(g.bar), "r"(NT) : "memory");
}

__device__ __forceinline__ void blk_mma(double (&d)[4], const double (&a)[4], const double (&b)[2]) {
    mma_16x8x8(d, a, b);
}
__device__ __forceinline__ void blk_mma(float (&d)[4], const float (&a)[4], const float (&b)[2]) {
    mma_16x8x8_x3(d, a, b);
}

// d += A(m0 .. m0 + 15, 0 .. 63) B(0 .. 63, n0 .. n0 + 7) on one warp; A stored [m][k], B
// stored [n][k], both with row stride kLD.  d holds (g, 2t), (g, 2t + 1), (g + 8, 2t),
// (g + 8, 2t + 1) of the tile (g = lane / 4, t = lane % 4; mma.cuh's fragment layout).
template <typename T>
__device__ __forceinline__ void warp_tile(T (&d)[4], const T *A, const T *B, int m0, int n0) {
    const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
#pragma unroll
    for (int ks = 0; ks < kSB; ks += 8) {
        const T a[4] = {A[(m0 + g) * kLD + ks + t], A[(m0 + g + 8) * kLD + ks + t], A[(m0 + g) * kLD + ks + t + 4],
                        A[(m0 + g + 8) * kLD + ks + t + 4]};
        const T b[2] = {B[(n0 + g) * kLD + ks + t], B[(n0 + g) * kLD + ks + t + 4]};
        blk_mma(d, a, b);
    }
}
__device__ __forceinline__ int tile_row(int m0, int v) { return m0 + ((threadIdx.x & 31) >> 2) + ((v & 2) ? 8 : 0); }
__device__ __forceinline__ int tile_col(int n0, int v) { return n0 + 2 * (threadIdx.x & 3) + (v & 1); }

// Forward then backward substitution with L and the inverses of its 64 x 64 diagonal blocks,
// on the n x nrhs block Y (the target of SolveMat), in T.  Block row j subtracts L(j, k) Y(k)
// for the rows k solved before it and applies the inverse of its diagonal block.
template <typename T, int NT>
__device__ void trsv(const Grp &g, const SolveMat &sm, const T *ws, int target, Smem sh) {
    constexpr int kL = kSB * kSB / NT;       // elements of a 64 x 64 block per thread
    constexpr int kY = kMaxRhs * kSB / NT;   // elements of a vector block per thread
    static_assert(kSB * kSB % NT == 0 && kMaxRhs * kSB % NT == 0, "whole elements per thread");
    T *Lb = sh.blocks<T>();
    T *Yb = sh.vecs<T>();
    T *Acc = sh.acc<T>();
    const int n = sm.n, nrhs = sm.nrhs, tid = g.tid;
    const T *L = static_cast<const T *>(sm.f);
    const int64_t ldl = sm.ldf;
    const T *W = ws + sm.ws_off;
    const int64_t ldw = sm.ws_ld;
    T *Y = target == kOnX ? reinterpret_cast<T *>(sm.x)
                          : (target == kOnR ? reinterpret_cast<T *>(sm.r) : static_cast<T *>(sm.d));
    const int64_t ldy = target == kOnX ? sm.ldx : n;
    const int nb = (n + kSB - 1) / kSB;
    // output tiles of a block product: 4 (rows) x 1 or 2 (columns), one per warp
    const int warp = tid >> 5, tiles = 4 * ((nrhs + 7) / 8);
    const int m0 = 16 * (warp & 3), n0 = 8 * (warp >> 2);
    static_assert(NT >= 256, "one warp per output tile of a 64 x 16 block");
    T lr[kL], yr[kY];
    for (int pass = 0; pass < 2; ++pass) {
        const bool back = pass == 1;
        for (int s = 0; s < nb; ++s) {
            const int j = back ? nb - 1 - s : s;
            const int rj = min(kSB, n - j * kSB);
            // step t < s: L(j, k_t) (transposed in the backward pass) and Y(k_t); t = s: W_j
            auto fetch = [&](int t) {
                if (t < s) {
                    const int k = back ? nb - 1 - t : t;
                    const int rk = min(kSB, n - k * kSB);
#pragma unroll
                    for (int q = 0; q < kL; ++q) {
                        const int e = tid + NT * q, a = e % kSB, c = e / kSB;
                        if (!back)
                            lr[q] = (a < rj && c < rk) ? ldcg(L + (int64_t(j) * kSB + a) + (int64_t(k) * kSB + c) * ldl)
                                                       : T(0);
                        else
                            lr[q] = (a < rk && c < rj) ? ldcg(L + (int64_t(k) * kSB + a) + (int64_t(j) * kSB + c) * ldl)
                                                       : T(0);
                    }
#pragma unroll
                    for (int q = 0; q < kY; ++q) {
                        const int e = tid + NT * q, r = e % kSB, c = e / kSB;
                        yr[q] = (c < nrhs && r < rk) ? Y[(int64_t(k) * kSB + r) + c * ldy] : T(0);
                    }
                } else {
#pragma unroll
                    for (int q = 0; q < kL; ++q) {
                        const int e = tid + NT * q, a = e % kSB, c = e / kSB;
                        lr[q] = (a < rj && c < rj) ? ldcg(W + (int64_t(j) * kSB + a) + int64_t(c) * ldw) : T(0);
                    }
                }
            };
            auto stash = [&](int t) {
                T *Ld = Lb + (t & 1) * kSB * kLD;
                const bool transposed = back;  // the backward pass multiplies with L^T
#pragma unroll
                for (int q = 0; q < kL; ++q) {
                    const int e = tid + NT * q, a = e % kSB, c = e / kSB;
                    Ld[transposed ? c * kLD + a : a * kLD + c] = lr[q];
                }
                if (t < s) {
                    T *Yd = Yb + (t & 1) * kMaxRhs * kLD;
#pragma unroll
                    for (int q = 0; q < kY; ++q) {
                        const int e = tid + NT * q, r = e % kSB, c = e / kSB;
                        Yd[c * kLD + r] = yr[q];
                    }
                }
            };
            fetch(0);
            for (int e = tid; e < kSB * kMaxRhs; e += NT) {
                const int r = e % kSB, c = e / kSB;
                Acc[c * kLD + r] = (r < rj && c < nrhs) ? Y[(int64_t(j) * kSB + r) + c * ldy] : T(0);
            }
            stash(0);
            gsync<NT>(g);
            for (int t = 0; t <= s; ++t) {
                if (t + 1 <= s) fetch(t + 1);  // in flight during the product below
                const T *Lc = Lb + (t & 1) * kSB * kLD;
                if (warp < tiles) {
                    T d[4] = {T(0), T(0), T(0), T(0)};
                    if (t < s) {  // Acc -= L(j, k_t) Y(k_t)
                        warp_tile(d, Lc, Yb + (t & 1) * kMaxRhs * kLD, m0, n0);
#pragma unroll
                        for (int v = 0; v < 4; ++v) Acc[tile_col(n0, v) * kLD + tile_row(m0, v)] -= d[v];
                    } else {      // Y(j) = W_j Acc
                        warp_tile(d, Lc, Acc, m0, n0);
#pragma unroll
                        for (int v = 0; v < 4; ++v) {
                            const int r = tile_row(m0, v), c = tile_col(n0, v);
                            if (r < rj && c < nrhs) Y[(int64_t(j) * kSB + r) + c * ldy] = d[v];
                        }
                    }
                }
                if (t + 1 <= s) stash(t + 1);  // the other buffer: last read in step t - 1
                gsync<NT>(g);  // Y(j) stored before later rows read it; the buffers change hands
            }
        }
    }
}

// The block (I, J) of the symmetric matrix whose lower triangle A holds: element e of a
// 64 x 64 block maps to (row r, column c) of A(I, J) so that consecutive e read consecutive
// addresses (columns of A(J, I) for J > I).
__device__ __forceinline__ void sym_coord(int I, int J, int e, int *r, int *c) {
    if (J > I) {
        *c = e % kSB;
        *r = e / kSB;
    } else {
        *r = e % kSB;
        *c = e / kSB;
    }
}
__device__ __forceinline__ int64_t sym_offset(int I, int J, int r, int c, int64_t lda) {
    const int64_t gi = int64_t(I) * kSB + r, gj = int64_t(J) * kSB + c;
    return gi >= gj ? gi + gj * lda : gj + gi * lda;
}

// Column maxima of |v| (nrhs columns, leading dimension ld) into red[which][c][warp].
template <int NT>
__device__ __forceinline__ void col_absmax(const Grp &g, const double *v, int64_t ld, int n, int nrhs, double *red,
                                           int which) {
    const int tid = g.tid;
    for (int c = 0; c < nrhs; ++c) {
        double m = 0.0;
        for (int i = tid; i < n; i += NT) m = fmax(m, fabs(v[i + int64_t(c) * ld]));
        for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
        if ((tid & 31) == 0) red[(which * kMaxRhs + c) * (NT / 32) + (tid >> 5)] = m;
    }
}

// r = b - A_sym x and the matrix's normwise backward error max_c ||r_c|| / (||A|| ||x_c|| +
// ||b_c||) (infinity norms), returned to every thread.  Block row I of r is formed in
// registers over the whole symmetric block row and written once.  With want_anorm the same
// pass sums |A| along each row and stores ||A_sym||_inf in *anorm (thread 0); otherwise
// *anorm is read.
template <int NT>
__device__ double residual(const Grp &g, const SolveMat &sm, double *anorm, bool want_anorm, Smem sh) {
    constexpr int kA = kSB * kSB / NT;
    constexpr int kX = kMaxRhs * kSB / NT;
    double *Ab = sh.blocks<double>();
    double *Xb = sh.vecs<double>();
    double *red = sh.red();
    const int n = sm.n, nrhs = sm.nrhs, tid = g.tid;
    const double *A = sm.a;
    const int64_t lda = sm.lda;
    const int nb = (n + kSB - 1) / kSB;
    const int warp = tid >> 5, tiles = 4 * ((nrhs + 7) / 8);  // output tiles of a block row, one per warp
    const int m0 = 16 * (warp & 3), n0 = 8 * (warp >> 2);
    double ar[kA], xr[kX];
    double amax = 0.0;
    for (int I = 0; I < nb; ++I) {
        const int ri = min(kSB, n - I * kSB);
        auto fetch = [&](int J) {
            const int cj = min(kSB, n - J * kSB);
#pragma unroll
            for (int q = 0; q < kA; ++q) {
                int r, c;
                sym_coord(I, J, tid + NT * q, &r, &c);
                ar[q] = (r < ri && c < cj) ? A[sym_offset(I, J, r, c, lda)] : 0.0;
            }
#pragma unroll
            for (int q = 0; q < kX; ++q) {
                const int e = tid + NT * q, k = e % kSB, c = e / kSB;
                xr[q] = (c < nrhs && k < cj) ? sm.x[(int64_t(J) * kSB + k) + c * sm.ldx] : 0.0;
            }
        };
        auto stash = [&](int J) {
            double *Ad = Ab + (J & 1) * kSB * kLD;
            double *Xd = Xb + (J & 1) * kMaxRhs * kLD;
#pragma unroll
            for (int q = 0; q < kA; ++q) {
                int r, c;
                sym_coord(I, J, tid + NT * q, &r, &c);
                Ad[r * kLD + c] = ar[q];
            }
#pragma unroll
            for (int q = 0; q < kX; ++q) {
                const int e = tid + NT * q, k = e % kSB, c = e / kSB;
                Xd[c * kLD + k] = xr[q];
            }
        };
        double d[4] = {0.0, 0.0, 0.0, 0.0};  // this warp's tile of A(I, :) x, over all J
        double rowsum = 0.0;
        fetch(0);
        stash(0);
        gsync<NT>(g);
        for (int J = 0; J < nb; ++J) {
            if (J + 1 < nb) fetch(J + 1);
            const double *Ac = Ab + (J & 1) * kSB * kLD;
            if (warp < tiles) warp_tile(d, Ac, Xb + (J & 1) * kMaxRhs * kLD, m0, n0);
            if (want_anorm && tid < kSB) {
#pragma unroll 8
                for (int k = 0; k < kSB; ++k) rowsum += fabs(Ac[tid * kLD + k]);
            }
            if (J + 1 < nb) stash(J + 1);
            gsync<NT>(g);
        }
        if (warp < tiles) {
#pragma unroll
            for (int v = 0; v < 4; ++v) {
                const int r = tile_row(m0, v), c = tile_col(n0, v);
                if (r < ri && c < nrhs)
                    sm.r[(int64_t(I) * kSB + r) + int64_t(c) * n] = sm.b[(int64_t(I) * kSB + r) + c * sm.ldb] - d[v];
            }
        }
        if (want_anorm && tid < ri) amax = fmax(amax, rowsum);
    }
    if (want_anorm) {
        for (int o = 16; o > 0; o >>= 1) amax = fmax(amax, __shfl_xor_sync(0xffffffffu, amax, o));
        if ((tid & 31) == 0) red[tid >> 5] = amax;
        gsync<NT>(g);
        if (tid == 0) {
            double m = 0.0;
            for (int w = 0; w < NT / 32; ++w) m = fmax(m, red[w]);
            *anorm = m;
        }
    }
    gsync<NT>(g);  // r written; the reduction area is free again; *anorm published
    col_absmax<NT>(g, sm.r, n, n, nrhs, red, 0);
    col_absmax<NT>(g, sm.x, sm.ldx, n, nrhs, red, 1);
    col_absmax<NT>(g, sm.b, sm.ldb, n, nrhs, red, 2);
    gsync<NT>(g);
    const double an = *anorm;
    double worst = 0.0;
    for (int c = 0; c < nrhs; ++c) {
        double mr = 0.0, mx = 0.0, mb = 0.0;
        for (int w = 0; w < NT / 32; ++w) {
            mr = fmax(mr, red[(0 * kMaxRhs + c) * (NT / 32) + w]);
            mx = fmax(mx, red[(1 * kMaxRhs + c) * (NT / 32) + w]);
            mb = fmax(mb, red[(2 * kMaxRhs + c) * (NT / 32) + w]);
        }
        const double den = an * mx + mb;
        worst = fmax(worst, den > 0 ? mr / den : mr);
    }
    gsync<NT>(g);  // every thread has read the reductions
    return worst;
}

// r = b, the residual of x = 0, and its backward error (1 for a column with b != 0, else 0:
// with x = 0 the error measure is ||b|| / ||b||), without reading A.
template <int NT>
__device__ double residual_of_zero(const Grp &g, const SolveMat &sm, Smem sh) {
    double *red = sh.red();
    const int n = sm.n, nrhs = sm.nrhs;
    for (int64_t e = g.tid; e < int64_t(n) * nrhs; e += NT) {
        const int64_t i = e % n, c = e / n;
        sm.r[i + c * n] = sm.b[i + c * sm.ldb];
    }
    col_absmax<NT>(g, sm.b, sm.ldb, n, nrhs, red, 2);
    gsync<NT>(g);
    double worst = 0.0;
    for (int c = 0; c < nrhs; ++c) {
        double mb = 0.0;
        for (int w = 0; w < NT / 32; ++w) mb = fmax(mb, red[(2 * kMaxRhs + c) * (NT / 32) + w]);
        worst = fmax(worst, mb > 0.0 ? 1.0 : 0.0);
    }
    gsync<NT>(g);  // every thread has read the reductions
    return worst;
}

// d = r / max|r| per column, rounded to T; the column scales go to scale[c].
template <typename T, int NT>
__device__ void scale_to_low(const Grp &g, const SolveMat &sm, double *scale, double *red) {
    const int n = sm.n, tid = g.tid;
    T *d = static_cast<T *>(sm.d);
    for (int c = 0; c < sm.nrhs; ++c) {
        double m = 0.0;
        for (int i = tid; i < n; i += NT) m = fmax(m, fabs(sm.r[i + int64_t(c) * n]));
        for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
        gsync<NT>(g);  // the previous column's reduction has been read
        if ((tid & 31) == 0) red[tid >> 5] = m;
        gsync<NT>(g);
        double s = 0.0;
        for (int w = 0; w < NT / 32; ++w) s = fmax(s, red[w]);
        if (s == 0.0) s = 1.0;
        if (tid == 0) scale[c] = s;
        for (int i = tid; i < n; i += NT) d[i + int64_t(c) * n] = static_cast<T>(sm.r[i + int64_t(c) * n] / s);
    }
    gsync<NT>(g);
}

// x += scale_c * d (the scaled low-precision correction).
template <typename T, int NT>
__device__ void add_scaled(const Grp &g, const SolveMat &sm, const double *scale) {
    const T *d = static_cast<const T *>(sm.d);
    for (int c = 0; c < sm.nrhs; ++c) {
        const double s = scale[c];
        for (int i = g.tid; i < sm.n; i += NT)
            sm.x[i + int64_t(c) * sm.ldx] += s * static_cast<double>(d[i + int64_t(c) * sm.n]);
    }
    gsync<NT>(g);
}

// x += r (FP64 correction).
template <int NT>
__device__ void add_r(const Grp &g, const SolveMat &sm) {
    for (int64_t e = g.tid; e < int64_t(sm.n) * sm.nrhs; e += NT) {
        const int64_t i = e % sm.n, c = e / sm.n;
        sm.x[i + c * sm.ldx] += sm.r[i + c * sm.n];
    }
    gsync<NT>(g);
}

// x = b, or x = 0.
template <int NT>
__device__ void copy_rhs(const Grp &g, const SolveMat &sm, bool zero) {
    for (int64_t e = g.tid; e < int64_t(sm.n) * sm.nrhs; e += NT) {
        const int64_t i = e % sm.n, c = e / sm.n;
        sm.x[i + c * sm.ldx] = zero ? 0.0 : sm.b[i + c * sm.ldb];
    }
    gsync<NT>(g);
}

// Columns [c0, c1) of F = lower triangle of A (+ shift on the diagonal), rounded to T.
template <typename T, int NT>
__device__ void convert(const Grp &g, const double *A, int64_t lda, T *F, int64_t ldf, int n, double shift, int c0,
                        int c1) {
    for (int j = c0; j < c1; ++j)
        for (int i = j + g.tid; i < n; i += NT) {
            double v = A[i + int64_t(j) * lda];
            if (i == j) v += shift;
            F[i + int64_t(j) * ldf] = static_cast<T>(v);
        }
}

// The whole solve of one matrix, as the host loop of mtd_batch_solve runs it over separate
// launches: FP64 factor: x = (L L^T)^-1 b, then (with A) the backward error and, for
// MTD_REFINE_IR, FP64 refinement steps x += (L L^T)^-1 r; low-precision factor: x = 0, then
// refinement steps x += s (L L^T)^-1 (r / s) with the correction solved in T and s = max|r|
// per column, until the backward error is <= tol after at least one step, or max_iter steps.
// *berr: the last backward error (-1 without A); *iters: the solves applied.
template <typename T, int NT>
__device__ void solve_refine(const Grp &g, const SolveMat &sm, const T *ws, int method, double tol, int max_iter,
                             Smem sh, double *berr, int *iters) {
    constexpr bool low = sizeof(T) != sizeof(double);
    double *scale = sh.scale<NT>();
    int steps = 0;
    double be = -1.0;
    if (!low) {
        copy_rhs<NT>(g, sm, false);
        trsv<T, NT>(g, sm, ws, kOnX, sh);
        steps = 1;
    } else {
        copy_rhs<NT>(g, sm, true);
    }
    if (sm.a) {
        for (int it = 0;; ++it) {
            // a low-precision solve starts from x = 0, whose residual is b itself
            if (low && it == 0) be = residual_of_zero<NT>(g, sm, sh);
            else be = residual<NT>(g, sm, sh.norm<NT>(), it == (low ? 1 : 0), sh);
            if (method == MTD_REFINE_NONE) break;
            if ((it > 0 || !low) && be <= tol) break;
            if (it >= max_iter) break;
            if constexpr (low) {
                scale_to_low<T, NT>(g, sm, scale, sh.red());
                trsv<T, NT>(g, sm, ws, kOnD, sh);
                add_scaled<T, NT>(g, sm, scale);
            } else {
                trsv<T, NT>(g, sm, ws, kOnR, sh);
                add_r<NT>(g, sm);
            }
            steps = it + 1 + (low ? 0 : 1);  // + the first FP64 solve
        }
    }
    *berr = be;
    *iters = steps;
}

}  // namespace bsolve
}  // namespace mtd
