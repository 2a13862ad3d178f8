// Batched factorisations and solves: many independent SPD matrices of different sizes
// run as ONE merged task graph on the persistent scheduler (one launch: graph-capturable),
// then solved with per-matrix triangular solves, in FP64 or in low precision with FP64
// iterative refinement.  No counterpart in the reference.
//
// Each matrix gets the reference's tiled Cholesky DAG for its own tile edge (chosen per
// size by the caller or by mtd_batch_autotune), lowered with nested diagonal
// factorisations, and the DAGs are concatenated with every task tagged by its matrix.  A
// bad pivot records LAPACK-style info for that matrix only; the rest of the batch runs on.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <map>
#include <new>
#include <vector>

#include "../../include/mustard_b200.h"
#include "dag.hpp"
#include "device_types.hpp"

namespace mtd {
int launch_run(const RunArgs &a, const int *deps_init, const int *roots, int n_roots, long long total_items,
               int prec, bool vec2, int grid, cudaStream_t s, bool adjoint);
}
using namespace mtd;

namespace {

constexpr int kSB = 64;        // solve block (= inverse block edge)
constexpr int kMaxRhs = 16;
constexpr int kBT = 256;       // threads of the batched solve kernels
constexpr int kInfoOk = 0x7f7f7f7f;  // per-matrix info sentinel (bytes 0x7f): no bad pivot

// Per-matrix arguments of the solve kernels.
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
    double *rowsum;   // n scratch for ||A||_inf
    int n, nrhs;
};

// One element copied global -> shared with cp.async (4 or 8 bytes, through L1: the solves
// read back blocks this CTA wrote); an invalid element is zero-filled (0 source bytes, the
// source address then only has to be a valid one).
template <typename T>
__device__ __forceinline__ void cp_elem(T *dst, const T *src, bool valid) {
    const uint32_t d = static_cast<uint32_t>(__cvta_generic_to_shared(dst));
    if constexpr (sizeof(T) == 8)
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(d), "l"(src), "r"(valid ? 8 : 0) : "memory");
    else
        asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(d), "l"(src), "r"(valid ? 4 : 0) : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

// Shared memory of the batched solve kernels: two 64 x 65 blocks, two nrhs x 64 vector
// blocks and (triangular solve) one nrhs x 64 accumulator.
template <typename T>
constexpr size_t trsv_smem() {
    return (2 * kSB * (kSB + 1) + 3 * kMaxRhs * kSB) * sizeof(T);
}
constexpr size_t residual_smem() { return (2 * kSB * (kSB + 1) + 2 * kMaxRhs * kSB) * sizeof(double); }

// Forward then backward substitution with L and the inverses of its 64 x 64 diagonal
// blocks, on the n x nrhs block Y (ld ldy), one CTA per matrix.  Block row j subtracts
// L(j, k) Y(k) for the rows k solved before it and applies the inverse of its diagonal
// block; the blocks it needs (L(j, k) with Y(k), then the inverse) stream through a
// two-deep cp.async ring, the next one in flight while the current product runs.  (The
// first version loaded every block element by element in dependent load / store loops:
// ~5 ms per launch for a batch of 4096 matrices of up to 1024.)
enum { kOnX = 0, kOnD = 1, kOnR = 2 };  // which block of SolveMat the solve overwrites

template <typename T>
__global__ void __launch_bounds__(kBT) batch_trsv_kernel(const SolveMat *mats, const T *ws, int target) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T *Lb = reinterpret_cast<T *>(smem_raw);  // 2 x [kSB][kSB + 1]
    T *Yb = Lb + 2 * kSB * (kSB + 1);         // 2 x [kMaxRhs][kSB]
    T *Acc = Yb + 2 * kMaxRhs * kSB;          // [kMaxRhs][kSB]
    const SolveMat &sm = mats[blockIdx.x];
    const int n = sm.n, nrhs = sm.nrhs, tid = threadIdx.x;
    const T *L = static_cast<const T *>(sm.f);
    const int64_t ldl = sm.ldf;
    const T *W = ws + sm.ws_off;
    const int64_t ldw = sm.ws_ld;
    T *Y = target == kOnX ? reinterpret_cast<T *>(sm.x)
                          : (target == kOnR ? reinterpret_cast<T *>(sm.r) : static_cast<T *>(sm.d));
    const int64_t ldy = target == kOnX ? sm.ldx : n;
    const int nb = (n + kSB - 1) / kSB;
    for (int pass = 0; pass < 2; ++pass) {
        const bool back = pass == 1;
        for (int s = 0; s < nb; ++s) {
            const int j = back ? nb - 1 - s : s;
            const int rj = min(kSB, n - j * kSB);
            // step t < s: L(j, k_t) (transposed in the backward pass) and Y(k_t); t = s: W_j
            auto issue = [&](int t) {
                T *Ld = Lb + (t & 1) * kSB * (kSB + 1);
                if (t < s) {
                    const int k = back ? nb - 1 - t : t;
                    const int rk = min(kSB, n - k * kSB);
                    for (int e = tid; e < kSB * kSB; e += kBT) {
                        const int a = e % kSB, c = e / kSB;
                        if (!back) {
                            const bool v = a < rj && c < rk;
                            cp_elem(Ld + a * (kSB + 1) + c, v ? L + (int64_t(j) * kSB + a) + (int64_t(k) * kSB + c) * ldl : L, v);
                        } else {
                            const bool v = a < rk && c < rj;
                            cp_elem(Ld + c * (kSB + 1) + a, v ? L + (int64_t(k) * kSB + a) + (int64_t(j) * kSB + c) * ldl : L, v);
                        }
                    }
                    T *Yd = Yb + (t & 1) * kMaxRhs * kSB;
                    for (int e = tid; e < kSB * nrhs; e += kBT) {
                        const int r = e % kSB, c = e / kSB;
                        cp_elem(Yd + c * kSB + r, r < rk ? Y + (int64_t(k) * kSB + r) + c * ldy : Y, r < rk);
                    }
                } else {
                    for (int e = tid; e < kSB * kSB; e += kBT) {
                        const int a = e % kSB, c = e / kSB;
                        const bool v = a < rj && c < rj;
                        cp_elem(back ? Ld + c * (kSB + 1) + a : Ld + a * (kSB + 1) + c,
                                v ? W + (int64_t(j) * kSB + a) + int64_t(c) * ldw : W, v);
                    }
                }
                cp_commit();
            };
            issue(0);
            for (int e = tid; e < kSB * nrhs; e += kBT) {
                const int r = e % kSB, c = e / kSB;
                Acc[c * kSB + r] = r < rj ? Y[(int64_t(j) * kSB + r) + c * ldy] : T(0);
            }
            for (int t = 0; t <= s; ++t) {
                cp_wait_all();
                __syncthreads();  // block t landed; every thread is done with the other buffer
                if (t + 1 <= s) issue(t + 1);
                const T *Lc = Lb + (t & 1) * kSB * (kSB + 1);
                if (t < s) {
                    const T *Yc = Yb + (t & 1) * kMaxRhs * kSB;
                    for (int o = tid; o < kSB * nrhs; o += kBT) {
                        const int r = o % kSB, c = o / kSB;
                        T acc = T(0);
#pragma unroll 8
                        for (int q = 0; q < kSB; ++q) acc += Lc[r * (kSB + 1) + q] * Yc[c * kSB + q];
                        Acc[c * kSB + r] -= acc;
                    }
                } else {
                    for (int o = tid; o < kSB * nrhs; o += kBT) {
                        const int r = o % kSB, c = o / kSB;
                        T acc = T(0);
#pragma unroll 8
                        for (int q = 0; q < kSB; ++q) acc += Lc[r * (kSB + 1) + q] * Acc[c * kSB + q];
                        if (r < rj) Y[(int64_t(j) * kSB + r) + c * ldy] = acc;
                    }
                }
            }
            __syncthreads();  // Y(j) stored before later rows read it; Acc and the ring are free
        }
    }
}

// r = b - A_sym x, then the matrix's normwise backward error (max over its columns) into
// berr[m]; one CTA per matrix.  A's infinity norm comes from anorm[m] (computed by
// batch_anorm_kernel).  Block row I of r is formed in registers over the whole symmetric
// block row (A(I, J) read from the lower triangle, transposed for J > I), the blocks of A
// and of x streaming through a two-deep cp.async ring; r(I) is written once.  (The first
// version read x from global memory inside its inner loop and accumulated the transposed
// contributions in global r: ~11 ms per launch for a batch of 4096 matrices of up to 1024.)
__global__ void __launch_bounds__(kBT) batch_residual_kernel(const SolveMat *mats, const double *anorm, double *berr) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double *Ab = reinterpret_cast<double *>(smem_raw);  // 2 x [kSB][kSB + 1]
    double *Xb = Ab + 2 * kSB * (kSB + 1);              // 2 x [kMaxRhs][kSB]
    __shared__ double red[3][kMaxRhs][kBT / 32];
    const SolveMat &sm = mats[blockIdx.x];
    const int n = sm.n, nrhs = sm.nrhs, tid = threadIdx.x;
    const double *A = sm.a;
    const int64_t lda = sm.lda;
    const int nb = (n + kSB - 1) / kSB;
    constexpr int kOut = kMaxRhs * kSB / kBT;  // outputs per thread: o = tid + kBT q
    static_assert(kMaxRhs * kSB % kBT == 0, "whole outputs per thread");
    for (int I = 0; I < nb; ++I) {
        const int ri = min(kSB, n - I * kSB);
        auto issue = [&](int J) {
            double *Ad = Ab + (J & 1) * kSB * (kSB + 1);
            const int cj = min(kSB, n - J * kSB);
            if (J < I) {  // A(I, J) straight from the lower triangle
                for (int e = tid; e < kSB * kSB; e += kBT) {
                    const int r = e % kSB, c = e / kSB;
                    const bool v = r < ri && c < cj;
                    cp_elem(Ad + r * (kSB + 1) + c, v ? A + (int64_t(I) * kSB + r) + (int64_t(J) * kSB + c) * lda : A, v);
                }
            } else if (J > I) {  // A(I, J) = A(J, I)^T
                for (int e = tid; e < kSB * kSB; e += kBT) {
                    const int c = e % kSB, r = e / kSB;
                    const bool v = r < ri && c < cj;
                    cp_elem(Ad + r * (kSB + 1) + c, v ? A + (int64_t(J) * kSB + c) + (int64_t(I) * kSB + r) * lda : A, v);
                }
            } else {  // diagonal block: the strict upper part mirrored from the lower one
                for (int e = tid; e < kSB * kSB; e += kBT) {
                    const int r = e % kSB, c = e / kSB;
                    const bool v = r < ri && c < cj;
                    const int64_t off = r >= c ? (int64_t(I) * kSB + r) + (int64_t(I) * kSB + c) * lda
                                               : (int64_t(I) * kSB + c) + (int64_t(I) * kSB + r) * lda;
                    cp_elem(Ad + r * (kSB + 1) + c, v ? A + off : A, v);
                }
            }
            double *Xd = Xb + (J & 1) * kMaxRhs * kSB;
            for (int e = tid; e < kSB * nrhs; e += kBT) {
                const int k = e % kSB, c = e / kSB;
                cp_elem(Xd + c * kSB + k, k < cj ? sm.x + (int64_t(J) * kSB + k) + c * sm.ldx : sm.x, k < cj);
            }
            cp_commit();
        };
        double acc[kOut];
#pragma unroll
        for (int q = 0; q < kOut; ++q) acc[q] = 0.0;
        issue(0);
        for (int J = 0; J < nb; ++J) {
            cp_wait_all();
            __syncthreads();  // block J landed; the other buffer is free
            if (J + 1 < nb) issue(J + 1);
            const double *Ac = Ab + (J & 1) * kSB * (kSB + 1);
            const double *Xc = Xb + (J & 1) * kMaxRhs * kSB;
#pragma unroll
            for (int q = 0; q < kOut; ++q) {
                const int o = tid + kBT * q, r = o % kSB, c = o / kSB;
                if (c < nrhs) {
                    double s = 0.0;
#pragma unroll 8
                    for (int k = 0; k < kSB; ++k) s += Ac[r * (kSB + 1) + k] * Xc[c * kSB + k];
                    acc[q] += s;
                }
            }
        }
#pragma unroll
        for (int q = 0; q < kOut; ++q) {
            const int o = tid + kBT * q, r = o % kSB, c = o / kSB;
            if (c < nrhs && r < ri)
                sm.r[(int64_t(I) * kSB + r) + int64_t(c) * n] = sm.b[(int64_t(I) * kSB + r) + c * sm.ldb] - acc[q];
        }
        __syncthreads();  // the ring is free for the next block row
    }
    __syncthreads();
    // column maxima of |r|, |x|, |b|
    for (int c = 0; c < nrhs; ++c) {
        double mr = 0.0, mx = 0.0, mb = 0.0;
        for (int i = tid; i < n; i += kBT) {
            mr = fmax(mr, fabs(sm.r[i + int64_t(c) * n]));
            mx = fmax(mx, fabs(sm.x[i + int64_t(c) * sm.ldx]));
            mb = fmax(mb, fabs(sm.b[i + int64_t(c) * sm.ldb]));
        }
        for (int o = 16; o > 0; o >>= 1) {
            mr = fmax(mr, __shfl_xor_sync(0xffffffffu, mr, o));
            mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
            mb = fmax(mb, __shfl_xor_sync(0xffffffffu, mb, o));
        }
        if ((tid & 31) == 0) {
            red[0][c][tid >> 5] = mr;
            red[1][c][tid >> 5] = mx;
            red[2][c][tid >> 5] = mb;
        }
    }
    __syncthreads();
    if (tid == 0) {
        double worst = 0.0;
        for (int c = 0; c < nrhs; ++c) {
            double mr = 0.0, mx = 0.0, mb = 0.0;
            for (int w = 0; w < kBT / 32; ++w) {
                mr = fmax(mr, red[0][c][w]);
                mx = fmax(mx, red[1][c][w]);
                mb = fmax(mb, red[2][c][w]);
            }
            const double den = anorm[blockIdx.x] * mx + mb;
            worst = fmax(worst, den > 0 ? mr / den : mr);
        }
        berr[blockIdx.x] = worst;
    }
}

// ||A_sym||_inf per matrix (max row sum of |A| over the full symmetric matrix).
__global__ void __launch_bounds__(kBT) batch_anorm_kernel(const SolveMat *mats, double *anorm) {
    __shared__ double red[kBT / 32];
    const SolveMat &sm = mats[blockIdx.x];
    const int n = sm.n, tid = threadIdx.x;
    double best = 0.0;
    for (int i = tid; i < n; i += kBT) {
        double s = 0.0;
        for (int j = 0; j <= i; ++j) s += fabs(sm.a[i + int64_t(j) * sm.lda]);  // row i, lower part
        for (int j = i + 1; j < n; ++j) s += fabs(sm.a[j + int64_t(i) * sm.lda]);  // column i below
        best = fmax(best, s);
    }
    for (int o = 16; o > 0; o >>= 1) best = fmax(best, __shfl_xor_sync(0xffffffffu, best, o));
    if ((tid & 31) == 0) red[tid >> 5] = best;
    __syncthreads();
    if (tid == 0) {
        double m = 0.0;
        for (int w = 0; w < kBT / 32; ++w) m = fmax(m, red[w]);
        anorm[blockIdx.x] = m;
    }
}

// d = r / max|r| per column (rounded to T), or x += max|r| * d; one CTA per matrix.
template <typename T>
__global__ void __launch_bounds__(kBT) batch_scale_kernel(const SolveMat *mats, double *colscale, bool to_low) {
    __shared__ double red[kBT / 32];
    const SolveMat &sm = mats[blockIdx.x];
    const int n = sm.n, tid = threadIdx.x;
    double *scale = colscale + int64_t(blockIdx.x) * kMaxRhs;
    T *d = static_cast<T *>(sm.d);
    for (int c = 0; c < sm.nrhs; ++c) {
        if (to_low) {
            double m = 0.0;
            for (int i = tid; i < n; i += kBT) m = fmax(m, fabs(sm.r[i + int64_t(c) * n]));
            for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
            __syncthreads();
            if ((tid & 31) == 0) red[tid >> 5] = m;
            __syncthreads();
            double s = 0.0;
            for (int w = 0; w < kBT / 32; ++w) s = fmax(s, red[w]);
            if (s == 0.0) s = 1.0;
            if (tid == 0) scale[c] = s;
            for (int i = tid; i < n; i += kBT) d[i + int64_t(c) * n] = static_cast<T>(sm.r[i + int64_t(c) * n] / s);
        } else {
            const double s = scale[c];
            for (int i = tid; i < n; i += kBT) sm.x[i + int64_t(c) * sm.ldx] += s * static_cast<double>(d[i + int64_t(c) * n]);
        }
    }
}

// x += r (FP64 correction), one CTA per matrix.
__global__ void batch_add_kernel(const SolveMat *mats) {
    const SolveMat &sm = mats[blockIdx.x];
    for (int64_t e = threadIdx.x; e < int64_t(sm.n) * sm.nrhs; e += blockDim.x) {
        const int64_t i = e % sm.n, c = e / sm.n;
        sm.x[i + c * sm.ldx] += sm.r[i + c * sm.n];
    }
}

// X = B (columns), one CTA per matrix.
__global__ void batch_copy_rhs_kernel(const SolveMat *mats, bool zero) {
    const SolveMat &sm = mats[blockIdx.x];
    for (int64_t e = threadIdx.x; e < int64_t(sm.n) * sm.nrhs; e += blockDim.x) {
        const int64_t i = e % sm.n, c = e / sm.n;
        sm.x[i + c * sm.ldx] = zero ? 0.0 : sm.b[i + c * sm.ldb];
    }
}

// dst = lower triangle of src (+ shift on the diagonal), as float; grid (chunks, count).
__global__ void batch_convert_kernel(const SolveMat *mats, double shift) {
    const SolveMat &sm = mats[blockIdx.y];
    const int64_t n = sm.n, total = n * n;
    float *f = static_cast<float *>(const_cast<void *>(sm.f));
    for (int64_t e = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; e < total; e += int64_t(gridDim.x) * blockDim.x) {
        const int64_t i = e % n, j = e / n;
        if (i < j) continue;
        double v = sm.a[i + j * sm.lda];
        if (i == j) v += shift;
        f[i + j * sm.ldf] = static_cast<float>(v);
    }
}

template <typename T>
int dalloc(T **p, size_t count) {
    if (cudaMalloc(reinterpret_cast<void **>(p), std::max<size_t>(count, 1) * sizeof(T)) != cudaSuccess) {
        cudaGetLastError();
        *p = nullptr;
        return MTD_ERR_OUT_OF_MEMORY;
    }
    return MTD_OK;
}

}  // namespace

struct mtd_batch {
    int count = 0;
    int prec = MTD_PREC_FP64;
    int sms = 148;
    std::vector<int64_t> n, tile, ws_off, ws_ld, rhs_off;
    std::vector<int> nest;
    int n_dev = 0, n_roots = 0;
    long long total_items = 0;
    long long qcap[kNumQueues] = {0, 0};
    DevTask *d_tasks = nullptr;
    int *d_succ = nullptr, *d_deps_init = nullptr, *d_deps = nullptr, *d_items_left = nullptr, *d_roots = nullptr;
    unsigned long long *d_queue[kNumQueues] = {nullptr, nullptr};
    QueueCtl *d_qctl = nullptr;
    RunCtl *d_ctl = nullptr;
    RunCtl *h_ctl = nullptr;       // pinned
    unsigned char *d_ws = nullptr;
    BatchMat *d_mats = nullptr;
    BatchMat *h_mats = nullptr;    // pinned staging of the per-run table
    int *d_info = nullptr;
    unsigned long long *d_done = nullptr;
    cudaStream_t last_stream = nullptr;
    bool pending = false;
    // solve state
    SolveMat *d_solve = nullptr, *h_solve = nullptr;  // pinned staging
    double *d_r = nullptr, *d_rowsum = nullptr, *d_anorm = nullptr, *d_berr = nullptr, *d_scale = nullptr;
    double *h_berr = nullptr;      // pinned
    void *d_low = nullptr;
    int64_t rhs_total = 0;
};

namespace {

size_t batch_elem(const mtd_batch *b) { return b->prec == MTD_PREC_FP64 ? sizeof(double) : sizeof(float); }

void release(mtd_batch *b) {
    cudaFree(b->d_tasks);
    cudaFree(b->d_succ);
    cudaFree(b->d_deps_init);
    cudaFree(b->d_deps);
    cudaFree(b->d_items_left);
    cudaFree(b->d_roots);
    for (int q = 0; q < kNumQueues; ++q) cudaFree(b->d_queue[q]);
    cudaFree(b->d_qctl);
    cudaFree(b->d_ctl);
    if (b->h_ctl) cudaFreeHost(b->h_ctl);
    cudaFree(b->d_ws);
    cudaFree(b->d_mats);
    if (b->h_mats) cudaFreeHost(b->h_mats);
    cudaFree(b->d_info);
    cudaFree(b->d_done);
    cudaFree(b->d_solve);
    if (b->h_solve) cudaFreeHost(b->h_solve);
    cudaFree(b->d_r);
    cudaFree(b->d_rowsum);
    cudaFree(b->d_anorm);
    cudaFree(b->d_berr);
    cudaFree(b->d_scale);
    if (b->h_berr) cudaFreeHost(b->h_berr);
    cudaFree(b->d_low);
}

// Default tile for a size when the caller gives none: one tile up to 512 (its diagonal
// factorisation nested at 128), 512-wide tiles above.
int64_t default_tile(int64_t n) { return n <= 512 ? n : 512; }

}  // namespace

extern "C" {

int mtd_batch_create(mtd_batch **out, int count, const int64_t *n, const int64_t *tile, const int *nest, int prec) {
    if (!out) return MTD_ERR_INVALID_ARG;
    *out = nullptr;
    if (count <= 0 || !n || (prec != MTD_PREC_FP64 && prec != MTD_PREC_TF32 && prec != MTD_PREC_FP32))
        return MTD_ERR_INVALID_ARG;
    mtd_batch *b = new (std::nothrow) mtd_batch();
    if (!b) return MTD_ERR_OUT_OF_MEMORY;
    b->count = count;
    b->prec = prec;
    int dev = 0;
    cudaGetDevice(&dev);
    int major = 0;
    cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev);
    if (major != 10) {
        delete b;
        return MTD_ERR_NO_DEVICE;
    }
    cudaDeviceGetAttribute(&b->sms, cudaDevAttrMultiProcessorCount, dev);

    std::vector<DevTask> tasks;
    std::vector<int> succ, deps_init, roots;
    int64_t ws_total = 0, rhs_total = 0;
    int rc = MTD_OK;
    for (int m = 0; m < count && !rc; ++m) {
        const int64_t nm = n[m];
        const int64_t tm = tile ? tile[m] : default_tile(nm);
        const int km = nest ? nest[m] : (nm > kNestTile ? kNestTile : 0);
        if (nm <= 0 || nm > (int64_t(1) << 20) || tm <= 0 || tm > nm || (tm != nm && tm % kSB != 0) || km < 0 ||
            km % kSB != 0) {
            rc = MTD_ERR_INVALID_ARG;
            break;
        }
        b->n.push_back(nm);
        b->tile.push_back(tm);
        b->nest.push_back(km);
        Dag dag(MTD_KIND_CHOLESKY, nm, tm);
        rc = dag.build_reference_order();
        Lowered low;
        if (!rc) rc = dag.lower(km, low);
        if (rc) break;
        const int base = static_cast<int>(tasks.size());
        const int sbase = static_cast<int>(succ.size());
        for (size_t t = 0; t < low.tasks.size(); ++t) {
            DevTask d = low.tasks[t];
            d.mat = m;
            d.succ_begin += sbase;
            tasks.push_back(d);
            deps_init.push_back(static_cast<int>(low.preds[t].size()));
            if (low.preds[t].empty()) roots.push_back(base + static_cast<int>(t));
        }
        for (int s : low.succ) succ.push_back(s + base);
        for (int q = 0; q < kNumQueues; ++q) b->qcap[q] += low.queue_cap[q];
        const int64_t wld = (nm + 3) & ~int64_t(3);
        b->ws_off.push_back(ws_total);
        b->ws_ld.push_back(wld);
        ws_total += wld * kSB;
        b->rhs_off.push_back(rhs_total);
        rhs_total += nm * kMaxRhs;
    }
    if (!rc && roots.empty()) rc = MTD_ERR_BAD_DAG;
    b->n_dev = static_cast<int>(tasks.size());
    b->n_roots = static_cast<int>(roots.size());
    b->total_items = b->qcap[0] + b->qcap[1];
    b->rhs_total = rhs_total;
    const int nt = b->n_dev;
    if (!rc) rc = dalloc(&b->d_tasks, nt);
    if (!rc) rc = dalloc(&b->d_succ, succ.size());
    if (!rc) rc = dalloc(&b->d_deps_init, nt);
    if (!rc) rc = dalloc(&b->d_deps, nt);
    if (!rc) rc = dalloc(&b->d_items_left, nt);
    if (!rc) rc = dalloc(&b->d_roots, roots.size());
    for (int q = 0; q < kNumQueues && !rc; ++q) rc = dalloc(&b->d_queue[q], size_t(b->qcap[q]));
    if (!rc) rc = dalloc(&b->d_qctl, kNumQueues);
    if (!rc) rc = dalloc(&b->d_ctl, 1);
    if (!rc) rc = dalloc(&b->d_ws, size_t(ws_total) * batch_elem(b));
    if (!rc) rc = dalloc(&b->d_mats, count);
    if (!rc) rc = dalloc(&b->d_info, count);
    if (!rc) rc = dalloc(&b->d_done, count);
    if (!rc && cudaMallocHost(reinterpret_cast<void **>(&b->h_ctl), sizeof(RunCtl)) != cudaSuccess) rc = MTD_ERR_OUT_OF_MEMORY;
    if (!rc && cudaMallocHost(reinterpret_cast<void **>(&b->h_mats), count * sizeof(BatchMat)) != cudaSuccess)
        rc = MTD_ERR_OUT_OF_MEMORY;
    if (!rc) {
        bool ok = cudaMemcpy(b->d_tasks, tasks.data(), nt * sizeof(DevTask), cudaMemcpyHostToDevice) == cudaSuccess;
        ok = ok && (succ.empty() ||
                    cudaMemcpy(b->d_succ, succ.data(), succ.size() * sizeof(int), cudaMemcpyHostToDevice) == cudaSuccess);
        ok = ok && cudaMemcpy(b->d_deps_init, deps_init.data(), nt * sizeof(int), cudaMemcpyHostToDevice) == cudaSuccess;
        ok = ok && cudaMemcpy(b->d_roots, roots.data(), roots.size() * sizeof(int), cudaMemcpyHostToDevice) == cudaSuccess;
        ok = ok && cudaMemset(b->d_ctl, 0, sizeof(RunCtl)) == cudaSuccess;
        if (!ok) rc = MTD_ERR_CUDA;
    }
    if (rc) {
        release(b);
        delete b;
        return rc;
    }
    std::memset(b->h_ctl, 0, sizeof(RunCtl));
    *out = b;
    return MTD_OK;
}

int mtd_batch_num_tasks(const mtd_batch *b) { return b ? b->n_dev : -MTD_ERR_INVALID_ARG; }

int mtd_batch_factor(mtd_batch *b, void *const *dA, const int64_t *lda, void *stream) {
    if (!b || !dA || !lda) return MTD_ERR_INVALID_ARG;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const int64_t epc = 16 / static_cast<int64_t>(batch_elem(b));
    bool vec2 = true;
    for (int m = 0; m < b->count; ++m) {
        if (!dA[m] || lda[m] < b->n[m]) return MTD_ERR_INVALID_ARG;
        b->h_mats[m] = BatchMat{dA[m], lda[m], b->ws_off[m], b->ws_ld[m]};
        vec2 = vec2 && reinterpret_cast<uintptr_t>(dA[m]) % 16 == 0 && lda[m] % epc == 0 && b->n[m] % epc == 0 &&
               b->tile[m] % epc == 0;
    }
    if (cudaMemcpyAsync(b->d_mats, b->h_mats, b->count * sizeof(BatchMat), cudaMemcpyHostToDevice, s) != cudaSuccess ||
        cudaMemsetAsync(b->d_info, 0x7f, b->count * sizeof(int), s) != cudaSuccess ||
        cudaMemsetAsync(b->d_done, 0, b->count * sizeof(unsigned long long), s) != cudaSuccess)
        return MTD_ERR_CUDA;
    RunArgs a{};
    a.n_tasks = b->n_dev;
    a.tasks = b->d_tasks;
    a.succ = b->d_succ;
    a.deps = b->d_deps;
    a.items_left = b->d_items_left;
    for (int q = 0; q < kNumQueues; ++q) {
        a.queue[q] = b->d_queue[q];
        a.queue_cap[q] = b->qcap[q];
    }
    a.qctl = b->d_qctl;
    a.ctl = b->d_ctl;
    a.ws_lower = b->d_ws;
    a.ws_upper = nullptr;
    a.timeout_ns = 10ull * 1000000000ull;
    a.mats = b->d_mats;
    a.mat_info = b->d_info;
    a.mat_done_ns = b->d_done;
    int rc = launch_run(a, b->d_deps_init, b->d_roots, b->n_roots, b->total_items, b->prec, vec2, b->sms, s, false);
    if (rc) return rc;
    if (cudaMemcpyAsync(b->h_ctl, b->d_ctl, sizeof(RunCtl), cudaMemcpyDeviceToHost, s) != cudaSuccess) return MTD_ERR_CUDA;
    b->last_stream = s;
    b->pending = true;
    return MTD_OK;
}

int mtd_batch_status(mtd_batch *b, int *info, double *latency_ms) {
    if (!b) return MTD_ERR_INVALID_ARG;
    if (!b->pending) return MTD_ERR_STATE;
    if (cudaStreamSynchronize(b->last_stream) != cudaSuccess) return MTD_ERR_CUDA;
    if (info) {
        if (cudaMemcpy(info, b->d_info, b->count * sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess) return MTD_ERR_CUDA;
        for (int m = 0; m < b->count; ++m)
            if (info[m] == kInfoOk) info[m] = 0;
    }
    if (latency_ms) {
        std::vector<unsigned long long> done(b->count);
        if (cudaMemcpy(done.data(), b->d_done, b->count * sizeof(unsigned long long), cudaMemcpyDeviceToHost) !=
            cudaSuccess)
            return MTD_ERR_CUDA;
        for (int m = 0; m < b->count; ++m)
            latency_ms[m] = done[m] > b->h_ctl->start_ns ? double(done[m] - b->h_ctl->start_ns) * 1e-6 : -1.0;
    }
    if (b->h_ctl->error) return b->h_ctl->error;
    if (b->h_ctl->tasks_done != b->n_dev) return MTD_ERR_TIMEOUT;
    return MTD_OK;
}

int mtd_batch_solve(mtd_batch *b, const double *const *dA, const int64_t *lda, void *const *dF, const int64_t *ldf,
                    const double *const *dB, const int64_t *ldb, double *const *dX, const int64_t *ldx,
                    const int *nrhs, int method, double tol, int max_iter, void *stream, mtd_batch_solve_stats *stats) {
    if (!b || !dF || !ldf || !dB || !ldb || !dX || !ldx || !nrhs || max_iter < 0) return MTD_ERR_INVALID_ARG;
    if (method != MTD_REFINE_NONE && method != MTD_REFINE_IR) return MTD_ERR_INVALID_ARG;
    const bool low = b->prec != MTD_PREC_FP64;
    if ((method == MTD_REFINE_IR || low) && (!dA || !lda)) return MTD_ERR_INVALID_ARG;
    if (low && method == MTD_REFINE_NONE) return MTD_ERR_INVALID_ARG;  // a low-precision factor needs refinement
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const int count = b->count;
    int rc = MTD_OK;
    if (!b->h_berr) {
        if (!b->h_solve && cudaMallocHost(reinterpret_cast<void **>(&b->h_solve), count * sizeof(SolveMat)) != cudaSuccess)
            return MTD_ERR_OUT_OF_MEMORY;
        if (cudaMallocHost(reinterpret_cast<void **>(&b->h_berr), count * sizeof(double)) != cudaSuccess)
            return MTD_ERR_OUT_OF_MEMORY;
        if (!b->d_solve) rc = dalloc(&b->d_solve, count);
        if (!rc) rc = dalloc(&b->d_r, size_t(b->rhs_total));
        if (!rc) rc = dalloc(&b->d_anorm, count);
        if (!rc) rc = dalloc(&b->d_berr, count);
        if (!rc) rc = dalloc(&b->d_scale, size_t(count) * kMaxRhs);
        if (!rc && cudaMalloc(&b->d_low, size_t(b->rhs_total) * sizeof(float)) != cudaSuccess) rc = MTD_ERR_OUT_OF_MEMORY;
        if (rc) return rc;
    }
    for (int m = 0; m < count; ++m) {
        if (nrhs[m] < 1 || nrhs[m] > kMaxRhs || ldb[m] < b->n[m] || ldx[m] < b->n[m] || ldf[m] < b->n[m])
            return MTD_ERR_INVALID_ARG;
        if (dA && lda[m] < b->n[m]) return MTD_ERR_INVALID_ARG;
        SolveMat &sm = b->h_solve[m];
        sm.a = dA ? dA[m] : nullptr;
        sm.lda = dA ? lda[m] : 0;
        sm.f = dF[m];
        sm.ldf = ldf[m];
        sm.ws_off = b->ws_off[m];
        sm.ws_ld = b->ws_ld[m];
        sm.b = dB[m];
        sm.ldb = ldb[m];
        sm.x = dX[m];
        sm.ldx = ldx[m];
        sm.r = b->d_r + b->rhs_off[m];
        sm.d = static_cast<float *>(b->d_low) + b->rhs_off[m];
        sm.rowsum = nullptr;
        sm.n = static_cast<int>(b->n[m]);
        sm.nrhs = nrhs[m];
    }
    const auto t0 = std::chrono::steady_clock::now();
    if (cudaMemcpyAsync(b->d_solve, b->h_solve, count * sizeof(SolveMat), cudaMemcpyHostToDevice, s) != cudaSuccess)
        return MTD_ERR_CUDA;
    const size_t smem64 = trsv_smem<double>(), smem32 = trsv_smem<float>(), smem_res = residual_smem();
    if (cudaFuncSetAttribute(batch_trsv_kernel<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem64)) !=
            cudaSuccess ||
        cudaFuncSetAttribute(batch_trsv_kernel<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem32)) !=
            cudaSuccess ||
        cudaFuncSetAttribute(batch_residual_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem_res)) !=
            cudaSuccess)
        return MTD_ERR_CUDA;
    const double *ws64 = reinterpret_cast<const double *>(b->d_ws);
    const float *ws32 = reinterpret_cast<const float *>(b->d_ws);
    mtd_batch_solve_stats st{};
    double worst = -1.0;
    if (!low) {  // one FP64 solve: x = (L L^T)^-1 b
        batch_copy_rhs_kernel<<<count, kBT, 0, s>>>(b->d_solve, false);
        batch_trsv_kernel<double><<<count, kBT, smem64, s>>>(b->d_solve, ws64, kOnX);
        st.iterations = 1;
    } else {
        batch_copy_rhs_kernel<<<count, kBT, 0, s>>>(b->d_solve, true);  // x = 0
    }
    if (dA) {
        batch_anorm_kernel<<<count, kBT, 0, s>>>(b->d_solve, b->d_anorm);
        for (int it = 0;; ++it) {
            batch_residual_kernel<<<count, kBT, smem_res, s>>>(b->d_solve, b->d_anorm, b->d_berr);
            if (cudaMemcpyAsync(b->h_berr, b->d_berr, count * sizeof(double), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
                cudaStreamSynchronize(s) != cudaSuccess)
                return MTD_ERR_CUDA;
            worst = 0.0;
            int done = 0;
            for (int m = 0; m < count; ++m) {
                worst = std::max(worst, b->h_berr[m]);
                done += b->h_berr[m] <= tol;
            }
            st.converged_count = done;
            if (method == MTD_REFINE_NONE) break;
            if ((it > 0 || !low) && done == count) break;
            if (it >= max_iter) break;
            if (low) {  // x += M^-1 r through the low-precision factor
                batch_scale_kernel<float><<<count, kBT, 0, s>>>(b->d_solve, b->d_scale, true);
                batch_trsv_kernel<float><<<count, kBT, smem32, s>>>(b->d_solve, ws32, kOnD);
                batch_scale_kernel<float><<<count, kBT, 0, s>>>(b->d_solve, b->d_scale, false);
            } else {    // x += (L L^T)^-1 r in FP64
                batch_trsv_kernel<double><<<count, kBT, smem64, s>>>(b->d_solve, ws64, kOnR);
                batch_add_kernel<<<count, kBT, 0, s>>>(b->d_solve);
            }
            st.iterations = it + 1;
        }
    }
    if (cudaStreamSynchronize(s) != cudaSuccess || cudaGetLastError() != cudaSuccess) return MTD_ERR_CUDA;
    st.max_backward_error = worst;
    st.solve_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    if (stats) *stats = st;
    return rc;
}

int mtd_batch_convert(mtd_batch *b, const double *const *dA, const int64_t *lda, void *const *dF, const int64_t *ldf,
                      double shift, void *stream) {
    if (!b || !dA || !lda || !dF || !ldf || b->prec == MTD_PREC_FP64) return MTD_ERR_INVALID_ARG;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (!b->h_solve) {
        if (cudaMallocHost(reinterpret_cast<void **>(&b->h_solve), b->count * sizeof(SolveMat)) != cudaSuccess)
            return MTD_ERR_OUT_OF_MEMORY;
        if (dalloc(&b->d_solve, b->count)) return MTD_ERR_OUT_OF_MEMORY;
    }
    for (int m = 0; m < b->count; ++m) {
        if (lda[m] < b->n[m] || ldf[m] < b->n[m]) return MTD_ERR_INVALID_ARG;
        SolveMat sm{};
        sm.a = dA[m];
        sm.lda = lda[m];
        sm.f = dF[m];
        sm.ldf = ldf[m];
        sm.n = static_cast<int>(b->n[m]);
        b->h_solve[m] = sm;
    }
    if (cudaMemcpyAsync(b->d_solve, b->h_solve, b->count * sizeof(SolveMat), cudaMemcpyHostToDevice, s) != cudaSuccess)
        return MTD_ERR_CUDA;
    batch_convert_kernel<<<dim3(16, b->count), 256, 0, s>>>(b->d_solve, shift);
    // the staging buffer is reused by the next call: wait until the copy has been consumed
    if (cudaStreamSynchronize(s) != cudaSuccess) return MTD_ERR_CUDA;
    return cudaGetLastError() == cudaSuccess ? MTD_OK : MTD_ERR_CUDA;
}

int mtd_batch_destroy(mtd_batch *b) {
    if (!b) return MTD_ERR_INVALID_ARG;
    if (b->pending && b->last_stream) cudaStreamSynchronize(b->last_stream);
    cudaDeviceSynchronize();
    release(b);
    delete b;
    return MTD_OK;
}

}  // extern "C"

namespace {

__global__ void to_float_kernel(const double *x, float *y, int64_t count) {
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < count; i += int64_t(gridDim.x) * blockDim.x)
        y[i] = static_cast<float>(x[i]);
}

// Trial settings for matrices of size n: one tile (tile = n), or tiles of 128 .. 512
// elements; each with no nesting or with 64- / 128-element nested diagonal factorisations.
std::vector<std::pair<int64_t, int>> tune_candidates(int64_t n) {
    std::vector<int64_t> tiles{n};
    for (int64_t t : {128, 256, 384, 512})
        if (t < n) tiles.push_back(t);
    std::vector<std::pair<int64_t, int>> out;
    for (int64_t t : tiles) {
        out.push_back({t, 0});
        for (int nest : {64, 128})
            if (nest < t) out.push_back({t, nest});
    }
    return out;
}

}  // namespace

extern "C" {

int mtd_batch_autotune(int count, const int64_t *n, int prec, int64_t *tile_out, int *nest_out, double *trial_ms,
                       void *stream) {
    if (count <= 0 || !n || !tile_out || !nest_out ||
        (prec != MTD_PREC_FP64 && prec != MTD_PREC_TF32 && prec != MTD_PREC_FP32))
        return MTD_ERR_INVALID_ARG;
    for (int m = 0; m < count; ++m)
        if (n[m] <= 0 || n[m] > (int64_t(1) << 20)) return MTD_ERR_INVALID_ARG;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const auto t0 = std::chrono::steady_clock::now();
    std::map<int64_t, int> per_size;
    for (int m = 0; m < count; ++m) ++per_size[n[m]];
    const size_t es = prec == MTD_PREC_FP64 ? sizeof(double) : sizeof(float);
    std::map<int64_t, std::pair<int64_t, int>> choice;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) return MTD_ERR_CUDA;
    int rc = MTD_OK;
    for (const auto &kv : per_size) {
        if (rc) break;
        const int64_t sz = kv.first;
        // a trial batch as large as this size's share of the batch (so the trial sees the
        // parallelism the real batch offers), capped at ~2^38 / 3 flop so it stays milliseconds
        const int k = std::max(1, std::min(kv.second, static_cast<int>(std::max<int64_t>(4, (int64_t(1) << 38) /
                                                                                         (sz * sz * sz)))));
        const size_t elems = size_t(k) * size_t(sz) * size_t(sz);
        double *src = nullptr;
        void *work = nullptr;
        float *src32 = nullptr;
        if (dalloc(&src, elems) || cudaMalloc(&work, std::max<size_t>(elems * es, 1)) != cudaSuccess ||
            (prec != MTD_PREC_FP64 && dalloc(&src32, elems))) {
            cudaFree(src);
            cudaFree(work);
            rc = MTD_ERR_OUT_OF_MEMORY;
            break;
        }
        for (int i = 0; i < k && !rc; ++i)
            rc = mtd_generate(src + size_t(i) * sz * sz, sz, sz, MTD_GEN_SPD, 0x5eed + uint64_t(i), 1.0, s);
        if (!rc && src32) to_float_kernel<<<1024, 256, 0, s>>>(src, src32, static_cast<int64_t>(elems));
        const void *pristine = src32 ? static_cast<const void *>(src32) : static_cast<const void *>(src);
        std::vector<void *> ptrs(k);
        std::vector<int64_t> lds(k, sz), sizes(k, sz), tiles(k);
        std::vector<int> nests(k);
        for (int i = 0; i < k; ++i) ptrs[i] = static_cast<unsigned char *>(work) + size_t(i) * sz * sz * es;
        double best_ms = 1e300;
        std::pair<int64_t, int> best{std::min<int64_t>(sz, 512), sz > kNestTile ? kNestTile : 0};
        for (const auto &cand : tune_candidates(sz)) {
            if (rc) break;
            std::fill(tiles.begin(), tiles.end(), cand.first);
            std::fill(nests.begin(), nests.end(), cand.second);
            mtd_batch *b = nullptr;
            rc = mtd_batch_create(&b, k, sizes.data(), tiles.data(), nests.data(), prec);
            if (rc) break;
            double ms_min = 1e300;
            for (int rep = 0; rep < 2 && !rc; ++rep) {  // the first run warms up
                if (cudaMemcpyAsync(work, pristine, elems * es, cudaMemcpyDeviceToDevice, s) != cudaSuccess ||
                    cudaEventRecord(e0, s) != cudaSuccess) {
                    rc = MTD_ERR_CUDA;
                    break;
                }
                rc = mtd_batch_factor(b, ptrs.data(), lds.data(), s);
                if (!rc && cudaEventRecord(e1, s) != cudaSuccess) rc = MTD_ERR_CUDA;
                if (!rc) rc = mtd_batch_status(b, nullptr, nullptr);
                float ms = 0.f;
                if (!rc && cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess) rc = MTD_ERR_CUDA;
                if (!rc && rep > 0) ms_min = std::min(ms_min, double(ms));
            }
            mtd_batch_destroy(b);
            if (!rc && ms_min < best_ms) {
                best_ms = ms_min;
                best = cand;
            }
        }
        choice[sz] = best;
        cudaFree(src);
        cudaFree(work);
        cudaFree(src32);
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc) return rc;
    for (int m = 0; m < count; ++m) {
        tile_out[m] = choice[n[m]].first;
        nest_out[m] = choice[n[m]].second;
    }
    if (trial_ms) *trial_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    return MTD_OK;
}

}  // extern "C"
