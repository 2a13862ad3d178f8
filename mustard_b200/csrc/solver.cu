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

__device__ __forceinline__ double ldcg(const double *p) { return __ldcg(p); }
__device__ __forceinline__ float ldcg(const float *p) { return __ldcg(p); }

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

// ---- FP64 symmetric block product: Y += alpha * A_sym * X (A lower triangle) ------

// One 64 x 64 block (I >= J) of the lower triangle per CTA; the strictly lower blocks
// contribute to both block rows I and J.  ABS uses |A| (for the infinity norm).
template <bool ABS>
__global__ void __launch_bounds__(kSolveThreads) symm_lower_kernel(const double *A, int64_t lda, int64_t n,
                                                                   const double *X, int64_t ldx, double *Y,
                                                                   int64_t ldy, int nrhs, double alpha) {
    constexpr int kChunk = 8;  // right-hand sides staged per pass (static shared memory < 48 KB)
    __shared__ double As[kSB][kSB + 1];
    __shared__ double XI[kChunk][kSB];
    __shared__ double XJ[kChunk][kSB];
    const int64_t b = blockIdx.x;
    int64_t I = static_cast<int64_t>((sqrt(8.0 * double(b) + 1.0) - 1.0) / 2.0);
    while (I * (I + 1) / 2 > b) --I;
    while ((I + 1) * (I + 2) / 2 <= b) ++I;
    const int64_t J = b - I * (I + 1) / 2;
    const int64_t r0 = I * kSB, c0 = J * kSB;
    const int ri = static_cast<int>(n - r0 < kSB ? n - r0 : kSB);
    const int cj = static_cast<int>(n - c0 < kSB ? n - c0 : kSB);
    const int tid = threadIdx.x;
    for (int e = tid; e < kSB * kSB; e += kSolveThreads) {
        const int r = e % kSB, c = e / kSB;
        double v = 0.0;
        if (r < ri && c < cj) {
            if (I != J || r >= c) v = A[(r0 + r) + (c0 + c) * lda];
            else v = A[(c0 + c) + (r0 + r) * lda];  // mirror inside the diagonal block
        }
        As[r][c] = ABS ? fabs(v) : v;
    }
    for (int cb = 0; cb < nrhs; cb += kChunk) {
        const int nc = min(kChunk, nrhs - cb);
        __syncthreads();
        for (int e = tid; e < kSB * nc; e += kSolveThreads) {
            const int r = e % kSB, c = e / kSB;
            XJ[c][r] = r < cj ? X[(c0 + r) + (cb + c) * ldx] : 0.0;
            XI[c][r] = r < ri ? X[(r0 + r) + (cb + c) * ldx] : 0.0;
        }
        __syncthreads();
        for (int o = tid; o < kSB * nc; o += kSolveThreads) {
            const int r = o % kSB, c = o / kSB;
            if (r < ri) {
                double s = 0.0;
#pragma unroll 8
                for (int k = 0; k < kSB; ++k) s += As[r][k] * XJ[c][k];
                atomicAdd(Y + (r0 + r) + (cb + c) * ldy, alpha * s);
            }
            if (I != J && r < cj) {
                double s = 0.0;
#pragma unroll 8
                for (int k = 0; k < kSB; ++k) s += As[k][r] * XI[c][k];
                atomicAdd(Y + (c0 + r) + (cb + c) * ldy, alpha * s);
            }
        }
    }
}

// ---- wavefront triangular solves with the factor ---------------------------------

// X <- L^-1 X (forward) or L^-T X (backward), L lower with the inverses of its 64 x 64
// diagonal blocks in W.  One CTA per 64-row block; a CTA takes its block from a ticket
// counter, so every block it waits for belongs to a CTA that started earlier (no CTA ever
// waits on one that may not be resident).  Each wait is bounded; a CTA that gives up or
// sees the shared error word set records MTD_ERR_TIMEOUT and returns.
template <typename T, bool BACKWARD>
__global__ void __launch_bounds__(kSolveThreads) trsv_wavefront_kernel(
    const T *L, int64_t ldl, const T *W, int64_t ldw, int n, T *X, int64_t ldx, int nrhs, int *ticket,
    int *flags, int epoch, unsigned long long timeout_ns, int *err) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T *Ls = reinterpret_cast<T *>(smem_raw);       // [kSB][kSB + 1], Ls[r * (kSB+1) + q]
    T *Ys = Ls + kSB * (kSB + 1);                  // [kMaxRhs][kSB]
    T *Acc = Ys + kMaxRhs * kSB;                   // [kMaxRhs][kSB]
    __shared__ int s_b, s_abort;
    const int tid = threadIdx.x;
    const int nb = (n + kSB - 1) / kSB;
    if (tid == 0) {
        s_b = atomicAdd(ticket, 1);
        s_abort = 0;
    }
    __syncthreads();
    const int b = s_b;
    if (b >= nb) return;
    const int j = BACKWARD ? nb - 1 - b : b;
    const int rj = min(kSB, n - j * kSB);
    for (int e = tid; e < kSB * nrhs; e += kSolveThreads) {
        const int r = e % kSB, c = e / kSB;
        Acc[c * kSB + r] = r < rj ? X[(int64_t(j) * kSB + r) + c * ldx] : T(0);
    }
    const int kfirst = BACKWARD ? nb - 1 : 0;
    const int count = BACKWARD ? nb - 1 - j : j;
    const unsigned long long t0 = global_ns();
    for (int step = 0; step < count; ++step) {
        const int k = BACKWARD ? kfirst - step : step;
        const int rk = min(kSB, n - k * kSB);
        __syncthreads();
        // Block of L that couples j and k, stored so both directions read Ls[r][q] with
        // r = row of the output block: forward L(j, k); backward L(k, j)^T.
        for (int e = tid; e < kSB * kSB; e += kSolveThreads) {
            const int a = e % kSB, c = e / kSB;  // a runs down a column of L: coalesced
            if (!BACKWARD) {
                Ls[a * (kSB + 1) + c] = (a < rj && c < rk) ? L[(int64_t(j) * kSB + a) + (int64_t(k) * kSB + c) * ldl] : T(0);
            } else {
                Ls[c * (kSB + 1) + a] = (a < rk && c < rj) ? L[(int64_t(k) * kSB + a) + (int64_t(j) * kSB + c) * ldl] : T(0);
            }
        }
        if (tid == 0) {
            const volatile int *f = flags + k;
            const volatile int *ev = err;
            while (*f != epoch) {
                if (*ev != 0) {
                    s_abort = 1;
                    break;
                }
                if (global_ns() - t0 > timeout_ns) {
                    atomicCAS(err, 0, MTD_ERR_TIMEOUT);
                    s_abort = 1;
                    break;
                }
                __nanosleep(64);
            }
            __threadfence();
        }
        __syncthreads();
        if (s_abort) return;
        for (int e = tid; e < kSB * nrhs; e += kSolveThreads) {
            const int r = e % kSB, c = e / kSB;
            Ys[c * kSB + r] = r < rk ? ldcg(X + (int64_t(k) * kSB + r) + c * ldx) : T(0);
        }
        __syncthreads();
        for (int o = tid; o < kSB * nrhs; o += kSolveThreads) {
            const int r = o % kSB, c = o / kSB;
            T s = T(0);
#pragma unroll 8
            for (int q = 0; q < kSB; ++q) s += Ls[r * (kSB + 1) + q] * Ys[c * kSB + q];
            Acc[c * kSB + r] -= s;
        }
    }
    __syncthreads();
    // Diagonal block: forward y_j = W_j acc, backward x_j = W_j^T acc.
    for (int e = tid; e < kSB * kSB; e += kSolveThreads) {
        const int a = e % kSB, c = e / kSB;
        const T v = (a < rj && c < rj) ? W[(int64_t(j) * kSB + a) + int64_t(c) * ldw] : T(0);
        if (!BACKWARD) Ls[a * (kSB + 1) + c] = v;
        else Ls[c * (kSB + 1) + a] = v;
    }
    __syncthreads();
    for (int o = tid; o < kSB * nrhs; o += kSolveThreads) {
        const int r = o % kSB, c = o / kSB;
        T s = T(0);
#pragma unroll 8
        for (int q = 0; q < kSB; ++q) s += Ls[r * (kSB + 1) + q] * Acc[c * kSB + q];
        Ys[c * kSB + r] = s;
    }
    __syncthreads();
    for (int e = tid; e < kSB * nrhs; e += kSolveThreads) {
        const int r = e % kSB, c = e / kSB;
        if (r < rj) X[(int64_t(j) * kSB + r) + c * ldx] = Ys[c * kSB + r];
    }
    __threadfence();
    __syncthreads();
    if (tid == 0) atomicExch(flags + j, epoch);
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
    int *ticket = nullptr, *flags = nullptr, *err = nullptr;
    int epoch = 0;
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

int symm(mtd_solver *s, const double *X, int64_t ldx, double *Y, int64_t ldy, int nrhs, double alpha, bool abs,
         cudaStream_t st) {
    const int64_t nb = (s->n + kSB - 1) / kSB;
    const unsigned blocks = static_cast<unsigned>(nb * (nb + 1) / 2);
    if (abs) symm_lower_kernel<true><<<blocks, kSolveThreads, 0, st>>>(s->a, s->lda, s->n, X, ldx, Y, ldy, nrhs, alpha);
    else symm_lower_kernel<false><<<blocks, kSolveThreads, 0, st>>>(s->a, s->lda, s->n, X, ldx, Y, ldy, nrhs, alpha);
    return cudaGetLastError() == cudaSuccess ? MTD_OK : MTD_ERR_CUDA;
}

template <typename T>
int trsv_pair(mtd_solver *s, T *X, int64_t ldx, int nrhs, cudaStream_t st) {
    const int nb = static_cast<int>((s->n + kSB - 1) / kSB);
    const T *L = static_cast<const T *>(s->fac);
    const T *W = static_cast<const T *>(mtd::graph_ws_lower(s->g));
    const int64_t ldw = mtd::graph_ws_ld(s->g);
    const size_t smem = (kSB * (kSB + 1) + 2 * kMaxRhs * kSB) * sizeof(T);
    const unsigned long long timeout = 10ull * 1000000000ull;
    for (int pass = 0; pass < 2; ++pass) {
        if (cudaMemsetAsync(s->ticket, 0, sizeof(int), st) != cudaSuccess) return MTD_ERR_CUDA;
        ++s->epoch;
        if (pass == 0)
            trsv_wavefront_kernel<T, false><<<nb, kSolveThreads, smem, st>>>(L, s->ldf, W, ldw, static_cast<int>(s->n),
                                                                             X, ldx, nrhs, s->ticket, s->flags,
                                                                             s->epoch, timeout, s->err);
        else
            trsv_wavefront_kernel<T, true><<<nb, kSolveThreads, smem, st>>>(L, s->ldf, W, ldw, static_cast<int>(s->n),
                                                                            X, ldx, nrhs, s->ticket, s->flags,
                                                                            s->epoch, timeout, s->err);
        if (cudaGetLastError() != cudaSuccess) return MTD_ERR_CUDA;
    }
    return MTD_OK;
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
    cudaFree(s->flags);
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
    if (prec != MTD_PREC_FP64 && prec != MTD_PREC_TF32 && prec != MTD_PREC_FP32) return MTD_ERR_INVALID_ARG;
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
    if (!rc) rc = alloc(&s->flags, nb);
    if (!rc) rc = alloc(&s->err, 1);
    if (!rc) rc = alloc(&s->V, size_t(n) * (s->gm_restart + 1));
    if (!rc) rc = alloc(&s->w, size_t(n));
    if (!rc) rc = alloc(&s->hbuf, s->gm_restart + 2);
    if (!rc) {
        cudaMemset(s->flags, 0, nb * sizeof(int));
        cudaMemset(s->err, 0, sizeof(int));
        const size_t smem64 = (kSB * (kSB + 1) + 2 * kMaxRhs * kSB) * sizeof(double);
        if (cudaFuncSetAttribute(trsv_wavefront_kernel<double, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 int(smem64)) != cudaSuccess ||
            cudaFuncSetAttribute(trsv_wavefront_kernel<double, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 int(smem64)) != cudaSuccess)
            rc = MTD_ERR_CUDA;
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
            rc = backward_error(s, dX, ldx, dB, ldb, nr, st, &berr, nullptr);  // leaves r = b - A x in s->r
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
