// Tile operations of the pivoted LU (mtd_lupiv): LU with partial pivoting as LAPACK's dgetrf
// defines it (row interchanges chosen by the largest |a| of each column, the first such row
// on ties; ipiv 1-based).  No counterpart in the reference, which factors without pivoting
// (lu_mustard.cu:361-369 passes no pivot array to cusolverDnDgetrf).
//
// A panel (the m x w block column below and including the diagonal tile) is one task whose P
// work items each hold a slab of R consecutive panel rows in shared memory.  Every CTA of the
// persistent launch is resident, and P never exceeds their number, so the items run
// together: they exchange their column candidates through global memory and meet at one
// bounded device barrier per column.  The row interchanges of the other block columns are
// their own tasks (gathered into shared memory, swapped there, written back); the trailing
// update reuses the TRSM (unit lower, with the inverse 64 x 64 blocks of L_kk the panel's
// item 0 leaves in the workspace) and GEMM_NN tile operations.
#pragma once

#include "device_types.hpp"
#include "sync_util.cuh"
#include "tile_ops.cuh"

namespace mtd {
namespace piv {

constexpr int kSwapCols = 64;    // columns of one row-interchange work item
constexpr int kSwapChunk = 128;  // pivots gathered at a time (a panel's worth)

// Shared memory of a panel item: the slab [w][R] (column-major, R rows), then the pivot row,
// the previous row c and the reduction scratch (panel_piv_extra_bytes).  After the slab is
// written back, item 0 forms the inverse blocks of L_kk in that space (two kNB x kDiagLd
// blocks, always within the kernel's shared memory).
static_assert(size_t(2) * kNB * kDiagLd * sizeof(double) <= size_t(kOpSmemBytes()), "inverse scratch fits");

// Largest |value| with the smallest row on ties (LAPACK's idamax takes the first maximum).
__device__ __forceinline__ void better(double &v, int &r, double v2, int r2) {
    if (v2 > v || (v2 == v && r2 < r)) {
        v = v2;
        r = r2;
    }
}

}  // namespace piv

// One item of a panel factorisation: rows [r0, r0 + rows) of the m x w panel at (cr, cc).
// DevTask: m = panel rows, n = w, k = R (rows per item), n_items = P, pad = panel index
// (its barrier counter).  On return the panel holds L (unit, below the diagonal) and U
// (its top w rows), ipiv[cr .. cr + w) the interchanges (1-based matrix rows).
static __device__ int op_panel_piv(const RunArgs &p, const MatCtx &m, const DevTask &t, int item, void *smem) {
    const int w = t.n, mrows = t.m, R = t.k, P = t.n_items;
    const int r0 = item * R, rows = min(R, mrows - r0);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    constexpr int kWarps = kThreads / 32;
    double *A = at<double>(m, t.cr, t.cc);
    const int64_t lda = m.lda;
    double *slab = static_cast<double *>(smem);
    double *urow = slab + size_t(w) * R;
    double *drow = urow + w;
    double *rv = drow + w;
    int *rr = reinterpret_cast<int *>(rv + kWarps);
    __shared__ int s_best, s_fail;
    double *slots = p.panel_slots;
    auto slot = [&](int par, int it) { return slots + (size_t(par) * P + it) * (w + 2); };
    double *diag = slots + size_t(2) * P * (w + 2);
    unsigned int *bar = p.panel_bar + t.pad;

    for (int e = tid; e < rows * w; e += kThreads) {
        const int i = e % rows, j = e / rows;
        slab[i + j * R] = ld_cg(A + (r0 + i) + int64_t(j) * lda);
    }
    if (tid == 0) s_fail = 0;
    __syncthreads();

    // This item's candidate for column col (the largest |a| over its rows at or below col)
    // with that row, and -- from the item that owns row col -- row col itself; then arrive.
    auto publish = [&](int col) {
        double bv = -1.0;
        int br = 0x7fffffff;
        for (int i = max(col - r0, 0) + tid; i < rows; i += kThreads) piv::better(bv, br, fabs(slab[i + col * R]), r0 + i);
        for (int o = 16; o > 0; o >>= 1)
            piv::better(bv, br, __shfl_xor_sync(0xffffffffu, bv, o), __shfl_xor_sync(0xffffffffu, br, o));
        if (lane == 0) {
            rv[warp] = bv;
            rr[warp] = br;
        }
        __syncthreads();
        if (tid == 0) {
            for (int q = 1; q < kWarps; ++q) piv::better(bv, br, rv[q], rr[q]);
            s_best = br;
            double *sl = slot(col & 1, item);
            sl[0] = bv;  // -1: no row of this item at or below col
            sl[1] = static_cast<double>(br);
        }
        __syncthreads();
        const int best = s_best;
        if (best != 0x7fffffff)
            for (int j = tid; j < w; j += kThreads) slot(col & 1, item)[2 + j] = slab[(best - r0) + j * R];
        if (col >= r0 && col < r0 + rows)
            for (int j = tid; j < w; j += kThreads) diag[(col & 1) * w + j] = slab[(col - r0) + j * R];
        __threadfence();  // the slot before the arrival that publishes it
        __syncthreads();
        if (tid == 0) atomicAdd(bar, 1u);
    };

    publish(0);
    for (int c = 0; c < w; ++c) {
        if (tid == 0) {  // every item's candidate for column c is in
            const unsigned int target = static_cast<unsigned int>(P) * static_cast<unsigned int>(c + 1);
            const unsigned long long t0 = global_ns();
            while (static_cast<unsigned int>(ld_volatile(reinterpret_cast<const int *>(bar))) < target) {
                if (global_ns() - t0 > p.timeout_ns || ld_volatile(&p.ctl->abort)) {
                    report_error(p.ctl, MTD_ERR_TIMEOUT, 0);
                    s_fail = 1;
                    break;
                }
                __nanosleep(32);
            }
            __threadfence();
        }
        __syncthreads();
        if (s_fail) return MTD_ERR_TIMEOUT;
        if (warp == 0) {  // the pivot: the best candidate over the items
            double bv = -1.0;
            int br = 0x7fffffff, bi = 0;
            for (int it = lane; it < P; it += 32) {
                const double *sl = slot(c & 1, it);
                const double v = ld_cg(sl);
                const int r = static_cast<int>(ld_cg(sl + 1));
                if (v >= 0.0 && (v > bv || (v == bv && r < br))) {
                    bv = v;
                    br = r;
                    bi = it;
                }
            }
            for (int o = 16; o > 0; o >>= 1) {
                const double v2 = __shfl_xor_sync(0xffffffffu, bv, o);
                const int r2 = __shfl_xor_sync(0xffffffffu, br, o), i2 = __shfl_xor_sync(0xffffffffu, bi, o);
                if (v2 > bv || (v2 == bv && r2 < br)) {
                    bv = v2;
                    br = r2;
                    bi = i2;
                }
            }
            if (lane == 0) {
                rr[0] = br;
                rr[1] = bi;
            }
        }
        __syncthreads();
        const int pr = rr[0], pitem = rr[1];
        for (int j = tid; j < w; j += kThreads) {
            urow[j] = ld_cg(slot(c & 1, pitem) + 2 + j);
            drow[j] = ld_cg(diag + (c & 1) * w + j);
        }
        if (item == 0 && tid == 0) p.ipiv[t.cr + c] = t.cr + pr + 1;
        __syncthreads();
        // the interchange: row c takes the pivot row, row pr the old row c
        if (c >= r0 && c < r0 + rows)
            for (int j = tid; j < w; j += kThreads) slab[(c - r0) + j * R] = urow[j];
        if (pr != c && pr >= r0 && pr < r0 + rows)
            for (int j = tid; j < w; j += kThreads) slab[(pr - r0) + j * R] = drow[j];
        __syncthreads();
        const double pv = urow[c];
        if (pv == 0.0 && item == 0 && tid == 0) atomicMin(&p.ctl->info, t.cc + c + 1);  // LAPACK's info
        const int lo = max(c + 1 - r0, 0);
        if (pv != 0.0) {  // with a zero pivot the column below is zero already (it was the largest)
            const double rinv = 1.0 / pv;
            for (int i = lo + tid; i < rows; i += kThreads) slab[i + c * R] *= rinv;
        }
        __syncthreads();
        const int cols = w - c - 1, span = rows - lo;
        for (int e = tid; e < span * cols; e += kThreads) {
            const int i = lo + e % span, j = c + 1 + e / span;
            slab[i + j * R] -= slab[i + c * R] * urow[j];
        }
        __syncthreads();
        if (c + 1 < w) publish(c + 1);
    }
    for (int e = tid; e < rows * w; e += kThreads) {
        const int i = e % rows, j = e / rows;
        A[(r0 + i) + int64_t(j) * lda] = slab[i + j * R];
    }
    if (item == 0) {  // inverses of L_kk's kNB-row diagonal blocks, for the TRSM tasks
        double *L = static_cast<double *>(smem);  // the slab is back in global memory
        double *X = L + kNB * kDiagLd;
        double *W = static_cast<double *>(m.wsl) + t.cr;
        __syncthreads();
        for (int jb = 0; jb < w; jb += kNB) {
            const int jn = min(kNB, w - jb);
            for (int e = tid; e < jn * jn; e += kThreads) {
                const int r = e % jn, c = e / jn;
                L[r + c * kDiagLd] = A[(jb + r) + int64_t(jb + c) * lda];  // written above by this CTA
            }
            __syncthreads();
            lower_inverse<true>(jn, [&](int i, int l) { return L[i + l * kDiagLd]; }, X);
            for (int e = tid; e < jn * jn; e += kThreads) {
                const int r = e % jn, c = e / jn;
                W[(jb + r) + int64_t(c) * m.wsld] = X[r + c * kDiagLd];
            }
            __syncthreads();
        }
    }
    return 0;
}

// One column strip of a row-interchange task: for r = ar .. ar + k - 1 in order, swap rows r
// and ipiv[r] - 1 of columns [cc + item * kSwapCols, ...) (LAPACK's dlaswp).  Each chunk of
// kSwapChunk pivots gathers the rows it touches into shared memory, swaps them there and
// writes them back.
static __device__ int op_laswp(const RunArgs &p, const MatCtx &m, const DevTask &t, int item, void *smem) {
    using namespace piv;
    const int c0 = item * kSwapCols, nc = min(kSwapCols, t.n - c0);
    const int tid = threadIdx.x;
    const int64_t lda = m.lda;
    double *buf = static_cast<double *>(smem);                           // [2 kSwapChunk][kSwapCols]
    int *rows_of = reinterpret_cast<int *>(buf + 2 * kSwapChunk * kSwapCols);  // [2 kSwapChunk]
    int *pslot = rows_of + 2 * kSwapChunk;                               // [kSwapChunk]
    int *prow = pslot + kSwapChunk;                                      // [kSwapChunk]
    int *first_of = prow + kSwapChunk;                                   // [kSwapChunk]
    __shared__ int s_extra;
    double *A = static_cast<double *>(m.a);
    for (int base = t.ar; base < t.ar + t.k; base += kSwapChunk) {
        const int cnt = min(kSwapChunk, t.ar + t.k - base);
        if (tid < cnt) prow[tid] = ld_volatile(p.ipiv + base + tid) - 1;
        __syncthreads();
        // slots: the chunk's own rows, then each row outside it at its first occurrence
        if (tid < cnt) {
            const int pr = prow[tid];
            int first = tid;
            if (pr >= base + cnt)
                for (int q = 0; q < tid; ++q)
                    if (prow[q] == pr) {
                        first = q;
                        break;
                    }
            first_of[tid] = (pr >= base + cnt) ? first : -1;
        }
        __syncthreads();
        if (tid == 0) {
            int extra = 0;
            for (int r = 0; r < cnt; ++r) {
                if (first_of[r] == r) {  // a new outside row
                    rows_of[cnt + extra] = prow[r];
                    pslot[r] = cnt + extra++;
                }
            }
            s_extra = extra;
        }
        __syncthreads();
        if (tid < cnt) {
            rows_of[tid] = base + tid;
            const int pr = prow[tid];
            if (pr < base + cnt) pslot[tid] = pr - base;
            else if (first_of[tid] != tid) pslot[tid] = pslot[first_of[tid]];
        }
        __syncthreads();
        const int S = cnt + s_extra;
        for (int e = tid; e < S * nc; e += kThreads) {
            const int s = e % S, c = e / S;
            buf[s + c * 2 * kSwapChunk] = ld_cg(A + rows_of[s] + int64_t(t.cc + c0 + c) * lda);
        }
        __syncthreads();
        if (tid < nc)
            for (int r = 0; r < cnt; ++r) {
                const int s = pslot[r];
                if (s != r) {
                    double *col = buf + tid * 2 * kSwapChunk;
                    const double v = col[r];
                    col[r] = col[s];
                    col[s] = v;
                }
            }
        __syncthreads();
        for (int e = tid; e < S * nc; e += kThreads) {
            const int s = e % S, c = e / S;
            A[rows_of[s] + int64_t(t.cc + c0 + c) * lda] = buf[s + c * 2 * kSwapChunk];
        }
        __syncthreads();
    }
    return 0;
}

}  // namespace mtd
