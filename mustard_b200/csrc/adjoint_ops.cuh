// Tile operations of the blocked Cholesky adjoint (reverse-mode derivative of A = L L^T).
//
// No counterpart in the reference.  Given L and Lbar = dLoss/dL (lower), the reverse sweep
// over block columns j = nb-1 .. 0 of the blocked (left-looking) factorisation
//     D = chol(A_jj - R R^T),   C = (A_{>j,j} - B R^T) D^-T,
// with R = L(j, <j), B = L(>j, <j), turns Lbar into Abar = dLoss/dA (the gradient with
// respect to the lower triangle of A, which is all the factorisation reads):
//     Cbar := Cbar D^-1                                   ADJ_TRSM
//     Dbar -= tril(Cbar^T C)                              ADJ_GEMM_TN (lower only)
//     Sbar  = chol_adjoint(D, Dbar), Y = Sbar + Sbar^T    ADJ_POTRF
//     Bbar -= Cbar R                                      ADJ_GEMM_NN
//     Rbar -= Cbar^T B + Y R                              ADJ_GEMM_TN, ADJ_GEMM_NN (A = Y)
// (I. Murray, "Differentiation of the Cholesky decomposition", arXiv:1602.07527, 2016).
// The diagonal adjoint of a 64 x 64 block is M = W^T Phi(D^T Dbar) W with W = D^-1 and
// Phi = lower triangle with the diagonal halved; Sbar = tril(M + M^T) - diag(M).
//
// Operands: a task's matrix index t.mat selects three entries of the run's matrix table:
// mats[t.mat] the adjoint (Lbar in, Abar out, updated in place), mats[t.mat + 1] the factor
// L (read only; its inverse diagonal blocks in the workspace slice of that entry), and
// mats[t.mat + 2] the Y workspace (rows of diagonal tile j, columns 0 .. tile).
#pragma once

#include "tile_ops.cuh"

namespace mtd {

template <typename T>
__device__ __forceinline__ MatCtx adj_ctx(const RunArgs &p, const DevTask &t, int which) {
    const BatchMat &bm = p.mats[t.mat + which];
    return MatCtx{bm.a, bm.lda, static_cast<T *>(p.ws_lower) + bm.ws_off, nullptr, bm.ws_ld, -1};
}

// C := C * L^-1 for a 64-row strip of C: column blocks from the last to the first,
// C_c = (C_c - C_{>c} L_{>c,c}) W_c with W_c the inverse of L's diagonal block c.
template <typename T, int VEC, int SPLIT>
__device__ int op_adj_trsm(const RunArgs &p, const DevTask &t, int item, void *smem) {
    using Mn = PanelMma<kBKContig, VEC, T, SPLIT>;
    const MatCtx xa = adj_ctx<T>(p, t, 0), lf = adj_ctx<T>(p, t, 1);
    const int r0 = item * kPanelRows;
    const int mm = min(kPanelRows, t.m - r0);
    const int nk = t.n;
    T *X = at<T>(xa, t.cr + r0, t.cc);
    const T *L = at<T>(lf, t.ar, t.ac);
    const T *W = ws_lo<T>(lf) + t.ar;
    const int64_t ldx = xa.lda, ldl = lf.lda, ldw = lf.wsld;
    for (int jb = ((nk - 1) / kNB) * kNB; jb >= 0; jb -= kNB) {
        const int jn = min(kNB, nk - jb);
        const int rest = nk - jb - jn;
        if (rest > 0) {
            Mn e;
            e.zero();
            e.run(smem, X + int64_t(jb + jn) * ldx, ldx, L + (jb + jn) + int64_t(jb) * ldl, ldl, mm, jn, rest);
            e.sub_from(X + int64_t(jb) * ldx, ldx, mm, jn);
            block_fence_sync();
        }
        Mn e;
        e.zero();
        e.run(smem, X + int64_t(jb) * ldx, ldx, W + jb, ldw, mm, jn, jn);
        e.store_to(X + int64_t(jb) * ldx, ldx, mm, jn);
        block_fence_sync();
    }
    return 0;
}

// C -= A B, one 128 x 128 output tile per item.
template <typename T, int VEC, int SPLIT>
__device__ int op_adj_gemm_nn(const RunArgs &p, const DevTask &t, int item, void *smem) {
    using Mg = GemmMma<kBKContig, VEC, T, SPLIT>;
    const MatCtx ca = adj_ctx<T>(p, t, 0), lf = adj_ctx<T>(p, t, 1), aa = adj_ctx<T>(p, t, t.pad == 2 ? 2 : 0);
    const int nbn = (t.n + kGemmTile - 1) / kGemmTile;
    const int r0 = (item / nbn) * kGemmTile, c0 = (item % nbn) * kGemmTile;
    const int mm = min(kGemmTile, t.m - r0), nn = min(kGemmTile, t.n - c0);
    Mg e;
    e.zero();
    e.run(smem, at<T>(aa, t.ar + r0, t.ac), aa.lda, at<T>(lf, t.br, t.bc + c0), lf.lda, mm, nn, t.k);
    e.sub_from(at<T>(ca, t.cr + r0, t.cc + c0), ca.lda, mm, nn);
    return 0;
}

// C -= A^T B with A stored k x m (column-major) in the adjoint: A^T staged k-contiguous.
template <typename T, int VEC, int SPLIT>
__device__ int op_adj_gemm_tn(const RunArgs &p, const DevTask &t, int item, void *smem) {
    using Mg = BlockMmaT<T, kGemmTile, kGemmTile, kGemmWarpsM, kGemmWarpsN, kBKContig, VEC, MTD_GEMM_STAGES,
                         MTD_GEMM_BK, SPLIT, kAKContig>;
    const MatCtx ca = adj_ctx<T>(p, t, 0), lf = adj_ctx<T>(p, t, 1);
    const int nbn = (t.n + kGemmTile - 1) / kGemmTile;
    const int r0 = (item / nbn) * kGemmTile, c0 = (item % nbn) * kGemmTile;
    const int mm = min(kGemmTile, t.m - r0), nn = min(kGemmTile, t.n - c0);
    Mg e;
    e.zero();
    e.run(smem, at<T>(ca, t.ar, t.ac + r0), ca.lda, at<T>(lf, t.br, t.bc + c0), lf.lda, mm, nn, t.k);
    e.sub_from(at<T>(ca, t.cr + r0, t.cc + c0), ca.lda, mm, nn, (t.pad & 1) != 0, r0, c0);
    return 0;
}

// Adjoint of one diagonal block of at most 64 x 64, all in shared memory:
//   in:  D (bn x bn lower, the factor), G (lower: Dbar), W = D^-1
//   out: G lower = Sbar = tril(M + M^T) - diag(M), Y = M + M^T, M = W^T Phi(D^T Dbar) W.
template <typename T>
__device__ void adj_diag_block(const T *D, int64_t ldd, T *G, int64_t ldg, const T *W, int64_t ldw, T *Y,
                               int64_t ldy, int bn, void *smem_raw) {
    T *Ds = static_cast<T *>(smem_raw);  // [c][r] at c * kDiagLd + r
    T *Gs = Ds + kNB * kDiagLd;
    T *Ws = Gs + kNB * kDiagLd;
    T *P = Ws + kNB * kDiagLd;
    T *Q = P + kNB * kDiagLd;
    const int tid = threadIdx.x;
    for (int e = tid; e < kNB * kNB; e += kThreads) {
        const int r = e % kNB, c = e / kNB;
        const bool in = r < bn && c < bn && r >= c;
        Ds[c * kDiagLd + r] = in ? ld_cg(D + r + int64_t(c) * ldd) : T(0);
        Gs[c * kDiagLd + r] = in ? ld_cg(G + r + int64_t(c) * ldg) : T(0);
        Ws[c * kDiagLd + r] = in ? ld_cg(W + r + int64_t(c) * ldw) : T(0);
    }
    __syncthreads();
    // P = Phi(D^T Dbar): P(r, c) = sum_{k >= r} D(k, r) Dbar(k, c), r >= c; diagonal halved
    for (int e = tid; e < kNB * kNB; e += kThreads) {
        const int r = e % kNB, c = e / kNB;
        T s = T(0);
        if (r >= c)
            for (int k = r; k < kNB; ++k) s += Ds[r * kDiagLd + k] * Gs[c * kDiagLd + k];
        P[c * kDiagLd + r] = r == c ? s * T(0.5) : s;
    }
    __syncthreads();
    // Q = P W: Q(r, c) = sum_{c <= k <= r} P(r, k) W(k, c)
    for (int e = tid; e < kNB * kNB; e += kThreads) {
        const int r = e % kNB, c = e / kNB;
        T s = T(0);
        for (int k = c; k <= r; ++k) s += P[k * kDiagLd + r] * Ws[c * kDiagLd + k];
        Q[c * kDiagLd + r] = s;
    }
    __syncthreads();
    // M = W^T Q: M(r, c) = sum_{k >= max(r, c)} W(k, r) Q(k, c)  (Q(k, c) = 0 for k < c)
    for (int e = tid; e < kNB * kNB; e += kThreads) {
        const int r = e % kNB, c = e / kNB;
        T s = T(0);
        for (int k = max(r, c); k < kNB; ++k) s += Ws[r * kDiagLd + k] * Q[c * kDiagLd + k];
        P[c * kDiagLd + r] = s;  // P now holds M
    }
    __syncthreads();
    for (int e = tid; e < bn * bn; e += kThreads) {
        const int r = e % bn, c = e / bn;
        const T m = P[c * kDiagLd + r], mt = P[r * kDiagLd + c];
        Y[r + int64_t(c) * ldy] = m + mt;
        if (r > c) G[r + int64_t(c) * ldg] = m + mt;
        else if (r == c) G[r + int64_t(c) * ldg] = m;
    }
}

// Adjoint of the m x m diagonal tile at (cr, cc) (m <= 256), the same reverse sweep inside
// the tile over its 64-blocks; writes the tile's Sbar (lower) over Dbar and
// Y = Sbar + Sbar^T (full m x m) to the Y workspace.  Products with the rows below a block
// go in 64-row pieces (the engine's output edge).
template <typename T, int VEC, int SPLIT>
__device__ int op_adj_potrf(const RunArgs &p, const DevTask &t, void *smem) {
    using Mnn = PanelMma<kBKContig, VEC, T, SPLIT>;
    using Mtn = BlockMmaT<T, 64, 64, kPanelWarpsM, kPanelWarpsN, kBKContig, VEC, 3, 16, SPLIT, kAKContig>;
    const MatCtx ga = adj_ctx<T>(p, t, 0), lf = adj_ctx<T>(p, t, 1), ya = adj_ctx<T>(p, t, 2);
    const int tn = t.m;
    T *G = at<T>(ga, t.cr, t.cc);
    const T *D = at<T>(lf, t.cr, t.cc);
    T *Y = at<T>(ya, t.cr, 0);
    const T *W = ws_lo<T>(lf) + t.cr;
    const int64_t ldg = ga.lda, ldd = lf.lda, ldy = ya.lda, ldw = lf.wsld;
    const int s = (tn + kNB - 1) / kNB;
    for (int b = s - 1; b >= 0; --b) {
        const int bo = b * kNB, bn = min(kNB, tn - bo), lo = bo + bn, below = tn - lo;
        if (below > 0) {
            for (int r0 = lo; r0 < tn; r0 += kNB) {  // X = G(below, b) W_b
                const int mm = min(kNB, tn - r0);
                Mnn e;
                e.zero();
                e.run(smem, G + r0 + int64_t(bo) * ldg, ldg, W + bo, ldw, mm, bn, bn);
                e.store_to(G + r0 + int64_t(bo) * ldg, ldg, mm, bn);
            }
            block_fence_sync();
            {  // Dbar_b -= tril(X^T D(below, b))
                Mtn e;
                e.zero();
                e.run(smem, G + lo + int64_t(bo) * ldg, ldg, D + lo + int64_t(bo) * ldd, ldd, bn, bn, below);
                e.sub_from(G + bo + int64_t(bo) * ldg, ldg, bn, bn, true, 0, 0);
            }
            block_fence_sync();
        }
        adj_diag_block<T>(D + bo + int64_t(bo) * ldd, ldd, G + bo + int64_t(bo) * ldg, ldg, W + bo, ldw,
                          Y + bo + int64_t(bo) * ldy, ldy, bn, smem);
        block_fence_sync();
        for (int kb = 0; kb < bo; kb += kNB) {
            const int kn = min(kNB, bo - kb);
            if (below > 0) {
                for (int r0 = lo; r0 < tn; r0 += kNB) {  // G(below, k) -= X D(b, k)
                    const int mm = min(kNB, tn - r0);
                    Mnn e;
                    e.zero();
                    e.run(smem, G + r0 + int64_t(bo) * ldg, ldg, D + bo + int64_t(kb) * ldd, ldd, mm, kn, bn);
                    e.sub_from(G + r0 + int64_t(kb) * ldg, ldg, mm, kn);
                }
                block_fence_sync();
                {  // G(b, k) -= X^T D(below, k)
                    Mtn e;
                    e.zero();
                    e.run(smem, G + lo + int64_t(bo) * ldg, ldg, D + lo + int64_t(kb) * ldd, ldd, bn, kn, below);
                    e.sub_from(G + bo + int64_t(kb) * ldg, ldg, bn, kn);
                }
                block_fence_sync();
            }
            {  // G(b, k) -= Y_b D(b, k)
                Mnn e;
                e.zero();
                e.run(smem, Y + bo + int64_t(bo) * ldy, ldy, D + bo + int64_t(kb) * ldd, ldd, bn, kn, bn);
                e.sub_from(G + bo + int64_t(kb) * ldg, ldg, bn, kn);
            }
            block_fence_sync();
        }
    }
    // off-diagonal 64-blocks of Y: Y(r, c) = Y(c, r) = Sbar(r, c), r in a lower block
    for (int e = threadIdx.x; e < tn * tn; e += kThreads) {
        const int r = e % tn, c = e / tn;
        if (r / kNB > c / kNB) {
            const T v = G[r + int64_t(c) * ldg];
            Y[r + int64_t(c) * ldy] = v;
            Y[c + int64_t(r) * ldy] = v;
        }
    }
    return 0;
}

template <typename T, int VEC, int SPLIT>
__device__ int dispatch_adjoint(const RunArgs &p, const DevTask &t, int item, void *smem) {
    switch (t.op) {
    case kOpAdjTrsm: return op_adj_trsm<T, VEC, SPLIT>(p, t, item, smem);
    case kOpAdjGemmNN: return op_adj_gemm_nn<T, VEC, SPLIT>(p, t, item, smem);
    case kOpAdjGemmTN: return op_adj_gemm_tn<T, VEC, SPLIT>(p, t, item, smem);
    case kOpAdjPotrf: return op_adj_potrf<T, VEC, SPLIT>(p, t, smem);
    default: break;
    }
    if (threadIdx.x == 0) report_error(p.ctl, MTD_ERR_INVALID_ARG, 0);
    return MTD_ERR_INVALID_ARG;
}

}  // namespace mtd
