// FP64 GEMM / SYRK work items with operands fed by TMA (one 128 x 128 output block per CTA).
//
// The cp.async engine (mma.cuh) has every thread compute addresses and issue 16-byte copies
// for each k-slice, then meets the whole CTA at a barrier before the slice is read; the
// register-only DMMA probe runs at 37.05 TFLOP/s, the same fragment loads from padded shared
// memory without barriers too, a barrier per 32-deep slice costs 3 %, and the staged k-loop
// measured 88.5 %.  Here one thread (thread 0) issues one TMA load per operand and k-slice
// into a ring of kStages stages, each stage has a `full` mbarrier (TMA transaction bytes) and
// an `empty` mbarrier (one arrival per thread once it has read the slice), every warp waits
// only for the slice it reads, and thread 0 refills the stage of slice kt - kLag at slice kt,
// so warps drift up to kLag - 1 slices apart without waiting for one another.
//
// Layout.  Operands land unpadded with the 128-byte swizzle (16-byte chunk c of 128-byte row
// r stored at chunk c ^ (r % 8)):
//   - m- or n-contiguous operands (A; B of GEMM_NT / SYRK) through a 3D tensor map
//     {16 rows of an atom, columns, atoms of 16 rows}, box {16, kBK, 8}: one load brings 128
//     rows x kBK columns, element (m, k) at (m / 16) kBK 128 + k 128 + (((m % 16) / 2) ^ (k % 8)) 16
//     + (m % 2) 8 bytes;
//   - k-contiguous operands (B of GEMM_NN) through a 2D map {rows, columns}, box {16, 128},
//     kBK / 16 boxes per slice: element (k, n) at (k / 16) 16384 + n 128 + (((k % 16) / 2) ^
//     (n % 8)) 16 + (k % 2) 8 bytes.
// Fragment loads of mma.sync.m16n8k8.f64 from these layouts are bank-conflict-free when the
// logical rows of each 16-row fragment group are mapped to physical rows by
//   P16(l) = (l & 1) | ((l >> 1) & 1) << 3 | ((l >> 2) & 1) << 1 | ((l >> 3) & 1) << 2
// (0, 1, 8, 9, 2, 3, 10, 11, 4, 5, ...), the columns of n-contiguous B likewise by P16 over
// each pair of 8-column fragments, and the columns of k-contiguous B by
// R8(g) = 2 (g % 4) + g / 4 within each fragment (0, 2, 4, 6, 1, 3, 5, 7).  A row or column
// permutation of the block product only permutes its output; the epilogue writes every
// accumulator element to its physical row and column.  The k order of every sum is the
// cp.async engine's (ascending slices, the same k8 steps), so both engines give the same bits.
//
// Every mbarrier wait is bounded by a %globaltimer deadline.  On expiry the item reports
// MTD_ERR_TIMEOUT; thread 0 first waits (bounded again) for the loads it issued that no
// thread consumed, so no TMA write is in flight when the CTA leaves.
#pragma once

#include <cstdint>

#include "device_types.hpp"
#include "mma.cuh"

namespace mtd {
namespace t64 {

#ifndef MTD_T64_BK
#define MTD_T64_BK 16
#endif
#ifndef MTD_T64_STAGES
#define MTD_T64_STAGES 6
#endif
#ifndef MTD_T64_LAG
#define MTD_T64_LAG 2
#endif
// 1: one arrival per warp on `empty` (lane 0, after the warp's reads); 0: one per thread
// 1: fragment offsets precomputed once per item (Engine::offsets); 0: computed per load
#ifndef MTD_T64_PRECOMP
#define MTD_T64_PRECOMP 0
#endif
#ifndef MTD_T64_WARP_ARRIVE
#define MTD_T64_WARP_ARRIVE 0
#endif
// 1: B fragments loaded per column fragment inside the row loop (12 live fragment registers
// instead of 24, twice the B loads)
#ifndef MTD_T64_BINNER
#define MTD_T64_BINNER 0
#endif
constexpr int kBK = MTD_T64_BK;                  // k per stage (a multiple of 16)
constexpr int kStages = MTD_T64_STAGES;
constexpr int kLag = MTD_T64_LAG;                // stage of slice kt - kLag is refilled at slice kt
constexpr int kArrivals = MTD_T64_WARP_ARRIVE ? kThreads / 32 : kThreads;
constexpr int kOperandBytes = 128 * kBK * 8;     // 16 KB at kBK = 16
constexpr int kStageBytes = 2 * kOperandBytes;   // 32 KB
constexpr int kSmemBytes = kStages * kStageBytes + 1024;  // + alignment of the stage ring
static_assert(kLag >= 1 && kLag < kStages, "refill lag");
static_assert(kBK % 16 == 0, "whole 16-deep boxes of the k-contiguous operand");

struct State {
    uint64_t full[kStages];   // stage loaded (TMA complete_tx)
    uint64_t empty[kStages];  // stage read by every thread
    uint32_t fbase;           // bit s: parity of the next completion of full[s]
    uint32_t ebase;           // bit s: parity of the next completion of empty[s]
};

__device__ __forceinline__ uint32_t saddr(const void *p) { return static_cast<uint32_t>(__cvta_generic_to_shared(p)); }

__device__ __forceinline__ unsigned long long now_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Once per CTA (all threads; thread 0 initialises).
__device__ __forceinline__ void init(State *st) {
    if (threadIdx.x == 0) {
        for (int s = 0; s < kStages; ++s) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(saddr(&st->full[s])), "r"(1));
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(saddr(&st->empty[s])), "r"(kArrivals));
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        st->fbase = 0;
        st->ebase = 0;
    }
    __syncthreads();
}

__device__ __forceinline__ bool wait_parity(uint64_t *bar, uint32_t parity, unsigned long long deadline) {
    const uint32_t a = saddr(bar);
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
        if ((it & 63) == 63 && now_ns() > deadline) return false;
    }
}

// This thread (or warp) has read the stage: every DMMA that used its fragments is issued,
// so those shared-memory loads have returned.
__device__ __forceinline__ void release(uint64_t *bar) {
    if (MTD_T64_WARP_ARRIVE) {
        __syncwarp();
        if ((threadIdx.x & 31) == 0) asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(saddr(bar)) : "memory");
    } else {
        asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(saddr(bar)) : "memory");
    }
}

__device__ __forceinline__ void load_3d(uint32_t dst, const void *map, int x, int y, int z, uint32_t bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(
            dst),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(bar)
        : "memory");
}

__device__ __forceinline__ void load_2d(uint32_t dst, const void *map, int x, int y, uint32_t bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
            dst),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(bar)
        : "memory");
}

// Logical row / column l of a 16-wide fragment group -> physical (see the header comment).
__host__ __device__ constexpr int p16(int l) {
    return (l & 1) | (((l >> 1) & 1) << 3) | (((l >> 2) & 1) << 1) | (((l >> 3) & 1) << 2);
}
__host__ __device__ constexpr int r8(int g) { return ((g & 3) << 1) | (g >> 2); }
constexpr bool maps_are_permutations() {
    for (int a = 0; a < 16; ++a)
        for (int b = a + 1; b < 16; ++b)
            if (p16(a) == p16(b) || p16(a) > 15) return false;
    for (int a = 0; a < 8; ++a)
        for (int b = a + 1; b < 8; ++b)
            if (r8(a) == r8(b) || r8(a) > 7) return false;
    return true;
}
static_assert(maps_are_permutations(), "fragment row / column maps");

// Byte offsets inside one operand of a stage.
__device__ __forceinline__ int off_mn(int m, int k) {
    return (m >> 4) * (kBK * 128) + k * 128 + ((((m & 15) >> 1) ^ (k & 7)) << 4) + ((m & 1) << 3);
}
__device__ __forceinline__ int off_k(int k, int n) {
    return (k >> 4) * (128 * 128) + n * 128 + ((((k & 15) >> 1) ^ (n & 7)) << 4) + ((k & 1) << 3);
}

// Where one item's operands start.  A: rows a_row .. a_row + 127, columns a_col .. (3D map).
// B of GEMM_NT / SYRK (kBNContig): rows b_row .., columns b_col .. (3D map).  B of GEMM_NN
// (kBKContig): rows b_row .. (the k range), columns b_col .. b_col + 127 (2D map).  Rows are
// multiples of 16 (the host enables the maps only then), K a multiple of kBK.
struct Coords {
    int a_row, a_col, b_row, b_col, K;
};

// 128 x 128 block product on 16 warps (4 x 4 warp tiles of 32 x 32), accumulators in
// registers exactly as BlockMmaT's, fragments read through the row / column maps.
template <int BL>
struct Engine {
    static constexpr int WARPS_N = 4, WM = 32, WN = 32, FM = 2, FN = 4;
    static_assert(kThreads == 512, "16 warps of 32 x 32");
    double acc[FM][FN][4];

    __device__ __forceinline__ void zero() {
#pragma unroll
        for (int i = 0; i < FM; ++i)
#pragma unroll
            for (int j = 0; j < FN; ++j)
#pragma unroll
                for (int v = 0; v < 4; ++v) acc[i][j][v] = 0.0;
    }

    // Physical row of fragment row l (0 .. 15) of row block i; physical column of column
    // l8 (0 .. 7) of column fragment j.
    __device__ __forceinline__ static int prow(int i, int l) {
        return ((threadIdx.x >> 5) / WARPS_N) * WM + i * 16 + p16(l);
    }
    __device__ __forceinline__ static int pcol(int j, int l8) {
        const int wn0 = ((threadIdx.x >> 5) % WARPS_N) * WN;
        if (BL == kBNContig) return wn0 + (j >> 1) * 16 + p16((j & 1) * 8 + l8);
        return wn0 + j * 8 + r8(l8);
    }

    // This thread's fragment offsets at k = t (t = lane % 4) inside a stage: A rows of the
    // fragments (i, g) and (i, g + 8), B columns of fragment j.  Every other k of a slice
    // follows by one add and one XOR: for k = ks + t (+ 4), ks a multiple of 8, the swizzled
    // chunk of an m- / n-contiguous operand is ((m % 16) / 2) ^ t (^ 4), i.e. +ks 128
    // (+ 512, ^ 64); of the k-contiguous operand ((k % 16) / 2) ^ (n % 8) = (t / 2 ^ n % 8)
    // ^ ((ks % 16 + 4c) / 2), i.e. ^ (ks % 16 + 4c) 8, plus (ks / 16) 16384.
    struct Offsets {
        int a[FM][2];
        int b[FN];
    };
    __device__ __forceinline__ static Offsets offsets() {
        Offsets o;
        const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
#pragma unroll
        for (int i = 0; i < FM; ++i) {
            o.a[i][0] = off_mn(prow(i, g), t);
            o.a[i][1] = off_mn(prow(i, g + 8), t);
        }
#pragma unroll
        for (int j = 0; j < FN; ++j) o.b[j] = BL == kBNContig ? off_mn(pcol(j, g), t) : off_k(t, pcol(j, g));
        return o;
    }

    __device__ __forceinline__ static void load_b(const uint8_t *Bs, int ob, int ks, double (&b)[2]) {
        if (BL == kBNContig) {
            b[0] = *reinterpret_cast<const double *>(Bs + ob + ks * 128);
            b[1] = *reinterpret_cast<const double *>(Bs + ((ob + ks * 128 + 512) ^ 64));
        } else {
            const int kb = (ks >> 4) * 16384, x0 = (ks & 15) * 8, x1 = ((ks & 15) + 4) * 8;
            b[0] = *reinterpret_cast<const double *>(Bs + kb + (ob ^ x0));
            b[1] = *reinterpret_cast<const double *>(Bs + kb + (ob ^ x1));
        }
    }

    __device__ __forceinline__ void compute_stage_pre(const uint8_t *st_base, const Offsets &o) {
        const uint8_t *As = st_base, *Bs = st_base + kOperandBytes;
#if MTD_T64_BINNER
#pragma unroll
        for (int ks = 0; ks < kBK; ks += 8) {
#pragma unroll
            for (int i = 0; i < FM; ++i) {
                double af[4];
                af[0] = *reinterpret_cast<const double *>(As + o.a[i][0] + ks * 128);
                af[1] = *reinterpret_cast<const double *>(As + o.a[i][1] + ks * 128);
                af[2] = *reinterpret_cast<const double *>(As + ((o.a[i][0] + ks * 128 + 512) ^ 64));
                af[3] = *reinterpret_cast<const double *>(As + ((o.a[i][1] + ks * 128 + 512) ^ 64));
#pragma unroll
                for (int j = 0; j < FN; ++j) {
                    double bf[2];
                    load_b(Bs, o.b[j], ks, bf);
                    dmma_16x8x8(acc[i][j], af, bf);
                }
            }
        }
        return;
#endif
#pragma unroll
        for (int ks = 0; ks < kBK; ks += 8) {
            double bf[FN][2];
#pragma unroll
            for (int j = 0; j < FN; ++j) {
                if (BL == kBNContig) {
                    bf[j][0] = *reinterpret_cast<const double *>(Bs + o.b[j] + ks * 128);
                    bf[j][1] = *reinterpret_cast<const double *>(Bs + ((o.b[j] + ks * 128 + 512) ^ 64));
                } else {
                    const int kb = (ks >> 4) * 16384, x0 = (ks & 15) * 8, x1 = ((ks & 15) + 4) * 8;
                    bf[j][0] = *reinterpret_cast<const double *>(Bs + kb + (o.b[j] ^ x0));
                    bf[j][1] = *reinterpret_cast<const double *>(Bs + kb + (o.b[j] ^ x1));
                }
            }
#pragma unroll
            for (int i = 0; i < FM; ++i) {
                double af[4];
                af[0] = *reinterpret_cast<const double *>(As + o.a[i][0] + ks * 128);
                af[1] = *reinterpret_cast<const double *>(As + o.a[i][1] + ks * 128);
                af[2] = *reinterpret_cast<const double *>(As + ((o.a[i][0] + ks * 128 + 512) ^ 64));
                af[3] = *reinterpret_cast<const double *>(As + ((o.a[i][1] + ks * 128 + 512) ^ 64));
#pragma unroll
                for (int j = 0; j < FN; ++j) dmma_16x8x8(acc[i][j], af, bf[j]);
            }
        }
    }

    __device__ __forceinline__ void compute_stage(const uint8_t *st_base) {
        const uint8_t *As = st_base, *Bs = st_base + kOperandBytes;
        const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
#pragma unroll
        for (int ks = 0; ks < kBK; ks += 8) {
            double bf[FN][2];
#pragma unroll
            for (int j = 0; j < FN; ++j) {
                const int n = pcol(j, g);
                if (BL == kBNContig) {
                    bf[j][0] = *reinterpret_cast<const double *>(Bs + off_mn(n, ks + t));
                    bf[j][1] = *reinterpret_cast<const double *>(Bs + off_mn(n, ks + t + 4));
                } else {
                    bf[j][0] = *reinterpret_cast<const double *>(Bs + off_k(ks + t, n));
                    bf[j][1] = *reinterpret_cast<const double *>(Bs + off_k(ks + t + 4, n));
                }
            }
#pragma unroll
            for (int i = 0; i < FM; ++i) {
                const int m0 = prow(i, g), m1 = prow(i, g + 8);
                double af[4];
                af[0] = *reinterpret_cast<const double *>(As + off_mn(m0, ks + t));
                af[1] = *reinterpret_cast<const double *>(As + off_mn(m1, ks + t));
                af[2] = *reinterpret_cast<const double *>(As + off_mn(m0, ks + t + 4));
                af[3] = *reinterpret_cast<const double *>(As + off_mn(m1, ks + t + 4));
#pragma unroll
                for (int j = 0; j < FN; ++j) dmma_16x8x8(acc[i][j], af, bf[j]);
            }
        }
    }

    // Thread 0: load slice kt of the item into stage s (one expect_tx, two loads).
    __device__ __noinline__ static void issue(State *st, uint8_t *ring, const void *map_mn, const void *map_k,
                                              const Coords &c, int s, int kt) {
        const uint32_t bar = saddr(&st->full[s]), dst = saddr(ring + s * kStageBytes);
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(kStageBytes) : "memory");
        load_3d(dst, map_mn, 0, c.a_col + kt * kBK, c.a_row >> 4, bar);
        if (BL == kBNContig) {
            load_3d(dst + kOperandBytes, map_mn, 0, c.b_col + kt * kBK, c.b_row >> 4, bar);
        } else {
#pragma unroll
            for (int kb = 0; kb < kBK / 16; ++kb)  // 16-deep boxes of 128 columns, 16 KB each
                load_2d(dst + kOperandBytes + kb * 16384, map_k, c.b_row + kt * kBK + 16 * kb, c.b_col, bar);
        }
    }

    // acc = A B over c.K (all threads of the CTA).  `ring`: kStages x kStageBytes, 1024-byte
    // aligned.  Returns false when a wait ran past the deadline.
    __device__ bool run(State *st, uint8_t *ring, const void *map_mn, const void *map_k, const Coords &c,
                        unsigned long long timeout_ns) {
        const int nk = c.K / kBK;
        const uint32_t fbase = st->fbase, ebase = st->ebase;
        const unsigned long long deadline = now_ns() + timeout_ns;
        int issued = 0;  // thread 0: slices loaded so far
        if (threadIdx.x == 0) {
            // the operands were written by other CTAs with generic stores (released and
            // acquired through the scheduler's counters), and earlier items of this CTA used
            // the ring's shared memory with generic loads and stores (ordered across threads
            // by the barrier before this item): order both before the async-proxy writes
            asm volatile("fence.proxy.async.global;" ::: "memory");
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            for (; issued < kStages && issued < nk; ++issued) issue(st, ring, map_mn, map_k, c, issued, issued);
        }
        bool ok = true;
        int kt = 0;
#if MTD_T64_PRECOMP
        const Offsets offs = offsets();
#endif
        for (; kt < nk; ++kt) {
            const int s = kt % kStages;
            if (threadIdx.x == 0 && kt >= kLag && issued < nk) {
                // slice `issued` (= kt - kLag + kStages) goes into the stage slice kt - kLag
                // used, once every thread has read that slice (its use prev / kStages of the
                // stage in this item)
                const int prev = issued - kStages, sp = issued % kStages;
                const uint32_t par = ((ebase >> sp) + prev / kStages) & 1u;
                ok = wait_parity(&st->empty[sp], par, deadline);
                if (!ok) break;
                issue(st, ring, map_mn, map_k, c, sp, issued++);
            }
            const uint32_t fpar = ((fbase >> s) + kt / kStages) & 1u;
            ok = wait_parity(&st->full[s], fpar, deadline);
            if (!ok) break;
#if MTD_T64_PRECOMP
            compute_stage_pre(ring + s * kStageBytes, offs);
#else
            compute_stage(ring + s * kStageBytes);
#endif
            release(&st->empty[s]);
        }
        if (!ok) {
            // thread 0: let the loads it issued and did not consume land before leaving
            if (threadIdx.x == 0) {
                const unsigned long long grace = now_ns() + 1000000ull;
                for (int q = kt; q < issued; ++q) {
                    const int s = q % kStages;
                    wait_parity(&st->full[s], ((fbase >> s) + q / kStages) & 1u, grace);
                }
            }
            return false;
        }
        // every thread consumed nk slices: advance the parities of each stage by its uses
        if (threadIdx.x == 0) {
            uint32_t f = fbase, e = ebase;
            for (int s = 0; s < kStages && s < nk; ++s) {
                const int uses = (nk - 1 - s) / kStages + 1;
                if (uses & 1) {
                    f ^= 1u << s;
                    e ^= 1u << s;
                }
            }
            st->fbase = f;
            st->ebase = e;
        }
        return true;
    }

    // C(r, c) -= acc at the physical rows / columns (r < M, c < N; r >= c when lower_only).
    __device__ __forceinline__ void sub_from(double *C, int64_t ldc, int M, int N, bool lower_only) const {
        const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
#pragma unroll
        for (int i = 0; i < FM; ++i)
#pragma unroll
            for (int jh = 0; jh < FN; jh += 2) {
                double cv[2][4];
#pragma unroll
                for (int jj = 0; jj < 2; ++jj)
#pragma unroll
                    for (int v = 0; v < 4; ++v) {
                        const int r = prow(i, g + ((v & 2) ? 8 : 0)), cc = pcol(jh + jj, 2 * t + (v & 1));
                        const bool in = r < M && cc < N && (!lower_only || r >= cc);
                        cv[jj][v] = in ? ld_cg(C + r + int64_t(cc) * ldc) : 0.0;
                    }
#pragma unroll
                for (int jj = 0; jj < 2; ++jj)
#pragma unroll
                    for (int v = 0; v < 4; ++v) {
                        const int r = prow(i, g + ((v & 2) ? 8 : 0)), cc = pcol(jh + jj, 2 * t + (v & 1));
                        if (r < M && cc < N && (!lower_only || r >= cc))
                            C[r + int64_t(cc) * ldc] = cv[jj][v] - acc[i][jh + jj][v];
                    }
            }
    }
};

}  // namespace t64
}  // namespace mtd
