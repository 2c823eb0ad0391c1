// ordered.cuh -- sums in the reference's order, row by row.
//
// The reference adds the terms of each row sequentially, with one rounding per
// product and per addition. A row of up to kWarpRow terms is summed by one
// thread; a longer row by one warp, whose lanes evaluate the terms together
// and then add them in row order. Both give the bit pattern of the sequential
// sum. Used by the FP64-exact kernels and by the device intake.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "engine.cuh"

namespace pdhg {

__host__ __device__ inline int ordered_blocks(int64_t n) {
    return static_cast<int>((n + kBlock - 1) / kBlock);
}

// acc = init; for k in [b, e): acc = acc + v[k] * g(ci[k]), rounded after each
// product and each sum, in k order. The loads of four terms are issued before
// their products are added, so the memory latency of a long row overlaps while
// the sum keeps the reference's order exactly.
template <class G>
__device__ __forceinline__ double ordered_dot(int b, int e, const int32_t* __restrict__ ci,
                                              const double* __restrict__ v, G g, double init) {
    double acc = init;
    int k = b;
    for (; k + 4 <= e; k += 4) {
        const int c0 = ci[k], c1 = ci[k + 1], c2 = ci[k + 2], c3 = ci[k + 3];
        const double v0 = v[k], v1 = v[k + 1], v2 = v[k + 2], v3 = v[k + 3];
        const double g0 = g(c0), g1 = g(c1), g2 = g(c2), g3 = g(c3);
        acc = __dadd_rn(acc, __dmul_rn(v0, g0));
        acc = __dadd_rn(acc, __dmul_rn(v1, g1));
        acc = __dadd_rn(acc, __dmul_rn(v2, g2));
        acc = __dadd_rn(acc, __dmul_rn(v3, g3));
    }
    for (; k < e; ++k) acc = __dadd_rn(acc, __dmul_rn(v[k], g(ci[k])));
    return acc;
}

constexpr int kWarps = kBlock / 32;
constexpr int kStage = 128;  // terms a warp evaluates per round

// 128 doubles of shared memory per warp of the block.
__device__ __forceinline__ double* warp_stage() {
    __shared__ __align__(16) double stage[kWarps][kStage];
    return stage[threadIdx.x >> 5];
}

// The same ordered sum when a whole warp owns the row: acc = init, then
// acc = acc + term(k) for k in [b, e), in k order. The 32 lanes evaluate 128
// rounded terms at a time (their loads in flight together), park them in
// `stage`, and every lane then adds the 128 in k order -- the rounding
// sequence of one thread, so each lane ends with exactly the thread result.
template <class Term>
__device__ __forceinline__ double ordered_sum_warp(int b, int e, Term term, double init,
                                                   double* stage) {
    const int lane = threadIdx.x & 31;
    double acc = init;
    for (int k0 = b; k0 < e; k0 += kStage) {
        const int cnt = min(kStage, e - k0);
        double t[kStage / 32];
#pragma unroll
        for (int q = 0; q < kStage / 32; ++q) {
            const int o = 32 * q + lane;
            t[q] = o < cnt ? term(k0 + o) : 0.0;
        }
#pragma unroll
        for (int q = 0; q < kStage / 32; ++q)
            if (32 * q + lane < cnt) stage[32 * q + lane] = t[q];
        __syncwarp();
        if (cnt == kStage) {
            const double2* s2 = reinterpret_cast<const double2*>(stage);
#pragma unroll 8
            for (int i = 0; i < kStage / 2; ++i) {
                const double2 p = s2[i];
                acc = __dadd_rn(acc, p.x);
                acc = __dadd_rn(acc, p.y);
            }
        } else {
            for (int i = 0; i < cnt; ++i) acc = __dadd_rn(acc, stage[i]);
        }
        __syncwarp();
    }
    return acc;
}

// The ordered dot of a long row by one warp with the loads pipelined
// ahead of the additions: acc = init, then acc = acc + v[k] * g(ci[k]) in k
// order, each product and sum rounded -- the sequence of ordered_dot, so the
// result is bit for bit the same. Rounds of kStage terms (four per lane): the
// indices and values of round r + 2 and the gathers of round r + 1 are in
// flight while the lanes add round r from shared memory (two buffers of
// kStage doubles per warp), so only the chain of additions is exposed.
// ordered_sum_warp evaluates a round's terms (index load, then gather) and
// only then adds it.
template <class G>
__device__ __forceinline__ double ordered_dot_warp_pipelined(int b, int e,
                                                             const int32_t* __restrict__ ci,
                                                             const double* __restrict__ v, G g,
                                                             double init, double* stage2) {
    constexpr int Q = kStage / 32;
    const int lane = threadIdx.x & 31;
    double acc = init;
    if (b >= e) return acc;
    auto load_cv = [&](int k0, int (&c)[Q], double (&w)[Q]) {
#pragma unroll
        for (int q = 0; q < Q; ++q) {
            const int k = k0 + 32 * q + lane;
            c[q] = k < e ? ci[k] : 0;
            w[q] = k < e ? v[k] : 0.0;
        }
    };
    // round 0's terms into buffer 0; round 1's indices and values in registers
    int c1[Q];
    double w1[Q];
    {
        int c0[Q];
        double w0[Q], t0[Q];
        load_cv(b, c0, w0);
        load_cv(b + kStage, c1, w1);
#pragma unroll
        for (int q = 0; q < Q; ++q) t0[q] = b + 32 * q + lane < e ? __dmul_rn(w0[q], g(c0[q])) : 0.0;
#pragma unroll
        for (int q = 0; q < Q; ++q) stage2[32 * q + lane] = t0[q];
    }
    __syncwarp();
    int buf = 0;
    for (int k0 = b; k0 < e; k0 += kStage) {
        const int cnt = min(kStage, e - k0);
        const int ka = k0 + kStage;  // round r + 1
        // round r + 1's gathers and round r + 2's indices and values
        double g1[Q];
#pragma unroll
        for (int q = 0; q < Q; ++q) g1[q] = ka + 32 * q + lane < e ? g(c1[q]) : 0.0;
        int c2[Q];
        double w2[Q];
        load_cv(ka + kStage, c2, w2);
        // add round r
        const double* cur = stage2 + buf * kStage;
        if (cnt == kStage) {
            const double2* s2 = reinterpret_cast<const double2*>(cur);
#pragma unroll 8
            for (int i = 0; i < kStage / 2; ++i) {
                const double2 p = s2[i];
                acc = __dadd_rn(acc, p.x);
                acc = __dadd_rn(acc, p.y);
            }
        } else {
            for (int i = 0; i < cnt; ++i) acc = __dadd_rn(acc, cur[i]);
        }
        // round r + 1's terms into the other buffer
        double* nxt = stage2 + (buf ^ 1) * kStage;
#pragma unroll
        for (int q = 0; q < Q; ++q)
            nxt[32 * q + lane] = ka + 32 * q + lane < e ? __dmul_rn(w1[q], g1[q]) : 0.0;
        __syncwarp();  // every lane has added `cur` and written `nxt`
        buf ^= 1;
#pragma unroll
        for (int q = 0; q < Q; ++q) {
            c1[q] = c2[q];
            w1[q] = w2[q];
        }
    }
    return acc;
}

// Two rounds of kStage doubles per warp for ordered_dot_warp_pipelined.
__device__ __forceinline__ double* warp_stage2() {
    __shared__ __align__(16) double stage2[kWarps][2 * kStage];
    return stage2[threadIdx.x >> 5];
}

// Row assignment of the ordered kernels over one matrix: rows of at most
// kWarpRow entries take one thread each (blocks [0, ordered_blocks(rows))); the
// longer rows listed in M.wrows take one warp each (the next warp_blocks(M)
// blocks), so a row of thousands of entries streams through 32 lanes instead
// of one. A matrix without the list runs every row on one thread.
__host__ __device__ inline int warp_blocks(const DevCsr& M) {
    return M.wrows != nullptr ? (M.n_wrows + kWarps - 1) / kWarps : 0;
}
__host__ __device__ inline int mat_blocks(const DevCsr& M) {
    return ordered_blocks(M.rows) + warp_blocks(M);
}

struct RowTask {
    int row = -1;       // -1: no row for this thread
    bool warp = false;  // the 32 lanes of this warp share the row
    bool lead = false;  // this thread stores the row's results
};

// `blk` is the block index within this matrix's range of blocks. Warp
// assignments are uniform across the warp.
__device__ __forceinline__ RowTask row_task(const DevCsr& M, int blk) {
    RowTask t;
    const int tb = ordered_blocks(M.rows);
    if (blk < tb) {
        const int r = blk * kBlock + threadIdx.x;
        if (r < M.rows && (M.wrows == nullptr || M.rp[r + 1] - M.rp[r] <= kWarpRow)) {
            t.row = r;
            t.lead = true;
        }
    } else {
        const int w = (blk - tb) * kWarps + (threadIdx.x >> 5);
        if (w < M.n_wrows) {
            t.row = M.wrows[w];
            t.warp = true;
            t.lead = (threadIdx.x & 31) == 0;
        }
    }
    return t;
}

// acc = init + sum_k v[k] * g(ci[k]) over row t.row in k order, by one thread
// or by the row's warp (all lanes of a warp row must call it).
template <class G>
__device__ __forceinline__ double row_dot(const RowTask& t, const DevCsr& M, G g, double init) {
    const int b = M.rp[t.row], e = M.rp[t.row + 1];
    if (!t.warp) return ordered_dot(b, e, M.ci, M.v64, g, init);
    const int32_t* __restrict__ ci = M.ci;
    const double* __restrict__ v = M.v64;
    return ordered_sum_warp(b, e, [=](int k) { return __dmul_rn(v[k], g(ci[k])); }, init,
                            warp_stage());
}

}  // namespace pdhg
