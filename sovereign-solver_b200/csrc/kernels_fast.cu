// kernels_fast.cu -- the throughput kernels (FP32-mixed and FP64-fast modes).
//
// One PDHG iteration is two launches, each an SpMV with the reference's
// row-local update fused into its epilogue (src/l1/pdhg.cpp:295-331):
//
//   primal: over the rows of A^T (= columns of A): grad = c - A^T y,
//           x+ = proj_X(x - tau grad), x_bar = 2x+ - x, Cesaro sum.
//   dual:   over the rows of A: s+ = proj_S(s - tau y), s_bar = 2s+ - s,
//           y += sigma (s_bar - A x_bar), Cesaro sum.
//
// Work split by row length (one or two launches per pass, see below):
//   rows of <= short_max nonzeros     VW lanes per row (VW = power of two ~
//                                     mean length), lanes stride the row in
//                                     rounds of four loads, shuffle reduction;
//   rows of short_max..kLongRow       one warp per row, 128-bit vector loads
//   (mode 1: ..kHugeRow)              of values and indices, shuffle reduction;
//   longer rows                       CTA work items of at most kSegLen
//                                     entries (a row of more is split into
//                                     segments whose partials the last CTA
//                                     adds in segment order), block reduction.
// The epilogue of a short row runs on the group's lane 0, so consecutive
// groups touch consecutive vector entries (coalesced).
//
// The check (every restart_check_period iterations) is ONE fused kernel: FP64
// values, the current point and the Cesaro average in the same pass, scaled
// residuals (kkt_residual, pdhg.cpp:87-136) and original-space residuals
// (original_space_residual, pdhg.cpp:145-199) derived elementwise from the
// scaled products: A_o x_o = D_r^-1 (A_s x_s) and (c - A^T y)_o = r_s / D_c.
// Its last CTA takes the candidate / termination / restart decision.
#include <algorithm>
#include <type_traits>

#include "engine.cuh"
#include "fast_common.cuh"

// CTAs per SM the iteration kernels are compiled to fit (register budget);
// build knobs, 1 = no constraint. The short-row kernel is lean: eight CTAs
// (32 registers) fit in FP32, six in FP64 without spills. The long-row kernel
// with only CTA items fits six; with the warp-row path as well, four (64
// registers; a few bytes of spill in FP32).
#ifndef PDHG_SHORT_MIN_CTAS
#define PDHG_SHORT_MIN_CTAS 8
#endif
#ifndef PDHG_SHORT_MIN_CTAS_F64
#define PDHG_SHORT_MIN_CTAS_F64 6
#endif
#ifndef PDHG_LONG_MIN_CTAS
#define PDHG_LONG_MIN_CTAS 6
#endif
#ifndef PDHG_WARPROW_MIN_CTAS
#define PDHG_WARPROW_MIN_CTAS 4
#endif
#ifndef PDHG_WARPITEM_MIN_CTAS
#define PDHG_WARPITEM_MIN_CTAS 4
#endif
#ifndef PDHG_UNIFORM_MIN_CTAS
#define PDHG_UNIFORM_MIN_CTAS 8
#endif
#ifndef PDHG_UNIFORM_MIN_CTAS_E4
#define PDHG_UNIFORM_MIN_CTAS_E4 6
#endif
#ifndef PDHG_UNIFORM_MIN_CTAS_F64
#define PDHG_UNIFORM_MIN_CTAS_F64 4
#endif
// FP32 slice kernel without the warp items: 40 registers, no spill
#ifndef PDHG_SLICE_MIN_CTAS_NW
#define PDHG_SLICE_MIN_CTAS_NW 6
#endif
#ifndef PDHG_SLICE_MIN_CTAS
#define PDHG_SLICE_MIN_CTAS 4
#endif

namespace pdhg {

namespace {

// ---------------------------------------------------------------------------
// Iteration kernels
// ---------------------------------------------------------------------------
//
// One SpMV-plus-update pass is split by row length into two kernels, so the
// short-row kernel keeps its registers (and occupancy) low:
//   fast_iter       rows of at most short_max entries, groups of VW lanes;
//   fast_iter_long  longer rows: one warp each up to kLongRow entries and CTA
//                   work items above (long_mode 0), or one warp each up to
//                   kHugeRow entries and CTA work items above (long_mode 1);
//   fast_iter_witems  or all of them as warp work items (long_mode 2).
// `reset` is set on the first kernel of a period's first pass: it clears the
// flags the previous period's restart kernel consumed.

__device__ __forceinline__ void iter_reset(DevState* st, int reset) {
    if (reset && blockIdx.x == 0 && threadIdx.x == 0) {
        st->restart = 0;
        st->fold = 0;
    }
}

// Two consecutive values of a row, loaded as one vector.
template <class T>
struct Pair;
template <>
struct Pair<float> {
    using type = float2;
};
template <>
struct Pair<double> {
    using type = double2;
};
template <class T>
__device__ __forceinline__ bool pair_aligned(const int32_t* ci, const T* v) {
    return ((reinterpret_cast<uintptr_t>(ci) & 7u) | (reinterpret_cast<uintptr_t>(v) & (2 * sizeof(T) - 1))) == 0;
}
template <class T>
__device__ __forceinline__ T fma_rn(T a, T b, T c) {
    if constexpr (std::is_same<T, float>::value) return __fmaf_rn(a, b, c);
    else return __fma_rn(a, b, c);
}
template <class T>
__device__ __forceinline__ T mul_rn(T a, T b) {
    if constexpr (std::is_same<T, float>::value) return __fmul_rn(a, b);
    else return __dmul_rn(a, b);
}

// The dot of long row `row` over entries [b, e), by one CTA (block-uniform)
// or one warp (warp-uniform); a dense row computes its columns.
template <class T>
__device__ __forceinline__ T cta_row_dot(const DevCsr& M, const T* vals, const T* xg, int row, int b,
                                         int e) {
    const int off = M.dense_off ? __ldg(M.dense_off + row) : kNotDense;
    if (off != kNotDense) return long_row_dot<T, true>(M.ci, vals, xg, b, e, off);
    return long_row_dot<T>(M.ci, vals, xg, b, e);
}
template <class T>
__device__ __forceinline__ T warp_dot(const DevCsr& M, const T* vals, const T* xg, int row, int b,
                                      int e) {
    return warp_row_dot<T>(M.ci, vals, xg, b, e, M.dense_off ? __ldg(M.dense_off + row) : kNotDense);
}

// PRIMAL = true: rows of A^T gather y; false: rows of A gather x_bar.
template <class T, int VW, bool PRIMAL>
__global__ void __launch_bounds__(kBlock, sizeof(T) == 4 ? PDHG_SHORT_MIN_CTAS : PDHG_SHORT_MIN_CTAS_F64)
    fast_iter(FastIter<T> a, int first, int reset) {
    DevState* st = a.st;
    iter_reset(st, reset);
    if (st->done) return;
    const DevCsr& M = PRIMAL ? a.AT : a.A;
    const T* __restrict__ vals = mvals<T>(M);
    const T* __restrict__ xg = PRIMAL ? a.it.y : a.it.xbar;
    const PV<T> pv = pvec<T>(a.P);
    const bool fresh = first && st->fresh;
    const T tau = static_cast<T>(st->tau), sigma = static_cast<T>(st->sigma);
    const Hw<T> hw = halpern_weight_warp<T>(a.it, st, a.hk);
    const int lane = threadIdx.x & (VW - 1);
    const int r = (blockIdx.x * kBlock + threadIdx.x) / VW;
    if (r >= M.rows) return;
    EpiIn<T> in{};
    if (lane == 0) in = epi_load<T, PRIMAL>(a.it, pv, r, first, fresh, hw);
    int b, e;
    if (M.rp_stride > 0) {  // rows of one length: the extent is computed
        b = r * M.rp_stride;
        e = b + M.rp_stride;
    } else {
        b = __ldcs(M.rp + r);
        e = __ldcs(M.rp + r + 1);
    }
    if (e - b > M.short_max) return;  // fast_iter_long handles it
    T acc = T(0);
    if (VW == 1 && M.rp_stride == 2 && pair_aligned<T>(M.ci, vals)) {
        // two entries per row (the columns of a transportation LP): one
        // 8-byte index load and one vector value load, the same sum order as
        // the loop below
        const int2 c2 = __ldcs(reinterpret_cast<const int2*>(M.ci + b));
        const typename Pair<T>::type v2 = __ldcs(reinterpret_cast<const typename Pair<T>::type*>(vals + b));
        const T g0 = __ldg(xg + c2.x), g1 = __ldg(xg + c2.y);
        acc = fma_rn<T>(v2.y, g1, mul_rn<T>(v2.x, g0));
        epi_store<T, PRIMAL>(a.it, r, acc, in, tau, sigma, hw, a.tz);
        return;
    }
    // rounds of four entries per lane: the index and value loads of a round
    // are all in flight before its gathers, the gathers before the adds
    for (int k0 = b + lane; k0 < e; k0 += 4 * VW) {
        int c[4];
        T v[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int k = k0 + u * VW;
            c[u] = k < e ? __ldcs(M.ci + k) : 0;
            v[u] = k < e ? __ldcs(vals + k) : T(0);
        }
#pragma unroll
        for (int u = 0; u < 4; ++u)
            if (k0 + u * VW < e) acc += v[u] * __ldg(xg + c[u]);
    }
    if (VW > 1) acc = group_sum(acc, VW);
    if (lane == 0) epi_store<T, PRIMAL>(a.it, r, acc, in, tau, sigma, hw, a.tz);
}

// E consecutive column indices / values of one lane, as one or two vector loads.
template <int E>
__device__ __forceinline__ void load_idx(const int32_t* p, int (&c)[E]) {
    if constexpr (E == 2) {
        const int2 q = __ldcs(reinterpret_cast<const int2*>(p));
        c[0] = q.x;
        c[1] = q.y;
    } else {
        const int4 q = __ldcs(reinterpret_cast<const int4*>(p));
        c[0] = q.x;
        c[1] = q.y;
        c[2] = q.z;
        c[3] = q.w;
    }
}
template <class T, int E>
__device__ __forceinline__ void load_vals(const T* p, T (&v)[E]) {
    if constexpr (std::is_same<T, float>::value) {
        if constexpr (E == 2) {
            const float2 q = __ldcs(reinterpret_cast<const float2*>(p));
            v[0] = q.x;
            v[1] = q.y;
        } else {
            const float4 q = __ldcs(reinterpret_cast<const float4*>(p));
            v[0] = q.x;
            v[1] = q.y;
            v[2] = q.z;
            v[3] = q.w;
        }
    } else {
#pragma unroll
        for (int h = 0; h < E / 2; ++h) {
            const double2 q = __ldcs(reinterpret_cast<const double2*>(p) + h);
            v[2 * h] = q.x;
            v[2 * h + 1] = q.y;
        }
    }
}

// Rows of one length S = E * VW (rp_stride 2, 4 or 8: the columns of a
// network or transportation LP have 2 entries, those of config 2's LP 8), a
// persistent grid (the resident CTAs): groups of VW lanes, lane l owning the
// row's entries [l E, (l + 1) E) as one index and one value vector load. Each
// group walks rows r, r + G, r + 2G, ... (G groups in the grid, so a warp's
// rows stay consecutive) and pipelines them: the next row's operand, index
// and value loads are issued before the current row's gathers are used, so
// the streamed arrays stay in flight while the gathers wait. One row per
// thread (fast_iter) leaves DRAM idle during every thread's gather phase and
// while CTAs retire and launch. A lane sums its E products in order, then the
// group adds its lanes (the two-entry rows' order is fast_iter's).
template <class T, int E, int VW>
constexpr int uniform_min_ctas() {
    return sizeof(T) == 8 ? PDHG_UNIFORM_MIN_CTAS_F64 : (E == 2 ? PDHG_UNIFORM_MIN_CTAS : PDHG_UNIFORM_MIN_CTAS_E4);
}

template <class T, int E, int VW, bool PRIMAL>
__global__ void __launch_bounds__(kBlock, (uniform_min_ctas<T, E, VW>()))
    fast_iter_uniform(FastIter<T> a, int first, int reset) {
    constexpr int S = E * VW;
    DevState* st = a.st;
    iter_reset(st, reset);
    if (st->done) return;
    const DevCsr& M = PRIMAL ? a.AT : a.A;
    const T* __restrict__ xg = PRIMAL ? a.it.y : a.it.xbar;
    const T* __restrict__ vals = mvals<T>(M);
    const PV<T> pv = pvec<T>(a.P);
    const bool fresh = first && st->fresh;
    const T tau = static_cast<T>(st->tau), sigma = static_cast<T>(st->sigma);
    const Hw<T> hw = halpern_weight_warp<T>(a.it, st, a.hk);
    const int lane = threadIdx.x & (VW - 1);
    const int groups = gridDim.x * (kBlock / VW);
    int r = (blockIdx.x * kBlock + static_cast<int>(threadIdx.x)) / VW;
    if (r >= M.rows) return;  // group-uniform
    EpiIn<T> in{};
    if (lane == 0) in = epi_load<T, PRIMAL>(a.it, pv, r, first, fresh, hw);
    int c[E];
    T v[E];
    load_idx<E>(M.ci + static_cast<int64_t>(r) * S + lane * E, c);
    load_vals<T, E>(vals + static_cast<int64_t>(r) * S + lane * E, v);
    for (;;) {
        T g[E];
#pragma unroll
        for (int q = 0; q < E; ++q) g[q] = __ldg(xg + c[q]);
        const int rn = r + groups;
        const bool more = rn < M.rows;  // group-uniform
        EpiIn<T> nin{};
        int nc[E];
        T nv[E];
        if (more) {
            if (lane == 0) nin = epi_load<T, PRIMAL>(a.it, pv, rn, first, fresh, hw);
            load_idx<E>(M.ci + static_cast<int64_t>(rn) * S + lane * E, nc);
            load_vals<T, E>(vals + static_cast<int64_t>(rn) * S + lane * E, nv);
        }
        T acc = mul_rn<T>(v[0], g[0]);
#pragma unroll
        for (int q = 1; q < E; ++q) acc = fma_rn<T>(v[q], g[q], acc);
        if (VW > 1) acc = group_sum(acc, VW);
        if (lane == 0) epi_store<T, PRIMAL>(a.it, r, acc, in, tau, sigma, hw, a.tz);
        if (!more) break;
        r = rn;
        in = nin;
#pragma unroll
        for (int q = 0; q < E; ++q) {
            c[q] = nc[q];
            v[q] = nv[q];
        }
    }
}

// One CTA work item of L (block-uniform): the dot of its entries, then for a
// whole row its update, for a segment its partial and ticket (and the row's
// update when this CTA completes the row).
template <class T, bool PRIMAL>
__device__ __forceinline__ void cta_item(const FastIter<T>& a, const DevCsr& M, const RowItems& L,
                                         int idx, int first, bool fresh, T tau, T sigma, Hw<T> hw) {
    const T* __restrict__ vals = mvals<T>(M);
    const T* __restrict__ xg = PRIMAL ? a.it.y : a.it.xbar;
    const PV<T> pv = pvec<T>(a.P);
    const int4 w = __ldg(L.item + idx);
    T acc = cta_row_dot<T>(M, vals, xg, w.x, w.y, w.z);
    if (w.w >= 0) {  // block-uniform
        double tot, unused;
        if (!segment_finish(L, idx, w.w, static_cast<double>(acc), 0.0, &tot, &unused)) return;
        acc = static_cast<T>(tot);
    }
    // the row's operands are loaded after its dot (rows here are long: the
    // load's latency is small beside the dot, and nothing stays live across it)
    if (threadIdx.x == 0) {
        const EpiIn<T> in = epi_load<T, PRIMAL>(a.it, pv, w.x, first, fresh, hw);
        epi_store<T, PRIMAL>(a.it, w.x, acc, in, tau, sigma, hw, a.tz);
    }
}

// WARPS = true: the first warp_blocks CTAs take the warp rows, one CTA per
// item after them. WARPS = false (the pass has no warp rows in this mode):
// a persistent grid (the resident CTAs) claims items one by one from L.fetch,
// so no wave of CTAs ends half empty; the warp path is compiled out, so more
// CTAs fit per SM.
template <class T, bool PRIMAL, int MODE, bool WARPS>
__global__ void __launch_bounds__(kBlock, WARPS ? PDHG_WARPROW_MIN_CTAS : PDHG_LONG_MIN_CTAS)
    fast_iter_long(FastIter<T> a, int first, int reset, int warp_blocks) {
    DevState* st = a.st;
    iter_reset(st, reset);
    if (st->done) return;
    const DevCsr& M = PRIMAL ? a.AT : a.A;
    const bool fresh = first && st->fresh;
    const T tau = static_cast<T>(st->tau), sigma = static_cast<T>(st->sigma);
    const Hw<T> hw = halpern_weight_warp<T>(a.it, st, a.hk);
    const RowItems& L = MODE == 0 ? M.items_long : M.items_huge;
    if (!WARPS) {
        for (;;) {
            const int idx = cta_fetch(L.fetch);
            if (idx >= L.n_item) break;
            cta_item<T, PRIMAL>(a, M, L, idx, first, fresh, tau, sigma, hw);
        }
        cta_exit(L.fetch);
        return;
    }
    if (static_cast<int>(blockIdx.x) < warp_blocks) {
        // one warp per row: rows above short_max up to kLongRow (mode 0) or
        // kHugeRow (mode 1) entries
        const int w = blockIdx.x * (kBlock / 32) + (threadIdx.x >> 5);
        if (w >= (MODE == 0 ? M.n_warp0 : M.n_warp1)) return;
        const int r = __ldg((MODE == 0 ? M.warp_rows0 : M.warp_rows1) + w);
        const int lane = threadIdx.x & 31;
        const PV<T> pv = pvec<T>(a.P);
        EpiIn<T> in{};
        if (lane == 0) in = epi_load<T, PRIMAL>(a.it, pv, r, first, fresh, hw);
        const T acc = warp_dot<T>(M, mvals<T>(M), PRIMAL ? a.it.y : a.it.xbar, r, __ldg(M.rp + r),
                                  __ldg(M.rp + r + 1));
        if (lane == 0) epi_store<T, PRIMAL>(a.it, r, acc, in, tau, sigma, hw, a.tz);
    } else {
        // CTA work items: rows above kLongRow (mode 0) or kHugeRow (mode 1),
        // those above the segment length in segments
        cta_item<T, PRIMAL>(a, M, L, static_cast<int>(blockIdx.x) - warp_blocks, first, fresh,
                            tau, sigma, hw);
    }
}

// One warp work item of long_mode 2 (warp-uniform): a whole row, or a segment
// of a longer one whose last warp adds the segments in order.
template <class T, bool PRIMAL>
__device__ __forceinline__ void warp_item(const FastIter<T>& a, const DevCsr& M, const RowItems& L,
                                          int idx, int first, bool fresh, T tau, T sigma, Hw<T> hw) {
    const T* __restrict__ vals = mvals<T>(M);
    const T* __restrict__ xg = PRIMAL ? a.it.y : a.it.xbar;
    const PV<T> pv = pvec<T>(a.P);
    const int lane = threadIdx.x & 31;
    const int4 w = __ldg(L.item + idx);
    EpiIn<T> in{};
    if (lane == 0 && w.w < 0) in = epi_load<T, PRIMAL>(a.it, pv, w.x, first, fresh, hw);
    T acc = warp_dot<T>(M, vals, xg, w.x, w.y, w.z);
    if (w.w >= 0) {  // warp-uniform
        double tot;
        if (!warp_segment_finish(L, idx, w.w, static_cast<double>(acc), &tot)) return;
        acc = static_cast<T>(tot);
        if (lane == 0) in = epi_load<T, PRIMAL>(a.it, pv, w.x, first, fresh, hw);
    }
    if (lane == 0) epi_store<T, PRIMAL>(a.it, w.x, acc, in, tau, sigma, hw, a.tz);
}

// long_mode 2: every row above short_max as warp work items; no block barrier
// anywhere, each warp finishes on its own.
template <class T, bool PRIMAL>
__global__ void __launch_bounds__(kBlock, PDHG_WARPITEM_MIN_CTAS)
    fast_iter_witems(FastIter<T> a, int first, int reset) {
    DevState* st = a.st;
    iter_reset(st, reset);
    if (st->done) return;
    const DevCsr& M = PRIMAL ? a.AT : a.A;
    const int idx = blockIdx.x * (kBlock / 32) + (threadIdx.x >> 5);
    if (idx >= M.items_warp.n_item) return;
    const bool fresh = first && st->fresh;
    const T tau = static_cast<T>(st->tau), sigma = static_cast<T>(st->sigma);
    const Hw<T> hw = halpern_weight_warp<T>(a.it, st, a.hk);
    warp_item<T, PRIMAL>(a, M, M.items_warp, idx, first, fresh, tau, sigma, hw);
}

template <class T>
__device__ __forceinline__ const T* slice_vals(const RowSlices& S);
template <>
__device__ __forceinline__ const float* slice_vals<float>(const RowSlices& S) { return S.v32; }
template <>
__device__ __forceinline__ const double* slice_vals<double>(const RowSlices& S) { return S.v64; }

// Lane l's dot product over steps [k0, k1) of a slice (k below kend), in
// rounds of eight: the next round's index and value loads are issued before
// this round's gathers.
template <class T>
__device__ __forceinline__ T slice_dot(const RowSlices& S, int off, int k0s, int k1, int kend, int lane,
                                       const T* __restrict__ xg) {
    const int32_t* __restrict__ col = S.col + off + lane;
    const T* __restrict__ val = slice_vals<T>(S) + off + lane;
    auto colk = [&](int k) -> int { return __ldcs(col + 32 * static_cast<int64_t>(k)); };
    T acc = T(0);
    int c[8];
    T v[8];
#pragma unroll
    for (int u = 0; u < 8; ++u) {
        const int k = k0s + u;
        c[u] = k < kend ? colk(k) : 0;
        v[u] = k < kend ? __ldcs(val + 32 * static_cast<int64_t>(k)) : T(0);
    }
    for (int k0 = k0s; k0 < k1; k0 += 8) {
        int cn[8];
        T vn[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            const int k = k0 + 8 + u;
            cn[u] = k < kend ? colk(k) : 0;
            vn[u] = k < kend ? __ldcs(val + 32 * static_cast<int64_t>(k)) : T(0);
        }
#pragma unroll
        for (int u = 0; u < 8; ++u)
            if (k0 + u < kend) acc += v[u] * __ldg(xg + c[u]);
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            c[u] = cn[u];
            v[u] = vn[u];
        }
    }
    return acc;
}

// The same dot over an affine slice (columns base + l + k stride, checked
// entry by entry at load): both streams, the lane-interleaved values and
// x_bar, have computed addresses, so a lane keeps 16 (FP64: 8) steps of both
// in flight per round; the sum runs in k order like slice_dot's.
template <class T>
__device__ __forceinline__ T slice_dot_affine(const RowSlices& S, int off, int k0s, int k1, int kend,
                                              int lane, const T* __restrict__ xg, int2 af) {
    constexpr int U = sizeof(T) == 4 ? 16 : 8;
    const T* __restrict__ val = slice_vals<T>(S) + off + lane;
    const T* __restrict__ g = xg + af.x + lane;
    T acc = T(0);
    for (int k0 = k0s; k0 < k1; k0 += U) {
        T v[U], x[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int k = k0 + u;
            const bool ok = k < kend;
            v[u] = ok ? __ldcs(val + 32 * static_cast<int64_t>(k)) : T(0);
            x[u] = ok ? __ldg(g + static_cast<int64_t>(k) * af.y) : T(0);
        }
#pragma unroll
        for (int u = 0; u < U; ++u)
            if (k0 + u < kend) acc += v[u] * x[u];
    }
    return acc;
}

// One warp item of the row slices (warp-uniform): entries [k0, k1) of one
// slice, lane l on the slice's row l, in rounds of eight steps; each step is
// one coalesced index load, one coalesced value load and one gather per lane.
// The next round's index and value loads are issued before this round's
// gathers, so the matrix stream and the gathers overlap. A slice cut into
// several items: every lane stores its partial, lane 0 takes the slice's
// ticket, and the last warp adds each lane's partials in item order (four
// interleaved sums, fixed) before the 32 rows' updates.
template <class T, bool PRIMAL>
__device__ __forceinline__ void slice_item(const FastIter<T>& a, const RowSlices& S, int idx,
                                           int first, bool fresh, T tau, T sigma, Hw<T> hw) {
    const int lane = threadIdx.x & 31;
    const int4 w = __ldg(S.item + idx);
    const int4 d = __ldg(S.slice + w.x);
    const int row = __ldg(S.row + 32 * w.x + lane);
    const int kend = min(w.z, __ldg(S.rlen + 32 * w.x + lane));
    const T* __restrict__ xg = PRIMAL ? a.it.y : a.it.xbar;
    // an affine slice's columns are computed, not loaded (warp-uniform)
    const int2 af = __ldg(S.affine + w.x);
    T acc = af.y > 0 ? slice_dot_affine<T>(S, d.y, w.y, w.z, kend, lane, xg, af)
                     : slice_dot<T>(S, d.y, w.y, w.z, kend, lane, xg);
    if (w.w >= 0) {
        S.part[32 * static_cast<int64_t>(idx) + lane] = static_cast<double>(acc);
        __threadfence();
        __syncwarp();
        const int2 sp = __ldg(S.split + w.w);
        int last = 0;
        if (lane == 0) last = atomicAdd(S.ticket + w.w, 1u) == static_cast<unsigned>(sp.y - 1) ? 1 : 0;
        last = __shfl_sync(0xffffffffu, last, 0);
        if (!last) return;
        __threadfence();
        double t0 = 0.0, t1 = 0.0, t2 = 0.0, t3 = 0.0;
        int q = sp.x;
        const int qe = sp.x + sp.y;
        for (; q + 4 <= qe; q += 4) {
            t0 += __ldcg(S.part + 32 * static_cast<int64_t>(q) + lane);
            t1 += __ldcg(S.part + 32 * static_cast<int64_t>(q + 1) + lane);
            t2 += __ldcg(S.part + 32 * static_cast<int64_t>(q + 2) + lane);
            t3 += __ldcg(S.part + 32 * static_cast<int64_t>(q + 3) + lane);
        }
        for (; q < qe; ++q) t0 += __ldcg(S.part + 32 * static_cast<int64_t>(q) + lane);
        if (lane == 0) S.ticket[w.w] = 0u;
        acc = static_cast<T>((t0 + t1) + (t2 + t3));
    }
    if (row < 0) return;
    const PV<T> pv = pvec<T>(a.P);
    const EpiIn<T> in = epi_load<T, PRIMAL>(a.it, pv, row, first, fresh, hw);
    epi_store<T, PRIMAL>(a.it, row, acc, in, tau, sigma, hw, a.tz);
}

// The row-slice kernel: a persistent grid (the resident CTAs) whose warps
// claim items one by one from S.fetch. With long_mode 2 (WITEMS) the queue
// goes on past the slice items into the warp items of the other long rows, so
// one kernel and one tail cover every long row of the pass.
template <class T, bool PRIMAL, bool WITEMS>
__global__ void __launch_bounds__(kBlock, (sizeof(T) == 4 && !WITEMS) ? PDHG_SLICE_MIN_CTAS_NW
                                                                      : PDHG_SLICE_MIN_CTAS)
    fast_iter_slices(FastIter<T> a, int first, int reset) {
    DevState* st = a.st;
    iter_reset(st, reset);
    if (st->done) return;
    const DevCsr& M = PRIMAL ? a.AT : a.A;
    const RowSlices& S = M.slices;
    const bool fresh = first && st->fresh;
    const T tau = static_cast<T>(st->tau), sigma = static_cast<T>(st->sigma);
    const Hw<T> hw = halpern_weight_warp<T>(a.it, st, a.hk);
    const int ns = S.n_item;
    const int nt = ns + (WITEMS ? M.items_warp.n_item : 0);
    for (;;) {
        const int idx = warp_fetch(S.fetch);
        if (idx >= nt) break;
        if (!WITEMS || idx < ns) slice_item<T, PRIMAL>(a, S, idx, first, fresh, tau, sigma, hw);
        else warp_item<T, PRIMAL>(a, M, M.items_warp, idx - ns, first, fresh, tau, sigma, hw);
    }
    warp_exit(S.fetch);
}

__global__ void k_clear_flags(DevState* st) {
    if (threadIdx.x == 0) {
        st->restart = 0;
        st->fold = 0;
    }
}

inline int iter_lanes(const DevCsr& M) { return M.iter_vw > 0 ? M.iter_vw : M.vw; }

inline int short_blocks_for(const DevCsr& M) {
    if (M.n_iter_short == 0) return 0;
    return static_cast<int>((static_cast<int64_t>(M.rows) * iter_lanes(M) + kBlock - 1) / kBlock);
}

// The matrix a pass runs on: with the row slices in use, the long-row tiers
// without the slices' rows replace the full ones.
inline DevCsr pass_matrix(const DevCsr& M) {
    if (!M.use_slices || M.slices.n_item == 0) return M;
    DevCsr X = M;
    const LongTiers& t = M.no_slice_tiers;
    X.warp_rows0 = t.warp_rows0;
    X.warp_rows1 = t.warp_rows1;
    X.n_warp0 = t.n_warp0;
    X.n_warp1 = t.n_warp1;
    X.items_long = t.items_long;
    X.items_huge = t.items_huge;
    X.items_warp = t.items_warp;
    return X;
}

// CTAs of a pass's kernels: short rows, the long-row kernel (of which the
// first `warp` run warp rows), the row slices.
struct PassPlan {
    int shrt = 0, warp = 0, lng = 0, slc = 0;
};

// Resident CTAs per device of the persistent kernels ([0] FP32, [1] FP64): the
// CTA-item kernel without warp rows and the row-slice kernel. Their grids are
// capped at these (set by init_fast_kernels from the occupancy calculator).
int g_cap_long[2] = {148 * PDHG_LONG_MIN_CTAS, 148 * PDHG_LONG_MIN_CTAS};
int g_cap_slice[2] = {148 * PDHG_SLICE_MIN_CTAS_NW, 148 * PDHG_SLICE_MIN_CTAS};
int g_cap_slice_w[2] = {148 * PDHG_SLICE_MIN_CTAS, 148 * PDHG_SLICE_MIN_CTAS};  // with warp items
// resident CTAs of the one-point check kernel, FP32 / FP64
int g_cap_check1[2] = {148 * 4, 148 * 4};
// resident CTAs of fast_iter_uniform for rows of 2, 4 and 8 entries, FP32 / FP64
int g_cap_uni[3][2] = {{148 * PDHG_UNIFORM_MIN_CTAS, 148 * PDHG_UNIFORM_MIN_CTAS_F64},
                       {148 * PDHG_UNIFORM_MIN_CTAS_E4, 148 * PDHG_UNIFORM_MIN_CTAS_F64},
                       {148 * PDHG_UNIFORM_MIN_CTAS_E4, 148 * PDHG_UNIFORM_MIN_CTAS_F64}};

inline PassPlan pass_plan(const DevCsr& M, int cap_long, int cap_slice, int cap_slice_w) {
    PassPlan p;
    if (M.rows == 0) return p;
    p.shrt = short_blocks_for(M);
    const int mode = M.long_mode;
    const bool sliced = M.use_slices && M.slices.n_item > 0;
    const int nw = mode == 2 ? M.items_warp.n_item : mode == 1 ? M.n_warp1 : M.n_warp0;
    p.warp = (nw + kBlock / 32 - 1) / (kBlock / 32);
    if (mode == 2 && sliced) {
        // the slice kernel takes the warp items too (fast_iter_slices)
        p.warp = 0;
        p.slc = std::min((M.slices.n_item + nw + kBlock / 32 - 1) / (kBlock / 32), std::max(cap_slice_w, 1));
        return p;
    }
    if (mode == 2) {
        p.lng = p.warp;
    } else {
        const int items = mode == 1 ? M.items_huge.n_item : M.items_long.n_item;
        // without warp rows the CTA-item kernel is persistent: resident CTAs only
        p.lng = p.warp > 0 ? p.warp + items : std::min(items, std::max(cap_long, 1));
    }
    if (M.use_slices && M.slices.n_item > 0)
        p.slc = std::min((M.slices.n_item + kBlock / 32 - 1) / (kBlock / 32), std::max(cap_slice, 1));
    return p;
}

// Kernels one pass over M launches besides the flag reset.
inline int pass_launches(const DevCsr& M0) {
    const PassPlan p = pass_plan(pass_matrix(M0), 1, 1, 1);
    return (p.shrt > 0 ? 1 : 0) + (p.lng > 0 ? 1 : 0) + (p.slc > 0 ? 1 : 0);
}

// Returns the number of kernels launched.
// Every row of 2, 4 or 8 entries, the arrays 16-byte aligned for the vector
// loads: the pass's short rows run fast_iter_uniform (slot 0, 1, 2), else -1.
template <class T>
int uniform_slot(const DevCsr& M) {
    const void* v = sizeof(T) == 4 ? static_cast<const void*>(M.v32) : static_cast<const void*>(M.v64);
    if (((reinterpret_cast<uintptr_t>(M.ci) | reinterpret_cast<uintptr_t>(v)) & 15u) != 0) return -1;
    return M.rp_stride == 2 ? 0 : M.rp_stride == 4 ? 1 : M.rp_stride == 8 ? 2 : -1;
}

template <class T, int E, int VW, bool PRIMAL>
void launch_uniform(const FastIter<T>& a, const DevCsr& M, int cap, int first, int reset,
                    cudaStream_t s) {
    const int64_t need = (static_cast<int64_t>(M.rows) * VW + kBlock - 1) / kBlock;
    const int grid = static_cast<int>(need < cap ? need : cap);
    fast_iter_uniform<T, E, VW, PRIMAL><<<grid, kBlock, 0, s>>>(a, first, reset);
}

template <class T, bool PRIMAL>
int launch_iter(const FastIter<T>& a0, int first, cudaStream_t s, const PassFork* f) {
    const DevCsr& M0 = PRIMAL ? a0.AT : a0.A;
    if (M0.rows == 0) {
        if (PRIMAL && first) {
            k_clear_flags<<<1, 32, 0, s>>>(a0.st);
            return 1;
        }
        return 0;
    }
    FastIter<T> a = a0;
    DevCsr& M = PRIMAL ? a.AT : a.A;
    M = pass_matrix(M0);
    const int pi = sizeof(T) == 4 ? 0 : 1;
    const PassPlan p = pass_plan(M, g_cap_long[pi], g_cap_slice[pi], g_cap_slice_w[pi]);
    const int mode = M.long_mode;
    // the flag reset rides on the first kernel of the period's first pass
    const int rs = PRIMAL && first ? 1 : 0;
    const int reset_short = rs;
    const int reset_long = rs && p.shrt == 0 ? 1 : 0;
    const int reset_slc = rs && p.shrt == 0 && p.lng == 0 ? 1 : 0;
    const int kernels = (p.shrt > 0) + (p.lng > 0) + (p.slc > 0);
    const bool fork = f != nullptr && f->side[0] != nullptr && kernels > 1;
    cudaStream_t ls = s, ss = s;
    if (fork) {
        cudaEventRecord(f->fork, s);
        cudaStreamWaitEvent(f->side[0], f->fork, 0);
        if (p.slc > 0) cudaStreamWaitEvent(f->side[1], f->fork, 0);
        ls = f->side[0];
        ss = f->side[1];
    }
    if (p.lng > 0 && mode == 2) {
        fast_iter_witems<T, PRIMAL><<<p.lng, kBlock, 0, ls>>>(a, first, reset_long);
    } else if (p.lng > 0) {
        const int mb = p.warp;
        if (mb == 0) {
            if (mode == 1) fast_iter_long<T, PRIMAL, 1, false><<<p.lng, kBlock, 0, ls>>>(a, first, reset_long, 0);
            else fast_iter_long<T, PRIMAL, 0, false><<<p.lng, kBlock, 0, ls>>>(a, first, reset_long, 0);
        } else {
            if (mode == 1) fast_iter_long<T, PRIMAL, 1, true><<<p.lng, kBlock, 0, ls>>>(a, first, reset_long, mb);
            else fast_iter_long<T, PRIMAL, 0, true><<<p.lng, kBlock, 0, ls>>>(a, first, reset_long, mb);
        }
    }
    if (p.slc > 0 && mode == 2)
        fast_iter_slices<T, PRIMAL, true><<<p.slc, kBlock, 0, ss>>>(a, first, reset_slc);
    else if (p.slc > 0)
        fast_iter_slices<T, PRIMAL, false><<<p.slc, kBlock, 0, ss>>>(a, first, reset_slc);
    const int us = p.shrt > 0 ? uniform_slot<T>(M) : -1;
    if (us == 0) launch_uniform<T, 2, 1, PRIMAL>(a, M, g_cap_uni[0][pi], first, reset_short, s);
    else if (us == 1) launch_uniform<T, 4, 1, PRIMAL>(a, M, g_cap_uni[1][pi], first, reset_short, s);
    else if (us == 2) launch_uniform<T, 4, 2, PRIMAL>(a, M, g_cap_uni[2][pi], first, reset_short, s);
    else if (p.shrt > 0) {
        const int sb = p.shrt;
        switch (iter_lanes(M)) {
            case 1: fast_iter<T, 1, PRIMAL><<<sb, kBlock, 0, s>>>(a, first, reset_short); break;
            case 2: fast_iter<T, 2, PRIMAL><<<sb, kBlock, 0, s>>>(a, first, reset_short); break;
            case 4: fast_iter<T, 4, PRIMAL><<<sb, kBlock, 0, s>>>(a, first, reset_short); break;
            case 8: fast_iter<T, 8, PRIMAL><<<sb, kBlock, 0, s>>>(a, first, reset_short); break;
            case 16: fast_iter<T, 16, PRIMAL><<<sb, kBlock, 0, s>>>(a, first, reset_short); break;
            default: fast_iter<T, 32, PRIMAL><<<sb, kBlock, 0, s>>>(a, first, reset_short); break;
        }
    }
    if (fork) {
        cudaEventRecord(f->join[0], f->side[0]);
        cudaStreamWaitEvent(s, f->join[0], 0);
        if (p.slc > 0) {
            cudaEventRecord(f->join[1], f->side[1]);
            cudaStreamWaitEvent(s, f->join[1], 0);
        }
    }
    return kernels;
}

// ---------------------------------------------------------------------------
// Check kernel
// ---------------------------------------------------------------------------

// Per-row terms, merged into the thread's running maxima / sums. INF: with
// the infeasibility tests (option infeasibility_detection), a separate
// instance so that the plain check keeps its registers.
template <class T, int F>
__device__ __forceinline__ void row_terms(const FastCheck<T>& a, int i, double act_c,
                                          double act_a, double inv, Terms& t) {
    constexpr bool INF = (F & kCheckInf) != 0;
    constexpr bool L2 = (F & kCheckL2) != 0;
    constexpr bool ONE = (F & kCheckOne) != 0;  // the current point's terms are not formed
    const DevProblem& P = a.P;
    a.cs.act_avg[i] = act_a;
    const double lo = P.rlo[i], hi = P.rhi[i];
    const double yc = ONE ? 0.0 : static_cast<double>(a.it.y[i]);
    const double ya = avg_y<T, ONE>(a.it, i, inv);
    if (!ONE) t.cp = smax(t.cp, primal_term(act_c, lo, hi));
    t.ap = smax(t.ap, primal_term(act_a, lo, hi));
    if (!ONE) t.cd = smax(t.cd, cs_term(yc, act_c, lo, hi, a.tol));
    t.ad = smax(t.ad, cs_term(ya, act_a, lo, hi, a.tol));
    const double rs = P.rs[i];
    const double lo_o = P.rlo_o[i], hi_o = P.rhi_o[i];
    const double aoc = act_c / rs, aoa = act_a / rs;
    if (!ONE) t.ocp = smax(t.ocp, primal_term(aoc, lo_o, hi_o));
    t.oap = smax(t.oap, primal_term(aoa, lo_o, hi_o));
    if (!ONE) t.ocd = smax(t.ocd, cs_term(yc * rs, aoc, lo_o, hi_o, a.bound_tol));
    t.oad = smax(t.oad, cs_term(ya * rs, aoa, lo_o, hi_o, a.bound_tol));
    if (a.termination_rule != 0) {  // internal (minimize) sense: y_int = y_s * rs
        if (!ONE) t.dobj_c += clipped_inf(yc * rs, lo_o, hi_o);
        t.dobj_a += clipped_inf(ya * rs, lo_o, hi_o);
    }
    if (L2) {  // termination rule 2: squares of the row violation and of y's sign violation
        const double pa = primal_term(aoa, lo_o, hi_o);
        const double da = sign_violation(ya * rs, lo_o, hi_o);
        if (!ONE) {
            const double pc = primal_term(aoc, lo_o, hi_o);
            const double dc = sign_violation(yc * rs, lo_o, hi_o);
            t.ppc += pc * pc;
            t.ddc += dc * dc;
        }
        t.ppa += pa * pa;
        t.dda += da * da;
    }
    if (INF) {  // the change of y since the previous check, original units
        const double dy = P.obj_sign * rs * (yc - a.ray_y_prev[i]);
        a.ray_y_prev[i] = yc;
        a.ray_y[i] = dy;
        ray_term(dy, lo_o, hi_o, t.rlo, t.rhi);
        t.raymax = smax(t.raymax, fabs(dy));
    }
}

template <class T, int F>
__device__ __forceinline__ void col_terms(const FastCheck<T>& a, int j, double aty_c,
                                          double aty_a, double inv, Terms& t) {
    constexpr bool INF = (F & kCheckInf) != 0;
    constexpr bool L2 = (F & kCheckL2) != 0;
    constexpr bool ONE = (F & kCheckOne) != 0;  // the current point's terms are not formed
    const DevProblem& P = a.P;
    const double cj = P.c[j];
    const double lo = P.col_bounds_uniform ? P.lo_u : P.lo[j];
    const double hi = P.col_bounds_uniform ? P.hi_u : P.hi[j];
    const double xc = ONE ? 0.0 : static_cast<double>(a.it.x[j]);
    const double xa = avg_x<T, ONE>(a.it, j, inv);
    const double rc = cj - aty_c, ra = cj - aty_a;
    if (!ONE) t.cd = smax(t.cd, cs_term(rc, xc, lo, hi, a.tol));
    t.ad = smax(t.ad, cs_term(ra, xa, lo, hi, a.tol));
    const double cs = P.cs[j];
    const double lo_o = P.col_bounds_uniform_o ? P.lo_uo : P.lo_o[j];
    const double hi_o = P.col_bounds_uniform_o ? P.hi_uo : P.hi_o[j];
    if (!ONE) t.ocd = smax(t.ocd, cs_term(rc / cs, xc * cs, lo_o, hi_o, a.bound_tol));
    t.oad = smax(t.oad, cs_term(ra / cs, xa * cs, lo_o, hi_o, a.bound_tol));
    if (L2) {  // termination rule 2: squares of the reduced cost's sign violation
        if (!ONE) {
            const double dc = sign_violation(rc / cs, lo_o, hi_o);
            t.ddc += dc * dc;
        }
        const double da = sign_violation(ra / cs, lo_o, hi_o);
        t.dda += da * da;
    }
    if (a.termination_rule != 0) {  // internal sense: c_int x = sign c_o x, r_int = r_s / cs
        if (!ONE) {
            t.pobj_c += P.obj_sign * P.c_o[j] * (xc * cs);
            t.dobj_c += clipped_inf(rc / cs, lo_o, hi_o);
        }
        t.pobj_a += P.obj_sign * P.c_o[j] * (xa * cs);
        t.dobj_a += clipped_inf(ra / cs, lo_o, hi_o);
    }
    if (INF) {  // d = A_o^T dy_o = sign (A_s^T dy_s) / cs, by linearity
        const double dd = P.obj_sign * (aty_c - a.ray_aty_prev[j]) / cs;
        a.ray_aty_prev[j] = aty_c;
        ray_term(dd, lo_o, hi_o, t.clo, t.chi);
        // ray test: the change of x since the previous check, projected onto
        // the recession cone of the column's bounds (no decrease at a finite
        // lower end, no increase at a finite upper end), into the buffer the
        // pending ray does not hold
        const double dxs = xc - a.xray_x_prev[j];
        a.xray_x_prev[j] = xc;
        const double ds = cone_violation(dxs, lo_o, hi_o) > 0.0 ? 0.0 : dxs;  // cs > 0
        (a.st->xray_buf ? a.xray_d[0] : a.xray_d[1])[j] = ds;
        const double dx = ds * cs;
        t.xmax = smax(t.xmax, fabs(dx));
        t.xobj += P.obj_sign * P.c_o[j] * dx;
    }
}

// Block maxima of the 8 residual terms (and with INF the 2 of the
// infeasibility tests), one atomicMax per CTA and slot.
template <bool INF>
__device__ void block_max_terms(const Terms& t, unsigned long long* acc) {
    constexpr int K = INF ? 10 : 8;
    __shared__ double sh[K][kBlock / 32];
    double v[10] = {t.cp, t.cd, t.ap, t.ad, t.ocp, t.ocd, t.oap, t.oad, t.raymax, t.xmax};
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int q = 0; q < K; ++q) {
        double x = v[q];
        for (int o = 16; o > 0; o >>= 1) x = fmax(x, __shfl_xor_sync(0xffffffffu, x, o));
        if (lane == 0) sh[q][warp] = x;
    }
    __syncthreads();
    if (threadIdx.x < K) {
        double x = 0.0;
        for (int w = 0; w < kBlock / 32; ++w) x = fmax(x, sh[threadIdx.x][w]);
        // v[0..3] -> ACC_CUR_P..ACC_AVG_D, v[4..7] -> ACC_OC_P..ACC_OA_D,
        // v[8..9] -> ACC_RAY, ACC_XRAY_MAX
        const int slot = threadIdx.x < 4   ? ACC_CUR_P + static_cast<int>(threadIdx.x)
                         : threadIdx.x < 8 ? ACC_OC_P + static_cast<int>(threadIdx.x) - 4
                                           : ACC_RAY + static_cast<int>(threadIdx.x) - 8;
        if (x > 0.0)
            atomicMax(&acc[slot], static_cast<unsigned long long>(__double_as_longlong(x)));
    }
    __syncthreads();
}

// Products of entries [k, e) (stride `step`) of a row of A (ROWS: with the
// current x and the Cesaro average of x) or of A^T (with y and its average).
// ONE: only the average (T(z) of the Halpern iteration) is measured. A dense
// row (off set) computes its columns k + off.
template <class T, bool ROWS, bool ONE>
__device__ __forceinline__ void row_products(const FastCheck<T>& a, const DevCsr& M, int k, int e,
                                             int step, double inv, double& ac, double& aa,
                                             int off = kNotDense) {
    if constexpr (ONE) {  // rounds of four terms: their loads in flight together, same order
        for (; k + 3 * step < e; k += 4 * step) {
            int j[4];
            double v[4], g[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const int kk = k + u * step;
                j[u] = off != kNotDense ? kk + off : M.ci[kk];
                v[u] = M.v64[kk];
            }
#pragma unroll
            for (int u = 0; u < 4; ++u)
                g[u] = ROWS ? avg_x<T, true>(a.it, j[u], inv) : avg_y<T, true>(a.it, j[u], inv);
#pragma unroll
            for (int u = 0; u < 4; ++u) aa += v[u] * g[u];
        }
    }
    for (; k < e; k += step) {
        const int j = off != kNotDense ? k + off : M.ci[k];
        const double v = M.v64[k];
        if (ROWS) {
            if (!ONE) ac += v * cur_x(a.it, j);
            aa += v * avg_x<T, ONE>(a.it, j, inv);
        } else {
            if (!ONE) ac += v * cur_y(a.it, j);
            aa += v * avg_y<T, ONE>(a.it, j, inv);
        }
    }
}

template <class T, bool ROWS, int F>
__device__ __forceinline__ void row_or_col_terms(const FastCheck<T>& a, int r, double ac, double aa,
                                                 double inv, Terms& t) {
    if (ROWS) row_terms<T, F>(a, r, ac, aa, inv, t);
    else col_terms<T, F>(a, r, ac, aa, inv, t);
}

// Virtual block vb of one matrix's part [short | warp rows | CTA items]:
// short rows on groups of M.vw lanes, rows up to kLongRow one warp each
// (warp_rows0), longer ones as CTA items (items_long). Block-uniform.
template <class T, bool ROWS, int F>
__device__ void check_part(const FastCheck<T>& a, const DevCsr& M, int vb, int sb, int wb,
                           double inv, Terms& t) {
    constexpr bool ONE = (F & kCheckOne) != 0;
    double ac = 0.0, aa = 0.0;
    if (vb < sb) {
        const int vw = M.vw;
        const int lane = threadIdx.x & (vw - 1);
        const int r = (vb * kBlock + threadIdx.x) / vw;
        if (r >= M.rows) return;
        // the one-point instance also skips what the LP's structure makes
        // constant (row extents of equal-length rows, dense rows' columns);
        // in the others the extra registers would spill
        const bool st = ONE && M.rp_stride > 0;
        const int b = st ? r * M.rp_stride : M.rp[r];
        const int e = st ? b + M.rp_stride : M.rp[r + 1];
        if (e - b > M.short_max) return;
        row_products<T, ROWS, (F & kCheckOne) != 0>(a, M, b + lane, e, vw, inv, ac, aa);
        ac = group_sum(ac, vw);
        aa = group_sum(aa, vw);
        if (lane == 0) row_or_col_terms<T, ROWS, F>(a, r, ac, aa, inv, t);
    } else if (vb < sb + wb) {
        const int w = (vb - sb) * (kBlock / 32) + (threadIdx.x >> 5);
        if (w >= M.n_warp0) return;
        const int r = M.warp_rows0[w];
        const int lane = threadIdx.x & 31;
        row_products<T, ROWS, (F & kCheckOne) != 0>(a, M, M.rp[r] + lane, M.rp[r + 1], 32, inv, ac, aa,
                                                    ONE && M.dense_off ? M.dense_off[r] : kNotDense);
        for (int o = 16; o > 0; o >>= 1) {
            ac += __shfl_xor_sync(0xffffffffu, ac, o);
            aa += __shfl_xor_sync(0xffffffffu, aa, o);
        }
        if (lane == 0) row_or_col_terms<T, ROWS, F>(a, r, ac, aa, inv, t);
    } else {
        const int idx = vb - sb - wb;
        const int4 w = M.items_long.item[idx];
        row_products<T, ROWS, (F & kCheckOne) != 0>(a, M, w.y + threadIdx.x, w.z, kBlock, inv, ac, aa,
                                                    ONE && M.dense_off ? M.dense_off[w.x] : kNotDense);
        ac = block_total(ac);
        aa = block_total(aa);
        if (w.w >= 0 && !segment_finish(M.items_long, idx, w.w, ac, aa, &ac, &aa)) return;
        if (threadIdx.x == 0) row_or_col_terms<T, ROWS, F>(a, w.x, ac, aa, inv, t);
    }
}

// The check over row slices: a virtual block is up to 8 slice items, one per
// warp, lane l on the slice's row l, so the index, FP64 value and gather loads
// of a step are coalesced where the rows gather consecutive columns (the
// demand rows of a transportation LP). Each lane sums in k order; a slice cut
// into several items combines each lane's two sums in item order through the
// check's own ticket and partials.
template <class T, bool ROWS, int F>
__device__ void check_slices(const FastCheck<T>& a, const DevCsr& M, int vb, double inv, Terms& t) {
    constexpr bool ONE = (F & kCheckOne) != 0;
    const RowSlices& S = M.slices;
    const int idx = vb * (kBlock / 32) + (threadIdx.x >> 5);
    if (idx >= S.n_item) return;  // warp-uniform
    const int lane = threadIdx.x & 31;
    const int4 w = __ldg(S.item + idx);
    const int4 d = __ldg(S.slice + w.x);
    const int row = __ldg(S.row + 32 * w.x + lane);
    const int kend = min(w.z, __ldg(S.rlen + 32 * w.x + lane));
    const int32_t* __restrict__ col = S.col + d.y + lane;
    const double* __restrict__ val = S.v64 + d.y + lane;
    // the one-point instance computes an affine slice's columns (warp-uniform)
    const int2 af = ONE ? __ldg(S.affine + w.x) : make_int2(0, 0);
    auto colk = [&](int kk) -> int {
        return af.y > 0 ? af.x + lane + kk * af.y : __ldcs(col + 32 * static_cast<int64_t>(kk));
    };
    double ac = 0.0, aa = 0.0;
    int k = w.y;
    for (; k + 2 <= kend; k += 2) {
        int j[2];
        double v[2];
#pragma unroll
        for (int u = 0; u < 2; ++u) {
            j[u] = colk(k + u);
            v[u] = __ldcs(val + 32 * static_cast<int64_t>(k + u));
        }
#pragma unroll
        for (int u = 0; u < 2; ++u) {
            if (ROWS) {
                if (!ONE) ac += v[u] * cur_x(a.it, j[u]);
                aa += v[u] * avg_x<T, ONE>(a.it, j[u], inv);
            } else {
                if (!ONE) ac += v[u] * cur_y(a.it, j[u]);
                aa += v[u] * avg_y<T, ONE>(a.it, j[u], inv);
            }
        }
    }
    for (; k < kend; ++k) {
        const int j = colk(k);
        const double v = __ldcs(val + 32 * static_cast<int64_t>(k));
        if (ROWS) {
            if (!ONE) ac += v * cur_x(a.it, j);
            aa += v * avg_x<T, ONE>(a.it, j, inv);
        } else {
            if (!ONE) ac += v * cur_y(a.it, j);
            aa += v * avg_y<T, ONE>(a.it, j, inv);
        }
    }
    if (w.w >= 0) {  // warp-uniform
        S.cpart[64 * static_cast<int64_t>(idx) + lane] = ac;
        S.cpart[64 * static_cast<int64_t>(idx) + 32 + lane] = aa;
        __threadfence();
        __syncwarp();
        const int2 sp = __ldg(S.split + w.w);
        int last = 0;
        if (lane == 0) last = atomicAdd(S.cticket + w.w, 1u) == static_cast<unsigned>(sp.y - 1) ? 1 : 0;
        last = __shfl_sync(0xffffffffu, last, 0);
        if (!last) return;
        __threadfence();
        double sc = 0.0, sa = 0.0;
        for (int q = sp.x; q < sp.x + sp.y; ++q) {
            sc += __ldcg(S.cpart + 64 * static_cast<int64_t>(q) + lane);
            sa += __ldcg(S.cpart + 64 * static_cast<int64_t>(q) + 32 + lane);
        }
        if (lane == 0) S.cticket[w.w] = 0u;
        ac = sc;
        aa = sa;
    }
    if (row >= 0) row_or_col_terms<T, ROWS, F>(a, row, ac, aa, inv, t);
}

// Virtual blocks of the check over one matrix: short-row blocks (M.vw lanes
// per row), warp-row blocks, CTA items, slice blocks (8 slice items each).
__host__ __device__ inline int check_short_blocks(const DevCsr& M) {
    if (M.n_iter_short == 0) return 0;
    return static_cast<int>((static_cast<int64_t>(M.rows) * M.vw + kBlock - 1) / kBlock);
}
__host__ __device__ inline int check_warp_blocks(const DevCsr& M) { return (M.n_warp0 + kBlock / 32 - 1) / (kBlock / 32); }
__host__ __device__ inline int check_slice_blocks(const DevCsr& M) {
    return M.slices.n_item > 0 ? (M.slices.n_item + kBlock / 32 - 1) / (kBlock / 32) : 0;
}
inline int check_blocks(const DevCsr& M) {
    return check_short_blocks(M) + check_warp_blocks(M) + M.items_long.n_item + check_slice_blocks(M);
}

// The matrix the check walks: where the matrix has row slices (whether or
// not the iteration passes use them), the long-row tiers without the slices'
// rows, the slices covering those rows.
inline DevCsr check_view(const DevCsr& M) {
    if (M.slices.n_item == 0) return M;
    DevCsr X = M;
    const LongTiers& t = M.no_slice_tiers;
    X.warp_rows0 = t.warp_rows0;
    X.warp_rows1 = t.warp_rows1;
    X.n_warp0 = t.n_warp0;
    X.n_warp1 = t.n_warp1;
    X.items_long = t.items_long;
    X.items_huge = t.items_huge;
    X.items_warp = t.items_warp;
    return X;
}

// The one-point check over the rows of A^T (the columns of A) when every
// row has S = 2 or 4 entries: each thread walks rows j, j + T, j + 2T, ...
// (T threads in the grid) and issues the next row's index and value loads
// (vector loads) before it gathers the current row's y and forms its column
// terms, so the streamed arrays stay in flight while the gathers wait. The
// products are added in k order, as row_products does with one lane per row.
template <int S>
__device__ __forceinline__ void load_col_row(const DevCsr& M, int j, int (&c)[S], double (&v)[S]) {
    const int64_t b = static_cast<int64_t>(j) * S;
    if constexpr (S == 2) {
        const int2 q = __ldcs(reinterpret_cast<const int2*>(M.ci + b));
        const double2 w = __ldcs(reinterpret_cast<const double2*>(M.v64 + b));
        c[0] = q.x;
        c[1] = q.y;
        v[0] = w.x;
        v[1] = w.y;
    } else {
        const int4 q = __ldcs(reinterpret_cast<const int4*>(M.ci + b));
        const double2 w0 = __ldcs(reinterpret_cast<const double2*>(M.v64 + b));
        const double2 w1 = __ldcs(reinterpret_cast<const double2*>(M.v64 + b) + 1);
        c[0] = q.x;
        c[1] = q.y;
        c[2] = q.z;
        c[3] = q.w;
        v[0] = w0.x;
        v[1] = w0.y;
        v[2] = w1.x;
        v[3] = w1.y;
    }
}

template <class T, int F, int S>
__device__ void check_uniform_cols(const FastCheck<T>& a, double inv, Terms& t) {
    const DevCsr& M = a.AT;
    const int stride = gridDim.x * kBlock;
    int j = blockIdx.x * kBlock + threadIdx.x;
    if (j >= M.rows) return;
    int c[S];
    double v[S];
    load_col_row<S>(M, j, c, v);
    for (;;) {
        double g[S];
#pragma unroll
        for (int q = 0; q < S; ++q) g[q] = avg_y<T, true>(a.it, c[q], inv);
        const int jn = j + stride;
        const bool more = jn < M.rows;
        int nc[S] = {};
        double nv[S] = {};
        if (more) load_col_row<S>(M, jn, nc, nv);
        double aa = 0.0;
#pragma unroll
        for (int q = 0; q < S; ++q) aa += v[q] * g[q];
        col_terms<T, F>(a, j, 0.0, aa, inv, t);
        if (!more) break;
        j = jn;
#pragma unroll
        for (int q = 0; q < S; ++q) {
            c[q] = nc[q];
            v[q] = nv[q];
        }
    }
}

// A^T rows the one-point check walks with check_uniform_cols: 2 or 4
// entries each (0: the virtual blocks take them), the arrays aligned.
__host__ __device__ inline int check_uniform_stride(const DevCsr& M) {
    if (M.rp_stride != 2 && M.rp_stride != 4) return 0;
    if (((reinterpret_cast<uintptr_t>(M.ci) | reinterpret_cast<uintptr_t>(M.v64)) & 15u) != 0) return 0;
    return M.rp_stride;
}

// Grid-stride over the virtual blocks of A (act = A x, current and average)
// then of A^T (aty = A^T y); the grid itself is capped (a few CTAs per SM),
// so each CTA sums its rows into per-thread running terms and takes part in
// one reduction. FP64 fits three CTAs per SM (80 registers, no spills). FP32
// keeps four (64 registers): with the slice walk that spills about 140 bytes,
// yet on the 10M-column transportation LP it ran 416 us against 517 at three
// CTAs without spills (and 484 before the slice walk). Unbounded it took
// 109-118 registers and two CTAs per SM. The instance with the infeasibility
// tests (INF) carries 11 more running terms: two CTAs per SM.
template <class T, int F>
__global__ void __launch_bounds__(kBlock, (F & kCheckInf) ? 2 : (sizeof(T) == 4 || (F & kCheckOne)) ? 4 : 3)
    fast_check(FastCheck<T> a) {
    constexpr bool INF = (F & kCheckInf) != 0;
    constexpr bool L2 = (F & kCheckL2) != 0;
    constexpr bool ONE = (F & kCheckOne) != 0;
    DevState* st = a.st;
    if (st->done) return;
    const long long k_avg = st->since_restart + a.period_iters;
    // Halpern: the sums' slots hold T(z) itself
    const double inv = a.it.halpern ? 1.0 : 1.0 / static_cast<double>(k_avg);
    Terms t;
    // the one-point instance walks equal-length rows of A^T with the
    // pipelined loop after the virtual blocks (their short blocks dropped)
    const int uni = ONE ? check_uniform_stride(a.AT) : 0;
    const int sbA = check_short_blocks(a.A), wbA = check_warp_blocks(a.A);
    const int sbT = uni ? 0 : check_short_blocks(a.AT), wbT = check_warp_blocks(a.AT);
    const int pA = sbA + wbA + a.A.items_long.n_item, pT = sbT + wbT + a.AT.items_long.n_item;
    const int nA = pA + check_slice_blocks(a.A);
    const int nT = pT + check_slice_blocks(a.AT);
    for (int bid = blockIdx.x; bid < nA + nT; bid += gridDim.x) {
        if (bid < pA) check_part<T, true, F>(a, a.A, bid, sbA, wbA, inv, t);
        else if (bid < nA) check_slices<T, true, F>(a, a.A, bid - pA, inv, t);
        else if (bid < nA + pT) check_part<T, false, F>(a, a.AT, bid - nA, sbT, wbT, inv, t);
        else check_slices<T, false, F>(a, a.AT, bid - nA - pT, inv, t);
    }
    if (uni == 2) check_uniform_cols<T, F, 2>(a, inv, t);
    else if (uni == 4) check_uniform_cols<T, F, 4>(a, inv, t);
    if (ONE) {  // the current point's slots carry the measured point's terms
        t.cp = t.ap;
        t.cd = t.ad;
        t.ocp = t.oap;
        t.ocd = t.oad;
        t.pobj_c = t.pobj_a;
        t.dobj_c = t.dobj_a;
        t.ppc = t.ppa;
        t.ddc = t.dda;
    }
    block_max_terms<INF>(t, st->acc);
    // per-CTA partial sums, kCheckSums per CTA: the objectives [0..3]
    // (relative-KKT rules), the infeasibility test's ranges [4..7], the ray
    // test's c^T dx [8], rule 2's sums of squares [9..12]
    const bool sum_obj = a.termination_rule != 0, sum_ray = INF;
    auto summed = [&](int q) { return q < 4 ? sum_obj : q < 9 ? sum_ray : L2; };
    if (sum_obj || sum_ray || L2) {
        double v[kCheckSums] = {};
        if (sum_obj) {
            v[0] = block_sum_det(t.pobj_c);
            v[1] = block_sum_det(t.dobj_c);
            v[2] = block_sum_det(t.pobj_a);
            v[3] = block_sum_det(t.dobj_a);
        }
        if (sum_ray) {
            v[4] = block_sum_det(t.rlo);
            v[5] = block_sum_det(t.rhi);
            v[6] = block_sum_det(t.clo);
            v[7] = block_sum_det(t.chi);
            v[8] = block_sum_det(t.xobj);
        }
        if (L2) {
            v[9] = block_sum_det(t.ppc);
            v[10] = block_sum_det(t.ddc);
            v[11] = block_sum_det(t.ppa);
            v[12] = block_sum_det(t.dda);
        }
        if (threadIdx.x == 0)
            for (int q = 0; q < kCheckSums; ++q) a.cs.part[kCheckSums * blockIdx.x + q] = v[q];
    }
    if (!last_block(&st->ticket[TK_FAST])) return;
    // the per-CTA partial sums, added by the whole last CTA in a fixed order
    // (strided, then a tree)
    double obj[kCheckSums] = {};
    if (sum_obj || sum_ray || L2) {
        for (unsigned b = threadIdx.x; b < gridDim.x; b += kBlock)
            for (int q = 0; q < kCheckSums; ++q) obj[q] += __ldcg(a.cs.part + kCheckSums * b + q);
        for (int q = 0; q < kCheckSums; ++q)
            if (summed(q)) obj[q] = block_sum_det(obj[q]);
    }
    if (threadIdx.x != 0) return;

    // ---- decision (one thread) ----
    const double cp = acc_read(&st->acc[ACC_CUR_P]), cd = acc_read(&st->acc[ACC_CUR_D]);
    const double ap = acc_read(&st->acc[ACC_AVG_P]), ad = acc_read(&st->acc[ACC_AVG_D]);
    const double ocp = acc_read(&st->acc[ACC_OC_P]), ocd = acc_read(&st->acc[ACC_OC_D]);
    const double oap = acc_read(&st->acc[ACC_OA_P]), oad = acc_read(&st->acc[ACC_OA_D]);
    const double ray_max = acc_read(&st->acc[ACC_RAY]);
    const double xray_v = acc_read(&st->acc[ACC_XRAY_V]), xray_max = acc_read(&st->acc[ACC_XRAY_MAX]);
    for (int q = ACC_CUR_P; q <= ACC_OA_D; ++q) st->acc[q] = 0ull;
    st->acc[ACC_RAY] = st->acc[ACC_XRAY_V] = st->acc[ACC_XRAY_MAX] = 0ull;
    st->ticket[TK_FAST] = 0u;
    double cur = smax(cp, cd), avg = smax(ap, ad);
    // termination rule 2: the three relative parts of the current point and
    // of the average (original units, l2 norms), and their l2 norm, which is
    // restart rule 2's measure
    double part_c[3] = {0, 0, 0}, part_a[3] = {0, 0, 0};
    if (L2) {
        const double k0 = a.P.obj_sign * a.P.obj_const;  // the constant shifts both objectives
        const double sides[2][3] = {{obj[9], obj[10], obj[0]}, {obj[11], obj[12], obj[2]}};
        const double dsum[2] = {obj[1], obj[3]};
        for (int w = 0; w < 2; ++w) {
            double* part = w ? part_a : part_c;
            const double ps = sides[w][2] + k0, ds = dsum[w] + k0;
            part[0] = sqrt(sides[w][0]) / (1.0 + a.P.bnorm2);
            part[1] = sqrt(sides[w][1]) / (1.0 + a.P.cnorm2);
            part[2] = fabs(ps - ds) / (1.0 + fabs(ps) + fabs(ds));
        }
        if (a.restart_rule == 2) {
            const double mc = sqrt(part_c[0] * part_c[0] + part_c[1] * part_c[1] + part_c[2] * part_c[2]);
            const double ma = sqrt(part_a[0] * part_a[0] + part_a[1] * part_a[1] + part_a[2] * part_a[2]);
            // a non-finite scaled residual still stops the solve below
            cur = isfinite(cur) ? mc : cur;
            avg = isfinite(avg) ? ma : avg;
        }
    }
    if (a.it.halpern) cur = avg;  // only T(z) is measured
    st->cur_res = cur;
    st->avg_res = avg;
    st->inv = inv;
    const long long it_idx = st->iter + a.period_iters - 1;
    st->checks += 1;
    st->restart = 0;
    st->fold = 0;
    if (!isfinite(cur) || !isfinite(avg)) {  // pdhg.cpp:347-352
        st->done = 1;
        st->status = kStatusNumericalFailure;
        st->fail_kind = 1;
        st->stop_iter = it_idx;
    } else {
        // pdhg.cpp:354; Halpern: the candidate is T(z) (z itself may lie
        // outside the column bounds)
        const bool ab = a.it.halpern ? true : avg <= cur;
        st->avg_better = ab ? 1 : 0;
        const double op = ab ? oap : ocp, od = ab ? oad : ocd;
        const double orig = smax(op, od);
        st->orig_res = orig;
        if (!isfinite(orig)) {  // pdhg.cpp:366-371
            st->done = 1;
            st->status = kStatusNumericalFailure;
            st->fail_kind = 2;
            st->stop_iter = it_idx;
        } else {
            double rel = 0.0;
            if (L2) {
                const double* part = ab ? part_a : part_c;
                rel = smax(smax(part[0], part[1]), part[2]);
            } else if (a.termination_rule == 1) {
                double ps = ab ? obj[2] : obj[0], ds = ab ? obj[3] : obj[1];
                ps += a.P.obj_sign * a.P.obj_const;  // the constant shifts both objectives
                ds += a.P.obj_sign * a.P.obj_const;
                const double gap = fabs(ps - ds) / (1.0 + fabs(ps) + fabs(ds));
                rel = smax(smax(op / (1.0 + a.P.bnorm), od / (1.0 + a.P.cnorm)), gap);
            }
            st->rel_kkt = rel;
            const bool conv = (a.termination_rule != 0) ? (rel < a.tol) : (orig < a.tol);
            // Infeasibility test (engine extension): the change of y since the
            // previous check as a FarkasCertificate (duals.cpp:36-79), scaled
            // to max |dy| = 1; certified when the row-side and column-side
            // ranges are disjoint by more than 1e-6 x (1 + their finite ends).
            // Else the ray test: the change of x at the previous check,
            // projected onto the columns' recession cones and scaled to
            // max |d| = 1, certifies dual infeasibility when c^T d < 0
            // (minimize sense) and A d leaves the rows' recession cones by at
            // most 1e-6 and 1e-6 |c^T d| (fast_xray_rows measured it after
            // that check). This check's change becomes the next candidate.
            bool infeasible = false, unbounded = false;
            if (INF) {
                if (st->ray_base && !conv && ray_max > 0.0 && isfinite(ray_max)) {
                    const double k = 1.0 / ray_max;
                    const double r[4] = {obj[4] * k, obj[5] * k, obj[6] * k, obj[7] * k};
                    double ref = 1.0;
                    bool nan = false;
                    for (int q = 0; q < 4; ++q) {
                        if (isfinite(r[q])) ref += fabs(r[q]);
                        nan = nan || isnan(r[q]);
                    }
                    const double slack = 1e-6 * ref;
                    infeasible = !nan && (r[1] < r[2] - slack || r[3] < r[0] - slack);
                    st->ray_scale = k;  // the last test's figures, reported either way
                    for (int q = 0; q < 4; ++q) st->ray_ranges[q] = r[q];
                }
                if (st->xray_pending && !conv && !infeasible) {
                    const double ob = st->xray_obj, vi = xray_v * st->xray_scale;
                    unbounded = ob < 0.0 && vi <= 1e-6 && vi <= 1e-6 * -ob;
                    st->xray_viol = vi;
                }
                if (!unbounded) {  // this check's projected change: the next candidate
                    const bool ok = st->ray_base && xray_max > 0.0 && isfinite(xray_max);
                    st->xray_pending = ok ? 1 : 0;
                    if (ok) {
                        st->xray_buf ^= 1;
                        st->xray_scale = 1.0 / xray_max;
                        st->xray_obj = obj[8] * st->xray_scale;
                    }
                }
                st->ray_base = 1;  // this check's x, A x, y and A^T y are stored
            }
            if (infeasible || unbounded) {
                st->done = 1;
                st->status = infeasible ? PDHG_STATUS_PRIMAL_INFEASIBLE : PDHG_STATUS_DUAL_INFEASIBLE;
                st->stop_iter = it_idx + 1;
            } else if (conv) {  // pdhg.cpp:383-389
                st->done = 1;
                st->converged = 1;
                st->status = kStatusOptimal;
                st->stop_iter = it_idx + 1;
            } else if (a.restart_rule == 0) {
                if (!isfinite(st->res_last)) st->res_last = cur;  // pdhg.cpp:391
                if (avg <= a.restart_decrease * st->res_last) {   // pdhg.cpp:393-408
                    st->restart = 1;
                    st->restart_to_avg = 1;
                    st->res_last = avg;
                    st->since_restart = 0;
                    st->restarts += 1;
                } else {
                    st->since_restart += a.period_iters;
                }
            } else {
                // adaptive (restart rules 1 and 2): candidate = the better of
                // average and current
                const double cand = ab ? avg : cur;
                if (!isfinite(st->res_last)) st->res_last = cur;
                const long long span = st->since_restart + a.period_iters;
                const long long total = st->iter + a.period_iters;
                const bool sufficient = cand <= 0.2 * st->res_last;
                const bool necessary = cand <= 0.8 * st->res_last && cand > st->res_prev_cand;
                const bool artificial = static_cast<double>(span) >= 0.36 * static_cast<double>(total);
                st->res_prev_cand = cand;
                if (sufficient || necessary || artificial) {
                    st->restart = 1;
                    st->restart_to_avg = ab ? 1 : 0;
                    st->res_last = cand;
                    st->since_restart = 0;
                    st->restarts += 1;
                } else {
                    st->since_restart = span;
                }
                st->fresh = st->restart;
                st->fold = std::is_same<T, float>::value && !a.it.halpern ? 1 : 0;
                const int stop = a.mail != nullptr ? a.mail->stop_request : 0;
                if (stop != 0) {
                    st->done = 1;
                    st->status = stop;
                    st->stop_iter = it_idx + 1;
                }
            }
            // a restart moves x and y: the next check has no base to difference with
            if (INF && st->restart) st->ray_base = 0;
        }
    }
    st->iter += a.period_iters;
    Mailbox* mail = a.mail;
    if (mail != nullptr) {
        mail->iter = st->iter;
        mail->restarts = st->restarts;
        mail->checks = st->checks;
        mail->cur_res = st->cur_res;
        mail->avg_res = st->avg_res;
        mail->orig_res = st->orig_res;
        mail->rel_kkt = st->rel_kkt;
        mail->restarted = st->restart;
        mail->status = st->status;
        __threadfence_system();
        mail->done = st->done;
        __threadfence_system();
    }
}

// The candidate in original units, for the checkpoint callback
// (unscale_to_original, pdhg.cpp:205-214).
template <class T>
__global__ void fast_candidate(FastCheck<T> a) {
    const DevState* st = a.st;
    const int t = blockIdx.x * kBlock + threadIdx.x;
    const bool ab = st->avg_better != 0;
    const double inv = st->inv;
    if (t < a.P.n) {
        const double xs = ab ? avg_x(a.it, t, inv) : static_cast<double>(a.it.x[t]);
        a.cs.cand_xo[t] = xs * a.P.cs[t];
    }
    if (t < a.P.m) {
        const double ys = ab ? avg_y(a.it, t, inv) : static_cast<double>(a.it.y[t]);
        a.cs.cand_yo[t] = ys * a.P.obj_sign * a.P.rs[t];
    }
}

// Restart to the average (pdhg.cpp:393-404) and, in mixed mode, the fold of
// the period's FP32 sums into the FP64 Cesaro sums.
template <class T>
__global__ void __launch_bounds__(kBlock) fast_restart(FastCheck<T> a) {
    DevState* st = a.st;
    const int restart = st->restart;
    const int fold = st->fold;
    if (!restart && !fold) return;  // uniform: every CTA returns, no ticket is taken
    const bool to_avg = st->restart_to_avg != 0;
    const double inv = st->inv;
    const int t = blockIdx.x * kBlock + threadIdx.x;
    const PV<T> pv = pvec<T>(a.P);
    double dx2 = 0.0, dy2 = 0.0;
    if (t < a.P.n) {
        if (restart && to_avg)
            a.it.x[t] = clampT<T>(static_cast<T>(avg_x(a.it, t, inv)), pv.lo[t], pv.hi[t]);
        if (restart && a.it.halpern) a.it.xa[t] = a.it.x[t];  // the new anchor
        if (restart && a.primal_weight_update) {
            const double xn = static_cast<double>(a.it.x[t]);
            const double d = xn - a.x_last[t];
            dx2 = d * d;
            a.x_last[t] = xn;
        }
        if constexpr (std::is_same<T, float>::value) {
            a.it.xsum[t] = restart ? 0.0 : a.it.xsum[t] + static_cast<double>(a.it.psx[t]);
        }
    }
    if (t < a.P.m) {
        if (restart && to_avg) {
            a.it.y[t] = static_cast<T>(avg_y(a.it, t, inv));
            a.it.s[t] = clampT<T>(static_cast<T>(a.cs.act_avg[t]), pv.rlo[t], pv.rhi[t]);
        }
        if (restart && a.it.halpern) {
            a.it.ya[t] = a.it.y[t];
            a.it.sa[t] = a.it.s[t];
        }
        if (restart && a.primal_weight_update) {
            const double yn = static_cast<double>(a.it.y[t]);
            const double d = yn - a.y_last[t];
            dy2 = d * d;
            a.y_last[t] = yn;
        }
        if constexpr (std::is_same<T, float>::value) {
            a.it.ysum[t] = restart ? 0.0 : a.it.ysum[t] + static_cast<double>(a.it.psy[t]);
        }
    }
    if (!(restart && a.primal_weight_update)) return;  // uniform across the grid
    const double bx = block_sum_det(dx2);
    const double by = block_sum_det(dy2);
    if (threadIdx.x == 0) {
        a.cs.part[2 * blockIdx.x] = bx;
        a.cs.part[2 * blockIdx.x + 1] = by;
    }
    if (!last_block(&st->ticket[TK_RESTART])) return;
    double sx = 0.0, sy = 0.0;  // the whole last CTA, fixed order
    for (unsigned b = threadIdx.x; b < gridDim.x; b += kBlock) {
        sx += __ldcg(a.cs.part + 2 * b);
        sy += __ldcg(a.cs.part + 2 * b + 1);
    }
    sx = block_sum_det(sx);
    sy = block_sum_det(sy);
    if (threadIdx.x != 0) return;
    st->ticket[TK_RESTART] = 0u;
    const double dx = sqrt(sx), dy = sqrt(sy);
    if (dx > 1e-10 && dy > 1e-10) {
        // omega <- exp(0.5 log(dy/dx) + 0.5 log(omega))
        st->omega = sqrt(st->omega * (dy / dx));
        st->tau = st->eta / st->omega;
        st->sigma = st->eta * st->omega;
    }
}

}  // namespace

template <class K>
int resident_per_sm(K kernel) {
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kernel, kBlock, 0) != cudaSuccess) return 0;
    return n;
}

int init_fast_kernels(int device) {
    int sms = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess || sms <= 0)
        return 1;
    const int l32 = resident_per_sm(fast_iter_long<float, false, 0, false>);
    const int l64 = resident_per_sm(fast_iter_long<double, false, 0, false>);
    const int s32 = resident_per_sm(fast_iter_slices<float, false, false>);
    const int s64 = resident_per_sm(fast_iter_slices<double, false, false>);
    const int u[3][2] = {{resident_per_sm(fast_iter_uniform<float, 2, 1, true>),
                          resident_per_sm(fast_iter_uniform<double, 2, 1, true>)},
                         {resident_per_sm(fast_iter_uniform<float, 4, 1, true>),
                          resident_per_sm(fast_iter_uniform<double, 4, 1, true>)},
                         {resident_per_sm(fast_iter_uniform<float, 4, 2, true>),
                          resident_per_sm(fast_iter_uniform<double, 4, 2, true>)}};
    for (int q = 0; q < 3; ++q)
        for (int t = 0; t < 2; ++t) {
            if (u[q][t] <= 0) return 1;
            g_cap_uni[q][t] = u[q][t] * sms;
        }
    if (l32 <= 0 || l64 <= 0 || s32 <= 0 || s64 <= 0) return 1;
    g_cap_long[0] = l32 * sms;
    g_cap_long[1] = l64 * sms;
    g_cap_slice[0] = s32 * sms;
    g_cap_slice[1] = s64 * sms;
    const int k32 = resident_per_sm(fast_check<float, kCheckL2 | kCheckOne>);
    const int k64 = resident_per_sm(fast_check<double, kCheckL2 | kCheckOne>);
    if (k32 <= 0 || k64 <= 0) return 1;
    g_cap_check1[0] = k32 * sms;
    g_cap_check1[1] = k64 * sms;
    const int w32 = resident_per_sm(fast_iter_slices<float, false, true>);
    const int w64 = resident_per_sm(fast_iter_slices<double, false, true>);
    if (w32 <= 0 || w64 <= 0) return 1;
    g_cap_slice_w[0] = w32 * sms;
    g_cap_slice_w[1] = w64 * sms;
    return 0;
}

template <class T>
int launch_fast_primal(const FastIter<T>& a, int first, cudaStream_t s, const PassFork* f) {
    return launch_iter<T, true>(a, first, s, f);
}
template <class T>
int launch_fast_dual(const FastIter<T>& a, int first, cudaStream_t s, const PassFork* f) {
    return launch_iter<T, false>(a, first, s, f);
}
template <class T>
int fast_launches_per_iteration(const FastIter<T>& a) {
    return pass_launches(a.AT) + pass_launches(a.A);
}

// Ray test, rows' half: after a check that left a pending ray d (projected
// onto the columns' recession cones, scaled units), the largest amount by
// which A_o d_o = (A_s d_s) / rs leaves a row's recession cone, one warp per
// row (original-space values, FP64), into ACC_XRAY_V for the next check.
// It runs even when that check ended the solve: a solve that goes on (the
// mixed mode's FP64 phase) tests the ray at its first check. Measuring the
// same ray again leaves the maximum as it was.
template <class T>
__global__ void __launch_bounds__(kBlock) fast_xray_rows(FastCheck<T> a) {
    const DevState* st = a.st;
    if (!st->xray_pending) return;
    const double* d = st->xray_buf ? a.xray_d[1] : a.xray_d[0];
    const DevCsr& M = a.A;
    const int lane = threadIdx.x & 31;
    double v = 0.0;
    for (int r = (blockIdx.x * kBlock + threadIdx.x) >> 5; r < M.rows; r += (gridDim.x * kBlock) >> 5) {
        double s = 0.0;
        for (int k = M.rp[r] + lane; k < M.rp[r + 1]; k += 32) s += M.v64[k] * d[M.ci[k]];
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        v = smax(v, cone_violation(s / a.P.rs[r], a.P.rlo_o[r], a.P.rhi_o[r]));
    }
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    if (lane == 0 && v > 0.0)
        atomicMax(&a.st->acc[ACC_XRAY_V], static_cast<unsigned long long>(__double_as_longlong(v)));
}

template <class T>
void launch_fast_check(const FastCheck<T>& a0, cudaStream_t s) {
    FastCheck<T> a = a0;
    a.A = check_view(a0.A);
    a.AT = check_view(a0.AT);
    int grid = check_blocks(a.A) + check_blocks(a.AT);
    if (a.grid_cap > 0 && grid > a.grid_cap) grid = a.grid_cap;
    const bool l2 = a.termination_rule == 2;
    // the one-point instance's pipelined column walk: at most one wave of
    // resident CTAs (only ever fewer CTAs than the grid the per-CTA partial
    // sums are allocated for, fast_check_grid)
    const int pi = sizeof(T) == 4 ? 0 : 1;
    if (l2 && a.it.halpern && !a.infeas && check_uniform_stride(a.AT) && grid > g_cap_check1[pi])
        grid = g_cap_check1[pi];
    if (grid == 0) grid = 1;
    if (a.infeas) {
        if (l2) fast_check<T, kCheckInf | kCheckL2><<<grid, kBlock, 0, s>>>(a);
        else fast_check<T, kCheckInf><<<grid, kBlock, 0, s>>>(a);
        const int rows_grid = (a.A.rows + kBlock / 32 - 1) / (kBlock / 32);
        const int xg = rows_grid < a.grid_cap || a.grid_cap <= 0 ? rows_grid : a.grid_cap;
        fast_xray_rows<T><<<xg > 0 ? xg : 1, kBlock, 0, s>>>(a);
    } else if (l2 && a.it.halpern) {  // only T(z) is measured
        fast_check<T, kCheckL2 | kCheckOne><<<grid, kBlock, 0, s>>>(a);
    } else if (l2) {
        fast_check<T, kCheckL2><<<grid, kBlock, 0, s>>>(a);
    } else {
        fast_check<T, 0><<<grid, kBlock, 0, s>>>(a);
    }
    if (a.want_candidate) {
        const int32_t nmax = a.P.n > a.P.m ? a.P.n : a.P.m;
        if (nmax > 0) fast_candidate<T><<<(nmax + kBlock - 1) / kBlock, kBlock, 0, s>>>(a);
    }
}
template <class T>
void launch_fast_restart(const FastCheck<T>& a, cudaStream_t s) {
    const int32_t nmax = a.P.n > a.P.m ? a.P.n : a.P.m;
    fast_restart<T><<<nmax > 0 ? (nmax + kBlock - 1) / kBlock : 1, kBlock, 0, s>>>(a);
}

// Upper bound on check-kernel CTAs (partial-sum buffer sizing).
int fast_check_grid(const DevCsr& A, const DevCsr& AT) {
    return check_blocks(check_view(A)) + check_blocks(check_view(AT)) + 1;
}

template int launch_fast_primal<float>(const FastIter<float>&, int, cudaStream_t, const PassFork*);
template int launch_fast_primal<double>(const FastIter<double>&, int, cudaStream_t, const PassFork*);
template int launch_fast_dual<float>(const FastIter<float>&, int, cudaStream_t, const PassFork*);
template int launch_fast_dual<double>(const FastIter<double>&, int, cudaStream_t, const PassFork*);
template int fast_launches_per_iteration<float>(const FastIter<float>&);
template int fast_launches_per_iteration<double>(const FastIter<double>&);
template void launch_fast_check<float>(const FastCheck<float>&, cudaStream_t);
template void launch_fast_check<double>(const FastCheck<double>&, cudaStream_t);
template void launch_fast_restart<float>(const FastCheck<float>&, cudaStream_t);
template void launch_fast_restart<double>(const FastCheck<double>&, cudaStream_t);

}  // namespace pdhg
