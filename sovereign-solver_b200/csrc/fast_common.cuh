// fast_common.cuh -- device helpers shared by the single-LP throughput kernels
// (kernels_fast.cu) and the batched kernels (batch.cu): precision-generic
// vector access, group/block reductions, the long-row dot product, the fused
// iteration epilogue and the residual terms of the check.
#pragma once

#include <type_traits>

#include "engine.cuh"

namespace pdhg {
namespace {

constexpr int kStatusOptimal = 0;
constexpr int kStatusNumericalFailure = 3;

__device__ __forceinline__ double smax(double a, double b) { return (a < b) ? b : a; }
__device__ __forceinline__ bool fb(double v) { return v > -INFINITY && v < INFINITY; }

template <class T>
__device__ __forceinline__ T clampT(T v, T lo, T hi) {
    if (v < lo) v = lo;
    if (v > hi) v = hi;
    return v;
}

template <class T>
__device__ __forceinline__ const T* mvals(const DevCsr& A);
template <>
__device__ __forceinline__ const float* mvals<float>(const DevCsr& A) { return A.v32; }
template <>
__device__ __forceinline__ const double* mvals<double>(const DevCsr& A) { return A.v64; }

template <class T>
struct PV {
    const T *c, *lo, *hi, *rlo, *rhi;
    int ub;       // every column has the bounds lo_u <= x <= hi_u
    T lo_u, hi_u;
};
template <class T>
__device__ __forceinline__ PV<T> pvec(const DevProblem& P);
template <>
__device__ __forceinline__ PV<float> pvec<float>(const DevProblem& P) {
    return {P.c32, P.lo32, P.hi32, P.rlo32, P.rhi32, P.col_bounds_uniform,
            static_cast<float>(P.lo_u), static_cast<float>(P.hi_u)};
}
template <>
__device__ __forceinline__ PV<double> pvec<double>(const DevProblem& P) {
    return {P.c, P.lo, P.hi, P.rlo, P.rhi, P.col_bounds_uniform, P.lo_u, P.hi_u};
}

__device__ __forceinline__ unsigned group_mask(int vw) {
    if (vw >= 32) return 0xffffffffu;
    const unsigned base = (threadIdx.x & 31u) & ~static_cast<unsigned>(vw - 1);
    return ((1u << vw) - 1u) << base;
}

template <class T>
__device__ __forceinline__ T group_sum(T v, int vw) {
    const unsigned mask = group_mask(vw);
    for (int o = vw / 2; o > 0; o >>= 1) v += __shfl_xor_sync(mask, v, o);
    return v;
}

// Block-wide sum; every thread calls it and gets the total.
template <class T>
__device__ T block_total(T v) {
    __shared__ T sh[kBlock / 32];
    __shared__ T tot;
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x < 32) {
        T w = threadIdx.x < kBlock / 32 ? sh[threadIdx.x] : T(0);
        for (int o = 16; o > 0; o >>= 1) w += __shfl_xor_sync(0xffffffffu, w, o);
        if (threadIdx.x == 0) tot = w;
    }
    __syncthreads();
    const T r = tot;
    __syncthreads();
    return r;
}

// Deterministic block sum for the check's partial sums.
__device__ double block_sum_det(double v) {
    __shared__ double sh[kBlock];
    sh[threadIdx.x] = v;
    __syncthreads();
    for (int s = kBlock / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) sh[threadIdx.x] += sh[threadIdx.x + s];
        __syncthreads();
    }
    const double r = sh[0];
    __syncthreads();
    return r;
}

__device__ __forceinline__ double acc_read(unsigned long long* slot) {
    return __longlong_as_double(
        static_cast<long long>(*reinterpret_cast<volatile unsigned long long*>(slot)));
}

__device__ __forceinline__ bool last_block(unsigned int* ticket) {
    __shared__ bool am_last;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) am_last = (atomicAdd(ticket, 1u) == gridDim.x - 1);
    __syncthreads();
    return am_last;
}

// Persistent kernels claim work items from a counter pair {next, exits}:
// cta_fetch (every thread of the CTA calls it) returns the next item index to
// all threads, warp_fetch the same for one warp. Each CTA (warp) that ran the
// loop reports its exit once; the last of the grid resets both counters for
// the next launch (launches on a stream are ordered, so nobody claims in
// between). Nothing ever waits on another CTA.
__device__ __forceinline__ int cta_fetch(unsigned int* fetch) {
    __shared__ int next;
    if (threadIdx.x == 0) next = static_cast<int>(atomicAdd(fetch, 1u));
    __syncthreads();
    const int v = next;
    __syncthreads();
    return v;
}

__device__ __forceinline__ void cta_exit(unsigned int* fetch) {
    if (threadIdx.x != 0) return;
    __threadfence();
    if (atomicAdd(fetch + 1, 1u) == gridDim.x - 1) {
        fetch[0] = 0u;
        fetch[1] = 0u;
    }
}

__device__ __forceinline__ int warp_fetch(unsigned int* fetch) {
    int v = 0;
    if ((threadIdx.x & 31) == 0) v = static_cast<int>(atomicAdd(fetch, 1u));
    return __shfl_sync(0xffffffffu, v, 0);
}

__device__ __forceinline__ void warp_exit(unsigned int* fetch) {
    if ((threadIdx.x & 31) != 0) return;
    __threadfence();
    if (atomicAdd(fetch + 1, 1u) == gridDim.x * (blockDim.x / 32) - 1) {
        fetch[0] = 0u;
        fetch[1] = 0u;
    }
}

// One segment of a split row done; every thread of the CTA calls it (block-
// uniform) with the CTA's two partials. Thread 0 stores them and takes the
// row's ticket. The CTA that draws the last ticket returns true on every
// thread with the row's totals: warp 0 reads the segments' partials (lane l
// takes segments l, l+32, ...) and adds them in a fixed shuffle order, so the
// result does not depend on which CTA finished when; it also resets the
// ticket for the next launch. The other CTAs return false.
__device__ __forceinline__ bool segment_finish(const RowItems& L, int idx, int split, double v0,
                                               double v1, double* t0, double* t1) {
    __shared__ int last;
    __shared__ double tot[2];
    if (threadIdx.x == 0) {
        L.part[2 * idx] = v0;
        L.part[2 * idx + 1] = v1;
        __threadfence();
        const int2 sp = __ldg(L.split + split);
        last = atomicAdd(L.ticket + split, 1u) == static_cast<unsigned>(sp.y - 1) ? 1 : 0;
    }
    __syncthreads();
    if (!last) return false;
    if (threadIdx.x < 32) {
        __threadfence();
        const int2 sp = __ldg(L.split + split);
        double a = 0.0, b = 0.0;
        for (int k = sp.x + static_cast<int>(threadIdx.x); k < sp.x + sp.y; k += 32) {
            a += __ldcg(L.part + 2 * k);
            b += __ldcg(L.part + 2 * k + 1);
        }
        for (int o = 16; o > 0; o >>= 1) {
            a += __shfl_xor_sync(0xffffffffu, a, o);
            b += __shfl_xor_sync(0xffffffffu, b, o);
        }
        if (threadIdx.x == 0) {
            tot[0] = a;
            tot[1] = b;
            L.ticket[split] = 0u;
        }
    }
    __syncthreads();
    *t0 = tot[0];
    *t1 = tot[1];
    return true;
}

// The same for a segment summed by one warp (every lane calls it, warp-
// uniform; no block barrier): lane 0 stores the warp's partial and takes the
// row's ticket; the warp drawing the last ticket returns true on every lane
// with the row's total (lane l adds segments l, l+32, ..., then a fixed
// shuffle tree) and resets the ticket.
__device__ __forceinline__ bool warp_segment_finish(const RowItems& L, int idx, int split,
                                                    double v, double* t) {
    const int lane = threadIdx.x & 31;
    const int2 sp = __ldg(L.split + split);
    int last = 0;
    if (lane == 0) {
        L.part[2 * idx] = v;
        __threadfence();
        last = atomicAdd(L.ticket + split, 1u) == static_cast<unsigned>(sp.y - 1) ? 1 : 0;
    }
    last = __shfl_sync(0xffffffffu, last, 0);
    if (!last) return false;
    __threadfence();
    double a = 0.0;
    for (int k = sp.x + lane; k < sp.x + sp.y; k += 32) a += __ldcg(L.part + 2 * k);
    for (int o = 16; o > 0; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
    if (lane == 0) L.ticket[split] = 0u;
    *t = a;
    return true;
}

// Vector types of the 128-bit loads (W = 16 / sizeof(T) entries).
template <class T>
struct Vec16;
template <>
struct Vec16<float> {
    using type = float4;
};
template <>
struct Vec16<double> {
    using type = double2;
};

// Gathered entries of one 128-bit vector of a row. DENSE: entry k of the row
// sits in column k + off, so the W entries are consecutive: one vector load
// when `va` (the gathered vector aligned with the row's values), else W
// scalar loads at computed addresses. Otherwise the columns come from `c`.
template <class T>
__device__ __forceinline__ typename Vec16<T>::type gather16(const T* __restrict__ xg, int k, int off,
                                                            bool va) {
    if (va) return __ldg(reinterpret_cast<const typename Vec16<T>::type*>(xg + k + off));
    typename Vec16<T>::type g;
    if constexpr (std::is_same<T, float>::value) {
        g.x = __ldg(xg + k + off);
        g.y = __ldg(xg + k + off + 1);
        g.z = __ldg(xg + k + off + 2);
        g.w = __ldg(xg + k + off + 3);
    } else {
        g.x = __ldg(xg + k + off);
        g.y = __ldg(xg + k + off + 1);
    }
    return g;
}

// Long-row dot product, one CTA: 128-bit loads of values and column indices
// on the aligned body (four of each in flight per thread), scalar head and
// tail. The matrix is streamed (evict-first, ld.global.cs) so that the
// gathered vector keeps its L2 lines; gathers go through the read-only path.
// DENSE: the columns are k + off (no index loads); the sum order is the same
// either way.
template <class T, bool DENSE = false>
__device__ __forceinline__ T long_row_dot(const int32_t* __restrict__ ci,
                                          const T* __restrict__ v, const T* __restrict__ xg,
                                          int b, int e, int off = 0) {
    constexpr int W = 16 / sizeof(T);
    constexpr int U = 2;  // vectors of each stream in flight per thread
    using V = typename Vec16<T>::type;
    using I = typename std::conditional<W == 4, int4, int2>::type;
    int bA = ((b + W - 1) / W) * W;
    if (bA > e) bA = e;
    const bool va = DENSE && ((bA + off) & (W - 1)) == 0;
    auto col = [&](int k) { return DENSE ? k + off : __ldcs(ci + k); };
    T acc = T(0);
    for (int k = b + threadIdx.x; k < bA; k += kBlock) acc += __ldcs(v + k) * __ldg(xg + col(k));
    const int nvec = (e - bA) / W;
    const V* vv = reinterpret_cast<const V*>(v + bA);
    const I* cc = reinterpret_cast<const I*>(ci + bA);
    // rounds of up to U vectors per thread, the last round predicated, so a
    // segment of a few thousand entries takes one or two rounds with all of a
    // round's loads in flight together (a one-vector remainder loop
    // serialised them); U = 2 keeps the 40-register kernels free of spills
    for (int q = threadIdx.x; q < nvec; q += U * kBlock) {
        V w[U], g[U];
        I c[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const bool ok = q + u * kBlock < nvec;
            const int qq = ok ? q + u * kBlock : 0;
            w[u] = ok ? __ldcs(vv + qq) : V{};
            if (DENSE) g[u] = ok ? gather16<T>(xg, bA + W * qq, off, va) : V{};
            else c[u] = ok ? __ldcs(cc + qq) : I{};
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
            if (q + u * kBlock >= nvec) continue;
            if constexpr (W == 4) {
                if (DENSE) {
                    acc += w[u].x * g[u].x + w[u].y * g[u].y + w[u].z * g[u].z + w[u].w * g[u].w;
                } else {
                    acc += w[u].x * __ldg(xg + c[u].x) + w[u].y * __ldg(xg + c[u].y) +
                           w[u].z * __ldg(xg + c[u].z) + w[u].w * __ldg(xg + c[u].w);
                }
            } else {
                if (DENSE) acc += w[u].x * g[u].x + w[u].y * g[u].y;
                else acc += w[u].x * __ldg(xg + c[u].x) + w[u].y * __ldg(xg + c[u].y);
            }
        }
    }
    for (int k = bA + nvec * W + threadIdx.x; k < e; k += kBlock)
        acc += __ldcs(v + k) * __ldg(xg + col(k));
    return block_total(acc);
}

// 128-bit vectors of each stream a lane keeps in flight in warp_row_dot (a
// build knob: registers against memory-level parallelism).
#ifndef PDHG_WARP_UNROLL
#define PDHG_WARP_UNROLL 4
#endif
constexpr int kWarpUnroll = PDHG_WARP_UNROLL;

// Load used for the x / y gathers of warp_row_dot (a build knob).
#ifndef PDHG_GATHER
#define PDHG_GATHER __ldg
#endif

// The same dot by one warp (rows of kLongRow..kHugeRow entries): 128-bit loads
// of values and indices, kWarpUnroll of each in flight per lane, then a
// shuffle reduction -- no block barrier, so a CTA's eight warps finish
// independently. Every lane returns the total.
template <class T>
__device__ __forceinline__ T warp_row_dot(const int32_t* __restrict__ ci,
                                          const T* __restrict__ v, const T* __restrict__ xg,
                                          int b, int e, int off = kNotDense) {
    constexpr int W = 16 / sizeof(T);
    using V = typename Vec16<T>::type;
    const int lane = threadIdx.x & 31;
    // a dense row (off set, warp-uniform) computes its columns k + off in the
    // same loop: one register set for both kinds of row
    const bool dense = off != kNotDense;
    int bA = ((b + W - 1) / W) * W;
    if (bA > e) bA = e;
    auto col = [&](int k) { return dense ? k + off : __ldcs(ci + k); };
    T acc = T(0);
    for (int k = b + lane; k < bA; k += 32) acc += __ldcs(v + k) * PDHG_GATHER(xg + col(k));
    const int nvec = (e - bA) / W;
    const V* vv = reinterpret_cast<const V*>(v + bA);
    // rounds of up to kWarpUnroll vectors per lane in flight; the last round
    // is predicated instead of falling back to one vector at a time
    if constexpr (W == 4) {
        const int4* ci4 = reinterpret_cast<const int4*>(ci + bA);
        for (int q = lane; q < nvec; q += 32 * kWarpUnroll) {
            int4 c[kWarpUnroll];
            float4 w[kWarpUnroll];
#pragma unroll
            for (int u = 0; u < kWarpUnroll; ++u) {
                const bool ok = q + 32 * u < nvec;
                const int k = bA + 4 * (q + 32 * u) + off;
                c[u] = !ok ? make_int4(0, 0, 0, 0) : dense ? make_int4(k, k + 1, k + 2, k + 3) : __ldcs(ci4 + q + 32 * u);
                w[u] = ok ? __ldcs(vv + q + 32 * u) : make_float4(0.f, 0.f, 0.f, 0.f);
            }
#pragma unroll
            for (int u = 0; u < kWarpUnroll; ++u)
                if (q + 32 * u < nvec)
                    acc += w[u].x * PDHG_GATHER(xg + c[u].x) + w[u].y * PDHG_GATHER(xg + c[u].y) +
                           w[u].z * PDHG_GATHER(xg + c[u].z) + w[u].w * PDHG_GATHER(xg + c[u].w);
        }
    } else {
        const int2* ci2 = reinterpret_cast<const int2*>(ci + bA);
        for (int q = lane; q < nvec; q += 32 * kWarpUnroll) {
            int2 c[kWarpUnroll];
            double2 w[kWarpUnroll];
#pragma unroll
            for (int u = 0; u < kWarpUnroll; ++u) {
                const bool ok = q + 32 * u < nvec;
                const int k = bA + 2 * (q + 32 * u) + off;
                c[u] = !ok ? make_int2(0, 0) : dense ? make_int2(k, k + 1) : __ldcs(ci2 + q + 32 * u);
                w[u] = ok ? __ldcs(vv + q + 32 * u) : make_double2(0.0, 0.0);
            }
#pragma unroll
            for (int u = 0; u < kWarpUnroll; ++u)
                if (q + 32 * u < nvec)
                    acc += w[u].x * PDHG_GATHER(xg + c[u].x) + w[u].y * PDHG_GATHER(xg + c[u].y);
        }
    }
    for (int k = bA + nvec * W + lane; k < e; k += 32)
        acc += __ldcs(v + k) * PDHG_GATHER(xg + col(k));
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    return acc;
}


// Epilogue traffic: every per-column array is streamed (evict-first loads and
// stores) except x_bar, whose lines the dual kernel gathers next and should
// find in L2; y likewise stays at normal priority for the next primal gather.
// The epilogue's operands are loaded before the row's SpMV loads are issued
// (they do not depend on them), so both streams are in flight together.
template <class T>
struct EpiIn {
    T a, b, lo, hi, ps;  // primal: c, x, lo, hi, sum; dual: y, s, row lo, row hi, sum
};

// The reflected Halpern weights of an iteration: w = (k+1)/(k+2), k the
// iterations since the last restart, and the previous iteration's w' =
// k/(k+1) (0 right after a restart, when z is the anchor). Both zero without
// the option.
template <class T>
struct Hw {
    T w, wp;
};

template <class T>
__device__ __forceinline__ Hw<T> halpern_weight(const Iterates<T>& it, long long since_restart,
                                                int hk) {
    if (!it.halpern) return {T(0), T(0)};
    const double k = static_cast<double>(since_restart + hk);
    return {static_cast<T>((k + 1.0) / (k + 2.0)), static_cast<T>(k / (k + 1.0))};
}

// The same weights where one k holds for the whole launch and every lane of
// the warp is converged (the single-LP kernels): lane 0 forms them and the
// warp shares them by shuffle, so the FP64 divisions run once per warp.
template <class T>
__device__ __forceinline__ Hw<T> halpern_weight_warp(const Iterates<T>& it, const DevState* st,
                                                     int hk) {
    if (!it.halpern) return {T(0), T(0)};
    Hw<T> h{T(0), T(0)};
    if ((threadIdx.x & 31) == 0) h = halpern_weight<T>(it, st->since_restart, hk);
    h.w = __shfl_sync(0xffffffffu, h.w, 0);
    h.wp = __shfl_sync(0xffffffffu, h.wp, 0);
    return h;
}

// z+ = w (2 T(z) - z) + (1 - w) z_a: the same rounding wherever it is formed
// (the primal's store, and its rebuild of x in lean mode)
template <class T>
__device__ __forceinline__ T halpern_mix(T w, T refl, T anchor) {
    if constexpr (std::is_same<T, float>::value) return __fmaf_rn(w, refl, (1.0f - w) * anchor);
    else return __fma_rn(w, refl, (1.0 - w) * anchor);
}

// LEAN = false compiles the lean Halpern form out (callers that never set it)
template <class T, bool PRIMAL, bool LEAN = true>
__device__ __forceinline__ EpiIn<T> epi_load(const Iterates<T>& it, const PV<T>& pv, int r,
                                             int first, bool fresh, const Hw<T>& hw) {
    EpiIn<T> in;
    // Halpern: the sums' slot is only written, so `ps` carries the anchor of x
    // (primal) or y (dual) instead; the slack's anchor is read at the store
    if (PRIMAL) {
        in.a = __ldcs(pv.c + r);
        if (LEAN && it.lean) {  // x = w' x_bar + (1 - w') x_a, x_a right after a restart
            in.ps = __ldcs(it.xa + r);
            in.b = hw.wp == T(0) ? in.ps : halpern_mix<T>(hw.wp, it.xbar[r], in.ps);
            in.lo = pv.ub ? pv.lo_u : __ldcs(pv.lo + r);
            in.hi = pv.ub ? pv.hi_u : __ldcs(pv.hi + r);
            return in;
        }
        in.b = __ldcs(it.x + r);
        in.lo = pv.ub ? pv.lo_u : __ldcs(pv.lo + r);
        in.hi = pv.ub ? pv.hi_u : __ldcs(pv.hi + r);
        if (it.halpern) in.ps = __ldcs(it.xa + r);
        else if constexpr (std::is_same<T, float>::value) in.ps = first ? T(0) : __ldcs(it.psx + r);
        else in.ps = fresh ? T(0) : __ldcs(it.xsum + r);
    } else {
        in.a = it.y[r];
        in.b = __ldcs(it.s + r);
        in.lo = __ldcs(pv.rlo + r);
        in.hi = __ldcs(pv.rhi + r);
        if (it.halpern) in.ps = __ldcs(it.ya + r);
        else if constexpr (std::is_same<T, float>::value) in.ps = first ? T(0) : __ldcs(it.psy + r);
        else in.ps = fresh ? T(0) : __ldcs(it.ysum + r);
    }
    return in;
}

// primal: x+ = proj(x - tau (c - aty)), x_bar = 2x+ - x, sum += x+
// dual:   s+ = proj(s - tau y), y+ = y + sigma (2s+ - s - ax), sum += y+
// With the Halpern option (weight hw = w) the step's output T(z) = (x+, s+, y+)
// goes to the sums' slot and z moves to w (2 T(z) - z) + (1 - w) z_a (the
// anchor of x or y arrives in in.ps).
template <class T, bool PRIMAL, bool LEAN = true>
__device__ __forceinline__ void epi_store(const Iterates<T>& it, int r, T dot, const EpiIn<T>& in,
                                          T tau, T sigma, const Hw<T>& hw, int tz) {
    // tz (lean Halpern): this iteration stores T(z) and z's x part; read from
    // the launch's parameters at the store so that it holds no register across
    // the SpMV
    const bool lean = LEAN && it.lean;
    const bool store_tz = !lean || tz != 0;
    T* ps = nullptr;
    if constexpr (std::is_same<T, float>::value) ps = PRIMAL ? it.psx : it.psy;
    else ps = PRIMAL ? it.xsum : it.ysum;
    if (PRIMAL) {
        const T xo = in.b;
        const T xn = clampT<T>(xo - tau * (in.a - dot), in.lo, in.hi);
        const T xb = T(2) * xn - xo;
        it.xbar[r] = xb;
        if (it.halpern) {
            if (store_tz) __stcs(it.x + r, halpern_mix<T>(hw.w, xb, in.ps));
            if (store_tz) __stcs(ps + r, xn);
        } else {
            __stcs(it.x + r, xn);
            __stcs(ps + r, in.ps + xn);
        }
    } else {
        const T yo = in.a, so = in.b;
        const T sn = clampT<T>(so - tau * yo, in.lo, in.hi);
        const T sb = T(2) * sn - so;
        const T yn = yo + sigma * (sb - dot);
        if (it.halpern) {
            it.y[r] = halpern_mix<T>(hw.w, T(2) * yn - yo, in.ps);
            __stcs(it.s + r, halpern_mix<T>(hw.w, sb, __ldcs(it.sa + r)));
            if (store_tz) __stcs(ps + r, yn);
        } else {
            it.y[r] = yn;
            __stcs(it.s + r, sn);
            __stcs(ps + r, in.ps + yn);
        }
    }
}

__device__ __forceinline__ double cs_term(double v, double act, double lo, double hi,
                                          double bt) {
    const bool at_lo = fb(lo) && fabs(act - lo) < bt;
    const bool at_hi = fb(hi) && fabs(act - hi) < bt;
    if (!at_lo && !at_hi) return fabs(v);
    if (at_lo && !at_hi) return smax(0.0, -v);
    if (at_hi && !at_lo) return smax(0.0, v);
    return 0.0;
}

__device__ __forceinline__ double primal_term(double act, double lo, double hi) {
    double p = 0.0;
    if (fb(lo)) p = smax(p, lo - act);
    if (fb(hi)) p = smax(p, act - hi);
    return p;
}

__device__ __forceinline__ double clipped_inf(double coeff, double lo, double hi) {
    if (coeff > 0.0) return fb(lo) ? coeff * lo : 0.0;
    if (coeff < 0.0) return fb(hi) ? coeff * hi : 0.0;
    return 0.0;
}

// Instances of the check kernel: with the infeasibility tests, with the sums
// of squares of termination rule 2.
constexpr int kCheckInf = 1;
constexpr int kCheckL2 = 2;
// ... measuring one point only (the Halpern iteration's T(z)): the current
// point's terms are not formed, and its slots carry the measured point's
constexpr int kCheckOne = 4;

// The part of a multiplier or reduced cost v (internal minimize sense)
// outside the sign the bounds of its row or column allow: >= 0 with only a
// finite lower end, <= 0 with only a finite upper end, any sign with both,
// 0 with neither.
__device__ __forceinline__ double sign_violation(double v, double lo, double hi) {
    const bool fl = fb(lo), fh = fb(hi);
    if (fl && fh) return 0.0;
    if (fl) return v < 0.0 ? -v : 0.0;
    if (fh) return v > 0.0 ? v : 0.0;
    return fabs(v);
}

struct Terms {
    double cp = 0, cd = 0, ap = 0, ad = 0;         // scaled: cur / avg, primal / dual
    double ocp = 0, ocd = 0, oap = 0, oad = 0;     // original space
    double pobj_c = 0, dobj_c = 0, pobj_a = 0, dobj_a = 0;
    // termination rule 2: sums of squares of the primal and dual violations
    // (original units), current and average
    double ppc = 0, ddc = 0, ppa = 0, dda = 0;
    // infeasibility test: row-side and column-side ranges of the change of y
    // (FarkasCertificate::row_side_range / column_side_range), max |dy|
    double rlo = 0, rhi = 0, clo = 0, chi = 0, raymax = 0;
    // ray test: max |d| and c^T d of the projected change of x
    double xmax = 0, xobj = 0;
};

// How far a change d of a bounded quantity leaves the recession cone of
// [lo, hi]: a finite lower end allows no decrease, a finite upper end no
// increase.
__device__ __forceinline__ double cone_violation(double d, double lo, double hi) {
    if (d < 0.0 && fb(lo)) return -d;
    if (d > 0.0 && fb(hi)) return d;
    return 0.0;
}

// term_range of the reference's certificate checker (duals.cpp:16-20):
// mult * [lo, hi] (reversed for a negative multiplier, exactly {0} for a zero
// one), added into the running range [lo_acc, hi_acc].
__device__ __forceinline__ void ray_term(double mult, double lo, double hi, double& lo_acc,
                                         double& hi_acc) {
    if (mult == 0.0) return;
    if (mult > 0.0) {
        lo_acc += mult * lo;
        hi_acc += mult * hi;
    } else {
        lo_acc += mult * hi;
        hi_acc += mult * lo;
    }
}

// H: the caller knows the Halpern form is on (the check's one-point instance)
template <class T, bool H = false>
__device__ __forceinline__ double avg_x(const Iterates<T>& it, int j, double inv) {
    if constexpr (std::is_same<T, float>::value) {
        if (H || it.halpern) return static_cast<double>(it.psx[j]);  // T(z); the FP64 sums stay 0
        return (it.xsum[j] + static_cast<double>(it.psx[j])) * inv;
    }
    if (H) return it.xsum[j];
    return it.xsum[j] * inv;
}
template <class T, bool H = false>
__device__ __forceinline__ double avg_y(const Iterates<T>& it, int i, double inv) {
    if constexpr (std::is_same<T, float>::value) {
        if (H || it.halpern) return static_cast<double>(it.psy[i]);
        return (it.ysum[i] + static_cast<double>(it.psy[i])) * inv;
    }
    if (H) return it.ysum[i];
    return it.ysum[i] * inv;
}
// The current point's entry for the check's products; the Halpern form
// measures T(z) alone (z itself is no candidate), so it skips the gather.
template <class T>
__device__ __forceinline__ double cur_x(const Iterates<T>& it, int j) {
    return it.halpern ? 0.0 : static_cast<double>(it.x[j]);
}
template <class T>
__device__ __forceinline__ double cur_y(const Iterates<T>& it, int i) {
    return it.halpern ? 0.0 : static_cast<double>(it.y[i]);
}

}  // namespace
}  // namespace pdhg
