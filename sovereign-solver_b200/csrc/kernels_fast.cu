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
//   rows with <= kLongRow nonzeros    VW lanes per row (VW = power of two ~
//                                     mean length), lanes stride the row,
//                                     shuffle reduction;
//   rows of kLongRow..kHugeRow        one warp per row, 128-bit vector loads
//                                     of values and indices, shuffle reduction;
//   longer rows                       one CTA per row, block reduction.
// The epilogue of a short row runs on the group's lane 0, so consecutive
// groups touch consecutive vector entries (coalesced).
//
// The check (every restart_check_period iterations) is ONE fused kernel: FP64
// values, the current point and the Cesaro average in the same pass, scaled
// residuals (kkt_residual, pdhg.cpp:87-136) and original-space residuals
// (original_space_residual, pdhg.cpp:145-199) derived elementwise from the
// scaled products: A_o x_o = D_r^-1 (A_s x_s) and (c - A^T y)_o = r_s / D_c.
// Its last CTA takes the candidate / termination / restart decision.
#include <type_traits>

#include "engine.cuh"
#include "fast_common.cuh"

// CTAs per SM the iteration kernels are compiled to fit (register budget);
// build knobs, 1 = no constraint. The short-row kernel is lean: eight CTAs
// (32 registers) fit in FP32, six in FP64 without spills.
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

namespace pdhg {

namespace {

// ---------------------------------------------------------------------------
// Iteration kernels
// ---------------------------------------------------------------------------
//
// One SpMV-plus-update pass is split by row length into two kernels, so the
// short-row kernel keeps its registers (and occupancy) low:
//   fast_iter       rows of at most kLongRow entries, groups of VW lanes;
//   fast_iter_long  rows longer than kLongRow: one CTA each (long_mode 0), or
//                   one warp each up to kHugeRow entries and one CTA each
//                   above (long_mode 1).
// `reset` is set on the first kernel of a period's first pass: it clears the
// flags the previous period's restart kernel consumed.

__device__ __forceinline__ void iter_reset(DevState* st, int reset) {
    if (reset && blockIdx.x == 0 && threadIdx.x == 0) {
        st->restart = 0;
        st->fold = 0;
    }
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
    const int lane = threadIdx.x & (VW - 1);
    const int r = (blockIdx.x * kBlock + threadIdx.x) / VW;
    if (r >= M.rows) return;
    EpiIn<T> in{};
    if (lane == 0) in = epi_load<T, PRIMAL>(a.it, pv, r, first, fresh);
    const int b = __ldcs(M.rp + r), e = __ldcs(M.rp + r + 1);
    if (e - b > kLongRow) return;  // fast_iter_long handles it
    T acc = T(0);
    for (int k = b + lane; k < e; k += VW) acc += __ldcs(vals + k) * __ldg(xg + __ldcs(M.ci + k));
    if (VW > 1) acc = group_sum(acc, VW);
    if (lane == 0) epi_store<T, PRIMAL>(a.it, r, acc, in, tau, sigma);
}

template <class T, bool PRIMAL, int MODE>
__global__ void __launch_bounds__(kBlock, MODE == 0 ? PDHG_LONG_MIN_CTAS : PDHG_WARPROW_MIN_CTAS)
    fast_iter_long(FastIter<T> a, int first, int reset, int mid_blocks) {
    DevState* st = a.st;
    iter_reset(st, reset);
    if (st->done) return;
    const DevCsr& M = PRIMAL ? a.AT : a.A;
    const T* __restrict__ vals = mvals<T>(M);
    const T* __restrict__ xg = PRIMAL ? a.it.y : a.it.xbar;
    const PV<T> pv = pvec<T>(a.P);
    const bool fresh = first && st->fresh;
    const T tau = static_cast<T>(st->tau), sigma = static_cast<T>(st->sigma);
    if (MODE == 1 && static_cast<int>(blockIdx.x) < mid_blocks) {
        // one warp per row
        const int w = blockIdx.x * (kBlock / 32) + (threadIdx.x >> 5);
        if (w >= M.n_mid) return;
        const int r = __ldg(M.mid_rows + w);
        const int lane = threadIdx.x & 31;
        EpiIn<T> in{};
        if (lane == 0) in = epi_load<T, PRIMAL>(a.it, pv, r, first, fresh);
        const T acc = warp_row_dot<T>(M.ci, vals, xg, __ldg(M.rp + r), __ldg(M.rp + r + 1));
        if (lane == 0) epi_store<T, PRIMAL>(a.it, r, acc, in, tau, sigma);
    } else {
        // one CTA per row: every long row (mode 0) or those above kHugeRow
        const int r = MODE == 0 ? __ldg(M.long_rows + blockIdx.x)
                                : __ldg(M.huge_rows + (blockIdx.x - mid_blocks));
        EpiIn<T> in{};
        if (threadIdx.x == 0) in = epi_load<T, PRIMAL>(a.it, pv, r, first, fresh);
        const int b = __ldg(M.rp + r), e = __ldg(M.rp + r + 1);
        const T acc = long_row_dot<T>(M.ci, vals, xg, b, e);
        if (threadIdx.x == 0) epi_store<T, PRIMAL>(a.it, r, acc, in, tau, sigma);
    }
}

__global__ void k_clear_flags(DevState* st) {
    if (threadIdx.x == 0) {
        st->restart = 0;
        st->fold = 0;
    }
}

inline int iter_lanes(const DevCsr& M) { return M.iter_vw > 0 ? M.iter_vw : M.vw; }

inline int short_blocks_for(const DevCsr& M) {
    if (M.n_short == 0) return 0;
    return static_cast<int>((static_cast<int64_t>(M.rows) * iter_lanes(M) + kBlock - 1) / kBlock);
}

// Kernels one pass over M launches besides the flag reset.
inline int pass_launches(const DevCsr& M) {
    if (M.rows == 0) return 0;
    return (short_blocks_for(M) > 0 ? 1 : 0) + (M.n_long > 0 ? 1 : 0);
}

// Returns the number of kernels launched.
template <class T, bool PRIMAL>
int launch_iter(const FastIter<T>& a, int first, cudaStream_t s) {
    const DevCsr& M = PRIMAL ? a.AT : a.A;
    if (M.rows == 0) {
        if (PRIMAL && first) {
            k_clear_flags<<<1, 32, 0, s>>>(a.st);
            return 1;
        }
        return 0;
    }
    const int sb = short_blocks_for(M);
    const int mode = M.long_mode;
    const int mb = mode == 1 ? (M.n_mid + kBlock / 32 - 1) / (kBlock / 32) : 0;
    const int lb = mode == 1 ? mb + M.n_huge : M.n_long;
    const int reset_short = (PRIMAL && first) ? 1 : 0;
    const int reset_long = (PRIMAL && first && sb == 0) ? 1 : 0;
    if (sb > 0) {
        switch (iter_lanes(M)) {
            case 1: fast_iter<T, 1, PRIMAL><<<sb, kBlock, 0, s>>>(a, first, reset_short); break;
            case 2: fast_iter<T, 2, PRIMAL><<<sb, kBlock, 0, s>>>(a, first, reset_short); break;
            case 4: fast_iter<T, 4, PRIMAL><<<sb, kBlock, 0, s>>>(a, first, reset_short); break;
            case 8: fast_iter<T, 8, PRIMAL><<<sb, kBlock, 0, s>>>(a, first, reset_short); break;
            case 16: fast_iter<T, 16, PRIMAL><<<sb, kBlock, 0, s>>>(a, first, reset_short); break;
            default: fast_iter<T, 32, PRIMAL><<<sb, kBlock, 0, s>>>(a, first, reset_short); break;
        }
    }
    if (lb > 0) {
        if (mode == 1) fast_iter_long<T, PRIMAL, 1><<<lb, kBlock, 0, s>>>(a, first, reset_long, mb);
        else fast_iter_long<T, PRIMAL, 0><<<lb, kBlock, 0, s>>>(a, first, reset_long, mb);
    }
    return (sb > 0 ? 1 : 0) + (lb > 0 ? 1 : 0);
}

// ---------------------------------------------------------------------------
// Check kernel
// ---------------------------------------------------------------------------

// Per-row terms, merged into the thread's running maxima / sums.
template <class T>
__device__ __forceinline__ void row_terms(const FastCheck<T>& a, int i, double act_c,
                                          double act_a, double inv, Terms& t) {
    const DevProblem& P = a.P;
    a.cs.act_avg[i] = act_a;
    const double lo = P.rlo[i], hi = P.rhi[i];
    const double yc = static_cast<double>(a.it.y[i]);
    const double ya = avg_y(a.it, i, inv);
    t.cp = smax(t.cp, primal_term(act_c, lo, hi));
    t.ap = smax(t.ap, primal_term(act_a, lo, hi));
    t.cd = smax(t.cd, cs_term(yc, act_c, lo, hi, a.tol));
    t.ad = smax(t.ad, cs_term(ya, act_a, lo, hi, a.tol));
    const double rs = P.rs[i];
    const double lo_o = P.rlo_o[i], hi_o = P.rhi_o[i];
    const double aoc = act_c / rs, aoa = act_a / rs;
    t.ocp = smax(t.ocp, primal_term(aoc, lo_o, hi_o));
    t.oap = smax(t.oap, primal_term(aoa, lo_o, hi_o));
    t.ocd = smax(t.ocd, cs_term(yc * rs, aoc, lo_o, hi_o, a.bound_tol));
    t.oad = smax(t.oad, cs_term(ya * rs, aoa, lo_o, hi_o, a.bound_tol));
    if (a.termination_rule == 1) {  // internal (minimize) sense: y_int = y_s * rs
        t.dobj_c += clipped_inf(yc * rs, lo_o, hi_o);
        t.dobj_a += clipped_inf(ya * rs, lo_o, hi_o);
    }
}

template <class T>
__device__ __forceinline__ void col_terms(const FastCheck<T>& a, int j, double aty_c,
                                          double aty_a, double inv, Terms& t) {
    const DevProblem& P = a.P;
    const double cj = P.c[j];
    const double lo = P.lo[j], hi = P.hi[j];
    const double xc = static_cast<double>(a.it.x[j]);
    const double xa = avg_x(a.it, j, inv);
    const double rc = cj - aty_c, ra = cj - aty_a;
    t.cd = smax(t.cd, cs_term(rc, xc, lo, hi, a.tol));
    t.ad = smax(t.ad, cs_term(ra, xa, lo, hi, a.tol));
    const double cs = P.cs[j];
    const double lo_o = P.lo_o[j], hi_o = P.hi_o[j];
    t.ocd = smax(t.ocd, cs_term(rc / cs, xc * cs, lo_o, hi_o, a.bound_tol));
    t.oad = smax(t.oad, cs_term(ra / cs, xa * cs, lo_o, hi_o, a.bound_tol));
    if (a.termination_rule == 1) {  // internal sense: c_int x = sign c_o x, r_int = r_s / cs
        t.pobj_c += P.obj_sign * P.c_o[j] * (xc * cs);
        t.pobj_a += P.obj_sign * P.c_o[j] * (xa * cs);
        t.dobj_c += clipped_inf(rc / cs, lo_o, hi_o);
        t.dobj_a += clipped_inf(ra / cs, lo_o, hi_o);
    }
}

// Block maxima of the 8 residual terms, one atomicMax per CTA and slot.
__device__ void block_max_terms(const Terms& t, unsigned long long* acc) {
    __shared__ double sh[8][kBlock / 32];
    double v[8] = {t.cp, t.cd, t.ap, t.ad, t.ocp, t.ocd, t.oap, t.oad};
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int q = 0; q < 8; ++q) {
        double x = v[q];
        for (int o = 16; o > 0; o >>= 1) x = fmax(x, __shfl_xor_sync(0xffffffffu, x, o));
        if (lane == 0) sh[q][warp] = x;
    }
    __syncthreads();
    if (threadIdx.x < 8) {
        double x = 0.0;
        for (int w = 0; w < kBlock / 32; ++w) x = fmax(x, sh[threadIdx.x][w]);
        // v[0..3] -> ACC_CUR_P..ACC_AVG_D, v[4..7] -> ACC_OC_P..ACC_OA_D
        const int slot = threadIdx.x < 4 ? ACC_CUR_P + static_cast<int>(threadIdx.x)
                                         : ACC_OC_P + static_cast<int>(threadIdx.x) - 4;
        if (x > 0.0)
            atomicMax(&acc[slot], static_cast<unsigned long long>(__double_as_longlong(x)));
    }
    __syncthreads();
}

// Grid-stride over virtual blocks [row short | row long | col short | col long];
// the grid itself is capped (a few CTAs per SM), so each CTA sums its rows into
// per-thread running terms and takes part in one reduction.
template <class T>
__global__ void __launch_bounds__(kBlock) fast_check(FastCheck<T> a, int rs_blocks, int cs_blocks) {
    DevState* st = a.st;
    if (st->done) return;
    const long long k_avg = st->since_restart + a.period_iters;
    const double inv = 1.0 / static_cast<double>(k_avg);
    Terms t;
    const int b0 = rs_blocks, b1 = b0 + a.A.n_long, b2 = b1 + cs_blocks, b3 = b2 + a.AT.n_long;
    for (int bid = blockIdx.x; bid < b3; bid += gridDim.x) {
        if (bid < b1) {
            // rows of A: act = A x (current and average)
            const DevCsr& M = a.A;
            if (bid < b0) {
                const int vw = M.vw;
                const int lane = threadIdx.x & (vw - 1);
                const int r = (bid * kBlock + threadIdx.x) / vw;
                if (r < M.rows) {
                    const int b = M.rp[r], e = M.rp[r + 1];
                    if (e - b <= kLongRow) {
                        double ac = 0.0, aa = 0.0;
                        for (int k = b + lane; k < e; k += vw) {
                            const int j = M.ci[k];
                            const double v = M.v64[k];
                            ac += v * static_cast<double>(a.it.x[j]);
                            aa += v * avg_x(a.it, j, inv);
                        }
                        ac = group_sum(ac, vw);
                        aa = group_sum(aa, vw);
                        if (lane == 0) row_terms(a, r, ac, aa, inv, t);
                    }
                }
            } else {
                const int r = M.long_rows[bid - b0];
                const int b = M.rp[r], e = M.rp[r + 1];
                double ac = 0.0, aa = 0.0;
                for (int k = b + threadIdx.x; k < e; k += kBlock) {
                    const int j = M.ci[k];
                    const double v = M.v64[k];
                    ac += v * static_cast<double>(a.it.x[j]);
                    aa += v * avg_x(a.it, j, inv);
                }
                ac = block_total(ac);
                aa = block_total(aa);
                if (threadIdx.x == 0) row_terms(a, r, ac, aa, inv, t);
            }
        } else {
            // rows of A^T: aty = A^T y (current and average)
            const DevCsr& M = a.AT;
            if (bid < b2) {
                const int vw = M.vw;
                const int lane = threadIdx.x & (vw - 1);
                const int r = ((bid - b1) * kBlock + threadIdx.x) / vw;
                if (r < M.rows) {
                    const int b = M.rp[r], e = M.rp[r + 1];
                    if (e - b <= kLongRow) {
                        double ac = 0.0, aa = 0.0;
                        for (int k = b + lane; k < e; k += vw) {
                            const int i = M.ci[k];
                            const double v = M.v64[k];
                            ac += v * static_cast<double>(a.it.y[i]);
                            aa += v * avg_y(a.it, i, inv);
                        }
                        ac = group_sum(ac, vw);
                        aa = group_sum(aa, vw);
                        if (lane == 0) col_terms(a, r, ac, aa, inv, t);
                    }
                }
            } else {
                const int r = M.long_rows[bid - b2];
                const int b = M.rp[r], e = M.rp[r + 1];
                double ac = 0.0, aa = 0.0;
                for (int k = b + threadIdx.x; k < e; k += kBlock) {
                    const int i = M.ci[k];
                    const double v = M.v64[k];
                    ac += v * static_cast<double>(a.it.y[i]);
                    aa += v * avg_y(a.it, i, inv);
                }
                ac = block_total(ac);
                aa = block_total(aa);
                if (threadIdx.x == 0) col_terms(a, r, ac, aa, inv, t);
            }
        }
    }
    block_max_terms(t, st->acc);
    if (a.termination_rule == 1) {
        const double s0 = block_sum_det(t.pobj_c);
        const double s1 = block_sum_det(t.dobj_c);
        const double s2 = block_sum_det(t.pobj_a);
        const double s3 = block_sum_det(t.dobj_a);
        if (threadIdx.x == 0) {
            double* p = a.cs.part + 4 * blockIdx.x;
            p[0] = s0; p[1] = s1; p[2] = s2; p[3] = s3;
        }
    }
    if (!last_block(&st->ticket[TK_FAST]) || threadIdx.x != 0) return;

    // ---- decision (one thread) ----
    const double cp = acc_read(&st->acc[ACC_CUR_P]), cd = acc_read(&st->acc[ACC_CUR_D]);
    const double ap = acc_read(&st->acc[ACC_AVG_P]), ad = acc_read(&st->acc[ACC_AVG_D]);
    const double ocp = acc_read(&st->acc[ACC_OC_P]), ocd = acc_read(&st->acc[ACC_OC_D]);
    const double oap = acc_read(&st->acc[ACC_OA_P]), oad = acc_read(&st->acc[ACC_OA_D]);
    for (int q = ACC_CUR_P; q <= ACC_OA_D; ++q) st->acc[q] = 0ull;
    st->ticket[TK_FAST] = 0u;
    const double cur = smax(cp, cd), avg = smax(ap, ad);
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
        const bool ab = avg <= cur;  // pdhg.cpp:354
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
            if (a.termination_rule == 1) {
                double ps = 0.0, ds = 0.0;
                const volatile double* part = a.cs.part;
                const int off = ab ? 2 : 0;
                for (unsigned b = 0; b < gridDim.x; ++b) {
                    ps += part[4 * b + off];
                    ds += part[4 * b + off + 1];
                }
                ps += a.P.obj_sign * a.P.obj_const;  // the constant shifts both objectives
                ds += a.P.obj_sign * a.P.obj_const;
                const double gap = fabs(ps - ds) / (1.0 + fabs(ps) + fabs(ds));
                rel = smax(smax(op / (1.0 + a.P.bnorm), od / (1.0 + a.P.cnorm)), gap);
            }
            st->rel_kkt = rel;
            const bool conv = (a.termination_rule == 1) ? (rel < a.tol) : (orig < a.tol);
            if (conv) {  // pdhg.cpp:383-389
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
                // adaptive: candidate = the better of average and current
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
                st->fold = std::is_same<T, float>::value ? 1 : 0;
                const int stop = a.mail != nullptr ? a.mail->stop_request : 0;
                if (stop != 0) {
                    st->done = 1;
                    st->status = stop;
                    st->stop_iter = it_idx + 1;
                }
            }
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
    if (!last_block(&st->ticket[TK_RESTART]) || threadIdx.x != 0) return;
    st->ticket[TK_RESTART] = 0u;
    double sx = 0.0, sy = 0.0;
    const volatile double* part = a.cs.part;
    for (unsigned b = 0; b < gridDim.x; ++b) {
        sx += part[2 * b];
        sy += part[2 * b + 1];
    }
    const double dx = sqrt(sx), dy = sqrt(sy);
    if (dx > 1e-10 && dy > 1e-10) {
        // omega <- exp(0.5 log(dy/dx) + 0.5 log(omega))
        st->omega = sqrt(st->omega * (dy / dx));
        st->tau = st->eta / st->omega;
        st->sigma = st->eta * st->omega;
    }
}

}  // namespace

template <class T>
int launch_fast_primal(const FastIter<T>& a, int first, cudaStream_t s) {
    return launch_iter<T, true>(a, first, s);
}
template <class T>
int launch_fast_dual(const FastIter<T>& a, int first, cudaStream_t s) {
    return launch_iter<T, false>(a, first, s);
}
template <class T>
int fast_launches_per_iteration(const FastIter<T>& a) {
    return pass_launches(a.AT) + pass_launches(a.A);
}

template <class T>
void launch_fast_check(const FastCheck<T>& a, cudaStream_t s) {
    const int rsb = short_blocks_for(a.A);
    const int csb = short_blocks_for(a.AT);
    int grid = rsb + a.A.n_long + csb + a.AT.n_long;
    if (a.grid_cap > 0 && grid > a.grid_cap) grid = a.grid_cap;
    if (grid == 0) grid = 1;
    fast_check<T><<<grid, kBlock, 0, s>>>(a, rsb, csb);
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
    return short_blocks_for(A) + A.n_long + short_blocks_for(AT) + AT.n_long + 1;
}

template int launch_fast_primal<float>(const FastIter<float>&, int, cudaStream_t);
template int launch_fast_primal<double>(const FastIter<double>&, int, cudaStream_t);
template int launch_fast_dual<float>(const FastIter<float>&, int, cudaStream_t);
template int launch_fast_dual<double>(const FastIter<double>&, int, cudaStream_t);
template int fast_launches_per_iteration<float>(const FastIter<float>&);
template int fast_launches_per_iteration<double>(const FastIter<double>&);
template void launch_fast_check<float>(const FastCheck<float>&, cudaStream_t);
template void launch_fast_check<double>(const FastCheck<double>&, cudaStream_t);
template void launch_fast_restart<float>(const FastCheck<float>&, cudaStream_t);
template void launch_fast_restart<double>(const FastCheck<double>&, cudaStream_t);

}  // namespace pdhg
