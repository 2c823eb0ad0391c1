// batch_kernels.cu -- kernels of the batched engine; see batch_kernels.cuh.
#include <algorithm>
#include <cmath>

#include "batch_kernels.cuh"
#include "fast_common.cuh"

namespace pdhg {

namespace {

__host__ __device__ inline int nblk(int64_t n) { return static_cast<int>((n + kBlock - 1) / kBlock); }

inline int short_blocks(const DevCsr& M) {
    if (M.n_short == 0) return 0;
    return static_cast<int>((static_cast<int64_t>(M.rows) * M.vw + kBlock - 1) / kBlock);
}

// Block reductions over all threads (every thread calls; result in all threads).
__device__ double bmax(double v) {
    __shared__ double sh[kBlock / 32];
    __shared__ double tot;
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < kBlock / 32; ++w) t = fmax(t, sh[w]);
        tot = t;
    }
    __syncthreads();
    const double r = tot;
    __syncthreads();
    return r;
}

// ---------------------------------------------------------------------------
// Iterations: the single engine's fused kernels with a per-row instance lookup
// ---------------------------------------------------------------------------

// One lane-group block of rows (kBlock / VW rows, groups of VW lanes): the
// rows of instances still iterating, rows above kLongRow left to the CTA path.
template <class T, int VW, bool PRIMAL>
__device__ __forceinline__ void batch_block(const BatchView& b, const Iterates<T>& it, int first,
                                            int hk, int blk) {
    const DevCsr& M = PRIMAL ? b.AT : b.A;
    const int32_t* inst_of = PRIMAL ? b.col_inst : b.row_inst;
    const T* __restrict__ vals = mvals<T>(M);
    const T* __restrict__ xg = PRIMAL ? it.y : it.xbar;
    const PV<T> pv = pvec<T>(b.P);
    const int lane = threadIdx.x & (VW - 1);
    const int r = (blk * kBlock + threadIdx.x) / VW;
    if (r >= M.rows) return;
    const InstState& s = b.is[inst_of[r]];
    if (s.done) return;  // uniform within the row's lane group
    const bool fresh = first && s.fresh;
    const T tau = static_cast<T>(s.tau), sigma = static_cast<T>(s.sigma);
    const Hw<T> hw = halpern_weight<T>(it, s.since_restart, hk);
    EpiIn<T> in{};
    if (lane == 0) in = epi_load<T, PRIMAL, false>(it, pv, r, first, fresh, hw);
    const int rb = __ldcs(M.rp + r), re = __ldcs(M.rp + r + 1);
    if (re - rb > kLongRow) return;
    // rounds of four entries per lane: the index and value loads of a round
    // are all in flight before its gathers
    T acc = T(0);
    for (int k0 = rb + lane; k0 < re; k0 += 4 * VW) {
        int c[4];
        T v[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int k = k0 + u * VW;
            c[u] = k < re ? __ldcs(M.ci + k) : 0;
            v[u] = k < re ? __ldcs(vals + k) : T(0);
        }
#pragma unroll
        for (int u = 0; u < 4; ++u)
            if (k0 + u * VW < re) acc += v[u] * __ldg(xg + c[u]);
    }
    if (VW > 1) acc = group_sum(acc, VW);
    if (lane == 0) epi_store<T, PRIMAL, false>(it, r, acc, in, tau, sigma, hw, 1);
}

// The first short_grid CTAs take one block each of the active block list (the
// grid covers every block; CTAs past the list's length exit at once); with
// LONG, one CTA per row above kLongRow follows. LONG = false (no such row)
// compiles the CTA-per-row path out, which keeps the registers of the
// lane-group path.
template <class T, int VW, bool PRIMAL, bool LONG>
__global__ void __launch_bounds__(kBlock) batch_iter(BatchView b, Iterates<T> it, int first,
                                                     int hk, int short_grid) {
    if (b.g->done) return;
    if (!LONG || static_cast<int>(blockIdx.x) < short_grid) {
        const int pi = PRIMAL ? 1 : 0;
        if (static_cast<int>(blockIdx.x) >= b.g->nblk[pi]) return;
        batch_block<T, VW, PRIMAL>(b, it, first, hk, b.blk_list[pi][blockIdx.x]);
    } else {
        const DevCsr& M = PRIMAL ? b.AT : b.A;
        const int32_t* inst_of = PRIMAL ? b.col_inst : b.row_inst;
        const int r = M.long_rows[blockIdx.x - short_grid];
        const InstState& s = b.is[inst_of[r]];
        if (s.done) return;  // uniform within the CTA
        const PV<T> pv = pvec<T>(b.P);
        const bool fresh = first && s.fresh;
        const T tau = static_cast<T>(s.tau), sigma = static_cast<T>(s.sigma);
        const Hw<T> hw = halpern_weight<T>(it, s.since_restart, hk);
        EpiIn<T> in{};
        if (threadIdx.x == 0) in = epi_load<T, PRIMAL, false>(it, pv, r, first, fresh, hw);
        const T acc = long_row_dot<T>(M.ci, mvals<T>(M), PRIMAL ? it.y : it.xbar, M.rp[r], M.rp[r + 1]);
        if (threadIdx.x == 0) epi_store<T, PRIMAL, false>(it, r, acc, in, tau, sigma, hw, 1);
    }
}

// ---------------------------------------------------------------------------
// Check: each instance in one or more CTA parts, the last part of an instance
// merging and deciding (kkt_residual, original_space_residual, candidate,
// termination, restart rule: pdhg.cpp:333-408)
// ---------------------------------------------------------------------------

template <class T>
__device__ __forceinline__ void inst_row_terms(const BatchView& b, const Iterates<T>& it,
                                               const BatchParams& p, int i, double act_c,
                                               double act_a, double inv, Terms& t) {
    const DevProblem& P = b.P;
    p.act_avg[i] = act_a;
    const double lo = P.rlo[i], hi = P.rhi[i];
    const double yc = static_cast<double>(it.y[i]);
    const double ya = avg_y(it, i, inv);
    t.cp = smax(t.cp, primal_term(act_c, lo, hi));
    t.ap = smax(t.ap, primal_term(act_a, lo, hi));
    t.cd = smax(t.cd, cs_term(yc, act_c, lo, hi, p.tol));
    t.ad = smax(t.ad, cs_term(ya, act_a, lo, hi, p.tol));
    const double rs = P.rs[i];
    const double lo_o = P.rlo_o[i], hi_o = P.rhi_o[i];
    const double aoc = act_c / rs, aoa = act_a / rs;
    t.ocp = smax(t.ocp, primal_term(aoc, lo_o, hi_o));
    t.oap = smax(t.oap, primal_term(aoa, lo_o, hi_o));
    t.ocd = smax(t.ocd, cs_term(yc * rs, aoc, lo_o, hi_o, p.bound_tol));
    t.oad = smax(t.oad, cs_term(ya * rs, aoa, lo_o, hi_o, p.bound_tol));
    if (p.termination_rule != 0) {
        t.dobj_c += clipped_inf(yc * rs, lo_o, hi_o);
        t.dobj_a += clipped_inf(ya * rs, lo_o, hi_o);
    }
    if (p.termination_rule == 2) {  // squares of the row violation and of y's sign violation
        const double pc = primal_term(aoc, lo_o, hi_o), pa = primal_term(aoa, lo_o, hi_o);
        const double dc = sign_violation(yc * rs, lo_o, hi_o);
        const double da = sign_violation(ya * rs, lo_o, hi_o);
        t.ppc += pc * pc;
        t.ppa += pa * pa;
        t.ddc += dc * dc;
        t.dda += da * da;
    }
}

template <class T>
__device__ __forceinline__ void inst_col_terms(const BatchView& b, const Iterates<T>& it,
                                               const BatchParams& p, double sign, int j,
                                               double aty_c, double aty_a, double inv,
                                               Terms& t) {
    const DevProblem& P = b.P;
    const double cj = P.c[j];
    const double lo = P.lo[j], hi = P.hi[j];
    const double xc = static_cast<double>(it.x[j]);
    const double xa = avg_x(it, j, inv);
    const double rc = cj - aty_c, ra = cj - aty_a;
    t.cd = smax(t.cd, cs_term(rc, xc, lo, hi, p.tol));
    t.ad = smax(t.ad, cs_term(ra, xa, lo, hi, p.tol));
    const double cs = P.cs[j];
    const double lo_o = P.lo_o[j], hi_o = P.hi_o[j];
    t.ocd = smax(t.ocd, cs_term(rc / cs, xc * cs, lo_o, hi_o, p.bound_tol));
    t.oad = smax(t.oad, cs_term(ra / cs, xa * cs, lo_o, hi_o, p.bound_tol));
    if (p.termination_rule == 2) {  // squares of the reduced cost's sign violation
        const double dc = sign_violation(rc / cs, lo_o, hi_o);
        const double da = sign_violation(ra / cs, lo_o, hi_o);
        t.ddc += dc * dc;
        t.dda += da * da;
    }
    if (p.termination_rule != 0) {
        t.pobj_c += sign * P.c_o[j] * (xc * cs);
        t.pobj_a += sign * P.c_o[j] * (xa * cs);
        t.dobj_c += clipped_inf(rc / cs, lo_o, hi_o);
        t.dobj_a += clipped_inf(ra / cs, lo_o, hi_o);
    }
}

// The instance's rows (or columns) in lane groups of M.vw: act / aty for the
// current point and the average in one pass.
template <class T, bool COLS>
__device__ __forceinline__ void inst_pass(const BatchView& b, const Iterates<T>& it,
                                          const BatchParams& p, int k, int part, int parts,
                                          double inv, double sign, Terms& t) {
    const DevCsr& M = COLS ? b.AT : b.A;
    const int vw = M.vw;
    const int lane = threadIdx.x & (vw - 1);
    const int groups = kBlock / vw;
    const int q0 = COLS ? b.col_off[k] : b.row_off[k];
    const int q1 = COLS ? b.col_off[k + 1] : b.row_off[k + 1];
    // part `part` of `parts` of the instance's rows (columns)
    const int r0 = q0 + static_cast<int>(static_cast<int64_t>(q1 - q0) * part / parts);
    const int r1 = q0 + static_cast<int>(static_cast<int64_t>(q1 - q0) * (part + 1) / parts);
    for (int r = r0 + static_cast<int>(threadIdx.x) / vw; r < r1; r += groups) {
        double ac = 0.0, aa = 0.0;
        for (int q = M.rp[r] + lane; q < M.rp[r + 1]; q += vw) {
            const int c = M.ci[q];
            const double v = M.v64[q];
            if (COLS) {
                ac += v * cur_y(it, c);
                aa += v * avg_y(it, c, inv);
            } else {
                ac += v * cur_x(it, c);
                aa += v * avg_x(it, c, inv);
            }
        }
        ac = group_sum(ac, vw);
        aa = group_sum(aa, vw);
        if (lane == 0) {
            if (COLS) inst_col_terms(b, it, p, sign, r, ac, aa, inv, t);
            else inst_row_terms(b, it, p, r, ac, aa, inv, t);
        }
    }
}

__device__ void finish_instance(const BatchView& b, InstState& s) {
    const int left = atomicSub(&b.g->active, 1);
    if (left == 1) b.g->done = 1;
    b.g->dirty = 1;
}

template <class T>
__global__ void __launch_bounds__(kBlock) batch_check(BatchView b, Iterates<T> it, BatchParams p) {
    const int4 item = b.chk_item[blockIdx.x];
    const int k = item.x, part = item.y, parts = item.z;
    InstState& s = b.is[k];
    // uniform per CTA. Only the instance's last CTA writes s.done, and only
    // after every CTA of the instance has taken its ticket -- each read this
    // flag before that -- so all parts of an instance agree. (The global done
    // flag is written by other CTAs of this launch, so it must not decide an
    // early exit here; when it is set every instance is done anyway.)
    if (s.done) return;
    const long long k_avg = s.since_restart + p.period;
    // Halpern: the sums' slots hold T(z) itself
    const double inv = it.halpern ? 1.0 : 1.0 / static_cast<double>(k_avg);
    Terms t;
    inst_pass<T, false>(b, it, p, k, part, parts, inv, s.obj_sign, t);
    inst_pass<T, true>(b, it, p, k, part, parts, inv, s.obj_sign, t);
    constexpr int K = kBatchCheckVals;
    double v[K];
    v[0] = bmax(t.cp); v[1] = bmax(t.cd); v[2] = bmax(t.ap); v[3] = bmax(t.ad);
    v[4] = bmax(t.ocp); v[5] = bmax(t.ocd); v[6] = bmax(t.oap); v[7] = bmax(t.oad);
    for (int q = 8; q < K; ++q) v[q] = 0.0;
    if (p.termination_rule != 0) {
        v[8] = block_sum_det(t.pobj_c);
        v[9] = block_sum_det(t.dobj_c);
        v[10] = block_sum_det(t.pobj_a);
        v[11] = block_sum_det(t.dobj_a);
    }
    if (p.termination_rule == 2) {
        v[12] = block_sum_det(t.ppc);
        v[13] = block_sum_det(t.ddc);
        v[14] = block_sum_det(t.ppa);
        v[15] = block_sum_det(t.dda);
    }
    if (threadIdx.x != 0) return;
    if (parts > 1) {
        // store this part, take the instance's ticket; the last part merges
        // (maxima order-free, sums in part order) and goes on to the decision
        double* mine = b.chk_part + K * static_cast<int64_t>(blockIdx.x);
        for (int q = 0; q < K; ++q) mine[q] = v[q];
        __threadfence();
        if (atomicAdd(b.chk_ticket + k, 1u) != static_cast<unsigned>(parts - 1)) return;
        __threadfence();
        const double* first = b.chk_part + K * (static_cast<int64_t>(blockIdx.x) - part);
        for (int q = 0; q < K; ++q) v[q] = q < 8 ? 0.0 : __ldcg(first + q);
        for (int j = 0; j < parts; ++j) {
            for (int q = 0; q < 8; ++q) v[q] = smax(v[q], __ldcg(first + K * j + q));
            if (j > 0)
                for (int q = 8; q < K; ++q) v[q] += __ldcg(first + K * j + q);
        }
        b.chk_ticket[k] = 0u;
    }
    const double cp = v[0], cd = v[1], ap = v[2], ad = v[3];
    const double ocp = v[4], ocd = v[5], oap = v[6], oad = v[7];
    const double s0 = v[8], s1 = v[9], s2 = v[10], s3 = v[11];
    // ---- the instance's decision (as the single engine's check) ----
    double cur = smax(cp, cd), avg = smax(ap, ad);
    // termination rule 2: relative parts of the current point and the average
    // (original units, l2 norms); their l2 norm is restart rule 2's measure
    double part_c[3] = {0, 0, 0}, part_a[3] = {0, 0, 0};
    if (p.termination_rule == 2) {
        const double k0 = s.obj_sign * s.obj_const;
        const double pp[2] = {v[12], v[14]}, dd[2] = {v[13], v[15]};
        const double ps[2] = {s0 + k0, s2 + k0}, ds[2] = {s1 + k0, s3 + k0};
        for (int w = 0; w < 2; ++w) {
            double* pt = w ? part_a : part_c;
            pt[0] = sqrt(pp[w]) / (1.0 + s.bnorm2);
            pt[1] = sqrt(dd[w]) / (1.0 + s.cnorm2);
            pt[2] = fabs(ps[w] - ds[w]) / (1.0 + fabs(ps[w]) + fabs(ds[w]));
        }
        if (p.restart_rule == 2) {
            const double mc = sqrt(part_c[0] * part_c[0] + part_c[1] * part_c[1] + part_c[2] * part_c[2]);
            const double ma = sqrt(part_a[0] * part_a[0] + part_a[1] * part_a[1] + part_a[2] * part_a[2]);
            cur = isfinite(cur) ? mc : cur;
            avg = isfinite(avg) ? ma : avg;
        }
    }
    if (it.halpern) cur = avg;  // only T(z) is measured
    s.cur_res = cur;
    s.avg_res = avg;
    s.inv = inv;
    s.restart = 0;
    s.fold = 0;
    const long long it_idx = b.g->iter + p.period - 1;
    if (!isfinite(cur) || !isfinite(avg)) {
        s.done = 1;
        s.status = kStatusNumericalFailure;
        s.fail_kind = 1;
        s.stop_iter = it_idx;
        finish_instance(b, s);
        return;
    }
    const bool ab = it.halpern ? true : avg <= cur;  // Halpern: the candidate is T(z)
    s.avg_better = ab ? 1 : 0;
    const double op = ab ? oap : ocp, od = ab ? oad : ocd;
    const double orig = smax(op, od);
    s.orig_res = orig;
    if (!isfinite(orig)) {
        s.done = 1;
        s.status = kStatusNumericalFailure;
        s.fail_kind = 2;
        s.stop_iter = it_idx;
        finish_instance(b, s);
        return;
    }
    double rel = 0.0;
    if (p.termination_rule == 2) {
        const double* pt = ab ? part_a : part_c;
        rel = smax(smax(pt[0], pt[1]), pt[2]);
    } else if (p.termination_rule == 1) {
        // the objective constant shifts both objectives
        const double ps = (ab ? s2 : s0) + s.obj_sign * s.obj_const;
        const double ds = (ab ? s3 : s1) + s.obj_sign * s.obj_const;
        const double gap = fabs(ps - ds) / (1.0 + fabs(ps) + fabs(ds));
        rel = smax(smax(op / (1.0 + s.bnorm), od / (1.0 + s.cnorm)), gap);
    }
    s.rel_kkt = rel;
    const bool conv = (p.termination_rule != 0) ? (rel < p.tol) : (orig < p.tol);
    if (conv) {
        s.done = 1;
        s.converged = 1;
        s.status = kStatusOptimal;
        s.stop_iter = it_idx + 1;
        finish_instance(b, s);
        return;
    }
    if (p.restart_rule == 0) {
        if (!isfinite(s.res_last)) s.res_last = cur;
        if (avg <= p.restart_decrease * s.res_last) {
            s.restart = 1;
            s.restart_to_avg = 1;
            s.res_last = avg;
            s.since_restart = 0;
            s.restarts += 1;
        } else {
            s.since_restart += p.period;
        }
    } else {
        const double cand = ab ? avg : cur;
        if (!isfinite(s.res_last)) s.res_last = cur;
        const long long span = s.since_restart + p.period;
        const long long total = b.g->iter + p.period;
        const bool sufficient = cand <= 0.2 * s.res_last;
        const bool necessary = cand <= 0.8 * s.res_last && cand > s.res_prev_cand;
        const bool artificial = static_cast<double>(span) >= 0.36 * static_cast<double>(total);
        s.res_prev_cand = cand;
        if (sufficient || necessary || artificial) {
            s.restart = 1;
            s.restart_to_avg = ab ? 1 : 0;
            s.res_last = cand;
            s.since_restart = 0;
            s.restarts += 1;
        } else {
            s.since_restart = span;
        }
    }
    s.fresh = s.restart;
    s.fold = std::is_same<T, float>::value && !it.halpern ? 1 : 0;
    if (p.allow_switch) {  // no 2% gain in 25 checks: the FP32 phase of this instance ends
        // under rule 2 only at FP32's precision floor (as the single engine:
        // plateaus above kFp32Zone are the method's own)
        const double r = p.termination_rule != 0 ? rel : orig;
        if (p.termination_rule == 2 && r > kFp32Zone) {
            s.since_improve = 0;
            if (r < s.best_res) s.best_res = r;
        } else if (r < 0.98 * s.best_res) {
            s.best_res = r;
            s.since_improve = 0;
        } else if (++s.since_improve >= 25) {
            s.done = 1;
            s.stalled = 1;
            s.status = kBatchStalled;
            s.stop_iter = it_idx + 1;
            finish_instance(b, s);
            return;
        }
    }
    const int stop = b.mail != nullptr ? b.mail->stop_request : 0;
    if (stop != 0) {
        s.done = 1;
        s.status = stop;
        s.stop_iter = it_idx + 1;
        finish_instance(b, s);
    }
}

// Restart (to the average or the current point), the fold of the mixed mode's
// period sums, and the primal-weight update: one CTA per instance.
template <class T>
__global__ void __launch_bounds__(kBlock) batch_restart(BatchView b, Iterates<T> it, BatchParams p) {
    const int k = blockIdx.x;
    InstState& s = b.is[k];
    const int restart = s.restart, fold = s.fold;
    if (!restart && !fold) return;  // uniform per CTA
    const bool to_avg = s.restart_to_avg != 0;
    const double inv = s.inv;
    const PV<T> pv = pvec<T>(b.P);
    double dx2 = 0.0, dy2 = 0.0;
    for (int j = b.col_off[k] + threadIdx.x; j < b.col_off[k + 1]; j += kBlock) {
        if (restart && to_avg) it.x[j] = clampT<T>(static_cast<T>(avg_x(it, j, inv)), pv.lo[j], pv.hi[j]);
        if (restart && it.halpern) it.xa[j] = it.x[j];  // the new anchor
        if (restart && p.primal_weight_update) {
            const double xn = static_cast<double>(it.x[j]);
            const double d = xn - p.x_last[j];
            dx2 += d * d;
            p.x_last[j] = xn;
        }
        if constexpr (std::is_same<T, float>::value)
            it.xsum[j] = restart ? 0.0 : it.xsum[j] + static_cast<double>(it.psx[j]);
    }
    for (int i = b.row_off[k] + threadIdx.x; i < b.row_off[k + 1]; i += kBlock) {
        if (restart && to_avg) {
            it.y[i] = static_cast<T>(avg_y(it, i, inv));
            it.s[i] = clampT<T>(static_cast<T>(p.act_avg[i]), pv.rlo[i], pv.rhi[i]);
        }
        if (restart && it.halpern) {
            it.ya[i] = it.y[i];
            it.sa[i] = it.s[i];
        }
        if (restart && p.primal_weight_update) {
            const double yn = static_cast<double>(it.y[i]);
            const double d = yn - p.y_last[i];
            dy2 += d * d;
            p.y_last[i] = yn;
        }
        if constexpr (std::is_same<T, float>::value)
            it.ysum[i] = restart ? 0.0 : it.ysum[i] + static_cast<double>(it.psy[i]);
    }
    const double sx = block_sum_det(dx2), sy = block_sum_det(dy2);
    if (threadIdx.x == 0) {
        if (restart && p.primal_weight_update) {
            const double dx = sqrt(sx), dy = sqrt(sy);
            if (dx > 1e-10 && dy > 1e-10) {
                s.omega = sqrt(s.omega * (dy / dx));
                s.tau = s.eta / s.omega;
                s.sigma = s.eta * s.omega;
            }
        }
        s.restart = 0;  // this CTA alone reads and clears the instance's flags
        s.fold = 0;
    }
}

// Period bookkeeping and the WHILE condition of the solve graph.
__global__ void batch_tick(BatchView b, long long period, long long budget_iters,
                           cudaGraphConditionalHandle handle, int use_handle) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    BatchGlobal* g = b.g;
    if (!g->done) {
        g->iter += period;
        g->checks += 1;
    }
    // the loop continues while an instance is active and a full period fits
    const bool cont = !g->done && g->iter + period <= budget_iters;
    if (b.mail != nullptr) {
        b.mail->iter = g->iter;
        b.mail->checks = g->checks;
        b.mail->restarts = g->active;
        __threadfence_system();
        b.mail->done = g->done;
        __threadfence_system();
    }
    if (use_handle) cudaGraphSetConditional(handle, cont ? 1u : 0u);
}

constexpr int kCompactThreads = 1024;

// Exclusive scan of one int per thread over the CTA (kCompactThreads); every
// thread gets its offset and the total.
__device__ int cta_scan(int v, int* total) {
    __shared__ int warp_tot[kCompactThreads / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int x = v;
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) warp_tot[warp] = x;
    __syncthreads();
    if (warp == 0) {
        int w = lane < kCompactThreads / 32 ? warp_tot[lane] : 0;
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += y;
        }
        if (lane < kCompactThreads / 32) warp_tot[lane] = w;  // inclusive warp totals
    }
    __syncthreads();
    const int before = warp > 0 ? warp_tot[warp - 1] : 0;
    *total = warp_tot[kCompactThreads / 32 - 1];
    __syncthreads();
    return before + x - v;
}

// One CTA: when g->dirty, for A's rows and A^T's rows, flag the lane-group
// blocks holding a row of an instance not done (an instance's rows [r0, r1)
// span blocks r0 vw / kBlock .. (r1 vw - 1) / kBlock; a block shared by two
// instances is flagged once), then write the flagged blocks in order into the
// list and their number into g->nblk. Clears g->dirty.
__global__ void __launch_bounds__(kCompactThreads) batch_compact(BatchView b, int nb_a, int nb_t) {
    __shared__ int dirty;
    if (threadIdx.x == 0) dirty = b.g->dirty;
    __syncthreads();
    if (!dirty) return;
    for (int mat = 0; mat < 2; ++mat) {
        const int nb = mat == 0 ? nb_a : nb_t;
        const int vw = mat == 0 ? b.A.vw : b.AT.vw;
        const int32_t* off = mat == 0 ? b.row_off : b.col_off;
        unsigned char* flag = b.blk_flag[mat];
        int32_t* list = b.blk_list[mat];
        for (int i = threadIdx.x; i < nb; i += kCompactThreads) flag[i] = 0;
        __syncthreads();
        for (int k = threadIdx.x; k < b.count; k += kCompactThreads) {
            if (b.is[k].done) continue;
            const int r0 = off[k], r1 = off[k + 1];
            if (r1 <= r0) continue;
            const int b0 = static_cast<int>(static_cast<int64_t>(r0) * vw / kBlock);
            const int b1 = static_cast<int>((static_cast<int64_t>(r1) * vw - 1) / kBlock);
            for (int q = b0; q <= b1 && q < nb; ++q) flag[q] = 1;
        }
        __syncthreads();
        int base = 0;
        for (int start = 0; start < nb; start += kCompactThreads) {
            const int i = start + static_cast<int>(threadIdx.x);
            const int f = i < nb ? flag[i] : 0;
            int total = 0;
            const int pos = cta_scan(f, &total);
            if (f) list[base + pos] = i;
            base += total;
        }
        if (threadIdx.x == 0) b.g->nblk[mat] = base;
        __syncthreads();
    }
    if (threadIdx.x == 0) b.g->dirty = 0;
}

__global__ void batch_fill_inst(const int32_t* off, int32_t* out) {
    const int k = blockIdx.x;
    for (int r = off[k] + threadIdx.x; r < off[k + 1]; r += kBlock) out[r] = k;
}

// Warm start into scaled space: x_s = x / cs, y_s = (y * obj_sign_k) / rs.
__global__ void batch_warm(BatchView b, double* x0, double* y0) {
    const int64_t t = blockIdx.x * static_cast<int64_t>(kBlock) + threadIdx.x;
    if (x0 != nullptr && t < b.n) x0[t] = x0[t] / b.P.cs[t];
    if (y0 != nullptr && t < b.m) y0[t] = (y0[t] * b.is[b.row_inst[t]].obj_sign) / b.P.rs[t];
}

// ---------------------------------------------------------------------------
// Power iteration per instance
// ---------------------------------------------------------------------------

// Group-lane FP64 dot of row r of M with g(col), lanes of M.vw (rows <= 512)
// or the whole warp (long rows). Every lane of the group returns the total.
template <class G>
__device__ __forceinline__ double row_dot64(const DevCsr& M, int r, int lane, int vw, G g) {
    double acc = 0.0;
    for (int q = M.rp[r] + lane; q < M.rp[r + 1]; q += vw) acc += M.v64[q] * g(M.ci[q]);
    return group_sum(acc, vw);
}

__global__ void __launch_bounds__(kBlock) batch_pw_w(BatchView b, const double* u, const double* v,
                                                     double* w) {
    const int vw = 32;  // one warp per row: setup only
    const int64_t r64 = (blockIdx.x * static_cast<int64_t>(kBlock) + threadIdx.x) / vw;
    if (r64 >= b.m) return;
    const int r = static_cast<int>(r64);
    if (b.is[b.row_inst[r]].pw_done) return;
    const int lane = threadIdx.x & 31;
    const double ax = row_dot64(b.A, r, lane, vw, [u](int j) { return u[j]; });
    if (lane == 0) w[r] = -ax + v[r];
}

__global__ void __launch_bounds__(kBlock) batch_pw_u(BatchView b, const double* w, double* u) {
    const int vw = 32;
    const int64_t r64 = (blockIdx.x * static_cast<int64_t>(kBlock) + threadIdx.x) / vw;
    if (r64 >= b.n) return;
    const int j = static_cast<int>(r64);
    if (b.is[b.col_inst[j]].pw_done) return;
    const int lane = threadIdx.x & 31;
    const double aty = row_dot64(b.AT, j, lane, vw, [w](int i) { return w[i]; });
    if (lane == 0) u[j] = -aty;
}

__global__ void __launch_bounds__(kBlock) batch_pw_norm_w(BatchView b, double* w) {
    const int k = blockIdx.x;
    InstState& s = b.is[k];
    if (s.pw_done) return;
    double ss = 0.0;
    for (int i = b.row_off[k] + threadIdx.x; i < b.row_off[k + 1]; i += kBlock) ss += w[i] * w[i];
    const double wn = sqrt(block_sum_det(ss));
    if (wn < 1e-300) {  // pdhg.cpp:63
        if (threadIdx.x == 0) s.pw_done = 1;
        return;
    }
    const double inv = 1.0 / wn;
    for (int i = b.row_off[k] + threadIdx.x; i < b.row_off[k + 1]; i += kBlock) w[i] *= inv;
}

__global__ void __launch_bounds__(kBlock) batch_pw_norm_uv(BatchView b, const double* w, double* u,
                                                           double* v) {
    const int k = blockIdx.x;
    InstState& s = b.is[k];
    if (s.pw_done) return;
    double su = 0.0, sv = 0.0;
    for (int j = b.col_off[k] + threadIdx.x; j < b.col_off[k + 1]; j += kBlock) su += u[j] * u[j];
    for (int i = b.row_off[k] + threadIdx.x; i < b.row_off[k + 1]; i += kBlock) {
        v[i] = w[i];
        sv += w[i] * w[i];
    }
    const double un = sqrt(block_sum_det(su)), vn = sqrt(block_sum_det(sv));
    const double est = sqrt(un * un + vn * vn);
    if (threadIdx.x == 0) s.opnorm = est;
    if (est < 1e-300) {  // pdhg.cpp:74
        if (threadIdx.x == 0) s.pw_done = 1;
        return;
    }
    const double inv = 1.0 / est;
    for (int j = b.col_off[k] + threadIdx.x; j < b.col_off[k + 1]; j += kBlock) u[j] *= inv;
    for (int i = b.row_off[k] + threadIdx.x; i < b.row_off[k + 1]; i += kBlock) v[i] *= inv;
}

// Step sizes (pdhg.cpp:261-265) and the initial primal weight.
__global__ void batch_steps(BatchView b, double safety, int primal_weight) {
    const int k = blockIdx.x * kBlock + threadIdx.x;
    if (k >= b.count) return;
    InstState& s = b.is[k];
    const double step = s.opnorm > 1e-9 ? safety / s.opnorm : safety;
    double omega = 1.0;
    if (primal_weight && s.cnorm2_s > 1e-10 && s.bnorm2_s > 1e-10) omega = s.cnorm2_s / s.bnorm2_s;
    s.eta = step;
    s.omega = omega;
    s.tau = omega == 1.0 ? step : step / omega;
    s.sigma = omega == 1.0 ? step : step * omega;
}

// ---------------------------------------------------------------------------
// Intake per instance
// ---------------------------------------------------------------------------

__global__ void __launch_bounds__(kBlock) batch_ruiz_max(BatchView b, DevCsr M, int transposed,
                                                         const int32_t* inst_of,
                                                         const double* rs, const double* cs,
                                                         double* out) {
    const int vw = 32;
    const int64_t r64 = (blockIdx.x * static_cast<int64_t>(kBlock) + threadIdx.x) / vw;
    if (r64 >= M.rows) return;
    const int r = static_cast<int>(r64);
    if (b.is[inst_of[r]].ruiz_done) return;
    const int lane = threadIdx.x & 31;
    double mx = 0.0;
    for (int q = M.rp[r] + lane; q < M.rp[r + 1]; q += vw) {
        const int c = M.ci[q];
        const double v = transposed ? fabs(M.v64[q]) * rs[c] * cs[r] : fabs(M.v64[q]) * rs[r] * cs[c];
        mx = smax(mx, v);
    }
    for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    if (lane == 0) out[r] = mx;
}

// One CTA per instance: r_i /= sqrt(row max), c_j /= sqrt(col max), and the
// instance's early exit when every norm is within tolerance of 1 (scaling.cpp:57-72).
__global__ void __launch_bounds__(kBlock) batch_ruiz_update(BatchView b, double* rs, double* cs,
                                                            const double* row_max,
                                                            const double* col_max, double tol) {
    const int k = blockIdx.x;
    InstState& s = b.is[k];
    if (s.ruiz_done) return;
    double worst = 0.0;
    for (int i = b.row_off[k] + threadIdx.x; i < b.row_off[k + 1]; i += kBlock)
        if (row_max[i] > 0.0) {
            rs[i] /= sqrt(row_max[i]);
            worst = smax(worst, fabs(row_max[i] - 1.0));
        }
    for (int j = b.col_off[k] + threadIdx.x; j < b.col_off[k + 1]; j += kBlock)
        if (col_max[j] > 0.0) {
            cs[j] /= sqrt(col_max[j]);
            worst = smax(worst, fabs(col_max[j] - 1.0));
        }
    const double w = bmax(worst);
    if (threadIdx.x == 0 && w < tol) s.ruiz_done = 1;
}

__global__ void batch_scale_vectors(BatchView b, double* c_s, double* lo_s, double* hi_s,
                                    double* rlo_s, double* rhi_s) {
    const int64_t t = blockIdx.x * static_cast<int64_t>(kBlock) + threadIdx.x;
    const DevProblem& P = b.P;
    if (t < b.n) {
        const double sc = P.cs[t];
        c_s[t] = (P.c_o[t] * sc) * b.is[b.col_inst[t]].obj_sign;
        lo_s[t] = fb(P.lo_o[t]) ? P.lo_o[t] / sc : P.lo_o[t];
        hi_s[t] = fb(P.hi_o[t]) ? P.hi_o[t] / sc : P.hi_o[t];
    }
    if (t < b.m) {
        const double sc = P.rs[t];
        rlo_s[t] = fb(P.rlo_o[t]) ? P.rlo_o[t] * sc : P.rlo_o[t];
        rhi_s[t] = fb(P.rhi_o[t]) ? P.rhi_o[t] * sc : P.rhi_o[t];
    }
}

// Relative-KKT norms (original) and the initial primal weight norms (scaled).
__global__ void __launch_bounds__(kBlock) batch_norms(BatchView b) {
    const int k = blockIdx.x;
    InstState& s = b.is[k];
    const DevProblem& P = b.P;
    double c2 = 0.0, b2 = 0.0, cm = 0.0, bm = 0.0, c2o = 0.0, b2o = 0.0;
    for (int j = b.col_off[k] + threadIdx.x; j < b.col_off[k + 1]; j += kBlock) {
        c2 += P.c[j] * P.c[j];
        cm = fmax(cm, fabs(P.c_o[j]));
        c2o += P.c_o[j] * P.c_o[j];
    }
    for (int i = b.row_off[k] + threadIdx.x; i < b.row_off[k + 1]; i += kBlock) {
        double bb = 0.0;
        if (fb(P.rlo[i])) bb = fabs(P.rlo[i]);
        if (fb(P.rhi[i])) bb = smax(bb, fabs(P.rhi[i]));
        b2 += bb * bb;
        double bo = 0.0;
        if (fb(P.rlo_o[i])) bo = fabs(P.rlo_o[i]);
        if (fb(P.rhi_o[i])) bo = smax(bo, fabs(P.rhi_o[i]));
        bm = fmax(bm, bo);
        b2o += bo * bo;
    }
    const double c2t = block_sum_det(c2), b2t = block_sum_det(b2);
    const double c2ot = block_sum_det(c2o), b2ot = block_sum_det(b2o);
    const double cmt = bmax(cm), bmt = bmax(bm);
    if (threadIdx.x == 0) {
        s.cnorm2_s = sqrt(c2t);
        s.bnorm2_s = sqrt(b2t);
        s.cnorm = cmt;
        s.bnorm = bmt;
        s.cnorm2 = sqrt(c2ot);
        s.bnorm2 = sqrt(b2ot);
    }
}

// ---------------------------------------------------------------------------
// Final result per instance (pdhg.cpp:420-498, duals.cpp:81-113)
// ---------------------------------------------------------------------------

__device__ __forceinline__ double inf_box(double coeff, double lo, double hi) {
    if (coeff == 0.0) return 0.0;
    if (coeff > 0.0) return fb(lo) ? coeff * lo : -INFINITY;
    return fb(hi) ? coeff * hi : -INFINITY;
}

__global__ void batch_widen(BatchView b, Iterates<float> f, Iterates<double> d) {
    const int64_t t = blockIdx.x * static_cast<int64_t>(kBlock) + threadIdx.x;
    // Halpern: the FP64 phase starts at T(z) as a restart point and anchor
    if (t < b.n) {
        d.x[t] = d.halpern ? f.psx[t] : f.x[t];
        d.xbar[t] = d.halpern ? f.psx[t] : f.xbar[t];
        if (d.halpern) d.xa[t] = d.x[t];
    }
    if (t < b.m) {
        d.y[t] = d.halpern ? f.psy[t] : f.y[t];
        d.s[t] = f.s[t];
        if (d.halpern) {
            d.ya[t] = d.y[t];
            d.sa[t] = d.s[t];
        }
    }
}

template <class T>
__global__ void __launch_bounds__(kBlock) batch_final(BatchView b, Iterates<T> it, double bt,
                                                      double* xo, double* yo, double* rc,
                                                      int which) {
    const int k = blockIdx.x;
    InstState& s = b.is[k];
    if (which >= 0 && s.polished != which) return;  // uniform per CTA
    const DevProblem& P = b.P;
    // Halpern: after a check the sums' slots hold T(z), the reported point
    const bool cand_avg = it.halpern ? b.g->checks > 0 : (s.converged && s.avg_better);
    const double inv = it.halpern ? 1.0 : s.inv, sign = s.obj_sign;
    // best point in original units (unscale_to_original, pdhg.cpp:205-214)
    for (int j = b.col_off[k] + threadIdx.x; j < b.col_off[k + 1]; j += kBlock) {
        const double xs = cand_avg ? avg_x(it, j, inv) : static_cast<double>(it.x[j]);
        xo[j] = xs * P.cs[j];
    }
    for (int i = b.row_off[k] + threadIdx.x; i < b.row_off[k + 1]; i += kBlock) {
        const double ys = cand_avg ? avg_y(it, i, inv) : static_cast<double>(it.y[i]);
        yo[i] = (ys * sign) * P.rs[i];
    }
    __syncthreads();  // xo / yo of this instance are read below by other threads of this CTA
    double pinf = 0.0, dinf = 0.0, obj = 0.0, dual = 0.0, inf = 0.0;
    const int lane = threadIdx.x & 31;
    const int groups = kBlock / 32;
    for (int i = b.row_off[k] + static_cast<int>(threadIdx.x) / 32; i < b.row_off[k + 1]; i += groups) {
        const double act = row_dot64(b.Ao, i, lane, 32, [xo](int j) { return xo[j]; });
        if (lane == 0) {
            const double lo = P.rlo_o[i], hi = P.rhi_o[i];
            pinf = smax(pinf, primal_term(act, lo, hi));
            const bool at_lo = fb(lo) && fabs(act - lo) <= bt;
            const bool at_hi = fb(hi) && fabs(act - hi) <= bt;
            if (!at_lo && !at_hi) dinf = smax(dinf, fabs(yo[i]));
            const double tr = inf_box(yo[i], lo, hi);
            if (isfinite(tr)) dual += tr; else inf = 1.0;
        }
    }
    for (int j = b.col_off[k] + static_cast<int>(threadIdx.x) / 32; j < b.col_off[k + 1]; j += groups) {
        const double aty = row_dot64(b.ATo, j, lane, 32, [yo](int i) { return yo[i]; });
        if (lane == 0) {
            const double r = P.c_o[j] - aty;
            rc[j] = r;
            const double lo = P.lo_o[j], hi = P.hi_o[j];
            const bool at_lo = fb(lo) && fabs(xo[j] - lo) <= bt;
            const bool at_hi = fb(hi) && fabs(xo[j] - hi) <= bt;
            if (!at_lo && !at_hi) dinf = smax(dinf, fabs(r));
            obj += P.c_o[j] * xo[j];
            const double tc = inf_box(r, lo, hi);
            if (isfinite(tc)) dual += tc; else inf = 1.0;
        }
    }
    const double pi = bmax(pinf), di = bmax(dinf);
    const double ob = block_sum_det(obj), du = block_sum_det(dual), nf = block_sum_det(inf);
    if (threadIdx.x == 0) {
        const double acc = s.obj_const + ob;
        s.objective = acc;
        s.dual_objective = du;
        s.gap = nf == 0.0 ? fabs(acc - du) / (1.0 + fabs(acc) + fabs(du)) : INFINITY;
        s.pinf = pi;
        s.dinf = di;
    }
}

// Relative KKT residual of a given point (x, y in original units and sense; a
// null pointer is the zero vector), per instance, the PDLP way with l2 norms:
// primal: ||bound violation of A clamp(x)||; dual: sign violations of the row
// duals and of the reduced costs against the column bounds (a boxed column
// admits any reduced cost); gap: |primal - dual objective| / (1 + |p| + |d|),
// infinite bounds dropped from the dual objective (their violations are in the
// dual term). Internal minimize sense: y and c times the objective sign.
__global__ void __launch_bounds__(kBlock) batch_point_kkt(BatchView b, const double* x,
                                                          const double* y, double* out) {
    const int k = blockIdx.x;
    const InstState& s = b.is[k];
    const DevProblem& P = b.P;
    const double sign = s.obj_sign;
    const int lane = threadIdx.x & 31;
    const int groups = kBlock / 32;
    double rp2 = 0.0, rd2 = 0.0, pobj = 0.0, dobj = 0.0, bn2 = 0.0, cn2 = 0.0;
    auto xc = [&](int j) {
        const double v = x != nullptr ? x[j] : 0.0;
        return clampT<double>(v, P.lo_o[j], P.hi_o[j]);
    };
    for (int i = b.row_off[k] + static_cast<int>(threadIdx.x) / 32; i < b.row_off[k + 1];
         i += groups) {
        const double act = row_dot64(b.Ao, i, lane, 32, xc);
        if (lane != 0) continue;
        const double lo = P.rlo_o[i], hi = P.rhi_o[i];
        double v = 0.0;
        if (fb(lo) && act < lo) v = lo - act;
        if (fb(hi) && act > hi) v = act - hi;
        rp2 += v * v;
        const double bb = smax(fb(lo) ? fabs(lo) : 0.0, fb(hi) ? fabs(hi) : 0.0);
        bn2 += bb * bb;
        const double yi = y != nullptr ? sign * y[i] : 0.0;
        double dv = 0.0;
        if (!fb(lo) && yi > 0.0) dv = yi;   // only an upper bound: y <= 0
        if (!fb(hi) && yi < 0.0) dv = -yi;  // only a lower bound: y >= 0
        rd2 += dv * dv;
        if (yi > 0.0 && fb(lo)) dobj += yi * lo;
        else if (yi < 0.0 && fb(hi)) dobj += yi * hi;
    }
    for (int j = b.col_off[k] + static_cast<int>(threadIdx.x) / 32; j < b.col_off[k + 1];
         j += groups) {
        const double aty = row_dot64(b.ATo, j, lane, 32, [y, sign](int i) {
            return y != nullptr ? sign * y[i] : 0.0;
        });
        if (lane != 0) continue;
        const double cj = sign * P.c_o[j];
        const double rc = cj - aty;
        const double lo = P.lo_o[j], hi = P.hi_o[j];
        pobj += cj * xc(j);
        cn2 += cj * cj;
        double dv = 0.0;
        if (fb(lo) && !fb(hi) && rc < 0.0) dv = -rc;
        else if (!fb(lo) && fb(hi) && rc > 0.0) dv = rc;
        else if (!fb(lo) && !fb(hi)) dv = fabs(rc);
        rd2 += dv * dv;
        if (rc > 0.0 && fb(lo)) dobj += rc * lo;
        else if (rc < 0.0 && fb(hi)) dobj += rc * hi;
    }
    const double a = block_sum_det(rp2), d2 = block_sum_det(rd2), p = block_sum_det(pobj);
    const double dd = block_sum_det(dobj), bn = block_sum_det(bn2), cn = block_sum_det(cn2);
    if (threadIdx.x == 0) {
        const double gap = fabs(p - dd) / (1.0 + fabs(p) + fabs(dd));
        out[k] = smax(smax(sqrt(a) / (1.0 + sqrt(bn)), sqrt(d2) / (1.0 + sqrt(cn))), gap);
    }
}

}  // namespace

void launch_batch_point_kkt(const BatchView& b, const double* x, const double* y, double* out,
                            cudaStream_t s) {
    if (b.count > 0) batch_point_kkt<<<b.count, kBlock, 0, s>>>(b, x, y, out);
}

// ---------------------------------------------------------------------------
// Launchers
// ---------------------------------------------------------------------------

template <class T>
void launch_batch_iter(const BatchView& b, const Iterates<T>& it, bool primal, int first,
                       int hk, cudaStream_t s) {
    const DevCsr& M = primal ? b.AT : b.A;
    if (M.rows == 0) return;
    const int sb = short_blocks(M);
    const int grid = sb + M.n_long;
#define PDHG_BATCH_ITER(VW)                                                                      \
    do {                                                                                         \
        if (M.n_long > 0) {                                                                      \
            if (primal) batch_iter<T, VW, true, true><<<grid, kBlock, 0, s>>>(b, it, first, hk, sb); \
            else batch_iter<T, VW, false, true><<<grid, kBlock, 0, s>>>(b, it, first, hk, sb);      \
        } else {                                                                                 \
            if (primal) batch_iter<T, VW, true, false><<<grid, kBlock, 0, s>>>(b, it, first, hk, sb);\
            else batch_iter<T, VW, false, false><<<grid, kBlock, 0, s>>>(b, it, first, hk, sb);     \
        }                                                                                        \
    } while (0)
    switch (M.vw) {
        case 1: PDHG_BATCH_ITER(1); break;
        case 2: PDHG_BATCH_ITER(2); break;
        case 4: PDHG_BATCH_ITER(4); break;
        case 8: PDHG_BATCH_ITER(8); break;
        case 16: PDHG_BATCH_ITER(16); break;
        default: PDHG_BATCH_ITER(32); break;
    }
#undef PDHG_BATCH_ITER
}

void launch_batch_compact(const BatchView& b, cudaStream_t s) {
    batch_compact<<<1, kCompactThreads, 0, s>>>(b, short_blocks(b.A), short_blocks(b.AT));
}

template <class T>
void launch_batch_check(const BatchView& b, const Iterates<T>& it, const BatchParams& p,
                        cudaStream_t s) {
    if (b.n_chk > 0) batch_check<T><<<b.n_chk, kBlock, 0, s>>>(b, it, p);
}

template <class T>
void launch_batch_restart(const BatchView& b, const Iterates<T>& it, const BatchParams& p,
                          cudaStream_t s) {
    if (b.count > 0) batch_restart<T><<<b.count, kBlock, 0, s>>>(b, it, p);
}

void launch_batch_tick(const BatchView& b, long long period, long long budget_iters,
                       cudaGraphConditionalHandle handle, int use_handle, cudaStream_t s) {
    batch_tick<<<1, 32, 0, s>>>(b, period, budget_iters, handle, use_handle);
}

void launch_batch_fill_inst(const int32_t* off, int32_t count, int32_t* out, cudaStream_t s) {
    if (count > 0) batch_fill_inst<<<count, kBlock, 0, s>>>(off, out);
}

void launch_batch_warm(const BatchView& b, double* x0, double* y0, cudaStream_t s) {
    const int32_t nmax = b.m > b.n ? b.m : b.n;
    if (nmax > 0) batch_warm<<<nblk(nmax), kBlock, 0, s>>>(b, x0, y0);
}

void launch_batch_pw_w(const BatchView& b, const double* u, const double* v, double* w,
                       cudaStream_t s) {
    if (b.m > 0) batch_pw_w<<<nblk(static_cast<int64_t>(b.m) * 32), kBlock, 0, s>>>(b, u, v, w);
}
void launch_batch_pw_norm_w(const BatchView& b, double* w, cudaStream_t s) {
    if (b.count > 0) batch_pw_norm_w<<<b.count, kBlock, 0, s>>>(b, w);
}
void launch_batch_pw_u(const BatchView& b, const double* w, double* u, cudaStream_t s) {
    if (b.n > 0) batch_pw_u<<<nblk(static_cast<int64_t>(b.n) * 32), kBlock, 0, s>>>(b, w, u);
}
void launch_batch_pw_norm_uv(const BatchView& b, const double* w, double* u, double* v,
                             cudaStream_t s) {
    if (b.count > 0) batch_pw_norm_uv<<<b.count, kBlock, 0, s>>>(b, w, u, v);
}
void launch_batch_steps(const BatchView& b, double safety, int primal_weight, cudaStream_t s) {
    if (b.count > 0) batch_steps<<<nblk(b.count), kBlock, 0, s>>>(b, safety, primal_weight);
}

void launch_batch_ruiz_max(const BatchView& b, const DevCsr& M, int transposed, const double* rs,
                           const double* cs, double* out, cudaStream_t s) {
    if (M.rows > 0)
        batch_ruiz_max<<<nblk(static_cast<int64_t>(M.rows) * 32), kBlock, 0, s>>>(
            b, M, transposed, transposed ? b.col_inst : b.row_inst, rs, cs, out);
}
void launch_batch_ruiz_update(const BatchView& b, double* rs, double* cs, const double* row_max,
                              const double* col_max, double tol, cudaStream_t s) {
    if (b.count > 0) batch_ruiz_update<<<b.count, kBlock, 0, s>>>(b, rs, cs, row_max, col_max, tol);
}
void launch_batch_scale_vectors(const BatchView& b, double* c_s, double* lo_s, double* hi_s,
                                double* rlo_s, double* rhi_s, cudaStream_t s) {
    const int32_t nmax = b.m > b.n ? b.m : b.n;
    if (nmax > 0) batch_scale_vectors<<<nblk(nmax), kBlock, 0, s>>>(b, c_s, lo_s, hi_s, rlo_s, rhi_s);
}
void launch_batch_norms(const BatchView& b, cudaStream_t s) {
    if (b.count > 0) batch_norms<<<b.count, kBlock, 0, s>>>(b);
}

void launch_batch_widen(const BatchView& b, const Iterates<float>& f, const Iterates<double>& d,
                        cudaStream_t s) {
    const int32_t nmax = b.m > b.n ? b.m : b.n;
    if (nmax > 0) batch_widen<<<nblk(nmax), kBlock, 0, s>>>(b, f, d);
}

template <class T>
void launch_batch_final(const BatchView& b, const Iterates<T>& it, double bound_tol, double* xo,
                        double* yo, double* rc, int which, cudaStream_t s) {
    if (b.count > 0) batch_final<T><<<b.count, kBlock, 0, s>>>(b, it, bound_tol, xo, yo, rc, which);
}

template void launch_batch_iter<float>(const BatchView&, const Iterates<float>&, bool, int, int, cudaStream_t);
template void launch_batch_iter<double>(const BatchView&, const Iterates<double>&, bool, int, int, cudaStream_t);
template void launch_batch_check<float>(const BatchView&, const Iterates<float>&, const BatchParams&, cudaStream_t);
template void launch_batch_check<double>(const BatchView&, const Iterates<double>&, const BatchParams&, cudaStream_t);
template void launch_batch_restart<float>(const BatchView&, const Iterates<float>&, const BatchParams&, cudaStream_t);
template void launch_batch_restart<double>(const BatchView&, const Iterates<double>&, const BatchParams&, cudaStream_t);
template void launch_batch_final<float>(const BatchView&, const Iterates<float>&, double, double*, double*, double*, int, cudaStream_t);
template void launch_batch_final<double>(const BatchView&, const Iterates<double>&, double, double*, double*, double*, int, cudaStream_t);

}  // namespace pdhg
