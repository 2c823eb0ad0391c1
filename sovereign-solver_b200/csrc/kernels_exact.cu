// kernels_exact.cu -- the FP64 kernels that reproduce the reference bit for bit.
//
// The reference's Host backend (src/l0/backend_host.cpp) and CsrMatrix
// (src/l0/sparse.cpp:130-154) add every sum sequentially, in row (or column)
// order, with a separate rounding for each product and each addition (its
// Release build targets generic x86-64: no FMA). These kernels give each row
// of A (or of A^T) to one thread -- or, for rows longer than kWarpRow, to one
// warp whose lanes evaluate the products together and then add them in row
// order -- with __dmul_rn / __dadd_rn, so nothing is contracted and nothing
// reordered.
// Max-reductions are exact in any order and use atomicMax on the bit patterns
// of non-negative doubles. Decisions (restart, termination) are taken by the
// last CTA of each check kernel, on the device.
//
// Also here: setup (exact pairwise norm for the power iteration), the final
// result kernels, the backend primitives and the device CSR transpose.
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include <cmath>
#include <cstdio>

#include "engine.cuh"
#include "ordered.cuh"

namespace pdhg {

namespace {

constexpr int kStatusOptimal = 0;
constexpr int kStatusNumericalFailure = 3;

__device__ __forceinline__ double smax(double a, double b) { return (a < b) ? b : a; }
__device__ __forceinline__ bool fb(double v) { return v > -INFINITY && v < INFINITY; }
__device__ __forceinline__ double clampd(double v, double lo, double hi) {
    // HostBackend::project_box, backend_host.cpp:453-456
    if (v < lo) v = lo;
    if (v > hi) v = hi;
    return v;
}

// Warp max then one atomicMax per warp. Every thread of the block must call it.
__device__ __forceinline__ void block_acc_max(unsigned long long* slot, double v) {
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    if ((threadIdx.x & 31) == 0 && v > 0.0)
        atomicMax(slot, static_cast<unsigned long long>(__double_as_longlong(v)));
}

__device__ __forceinline__ double acc_read(unsigned long long* slot) {
    return __longlong_as_double(static_cast<long long>(*reinterpret_cast<volatile unsigned long long*>(slot)));
}

__device__ __forceinline__ bool last_block(unsigned int* ticket) {
    __shared__ bool am_last;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) am_last = (atomicAdd(ticket, 1u) == gridDim.x - 1);
    __syncthreads();
    return am_last;
}

// Deterministic block sum (fixed tree over the block's threads).
__device__ double block_sum(double v) {
    __shared__ double sh[kBlock];
    sh[threadIdx.x] = v;
    __syncthreads();
    for (int s = kBlock / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) sh[threadIdx.x] = sh[threadIdx.x] + sh[threadIdx.x + s];
        __syncthreads();
    }
    const double r = sh[0];
    __syncthreads();
    return r;
}

__device__ void publish(DevState* st, Mailbox* mail) {
    if (mail == nullptr) return;
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

__host__ __device__ inline int blocks_for(int64_t n) {
    return static_cast<int>((n + kBlock - 1) / kBlock);
}


// ---------------------------------------------------------------------------
// One PDHG iteration (src/l1/pdhg.cpp:295-331)
// ---------------------------------------------------------------------------

// K1: per column j -- grad = c - A^T y (pdhg.cpp:296-297: grad starts at c,
// then every row adds val * (-y_r) in row order), x_new = proj(x - tau grad),
// x_bar = 2 x_new - x, Cesaro sum.
__global__ void __launch_bounds__(kBlock) ex_primal(ExactIter a, int first) {
    DevState* st = a.st;
    if (first && blockIdx.x == 0 && threadIdx.x == 0) st->restart = 0;  // consumed by ex_restart
    if (st->done) return;
    const RowTask t = row_task(a.AT, blockIdx.x);
    if (t.row < 0) return;
    const int j = t.row;
    const double* y = a.it.y;
    const double g = row_dot(t, a.AT, [y](int i) { return -y[i]; }, a.P.c[j]);
    if (!t.lead) return;
    const double xo = a.it.x[j];
    const double xn = clampd(__dadd_rn(xo, __dmul_rn(-st->tau, g)), a.P.lo[j], a.P.hi[j]);
    a.it.xbar[j] = __dadd_rn(2.0 * xn, -xo);  // scale(2.0) then axpy(-1.0, x)
    a.it.x[j] = xn;
    const bool fresh = first && st->fresh;
    a.it.xsum[j] = fresh ? xn : __dadd_rn(a.it.xsum[j], xn);
}

// K2: per row i -- s_new = proj(s - tau y), s_bar = 2 s_new - s,
// k = -(A x_bar) + s_bar, y += sigma k (pdhg.cpp:302-318), Cesaro sum.
__global__ void __launch_bounds__(kBlock) ex_dual(ExactIter a, int first) {
    DevState* st = a.st;
    if (st->done) return;
    const RowTask t = row_task(a.A, blockIdx.x);
    if (t.row < 0) return;
    const int i = t.row;
    const double* xbar = a.it.xbar;
    const double sum = row_dot(t, a.A, [xbar](int j) { return xbar[j]; }, 0.0);
    if (!t.lead) return;
    const double yo = a.it.y[i];
    const double so = a.it.s[i];
    const double sn = clampd(__dadd_rn(so, __dmul_rn(-st->tau, yo)), a.P.rlo[i], a.P.rhi[i]);
    const double sbar = __dadd_rn(2.0 * sn, -so);
    const double kb = __dadd_rn(-sum, sbar);
    const double yn = __dadd_rn(yo, __dmul_rn(st->sigma, kb));
    a.it.y[i] = yn;
    a.it.s[i] = sn;
    const bool fresh = first && st->fresh;
    a.it.ysum[i] = fresh ? yn : __dadd_rn(a.it.ysum[i], yn);
}

// ---------------------------------------------------------------------------
// Check period (pdhg.cpp:333-408)
// ---------------------------------------------------------------------------

// Row-dual / reduced-cost classification shared by kkt_residual
// (pdhg.cpp:113-119, 128-133) and original_space_residual (pdhg.cpp:174-180,
// 192-196): strict `<` at-bound test.
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

// Check 1: kkt_residual (pdhg.cpp:87-136) of the current point and of the
// Cesaro average (pdhg.cpp:336-345), scaled space, bound_tol = tolerance.
// Blocks [0, row_blocks) take rows of A, the rest take rows of A^T.
__global__ void __launch_bounds__(kBlock) ex_check1(ExactCheck a) {
    DevState* st = a.st;
    if (st->done) return;
    const long long k_avg = st->since_restart + a.period_iters;
    const double inv = 1.0 / static_cast<double>(k_avg);
    const int row_blocks = mat_blocks(a.A);
    const double bt = a.tol;
    double cp = 0.0, cd = 0.0, ap = 0.0, ad = 0.0;
    if (static_cast<int>(blockIdx.x) < row_blocks) {
        const RowTask t = row_task(a.A, blockIdx.x);
        if (t.row >= 0) {
            const int i = t.row;
            const double* x = a.it.x;
            const double* xs = a.it.xsum;
            const double act_c = row_dot(t, a.A, [x](int j) { return x[j]; }, 0.0);
            const double act_a = row_dot(t, a.A, [xs, inv](int j) { return __dmul_rn(xs[j], inv); }, 0.0);
            if (t.lead) {
                a.cs.act_avg[i] = act_a;
                const double lo = a.P.rlo[i], hi = a.P.rhi[i];
                cp = primal_term(act_c, lo, hi);
                ap = primal_term(act_a, lo, hi);
                cd = cs_term(a.it.y[i], act_c, lo, hi, bt);
                ad = cs_term(__dmul_rn(a.it.ysum[i], inv), act_a, lo, hi, bt);
            }
        }
    } else {
        const RowTask t = row_task(a.AT, blockIdx.x - row_blocks);
        if (t.row >= 0) {
            const int j = t.row;
            const double* y = a.it.y;
            const double* ys = a.it.ysum;
            const double aty_c = row_dot(t, a.AT, [y](int i) { return y[i]; }, 0.0);
            const double aty_a = row_dot(t, a.AT, [ys, inv](int i) { return __dmul_rn(ys[i], inv); }, 0.0);
            if (t.lead) {
                const double cj = a.P.c[j];
                const double lo = a.P.lo[j], hi = a.P.hi[j];
                cd = cs_term(__dadd_rn(cj, -aty_c), a.it.x[j], lo, hi, bt);
                ad = cs_term(__dadd_rn(cj, -aty_a), __dmul_rn(a.it.xsum[j], inv), lo, hi, bt);
            }
        }
    }
    block_acc_max(&st->acc[ACC_CUR_P], cp);
    block_acc_max(&st->acc[ACC_CUR_D], cd);
    block_acc_max(&st->acc[ACC_AVG_P], ap);
    block_acc_max(&st->acc[ACC_AVG_D], ad);
    if (last_block(&st->ticket[TK_CHECK1]) && threadIdx.x == 0) {
        const double cur = smax(acc_read(&st->acc[ACC_CUR_P]), acc_read(&st->acc[ACC_CUR_D]));
        const double avg = smax(acc_read(&st->acc[ACC_AVG_P]), acc_read(&st->acc[ACC_AVG_D]));
        st->acc[ACC_CUR_P] = st->acc[ACC_CUR_D] = st->acc[ACC_AVG_P] = st->acc[ACC_AVG_D] = 0ull;
        st->ticket[TK_CHECK1] = 0u;
        st->cur_res = cur;
        st->avg_res = avg;
        st->inv = inv;
        if (!isfinite(cur) || !isfinite(avg)) {  // pdhg.cpp:347-352
            st->done = 1;
            st->status = kStatusNumericalFailure;
            st->fail_kind = 1;
            st->stop_iter = st->iter + a.period_iters - 1;
            st->restart = 0;
            publish(st, a.mail);
        }
        st->avg_better = avg <= cur;  // pdhg.cpp:354
        __threadfence();
    }
}

// Check 2: original_space_residual (pdhg.cpp:145-199) of the candidate with
// bound_tol = max(tol, 1e-6) on the ORIGINAL matrix, then termination
// (pdhg.cpp:383-389) and the restart rule (pdhg.cpp:391-408).
__global__ void __launch_bounds__(kBlock) ex_check2(ExactCheck a) {
    DevState* st = a.st;
    if (st->done) return;
    const double inv = st->inv;
    const bool ab = st->avg_better != 0;
    const double sign = a.P.obj_sign;
    const int row_blocks = mat_blocks(a.Ao);
    const double bt = a.bound_tol;
    double op = 0.0, od = 0.0, pobj = 0.0, dobj = 0.0;
    if (static_cast<int>(blockIdx.x) < row_blocks) {
        const RowTask t = row_task(a.Ao, blockIdx.x);
        if (t.row >= 0) {
            const int i = t.row;
            const double* xv = a.it.x;
            const double* xsum = a.it.xsum;
            const double* cs = a.P.cs;
            const double act = row_dot(
                t, a.Ao,
                [=](int j) { return __dmul_rn(ab ? __dmul_rn(xsum[j], inv) : xv[j], cs[j]); }, 0.0);
          if (t.lead) {
            const double ys = ab ? __dmul_rn(a.it.ysum[i], inv) : a.it.y[i];
            const double yo = __dmul_rn(__dmul_rn(ys, sign), a.P.rs[i]);
            if (a.want_candidate) a.cs.cand_yo[i] = yo;
            const double lo = a.P.rlo_o[i], hi = a.P.rhi_o[i];
            op = primal_term(act, lo, hi);
            od = cs_term(__dmul_rn(sign, yo), act, lo, hi, bt);
            if (a.termination_rule == 1) {  // gap terms in the internal (minimize) sense
                const double yi = sign * yo;
                if (yi > 0.0) dobj = fb(lo) ? yi * lo : 0.0;
                else if (yi < 0.0) dobj = fb(hi) ? yi * hi : 0.0;
            }
          }
        }
    } else {
        const RowTask t = row_task(a.ATo, blockIdx.x - row_blocks);
        if (t.row >= 0) {
            const int j = t.row;
            const double* yv = a.it.y;
            const double* ysum = a.it.ysum;
            const double* rsv = a.P.rs;
            const double aty = row_dot(
                t, a.ATo,
                [=](int i) {
                    const double ys = ab ? __dmul_rn(ysum[i], inv) : yv[i];
                    return __dmul_rn(__dmul_rn(ys, sign), rsv[i]);
                },
                0.0);
          if (t.lead) {
            const double xs = ab ? __dmul_rn(a.it.xsum[j], inv) : a.it.x[j];
            const double xo = __dmul_rn(xs, a.P.cs[j]);
            if (a.want_candidate) a.cs.cand_xo[j] = xo;
            const double r = __dadd_rn(a.P.c_o[j], -aty);
            const double lo = a.P.lo_o[j], hi = a.P.hi_o[j];
            od = cs_term(__dmul_rn(sign, r), xo, lo, hi, bt);
            if (a.termination_rule == 1) {
                pobj = sign * a.P.c_o[j] * xo;
                const double ri = sign * r;
                if (ri > 0.0) dobj = fb(lo) ? ri * lo : 0.0;
                else if (ri < 0.0) dobj = fb(hi) ? ri * hi : 0.0;
            }
          }
        }
    }
    block_acc_max(&st->acc[ACC_ORIG_P], op);
    block_acc_max(&st->acc[ACC_ORIG_D], od);
    if (a.termination_rule == 1) {
        const double bp = block_sum(pobj);
        const double bd = block_sum(dobj);
        if (threadIdx.x == 0) {
            a.cs.part[2 * blockIdx.x] = bp;
            a.cs.part[2 * blockIdx.x + 1] = bd;
        }
    }
    if (last_block(&st->ticket[TK_CHECK2]) && threadIdx.x == 0) {
        const double opv = acc_read(&st->acc[ACC_ORIG_P]);
        const double odv = acc_read(&st->acc[ACC_ORIG_D]);
        const double orig = smax(opv, odv);
        st->acc[ACC_ORIG_P] = st->acc[ACC_ORIG_D] = 0ull;
        st->ticket[TK_CHECK2] = 0u;
        st->orig_res = orig;
        const long long it_idx = st->iter + a.period_iters - 1;
        st->checks += 1;
        if (!isfinite(orig)) {  // pdhg.cpp:366-371
            st->done = 1;
            st->status = kStatusNumericalFailure;
            st->fail_kind = 2;
            st->stop_iter = it_idx;
            st->restart = 0;
        } else {
            double rel = 0.0;
            if (a.termination_rule == 1) {
                double ps = 0.0, ds = 0.0;
                const volatile double* part = a.cs.part;
                for (unsigned b = 0; b < gridDim.x; ++b) {
                    ps += part[2 * b];
                    ds += part[2 * b + 1];
                }
                ps += sign * a.P.obj_const;  // the constant shifts both objectives
                ds += sign * a.P.obj_const;
                const double gap = fabs(ps - ds) / (1.0 + fabs(ps) + fabs(ds));
                rel = smax(smax(opv / (1.0 + a.P.bnorm), odv / (1.0 + a.P.cnorm)), gap);
            }
            st->rel_kkt = rel;
            const bool conv = (a.termination_rule == 1) ? (rel < a.tol) : (orig < a.tol);
            if (conv) {
                st->done = 1;
                st->converged = 1;
                st->status = kStatusOptimal;
                st->stop_iter = it_idx + 1;
                st->restart = 0;
            } else {
                if (!isfinite(st->res_last)) st->res_last = st->cur_res;  // pdhg.cpp:391
                if (st->avg_res <= a.restart_decrease * st->res_last) {
                    st->restart = 1;
                    st->res_last = st->avg_res;
                    st->since_restart = 0;
                    st->restarts += 1;
                } else {
                    st->restart = 0;
                    st->since_restart += a.period_iters;
                }
                st->fresh = st->restart;
                const int stop = a.mail != nullptr ? a.mail->stop_request : 0;
                if (stop != 0) {
                    st->done = 1;
                    st->status = stop;
                    st->stop_iter = it_idx + 1;
                }
            }
        }
        st->iter += a.period_iters;
        publish(st, a.mail);
    }
}

// Restart to the average (pdhg.cpp:393-404): x = proj(x_avg), y = y_avg,
// s = proj(A x_avg) with the UNprojected average.
__global__ void __launch_bounds__(kBlock) ex_restart(ExactCheck a) {
    const DevState* st = a.st;
    if (!st->restart) return;
    const double inv = st->inv;
    const int t = blockIdx.x * kBlock + threadIdx.x;
    if (t < a.AT.rows)
        a.it.x[t] = clampd(__dmul_rn(a.it.xsum[t], inv), a.P.lo[t], a.P.hi[t]);
    if (t < a.A.rows) {
        a.it.y[t] = __dmul_rn(a.it.ysum[t], inv);
        a.it.s[t] = clampd(a.cs.act_avg[t], a.P.rlo[t], a.P.rhi[t]);
    }
}

// ---------------------------------------------------------------------------
// Setup: power iteration pieces and the exact pairwise norm
// ---------------------------------------------------------------------------

// w = -(A u) + v  (spmv(A, -1, u, 0, w) then axpy(1, v, w), pdhg.cpp:59-60).
// uscale (null: 1): u is read as u * uscale, the previous iteration's scaling
// of u by 1 / estimate (pdhg.cpp:75) applied where u is gathered -- the same
// rounded value as the scaled vector, without a pass over u.
// FAST (the mixed and FP64 modes, whose estimate need not be the
// reference's bit for bit): a warp row's products are added by its lanes in
// parallel (four strided partial sums per lane, then a shuffle tree) instead
// of in the row's order, which takes a long row from a chain of dependent
// additions to a streaming pass.
template <bool FAST>
__global__ void __launch_bounds__(kBlock) k_pw_w(DevCsr A, const double* u, const double* v,
                                                 double* w, const int* stop, const double* uscale) {
    if (stop != nullptr && *stop) return;
    const RowTask t = row_task(A, blockIdx.x);
    if (t.row < 0) return;
    const double us = uscale != nullptr ? *uscale : 1.0;
    const auto g = [u, us](int j) { return __dmul_rn(u[j], us); };
    double sum;
    if (FAST && t.warp) {
        const int lane = threadIdx.x & 31;
        const int b = A.rp[t.row], e = A.rp[t.row + 1];
        double p0 = 0.0, p1 = 0.0, p2 = 0.0, p3 = 0.0;
        int k = b + lane;
        for (; k + 96 < e; k += 128) {
            p0 += A.v64[k] * g(A.ci[k]);
            p1 += A.v64[k + 32] * g(A.ci[k + 32]);
            p2 += A.v64[k + 64] * g(A.ci[k + 64]);
            p3 += A.v64[k + 96] * g(A.ci[k + 96]);
        }
        for (; k < e; k += 32) p0 += A.v64[k] * g(A.ci[k]);
        sum = (p0 + p1) + (p2 + p3);
        for (int o = 16; o > 0; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
    } else if (t.warp) {
        sum = ordered_dot_warp_pipelined(A.rp[t.row], A.rp[t.row + 1], A.ci, A.v64, g, 0.0,
                                         warp_stage2());
    } else {
        sum = row_dot(t, A, g, 0.0);
    }
    if (t.lead) w[t.row] = __dadd_rn(-sum, v[t.row]);
}

// u = A^T (-w) via spmv_transpose(A, -1, w, 0, u) (pdhg.cpp:67): u starts at
// 0 and adds val * (-w_r) in row order.
__global__ void __launch_bounds__(kBlock) k_pw_u(DevCsr AT, const double* w, double* u,
                                                 const int* stop) {
    if (stop != nullptr && *stop) return;
    const RowTask t = row_task(AT, blockIdx.x);
    if (t.row < 0) return;
    const double sum = row_dot(t, AT, [w](int i) { return -w[i]; }, 0.0);
    if (t.lead) u[t.row] = sum;
}

// The power iteration's scalar steps on the device (pdhg.cpp:58-75, the
// host's arithmetic: IEEE square roots and divisions, no contraction), so the
// loop runs without a host round trip. st[0] = 1 / ||w||, st[1] = the
// estimate, st[2] = 1 / estimate; *stop = 1 where the host loop breaks
// (||w|| or the estimate below 1e-300), after which every step is a no-op.
__global__ void k_pw_norm_w(const double* dot, double* st, int* stop) {
    if (*stop) return;
    const double wn = sqrt(dot[0]);
    if (wn < 1e-300) {
        *stop = 1;
        return;
    }
    st[0] = 1.0 / wn;
}
__global__ void k_pw_norm_e(const double* dots, double* st, int* stop) {
    if (*stop) return;
    const double un = sqrt(dots[0]), vn = sqrt(dots[1]);
    const double est = sqrt(__dadd_rn(__dmul_rn(un, un), __dmul_rn(vn, vn)));
    st[1] = est;
    if (est < 1e-300) {
        *stop = 1;
        return;
    }
    st[2] = 1.0 / est;
}
__global__ void k_scale_by(double* x, int64_t n, const double* alpha, const int* stop) {
    if (*stop) return;
    const double a = *alpha;
    const int64_t t = blockIdx.x * static_cast<int64_t>(kBlock) + threadIdx.x;
    if (t < n) x[t] = __dmul_rn(x[t], a);
}
__global__ void k_copy_unless(double* dst, const double* src, int64_t n, const int* stop) {
    if (*stop) return;
    const int64_t t = blockIdx.x * static_cast<int64_t>(kBlock) + threadIdx.x;
    if (t < n) dst[t] = src[t];
}

__global__ void k_scale(double* x, int64_t n, double alpha) {
    const int64_t t = blockIdx.x * static_cast<int64_t>(kBlock) + threadIdx.x;
    if (t < n) x[t] = __dmul_rn(x[t], alpha);
}

__global__ void k_fill(double* x, int64_t n, double v) {
    const int64_t t = blockIdx.x * static_cast<int64_t>(kBlock) + threadIdx.x;
    if (t < n) x[t] = v;
}

// Pairwise dot (HostBackend::pairwise_dot, backend_host.cpp:480-490):
// P(x, n) = n <= 128 ? sequential sum : P(x, n/2) + P(x + n/2, n - n/2).
// At depth d every node has size floor or ceil of n / 2^d, so the nodes of
// depth D-1 (D = first depth whose sizes are all <= 128) are either leaves
// (size <= 128) or parents of two leaves, and every node above is internal.
// Kernel 1 evaluates depth D-1 (k_pw_level_staged); kernel 2 folds the levels
// pairwise, left + right, exactly like the recursion.
__host__ __device__ inline void pw_node(int64_t n, int depth, int64_t idx, int64_t* off,
                                        int64_t* size) {
    int64_t o = 0, s = n;
    for (int b = depth - 1; b >= 0; --b) {
        const int64_t h = s / 2;
        if ((idx >> b) & 1) {
            o += h;
            s -= h;
        } else {
            s = h;
        }
    }
    *off = o;
    *size = s;
}

// The nodes of depth D-1, 32 consecutive nodes per CTA: their entries form
// one contiguous range of at most 32 x 256 products, which all 256 threads
// load with coalesced reads into shared memory; then thread l adds the
// products of node l in index order (its left and right leaf sums, then
// their sum), the recursion's sequence of additions for that node, so the
// result is identical. (One thread per node reading its ~150 consecutive
// entries from global memory alone made every warp-wide load touch 32 lines;
// one warp per 32 nodes streaming the range in chunks left most lanes idle
// while the others added.)
constexpr int kPwNodes = 32;
constexpr int kPwMaxNode = 256;  // a depth D-1 node: at most two leaves of 128
__global__ void __launch_bounds__(kBlock) k_pw_level_staged(const double* x, const double* y,
                                                            int64_t n, int depth, double* out) {
    extern __shared__ double prod[];
    __shared__ int64_t off[kPwNodes + 1];
    const int64_t nodes = int64_t{1} << depth;
    const int64_t t0 = static_cast<int64_t>(blockIdx.x) * kPwNodes;
    const int cnt = nodes - t0 < kPwNodes ? static_cast<int>(nodes - t0) : kPwNodes;
    int64_t o = 0, sz = 0;
    if (threadIdx.x < cnt) {
        pw_node(n, depth, t0 + threadIdx.x, &o, &sz);
        off[threadIdx.x] = o;
        if (threadIdx.x == cnt - 1) off[cnt] = o + sz;
    }
    __syncthreads();
    const int64_t r0 = off[0], len = off[cnt] - r0;
#pragma unroll 4
    for (int64_t i = threadIdx.x; i < len; i += kBlock) prod[i] = __dmul_rn(x[r0 + i], y[r0 + i]);
    __syncthreads();
    if (threadIdx.x >= cnt) return;
    const double* p = prod + (o - r0);
    const int h = sz <= 128 ? static_cast<int>(sz) : static_cast<int>(sz / 2);
    double accl = 0.0, accr = 0.0;
#pragma unroll 8
    for (int i = 0; i < h; ++i) accl = __dadd_rn(accl, p[i]);
#pragma unroll 8
    for (int i = h; i < static_cast<int>(sz); ++i) accr = __dadd_rn(accr, p[i]);
    out[t0 + threadIdx.x] = sz <= 128 ? accl : __dadd_rn(accl, accr);
}

int pw_depth(int64_t n) {
    // smallest D with ceil(n / 2^D) <= 128; the kernel evaluates depth D-1
    // (or depth 0 when n itself is a leaf).
    if (n <= 128) return 0;
    int D = 0;
    while (true) {
        const int64_t mx = (n + (int64_t{1} << D) - 1) >> D;
        if (mx <= 128) break;
        ++D;
    }
    return D - 1;
}

// Uniform-barrier fold: one level per launch of a simple kernel (setup only).
__global__ void k_pw_fold_level(const double* in, double* out, int64_t half) {
    const int64_t t = blockIdx.x * static_cast<int64_t>(kBlock) + threadIdx.x;
    if (t < half) out[t] = __dadd_rn(in[2 * t], in[2 * t + 1]);
}

// Folds the remaining 2^levels (<= 1024) values in one CTA, level by level,
// pairs (2t, 2t+1) -> t exactly as k_pw_fold_level; every thread runs the same
// number of levels, so the barriers are uniform.
__global__ void __launch_bounds__(512) k_pw_fold_tail(double* a, double* b, int levels,
                                                      double* out) {
    for (int lvl = levels; lvl > 0; --lvl) {
        const int half = 1 << (lvl - 1);
        for (int t = threadIdx.x; t < half; t += blockDim.x) b[t] = __dadd_rn(a[2 * t], a[2 * t + 1]);
        __syncthreads();
        double* tmp = a;
        a = b;
        b = tmp;
    }
    if (threadIdx.x == 0) *out = a[0];
}

// ---------------------------------------------------------------------------
// Final result (pdhg.cpp:428-498)
// ---------------------------------------------------------------------------

__global__ void k_fin_unscale(FinalArgs a) {
    // unscale_to_original (pdhg.cpp:205-214): x *= col_scale; y = (y * sign) * row_scale
    const int t = blockIdx.x * kBlock + threadIdx.x;
    if (t < a.P.n) a.f.xo[t] = __dmul_rn(a.best_x64[t], a.P.cs[t]);
    if (t < a.P.m) a.f.yo[t] = __dmul_rn(__dmul_rn(a.best_y64[t], a.P.obj_sign), a.P.rs[t]);
}

__device__ __forceinline__ double inf_over_box(double coeff, double lo, double hi) {
    // pdhg.cpp:36-40
    if (coeff == 0.0) return 0.0;
    if (coeff > 0.0) return fb(lo) ? coeff * lo : -INFINITY;
    return fb(hi) ? coeff * hi : -INFINITY;
}

// primal infeasibility (pdhg.cpp:444-457), complementary slackness with `<=`
// (src/l1/duals.cpp:81-113), reduced costs (pdhg.cpp:434-442), dual-objective
// terms (pdhg.cpp:476-491). Exact order in both orientations.
__global__ void __launch_bounds__(kBlock) k_fin_rowscols(FinalArgs a) {
    DevState* st = a.st;
    const int row_blocks = mat_blocks(a.Ao);
    const double bt = a.bound_tol;
    double pinf = 0.0, dinf = 0.0;
    if (static_cast<int>(blockIdx.x) < row_blocks) {
        const RowTask t = row_task(a.Ao, blockIdx.x);
        if (t.row >= 0) {
            const int i = t.row;
            const double* xo = a.f.xo;
            const double act = row_dot(t, a.Ao, [xo](int j) { return xo[j]; }, 0.0);
          if (t.lead) {
            const double lo = a.P.rlo_o[i], hi = a.P.rhi_o[i];
            pinf = primal_term(act, lo, hi);
            const bool at_lo = fb(lo) && fabs(act - lo) <= bt;
            const bool at_hi = fb(hi) && fabs(act - hi) <= bt;
            if (!at_lo && !at_hi) dinf = fabs(a.f.yo[i]);
            a.f.trow[i] = inf_over_box(a.f.yo[i], lo, hi);
          }
        }
    } else {
        const RowTask t = row_task(a.ATo, blockIdx.x - row_blocks);
        if (t.row >= 0) {
            const int j = t.row;
            const double* yo = a.f.yo;
            const double aty = row_dot(t, a.ATo, [yo](int i) { return yo[i]; }, 0.0);
          if (t.lead) {
            const double rc = __dadd_rn(a.P.c_o[j], -aty);
            a.f.rc[j] = rc;
            const double lo = a.P.lo_o[j], hi = a.P.hi_o[j];
            const double xo = a.f.xo[j];
            const bool at_lo = fb(lo) && fabs(xo - lo) <= bt;
            const bool at_hi = fb(hi) && fabs(xo - hi) <= bt;
            if (!at_lo && !at_hi) dinf = fabs(rc);
            a.f.tcol[j] = inf_over_box(rc, lo, hi);
          }
        }
    }
    block_acc_max(&st->acc[ACC_FIN_PINF], pinf);
    block_acc_max(&st->acc[ACC_FIN_DINF], dinf);
}

// Sequential sums in the reference's order (objective: problem.cpp:13-19;
// dual objective: columns then rows, stopping at the first infinite term).
__global__ void k_fin_sums_exact(FinalArgs a) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    DevState* st = a.st;
    double acc = a.P.obj_const;
    for (int j = 0; j < a.P.n; ++j) acc = __dadd_rn(acc, __dmul_rn(a.P.c_o[j], a.f.xo[j]));
    double dual = 0.0;
    bool fin = true;
    for (int j = 0; j < a.P.n && fin; ++j) {
        const double t = a.f.tcol[j];
        if (!isfinite(t)) { fin = false; break; }
        dual = __dadd_rn(dual, t);
    }
    for (int i = 0; i < a.P.m && fin; ++i) {
        const double t = a.f.trow[i];
        if (!isfinite(t)) { fin = false; break; }
        dual = __dadd_rn(dual, t);
    }
    st->objective = acc;
    st->dual_objective = dual;
    st->gap_finite = fin ? 1 : 0;
    st->duality_gap = fin ? fabs(acc - dual) / (1.0 + fabs(acc) + fabs(dual)) : INFINITY;
    st->pinf = acc_read(&st->acc[ACC_FIN_PINF]);
    st->dinf = acc_read(&st->acc[ACC_FIN_DINF]);
    st->acc[ACC_FIN_PINF] = st->acc[ACC_FIN_DINF] = 0ull;
}

// Deterministic tree sums (fast modes): grid-stride over a capped grid, block
// partials in a.f.trow's tail-free scratch (st->acc is not used for sums), and
// the partials folded in block order by the last CTA.
__global__ void __launch_bounds__(kBlock) k_fin_sums_tree(FinalArgs a, double* part) {
    DevState* st = a.st;
    double po = 0.0, du = 0.0, inf = 0.0;
    const int64_t stride = static_cast<int64_t>(gridDim.x) * kBlock;
    for (int64_t j = blockIdx.x * static_cast<int64_t>(kBlock) + threadIdx.x; j < a.P.n; j += stride) {
        po += a.P.c_o[j] * a.f.xo[j];
        const double t = a.f.tcol[j];
        if (!isfinite(t)) inf = 1.0; else du += t;
    }
    for (int64_t i = blockIdx.x * static_cast<int64_t>(kBlock) + threadIdx.x; i < a.P.m; i += stride) {
        const double t = a.f.trow[i];
        if (!isfinite(t)) inf = 1.0; else du += t;
    }
    po = block_sum(po);
    du = block_sum(du);
    inf = block_sum(inf);
    if (threadIdx.x == 0) {
        part[3 * blockIdx.x] = po;
        part[3 * blockIdx.x + 1] = du;
        part[3 * blockIdx.x + 2] = inf;
    }
    if (!last_block(&st->ticket[TK_RESTART])) return;
    double rp = 0.0, rd = 0.0, ri = 0.0;
    const volatile double* p = part;
    for (unsigned b = threadIdx.x; b < gridDim.x; b += kBlock) {
        rp += p[3 * b];
        rd += p[3 * b + 1];
        ri += p[3 * b + 2];
    }
    po = block_sum(rp);
    du = block_sum(rd);
    inf = block_sum(ri);
    if (threadIdx.x == 0) {
        st->ticket[TK_RESTART] = 0u;
        const double acc = a.P.obj_const + po;
        const bool fin = inf == 0.0;
        st->objective = acc;
        st->dual_objective = du;
        st->gap_finite = fin ? 1 : 0;
        st->duality_gap = fin ? fabs(acc - du) / (1.0 + fabs(acc) + fabs(du)) : INFINITY;
        st->pinf = acc_read(&st->acc[ACC_FIN_PINF]);
        st->dinf = acc_read(&st->acc[ACC_FIN_DINF]);
        st->acc[ACC_FIN_PINF] = st->acc[ACC_FIN_DINF] = 0ull;
    }
}

// ---------------------------------------------------------------------------
// Point selection and initialisation
// ---------------------------------------------------------------------------

template <class T>
__global__ void k_select_point(Iterates<T> it, const DevState* st, int32_t n, int32_t m,
                               double* bx, double* by) {
    const int t = blockIdx.x * kBlock + threadIdx.x;
    // Halpern: after a check the sums' slots hold T(z), the reported point
    const bool cand_avg = it.halpern ? st->checks > 0 : (st->converged && st->avg_better);
    const double inv = it.halpern ? 1.0 : st->inv;
    if (t < n) {
        if (cand_avg) {
            const double s = it.psx ? it.xsum[t] + static_cast<double>(it.psx[t]) : it.xsum[t];
            bx[t] = __dmul_rn(s, inv);
        } else {
            bx[t] = static_cast<double>(it.x[t]);
        }
    }
    if (t < m) {
        if (cand_avg) {
            const double s = it.psy ? it.ysum[t] + static_cast<double>(it.psy[t]) : it.ysum[t];
            by[t] = __dmul_rn(s, inv);
        } else {
            by[t] = static_cast<double>(it.y[t]);
        }
    }
}

// x = proj_X(x0), y = y0, s = proj_S(A x0) for a warm start; with no warm start
// x0 = 0, y0 = 0 and s = proj_S(0) (pdhg.cpp:268-270).
template <class T>
__global__ void k_init_point(DevProblem P, DevCsr A, const double* x0s, const double* y0s,
                             Iterates<T> it) {
    const int t = blockIdx.x * kBlock + threadIdx.x;
    if (t < P.n) {
        const double x = clampd(x0s ? x0s[t] : 0.0, P.lo[t], P.hi[t]);
        it.x[t] = static_cast<T>(x);
        it.xbar[t] = static_cast<T>(x);
        if (it.xsum) it.xsum[t] = 0.0;
        if (it.psx) it.psx[t] = static_cast<T>(0);
    }
    if (t < P.m) {
        double s = 0.0;
        if (x0s) {
            for (int k = A.rp[t]; k < A.rp[t + 1]; ++k)
                s = __dadd_rn(s, __dmul_rn(A.v64[k], clampd(x0s[A.ci[k]], P.lo[A.ci[k]], P.hi[A.ci[k]])));
        }
        it.s[t] = static_cast<T>(clampd(s, P.rlo[t], P.rhi[t]));
        it.y[t] = static_cast<T>(y0s ? y0s[t] : 0.0);
        if (it.ysum) it.ysum[t] = 0.0;
        if (it.psy) it.psy[t] = static_cast<T>(0);
    }
}

// ---------------------------------------------------------------------------
// Backend primitives
// ---------------------------------------------------------------------------

__global__ void k_spmv_exact(DevCsr A, double alpha, const double* x, double beta, double* y) {
    // HostBackend::spmv, backend_host.cpp:415-423 (beta == 0 overwrites)
    const RowTask t = row_task(A, blockIdx.x);
    if (t.row < 0) return;
    const double sum = row_dot(t, A, [x](int j) { return x[j]; }, 0.0);
    if (!t.lead) return;
    const int r = t.row;
    y[r] = (beta == 0.0) ? __dmul_rn(alpha, sum)
                         : __dadd_rn(__dmul_rn(alpha, sum), __dmul_rn(beta, y[r]));
}

// HostBackend::spmv_transpose, backend_host.cpp:434-444, on the transposed
// CSR: y_c starts at 0 (beta == 0) or y_c * beta, then adds val * (alpha x_r)
// in ascending row order.
__global__ void k_spmvT_exact(DevCsr AT, double alpha, const double* x, double beta, double* y) {
    const RowTask t = row_task(AT, blockIdx.x);
    if (t.row < 0) return;
    const int c = t.row;
    const double init = (beta == 0.0) ? 0.0 : __dmul_rn(y[c], beta);
    const double sum = row_dot(t, AT, [x, alpha](int r) { return __dmul_rn(alpha, x[r]); }, init);
    if (t.lead) y[c] = sum;
}

__global__ void k_project_box(int32_t n, const double* lo, const double* hi, double* x) {
    const int i = blockIdx.x * kBlock + threadIdx.x;
    if (i >= n) return;
    double v = x[i];
    if (lo != nullptr && v < lo[i]) v = lo[i];
    if (hi != nullptr && v > hi[i]) v = hi[i];
    x[i] = v;
}

// ---------------------------------------------------------------------------
// Transpose
// ---------------------------------------------------------------------------

// Groups of `lanes` threads (about the mean row length) fill a row each.
__global__ void k_row_of_entry(int32_t m, const int32_t* rp, int32_t* row, int lanes) {
    const int64_t tid = blockIdx.x * static_cast<int64_t>(kBlock) + threadIdx.x;
    const int64_t r = tid / lanes;
    if (r >= m) return;
    const int e = rp[r + 1];
    for (int k = rp[r] + static_cast<int>(tid % lanes); k < e; k += lanes) row[k] = static_cast<int32_t>(r);
}

__global__ void k_iota(int32_t* v, int64_t n) {
    const int64_t t = blockIdx.x * static_cast<int64_t>(kBlock) + threadIdx.x;
    if (t < n) v[t] = static_cast<int32_t>(t);
}

__global__ void k_col_count(const int32_t* ci, int64_t nnz, int32_t* cnt) {
    const int64_t t = blockIdx.x * static_cast<int64_t>(kBlock) + threadIdx.x;
    if (t < nnz) atomicAdd(&cnt[ci[t]], 1);
}

__global__ void k_gather_t(const int32_t* perm, const int32_t* row, const double* v,
                           int64_t nnz, int32_t* ci_t, double* v_t) {
    const int64_t t = blockIdx.x * static_cast<int64_t>(kBlock) + threadIdx.x;
    if (t >= nnz) return;
    const int32_t e = perm[t];
    ci_t[t] = row[e];
    v_t[t] = v[e];
}

__global__ void k_to_float(const double* src, float* dst, int64_t n) {
    const int64_t t = blockIdx.x * static_cast<int64_t>(kBlock) + threadIdx.x;
    if (t < n) dst[t] = static_cast<float>(src[t]);
}

inline int grid64(int64_t n) { return static_cast<int>((n + kBlock - 1) / kBlock); }

}  // namespace

// ---------------------------------------------------------------------------
// Launchers
// ---------------------------------------------------------------------------

int exact_check_grid(const DevCsr& A, const DevCsr& AT) { return mat_blocks(A) + mat_blocks(AT); }

void launch_exact_primal(const ExactIter& a, int first, cudaStream_t s) {
    if (a.AT.rows > 0) ex_primal<<<mat_blocks(a.AT), kBlock, 0, s>>>(a, first);
}
void launch_exact_dual(const ExactIter& a, int first, cudaStream_t s) {
    if (a.A.rows > 0) ex_dual<<<mat_blocks(a.A), kBlock, 0, s>>>(a, first);
}
void launch_exact_check(const ExactCheck& a, cudaStream_t s) {
    const int g1 = mat_blocks(a.A) + mat_blocks(a.AT);
    const int g2 = mat_blocks(a.Ao) + mat_blocks(a.ATo);
    ex_check1<<<g1 > 0 ? g1 : 1, kBlock, 0, s>>>(a);
    ex_check2<<<g2 > 0 ? g2 : 1, kBlock, 0, s>>>(a);
}
void launch_exact_restart(const ExactCheck& a, cudaStream_t s) {
    const int32_t nmax = a.AT.rows > a.A.rows ? a.AT.rows : a.A.rows;
    ex_restart<<<nmax > 0 ? blocks_for(nmax) : 1, kBlock, 0, s>>>(a);
}

int64_t pairwise_partial_size(int64_t n) {
    const int d = pw_depth(n);
    return (int64_t{1} << d) * 2 + 2;
}

void launch_pairwise_dot(const double* x, const double* y, int64_t n, double* partial,
                         double* out, cudaStream_t s) {
    if (n <= 0) {
        launch_fill(out, 1, 0.0, s);
        return;
    }
    const int d = pw_depth(n);
    const int64_t count = int64_t{1} << d;
    double* a = partial;
    double* b = partial + count;
    // the CTA's range: 32 nodes of at most ceil(n / 2^d) <= 256 entries
    const int64_t per = (n + count - 1) / count;
    const size_t smem = sizeof(double) * static_cast<size_t>(kPwNodes * per);
    if (smem > 48 * 1024)  // up to 64 KB: above the default dynamic limit
        cudaFuncSetAttribute(k_pw_level_staged, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             static_cast<int>(sizeof(double) * kPwNodes * kPwMaxNode));
    k_pw_level_staged<<<static_cast<unsigned>((count + kPwNodes - 1) / kPwNodes), kBlock, smem, s>>>(
        x, y, n, d, a);
    int lvl = d;
    for (; lvl > 10; --lvl) {  // wide levels: one launch each
        const int64_t half = int64_t{1} << (lvl - 1);
        k_pw_fold_level<<<grid64(half), kBlock, 0, s>>>(a, b, half);
        double* t = a;
        a = b;
        b = t;
    }
    k_pw_fold_tail<<<1, 512, 0, s>>>(a, b, lvl, out);  // the last <= 1024 values in one CTA
}

void launch_pw_w(const DevCsr& A, const double* u, const double* v, double* w, cudaStream_t s,
                 const int* stop, const double* uscale, bool fast) {
    if (A.rows == 0) return;
    if (fast) k_pw_w<true><<<mat_blocks(A), kBlock, 0, s>>>(A, u, v, w, stop, uscale);
    else k_pw_w<false><<<mat_blocks(A), kBlock, 0, s>>>(A, u, v, w, stop, uscale);
}
void launch_pw_u(const DevCsr& AT, const double* w, double* u, cudaStream_t s, const int* stop) {
    if (AT.rows > 0) k_pw_u<<<mat_blocks(AT), kBlock, 0, s>>>(AT, w, u, stop);
}
void launch_scale(double* x, int64_t n, double alpha, cudaStream_t s) {
    if (n > 0) k_scale<<<grid64(n), kBlock, 0, s>>>(x, n, alpha);
}
void launch_pw_norm_w(const double* dot, double* st, int* stop, cudaStream_t s) {
    k_pw_norm_w<<<1, 1, 0, s>>>(dot, st, stop);
}
void launch_pw_norm_e(const double* dots, double* st, int* stop, cudaStream_t s) {
    k_pw_norm_e<<<1, 1, 0, s>>>(dots, st, stop);
}
void launch_scale_by(double* x, int64_t n, const double* alpha, const int* stop, cudaStream_t s) {
    if (n > 0) k_scale_by<<<grid64(n), kBlock, 0, s>>>(x, n, alpha, stop);
}
void launch_copy_unless(double* dst, const double* src, int64_t n, const int* stop, cudaStream_t s) {
    if (n > 0) k_copy_unless<<<grid64(n), kBlock, 0, s>>>(dst, src, n, stop);
}
void launch_fill(double* x, int64_t n, double v, cudaStream_t s) {
    if (n > 0) k_fill<<<grid64(n), kBlock, 0, s>>>(x, n, v);
}

void launch_final(const FinalArgs& a, cudaStream_t s) {
    const int32_t nmax = a.P.n > a.P.m ? a.P.n : a.P.m;
    if (nmax > 0) k_fin_unscale<<<blocks_for(nmax), kBlock, 0, s>>>(a);
    const int g = mat_blocks(a.Ao) + mat_blocks(a.ATo);
    if (g > 0) k_fin_rowscols<<<g, kBlock, 0, s>>>(a);
    if (a.exact) {
        k_fin_sums_exact<<<1, 32, 0, s>>>(a);
    } else {
        int gs = blocks_for(nmax > 0 ? nmax : 1);
        if (gs > a.part_blocks) gs = a.part_blocks;
        k_fin_sums_tree<<<gs > 0 ? gs : 1, kBlock, 0, s>>>(a, a.part);
    }
}

template <class T>
void launch_select_point(const Iterates<T>& it, const DevState* st, int32_t n, int32_t m,
                         double* bx, double* by, cudaStream_t s) {
    const int32_t nmax = n > m ? n : m;
    if (nmax > 0) k_select_point<T><<<blocks_for(nmax), kBlock, 0, s>>>(it, st, n, m, bx, by);
}
template void launch_select_point<double>(const Iterates<double>&, const DevState*, int32_t,
                                          int32_t, double*, double*, cudaStream_t);
template void launch_select_point<float>(const Iterates<float>&, const DevState*, int32_t,
                                         int32_t, double*, double*, cudaStream_t);

// The Halpern anchor z_a <- z (the initial point).
template <class T>
__global__ void k_set_anchor(Iterates<T> it, int32_t n, int32_t m) {
    const int t = blockIdx.x * kBlock + threadIdx.x;
    if (t < n) it.xa[t] = it.x[t];
    if (t < m) {
        it.sa[t] = it.s[t];
        it.ya[t] = it.y[t];
    }
}

template <class T>
void launch_set_anchor(const Iterates<T>& it, int32_t n, int32_t m, cudaStream_t s) {
    const int32_t nmax = n > m ? n : m;
    if (nmax > 0) k_set_anchor<T><<<blocks_for(nmax), kBlock, 0, s>>>(it, n, m);
}
template void launch_set_anchor<float>(const Iterates<float>&, int32_t, int32_t, cudaStream_t);
template void launch_set_anchor<double>(const Iterates<double>&, int32_t, int32_t, cudaStream_t);

template <class T>
void launch_init_point(const DevProblem& P, const DevCsr& A, const double* x0s,
                       const double* y0s, Iterates<T> it, cudaStream_t s) {
    const int32_t nmax = P.n > P.m ? P.n : P.m;
    if (nmax > 0) k_init_point<T><<<blocks_for(nmax), kBlock, 0, s>>>(P, A, x0s, y0s, it);
}
template void launch_init_point<double>(const DevProblem&, const DevCsr&, const double*,
                                        const double*, Iterates<double>, cudaStream_t);
template void launch_init_point<float>(const DevProblem&, const DevCsr&, const double*,
                                       const double*, Iterates<float>, cudaStream_t);

void launch_spmv_exact(const DevCsr& A, double alpha, const double* x, double beta, double* y,
                       cudaStream_t s) {
    if (A.rows > 0) k_spmv_exact<<<mat_blocks(A), kBlock, 0, s>>>(A, alpha, x, beta, y);
}
void launch_spmvT_exact(const DevCsr& AT, double alpha, const double* x, double beta, double* y,
                        cudaStream_t s) {
    if (AT.rows > 0) k_spmvT_exact<<<mat_blocks(AT), kBlock, 0, s>>>(AT, alpha, x, beta, y);
}
void launch_project_box(int32_t n, const double* lo, const double* hi, double* x,
                        cudaStream_t s) {
    if (n > 0) k_project_box<<<blocks_for(n), kBlock, 0, s>>>(n, lo, hi, x);
}
void launch_to_float(const double* src, float* dst, int64_t n, cudaStream_t s) {
    if (n > 0) k_to_float<<<grid64(n), kBlock, 0, s>>>(src, dst, n);
}

int prefix_rows(const int32_t* cnt, int32_t n, int32_t* out, cudaStream_t s) {
    cudaMemsetAsync(out, 0, sizeof(int32_t), s);
    if (n <= 0) return static_cast<int>(cudaGetLastError() != cudaSuccess);
    size_t bytes = 0;
    cub::DeviceScan::InclusiveSum(nullptr, bytes, cnt, out + 1, n, s);
    void* tmp = nullptr;
    if (cudaMallocAsync(&tmp, bytes + 16, s) != cudaSuccess) return 1;
    cub::DeviceScan::InclusiveSum(tmp, bytes, cnt, out + 1, n, s);
    cudaFreeAsync(tmp, s);
    return static_cast<int>(cudaGetLastError() != cudaSuccess);
}

namespace {

// Scratch layout of build_transpose: column counts, scan temp, row of each
// entry, sorted keys, entry ids in and out, sort temp; 256-byte aligned parts.
struct TransposeLayout {
    size_t cnt = 0, scan_tmp = 0, row = 0, keys = 0, ids_in = 0, ids_out = 0, sort_tmp = 0;
    size_t scan_bytes = 0, sort_bytes = 0, total = 0;
    int bits = 1;
};

size_t align256(size_t b) { return (b + 255) & ~static_cast<size_t>(255); }

TransposeLayout transpose_layout(int32_t m, int32_t n, int64_t nnz) {
    TransposeLayout L;
    while ((int64_t{1} << L.bits) < static_cast<int64_t>(n)) ++L.bits;
    cub::DeviceScan::InclusiveSum(nullptr, L.scan_bytes, static_cast<const int32_t*>(nullptr),
                                  static_cast<int32_t*>(nullptr), n > 0 ? n : 1);
    cub::DeviceRadixSort::SortPairs(nullptr, L.sort_bytes, static_cast<const int32_t*>(nullptr),
                                    static_cast<int32_t*>(nullptr),
                                    static_cast<const int32_t*>(nullptr),
                                    static_cast<int32_t*>(nullptr),
                                    static_cast<int>(nnz > 0 ? nnz : 1), 0, L.bits);
    size_t off = 0;
    auto take = [&off](size_t bytes) {
        const size_t at = off;
        off += align256(bytes);
        return at;
    };
    const size_t e = sizeof(int32_t) * static_cast<size_t>(nnz > 0 ? nnz : 1);
    L.cnt = take(sizeof(int32_t) * (static_cast<size_t>(n) + 1));
    L.scan_tmp = take(L.scan_bytes + 16);
    L.row = take(e);
    L.keys = take(e);
    L.ids_in = take(e);
    L.ids_out = take(e);
    L.sort_tmp = take(L.sort_bytes + 16);
    L.total = off;
    (void)m;
    return L;
}

}  // namespace

size_t transpose_scratch_bytes(int32_t m, int32_t n, int64_t nnz) {
    return transpose_layout(m, n, nnz).total;
}

int build_transpose(int32_t m, int32_t n, int64_t nnz, const int32_t* rp, const int32_t* ci,
                    const double* v, TransposeOut out, void* scratch, cudaStream_t s) {
    const TransposeLayout L = transpose_layout(m, n, nnz);
    char* base = static_cast<char*>(scratch);
    // counts -> row pointer of A^T
    int32_t* cnt = reinterpret_cast<int32_t*>(base + L.cnt);
    cudaMemsetAsync(cnt, 0, sizeof(int32_t) * (static_cast<size_t>(n) + 1), s);
    if (nnz > 0) k_col_count<<<grid64(nnz), kBlock, 0, s>>>(ci, nnz, cnt + 1);
    cudaMemsetAsync(out.rp, 0, sizeof(int32_t), s);
    size_t scan_bytes = L.scan_bytes;
    if (n > 0) cub::DeviceScan::InclusiveSum(base + L.scan_tmp, scan_bytes, cnt + 1, out.rp + 1, n, s);
    if (nnz == 0) return static_cast<int>(cudaGetLastError() != cudaSuccess);
    // stable sort of entry ids by column
    int32_t* row = reinterpret_cast<int32_t*>(base + L.row);
    int32_t* keys_out = reinterpret_cast<int32_t*>(base + L.keys);
    int32_t* ids_in = reinterpret_cast<int32_t*>(base + L.ids_in);
    int32_t* ids_out = reinterpret_cast<int32_t*>(base + L.ids_out);
    if (m > 0) {
        int lanes = 1;
        while (lanes < 32 && static_cast<int64_t>(lanes) * m < nnz) lanes *= 2;
        k_row_of_entry<<<grid64(static_cast<int64_t>(m) * lanes), kBlock, 0, s>>>(m, rp, row, lanes);
    }
    k_iota<<<grid64(nnz), kBlock, 0, s>>>(ids_in, nnz);
    size_t sort_bytes = L.sort_bytes;
    cub::DeviceRadixSort::SortPairs(base + L.sort_tmp, sort_bytes, ci, keys_out, ids_in, ids_out,
                                    static_cast<int>(nnz), 0, L.bits, s);
    k_gather_t<<<grid64(nnz), kBlock, 0, s>>>(ids_out, row, v, nnz, out.ci, out.v);
    return static_cast<int>(cudaGetLastError() != cudaSuccess);
}

}  // namespace pdhg
