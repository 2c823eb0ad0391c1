// engine.cu -- host orchestration of the PDHG engine and the C-ABI
// (include/pdhg_b200.h).
//
// pdhg_solve follows Pdhg::solve (src/l1/pdhg.cpp:218-502) step for step:
// validation, scaling, step size from the power iteration, the iteration loop
// with a check every restart_check_period iterations, and the final result.
// What changes is where the work runs: every iteration and every check is a
// device kernel; the host only enqueues. One check period (period x 2 fused
// iteration kernels + the check kernels) is captured once as a CUDA graph and
// launched repeatedly; the device decides convergence, restarts and failure
// and every later kernel returns at once after a stop, so the host can keep
// several periods in flight and only waits on an event ring. Time limit and
// cancellation reach the device through a host-mapped mailbox that the check
// reads (granularity: one check period, where the reference polls every
// iteration, pdhg.cpp:288-293).
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <limits>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/pdhg_b200.h"
#include "dev_buffer.cuh"
#include "engine.cuh"
#include "host_prep.hpp"

namespace pdhg {

namespace {

constexpr double kInf = std::numeric_limits<double>::infinity();
constexpr int kLookahead = 4;
constexpr int kStopSwitchPrecision = 100;  // internal stop code: FP32 phase stalled

// Everything a captured check-period graph bakes into its kernel parameters.
struct GraphSig {
    int prec = -1;
    long long period = 0;
    int cand = 0;
    double tol = 0, bt = 0, dec = 0;
    int rule = 0, restart_rule = 0, pw = 0, infeas = 0, halpern = 0;
    long long gen = -1;
    bool operator==(const GraphSig& o) const {
        return prec == o.prec && period == o.period && cand == o.cand && tol == o.tol &&
               bt == o.bt && dec == o.dec && rule == o.rule && restart_rule == o.restart_rule &&
               pw == o.pw && infeas == o.infeas && halpern == o.halpern && gen == o.gen;
    }
};

}  // namespace

struct Ctx {
    int device = 0;
    int sm_count = 148;
    cudaStream_t stream = nullptr;
    PassFork fork;  // side stream + events: short- and long-row kernels side by side
    std::string err;
    long long gen = 0;  // bumps on every load / rescale

    bool loaded = false, valid = false;
    std::string why;
    HostLp lp;
    ScalingParams sp;
    bool scaled = false;
    double bnorm = 0, cnorm = 0;       // relative-KKT norms, original space (inf-norms)
    double bnorm2 = 0, cnorm2 = 0;     // termination rule 2 norms, original space (l2)
    int col_uniform = 0;               // every column has the scaled bounds lo_u, hi_u
    double lo_u = 0, hi_u = 0;
    int col_uniform_o = 0;             // ... and the original bounds lo_uo, hi_uo
    double lo_uo = 0, hi_uo = 0;
    double cnorm2_s = 0, bnorm2_s = 0;  // initial primal weight |c|_2 / |b|_2, scaled space

    MatDev Ao, ATo, As, ATs;
    DBuf<double> c_o, lo_o, hi_o, rlo_o, rhi_o, c_s, lo_s, hi_s, rlo_s, rhi_s, rs_d, cs_d;
    DBuf<float> c32, lo32, hi32, rlo32, rhi32;

    bool have_opnorm = false;
    int opnorm_iters = -1;
    bool opnorm_fast = false;  // the estimate's rows were summed in parallel (non-exact modes)
    double opnorm = 0;

    DBuf<double> x64, xbar64, s64, y64, xsum, ysum;
    DBuf<float> x32, xbar32, s32, y32, psx, psy;
    bool halpern = false;  // the current solve runs the Halpern iteration (its anchors below)
    bool lean = false;     // ... without storing z's x part (Iterates::lean); off when tracing
    DBuf<double> xa64, sa64, ya64;
    DBuf<float> xa32, sa32, ya32;
    DBuf<double> act_avg, cand_xo, cand_yo, part, bx, by, xo, yo, rc, trow, tcol;
    DBuf<double> pw_u, pw_v, pw_w, pw_part, pw_out, x0s, y0s;
    DBuf<int> pw_stop;
    DBuf<double> x_last, y_last;  // restart points (primal-weight update)
    DBuf<double> ray_yp, ray_atyp, ray_y;  // infeasibility test: previous y, A^T y; dy (original)
    DBuf<double> xray_xp, xray_d0, xray_d1;  // ray test: previous x; two projected rays (scaled)
    DBuf<DevState> st;
    Mailbox* mail = nullptr;
    Mailbox* mail_dev = nullptr;

    cudaGraphExec_t graph = nullptr;
    GraphSig graph_sig;
    long long launches = 0;

    // Checkpoint feed: two pinned slots, each the candidate (x: n, y: m, original
    // units) and the solver state of one period, copied on the stream behind
    // the period so that the callback reads them while the next period runs.
    double* cb_pin = nullptr;
    DevState* cb_state = nullptr;
    size_t cb_cap = 0;  // doubles per slot

    BatchCtx* batch = nullptr;  // pdhg_load_batch / pdhg_solve_batch

    // Iteration-kernel shapes per fast precision ([0] MIXED, [1] FP64):
    // {primal lanes, primal long mode, dual lanes, dual long mode}; reset on load.
    struct Tuning {
        bool have = false;
        bool timed = false;
        int shape[4] = {0, 0, 0, 0};
    } tuning[2];

    ~Ctx() {
        if (batch != nullptr) batch_delete(batch);
        if (graph != nullptr) cudaGraphExecDestroy(graph);
        if (mail != nullptr) cudaFreeHost(mail);
        if (cb_pin != nullptr) cudaFreeHost(cb_pin);
        if (cb_state != nullptr) cudaFreeHost(cb_state);
        if (fork.fork != nullptr) cudaEventDestroy(fork.fork);
        for (int i = 0; i < 2; ++i) {
            if (fork.join[i] != nullptr) cudaEventDestroy(fork.join[i]);
            if (fork.side[i] != nullptr) cudaStreamDestroy(fork.side[i]);
        }
        if (stream != nullptr) cudaStreamDestroy(stream);
    }

    DevProblem problem() const {
        DevProblem P;
        P.m = lp.m;
        P.n = lp.n;
        P.obj_sign = lp.maximize ? -1.0 : 1.0;
        P.obj_const = lp.obj_const;
        P.c = c_s.p;
        P.lo = lo_s.p;
        P.hi = hi_s.p;
        P.rlo = rlo_s.p;
        P.rhi = rhi_s.p;
        P.c_o = c_o.p;
        P.lo_o = lo_o.p;
        P.hi_o = hi_o.p;
        P.rlo_o = rlo_o.p;
        P.rhi_o = rhi_o.p;
        P.rs = rs_d.p;
        P.cs = cs_d.p;
        P.c32 = c32.p;
        P.lo32 = lo32.p;
        P.hi32 = hi32.p;
        P.rlo32 = rlo32.p;
        P.rhi32 = rhi32.p;
        P.bnorm = bnorm;
        P.cnorm = cnorm;
        P.bnorm2 = bnorm2;
        P.cnorm2 = cnorm2;
        P.col_bounds_uniform = col_uniform;
        P.col_bounds_uniform_o = col_uniform_o;
        P.lo_uo = lo_uo;
        P.hi_uo = hi_uo;
        P.lo_u = lo_u;
        P.hi_u = hi_u;
        return P;
    }
};

}  // namespace pdhg

struct pdhg_ctx {
    pdhg::Ctx c;
};

namespace pdhg {
namespace {

int fail(Ctx& c, cudaError_t e, const char* what) {
    c.err = std::string(what) + ": " + cudaGetErrorString(e);
    return e == cudaErrorMemoryAllocation ? PDHG_ERR_OUT_OF_MEMORY : PDHG_ERR_BACKEND;
}

#define CK(expr)                                               \
    do {                                                       \
        cudaError_t e_ = (expr);                               \
        if (e_ != cudaSuccess) return fail(c, e_, #expr);      \
    } while (0)

// Scaling::equilibrate(Problem) (scaling.cpp:155-205) on the device, from the
// original A / A^T already resident: factors, scaled matrices, scaled vectors.
int ensure_scaled(Ctx& c, const ScalingParams& sp) {
    if (c.scaled && c.sp == sp) return PDHG_OK;
    cudaStream_t s = c.stream;
    const int32_t m = c.lp.m, n = c.lp.n;
    const int64_t nnz = c.Ao.nnz;
    c.sp = sp;
    PhaseClock pc(s);
    CK(c.rs_d.alloc(static_cast<size_t>(m) + 1));
    CK(c.cs_d.alloc(static_cast<size_t>(n) + 1));
    launch_fill(c.rs_d.p, m, 1.0, s);
    launch_fill(c.cs_d.p, n, 1.0, s);
    DBuf<double> rbuf, cbuf;
    CK(rbuf.alloc(static_cast<size_t>(m) + 1));
    CK(cbuf.alloc(static_cast<size_t>(n) + 1));
    DBuf<IntakeState> is;
    CK(is.alloc(1));
    CK(cudaMemsetAsync(is.p, 0, sizeof(IntakeState), s));
    const DevCsr A = c.Ao.view(), AT = c.ATo.view();
    if (sp.apply_ruiz)  // scaling.cpp:36-74
        for (int sweep = 0; sweep < sp.ruiz_iterations; ++sweep)
            launch_ruiz_sweep(A, AT, c.rs_d.p, c.cs_d.p, rbuf.p, cbuf.p, sp.ruiz_tolerance, is.p, s);
    pc.mark("scale: ruiz");
    if (sp.apply_pock_chambolle)  // scaling.cpp:80-101
        launch_pock_chambolle(A, AT, c.rs_d.p, c.cs_d.p, rbuf.p, cbuf.p, sp.pock_chambolle_alpha, s);
    pc.mark("scale: pock-chambolle");
    // scaled values of A and A^T; entries the reference's rebuild drops are counted
    DBuf<unsigned long long> dropped;
    CK(dropped.alloc(1));
    CK(cudaMemsetAsync(dropped.p, 0, sizeof(unsigned long long), s));
    CK(c.As.v64.alloc(static_cast<size_t>(nnz)));
    launch_scale_values(A, 0, c.rs_d.p, c.cs_d.p, c.As.v64.p, dropped.p, s);
    unsigned long long ndrop = 0;
    CK(cudaMemcpyAsync(&ndrop, dropped.p, sizeof ndrop, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    c.As.rows = m;
    c.As.cols = n;
    c.ATs.rows = n;
    c.ATs.cols = m;
    if (ndrop == 0) {
        c.As.nnz = nnz;
        c.ATs.nnz = nnz;
        CK(copy_dev(c.As.rp, c.Ao.rp.p, static_cast<size_t>(m) + 1, s));
        CK(copy_dev(c.As.ci, c.Ao.ci.p, static_cast<size_t>(nnz), s));
        CK(copy_dev(c.ATs.rp, c.ATo.rp.p, static_cast<size_t>(n) + 1, s));
        CK(copy_dev(c.ATs.ci, c.ATo.ci.p, static_cast<size_t>(nnz), s));
        CK(c.ATs.v64.alloc(static_cast<size_t>(nnz)));
        CK(cudaMemsetAsync(dropped.p, 0, sizeof(unsigned long long), s));
        launch_scale_values(AT, 1, c.rs_d.p, c.cs_d.p, c.ATs.v64.p, dropped.p, s);
    } else {
        // compaction (sparse.cpp:55 drops |v| <= 1e-14), then a fresh transpose
        DBuf<int32_t> kept;
        CK(kept.alloc(static_cast<size_t>(m) + 1));
        launch_kept_counts(A, c.As.v64.p, kept.p, s);
        CK(c.As.rp.alloc(static_cast<size_t>(m) + 1));
        if (prefix_rows(kept.p, m, c.As.rp.p, s) != 0) return fail(c, cudaGetLastError(), "prefix_rows");
        const int64_t nk = static_cast<int64_t>(nnz - static_cast<int64_t>(ndrop));
        DBuf<double> vk;
        CK(c.As.ci.alloc(static_cast<size_t>(nk)));
        CK(vk.alloc(static_cast<size_t>(nk)));
        launch_compact(A, c.As.v64.p, c.As.rp.p, c.As.ci.p, vk.p, s);
        CK(copy_dev(c.As.v64, vk.p, static_cast<size_t>(nk), s));
        c.As.nnz = nk;
        c.ATs.nnz = nk;
        CK(c.ATs.rp.alloc(static_cast<size_t>(n) + 1));
        CK(c.ATs.ci.alloc(static_cast<size_t>(nk)));
        CK(c.ATs.v64.alloc(static_cast<size_t>(nk)));
        CK(c.ATs.tscratch.alloc(transpose_scratch_bytes(m, n, nk)));
        TransposeOut out{c.ATs.rp.p, c.ATs.ci.p, c.ATs.v64.p};
        if (build_transpose(m, n, nk, c.As.rp.p, c.As.ci.p, c.As.v64.p, out, c.ATs.tscratch.p, s) != 0)
            return fail(c, cudaGetLastError(), "build_transpose");
    }
    pc.mark("scale: values");
    CK(to_float(c.As.v32, c.As.v64, s));
    CK(to_float(c.ATs.v32, c.ATs.v64, s));
    int rc = bin_matrix(c.As, s, &c.err);
    if (rc != PDHG_OK) return rc;
    rc = bin_matrix(c.ATs, s, &c.err);
    if (rc != PDHG_OK) return rc;
    rc = build_slices(c.As, s, &c.err);
    if (rc != PDHG_OK) return rc;
    rc = build_slices(c.ATs, s, &c.err);
    if (rc != PDHG_OK) return rc;
    rc = build_dense_rows(c.As, s, &c.err);
    if (rc != PDHG_OK) return rc;
    rc = build_dense_rows(c.ATs, s, &c.err);
    if (rc != PDHG_OK) return rc;
    const double sign = c.lp.maximize ? -1.0 : 1.0;
    CK(c.c_s.alloc(static_cast<size_t>(n) + 1));
    CK(c.lo_s.alloc(static_cast<size_t>(n) + 1));
    CK(c.hi_s.alloc(static_cast<size_t>(n) + 1));
    CK(c.rlo_s.alloc(static_cast<size_t>(m) + 1));
    CK(c.rhi_s.alloc(static_cast<size_t>(m) + 1));
    launch_scale_vectors(m, n, c.rs_d.p, c.cs_d.p, c.c_o.p, c.lo_o.p, c.hi_o.p, c.rlo_o.p,
                         c.rhi_o.p, sign, c.c_s.p, c.lo_s.p, c.hi_s.p, c.rlo_s.p, c.rhi_s.p, s);
    CK(to_float(c.c32, c.c_s, s));
    CK(to_float(c.lo32, c.lo_s, s));
    CK(to_float(c.hi32, c.hi_s, s));
    CK(to_float(c.rlo32, c.rlo_s, s));
    CK(to_float(c.rhi32, c.rhi_s, s));
    DBuf<double> part;
    CK(part.alloc(static_cast<size_t>(norms_part_size(m, n))));
    launch_norms(m, n, c.c_s.p, c.rlo_s.p, c.rhi_s.p, c.c_o.p, c.rlo_o.p, c.rhi_o.p, part.p, is.p, s);
    // columns that all share their scaled bounds (x >= 0 LPs): the iteration
    // kernels then skip the bound loads
    // (and the check kernels those of the original bounds)
    DBuf<unsigned> uflag;
    CK(uflag.alloc(2));
    CK(cudaMemsetAsync(uflag.p, 0, 2 * sizeof(unsigned), s));
    launch_uniform_vec(c.lo_s.p, n, uflag.p, s);
    launch_uniform_vec(c.hi_s.p, n, uflag.p, s);
    launch_uniform_vec(c.lo_o.p, n, uflag.p + 1, s);
    launch_uniform_vec(c.hi_o.p, n, uflag.p + 1, s);
    unsigned uh[2] = {1, 1};
    double b0[4] = {0.0, 0.0, 0.0, 0.0};
    CK(cudaMemcpyAsync(uh, uflag.p, sizeof uh, cudaMemcpyDeviceToHost, s));
    if (n > 0) {
        CK(cudaMemcpyAsync(&b0[0], c.lo_s.p, sizeof(double), cudaMemcpyDeviceToHost, s));
        CK(cudaMemcpyAsync(&b0[1], c.hi_s.p, sizeof(double), cudaMemcpyDeviceToHost, s));
        CK(cudaMemcpyAsync(&b0[2], c.lo_o.p, sizeof(double), cudaMemcpyDeviceToHost, s));
        CK(cudaMemcpyAsync(&b0[3], c.hi_o.p, sizeof(double), cudaMemcpyDeviceToHost, s));
    }
    IntakeState h;
    CK(cudaMemcpyAsync(&h, is.p, sizeof h, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    c.col_uniform = (n > 0 && uh[0] == 0) ? 1 : 0;
    c.lo_u = b0[0];
    c.hi_u = b0[1];
    c.col_uniform_o = (n > 0 && uh[1] == 0) ? 1 : 0;
    c.lo_uo = b0[2];
    c.hi_uo = b0[3];
    pc.mark("scale: bins, vectors");
    c.cnorm2_s = std::sqrt(h.norms[0]);
    c.bnorm2_s = std::sqrt(h.norms[1]);
    c.cnorm = h.norms[2];
    c.bnorm = h.norms[3];
    c.cnorm2 = std::sqrt(h.norms[4]);
    c.bnorm2 = std::sqrt(h.norms[5]);
    c.scaled = true;
    c.have_opnorm = false;
    c.gen += 1;
    c.tuning[0] = Ctx::Tuning{};  // new matrices: shapes are chosen again
    c.tuning[1] = Ctx::Tuning{};
    rbuf.release();
    cbuf.release();
    part.release();
    pc.mark("scale: free scratch");
    return PDHG_OK;
}

// estimate_operator_norm (pdhg.cpp:48-79) with the exact kernels; the scalar
// tail (sqrt, 1/x) runs on the host exactly as in the reference.
// The power iteration of pdhg.cpp:50-78 with the reference's arithmetic
// (ordered sums, pairwise norms, IEEE square roots and divisions). Its scalar
// steps run on the device (k_pw_norm_w / _e), so the loop issues every
// iteration without waiting on the host; a device flag stands in for the
// loop's two early exits and turns the remaining launches into no-ops.
int operator_norm(Ctx& c, int iterations, bool fast, double* out) {
    cudaStream_t s = c.stream;
    const int32_t n = c.lp.n, m = c.lp.m;
    CK(c.pw_u.alloc(static_cast<size_t>(n) + 1));
    CK(c.pw_v.alloc(static_cast<size_t>(m) + 1));
    CK(c.pw_w.alloc(static_cast<size_t>(m) + 1));
    const int64_t ps = std::max(pairwise_partial_size(n), pairwise_partial_size(m));
    CK(c.pw_part.alloc(static_cast<size_t>(ps)));
    CK(c.pw_out.alloc(8));  // [0..1] norms' squares, [4..6] the scalar state
    CK(c.pw_stop.alloc(1));
    launch_fill(c.pw_u.p, n, 1.0, s);
    launch_fill(c.pw_v.p, m, 1.0, s);
    launch_fill(c.pw_w.p, m, 0.0, s);
    launch_fill(c.pw_out.p, 8, 0.0, s);
    launch_fill(c.pw_out.p + 6, 1, 1.0, s);  // u's scale before the first iteration
    CK(cudaMemsetAsync(c.pw_stop.p, 0, sizeof(int), s));
    const DevCsr A = c.As.view(), AT = c.ATs.view();
    double* dots = c.pw_out.p;
    double* st = c.pw_out.p + 4;
    int* stop = c.pw_stop.p;
    for (int it = 0; it < iterations; ++it) {
        launch_pw_w(A, c.pw_u.p, c.pw_v.p, c.pw_w.p, s, stop, st + 2, fast);  // u scaled where gathered
        launch_pairwise_dot(c.pw_w.p, c.pw_w.p, m, c.pw_part.p, dots, s);
        launch_pw_norm_w(dots, st, stop, s);
        launch_scale_by(c.pw_w.p, m, st, stop, s);
        launch_pw_u(AT, c.pw_w.p, c.pw_u.p, s, stop);
        launch_copy_unless(c.pw_v.p, c.pw_w.p, m, stop, s);
        launch_pairwise_dot(c.pw_u.p, c.pw_u.p, n, c.pw_part.p, dots, s);
        launch_pairwise_dot(c.pw_v.p, c.pw_v.p, m, c.pw_part.p, dots + 1, s);
        launch_pw_norm_e(dots, st, stop, s);
        launch_scale_by(c.pw_v.p, m, st + 2, stop, s);
    }
    CK(cudaGetLastError());
    double estimate = 0.0;
    CK(cudaMemcpyAsync(&estimate, st + 1, sizeof(double), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    *out = estimate;
    return PDHG_OK;
}

template <class T>
Iterates<T> iterates(Ctx& c);
template <>
Iterates<double> iterates<double>(Ctx& c) {
    Iterates<double> it;
    it.x = c.x64.p;
    it.xbar = c.xbar64.p;
    it.s = c.s64.p;
    it.y = c.y64.p;
    it.xsum = c.xsum.p;
    it.ysum = c.ysum.p;
    if (c.halpern) {
        it.xa = c.xa64.p;
        it.sa = c.sa64.p;
        it.ya = c.ya64.p;
        it.halpern = 1;
        it.lean = c.lean ? 1 : 0;
    }
    return it;
}
template <>
Iterates<float> iterates<float>(Ctx& c) {
    Iterates<float> it;
    it.x = c.x32.p;
    it.xbar = c.xbar32.p;
    it.s = c.s32.p;
    it.y = c.y32.p;
    it.psx = c.psx.p;
    it.psy = c.psy.p;
    it.xsum = c.xsum.p;
    it.ysum = c.ysum.p;
    if (c.halpern) {
        it.xa = c.xa32.p;
        it.sa = c.sa32.p;
        it.ya = c.ya32.p;
        it.halpern = 1;
        it.lean = c.lean ? 1 : 0;
    }
    return it;
}

int alloc_iterates(Ctx& c, bool f32) {
    const size_t n = static_cast<size_t>(c.lp.n) + 1, m = static_cast<size_t>(c.lp.m) + 1;
    CK(c.xsum.alloc(n));
    CK(c.ysum.alloc(m));
    if (c.halpern) {  // anchors: FP64 always (the mixed mode's FP64 phase), FP32 with f32
        CK(c.xa64.alloc(n));
        CK(c.sa64.alloc(m));
        CK(c.ya64.alloc(m));
        if (f32) {
            CK(c.xa32.alloc(n));
            CK(c.sa32.alloc(m));
            CK(c.ya32.alloc(m));
        }
    }
    if (f32) {
        CK(c.x32.alloc(n));
        CK(c.xbar32.alloc(n));
        CK(c.s32.alloc(m));
        CK(c.y32.alloc(m));
        CK(c.psx.alloc(n));
        CK(c.psy.alloc(m));
    }
    CK(c.x64.alloc(n));
    CK(c.xbar64.alloc(n));
    CK(c.s64.alloc(m));
    CK(c.y64.alloc(m));
    CK(c.act_avg.alloc(m));
    CK(c.cand_xo.alloc(n));
    CK(c.cand_yo.alloc(m));
    const int g = std::max({fast_check_grid(c.As.view(), c.ATs.view()),
                            exact_check_grid(c.As.view(), c.ATs.view()),
                            exact_check_grid(c.Ao.view(), c.ATo.view())}) + 1;
    CK(c.part.alloc(static_cast<size_t>(g) * kCheckSums + kCheckSums));
    CK(c.bx.alloc(n));
    CK(c.by.alloc(m));
    CK(c.xo.alloc(n));
    CK(c.yo.alloc(m));
    CK(c.rc.alloc(n));
    CK(c.trow.alloc(m));
    CK(c.tcol.alloc(n));
    return PDHG_OK;
}

struct Launcher {
    Ctx& c;
    int prec;
    ExactIter ei;
    ExactCheck ec;
    FastIter<float> fi32;
    FastIter<double> fi64;
    FastCheck<float> fc32;
    FastCheck<double> fc64;

    // iteration t of a check period (t = 0 first): the Halpern weight uses t;
    // tz: a check or the final selection reads this iteration's T(z)
    void iteration(long long t, cudaStream_t s, bool tz) {
        const int first = t == 0 ? 1 : 0;
        fi32.hk = fi64.hk = static_cast<int>(t);
        fi32.tz = fi64.tz = tz ? 1 : 0;
        if (prec == PDHG_PREC_FP64_EXACT) {
            launch_exact_primal(ei, first, s);
            launch_exact_dual(ei, first, s);
            c.launches += 2;
        } else if (prec == PDHG_PREC_MIXED) {
            c.launches += launch_fast_primal(fi32, first, s, &c.fork);
            c.launches += launch_fast_dual(fi32, first, s, &c.fork);
        } else {
            c.launches += launch_fast_primal(fi64, first, s, &c.fork);
            c.launches += launch_fast_dual(fi64, first, s, &c.fork);
        }
    }
    void check(long long period, cudaStream_t s) {
        if (prec == PDHG_PREC_FP64_EXACT) {
            ec.period_iters = period;
            launch_exact_check(ec, s);
            launch_exact_restart(ec, s);
            c.launches += 3;
        } else if (prec == PDHG_PREC_MIXED) {
            fc32.period_iters = period;
            launch_fast_check(fc32, s);
            launch_fast_restart(fc32, s);
            c.launches += 2 + (fc32.want_candidate ? 1 : 0) + fc32.infeas;
        } else {
            fc64.period_iters = period;
            launch_fast_check(fc64, s);
            launch_fast_restart(fc64, s);
            c.launches += 2 + (fc64.want_candidate ? 1 : 0) + fc64.infeas;
        }
    }
    long long launches_per_period(long long period) const {
        const long long chk =
            prec == PDHG_PREC_FP64_EXACT ? 3 : 2 + (fc32.want_candidate ? 1 : 0) + fc32.infeas;
        long long per_iter = 2;
        long long clear = 0;  // the flag reset when the primal pass has no rows
        if (prec != PDHG_PREC_FP64_EXACT) {
            per_iter = prec == PDHG_PREC_MIXED ? fast_launches_per_iteration(fi32)
                                               : fast_launches_per_iteration(fi64);
            clear = c.lp.n == 0 ? 1 : 0;
        }
        return per_iter * period + clear + chk;
    }
};

template <class T>
void apply_tuning(const Ctx::Tuning& t, FastIter<T>& fi) {
    if (!t.have) return;
    fi.AT.iter_vw = t.shape[0];
    fi.AT.long_mode = t.shape[1] & 3;
    fi.AT.use_slices = t.shape[1] >> 2;
    fi.A.iter_vw = t.shape[2];
    fi.A.long_mode = t.shape[3] & 3;
    fi.A.use_slices = t.shape[3] >> 2;
}

Launcher make_launcher(Ctx& c, int prec, const pdhg_options& o, bool want_candidate) {
    Launcher L{c, prec, {}, {}, {}, {}, {}, {}};
    const DevProblem P = c.problem();
    const double bt = o.tolerance > 1e-6 ? o.tolerance : 1e-6;
    L.ei = ExactIter{c.As.view(), c.ATs.view(), P, iterates<double>(c), c.st.p};
    CheckScratch cs{c.act_avg.p, c.cand_xo.p, c.cand_yo.p, c.part.p, 0};
    L.ec = ExactCheck{c.As.view(), c.ATs.view(), c.Ao.view(), c.ATo.view(), P,
                      iterates<double>(c), cs, o.tolerance, bt, o.restart_sufficient_decrease,
                      o.restart_check_period, o.termination_rule, want_candidate ? 1 : 0,
                      c.st.p, c.mail_dev};
    L.fi32 = FastIter<float>{c.As.view(), c.ATs.view(), P, iterates<float>(c), c.st.p};
    L.fi64 = FastIter<double>{c.As.view(), c.ATs.view(), P, iterates<double>(c), c.st.p};
    if (o.autotune) {
        apply_tuning(c.tuning[0], L.fi32);
        apply_tuning(c.tuning[1], L.fi64);
    }
    L.fc32 = FastCheck<float>{c.As.view(), c.ATs.view(), P, iterates<float>(c), cs,
                              o.tolerance, bt, o.restart_sufficient_decrease,
                              o.restart_check_period, o.termination_rule,
                              want_candidate ? 1 : 0, c.st.p, c.mail_dev, o.restart_rule,
                              o.primal_weight_update, c.x_last.p, c.y_last.p, 8 * c.sm_count};
    L.fc64 = FastCheck<double>{c.As.view(), c.ATs.view(), P, iterates<double>(c), cs,
                               o.tolerance, bt, o.restart_sufficient_decrease,
                               o.restart_check_period, o.termination_rule,
                               want_candidate ? 1 : 0, c.st.p, c.mail_dev, o.restart_rule,
                               o.primal_weight_update, c.x_last.p, c.y_last.p, 8 * c.sm_count};
    if (o.infeasibility_detection) {
        L.fc32.infeas = L.fc64.infeas = 1;
        L.fc32.ray_y_prev = L.fc64.ray_y_prev = c.ray_yp.p;
        L.fc32.ray_aty_prev = L.fc64.ray_aty_prev = c.ray_atyp.p;
        L.fc32.ray_y = L.fc64.ray_y = c.ray_y.p;
        L.fc32.xray_x_prev = L.fc64.xray_x_prev = c.xray_xp.p;
        L.fc32.xray_d[0] = L.fc64.xray_d[0] = c.xray_d0.p;
        L.fc32.xray_d[1] = L.fc64.xray_d[1] = c.xray_d1.p;
    }
    return L;
}

// Fresh control state: tau = eta / omega, sigma = eta * omega.
int reset_state(Ctx& c, double eta, double omega) {
    DevState h;
    std::memset(&h, 0, sizeof h);
    h.status = PDHG_STATUS_NOT_SOLVED;
    h.fresh = 1;
    h.res_last = kInf;
    h.res_prev_cand = kInf;
    h.eta = eta;
    h.omega = omega;
    h.tau = omega == 1.0 ? eta : eta / omega;
    h.sigma = omega == 1.0 ? eta : eta * omega;
    CK(cudaMemcpyAsync(c.st.p, &h, sizeof h, cudaMemcpyHostToDevice, c.stream));
    CK(cudaStreamSynchronize(c.stream));
    std::memset(const_cast<Mailbox*>(c.mail), 0, sizeof(Mailbox));
    return PDHG_OK;
}

int build_graph(Ctx& c, Launcher& L, long long period, const GraphSig& sig) {
    if (c.graph != nullptr && c.graph_sig == sig) return PDHG_OK;
    if (c.graph != nullptr) {
        cudaGraphExecDestroy(c.graph);
        c.graph = nullptr;
    }
    cudaGraph_t g = nullptr;
    const long long before = c.launches;
    CK(cudaStreamBeginCapture(c.stream, cudaStreamCaptureModeThreadLocal));
    for (long long t = 0; t < period; ++t) L.iteration(t, c.stream, t == period - 1);
    L.check(period, c.stream);
    cudaError_t e = cudaStreamEndCapture(c.stream, &g);
    c.launches = before;
    if (e != cudaSuccess) return fail(c, e, "cudaStreamEndCapture");
    e = cudaGraphInstantiate(&c.graph, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return fail(c, e, "cudaGraphInstantiate");
    c.graph_sig = sig;
    return PDHG_OK;
}

double elapsed_since(std::chrono::steady_clock::time_point t0) {
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

// Host copies of the scaled iterates for the trace option.
int trace_copy(Ctx& c, int prec, long long k, const pdhg_options& o) {
    const int32_t n = c.lp.n, m = c.lp.m;
    if (prec == PDHG_PREC_MIXED) {
        std::vector<float> hx(static_cast<size_t>(n)), hy(static_cast<size_t>(m));
        if (n) CK(cudaMemcpyAsync(hx.data(), c.x32.p, sizeof(float) * n, cudaMemcpyDeviceToHost, c.stream));
        if (m) CK(cudaMemcpyAsync(hy.data(), c.y32.p, sizeof(float) * m, cudaMemcpyDeviceToHost, c.stream));
        CK(cudaStreamSynchronize(c.stream));
        if (o.trace_x) for (int32_t j = 0; j < n; ++j) o.trace_x[k * n + j] = hx[j];
        if (o.trace_y) for (int32_t i = 0; i < m; ++i) o.trace_y[k * m + i] = hy[i];
    } else {
        if (o.trace_x && n)
            CK(cudaMemcpyAsync(o.trace_x + k * n, c.x64.p, sizeof(double) * n, cudaMemcpyDeviceToHost, c.stream));
        if (o.trace_y && m)
            CK(cudaMemcpyAsync(o.trace_y + k * m, c.y64.p, sizeof(double) * m, cudaMemcpyDeviceToHost, c.stream));
        CK(cudaStreamSynchronize(c.stream));
    }
    return PDHG_OK;
}

struct LoopOut {
    long long iterations = 0;
    int status = PDHG_STATUS_NOT_SOLVED;
    bool device_done = false;
    bool switch_precision = false;
    long long budget_used = 0;
};

// Runs up to `budget` iterations with launcher L. Handles checkpoints, the
// time limit, cancellation, verbose output and (mixed mode) stall detection.
int run_loop(Ctx& c, Launcher& L, const pdhg_options& o, long long budget, long long iter0,
             std::chrono::steady_clock::time_point t0, bool allow_switch, LoopOut* out) {
    const long long period = o.restart_check_period;
    const long long n_periods = budget / period;
    const long long tail = budget % period;
    const bool want_cb = o.checkpoint != nullptr;
    // With a checkpoint callback two periods are in flight and each hands its
    // candidate over through a pinned slot (the callback runs while the next
    // period computes); verbose output reads the mailbox, one period at a time.
    const int lookahead = o.verbose ? 1 : want_cb ? 2 : kLookahead;
    const bool feed = want_cb && lookahead == 2;
    if (feed) {
        const size_t need = static_cast<size_t>(c.lp.n) + static_cast<size_t>(c.lp.m) + 1;
        if (c.cb_cap < need) {
            if (c.cb_pin != nullptr) cudaFreeHost(c.cb_pin);
            c.cb_pin = nullptr;
            c.cb_cap = 0;
            CK(cudaHostAlloc(reinterpret_cast<void**>(&c.cb_pin), 2 * need * sizeof(double),
                             cudaHostAllocDefault));
            c.cb_cap = need;
        }
        if (c.cb_state == nullptr)
            CK(cudaHostAlloc(reinterpret_cast<void**>(&c.cb_state), 2 * sizeof(DevState),
                             cudaHostAllocDefault));
    }
    long long seen_checks = c.mail->checks;
    bool stop_sent = false;
    int stop_code = 0;
    double best = kInf;
    long long since_improve = 0;

    // Called after a period's event completed. slot >= 0: the period's pinned
    // snapshot (checkpoint feed); slot < 0: the mailbox and a synchronous copy.
    auto on_check = [&](int slot) -> int {
        const DevState* snap = slot >= 0 ? c.cb_state + slot : nullptr;
        const long long checks = snap ? snap->checks : static_cast<long long>(c.mail->checks);
        if (checks == seen_checks) return PDHG_OK;
        seen_checks = checks;
        const bool done = snap ? snap->done != 0 : c.mail->done != 0;
        const int status = snap ? snap->status : c.mail->status;
        const bool failed = done && status == PDHG_STATUS_NUMERICAL_FAILURE;
        const long long it = snap ? snap->iter : static_cast<long long>(c.mail->iter);
        const double orig_res = snap ? snap->orig_res : static_cast<double>(c.mail->orig_res);
        const double rel_kkt = snap ? snap->rel_kkt : static_cast<double>(c.mail->rel_kkt);
        if (o.verbose && c.mail->restarted && !failed)
            std::fprintf(stderr, "  [pdhg] restart at iter %lld, residual %.3g\n", it,
                         static_cast<double>(c.mail->avg_res));
        if (want_cb && !failed) {
            const int32_t n = c.lp.n, m = c.lp.m;
            if (snap) {
                const double* hx = c.cb_pin + static_cast<size_t>(slot) * c.cb_cap;
                o.checkpoint(o.checkpoint_user, it - 1, hx, hx + n, orig_res);
            } else {
                std::vector<double> hx(static_cast<size_t>(n)), hy(static_cast<size_t>(m));
                if (n) CK(cudaMemcpyAsync(hx.data(), c.cand_xo.p, sizeof(double) * n, cudaMemcpyDeviceToHost, c.stream));
                if (m) CK(cudaMemcpyAsync(hy.data(), c.cand_yo.p, sizeof(double) * m, cudaMemcpyDeviceToHost, c.stream));
                CK(cudaStreamSynchronize(c.stream));
                o.checkpoint(o.checkpoint_user, it - 1, hx.data(), hy.data(), orig_res);
            }
        }
        if (allow_switch && !done) {
            // The FP32 phase hands over to FP64 when it stops improving (no 2%
            // gain in 25 checks). Under rule 2 (l2 relative KKT) a plateau
            // counts only within kFp32Zone of FP32's unit roundoff: higher
            // plateaus are the method's, and FP64 iterations would not end
            // them sooner. The max-norm rules (0, 1) react to single entries,
            // whose FP32 rounding sets floors far above that, so any plateau
            // counts there.
            const double r = o.termination_rule != 0 ? rel_kkt : orig_res;
            if (o.termination_rule == 2 && r > kFp32Zone) {
                since_improve = 0;
                if (r < best) best = r;
            } else if (r < 0.98 * best) {
                best = r;
                since_improve = 0;
            } else if (++since_improve >= 25 && !stop_sent) {
                c.mail->stop_request = kStopSwitchPrecision;
                stop_sent = true;
                stop_code = kStopSwitchPrecision;
            }
        }
        return PDHG_OK;
    };
    auto poll_stop = [&]() {
        if (stop_sent) return;
        if (o.cancel_flag != nullptr && *o.cancel_flag) {
            stop_code = PDHG_STATUS_CANCELLED;
        } else if (o.time_limit_seconds > 0.0 && elapsed_since(t0) > o.time_limit_seconds) {
            stop_code = PDHG_STATUS_TIME_LIMIT;
        }
        if (stop_code != 0) {
            c.mail->stop_request = stop_code;
            stop_sent = true;
        }
    };

    long long p = 0;
    // Traced periods run kernel by kernel with a copy after each iteration.
    const long long traced = o.trace_iters > 0 ? o.trace_iters - iter0 : 0;
    while (p < n_periods && p * period < traced && !c.mail->done) {
        poll_stop();
        for (long long t = 0; t < period; ++t) {
            L.iteration(t, c.stream, t == period - 1);
            const long long k = iter0 + p * period + t;
            if (k < o.trace_iters) {
                int rc = trace_copy(c, L.prec, k, o);
                if (rc != PDHG_OK) return rc;
            }
        }
        L.check(period, c.stream);
        CK(cudaStreamSynchronize(c.stream));
        ++p;
        int rc = on_check(-1);
        if (rc != PDHG_OK) return rc;
    }
    if (p < n_periods && !c.mail->done) {
        GraphSig sig;
        sig.prec = L.prec;
        sig.period = period;
        sig.cand = want_cb ? 1 : 0;
        sig.tol = o.tolerance;
        sig.bt = L.ec.bound_tol;
        sig.dec = o.restart_sufficient_decrease;
        sig.rule = o.termination_rule;
        sig.restart_rule = o.restart_rule;
        sig.pw = o.primal_weight_update;
        sig.infeas = o.infeasibility_detection;
        sig.halpern = o.halpern ? (c.lean ? 2 : 1) : 0;
        sig.gen = c.gen;
        int rc = build_graph(c, L, period, sig);
        if (rc != PDHG_OK) return rc;
        std::deque<std::pair<cudaEvent_t, int>> inflight;  // event, pool slot
        std::vector<cudaEvent_t> pool;
        for (int i = 0; i < lookahead; ++i) {
            cudaEvent_t e;
            CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
            pool.push_back(e);
        }
        int next_ev = 0;
        const long long per = L.launches_per_period(period);
        while (true) {
            const bool can_launch = p < n_periods && !c.mail->done && !(stop_sent && stop_code != 0 && c.mail->done);
            if (can_launch && static_cast<int>(inflight.size()) < lookahead) {
                poll_stop();
                CK(cudaGraphLaunch(c.graph, c.stream));
                c.launches += per;
                const int slot = next_ev;
                if (feed) {
                    // this period's candidate and state into its pinned slot
                    // (reused two launches later, after this slot's callback)
                    const int32_t n = c.lp.n, m = c.lp.m;
                    double* hx = c.cb_pin + static_cast<size_t>(slot) * c.cb_cap;
                    if (n) CK(cudaMemcpyAsync(hx, c.cand_xo.p, sizeof(double) * n, cudaMemcpyDeviceToHost, c.stream));
                    if (m) CK(cudaMemcpyAsync(hx + n, c.cand_yo.p, sizeof(double) * m, cudaMemcpyDeviceToHost, c.stream));
                    CK(cudaMemcpyAsync(c.cb_state + slot, c.st.p, sizeof(DevState), cudaMemcpyDeviceToHost, c.stream));
                }
                cudaEvent_t e = pool[slot];
                next_ev = (next_ev + 1) % lookahead;
                CK(cudaEventRecord(e, c.stream));
                inflight.push_back({e, slot});
                ++p;
                continue;
            }
            if (inflight.empty()) break;
            const std::pair<cudaEvent_t, int> front = inflight.front();
            CK(cudaEventSynchronize(front.first));
            inflight.pop_front();
            int rc2 = on_check(feed ? front.second : -1);
            if (rc2 != PDHG_OK) return rc2;
        }
        for (cudaEvent_t e : pool) cudaEventDestroy(e);
    }
    CK(cudaStreamSynchronize(c.stream));
    const bool done = c.mail->done != 0;
    if (!done && tail > 0 && !stop_sent) {
        poll_stop();
        if (!stop_sent) {
            for (long long t = 0; t < tail; ++t) {
                L.iteration(t, c.stream, t == tail - 1);
                const long long k = iter0 + n_periods * period + t;
                if (k < o.trace_iters) {
                    int rc = trace_copy(c, L.prec, k, o);
                    if (rc != PDHG_OK) return rc;
                }
            }
            CK(cudaStreamSynchronize(c.stream));
        }
    }
    DevState h;
    CK(cudaMemcpy(&h, c.st.p, sizeof h, cudaMemcpyDeviceToHost));
    out->device_done = h.done != 0;
    if (h.done) {
        out->iterations = h.stop_iter - iter0;
        out->status = h.status;
        if (h.status == kStopSwitchPrecision) out->switch_precision = true;
    } else if (stop_sent && stop_code != 0 && stop_code != kStopSwitchPrecision) {
        out->iterations = h.iter - iter0;
        out->status = stop_code;
    } else {
        const bool ran_tail = !stop_sent && tail > 0;
        out->iterations = n_periods * period + (ran_tail ? tail : 0);
        out->status = PDHG_STATUS_ITERATION_LIMIT;
    }
    return PDHG_OK;
}

// Copies the scaled FP32 state into the FP64 iterates and restarts the
// Cesaro average there (the FP64 polish phase of the mixed mode).
__global__ void k_widen(Iterates<float> a, Iterates<double> b, int32_t n, int32_t m) {
    const int t = blockIdx.x * kBlock + threadIdx.x;
    // Halpern: the FP64 phase starts at T(z) (inside the bounds) as a restart
    // point, which is also its first anchor and (in the T(z) slot) its
    // reported point until its first iteration
    if (t < n) {
        b.x[t] = b.halpern ? a.psx[t] : a.x[t];
        b.xbar[t] = b.halpern ? a.psx[t] : a.xbar[t];
        b.xsum[t] = b.halpern ? static_cast<double>(a.psx[t]) : 0.0;
        if (b.halpern) b.xa[t] = b.x[t];
    }
    if (t < m) {
        b.y[t] = b.halpern ? a.psy[t] : a.y[t];
        b.s[t] = a.s[t];
        b.ysum[t] = b.halpern ? static_cast<double>(a.psy[t]) : 0.0;
        if (b.halpern) {
            b.ya[t] = b.y[t];
            b.sa[t] = b.s[t];
        }
    }
}

// v <- v / scale (primal) or (v * sign) / scale (dual), in place.
__global__ void k_to_scaled(double* v, const double* scale, double sign, int dual, int32_t n) {
    const int t = blockIdx.x * kBlock + threadIdx.x;
    if (t >= n) return;
    v[t] = dual ? (v[t] * sign) / scale[t] : v[t] / scale[t];
}

template <class T>
__global__ void k_snapshot(Iterates<T> it, double* xl, double* yl, int32_t n, int32_t m) {
    const int t = blockIdx.x * kBlock + threadIdx.x;
    if (t < n) xl[t] = static_cast<double>(it.x[t]);
    if (t < m) yl[t] = static_cast<double>(it.y[t]);
}

__global__ void k_restart_state(DevState* st) {
    st->done = 0;
    st->status = PDHG_STATUS_NOT_SOLVED;
    st->converged = 0;
    st->fresh = 1;
    st->restart = 0;
    st->fold = 0;
    st->since_restart = 0;
    st->res_last = INFINITY;
}

// ---- autotuner of the iteration kernels ----------------------------------------
//
// For each pass (primal over A^T, dual over A) the candidates are the lanes
// per short row around the binning's choice (vw/2, vw, 2vw) and, for the rows
// past the short ones, the long-row strategies that differ on this matrix
// (1 only when it has rows of kLongRow..kHugeRow entries). Each is
// timed with CUDA events on the engine's stream (2 launches to warm, 5
// timed) and replaces the current best only when faster by more than 5%, so
// noise does not flip the choice. LPs below kTuneMinNnz nonzeros are
// launch-latency bound and keep the defaults (and their summation order).
// Choices are cached per shape signature for the process, and in the JSON
// file named by PDHG_B200_TUNE_CACHE ({"signature": [lanes, mode], ...}).

constexpr int64_t kTuneMinNnz = int64_t{1} << 20;

std::mutex g_tune_mutex;
std::map<std::string, std::pair<int, int>> g_tune_cache;
bool g_tune_file_read = false;

const char* tune_file() {
    const char* f = std::getenv("PDHG_B200_TUNE_CACHE");
    return (f != nullptr && f[0] != '\0') ? f : nullptr;
}

// Reads `"key": [a, b]` entries of the cache file (called with the mutex held).
void tune_read_file() {
    if (g_tune_file_read) return;
    g_tune_file_read = true;
    const char* path = tune_file();
    if (path == nullptr) return;
    std::FILE* f = std::fopen(path, "r");
    if (f == nullptr) return;
    std::string txt;
    char buf[4096];
    size_t k;
    while ((k = std::fread(buf, 1, sizeof buf, f)) > 0) txt.append(buf, k);
    std::fclose(f);
    size_t pos = 0;
    while ((pos = txt.find('"', pos)) != std::string::npos) {
        const size_t end = txt.find('"', pos + 1);
        if (end == std::string::npos) break;
        const std::string key = txt.substr(pos + 1, end - pos - 1);
        int a = 0, b = 0;
        const size_t lb = txt.find('[', end);
        if (lb != std::string::npos && std::sscanf(txt.c_str() + lb, "[%d , %d]", &a, &b) == 2 &&
            a >= 1 && a <= 32 && (a & (a - 1)) == 0 && b >= 0 && b <= 6 && (b & 3) <= 2)
            g_tune_cache[key] = {a, b};
        pos = end + 1;
    }
}

void tune_write_file() {
    const char* path = tune_file();
    if (path == nullptr) return;
    std::FILE* f = std::fopen(path, "w");
    if (f == nullptr) return;
    std::fprintf(f, "{\n");
    size_t i = 0;
    for (const auto& kv : g_tune_cache)
        std::fprintf(f, "  \"%s\": [%d, %d]%s\n", kv.first.c_str(), kv.second.first,
                     kv.second.second, ++i < g_tune_cache.size() ? "," : "");
    std::fprintf(f, "}\n");
    std::fclose(f);
}

std::string tune_sig(const char* prec, const char* pass, const DevCsr& M) {
    char b[256];
    std::snprintf(b, sizeof b, "%s/%s/rows%d/cols%d/nnz%lld/short%d/long%d/mid%d/huge%d/vw%d/sl%d",
                  prec, pass, M.rows, M.cols, static_cast<long long>(M.nnz), M.n_short, M.n_long,
                  M.n_mid, M.n_huge, M.vw, M.slices.n_slice);
    return b;
}

template <class T>
float time_pass(Ctx& c, FastIter<T>& fi, bool primal, cudaEvent_t e0, cudaEvent_t e1) {
    auto run = [&]() {
        if (primal) launch_fast_primal(fi, 0, c.stream, &c.fork);
        else launch_fast_dual(fi, 0, c.stream, &c.fork);
    };
    run();
    run();
    cudaEventRecord(e0, c.stream);
    for (int r = 0; r < 5; ++r) run();
    cudaEventRecord(e1, c.stream);
    cudaEventSynchronize(e1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    return ms;
}

// Chooses {lanes, mode} for one pass (mode = long-row strategy + 4 when the
// row slices are used); fi's matrix fields are set to the choice.
template <class T>
void tune_pass(Ctx& c, FastIter<T>& fi, bool primal, const char* prec_tag, int* lanes,
               int* mode, cudaEvent_t e0, cudaEvent_t e1) {
    DevCsr& M = primal ? fi.AT : fi.A;
    M.iter_vw = M.vw;
    M.long_mode = 0;
    M.use_slices = 0;
    *lanes = M.vw;
    *mode = 0;
    if (M.rows == 0 || M.nnz < kTuneMinNnz) return;
    const std::string key = tune_sig(prec_tag, primal ? "primal" : "dual", M);
    {
        std::lock_guard<std::mutex> lock(g_tune_mutex);
        tune_read_file();
        const auto it = g_tune_cache.find(key);
        if (it != g_tune_cache.end()) {
            M.iter_vw = *lanes = it->second.first;
            *mode = it->second.second;
            M.long_mode = *mode & 3;
            M.use_slices = (*mode >> 2) != 0 && M.slices.n_item > 0 ? 1 : 0;
            return;
        }
    }
    // candidates, the binning's choice first
    std::vector<std::pair<int, int>> cand{{M.vw, 0}};
    std::vector<int> vws{M.vw};
    if (M.n_short > 0) {
        if (M.vw > 1) vws.push_back(M.vw / 2);
        if (M.vw < 32) vws.push_back(M.vw * 2);
    }
    for (int vw : vws) {
        if (vw != M.vw) cand.push_back({vw, 0});
        if (M.n_mid > 0) cand.push_back({vw, 1});
        if (M.items_warp.n_item > 0) cand.push_back({vw, 2});
    }
    // two rounds over all candidates, each keeping its faster time, so no
    // candidate is timed only on a cold GPU (clocks ramping, first launches)
    std::vector<float> t(cand.size(), 3.0e38f);
    for (int round = 0; round < 2; ++round)
        for (size_t i = 0; i < cand.size(); ++i) {
            M.iter_vw = cand[i].first;
            M.long_mode = cand[i].second;
            t[i] = std::min(t[i], time_pass(c, fi, primal, e0, e1));
        }
    size_t pick = 0;
    for (size_t i = 1; i < cand.size(); ++i)
        if (t[i] < 0.95f * t[pick]) pick = i;
    *lanes = cand[pick].first;
    *mode = cand[pick].second;
    M.iter_vw = *lanes;
    M.long_mode = *mode;
    if (M.slices.n_item > 0) {
        // the row slices on top of the best shape, each strategy over the
        // remaining long rows
        float best = t[pick];
        int best_mode = *mode;
        M.use_slices = 1;
        for (int m = 0; m <= 2; ++m) {
            if (m == 1 && M.n_mid == 0) continue;
            M.long_mode = m;
            float ts = 3.0e38f;
            for (int round = 0; round < 2; ++round) ts = std::min(ts, time_pass(c, fi, primal, e0, e1));
            if (ts < 0.95f * best) {
                best = ts;
                best_mode = m + 4;
            }
        }
        *mode = best_mode;
        M.long_mode = best_mode & 3;
        M.use_slices = best_mode >> 2;
    }
    std::lock_guard<std::mutex> lock(g_tune_mutex);
    g_tune_cache[key] = {*lanes, *mode};
    tune_write_file();
}

// Runs on the solve's own buffers before the initial point is written (the
// timed passes only overwrite iterates that the initial point resets).
template <class T>
int tune_iteration(Ctx& c, Launcher& L, FastIter<T>& fi, Ctx::Tuning& t, const char* tag) {
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    tune_pass(c, fi, true, tag, &t.shape[0], &t.shape[1], e0, e1);
    tune_pass(c, fi, false, tag, &t.shape[2], &t.shape[3], e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    CK(cudaGetLastError());
    t.have = true;
    t.timed = c.ATs.nnz >= kTuneMinNnz;
    (void)L;
    return PDHG_OK;
}

int solve(Ctx& c, const pdhg_options& o, pdhg_info* info, double* x, double* y, double* rcv) {
    const auto t0 = std::chrono::steady_clock::now();
    std::memset(info, 0, sizeof *info);
    info->status = PDHG_STATUS_NOT_SOLVED;
    c.launches = 0;
    if (!c.loaded) {
        c.err = "pdhg_solve: no problem loaded";
        return PDHG_ERR_INVALID_ARGUMENT;
    }
    if (!c.valid) {  // pdhg.cpp:223-228
        info->status = PDHG_STATUS_NUMERICAL_FAILURE;
        std::snprintf(info->message, sizeof info->message, "invalid problem: %s", c.why.c_str());
        return PDHG_OK;
    }
    if (o.restart_check_period < 1 || o.power_iterations < 0 || o.precision < 0 ||
        o.precision > 2 || o.termination_rule < 0 || o.termination_rule > 2 ||
        o.restart_rule < 0 || o.restart_rule > 2 || o.primal_weight_update < 0 ||
        o.primal_weight_update > 1) {
        c.err = "pdhg_solve: invalid options";
        return PDHG_ERR_INVALID_ARGUMENT;
    }
    if ((o.termination_rule == 2 && o.precision == PDHG_PREC_FP64_EXACT) ||
        (o.restart_rule == 2 && o.termination_rule != 2)) {
        c.err = "pdhg_solve: termination rule 2 needs precision mixed or fp64, and restart rule 2 "
                "needs termination rule 2 (it restarts on rule 2's measure)";
        return PDHG_ERR_INVALID_ARGUMENT;
    }
    if (o.precision == PDHG_PREC_FP64_EXACT && (o.restart_rule != 0 || o.primal_weight_update)) {
        c.err = "pdhg_solve: the adaptive restart rule and the primal weight need precision "
                "mixed or fp64 (fp64_exact reproduces the reference, which has neither)";
        return PDHG_ERR_INVALID_ARGUMENT;
    }
    if (o.halpern < 0 || o.halpern > 1 ||
        (o.halpern && (o.precision == PDHG_PREC_FP64_EXACT || o.termination_rule != 2 ||
                       o.restart_rule != 2 || o.infeasibility_detection))) {
        c.err = "pdhg_solve: halpern is 0 or 1 and needs precision mixed or fp64, termination "
                "rule 2 and restart rule 2, and no infeasibility detection";
        return PDHG_ERR_INVALID_ARGUMENT;
    }
    if (o.infeasibility_detection < 0 || o.infeasibility_detection > 1 ||
        (o.precision == PDHG_PREC_FP64_EXACT && o.infeasibility_detection)) {
        c.err = "pdhg_solve: infeasibility_detection is 0 or 1 and needs precision mixed or "
                "fp64 (fp64_exact reproduces the reference, which never reports infeasible)";
        return PDHG_ERR_INVALID_ARGUMENT;
    }
    CK(cudaSetDevice(c.device));
    c.halpern = o.halpern != 0;
    c.lean = c.halpern && o.trace_iters <= 0;
    ScalingParams sp;
    sp.ruiz_iterations = o.ruiz_iterations;
    sp.ruiz_tolerance = o.ruiz_tolerance;
    sp.pock_chambolle_alpha = o.pock_chambolle_alpha;
    sp.apply_ruiz = o.apply_ruiz != 0;
    sp.apply_pock_chambolle = o.apply_pock_chambolle != 0;
    PhaseClock pc(c.stream);
    int rc = ensure_scaled(c, sp);
    if (rc != PDHG_OK) return rc;
    pc.mark("solve: scaling");
    // FP64-exact reproduces the reference's estimate bit for bit; the other
    // modes sum A u's long rows in parallel (the same estimate up to rounding)
    const bool fast_norm = o.precision != PDHG_PREC_FP64_EXACT;
    if (!c.have_opnorm || c.opnorm_iters != o.power_iterations || c.opnorm_fast != fast_norm) {
        rc = operator_norm(c, o.power_iterations, fast_norm, &c.opnorm);
        if (rc != PDHG_OK) return rc;
        c.have_opnorm = true;
        c.opnorm_iters = o.power_iterations;
        c.opnorm_fast = fast_norm;
    }
    pc.mark("solve: operator norm");
    const double op = c.opnorm;
    info->operator_norm_estimate = op;  // pdhg.cpp:261-265
    const double step = (op > 1e-9) ? o.step_size_safety / op : o.step_size_safety;
    // primal weight: 1 (tau = sigma = step) unless updated; then it starts at |c|/|b|
    double omega = 1.0;
    if (o.primal_weight_update && c.cnorm2_s > 1e-10 && c.bnorm2_s > 1e-10)
        omega = c.cnorm2_s / c.bnorm2_s;

    int prec = o.precision;
    rc = alloc_iterates(c, prec == PDHG_PREC_MIXED);
    if (rc != PDHG_OK) return rc;
    if (o.infeasibility_detection) {
        // the first check only stores its x, A x, y and A^T y (DevState.ray_base = 0)
        const size_t m1 = static_cast<size_t>(c.lp.m) + 1, n1 = static_cast<size_t>(c.lp.n) + 1;
        CK(c.ray_yp.alloc(m1));
        CK(c.ray_atyp.alloc(n1));
        CK(c.ray_y.alloc(m1));
        CK(c.xray_xp.alloc(n1));
        CK(c.xray_d0.alloc(n1));
        CK(c.xray_d1.alloc(n1));
        for (DBuf<double>* b : {&c.ray_yp, &c.ray_atyp, &c.ray_y, &c.xray_xp, &c.xray_d0, &c.xray_d1})
            CK(cudaMemsetAsync(b->p, 0, sizeof(double) * b->n, c.stream));
    }
    CK(c.st.alloc(1));
    if (prec != PDHG_PREC_FP64_EXACT && o.autotune) {
        Ctx::Tuning& t = c.tuning[prec == PDHG_PREC_MIXED ? 0 : 1];
        if (!t.have) {
            rc = reset_state(c, step, omega);  // live state for the timed passes
            if (rc != PDHG_OK) return rc;
            Launcher L = make_launcher(c, prec, o, false);
            rc = prec == PDHG_PREC_MIXED ? tune_iteration(c, L, L.fi32, t, "f32")
                                         : tune_iteration(c, L, L.fi64, t, "f64");
            if (rc != PDHG_OK) return rc;
        }
        pc.mark("solve: autotune");
    }

    // Initial point (pdhg.cpp:268-270) or the warm start, in scaled space.
    const int32_t n = c.lp.n, m = c.lp.m;
    const double sign = c.lp.maximize ? -1.0 : 1.0;
    const double* x0d = nullptr;
    const double* y0d = nullptr;
    // x_s = x / col_scale, y_s = (y * obj_sign) / row_scale (inverse of
    // unscale_to_original, pdhg.cpp:205-214)
    if (o.x0 != nullptr) {
        CK(upload(c.x0s, o.x0, static_cast<size_t>(n), c.stream));
        if (n > 0)
            k_to_scaled<<<(n + kBlock - 1) / kBlock, kBlock, 0, c.stream>>>(c.x0s.p, c.cs_d.p, 1.0, 0, n);
        x0d = c.x0s.p;
    }
    if (o.y0 != nullptr) {
        CK(upload(c.y0s, o.y0, static_cast<size_t>(m), c.stream));
        if (m > 0)
            k_to_scaled<<<(m + kBlock - 1) / kBlock, kBlock, 0, c.stream>>>(c.y0s.p, c.rs_d.p, sign, 1, m);
        y0d = c.y0s.p;
    }
    const DevProblem P = c.problem();
    if (prec == PDHG_PREC_MIXED)
        launch_init_point<float>(P, c.As.view(), x0d, y0d, iterates<float>(c), c.stream);
    else
        launch_init_point<double>(P, c.As.view(), x0d, y0d, iterates<double>(c), c.stream);
    c.launches += 1;
    if (c.halpern) {  // the first anchor is the initial point
        if (prec == PDHG_PREC_MIXED) launch_set_anchor<float>(iterates<float>(c), n, m, c.stream);
        else launch_set_anchor<double>(iterates<double>(c), n, m, c.stream);
        c.launches += 1;
    }
    if (o.primal_weight_update) {
        CK(c.x_last.alloc(static_cast<size_t>(n) + 1));
        CK(c.y_last.alloc(static_cast<size_t>(m) + 1));
        const int g = (std::max(n, m) + kBlock) / kBlock;
        if (prec == PDHG_PREC_MIXED)
            k_snapshot<float><<<g, kBlock, 0, c.stream>>>(iterates<float>(c), c.x_last.p, c.y_last.p, n, m);
        else
            k_snapshot<double><<<g, kBlock, 0, c.stream>>>(iterates<double>(c), c.x_last.p, c.y_last.p, n, m);
        c.launches += 1;
    }
    rc = reset_state(c, step, omega);
    if (rc != PDHG_OK) return rc;

    long long iterations = 0;
    int status = PDHG_STATUS_NOT_SOLVED;
    const long long max_it = o.max_iterations > 0 ? o.max_iterations : 0;
    // The reference checks cancellation, then the time limit, before every
    // iteration (pdhg.cpp:288-293); these two catch the iteration-0 case.
    bool early = false;
    if (max_it > 0 && o.cancel_flag != nullptr && *o.cancel_flag) {
        status = PDHG_STATUS_CANCELLED;
        early = true;
    } else if (max_it > 0 && o.time_limit_seconds > 0.0 && elapsed_since(t0) > o.time_limit_seconds) {
        status = PDHG_STATUS_TIME_LIMIT;
        early = true;
    }
    cudaEvent_t ev0, ev1;
    CK(cudaEventCreate(&ev0));
    CK(cudaEventCreate(&ev1));
    pc.mark("solve: initial point");
    CK(cudaEventRecord(ev0, c.stream));
    long long fp64_its = 0;
    if (!early) {
        const bool want_cb = o.checkpoint != nullptr;
        Launcher L = make_launcher(c, prec, o, want_cb);
        LoopOut lo;
        const bool allow_switch = prec == PDHG_PREC_MIXED && o.polish_iterations != 0;
        rc = run_loop(c, L, o, max_it, 0, t0, allow_switch, &lo);
        if (rc != PDHG_OK) return rc;
        iterations = lo.iterations;
        status = lo.status;
        if (lo.switch_precision) {
            // FP64 phase from the FP32 point, for the remaining budget.
            long long left = max_it - iterations;
            if (o.polish_iterations > 0 && o.polish_iterations < left) left = o.polish_iterations;
            k_widen<<<(std::max(n, m) + kBlock) / kBlock, kBlock, 0, c.stream>>>(
                iterates<float>(c), iterates<double>(c), n, m);
            k_restart_state<<<1, 1, 0, c.stream>>>(c.st.p);
            c.launches += 2;
            std::memset(const_cast<Mailbox*>(c.mail), 0, sizeof(Mailbox));
            prec = PDHG_PREC_FP64;
            Launcher L2 = make_launcher(c, prec, o, want_cb);
            LoopOut lo2;
            rc = run_loop(c, L2, o, left, iterations, t0, false, &lo2);
            if (rc != PDHG_OK) return rc;
            iterations += lo2.iterations;
            fp64_its = lo2.iterations;
            status = lo2.status;
        }
    }
    CK(cudaEventRecord(ev1, c.stream));
    CK(cudaEventSynchronize(ev1));
    float loop_ms = 0.f;
    cudaEventElapsedTime(&loop_ms, ev0, ev1);
    cudaEventDestroy(ev0);
    cudaEventDestroy(ev1);
    pc.mark("solve: iterations");

    DevState h;
    CK(cudaMemcpy(&h, c.st.p, sizeof h, cudaMemcpyDeviceToHost));
    info->iterations = iterations;
    info->restarts = h.restarts;
    info->relative_kkt = h.rel_kkt;
    info->fp64_iterations = prec == PDHG_PREC_MIXED ? 0 : (fp64_its > 0 ? fp64_its : iterations);
    info->device_seconds = loop_ms * 1e-3;
    if (status == PDHG_STATUS_NUMERICAL_FAILURE) {  // pdhg.cpp:347-371 return early
        info->status = status;
        std::snprintf(info->message, sizeof info->message,
                      h.fail_kind == 2 ? "non-finite KKT residual (original units) at iteration %lld"
                                       : "non-finite KKT residual at iteration %lld",
                      iterations);
        info->has_point = 0;
        info->kernel_launches = c.launches;
        return PDHG_OK;
    }
    if (status == PDHG_STATUS_PRIMAL_INFEASIBLE) {  // engine extension: a certificate
        info->status = status;
        info->has_point = 0;
        info->kernel_launches = c.launches;
        std::snprintf(info->message, sizeof info->message,
                      "primal infeasible at iteration %lld: the row multipliers in y force "
                      "sum_i y_i (Ax)_i into [%.6g, %.6g] through the row bounds and into "
                      "[%.6g, %.6g] through the column bounds",
                      iterations, h.ray_ranges[0], h.ray_ranges[1], h.ray_ranges[2],
                      h.ray_ranges[3]);
        if (y != nullptr && m > 0) {
            CK(cudaMemcpy(y, c.ray_y.p, sizeof(double) * m, cudaMemcpyDeviceToHost));
            for (int32_t i = 0; i < m; ++i) y[i] *= h.ray_scale;
        }
        return PDHG_OK;
    }
    if (status == PDHG_STATUS_DUAL_INFEASIBLE) {  // engine extension: a ray in x
        info->status = status;
        info->has_point = 0;
        info->kernel_launches = c.launches;
        std::snprintf(info->message, sizeof info->message,
                      "dual infeasible (unbounded if feasible) at iteration %lld: along the ray "
                      "d in x (max |d_j| = 1) the objective falls by %.6g (minimize sense) and "
                      "the bounds are left by at most %.3g",
                      iterations, -h.xray_obj, h.xray_viol);
        if (x != nullptr && n > 0) {  // original units: d_o = d_s * cs, then max |d_j| = 1
            std::vector<double> cs(static_cast<size_t>(n));
            CK(cudaMemcpy(x, h.xray_buf ? c.xray_d1.p : c.xray_d0.p, sizeof(double) * n,
                          cudaMemcpyDeviceToHost));
            CK(cudaMemcpy(cs.data(), P.cs, sizeof(double) * n, cudaMemcpyDeviceToHost));
            for (int32_t j = 0; j < n; ++j) x[j] = x[j] * cs[j] * h.xray_scale;
        }
        return PDHG_OK;
    }
    if (status == PDHG_STATUS_NOT_SOLVED) status = PDHG_STATUS_ITERATION_LIMIT;
    info->status = status;

    // Final result (pdhg.cpp:420-498) on the original problem.
    if (prec == PDHG_PREC_MIXED)
        launch_select_point<float>(iterates<float>(c), c.st.p, n, m, c.bx.p, c.by.p, c.stream);
    else
        launch_select_point<double>(iterates<double>(c), c.st.p, n, m, c.bx.p, c.by.p, c.stream);
    FinalArgs fa;
    fa.Ao = c.Ao.view();
    fa.ATo = c.ATo.view();
    fa.P = P;
    fa.best_x64 = c.bx.p;
    fa.best_y64 = c.by.p;
    fa.f = FinalScratch{c.xo.p, c.yo.p, c.rc.p, c.trow.p, c.tcol.p};
    fa.bound_tol = o.tolerance > 1e-6 ? o.tolerance : 1e-6;
    fa.exact = o.precision == PDHG_PREC_FP64_EXACT ? 1 : 0;
    fa.st = c.st.p;
    fa.part = c.part.p;
    fa.part_blocks = static_cast<int>(std::min<size_t>(c.part.n / 3, 8 * static_cast<size_t>(c.sm_count)));
    launch_final(fa, c.stream);
    c.launches += 5;
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(&h, c.st.p, sizeof h, cudaMemcpyDeviceToHost, c.stream));
    if (x != nullptr && n) CK(cudaMemcpyAsync(x, c.xo.p, sizeof(double) * n, cudaMemcpyDeviceToHost, c.stream));
    if (y != nullptr && m) CK(cudaMemcpyAsync(y, c.yo.p, sizeof(double) * m, cudaMemcpyDeviceToHost, c.stream));
    if (rcv != nullptr && n) CK(cudaMemcpyAsync(rcv, c.rc.p, sizeof(double) * n, cudaMemcpyDeviceToHost, c.stream));
    CK(cudaStreamSynchronize(c.stream));
    pc.mark("solve: result, download");
    info->objective = h.objective;
    info->primal_infeasibility = h.pinf;
    info->dual_infeasibility = h.dinf;
    info->duality_gap = h.duality_gap;
    info->has_point = 1;
    info->kernel_launches = c.launches;
    info->seconds = elapsed_since(t0);
    if (o.infeasibility_detection && status != PDHG_STATUS_OPTIMAL)
        std::snprintf(info->message, sizeof info->message,
                      "no certificate; at the last test the multipliers' ranges were [%.6g, %.6g] "
                      "(rows) and [%.6g, %.6g] (columns), the ray's c^T d %.6g with cone "
                      "violation %.3g",
                      h.ray_ranges[0], h.ray_ranges[1], h.ray_ranges[2], h.ray_ranges[3],
                      h.xray_obj, h.xray_viol);
    return PDHG_OK;
}

int load(Ctx& c, int32_t m, int32_t n, int64_t nnz, const int32_t* row_ptr,
         const int32_t* col_idx, const double* values, const double* cv, double obj_const,
         int maximize, const double* col_lo, const double* col_hi, const double* row_lo,
         const double* row_hi) {
    if (m < 0 || n < 0 || nnz < 0 || nnz > std::numeric_limits<int32_t>::max()) {
        c.err = "pdhg_load_problem: sizes must be non-negative and fit int32 indices";
        return PDHG_ERR_INVALID_ARGUMENT;
    }
    if (row_ptr == nullptr || (nnz > 0 && (col_idx == nullptr || values == nullptr)) ||
        (n > 0 && (cv == nullptr || col_lo == nullptr || col_hi == nullptr)) ||
        (m > 0 && (row_lo == nullptr || row_hi == nullptr))) {
        c.err = "pdhg_load_problem: null array";
        return PDHG_ERR_INVALID_ARGUMENT;
    }
    CK(cudaSetDevice(c.device));
    c.loaded = false;
    c.scaled = false;
    c.have_opnorm = false;
    c.gen += 1;
    HostLp& lp = c.lp;  // scalars only: the arrays stay with the caller / on the device
    lp.m = m;
    lp.n = n;
    lp.obj_const = obj_const;
    lp.maximize = maximize != 0;
    lp.A.rows = m;
    lp.A.cols = n;
    LpView view;
    view.m = m;
    view.n = n;
    view.nnz = nnz;
    view.rp = row_ptr;
    view.ci = col_idx;
    view.v = values;
    view.c = cv;
    view.obj_const = obj_const;
    view.col_lo = col_lo;
    view.col_hi = col_hi;
    view.row_lo = row_lo;
    view.row_hi = row_hi;
    c.loaded = true;
    PhaseClock pc(c.stream);
    // Validation (problem.cpp:50-, sparse.cpp:94-128). row_ptr and the
    // objective constant are checked here; everything else on the device
    // after the upload. Whenever anything fails, the host check runs over the
    // whole problem for the reference's first failure and message.
    if (!std::isfinite(obj_const) || !row_ptr_ok(m, nnz, row_ptr)) {
        c.valid = validate_lp(view, &c.why);
        if (!c.valid) return PDHG_OK;
    }
    cudaStream_t s = c.stream;
    int rc = upload_csr(m, n, nnz, row_ptr, col_idx, values, c.Ao, s, &c.err);
    if (rc != PDHG_OK) return rc;
    CK(upload(c.c_o, cv, static_cast<size_t>(n), s));
    CK(upload(c.lo_o, col_lo, static_cast<size_t>(n), s));
    CK(upload(c.hi_o, col_hi, static_cast<size_t>(n), s));
    CK(upload(c.rlo_o, row_lo, static_cast<size_t>(m), s));
    CK(upload(c.rhi_o, row_hi, static_cast<size_t>(m), s));
    pc.mark("load: upload");
    unsigned flags = 0;
    rc = device_checks(c.Ao, c.c_o.p, c.lo_o.p, c.hi_o.p, c.rlo_o.p, c.rhi_o.p, &flags, s, &c.err);
    if (rc != PDHG_OK) return rc;
    pc.mark("load: device checks");
    c.valid = true;
    c.why.clear();
    if (flags != 0) {
        c.valid = validate_lp(view, &c.why);
        if (!c.valid) return PDHG_OK;
    }
    rc = finish_matrix(c.Ao, c.ATo, s, &c.err);
    if (rc != PDHG_OK) return rc;
    pc.mark("load: transpose, bins");
    return ensure_scaled(c, ScalingParams{});
}

// ---- profiling ----------------------------------------------------------------

// Algorithmic bytes of one pass: the matrix stream (row pointer, index,
// value), one read of each gathered vector entry, and the fused epilogue's
// vector reads and writes per row. Averaged iteration: 5 reads (c, x, lo, hi,
// sum; y, s, row bounds, sum) and 3 writes. Lean Halpern primal: 5 reads (c,
// x_bar, anchor, lo, hi) and 1 write (x_bar), plus x and T(z) once a check
// period; Halpern dual: 6 reads (y, s, row bounds, the two anchors), 2 writes,
// plus T(z) once a period. What this LP's structure makes constant carries
// no information and is not counted: the row pointer where every row has the
// same length, the column bounds where all are equal, the column indices of
// dense rows and (where the pass uses them) of affine row slices -- the
// kernels compute those instead of loading them.
double iter_bytes(const Ctx& c, int prec, bool primal, bool halpern, long long period,
                  const DevCsr& D) {
    const double vb = prec == PDHG_PREC_MIXED ? 4.0 : 8.0;  // value / vector element bytes
    const MatDev& M = primal ? c.ATs : c.As;
    const double nnz = static_cast<double>(M.nnz);
    const double rows = M.rows, cols = M.cols;
    const double per = period > 0 ? 1.0 / static_cast<double>(period) : 0.0;
    const double touches = primal ? (halpern ? 6.0 + 2.0 * per : 8.0) : (halpern ? 8.0 + per : 8.0);
    double b = 4.0 * (rows + 1) + (4.0 + vb) * nnz + vb * cols + vb * touches * rows;
    if (prec == PDHG_PREC_FP64_EXACT) return b;  // the ordered kernels load everything
    if (D.rp_stride > 0) b -= 4.0 * (rows + 1);
    if (primal && c.col_uniform) b -= 2.0 * vb * rows;
    b -= 4.0 * static_cast<double>(M.nnz_dense + (D.use_slices ? M.slices.nnz_affine : 0));
    return b;
}

int profile(Ctx& c, int prec, int warmup, int iters, pdhg_kernel_stats* out) {
    std::memset(out, 0, sizeof *out);
    if (!c.loaded || !c.valid || !c.have_opnorm) {
        c.err = "pdhg_profile_kernels: solve a valid problem first";
        return PDHG_ERR_INVALID_ARGUMENT;
    }
    CK(cudaSetDevice(c.device));
    // the kernels are timed in the form the last solve ran: averaged, or the
    // lean Halpern iteration (its T(z) and x stores, once a check period, left out)
    const bool hal = c.halpern && prec != PDHG_PREC_FP64_EXACT;
    c.halpern = hal;
    c.lean = hal;
    int rc = alloc_iterates(c, prec == PDHG_PREC_MIXED);
    if (rc != PDHG_OK) return rc;
    CK(c.st.alloc(1));
    pdhg_options o;
    pdhg_default_options(&o);
    o.precision = prec;
    o.termination_rule = hal ? 2 : 1;  // the check instance the solve's form runs
    o.restart_rule = hal ? 2 : o.restart_rule;
    const double step = c.opnorm > 1e-9 ? 0.9 / c.opnorm : 0.9;
    Launcher L = make_launcher(c, prec, o, false);
    rc = reset_state(c, step, 1.0);
    if (rc != PDHG_OK) return rc;
    const DevProblem P = c.problem();
    if (prec == PDHG_PREC_MIXED)
        launch_init_point<float>(P, c.As.view(), nullptr, nullptr, iterates<float>(c), c.stream);
    else
        launch_init_point<double>(P, c.As.view(), nullptr, nullptr, iterates<double>(c), c.stream);
    if (hal) {
        if (prec == PDHG_PREC_MIXED) launch_set_anchor<float>(iterates<float>(c), c.lp.n, c.lp.m, c.stream);
        else launch_set_anchor<double>(iterates<double>(c), c.lp.n, c.lp.m, c.stream);
    }
    for (int i = 0; i < warmup; ++i) L.iteration(i, c.stream, true);
    L.fi32.tz = L.fi64.tz = 0;
    std::vector<cudaEvent_t> ev(3 * static_cast<size_t>(iters) + 2);
    for (auto& e : ev) CK(cudaEventCreate(&e));
    for (int i = 0; i < iters; ++i) {
        CK(cudaEventRecord(ev[3 * i], c.stream));
        if (prec == PDHG_PREC_FP64_EXACT) launch_exact_primal(L.ei, 0, c.stream);
        else if (prec == PDHG_PREC_MIXED) launch_fast_primal(L.fi32, 0, c.stream, &c.fork);
        else launch_fast_primal(L.fi64, 0, c.stream, &c.fork);
        CK(cudaEventRecord(ev[3 * i + 1], c.stream));
        if (prec == PDHG_PREC_FP64_EXACT) launch_exact_dual(L.ei, 0, c.stream);
        else if (prec == PDHG_PREC_MIXED) launch_fast_dual(L.fi32, 0, c.stream, &c.fork);
        else launch_fast_dual(L.fi64, 0, c.stream, &c.fork);
        CK(cudaEventRecord(ev[3 * i + 2], c.stream));
    }
    CK(cudaEventRecord(ev[3 * iters], c.stream));
    L.check(1, c.stream);
    CK(cudaEventRecord(ev[3 * iters + 1], c.stream));
    CK(cudaStreamSynchronize(c.stream));
    double tp = 0, td = 0;
    for (int i = 0; i < iters; ++i) {
        float a = 0, b = 0;
        cudaEventElapsedTime(&a, ev[3 * i], ev[3 * i + 1]);
        cudaEventElapsedTime(&b, ev[3 * i + 1], ev[3 * i + 2]);
        tp += a;
        td += b;
    }
    float tc = 0;
    cudaEventElapsedTime(&tc, ev[3 * iters], ev[3 * iters + 1]);
    for (auto& e : ev) cudaEventDestroy(e);
    out->count = 3;
    std::snprintf(out->name[0], 32, "primal");
    std::snprintf(out->name[1], 32, "dual");
    std::snprintf(out->name[2], 32, "check");
    out->avg_ms[0] = iters ? tp / iters : 0;
    out->avg_ms[1] = iters ? td / iters : 0;
    out->avg_ms[2] = tc;
    const FastIter<float>& F32 = L.fi32;
    const FastIter<double>& F64 = L.fi64;
    const bool f32 = prec == PDHG_PREC_MIXED;
    out->bytes[0] = iter_bytes(c, prec, true, hal, o.restart_check_period, f32 ? F32.AT : F64.AT);
    out->bytes[1] = iter_bytes(c, prec, false, hal, o.restart_check_period, f32 ? F32.A : F64.A);
    out->bytes[2] = 2.0 * (12.0 * c.As.nnz) + 8.0 * 10 * (c.lp.n + c.lp.m);
    out->launches[0] = iters;
    out->launches[1] = iters;
    out->launches[2] = 1;
    return PDHG_OK;
}

}  // namespace
}  // namespace pdhg

// ============================================================================
// C-ABI
// ============================================================================

extern "C" {

int pdhg_abi_version(void) { return PDHG_B200_ABI_VERSION; }

void pdhg_default_options(pdhg_options* o) {
    if (o == nullptr) return;
    std::memset(o, 0, sizeof *o);
    o->tolerance = 1e-4;  // pdhg.hpp:89-117
    o->max_iterations = 1000000;
    o->time_limit_seconds = 0.0;
    o->restart_check_period = 40;
    o->restart_sufficient_decrease = 0.5;
    o->step_size_safety = 0.9;
    o->power_iterations = 30;
    o->verbose = 0;
    o->ruiz_iterations = 8;  // scaling.hpp:299-309
    o->ruiz_tolerance = 1e-2;
    o->pock_chambolle_alpha = 1.0;
    o->apply_ruiz = 1;
    o->apply_pock_chambolle = 1;
    o->precision = PDHG_PREC_FP64_EXACT;
    o->termination_rule = 0;
    o->polish_iterations = -1;
    o->autotune = 1;
    o->infeasibility_detection = 0;
    o->halpern = 0;
}

const char* pdhg_status_string(int s) {
    switch (s) {  // pdhg.cpp:17-27
        case PDHG_STATUS_OPTIMAL: return "optimal";
        case PDHG_STATUS_ITERATION_LIMIT: return "iteration_limit";
        case PDHG_STATUS_TIME_LIMIT: return "time_limit";
        case PDHG_STATUS_NUMERICAL_FAILURE: return "numerical_failure";
        case PDHG_STATUS_NOT_SOLVED: return "not_solved";
        case PDHG_STATUS_CANCELLED: return "cancelled";
        case PDHG_STATUS_PRIMAL_INFEASIBLE: return "primal_infeasible";  // engine extension
        case PDHG_STATUS_DUAL_INFEASIBLE: return "dual_infeasible";      // engine extension
    }
    return "unknown";
}

const char* pdhg_error_string(int e) {
    switch (e) {  // status.hpp:36-48
        case PDHG_OK: return "ok";
        case PDHG_ERR_UNSUPPORTED: return "unsupported by this backend";
        case PDHG_ERR_NOT_IMPLEMENTED: return "not implemented yet";
        case PDHG_ERR_INVALID_ARGUMENT: return "invalid argument";
        case PDHG_ERR_DIMENSION_MISMATCH: return "dimension mismatch";
        case PDHG_ERR_OUT_OF_MEMORY: return "out of memory";
        case PDHG_ERR_BACKEND: return "backend error";
        case PDHG_ERR_NUMERICAL_FAILURE: return "numerical failure";
    }
    return "unknown status";
}

int pdhg_create(int device, pdhg_ctx** out) {
    if (out == nullptr) return PDHG_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || device < 0 || device >= count)
        return PDHG_ERR_UNSUPPORTED;
    std::unique_ptr<pdhg_ctx> h;
    try {
        h.reset(new pdhg_ctx());
    } catch (...) {
        return PDHG_ERR_OUT_OF_MEMORY;
    }
    pdhg::Ctx& c = h->c;
    c.device = device;
    if (cudaSetDevice(device) != cudaSuccess) return PDHG_ERR_BACKEND;
    cudaDeviceGetAttribute(&c.sm_count, cudaDevAttrMultiProcessorCount, device);
    if (c.sm_count <= 0) c.sm_count = 148;
    if (pdhg::init_fast_kernels(device) != 0) return PDHG_ERR_BACKEND;
    if (cudaStreamCreateWithFlags(&c.stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaStreamCreateWithFlags(&c.fork.side[0], cudaStreamNonBlocking) != cudaSuccess ||
        cudaStreamCreateWithFlags(&c.fork.side[1], cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&c.fork.fork, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&c.fork.join[0], cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&c.fork.join[1], cudaEventDisableTiming) != cudaSuccess)
        return PDHG_ERR_BACKEND;
    void* mp = nullptr;
    if (cudaHostAlloc(&mp, sizeof(pdhg::Mailbox), cudaHostAllocMapped) != cudaSuccess)
        return PDHG_ERR_BACKEND;
    c.mail = static_cast<pdhg::Mailbox*>(mp);
    std::memset(mp, 0, sizeof(pdhg::Mailbox));
    void* dp = nullptr;
    if (cudaHostGetDevicePointer(&dp, mp, 0) != cudaSuccess) return PDHG_ERR_BACKEND;
    c.mail_dev = static_cast<pdhg::Mailbox*>(dp);
    *out = h.release();
    return PDHG_OK;
}

int pdhg_destroy(pdhg_ctx* ctx) {
    if (ctx == nullptr) return PDHG_ERR_INVALID_ARGUMENT;
    cudaSetDevice(ctx->c.device);
    if (ctx->c.stream != nullptr) cudaStreamSynchronize(ctx->c.stream);
    delete ctx;
    return PDHG_OK;
}

const char* pdhg_last_error(const pdhg_ctx* ctx) {
    return ctx == nullptr ? "null context" : ctx->c.err.c_str();
}

void* pdhg_stream(const pdhg_ctx* ctx) {
    return ctx == nullptr ? nullptr : static_cast<void*>(ctx->c.stream);
}

int pdhg_get_scaling(pdhg_ctx* ctx, double* row_scale, double* col_scale) {
    if (ctx == nullptr || row_scale == nullptr || col_scale == nullptr)
        return PDHG_ERR_INVALID_ARGUMENT;
    pdhg::Ctx& c = ctx->c;
    if (!c.loaded || !c.valid || !c.scaled) {
        c.err = "pdhg_get_scaling: no valid problem loaded";
        return PDHG_ERR_INVALID_ARGUMENT;
    }
    if (cudaSetDevice(c.device) != cudaSuccess) return PDHG_ERR_BACKEND;
    if (c.lp.m > 0 && cudaMemcpy(row_scale, c.rs_d.p, sizeof(double) * c.lp.m,
                                 cudaMemcpyDeviceToHost) != cudaSuccess)
        return PDHG_ERR_BACKEND;
    if (c.lp.n > 0 && cudaMemcpy(col_scale, c.cs_d.p, sizeof(double) * c.lp.n,
                                 cudaMemcpyDeviceToHost) != cudaSuccess)
        return PDHG_ERR_BACKEND;
    return PDHG_OK;
}

int pdhg_load_problem(pdhg_ctx* ctx, int32_t m, int32_t n, int64_t nnz, const int32_t* row_ptr,
                      const int32_t* col_idx, const double* values, const double* c,
                      double obj_const, int maximize, const double* col_lo,
                      const double* col_hi, const double* row_lo, const double* row_hi) {
    if (ctx == nullptr) return PDHG_ERR_INVALID_ARGUMENT;
    try {
        pdhg::PhaseClock pc(ctx->c.stream);
        const int rc = pdhg::load(ctx->c, m, n, nnz, row_ptr, col_idx, values, c, obj_const,
                                  maximize, col_lo, col_hi, row_lo, row_hi);
        pc.mark("pdhg_load_problem");
        return rc;
    } catch (const std::bad_alloc&) {
        ctx->c.err = "host allocation failed";
        return PDHG_ERR_OUT_OF_MEMORY;
    } catch (const std::exception& e) {
        ctx->c.err = e.what();
        return PDHG_ERR_BACKEND;
    }
}

int pdhg_solve(pdhg_ctx* ctx, const pdhg_options* options, pdhg_info* info, double* x,
               double* y, double* rc) {
    if (ctx == nullptr || info == nullptr) return PDHG_ERR_INVALID_ARGUMENT;
    pdhg_options o;
    if (options == nullptr) pdhg_default_options(&o);
    else o = *options;
    try {
        pdhg::PhaseClock pc(ctx->c.stream);
        const int r = pdhg::solve(ctx->c, o, info, x, y, rc);
        pc.mark("pdhg_solve");
        return r;
    } catch (const std::bad_alloc&) {
        ctx->c.err = "host allocation failed";
        return PDHG_ERR_OUT_OF_MEMORY;
    } catch (const std::exception& e) {
        ctx->c.err = e.what();
        return PDHG_ERR_BACKEND;
    }
}

int pdhg_profile_kernels(pdhg_ctx* ctx, int precision, int warmup, int iterations,
                         pdhg_kernel_stats* out) {
    if (ctx == nullptr || out == nullptr || iterations < 1 || warmup < 0 || precision < 0 ||
        precision > 2)
        return PDHG_ERR_INVALID_ARGUMENT;
    try {
        return pdhg::profile(ctx->c, precision, warmup, iterations, out);
    } catch (const std::exception& e) {
        ctx->c.err = e.what();
        return PDHG_ERR_BACKEND;
    }
}

int pdhg_get_tuning(const pdhg_ctx* ctx, int precision, int* out) {
    if (ctx == nullptr || out == nullptr ||
        (precision != PDHG_PREC_MIXED && precision != PDHG_PREC_FP64))
        return PDHG_ERR_INVALID_ARGUMENT;
    const pdhg::Ctx& c = ctx->c;
    const pdhg::Ctx::Tuning& t = c.tuning[precision == PDHG_PREC_MIXED ? 0 : 1];
    if (t.have) {
        for (int i = 0; i < 4; ++i) out[i] = t.shape[i];
    } else {
        out[0] = c.ATs.vw;
        out[1] = 0;
        out[2] = c.As.vw;
        out[3] = 0;
    }
    out[4] = t.timed ? 1 : 0;
    return PDHG_OK;
}

int pdhg_get_batch_tuning(const pdhg_ctx* ctx, int precision, int* out) {
    if (ctx == nullptr || out == nullptr ||
        (precision != PDHG_PREC_MIXED && precision != PDHG_PREC_FP64))
        return PDHG_ERR_INVALID_ARGUMENT;
    const pdhg::Ctx& cx = ctx->c;
    if (cx.batch == nullptr || pdhg::batch_count(*cx.batch) == 0) return PDHG_ERR_INVALID_ARGUMENT;
    return pdhg::batch_tuning_abi(*cx.batch, precision, out);
}

int pdhg_load_batch(pdhg_ctx* ctx, int32_t count, const int32_t* row_off, const int32_t* col_off,
                    int64_t nnz, const int32_t* row_ptr, const int32_t* col_idx,
                    const double* values, const double* c, const double* obj_const,
                    const int* maximize, const double* col_lo, const double* col_hi,
                    const double* row_lo, const double* row_hi) {
    if (ctx == nullptr) return PDHG_ERR_INVALID_ARGUMENT;
    pdhg::Ctx& cx = ctx->c;
    try {
        if (cudaSetDevice(cx.device) != cudaSuccess) return PDHG_ERR_BACKEND;
        if (cx.batch == nullptr) {
            cx.batch = pdhg::batch_new(cx.device, cx.stream, cx.err);
            if (cx.batch == nullptr) {
                cx.err = "pdhg_load_batch: cannot allocate the batch state";
                return PDHG_ERR_OUT_OF_MEMORY;
            }
        }
        return pdhg::batch_load_abi(*cx.batch, count, row_off, col_off, nnz, row_ptr, col_idx,
                                    values, c, obj_const, maximize, col_lo, col_hi, row_lo, row_hi);
    } catch (const std::exception& e) {
        cx.err = e.what();
        return PDHG_ERR_BACKEND;
    }
}

int pdhg_solve_batch(pdhg_ctx* ctx, const pdhg_options* options, pdhg_info* infos, double* x,
                     double* y, double* rc) {
    if (ctx == nullptr) return PDHG_ERR_INVALID_ARGUMENT;
    pdhg::Ctx& cx = ctx->c;
    if (cx.batch == nullptr || pdhg::batch_count(*cx.batch) == 0) {
        cx.err = "pdhg_solve_batch: no batch loaded";
        return PDHG_ERR_INVALID_ARGUMENT;
    }
    try {
        return pdhg::batch_solve_abi(*cx.batch, options, infos, x, y, rc);
    } catch (const std::exception& e) {
        cx.err = e.what();
        return PDHG_ERR_BACKEND;
    }
}

int pdhg_batch_start_kkt(pdhg_ctx* ctx, const double* x, const double* y, double* kkt) {
    if (ctx == nullptr) return PDHG_ERR_INVALID_ARGUMENT;
    pdhg::Ctx& cx = ctx->c;
    if (cx.batch == nullptr || pdhg::batch_count(*cx.batch) == 0) {
        cx.err = "pdhg_batch_start_kkt: no batch loaded";
        return PDHG_ERR_INVALID_ARGUMENT;
    }
    try {
        return pdhg::batch_point_kkt_abi(*cx.batch, x, y, kkt);
    } catch (const std::exception& e) {
        cx.err = e.what();
        return PDHG_ERR_BACKEND;
    }
}

int pdhg_csr_spmv(int device, int transpose, int32_t m, int32_t n, int64_t nnz,
                  const int32_t* row_ptr, const int32_t* col_idx, const double* values,
                  double alpha, const double* x, double beta, double* y) {
    if (m < 0 || n < 0 || nnz < 0 || nnz > std::numeric_limits<int32_t>::max() ||
        row_ptr == nullptr || y == nullptr || (nnz > 0 && (col_idx == nullptr || values == nullptr)))
        return PDHG_ERR_INVALID_ARGUMENT;
    pdhg_ctx* h = nullptr;
    int rc = pdhg_create(device, &h);
    if (rc != PDHG_OK) return rc;
    std::unique_ptr<pdhg_ctx> guard(h);
    pdhg::Ctx& c = h->c;
    rc = pdhg::upload_matrix(m, n, nnz, row_ptr, col_idx, values, c.Ao, c.ATo, c.stream, &c.err);
    if (rc != PDHG_OK) return rc;
    const int32_t nx = transpose ? m : n, ny = transpose ? n : m;
    pdhg::DBuf<double> dx, dy;
    if (pdhg::upload(dx, x, static_cast<size_t>(nx), c.stream) != cudaSuccess ||
        pdhg::upload(dy, y, static_cast<size_t>(ny), c.stream) != cudaSuccess)
        return PDHG_ERR_BACKEND;
    if (transpose)
        pdhg::launch_spmvT_exact(c.ATo.view(), alpha, dx.p, beta, dy.p, c.stream);
    else
        pdhg::launch_spmv_exact(c.Ao.view(), alpha, dx.p, beta, dy.p, c.stream);
    if (ny > 0 && cudaMemcpyAsync(y, dy.p, sizeof(double) * ny, cudaMemcpyDeviceToHost, c.stream) != cudaSuccess)
        return PDHG_ERR_BACKEND;
    if (cudaStreamSynchronize(c.stream) != cudaSuccess) return PDHG_ERR_BACKEND;
    return PDHG_OK;
}

int pdhg_project_box(int device, int32_t n, const double* lo, const double* hi, double* x) {
    if (n < 0 || (n > 0 && x == nullptr)) return PDHG_ERR_INVALID_ARGUMENT;
    pdhg_ctx* h = nullptr;
    int rc = pdhg_create(device, &h);
    if (rc != PDHG_OK) return rc;
    std::unique_ptr<pdhg_ctx> guard(h);
    pdhg::Ctx& c = h->c;
    pdhg::DBuf<double> dx, dl, dh;
    if (pdhg::upload(dx, x, static_cast<size_t>(n), c.stream) != cudaSuccess) return PDHG_ERR_BACKEND;
    if (lo != nullptr && pdhg::upload(dl, lo, static_cast<size_t>(n), c.stream) != cudaSuccess)
        return PDHG_ERR_BACKEND;
    if (hi != nullptr && pdhg::upload(dh, hi, static_cast<size_t>(n), c.stream) != cudaSuccess)
        return PDHG_ERR_BACKEND;
    pdhg::launch_project_box(n, lo ? dl.p : nullptr, hi ? dh.p : nullptr, dx.p, c.stream);
    if (n > 0 && cudaMemcpyAsync(x, dx.p, sizeof(double) * n, cudaMemcpyDeviceToHost, c.stream) != cudaSuccess)
        return PDHG_ERR_BACKEND;
    if (cudaStreamSynchronize(c.stream) != cudaSuccess) return PDHG_ERR_BACKEND;
    return PDHG_OK;
}

int pdhg_scaling(int32_t m, int32_t n, int64_t nnz, const int32_t* row_ptr,
                 const int32_t* col_idx, const double* values, const pdhg_options* options,
                 double* row_scale, double* col_scale) {
    if (m < 0 || n < 0 || nnz < 0 || row_ptr == nullptr || row_scale == nullptr ||
        col_scale == nullptr || (nnz > 0 && (col_idx == nullptr || values == nullptr)))
        return PDHG_ERR_INVALID_ARGUMENT;
    pdhg_options o;
    if (options == nullptr) pdhg_default_options(&o);
    else o = *options;
    pdhg::HostCsr A;
    A.rows = m;
    A.cols = n;
    A.rp.assign(row_ptr, row_ptr + m + 1);
    A.ci.assign(col_idx, col_idx + nnz);
    A.v.assign(values, values + nnz);
    pdhg::ScalingParams sp;
    sp.ruiz_iterations = o.ruiz_iterations;
    sp.ruiz_tolerance = o.ruiz_tolerance;
    sp.pock_chambolle_alpha = o.pock_chambolle_alpha;
    sp.apply_ruiz = o.apply_ruiz != 0;
    sp.apply_pock_chambolle = o.apply_pock_chambolle != 0;
    std::vector<double> rs, cs;
    pdhg::equilibrate(A, sp, &rs, &cs);
    std::memcpy(row_scale, rs.data(), sizeof(double) * m);
    std::memcpy(col_scale, cs.data(), sizeof(double) * n);
    return PDHG_OK;
}

}  // extern "C"
