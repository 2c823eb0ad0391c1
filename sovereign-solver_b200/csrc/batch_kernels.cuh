// batch_kernels.cuh -- device side of the batched engine (batch.cu).
//
// A batch is a block-diagonal LP: instance k owns rows [row_off[k],
// row_off[k+1]) and columns [col_off[k], col_off[k+1]) of one CSR (and of its
// device-built transpose). Each instance keeps its own PDHG state on the
// device (InstState: step sizes, primal weight, Cesaro window, restart and
// termination state), exactly the per-LP state of the single engine.
//
// Two kinds of kernels:
//   * row kernels (iterations, power-iteration products, Ruiz maxima): the
//     single engine's kernels with an instance lookup per row (row_inst /
//     col_inst) for the instance's step sizes and done flag;
//   * instance kernels: one CTA per instance (check + decision, restart,
//     norms, Ruiz update, final result), so every per-instance reduction and
//     decision is made inside one CTA without atomics or tickets.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "engine.cuh"

namespace pdhg {

struct InstState {
    int done, status, converged, fresh;
    int restart, restart_to_avg, avg_better, fold;
    int fail_kind, ruiz_done, pw_done, valid;
    int stalled, polished;  // mixed mode: FP32 phase stopped improving / finished in FP64
    long long since_restart, restarts, stop_iter;
    long long since_improve, switch_iter;
    long long idle;  // global iterations a stalled instance waited for the FP64 phase
    double best_res;
    double res_last, res_prev_cand, cur_res, avg_res, orig_res, rel_kkt, inv;
    double tau, sigma, omega, eta;
    double obj_sign, obj_const, bnorm, cnorm, cnorm2_s, bnorm2_s;
    double bnorm2, cnorm2;  // termination rule 2 norms (original, l2)
    double opnorm;
    double objective, dual_objective, gap, pinf, dinf;
};

// Values per check item: 8 maxima, 4 objective sums, 4 sums of squares of
// termination rule 2.
constexpr int kBatchCheckVals = 16;

struct BatchGlobal {
    int done;          // every instance finished (or the budget ended)
    int active;        // instances still iterating
    long long iter;    // iterations completed before the current period
    long long checks;
    int dirty;         // an instance finished (or restarted): rebuild the block lists
    int nblk[2];       // active lane-group blocks of A's rows [0] and A^T's rows [1]
};

struct BatchView {
    int32_t count = 0, m = 0, n = 0;
    const int32_t *row_off = nullptr, *col_off = nullptr;
    const int32_t *row_inst = nullptr, *col_inst = nullptr;
    DevCsr A, AT;    // scaled
    DevCsr Ao, ATo;  // original
    DevProblem P;    // vectors; obj_sign / obj_const are per instance
    InstState* is = nullptr;
    BatchGlobal* g = nullptr;
    Mailbox* mail = nullptr;
    // The check's CTA items: instance k's rows and columns in C parts, part j
    // of C = {k, j, C, -} (C by the instance's size, so that no single CTA
    // sums a large instance while the rest of the GPU waits). A CTA stores its
    // partial maxima and sums (kBatchCheckVals per item) and takes the instance's ticket;
    // the last CTA of the instance merges them in item order and decides.
    const int4* chk_item = nullptr;
    int32_t n_chk = 0;
    double* chk_part = nullptr;
    unsigned int* chk_ticket = nullptr;  // per instance, 0 between launches
    // Active block lists of the iteration kernels' lane-group path ([0] rows
    // of A, [1] rows of A^T): the blocks (kBlock / vw rows each) holding a row
    // of an instance still iterating, rebuilt by batch_compact whenever an
    // instance finishes, so that finished instances stop costing CTAs. flag is
    // the rebuild's scratch (one byte per block).
    int32_t* blk_list[2] = {nullptr, nullptr};
    unsigned char* blk_flag[2] = {nullptr, nullptr};
};

struct BatchParams {
    double tol, bound_tol, restart_decrease;
    long long period;
    int termination_rule, restart_rule, primal_weight_update;
    int allow_switch;  // FP32 phase: hand a stalled instance over to FP64
    double* x_last;
    double* y_last;
    double* act_avg;
};

// launchers (batch_kernels.cu)
template <class T>
void launch_batch_iter(const BatchView& b, const Iterates<T>& it, bool primal, int first,
                       int hk, cudaStream_t s);
template <class T>
void launch_batch_check(const BatchView& b, const Iterates<T>& it, const BatchParams& p,
                        cudaStream_t s);
template <class T>
void launch_batch_restart(const BatchView& b, const Iterates<T>& it, const BatchParams& p,
                          cudaStream_t s);
void launch_batch_tick(const BatchView& b, long long period, long long budget_iters,
                       cudaGraphConditionalHandle handle, int use_handle, cudaStream_t s);
// Rebuilds the active block lists when g->dirty is set (one CTA; a no-op otherwise).
void launch_batch_compact(const BatchView& b, cudaStream_t s);
void launch_batch_fill_inst(const int32_t* off, int32_t count, int32_t* out, cudaStream_t s);
void launch_batch_warm(const BatchView& b, double* x0, double* y0, cudaStream_t s);

// power iteration per instance (estimate_operator_norm, pdhg.cpp:48-79)
void launch_batch_pw_w(const BatchView& b, const double* u, const double* v, double* w,
                       cudaStream_t s);
void launch_batch_pw_norm_w(const BatchView& b, double* w, cudaStream_t s);
void launch_batch_pw_u(const BatchView& b, const double* w, double* u, cudaStream_t s);
void launch_batch_pw_norm_uv(const BatchView& b, const double* w, double* u, double* v,
                             cudaStream_t s);
void launch_batch_steps(const BatchView& b, double safety, int primal_weight, cudaStream_t s);

// intake per instance (Scaling::equilibrate, scaling.cpp:19-104)
void launch_batch_ruiz_max(const BatchView& b, const DevCsr& M, int transposed, const double* rs,
                           const double* cs, double* out, cudaStream_t s);
void launch_batch_ruiz_update(const BatchView& b, double* rs, double* cs, const double* row_max,
                              const double* col_max, double tol, cudaStream_t s);
void launch_batch_scale_vectors(const BatchView& b, double* c_s, double* lo_s, double* hi_s,
                                double* rlo_s, double* rhi_s, cudaStream_t s);
void launch_batch_norms(const BatchView& b, cudaStream_t s);

// PDLP-style relative KKT residual of a given point per instance (original
// units and sense; a null x or y is the zero vector).
void launch_batch_point_kkt(const BatchView& b, const double* x, const double* y, double* out,
                            cudaStream_t s);

// Internal status of an instance whose FP32 phase stalled (mixed mode).
constexpr int kBatchStalled = 100;

// FP32 iterates widened into the FP64 ones (the polish phase starts there).
void launch_batch_widen(const BatchView& b, const Iterates<float>& f, const Iterates<double>& d,
                        cudaStream_t s);

// final result per instance (pdhg.cpp:420-498); `which`: -1 every instance,
// 0 those not polished, 1 the polished ones.
template <class T>
void launch_batch_final(const BatchView& b, const Iterates<T>& it, double bound_tol,
                        double* xo, double* yo, double* rc, int which, cudaStream_t s);

}  // namespace pdhg
