/*
 * pdhg_oracle.h -- TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C, single-threaded restatement of the reference PDHG path
 * (AtharvPhutela/sovereign-solver: src/l1/pdhg.cpp, src/l1/scaling.cpp,
 * src/l1/duals.cpp, src/l0/sparse.cpp, src/l0/backend_host.cpp,
 * src/io/problem.cpp). It exists to CHECK the CUDA engine: only tests/,
 * __graft_entry__.smoke() and bench.py's CPU-baseline leg may load it. The
 * product never links or calls it.
 *
 * Parity status: pinned. tests/test_oracle_pin.py runs this restatement and
 * the reference itself (oracle/_ref, compiled from the reference sources by
 * oracle/Makefile) on the same inputs and requires bit-identical results;
 * tests/golden/ holds fixtures produced by the reference for the GPU box,
 * where the reference sources are absent.
 *
 * Arithmetic is IEEE double, compiled with -ffp-contract=off so that no
 * multiply-add is fused: the reference's Release build (g++ -O3, generic
 * x86-64, no -march) never emits FMA either.
 */
#ifndef PDHG_ORACLE_H
#define PDHG_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes: the order of sov::PdhgStatus (include/sovereign/pdhg.hpp:74-81). */
enum {
    ORC_OPTIMAL = 0,
    ORC_ITERATION_LIMIT = 1,
    ORC_TIME_LIMIT = 2,
    ORC_NUMERICAL_FAILURE = 3,
    ORC_NOT_SOLVED = 4,
    ORC_CANCELLED = 5
};

/* An LP in the reference's canonical form (include/sovereign/problem.hpp:5-8):
 *   optimize c^T x + obj_const  s.t.  row_lo <= A x <= row_hi,  col_lo <= x <= col_hi
 * A is CSR with int32 indices (Idx = int32_t, include/sovereign/numeric.hpp:65-71).
 * Infinite bounds are +-INFINITY. */
typedef struct {
    int32_t m, n;
    int64_t nnz;
    const int32_t* row_ptr;
    const int32_t* col_idx;
    const double* val;
    const double* c;
    double obj_const;
    int maximize;
    const double* col_lo;
    const double* col_hi;
    const double* row_lo;
    const double* row_hi;
} orc_problem;

typedef void (*orc_checkpoint_fn)(void* user, long long iteration, const double* x,
                                  const double* y, double original_residual);

/* sov::PdhgOptions (include/sovereign/pdhg.hpp:85-134) + sov::ScalingOptions
 * (include/sovereign/scaling.hpp:296-310), plus extensions that are OFF by
 * default (the reference has none of them):
 *   termination_rule  0 = reference absolute original-space residual < tol,
 *                     1 = relative KKT on the reference's max-norm residual
 *                         terms (original_residual in pdhg_oracle.c),
 *                     2 = PDLP's relative KKT with l2 norms (pdlp_kkt in
 *                         pdhg_oracle.c): max(||row violation||/(1+||b||),
 *                         ||dual sign violation||/(1+||c||), gap) < tol;
 *   trace_iters       record x, y after each of the first trace_iters iterations. */
typedef struct {
    double tolerance;
    long long max_iterations;
    double time_limit_seconds;
    long long restart_check_period;
    double restart_sufficient_decrease;
    double step_size_safety;
    int power_iterations;
    int verbose;
    /* scaling */
    int ruiz_iterations;
    double ruiz_tolerance;
    double pock_chambolle_alpha;
    int apply_ruiz;
    int apply_pock_chambolle;
    /* extensions */
    int termination_rule;
    int trace_iters;
    double* trace_x; /* trace_iters * n */
    double* trace_y; /* trace_iters * m */
    orc_checkpoint_fn checkpoint;
    void* checkpoint_user;
    const volatile int* cancel_flag;
    /* monotonic seconds at the start of each of the first iter_times_cap
     * iterations (CPU-baseline timing without the setup) */
    double* iter_times;
    long long iter_times_cap;
    /* restart_rule 1 (adaptive) and primal_weight_update 1: the engine's
     * extensions, restated here so its FP64 mode has a CPU check:
     * restart to the better of average/current when its residual is
     * <= 0.2x the residual at the last restart, or <= 0.8x without progress
     * since the previous check, or when the average spans >= 36% of all
     * iterations; at each restart omega <- sqrt(omega |dy|/|dx|) (distances
     * between consecutive restart points, scaled space), tau = eta/omega,
     * sigma = eta*omega, omega0 = |c|_2/|b|_2 (scaled; b_i = largest finite
     * |row bound|). */
    int restart_rule;
    int primal_weight_update;
    /* halpern 1 (needs termination_rule 2 and restart_rule 2): the reflected
     * Halpern iteration (Lu and Yang, "Restarted Halpern PDHG for linear
     * programming", 2024): with T the PDHG step above and k the iterations
     * since the last restart, z <- (k+1)/(k+2) (2 T(z) - z) + 1/(k+2) z_a for
     * z = (x, s, y) and the anchor z_a = the last restart point. Candidates
     * are T(z) (inside the column bounds; z itself need not be); a restart
     * moves z and the anchor to T(z) (s to the row bounds' projection of A x). */
    int halpern;
    /* warm start (the engine's x0 / y0 options), original units and sense:
     * x = proj_X(x0 / col_scale), y = y0 obj_sign / row_scale,
     * s = proj_S(A_scaled x); NULL = the reference's start (pdhg.cpp:268-283) */
    const double* x0;
    const double* y0;
    /* primal_weight_update: the starting primal weight (scaled space);
     * 0 = |c|_2 / |b|_2 */
    double primal_weight0;
} orc_options;

typedef struct {
    int status;
    double objective;
    double primal_infeasibility;
    double dual_infeasibility;
    double duality_gap;
    long long iterations;
    long long restarts;
    double seconds;
    double operator_norm_estimate;
    int has_point; /* 0 when the reference returns empty primal/dual vectors */
    char message[256];
    /* extension: the relative-KKT value (termination_rule 1 or 2) of the last
     * check's candidate; 0 under rule 0 and in the reference */
    double relative_kkt;
    /* extension: the primal weight at the end (1 without primal_weight_update) */
    double primal_weight;
} orc_info;

void orc_default_options(orc_options* opt);
const char* orc_status_string(int status);

/* Pdhg::solve (src/l1/pdhg.cpp:218-502). x (n), y (m), rc (n) are written only
 * when info->has_point is set. Returns 0. */
int orc_pdhg_solve(const orc_problem* p, const orc_options* opt, orc_info* info,
                   double* x, double* y, double* rc);

/* Scaling::equilibrate(CsrMatrix) (src/l1/scaling.cpp:19-104). */
void orc_scaling(int32_t m, int32_t n, const int32_t* row_ptr, const int32_t* col_idx,
                 const double* val, const orc_options* opt, double* row_scale,
                 double* col_scale);

/* Host backend primitives (src/l0/backend_host.cpp:409-458). */
void orc_spmv(int32_t m, const int32_t* row_ptr, const int32_t* col_idx, const double* val,
              double alpha, const double* x, double beta, double* y);
void orc_spmv_transpose(int32_t m, int32_t n, const int32_t* row_ptr, const int32_t* col_idx,
                        const double* val, double alpha, const double* x, double beta,
                        double* y);
void orc_project_box(int32_t n, const double* lo, const double* hi, double* x);
double orc_pairwise_dot(const double* x, const double* y, int64_t n);

/* FarkasCertificate{y}.certifies_infeasibility(problem, slack)
 * (src/l1/duals.cpp:16-79): the row-side range of S = sum_i y_i (Ax)_i forced
 * by the row bounds, the column-side range forced by the column bounds through
 * d = A^T y, and whether they are disjoint by more than `slack`. ranges (4,
 * optional) = row lo, row hi, column lo, column hi. Returns 1 or 0. */
int orc_certifies(const orc_problem* p, const double* y, double slack, double* ranges);

/* The power iteration of estimate_operator_norm (src/l1/pdhg.cpp:48-79) on a
 * CSR matrix as given. */
double orc_operator_norm(int32_t m, int32_t n, const int32_t* row_ptr, const int32_t* col_idx,
                         const double* val, int iterations);

#ifdef __cplusplus
}
#endif
#endif
