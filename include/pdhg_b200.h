/*
 * pdhg_b200.h -- C-ABI of the B200-native PDHG LP engine (libpdhg_b200.so).
 *
 * Drop-in for the reference's PDHG engine, sov::Pdhg::solve
 * (AtharvPhutela/sovereign-solver: include/sovereign/pdhg.hpp:155-172,
 * src/l1/pdhg.cpp:218-502). The reference has no FFI of its own; this is the
 * plain-C surface its C++ call sites (apps/sovereign_cli.cpp:196-236,
 * src/l1/race.cpp:123-129, src/l1/crossover.cpp:192-237) would bind. Only POD
 * types cross it, no exception crosses it, and every entry returns a
 * pdhg_error code that mirrors sov::Status (include/sovereign/status.hpp:25-34).
 *
 * Units and sense: everything that crosses the ABI is in the ORIGINAL problem's
 * units and objective sense, exactly like sov::PdhgResult. Scaling (Ruiz +
 * Pock-Chambolle, src/l1/scaling.cpp:155-205) happens inside the engine.
 *
 * Threading: a context is not thread-safe, like sov::Backend (one per thread,
 * src/l1/race.cpp:126). pdhg_solve is synchronous on the caller's thread; the
 * checkpoint callback runs on that thread.
 */
#ifndef PDHG_B200_H
#define PDHG_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PDHG_B200_ABI_VERSION 4

/* Return codes: the order and meaning of sov::Status (status.hpp:25-34). */
typedef enum {
    PDHG_OK = 0,
    PDHG_ERR_UNSUPPORTED = 1,
    PDHG_ERR_NOT_IMPLEMENTED = 2,
    PDHG_ERR_INVALID_ARGUMENT = 3,
    PDHG_ERR_DIMENSION_MISMATCH = 4,
    PDHG_ERR_OUT_OF_MEMORY = 5,
    PDHG_ERR_BACKEND = 6, /* the CUDA runtime reported a failure */
    PDHG_ERR_NUMERICAL_FAILURE = 7
} pdhg_error;

/* Solve outcomes: sov::PdhgStatus (include/sovereign/pdhg.hpp:74-81). */
typedef enum {
    PDHG_STATUS_OPTIMAL = 0,
    PDHG_STATUS_ITERATION_LIMIT = 1,
    PDHG_STATUS_TIME_LIMIT = 2,
    PDHG_STATUS_NUMERICAL_FAILURE = 3,
    PDHG_STATUS_NOT_SOLVED = 4,
    PDHG_STATUS_CANCELLED = 5,
    /* engine extension (option infeasibility_detection): a certificate proves
     * that no x meets the row and column bounds; pdhg_solve writes its row
     * multipliers to y (the reference's FarkasCertificate, duals.hpp:47-70,
     * which the reference's PDHG never produces: its verdict there stays
     * iteration_limit) */
    PDHG_STATUS_PRIMAL_INFEASIBLE = 6,
    /* engine extension (option infeasibility_detection): a ray d in x proves
     * that the dual has no solution, so the LP is unbounded if it is feasible
     * (the reference's simplex names this outcome Unbounded, simplex.hpp:42);
     * pdhg_solve writes the ray to x */
    PDHG_STATUS_DUAL_INFEASIBLE = 7
} pdhg_status;

/* Arithmetic of the iteration kernels. */
typedef enum {
    /* FP64, each sum accumulated in the reference's own order with no fused
     * multiply-add: iterates, restarts, statuses and results are bit-identical
     * to the reference's Host backend (src/l0/backend_host.cpp). */
    PDHG_PREC_FP64_EXACT = 0,
    /* FP32 matrix values and iterates in the per-iteration kernels; FP64 for
     * the KKT residuals, the restart decision, the objective and the result. */
    PDHG_PREC_MIXED = 1,
    /* FP64 everywhere, warp-parallel sums (not in the reference's order). */
    PDHG_PREC_FP64 = 2
} pdhg_precision;

/* Checkpoint (pdhg.hpp:121-134): at every check, on the solving thread, the
 * candidate in original units and its original-space residual. x_original and
 * y_original are valid only during the call (the engine reuses the buffers).
 * While the callback runs the GPU already works on the next check period; a
 * stop request (cancellation, time limit) is honoured at the check after it. */
typedef void (*pdhg_checkpoint_fn)(void* user, long long iteration, const double* x_original,
                                   const double* y_original, double original_residual);

/* sov::PdhgOptions (pdhg.hpp:85-134) + sov::ScalingOptions (scaling.hpp:296-310)
 * + engine extensions. pdhg_default_options() gives the reference defaults
 * with every extension off. */
typedef struct pdhg_options {
    double tolerance;                   /* 1e-4 */
    long long max_iterations;           /* 1000000 */
    double time_limit_seconds;          /* 0 = none */
    long long restart_check_period;     /* 40 */
    double restart_sufficient_decrease; /* 0.5 */
    double step_size_safety;            /* 0.9 */
    int power_iterations;               /* 30 */
    int verbose;                        /* restart lines on stderr, as pdhg.cpp:405-407 */
    /* Ruiz + Pock-Chambolle (scaling.hpp:296-310) */
    int ruiz_iterations;          /* 8 */
    double ruiz_tolerance;        /* 1e-2 */
    double pock_chambolle_alpha;  /* 1.0 */
    int apply_ruiz;               /* 1 */
    int apply_pock_chambolle;     /* 1 */
    /* extensions (off = reference behaviour) */
    int precision;           /* pdhg_precision; default PDHG_PREC_FP64_EXACT */
    int termination_rule;    /* 0 = reference absolute residual (pdhg.cpp:383);
                                1 = relative KKT on the reference's residual terms:
                                    max(primal/(1+|b|inf), dual/(1+|c|inf), gap), primal and
                                    dual the max-norm terms of pdhg.cpp:166-197;
                                2 = PDLP's relative KKT error (MIXED / FP64):
                                    max(|row violation|_2/(1+|b|_2),
                                        |sign violations of y and c - A^T y|_2/(1+|c|_2), gap),
                                    b_i the larger finite |row bound|; the gap of rules 1 and 2
                                    is |p - d|/(1 + |p| + |d|) on the bounded dual objective */
    long long polish_iterations; /* MIXED only: FP64 iterations allowed after the FP32
                                    phase stalls (no 2% gain in 25 checks; under
                                    termination_rule 2 only below 1024 FP32 ulps, 1.2e-4);
                                    -1 = the rest of max_iterations, 0 = never leave FP32 */
    int restart_rule;        /* 0 = reference (pdhg.cpp:391-408); 1 = adaptive: restart to
                                the better of average/current on sufficient (0.2x) or
                                necessary (0.8x, no progress) decay or when the average
                                spans 36% of all iterations, residuals measured by the
                                scaled max-norm KKT residual (pdhg.cpp:87-136); 2 = the same
                                rule measured by the l2 norm of termination rule 2's three
                                parts (needs termination_rule 2). 1, 2 need MIXED or FP64. */
    int primal_weight_update; /* 0 = reference tau = sigma (pdhg.cpp:263-265); 1 = primal
                                weight omega (tau = eta/omega, sigma = eta*omega) starts at
                                |c|/|b| and moves to sqrt(omega |dy|/|dx|) at each restart */
    const double* x0;        /* optional warm start, original units (n); NULL = proj(0) */
    const double* y0;        /* optional warm start, original units and sense (m); NULL = 0 */
    pdhg_checkpoint_fn checkpoint; /* pdhg.hpp:121-134; NULL = none */
    void* checkpoint_user;
    const volatile int* cancel_flag; /* CancellationToken (cancellation.hpp:23-30); NULL = none */
    int trace_iters;         /* record scaled-space x, y after each of the first trace_iters */
    double* trace_x;         /* iterations: trace_iters * n, host (test support) */
    double* trace_y;         /* trace_iters * m, host */
    int autotune;            /* 1 (default): MIXED / FP64 time the iteration kernels' shapes
                                on the first solve of a loaded LP with >= 2^20 nonzeros and
                                keep the fastest (see pdhg_get_tuning); 0 = fixed defaults */
    int infeasibility_detection; /* 0 (default) = reference behaviour. 1 (MIXED / FP64): at
                                every check the change of y since the previous check (original
                                units) is tested as a FarkasCertificate (duals.cpp:36-79): when
                                the ranges the row bounds and the column bounds force on
                                sum_i y_i (Ax)_i are disjoint by more than 1e-6 relative, the
                                solve stops with PDHG_STATUS_PRIMAL_INFEASIBLE and y receives
                                the multipliers, scaled to max |y_i| = 1. Else the change of x,
                                scaled to d with max |d_j| = 1, is tested as a ray: when the
                                objective falls along it (c^T d < 0 in the minimize sense) and
                                it leaves the recession cones of the column and row bounds (a
                                finite lower end allows no decrease of x_j or (Ad)_i, a finite
                                upper end no increase) by at most 1e-6 and 1e-6 |c^T d|, the
                                solve stops with PDHG_STATUS_DUAL_INFEASIBLE and x receives d */
    int halpern;             /* 0 (default) = the averaged PDHG of the reference. 1 (MIXED / FP64,
                                with termination_rule 2 and restart_rule 2; not with
                                infeasibility_detection): the reflected restarted Halpern
                                iteration (Lu and Yang, 2024) -- with T the PDHG step and k the
                                iterations since the last restart, z <- (k+1)/(k+2) (2 T(z) - z)
                                + 1/(k+2) z_a for z = (x, s, y) and the anchor z_a = the last
                                restart point; candidates and the reported point are T(z) */
} pdhg_options;

/* sov::PdhgResult (pdhg.hpp:136-153) minus the vectors, which pdhg_solve
 * writes into caller-owned buffers. */
typedef struct pdhg_info {
    int status;                    /* pdhg_status */
    double objective;
    double primal_infeasibility;
    double dual_infeasibility;
    double duality_gap;
    long long iterations;
    long long restarts;
    double seconds;
    double operator_norm_estimate;
    int has_point;                 /* 0 where the reference returns empty vectors */
    char message[256];
    /* engine extensions */
    double relative_kkt;           /* the relative-KKT value of the reported point */
    long long fp64_iterations;     /* iterations run by FP64 kernels (MIXED: the polish) */
    long long kernel_launches;     /* engine kernels launched by this solve */
    double device_seconds;         /* iteration-loop time measured with CUDA events */
} pdhg_info;

typedef struct pdhg_ctx pdhg_ctx;

int pdhg_abi_version(void);
void pdhg_default_options(pdhg_options* options);
const char* pdhg_status_string(int status);      /* to_string(PdhgStatus), pdhg.cpp:17-27 */
const char* pdhg_error_string(int error);        /* to_string(Status), status.hpp:36-48 */

/* One context per device and thread (replaces make_backend, backend.hpp:172-184). */
int pdhg_create(int device, pdhg_ctx** out);
int pdhg_destroy(pdhg_ctx* ctx);
/* Text of the last error on this context ("" if none). */
const char* pdhg_last_error(const pdhg_ctx* ctx);
/* The cudaStream_t every kernel of this context is launched on (for callers
 * that time or order work against it); NULL for a NULL context. */
void* pdhg_stream(const pdhg_ctx* ctx);

/* Hands the engine an LP (host buffers, copied). Replaces the Problem handed to
 * Pdhg::solve plus DeviceCsr::upload (src/l0/backend.cpp:154-188): validation,
 * scaling, the device CSR of A and the device-built CSR of A^T happen here.
 * An invalid problem is NOT an error here: like the reference (pdhg.cpp:223-228)
 * pdhg_solve then reports PDHG_STATUS_NUMERICAL_FAILURE "invalid problem: ...".
 * Sizes that do not fit int32 indices return PDHG_ERR_INVALID_ARGUMENT. */
int pdhg_load_problem(pdhg_ctx* ctx, int32_t m, int32_t n, int64_t nnz, const int32_t* row_ptr,
                      const int32_t* col_idx, const double* values, const double* c,
                      double obj_const, int maximize, const double* col_lo,
                      const double* col_hi, const double* row_lo, const double* row_hi);

/* Pdhg::solve (pdhg.cpp:218-502) on the loaded problem. x (n), y (m) and rc (n)
 * are caller-owned HOST buffers in original units (any may be NULL); they are
 * written only when info->has_point is set. */
int pdhg_solve(pdhg_ctx* ctx, const pdhg_options* options, pdhg_info* info, double* x,
               double* y, double* rc);

/* Batched extension: `count` independent LPs solved together, each exactly as
 * its own Pdhg::solve would (pdhg.cpp:218-502; the reference runs one per
 * thread, race.cpp:126) -- own scaling, step sizes, restarts, termination and
 * result -- in one device loop. The instances are stacked block-diagonally:
 * instance k owns rows [row_off[k], row_off[k+1]) and columns
 * [col_off[k], col_off[k+1]) of one CSR (row_ptr over all rows, col_idx global,
 * each row's columns inside its instance's range); c, col_lo, col_hi (n) and
 * row_lo, row_hi (m) are stacked the same way; obj_const and maximize have one
 * entry per instance. Validation is per instance (problem.cpp:50-,
 * sparse.cpp:94-128): an invalid instance gets PDHG_STATUS_NUMERICAL_FAILURE
 * "invalid problem: ..." in its info and the others solve. Structure the
 * stacking cannot hold (offsets, a column outside the instance) returns
 * PDHG_ERR_INVALID_ARGUMENT. Precision MIXED or FP64 only; no checkpoint and
 * no trace. x, y, rc are stacked like the inputs (any may be NULL); infos has
 * `count` entries. A loaded batch stays on the context beside the single LP. */
int pdhg_load_batch(pdhg_ctx* ctx, int32_t count, const int32_t* row_off,
                    const int32_t* col_off, int64_t nnz, const int32_t* row_ptr,
                    const int32_t* col_idx, const double* values, const double* c,
                    const double* obj_const, const int* maximize, const double* col_lo,
                    const double* col_hi, const double* row_lo, const double* row_hi);
int pdhg_solve_batch(pdhg_ctx* ctx, const pdhg_options* options, pdhg_info* infos, double* x,
                     double* y, double* rc);
/* Relative KKT residual of candidate starting points for the loaded batch,
 * one value per instance: x (n) and y (m) stacked like pdhg_solve_batch's
 * outputs, original units and sense, NULL = zero vector (the cold start).
 * PDLP's measure with l2 norms -- max(||primal bound violation of A clamp(x)||
 * / (1 + ||b||), ||dual sign violations|| / (1 + ||c||), objective gap) -- so a
 * point near the optimum scores near 0 even where it is not exactly at its
 * bounds. Engine extension for the learned warm start, which keeps a
 * predicted start only where it beats the cold start on this measure (the
 * reference has no warm start: pdhg.cpp:268-270). */
int pdhg_batch_start_kkt(pdhg_ctx* ctx, const double* x, const double* y, double* kkt);

/* Iteration-kernel shapes in use for the loaded problem in `precision`
 * (PDHG_PREC_MIXED or PDHG_PREC_FP64): out[0] lanes per short row and out[1]
 * long-row strategy (0: a warp per row up to 512 entries, CTA work items
 * above; 1: a warp per row up to 4,096 entries, CTA items above; 2: warp work
 * items for every row past the short ones; rows longer than a work item are
 * split into segments; plus 4 when row slices -- lane-interleaved copies of
 * runs of 32 equal-length rows whose gathers coalesce across rows -- take
 * their rows) of the primal pass (rows of A^T), out[2], out[3] the same for the
 * dual pass (rows of A), out[4] = 1 when chosen by timing, 0 for the defaults
 * (no solve yet, autotune off, or a small LP). Engine extension: the autotuner
 * times the candidates once per matrix shape and precision, and keeps the
 * choice in memory, and also in the JSON file named by the environment
 * variable PDHG_B200_TUNE_CACHE when it is set. */
int pdhg_get_tuning(const pdhg_ctx* ctx, int precision, int* out);

/* Lanes per row of the batched engine's iteration kernels for the loaded
 * batch in `precision` (PDHG_PREC_MIXED or PDHG_PREC_FP64): out[0] the primal
 * pass (rows of A^T), out[1] the dual pass (rows of A), out[2] = 1 when chosen
 * by timing. Engine extension: on the first pdhg_solve_batch of a loaded batch
 * with >= 2^20 nonzeros (option autotune on) each pass's width is timed at the
 * binning's choice, half and twice it, and the fastest kept until the next
 * load; smaller batches and autotune = 0 keep the binning's choice. */
int pdhg_get_batch_tuning(const pdhg_ctx* ctx, int precision, int* out);

/* Per-kernel timing of the iteration kernels on the loaded problem (CUDA events
 * on the engine's stream around each launch, after `warmup` untimed iterations).
 * Runs `iterations` iterations from the cold start, in the form the last
 * pdhg_solve ran: the averaged iteration, or (option halpern) the Halpern
 * iteration without its once-a-period stores; then one check. bytes[] are the
 * algorithmic bytes of that form. */
typedef struct pdhg_kernel_stats {
    int count;                   /* kernels reported */
    char name[8][32];
    double avg_ms[8];            /* mean launch duration */
    double bytes[8];             /* algorithmic bytes per launch */
    int launches[8];
} pdhg_kernel_stats;
int pdhg_profile_kernels(pdhg_ctx* ctx, int precision, int warmup, int iterations,
                         pdhg_kernel_stats* out);

/* Backend primitives on the engine's kernels (FP64 exact order), host buffers:
 * y := alpha*op(A)*x + beta*y (Backend::spmv / spmv_transpose, backend.hpp:120-126;
 * beta == 0 overwrites y, backend_host.cpp:420-422) and x := clamp(x, lo, hi)
 * with NULL = unbounded side (Backend::project_box, backend.hpp:131). */
int pdhg_csr_spmv(int device, int transpose, int32_t m, int32_t n, int64_t nnz,
                  const int32_t* row_ptr, const int32_t* col_idx, const double* values,
                  double alpha, const double* x, double beta, double* y);
int pdhg_project_box(int device, int32_t n, const double* lo, const double* hi, double* x);

/* pdhg_csr_spmv for callers that cannot allocate device memory. This entry has
 * no counterpart in the reference; it exists for code that must not call
 * cudaMalloc or any allocating routine where it needs the product: frameworks
 * that own every device byte through their own pool (an allocation behind the
 * pool's back can fail or fragment it), latency-critical loops that must stay
 * away from the driver's allocator (an allocation can synchronise the device).
 * Every pointer is a DEVICE pointer the caller owns (d_x and d_y may be NULL
 * when their length is 0); the work is queued on `stream` (a cudaStream_t,
 * NULL = default stream) on the current device and the call returns without
 * waiting. Results are bit-identical to pdhg_csr_spmv's, duplicate
 * (row, column) entries included.
 * The CSR must be well formed: d_row_ptr[0] = 0, d_row_ptr[m] = nnz, no row
 * pointer decreasing, every column index in [0, n). The call cannot check this
 * on the host (the arrays live on the device); its kernels check it first, and
 * a CSR that breaks it fills every entry of y with NaN and touches nothing
 * outside the caller's buffers (pdhg_csr_spmv returns
 * PDHG_ERR_INVALID_ARGUMENT for the same input).
 * The transposed product needs A^T: it is built in a fixed scratch array that
 * every GPU loading this library reserves until exit (about 6 MB; the check
 * above keeps its flag there too). Limits for transpose != 0: n <= 262,144
 * columns and nnz <= 262,144 nonzeros; larger sizes return
 * PDHG_ERR_INVALID_ARGUMENT before any work is queued (transpose == 0 has no
 * limit). The first call on a device looks up the scratch address for that
 * device: make it before any stream capture. All calls share the one array,
 * so calls that overlap on the GPU (different streams, no ordering between
 * them) race; serialise them. */
int pdhg_csr_spmv_noalloc(int transpose, int32_t m, int32_t n, int64_t nnz,
                          const int32_t* d_row_ptr, const int32_t* d_col_idx,
                          const double* d_values, double alpha, const double* d_x, double beta,
                          double* d_y, void* stream);

/* Learned warm start: the network that maps an LP family's parameters to
 * solution-basis coefficients. No counterpart in the reference (its PDHG has
 * no warm start, pdhg.cpp:268-270 starts from proj(0), 0); the engine uses
 * the prediction through pdhg_options.x0 / y0. A 2-hidden-layer ReLU MLP
 * (n_in -> hidden -> hidden -> n_out, all multiples of 8) whose products run
 * on the tensor cores (tcgen05, BF16 operands, FP32 accumulation) and whose
 * training is Adam on FP32 master weights. Parameter order everywhere:
 * W1 (hidden x n_in, row-major), b1, W2 (hidden x hidden), b2,
 * W3 (n_out x hidden), b3. Batches are multiples of 8 up to max_batch; all
 * buffers are host FP32. */
typedef struct pdhg_mlp pdhg_mlp;
int pdhg_mlp_create(int device, int n_in, int hidden, int n_out, int max_batch, pdhg_mlp** out);
int pdhg_mlp_destroy(pdhg_mlp* mlp);
const char* pdhg_mlp_last_error(const pdhg_mlp* mlp);
int64_t pdhg_mlp_param_count(const pdhg_mlp* mlp);
int pdhg_mlp_set_params(pdhg_mlp* mlp, const float* params); /* also resets Adam */
int pdhg_mlp_get_params(pdhg_mlp* mlp, float* params);
/* y (batch x n_out) = network(x (batch x n_in)) */
int pdhg_mlp_forward(pdhg_mlp* mlp, int batch, const float* x, float* y);
/* One forward + backward: gradients of L = sum (y - t)^2 / (batch n_out)
 * in parameter order, and L itself. */
int pdhg_mlp_gradients(pdhg_mlp* mlp, int batch, const float* x, const float* t,
                       float* grads, float* loss);
/* Adam over `epochs` shuffled passes of `samples` rows of x / t (seeded),
 * mini-batches of `batch`; epoch_loss (epochs entries, may be NULL) gets each
 * epoch's mean loss. */
int pdhg_mlp_train(pdhg_mlp* mlp, int64_t samples, const float* x, const float* t, int epochs,
                   int batch, float lr, uint64_t seed, float* epoch_loss);
/* One Adam step (the hyper-parameters and step counter of pdhg_mlp_train)
 * with caller-supplied gradients in parameter order: the update of
 * data-parallel training, where each replica applies the gradients of
 * pdhg_mlp_gradients averaged over all ranks (one allreduce), so every
 * replica keeps the same parameters. */
int pdhg_mlp_adam_step(pdhg_mlp* mlp, const float* grads, float lr);
/* The network's tensor-core GEMM alone (engine extension, for tests):
 * c (m x n) = a (m x k) b (n x k)^T (+ bias (n), ReLU), operands rounded to
 * BF16, FP32 accumulation; k a multiple of 8; host FP32 buffers. */
int pdhg_gemm_bf16(int device, int m, int n, int k, const float* a, const float* b,
                   const float* bias, int relu, float* c);

/* Scaling::equilibrate(CsrMatrix) (src/l1/scaling.cpp:19-104) on the host
 * (FP64, the reference's order), for callers without a device. */
int pdhg_scaling(int32_t m, int32_t n, int64_t nnz, const int32_t* row_ptr,
                 const int32_t* col_idx, const double* values, const pdhg_options* options,
                 double* row_scale, double* col_scale);

/* The row / column factors the engine computed on the device for the loaded
 * problem (Scaling::row_scale / col_scale, scaling.hpp:332-333), bit-identical
 * to pdhg_scaling's. Host buffers of m and n doubles. */
int pdhg_get_scaling(pdhg_ctx* ctx, double* row_scale, double* col_scale);

/* ---- MPS reader ----------------------------------------------------------
 * sov::read_mps_string / sov::read_mps (include/sovereign/io.hpp:57-59,
 * src/io/mps_reader.cpp): the same dialect, the same model (rows and columns
 * in file order, the CSR of Problem::Builder::finish with duplicates summed
 * and zeros dropped, bounds, integrality, names), the same warnings and
 * error messages, the same fixed-column retry. Host only (no device). */

/* sov::MpsOptions (io.hpp:46-54) + threads. */
typedef struct pdhg_mps_options {
    int negative_upper_bound; /* 0 (default) = LowerBecomesMinusInfinity, 1 = KeepLowerAtZero */
    int keep_free_rows;       /* 1 (default) = non-objective N rows stay as free rows */
    int threads;              /* host threads; 0 (default) = all hardware threads */
} pdhg_mps_options;

typedef struct pdhg_model pdhg_model; /* sov::ReadResult (io.hpp:29-33) */

typedef struct pdhg_model_info {
    int32_t m, n;
    int64_t nnz;
    double obj_const;   /* Problem::objective_constant */
    int maximize;       /* Problem::sense */
    int32_t warnings;   /* ReadResult::warnings.size() */
    int fixed_format;   /* 1 when the free-form read failed and the fixed-column one succeeded */
} pdhg_model_info;

/* MpsOptions{} (io.hpp:46-54): the defaults above. */
void pdhg_default_mps_options(pdhg_mps_options* options);

/* read_mps_string(text, options, origin) (io.hpp:58-59, mps_reader.cpp:538-564):
 * MPS text of len bytes (need not be NUL-terminated); origin names it in
 * messages (NULL = "<string>"). On a malformed model: PDHG_ERR_INVALID_ARGUMENT,
 * *out = NULL and err (err_cap bytes, may be NULL) gets the reference's
 * sov::Error message. */
int pdhg_read_mps(const char* text, size_t len, const char* origin,
                  const pdhg_mps_options* options, pdhg_model** out, char* err, size_t err_cap);
/* read_mps(path, options) (io.hpp:57, mps_reader.cpp:566-572): the file's bytes
 * as they are (no decompression, like the reference), origin = path;
 * "cannot open '<path>'" when it cannot be read. */
int pdhg_read_mps_file(const char* path, const pdhg_mps_options* options, pdhg_model** out,
                       char* err, size_t err_cap);
/* Frees a model (the ReadResult, io.hpp:29-33). */
void pdhg_model_free(pdhg_model* model);
/* Problem::num_rows / num_cols / num_nonzeros / objective_constant / sense
 * (problem.hpp:52-64) and ReadResult::warnings.size() (io.hpp:31). */
int pdhg_model_get_info(const pdhg_model* model, pdhg_model_info* info);
/* Problem::matrix / objective / row and column bounds / col_kind
 * (problem.hpp:56-78), as pointers into the model (valid until
 * pdhg_model_free), any may be NULL: CSR (m + 1, nnz, nnz), c (n), bounds
 * (n, n, m, m), is_integer (n, 0 / 1). They go straight into pdhg_load_problem. */
int pdhg_model_arrays(const pdhg_model* model, const int32_t** row_ptr, const int32_t** col_idx,
                      const double** values, const double** c, const double** col_lo,
                      const double** col_hi, const double** row_lo, const double** row_hi,
                      const uint8_t** is_integer);
/* Problem::name (problem.hpp:83): the NAME card. */
const char* pdhg_model_name(const pdhg_model* model);
/* Problem::objective_name (problem.hpp:84): the first N row. */
const char* pdhg_model_objective_name(const pdhg_model* model);
/* Problem::row_names()[i] (problem.hpp:85); NULL when out of range. */
const char* pdhg_model_row_name(const pdhg_model* model, int32_t i);
/* Problem::col_names()[j] (problem.hpp:86); NULL when out of range. */
const char* pdhg_model_col_name(const pdhg_model* model, int32_t j);
/* Problem::row_names / col_names (problem.hpp:85-86) at once: row (columns = 0)
 * or column (columns = 1) name k is the NUL-terminated string at
 * chars + offsets[k]; offsets has count + 1 entries. */
int pdhg_model_name_table(const pdhg_model* model, int columns, const char** chars,
                          const int64_t** offsets);
/* ReaderWarning k (io.hpp:23-27): line (0 for the layout note), section, text. */
int pdhg_model_warning(const pdhg_model* model, int32_t k, int64_t* line, const char** section,
                       const char** message);

#ifdef __cplusplus
}
#endif
#endif /* PDHG_B200_H */
