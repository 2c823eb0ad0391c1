// engine.cuh -- device-side data layout of the PDHG engine.
//
// One LP lives in HBM for the whole solve (the reference keeps A resident the
// same way, include/sovereign/backend.hpp:225-263, but stores only A and runs
// A^T through a transpose flag; here A^T is a second CSR built on the device).
//
//   A_s, AT_s : the Ruiz+Pock-Chambolle scaled matrix and its transpose,
//               FP64 values (+ FP32 copies for the mixed-precision kernels).
//   A_o, AT_o : the original matrix and its transpose, FP64 (original-space
//               residuals and the final result). Index arrays are shared with
//               A_s/AT_s when scaling dropped no entry.
//   vectors   : scaled c (objective sign applied), bounds, scale factors,
//               iterates x, x_bar, s, y and the Cesaro sums, all dense.
//   DevState  : the solver's control state (iteration counters, restart state,
//               residuals, stop flag) -- decided on the device every check
//               period, so the loop needs no host round trip.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <string>

#include "../../include/pdhg_b200.h"

namespace pdhg {

constexpr int kBlock = 256;  // threads per CTA for every engine kernel

// Row-length tiers of the binning (entries per row).
constexpr int kLongRow = 512;   // above: a CTA per row (CTA items in the throughput kernels)
constexpr int kWarpRow = 32;    // ordered kernels: above, one warp per row
constexpr int kHugeRow = 4096;  // long_mode 1: above, CTA items instead of a warp

// CTA work items over long rows. A row of at most kSegLen entries (more when
// the long rows hold enough entries to fill the GPU without splitting) is one
// item; a longer row is cut into near-equal segments, one item each, so that
// no single CTA walks a row of hundreds of thousands of entries while the rest
// of the GPU idles. Each segment's CTA stores its
// partial dot products and takes a ticket; the CTA that draws the row's last
// ticket adds the partials in segment order (deterministic whatever the
// arrival order), resets the ticket and runs the row's epilogue.
constexpr int kSegLen = 4096;
constexpr int kWarpSegLen = 1024;  // the same for warp work items (long_mode 2)

struct RowItems {
    const int4* item = nullptr;      // {row, begin, end, split}; split -1 = the whole row
    const int2* split = nullptr;     // per split row: {first item, segments}
    unsigned int* ticket = nullptr;  // per split row, 0 between launches
    double* part = nullptr;          // 2 partials per item
    unsigned int* fetch = nullptr;   // persistent kernels: {next item, exits}, 0 between launches
    int32_t n_item = 0;
};

// Row slices: 32 long rows of about the same length stored lane-interleaved
// (entry k of lane l at off + 32 k + l). Chosen for rows whose gathers
// coalesce across rows but not along a row -- consecutive entries of a row
// far apart in the gathered vector, the k-th entries of the 32 rows next to
// each other (the demand rows of a transportation LP). A warp item covers
// entries [k0, k1) of one slice, lane l summing row l, so the value, index
// and gather loads of a step are each one or two lines. A slice cut into
// several items combines per lane like a split row (ticket per slice, 32
// partials per item, added in item order by the last warp).
struct RowSlices {
    int32_t n_slice = 0, n_item = 0;
    const int4* slice = nullptr;     // {len (longest lane), off, rows in use, -}
    const int32_t* row = nullptr;    // 32 per slice: row id, -1 for an unused lane
    const int32_t* rlen = nullptr;   // 32 per slice: the lane's row length
    const int32_t* col = nullptr;    // lane-interleaved column indices (scaled matrix)
    const float* v32 = nullptr;      // lane-interleaved scaled values, FP32 and FP64
    const double* v64 = nullptr;
    const int4* item = nullptr;      // {slice, k0, k1, split}; split -1 = the whole slice
    const int2* split = nullptr;     // per split slice: {first item, items}
    unsigned int* ticket = nullptr;  // per split slice, 0 between launches
    double* part = nullptr;          // 32 partials per item
    unsigned int* fetch = nullptr;   // {next item, exits}, 0 between launches
    const int2* affine = nullptr;    // per slice {base, stride}: column base + l + k stride, or {0, 0}
    unsigned int* cticket = nullptr; // the check's: per split slice, 0 between launches
    double* cpart = nullptr;         // the check's: 64 partials per item (current, average)
};

// The long-row tiers of the throughput kernels (see DevCsr).
struct LongTiers {
    const int32_t* warp_rows0 = nullptr;
    const int32_t* warp_rows1 = nullptr;
    int32_t n_warp0 = 0, n_warp1 = 0;
    RowItems items_long, items_huge, items_warp;
};

struct DevCsr {
    int32_t rows = 0, cols = 0;
    int64_t nnz = 0;
    const int32_t* rp = nullptr;
    const int32_t* ci = nullptr;
    const double* v64 = nullptr;
    const float* v32 = nullptr;
    // Row binning for the warp-parallel kernels: rows longer than kLongRow are
    // listed in long_rows and handled one CTA per row; the others by groups of
    // `vw` lanes.
    const int32_t* long_rows = nullptr;
    int32_t n_long = 0;
    int32_t n_short = 0;
    int vw = 1;
    // Row binning for the ordered (FP64-exact) kernels: rows longer than
    // kWarpRow are listed in wrows and handled one warp per row; without the
    // list every row runs on one thread.
    const int32_t* wrows = nullptr;
    int32_t n_wrows = 0;
    // The throughput kernels (iteration and check) bin once more. Rows of at
    // most short_max entries (16 lanes' worth at the binning's lanes per row,
    // within [kWarpRow, kLongRow]) run on lane groups, n_iter_short of them;
    // longer rows one warp per row up to kLongRow entries (warp_rows0:
    // long_mode 0 and the check) or up to kHugeRow entries (warp_rows1:
    // long_mode 1), and CTA work items above. n_mid counts the rows of
    // kLongRow..kHugeRow entries, n_huge those above.
    int32_t short_max = kLongRow;
    int32_t n_iter_short = 0;
    const int32_t* warp_rows0 = nullptr;
    const int32_t* warp_rows1 = nullptr;
    int32_t n_warp0 = 0, n_warp1 = 0;
    int32_t n_mid = 0, n_huge = 0;
    // CTA work items over every row above kLongRow (long_mode 0 and the check
    // kernel) and over the rows above kHugeRow (long_mode 1); warp work items
    // over every row above short_max (long_mode 2).
    RowItems items_long, items_huge, items_warp;
    // Row slices (iteration kernels only) and the long-row tiers without the
    // slices' rows, which replace the fields above when use_slices is set.
    RowSlices slices;
    LongTiers no_slice_tiers;
    // Iteration-kernel shape (the autotuner's choice): lanes per short row
    // (0 = vw), the long-row strategy (0: warp_rows0 + items_long;
    // 1: warp_rows1 + items_huge; 2: items_warp) and whether the row slices
    // take their rows.
    int iter_vw = 0;
    int long_mode = 0;
    int use_slices = 0;
    // > 0 when every row has exactly this many entries (rp[r] = r * rp_stride):
    // the short-row iteration kernel computes the row's extent instead of
    // loading it
    int32_t rp_stride = 0;
    // per row (null when the matrix has no row above short_max): off when
    // entry k of the row sits in column k + off (every entry, consecutive
    // columns), kNotDense otherwise; the long-row iteration paths then compute
    // the columns and stream the gathered vector
    const int32_t* dense_off = nullptr;
};
constexpr int32_t kNotDense = static_cast<int32_t>(0x80808080u);  // a byte-wise memset value


// Accumulator slots (bit patterns of non-negative doubles, combined with
// atomicMax -- order-independent, so exact).
enum Acc {
    ACC_CUR_P = 0, ACC_CUR_D, ACC_AVG_P, ACC_AVG_D,        // scaled-space residual parts
    ACC_ORIG_P, ACC_ORIG_D,                               // exact mode: candidate, original space
    ACC_OC_P, ACC_OC_D, ACC_OA_P, ACC_OA_D,               // fast mode: cur / avg, original space
    ACC_FIN_PINF, ACC_FIN_DINF,                           // final result
    ACC_RAY,                                              // infeasibility test: max |dy| (original)
    ACC_XRAY_MAX, ACC_XRAY_V,                             // ray test: max |d|, rows' cone violation
    ACC_COUNT = 16
};

enum Ticket { TK_CHECK1 = 0, TK_CHECK2, TK_FAST, TK_RESTART, TK_COUNT = 4 };

// Per-CTA partial sums of the fast check kernel: the objectives (4), the
// Farkas ranges (4), c^T dx of the ray test (1).
constexpr int kCheckSums = 13;

// Mixed precision under termination rule 2: a relative-KKT plateau above this
// value (1024 units of FP32 roundoff) is the method's own, not FP32's
// precision floor, so the FP32 phase keeps running there.
constexpr double kFp32Zone = 1024.0 * 1.1920928955078125e-7;

struct DevState {
    int done;         // 1 = every later kernel returns at once
    int status;       // pdhg_status once done
    int converged;
    int fresh;        // the next period starts right after a restart
    int restart;      // the last check restarted
    int avg_better;   // the last check picked the average as candidate
    int fail_kind;    // 1 = scaled residual non-finite, 2 = original residual non-finite
    int fold;         // mixed mode: fold the FP32 period sums into the FP64 sums
    long long iter;           // iterations completed before the current period
    long long since_restart;  // iterations averaged at the last check
    long long restarts;
    long long stop_iter;      // iteration count reported on stop
    long long checks;
    double res_last;          // residual at the last restart (+inf before the first check)
    double cur_res, avg_res, orig_res, rel_kkt;
    double inv;               // 1 / iterations in the Cesaro average at the last check
    double objective, dual_objective, duality_gap, pinf, dinf;
    // step sizes: tau = eta / omega, sigma = eta * omega (omega = primal weight;
    // the reference keeps omega = 1, tau = sigma, pdhg.cpp:263-265)
    double tau, sigma, omega, eta;
    double res_prev_cand;     // adaptive rule: candidate residual at the previous check
    int restart_to_avg;       // adaptive rule: restart point is the average (else current)
    int gap_finite;
    int ray_base;             // infeasibility test: the previous check's y / A^T y are stored
    double ray_scale;         // 1 / max |dy| of the certifying check
    double ray_ranges[4];     // its row-side lo, hi and column-side lo, hi (scaled by ray_scale)
    int xray_pending;         // ray test: a projected ray awaits its rows' test
    int xray_buf;             // which of the two ray buffers holds it
    double xray_scale;        // its 1 / max |d_j| (original units)
    double xray_obj, xray_viol;  // its c^T d (minimize sense) and cone violation, max |d| = 1
    unsigned long long acc[ACC_COUNT];
    unsigned int ticket[TK_COUNT];
};

// Host-mapped pinned mailbox: the host writes stop requests (time limit,
// cancellation), the last block of every check writes its decision here.
struct Mailbox {
    volatile int stop_request;  // 0, or the pdhg_status to stop with
    volatile int done;
    volatile int status;
    volatile int restarted;
    volatile long long iter;
    volatile long long restarts;
    volatile long long checks;
    volatile double cur_res, avg_res, orig_res, rel_kkt;
};

// Problem vectors (device, FP64 unless noted).
struct DevProblem {
    int32_t m = 0, n = 0;
    double obj_sign = 1.0;
    double obj_const = 0.0;
    const double *c = nullptr, *lo = nullptr, *hi = nullptr;    // scaled, c signed
    const double *rlo = nullptr, *rhi = nullptr;                // scaled row bounds
    const double *c_o = nullptr, *lo_o = nullptr, *hi_o = nullptr;
    const double *rlo_o = nullptr, *rhi_o = nullptr;            // original
    const double *rs = nullptr, *cs = nullptr;                  // row / column scale
    const float *c32 = nullptr, *lo32 = nullptr, *hi32 = nullptr;
    const float *rlo32 = nullptr, *rhi32 = nullptr;
    double bnorm = 0.0, cnorm = 0.0;    // relative-KKT norms (original space, inf-norms)
    double bnorm2 = 0.0, cnorm2 = 0.0;  // termination rule 2 norms (original space, l2)
    // every column has the same scaled bounds lo_u <= x <= hi_u (x >= 0 LPs):
    // the iteration kernels use the two values instead of loading the vectors
    int col_bounds_uniform = 0;
    double lo_u = 0.0, hi_u = 0.0;
    // ... the original bounds likewise (the check kernels' column terms)
    int col_bounds_uniform_o = 0;
    double lo_uo = 0.0, hi_uo = 0.0;
};

// Iterates. T = double for the FP64 modes, float for the mixed mode; the
// mixed mode keeps per-period FP32 partial sums (psx, psy) that the check
// folds into the FP64 Cesaro sums (xsum, ysum).
template <class T>
struct Iterates {
    T *x = nullptr, *xbar = nullptr, *s = nullptr, *y = nullptr;
    T *psx = nullptr, *psy = nullptr;
    double *xsum = nullptr, *ysum = nullptr;
    // option halpern: the anchor (the last restart point) of the reflected
    // Halpern iteration; the sums' slots (psx / psy, or xsum / ysum in FP64)
    // then hold the last PDHG output T(z) instead of running sums
    T *xa = nullptr, *sa = nullptr, *ya = nullptr;
    int halpern = 0;
    // with halpern, lean = 1: z's x part and T(z) are stored only by the
    // iterations whose point a check or the result reads (the last of a check
    // period or of the solve). The primal pass rebuilds x as
    // w' x_bar + (1 - w') x_a (w' the previous iteration's weight, x_bar its
    // reflected point, which every iteration writes).
    int lean = 0;
};

struct CheckScratch {
    double* act_avg = nullptr;   // m: A x_avg (unprojected), for the restart's slack
    double* cand_xo = nullptr;   // n: the candidate in original units
    double* cand_yo = nullptr;   // m
    double* part = nullptr;      // block partial sums (deterministic reduction)
    int part_blocks = 0;
};

struct FinalScratch {
    double* xo = nullptr;   // n
    double* yo = nullptr;   // m
    double* rc = nullptr;   // n
    double* trow = nullptr; // m: dual-objective row terms
    double* tcol = nullptr; // n: dual-objective column terms
};

// ---- launchers (kernels_exact.cu) ------------------------------------------
// tau and sigma live in DevState (they change with the primal weight).
struct ExactIter {
    DevCsr A, AT;
    DevProblem P;
    Iterates<double> it;
    DevState* st;
};
void launch_exact_primal(const ExactIter& a, int first, cudaStream_t s);
void launch_exact_dual(const ExactIter& a, int first, cudaStream_t s);

struct ExactCheck {
    DevCsr A, AT, Ao, ATo;
    DevProblem P;
    Iterates<double> it;
    CheckScratch cs;
    double tol, bound_tol, restart_decrease;
    long long period_iters;
    int termination_rule;
    int want_candidate;
    DevState* st;
    Mailbox* mail;
};
void launch_exact_check(const ExactCheck& a, cudaStream_t s);
void launch_exact_restart(const ExactCheck& a, cudaStream_t s);

// ---- launchers (kernels_fast.cu) -------------------------------------------
template <class T>
struct FastIter {
    DevCsr A, AT;
    DevProblem P;
    Iterates<T> it;
    DevState* st;
    int hk = 0;  // the iteration's index in its check period (Halpern weight)
    int tz = 1;  // Halpern: this iteration stores T(z) (lean mode: only before a check / the end)
};
// A pass's short-row, long-row and row-slice kernels touch disjoint rows and
// only read the gathered vector, so they may run side by side: with a
// PassFork the long-row kernel goes to side[0] and the slice kernel to side[1]
// (fork: s -> sides, join: sides -> s), else all run in order on s. Inside a
// stream capture these become parallel graph branches.
struct PassFork {
    cudaStream_t side[2] = {nullptr, nullptr};
    cudaEvent_t fork = nullptr, join[2] = {nullptr, nullptr};
};
template <class T>
int launch_fast_primal(const FastIter<T>& a, int first, cudaStream_t s,
                       const PassFork* f = nullptr);  // kernels launched
template <class T>
int launch_fast_dual(const FastIter<T>& a, int first, cudaStream_t s,
                     const PassFork* f = nullptr);
template <class T>
int fast_launches_per_iteration(const FastIter<T>& a);
// Once per device, before the first launch and outside any stream capture:
// records how many CTAs of the persistent iteration kernels are resident per
// device (their grids). 0 on success.
int init_fast_kernels(int device);

// Restart rules: 0 = the reference's (restart to the average when its residual
// is <= restart_decrease x the residual at the last restart, pdhg.cpp:391-408);
// 1 = adaptive: restart to the better of average / current on sufficient decay
// (<= 0.2x), on necessary decay (<= 0.8x) without progress since the previous
// check, or when the average spans >= 36% of all iterations.
template <class T>
struct FastCheck {
    DevCsr A, AT;  // scaled, FP64 values used
    DevProblem P;
    Iterates<T> it;
    CheckScratch cs;
    double tol, bound_tol, restart_decrease;
    long long period_iters;
    int termination_rule;
    int want_candidate;
    DevState* st;
    Mailbox* mail;
    int restart_rule;
    int primal_weight_update;  // omega <- sqrt(omega * |dy| / |dx|) at each restart
    double* x_last;            // scaled point of the last restart (n)
    double* y_last;            // (m)
    int grid_cap;              // CTAs of the (grid-stride) check kernel: SMs x 8
    // infeasibility test (option infeasibility_detection): y and A^T y of the
    // previous check (scaled; m, n) and the change of y in original units (m);
    // the ray test: x of the previous check (scaled; n) and two buffers for
    // the change of x projected onto the columns' recession cones (scaled; n)
    int infeas = 0;
    double* ray_y_prev = nullptr;
    double* ray_aty_prev = nullptr;
    double* ray_y = nullptr;
    double* xray_x_prev = nullptr;
    double* xray_d[2] = {nullptr, nullptr};
};
template <class T>
void launch_fast_check(const FastCheck<T>& a, cudaStream_t s);
template <class T>
void launch_fast_restart(const FastCheck<T>& a, cudaStream_t s);

// ---- setup / final (kernels_exact.cu) ------------------------------------------
// Exact pairwise sum of x[i]*y[i] (HostBackend::pairwise_dot order) into *out.
void launch_pairwise_dot(const double* x, const double* y, int64_t n, double* partial,
                         double* out, cudaStream_t s);
int64_t pairwise_partial_size(int64_t n);
// Power-iteration pieces (estimate_operator_norm, pdhg.cpp:48-79).
// stop: a device flag that turns the launch into a no-op (null: always run)
// fast: the rows' products added in parallel (not the reference's order)
void launch_pw_w(const DevCsr& A, const double* u, const double* v, double* w, cudaStream_t s,
                 const int* stop = nullptr, const double* uscale = nullptr, bool fast = false);
void launch_pw_u(const DevCsr& AT, const double* w, double* u, cudaStream_t s,
                 const int* stop = nullptr);
void launch_scale(double* x, int64_t n, double alpha, cudaStream_t s);
// the power iteration's scalar steps on the device (k_pw_norm_w / _e)
void launch_pw_norm_w(const double* dot, double* st, int* stop, cudaStream_t s);
void launch_pw_norm_e(const double* dots, double* st, int* stop, cudaStream_t s);
void launch_scale_by(double* x, int64_t n, const double* alpha, const int* stop, cudaStream_t s);
void launch_copy_unless(double* dst, const double* src, int64_t n, const int* stop, cudaStream_t s);
void launch_fill(double* x, int64_t n, double v, cudaStream_t s);

struct FinalArgs {
    DevCsr Ao, ATo;
    DevProblem P;
    const double* best_x64 = nullptr;  // scaled best point, FP64 (or null)
    const double* best_y64 = nullptr;
    const float* best_x32 = nullptr;   // mixed mode current point
    const float* best_y32 = nullptr;
    FinalScratch f;
    double bound_tol;
    int exact;
    DevState* st;
    double* part = nullptr;   // 3 doubles per CTA of the fast-mode sums
    int part_blocks = 0;      // CTAs that fit in part (and at most a few per SM)
};
void launch_final(const FinalArgs& a, cudaStream_t s);

// Best point selection for the final result: the check's candidate when
// converged, else the current iterate (pdhg.cpp:420-423). Materialises the
// scaled FP64 point into (bx, by).
template <class T>
void launch_select_point(const Iterates<T>& it, const DevState* st, int32_t n, int32_t m,
                         double* bx, double* by, cudaStream_t s);

// Initial point (pdhg.cpp:268-270) or warm start; FP64 scaled inputs.
// z_a <- z for the Halpern option's anchor (x, s, y); n, m entries.
template <class T>
void launch_set_anchor(const Iterates<T>& it, int32_t n, int32_t m, cudaStream_t s);
template <class T>
void launch_init_point(const DevProblem& P, const DevCsr& A, const double* x0s,
                       const double* y0s, Iterates<T> it, cudaStream_t s);

// Backend primitives for the known-answer tests.
void launch_spmv_exact(const DevCsr& A, double alpha, const double* x, double beta, double* y,
                       cudaStream_t s);
void launch_spmvT_exact(const DevCsr& AT, double alpha, const double* x, double beta, double* y,
                        cudaStream_t s);
int fast_check_grid(const DevCsr& A, const DevCsr& AT);
int exact_check_grid(const DevCsr& A, const DevCsr& AT);  // blocks of an exact check / final launch
void launch_project_box(int32_t n, const double* lo, const double* hi, double* x,
                        cudaStream_t s);

// Device CSR transpose: stable by column, so each A^T row lists its entries in
// ascending original row order (the order the reference's scatter adds them,
// src/l0/backend_host.cpp:439-444).
struct TransposeOut {
    int32_t* rp;
    int32_t* ci;
    double* v;
};
// The transpose works in caller-owned scratch of transpose_scratch_bytes()
// bytes (256-byte aligned), so repeated loads of one size reuse it.
size_t transpose_scratch_bytes(int32_t m, int32_t n, int64_t nnz);
int build_transpose(int32_t m, int32_t n, int64_t nnz, const int32_t* rp, const int32_t* ci,
                    const double* v, TransposeOut out, void* scratch, cudaStream_t s);

void launch_to_float(const double* src, float* dst, int64_t n, cudaStream_t s);

// ---- intake (intake.cu) --------------------------------------------------------
constexpr int kNorms = 6;
struct IntakeState {
    unsigned long long worst;  // Ruiz: max |row/col max - 1| of the sweep (bit pattern)
    unsigned int ticket;
    int ruiz_done;             // set when a sweep's worst < tolerance (scaling.cpp:72)
    // |c_s|_2^2, |b_s|_2^2, |c_o|_inf, |b_o|_inf, |c_o|_2^2, |b_o|_2^2, with b_i
    // the larger finite |row bound| of row i (0 if none)
    double norms[kNorms];
};
// Device problem checks, OR-ed into *flags: 1 a column, 2 a row, 4 an entry's
// column out of range, 8 an entry out of order or non-finite. c == NULL skips
// the column checks and rlo == NULL the row checks.
void launch_validate(int32_t m, int32_t n, const int32_t* rp, const int32_t* ci, const double* v,
                     const double* c, const double* clo, const double* chi, const double* rlo,
                     const double* rhi, int64_t nnz, unsigned* flags, cudaStream_t s);
// Rows with lo < length <= hi appended to `list`, their number added to *count.
void launch_bin_range(const int32_t* rp, int32_t rows, int lo, int hi, int32_t* list,
                      unsigned long long* count, cudaStream_t s);
// *flag |= 1 when the rows' lengths are not all equal / the entries of v not
// all equal (flag zeroed by the caller).
void launch_uniform_rows(const int32_t* rp, int32_t rows, unsigned* flag, cudaStream_t s);
void launch_uniform_vec(const double* v, int32_t n, unsigned* flag, cudaStream_t s);
void launch_bin(const int32_t* rp, int32_t rows, int long_threshold, int32_t* long_rows,
                unsigned long long* counters, cudaStream_t s);
// out[k] = {rows[k], rp[rows[k]], rp[rows[k] + 1], 0} for k < n.
void launch_row_extents(const int32_t* rows, int32_t n, const int32_t* rp, int4* out,
                        cudaStream_t s);
// Column indices of sampled entries: out[q] = ci[pos[q]] for q < n.
void launch_gather_cols(const int32_t* ci, const int64_t* pos, int32_t n, int32_t* out,
                        cudaStream_t s);
// Lane-interleaved copy of the slices' rows: for slice s, lane l, entry k <
// rlen: col/v32/v64[off + 32 k + l] = the row's k-th entry; padding entries
// get column 0 and value 0.
// nnz_affine / nnz_dense: device counters that the kernels add the entries
// of affine slices / dense rows to
void launch_affine_slices(const RowSlices& S, int2* affine, unsigned long long* nnz_affine,
                          cudaStream_t s);
void launch_dense_rows(const int32_t* ci, const int4* ext, int32_t n_ext, int32_t* dense_off,
                       unsigned long long* nnz_dense, cudaStream_t s);
void launch_fill_slices(const DevCsr& M, RowSlices S, int32_t* col, float* v32, double* v64,
                        int64_t total, cudaStream_t s);
void launch_ruiz_sweep(const DevCsr& A, const DevCsr& AT, double* rs, double* cs,
                       double* row_max, double* col_max, double tol, IntakeState* is,
                       cudaStream_t s);
void launch_pock_chambolle(const DevCsr& A, const DevCsr& AT, double* rs, double* cs,
                           double* row_sum, double* col_sum, double alpha, cudaStream_t s);
void launch_scale_values(const DevCsr& M, int transposed, const double* rs, const double* cs,
                         double* out, unsigned long long* dropped, cudaStream_t s);
void launch_kept_counts(const DevCsr& M, const double* vs, int32_t* cnt, cudaStream_t s);
void launch_compact(const DevCsr& M, const double* vs, const int32_t* new_rp, int32_t* ci_out,
                    double* v_out, cudaStream_t s);
void launch_scale_vectors(int32_t m, int32_t n, const double* rs, const double* cs,
                          const double* c, const double* lo, const double* hi, const double* rlo,
                          const double* rhi, double sign, double* c_s, double* lo_s,
                          double* hi_s, double* rlo_s, double* rhi_s, cudaStream_t s);
int norms_part_size(int32_t m, int32_t n);
void launch_norms(int32_t m, int32_t n, const double* c_s, const double* rlo_s,
                  const double* rhi_s, const double* c_o, const double* rlo_o,
                  const double* rhi_o, double* part, IntakeState* is, cudaStream_t s);
// Inclusive prefix sum of n int32 counts into out[1..n], out[0] = 0 (CUB).
int prefix_rows(const int32_t* cnt, int32_t n, int32_t* out, cudaStream_t s);

// The batched engine (batch.cu), owned by a context: it uses the context's
// stream and writes its errors into the context's error text.
struct BatchCtx;
BatchCtx* batch_new(int device, cudaStream_t stream, std::string& err);
void batch_delete(BatchCtx* b);
int batch_load_abi(BatchCtx& c, int32_t count, const int32_t* row_off, const int32_t* col_off,
                   int64_t nnz, const int32_t* rp, const int32_t* ci, const double* v,
                   const double* cv, const double* obj_const, const int* maximize,
                   const double* col_lo, const double* col_hi, const double* row_lo,
                   const double* row_hi);
int batch_solve_abi(BatchCtx& c, const pdhg_options* options, pdhg_info* infos, double* x,
                    double* y, double* rc);
int32_t batch_count(const BatchCtx& c);
int batch_point_kkt_abi(BatchCtx& c, const double* x, const double* y, double* kkt);
int batch_tuning_abi(const BatchCtx& c, int precision, int* out);

}  // namespace pdhg
