/*
 * pdhg_oracle.c -- TEST INFRASTRUCTURE ONLY: a plain-C restatement of the
 * reference PDHG path, used as the checker for the CUDA engine. See
 * pdhg_oracle.h for the file map and the pinning status. Every function cites
 * the reference lines it restates (paths relative to the reference project).
 *
 * Built with -O2 -ffp-contract=off (oracle/Makefile): no fused multiply-add,
 * so each `a + b * c` rounds twice exactly as the reference's host build does.
 */
#define _POSIX_C_SOURCE 200809L
#include "pdhg_oracle.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

static double now_seconds(void) {
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}

/* std::max(a, b) == (a < b) ? b : a -- NaN in b is ignored, as in the
 * reference's residual loops. */
static double smax(double a, double b) { return (a < b) ? b : a; }

/* is_finite_bound (include/sovereign/problem.hpp:31-33). */
static int finite_bound(double v) { return v > -INFINITY && v < INFINITY; }

void orc_default_options(orc_options* o) {
    memset(o, 0, sizeof *o);
    /* include/sovereign/pdhg.hpp:89-117 */
    o->tolerance = 1e-4;
    o->max_iterations = 1000000;
    o->time_limit_seconds = 0.0;
    o->restart_check_period = 40;
    o->restart_sufficient_decrease = 0.5;
    o->step_size_safety = 0.9;
    o->power_iterations = 30;
    /* include/sovereign/scaling.hpp:299-309 */
    o->ruiz_iterations = 8;
    o->ruiz_tolerance = 1e-2;
    o->pock_chambolle_alpha = 1.0;
    o->apply_ruiz = 1;
    o->apply_pock_chambolle = 1;
}

const char* orc_status_string(int s) {
    /* src/l1/pdhg.cpp:17-27 */
    switch (s) {
        case ORC_OPTIMAL: return "optimal";
        case ORC_ITERATION_LIMIT: return "iteration_limit";
        case ORC_TIME_LIMIT: return "time_limit";
        case ORC_NUMERICAL_FAILURE: return "numerical_failure";
        case ORC_NOT_SOLVED: return "not_solved";
        case ORC_CANCELLED: return "cancelled";
    }
    return "unknown";
}

/* ---------------------------------------------------------------------------
 * Host backend primitives (src/l0/backend_host.cpp)
 * ------------------------------------------------------------------------- */

/* HostBackend::pairwise_dot, backend_host.cpp:480-490 (block 128). */
double orc_pairwise_dot(const double* x, const double* y, int64_t n) {
    if (n <= 0) return 0.0;
    if (n <= 128) {
        double s = 0.0;
        for (int64_t i = 0; i < n; ++i) s += x[i] * y[i];
        return s;
    }
    const int64_t half = n / 2;
    return orc_pairwise_dot(x, y, half) + orc_pairwise_dot(x + half, y + half, n - half);
}

static double norm2(const double* x, int64_t n) {
    /* HostBackend::norm2, backend_host.cpp:390-396 */
    return sqrt(orc_pairwise_dot(x, x, n));
}

/* HostBackend::spmv, backend_host.cpp:409-425. */
void orc_spmv(int32_t m, const int32_t* rp, const int32_t* ci, const double* v, double alpha,
              const double* x, double beta, double* y) {
    for (int32_t r = 0; r < m; ++r) {
        double sum = 0.0;
        for (int32_t k = rp[r]; k < rp[r + 1]; ++k) sum += v[k] * x[ci[k]];
        y[r] = (beta == 0.0) ? alpha * sum : alpha * sum + beta * y[r];
    }
}

/* HostBackend::spmv_transpose, backend_host.cpp:427-446 (scatter in row order). */
void orc_spmv_transpose(int32_t m, int32_t n, const int32_t* rp, const int32_t* ci,
                        const double* v, double alpha, const double* x, double beta,
                        double* y) {
    if (beta == 0.0) {
        for (int32_t c = 0; c < n; ++c) y[c] = 0.0;
    } else {
        for (int32_t c = 0; c < n; ++c) y[c] *= beta;
    }
    for (int32_t r = 0; r < m; ++r) {
        const double ax = alpha * x[r];
        for (int32_t k = rp[r]; k < rp[r + 1]; ++k) y[ci[k]] += v[k] * ax;
    }
}

/* HostBackend::project_box, backend_host.cpp:450-458 (NULL = unbounded side). */
void orc_project_box(int32_t n, const double* lo, const double* hi, double* x) {
    for (int32_t i = 0; i < n; ++i) {
        if (lo != NULL && x[i] < lo[i]) x[i] = lo[i];
        if (hi != NULL && x[i] > hi[i]) x[i] = hi[i];
    }
}

static void axpy(int64_t n, double alpha, const double* x, double* y) {
    /* backend_host.cpp:366-371 */
    for (int64_t i = 0; i < n; ++i) y[i] += alpha * x[i];
}

static void scale(int64_t n, double alpha, double* x) {
    /* backend_host.cpp:373-378 */
    for (int64_t i = 0; i < n; ++i) x[i] *= alpha;
}

/* CsrMatrix::multiply, src/l0/sparse.cpp:130-141. */
static void csr_multiply(int32_t m, const int32_t* rp, const int32_t* ci, const double* v,
                         const double* x, double* y) {
    for (int32_t r = 0; r < m; ++r) {
        double sum = 0.0;
        for (int32_t k = rp[r]; k < rp[r + 1]; ++k) sum += v[k] * x[ci[k]];
        y[r] = sum;
    }
}

/* CsrMatrix::multiply_transpose, src/l0/sparse.cpp:143-154. */
static void csr_multiply_transpose(int32_t m, int32_t n, const int32_t* rp, const int32_t* ci,
                                   const double* v, const double* x, double* y) {
    for (int32_t c = 0; c < n; ++c) y[c] = 0.0;
    for (int32_t r = 0; r < m; ++r) {
        const double xr = x[r];
        for (int32_t k = rp[r]; k < rp[r + 1]; ++k) y[ci[k]] += v[k] * xr;
    }
}

/* ---------------------------------------------------------------------------
 * Scaling (src/l1/scaling.cpp)
 * ------------------------------------------------------------------------- */

static double safe_sqrt(double v) { return v > 0.0 ? sqrt(v) : 1.0; } /* scaling.cpp:11 */

/* Scaling::equilibrate(const CsrMatrix&), scaling.cpp:19-104. */
void orc_scaling(int32_t m, int32_t n, const int32_t* rp, const int32_t* ci, const double* val,
                 const orc_options* opt, double* rs, double* cs) {
    for (int32_t r = 0; r < m; ++r) rs[r] = 1.0;
    for (int32_t c = 0; c < n; ++c) cs[c] = 1.0;

    if (opt->apply_ruiz) { /* scaling.cpp:36-74 */
        double* row_max = (double*)calloc((size_t)m + 1, sizeof(double));
        double* col_max = (double*)calloc((size_t)n + 1, sizeof(double));
        for (int sweep = 0; sweep < opt->ruiz_iterations; ++sweep) {
            memset(row_max, 0, sizeof(double) * (size_t)m);
            memset(col_max, 0, sizeof(double) * (size_t)n);
            for (int32_t r = 0; r < m; ++r) {
                for (int32_t k = rp[r]; k < rp[r + 1]; ++k) {
                    const int32_t c = ci[k];
                    const double s = fabs(val[k]) * rs[r] * cs[c];
                    row_max[r] = smax(row_max[r], s);
                    col_max[c] = smax(col_max[c], s);
                }
            }
            double worst = 0.0;
            for (int32_t r = 0; r < m; ++r) {
                if (row_max[r] > 0.0) {
                    rs[r] /= safe_sqrt(row_max[r]);
                    worst = smax(worst, fabs(row_max[r] - 1.0));
                }
            }
            for (int32_t c = 0; c < n; ++c) {
                if (col_max[c] > 0.0) {
                    cs[c] /= safe_sqrt(col_max[c]);
                    worst = smax(worst, fabs(col_max[c] - 1.0));
                }
            }
            if (worst < opt->ruiz_tolerance) break;
        }
        free(row_max);
        free(col_max);
    }

    if (opt->apply_pock_chambolle) { /* scaling.cpp:80-101 */
        const double a = opt->pock_chambolle_alpha;
        double* row_sum = (double*)calloc((size_t)m + 1, sizeof(double));
        double* col_sum = (double*)calloc((size_t)n + 1, sizeof(double));
        for (int32_t r = 0; r < m; ++r) {
            for (int32_t k = rp[r]; k < rp[r + 1]; ++k) {
                const int32_t c = ci[k];
                const double mag = fabs(val[k]) * rs[r] * cs[c];
                if (mag <= 0.0) continue;
                row_sum[r] += pow(mag, 2.0 - a);
                col_sum[c] += pow(mag, a);
            }
        }
        for (int32_t r = 0; r < m; ++r)
            if (row_sum[r] > 0.0) rs[r] /= safe_sqrt(row_sum[r]);
        for (int32_t c = 0; c < n; ++c)
            if (col_sum[c] > 0.0) cs[c] /= safe_sqrt(col_sum[c]);
        free(row_sum);
        free(col_sum);
    }
}

/* ---------------------------------------------------------------------------
 * Validation (src/io/problem.cpp:50-, src/l0/sparse.cpp:94-128)
 * Names: the reference reports a row/column by its model name; the oracle and
 * the engine name them R<i> / C<j>, which is also what the reference shim
 * (oracle/ref_shim.cpp) assigns when it builds a sov::Problem.
 * ------------------------------------------------------------------------- */

static int validate(const orc_problem* p, char* why, size_t len) {
    if (!isfinite(p->obj_const)) {
        snprintf(why, len, "objective constant is not finite");
        return 0;
    }
    for (int32_t j = 0; j < p->n; ++j) {
        if (!isfinite(p->c[j])) {
            snprintf(why, len, "non-finite objective coefficient in column C%d", j);
            return 0;
        }
        if (isnan(p->col_lo[j]) || isnan(p->col_hi[j])) {
            snprintf(why, len, "NaN bound on column C%d", j);
            return 0;
        }
        if (p->col_lo[j] > p->col_hi[j]) {
            snprintf(why, len, "crossed bounds on column C%d", j);
            return 0;
        }
    }
    for (int32_t i = 0; i < p->m; ++i) {
        if (isnan(p->row_lo[i]) || isnan(p->row_hi[i])) {
            snprintf(why, len, "NaN bound on row R%d", i);
            return 0;
        }
        if (p->row_lo[i] > p->row_hi[i]) {
            snprintf(why, len, "crossed bounds on row R%d", i);
            return 0;
        }
    }
    /* CsrMatrix::validate, sparse.cpp:94-128 */
    if (p->m >= 0 && p->row_ptr[0] != 0) {
        snprintf(why, len, "row_ptr does not start at 0");
        return 0;
    }
    if (p->row_ptr[p->m] != p->nnz) {
        snprintf(why, len, "row_ptr does not end at nnz");
        return 0;
    }
    for (int32_t r = 0; r < p->m; ++r) {
        const int32_t b = p->row_ptr[r], e = p->row_ptr[r + 1];
        if (b > e) {
            snprintf(why, len, "row_ptr is not monotone");
            return 0;
        }
        for (int32_t k = b; k < e; ++k) {
            const int32_t c = p->col_idx[k];
            if (c < 0 || c >= p->n) {
                snprintf(why, len, "column index out of range");
                return 0;
            }
            if (k > b && p->col_idx[k - 1] >= c) {
                snprintf(why, len, "column indices not strictly ascending");
                return 0;
            }
            if (!isfinite(p->val[k])) {
                snprintf(why, len, "non-finite coefficient");
                return 0;
            }
        }
    }
    return 1;
}

/* ---------------------------------------------------------------------------
 * The scaled problem (Scaling::equilibrate(Problem), scaling.cpp:155-205)
 * ------------------------------------------------------------------------- */

typedef struct {
    int32_t m, n;
    int64_t nnz;
    int32_t* rp;
    int32_t* ci;
    double* v;
    double* c; /* scaled objective, NOT yet sign-adjusted */
    double *col_lo, *col_hi, *row_lo, *row_hi;
} scaled_problem;

static void build_scaled(const orc_problem* p, const double* rs, const double* cs,
                         scaled_problem* s) {
    s->m = p->m;
    s->n = p->n;
    s->c = (double*)malloc(sizeof(double) * ((size_t)p->n + 1));
    s->col_lo = (double*)malloc(sizeof(double) * ((size_t)p->n + 1));
    s->col_hi = (double*)malloc(sizeof(double) * ((size_t)p->n + 1));
    s->row_lo = (double*)malloc(sizeof(double) * ((size_t)p->m + 1));
    s->row_hi = (double*)malloc(sizeof(double) * ((size_t)p->m + 1));
    for (int32_t j = 0; j < p->n; ++j) { /* scaling.cpp:172-183 */
        const double c = cs[j];
        s->c[j] = p->c[j] * c;
        s->col_lo[j] = finite_bound(p->col_lo[j]) ? p->col_lo[j] / c : p->col_lo[j];
        s->col_hi[j] = finite_bound(p->col_hi[j]) ? p->col_hi[j] / c : p->col_hi[j];
    }
    for (int32_t i = 0; i < p->m; ++i) { /* scaling.cpp:184-192 */
        const double r = rs[i];
        s->row_lo[i] = finite_bound(p->row_lo[i]) ? p->row_lo[i] * r : p->row_lo[i];
        s->row_hi[i] = finite_bound(p->row_hi[i]) ? p->row_hi[i] * r : p->row_hi[i];
    }
    /* Scaling::apply (scaling.cpp:110-133), then the Builder/from_triplets
     * rebuild (scaling.cpp:194-204, sparse.cpp:30-70), which drops entries
     * with |v| <= tol::numeric_zero = 1e-14 (numeric.hpp:95). */
    s->rp = (int32_t*)malloc(sizeof(int32_t) * ((size_t)p->m + 1));
    s->ci = (int32_t*)malloc(sizeof(int32_t) * ((size_t)p->nnz + 1));
    s->v = (double*)malloc(sizeof(double) * ((size_t)p->nnz + 1));
    int64_t out = 0;
    s->rp[0] = 0;
    for (int32_t r = 0; r < p->m; ++r) {
        const double rr = rs[r];
        for (int32_t k = p->row_ptr[r]; k < p->row_ptr[r + 1]; ++k) {
            const double v = p->val[k] * rr * cs[p->col_idx[k]];
            if (fabs(v) <= 1e-14) continue;
            s->ci[out] = p->col_idx[k];
            s->v[out] = v;
            ++out;
        }
        s->rp[r + 1] = (int32_t)out;
    }
    s->nnz = out;
}

static void free_scaled(scaled_problem* s) {
    free(s->rp);
    free(s->ci);
    free(s->v);
    free(s->c);
    free(s->col_lo);
    free(s->col_hi);
    free(s->row_lo);
    free(s->row_hi);
}

/* estimate_operator_norm, src/l1/pdhg.cpp:48-79. */
double orc_operator_norm(int32_t m, int32_t n, const int32_t* rp, const int32_t* ci,
                         const double* v, int iterations) {
    double* u = (double*)malloc(sizeof(double) * ((size_t)n + 1));
    double* vv = (double*)malloc(sizeof(double) * ((size_t)m + 1));
    double* w = (double*)calloc((size_t)m + 1, sizeof(double));
    for (int32_t j = 0; j < n; ++j) u[j] = 1.0;
    for (int32_t i = 0; i < m; ++i) vv[i] = 1.0;
    double estimate = 0.0;
    for (int it = 0; it < iterations; ++it) {
        orc_spmv(m, rp, ci, v, -1.0, u, 0.0, w);
        axpy(m, 1.0, vv, w);
        const double wn = norm2(w, m);
        if (wn < 1e-300) break;
        scale(m, 1.0 / wn, w);
        orc_spmv_transpose(m, n, rp, ci, v, -1.0, w, 0.0, u);
        memcpy(vv, w, sizeof(double) * (size_t)m);
        const double un = norm2(u, n);
        const double vn = norm2(vv, m);
        estimate = sqrt(un * un + vn * vn);
        if (estimate < 1e-300) break;
        scale(n, 1.0 / estimate, u);
        scale(m, 1.0 / estimate, vv);
    }
    free(u);
    free(vv);
    free(w);
    return estimate;
}

/* kkt_residual, src/l1/pdhg.cpp:87-136 (scaled space, strict `<` at-bound test). */
static double kkt_residual(const scaled_problem* s, const double* c, const double* x,
                           const double* y, double bound_tol, double* act, double* aty) {
    csr_multiply(s->m, s->rp, s->ci, s->v, x, act);
    double primal_res = 0.0, dual_res = 0.0;
    for (int32_t i = 0; i < s->m; ++i) {
        const double lo = s->row_lo[i], hi = s->row_hi[i];
        if (finite_bound(lo)) primal_res = smax(primal_res, lo - act[i]);
        if (finite_bound(hi)) primal_res = smax(primal_res, act[i] - hi);
        const int at_lo = finite_bound(lo) && fabs(act[i] - lo) < bound_tol;
        const int at_hi = finite_bound(hi) && fabs(act[i] - hi) < bound_tol;
        if (!at_lo && !at_hi) dual_res = smax(dual_res, fabs(y[i]));
        else if (at_lo && !at_hi) dual_res = smax(dual_res, smax(0.0, -y[i]));
        else if (at_hi && !at_lo) dual_res = smax(dual_res, smax(0.0, y[i]));
    }
    csr_multiply_transpose(s->m, s->n, s->rp, s->ci, s->v, y, aty);
    for (int32_t j = 0; j < s->n; ++j) {
        const double r = c[j] - aty[j];
        const double lo = s->col_lo[j], hi = s->col_hi[j];
        const int at_lo = finite_bound(lo) && fabs(x[j] - lo) < bound_tol;
        const int at_hi = finite_bound(hi) && fabs(x[j] - hi) < bound_tol;
        if (!at_lo && !at_hi) dual_res = smax(dual_res, fabs(r));
        else if (at_lo && !at_hi) dual_res = smax(dual_res, smax(0.0, -r));
        else if (at_hi && !at_lo) dual_res = smax(dual_res, smax(0.0, r));
    }
    return smax(primal_res, dual_res);
}

/* inf_over_box, src/l1/pdhg.cpp:36-40. */
static double inf_over_box(double coeff, double lo, double hi) {
    if (coeff == 0.0) return 0.0;
    if (coeff > 0.0) return finite_bound(lo) ? coeff * lo : -INFINITY;
    return finite_bound(hi) ? coeff * hi : -INFINITY;
}

/* The bounded part of inf_over_box: an infinite side contributes 0 (its
 * violation is already charged to the dual residual). Used only by the
 * relative-KKT extension; the reported duality_gap keeps the reference rule. */
static double clipped_inf_over_box(double coeff, double lo, double hi) {
    if (coeff > 0.0) return finite_bound(lo) ? coeff * lo : 0.0;
    if (coeff < 0.0) return finite_bound(hi) ? coeff * hi : 0.0;
    return 0.0;
}

/* original_space_residual, src/l1/pdhg.cpp:145-199, split into its primal and
 * dual parts. When rel != NULL also fills the relative-KKT extension value:
 *   max(primal/(1+||finite row bounds||_inf), dual/(1+||c||_inf), gap)
 * with gap = |p - d| / (1 + |p| + |d|) on the clipped dual objective. */
static double original_residual(const orc_problem* p, double obj_sign, const double* rs,
                                const double* cs, const double* xs, const double* ys,
                                double bound_tol, double* xo, double* yo, double* act,
                                double* aty, double* rel) {
    for (int32_t j = 0; j < p->n; ++j) xo[j] = xs[j] * cs[j];
    for (int32_t i = 0; i < p->m; ++i) {
        yo[i] = ys[i] * obj_sign;
        yo[i] *= rs[i];
    }
    csr_multiply(p->m, p->row_ptr, p->col_idx, p->val, xo, act);
    double primal_res = 0.0, dual_res = 0.0;
    for (int32_t i = 0; i < p->m; ++i) {
        const double lo = p->row_lo[i], hi = p->row_hi[i];
        if (finite_bound(lo)) primal_res = smax(primal_res, lo - act[i]);
        if (finite_bound(hi)) primal_res = smax(primal_res, act[i] - hi);
        const double y_int = obj_sign * yo[i];
        const int at_lo = finite_bound(lo) && fabs(act[i] - lo) < bound_tol;
        const int at_hi = finite_bound(hi) && fabs(act[i] - hi) < bound_tol;
        if (!at_lo && !at_hi) dual_res = smax(dual_res, fabs(y_int));
        else if (at_lo && !at_hi) dual_res = smax(dual_res, smax(0.0, -y_int));
        else if (at_hi && !at_lo) dual_res = smax(dual_res, smax(0.0, y_int));
    }
    csr_multiply_transpose(p->m, p->n, p->row_ptr, p->col_idx, p->val, yo, aty);
    for (int32_t j = 0; j < p->n; ++j) {
        const double r_int = obj_sign * (p->c[j] - aty[j]);
        const double lo = p->col_lo[j], hi = p->col_hi[j];
        const int at_lo = finite_bound(lo) && fabs(xo[j] - lo) < bound_tol;
        const int at_hi = finite_bound(hi) && fabs(xo[j] - hi) < bound_tol;
        if (!at_lo && !at_hi) dual_res = smax(dual_res, fabs(r_int));
        else if (at_lo && !at_hi) dual_res = smax(dual_res, smax(0.0, -r_int));
        else if (at_hi && !at_lo) dual_res = smax(dual_res, smax(0.0, r_int));
    }
    if (rel != NULL) {
        /* Gap in the internal always-minimize sense (objective and duals times
         * obj_sign), where inf over the box is the weak-duality bound for
         * either original sense. The objective constant shifts both sides. */
        double bnorm = 0.0, cnorm = 0.0, pobj = obj_sign * p->obj_const;
        double dobj = obj_sign * p->obj_const;
        for (int32_t i = 0; i < p->m; ++i) {
            if (finite_bound(p->row_lo[i])) bnorm = smax(bnorm, fabs(p->row_lo[i]));
            if (finite_bound(p->row_hi[i])) bnorm = smax(bnorm, fabs(p->row_hi[i]));
        }
        for (int32_t j = 0; j < p->n; ++j) {
            cnorm = smax(cnorm, fabs(p->c[j]));
            pobj += obj_sign * p->c[j] * xo[j];
            dobj += clipped_inf_over_box(obj_sign * (p->c[j] - aty[j]), p->col_lo[j],
                                         p->col_hi[j]);
        }
        for (int32_t i = 0; i < p->m; ++i)
            dobj += clipped_inf_over_box(obj_sign * yo[i], p->row_lo[i], p->row_hi[i]);
        const double gap = fabs(pobj - dobj) / (1.0 + fabs(pobj) + fabs(dobj));
        *rel = smax(smax(primal_res / (1.0 + bnorm), dual_res / (1.0 + cnorm)), gap);
    }
    return smax(primal_res, dual_res);
}

/* The part of v outside the sign its bounds allow a multiplier or reduced
 * cost (internal minimize sense): >= 0 with only a finite lower end, <= 0
 * with only a finite upper end, any sign with both, 0 with neither. */
static double sign_violation(double v, double lo, double hi) {
    const int fl = finite_bound(lo), fh = finite_bound(hi);
    if (fl && fh) return 0.0;
    if (fl) return v < 0.0 ? -v : 0.0;
    if (fh) return v > 0.0 ? v : 0.0;
    return fabs(v);
}

/* Termination rule 2 (engine extension, PDLP's relative KKT error; the
 * reference defines no relative measure): the scaled point (xs, ys) in
 * original units (xo, yo as in original_residual) gives
 *   part[0] = ||row bound violation of A xo||_2 / (1 + ||b||_2)
 *   part[1] = ||(sign violations of y, of c - A^T y)||_2 / (1 + ||c||_2)
 *   part[2] = |p - d| / (1 + |p| + |d|)
 * in the internal minimize sense, b_i = the largest finite |row bound|, d the
 * dual objective on the bounded parts (clipped_inf_over_box), the objective
 * constant added to both p and d. Returns max(part). */
static double pdlp_kkt(const orc_problem* p, double obj_sign, const double* rs, const double* cs,
                       const double* xs, const double* ys, double* xo, double* yo, double* act,
                       double* aty, double part[3]) {
    for (int32_t j = 0; j < p->n; ++j) xo[j] = xs[j] * cs[j];
    for (int32_t i = 0; i < p->m; ++i) {
        yo[i] = ys[i] * obj_sign;
        yo[i] *= rs[i];
    }
    csr_multiply(p->m, p->row_ptr, p->col_idx, p->val, xo, act);
    csr_multiply_transpose(p->m, p->n, p->row_ptr, p->col_idx, p->val, yo, aty);
    double pp = 0.0, dd = 0.0, bn = 0.0, cn = 0.0;
    double pobj = obj_sign * p->obj_const, dobj = obj_sign * p->obj_const;
    for (int32_t i = 0; i < p->m; ++i) {
        const double lo = p->row_lo[i], hi = p->row_hi[i];
        double v = 0.0, b = 0.0;
        if (finite_bound(lo)) {
            v += smax(lo - act[i], 0.0);
            b = fabs(lo);
        }
        if (finite_bound(hi)) {
            v += smax(act[i] - hi, 0.0);
            b = smax(b, fabs(hi));
        }
        pp += v * v;
        bn += b * b;
        const double y_int = obj_sign * yo[i];
        const double dv = sign_violation(y_int, lo, hi);
        dd += dv * dv;
        dobj += clipped_inf_over_box(y_int, lo, hi);
    }
    for (int32_t j = 0; j < p->n; ++j) {
        const double r_int = obj_sign * (p->c[j] - aty[j]);
        const double dv = sign_violation(r_int, p->col_lo[j], p->col_hi[j]);
        dd += dv * dv;
        cn += p->c[j] * p->c[j];
        pobj += obj_sign * p->c[j] * xo[j];
        dobj += clipped_inf_over_box(r_int, p->col_lo[j], p->col_hi[j]);
    }
    part[0] = sqrt(pp) / (1.0 + sqrt(bn));
    part[1] = sqrt(dd) / (1.0 + sqrt(cn));
    part[2] = fabs(pobj - dobj) / (1.0 + fabs(pobj) + fabs(dobj));
    return smax(smax(part[0], part[1]), part[2]);
}

/* The restart measure of restart_rule 2: the l2 norm of the three relative
 * parts of pdlp_kkt. */
static double l2_of_parts(const double part[3]) {
    return sqrt(part[0] * part[0] + part[1] * part[1] + part[2] * part[2]);
}

/* ---------------------------------------------------------------------------
 * Pdhg::solve, src/l1/pdhg.cpp:218-502
 * ------------------------------------------------------------------------- */

#define NEWV(T, k) ((T*)calloc((size_t)(k) + 1, sizeof(T)))

int orc_pdhg_solve(const orc_problem* p, const orc_options* opt, orc_info* info, double* x_out,
                   double* y_out, double* rc_out) {
    memset(info, 0, sizeof *info);
    info->status = ORC_NOT_SOLVED;
    const double t0 = now_seconds();

    char why[200];
    if (!validate(p, why, sizeof why)) { /* pdhg.cpp:223-228 */
        info->status = ORC_NUMERICAL_FAILURE;
        snprintf(info->message, sizeof info->message, "invalid problem: %s", why);
        return 0;
    }
    /* pdhg.cpp:229-237: has_crossed_bounds is unreachable after validate
     * (validate already rejects crossed bounds), kept for the same order. */

    const int32_t m = p->m, n = p->n;
    double* rs = NEWV(double, m);
    double* cs = NEWV(double, n);
    orc_scaling(m, n, p->row_ptr, p->col_idx, p->val, opt, rs, cs); /* pdhg.cpp:240 */
    scaled_problem s;
    build_scaled(p, rs, cs, &s);

    const double obj_sign = p->maximize ? -1.0 : 1.0; /* pdhg.cpp:250-252 */
    double* c = NEWV(double, n);
    for (int32_t j = 0; j < n; ++j) c[j] = s.c[j] * obj_sign;

    const double op_norm = orc_operator_norm(m, n, s.rp, s.ci, s.v, opt->power_iterations);
    info->operator_norm_estimate = op_norm; /* pdhg.cpp:261-265 */
    const double step = (op_norm > 1e-9) ? opt->step_size_safety / op_norm
                                         : opt->step_size_safety;
    double tau = step, sigma = step;
    double omega = 1.0; /* extension: primal weight (reference: tau = sigma) */
    if (opt->primal_weight_update) {
        double cn = 0.0, bn = 0.0;
        for (int32_t j = 0; j < n; ++j) cn += c[j] * c[j];
        for (int32_t i = 0; i < m; ++i) {
            double b = 0.0;
            if (finite_bound(s.row_lo[i])) b = fabs(s.row_lo[i]);
            if (finite_bound(s.row_hi[i])) b = smax(b, fabs(s.row_hi[i]));
            bn += b * b;
        }
        cn = sqrt(cn);
        bn = sqrt(bn);
        if (cn > 1e-10 && bn > 1e-10) omega = cn / bn;
        if (opt->primal_weight0 > 0.0) omega = opt->primal_weight0;
        tau = step / omega;
        sigma = step * omega;
    }

    double* x = NEWV(double, n); /* pdhg.cpp:268-283 */
    double* sl = NEWV(double, m);
    double* y = NEWV(double, m);
    if (opt->x0 != NULL) /* extension: warm start */
        for (int32_t j = 0; j < n; ++j) x[j] = opt->x0[j] / cs[j];
    if (opt->y0 != NULL)
        for (int32_t i = 0; i < m; ++i) y[i] = (opt->y0[i] * obj_sign) / rs[i];
    orc_project_box(n, s.col_lo, s.col_hi, x);
    if (opt->x0 != NULL) csr_multiply(m, s.rp, s.ci, s.v, x, sl);
    orc_project_box(m, s.row_lo, s.row_hi, sl);
    double* x_new = NEWV(double, n);
    double* s_new = NEWV(double, m);
    double* x_bar = NEWV(double, n);
    double* s_bar = NEWV(double, m);
    double* grad = NEWV(double, n);
    double* kb = NEWV(double, m);
    double* x_sum = NEWV(double, n);
    double* y_sum = NEWV(double, m);
    double* x_avg = NEWV(double, n);
    double* y_avg = NEWV(double, m);
    double* act = NEWV(double, m);
    double* aty = NEWV(double, n);
    double* xo = NEWV(double, n);
    double* yo = NEWV(double, m);
    long long since_restart = 0;
    double res_last = INFINITY;
    double res_prev_cand = INFINITY;
    double* x_last = NEWV(double, n); /* restart points for the primal weight */
    double* y_last = NEWV(double, m);
    memcpy(x_last, x, sizeof(double) * (size_t)n);
    memcpy(y_last, y, sizeof(double) * (size_t)m);
    /* extension (halpern): the anchor z_a = (xa, sa, ya) and y before the dual step */
    const int halpern = opt->halpern;
    double* xa = NEWV(double, n);
    double* sa = NEWV(double, m);
    double* ya = NEWV(double, m);
    double* y_old = NEWV(double, m);
    memcpy(xa, x, sizeof(double) * (size_t)n);
    memcpy(sa, sl, sizeof(double) * (size_t)m);
    memcpy(ya, y, sizeof(double) * (size_t)m);
    const double* best_x = NULL;
    const double* best_y = NULL;
    int converged = 0, failed = 0;

    long long it;
    for (it = 0; it < opt->max_iterations; ++it) {
        if (opt->cancel_flag != NULL && *opt->cancel_flag) { /* pdhg.cpp:288 */
            info->status = ORC_CANCELLED;
            break;
        }
        if (opt->time_limit_seconds > 0.0 && now_seconds() - t0 > opt->time_limit_seconds) {
            info->status = ORC_TIME_LIMIT; /* pdhg.cpp:289-293 */
            break;
        }
        if (opt->iter_times != NULL && it < opt->iter_times_cap) opt->iter_times[it] = now_seconds();
        /* pdhg.cpp:295-300 */
        memcpy(grad, c, sizeof(double) * (size_t)n);
        orc_spmv_transpose(m, n, s.rp, s.ci, s.v, -1.0, y, 1.0, grad);
        memcpy(x_new, x, sizeof(double) * (size_t)n);
        axpy(n, -tau, grad, x_new);
        orc_project_box(n, s.col_lo, s.col_hi, x_new);
        /* pdhg.cpp:302-305 */
        memcpy(s_new, sl, sizeof(double) * (size_t)m);
        axpy(m, -tau, y, s_new);
        orc_project_box(m, s.row_lo, s.row_hi, s_new);
        /* pdhg.cpp:307-313 */
        memcpy(x_bar, x_new, sizeof(double) * (size_t)n);
        scale(n, 2.0, x_bar);
        axpy(n, -1.0, x, x_bar);
        memcpy(s_bar, s_new, sizeof(double) * (size_t)m);
        scale(m, 2.0, s_bar);
        axpy(m, -1.0, sl, s_bar);
        /* pdhg.cpp:315-318 */
        if (halpern) memcpy(y_old, y, sizeof(double) * (size_t)m);
        orc_spmv(m, s.rp, s.ci, s.v, -1.0, x_bar, 0.0, kb);
        axpy(m, 1.0, s_bar, kb);
        axpy(m, sigma, kb, y);
        if (halpern) {
            /* T(z) = (x_new, s_new, y) is the candidate (kept in the sums'
             * place, averaged over one term); z moves to the reflected
             * Halpern point w (2 T(z) - z) + (1 - w) z_a, w = (k+1)/(k+2) */
            const double w = (double)(since_restart + 1) / (double)(since_restart + 2);
            const double wa = 1.0 - w;
            memcpy(x_sum, x_new, sizeof(double) * (size_t)n);
            memcpy(y_sum, y, sizeof(double) * (size_t)m);
            for (int32_t j = 0; j < n; ++j) x[j] = w * x_bar[j] + wa * xa[j];
            for (int32_t i = 0; i < m; ++i) {
                sl[i] = w * s_bar[i] + wa * sa[i];
                y[i] = w * (2.0 * y[i] - y_old[i]) + wa * ya[i];
            }
            ++since_restart;
        } else {
            /* pdhg.cpp:320-321 */
            memcpy(x, x_new, sizeof(double) * (size_t)n);
            memcpy(sl, s_new, sizeof(double) * (size_t)m);
            /* pdhg.cpp:323-331 */
            if (since_restart == 0) {
                memcpy(x_sum, x, sizeof(double) * (size_t)n);
                memcpy(y_sum, y, sizeof(double) * (size_t)m);
            } else {
                axpy(n, 1.0, x, x_sum);
                axpy(m, 1.0, y, y_sum);
            }
            ++since_restart;
        }
        if (opt->trace_iters > 0 && it < opt->trace_iters) {
            if (opt->trace_x) memcpy(opt->trace_x + (size_t)it * n, x, sizeof(double) * (size_t)n);
            if (opt->trace_y) memcpy(opt->trace_y + (size_t)it * m, y, sizeof(double) * (size_t)m);
        }

        if ((it + 1) % opt->restart_check_period != 0) continue; /* pdhg.cpp:333-334 */

        /* pdhg.cpp:336-345 */
        const double inv = halpern ? 1.0 : 1.0 / (double)since_restart;
        for (int32_t j = 0; j < n; ++j) x_avg[j] = x_sum[j] * inv;
        for (int32_t i = 0; i < m; ++i) y_avg[i] = y_sum[i] * inv;
        /* restart_rule 2: current and average measured by rule 2's parts */
        double part_cur[3] = {0, 0, 0}, part_avg[3] = {0, 0, 0};
        double cur, avg;
        if (opt->restart_rule == 2) {
            pdlp_kkt(p, obj_sign, rs, cs, x, y, xo, yo, act, aty, part_cur);
            pdlp_kkt(p, obj_sign, rs, cs, x_avg, y_avg, xo, yo, act, aty, part_avg);
            cur = l2_of_parts(part_cur);
            avg = l2_of_parts(part_avg);
        } else {
            cur = kkt_residual(&s, c, x, y, opt->tolerance, act, aty);
            avg = kkt_residual(&s, c, x_avg, y_avg, opt->tolerance, act, aty);
        }
        if (!isfinite(cur) || !isfinite(avg)) { /* pdhg.cpp:347-352 */
            info->status = ORC_NUMERICAL_FAILURE;
            snprintf(info->message, sizeof info->message,
                     "non-finite KKT residual at iteration %lld", it);
            failed = 1;
            break;
        }
        /* pdhg.cpp:354-364; Halpern: the candidate is T(z) */
        const int avg_better = halpern ? 1 : avg <= cur;
        const double* cx = avg_better ? x_avg : x;
        const double* cy = avg_better ? y_avg : y;
        const double bound_tol = opt->tolerance > 1e-6 ? opt->tolerance : 1e-6;
        double rel = 0.0;
        double part[3];
        if (opt->termination_rule == 2)
            rel = (opt->restart_rule == 2)
                      ? smax(smax((avg_better ? part_avg : part_cur)[0],
                                  (avg_better ? part_avg : part_cur)[1]),
                             (avg_better ? part_avg : part_cur)[2])
                      : pdlp_kkt(p, obj_sign, rs, cs, cx, cy, xo, yo, act, aty, part);
        const double orig = original_residual(p, obj_sign, rs, cs, cx, cy, bound_tol, xo, yo,
                                              act, aty,
                                              opt->termination_rule == 1 ? &rel : NULL);
        if (!isfinite(orig)) { /* pdhg.cpp:366-371 */
            info->status = ORC_NUMERICAL_FAILURE;
            snprintf(info->message, sizeof info->message,
                     "non-finite KKT residual (original units) at iteration %lld", it);
            failed = 1;
            break;
        }
        if (opt->checkpoint != NULL) /* pdhg.cpp:378-381 (xo, yo are unscale_to_original) */
            opt->checkpoint(opt->checkpoint_user, it, xo, yo, orig);

        info->relative_kkt = rel;
        const int done = (opt->termination_rule != 0) ? (rel < opt->tolerance)
                                                        : (orig < opt->tolerance);
        if (done) { /* pdhg.cpp:383-389 */
            best_x = cx;
            best_y = cy;
            converged = 1;
            ++it;
            break;
        }
        if (!isfinite(res_last)) res_last = cur; /* pdhg.cpp:391 */
        int restart = 0, to_avg = 1;
        if (opt->restart_rule == 0) {
            restart = avg <= opt->restart_sufficient_decrease * res_last; /* pdhg.cpp:393 */
            if (restart) res_last = avg;
        } else { /* extension: adaptive rule (restart_rule 1 and 2) */
            const double cand = avg_better ? avg : cur;
            const int sufficient = cand <= 0.2 * res_last;
            const int necessary = cand <= 0.8 * res_last && cand > res_prev_cand;
            const int artificial = (double)since_restart >= 0.36 * (double)(it + 1);
            res_prev_cand = cand;
            restart = sufficient || necessary || artificial;
            to_avg = avg_better;
            if (restart) res_last = cand;
        }
        if (restart) { /* pdhg.cpp:394-408 */
            if (to_avg) {
                memcpy(x, x_avg, sizeof(double) * (size_t)n);
                memcpy(y, y_avg, sizeof(double) * (size_t)m);
                orc_project_box(n, s.col_lo, s.col_hi, x);
                csr_multiply(m, s.rp, s.ci, s.v, x_avg, sl);
                orc_project_box(m, s.row_lo, s.row_hi, sl);
            }
            if (halpern) { /* the restart point is the new anchor */
                memcpy(xa, x, sizeof(double) * (size_t)n);
                memcpy(sa, sl, sizeof(double) * (size_t)m);
                memcpy(ya, y, sizeof(double) * (size_t)m);
            }
            if (opt->primal_weight_update) {
                double dx = 0.0, dy = 0.0;
                for (int32_t j = 0; j < n; ++j) {
                    const double d = x[j] - x_last[j];
                    dx += d * d;
                }
                for (int32_t i = 0; i < m; ++i) {
                    const double d = y[i] - y_last[i];
                    dy += d * d;
                }
                dx = sqrt(dx);
                dy = sqrt(dy);
                memcpy(x_last, x, sizeof(double) * (size_t)n);
                memcpy(y_last, y, sizeof(double) * (size_t)m);
                if (dx > 1e-10 && dy > 1e-10) {
                    omega = sqrt(omega * (dy / dx));
                    tau = step / omega;
                    sigma = step * omega;
                }
            }
            since_restart = 0;
            ++info->restarts;
            if (opt->verbose)
                fprintf(stderr, "  [pdhg] restart at iter %lld, residual %.3g\n", it + 1,
                        res_last);
        }
    }
    free(x_last);
    free(y_last);
    free(xa);
    free(sa);
    free(ya);
    free(y_old);
    info->iterations = it;
    info->primal_weight = omega;

    if (!failed) {
        if (best_x == NULL) { /* pdhg.cpp:420-425 */
            best_x = x;
            best_y = y;
        }
        if (converged) info->status = ORC_OPTIMAL;
        else if (info->status == ORC_NOT_SOLVED) info->status = ORC_ITERATION_LIMIT;

        /* unscale_to_original, pdhg.cpp:205-214, 428 */
        for (int32_t j = 0; j < n; ++j) xo[j] = best_x[j] * cs[j];
        for (int32_t i = 0; i < m; ++i) {
            yo[i] = best_y[i] * obj_sign;
            yo[i] *= rs[i];
        }
        /* Problem::evaluate_objective, src/io/problem.cpp:13-19 */
        double acc = p->obj_const;
        for (int32_t j = 0; j < n; ++j) acc += p->c[j] * xo[j];
        info->objective = acc;
        /* pdhg.cpp:434-442 */
        csr_multiply_transpose(m, n, p->row_ptr, p->col_idx, p->val, yo, aty);
        double* rc = NEWV(double, n);
        for (int32_t j = 0; j < n; ++j) rc[j] = p->c[j] - aty[j];
        /* pdhg.cpp:444-457 */
        csr_multiply(m, p->row_ptr, p->col_idx, p->val, xo, act);
        double pinf = 0.0;
        for (int32_t i = 0; i < m; ++i) {
            if (finite_bound(p->row_lo[i])) pinf = smax(pinf, p->row_lo[i] - act[i]);
            if (finite_bound(p->row_hi[i])) pinf = smax(pinf, act[i] - p->row_hi[i]);
        }
        info->primal_infeasibility = pinf;
        /* DualSolution::complementary_slackness_violation, src/l1/duals.cpp:81-113,
         * with bound_tol = max(tol, 1e-6) (pdhg.cpp:459-472); note `<=` here. */
        const double bt = opt->tolerance > 1e-6 ? opt->tolerance : 1e-6;
        double worst = 0.0;
        if (m > 0) {
            for (int32_t i = 0; i < m; ++i) {
                const double lo = p->row_lo[i], hi = p->row_hi[i];
                const int at_lo = finite_bound(lo) && fabs(act[i] - lo) <= bt;
                const int at_hi = finite_bound(hi) && fabs(act[i] - hi) <= bt;
                if (!at_lo && !at_hi) worst = smax(worst, fabs(yo[i]));
            }
        }
        if (n > 0) {
            for (int32_t j = 0; j < n; ++j) {
                const double lo = p->col_lo[j], hi = p->col_hi[j];
                const int at_lo = finite_bound(lo) && fabs(xo[j] - lo) <= bt;
                const int at_hi = finite_bound(hi) && fabs(xo[j] - hi) <= bt;
                if (!at_lo && !at_hi) worst = smax(worst, fabs(rc[j]));
            }
        }
        info->dual_infeasibility = worst;
        /* pdhg.cpp:474-498 */
        double dual_obj = 0.0;
        int fin = 1;
        for (int32_t j = 0; j < n && fin; ++j) {
            const double term = inf_over_box(rc[j], p->col_lo[j], p->col_hi[j]);
            if (!isfinite(term)) { fin = 0; break; }
            dual_obj += term;
        }
        for (int32_t i = 0; i < m && fin; ++i) {
            const double term = inf_over_box(yo[i], p->row_lo[i], p->row_hi[i]);
            if (!isfinite(term)) { fin = 0; break; }
            dual_obj += term;
        }
        if (fin) {
            const double denom = 1.0 + fabs(info->objective) + fabs(dual_obj);
            info->duality_gap = fabs(info->objective - dual_obj) / denom;
        } else {
            info->duality_gap = INFINITY;
        }
        info->has_point = 1;
        if (x_out) memcpy(x_out, xo, sizeof(double) * (size_t)n);
        if (y_out) memcpy(y_out, yo, sizeof(double) * (size_t)m);
        if (rc_out) memcpy(rc_out, rc, sizeof(double) * (size_t)n);
        free(rc);
    }
    if (!failed) info->seconds = now_seconds() - t0; /* pdhg.cpp:500 (early returns leave 0) */

    free(rs); free(cs); free(c); free(x); free(sl); free(y); free(x_new); free(s_new);
    free(x_bar); free(s_bar); free(grad); free(kb); free(x_sum); free(y_sum); free(x_avg);
    free(y_avg); free(act); free(aty); free(xo); free(yo);
    free_scaled(&s);
    return 0;
}

/* ---------------------------------------------------------------------------
 * FarkasCertificate (src/l1/duals.cpp:16-79)
 * ------------------------------------------------------------------------- */

/* term_range (duals.cpp:16-20): mult * [lo, hi], reversed for a negative
 * multiplier, exactly {0} for a zero one. */
static void term_range(double mult, double lo, double hi, double* tlo, double* thi) {
    if (mult == 0.0) {
        *tlo = 0.0;
        *thi = 0.0;
    } else if (mult > 0.0) {
        *tlo = mult * lo;
        *thi = mult * hi;
    } else {
        *tlo = mult * hi;
        *thi = mult * lo;
    }
}

int orc_certifies(const orc_problem* p, const double* y, double slack, double* ranges) {
    /* row_side_range (duals.cpp:36-43): rows in order */
    double rlo = 0.0, rhi = 0.0;
    for (int32_t i = 0; i < p->m; ++i) {
        double tlo, thi;
        term_range(y[i], p->row_lo[i], p->row_hi[i], &tlo, &thi);
        rlo = rlo + tlo;
        rhi = rhi + thi;
    }
    /* column_side_range (duals.cpp:45-69): d = A^T y by a row-major scatter
     * (zero multipliers skipped), then columns in order */
    double* d = (double*)calloc((size_t)p->n + 1, sizeof(double));
    for (int32_t r = 0; r < p->m; ++r) {
        const double yr = y[r];
        if (yr == 0.0) continue;
        for (int32_t k = p->row_ptr[r]; k < p->row_ptr[r + 1]; ++k) d[p->col_idx[k]] += yr * p->val[k];
    }
    double clo = 0.0, chi = 0.0;
    for (int32_t j = 0; j < p->n; ++j) {
        double tlo, thi;
        term_range(d[j], p->col_lo[j], p->col_hi[j], &tlo, &thi);
        clo = clo + tlo;
        chi = chi + thi;
    }
    free(d);
    if (ranges != NULL) {
        ranges[0] = rlo;
        ranges[1] = rhi;
        ranges[2] = clo;
        ranges[3] = chi;
    }
    /* certifies_infeasibility (duals.cpp:71-79): NaN never certifies;
     * Range::disjoint_from (duals.hpp) */
    if (isnan(rlo) || isnan(rhi) || isnan(clo) || isnan(chi)) return 0;
    return (rhi < clo - slack || chi < rlo - slack) ? 1 : 0;
}
