// host_prep.cpp -- see host_prep.hpp. Compiled with -ffp-contract=off so that
// every product and sum rounds separately, like the reference's build.
#include "host_prep.hpp"

#include <cmath>
#include <cstdio>
#include <limits>

namespace pdhg {

namespace {

constexpr double kInf = std::numeric_limits<double>::infinity();

bool finite_bound(double v) { return v > -kInf && v < kInf; }  // problem.hpp:31-33
double smax(double a, double b) { return (a < b) ? b : a; }     // std::max
double safe_sqrt(double v) { return v > 0.0 ? std::sqrt(v) : 1.0; }  // scaling.cpp:11

std::string col_name(int32_t j) { return "C" + std::to_string(j); }
std::string row_name(int32_t i) { return "R" + std::to_string(i); }

}  // namespace

bool validate_lp(const LpView& lp, std::string* why) {
    // Problem::validate (src/io/problem.cpp:50-), in its order.
    if (!std::isfinite(lp.obj_const)) {
        *why = "objective constant is not finite";
        return false;
    }
    for (int32_t j = 0; j < lp.n; ++j) {
        if (!std::isfinite(lp.c[j])) {
            *why = "non-finite objective coefficient in column " + col_name(j);
            return false;
        }
        if (std::isnan(lp.col_lo[j]) || std::isnan(lp.col_hi[j])) {
            *why = "NaN bound on column " + col_name(j);
            return false;
        }
        if (lp.col_lo[j] > lp.col_hi[j]) {
            *why = "crossed bounds on column " + col_name(j);
            return false;
        }
    }
    for (int32_t i = 0; i < lp.m; ++i) {
        if (std::isnan(lp.row_lo[i]) || std::isnan(lp.row_hi[i])) {
            *why = "NaN bound on row " + row_name(i);
            return false;
        }
        if (lp.row_lo[i] > lp.row_hi[i]) {
            *why = "crossed bounds on row " + row_name(i);
            return false;
        }
    }
    // CsrMatrix::validate (src/l0/sparse.cpp:94-128).
    if (lp.rp[0] != 0) {
        *why = "row_ptr does not start at 0";
        return false;
    }
    if (lp.rp[lp.m] != lp.nnz) {
        *why = "row_ptr does not end at nnz";
        return false;
    }
    for (int32_t r = 0; r < lp.m; ++r) {
        const int32_t b = lp.rp[r], e = lp.rp[r + 1];
        if (b > e) {
            *why = "row_ptr is not monotone";
            return false;
        }
        if (b < 0 || e > lp.nnz) {  // guards the reads below for any row_ptr
            *why = "row_ptr is not monotone";
            return false;
        }
        for (int32_t k = b; k < e; ++k) {
            const int32_t c = lp.ci[k];
            if (c < 0 || c >= lp.n) {
                *why = "column index out of range";
                return false;
            }
            if (k > b && lp.ci[k - 1] >= c) {
                *why = "column indices not strictly ascending";
                return false;
            }
            if (!std::isfinite(lp.v[k])) {
                *why = "non-finite coefficient";
                return false;
            }
        }
    }
    why->clear();
    return true;
}

void equilibrate(const HostCsr& A, const ScalingParams& p, std::vector<double>* rs_out,
                 std::vector<double>* cs_out) {
    std::vector<double>& rs = *rs_out;
    std::vector<double>& cs = *cs_out;
    rs.assign(static_cast<size_t>(A.rows), 1.0);
    cs.assign(static_cast<size_t>(A.cols), 1.0);
    if (p.apply_ruiz) {  // scaling.cpp:36-74
        std::vector<double> row_max(static_cast<size_t>(A.rows)), col_max(static_cast<size_t>(A.cols));
        for (int sweep = 0; sweep < p.ruiz_iterations; ++sweep) {
            std::fill(row_max.begin(), row_max.end(), 0.0);
            std::fill(col_max.begin(), col_max.end(), 0.0);
            for (int32_t r = 0; r < A.rows; ++r) {
                for (int32_t k = A.rp[r]; k < A.rp[r + 1]; ++k) {
                    const int32_t c = A.ci[k];
                    const double s = std::fabs(A.v[k]) * rs[r] * cs[c];
                    row_max[r] = smax(row_max[r], s);
                    col_max[c] = smax(col_max[c], s);
                }
            }
            double worst = 0.0;
            for (int32_t r = 0; r < A.rows; ++r) {
                if (row_max[r] > 0.0) {
                    rs[r] /= safe_sqrt(row_max[r]);
                    worst = smax(worst, std::fabs(row_max[r] - 1.0));
                }
            }
            for (int32_t c = 0; c < A.cols; ++c) {
                if (col_max[c] > 0.0) {
                    cs[c] /= safe_sqrt(col_max[c]);
                    worst = smax(worst, std::fabs(col_max[c] - 1.0));
                }
            }
            if (worst < p.ruiz_tolerance) break;
        }
    }
    if (p.apply_pock_chambolle) {  // scaling.cpp:80-101
        const double a = p.pock_chambolle_alpha;
        std::vector<double> row_sum(static_cast<size_t>(A.rows), 0.0),
            col_sum(static_cast<size_t>(A.cols), 0.0);
        for (int32_t r = 0; r < A.rows; ++r) {
            for (int32_t k = A.rp[r]; k < A.rp[r + 1]; ++k) {
                const int32_t c = A.ci[k];
                const double mag = std::fabs(A.v[k]) * rs[r] * cs[c];
                if (mag <= 0.0) continue;
                row_sum[r] += std::pow(mag, 2.0 - a);
                col_sum[c] += std::pow(mag, a);
            }
        }
        for (int32_t r = 0; r < A.rows; ++r)
            if (row_sum[r] > 0.0) rs[r] /= safe_sqrt(row_sum[r]);
        for (int32_t c = 0; c < A.cols; ++c)
            if (col_sum[c] > 0.0) cs[c] /= safe_sqrt(col_sum[c]);
    }
}

void build_scaled(const HostLp& lp, const std::vector<double>& rs, const std::vector<double>& cs,
                  HostLp* out) {
    out->m = lp.m;
    out->n = lp.n;
    out->obj_const = lp.obj_const;
    out->maximize = lp.maximize;
    out->c.resize(static_cast<size_t>(lp.n));
    out->col_lo.resize(static_cast<size_t>(lp.n));
    out->col_hi.resize(static_cast<size_t>(lp.n));
    out->row_lo.resize(static_cast<size_t>(lp.m));
    out->row_hi.resize(static_cast<size_t>(lp.m));
    for (int32_t j = 0; j < lp.n; ++j) {  // scaling.cpp:172-183
        const double c = cs[j];
        out->c[j] = lp.c[j] * c;
        out->col_lo[j] = finite_bound(lp.col_lo[j]) ? lp.col_lo[j] / c : lp.col_lo[j];
        out->col_hi[j] = finite_bound(lp.col_hi[j]) ? lp.col_hi[j] / c : lp.col_hi[j];
    }
    for (int32_t i = 0; i < lp.m; ++i) {  // scaling.cpp:184-192
        const double r = rs[i];
        out->row_lo[i] = finite_bound(lp.row_lo[i]) ? lp.row_lo[i] * r : lp.row_lo[i];
        out->row_hi[i] = finite_bound(lp.row_hi[i]) ? lp.row_hi[i] * r : lp.row_hi[i];
    }
    // Scaling::apply (scaling.cpp:110-133) then the from_triplets rebuild
    // (scaling.cpp:194-204), which drops |v| <= tol::numeric_zero = 1e-14.
    HostCsr& S = out->A;
    S.rows = lp.A.rows;
    S.cols = lp.A.cols;
    S.rp.assign(static_cast<size_t>(lp.m) + 1, 0);
    S.ci.clear();
    S.v.clear();
    S.ci.reserve(lp.A.ci.size());
    S.v.reserve(lp.A.v.size());
    for (int32_t r = 0; r < lp.m; ++r) {
        const double rr = rs[r];
        for (int32_t k = lp.A.rp[r]; k < lp.A.rp[r + 1]; ++k) {
            const double v = lp.A.v[k] * rr * cs[lp.A.ci[k]];
            if (std::fabs(v) <= 1e-14) continue;
            S.ci.push_back(lp.A.ci[k]);
            S.v.push_back(v);
        }
        S.rp[r + 1] = static_cast<int32_t>(S.ci.size());
    }
}

void bin_rows(const std::vector<int32_t>& rp, int long_threshold, std::vector<int32_t>* long_rows,
              int32_t* n_short, int* vw) {
    long_rows->clear();
    const int32_t rows = static_cast<int32_t>(rp.size()) - 1;
    int64_t short_nnz = 0;
    int32_t shorts = 0;
    for (int32_t r = 0; r < rows; ++r) {
        const int32_t len = rp[r + 1] - rp[r];
        if (len > long_threshold) {
            long_rows->push_back(r);
        } else {
            ++shorts;
            short_nnz += len;
        }
    }
    *n_short = shorts;
    const double mean = shorts > 0 ? static_cast<double>(short_nnz) / shorts : 0.0;
    // Lanes per short row: about half the mean length, a power of two in [1, 32].
    int w = 1;
    while (w < 32 && 2.0 * w <= mean / 2.0 + 1e-9) w *= 2;
    *vw = w;
}

}  // namespace pdhg
