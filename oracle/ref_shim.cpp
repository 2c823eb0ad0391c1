// ref_shim.cpp -- TEST INFRASTRUCTURE ONLY.
//
// An extern "C" face over the UNMODIFIED reference PDHG path, compiled by
// oracle/Makefile together with the reference's own sources into
// oracle/_ref/libsovref.so. It lets the Python tests and bench.py's reference
// arm call sov::Pdhg::solve on the reference's Host backend through ctypes,
// and read the reference's LP/MPS fixtures into plain CSR arrays.
//
// Nothing here changes what the reference computes. Per-iteration iterates are
// observed through a Backend decorator (RecordingBackend): the Backend virtuals
// are public (include/sovereign/backend.hpp:82-165), so the decorator forwards
// every call to the Host backend and only watches the call sequence of the
// PDHG loop (src/l1/pdhg.cpp:295-330).
#include <chrono>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "pdhg_oracle.h"  // the shared orc_problem / orc_options / orc_info structs
#include "sovereign/backend.hpp"
#include "sovereign/duals.hpp"
#include "sovereign/io.hpp"
#include "sovereign/pdhg.hpp"
#include "sovereign/problem.hpp"
#include "sovereign/scaling.hpp"

namespace {

using Clock = std::chrono::steady_clock;

// Forwards every primitive to the Host backend; records x after the primal
// projection (pdhg.cpp:300) and y after the dual axpy (pdhg.cpp:318) for the
// first `trace_iters` iterations, and stamps the start of each iteration's
// primal SpMV (pdhg.cpp:297) so the loop can be timed without setup cost.
class RecordingBackend final : public sov::Backend {
public:
    RecordingBackend(std::unique_ptr<sov::Backend> inner, int n, int m, int trace_iters,
                     double* tx, double* ty, double* times, long long times_cap)
        : in_(std::move(inner)), n_(n), m_(m), trace_(trace_iters), tx_(tx), ty_(ty),
          times_(times), times_cap_(times_cap) {}

    std::string_view name() const noexcept override { return in_->name(); }
    sov::BackendKind kind() const noexcept override { return in_->kind(); }
    bool has_discrete_memory() const noexcept override { return in_->has_discrete_memory(); }
    std::string_view device_description() const noexcept override {
        return in_->device_description();
    }
    sov::Status allocate(std::size_t b, void** o) override { return in_->allocate(b, o); }
    void deallocate(void* p) noexcept override { in_->deallocate(p); }
    sov::Status copy_to_device(const void* s, void* d, std::size_t b) override {
        return in_->copy_to_device(s, d, b);
    }
    sov::Status copy_to_host(const void* s, void* d, std::size_t b) override {
        return in_->copy_to_host(s, d, b);
    }
    sov::Status copy_device_to_device(const void* s, void* d, std::size_t b) override {
        return in_->copy_device_to_device(s, d, b);
    }
    sov::Status fill_zero(void* d, std::size_t b) override { return in_->fill_zero(d, b); }
    sov::Status synchronize() override { return in_->synchronize(); }
    sov::Status axpy(sov::Idx n, sov::Real a, const sov::Real* x, sov::Real* y) override {
        const sov::Status s = in_->axpy(n, a, x, y);
        if (loop_ && want_y_ > 0 && --want_y_ == 0) {
            if (yi_ < trace_ && ty_ != nullptr)
                std::memcpy(ty_ + static_cast<std::size_t>(yi_) * m_, y, sizeof(double) * m_);
            ++yi_;
        }
        return s;
    }
    sov::Status scale(sov::Idx n, sov::Real a, sov::Real* x) override { return in_->scale(n, a, x); }
    sov::Status dot(sov::Idx n, const sov::Real* x, const sov::Real* y, sov::Real* r) override {
        return in_->dot(n, x, y, r);
    }
    sov::Status norm2(sov::Idx n, const sov::Real* x, sov::Real* r) override {
        return in_->norm2(n, x, r);
    }
    sov::Status max_abs(sov::Idx n, const sov::Real* x, sov::Real* r) override {
        return in_->max_abs(n, x, r);
    }
    sov::Status spmv(const sov::CsrView& A, sov::Real a, const sov::Real* x, sov::Real b,
                     sov::Real* y) override {
        if (loop_) want_y_ = 2;  // axpy(k += s_bar), then axpy(y += sigma k)
        return in_->spmv(A, a, x, b, y);
    }
    sov::Status spmv_transpose(const sov::CsrView& A, sov::Real a, const sov::Real* x,
                               sov::Real b, sov::Real* y) override {
        if (loop_) {
            want_x_ = true;
            const auto t = Clock::now();
            if (loop_calls_ == 0) first_ = t;
            last_ = t;
            if (times_ != nullptr && loop_calls_ < times_cap_)
                times_[loop_calls_] = std::chrono::duration<double>(t.time_since_epoch()).count();
            ++loop_calls_;
        }
        return in_->spmv_transpose(A, a, x, b, y);
    }
    sov::Status project_box(sov::Idx n, const sov::Real* lo, const sov::Real* hi,
                            sov::Real* x) override {
        const sov::Status s = in_->project_box(n, lo, hi, x);
        if (!loop_) {
            // The two initial projections (pdhg.cpp:269-270) end the setup phase.
            if (++setup_projections_ == 2) loop_ = true;
        } else if (want_x_) {
            want_x_ = false;
            if (xi_ < trace_ && tx_ != nullptr)
                std::memcpy(tx_ + static_cast<std::size_t>(xi_) * n_, x, sizeof(double) * n_);
            ++xi_;
        }
        return s;
    }

    // Seconds from the first to the last loop iteration start, and how many
    // iteration starts that span covers.
    double loop_seconds() const {
        return loop_calls_ > 1 ? std::chrono::duration<double>(last_ - first_).count() : 0.0;
    }
    long long loop_spans() const { return loop_calls_ > 1 ? loop_calls_ - 1 : 0; }

private:
    std::unique_ptr<sov::Backend> in_;
    int n_, m_, trace_;
    double* tx_;
    double* ty_;
    double* times_;
    long long times_cap_;
    bool loop_ = false, want_x_ = false;
    int want_y_ = 0, setup_projections_ = 0;
    long long xi_ = 0, yi_ = 0, loop_calls_ = 0;
    Clock::time_point first_{}, last_{};
};

sov::Problem build_problem(const orc_problem* p) {
    sov::Problem::Builder b;
    b.set_sense(p->maximize ? sov::ObjSense::Maximize : sov::ObjSense::Minimize);
    b.set_objective_constant(p->obj_const);
    for (int32_t j = 0; j < p->n; ++j) {
        const sov::Idx col = b.add_column("C" + std::to_string(j));
        b.set_objective_coefficient(col, p->c[j]);
        b.set_column_bounds(col, p->col_lo[j], p->col_hi[j]);
    }
    for (int32_t i = 0; i < p->m; ++i)
        b.add_row("R" + std::to_string(i), p->row_lo[i], p->row_hi[i]);
    for (int32_t r = 0; r < p->m; ++r)
        for (int32_t k = p->row_ptr[r]; k < p->row_ptr[r + 1]; ++k)
            b.add_coefficient(r, p->col_idx[k], p->val[k]);
    return b.finish();
}

sov::PdhgOptions to_options(const orc_options* o) {
    sov::PdhgOptions opt;
    opt.tolerance = o->tolerance;
    opt.max_iterations = o->max_iterations;
    opt.time_limit_seconds = o->time_limit_seconds;
    opt.restart_check_period = o->restart_check_period;
    opt.restart_sufficient_decrease = o->restart_sufficient_decrease;
    opt.step_size_safety = o->step_size_safety;
    opt.power_iterations = o->power_iterations;
    opt.verbose = o->verbose != 0;
    if (o->checkpoint != nullptr) {
        const orc_checkpoint_fn fn = o->checkpoint;
        void* user = o->checkpoint_user;
        opt.checkpoint = [fn, user](long long it, const std::vector<sov::Real>& x,
                                    const std::vector<sov::Real>& y, sov::Real res) {
            fn(user, it, x.data(), y.data(), res);
        };
    }
    return opt;
}

struct Loaded {
    sov::Problem problem;
    std::vector<sov::ReaderWarning> warnings;
};

}  // namespace

extern "C" {

// sov::Pdhg(opt).solve(problem, HostBackend) -- the stock reference call
// (tests/test_pdhg.cpp:20-25). loop_stats (optional, 2 doubles) receives the
// timed loop span in seconds and the number of iterations it covers.
int ref_pdhg_solve(const orc_problem* p, const orc_options* o, orc_info* info, double* x,
                   double* y, double* rc, double* loop_stats) {
    std::memset(info, 0, sizeof *info);
    try {
        const sov::Problem problem = build_problem(p);
        RecordingBackend backend(sov::make_backend(sov::BackendKind::Host), p->n, p->m,
                                 o->trace_iters, o->trace_x, o->trace_y, o->iter_times,
                                 o->iter_times_cap);
        sov::CancellationToken token;
        const sov::Pdhg pdhg(to_options(o));
        const sov::PdhgResult r = pdhg.solve(problem, backend, &token);
        info->status = static_cast<int>(r.status);
        info->objective = r.objective;
        info->primal_infeasibility = r.primal_infeasibility;
        info->dual_infeasibility = r.dual_infeasibility;
        info->duality_gap = r.duality_gap;
        info->iterations = r.iterations;
        info->restarts = r.restarts;
        info->seconds = r.seconds;
        info->operator_norm_estimate = r.operator_norm_estimate;
        // Both NumericalFailure exits return before the point is filled in
        // (pdhg.cpp:223-237, 347-371); every other exit reports one.
        info->has_point = r.status != sov::PdhgStatus::NumericalFailure;
        std::snprintf(info->message, sizeof info->message, "%s", r.message.c_str());
        if (info->has_point) {
            if (x && !r.primal.empty()) std::memcpy(x, r.primal.data(), sizeof(double) * p->n);
            if (y && !r.dual.empty()) std::memcpy(y, r.dual.data(), sizeof(double) * p->m);
            if (rc && !r.reduced_costs.empty())
                std::memcpy(rc, r.reduced_costs.data(), sizeof(double) * p->n);
        }
        if (loop_stats != nullptr) {
            loop_stats[0] = backend.loop_seconds();
            loop_stats[1] = static_cast<double>(backend.loop_spans());
        }
        return 0;
    } catch (const std::exception& e) {
        std::snprintf(info->message, sizeof info->message, "exception: %s", e.what());
        return 1;
    }
}

// FarkasCertificate{y}.certifies_infeasibility(problem, slack) and its two
// ranges (src/l1/duals.cpp:36-79): ranges[0..3] = row-side lo, hi, column-side
// lo, hi. Returns 1 when the ranges are disjoint by more than `slack`, 0 when
// not, -1 on an exception.
int ref_certifies(const orc_problem* p, const double* y, double slack, double* ranges) {
    try {
        const sov::Problem problem = build_problem(p);
        sov::FarkasCertificate cert;
        cert.row_multipliers.assign(y, y + p->m);
        const auto rr = cert.row_side_range(problem);
        const auto cr = cert.column_side_range(problem);
        if (ranges != nullptr) {
            ranges[0] = rr.lo;
            ranges[1] = rr.hi;
            ranges[2] = cr.lo;
            ranges[3] = cr.hi;
        }
        return cert.certifies_infeasibility(problem, slack) ? 1 : 0;
    } catch (const std::exception&) {
        return -1;
    }
}

// Scaling::equilibrate(CsrMatrix) (src/l1/scaling.cpp:19-104).
int ref_scaling(int32_t m, int32_t n, int64_t nnz, const int32_t* rp, const int32_t* ci,
                const double* val, const orc_options* o, double* rs, double* cs) {
    try {
        std::vector<sov::Idx> r(rp, rp + m + 1), c(ci, ci + nnz);
        std::vector<sov::Real> v(val, val + nnz);
        const sov::CsrMatrix A(m, n, std::move(r), std::move(c), std::move(v));
        sov::ScalingOptions so;
        so.ruiz_iterations = o->ruiz_iterations;
        so.ruiz_tolerance = o->ruiz_tolerance;
        so.pock_chambolle_alpha = o->pock_chambolle_alpha;
        so.apply_ruiz = o->apply_ruiz != 0;
        so.apply_pock_chambolle = o->apply_pock_chambolle != 0;
        const sov::Scaling s = sov::Scaling::equilibrate(A, so);
        std::memcpy(rs, s.row_scale().data(), sizeof(double) * m);
        std::memcpy(cs, s.col_scale().data(), sizeof(double) * n);
        return 0;
    } catch (const std::exception&) {
        return 1;
    }
}

// Host backend SpMV / SpMV-transpose / project_box (src/l0/backend_host.cpp:409-458),
// through DeviceCsr/DeviceBuffer like the reference's own backend tests.
int ref_backend_spmv(int transpose, int32_t m, int32_t n, int64_t nnz, const int32_t* rp,
                     const int32_t* ci, const double* val, double alpha, const double* x,
                     double beta, double* y) {
    try {
        auto be = sov::make_backend(sov::BackendKind::Host);
        std::vector<sov::Idx> r(rp, rp + m + 1), c(ci, ci + nnz);
        std::vector<sov::Real> v(val, val + nnz);
        const sov::CsrMatrix A(m, n, std::move(r), std::move(c), std::move(v));
        sov::DeviceCsr dA = sov::DeviceCsr::upload(*be, A);
        const int nx = transpose ? m : n, ny = transpose ? n : m;
        sov::DeviceBuffer dx = sov::DeviceBuffer::upload(*be, std::vector<double>(x, x + nx));
        sov::DeviceBuffer dy = sov::DeviceBuffer::upload(*be, std::vector<double>(y, y + ny));
        const sov::Status s = transpose ? be->spmv_transpose(dA.view(), alpha, dx.data(), beta, dy.data())
                                        : be->spmv(dA.view(), alpha, dx.data(), beta, dy.data());
        if (s != sov::Status::Ok) return 2;
        const std::vector<double> out = dy.to_host();
        std::memcpy(y, out.data(), sizeof(double) * ny);
        return 0;
    } catch (const std::exception&) {
        return 1;
    }
}

// read_lp_string / read_mps_string (include/sovereign/io.hpp:57-64) into a handle.
void* ref_read_model_string(const char* text, int is_mps) {
    try {
        sov::ReadResult r = is_mps ? sov::read_mps_string(text) : sov::read_lp_string(text);
        return new Loaded{std::move(r.problem), std::move(r.warnings)};
    } catch (const std::exception&) {
        return nullptr;
    }
}

// read_mps_string(text, MpsOptions, origin) with the options spelled out; on
// an error the handle is null and err gets e.what().
void* ref_read_mps(const char* text, size_t len, const char* origin, int keep_lower_at_zero,
                   int keep_free_rows, char* err, size_t err_cap) {
    err[0] = '\0';
    try {
        sov::MpsOptions o;
        o.negative_upper_bound = keep_lower_at_zero
                                     ? sov::NegativeUpperBoundRule::KeepLowerAtZero
                                     : sov::NegativeUpperBoundRule::LowerBecomesMinusInfinity;
        o.keep_free_rows = keep_free_rows != 0;
        sov::ReadResult r = sov::read_mps_string(std::string(text, len), o, origin);
        return new Loaded{std::move(r.problem), std::move(r.warnings)};
    } catch (const std::exception& e) {
        std::strncpy(err, e.what(), err_cap - 1);
        err[err_cap - 1] = '\0';
        return nullptr;
    }
}

void ref_model_kinds(void* h, uint8_t* is_integer) {
    const sov::Problem& p = static_cast<Loaded*>(h)->problem;
    for (sov::Idx j = 0; j < p.num_cols(); ++j)
        is_integer[j] = p.col_kind()[j] == sov::VarKind::Integer ? 1 : 0;
}

const char* ref_model_name(void* h) { return static_cast<Loaded*>(h)->problem.name().c_str(); }
const char* ref_model_objective_name(void* h) {
    return static_cast<Loaded*>(h)->problem.objective_name().c_str();
}
const char* ref_model_row_name(void* h, int32_t i) {
    return static_cast<Loaded*>(h)->problem.row_names()[i].c_str();
}
const char* ref_model_col_name(void* h, int32_t j) {
    return static_cast<Loaded*>(h)->problem.col_names()[j].c_str();
}
int32_t ref_model_n_warnings(void* h) {
    return static_cast<int32_t>(static_cast<Loaded*>(h)->warnings.size());
}
void ref_model_warning(void* h, int32_t k, int64_t* line, const char** section,
                       const char** message) {
    const sov::ReaderWarning& w = static_cast<Loaded*>(h)->warnings[static_cast<size_t>(k)];
    *line = w.line;
    *section = w.section.c_str();
    *message = w.message.c_str();
}

void ref_model_shape(void* h, int32_t* m, int32_t* n, int64_t* nnz, int* maximize,
                     double* obj_const) {
    const sov::Problem& p = static_cast<Loaded*>(h)->problem;
    *m = p.num_rows();
    *n = p.num_cols();
    *nnz = p.num_nonzeros();
    *maximize = p.sense() == sov::ObjSense::Maximize;
    *obj_const = p.objective_constant();
}

void ref_model_arrays(void* h, int32_t* rp, int32_t* ci, double* val, double* c, double* col_lo,
                      double* col_hi, double* row_lo, double* row_hi) {
    const sov::Problem& p = static_cast<Loaded*>(h)->problem;
    const sov::CsrMatrix& A = p.matrix();
    std::memcpy(rp, A.row_ptr().data(), sizeof(int32_t) * (A.rows() + 1));
    std::memcpy(ci, A.col_idx().data(), sizeof(int32_t) * A.nnz());
    std::memcpy(val, A.values().data(), sizeof(double) * A.nnz());
    std::memcpy(c, p.objective().data(), sizeof(double) * p.num_cols());
    std::memcpy(col_lo, p.col_lower().data(), sizeof(double) * p.num_cols());
    std::memcpy(col_hi, p.col_upper().data(), sizeof(double) * p.num_cols());
    std::memcpy(row_lo, p.row_lower().data(), sizeof(double) * p.num_rows());
    std::memcpy(row_hi, p.row_upper().data(), sizeof(double) * p.num_rows());
}

void ref_model_free(void* h) { delete static_cast<Loaded*>(h); }

}  // extern "C"
