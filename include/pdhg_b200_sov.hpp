/*
 * pdhg_b200_sov.hpp -- sov::PdhgB200, the reference's PDHG interface
 * (sov::Pdhg, include/sovereign/pdhg.hpp:155-172) over the B200 engine's C-ABI
 * (pdhg_b200.h). Header-only; include it inside the reference's source tree
 * (it uses sov::Problem, sov::PdhgOptions, sov::PdhgResult, sov::Backend,
 * sov::CancellationToken, sov::Error) and link libpdhg_b200.so.
 *
 * Drop-in: the same constructor argument, the same solve() signature and
 * result, the same options with the reference's defaults. The Backend argument
 * is accepted and ignored: the engine owns its device. By default the engine
 * runs in PDHG_PREC_FP64_EXACT, which reproduces the reference's Host backend
 * bit for bit; a second constructor argument selects the fast precisions.
 * Engine errors (no device, CUDA failure) throw sov::Error with the matching
 * sov::Status, like the reference's backend errors; solver outcomes come back
 * in PdhgResult::status and ::message, never as exceptions (pdhg.cpp:223-237).
 * Validation messages name rows and columns by the problem's own names.
 *
 * sov::MpsModelB200 is the MPS reader over the engine's pdhg_read_mps: the
 * model sov::read_mps / read_mps_string (include/sovereign/io.hpp:57-59) would
 * build, with the same warnings and errors (sov::Error with the reference's
 * message). to_read_result() rebuilds it as a sov::ReadResult through
 * sov::Problem::Builder for code that needs a sov::Problem;
 * PdhgB200::solve(model, ...) hands the reader's arrays to the engine without
 * that rebuild.
 */
#pragma once

#include <atomic>
#include <chrono>
#include <cstring>
#include <memory>
#include <string>
#include <thread>
#include <vector>

#include "pdhg_b200.h"
#include "sovereign/cancellation.hpp"
#include "sovereign/io.hpp"
#include "sovereign/pdhg.hpp"
#include "sovereign/problem.hpp"
#include "sovereign/status.hpp"

namespace sov {

class MpsModelB200 {
public:
    // read_mps_string(text, options, origin) (io.hpp:58-59); threads 0 = all.
    static MpsModelB200 read_string(const std::string& text, const MpsOptions& options = {},
                                    const std::string& origin = "<string>", int threads = 0) {
        pdhg_mps_options o = convert(options, threads);
        pdhg_model* raw = nullptr;
        char err[4096];
        if (pdhg_read_mps(text.data(), text.size(), origin.c_str(), &o, &raw, err, sizeof err) !=
            PDHG_OK)
            throw Error(std::string(err));
        return MpsModelB200(raw);
    }
    // read_mps(path, options) (io.hpp:57).
    static MpsModelB200 read_file(const std::string& path, const MpsOptions& options = {},
                                  int threads = 0) {
        pdhg_mps_options o = convert(options, threads);
        pdhg_model* raw = nullptr;
        char err[4096];
        if (pdhg_read_mps_file(path.c_str(), &o, &raw, err, sizeof err) != PDHG_OK)
            throw Error(std::string(err));
        return MpsModelB200(raw);
    }

    const pdhg_model* get() const noexcept { return model_.get(); }
    const pdhg_model_info& info() const noexcept { return info_; }
    std::string row_name(int32_t i) const { return pdhg_model_row_name(model_.get(), i); }
    std::string col_name(int32_t j) const { return pdhg_model_col_name(model_.get(), j); }

    std::vector<ReaderWarning> warnings() const {
        std::vector<ReaderWarning> out;
        for (int32_t k = 0; k < info_.warnings; ++k) {
            int64_t line = 0;
            const char* section = nullptr;
            const char* message = nullptr;
            pdhg_model_warning(model_.get(), k, &line, &section, &message);
            out.push_back(ReaderWarning{static_cast<int>(line), section, message});
        }
        return out;
    }

    // The same model as a sov::ReadResult, through sov::Problem::Builder in
    // file order (rows, then columns with bounds, kinds and costs, then the
    // matrix row by row).
    ReadResult to_read_result() const {
        const int32_t *rp = nullptr, *ci = nullptr;
        const double *v = nullptr, *c = nullptr, *cl = nullptr, *cu = nullptr, *rl = nullptr,
                     *ru = nullptr;
        const uint8_t* integer = nullptr;
        pdhg_model_arrays(model_.get(), &rp, &ci, &v, &c, &cl, &cu, &rl, &ru, &integer);
        Problem::Builder b;
        b.set_name(pdhg_model_name(model_.get()));
        b.set_sense(info_.maximize ? ObjSense::Maximize : ObjSense::Minimize);
        b.set_objective_name(pdhg_model_objective_name(model_.get()));
        b.set_objective_constant(info_.obj_const);
        for (int32_t i = 0; i < info_.m; ++i) b.add_row(row_name(i), rl[i], ru[i]);
        for (int32_t j = 0; j < info_.n; ++j) {
            const Idx col = b.add_column(col_name(j));
            b.set_column_bounds(col, cl[j], cu[j]);
            if (integer[j]) b.set_column_kind(col, VarKind::Integer);
            b.set_objective_coefficient(col, c[j]);
        }
        for (int32_t i = 0; i < info_.m; ++i)
            for (int32_t k = rp[i]; k < rp[i + 1]; ++k) b.add_coefficient(i, ci[k], v[k]);
        ReadResult r;
        r.problem = b.finish();
        r.warnings = warnings();
        r.format = "mps";
        return r;
    }

private:
    explicit MpsModelB200(pdhg_model* m) : model_(m, pdhg_model_free) {
        pdhg_model_get_info(m, &info_);
    }
    static pdhg_mps_options convert(const MpsOptions& options, int threads) {
        pdhg_mps_options o;
        pdhg_default_mps_options(&o);
        o.negative_upper_bound =
            options.negative_upper_bound == NegativeUpperBoundRule::KeepLowerAtZero ? 1 : 0;
        o.keep_free_rows = options.keep_free_rows ? 1 : 0;
        o.threads = threads;
        return o;
    }
    std::shared_ptr<pdhg_model> model_;
    pdhg_model_info info_{};
};

class PdhgB200 {
public:
    explicit PdhgB200(PdhgOptions options = {}, int precision = PDHG_PREC_FP64_EXACT,
                      int device = 0)
        : options_(std::move(options)), precision_(precision), device_(device) {}

    PdhgResult solve(const Problem& problem, Backend& /*backend*/,
                     const CancellationToken* cancel = nullptr) const {
        pdhg_ctx* raw = nullptr;
        check(pdhg_create(device_, &raw), nullptr, "pdhg_create");
        std::unique_ptr<pdhg_ctx, int (*)(pdhg_ctx*)> ctx(raw, pdhg_destroy);
        const CsrMatrix& A = problem.matrix();
        const int32_t m = static_cast<int32_t>(problem.num_rows());
        const int32_t n = static_cast<int32_t>(problem.num_cols());
        std::vector<int32_t> rp32, ci32;  // only for a 64-bit-index build
        const int32_t* rp = nullptr;
        const int32_t* ci = nullptr;
        if constexpr (sizeof(Idx) == sizeof(int32_t)) {
            rp = reinterpret_cast<const int32_t*>(A.row_ptr().data());
            ci = reinterpret_cast<const int32_t*>(A.col_idx().data());
        } else {
            rp32.assign(A.row_ptr().begin(), A.row_ptr().end());
            ci32.assign(A.col_idx().begin(), A.col_idx().end());
            rp = rp32.data();
            ci = ci32.data();
        }
        check(pdhg_load_problem(ctx.get(), m, n, A.nnz(), rp, ci, A.values().data(),
                                problem.objective().data(), problem.objective_constant(),
                                problem.sense() == ObjSense::Maximize ? 1 : 0,
                                problem.col_lower().data(), problem.col_upper().data(),
                                problem.row_lower().data(), problem.row_upper().data()),
              ctx.get(), "pdhg_load_problem");
        return run(ctx.get(), m, n, cancel, [&](bool column, long idx) -> std::string {
            const auto names = column ? problem.col_names() : problem.row_names();
            return idx >= 0 && static_cast<std::size_t>(idx) < names.size()
                       ? names[static_cast<std::size_t>(idx)]
                       : std::string();
        });
    }

    // The model read by MpsModelB200, its arrays loaded as they are (no
    // sov::Problem in between); messages name rows and columns as the file does.
    PdhgResult solve(const MpsModelB200& model, Backend& /*backend*/,
                     const CancellationToken* cancel = nullptr) const {
        pdhg_ctx* raw = nullptr;
        check(pdhg_create(device_, &raw), nullptr, "pdhg_create");
        std::unique_ptr<pdhg_ctx, int (*)(pdhg_ctx*)> ctx(raw, pdhg_destroy);
        const pdhg_model_info& mi = model.info();
        const int32_t *rp = nullptr, *ci = nullptr;
        const double *v = nullptr, *c = nullptr, *cl = nullptr, *cu = nullptr, *rl = nullptr,
                     *ru = nullptr;
        pdhg_model_arrays(model.get(), &rp, &ci, &v, &c, &cl, &cu, &rl, &ru, nullptr);
        check(pdhg_load_problem(ctx.get(), mi.m, mi.n, mi.nnz, rp, ci, v, c, mi.obj_const,
                                mi.maximize, cl, cu, rl, ru),
              ctx.get(), "pdhg_load_problem");
        return run(ctx.get(), mi.m, mi.n, cancel, [&](bool column, long idx) -> std::string {
            const long count = column ? mi.n : mi.m;
            if (idx < 0 || idx >= count) return std::string();
            return column ? model.col_name(static_cast<int32_t>(idx))
                          : model.row_name(static_cast<int32_t>(idx));
        });
    }

    const PdhgOptions& options() const noexcept { return options_; }

private:
    // Options, cancellation, checkpoints, the solve and the result, for a
    // problem already loaded into ctx; name(column?, index) for messages.
    template <class NameFn>
    PdhgResult run(pdhg_ctx* ctx, int32_t m, int32_t n, const CancellationToken* cancel,
                   NameFn&& name) const {

        pdhg_options o;
        pdhg_default_options(&o);
        o.tolerance = options_.tolerance;
        o.max_iterations = options_.max_iterations;
        o.time_limit_seconds = options_.time_limit_seconds;
        o.restart_check_period = options_.restart_check_period;
        o.restart_sufficient_decrease = options_.restart_sufficient_decrease;
        o.step_size_safety = options_.step_size_safety;
        o.power_iterations = options_.power_iterations;
        o.verbose = options_.verbose ? 1 : 0;
        o.precision = precision_;

        // CancellationToken is an atomic<bool>; the engine polls a plain int,
        // mirrored from the token by a watcher thread while the solve runs.
        volatile int flag = (cancel != nullptr && cancel->is_cancelled()) ? 1 : 0;
        std::atomic<bool> running{true};
        std::thread watcher;
        if (cancel != nullptr) {
            o.cancel_flag = &flag;
            watcher = std::thread([&] {
                while (running.load(std::memory_order_relaxed)) {
                    if (cancel->is_cancelled()) flag = 1;
                    std::this_thread::sleep_for(std::chrono::microseconds(200));
                }
            });
        }
        Bridge bridge{&options_, static_cast<std::size_t>(n), static_cast<std::size_t>(m)};
        if (options_.checkpoint) {
            o.checkpoint = &Bridge::call;
            o.checkpoint_user = &bridge;
        }
        PdhgResult r;
        r.primal.resize(static_cast<std::size_t>(n));
        r.dual.resize(static_cast<std::size_t>(m));
        r.reduced_costs.resize(static_cast<std::size_t>(n));
        pdhg_info info;
        const int rc = pdhg_solve(ctx, &o, &info, r.primal.data(), r.dual.data(),
                                  r.reduced_costs.data());
        running.store(false);
        if (watcher.joinable()) watcher.join();
        check(rc, ctx, "pdhg_solve");
        if (!info.has_point) {
            r.primal.clear();
            r.dual.clear();
            r.reduced_costs.clear();
        }
        r.status = static_cast<PdhgStatus>(info.status);  // same enumerator order
        r.objective = info.objective;
        r.primal_infeasibility = info.primal_infeasibility;
        r.dual_infeasibility = info.dual_infeasibility;
        r.duality_gap = info.duality_gap;
        r.iterations = info.iterations;
        r.restarts = info.restarts;
        r.seconds = info.seconds;
        r.operator_norm_estimate = info.operator_norm_estimate;
        r.message = with_names(info.message, name);
        return r;
    }

    // std::function checkpoint behind the C callback (same thread, same cadence).
    struct Bridge {
        const PdhgOptions* opt;
        std::size_t n, m;
        static void call(void* user, long long it, const double* x, const double* y,
                         double res) {
            const auto* b = static_cast<const Bridge*>(user);
            b->opt->checkpoint(it, std::vector<Real>(x, x + b->n),
                               std::vector<Real>(y, y + b->m), res);
        }
    };

    static void check(int rc, const pdhg_ctx* ctx, const char* what) {
        if (rc == PDHG_OK) return;
        std::string detail = ctx != nullptr ? pdhg_last_error(ctx) : "";
        throw Error(static_cast<Status>(rc),  // same enumerator order as sov::Status
                    detail.empty() ? std::string(what) : std::string(what) + ": " + detail);
    }

    // The ABI names rows R<i> and columns C<j>; put the problem's names back.
    template <class NameFn>
    static std::string with_names(const char* msg, NameFn&& name) {
        std::string s(msg);
        const struct {
            const char* word;
            char tag;
        } kinds[2] = {{"column ", 'C'}, {"row ", 'R'}};
        for (const auto& k : kinds) {
            const std::size_t at = s.find(std::string(k.word) + k.tag);
            if (at == std::string::npos) continue;
            const std::size_t num = at + std::strlen(k.word) + 1;
            std::size_t end = num;
            while (end < s.size() && s[end] >= '0' && s[end] <= '9') ++end;
            if (end == num) continue;
            const long idx = std::stol(s.substr(num, end - num));
            const std::string nm = name(k.tag == 'C', idx);
            if (!nm.empty()) s.replace(num - 1, end - num + 1, nm);
        }
        return s;
    }

    PdhgOptions options_;
    int precision_;
    int device_;
};

}  // namespace sov
