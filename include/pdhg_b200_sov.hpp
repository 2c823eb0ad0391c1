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
#include "sovereign/pdhg.hpp"
#include "sovereign/problem.hpp"
#include "sovereign/status.hpp"

namespace sov {

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
        const int rc = pdhg_solve(ctx.get(), &o, &info, r.primal.data(), r.dual.data(),
                                  r.reduced_costs.data());
        running.store(false);
        if (watcher.joinable()) watcher.join();
        check(rc, ctx.get(), "pdhg_solve");
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
        r.message = with_names(problem, info.message);
        return r;
    }

    const PdhgOptions& options() const noexcept { return options_; }

private:
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
    static std::string with_names(const Problem& p, const char* msg) {
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
            const auto names = k.tag == 'C' ? p.col_names() : p.row_names();
            if (idx >= 0 && static_cast<std::size_t>(idx) < names.size())
                s.replace(num - 1, end - num + 1, names[static_cast<std::size_t>(idx)]);
        }
        return s;
    }

    PdhgOptions options_;
    int precision_;
    int device_;
};

}  // namespace sov
