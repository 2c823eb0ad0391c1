// adapter_check.cpp -- the drop-in check of include/pdhg_b200_sov.hpp.
//
// Builds LPs through the reference's own sov::Problem::Builder (named rows and
// columns), solves each with the reference's sov::Pdhg on its Host backend and
// with sov::PdhgB200 (the B200 engine behind the same interface, exact mode),
// and requires identical results: status, message, iterations, restarts,
// objective, infeasibilities, gap, operator-norm estimate, x, y, reduced
// costs; the same checkpoint calls; cancellation before the first iteration;
// and an MPS model read by the reference (read_mps_string, then Pdhg) and by
// sov::MpsModelB200 (its arrays straight to the engine).
// Built by oracle/Makefile (target ref) against the reference's headers and
// its compiled PDHG path; prints one line per case and exits non-zero on any
// difference. Test infrastructure only.
#include <cstdio>
#include <cstring>
#include <random>
#include <string>
#include <vector>

#include "pdhg_b200_sov.hpp"
#include "sovereign/backend.hpp"
#include "sovereign/io.hpp"

namespace {

int failures = 0;

void report(const std::string& name, bool ok, const std::string& detail = "") {
    std::printf("%s %s%s%s\n", ok ? "OK" : "FAIL", name.c_str(), detail.empty() ? "" : ": ",
                detail.c_str());
    if (!ok) ++failures;
}

// Equality rows A x = A x0, 0 <= x <= 10, c = A^T y0 + s (feasible, bounded),
// k nonzeros per column at distinct random rows; optional <= rows, maximize.
sov::Problem random_lp(int m, int n, int k, unsigned seed, bool with_le, bool maximize,
                       double obj_const) {
    std::mt19937_64 rng(seed);
    std::uniform_int_distribution<int> pick(0, m - 1);
    std::normal_distribution<double> gauss(0.0, 1.0);
    std::uniform_real_distribution<double> unif(0.0, 1.0);
    std::vector<std::vector<std::pair<int, double>>> col(static_cast<size_t>(n));
    for (int j = 0; j < n; ++j) {
        std::vector<int> rows;
        while (static_cast<int>(rows.size()) < k) {
            const int r = pick(rng);
            bool dup = false;
            for (int q : rows) dup |= q == r;
            if (!dup) rows.push_back(r);
        }
        for (int r : rows) col[static_cast<size_t>(j)].push_back({r, gauss(rng)});
    }
    std::vector<double> x0(static_cast<size_t>(n)), y0(static_cast<size_t>(m)), ax(static_cast<size_t>(m), 0.0);
    for (auto& v : x0) v = 10.0 * unif(rng);
    for (auto& v : y0) v = gauss(rng);
    for (int j = 0; j < n; ++j)
        for (auto [r, v] : col[static_cast<size_t>(j)]) ax[static_cast<size_t>(r)] += v * x0[static_cast<size_t>(j)];
    sov::Problem::Builder b;
    b.set_sense(maximize ? sov::ObjSense::Maximize : sov::ObjSense::Minimize);
    b.set_objective_constant(obj_const);
    for (int j = 0; j < n; ++j) {
        const sov::Idx c = b.add_column("flow_" + std::to_string(j));
        double cj = unif(rng);
        for (auto [r, v] : col[static_cast<size_t>(j)]) cj += v * y0[static_cast<size_t>(r)];
        b.set_objective_coefficient(c, maximize ? -cj : cj);
        b.set_column_bounds(c, 0.0, 10.0);
    }
    for (int i = 0; i < m; ++i) {
        const bool le = with_le && i % 3 == 0;
        b.add_row("balance_" + std::to_string(i), le ? -std::numeric_limits<double>::infinity()
                                                     : ax[static_cast<size_t>(i)],
                  ax[static_cast<size_t>(i)] + (le ? 1.0 : 0.0));
    }
    for (int j = 0; j < n; ++j)
        for (auto [r, v] : col[static_cast<size_t>(j)]) b.add_coefficient(r, j, v);
    return b.finish();
}

bool same_vec(const std::vector<double>& a, const std::vector<double>& b) {
    return a.size() == b.size() && (a.empty() || std::memcmp(a.data(), b.data(), sizeof(double) * a.size()) == 0);
}

void compare(const std::string& name, const sov::PdhgResult& r, const sov::PdhgResult& g) {
    std::string d;
    if (r.status != g.status) d += " status";
    if (r.message != g.message) d += " message[" + r.message + " | " + g.message + "]";
    if (r.iterations != g.iterations) d += " iterations";
    if (r.restarts != g.restarts) d += " restarts";
    if (r.objective != g.objective) d += " objective";
    if (r.primal_infeasibility != g.primal_infeasibility) d += " primal_infeasibility";
    if (r.dual_infeasibility != g.dual_infeasibility) d += " dual_infeasibility";
    if (r.duality_gap != g.duality_gap) d += " duality_gap";
    if (r.operator_norm_estimate != g.operator_norm_estimate) d += " operator_norm";
    if (!same_vec(r.primal, g.primal)) d += " primal";
    if (!same_vec(r.dual, g.dual)) d += " dual";
    if (!same_vec(r.reduced_costs, g.reduced_costs)) d += " reduced_costs";
    char buf[128];
    std::snprintf(buf, sizeof buf, " (status %d, %lld iterations)", static_cast<int>(g.status),
                  g.iterations);
    report(name, d.empty(), d.empty() ? buf : d);
}

}  // namespace

int main() {
    auto host = sov::make_backend(sov::BackendKind::Host);
    sov::PdhgOptions opt;
    opt.max_iterations = 30000;

    // feasible LPs, bit-identical in exact mode
    struct Case {
        const char* name;
        int m, n, k;
        unsigned seed;
        bool le, max;
        double k0;
    } cases[] = {{"equality_60x150", 60, 150, 4, 7u, false, false, 0.0},
                 {"mixed_rows_maximize_40x120", 40, 120, 3, 8u, true, true, 2.5},
                 {"iteration_limit_80x200", 80, 200, 5, 9u, false, false, 0.0}};
    for (const Case& c : cases) {
        const sov::Problem p = random_lp(c.m, c.n, c.k, c.seed, c.le, c.max, c.k0);
        sov::PdhgOptions o = opt;
        if (std::string(c.name).rfind("iteration_limit", 0) == 0) o.max_iterations = 777;
        const sov::PdhgResult ref = sov::Pdhg(o).solve(p, *host);
        const sov::PdhgResult b200 = sov::PdhgB200(o).solve(p, *host);
        compare(c.name, ref, b200);
    }

    // invalid problem: the message names the problem's column
    {
        sov::Problem::Builder b;
        const sov::Idx c0 = b.add_column("pump_0");
        const sov::Idx c1 = b.add_column("pump_1");
        b.set_objective_coefficient(c0, 1.0);
        b.set_column_bounds(c1, 3.0, 2.0);
        b.add_row("demand", 1.0, 1.0);
        b.add_coefficient(0, c0, 1.0);
        b.add_coefficient(0, c1, 1.0);
        const sov::Problem p = b.finish();
        compare("invalid_crossed_bounds", sov::Pdhg(opt).solve(p, *host),
                sov::PdhgB200(opt).solve(p, *host));
    }

    // cancellation before the first iteration
    {
        const sov::Problem p = random_lp(30, 80, 3, 11u, false, false, 0.0);
        sov::CancellationToken t;
        t.cancel();
        compare("cancelled", sov::Pdhg(opt).solve(p, *host, &t),
                sov::PdhgB200(opt).solve(p, *host, &t));
    }

    // checkpoint callbacks: same iterations, same points
    {
        const sov::Problem p = random_lp(30, 80, 3, 12u, false, false, 0.0);
        std::vector<long long> it_r, it_g;
        std::vector<double> x_r, x_g;
        sov::PdhgOptions o = opt;
        o.max_iterations = 400;
        o.checkpoint = [&](long long it, const std::vector<double>& x, const std::vector<double>&,
                           double) {
            it_r.push_back(it);
            x_r.insert(x_r.end(), x.begin(), x.end());
        };
        const sov::PdhgResult ref = sov::Pdhg(o).solve(p, *host);
        o.checkpoint = [&](long long it, const std::vector<double>& x, const std::vector<double>&,
                           double) {
            it_g.push_back(it);
            x_g.insert(x_g.end(), x.begin(), x.end());
        };
        const sov::PdhgResult b200 = sov::PdhgB200(o).solve(p, *host);
        compare("checkpoint_result", ref, b200);
        report("checkpoint_calls", it_r == it_g && same_vec(x_r, x_g),
               std::to_string(it_r.size()) + " calls");
    }
    // an MPS model: the reference reads it and solves the Problem; the B200
    // reader's model goes to the engine without a sov::Problem in between.
    // Ranges, bounds of several types, a second N row and an objective
    // constant; and a crossed bound, whose message names the file's column.
    {
        const std::string text =
            "NAME          MPSCASE\n"
            "ROWS\n N  COST\n L  CAP\n G  NEED\n E  BAL\n N  SPARE\n"
            "COLUMNS\n"
            "    X1   COST  1.0   CAP  1.0\n    X1   NEED  1.0   SPARE  3.0\n"
            "    X2   COST  2.0   CAP  1.0\n    X2   BAL  -1.0\n"
            "    X3   COST  -1.0  BAL  1.0\n    X3   NEED  0.5\n"
            "    X4   COST  0.25  CAP  2.0\n    X4   BAL   1.0\n"
            "RHS\n    RHS  COST  -3.5\n    RHS  CAP  8.0   NEED  1.0\n    RHS  BAL  2.0\n"
            "RANGES\n    RNG  CAP  6.0   BAL  -1.0\n"
            "BOUNDS\n UP BND  X1  4.0\n LO BND  X3  -5.0\n UP BND  X3  5.0\n UP BND  X4  3.0\n"
            "ENDATA\n";
        const sov::ReadResult rr = sov::read_mps_string(text);
        const sov::MpsModelB200 model = sov::MpsModelB200::read_string(text);
        sov::PdhgOptions o = opt;
        o.max_iterations = 5000;
        compare("mps_model", sov::Pdhg(o).solve(rr.problem, *host),
                sov::PdhgB200(o).solve(model, *host));
        std::string crossed = text;
        crossed.replace(crossed.find(" UP BND  X4  3.0"), 16, " UP BND  X4 -3.0");
        sov::MpsOptions literal;
        literal.negative_upper_bound = sov::NegativeUpperBoundRule::KeepLowerAtZero;
        std::string ref_err, our_err;
        try {
            sov::read_mps_string(crossed, literal);
        } catch (const sov::Error& e) {
            ref_err = e.what();
        }
        try {
            sov::MpsModelB200::read_string(crossed, literal);
        } catch (const sov::Error& e) {
            our_err = e.what();
        }
        report("mps_crossed_bound_message", !ref_err.empty() && ref_err == our_err, our_err);
    }
    std::printf("%s\n", failures == 0 ? "ALL OK" : "FAILURES");
    return failures == 0 ? 0 : 1;
}
