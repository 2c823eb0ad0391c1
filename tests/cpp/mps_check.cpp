// mps_check.cpp -- the reader half of include/pdhg_b200_sov.hpp, on the CPU.
//
// For every MPS file named on the command line (and both negative-upper-bound
// rules), reads it with the reference's own sov::read_mps and with
// sov::MpsModelB200::read_file(...).to_read_result(), and requires the same
// outcome: the same sov::Error text, or the same Problem (name, objective
// name, sense, constant, row and column names, bounds, kinds, objective, CSR
// bit for bit) and the same warnings. Built by oracle/Makefile (target ref)
// against the reference's headers and its compiled reader; prints one line per
// case, "ALL OK" at the end, exits non-zero on any difference. Test
// infrastructure only.
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "pdhg_b200_sov.hpp"
#include "sovereign/io.hpp"

namespace {

template <class A, class B>
bool same_bits(const A& a, const B& b) {
    if (a.size() != b.size()) return false;
    return a.size() == 0 || std::memcmp(a.data(), b.data(), sizeof(a[0]) * a.size()) == 0;
}

std::string compare(const sov::ReadResult& a, const sov::ReadResult& b) {
    const sov::Problem& p = a.problem;
    const sov::Problem& q = b.problem;
    if (p.name() != q.name()) return "name";
    if (p.objective_name() != q.objective_name()) return "objective name";
    if (p.sense() != q.sense()) return "sense";
    const double pc = p.objective_constant(), qc = q.objective_constant();
    if (std::memcmp(&pc, &qc, sizeof(double)) != 0) return "objective constant";
    if (p.num_rows() != q.num_rows() || p.num_cols() != q.num_cols()) return "shape";
    if (!same_bits(p.objective(), q.objective())) return "objective";
    if (!same_bits(p.row_lower(), q.row_lower()) || !same_bits(p.row_upper(), q.row_upper()))
        return "row bounds";
    if (!same_bits(p.col_lower(), q.col_lower()) || !same_bits(p.col_upper(), q.col_upper()))
        return "column bounds";
    if (!same_bits(p.col_kind(), q.col_kind())) return "column kinds";
    for (sov::Idx i = 0; i < p.num_rows(); ++i)
        if (p.row_names()[i] != q.row_names()[i]) return "row names";
    for (sov::Idx j = 0; j < p.num_cols(); ++j)
        if (p.col_names()[j] != q.col_names()[j]) return "column names";
    const sov::CsrMatrix& A = p.matrix();
    const sov::CsrMatrix& B = q.matrix();
    if (!same_bits(A.row_ptr(), B.row_ptr()) || !same_bits(A.col_idx(), B.col_idx()) ||
        !same_bits(A.values(), B.values()))
        return "matrix";
    if (a.warnings.size() != b.warnings.size()) return "warning count";
    for (std::size_t k = 0; k < a.warnings.size(); ++k) {
        const auto& u = a.warnings[k];
        const auto& w = b.warnings[k];
        if (u.line != w.line || u.section != w.section || u.message != w.message)
            return "warning " + std::to_string(k);
    }
    if (a.format != b.format) return "format";
    return "";
}

}  // namespace

int main(int argc, char** argv) {
    int failures = 0;
    for (int f = 1; f < argc; ++f) {
        for (int rule = 0; rule < 2; ++rule) {
            sov::MpsOptions o;
            o.negative_upper_bound = rule ? sov::NegativeUpperBoundRule::KeepLowerAtZero
                                          : sov::NegativeUpperBoundRule::LowerBecomesMinusInfinity;
            std::string ref_err, our_err, diff;
            sov::ReadResult ref, ours;
            try {
                ref = sov::read_mps(argv[f], o);
            } catch (const sov::Error& e) {
                ref_err = e.what();
            }
            try {
                ours = sov::MpsModelB200::read_file(argv[f], o).to_read_result();
            } catch (const sov::Error& e) {
                our_err = e.what();
            }
            if (!ref_err.empty() || !our_err.empty())
                diff = ref_err == our_err ? "" : "errors differ: [" + ref_err + "] vs [" + our_err + "]";
            else
                diff = compare(ref, ours);
            std::printf("%s %s rule %d%s%s\n", diff.empty() ? "OK" : "FAIL", argv[f], rule,
                        diff.empty() ? "" : ": ", diff.c_str());
            if (!diff.empty()) ++failures;
        }
    }
    if (failures == 0) std::printf("ALL OK\n");
    return failures == 0 ? 0 : 1;
}
