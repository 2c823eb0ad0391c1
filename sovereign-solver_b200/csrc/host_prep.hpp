// host_prep.hpp -- host-side preparation of an LP for the device engine.
//
// Validation (Problem::validate, src/io/problem.cpp:50-; CsrMatrix::validate,
// src/l0/sparse.cpp:94-128), Ruiz + Pock-Chambolle scaling
// (Scaling::equilibrate, src/l1/scaling.cpp:19-104) and the scaled-problem
// rebuild (scaling.cpp:155-205). FP64, sequential, in the reference's order:
// the scale factors are bit-identical to the reference's.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

namespace pdhg {

struct HostCsr {
    int32_t rows = 0, cols = 0;
    std::vector<int32_t> rp, ci;
    std::vector<double> v;
    int64_t nnz() const { return static_cast<int64_t>(ci.size()); }
};

struct HostLp {
    int32_t m = 0, n = 0;
    HostCsr A;
    std::vector<double> c, col_lo, col_hi, row_lo, row_hi;
    double obj_const = 0.0;
    bool maximize = false;
};

struct ScalingParams {
    int ruiz_iterations = 8;
    double ruiz_tolerance = 1e-2;
    double pock_chambolle_alpha = 1.0;
    bool apply_ruiz = true;
    bool apply_pock_chambolle = true;
    bool operator==(const ScalingParams& o) const {
        return ruiz_iterations == o.ruiz_iterations && ruiz_tolerance == o.ruiz_tolerance &&
               pock_chambolle_alpha == o.pock_chambolle_alpha && apply_ruiz == o.apply_ruiz &&
               apply_pock_chambolle == o.apply_pock_chambolle;
    }
};

// The caller's arrays, read in place (no copy).
struct LpView {
    int32_t m = 0, n = 0;
    int64_t nnz = 0;
    const int32_t* rp = nullptr;
    const int32_t* ci = nullptr;
    const double* v = nullptr;
    const double* c = nullptr;
    double obj_const = 0.0;
    const double *col_lo = nullptr, *col_hi = nullptr, *row_lo = nullptr, *row_hi = nullptr;
};

// True when the LP passes the reference's checks; otherwise `why` gets the
// reference's message (rows/columns named R<i>/C<j>).
bool validate_lp(const LpView& lp, std::string* why);

// Scaling::equilibrate(CsrMatrix): row_scale (rows), col_scale (cols).
void equilibrate(const HostCsr& A, const ScalingParams& p, std::vector<double>* rs,
                 std::vector<double>* cs);

// The scaled problem of Scaling::equilibrate(Problem): values (v*rs)*cs with
// |v| <= 1e-14 dropped (the Builder/from_triplets rebuild, sparse.cpp:55),
// objective c*cs, column bounds lo/cs, row bounds lo*rs.
void build_scaled(const HostLp& lp, const std::vector<double>& rs,
                  const std::vector<double>& cs, HostLp* out);

// Row lengths -> (long-row list, number of short rows, lanes per short row).
void bin_rows(const std::vector<int32_t>& rp, int long_threshold, std::vector<int32_t>* long_rows,
              int32_t* n_short, int* vw);

}  // namespace pdhg
