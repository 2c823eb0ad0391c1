// batch.cu -- the batched engine: many LPs of uneven size solved together,
// each with its own scaling, step sizes, restarts and termination, in ONE
// launch of a CUDA graph whose WHILE node repeats check periods until every
// instance is done (the condition is set on the device by the last kernel of
// each period). Per instance the algorithm is the single engine's
// (Pdhg::solve, src/l1/pdhg.cpp:218-502) in its fast precisions. A batch
// lives inside a pdhg_ctx (pdhg_load_batch / pdhg_solve_batch) and shares its
// stream and error text.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <limits>
#include <memory>
#include <string>
#include <thread>
#include <vector>

#include "../../include/pdhg_b200.h"
#include "batch_kernels.cuh"
#include "dev_buffer.cuh"
#include "engine.cuh"

namespace pdhg {

namespace {

constexpr double kInfB = std::numeric_limits<double>::infinity();

}  // namespace

struct BatchCtx {
    int device = 0;
    cudaStream_t stream = nullptr;  // the owning context's
    std::string& err;               // the owning context's error text
    bool loaded = false;
    int32_t count = 0, m = 0, n = 0;
    int64_t nnz = 0;
    std::vector<int32_t> row_off, col_off;
    std::vector<int> valid;
    std::vector<std::string> why;
    std::vector<double> obj_const;
    std::vector<int> maximize;

    MatDev Ao, ATo, As, ATs;
    DBuf<int32_t> row_off_d, col_off_d, row_inst, col_inst;
    DBuf<int4> chk_item;
    DBuf<double> chk_part;
    DBuf<unsigned int> chk_ticket;
    int32_t n_chk = 0;
    DBuf<int32_t> blk_list_a, blk_list_t;
    DBuf<unsigned char> blk_flag_a, blk_flag_t;
    DBuf<double> c_o, lo_o, hi_o, rlo_o, rhi_o, c_s, lo_s, hi_s, rlo_s, rhi_s, rs_d, cs_d;
    DBuf<float> c32, lo32, hi32, rlo32, rhi32;
    DBuf<InstState> is;
    DBuf<BatchGlobal> g;
    Mailbox* mail = nullptr;
    Mailbox* mail_dev = nullptr;

    bool have_opnorm = false;
    int opnorm_iters = -1;
    DBuf<double> x64, xbar64, s64, y64, xsum, ysum, act_avg, xo, yo, rc, x_last, y_last;
    DBuf<double> pw_u, pw_v, pw_w, x0s, y0s;
    DBuf<float> x32, xbar32, s32, y32, psx, psy;
    bool halpern = false;  // the current solve runs the Halpern iteration (its anchors below)
    DBuf<double> xa64, sa64, ya64;
    DBuf<float> xa32, sa32, ya32;

    // solve graphs, [0] FP32 and [1] FP64, with what they bake in
    cudaGraphExec_t graph[2] = {nullptr, nullptr};
    long long graph_key[2][11] = {};

    // lanes per row of the lane-group path: the binning's choice for A's rows
    // [0] and A^T's rows [1], and the autotuner's per precision ([0] FP32, [1]
    // FP64; 0 = not tuned since the load)
    int bin_vw[2] = {1, 1};
    int tuned_vw[2][2] = {{0, 0}, {0, 0}};
    bool tune_timed[2] = {false, false};

    BatchCtx(int dev, cudaStream_t s, std::string& e) : device(dev), stream(s), err(e) {}
    ~BatchCtx() {
        drop_graphs();
        if (mail != nullptr) cudaFreeHost(mail);
    }
    void drop_graphs() {
        for (auto& g : graph)
            if (g != nullptr) {
                cudaGraphExecDestroy(g);
                g = nullptr;
            }
    }

    BatchView view() const {
        BatchView b;
        b.count = count;
        b.m = m;
        b.n = n;
        b.row_off = row_off_d.p;
        b.col_off = col_off_d.p;
        b.row_inst = row_inst.p;
        b.col_inst = col_inst.p;
        b.chk_item = chk_item.p;
        b.n_chk = n_chk;
        b.chk_part = chk_part.p;
        b.chk_ticket = chk_ticket.p;
        b.blk_list[0] = blk_list_a.p;
        b.blk_list[1] = blk_list_t.p;
        b.blk_flag[0] = blk_flag_a.p;
        b.blk_flag[1] = blk_flag_t.p;
        b.A = As.view();
        b.AT = ATs.view();
        b.Ao = Ao.view();
        b.ATo = ATo.view();
        DevProblem& P = b.P;
        P.m = m;
        P.n = n;
        P.c = c_s.p;
        P.lo = lo_s.p;
        P.hi = hi_s.p;
        P.rlo = rlo_s.p;
        P.rhi = rhi_s.p;
        P.c_o = c_o.p;
        P.lo_o = lo_o.p;
        P.hi_o = hi_o.p;
        P.rlo_o = rlo_o.p;
        P.rhi_o = rhi_o.p;
        P.rs = rs_d.p;
        P.cs = cs_d.p;
        P.c32 = c32.p;
        P.lo32 = lo32.p;
        P.hi32 = hi32.p;
        P.rlo32 = rlo32.p;
        P.rhi32 = rhi32.p;
        b.is = is.p;
        b.g = g.p;
        b.mail = mail_dev;
        return b;
    }
};

namespace {

#define BCK(expr)                                                          \
    do {                                                                   \
        cudaError_t e_ = (expr);                                           \
        if (e_ != cudaSuccess) return cuda_fail(&c.err, e_, #expr);        \
    } while (0)

// Per-instance validation with the reference's messages (problem.cpp:50-,
// sparse.cpp:94-128), rows and columns named within their instance. Returns
// false (and fills err) only for structure the device code cannot hold.
bool validate_batch(BatchCtx& c, const int32_t* rp, const int32_t* ci, const double* v,
                    const double* cv, const double* col_lo, const double* col_hi,
                    const double* row_lo, const double* row_hi) {
    if (rp[0] != 0 || rp[c.m] != c.nnz) {
        c.err = "pdhg_load_batch: row_ptr must start at 0 and end at nnz";
        return false;
    }
    c.valid.assign(static_cast<size_t>(c.count), 1);
    c.why.assign(static_cast<size_t>(c.count), std::string());
    for (int32_t k = 0; k < c.count; ++k) {
        const int32_t r0 = c.row_off[k], r1 = c.row_off[k + 1];
        const int32_t c0 = c.col_off[k], c1 = c.col_off[k + 1];
        auto bad = [&](const std::string& w) {
            if (c.valid[k]) {
                c.valid[k] = 0;
                c.why[k] = w;
            }
        };
        if (!std::isfinite(c.obj_const[k])) bad("objective constant is not finite");
        for (int32_t j = c0; j < c1 && c.valid[k]; ++j) {
            const std::string name = "C" + std::to_string(j - c0);
            if (!std::isfinite(cv[j])) bad("non-finite objective coefficient in column " + name);
            else if (std::isnan(col_lo[j]) || std::isnan(col_hi[j])) bad("NaN bound on column " + name);
            else if (col_lo[j] > col_hi[j]) bad("crossed bounds on column " + name);
        }
        for (int32_t i = r0; i < r1 && c.valid[k]; ++i) {
            const std::string name = "R" + std::to_string(i - r0);
            if (std::isnan(row_lo[i]) || std::isnan(row_hi[i])) bad("NaN bound on row " + name);
            else if (row_lo[i] > row_hi[i]) bad("crossed bounds on row " + name);
        }
        for (int32_t i = r0; i < r1; ++i) {
            const int32_t b = rp[i], e = rp[i + 1];
            if (b > e || b < 0 || e > c.nnz) {
                c.err = "pdhg_load_batch: row_ptr is not monotone";
                return false;
            }
            for (int32_t q = b; q < e; ++q) {
                if (ci[q] < c0 || ci[q] >= c1) {
                    c.err = "pdhg_load_batch: instance " + std::to_string(k) +
                            ": column index outside the instance's columns";
                    return false;
                }
                if (q > b && ci[q - 1] >= ci[q]) bad("column indices not strictly ascending");
                if (!std::isfinite(v[q])) bad("non-finite coefficient");
            }
        }
    }
    return true;
}

int batch_intake(BatchCtx& c, const pdhg_options& o) {
    cudaStream_t s = c.stream;
    BCK(c.rs_d.alloc(static_cast<size_t>(c.m) + 1));
    BCK(c.cs_d.alloc(static_cast<size_t>(c.n) + 1));
    launch_fill(c.rs_d.p, c.m, 1.0, s);
    launch_fill(c.cs_d.p, c.n, 1.0, s);
    DBuf<double> rbuf, cbuf;
    BCK(rbuf.alloc(static_cast<size_t>(c.m) + 1));
    BCK(cbuf.alloc(static_cast<size_t>(c.n) + 1));
    // reset the instances' Ruiz flags
    {
        std::vector<InstState> h(static_cast<size_t>(c.count));
        BCK(cudaMemcpy(h.data(), c.is.p, sizeof(InstState) * c.count, cudaMemcpyDeviceToHost));
        for (auto& st : h) st.ruiz_done = 0;
        BCK(cudaMemcpy(c.is.p, h.data(), sizeof(InstState) * c.count, cudaMemcpyHostToDevice));
    }
    BatchView b = c.view();
    if (o.apply_ruiz) {
        for (int sweep = 0; sweep < o.ruiz_iterations; ++sweep) {
            launch_batch_ruiz_max(b, c.Ao.view(), 0, c.rs_d.p, c.cs_d.p, rbuf.p, s);
            launch_batch_ruiz_max(b, c.ATo.view(), 1, c.rs_d.p, c.cs_d.p, cbuf.p, s);
            launch_batch_ruiz_update(b, c.rs_d.p, c.cs_d.p, rbuf.p, cbuf.p, o.ruiz_tolerance, s);
        }
    }
    if (o.apply_pock_chambolle)
        launch_pock_chambolle(c.Ao.view(), c.ATo.view(), c.rs_d.p, c.cs_d.p, rbuf.p, cbuf.p,
                              o.pock_chambolle_alpha, s);
    DBuf<unsigned long long> dropped;
    BCK(dropped.alloc(1));
    BCK(cudaMemsetAsync(dropped.p, 0, sizeof(unsigned long long), s));
    BCK(c.As.v64.alloc(static_cast<size_t>(c.nnz)));
    launch_scale_values(c.Ao.view(), 0, c.rs_d.p, c.cs_d.p, c.As.v64.p, dropped.p, s);
    unsigned long long ndrop = 0;
    BCK(cudaMemcpyAsync(&ndrop, dropped.p, sizeof ndrop, cudaMemcpyDeviceToHost, s));
    BCK(cudaStreamSynchronize(s));
    c.As.rows = c.m;
    c.As.cols = c.n;
    c.ATs.rows = c.n;
    c.ATs.cols = c.m;
    if (ndrop == 0) {
        c.As.nnz = c.ATs.nnz = c.nnz;
        BCK(copy_dev(c.As.rp, c.Ao.rp.p, static_cast<size_t>(c.m) + 1, s));
        BCK(copy_dev(c.As.ci, c.Ao.ci.p, static_cast<size_t>(c.nnz), s));
        BCK(copy_dev(c.ATs.rp, c.ATo.rp.p, static_cast<size_t>(c.n) + 1, s));
        BCK(copy_dev(c.ATs.ci, c.ATo.ci.p, static_cast<size_t>(c.nnz), s));
        BCK(c.ATs.v64.alloc(static_cast<size_t>(c.nnz)));
        launch_scale_values(c.ATo.view(), 1, c.rs_d.p, c.cs_d.p, c.ATs.v64.p, dropped.p, s);
    } else {
        DBuf<int32_t> kept;
        BCK(kept.alloc(static_cast<size_t>(c.m) + 1));
        launch_kept_counts(c.Ao.view(), c.As.v64.p, kept.p, s);
        BCK(c.As.rp.alloc(static_cast<size_t>(c.m) + 1));
        if (prefix_rows(kept.p, c.m, c.As.rp.p, s) != 0) return cuda_fail(&c.err, cudaGetLastError(), "prefix_rows");
        const int64_t nk = c.nnz - static_cast<int64_t>(ndrop);
        DBuf<double> vk;
        BCK(c.As.ci.alloc(static_cast<size_t>(nk)));
        BCK(vk.alloc(static_cast<size_t>(nk)));
        launch_compact(c.Ao.view(), c.As.v64.p, c.As.rp.p, c.As.ci.p, vk.p, s);
        BCK(copy_dev(c.As.v64, vk.p, static_cast<size_t>(nk), s));
        c.As.nnz = c.ATs.nnz = nk;
        BCK(c.ATs.rp.alloc(static_cast<size_t>(c.n) + 1));
        BCK(c.ATs.ci.alloc(static_cast<size_t>(nk)));
        BCK(c.ATs.v64.alloc(static_cast<size_t>(nk)));
        BCK(c.ATs.tscratch.alloc(transpose_scratch_bytes(c.m, c.n, nk)));
        TransposeOut out{c.ATs.rp.p, c.ATs.ci.p, c.ATs.v64.p};
        if (build_transpose(c.m, c.n, nk, c.As.rp.p, c.As.ci.p, c.As.v64.p, out, c.ATs.tscratch.p, s) != 0)
            return cuda_fail(&c.err, cudaGetLastError(), "build_transpose");
    }
    BCK(to_float(c.As.v32, c.As.v64, s));
    BCK(to_float(c.ATs.v32, c.ATs.v64, s));
    int rc = bin_matrix(c.As, s, &c.err);
    if (rc != PDHG_OK) return rc;
    rc = bin_matrix(c.ATs, s, &c.err);
    if (rc != PDHG_OK) return rc;
    c.bin_vw[0] = c.As.vw;
    c.bin_vw[1] = c.ATs.vw;
    c.tuned_vw[0][0] = c.tuned_vw[0][1] = c.tuned_vw[1][0] = c.tuned_vw[1][1] = 0;
    c.tune_timed[0] = c.tune_timed[1] = false;
    {
        // active block lists of the iteration kernels (one entry per lane-group
        // block), sized for the widest lane group the autotuner may pick
        const int64_t wa = std::min(32, 2 * c.As.vw), wt = std::min(32, 2 * c.ATs.vw);
        const size_t nba = static_cast<size_t>((static_cast<int64_t>(c.As.rows) * wa + kBlock - 1) / kBlock) + 1;
        const size_t nbt = static_cast<size_t>((static_cast<int64_t>(c.ATs.rows) * wt + kBlock - 1) / kBlock) + 1;
        BCK(c.blk_list_a.alloc(nba));
        BCK(c.blk_flag_a.alloc(nba));
        BCK(c.blk_list_t.alloc(nbt));
        BCK(c.blk_flag_t.alloc(nbt));
    }
    BCK(c.c_s.alloc(static_cast<size_t>(c.n) + 1));
    BCK(c.lo_s.alloc(static_cast<size_t>(c.n) + 1));
    BCK(c.hi_s.alloc(static_cast<size_t>(c.n) + 1));
    BCK(c.rlo_s.alloc(static_cast<size_t>(c.m) + 1));
    BCK(c.rhi_s.alloc(static_cast<size_t>(c.m) + 1));
    b = c.view();
    launch_batch_scale_vectors(b, c.c_s.p, c.lo_s.p, c.hi_s.p, c.rlo_s.p, c.rhi_s.p, s);
    BCK(to_float(c.c32, c.c_s, s));
    BCK(to_float(c.lo32, c.lo_s, s));
    BCK(to_float(c.hi32, c.hi_s, s));
    BCK(to_float(c.rlo32, c.rlo_s, s));
    BCK(to_float(c.rhi32, c.rhi_s, s));
    b = c.view();
    launch_batch_norms(b, s);
    BCK(cudaStreamSynchronize(s));
    c.have_opnorm = false;
    return PDHG_OK;
}

int batch_load(BatchCtx& c, int32_t count, const int32_t* row_off, const int32_t* col_off,
               int64_t nnz, const int32_t* rp, const int32_t* ci, const double* v,
               const double* cv, const double* obj_const, const int* maximize,
               const double* col_lo, const double* col_hi, const double* row_lo,
               const double* row_hi) {
    if (count < 1 || row_off == nullptr || col_off == nullptr || rp == nullptr ||
        obj_const == nullptr || maximize == nullptr || nnz < 0 ||
        nnz > std::numeric_limits<int32_t>::max()) {
        c.err = "pdhg_load_batch: invalid arguments";
        return PDHG_ERR_INVALID_ARGUMENT;
    }
    for (int32_t k = 0; k < count; ++k)
        if (row_off[k + 1] < row_off[k] || col_off[k + 1] < col_off[k]) {
            c.err = "pdhg_load_batch: offsets must be non-decreasing";
            return PDHG_ERR_INVALID_ARGUMENT;
        }
    if (row_off[0] != 0 || col_off[0] != 0) {
        c.err = "pdhg_load_batch: offsets must start at 0";
        return PDHG_ERR_INVALID_ARGUMENT;
    }
    const int32_t m = row_off[count], n = col_off[count];
    if ((nnz > 0 && (ci == nullptr || v == nullptr)) ||
        (n > 0 && (cv == nullptr || col_lo == nullptr || col_hi == nullptr)) ||
        (m > 0 && (row_lo == nullptr || row_hi == nullptr))) {
        c.err = "pdhg_load_batch: null array";
        return PDHG_ERR_INVALID_ARGUMENT;
    }
    BCK(cudaSetDevice(c.device));
    c.loaded = false;
    c.drop_graphs();  // their kernels hold the previous batch's buffers
    c.count = count;
    c.m = m;
    c.n = n;
    c.nnz = nnz;
    c.row_off.assign(row_off, row_off + count + 1);
    c.col_off.assign(col_off, col_off + count + 1);
    c.obj_const.assign(obj_const, obj_const + count);
    c.maximize.assign(maximize, maximize + count);
    if (!validate_batch(c, rp, ci, v, cv, col_lo, col_hi, row_lo, row_hi))
        return PDHG_ERR_INVALID_ARGUMENT;
    cudaStream_t s = c.stream;
    // structure checked on the host above (columns inside their instance)
    int rc = upload_csr(m, n, nnz, rp, ci, v, c.Ao, s, &c.err);
    if (rc != PDHG_OK) return rc;
    rc = finish_matrix(c.Ao, c.ATo, s, &c.err);
    if (rc != PDHG_OK) return rc;
    BCK(upload(c.row_off_d, row_off, static_cast<size_t>(count) + 1, s));
    BCK(upload(c.col_off_d, col_off, static_cast<size_t>(count) + 1, s));
    BCK(c.row_inst.alloc(static_cast<size_t>(m) + 1));
    BCK(c.col_inst.alloc(static_cast<size_t>(n) + 1));
    launch_batch_fill_inst(c.row_off_d.p, count, c.row_inst.p, s);
    launch_batch_fill_inst(c.col_off_d.p, count, c.col_inst.p, s);
    {
        // the check's CTA items: about kCheckWork units (entries of both
        // matrices plus rows and columns) per part, at most kCheckParts parts
        constexpr int64_t kCheckWork = 16384;
        constexpr int64_t kCheckParts = 64;
        std::vector<int4> items;
        for (int32_t k = 0; k < count; ++k) {
            const int64_t nnz_k = static_cast<int64_t>(rp[row_off[k + 1]]) - rp[row_off[k]];
            const int64_t work = 2 * nnz_k + (row_off[k + 1] - row_off[k]) + (col_off[k + 1] - col_off[k]);
            const int parts = static_cast<int>(
                std::min<int64_t>(kCheckParts, std::max<int64_t>(1, (work + kCheckWork - 1) / kCheckWork)));
            for (int j = 0; j < parts; ++j) items.push_back(make_int4(k, j, parts, 0));
        }
        c.n_chk = static_cast<int32_t>(items.size());
        BCK(upload(c.chk_item, items, s));
        BCK(c.chk_part.alloc(kBatchCheckVals * items.size()));
        BCK(c.chk_ticket.alloc(static_cast<size_t>(count)));
        BCK(cudaMemsetAsync(c.chk_ticket.p, 0, sizeof(unsigned int) * count, s));
        BCK(cudaStreamSynchronize(s));  // the host vector is read by the copy above
    }
    BCK(upload(c.c_o, cv, static_cast<size_t>(n), s));
    BCK(upload(c.lo_o, col_lo, static_cast<size_t>(n), s));
    BCK(upload(c.hi_o, col_hi, static_cast<size_t>(n), s));
    BCK(upload(c.rlo_o, row_lo, static_cast<size_t>(m), s));
    BCK(upload(c.rhi_o, row_hi, static_cast<size_t>(m), s));
    std::vector<InstState> h(static_cast<size_t>(count));
    std::memset(h.data(), 0, sizeof(InstState) * count);
    for (int32_t k = 0; k < count; ++k) {
        h[k].valid = c.valid[k];
        h[k].obj_sign = c.maximize[k] ? -1.0 : 1.0;
        h[k].obj_const = c.obj_const[k];
    }
    BCK(c.is.alloc(static_cast<size_t>(count)));
    BCK(cudaMemcpyAsync(c.is.p, h.data(), sizeof(InstState) * count, cudaMemcpyHostToDevice, s));
    BCK(c.g.alloc(1));
    BCK(cudaStreamSynchronize(s));
    pdhg_options o;
    pdhg_default_options(&o);
    rc = batch_intake(c, o);
    if (rc != PDHG_OK) return rc;
    c.loaded = true;
    return PDHG_OK;
}

int batch_opnorm(BatchCtx& c, int iterations) {
    cudaStream_t s = c.stream;
    BCK(c.pw_u.alloc(static_cast<size_t>(c.n) + 1));
    BCK(c.pw_v.alloc(static_cast<size_t>(c.m) + 1));
    BCK(c.pw_w.alloc(static_cast<size_t>(c.m) + 1));
    launch_fill(c.pw_u.p, c.n, 1.0, s);
    launch_fill(c.pw_v.p, c.m, 1.0, s);
    launch_fill(c.pw_w.p, c.m, 0.0, s);
    const BatchView b = c.view();
    for (int it = 0; it < iterations; ++it) {
        launch_batch_pw_w(b, c.pw_u.p, c.pw_v.p, c.pw_w.p, s);
        launch_batch_pw_norm_w(b, c.pw_w.p, s);
        launch_batch_pw_u(b, c.pw_w.p, c.pw_u.p, s);
        launch_batch_pw_norm_uv(b, c.pw_w.p, c.pw_u.p, c.pw_v.p, s);
    }
    BCK(cudaGetLastError());
    c.have_opnorm = true;
    c.opnorm_iters = iterations;
    return PDHG_OK;
}

template <class T>
Iterates<T> batch_iterates(BatchCtx& c);
template <>
Iterates<double> batch_iterates<double>(BatchCtx& c) {
    Iterates<double> it;
    it.x = c.x64.p;
    it.xbar = c.xbar64.p;
    it.s = c.s64.p;
    it.y = c.y64.p;
    it.xsum = c.xsum.p;
    it.ysum = c.ysum.p;
    if (c.halpern) {
        it.xa = c.xa64.p;
        it.sa = c.sa64.p;
        it.ya = c.ya64.p;
        it.halpern = 1;
    }
    return it;
}
template <>
Iterates<float> batch_iterates<float>(BatchCtx& c) {
    Iterates<float> it;
    it.x = c.x32.p;
    it.xbar = c.xbar32.p;
    it.s = c.s32.p;
    it.y = c.y32.p;
    it.psx = c.psx.p;
    it.psy = c.psy.p;
    it.xsum = c.xsum.p;
    it.ysum = c.ysum.p;
    if (c.halpern) {
        it.xa = c.xa32.p;
        it.sa = c.sa32.p;
        it.ya = c.ya32.p;
        it.halpern = 1;
    }
    return it;
}

template <class T>
void batch_period(BatchCtx& c, const BatchParams& p, long long iters, bool with_check,
                  long long budget, cudaGraphConditionalHandle h, int use_h, cudaStream_t s) {
    const BatchView b = c.view();
    const Iterates<T> it = batch_iterates<T>(c);
    for (long long t = 0; t < iters; ++t) {
        launch_batch_iter<T>(b, it, true, t == 0 ? 1 : 0, static_cast<int>(t), s);
        launch_batch_iter<T>(b, it, false, t == 0 ? 1 : 0, static_cast<int>(t), s);
    }
    if (with_check) {
        launch_batch_check<T>(b, it, p, s);
        launch_batch_restart<T>(b, it, p, s);
        launch_batch_compact(b, s);
        launch_batch_tick(b, iters, budget, h, use_h, s);
    }
}

// The solve graph: WHILE (condition set by batch_tick) { one check period }.
template <class T>
int build_batch_graph(BatchCtx& c, const BatchParams& p, long long budget) {
    cudaGraphExec_t& exec = c.graph[std::is_same<T, float>::value ? 0 : 1];
    if (exec != nullptr) {
        cudaGraphExecDestroy(exec);
        exec = nullptr;
    }
    cudaGraph_t graph = nullptr;
    BCK(cudaGraphCreate(&graph, 0));
    cudaGraphConditionalHandle handle;
    BCK(cudaGraphConditionalHandleCreate(&handle, graph, 1, cudaGraphCondAssignDefault));
    cudaGraphNodeParams cp = {};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = handle;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    cudaGraphNode_t node;
    BCK(cudaGraphAddNode(&node, graph, nullptr, 0, &cp));
    cudaGraph_t body = cp.conditional.phGraph_out[0];
    BCK(cudaStreamBeginCaptureToGraph(c.stream, body, nullptr, nullptr, 0,
                                      cudaStreamCaptureModeThreadLocal));
    batch_period<T>(c, p, p.period, true, budget, handle, 1, c.stream);
    cudaError_t e = cudaStreamEndCapture(c.stream, &body);
    if (e != cudaSuccess) {
        cudaGraphDestroy(graph);
        return cuda_fail(&c.err, e, "cudaStreamEndCapture");
    }
    e = cudaGraphInstantiate(&exec, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) return cuda_fail(&c.err, e, "cudaGraphInstantiate");
    return PDHG_OK;
}

// ---- autotuner of the lane-group width (lanes per row) of each pass --------

constexpr int64_t kBatchTuneMinNnz = int64_t{1} << 20;

// Rebuilds the active block lists for the current lane widths.
int batch_relist(BatchCtx& c, cudaStream_t s) {
    const int one = 1;
    BCK(cudaMemcpyAsync(&c.g.p->dirty, &one, sizeof one, cudaMemcpyHostToDevice, s));
    launch_batch_compact(c.view(), s);
    BCK(cudaGetLastError());
    return PDHG_OK;
}

// Device time of 5 launches of one pass after 2 untimed ones.
template <class T>
float batch_time_pass(BatchCtx& c, bool primal, cudaEvent_t e0, cudaEvent_t e1) {
    const BatchView b = c.view();
    const Iterates<T> it = batch_iterates<T>(c);
    launch_batch_iter<T>(b, it, primal, 0, 0, c.stream);
    launch_batch_iter<T>(b, it, primal, 0, 0, c.stream);
    cudaEventRecord(e0, c.stream);
    for (int r = 0; r < 5; ++r) launch_batch_iter<T>(b, it, primal, 0, 0, c.stream);
    cudaEventRecord(e1, c.stream);
    cudaEventSynchronize(e1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    return ms;
}

// Lanes per row for each pass of this precision: the binning's width (about
// half the mean row length), half of it and twice it, each timed in two
// rounds (so none is timed only on a cold GPU), a candidate replacing the
// current pick only when 5% faster. Runs on the solve's own iterates before
// the initial point is written (the initial point resets them). Batches
// under 2^20 nonzeros keep the binning's width (their passes are
// launch-bound). The choice holds until the next load.
template <class T>
int batch_tune(BatchCtx& c, bool autotune) {
    const int pi = std::is_same<T, float>::value ? 0 : 1;
    if (!autotune || c.nnz < kBatchTuneMinNnz) {
        c.As.vw = c.bin_vw[0];
        c.ATs.vw = c.bin_vw[1];
        return PDHG_OK;
    }
    if (c.tuned_vw[pi][0] != 0) {
        c.As.vw = c.tuned_vw[pi][0];
        c.ATs.vw = c.tuned_vw[pi][1];
        return PDHG_OK;
    }
    cudaEvent_t e0, e1;
    BCK(cudaEventCreate(&e0));
    BCK(cudaEventCreate(&e1));
    for (int pass = 0; pass < 2; ++pass) {  // 0: rows of A (dual), 1: rows of A^T (primal)
        MatDev& M = pass ? c.ATs : c.As;
        const int base = c.bin_vw[pass];
        std::vector<int> cand{base};
        if (M.n_short > 0) {
            if (base > 1) cand.push_back(base / 2);
            if (base < 32) cand.push_back(base * 2);
        }
        std::vector<float> t(cand.size(), 3.0e38f);
        for (int round = 0; round < 2; ++round)
            for (size_t i = 0; i < cand.size(); ++i) {
                M.vw = cand[i];
                int rc = batch_relist(c, c.stream);
                if (rc != PDHG_OK) return rc;
                t[i] = std::min(t[i], batch_time_pass<T>(c, pass == 1, e0, e1));
            }
        size_t pick = 0;
        for (size_t i = 1; i < cand.size(); ++i)
            if (t[i] < 0.95f * t[pick]) pick = i;
        M.vw = cand[pick];
        c.tuned_vw[pi][pass] = cand[pick];
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    BCK(cudaGetLastError());
    c.tune_timed[pi] = true;
    return PDHG_OK;
}

// Runs check periods from iteration iter0 (the global count) until every
// instance is done or iteration `last` (absolute) is reached; returns the
// negated stop code when the host asked the device to stop.
template <class T>
int batch_run(BatchCtx& c, const pdhg_options& o, std::chrono::steady_clock::time_point t0,
              long long* launches, bool allow_switch, long long iter0, long long last) {
    cudaStream_t s = c.stream;
    BatchParams p;
    p.tol = o.tolerance;
    p.bound_tol = o.tolerance > 1e-6 ? o.tolerance : 1e-6;
    p.restart_decrease = o.restart_sufficient_decrease;
    p.period = o.restart_check_period;
    p.termination_rule = o.termination_rule;
    p.restart_rule = o.restart_rule;
    p.primal_weight_update = o.primal_weight_update;
    p.x_last = c.x_last.p;
    p.y_last = c.y_last.p;
    p.act_avg = c.act_avg.p;
    p.allow_switch = allow_switch ? 1 : 0;
    launch_batch_compact(c.view(), s);  // the block lists of the instances now active
    const long long span = last > iter0 ? last - iter0 : 0;
    const long long n_periods = span / p.period;
    const long long tail = span % p.period;
    const long long budget = iter0 + n_periods * p.period;
    bool stop_sent = false;
    auto poll = [&]() {
        if (stop_sent) return;
        int code = 0;
        if (o.cancel_flag != nullptr && *o.cancel_flag) code = PDHG_STATUS_CANCELLED;
        else if (o.time_limit_seconds > 0.0 &&
                 std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count() >
                     o.time_limit_seconds)
            code = PDHG_STATUS_TIME_LIMIT;
        if (code != 0) {
            c.mail->stop_request = code;
            stop_sent = true;
        }
    };
    if (n_periods > 0) {
        const int gi = std::is_same<T, float>::value ? 0 : 1;
        long long key[11];
        key[0] = 1;
        key[1] = p.period;
        key[2] = budget;
        key[3] = p.termination_rule;
        key[4] = p.restart_rule;
        key[5] = p.primal_weight_update;
        key[6] = p.allow_switch;
        std::memcpy(&key[7], &p.tol, sizeof(double));
        std::memcpy(&key[8], &p.restart_decrease, sizeof(double));
        key[9] = c.As.vw;  // the lane groups baked into the iteration launches
        key[10] = c.ATs.vw;
        if (c.graph[gi] == nullptr || std::memcmp(key, c.graph_key[gi], sizeof key) != 0) {
            int rc = build_batch_graph<T>(c, p, budget);
            if (rc != PDHG_OK) return rc;
            std::memcpy(c.graph_key[gi], key, sizeof key);
        }
        BCK(cudaGraphLaunch(c.graph[gi], s));
        *launches += 1;
        while (true) {  // the graph runs to the end on the device; the host only polls limits
            const cudaError_t q = cudaStreamQuery(s);
            if (q == cudaSuccess) break;
            if (q != cudaErrorNotReady) return cuda_fail(&c.err, q, "cudaStreamQuery");
            poll();
            std::this_thread::sleep_for(std::chrono::microseconds(200));
        }
    }
    BatchGlobal gh;
    BCK(cudaMemcpy(&gh, c.g.p, sizeof gh, cudaMemcpyDeviceToHost));
    if (!gh.done && tail > 0 && !stop_sent) {
        batch_period<T>(c, p, tail, false, budget, cudaGraphConditionalHandle{}, 0, s);
        *launches += 2 * tail;
        BCK(cudaStreamSynchronize(s));
        gh.iter += tail;
        BCK(cudaMemcpy(c.g.p, &gh, sizeof gh, cudaMemcpyHostToDevice));
    }
    return stop_sent ? -c.mail->stop_request : PDHG_OK;
}

int batch_solve(BatchCtx& c, const pdhg_options& o, pdhg_info* infos, double* x, double* y,
                double* rcv) {
    const auto t0 = std::chrono::steady_clock::now();
    if (!c.loaded) {
        c.err = "pdhg_solve_batch: no batch loaded";
        return PDHG_ERR_INVALID_ARGUMENT;
    }
    if (o.precision != PDHG_PREC_MIXED && o.precision != PDHG_PREC_FP64) {
        c.err = "pdhg_solve_batch: the batched engine runs in precision mixed or fp64";
        return PDHG_ERR_UNSUPPORTED;
    }
    if (o.checkpoint != nullptr || o.trace_iters > 0 || o.infeasibility_detection != 0 ||
        o.restart_check_period < 1 ||
        o.termination_rule < 0 || o.termination_rule > 2 || o.restart_rule < 0 ||
        o.restart_rule > 2 || o.power_iterations < 0 ||
        (o.restart_rule == 2 && o.termination_rule != 2) || o.halpern < 0 || o.halpern > 1 ||
        (o.halpern && (o.termination_rule != 2 || o.restart_rule != 2))) {
        c.err = "pdhg_solve_batch: invalid options (no checkpoint / trace / infeasibility "
                "detection in batches; restart rule 2 needs termination rule 2; halpern needs "
                "both rules 2)";
        return PDHG_ERR_INVALID_ARGUMENT;
    }
    BCK(cudaSetDevice(c.device));
    cudaStream_t s = c.stream;
    pdhg_options def;
    pdhg_default_options(&def);
    const bool same_scaling = o.ruiz_iterations == def.ruiz_iterations &&
                              o.ruiz_tolerance == def.ruiz_tolerance &&
                              o.pock_chambolle_alpha == def.pock_chambolle_alpha &&
                              o.apply_ruiz == def.apply_ruiz &&
                              o.apply_pock_chambolle == def.apply_pock_chambolle;
    if (!same_scaling) {  // non-default scaling: redo the intake with it
        int rc = batch_intake(c, o);
        if (rc != PDHG_OK) return rc;
    }
    const bool f32 = o.precision == PDHG_PREC_MIXED;
    const size_t n1 = static_cast<size_t>(c.n) + 1, m1 = static_cast<size_t>(c.m) + 1;
    BCK(c.x64.alloc(n1));
    BCK(c.xbar64.alloc(n1));
    BCK(c.s64.alloc(m1));
    BCK(c.y64.alloc(m1));
    BCK(c.xsum.alloc(n1));
    BCK(c.ysum.alloc(m1));
    BCK(c.act_avg.alloc(m1));
    BCK(c.xo.alloc(n1));
    BCK(c.yo.alloc(m1));
    BCK(c.rc.alloc(n1));
    if (f32) {
        BCK(c.x32.alloc(n1));
        BCK(c.xbar32.alloc(n1));
        BCK(c.s32.alloc(m1));
        BCK(c.y32.alloc(m1));
        BCK(c.psx.alloc(n1));
        BCK(c.psy.alloc(m1));
    }
    if (o.primal_weight_update) {
        BCK(c.x_last.alloc(n1));
        BCK(c.y_last.alloc(m1));
    }
    c.halpern = o.halpern != 0;
    if (c.halpern) {  // anchors: FP64 always (the FP64 phase), FP32 with f32
        BCK(c.xa64.alloc(n1));
        BCK(c.sa64.alloc(m1));
        BCK(c.ya64.alloc(m1));
        if (f32) {
            BCK(c.xa32.alloc(n1));
            BCK(c.sa32.alloc(m1));
            BCK(c.ya32.alloc(m1));
        }
    }
    // reset the solver part of every instance's state
    std::vector<InstState> h(static_cast<size_t>(c.count));
    BCK(cudaMemcpy(h.data(), c.is.p, sizeof(InstState) * c.count, cudaMemcpyDeviceToHost));
    int active = 0;
    for (auto& st : h) {
        st.done = st.valid ? 0 : 1;
        st.status = st.valid ? PDHG_STATUS_NOT_SOLVED : PDHG_STATUS_NUMERICAL_FAILURE;
        st.converged = 0;
        st.fresh = 1;
        st.restart = st.restart_to_avg = st.avg_better = st.fold = st.fail_kind = 0;
        st.since_restart = st.restarts = st.stop_iter = 0;
        st.res_last = st.res_prev_cand = kInfB;
        st.cur_res = st.avg_res = st.orig_res = st.rel_kkt = 0.0;
        st.inv = 1.0;
        st.stalled = st.polished = 0;
        st.since_improve = st.switch_iter = st.idle = 0;
        st.best_res = kInfB;
        if (!c.have_opnorm || c.opnorm_iters != o.power_iterations) {
            st.pw_done = 0;
            st.opnorm = 0.0;
        }
        active += st.valid ? 1 : 0;
    }
    BCK(cudaMemcpy(c.is.p, h.data(), sizeof(InstState) * c.count, cudaMemcpyHostToDevice));
    BatchGlobal gh{};
    gh.active = active;
    gh.dirty = 1;  // the block lists are rebuilt before the first iteration
    gh.done = active == 0 ? 1 : 0;
    BCK(cudaMemcpy(c.g.p, &gh, sizeof gh, cudaMemcpyHostToDevice));
    std::memset(const_cast<Mailbox*>(c.mail), 0, sizeof(Mailbox));
    long long launches = 0;
    if (!c.have_opnorm || c.opnorm_iters != o.power_iterations) {
        int rc = batch_opnorm(c, o.power_iterations);
        if (rc != PDHG_OK) return rc;
        launches += 4LL * o.power_iterations;
    }
    BatchView b = c.view();
    launch_batch_steps(b, o.step_size_safety, o.primal_weight_update, s);
    {
        const int rc = f32 ? batch_tune<float>(c, o.autotune != 0)
                           : batch_tune<double>(c, o.autotune != 0);
        if (rc != PDHG_OK) return rc;
        BCK(cudaMemcpyAsync(c.g.p, &gh, sizeof gh, cudaMemcpyHostToDevice, s));  // lists rebuilt
        b = c.view();
    }
    // initial point (pdhg.cpp:268-270) or the warm start
    const double* x0d = nullptr;
    const double* y0d = nullptr;
    if (o.x0 != nullptr) {
        BCK(upload(c.x0s, o.x0, static_cast<size_t>(c.n), s));
        x0d = c.x0s.p;
    }
    if (o.y0 != nullptr) {
        BCK(upload(c.y0s, o.y0, static_cast<size_t>(c.m), s));
        y0d = c.y0s.p;
    }
    if (x0d != nullptr || y0d != nullptr)
        launch_batch_warm(b, const_cast<double*>(x0d), const_cast<double*>(y0d), s);
    if (f32)
        launch_init_point<float>(b.P, b.A, x0d, y0d, batch_iterates<float>(c), s);
    else
        launch_init_point<double>(b.P, b.A, x0d, y0d, batch_iterates<double>(c), s);
    if (c.halpern) {  // the first anchor is the initial point
        if (f32) launch_set_anchor<float>(batch_iterates<float>(c), c.n, c.m, s);
        else launch_set_anchor<double>(batch_iterates<double>(c), c.n, c.m, s);
    }
    if (o.primal_weight_update) {
        // restart points start at the initial point
        BCK(cudaStreamSynchronize(s));
        if (f32) {
            std::vector<float> hx(static_cast<size_t>(c.n)), hy(static_cast<size_t>(c.m));
            if (c.n) BCK(cudaMemcpy(hx.data(), c.x32.p, sizeof(float) * c.n, cudaMemcpyDeviceToHost));
            if (c.m) BCK(cudaMemcpy(hy.data(), c.y32.p, sizeof(float) * c.m, cudaMemcpyDeviceToHost));
            std::vector<double> dx(hx.begin(), hx.end()), dy(hy.begin(), hy.end());
            if (c.n) BCK(cudaMemcpy(c.x_last.p, dx.data(), sizeof(double) * c.n, cudaMemcpyHostToDevice));
            if (c.m) BCK(cudaMemcpy(c.y_last.p, dy.data(), sizeof(double) * c.m, cudaMemcpyHostToDevice));
        } else {
            if (c.n) BCK(cudaMemcpyAsync(c.x_last.p, c.x64.p, sizeof(double) * c.n, cudaMemcpyDeviceToDevice, s));
            if (c.m) BCK(cudaMemcpyAsync(c.y_last.p, c.y64.p, sizeof(double) * c.m, cudaMemcpyDeviceToDevice, s));
        }
    }
    BCK(cudaStreamSynchronize(s));
    // cancellation / time limit before the first iteration (pdhg.cpp:288-293)
    int early = 0;
    if (o.max_iterations > 0 && o.cancel_flag != nullptr && *o.cancel_flag) early = PDHG_STATUS_CANCELLED;
    else if (o.max_iterations > 0 && o.time_limit_seconds > 0.0 &&
             std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count() >
                 o.time_limit_seconds)
        early = PDHG_STATUS_TIME_LIMIT;
    cudaEvent_t e0, e1;
    BCK(cudaEventCreate(&e0));
    BCK(cudaEventCreate(&e1));
    BCK(cudaEventRecord(e0, s));
    int stop = 0;
    bool any_polished = false;
    const long long max_it = o.max_iterations > 0 ? o.max_iterations : 0;
    if (!early) {
        const bool allow_switch = f32 && o.polish_iterations != 0;
        int rc = f32 ? batch_run<float>(c, o, t0, &launches, allow_switch, 0, max_it)
                     : batch_run<double>(c, o, t0, &launches, false, 0, max_it);
        if (rc > 0) return rc;
        stop = -rc;
        if (allow_switch && stop == 0) {
            // Instances whose FP32 phase stalled continue in FP64 from their
            // point, with fresh averages and restart state (the single
            // engine's polish, per instance); the others stay done.
            BatchGlobal gh;
            BCK(cudaMemcpy(&gh, c.g.p, sizeof gh, cudaMemcpyDeviceToHost));
            BCK(cudaMemcpy(h.data(), c.is.p, sizeof(InstState) * c.count, cudaMemcpyDeviceToHost));
            int stalled = 0;
            for (auto& st : h) {
                if (!(st.stalled && st.status == kBatchStalled)) continue;
                ++stalled;
                st.done = 0;
                st.status = PDHG_STATUS_NOT_SOLVED;
                st.stalled = 0;
                st.polished = 1;
                st.switch_iter = st.stop_iter;
                st.idle = gh.iter - st.stop_iter;
                st.fresh = 1;
                st.restart = st.restart_to_avg = st.avg_better = st.fold = 0;
                st.since_restart = 0;
                st.res_last = st.res_prev_cand = kInfB;
            }
            long long last = max_it;
            if (o.polish_iterations > 0 && gh.iter + o.polish_iterations < last)
                last = gh.iter + o.polish_iterations;
            if (stalled > 0 && last > gh.iter) {
                any_polished = true;
                gh.active = stalled;
                gh.dirty = 1;
                gh.done = 0;
                BCK(cudaMemcpy(c.is.p, h.data(), sizeof(InstState) * c.count, cudaMemcpyHostToDevice));
                BCK(cudaMemcpy(c.g.p, &gh, sizeof gh, cudaMemcpyHostToDevice));
                launch_batch_widen(c.view(), batch_iterates<float>(c), batch_iterates<double>(c), s);
                launches += 1;
                rc = batch_run<double>(c, o, t0, &launches, false, gh.iter, last);
                if (rc > 0) return rc;
                stop = -rc;
            }
        }
    }
    BCK(cudaEventRecord(e1, s));
    BCK(cudaEventSynchronize(e1));
    float loop_ms = 0.f;
    cudaEventElapsedTime(&loop_ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    b = c.view();
    const double bt = o.tolerance > 1e-6 ? o.tolerance : 1e-6;
    if (f32) {
        launch_batch_final<float>(b, batch_iterates<float>(c), bt, c.xo.p, c.yo.p, c.rc.p, 0, s);
        launches += 1;
        if (any_polished) {
            launch_batch_final<double>(b, batch_iterates<double>(c), bt, c.xo.p, c.yo.p, c.rc.p, 1, s);
            launches += 1;
        }
    } else {
        launch_batch_final<double>(b, batch_iterates<double>(c), bt, c.xo.p, c.yo.p, c.rc.p, -1, s);
        launches += 1;
    }
    BCK(cudaMemcpyAsync(h.data(), c.is.p, sizeof(InstState) * c.count, cudaMemcpyDeviceToHost, s));
    BatchGlobal g2;
    BCK(cudaMemcpyAsync(&g2, c.g.p, sizeof g2, cudaMemcpyDeviceToHost, s));
    if (x != nullptr && c.n) BCK(cudaMemcpyAsync(x, c.xo.p, sizeof(double) * c.n, cudaMemcpyDeviceToHost, s));
    if (y != nullptr && c.m) BCK(cudaMemcpyAsync(y, c.yo.p, sizeof(double) * c.m, cudaMemcpyDeviceToHost, s));
    if (rcv != nullptr && c.n) BCK(cudaMemcpyAsync(rcv, c.rc.p, sizeof(double) * c.n, cudaMemcpyDeviceToHost, s));
    BCK(cudaStreamSynchronize(s));
    const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    for (int32_t k = 0; k < c.count; ++k) {
        pdhg_info& inf = infos[k];
        std::memset(&inf, 0, sizeof inf);
        const InstState& st = h[k];
        inf.operator_norm_estimate = st.opnorm;
        inf.restarts = st.restarts;
        inf.relative_kkt = st.rel_kkt;
        inf.kernel_launches = launches;
        inf.device_seconds = loop_ms * 1e-3;
        if (!st.valid) {
            inf.status = PDHG_STATUS_NUMERICAL_FAILURE;
            inf.operator_norm_estimate = 0.0;
            std::snprintf(inf.message, sizeof inf.message, "invalid problem: %s", c.why[k].c_str());
            continue;
        }
        if (early) {
            inf.status = early;
            inf.iterations = 0;
        } else if (st.done && st.status != kBatchStalled) {
            inf.status = st.status;
            inf.iterations = st.stop_iter;
        } else if (st.done) {  // stalled with no budget left for FP64
            inf.status = PDHG_STATUS_ITERATION_LIMIT;
            inf.iterations = st.stop_iter;
        } else {
            inf.status = stop != 0 ? stop : PDHG_STATUS_ITERATION_LIMIT;
            inf.iterations = g2.iter;
        }
        if (st.polished) inf.iterations -= st.idle;  // this instance's own iterations
        if (o.precision == PDHG_PREC_FP64) inf.fp64_iterations = inf.iterations;
        else if (st.polished) inf.fp64_iterations = inf.iterations - st.switch_iter;
        if (inf.status == PDHG_STATUS_NUMERICAL_FAILURE) {
            std::snprintf(inf.message, sizeof inf.message,
                          st.fail_kind == 2 ? "non-finite KKT residual (original units) at iteration %lld"
                                            : "non-finite KKT residual at iteration %lld",
                          inf.iterations);
            continue;
        }
        inf.has_point = 1;
        inf.objective = st.objective;
        inf.primal_infeasibility = st.pinf;
        inf.dual_infeasibility = st.dinf;
        inf.duality_gap = st.gap;
        inf.seconds = secs;
    }
    return PDHG_OK;
}

}  // namespace

BatchCtx* batch_new(int device, cudaStream_t stream, std::string& err) {
    std::unique_ptr<BatchCtx> b(new (std::nothrow) BatchCtx(device, stream, err));
    if (!b) return nullptr;
    void* mp = nullptr;
    if (cudaHostAlloc(&mp, sizeof(Mailbox), cudaHostAllocMapped) != cudaSuccess) return nullptr;
    b->mail = static_cast<Mailbox*>(mp);
    std::memset(mp, 0, sizeof(Mailbox));
    void* dp = nullptr;
    if (cudaHostGetDevicePointer(&dp, mp, 0) != cudaSuccess) return nullptr;
    b->mail_dev = static_cast<Mailbox*>(dp);
    return b.release();
}

void batch_delete(BatchCtx* b) { delete b; }

int batch_load_abi(BatchCtx& c, int32_t count, const int32_t* row_off, const int32_t* col_off,
                   int64_t nnz, const int32_t* rp, const int32_t* ci, const double* v,
                   const double* cv, const double* obj_const, const int* maximize,
                   const double* col_lo, const double* col_hi, const double* row_lo,
                   const double* row_hi) {
    return batch_load(c, count, row_off, col_off, nnz, rp, ci, v, cv, obj_const, maximize, col_lo,
                      col_hi, row_lo, row_hi);
}

int batch_solve_abi(BatchCtx& c, const pdhg_options* options, pdhg_info* infos, double* x,
                    double* y, double* rc) {
    if (infos == nullptr) {
        c.err = "pdhg_solve_batch: infos is NULL";
        return PDHG_ERR_INVALID_ARGUMENT;
    }
    pdhg_options o;
    if (options == nullptr) {
        pdhg_default_options(&o);
        o.precision = PDHG_PREC_MIXED;
    } else {
        o = *options;
    }
    return batch_solve(c, o, infos, x, y, rc);
}

int32_t batch_count(const BatchCtx& c) { return c.loaded ? c.count : 0; }

int batch_tuning_abi(const BatchCtx& c, int precision, int* out) {
    const int pi = precision == PDHG_PREC_MIXED ? 0 : 1;
    const bool have = c.tuned_vw[pi][0] != 0;
    out[0] = have ? c.tuned_vw[pi][1] : c.bin_vw[1];
    out[1] = have ? c.tuned_vw[pi][0] : c.bin_vw[0];
    out[2] = c.tune_timed[pi] ? 1 : 0;
    return PDHG_OK;
}

int batch_point_kkt_abi(BatchCtx& c, const double* x, const double* y, double* kkt) {
    if (!c.loaded || kkt == nullptr) {
        c.err = "pdhg_batch_start_kkt: no batch loaded or kkt is NULL";
        return PDHG_ERR_INVALID_ARGUMENT;
    }
    BCK(cudaSetDevice(c.device));
    cudaStream_t s = c.stream;
    DBuf<double> xd, yd, out;
    if (x != nullptr) BCK(upload(xd, x, static_cast<size_t>(c.n), s));
    if (y != nullptr) BCK(upload(yd, y, static_cast<size_t>(c.m), s));
    BCK(out.alloc(static_cast<size_t>(c.count)));
    launch_batch_point_kkt(c.view(), x != nullptr ? xd.p : nullptr, y != nullptr ? yd.p : nullptr,
                           out.p, s);
    BCK(cudaGetLastError());
    BCK(cudaMemcpyAsync(kkt, out.p, sizeof(double) * c.count, cudaMemcpyDeviceToHost, s));
    BCK(cudaStreamSynchronize(s));
    return PDHG_OK;
}

}  // namespace pdhg
