// dev_buffer.cuh -- owning device buffers and the resident CSR used by the
// single-LP engine (engine.cu) and the batched engine (batch.cu).
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "../../include/pdhg_b200.h"
#include "engine.cuh"

namespace pdhg {

template <class T>
struct DBuf {
    T* p = nullptr;
    size_t n = 0;
    DBuf() = default;
    DBuf(const DBuf&) = delete;
    DBuf& operator=(const DBuf&) = delete;
    ~DBuf() { release(); }
    void release() {
        if (p != nullptr) cudaFree(p);
        p = nullptr;
        n = 0;
    }
    cudaError_t alloc(size_t count) {
        if (count == n && p != nullptr) return cudaSuccess;
        release();
        n = count;
        if (count == 0) return cudaSuccess;
        return cudaMalloc(reinterpret_cast<void**>(&p), sizeof(T) * count);
    }
};

// Owning storage of a RowItems list.
struct ItemsDev {
    DBuf<int4> item;
    DBuf<int2> split;
    DBuf<unsigned int> ticket;
    DBuf<double> part;
    int32_t n_item = 0;
    RowItems view() const {
        RowItems v;
        v.item = item.p;
        v.split = split.p;
        v.ticket = ticket.p;
        v.part = part.p;
        v.n_item = n_item;
        return v;
    }
};

struct MatDev {
    int32_t rows = 0, cols = 0;
    int64_t nnz = 0;
    DBuf<int32_t> rp, ci, long_rows, wrows, warp_rows0, warp_rows1;
    ItemsDev items_long, items_huge, items_warp;
    DBuf<double> v64;
    DBuf<float> v32;
    DBuf<char> tscratch;  // build_transpose scratch when this matrix is a transpose
    int32_t n_long = 0, n_short = 0, n_wrows = 0, n_mid = 0, n_huge = 0;
    int32_t short_max = kLongRow, n_iter_short = 0, n_warp0 = 0, n_warp1 = 0;
    int vw = 1;
    DevCsr view() const {
        DevCsr d;
        d.rows = rows;
        d.cols = cols;
        d.nnz = nnz;
        d.rp = rp.p;
        d.ci = ci.p;
        d.v64 = v64.p;
        d.v32 = v32.p;
        d.long_rows = long_rows.p;
        d.n_long = n_long;
        d.n_short = n_short;
        d.vw = vw;
        d.wrows = wrows.p;
        d.n_wrows = n_wrows;
        d.short_max = short_max;
        d.n_iter_short = n_iter_short;
        d.warp_rows0 = warp_rows0.p;
        d.warp_rows1 = warp_rows1.p;
        d.n_warp0 = n_warp0;
        d.n_warp1 = n_warp1;
        d.n_mid = n_mid;
        d.n_huge = n_huge;
        d.items_long = items_long.view();
        d.items_huge = items_huge.view();
        d.items_warp = items_warp.view();
        return d;
    }
};

template <class T>
inline cudaError_t upload(DBuf<T>& d, const T* h, size_t n, cudaStream_t s) {
    cudaError_t e = d.alloc(n);
    if (e != cudaSuccess || n == 0) return e;
    return cudaMemcpyAsync(d.p, h, sizeof(T) * n, cudaMemcpyHostToDevice, s);
}

template <class T>
inline cudaError_t upload(DBuf<T>& d, const std::vector<T>& h, cudaStream_t s) {
    return upload(d, h.data(), h.size(), s);
}

template <class T>
inline cudaError_t copy_dev(DBuf<T>& d, const T* src, size_t n, cudaStream_t s) {
    cudaError_t e = d.alloc(n);
    if (e != cudaSuccess || n == 0) return e;
    return cudaMemcpyAsync(d.p, src, sizeof(T) * n, cudaMemcpyDeviceToDevice, s);
}

inline cudaError_t to_float(DBuf<float>& d, const DBuf<double>& src, cudaStream_t s) {
    cudaError_t e = d.alloc(src.n);
    if (e != cudaSuccess) return e;
    launch_to_float(src.p, d.p, static_cast<int64_t>(src.n), s);
    return cudaGetLastError();
}

// Opt-in phase timing for load and solve: with PDHG_B200_PHASE_TIMES=1 in the
// environment every mark waits for the stream and prints, to stderr, the host
// wall time since the previous mark. Off (no waits, no output) otherwise.
inline bool phase_times_enabled() {
    static const bool on = [] {
        const char* e = std::getenv("PDHG_B200_PHASE_TIMES");
        return e != nullptr && e[0] == '1';
    }();
    return on;
}

struct PhaseClock {
    bool on;
    cudaStream_t s;
    std::chrono::steady_clock::time_point t;
    explicit PhaseClock(cudaStream_t st)
        : on(phase_times_enabled()), s(st), t(std::chrono::steady_clock::now()) {}
    void mark(const char* what) {
        if (!on) return;
        cudaStreamSynchronize(s);
        const auto now = std::chrono::steady_clock::now();
        std::fprintf(stderr, "[pdhg phase] %-22s %10.3f ms\n", what,
                     std::chrono::duration<double, std::milli>(now - t).count());
        t = now;
    }
};

inline int cuda_fail(std::string* err, cudaError_t e, const char* what) {
    *err = std::string(what) + ": " + cudaGetErrorString(e);
    return e == cudaErrorMemoryAllocation ? PDHG_ERR_OUT_OF_MEMORY : PDHG_ERR_BACKEND;
}

// Work items (RowItems) over the rows of `ext` ({row, begin, end, -}, in row
// order) longer than min_len: one item per row of at most seg entries, else
// ceil(len / seg) near-equal segments. seg is min_seg, or more when the rows'
// entries would make more than two items per resident CTA (or warp) of the
// GPU (`resident`): rows are split only as far as filling the GPU needs.
inline int build_items(const std::vector<int4>& ext, int min_len, int min_seg, int resident,
                       ItemsDev& D, cudaStream_t s, std::string* err) {
    int64_t total = 0;
    for (const int4& r : ext)
        if (r.z - r.y > min_len) total += static_cast<int64_t>(r.z) - r.y;
    const int64_t seg = std::max<int64_t>(min_seg, (total + 2 * resident - 1) / (2 * resident));
    std::vector<int4> items;
    std::vector<int2> splits;
    for (const int4& r : ext) {
        const int64_t len = static_cast<int64_t>(r.z) - r.y;
        if (len <= min_len) continue;
        const int64_t nseg = (len + seg - 1) / seg;
        if (nseg <= 1) {
            items.push_back(make_int4(r.x, r.y, r.z, -1));
            continue;
        }
        const int sid = static_cast<int>(splits.size());
        splits.push_back(make_int2(static_cast<int>(items.size()), static_cast<int>(nseg)));
        for (int64_t k = 0; k < nseg; ++k) {
            const int b = r.y + static_cast<int>(len * k / nseg);
            const int e = r.y + static_cast<int>(len * (k + 1) / nseg);
            items.push_back(make_int4(r.x, b, e, sid));
        }
    }
    D.n_item = static_cast<int32_t>(items.size());
    cudaError_t e;
    if ((e = upload(D.item, items.data(), items.size(), s)) != cudaSuccess ||
        (e = upload(D.split, splits.data(), splits.size(), s)) != cudaSuccess ||
        (e = D.ticket.alloc(splits.size())) != cudaSuccess ||
        (e = D.part.alloc(2 * items.size())) != cudaSuccess)
        return cuda_fail(err, e, "build_items");
    if (!splits.empty()) cudaMemsetAsync(D.ticket.p, 0, sizeof(unsigned int) * splits.size(), s);
    // the host vectors are read by the copies above before they go out of scope
    if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return cuda_fail(err, e, "build_items");
    return PDHG_OK;
}

// Row binning on the device: long-row list, short-row count, lanes per short
// row (about half the mean short-row length, a power of two in [1, 32]), the
// warp-row list of the ordered kernels, and the throughput kernels' tiers:
// short rows up to short_max, the two warp-row lists and the CTA work items.
inline int bin_matrix(MatDev& M, cudaStream_t s, std::string* err) {
    cudaError_t e = M.long_rows.alloc(static_cast<size_t>(M.rows) + 1);
    if (e != cudaSuccess) return cuda_fail(err, e, "bin_matrix");
    if ((e = M.wrows.alloc(static_cast<size_t>(M.rows) + 1)) != cudaSuccess ||
        (e = M.warp_rows0.alloc(static_cast<size_t>(M.rows) + 1)) != cudaSuccess ||
        (e = M.warp_rows1.alloc(static_cast<size_t>(M.rows) + 1)) != cudaSuccess)
        return cuda_fail(err, e, "bin_matrix");
    DBuf<unsigned long long> cnt;
    if ((e = cnt.alloc(8)) != cudaSuccess) return cuda_fail(err, e, "bin_matrix");
    cudaMemsetAsync(cnt.p, 0, 8 * sizeof(unsigned long long), s);
    launch_bin(M.rp.p, M.rows, kLongRow, M.long_rows.p, cnt.p, s);
    launch_bin(M.rp.p, M.rows, kWarpRow, M.wrows.p, cnt.p + 3, s);
    unsigned long long h[8];
    cudaMemcpyAsync(h, cnt.p, sizeof h, cudaMemcpyDeviceToHost, s);
    if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return cuda_fail(err, e, "bin_matrix");
    M.n_long = static_cast<int32_t>(h[0]);
    M.n_short = static_cast<int32_t>(h[1]);
    M.n_wrows = static_cast<int32_t>(h[3]);
    const double mean = h[1] > 0 ? static_cast<double>(h[2]) / static_cast<double>(h[1]) : 0.0;
    int w = 1;
    while (w < 32 && 2.0 * w <= mean / 2.0 + 1e-9) w *= 2;
    M.vw = w;
    // lane groups take rows of up to 16 lanes' worth (a few unrolled rounds
    // per lane); longer rows go to a warp each
    M.short_max = std::min(kLongRow, std::max(kWarpRow, 16 * w));
    launch_bin_range(M.rp.p, M.rows, M.short_max, kLongRow, M.warp_rows0.p, cnt.p + 6, s);
    launch_bin_range(M.rp.p, M.rows, M.short_max, kHugeRow, M.warp_rows1.p, cnt.p + 7, s);
    cudaMemcpyAsync(h, cnt.p, sizeof h, cudaMemcpyDeviceToHost, s);
    if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return cuda_fail(err, e, "bin_matrix");
    M.n_warp0 = static_cast<int32_t>(h[6]);
    M.n_warp1 = static_cast<int32_t>(h[7]);

    // extents of every row above short_max (warp_rows0 + long rows), in row
    // order (the binning kernels append in arrival order)
    std::vector<int4> ext(static_cast<size_t>(M.n_long) + static_cast<size_t>(M.n_warp0));
    if (!ext.empty()) {
        DBuf<int4> d_ext;
        if ((e = d_ext.alloc(ext.size())) != cudaSuccess) return cuda_fail(err, e, "bin_matrix");
        launch_row_extents(M.long_rows.p, M.n_long, M.rp.p, d_ext.p, s);
        launch_row_extents(M.warp_rows0.p, M.n_warp0, M.rp.p, d_ext.p + M.n_long, s);
        cudaMemcpyAsync(ext.data(), d_ext.p, sizeof(int4) * ext.size(), cudaMemcpyDeviceToHost, s);
        if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return cuda_fail(err, e, "bin_matrix");
        std::sort(ext.begin(), ext.end(), [](const int4& a, const int4& b) { return a.x < b.x; });
    }
    M.n_huge = 0;
    for (const int4& r : ext) M.n_huge += (r.z - r.y > kHugeRow) ? 1 : 0;
    M.n_mid = M.n_long - M.n_huge;
    M.n_iter_short = M.rows - M.n_warp1 - M.n_huge;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    sms = std::max(sms, 1);
    const int resident = 4 * sms;  // the long-row kernel's CTAs per SM
    int rc = build_items(ext, kLongRow, kSegLen, resident, M.items_long, s, err);
    if (rc != PDHG_OK) return rc;
    rc = build_items(ext, kHugeRow, kSegLen, resident, M.items_huge, s, err);
    if (rc != PDHG_OK) return rc;
    return build_items(ext, M.short_max, kWarpSegLen, 32 * sms, M.items_warp, s, err);
}

// row_ptr structure on the host (rows + 1 reads): starts at 0, ends at nnz,
// non-decreasing. Every device kernel that walks rows relies on it.
inline bool row_ptr_ok(int32_t rows, int64_t nnz, const int32_t* rp) {
    if (rp[0] != 0 || rp[rows] != nnz) return false;
    for (int32_t r = 0; r < rows; ++r)
        if (rp[r] > rp[r + 1]) return false;
    return true;
}

// A's arrays to the device, read in place from the caller's host buffers.
inline int upload_csr(int32_t rows, int32_t cols, int64_t nnz, const int32_t* rp,
                      const int32_t* ci, const double* v, MatDev& M, cudaStream_t s,
                      std::string* err) {
    cudaError_t e;
    M.rows = rows;
    M.cols = cols;
    M.nnz = nnz;
    if ((e = upload(M.rp, rp, static_cast<size_t>(rows) + 1, s)) != cudaSuccess ||
        (e = upload(M.ci, ci, static_cast<size_t>(nnz), s)) != cudaSuccess ||
        (e = upload(M.v64, v, static_cast<size_t>(nnz), s)) != cudaSuccess)
        return cuda_fail(err, e, "upload_csr");
    return PDHG_OK;
}

// The device problem checks (launch_validate) on data already resident;
// *flags gets the OR of the failing kinds (0: nothing failed).
inline int device_checks(const MatDev& M, const double* c, const double* clo, const double* chi,
                         const double* rlo, const double* rhi, unsigned* flags, cudaStream_t s,
                         std::string* err) {
    DBuf<unsigned> f;
    cudaError_t e = f.alloc(1);
    if (e != cudaSuccess) return cuda_fail(err, e, "device_checks");
    cudaMemsetAsync(f.p, 0, sizeof(unsigned), s);
    launch_validate(M.rows, M.cols, M.rp.p, M.ci.p, M.v64.p, c, clo, chi, rlo, rhi, M.nnz, f.p, s);
    cudaMemcpyAsync(flags, f.p, sizeof(unsigned), cudaMemcpyDeviceToHost, s);
    if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return cuda_fail(err, e, "device_checks");
    return PDHG_OK;
}

// A^T built on the device from the resident A, then both binned.
inline int finish_matrix(MatDev& M, MatDev& MT, cudaStream_t s, std::string* err) {
    cudaError_t e;
    PhaseClock pc(s);
    MT.rows = M.cols;
    MT.cols = M.rows;
    MT.nnz = M.nnz;
    if ((e = MT.rp.alloc(static_cast<size_t>(M.cols) + 1)) != cudaSuccess ||
        (e = MT.ci.alloc(static_cast<size_t>(M.nnz))) != cudaSuccess ||
        (e = MT.v64.alloc(static_cast<size_t>(M.nnz))) != cudaSuccess)
        return cuda_fail(err, e, "finish_matrix");
    if ((e = MT.tscratch.alloc(transpose_scratch_bytes(M.rows, M.cols, M.nnz))) != cudaSuccess)
        return cuda_fail(err, e, "finish_matrix");
    TransposeOut out{MT.rp.p, MT.ci.p, MT.v64.p};
    if (build_transpose(M.rows, M.cols, M.nnz, M.rp.p, M.ci.p, M.v64.p, out, MT.tscratch.p, s) != 0)
        return cuda_fail(err, cudaGetLastError(), "build_transpose");
    pc.mark("matrix: transpose");
    int rc = bin_matrix(M, s, err);
    if (rc != PDHG_OK) return rc;
    rc = bin_matrix(MT, s, err);
    pc.mark("matrix: bins");
    return rc;
}

// A matrix on its own (no problem around it): row_ptr checked on the host and
// the column indices on the device, then A^T and the bins. A matrix whose
// structure would send a kernel out of bounds returns PDHG_ERR_INVALID_ARGUMENT
// before any kernel indexes by it; unsorted columns and non-finite values are
// the caller's (the product is formed as given).
inline int upload_matrix(int32_t rows, int32_t cols, int64_t nnz, const int32_t* rp,
                         const int32_t* ci, const double* v, MatDev& M, MatDev& MT,
                         cudaStream_t s, std::string* err) {
    if (!row_ptr_ok(rows, nnz, rp)) {
        *err = "invalid CSR matrix: row_ptr must start at 0, end at nnz and not decrease";
        return PDHG_ERR_INVALID_ARGUMENT;
    }
    int rc = upload_csr(rows, cols, nnz, rp, ci, v, M, s, err);
    if (rc != PDHG_OK) return rc;
    unsigned flags = 0;
    rc = device_checks(M, nullptr, nullptr, nullptr, nullptr, nullptr, &flags, s, err);
    if (rc != PDHG_OK) return rc;
    if (flags & 4u) {
        *err = "invalid CSR matrix: column index out of range";
        return PDHG_ERR_INVALID_ARGUMENT;
    }
    return finish_matrix(M, MT, s, err);
}

}  // namespace pdhg
