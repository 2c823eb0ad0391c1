// dev_buffer.cuh -- owning device buffers and the resident CSR used by the
// single-LP engine (engine.cu) and the batched engine (batch.cu).
#pragma once

#include <cuda_runtime.h>

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

struct MatDev {
    int32_t rows = 0, cols = 0;
    int64_t nnz = 0;
    DBuf<int32_t> rp, ci, long_rows, wrows, mid_rows, huge_rows;
    DBuf<double> v64;
    DBuf<float> v32;
    DBuf<char> tscratch;  // build_transpose scratch when this matrix is a transpose
    int32_t n_long = 0, n_short = 0, n_wrows = 0, n_mid = 0, n_huge = 0;
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
        d.mid_rows = mid_rows.p;
        d.huge_rows = huge_rows.p;
        d.n_mid = n_mid;
        d.n_huge = n_huge;
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

// Row binning on the device: long-row list, short-row count, lanes per short
// row (about half the mean short-row length, a power of two in [1, 32]), and
// the warp-row list of the ordered kernels.
inline int bin_matrix(MatDev& M, cudaStream_t s, std::string* err) {
    cudaError_t e = M.long_rows.alloc(static_cast<size_t>(M.rows) + 1);
    if (e != cudaSuccess) return cuda_fail(err, e, "bin_matrix");
    if ((e = M.wrows.alloc(static_cast<size_t>(M.rows) + 1)) != cudaSuccess ||
        (e = M.mid_rows.alloc(static_cast<size_t>(M.rows) + 1)) != cudaSuccess ||
        (e = M.huge_rows.alloc(static_cast<size_t>(M.rows) + 1)) != cudaSuccess)
        return cuda_fail(err, e, "bin_matrix");
    DBuf<unsigned long long> cnt;
    if ((e = cnt.alloc(8)) != cudaSuccess) return cuda_fail(err, e, "bin_matrix");
    cudaMemsetAsync(cnt.p, 0, 8 * sizeof(unsigned long long), s);
    launch_bin(M.rp.p, M.rows, kLongRow, M.long_rows.p, cnt.p, s);
    launch_bin(M.rp.p, M.rows, kWarpRow, M.wrows.p, cnt.p + 3, s);
    launch_bin_range(M.rp.p, M.rows, kLongRow, kHugeRow, M.mid_rows.p, cnt.p + 6, s);
    launch_bin_range(M.rp.p, M.rows, kHugeRow, 0x7fffffff, M.huge_rows.p, cnt.p + 7, s);
    unsigned long long h[8];
    cudaMemcpyAsync(h, cnt.p, sizeof h, cudaMemcpyDeviceToHost, s);
    if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return cuda_fail(err, e, "bin_matrix");
    M.n_long = static_cast<int32_t>(h[0]);
    M.n_short = static_cast<int32_t>(h[1]);
    M.n_wrows = static_cast<int32_t>(h[3]);
    M.n_mid = static_cast<int32_t>(h[6]);
    M.n_huge = static_cast<int32_t>(h[7]);
    const double mean = h[1] > 0 ? static_cast<double>(h[2]) / static_cast<double>(h[1]) : 0.0;
    int w = 1;
    while (w < 32 && 2.0 * w <= mean / 2.0 + 1e-9) w *= 2;
    M.vw = w;
    return PDHG_OK;
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
