// dev_buffer.cuh -- owning device buffers and the resident CSR used by the
// single-LP engine (engine.cu) and the batched engine (batch.cu).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
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
    DBuf<int32_t> rp, ci, long_rows;
    DBuf<double> v64;
    DBuf<float> v32;
    int32_t n_long = 0, n_short = 0;
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

inline int cuda_fail(std::string* err, cudaError_t e, const char* what) {
    *err = std::string(what) + ": " + cudaGetErrorString(e);
    return e == cudaErrorMemoryAllocation ? PDHG_ERR_OUT_OF_MEMORY : PDHG_ERR_BACKEND;
}

// Row binning on the device: long-row list, short-row count, lanes per short
// row (about half the mean short-row length, a power of two in [1, 32]).
inline int bin_matrix(MatDev& M, cudaStream_t s, std::string* err) {
    cudaError_t e = M.long_rows.alloc(static_cast<size_t>(M.rows) + 1);
    if (e != cudaSuccess) return cuda_fail(err, e, "bin_matrix");
    DBuf<unsigned long long> cnt;
    if ((e = cnt.alloc(3)) != cudaSuccess) return cuda_fail(err, e, "bin_matrix");
    cudaMemsetAsync(cnt.p, 0, 3 * sizeof(unsigned long long), s);
    launch_bin(M.rp.p, M.rows, kLongRow, M.long_rows.p, cnt.p, s);
    unsigned long long h[3];
    cudaMemcpyAsync(h, cnt.p, sizeof h, cudaMemcpyDeviceToHost, s);
    if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return cuda_fail(err, e, "bin_matrix");
    M.n_long = static_cast<int32_t>(h[0]);
    M.n_short = static_cast<int32_t>(h[1]);
    const double mean = h[1] > 0 ? static_cast<double>(h[2]) / static_cast<double>(h[1]) : 0.0;
    int w = 1;
    while (w < 32 && 2.0 * w <= mean / 2.0 + 1e-9) w *= 2;
    M.vw = w;
    return PDHG_OK;
}

// A from host arrays (read in place) and A^T built on the device, both binned.
inline int upload_matrix(int32_t rows, int32_t cols, int64_t nnz, const int32_t* rp,
                         const int32_t* ci, const double* v, MatDev& M, MatDev& MT,
                         cudaStream_t s, std::string* err) {
    cudaError_t e;
    M.rows = rows;
    M.cols = cols;
    M.nnz = nnz;
    if ((e = upload(M.rp, rp, static_cast<size_t>(rows) + 1, s)) != cudaSuccess ||
        (e = upload(M.ci, ci, static_cast<size_t>(nnz), s)) != cudaSuccess ||
        (e = upload(M.v64, v, static_cast<size_t>(nnz), s)) != cudaSuccess)
        return cuda_fail(err, e, "upload_matrix");
    MT.rows = cols;
    MT.cols = rows;
    MT.nnz = nnz;
    if ((e = MT.rp.alloc(static_cast<size_t>(cols) + 1)) != cudaSuccess ||
        (e = MT.ci.alloc(static_cast<size_t>(nnz))) != cudaSuccess ||
        (e = MT.v64.alloc(static_cast<size_t>(nnz))) != cudaSuccess)
        return cuda_fail(err, e, "upload_matrix");
    TransposeOut out{MT.rp.p, MT.ci.p, MT.v64.p};
    if (build_transpose(rows, cols, nnz, M.rp.p, M.ci.p, M.v64.p, out, s) != 0)
        return cuda_fail(err, cudaGetLastError(), "build_transpose");
    int rc = bin_matrix(M, s, err);
    if (rc != PDHG_OK) return rc;
    return bin_matrix(MT, s, err);
}

}  // namespace pdhg
