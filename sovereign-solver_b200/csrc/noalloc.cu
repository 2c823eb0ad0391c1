// noalloc.cu -- y := alpha * op(A) * x + beta * y on caller-owned device
// buffers, with no device allocation at all.
//
// Who needs this: callers that cannot call cudaMalloc (or any allocating
// routine) at the point they need a product -- code inside a framework that
// owns all device memory through its own pool (an allocation outside the pool
// can fail or fragment it), or a real-time loop that must not touch the
// driver's allocator (an allocation can synchronise the device). They hand
// over device buffers they already own; the transposed
// product still needs A^T, so that scratch lives in one file-scope __device__
// array of fixed size, reserved when the library is loaded.
//
// The arithmetic is the one of pdhg_csr_spmv: each output sums its terms in
// the reference's order (src/l0/backend_host.cpp:415-423 and 434-444), so the
// two entry points return bit-identical results.
#include <cstddef>
#include <mutex>

#include "../../include/pdhg_b200.h"
#include "engine.cuh"

namespace pdhg {

namespace {

// Limits of the no-allocation path (see pdhg_csr_spmv_noalloc in the header).
constexpr int32_t kNaMaxCols = 1 << 18;  // columns of A (rows of A^T)
constexpr int32_t kNaMaxNnz = 1 << 18;   // nonzeros of A

struct NaScratch {
    int32_t rp[kNaMaxCols + 1];  // A^T row pointer
    int32_t cursor[kNaMaxCols];  // per-column fill position
    int32_t ci[kNaMaxNnz];       // A^T column index (= row of A)
    double v[kNaMaxNnz];         // A^T values
};

// Every GPU that loads the library holds this (about 5 MB) until exit.
static __device__ __align__(256) NaScratch g_na_scratch;

constexpr int kNaBlock = 256;

__global__ void k_na_zero(NaScratch* s, int32_t n) {
    const int t = blockIdx.x * kNaBlock + threadIdx.x;
    if (t <= n) s->rp[t] = 0;
    if (t < n) s->cursor[t] = 0;
}

// Column indices outside [0, n) are skipped here and in k_na_place, so a bad
// index can never write outside the fixed array.
__global__ void k_na_count(int32_t m, int32_t n, const int32_t* rp, const int32_t* ci,
                           NaScratch* s) {
    const int r = blockIdx.x * kNaBlock + threadIdx.x;
    if (r >= m) return;
    for (int k = rp[r]; k < rp[r + 1]; ++k) {
        const int c = ci[k];
        if (c >= 0 && c < n) atomicAdd(&s->cursor[c], 1);
    }
}

// Exclusive scan of the n column counts into rp (one CTA of 1024 threads,
// each owning a contiguous chunk); cursor becomes each column's start.
__global__ void __launch_bounds__(1024) k_na_scan(NaScratch* s, int32_t n) {
    __shared__ int32_t tot[1024];
    const int t = threadIdx.x;
    const int chunk = (n + 1023) / 1024;
    const int b = t * chunk;
    const int e = b + chunk < n ? b + chunk : n;
    int32_t sum = 0;
    for (int c = b; c < e; ++c) sum += s->cursor[c];
    tot[t] = sum;
    __syncthreads();
    for (int o = 1; o < 1024; o <<= 1) {  // Hillis-Steele inclusive scan of chunk totals
        const int32_t add = t >= o ? tot[t - o] : 0;
        __syncthreads();
        tot[t] += add;
        __syncthreads();
    }
    int32_t run = tot[t] - sum;  // exclusive start of this chunk
    for (int c = b; c < e; ++c) {
        const int32_t len = s->cursor[c];
        s->rp[c] = run;
        s->cursor[c] = run;
        run += len;
    }
    if (t == 1023) s->rp[n] = tot[1023];
}

__global__ void k_na_place(int32_t m, int32_t n, const int32_t* rp, const int32_t* ci,
                           const double* v, NaScratch* s) {
    const int r = blockIdx.x * kNaBlock + threadIdx.x;
    if (r >= m) return;
    for (int k = rp[r]; k < rp[r + 1]; ++k) {
        const int c = ci[k];
        if (c < 0 || c >= n) continue;
        const int pos = atomicAdd(&s->cursor[c], 1);
        s->ci[pos] = r;
        s->v[pos] = v[k];
    }
}

// Atomic placement leaves each column's entries in arbitrary order; a heap
// sort by row (rows are distinct within a column) restores ascending rows.
__device__ void na_sift(int32_t* key, double* val, int root, int len) {
    while (true) {
        int child = 2 * root + 1;
        if (child >= len) return;
        if (child + 1 < len && key[child + 1] > key[child]) ++child;
        if (key[root] >= key[child]) return;
        const int32_t tk = key[root];
        key[root] = key[child];
        key[child] = tk;
        const double tv = val[root];
        val[root] = val[child];
        val[child] = tv;
        root = child;
    }
}

__global__ void k_na_sort(NaScratch* s, int32_t n) {
    const int c = blockIdx.x * kNaBlock + threadIdx.x;
    if (c >= n) return;
    int32_t* key = s->ci + s->rp[c];
    double* val = s->v + s->rp[c];
    const int len = s->rp[c + 1] - s->rp[c];
    for (int i = len / 2 - 1; i >= 0; --i) na_sift(key, val, i, len);
    for (int end = len - 1; end > 0; --end) {
        const int32_t tk = key[0];
        key[0] = key[end];
        key[end] = tk;
        const double tv = val[0];
        val[0] = val[end];
        val[end] = tv;
        na_sift(key, val, 0, end);
    }
}

// The device address of g_na_scratch for each device, looked up once per
// device (host code may not use the symbol itself as a device address).
constexpr int kNaMaxDevices = 64;
NaScratch* g_na_ptr[kNaMaxDevices] = {};
std::mutex g_na_mutex;

int na_scratch(int device, NaScratch** out) {
    if (device < 0 || device >= kNaMaxDevices) return PDHG_ERR_UNSUPPORTED;
    std::lock_guard<std::mutex> lock(g_na_mutex);
    if (g_na_ptr[device] == nullptr) {
        void* p = nullptr;
        if (cudaGetSymbolAddress(&p, g_na_scratch) != cudaSuccess || p == nullptr)
            return PDHG_ERR_BACKEND;
        g_na_ptr[device] = static_cast<NaScratch*>(p);
    }
    *out = g_na_ptr[device];
    return PDHG_OK;
}

}  // namespace
}  // namespace pdhg

extern "C" int pdhg_csr_spmv_noalloc(int transpose, int32_t m, int32_t n, int64_t nnz,
                                     const int32_t* d_row_ptr, const int32_t* d_col_idx,
                                     const double* d_values, double alpha, const double* d_x,
                                     double beta, double* d_y, void* stream) {
    using namespace pdhg;
    if (m < 0 || n < 0 || nnz < 0 || d_row_ptr == nullptr || d_y == nullptr ||
        (nnz > 0 && (d_col_idx == nullptr || d_values == nullptr || d_x == nullptr)))
        return PDHG_ERR_INVALID_ARGUMENT;
    if (transpose && (n > kNaMaxCols || nnz > kNaMaxNnz))
        return PDHG_ERR_INVALID_ARGUMENT;  // beyond the fixed scratch of the no-allocation path
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    DevCsr A;
    A.rows = m;
    A.cols = n;
    A.nnz = nnz;
    A.rp = d_row_ptr;
    A.ci = d_col_idx;
    A.v64 = d_values;
    if (!transpose) {
        launch_spmv_exact(A, alpha, d_x, beta, d_y, s);
        return cudaGetLastError() == cudaSuccess ? PDHG_OK : PDHG_ERR_BACKEND;
    }
    int device = 0;
    if (cudaGetDevice(&device) != cudaSuccess) return PDHG_ERR_BACKEND;
    NaScratch* sc = nullptr;
    const int rc = na_scratch(device, &sc);
    if (rc != PDHG_OK) return rc;
    const int gn = (n + 1 + kNaBlock - 1) / kNaBlock;
    const int gm = (m + kNaBlock - 1) / kNaBlock;
    k_na_zero<<<gn, kNaBlock, 0, s>>>(sc, n);  // the array keeps the previous call's contents
    if (m > 0) k_na_count<<<gm, kNaBlock, 0, s>>>(m, n, d_row_ptr, d_col_idx, sc);
    k_na_scan<<<1, 1024, 0, s>>>(sc, n);
    if (m > 0) k_na_place<<<gm, kNaBlock, 0, s>>>(m, n, d_row_ptr, d_col_idx, d_values, sc);
    if (n > 0) k_na_sort<<<(n + kNaBlock - 1) / kNaBlock, kNaBlock, 0, s>>>(sc, n);
    // member addresses inside the device array (offsets only; nothing is read here)
    char* base = reinterpret_cast<char*>(sc);
    DevCsr AT;
    AT.rows = n;
    AT.cols = m;
    AT.nnz = nnz;
    AT.rp = reinterpret_cast<const int32_t*>(base + offsetof(NaScratch, rp));
    AT.ci = reinterpret_cast<const int32_t*>(base + offsetof(NaScratch, ci));
    AT.v64 = reinterpret_cast<const double*>(base + offsetof(NaScratch, v));
    launch_spmvT_exact(AT, alpha, d_x, beta, d_y, s);
    return cudaGetLastError() == cudaSuccess ? PDHG_OK : PDHG_ERR_BACKEND;
}
