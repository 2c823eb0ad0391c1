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
#include <algorithm>
#include <cstddef>
#include <limits>
#include <mutex>

#include <math_constants.h>

#include "../../include/pdhg_b200.h"
#include "engine.cuh"
#include "ordered.cuh"

namespace pdhg {

namespace {

// Limits of the no-allocation path (see pdhg_csr_spmv_noalloc in the header).
constexpr int32_t kNaMaxCols = 1 << 18;  // columns of A (rows of A^T)
constexpr int32_t kNaMaxNnz = 1 << 18;   // nonzeros of A

struct NaScratch {
    int32_t rp[kNaMaxCols + 1];  // A^T row pointer
    int32_t cursor[kNaMaxCols];  // per-column fill position
    int32_t ci[kNaMaxNnz];       // A^T column index (= row of A)
    int32_t src[kNaMaxNnz];      // position k of the entry in A (sort key)
    double v[kNaMaxNnz];         // A^T values
    int32_t bad;                 // the caller's CSR broke the contract (set by k_na_validate)
};

// Every GPU that loads the library holds this (about 6 MB) until exit.
static __device__ __align__(256) NaScratch g_na_scratch;

constexpr int kNaBlock = 256;
constexpr int kNaGridCap = 4096;

int na_grid(int64_t work) {
    const int64_t g = (work + kNaBlock - 1) / kNaBlock;
    return static_cast<int>(g < 1 ? 1 : (g > kNaGridCap ? kNaGridCap : g));
}

// Clears the column counters, the A^T row pointer (transposed products) and
// the error flag. The array keeps the previous call's contents otherwise.
__global__ void k_na_zero(NaScratch* s, int32_t n) {
    const int t = blockIdx.x * kNaBlock + threadIdx.x;
    if (t == 0) s->bad = 0;
    if (t <= n) s->rp[t] = 0;
    if (t < n) s->cursor[t] = 0;
}

// The caller's CSR must be well formed: rp[0] = 0, rp[m] = nnz, no row
// pointer decreasing, every column index in [0, n). Grid-stride over the m
// row pointers and the nnz column indices, reading nothing past them. Any
// violation sets s->bad; every later kernel of the call then leaves the
// scratch alone and fills y with NaN, so a malformed CSR can neither index
// outside the caller's buffers and the fixed array nor go unnoticed.
__global__ void k_na_validate(int32_t m, int32_t n, int64_t nnz, const int32_t* rp,
                              const int32_t* ci, NaScratch* s) {
    const int64_t stride = static_cast<int64_t>(gridDim.x) * kNaBlock;
    const int64_t t0 = static_cast<int64_t>(blockIdx.x) * kNaBlock + threadIdx.x;
    bool bad = false;
    if (t0 == 0) bad = rp[0] != 0 || static_cast<int64_t>(rp[m]) != nnz;
    for (int64_t r = t0; r < m; r += stride) bad = bad || rp[r] > rp[r + 1];
    for (int64_t k = t0; k < nnz; k += stride) {
        const int32_t c = ci[k];
        bad = bad || c < 0 || c >= n;
    }
    if (bad) atomicOr(&s->bad, 1);
}

__global__ void k_na_count(int32_t m, const int32_t* rp, const int32_t* ci, NaScratch* s) {
    if (s->bad) return;
    const int r = blockIdx.x * kNaBlock + threadIdx.x;
    if (r >= m) return;
    for (int k = rp[r]; k < rp[r + 1]; ++k) atomicAdd(&s->cursor[ci[k]], 1);
}

// Exclusive scan of the n column counts into rp (one CTA of 1024 threads,
// each owning a contiguous chunk); cursor becomes each column's start.
__global__ void __launch_bounds__(1024) k_na_scan(NaScratch* s, int32_t n) {
    if (s->bad) return;
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

__global__ void k_na_place(int32_t m, const int32_t* rp, const int32_t* ci, const double* v,
                           NaScratch* s) {
    if (s->bad) return;
    const int r = blockIdx.x * kNaBlock + threadIdx.x;
    if (r >= m) return;
    for (int k = rp[r]; k < rp[r + 1]; ++k) {
        const int pos = atomicAdd(&s->cursor[ci[k]], 1);
        s->ci[pos] = r;
        s->src[pos] = k;
        s->v[pos] = v[k];
    }
}

// Atomic placement leaves each column's entries in arbitrary order. A heap
// sort by the entries' positions in A restores the order of a stable sort by
// column: ascending rows, and duplicates of one (row, column) pair in the
// order A lists them -- the order in which pdhg_csr_spmv's A^T holds them.
__device__ void na_sift(int32_t* key, int32_t* row, double* val, int root, int len) {
    while (true) {
        int child = 2 * root + 1;
        if (child >= len) return;
        if (child + 1 < len && key[child + 1] > key[child]) ++child;
        if (key[root] >= key[child]) return;
        const int32_t tk = key[root];
        key[root] = key[child];
        key[child] = tk;
        const int32_t tr = row[root];
        row[root] = row[child];
        row[child] = tr;
        const double tv = val[root];
        val[root] = val[child];
        val[child] = tv;
        root = child;
    }
}

__global__ void k_na_sort(NaScratch* s, int32_t n) {
    if (s->bad) return;
    const int c = blockIdx.x * kNaBlock + threadIdx.x;
    if (c >= n) return;
    const int b = s->rp[c];
    int32_t* key = s->src + b;
    int32_t* row = s->ci + b;
    double* val = s->v + b;
    const int len = s->rp[c + 1] - b;
    for (int i = len / 2 - 1; i >= 0; --i) na_sift(key, row, val, i, len);
    for (int end = len - 1; end > 0; --end) {
        const int32_t tk = key[0];
        key[0] = key[end];
        key[end] = tk;
        const int32_t tr = row[0];
        row[0] = row[end];
        row[end] = tr;
        const double tv = val[0];
        val[0] = val[end];
        val[end] = tv;
        na_sift(key, row, val, 0, end);
    }
}

// y := alpha A x + beta y, one thread per row summing in the row's order
// (HostBackend::spmv, backend_host.cpp:415-423; beta == 0 overwrites), the
// arithmetic of the engine's exact kernel for rows of up to 32 entries and
// of its warp kernel, which adds in the same order, for longer ones.
__global__ void k_na_spmv(int32_t m, const int32_t* rp, const int32_t* ci, const double* v,
                          double alpha, const double* x, double beta, double* y,
                          const NaScratch* s) {
    const int r = blockIdx.x * kNaBlock + threadIdx.x;
    if (r >= m) return;
    if (s->bad) {
        y[r] = CUDART_NAN;
        return;
    }
    const double sum = ordered_dot(rp[r], rp[r + 1], ci, v, [x](int j) { return x[j]; }, 0.0);
    y[r] = (beta == 0.0) ? __dmul_rn(alpha, sum)
                         : __dadd_rn(__dmul_rn(alpha, sum), __dmul_rn(beta, y[r]));
}

// y := alpha A^T x + beta y on the A^T built in the scratch
// (HostBackend::spmv_transpose, backend_host.cpp:434-444): y_c starts at 0
// (beta == 0) or y_c beta, then adds val (alpha x_r) in ascending row order.
__global__ void k_na_spmvT(int32_t n, double alpha, const double* x, double beta, double* y,
                           const NaScratch* s) {
    const int c = blockIdx.x * kNaBlock + threadIdx.x;
    if (c >= n) return;
    if (s->bad) {
        y[c] = CUDART_NAN;
        return;
    }
    const double init = (beta == 0.0) ? 0.0 : __dmul_rn(y[c], beta);
    y[c] = ordered_dot(s->rp[c], s->rp[c + 1], s->ci, s->v,
                       [x, alpha](int r) { return __dmul_rn(alpha, x[r]); }, init);
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
    const int32_t nx = transpose ? m : n, ny = transpose ? n : m;
    if (m < 0 || n < 0 || nnz < 0 || nnz > std::numeric_limits<int32_t>::max() ||
        d_row_ptr == nullptr || (ny > 0 && d_y == nullptr) || (nx > 0 && d_x == nullptr) ||
        (nnz > 0 && (d_col_idx == nullptr || d_values == nullptr)))
        return PDHG_ERR_INVALID_ARGUMENT;
    if (transpose && (n > kNaMaxCols || nnz > kNaMaxNnz))
        return PDHG_ERR_INVALID_ARGUMENT;  // beyond the fixed scratch of the no-allocation path
    int device = 0;
    if (cudaGetDevice(&device) != cudaSuccess) return PDHG_ERR_BACKEND;
    NaScratch* sc = nullptr;
    const int rc = na_scratch(device, &sc);
    if (rc != PDHG_OK) return rc;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const int gn = ((transpose ? n : 0) + 1 + kNaBlock - 1) / kNaBlock;
    const int gm = (m + kNaBlock - 1) / kNaBlock;
    k_na_zero<<<gn, kNaBlock, 0, s>>>(sc, transpose ? n : 0);
    k_na_validate<<<na_grid(std::max<int64_t>(m, nnz)), kNaBlock, 0, s>>>(m, n, nnz, d_row_ptr,
                                                                          d_col_idx, sc);
    if (!transpose) {
        if (m > 0)
            k_na_spmv<<<gm, kNaBlock, 0, s>>>(m, d_row_ptr, d_col_idx, d_values, alpha, d_x, beta,
                                              d_y, sc);
        return cudaGetLastError() == cudaSuccess ? PDHG_OK : PDHG_ERR_BACKEND;
    }
    if (m > 0) k_na_count<<<gm, kNaBlock, 0, s>>>(m, d_row_ptr, d_col_idx, sc);
    k_na_scan<<<1, 1024, 0, s>>>(sc, n);
    if (m > 0) k_na_place<<<gm, kNaBlock, 0, s>>>(m, d_row_ptr, d_col_idx, d_values, sc);
    if (n > 0) {
        const int gc = (n + kNaBlock - 1) / kNaBlock;
        k_na_sort<<<gc, kNaBlock, 0, s>>>(sc, n);
        k_na_spmvT<<<gc, kNaBlock, 0, s>>>(n, alpha, d_x, beta, d_y, sc);
    }
    return cudaGetLastError() == cudaSuccess ? PDHG_OK : PDHG_ERR_BACKEND;
}
