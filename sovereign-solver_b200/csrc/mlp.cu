// mlp.cu -- the learned warm start's network on the tensor cores: a
// 2-hidden-layer ReLU MLP (n_in -> hidden -> hidden -> n_out) whose forward
// and backward passes are BF16 GEMMs with FP32 accumulation on tcgen05
// (k_gemm_tn), trained with Adam on FP32 master weights.
//
// One GEMM form covers every product: C[M x N] = A[M x K] * B[N x K]^T with
// both operands K-contiguous (row-major A and B), fused epilogue (bias, ReLU,
// a ReLU-derivative mask, FP32 and/or BF16 outputs). Products that need a
// transposed operand (the weight gradients dY^T H, the input gradients dY W)
// take a transposed copy made by k_transpose (the matrices are at most
// hidden x batch).
//
// Forward (batch B):  H1 = relu(X W1^T + b1), H2 = relu(H1 W2^T + b2),
//                     Y = H2 W3^T + b3.
// Loss:               L = sum (Y - T)^2 / (B n_out).
// Backward:           dY = 2 (Y - T) / (B n_out); dW3 = dY^T H2, db3 = sum_b dY;
//                     dZ2 = (dY W3) * [H2 > 0]; dW2 = dZ2^T H1; db2 = sum_b dZ2;
//                     dZ1 = (dZ2 W2) * [H1 > 0]; dW1 = dZ1^T X; db1 = sum_b dZ1.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <random>
#include <string>
#include <vector>

#include "../../include/pdhg_b200.h"
#include "tcgen05.cuh"

namespace pdhg {
namespace {

using bf16 = __nv_bfloat16;

constexpr int kGemmThreads = 128;
constexpr int kGemmBN = 128;                 // N per CTA (TMEM columns)
constexpr long long kSpinLimit = 1LL << 24;  // bounded mbarrier waits

struct GemmArgs {
    int M, N, K;
    const bf16* A;
    int lda;
    const bf16* B;
    int ldb;
    const float* bias;  // N, or null
    int relu;
    const bf16* mask;   // M x N: output * [mask > 0], or null
    int ldm;
    float* out32;       // M x N, or null
    int ld32;
    bf16* out16;        // M x N, or null
    int ld16;
    int* err;           // set when a bounded wait gives up
    int vec;            // 1: every row of bias / mask / outputs starts 16-byte aligned
};

// 16-byte asynchronous global -> shared copy (cp.async, no register staging);
// src_bytes = 0 writes zeros and reads nothing.
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem, int src_bytes) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(tc::smem_u32(smem)),
                 "l"(gmem), "r"(src_bytes)
                 : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

// C = A B^T on one 128 x kGemmBN tile: the K loop stages a 128 x 64 slice of
// A and a kGemmBN x 64 slice of B in shared memory (core-matrix layout, see
// tcgen05.cuh) with asynchronous 16-byte copies, all of a slice in flight at
// once, one thread issues the four 16-deep MMAs into the TMEM accumulator and
// commits them to an mbarrier that every thread waits on before the slices
// are overwritten. The epilogue reads the accumulator with tcgen05.ld, one
// TMEM lane (= output row) per thread.
__global__ void __launch_bounds__(kGemmThreads) k_gemm_tn(GemmArgs g) {
    __shared__ __align__(1024) bf16 sA[tc::kTileM * tc::kTileK];
    __shared__ __align__(1024) bf16 sB[kGemmBN * tc::kTileK];
    __shared__ __align__(8) uint64_t bar;
    __shared__ uint32_t tmem_base;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int m0 = blockIdx.x * tc::kTileM, n0 = blockIdx.y * kGemmBN;
    if (warp == 0) {
        tc::tmem_alloc(&tmem_base, kGemmBN);
        tc::tmem_relinquish();
    }
    if (tid == 0) {
        tc::mbar_init(&bar, 1);
        tc::fence_mbar_init();
    }
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = tmem_base;
    const uint32_t idesc = tc::instr_desc_bf16(kGemmBN);
    const uint32_t a_base = tc::smem_u32(sA), b_base = tc::smem_u32(sB);
    int round = 0;
    bool aborted = false;
    for (int k0 = 0; k0 < g.K; k0 += tc::kTileK, ++round) {
#pragma unroll
        for (int c = tid; c < tc::kTileM * (tc::kTileK / 8); c += kGemmThreads) {
            const int row = c >> 3, kc = (c & 7) * 8;
            const int gr = m0 + row, gk = k0 + kc;
            const bool in = gr < g.M && gk < g.K;
            cp_async16(sA + tc::tile_offset(row, kc),
                       in ? g.A + static_cast<size_t>(gr) * g.lda + gk : g.A, in ? 16 : 0);
        }
#pragma unroll
        for (int c = tid; c < kGemmBN * (tc::kTileK / 8); c += kGemmThreads) {
            const int row = c >> 3, kc = (c & 7) * 8;
            const int gr = n0 + row, gk = k0 + kc;
            const bool in = gr < g.N && gk < g.K;
            cp_async16(sB + tc::tile_offset(row, kc),
                       in ? g.B + static_cast<size_t>(gr) * g.ldb + gk : g.B, in ? 16 : 0);
        }
        cp_async_wait_all();
        tc::fence_proxy_async_smem();
        __syncthreads();
        if (tid == 0) {
            tc::fence_after_sync();
#pragma unroll
            for (int s = 0; s < tc::kTileK / 16; ++s) {
                const uint64_t ad = tc::smem_desc(a_base + s * 2 * tc::kChunkBytes);
                const uint64_t bd = tc::smem_desc(b_base + s * 2 * tc::kChunkBytes);
                tc::mma_bf16(tmem, ad, bd, idesc, (k0 > 0 || s > 0) ? 1u : 0u);
            }
            tc::mma_commit(&bar);
        }
        long long spins = 0;
        bool timed_out = false;
        while (!tc::mbar_try_wait(&bar, static_cast<uint32_t>(round & 1))) {
            if (++spins > kSpinLimit) {
                timed_out = true;
                break;
            }
        }
        if (__syncthreads_or(timed_out)) {
            aborted = true;
            break;
        }
    }
    tc::fence_after_sync();
    if (aborted) {
        if (tid == 0) atomicExch(g.err, 1);
        // give the MMAs in flight one more bounded chance to finish
        long long spins = 0;
        while (!tc::mbar_try_wait(&bar, static_cast<uint32_t>(round & 1)) && ++spins < kSpinLimit) {
        }
    } else {
        const int row = m0 + warp * 32 + lane;
        for (int cb = 0; cb < kGemmBN; cb += 32) {
            float v[32];
            tc::tmem_load32(tmem + (static_cast<uint32_t>(warp * 32) << 16) + cb, v);
            if (row >= g.M) continue;
            const int c0 = n0 + cb;
            if (g.vec && c0 + 32 <= g.N) {
                // a thread's 32 columns are contiguous in its row: 16-byte
                // loads of bias and mask, all issued before they are used,
                // and 16-byte stores
                if (g.bias != nullptr) {
                    const float4* b4 = reinterpret_cast<const float4*>(g.bias + c0);
#pragma unroll
                    for (int q = 0; q < 8; ++q) {
                        const float4 b = __ldg(b4 + q);
                        v[4 * q] += b.x;
                        v[4 * q + 1] += b.y;
                        v[4 * q + 2] += b.z;
                        v[4 * q + 3] += b.w;
                    }
                }
                if (g.relu)
#pragma unroll
                    for (int j = 0; j < 32; ++j) v[j] = fmaxf(v[j], 0.f);
                if (g.mask != nullptr) {
                    const uint4* m4 = reinterpret_cast<const uint4*>(g.mask + static_cast<size_t>(row) * g.ldm + c0);
                    uint4 mk[4];
#pragma unroll
                    for (int q = 0; q < 4; ++q) mk[q] = __ldg(m4 + q);
#pragma unroll
                    for (int q = 0; q < 4; ++q) {
                        const bf16* mb = reinterpret_cast<const bf16*>(&mk[q]);
#pragma unroll
                        for (int j = 0; j < 8; ++j)
                            if (!(__bfloat162float(mb[j]) > 0.f)) v[8 * q + j] = 0.f;
                    }
                }
                if (g.out32 != nullptr) {
                    float4* o4 = reinterpret_cast<float4*>(g.out32 + static_cast<size_t>(row) * g.ld32 + c0);
#pragma unroll
                    for (int q = 0; q < 8; ++q)
                        o4[q] = make_float4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
                }
                if (g.out16 != nullptr) {
                    uint4* o4 = reinterpret_cast<uint4*>(g.out16 + static_cast<size_t>(row) * g.ld16 + c0);
#pragma unroll
                    for (int q = 0; q < 4; ++q) {
                        uint4 w;
                        bf16* wb = reinterpret_cast<bf16*>(&w);
#pragma unroll
                        for (int j = 0; j < 8; ++j) wb[j] = __float2bfloat16_rn(v[8 * q + j]);
                        o4[q] = w;
                    }
                }
                continue;
            }
#pragma unroll
            for (int j = 0; j < 32; ++j) {
                const int col = c0 + j;
                if (col >= g.N) continue;
                float x = v[j];
                if (g.bias != nullptr) x += g.bias[col];
                if (g.relu) x = fmaxf(x, 0.f);
                if (g.mask != nullptr &&
                    !(__bfloat162float(g.mask[static_cast<size_t>(row) * g.ldm + col]) > 0.f))
                    x = 0.f;
                if (g.out32 != nullptr) g.out32[static_cast<size_t>(row) * g.ld32 + col] = x;
                if (g.out16 != nullptr)
                    g.out16[static_cast<size_t>(row) * g.ld16 + col] = __float2bfloat16_rn(x);
            }
        }
    }
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 0) tc::tmem_dealloc(tmem, kGemmBN);
}

// out[c * ldo + r] = in[r * ldi + c] for an R x C BF16 matrix (32 x 32 tiles).
__global__ void k_transpose(const bf16* in, int ldi, bf16* out, int ldo, int R, int C) {
    __shared__ bf16 t[32][33];
    const int r0 = blockIdx.y * 32, c0 = blockIdx.x * 32;
    for (int i = threadIdx.y; i < 32; i += 8) {
        const int r = r0 + i, c = c0 + threadIdx.x;
        if (r < R && c < C) t[i][threadIdx.x] = in[static_cast<size_t>(r) * ldi + c];
    }
    __syncthreads();
    for (int i = threadIdx.y; i < 32; i += 8) {
        const int c = c0 + i, r = r0 + threadIdx.x;
        if (r < R && c < C) out[static_cast<size_t>(c) * ldo + r] = t[threadIdx.x][i];
    }
}

__global__ void k_to_bf16(const float* in, bf16* out, int64_t n) {
    const int64_t t = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (t < n) out[t] = __float2bfloat16_rn(in[t]);
}

// Rows idx[0..B) of src (S x d, FP32) -> dst32 / dst16 (B x d).
__global__ void k_gather_rows(const float* src, int d, const int32_t* idx, int B, float* dst32,
                              bf16* dst16) {
    const int64_t t = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (t >= static_cast<int64_t>(B) * d) return;
    const int b = static_cast<int>(t / d), j = static_cast<int>(t % d);
    const float v = src[static_cast<int64_t>(idx[b]) * d + j];
    if (dst32 != nullptr) dst32[t] = v;
    if (dst16 != nullptr) dst16[t] = __float2bfloat16_rn(v);
}

// dY = 2 (Y - T) / (B n), FP32 and BF16; per-block partial losses.
__global__ void k_loss_grad(const float* Y, const float* T, int64_t count, float scale,
                            float* dY32, bf16* dY16, double* part) {
    __shared__ double sh[256];
    const int64_t t = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    double l = 0.0;
    if (t < count) {
        const float d = Y[t] - T[t];
        const float gv = 2.f * d * scale;
        dY32[t] = gv;
        dY16[t] = __float2bfloat16_rn(gv);
        l = static_cast<double>(d) * d * scale;
    }
    sh[threadIdx.x] = l;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) sh[threadIdx.x] += sh[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) part[blockIdx.x] = sh[0];
}

__global__ void k_sum_parts(const double* part, int n, double* out) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double s = 0.0;
    for (int i = 0; i < n; ++i) s += part[i];
    *out = s;
}

// db[j] = sum_b dZ[b, j] (fixed order per column).
__global__ void k_colsum(const float* dZ, int B, int N, float* db) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= N) return;
    float s = 0.f;
    for (int b = 0; b < B; ++b) s += dZ[static_cast<size_t>(b) * N + j];
    db[j] = s;
}

// Adam (bias-corrected) on FP32 master weights; refreshes the BF16 copy.
__global__ void k_adam(float* w, const float* g, float* m, float* v, bf16* w16, int64_t n,
                       float lr, float b1, float b2, float eps, float c1, float c2) {
    const int64_t t = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (t >= n) return;
    const float gt = g[t];
    const float mt = b1 * m[t] + (1.f - b1) * gt;
    const float vt = b2 * v[t] + (1.f - b2) * gt * gt;
    m[t] = mt;
    v[t] = vt;
    const float wt = w[t] - lr * (mt / c1) / (sqrtf(vt / c2) + eps);
    w[t] = wt;
    if (w16 != nullptr) w16[t] = __float2bfloat16_rn(wt);
}

inline int blocks(int64_t n, int t) { return static_cast<int>((n + t - 1) / t); }

// Host checks of the GEMM's layout contract, then the launch.
int gemm(const GemmArgs& g, cudaStream_t s) {
    if (g.M < 1 || g.N < 1 || g.K < 8 || g.K % 8 != 0 || g.lda % 8 != 0 || g.ldb % 8 != 0 ||
        (reinterpret_cast<uintptr_t>(g.A) & 15u) || (reinterpret_cast<uintptr_t>(g.B) & 15u))
        return PDHG_ERR_INVALID_ARGUMENT;
    const dim3 grid((g.M + tc::kTileM - 1) / tc::kTileM, (g.N + kGemmBN - 1) / kGemmBN);
    GemmArgs a = g;
    auto al16 = [](const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; };
    a.vec = al16(g.bias) && (g.mask == nullptr || (al16(g.mask) && g.ldm % 8 == 0)) &&
            (g.out32 == nullptr || (al16(g.out32) && g.ld32 % 4 == 0)) &&
            (g.out16 == nullptr || (al16(g.out16) && g.ld16 % 8 == 0)) ? 1 : 0;
    k_gemm_tn<<<grid, kGemmThreads, 0, s>>>(a);
    return cudaGetLastError() == cudaSuccess ? PDHG_OK : PDHG_ERR_BACKEND;
}

void transpose(const bf16* in, int ldi, bf16* out, int ldo, int R, int C, cudaStream_t s) {
    const dim3 grid((C + 31) / 32, (R + 31) / 32);
    k_transpose<<<grid, dim3(32, 8), 0, s>>>(in, ldi, out, ldo, R, C);
}

template <class T>
struct Dev {
    T* p = nullptr;
    size_t n = 0;
    Dev() = default;
    Dev(const Dev&) = delete;
    Dev& operator=(const Dev&) = delete;
    ~Dev() {
        if (p != nullptr) cudaFree(p);
    }
    cudaError_t alloc(size_t count) {
        if (p != nullptr) cudaFree(p);
        p = nullptr;
        n = count;
        return count ? cudaMalloc(reinterpret_cast<void**>(&p), sizeof(T) * count) : cudaSuccess;
    }
};

}  // namespace

struct Mlp {
    int device = 0;
    int n_in = 0, hidden = 0, n_out = 0, max_batch = 0;
    cudaStream_t stream = nullptr;
    std::string err;
    // parameters, one FP32 block [W1 b1 W2 b2 W3 b3] and its gradient / Adam moments
    int64_t off[6] = {}, cnt[6] = {}, total = 0;
    Dev<float> w, g, m, v;
    Dev<bf16> w16, w2t, w3t;  // BF16 weights, transposed W2 and W3 (for dX products)
    long long adam_t = 0;
    // activations (max_batch rows)
    Dev<bf16> x16, xt, h1, h1t, h2, h2t, dy16, dyt, dz2_16, dz2t, dz1_16, dz1t;
    Dev<float> t32, y32, dy32, dz2_32, dz1_32;
    Dev<double> part;
    Dev<int32_t> idx;
    Dev<int> errflag;
    // training set on the device
    Dev<float> xs, ts;

    ~Mlp() {
        if (stream != nullptr) cudaStreamDestroy(stream);
    }
    float* W(int i) { return w.p + off[2 * i]; }
    float* Bv(int i) { return w.p + off[2 * i + 1]; }
    bf16* W16(int i) { return w16.p + off[2 * i]; }
    float* gW(int i) { return g.p + off[2 * i]; }
    float* gB(int i) { return g.p + off[2 * i + 1]; }
};

namespace {

#define MCK(expr)                                                           \
    do {                                                                    \
        cudaError_t e_ = (expr);                                            \
        if (e_ != cudaSuccess) {                                            \
            h.err = std::string(#expr) + ": " + cudaGetErrorString(e_);     \
            return e_ == cudaErrorMemoryAllocation ? PDHG_ERR_OUT_OF_MEMORY \
                                                   : PDHG_ERR_BACKEND;      \
        }                                                                   \
    } while (0)

int check_err(Mlp& h) {
    int e = 0;
    MCK(cudaMemcpyAsync(&e, h.errflag.p, sizeof e, cudaMemcpyDeviceToHost, h.stream));
    MCK(cudaStreamSynchronize(h.stream));
    if (e != 0) {
        h.err = "tensor-core GEMM: an MMA did not complete within its wait limit";
        return PDHG_ERR_BACKEND;
    }
    return PDHG_OK;
}

GemmArgs args(int M, int N, int K, const bf16* A, int lda, const bf16* B, int ldb, int* err) {
    GemmArgs g{};
    g.M = M;
    g.N = N;
    g.K = K;
    g.A = A;
    g.lda = lda;
    g.B = B;
    g.ldb = ldb;
    g.err = err;
    return g;
}

// Refresh the BF16 weights and the transposed copies from the FP32 masters.
void refresh_weights(Mlp& h) {
    k_to_bf16<<<blocks(h.total, 256), 256, 0, h.stream>>>(h.w.p, h.w16.p, h.total);
    transpose(h.W16(1), h.hidden, h.w2t.p, h.hidden, h.hidden, h.hidden, h.stream);
    transpose(h.W16(2), h.hidden, h.w3t.p, h.n_out, h.n_out, h.hidden, h.stream);
}

int forward(Mlp& h, int B) {
    int rc;
    GemmArgs g = args(B, h.hidden, h.n_in, h.x16.p, h.n_in, h.W16(0), h.n_in, h.errflag.p);
    g.bias = h.Bv(0);
    g.relu = 1;
    g.out16 = h.h1.p;
    g.ld16 = h.hidden;
    if ((rc = gemm(g, h.stream)) != PDHG_OK) return rc;
    g = args(B, h.hidden, h.hidden, h.h1.p, h.hidden, h.W16(1), h.hidden, h.errflag.p);
    g.bias = h.Bv(1);
    g.relu = 1;
    g.out16 = h.h2.p;
    g.ld16 = h.hidden;
    if ((rc = gemm(g, h.stream)) != PDHG_OK) return rc;
    g = args(B, h.n_out, h.hidden, h.h2.p, h.hidden, h.W16(2), h.hidden, h.errflag.p);
    g.bias = h.Bv(2);
    g.out32 = h.y32.p;
    g.ld32 = h.n_out;
    return gemm(g, h.stream);
}

// Gradients into h.g for the batch already in x16 / t32; loss -> part[0] sum.
int backward(Mlp& h, int B) {
    int rc;
    const int64_t cnt = static_cast<int64_t>(B) * h.n_out;
    const int lb = blocks(cnt, 256);
    k_loss_grad<<<lb, 256, 0, h.stream>>>(h.y32.p, h.t32.p, cnt,
                                          1.f / static_cast<float>(cnt), h.dy32.p, h.dy16.p,
                                          h.part.p + 1);
    k_sum_parts<<<1, 32, 0, h.stream>>>(h.part.p + 1, lb, h.part.p);
    // layer 3
    transpose(h.dy16.p, h.n_out, h.dyt.p, B, B, h.n_out, h.stream);
    transpose(h.h2.p, h.hidden, h.h2t.p, B, B, h.hidden, h.stream);
    GemmArgs g = args(h.n_out, h.hidden, B, h.dyt.p, B, h.h2t.p, B, h.errflag.p);
    g.out32 = h.gW(2);
    g.ld32 = h.hidden;
    if ((rc = gemm(g, h.stream)) != PDHG_OK) return rc;
    k_colsum<<<blocks(h.n_out, 128), 128, 0, h.stream>>>(h.dy32.p, B, h.n_out, h.gB(2));
    g = args(B, h.hidden, h.n_out, h.dy16.p, h.n_out, h.w3t.p, h.n_out, h.errflag.p);
    g.mask = h.h2.p;
    g.ldm = h.hidden;
    g.out32 = h.dz2_32.p;
    g.ld32 = h.hidden;
    g.out16 = h.dz2_16.p;
    g.ld16 = h.hidden;
    if ((rc = gemm(g, h.stream)) != PDHG_OK) return rc;
    // layer 2
    transpose(h.dz2_16.p, h.hidden, h.dz2t.p, B, B, h.hidden, h.stream);
    transpose(h.h1.p, h.hidden, h.h1t.p, B, B, h.hidden, h.stream);
    g = args(h.hidden, h.hidden, B, h.dz2t.p, B, h.h1t.p, B, h.errflag.p);
    g.out32 = h.gW(1);
    g.ld32 = h.hidden;
    if ((rc = gemm(g, h.stream)) != PDHG_OK) return rc;
    k_colsum<<<blocks(h.hidden, 128), 128, 0, h.stream>>>(h.dz2_32.p, B, h.hidden, h.gB(1));
    g = args(B, h.hidden, h.hidden, h.dz2_16.p, h.hidden, h.w2t.p, h.hidden, h.errflag.p);
    g.mask = h.h1.p;
    g.ldm = h.hidden;
    g.out32 = h.dz1_32.p;
    g.ld32 = h.hidden;
    g.out16 = h.dz1_16.p;
    g.ld16 = h.hidden;
    if ((rc = gemm(g, h.stream)) != PDHG_OK) return rc;
    // layer 1
    transpose(h.dz1_16.p, h.hidden, h.dz1t.p, B, B, h.hidden, h.stream);
    transpose(h.x16.p, h.n_in, h.xt.p, B, B, h.n_in, h.stream);
    g = args(h.hidden, h.n_in, B, h.dz1t.p, B, h.xt.p, B, h.errflag.p);
    g.out32 = h.gW(0);
    g.ld32 = h.n_in;
    if ((rc = gemm(g, h.stream)) != PDHG_OK) return rc;
    k_colsum<<<blocks(h.hidden, 128), 128, 0, h.stream>>>(h.dz1_32.p, B, h.hidden, h.gB(0));
    return PDHG_OK;
}

int upload_batch(Mlp& h, int B, const float* x, const float* t) {
    std::vector<int32_t> id(static_cast<size_t>(B));
    for (int i = 0; i < B; ++i) id[i] = i;
    Dev<float> xs, ts;
    MCK(xs.alloc(static_cast<size_t>(B) * h.n_in));
    MCK(cudaMemcpyAsync(xs.p, x, sizeof(float) * B * h.n_in, cudaMemcpyHostToDevice, h.stream));
    MCK(cudaMemcpyAsync(h.idx.p, id.data(), sizeof(int32_t) * B, cudaMemcpyHostToDevice, h.stream));
    k_gather_rows<<<blocks(static_cast<int64_t>(B) * h.n_in, 256), 256, 0, h.stream>>>(
        xs.p, h.n_in, h.idx.p, B, nullptr, h.x16.p);
    if (t != nullptr) {
        MCK(ts.alloc(static_cast<size_t>(B) * h.n_out));
        MCK(cudaMemcpyAsync(ts.p, t, sizeof(float) * B * h.n_out, cudaMemcpyHostToDevice, h.stream));
        k_gather_rows<<<blocks(static_cast<int64_t>(B) * h.n_out, 256), 256, 0, h.stream>>>(
            ts.p, h.n_out, h.idx.p, B, h.t32.p, nullptr);
    }
    MCK(cudaStreamSynchronize(h.stream));  // xs / ts are freed on return
    return PDHG_OK;
}

bool batch_ok(const Mlp& h, int B) { return B >= 8 && B % 8 == 0 && B <= h.max_batch; }

}  // namespace
}  // namespace pdhg

struct pdhg_mlp {
    pdhg::Mlp h;
};

extern "C" {

int pdhg_mlp_create(int device, int n_in, int hidden, int n_out, int max_batch, pdhg_mlp** out) {
    using namespace pdhg;
    if (out == nullptr) return PDHG_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    if (n_in < 8 || n_in % 8 || hidden < 8 || hidden % 8 || n_out < 8 || n_out % 8 ||
        max_batch < 8 || max_batch % 8)
        return PDHG_ERR_INVALID_ARGUMENT;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev)
        return PDHG_ERR_UNSUPPORTED;
    std::unique_ptr<pdhg_mlp> p(new (std::nothrow) pdhg_mlp());
    if (!p) return PDHG_ERR_OUT_OF_MEMORY;
    Mlp& h = p->h;
    h.device = device;
    h.n_in = n_in;
    h.hidden = hidden;
    h.n_out = n_out;
    h.max_batch = max_batch;
    MCK(cudaSetDevice(device));
    MCK(cudaStreamCreateWithFlags(&h.stream, cudaStreamNonBlocking));
    const int64_t sizes[6] = {static_cast<int64_t>(hidden) * n_in, hidden,
                              static_cast<int64_t>(hidden) * hidden, hidden,
                              static_cast<int64_t>(n_out) * hidden, n_out};
    int64_t o = 0;
    for (int i = 0; i < 6; ++i) {
        h.off[i] = o;
        h.cnt[i] = sizes[i];
        o += (sizes[i] + 7) / 8 * 8;  // 16-byte aligned BF16 sub-arrays
    }
    h.total = o;
    const size_t B = static_cast<size_t>(max_batch), H = hidden;
    MCK(h.w.alloc(o));
    MCK(h.g.alloc(o));
    MCK(h.m.alloc(o));
    MCK(h.v.alloc(o));
    MCK(h.w16.alloc(o));
    MCK(h.w2t.alloc(H * H));
    MCK(h.w3t.alloc(H * n_out));
    MCK(h.x16.alloc(B * n_in));
    MCK(h.xt.alloc(B * n_in));
    MCK(h.h1.alloc(B * H));
    MCK(h.h1t.alloc(B * H));
    MCK(h.h2.alloc(B * H));
    MCK(h.h2t.alloc(B * H));
    MCK(h.dy16.alloc(B * n_out));
    MCK(h.dyt.alloc(B * n_out));
    MCK(h.dz2_16.alloc(B * H));
    MCK(h.dz2t.alloc(B * H));
    MCK(h.dz1_16.alloc(B * H));
    MCK(h.dz1t.alloc(B * H));
    MCK(h.t32.alloc(B * n_out));
    MCK(h.y32.alloc(B * n_out));
    MCK(h.dy32.alloc(B * n_out));
    MCK(h.dz2_32.alloc(B * H));
    MCK(h.dz1_32.alloc(B * H));
    MCK(h.part.alloc(B * n_out / 256 + 4));
    MCK(h.idx.alloc(B));
    MCK(h.errflag.alloc(1));
    MCK(cudaMemsetAsync(h.w.p, 0, sizeof(float) * o, h.stream));
    MCK(cudaMemsetAsync(h.m.p, 0, sizeof(float) * o, h.stream));
    MCK(cudaMemsetAsync(h.v.p, 0, sizeof(float) * o, h.stream));
    MCK(cudaMemsetAsync(h.errflag.p, 0, sizeof(int), h.stream));
    MCK(cudaStreamSynchronize(h.stream));
    *out = p.release();
    return PDHG_OK;
}

int pdhg_mlp_destroy(pdhg_mlp* p) {
    if (p == nullptr) return PDHG_ERR_INVALID_ARGUMENT;
    cudaSetDevice(p->h.device);
    if (p->h.stream != nullptr) cudaStreamSynchronize(p->h.stream);
    delete p;
    return PDHG_OK;
}

const char* pdhg_mlp_last_error(const pdhg_mlp* p) {
    return p == nullptr ? "null network" : p->h.err.c_str();
}

int64_t pdhg_mlp_param_count(const pdhg_mlp* p) {
    if (p == nullptr) return -1;
    int64_t s = 0;
    for (int i = 0; i < 6; ++i) s += p->h.cnt[i];
    return s;
}

// params: [W1 (hidden x n_in), b1, W2 (hidden x hidden), b2, W3 (n_out x hidden), b3]
int pdhg_mlp_set_params(pdhg_mlp* p, const float* params) {
    using namespace pdhg;
    if (p == nullptr || params == nullptr) return PDHG_ERR_INVALID_ARGUMENT;
    Mlp& h = p->h;
    MCK(cudaSetDevice(h.device));
    int64_t src = 0;
    for (int i = 0; i < 6; ++i) {
        MCK(cudaMemcpyAsync(h.w.p + h.off[i], params + src, sizeof(float) * h.cnt[i],
                            cudaMemcpyHostToDevice, h.stream));
        src += h.cnt[i];
    }
    MCK(cudaMemsetAsync(h.m.p, 0, sizeof(float) * h.total, h.stream));
    MCK(cudaMemsetAsync(h.v.p, 0, sizeof(float) * h.total, h.stream));
    h.adam_t = 0;
    refresh_weights(h);
    MCK(cudaStreamSynchronize(h.stream));
    return PDHG_OK;
}

int pdhg_mlp_get_params(pdhg_mlp* p, float* params) {
    using namespace pdhg;
    if (p == nullptr || params == nullptr) return PDHG_ERR_INVALID_ARGUMENT;
    Mlp& h = p->h;
    MCK(cudaSetDevice(h.device));
    int64_t dst = 0;
    for (int i = 0; i < 6; ++i) {
        MCK(cudaMemcpyAsync(params + dst, h.w.p + h.off[i], sizeof(float) * h.cnt[i],
                            cudaMemcpyDeviceToHost, h.stream));
        dst += h.cnt[i];
    }
    MCK(cudaStreamSynchronize(h.stream));
    return PDHG_OK;
}

int pdhg_mlp_forward(pdhg_mlp* p, int batch, const float* x, float* y) {
    using namespace pdhg;
    if (p == nullptr || x == nullptr || y == nullptr || !batch_ok(p->h, batch))
        return PDHG_ERR_INVALID_ARGUMENT;
    Mlp& h = p->h;
    MCK(cudaSetDevice(h.device));
    int rc = upload_batch(h, batch, x, nullptr);
    if (rc != PDHG_OK) return rc;
    if ((rc = forward(h, batch)) != PDHG_OK) return rc;
    MCK(cudaMemcpyAsync(y, h.y32.p, sizeof(float) * batch * h.n_out, cudaMemcpyDeviceToHost,
                        h.stream));
    return check_err(h);
}

int pdhg_mlp_gradients(pdhg_mlp* p, int batch, const float* x, const float* t, float* grads,
                       float* loss) {
    using namespace pdhg;
    if (p == nullptr || x == nullptr || t == nullptr || grads == nullptr ||
        !batch_ok(p->h, batch))
        return PDHG_ERR_INVALID_ARGUMENT;
    Mlp& h = p->h;
    MCK(cudaSetDevice(h.device));
    int rc = upload_batch(h, batch, x, t);
    if (rc != PDHG_OK) return rc;
    if ((rc = forward(h, batch)) != PDHG_OK) return rc;
    if ((rc = backward(h, batch)) != PDHG_OK) return rc;
    int64_t dst = 0;
    for (int i = 0; i < 6; ++i) {
        MCK(cudaMemcpyAsync(grads + dst, h.g.p + h.off[i], sizeof(float) * h.cnt[i],
                            cudaMemcpyDeviceToHost, h.stream));
        dst += h.cnt[i];
    }
    double l = 0.0;
    MCK(cudaMemcpyAsync(&l, h.part.p, sizeof l, cudaMemcpyDeviceToHost, h.stream));
    rc = check_err(h);
    if (loss != nullptr) *loss = static_cast<float>(l);
    return rc;
}

// One Adam step with gradients from outside (parameter order, host FP32):
// the update of data-parallel training, where every replica applies the
// gradients all ranks have averaged. The step counter is the one
// pdhg_mlp_train advances, and the hyper-parameters are its own.
int pdhg_mlp_adam_step(pdhg_mlp* p, const float* grads, float lr) {
    using namespace pdhg;
    if (p == nullptr || grads == nullptr || !(lr > 0.f)) return PDHG_ERR_INVALID_ARGUMENT;
    Mlp& h = p->h;
    MCK(cudaSetDevice(h.device));
    int64_t src = 0;
    for (int i = 0; i < 6; ++i) {
        MCK(cudaMemcpyAsync(h.g.p + h.off[i], grads + src, sizeof(float) * h.cnt[i],
                            cudaMemcpyHostToDevice, h.stream));
        src += h.cnt[i];
    }
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    h.adam_t += 1;
    const float c1 = 1.f - std::pow(b1, static_cast<float>(h.adam_t));
    const float c2 = 1.f - std::pow(b2, static_cast<float>(h.adam_t));
    k_adam<<<blocks(h.total, 256), 256, 0, h.stream>>>(h.w.p, h.g.p, h.m.p, h.v.p, h.w16.p,
                                                      h.total, lr, b1, b2, eps, c1, c2);
    transpose(h.W16(1), h.hidden, h.w2t.p, h.hidden, h.hidden, h.hidden, h.stream);
    transpose(h.W16(2), h.hidden, h.w3t.p, h.n_out, h.n_out, h.hidden, h.stream);
    MCK(cudaStreamSynchronize(h.stream));
    return check_err(h);
}

// Adam over `epochs` passes of shuffled mini-batches of the samples x (S x
// n_in) with targets t (S x n_out); the last incomplete batch of an epoch is
// dropped. epoch_loss (epochs entries, may be NULL) gets each epoch's mean
// batch loss.
int pdhg_mlp_train(pdhg_mlp* p, int64_t samples, const float* x, const float* t, int epochs,
                   int batch, float lr, uint64_t seed, float* epoch_loss) {
    using namespace pdhg;
    if (p == nullptr || x == nullptr || t == nullptr || epochs < 0 || samples < batch ||
        !batch_ok(p->h, batch) || !(lr > 0.f))
        return PDHG_ERR_INVALID_ARGUMENT;
    Mlp& h = p->h;
    MCK(cudaSetDevice(h.device));
    MCK(h.xs.alloc(static_cast<size_t>(samples) * h.n_in));
    MCK(h.ts.alloc(static_cast<size_t>(samples) * h.n_out));
    MCK(cudaMemcpyAsync(h.xs.p, x, sizeof(float) * samples * h.n_in, cudaMemcpyHostToDevice,
                        h.stream));
    MCK(cudaMemcpyAsync(h.ts.p, t, sizeof(float) * samples * h.n_out, cudaMemcpyHostToDevice,
                        h.stream));
    std::mt19937_64 rng(seed);
    std::vector<int32_t> perm(static_cast<size_t>(samples));
    const int steps = static_cast<int>(samples / batch);
    Dev<int32_t> perm_d;
    MCK(perm_d.alloc(static_cast<size_t>(samples)));
    std::vector<double> losses(static_cast<size_t>(steps));
    Dev<double> lsum;
    MCK(lsum.alloc(static_cast<size_t>(steps) + 1));
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    for (int ep = 0; ep < epochs; ++ep) {
        for (int64_t i = 0; i < samples; ++i) perm[i] = static_cast<int32_t>(i);
        std::shuffle(perm.begin(), perm.end(), rng);
        MCK(cudaMemcpyAsync(perm_d.p, perm.data(), sizeof(int32_t) * samples,
                            cudaMemcpyHostToDevice, h.stream));
        for (int sI = 0; sI < steps; ++sI) {
            const int32_t* idx = perm_d.p + static_cast<int64_t>(sI) * batch;
            k_gather_rows<<<blocks(static_cast<int64_t>(batch) * h.n_in, 256), 256, 0, h.stream>>>(
                h.xs.p, h.n_in, idx, batch, nullptr, h.x16.p);
            k_gather_rows<<<blocks(static_cast<int64_t>(batch) * h.n_out, 256), 256, 0, h.stream>>>(
                h.ts.p, h.n_out, idx, batch, h.t32.p, nullptr);
            int rc = forward(h, batch);
            if (rc == PDHG_OK) rc = backward(h, batch);
            if (rc != PDHG_OK) return rc;
            MCK(cudaMemcpyAsync(lsum.p + sI, h.part.p, sizeof(double), cudaMemcpyDeviceToDevice,
                                h.stream));
            h.adam_t += 1;
            const float c1 = 1.f - std::pow(b1, static_cast<float>(h.adam_t));
            const float c2 = 1.f - std::pow(b2, static_cast<float>(h.adam_t));
            k_adam<<<blocks(h.total, 256), 256, 0, h.stream>>>(h.w.p, h.g.p, h.m.p, h.v.p, h.w16.p,
                                                              h.total, lr, b1, b2, eps, c1, c2);
            transpose(h.W16(1), h.hidden, h.w2t.p, h.hidden, h.hidden, h.hidden, h.stream);
            transpose(h.W16(2), h.hidden, h.w3t.p, h.n_out, h.n_out, h.hidden, h.stream);
        }
        MCK(cudaMemcpyAsync(losses.data(), lsum.p, sizeof(double) * steps, cudaMemcpyDeviceToHost,
                            h.stream));
        MCK(cudaStreamSynchronize(h.stream));
        if (epoch_loss != nullptr) {
            double s = 0.0;
            for (double l : losses) s += l;
            epoch_loss[ep] = static_cast<float>(s / steps);
        }
    }
    return check_err(h);
}

// The tensor-core GEMM on its own (test entry): C = A B^T (+ bias, ReLU) with
// A (m x k) and B (n x k) given in FP32 on the host and rounded to BF16, FP32
// accumulation, C (m x n) FP32 on the host. k must be a multiple of 8.
int pdhg_gemm_bf16(int device, int m, int n, int k, const float* a, const float* b,
                   const float* bias, int relu, float* c) {
    using namespace pdhg;
    if (m < 1 || n < 1 || k < 8 || k % 8 || a == nullptr || b == nullptr || c == nullptr)
        return PDHG_ERR_INVALID_ARGUMENT;
    if (cudaSetDevice(device) != cudaSuccess) return PDHG_ERR_UNSUPPORTED;
    Dev<float> a32, b32, c32, bias32;
    Dev<bf16> a16, b16;
    Dev<int> err;
    const size_t na = static_cast<size_t>(m) * k, nb = static_cast<size_t>(n) * k;
    if (a32.alloc(na) || b32.alloc(nb) || c32.alloc(static_cast<size_t>(m) * n) ||
        a16.alloc(na) || b16.alloc(nb) || err.alloc(1) || (bias && bias32.alloc(n)))
        return PDHG_ERR_OUT_OF_MEMORY;
    cudaMemcpy(a32.p, a, sizeof(float) * na, cudaMemcpyHostToDevice);
    cudaMemcpy(b32.p, b, sizeof(float) * nb, cudaMemcpyHostToDevice);
    if (bias) cudaMemcpy(bias32.p, bias, sizeof(float) * n, cudaMemcpyHostToDevice);
    cudaMemset(err.p, 0, sizeof(int));
    k_to_bf16<<<blocks(na, 256), 256>>>(a32.p, a16.p, na);
    k_to_bf16<<<blocks(nb, 256), 256>>>(b32.p, b16.p, nb);
    GemmArgs g = args(m, n, k, a16.p, k, b16.p, k, err.p);
    g.bias = bias ? bias32.p : nullptr;
    g.relu = relu;
    g.out32 = c32.p;
    g.ld32 = n;
    int rc = gemm(g, nullptr);
    if (rc != PDHG_OK) return rc;
    int e = 0;
    if (cudaMemcpy(&e, err.p, sizeof e, cudaMemcpyDeviceToHost) != cudaSuccess) return PDHG_ERR_BACKEND;
    if (e != 0) return PDHG_ERR_BACKEND;
    if (cudaMemcpy(c, c32.p, sizeof(float) * m * n, cudaMemcpyDeviceToHost) != cudaSuccess)
        return PDHG_ERR_BACKEND;
    return PDHG_OK;
}

}  // extern "C"
