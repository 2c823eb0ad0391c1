// tcgen05.cuh -- thin wrappers over the Blackwell (sm_100a) tensor-core
// instructions the warm-start network's GEMM uses: TMEM allocation, the
// tcgen05.mma issue (kind::f16, BF16 operands from shared memory, FP32
// accumulator in TMEM), commit to an mbarrier, and the TMEM -> register load.
//
// Shared-memory operand layout (both operands K-major, no swizzle): a tile of
// R rows x 64 K-elements of BF16 is stored as 8 x 8 "core matrices" (8 rows x
// 16 bytes each, 128 contiguous bytes), core matrix (row group g, K chunk j)
// at byte (g * 8 + j) * 128, row r of the core matrix at r * 16. One MMA
// consumes 16 K-elements = two K chunks: its descriptor starts at chunk 2s,
// the leading byte offset (between the two K chunks) is 128 B and the stride
// byte offset (between 8-row groups) is 8 * 128 = 1024 B.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace pdhg {
namespace tc {

constexpr int kTileM = 128;   // rows of A per CTA (one TMEM lane per row)
constexpr int kTileK = 64;    // K-elements staged per round
constexpr int kChunkBytes = 128;                       // one core matrix
constexpr int kGroupBytes = (kTileK / 8) * kChunkBytes;  // one 8-row group: 1024 B

// Element offset (in BF16 elements) of (row, k) inside a staged tile.
__host__ __device__ constexpr int tile_offset(int row, int k) {
    return ((row >> 3) * (kTileK / 8) + (k >> 3)) * 64 + (row & 7) * 8 + (k & 7);
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Shared-memory matrix descriptor: start address, LBO, SBO (all >> 4),
// descriptor version 1 (sm_100), no swizzle.
__host__ __device__ constexpr uint64_t smem_desc(uint32_t smem_addr) {
    return static_cast<uint64_t>((smem_addr >> 4) & 0x3FFFu) |
           (static_cast<uint64_t>(kChunkBytes >> 4) << 16) |
           (static_cast<uint64_t>(kGroupBytes >> 4) << 32) | (uint64_t{1} << 46);
}

// Instruction descriptor: BF16 x BF16 -> FP32, both K-major, M = 128, N = n.
__host__ __device__ constexpr uint32_t instr_desc_bf16(int n) {
    return (1u << 4) |                              // D format: F32
           (1u << 7) | (1u << 10) |                 // A, B format: BF16
           (static_cast<uint32_t>(n >> 3) << 17) |  // N / 8
           (static_cast<uint32_t>(kTileM >> 4) << 24);  // M / 16
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
                 : "memory");
}

__device__ __forceinline__ void fence_mbar_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Makes generic-proxy shared-memory writes visible to the tensor cores.
__device__ __forceinline__ void fence_proxy_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// Whole warp: allocate `ncols` TMEM columns (power of two >= 32); the base
// address is written to *dst (shared memory).
__device__ __forceinline__ void tmem_alloc(uint32_t* dst, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(dst)),
                 "r"(ncols)
                 : "memory");
}

__device__ __forceinline__ void tmem_relinquish() {
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols)
                 : "memory");
}

// D[tmem] (+)= A[smem] * B[smem]^T, issued by one thread.
__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc,
                                         uint32_t idesc, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %5, %5, %5}, p;\n\t}" ::"r"(
            tmem_d),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(0u)
        : "memory");
}

// The mbarrier gets one arrival when every MMA this thread issued so far is done.
__device__ __forceinline__ void mma_commit(uint64_t* bar) {
    asm volatile(
        "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
            smem_u32(bar))
        : "memory");
}

__device__ __forceinline__ void fence_after_sync() {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

__device__ __forceinline__ void fence_before_sync() {
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}

// 32 consecutive FP32 columns of this thread's TMEM lane.
__device__ __forceinline__ void tmem_load32(uint32_t taddr, float (&v)[32]) {
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
        "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
        "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, "
        "[%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
          "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]),
          "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]),
          "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
          "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]),
          "=r"(r[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

}  // namespace tc
}  // namespace pdhg
