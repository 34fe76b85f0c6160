// Fifth-generation tensor-core (tcgen05) building blocks for sm_100a, written as inline PTX: tensor-memory
// allocation, shared-memory matrix descriptors in the canonical K-major layout without swizzle, the BF16 MMA with
// FP32 accumulation in tensor memory, its completion barrier and the tensor-memory loads of the epilogue.
//
// Canonical K-major layout without swizzle (the one these descriptors describe): a matrix of R rows and K BF16
// columns is stored in "core matrices" of 8 rows x 16 bytes (8 BF16), each 128 contiguous bytes, row r of a core
// matrix at byte 16 r.  Core matrices adjacent along K are kLbo = 128 bytes apart; groups of 8 rows are
// (K / 8) * 128 bytes apart (the stride byte offset).  Element (r, k) therefore sits at byte
//     (r / 8) * (K / 8) * 128 + (k / 8) * 128 + (r % 8) * 16 + (k % 8) * 2,
// and one MMA step of K = 16 starts 256 bytes after the previous one.
#pragma once
#include <cstdint>

namespace kq {
namespace umma {

constexpr uint32_t kLbo = 128;

__device__ __forceinline__ uint32_t smem_u32(const void *p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// byte offset of element (r, k) of a K-major matrix with K columns (K a multiple of 16)
__host__ __device__ constexpr uint32_t kmajor_offset(int r, int k, int K)
{
    return (uint32_t)((r >> 3) * (K >> 3) * 128 + (k >> 3) * 128 + (r & 7) * 16 + (k & 7) * 2);
}

// shared-memory matrix descriptor: start address, leading byte offset (between K-adjacent core matrices), stride
// byte offset (between 8-row groups), descriptor version 1 (sm_100), no swizzle
__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr, uint32_t sbo)
{
    return (uint64_t)((saddr >> 4) & 0x3FFF) | ((uint64_t)((kLbo >> 4) & 0x3FFF) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFF) << 32) | (1ull << 46);
}

// shared-memory matrix descriptor with explicit offsets.  K-major: lbo = between K-adjacent core matrices, sbo =
// between M/N-adjacent ones.  MN-major (no swizzle): sbo = between M/N-adjacent core matrices (each 8 K-rows of
// 16 bytes = 8 M/N elements), lbo = between K-adjacent ones.
__device__ __forceinline__ uint64_t smem_desc2(uint32_t saddr, uint32_t lbo, uint32_t sbo)
{
    return (uint64_t)((saddr >> 4) & 0x3FFF) | ((uint64_t)((lbo >> 4) & 0x3FFF) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFF) << 32) | (1ull << 46);
}

// instruction descriptor of kind::f16: BF16 A and B, FP32 accumulator, M x N; a_mn / b_mn select the MN-major
// operand layout (default K-major)
__host__ __device__ constexpr uint32_t idesc_bf16_f32(int M, int N, bool a_mn = false, bool b_mn = false)
{
    return (1u << 4) | (1u << 7) | (1u << 10) | ((a_mn ? 1u : 0u) << 15) | ((b_mn ? 1u : 0u) << 16) |
           ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

// tensor-memory allocation of ncols columns (power of two >= 32) by one full warp; the base address is written to
// shared memory at slot
__device__ __forceinline__ void tmem_alloc(uint32_t *slot, uint32_t ncols)
{
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(slot)),
                 "r"(ncols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
}

__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols)
{
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols));
}

// D[tmem] (+)= A[smem] * B[smem]^T, issued by one thread
__device__ __forceinline__ void mma_bf16(uint32_t d_tmem, uint64_t a_desc, uint64_t b_desc, uint32_t idesc,
                                         uint32_t accumulate)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d_tmem),
        "l"(a_desc), "l"(b_desc), "r"(idesc), "r"(accumulate));
}

// arrive on the mbarrier once every MMA this thread issued before has completed
__device__ __forceinline__ void mma_commit(uint64_t *mbar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(mbar))
                 : "memory");
}

__device__ __forceinline__ void mbar_init(uint64_t *mbar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(mbar)), "r"(count) : "memory");
}

// bounded wait for phase `parity` of the mbarrier; false when the limit ran out
__device__ __forceinline__ bool mbar_wait(uint64_t *mbar, uint32_t parity, uint32_t limit)
{
    const uint32_t a = smem_u32(mbar);
    for (uint32_t it = 0; it < limit; ++it) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(done)
            : "r"(a), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

__device__ __forceinline__ void fence_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
// generic-proxy shared-memory writes made visible to the tensor cores' (async-proxy) reads
__device__ __forceinline__ void fence_smem_to_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// 16 consecutive FP32 columns of this warp's 32 tensor-memory lanes (thread t: lane 32 * (warp % 4) + t)
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float v[16])
{
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int j = 0; j < 16; ++j) v[j] = __uint_as_float(r[j]);
}

}  // namespace umma
}  // namespace kq
