// Fifth-generation tensor cores (tcgen05) for sm_100a, written as inline PTX: tensor-memory
// allocation, the BF16 x BF16 -> FP32 MMA with shared-memory operand descriptors, its completion
// through an mbarrier, and loads of the FP32 accumulator from tensor memory.
//
// Operand tiles live in shared memory in the canonical no-swizzle layout of 8 x 16-byte core
// matrices. A tile of R rows (the M or N side) by K columns (the reduction side) is stored
// K-chunk by K-chunk: element (r, k) at byte
//     ((k / 8) * (R / 8) + r / 8) * 128 + (r % 8) * 16 + (k % 8) * 2,
// so that one MMA step (16 columns of K) reads two K-chunks (R / 8 * 128 bytes apart, the
// leading byte offset) of R / 8 core matrices each (128 bytes apart, the stride byte offset).
// The same bytes read with rows as the reduction side and columns as the M or N side form the
// MN-major layout (core matrices 8 K-rows by 16 bytes of MN): stride byte offset R / 8 * 128
// between 8-column groups, leading byte offset 128 between 8-row groups. The weight gradients
// use that second reading, so no tile is transposed.
#pragma once

#include <cstdint>

namespace gsb {
namespace umma {

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// byte offset of element (r, k) in a K-chunked tile of R rows
__host__ __device__ constexpr uint32_t tile_offset(int R, int r, int k) {
    return (uint32_t)(((k >> 3) * (R >> 3) + (r >> 3)) * 128 + (r & 7) * 16 + (k & 7) * 2);
}

// Shared-memory matrix descriptor (sm_100): start address, leading and stride byte offsets
// (all in 16-byte units), version 1, no swizzle.
__device__ __forceinline__ uint64_t desc(uint32_t saddr, uint32_t lbo_bytes, uint32_t sbo_bytes) {
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo_bytes >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo_bytes >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// Descriptor of MMA step s (reduction columns 16 s .. 16 s + 15) of a tile with R rows:
// K-major (the rows are M or N) or MN-major (the rows are the reduction side, 8-column groups of
// the tile are M or N).
__device__ __forceinline__ uint64_t desc_kmajor(uint32_t base, int R, int s) {
    return desc(base + (uint32_t)(2 * s * (R >> 3) * 128), (uint32_t)((R >> 3) * 128), 128u);
}
__device__ __forceinline__ uint64_t desc_mnmajor(uint32_t base, int R, int s) {
    return desc(base + (uint32_t)(2 * s * 128), 128u, (uint32_t)((R >> 3) * 128));
}

// Instruction descriptor, kind::f16: BF16 operands, FP32 accumulator, M x N, each operand
// K-major (0) or MN-major (1).
__host__ __device__ constexpr uint32_t idesc_bf16(int M, int N, int a_mn, int b_mn) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)a_mn << 15) | ((uint32_t)b_mn << 16) |
           ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

// Tensor memory: one warp allocates `ncols` columns (a power of two >= 32) and writes the base
// address to shared memory; the same warp frees them.
__device__ __forceinline__ void tmem_alloc(uint32_t* dst_smem, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(dst_smem)),
                 "r"(ncols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
}
__device__ __forceinline__ void tmem_free(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols));
}

// D (+)= A B with descriptors; issued by one thread.
__device__ __forceinline__ void mma(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t idesc,
                                    bool accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
        "l"(a), "l"(b), "r"(idesc), "r"((uint32_t)accumulate));
}

// The mbarrier arrives when every MMA this thread issued before has completed.
__device__ __forceinline__ void commit(uint64_t* mbar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                     smem_u32(mbar))
                 : "memory");
}

__device__ __forceinline__ void mbar_init(uint64_t* mbar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(mbar)), "r"(count)
                 : "memory");
}

// Wait for the phase `parity` of the mbarrier to complete, at most `limit` polls; false when
// the limit ran out (the caller records the failure and stops using the tile).
__device__ __forceinline__ bool mbar_wait(uint64_t* mbar, uint32_t parity, uint32_t limit) {
    const uint32_t a = smem_u32(mbar);
    for (uint32_t i = 0; i < limit; ++i) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(a), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

__device__ __forceinline__ void fence_async_shared() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void fence_before_sync() {
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void fence_after_sync() {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

// 16 consecutive FP32 columns of this thread's lane (warp w reads lanes 32 w .. 32 w + 31; the
// address carries the warp's lane base in its upper half).
__device__ __forceinline__ void ld16(uint32_t taddr, float (&v)[16]) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, "
        "%11, %12, %13, %14, %15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
          "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]),
          "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ uint32_t lane_base(uint32_t tmem) {
    return tmem + ((uint32_t)((threadIdx.x >> 5) * 32) << 16);
}

}  // namespace umma
}  // namespace gsb
