// Fifth-generation tensor-core primitives (tcgen05, sm_100a) in inline PTX:
// shared-memory matrix descriptors, the instruction descriptor of a BF16 x
// BF16 -> FP32 MMA, tensor-memory allocation, MMA issue and completion,
// tensor-memory loads, and bulk global -> shared copies on an mbarrier.
//
// Operand layout used with these descriptors (K-major, no swizzle): the matrix
// is cut into "core matrices" of 8 rows x 16 bytes (8 BF16 along K), each
// stored as 128 contiguous bytes (row r at byte 16 r).  Core matrix (row group
// g, K chunk c) of a `rows`-row operand sits at byte c * (rows * 16) + g * 128,
// so the K-chunk stride ("leading byte offset") is rows * 16 and the row-group
// stride ("stride byte offset") is 128.  One MMA instruction of K = 16 reads
// two K chunks from its start address.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace tsm {
namespace umma {

// Byte offset of element (row, k) in the layout above.
__device__ __forceinline__ uint32_t core_offset(int row, int k, int rows) {
    return (uint32_t)((k >> 3) * (rows * 16) + (row >> 3) * 128 + (row & 7) * 16 + (k & 7) * 2);
}

// Shared-memory matrix descriptor (sm_100 format): start address, leading and
// stride byte offsets in 16-byte units (14 bits each), version 1 (bits 46-47),
// base offset 0, layout type 0 = no swizzle (bits 61-63).
__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr, uint32_t lbo_bytes, uint32_t sbo_bytes) {
    uint64_t d = (uint64_t)((saddr >> 4) & 0x3FFFu);
    d |= (uint64_t)((lbo_bytes >> 4) & 0x3FFFu) << 16;
    d |= (uint64_t)((sbo_bytes >> 4) & 0x3FFFu) << 32;
    d |= (uint64_t)1 << 46;
    return d;
}

// Instruction descriptor of kind::f16 with FP16 A and B (both K-major) and an
// FP32 accumulator: the BF16 form below with A and B format 0 (F16).
__host__ __device__ constexpr uint32_t idesc_f16_f32(int m, int n) {
    return (1u << 4) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(m >> 4) << 24);
}

// Instruction descriptor of kind::f16 with BF16 A and B (both K-major) and an
// FP32 accumulator: D format bits 4-5 = 1 (F32), A format bits 7-9 = 1 (BF16),
// B format bits 10-12 = 1 (BF16), N / 8 in bits 17-22, M / 16 in bits 24-28.
__host__ __device__ constexpr uint32_t idesc_bf16_f32(int m, int n) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(m >> 4) << 24);
}

// D[tmem] (+)= A[smem] * B[smem]^T, issued by one thread.  accumulate = 0
// overwrites D.
__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                         uint32_t accumulate) {
    const uint32_t mask0 = 0, mask1 = 0, mask2 = 0, mask3 = 0;  // no output lane disabled
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n"
        :
        : "r"(tmem_d), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(mask0), "r"(mask1), "r"(mask2),
          "r"(mask3));
}

// The mbarrier at bar_saddr receives one arrival when every MMA this thread
// issued so far has completed.
__device__ __forceinline__ void commit(uint32_t bar_saddr) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar_saddr)
                 : "memory");
}

__device__ __forceinline__ void fence_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
// Makes this thread's generic shared-memory writes visible to the tensor cores.
__device__ __forceinline__ void fence_smem_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void mbar_init(uint32_t bar_saddr, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar_saddr), "r"(count) : "memory");
}

// Waits for the mbarrier phase with the given parity to complete, for at
// most max_cycles SM clocks.  Returns false if it gave up.
__device__ __forceinline__ bool mbar_wait(uint32_t bar_saddr, uint32_t parity, long long max_cycles) {
    const long long t0 = clock64();
    for (;;) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred P;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 P, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, P;\n\t}\n"
            : "=r"(done)
            : "r"(bar_saddr), "r"(parity)
            : "memory");
        if (done) return true;
        if (clock64() - t0 > max_cycles) return false;
    }
}

// One plain arrival on the mbarrier.
__device__ __forceinline__ void mbar_arrive(uint32_t bar_saddr) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar_saddr) : "memory");
}

// Arrival on the mbarrier that also expects `bytes` of asynchronous copies
// to land in the current phase.
__device__ __forceinline__ void mbar_arrive_expect_tx(uint32_t bar_saddr, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%1], %0;" ::"r"(bytes), "r"(bar_saddr) : "memory");
}

// Bulk copy of `bytes` (a multiple of 16, both addresses 16-byte aligned)
// from this GPU's global memory into shared memory, completing on the
// mbarrier's transaction count (no multicast).
__device__ __forceinline__ void bulk_load(uint32_t dst_saddr, const void* src, uint32_t bytes, uint32_t bar_saddr) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     dst_saddr),
                 "l"(src), "r"(bytes), "r"(bar_saddr)
                 : "memory");
}

// Tensor-memory allocation by one whole warp: ncols columns (a power of two
// >= 32); the address is written to shared memory at slot_saddr.
__device__ __forceinline__ void tmem_alloc(uint32_t slot_saddr, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(slot_saddr), "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

// 16 consecutive 32-bit columns of this thread's tensor-memory lane (the
// warp reads lanes 32 * (warp % 4) .. +31; taddr carries that lane base in
// bits 16-31).  The registers hold the values only after wait_ld(r): the
// wait takes them as operands, so no use can be scheduled before it.
__device__ __forceinline__ void ld16(uint32_t taddr, uint32_t (&r)[16]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
          "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
}

// Waits for this thread's tensor-memory loads; r (one load's registers) is
// tied to the wait.  Call it once per loaded array (the later calls return at
// once) so that every array is ordered after the wait.
__device__ __forceinline__ void wait_ld(uint32_t (&r)[16]) {
    asm volatile("tcgen05.wait::ld.sync.aligned;"
                 : "+r"(r[0]), "+r"(r[1]), "+r"(r[2]), "+r"(r[3]), "+r"(r[4]), "+r"(r[5]), "+r"(r[6]), "+r"(r[7]),
                   "+r"(r[8]), "+r"(r[9]), "+r"(r[10]), "+r"(r[11]), "+r"(r[12]), "+r"(r[13]), "+r"(r[14]),
                   "+r"(r[15])
                 :
                 : "memory");
}

}  // namespace umma
}  // namespace tsm
