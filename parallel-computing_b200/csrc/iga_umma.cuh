// 5th-generation tensor cores (tcgen05) for sm_100a: TMEM allocation, shared
// memory matrix descriptors, the TF32 MMA, completion through an mbarrier and
// accumulator loads. PTX forms and descriptor bit layouts follow the PTX ISA
// (tcgen05 family) and CUTLASS's cute/arch/mma_sm100_desc.hpp.
//
// Operands are K-major without swizzle: a tile of R rows x K values is stored
// as "core matrices" of 8 rows x 16 bytes (8 rows x 4 TF32 values, rows 16
// bytes apart); 8-row groups are SBO bytes apart, 16-byte K chunks LBO bytes
// apart. One MMA consumes K = 8 TF32 values (two chunks) per row.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "iga_device.cuh"

namespace iga {
namespace umma {

// Shared memory matrix descriptor (no swizzle, K-major), Blackwell version 1.
__device__ __forceinline__ uint64_t smem_desc(const void *smem, uint32_t lbo_bytes, uint32_t sbo_bytes)
{
    const uint32_t a = smem_u32(smem);
    uint64_t d = 0;
    d |= (uint64_t)((a >> 4) & 0x3FFFu);                  // start address, bits [0,14)
    d |= (uint64_t)((lbo_bytes >> 4) & 0x3FFFu) << 16;    // leading byte offset, bits [16,30)
    d |= (uint64_t)((sbo_bytes >> 4) & 0x3FFFu) << 32;    // stride byte offset, bits [32,46)
    d |= (uint64_t)1 << 46;                               // version (Blackwell), bits [46,48)
    return d;                                             // base offset 0, lbo mode 0, no swizzle
}

// Instruction descriptor of kind::tf32: FP32 accumulator, TF32 A and B, both
// K-major, no negation, M x N tile.
template <int M, int N>
__host__ __device__ constexpr uint32_t idesc_tf32()
{
    static_assert(M == 64 || M == 128, "M is 64 or 128");
    static_assert(N % 8 == 0 && N >= 8 && N <= 256, "N is a multiple of 8 in [8, 256]");
    return (1u << 4)                      // C format F32, bits [4,6)
           | (2u << 7)                    // A format TF32, bits [7,10)
           | (2u << 10)                   // B format TF32, bits [10,13)
           | ((uint32_t)(N >> 3) << 17)   // N >> 3, bits [17,23)
           | ((uint32_t)(M >> 4) << 24);  // M >> 4, bits [24,29)
}

// D[tmem] (+)= A[smem] x B[smem]^T; accumulate = 0 overwrites D. One thread issues.
__device__ __forceinline__ void mma_tf32(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                         uint32_t accumulate)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}"
        :
        : "r"(tmem_d), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
        : "memory");
}

// The mbarrier tracks completion of every tcgen05.mma this thread issued so far.
__device__ __forceinline__ void commit(uint64_t *bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}

// TMEM allocation by one whole warp; the address is written to *dst (shared).
__device__ __forceinline__ void alloc(uint32_t *dst, uint32_t ncols)
{
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(dst)), "r"(ncols)
                 : "memory");
}

__device__ __forceinline__ void relinquish() { asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory"); }

__device__ __forceinline__ void dealloc(uint32_t taddr, uint32_t ncols)
{
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

__device__ __forceinline__ void fence_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// 16 consecutive 32-bit columns of this warp's 32 TMEM lanes (lane i of the
// warp gets row 32 * (warp % 4) + i); taddr carries the lane in bits [16,32).
__device__ __forceinline__ void ld16(uint32_t taddr, float (&v)[16])
{
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
          "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

}  // namespace umma
}  // namespace iga
