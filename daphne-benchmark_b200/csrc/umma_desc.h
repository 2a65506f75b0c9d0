// Encoders of the two descriptors a tcgen05.mma of kind::f16 takes (the
// field positions are those of the PTX ISA's shared-memory matrix descriptor
// and instruction descriptor; tests/test_umma_desc.py checks these encoders
// bit for bit against CUTLASS's CuTe implementation on the shapes used here).
#pragma once
#include <stdint.h>

namespace umma {

// Shared-memory matrix descriptor, no swizzle ("interleaved" core matrices of
// 8 rows x 16 bytes), K-major:
//   bits  0-13  start address >> 4
//   bits 16-29  leading byte offset >> 4 (next 8 K-elements)
//   bits 32-45  stride byte offset >> 4 (next 8 rows)
//   bits 46-47  version (1 on this architecture)
//   bits 49-51  base offset (0), bit 52 leading-offset mode (0)
//   bits 61-63  layout (0 = no swizzle)
__host__ __device__ inline uint64_t smem_desc_kmajor_interleaved(uint32_t smem_addr, uint32_t lbo_bytes,
                                                                  uint32_t sbo_bytes) {
    uint64_t d = 0;
    d |= (uint64_t)((smem_addr >> 4) & 0x3fffu);
    d |= (uint64_t)((lbo_bytes >> 4) & 0x3fffu) << 16;
    d |= (uint64_t)((sbo_bytes >> 4) & 0x3fffu) << 32;
    d |= (uint64_t)1u << 46;
    return d;
}

// Instruction descriptor for BF16 x BF16 -> FP32, both operands K-major:
//   bits 4-5 D format (1 = F32), 7-9 A format (1 = BF16), 10-12 B format
//   (1 = BF16), 13/14 negate A/B (0), 15/16 A/B major (0 = K), 17-22 N >> 3,
//   24-28 M >> 4.
__host__ __device__ inline uint32_t instr_desc_bf16_f32(int M, int N) {
    uint32_t d = 0;
    d |= 1u << 4;
    d |= 1u << 7;
    d |= 1u << 10;
    d |= ((uint32_t)(N >> 3) & 0x3fu) << 17;
    d |= ((uint32_t)(M >> 4) & 0x1fu) << 24;
    return d;
}

}  // namespace umma
