// Descriptors of the 5th-generation tensor-core MMA (tcgen05.mma), as the PTX
// ISA defines them for sm_100:
//
// * shared-memory matrix descriptor (64 bits): the operand tile's start
//   address, leading and stride byte offsets (each in 16-byte units, 14 bits
//   at bits 0, 16 and 32), the descriptor version (1 for sm_100, bits 46-47),
//   the matrix base offset (bits 49-51, 0 here: tiles are aligned to their
//   swizzle pattern), the leading-offset mode (bit 52, 0: relative) and the
//   swizzle mode (bits 61-63);
// * instruction descriptor of kind::f16 (32 bits): accumulator format (bits
//   4-5, 1 = F32), A and B formats (bits 7-9 and 10-12, 1 = BF16), A and B
//   majorness (bits 15 and 16, 0 = K-major, 1 = MN-major), N >> 3 (bits 17-22)
//   and M >> 4 (bits 24-28).
//
// tests/test_umma_desc.py checks these encodings against CuTe's bitfield
// definitions of the same descriptors (cute/arch/mma_sm100_desc.hpp) where a
// CUTLASS tree is available; the build itself needs none.
#ifndef GG_UMMA_DESC_CUH
#define GG_UMMA_DESC_CUH

#include <cstdint>

namespace gg {

// Swizzle modes of the shared-memory descriptor (bits 61-63).
enum class UmmaSwizzle : uint64_t { kNone = 0, k128B = 2, k64B = 4, k32B = 6 };

__host__ __device__ constexpr uint64_t umma_smem_desc(uint32_t address, uint32_t leading_bytes,
                                                      uint32_t stride_bytes, UmmaSwizzle swizzle) {
  return (static_cast<uint64_t>((address >> 4) & 0x3FFFu)) |
         (static_cast<uint64_t>((leading_bytes >> 4) & 0x3FFFu) << 16) |
         (static_cast<uint64_t>((stride_bytes >> 4) & 0x3FFFu) << 32) | (uint64_t{1} << 46) |
         (static_cast<uint64_t>(swizzle) << 61);
}

// The swizzle that matches a K-major row of `row_bytes` (32, 64 or 128) bytes.
__host__ __device__ constexpr UmmaSwizzle umma_row_swizzle(int row_bytes) {
  return row_bytes == 128 ? UmmaSwizzle::k128B : row_bytes == 64 ? UmmaSwizzle::k64B : UmmaSwizzle::k32B;
}

// BF16 x BF16 -> F32 MMA of an M x N tile (kind::f16).
__host__ __device__ constexpr uint32_t umma_idesc_bf16_f32(int m, int n, bool a_mn_major, bool b_mn_major) {
  return (1u << 4) | (1u << 7) | (1u << 10) | (static_cast<uint32_t>(a_mn_major) << 15) |
         (static_cast<uint32_t>(b_mn_major) << 16) | ((static_cast<uint32_t>(n >> 3) & 0x3Fu) << 17) |
         ((static_cast<uint32_t>(m >> 4) & 0x1Fu) << 24);
}

}  // namespace gg

#endif
