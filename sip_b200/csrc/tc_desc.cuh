// Operand descriptors of tcgen05.mma (kind::f16) for the tensor-core FFT
// stages.  Host and device callable so that the CPU tests can compare the bit
// packing with CUTLASS's UMMA::SmemDescriptor / UMMA::InstrDescriptor.
#pragma once
#include <stdint.h>

#ifdef __CUDACC__
#define SIPFFT_TC_HD __host__ __device__
#else
#define SIPFFT_TC_HD
#endif

namespace sipfft {

// Shared-memory matrix descriptor, K-major, no swizzle: core matrices of
// 8 rows x 16 bytes; LBO = distance of the two 8-element K halves of one
// MMA (128 B here), SBO = distance of consecutive 8-row groups.
SIPFFT_TC_HD constexpr uint64_t umma_smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo)
{
    return uint64_t((addr >> 4) & 0x3FFFu) | (uint64_t((lbo >> 4) & 0x3FFFu) << 16) |
           (uint64_t((sbo >> 4) & 0x3FFFu) << 32) | (uint64_t(1) << 46);
}

// Instruction descriptor of kind::f16 with FP32 accumulation; fmt 0 = F16,
// 1 = BF16; a_mn / b_mn = 1 when that operand is MN-major (else K-major).
SIPFFT_TC_HD constexpr uint32_t umma_instr_desc(int m, int n, int fmt, int a_mn = 0, int b_mn = 0)
{
    return (1u << 4) | (uint32_t(fmt) << 7) | (uint32_t(fmt) << 10) | (uint32_t(a_mn) << 15) |
           (uint32_t(b_mn) << 16) | (uint32_t(n >> 3) << 17) | (uint32_t(m >> 4) << 24);
}

// Byte offset of element (m, k) of an MN-major operand, no swizzle: core
// matrices of 8 K-rows x 16 bytes (8 consecutive m), K groups 128 bytes apart
// (LBO = 128), 8-row M groups `sbo` bytes apart (SBO; may be padded so that
// consecutive groups start in different shared-memory banks).
SIPFFT_TC_HD constexpr uint32_t umma_offset_mn(int m, int k, uint32_t sbo)
{
    return uint32_t((m >> 3) * sbo + (k >> 3) * 128 + (k & 7) * 16 + (m & 7) * 2);
}

// Byte offset of element (row, k) of a K-major operand with K columns.
SIPFFT_TC_HD constexpr uint32_t umma_offset(int row, int k, int K)
{
    return uint32_t((row >> 3) * (K * 16) + (k >> 3) * 128 + (row & 7) * 16 + (k & 7) * 2);
}

}  // namespace sipfft
