// Host check of the tcgen05 operand descriptors of the tensor-core FFT stages
// (sip_b200/csrc/tc_desc.cuh) against CUTLASS's UMMA descriptor unions, and of
// the operand byte layout against the canonical K-major no-swizzle layout
// ((8,m),(8,2)) : ((16 B, SBO), (2 B, LBO)) that the descriptor describes.
#include <cstdio>

#include <cute/arch/mma_sm100_desc.hpp>
#include <cute/atom/mma_traits_sm100.hpp>
#include <cute/tensor.hpp>

#include "tc_desc.cuh"

int main()
{
    int bad = 0;
    for (uint32_t addr : {0u, 128u, 4096u, 65536u, 200000u}) {
        for (uint32_t K : {64u, 128u}) {
            const uint32_t lbo = 128, sbo = K * 16;
            cute::UMMA::SmemDescriptor d;
            d.start_address_ = addr >> 4;
            d.leading_byte_offset_ = lbo >> 4;
            d.stride_byte_offset_ = sbo >> 4;
            d.version_ = 1;
            d.base_offset_ = 0;
            d.lbo_mode_ = 0;
            d.layout_type_ = uint8_t(cute::UMMA::LayoutType::SWIZZLE_NONE);
            const uint64_t mine = sipfft::umma_smem_desc(addr, lbo, sbo);
            if (uint64_t(d) != mine) {
                std::printf("smem desc mismatch addr=%u K=%u: cute %llx mine %llx\n", addr, K,
                            (unsigned long long)uint64_t(d), (unsigned long long)mine);
                bad++;
            }
        }
    }
    for (int fmt = 0; fmt < 2; fmt++) {
        for (int n : {16, 32, 64, 128, 256}) {
            cute::UMMA::InstrDescriptor d;
            d.desc_ = 0;
            d.c_format_ = 1;  // F32
            d.a_format_ = uint8_t(fmt);
            d.b_format_ = uint8_t(fmt);
            d.a_major_ = 0;
            d.b_major_ = 0;
            d.n_dim_ = n >> 3;
            d.m_dim_ = 128 >> 4;
            const uint32_t mine = sipfft::umma_instr_desc(128, n, fmt);
            if (uint32_t(d) != mine) {
                std::printf("instr desc mismatch fmt=%d n=%d: cute %x mine %x\n", fmt, n, uint32_t(d), mine);
                bad++;
            }
        }
    }
    // CUTLASS's own constructor for the F16 / BF16 x F32 case
    {
        const auto c16 = cute::UMMA::make_instr_desc<cute::half_t, cute::half_t, float, 128, 64, cute::UMMA::Major::K,
                                                     cute::UMMA::Major::K>();
        const auto cbf = cute::UMMA::make_instr_desc<cute::bfloat16_t, cute::bfloat16_t, float, 128, 128,
                                                     cute::UMMA::Major::K, cute::UMMA::Major::K>();
        if (uint32_t(c16) != sipfft::umma_instr_desc(128, 64, 0)) {
            std::printf("make_instr_desc f16 mismatch %x %x\n", uint32_t(c16), sipfft::umma_instr_desc(128, 64, 0));
            bad++;
        }
        if (uint32_t(cbf) != sipfft::umma_instr_desc(128, 128, 1)) {
            std::printf("make_instr_desc bf16 mismatch %x %x\n", uint32_t(cbf), sipfft::umma_instr_desc(128, 128, 1));
            bad++;
        }
    }
    // CUTLASS's descriptor builder on the two operand layouts of the row pipeline
    // (start address is not representable on the host; LBO / SBO / layout are)
    {
        using namespace cute;
        half_t *p = reinterpret_cast<half_t *>(0x400);
        // MN-major A operand, K = 128, padded SBO of 2064 bytes (1032 elements)
        auto mn = make_layout(make_shape(make_shape(Int<8>{}, Int<16>{}), make_shape(Int<8>{}, Int<16>{})),
                              make_stride(make_stride(Int<1>{}, Int<1032>{}), make_stride(Int<8>{}, Int<64>{})));
        UMMA::SmemDescriptor dm = UMMA::make_umma_desc<UMMA::Major::MN>(make_tensor(make_smem_ptr(p), mn));
        const uint64_t mine_mn = sipfft::umma_smem_desc(0, 128, 2064);
        if ((uint64_t(dm) & ~uint64_t(0x3FFF)) != (mine_mn & ~uint64_t(0x3FFF))) {
            std::printf("MN-major smem desc mismatch: cute %llx mine %llx\n", (unsigned long long)uint64_t(dm),
                        (unsigned long long)mine_mn);
            bad++;
        }
        // K-major B operand (DFT matrix), K = 128, packed
        auto km = make_layout(make_shape(make_shape(Int<8>{}, Int<16>{}), make_shape(Int<8>{}, Int<16>{})),
                              make_stride(make_stride(Int<8>{}, Int<1024>{}), make_stride(Int<1>{}, Int<64>{})));
        UMMA::SmemDescriptor dk = UMMA::make_umma_desc<UMMA::Major::K>(make_tensor(make_smem_ptr(p), km));
        const uint64_t mine_k = sipfft::umma_smem_desc(0, 128, 2048);
        if ((uint64_t(dk) & ~uint64_t(0x3FFF)) != (mine_k & ~uint64_t(0x3FFF))) {
            std::printf("K-major smem desc mismatch: cute %llx mine %llx\n", (unsigned long long)uint64_t(dk),
                        (unsigned long long)mine_k);
            bad++;
        }
    }
    // MN-major operand: K groups LBO = 128 bytes apart, 8-row M groups SBO apart
    for (int mn = 0; mn < 2; mn++) {
        const auto c = mn ? cute::UMMA::make_instr_desc<cute::half_t, cute::half_t, float, 128, 128,
                                                        cute::UMMA::Major::MN, cute::UMMA::Major::K>()
                          : cute::UMMA::make_instr_desc<cute::bfloat16_t, cute::bfloat16_t, float, 128, 64,
                                                        cute::UMMA::Major::MN, cute::UMMA::Major::K>();
        const uint32_t mine = mn ? sipfft::umma_instr_desc(128, 128, 0, 1, 0) : sipfft::umma_instr_desc(128, 64, 1, 1, 0);
        if (uint32_t(c) != mine) {
            std::printf("MN-major instr desc mismatch: cute %x mine %x\n", uint32_t(c), mine);
            bad++;
        }
    }
    for (int m = 0; m < 128; m++)
        for (int k = 0; k < 128; k++) {
            const uint32_t sbo = 2064;
            const uint32_t canon = (m / 8) * sbo + (k / 8) * 128 + (k % 8) * 16 + (m % 8) * 2;
            if (sipfft::umma_offset_mn(m, k, sbo) != canon) {
                std::printf("mn layout error m=%d k=%d\n", m, k);
                bad++;
            }
        }
    // layout: element (r, k) sits at (r/8)*SBO + (k/8)*LBO + (r%8)*16 + (k%8)*2, every byte once
    for (int K : {64, 128}) {
        const int rows = 128;
        static unsigned char seen[128 * 128 * 2];
        for (int i = 0; i < rows * K * 2; i++) seen[i] = 0;
        for (int r = 0; r < rows; r++)
            for (int k = 0; k < K; k++) {
                const uint32_t o = sipfft::umma_offset(r, k, K);
                const uint32_t canon = (r / 8) * (K * 16) + (k / 8) * 128 + (r % 8) * 16 + (k % 8) * 2;
                if (o != canon || o + 2 > uint32_t(rows * K * 2) || seen[o]) {
                    std::printf("layout error r=%d k=%d K=%d off=%u\n", r, k, K, o);
                    bad++;
                    break;
                }
                seen[o] = 1;
            }
    }
    if (bad == 0) std::printf("ALL OK\n");
    return bad ? 1 : 0;
}
