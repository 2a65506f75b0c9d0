// Host-side check of daphne-benchmark_b200/csrc/umma_desc.h against CUTLASS's
// CuTe descriptor types (compiled and run by tests/test_umma_desc.py; no GPU).
#include <cstdio>
#include <cute/arch/mma_sm100_desc.hpp>
#include <cute/numeric/numeric_types.hpp>

#include "umma_desc.h"

int main() {
    int bad = 0;
    // instruction descriptor: BF16 x BF16 -> FP32, K-major A and B
    const int shapes[][2] = {{128, 128}, {128, 64}, {64, 128}, {128, 256}};
    for (auto &mn : shapes) {
        uint32_t ref = 0;
        if (mn[0] == 128 && mn[1] == 128)
            ref = (uint32_t)cute::UMMA::make_instr_desc<cute::bfloat16_t, cute::bfloat16_t, float, 128, 128,
                                                        cute::UMMA::Major::K, cute::UMMA::Major::K>();
        else if (mn[0] == 128 && mn[1] == 64)
            ref = (uint32_t)cute::UMMA::make_instr_desc<cute::bfloat16_t, cute::bfloat16_t, float, 128, 64,
                                                        cute::UMMA::Major::K, cute::UMMA::Major::K>();
        else if (mn[0] == 64)
            ref = (uint32_t)cute::UMMA::make_instr_desc<cute::bfloat16_t, cute::bfloat16_t, float, 64, 128,
                                                        cute::UMMA::Major::K, cute::UMMA::Major::K>();
        else
            ref = (uint32_t)cute::UMMA::make_instr_desc<cute::bfloat16_t, cute::bfloat16_t, float, 128, 256,
                                                        cute::UMMA::Major::K, cute::UMMA::Major::K>();
        const uint32_t ours = umma::instr_desc_bf16_f32(mn[0], mn[1]);
        printf("idesc M=%d N=%d ours=%08x cute=%08x\n", mn[0], mn[1], ours, ref);
        bad += ours != ref;
    }
    // shared-memory descriptor: no swizzle, K-major, as CuTe's make_umma_desc
    // fills it (version 1, legacy offset mode, base offset 0)
    const uint32_t addrs[] = {0u, 1024u, 16384u + 256u, 0x3fff0u};
    for (uint32_t a : addrs) {
        cute::UMMA::SmemDescriptor d;
        d.version_ = 1;
        d.lbo_mode_ = 0;
        d.layout_type_ = uint8_t(cute::UMMA::LayoutType::SWIZZLE_NONE);
        d.start_address_ = static_cast<uint16_t>(a >> 4);
        d.base_offset_ = 0;
        d.leading_byte_offset_ = 128 >> 4;
        d.stride_byte_offset_ = 1024 >> 4;
        const uint64_t ours = umma::smem_desc_kmajor_interleaved(a, 128, 1024);
        printf("sdesc addr=%u ours=%016llx cute=%016llx\n", a, (unsigned long long)ours,
               (unsigned long long)(uint64_t)d);
        bad += ours != (uint64_t)d;
    }
    printf(bad ? "MISMATCH\n" : "OK\n");
    return bad ? 1 : 0;
}
