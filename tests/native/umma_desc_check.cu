// Host-only check that the tcgen05 descriptor encoders of sonium_b200/csrc/sb_umma.cuh put every
// field where CUTLASS's cute::UMMA descriptor types put it (built and run by tests/test_capi.py).
#include <cstdio>
#include <cute/arch/mma_sm100_desc.hpp>
#include <cute/numeric/numeric_types.hpp>

#include "sb_umma.cuh"

int main() {
    int bad = 0;
    const int shapes[][2] = {{128, 256}, {128, 128}, {64, 64}, {128, 16}};
    for (auto& mn : shapes) {
        uint32_t ref = 0;
        if (mn[0] == 128 && mn[1] == 256)
            ref = uint32_t(cute::UMMA::make_instr_desc<cute::bfloat16_t, cute::bfloat16_t, float, 128, 256,
                                                       cute::UMMA::Major::K, cute::UMMA::Major::K>());
        else if (mn[0] == 128 && mn[1] == 128)
            ref = uint32_t(cute::UMMA::make_instr_desc<cute::bfloat16_t, cute::bfloat16_t, float, 128, 128,
                                                       cute::UMMA::Major::K, cute::UMMA::Major::K>());
        else if (mn[0] == 64)
            ref = uint32_t(cute::UMMA::make_instr_desc<cute::bfloat16_t, cute::bfloat16_t, float, 64, 64,
                                                       cute::UMMA::Major::K, cute::UMMA::Major::K>());
        else
            ref = uint32_t(cute::UMMA::make_instr_desc<cute::bfloat16_t, cute::bfloat16_t, float, 128, 16,
                                                       cute::UMMA::Major::K, cute::UMMA::Major::K>());
        const uint32_t ours = sb::umma::instr_desc_bf16_f32(mn[0], mn[1]);
        if (ours != ref) {
            std::printf("instr %dx%d: ours %08x cutlass %08x\n", mn[0], mn[1], ours, ref);
            bad = 1;
        }
    }
    {
        const uint32_t ref = uint32_t(cute::UMMA::make_instr_desc<int8_t, int8_t, int32_t, 128, 256,
                                                                  cute::UMMA::Major::K, cute::UMMA::Major::K>());
        const uint32_t ours = sb::umma::instr_desc_s8_s32(128, 256);
        if (ours != ref) {
            std::printf("instr s8 128x256: ours %08x cutlass %08x\n", ours, ref);
            bad = 1;
        }
    }
    for (uint32_t addr : {0x0u, 0x400u, 0x12340u, 0x3FFF0u}) {
        cute::UMMA::SmemDescriptor d;
        d.start_address_ = static_cast<uint16_t>(addr >> 4);
        d.leading_byte_offset_ = 1;
        d.stride_byte_offset_ = 1024 >> 4;
        d.version_ = 1;
        d.base_offset_ = 0;
        d.lbo_mode_ = 0;
        d.layout_type_ = uint8_t(cute::UMMA::LayoutType::SWIZZLE_128B);
        const uint64_t ours = sb::umma::smem_desc_k_sw128(addr);
        if (ours != d.desc_) {
            std::printf("smem %x: ours %016llx cutlass %016llx\n", addr, (unsigned long long)ours,
                        (unsigned long long)d.desc_);
            bad = 1;
        }
    }
    for (uint32_t addr : {0x0u, 0x200u, 0x12340u, 0x3FFF0u}) {
        cute::UMMA::SmemDescriptor d;
        d.start_address_ = static_cast<uint16_t>(addr >> 4);
        d.leading_byte_offset_ = 1;
        d.stride_byte_offset_ = 512 >> 4;
        d.version_ = 1;
        d.base_offset_ = 0;
        d.lbo_mode_ = 0;
        d.layout_type_ = uint8_t(cute::UMMA::LayoutType::SWIZZLE_64B);
        const uint64_t ours = sb::umma::smem_desc_k_sw64(addr);
        if (ours != d.desc_) {
            std::printf("smem64 %x: ours %016llx cutlass %016llx\n", addr, (unsigned long long)ours,
                        (unsigned long long)d.desc_);
            bad = 1;
        }
    }
    std::printf(bad ? "MISMATCH\n" : "OK\n");
    return bad;
}
