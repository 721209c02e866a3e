// Tables of the pair-kernel instantiations (k_pair of nb_kernels.cuh) for
// one arithmetic type, tile row-group size and parameter mode: 16 output
// selections for single-window and multi-window lists each. Every table is
// compiled in a translation unit of its own (pair_*.cu), so the builds of the
// variants run in parallel.
#pragma once

#include "nb_kernels.cuh"

#include <utility>

namespace tmb {

typedef void (*pair_kernel_t)(PairArgs);

// index: bit3 U, bit2 DU_DX, bit1 DU_DL, bit0 DU_DP -- the flag order of
// timemachine/cpp/src/nonbonded_all_pairs.cu:374-379
struct PairKernels {
    pair_kernel_t single[16];
    pair_kernel_t multi[16];
};

template <typename Real, int RG, bool INTERP, size_t... Is>
void fill_pair_kernels(PairKernels &out, std::index_sequence<Is...>) {
    ((out.single[Is] = &k_pair<Real, bool((Is >> 3) & 1), bool((Is >> 2) & 1), bool((Is >> 1) & 1), bool(Is & 1),
                               INTERP, false, RG>),
     ...);
    ((out.multi[Is] = &k_pair<Real, bool((Is >> 3) & 1), bool((Is >> 2) & 1), bool((Is >> 1) & 1), bool(Is & 1),
                              INTERP, true, RG>),
     ...);
}

#define TMB_PAIR_TABLE(NAME, REAL, RG, INTERP)                                                                      \
    namespace tmb {                                                                                                  \
    void pair_kernels_##NAME(PairKernels &out) {                                                                     \
        fill_pair_kernels<REAL, RG, INTERP>(out, std::make_index_sequence<16>{});                                     \
    }                                                                                                                \
    }

void pair_kernels_f32_r32(PairKernels &out);
void pair_kernels_f32_r32_interp(PairKernels &out);
void pair_kernels_f32_r16(PairKernels &out);
void pair_kernels_f32_r16_interp(PairKernels &out);
void pair_kernels_f32_r8(PairKernels &out);
void pair_kernels_f32_r8_interp(PairKernels &out);
void pair_kernels_f64_r16(PairKernels &out);
void pair_kernels_f64_r16_interp(PairKernels &out);

} // namespace tmb
