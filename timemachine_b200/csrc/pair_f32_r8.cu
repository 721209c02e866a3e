// Pair-kernel table: float arithmetic, 8-row tiles, interpolated parameters: false.
#include "pair_kernels.hpp"

TMB_PAIR_TABLE(f32_r8, float, 8, false)
