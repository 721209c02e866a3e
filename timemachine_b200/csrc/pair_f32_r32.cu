// Pair-kernel table: float arithmetic, 32-row tiles, interpolated parameters: false.
#include "pair_kernels.hpp"

TMB_PAIR_TABLE(f32_r32, float, 32, false)
