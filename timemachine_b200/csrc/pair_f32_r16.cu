// Pair-kernel table: float arithmetic, 16-row tiles, interpolated parameters: false.
#include "pair_kernels.hpp"

TMB_PAIR_TABLE(f32_r16, float, 16, false)
