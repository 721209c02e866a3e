// Pair-kernel table: float arithmetic, 8-row tiles, interpolated parameters: true.
#include "pair_kernels.hpp"

TMB_PAIR_TABLE(f32_r8_interp, float, 8, true)
