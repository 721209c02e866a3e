// Pair-kernel table: float arithmetic, 16-row tiles, interpolated parameters: true.
#include "pair_kernels.hpp"

TMB_PAIR_TABLE(f32_r16_interp, float, 16, true)
