// Pair-kernel table: float arithmetic, 32-row tiles, interpolated parameters: true.
#include "pair_kernels.hpp"

TMB_PAIR_TABLE(f32_r32_interp, float, 32, true)
