// Pair-kernel table: double arithmetic, 16-row tiles, interpolated parameters: true.
#include "pair_kernels.hpp"

TMB_PAIR_TABLE(f64_r16_interp, double, 16, true)
