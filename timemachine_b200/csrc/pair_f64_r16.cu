// Pair-kernel table: double arithmetic, 16-row tiles, interpolated parameters: false.
#include "pair_kernels.hpp"

TMB_PAIR_TABLE(f64_r16, double, 16, false)
