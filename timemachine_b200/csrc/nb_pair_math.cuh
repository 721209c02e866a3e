// Per-pair arithmetic of the nonbonded potential: LJ 12-6 + erfc-screened
// (real-space Ewald) electrostatics in 4D, and the int64 fixed-point encoding
// of every output.
//
// Bit-exactness contract. The int64 accumulators are sums of per-pair
// fixed-point integers, so they are order-independent; they equal the
// reference kernel's accumulators exactly when every per-pair FP32 value is
// bit-identical. The expressions below therefore keep the reference's
// expression trees (operand order and association) so that nvcc forms the
// same fused multiply-adds:
//   - pair arithmetic: timemachine/cpp/src/kernels/nonbonded_common.cuh:38-48
//     (erfc factor), :78-102 (electrostatics), :108-140 (Lennard-Jones);
//   - fixed-point encoding: timemachine/cpp/src/fixed_point.hpp:3-8 and
//     timemachine/cpp/src/kernels/k_fixed_point.cuh:51-65 (llrint(v * 2^e));
//   - periodic minimum image: timemachine/cpp/src/kernels/k_nonbonded.cuh:430-432;
//   - the two-product sum with pinned rounding:
//     timemachine/cpp/src/kernels/kernel_utils.cuh:92-98.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace tmb {

// Fixed-point exponents of the accumulators.
constexpr unsigned long long FX_EXPONENT = 0x1000000000ULL;     // 2^36: du_dx, u, du_dl, du_dq
constexpr unsigned long long FX_EXPONENT_SIG = 0x2000000000ULL; // 2^37: du_dsig
constexpr unsigned long long FX_EXPONENT_EPS = 0x4000000000ULL; // 2^38: du_deps

__device__ __forceinline__ unsigned long long to_fixed(float v, unsigned long long exponent) {
    return static_cast<unsigned long long>(llrintf(v * exponent));
}
__device__ __forceinline__ unsigned long long to_fixed(double v, unsigned long long exponent) {
    return static_cast<unsigned long long>(llrint(v * exponent));
}

// a*b + c*d with both products rounded before the sum (no contraction).
__device__ __forceinline__ float sum_of_products_rn(float a, float b, float c, float d) {
    return __fmul_rn(a, b) + __fmul_rn(c, d);
}
__device__ __forceinline__ double sum_of_products_rn(double a, double b, double c, double d) {
    return __dmul_rn(a, b) + __dmul_rn(c, d);
}

__device__ __forceinline__ float inv_sqrt(float x) { return rsqrtf(x); }
__device__ __forceinline__ double inv_sqrt(double x) { return rsqrt(x); }

// Round-half-even to an integral value. For float this is two adds of
// 1.5*2^23, exact for |t| < 2^22 (the periodic image count of a pair is a
// small integer), and bit-identical to nearbyintf there; it keeps the
// minimum-image step on the FP32 pipe instead of the conversion pipe.
__device__ __forceinline__ float round_half_even(float t) {
    const float magic = 12582912.0f; // 1.5 * 2^23
    return __fsub_rn(__fadd_rn(t, magic), magic);
}
__device__ __forceinline__ double round_half_even(double t) { return nearbyint(t); }

// Minimum-image displacement along one axis of an orthorhombic box.
template <typename Real> __device__ __forceinline__ Real min_image(Real delta, Real box, Real inv_box) {
    delta -= box * round_half_even(delta * inv_box);
    return delta;
}

// Derivative factor of qq*erfc(beta d)/d w.r.t. d (divided by d), FP32 form:
// erfc from Abramowitz & Stegun 7.1.26 (five-term rational-exponential fit,
// |error| <= 1.5e-7), reusing exp(-(beta d)^2) for the chain rule.
__device__ __forceinline__ float es_factor(float beta, float d, float inv_d2, float &erfc_bd) {
    float bd = beta * d;
    float e = __expf(-bd * bd);
    float t = 1.0f / (1.0f + 0.3275911f * bd);
    erfc_bd = (0.254829592f + (-0.284496736f + (1.421413741f + (-1.453152027f + 1.061405429f * t) * t) * t) * t) * t * e;
    return -inv_d2 * (static_cast<float>(1.128379167095512595889238330988549829708) * bd * e + erfc_bd);
}
__device__ __forceinline__ double es_factor(double beta, double d, double inv_d2, double &erfc_bd) {
    double bd = beta * d;
    double e = exp(-bd * bd);
    erfc_bd = erfc(bd);
    return -inv_d2 * (static_cast<double>(1.128379167095512595889238330988549829708) * bd * e + erfc_bd);
}

// Electrostatic part of one pair (charge-scaled): fills the distance terms,
// the erfc value, the force prefactor and (if requested) the energy.
template <typename Real, bool COMPUTE_U>
__device__ __forceinline__ void electrostatics(
    const Real charge_scale,
    const Real qi,
    const Real qj,
    const Real d2,
    const Real beta,
    Real &d,
    Real &inv_d,
    Real &inv_d2,
    Real &erfc_bd,
    Real &prefactor,
    Real &u) {
    inv_d = inv_sqrt(d2);
    d = d2 * inv_d;
    inv_d2 = inv_d * inv_d;
    Real qij = qi * qj;
    prefactor = charge_scale * qij * inv_d * es_factor(beta, d, inv_d2, erfc_bd);
    if (COMPUTE_U) {
        u = charge_scale * qij * inv_d * erfc_bd;
    }
}

// Lennard-Jones part of one pair with sigma stored as sigma/2 and epsilon as
// sqrt(epsilon): sig_ij = sig_i + sig_j, eps_ij = eps_i * eps_j.
template <typename Real, bool COMPUTE_U>
__device__ __forceinline__ void lennard_jones(
    const Real lj_scale,
    const Real eps_i,
    const Real eps_j,
    const Real sig_i,
    const Real sig_j,
    const Real inv_d,
    const Real inv_d2,
    Real &u,
    Real &prefactor,
    Real &sig_grad,
    Real &eps_grad) {
    Real eps_ij = eps_i * eps_j;
    Real sig_ij = sig_i + sig_j;

    Real s1 = sig_ij * inv_d;
    Real s2 = s1 * s1;
    Real s4 = s2 * s2;
    Real s6 = s4 * s2;
    Real s6_inv_d2 = s6 * inv_d2;
    Real s5_inv_d = sig_ij * s4 * inv_d2;

    Real lj_prefactor = lj_scale * eps_ij * s6_inv_d2 * (s6 * 48 - 24);
    if (COMPUTE_U) {
        u += lj_scale * 4 * eps_ij * (s6 - 1) * s6;
    }
    prefactor -= lj_prefactor;

    sig_grad = lj_scale * 24 * eps_ij * s5_inv_d * (2 * s6 - 1);
    eps_grad = lj_scale * 4 * (s6 - 1) * s6;
}

} // namespace tmb
