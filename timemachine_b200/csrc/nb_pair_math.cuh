// Per-pair arithmetic of the nonbonded potential: LJ 12-6 + erfc-screened
// (real-space Ewald) electrostatics in 4D, and the int64 fixed-point encoding
// of every output.
//
// Bit-exactness contract. The int64 accumulators are sums of per-pair
// fixed-point integers, so they are order-independent; they equal the
// reference kernel's accumulators exactly when every per-pair FP32 value is
// bit-identical. Every FP32 operation below is therefore written with an
// explicit rounding intrinsic (__fmaf_rn, __fmul_rn, __fadd_rn, __fsub_rn):
// the compiler cannot contract or re-associate them, so each pair gets the
// same rounding in every kernel, loop copy and output variant, and the fused
// multiply-adds sit where the reference's compiled expressions put them.
// The expression trees follow
//   - pair arithmetic: timemachine/cpp/src/kernels/nonbonded_common.cuh:38-48
//     (erfc factor), :78-102 (electrostatics), :108-140 (Lennard-Jones);
//   - distances and minimum image: timemachine/cpp/src/kernels/k_nonbonded.cuh:426-442;
//   - fixed-point encoding: timemachine/cpp/src/fixed_point.hpp:3-8 and
//     timemachine/cpp/src/kernels/k_fixed_point.cuh:51-65 (llrint(v * 2^e));
//   - the two-product sum: timemachine/cpp/src/kernels/kernel_utils.cuh:92-98.
// TMNB_DAG_* select, at each point where a multiply feeds an add, which of
// the two rounding patterns is used (1 = fused multiply-add).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#ifndef TMNB_DAG_D2
#define TMNB_DAG_D2 0 // 0: fma(dz,dz,fma(dx,dx,dy*dy)); 1: fma(dz,dz,fma(dy,dy,dx*dx)); 2: unfused
#endif
#ifndef TMNB_DAG_MINIMG
#define TMNB_DAG_MINIMG 1 // d - box*n: 1 fused, 0 unfused
#endif
#ifndef TMNB_DAG_DEN
#define TMNB_DAG_DEN 1 // 1 + 0.3275911*bd: 1 fused, 0 unfused
#endif
#ifndef TMNB_DAG_POLY
#define TMNB_DAG_POLY 1 // Horner steps: 1 fused, 0 unfused
#endif
#ifndef TMNB_DAG_ERF
#define TMNB_DAG_ERF 1 // c*bd*e + erfc: 1 fma((c*bd), e, erfc); 0 unfused; 2 fma(erfc_factors, e, c*bd*e)
#endif
#ifndef TMNB_DAG_PRE
#define TMNB_DAG_PRE 1 // es_pref - lj_pref: 1 fma(-X,Y,es); 0 unfused; 2 fma(qij_inv, factor, -(X*Y))
#endif
#ifndef TMNB_DAG_LJP
#define TMNB_DAG_LJP 1 // s6*48 - 24: 1 fused, 0 unfused
#endif
#ifndef TMNB_DAG_U
#define TMNB_DAG_U 1 // u_es + A*s6: 1 fma(A,s6,u_es); 0 unfused; 2 fma(qij_inv, erfc, A*s6)
#endif
#ifndef TMNB_DAG_S6M1
#define TMNB_DAG_S6M1 0 // s6 - 1: 0 fsub(s6,1); 1 fma(s4,s2,-1)
#endif
#ifndef TMNB_DAG_2S6M1
#define TMNB_DAG_2S6M1 0 // 2*s6 - 1: 0 fma(2,s6,-1) (= fl(2 s6 - 1)); 1 fl(fma(s4,s2,s6) - 1)
#endif
#ifndef TMNB_DAG_D4
#define TMNB_DAG_D4 1 // d2 + dw*dw: 1 fused, 0 unfused
#endif

namespace tmb {

// Waits until the previous kernel in the stream has completed and its memory
// is visible (a no-op unless this kernel was launched with programmatic
// stream serialization).
__device__ __forceinline__ void grid_dependency_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

// explicit-rounding helpers (FP32 and FP64)
__device__ __forceinline__ float fmul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float fadd(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float fsub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float ffma(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ double fmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double fadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double fsub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double ffma(double a, double b, double c) { return __fma_rn(a, b, c); }

// Fixed-point exponents of the accumulators.
constexpr unsigned long long FX_EXPONENT = 0x1000000000ULL;     // 2^36: du_dx, u, du_dl, du_dq
constexpr unsigned long long FX_EXPONENT_SIG = 0x2000000000ULL; // 2^37: du_dsig
constexpr unsigned long long FX_EXPONENT_EPS = 0x4000000000ULL; // 2^38: du_deps

__device__ __forceinline__ unsigned long long to_fixed(float v, unsigned long long exponent) {
    return static_cast<unsigned long long>(llrintf(__fmul_rn(v, static_cast<float>(exponent))));
}
__device__ __forceinline__ unsigned long long to_fixed(double v, unsigned long long exponent) {
    return static_cast<unsigned long long>(llrint(__dmul_rn(v, static_cast<double>(exponent))));
}

// Round-half-even to int64 of an already scaled value (llrintf / llrint), and
// the magnitude from which that conversion saturates.
__device__ __forceinline__ unsigned long long fixed_round(float y) {
    return static_cast<unsigned long long>(llrintf(y));
}
__device__ __forceinline__ unsigned long long fixed_round(double y) {
    return static_cast<unsigned long long>(llrint(y));
}
__device__ __forceinline__ bool fixed_in_range(float y) { return fabsf(y) < 0x1p63f; }
__device__ __forceinline__ bool fixed_in_range(double y) { return fabs(y) < 0x1p63; }

// Fixed-point encodings of a pair term v and of its negation -v, for the two
// atoms of the pair. llrint is odd under round-half-even, so the second is
// -first (one conversion instead of two) -- except where the conversion
// saturates (|v * 2^e| >= 2^63) or v is NaN, where the negated value is
// converted on its own to keep the reference's exact result.
template <typename Real>
__device__ __forceinline__ void to_fixed_pair(
    Real v, unsigned long long exponent, unsigned long long &pos, unsigned long long &neg) {
    const Real y = fmul(v, static_cast<Real>(exponent));
    pos = fixed_round(y);
    if (fixed_in_range(y)) { // strictly inside the int64 range
        neg = 0ULL - pos;
    } else {
        neg = fixed_round(-y);
    }
}


// Packed FP32x2 arithmetic (sm_100: mul/add/sub/fma .rn.f32x2): each
// component rounds exactly as the scalar __fmul_rn / __fadd_rn / __fsub_rn /
// __fmaf_rn. Inline PTX, so the compiler never contracts a product and a sum.
__device__ __forceinline__ float2 f2(float v) { return make_float2(v, v); }
__device__ __forceinline__ float2 fmul2(float2 a, float2 b) {
    float2 r;
    asm("{\n\t.reg .b64 ra, rb, rd;\n\tmov.b64 ra, {%2, %3};\n\tmov.b64 rb, {%4, %5};\n\t"
        "mul.rn.f32x2 rd, ra, rb;\n\tmov.b64 {%0, %1}, rd;\n\t}"
        : "=f"(r.x), "=f"(r.y)
        : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
    return r;
}
__device__ __forceinline__ float2 fadd2(float2 a, float2 b) {
    float2 r;
    asm("{\n\t.reg .b64 ra, rb, rd;\n\tmov.b64 ra, {%2, %3};\n\tmov.b64 rb, {%4, %5};\n\t"
        "add.rn.f32x2 rd, ra, rb;\n\tmov.b64 {%0, %1}, rd;\n\t}"
        : "=f"(r.x), "=f"(r.y)
        : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
    return r;
}
__device__ __forceinline__ float2 fsub2(float2 a, float2 b) {
    float2 r;
    asm("{\n\t.reg .b64 ra, rb, rd;\n\tmov.b64 ra, {%2, %3};\n\tmov.b64 rb, {%4, %5};\n\t"
        "sub.rn.f32x2 rd, ra, rb;\n\tmov.b64 {%0, %1}, rd;\n\t}"
        : "=f"(r.x), "=f"(r.y)
        : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
    return r;
}
__device__ __forceinline__ float2 ffma2(float2 a, float2 b, float2 c) {
    float2 r;
    asm("{\n\t.reg .b64 ra, rb, rc, rd;\n\tmov.b64 ra, {%2, %3};\n\tmov.b64 rb, {%4, %5};\n\t"
        "mov.b64 rc, {%6, %7};\n\tfma.rn.f32x2 rd, ra, rb, rc;\n\tmov.b64 {%0, %1}, rd;\n\t}"
        : "=f"(r.x), "=f"(r.y)
        : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y), "f"(c.x), "f"(c.y));
    return r;
}
__device__ __forceinline__ float2 madd2(float2 a, float2 b, float2 c, int fused) {
    return fused ? ffma2(a, b, c) : fadd2(fmul2(a, b), c);
}

// a*b + c*d with both products rounded before the sum.
template <typename Real> __device__ __forceinline__ Real sum_of_products_rn(Real a, Real b, Real c, Real d) {
    return fadd(fmul(a, b), fmul(c, d));
}

// acc + a*b with the reference's fused rounding
template <typename Real> __device__ __forceinline__ Real mul_add(Real a, Real b, Real acc) { return ffma(a, b, acc); }

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

// Minimum-image displacement along one axis of an orthorhombic box:
// delta - box * nearbyint(delta / box).
template <typename Real> __device__ __forceinline__ Real min_image(Real delta, Real box, Real inv_box) {
    const Real n = round_half_even(fmul(delta, inv_box));
#if TMNB_DAG_MINIMG
    return ffma(-box, n, delta);
#else
    return fsub(delta, fmul(box, n));
#endif
}

// squared 3D distance
template <typename Real> __device__ __forceinline__ Real dist2(Real dx, Real dy, Real dz) {
#if TMNB_DAG_D2 == 0
    return ffma(dz, dz, ffma(dx, dx, fmul(dy, dy)));
#elif TMNB_DAG_D2 == 1
    return ffma(dz, dz, ffma(dy, dy, fmul(dx, dx)));
#else
    return fadd(fadd(fmul(dx, dx), fmul(dy, dy)), fmul(dz, dz));
#endif
}

template <typename Real> __device__ __forceinline__ Real add_w2(Real d2, Real dw) {
#if TMNB_DAG_D4
    return ffma(dw, dw, d2);
#else
    return fadd(d2, fmul(dw, dw));
#endif
}

// min_image per component; neg_box = -box.
__device__ __forceinline__ float2 min_image2(float2 delta, float2 neg_box, float2 inv_box) {
    const float2 magic = f2(12582912.0f); // round_half_even
    const float2 n = fsub2(fadd2(fmul2(delta, inv_box), magic), magic);
#if TMNB_DAG_MINIMG
    return ffma2(neg_box, n, delta);
#else
    return fadd2(delta, fmul2(neg_box, n));
#endif
}

template <typename Real> __device__ __forceinline__ Real madd(Real a, Real b, Real c, int fused) {
    return fused ? ffma(a, b, c) : fadd(fmul(a, b), c);
}

// Derivative factor of qq*erfc(beta d)/d w.r.t. d (divided by d), FP32 form:
// erfc from Abramowitz & Stegun 7.1.26 (five-term rational-exponential fit,
// |error| <= 1.5e-7), reusing exp(-(beta d)^2) for the chain rule. The IEEE
// reciprocal __frcp_rn equals the correctly rounded 1.0f/x of the reference.
__device__ __forceinline__ float es_factor(float beta, float d, float inv_d2, float &erfc_bd) {
    const float bd = fmul(beta, d);
    const float e = __expf(fmul(-bd, bd));
    const float t = __frcp_rn(madd(0.3275911f, bd, 1.0f, TMNB_DAG_DEN));
    float poly = madd(1.061405429f, t, -1.453152027f, TMNB_DAG_POLY);
    poly = madd(poly, t, 1.421413741f, TMNB_DAG_POLY);
    poly = madd(poly, t, -0.284496736f, TMNB_DAG_POLY);
    poly = madd(poly, t, 0.254829592f, TMNB_DAG_POLY);
    erfc_bd = fmul(fmul(poly, t), e);
    const float cbd = fmul(static_cast<float>(1.128379167095512595889238330988549829708), bd);
#if TMNB_DAG_ERF == 1
    const float s = ffma(cbd, e, erfc_bd);
#elif TMNB_DAG_ERF == 0
    const float s = fadd(fmul(cbd, e), erfc_bd);
#else
    const float s = ffma(fmul(poly, t), e, fmul(cbd, e));
#endif
    return fmul(-inv_d2, s);
}
__device__ __forceinline__ double es_factor(double beta, double d, double inv_d2, double &erfc_bd) {
    const double bd = beta * d;
    const double e = exp(-bd * bd);
    erfc_bd = erfc(bd);
    return -inv_d2 * (static_cast<double>(1.128379167095512595889238330988549829708) * bd * e + erfc_bd);
}

// Electrostatic part of one pair (charge-scaled): distance terms, the erfc
// value, the force prefactor and (if requested) the energy. `qij_inv` is
// (charge_scale * q_i q_j) / d, shared by prefactor and energy.
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
    Real &u,
    Real &qij_inv,
    Real &factor) {
    inv_d = inv_sqrt(d2);
    d = fmul(d2, inv_d);
    inv_d2 = fmul(inv_d, inv_d);
    const Real qij = fmul(qi, qj);
    qij_inv = fmul(fmul(charge_scale, qij), inv_d);
    factor = es_factor(beta, d, inv_d2, erfc_bd);
    prefactor = fmul(qij_inv, factor);
    if (COMPUTE_U) {
        u = fmul(qij_inv, erfc_bd);
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
    const Real qij_inv,
    const Real factor,
    const Real erfc_bd,
    Real &u,
    Real &prefactor,
    Real &sig_grad,
    Real &eps_grad) {
    const Real eps_ij = fmul(eps_i, eps_j);
    const Real sig_ij = fadd(sig_i, sig_j);
    const Real s1 = fmul(sig_ij, inv_d);
    const Real s2 = fmul(s1, s1);
    const Real s4 = fmul(s2, s2);
    const Real s6 = fmul(s4, s2);
    const Real s6_inv_d2 = fmul(s6, inv_d2);
    const Real s5_inv_d = fmul(fmul(sig_ij, s4), inv_d2);
#if TMNB_DAG_S6M1
    const Real s6m1 = ffma(s4, s2, (Real)-1);
#else
    const Real s6m1 = fsub(s6, (Real)1);
#endif
    const Real ljx = fmul(fmul(lj_scale, eps_ij), s6_inv_d2);
    const Real ljy = madd(s6, (Real)48, (Real)-24, TMNB_DAG_LJP);
#if TMNB_DAG_PRE == 1
    prefactor = ffma(-ljx, ljy, prefactor);
#elif TMNB_DAG_PRE == 0
    prefactor = fsub(prefactor, fmul(ljx, ljy));
#else
    prefactor = ffma(qij_inv, factor, -fmul(ljx, ljy));
#endif
    if (COMPUTE_U) {
        const Real A = fmul(fmul(fmul(lj_scale, (Real)4), eps_ij), s6m1);
#if TMNB_DAG_U == 1
        u = ffma(A, s6, u);
#elif TMNB_DAG_U == 0
        u = fadd(u, fmul(A, s6));
#else
        u = ffma(qij_inv, erfc_bd, fmul(A, s6));
#endif
    }
#if TMNB_DAG_2S6M1
    const Real two_s6_m1 = fsub(ffma(s4, s2, s6), (Real)1);
#else
    const Real two_s6_m1 = ffma((Real)2, s6, (Real)-1);
#endif
    sig_grad = fmul(fmul(fmul(fmul(lj_scale, (Real)24), eps_ij), s5_inv_d), two_s6_m1);
    eps_grad = fmul(fmul(fmul(lj_scale, (Real)4), s6m1), s6);
}

// Neighbour-list validity: true when an atom moved more than half the padding
// since the last rebuild (squared displacement against (padding / 2)^2).
// Explicit rounding, so the pair kernel's own check and the MD integrator's
// fused check take the same decision for the same coordinates.
__device__ __forceinline__ bool moved_beyond_half_padding(double dx, double dy, double dz, double half_pad2) {
    return __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz)) > half_pad2;
}

} // namespace tmb
