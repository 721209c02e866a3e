// Per-term device functions of the harmonic bond and (cosine) harmonic angle
// potentials, shared by the bonded potentials (bonded.cu) and the replica
// batch (batch.cu). Functional forms of the reference:
//   bond  U = kb/2 (|r_ij| - b0)^2        timemachine/cpp/src/kernels/k_harmonic_bond.cuh:4-76
//   angle U = ka/2 (cos(theta) - cos a0)^2 timemachine/cpp/src/kernels/k_harmonic_angle.cuh:4-90
// each scaled by (lambda_offset + lambda_mult * lambda). FP32 arithmetic with
// every operation rounded explicitly (no contraction left to the compiler),
// so a term rounds the same wherever it is inlined; outputs accumulate in
// int64 fixed point; du_dp points at the term's two parameter slots (or null).
#pragma once

#include "nb_pair_math.cuh"

namespace tmb {

__device__ __forceinline__ float fdiv(float a, float b) { return __fdiv_rn(a, b); }

__device__ __forceinline__ float lambda_prefactor(int lmult, int loff, double lambda) {
    return fadd((float)loff, fmul((float)lmult, (float)lambda));
}

__device__ __forceinline__ void harmonic_bond_term(
    const double *__restrict__ x,
    int i,
    int j,
    double kb_d,
    double b0_d,
    int lmult,
    int loff,
    double lambda,
    unsigned long long *__restrict__ du_dx,
    unsigned long long *__restrict__ du_dp,
    unsigned long long *__restrict__ du_dl,
    unsigned long long *__restrict__ u) {
    float dx[3];
    float d2 = 0.f;
    for (int d = 0; d < 3; d++) {
        dx[d] = fsub((float)x[3 * i + d], (float)x[3 * j + d]);
        d2 = ffma(dx[d], dx[d], d2);
    }
    const float kb = (float)kb_d, b0 = (float)b0_d;
    const float dij = __fsqrt_rn(d2);
    const float db = fsub(dij, b0);
    const float pre = lambda_prefactor(lmult, loff, lambda);
    if (du_dx) {
        for (int d = 0; d < 3; d++) {
            const float g =
                fmul(b0 != 0.f ? fdiv(fmul(fmul(kb, db), dx[d]), dij) : fmul(kb, dx[d]), pre);
            const unsigned long long f = to_fixed(g, FX_EXPONENT);
            atomicAdd(du_dx + 3 * i + d, f);
            atomicAdd(du_dx + 3 * j + d, 0ULL - f);
        }
    }
    const float half_db2 = fmul(fmul(0.5f, db), db);
    if (du_dp) {
        atomicAdd(du_dp + 0, to_fixed(fmul(half_db2, pre), FX_EXPONENT));
        atomicAdd(du_dp + 1, to_fixed(fmul(fmul(-kb, db), pre), FX_EXPONENT));
    }
    if (u) {
        atomicAdd(u + i, to_fixed(fmul(fmul(kb, half_db2), pre), FX_EXPONENT));
    }
    if (du_dl) {
        atomicAdd(du_dl + i, to_fixed(fmul(fmul((float)lmult, kb), half_db2), FX_EXPONENT));
    }
}

__device__ __forceinline__ void harmonic_angle_term(
    const double *__restrict__ x,
    int i,
    int j,
    int k,
    double ka_d,
    double a0_d,
    int lmult,
    int loff,
    double lambda,
    unsigned long long *__restrict__ du_dx,
    unsigned long long *__restrict__ du_dp,
    unsigned long long *__restrict__ du_dl,
    unsigned long long *__restrict__ u) {
    float rij[3], rkj[3];
    float nij2 = 0.f, nkj2 = 0.f, dot = 0.f;
    for (int d = 0; d < 3; d++) {
        rij[d] = fsub((float)x[3 * i + d], (float)x[3 * j + d]); // j -> i
        rkj[d] = fsub((float)x[3 * k + d], (float)x[3 * j + d]); // j -> k
        nij2 = ffma(rij[d], rij[d], nij2);
        nkj2 = ffma(rkj[d], rkj[d], nkj2);
        dot = ffma(rij[d], rkj[d], dot);
    }
    const float inij = fdiv(1.f, __fsqrt_rn(nij2)), inkj = fdiv(1.f, __fsqrt_rn(nkj2));
    const float cos_t = fmul(fmul(dot, inij), inkj);
    const float ka = (float)ka_d, a0 = (float)a0_d;
    const float delta = fsub(cos_t, cosf(a0));
    const float pre = lambda_prefactor(lmult, loff, lambda);
    if (du_dx) {
        const float f = fmul(fmul(ka, delta), pre);
        const float ii = fmul(inij, inkj);
        for (int d = 0; d < 3; d++) {
            // d cos / d x_i and d x_k; x_j takes the negated sum
            const float gi = fmul(fsub(fmul(rkj[d], ii), fmul(fmul(fmul(cos_t, rij[d]), inij), inij)), f);
            const float gk = fmul(fsub(fmul(rij[d], ii), fmul(fmul(fmul(cos_t, rkj[d]), inkj), inkj)), f);
            const unsigned long long fi = to_fixed(gi, FX_EXPONENT);
            const unsigned long long fk = to_fixed(gk, FX_EXPONENT);
            atomicAdd(du_dx + 3 * i + d, fi);
            atomicAdd(du_dx + 3 * k + d, fk);
            atomicAdd(du_dx + 3 * j + d, 0ULL - fi - fk);
        }
    }
    const float half_d2 = fmul(fmul(0.5f, delta), delta);
    if (du_dp) {
        atomicAdd(du_dp + 0, to_fixed(fmul(half_d2, pre), FX_EXPONENT));
        atomicAdd(du_dp + 1, to_fixed(fmul(fmul(fmul(delta, ka), sinf(a0)), pre), FX_EXPONENT));
    }
    if (u) {
        atomicAdd(u + i, to_fixed(fmul(fmul(ka, half_d2), pre), FX_EXPONENT));
    }
    if (du_dl) {
        atomicAdd(du_dl + i, to_fixed(fmul(fmul((float)lmult, ka), half_d2), FX_EXPONENT));
    }
}

} // namespace tmb
