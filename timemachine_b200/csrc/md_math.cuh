// Device helpers of the Langevin integrator shared by the single-system
// Context (md.cu) and the replica batch (batch.cu): a counter-based
// Philox4x32-10 generator (Salmon, Moraes, Dror, Shaw, "Parallel random
// numbers: as easy as 1, 2, 3", SC'11), Box-Muller normals, and the per-atom
// update of timemachine/cpp/src/integrator.cu:37-69 (BAOAB rotated by half a
// step) with the force read from the int64 fixed-point accumulator.
#pragma once

#include "nb_pair_math.cuh"

namespace tmb {

__device__ __forceinline__ uint4 philox4x32_10(uint4 c, uint2 k) {
    const unsigned M0 = 0xD2511F53u, M1 = 0xCD9E8D57u, W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
#pragma unroll
    for (int r = 0; r < 10; r++) {
        const unsigned hi0 = __umulhi(M0, c.x), lo0 = M0 * c.x;
        const unsigned hi1 = __umulhi(M1, c.z), lo1 = M1 * c.z;
        c = make_uint4(hi1 ^ c.y ^ k.x, lo1, hi0 ^ c.w ^ k.y, lo0);
        k.x += W0;
        k.y += W1;
    }
    return c;
}

// uniform double in (0, 1) from 53 random bits
__device__ __forceinline__ double u01(unsigned a, unsigned b) {
    const unsigned long long m = ((unsigned long long)(a >> 5) << 26) | (b >> 6);
    return ((double)m + 0.5) * (1.0 / 9007199254740992.0);
}

// two standard normals (Box-Muller)
__device__ __forceinline__ double2 normal2(unsigned a, unsigned b, unsigned c, unsigned d) {
    const double u1 = u01(a, b);
    const double u2 = u01(c, d);
    const double r = sqrt(-2.0 * log(u1));
    double s, co;
    sincospi(2.0 * u2, &s, &co);
    return make_double2(r * co, r * s);
}

// One component's update with its noise; the force accumulator is zeroed for
// the next step. `extra` is added to the accumulator first (fixed point: the
// forces a fused potential left in its own slot-ordered accumulators).
// Returns the new coordinate.
__device__ __forceinline__ double langevin_dim(
    int k,
    double noise,
    double ca,
    double cb,
    double cc,
    double dt,
    double *__restrict__ x,
    double *__restrict__ v,
    unsigned long long *__restrict__ du_dx,
    unsigned long long extra = 0) {
    const double force = static_cast<double>(static_cast<long long>(du_dx[k] + extra)) / FX_EXPONENT;
    const double v_mid = v[k] + cb * force;
    const double v_new = ca * v_mid + cc * noise;
    v[k] = v_new;
    const double x_new = x[k] + 0.5 * dt * (v_mid + v_new);
    x[k] = x_new;
    du_dx[k] = 0; // the next step accumulates from zero
    return x_new;
}

// One atom's update: v_mid = v + cb * F, v' = ca * v_mid + cc * noise,
// x' = x + dt/2 * (v_mid + v'); the force accumulator is zeroed for the next
// step. Noise: Philox keyed by `key`, counter (atom, step).
__device__ __forceinline__ void langevin_atom(
    int i,
    unsigned long long step,
    uint2 key,
    double ca,
    double cb,
    double cc,
    double dt,
    double *__restrict__ x,
    double *__restrict__ v,
    unsigned long long *__restrict__ du_dx) {
    const uint4 r0 = philox4x32_10(make_uint4((unsigned)i, (unsigned)step, (unsigned)(step >> 32), 0u), key);
    const uint4 r1 = philox4x32_10(make_uint4((unsigned)i, (unsigned)step, (unsigned)(step >> 32), 1u), key);
    const double2 n01 = normal2(r0.x, r0.y, r0.z, r0.w);
    const double2 n23 = normal2(r1.x, r1.y, r1.z, r1.w);
    const double noise[3] = {n01.x, n01.y, n23.x};
#pragma unroll
    for (int d = 0; d < 3; d++) {
        langevin_dim(3 * i + d, noise[d], ca, cb, cc, dt, x, v, du_dx);
    }
}

// The same update split over two threads: half 0 draws the first Philox
// block and updates x and y, half 1 the second block and z (the same numbers
// and arithmetic per component as langevin_atom).
__device__ __forceinline__ void langevin_atom_half(
    int i,
    int half,
    unsigned long long step,
    uint2 key,
    double ca,
    double cb,
    double cc,
    double dt,
    double *__restrict__ x,
    double *__restrict__ v,
    unsigned long long *__restrict__ du_dx) {
    const uint4 r = philox4x32_10(make_uint4((unsigned)i, (unsigned)step, (unsigned)(step >> 32), (unsigned)half), key);
    const double2 n = normal2(r.x, r.y, r.z, r.w);
    if (half == 0) {
        langevin_dim(3 * i + 0, n.x, ca, cb, cc, dt, x, v, du_dx);
        langevin_dim(3 * i + 1, n.y, ca, cb, cc, dt, x, v, du_dx);
    } else {
        langevin_dim(3 * i + 2, n.x, ca, cb, cc, dt, x, v, du_dx);
    }
}

} // namespace tmb
