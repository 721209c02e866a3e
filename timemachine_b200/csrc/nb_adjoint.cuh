// Adjoint of the nonbonded forces and du/dlambda with respect to the per-atom
// parameters (charge, sigma/2, sqrt(epsilon)) and the per-atom w offsets.
//
// For upstream gradients G (of du_dx, [N,3]) and g (of du_dl, scalar) it
// accumulates the vector-Jacobian product
//   dPhi/dtheta,  Phi = sum_i G_i . du_dx_i + g * du_dl,
// pair by pair, recomputing each pair's terms in FP64 from the original
// coordinates and parameters (nothing is stored by the forward pass). It walks
// the same tile list and scaled-pair list as the forward kernels.
//
// Per pair (r = x_i - x_j minimum image, dw = w_i - w_j,
// w = cutoff * (plane + offset * lambda), d^2 = r.r + dw^2 < cutoff^2) the
// energy is U(d) = s * [cs * q_i q_j erfc(beta d)/d + ls * 4 e_i e_j ((S/d)^12 - (S/d)^6)]
// (S = sig_i + sig_j; s = +1 for all pairs, -1 for the scaled exclusions;
// LJ only where e_i e_j != 0), as timemachine/potentials/nonbonded.py:29-59,
// 133-264 define it. With h = U'(d)/d the pair adds h r to du_dx_i, -h r to
// du_dx_j and h dw cutoff (off_i - off_j) to du_dl, so
//   Phi_pair = h * B,  B = (G_i - G_j).r + g * dw * cutoff * (off_i - off_j),
//   dPhi/dp      = B * dh/dp                         (p: q, sig, eps of i or j)
//   dPhi/doff_i  = B * h'(d) * dw * cutoff * lambda / d
//                  + g * h * cutoff * (cutoff * lambda * (off_i - off_j) + dw)
//   dPhi/doff_j  = -(the same).
// The derivatives of erfc(beta d)/d follow from d/dd erfc(beta d) =
// -2 beta / sqrt(pi) exp(-beta^2 d^2).
#pragma once

#include "nb_kernels.cuh"

namespace tmb {

struct AdjointArgs {
    int N;
    int S;
    const double *x;      // [N,3]
    const double *p;      // [N,3]
    const double *box;    // [9]
    const int *plane;     // [N]
    const int *offset;    // [N]
    double lambda, beta, cutoff;
    const unsigned *perm; // [S] slot -> atom
    const unsigned *tile_cols;
    const int4 *items;
    int rows;             // slots per row group of the tile list
    int M;
    const int *pair_idxs; // [M,2] atoms
    const double *scales; // [M,2]
    double pair_sign;     // -1: the listed pairs are subtracted (exclusions), +1: added
    const double *g_dx;   // [N,3]
    double g_dl;
    double *grad_p; // [N,3] +=
    double *grad_w; // [N] +=
    DevState *state;
};

// What the pair terms need of one atom: coordinates, parameters (q, sigma/2,
// sqrt eps), the upstream gradient of its du_dx, and its lambda plane/offset.
struct AdjAtom {
    double x[3];
    double p[3];
    double g[3];
    int plane;
    int offset;
};

__device__ __forceinline__ AdjAtom load_adj_atom(const AdjointArgs &a, int atom) {
    AdjAtom t;
    for (int d = 0; d < 3; d++) {
        t.x[d] = a.x[3 * (size_t)atom + d];
        t.p[d] = a.p[3 * (size_t)atom + d];
        t.g[d] = a.g_dx[3 * (size_t)atom + d];
    }
    t.plane = a.plane[atom];
    t.offset = a.offset[atom];
    return t;
}

// Gradient contributions of one pair: to atom i (q, sig, eps, off) and atom j.
struct PairGrad {
    double qi, si, ei, wi;
    double qj, sj, ej, wj;
};

__device__ __forceinline__ PairGrad
adjoint_pair(const AdjointArgs &a, const AdjAtom &I, const AdjAtom &J, double cs, double ls, double sign) {
    PairGrad out = {0, 0, 0, 0, 0, 0, 0, 0};
    double r[3];
    double r2 = 0;
    for (int d = 0; d < 3; d++) {
        const double L = a.box[4 * d];
        double v = I.x[d] - J.x[d];
        v -= L * floor(v / L + 0.5);
        r[d] = v;
        r2 += v * v;
    }
    const double c = a.cutoff;
    const double doff = (double)(I.offset - J.offset);
    const double dw = c * ((I.plane - J.plane) + doff * a.lambda);
    const double d2 = r2 + dw * dw;
    if (!(d2 < c * c)) {
        return out;
    }
    const double d = sqrt(d2);
    const double inv_d = 1.0 / d;
    const double qi = I.p[0], si = I.p[1], ei = I.p[2];
    const double qj = J.p[0], sj = J.p[1], ej = J.p[2];

    // electrostatics: E = erfc(beta d)/d
    const double bd = a.beta * d;
    const double g0 = erfc(bd);
    const double g1 = -2.0 * a.beta * 0.56418958354775628695 * exp(-bd * bd); // d erfc(beta d)/dd
    const double g2 = -2.0 * a.beta * a.beta * d * g1;                           // second derivative
    const double E1 = g1 * inv_d - g0 * inv_d * inv_d;
    const double E2 = g2 * inv_d - 2.0 * g1 * inv_d * inv_d + 2.0 * g0 * inv_d * inv_d * inv_d;
    double h = cs * qi * qj * E1 * inv_d;
    double hp = cs * qi * qj * (E2 * inv_d - E1 * inv_d * inv_d);
    double dh_qi = cs * qj * E1 * inv_d, dh_qj = cs * qi * E1 * inv_d;
    double dh_s = 0, dh_ei = 0, dh_ej = 0;
    if (ei * ej != 0) {
        const double S = si + sj;
        const double sd = S * inv_d;
        const double sd6 = sd * sd * sd * sd * sd * sd;
        const double inv_d2 = inv_d * inv_d;
        // U_lj = 4 e e (sd^12 - sd^6); h_lj = U'/d = 4 e e (-12 sd^12 + 6 sd^6) / d^2
        const double base = (-12.0 * sd6 * sd6 + 6.0 * sd6) * inv_d2;
        const double ee = 4.0 * ls * ei * ej;
        h += ee * base;
        hp += ee * (168.0 * sd6 * sd6 - 48.0 * sd6) * inv_d2 * inv_d;
        dh_s = ee * (-144.0 * sd6 * sd6 + 36.0 * sd6) * inv_d2 / S;
        dh_ei = 4.0 * ls * ej * base;
        dh_ej = 4.0 * ls * ei * base;
    }
    h *= sign;
    hp *= sign;
    const double B = (I.g[0] - J.g[0]) * r[0] + (I.g[1] - J.g[1]) * r[1] + (I.g[2] - J.g[2]) * r[2] +
                     a.g_dl * dw * c * doff;
    out.qi = sign * B * dh_qi;
    out.qj = sign * B * dh_qj;
    out.si = sign * B * dh_s;
    out.sj = out.si;
    out.ei = sign * B * dh_ei;
    out.ej = sign * B * dh_ej;
    const double dphi_doff_i = B * hp * dw * c * a.lambda * inv_d + a.g_dl * h * c * (c * a.lambda * doff + dw);
    out.wi = dphi_doff_i;
    out.wj = -dphi_doff_i;
    return out;
}

__device__ __forceinline__ void adjoint_add(const AdjointArgs &a, int atom, double q, double s, double e, double w) {
    atomicAdd(a.grad_p + 3 * (size_t)atom + 0, q);
    atomicAdd(a.grad_p + 3 * (size_t)atom + 1, s);
    atomicAdd(a.grad_p + 3 * (size_t)atom + 2, e);
    atomicAdd(a.grad_w + atom, w);
}

constexpr int ADJ_WARPS = 4;

// A tile's 32 column atoms, structure-of-arrays in shared memory (one per
// warp), and their gradient accumulators.
struct AdjTileSmem {
    double x[3][TILE];
    double p[3][TILE];
    double g[3][TILE];
    int plane[TILE];
    int offset[TILE];
    unsigned slot[TILE];
    int atom[TILE];
    double acc[4][TILE];
};

// One warp per tile. The tile's 32 column atoms are staged in shared memory.
// With 32-slot row groups lane l holds row l and in round r pairs it with
// column (l + r) mod 32; with smaller groups of R rows, lane l holds row
// l mod R and its lane group sweeps its own R columns in R rounds. Either way
// the lanes of a round touch distinct columns and add into their
// shared-memory accumulators without conflicts. Each tile ends with one FP64
// atomic per (lane, output) for its row and one per (column, output). The
// scaled pairs follow as one lane per pair. Dynamic work counter
// state->next_item (reset by k_check_prepare).
static __global__ void __launch_bounds__(ADJ_WARPS * 32) k_adjoint(AdjointArgs a) {
    __shared__ AdjTileSmem smem[ADJ_WARPS];
    if (a.state->error) {
        return;
    }
    AdjTileSmem &sm = smem[threadIdx.x >> 5];
    const int lane = threadIdx.x & 31;
    const unsigned S = (unsigned)a.S;
    const int chunk = max(1, a.state->items_chunk); // the list's, whichever call built it
    const int n_tile_units = a.tile_cols ? a.state->n_items * chunk : 0;
    const int n_total = n_tile_units + (a.M + TILE - 1) / TILE;
    for (;;) {
        int unit = 0;
        if (lane == 0) {
            unit = atomicAdd(&a.state->next_item, 1);
        }
        unit = __shfl_sync(FULL_MASK, unit, 0);
        if (unit >= n_total) {
            break;
        }
        if (unit >= n_tile_units) {
            const int pair = (unit - n_tile_units) * TILE + lane;
            if (pair < a.M) {
                const int ai = a.pair_idxs[2 * pair], aj = a.pair_idxs[2 * pair + 1];
                const PairGrad g = adjoint_pair(
                    a, load_adj_atom(a, ai), load_adj_atom(a, aj), a.scales[2 * pair], a.scales[2 * pair + 1],
                    a.pair_sign);
                adjoint_add(a, ai, g.qi, g.si, g.ei, g.wi);
                adjoint_add(a, aj, g.qj, g.sj, g.ej, g.wj);
            }
            continue;
        }
        const int4 it = a.items[unit / chunk];
        const int t = unit - (unit / chunk) * chunk;
        if (t >= it.z) {
            continue; // warp-uniform
        }
        const long long tile = (long long)it.y + t;
        // row groups of `rows` slots: lane l holds row l mod rows and sweeps
        // the `rows` columns of its lane group (all 32 when rows = 32)
        const int rows = a.rows;
        const unsigned i = (unsigned)(it.x * rows + (lane & (rows - 1)));
        const int ai = i < S ? (int)a.perm[i] : -1;
        AdjAtom I = {};
        if (ai >= 0) {
            I = load_adj_atom(a, ai);
        }
        {
            const unsigned j = a.tile_cols[tile * TILE + lane];
            const int aj = j < S ? (int)a.perm[j] : -1;
            sm.slot[lane] = j;
            sm.atom[lane] = aj;
            if (aj >= 0) {
                const AdjAtom J = load_adj_atom(a, aj);
                for (int d = 0; d < 3; d++) {
                    sm.x[d][lane] = J.x[d];
                    sm.p[d][lane] = J.p[d];
                    sm.g[d][lane] = J.g[d];
                }
                sm.plane[lane] = J.plane;
                sm.offset[lane] = J.offset;
            }
            for (int k = 0; k < 4; k++) {
                sm.acc[k][lane] = 0.0;
            }
        }
        __syncwarp();
        double rq = 0, rs = 0, re = 0, rw = 0;
        for (int r = 0; r < rows; r++) {
            const int c = (lane & ~(rows - 1)) | (((lane & (rows - 1)) + r) & (rows - 1));
            if (ai >= 0 && sm.atom[c] >= 0 && i < sm.slot[c]) {
                AdjAtom J;
                for (int d = 0; d < 3; d++) {
                    J.x[d] = sm.x[d][c];
                    J.p[d] = sm.p[d][c];
                    J.g[d] = sm.g[d][c];
                }
                J.plane = sm.plane[c];
                J.offset = sm.offset[c];
                const PairGrad g = adjoint_pair(a, I, J, 1.0, 1.0, 1.0);
                rq += g.qi;
                rs += g.si;
                re += g.ei;
                rw += g.wi;
                sm.acc[0][c] += g.qj;
                sm.acc[1][c] += g.sj;
                sm.acc[2][c] += g.ej;
                sm.acc[3][c] += g.wj;
            }
            __syncwarp();
        }
        if (ai >= 0) {
            adjoint_add(a, ai, rq, rs, re, rw);
        }
        if (sm.atom[lane] >= 0) {
            adjoint_add(a, sm.atom[lane], sm.acc[0][lane], sm.acc[1][lane], sm.acc[2][lane], sm.acc[3][lane]);
        }
        __syncwarp();
    }
}

} // namespace tmb
