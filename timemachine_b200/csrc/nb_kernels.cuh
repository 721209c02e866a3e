// Device pipeline of one nonbonded evaluation on sm_100a.
//
// Per evaluation (stream-ordered, no host synchronisation):
//   k_check_prepare   rebuild decision (any atom moved > padding/2, or box
//                     changed), box validation, and the per-slot FP32 staging
//                     of coordinates, w, parameters (and dp/dlambda) using the
//                     current slot order.
//   k_bin_keys / k_bin_scan / k_bin_scatter / k_block_bounds / k_build_tiles
//                     neighbour-list rebuild; every one returns at once unless
//                     the rebuild flag is set, so the sequence is graph-capturable.
//   k_pair            persistent kernel over the tile work items and the
//                     exclusion / scaled-pair chunks (dynamic scheduling).
//   k_finalize        scatter of the slot-ordered int64 accumulators into the
//                     caller's original-order outputs, then zeroing.
//
// The work of each stage follows the reference pipeline
// (timemachine/cpp/src/nonbonded_all_pairs.cu:222-433,
//  timemachine/cpp/src/neighborlist.cu:126-185,
//  timemachine/cpp/src/nonbonded_pair_list.cu:95-166); the data layout,
// spatial sort, scheduling and fusion are this file's own.
//
// The non-template kernels have internal linkage (static), so that several
// translation units can include this file.
#pragma once

#include "nb_pair_math.cuh"
#include "tmnb.h"

namespace tmb {

constexpr unsigned FULL_MASK = 0xffffffffu;
constexpr int TILE = 32;

// Forces-only FP32 evaluations of 16-row tiles use the packed two-rows-per-lane
// sweep (sweep_forces_p2); 0 selects the one-row sweep for them too. Measured
// on B200 (bit-identical results): MD step of the 22,840-atom box 137.9 ->
// 132.9 us, batched MD step of 128 replicas 4.14 -> 3.93 ms. The packed
// kernels run at 6 CTAs/SM (80 registers); 5 measured slower.
#ifndef TMNB_PACKED_FORCES
#define TMNB_PACKED_FORCES 1
#endif
#ifndef TMNB_PACKED_FORCES_CTAS
#define TMNB_PACKED_FORCES_CTAS 6
#endif
// Energy-only FP32 evaluations of 16-row tiles (the barostat's) use the same
// packed sweep.
#ifndef TMNB_PACKED_ENERGY
#define TMNB_PACKED_ENERGY 1
#endif
// The one-row sweep evaluates the independent x / y steps of a pair (minimum
// image, force components) and the paired charge / epsilon derivatives in
// the two components of packed FP32x2 operations.
#ifndef TMNB_PACKED_SCALAR
#define TMNB_PACKED_SCALAR 1
#endif

// Sticky device-side state of one potential instance.
struct DevState {
    int rebuild;          // 1: the neighbour list must be rebuilt in this evaluation
    int error;            // sticky error code (TMNB_ERR_* values), 0 = ok
    int n_items;          // tile work items produced by the last rebuild
    int next_item;        // dynamic work counter of k_pair (reset by k_check_prepare, or in a
                          // fused MD step by the integrator kernel that staged the coordinates)
    unsigned done_ctas;   // completion counter of k_build_tiles
    unsigned total_tiles; // tiles produced by the last rebuild
    int rebuilds;         // number of rebuilds performed (diagnostics)
    int n_dep;            // lambda-dependent tiles listed by k_dep_tiles (multi-window calls)
    int dep_dirty;        // 1: the list of lambda-dependent tiles must be redone (rebuild, or lamdep changed)
    int items_chunk;      // tiles per work item in the list of the last rebuild
    int item_count;       // work items reserved so far by the rebuild in progress (0 between rebuilds)
};

// Error codes written into DevState::error (mirrored in include/tmnb.h).
constexpr int DEV_ERR_NONORTHO_BOX = 3;
constexpr int DEV_ERR_BOX_TOO_SMALL = 4;

// Up to this many lambda windows are evaluated together (one launch sequence).
constexpr int MAX_WINDOWS = TMNB_MAX_WINDOWS;

struct SlotArrays {
    float4 *posw;            // [K][S] x, y, z, w(lambda_k)
    float4 *prm;             // [K][S] q, sig, eps, dw/dlambda (parameters at lambda_k)
    float4 *dprm;            // [K][S] dq/dl, dsig/dl, deps/dl, 0 (interpolated only)
    unsigned char *lamdep;   // [S] 1 when the atom's staged values depend on lambda
    // FP64 pair arithmetic only (nullptr otherwise): the same values unrounded
    double4 *posw64;         // [K][S]
    double4 *prm64;          // [K][S]
    double4 *dprm64;         // [K][S] (interpolated only)
};

// One lambda window as the staging sees it: the values f(lambda) and
// derivatives g = df/dlambda of the four lambda transforms (charge, sigma,
// epsilon, w) of timemachine/cpp/src/kernels/k_lambda_transformer_jit.cuh:8-22,
// evaluated on the host for each call (identity transform: f = lambda, g = 1).
struct LambdaWindow {
    double f_q, g_q;
    double f_s, g_s;
    double f_e, g_e;
    double f_w, g_w;
};

struct PrepareArgs {
    int N;                      // atoms in the system
    int S;                      // slots (atoms in the evaluated set)
    const double *x;            // [N,3]
    const double *p;            // [N,3] or [2N,3] (interpolated)
    const double *box;          // [3,3]
    int K;                      // lambda windows
    LambdaWindow lam[MAX_WINDOWS];
    double cutoff;
    double padding;
    const int *plane;           // [N]
    const int *offset;          // [N]
    int interpolated;
    SlotArrays slots;
};

// Staging of one atom for window k, with the transforms of window k:
// w = cutoff*(plane + offset*f_w), dw/dlambda = offset*g_w*cutoff
// (timemachine/cpp/src/kernels/k_lambda_transformer_jit.cuh:25-55);
// interpolated parameters p = (1-f) p0 + f p1 and dp/dlambda = g (p1 - p0)
// per parameter column (same file :57-98). v[0..5] receives the staged
// parameters and their lambda derivatives in FP64.
__device__ __forceinline__ void window_values(const PrepareArgs &a, int atom, int k, double &w, double &dw_dl,
                                              double (&v)[6]) {
    const int plane = a.plane[atom];
    const int offset = a.offset[atom];
    const LambdaWindow &L = a.lam[k];
    w = (plane + offset * L.f_w) * a.cutoff;
    dw_dl = offset * L.g_w * a.cutoff;
    const double *p0 = a.p + 3 * (size_t)atom;
    v[0] = p0[0];
    v[1] = p0[1];
    v[2] = p0[2];
    v[3] = v[4] = v[5] = 0.0;
    if (a.interpolated) {
        const double *p1 = a.p + 3 * ((size_t)a.N + atom);
        v[0] = (1 - L.f_q) * p0[0] + L.f_q * p1[0];
        v[1] = (1 - L.f_s) * p0[1] + L.f_s * p1[1];
        v[2] = (1 - L.f_e) * p0[2] + L.f_e * p1[2];
        v[3] = L.g_q * (p1[0] - p0[0]);
        v[4] = L.g_s * (p1[1] - p0[1]);
        v[5] = L.g_e * (p1[2] - p0[2]);
    }
}

__device__ __forceinline__ void stage_window(const PrepareArgs &a, int s, int atom, int k) {
    double w, dw_dl, v[6];
    window_values(a, atom, k, w, dw_dl, v);
    const double *xa = a.x + 3 * (size_t)atom;
    const size_t o = (size_t)k * a.S + s;
    a.slots.posw[o] = make_float4((float)xa[0], (float)xa[1], (float)xa[2], (float)w);
    a.slots.prm[o] = make_float4((float)v[0], (float)v[1], (float)v[2], (float)dw_dl);
    if (a.interpolated) {
        a.slots.dprm[o] = make_float4((float)v[3], (float)v[4], (float)v[5], 0.0f);
    }
    if (a.slots.posw64 != nullptr) {
        a.slots.posw64[o] = make_double4(xa[0], xa[1], xa[2], w);
        a.slots.prm64[o] = make_double4(v[0], v[1], v[2], dw_dl);
        if (a.interpolated) {
            a.slots.dprm64[o] = make_double4(v[3], v[4], v[5], 0.0);
        }
    }
}

// An atom is lambda-dependent when its offset is nonzero, its end states
// differ, or any window stages parameter values other than window 0's: pairs
// of lambda-independent atoms give the same per-pair values in every window,
// bit for bit.
__device__ __forceinline__ bool lambda_dependent(const PrepareArgs &a, int atom) {
    if (a.offset[atom] != 0) {
        return true;
    }
    if (!a.interpolated) {
        return false;
    }
    const double *p0 = a.p + 3 * (size_t)atom;
    const double *p1 = a.p + 3 * ((size_t)a.N + atom);
    if (p0[0] != p1[0] || p0[1] != p1[1] || p0[2] != p1[2]) {
        return true;
    }
    double w, dw_dl, first[6], v[6];
    window_values(a, atom, 0, w, dw_dl, first);
    for (int k = 1; k < a.K; k++) {
        window_values(a, atom, k, w, dw_dl, v);
        for (int c = 0; c < 6; c++) {
            if (v[c] != first[c]) {
                return true;
            }
        }
    }
    return false;
}

// Stage one atom into its slot for every window and record its lambda dependence.
__device__ __forceinline__ void prepare_slot(const PrepareArgs &a, int s, int atom) {
    for (int k = 0; k < a.K; k++) {
        stage_window(a, s, atom, k);
    }
    a.slots.lamdep[s] = lambda_dependent(a, atom) ? 1 : 0;
}

// ---------------------------------------------------------------------------
// Rebuild decision + staging.
// ---------------------------------------------------------------------------
static __global__ void k_check_prepare(
    PrepareArgs a,
    const unsigned *__restrict__ perm, // [S] slot -> atom
    const double *__restrict__ nb_x,   // [N,3] coordinates at the last rebuild (nullptr: no neighbour list)
    const double *__restrict__ nb_box, // [9]
    DevState *state) {
    grid_dependency_wait();
    const int tid = blockIdx.x * blockDim.x + threadIdx.x;
    if (tid == 0) {
        state->next_item = 0;
        if (nb_x != nullptr) {
            // Orthorhombic box whose every edge is at least twice cutoff+padding
            // (timemachine/cpp/src/nonbonded_all_pairs.cu:315-329); checked in
            // the reference's order, so an off-diagonal entry wins.
            const double db_cutoff = (a.cutoff + a.padding) * 2;
            int err = 0;
            for (int k = 0; k < 9 && err == 0; k++) {
                if (k == 0 || k == 4 || k == 8) {
                    if (a.box[k] < db_cutoff) {
                        err = DEV_ERR_BOX_TOO_SMALL;
                    }
                } else if (a.box[k] != 0.0) {
                    err = DEV_ERR_NONORTHO_BOX;
                }
            }
            if (err != 0) {
                state->error = err;
            }
            for (int k = 0; k < 9; k++) {
                if (a.box[k] != nb_box[k]) {
                    state->rebuild = 1;
                }
            }
        }
    }
    // one thread per (window, slot), slots fastest: the K windows' staging
    // stores spread over the grid; the window-0 thread of a slot also takes
    // the rebuild test and the slot's lambda dependence
    const double half_pad2 = 0.25 * a.padding * a.padding;
    const size_t total = (size_t)a.S * (size_t)a.K;
    for (size_t t = tid; t < total; t += (size_t)gridDim.x * blockDim.x) {
        const int k = (int)(t / (size_t)a.S);
        const int s = (int)(t - (size_t)k * a.S);
        const int atom = perm[s];
        stage_window(a, s, atom, k);
        if (k != 0) {
            continue;
        }
        if (nb_x != nullptr) {
            const double *xn = a.x + 3 * (size_t)atom;
            const double *xo = nb_x + 3 * (size_t)atom;
            const double dx = xn[0] - xo[0];
            const double dy = xn[1] - xo[1];
            const double dz = xn[2] - xo[2];
            if (moved_beyond_half_padding(dx, dy, dz, half_pad2)) {
                state->rebuild = 1; // benign race: every writer stores 1
            }
        }
        const unsigned char dep = lambda_dependent(a, atom) ? 1 : 0;
        if (a.slots.lamdep[s] != dep) {
            a.slots.lamdep[s] = dep;
            // the lambda-dependent tiles change with it (benign race: every writer stores the same)
            state->dep_dirty = 1;
            state->n_dep = 0;
        }
    }
}

// ---------------------------------------------------------------------------
// Spatial sort: atoms are binned into a 2^b x 2^b x 2^b grid whose cells are
// ordered along a 3D Hilbert curve; a counting sort over the cells gives the
// slot order. The Hilbert index uses Skilling's transposed-axes algorithm
// (J. Skilling, "Programming the Hilbert curve", AIP Conf. Proc. 707, 2004).
// Order inside a cell is arbitrary: results do not depend on it because all
// accumulation is exact integer arithmetic.
// ---------------------------------------------------------------------------
__device__ __forceinline__ unsigned hilbert_index_3d(unsigned x, unsigned y, unsigned z, int bits) {
    unsigned X[3] = {x, y, z};
    const unsigned M = 1u << (bits - 1);
    for (unsigned Q = M; Q > 1; Q >>= 1) {
        const unsigned P = Q - 1;
        for (int i = 0; i < 3; i++) {
            if (X[i] & Q) {
                X[0] ^= P;
            } else {
                const unsigned t = (X[0] ^ X[i]) & P;
                X[0] ^= t;
                X[i] ^= t;
            }
        }
    }
    X[1] ^= X[0];
    X[2] ^= X[1];
    unsigned t = 0;
    for (unsigned Q = M; Q > 1; Q >>= 1) {
        if (X[2] & Q) {
            t ^= Q - 1;
        }
    }
    X[0] ^= t;
    X[1] ^= t;
    X[2] ^= t;
    unsigned h = 0;
    for (int b = bits - 1; b >= 0; b--) {
        h = (h << 3) | (((X[0] >> b) & 1u) << 2) | (((X[1] >> b) & 1u) << 1) | ((X[2] >> b) & 1u);
    }
    return h;
}

struct SortArgs {
    int N;
    int S;
    const double *x;
    const double *box;
    const int *set_atoms; // [S] atoms of the evaluated set, nullptr: identity (S == N)
    int n_first;          // set entries [0, n_first) sort before the others (interaction
                          // group rows before columns); S: one group
    int grid_bits;        // b: 2^b cells per axis
    int hilbert;          // 0: keep the set order
    unsigned *keys;       // [S]
    int *bin_count;       // [8^b]
    int *bin_cursor;      // [8^b]
};

__device__ __forceinline__ int set_atom(const SortArgs &a, int k) { return a.set_atoms ? a.set_atoms[k] : k; }

__device__ __forceinline__ void bin_key(const SortArgs &a, int k) {
    const int G = 1 << a.grid_bits;
    {
        const int atom = set_atom(a, k);
        unsigned c[3];
        for (int d = 0; d < 3; d++) {
            const double L = a.box[d * 4];
            double v = a.x[3 * (size_t)atom + d];
            v -= L * floor(v / L);
            int ci = (int)(v / L * G);
            ci = ci < 0 ? 0 : (ci >= G ? G - 1 : ci);
            c[d] = (unsigned)ci;
        }
        unsigned key = hilbert_index_3d(c[0], c[1], c[2], a.grid_bits);
        if (k >= a.n_first) {
            key += 1u << (3 * a.grid_bits);
        }
        a.keys[k] = key;
        atomicAdd(&a.bin_count[key], 1);
    }
}

static __global__ void k_bin_keys(SortArgs a, const DevState *state) {
    grid_dependency_wait();
    if (!state->rebuild || state->error || !a.hilbert) {
        return;
    }
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < a.S; k += gridDim.x * blockDim.x) {
        bin_key(a, k);
    }
}

// Single-CTA exclusive scan of the cell counts (and reset of the counts and
// of the tile-build counters).
__device__ __forceinline__ void bin_scan_cta(const SortArgs &a, DevState *state) {
    if (threadIdx.x == 0) {
        state->done_ctas = 0;
        state->total_tiles = 0;
    }
    if (!a.hilbert) {
        return;
    }
    const int NB = (1 << (3 * a.grid_bits)) * (a.n_first < a.S ? 2 : 1);
    __shared__ int warp_sums[32];
    __shared__ int carry;
    if (threadIdx.x == 0) {
        carry = 0;
    }
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const int wid = threadIdx.x >> 5;
    const int nwarps = blockDim.x >> 5;
    // four consecutive cells per thread (NB is a multiple of 64, the counts
    // 256-byte aligned): a quarter of the passes and barriers
    for (int base = 0; base < NB; base += 4 * (int)blockDim.x) {
        const int b = base + 4 * (int)threadIdx.x;
        const int4 c4 = b < NB ? *reinterpret_cast<const int4 *>(a.bin_count + b) : make_int4(0, 0, 0, 0);
        const int v = c4.x + c4.y + c4.z + c4.w;
        int incl = v;
        for (int o = 1; o < 32; o <<= 1) {
            const int n = __shfl_up_sync(FULL_MASK, incl, o);
            if (lane >= o) {
                incl += n;
            }
        }
        if (lane == 31) {
            warp_sums[wid] = incl;
        }
        __syncthreads();
        if (wid == 0) {
            int ws = lane < nwarps ? warp_sums[lane] : 0;
            for (int o = 1; o < 32; o <<= 1) {
                const int n = __shfl_up_sync(FULL_MASK, ws, o);
                if (lane >= o) {
                    ws += n;
                }
            }
            if (lane < nwarps) {
                warp_sums[lane] = ws; // inclusive
            }
        }
        __syncthreads();
        const int warp_prefix = wid > 0 ? warp_sums[wid - 1] : 0;
        if (b < NB) {
            const int e = carry + warp_prefix + incl - v;
            *reinterpret_cast<int4 *>(a.bin_cursor + b) = make_int4(e, e + c4.x, e + c4.x + c4.y, e + c4.x + c4.y + c4.z);
            *reinterpret_cast<int4 *>(a.bin_count + b) = make_int4(0, 0, 0, 0);
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            carry += warp_sums[nwarps - 1];
        }
        __syncthreads();
    }
}

static __global__ void k_bin_scan(SortArgs a, DevState *state) {
    grid_dependency_wait();
    if (!state->rebuild || state->error) {
        return;
    }
    bin_scan_cta(a, state);
}

// Slot of set entry k after the counting sort; records the slot order and the
// coordinates of the rebuild.
__device__ __forceinline__ int scatter_slot(
    const SortArgs &sa, int k, unsigned *__restrict__ perm, int *__restrict__ slot_of, double *__restrict__ nb_x) {
    const int atom = set_atom(sa, k);
    const int s = sa.hilbert ? atomicAdd(&sa.bin_cursor[sa.keys[k]], 1) : k;
    perm[s] = (unsigned)atom;
    if (slot_of) {
        slot_of[atom] = s;
    }
    nb_x[3 * (size_t)atom + 0] = sa.x[3 * (size_t)atom + 0];
    nb_x[3 * (size_t)atom + 1] = sa.x[3 * (size_t)atom + 1];
    nb_x[3 * (size_t)atom + 2] = sa.x[3 * (size_t)atom + 2];
    return s;
}

static __global__ void k_bin_scatter(
    SortArgs sa,
    PrepareArgs pa,
    unsigned *__restrict__ perm,    // [S] slot -> atom
    int *__restrict__ slot_of,      // [N] atom -> slot (nullptr: not needed)
    double *__restrict__ nb_x,      // [N,3]
    double *__restrict__ nb_box,    // [9]
    const DevState *state) {
    grid_dependency_wait();
    if (!state->rebuild || state->error) {
        return;
    }
    const int tid = blockIdx.x * blockDim.x + threadIdx.x;
    if (tid < 9) {
        nb_box[tid] = sa.box[tid];
    }
    for (int k = tid; k < sa.S; k += gridDim.x * blockDim.x) {
        const int atom = set_atom(sa, k);
        const int s = scatter_slot(sa, k, perm, slot_of, nb_x);
        prepare_slot(pa, s, atom);
    }
}

// ---------------------------------------------------------------------------
// Block bounding boxes: one warp per 32-slot block; every atom is imaged
// next to the block's first atom, then min/max give centre and half-extent.
// ---------------------------------------------------------------------------
__device__ __forceinline__ float wrap_delta(float d, float L, float inv_L) { return d - L * rintf(d * inv_L); }

// Lennard-Jones atoms first within each row group (`rows` slots) of the
// 32-slot block rb (one warp): the pair kernel's LJ branch is taken in a
// rotation round only when some lane pairs two LJ atoms, and with LJ rows and
// LJ columns both leading the tile those pairs fall in fewer rounds. Sorting
// within row groups, not across them, keeps each group spatially compact.
// Blocks that straddle the interaction group's row/column boundary keep their
// order. Restages the moved atoms' slots.
__device__ __forceinline__ void lj_first_warp(
    const PrepareArgs &pa, int S, int n_first, int rb, unsigned *__restrict__ perm, int *__restrict__ slot_of,
    int rows = TILE) {
    const int lane = threadIdx.x & 31;
    const int lo = rb * TILE;
    const int hi = min(S, lo + TILE);
    if (lo < n_first && hi > n_first) {
        return;
    }
    const int s = lo + lane;
    const bool valid = s < S;
    const unsigned atom = valid ? perm[s] : 0u;
    bool lj = false;
    if (valid) {
        lj = pa.p[3 * (size_t)atom + 2] != 0.0;
        if (pa.interpolated) {
            lj = lj || pa.p[3 * ((size_t)pa.N + atom) + 2] != 0.0;
        }
    }
    const unsigned m = __ballot_sync(FULL_MASK, lj);
    const unsigned vm = __ballot_sync(FULL_MASK, valid);
    if (m == 0u || m == vm) {
        return;
    }
    const unsigned lt = (1u << lane) - 1u;
    const int seg = lane / rows;
    const unsigned segm = (rows == TILE ? FULL_MASK : ((1u << rows) - 1u)) << (seg * rows);
    const int pos = seg * rows +
                    (lj ? __popc(m & lt & segm) : __popc(m & segm) + __popc(vm & ~m & lt & segm));
    __syncwarp();
    if (valid && lo + pos != s) {
        const int ns = lo + pos;
        perm[ns] = atom;
        if (slot_of) {
            slot_of[atom] = ns;
        }
        prepare_slot(pa, ns, (int)atom);
    }
    __syncwarp();
}

// Writes one tile's 32 column slots with the LJ atoms first (prm: staged
// parameters, eps in .z; nullptr keeps the order).
__device__ __forceinline__ void store_tile_lj_first(
    unsigned *__restrict__ dst, unsigned s, unsigned S, const float4 *__restrict__ prm) {
    const int lane = threadIdx.x & 31;
    if (prm == nullptr) {
        dst[lane] = s;
        return;
    }
    const bool lj = s < S && prm[s].z != 0.f;
    const unsigned m = __ballot_sync(FULL_MASK, lj);
    const unsigned lt = (1u << lane) - 1u;
    const int pos = lj ? __popc(m & lt) : __popc(m) + __popc(~m & lt);
    dst[pos] = s;
}

// Bounding box of the 32-slot block rb (one warp).
__device__ __forceinline__ void block_bounds_warp(
    int S,
    int rb,
    const double *__restrict__ box,
    const float4 *__restrict__ posw,
    float4 *__restrict__ bb_ctr,
    float4 *__restrict__ bb_ext) {
    const int lane = threadIdx.x & 31;
    const float Lx = (float)box[0], Ly = (float)box[4], Lz = (float)box[8];
    const float iLx = 1.0f / Lx, iLy = 1.0f / Ly, iLz = 1.0f / Lz;
    {
        const int s = rb * TILE + lane;
        const bool valid = s < S;
        float4 p = valid ? posw[s] : make_float4(0.f, 0.f, 0.f, 0.f);
        const float rx = __shfl_sync(FULL_MASK, p.x, 0);
        const float ry = __shfl_sync(FULL_MASK, p.y, 0);
        const float rz = __shfl_sync(FULL_MASK, p.z, 0);
        float dx = wrap_delta(p.x - rx, Lx, iLx);
        float dy = wrap_delta(p.y - ry, Ly, iLy);
        float dz = wrap_delta(p.z - rz, Lz, iLz);
        float mnx = valid ? dx : 3.0e38f, mny = valid ? dy : 3.0e38f, mnz = valid ? dz : 3.0e38f;
        float mxx = valid ? dx : -3.0e38f, mxy = valid ? dy : -3.0e38f, mxz = valid ? dz : -3.0e38f;
        for (int o = 16; o > 0; o >>= 1) {
            mnx = fminf(mnx, __shfl_xor_sync(FULL_MASK, mnx, o));
            mny = fminf(mny, __shfl_xor_sync(FULL_MASK, mny, o));
            mnz = fminf(mnz, __shfl_xor_sync(FULL_MASK, mnz, o));
            mxx = fmaxf(mxx, __shfl_xor_sync(FULL_MASK, mxx, o));
            mxy = fmaxf(mxy, __shfl_xor_sync(FULL_MASK, mxy, o));
            mxz = fmaxf(mxz, __shfl_xor_sync(FULL_MASK, mxz, o));
        }
        if (lane == 0) {
            bb_ctr[rb] = make_float4(rx + 0.5f * (mnx + mxx), ry + 0.5f * (mny + mxy), rz + 0.5f * (mnz + mxz), 0.f);
            // widen by a relative rounding allowance so the box test stays conservative
            bb_ext[rb] = make_float4(
                0.5f * (mxx - mnx) * 1.000001f + 1e-6f,
                0.5f * (mxy - mny) * 1.000001f + 1e-6f,
                0.5f * (mxz - mnz) * 1.000001f + 1e-6f,
                0.f);
        }
    }
}

static __global__ void k_block_bounds(
    int S,
    const double *__restrict__ box,
    const float4 *__restrict__ posw,
    float4 *__restrict__ bb_ctr,
    float4 *__restrict__ bb_ext,
    const DevState *state,
    PrepareArgs pa,
    int n_first,
    unsigned *__restrict__ perm,
    int *__restrict__ slot_of,
    int rows) {
    grid_dependency_wait();
    if (!state->rebuild || state->error) {
        return;
    }
    const int RB = (S + TILE - 1) / TILE;
    for (int rb = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; rb < RB; rb += (gridDim.x * blockDim.x) >> 5) {
        lj_first_warp(pa, S, n_first, rb, perm, slot_of, rows);
        block_bounds_warp(S, rb, box, posw, bb_ctr, bb_ext);
    }
}

// ---------------------------------------------------------------------------
// Tile list. Rows come in groups of `rows` (32, 16 or 8) consecutive slots;
// one CTA (TB_WARPS warps) per row group g. For every 32-slot column block from
// the one holding the group's first slot on (upper triangle) whose bounding
// box is within the list radius of the group's box, each column atom at or
// after the group's first slot is kept when any row atom lies within the list
// radius (minimum image, 3D). Kept atoms are packed 32 to a tile, so a tile is
// rows x 32 pairs; smaller row groups sit in smaller regions and list fewer
// out-of-range column atoms. The tiles of row group g occupy a fixed range
// (tile_base) sized by the column blocks it can reach. Each group's CTA cuts
// its tiles into work items of at most `chunk` tiles, written at a range it
// reserves from a counter; the last CTA to finish publishes the item count.
// (Same selection rule as timemachine/cpp/src/kernels/k_neighborlist.cuh:168-427,
// which uses 32-atom row blocks.)
// ---------------------------------------------------------------------------
struct TileArgs {
    int S;
    int RB;           // blocks of 32 slots = ceil(S/32) (column blocks)
    int rows;         // slots per row group: 32, 16 or 8
    int group;        // 1: interaction group (rows [0, row_end) x columns [col_begin, S))
    int row_end;      // S, or the number of row atoms
    int col_begin;    // 0, or the number of row atoms
    int n_row_blocks; // row groups: ceil(row_end/rows)
    int cb_first;     // group: first column block (col_begin/32)
    float radius;     // list radius (cutoff + padding + margin)
    const double *box;
    const float4 *posw;
    const float4 *prm;     // staged parameters (eps in .z) to put LJ atoms first in a tile; nullptr: keep order
    const float4 *bb_ctr;
    const float4 *bb_ext;
    unsigned *tile_cols;   // [capacity*32] slot of each column atom (S = empty)
    int *rb_ntiles;        // [n_row_blocks] tiles of each row group
    int4 *items;           // [item_capacity] (row group, first tile, tile count, 0)
    int chunk;             // tiles per work item
};

__host__ __device__ __forceinline__ long long tile_offset(int rb, int RB) {
    return (long long)rb * RB - ((long long)rb * (rb - 1)) / 2;
}

// First tile of row group g. Upper triangle: the group reaches the RB - b
// column blocks from its own block b = g*rows/32 on, one tile per block at
// most; with m = 32/rows groups per block that sums to
// m * tile_offset(b, RB) + (g mod m) * (RB - b). Interaction group:
// RB - cb_first tiles per row group.
__host__ __device__ __forceinline__ long long tile_base_rows(int g, int rows, int RB, int group, int cb_first) {
    if (group) {
        return (long long)g * (RB - cb_first);
    }
    const int m = TILE / rows;
    const int b = g / m;
    return (long long)m * tile_offset(b, RB) + (long long)(g - b * m) * (RB - b);
}
__host__ __device__ __forceinline__ long long tile_base(const TileArgs &a, int g) {
    return tile_base_rows(g, a.rows, a.RB, a.group, a.cb_first);
}

constexpr int TB_WARPS = 8;
// Tile-build CTAs per SM the compiler must fit (40 registers). The packed row
// tests left to the compiler take 57 registers (4 CTAs/SM): measured on B200,
// one rebuild 87.3 us with the scalar tests, 90.0 us packed at 57 registers,
// 81.3 us packed at 40.
#ifndef TMNB_TB_CTAS
#define TMNB_TB_CTAS 6
#endif

__device__ __forceinline__ void build_tiles_cta(const TileArgs &a, const int rb, DevState *state) {
    __shared__ float4 row_pos[TILE];
    // the same positions as x, y, z arrays: element pair m holds rows 2m, 2m + 1
    __shared__ __align__(8) float row_x[TILE];
    __shared__ __align__(8) float row_y[TILE];
    __shared__ __align__(8) float row_z[TILE];
    __shared__ float4 row_box[2]; // the row group's box: centre, half-extent
    __shared__ unsigned buf[TB_WARPS][2 * TILE];
    __shared__ unsigned rem[TB_WARPS * TILE];
    __shared__ int cand[TB_WARPS * 32]; // column blocks of the current window that pass the box test
    __shared__ int warp_pass[TB_WARPS];
    __shared__ int tile_count;
    __shared__ int rem_count;
    __shared__ int is_last;

    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int S = a.S;
    const float Lx = (float)a.box[0], Ly = (float)a.box[4], Lz = (float)a.box[8];
    const float iLx = 1.0f / Lx, iLy = 1.0f / Ly, iLz = 1.0f / Lz;
    const float r2 = a.radius * a.radius;
    const float r2_box = (a.radius + 1e-4f) * (a.radius + 1e-4f);
    const int rows = a.rows;
    const int row_first = rb * rows;
    const int row_n = min(rows, a.row_end - row_first);
    if (warp == 0) {
        // the row group's box, as block_bounds_warp computes a 32-slot block's
        const bool valid = lane < row_n;
        const float4 p = valid ? a.posw[row_first + lane] : make_float4(0.f, 0.f, 0.f, 0.f);
        const float rx = __shfl_sync(FULL_MASK, p.x, 0);
        const float ry = __shfl_sync(FULL_MASK, p.y, 0);
        const float rz = __shfl_sync(FULL_MASK, p.z, 0);
        const float dx = wrap_delta(p.x - rx, Lx, iLx);
        const float dy = wrap_delta(p.y - ry, Ly, iLy);
        const float dz = wrap_delta(p.z - rz, Lz, iLz);
        float mnx = valid ? dx : 3.0e38f, mny = valid ? dy : 3.0e38f, mnz = valid ? dz : 3.0e38f;
        float mxx = valid ? dx : -3.0e38f, mxy = valid ? dy : -3.0e38f, mxz = valid ? dz : -3.0e38f;
        for (int o = 16; o > 0; o >>= 1) {
            mnx = fminf(mnx, __shfl_xor_sync(FULL_MASK, mnx, o));
            mny = fminf(mny, __shfl_xor_sync(FULL_MASK, mny, o));
            mnz = fminf(mnz, __shfl_xor_sync(FULL_MASK, mnz, o));
            mxx = fmaxf(mxx, __shfl_xor_sync(FULL_MASK, mxx, o));
            mxy = fmaxf(mxy, __shfl_xor_sync(FULL_MASK, mxy, o));
            mxz = fmaxf(mxz, __shfl_xor_sync(FULL_MASK, mxz, o));
        }
        if (lane == 0) {
            row_box[0] = make_float4(rx + 0.5f * (mnx + mxx), ry + 0.5f * (mny + mxy), rz + 0.5f * (mnz + mxz), 0.f);
            row_box[1] = make_float4(
                0.5f * (mxx - mnx) * 1.000001f + 1e-6f, 0.5f * (mxy - mny) * 1.000001f + 1e-6f,
                0.5f * (mxz - mnz) * 1.000001f + 1e-6f, 0.f);
        }
    }
    __syncthreads();
    const float4 rc = row_box[0];
    const float4 re = row_box[1];

    // Row atoms are imaged next to the row block's centre. When every box
    // edge satisfies L/2 - extent >= radius, a column atom imaged next to the
    // centre (once) is at its minimum image from every row atom whenever that
    // distance is below the radius, so the per-pair test needs no wrapping.
    const bool shifted = 0.5f * Lx - re.x >= a.radius + 1e-3f && 0.5f * Ly - re.y >= a.radius + 1e-3f &&
                         0.5f * Lz - re.z >= a.radius + 1e-3f;
    if (threadIdx.x < rows) {
        const int s = row_first + threadIdx.x;
        float4 p = s < a.row_end ? a.posw[s] : make_float4(rc.x, rc.y, rc.z, 0.f);
        p.x = rc.x + wrap_delta(p.x - rc.x, Lx, iLx);
        p.y = rc.y + wrap_delta(p.y - rc.y, Ly, iLy);
        p.z = rc.z + wrap_delta(p.z - rc.z, Lz, iLz);
        row_pos[threadIdx.x] = p;
        row_x[threadIdx.x] = p.x;
        row_y[threadIdx.x] = p.y;
        row_z[threadIdx.x] = p.z;
    }
    if (threadIdx.x == 0) {
        tile_count = 0;
        rem_count = 0;
    }
    __syncthreads();
    const int col_lo = a.group ? a.col_begin : row_first; // first column slot of the group's pairs
    const long long base_tile = tile_base(a, rb);
    const unsigned lane_lt = (1u << lane) - 1;

    int count = 0; // atoms in this warp's buffer
    // Column blocks in windows of one block per thread: the box test of the
    // window compacts the passing blocks in index order, then each warp takes
    // an equal contiguous share of them. Passing blocks cluster at nearby
    // indices, so a fixed split of the window by index would leave most warps
    // idle; contiguous shares keep each warp's tiles spatially compact (the
    // slot order is a space-filling curve), which the pair kernel's
    // divergence depends on.
    for (int wbase = a.group ? a.cb_first : row_first / TILE; wbase < a.RB; wbase += TB_WARPS * 32) {
        const int cb = wbase + (int)threadIdx.x;
        bool pass = false;
        if (cb < a.RB) {
            const float4 cc = a.bb_ctr[cb];
            const float4 ce = a.bb_ext[cb];
            float dx = fmaxf(0.f, fabsf(wrap_delta(rc.x - cc.x, Lx, iLx)) - re.x - ce.x);
            float dy = fmaxf(0.f, fabsf(wrap_delta(rc.y - cc.y, Ly, iLy)) - re.y - ce.y);
            float dz = fmaxf(0.f, fabsf(wrap_delta(rc.z - cc.z, Lz, iLz)) - re.z - ce.z);
            pass = dx * dx + dy * dy + dz * dz < r2;
        }
        const unsigned m = __ballot_sync(FULL_MASK, pass);
        if (lane == 0) {
            warp_pass[warp] = __popc(m);
        }
        __syncthreads();
        int base = 0, nc = 0;
        for (int w = 0; w < TB_WARPS; w++) {
            const int c = warp_pass[w];
            base += w < warp ? c : 0;
            nc += c;
        }
        if (pass) {
            cand[base + __popc(m & lane_lt)] = cb;
        }
        __syncthreads();
        const int k_end = ((warp + 1) * nc) / TB_WARPS;
        for (int k = (warp * nc) / TB_WARPS; k < k_end; k++) {
            const int cb_sel = cand[k];
            const int s = cb_sel * TILE + lane;
            const bool valid = s < S;
            const float4 pj = valid ? a.posw[s] : make_float4(0.f, 0.f, 0.f, 0.f);
            // an atom farther than the radius from the row block's box is
            // farther than the radius from every row atom (widened test,
            // conservative under rounding): skip its per-row test
            const float wx = wrap_delta(pj.x - rc.x, Lx, iLx);
            const float wy = wrap_delta(pj.y - rc.y, Ly, iLy);
            const float wz = wrap_delta(pj.z - rc.z, Lz, iLz);
            const float bx = fmaxf(0.f, fabsf(wx) - re.x);
            const float by = fmaxf(0.f, fabsf(wy) - re.y);
            const float bz = fmaxf(0.f, fabsf(wz) - re.z);
            const bool need = valid && s >= col_lo && bx * bx + by * by + bz * bz < r2_box;
            bool hit = false;
            if (__any_sync(FULL_MASK, need)) {
                if (shifted) {
                    // two rows per packed FP32x2 test (rows past row_n sit at
                    // the centre and are masked)
                    const float2 qx = f2(rc.x + wx), qy = f2(rc.y + wy), qz = f2(rc.z + wz);
                    const float2 *rx2 = reinterpret_cast<const float2 *>(row_x);
                    const float2 *ry2 = reinterpret_cast<const float2 *>(row_y);
                    const float2 *rz2 = reinterpret_cast<const float2 *>(row_z);
                    for (int r0 = 0; r0 < row_n; r0 += 8) {
#pragma unroll
                        for (int r = r0; r < r0 + 8; r += 2) {
                            const float2 dx = fsub2(rx2[r >> 1], qx);
                            const float2 dy = fsub2(ry2[r >> 1], qy);
                            const float2 dz = fsub2(rz2[r >> 1], qz);
                            const float2 d2 = ffma2(dz, dz, ffma2(dy, dy, fmul2(dx, dx)));
                            hit |= ((r < row_n) && (d2.x < r2)) || ((r + 1 < row_n) && (d2.y < r2));
                        }
                        if (__all_sync(FULL_MASK, hit || !need)) {
                            break;
                        }
                    }
                } else {
                    // rows in groups of 8 (independent tests, then one vote)
                    for (int r0 = 0; r0 < row_n; r0 += 8) {
#pragma unroll
                        for (int r = r0; r < r0 + 8; r++) {
                            const float4 pi = row_pos[r];
                            const float dx = wrap_delta(pi.x - pj.x, Lx, iLx);
                            const float dy = wrap_delta(pi.y - pj.y, Ly, iLy);
                            const float dz = wrap_delta(pi.z - pj.z, Lz, iLz);
                            hit |= (r < row_n) && (dx * dx + dy * dy + dz * dz < r2);
                        }
                        if (__all_sync(FULL_MASK, hit || !need)) {
                            break;
                        }
                    }
                }
            }
            hit = hit && need;
            const unsigned hmask = __ballot_sync(FULL_MASK, hit);
            if (hit) {
                buf[warp][count + __popc(hmask & lane_lt)] = (unsigned)s;
            }
            count += __popc(hmask);
            __syncwarp();
            if (count >= TILE) {
                int t = 0;
                if (lane == 0) {
                    t = atomicAdd(&tile_count, 1);
                }
                t = __shfl_sync(FULL_MASK, t, 0);
                store_tile_lj_first(a.tile_cols + (base_tile + t) * TILE, buf[warp][lane], (unsigned)S, a.prm);
                __syncwarp();
                buf[warp][lane] = buf[warp][TILE + lane];
                __syncwarp();
                count -= TILE;
            }
        }
        __syncthreads(); // cand / warp_pass are rewritten by the next window
    }
    // merge the partial buffers of the warps
    int off = 0;
    if (lane == 0) {
        off = atomicAdd(&rem_count, count);
    }
    off = __shfl_sync(FULL_MASK, off, 0);
    if (lane < count) {
        rem[off + lane] = buf[warp][lane];
    }
    __syncthreads();
    if (warp == 0) {
        const int n = rem_count;
        for (int b = 0; b < n; b += TILE) {
            const int t = tile_count + b / TILE;
            store_tile_lj_first(a.tile_cols + (base_tile + t) * TILE, b + lane < n ? rem[b + lane] : (unsigned)S,
                                (unsigned)S, a.prm);
        }
        __syncwarp();
        const int total = tile_count + (n + TILE - 1) / TILE;
        // the group's work items, at a range reserved from the list's
        // counter (items are in any order: the pair kernel schedules them
        // dynamically and its sums do not depend on the order)
        const int ni = (total + a.chunk - 1) / a.chunk;
        int first_item = 0;
        if (lane == 0) {
            a.rb_ntiles[rb] = total;
            atomicAdd(&state->total_tiles, (unsigned)total);
            first_item = atomicAdd(&state->item_count, ni);
        }
        first_item = __shfl_sync(FULL_MASK, first_item, 0);
        const long long first_tile = tile_base(a, rb);
        for (int c = lane; c < ni; c += TILE) {
            const int first = c * a.chunk;
            a.items[first_item + c] = make_int4(rb, (int)(first_tile + first), min(a.chunk, total - first), 0);
        }
    }
    // the last CTA to finish publishes the list
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) {
        const unsigned prev = atomicAdd(&state->done_ctas, 1u);
        is_last = (prev == (unsigned)a.n_row_blocks - 1);
    }
    __syncthreads();
    if (!is_last) {
        return;
    }
    if (threadIdx.x == 0) {
        __threadfence();
        state->n_items = *((volatile int *)&state->item_count);
        state->item_count = 0;
        state->items_chunk = a.chunk;
        state->dep_dirty = 1; // the lambda-dependent tiles follow the new list
        state->n_dep = 0;
        state->rebuilds += 1;
        state->done_ctas = 0;
        state->rebuild = 0;
    }
}

static __global__ void __launch_bounds__(TB_WARPS * 32, TMNB_TB_CTAS) k_build_tiles(TileArgs a, DevState *state) {
    grid_dependency_wait();
    if (!state->rebuild || state->error) {
        return;
    }
    build_tiles_cta(a, blockIdx.x, state);
}

// Clears the rebuild flag when no neighbour list exists (pair lists only).
static __global__ void k_clear_rebuild(DevState *state) { state->rebuild = 0; }

// ---------------------------------------------------------------------------
// Pair kernel.
// ---------------------------------------------------------------------------
struct Accum {
    unsigned long long *x, *y, *z;       // du_dx [S] each
    unsigned long long *q, *sig, *eps;   // du_dp [S] each
    unsigned long long *u, *dl;          // per-slot energy and du_dl [S]
    unsigned long long *pq, *psig, *peps; // du_dp of the scaled-pair part (interpolated), else == q/sig/eps
};

// Accumulator block b (0: contributions shared by all windows, 1 + k: window k)
// lies `block` elements after block 0.
__device__ __forceinline__ Accum acc_block(const Accum &a, size_t block, int b) {
    const size_t o = block * (size_t)b;
    Accum r;
    r.x = a.x + o;
    r.y = a.y + o;
    r.z = a.z + o;
    r.q = a.q + o;
    r.sig = a.sig + o;
    r.eps = a.eps + o;
    r.u = a.u + o;
    r.dl = a.dl + o;
    r.pq = a.pq + o;
    r.psig = a.psig + o;
    r.peps = a.peps + o;
    return r;
}

struct PairArgs {
    int S;
    int row_end;                // slots [0, row_end) act as rows (S, or the interaction group's rows)
    int K;                      // lambda windows
    const float4 *posw;         // [K][S]
    const float4 *prm;          // [K][S]
    const float4 *dprm;         // [K][S]
    const unsigned char *lamdep; // [S]
    const double4 *posw64;      // [K][S] FP64 pair arithmetic (else nullptr)
    const double4 *prm64;       // [K][S]
    const double4 *dprm64;      // [K][S]
    const double *box;
    double beta;
    double cutoff;
    const unsigned *tile_cols;
    const int4 *items;
    // scaled pairs (exclusions / 1-4): original atom indices and scales
    int M;
    const int *pair_idxs;  // [M,2]
    const double *scales;  // [M,2]
    const int *slot_of;    // [N] atom -> slot, nullptr: identity
    int negated;
    Accum acc;             // block 0
    size_t acc_block;      // elements between accumulator blocks
    const int2 *dep_tiles; // [n_dep] (row group, tile) of the lambda-dependent tiles (multi-window)
    DevState *state;
};

__device__ __forceinline__ void red_add(unsigned long long *p, unsigned long long v) { atomicAdd(p, v); }

// The staged slot arrays the pair arithmetic of type Real reads: FP32 float4
// or FP64 double4 copies of the same values.
template <typename Real> struct Staged;
template <> struct Staged<float> {
    using V = float4;
    static __device__ __forceinline__ const float4 *posw(const PairArgs &a) { return a.posw; }
    static __device__ __forceinline__ const float4 *prm(const PairArgs &a) { return a.prm; }
    static __device__ __forceinline__ const float4 *dprm(const PairArgs &a) { return a.dprm; }
    static __device__ __forceinline__ float4 make(float x, float y, float z, float w) { return make_float4(x, y, z, w); }
};
template <> struct Staged<double> {
    using V = double4;
    static __device__ __forceinline__ const double4 *posw(const PairArgs &a) { return a.posw64; }
    static __device__ __forceinline__ const double4 *prm(const PairArgs &a) { return a.prm64; }
    static __device__ __forceinline__ const double4 *dprm(const PairArgs &a) { return a.dprm64; }
    static __device__ __forceinline__ double4 make(double x, double y, double z, double w) {
        return make_double4(x, y, z, w);
    }
};

// The arithmetic of one in-range pair (row atom i, column atom j) from its
// minimum-image deltas and 4D d2: adds the row's and the column's fixed-point
// contributions. Every sweep calls this one function, so a pair rounds the
// same whichever schedule evaluates it. Per-pair arithmetic and validity follow
// timemachine/cpp/src/kernels/k_nonbonded.cuh:424-546; the column
// contribution of du_dx is the exact negation of the row contribution
// (llrint is odd under round-half-even), so it is converted once.
template <typename Real, bool U, bool DX, bool DL, bool DP, bool INTERP, bool ALCH>
__device__ __forceinline__ void pair_terms(
    const Real delta_x,
    const Real delta_y,
    const Real delta_z,
    const Real delta_w,
    const Real d2,
    const Real qi,
    const Real sig_i,
    const Real eps_i,
    const Real dw_dl_i,
    const Real dq_dl_i,
    const Real dsig_dl_i,
    const Real deps_dl_i,
    const Real qj,
    const Real sig_j,
    const Real eps_j,
    const Real dw_dl_j,
    const Real dq_dl_j,
    const Real dsig_dl_j,
    const Real deps_dl_j,
    const Real beta,
    unsigned long long &gi_x,
    unsigned long long &gi_y,
    unsigned long long &gi_z,
    unsigned long long &g_qi,
    unsigned long long &g_sigi,
    unsigned long long &g_epsi,
    unsigned long long &du_dl,
    unsigned long long &energy,
    unsigned long long &gj_x,
    unsigned long long &gj_y,
    unsigned long long &gj_z,
    unsigned long long &g_qj,
    unsigned long long &g_sigj,
    unsigned long long &g_epsj) {
    Real u;
    Real prefactor;
    Real erfc_bd;
    Real d;
    Real inv_d;
    Real inv_d2;
    Real qij_inv;
    Real factor;
    electrostatics<Real, U>((Real)1, qi, qj, d2, beta, d, inv_d, inv_d2, erfc_bd, prefactor, u, qij_inv, factor);
    Real real_du_dl = 0;
    if (eps_i != 0 && eps_j != 0) {
        Real sig_grad;
        Real eps_grad;
        lennard_jones<Real, U>(
            (Real)1, eps_i, eps_j, sig_i, sig_j, inv_d, inv_d2, qij_inv, factor, erfc_bd, u, prefactor, sig_grad,
            eps_grad);
        if (DP) {
            const unsigned long long gs = to_fixed(sig_grad, FX_EXPONENT_SIG);
            g_sigi += gs;
            g_sigj += gs;
            if constexpr (TMNB_PACKED_SCALAR && sizeof(Real) == 4) {
                const float2 ge = fmul2(fmul2(f2(eps_grad), make_float2(eps_j, eps_i)),
                                        f2(static_cast<float>(FX_EXPONENT_EPS)));
                g_epsi += fixed_round(ge.x);
                g_epsj += fixed_round(ge.y);
            } else {
                g_epsi += to_fixed(fmul(eps_grad, eps_j), FX_EXPONENT_EPS);
                g_epsj += to_fixed(fmul(eps_grad, eps_i), FX_EXPONENT_EPS);
            }
        }
        if (DL && ALCH && INTERP) {
            real_du_dl = ffma(sig_grad, fadd(dsig_dl_i, dsig_dl_j), real_du_dl);
            real_du_dl = ffma(eps_grad, sum_of_products_rn(eps_j, deps_dl_i, eps_i, deps_dl_j), real_du_dl);
        }
    }
    if (DX) {
        // The column's term llrint(-y) equals -llrint(y) (round-half-even is
        // odd) except where the conversion saturates (|y| >= 2^63) or y is NaN;
        // those lanes add the difference afterwards.
        const Real ex = static_cast<Real>(FX_EXPONENT);
        Real yx, yy;
        if constexpr (TMNB_PACKED_SCALAR && sizeof(Real) == 4) {
            const float2 yxy = fmul2(fmul2(f2(prefactor), make_float2(delta_x, delta_y)), f2(ex));
            yx = yxy.x;
            yy = yxy.y;
        } else {
            yx = fmul(fmul(prefactor, delta_x), ex);
            yy = fmul(fmul(prefactor, delta_y), ex);
        }
        const Real yz = fmul(fmul(prefactor, delta_z), ex);
        const unsigned long long fx = fixed_round(yx);
        const unsigned long long fy = fixed_round(yy);
        const unsigned long long fz = fixed_round(yz);
        gi_x += fx;
        gi_y += fy;
        gi_z += fz;
        gj_x -= fx;
        gj_y -= fy;
        gj_z -= fz;
        if (!fixed_in_range(yx) || !fixed_in_range(yy) || !fixed_in_range(yz)) {
            gj_x += fixed_round(-yx) + fx;
            gj_y += fixed_round(-yy) + fy;
            gj_z += fixed_round(-yz) + fz;
        }
    }
    if (DP) {
        if constexpr (TMNB_PACKED_SCALAR && sizeof(Real) == 4) {
            const float2 gq = fmul2(fmul2(fmul2(make_float2(qj, qi), f2(inv_d)), f2(erfc_bd)),
                                    f2(static_cast<float>(FX_EXPONENT)));
            g_qi += fixed_round(gq.x);
            g_qj += fixed_round(gq.y);
        } else {
            g_qi += to_fixed(fmul(fmul(qj, inv_d), erfc_bd), FX_EXPONENT);
            g_qj += to_fixed(fmul(fmul(qi, inv_d), erfc_bd), FX_EXPONENT);
        }
    }
    if (DL && ALCH) {
        real_du_dl = ffma(fmul(delta_w, prefactor), fsub(dw_dl_i, dw_dl_j), real_du_dl);
        if (INTERP) {
            real_du_dl = ffma(fmul(inv_d, erfc_bd), sum_of_products_rn(qj, dq_dl_i, qi, dq_dl_j), real_du_dl);
        }
        du_dl += to_fixed(real_du_dl, FX_EXPONENT);
    }
    if (U) {
        energy += to_fixed(u, FX_EXPONENT);
    }
}

// One tile of RG rows x 32 columns: lane l owns row slot i (row l mod RG);
// the column atoms rotate through the lanes of each RG-lane group by one
// position per round (RG rounds), carrying their accumulators.
// Per-pair arithmetic and validity follow
// timemachine/cpp/src/kernels/k_nonbonded.cuh:424-546; the column
// contribution of du_dx is the exact negation of the row contribution
// (llrint is odd under round-half-even), so it is converted once.
template <typename Real, bool U, bool DX, bool DL, bool DP, bool INTERP, bool ALCH, bool CHECK, int RG = TILE>
__device__ __forceinline__ void sweep_tile(
    const int lane,
    const unsigned S,
    const unsigned i,
    unsigned j,
    const Real ci_x,
    const Real ci_y,
    const Real ci_z,
    const Real ci_w,
    const Real qi,
    const Real sig_i,
    const Real eps_i,
    const Real dw_dl_i,
    const Real dq_dl_i,
    const Real dsig_dl_i,
    const Real deps_dl_i,
    Real cj_x,
    Real cj_y,
    Real cj_z,
    Real cj_w,
    Real qj,
    Real sig_j,
    Real eps_j,
    Real dw_dl_j,
    Real dq_dl_j,
    Real dsig_dl_j,
    Real deps_dl_j,
    const Real box_x,
    const Real box_y,
    const Real box_z,
    const Real inv_box_x,
    const Real inv_box_y,
    const Real inv_box_z,
    const Real cutoff_squared,
    const Real beta,
    unsigned long long &gi_x,
    unsigned long long &gi_y,
    unsigned long long &gi_z,
    unsigned long long &g_qi,
    unsigned long long &g_sigi,
    unsigned long long &g_epsi,
    unsigned long long &du_dl,
    unsigned long long &energy,
    unsigned long long &gj_x,
    unsigned long long &gj_y,
    unsigned long long &gj_z,
    unsigned long long &g_qj,
    unsigned long long &g_sigj,
    unsigned long long &g_epsj) {
    // rows of RG < 32 slots: the warp is 32/RG lane groups, each sweeping RG
    // of the tile's columns against the RG rows (lane l holds row l mod RG), so
    // the columns rotate inside their lane group and a tile takes RG rounds
    const int src = (lane & ~(RG - 1)) | ((lane + 1) & (RG - 1));
    // measured on B200: 4 rounds per iteration for the force-only variant,
    // no unrolling for the variants with more outputs (register pressure)
    constexpr int UNROLL = (DX && !U && !DL && !DP) ? 4 : 1;
#pragma unroll UNROLL
    for (int round = 0; round < RG; round++) {
        Real delta_x, delta_y;
        if constexpr (TMNB_PACKED_SCALAR && sizeof(Real) == 4) {
            // x and y in the two components of one packed operation each
            const float2 dxy = min_image2(
                fsub2(make_float2(ci_x, ci_y), make_float2(cj_x, cj_y)), make_float2(-box_x, -box_y),
                make_float2(inv_box_x, inv_box_y));
            delta_x = dxy.x;
            delta_y = dxy.y;
        } else {
            delta_x = min_image(fsub(ci_x, cj_x), box_x, inv_box_x);
            delta_y = min_image(fsub(ci_y, cj_y), box_y, inv_box_y);
        }
        const Real delta_z = min_image(fsub(ci_z, cj_z), box_z, inv_box_z);
        Real d2 = dist2(delta_x, delta_y, delta_z);
        Real delta_w;
        if (ALCH) {
            delta_w = fsub(ci_w, cj_w);
            d2 = add_w2(d2, delta_w);
        }
        // CHECK: the tile holds atoms of the row group itself, so i < j decides
        // which lane evaluates each pair. Otherwise every column slot exceeds
        // every row slot, and padding rows/columns carry NaN coordinates,
        // which fail the cutoff test.
        const bool valid = !CHECK || (i < S && j < S && i < j);
        if (valid && d2 < cutoff_squared) {
            pair_terms<Real, U, DX, DL, DP, INTERP, ALCH>(
                delta_x, delta_y, delta_z, ALCH ? delta_w : (Real)0, d2, qi, sig_i, eps_i, dw_dl_i, dq_dl_i, dsig_dl_i,
                deps_dl_i, qj, sig_j, eps_j, dw_dl_j, dq_dl_j, dsig_dl_j, deps_dl_j, beta, gi_x, gi_y, gi_z, g_qi,
                g_sigi, g_epsi, du_dl, energy, gj_x, gj_y, gj_z, g_qj, g_sigj, g_epsj);
        }
        if (CHECK) {
            j = __shfl_sync(FULL_MASK, j, src);
        }
        qj = __shfl_sync(FULL_MASK, qj, src);
        eps_j = __shfl_sync(FULL_MASK, eps_j, src);
        sig_j = __shfl_sync(FULL_MASK, sig_j, src);
        cj_x = __shfl_sync(FULL_MASK, cj_x, src);
        cj_y = __shfl_sync(FULL_MASK, cj_y, src);
        cj_z = __shfl_sync(FULL_MASK, cj_z, src);
        if (ALCH) {
            cj_w = __shfl_sync(FULL_MASK, cj_w, src);
            dw_dl_j = __shfl_sync(FULL_MASK, dw_dl_j, src);
        }
        if (DX) {
            gj_x = __shfl_sync(FULL_MASK, gj_x, src);
            gj_y = __shfl_sync(FULL_MASK, gj_y, src);
            gj_z = __shfl_sync(FULL_MASK, gj_z, src);
        }
        if (DP) {
            g_qj = __shfl_sync(FULL_MASK, g_qj, src);
            g_sigj = __shfl_sync(FULL_MASK, g_sigj, src);
            g_epsj = __shfl_sync(FULL_MASK, g_epsj, src);
        }
        if (DL && ALCH && INTERP) {
            dsig_dl_j = __shfl_sync(FULL_MASK, dsig_dl_j, src);
            deps_dl_j = __shfl_sync(FULL_MASK, deps_dl_j, src);
            dq_dl_j = __shfl_sync(FULL_MASK, dq_dl_j, src);
        }
    }
}

// One scaled pair (exclusion / 1-4 correction), arithmetic of
// timemachine/cpp/src/kernels/k_nonbonded_pair_list.cuh:103-215.
template <typename Real, bool U, bool DX, bool DL, bool DP, bool INTERP>
__device__ __forceinline__ void scaled_pair(
    const PairArgs &a,
    int pair,
    int si,
    int sj,
    int window,
    const Accum &acc_out,
    const Real box_x,
    const Real box_y,
    const Real box_z,
    const Real inv_box_x,
    const Real inv_box_y,
    const Real inv_box_z,
    const Real cutoff_squared) {
    using St = Staged<Real>;
    const size_t wo = (size_t)window * a.S;
    const typename St::V pwi = St::posw(a)[wo + si];
    const typename St::V pwj = St::posw(a)[wo + sj];
    const typename St::V pri = St::prm(a)[wo + si];
    const typename St::V prj = St::prm(a)[wo + sj];
    typename St::V dpi = St::make(0, 0, 0, 0);
    typename St::V dpj = dpi;
    if (INTERP) {
        dpi = St::dprm(a)[wo + si];
        dpj = St::dprm(a)[wo + sj];
    }
    const Real ci_x = pwi.x, ci_y = pwi.y, ci_z = pwi.z, ci_w = pwi.w;
    const Real cj_x = pwj.x, cj_y = pwj.y, cj_z = pwj.z, cj_w = pwj.w;
    const Real qi = pri.x, sig_i = pri.y, eps_i = pri.z, dw_dl_i = pri.w;
    const Real qj = prj.x, sig_j = prj.y, eps_j = prj.z, dw_dl_j = prj.w;
    const Real dq_dl_i = dpi.x, dsig_dl_i = dpi.y, deps_dl_i = dpi.z;
    const Real dq_dl_j = dpj.x, dsig_dl_j = dpj.y, deps_dl_j = dpj.z;
    const Real beta = a.beta;
    const Real charge_scale = a.scales[2 * pair + 0];
    const Real lj_scale = a.scales[2 * pair + 1];

    Real delta_x = fsub(ci_x, cj_x);
    Real delta_y = fsub(ci_y, cj_y);
    Real delta_z = fsub(ci_z, cj_z);
    delta_x = min_image(delta_x, box_x, inv_box_x);
    delta_y = min_image(delta_y, box_y, inv_box_y);
    delta_z = min_image(delta_z, box_z, inv_box_z);
    const Real delta_w = fsub(ci_w, cj_w);
    const Real d2 = add_w2(dist2(delta_x, delta_y, delta_z), delta_w);

    const bool is_vanilla = (ci_w == 0 && dq_dl_i == 0 && dsig_dl_i == 0 && deps_dl_i == 0 && cj_w == 0 &&
                             dq_dl_j == 0 && dsig_dl_j == 0 && deps_dl_j == 0);
    if (!(d2 < cutoff_squared)) {
        return;
    }
    Real u;
    Real erfc_bd;
    Real prefactor;
    Real d;
    Real inv_d;
    Real inv_d2;
    Real qij_inv;
    Real factor;
    electrostatics<Real, true>(
        charge_scale, qi, qj, d2, beta, d, inv_d, inv_d2, erfc_bd, prefactor, u, qij_inv, factor);
    Real real_du_dl = 0;
    unsigned long long g_sig = 0, g_epsi = 0, g_epsj = 0;
    if (eps_i != 0 && eps_j != 0) {
        Real sig_grad;
        Real eps_grad;
        lennard_jones<Real, true>(
            lj_scale, eps_i, eps_j, sig_i, sig_j, inv_d, inv_d2, qij_inv, factor, erfc_bd, u, prefactor, sig_grad,
            eps_grad);
        g_sig = to_fixed(sig_grad, FX_EXPONENT_SIG);
        g_epsi = to_fixed(fmul(eps_grad, eps_j), FX_EXPONENT_EPS);
        g_epsj = to_fixed(fmul(eps_grad, eps_i), FX_EXPONENT_EPS);
        if (INTERP) {
            real_du_dl = ffma(sig_grad, fadd(dsig_dl_i, dsig_dl_j), real_du_dl);
            real_du_dl = ffma(eps_grad, sum_of_products_rn(eps_j, deps_dl_i, eps_i, deps_dl_j), real_du_dl);
        }
    }
    const bool neg = a.negated != 0;
    auto acc = [neg](unsigned long long *p, unsigned long long v) { red_add(p, neg ? (0ULL - v) : v); };
    if (DX) {
        unsigned long long fx, fy, fz, nx, ny, nz;
        to_fixed_pair(fmul(prefactor, delta_x), FX_EXPONENT, fx, nx);
        to_fixed_pair(fmul(prefactor, delta_y), FX_EXPONENT, fy, ny);
        to_fixed_pair(fmul(prefactor, delta_z), FX_EXPONENT, fz, nz);
        acc(acc_out.x + si, fx);
        acc(acc_out.y + si, fy);
        acc(acc_out.z + si, fz);
        acc(acc_out.x + sj, nx);
        acc(acc_out.y + sj, ny);
        acc(acc_out.z + sj, nz);
    }
    if (DP) {
        acc(acc_out.pq + si, to_fixed(fmul(fmul(fmul(charge_scale, qj), inv_d), erfc_bd), FX_EXPONENT));
        acc(acc_out.pq + sj, to_fixed(fmul(fmul(fmul(charge_scale, qi), inv_d), erfc_bd), FX_EXPONENT));
        acc(acc_out.psig + si, g_sig);
        acc(acc_out.peps + si, g_epsi);
        acc(acc_out.psig + sj, g_sig);
        acc(acc_out.peps + sj, g_epsj);
    }
    if (DL && !is_vanilla) {
        real_du_dl = ffma(fmul(delta_w, prefactor), fsub(dw_dl_i, dw_dl_j), real_du_dl);
        if (INTERP) {
            real_du_dl = ffma(
                fmul(fmul(charge_scale, inv_d), erfc_bd), sum_of_products_rn(qj, dq_dl_i, qi, dq_dl_j), real_du_dl);
        }
        acc(acc_out.dl + si, to_fixed(real_du_dl, FX_EXPONENT));
    }
    if (U) {
        acc(acc_out.u + si, to_fixed(u, FX_EXPONENT));
    }
}

// One tile of a row group's rows (lane: row slot i) against the 32 column slots
// j, for one window: load, sweep, column atomics. Row accumulators are
// returned to the caller.
template <typename Real, bool U, bool DX, bool DL, bool DP, bool INTERP, int RG = TILE>
__device__ __forceinline__ void tile_pass(
    const PairArgs &a,
    const int lane,
    const unsigned S,
    const unsigned i,
    const unsigned j,
    const int window,
    const Accum &acc_out,
    const Real box_x,
    const Real box_y,
    const Real box_z,
    const Real inv_box_x,
    const Real inv_box_y,
    const Real inv_box_z,
    const Real cutoff_squared,
    const Real beta,
    unsigned long long &gi_x,
    unsigned long long &gi_y,
    unsigned long long &gi_z,
    unsigned long long &g_qi,
    unsigned long long &g_sigi,
    unsigned long long &g_epsi,
    unsigned long long &du_dl,
    unsigned long long &energy) {
    using St = Staged<Real>;
    using V = typename St::V;
    const size_t wo = (size_t)window * a.S;
    const bool row_ok = i < (unsigned)a.row_end;
    const bool col_ok = j < S;
    const unsigned i_eff = row_ok ? i : 0xffffffffu; // invalid rows pair with nothing
    // padding rows and columns: NaN coordinates (no pair passes the cutoff test), w = 0
    const Real nan = static_cast<Real>(__int_as_float(0x7fffffff));
    const V pwi = row_ok ? St::posw(a)[wo + i] : St::make(nan, nan, nan, 0);
    const V pri = row_ok ? St::prm(a)[wo + i] : St::make(0, 0, 0, 0);
    const V pwj = col_ok ? St::posw(a)[wo + j] : St::make(nan, nan, nan, 0);
    const V prj = col_ok ? St::prm(a)[wo + j] : St::make(0, 0, 0, 0);
    V dpi = St::make(0, 0, 0, 0);
    V dpj = dpi;
    if (INTERP) {
        if (row_ok) {
            dpi = St::dprm(a)[wo + i];
        }
        if (col_ok) {
            dpj = St::dprm(a)[wo + j];
        }
    }
    const bool row_alch = pwi.w != 0 || (INTERP && (dpi.x != 0 || dpi.y != 0 || dpi.z != 0));
    const bool col_alch = pwj.w != 0 || (INTERP && (dpj.x != 0 || dpj.y != 0 || dpj.z != 0));
    const bool alch = __any_sync(FULL_MASK, row_alch || col_alch);
    unsigned long long gj_x = 0, gj_y = 0, gj_z = 0, g_qj = 0, g_sigj = 0, g_epsj = 0;
    // Only a tile holding atoms of the row group itself (the diagonal block)
    // needs the per-pair i < j test. The diagonal block is the first
    // candidate of the list builder's first warp, so a full one fills a tile
    // of its own; the flag is computed per tile either way.
    const unsigned row_first = i & ~(unsigned)(RG - 1);
    const bool check = __any_sync(FULL_MASK, col_ok && j < row_first + RG);
#define TMB_SWEEP(ALCH_, CHECK_)                                                                                      \
    sweep_tile<Real, U, DX, DL, DP, INTERP, ALCH_, CHECK_, RG>(                                                       \
        lane, S, i_eff, j, pwi.x, pwi.y, pwi.z, pwi.w, pri.x, pri.y, pri.z, pri.w, dpi.x, dpi.y, dpi.z, pwj.x, pwj.y,   \
        pwj.z, pwj.w, prj.x, prj.y, prj.z, prj.w, dpj.x, dpj.y, dpj.z, box_x, box_y, box_z, inv_box_x, inv_box_y,       \
        inv_box_z, cutoff_squared, beta, gi_x, gi_y, gi_z, g_qi, g_sigi, g_epsi, du_dl, energy, gj_x, gj_y, gj_z, g_qj, \
        g_sigj, g_epsj)
    if (alch) {
        if (check) {
            TMB_SWEEP(true, true);
        } else {
            TMB_SWEEP(true, false);
        }
    } else {
        if (check) {
            TMB_SWEEP(false, true);
        } else {
            TMB_SWEEP(false, false);
        }
    }
#undef TMB_SWEEP
    if (col_ok) {
        if (DX) {
            red_add(acc_out.x + j, gj_x);
            red_add(acc_out.y + j, gj_y);
            red_add(acc_out.z + j, gj_z);
        }
        if (DP) {
            red_add(acc_out.q + j, g_qj);
            red_add(acc_out.sig + j, g_sigj);
            red_add(acc_out.eps + j, g_epsj);
        }
    }
}

template <bool U, bool DX, bool DL, bool DP>
__device__ __forceinline__ void flush_row(
    const Accum &acc_out,
    unsigned i,
    unsigned long long gi_x,
    unsigned long long gi_y,
    unsigned long long gi_z,
    unsigned long long g_qi,
    unsigned long long g_sigi,
    unsigned long long g_epsi,
    unsigned long long du_dl,
    unsigned long long energy) {
    if (DX) {
        red_add(acc_out.x + i, gi_x);
        red_add(acc_out.y + i, gi_y);
        red_add(acc_out.z + i, gi_z);
    }
    if (DP) {
        red_add(acc_out.q + i, g_qi);
        red_add(acc_out.sig + i, g_sigi);
        red_add(acc_out.eps + i, g_epsi);
    }
    if (DL) {
        red_add(acc_out.dl + i, du_dl);
    }
    if (U) {
        red_add(acc_out.u + i, energy);
    }
}

// Row sums of a tile sweep with RG-slot row groups: the 32/RG lanes holding
// one row combine their partial sums, and the first of them flushes.
template <int RG, bool U, bool DX, bool DL, bool DP>
__device__ __forceinline__ void flush_row_rg(
    const Accum &acc_out,
    unsigned i,
    bool row_ok,
    unsigned long long gi_x,
    unsigned long long gi_y,
    unsigned long long gi_z,
    unsigned long long g_qi,
    unsigned long long g_sigi,
    unsigned long long g_epsi,
    unsigned long long du_dl,
    unsigned long long energy) {
    if (RG < TILE) {
#pragma unroll
        for (int o = RG; o < TILE; o <<= 1) {
            if (DX) {
                gi_x += __shfl_xor_sync(FULL_MASK, gi_x, o);
                gi_y += __shfl_xor_sync(FULL_MASK, gi_y, o);
                gi_z += __shfl_xor_sync(FULL_MASK, gi_z, o);
            }
            if (DP) {
                g_qi += __shfl_xor_sync(FULL_MASK, g_qi, o);
                g_sigi += __shfl_xor_sync(FULL_MASK, g_sigi, o);
                g_epsi += __shfl_xor_sync(FULL_MASK, g_epsi, o);
            }
            if (DL) {
                du_dl += __shfl_xor_sync(FULL_MASK, du_dl, o);
            }
            if (U) {
                energy += __shfl_xor_sync(FULL_MASK, energy, o);
            }
        }
        if ((threadIdx.x & (TILE - 1)) >= RG) {
            return;
        }
    }
    if (row_ok) {
        flush_row<U, DX, DL, DP>(acc_out, i, gi_x, gi_y, gi_z, g_qi, g_sigi, g_epsi, du_dl, energy);
    }
}

// ---------------------------------------------------------------------------
// Forces-only sweep with packed FP32 pairs (16-row tiles).
//
// sm_100 executes FP32x2 instructions (mul/add/sub/fma .rn.f32x2) whose two
// components round exactly as the scalar __fmul_rn / __fadd_rn / __fsub_rn /
// __fmaf_rn do. The forces-only sweep holds two rows per lane (rows r and
// r + 8 of the 16-row group; the warp is four 8-lane groups, each rotating
// its 8 columns through its lanes in 8 rounds) and evaluates the lane's two
// pairs in the two components: the same per-pair roundings as pair_terms in
// about half the FP32 instructions, and one column rotation for two pairs.
// The transcendental steps (rsqrt, exp, the IEEE reciprocal) and the
// fixed-point conversions stay per component, and the row and column forces
// of a pair are converted once, as in pair_terms. The packed operations
// (fmul2 and the others, nb_pair_math.cuh) are inline PTX, so a product
// followed by a sum keeps both roundings. (The all-outputs variants keep the
// one-row sweep: with two rows per lane they need 127 registers, 4 CTAs/SM,
// and the 12-window call measured 2 % slower.)
// ---------------------------------------------------------------------------
// Row accumulators of the packed sweep: forces and energy.
struct RowForces {
    unsigned long long x = 0, y = 0, z = 0, u = 0;
};

// U: energy; DX: forces (one of them or both).
template <bool U, bool DX, bool ALCH, bool CHECK>
__device__ __forceinline__ void sweep_forces_p2(
    const int lane,
    const unsigned S,
    const unsigned ia,
    const unsigned ib,
    unsigned j,
    const float2 ci_x,
    const float2 ci_y,
    const float2 ci_z,
    const float2 ci_w,
    const float2 qi,
    const float2 sig_i,
    const float2 eps_i,
    float cj_x,
    float cj_y,
    float cj_z,
    float cj_w,
    float qj,
    float sig_j,
    float eps_j,
    const float2 neg_box_x,
    const float2 neg_box_y,
    const float2 neg_box_z,
    const float2 inv_box_x,
    const float2 inv_box_y,
    const float2 inv_box_z,
    const float cutoff_squared,
    const float beta,
    RowForces &A,
    RowForces &B,
    unsigned long long &gj_x,
    unsigned long long &gj_y,
    unsigned long long &gj_z) {
    const int src = (lane & ~7) | ((lane + 1) & 7);
#pragma unroll 1
    for (int round = 0; round < 8; round++) {
        const float2 dx = min_image2(fsub2(ci_x, f2(cj_x)), neg_box_x, inv_box_x);
        const float2 dy = min_image2(fsub2(ci_y, f2(cj_y)), neg_box_y, inv_box_y);
        const float2 dz = min_image2(fsub2(ci_z, f2(cj_z)), neg_box_z, inv_box_z);
#if TMNB_DAG_D2 == 0
        float2 d2 = ffma2(dz, dz, ffma2(dx, dx, fmul2(dy, dy)));
#elif TMNB_DAG_D2 == 1
        float2 d2 = ffma2(dz, dz, ffma2(dy, dy, fmul2(dx, dx)));
#else
        float2 d2 = fadd2(fadd2(fmul2(dx, dx), fmul2(dy, dy)), fmul2(dz, dz));
#endif
        if (ALCH) {
            const float2 dw = fsub2(ci_w, f2(cj_w));
            d2 = madd2(dw, dw, d2, TMNB_DAG_D4);
        }
        // validity as in sweep_tile
        const bool in_a = (!CHECK || (ia < S && j < S && ia < j)) && d2.x < cutoff_squared;
        const bool in_b = (!CHECK || (ib < S && j < S && ib < j)) && d2.y < cutoff_squared;
        if (in_a || in_b) {
            // electrostatics (nb_pair_math.cuh electrostatics / es_factor),
            // charge scale 1
            const float2 inv_d = make_float2(inv_sqrt(d2.x), inv_sqrt(d2.y));
            const float2 d = fmul2(d2, inv_d);
            const float2 inv_d2 = fmul2(inv_d, inv_d);
            const float2 qij_inv = fmul2(fmul2(qi, f2(qj)), inv_d);
            const float2 bd = fmul2(f2(beta), d);
            const float2 bd2 = fmul2(bd, bd); // fmul(-bd, bd) == -(bd * bd)
            const float2 e = make_float2(__expf(-bd2.x), __expf(-bd2.y));
            const float2 den = madd2(f2(0.3275911f), bd, f2(1.0f), TMNB_DAG_DEN);
            const float2 t = make_float2(__frcp_rn(den.x), __frcp_rn(den.y));
            float2 poly = madd2(f2(1.061405429f), t, f2(-1.453152027f), TMNB_DAG_POLY);
            poly = madd2(poly, t, f2(1.421413741f), TMNB_DAG_POLY);
            poly = madd2(poly, t, f2(-0.284496736f), TMNB_DAG_POLY);
            poly = madd2(poly, t, f2(0.254829592f), TMNB_DAG_POLY);
            const float2 pt = fmul2(poly, t);
            const float2 erfc_bd = fmul2(pt, e);
            float2 pre = f2(0.0f);
            if (DX) {
                const float2 cbd = fmul2(f2(static_cast<float>(1.128379167095512595889238330988549829708)), bd);
#if TMNB_DAG_ERF == 1
                const float2 s = ffma2(cbd, e, erfc_bd);
#elif TMNB_DAG_ERF == 0
                const float2 s = fadd2(fmul2(cbd, e), erfc_bd);
#else
                const float2 s = ffma2(pt, e, fmul2(cbd, e));
#endif
                pre = fmul2(qij_inv, fmul2(make_float2(-inv_d2.x, -inv_d2.y), s));
            }
            float2 u = f2(0.0f);
            if (U) {
                u = fmul2(qij_inv, erfc_bd);
            }
            // Lennard-Jones where both atoms carry epsilon (per pair)
            const bool lj_a = eps_i.x != 0 && eps_j != 0;
            const bool lj_b = eps_i.y != 0 && eps_j != 0;
            if ((in_a && lj_a) || (in_b && lj_b)) {
                const float2 eps_ij = fmul2(eps_i, f2(eps_j));
                const float2 sig_ij = fadd2(sig_i, f2(sig_j));
                const float2 s1 = fmul2(sig_ij, inv_d);
                const float2 s2 = fmul2(s1, s1);
                const float2 s4 = fmul2(s2, s2);
                const float2 s6 = fmul2(s4, s2);
                if (DX) {
                    const float2 ljx = fmul2(eps_ij, fmul2(s6, inv_d2));
                    const float2 ljy = madd2(s6, f2(48.0f), f2(-24.0f), TMNB_DAG_LJP);
#if TMNB_DAG_PRE == 1
                    const float2 pre_lj = ffma2(make_float2(-ljx.x, -ljx.y), ljy, pre);
#elif TMNB_DAG_PRE == 0
                    const float2 pre_lj = fsub2(pre, fmul2(ljx, ljy));
#else
#error "TMNB_DAG_PRE == 2 has no packed form"
#endif
                    pre = make_float2(lj_a ? pre_lj.x : pre.x, lj_b ? pre_lj.y : pre.y);
                }
                if (U) {
                    // lennard_jones of nb_pair_math.cuh: A = (4 eps_ij)(s6 - 1), u += A s6
#if TMNB_DAG_S6M1
                    const float2 s6m1 = ffma2(s4, s2, f2(-1.0f));
#else
                    const float2 s6m1 = fsub2(s6, f2(1.0f));
#endif
                    const float2 Acoef = fmul2(fmul2(f2(4.0f), eps_ij), s6m1);
#if TMNB_DAG_U == 1
                    const float2 u_lj = ffma2(Acoef, s6, u);
#elif TMNB_DAG_U == 0
                    const float2 u_lj = fadd2(u, fmul2(Acoef, s6));
#else
                    const float2 u_lj = ffma2(qij_inv, erfc_bd, fmul2(Acoef, s6));
#endif
                    u = make_float2(lj_a ? u_lj.x : u.x, lj_b ? u_lj.y : u.y);
                }
            }
            if (U) {
                const float2 yu = fmul2(u, f2(static_cast<float>(FX_EXPONENT)));
                if (in_a) {
                    A.u += fixed_round(yu.x);
                }
                if (in_b) {
                    B.u += fixed_round(yu.y);
                }
            }
            const float2 ex = f2(static_cast<float>(FX_EXPONENT));
            const float2 yx = fmul2(fmul2(pre, dx), ex);
            const float2 yy = fmul2(fmul2(pre, dy), ex);
            const float2 yz = fmul2(fmul2(pre, dz), ex);
            if (DX && in_a) {
                const unsigned long long fx = fixed_round(yx.x), fy = fixed_round(yy.x), fz = fixed_round(yz.x);
                A.x += fx;
                A.y += fy;
                A.z += fz;
                gj_x -= fx;
                gj_y -= fy;
                gj_z -= fz;
                if (!fixed_in_range(yx.x) || !fixed_in_range(yy.x) || !fixed_in_range(yz.x)) {
                    gj_x += fixed_round(-yx.x) + fx;
                    gj_y += fixed_round(-yy.x) + fy;
                    gj_z += fixed_round(-yz.x) + fz;
                }
            }
            if (DX && in_b) {
                const unsigned long long fx = fixed_round(yx.y), fy = fixed_round(yy.y), fz = fixed_round(yz.y);
                B.x += fx;
                B.y += fy;
                B.z += fz;
                gj_x -= fx;
                gj_y -= fy;
                gj_z -= fz;
                if (!fixed_in_range(yx.y) || !fixed_in_range(yy.y) || !fixed_in_range(yz.y)) {
                    gj_x += fixed_round(-yx.y) + fx;
                    gj_y += fixed_round(-yy.y) + fy;
                    gj_z += fixed_round(-yz.y) + fz;
                }
            }
        }
        if (CHECK) {
            j = __shfl_sync(FULL_MASK, j, src);
        }
        qj = __shfl_sync(FULL_MASK, qj, src);
        eps_j = __shfl_sync(FULL_MASK, eps_j, src);
        sig_j = __shfl_sync(FULL_MASK, sig_j, src);
        cj_x = __shfl_sync(FULL_MASK, cj_x, src);
        cj_y = __shfl_sync(FULL_MASK, cj_y, src);
        cj_z = __shfl_sync(FULL_MASK, cj_z, src);
        if (ALCH) {
            cj_w = __shfl_sync(FULL_MASK, cj_w, src);
        }
        if (DX) {
            gj_x = __shfl_sync(FULL_MASK, gj_x, src);
            gj_y = __shfl_sync(FULL_MASK, gj_y, src);
            gj_z = __shfl_sync(FULL_MASK, gj_z, src);
        }
    }
}

// One 16-row tile of a forces and / or energy evaluation (U, DX), window
// `window`: the lane's rows ia and ia + 8 against column slot j.
template <bool U, bool DX>
__device__ __forceinline__ void tile_forces_p2(
    const PairArgs &a,
    const int lane,
    const unsigned S,
    const unsigned ia,
    const unsigned j,
    const int window,
    const Accum &acc_out,
    const float box_x,
    const float box_y,
    const float box_z,
    const float inv_box_x,
    const float inv_box_y,
    const float inv_box_z,
    const float cutoff_squared,
    const float beta,
    RowForces &A,
    RowForces &B) {
    const unsigned ib = ia + 8;
    const size_t wo = (size_t)window * a.S;
    const bool a_ok = ia < (unsigned)a.row_end;
    const bool b_ok = ib < (unsigned)a.row_end;
    const bool col_ok = j < S;
    const float nan = __int_as_float(0x7fffffff);
    const float4 pwa = a_ok ? a.posw[wo + ia] : make_float4(nan, nan, nan, 0.f);
    const float4 pra = a_ok ? a.prm[wo + ia] : make_float4(0.f, 0.f, 0.f, 0.f);
    const float4 pwb = b_ok ? a.posw[wo + ib] : make_float4(nan, nan, nan, 0.f);
    const float4 prb = b_ok ? a.prm[wo + ib] : make_float4(0.f, 0.f, 0.f, 0.f);
    const float4 pwj = col_ok ? a.posw[wo + j] : make_float4(nan, nan, nan, 0.f);
    const float4 prj = col_ok ? a.prm[wo + j] : make_float4(0.f, 0.f, 0.f, 0.f);
    // Forces and energies depend on the parameters' lambda derivatives only
    // through w: a tile whose w are all zero adds dw*dw = 0 exactly, so it
    // skips the 4th dimension whatever the interpolated parameters do.
    const bool alch = __any_sync(FULL_MASK, pwa.w != 0.f || pwb.w != 0.f || pwj.w != 0.f);
    const unsigned ia_eff = a_ok ? ia : 0xffffffffu;
    const unsigned ib_eff = b_ok ? ib : 0xffffffffu;
    const unsigned row_first = ia & ~15u;
    const bool check = __any_sync(FULL_MASK, col_ok && j < row_first + 16);
    unsigned long long gj_x = 0, gj_y = 0, gj_z = 0;
#define TMB_SWEEP_P2(ALCH_, CHECK_)                                                                                    \
    sweep_forces_p2<U, DX, ALCH_, CHECK_>(                                                                              \
        lane, S, ia_eff, ib_eff, j, make_float2(pwa.x, pwb.x), make_float2(pwa.y, pwb.y), make_float2(pwa.z, pwb.z),   \
        make_float2(pwa.w, pwb.w), make_float2(pra.x, prb.x), make_float2(pra.y, prb.y), make_float2(pra.z, prb.z),   \
        pwj.x, pwj.y, pwj.z, pwj.w, prj.x, prj.y, prj.z, f2(-box_x), f2(-box_y), f2(-box_z), f2(inv_box_x),           \
        f2(inv_box_y), f2(inv_box_z), cutoff_squared, beta, A, B, gj_x, gj_y, gj_z)
    if (alch) {
        if (check) {
            TMB_SWEEP_P2(true, true);
        } else {
            TMB_SWEEP_P2(true, false);
        }
    } else {
        if (check) {
            TMB_SWEEP_P2(false, true);
        } else {
            TMB_SWEEP_P2(false, false);
        }
    }
#undef TMB_SWEEP_P2
    if (DX && col_ok) {
        red_add(acc_out.x + j, gj_x);
        red_add(acc_out.y + j, gj_y);
        red_add(acc_out.z + j, gj_z);
    }
}

// Row sums of a packed sweep: the four lanes holding rows ia / ia + 8
// (lanes l, l^8, l^16, l^24) combine, and lanes 0-7 flush.
template <bool U, bool DX>
__device__ __forceinline__ void flush_forces_p2(const Accum &acc_out, unsigned ia, unsigned row_end, RowForces A,
                                                RowForces B) {
#pragma unroll
    for (int o = 8; o < TILE; o <<= 1) {
        if (DX) {
            A.x += __shfl_xor_sync(FULL_MASK, A.x, o);
            A.y += __shfl_xor_sync(FULL_MASK, A.y, o);
            A.z += __shfl_xor_sync(FULL_MASK, A.z, o);
            B.x += __shfl_xor_sync(FULL_MASK, B.x, o);
            B.y += __shfl_xor_sync(FULL_MASK, B.y, o);
            B.z += __shfl_xor_sync(FULL_MASK, B.z, o);
        }
        if (U) {
            A.u += __shfl_xor_sync(FULL_MASK, A.u, o);
            B.u += __shfl_xor_sync(FULL_MASK, B.u, o);
        }
    }
    if ((threadIdx.x & (TILE - 1)) >= 8) {
        return;
    }
    if (ia < row_end) {
        if (DX) {
            red_add(acc_out.x + ia, A.x);
            red_add(acc_out.y + ia, A.y);
            red_add(acc_out.z + ia, A.z);
        }
        if (U) {
            red_add(acc_out.u + ia, A.u);
        }
    }
    if (ia + 8 < row_end) {
        if (DX) {
            red_add(acc_out.x + ia + 8, B.x);
            red_add(acc_out.y + ia + 8, B.y);
            red_add(acc_out.z + ia + 8, B.z);
        }
        if (U) {
            red_add(acc_out.u + ia + 8, B.u);
        }
    }
}

// Multi-window calls: lists the tiles with at least one lambda-dependent row
// or column atom (the tiles the pair kernel evaluates once per window). One
// warp per work item, grid-stride.
struct DepArgs {
    int S;
    int rows; // slots per row group
    int row_end;
    const int4 *items;
    const unsigned *tile_cols;
    const unsigned char *lamdep;
    int2 *dep_tiles;
};

// The list only changes with the tile list or the atoms' lambda dependence,
// so a call with neither keeps the previous one (state->dep_dirty).
static __global__ void k_dep_tiles(DepArgs a, DevState *state) {
    grid_dependency_wait();
    if (state->error || !state->dep_dirty) {
        return;
    }
    const int lane = threadIdx.x & 31;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int n_warps = (gridDim.x * blockDim.x) >> 5;
    const unsigned S = (unsigned)a.S;
    const int n_items = state->n_items;
    for (int w = warp; w < n_items; w += n_warps) {
        const int4 it = a.items[w];
        const unsigned i = (unsigned)(it.x * a.rows + (lane & (a.rows - 1)));
        const bool row_dep = i < (unsigned)a.row_end && a.lamdep[i];
        for (int t = 0; t < it.z; t++) {
            const int tile = it.y + t;
            const unsigned j = a.tile_cols[(long long)tile * TILE + lane];
            if (__any_sync(FULL_MASK, row_dep || (j < S && a.lamdep[j])) && lane == 0) {
                a.dep_tiles[atomicAdd(&state->n_dep, 1)] = make_int2(it.x, tile);
            }
        }
    }
}

// Persistent pair kernel over dynamically scheduled work units:
//   [0, n_items)                 tile work items (row group, first tile, count);
//   MULTI only: [n_items, + n_dep*K)  one lambda-dependent tile at one window;
//   then                         chunks of 32 scaled pairs (one per lane).
// MULTI (K > 1 windows): the tile items skip lambda-dependent tiles and add
// into the shared accumulator block; each (tile, window) unit adds into the
// window's block; a lambda-dependent scaled pair is evaluated for every window.
// CTAs per SM the compiler must fit for each pair-kernel variant (its
// register budget): measured on B200, see the kernel below.
template <typename Real, bool U, bool DX, bool DL, bool DP, bool INTERP, int RG>
constexpr int pair_min_ctas() {
    if (sizeof(Real) != 4) {
        return 5;
    }
    if (U && DX && DL && DP && !INTERP) {
        return 6;
    }
    if (DX && !U && !DL && !DP) {
        return (TMNB_PACKED_FORCES && RG == 16) ? TMNB_PACKED_FORCES_CTAS : 8;
    }
    if (U && !DX && !DL && !DP && TMNB_PACKED_FORCES && TMNB_PACKED_ENERGY && RG == 16) {
        return TMNB_PACKED_FORCES_CTAS;
    }
    return 1;
}

template <typename Real, bool U, bool DX, bool DL, bool DP, bool INTERP, bool MULTI, int RG = TILE>
// Occupancy, measured on B200: all four outputs at 6 CTAs/SM (80 registers,
// no spills; 12-window call -3.5 % against 5); forces only or energy only
// with the packed two-rows sweep at 6 (80), forces only with 8 or 32 rows per
// tile at 8 (64). FP64
// variants at 5 (96 registers, a few spilled words): the 12-window call
// took 0.407 ms against 0.455 ms at the compiler's 154 registers (3 CTAs).
__global__ void __launch_bounds__(128, (pair_min_ctas<Real, U, DX, DL, DP, INTERP, RG>())) k_pair(PairArgs a) {
    grid_dependency_wait();
    if (a.state->error) {
        return;
    }
    const int lane = threadIdx.x & 31;
    const Real box_x = a.box[0 * 3 + 0];
    const Real box_y = a.box[1 * 3 + 1];
    const Real box_z = a.box[2 * 3 + 2];
    const Real inv_box_x = 1 / box_x;
    const Real inv_box_y = 1 / box_y;
    const Real inv_box_z = 1 / box_z;
    const Real real_cutoff = static_cast<Real>(a.cutoff);
    const Real cutoff_squared = real_cutoff * real_cutoff;
    const Real beta = static_cast<Real>(a.beta);
    const unsigned S = (unsigned)a.S;
    const int n_items = a.state->n_items;
    const int n_dep_units = MULTI ? a.state->n_dep * a.K : 0;
    if (MULTI && blockIdx.x == 0 && threadIdx.x == 0 && !a.state->error) {
        // k_dep_tiles (before this launch) has redone the list; after an
        // error it did not, so the list stays dirty for the next call
        a.state->dep_dirty = 0;
    }
    const int n_tiles_units = n_items + n_dep_units;
    const int n_total = n_tiles_units + (a.M + TILE - 1) / TILE;
    // forces-only FP32 evaluations of 16-row tiles take the packed sweep
    constexpr bool PACKED =
        TMNB_PACKED_FORCES && sizeof(Real) == 4 && RG == 16 && !DL && !DP && ((DX && !U) || (U && !DX && TMNB_PACKED_ENERGY));

    for (;;) {
        int item = 0;
        if (lane == 0) {
            item = atomicAdd(&a.state->next_item, 1);
        }
        item = __shfl_sync(FULL_MASK, item, 0);
        if (item >= n_total) {
            break;
        }
        if (item >= n_tiles_units) {
            const int pair = (item - n_tiles_units) * TILE + lane;
            if (pair < a.M) {
                const int atom_i = a.pair_idxs[2 * pair + 0];
                const int atom_j = a.pair_idxs[2 * pair + 1];
                const int si = a.slot_of ? a.slot_of[atom_i] : atom_i;
                const int sj = a.slot_of ? a.slot_of[atom_j] : atom_j;
                if (!MULTI || !(a.lamdep[si] || a.lamdep[sj])) {
                    scaled_pair<Real, U, DX, DL, DP, INTERP>(
                        a, pair, si, sj, 0, a.acc, box_x, box_y, box_z, inv_box_x, inv_box_y, inv_box_z,
                        cutoff_squared);
                } else {
                    for (int k = 0; k < a.K; k++) {
                        scaled_pair<Real, U, DX, DL, DP, INTERP>(
                            a, pair, si, sj, k, acc_block(a.acc, a.acc_block, 1 + k), box_x, box_y, box_z, inv_box_x,
                            inv_box_y, inv_box_z, cutoff_squared);
                    }
                }
            }
            continue;
        }
        if constexpr (PACKED) {
            // two rows per lane: ia and ia + 8 of the 16-row group
            if (MULTI && item >= n_items) {
                const int unit = item - n_items;
                const int2 dt = a.dep_tiles[unit / a.K];
                const int k = unit % a.K;
                const unsigned ia = (unsigned)(dt.x * RG + (lane & 7));
                const unsigned j = a.tile_cols[(long long)dt.y * TILE + lane];
                const Accum wk = acc_block(a.acc, a.acc_block, 1 + k);
                RowForces A, B;
                tile_forces_p2<U, DX>(a, lane, S, ia, j, k, wk, box_x, box_y, box_z, inv_box_x, inv_box_y, inv_box_z,
                               cutoff_squared, beta, A, B);
                flush_forces_p2<U, DX>(wk, ia, (unsigned)a.row_end, A, B);
                continue;
            }
            const int4 it = a.items[item];
            const unsigned ia = (unsigned)(it.x * RG + (lane & 7));
            const bool row_dep = MULTI && ((ia < (unsigned)a.row_end && a.lamdep[ia]) ||
                                           (ia + 8 < (unsigned)a.row_end && a.lamdep[ia + 8]));
            RowForces A, B;
            for (int t = 0; t < it.z; t++) {
                const long long tile = (long long)it.y + t;
                const unsigned j = a.tile_cols[tile * TILE + lane];
                if (MULTI && __any_sync(FULL_MASK, row_dep || (j < S && a.lamdep[j]))) {
                    continue; // evaluated per window by the (tile, window) units
                }
                tile_forces_p2<U, DX>(a, lane, S, ia, j, 0, a.acc, box_x, box_y, box_z, inv_box_x, inv_box_y, inv_box_z,
                               cutoff_squared, beta, A, B);
            }
            flush_forces_p2<U, DX>(a.acc, ia, (unsigned)a.row_end, A, B);
            continue;
        }
        if (MULTI && item >= n_items) {
            const int unit = item - n_items;
            const int2 dt = a.dep_tiles[unit / a.K];
            const int k = unit % a.K;
            const unsigned i = (unsigned)(dt.x * RG + (lane & (RG - 1)));
            const unsigned j = a.tile_cols[(long long)dt.y * TILE + lane];
            const Accum wk = acc_block(a.acc, a.acc_block, 1 + k);
            unsigned long long wx = 0, wy = 0, wz = 0, wq = 0, ws = 0, we = 0, wl = 0, wu = 0;
            tile_pass<Real, U, DX, DL, DP, INTERP, RG>(
                a, lane, S, i, j, k, wk, box_x, box_y, box_z, inv_box_x, inv_box_y, inv_box_z, cutoff_squared, beta,
                wx, wy, wz, wq, ws, we, wl, wu);
            flush_row_rg<RG, U, DX, DL, DP>(wk, i, i < (unsigned)a.row_end, wx, wy, wz, wq, ws, we, wl, wu);
            continue;
        }
        const int4 it = a.items[item];
        const unsigned i = (unsigned)(it.x * RG + (lane & (RG - 1)));
        const bool row_dep = MULTI && i < (unsigned)a.row_end && a.lamdep[i];
        unsigned long long gi_x = 0, gi_y = 0, gi_z = 0, g_qi = 0, g_sigi = 0, g_epsi = 0, du_dl = 0, energy = 0;
        for (int t = 0; t < it.z; t++) {
            const long long tile = (long long)it.y + t;
            const unsigned j = a.tile_cols[tile * TILE + lane];
            if (MULTI && __any_sync(FULL_MASK, row_dep || (j < S && a.lamdep[j]))) {
                continue; // evaluated per window by the (tile, window) units
            }
            tile_pass<Real, U, DX, DL, DP, INTERP, RG>(
                a, lane, S, i, j, 0, a.acc, box_x, box_y, box_z, inv_box_x, inv_box_y, inv_box_z, cutoff_squared,
                beta, gi_x, gi_y, gi_z, g_qi, g_sigi, g_epsi, du_dl, energy);
        }
        flush_row_rg<RG, U, DX, DL, DP>(
            a.acc, i, i < (unsigned)a.row_end, gi_x, gi_y, gi_z, g_qi, g_sigi, g_epsi, du_dl, energy);
    }
}

// ---------------------------------------------------------------------------
// Scatter of the slot-ordered accumulators into the caller's outputs (which
// accumulate, +=), and reset of the accumulators. Window k's result is the
// shared block plus block 1 + k (one window: block 0 only).
// du_dp of interpolated potentials is split into the lambda=0 and lambda=1
// halves per potential part, with the rounding of
// timemachine/cpp/src/kernels/k_lambda_transformer_jit.cuh:100-137.
// ---------------------------------------------------------------------------
struct FinalizeArgs {
    int N;
    int S;
    int K;
    double f_dp[MAX_WINDOWS][3]; // interpolated: f(lambda_k) of the charge, sigma and epsilon transforms
    const int *set_atoms; // [S] atoms of the evaluated set in ascending order, nullptr: 0..S-1
    const int *slot_of;   // [N] atom -> slot, nullptr: identity
    int take;             // 1: zero each accumulator after reading it; 0: the caller zeroes them
    Accum acc;
    size_t acc_block;
    int split_pair_dp; // 1: acc.pq/psig/peps are separate buffers
    int interpolated;
    unsigned long long *du_dx; // [K][N,3] (window stride out_stride_x)
    unsigned long long *du_dp; // [K][P]
    unsigned long long *du_dl; // [K][N]
    unsigned long long *u;     // [K][N]
    size_t stride_x, stride_p, stride_n;
    const DevState *state;
};

__device__ __forceinline__ unsigned long long interp_part(double f, unsigned long long v, unsigned long long e) {
    const double real = static_cast<double>(static_cast<long long>(v)) / e;
    return static_cast<unsigned long long>(llrint((f * real) * e));
}

__device__ __forceinline__ unsigned long long take(unsigned long long *p) {
    const unsigned long long v = *p;
    *p = 0;
    return v;
}

// One thread per (window k, set atom), consecutive threads on consecutive
// atoms, so the output updates are coalesced and the slot-ordered
// accumulators are gathered through slot_of. Only the accumulators of
// requested outputs are read (the others were never written and stay zero).
// take = 1 zeroes each accumulator after the read (one window: every slot is
// read by exactly one thread); otherwise the caller zeroes the accumulator
// blocks after this kernel. Outputs are added with integer atomics, so other
// potentials may accumulate into the same buffers concurrently (the sums are
// order-independent).
static __global__ void k_finalize(FinalizeArgs a) {
    grid_dependency_wait();
    const bool ok = a.state->error == 0;
    const bool multi = a.K > 1;
    const size_t total = (size_t)a.S * (size_t)a.K;
    const Accum &c = a.acc;
    for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < total; t += (size_t)gridDim.x * blockDim.x) {
        const int k = (int)(t / (size_t)a.S);
        const int idx = (int)(t - (size_t)k * a.S);
        const int atom = a.set_atoms ? a.set_atoms[idx] : idx;
        const int s = a.slot_of ? a.slot_of[atom] : atom;
        const size_t o = a.acc_block * (size_t)(1 + k) + s;
        auto get = [&](unsigned long long *p) -> unsigned long long {
            if (multi) {
                return p[s] + p[o];
            }
            return a.take ? take(p + s) : p[s];
        };
        if (a.du_dx) {
            const unsigned long long vx = get(c.x), vy = get(c.y), vz = get(c.z);
            if (ok) {
                unsigned long long *out = a.du_dx + a.stride_x * k + 3 * (size_t)atom;
                atomicAdd(out + 0, vx);
                atomicAdd(out + 1, vy);
                atomicAdd(out + 2, vz);
            }
        }
        if (a.du_dp) {
            unsigned long long v0[3] = {get(c.q), get(c.sig), get(c.eps)};
            unsigned long long v1[3] = {0, 0, 0};
            if (a.split_pair_dp) {
                v1[0] = get(c.pq);
                v1[1] = get(c.psig);
                v1[2] = get(c.peps);
            }
            if (ok) {
                const unsigned long long ex[3] = {FX_EXPONENT, FX_EXPONENT_SIG, FX_EXPONENT_EPS};
                unsigned long long *out = a.du_dp + a.stride_p * k;
                for (int d = 0; d < 3; d++) {
                    if (a.interpolated) {
                        const double f = a.f_dp[k][d];
                        unsigned long long lo = interp_part(1 - f, v0[d], ex[d]) + interp_part(1 - f, v1[d], ex[d]);
                        unsigned long long hi = interp_part(f, v0[d], ex[d]) + interp_part(f, v1[d], ex[d]);
                        atomicAdd(out + 3 * (size_t)atom + d, lo);
                        atomicAdd(out + 3 * ((size_t)a.N + atom) + d, hi);
                    } else {
                        atomicAdd(out + 3 * (size_t)atom + d, v0[d] + v1[d]);
                    }
                }
            }
        }
        if (a.u) {
            const unsigned long long vu = get(c.u);
            if (ok) {
                atomicAdd(a.u + a.stride_n * k + atom, vu);
            }
        }
        if (a.du_dl) {
            const unsigned long long vl = get(c.dl);
            if (ok) {
                atomicAdd(a.du_dl + a.stride_n * k + atom, vl);
            }
        }
    }
}

} // namespace tmb
