// Replica batch: many independent systems (each at its own lambda) evaluated,
// and advanced by Langevin MD, together. One launch sequence per step covers
// every replica, whatever its size: each kernel maps its blocks to replicas
// through host-built block maps, and the pair kernel is ONE persistent launch
// whose warps pull (replica, tile item | scaled-pair chunk) work units from a
// device-side prefix over all replicas. A whole MD chunk is captured in one
// CUDA graph and replayed.
//
// No reference counterpart as a whole: the reference evaluates replicas one at
// a time (one Potential::execute_device per replica and lambda, e.g. the
// window loops of timemachine/cpp/src/context.cu:139-234 and
// timemachine/cpp/src/wrap_kernels.cpp:381-551, one Context per replica for
// MD). Per replica the arithmetic is exactly the single-system pipeline's
// (nb_kernels.cuh), so each replica's outputs equal a single-system
// evaluation bit for bit, alone or in any mix.
//
// Membership can change between steps (add/remove replicas): each replica
// owns one device arena; the descriptor table and block maps are rebuilt on
// the host and uploaded, and captured graphs are discarded.
#include "bonded_math.cuh"
#include "engine.hpp"
#include "md_math.cuh"
#include "nb_kernels.cuh"

#include <algorithm>
#include <cmath>
#include <map>
#include <memory>
#include <string>
#include <vector>

namespace tmb {
namespace {

constexpr int ATOM_BLOCK = 256; // atoms per block of the per-atom kernels
constexpr int TERM_BLOCK = 128; // bonded terms per block

// Device-side descriptor of one replica (pointers into its arena).
struct Rep {
    int N, RB, grid_bits, M;
    int rows, NG; // slots per row group of the tile list, row groups
    int n_bonds, n_angles;
    int chunk, item_cap;
    double lambda, beta, cutoff, padding;
    double ca, dt;
    uint2 key;
    double *x, *v, *box;
    const double *p;
    const int *plane, *offset;
    const int *pair_idxs;
    const double *scales;
    const int *bond_idxs;
    const double *bond_params;
    const int *angle_idxs;
    const double *angle_params;
    const double *cbs, *ccs;
    float4 *posw, *prm;
    unsigned char *lamdep;
    unsigned *keys, *perm;
    int *slot_of;
    double *nb_x, *nb_box;
    int *bin_count, *bin_cursor;
    float4 *bb_ctr, *bb_ext;
    int *rb_ntiles;
    unsigned *tile_cols;
    int4 *items;
    unsigned long long *acc; // [8][N]
    unsigned long long *du_dx, *du_dp, *du_dl, *u;
    unsigned long long *md_step;
    DevState *state;
};

__device__ __forceinline__ SortArgs sort_args(const Rep &r) {
    SortArgs sa;
    sa.N = r.N;
    sa.S = r.N;
    sa.x = r.x;
    sa.box = r.box;
    sa.set_atoms = nullptr;
    sa.n_first = r.N;
    sa.grid_bits = r.grid_bits;
    sa.hilbert = 1;
    sa.keys = r.keys;
    sa.bin_count = r.bin_count;
    sa.bin_cursor = r.bin_cursor;
    return sa;
}

// One slot's FP32 staging at the replica's lambda (one window, parameters not
// interpolated): the same values as prepare_slot.
__device__ __forceinline__ void stage_slot(const Rep &r, int s, int atom) {
    const int plane = r.plane[atom];
    const int offset = r.offset[atom];
    const double f_lambda_grad = 1.0;
    const double dw_dl = offset * f_lambda_grad * r.cutoff;
    const double *xa = r.x + 3 * (size_t)atom;
    const double *p0 = r.p + 3 * (size_t)atom;
    const double w = (plane + offset * r.lambda) * r.cutoff;
    r.posw[s] = make_float4((float)xa[0], (float)xa[1], (float)xa[2], (float)w);
    r.prm[s] = make_float4((float)p0[0], (float)p0[1], (float)p0[2], (float)dw_dl);
    r.lamdep[s] = offset != 0 ? 1 : 0;
}

__global__ void k_b_prepare(const Rep *__restrict__ reps, const int2 *__restrict__ ablk) {
    const int2 m = ablk[blockIdx.x];
    const Rep &r = reps[m.x];
    const int s = m.y + threadIdx.x;
    if (s == 0) {
        DevState *st = r.state;
        st->next_item = 0;
        const double db_cutoff = (r.cutoff + r.padding) * 2;
        int err = 0;
        for (int k = 0; k < 9 && err == 0; k++) {
            if (k == 0 || k == 4 || k == 8) {
                if (r.box[k] < db_cutoff) {
                    err = DEV_ERR_BOX_TOO_SMALL;
                }
            } else if (r.box[k] != 0.0) {
                err = DEV_ERR_NONORTHO_BOX;
            }
        }
        if (err != 0) {
            st->error = err;
        }
        for (int k = 0; k < 9; k++) {
            if (r.box[k] != r.nb_box[k]) {
                st->rebuild = 1;
            }
        }
    }
    if (s < r.N) {
        const int atom = r.perm[s];
        const double *xn = r.x + 3 * (size_t)atom;
        const double *xo = r.nb_x + 3 * (size_t)atom;
        const double dx = xn[0] - xo[0], dy = xn[1] - xo[1], dz = xn[2] - xo[2];
        if (dx * dx + dy * dy + dz * dz > 0.25 * r.padding * r.padding) {
            r.state->rebuild = 1; // benign race: every writer stores 1
        }
        stage_slot(r, s, atom);
    }
}

__global__ void k_b_keys(const Rep *__restrict__ reps, const int2 *__restrict__ ablk) {
    const int2 m = ablk[blockIdx.x];
    const Rep &r = reps[m.x];
    const int k = m.y + threadIdx.x;
    if (!r.state->rebuild || r.state->error || k >= r.N) {
        return;
    }
    bin_key(sort_args(r), k);
}

__global__ void k_b_scan(const Rep *__restrict__ reps) {
    const Rep &r = reps[blockIdx.x];
    if (!r.state->rebuild || r.state->error) {
        return;
    }
    bin_scan_cta(sort_args(r), r.state);
}

__global__ void k_b_scatter(const Rep *__restrict__ reps, const int2 *__restrict__ ablk) {
    const int2 m = ablk[blockIdx.x];
    const Rep &r = reps[m.x];
    if (!r.state->rebuild || r.state->error) {
        return;
    }
    const int k = m.y + threadIdx.x;
    if (m.y == 0 && threadIdx.x < 9) {
        r.nb_box[threadIdx.x] = r.box[threadIdx.x];
    }
    if (k < r.N) {
        const int s = scatter_slot(sort_args(r), k, r.perm, r.slot_of, r.nb_x);
        stage_slot(r, s, k);
    }
}

// Lennard-Jones atoms first within the replica's 32-slot block rb (one warp),
// as lj_first_warp does for a single system; restages the moved slots.
__device__ __forceinline__ void lj_first_rep(const Rep &r, int rb) {
    const int lane = threadIdx.x & 31;
    const int lo = rb * TILE;
    const int s = lo + lane;
    const bool valid = s < r.N;
    const unsigned atom = valid ? r.perm[s] : 0u;
    const bool lj = valid && r.p[3 * (size_t)atom + 2] != 0.0;
    const unsigned m = __ballot_sync(FULL_MASK, lj);
    const unsigned vm = __ballot_sync(FULL_MASK, valid);
    if (m == 0u || m == vm) {
        return;
    }
    const unsigned lt = (1u << lane) - 1u;
    const int seg = lane / r.rows; // LJ atoms first within each row group
    const unsigned segm = (r.rows == TILE ? FULL_MASK : ((1u << r.rows) - 1u)) << (seg * r.rows);
    const int pos = seg * r.rows +
                    (lj ? __popc(m & lt & segm) : __popc(m & segm) + __popc(vm & ~m & lt & segm));
    __syncwarp();
    if (valid && lo + pos != s) {
        const int ns = lo + pos;
        r.perm[ns] = atom;
        r.slot_of[atom] = ns;
        stage_slot(r, ns, (int)atom);
    }
    __syncwarp();
}

__global__ void k_b_bounds(const Rep *__restrict__ reps, const int2 *__restrict__ rbmap, int n_rb) {
    const int g = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (g >= n_rb) {
        return;
    }
    const int2 m = rbmap[g];
    const Rep &r = reps[m.x];
    if (!r.state->rebuild || r.state->error) {
        return;
    }
    lj_first_rep(r, m.y);
    block_bounds_warp(r.N, m.y, r.box, r.posw, r.bb_ctr, r.bb_ext);
}

// Exclusive prefix over replicas of count(replica) into prefix[0..R-1], the
// total into prefix[R]. One CTA.
template <typename Count>
__device__ __forceinline__ void replica_prefix(int R, int *__restrict__ prefix, Count count) {
    __shared__ int warp_sums[32];
    __shared__ int carry;
    if (threadIdx.x == 0) {
        carry = 0;
    }
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const int wid = threadIdx.x >> 5;
    const int nwarps = blockDim.x >> 5;
    for (int base = 0; base < R; base += blockDim.x) {
        const int q = base + threadIdx.x;
        const int v = q < R ? count(q) : 0;
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
                warp_sums[lane] = ws;
            }
        }
        __syncthreads();
        if (q < R) {
            prefix[q] = carry + (wid > 0 ? warp_sums[wid - 1] : 0) + incl - v;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            carry += warp_sums[nwarps - 1];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        prefix[R] = carry;
    }
}

// Last replica q with prefix[q] <= unit (replicas without units are skipped).
__device__ __forceinline__ int replica_of(const int *__restrict__ prefix, int R, int unit) {
    int lo = 0, hi = R - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (prefix[mid] <= unit) {
            lo = mid;
        } else {
            hi = mid - 1;
        }
    }
    return lo;
}

// Persistent over the row groups of the replicas that rebuild this step (the
// prefix of k_b_tile_units), claimed one at a time from a counter: a step in
// which few replicas rebuild launches a few CTAs per SM instead of one CTA per
// row group of every replica.
__global__ void __launch_bounds__(TB_WARPS * 32, TMNB_TB_CTAS)
    k_b_tiles(const Rep *__restrict__ reps, int R, const int *__restrict__ tprefix, int *__restrict__ tcounter) {
    const int total = tprefix[R];
    __shared__ int next;
    for (;;) {
        __syncthreads(); // the previous row group's shared state is no longer read
        if (threadIdx.x == 0) {
            next = atomicAdd(tcounter, 1); // row groups are claimed dynamically: their costs differ
        }
        __syncthreads();
        const int u = next;
        if (u >= total) {
            break;
        }
        const int q = replica_of(tprefix, R, u);
        const Rep &r = reps[q];
        TileArgs ta;
        ta.S = r.N;
        ta.RB = r.RB;
        ta.rows = r.rows;
        ta.group = 0;
        ta.row_end = r.N;
        ta.col_begin = 0;
        ta.n_row_blocks = r.NG;
        ta.cb_first = 0;
        ta.radius = (float)(r.cutoff + r.padding + 1e-5);
        ta.box = r.box;
        ta.posw = r.posw;
        ta.prm = r.prm;
        ta.bb_ctr = r.bb_ctr;
        ta.bb_ext = r.bb_ext;
        ta.tile_cols = r.tile_cols;
        ta.rb_ntiles = r.rb_ntiles;
        ta.items = r.items;
        ta.chunk = r.chunk;
        build_tiles_cta(ta, u - tprefix[q], r.state);
    }
}

// Exclusive prefix over replicas of their work units (tile items + chunks of
// 32 scaled pairs); replicas with an error contribute none. One CTA.
__global__ void k_b_units(const Rep *__restrict__ reps, int R, int *__restrict__ prefix, int *__restrict__ counter) {
    if (threadIdx.x == 0) {
        *counter = 0;
    }
    replica_prefix(R, prefix, [&](int q) {
        const Rep &r = reps[q];
        return r.state->error ? 0 : r.state->n_items + (r.M + TILE - 1) / TILE;
    });
}

// Exclusive prefix over replicas of the row groups whose lists this step
// rebuilds (none for a replica without the rebuild flag or with an error).
// One CTA.
__global__ void k_b_tile_units(const Rep *__restrict__ reps, int R, int *__restrict__ tprefix,
                               int *__restrict__ tcounter) {
    if (threadIdx.x == 0) {
        *tcounter = 0;
    }
    replica_prefix(R, tprefix, [&](int q) {
        const Rep &r = reps[q];
        return (r.state->rebuild && !r.state->error) ? r.NG : 0;
    });
}

__device__ __forceinline__ PairArgs pair_args(const Rep &r) {
    PairArgs a;
    a.S = r.N;
    a.row_end = r.N;
    a.K = 1;
    a.posw = r.posw;
    a.prm = r.prm;
    a.dprm = nullptr;
    a.posw64 = nullptr;
    a.prm64 = nullptr;
    a.dprm64 = nullptr;
    a.lamdep = r.lamdep;
    a.box = r.box;
    a.beta = r.beta;
    a.cutoff = r.cutoff;
    a.tile_cols = r.tile_cols;
    a.items = r.items;
    a.M = r.M;
    a.pair_idxs = r.pair_idxs;
    a.scales = r.scales;
    a.slot_of = r.slot_of;
    a.negated = 1;
    const size_t N = r.N;
    a.acc.x = r.acc + 0 * N;
    a.acc.y = r.acc + 1 * N;
    a.acc.z = r.acc + 2 * N;
    a.acc.q = r.acc + 3 * N;
    a.acc.sig = r.acc + 4 * N;
    a.acc.eps = r.acc + 5 * N;
    a.acc.u = r.acc + 6 * N;
    a.acc.dl = r.acc + 7 * N;
    a.acc.pq = a.acc.q;
    a.acc.psig = a.acc.sig;
    a.acc.peps = a.acc.eps;
    a.acc_block = 8 * N;
    a.dep_tiles = nullptr;
    a.state = r.state;
    return a;
}

// Persistent pair kernel over every replica's work units.
template <bool U, bool DX, bool DL, bool DP, int RG>
__global__ void __launch_bounds__(
    128, (DX && !U && !DL && !DP) ? (TMNB_PACKED_FORCES && RG == 16 ? TMNB_PACKED_FORCES_CTAS : 8) : 5)
    k_b_pair(const Rep *__restrict__ reps, int R, const int *__restrict__ prefix, int *counter) {
    // forces-only evaluations of 16-row tiles take the packed sweep, as in k_pair
    constexpr bool PACKED = TMNB_PACKED_FORCES && RG == 16 && DX && !U && !DL && !DP;
    const int lane = threadIdx.x & 31;
    const int total = prefix[R];
    for (;;) {
        int unit = 0;
        if (lane == 0) {
            unit = atomicAdd(counter, 1);
        }
        unit = __shfl_sync(FULL_MASK, unit, 0);
        if (unit >= total) {
            break;
        }
        const int q = replica_of(prefix, R, unit);
        const Rep &r = reps[q];
        const PairArgs a = pair_args(r);
        const int local = unit - prefix[q];
        const float box_x = (float)r.box[0], box_y = (float)r.box[4], box_z = (float)r.box[8];
        const float inv_box_x = 1 / box_x, inv_box_y = 1 / box_y, inv_box_z = 1 / box_z;
        const float real_cutoff = (float)r.cutoff;
        const float cutoff_squared = real_cutoff * real_cutoff;
        const float beta = (float)r.beta;
        const unsigned S = (unsigned)r.N;
        const int n_items = r.state->n_items;
        if (local >= n_items) {
            const int pair = (local - n_items) * TILE + lane;
            if (pair < r.M) {
                const int si = r.slot_of[r.pair_idxs[2 * pair + 0]];
                const int sj = r.slot_of[r.pair_idxs[2 * pair + 1]];
                scaled_pair<float, U, DX, DL, DP, false>(
                    a, pair, si, sj, 0, a.acc, box_x, box_y, box_z, inv_box_x, inv_box_y, inv_box_z, cutoff_squared);
            }
            continue;
        }
        const int4 it = r.items[local];
        if constexpr (PACKED) {
            const unsigned ia = (unsigned)(it.x * RG + (lane & 7));
            RowForces A, B;
            for (int t = 0; t < it.z; t++) {
                const long long tile = (long long)it.y + t;
                const unsigned j = r.tile_cols[tile * TILE + lane];
                tile_forces_p2<U, DX>(a, lane, S, ia, j, 0, a.acc, box_x, box_y, box_z, inv_box_x, inv_box_y, inv_box_z,
                               cutoff_squared, beta, A, B);
            }
            flush_forces_p2<U, DX>(a.acc, ia, S, A, B);
            continue;
        }
        const unsigned i = (unsigned)(it.x * RG + (lane & (RG - 1)));
        unsigned long long gi_x = 0, gi_y = 0, gi_z = 0, g_qi = 0, g_sigi = 0, g_epsi = 0, du_dl = 0, energy = 0;
        for (int t = 0; t < it.z; t++) {
            const long long tile = (long long)it.y + t;
            const unsigned j = r.tile_cols[tile * TILE + lane];
            tile_pass<float, U, DX, DL, DP, false, RG>(
                a, lane, S, i, j, 0, a.acc, box_x, box_y, box_z, inv_box_x, inv_box_y, inv_box_z, cutoff_squared, beta,
                gi_x, gi_y, gi_z, g_qi, g_sigi, g_epsi, du_dl, energy);
        }
        flush_row_rg<RG, U, DX, DL, DP>(a.acc, i, i < S, gi_x, gi_y, gi_z, g_qi, g_sigi, g_epsi, du_dl, energy);
    }
}

// Slot accumulators -> the replica's original-order outputs (+=); k_b_zero_acc
// then clears the accumulators.
__global__ void k_b_finalize(const Rep *__restrict__ reps, const int2 *__restrict__ ablk, int flags) {
    const int2 m = ablk[blockIdx.x];
    const Rep &r = reps[m.x];
    const int atom = m.y + threadIdx.x;
    if (atom >= r.N) {
        return;
    }
    const bool ok = r.state->error == 0;
    const int s = r.slot_of[atom];
    const size_t N = r.N;
    unsigned long long *acc = r.acc;
    if (flags & 4) {
        const unsigned long long vx = acc[0 * N + s], vy = acc[1 * N + s], vz = acc[2 * N + s];
        if (ok) {
            r.du_dx[3 * (size_t)atom + 0] += vx;
            r.du_dx[3 * (size_t)atom + 1] += vy;
            r.du_dx[3 * (size_t)atom + 2] += vz;
        }
    }
    if (flags & 1) {
        const unsigned long long q = acc[3 * N + s], sg = acc[4 * N + s], ep = acc[5 * N + s];
        if (ok) {
            r.du_dp[3 * (size_t)atom + 0] += q;
            r.du_dp[3 * (size_t)atom + 1] += sg;
            r.du_dp[3 * (size_t)atom + 2] += ep;
        }
    }
    if (flags & 8) {
        const unsigned long long vu = acc[6 * N + s];
        if (ok) {
            r.u[atom] += vu;
        }
    }
    if (flags & 2) {
        const unsigned long long vl = acc[7 * N + s];
        if (ok) {
            r.du_dl[atom] += vl;
        }
    }
}

// Zeroes the selected outputs of every replica.
// Zeroes the slot accumulators k_b_finalize read, in slot order (coalesced;
// zeroing each one at its gathered read measured ~30x slower).
__global__ void k_b_zero_acc(const Rep *__restrict__ reps, const int2 *__restrict__ ablk, int flags) {
    const int2 m = ablk[blockIdx.x];
    const Rep &r = reps[m.x];
    const int s = m.y + threadIdx.x;
    if (s >= r.N) {
        return;
    }
    const size_t N = r.N;
    unsigned long long *acc = r.acc;
    for (int k = 0; k < 3; k++) {
        if (flags & 4) {
            acc[k * N + s] = 0;
        }
        if (flags & 1) {
            acc[(3 + k) * N + s] = 0;
        }
    }
    if (flags & 8) {
        acc[6 * N + s] = 0;
    }
    if (flags & 2) {
        acc[7 * N + s] = 0;
    }
}

__global__ void k_b_zero_outputs(const Rep *__restrict__ reps, const int2 *__restrict__ ablk, int flags) {
    const int2 m = ablk[blockIdx.x];
    const Rep &r = reps[m.x];
    const int atom = m.y + threadIdx.x;
    if (atom >= r.N) {
        return;
    }
    for (int d = 0; d < 3; d++) {
        if (flags & 4) {
            r.du_dx[3 * (size_t)atom + d] = 0;
        }
        if (flags & 1) {
            r.du_dp[3 * (size_t)atom + d] = 0;
        }
    }
    if (flags & 8) {
        r.u[atom] = 0;
    }
    if (flags & 2) {
        r.du_dl[atom] = 0;
    }
}

// Harmonic bonds / angles of every replica (map: replica, first term).
__global__ void k_b_bonds(const Rep *__restrict__ reps, const int2 *__restrict__ bmap, int flags) {
    const int2 m = bmap[blockIdx.x];
    const Rep &r = reps[m.x];
    const int b = m.y + threadIdx.x;
    if (b >= r.n_bonds || r.state->error) {
        return;
    }
    harmonic_bond_term(
        r.x, r.bond_idxs[2 * b], r.bond_idxs[2 * b + 1], r.bond_params[2 * b], r.bond_params[2 * b + 1], 0, 1, r.lambda,
        (flags & 4) ? r.du_dx : nullptr, nullptr, nullptr, (flags & 8) ? r.u : nullptr);
}

__global__ void k_b_angles(const Rep *__restrict__ reps, const int2 *__restrict__ amap, int flags) {
    const int2 m = amap[blockIdx.x];
    const Rep &r = reps[m.x];
    const int a = m.y + threadIdx.x;
    if (a >= r.n_angles || r.state->error) {
        return;
    }
    harmonic_angle_term(
        r.x, r.angle_idxs[3 * a], r.angle_idxs[3 * a + 1], r.angle_idxs[3 * a + 2], r.angle_params[2 * a],
        r.angle_params[2 * a + 1], 0, 1, r.lambda, (flags & 4) ? r.du_dx : nullptr, nullptr, nullptr,
        (flags & 8) ? r.u : nullptr);
}

__global__ void k_b_langevin(const Rep *__restrict__ reps, const int2 *__restrict__ ablk) {
    const int2 m = ablk[blockIdx.x];
    const Rep &r = reps[m.x];
    const int i = m.y + threadIdx.x;
    if (i >= r.N) {
        return;
    }
    const unsigned long long step = *r.md_step;
    langevin_atom(i, step, r.key, r.ca, r.cbs[i], r.ccs[i], r.dt, r.x, r.v, r.du_dx);
}

__global__ void k_b_step_done(const Rep *__restrict__ reps, int R) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q < R) {
        *reps[q].md_step += 1;
    }
}

typedef void (*bpair_t)(const Rep *, int, const int *, int *);
template <int I, int RG> constexpr bpair_t bpair() {
    return &k_b_pair<(I >> 3) & 1, (I >> 2) & 1, (I >> 1) & 1, I & 1, RG>;
}
// [row-group size index: 0 -> 32, 1 -> 16, 2 -> 8][output flags]
template <int... Is> struct BPairTable {
    static void fill(bpair_t (*out)[16]) {
        ((out[0][Is] = bpair<Is, 32>()), ...);
        ((out[1][Is] = bpair<Is, 16>()), ...);
        ((out[2][Is] = bpair<Is, 8>()), ...);
    }
};

size_t align256(size_t b) { return (b + 255) & ~size_t(255); }

} // namespace

// Host description of one system (host arrays; the batch keeps copies).
struct BatchSystem {
    int N;
    const double *x, *v, *box, *params;
    const int *plane, *offset;
    int M;
    const int *pair_idxs;
    const double *scales;
    int B;
    const int *bond_idxs;
    const double *bond_params;
    int A;
    const int *angle_idxs;
    const double *angle_params;
    const double *cbs, *ccs; // Langevin per-atom coefficients (nullable: no MD)
    double beta, cutoff, lambda, ca, dt;
    unsigned long long seed;
};

// A replica's device arena, allocated and freed in stream order on the
// engine's stream (cudaMallocAsync / cudaFreeAsync from the device's default
// memory pool). Unlike cudaFree, releasing it does not wait for the whole
// device, so removing a finished replica does not stall on work that another
// engine has in flight.
struct StreamArena {
    unsigned char *p = nullptr;
    size_t n = 0;
    cudaStream_t stream = nullptr;
    StreamArena() = default;
    StreamArena(const StreamArena &) = delete;
    StreamArena &operator=(const StreamArena &) = delete;
    ~StreamArena() { release(); }
    void release() {
        if (p) {
            cudaFreeAsync(p, stream);
        }
        p = nullptr;
        n = 0;
    }
    void alloc(size_t count, cudaStream_t s) {
        release();
        stream = s;
        CK(cudaMallocAsync(reinterpret_cast<void **>(&p), count, s));
        n = count;
    }
};

// Host-to-device copy into a device buffer that grows by doubling, on `s`
// (a buffer only reallocates, with its device-wide cudaFree, when it grows).
template <typename T> void upload_on(DevBuf<T> &b, const T *h, size_t n, cudaStream_t s) {
    if (b.n < n) {
        b.alloc(std::max(n, 2 * b.n));
    }
    CK(cudaMemcpyAsync(b.p, h, n * sizeof(T), cudaMemcpyHostToDevice, s));
}

class BatchEngine {
  public:
    BatchEngine() {
        CK(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
        // keep freed arenas in the pool for reuse instead of returning them
        // to the driver at every synchronisation
        int dev = 0;
        CK(cudaGetDevice(&dev));
        cudaMemPool_t pool;
        CK(cudaDeviceGetDefaultMemPool(&pool, dev));
        unsigned long long keep = ~0ULL;
        CK(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep));
        BPairTable<0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 13, 14, 15>::fill(pair_kernels_);
        counter_.alloc(1);
        tcounter_.alloc(1);
    }
    ~BatchEngine() {
        drop_graphs();
        reps_.clear();
        if (stream_) {
            cudaStreamDestroy(stream_);
        }
    }

    void set_tuning(int chunk, double padding, int grid_bits_offset, int pair_ctas_per_sm) {
        if (chunk < 1 || !(padding >= 0) || grid_bits_offset < -2 || grid_bits_offset > 2 || pair_ctas_per_sm < 0) {
            throw Error(TMNB_ERR_INVALID_ARGUMENT, "invalid tuning parameters");
        }
        chunk_ = chunk;
        padding_ = padding;
        bits_off_ = grid_bits_offset;
        pair_ctas_ = pair_ctas_per_sm;
        // every replica is re-laid out; the new geometry takes effect at its (forced) rebuild
        for (auto &kv : reps_) {
            reconfigure(*kv.second);
        }
        table_dirty_ = true;
    }

    // Slots per row group of the replicas' tile lists (32, 16 or 8); every
    // replica is re-laid out and rebuilds its list.
    void set_tile_rows(int rows) {
        if (rows != 32 && rows != 16 && rows != 8) {
            throw Error(TMNB_ERR_INVALID_ARGUMENT, "rows per tile must be 32, 16 or 8");
        }
        rows_ = rows;
        for (auto &kv : reps_) {
            reconfigure(*kv.second);
        }
        table_dirty_ = true;
    }

    int add(const BatchSystem &s) {
        if (s.N <= 0 || !s.x || !s.box || !s.params || !s.plane || !s.offset) {
            throw Error(TMNB_ERR_INVALID_ARGUMENT, "system needs N > 0, x, box, params, plane and offset");
        }
        if (s.M < 0 || (s.M > 0 && (!s.pair_idxs || !s.scales)) || s.B < 0 || (s.B > 0 && (!s.bond_idxs || !s.bond_params)) ||
            s.A < 0 || (s.A > 0 && (!s.angle_idxs || !s.angle_params))) {
            throw Error(TMNB_ERR_INVALID_ARGUMENT, "invalid term lists");
        }
        for (int k = 0; k < 2 * s.M; k++) {
            if (s.pair_idxs[k] < 0 || s.pair_idxs[k] >= s.N) {
                throw Error(TMNB_ERR_INVALID_ARGUMENT, "pair index out of range [0, N)");
            }
        }
        for (int k = 0; k < 2 * s.B; k++) {
            if (s.bond_idxs[k] < 0 || s.bond_idxs[k] >= s.N) {
                throw Error(TMNB_ERR_INVALID_ARGUMENT, "bond index out of range [0, N)");
            }
        }
        for (int k = 0; k < 3 * s.A; k++) {
            if (s.angle_idxs[k] < 0 || s.angle_idxs[k] >= s.N) {
                throw Error(TMNB_ERR_INVALID_ARGUMENT, "angle index out of range [0, N)");
            }
        }
        auto slot = std::make_unique<Slot>();
        slot->keep(s);
        slot->has_md = s.cbs != nullptr && s.ccs != nullptr;
        allocate(*slot, slot->sys);
        const int id = next_id_++;
        reps_[id] = std::move(slot);
        table_dirty_ = true;
        return id;
    }

    void remove(int id) {
        auto it = reps_.find(id);
        if (it == reps_.end()) {
            throw Error(TMNB_ERR_INVALID_ARGUMENT, "unknown replica id " + std::to_string(id));
        }
        CK(cudaStreamSynchronize(stream_));
        reps_.erase(it);
        table_dirty_ = true;
    }

    // Device bytes one replica of N atoms (M scaled pairs, B bonds, A angles) holds.
    size_t footprint(int N, int M, int B, int A) const {
        if (N <= 0 || M < 0 || B < 0 || A < 0) {
            throw Error(TMNB_ERR_INVALID_ARGUMENT, "footprint needs N > 0 and non-negative term counts");
        }
        return layout(N, M, B, A).total;
    }

    size_t bytes_in_use() const {
        size_t b = 0;
        for (auto &kv : reps_) {
            b += kv.second->arena.n;
        }
        return b;
    }

    // One evaluation of every replica at its coordinates and lambda; flags as
    // the kernel index (bit3 u, bit2 du_dx, bit1 du_dl, bit0 du_dp). Outputs
    // are overwritten.
    void evaluate(int flags) {
        sync_table();
        if (R_ == 0 || flags == 0) {
            return;
        }
        k_b_zero_outputs<<<n_ablk_, ATOM_BLOCK, 0, stream_>>>(table_.p, ablk_.p, flags);
        record_nonbonded(flags);
        record_bonded(flags);
        CK(cudaPeekAtLastError());
    }

    // n_steps Langevin steps of every replica (all need MD coefficients).
    // use_graph: the chunk of `chunk` steps is captured once and replayed.
    void md(int n_steps, int chunk, bool use_graph) {
        sync_table();
        if (R_ == 0 || n_steps <= 0) {
            return;
        }
        for (auto &kv : reps_) {
            if (!kv.second->has_md) {
                throw Error(TMNB_ERR_INVALID_ARGUMENT, "replica " + std::to_string(kv.first) + " has no MD coefficients");
            }
        }
        chunk = std::max(1, std::min(chunk, n_steps));
        // the force accumulators start each step at zero (an evaluation may have left outputs there)
        k_b_zero_outputs<<<n_ablk_, ATOM_BLOCK, 0, stream_>>>(table_.p, ablk_.p, 4);
        int done = 0;
        if (use_graph) {
            cudaGraphExec_t g = graph_for(chunk);
            while (done + chunk <= n_steps) {
                CK(cudaGraphLaunch(g, stream_));
                done += chunk;
            }
        }
        for (; done < n_steps; done++) {
            record_md_step();
        }
        CK(cudaPeekAtLastError());
    }

    void synchronize() { CK(cudaStreamSynchronize(stream_)); }

    // Copies replica `id`'s state or outputs to host (synchronises):
    // which: 0 x, 1 v, 2 box (doubles), 3 du_dx, 4 du_dp, 5 du_dl, 6 u (int64 fixed point).
    void get(int id, int which, void *out) {
        Slot &s = slot(id);
        CK(cudaStreamSynchronize(stream_));
        const Rep &r = s.rep;
        const size_t N = r.N;
        const void *src = nullptr;
        size_t bytes = 0;
        switch (which) {
        case 0:
            src = r.x, bytes = 24 * N;
            break;
        case 1:
            src = r.v, bytes = 24 * N;
            break;
        case 2:
            src = r.box, bytes = 72;
            break;
        case 3:
            src = r.du_dx, bytes = 24 * N;
            break;
        case 4:
            src = r.du_dp, bytes = 24 * N;
            break;
        case 5:
            src = r.du_dl, bytes = 8 * N;
            break;
        case 6:
            src = r.u, bytes = 8 * N;
            break;
        default:
            throw Error(TMNB_ERR_INVALID_ARGUMENT, "unknown state selector");
        }
        CK(cudaMemcpyAsync(out, src, bytes, cudaMemcpyDeviceToHost, stream_));
        CK(cudaStreamSynchronize(stream_));
    }

    // Overwrites replica `id`'s coordinates (0), velocities (1) or box (2).
    void set(int id, int which, const double *in) {
        if (which < 0 || which > 2) {
            throw Error(TMNB_ERR_INVALID_ARGUMENT, "unknown state selector");
        }
        Slot &s = slot(id);
        CK(cudaStreamSynchronize(stream_));
        const Rep &r = s.rep;
        const size_t n = which == 2 ? 9 : 3 * (size_t)r.N;
        double *dst = which == 0 ? r.x : (which == 1 ? r.v : r.box);
        CK(cudaMemcpyAsync(dst, in, n * 8, cudaMemcpyHostToDevice, stream_));
        CK(cudaStreamSynchronize(stream_));
    }

    // Sticky device error of replica `id` (0: none); cleared when read.
    int error(int id) {
        Slot &s = slot(id);
        CK(cudaStreamSynchronize(stream_));
        int e = 0;
        CK(cudaMemcpyAsync(&e, &s.rep.state->error, sizeof(int), cudaMemcpyDeviceToHost, stream_));
        CK(cudaStreamSynchronize(stream_));
        if (e) {
            const int z = 0;
            CK(cudaMemcpyAsync(&s.rep.state->error, &z, sizeof(int), cudaMemcpyHostToDevice, stream_));
            CK(cudaStreamSynchronize(stream_));
        }
        return e;
    }

    void stats(int id, int *tiles, int *items, int *rebuilds) {
        Slot &s = slot(id);
        CK(cudaStreamSynchronize(stream_));
        DevState st;
        CK(cudaMemcpyAsync(&st, s.rep.state, sizeof(st), cudaMemcpyDeviceToHost, stream_));
        CK(cudaStreamSynchronize(stream_));
        if (tiles) {
            *tiles = (int)st.total_tiles;
        }
        if (items) {
            *items = st.n_items;
        }
        if (rebuilds) {
            *rebuilds = st.rebuilds;
        }
    }

    int size() const { return (int)reps_.size(); }
    cudaStream_t stream() const { return stream_; }

    // Scheduling priority of the batch's stream (cudaStreamCreateWithPriority;
    // lower numbers run first where blocks of several streams wait for SMs).
    // The stream is replaced after the work on it finished; captured graphs
    // are dropped.
    void set_priority(int priority) {
        int least = 0, greatest = 0;
        CK(cudaDeviceGetStreamPriorityRange(&least, &greatest));
        priority = std::max(greatest, std::min(least, priority));
        CK(cudaStreamSynchronize(stream_));
        drop_graphs();
        cudaStream_t s = nullptr;
        CK(cudaStreamCreateWithPriority(&s, cudaStreamNonBlocking, priority));
        // arenas were allocated in order on the old stream: it has finished
        for (auto &kv : reps_) {
            kv.second->arena.stream = s;
        }
        CK(cudaStreamDestroy(stream_));
        stream_ = s;
    }

  private:
    struct Layout {
        size_t x, v, box, p, plane, offset, pairs, scales, bonds, bparams, angles, aparams, cbs, ccs;
        size_t posw, prm, lamdep, keys, perm, slot_of, nb_x, nb_box, bins_count, bins_cursor, bb_ctr, bb_ext, rb_ntiles;
        size_t tile_cols, items, acc, du_dx, du_dp, du_dl, u, md_step, state;
        size_t total;
        int RB, NG, grid_bits, item_cap;
        long long tiles;
    };

    struct Slot {
        BatchSystem sys; // pointers into the host copies below
        bool has_md = false;
        StreamArena arena;
        Rep rep;
        std::vector<double> h_x, h_v, h_box, h_p, h_scales, h_bparams, h_aparams, h_cbs, h_ccs;
        std::vector<int> h_plane, h_offset, h_pairs, h_bonds, h_angles;

        // Host copies of the system's arrays (the caller's may go away).
        void keep(const BatchSystem &s) {
            const size_t N = s.N;
            auto cp = [](auto &dst, const auto *src, size_t n) {
                if (src) {
                    dst.assign(src, src + n);
                }
                return src ? dst.data() : nullptr;
            };
            sys = s;
            sys.x = cp(h_x, s.x, 3 * N);
            sys.v = cp(h_v, s.v, 3 * N);
            sys.box = cp(h_box, s.box, 9);
            sys.params = cp(h_p, s.params, 3 * N);
            sys.plane = cp(h_plane, s.plane, N);
            sys.offset = cp(h_offset, s.offset, N);
            sys.pair_idxs = cp(h_pairs, s.pair_idxs, 2 * (size_t)s.M);
            sys.scales = cp(h_scales, s.scales, 2 * (size_t)s.M);
            sys.bond_idxs = cp(h_bonds, s.bond_idxs, 2 * (size_t)s.B);
            sys.bond_params = cp(h_bparams, s.bond_params, 2 * (size_t)s.B);
            sys.angle_idxs = cp(h_angles, s.angle_idxs, 3 * (size_t)s.A);
            sys.angle_params = cp(h_aparams, s.angle_params, 2 * (size_t)s.A);
            sys.cbs = cp(h_cbs, s.cbs, N);
            sys.ccs = cp(h_ccs, s.ccs, N);
        }
    };

    int grid_bits_for(int N) const {
        const int b = (int)std::ceil(std::log2(std::cbrt(std::max(1.0, N / 8.0)))) + bits_off_;
        return std::min(6, std::max(2, b));
    }

    Layout layout(int N, int M, int B, int A) const {
        Layout L{};
        L.RB = (N + TILE - 1) / TILE;
        L.NG = (N + rows_ - 1) / rows_;
        L.grid_bits = grid_bits_for(N);
        L.tiles = tile_base_rows(L.NG, rows_, L.RB, 0, 0);
        long long cap = 0;
        for (int g = 0; g < L.NG; g++) {
            cap += ((L.RB - (long long)g * rows_ / TILE) + chunk_ - 1) / chunk_;
        }
        L.item_cap = (int)std::max(1LL, cap);
        const size_t bins = (size_t)1 << (3 * L.grid_bits);
        size_t o = 0;
        auto take = [&](size_t bytes) {
            const size_t at = o;
            o += align256(std::max<size_t>(bytes, 1));
            return at;
        };
        L.x = take(24 * (size_t)N);
        L.v = take(24 * (size_t)N);
        L.box = take(72);
        L.p = take(24 * (size_t)N);
        L.plane = take(4 * (size_t)N);
        L.offset = take(4 * (size_t)N);
        L.pairs = take(8 * (size_t)M);
        L.scales = take(16 * (size_t)M);
        L.bonds = take(8 * (size_t)B);
        L.bparams = take(16 * (size_t)B);
        L.angles = take(12 * (size_t)A);
        L.aparams = take(16 * (size_t)A);
        L.cbs = take(8 * (size_t)N);
        L.ccs = take(8 * (size_t)N);
        L.posw = take(16 * (size_t)N);
        L.prm = take(16 * (size_t)N);
        L.lamdep = take((size_t)N);
        L.keys = take(4 * (size_t)N);
        L.perm = take(4 * (size_t)N);
        L.slot_of = take(4 * (size_t)N);
        L.nb_x = take(24 * (size_t)N);
        L.nb_box = take(72);
        L.bins_count = take(4 * bins);
        L.bins_cursor = take(4 * bins);
        L.bb_ctr = take(16 * (size_t)L.RB);
        L.bb_ext = take(16 * (size_t)L.RB);
        L.rb_ntiles = take(4 * (size_t)L.NG);
        L.tile_cols = take(4 * (size_t)TILE * L.tiles);
        L.items = take(16 * (size_t)L.item_cap);
        L.acc = take(64 * (size_t)N);
        L.du_dx = take(24 * (size_t)N);
        L.du_dp = take(24 * (size_t)N);
        L.du_dl = take(8 * (size_t)N);
        L.u = take(8 * (size_t)N);
        L.md_step = take(8);
        L.state = take(sizeof(DevState));
        L.total = o;
        return L;
    }

    void allocate(Slot &slot, const BatchSystem &s) {
        const Layout L = layout(s.N, s.M, s.B, s.A);
        slot.arena.alloc(L.total, stream_);
        CK(cudaMemsetAsync(slot.arena.p, 0, L.total, stream_));
        unsigned char *b = slot.arena.p;
        Rep &r = slot.rep;
        r.N = s.N;
        r.RB = L.RB;
        r.rows = rows_;
        r.NG = L.NG;
        r.grid_bits = L.grid_bits;
        r.M = s.M;
        r.n_bonds = s.B;
        r.n_angles = s.A;
        r.chunk = chunk_;
        r.item_cap = L.item_cap;
        r.lambda = s.lambda;
        r.beta = s.beta;
        r.cutoff = s.cutoff;
        r.padding = padding_;
        r.ca = s.ca;
        r.dt = s.dt;
        r.key = make_uint2((unsigned)s.seed, (unsigned)(s.seed >> 32) ^ 0x5bd1e995u);
        r.x = reinterpret_cast<double *>(b + L.x);
        r.v = reinterpret_cast<double *>(b + L.v);
        r.box = reinterpret_cast<double *>(b + L.box);
        r.p = reinterpret_cast<double *>(b + L.p);
        r.plane = reinterpret_cast<int *>(b + L.plane);
        r.offset = reinterpret_cast<int *>(b + L.offset);
        r.pair_idxs = reinterpret_cast<int *>(b + L.pairs);
        r.scales = reinterpret_cast<double *>(b + L.scales);
        r.bond_idxs = reinterpret_cast<int *>(b + L.bonds);
        r.bond_params = reinterpret_cast<double *>(b + L.bparams);
        r.angle_idxs = reinterpret_cast<int *>(b + L.angles);
        r.angle_params = reinterpret_cast<double *>(b + L.aparams);
        r.cbs = reinterpret_cast<double *>(b + L.cbs);
        r.ccs = reinterpret_cast<double *>(b + L.ccs);
        r.posw = reinterpret_cast<float4 *>(b + L.posw);
        r.prm = reinterpret_cast<float4 *>(b + L.prm);
        r.lamdep = b + L.lamdep;
        r.keys = reinterpret_cast<unsigned *>(b + L.keys);
        r.perm = reinterpret_cast<unsigned *>(b + L.perm);
        r.slot_of = reinterpret_cast<int *>(b + L.slot_of);
        r.nb_x = reinterpret_cast<double *>(b + L.nb_x);
        r.nb_box = reinterpret_cast<double *>(b + L.nb_box);
        r.bin_count = reinterpret_cast<int *>(b + L.bins_count);
        r.bin_cursor = reinterpret_cast<int *>(b + L.bins_cursor);
        r.bb_ctr = reinterpret_cast<float4 *>(b + L.bb_ctr);
        r.bb_ext = reinterpret_cast<float4 *>(b + L.bb_ext);
        r.rb_ntiles = reinterpret_cast<int *>(b + L.rb_ntiles);
        r.tile_cols = reinterpret_cast<unsigned *>(b + L.tile_cols);
        r.items = reinterpret_cast<int4 *>(b + L.items);
        r.acc = reinterpret_cast<unsigned long long *>(b + L.acc);
        r.du_dx = reinterpret_cast<unsigned long long *>(b + L.du_dx);
        r.du_dp = reinterpret_cast<unsigned long long *>(b + L.du_dp);
        r.du_dl = reinterpret_cast<unsigned long long *>(b + L.du_dl);
        r.u = reinterpret_cast<unsigned long long *>(b + L.u);
        r.md_step = reinterpret_cast<unsigned long long *>(b + L.md_step);
        r.state = reinterpret_cast<DevState *>(b + L.state);
        const size_t N = s.N;
        CK(cudaMemcpyAsync(r.x, s.x, 24 * N, cudaMemcpyHostToDevice, stream_));
        if (s.v) {
            CK(cudaMemcpyAsync(r.v, s.v, 24 * N, cudaMemcpyHostToDevice, stream_));
        }
        CK(cudaMemcpyAsync(r.box, s.box, 72, cudaMemcpyHostToDevice, stream_));
        CK(cudaMemcpyAsync((void *)r.p, s.params, 24 * N, cudaMemcpyHostToDevice, stream_));
        CK(cudaMemcpyAsync((void *)r.plane, s.plane, 4 * N, cudaMemcpyHostToDevice, stream_));
        CK(cudaMemcpyAsync((void *)r.offset, s.offset, 4 * N, cudaMemcpyHostToDevice, stream_));
        if (s.M > 0) {
            CK(cudaMemcpyAsync((void *)r.pair_idxs, s.pair_idxs, 8 * (size_t)s.M, cudaMemcpyHostToDevice, stream_));
            CK(cudaMemcpyAsync((void *)r.scales, s.scales, 16 * (size_t)s.M, cudaMemcpyHostToDevice, stream_));
        }
        if (s.B > 0) {
            CK(cudaMemcpyAsync((void *)r.bond_idxs, s.bond_idxs, 8 * (size_t)s.B, cudaMemcpyHostToDevice, stream_));
            CK(cudaMemcpyAsync((void *)r.bond_params, s.bond_params, 16 * (size_t)s.B, cudaMemcpyHostToDevice, stream_));
        }
        if (s.A > 0) {
            CK(cudaMemcpyAsync((void *)r.angle_idxs, s.angle_idxs, 12 * (size_t)s.A, cudaMemcpyHostToDevice, stream_));
            CK(cudaMemcpyAsync((void *)r.angle_params, s.angle_params, 16 * (size_t)s.A, cudaMemcpyHostToDevice, stream_));
        }
        if (s.cbs && s.ccs) {
            CK(cudaMemcpyAsync((void *)r.cbs, s.cbs, 8 * N, cudaMemcpyHostToDevice, stream_));
            CK(cudaMemcpyAsync((void *)r.ccs, s.ccs, 8 * N, cudaMemcpyHostToDevice, stream_));
        }
        // identity slot order until the first (forced) rebuild
        std::vector<unsigned> perm(N);
        std::vector<int> slot_of(N);
        for (size_t k = 0; k < N; k++) {
            perm[k] = (unsigned)k;
            slot_of[k] = (int)k;
        }
        CK(cudaMemcpyAsync(r.perm, perm.data(), 4 * N, cudaMemcpyHostToDevice, stream_));
        CK(cudaMemcpyAsync(r.slot_of, slot_of.data(), 4 * N, cudaMemcpyHostToDevice, stream_));
        DevState st{};
        st.rebuild = 1;
        CK(cudaMemcpyAsync(r.state, &st, sizeof(st), cudaMemcpyHostToDevice, stream_));
        // the host staging (perm, slot_of, st) is local: finish the copies here
        CK(cudaStreamSynchronize(stream_));
    }

    // New tuning: re-lay the replica out (arena sizes depend on the chunk and
    // the Hilbert grid), keeping its coordinates, velocities, box and MD step.
    void reconfigure(Slot &slot) {
        CK(cudaStreamSynchronize(stream_));
        const int N = slot.rep.N;
        std::vector<double> x(3 * (size_t)N), v(3 * (size_t)N), box(9);
        unsigned long long step = 0;
        CK(cudaMemcpyAsync(x.data(), slot.rep.x, 24 * (size_t)N, cudaMemcpyDeviceToHost, stream_));
        CK(cudaMemcpyAsync(v.data(), slot.rep.v, 24 * (size_t)N, cudaMemcpyDeviceToHost, stream_));
        CK(cudaMemcpyAsync(box.data(), slot.rep.box, 72, cudaMemcpyDeviceToHost, stream_));
        CK(cudaMemcpyAsync(&step, slot.rep.md_step, 8, cudaMemcpyDeviceToHost, stream_));
        CK(cudaStreamSynchronize(stream_));
        BatchSystem s = slot.sys;
        s.x = x.data();
        s.v = v.data();
        s.box = box.data();
        allocate(slot, s);
        CK(cudaMemcpyAsync(slot.rep.md_step, &step, 8, cudaMemcpyHostToDevice, stream_));
        CK(cudaStreamSynchronize(stream_));
    }

    Slot &slot(int id) {
        auto it = reps_.find(id);
        if (it == reps_.end()) {
            throw Error(TMNB_ERR_INVALID_ARGUMENT, "unknown replica id " + std::to_string(id));
        }
        return *it->second;
    }

    void sync_table() {
        if (!table_dirty_) {
            return;
        }
        CK(cudaStreamSynchronize(stream_));
        drop_graphs();
        std::vector<Rep> table;
        std::vector<int2> ablk, rbmap, bmap, amap;
        int n_groups = 0; // row groups of all replicas
        int q = 0;
        for (auto &kv : reps_) {
            const Rep &r = kv.second->rep;
            table.push_back(r);
            for (int s0 = 0; s0 < r.N; s0 += ATOM_BLOCK) {
                ablk.push_back(make_int2(q, s0));
            }
            for (int rb = 0; rb < r.RB; rb++) {
                rbmap.push_back(make_int2(q, rb));
            }
            n_groups += r.NG;
            for (int b0 = 0; b0 < r.n_bonds; b0 += TERM_BLOCK) {
                bmap.push_back(make_int2(q, b0));
            }
            for (int a0 = 0; a0 < r.n_angles; a0 += TERM_BLOCK) {
                amap.push_back(make_int2(q, a0));
            }
            q++;
        }
        R_ = q;
        n_ablk_ = (int)ablk.size();
        n_rb_ = (int)rbmap.size();
        n_groups_ = n_groups;
        n_bmap_ = (int)bmap.size();
        n_amap_ = (int)amap.size();
        if (R_ > 0) {
            upload_on(table_, table.data(), table.size(), stream_);
            upload_on(ablk_, ablk.data(), ablk.size(), stream_);
            upload_on(rbmap_, rbmap.data(), rbmap.size(), stream_);
            if (n_bmap_) {
                upload_on(bmap_, bmap.data(), bmap.size(), stream_);
            }
            if (n_amap_) {
                upload_on(amap_, amap.data(), amap.size(), stream_);
            }
            prefix_.ensure(R_ + 1);
            tprefix_.ensure(R_ + 1);
            CK(cudaStreamSynchronize(stream_)); // the host tables above are local
        }
        table_dirty_ = false;
    }

    bpair_t pair_kernel(int flags) const { return pair_kernels_[rows_ == 32 ? 0 : (rows_ == 16 ? 1 : 2)][flags]; }

    // persistent tile-build CTAs: as many as are resident at once, and never
    // more than the row groups of all replicas
    int tiles_grid() {
        int per_sm = 0;
        CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_b_tiles, TB_WARPS * 32, 0));
        return std::max(1, std::min(std::max(1, per_sm) * num_sms(), n_groups_));
    }

    int pair_grid(int flags) {
        int per_sm = 0;
        CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, pair_kernel(flags), 128, 0));
        per_sm = std::max(1, per_sm);
        if (pair_ctas_ > 0) {
            per_sm = std::min(per_sm, pair_ctas_);
        }
        return per_sm * num_sms();
    }

    void record_nonbonded(int flags) {
        k_b_prepare<<<n_ablk_, ATOM_BLOCK, 0, stream_>>>(table_.p, ablk_.p);
        k_b_keys<<<n_ablk_, ATOM_BLOCK, 0, stream_>>>(table_.p, ablk_.p);
        k_b_scan<<<R_, 1024, 0, stream_>>>(table_.p);
        k_b_scatter<<<n_ablk_, ATOM_BLOCK, 0, stream_>>>(table_.p, ablk_.p);
        k_b_bounds<<<(n_rb_ * 32 + 255) / 256, 256, 0, stream_>>>(table_.p, rbmap_.p, n_rb_);
        k_b_tile_units<<<1, 1024, 0, stream_>>>(table_.p, R_, tprefix_.p, tcounter_.p);
        k_b_tiles<<<tiles_grid(), TB_WARPS * 32, 0, stream_>>>(table_.p, R_, tprefix_.p, tcounter_.p);
        k_b_units<<<1, 1024, 0, stream_>>>(table_.p, R_, prefix_.p, counter_.p);
        pair_kernel(flags)<<<pair_grid(flags), 128, 0, stream_>>>(table_.p, R_, prefix_.p, counter_.p);
        k_b_finalize<<<n_ablk_, ATOM_BLOCK, 0, stream_>>>(table_.p, ablk_.p, flags);
        k_b_zero_acc<<<n_ablk_, ATOM_BLOCK, 0, stream_>>>(table_.p, ablk_.p, flags);
    }

    void record_bonded(int flags) {
        if (!(flags & (4 | 8))) {
            return;
        }
        if (n_bmap_) {
            k_b_bonds<<<n_bmap_, TERM_BLOCK, 0, stream_>>>(table_.p, bmap_.p, flags);
        }
        if (n_amap_) {
            k_b_angles<<<n_amap_, TERM_BLOCK, 0, stream_>>>(table_.p, amap_.p, flags);
        }
    }

    void record_md_step() {
        record_nonbonded(4);
        record_bonded(4);
        k_b_langevin<<<n_ablk_, ATOM_BLOCK, 0, stream_>>>(table_.p, ablk_.p);
        k_b_step_done<<<(R_ + 255) / 256, 256, 0, stream_>>>(table_.p, R_);
    }

    cudaGraphExec_t graph_for(int steps) {
        auto it = graphs_.find(steps);
        if (it != graphs_.end()) {
            return it->second;
        }
        cudaGraph_t g = nullptr;
        CK(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeRelaxed));
        try {
            for (int k = 0; k < steps; k++) {
                record_md_step();
            }
        } catch (...) {
            cudaStreamEndCapture(stream_, &g);
            if (g) {
                cudaGraphDestroy(g);
            }
            throw;
        }
        CK(cudaStreamEndCapture(stream_, &g));
        cudaGraphExec_t ge;
        CK(cudaGraphInstantiate(&ge, g, 0));
        CK(cudaGraphDestroy(g));
        graphs_[steps] = ge;
        return ge;
    }

    void drop_graphs() {
        for (auto &kv : graphs_) {
            cudaGraphExecDestroy(kv.second);
        }
        graphs_.clear();
    }

    cudaStream_t stream_ = nullptr;
    std::map<int, std::unique_ptr<Slot>> reps_;
    int next_id_ = 0;
    bool table_dirty_ = true;
    int R_ = 0, n_ablk_ = 0, n_rb_ = 0, n_groups_ = 0, n_bmap_ = 0, n_amap_ = 0;
    DevBuf<Rep> table_;
    DevBuf<int2> ablk_, rbmap_, bmap_, amap_;
    DevBuf<int> prefix_, counter_, tprefix_, tcounter_;
    bpair_t pair_kernels_[3][16];
    int rows_ = 16; // slots per row group of every replica's tile list
    std::map<int, cudaGraphExec_t> graphs_;
    int chunk_ = 4;
    double padding_ = 0.1;
    int bits_off_ = 0;
    int pair_ctas_ = 0;
};

} // namespace tmb

struct tmnb_batch {
    std::unique_ptr<tmb::BatchEngine> impl;
};

namespace {
tmnb_status check_batch(const tmnb_batch *b) {
    if (!b || !b->impl) {
        tmb::g_last_error = "null batch handle";
        return TMNB_ERR_INVALID_ARGUMENT;
    }
    return TMNB_OK;
}

tmnb_status null_argument() {
    tmb::g_last_error = "null argument";
    return TMNB_ERR_INVALID_ARGUMENT;
}
} // namespace

extern "C" {

tmnb_status tmnb_batch_create(tmnb_batch **out) {
    if (!out) {
        return null_argument();
    }
    return tmb::guarded([&] {
        auto b = std::make_unique<tmnb_batch>();
        b->impl = std::make_unique<tmb::BatchEngine>();
        *out = b.release();
    });
}

tmnb_status tmnb_batch_set_priority(tmnb_batch *b, int priority) {
    if (!b) {
        return null_argument();
    }
    return tmb::guarded([&] { b->impl->set_priority(priority); });
}

tmnb_status tmnb_batch_destroy(tmnb_batch *b) {
    if (!b) {
        return TMNB_OK;
    }
    return tmb::guarded([&] { delete b; });
}

tmnb_status tmnb_batch_add(
    tmnb_batch *b,
    int N,
    const double *x,
    const double *v,
    const double *box,
    const double *params,
    const int32_t *lambda_plane_idxs,
    const int32_t *lambda_offset_idxs,
    int M,
    const int32_t *exclusion_idxs,
    const double *scales,
    int B,
    const int32_t *bond_idxs,
    const double *bond_params,
    int A,
    const int32_t *angle_idxs,
    const double *angle_params,
    double beta,
    double cutoff,
    double lambda,
    double dt,
    double ca,
    const double *cbs,
    const double *ccs,
    unsigned long long seed,
    int *id) {
    if (tmnb_status s = check_batch(b)) {
        return s;
    }
    if (!id) {
        return null_argument();
    }
    return tmb::guarded([&] {
        if (!(cutoff > 0)) {
            throw tmb::Error(TMNB_ERR_INVALID_ARGUMENT, "cutoff must be positive");
        }
        tmb::BatchSystem s{};
        s.N = N;
        s.x = x;
        s.v = v;
        s.box = box;
        s.params = params;
        s.plane = lambda_plane_idxs;
        s.offset = lambda_offset_idxs;
        s.M = M;
        s.pair_idxs = exclusion_idxs;
        s.scales = scales;
        s.B = B;
        s.bond_idxs = bond_idxs;
        s.bond_params = bond_params;
        s.A = A;
        s.angle_idxs = angle_idxs;
        s.angle_params = angle_params;
        s.beta = beta;
        s.cutoff = cutoff;
        s.lambda = lambda;
        s.dt = dt;
        s.ca = ca;
        s.cbs = cbs;
        s.ccs = ccs;
        s.seed = seed;
        *id = b->impl->add(s);
    });
}

tmnb_status tmnb_batch_remove(tmnb_batch *b, int id) {
    if (tmnb_status s = check_batch(b)) {
        return s;
    }
    return tmb::guarded([&] { b->impl->remove(id); });
}

tmnb_status tmnb_batch_footprint(tmnb_batch *b, int N, int M, int B, int A, unsigned long long *bytes) {
    if (tmnb_status s = check_batch(b)) {
        return s;
    }
    if (!bytes) {
        return null_argument();
    }
    return tmb::guarded([&] { *bytes = b->impl->footprint(N, M, B, A); });
}

tmnb_status tmnb_batch_bytes_in_use(tmnb_batch *b, unsigned long long *bytes) {
    if (tmnb_status s = check_batch(b)) {
        return s;
    }
    if (!bytes) {
        return null_argument();
    }
    return tmb::guarded([&] { *bytes = b->impl->bytes_in_use(); });
}

tmnb_status tmnb_batch_set_tile_rows(tmnb_batch *b, int rows) {
    if (tmnb_status s = check_batch(b)) {
        return s;
    }
    return tmb::guarded([&] { b->impl->set_tile_rows(rows); });
}

tmnb_status tmnb_batch_set_tuning(tmnb_batch *b, int chunk, double padding, int grid_bits_offset, int pair_ctas_per_sm) {
    if (tmnb_status s = check_batch(b)) {
        return s;
    }
    return tmb::guarded([&] { b->impl->set_tuning(chunk, padding, grid_bits_offset, pair_ctas_per_sm); });
}

tmnb_status tmnb_batch_evaluate(tmnb_batch *b, int compute_du_dx, int compute_du_dp, int compute_du_dl, int compute_u) {
    if (tmnb_status s = check_batch(b)) {
        return s;
    }
    const int flags = (compute_du_dp ? 1 : 0) | (compute_du_dl ? 2 : 0) | (compute_du_dx ? 4 : 0) | (compute_u ? 8 : 0);
    return tmb::guarded([&] { b->impl->evaluate(flags); });
}

tmnb_status tmnb_batch_md(tmnb_batch *b, int n_steps, int chunk, int use_graph) {
    if (tmnb_status s = check_batch(b)) {
        return s;
    }
    return tmb::guarded([&] { b->impl->md(n_steps, chunk, use_graph != 0); });
}

tmnb_status tmnb_batch_synchronize(tmnb_batch *b) {
    if (tmnb_status s = check_batch(b)) {
        return s;
    }
    return tmb::guarded([&] { b->impl->synchronize(); });
}

tmnb_status tmnb_batch_get(tmnb_batch *b, int id, int which, void *out) {
    if (tmnb_status s = check_batch(b)) {
        return s;
    }
    if (!out) {
        return null_argument();
    }
    return tmb::guarded([&] { b->impl->get(id, which, out); });
}

tmnb_status tmnb_batch_set(tmnb_batch *b, int id, int which, const double *in) {
    if (tmnb_status s = check_batch(b)) {
        return s;
    }
    if (!in) {
        return null_argument();
    }
    return tmb::guarded([&] { b->impl->set(id, which, in); });
}

tmnb_status tmnb_batch_error(tmnb_batch *b, int id, int *code) {
    if (tmnb_status s = check_batch(b)) {
        return s;
    }
    if (!code) {
        return null_argument();
    }
    return tmb::guarded([&] { *code = b->impl->error(id); });
}

tmnb_status tmnb_batch_stats(tmnb_batch *b, int id, int *tiles, int *items, int *rebuilds) {
    if (tmnb_status s = check_batch(b)) {
        return s;
    }
    return tmb::guarded([&] { b->impl->stats(id, tiles, items, rebuilds); });
}

tmnb_status tmnb_batch_stream(tmnb_batch *b, void **stream) {
    if (tmnb_status s = check_batch(b)) {
        return s;
    }
    if (!stream) {
        return null_argument();
    }
    *stream = static_cast<void *>(b->impl->stream());
    return TMNB_OK;
}

int tmnb_batch_size(const tmnb_batch *b) { return (b && b->impl) ? b->impl->size() : -1; }

} // extern "C"
