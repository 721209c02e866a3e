// MD runtime on top of the nonbonded potential: Langevin (BAOAB rotated by
// half a step) integrator, isotropic Monte Carlo barostat and a Context that
// replays each step as a CUDA graph. Nothing in a step synchronises with the
// host: the neighbour-list rebuild decision, the barostat's Metropolis test and
// the random numbers all live on the device.
//
// Semantics follow the reference runtime:
//   Context::_step               timemachine/cpp/src/context.cu:240-280
//   LangevinIntegrator/update_forward  timemachine/cpp/src/integrator.cu:37-86
//   MonteCarloBarostat::inplace_move   timemachine/cpp/src/barostat.cu:286-373
// The reference draws its Gaussian noise with cuRAND into a buffer; here a
// counter-based Philox4x32-10 generator (Salmon, Moraes, Dror, Shaw,
// "Parallel random numbers: as easy as 1, 2, 3", SC'11) is evaluated inside
// the integrator kernel, keyed by (seed, step, atom), so a step has no RNG
// launch and a replayed graph draws fresh numbers.
#include "engine.hpp"
#include "md_math.cuh"
#include "nb_pair_math.cuh"

#include <algorithm>
#include <map>
#include <vector>

namespace tmb {

namespace {

constexpr double BOLTZ = 0.008314462618; // kJ/mol/K
constexpr double AVOGADRO = 6.0221367e23;

struct MDState {
    unsigned long long step;  // integrator step counter (RNG counter)
    unsigned done_blocks;     // completion counter of k_langevin
    int dl_slot;              // next du_dl output slot
    // barostat
    unsigned long long move;  // barostat move counter (RNG counter)
    double volume_scale;
    double volume_delta;
    double length_scale;
    double rand0, rand1;
    int num_accepted;
    int num_attempted;
    int accepted;
    int total_accepted;
    int total_attempted;
    // the last move, as proposed and decided (inspection)
    double proposal_scale;                // volume scale the proposal used
    unsigned long long last_u_before;     // fixed-point total energy before the move
    unsigned long long last_u_after;      // and at the trial coordinates
};

__global__ void k_langevin(
    int N,
    double ca,
    const double *__restrict__ cbs,
    const double *__restrict__ ccs,
    double dt,
    double *__restrict__ x,
    double *__restrict__ v,
    unsigned long long *__restrict__ du_dx,
    uint2 key,
    MDState *st) {
    grid_dependency_wait();
    __shared__ unsigned long long s_step;
    if (threadIdx.x == 0) {
        s_step = st->step;
    }
    __syncthreads();
    // two threads per atom (halves of its Philox draws and components)
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int i = t >> 1;
    if (i < N) {
        langevin_atom_half(i, t & 1, s_step, key, ca, cbs[i], ccs[i], dt, x, v, du_dx);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        if (atomicAdd(&st->done_blocks, 1u) == gridDim.x - 1) {
            st->step += 1;
            st->done_blocks = 0;
        }
    }
}

// The integrator step fused with a potential's per-step staging and force
// scatter (MDFusion). Each atom's force adds the potential's slot-ordered
// fixed-point accumulator (what k_finalize would have added; integer sums, so
// the order does not matter); a memset after the kernel clears the
// accumulators for the next step (clearing each slot here, from the gathered
// reads, measured slower). With `stage_next` the
// new coordinates are staged into the potential's slots and the
// neighbour-list test of k_check_prepare is taken, so the next step's forces
// start at the rebuild chain and the pair kernel.
__global__ void k_langevin_fused(
    int N,
    double ca,
    const double *__restrict__ cbs,
    const double *__restrict__ ccs,
    double dt,
    double *__restrict__ x,
    double *__restrict__ v,
    unsigned long long *__restrict__ du_dx,
    uint2 key,
    MDState *st,
    MDFusion f,
    int stage_next) {
    grid_dependency_wait();
    __shared__ unsigned long long s_step;
    if (threadIdx.x == 0) {
        s_step = st->step;
    }
    __syncthreads();
    // two threads per atom, as k_langevin: half 0 updates x and y, half 1 z
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int i = t >> 1;
    const int half = t & 1;
    const bool ok = *f.error == 0; // k_finalize adds nothing after an error
    double c0 = 0.0, c1 = 0.0;     // the new coordinates: x, y (half 0) or z (half 1)
    int s = 0;
    if (i < N) {
        s = f.slot_of[i];
        const uint4 r = philox4x32_10(make_uint4((unsigned)i, (unsigned)s_step, (unsigned)(s_step >> 32), (unsigned)half), key);
        const double2 n = normal2(r.x, r.y, r.z, r.w);
        if (half == 0) {
            const unsigned long long ax = f.acc[s];
            const unsigned long long ay = f.acc[(size_t)f.S + s];
            c0 = langevin_dim(3 * i + 0, n.x, ca, cbs[i], ccs[i], dt, x, v, du_dx, ok ? ax : 0ull);
            c1 = langevin_dim(3 * i + 1, n.y, ca, cbs[i], ccs[i], dt, x, v, du_dx, ok ? ay : 0ull);
        } else {
            const unsigned long long az = f.acc[2 * (size_t)f.S + s];
            c0 = langevin_dim(3 * i + 2, n.x, ca, cbs[i], ccs[i], dt, x, v, du_dx, ok ? az : 0ull);
        }
    }
    if (stage_next) {
        // the pair of lanes (2m, 2m + 1) holds one atom; half 0 takes its z
        const double z_new = __shfl_down_sync(0xffffffffu, c0, 1);
        if (half == 0 && i < N) {
            // the staged values of k_check_prepare: FP32 coordinates, w kept
            *reinterpret_cast<float2 *>(f.posw + s) = make_float2((float)c0, (float)c1);
            reinterpret_cast<float *>(f.posw + s)[2] = (float)z_new;
            const double *xo = f.nb_x + 3 * (size_t)i;
            if (moved_beyond_half_padding(c0 - xo[0], c1 - xo[1], z_new - xo[2], f.half_pad2)) {
                *f.rebuild = 1; // benign race: every writer stores 1
            }
        }
        if (t == 0) {
            *f.next_item = 0;
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        if (atomicAdd(&st->done_blocks, 1u) == gridDim.x - 1) {
            st->step += 1;
            st->done_blocks = 0;
        }
    }
}

// Per-window sums of a [K][N] per-atom buffer into out[0..K) (one block per
// window); zeroes the buffer.
__global__ void k_reduce_windows(int N, unsigned long long *__restrict__ buf, unsigned long long *__restrict__ out) {
    __shared__ unsigned long long part[32];
    unsigned long long *row = buf + (size_t)blockIdx.x * N;
    unsigned long long acc = 0;
    for (int i = threadIdx.x; i < N; i += blockDim.x) {
        acc += row[i];
        row[i] = 0;
    }
    for (int o = 16; o > 0; o >>= 1) {
        acc += __shfl_xor_sync(0xffffffffu, acc, o);
    }
    if ((threadIdx.x & 31) == 0) {
        part[threadIdx.x >> 5] = acc;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned long long t = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) {
            t += part[w];
        }
        out[blockIdx.x] = t;
    }
}

// Sum of the per-atom du_dl buffer into the next output slot; zeroes the buffer.
__global__ void k_reduce_dl(int N, unsigned long long *__restrict__ buf, unsigned long long *__restrict__ out, MDState *st) {
    __shared__ unsigned long long part[32];
    unsigned long long acc = 0;
    for (int i = threadIdx.x; i < N; i += blockDim.x) {
        acc += buf[i];
        buf[i] = 0;
    }
    for (int o = 16; o > 0; o >>= 1) {
        acc += __shfl_xor_sync(0xffffffffu, acc, o);
    }
    if ((threadIdx.x & 31) == 0) {
        part[threadIdx.x >> 5] = acc;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned long long t = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) {
            t += part[w];
        }
        out[st->dl_slot] = t;
        st->dl_slot += 1;
    }
}

// Barostat proposal: volume change from a uniform draw, then group centroids
// in fixed point (timemachine/cpp/src/barostat.cu:186-228).
__global__ void k_baro_propose(
    int N,
    const double *__restrict__ x,
    const double *__restrict__ box,
    const int *__restrict__ group_of,
    unsigned long long *__restrict__ centroids,
    uint2 key,
    MDState *st) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i == 0) {
        const uint4 r = philox4x32_10(make_uint4((unsigned)st->move, (unsigned)(st->move >> 32), 0x9a7u, 0u), key);
        st->rand0 = u01(r.x, r.y);
        st->rand1 = u01(r.z, r.w);
        st->move += 1;
        const double volume = box[0] * box[4] * box[8];
        if (st->volume_scale == 0) {
            st->volume_scale = 0.01 * volume;
        }
        st->proposal_scale = st->volume_scale;
        const double delta_volume = st->volume_scale * 2 * (st->rand0 - 0.5);
        const double new_volume = volume + delta_volume;
        st->volume_delta = delta_volume;
        st->length_scale = cbrt(new_volume / volume);
    }
    if (i < N) {
        const int g = group_of[i];
        if (g >= 0) {
            for (int d = 0; d < 3; d++) {
                atomicAdd(centroids + 3 * g + d, (unsigned long long)llrint(x[3 * i + d] * FX_EXPONENT));
            }
        }
    }
}

// Scaled trial coordinates and box (timemachine/cpp/src/barostat.cu:140-184).
__global__ void k_baro_rescale(
    int N,
    const double *__restrict__ x,
    const double *__restrict__ box,
    const int *__restrict__ group_of,
    const int *__restrict__ group_size,
    const unsigned long long *__restrict__ centroids,
    double *__restrict__ x_after,
    double *__restrict__ box_after,
    const MDState *st) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const double scale = st->length_scale;
    if (i < 9) {
        box_after[i] = (i == 0 || i == 4 || i == 8) ? box[i] * scale : box[i];
    }
    if (i >= N) {
        return;
    }
    const int g = group_of[i];
    for (int d = 0; d < 3; d++) {
        double xd = x[3 * i + d];
        if (g >= 0) {
            const double center = box[d * 4] * 0.5;
            const double n = static_cast<double>(group_size[g]);
            const double c = static_cast<double>(static_cast<long long>(centroids[3 * g + d])) / FX_EXPONENT / n;
            xd += ((c - center) * scale) + center - c;
        }
        x_after[3 * i + d] = xd;
    }
}

// Metropolis test and step-size adaptation (timemachine/cpp/src/barostat.cu:229-279).
__global__ void k_baro_decide(
    int N,
    int num_groups,
    double kt,
    double pressure,
    const unsigned long long *__restrict__ u_before,
    const unsigned long long *__restrict__ u_after,
    const double *__restrict__ box,
    MDState *st) {
    __shared__ unsigned long long part0[32], part1[32];
    unsigned long long a = 0, b = 0;
    for (int i = threadIdx.x; i < N; i += blockDim.x) {
        a += u_before[i];
        b += u_after[i];
    }
    for (int o = 16; o > 0; o >>= 1) {
        a += __shfl_xor_sync(0xffffffffu, a, o);
        b += __shfl_xor_sync(0xffffffffu, b, o);
    }
    if ((threadIdx.x & 31) == 0) {
        part0[threadIdx.x >> 5] = a;
        part1[threadIdx.x >> 5] = b;
    }
    __syncthreads();
    if (threadIdx.x != 0) {
        return;
    }
    unsigned long long init_u = 0, final_u = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) {
        init_u += part0[w];
        final_u += part1[w];
    }
    st->last_u_before = init_u;
    st->last_u_after = final_u;
    const double volume = box[0] * box[4] * box[8];
    const double new_volume = volume + st->volume_delta;
    const double energy_delta = static_cast<double>(static_cast<long long>(final_u - init_u)) / FX_EXPONENT;
    const double w = energy_delta + pressure * st->volume_delta - num_groups * kt * log(new_volume / volume);
    const bool rejected = w > 0 && st->rand1 > exp(-w / kt);
    if (!rejected) {
        st->num_accepted++;
        st->total_accepted++;
    }
    st->num_attempted++;
    st->total_attempted++;
    if (st->num_attempted >= 10) {
        if (st->num_accepted < 0.25 * st->num_attempted) {
            st->volume_scale /= 1.1;
            st->num_attempted = 0;
            st->num_accepted = 0;
        } else if (st->num_accepted > 0.75 * st->num_attempted) {
            st->volume_scale = fmin(st->volume_scale * 1.1, volume * 0.3);
            st->num_attempted = 0;
            st->num_accepted = 0;
        }
    }
    st->accepted = rejected ? 0 : 1;
}

__global__ void k_baro_apply(
    int N,
    int num_groups,
    double *__restrict__ x,
    double *__restrict__ box,
    const double *__restrict__ x_after,
    const double *__restrict__ box_after,
    unsigned long long *__restrict__ centroids,
    unsigned long long *__restrict__ u_before,
    unsigned long long *__restrict__ u_after,
    const MDState *st) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const bool acc = st->accepted != 0;
    if (i < 9 && acc) {
        box[i] = box_after[i];
    }
    if (i < N) {
        if (acc) {
            x[3 * i + 0] = x_after[3 * i + 0];
            x[3 * i + 1] = x_after[3 * i + 1];
            x[3 * i + 2] = x_after[3 * i + 2];
        }
        u_before[i] = 0;
        u_after[i] = 0;
    }
    if (i < 3 * num_groups) {
        centroids[i] = 0;
    }
}

} // namespace

struct BoundPot {
    PotentialBase *pot;                    // caller-owned, drives the steps
    std::unique_ptr<PotentialBase> trial;  // own instance for barostat trial moves
    DevBuf<double> params;
    int P = 0;
};

class Context {
  public:
    Context(
        int N,
        const double *x0,
        const double *v0,
        const double *box0,
        double dt,
        double ca,
        const double *cbs,
        const double *ccs,
        unsigned long long seed,
        int n_pots,
        PotentialBase *const *pots,
        const double *const *params,
        const int *param_sizes)
        : N_(N), dt_(dt), ca_(ca) {
        if (N <= 0) {
            throw Error(TMNB_ERR_INVALID_ARGUMENT, "N must be positive");
        }
        key_ = make_uint2((unsigned)seed, (unsigned)(seed >> 32) ^ 0x5bd1e995u);
        x_.upload(x0, 3 * (size_t)N);
        v_.upload(v0, 3 * (size_t)N);
        box_.upload(box0, 9);
        cbs_.upload(cbs, N);
        ccs_.upload(ccs, N);
        du_dx_.alloc(3 * (size_t)N);
        du_dx_.zero();
        du_dl_buf_.alloc(N);
        du_dl_buf_.zero();
        st_.alloc(1);
        MDState s{};
        CK(cudaMemcpy(st_.p, &s, sizeof(s), cudaMemcpyHostToDevice));
        for (int k = 0; k < n_pots; k++) {
            if (pots[k]->num_atoms() >= 0 && pots[k]->num_atoms() != N) {
                throw Error(TMNB_ERR_INVALID_ARGUMENT, "potential atom count differs from the context's N");
            }
            if (pots[k]->num_params() != param_sizes[k]) {
                throw Error(TMNB_ERR_INVALID_ARGUMENT, "parameter size does not match the potential");
            }
            auto b = std::make_unique<BoundPot>();
            b->pot = pots[k];
            b->P = param_sizes[k];
            b->params.upload(params[k], param_sizes[k]);
            bps_.push_back(std::move(b));
        }
        CK(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
    }

    ~Context() {
        for (auto &kv : graphs_) {
            cudaGraphExecDestroy(kv.second);
        }
        for (cudaStream_t s : side_) {
            cudaStreamDestroy(s);
        }
        for (cudaEvent_t e : join_ev_) {
            cudaEventDestroy(e);
        }
        if (fork_ev_) {
            cudaEventDestroy(fork_ev_);
        }
        if (stream_) {
            cudaStreamDestroy(stream_);
        }
    }

    void set_barostat(double pressure, double temperature, const int *group_of, int interval, unsigned long long seed) {
        if (interval <= 0) {
            throw Error(TMNB_ERR_INVALID_ARGUMENT, "Barostat interval must be greater than 0");
        }
        std::vector<int> g(group_of, group_of + N_);
        int ng = 0;
        for (int a : g) {
            if (a < -1) {
                throw Error(TMNB_ERR_INVALID_ARGUMENT, "group index must be >= -1");
            }
            ng = std::max(ng, a + 1);
        }
        std::vector<int> sizes(std::max(1, ng), 0);
        for (int a : g) {
            if (a >= 0) {
                sizes[a]++;
            }
        }
        group_of_.upload(g.data(), N_);
        group_size_.upload(sizes.data(), sizes.size());
        num_groups_ = ng;
        centroids_.alloc(3 * (size_t)std::max(1, ng));
        centroids_.zero();
        x_after_.alloc(3 * (size_t)N_);
        box_after_.alloc(9);
        u_before_.alloc(N_);
        u_before_.zero();
        u_after_.alloc(N_);
        u_after_.zero();
        baro_pressure_ = pressure * AVOGADRO * 1e-25;
        baro_kt_ = BOLTZ * temperature;
        baro_interval_ = interval;
        baro_key_ = make_uint2((unsigned)seed ^ 0x2545f491u, (unsigned)(seed >> 32));
        for (auto &b : bps_) {
            b->trial = b->pot->clone();
        }
        has_baro_ = true;
        baro_step_ = 0;
        invalidate_graphs();
    }

    std::vector<unsigned long long> buffer_generations() const {
        std::vector<unsigned long long> g;
        for (const auto &b : bps_) {
            g.push_back(b->pot->buffer_generation());
            g.push_back(b->trial ? b->trial->buffer_generation() : 0);
        }
        return g;
    }

    void invalidate_graphs() {
        for (auto &kv : graphs_) {
            cudaGraphExecDestroy(kv.second);
        }
        graphs_.clear();
    }

    // One step: forces (+ du_dl) from every potential, then the integrator.
    // With `branch` (graph capture) each potential after the first is recorded
    // on its own forked stream, so the captured graph runs the potentials
    // concurrently; they all add into du_dx / du_dl with integer atomics, so
    // the sums do not depend on the order.
    //
    // With `fuse` (forces only), the first potential that offers it hands its
    // coordinate staging and force scatter to the integrator kernel
    // (k_langevin_fused): `prestaged` = the previous step's integrator kernel
    // staged this step's coordinates, `stage_next` = this step's integrator
    // kernel stages the next step's (same lambda, no barostat move between).
    void record_step(
        double lambda, unsigned long long *dl_out, bool branch = false, bool fuse = false, bool prestaged = false,
        bool stage_next = false) {
        const size_t n = bps_.size();
        const bool fork = branch && n > 1;
        MDFusion f{};
        int fk = -1;
        if (fuse && !dl_out) {
            for (size_t k = 0; k < n && fk < 0; k++) {
                if (bps_[k]->pot->md_fusion(f)) {
                    fk = (int)k;
                }
            }
        }
        if (fork) {
            ensure_branches(n - 1);
            CK(cudaEventRecord(fork_ev_, stream_));
        }
        for (size_t k = 0; k < n; k++) {
            cudaStream_t s = stream_;
            if (fork && k > 0) {
                s = side_[k - 1];
                CK(cudaStreamWaitEvent(s, fork_ev_, 0));
            }
            BoundPot &b = *bps_[k];
            if ((int)k == fk) {
                b.pot->execute_md_fused(N_, b.P, x_.p, b.params.p, box_.p, lambda, prestaged, s);
            } else {
                b.pot->execute_device(
                    N_, b.P, x_.p, b.params.p, box_.p, lambda, du_dx_.p, nullptr, dl_out ? du_dl_buf_.p : nullptr,
                    nullptr, s);
            }
            if (fork && k > 0) {
                CK(cudaEventRecord(join_ev_[k - 1], s));
                CK(cudaStreamWaitEvent(stream_, join_ev_[k - 1], 0));
            }
        }
        if (dl_out) {
            k_reduce_dl<<<1, 1024, 0, stream_>>>(N_, du_dl_buf_.p, dl_out, st_.p);
        }
        const int tpb = 128;
        if (fk >= 0) {
            launch_dependent(
                k_langevin_fused, dim3((2 * N_ + tpb - 1) / tpb), dim3(tpb), 0, stream_, N_, ca_,
                (const double *)cbs_.p, (const double *)ccs_.p, dt_, x_.p, v_.p, du_dx_.p, key_, st_.p, f,
                stage_next ? 1 : 0);
            CK(cudaPeekAtLastError());
            CK(cudaMemsetAsync(f.acc, 0, 3 * (size_t)f.S * sizeof(unsigned long long), stream_));
            return;
        }
        launch_dependent(
            k_langevin, dim3((2 * N_ + tpb - 1) / tpb), dim3(tpb), 0, stream_, N_, ca_, (const double *)cbs_.p,
            (const double *)ccs_.p, dt_, x_.p, v_.p, du_dx_.p, key_, st_.p);
        CK(cudaPeekAtLastError());
    }

    void record_barostat(double lambda) {
        for (auto &b : bps_) {
            b->pot->execute_device(N_, b->P, x_.p, b->params.p, box_.p, lambda, nullptr, nullptr, nullptr, u_before_.p, stream_);
        }
        const int tpb = 256;
        const int blocks = (N_ + tpb - 1) / tpb;
        k_baro_propose<<<blocks, tpb, 0, stream_>>>(N_, x_.p, box_.p, group_of_.p, centroids_.p, baro_key_, st_.p);
        k_baro_rescale<<<blocks, tpb, 0, stream_>>>(
            N_, x_.p, box_.p, group_of_.p, group_size_.p, centroids_.p, x_after_.p, box_after_.p, st_.p);
        for (auto &b : bps_) {
            b->trial->execute_device(
                N_, b->P, x_after_.p, b->params.p, box_after_.p, lambda, nullptr, nullptr, nullptr, u_after_.p, stream_);
        }
        k_baro_decide<<<1, 1024, 0, stream_>>>(
            N_, num_groups_, baro_kt_, baro_pressure_, u_before_.p, u_after_.p, box_.p, st_.p);
        const int ablocks = (std::max(N_, 3 * num_groups_) + tpb - 1) / tpb;
        k_baro_apply<<<ablocks, tpb, 0, stream_>>>(
            N_, num_groups_, x_.p, box_.p, x_after_.p, box_after_.p, centroids_.p, u_before_.p, u_after_.p, st_.p);
        CK(cudaPeekAtLastError());
    }

    // kind 0: one step (du_dl into dl_out if given); 1: the barostat move;
    // 2: `steps` steps.
    cudaGraphExec_t graph_for(int kind, double lambda, unsigned long long *dl_out, int steps = 1) {
        // a potential that reallocated buffers since the graphs were captured
        // (e.g. grown by a multi-window evaluation) invalidates all of them
        const std::vector<unsigned long long> gens = buffer_generations();
        if (gens != graph_generations_) {
            invalidate_graphs();
            graph_generations_ = gens;
        }
        const auto key = std::make_tuple(kind, lambda, (const void *)dl_out, steps);
        auto it = graphs_.find(key);
        if (it != graphs_.end()) {
            return it->second;
        }
        cudaGraph_t g;
        if (kind != 1 && bps_.size() > 1) {
            ensure_branches(bps_.size() - 1); // created outside the capture
        }
        CK(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeRelaxed));
        try {
            if (kind == 0) {
                record_step(lambda, dl_out, true);
            } else if (kind == 2) {
                // steps after the first take the coordinates the previous
                // step's integrator kernel staged
                for (int k = 0; k < steps; k++) {
                    record_step(lambda, nullptr, true, true, k > 0, k + 1 < steps);
                }
            } else {
                record_barostat(lambda);
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
        graphs_[key] = ge;
        return ge;
    }

    void multiple_steps(
        int n_steps,
        const double *lambdas,
        int dl_interval,
        double *dl_out_host,
        int x_interval,
        double *x_out_host,
        double *box_out_host,
        bool use_graphs) {
        if (n_steps < 0) {
            throw Error(TMNB_ERR_INVALID_ARGUMENT, "n_steps must be >= 0");
        }
        const int n_dl = dl_interval > 0 ? n_steps / dl_interval : 0;
        DevBuf<unsigned long long> dl_dev;
        if (n_dl > 0) {
            dl_dev.alloc(n_dl);
            int zero = 0;
            CK(cudaMemcpyAsync(&st_.p->dl_slot, &zero, sizeof(int), cudaMemcpyHostToDevice, stream_));
        }
        int frame = 0;
        const bool store_x = x_interval > 0 && x_out_host;
        for (int i = 1; i <= n_steps;) {
            const double lam = lambdas[i - 1];
            unsigned long long *dl_slot_base = (dl_interval > 0 && i % dl_interval == 0) ? dl_dev.p : nullptr;
            // Replayed steps run in chunks of up to MAX_GRAPH_STEPS steps per
            // graph: the same lambda, no du_dl store inside, frames and the
            // barostat move only after the chunk's last step.
            int L = 1;
            if (use_graphs && !dl_slot_base) {
                const int baro_left = has_baro_ ? baro_interval_ - (int)(baro_step_ % baro_interval_) : MAX_GRAPH_STEPS;
                while (L < MAX_GRAPH_STEPS && L < baro_left && i + L <= n_steps && lambdas[i + L - 1] == lam &&
                       !(dl_interval > 0 && (i + L) % dl_interval == 0) && !(store_x && (i + L - 1) % x_interval == 0)) {
                    L++;
                }
            }
            if (L > 1) {
                CK(cudaGraphLaunch(graph_for(2, lam, nullptr, L), stream_));
                barostat_after(lam, L, use_graphs);
            } else {
                advance(lam, dl_slot_base, use_graphs);
            }
            i += L;
            if (store_x && (i - 1) % x_interval == 0) {
                store_frame(frame, x_out_host, box_out_host);
                frame++;
            }
        }
        if (n_dl > 0 && dl_out_host) {
            std::vector<unsigned long long> h(n_dl);
            CK(cudaMemcpyAsync(h.data(), dl_dev.p, n_dl * sizeof(unsigned long long), cudaMemcpyDeviceToHost, stream_));
            CK(cudaStreamSynchronize(stream_));
            for (int k = 0; k < n_dl; k++) {
                dl_out_host[k] = static_cast<double>(static_cast<long long>(h[k])) / FX_EXPONENT;
            }
        }
        CK(cudaStreamSynchronize(stream_));
        for (auto &b : bps_) {
            b->pot->check_device_error(stream_);
        }
    }

    // Context::multiple_steps_U (timemachine/cpp/src/context.cu:139-234):
    // n_steps at `lambda`; every u_interval steps the total potential energy
    // at each of the K lambda windows, from one multi-window evaluation per
    // potential; x and box every x_interval steps.
    void multiple_steps_U(
        double lambda,
        int n_steps,
        int K,
        const double *windows,
        int u_interval,
        int x_interval,
        double *u_out_host,
        double *x_out_host,
        double *box_out_host,
        bool use_graphs) {
        if (n_steps < 0) {
            throw Error(TMNB_ERR_INVALID_ARGUMENT, "n_steps must be >= 0");
        }
        if (u_interval <= 0) {
            throw Error(TMNB_ERR_INVALID_ARGUMENT, "store_u_interval <= 0");
        }
        if (x_interval <= 0) {
            throw Error(TMNB_ERR_INVALID_ARGUMENT, "store_x_interval <= 0");
        }
        if (K < 0 || (K > 0 && !windows)) {
            throw Error(TMNB_ERR_INVALID_ARGUMENT, "invalid lambda windows");
        }
        const int n_u = n_steps / u_interval;
        DevBuf<unsigned long long> u_dev, u_win;
        if (n_u > 0 && K > 0) {
            u_dev.alloc((size_t)n_u * K);
            u_win.alloc((size_t)std::min(K, TMNB_MAX_WINDOWS) * N_);
            CK(cudaMemsetAsync(u_win.p, 0, u_win.n * sizeof(unsigned long long), stream_));
        }
        int frame = 0;
        for (int i = 1; i <= n_steps;) {
            // replayed steps in chunks (as in multiple_steps) that end at the
            // next frame, energy sample or barostat move
            int L = 1;
            if (use_graphs) {
                const int baro_left = has_baro_ ? baro_interval_ - (int)(baro_step_ % baro_interval_) : MAX_GRAPH_STEPS;
                while (L < MAX_GRAPH_STEPS && L < baro_left && i + L <= n_steps && (i + L - 1) % x_interval != 0 &&
                       (i + L - 1) % u_interval != 0) {
                    L++;
                }
            }
            if (L > 1) {
                CK(cudaGraphLaunch(graph_for(2, lambda, nullptr, L), stream_));
                barostat_after(lambda, L, use_graphs);
            } else {
                advance(lambda, nullptr, use_graphs);
            }
            i += L - 1; // the chunk's last step
            if (i % x_interval == 0 && x_out_host) {
                store_frame(frame, x_out_host, box_out_host);
                frame++;
            }
            if (i % u_interval == 0 && K > 0) {
                unsigned long long *row = u_dev.p + (size_t)(i / u_interval - 1) * K;
                for (int w = 0; w < K; w += TMNB_MAX_WINDOWS) {
                    const int kc = std::min(TMNB_MAX_WINDOWS, K - w);
                    for (auto &b : bps_) {
                        b->pot->execute_windows_device(
                            N_, b->P, x_.p, b->params.p, box_.p, kc, windows + w, nullptr, nullptr, nullptr, u_win.p,
                            stream_);
                    }
                    k_reduce_windows<<<kc, 1024, 0, stream_>>>(N_, u_win.p, row + w);
                    CK(cudaPeekAtLastError());
                }
            }
            i++;
        }
        if (n_u > 0 && K > 0 && u_out_host) {
            std::vector<unsigned long long> h((size_t)n_u * K);
            CK(cudaMemcpyAsync(h.data(), u_dev.p, h.size() * sizeof(unsigned long long), cudaMemcpyDeviceToHost, stream_));
            CK(cudaStreamSynchronize(stream_));
            for (size_t k = 0; k < h.size(); k++) {
                u_out_host[k] = static_cast<double>(static_cast<long long>(h[k])) / FX_EXPONENT;
            }
        }
        CK(cudaStreamSynchronize(stream_));
        for (auto &b : bps_) {
            b->pot->check_device_error(stream_);
        }
    }

    void get(int which, double *out) {
        CK(cudaStreamSynchronize(stream_));
        const DevBuf<double> &b = which == 0 ? x_ : (which == 1 ? v_ : box_);
        CK(cudaMemcpy(out, b.p, b.n * sizeof(double), cudaMemcpyDeviceToHost));
    }

    void set(int which, const double *in) {
        CK(cudaStreamSynchronize(stream_));
        DevBuf<double> &b = which == 0 ? x_ : (which == 1 ? v_ : box_);
        CK(cudaMemcpy(b.p, in, b.n * sizeof(double), cudaMemcpyHostToDevice));
    }

    // MonteCarloBarostat::set_pressure (timemachine/cpp/src/barostat.cu:386-389)
    void set_barostat_pressure(double pressure_bar) {
        if (!has_baro_) {
            throw Error(TMNB_ERR_INVALID_ARGUMENT, "no barostat");
        }
        baro_pressure_ = pressure_bar * AVOGADRO * 1e-25;
        invalidate_graphs(); // the captured moves hold the old pressure
    }

    // MonteCarloBarostat::set_interval: the move counter restarts
    // (timemachine/cpp/src/barostat.cu:391-397)
    void set_barostat_interval(int interval) {
        if (!has_baro_) {
            throw Error(TMNB_ERR_INVALID_ARGUMENT, "no barostat");
        }
        if (interval <= 0) {
            throw Error(TMNB_ERR_INVALID_ARGUMENT, "Barostat interval must be greater than 0");
        }
        baro_interval_ = interval;
        baro_step_ = 0;
    }

    // The last move: rand0, rand1, the proposal's volume scale, volume delta,
    // length scale, energies before and after (fixed point, as int64 bit
    // patterns), accepted (1/0), and the volume scale after the adaptation.
    void barostat_last_move(double *out, unsigned long long *u) {
        CK(cudaStreamSynchronize(stream_));
        MDState st;
        CK(cudaMemcpy(&st, st_.p, sizeof(st), cudaMemcpyDeviceToHost));
        out[0] = st.rand0;
        out[1] = st.rand1;
        out[2] = st.proposal_scale;
        out[3] = st.volume_delta;
        out[4] = st.length_scale;
        out[5] = st.accepted;
        out[6] = st.volume_scale;
        out[7] = baro_pressure_;
        u[0] = st.last_u_before;
        u[1] = st.last_u_after;
    }

    void barostat_stats(int *accepted, int *attempted, double *volume_scale) {
        CK(cudaStreamSynchronize(stream_));
        MDState s;
        CK(cudaMemcpy(&s, st_.p, sizeof(s), cudaMemcpyDeviceToHost));
        if (accepted) {
            *accepted = s.total_accepted;
        }
        if (attempted) {
            *attempted = s.total_attempted;
        }
        if (volume_scale) {
            *volume_scale = s.volume_scale;
        }
    }

    cudaStream_t stream() const { return stream_; }

  private:
    // One integrator step (with the barostat move on its interval), as
    // Context::_step (timemachine/cpp/src/context.cu:240-282).
    void advance(double lam, unsigned long long *dl_slot_base, bool use_graphs) {
        if (use_graphs) {
            CK(cudaGraphLaunch(graph_for(0, lam, dl_slot_base), stream_));
        } else {
            record_step(lam, dl_slot_base);
        }
        barostat_after(lam, 1, use_graphs);
    }

    // The barostat's step count after `steps` integrator steps, and its move
    // when the count reaches the interval.
    void barostat_after(double lam, int steps, bool use_graphs) {
        if (has_baro_) {
            baro_step_ += steps;
            if (baro_step_ % baro_interval_ == 0) {
                if (use_graphs) {
                    CK(cudaGraphLaunch(graph_for(1, lam, nullptr), stream_));
                } else {
                    record_barostat(lam);
                }
            }
        }
    }

    // Streams and events of the forked potential branches of a captured step.
    void ensure_branches(size_t n) {
        if (!fork_ev_) {
            CK(cudaEventCreateWithFlags(&fork_ev_, cudaEventDisableTiming));
        }
        while (side_.size() < n) {
            cudaStream_t s;
            CK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
            side_.push_back(s);
            cudaEvent_t e;
            CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
            join_ev_.push_back(e);
        }
    }

    void store_frame(int frame, double *x_out_host, double *box_out_host) {
        CK(cudaMemcpyAsync(
            x_out_host + (size_t)frame * N_ * 3, x_.p, 3 * (size_t)N_ * sizeof(double), cudaMemcpyDeviceToHost, stream_));
        if (box_out_host) {
            CK(cudaMemcpyAsync(box_out_host + (size_t)frame * 9, box_.p, 9 * sizeof(double), cudaMemcpyDeviceToHost, stream_));
        }
    }

    int N_;
    double dt_, ca_;
    uint2 key_;
    DevBuf<double> x_, v_, box_, cbs_, ccs_;
    DevBuf<unsigned long long> du_dx_, du_dl_buf_;
    DevBuf<MDState> st_;
    std::vector<std::unique_ptr<BoundPot>> bps_;
    cudaStream_t stream_ = nullptr;
    std::map<std::tuple<int, double, const void *, int>, cudaGraphExec_t> graphs_;
    std::vector<unsigned long long> graph_generations_; // buffer_generations() when graphs_ were captured
    static constexpr int MAX_GRAPH_STEPS = 25; // steps captured in one graph at most
    std::vector<cudaStream_t> side_;
    std::vector<cudaEvent_t> join_ev_;
    cudaEvent_t fork_ev_ = nullptr;

    bool has_baro_ = false;
    int baro_interval_ = 0;
    long long baro_step_ = 0;
    double baro_pressure_ = 0, baro_kt_ = 0;
    uint2 baro_key_;
    int num_groups_ = 0;
    DevBuf<int> group_of_, group_size_;
    DevBuf<unsigned long long> centroids_, u_before_, u_after_;
    DevBuf<double> x_after_, box_after_;
};

} // namespace tmb

struct tmnb_context {
    std::unique_ptr<tmb::Context> impl;
};

namespace {
tmnb_status check_ctx(const tmnb_context *c) {
    if (!c || !c->impl) {
        tmb::g_last_error = "null context handle";
        return TMNB_ERR_INVALID_ARGUMENT;
    }
    return TMNB_OK;
}
} // namespace

extern "C" {

tmnb_status tmnb_context_create(
    int N,
    const double *x0,
    const double *v0,
    const double *box0,
    double dt,
    double ca,
    const double *cbs,
    const double *ccs,
    unsigned long long seed,
    int n_potentials,
    tmnb_potential *const *potentials,
    const double *const *params,
    const int *param_sizes,
    tmnb_context **out) {
    if (!out || !x0 || !v0 || !box0 || !cbs || !ccs || n_potentials < 0 || (n_potentials > 0 && (!potentials || !params || !param_sizes))) {
        tmb::g_last_error = "null argument";
        return TMNB_ERR_INVALID_ARGUMENT;
    }
    return tmb::guarded([&] {
        std::vector<tmb::PotentialBase *> pots(n_potentials);
        for (int k = 0; k < n_potentials; k++) {
            if (!potentials[k] || !potentials[k]->impl) {
                throw tmb::Error(TMNB_ERR_INVALID_ARGUMENT, "null potential handle");
            }
            pots[k] = potentials[k]->impl.get();
        }
        auto c = std::make_unique<tmnb_context>();
        c->impl = std::make_unique<tmb::Context>(
            N, x0, v0, box0, dt, ca, cbs, ccs, seed, n_potentials, pots.data(), params, param_sizes);
        *out = c.release();
    });
}

tmnb_status tmnb_context_set_barostat(
    tmnb_context *ctx, double pressure_bar, double temperature_k, const int32_t *group_of, int interval, unsigned long long seed) {
    if (tmnb_status s = check_ctx(ctx)) {
        return s;
    }
    if (!group_of) {
        tmb::g_last_error = "null argument";
        return TMNB_ERR_INVALID_ARGUMENT;
    }
    return tmb::guarded([&] { ctx->impl->set_barostat(pressure_bar, temperature_k, group_of, interval, seed); });
}

tmnb_status tmnb_context_multiple_steps(
    tmnb_context *ctx,
    int n_steps,
    const double *lambda_schedule,
    int store_du_dl_interval,
    double *du_dl_out,
    int store_x_interval,
    double *x_out,
    double *box_out,
    int use_graphs) {
    if (tmnb_status s = check_ctx(ctx)) {
        return s;
    }
    if (n_steps > 0 && !lambda_schedule) {
        tmb::g_last_error = "null lambda schedule";
        return TMNB_ERR_INVALID_ARGUMENT;
    }
    return tmb::guarded([&] {
        ctx->impl->multiple_steps(
            n_steps, lambda_schedule, store_du_dl_interval, du_dl_out, store_x_interval, x_out, box_out, use_graphs != 0);
    });
}

tmnb_status tmnb_context_multiple_steps_U(
    tmnb_context *ctx,
    double lambda,
    int n_steps,
    int n_windows,
    const double *lambda_windows,
    int store_u_interval,
    int store_x_interval,
    double *u_out,
    double *x_out,
    double *box_out,
    int use_graphs) {
    if (tmnb_status s = check_ctx(ctx)) {
        return s;
    }
    return tmb::guarded([&] {
        ctx->impl->multiple_steps_U(
            lambda, n_steps, n_windows, lambda_windows, store_u_interval, store_x_interval, u_out, x_out, box_out,
            use_graphs != 0);
    });
}

tmnb_status tmnb_context_get_x(tmnb_context *ctx, double *out) {
    if (tmnb_status s = check_ctx(ctx)) {
        return s;
    }
    return tmb::guarded([&] { ctx->impl->get(0, out); });
}

tmnb_status tmnb_context_get_v(tmnb_context *ctx, double *out) {
    if (tmnb_status s = check_ctx(ctx)) {
        return s;
    }
    return tmb::guarded([&] { ctx->impl->get(1, out); });
}

tmnb_status tmnb_context_get_box(tmnb_context *ctx, double *out) {
    if (tmnb_status s = check_ctx(ctx)) {
        return s;
    }
    return tmb::guarded([&] { ctx->impl->get(2, out); });
}

tmnb_status tmnb_context_set_x(tmnb_context *ctx, const double *in) {
    if (tmnb_status s = check_ctx(ctx)) {
        return s;
    }
    return tmb::guarded([&] { ctx->impl->set(0, in); });
}

tmnb_status tmnb_context_set_v(tmnb_context *ctx, const double *in) {
    if (tmnb_status s = check_ctx(ctx)) {
        return s;
    }
    return tmb::guarded([&] { ctx->impl->set(1, in); });
}

tmnb_status tmnb_context_set_box(tmnb_context *ctx, const double *in) {
    if (tmnb_status s = check_ctx(ctx)) {
        return s;
    }
    return tmb::guarded([&] { ctx->impl->set(2, in); });
}

tmnb_status tmnb_context_barostat_stats(tmnb_context *ctx, int *accepted, int *attempted, double *volume_scale) {
    if (tmnb_status s = check_ctx(ctx)) {
        return s;
    }
    return tmb::guarded([&] { ctx->impl->barostat_stats(accepted, attempted, volume_scale); });
}

tmnb_status tmnb_context_barostat_set_pressure(tmnb_context *ctx, double pressure_bar) {
    if (tmnb_status s = check_ctx(ctx)) {
        return s;
    }
    return tmb::guarded([&] { ctx->impl->set_barostat_pressure(pressure_bar); });
}

tmnb_status tmnb_context_barostat_set_interval(tmnb_context *ctx, int interval) {
    if (tmnb_status s = check_ctx(ctx)) {
        return s;
    }
    return tmb::guarded([&] { ctx->impl->set_barostat_interval(interval); });
}

tmnb_status tmnb_context_barostat_last_move(tmnb_context *ctx, double *values, unsigned long long *energies) {
    if (tmnb_status s = check_ctx(ctx)) {
        return s;
    }
    if (!values || !energies) {
        tmb::g_last_error = "null argument";
        return TMNB_ERR_INVALID_ARGUMENT;
    }
    return tmb::guarded([&] { ctx->impl->barostat_last_move(values, energies); });
}

tmnb_status tmnb_context_destroy(tmnb_context *ctx) {
    if (!ctx) {
        return TMNB_OK;
    }
    return tmb::guarded([&] { delete ctx; });
}

} // extern "C"
