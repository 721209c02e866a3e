// Host side of the B200 nonbonded potential: instance state, launch
// sequence and the C ABI declared in include/tmnb.h.
//
// One class covers the three reference potentials of the path:
//   AllPairs  (timemachine/cpp/src/nonbonded_all_pairs.cu)
//   PairList  (timemachine/cpp/src/nonbonded_pair_list.cu, plain or negated)
//   Nonbonded (timemachine/lib/potentials.py:269-301: AllPairs + negated
//              PairList of the exclusions), evaluated as ONE pipeline whose
//              exclusion pairs run inside the pair kernel's launch.
//   Group     (timemachine/cpp/src/nonbonded_interaction_group.cu): pairs of
//              one row atom and one column atom (the complement); slots hold
//              the spatially sorted rows, then the sorted columns.
#include "engine.hpp"
#include "lambda_transform.hpp"
#include "nb_adjoint.cuh"
#include "pair_kernels.hpp"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <set>
#include <stdexcept>
#include <string>
#include <vector>

// Tiles per work item of lists built by single-window calls.
#ifndef TMNB_SINGLE_CHUNK
#define TMNB_SINGLE_CHUNK 2
#endif
// Tiles per work item of lists built by multi-window calls.
#ifndef TMNB_MULTI_CHUNK
#define TMNB_MULTI_CHUNK 4
#endif

namespace tmb {

enum class Kind { AllPairs, PairList, Nonbonded, Group };

// Pair-kernel tables: [0] 32-row, [1] 16-row, [2] 8-row tiles (FP32); FP64
// potentials use 16-row tiles only.
inline int row_table(int rows) { return rows == 32 ? 0 : (rows == 16 ? 1 : 2); }

class NonbondedPotential : public PotentialBase {
  public:
    NonbondedPotential(
        Kind kind,
        int N,
        const int *plane,
        const int *offset,
        double beta,
        double cutoff,
        const int *atom_idxs,
        int K,
        const int *pair_idxs,
        const double *scales,
        int M,
        bool negated,
        bool interpolated,
        bool fp64 = false)
        : kind_(kind), N_(N), beta_(beta), cutoff_(cutoff), interp_(interpolated), negated_(negated), fp64_(fp64),
          M_(M),
          h_plane_(plane, plane + N), h_offset_(offset, offset + N),
          h_atom_idxs_(atom_idxs ? std::vector<int>(atom_idxs, atom_idxs + K) : std::vector<int>()),
          h_pairs_(pair_idxs ? std::vector<int>(pair_idxs, pair_idxs + 2 * (size_t)M) : std::vector<int>()),
          h_scales_(scales ? std::vector<double>(scales, scales + 2 * (size_t)M) : std::vector<double>()) {
        if (N <= 0) {
            throw Error(TMNB_ERR_INVALID_ARGUMENT, "N must be positive");
        }
        if (!(cutoff > 0)) {
            throw Error(TMNB_ERR_INVALID_ARGUMENT, "cutoff must be positive");
        }
        has_nblist_ = kind != Kind::PairList;
        S_ = N;
        std::vector<int> set_atoms;
        if (kind == Kind::Group) {
            // timemachine/cpp/src/nonbonded_interaction_group.cu:62-64 and
            // timemachine/cpp/src/neighborlist.cu:215-228
            if (atom_idxs == nullptr || K <= 0) {
                throw Error(TMNB_ERR_INVALID_ARGUMENT, "row_atom_idxs must be nonempty");
            }
            std::set<int> uniq(atom_idxs, atom_idxs + K);
            if ((int)uniq.size() != K) {
                throw Error(TMNB_ERR_INVALID_ARGUMENT, "atom indices must be unique");
            }
            if (K >= N) {
                throw Error(TMNB_ERR_INVALID_ARGUMENT, "number of idxs must be less than N");
            }
            if (*uniq.rbegin() >= N || *uniq.begin() < 0) {
                throw Error(TMNB_ERR_INVALID_ARGUMENT, "indices values must be less than N");
            }
            set_atoms.assign(uniq.begin(), uniq.end());
            for (int a = 0; a < N; a++) {
                if (!uniq.count(a)) {
                    set_atoms.push_back(a);
                }
            }
            NR_ = K;
        }
        if (kind == Kind::AllPairs && atom_idxs != nullptr) {
            std::set<int> uniq(atom_idxs, atom_idxs + K);
            if ((int)uniq.size() != K) {
                throw Error(TMNB_ERR_INVALID_ARGUMENT, "atom indices must be unique");
            }
            if (K <= 0) {
                throw Error(TMNB_ERR_INVALID_ARGUMENT, "atom indices can't be empty");
            }
            for (int a : uniq) {
                if (a < 0 || a >= N) {
                    throw Error(TMNB_ERR_INVALID_ARGUMENT, "atom indices must be in [0, N)");
                }
            }
            set_atoms.assign(uniq.begin(), uniq.end()); // the reference keeps a sorted std::set
            S_ = K;
        }
        if (kind != Kind::AllPairs) {
            for (int i = 0; i < M; i++) {
                const int src = pair_idxs[2 * i], dst = pair_idxs[2 * i + 1];
                if (src == dst) {
                    throw Error(
                        TMNB_ERR_INVALID_ARGUMENT,
                        "illegal pair with src == dst: " + std::to_string(src) + ", " + std::to_string(dst));
                }
                if (src < 0 || src >= N || dst < 0 || dst >= N) {
                    throw Error(TMNB_ERR_INVALID_ARGUMENT, "pair index out of range [0, N)");
                }
            }
        } else {
            M_ = 0;
        }

        CK(cudaSetDevice(current_device()));
        plane_.upload(plane, N);
        offset_.upload(offset, N);
        if (!set_atoms.empty()) {
            set_atoms_.upload(set_atoms.data(), set_atoms.size());
        }
        if (M_ > 0) {
            pair_idxs_.upload(pair_idxs, 2 * (size_t)M_);
            scales_.upload(scales, 2 * (size_t)M_);
        }

        // slot order: initially the set order
        std::vector<unsigned> perm(S_);
        for (int s = 0; s < S_; s++) {
            perm[s] = set_atoms.empty() ? (unsigned)s : (unsigned)set_atoms[s];
        }
        perm_.upload(perm.data(), S_);
        if (has_nblist_ || kind == Kind::Nonbonded) {
            std::vector<int> slot(N, -1);
            for (int s = 0; s < S_; s++) {
                slot[perm[s]] = s;
            }
            slot_of_.upload(slot.data(), N);
        }
        if (kind == Kind::AllPairs && !set_atoms.empty()) {
            fin_atoms_.upload(set_atoms.data(), S_); // ascending
        }

        posw_.alloc(S_);
        prm_.alloc(S_);
        lamdep_.alloc(S_);
        if (interp_) {
            dprm_.alloc(S_);
        }
        if (fp64_) {
            posw64_.alloc(S_);
            prm64_.alloc(S_);
            if (interp_) {
                dprm64_.alloc(S_);
            }
        }
        split_pair_dp_ = interp_ && kind == Kind::Nonbonded;
        acc_.alloc(acc_block_elems());
        acc_.zero();

        if (has_nblist_) {
            RB_ = (S_ + TILE - 1) / TILE;
            cb_first_ = kind == Kind::Group ? NR_ / TILE : 0;
            nb_x_.alloc(3 * (size_t)N);
            nb_x_.zero();
            nb_box_.alloc(9);
            nb_box_.zero();
            // cells ~ S/8 atoms-per-cell target: 2^b per axis, b in [2, 6]
            int b = (int)std::ceil(std::log2(std::cbrt(std::max(1.0, S_ / 8.0))));
            grid_bits_ = std::min(6, std::max(2, b));
            keys_.alloc(S_);
            const size_t bins = ((size_t)1 << (3 * grid_bits_)) * (kind == Kind::Group ? 2 : 1);
            bin_count_.alloc(bins);
            bin_count_.zero();
            bin_cursor_.alloc(bins);
            bb_ctr_.alloc(RB_);
            bb_ext_.alloc(RB_);
            alloc_list(); // row groups of rows_ slots
        }
        state_.alloc(1);
        DevState st{};
        st.rebuild = has_nblist_ ? 1 : 0;
        CK(cudaMemcpy(state_.p, &st, sizeof(st), cudaMemcpyHostToDevice));
        if (fp64_) {
            if (interp_) {
                pair_kernels_f64_r16_interp(kernels_[1]);
            } else {
                pair_kernels_f64_r16(kernels_[1]);
            }
        } else if (interp_) {
            pair_kernels_f32_r32_interp(kernels_[0]);
            pair_kernels_f32_r16_interp(kernels_[1]);
            pair_kernels_f32_r8_interp(kernels_[2]);
        } else {
            pair_kernels_f32_r32(kernels_[0]);
            pair_kernels_f32_r16(kernels_[1]);
            pair_kernels_f32_r8(kernels_[2]);
        }
        CK(cudaDeviceSynchronize());
    }

    ~NonbondedPotential() {
        if (timing_) {
            for (auto &e : ev_) {
                cudaEventDestroy(e[0]);
                cudaEventDestroy(e[1]);
            }
        }
    }

    // CUDA events around every stage of a call (on the launching stream):
    // TMNB_STAGE_PREPARE (k_check_prepare), _REBUILD (the five rebuild-chain
    // kernels, which return at once when no rebuild is due), _PAIR (k_pair),
    // _FINALIZE (k_finalize and the accumulator memset).
    void enable_timing(bool on) {
        if (on && !timing_) {
            for (auto &e : ev_) {
                CK(cudaEventCreate(&e[0]));
                CK(cudaEventCreate(&e[1]));
            }
        } else if (!on && timing_) {
            for (auto &e : ev_) {
                CK(cudaEventDestroy(e[0]));
                CK(cudaEventDestroy(e[1]));
            }
        }
        timing_ = on;
        for (bool &t : timed_) {
            t = false;
        }
    }

    void stage_begin(int stage, cudaStream_t stream) {
        if (timing_) {
            CK(cudaEventRecord(ev_[stage][0], stream));
        }
    }
    void stage_end(int stage, cudaStream_t stream) {
        if (timing_) {
            CK(cudaEventRecord(ev_[stage][1], stream));
            timed_[stage] = true;
        }
    }

    float last_stage_ms(int stage) {
        if (stage < 0 || stage >= N_STAGES) {
            throw Error(TMNB_ERR_INVALID_ARGUMENT, "unknown stage");
        }
        if (!timing_ || !timed_[stage]) {
            throw Error(TMNB_ERR_INVALID_ARGUMENT, "no timed launch of this stage (enable timing first)");
        }
        CK(cudaEventSynchronize(ev_[stage][1]));
        float ms = 0.f;
        CK(cudaEventElapsedTime(&ms, ev_[stage][0], ev_[stage][1]));
        return ms;
    }
    float last_pair_ms() { return last_stage_ms(TMNB_STAGE_PAIR); }

    static int current_device() {
        int d = 0;
        CK(cudaGetDevice(&d));
        return d;
    }

    // Tile slots of row block rb, and of the whole list.
    // tiles row group g can hold: one per column block it reaches
    long long tiles_of_row_block(int g) const {
        return kind_ == Kind::Group ? RB_ - cb_first_ : RB_ - (long long)g * rows_ / TILE;
    }
    long long tile_slots() const {
        return tile_base_rows(n_row_blocks_, rows_, RB_, kind_ == Kind::Group ? 1 : 0, cb_first_);
    }

    // Tile storage for row groups of rows_ slots (and the work-item capacity).
    void alloc_list() {
        generation_++;
        n_row_blocks_ = ((kind_ == Kind::Group ? NR_ : S_) + rows_ - 1) / rows_;
        tile_cols_.alloc((size_t)tile_slots() * TILE);
        rb_ntiles_.alloc(n_row_blocks_);
        set_chunk(1); // item capacity for the finest list
        if (dep_tiles_.n > 0) {
            dep_tiles_.alloc((size_t)std::max(1LL, tile_slots()));
        }
    }

    // Slots per row group of the tile list (32, 16 or 8); the next call rebuilds.
    void set_row_group(int rows) {
        if (rows != 32 && rows != 16 && rows != 8) {
            throw Error(TMNB_ERR_INVALID_ARGUMENT, "rows per tile must be 32, 16 or 8");
        }
        if (fp64_ && rows != 16) {
            throw Error(TMNB_ERR_UNSUPPORTED, "FP64 potentials use tiles of 16 rows");
        }
        if (!has_nblist_ || rows == rows_) {
            rows_ = rows;
            return;
        }
        CK(cudaDeviceSynchronize());
        rows_ = rows;
        alloc_list();
        int one = 1;
        CK(cudaMemcpy(&state_.p->rebuild, &one, sizeof(int), cudaMemcpyHostToDevice));
    }
    int row_group() const { return rows_; }

    void set_chunk(int chunk) {
        chunk_ = std::max(1, chunk);
        long long cap = 0;
        for (int rb = 0; rb < n_row_blocks_; rb++) {
            cap += (tiles_of_row_block(rb) + chunk_ - 1) / chunk_;
        }
        items_.alloc((size_t)std::max(1LL, cap));
    }

    int num_params() const override { return (interp_ ? 2 : 1) * N_ * 3; }
    int num_atoms() const override { return N_; }

    std::unique_ptr<PotentialBase> clone() const override {
        auto c = std::make_unique<NonbondedPotential>(
            kind_,
            N_,
            h_plane_.data(),
            h_offset_.data(),
            beta_,
            cutoff_,
            h_atom_idxs_.empty() ? nullptr : h_atom_idxs_.data(),
            (int)h_atom_idxs_.size(),
            h_pairs_.empty() ? nullptr : h_pairs_.data(),
            h_scales_.empty() ? nullptr : h_scales_.data(),
            M_,
            negated_,
            interp_,
            fp64_);
        c->padding_ = padding_;
        c->hilbert_ = hilbert_;
        c->set_chunk(chunk_);
        c->set_row_group(rows_);
        c->xf_ = xf_;
        return c;
    }

    const char *name() const {
        switch (kind_) {
        case Kind::AllPairs:
            return "NonbondedAllPairs";
        case Kind::PairList:
            return "NonbondedPairList";
        case Kind::Group:
            return "NonbondedInteractionGroup";
        default:
            return "Nonbonded";
        }
    }

    void set_padding(double p) {
        if (!(p >= 0)) {
            throw Error(TMNB_ERR_INVALID_ARGUMENT, "padding must be non-negative");
        }
        padding_ = p;
        generation_++; // captured launches hold the padding
    }
    void disable_hilbert() {
        hilbert_ = false;
        generation_++;
    }

    // The four lambda schedules (timemachine/cpp/src/wrap_kernels.cpp:843-893);
    // nullptr keeps the identity "lambda". Parse errors throw.
    void set_transforms(const char *q, const char *sig, const char *eps, const char *w) {
        LambdaTransforms t;
        try {
            t.charge = LambdaExpr(q ? q : "lambda");
            t.sigma = LambdaExpr(sig ? sig : "lambda");
            t.epsilon = LambdaExpr(eps ? eps : "lambda");
            t.w = LambdaExpr(w ? w : "lambda");
        } catch (const std::invalid_argument &e) {
            throw Error(TMNB_ERR_INVALID_ARGUMENT, e.what());
        }
        // (non-interpolated potentials, like the reference's, read only the w schedule)
        xf_ = t;
        generation_++; // captured launches hold the schedules' values
    }
    const LambdaTransforms &transforms() const { return xf_; }

    // f and df/dlambda of the four schedules at one lambda
    LambdaWindow lambda_window(double lambda) const {
        LambdaWindow L;
        xf_.charge.eval(lambda, L.f_q, L.g_q);
        xf_.sigma.eval(lambda, L.f_s, L.g_s);
        xf_.epsilon.eval(lambda, L.f_e, L.g_e);
        xf_.w.eval(lambda, L.f_w, L.g_w);
        return L;
    }

    int row_end() const { return kind_ == Kind::Group ? NR_ : S_; }

    // Elements of one accumulator block (8 or 11 arrays of S slots).
    size_t acc_block_elems() const { return (size_t)S_ * (split_pair_dp_ ? 11 : 8); }

    // Staging and accumulator capacity for K windows: K staged copies of the
    // slots and, for K > 1, the shared block plus one block per window.
    void ensure_windows(int K) {
        if (posw_.n < (size_t)K * S_ || acc_.n < acc_block_elems() * (K > 1 ? 1 + K : 1) ||
            (K > 1 && has_nblist_ && dep_tiles_.n == 0)) {
            generation_++; // buffers below are reallocated
        }
        if (posw_.n < (size_t)K * S_) {
            posw_.alloc((size_t)K * S_);
            prm_.alloc((size_t)K * S_);
            if (interp_) {
                dprm_.alloc((size_t)K * S_);
            }
            if (fp64_) {
                posw64_.alloc((size_t)K * S_);
                prm64_.alloc((size_t)K * S_);
                if (interp_) {
                    dprm64_.alloc((size_t)K * S_);
                }
            }
        }
        const size_t need = acc_block_elems() * (K > 1 ? 1 + K : 1);
        if (acc_.n < need) {
            acc_.alloc(need);
            acc_.zero();
        }
        if (K > 1 && has_nblist_ && dep_tiles_.n == 0) {
            dep_tiles_.alloc((size_t)std::max(1LL, tile_slots()));
        }
    }

    void execute_device(
        int N,
        int P,
        const double *d_x,
        const double *d_p,
        const double *d_box,
        double lambda,
        unsigned long long *d_du_dx,
        unsigned long long *d_du_dp,
        unsigned long long *d_du_dl,
        unsigned long long *d_u,
        cudaStream_t stream) override {
        execute_windows_device(N, P, d_x, d_p, d_box, 1, &lambda, d_du_dx, d_du_dp, d_du_dl, d_u, stream);
    }

    // All windows in one launch sequence: one neighbour-list check/rebuild, one
    // pair kernel in which tiles of lambda-independent atoms are evaluated once
    // and the others once per window, one finalize writing K outputs.
    void execute_windows_device(
        int N,
        int P,
        const double *d_x,
        const double *d_p,
        const double *d_box,
        int K,
        const double *lambdas,
        unsigned long long *d_du_dx,
        unsigned long long *d_du_dp,
        unsigned long long *d_du_dl,
        unsigned long long *d_u,
        cudaStream_t stream) override {
        if (N != N_) {
            throw Error(
                TMNB_ERR_INVALID_ARGUMENT,
                std::string(name()) + "::execute_device(): expected N == N_, got N=" + std::to_string(N) +
                    ", N_=" + std::to_string(N_));
        }
        const int Mult = interp_ ? 2 : 1;
        if (P != Mult * N_ * 3) {
            throw Error(
                TMNB_ERR_INVALID_ARGUMENT,
                std::string(name()) + "::execute_device(): expected P == M*N_*3, got P=" + std::to_string(P) +
                    ", M*N_*3=" + std::to_string(Mult * N_ * 3));
        }
        if (!d_x || !d_p || !d_box) {
            throw Error(TMNB_ERR_INVALID_ARGUMENT, "x, params and box must be non-null");
        }
        if (K < 1 || K > MAX_WINDOWS || !lambdas) {
            throw Error(
                TMNB_ERR_INVALID_ARGUMENT,
                "number of lambda windows must be in [1, " + std::to_string(MAX_WINDOWS) + "], got " +
                    std::to_string(K));
        }
        ensure_windows(K);

        PrepareArgs pa;
        pa.N = N_;
        pa.S = S_;
        pa.x = d_x;
        pa.p = d_p;
        pa.box = d_box;
        pa.K = K;
        for (int k = 0; k < MAX_WINDOWS; k++) {
            pa.lam[k] = lambda_window(k < K ? lambdas[k] : 0.0);
        }
        pa.cutoff = cutoff_;
        pa.padding = padding_;
        pa.plane = plane_.p;
        pa.offset = offset_.p;
        pa.interpolated = interp_ ? 1 : 0;
        pa.slots.posw = posw_.p;
        pa.slots.prm = prm_.p;
        pa.slots.dprm = dprm_.p;
        pa.slots.lamdep = lamdep_.p;
        pa.slots.posw64 = posw64_.p;
        pa.slots.prm64 = prm64_.p;
        pa.slots.dprm64 = dprm64_.p;

        const int tpb = 256;
        const int sgrid = std::max(1, std::min((S_ + tpb - 1) / tpb, 8 * num_sms()));
        // k_check_prepare: one thread per (window, slot)
        const int pgrid = (int)std::max<size_t>(
            1, std::min<size_t>(((size_t)S_ * K + tpb - 1) / tpb, 8 * (size_t)num_sms()));
        if (!(fuse_ & FUSE_PRESTAGED)) {
            stage_begin(TMNB_STAGE_PREPARE, stream);
            launch_dependent(
                k_check_prepare, dim3(pgrid), dim3(tpb), 0, stream, pa, (const unsigned *)perm_.p,
                (const double *)(has_nblist_ ? nb_x_.p : nullptr), (const double *)nb_box_.p, state_.p);
            CK(cudaPeekAtLastError());
            stage_end(TMNB_STAGE_PREPARE, stream);
        }
        if (has_nblist_) {
            stage_begin(TMNB_STAGE_REBUILD, stream);
            record_rebuild_chain(d_x, d_box, pa, sgrid, tpb, stream, K);
            stage_end(TMNB_STAGE_REBUILD, stream);
        }

        const int kidx = (d_du_dp ? 1 : 0) | (d_du_dl ? 2 : 0) | (d_du_dx ? 4 : 0) | (d_u ? 8 : 0);
        if (kidx != 0 && K > 1 && has_nblist_) {
            DepArgs da;
            da.S = S_;
            da.rows = rows_;
            da.row_end = row_end();
            da.items = items_.p;
            da.tile_cols = tile_cols_.p;
            da.lamdep = lamdep_.p;
            da.dep_tiles = dep_tiles_.p;
            launch_dependent(k_dep_tiles, dim3(4 * num_sms()), dim3(128), 0, stream, da, state_.p);
            CK(cudaPeekAtLastError());
        }
        if (kidx != 0) {
            PairArgs a;
            a.S = S_;
            a.row_end = row_end();
            a.K = K;
            a.lamdep = lamdep_.p;
            a.acc_block = acc_block_elems();
            a.posw = posw_.p;
            a.prm = prm_.p;
            a.dprm = dprm_.p;
            a.posw64 = posw64_.p;
            a.prm64 = prm64_.p;
            a.dprm64 = dprm64_.p;
            a.box = d_box;
            a.beta = beta_;
            a.cutoff = cutoff_;
            a.tile_cols = tile_cols_.p;
            a.items = items_.p;
            a.M = M_;
            a.pair_idxs = pair_idxs_.p;
            a.scales = scales_.p;
            a.slot_of = slot_of_.p;
            a.negated = negated_ ? 1 : 0;
            a.acc = accum();
            a.dep_tiles = dep_tiles_.p;
            a.state = state_.p;
            const PairKernels &table = kernels_[row_table(rows_)];
            pair_kernel_t k = K > 1 ? table.multi[kidx] : table.single[kidx];
            const size_t smem = 0;
            stage_begin(TMNB_STAGE_PAIR, stream);
            launch_dependent(k, dim3(pair_grid(k, smem)), dim3(128), smem, stream, a);
            CK(cudaPeekAtLastError());
            stage_end(TMNB_STAGE_PAIR, stream);
            if (fuse_ & FUSE_KEEP_FORCES) {
                return; // the integrator kernel reads and clears the accumulators
            }

            FinalizeArgs fa;
            fa.N = N_;
            fa.S = S_;
            fa.set_atoms = fin_atoms_.p;
            fa.slot_of = slot_of_.p;
            fa.take = 0;
            fa.acc = accum();
            fa.acc_block = acc_block_elems();
            fa.K = K;
            for (int w = 0; w < MAX_WINDOWS; w++) {
                fa.f_dp[w][0] = pa.lam[w].f_q;
                fa.f_dp[w][1] = pa.lam[w].f_s;
                fa.f_dp[w][2] = pa.lam[w].f_e;
            }
            fa.stride_x = 3 * (size_t)N_;
            fa.stride_p = (size_t)P;
            fa.stride_n = (size_t)N_;
            fa.split_pair_dp = split_pair_dp_ ? 1 : 0;
            fa.interpolated = interp_ ? 1 : 0;
            fa.du_dx = d_du_dx;
            fa.du_dp = d_du_dp;
            fa.du_dl = d_du_dl;
            fa.u = d_u;
            fa.state = state_.p;
            const size_t fin_threads = (size_t)S_ * K;
            const int fgrid = (int)std::max<size_t>(1, std::min<size_t>((fin_threads + tpb - 1) / tpb, 16 * (size_t)num_sms()));
            stage_begin(TMNB_STAGE_FINALIZE, stream);
            launch_dependent(k_finalize, dim3(fgrid), dim3(tpb), 0, stream, fa);
            CK(cudaPeekAtLastError());
            // Zero the accumulator blocks k_finalize read (one coalesced memset;
            // zeroing each slot as it is read, from k_finalize's gathered
            // accesses, measured 2.5x slower). Forces only: the first three
            // arrays of the block are the only ones written.
            const size_t used = (kidx == 4 && K == 1) ? 3 * (size_t)S_ : acc_block_elems() * (K > 1 ? 1 + K : 1);
            CK(cudaMemsetAsync(acc_.p, 0, used * sizeof(unsigned long long), stream));
            stage_end(TMNB_STAGE_FINALIZE, stream);
        }
    }

    unsigned long long buffer_generation() const override { return generation_; }

    bool md_fusion(MDFusion &f) override {
        // every atom in the set (slot_of a bijection), FP32 staging, a neighbour list
        if (!has_nblist_ || fp64_ || kind_ == Kind::Group || S_ != N_ || set_atoms_.p != nullptr) {
            return false;
        }
        ensure_windows(1);
        f.slot_of = slot_of_.p;
        f.posw = posw_.p;
        f.nb_x = nb_x_.p;
        f.half_pad2 = 0.25 * padding_ * padding_;
        f.rebuild = &state_.p->rebuild;
        f.next_item = &state_.p->next_item;
        f.error = &state_.p->error;
        f.acc = acc_.p;
        f.S = S_;
        return true;
    }

    void execute_md_fused(
        int N, int P, const double *d_x, const double *d_p, const double *d_box, double lambda, bool prestaged,
        cudaStream_t stream) override {
        struct Reset {
            int &v;
            ~Reset() { v = 0; }
        } reset{fuse_};
        fuse_ = FUSE_KEEP_FORCES | (prestaged ? FUSE_PRESTAGED : 0);
        // forces only; the du_dx argument selects the variant and is not written
        execute_windows_device(N, P, d_x, d_p, d_box, 1, &lambda, acc_.p, nullptr, nullptr, nullptr, stream);
    }

    // Neighbour-list rebuild: spatial sort (keys, scan, scatter), block
    // bounds, tile build. Each kernel returns at once unless state->rebuild.
    void record_rebuild_chain(
        const double *d_x, const double *d_box, const PrepareArgs &pa, int sgrid, int tpb, cudaStream_t stream, int K) {
        SortArgs sa;
        sa.N = N_;
        sa.S = S_;
        sa.x = d_x;
        sa.box = d_box;
        sa.set_atoms = set_atoms_.p;
        sa.n_first = kind_ == Kind::Group ? NR_ : S_;
        sa.grid_bits = grid_bits_;
        sa.hilbert = hilbert_ ? 1 : 0;
        sa.keys = keys_.p;
        sa.bin_count = bin_count_.p;
        sa.bin_cursor = bin_cursor_.p;
        TileArgs ta;
        ta.S = S_;
        ta.RB = RB_;
        ta.rows = rows_;
        ta.group = kind_ == Kind::Group ? 1 : 0;
        ta.row_end = kind_ == Kind::Group ? NR_ : S_;
        ta.col_begin = kind_ == Kind::Group ? NR_ : 0;
        ta.n_row_blocks = n_row_blocks_;
        ta.cb_first = cb_first_;
        ta.radius = (float)(cutoff_ + padding_ + 1e-5);
        ta.box = d_box;
        ta.posw = posw_.p;
        ta.prm = prm_.p;
        ta.bb_ctr = bb_ctr_.p;
        ta.bb_ext = bb_ext_.p;
        ta.tile_cols = tile_cols_.p;
        ta.rb_ntiles = rb_ntiles_.p;
        ta.items = items_.p;
        // tiles per work item, measured on B200 at 22,840 atoms: two for a
        // single window with the packed forces sweep (MD step 125.7 -> 121.3
        // us against one; one had been -8 % against four with the one-row
        // sweep), four for several windows (fewer row flushes: -3 %)
        ta.chunk = K > 1 ? TMNB_MULTI_CHUNK : TMNB_SINGLE_CHUNK;
        const DevState *cst = state_.p;
        launch_dependent(k_bin_keys, dim3(sgrid), dim3(tpb), 0, stream, sa, cst);
        launch_dependent(k_bin_scan, dim3(1), dim3(1024), 0, stream, sa, state_.p);
        launch_dependent(
            k_bin_scatter, dim3(sgrid), dim3(tpb), 0, stream, sa, pa, perm_.p, slot_of_.p, nb_x_.p, nb_box_.p, cst);
        const int bb_grid = std::max(1, (RB_ * 32 + tpb - 1) / tpb);
        launch_dependent(
            k_block_bounds, dim3(bb_grid), dim3(tpb), 0, stream, S_, d_box, (const float4 *)posw_.p, bb_ctr_.p,
            bb_ext_.p, cst, pa, sa.n_first, perm_.p, slot_of_.p, rows_);
        launch_dependent(k_build_tiles, dim3(n_row_blocks_), dim3(TB_WARPS * 32), 0, stream, ta, state_.p);
        CK(cudaPeekAtLastError());
    }

    Accum accum() const {
        Accum c;
        unsigned long long *b = acc_.p;
        const size_t S = S_;
        c.x = b + 0 * S;
        c.y = b + 1 * S;
        c.z = b + 2 * S;
        c.q = b + 3 * S;
        c.sig = b + 4 * S;
        c.eps = b + 5 * S;
        c.u = b + 6 * S;
        c.dl = b + 7 * S;
        if (split_pair_dp_) {
            c.pq = b + 8 * S;
            c.psig = b + 9 * S;
            c.peps = b + 10 * S;
        } else {
            c.pq = c.q;
            c.psig = c.sig;
            c.peps = c.eps;
        }
        return c;
    }

    // persistent grid of the pair kernel k: occupancy x SMs (cached per kernel)
    int pair_grid(pair_kernel_t k, size_t smem) {
        for (const auto &e : grid_cache_) {
            if (e.first == k) {
                return e.second;
            }
        }
        int per_sm = 0;
        CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, 128, smem));
        const int grid = std::max(1, per_sm) * num_sms();
        grid_cache_.emplace_back(k, grid);
        return grid;
    }

    // Returns the sticky device error (and clears it).
    tmnb_status check_device_error(cudaStream_t stream) override {
        CK(cudaStreamSynchronize(stream));
        DevState st;
        CK(cudaMemcpy(&st, state_.p, sizeof(st), cudaMemcpyDeviceToHost));
        if (st.error != 0) {
            int zero = 0;
            CK(cudaMemcpy(&state_.p->error, &zero, sizeof(int), cudaMemcpyHostToDevice));
            if (st.error == DEV_ERR_NONORTHO_BOX) {
                throw Error(TMNB_ERR_NONORTHO_BOX, "Provided non-ortholinear box, unable to compute nonbonded energy");
            }
            throw Error(
                TMNB_ERR_BOX_TOO_SMALL,
                "Cutoff with padding is more than half of the box width, neighborlist is no longer reliable");
        }
        return TMNB_OK;
    }

    // Copies the neighbour list of the last rebuild: slot order (perm, [S]),
    // tiles per row block ([RB]) and the fixed-stride tile storage
    // ([tile_offset(RB) * 32] column slots; row block rb owns tiles
    // tile_offset(rb) .. + rb_ntiles[rb]).
    void copy_nblist(cudaStream_t stream, unsigned *perm, int *rb_ntiles, unsigned *tile_cols) {
        if (!has_nblist_) {
            throw Error(TMNB_ERR_INVALID_ARGUMENT, "potential has no neighbour list");
        }
        CK(cudaStreamSynchronize(stream));
        if (perm) {
            CK(cudaMemcpy(perm, perm_.p, S_ * sizeof(unsigned), cudaMemcpyDeviceToHost));
        }
        if (rb_ntiles) {
            CK(cudaMemcpy(rb_ntiles, rb_ntiles_.p, n_row_blocks_ * sizeof(int), cudaMemcpyDeviceToHost));
        }
        if (tile_cols) {
            CK(cudaMemcpy(tile_cols, tile_cols_.p, tile_cols_.n * sizeof(unsigned), cudaMemcpyDeviceToHost));
        }
    }

    // Vector-Jacobian product of (du_dx, du_dl) at (x, params, lambda) with
    // upstream (g_du_dx [N,3], g_du_dl): adds d/dparams into grad_p [N,3] and
    // d/d(lambda offset) into grad_w [N] (FP64, nb_adjoint.cuh). The
    // neighbour list is brought up to date for x first.
    void adjoint_device(
        int N,
        int P,
        const double *d_x,
        const double *d_p,
        const double *d_box,
        double lambda,
        const double *d_g_dx,
        double g_dl,
        double *d_grad_p,
        double *d_grad_w,
        cudaStream_t stream) {
        if (interp_ || kind_ == Kind::Group) {
            throw Error(TMNB_ERR_UNSUPPORTED, "the adjoint covers non-interpolated AllPairs, PairList and Nonbonded");
        }
        if (!xf_.w.is_identity()) {
            throw Error(TMNB_ERR_UNSUPPORTED, "the adjoint covers the identity lambda transform of w only");
        }
        if (!d_g_dx || !d_grad_p || !d_grad_w) {
            throw Error(TMNB_ERR_INVALID_ARGUMENT, "upstream gradient and outputs must be non-null");
        }
        // check, stage and (when needed) rebuild, no pair work
        execute_windows_device(N, P, d_x, d_p, d_box, 1, &lambda, nullptr, nullptr, nullptr, nullptr, stream);
        AdjointArgs a;
        a.N = N_;
        a.S = S_;
        a.x = d_x;
        a.p = d_p;
        a.box = d_box;
        a.plane = plane_.p;
        a.offset = offset_.p;
        a.lambda = lambda;
        a.beta = beta_;
        a.cutoff = cutoff_;
        a.perm = perm_.p;
        a.tile_cols = has_nblist_ ? tile_cols_.p : nullptr;
        a.items = items_.p;
        a.rows = rows_;
        a.M = M_;
        a.pair_idxs = pair_idxs_.p;
        a.scales = scales_.p;
        a.pair_sign = negated_ ? -1.0 : 1.0;
        a.g_dx = d_g_dx;
        a.g_dl = g_dl;
        a.grad_p = d_grad_p;
        a.grad_w = d_grad_w;
        a.state = state_.p;
        int per_sm = 0;
        CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_adjoint, ADJ_WARPS * 32, 0));
        k_adjoint<<<std::max(1, per_sm) * num_sms(), ADJ_WARPS * 32, 0, stream>>>(a);
        CK(cudaPeekAtLastError());
    }

    void nblist_rows(int *rows, int *column_blocks) const {
        if (rows) {
            *rows = rows_;
        }
        if (column_blocks) {
            *column_blocks = RB_;
        }
    }

    void nblist_shape(int *S, int *RB, long long *tile_capacity) const {
        if (S) {
            *S = S_;
        }
        if (RB) {
            *RB = n_row_blocks_;
        }
        if (tile_capacity) {
            *tile_capacity = has_nblist_ ? tile_slots() : 0;
        }
    }

    void stats(cudaStream_t stream, int *n_tiles, int *n_items, int *n_rebuilds) {
        CK(cudaStreamSynchronize(stream));
        DevState st;
        CK(cudaMemcpy(&st, state_.p, sizeof(st), cudaMemcpyDeviceToHost));
        if (n_tiles) {
            *n_tiles = (int)st.total_tiles;
        }
        if (n_items) {
            *n_items = st.n_items;
        }
        if (n_rebuilds) {
            *n_rebuilds = st.rebuilds;
        }
    }

    void du_dp_fixed_to_float(int N, int P, const unsigned long long *du_dp, double *out) const override {
        const int tuples = P / 3;
        for (int i = 0; i < tuples; i++) {
            out[3 * i + 0] = (double)(long long)du_dp[3 * i + 0] / (double)FX_EXPONENT;
            out[3 * i + 1] = (double)(long long)du_dp[3 * i + 1] / (double)FX_EXPONENT_SIG;
            out[3 * i + 2] = (double)(long long)du_dp[3 * i + 2] / (double)FX_EXPONENT_EPS;
        }
        (void)N;
    }

  private:
    Kind kind_;
    int N_;
    int S_ = 0;
    double beta_;
    double cutoff_;
    double padding_ = 0.1;
    bool interp_;
    bool negated_;
    bool fp64_;
    LambdaTransforms xf_;
    bool hilbert_ = true;
    bool has_nblist_ = false;
    bool split_pair_dp_ = false;
    int M_;
    int RB_ = 0;
    int NR_ = 0;           // interaction group: row atoms
    int n_row_blocks_ = 0; // blocks whose slots act as rows
    int cb_first_ = 0;     // interaction group: first column block
    int grid_bits_ = 4;
    int chunk_ = 1; // item capacity: one item per tile at most
    std::vector<std::pair<pair_kernel_t, int>> grid_cache_;
    // slots per row group of the tile list; 16 measured fastest on B200 at
    // 22,840 atoms (MD step -7 %, 12-window call -6 % against 32)
    int rows_ = 16;

    std::vector<int> h_plane_, h_offset_, h_atom_idxs_, h_pairs_;
    std::vector<double> h_scales_;

    DevBuf<int> plane_, offset_, set_atoms_, pair_idxs_, slot_of_, fin_atoms_;
    DevBuf<double> scales_;
    DevBuf<unsigned> perm_;
    DevBuf<float4> posw_, prm_, dprm_;
    DevBuf<double4> posw64_, prm64_, dprm64_;
    DevBuf<unsigned char> lamdep_;
    DevBuf<unsigned long long> acc_;
    // MD integrator fusion of the call in progress (execute_md_fused)
    static constexpr int FUSE_PRESTAGED = 1;   // coordinates staged by the integrator kernel
    static constexpr int FUSE_KEEP_FORCES = 2; // forces left in acc_ (no k_finalize, no clear)
    int fuse_ = 0;
    unsigned long long generation_ = 0; // buffer_generation()
    DevBuf<double> nb_x_, nb_box_;
    DevBuf<unsigned> keys_;
    DevBuf<int> bin_count_, bin_cursor_;
    DevBuf<float4> bb_ctr_, bb_ext_;
    DevBuf<unsigned> tile_cols_;
    DevBuf<int> rb_ntiles_;
    DevBuf<int4> items_;
    DevBuf<int2> dep_tiles_;
    DevBuf<DevState> state_;
    PairKernels kernels_[3] = {};

    // pair-kernel timing
    static constexpr int N_STAGES = 4;
    bool timing_ = false;
    bool timed_[N_STAGES] = {};
    cudaEvent_t ev_[N_STAGES][2] = {};

};

} // namespace tmb

namespace tmb {

// FP32 FMA throughput probe: 8 independent FMA chains per thread, enough
// resident warps to fill every SM; the denominator of the pair kernel's
// FP32 roofline.
__global__ void __launch_bounds__(256) k_fp32_peak(float *out, int iters, float a, float b) {
    float v0 = threadIdx.x * 1e-7f, v1 = v0 + 1e-7f, v2 = v0 + 2e-7f, v3 = v0 + 3e-7f;
    float v4 = v0 + 4e-7f, v5 = v0 + 5e-7f, v6 = v0 + 6e-7f, v7 = v0 + 7e-7f;
    for (int i = 0; i < iters; i++) {
#pragma unroll
        for (int k = 0; k < 16; k++) {
            v0 = fmaf(v0, a, b);
            v1 = fmaf(v1, a, b);
            v2 = fmaf(v2, a, b);
            v3 = fmaf(v3, a, b);
            v4 = fmaf(v4, a, b);
            v5 = fmaf(v5, a, b);
            v6 = fmaf(v6, a, b);
            v7 = fmaf(v7, a, b);
        }
    }
    const float s = v0 + v1 + v2 + v3 + v4 + v5 + v6 + v7;
    if (s == 1.2345f) {
        out[blockIdx.x * blockDim.x + threadIdx.x] = s; // practically never; keeps the chains live
    }
}

double fp32_peak_tflops() {
    const int sms = num_sms();
    const int blocks = sms * 8;
    const int threads = 256;
    const int iters = 4096;
    DevBuf<float> out;
    out.alloc((size_t)blocks * threads);
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    k_fp32_peak<<<blocks, threads>>>(out.p, 16, 0.999f, 1e-6f); // warm-up
    CK(cudaEventRecord(e0));
    k_fp32_peak<<<blocks, threads>>>(out.p, iters, 0.999f, 1e-6f);
    CK(cudaEventRecord(e1));
    CK(cudaEventSynchronize(e1));
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, e0, e1));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    const double flops = 2.0 * 8 * 16 * (double)iters * blocks * threads;
    return flops / (ms * 1e-3) / 1e12;
}

} // namespace tmb

namespace {

tmb::NonbondedPotential *as_nb(tmnb_potential *p) {
    auto *nb = dynamic_cast<tmb::NonbondedPotential *>(p->impl.get());
    if (!nb) {
        throw tmb::Error(TMNB_ERR_INVALID_ARGUMENT, "operation only defined for nonbonded potentials");
    }
    return nb;
}

tmnb_status check_handle(const tmnb_potential *p) {
    if (p == nullptr || !p->impl) {
        tmb::g_last_error = "null potential handle";
        return TMNB_ERR_INVALID_ARGUMENT;
    }
    return TMNB_OK;
}

tmnb_status check_precision(int precision) {
    if (precision != 32 && precision != 64) {
        tmb::g_last_error = "precision must be 32 (FP32 pair arithmetic) or 64 (FP64)";
        return TMNB_ERR_UNSUPPORTED;
    }
    return TMNB_OK;
}

} // namespace

extern "C" {

const char *tmnb_last_error(void) { return tmb::g_last_error.c_str(); }

const char *tmnb_version(void) { return "tmnb 0.1 sm_100a"; }

tmnb_status tmnb_all_pairs_create(
    int N,
    const int32_t *lambda_plane_idxs,
    const int32_t *lambda_offset_idxs,
    double beta,
    double cutoff,
    const int32_t *atom_idxs,
    int K,
    int interpolated,
    int precision,
    tmnb_potential **out) {
    if (tmnb_status s = check_precision(precision)) {
        return s;
    }
    if (!out || !lambda_plane_idxs || !lambda_offset_idxs) {
        tmb::g_last_error = "null argument";
        return TMNB_ERR_INVALID_ARGUMENT;
    }
    return tmb::guarded([&] {
        auto h = std::make_unique<tmnb_potential>();
        h->impl = std::make_unique<tmb::NonbondedPotential>(
            tmb::Kind::AllPairs,
            N,
            lambda_plane_idxs,
            lambda_offset_idxs,
            beta,
            cutoff,
            atom_idxs,
            K,
            nullptr,
            nullptr,
            0,
            false,
            interpolated != 0,
            precision == 64);
        *out = h.release();
    });
}

tmnb_status tmnb_interaction_group_create(
    int N,
    const int32_t *row_atom_idxs,
    int NR,
    const int32_t *lambda_plane_idxs,
    const int32_t *lambda_offset_idxs,
    double beta,
    double cutoff,
    int interpolated,
    int precision,
    tmnb_potential **out) {
    if (tmnb_status s = check_precision(precision)) {
        return s;
    }
    if (!out || !lambda_plane_idxs || !lambda_offset_idxs || NR < 0 || (NR > 0 && !row_atom_idxs)) {
        tmb::g_last_error = "null argument";
        return TMNB_ERR_INVALID_ARGUMENT;
    }
    return tmb::guarded([&] {
        auto h = std::make_unique<tmnb_potential>();
        h->impl = std::make_unique<tmb::NonbondedPotential>(
            tmb::Kind::Group,
            N,
            lambda_plane_idxs,
            lambda_offset_idxs,
            beta,
            cutoff,
            row_atom_idxs,
            NR,
            nullptr,
            nullptr,
            0,
            false,
            interpolated != 0,
            precision == 64);
        *out = h.release();
    });
}

tmnb_status tmnb_pair_list_create(
    int N,
    const int32_t *pair_idxs,
    const double *scales,
    int M,
    const int32_t *lambda_plane_idxs,
    const int32_t *lambda_offset_idxs,
    double beta,
    double cutoff,
    int negated,
    int interpolated,
    int precision,
    tmnb_potential **out) {
    if (tmnb_status s = check_precision(precision)) {
        return s;
    }
    if (!out || !lambda_plane_idxs || !lambda_offset_idxs || (M > 0 && (!pair_idxs || !scales)) || M < 0) {
        tmb::g_last_error = "null argument";
        return TMNB_ERR_INVALID_ARGUMENT;
    }
    return tmb::guarded([&] {
        auto h = std::make_unique<tmnb_potential>();
        h->impl = std::make_unique<tmb::NonbondedPotential>(
            tmb::Kind::PairList,
            N,
            lambda_plane_idxs,
            lambda_offset_idxs,
            beta,
            cutoff,
            nullptr,
            0,
            pair_idxs,
            scales,
            M,
            negated != 0,
            interpolated != 0,
            precision == 64);
        *out = h.release();
    });
}

tmnb_status tmnb_nonbonded_create(
    int N,
    const int32_t *exclusion_idxs,
    const double *scales,
    int M,
    const int32_t *lambda_plane_idxs,
    const int32_t *lambda_offset_idxs,
    double beta,
    double cutoff,
    int interpolated,
    int precision,
    tmnb_potential **out) {
    if (tmnb_status s = check_precision(precision)) {
        return s;
    }
    if (!out || !lambda_plane_idxs || !lambda_offset_idxs || (M > 0 && (!exclusion_idxs || !scales)) || M < 0) {
        tmb::g_last_error = "null argument";
        return TMNB_ERR_INVALID_ARGUMENT;
    }
    return tmb::guarded([&] {
        auto h = std::make_unique<tmnb_potential>();
        h->impl = std::make_unique<tmb::NonbondedPotential>(
            tmb::Kind::Nonbonded,
            N,
            lambda_plane_idxs,
            lambda_offset_idxs,
            beta,
            cutoff,
            nullptr,
            0,
            exclusion_idxs,
            scales,
            M,
            true,
            interpolated != 0,
            precision == 64);
        *out = h.release();
    });
}

tmnb_status tmnb_potential_destroy(tmnb_potential *pot) {
    if (pot == nullptr) {
        return TMNB_OK;
    }
    return tmb::guarded([&] { delete pot; });
}

tmnb_status tmnb_potential_execute_device(
    tmnb_potential *pot,
    int N,
    int P,
    const double *d_x,
    const double *d_p,
    const double *d_box,
    double lambda,
    unsigned long long *d_du_dx,
    unsigned long long *d_du_dp,
    unsigned long long *d_du_dl,
    unsigned long long *d_u,
    void *stream) {
    if (tmnb_status s = check_handle(pot)) {
        return s;
    }
    return tmb::guarded([&] {
        pot->impl->execute_device(
            N, P, d_x, d_p, d_box, lambda, d_du_dx, d_du_dp, d_du_dl, d_u, static_cast<cudaStream_t>(stream));
    });
}

tmnb_status tmnb_potential_execute_host(
    tmnb_potential *pot,
    int N,
    int P,
    const double *h_x,
    const double *h_p,
    const double *h_box,
    double lambda,
    unsigned long long *h_du_dx,
    unsigned long long *h_du_dp,
    unsigned long long *h_du_dl,
    unsigned long long *h_u) {
    if (tmnb_status s = check_handle(pot)) {
        return s;
    }
    if (!h_x || !h_box || (P > 0 && !h_p)) {
        tmb::g_last_error = "null argument";
        return TMNB_ERR_INVALID_ARGUMENT;
    }
    return tmb::guarded([&] { pot->impl->execute_host(N, P, h_x, h_p, h_box, lambda, h_du_dx, h_du_dp, h_du_dl, h_u); });
}

tmnb_status tmnb_potential_execute_windows_device(
    tmnb_potential *pot,
    int N,
    int P,
    const double *d_x,
    const double *d_p,
    const double *d_box,
    int K,
    const double *lambdas,
    unsigned long long *d_du_dx,
    unsigned long long *d_du_dp,
    unsigned long long *d_du_dl,
    unsigned long long *d_u,
    void *stream) {
    if (tmnb_status s = check_handle(pot)) {
        return s;
    }
    if (K < 1 || !lambdas) {
        tmb::g_last_error = "K must be positive and lambdas non-null";
        return TMNB_ERR_INVALID_ARGUMENT;
    }
    return tmb::guarded([&] {
        pot->impl->execute_windows_device(
            N, P, d_x, d_p, d_box, K, lambdas, d_du_dx, d_du_dp, d_du_dl, d_u, static_cast<cudaStream_t>(stream));
    });
}

tmnb_status tmnb_potential_execute_windows_host(
    tmnb_potential *pot,
    int N,
    int P,
    const double *h_x,
    const double *h_p,
    const double *h_box,
    int K,
    const double *lambdas,
    unsigned long long *h_du_dx,
    unsigned long long *h_du_dp,
    unsigned long long *h_du_dl,
    unsigned long long *h_u) {
    if (tmnb_status s = check_handle(pot)) {
        return s;
    }
    if (!h_x || !h_box || (P > 0 && !h_p) || K < 1 || !lambdas) {
        tmb::g_last_error = "null argument or K < 1";
        return TMNB_ERR_INVALID_ARGUMENT;
    }
    return tmb::guarded([&] {
        pot->impl->execute_windows_host(N, P, h_x, h_p, h_box, K, lambdas, h_du_dx, h_du_dp, h_du_dl, h_u);
    });
}

tmnb_status tmnb_potential_execute_batch_host(
    tmnb_potential *pot,
    int coord_batches,
    int N,
    int param_batches,
    int P,
    int lambda_batches,
    const double *h_x,
    const double *h_p,
    const double *h_boxes,
    const double *h_lambdas,
    unsigned long long *h_du_dx,
    unsigned long long *h_du_dp,
    unsigned long long *h_du_dl,
    unsigned long long *h_u) {
    if (tmnb_status s = check_handle(pot)) {
        return s;
    }
    if (coord_batches <= 0 || param_batches <= 0 || lambda_batches <= 0 || !h_x || !h_p || !h_boxes || !h_lambdas) {
        tmb::g_last_error = "invalid batch arguments";
        return TMNB_ERR_INVALID_ARGUMENT;
    }
    return tmb::guarded([&] {
        size_t e = 0;
        for (int c = 0; c < coord_batches; c++) {
            for (int p = 0; p < param_batches; p++) {
                for (int l = 0; l < lambda_batches; l += tmb::MAX_WINDOWS) {
                    const int K = std::min(tmb::MAX_WINDOWS, lambda_batches - l);
                    pot->impl->execute_windows_host(
                        N,
                        P,
                        h_x + (size_t)c * N * 3,
                        h_p + (size_t)p * P,
                        h_boxes + (size_t)c * 9,
                        K,
                        h_lambdas + l,
                        h_du_dx ? h_du_dx + e * N * 3 : nullptr,
                        h_du_dp ? h_du_dp + e * P : nullptr,
                        h_du_dl ? h_du_dl + e * N : nullptr,
                        h_u ? h_u + e * N : nullptr);
                    e += K;
                }
            }
        }
    });
}

tmnb_status tmnb_potential_du_dp_fixed_to_float(
    tmnb_potential *pot, int N, int P, const unsigned long long *du_dp, double *du_dp_float) {
    if (tmnb_status s = check_handle(pot)) {
        return s;
    }
    if (!du_dp || !du_dp_float) {
        tmb::g_last_error = "null argument";
        return TMNB_ERR_INVALID_ARGUMENT;
    }
    return tmb::guarded([&] { pot->impl->du_dp_fixed_to_float(N, P, du_dp, du_dp_float); });
}

tmnb_status tmnb_potential_set_nblist_padding(tmnb_potential *pot, double padding) {
    if (tmnb_status s = check_handle(pot)) {
        return s;
    }
    return tmb::guarded([&] { as_nb(pot)->set_padding(padding); });
}

tmnb_status tmnb_potential_disable_hilbert_sort(tmnb_potential *pot) {
    if (tmnb_status s = check_handle(pot)) {
        return s;
    }
    return tmb::guarded([&] { as_nb(pot)->disable_hilbert(); });
}

tmnb_status tmnb_lambda_transform_eval(const char *expression, double lambda, double *f, double *df) {
    if (!expression || !f || !df) {
        tmb::g_last_error = "null argument";
        return TMNB_ERR_INVALID_ARGUMENT;
    }
    return tmb::guarded([&] {
        try {
            tmb::LambdaExpr(expression).eval(lambda, *f, *df);
        } catch (const std::invalid_argument &e) {
            throw tmb::Error(TMNB_ERR_INVALID_ARGUMENT, e.what());
        }
    });
}

tmnb_status tmnb_potential_set_lambda_transforms(
    tmnb_potential *pot, const char *charge, const char *sigma, const char *epsilon, const char *w) {
    if (tmnb_status s = check_handle(pot)) {
        return s;
    }
    return tmb::guarded([&] { as_nb(pot)->set_transforms(charge, sigma, epsilon, w); });
}

tmnb_status tmnb_potential_set_tile_rows(tmnb_potential *pot, int rows) {
    if (tmnb_status s = check_handle(pot)) {
        return s;
    }
    return tmb::guarded([&] { as_nb(pot)->set_row_group(rows); });
}

tmnb_status tmnb_potential_nblist_rows(tmnb_potential *pot, int *rows, int *column_blocks) {
    if (tmnb_status s = check_handle(pot)) {
        return s;
    }
    return tmb::guarded([&] { as_nb(pot)->nblist_rows(rows, column_blocks); });
}

tmnb_status tmnb_potential_check_device_error(tmnb_potential *pot, void *stream) {
    if (tmnb_status s = check_handle(pot)) {
        return s;
    }
    return tmb::guarded([&] { pot->impl->check_device_error(static_cast<cudaStream_t>(stream)); });
}

tmnb_status tmnb_potential_nblist_stats(
    tmnb_potential *pot, void *stream, int *n_tiles, int *n_items, int *n_rebuilds) {
    if (tmnb_status s = check_handle(pot)) {
        return s;
    }
    return tmb::guarded([&] { as_nb(pot)->stats(static_cast<cudaStream_t>(stream), n_tiles, n_items, n_rebuilds); });
}

tmnb_status tmnb_potential_nblist_shape(tmnb_potential *pot, int *S, int *RB, long long *tile_capacity) {
    if (tmnb_status s = check_handle(pot)) {
        return s;
    }
    return tmb::guarded([&] { as_nb(pot)->nblist_shape(S, RB, tile_capacity); });
}

tmnb_status tmnb_potential_copy_nblist(
    tmnb_potential *pot, void *stream, unsigned *perm, int *row_block_ntiles, unsigned *tile_cols) {
    if (tmnb_status s = check_handle(pot)) {
        return s;
    }
    return tmb::guarded(
        [&] { as_nb(pot)->copy_nblist(static_cast<cudaStream_t>(stream), perm, row_block_ntiles, tile_cols); });
}

tmnb_status tmnb_potential_adjoint_device(
    tmnb_potential *pot,
    int N,
    int P,
    const double *d_x,
    const double *d_p,
    const double *d_box,
    double lambda,
    const double *d_g_du_dx,
    double g_du_dl,
    double *d_grad_p,
    double *d_grad_w,
    void *stream) {
    if (tmnb_status s = check_handle(pot)) {
        return s;
    }
    return tmb::guarded([&] {
        as_nb(pot)->adjoint_device(
            N, P, d_x, d_p, d_box, lambda, d_g_du_dx, g_du_dl, d_grad_p, d_grad_w, static_cast<cudaStream_t>(stream));
    });
}

tmnb_status tmnb_potential_enable_timing(tmnb_potential *pot, int on) {
    if (tmnb_status s = check_handle(pot)) {
        return s;
    }
    return tmb::guarded([&] { as_nb(pot)->enable_timing(on != 0); });
}

tmnb_status tmnb_potential_last_pair_kernel_ms(tmnb_potential *pot, float *ms) {
    if (tmnb_status s = check_handle(pot)) {
        return s;
    }
    if (!ms) {
        tmb::g_last_error = "null argument";
        return TMNB_ERR_INVALID_ARGUMENT;
    }
    return tmb::guarded([&] { *ms = as_nb(pot)->last_pair_ms(); });
}

tmnb_status tmnb_potential_last_stage_ms(tmnb_potential *pot, int stage, float *ms) {
    if (tmnb_status s = check_handle(pot)) {
        return s;
    }
    if (!ms) {
        tmb::g_last_error = "null argument";
        return TMNB_ERR_INVALID_ARGUMENT;
    }
    return tmb::guarded([&] { *ms = as_nb(pot)->last_stage_ms(stage); });
}

tmnb_status tmnb_probe_fp32_peak(double *tflops) {
    if (!tflops) {
        tmb::g_last_error = "null argument";
        return TMNB_ERR_INVALID_ARGUMENT;
    }
    return tmb::guarded([&] { *tflops = tmb::fp32_peak_tflops(); });
}

int tmnb_potential_num_params(const tmnb_potential *pot) {
    return (pot && pot->impl) ? pot->impl->num_params() : -1;
}

int tmnb_potential_num_atoms(const tmnb_potential *pot) {
    return (pot && pot->impl) ? pot->impl->num_atoms() : -1;
}

} // extern "C"
