// Test/baseline harness around the REFERENCE timemachine CUDA implementation.
//
// This file is test infrastructure: it is compiled together with the
// reference's own sources (timemachine/cpp/src/*.cu, built from the reference
// tree by oracle/refgpu/Makefile into oracle/_ref/libtmref.so) and gives them
// a plain C entry so the parity tests can compare the B200 kernels with the
// reference kernels bit for bit, and the benchmark's reference arm can time
// the reference's own GPU path. Nothing in the product links or loads it.
//
// The objects built here are exactly the reference's:
//   Nonbonded.unbound_impl  -> FanoutSummedPotential([NonbondedAllPairs, NonbondedPairList<Negated>])
//                              (timemachine/lib/potentials.py:284-301)
//   NonbondedInteractionGroup(_Interpolated)<float>
//                              (timemachine/cpp/src/nonbonded_interaction_group.cu)
//   Context + LangevinIntegrator + MonteCarloBarostat for MD throughput
//                              (timemachine/cpp/src/context.cu, integrator.cu, barostat.cu)
#include "bound_potential.hpp"
#include "barostat.hpp"
#include "context.hpp"
#include "fanout_summed_potential.hpp"
#include "harmonic_angle.hpp"
#include "harmonic_bond.hpp"
#include "integrator.hpp"
#include "nonbonded_all_pairs.hpp"
#include "nonbonded_interaction_group.hpp"
#include "nonbonded_pair_list.hpp"

#include <fstream>
#include <memory>
#include <regex>
#include <set>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

namespace {

thread_local std::string g_err;

std::string jit_source(
    const std::string &kernel_dir,
    const char *tq = nullptr,
    const char *ts = nullptr,
    const char *te = nullptr,
    const char *tw = nullptr) {
    // the reference's constructor binding reads and patches this file
    // (timemachine/cpp/src/wrap_kernels.cpp:869-879) with the four transforms
    std::ifstream t(kernel_dir + "/k_lambda_transformer_jit.cuh");
    if (!t) {
        throw std::runtime_error("cannot read " + kernel_dir + "/k_lambda_transformer_jit.cuh");
    }
    std::string src((std::istreambuf_iterator<char>(t)), std::istreambuf_iterator<char>());
    src = std::regex_replace(src, std::regex("KERNEL_DIR"), kernel_dir);
    src = std::regex_replace(src, std::regex("CUSTOM_EXPRESSION_CHARGE"), tq ? tq : "lambda");
    src = std::regex_replace(src, std::regex("CUSTOM_EXPRESSION_SIGMA"), ts ? ts : "lambda");
    src = std::regex_replace(src, std::regex("CUSTOM_EXPRESSION_EPSILON"), te ? te : "lambda");
    src = std::regex_replace(src, std::regex("CUSTOM_EXPRESSION_W"), tw ? tw : "lambda");
    return src;
}

// Applies f to the AllPairs part, whatever its precision and parameter mode.
template <typename F> void with_all_pairs(timemachine::Potential *p, F &&f) {
    if (auto *a = dynamic_cast<timemachine::NonbondedAllPairs<float, false> *>(p)) {
        f(a);
    } else if (auto *b = dynamic_cast<timemachine::NonbondedAllPairs<float, true> *>(p)) {
        f(b);
    } else if (auto *c = dynamic_cast<timemachine::NonbondedAllPairs<double, false> *>(p)) {
        f(c);
    } else if (auto *d = dynamic_cast<timemachine::NonbondedAllPairs<double, true> *>(p)) {
        f(d);
    }
}

struct RefNonbonded {
    std::shared_ptr<timemachine::Potential> all_pairs;
    std::shared_ptr<timemachine::Potential> exclusions;
    std::shared_ptr<timemachine::FanoutSummedPotential> fanout;
    bool interpolated;
};

template <typename F> int guarded(F &&f) {
    try {
        f();
        return 0;
    } catch (const std::exception &e) {
        g_err = e.what();
        return 1;
    }
}

struct RefMD {
    std::unique_ptr<timemachine::LangevinIntegrator> intg;
    std::unique_ptr<timemachine::BoundPotential> bp;
    std::vector<std::unique_ptr<timemachine::BoundPotential>> bonded;
    std::unique_ptr<timemachine::MonteCarloBarostat> baro;
    std::unique_ptr<timemachine::Context> ctx;
};

} // namespace

extern "C" {

const char *tmref_last_error(void) { return g_err.c_str(); }

void *tmref_nonbonded_create(
    const char *kernel_dir,
    int N,
    const int *exclusion_idxs,
    const double *scales,
    int M,
    const int *plane,
    const int *offset,
    double beta,
    double cutoff,
    int interpolated,
    int precision,     // 32 (_f32 kernels) or 64 (_f64 kernels)
    const char *tq,    // lambda transforms (NULL: "lambda")
    const char *ts,
    const char *te,
    const char *tw) {
    RefNonbonded *h = nullptr;
    int rc = guarded([&] {
        const std::string src = jit_source(kernel_dir, tq, ts, te, tw);
        std::vector<int> pl(plane, plane + N), of(offset, offset + N);
        std::vector<int> ex(exclusion_idxs, exclusion_idxs + 2 * (size_t)M);
        std::vector<double> sc(scales, scales + 2 * (size_t)M);
        auto r = std::make_unique<RefNonbonded>();
        r->interpolated = interpolated != 0;
        auto build = [&](auto real_tag) {
            using Real = decltype(real_tag);
            if (interpolated) {
                r->all_pairs = std::make_shared<timemachine::NonbondedAllPairs<Real, true>>(
                    pl, of, beta, cutoff, std::nullopt, src);
                r->exclusions = std::make_shared<timemachine::NonbondedPairList<Real, true, true>>(
                    ex, sc, pl, of, beta, cutoff, src);
            } else {
                r->all_pairs = std::make_shared<timemachine::NonbondedAllPairs<Real, false>>(
                    pl, of, beta, cutoff, std::nullopt, src);
                r->exclusions = std::make_shared<timemachine::NonbondedPairList<Real, true, false>>(
                    ex, sc, pl, of, beta, cutoff, src);
            }
        };
        if (precision == 64) {
            build(double{});
        } else {
            build(float{});
        }
        r->fanout = std::make_shared<timemachine::FanoutSummedPotential>(
            std::vector<std::shared_ptr<timemachine::Potential>>{r->all_pairs, r->exclusions});
        h = r.release();
    });
    return rc == 0 ? h : nullptr;
}

void tmref_nonbonded_destroy(void *h) { delete static_cast<RefNonbonded *>(h); }

int tmref_set_nblist_padding(void *h, double padding) {
    auto *r = static_cast<RefNonbonded *>(h);
    return guarded([&] { with_all_pairs(r->all_pairs.get(), [&](auto *a) { a->set_nblist_padding(padding); }); });
}

int tmref_disable_hilbert_sort(void *h) {
    auto *r = static_cast<RefNonbonded *>(h);
    return guarded([&] { with_all_pairs(r->all_pairs.get(), [&](auto *a) { a->disable_hilbert_sort(); }); });
}

int tmref_execute_device(
    void *h,
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
    auto *r = static_cast<RefNonbonded *>(h);
    return guarded([&] {
        r->fanout->execute_device(
            N, P, d_x, d_p, d_box, lambda, d_du_dx, d_du_dp, d_du_dl, d_u, static_cast<cudaStream_t>(stream));
    });
}

// A single reference potential (interaction group).
struct RefPot {
    std::shared_ptr<timemachine::Potential> pot;
};

void *tmref_group_create(
    const char *kernel_dir,
    int N,
    const int *row_idxs,
    int NR,
    const int *plane,
    const int *offset,
    double beta,
    double cutoff,
    int interpolated,
    int precision) { // 32 or 64
    RefPot *h = nullptr;
    int rc = guarded([&] {
        const std::string src = jit_source(kernel_dir);
        std::vector<int> pl(plane, plane + N), of(offset, offset + N);
        std::set<int> rows(row_idxs, row_idxs + NR);
        auto r = std::make_unique<RefPot>();
        auto build = [&](auto real_tag) {
            using Real = decltype(real_tag);
            if (interpolated) {
                r->pot = std::make_shared<timemachine::NonbondedInteractionGroup<Real, true>>(rows, pl, of, beta, cutoff, src);
            } else {
                r->pot = std::make_shared<timemachine::NonbondedInteractionGroup<Real, false>>(rows, pl, of, beta, cutoff, src);
            }
        };
        if (precision == 64) {
            build(double{});
        } else {
            build(float{});
        }
        h = r.release();
    });
    return rc == 0 ? h : nullptr;
}

void tmref_pot_destroy(void *h) { delete static_cast<RefPot *>(h); }

int tmref_pot_execute_host(
    void *h,
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
    auto *r = static_cast<RefPot *>(h);
    return guarded([&] { r->pot->execute_host(N, P, h_x, h_p, h_box, lambda, h_du_dx, h_du_dp, h_du_dl, h_u); });
}

int tmref_execute_host(
    void *h,
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
    auto *r = static_cast<RefNonbonded *>(h);
    return guarded([&] { r->fanout->execute_host(N, P, h_x, h_p, h_box, lambda, h_du_dx, h_du_dp, h_du_dl, h_u); });
}

// MD throughput of the reference runtime: Context(LangevinIntegrator, [Nonbonded], MonteCarloBarostat).
void *tmref_md_create(
    void *nonbonded,
    int N,
    const double *params, // [P]
    int P,
    const double *x0,
    const double *v0,
    const double *box0,
    double dt,
    double ca,
    const double *cbs,
    const double *ccs,
    int seed,
    double pressure,     // bar; <= 0: no barostat
    double temperature,  // K
    const int *group_of, // [N] molecule id of each atom (barostat groups)
    int barostat_interval,
    const int *bond_idxs, // [B,2]
    int B,
    const double *bond_params, // [B,2]
    const int *angle_idxs,     // [A,3]
    int A,
    const double *angle_params) { // [A,2]
    RefMD *h = nullptr;
    auto *nb = static_cast<RefNonbonded *>(nonbonded);
    int rc = guarded([&] {
        auto m = std::make_unique<RefMD>();
        m->intg = std::make_unique<timemachine::LangevinIntegrator>(N, dt, ca, cbs, ccs, seed);
        m->bp = std::make_unique<timemachine::BoundPotential>(nb->fanout, std::vector<int>{P / 3, 3}, params);
        std::vector<timemachine::BoundPotential *> bps;
        if (B > 0) {
            auto hb = std::make_shared<timemachine::HarmonicBond<float>>(
                std::vector<int>(bond_idxs, bond_idxs + 2 * (size_t)B), std::vector<int>(), std::vector<int>());
            m->bonded.push_back(std::make_unique<timemachine::BoundPotential>(hb, std::vector<int>{B, 2}, bond_params));
            bps.push_back(m->bonded.back().get());
        }
        if (A > 0) {
            auto ha = std::make_shared<timemachine::HarmonicAngle<float>>(
                std::vector<int>(angle_idxs, angle_idxs + 3 * (size_t)A), std::vector<int>(), std::vector<int>());
            m->bonded.push_back(std::make_unique<timemachine::BoundPotential>(ha, std::vector<int>{A, 2}, angle_params));
            bps.push_back(m->bonded.back().get());
        }
        bps.push_back(m->bp.get());
        if (pressure > 0) {
            int ngroups = 0;
            for (int i = 0; i < N; i++) {
                ngroups = std::max(ngroups, group_of[i] + 1);
            }
            std::vector<std::vector<int>> groups(ngroups);
            for (int i = 0; i < N; i++) {
                groups[group_of[i]].push_back(i);
            }
            m->baro = std::make_unique<timemachine::MonteCarloBarostat>(
                N, pressure, temperature, groups, barostat_interval, bps, seed + 1);
        }
        m->ctx = std::make_unique<timemachine::Context>(N, x0, v0, box0, m->intg.get(), bps, m->baro.get());
        h = m.release();
    });
    return rc == 0 ? h : nullptr;
}

int tmref_md_run(void *h, int n_steps, double lambda, double *x_out, double *box_out) {
    auto *m = static_cast<RefMD *>(h);
    return guarded([&] {
        std::vector<double> sched(n_steps, lambda);
        m->ctx->multiple_steps(sched, n_steps, n_steps);
        if (x_out) {
            m->ctx->get_x_t(x_out);
        }
        if (box_out) {
            m->ctx->get_box(box_out);
        }
    });
}

void tmref_md_destroy(void *h) { delete static_cast<RefMD *>(h); }

} // extern "C"
