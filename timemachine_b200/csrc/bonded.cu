// Harmonic bond and (cosine) harmonic angle potentials, FP32 with int64
// fixed-point accumulation. They are MD-driver dependencies of the nonbonded
// path (molecules need their bonded terms for a stable trajectory), with the
// reference's functional forms:
//   bond  U = kb/2 (|r_ij| - b0)^2        timemachine/cpp/src/kernels/k_harmonic_bond.cuh:4-76
//   angle U = ka/2 (cos(theta) - cos a0)^2 timemachine/cpp/src/kernels/k_harmonic_angle.cuh:4-90
// each scaled by (lambda_offset + lambda_mult * lambda); params [T, 2] = (k, r0 | a0).
// No periodic wrapping (molecules are kept whole), as in the reference.
#include "engine.hpp"
#include "bonded_math.cuh"
#include "nb_pair_math.cuh"

#include <algorithm>
#include <vector>

namespace tmb {

namespace {

template <typename Real>
__global__ void k_harmonic_bond(
    int B,
    const double *__restrict__ x,
    const double *__restrict__ params,
    double lambda,
    const int *__restrict__ lmult,
    const int *__restrict__ loff,
    const int *__restrict__ idxs,
    unsigned long long *__restrict__ du_dx,
    unsigned long long *__restrict__ du_dp,
    unsigned long long *__restrict__ du_dl,
    unsigned long long *__restrict__ u) {
    grid_dependency_wait();
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= B) {
        return;
    }
    harmonic_bond_term(
        x, idxs[2 * b], idxs[2 * b + 1], params[2 * b], params[2 * b + 1], lmult[b], loff[b], lambda, du_dx,
        du_dp ? du_dp + 2 * b : nullptr, du_dl, u);
}

template <typename Real>
__global__ void k_harmonic_angle(
    int A,
    const double *__restrict__ x,
    const double *__restrict__ params,
    double lambda,
    const int *__restrict__ lmult,
    const int *__restrict__ loff,
    const int *__restrict__ idxs,
    unsigned long long *__restrict__ du_dx,
    unsigned long long *__restrict__ du_dp,
    unsigned long long *__restrict__ du_dl,
    unsigned long long *__restrict__ u) {
    grid_dependency_wait();
    const int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= A) {
        return;
    }
    harmonic_angle_term(
        x, idxs[3 * a], idxs[3 * a + 1], idxs[3 * a + 2], params[2 * a], params[2 * a + 1], lmult[a], loff[a], lambda,
        du_dx, du_dp ? du_dp + 2 * a : nullptr, du_dl, u);
}

} // namespace

class BondedPotential : public PotentialBase {
  public:
    // arity 2: harmonic bond, 3: harmonic angle
    BondedPotential(int N, int arity, int T, const int *idxs, const int *lmult, const int *loff)
        : N_(N), arity_(arity), T_(T), h_idxs_(idxs, idxs + (size_t)arity * T) {
        if (T < 0) {
            throw Error(TMNB_ERR_INVALID_ARGUMENT, "invalid bonded term count");
        }
        int max_idx = -1;
        for (int v : h_idxs_) {
            if (v < 0 || (N > 0 && v >= N)) {
                throw Error(TMNB_ERR_INVALID_ARGUMENT, "bonded atom index out of range [0, N)");
            }
            max_idx = std::max(max_idx, v);
        }
        // N <= 0: like the reference, the term list does not fix N; any N above
        // the largest index is accepted at execution time
        min_N_ = max_idx + 1;
        h_mult_ = lmult ? std::vector<int>(lmult, lmult + T) : std::vector<int>(T, 0);
        h_off_ = loff ? std::vector<int>(loff, loff + T) : std::vector<int>(T, 1);
        idxs_.upload(h_idxs_.data(), h_idxs_.size());
        mult_.upload(h_mult_.data(), T);
        off_.upload(h_off_.data(), T);
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
        if ((N_ > 0 && N != N_) || N < min_N_) {
            throw Error(TMNB_ERR_INVALID_ARGUMENT, "bonded potential: atom count does not cover the term indices");
        }
        if (P != 2 * T_) {
            throw Error(TMNB_ERR_INVALID_ARGUMENT, "bonded potential: expected P == 2*T");
        }
        (void)d_box;
        if (T_ == 0 || !(d_du_dx || d_du_dp || d_du_dl || d_u)) {
            return;
        }
        const int tpb = 128;
        const int blocks = (T_ + tpb - 1) / tpb;
        if (arity_ == 2) {
            launch_dependent(
                k_harmonic_bond<float>, dim3(blocks), dim3(tpb), 0, stream, T_, d_x, d_p, lambda, mult_.p, off_.p, idxs_.p,
                d_du_dx, d_du_dp, d_du_dl, d_u);
        } else {
            launch_dependent(
                k_harmonic_angle<float>, dim3(blocks), dim3(tpb), 0, stream, T_, d_x, d_p, lambda, mult_.p, off_.p,
                idxs_.p, d_du_dx, d_du_dp, d_du_dl, d_u);
        }
        CK(cudaPeekAtLastError());
    }

    std::unique_ptr<PotentialBase> clone() const override {
        return std::make_unique<BondedPotential>(N_, arity_, T_, h_idxs_.data(), h_mult_.data(), h_off_.data());
    }
    int num_atoms() const override { return N_ > 0 ? N_ : -1; }
    int num_params() const override { return 2 * T_; }
    tmnb_status check_device_error(cudaStream_t) override { return TMNB_OK; }

  private:
    int N_, arity_, T_;
    int min_N_ = 0;
    std::vector<int> h_idxs_, h_mult_, h_off_;
    DevBuf<int> idxs_, mult_, off_;
};

} // namespace tmb

extern "C" {

tmnb_status tmnb_harmonic_bond_create(
    int N, int B, const int32_t *bond_idxs, const int32_t *lambda_mult, const int32_t *lambda_offset, tmnb_potential **out) {
    if (!out || (B > 0 && !bond_idxs)) {
        tmb::g_last_error = "null argument";
        return TMNB_ERR_INVALID_ARGUMENT;
    }
    return tmb::guarded([&] {
        auto h = std::make_unique<tmnb_potential>();
        h->impl = std::make_unique<tmb::BondedPotential>(N, 2, B, bond_idxs, lambda_mult, lambda_offset);
        *out = h.release();
    });
}

tmnb_status tmnb_harmonic_angle_create(
    int N, int A, const int32_t *angle_idxs, const int32_t *lambda_mult, const int32_t *lambda_offset, tmnb_potential **out) {
    if (!out || (A > 0 && !angle_idxs)) {
        tmb::g_last_error = "null argument";
        return TMNB_ERR_INVALID_ARGUMENT;
    }
    return tmb::guarded([&] {
        auto h = std::make_unique<tmnb_potential>();
        h->impl = std::make_unique<tmb::BondedPotential>(N, 3, A, angle_idxs, lambda_mult, lambda_offset);
        *out = h.release();
    });
}

} // extern "C"
