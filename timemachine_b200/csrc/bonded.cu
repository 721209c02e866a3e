// Harmonic bond and (cosine) harmonic angle potentials, FP32 with int64
// fixed-point accumulation. They are MD-driver dependencies of the nonbonded
// path (molecules need their bonded terms for a stable trajectory), with the
// reference's functional forms:
//   bond  U = kb/2 (|r_ij| - b0)^2        timemachine/cpp/src/kernels/k_harmonic_bond.cuh:4-76
//   angle U = ka/2 (cos(theta) - cos a0)^2 timemachine/cpp/src/kernels/k_harmonic_angle.cuh:4-90
// each scaled by (lambda_offset + lambda_mult * lambda); params [T, 2] = (k, r0 | a0).
// No periodic wrapping (molecules are kept whole), as in the reference.
#include "engine.hpp"
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
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= B) {
        return;
    }
    const int i = idxs[2 * b], j = idxs[2 * b + 1];
    Real dx[3];
    Real d2 = 0;
    for (int d = 0; d < 3; d++) {
        dx[d] = (Real)x[3 * i + d] - (Real)x[3 * j + d];
        d2 += dx[d] * dx[d];
    }
    const Real kb = params[2 * b], b0 = params[2 * b + 1];
    const Real dij = sqrt(d2);
    const Real db = dij - b0;
    const Real pre = loff[b] + lmult[b] * (Real)lambda;
    if (du_dx) {
        for (int d = 0; d < 3; d++) {
            const Real g = (b0 != 0 ? kb * db * dx[d] / dij : kb * dx[d]) * pre;
            const unsigned long long f = to_fixed(g, FX_EXPONENT);
            atomicAdd(du_dx + 3 * i + d, f);
            atomicAdd(du_dx + 3 * j + d, 0ULL - f);
        }
    }
    if (du_dp) {
        atomicAdd(du_dp + 2 * b, to_fixed((Real)0.5 * db * db * pre, FX_EXPONENT));
        atomicAdd(du_dp + 2 * b + 1, to_fixed(-kb * db * pre, FX_EXPONENT));
    }
    if (u) {
        atomicAdd(u + i, to_fixed(kb / 2 * db * db * pre, FX_EXPONENT));
    }
    if (du_dl) {
        atomicAdd(du_dl + i, to_fixed(lmult[b] * kb / 2 * db * db, FX_EXPONENT));
    }
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
    const int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= A) {
        return;
    }
    const int i = idxs[3 * a], j = idxs[3 * a + 1], k = idxs[3 * a + 2];
    Real rij[3], rkj[3];
    Real nij2 = 0, nkj2 = 0, dot = 0;
    for (int d = 0; d < 3; d++) {
        rij[d] = (Real)x[3 * i + d] - (Real)x[3 * j + d]; // j -> i
        rkj[d] = (Real)x[3 * k + d] - (Real)x[3 * j + d]; // j -> k
        nij2 += rij[d] * rij[d];
        nkj2 += rkj[d] * rkj[d];
        dot += rij[d] * rkj[d];
    }
    const Real inij = (Real)1 / sqrt(nij2), inkj = (Real)1 / sqrt(nkj2);
    const Real cos_t = dot * inij * inkj;
    const Real ka = params[2 * a], a0 = params[2 * a + 1];
    const Real delta = cos_t - cos(a0);
    const Real pre = loff[a] + lmult[a] * (Real)lambda;
    if (du_dx) {
        const Real f = ka * delta * pre;
        for (int d = 0; d < 3; d++) {
            // d cos / d x_i and d x_k; x_j takes the negated sum
            const Real gi = (rkj[d] * inij * inkj - cos_t * rij[d] * inij * inij) * f;
            const Real gk = (rij[d] * inij * inkj - cos_t * rkj[d] * inkj * inkj) * f;
            const unsigned long long fi = to_fixed(gi, FX_EXPONENT);
            const unsigned long long fk = to_fixed(gk, FX_EXPONENT);
            atomicAdd(du_dx + 3 * i + d, fi);
            atomicAdd(du_dx + 3 * k + d, fk);
            atomicAdd(du_dx + 3 * j + d, 0ULL - fi - fk);
        }
    }
    if (du_dp) {
        atomicAdd(du_dp + 2 * a, to_fixed(delta * delta / 2 * pre, FX_EXPONENT));
        atomicAdd(du_dp + 2 * a + 1, to_fixed(delta * ka * sin(a0) * pre, FX_EXPONENT));
    }
    if (u) {
        atomicAdd(u + i, to_fixed(ka / 2 * delta * delta * pre, FX_EXPONENT));
    }
    if (du_dl) {
        atomicAdd(du_dl + i, to_fixed(lmult[a] * ka / 2 * delta * delta, FX_EXPONENT));
    }
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
            k_harmonic_bond<float><<<blocks, tpb, 0, stream>>>(
                T_, d_x, d_p, lambda, mult_.p, off_.p, idxs_.p, d_du_dx, d_du_dp, d_du_dl, d_u);
        } else {
            k_harmonic_angle<float><<<blocks, tpb, 0, stream>>>(
                T_, d_x, d_p, lambda, mult_.p, off_.p, idxs_.p, d_du_dx, d_du_dp, d_du_dl, d_u);
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
