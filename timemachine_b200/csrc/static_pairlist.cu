// Allocation-free evaluation of a NonbondedPairList (FP32, not interpolated):
// the scaled-pair part of the nonbonded pipeline (k_check_prepare, k_pair,
// k_finalize of nb_kernels.cuh) run on caller-owned device buffers, with the
// slot staging, the accumulators and the device state in one file-scope
// static device array instead of instance buffers from cudaMalloc.
//
// Declared in include/tmnb.h as tmnb_pair_list_execute_static. It has no
// reference counterpart; its results equal tmnb_potential_execute_device of a
// tmnb_pair_list_create handle with the same arguments.
#include "engine.hpp"
#include "nb_kernels.cuh"

#include <mutex>
#include <string>

namespace tmb {
namespace {

constexpr int SMAX = TMNB_STATIC_MAX_ATOMS;

constexpr size_t align256(size_t b) { return (b + 255) & ~size_t(255); }

// Byte offsets of the sections of the static scratch.
constexpr size_t OFF_POSW = 0;                                                     // float4 [SMAX]
constexpr size_t OFF_PRM = OFF_POSW + align256(sizeof(float4) * SMAX);             // float4 [SMAX]
constexpr size_t OFF_ACC = OFF_PRM + align256(sizeof(float4) * SMAX);              // u64 [8][SMAX]
constexpr size_t OFF_PERM = OFF_ACC + align256(sizeof(unsigned long long) * 8 * SMAX); // u32 [SMAX]
constexpr size_t OFF_LAMDEP = OFF_PERM + align256(sizeof(unsigned) * SMAX);        // u8 [SMAX]
constexpr size_t OFF_STATE = OFF_LAMDEP + align256(SMAX);                          // DevState
constexpr size_t SCRATCH_BYTES = OFF_STATE + align256(sizeof(DevState));           // 3.16 MiB

// Zero at module load. The accumulators and the device state's error word
// must be zero when a call starts: each call clears both on its stream before
// its first kernel (so a call that failed half-way cannot leak into the
// next), k_finalize takes (reads and zeroes) every accumulator it reads, and
// the error word is read back at the end. The slot order section holds the
// identity, written once by the set-up.
static __device__ __align__(256) unsigned char g_static_scratch[SCRATCH_BYTES];

constexpr int DEV_ERR_BAD_PAIR = 5;

__global__ void k_static_identity(unsigned *perm) {
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < SMAX; s += gridDim.x * blockDim.x) {
        perm[s] = (unsigned)s;
    }
}

// Pair indices must lie in [0, N) and differ (the check tmnb_pair_list_create
// makes on the host); otherwise the error word is set, and k_pair, which
// starts by reading it, returns before reading any pair.
__global__ void k_static_check_pairs(int N, int M, const int *pairs, DevState *state) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < M; k += gridDim.x * blockDim.x) {
        const int i = pairs[2 * k], j = pairs[2 * k + 1];
        if (i < 0 || i >= N || j < 0 || j >= N || i == j) {
            state->error = DEV_ERR_BAD_PAIR;
        }
    }
}

typedef void (*static_pair_kernel_t)(PairArgs);

template <int I> constexpr static_pair_kernel_t static_kernel() {
    return &k_pair<float, bool((I >> 3) & 1), bool((I >> 2) & 1), bool((I >> 1) & 1), bool((I >> 0) & 1), false,
                   false>;
}
template <int... Is> struct StaticKernels {
    static void fill(static_pair_kernel_t *out) { ((out[Is] = static_kernel<Is>()), ...); }
};

struct DeviceSetup {
    unsigned char *scratch = nullptr;
    int pair_grid[16] = {};
};

constexpr int MAX_DEVICES = 64;
std::mutex g_setup_mutex;
DeviceSetup g_setup[MAX_DEVICES];
static_pair_kernel_t g_kernels[16];
bool g_kernels_filled = false;

// Once per device, with that device current: loads the kernels, looks up the
// scratch address (cudaGetSymbolAddress, return code checked), writes the
// identity slot order and synchronises the device. Later calls only read the
// cached values.
const DeviceSetup &setup_for_current_device() {
    int dev = 0;
    CK(cudaGetDevice(&dev));
    if (dev < 0 || dev >= MAX_DEVICES) {
        throw Error(TMNB_ERR_UNSUPPORTED, "device ordinal beyond the static scratch table");
    }
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (!g_kernels_filled) {
        StaticKernels<0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 13, 14, 15>::fill(g_kernels);
        g_kernels_filled = true;
    }
    DeviceSetup &d = g_setup[dev];
    if (d.scratch == nullptr) {
        void *p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_static_scratch);
        if (e != cudaSuccess || p == nullptr) {
            throw Error(
                TMNB_ERR_CUDA, std::string("cudaGetSymbolAddress(static scratch) failed: ") + cudaGetErrorString(e));
        }
        const int sms = num_sms();
        for (int k = 0; k < 16; k++) {
            int per_sm = 0;
            CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, g_kernels[k], 128, 0));
            d.pair_grid[k] = (per_sm > 0 ? per_sm : 1) * sms;
        }
        cudaFuncAttributes attr;
        CK(cudaFuncGetAttributes(&attr, k_check_prepare));
        CK(cudaFuncGetAttributes(&attr, k_finalize));
        CK(cudaFuncGetAttributes(&attr, k_static_check_pairs));
        unsigned char *base = static_cast<unsigned char *>(p);
        k_static_identity<<<64, 256>>>(reinterpret_cast<unsigned *>(base + OFF_PERM));
        CK(cudaPeekAtLastError());
        CK(cudaDeviceSynchronize());
        d.scratch = base;
    }
    return d;
}

void execute_static(
    int N,
    int M,
    const int *d_pair_idxs,
    const double *d_scales,
    const int *d_plane,
    const int *d_offset,
    double beta,
    double cutoff,
    int negated,
    const double *d_x,
    const double *d_p,
    const double *d_box,
    double lambda,
    unsigned long long *d_du_dx,
    unsigned long long *d_du_dp,
    unsigned long long *d_du_dl,
    unsigned long long *d_u,
    cudaStream_t stream) {
    if (N <= 0) {
        throw Error(TMNB_ERR_INVALID_ARGUMENT, "N must be positive");
    }
    if (N > SMAX) {
        throw Error(
            TMNB_ERR_INVALID_ARGUMENT,
            "N=" + std::to_string(N) + " exceeds the static scratch capacity of " + std::to_string(SMAX) +
                " atoms (TMNB_STATIC_MAX_ATOMS)");
    }
    if (M < 0 || (M > 0 && (!d_pair_idxs || !d_scales))) {
        throw Error(TMNB_ERR_INVALID_ARGUMENT, "M must be >= 0, with pair indices and scales when M > 0");
    }
    if (!(cutoff > 0)) {
        throw Error(TMNB_ERR_INVALID_ARGUMENT, "cutoff must be positive");
    }
    if (!d_plane || !d_offset || !d_x || !d_p || !d_box) {
        throw Error(TMNB_ERR_INVALID_ARGUMENT, "plane, offset, x, params and box must be non-null");
    }
    const DeviceSetup &d = setup_for_current_device();
    unsigned char *base = d.scratch;
    float4 *posw = reinterpret_cast<float4 *>(base + OFF_POSW);
    float4 *prm = reinterpret_cast<float4 *>(base + OFF_PRM);
    unsigned long long *acc = reinterpret_cast<unsigned long long *>(base + OFF_ACC);
    const unsigned *perm = reinterpret_cast<const unsigned *>(base + OFF_PERM);
    unsigned char *lamdep = base + OFF_LAMDEP;
    DevState *state = reinterpret_cast<DevState *>(base + OFF_STATE);

    Accum c;
    c.x = acc + 0 * (size_t)SMAX;
    c.y = acc + 1 * (size_t)SMAX;
    c.z = acc + 2 * (size_t)SMAX;
    c.q = acc + 3 * (size_t)SMAX;
    c.sig = acc + 4 * (size_t)SMAX;
    c.eps = acc + 5 * (size_t)SMAX;
    c.u = acc + 6 * (size_t)SMAX;
    c.dl = acc + 7 * (size_t)SMAX;
    c.pq = c.q;
    c.psig = c.sig;
    c.peps = c.eps;

    PrepareArgs pa;
    pa.N = N;
    pa.S = N;
    pa.x = d_x;
    pa.p = d_p;
    pa.box = d_box;
    pa.K = 1;
    for (int k = 0; k < MAX_WINDOWS; k++) {
        // identity lambda transform: f = lambda, df/dlambda = 1
        const double l = k == 0 ? lambda : 0.0;
        pa.lam[k] = LambdaWindow{l, 1.0, l, 1.0, l, 1.0, l, 1.0};
    }
    pa.cutoff = cutoff;
    pa.padding = 0.0;
    pa.plane = d_plane;
    pa.offset = d_offset;
    pa.interpolated = 0;
    pa.slots.posw = posw;
    pa.slots.prm = prm;
    pa.slots.dprm = nullptr;
    pa.slots.lamdep = lamdep;
    pa.slots.posw64 = nullptr;
    pa.slots.prm64 = nullptr;
    pa.slots.dprm64 = nullptr;

    // Every call starts from a clean state on the caller's stream: the error
    // word and the accumulators are cleared here, not only at the end of the
    // previous call, so a call that stopped half-way leaves nothing behind.
    CK(cudaMemsetAsync(&state->error, 0, sizeof(int), stream));
    CK(cudaMemsetAsync(acc, 0, sizeof(unsigned long long) * 8 * (size_t)SMAX, stream));

    const int tpb = 256;
    const int sgrid = std::max(1, std::min((N + tpb - 1) / tpb, 8 * num_sms()));
    k_check_prepare<<<sgrid, tpb, 0, stream>>>(pa, perm, nullptr, nullptr, state);
    CK(cudaPeekAtLastError());
    if (M > 0) {
        const int cgrid = std::max(1, std::min((M + tpb - 1) / tpb, 8 * num_sms()));
        k_static_check_pairs<<<cgrid, tpb, 0, stream>>>(N, M, d_pair_idxs, state);
        CK(cudaPeekAtLastError());
    }

    const int kidx = (d_du_dp ? 1 : 0) | (d_du_dl ? 2 : 0) | (d_du_dx ? 4 : 0) | (d_u ? 8 : 0);
    if (kidx != 0) {
        PairArgs a;
        a.S = N;
        a.row_end = N;
        a.K = 1;
        a.posw = posw;
        a.prm = prm;
        a.dprm = nullptr;
        a.posw64 = nullptr;
        a.prm64 = nullptr;
        a.dprm64 = nullptr;
        a.lamdep = lamdep;
        a.box = d_box;
        a.beta = beta;
        a.cutoff = cutoff;
        a.tile_cols = nullptr;
        a.items = nullptr;
        a.M = M;
        a.pair_idxs = d_pair_idxs;
        a.scales = d_scales;
        a.slot_of = nullptr;
        a.negated = negated ? 1 : 0;
        a.acc = c;
        a.acc_block = 8 * (size_t)SMAX;
        a.dep_tiles = nullptr;
        a.state = state;
        g_kernels[kidx]<<<d.pair_grid[kidx], 128, 0, stream>>>(a);
        CK(cudaPeekAtLastError());

        FinalizeArgs fa;
        fa.N = N;
        fa.S = N;
        fa.K = 1;
        for (int k = 0; k < MAX_WINDOWS; k++) {
            fa.f_dp[k][0] = fa.f_dp[k][1] = fa.f_dp[k][2] = pa.lam[k].f_q;
        }
        fa.set_atoms = nullptr;
        fa.slot_of = nullptr;
        fa.take = 1;
        fa.acc = c;
        fa.acc_block = 8 * (size_t)SMAX;
        fa.split_pair_dp = 0;
        fa.interpolated = 0;
        fa.du_dx = d_du_dx;
        fa.du_dp = d_du_dp;
        fa.du_dl = d_du_dl;
        fa.u = d_u;
        fa.stride_x = 3 * (size_t)N;
        fa.stride_p = 3 * (size_t)N;
        fa.stride_n = (size_t)N;
        fa.state = state;
        k_finalize<<<sgrid, tpb, 0, stream>>>(fa);
        CK(cudaPeekAtLastError());
    }

    // report (and clear) a pair-index error found on the device; all traffic
    // stays on the caller's stream (no legacy-default-stream copies)
    int err = 0;
    CK(cudaMemcpyAsync(&err, &state->error, sizeof(int), cudaMemcpyDeviceToHost, stream));
    CK(cudaStreamSynchronize(stream));
    if (err != 0) {
        CK(cudaMemsetAsync(&state->error, 0, sizeof(int), stream));
        throw Error(TMNB_ERR_INVALID_ARGUMENT, "pair index out of range [0, N) or src == dst; outputs left unchanged");
    }
}

} // namespace
} // namespace tmb

extern "C" tmnb_status tmnb_pair_list_execute_static(
    int N,
    int M,
    const int32_t *d_pair_idxs,
    const double *d_scales,
    const int32_t *d_lambda_plane_idxs,
    const int32_t *d_lambda_offset_idxs,
    double beta,
    double cutoff,
    int negated,
    const double *d_x,
    const double *d_p,
    const double *d_box,
    double lambda,
    unsigned long long *d_du_dx,
    unsigned long long *d_du_dp,
    unsigned long long *d_du_dl,
    unsigned long long *d_u,
    void *stream) {
    return tmb::guarded([&] {
        tmb::execute_static(
            N, M, d_pair_idxs, d_scales, d_lambda_plane_idxs, d_lambda_offset_idxs, beta, cutoff, negated, d_x, d_p,
            d_box, lambda, d_du_dx, d_du_dp, d_du_dl, d_u, static_cast<cudaStream_t>(stream));
    });
}
