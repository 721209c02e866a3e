// Shared host-side plumbing of libtmnb: error type, CUDA checks, device
// buffers and the abstract potential interface that the MD context drives.
#pragma once

#include "tmnb.h"

#include <cuda_runtime.h>

#include <memory>
#include <stdexcept>
#include <string>
#include <utility>

namespace tmb {

inline thread_local std::string g_last_error;

struct Error : std::runtime_error {
    tmnb_status status;
    Error(tmnb_status s, const std::string &msg) : std::runtime_error(msg), status(s) {}
};

inline void cuda_check(cudaError_t e, const char *what) {
    if (e != cudaSuccess) {
        throw Error(TMNB_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
    }
}
#define CK(call) ::tmb::cuda_check((call), #call)

// Launch with programmatic stream serialization: the kernel's launch may
// overlap the drain of the previous kernel in the stream, so the kernel must
// execute griddepcontrol.wait (grid_dependency_wait()) before it reads or
// writes anything the previous kernel touches.
template <typename... KArgs, typename... Args>
inline void launch_dependent(
    void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t stream, Args &&...args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    CK(cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...));
}

template <typename T> struct DevBuf {
    T *p = nullptr;
    size_t n = 0;
    DevBuf() = default;
    DevBuf(const DevBuf &) = delete;
    DevBuf &operator=(const DevBuf &) = delete;
    ~DevBuf() { release(); }
    void release() {
        if (p) {
            cudaFree(p);
        }
        p = nullptr;
        n = 0;
    }
    void alloc(size_t count) {
        release();
        if (count == 0) {
            return;
        }
        CK(cudaMalloc(&p, count * sizeof(T)));
        n = count;
    }
    void ensure(size_t count) {
        if (count > n) {
            alloc(count);
        }
    }
    void upload(const T *h, size_t count) {
        alloc(count);
        if (count) {
            CK(cudaMemcpy(p, h, count * sizeof(T), cudaMemcpyHostToDevice));
        }
    }
    void zero() {
        if (n) {
            CK(cudaMemset(p, 0, n * sizeof(T)));
        }
    }
};

inline int num_sms() {
    static int sms = -1;
    if (sms < 0) {
        int dev = 0;
        CK(cudaGetDevice(&dev));
        CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    }
    return sms;
}

// Device-level contract of a potential (timemachine/cpp/src/potential.hpp:51-62).
// What an MD integrator kernel needs to take over a potential's per-step
// coordinate staging and force scatter (single lambda window, forces only):
// the slot order, the staged coordinates, the neighbour-list reference
// coordinates and flags, and the slot-ordered fixed-point force accumulators.
struct MDFusion {
    const int *slot_of;      // [N] atom -> slot
    float4 *posw;            // [S] staged x, y, z, w (the integrator writes x, y, z)
    const double *nb_x;      // [N,3] coordinates at the last neighbour-list rebuild
    double half_pad2;        // (padding / 2)^2
    int *rebuild;            // set to 1 when an atom moved more than padding / 2
    int *next_item;          // the pair kernel's work counter, reset for the next step
    const int *error;        // nonzero: the potential failed, its forces are not added
    unsigned long long *acc; // [3][S] slot-ordered fixed-point forces x, y, z
    int S;
};

class PotentialBase {
  public:
    virtual ~PotentialBase() { release_host_stream(); }
    virtual void execute_device(
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
        cudaStream_t stream) = 0;
    // An independent instance with the same parameters (own neighbour list).
    virtual std::unique_ptr<PotentialBase> clone() const = 0;
    virtual int num_atoms() const = 0;
    virtual int num_params() const = 0;
    virtual tmnb_status check_device_error(cudaStream_t stream) = 0;

    // Fixed-point du_dp to float (2^36 for every entry unless overridden).
    virtual void du_dp_fixed_to_float(int N, int P, const unsigned long long *du_dp, double *out) const {
        (void)N;
        for (int i = 0; i < P; i++) {
            out[i] = static_cast<double>(static_cast<long long>(du_dp[i])) / static_cast<double>(0x1000000000ULL);
        }
    }

    // Counts the changes to what launches recorded in a CUDA graph hold:
    // reallocated device buffers (staging, accumulators, tile lists) and
    // settings passed by value (padding, lambda schedules, sort order). A
    // graph captured before a change must not be replayed after it.
    virtual unsigned long long buffer_generation() const { return 0; }

    // MD integrator fusion: fills `f` and returns true when this potential can
    // leave its forces in slot-ordered accumulators for the integrator kernel
    // and take coordinates staged by it.
    virtual bool md_fusion(MDFusion &f) {
        (void)f;
        return false;
    }

    // Forces of one MD step for a fused integrator (only when md_fusion() is
    // true): the forces stay in MDFusion::acc, where the integrator kernel
    // reads them; `prestaged` = the previous integrator kernel staged these
    // coordinates, took the neighbour-list test and reset the work counter
    // (same lambda, parameters and box as the previous call).
    virtual void execute_md_fused(
        int N, int P, const double *d_x, const double *d_p, const double *d_box, double lambda, bool prestaged,
        cudaStream_t stream) {
        (void)N, (void)P, (void)d_x, (void)d_p, (void)d_box, (void)lambda, (void)prestaged, (void)stream;
        throw Error(TMNB_ERR_INTERNAL, "potential has no fused MD path");
    }

    // K lambda windows on the same coordinates and parameters; output k of
    // each array starts at k * (3N | P | N). Potentials without a fused
    // multi-window path evaluate the windows one after the other.
    virtual void execute_windows_device(
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
        cudaStream_t stream) {
        for (int k = 0; k < K; k++) {
            execute_device(
                N,
                P,
                d_x,
                d_p,
                d_box,
                lambdas[k],
                d_du_dx ? d_du_dx + (size_t)k * 3 * N : nullptr,
                d_du_dp ? d_du_dp + (size_t)k * P : nullptr,
                d_du_dl ? d_du_dl + (size_t)k * N : nullptr,
                d_u ? d_u + (size_t)k * N : nullptr,
                stream);
        }
    }

    // Potential::execute_host (timemachine/cpp/src/potential.cu:110-185): copy in,
    // zero and compute the selected outputs, copy out, synchronise. The device
    // staging buffers are kept by the instance and reused.
    void execute_host(
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
        execute_windows_host(N, P, h_x, h_p, h_box, 1, &lambda, h_du_dx, h_du_dp, h_du_dl, h_u);
    }

    // execute_host over K lambda windows (outputs laid out as in
    // execute_windows_device).
    void execute_windows_host(
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
        if (!host_stream_) {
            CK(cudaStreamCreateWithFlags(&host_stream_, cudaStreamNonBlocking));
        }
        cudaStream_t s = host_stream_;
        const size_t nx = 3 * (size_t)N;
        const size_t np = P > 0 ? (size_t)P : 1;
        const size_t kk = K > 0 ? (size_t)K : 1;
        hx_.ensure(nx);
        hp_.ensure(np);
        hbox_.ensure(9);
        CK(cudaMemcpyAsync(hx_.p, h_x, nx * sizeof(double), cudaMemcpyHostToDevice, s));
        if (P > 0) {
            CK(cudaMemcpyAsync(hp_.p, h_p, (size_t)P * sizeof(double), cudaMemcpyHostToDevice, s));
        }
        CK(cudaMemcpyAsync(hbox_.p, h_box, 9 * sizeof(double), cudaMemcpyHostToDevice, s));
        unsigned long long *dx = nullptr, *dp = nullptr, *dl = nullptr, *du = nullptr;
        if (h_du_dx) {
            hdx_.ensure(kk * nx);
            dx = hdx_.p;
            CK(cudaMemsetAsync(dx, 0, kk * nx * sizeof(*dx), s));
        }
        if (h_du_dp) {
            hdp_.ensure(kk * np);
            dp = hdp_.p;
            CK(cudaMemsetAsync(dp, 0, kk * np * sizeof(*dp), s));
        }
        if (h_du_dl) {
            hdl_.ensure(kk * N);
            dl = hdl_.p;
            CK(cudaMemsetAsync(dl, 0, kk * N * sizeof(*dl), s));
        }
        if (h_u) {
            hu_.ensure(kk * N);
            du = hu_.p;
            CK(cudaMemsetAsync(du, 0, kk * N * sizeof(*du), s));
        }
        execute_windows_device(N, P, hx_.p, hp_.p, hbox_.p, K, lambdas, dx, dp, dl, du, s);
        if (h_du_dx) {
            CK(cudaMemcpyAsync(h_du_dx, dx, kk * nx * sizeof(*dx), cudaMemcpyDeviceToHost, s));
        }
        if (h_du_dp) {
            CK(cudaMemcpyAsync(h_du_dp, dp, kk * (size_t)P * sizeof(*dp), cudaMemcpyDeviceToHost, s));
        }
        if (h_du_dl) {
            CK(cudaMemcpyAsync(h_du_dl, dl, kk * N * sizeof(*dl), cudaMemcpyDeviceToHost, s));
        }
        if (h_u) {
            CK(cudaMemcpyAsync(h_u, du, kk * N * sizeof(*du), cudaMemcpyDeviceToHost, s));
        }
        CK(cudaStreamSynchronize(s));
        check_device_error(s);
    }

  protected:
    void release_host_stream() {
        if (host_stream_) {
            cudaStreamDestroy(host_stream_);
            host_stream_ = nullptr;
        }
    }
    cudaStream_t host_stream_ = nullptr;
    DevBuf<double> hx_, hp_, hbox_;
    DevBuf<unsigned long long> hdx_, hdp_, hdl_, hu_;
};

template <typename F> tmnb_status guarded(F &&f) {
    try {
        f();
        return TMNB_OK;
    } catch (const Error &e) {
        g_last_error = e.what();
        return e.status;
    } catch (const std::bad_alloc &) {
        g_last_error = "host allocation failed";
        return TMNB_ERR_INTERNAL;
    } catch (const std::exception &e) {
        g_last_error = e.what();
        return TMNB_ERR_INTERNAL;
    }
}

} // namespace tmb

struct tmnb_potential {
    std::unique_ptr<tmb::PotentialBase> impl;
};
