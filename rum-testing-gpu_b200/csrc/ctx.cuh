// The library context: one device, one stream, cached lattice tables and workspaces.
#pragma once
#include <atomic>
#include <array>
#include <map>
#include <memory>
#include <mutex>

#include "common.cuh"

struct rumb_ctx;

namespace rumb {

struct BmWorkBase {
    virtual ~BmWorkBase() {}
};

struct Ctx {
    int device = 0;
    cudaStream_t own = nullptr;       // the context's stream (work always runs here)
    cudaStream_t user = nullptr;      // optional caller stream, joined by events
    cudaEvent_t ev_a = nullptr, ev_b = nullptr;
    std::atomic<int> cancel{0};
    // popcount-ordered node ids per n (int32, ascending inside a layer) and layer bounds
    std::map<int, std::shared_ptr<DevBuf>> layers;
    std::map<int, std::vector<ll>> layer_bounds;
    std::unique_ptr<BmWorkBase> bm64, bm32;     // BM-ADMM workspaces
    std::unique_ptr<BmWorkBase> batch64, batch32;  // batched-draw workspaces
    std::unique_ptr<BmWorkBase> cert;           // float64 certificate workspace
    std::unique_ptr<BmWorkBase> scratch;        // primitive calls' scratch
    // the iteration's tuned schedule per (n, state bytes): transform low-window size, prox form,
    // fused passes (0 / 1)
    std::map<std::pair<int, int>, std::array<int, 3>> tuned;
    // overlapped checks: a second stream, its two events and pinned result words (made on first use)
    cudaStream_t aux = nullptr;
    cudaEvent_t ev_snap = nullptr, ev_done = nullptr;
    double *res_host = nullptr;
    void ensure_aux() {
        if (aux) return;
        RUMB_CUDA(cudaStreamCreateWithFlags(&aux, cudaStreamNonBlocking));
        RUMB_CUDA(cudaEventCreateWithFlags(&ev_snap, cudaEventDisableTiming));
        RUMB_CUDA(cudaEventCreateWithFlags(&ev_done, cudaEventDisableTiming));
        RUMB_CUDA(cudaMallocHost(&res_host, 64 * sizeof(double)));
    }

    // Make the context's stream wait for the caller's stream (call start) ...
    void join_in() {
        if (user) {
            RUMB_CUDA(cudaEventRecord(ev_a, user));
            RUMB_CUDA(cudaStreamWaitEvent(own, ev_a, 0));
        }
    }
    // ... and the caller's stream wait for the context's (call end).
    void join_out() {
        if (user) {
            RUMB_CUDA(cudaEventRecord(ev_b, own));
            RUMB_CUDA(cudaStreamWaitEvent(user, ev_b, 0));
        }
    }
    const int *layer_table(int n, std::vector<ll> &bounds);
};

// RAII: make ctx's device current for the duration of a call
struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int dev) {
        cudaGetDevice(&prev);
        if (prev != dev) RUMB_CUDA(cudaSetDevice(dev));
    }
    ~DeviceGuard() {
        int cur = -1;
        cudaGetDevice(&cur);
        if (prev >= 0 && cur != prev) cudaSetDevice(prev);
    }
};

}  // namespace rumb

struct rumb_ctx {
    rumb::Ctx c;
};

// A kept ADMM state (x2, s, y, z) on the device.
struct rumb_bm_state {
    int n = 0;
    int dtype = RUMB_F64;   // element type of the slabs (RUMB_F64 or RUMB_F32)
    int device = 0;
    rumb::DevBuf x2, s, y, z;
};
