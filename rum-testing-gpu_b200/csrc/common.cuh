// Shared definitions of the rumb CUDA library (sm_100a): error handling, the context, the slab
// layout helpers and small device utilities.
//
// Slab layout (the reference's Block-Marschak layout, solver/bm_admm/kernels.py:24-35): a slab holds
// one value per (alternative x, menu S containing x) at x * 2^(n-1) + compress(S \ {x}, x), where
// compress drops bit x and shifts the higher bits down. Alternative x's 2^(n-1) entries form its
// "block"; the butterflies act on the n-1 "rest" bits of each block.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <atomic>
#include <cmath>
#include <cstdlib>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/rumb.h"

namespace rumb {

typedef long long ll;
typedef unsigned long long ull;

// ---------------------------------------------------------------- errors (host)
struct Error : public std::runtime_error {
    int code;
    Error(int c, const std::string &m) : std::runtime_error(m), code(c) {}
};

inline void fail(int code, const std::string &msg) { throw Error(code, msg); }

inline void cuda_check(cudaError_t e, const char *what) {
    if (e == cudaSuccess) return;
    cudaGetLastError();  // clear a sticky launch error so the context stays usable
    int code = (e == cudaErrorMemoryAllocation) ? RUMB_E_OOM : RUMB_E_CUDA;
    throw Error(code, std::string(what) + ": " + cudaGetErrorString(e));
}

#define RUMB_CUDA(call) ::rumb::cuda_check((call), #call)
// Kernels launched by the calling thread: RUMB_LAUNCH counts each launch, a CUDA graph replay adds
// the kernels it captured; the C ABI reports the difference over a call.
inline thread_local long long g_launches = 0;
#define RUMB_LAUNCH(what) (++::rumb::g_launches, ::rumb::cuda_check(cudaGetLastError(), what))

void set_last_error(const std::string &msg);

// ---------------------------------------------------------------- device buffers
// An owning device allocation. The library allocates through the context only (cudaMalloc on
// the context's device); buffers are reused across solves of one shape.
struct DevBuf {
    void *ptr = nullptr;
    size_t bytes = 0;
    DevBuf() {}
    DevBuf(const DevBuf &) = delete;
    DevBuf &operator=(const DevBuf &) = delete;
    DevBuf(DevBuf &&o) noexcept : ptr(o.ptr), bytes(o.bytes) {
        o.ptr = nullptr;
        o.bytes = 0;
    }
    DevBuf &operator=(DevBuf &&o) noexcept {
        if (this != &o) {
            release();
            ptr = o.ptr;
            bytes = o.bytes;
            o.ptr = nullptr;
            o.bytes = 0;
        }
        return *this;
    }
    ~DevBuf() { release(); }
    void release() {
        if (ptr) cudaFree(ptr);
        ptr = nullptr;
        bytes = 0;
    }
    void ensure(size_t b) {
        if (b <= bytes && ptr) return;
        release();
        if (b == 0) return;
        RUMB_CUDA(cudaMalloc(&ptr, b));
        bytes = b;
    }
    template <class T> T *as() const { return reinterpret_cast<T *>(ptr); }
};

// ---------------------------------------------------------------- lattice helpers
__host__ __device__ __forceinline__ ull compress_bit(ull mask, int x) {
    return (mask & ((1ULL << x) - 1ULL)) | ((mask >> (x + 1)) << x);
}
__host__ __device__ __forceinline__ ull expand_bit(ull rest, int x) {
    return (rest & ((1ULL << x) - 1ULL)) | ((rest >> x) << (x + 1));
}

// The opt-in for more than 48 KB of dynamic shared memory is an attribute of a kernel on one
// device: set it once per (kernel, device), `done` holding one bit per device already set.
template <class K>
inline void smem_optin(K *kernel, int bytes, std::atomic<unsigned long long> &done) {
    int dev = 0;
    RUMB_CUDA(cudaGetDevice(&dev));
    const unsigned long long bit = 1ULL << (dev & 63);
    if (done.load(std::memory_order_acquire) & bit) return;
    RUMB_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
    done.fetch_or(bit, std::memory_order_release);
}

// Programmatic dependent launch for the iteration's kernels. A kernel launched by launch_pdl may be
// scheduled while the kernel before it on the stream is still finishing (its CTAs take SMs as the
// earlier kernel's last CTAs retire, and the launch latency is hidden); every such kernel calls
// pdl_grid_sync() first, before it touches memory: it lets the kernel after it be scheduled in turn,
// then waits until the kernel before it has completed and its writes are visible. Because every
// kernel so launched waits before it can complete, completion stays ordered down the stream.
// RUMB_PDL=0 launches them in plain stream order.
__device__ __forceinline__ void pdl_grid_sync() {
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    asm volatile("griddepcontrol.wait;" ::: "memory");
}

inline bool pdl_enabled() {
    static const bool on = [] {
        const char *e = getenv("RUMB_PDL");
        return !(e && e[0] == '0');
    }();
    return on;
}

template <class... KArgs, class... Args>
inline void launch_pdl(void (*kern)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t st, Args... args) {
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = pdl_enabled() ? 1 : 0;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    cuda_check(cudaLaunchKernelEx(&cfg, kern, args...), "cudaLaunchKernelEx");
}

inline int num_sms(int dev) {
    int v = 0;
    cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev);
    return v > 0 ? v : 148;
}

// ---------------------------------------------------------------- launch profiler
// When a profiler is installed on the calling thread (rumb_bm_profile), every kernel launch site
// brackets its launch with CUDA events and reports its algorithmic bytes; otherwise these are
// no-ops. Recorded while a stream is captured, the events become nodes of the CUDA graph and time
// the kernels as the graph replays them.
struct ProfRec {
    std::string name;
    cudaEvent_t a, b;
    double bytes;
};
struct Prof {
    cudaStream_t st = nullptr;
    std::vector<ProfRec> recs;
    std::vector<cudaEvent_t> pool;     // events made ahead (a profile captured into a CUDA graph)
    cudaEvent_t event() {
        cudaEvent_t e = nullptr;
        if (!pool.empty()) {
            e = pool.back();
            pool.pop_back();
        } else {
            cudaEventCreate(&e);
        }
        return e;
    }
    ~Prof() {
        for (cudaEvent_t e : pool) cudaEventDestroy(e);
    }
};
extern thread_local Prof *g_prof;

// An event recorded on st; while st is being captured the record becomes a node of the graph
// (cudaEventRecordExternal), so each replay records it.
inline void prof_record(cudaEvent_t e, cudaStream_t st) {
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    cudaStreamIsCapturing(st, &cs);
    if (cs == cudaStreamCaptureStatusActive) cudaEventRecordWithFlags(e, st, cudaEventRecordExternal);
    else cudaEventRecord(e, st);
}
inline void prof_begin(const std::string &name, double bytes, cudaStream_t st) {
    if (!g_prof || st != g_prof->st) return;
    ProfRec r{name, g_prof->event(), g_prof->event(), bytes};
    prof_record(r.a, st);
    g_prof->recs.push_back(r);
}
inline void prof_end(cudaStream_t st) {
    if (!g_prof || st != g_prof->st || g_prof->recs.empty()) return;
    prof_record(g_prof->recs.back().b, st);
}

inline unsigned grid_for(ll n, int block) {
    ll g = (n + block - 1) / block;
    if (g < 1) g = 1;
    return (unsigned)g;
}

}  // namespace rumb
