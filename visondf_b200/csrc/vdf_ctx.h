// vdf_ctx.h -- the library context behind the opaque vdf_ctx handle and the
// small helpers every entry point uses (error reporting, device guard,
// grow-only workspace, device error word).  Internal to the library.
#pragma once
#include <algorithm>
#include <atomic>
#include <cstdarg>
#include <cstdio>
#include <mutex>
#include <string>
#include <vector>

#include "vdf_capi.h"
#include "vdf_common.cuh"
#include "vdf_internal.h"

// Per-launch CUDA-event timing, enabled by vdf_ctx_profile().  Events come
// from a pool and are resolved (synchronised) only when read.
struct EventProfiler final : vdf::Profiler {
    std::vector<cudaEvent_t> pool;
    size_t used = 0;
    struct Pending { int cls; size_t b, e; };
    std::vector<Pending> pending;
    double total_ms[vdf::KC_COUNT] = {};
    uint64_t count[vdf::KC_COUNT] = {};
    int open_cls = -1;
    size_t open_b = 0;

    cudaEvent_t next() {
        if (used == pool.size()) {
            cudaEvent_t ev;
            if (cudaEventCreate(&ev) != cudaSuccess) return nullptr;
            pool.push_back(ev);
        }
        return pool[used++];
    }
    void begin(int cls, cudaStream_t s) override {
        cudaEvent_t ev = next();
        if (!ev) return;
        cudaEventRecord(ev, s);
        open_cls = cls;
        open_b = used - 1;
    }
    void end(int cls, cudaStream_t s) override {
        if (open_cls != cls) return;
        cudaEvent_t ev = next();
        if (!ev) return;
        cudaEventRecord(ev, s);
        pending.push_back({cls, open_b, used - 1});
        open_cls = -1;
    }
    cudaError_t resolve() {
        for (const Pending& p : pending) {
            cudaError_t e = cudaEventSynchronize(pool[p.e]);
            if (e != cudaSuccess) return e;
            float ms = 0;
            cudaEventElapsedTime(&ms, pool[p.b], pool[p.e]);
            total_ms[p.cls] += ms;
            count[p.cls]++;
        }
        pending.clear();
        used = 0;
        return cudaSuccess;
    }
    ~EventProfiler() override {
        for (cudaEvent_t ev : pool) cudaEventDestroy(ev);
    }
};

struct vdf_ctx {
    int device = 0;
    bool profiling = false;
    unsigned char* io = nullptr;  // staging for the host-memory entry points
    size_t io_cap = 0;
    vdf::SortTuning tuning = vdf::default_sort_tuning();
    EventProfiler prof;
    std::mutex mu;
    unsigned char* ws = nullptr;
    size_t ws_cap = 0;
    unsigned char* dev_small = nullptr;  // [0,4): error bits; [8,16): group count scratch;
                                         // [16,20): tie flag; [24,28): MSD fallbacks;
                                         // [28,32): dictionary passes taken
    uint64_t* host_pinned = nullptr;     // [0]: group count, [1]: error bits, [2]: tie flag, [3]: fallbacks,
                                         // [4]: pivot key counts (two words), [5]: dictionary passes
                                         // taken, [6..7] spare
    uint64_t msd_sorts = 0;              // sorts planned MSD-first
    uint64_t dict_sorts = 0;             // sorts that tried the dictionary plan
    uint32_t emit_min_heads = 0;         // group-by emit: striped-path threshold (0 = default)
    uint32_t fail_allocs = 0;            // test hook: workspace allocations to fail
    int multikey_mode = VDF_MULTIKEY_PRIMARY_FIRST;
    std::atomic<uint64_t> launches{0};
    std::string last_error;
};

namespace vdfc {


constexpr uint64_t kMaxRows = (1ull << 30) - 1;

inline vdf_status fail(vdf_ctx* c, vdf_status s, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    if (c) c->last_error = buf;
    return s;
}

inline vdf_status from_cuda(vdf_ctx* c, cudaError_t e, const char* what) {
    if (e == cudaSuccess) return VDF_OK;
    vdf_status s = (e == cudaErrorMemoryAllocation) ? VDF_ERR_OOM : VDF_ERR_DEVICE;
    return fail(c, s, "%s: %s", what, cudaGetErrorString(e));
}

struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int d) {
        if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
        if (prev != d) cudaSetDevice(d);
    }
    ~DeviceGuard() {
        int cur = -1;
        if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
    }
};

inline bool valid_dtype(int32_t dt) { return dt >= VDF_I32 && dt <= VDF_F32; }

inline size_t align256(size_t x) { return (x + 255) / 256 * 256; }

inline vdf::Profiler* prof_of(vdf_ctx* c) { return c->profiling ? &c->prof : nullptr; }

inline uint32_t* err_word(vdf_ctx* c) { return reinterpret_cast<uint32_t*>(c->dev_small); }
inline uint64_t* count_word(vdf_ctx* c) { return reinterpret_cast<uint64_t*>(c->dev_small + 8); }
inline uint32_t* tie_word(vdf_ctx* c) { return reinterpret_cast<uint32_t*>(c->dev_small + 16); }
inline uint32_t* fallback_word(vdf_ctx* c) { return reinterpret_cast<uint32_t*>(c->dev_small + 24); }
inline uint32_t* dict_word(vdf_ctx* c) { return reinterpret_cast<uint32_t*>(c->dev_small + 28); }

// run_sort with the context's error word, profiler and MSD bookkeeping.
inline cudaError_t ctx_run_sort(vdf_ctx* c, const vdf::SortPlan& p, const void* const* cols, int order,
                                uint32_t* perm_out, void* key0_out, unsigned char* ws, cudaStream_t s,
                                const uint32_t* perm_in = nullptr) {
    if (p.msd && p.n) c->msd_sorts++;
    if (p.dict && p.n) c->dict_sorts++;
    c->launches += (uint64_t)vdf::sort_launches(p);
    return vdf::run_sort(p, cols, order, perm_out, key0_out, ws, err_word(c), s, prof_of(c), perm_in,
                         fallback_word(c), dict_word(c));
}

inline vdf_status ws_ensure(vdf_ctx* c, size_t bytes) {
    if (bytes <= c->ws_cap) return VDF_OK;
    if (c->ws) {
        cudaError_t e = cudaFree(c->ws);  // waits for work still using the old buffer
        c->ws = nullptr;
        c->ws_cap = 0;
        if (e != cudaSuccess) return from_cuda(c, e, "cudaFree(workspace)");
    }
    size_t cap = align256(bytes + bytes / 8);
    if (c->fail_allocs) {  // failure injection (vdf_ctx_set_test_hooks)
        c->fail_allocs--;
        return fail(c, VDF_ERR_OOM, "workspace allocation of %zu bytes failed (injected by a test hook)", cap);
    }
    cudaError_t e = cudaMalloc(&c->ws, cap);
    if (e != cudaSuccess) {
        c->ws = nullptr;
        cudaGetLastError();
        return fail(c, VDF_ERR_OOM, "workspace allocation of %zu bytes failed: %s", cap, cudaGetErrorString(e));
    }
    c->ws_cap = cap;
    return VDF_OK;
}

// Grow-only device staging for the host-memory entry points.
inline vdf_status io_ensure(vdf_ctx* c, size_t bytes) {
    if (bytes <= c->io_cap) return VDF_OK;
    if (c->io) {
        cudaFree(c->io);
        c->io = nullptr;
        c->io_cap = 0;
    }
    const size_t cap = align256(bytes + bytes / 8);
    if (cudaMalloc(&c->io, cap) != cudaSuccess) {
        cudaGetLastError();
        return fail(c, VDF_ERR_OOM, "I/O staging allocation of %zu bytes failed", cap);
    }
    c->io_cap = cap;
    return VDF_OK;
}

// vdf_sort_groupby on device pointers with the context lock already held.
vdf_status sort_groupby_device(vdf_ctx* c, const vdf_sort_groupby_args* x, cudaStream_t s);

// Reads and clears the device error bits after the stream has drained.
inline vdf_status drain_and_check(vdf_ctx* c, cudaStream_t s) {
    cudaError_t e = cudaMemcpyAsync(&c->host_pinned[1], err_word(c), sizeof(uint32_t), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return from_cuda(c, e, "stream synchronize");
    uint32_t bits = (uint32_t)c->host_pinned[1];
    if (bits) {
        cudaMemsetAsync(err_word(c), 0, sizeof(uint32_t), s);
        cudaStreamSynchronize(s);
        return fail(c, VDF_ERR_TIMEOUT, "device error bits 0x%x (look-back wait gave up or bad index)", bits);
    }
    return VDF_OK;
}

}  // namespace vdfc
