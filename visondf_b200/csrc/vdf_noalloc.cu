// vdf_noalloc.cu -- a radix argsort entry point that allocates nothing.
//
// Every other entry point of this library works out of a context workspace
// that grows with cudaMalloc (or out of a buffer the caller allocated).  Some
// callers cannot allocate at the moment they need a sort: code running inside
// another allocator's callback or a memory-pool hook, code whose device
// memory is carved up ahead of time by a host framework that forbids new
// allocations at run time, and latency-critical code that cannot afford the
// device-wide synchronisation cudaMalloc/cudaFree may imply.  For them,
// vdf_sort_argsort_noalloc keeps its scratch in one file-scope device array
// of fixed size; the caller still provides the key columns and the outputs.
//
// The scratch array's name is only a host-side handle in host code, so its
// device address is looked up once per device with cudaGetSymbolAddress (the
// lookup happens on the first call on a device, with that device current).
#include <cstring>
#include <mutex>

#include "vdf_capi.h"
#include "vdf_common.cuh"
#include "vdf_internal.h"

namespace {

// 24 bytes per row of radix buffers (8-byte keys and u32 row ids, both
// double-buffered) for VDF_NOALLOC_MAX_ROWS rows, plus the per-digit tables,
// the look-back status words and the error word.
constexpr size_t kScratchBytes = 28ull << 20;
constexpr size_t kErrBytes = 256;  // error word at the start, workspace after it

static __device__ __align__(256) unsigned char g_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
unsigned char* g_scratch_addr[kMaxDevices];

// Device address of g_scratch on `dev` (the current device), looked up once.
vdf_status scratch_on(int dev, unsigned char** out) {
    if (dev < 0 || dev >= kMaxDevices) return VDF_ERR_UNSUPPORTED;
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_scratch_addr[dev]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_scratch);
        if (e != cudaSuccess || !p) {
            cudaGetLastError();
            return VDF_ERR_DEVICE;
        }
        if (vdf::prepare_sort_kernels() != cudaSuccess) {
            cudaGetLastError();
            return VDF_ERR_DEVICE;
        }
        g_scratch_addr[dev] = static_cast<unsigned char*>(p);
    }
    *out = g_scratch_addr[dev];
    return VDF_OK;
}

}  // namespace

extern "C" vdf_status vdf_sort_argsort_noalloc(uint64_t n, const vdf_col* keys, int nkeys, int order,
                                               uint32_t* perm_out, void* const* sorted_keys_out, void* stream) {
    if (n > VDF_NOALLOC_MAX_ROWS) return VDF_ERR_UNSUPPORTED;
    if (!keys || nkeys < 1 || nkeys > vdf::kMaxKeys) return VDF_ERR_INVALID_ARG;
    if (order < VDF_ORDER_ASC || order > VDF_ORDER_DESC_REVERSE) return VDF_ERR_INVALID_ARG;
    int32_t dts[vdf::kMaxKeys];
    const void* cols[vdf::kMaxKeys];
    for (int k = 0; k < nkeys; ++k) {
        if (keys[k].dtype < VDF_I32 || keys[k].dtype > VDF_F32) return VDF_ERR_INVALID_ARG;
        if (n && !keys[k].data) return VDF_ERR_INVALID_ARG;
        dts[k] = keys[k].dtype;
        cols[k] = keys[k].data;
    }
    if (n == 0) return VDF_OK;
    if (!perm_out) return VDF_ERR_INVALID_ARG;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) {
        cudaGetLastError();
        return VDF_ERR_DEVICE;
    }
    unsigned char* base = nullptr;
    vdf_status st = scratch_on(dev, &base);
    if (st != VDF_OK) return st;
    const vdf::SortPlan plan = vdf::make_sort_plan(n, dts, nkeys, vdf::default_sort_tuning());
    if (plan.ws_bytes > kScratchBytes - kErrBytes) return VDF_ERR_UNSUPPORTED;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    uint32_t* err = reinterpret_cast<uint32_t*>(base);
    // The array keeps the previous call's contents: the error word is cleared
    // here and run_sort clears its histograms, tile counters, look-back status
    // and plan flag itself.
    cudaError_t e = cudaMemsetAsync(err, 0, sizeof(uint32_t), s);
    if (e == cudaSuccess) {
        void* key0 = sorted_keys_out ? sorted_keys_out[0] : nullptr;
        e = vdf::run_sort(plan, cols, order, perm_out, key0, base + kErrBytes, err, s);
    }
    if (e == cudaSuccess && sorted_keys_out) {
        vdf::GatherArgs g{};
        g.perm = perm_out;
        g.err = err;
        g.n = n;
        for (int k = 1; k < nkeys; ++k) {
            if (!sorted_keys_out[k]) continue;
            g.src[g.ncols] = cols[k];
            g.dst[g.ncols] = sorted_keys_out[k];
            g.width[g.ncols] = vdf::dtype_width(dts[k]);
            g.ncols++;
        }
        e = vdf::run_gather(g, s);  // column by column: no record buffer
    }
    if (e != cudaSuccess) {
        cudaGetLastError();
        return e == cudaErrorMemoryAllocation ? VDF_ERR_OOM : VDF_ERR_DEVICE;
    }
    return VDF_OK;
}

// The error word of the last call on the current device: bounded waits that
// gave up and out-of-range row ids set bits in it (the same bits
// vdf_ctx_check reports for a context).  A 4-byte device-to-host copy into
// the caller's memory, then a wait for `stream`; nothing is allocated.
extern "C" vdf_status vdf_sort_noalloc_error(uint32_t* host_out, void* stream) {
    if (!host_out) return VDF_ERR_INVALID_ARG;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) {
        cudaGetLastError();
        return VDF_ERR_DEVICE;
    }
    unsigned char* base = nullptr;
    vdf_status st = scratch_on(dev, &base);
    if (st != VDF_OK) return st;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    cudaError_t e = cudaMemcpyAsync(host_out, base, sizeof(uint32_t), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return VDF_ERR_DEVICE;
    }
    return VDF_OK;
}
