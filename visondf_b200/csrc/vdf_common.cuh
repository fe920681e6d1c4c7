// vdf_common.cuh -- device helpers shared by the sort, gather and group-by
// kernels: column dtypes, order-preserving key images, acquire/release
// accesses for the decoupled look-back, and bounded waits.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace vdf {

// Column dtypes.  Codes match vdf_dtype in include/vdf_capi.h.
enum Dtype : int { I32 = 0, I64 = 1, U32 = 2, U64 = 3, F64 = 4, F32 = 5 };

__host__ __device__ inline int dtype_width(int dt) {
    return (dt == I32 || dt == U32 || dt == F32) ? 4 : (dt == I64 || dt == U64 || dt == F64) ? 8 : 0;
}

// Order-preserving unsigned image of a raw key (sort_integers.inl:46 flips the
// sign bit of signed integers; sort_uintegers copies; sort_flt.inl:123-129
// maps IEEE doubles with bits ^ (mask(sign) | signbit)).  `invert` gives the
// stable descending order (all bits flipped).
__device__ __forceinline__ uint32_t order32(uint32_t raw, int dt, bool invert) {
    uint32_t k;
    if (dt == I32) k = raw ^ 0x80000000u;
    else if (dt == F32) k = raw ^ ((0u - (raw >> 31)) | 0x80000000u);
    else k = raw;
    return invert ? ~k : k;
}
__device__ __forceinline__ uint64_t order64(uint64_t raw, int dt, bool invert) {
    uint64_t k;
    if (dt == I64) k = raw ^ 0x8000000000000000ull;
    else if (dt == F64) k = raw ^ ((0ull - (raw >> 63)) | 0x8000000000000000ull);
    else k = raw;
    return invert ? ~k : k;
}
// Inverses of the above (used when the last radix pass writes raw sorted keys).
__device__ __forceinline__ uint32_t unorder32(uint32_t k, int dt, bool invert) {
    if (invert) k = ~k;
    if (dt == I32) return k ^ 0x80000000u;
    if (dt == F32) return (k & 0x80000000u) ? (k ^ 0x80000000u) : ~k;
    return k;
}
__device__ __forceinline__ uint64_t unorder64(uint64_t k, int dt, bool invert) {
    if (invert) k = ~k;
    if (dt == I64) return k ^ 0x8000000000000000ull;
    if (dt == F64) return (k & 0x8000000000000000ull) ? (k ^ 0x8000000000000000ull) : ~k;
    return k;
}

template <typename K> struct KeyOps;
template <> struct KeyOps<uint32_t> {
    static __device__ __forceinline__ uint32_t order(uint32_t r, int dt, bool inv) { return order32(r, dt, inv); }
    static __device__ __forceinline__ uint32_t unorder(uint32_t k, int dt, bool inv) { return unorder32(k, dt, inv); }
};
template <> struct KeyOps<uint64_t> {
    static __device__ __forceinline__ uint64_t order(uint64_t r, int dt, bool inv) { return order64(r, dt, inv); }
    static __device__ __forceinline__ uint64_t unorder(uint64_t k, int dt, bool inv) { return unorder64(k, dt, inv); }
};

// ---- memory-model helpers for the decoupled look-back ---------------------
__device__ __forceinline__ uint32_t ld_acquire_u32(const uint32_t* p) {
    uint32_t v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release_u32(uint32_t* p, uint32_t v) {
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ uint32_t ld_relaxed_u32(const uint32_t* p) {
    uint32_t v;
    asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_relaxed_u32(uint32_t* p, uint32_t v) {
    asm volatile("st.relaxed.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ uint64_t ld_relaxed_u64(const uint64_t* p) {
    uint64_t v;
    asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_relaxed_u64(uint64_t* p, uint64_t v) {
    asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

// Streaming (evict-first) loads/stores for data touched exactly once.
template <typename T> __device__ __forceinline__ T ldg_stream(const T* p) { return __ldcs(p); }
template <typename T> __device__ __forceinline__ void stg_stream(T* p, T v) { __stcs(p, v); }

// Random reads of read-only data (gathers through a permutation): the
// non-coherent path with the L2 fetch limited to 64 bytes.  Measured on B200
// for 100M random 32-byte records: one 32-byte load of this form took 2.15 ms
// and read 75 B of DRAM per record, against 4.1 ms and 137 B for two 16-byte
// L2-only loads (the second half of a record then costs a second L2 request,
// and a miss fetches 128 bytes by default).
__device__ __forceinline__ void ld_rand32(const void* p, unsigned long long (&v)[4]) {  // 32-byte aligned
    asm("ld.global.nc.L2::64B.v4.u64 {%0,%1,%2,%3}, [%4];"
        : "=l"(v[0]), "=l"(v[1]), "=l"(v[2]), "=l"(v[3])
        : "l"(p));
}
__device__ __forceinline__ ulonglong2 ld_rand16(const void* p) {  // 16-byte aligned
    ulonglong2 v;
    asm("ld.global.nc.L2::64B.v2.u64 {%0,%1}, [%2];" : "=l"(v.x), "=l"(v.y) : "l"(p));
    return v;
}
__device__ __forceinline__ unsigned long long ld_rand8(const void* p) {
    unsigned long long v;
    asm("ld.global.nc.L2::64B.u64 %0, [%1];" : "=l"(v) : "l"(p));
    return v;
}
__device__ __forceinline__ uint32_t ld_rand4(const void* p) {
    uint32_t v;
    asm("ld.global.nc.L2::64B.u32 %0, [%1];" : "=r"(v) : "l"(p));
    return v;
}

// Bounded waits: every spin in these kernels gives up after this many polls
// (each poll sleeps 32-128 ns, so about 0.1 s), records an error bit in the
// context's error word and carries on, so a broken dependency ends the kernel
// with an error status instead of hanging the GPU.  Legitimate waits on an
// earlier tile last microseconds.
constexpr uint32_t kSpinLimit = 1u << 20;
enum ErrBits : uint32_t { ERR_LOOKBACK_TIMEOUT = 1u, ERR_BAD_INDEX = 2u };

__device__ __forceinline__ void backoff(uint32_t it) {
    __nanosleep(it < 16 ? 32 : 128);
}

__device__ __forceinline__ uint32_t lanemask_lt() {
    uint32_t m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

// ---- bulk copies from this GPU's global memory into shared memory, behind
//      an mbarrier (1-D cp.async.bulk, no cluster sharing).  Both addresses
//      16-byte aligned and the size a multiple of 16 bytes.
__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t arrivals) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(arrivals) : "memory");
}
// makes initialised barriers visible to the copy engine
__device__ __forceinline__ void mbar_init_fence() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
// orders this thread's earlier shared-memory accesses before later bulk copies into it
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
// one arrival that also expects `bytes` of copies to complete this phase
__device__ __forceinline__ void mbar_expect(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void bulk_load(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                 ::"r"(smem_u32(dst)), "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}
__device__ __forceinline__ bool mbar_test(uint64_t* bar, uint32_t parity) {
    uint32_t done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
        : "=r"(done)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return done != 0;
}
// Waits for phase `parity` of the barrier to complete, at most `limit` polls
// (each try_wait suspends the thread for a while); false when it ran out.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, uint32_t limit) {
    for (uint32_t i = 0; i < limit; ++i)
        if (mbar_test(bar, parity)) return true;
    return false;
}

}  // namespace vdf
