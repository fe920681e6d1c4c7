// vdf_unique.cu -- de-duplication and left-join row matching on the sorted
// path.  Both start from a stable ascending radix sort of the key column, in
// which the rows of one key value form a run in row order: the run's first
// row is the key's first occurrence and its last row the last occurrence.
//   * k_unique_mark  marks those rows in a per-row keep mask (one pass over
//                    the sorted keys, a scatter through the permutation);
//   * k_join_probe   looks each left key up among the right side's distinct
//                    sorted keys (binary search over the run starts the
//                    group-by's segment pass produced).
// Keys compare by their raw bits, so -0.0 and +0.0 are different keys and a
// NaN equals a NaN with the same bits, as with the reference's byte-wise
// hash lookups.
#include <cstdint>

#include "vdf_common.cuh"
#include "vdf_internal.h"

namespace vdf {
namespace {

uint32_t grid_size(uint64_t n) {
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const uint64_t want = (n + 255) / 256;
    const uint64_t cap = (uint64_t)sms * 8;
    return (uint32_t)(want < cap ? (want ? want : 1) : cap);
}

// Warp sum of a per-thread count, added once per warp.
__device__ __forceinline__ void add_count(unsigned long long* total, uint32_t mine) {
    const uint32_t w = __reduce_add_sync(0xffffffffu, mine);
    if ((threadIdx.x & 31) == 0 && w) atomicAdd(total, (unsigned long long)w);
}

template <typename T>
__global__ void __launch_bounds__(256) k_unique_mark(const T* __restrict__ sk, const uint32_t* __restrict__ perm,
                                                      uint64_t n, int last, uint8_t* __restrict__ keep,
                                                      unsigned long long* count, uint32_t* err) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    uint32_t kept = 0;
    // every lane runs the same number of rounds (the warp sum needs them all)
    for (uint64_t base = (uint64_t)blockIdx.x * blockDim.x; base < n; base += stride) {
        const uint64_t i = base + threadIdx.x;
        if (i < n) {
            const T k = sk[i];
            const bool mark = last ? (i + 1 == n || sk[i + 1] != k) : (i == 0 || sk[i - 1] != k);
            const uint32_t r = perm[i];
            if (r >= n) {
                atomicOr(err, ERR_BAD_INDEX);
            } else {
                keep[r] = mark ? 1 : 0;
                kept += mark ? 1u : 0u;
            }
        }
    }
    add_count(count, kept);
}

template <typename T>
__device__ __forceinline__ T order_of(T raw, int dt) {
    if constexpr (sizeof(T) == 8) return (T)order64((uint64_t)raw, dt, false);
    else return (T)order32((uint32_t)raw, dt, false);
}

template <typename T>
__global__ void __launch_bounds__(256) k_join_probe(const T* __restrict__ left, uint64_t n_left, int dt,
                                                     const T* __restrict__ ukeys, const uint32_t* __restrict__ gstart,
                                                     const uint64_t* n_groups, const uint32_t* __restrict__ perm_r,
                                                     uint64_t n_right, int last, uint32_t* __restrict__ match,
                                                     unsigned long long* matched, uint32_t* err) {
    const uint64_t G = *n_groups;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    uint32_t found = 0;
    for (uint64_t base = (uint64_t)blockIdx.x * blockDim.x; base < n_left; base += stride) {
        const uint64_t i = base + threadIdx.x;
        if (i >= n_left) continue;
        const T raw = left[i];
        const T x = order_of(raw, dt);
        uint64_t lo = 0, hi = G;  // first distinct key whose image is >= x
        while (lo < hi) {
            const uint64_t mid = (lo + hi) >> 1;
            if (order_of(ukeys[mid], dt) < x) lo = mid + 1;
            else hi = mid;
        }
        uint32_t m = 0xffffffffu;
        if (lo < G && ukeys[lo] == raw) {
            const uint64_t pos = last ? (lo + 1 < G ? (uint64_t)gstart[lo + 1] - 1 : n_right - 1) : gstart[lo];
            if (pos >= n_right) {
                atomicOr(err, ERR_BAD_INDEX);
            } else {
                m = perm_r[pos];
                ++found;
            }
        }
        match[i] = m;
    }
    add_count(matched, found);
}

}  // namespace

cudaError_t run_unique_mark(const void* sorted_keys, int width, const uint32_t* perm, uint64_t n, int last,
                            uint8_t* keep, unsigned long long* count, uint32_t* err, cudaStream_t s) {
    if (n == 0) return cudaSuccess;
    const uint32_t grid = grid_size(n);
    if (width == 8)
        k_unique_mark<unsigned long long><<<grid, 256, 0, s>>>(
            static_cast<const unsigned long long*>(sorted_keys), perm, n, last, keep, count, err);
    else
        k_unique_mark<uint32_t><<<grid, 256, 0, s>>>(static_cast<const uint32_t*>(sorted_keys), perm, n, last, keep,
                                                     count, err);
    return cudaGetLastError();
}

cudaError_t run_join_probe(const void* left, uint64_t n_left, int dtype, const void* ukeys, const uint32_t* gstart,
                           const uint64_t* n_groups, const uint32_t* perm_right, uint64_t n_right, int last,
                           uint32_t* match, unsigned long long* matched, uint32_t* err, cudaStream_t s) {
    if (n_left == 0) return cudaSuccess;
    const uint32_t grid = grid_size(n_left);
    if (dtype_width(dtype) == 8)
        k_join_probe<unsigned long long><<<grid, 256, 0, s>>>(
            static_cast<const unsigned long long*>(left), n_left, dtype,
            static_cast<const unsigned long long*>(ukeys), gstart, n_groups, perm_right, n_right, last, match, matched,
            err);
    else
        k_join_probe<uint32_t><<<grid, 256, 0, s>>>(static_cast<const uint32_t*>(left), n_left, dtype,
                                                     static_cast<const uint32_t*>(ukeys), gstart, n_groups, perm_right,
                                                     n_right, last, match, matched, err);
    return cudaGetLastError();
}

}  // namespace vdf
