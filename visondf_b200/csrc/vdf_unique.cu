// vdf_unique.cu -- de-duplication and left-join row matching on the sorted
// path.  Both start from a stable ascending radix sort of the key column, in
// which the rows of one key value form a run in row order: the run's first
// row is the key's first occurrence and its last row the last occurrence.
//   * k_unique_mark  marks those rows in a per-row keep mask (one pass over
//                    the sorted keys, a scatter through the permutation);
//   * k_join_build   puts the right side's distinct sorted keys (the
//                    group-by's segment pass finds them) with the row of each
//                    one's first or last occurrence into a hash table;
//   * k_join_probe   looks each left key up in it.
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

// Marks go into a bit per row (atomicOr on 32-row words: the n/8-byte mask
// stays in L2 while the permutation scatters into it), then one coalesced
// pass expands the bits into the caller's byte mask.
template <typename T>
__global__ void __launch_bounds__(256) k_unique_mark(const T* __restrict__ sk, const uint32_t* __restrict__ perm,
                                                      uint64_t n, int last, uint32_t* __restrict__ bits,
                                                      unsigned long long* count, uint32_t* err) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    uint32_t kept = 0;
    // every lane runs the same number of rounds (the warp sum needs them all)
    for (uint64_t base = (uint64_t)blockIdx.x * blockDim.x; base < n; base += stride) {
        const uint64_t i = base + threadIdx.x;
        if (i < n) {
            const T k = sk[i];
            const bool mark = last ? (i + 1 == n || sk[i + 1] != k) : (i == 0 || sk[i - 1] != k);
            if (mark) {
                const uint32_t r = perm[i];
                if (r >= n) {
                    atomicOr(err, ERR_BAD_INDEX);
                } else {
                    atomicOr(&bits[r >> 5], 1u << (r & 31));
                    ++kept;
                }
            }
        }
    }
    add_count(count, kept);
}

// keep[r] = bit r; one 32-row word per thread, 32 bytes written per thread.
__global__ void __launch_bounds__(256) k_expand_bits(const uint32_t* __restrict__ bits, uint64_t n,
                                                      uint8_t* __restrict__ keep) {
    const uint64_t words = (n + 31) / 32;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    const bool vec = (reinterpret_cast<uintptr_t>(keep) & 15) == 0;
    for (uint64_t w = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; w < words; w += stride) {
        const uint32_t b = bits[w];
        uint32_t q[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            const uint32_t nib = (b >> (4 * k)) & 0xfu;
            q[k] = (nib & 1u) | ((nib & 2u) << 7) | ((nib & 4u) << 14) | ((nib & 8u) << 21);
        }
        const uint64_t r0 = w * 32;
        if (vec && r0 + 32 <= n) {
            uint4* d = reinterpret_cast<uint4*>(keep + r0);
            d[0] = make_uint4(q[0], q[1], q[2], q[3]);
            d[1] = make_uint4(q[4], q[5], q[6], q[7]);
        } else {
            for (uint32_t j = 0; j < 32 && r0 + j < n; ++j) keep[r0 + j] = (uint8_t)((b >> j) & 1u);
        }
    }
}

// Hash table of the right side's distinct keys: 16-byte slots {raw key,
// row + 1 (0 = empty)}, open addressing with linear probing over a
// power-of-two capacity of at least twice the right side's rows.  The keys
// inserted are distinct, so a slot is claimed by a CAS of its row field and
// its key written after; the probe kernel runs after the build completes.
struct JoinSlot {
    unsigned long long key;
    uint32_t row1;
    uint32_t pad;
};

__device__ __forceinline__ uint64_t mix64(uint64_t x) {
    // 64-bit finaliser of MurmurHash3 (fmix64)
    x ^= x >> 33;
    x *= 0xff51afd7ed558ccdull;
    x ^= x >> 33;
    x *= 0xc4ceb9fe1a85ec53ull;
    x ^= x >> 33;
    return x;
}

// method 0 / 1: the slot holds the row of the key's first / last occurrence;
// method 2 (aligned): it holds the key's run index g.
template <typename T>
__global__ void __launch_bounds__(256) k_join_build(const T* __restrict__ ukeys, const uint32_t* __restrict__ gstart,
                                                     const uint64_t* n_groups, const uint32_t* __restrict__ perm_r,
                                                     uint64_t n_right, int method, JoinSlot* table, uint64_t mask,
                                                     uint32_t* err) {
    const uint64_t G = *n_groups;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t g = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; g < G; g += stride) {
        const uint64_t pos = method == 1 ? (g + 1 < G ? (uint64_t)gstart[g + 1] - 1 : n_right - 1) : gstart[g];
        if (pos >= n_right) {
            atomicOr(err, ERR_BAD_INDEX);
            continue;
        }
        const uint32_t row1 = (method == 2 ? (uint32_t)g : perm_r[pos]) + 1u;
        const unsigned long long key = (unsigned long long)ukeys[g];
        uint64_t s = mix64(key) & mask;
        bool placed = false;
        for (uint64_t t = 0; t <= mask; ++t) {  // at most one lap of the table
            if (atomicCAS(&table[s].row1, 0u, row1) == 0u) {
                table[s].key = key;
                placed = true;
                break;
            }
            s = (s + 1) & mask;
        }
        if (!placed) atomicOr(err, ERR_BAD_INDEX);
    }
}

template <typename T>
__global__ void __launch_bounds__(256) k_join_probe(const T* __restrict__ left, uint64_t n_left,
                                                     const JoinSlot* __restrict__ table, uint64_t mask,
                                                     uint32_t* __restrict__ match, unsigned long long* matched) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    uint32_t found = 0;
    for (uint64_t base = (uint64_t)blockIdx.x * blockDim.x; base < n_left; base += stride) {
        const uint64_t i = base + threadIdx.x;
        if (i >= n_left) continue;
        const unsigned long long x = (unsigned long long)left[i];
        uint64_t s = mix64(x) & mask;
        uint32_t m = 0xffffffffu;
        for (uint64_t t = 0; t <= mask; ++t) {  // an empty slot ends every chain (load <= 1/2)
            const ulonglong2 v = ld_rand16(reinterpret_cast<const ulonglong2*>(table + s));
            const uint32_t row1 = (uint32_t)v.y;
            if (row1 == 0u) break;
            if (v.x == x) {
                m = row1 - 1u;
                ++found;
                break;
            }
            s = (s + 1) & mask;
        }
        match[i] = m;
    }
    add_count(matched, found);
}

// Aligned matching over the left side's stable sort: sorted left row i is
// occurrence r = i - (start of its run) of its key; it takes the right row
// at position r of that key's run in the right side's sort, if the run is
// long enough.  Results are scattered back through the left permutation.
template <typename T>
__global__ void __launch_bounds__(256) k_join_probe_aligned(
    const T* __restrict__ sorted_l, const uint32_t* __restrict__ perm_l, const uint32_t* __restrict__ group_l,
    const uint32_t* __restrict__ gstart_l, uint64_t n_left, const JoinSlot* __restrict__ table, uint64_t mask,
    const uint32_t* __restrict__ gstart_r, const uint64_t* n_groups_r, const uint32_t* __restrict__ perm_r,
    uint64_t n_right, uint32_t* __restrict__ match, unsigned long long* matched, uint32_t* err) {
    const uint64_t Gr = *n_groups_r;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    uint32_t found = 0;
    for (uint64_t base = (uint64_t)blockIdx.x * blockDim.x; base < n_left; base += stride) {
        const uint64_t i = base + threadIdx.x;
        if (i >= n_left) continue;
        const unsigned long long x = (unsigned long long)sorted_l[i];
        const uint32_t rank = (uint32_t)i - gstart_l[group_l[i]];
        uint64_t s = mix64(x) & mask;
        uint32_t m = 0xffffffffu;
        for (uint64_t t = 0; t <= mask; ++t) {
            const ulonglong2 v = ld_rand16(reinterpret_cast<const ulonglong2*>(table + s));
            const uint32_t g1 = (uint32_t)v.y;
            if (g1 == 0u) break;
            if (v.x == x) {
                const uint64_t g = g1 - 1u;
                const uint64_t start = g < Gr ? gstart_r[g] : n_right;
                const uint64_t end = g + 1 < Gr ? gstart_r[g + 1] : n_right;
                if (start + rank < end) {
                    m = perm_r[start + rank];
                    ++found;
                }
                break;
            }
            s = (s + 1) & mask;
        }
        const uint32_t r = perm_l[i];
        if (r >= n_left) atomicOr(err, ERR_BAD_INDEX);
        else match[r] = m;
    }
    add_count(matched, found);
}

}  // namespace

size_t unique_workspace_bytes(uint64_t n) { return ((n + 31) / 32) * 4; }

cudaError_t run_unique_mark(const void* sorted_keys, int width, const uint32_t* perm, uint64_t n, int last,
                            uint8_t* keep, unsigned long long* count, uint32_t* bits, uint32_t* err,
                            cudaStream_t s) {
    if (n == 0) return cudaSuccess;
    cudaError_t e = cudaMemsetAsync(bits, 0, unique_workspace_bytes(n), s);
    if (e != cudaSuccess) return e;
    const uint32_t grid = grid_size(n);
    if (width == 8)
        k_unique_mark<unsigned long long><<<grid, 256, 0, s>>>(
            static_cast<const unsigned long long*>(sorted_keys), perm, n, last, bits, count, err);
    else
        k_unique_mark<uint32_t><<<grid, 256, 0, s>>>(static_cast<const uint32_t*>(sorted_keys), perm, n, last, bits,
                                                     count, err);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    k_expand_bits<<<grid_size((n + 31) / 32), 256, 0, s>>>(bits, n, keep);
    return cudaGetLastError();
}

uint64_t join_table_slots(uint64_t n_right) {
    uint64_t cap = 1024;
    while (cap < 2 * n_right) cap <<= 1;
    return cap;
}
size_t join_workspace_bytes(uint64_t n_right) { return join_table_slots(n_right) * sizeof(JoinSlot); }

cudaError_t run_join_build(const void* ukeys, int width, const uint32_t* gstart, const uint64_t* n_groups,
                           const uint32_t* perm_right, uint64_t n_right, int method, void* table_ws, uint32_t* err,
                           cudaStream_t s) {
    const uint64_t slots = join_table_slots(n_right);
    JoinSlot* table = static_cast<JoinSlot*>(table_ws);
    cudaError_t e = cudaMemsetAsync(table, 0, slots * sizeof(JoinSlot), s);
    if (e != cudaSuccess || n_right == 0) return e;
    if (width == 8)
        k_join_build<unsigned long long><<<grid_size(n_right), 256, 0, s>>>(
            static_cast<const unsigned long long*>(ukeys), gstart, n_groups, perm_right, n_right, method, table,
            slots - 1, err);
    else
        k_join_build<uint32_t><<<grid_size(n_right), 256, 0, s>>>(static_cast<const uint32_t*>(ukeys), gstart,
                                                                   n_groups, perm_right, n_right, method, table,
                                                                   slots - 1, err);
    return cudaGetLastError();
}

cudaError_t run_join_probe(const void* left, uint64_t n_left, int width, const void* table_ws, uint64_t n_right,
                           uint32_t* match, unsigned long long* matched, cudaStream_t s) {
    if (n_left == 0) return cudaSuccess;
    const uint64_t mask = join_table_slots(n_right) - 1;
    const JoinSlot* table = static_cast<const JoinSlot*>(table_ws);
    const uint32_t grid = grid_size(n_left);
    if (width == 8)
        k_join_probe<unsigned long long><<<grid, 256, 0, s>>>(static_cast<const unsigned long long*>(left), n_left,
                                                              table, mask, match, matched);
    else
        k_join_probe<uint32_t><<<grid, 256, 0, s>>>(static_cast<const uint32_t*>(left), n_left, table, mask, match,
                                                    matched);
    return cudaGetLastError();
}

cudaError_t run_join_probe_aligned(const void* sorted_left, int width, const uint32_t* perm_left,
                                   const uint32_t* group_left, const uint32_t* gstart_left, uint64_t n_left,
                                   const void* table_ws, const uint32_t* gstart_right, const uint64_t* n_groups_right,
                                   const uint32_t* perm_right, uint64_t n_right, uint32_t* match,
                                   unsigned long long* matched, uint32_t* err, cudaStream_t s) {
    if (n_left == 0) return cudaSuccess;
    const uint64_t mask = join_table_slots(n_right) - 1;
    const JoinSlot* table = static_cast<const JoinSlot*>(table_ws);
    const uint32_t grid = grid_size(n_left);
    if (width == 8)
        k_join_probe_aligned<unsigned long long><<<grid, 256, 0, s>>>(
            static_cast<const unsigned long long*>(sorted_left), perm_left, group_left, gstart_left, n_left, table,
            mask, gstart_right, n_groups_right, perm_right, n_right, match, matched, err);
    else
        k_join_probe_aligned<uint32_t><<<grid, 256, 0, s>>>(
            static_cast<const uint32_t*>(sorted_left), perm_left, group_left, gstart_left, n_left, table, mask,
            gstart_right, n_groups_right, perm_right, n_right, match, matched, err);
    return cudaGetLastError();
}

}  // namespace vdf
