// vdf_dict.cu -- the dictionary plan of a one-key sort: a key column that
// takes at most kDictMax distinct values is sorted by ONE stable radix pass
// whose digit is each key's rank among those values, instead of one pass per
// byte of the key.
//
// The reference sorts such columns like any other (radix_sort_uint64_mt.inl:
// 6-166, every 16-bit digit); low-cardinality keys (categories, flags, small
// enums: the 16-key group-by of the benchmark configs) are where its passes
// are most wasted.  Here:
//   1. k_dict_collect  every CTA inserts its rows' order images into a
//                      shared-memory table (warp-aggregated counts), stops as
//                      soon as it has seen more than kDictMax distinct
//                      values (setting the overflow word, which the other
//                      CTAs poll), and otherwise merges its table into the
//                      global one;
//   2. k_dict_rank     one CTA ranks the distinct values (count of smaller
//                      ones), scans their counts into the pass's bin starts,
//                      fills the lookup table and sets the plan word to 2;
//                      with an overflow it sets the word to the plan that
//                      runs instead (MSD-first or LSD);
//   3. the dictionary pass (k_onesweep with DICT, vdf_radix.cu) runs only
//      when the word is 2.
// Nothing is read back to the host.  Waits on a slot being written are
// bounded; one that gives up records an error and abandons the plan (the
// LSD or MSD-first passes then sort correctly).
#include <algorithm>

#include "vdf_common.cuh"
#include "vdf_internal.h"

namespace vdf {
namespace {

__device__ __forceinline__ uint32_t ld_volatile(const uint32_t* p) { return *static_cast<const volatile uint32_t*>(p); }
__device__ __forceinline__ unsigned long long ld_volatile(const unsigned long long* p) {
    return *static_cast<const volatile unsigned long long*>(p);
}

// Adds `add` rows of value x to a CTA's open-addressing table in shared
// memory (keys / counts / states).  A new value takes the next index of
// *distinct; more than kDictMax of them, a full table or a wait that gives up
// set *over.  Returns false when the value was not recorded.  The fences are
// CTA-scoped: only the CTA's own threads read the table.
__device__ bool dict_add(unsigned long long* keys, uint32_t* cnt, uint32_t* st, uint32_t mask, unsigned long long x,
                         uint32_t add, uint32_t limit, uint32_t* distinct, uint32_t* over, uint32_t* err) {
    uint32_t s = dict_hash(x) & mask;
    for (uint32_t probe = 0; probe <= mask; ++probe) {
        // too many values already: the table is not filled further.  Checked
        // at every step, before a slot is claimed: with many distinct keys all
        // the CTA's threads insert at once, and without it they would fill
        // the table and probe it end to end after the plan has failed.
        if (ld_volatile(over)) return false;
        uint32_t state = ld_volatile(st + s);
        if (state == 0) {
            state = atomicCAS(st + s, 0u, 1u);
            if (state == 0) {  // this thread owns the slot: key, then count, then publish
                keys[s] = x;
                atomicAdd(cnt + s, add);
                __threadfence_block();
                atomicExch(st + s, 2u);
                if (atomicAdd(distinct, 1u) >= kDictMax) atomicOr(over, 1u);
                return true;
            }
        }
        uint32_t spins = 0;
        while (state != 2) {  // another thread is writing the slot's key
            if (ld_volatile(over)) return false;
            if (++spins > limit) {
                atomicOr(err, ERR_LOOKBACK_TIMEOUT);
                atomicOr(over, 1u);
                return false;
            }
            if (spins > 16) __nanosleep(32);
            state = ld_volatile(st + s);
        }
        __threadfence_block();
        if (ld_volatile(keys + s) == x) {
            atomicAdd(cnt + s, add);
            return true;
        }
        s = (s + 1) & mask;
    }
    atomicOr(over, 1u);  // never with the planned sizes: more values than slots
    return false;
}

template <typename K>
__global__ void __launch_bounds__(512) k_dict_collect(DictArgs a) {
    __shared__ unsigned long long skey[kDictCtaSlots];
    __shared__ uint32_t scnt[kDictCtaSlots], sst[kDictCtaSlots];
    __shared__ uint32_t sdist, sover;
    for (uint32_t i = threadIdx.x; i < kDictCtaSlots; i += blockDim.x) {
        scnt[i] = 0;
        sst[i] = 0;
    }
    if (threadIdx.x == 0) {
        sdist = 0;
        sover = 0;
    }
    __syncthreads();
    const uint32_t limit = a.spin_limit ? a.spin_limit : kSpinLimit;
    const K* src = static_cast<const K*>(a.keys);
    const uint64_t n = a.n;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    const int lane = threadIdx.x & 31;
    constexpr int R = 4;  // rows per thread per round, all loaded first
    uint32_t round = 0;
    // the loop runs the same number of rounds in every lane of a warp (the
    // bound depends on the warp's first row only), so the warp-wide match
    // below always has all 32 lanes
    const uint64_t warp_first = (uint64_t)blockIdx.x * blockDim.x + (threadIdx.x & ~31u);
    // every early exit is decided for the whole warp at once (__any_sync): a
    // lane leaving alone would leave its warp-mates waiting in the warp-wide
    // ballot below
    for (uint64_t w0 = warp_first; w0 < n; w0 += R * stride, ++round) {
        if (__any_sync(0xffffffffu, ld_volatile(&sover) != 0)) break;
        // another CTA has seen too many values
        if ((round & 7) == 7 && __any_sync(0xffffffffu, ld_volatile(a.overflow) != 0)) break;
        const uint64_t i0 = w0 + lane;
        K k[R];
#pragma unroll
        for (int r = 0; r < R; ++r) k[r] = i0 + r * stride < n ? ldg_stream(src + i0 + r * stride) : K(0);
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const bool valid = i0 + r * stride < n;
            const K kx = KeyOps<K>::order(k[r], a.dtype, a.invert != 0);
            const unsigned long long x = (unsigned long long)kx;
            const uint32_t vb = __ballot_sync(0xffffffffu, valid);
            const uint32_t peers = __match_any_sync(0xffffffffu, kx) & vb;
            // every lane looks its value up at once in its first two slots
            // (read only; with at most 256 values in 512 slots nearly every
            // value is there); the group's leader then adds the group's rows,
            // or takes the insertion path (a new value, or one further on)
            const uint32_t h0 = dict_hash(x) & (kDictCtaSlots - 1), h1 = (h0 + 1) & (kDictCtaSlots - 1);
            const uint32_t st0 = ld_volatile(&sst[h0]), st1 = ld_volatile(&sst[h1]);
            const unsigned long long k0 = ld_volatile(&skey[h0]), k1 = ld_volatile(&skey[h1]);
            uint32_t found = kDictEmpty;
            if (st0 == 2 && k0 == x) found = h0;
            else if (st0 != 0 && st1 == 2 && k1 == x) found = h1;
            if (valid && lane == __ffs(peers) - 1) {
                if (found != kDictEmpty)
                    atomicAdd(&scnt[found], (uint32_t)__popc(peers));
                else
                    dict_add(skey, scnt, sst, kDictCtaSlots - 1, x, (uint32_t)__popc(peers), limit, &sdist, &sover,
                             a.err);
            }
        }
    }
    __syncthreads();
    if (sover) {
        if (threadIdx.x == 0) atomicOr(a.overflow, 1u);
        return;
    }
    if (ld_volatile(a.overflow)) return;
    for (uint32_t s = threadIdx.x; s < kDictCtaSlots; s += blockDim.x) {
        if (sst[s] != 2 || ld_volatile(a.overflow)) continue;
        DictSlot* t = a.table;
        uint32_t g = dict_hash(skey[s]) & (kDictSlots - 1);
        bool done = false;
        for (uint32_t probe = 0; probe < kDictSlots && !done; ++probe) {
            uint32_t state = ld_volatile(&t[g].state);
            if (state == 0) {
                state = atomicCAS(&t[g].state, 0u, 1u);
                if (state == 0) {
                    t[g].key = skey[s];
                    atomicAdd(&t[g].count, scnt[s]);
                    __threadfence();
                    atomicExch(&t[g].state, 2u);
                    if (atomicAdd(a.distinct, 1u) >= kDictMax) atomicOr(a.overflow, 1u);
                    done = true;
                    break;
                }
            }
            uint32_t spins = 0;
            while (state != 2) {
                if (++spins > limit) {
                    atomicOr(a.err, ERR_LOOKBACK_TIMEOUT);
                    atomicOr(a.overflow, 1u);
                    return;
                }
                if (spins > 16) __nanosleep(32);
                state = ld_volatile(&t[g].state);
            }
            __threadfence();
            if (ld_volatile(&t[g].key) == skey[s]) {
                atomicAdd(&t[g].count, scnt[s]);
                done = true;
                break;
            }
            g = (g + 1) & (kDictSlots - 1);
        }
        if (!done) atomicOr(a.overflow, 1u);
    }
}

// One CTA of 1024 threads: ranks, bin starts, lookup table, plan word.
__global__ void __launch_bounds__(1024) k_dict_rank(DictArgs a) {
    __shared__ unsigned long long dk[kDictMax];
    __shared__ uint32_t dc[kDictMax], bycnt[kDictMax], wsum[8];
    __shared__ uint32_t m;
    __shared__ unsigned long long total;
    const uint32_t tid = threadIdx.x;
    if (ld_volatile(a.overflow)) {
        if (tid == 0) *a.state = a.fail_state;
        return;
    }
    if (tid == 0) {
        m = 0;
        total = 0;
    }
    if (tid < kDictMax) bycnt[tid] = 0;
    __syncthreads();
    for (uint32_t s = tid; s < kDictSlots; s += blockDim.x) {
        const DictSlot& t = a.table[s];
        if (t.state == 2) {
            const uint32_t i = atomicAdd(&m, 1u);
            if (i < kDictMax) {
                dk[i] = t.key;
                dc[i] = t.count;
            }
            atomicAdd(&total, (unsigned long long)t.count);
        }
    }
    __syncthreads();
    const uint32_t d = m;
    // every row counted exactly once, or the plan does not apply
    if (d == 0 || d > kDictMax || total != a.n) {
        if (tid == 0) *a.state = a.fail_state;
        return;
    }
    uint32_t rank = 0;
    if (tid < d) {
        const unsigned long long x = dk[tid];
        for (uint32_t j = 0; j < d; ++j) rank += dk[j] < x ? 1u : 0u;
        bycnt[rank] = dc[tid];
    }
    for (uint32_t s = tid; s < kDictLutSlots; s += blockDim.x) a.lut->rank[s] = kDictEmpty;
    __syncthreads();
    // exclusive scan of the counts in rank order (256 threads, one rank each)
    if (tid < kDictMax) {
        const uint32_t v = bycnt[tid];
        uint32_t incl = v;
        const int lane = tid & 31, warp = tid >> 5;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += t;
        }
        if (lane == 31) wsum[warp] = incl;
        __syncwarp();
        bycnt[tid] = incl - v;  // this warp's exclusive part, completed below
    }
    __syncthreads();
    if (tid < kDictMax) {
        uint32_t base = 0;
        for (int w = 0; w < (int)(tid >> 5); ++w) base += wsum[w];
        a.bin_offsets[tid] = base + bycnt[tid];
    }
    // lookup table: claim a free rank slot, then write the key
    if (tid < d) {
        const unsigned long long x = dk[tid];
        uint32_t h = dict_hash(x) & (kDictLutSlots - 1);
        for (uint32_t probe = 0; probe < kDictLutSlots; ++probe) {
            if (atomicCAS(&a.lut->rank[h], kDictEmpty, rank) == kDictEmpty) {
                a.lut->key[h] = x;
                break;
            }
            h = (h + 1) & (kDictLutSlots - 1);
        }
    }
    if (tid == 0) {
        *a.state = 2;
        if (a.taken) atomicAdd(a.taken, 1u);
    }
}

}  // namespace

cudaError_t dict_collect(const DictArgs& a, cudaStream_t s) {
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const uint64_t want = (a.n + 2047) / 2048;
    const uint32_t grid = (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>(want, (uint64_t)sms * 4));
    if (a.width == 8) k_dict_collect<uint64_t><<<grid, 512, 0, s>>>(a);
    else k_dict_collect<uint32_t><<<grid, 512, 0, s>>>(a);
    return cudaGetLastError();
}

cudaError_t dict_rank(const DictArgs& a, cudaStream_t s) {
    k_dict_rank<<<1, 1024, 0, s>>>(a);
    return cudaGetLastError();
}

}  // namespace vdf
