// vdf_msd.cu -- most-significant-digit-first radix sort with a shared-memory
// finish, for sorts by one or two key columns.
//
// The reference sorts with LSD radix passes over every 16-bit digit of the
// key (radix_sort_uint64_mt.inl:6-166: four passes for an 8-byte key, each a
// histogram and a scatter of (key, size_t idx)), and composes a second key by
// a second sort through the in/out idx.  The LSD onesweep passes of
// vdf_radix.cu follow that shape with 8-bit digits: eight passes over HBM for
// an 8-byte key.  Here only the top P digits of key 0 go through HBM-wide
// passes, so that rows sharing the top 8P bits ("buckets") end up
// contiguous; the rest is finished per chunk of whole buckets in shared
// memory:
//
//   1. k_msd_hist    histograms of the top P digits of key 0 (one read)
//   2. k_msd_scan    their exclusive scans; a top-digit bin holding more rows
//                    than chunks could take for every bucket possible under it
//                    (bounded by the lower digits' non-empty bins) flags the
//                    MSD path as failed up front
//   3. P onesweep passes (vdf_radix.cu kernels), stable, over digits
//      W-P .. W-1 of key 0, least significant first: afterwards the rows
//      are stably sorted by their top 8P bits
//   4. k_msd_chunks  chunk c holds the whole buckets that start in
//                    [c*T, (c+1)*T); found by a two-level warp search for
//                    the first bucket boundary at or after c*T
//   5. k_msd_local   one CTA per chunk (<= kMsdCap rows): one counting pass
//                    over 8192 bins of (key - chunk minimum) >> S puts the
//                    rows of spread keys about one per bin; the rows sharing
//                    a bin are ranked by (key 0, key 1's order image,
//                    position in the chunk) -- key 1 is read through the row
//                    id only where key 0 ties -- and the raw sorted key 0 and
//                    the permutation are written.  A chunk where a bin holds
//                    a run longer than kMsdRunMax (many equal or clustered
//                    keys) is sorted instead by stable 8-bit LSD passes in
//                    shared memory over the digits of key 0 above its low F
//                    bits that vary inside it, with runs of equal high bits
//                    ranked the same way (F = 32 for 8-byte keys, 0 for
//                    4-byte keys).
//
// Every pass is stable and ties keep their row order, so the result is
// exactly the stable order over all keys.  A one-key chunk with a run longer
// than kMsdRunMax out of order is finished with more shared-memory passes.
// Where the data defeats the plan (a chunk above kMsdCap rows, or with two
// keys a long run whose key 0 ties or is out of order),
// a device flag is set and the LSD passes that follow in the same stream run
// from the raw columns instead (they return at once while the flag is
// clear); no host round trip either way.
#include "vdf_common.cuh"
#include "vdf_internal.h"

namespace vdf {

// ---------------------------------------------------------------------------
// 1. histograms of the top digits of key 0
// ---------------------------------------------------------------------------
template <typename K>
__global__ void __launch_bounds__(512) k_msd_hist(MsdHistArgs a) {
    // the plan word (written by an earlier launch): this plan runs only at 0
    if (a.flag && *a.flag != 0) return;
    __shared__ uint32_t h[kMsdMaxPasses * 256];
    for (int i = threadIdx.x; i < a.ndig * 256; i += blockDim.x) h[i] = 0;
    __syncthreads();
    const K* src = static_cast<const K*>(a.keys);
    const uint64_t n = a.n;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    constexpr int R = 4;  // four keys per thread per round, all loaded first
    for (uint64_t i0 = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i0 < n; i0 += R * stride) {
        K k[R];
#pragma unroll
        for (int r = 0; r < R; ++r) k[r] = i0 + r * stride < n ? ldg_stream(src + i0 + r * stride) : K(0);
#pragma unroll
        for (int r = 0; r < R; ++r) {
            if (i0 + r * stride >= n) break;
            const K x = KeyOps<K>::order(k[r], a.dtype, a.invert);
            for (int p = 0; p < a.ndig; ++p)
                atomicAdd(&h[p * 256 + (uint32_t)((x >> (8 * (a.first_digit + p))) & 0xff)], 1u);
        }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < a.ndig * 256; i += blockDim.x)
        if (h[i]) atomicAdd(&a.hist[i], h[i]);
}

// ---------------------------------------------------------------------------
// 2. exclusive scans (one CTA of 256 threads, one bin per thread) + the
//    up-front check
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_msd_scan(const uint32_t* hist, uint32_t* offs, int ndig, uint32_t cap,
                                                  uint32_t* flag) {
    __shared__ uint32_t wsum[8];
    __shared__ uint32_t nonempty[kMsdMaxPasses];
    if (*static_cast<volatile uint32_t*>(flag) != 0) return;  // another plan sorts (written by an earlier launch)
    const int b = threadIdx.x, lane = b & 31, warp = b >> 5;
    if (b < kMsdMaxPasses) nonempty[b] = 0;
    uint32_t top = 0;
    for (int p = 0; p < ndig; ++p) {
        __syncthreads();  // wsum of the previous digit has been read
        const uint32_t v = hist[p * 256 + b];
        uint32_t incl = v;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const uint32_t t = __shfl_up_sync(0xffffffffu, incl, d);
            if (lane >= d) incl += t;
        }
        if (lane == 31) wsum[warp] = incl;
        const uint32_t ne = __popc(__ballot_sync(0xffffffffu, v != 0));
        if (lane == 0) atomicAdd(&nonempty[p], ne);
        __syncthreads();
        uint32_t base = 0;
        for (int w = 0; w < warp; ++w) base += wsum[w];
        offs[p * 256 + b] = base + incl - v;
        if (p == ndig - 1) top = v;
    }
    __syncthreads();
    // Rows under one top-digit value can form at most as many buckets as the
    // lower digits have distinct values (the product of their non-empty
    // bins); more rows than that many full chunks hold means some bucket
    // cannot fit a chunk.
    uint64_t under = 1;
    for (int p = 0; p + 1 < ndig; ++p) under *= nonempty[p];
    if ((uint64_t)top > (uint64_t)cap * under) atomicOr(flag, 1u);
}

// ---------------------------------------------------------------------------
// 4. chunk starts: one warp per chunk
// ---------------------------------------------------------------------------
template <typename K, uint32_t CAP>
__global__ void __launch_bounds__(256) k_msd_chunks(MsdChunkArgs a) {
    const int lane = threadIdx.x & 31;
    const uint32_t c = blockIdx.x * 8 + (threadIdx.x >> 5);
    if (c > a.nchunks) return;
    const K* keys = static_cast<const K*>(a.keys);
    // chunk c starts at or after row x of rows [start, end) sorted by their
    // top bits (key >> pshift); a segmented sort gives each chunk its
    // segment's bounds, shift and failure flag
    uint64_t x = 0, start = 0, end = a.n;
    uint32_t pshift = a.pshift;
    uint32_t* flag = a.flag;
    if (c < a.nchunks) {
        if (a.seg_chunks) {
            const MsdSegChunk d = a.seg_chunks[c];
            x = d.x;
            start = d.seg_start;
            end = min((uint64_t)d.seg_end, a.n);
            pshift = d.pshift;
            flag = a.seg_flag + d.seg;
        } else {
            x = (uint64_t)c * a.chunk_rows;
        }
    }
    uint64_t out;
    if (c == a.nchunks) {
        out = a.n;
    } else if (x <= start || x >= end) {
        // a segment's first chunk starts with it (written even when the
        // segment has failed: the chunk before it may end another segment)
        out = min(max(x, start), end);
    } else {
        uint32_t failed = 0;  // read once per warp: the ballots below need the whole warp
        if (lane == 0) failed = *static_cast<volatile uint32_t*>(flag);
        if (__shfl_sync(0xffffffffu, failed, 0)) return;
        // first i >= x whose top bits differ from row x-1's; rows are sorted
        // by their top bits, so "differs" is false up to the boundary and
        // true after it, and a probe tells on which side it lies
        const K p0 = keys[x - 1] >> pshift;
        constexpr uint32_t S = CAP / 32;  // level-1 probe spacing
        const uint64_t q = min(x + (uint64_t)(lane + 1) * S - 1, end - 1);
        const uint32_t hit = __ballot_sync(0xffffffffu, (keys[q] >> pshift) != p0);
        if (!hit) {
            // CAP rows after x still share row x-1's top bits: that bucket
            // is larger than a chunk can hold (or runs to the end)
            out = end;
            if (x + (uint64_t)32 * S - 1 < end - 1 && lane == 0) atomicOr(flag, 1u);
        } else {
            const uint32_t L = __ffs(hit) - 1;
            const uint64_t lo = x + (uint64_t)L * S;  // every row before lo shares p0
            const uint64_t hi = min(x + (uint64_t)(L + 1) * S - 1, end - 1);  // differs at hi
            out = hi;
#pragma unroll
            for (uint32_t r = 0; r < S / 32; ++r) {
                const uint64_t pos = lo + r * 32 + lane;
                const bool d = pos >= hi || (keys[pos] >> pshift) != p0;
                const uint32_t b = __ballot_sync(0xffffffffu, d);
                if (b) {
                    out = lo + r * 32 + (__ffs(b) - 1);
                    break;
                }
            }
        }
    }
    if (lane == 0) a.chunk_start[c] = (uint32_t)out;
}

// ---------------------------------------------------------------------------
// 5. shared-memory finish, one CTA per chunk
// ---------------------------------------------------------------------------
template <typename K, int THREADS, int ITEMS>
struct LocalCfg {
    static constexpr int WARPS = THREADS / 32;
    static constexpr int CAP = THREADS * ITEMS;
    static constexpr size_t KEYS = (size_t)CAP * sizeof(K);
    static constexpr size_t VALS = (size_t)CAP * 4;
    static constexpr size_t SEC = (size_t)CAP * 8;  // key 1 images of rows in runs; the counting pass's bins
    static constexpr size_t MISC = 16 * 4 + (size_t)WARPS * 4 + (size_t)2 * WARPS * 8;
    static constexpr size_t ORIG = (size_t)CAP * 2;  // chunk position of each slot's row
    static constexpr size_t SBIN = (size_t)CAP * 2;  // bin of each slot's row
    static constexpr size_t SMEM = KEYS + VALS + SEC + MISC + ORIG + SBIN;
    // the counting pass's 8192 bins and the LSD passes' per-warp counters
    // live in the key-1 buffer, which is only needed after either is done
    static_assert(SEC >= (size_t)2 * CAP * 4 && SEC >= (size_t)WARPS * 256 * 4, "key-1 buffer doubles as counters");
};

template <int THREADS>
__device__ __forceinline__ uint32_t local_excl_scan(uint32_t v, uint32_t* wsum, uint32_t* total) {
    constexpr int WARPS = THREADS / 32;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t incl = v;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const uint32_t t = __shfl_up_sync(0xffffffffu, incl, d);
        if (lane >= d) incl += t;
    }
    if (lane == 31) wsum[warp] = incl;
    __syncthreads();
    uint32_t base = 0, all = 0;
#pragma unroll
    for (int w = 0; w < WARPS; ++w) {
        const uint32_t x = wsum[w];
        base += (w < warp) ? x : 0u;
        all += x;
    }
    *total = all;
    return base + incl - v;
}

__device__ __forceinline__ uint64_t sec_image(const void* col, int dt, uint32_t row, bool invert) {
    if (dtype_width(dt) == 8) return order64(ld_rand8(static_cast<const unsigned long long*>(col) + row), dt, invert);
    return (uint64_t)order32(ld_rand4(static_cast<const uint32_t*>(col) + row), dt, invert);
}

// One stable 8-bit LSD pass in shared memory over the digit digit(key) of
// the CTA's rows (item j of a thread at position (warp * ia + j) * 32 + lane;
// slots past the chunk hold all-ones keys, whose digit must be the largest,
// and rank last).  Afterwards the rows are in sk / sv in the new order and
// back in key / val by position.
template <typename K, int THREADS, int ITEMS, int MATCH, typename DigitF>
__device__ __forceinline__ void local_pass(K (&key)[ITEMS], uint32_t (&val)[ITEMS], DigitF digit, uint32_t ia,
                                           K* sk, uint32_t* sv, uint32_t* wcnt, uint32_t* wsum, uint32_t* err) {
    constexpr int WARPS = THREADS / 32, RADIX = 256;
    constexpr uint32_t CAP = (uint32_t)(THREADS * ITEMS);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const uint32_t lt = lanemask_lt();
    uint32_t* my = wcnt + warp * RADIX;
    for (int i = tid; i < WARPS * RADIX; i += THREADS) wcnt[i] = 0;
    __syncthreads();
    uint32_t rank[ITEMS];
#pragma unroll
    for (int j = 0; j < ITEMS; ++j) {
        rank[j] = 0;
        if (j < (int)ia) {
            const uint32_t d = digit(key[j]);
            uint32_t peers;
            if constexpr (MATCH == 1) {
                peers = __match_any_sync(0xffffffffu, d);
            } else {
                peers = 0xffffffffu;
#pragma unroll
                for (int bt = 0; bt < 8; ++bt) {
                    const uint32_t bal = __ballot_sync(0xffffffffu, (d >> bt) & 1u);
                    peers &= ((d >> bt) & 1u) ? bal : ~bal;
                }
            }
            const int leader = __ffs(peers) - 1;
            uint32_t base = 0;
            if (lane == leader) {
                base = my[d];
                my[d] = base + __popc(peers);
            }
            __syncwarp();
            base = __shfl_sync(0xffffffffu, base, leader);
            rank[j] = base + __popc(peers & lt);
        }
    }
    __syncthreads();
    // bin-major exclusive prefix over (bin, warp)
    uint32_t tot = 0;
    if (tid < RADIX) {
#pragma unroll
        for (int w = 0; w < WARPS; ++w) {
            const uint32_t c = wcnt[w * RADIX + tid];
            wcnt[w * RADIX + tid] = tot;
            tot += c;
        }
    }
    uint32_t all;
    const uint32_t start = local_excl_scan<THREADS>(tot, wsum, &all);
    if (tid < RADIX)
#pragma unroll
        for (int w = 0; w < WARPS; ++w) wcnt[w * RADIX + tid] += start;
    __syncthreads();
#pragma unroll
    for (int j = 0; j < ITEMS; ++j) {
        if (j < (int)ia) {
            const uint32_t d = digit(key[j]);
            uint32_t r = rank[j] + my[d];
            if (r >= CAP) {  // never when the counts are consistent
                atomicOr(err, ERR_BAD_INDEX);
                r = ((uint32_t)warp * ia + j) * 32 + lane;
            }
            sk[r] = key[j];
            sv[r] = val[j];
        }
    }
    __syncthreads();
#pragma unroll
    for (int j = 0; j < ITEMS; ++j) {
        if (j < (int)ia) {
            const uint32_t pos = ((uint32_t)warp * ia + j) * 32 + lane;
            key[j] = sk[pos];
            val[j] = sv[pos];
        }
    }
}

// The chunk's rows in one counting pass: bin = (key - min) >> S with S the
// smallest shift that brings the chunk's key range below 8192 bins, so rows
// of spread keys fall about one per bin or fewer.  Rows land in their bin in no
// particular order (shared-memory atomics); then each run of rows sharing a
// bin is ranked by (key, key 1's order image, position in the chunk) --
// positions are the rows' stable order so far -- which restores the exact
// stable order.  Returns false, with nothing written to global memory, when
// some run is longer than kMsdRunMax (many equal or clustered keys): the
// caller then sorts the chunk with LSD passes instead.  On success item j of
// a thread holds the row of slot (warp * ia + j) * 32 + lane and its final
// position in the chunk is newpos[j].
// Warp-wide minimum / maximum with the 32-bit reduce instructions: 8-byte
// keys reduce their high halves first, then the low halves of the lanes that
// hold the extreme high half.
__device__ __forceinline__ uint32_t warp_min(uint32_t x) { return __reduce_min_sync(0xffffffffu, x); }
__device__ __forceinline__ uint32_t warp_max(uint32_t x) { return __reduce_max_sync(0xffffffffu, x); }
__device__ __forceinline__ uint64_t warp_min(uint64_t x) {
    const uint32_t hi = __reduce_min_sync(0xffffffffu, (uint32_t)(x >> 32));
    const uint32_t lo = __reduce_min_sync(0xffffffffu, (uint32_t)(x >> 32) == hi ? (uint32_t)x : 0xffffffffu);
    return ((uint64_t)hi << 32) | lo;
}
__device__ __forceinline__ uint64_t warp_max(uint64_t x) {
    const uint32_t hi = __reduce_max_sync(0xffffffffu, (uint32_t)(x >> 32));
    const uint32_t lo = __reduce_max_sync(0xffffffffu, (uint32_t)(x >> 32) == hi ? (uint32_t)x : 0u);
    return ((uint64_t)hi << 32) | lo;
}

template <typename K, int THREADS, int ITEMS, int MATCH>
__device__ __forceinline__ bool counting_finish(K (&key)[ITEMS], uint32_t (&val)[ITEMS], uint32_t (&newpos)[ITEMS],
                                                uint32_t m, uint32_t ia, const MsdLocalArgs& a, K* sk, uint32_t* sv,
                                                uint16_t* so, uint16_t* sbin, uint64_t* ssec, uint32_t* misc,
                                                uint32_t* wsum, K* wmin, K* wmax) {
    // the bins live in the key-1 buffer, which is not needed before the
    // scatter is done
    uint32_t* bins = reinterpret_cast<uint32_t*>(ssec);
    constexpr int WARPS = THREADS / 32;
    // bins (two per slot: 8192 for 4096-row chunks), bins per thread
    constexpr int NB = 2 * THREADS * ITEMS, BPT = NB / THREADS;
    constexpr int LNB = NB == 16384 ? 14 : 13;
    static_assert((1 << LNB) == NB && BPT % 4 == 0, "bin layout");
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    // ---- key range of the chunk
    K kmin = ~K(0), kmax = 0;
#pragma unroll
    for (int j = 0; j < ITEMS; ++j) {
        const uint32_t pos = ((uint32_t)warp * ia + j) * 32 + lane;
        if (j < (int)ia && pos < m) {
            kmin = min(kmin, key[j]);
            kmax = max(kmax, key[j]);
        }
    }
    kmin = warp_min(kmin);
    kmax = warp_max(kmax);
    if (lane == 0) {
        wmin[warp] = kmin;
        wmax[warp] = kmax;
    }
#pragma unroll
    for (int i = 0; i < BPT; i += 4) *reinterpret_cast<uint4*>(bins + tid * BPT + i) = make_uint4(0, 0, 0, 0);
    __syncthreads();
    kmin = warp_min(lane < WARPS ? wmin[lane] : ~K(0));
    kmax = warp_max(lane < WARPS ? wmax[lane] : K(0));
    const K range = kmax - kmin;
    int bl = 0;  // bit length of the range
    if constexpr (sizeof(K) == 8) bl = range ? 64 - __clzll((long long)range) : 0;
    else bl = range ? 32 - __clz((int)range) : 0;
    const uint32_t S = bl > 13 ? (uint32_t)(bl - 13) : 0u;
    auto bin_of = [&](K k) -> uint32_t { return (uint32_t)((k - kmin) >> S); };
    // ---- histogram, exclusive scan, scatter
#pragma unroll
    for (int j = 0; j < ITEMS; ++j) {
        const uint32_t pos = ((uint32_t)warp * ia + j) * 32 + lane;
        if (j < (int)ia && pos < m) atomicAdd(&bins[bin_of(key[j])], 1u);
    }
    __syncthreads();
    // one scan of packed words: rows before the bin (low 16 bits) and
    // occupied bins before it (high 16 bits: the bin's dense index)
    uint32_t b[BPT];
    uint32_t tsum = 0, tmax = 0;
#pragma unroll
    for (int i = 0; i < BPT; i += 4) {
        const uint4 q = *reinterpret_cast<const uint4*>(bins + tid * BPT + i);
        b[i] = q.x;
        b[i + 1] = q.y;
        b[i + 2] = q.z;
        b[i + 3] = q.w;
    }
#pragma unroll
    for (int i = 0; i < BPT; ++i) {
        const uint32_t c = b[i];
        tmax = max(tmax, c);
        b[i] = tsum;
        tsum += c + (c ? (1u << 16) : 0u);
    }
    uint32_t all;
    const uint32_t start = local_excl_scan<THREADS>(tsum, wsum, &all);
    if (__syncthreads_or(tmax > kMsdRunMax)) {
        // A bin holds a run longer than the direct ranking takes (many equal
        // or clustered keys): stable passes over the dense bin index instead
        // of the scatter -- one when at most 256 bins are occupied, else two
        // -- keep each bin's rows in their stable order, which is the final
        // order wherever a bin holds one key value.  The dense index table
        // takes the position and bin buffers (unused on this path).
        static_assert(2 * (size_t)THREADS * ITEMS >= NB, "dense table fits the position and bin buffers");
        uint16_t* dt = so;
#pragma unroll
        for (int i = 0; i < BPT; ++i) dt[tid * BPT + i] = (uint16_t)((start + b[i]) >> 16);
        __syncthreads();
        // slots past the chunk (all-ones keys) take the largest index, so they stay last
        auto dense = [&](K k) -> uint32_t {
            const K off = (k - kmin) >> S;
            return off < (K)NB ? (uint32_t)dt[(uint32_t)off] : 0xffffu;
        };
        uint32_t* wcnt = bins;  // the bin counts are no longer needed
        if ((all >> 16) <= 256) {
            local_pass<K, THREADS, ITEMS, MATCH>(
                key, val, [&](K k) { return min(dense(k), 255u); }, ia, sk, sv, wcnt, wsum, a.err);
        } else {
            local_pass<K, THREADS, ITEMS, MATCH>(
                key, val, [&](K k) { return dense(k) & 0xffu; }, ia, sk, sv, wcnt, wsum, a.err);
            local_pass<K, THREADS, ITEMS, MATCH>(
                key, val, [&](K k) { return dense(k) >> 8; }, ia, sk, sv, wcnt, wsum, a.err);
        }
        // in order now unless some bin holds several key values (or, with a
        // second key, key 0 ties): then the caller's LSD passes take over
        bool bad = false;
#pragma unroll
        for (int j = 0; j < ITEMS; ++j) {
            const uint32_t pos = ((uint32_t)warp * ia + j) * 32 + lane;
            if (j < (int)ia && pos > 0 && pos < m) {
                const K prev = sk[pos - 1];
                bad |= a.sec ? !(prev < key[j]) : (prev > key[j]);
            }
        }
        return __syncthreads_or(bad) == 0;
    }
#pragma unroll
    for (int i = 0; i < BPT; i += 4)
        *reinterpret_cast<uint4*>(bins + tid * BPT + i) =
            make_uint4((start + b[i]) & 0xffffu, (start + b[i + 1]) & 0xffffu, (start + b[i + 2]) & 0xffffu,
                       (start + b[i + 3]) & 0xffffu);
    __syncthreads();
#pragma unroll
    for (int j = 0; j < ITEMS; ++j) {
        const uint32_t pos = ((uint32_t)warp * ia + j) * 32 + lane;
        if (j < (int)ia && pos < m) {
            const uint32_t bn = bin_of(key[j]);
            uint32_t slot = atomicAdd(&bins[bn], 1u);
            if (slot >= m) {  // never when the counts are consistent
                atomicOr(a.err, ERR_BAD_INDEX);
                slot = pos;
            }
            sk[slot] = key[j];
            sv[slot] = val[j];
            so[slot] = (uint16_t)pos;
            sbin[slot] = (uint16_t)bn;
        }
    }
    __syncthreads();
    // ---- rows by slot; runs of one bin (bounds from ballots over each
    //      32-slot group, loops only for runs that cross a group), and key 1
    //      where key 0 ties inside a run
    uint32_t run[ITEMS];  // s | e << 16; 0: alone in its bin
    const uint32_t lt = lanemask_lt();
#pragma unroll
    for (int j = 0; j < ITEMS; ++j) {
        const uint32_t base = ((uint32_t)warp * ia + j) * 32;
        const uint32_t p = base + lane;
        newpos[j] = p;
        run[j] = 0;
        if (j < (int)ia) {
            bool first = true, last = true;
            uint32_t h = 0;
            if (p < m) {
                key[j] = sk[p];
                val[j] = sv[p];
                h = sbin[p];
                first = p == 0 || sbin[p - 1] != h;
                last = p + 1 >= m || sbin[p + 1] != h;
            }
            const uint32_t starts = __ballot_sync(0xffffffffu, first);
            const uint32_t ends = __ballot_sync(0xffffffffu, last);
            if (!(first && last)) {
                const uint32_t sm = starts & (lt | (1u << lane));  // starts at lanes <= this one
                const uint32_t em = ends & ~lt;                    // ends at lanes >= this one
                uint32_t s = sm ? base + 31 - __clz(sm) : base;
                uint32_t e = em ? base + __ffs(em) : base + 32;
                if (!sm)
                    while (s > 0 && p - s < kMsdRunMax && sbin[s - 1] == h) --s;
                if (!em)
                    while (e < m && e - p <= kMsdRunMax && sbin[e] == h) ++e;
                run[j] = s | (e << 16);
                if (e - s > kMsdRunMax) {
                    misc[4] = 1;
                } else if (a.sec) {
                    bool tie = false;
                    for (uint32_t t = s; t < e; ++t) tie |= (t != p) && sk[t] == key[j];
                    if (tie) {
                        uint32_t row = val[j];
                        if (row >= a.n) {  // never for a permutation of [0, n)
                            atomicOr(a.err, ERR_BAD_INDEX);
                            row = 0;
                        }
                        ssec[p] = sec_image(a.sec, a.sec_dtype, row, a.invert != 0);
                    }
                }
            }
        }
    }
    __syncthreads();
    if (misc[4]) return false;
#pragma unroll
    for (int j = 0; j < ITEMS; ++j) {
        if (run[j] == 0) continue;
        const uint32_t p = ((uint32_t)warp * ia + j) * 32 + lane;
        const uint32_t s = run[j] & 0xffffu, e = run[j] >> 16;
        const K k = key[j];
        const uint32_t o = so[p];
        uint32_t r = 0;
        for (uint32_t t = s; t < e; ++t) {
            const K tk = sk[t];
            bool less = tk < k;
            if (tk == k && t != p) {
                const uint32_t to = so[t];
                if (a.sec) {
                    const uint64_t sc = ssec[p], tsc = ssec[t];
                    less = tsc < sc || (tsc == sc && to < o);
                } else {
                    less = to < o;
                }
            }
            r += less ? 1u : 0u;
        }
        newpos[j] = s + r;
    }
    return true;
}

// MATCH: 0 = one ballot per digit bit, 1 = match.any.
template <typename K, int THREADS, int ITEMS, int MATCH>
__global__ void __launch_bounds__(THREADS, THREADS >= 1024 ? 1 : 2) k_msd_local(MsdLocalArgs a) {
    using C = LocalCfg<K, THREADS, ITEMS>;
    constexpr int WARPS = C::WARPS, RADIX = 256;
    constexpr uint32_t CAP = (uint32_t)C::CAP;
    constexpr int KBITS = 8 * (int)sizeof(K);
    extern __shared__ __align__(16) unsigned char smem[];
    K* sk = reinterpret_cast<K*>(smem);
    uint32_t* sv = reinterpret_cast<uint32_t*>(smem + C::KEYS);
    uint64_t* ssec = reinterpret_cast<uint64_t*>(smem + C::KEYS + C::VALS);
    uint32_t* wcnt = reinterpret_cast<uint32_t*>(ssec);                                 // [WARPS][RADIX]
    uint32_t* misc = reinterpret_cast<uint32_t*>(smem + C::KEYS + C::VALS + C::SEC);  // [0], [4]: long runs
    uint32_t* wsum = misc + 16;                                                       // [WARPS]
    K* wor = reinterpret_cast<K*>(smem + C::KEYS + C::VALS + C::SEC + 16 * 4 + WARPS * 4);
    K* wand = wor + WARPS;
    uint16_t* so = reinterpret_cast<uint16_t*>(smem + C::KEYS + C::VALS + C::SEC + C::MISC);
    uint16_t* sbin = so + CAP;

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    // the flag a failing chunk raises: the sort's, or its segment's
    uint32_t* const fail_word = a.seg_chunks ? a.seg_flag + a.seg_chunks[blockIdx.x].seg : a.flag;
    // One thread reads the flag and the chunk bounds for the whole CTA (the
    // flag may be raised by another CTA meanwhile; every thread must take
    // the same branch around the barriers below).
    if (tid == 0) {
        misc[1] = *static_cast<volatile uint32_t*>(fail_word);
        misc[2] = a.chunk_start[blockIdx.x];
        uint32_t e = a.chunk_start[blockIdx.x + 1];
        if (a.seg_chunks) e = min(e, a.seg_chunks[blockIdx.x].seg_end);  // the segment's last chunk
        misc[3] = e;
        misc[0] = 0;
        misc[4] = 0;
    }
    __syncthreads();
    if (misc[1]) return;  // the plan failed earlier: the LSD passes take over
    const uint32_t s0 = misc[2], s1 = misc[3];
    if (s1 <= s0) return;
    const uint32_t m = s1 - s0;
    if (m > CAP || s1 > a.n) {
        if (tid == 0) atomicOr(fail_word, 1u);
        return;
    }
    const uint32_t ia = (m + THREADS - 1) / THREADS;  // items per thread in use

    // ---- load: item j of a thread sits at position (warp * ia + j) * 32 + lane;
    //      slots past m hold all-ones keys, which every pass ranks last
    K key[ITEMS];
    uint32_t val[ITEMS];
    const K* kin = static_cast<const K*>(a.keys) + s0;
    const uint32_t* vin = a.vals + s0;
#pragma unroll
    for (int j = 0; j < ITEMS; ++j) {
        const uint32_t pos = ((uint32_t)warp * ia + j) * 32 + lane;
        key[j] = ~K(0);
        val[j] = 0;
        if (j < (int)ia && pos < m) {
            key[j] = ldg_stream(kin + pos);
            val[j] = ldg_stream(vin + pos);
        }
    }

    // ---- rows already in order (with one key: non-decreasing; with two:
    //      increasing, so key 1 decides nothing) stay where they are; this is
    //      the common case when each bucket holds one key value
    bool in_order = true;
#pragma unroll
    for (int j = 0; j < ITEMS; ++j) {
        const uint32_t pos = ((uint32_t)warp * ia + j) * 32 + lane;
        if (j < (int)ia) {
            K prev = __shfl_up_sync(0xffffffffu, key[j], 1);
            if (lane == 0 && pos > 0 && pos < m) prev = kin[pos - 1];
            if (pos > 0 && pos < m) in_order = in_order && (a.sec ? prev < key[j] : prev <= key[j]);
        }
    }
    in_order = __syncthreads_and(in_order) != 0;
    uint32_t newpos[ITEMS];
#pragma unroll
    for (int j = 0; j < ITEMS; ++j) newpos[j] = ((uint32_t)warp * ia + j) * 32 + lane;

    // ---- one counting pass over the chunk's key range; where that leaves a
    //      long run (many equal or clustered keys), stable LSD passes instead
    const bool counted = in_order || counting_finish<K, THREADS, ITEMS, MATCH>(key, val, newpos, m, ia, a, sk, sv, so,
                                                                               sbin, ssec, misc, wsum, wor, wand);
    if (!counted) {
        __syncthreads();
#pragma unroll
        for (int j = 0; j < ITEMS; ++j) {
            const uint32_t pos = ((uint32_t)warp * ia + j) * 32 + lane;
            key[j] = ~K(0);
            val[j] = 0;
            if (j < (int)ia && pos < m) {
                key[j] = ldg_stream(kin + pos);
                val[j] = ldg_stream(vin + pos);
            }
        }
        // ---- which digits vary inside the chunk
        K vor = 0, vand = ~K(0);
    #pragma unroll
        for (int j = 0; j < ITEMS; ++j) {
            const uint32_t pos = ((uint32_t)warp * ia + j) * 32 + lane;
            if (j < (int)ia && pos < m) {
                vor |= key[j];
                vand &= key[j];
            }
        }
    #pragma unroll
        for (int d = 16; d >= 1; d >>= 1) {
            vor |= __shfl_xor_sync(0xffffffffu, vor, d);
            vand &= __shfl_xor_sync(0xffffffffu, vand, d);
        }
        if (lane == 0) {
            wor[warp] = vor;
            wand[warp] = vand;
        }
        __syncthreads();
        vor = 0;
        vand = ~K(0);
    #pragma unroll
        for (int w = 0; w < WARPS; ++w) {
            vor |= wor[w];
            vand &= wand[w];
        }
        const K vary = vor ^ vand;

        // ---- stable 8-bit LSD passes in shared memory over the varying digits
        //      of key 0 from digit lo_bits / 8 up
        bool sorted_in_smem = false;
        for (int dg = (int)(a.lo_bits / 8); dg < KBITS / 8; ++dg) {
            const uint32_t shift = 8u * dg;
            if (((vary >> shift) & 0xff) == 0) continue;
            local_pass<K, THREADS, ITEMS, MATCH>(
                key, val, [shift](K k) { return (uint32_t)(k >> shift) & 0xffu; }, ia, sk, sv, wcnt, wsum, a.err);
            sorted_in_smem = true;
        }
        if (!sorted_in_smem) {
    #pragma unroll
            for (int j = 0; j < ITEMS; ++j) {
                if (j < (int)ia) {
                    const uint32_t pos = ((uint32_t)warp * ia + j) * 32 + lane;
                    sk[pos] = key[j];
                    sv[pos] = val[j];
                }
            }
            __syncthreads();
        }

        // ---- runs of equal high bits, ranked by (low bits, key 1, position).
        //      Key 1 is read (through the row id) only for rows whose low bits
        //      tie with another row of their run, i.e. rows whose key 0 ties.
        const bool fix = a.lo_bits > 0 || a.sec != nullptr;
        const uint32_t hs = a.lo_bits;  // high part = key >> hs
        const K lo_mask = hs ? (K)((((K)1) << hs) - 1) : K(0);
        uint32_t run[ITEMS];  // run bounds s | e << 16 (positions < 2^16); 0: not in a run
    #pragma unroll
        for (int j = 0; j < ITEMS; ++j) {
            const uint32_t pos = ((uint32_t)warp * ia + j) * 32 + lane;
            newpos[j] = pos;
            run[j] = 0;
            if (fix && j < (int)ia && pos < m) {
                const K h = key[j] >> hs;
                if ((pos > 0 && (sk[pos - 1] >> hs) == h) || (pos + 1 < m && (sk[pos + 1] >> hs) == h)) {
                    uint32_t s = pos, e = pos + 1;
                    while (s > 0 && pos - s < kMsdRunMax && (sk[s - 1] >> hs) == h) --s;
                    while (e < m && e - pos <= kMsdRunMax && (sk[e] >> hs) == h) ++e;
                    run[j] = s | (e << 16);
                    if (a.sec && e - s <= kMsdRunMax) {
                        const K lo = key[j] & lo_mask;
                        bool tie = false;
                        for (uint32_t t = s; t < e; ++t) tie |= (t != pos) && ((sk[t] & lo_mask) == lo);
                        if (tie) {
                            uint32_t row = val[j];
                            if (row >= a.n) {  // never for a permutation of [0, n)
                                atomicOr(a.err, ERR_BAD_INDEX);
                                row = 0;
                            }
                            ssec[pos] = sec_image(a.sec, a.sec_dtype, row, a.invert != 0);
                        }
                    }
                }
            }
        }
        if (fix) {
            __syncthreads();
    #pragma unroll
            for (int j = 0; j < ITEMS; ++j) {
                if (run[j] == 0) continue;
                const uint32_t pos = ((uint32_t)warp * ia + j) * 32 + lane;
                const uint32_t s = run[j] & 0xffffu, e = run[j] >> 16;
                const K lo = key[j] & lo_mask;
                if (e - s > kMsdRunMax) {
                    // a long run: fine if it already is in order (e.g. equal
                    // keys of a one-key sort); otherwise see below
                    if (pos > s) {
                        const K plo = sk[pos - 1] & lo_mask;
                        if (plo > lo || (plo == lo && a.sec)) misc[0] = 1;
                    }
                    continue;
                }
                uint32_t r = 0;
                bool have_sec = false;
                uint64_t sc = 0;
                for (uint32_t t = s; t < e; ++t) {
                    const K tlo = sk[t] & lo_mask;
                    bool less = tlo < lo;
                    if (tlo == lo && t != pos) {
                        if (a.sec) {
                            if (!have_sec) {
                                sc = ssec[pos];
                                have_sec = true;
                            }
                            const uint64_t tsc = ssec[t];
                            less = tsc < sc || (tsc == sc && t < pos);
                        } else {
                            less = t < pos;
                        }
                    }
                    r += less ? 1u : 0u;
                }
                newpos[j] = s + r;
            }
            __syncthreads();
            if (misc[0]) {
                // A run longer than the direct ranking handles is out of order.
                // With a second key that needs key 1 for every row: the plan
                // fails.  With one key the chunk is finished in shared memory:
                // LSD passes over the varying low digits, then the high ones
                // again (every pass is stable, so ties keep their row order).
                if (a.sec) {
                    if (tid == 0) atomicOr(fail_word, 1u);
                    return;
                }
                for (int dg = 0; dg < KBITS / 8; ++dg) {
                    const uint32_t shift = 8u * dg;
                    if (((vary >> shift) & 0xff) == 0) continue;
                    local_pass<K, THREADS, ITEMS, MATCH>(
                        key, val, [shift](K k) { return (uint32_t)(k >> shift) & 0xffu; }, ia, sk, sv, wcnt, wsum,
                        a.err);
                }
    #pragma unroll
                for (int j = 0; j < ITEMS; ++j) newpos[j] = ((uint32_t)warp * ia + j) * 32 + lane;
            }
        }
    }

    // ---- output: raw sorted key 0 and the permutation
    K* kout = static_cast<K*>(a.keys_out);
#pragma unroll
    for (int j = 0; j < ITEMS; ++j) {
        const uint32_t pos = ((uint32_t)warp * ia + j) * 32 + lane;
        if (j < (int)ia && pos < m) {
            uint64_t gp = (uint64_t)s0 + newpos[j];
            if (a.reverse) gp = a.n - 1 - gp;
            stg_stream(a.perm_out + gp, val[j]);
            if (kout) stg_stream(kout + gp, KeyOps<K>::unorder(key[j], a.dtype, a.invert != 0));
        }
    }
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
namespace {
constexpr int kLocalThreads = 512, kLocalItems = 8;
static_assert(kLocalThreads * kLocalItems == (int)kMsdCap, "chunk capacity");
static_assert(2 * kLocalThreads * kLocalItems == (int)kMsdWideCap, "wide chunk capacity");
static_assert(kMsdWideCap < (1u << 16), "run bounds are packed in 16 bits");
using Local64 = LocalCfg<uint64_t, kLocalThreads, kLocalItems>;
using Local32 = LocalCfg<uint32_t, kLocalThreads, kLocalItems>;
using Wide64 = LocalCfg<uint64_t, 2 * kLocalThreads, kLocalItems>;
using Wide32 = LocalCfg<uint32_t, 2 * kLocalThreads, kLocalItems>;
template <int MATCH>
struct LocalKernels {
    static constexpr auto k64 = k_msd_local<uint64_t, kLocalThreads, kLocalItems, MATCH>;
    static constexpr auto k32 = k_msd_local<uint32_t, kLocalThreads, kLocalItems, MATCH>;
    // wide chunks (<= 8192 rows): one CTA of 1024 threads per SM
    static constexpr auto w64 = k_msd_local<uint64_t, 2 * kLocalThreads, kLocalItems, MATCH>;
    static constexpr auto w32 = k_msd_local<uint32_t, 2 * kLocalThreads, kLocalItems, MATCH>;
};

int sm_count() {
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    return sms;
}
}  // namespace

cudaError_t prepare_msd_kernels() {
    const void* k64[2] = {(const void*)LocalKernels<0>::k64, (const void*)LocalKernels<1>::k64};
    const void* k32[2] = {(const void*)LocalKernels<0>::k32, (const void*)LocalKernels<1>::k32};
    const void* w64[2] = {(const void*)LocalKernels<0>::w64, (const void*)LocalKernels<1>::w64};
    const void* w32[2] = {(const void*)LocalKernels<0>::w32, (const void*)LocalKernels<1>::w32};
    for (int m = 0; m < 2; ++m) {
        cudaError_t e = cudaFuncSetAttribute(k64[m], cudaFuncAttributeMaxDynamicSharedMemorySize, (int)Local64::SMEM);
        if (e != cudaSuccess) return e;
        e = cudaFuncSetAttribute(k32[m], cudaFuncAttributeMaxDynamicSharedMemorySize, (int)Local32::SMEM);
        if (e != cudaSuccess) return e;
        e = cudaFuncSetAttribute(w64[m], cudaFuncAttributeMaxDynamicSharedMemorySize, (int)Wide64::SMEM);
        if (e != cudaSuccess) return e;
        e = cudaFuncSetAttribute(w32[m], cudaFuncAttributeMaxDynamicSharedMemorySize, (int)Wide32::SMEM);
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

cudaError_t msd_hist(const MsdHistArgs& a, int width, cudaStream_t s) {
    const uint64_t want = (a.n + 511) / 512;
    const uint32_t grid = (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>(want, (uint64_t)sm_count() * 4));
    if (width == 8) k_msd_hist<uint64_t><<<grid, 512, 0, s>>>(a);
    else k_msd_hist<uint32_t><<<grid, 512, 0, s>>>(a);
    return cudaGetLastError();
}

cudaError_t msd_scan(const uint32_t* hist, uint32_t* offs, int ndig, uint32_t cap, uint32_t* flag, cudaStream_t s) {
    k_msd_scan<<<1, 256, 0, s>>>(hist, offs, ndig, cap, flag);
    return cudaGetLastError();
}

cudaError_t msd_chunks(const MsdChunkArgs& a, int width, cudaStream_t s, uint32_t cap) {
    const uint32_t grid = (a.nchunks + 1 + 7) / 8;
    if (cap == kMsdWideCap) {
        if (width == 8) k_msd_chunks<uint64_t, kMsdWideCap><<<grid, 256, 0, s>>>(a);
        else k_msd_chunks<uint32_t, kMsdWideCap><<<grid, 256, 0, s>>>(a);
    } else {
        if (width == 8) k_msd_chunks<uint64_t, kMsdCap><<<grid, 256, 0, s>>>(a);
        else k_msd_chunks<uint32_t, kMsdCap><<<grid, 256, 0, s>>>(a);
    }
    return cudaGetLastError();
}

cudaError_t msd_local(const MsdLocalArgs& a, int width, uint32_t nchunks, int match, cudaStream_t s, uint32_t cap) {
    if (nchunks == 0) return cudaSuccess;
    constexpr int WT = 2 * kLocalThreads;
    if (cap == kMsdWideCap) {
        if (width == 8) {
            if (match) LocalKernels<1>::w64<<<nchunks, WT, Wide64::SMEM, s>>>(a);
            else LocalKernels<0>::w64<<<nchunks, WT, Wide64::SMEM, s>>>(a);
        } else {
            if (match) LocalKernels<1>::w32<<<nchunks, WT, Wide32::SMEM, s>>>(a);
            else LocalKernels<0>::w32<<<nchunks, WT, Wide32::SMEM, s>>>(a);
        }
    } else if (width == 8) {
        if (match) LocalKernels<1>::k64<<<nchunks, kLocalThreads, Local64::SMEM, s>>>(a);
        else LocalKernels<0>::k64<<<nchunks, kLocalThreads, Local64::SMEM, s>>>(a);
    } else {
        if (match) LocalKernels<1>::k32<<<nchunks, kLocalThreads, Local32::SMEM, s>>>(a);
        else LocalKernels<0>::k32<<<nchunks, kLocalThreads, Local32::SMEM, s>>>(a);
    }
    return cudaGetLastError();
}

}  // namespace vdf
