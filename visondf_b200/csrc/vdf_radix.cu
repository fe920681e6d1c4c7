// vdf_radix.cu -- stable LSD radix argsort for sm_100a.
//
// Replaces the reference's radix_sort_uint{32,64}[_mt] family
// (V/inlines/radix_sorts/radix_sort_uint64_mt.inl:6-166: per-pass histogram,
// serial exclusive scan over 65,536 buckets, per-thread bucket offsets, stable
// scatter of (key, size_t idx), swap + memcpy) with a single-pass-per-digit
// ("onesweep") design:
//
//   1. k_digit_hist   one read of every key column computes the histograms of
//                     ALL digit positions at once (a histogram does not depend
//                     on row order, so the columns are read unpermuted).
//   2. k_hist_scan    exclusive scan per digit position -> global bin offsets.
//   3. k_onesweep     one launch per digit: each CTA ranks a tile of keys
//                     (warp match/ballot, per-warp shared-memory counters),
//                     publishes its per-bin counts early, resolves its global
//                     per-bin base with a decoupled look-back over earlier
//                     tiles, and scatters (key, u32 row id) through a
//                     shared-memory reorder buffer so global writes are runs.
//
// Key transforms (sign flip / IEEE image / descending inversion) are applied
// on the fly when a raw column is read, and undone when the last pass writes
// raw sorted keys; no transformed copy of a column is ever materialised.
// Multi-key sorts run least-significant key first; the first pass of each
// later key reads its raw column through the current permutation.
#include <algorithm>

#include "vdf_common.cuh"
#include "vdf_internal.h"

namespace vdf {

// ---------------------------------------------------------------------------
// 1. all-digit histogram
// ---------------------------------------------------------------------------
// Digit widths are per column (8 or 11 bits).  FIXED_BITS = 8 compiles the
// shifts and masks for plans whose keys all use 8-bit digits; 0 reads each
// column's width at run time.  The histograms of all passes sit back to back
// in shared memory.
template <int FIXED_BITS>
__global__ void __launch_bounds__(512) k_digit_hist(HistArgs a) {
    extern __shared__ uint32_t sh_hist[];  // [hist_words]
    if (a.run_flag && *a.run_flag != 1) return;  // conditional launch (the LSD fallback) not taken
    if (a.run_count && blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(a.run_count, 1u);
    for (int i = threadIdx.x; i < a.hist_words; i += blockDim.x) sh_hist[i] = 0;
    __syncthreads();

    const uint64_t n = a.n;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (int c = 0; c < a.ncols; ++c) {
        const HistCol col = a.col[c];
        uint32_t* h = sh_hist + col.hist_off;
        const int w = dtype_width(col.dtype);
        const uint32_t bits = FIXED_BITS ? (uint32_t)FIXED_BITS : (uint32_t)col.bits;
        const uint32_t radix = 1u << bits, mask = radix - 1;
        // four keys per thread per round, all loaded before any is used
        constexpr int R = 4;
        if (w == 4) {
            const uint32_t* src = static_cast<const uint32_t*>(col.data);
            for (uint64_t i0 = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i0 < n; i0 += R * stride) {
                uint32_t k[R];
#pragma unroll
                for (int r = 0; r < R; ++r) k[r] = i0 + r * stride < n ? ldg_stream(src + i0 + r * stride) : 0u;
#pragma unroll
                for (int r = 0; r < R; ++r) {
                    if (i0 + r * stride >= n) break;
                    const uint32_t x = order32(k[r], col.dtype, col.invert);
#pragma unroll 4
                    for (int p = 0; p < col.passes; ++p) atomicAdd(&h[p * radix + ((x >> (p * bits)) & mask)], 1u);
                }
            }
        } else {
            const uint64_t* src = static_cast<const uint64_t*>(col.data);
            for (uint64_t i0 = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i0 < n; i0 += R * stride) {
                uint64_t k[R];
#pragma unroll
                for (int r = 0; r < R; ++r) k[r] = i0 + r * stride < n ? ldg_stream(src + i0 + r * stride) : 0ull;
#pragma unroll
                for (int r = 0; r < R; ++r) {
                    if (i0 + r * stride >= n) break;
                    const uint64_t x = order64(k[r], col.dtype, col.invert);
#pragma unroll 8
                    for (int p = 0; p < col.passes; ++p)
                        atomicAdd(&h[p * radix + (uint32_t)((x >> (p * bits)) & mask)], 1u);
                }
            }
        }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < a.hist_words; i += blockDim.x) {
        uint32_t v = sh_hist[i];
        if (v) atomicAdd(&a.hist[i], v);
    }
}

// ---------------------------------------------------------------------------
// 2. exclusive scan of each digit position's histogram (one CTA per position)
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_hist_scan(ScanArgs a) {
    constexpr int PER = kMaxRadix / 256;
    __shared__ uint32_t warp_tot[8];
    if (a.run_flag && *a.run_flag != 1) return;  // conditional launch (the LSD fallback) not taken
    const uint32_t radix = a.radix[blockIdx.x];
    const uint32_t* h = a.hist + a.off[blockIdx.x];
    uint32_t* o = a.offs + a.off[blockIdx.x];
    uint32_t v[PER];
    uint32_t sum = 0;
#pragma unroll
    for (int j = 0; j < PER; ++j) {
        uint32_t b = threadIdx.x * PER + j;
        v[j] = b < radix ? h[b] : 0;
        sum += v[j];
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t incl = sum;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        uint32_t t = __shfl_up_sync(0xffffffffu, incl, d);
        if (lane >= d) incl += t;
    }
    if (lane == 31) warp_tot[warp] = incl;
    __syncthreads();
    uint32_t wbase = 0;
    for (int w = 0; w < warp; ++w) wbase += warp_tot[w];
    uint32_t run = wbase + incl - sum;
#pragma unroll
    for (int j = 0; j < PER; ++j) {
        uint32_t b = threadIdx.x * PER + j;
        if (b < radix) o[b] = run;
        run += v[j];
    }
}

// Segmented histograms: one CTA per chunk of one segment, all of that
// segment's passes at once (digits first_digit .. first_digit + passes - 1),
// flushed into the segment's own rows [seg][pass][radix] of the global
// histogram.  With seg_flag set, chunks of segments whose flag is clear
// return at once.
struct SegHistArgs {
    const void* keys;
    int key_width;
    const SegChunk* chunks;
    const SegDesc* segs;
    uint32_t* hist;
    uint32_t stride;   // words per segment
    uint32_t bits;
    uint32_t nsegs;
    uint64_t n;
    const uint32_t* seg_flag;
};
__global__ void __launch_bounds__(512) k_seg_hist(SegHistArgs a) {
    extern __shared__ uint32_t sh_hist[];
    const SegChunk ch = a.chunks[blockIdx.x];
    if (ch.seg >= a.nsegs || ch.row_start + ch.rows > a.n) return;  // host-built tables are consistent
    if (a.seg_flag && a.seg_flag[ch.seg] == 0) return;  // flag written by an earlier launch
    const uint32_t passes = a.segs[ch.seg].passes;
    const uint32_t shift0 = a.segs[ch.seg].first_digit * a.bits;
    const uint32_t radix = 1u << a.bits, mask = radix - 1;
    const uint32_t words = passes * radix;
    if (words > a.stride) return;
    for (uint32_t i = threadIdx.x; i < words; i += blockDim.x) sh_hist[i] = 0;
    __syncthreads();
    // four rows per thread per round, all loaded before any is counted
    constexpr int R = 4;
    const uint32_t step = blockDim.x;
    for (uint32_t r0 = threadIdx.x; r0 < ch.rows; r0 += R * step) {
        uint64_t k[R];
        if (a.key_width == 8) {
            const unsigned long long* src = static_cast<const unsigned long long*>(a.keys) + ch.row_start;
#pragma unroll
            for (int q = 0; q < R; ++q) k[q] = r0 + q * step < ch.rows ? ldg_stream(src + r0 + q * step) : 0ull;
        } else {
            const uint32_t* src = static_cast<const uint32_t*>(a.keys) + ch.row_start;
#pragma unroll
            for (int q = 0; q < R; ++q) k[q] = r0 + q * step < ch.rows ? (uint64_t)ldg_stream(src + r0 + q * step) : 0ull;
        }
#pragma unroll
        for (int q = 0; q < R; ++q) {
            if (r0 + q * step >= ch.rows) break;
            for (uint32_t p = 0; p < passes; ++p)
                atomicAdd(&sh_hist[p * radix + (uint32_t)((k[q] >> (shift0 + p * a.bits)) & mask)], 1u);
        }
    }
    __syncthreads();
    uint32_t* g = a.hist + (size_t)ch.seg * a.stride;
    for (uint32_t i = threadIdx.x; i < words; i += blockDim.x) {
        const uint32_t v = sh_hist[i];
        if (v) atomicAdd(&g[i], v);
    }
}

// Exclusive scan of consecutive rows of `radix` words, one CTA per row.
__global__ void __launch_bounds__(256) k_row_scan(const uint32_t* hist, uint32_t* offs, uint32_t radix) {
    constexpr int PER = kMaxRadix / 256;
    __shared__ uint32_t warp_tot[8];
    const uint32_t* h = hist + (size_t)blockIdx.x * radix;
    uint32_t* o = offs + (size_t)blockIdx.x * radix;
    uint32_t v[PER];
    uint32_t sum = 0;
#pragma unroll
    for (int j = 0; j < PER; ++j) {
        uint32_t b = threadIdx.x * PER + j;
        v[j] = b < radix ? h[b] : 0;
        sum += v[j];
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t incl = sum;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        uint32_t t = __shfl_up_sync(0xffffffffu, incl, d);
        if (lane >= d) incl += t;
    }
    if (lane == 31) warp_tot[warp] = incl;
    __syncthreads();
    uint32_t wbase = 0;
    for (int w = 0; w < warp; ++w) wbase += warp_tot[w];
    uint32_t run = wbase + incl - sum;
#pragma unroll
    for (int j = 0; j < PER; ++j) {
        uint32_t b = threadIdx.x * PER + j;
        if (b < radix) o[b] = run;
        run += v[j];
    }
}

// ---------------------------------------------------------------------------
// 3. onesweep pass
// ---------------------------------------------------------------------------
// Look-back status word: [31:30] flag, [29:0] count.  n < 2^30 is required.
constexpr uint32_t ST_AGG = 1u << 30;
constexpr uint32_t ST_INC = 2u << 30;
constexpr uint32_t ST_CNT = (1u << 30) - 1;

// Digit of a key at bit `shift`.  8-bit digits of 8-byte keys never straddle
// the two 32-bit halves, so the digit comes from the half that holds it.
template <typename K, int BITS>
__device__ __forceinline__ uint32_t digit_of(K key, uint32_t shift) {
    constexpr uint32_t MASK = (1u << BITS) - 1;
    if constexpr (sizeof(K) == 8 && BITS == 8) {
        const uint32_t w = (shift >= 32) ? (uint32_t)(key >> 32) : (uint32_t)key;
        return (w >> (shift & 31)) & MASK;
    } else {
        return (uint32_t)(key >> shift) & MASK;
    }
}

template <typename K, int BITS, int THREADS, int ITEMS, int MATCH = 0>
struct OnesweepCfg {
    static constexpr int RADIX = 1 << BITS;
    static constexpr int WARPS = THREADS / 32;
    static constexpr int TILE = THREADS * ITEMS;
    static constexpr int BPT = (RADIX + THREADS - 1) / THREADS;  // bins per thread
    // shared memory: keys | row ids | per-warp counters | bin bases | misc
    static constexpr size_t KEY_BYTES = (size_t)TILE * sizeof(K);
    static constexpr size_t VAL_BYTES = (size_t)TILE * 4;
    static constexpr size_t CNT_BYTES = (size_t)WARPS * RADIX * 4;
    static constexpr size_t GLOB_BYTES = (size_t)RADIX * 4;
    // match method 3: two per-warp words per digit, the lanes holding it
    static constexpr size_t MASK_BYTES = MATCH == 3 ? (size_t)2 * WARPS * RADIX * 4 : 0;
    static constexpr size_t SMEM = KEY_BYTES + VAL_BYTES + CNT_BYTES + GLOB_BYTES + 64 + WARPS * 4 + MASK_BYTES;
    // the bulk-load variant stages the next tile in a second key / row-id buffer
    static constexpr size_t SMEM_BULK = SMEM + KEY_BYTES + VAL_BYTES;
    static_assert(SMEM % 16 == 0 && KEY_BYTES % 16 == 0 && VAL_BYTES % 16 == 0, "bulk copies need 16-byte alignment");
};

// MATCH selects how a warp finds the lanes holding the same digit:
// 0 = one ballot per digit bit (ALU/vote pipes), 1 = match.any (XU pipe),
// 2 = alternate the two by item, so both pipes work at once, 3 = each lane
// ORs its bit into a per-warp shared-memory word of its digit and reads the
// word back (two words per digit, alternating by item, so a word is cleared
// well before it is used again).
// MINB: CTAs per SM the register allocation is sized for.
// SEG: segmented sort of many independent row ranges (the queries of a
// batch) in one launch.  Tiles never straddle a segment; a tile's bin bases
// come from its segment's own histogram, its look-back stops at the
// segment's first tile, and each segment has its own number of passes (the
// last one writes to the final buffers, later passes skip its tiles).
// Each CTA takes tile ids from the pass's counter until none is left, so a
// grid smaller than the tile count works (a conditional pass not taken then
// costs one short wave).  Tiles are taken in counter order, so the tile a
// look-back waits on always belongs to a running CTA.
// TMA: while a tile is ranked, one thread stages the next tile's keys and
// row ids into a second shared-memory buffer with a bulk copy behind an
// mbarrier (full, 16-byte aligned tiles; others load as usual); meant for a
// persistent grid of a few CTAs per SM.
// DICT: the dictionary pass of a one-key sort: a key's digit is its rank
// among the sort's distinct keys, looked up (open addressing) in a table
// staged in shared memory once per CTA.
__device__ __forceinline__ uint32_t dict_digit(const unsigned long long* lk, const uint32_t* lr, unsigned long long x) {
    uint32_t h = dict_hash(x) & (kDictLutSlots - 1);
    for (uint32_t probe = 0; probe < kDictLutSlots; ++probe) {
        const uint32_t r = lr[h];
        if (r == kDictEmpty) break;
        if (lk[h] == x) return r;
        h = (h + 1) & (kDictLutSlots - 1);
    }
    return 255;  // slots past the chunk: their all-ones keys rank last
}

template <typename K, int BITS, int THREADS, int ITEMS, int IN_MODE, bool FINAL, int MATCH, int MINB,
          bool SEG = false, bool TMA = false, bool DICT = false>
__global__ void __launch_bounds__(THREADS, MINB) k_onesweep(PassArgs a) {
    static_assert(!DICT || (BITS == 8 && !SEG && !TMA), "the dictionary pass is a plain 8-bit pass");
    using C = OnesweepCfg<K, BITS, THREADS, ITEMS, MATCH>;
    constexpr int RADIX = C::RADIX, WARPS = C::WARPS, TILE = C::TILE, BPT = C::BPT;
    constexpr bool BULK = TMA && !SEG;
    extern __shared__ __align__(16) unsigned char smem[];
    K* const kbuf0 = reinterpret_cast<K*>(smem);
    uint32_t* const vbuf0 = reinterpret_cast<uint32_t*>(smem + C::KEY_BYTES);
    uint32_t* wcnt = reinterpret_cast<uint32_t*>(smem + C::KEY_BYTES + C::VAL_BYTES);  // [WARPS][RADIX]
    uint32_t* bglob = wcnt + WARPS * RADIX;                                            // [RADIX]
    // misc: [2 + (it & 1)] the tile of iteration it, [4 + b] buffer b holds a
    // bulk-loaded tile, [8..11] the two buffers' mbarriers
    uint32_t* misc = bglob + RADIX;
    uint32_t* wsum = misc + 16;                                                        // [WARPS]
    uint32_t* wmask = wsum + WARPS;  // match method 3: [2][WARPS][RADIX]
    uint64_t* mbar = reinterpret_cast<uint64_t*>(misc + 8);
    K* const kbuf1 = reinterpret_cast<K*>(smem + C::SMEM);
    uint32_t* const vbuf1 = reinterpret_cast<uint32_t*>(smem + C::SMEM + C::KEY_BYTES);
    unsigned long long* const dlk = reinterpret_cast<unsigned long long*>(smem + C::SMEM);  // DICT: the table
    uint32_t* const dlr = reinterpret_cast<uint32_t*>(smem + C::SMEM + kDictLutSlots * 8);
    uint8_t* const ex_dig = smem + C::SMEM + sizeof(DictLut);  // DICT: digits beside the exchanged keys

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    // A conditional pass not taken returns before touching anything; the
    // flag was written by an earlier launch, so every thread reads the same.
    if (a.run_flag && *a.run_flag != a.run_when) return;
    if constexpr (DICT) {  // the lookup table, used after the first barrier below
        for (uint32_t i = threadIdx.x; i < kDictLutSlots; i += THREADS) {
            dlk[i] = a.dict_lut->key[i];
            dlr[i] = a.dict_lut->rank[i];
        }
    }
    const uint32_t ntiles = a.ntiles ? a.ntiles : gridDim.x;
    const uint32_t spin_limit = a.spin_limit ? a.spin_limit : kSpinLimit;
    const uint64_t n = a.n;
    // bulk loads (thread 0): the keys (unless read through the permutation)
    // and row ids (unless the rows themselves) of a full, aligned tile t
    constexpr bool LOAD_K = IN_MODE != IN_GATHER, LOAD_V = IN_MODE != IN_RAW;
    auto issue = [&](uint32_t t, int b) {
        bool ok = false;
        if (t < ntiles && (uint64_t)(t + 1) * TILE <= n) {
            const K* ks = LOAD_K ? static_cast<const K*>(a.keys_in) + (uint64_t)t * TILE : nullptr;
            const uint32_t* vs = LOAD_V ? a.vals_in + (uint64_t)t * TILE : nullptr;
            ok = (!LOAD_K || (reinterpret_cast<uintptr_t>(ks) & 15) == 0) &&
                 (!LOAD_V || (reinterpret_cast<uintptr_t>(vs) & 15) == 0);
            if (ok) {
                fence_async_smem();  // the buffer's earlier reads come first
                mbar_expect(&mbar[b], (LOAD_K ? (uint32_t)C::KEY_BYTES : 0u) + (LOAD_V ? (uint32_t)C::VAL_BYTES : 0u));
                if (LOAD_K) bulk_load(b ? kbuf1 : kbuf0, ks, (uint32_t)C::KEY_BYTES, &mbar[b]);
                if (LOAD_V) bulk_load(b ? vbuf1 : vbuf0, vs, (uint32_t)C::VAL_BYTES, &mbar[b]);
            }
        }
        misc[4 + b] = ok ? 1u : 0u;
    };
    if (tid == 0) {
        if constexpr (BULK) {
            mbar_init(&mbar[0], 1);
            mbar_init(&mbar[1], 1);
            mbar_init_fence();
        }
        misc[2] = atomicAdd(a.tile_counter, 1u);
        if constexpr (BULK) issue(misc[2], 0);
    }
    uint32_t phase = 0;  // bit b: parity of buffer b's next completed load
    uint32_t lost = 0;   // bit b: a load into buffer b that a wait gave up on
    for (uint32_t it = 0;; ++it) {
        const int cb = BULK ? (int)(it & 1) : 0;  // this tile's buffer
        K* const ex_keys = cb ? kbuf1 : kbuf0;
        uint32_t* const ex_vals = cb ? vbuf1 : vbuf0;
        uint32_t* const next_slot = misc + 2 + ((it + 1) & 1);
        // this thread's accesses to the buffers come before the bulk copies
        // into them that follow the barrier below
        if constexpr (BULK) fence_async_smem();
        for (int i = tid; i < WARPS * RADIX; i += THREADS) wcnt[i] = 0;
        if constexpr (MATCH == 3)
            for (int i = tid; i < 2 * WARPS * RADIX; i += THREADS) wmask[i] = 0;
        __syncthreads();
        const uint32_t tile = misc[2 + (it & 1)];
        if (tile >= ntiles) break;
        const bool bulk = BULK && misc[4 + cb] != 0;
        if constexpr (BULK) {
            if (tid == 0) {  // the next tile, so that its load overlaps this one
                *next_slot = atomicAdd(a.tile_counter, 1u);
                issue(*next_slot, cb ^ 1);
            }
            if (bulk) {
                if (!mbar_wait(&mbar[cb], (phase >> cb) & 1u, spin_limit)) {
                    lost |= 1u << cb;
                    if (tid == 0) atomicOr(a.err, ERR_LOOKBACK_TIMEOUT);
                }
                phase ^= 1u << cb;
            }
        }
        // failure injection for tests: this tile publishes nothing, so the
        // look-back waits on it run out (bounded, reported)
        if (tile == a.stall_tile) {
            if (!BULK && tid == 0) *next_slot = atomicAdd(a.tile_counter, 1u);
            continue;
        }
        uint64_t tile_base = (uint64_t)tile * TILE;
        uint32_t valid = (uint32_t)min((uint64_t)TILE, n - tile_base);
        uint32_t first_tile = 0;   // look-back stops here
        uint32_t seg = 0;
        uint32_t shift = a.shift;
        bool fin = FINAL;
        if constexpr (SEG) {
            valid = 0;
            if (tile < a.status_rows) {
                seg = a.tile_seg[tile];
                const SegDesc sd = a.segs[seg];
                // a segment left out by its flag (written by an earlier launch,
                // so every tile of the segment sees the same) only clears status
                const bool skip = a.seg_flag && ((a.seg_flag[seg] != 0) != (a.seg_flag_when != 0));
                if (tile < sd.first_tile || sd.row_start + sd.rows > n ||
                    (uint64_t)(tile - sd.first_tile) * TILE >= sd.rows) {
                    if (tid == 0) atomicOr(a.err, ERR_BAD_INDEX);  // inconsistent tile table
                } else if (a.pass < sd.passes && !skip) {
                    first_tile = sd.first_tile;
                    shift = (sd.first_digit + a.pass) * BITS;
                    tile_base = sd.row_start + (uint64_t)(tile - sd.first_tile) * TILE;
                    valid = (uint32_t)min((uint64_t)TILE, sd.row_start + sd.rows - tile_base);
                    fin = (a.pass + 1 == sd.passes);
                }
            } else if (tid == 0) {
                atomicOr(a.err, ERR_BAD_INDEX);
            }
        }

        // ---- load keys and row ids (warp-striped: item j of lane l is tile
        //      position warp*ITEMS*32 + j*32 + l, so positions follow row order) --
        // Every load of the tile is issued before any key is transformed (a
        // transform between loads keeps the compiler from overlapping them).
        K key[ITEMS];
        uint32_t val[ITEMS];
        const uint32_t wpos = (uint32_t)warp * ITEMS * 32;
        if (bulk) {  // a full tile, staged in shared memory
    #pragma unroll
            for (int j = 0; j < ITEMS; ++j) {
                const uint32_t pos = wpos + j * 32 + lane;
                key[j] = LOAD_K ? ex_keys[pos] : ~K(0);
                val[j] = LOAD_V ? ex_vals[pos] : (uint32_t)(tile_base + pos);
                if (IN_MODE == IN_GATHER && val[j] >= n) {  // never for a valid permutation
                    atomicOr(a.err, ERR_BAD_INDEX);
                    val[j] = 0;
                }
            }
        } else
    #pragma unroll
        for (int j = 0; j < ITEMS; ++j) {
            const uint32_t pos = wpos + j * 32 + lane;
            const uint64_t i = tile_base + pos;
            key[j] = ~K(0);
            val[j] = (uint32_t)i;  // IN_RAW: the row itself
            if (pos < valid) {
                if (IN_MODE == IN_RAW) {
                    key[j] = ldg_stream(static_cast<const K*>(a.keys_in) + i);
                } else if (IN_MODE == IN_GATHER) {
                    uint32_t src = ldg_stream(a.vals_in + i);
                    if (src >= n) {  // never for a valid permutation
                        atomicOr(a.err, ERR_BAD_INDEX);
                        src = 0;
                    }
                    val[j] = src;
                } else {
                    key[j] = ldg_stream(static_cast<const K*>(a.keys_in) + i);
                    val[j] = ldg_stream(a.vals_in + i);
                }
            }
        }
        if constexpr (IN_MODE == IN_GATHER) {
            // keys through the current permutation: all random loads, then the transform
    #pragma unroll
            for (int j = 0; j < ITEMS; ++j) {
                if (wpos + j * 32 + lane < valid) {
                    const K* kp = static_cast<const K*>(a.keys_in) + val[j];
                    if constexpr (sizeof(K) == 8) key[j] = ld_rand8(kp);
                    else key[j] = ld_rand4(kp);
                }
            }
        }
        if constexpr ((IN_MODE == IN_RAW && !SEG) || IN_MODE == IN_GATHER) {
            // raw keys -> order images (a batch arena already holds images)
    #pragma unroll
            for (int j = 0; j < ITEMS; ++j)
                if (wpos + j * 32 + lane < valid) key[j] = KeyOps<K>::order(key[j], a.dtype, a.invert);
        }

        // Clear this tile's row of the other status buffer for the next pass
        // (that buffer's previous user, the pass before this one, has finished).
        // Rows tile, tile + gridDim.x, ... so that every row a later pass with
        // more tiles could read is cleared too.
        if (a.status_next) {
            if (a.status_row_words == RADIX) {  // every pass of the plan has this radix
                for (uint32_t r = tile; r < a.status_rows; r += ntiles)
                    for (int b = tid; b < RADIX; b += THREADS) a.status_next[(size_t)r * RADIX + b] = 0;
            } else {
                for (uint32_t r = tile; r < a.status_rows; r += ntiles)
                    for (uint32_t b = tid; b < a.status_row_words; b += THREADS)
                        a.status_next[(size_t)r * a.status_row_words + b] = 0;
            }
        }
        if (SEG && valid == 0) {  // segment finished in an earlier pass, or left out
            if (!BULK && tid == 0) *next_slot = atomicAdd(a.tile_counter, 1u);
            continue;
        }

        // ---- warp-local ranks and per-warp digit counts --------------------------
        // First the lanes holding the same digit are found for every item (one
        // ballot per digit bit, or match.any); these are independent and
        // overlap.  Then the warp's per-digit counters advance item by item (the
        // lowest lane of each peer group adds the group's size), which is the
        // only serial part.  Slots past the end of the last tile hold all-ones
        // keys, whose digit is the largest in every pass: ranked like any key,
        // they come after every real key of that digit (their positions are
        // last), so they fill the tile's last slots and are never written out.
        uint32_t rank[ITEMS];
        uint32_t peers[ITEMS];
        uint32_t* my_cnt = wcnt + warp * RADIX;
        const uint32_t lt = lanemask_lt();
        // 8-bit digits are computed once and kept four to a register
        constexpr bool PACKED = (BITS == 8);
        uint32_t dpk[(ITEMS + 3) / 4];
    #pragma unroll
        for (int i = 0; i < (ITEMS + 3) / 4; ++i) dpk[i] = 0;
        auto digit = [&](int j) -> uint32_t {
            if constexpr (PACKED) return (dpk[j / 4] >> (8 * (j % 4))) & 0xffu;
            else if constexpr (DICT) return dict_digit(dlk, dlr, (unsigned long long)key[j]);
            else return digit_of<K, BITS>(key[j], shift);
        };
    #pragma unroll
        for (int j = 0; j < ITEMS; ++j) {
            uint32_t d;
            if constexpr (DICT) d = dict_digit(dlk, dlr, (unsigned long long)key[j]);
            else d = digit_of<K, BITS>(key[j], shift);
            if constexpr (PACKED) dpk[j / 4] |= d << (8 * (j % 4));
            if constexpr (MATCH == 3) {
                uint32_t* word = wmask + ((j & 1) * WARPS + warp) * RADIX + d;
                atomicOr(word, 1u << lane);
                __syncwarp();
                const uint32_t pm = *word;
                __syncwarp();  // every peer has read the word before its leader clears it
                if (lane == __ffs(pm) - 1) *word = 0;
                peers[j] = pm;
            } else if (MATCH == 1 || (MATCH == 2 && (j & 1) == 0)) {
                peers[j] = __match_any_sync(0xffffffffu, d);
            } else {
                uint32_t pm = 0xffffffffu;
    #pragma unroll
                for (int b = 0; b < BITS; ++b) {
                    const uint32_t bal = __ballot_sync(0xffffffffu, (d >> b) & 1u);
                    pm &= ((d >> b) & 1u) ? bal : ~bal;
                }
                peers[j] = pm;
            }
        }
        // The leader's add returns before the full-warp shuffle that hands its
        // result out, and the next item's add comes after that shuffle, so the
        // items' adds on a counter happen in item order (stable ranks).
    #pragma unroll
        for (int j = 0; j < ITEMS; ++j) {
            const uint32_t d = digit(j);
            const int leader = __ffs(peers[j]) - 1;
            uint32_t base = 0;
            if (lane == leader) base = atomicAdd(&my_cnt[d], (uint32_t)__popc(peers[j]));
            base = __shfl_sync(0xffffffffu, base, leader);
            rank[j] = base + __popc(peers[j] & lt);
        }
        __syncthreads();

        // ---- per-bin totals, early publish, tile-local bin starts --------------
        uint32_t tot[BPT];
        uint32_t tsum = 0;
    #pragma unroll
        for (int k = 0; k < BPT; ++k) {
            const int b = tid * BPT + k;
            uint32_t run = 0;
            if (b < RADIX) {
    #pragma unroll
                for (int w = 0; w < WARPS; ++w) {
                    uint32_t c = wcnt[w * RADIX + b];
                    wcnt[w * RADIX + b] = run;
                    run += c;
                }
                uint32_t* st = a.status + (size_t)tile * RADIX + b;
                st_relaxed_u32(st, (tile == first_tile ? ST_INC : ST_AGG) | run);
            }
            tot[k] = run;
            tsum += run;
        }
        // block exclusive scan of tsum over threads (bins are blocked per thread)
        uint32_t incl = tsum;
    #pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            uint32_t t = __shfl_up_sync(0xffffffffu, incl, d);
            if (lane >= d) incl += t;
        }
        if (lane == 31) wsum[warp] = incl;
        __syncthreads();
        uint32_t wb = 0;
    #pragma unroll
        for (int w = 0; w < WARPS; ++w) wb += (w < warp) ? wsum[w] : 0u;
        uint32_t bstart[BPT];
        {
            uint32_t run = wb + incl - tsum;
    #pragma unroll
            for (int k = 0; k < BPT; ++k) {
                bstart[k] = run;
                run += tot[k];
                const int b = tid * BPT + k;
                if (b < RADIX)
    #pragma unroll
                    for (int w = 0; w < WARPS; ++w) wcnt[w * RADIX + b] += bstart[k];
            }
        }
        __syncthreads();

        // ---- tile-local ranks; keys and row ids into shared memory --------------
        // (overlaps the look-back below: other warps' global writes wait on it)
    #pragma unroll
        for (int j = 0; j < ITEMS; ++j) {
            const uint32_t d = digit(j);
            uint32_t r = rank[j] + wcnt[warp * RADIX + d];
            if (r >= (uint32_t)TILE) {  // never when the counts are consistent
                atomicOr(a.err, ERR_BAD_INDEX);
                r = wpos + j * 32 + lane;
            }
            ex_keys[r] = key[j];
            ex_vals[r] = val[j];
            if constexpr (DICT) ex_dig[r] = (uint8_t)d;  // spares a second table lookup
        }

        // ---- decoupled look-back per bin ---------------------------------------
        // Each bin's thread reads the status words of LB predecessors at once (one
        // round trip per window), adds counts from the nearest one backwards and
        // stops at the first inclusive prefix.  A thread owning several bins (wide
        // digits) issues the windows of all its unfinished bins together.
        const int64_t lo = first_tile;
        if constexpr (BPT == 1) {
            constexpr int LB = 8;
            const int b = tid;
            if (b < RADIX) {
                uint32_t excl = 0;
                if (tile > first_tile) {
                    int64_t p = (int64_t)tile - 1;
                    uint32_t spins = 0;
                    bool done = false;
                    while (!done) {
                        uint32_t sw[LB];
    #pragma unroll
                        for (int w = 0; w < LB; ++w)
                            sw[w] = (p - w >= lo) ? ld_relaxed_u32(a.status + (size_t)(p - w) * RADIX + b) : ST_INC;
    #pragma unroll
                        for (int w = 0; w < LB; ++w) {
                            if (done) break;
                            uint32_t st = sw[w];
                            while ((st & ~ST_CNT) == 0) {  // not yet published: wait for this one
                                if (++spins > spin_limit) {
                                    atomicOr(a.err, ERR_LOOKBACK_TIMEOUT);
                                    st = ST_INC;
                                    break;
                                }
                                backoff(spins);
                                st = ld_relaxed_u32(a.status + (size_t)(p - w) * RADIX + b);
                            }
                            excl += st & ST_CNT;
                            if (st & ST_INC) done = true;
                        }
                        p -= LB;
                        if (p < lo) done = true;
                    }
                    st_relaxed_u32(a.status + (size_t)tile * RADIX + b, ST_INC | (excl + tot[0]));
                }
                uint32_t base;
                if constexpr (SEG)
                    base = (uint32_t)a.segs[seg].row_start + a.seg_offs[(size_t)seg * a.seg_stride + a.pass * RADIX + b];
                else
                    base = a.bin_offsets[b];
                bglob[b] = base + excl - bstart[0];
            }
        } else {
            constexpr int LB = (BPT >= 8) ? 2 : 4;
            uint32_t excl[BPT];
            bool done[BPT];
    #pragma unroll
            for (int k = 0; k < BPT; ++k) {
                excl[k] = 0;
                done[k] = (tile == first_tile) || (tid * BPT + k >= RADIX);
            }
            int64_t p = (int64_t)tile - 1;
            uint32_t spins = 0;
            bool all_done = false;
            while (!all_done) {
                uint32_t sw[BPT][LB];
    #pragma unroll
                for (int k = 0; k < BPT; ++k)
    #pragma unroll
                    for (int w = 0; w < LB; ++w)
                        sw[k][w] = (!done[k] && p - w >= lo)
                                       ? ld_relaxed_u32(a.status + (size_t)(p - w) * RADIX + tid * BPT + k)
                                       : ST_INC;
                all_done = true;
    #pragma unroll
                for (int k = 0; k < BPT; ++k) {
                    if (done[k]) continue;
    #pragma unroll
                    for (int w = 0; w < LB; ++w) {
                        if (done[k]) break;
                        uint32_t st = sw[k][w];
                        while ((st & ~ST_CNT) == 0) {  // not yet published: wait for this one
                            if (++spins > spin_limit) {
                                atomicOr(a.err, ERR_LOOKBACK_TIMEOUT);
                                st = ST_INC;
                                break;
                            }
                            backoff(spins);
                            st = ld_relaxed_u32(a.status + (size_t)(p - w) * RADIX + tid * BPT + k);
                        }
                        excl[k] += st & ST_CNT;
                        if (st & ST_INC) done[k] = true;
                    }
                    if (p - LB < lo) done[k] = true;
                    all_done = all_done && done[k];
                }
                p -= LB;
            }
    #pragma unroll
            for (int k = 0; k < BPT; ++k) {
                const int b = tid * BPT + k;
                if (b >= RADIX) break;
                if (tile > first_tile) st_relaxed_u32(a.status + (size_t)tile * RADIX + b, ST_INC | (excl[k] + tot[k]));
                uint32_t base;
                if constexpr (SEG)
                    base = (uint32_t)a.segs[seg].row_start + a.seg_offs[(size_t)seg * a.seg_stride + a.pass * RADIX + b];
                else
                    base = a.bin_offsets[b];
                bglob[b] = base + excl[k] - bstart[k];
            }
        }
        __syncthreads();

        // ---- run-coalesced writes of keys and row ids ----------------------------
        K* kout = static_cast<K*>((SEG && fin) ? a.keys_final : a.keys_out);
        uint32_t* vout = (SEG && fin) ? a.vals_final : a.vals_out;
    #pragma unroll
        for (int r = 0; r < ITEMS; ++r) {
            const uint32_t i = r * THREADS + tid;
            if (i < valid) {
                const K k = ex_keys[i];
                const uint32_t v = ex_vals[i];
                uint32_t d;
                if constexpr (DICT) d = ex_dig[i];
                else d = digit_of<K, BITS>(k, shift);
                uint32_t p = bglob[d] + i;
                if (p >= n) {  // only after a look-back timeout: never write out of bounds
                    atomicOr(a.err, ERR_BAD_INDEX);
                    continue;
                }
                if constexpr (SEG) {
                    // a batch arena holds order images sorted ascending: the final
                    // pass differs from the others only in its output buffers
                    stg_stream(kout + p, k);
                } else {
                    if (fin && a.reverse) p = (uint32_t)(n - 1) - p;
                    if (fin) {
                        if (kout) stg_stream(kout + p, KeyOps<K>::unorder(k, a.dtype, a.invert));
                    } else {
                        stg_stream(kout + p, k);
                    }
                }
                stg_stream(vout + p, v);
            }
        }
        if (!BULK && tid == 0) *next_slot = atomicAdd(a.tile_counter, 1u);
    }  // tiles
    if constexpr (BULK) {
        // a load a wait gave up on must land before the CTA's shared memory
        // is handed on (bounded again; an error is already recorded)
        for (int b = 0; b < 2; ++b)
            if (lost & (1u << b)) mbar_wait(&mbar[b], ((phase >> b) & 1u) ^ 1u, spin_limit);
    }
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
namespace {
using PassKernel = void (*)(PassArgs);

// One compiled configuration of the radix pass.  The variant table is the
// autotuner's search space; a context selects one variant per key width.
// tma: tiles staged by bulk copies, on a persistent grid of `resident` CTAs
// per SM (found with the occupancy calculator when the kernels are prepared).
struct PassVariant {
    int width, threads, items, bits, match, minb, tma;
    size_t smem;
    PassKernel k[3][2];  // [IN_MODE][FINAL]
};

template <typename K, int BITS, int THREADS, int ITEMS, int MATCH, int MINB, bool TMA = false>
PassVariant make_variant() {
    using C = OnesweepCfg<K, BITS, THREADS, ITEMS, MATCH>;
    static_assert(BITS <= kMaxBits, "digit wider than the histogram layout allows");
    PassVariant v{};
    v.width = (int)sizeof(K);
    v.threads = THREADS;
    v.items = ITEMS;
    v.bits = BITS;
    v.match = MATCH;
    v.minb = MINB;
    v.tma = TMA ? 1 : 0;
    v.smem = TMA ? C::SMEM_BULK : C::SMEM;
    v.k[IN_RAW][0] = k_onesweep<K, BITS, THREADS, ITEMS, IN_RAW, false, MATCH, MINB, false, TMA>;
    v.k[IN_GATHER][0] = k_onesweep<K, BITS, THREADS, ITEMS, IN_GATHER, false, MATCH, MINB, false, TMA>;
    v.k[IN_BUF][0] = k_onesweep<K, BITS, THREADS, ITEMS, IN_BUF, false, MATCH, MINB, false, TMA>;
    v.k[IN_RAW][1] = k_onesweep<K, BITS, THREADS, ITEMS, IN_RAW, true, MATCH, MINB, false, TMA>;
    v.k[IN_GATHER][1] = k_onesweep<K, BITS, THREADS, ITEMS, IN_GATHER, true, MATCH, MINB, false, TMA>;
    v.k[IN_BUF][1] = k_onesweep<K, BITS, THREADS, ITEMS, IN_BUF, true, MATCH, MINB, false, TMA>;
    return v;
}

// key type, digit bits, threads per CTA, keys per thread, match method, CTAs per SM
const PassVariant kVariants[] = {
    make_variant<uint32_t, 8, 256, 16, 0, 3>(),  // 0
    make_variant<uint32_t, 8, 256, 16, 1, 3>(),  // 1
    make_variant<uint64_t, 8, 256, 12, 0, 3>(),  // 2
    make_variant<uint64_t, 8, 256, 12, 1, 3>(),  // 3
    make_variant<uint32_t, 8, 256, 16, 1, 2>(),  // 4
    make_variant<uint64_t, 8, 256, 12, 0, 2>(),  // 5
    make_variant<uint32_t, 8, 256, 12, 1, 4>(),  // 6
    make_variant<uint64_t, 8, 256, 8, 0, 4>(),   // 7
    make_variant<uint64_t, 8, 256, 16, 0, 2>(),  // 8
    make_variant<uint32_t, 8, 256, 24, 1, 2>(),  // 9
    make_variant<uint32_t, 8, 256, 12, 2, 4>(),  // 10
    make_variant<uint64_t, 8, 256, 12, 2, 3>(),  // 11
    make_variant<uint64_t, 8, 256, 8, 2, 4>(),   // 12
    make_variant<uint32_t, 8, 256, 16, 2, 3>(),  // 13
    // 11-bit digits: 3 passes for a 4-byte key, 6 for an 8-byte key
    make_variant<uint32_t, 11, 256, 16, 1, 2>(),  // 14
    make_variant<uint64_t, 11, 256, 8, 1, 2>(),   // 15
    make_variant<uint32_t, 11, 256, 16, 2, 2>(),  // 16
    make_variant<uint64_t, 11, 256, 12, 2, 2>(),  // 17
    // digit match through shared-memory words (match method 3); its cost
    // grows when many lanes share a digit, so it is the autotuner's pick for
    // a workload rather than the default
    make_variant<uint64_t, 8, 256, 12, 3, 3>(),   // 18
    // tiles staged in shared memory by bulk copies, the next tile's copy
    // overlapping the current tile's ranking (persistent grid)
    make_variant<uint64_t, 8, 256, 12, 0, 2, true>(),  // 19
    make_variant<uint64_t, 8, 256, 12, 2, 2, true>(),  // 20
    make_variant<uint32_t, 8, 256, 16, 1, 2, true>(),  // 21
    make_variant<uint32_t, 8, 256, 16, 2, 2, true>(),  // 22
};
constexpr int kNumVariants = (int)(sizeof(kVariants) / sizeof(kVariants[0]));
// resident CTAs per SM of each variant's kernels (the fewest over its six)
int g_resident[kNumVariants];
int g_seg_resident[16][2];
int g_sms = 0;

// Grid of a radix pass over `tiles` tiles: one CTA per tile, or (persistent:
// bulk-load variants, and conditional passes, which usually return at once)
// as many CTAs as fit on the GPU, each looping over tiles.
uint32_t pass_grid(uint32_t tiles, int resident, bool persistent) {
    if (!persistent || g_sms <= 0 || resident <= 0) return tiles;
    return (uint32_t)std::min<uint64_t>(tiles, (uint64_t)g_sms * (uint64_t)resident);
}

// Segmented sorts run over ordered key images of 8 or 4 bytes; k[w][m]: w = 1
// for 8-byte images, m = 0 for the first pass (arena rows), 1 for later
// passes (ping-pong buffers).  Both widths of a variant share its digit width
// and tile.
struct SegVariant {
    int bits, tile;
    size_t smem[2];
    PassKernel k[2][2];
};
template <int BITS, int THREADS, int ITEMS, int MATCH, int MINB>
SegVariant make_seg_variant() {
    using C4 = OnesweepCfg<uint32_t, BITS, THREADS, ITEMS, MATCH>;
    using C8 = OnesweepCfg<uint64_t, BITS, THREADS, ITEMS, MATCH>;
    SegVariant v{};
    v.bits = BITS;
    v.tile = THREADS * ITEMS;
    v.smem[0] = C4::SMEM;
    v.smem[1] = C8::SMEM;
    v.k[0][0] = k_onesweep<uint32_t, BITS, THREADS, ITEMS, IN_RAW, false, MATCH, MINB, true>;
    v.k[0][1] = k_onesweep<uint32_t, BITS, THREADS, ITEMS, IN_BUF, false, MATCH, MINB, true>;
    v.k[1][0] = k_onesweep<uint64_t, BITS, THREADS, ITEMS, IN_RAW, false, MATCH, MINB, true>;
    v.k[1][1] = k_onesweep<uint64_t, BITS, THREADS, ITEMS, IN_BUF, false, MATCH, MINB, true>;
    return v;
}
const SegVariant kSegVariants[] = {
    make_seg_variant<8, 256, 8, 2, 4>(),    // 0
    make_seg_variant<8, 256, 12, 2, 2>(),   // 1
    make_seg_variant<8, 256, 16, 0, 2>(),   // 2
    make_seg_variant<11, 256, 8, 1, 2>(),   // 3
    make_seg_variant<8, 256, 12, 2, 4>(),   // 4
};
constexpr int kNumSegVariants = (int)(sizeof(kSegVariants) / sizeof(kSegVariants[0]));

// Dictionary-pass kernels (one final 8-bit pass over each key's rank), for
// 4- and 8-byte keys; k[0] reads the raw column, k[1] the keys through the
// input permutation.
struct DictVariant {
    int width, threads, items;
    size_t smem;
    PassKernel k[2];
};
template <typename K, int THREADS, int ITEMS, int MATCH, int MINB>
DictVariant make_dict_variant() {
    using C = OnesweepCfg<K, 8, THREADS, ITEMS, MATCH>;
    DictVariant v{};
    v.width = (int)sizeof(K);
    v.threads = THREADS;
    v.items = ITEMS;
    v.smem = C::SMEM + sizeof(DictLut) + (size_t)C::TILE;
    v.k[0] = k_onesweep<K, 8, THREADS, ITEMS, IN_RAW, true, MATCH, MINB, false, false, true>;
    v.k[1] = k_onesweep<K, 8, THREADS, ITEMS, IN_GATHER, true, MATCH, MINB, false, false, true>;
    return v;
}
const DictVariant kDictVariants[] = {
    make_dict_variant<uint32_t, 256, 16, 1, 3>(),  // 0: 4-byte keys
    make_dict_variant<uint64_t, 256, 12, 1, 3>(),  // 1: 8-byte keys
};
int g_dict_resident[2];

const PassVariant& variant_for(const SortTuning& t, int width) {
    const int v = (width == 4) ? t.variant32 : t.variant64;
    return kVariants[v];
}
int resident_of(const PassVariant& v) { return g_resident[&v - kVariants]; }

inline size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }
}  // namespace

int sort_variant_count() { return kNumVariants; }

bool sort_variant_uses_tma(int i) { return i >= 0 && i < kNumVariants && kVariants[i].tma != 0; }

bool sort_variant_info(int i, int* width, int* threads, int* items, int* bits, int* match) {
    if (i < 0 || i >= kNumVariants) return false;
    const PassVariant& v = kVariants[i];
    *width = v.width;
    *threads = v.threads;
    *items = v.items;
    *bits = v.bits;
    *match = v.match;
    return true;
}

bool sort_tuning_valid(const SortTuning& t) {
    return t.variant32 >= 0 && t.variant32 < kNumVariants && kVariants[t.variant32].width == 4 &&
           t.variant64 >= 0 && t.variant64 < kNumVariants && kVariants[t.variant64].width == 8;
}

SortTuning default_sort_tuning() {
    SortTuning t{1, 2, 1, kMsdDefaultMinRows};
    t.dict = 1;
    return t;
}

static int tile_rows(const SortTuning& t, int width) {
    const PassVariant& v = variant_for(t, width);
    return v.threads * v.items;
}

// Global MSD passes for n rows: the fewest top digits after which a bucket
// averages at most bucket_rows rows (kMsdBucketRows for chunks of nominal
// kMsdCap / 2 rows, twice that for wide chunks), so that a chunk of whole
// buckets stays within its capacity for uniformly spread keys (the average
// bucket plus six standard deviations).
int msd_passes_for(uint64_t n, int width, uint32_t bucket_rows) {
    const int maxp = std::min(kMsdMaxPasses, width - 1);
    for (int p = 1; p <= maxp; ++p)
        if (n <= (uint64_t)bucket_rows << (8 * p)) return p;
    return 0;
}

SortPlan make_sort_plan(uint64_t n, const int32_t* dtypes, int nkeys, const SortTuning& tuning) {
    SortPlan p{};
    p.n = n;
    p.nkeys = nkeys;
    p.tuning = tuning;
    int maxw = 4;
    uint32_t max_tiles = 0;
    p.max_radix = 0;
    for (int k = 0; k < nkeys; ++k) {
        p.dtype[k] = dtypes[k];
        p.width[k] = dtype_width(dtypes[k]);
        p.bits[k] = variant_for(tuning, p.width[k]).bits;
        p.radix[k] = 1 << p.bits[k];
        p.passes[k] = (p.width[k] * 8 + p.bits[k] - 1) / p.bits[k];
        if (p.width[k] > maxw) maxw = p.width[k];
        if (p.radix[k] > p.max_radix) p.max_radix = p.radix[k];
        const int rows = tile_rows(tuning, p.width[k]);
        uint32_t t = (uint32_t)((n + rows - 1) / rows);
        if (t > max_tiles) max_tiles = t;
    }
    // MSD-first for one or two keys when the key-0 passes use 8-bit digits
    if (tuning.msd && nkeys <= 2 && n >= 2 && n >= tuning.msd_min_rows && p.bits[0] == 8 &&
        (tuning.msd == 2 || p.width[0] == 8)) {
        p.msd_passes = msd_passes_for(n, p.width[0]);
        p.msd_cap = kMsdCap;
        // wide chunks where they save the third top-digit pass (100.7M-201M
        // rows: two digits instead of three; measured 0.3 ms faster on 200M
        // rows, the finish of twice the rows per CTA costing most of the pass
        // it saves)
        const int wide = msd_passes_for(n, p.width[0], 2 * kMsdBucketRows);
        if (wide > 0 && ((wide < p.msd_passes && p.msd_passes == 3) || (tuning.msd_match & 2))) {  // bit 1: always
            p.msd_passes = wide;
            p.msd_cap = kMsdWideCap;
        }
        p.msd = p.msd_passes > 0;
        // low bits ranked directly in runs of equal high bits: the low half of
        // an 8-byte key (such runs are rare for spread keys, and ranking
        // every row of frequent short runs measured slower than the shared-
        // memory passes it saves); none for 4-byte keys
        p.msd_lo_bits = p.width[0] == 8 ? 32 : 0;
    }
    // dictionary plan for one key (tried first; the device decides), from
    // four times the MSD-first plan's row threshold: where the keys take
    // many values the attempt costs a few short launches, which at 1M-4M
    // rows is several percent of the sort
    if (tuning.dict && nkeys == 1 && n >= 2 && n >= 4 * tuning.msd_min_rows) {
        p.dict = true;
        p.dict_variant = p.width[0] == 8 ? 1 : 0;
        const DictVariant& dv = kDictVariants[p.dict_variant];
        const uint32_t rows = (uint32_t)(dv.threads * dv.items);
        p.dict_tiles = (uint32_t)((n + rows - 1) / rows);
        if (p.dict_tiles > max_tiles) max_tiles = p.dict_tiles;
    }
    // passes are numbered in processing order (least-significant key first);
    // their histograms follow one another in that order
    int total = 0, words = 0;
    for (int k = nkeys - 1; k >= 0; --k) {
        p.pass_base[k] = total;
        p.hist_off[k] = words;
        total += p.passes[k];
        words += p.passes[k] * p.radix[k];
    }
    p.total_passes = total;
    p.hist_words = words;
    p.max_tiles = max_tiles;
    size_t off = 0;
    const size_t A = 256;
    const size_t status_bytes = (size_t)max_tiles * p.max_radix * 4;
    const int msd_p = p.msd ? p.msd_passes : 0;
    p.off_keys[0] = off; off = align_up(off + n * (size_t)maxw, A);
    p.off_keys[1] = off; off = align_up(off + n * (size_t)maxw, A);
    p.off_vals[0] = off; off = align_up(off + n * 4, A);
    p.off_vals[1] = off; off = align_up(off + n * 4, A);
    p.off_offs = off; off = align_up(off + (size_t)words * 4, A);
    if (p.msd) {
        p.msd_chunk_rows = p.msd_cap / 2;
        p.msd_chunks = (uint32_t)((n + p.msd_chunk_rows - 1) / p.msd_chunk_rows);
        p.off_msd_offs = off; off = align_up(off + (size_t)msd_p * 256 * 4, A);
        p.off_chunks = off; off = align_up(off + ((size_t)p.msd_chunks + 1) * 4, A);
    }
    if (p.dict) {
        p.off_dict_lut = off; off = align_up(off + sizeof(DictLut), A);
        p.off_dict_offs = off; off = align_up(off + 256 * 4, A);
    }
    // zeroed region: hist | counters+err | status[0] (| status[1] | MSD
    // histograms | plan word | dictionary table and words: with the MSD-first
    // or dictionary plan the LSD passes may start after passes that never
    // ran, so both status buffers start clear)
    p.off_zero = off;
    p.off_hist = off; off = align_up(off + (size_t)words * 4, A);
    p.off_counters = off; off = align_up(off + (size_t)(total + msd_p + 2) * 4, A);
    p.off_status[0] = off; off = align_up(off + status_bytes, A);
    if (p.msd || p.dict) {
        p.off_status[1] = off; off = align_up(off + status_bytes, A);
        if (p.msd) { p.off_msd_hist = off; off = align_up(off + (size_t)msd_p * 256 * 4, A); }
        p.off_msd_flag = off; off = align_up(off + 4, A);
        if (p.dict) {
            p.off_dict_table = off; off = align_up(off + sizeof(DictSlot) * kDictSlots, A);
            p.off_dict_words = off; off = align_up(off + 16, A);
        }
        p.zero_bytes = off - p.off_zero;
    } else {
        p.zero_bytes = off - p.off_zero;
        p.off_status[1] = off; off = align_up(off + status_bytes, A);
    }
    p.ws_bytes = off;
    return p;
}

int sort_launches(const SortPlan& p) {
    // histogram + scan + passes, plus for the MSD plan its histogram, scan,
    // passes, chunk search and shared-memory finish (the LSD kernels are
    // launched in either case and return at once when not needed)
    return 2 + p.total_passes + (p.msd ? 4 + p.msd_passes : 0) + (p.dict ? 3 : 0);
}

namespace {
// The LSD passes over all keys (first_g: global index of the first pass, for
// tile counters and status parity; run_flag: conditional launches).
cudaError_t run_lsd(const SortPlan& p, const void* const* key_cols, int order, uint32_t* perm_out, void* key0_out,
                    unsigned char* ws, uint32_t* err, cudaStream_t s, Profiler* prof, const uint32_t* perm_in,
                    int first_g, const uint32_t* run_flag, uint32_t* run_count) {
    const uint64_t n = p.n;
    cudaError_t e;
    uint32_t* hist = reinterpret_cast<uint32_t*>(ws + p.off_hist);
    uint32_t* offs = reinterpret_cast<uint32_t*>(ws + p.off_offs);
    uint32_t* counters = reinterpret_cast<uint32_t*>(ws + p.off_counters);
    uint32_t* status[2] = {reinterpret_cast<uint32_t*>(ws + p.off_status[0]),
                           reinterpret_cast<uint32_t*>(ws + p.off_status[1])};
    void* kbuf[2] = {ws + p.off_keys[0], ws + p.off_keys[1]};
    uint32_t* vbuf[2] = {reinterpret_cast<uint32_t*>(ws + p.off_vals[0]),
                         reinterpret_cast<uint32_t*>(ws + p.off_vals[1])};
    const bool invert = (order == 1);
    const bool reverse = (order == 2);

    HistArgs h{};
    h.n = n;
    h.hist = hist;
    h.ncols = p.nkeys;
    h.hist_words = p.hist_words;
    h.run_flag = run_flag;
    h.run_count = run_count;
    ScanArgs sc{};
    sc.hist = hist;
    sc.offs = offs;
    sc.run_flag = run_flag;
    for (int k = 0; k < p.nkeys; ++k) {
        h.col[k].data = key_cols[k];
        h.col[k].dtype = p.dtype[k];
        h.col[k].passes = p.passes[k];
        h.col[k].bits = p.bits[k];
        h.col[k].hist_off = p.hist_off[k];
        h.col[k].invert = invert;
        for (int q = 0; q < p.passes[k]; ++q) {
            sc.off[p.pass_base[k] + q] = (uint32_t)(p.hist_off[k] + q * p.radix[k]);
            sc.radix[p.pass_base[k] + q] = (uint32_t)p.radix[k];
        }
    }
    {
        size_t smem = (size_t)p.hist_words * 4;
        int dev = 0, sms = 148;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        uint64_t want = (n + 511) / 512;
        uint32_t grid = (uint32_t)(want < (uint64_t)sms * 4 ? want : (uint64_t)sms * 4);
        if (grid == 0) grid = 1;
        if (prof) prof->begin(run_flag ? KC_FALLBACK : KC_HIST, s);
        bool all8 = true;
        for (int k = 0; k < p.nkeys; ++k) all8 = all8 && p.bits[k] == 8;
        if (all8) k_digit_hist<8><<<grid, 512, smem, s>>>(h);
        else k_digit_hist<0><<<grid, 512, smem, s>>>(h);
        if (prof) prof->end(run_flag ? KC_FALLBACK : KC_HIST, s);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
        if (prof) prof->begin(run_flag ? KC_FALLBACK : KC_SCAN, s);
        k_hist_scan<<<p.total_passes, 256, 0, s>>>(sc);
        if (prof) prof->end(run_flag ? KC_FALLBACK : KC_SCAN, s);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
    }

    const int last_g = first_g + p.total_passes - 1;
    int kcur = -1, vcur = -1;
    int g = first_g;  // global pass counter (processing order)
    for (int k = p.nkeys - 1; k >= 0; --k) {
        const int w = p.width[k];
        const PassVariant& var = variant_for(p.tuning, w);
        const uint32_t tiles = (uint32_t)((n + var.threads * var.items - 1) / (var.threads * var.items));
        for (int q = 0; q < p.passes[k]; ++q, ++g) {
            PassArgs a{};
            a.n = n;
            a.shift = (uint32_t)(q * p.bits[k]);
            a.dtype = p.dtype[k];
            a.invert = invert;
            a.reverse = reverse;
            a.bin_offsets = offs + p.hist_off[k] + (size_t)q * p.radix[k];
            a.status = status[g & 1];
            a.status_next = (g < last_g) ? status[(g + 1) & 1] : nullptr;
            a.status_rows = p.max_tiles;
            a.status_row_words = (uint32_t)p.max_radix;
            a.tile_counter = counters + g;
            a.err = err;
            a.run_flag = run_flag;
            a.run_when = 1;
            a.spin_limit = p.tuning.spin_limit;
            a.stall_tile = g == first_g ? p.tuning.stall_tile : 0xffffffffu;
            int mode;
            if (q == 0 && k == p.nkeys - 1) {
                // first pass: the rows themselves, or the rows as seen through
                // an input permutation (the reference radix sort's in/out idx)
                mode = perm_in ? IN_GATHER : IN_RAW;
                a.keys_in = key_cols[k];
                a.vals_in = perm_in;
            } else if (q == 0) {
                mode = IN_GATHER;
                a.keys_in = key_cols[k];
                a.vals_in = vbuf[vcur];
            } else {
                mode = IN_BUF;
                a.keys_in = kbuf[kcur];
                a.vals_in = vbuf[vcur];
            }
            const bool fin = (k == 0 && q == p.passes[k] - 1);
            const int kn = (kcur < 0) ? 0 : kcur ^ 1;
            const int vn = (vcur < 0) ? 0 : vcur ^ 1;
            if (fin) {
                a.keys_out = key0_out;
                a.vals_out = perm_out;
            } else {
                a.keys_out = kbuf[kn];
                a.vals_out = vbuf[vn];
            }
            // conditional passes (the MSD plan's fallback) are timed apart
            // from the passes that always run
            const int cls = run_flag ? KC_FALLBACK : (w == 4 ? KC_ONESWEEP32 : KC_ONESWEEP64);
            // a fallback pass usually returns at once: a persistent grid
            // makes that one short wave
            a.ntiles = tiles;
            const uint32_t grid = pass_grid(tiles, resident_of(var), var.tma || run_flag != nullptr);
            if (prof) prof->begin(cls, s);
            var.k[mode][fin ? 1 : 0]<<<grid, var.threads, var.smem, s>>>(a);
            e = cudaGetLastError();
            if (prof) prof->end(cls, s);
            if (e != cudaSuccess) return e;
            kcur = kn;
            vcur = vn;
        }
    }
    return cudaSuccess;
}

// MSD-first front half: top-digit histograms and scans, the global passes
// over the top digits of key 0, the chunk search and the shared-memory
// finish.  Leaves the flag at ws + off_msd_flag set if the plan failed.
cudaError_t run_msd(const SortPlan& p, const void* const* key_cols, int order, uint32_t* perm_out, void* key0_out,
                    unsigned char* ws, uint32_t* err, cudaStream_t s, Profiler* prof, const uint32_t* perm_in) {
    const uint64_t n = p.n;
    const int w = p.width[0];
    const int P = p.msd_passes;
    const int ndigits = w;  // 8-bit digits
    const int first = ndigits - P;
    cudaError_t e;
    uint32_t* mhist = reinterpret_cast<uint32_t*>(ws + p.off_msd_hist);
    uint32_t* moffs = reinterpret_cast<uint32_t*>(ws + p.off_msd_offs);
    uint32_t* flag = reinterpret_cast<uint32_t*>(ws + p.off_msd_flag);
    uint32_t* counters = reinterpret_cast<uint32_t*>(ws + p.off_counters);
    uint32_t* status[2] = {reinterpret_cast<uint32_t*>(ws + p.off_status[0]),
                           reinterpret_cast<uint32_t*>(ws + p.off_status[1])};
    void* kbuf[2] = {ws + p.off_keys[0], ws + p.off_keys[1]};
    uint32_t* vbuf[2] = {reinterpret_cast<uint32_t*>(ws + p.off_vals[0]),
                         reinterpret_cast<uint32_t*>(ws + p.off_vals[1])};
    const bool invert = (order == 1);

    MsdHistArgs mh{key_cols[0], p.dtype[0], invert ? 1 : 0, first, P, n, mhist, flag};
    if (prof) prof->begin(KC_HIST, s);
    e = msd_hist(mh, w, s);
    if (prof) prof->end(KC_HIST, s);
    if (e != cudaSuccess) return e;
    if (prof) prof->begin(KC_SCAN, s);
    e = msd_scan(mhist, moffs, P, p.msd_cap, flag, s);
    if (prof) prof->end(KC_SCAN, s);
    if (e != cudaSuccess) return e;

    const PassVariant& var = variant_for(p.tuning, w);
    const uint32_t tiles = (uint32_t)((n + var.threads * var.items - 1) / (var.threads * var.items));
    for (int q = 0; q < P; ++q) {
        PassArgs a{};
        a.n = n;
        a.shift = (uint32_t)(8 * (first + q));
        a.dtype = p.dtype[0];
        a.invert = invert;
        a.reverse = 0;
        a.bin_offsets = moffs + (size_t)q * 256;
        a.status = status[q & 1];
        a.status_next = status[(q + 1) & 1];
        a.status_rows = p.max_tiles;
        a.status_row_words = (uint32_t)p.max_radix;
        a.tile_counter = counters + q;
        a.err = err;
        a.run_flag = flag;
        a.run_when = 0;
        a.spin_limit = p.tuning.spin_limit;
        a.stall_tile = q == 0 ? p.tuning.stall_tile : 0xffffffffu;
        int mode;
        if (q == 0) {
            mode = perm_in ? IN_GATHER : IN_RAW;
            a.keys_in = key_cols[0];
            a.vals_in = perm_in;
        } else {
            mode = IN_BUF;
            a.keys_in = kbuf[(q - 1) & 1];
            a.vals_in = vbuf[(q - 1) & 1];
        }
        a.keys_out = kbuf[q & 1];
        a.vals_out = vbuf[q & 1];
        a.ntiles = tiles;
        if (prof) prof->begin(w == 4 ? KC_ONESWEEP32 : KC_ONESWEEP64, s);
        var.k[mode][0]<<<pass_grid(tiles, resident_of(var), var.tma != 0), var.threads, var.smem, s>>>(a);
        e = cudaGetLastError();
        if (prof) prof->end(w == 4 ? KC_ONESWEEP32 : KC_ONESWEEP64, s);
        if (e != cudaSuccess) return e;
    }
    const void* skeys = kbuf[(P - 1) & 1];
    const uint32_t* svals = vbuf[(P - 1) & 1];
    uint32_t* chunk_start = reinterpret_cast<uint32_t*>(ws + p.off_chunks);
    MsdChunkArgs ca{skeys, n, p.msd_chunk_rows, p.msd_chunks, (uint32_t)(8 * (ndigits - P)), chunk_start, flag};
    if (prof) prof->begin(KC_LOCALSORT, s);
    e = msd_chunks(ca, w, s, p.msd_cap);
    if (e == cudaSuccess) {
        MsdLocalArgs la{};
        la.keys = skeys;
        la.vals = svals;
        la.chunk_start = chunk_start;
        la.n = n;
        la.sec = p.nkeys > 1 ? key_cols[1] : nullptr;
        la.sec_dtype = p.nkeys > 1 ? p.dtype[1] : 0;
        la.dtype = p.dtype[0];
        la.invert = invert ? 1 : 0;
        la.reverse = order == 2 ? 1 : 0;
        la.lo_bits = (uint32_t)p.msd_lo_bits;
        la.flag = flag;
        la.err = err;
        la.keys_out = key0_out;
        la.perm_out = perm_out;
        e = msd_local(la, w, p.msd_chunks, p.tuning.msd_match & 1, s, p.msd_cap);
    }
    if (prof) prof->end(KC_LOCALSORT, s);
    return e;
}

// The dictionary plan: the distinct keys and their ranks, then the one pass
// (taken only when the plan word says 2).
cudaError_t run_dict(const SortPlan& p, const void* const* key_cols, int order, uint32_t* perm_out, void* key0_out,
                     unsigned char* ws, uint32_t* err, cudaStream_t s, Profiler* prof, const uint32_t* perm_in,
                     uint32_t* taken) {
    uint32_t* word = reinterpret_cast<uint32_t*>(ws + p.off_msd_flag);
    uint32_t* words = reinterpret_cast<uint32_t*>(ws + p.off_dict_words);
    DictLut* lut = reinterpret_cast<DictLut*>(ws + p.off_dict_lut);
    uint32_t* offs = reinterpret_cast<uint32_t*>(ws + p.off_dict_offs);
    uint32_t* counters = reinterpret_cast<uint32_t*>(ws + p.off_counters);
    const bool invert = (order == 1);
    DictArgs da{};
    da.keys = key_cols[0];
    da.dtype = p.dtype[0];
    da.invert = invert ? 1 : 0;
    da.width = p.width[0];
    da.n = p.n;
    da.table = reinterpret_cast<DictSlot*>(ws + p.off_dict_table);
    da.distinct = words;
    da.overflow = words + 1;
    da.state = word;
    da.fail_state = p.msd ? 0u : 1u;  // next: the MSD-first plan, or the LSD passes
    da.lut = lut;
    da.bin_offsets = offs;
    da.taken = taken;
    da.spin_limit = p.tuning.spin_limit;
    da.err = err;
    if (prof) prof->begin(KC_DICT, s);
    cudaError_t e = dict_collect(da, s);
    if (e == cudaSuccess) e = dict_rank(da, s);
    if (prof) prof->end(KC_DICT, s);
    if (e != cudaSuccess) return e;
    const DictVariant& dv = kDictVariants[p.dict_variant];
    PassArgs a{};
    a.n = p.n;
    a.shift = 0;
    a.dtype = p.dtype[0];
    a.invert = invert;
    a.reverse = order == 2 ? 1 : 0;
    a.bin_offsets = offs;
    a.status = reinterpret_cast<uint32_t*>(ws + p.off_status[0]);
    a.status_next = nullptr;  // nothing runs after this pass when it runs
    a.status_rows = p.max_tiles;
    a.status_row_words = (uint32_t)p.max_radix;
    a.tile_counter = counters + p.total_passes + (p.msd ? p.msd_passes : 0);
    a.err = err;
    a.run_flag = word;
    a.run_when = 2;
    a.spin_limit = p.tuning.spin_limit;
    a.stall_tile = p.tuning.stall_tile;
    a.keys_in = key_cols[0];
    a.vals_in = perm_in;
    a.keys_out = key0_out;
    a.vals_out = perm_out;
    a.dict_lut = lut;
    a.ntiles = p.dict_tiles;
    const int cls = dv.width == 4 ? KC_ONESWEEP32 : KC_ONESWEEP64;
    if (prof) prof->begin(cls, s);
    dv.k[perm_in ? 1 : 0]<<<pass_grid(p.dict_tiles, g_dict_resident[p.dict_variant], true), dv.threads, dv.smem, s>>>(a);
    e = cudaGetLastError();
    if (prof) prof->end(cls, s);
    return e;
}
}  // namespace

cudaError_t run_sort(const SortPlan& p, const void* const* key_cols, int order, uint32_t* perm_out,
                     void* key0_out, unsigned char* ws, uint32_t* err, cudaStream_t s, Profiler* prof,
                     const uint32_t* perm_in, uint32_t* msd_fallbacks, uint32_t* dict_taken) {
    if (p.n == 0) return cudaSuccess;
    cudaError_t e = cudaMemsetAsync(ws + p.off_zero, 0, p.zero_bytes, s);
    if (e != cudaSuccess) return e;
    if (!p.msd && !p.dict)
        return run_lsd(p, key_cols, order, perm_out, key0_out, ws, err, s, prof, perm_in, 0, nullptr, nullptr);
    // the plan word picks what runs: 2 the dictionary pass, 0 the MSD-first
    // plan, 1 the LSD passes over all keys (each launch returns at once
    // unless the word selects it)
    if (p.dict && (e = run_dict(p, key_cols, order, perm_out, key0_out, ws, err, s, prof, perm_in, dict_taken)) !=
                      cudaSuccess)
        return e;
    if (p.msd && (e = run_msd(p, key_cols, order, perm_out, key0_out, ws, err, s, prof, perm_in)) != cudaSuccess)
        return e;
    const uint32_t* flag = reinterpret_cast<const uint32_t*>(ws + p.off_msd_flag);
    return run_lsd(p, key_cols, order, perm_out, key0_out, ws, err, s, prof, perm_in, p.msd ? p.msd_passes : 0, flag,
                   p.msd ? msd_fallbacks : nullptr);
}

// ---------------------------------------------------------------------------
// segmented sort (host side)
// ---------------------------------------------------------------------------
int seg_sort_variant_count() { return kNumSegVariants; }

bool seg_sort_variant_info(int v, int* bits, int* tile_rows) {
    if (v < 0 || v >= kNumSegVariants) return false;
    *bits = kSegVariants[v].bits;
    *tile_rows = kSegVariants[v].tile;
    return true;
}

namespace {
struct SegLayout {
    size_t keys[2], vals[2], offs, zero, hist, counters, status[2], zero_bytes, total;
    uint32_t stride, radix;
};
SegLayout seg_layout(uint64_t n, uint32_t nsegs, uint32_t ntiles, int max_passes, int variant, int key_width) {
    SegLayout L{};
    const SegVariant& v = kSegVariants[variant];
    L.radix = 1u << v.bits;
    L.stride = (uint32_t)max_passes * L.radix;
    const size_t A = 256;
    size_t off = 0;
    L.keys[0] = off; off = align_up(off + n * (size_t)key_width, A);
    L.keys[1] = off; off = align_up(off + n * (size_t)key_width, A);
    L.vals[0] = off; off = align_up(off + n * 4, A);
    L.vals[1] = off; off = align_up(off + n * 4, A);
    L.offs = off; off = align_up(off + (size_t)nsegs * L.stride * 4, A);
    L.zero = off;
    L.hist = off; off = align_up(off + (size_t)nsegs * L.stride * 4, A);
    L.counters = off; off = align_up(off + (size_t)(max_passes + 1) * 4, A);
    L.status[0] = off; off = align_up(off + (size_t)ntiles * L.radix * 4, A);
    L.zero_bytes = off - L.zero;
    L.status[1] = off; off = align_up(off + (size_t)ntiles * L.radix * 4, A);
    L.total = off;
    return L;
}
}  // namespace

size_t seg_sort_workspace_bytes(uint64_t n, uint32_t nsegs, uint32_t ntiles, int max_passes, int variant,
                                int key_width) {
    if (variant < 0 || variant >= kNumSegVariants) return 0;
    return seg_layout(n, nsegs, ntiles, max_passes, variant, key_width).total;
}

cudaError_t run_seg_sort(const SegSortArgs& sa, unsigned char* ws, cudaStream_t s, Profiler* prof) {
    if (sa.n == 0 || sa.ntiles == 0) return cudaSuccess;
    if (sa.variant < 0 || sa.variant >= kNumSegVariants || sa.max_passes < 1 || sa.max_passes > 16)
        return cudaErrorInvalidValue;
    if (sa.key_width != 4 && sa.key_width != 8) return cudaErrorInvalidValue;
    const SegVariant& var = kSegVariants[sa.variant];
    const int wi = sa.key_width == 8 ? 1 : 0;
    const SegLayout L = seg_layout(sa.n, sa.nsegs, sa.ntiles, sa.max_passes, sa.variant, sa.key_width);
    cudaError_t e = cudaMemsetAsync(ws + L.zero, 0, L.zero_bytes, s);
    if (e != cudaSuccess) return e;
    uint32_t* hist = reinterpret_cast<uint32_t*>(ws + L.hist);
    uint32_t* offs = reinterpret_cast<uint32_t*>(ws + L.offs);
    uint32_t* counters = reinterpret_cast<uint32_t*>(ws + L.counters);
    uint32_t* status[2] = {reinterpret_cast<uint32_t*>(ws + L.status[0]),
                           reinterpret_cast<uint32_t*>(ws + L.status[1])};
    void* kbuf[2] = {ws + L.keys[0], ws + L.keys[1]};
    uint32_t* vbuf[2] = {reinterpret_cast<uint32_t*>(ws + L.vals[0]), reinterpret_cast<uint32_t*>(ws + L.vals[1])};

    SegHistArgs h{sa.keys, sa.key_width, sa.chunks, sa.segs, hist, L.stride, (uint32_t)var.bits, sa.nsegs, sa.n,
                  sa.seg_flag};
    if (prof) prof->begin(KC_HIST, s);
    k_seg_hist<<<sa.nchunks, 512, (size_t)L.stride * 4, s>>>(h);
    if (prof) prof->end(KC_HIST, s);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    if (prof) prof->begin(KC_SCAN, s);
    k_row_scan<<<sa.nsegs * (uint32_t)sa.max_passes, 256, 0, s>>>(hist, offs, L.radix);
    if (prof) prof->end(KC_SCAN, s);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;

    for (int g = 0; g < sa.max_passes; ++g) {
        const uint32_t grid = sa.tiles_in_pass[g];
        if (grid == 0) break;
        PassArgs a{};
        a.n = sa.n;
        a.shift = (uint32_t)(g * var.bits);
        a.dtype = sa.key_width == 8 ? U64 : U32;
        a.status = status[g & 1];
        a.status_next = (g + 1 < sa.max_passes) ? status[(g + 1) & 1] : nullptr;
        a.status_rows = sa.ntiles;
        a.status_row_words = L.radix;
        a.tile_counter = counters + g;
        a.err = sa.err;
        a.tile_seg = sa.tile_seg;
        a.segs = sa.segs;
        a.seg_offs = offs;
        a.seg_stride = L.stride;
        a.pass = (uint32_t)g;
        a.keys_in = g == 0 ? sa.keys : static_cast<const void*>(kbuf[(g - 1) & 1]);
        a.vals_in = g == 0 ? nullptr : vbuf[(g - 1) & 1];
        a.keys_out = kbuf[g & 1];
        a.vals_out = vbuf[g & 1];
        a.keys_final = sa.keys_out;
        a.vals_final = sa.perm_out;
        a.seg_flag = sa.seg_flag;
        a.seg_flag_when = 1;
        // passes over flagged segments only (usually a few): a persistent grid
        a.ntiles = grid;
        const uint32_t launch = pass_grid(grid, g_seg_resident[sa.variant][wi], sa.seg_flag != nullptr);
        const int cls = wi ? KC_ONESWEEP64 : KC_ONESWEEP32;
        if (prof) prof->begin(cls, s);
        var.k[wi][g == 0 ? 0 : 1]<<<launch, 256, var.smem[wi], s>>>(a);
        e = cudaGetLastError();
        if (prof) prof->end(cls, s);
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

// ---------------------------------------------------------------------------
// equal neighbours in a sorted column
// ---------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(256) k_adjacent_ties(const T* keys, uint64_t n, uint32_t* flag) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    bool eq = false;
    // four rows per thread per round, all loads issued first (the previous
    // row's key comes from the neighbouring lane's load, an L1 hit)
    constexpr int R = 4;
    for (uint64_t i0 = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x + 1; i0 < n; i0 += R * stride) {
        T cur[R], prev[R];
#pragma unroll
        for (int q = 0; q < R; ++q) {
            const uint64_t i = i0 + q * stride;
            cur[q] = i < n ? __ldg(keys + i) : T(0);
            prev[q] = i < n ? __ldg(keys + i - 1) : T(0);
        }
#pragma unroll
        for (int q = 0; q < R; ++q) eq |= (i0 + q * stride < n) && cur[q] == prev[q];
    }
    if (__any_sync(0xffffffffu, eq) && (threadIdx.x & 31) == 0) atomicOr(flag, 1u);
}

cudaError_t flag_adjacent_ties(const void* sorted_keys, int width, uint64_t n, uint32_t* flag, cudaStream_t s,
                               Profiler* prof) {
    if (n < 2) return cudaSuccess;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const uint64_t want = (n + 255) / 256;
    const uint32_t grid = (uint32_t)std::min<uint64_t>(want, (uint64_t)sms * 16);
    if (prof) prof->begin(KC_TIES, s);
    if (width == 8)
        k_adjacent_ties<unsigned long long><<<grid, 256, 0, s>>>(static_cast<const unsigned long long*>(sorted_keys),
                                                                 n, flag);
    else
        k_adjacent_ties<uint32_t><<<grid, 256, 0, s>>>(static_cast<const uint32_t*>(sorted_keys), n, flag);
    if (prof) prof->end(KC_TIES, s);
    return cudaGetLastError();
}

// Raises the dynamic shared-memory limit of every sort kernel on the current
// device; called once per device before the first sort.
cudaError_t prepare_sort_kernels() {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaError_t e0 = cudaDeviceGetAttribute(&g_sms, cudaDevAttrMultiProcessorCount, dev);
    if (e0 != cudaSuccess) return e0;
    for (int i = 0; i < kNumVariants; ++i) {
        const PassVariant& v = kVariants[i];
        int res = 1 << 30;
        for (int m = 0; m < 3; ++m)
            for (int f = 0; f < 2; ++f) {
                cudaError_t e = cudaFuncSetAttribute(v.k[m][f], cudaFuncAttributeMaxDynamicSharedMemorySize, (int)v.smem);
                if (e != cudaSuccess) return e;
                int nb = 0;
                e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, v.k[m][f], v.threads, v.smem);
                if (e != cudaSuccess) return e;
                res = std::min(res, nb);
            }
        g_resident[i] = std::max(res, 1);
    }
    for (int i = 0; i < 2; ++i) {
        const DictVariant& v = kDictVariants[i];
        int res = 1 << 30;
        for (int m = 0; m < 2; ++m) {
            cudaError_t e = cudaFuncSetAttribute(v.k[m], cudaFuncAttributeMaxDynamicSharedMemorySize, (int)v.smem);
            if (e != cudaSuccess) return e;
            int nb = 0;
            e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, v.k[m], v.threads, v.smem);
            if (e != cudaSuccess) return e;
            res = std::min(res, nb);
        }
        g_dict_resident[i] = std::max(res, 1);
    }
    static_assert(kNumSegVariants <= 16, "residency table");
    for (int i = 0; i < kNumSegVariants; ++i) {
        const SegVariant& v = kSegVariants[i];
        for (int w = 0; w < 2; ++w) {
            int res = 1 << 30;
            for (int m = 0; m < 2; ++m) {
                cudaError_t e =
                    cudaFuncSetAttribute(v.k[w][m], cudaFuncAttributeMaxDynamicSharedMemorySize, (int)v.smem[w]);
                if (e != cudaSuccess) return e;
                int nb = 0;
                e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, v.k[w][m], 256, v.smem[w]);
                if (e != cudaSuccess) return e;
                res = std::min(res, nb);
            }
            g_seg_resident[i][w] = std::max(res, 1);
        }
    }
    {
        cudaError_t e = cudaFuncSetAttribute(k_seg_hist, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             8 * kMaxRadix * 4);
        if (e != cudaSuccess) return e;
    }
    {
        cudaError_t e = prepare_msd_kernels();
        if (e != cudaSuccess) return e;
    }
    // all histograms of a sort in shared memory: at most 4 keys x 6 passes x
    // 2048 bins (11-bit digits) or 4 x 8 x 256 (8-bit)
    cudaError_t e = cudaFuncSetAttribute(k_digit_hist<8>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         kMaxKeys * 8 * 256 * 4);
    if (e != cudaSuccess) return e;
    return cudaFuncSetAttribute(k_digit_hist<0>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                kMaxKeys * 6 * kMaxRadix * 4);
}

}  // namespace vdf
