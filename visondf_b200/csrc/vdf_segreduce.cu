// vdf_segreduce.cu -- sort-based group-by: segment boundaries + segmented
// count / sum / min / max / mean over rows already in key order.
//
// The reference group-by is hash based (transform_group_by_onecol_mt.hpp:
// 182-337 with AddLookupOneCol / OccLookupOneCol, onecol_functions.inl:4-86:
// one ankerl map probe per row, per-thread maps merged serially,
// merge_functions.inl:3-36; output via CreateValueCol, create_value_col.inl:
// 36-61).  On the GPU the rows are first sorted, so each group is a contiguous
// segment and the whole aggregation is one streaming pass ("reduce by key"):
//
//   * a row is a segment head when any key differs from the previous row;
//   * each thread folds its ITEMS rows into an aggregate
//       (heads, open-segment partial {count, per column sum/min/max}),
//     combined with the associative reduce-by-key operator
//       A (+) B = (A.heads + B.heads, B.heads ? B.partial : A.partial (+) B.partial);
//   * k_seg_tiles reduces every tile of rows to one aggregate (all tiles in
//     parallel, no waiting on other tiles);
//   * k_seg_scan (one CTA) turns the tile aggregates into exclusive tile
//     prefixes: the number of groups before each tile and the partial of the
//     segment that runs into it;
//   * k_seg_emit re-reads each tile, block-scans it seeded with its prefix,
//     and writes every segment that ends inside it (keys, count, sum, min,
//     max, mean), staged per warp in shared memory so that each output
//     column is written by consecutive lanes at consecutive group ids; a
//     tile without a segment head (known from the prefixes) is skipped.
// Nothing spins on another CTA, so there is no look-back latency chain: the
// price is one extra sequential read of the key and value columns (of the
// tiles that hold a head).
//
// Exactness: integer sums are 128-bit (lo, hi words); float sums are carried
// as (sum, compensation) with an error-free TwoSum at every combine, so a
// group's f64 sum is accurate to about one rounding of the exact value,
// independent of how the rows were split over threads and tiles.
//
// All columns are read in sorted row order (the fused sort + group-by call
// gathers them first with the high-occupancy gather kernel: a random read
// costs a full DRAM access of 64 bytes, so each gathered value is read
// randomly exactly once and everything here is sequential).
#include <algorithm>

#include "vdf_agg.cuh"
#include "vdf_common.cuh"
#include "vdf_internal.h"

namespace vdf {

namespace {

// Raw bits of a key / emitted element (zero-extended).
__device__ __forceinline__ uint64_t load_raw(const void* src, int w, uint64_t i) {
    return w == 4 ? (uint64_t)__ldg(static_cast<const uint32_t*>(src) + i)
                  : (uint64_t)__ldg(static_cast<const unsigned long long*>(src) + i);
}
__device__ __forceinline__ void store_raw(void* dst, int w, uint64_t i, uint64_t v) {
    if (w == 4) static_cast<uint32_t*>(dst)[i] = (uint32_t)v;
    else static_cast<unsigned long long*>(dst)[i] = v;
}

// Rows row0 .. row0+ITEMS-1 of a column into arr[j][c] (raw bits, zero-
// extended), with 16-byte vector loads when the rows are in bounds and
// aligned (row0 is a multiple of ITEMS; tile starts are multiples of it).
template <int ITEMS, int W>
__device__ __forceinline__ void load_rows(const void* src, int w, uint64_t row0, uint64_t n, uint64_t (&arr)[ITEMS][W],
                                          int c) {
    const bool full = row0 + ITEMS <= n;
    if (w == 8) {
        const unsigned long long* p = static_cast<const unsigned long long*>(src) + row0;
        if (full && ITEMS % 2 == 0 && (reinterpret_cast<uintptr_t>(p) & 15) == 0) {
#pragma unroll
            for (int j = 0; j < ITEMS; j += 2) {
                const ulonglong2 v = __ldg(reinterpret_cast<const ulonglong2*>(p + j));
                arr[j][c] = v.x;
                arr[j + 1][c] = v.y;
            }
            return;
        }
#pragma unroll
        for (int j = 0; j < ITEMS; ++j) arr[j][c] = row0 + j < n ? __ldg(p + j) : 0ull;
    } else {
        const uint32_t* p = static_cast<const uint32_t*>(src) + row0;
        if (full && ITEMS % 4 == 0 && (reinterpret_cast<uintptr_t>(p) & 15) == 0) {
#pragma unroll
            for (int j = 0; j < ITEMS; j += 4) {
                const uint4 v = __ldg(reinterpret_cast<const uint4*>(p + j));
                arr[j][c] = v.x;
                arr[j + 1][c] = v.y;
                arr[j + 2][c] = v.z;
                arr[j + 3][c] = v.w;
            }
            return;
        }
#pragma unroll
        for (int j = 0; j < ITEMS; ++j) arr[j][c] = row0 + j < n ? (uint64_t)__ldg(p + j) : 0ull;
    }
}

// Canonical images (see load_val) of rows row0 .. row0+ITEMS-1.
template <int ITEMS, int W>
__device__ __forceinline__ void load_vals(const void* src, int dt, uint64_t row0, uint64_t n, uint64_t (&arr)[ITEMS][W],
                                          int c) {
    load_rows<ITEMS>(src, dtype_width(dt), row0, n, arr, c);
#pragma unroll
    for (int j = 0; j < ITEMS; ++j) {
        const uint64_t x = arr[j][c];
        if (dt == I32) arr[j][c] = (uint64_t)(int64_t)(int32_t)(uint32_t)x;
        else if (dt == F32) arr[j][c] = as_b((double)__uint_as_float((uint32_t)x));
    }
}

template <int NV>
struct Agg {
    uint32_t heads;  // segment heads in the covered rows
    uint32_t cnt;    // rows of the open (last) segment inside the covered rows
    uint64_t w[NV > 0 ? NV : 1][4];
};

template <int NV>
__device__ __forceinline__ Agg<NV> agg_identity() {
    Agg<NV> r;
    r.heads = 0;
    r.cnt = 0;
#pragma unroll
    for (int v = 0; v < (NV > 0 ? NV : 1); ++v)
#pragma unroll
        for (int q = 0; q < 4; ++q) r.w[v][q] = 0;
    return r;
}

// A is earlier in row order than B.
template <int NV>
__device__ __forceinline__ Agg<NV> agg_combine(const Agg<NV>& A, const Agg<NV>& B, const int* vc) {
    Agg<NV> r;
    r.heads = A.heads + B.heads;
    if (B.heads > 0 || A.cnt == 0) {
        r.cnt = B.cnt;
#pragma unroll
        for (int v = 0; v < NV; ++v)
#pragma unroll
            for (int q = 0; q < 4; ++q) r.w[v][q] = B.w[v][q];
    } else if (B.cnt == 0) {
        r.cnt = A.cnt;
#pragma unroll
        for (int v = 0; v < NV; ++v)
#pragma unroll
            for (int q = 0; q < 4; ++q) r.w[v][q] = A.w[v][q];
    } else {
        r.cnt = A.cnt + B.cnt;
#pragma unroll
        for (int v = 0; v < NV; ++v) {
#pragma unroll
            for (int q = 0; q < 4; ++q) r.w[v][q] = A.w[v][q];
            col_merge(r.w[v], B.w[v], vc[v]);
        }
    }
    if (NV == 0) r.w[0][0] = 0;
    return r;
}

template <int NV>
__device__ __forceinline__ Agg<NV> agg_shfl_up(const Agg<NV>& a, int d) {
    Agg<NV> r;
    r.heads = __shfl_up_sync(0xffffffffu, a.heads, d);
    r.cnt = __shfl_up_sync(0xffffffffu, a.cnt, d);
#pragma unroll
    for (int v = 0; v < NV; ++v)
#pragma unroll
        for (int q = 0; q < 4; ++q) r.w[v][q] = __shfl_up_sync(0xffffffffu, a.w[v][q], d);
    return r;
}
template <int NV>
__device__ __forceinline__ Agg<NV> agg_shfl_down(const Agg<NV>& a, int d) {
    Agg<NV> r;
    r.heads = __shfl_down_sync(0xffffffffu, a.heads, d);
    r.cnt = __shfl_down_sync(0xffffffffu, a.cnt, d);
#pragma unroll
    for (int v = 0; v < NV; ++v)
#pragma unroll
        for (int q = 0; q < 4; ++q) r.w[v][q] = __shfl_down_sync(0xffffffffu, a.w[v][q], d);
    return r;
}
template <int NV>
__device__ __forceinline__ Agg<NV> agg_shfl(const Agg<NV>& a, int src) {
    Agg<NV> r;
    r.heads = __shfl_sync(0xffffffffu, a.heads, src);
    r.cnt = __shfl_sync(0xffffffffu, a.cnt, src);
#pragma unroll
    for (int v = 0; v < NV; ++v)
#pragma unroll
        for (int q = 0; q < 4; ++q) r.w[v][q] = __shfl_sync(0xffffffffu, a.w[v][q], src);
    return r;
}

template <int NV>
__device__ __forceinline__ void emit_group(const SegArgs& a, uint32_t g, uint32_t cnt, const uint64_t (*w)[4],
                                           const int* vc) {
    if (a.count_out) a.count_out[g] = (int64_t)cnt;
#pragma unroll
    for (int v = 0; v < NV; ++v) {
        const SegAggOut& o = a.agg[v];
        const int dt = a.val[v].dtype;
        if (vc[v] == VC_FLOAT) {
            const double s = __dadd_rn(as_f(w[v][0]), as_f(w[v][1]));
            if (o.sum) static_cast<double*>(o.sum)[g] = s;
            if (o.mean) o.mean[g] = s / (double)cnt;
            if (dt == F64) {
                if (o.min) static_cast<double*>(o.min)[g] = as_f(w[v][2]);
                if (o.max) static_cast<double*>(o.max)[g] = as_f(w[v][3]);
            } else {
                if (o.min) static_cast<float*>(o.min)[g] = (float)as_f(w[v][2]);
                if (o.max) static_cast<float*>(o.max)[g] = (float)as_f(w[v][3]);
            }
        } else {
            if (o.sum) static_cast<int64_t*>(o.sum)[g] = (int64_t)w[v][0];
            if (o.sum_hi) o.sum_hi[g] = (int64_t)w[v][1];
            if (o.mean) o.mean[g] = i128_to_double(w[v][0], w[v][1], vc[v] == VC_SINT) / (double)cnt;
            const int wd = dtype_width(dt);
            if (o.min) store_raw(o.min, wd, g, w[v][2]);
            if (o.max) store_raw(o.max, wd, g, w[v][3]);
        }
    }
}

// Rows per lane of a warp tile: more rows amortise the tile's look-back;
// fewer keep registers free when many value columns are aggregated.

// Per-warp staging of completed groups (records) and new groups (keys),
// column-major with one padding slot per 32 entries: a thread fills entries
// ITEMS*t .. ITEMS*t+ITEMS-1 and the write-out reads consecutive entries
// across lanes; the skew keeps both patterns (nearly) bank-conflict free.
template <int NK, int NV, int ITEMS>
struct WarpStage {
    static constexpr int ROWS = ITEMS * 32;
    static constexpr int SLOTS = ROWS + 1 + (ROWS + 1) / 32 + 1;
    static __device__ __forceinline__ int at(uint32_t i) { return (int)(i + (i >> 5)); }
    uint64_t w[NV > 0 ? NV : 1][4][SLOTS];
    uint64_t key[NK][SLOTS];
    uint32_t cnt[SLOTS];
    uint32_t start[SLOTS];
    __device__ __forceinline__ void put(uint32_t i, uint32_t c, const uint64_t (*src)[4]) {
        const int x = at(i);
        cnt[x] = c;
#pragma unroll
        for (int v = 0; v < NV; ++v)
#pragma unroll
            for (int q = 0; q < 4; ++q) w[v][q][x] = src[v][q];
    }
};

constexpr int kSegThreads = 256;
constexpr int kSegItems = 2;
constexpr int kSegTile = kSegThreads * kSegItems;  // rows per tile
constexpr int kSegTilesPerCta = 1;                  // tiles each CTA of the reduce and emit passes takes

extern __shared__ __align__(16) unsigned char seg_smem[];

template <int NK, int NV>
__host__ __device__ constexpr size_t stage_offset() {
    return ((sizeof(Agg<NV>) * 2 * (kSegThreads / 32 + 1) + 15) / 16) * 16;
}
template <int NK, int NV>
__host__ __device__ constexpr size_t emit_smem_bytes() {
    return stage_offset<NK, NV>() + sizeof(WarpStage<NK, NV, kSegItems>) * (kSegThreads / 32);
}

// Head flags of this thread's rows (bit j: row row0 + j starts a group).
template <int NK>
__device__ __forceinline__ uint32_t row_heads(const SegArgs& a, uint64_t row0, int lane, const int* kw) {
    constexpr int ITEMS = kSegItems;
    const uint64_t n = a.n;
    uint64_t key[ITEMS][NK];
#pragma unroll
    for (int k = 0; k < NK; ++k) load_rows<ITEMS>(a.key[k].src, kw[k], row0, n, key, k);
    uint64_t prev[NK];
#pragma unroll
    for (int k = 0; k < NK; ++k) prev[k] = __shfl_up_sync(0xffffffffu, key[ITEMS - 1][k], 1);
    if (lane == 0 && row0 > 0 && row0 < n) {
#pragma unroll
        for (int k = 0; k < NK; ++k) prev[k] = load_raw(a.key[k].src, kw[k], row0 - 1);
    }
    uint32_t hmask = 0;
#pragma unroll
    for (int j = 0; j < ITEMS; ++j) {
        const uint64_t r = row0 + j;
        bool h = (r == 0);
#pragma unroll
        for (int k = 0; k < NK; ++k) h |= (j == 0 ? prev[k] : key[j - 1][k]) != key[j][k];
        if (r < n && h) hmask |= 1u << j;
    }
    return hmask;
}

// The fold of this thread's rows into one aggregate, given their head flags.
template <int NV>
__device__ __forceinline__ Agg<NV> fold_rows(const SegArgs& a, uint64_t row0, const int* vc, uint32_t hmask) {
    constexpr int ITEMS = kSegItems;
    const uint64_t n = a.n;
    uint64_t val[ITEMS][NV > 0 ? NV : 1];
#pragma unroll
    for (int v = 0; v < NV; ++v) load_vals<ITEMS>(a.val[v].src, a.val[v].dtype, row0, n, val, v);
    Agg<NV> t = agg_identity<NV>();
#pragma unroll
    for (int j = 0; j < ITEMS; ++j) {
        if (row0 + j >= n) break;
        if (((hmask >> j) & 1u) || t.cnt == 0) {
            if ((hmask >> j) & 1u) t.heads++;
            t.cnt = 1;
#pragma unroll
            for (int v = 0; v < NV; ++v) col_init(t.w[v], val[j][v], vc[v]);
        } else {
            t.cnt++;
#pragma unroll
            for (int v = 0; v < NV; ++v) {
                uint64_t one[4];
                col_init(one, val[j][v], vc[v]);
                col_merge(t.w[v], one, vc[v]);
            }
        }
    }
    return t;
}

// Value-class patterns fixed at compile time (VCP): 0 = read from the column
// dtypes at run time; 1 = two columns, float then signed integer (the
// aggregation every workload here runs).  With the pattern fixed, the
// per-row merges carry no branches on the class.
template <int NV, int VCP>
__device__ __forceinline__ void fix_classes(int* vc) {
    if constexpr (VCP == 1 && NV == 2) {
        vc[0] = VC_FLOAT;
        vc[1] = VC_SINT;
    }
}
// Key-width patterns fixed at compile time (KWP): 0 = run time; otherwise
// key k is (KWP >> 4k) & 15 bytes wide (two keys: 0x48 = 8 then 4 bytes).
template <int NK, int KWP>
__device__ __forceinline__ void fix_widths(int* kw) {
    if constexpr (KWP != 0) {
#pragma unroll
        for (int k = 0; k < NK; ++k) kw[k] = (KWP >> (4 * k)) & 15;
    }
}
inline int key_width_pattern(const SegArgs& a) {
    int p = 0;
    for (int k = 0; k < a.nkeys; ++k) p |= (dtype_width(a.key[k].dtype) & 15) << (4 * k);
    return p;
}
inline int value_class_pattern(const SegArgs& a) {
    auto cls = [](int dt) { return (dt == F64 || dt == F32) ? 0 : (dt == I32 || dt == I64) ? 1 : 2; };
    return (a.nvals == 2 && cls(a.val[0].dtype) == 0 && cls(a.val[1].dtype) == 1) ? 1 : 0;
}

template <int NK, int NV>
__device__ __forceinline__ void seg_setup(const SegArgs& a, int* vc, int* kw) {
#pragma unroll
    for (int v = 0; v < NV; ++v) vc[v] = vclass(a.val[v].dtype);
#pragma unroll
    for (int k = 0; k < NK; ++k) kw[k] = dtype_width(a.key[k].dtype);
}

// ---- phase 1: one aggregate per tile ----------------------------------------
// A tile's aggregate is its head count plus the aggregate of its trailing
// open segment (the rows from its last head, or all its rows if it has none).
// So the keys are read to find the heads and the last head, and only the
// threads whose rows lie in the trailing segment read values and fold them;
// only warps overlapping it reduce.  With many groups (one per few rows)
// almost no values are read here.
template <int NV>
struct TileSmem {
    Agg<NV> s_warp[kSegThreads / 32];
    uint32_t s_heads[kSegThreads / 32];
    int s_last[kSegThreads / 32];
};

template <int NK, int NV>
__device__ __forceinline__ void seg_tile_body(const SegArgs& a, Agg<NV>* tile_agg, uint32_t tile, TileSmem<NV>& sm) {
    constexpr int ITEMS = kSegItems, WARPS = kSegThreads / 32;
    Agg<NV>* s_warp = sm.s_warp;
    uint32_t* s_heads = sm.s_heads;
    int* s_last = sm.s_last;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const uint64_t n = a.n;
    const uint64_t tile0 = (uint64_t)tile * kSegTile;
    const uint64_t row0 = tile0 + (uint64_t)tid * ITEMS;
    int vc[NV > 0 ? NV : 1], kw[NK];
    seg_setup<NK, NV>(a, vc, kw);

    // keys and head flags
    uint64_t key[ITEMS][NK];
#pragma unroll
    for (int k = 0; k < NK; ++k) load_rows<ITEMS>(a.key[k].src, kw[k], row0, n, key, k);
    uint64_t prev[NK];
#pragma unroll
    for (int k = 0; k < NK; ++k) prev[k] = __shfl_up_sync(0xffffffffu, key[ITEMS - 1][k], 1);
    if (lane == 0 && row0 > 0 && row0 < n) {
#pragma unroll
        for (int k = 0; k < NK; ++k) prev[k] = load_raw(a.key[k].src, kw[k], row0 - 1);
    }
    uint32_t hmask = 0;
#pragma unroll
    for (int j = 0; j < ITEMS; ++j) {
        const uint64_t r = row0 + j;
        bool h = (r == 0);
#pragma unroll
        for (int k = 0; k < NK; ++k) h |= (j == 0 ? prev[k] : key[j - 1][k]) != key[j][k];
        if (r < n && h) hmask |= 1u << j;
    }
    // head count and the last head (row within the tile, -1 for none)
    uint32_t heads = __popc(hmask);
    int last = hmask ? tid * ITEMS + (31 - __clz(hmask)) : -1;
#pragma unroll
    for (int d = 16; d >= 1; d >>= 1) {
        heads += __shfl_down_sync(0xffffffffu, heads, d);
        last = max(last, __shfl_down_sync(0xffffffffu, last, d));
    }
    if (lane == 0) {
        s_heads[warp] = heads;
        s_last[warp] = last;
    }
    __syncthreads();
    uint32_t tile_heads = 0;
    int tile_last = -1;
#pragma unroll
    for (int w = 0; w < WARPS; ++w) {
        tile_heads += s_heads[w];
        tile_last = max(tile_last, s_last[w]);
    }
    const int from = tile_last >= 0 ? tile_last : 0;  // first row of the trailing segment

    // fold this thread's rows of the trailing segment
    Agg<NV> t = agg_identity<NV>();
    if (tid * ITEMS + ITEMS - 1 >= from && row0 < n) {
        uint64_t val[ITEMS][NV > 0 ? NV : 1];
#pragma unroll
        for (int v = 0; v < NV; ++v) load_vals<ITEMS>(a.val[v].src, a.val[v].dtype, row0, n, val, v);
#pragma unroll
        for (int j = 0; j < ITEMS; ++j) {
            if (row0 + j >= n || tid * ITEMS + j < from) continue;
            if (t.cnt == 0) {
#pragma unroll
                for (int v = 0; v < NV; ++v) col_init(t.w[v], val[j][v], vc[v]);
            } else {
#pragma unroll
                for (int v = 0; v < NV; ++v) {
                    uint64_t one[4];
                    col_init(one, val[j][v], vc[v]);
                    col_merge(t.w[v], one, vc[v]);
                }
            }
            t.cnt++;
        }
    }
    // ordered reduction over the warps that hold trailing rows (lower lanes
    // are earlier rows; heads stay 0, so the combine merges)
    const bool active = (warp + 1) * 32 * ITEMS - 1 >= from;
    if (active) {
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const Agg<NV> o = agg_shfl_down(t, d);
            if (lane + d < 32) t = agg_combine(t, o, vc);
        }
        if (lane == 0) s_warp[warp] = t;
    }
    __syncthreads();
    if (tid == 0) {
        Agg<NV> r = agg_identity<NV>();
        for (int w = 0; w < WARPS; ++w)
            if ((w + 1) * 32 * ITEMS - 1 >= from) r = agg_combine(r, s_warp[w], vc);
        r.heads = tile_heads;
        tile_agg[tile] = r;
    }
}

// Each CTA reduces several tiles in turn: 512-row tiles are too short to
// amortise a CTA's launch.
template <int NK, int NV>
__global__ void __launch_bounds__(kSegThreads) k_seg_tiles(SegArgs a, Agg<NV>* tile_agg, uint32_t tiles) {
    __shared__ TileSmem<NV> sm;
    for (uint32_t t = blockIdx.x; t < tiles; t += gridDim.x) {
        seg_tile_body<NK, NV>(a, tile_agg, t, sm);
        __syncthreads();  // shared memory is reused by the next tile
    }
}

// The same tile aggregates with eight rows per thread: one CTA covers
// kSubTiles consecutive 512-row tiles (two warps each), so the pass runs a
// quarter as many CTAs with four times the loads in flight per thread.
constexpr int kWideItems = 8;
constexpr int kSubTiles = kSegThreads * kWideItems / kSegTile;  // 4
constexpr int kWarpsPerSub = kSegThreads / 32 / kSubTiles;      // 2

template <int NK, int NV, int VCP = 0, int KWP = 0>
__global__ void __launch_bounds__(kSegThreads) k_seg_tiles_wide(SegArgs a, Agg<NV>* tile_agg, uint32_t tiles) {
    constexpr int ITEMS = kWideItems, WARPS = kSegThreads / 32;
    __shared__ Agg<NV> s_warp[WARPS];
    __shared__ uint32_t s_heads[WARPS];
    __shared__ int s_last[WARPS];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int sub = warp / kWarpsPerSub;                    // sub-tile of this warp
    const uint32_t tile = blockIdx.x * kSubTiles + sub;     // global tile index
    const int sub_tid = tid - sub * kWarpsPerSub * 32;      // thread within the sub-tile
    const uint64_t n = a.n;
    const uint64_t row0 = (uint64_t)tile * kSegTile + (uint64_t)sub_tid * ITEMS;
    int vc[NV > 0 ? NV : 1], kw[NK];
    seg_setup<NK, NV>(a, vc, kw);
    fix_classes<NV, VCP>(vc);
    fix_widths<NK, KWP>(kw);

    uint64_t key[ITEMS][NK];
#pragma unroll
    for (int k = 0; k < NK; ++k) load_rows<ITEMS>(a.key[k].src, kw[k], row0, n, key, k);
    uint64_t prev[NK];
#pragma unroll
    for (int k = 0; k < NK; ++k) prev[k] = __shfl_up_sync(0xffffffffu, key[ITEMS - 1][k], 1);
    if (lane == 0 && row0 > 0 && row0 < n) {
#pragma unroll
        for (int k = 0; k < NK; ++k) prev[k] = load_raw(a.key[k].src, kw[k], row0 - 1);
    }
    uint32_t hmask = 0;
#pragma unroll
    for (int j = 0; j < ITEMS; ++j) {
        const uint64_t r = row0 + j;
        bool h = (r == 0);
#pragma unroll
        for (int k = 0; k < NK; ++k) h |= (j == 0 ? prev[k] : key[j - 1][k]) != key[j][k];
        if (r < n && h) hmask |= 1u << j;
    }
    uint32_t heads = __popc(hmask);
    int last = hmask ? sub_tid * ITEMS + (31 - __clz(hmask)) : -1;
#pragma unroll
    for (int d = 16; d >= 1; d >>= 1) {
        heads += __shfl_down_sync(0xffffffffu, heads, d);
        last = max(last, __shfl_down_sync(0xffffffffu, last, d));
    }
    if (lane == 0) {
        s_heads[warp] = heads;
        s_last[warp] = last;
    }
    __syncthreads();
    uint32_t tile_heads = 0;
    int tile_last = -1;
#pragma unroll
    for (int w = 0; w < kWarpsPerSub; ++w) {
        tile_heads += s_heads[sub * kWarpsPerSub + w];
        tile_last = max(tile_last, s_last[sub * kWarpsPerSub + w]);
    }
    const int from = tile_last >= 0 ? tile_last : 0;

    Agg<NV> t = agg_identity<NV>();
    if (sub_tid * ITEMS + ITEMS - 1 >= from && row0 < n) {
        uint64_t val[ITEMS][NV > 0 ? NV : 1];
#pragma unroll
        for (int v = 0; v < NV; ++v) load_vals<ITEMS>(a.val[v].src, a.val[v].dtype, row0, n, val, v);
#pragma unroll
        for (int j = 0; j < ITEMS; ++j) {
            if (row0 + j >= n || sub_tid * ITEMS + j < from) continue;
            if (t.cnt == 0) {
#pragma unroll
                for (int v = 0; v < NV; ++v) col_init(t.w[v], val[j][v], vc[v]);
            } else {
#pragma unroll
                for (int v = 0; v < NV; ++v) {
                    uint64_t one[4];
                    col_init(one, val[j][v], vc[v]);
                    col_merge(t.w[v], one, vc[v]);
                }
            }
            t.cnt++;
        }
    }
    const int wsub = warp - sub * kWarpsPerSub;  // warp within the sub-tile
    const bool active = (wsub + 1) * 32 * ITEMS - 1 >= from;
    if (active) {
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const Agg<NV> o = agg_shfl_down(t, d);
            if (lane + d < 32) t = agg_combine(t, o, vc);
        }
        if (lane == 0) s_warp[warp] = t;
    }
    __syncthreads();
    if (sub_tid == 0 && tile < tiles) {
        Agg<NV> r = agg_identity<NV>();
        for (int w = 0; w < kWarpsPerSub; ++w)
            if ((w + 1) * 32 * ITEMS - 1 >= from) r = agg_combine(r, s_warp[sub * kWarpsPerSub + w], vc);
        r.heads = tile_heads;
        tile_agg[tile] = r;
    }
}

// ---- phase 2: exclusive prefixes of the tile aggregates ----------------------
// Level 1: each CTA scans kScanTiles consecutive tile aggregates in place
// (exclusive, within the CTA) and writes the CTA total; level 2: one CTA
// turns the CTA totals into exclusive prefixes.  The emit pass combines the
// two.
constexpr int kScanTiles = 256;

template <int NV>
__device__ __forceinline__ Agg<NV> block_exclusive_scan(Agg<NV> x, Agg<NV>* s_warp, const int* vc, Agg<NV>& total) {
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    Agg<NV> incl = x;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const Agg<NV> o = agg_shfl_up(incl, d);
        if (lane >= d) incl = agg_combine(o, incl, vc);
    }
    if (lane == 31) s_warp[warp] = incl;
    __syncthreads();
    Agg<NV> pre = agg_identity<NV>();
    for (int w = 0; w < warp; ++w) pre = agg_combine(pre, s_warp[w], vc);
    Agg<NV> lx = agg_shfl_up(incl, 1);
    if (lane == 0) lx = agg_identity<NV>();
    total = agg_identity<NV>();
    for (int w = 0; w < (int)(blockDim.x / 32); ++w) total = agg_combine(total, s_warp[w], vc);
    return agg_combine(pre, lx, vc);
}

template <int NV>
__global__ void __launch_bounds__(kScanTiles) k_seg_scan1(const SegArgs a, Agg<NV>* tile_agg, Agg<NV>* block_tot,
                                                          uint32_t tiles) {
    __shared__ Agg<NV> s_warp[kScanTiles / 32];
    int vc[NV > 0 ? NV : 1];
#pragma unroll
    for (int v = 0; v < NV; ++v) vc[v] = vclass(a.val[v].dtype);
    const uint32_t t = blockIdx.x * kScanTiles + threadIdx.x;
    const Agg<NV> x = t < tiles ? tile_agg[t] : agg_identity<NV>();
    Agg<NV> total;
    const Agg<NV> ex = block_exclusive_scan(x, s_warp, vc, total);
    if (t < tiles) tile_agg[t] = ex;
    if (threadIdx.x == 0) block_tot[blockIdx.x] = total;
}

template <int NV>
__global__ void __launch_bounds__(kScanTiles) k_seg_scan2(const SegArgs a, Agg<NV>* block_tot, uint32_t blocks) {
    __shared__ Agg<NV> s_warp[kScanTiles / 32];
    int vc[NV > 0 ? NV : 1];
#pragma unroll
    for (int v = 0; v < NV; ++v) vc[v] = vclass(a.val[v].dtype);
    const uint32_t per = (blocks + kScanTiles - 1) / kScanTiles;
    const uint32_t b0 = min(blocks, threadIdx.x * per), b1 = min(blocks, b0 + per);
    Agg<NV> acc = agg_identity<NV>();
    for (uint32_t b = b0; b < b1; ++b) acc = agg_combine(acc, block_tot[b], vc);
    Agg<NV> total;
    Agg<NV> run = block_exclusive_scan(acc, s_warp, vc, total);
    for (uint32_t b = b0; b < b1; ++b) {
        const Agg<NV> cur = block_tot[b];
        block_tot[b] = run;
        run = agg_combine(run, cur, vc);
    }
}

// ---- phase 3: scan each tile from its prefix and emit the groups -------------
// A tile where every row starts a group (typical when most keys are
// distinct) needs no scan: row r is group H + (r - first row), H = heads
// before the tile, and the group ending at row r - 1 is emitted at row r as
// everywhere else, so a row's own one-row record is written here when the
// next row is in the tile (or r is the last row) and the tile's first row
// emits the group carried in from earlier tiles.  Every column is written
// by consecutive lanes.  Records are built with the same operations as the
// scanning path, so results are bit-identical.
// TPT threads cover the tile, RPT rows each (row tile_first + j * TPT + tt),
// loaded BATCH rows at a time before they are stored.
template <int NK, int NV, int TPT, int RPT, int BATCH>
__device__ __forceinline__ void emit_single_rows(const SegArgs& a, const Agg<NV>* tile_prefix,
                                                 const Agg<NV>* block_prefix, uint32_t tile, uint32_t H,
                                                 const int* vc, const int* kw, int tt) {
    static_assert(TPT * RPT == kSegTile && RPT % BATCH == 0, "tile layout");
    const uint64_t n = a.n;
    const uint64_t first = (uint64_t)tile * kSegTile;
    if (tt == 0 && H > 0) {
        const Agg<NV> P = agg_combine(block_prefix[tile / kScanTiles], tile_prefix[tile], vc);
        emit_group<NV>(a, H - 1, P.cnt, P.w, vc);
    }
#pragma unroll
    for (int j0 = 0; j0 < RPT; j0 += BATCH) {
        // every load of the batch before its first store (outputs may not be
        // assumed apart from inputs, so the compiler would not reorder them)
        uint64_t kx[BATCH][NK];
        uint64_t vx[BATCH][NV > 0 ? NV : 1];
#pragma unroll
        for (int j = 0; j < BATCH; ++j) {
            const uint64_t r = first + (uint64_t)(j0 + j) * TPT + tt;
#pragma unroll
            for (int k = 0; k < NK; ++k) kx[j][k] = r < n ? load_raw(a.key[k].src, kw[k], r) : 0ull;
#pragma unroll
            for (int v = 0; v < NV; ++v) vx[j][v] = r < n ? load_val(a.val[v].src, a.val[v].dtype, r) : 0ull;
        }
#pragma unroll
        for (int j = 0; j < BATCH; ++j) {
            const uint32_t o = (uint32_t)(j0 + j) * TPT + (uint32_t)tt;
            const uint64_t r = first + o;
            if (r >= n) break;
            const uint32_t g = H + o;
#pragma unroll
            for (int k = 0; k < NK; ++k)
                if (a.key_out[k]) store_raw(a.key_out[k], kw[k], g, kx[j][k]);
            if (a.group_start) a.group_start[g] = (uint32_t)r;
            if (a.row_group) a.row_group[r] = g;
            if (o + 1 < (uint32_t)kSegTile || r == n - 1) {
                uint64_t w[NV > 0 ? NV : 1][4];
#pragma unroll
                for (int v = 0; v < NV; ++v) col_init(w[v], vx[j][v], vc[v]);
                emit_group<NV>(a, g, 1, w, vc);
            }
            if (r == n - 1 && a.n_groups) *a.n_groups = g + 1;
        }
    }
}

// Tiles where nearly every row starts a group (few groups of two or more
// rows): rows are striped over the TPT threads (row first + j * TPT + tt),
// so that records of one-row groups go out with consecutive lanes at
// (nearly) consecutive group ids; the head row of a longer group walks that
// group's few rows itself.  A group is emitted by the tile holding its last
// row: one that runs past the tile's end is left to the next tile, whose
// prefix carries it.  hm[t] / hp[t]: head mask of the sub-tile's 8-row block
// t (consecutive rows 8t .. 8t+7) and the number of heads in blocks before
// it within its warp of blocks (32 blocks), wh[w]: heads in warp w's blocks.
template <int NK, int NV, int TPT, int RPT>
__device__ __forceinline__ void emit_mostly_single(const SegArgs& a, const Agg<NV>* tile_prefix,
                                                   const Agg<NV>* block_prefix, uint32_t tile, uint32_t H,
                                                   const uint32_t* hm, const uint32_t* hp, const uint32_t* wh,
                                                   const int* vc, const int* kw, int tt) {
    constexpr int B = 8;  // rows per head-mask block
    static_assert(TPT * RPT == kSegTile && kSegTile / B <= TPT * RPT, "tile layout");
    const uint64_t n = a.n;
    const uint64_t first = (uint64_t)tile * kSegTile;
    const uint32_t rows = (uint32_t)min((uint64_t)kSegTile, n - first);
    // is tile row o a head? (o == rows: the row after the tile)
    auto is_head = [&](uint32_t o) -> bool {
        if (o >= rows) {
            if (first + o >= n) return true;
            bool d = false;
#pragma unroll
            for (int k = 0; k < NK; ++k)
                d |= load_raw(a.key[k].src, kw[k], first + o) != load_raw(a.key[k].src, kw[k], first + o - 1);
            return d;
        }
        return (hm[o / B] >> (o % B)) & 1u;
    };
    auto heads_before = [&](uint32_t o) -> uint32_t {  // heads among tile rows < o
        const uint32_t t = o / B;
        uint32_t c = hp[t] + __popc(hm[t] & ((1u << (o % B)) - 1u));
        for (uint32_t w = 0; w < t / 32; ++w) c += wh[w];
        return c;
    };
    // Aggregate of tile rows [o, end) up to the next head; returns the end.
    auto walk = [&](uint32_t o, uint64_t (*w)[4], uint32_t& cnt) -> uint32_t {
        uint32_t e = o;
        while (e < rows && (e == o || !is_head(e))) {
            const uint64_t r = first + e;
#pragma unroll
            for (int v = 0; v < NV; ++v) {
                const uint64_t x = load_val(a.val[v].src, a.val[v].dtype, r);
                if (cnt == 0) {
                    col_init(w[v], x, vc[v]);
                } else {
                    uint64_t one[4];
                    col_init(one, x, vc[v]);
                    col_merge(w[v], one, vc[v]);
                }
            }
            ++cnt;
            ++e;
        }
        return e;
    };
    // the group carried in from earlier tiles (id H - 1): it ends before the
    // first row if that is a head, else at the tile's first head after it
    if (tt == 0 && H > 0) {
        const Agg<NV> P = agg_combine(block_prefix[tile / kScanTiles], tile_prefix[tile], vc);
        uint64_t w[NV > 0 ? NV : 1][4];
#pragma unroll
        for (int v = 0; v < NV; ++v)
#pragma unroll
            for (int q = 0; q < 4; ++q) w[v][q] = P.w[v][q];
        uint32_t cnt = P.cnt;
        bool ends = true;
        if (!is_head(0)) {
            uint32_t e = 0;
            while (e < rows && !is_head(e)) {
                const uint64_t r = first + e;
#pragma unroll
                for (int v = 0; v < NV; ++v) {
                    uint64_t one[4];
                    col_init(one, load_val(a.val[v].src, a.val[v].dtype, r), vc[v]);
                    col_merge(w[v], one, vc[v]);
                }
                ++cnt;
                ++e;
            }
            ends = e < rows || first + e == n || is_head(e);
        }
        if (ends) emit_group<NV>(a, H - 1, cnt, w, vc);
    }
#pragma unroll 1
    for (int j = 0; j < RPT; ++j) {
        const uint32_t o = (uint32_t)j * TPT + (uint32_t)tt;
        if (o >= rows) break;
        const uint64_t r = first + o;
        const bool h = is_head(o);
        const uint32_t hb = heads_before(o);
        const uint32_t grow = h ? H + hb : H + hb - 1;  // the group of row r
        if (a.row_group) a.row_group[r] = grow;
        if (r == n - 1 && a.n_groups) *a.n_groups = grow + 1;
        if (!h) continue;
        const uint32_t g = H + hb;
#pragma unroll
        for (int k = 0; k < NK; ++k)
            if (a.key_out[k]) store_raw(a.key_out[k], kw[k], g, load_raw(a.key[k].src, kw[k], r));
        if (a.group_start) a.group_start[g] = (uint32_t)r;
        uint64_t w[NV > 0 ? NV : 1][4];
        uint32_t cnt = 0;
        const uint32_t e = walk(o, w, cnt);
        // complete when the next head (or the last row) is inside this tile
        if (e < rows || first + e == n || is_head(e)) emit_group<NV>(a, g, cnt, w, vc);
    }
}

template <int NK, int NV>
__device__ __forceinline__ void seg_emit_body(const SegArgs& a, const Agg<NV>* tile_prefix, const Agg<NV>* block_prefix,
                                              uint32_t tile) {
    constexpr int ITEMS = kSegItems;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const uint64_t n = a.n;
    const uint64_t row0 = (uint64_t)tile * kSegTile + (uint64_t)tid * ITEMS;
    Agg<NV>* s_warp = reinterpret_cast<Agg<NV>*>(seg_smem);  // two buffers of [1 + 8] (see below)
    int vc[NV > 0 ? NV : 1], kw[NK];
    seg_setup<NK, NV>(a, vc, kw);
    // heads before the tile, loaded first so that its latency overlaps the key loads
    const uint32_t H_tile = block_prefix[tile / kScanTiles].heads + tile_prefix[tile].heads;
    const uint32_t hmask = row_heads<NK>(a, row0, lane, kw);
    const uint32_t nvalid = row0 >= n ? 0u : (n - row0 >= (uint64_t)ITEMS ? (uint32_t)ITEMS : (uint32_t)(n - row0));
    if (__syncthreads_and(hmask == (1u << nvalid) - 1u)) {
        emit_single_rows<NK, NV, kSegThreads, kSegItems, kSegItems>(a, tile_prefix, block_prefix, tile, H_tile, vc,
                                                                     kw, tid);
        return;
    }
    const Agg<NV> t = fold_rows<NV>(a, row0, vc, hmask);
    // Per warp: the aggregate of the lanes before each lane (lx) and the
    // warp's total.  When every lane's first row starts a group (typical with
    // many groups), no segment crosses into a lane, so a lane's carry is just
    // the previous lane's trailing segment plus a count of heads: one shuffle
    // of the aggregate and a 32-bit scan instead of a scan of aggregates.
    Agg<NV> lx, wtot;
    if (__all_sync(0xffffffffu, row0 >= n || (hmask & 1u))) {
        const uint32_t h = __popc(hmask);
        uint32_t ih = h;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const uint32_t o = __shfl_up_sync(0xffffffffu, ih, d);
            if (lane >= d) ih += o;
        }
        lx = agg_shfl_up(t, 1);  // previous lane's trailing segment
        lx.heads = ih - h;
        if (lane == 0) lx = agg_identity<NV>();
        wtot = t;  // (read at lane 31) its trailing segment, and all heads
        wtot.heads = ih;
    } else {
        Agg<NV> incl = t;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const Agg<NV> o = agg_shfl_up(incl, d);
            if (lane >= d) incl = agg_combine(o, incl, vc);
        }
        lx = agg_shfl_up(incl, 1);
        if (lane == 0) lx = agg_identity<NV>();
        wtot = incl;
    }
    // [0] tile prefix, [1 + w] total of warp w; warp 0 scans these nine
    // entries in shared memory (double-buffered, four steps) into each warp's
    // exclusive prefix, so every thread then combines once
    constexpr int WARPS = kSegThreads / 32;
    if (lane == 31) s_warp[1 + warp] = wtot;
    if (tid == 0) s_warp[0] = agg_combine(block_prefix[tile / kScanTiles], tile_prefix[tile], vc);
    __syncthreads();
    if (warp == 0) {
        Agg<NV>* src = s_warp;
        Agg<NV>* dst = s_warp + (WARPS + 1);
#pragma unroll 1
        for (int d = 1; d <= WARPS; d <<= 1) {
            if (lane <= WARPS) dst[lane] = lane >= d ? agg_combine(src[lane - d], src[lane], vc) : src[lane];
            __syncwarp();
            Agg<NV>* t2 = src;
            src = dst;
            dst = t2;
        }
    }
    __syncthreads();
    const Agg<NV> pre = agg_combine(s_warp[warp], lx, vc);  // four steps: the result is back in s_warp

    // A segment is complete when the next head (or the last row) is reached;
    // the thread that reaches it produces the group's record.  The groups a
    // warp completes, and the groups whose heads lie in its rows, have
    // consecutive ids, so records and keys are staged in the warp's shared
    // memory and every output column is then written by consecutive lanes.
    using Stage = WarpStage<NK, NV, ITEMS>;
    Stage& st = reinterpret_cast<Stage*>(seg_smem + stage_offset<NK, NV>())[warp];
    const uint32_t H_w = __shfl_sync(0xffffffffu, pre.heads, 0);  // heads before the warp's first row
    const uint32_t g0 = H_w > 0 ? H_w - 1 : 0;                     // first group the warp completes
    uint32_t gid = pre.heads;
    uint32_t cnt = pre.cnt;
    uint64_t w[NV > 0 ? NV : 1][4];
#pragma unroll
    for (int v = 0; v < NV; ++v)
#pragma unroll
        for (int q = 0; q < 4; ++q) w[v][q] = pre.w[v][q];
    uint32_t rg[ITEMS];
    uint32_t emitted = 0;
#pragma unroll
    for (int j = 0; j < ITEMS; ++j) {
        const uint64_t r = row0 + j;
        rg[j] = 0;
        if (r >= n) break;
        uint64_t val[NV > 0 ? NV : 1];
#pragma unroll
        for (int v = 0; v < NV; ++v) val[v] = load_val(a.val[v].src, a.val[v].dtype, r);
        if ((hmask >> j) & 1u) {
            if (gid > 0) {
                st.put(gid - 1 - g0, cnt, w);
                ++emitted;
            }
            ++gid;
            const int ki = Stage::at(gid - 1 - H_w);
#pragma unroll
            for (int k = 0; k < NK; ++k) st.key[k][ki] = load_raw(a.key[k].src, kw[k], r);
            st.start[ki] = (uint32_t)r;
            cnt = 1;
#pragma unroll
            for (int v = 0; v < NV; ++v) col_init(w[v], val[v], vc[v]);
        } else {
            ++cnt;
#pragma unroll
            for (int v = 0; v < NV; ++v) {
                uint64_t one[4];
                col_init(one, val[v], vc[v]);
                col_merge(w[v], one, vc[v]);
            }
        }
        rg[j] = gid - 1;
        if (r == n - 1) {
            st.put(gid - 1 - g0, cnt, w);
            ++emitted;
            if (a.n_groups) *a.n_groups = gid;
        }
    }
    if (a.row_group && row0 < n) {
        if (row0 + ITEMS <= n && (reinterpret_cast<uintptr_t>(a.row_group + row0) & 7) == 0) {
            *reinterpret_cast<uint2*>(a.row_group + row0) = make_uint2(rg[0], rg[1]);
        } else {
#pragma unroll
            for (int j = 0; j < ITEMS; ++j)
                if (row0 + j < n) a.row_group[row0 + j] = rg[j];
        }
    }
    uint32_t E = emitted;
    uint32_t K = __popc(hmask);
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) {
        E += __shfl_xor_sync(0xffffffffu, E, d);
        K += __shfl_xor_sync(0xffffffffu, K, d);
    }
    __syncwarp();
    for (uint32_t i = lane; i < E; i += 32) {
        const int x = Stage::at(i);
        uint64_t gw[NV > 0 ? NV : 1][4];
#pragma unroll
        for (int v = 0; v < NV; ++v)
#pragma unroll
            for (int q = 0; q < 4; ++q) gw[v][q] = st.w[v][q][x];
        emit_group<NV>(a, g0 + i, st.cnt[x], gw, vc);
    }
    for (uint32_t i = lane; i < K; i += 32) {
        const int x = Stage::at(i);
#pragma unroll
        for (int k = 0; k < NK; ++k)
            if (a.key_out[k]) store_raw(a.key_out[k], kw[k], H_w + i, st.key[k][x]);
        if (a.group_start) a.group_start[H_w + i] = st.start[x];
    }
}

// Tiles t0 .. t1-1 write nothing in the emit pass when no segment head lies
// in their rows and no row's group is wanted (row_group): a tile writes the
// group that ends before each head in it (with the new group's key and first
// row), and the group running through head-less tiles is written where the
// next head is.  The tile holding the last row (which writes the last group
// and the group count) is never quiet; nor is t1 past the last tile, whose
// prefix is not stored.  Heads before tile t are the exclusive prefix of the
// tile pass's head counts, so the heads in the range are H(t1) - H(t0).  With
// few groups over many rows (a low-cardinality key) nearly every tile is
// quiet, and its rows are not read a second time.
template <int NV>
__device__ __forceinline__ bool quiet_tiles(const SegArgs& a, const Agg<NV>* tile_prefix, const Agg<NV>* block_prefix,
                                            uint32_t t0, uint32_t t1, uint32_t tiles) {
    if (a.row_group || t1 >= tiles) return false;
    const uint32_t h0 = block_prefix[t0 / kScanTiles].heads + tile_prefix[t0].heads;
    const uint32_t h1 = block_prefix[t1 / kScanTiles].heads + tile_prefix[t1].heads;
    return h1 == h0;
}

template <int NK, int NV>
__global__ void __launch_bounds__(kSegThreads, (NV >= 3 ? 1 : (NV == 2 ? 4 : 3))) k_seg_emit(SegArgs a, const Agg<NV>* tile_prefix,
                                                                          const Agg<NV>* block_prefix, uint32_t tiles) {
    for (uint32_t t = blockIdx.x; t < tiles; t += gridDim.x) {
        if (quiet_tiles(a, tile_prefix, block_prefix, t, t + 1, tiles)) continue;  // the same for the whole CTA
        seg_emit_body<NK, NV>(a, tile_prefix, block_prefix, t);
        __syncthreads();  // the warp totals and staging are reused by the next tile
    }
}

// The emit pass with eight rows per thread: each 512-row tile is taken by
// two warps (kSubTiles tiles per CTA, as in the reduce pass), so a warp scan
// of aggregates and the cross-warp step are shared by eight rows instead of
// two, and each row costs one merge in the final walk.  A thread's rows are
// consecutive: its groups complete in order and are written as they
// complete.  Tiles where every row starts a group take the one-row-record
// path with coalesced writes.
template <int NK, int NV, int VCP = 0, int KWP = 0>
__global__ void __launch_bounds__(kSegThreads, (NV >= 3 ? 1 : 3))
    k_seg_emit_wide(SegArgs a, const Agg<NV>* tile_prefix, const Agg<NV>* block_prefix, uint32_t tiles) {
    constexpr int ITEMS = kWideItems, WARPS = kSegThreads / 32;
    __shared__ Agg<NV> s_wtot[WARPS];
    __shared__ Agg<NV> s_pre[kSubTiles];
    __shared__ uint32_t s_all[WARPS];
    __shared__ uint32_t s_hm[kSegThreads];  // head mask of each thread's rows
    __shared__ uint32_t s_hp[kSegThreads];  // heads before them in the warp
    __shared__ uint32_t s_wh[WARPS];        // heads in each warp's rows
    // tiles without a segment head write nothing (uniform over the CTA, so
    // before any barrier)
    if (quiet_tiles(a, tile_prefix, block_prefix, blockIdx.x * kSubTiles, (blockIdx.x + 1) * kSubTiles, tiles))
        return;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int sub = warp / kWarpsPerSub, wsub = warp - sub * kWarpsPerSub;
    const uint32_t tile = blockIdx.x * kSubTiles + sub;
    const bool tvalid = tile < tiles;
    const int sub_tid = tid - sub * kWarpsPerSub * 32;
    const uint64_t n = a.n;
    const uint64_t row0 = (uint64_t)tile * kSegTile + (uint64_t)sub_tid * ITEMS;
    int vc[NV > 0 ? NV : 1], kw[NK];
    seg_setup<NK, NV>(a, vc, kw);
    fix_classes<NV, VCP>(vc);
    fix_widths<NK, KWP>(kw);
    // heads before the tile, loaded first so that its latency overlaps the key loads
    const uint32_t H_tile = tvalid ? block_prefix[tile / kScanTiles].heads + tile_prefix[tile].heads : 0u;

    uint32_t hmask = 0;
    {
        uint64_t key[ITEMS][NK];
#pragma unroll
        for (int k = 0; k < NK; ++k) load_rows<ITEMS>(a.key[k].src, kw[k], row0, n, key, k);
        uint64_t prev[NK];
#pragma unroll
        for (int k = 0; k < NK; ++k) prev[k] = __shfl_up_sync(0xffffffffu, key[ITEMS - 1][k], 1);
        if (lane == 0 && row0 > 0 && row0 < n) {
#pragma unroll
            for (int k = 0; k < NK; ++k) prev[k] = load_raw(a.key[k].src, kw[k], row0 - 1);
        }
#pragma unroll
        for (int j = 0; j < ITEMS; ++j) {
            const uint64_t r = row0 + j;
            bool h = (r == 0);
#pragma unroll
            for (int k = 0; k < NK; ++k) h |= (j == 0 ? prev[k] : key[j - 1][k]) != key[j][k];
            if (r < n && h) hmask |= 1u << j;
        }
    }
    const uint32_t nvalid = row0 >= n ? 0u : (n - row0 >= (uint64_t)ITEMS ? (uint32_t)ITEMS : (uint32_t)(n - row0));
    const bool wall = __all_sync(0xffffffffu, hmask == (1u << nvalid) - 1u);
    if (lane == 0) s_all[warp] = wall ? 1u : 0u;
    {
        const uint32_t h = __popc(hmask);
        uint32_t ih = h;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const uint32_t o = __shfl_up_sync(0xffffffffu, ih, d);
            if (lane >= d) ih += o;
        }
        s_hm[tid] = hmask;
        s_hp[tid] = ih - h;
        if (lane == 31) s_wh[warp] = ih;
    }
    __syncthreads();
    bool sub_all = true;
    uint32_t sub_heads = 0;
#pragma unroll
    for (int w = 0; w < kWarpsPerSub; ++w) {
        sub_all = sub_all && s_all[sub * kWarpsPerSub + w] != 0u;
        sub_heads += s_wh[sub * kWarpsPerSub + w];
    }
    // many rows start a group (by default at most 32 rows continue one): the
    // striped path
    const uint32_t min_heads = a.striped_min_heads ? a.striped_min_heads : kStripedMinHeads;
    const bool sub_most = !sub_all && sub_heads >= min_heads;

    Agg<NV> lx = agg_identity<NV>();
    if (!sub_all && !sub_most) {
        // this thread's trailing segment: rows from its last head (all rows
        // when it has none).  Rows are consumed from the front of a shift
        // register, so the loop stays rolled (one copy of the merge code)
        // while the values stay in registers.
        uint64_t val[ITEMS][NV > 0 ? NV : 1];
#pragma unroll
        for (int v = 0; v < NV; ++v) load_vals<ITEMS>(a.val[v].src, a.val[v].dtype, row0, n, val, v);
        const int from = hmask ? 31 - __clz(hmask) : 0;
        const int upto = (int)nvalid;
        Agg<NV> t = agg_identity<NV>();
        t.heads = __popc(hmask);
#pragma unroll 1
        for (int j = 0; j < upto; ++j) {
            if (j >= from) {
                if (t.cnt == 0) {
#pragma unroll
                    for (int v = 0; v < NV; ++v) col_init(t.w[v], val[0][v], vc[v]);
                } else {
#pragma unroll
                    for (int v = 0; v < NV; ++v) {
                        uint64_t one[4];
                        col_init(one, val[0][v], vc[v]);
                        col_merge(t.w[v], one, vc[v]);
                    }
                }
                t.cnt++;
            }
#pragma unroll
            for (int i = 0; i + 1 < ITEMS; ++i)
#pragma unroll
                for (int v = 0; v < NV; ++v) val[i][v] = val[i + 1][v];
        }
        // per warp: the aggregate of the lanes before each lane, and the total
        Agg<NV> wtot;
        if (__all_sync(0xffffffffu, row0 >= n || (hmask & 1u))) {
            // no segment crosses into a lane: carry = previous lane's trailing
            // segment, plus a count of heads
            const uint32_t h = __popc(hmask);
            uint32_t ih = h;
#pragma unroll
            for (int d = 1; d < 32; d <<= 1) {
                const uint32_t o = __shfl_up_sync(0xffffffffu, ih, d);
                if (lane >= d) ih += o;
            }
            lx = agg_shfl_up(t, 1);
            lx.heads = ih - h;
            if (lane == 0) lx = agg_identity<NV>();
            wtot = t;
            wtot.heads = ih;
        } else {
            Agg<NV> incl = t;
#pragma unroll 1
            for (int d = 1; d < 32; d <<= 1) {
                const Agg<NV> o = agg_shfl_up(incl, d);
                if (lane >= d) incl = agg_combine(o, incl, vc);
            }
            lx = agg_shfl_up(incl, 1);
            if (lane == 0) lx = agg_identity<NV>();
            wtot = incl;
        }
        if (lane == 31) s_wtot[warp] = wtot;
        if (wsub == 0 && lane == 0 && tvalid)
            s_pre[sub] = agg_combine(block_prefix[tile / kScanTiles], tile_prefix[tile], vc);
    }
    __syncthreads();

    if (sub_all) {
        if (tvalid)
            emit_single_rows<NK, NV, kWarpsPerSub * 32, ITEMS, ITEMS / 2>(a, tile_prefix, block_prefix, tile, H_tile,
                                                                          vc, kw, sub_tid);
        return;
    }
    if (sub_most) {
        if (tvalid) {
            const int base = sub * kWarpsPerSub * 32;
            emit_mostly_single<NK, NV, kWarpsPerSub * 32, ITEMS>(a, tile_prefix, block_prefix, tile, H_tile,
                                                                s_hm + base, s_hp + base, s_wh + sub * kWarpsPerSub,
                                                                vc, kw, sub_tid);
        }
        return;
    }
    if (row0 >= n) return;
    Agg<NV> pre = s_pre[sub];
#pragma unroll
    for (int w = 0; w < kWarpsPerSub; ++w)
        if (w < wsub) pre = agg_combine(pre, s_wtot[sub * kWarpsPerSub + w], vc);
    pre = agg_combine(pre, lx, vc);

    // walk this thread's rows (rolled; each row's values read again, from L1
    // after the fold above brought them in): a head completes the group
    // before it.  Rows after the last head belong to a group that ends in a
    // later thread, so the walk stops at the last head unless the rows' groups
    // are wanted (row_group) or the thread holds the table's last row.
    uint32_t gid = pre.heads;
    uint32_t cnt = pre.cnt;
    uint64_t w[NV > 0 ? NV : 1][4];
#pragma unroll
    for (int v = 0; v < NV; ++v)
#pragma unroll
        for (int q = 0; q < 4; ++q) w[v][q] = pre.w[v][q];
    const bool holds_last = row0 + nvalid == n;
    const int upto = (a.row_group || holds_last) ? (int)nvalid : (hmask ? 32 - __clz(hmask) : 0);
#pragma unroll 1
    for (int j = 0; j < upto; ++j) {
        const uint64_t r = row0 + j;
        uint64_t x[NV > 0 ? NV : 1];
#pragma unroll
        for (int v = 0; v < NV; ++v) x[v] = load_val(a.val[v].src, a.val[v].dtype, r);
        if ((hmask >> j) & 1u) {
            if (gid > 0) emit_group<NV>(a, gid - 1, cnt, w, vc);
#pragma unroll
            for (int k = 0; k < NK; ++k)
                if (a.key_out[k]) store_raw(a.key_out[k], kw[k], gid, load_raw(a.key[k].src, kw[k], r));
            if (a.group_start) a.group_start[gid] = (uint32_t)r;
            ++gid;
            cnt = 1;
#pragma unroll
            for (int v = 0; v < NV; ++v) col_init(w[v], x[v], vc[v]);
        } else {
            ++cnt;
#pragma unroll
            for (int v = 0; v < NV; ++v) {
                uint64_t one[4];
                col_init(one, x[v], vc[v]);
                col_merge(w[v], one, vc[v]);
            }
        }
        if (a.row_group) a.row_group[r] = gid - 1;
    }
    if (holds_last) {  // this thread holds the last row: its group ends there
        emit_group<NV>(a, gid - 1, cnt, w, vc);
        if (a.n_groups) *a.n_groups = gid;
    }
}

template <int NK, int NV>
cudaError_t seg_run(const SegArgs& a, unsigned char* aggs, uint32_t tiles, cudaStream_t s, Profiler* prof) {
    Agg<NV>* ta = reinterpret_cast<Agg<NV>*>(aggs);
    const uint32_t blocks = (tiles + kScanTiles - 1) / kScanTiles;
    Agg<NV>* bt = ta + tiles;
    if (prof) prof->begin(KC_SEGREDUCE, s);
    const uint32_t grid = (tiles + kSegTilesPerCta - 1) / kSegTilesPerCta;
    // the float + signed-integer value pair with two keys of fixed widths
    // (8+4, 4+8, 4+4 bytes) gets fully specialised kernels
    const bool fixed = NV == 2 && value_class_pattern(a) == 1;
    const int kwp = (fixed && NK == 2) ? key_width_pattern(a) : 0;
    const uint32_t wide_grid = (tiles + kSubTiles - 1) / kSubTiles;
    bool launched_tiles = false;
    if constexpr (NK == 2 && NV == 2) {
        launched_tiles = true;
        if (kwp == 0x48)
            k_seg_tiles_wide<NK, NV, 1, 0x48><<<wide_grid, kSegThreads, 0, s>>>(a, ta, tiles);
        else if (kwp == 0x84)
            k_seg_tiles_wide<NK, NV, 1, 0x84><<<wide_grid, kSegThreads, 0, s>>>(a, ta, tiles);
        else if (kwp == 0x44)
            k_seg_tiles_wide<NK, NV, 1, 0x44><<<wide_grid, kSegThreads, 0, s>>>(a, ta, tiles);
        else
            launched_tiles = false;
    }
    if (!launched_tiles) {
        if constexpr (NV == 2) {
            if (fixed) k_seg_tiles_wide<NK, NV, 1><<<wide_grid, kSegThreads, 0, s>>>(a, ta, tiles);
            else k_seg_tiles_wide<NK, NV, 0><<<wide_grid, kSegThreads, 0, s>>>(a, ta, tiles);
        } else {
            k_seg_tiles_wide<NK, NV, 0><<<wide_grid, kSegThreads, 0, s>>>(a, ta, tiles);
        }
    }
    if (prof) prof->end(KC_SEGREDUCE, s);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    if (prof) prof->begin(KC_SEGSCAN, s);
    k_seg_scan1<NV><<<blocks, kScanTiles, 0, s>>>(a, ta, bt, tiles);
    k_seg_scan2<NV><<<1, kScanTiles, 0, s>>>(a, bt, blocks);
    if (prof) prof->end(KC_SEGSCAN, s);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    if (prof) prof->begin(KC_SEGEMIT, s);
    if constexpr (NV <= 2)
    {
        bool launched_emit = false;
        if constexpr (NK == 2 && NV == 2) {
            launched_emit = true;
            if (kwp == 0x48)
                k_seg_emit_wide<NK, NV, 1, 0x48><<<wide_grid, kSegThreads, 0, s>>>(a, ta, bt, tiles);
            else if (kwp == 0x84)
                k_seg_emit_wide<NK, NV, 1, 0x84><<<wide_grid, kSegThreads, 0, s>>>(a, ta, bt, tiles);
            else if (kwp == 0x44)
                k_seg_emit_wide<NK, NV, 1, 0x44><<<wide_grid, kSegThreads, 0, s>>>(a, ta, bt, tiles);
            else
                launched_emit = false;
        }
        if (!launched_emit) {
            if constexpr (NV == 2) {
                if (fixed) k_seg_emit_wide<NK, NV, 1><<<wide_grid, kSegThreads, 0, s>>>(a, ta, bt, tiles);
                else k_seg_emit_wide<NK, NV, 0><<<wide_grid, kSegThreads, 0, s>>>(a, ta, bt, tiles);
            } else {
                k_seg_emit_wide<NK, NV, 0><<<wide_grid, kSegThreads, 0, s>>>(a, ta, bt, tiles);
            }
        }
    }
    else
        k_seg_emit<NK, NV><<<grid, kSegThreads, emit_smem_bytes<NK, NV>(), s>>>(a, ta, bt, tiles);
    if (prof) prof->end(KC_SEGEMIT, s);
    return cudaGetLastError();
}

template <int NK, int NV>
cudaError_t seg_attr() {
    constexpr size_t smem = emit_smem_bytes<NK, NV>();
    static_assert(smem <= 227 * 1024, "group-by shared memory exceeds the per-CTA limit");
    return cudaFuncSetAttribute(k_seg_emit<NK, NV>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
}

template <int NK>
cudaError_t seg_attrs() {
    cudaError_t e;
    if ((e = seg_attr<NK, 0>()) != cudaSuccess) return e;
    if ((e = seg_attr<NK, 1>()) != cudaSuccess) return e;
    if ((e = seg_attr<NK, 2>()) != cudaSuccess) return e;
    if ((e = seg_attr<NK, 3>()) != cudaSuccess) return e;
    return seg_attr<NK, 4>();
}

template <int NK>
cudaError_t seg_run_nv(const SegArgs& a, unsigned char* aggs, uint32_t tiles, cudaStream_t s, Profiler* prof) {
    switch (a.nvals) {
    case 0: return seg_run<NK, 0>(a, aggs, tiles, s, prof);
    case 1: return seg_run<NK, 1>(a, aggs, tiles, s, prof);
    case 2: return seg_run<NK, 2>(a, aggs, tiles, s, prof);
    case 3: return seg_run<NK, 3>(a, aggs, tiles, s, prof);
    default: return seg_run<NK, 4>(a, aggs, tiles, s, prof);
    }
}

size_t agg_bytes(int nvals) {
    switch (nvals) {
    case 0: return sizeof(Agg<0>);
    case 1: return sizeof(Agg<1>);
    case 2: return sizeof(Agg<2>);
    case 3: return sizeof(Agg<3>);
    default: return sizeof(Agg<4>);
    }
}

uint32_t seg_tiles(uint64_t n) { return (uint32_t)((n + kSegTile - 1) / kSegTile); }

}  // namespace

cudaError_t prepare_segreduce_kernels() {
    cudaError_t e;
    if ((e = seg_attrs<1>()) != cudaSuccess) return e;
    if ((e = seg_attrs<2>()) != cudaSuccess) return e;
    if ((e = seg_attrs<3>()) != cudaSuccess) return e;
    return seg_attrs<4>();
}

// [256 B][tile aggregates][CTA totals of the level-1 scan]
size_t segreduce_workspace_bytes(uint64_t n, int nvals) {
    const size_t tiles = seg_tiles(n);
    return 256 + (tiles + (tiles + kScanTiles - 1) / kScanTiles) * agg_bytes(nvals);
}

cudaError_t run_segreduce(SegArgs a, unsigned char* ws, cudaStream_t s, Profiler* prof, int* launches) {
    if (a.n == 0) {
        if (a.n_groups) return cudaMemsetAsync(a.n_groups, 0, sizeof(uint64_t), s);
        return cudaSuccess;
    }
    const uint32_t tiles = seg_tiles(a.n);
    cudaError_t e;
    switch (a.nkeys) {
    case 1: e = seg_run_nv<1>(a, ws + 256, tiles, s, prof); break;
    case 2: e = seg_run_nv<2>(a, ws + 256, tiles, s, prof); break;
    case 3: e = seg_run_nv<3>(a, ws + 256, tiles, s, prof); break;
    default: e = seg_run_nv<4>(a, ws + 256, tiles, s, prof); break;
    }
    if (launches) *launches += 4;
    return e;
}

}  // namespace vdf
