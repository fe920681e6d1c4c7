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
//   * a block scan gives each thread its in-tile prefix, and a decoupled
//     look-back over earlier tiles' published aggregates (32 predecessors
//     per warp step) gives the tile's global prefix: the number of groups
//     before it and the partial of the segment that runs into it;
//   * each thread then walks its rows once more and writes every segment
//     that ends inside its rows (keys, count, sum, min, max, mean).
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

#include "vdf_common.cuh"
#include "vdf_internal.h"

namespace vdf {

namespace {

enum VClass : int { VC_FLOAT = 0, VC_SINT = 1, VC_UINT = 2 };
__device__ __forceinline__ int vclass(int dt) {
    return (dt == F64 || dt == F32) ? VC_FLOAT : (dt == I32 || dt == I64) ? VC_SINT : VC_UINT;
}
__device__ __forceinline__ double as_f(uint64_t b) { return __longlong_as_double((long long)b); }
__device__ __forceinline__ uint64_t as_b(double d) { return (uint64_t)__double_as_longlong(d); }

// Canonical 64-bit image of a value: double bits for float columns, the
// sign- or zero-extended integer otherwise.
__device__ __forceinline__ uint64_t load_val(const void* src, int dt, uint64_t i) {
    switch (dt) {
    case I32: return (uint64_t)(int64_t)__ldg(static_cast<const int32_t*>(src) + i);
    case U32: return (uint64_t)__ldg(static_cast<const uint32_t*>(src) + i);
    case F32: return as_b((double)__ldg(static_cast<const float*>(src) + i));
    default: return (uint64_t)__ldg(static_cast<const unsigned long long*>(src) + i);
    }
}
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

// Per value column accumulator words:
//   float : w0 sum, w1 compensation, w2 min, w3 max   (double bits)
//   int   : w0 sum low, w1 sum high (128-bit two's complement), w2 min, w3 max
__device__ __forceinline__ void col_init(uint64_t* w, uint64_t x, int vc) {
    w[0] = x;
    w[1] = (vc == VC_SINT && (int64_t)x < 0) ? ~0ull : 0ull;  // 0.0 for floats
    w[2] = x;
    w[3] = x;
}
__device__ __forceinline__ void col_merge(uint64_t* a, const uint64_t* b, int vc) {
    if (vc == VC_FLOAT) {
        const double x = as_f(a[0]), y = as_f(b[0]);
        const double s = __dadd_rn(x, y);
        const double bp = __dsub_rn(s, x);
        const double e = __dadd_rn(__dsub_rn(x, __dsub_rn(s, bp)), __dsub_rn(y, bp));  // TwoSum error
        a[0] = as_b(s);
        a[1] = as_b(__dadd_rn(__dadd_rn(as_f(a[1]), as_f(b[1])), e));
        a[2] = as_b(fmin(as_f(a[2]), as_f(b[2])));
        a[3] = as_b(fmax(as_f(a[3]), as_f(b[3])));
    } else {
        const uint64_t lo = a[0] + b[0];
        a[1] = a[1] + b[1] + (lo < a[0] ? 1ull : 0ull);
        a[0] = lo;
        if (vc == VC_SINT) {
            a[2] = (uint64_t)min((long long)a[2], (long long)b[2]);
            a[3] = (uint64_t)max((long long)a[3], (long long)b[3]);
        } else {
            a[2] = min((unsigned long long)a[2], (unsigned long long)b[2]);
            a[3] = max((unsigned long long)a[3], (unsigned long long)b[3]);
        }
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

// Look-back record of one tile.  The aggregate and the inclusive prefix live
// in separate slots, each written once before its flag is raised, so a
// reader never sees a slot being overwritten.
constexpr uint32_t REC_AGG = 1, REC_INC = 2;
template <int NV>
struct Rec {
    uint32_t flag;
    uint32_t pad;
    Agg<NV> slot[2];  // [0] aggregate, [1] inclusive prefix
};

template <int NV>
__device__ __forceinline__ void rec_write(Rec<NV>* r, const Agg<NV>& a, uint32_t flag) {
    Agg<NV>* dst = &r->slot[flag == REC_INC ? 1 : 0];
    st_relaxed_u32(&dst->heads, a.heads);
    st_relaxed_u32(&dst->cnt, a.cnt);
#pragma unroll
    for (int v = 0; v < NV; ++v)
#pragma unroll
        for (int q = 0; q < 4; ++q) st_relaxed_u64(&dst->w[v][q], a.w[v][q]);
    __threadfence();
    st_release_u32(&r->flag, flag);
}
template <int NV>
__device__ __forceinline__ Agg<NV> rec_read(const Rec<NV>* r, uint32_t flag) {
    const Agg<NV>* src = &r->slot[flag == REC_INC ? 1 : 0];
    Agg<NV> a;
    a.heads = ld_relaxed_u32(&src->heads);
    a.cnt = ld_relaxed_u32(&src->cnt);
#pragma unroll
    for (int v = 0; v < NV; ++v)
#pragma unroll
        for (int q = 0; q < 4; ++q) a.w[v][q] = ld_relaxed_u64(&src->w[v][q]);
    if (NV == 0) a.w[0][0] = 0;
    return a;
}

__device__ __forceinline__ double i128_to_double(uint64_t lo, uint64_t hi, bool is_signed) {
    if (is_signed) {
        if ((int64_t)hi == ((int64_t)lo >> 63)) return (double)(int64_t)lo;
        return ldexp((double)(int64_t)hi, 64) + (double)lo;
    }
    if (hi == 0) return (double)lo;
    return ldexp((double)hi, 64) + (double)lo;
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
// 8 rows per lane: one byte of the head bitmap per lane, 256 rows per tile.
struct SegShape {
    static constexpr int ITEMS = 8;
    static constexpr int ROWS = 32 * ITEMS;  // rows per warp tile
};
constexpr int kSegThreads = 256;  // 8 independent warp tiles per CTA

// One WARP is one tile: it loads 32 x ITEMS consecutive rows (ITEMS per lane),
// scans them with shuffles, resolves its prefix with a decoupled look-back
// over earlier warp tiles and emits the groups that end in its rows.  There
// is no CTA-wide barrier, so while one warp waits on a predecessor's record
// the other resident warps keep the memory system busy.
// NK > 0: segment heads are found by comparing the NK key columns of
// adjacent rows (and written to a.heads_out, one bit per row, when set);
// NK == 0: they are read from a.heads_in, so a value column can be reduced
// in its own launch without re-reading the keys.
template <int NK, int NV>
__global__ void __launch_bounds__(kSegThreads, (NV > 0 || NK > 2) ? 3 : 4) k_segreduce(SegArgs a, uint32_t tiles) {
    constexpr int ITEMS = SegShape::ITEMS;
    constexpr int ROWS = SegShape::ROWS;
    const int lane = threadIdx.x & 31;
    uint32_t tile = 0;
    if (lane == 0) tile = atomicAdd(a.tile_counter, 1u);
    tile = __shfl_sync(0xffffffffu, tile, 0);
    if (tile >= tiles) return;  // whole warp
    const uint64_t n = a.n;
    const uint64_t row0 = (uint64_t)tile * ROWS + (uint64_t)lane * ITEMS;
    Rec<NV>* recs = reinterpret_cast<Rec<NV>*>(a.status);

    int vc[NV > 0 ? NV : 1];
#pragma unroll
    for (int v = 0; v < NV; ++v) vc[v] = vclass(a.val[v].dtype);
    int kw[NK > 0 ? NK : 1];
#pragma unroll
    for (int k = 0; k < NK; ++k) kw[k] = dtype_width(a.key[k].dtype);

    // ---- phase A: load this lane's rows, find segment heads, fold ----------
    uint32_t hmask = 0;
    Agg<NV> t = agg_identity<NV>();
    {
        uint64_t val[ITEMS][NV > 0 ? NV : 1];
#pragma unroll
        for (int v = 0; v < NV; ++v) load_vals<ITEMS>(a.val[v].src, a.val[v].dtype, row0, n, val, v);
        if (NK == 0) {
            hmask = row0 < n ? a.heads_in[(uint64_t)tile * 32 + lane] : 0u;
        } else {
            uint64_t key[ITEMS][NK > 0 ? NK : 1];
#pragma unroll
            for (int k = 0; k < NK; ++k) load_rows<ITEMS>(a.key[k].src, kw[k], row0, n, key, k);
            uint64_t prev[NK > 0 ? NK : 1];
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
            if (a.heads_out) a.heads_out[(uint64_t)tile * 32 + lane] = (uint8_t)hmask;
        }
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
    }

    // ---- warp scan and decoupled look-back -------------------------------
    Agg<NV> incl = t;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const Agg<NV> o = agg_shfl_up(incl, d);
        if (lane >= d) incl = agg_combine(o, incl, vc);
    }
    Agg<NV> X = agg_identity<NV>();
    {
        const Agg<NV> total = agg_shfl(incl, 31);
        if (tile == 0) {
            if (lane == 0) rec_write(&recs[0], total, REC_INC);
        } else {
            if (lane == 0) rec_write(&recs[tile], total, REC_AGG);
            int64_t base = (int64_t)tile - 1;
            while (true) {
                const int64_t p = base - lane;
                uint32_t f = REC_INC;
                if (p >= 0) {
                    uint32_t spins = 0;
                    while ((f = ld_acquire_u32(&recs[p].flag)) == 0) {
                        if (++spins > kSpinLimit) { atomicOr(a.err, ERR_LOOKBACK_TIMEOUT); f = REC_INC; break; }
                        backoff(spins);
                    }
                }
                const uint32_t incmask = __ballot_sync(0xffffffffu, f == REC_INC);
                const int stop = incmask ? __ffs(incmask) - 1 : 31;
                Agg<NV> r = agg_identity<NV>();
                if (p >= 0 && lane <= stop) r = rec_read(&recs[p], f);
                // chronological fold: higher lanes are older tiles
#pragma unroll
                for (int d = 1; d < 32; d <<= 1) {
                    const Agg<NV> o = agg_shfl_down(r, d);
                    if (lane + d < 32) r = agg_combine(o, r, vc);
                }
                X = agg_combine(agg_shfl(r, 0), X, vc);
                if (incmask) break;
                base -= 32;
            }
            if (lane == 0) rec_write(&recs[tile], agg_combine(X, total, vc), REC_INC);
        }
    }
    Agg<NV> lane_excl = agg_shfl_up(incl, 1);
    if (lane == 0) lane_excl = agg_identity<NV>();
    const Agg<NV> pre = agg_combine(X, lane_excl, vc);

    // ---- phase B: emit the segments that end in this lane's rows -------------
    // Every row contributes at most one head, so a prefix claiming more heads
    // (or a longer open segment) than rows before row0 can only come from a
    // timed-out look-back: record it and write nothing rather than out of bounds.
    if (row0 < n && (pre.heads > row0 || pre.cnt > row0 || (row0 > 0 && pre.heads == 0))) {
        atomicOr(a.err, ERR_BAD_INDEX);
        return;
    }
    uint32_t gid = pre.heads;
    uint32_t cnt = pre.cnt;
    uint64_t w[NV > 0 ? NV : 1][4];
#pragma unroll
    for (int v = 0; v < NV; ++v)
#pragma unroll
        for (int q = 0; q < 4; ++q) w[v][q] = pre.w[v][q];
#pragma unroll
    for (int j = 0; j < ITEMS; ++j) {
        const uint64_t r = row0 + j;
        if (r >= n) break;
        uint64_t val[NV > 0 ? NV : 1];
#pragma unroll
        for (int v = 0; v < NV; ++v) val[v] = load_val(a.val[v].src, a.val[v].dtype, r);
        if ((hmask >> j) & 1u) {
            if (gid > 0) emit_group<NV>(a, gid - 1, cnt, w, vc);
            ++gid;
#pragma unroll
            for (int k = 0; k < NK; ++k)
                if (a.key_out[k]) store_raw(a.key_out[k], kw[k], gid - 1, load_raw(a.key[k].src, kw[k], r));
            if (a.group_start) a.group_start[gid - 1] = (uint32_t)r;
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
        if (a.row_group) a.row_group[r] = gid - 1;
        if (r == n - 1) {
            emit_group<NV>(a, gid - 1, cnt, w, vc);
            if (a.n_groups) *a.n_groups = gid;
        }
    }
}

template <int NK, int NV>
cudaError_t launch_seg(const SegArgs& a, uint32_t tiles, cudaStream_t s) {
    const uint32_t blocks = (tiles + kSegThreads / 32 - 1) / (kSegThreads / 32);
    k_segreduce<NK, NV><<<blocks, kSegThreads, 0, s>>>(a, tiles);
    return cudaGetLastError();
}

cudaError_t launch_heads(const SegArgs& a, uint32_t tiles, cudaStream_t s) {
    switch (a.nkeys) {
    case 1: return launch_seg<1, 0>(a, tiles, s);
    case 2: return launch_seg<2, 0>(a, tiles, s);
    case 3: return launch_seg<3, 0>(a, tiles, s);
    default: return launch_seg<4, 0>(a, tiles, s);
    }
}

size_t rec_bytes(int nvals) {
    switch (nvals) {
    case 0: return sizeof(Rec<0>);
    case 1: return sizeof(Rec<1>);
    case 2: return sizeof(Rec<2>);
    case 3: return sizeof(Rec<3>);
    default: return sizeof(Rec<4>);
    }
}

}  // namespace

cudaError_t prepare_segreduce_kernels() { return cudaSuccess; }

uint32_t seg_tiles(uint64_t n) { return (uint32_t)((n + SegShape::ROWS - 1) / SegShape::ROWS); }

// [counter+err 256 B][head bitmap: 32 B per tile][look-back records]
size_t segreduce_workspace_bytes(uint64_t n, int nvals) {
    (void)nvals;
    const size_t tiles = seg_tiles(n);
    return 256 + tiles * 32 + tiles * std::max(rec_bytes(0), rec_bytes(1));
}

// The keys pass (group boundaries, keys, counts, group starts, row groups,
// head bitmap) runs first; then one launch per value column reads the head
// bitmap and that column.  Each launch carries only its own small scan state.
cudaError_t run_segreduce(SegArgs a, unsigned char* ws, cudaStream_t s, Profiler* prof, int* launches) {
    cudaError_t e;
    if (a.n == 0) {
        if (a.n_groups) return cudaMemsetAsync(a.n_groups, 0, sizeof(uint64_t), s);
        return cudaSuccess;
    }
    const uint32_t tiles = seg_tiles(a.n);
    uint8_t* bitmap = ws + 256;
    unsigned char* recs = bitmap + (size_t)tiles * 32;
    a.tile_counter = reinterpret_cast<uint32_t*>(ws);
    a.status = recs;
    a.heads_out = bitmap;
    a.heads_in = bitmap;
    const size_t rb0 = rec_bytes(0), rb1 = rec_bytes(1);
    if ((e = cudaMemsetAsync(ws, 0, 256, s)) != cudaSuccess) return e;
    if ((e = cudaMemsetAsync(recs, 0, (size_t)tiles * rb0, s)) != cudaSuccess) return e;
    SegArgs k1 = a;
    k1.nvals = 0;
    if (prof) prof->begin(KC_SEGREDUCE, s);
    e = launch_heads(k1, tiles, s);
    if (prof) prof->end(KC_SEGREDUCE, s);
    if (launches) ++*launches;
    if (e != cudaSuccess) return e;
    for (int v = 0; v < a.nvals; ++v) {
        if ((e = cudaMemsetAsync(ws, 0, 4, s)) != cudaSuccess) return e;
        if ((e = cudaMemsetAsync(recs, 0, (size_t)tiles * rb1, s)) != cudaSuccess) return e;
        SegArgs k2{};
        k2.n = a.n;
        k2.nkeys = 0;
        k2.nvals = 1;
        k2.val[0] = a.val[v];
        k2.agg[0] = a.agg[v];
        k2.heads_in = bitmap;
        k2.tile_counter = a.tile_counter;
        k2.status = recs;
        k2.err = a.err;
        if (prof) prof->begin(KC_SEGREDUCE, s);
        e = launch_seg<0, 1>(k2, tiles, s);
        if (prof) prof->end(KC_SEGREDUCE, s);
        if (launches) ++*launches;
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

}  // namespace vdf
