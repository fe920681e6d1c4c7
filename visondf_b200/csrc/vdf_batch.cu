// vdf_batch.cu -- many independent sort + group-by queries as one unit of
// device work.
//
// The reference runs one query per call (sort_by_mt.hpp:3-180 then
// transform_group_by_onecol_mt.hpp:14-373, each an OpenMP region over one
// frame).  A batch here is planned once on the host and then enqueued as a
// fixed sequence of launches that touch no host memory, so it can be captured
// into a CUDA graph and replayed:
//
//   small queries  (rows <= tuning.small_rows): one persistent kernel, one
//                  CTA per query at a time, sorting and grouping the query in
//                  shared memory (vdf_batch_small.cu);
//   large queries: packed back to back into an arena of ordered 8-byte keys
//                  (the query index is the segment), sorted by the segmented
//                  radix passes (tiles never straddle a query, each query has
//                  its own histograms and pass count), payload-gathered, and
//                  grouped by the segmented reduction over (segment, key), so
//                  no group spans two queries.  Two small kernels then turn
//                  arena row ids into per-query row ids and record each
//                  query's group range.
//
// Output layout (arena): query q owns rows [row_offset[q], row_offset[q] +
// n_q) of perm_out and group slots [group_offset[q], group_offset[q] +
// n_groups[q]) of the group arrays; its group keys are packed in its own key
// width starting at byte 8 * group_offset[q] of group_keys_out.
#include <algorithm>
#include <cstring>

#include "vdf_ctx.h"
#include "vdf_batch.h"

namespace vdf {
namespace {

// A 4-byte key's image has a zero high half, so it also fits a 4-byte arena.
__device__ __forceinline__ uint64_t ordered_image(const void* col, uint64_t i, int dt) {
    switch (dt) {
    case I32: case U32: case F32:
        return (uint64_t)order32(__ldg(static_cast<const uint32_t*>(col) + i), dt, false);
    default:
        return order64(__ldg(static_cast<const uint64_t*>(col) + i), dt, false);
    }
}

// Copies each large query's rows into the arena: ordered key image (8 or 4
// bytes), segment index, and the value columns; one CTA per chunk of one
// segment.
__global__ void __launch_bounds__(256) k_batch_pack(BatchDev b) {
    const SegChunk ch = b.chunks[blockIdx.x];
    if (ch.seg >= b.nsegs) return;
    const SegDesc sd = b.segs[ch.seg];
    const BatchQuery q = b.queries[b.seg_query[ch.seg]];
    if (ch.row_start < sd.row_start || ch.row_start + ch.rows > sd.row_start + sd.rows ||
        sd.row_start + sd.rows > b.n_large) {
        if (threadIdx.x == 0) atomicOr(b.err, ERR_BAD_INDEX);
        return;
    }
    // four rows per thread per round (rows k * blockDim + thread, so every
    // load and store instruction is coalesced), all loads issued before the
    // stores
    constexpr int R = 4;
    const uint32_t step = blockDim.x * R;
    for (uint32_t r0 = 0; r0 < ch.rows; r0 += step) {
        uint64_t kimg[R];
        unsigned long long slot[R][VDF_BATCH_MAX_VALS];
#pragma unroll
        for (int k = 0; k < R; ++k) {
            const uint32_t r = r0 + k * blockDim.x + threadIdx.x;
            kimg[k] = 0;
#pragma unroll
            for (int j = 0; j < VDF_BATCH_MAX_VALS; ++j) slot[k][j] = 0;
            if (r >= ch.rows) continue;
            const uint64_t local = ch.row_start + r - sd.row_start;  // row within the query
            kimg[k] = ordered_image(q.key, local, q.key_dtype);
#pragma unroll
            for (int j = 0; j < VDF_BATCH_MAX_VALS; ++j)
                if (j < b.nvals)
                    slot[k][j] = b.val_width[j] == 8
                                     ? __ldg(static_cast<const unsigned long long*>(q.vals[j]) + local)
                                     : (unsigned long long)__ldg(static_cast<const uint32_t*>(q.vals[j]) + local);
        }
#pragma unroll
        for (int k = 0; k < R; ++k) {
            const uint32_t r = r0 + k * blockDim.x + threadIdx.x;
            if (r >= ch.rows) continue;
            const uint64_t i = ch.row_start + r;  // arena row
            if (b.key_width == 8) static_cast<uint64_t*>(b.arena_keys)[i] = kimg[k];
            else static_cast<uint32_t*>(b.arena_keys)[i] = (uint32_t)kimg[k];
            b.arena_seg[i] = ch.seg;
            if (b.rec_bytes) {
                // the packed gather's record: 8-byte slots, zero-extended
                ulonglong2* dst = reinterpret_cast<ulonglong2*>(b.arena_recs + i * (uint64_t)b.rec_bytes);
                dst[0] = make_ulonglong2(slot[k][0], slot[k][1]);
                if (b.rec_bytes == 32) dst[1] = make_ulonglong2(slot[k][2], slot[k][3]);
            } else {
#pragma unroll
                for (int j = 0; j < VDF_BATCH_MAX_VALS; ++j) {
                    if (j >= b.nvals) break;
                    if (b.val_width[j] == 8) static_cast<uint64_t*>(b.arena_vals[j])[i] = slot[k][j];
                    else static_cast<uint32_t*>(b.arena_vals[j])[i] = (uint32_t)slot[k][j];
                }
            }
        }
    }
}

// Sorted arena row ids -> row ids within each query (in place in perm_out).
__global__ void __launch_bounds__(256) k_batch_localize(BatchDev b) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    // four rows per thread per round, every load issued before the first use
    constexpr int R = 4;
    for (uint64_t i0 = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i0 < b.n_large; i0 += R * stride) {
        uint32_t sg[R], rr[R];
#pragma unroll
        for (int q = 0; q < R; ++q) {
            const uint64_t i = i0 + q * stride;
            sg[q] = 0;
            rr[q] = 0;
            if (i < b.n_large) {
                sg[q] = b.arena_seg[i];  // the sort keeps every segment in place
                rr[q] = b.perm_out[b.large_base + i];
            }
        }
#pragma unroll
        for (int q = 0; q < R; ++q) {
            const uint64_t i = i0 + q * stride;
            if (i >= b.n_large) break;
            if (sg[q] >= b.nsegs) {
                atomicOr(b.err, ERR_BAD_INDEX);
                continue;
            }
            const SegDesc d = b.segs[sg[q]];
            if (rr[q] < d.row_start || rr[q] - d.row_start >= d.rows) {
                atomicOr(b.err, ERR_BAD_INDEX);
                continue;
            }
            b.perm_out[b.large_base + i] = (uint32_t)(rr[q] - d.row_start);
        }
    }
}

// Per segment: its first group and group count (binary search over the
// ascending group segment ids), written to the query's outputs.
__global__ void __launch_bounds__(256) k_batch_seg_groups(BatchDev b) {
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= b.nsegs) return;
    const uint64_t G = *b.n_groups_large;
    uint64_t lo = 0, hi = G;
    while (lo < hi) {
        const uint64_t mid = (lo + hi) >> 1;
        if (b.group_seg[mid] < s) lo = mid + 1; else hi = mid;
    }
    const uint64_t first = lo;
    hi = G;
    while (lo < hi) {
        const uint64_t mid = (lo + hi) >> 1;
        if (b.group_seg[mid] <= s) lo = mid + 1; else hi = mid;
    }
    b.seg_first_group[s] = (uint32_t)first;
    const uint32_t q = b.seg_query[s];
    b.group_offset_out[q] = b.large_base + first;
    b.n_groups_out[q] = lo - first;
}

// Group keys of the large queries: ordered image -> the query's own dtype,
// packed in its width at byte 8 * group_offset of the key arena.
__global__ void __launch_bounds__(256) k_batch_group_keys(BatchDev b) {
    const uint64_t G = *b.n_groups_large;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    unsigned char* out = static_cast<unsigned char*>(b.group_keys_out);
    for (uint64_t g = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; g < G; g += stride) {
        const uint32_t s = b.group_seg[g];
        if (s >= b.nsegs) {
            atomicOr(b.err, ERR_BAD_INDEX);
            continue;
        }
        const uint32_t first = b.seg_first_group[s];
        const int dt = b.queries[b.seg_query[s]].key_dtype;
        const uint64_t img = b.key_width == 8 ? static_cast<const uint64_t*>(b.group_key_img)[g]
                                              : static_cast<const uint32_t*>(b.group_key_img)[g];
        unsigned char* base = out + 8 * (b.large_base + first);
        if (dtype_width(dt) == 4)
            reinterpret_cast<uint32_t*>(base)[g - first] = unorder32((uint32_t)img, dt, false);
        else
            reinterpret_cast<uint64_t*>(base)[g - first] = unorder64(img, dt, false);
    }
}

inline size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

uint32_t grid_for(uint64_t n, int sms) {
    uint64_t want = (n + 255) / 256;
    uint64_t cap = (uint64_t)sms * 8;
    return (uint32_t)std::max<uint64_t>(1, std::min(want, cap));
}

}  // namespace

// segmented variant 4 (8-bit digits, 256 x 12 keys, four CTAs per SM) measured
// fastest for both key widths on the batch and request-stream workloads
BatchTuning default_batch_tuning() { return BatchTuning{4096, 8, 4}; }

bool batch_tuning_valid(const BatchTuning& t) {
    int bits, tile;
    return seg_sort_variant_info(t.seg_variant, &bits, &tile) && (t.small_bits == 4 || t.small_bits == 8) &&
           t.small_rows <= kSmallMaxRows;
}

// Host-side plan: classifies the queries, lays out the arena and the tables,
// and sizes the workspace.  Everything device-side is relative to `ws`.
bool plan_batch(BatchPlan& P, const vdf_batch_args& a, const BatchTuning& t, std::string& why, int msd,
                int msd_match) {
    P = BatchPlan{};
    P.tuning = t;
    P.msd_match = msd_match;
    P.nq = a.nqueries;
    P.nvals = a.nvals;
    int bits = 8, tile = 2048;
    seg_sort_variant_info(t.seg_variant, &bits, &tile);
    P.tile_rows = (uint32_t)tile;
    P.key_width = 4;
    for (int j = 0; j < a.nvals; ++j) P.val_width[j] = dtype_width(a.val_dtypes[j]);

    // small queries first (in query order), then large ones with 8-byte keys,
    // then large ones with 4-byte keys (segments with more passes first)
    std::vector<uint32_t> small, large8, large4;
    for (uint32_t q = 0; q < a.nqueries; ++q) {
        const vdf_batch_query& Q = a.queries[q];
        if (Q.n == 0) continue;
        if (Q.n <= t.small_rows) small.push_back(q);
        else if (dtype_width(Q.key.dtype) == 8) large8.push_back(q);
        else large4.push_back(q);
    }
    if (!large8.empty()) P.key_width = 8;  // one 8-byte key widens every image
    P.row_offset.assign(a.nqueries, 0);
    uint64_t off = 0;
    for (uint32_t q : small) { P.row_offset[q] = off; off += a.queries[q].n; }
    P.n_small = off;
    P.small_queries = small;
    const uint64_t large_base = off;
    P.large_base = large_base;
    std::vector<uint32_t> large = large8;
    large.insert(large.end(), large4.begin(), large4.end());
    uint32_t tiles = 0;
    int maxp = 0;
    for (uint32_t s = 0; s < large.size(); ++s) {
        const uint32_t q = large[s];
        const uint64_t n = a.queries[q].n;
        P.row_offset[q] = off;
        SegDesc d{};
        d.row_start = off - large_base;
        d.rows = (uint32_t)n;
        d.first_tile = tiles;
        d.passes = (uint32_t)((dtype_width(a.queries[q].key.dtype) * 8 + bits - 1) / bits);
        maxp = std::max(maxp, (int)d.passes);
        const uint32_t nt = (uint32_t)((n + tile - 1) / tile);
        for (uint32_t k = 0; k < nt; ++k) P.tile_seg.push_back(s);
        tiles += nt;
        for (uint64_t r = 0; r < n; r += kChunkRows) {
            SegChunk c{};
            c.row_start = d.row_start + r;
            c.rows = (uint32_t)std::min<uint64_t>(kChunkRows, n - r);
            c.seg = s;
            P.chunks.push_back(c);
        }
        P.segs.push_back(d);
        P.seg_query.push_back(q);
        off += n;
    }
    for (uint32_t q = 0; q < a.nqueries; ++q)
        if (a.queries[q].n == 0) P.row_offset[q] = off;  // empty: no rows, no groups
    P.n_total = off;
    P.n_large = off - large_base;
    P.max_passes = maxp;
    for (int g = 0; g < 16; ++g) {
        uint32_t c = 0;
        for (const SegDesc& d : P.segs)
            if ((int)d.passes > g) c += (uint32_t)((d.rows + tile - 1) / tile);
        P.tiles_in_pass[g] = c;
    }
    if (P.n_total > kMaxBatchRows) {
        why = "batch of " + std::to_string(P.n_total) + " rows exceeds the row limit";
        return false;
    }

    // MSD-first tables: segment s with D digits and P = msd_passes_for top
    // digits sorts by digits D-P .. D-1 first; its chunks start every
    // kMsdCap / 2 rows (moved forward to a bucket boundary on the device).
    // Taken (msd 1) where it saves time: 8-byte keys (P of 8 passes, then
    // the shared-memory finish); the top digits of a 4-byte key plus the
    // finish measured slower than its four LSD passes on served batches.
    // msd 2 takes it for every width.
    P.seg_flag_init.assign(P.segs.size(), 1);
    if (msd && bits == 8) {
        std::vector<uint32_t> order;
        std::vector<int> mp(P.segs.size(), 0);
        for (uint32_t s = 0; s < P.segs.size(); ++s) {
            const int w = dtype_width(a.queries[P.seg_query[s]].key.dtype);
            mp[s] = msd_passes_for(P.segs[s].rows, w);
            if (w == 4 && msd != 2) mp[s] = 0;
            if (mp[s] > 0) order.push_back(s);
        }
        std::stable_sort(order.begin(), order.end(), [&](uint32_t x, uint32_t y) { return mp[x] > mp[y]; });
        uint32_t mt = 0;
        for (uint32_t i = 0; i < order.size(); ++i) {
            const uint32_t s = order[i];
            const SegDesc& d0 = P.segs[s];
            SegDesc d = d0;
            d.first_tile = mt;
            d.passes = (uint32_t)mp[s];
            d.first_digit = d0.passes - (uint32_t)mp[s];
            const uint32_t nt = (uint32_t)((d.rows + tile - 1) / tile);
            for (uint32_t k = 0; k < nt; ++k) P.msd_tile_seg.push_back(i);
            mt += nt;
            for (uint64_t r = 0; r < d.rows; r += kChunkRows) {
                SegChunk c{};
                c.row_start = d.row_start + r;
                c.rows = (uint32_t)std::min<uint64_t>(kChunkRows, d.rows - r);
                c.seg = i;
                P.msd_hist_chunks.push_back(c);
            }
            P.msd_segs.push_back(d);
            P.msd_seg_of.push_back(s);
            P.msd_max_passes = std::max(P.msd_max_passes, mp[s]);
            P.seg_flag_init[s] = 0;
        }
        for (uint32_t s = 0; s < P.segs.size(); ++s) {  // chunks in arena order
            if (mp[s] == 0) continue;
            const SegDesc& d = P.segs[s];
            for (uint64_t r = 0; r < d.rows; r += kMsdCap / 2) {
                MsdSegChunk c{};
                c.x = (uint32_t)(d.row_start + r);
                c.seg_start = (uint32_t)d.row_start;
                c.seg_end = (uint32_t)(d.row_start + d.rows);
                c.pshift = 8u * (d.passes - (uint32_t)mp[s]);
                c.seg = s;
                P.msd_chunks.push_back(c);
            }
        }
        for (int g = 0; g < 16; ++g) {
            uint32_t c = 0;
            for (const SegDesc& d : P.msd_segs)
                if ((int)d.passes > g) c += (uint32_t)((d.rows + tile - 1) / tile);
            P.msd_tiles_in_pass[g] = c;
        }
        P.msd_queries = (uint32_t)order.size();
        P.msd = !order.empty();
    }

    // workspace layout
    const size_t A = 256;
    size_t o = 0;
    const uint64_t nl = P.n_large;
    P.o_queries = o; o = align_up(o + sizeof(BatchQuery) * std::max<size_t>(1, a.nqueries), A);
    P.o_segs = o; o = align_up(o + sizeof(SegDesc) * std::max<size_t>(1, P.segs.size()), A);
    P.o_seg_query = o; o = align_up(o + 4 * std::max<size_t>(1, P.segs.size()), A);
    P.o_tile_seg = o; o = align_up(o + 4 * std::max<size_t>(1, P.tile_seg.size()), A);
    P.o_chunks = o; o = align_up(o + sizeof(SegChunk) * std::max<size_t>(1, P.chunks.size()), A);
    P.o_small = o; o = align_up(o + 4 * std::max<size_t>(1, small.size()), A);
    P.o_msd_segs = o; o = align_up(o + sizeof(SegDesc) * std::max<size_t>(1, P.msd_segs.size()), A);
    P.o_msd_tile_seg = o; o = align_up(o + 4 * std::max<size_t>(1, P.msd_tile_seg.size()), A);
    P.o_msd_hist_chunks = o; o = align_up(o + sizeof(SegChunk) * std::max<size_t>(1, P.msd_hist_chunks.size()), A);
    P.o_msd_chunks = o; o = align_up(o + sizeof(MsdSegChunk) * std::max<size_t>(1, P.msd_chunks.size()), A);
    P.o_flag_init = o; o = align_up(o + 4 * std::max<size_t>(1, P.segs.size()), A);
    P.desc_bytes = o;
    P.o_counters = o; o = align_up(o + 64, A);  // [0]: small-kernel work counter, [8]: large group count
    P.o_seg_flag = o; o = align_up(o + 4 * std::max<size_t>(1, P.segs.size()), A);
    P.o_chunk_start = o; o = align_up(o + 4 * (P.msd_chunks.size() + 1), A);
    P.o_seg_first = o; o = align_up(o + 4 * std::max<size_t>(1, P.segs.size()), A);
    const size_t kw = (size_t)P.key_width;
    P.o_arena_keys = o; o = align_up(o + kw * nl, A);
    P.o_arena_seg = o; o = align_up(o + 4 * nl, A);
    P.rec_bytes = gather_record_bytes(a.nvals);  // 0 for fewer than two value columns
    if (P.rec_bytes) {
        P.o_arena_recs = o;
        o = align_up(o + P.rec_bytes * nl, A);
    } else {
        for (int j = 0; j < a.nvals; ++j) { P.o_arena_vals[j] = o; o = align_up(o + (size_t)P.val_width[j] * nl, A); }
    }
    P.o_sorted_keys = o; o = align_up(o + kw * nl, A);
    for (int j = 0; j < a.nvals; ++j) { P.o_sorted_vals[j] = o; o = align_up(o + (size_t)P.val_width[j] * nl, A); }
    P.o_group_seg = o; o = align_up(o + 4 * nl, A);
    P.o_group_key = o; o = align_up(o + kw * nl, A);
    P.o_tail = o;
    size_t tail = seg_sort_workspace_bytes(nl, (uint32_t)P.segs.size(), (uint32_t)P.tile_seg.size(),
                                           std::max(1, maxp), t.seg_variant, P.key_width);
    if (P.msd)
        tail = std::max(tail, seg_sort_workspace_bytes(nl, (uint32_t)P.msd_segs.size(), (uint32_t)P.msd_tile_seg.size(),
                                                       P.msd_max_passes, t.seg_variant, P.key_width));
    tail = std::max(tail, segreduce_workspace_bytes(nl, a.nvals));
    P.ws_bytes = o + tail;
    return true;
}

// Fills the device-side view of the plan for a workspace at `ws`.
BatchDev batch_dev_view(const BatchPlan& P, const vdf_batch_args& a, unsigned char* ws, uint32_t* err) {
    BatchDev b{};
    b.queries = reinterpret_cast<const BatchQuery*>(ws + P.o_queries);
    b.segs = reinterpret_cast<const SegDesc*>(ws + P.o_segs);
    b.seg_query = reinterpret_cast<const uint32_t*>(ws + P.o_seg_query);
    b.chunks = reinterpret_cast<const SegChunk*>(ws + P.o_chunks);
    b.small_queries = reinterpret_cast<const uint32_t*>(ws + P.o_small);
    b.n_small_queries = (uint32_t)P.small_queries.size();
    b.work_counter = reinterpret_cast<uint32_t*>(ws + P.o_counters);
    b.n_groups_large = reinterpret_cast<uint64_t*>(ws + P.o_counters + 8);
    b.seg_first_group = reinterpret_cast<uint32_t*>(ws + P.o_seg_first);
    b.nsegs = (uint32_t)P.segs.size();
    b.nvals = P.nvals;
    for (int j = 0; j < P.nvals; ++j) {
        b.val_width[j] = P.val_width[j];
        b.val_dtype[j] = a.val_dtypes[j];
        b.arena_vals[j] = P.rec_bytes ? nullptr : ws + P.o_arena_vals[j];
        b.aggs[j] = a.aggs[j];
    }
    b.arena_recs = P.rec_bytes ? ws + P.o_arena_recs : nullptr;
    b.rec_bytes = (int)P.rec_bytes;
    b.arena_keys = ws + P.o_arena_keys;
    b.key_width = P.key_width;
    b.arena_seg = reinterpret_cast<uint32_t*>(ws + P.o_arena_seg);
    b.group_seg = reinterpret_cast<uint32_t*>(ws + P.o_group_seg);
    b.group_key_img = ws + P.o_group_key;
    b.n_large = P.n_large;
    b.large_base = P.large_base;
    b.perm_out = a.perm_out;
    b.group_keys_out = a.group_keys_out;
    b.group_count_out = a.group_count_out;
    b.group_offset_out = a.group_offset_out;
    b.n_groups_out = a.n_groups_out;
    b.small_bits = P.tuning.small_bits;
    b.small_cap = P.tuning.small_rows;
    b.err = err;
    return b;
}

cudaError_t launch_batch(const BatchPlan& P, const vdf_batch_args& a, unsigned char* ws, uint32_t* err,
                         cudaStream_t s, cudaStream_t side, cudaEvent_t fork, cudaEvent_t join, Profiler* prof,
                         int* launches) {
    cudaError_t e;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const BatchDev b = batch_dev_view(P, a, ws, err);
    int n = 0;

    // small queries on the side stream, overlapping the large-query pipeline
    const bool have_small = !P.small_queries.empty();
    if (have_small) {
        if ((e = cudaMemsetAsync(b.work_counter, 0, 4, s)) != cudaSuccess) return e;
        if ((e = cudaEventRecord(fork, s)) != cudaSuccess) return e;
        if ((e = cudaStreamWaitEvent(side, fork, 0)) != cudaSuccess) return e;
        if ((e = launch_small_queries(b, side, sms)) != cudaSuccess) return e;
        ++n;
        if ((e = cudaEventRecord(join, side)) != cudaSuccess) return e;
    }

    if (P.n_large) {
        if (prof) prof->begin(KC_PACK, s);
        k_batch_pack<<<(uint32_t)P.chunks.size(), 256, 0, s>>>(b);
        if (prof) prof->end(KC_PACK, s);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
        ++n;
        SegSortArgs sa{};
        sa.n = P.n_large;
        sa.keys = b.arena_keys;
        sa.key_width = P.key_width;
        sa.segs = b.segs;
        sa.nsegs = b.nsegs;
        sa.tile_seg = reinterpret_cast<const uint32_t*>(ws + P.o_tile_seg);
        sa.ntiles = (uint32_t)P.tile_seg.size();
        sa.chunks = b.chunks;
        sa.nchunks = (uint32_t)P.chunks.size();
        sa.max_passes = P.max_passes;
        for (int g = 0; g < 16; ++g) sa.tiles_in_pass[g] = P.tiles_in_pass[g];
        sa.variant = P.tuning.seg_variant;
        sa.keys_out = ws + P.o_sorted_keys;
        sa.perm_out = a.perm_out + P.large_base;
        sa.err = err;
        unsigned char* tail = ws + P.o_tail;
        if (P.msd) {
            // top-digit passes of the MSD segments straight into the sorted
            // buffers, then each chunk of whole buckets is finished in place
            // (a CTA reads its rows before it writes them)
            uint32_t* flags = reinterpret_cast<uint32_t*>(ws + P.o_seg_flag);
            if ((e = cudaMemcpyAsync(flags, ws + P.o_flag_init, 4 * P.segs.size(), cudaMemcpyDeviceToDevice, s)) !=
                cudaSuccess)
                return e;
            SegSortArgs ma = sa;
            ma.segs = reinterpret_cast<const SegDesc*>(ws + P.o_msd_segs);
            ma.nsegs = (uint32_t)P.msd_segs.size();
            ma.tile_seg = reinterpret_cast<const uint32_t*>(ws + P.o_msd_tile_seg);
            ma.ntiles = (uint32_t)P.msd_tile_seg.size();
            ma.chunks = reinterpret_cast<const SegChunk*>(ws + P.o_msd_hist_chunks);
            ma.nchunks = (uint32_t)P.msd_hist_chunks.size();
            ma.max_passes = P.msd_max_passes;
            for (int g = 0; g < 16; ++g) ma.tiles_in_pass[g] = P.msd_tiles_in_pass[g];
            if ((e = run_seg_sort(ma, tail, s, prof)) != cudaSuccess) return e;
            n += 2;
            for (int g = 0; g < P.msd_max_passes; ++g) n += P.msd_tiles_in_pass[g] ? 1 : 0;
            uint32_t* chunk_start = reinterpret_cast<uint32_t*>(ws + P.o_chunk_start);
            const uint32_t nch = (uint32_t)P.msd_chunks.size();
            const MsdSegChunk* sc = reinterpret_cast<const MsdSegChunk*>(ws + P.o_msd_chunks);
            MsdChunkArgs ca{};
            ca.keys = sa.keys_out;
            ca.n = P.n_large;
            ca.nchunks = nch;
            ca.chunk_start = chunk_start;
            ca.seg_chunks = sc;
            ca.seg_flag = flags;
            if (prof) prof->begin(KC_LOCALSORT, s);
            e = msd_chunks(ca, P.key_width, s);
            if (e == cudaSuccess) {
                MsdLocalArgs la{};
                la.keys = sa.keys_out;
                la.vals = sa.perm_out;
                la.chunk_start = chunk_start;
                la.n = P.n_large;
                la.dtype = P.key_width == 8 ? U64 : U32;  // the arena holds order images
                la.err = err;
                la.keys_out = sa.keys_out;
                la.perm_out = sa.perm_out;
                la.seg_chunks = sc;
                la.seg_flag = flags;
                e = msd_local(la, P.key_width, nch, P.msd_match & 1, s);
            }
            if (prof) prof->end(KC_LOCALSORT, s);
            if (e != cudaSuccess) return e;
            n += 2;
            sa.seg_flag = flags;  // the LSD passes: planned and failed segments only
        }
        if ((e = run_seg_sort(sa, tail, s, prof)) != cudaSuccess) return e;
        n += 2;
        for (int g = 0; g < P.max_passes; ++g) n += P.tiles_in_pass[g] ? 1 : 0;

        // values in sorted order (arena row ids index the packed values)
        if (P.nvals) {
            GatherArgs g{};
            g.perm = sa.perm_out;
            g.err = err;
            g.n = P.n_large;
            g.ncols = P.nvals;
            for (int j = 0; j < P.nvals; ++j) {
                g.src[j] = P.rec_bytes ? nullptr : ws + P.o_arena_vals[j];
                g.dst[j] = ws + P.o_sorted_vals[j];
                g.width[j] = P.val_width[j];
            }
            int gl = 0;
            if (P.rec_bytes)
                e = run_gather_records(g, b.arena_recs, P.rec_bytes, s, prof, &gl);
            else
                e = run_gather(g, s, prof, nullptr, 0, &gl);
            if (e != cudaSuccess) return e;
            n += gl;
        }

        // groups over (segment, key); the arena segment column is also the
        // sorted one, since the sort keeps every segment in place
        SegArgs r{};
        r.n = P.n_large;
        r.striped_min_heads = P.emit_min_heads;
        r.nkeys = 2;
        r.nvals = P.nvals;
        r.key[0] = SegCol{b.arena_seg, U32};
        r.key[1] = SegCol{sa.keys_out, P.key_width == 8 ? U64 : U32};
        r.key_out[0] = b.group_seg;
        r.key_out[1] = b.group_key_img;
        for (int j = 0; j < P.nvals; ++j) {
            r.val[j] = SegCol{ws + P.o_sorted_vals[j], a.val_dtypes[j]};
            const vdf_agg_out& o = a.aggs[j];
            const size_t w = (size_t)P.val_width[j];
            const bool fl = (a.val_dtypes[j] == VDF_F64 || a.val_dtypes[j] == VDF_F32);
            r.agg[j].sum = o.sum ? static_cast<unsigned char*>(o.sum) + 8 * P.large_base : nullptr;
            r.agg[j].sum_hi = (o.sum_hi && !fl) ? o.sum_hi + P.large_base : nullptr;
            r.agg[j].min = o.min ? static_cast<unsigned char*>(o.min) + w * P.large_base : nullptr;
            r.agg[j].max = o.max ? static_cast<unsigned char*>(o.max) + w * P.large_base : nullptr;
            r.agg[j].mean = o.mean ? o.mean + P.large_base : nullptr;
        }
        r.count_out = a.group_count_out ? a.group_count_out + P.large_base : nullptr;
        r.n_groups = b.n_groups_large;
        r.err = err;
        int rl = 0;
        if ((e = run_segreduce(r, tail, s, prof, &rl)) != cudaSuccess) return e;
        n += rl;

        if (prof) prof->begin(KC_BATCH, s);
        k_batch_localize<<<grid_for(P.n_large, sms), 256, 0, s>>>(b);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
        k_batch_seg_groups<<<(b.nsegs + 255) / 256, 256, 0, s>>>(b);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
        n += 2;
        if (a.group_keys_out) {
            k_batch_group_keys<<<grid_for(P.n_large, sms), 256, 0, s>>>(b);
            if ((e = cudaGetLastError()) != cudaSuccess) return e;
            ++n;
        }
        if (prof) prof->end(KC_BATCH, s);
    }
    if (have_small && (e = cudaStreamWaitEvent(s, join, 0)) != cudaSuccess) return e;
    if (launches) *launches += n;
    return cudaSuccess;
}

}  // namespace vdf

// ---------------------------------------------------------------------------
// C-ABI
// ---------------------------------------------------------------------------
using namespace vdfc;

struct vdf_batch {
    vdf_ctx* ctx = nullptr;
    vdf_batch_args args{};
    std::vector<vdf_batch_query> queries;
    vdf::BatchPlan plan;
    unsigned char* ws = nullptr;   // the context workspace the plan was uploaded to
    cudaStream_t side = nullptr;
    cudaEvent_t fork = nullptr, join = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    cudaStream_t graph_stream = nullptr;
};

namespace {

vdf_status check_batch_args(vdf_ctx* c, const vdf_batch_args* a) {
    if (!a) return fail(c, VDF_ERR_INVALID_ARG, "batch args is NULL");
    if (a->nqueries && !a->queries) return fail(c, VDF_ERR_INVALID_ARG, "queries is NULL");
    if (a->nvals < 0 || a->nvals > VDF_BATCH_MAX_VALS)
        return fail(c, VDF_ERR_INVALID_ARG, "nvals must be 0..%d", VDF_BATCH_MAX_VALS);
    for (int j = 0; j < a->nvals; ++j)
        if (!valid_dtype(a->val_dtypes[j])) return fail(c, VDF_ERR_INVALID_ARG, "value %d: bad dtype", j);
    if (!a->perm_out || !a->row_offset_out || !a->group_offset_out || !a->n_groups_out)
        return fail(c, VDF_ERR_INVALID_ARG, "perm_out and the per-query offset/count outputs are required");
    for (uint32_t q = 0; q < a->nqueries; ++q) {
        const vdf_batch_query& Q = a->queries[q];
        if (!valid_dtype(Q.key.dtype)) return fail(c, VDF_ERR_INVALID_ARG, "query %u: bad key dtype", q);
        if (Q.n && !Q.key.data) return fail(c, VDF_ERR_INVALID_ARG, "query %u: NULL key", q);
        for (int j = 0; j < a->nvals; ++j)
            if (Q.n && !Q.vals[j]) return fail(c, VDF_ERR_INVALID_ARG, "query %u: NULL value column %d", q, j);
        if (Q.n > vdf::kMaxBatchRows) return fail(c, VDF_ERR_UNSUPPORTED, "query %u: too many rows", q);
    }
    return VDF_OK;
}

void release_graph(vdf_batch* b) {
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    b->exec = nullptr;
    b->graph = nullptr;
}

}  // namespace

extern "C" {

int vdf_batch_variant_count(void) { return vdf::seg_sort_variant_count(); }

vdf_status vdf_batch_variant_info(int index, int32_t* digit_bits, int32_t* tile_rows) {
    int b, t;
    if (!vdf::seg_sort_variant_info(index, &b, &t)) return VDF_ERR_INVALID_ARG;
    if (digit_bits) *digit_bits = b;
    if (tile_rows) *tile_rows = t;
    return VDF_OK;
}

vdf_status vdf_batch_default_tuning(vdf_batch_tuning* t) {
    if (!t) return VDF_ERR_INVALID_ARG;
    const vdf::BatchTuning d = vdf::default_batch_tuning();
    t->small_rows = d.small_rows;
    t->small_bits = d.small_bits;
    t->seg_variant = d.seg_variant;
    return VDF_OK;
}

vdf_status vdf_batch_create(vdf_ctx* c, const vdf_batch_args* a, const vdf_batch_tuning* tuning, vdf_batch** out) {
    if (!c || !out) return VDF_ERR_INVALID_ARG;
    *out = nullptr;
    std::lock_guard<std::mutex> lk(c->mu);
    vdf_status st = check_batch_args(c, a);
    if (st != VDF_OK) return st;
    vdf::BatchTuning t = vdf::default_batch_tuning();
    if (tuning) t = vdf::BatchTuning{tuning->small_rows, tuning->small_bits, tuning->seg_variant};
    if (!vdf::batch_tuning_valid(t)) return fail(c, VDF_ERR_INVALID_ARG, "invalid batch tuning");
    DeviceGuard g(c->device);
    vdf_batch* b = new vdf_batch();
    b->ctx = c;
    b->args = *a;
    b->queries.assign(a->queries, a->queries + a->nqueries);
    b->args.queries = b->queries.data();
    std::string why;
    if (!vdf::plan_batch(b->plan, b->args, t, why, c->tuning.msd, c->tuning.msd_match)) {
        delete b;
        return fail(c, VDF_ERR_UNSUPPORTED, "%s", why.c_str());
    }
    b->plan.emit_min_heads = c->emit_min_heads;
    st = ws_ensure(c, b->plan.ws_bytes);
    if (st != VDF_OK) {
        delete b;
        return st;
    }
    b->ws = c->ws;
    // descriptor tables, built on the host and uploaded once
    const vdf::BatchPlan& P = b->plan;
    std::vector<unsigned char> host(P.desc_bytes, 0);
    auto* hq = reinterpret_cast<vdf::BatchQuery*>(host.data() + P.o_queries);
    for (uint32_t q = 0; q < a->nqueries; ++q) {
        hq[q].key = a->queries[q].key.data;
        hq[q].key_dtype = a->queries[q].key.dtype;
        hq[q].n = a->queries[q].n;
        hq[q].row_offset = P.row_offset[q];
        for (int j = 0; j < a->nvals; ++j) hq[q].vals[j] = a->queries[q].vals[j];
    }
    if (!P.segs.empty()) std::memcpy(host.data() + P.o_segs, P.segs.data(), sizeof(vdf::SegDesc) * P.segs.size());
    if (!P.seg_query.empty()) std::memcpy(host.data() + P.o_seg_query, P.seg_query.data(), 4 * P.seg_query.size());
    if (!P.tile_seg.empty()) std::memcpy(host.data() + P.o_tile_seg, P.tile_seg.data(), 4 * P.tile_seg.size());
    if (!P.chunks.empty())
        std::memcpy(host.data() + P.o_chunks, P.chunks.data(), sizeof(vdf::SegChunk) * P.chunks.size());
    if (!P.small_queries.empty())
        std::memcpy(host.data() + P.o_small, P.small_queries.data(), 4 * P.small_queries.size());
    if (P.msd) {
        std::memcpy(host.data() + P.o_msd_segs, P.msd_segs.data(), sizeof(vdf::SegDesc) * P.msd_segs.size());
        std::memcpy(host.data() + P.o_msd_tile_seg, P.msd_tile_seg.data(), 4 * P.msd_tile_seg.size());
        std::memcpy(host.data() + P.o_msd_hist_chunks, P.msd_hist_chunks.data(),
                    sizeof(vdf::SegChunk) * P.msd_hist_chunks.size());
        std::memcpy(host.data() + P.o_msd_chunks, P.msd_chunks.data(), sizeof(vdf::MsdSegChunk) * P.msd_chunks.size());
        std::memcpy(host.data() + P.o_flag_init, P.seg_flag_init.data(), 4 * P.seg_flag_init.size());
    }
    // per-query outputs known on the host: row offsets; empty queries' ranges.
    // Uploaded on the batch's own non-blocking stream, so creating a batch
    // does not wait for other work on the device (only for these copies).
    std::vector<uint64_t> zeros(std::max<uint32_t>(1, a->nqueries), 0);
    cudaError_t e = cudaStreamCreateWithFlags(&b->side, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaMemcpyAsync(b->ws, host.data(), P.desc_bytes, cudaMemcpyHostToDevice, b->side);
    if (e == cudaSuccess && a->nqueries) {
        e = cudaMemcpyAsync(a->row_offset_out, P.row_offset.data(), 8 * a->nqueries, cudaMemcpyHostToDevice, b->side);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(a->group_offset_out, P.row_offset.data(), 8 * a->nqueries, cudaMemcpyHostToDevice,
                                b->side);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(a->n_groups_out, zeros.data(), 8 * a->nqueries, cudaMemcpyHostToDevice, b->side);
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(b->side);  // the host vectors die here
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->join, cudaEventDisableTiming);
    if (e != cudaSuccess) {
        vdf_batch_destroy(b);
        return from_cuda(c, e, "batch setup");
    }
    *out = b;
    return VDF_OK;
}

uint64_t vdf_batch_rows(const vdf_batch* b) { return b ? b->plan.n_total : 0; }

vdf_status vdf_batch_info(const vdf_batch* b, uint32_t* small_queries, uint64_t* small_rows, uint32_t* large_queries,
                          uint64_t* large_rows) {
    if (!b) return VDF_ERR_INVALID_ARG;
    if (small_queries) *small_queries = (uint32_t)b->plan.small_queries.size();
    if (small_rows) *small_rows = b->plan.n_small;
    if (large_queries) *large_queries = (uint32_t)b->plan.segs.size();
    if (large_rows) *large_rows = b->plan.n_large;
    return VDF_OK;
}

vdf_status vdf_batch_sort_info(vdf_batch* b, uint32_t* msd_queries, uint32_t* lsd_queries, uint32_t* fallbacks) {
    if (!b) return VDF_ERR_INVALID_ARG;
    const vdf::BatchPlan& P = b->plan;
    if (msd_queries) *msd_queries = P.msd_queries;
    if (lsd_queries) *lsd_queries = (uint32_t)P.segs.size() - P.msd_queries;
    if (!fallbacks) return VDF_OK;
    *fallbacks = 0;
    if (!P.msd) return VDF_OK;
    vdf_ctx* c = b->ctx;
    std::lock_guard<std::mutex> lk(c->mu);
    if (c->ws != b->ws) return fail(c, VDF_ERR_WORKSPACE, "the context workspace moved since vdf_batch_create");
    DeviceGuard g(c->device);
    std::vector<uint32_t> flags(P.segs.size());
    cudaError_t e = cudaDeviceSynchronize();
    if (e == cudaSuccess)
        e = cudaMemcpy(flags.data(), b->ws + P.o_seg_flag, 4 * flags.size(), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return from_cuda(c, e, "batch sort info");
    for (size_t s = 0; s < flags.size(); ++s) *fallbacks += (P.seg_flag_init[s] == 0 && flags[s] != 0) ? 1u : 0u;
    return VDF_OK;
}

vdf_status vdf_batch_launch(vdf_batch* b, void* stream) {
    if (!b) return VDF_ERR_INVALID_ARG;
    vdf_ctx* c = b->ctx;
    std::lock_guard<std::mutex> lk(c->mu);
    if (c->ws != b->ws) return fail(c, VDF_ERR_WORKSPACE, "the context workspace moved since vdf_batch_create");
    DeviceGuard g(c->device);
    int n = 0;
    cudaError_t e = vdf::launch_batch(b->plan, b->args, b->ws, err_word(c), static_cast<cudaStream_t>(stream),
                                      b->side, b->fork, b->join, prof_of(c), &n);
    c->launches += n;
    return from_cuda(c, e, "batch launch");
}

vdf_status vdf_batch_launch_graph(vdf_batch* b, void* stream) {
    if (!b) return VDF_ERR_INVALID_ARG;
    vdf_ctx* c = b->ctx;
    std::lock_guard<std::mutex> lk(c->mu);
    if (c->ws != b->ws) return fail(c, VDF_ERR_WORKSPACE, "the context workspace moved since vdf_batch_create");
    DeviceGuard g(c->device);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    cudaError_t e = cudaSuccess;
    if (!b->exec) {
        // capture on a private stream (the legacy stream cannot be captured)
        if (!b->graph_stream) e = cudaStreamCreateWithFlags(&b->graph_stream, cudaStreamNonBlocking);
        if (e == cudaSuccess) e = cudaStreamBeginCapture(b->graph_stream, cudaStreamCaptureModeThreadLocal);
        if (e == cudaSuccess) {
            int n = 0;
            cudaError_t le = vdf::launch_batch(b->plan, b->args, b->ws, err_word(c), b->graph_stream, b->side,
                                               b->fork, b->join, nullptr, &n);
            e = cudaStreamEndCapture(b->graph_stream, &b->graph);
            if (le != cudaSuccess) e = le;
            b->plan.graph_launches = n;
        }
        if (e == cudaSuccess) e = cudaGraphInstantiate(&b->exec, b->graph, 0);
        if (e != cudaSuccess) {
            release_graph(b);
            cudaGetLastError();
            return from_cuda(c, e, "batch graph capture");
        }
    }
    e = cudaGraphLaunch(b->exec, s);
    c->launches += b->plan.graph_launches;
    return from_cuda(c, e, "batch graph launch");
}

void vdf_batch_destroy(vdf_batch* b) {
    if (!b) return;
    DeviceGuard g(b->ctx->device);
    release_graph(b);
    if (b->graph_stream) cudaStreamDestroy(b->graph_stream);
    if (b->side) cudaStreamDestroy(b->side);
    if (b->fork) cudaEventDestroy(b->fork);
    if (b->join) cudaEventDestroy(b->join);
    delete b;
}

}  // extern "C"
