// vdf_batch.h -- internal structures of the batched executor (vdf_batch.cu,
// vdf_batch_small.cu).  The public interface is vdf_batch_* in vdf_capi.h.
#pragma once
#include <string>
#include <vector>

#include "vdf_capi.h"
#include "vdf_internal.h"

namespace vdf {

constexpr uint64_t kMaxBatchRows = (1ull << 30) - 1;  // look-back counts are 30 bits
constexpr uint32_t kSmallMaxRows = 8192;              // widest one-CTA query
constexpr uint32_t kChunkRows = 16384;                // rows per pack / histogram CTA

// One query as the kernels see it.
struct BatchQuery {
    const void* key;
    const void* vals[VDF_BATCH_MAX_VALS];
    uint64_t n;
    uint64_t row_offset;  // first row (and first group slot) in the output arena
    int32_t key_dtype;
    int32_t pad;
};

struct BatchTuning {
    uint32_t small_rows;  // queries of at most this many rows run one CTA each
    int small_bits;       // digit width of the one-CTA sort: 4 or 8
    int seg_variant;      // segmented radix-pass variant for the other queries
};
BatchTuning default_batch_tuning();
bool batch_tuning_valid(const BatchTuning& t);

// Device view of a planned batch (pointers into the workspace and the
// caller's outputs), passed by value to every batch kernel.
struct BatchDev {
    const BatchQuery* queries;
    const SegDesc* segs;
    const uint32_t* seg_query;   // [nsegs] query of each large segment
    const SegChunk* chunks;
    const uint32_t* small_queries;
    uint32_t n_small_queries;
    uint32_t small_cap;          // rows of the largest small query allowed (tuning)
    uint32_t nsegs;
    uint32_t* work_counter;      // next small query to take
    uint64_t* n_groups_large;    // groups over all large queries
    uint32_t* seg_first_group;   // [nsegs]
    int nvals;
    int small_bits;
    int val_width[VDF_BATCH_MAX_VALS];
    int val_dtype[VDF_BATCH_MAX_VALS];
    void* arena_vals[VDF_BATCH_MAX_VALS];  // one value column each (fewer than two columns)
    unsigned char* arena_recs;             // or one record per row (two or more)
    int rec_bytes;
    vdf_agg_out aggs[VDF_BATCH_MAX_VALS];
    void* arena_keys;            // [n_large] ordered key images, key_width bytes each
    int key_width;               // 8, or 4 when every large query's keys are 4 bytes
    uint32_t* arena_seg;         // [n_large] segment of each arena row
    uint32_t* group_seg;         // [groups] segment of each large-query group
    void* group_key_img;         // [groups] ordered key image of each group (key_width bytes)
    uint64_t n_large;
    uint64_t large_base;         // first arena row of the large queries
    uint32_t* perm_out;
    void* group_keys_out;
    int64_t* group_count_out;
    uint64_t* group_offset_out;
    uint64_t* n_groups_out;
    uint32_t* err;
};

struct BatchPlan {
    BatchTuning tuning{};
    uint32_t nq = 0;
    int nvals = 0;
    int val_width[VDF_BATCH_MAX_VALS] = {};
    uint32_t tile_rows = 0;
    int key_width = 8;  // arena key image width
    std::vector<uint64_t> row_offset;
    std::vector<uint32_t> small_queries;
    std::vector<SegDesc> segs;
    std::vector<uint32_t> seg_query;
    std::vector<uint32_t> tile_seg;
    std::vector<SegChunk> chunks;
    uint64_t n_small = 0, n_large = 0, n_total = 0, large_base = 0;
    int max_passes = 0;
    uint32_t tiles_in_pass[16] = {};
    // MSD-first plan for the large queries: the segments that take it sort
    // by their top digits (msd_segs: passes over those digits only), then
    // chunks of whole buckets are finished in shared memory; afterwards the
    // LSD passes run only for segments whose flag is set (those planned for
    // them, and those whose chunks defeated the plan)
    bool msd = false;
    int msd_match = 0;
    uint32_t emit_min_heads = 0;  // the group-by emit's striped-path threshold (0 = default)
    uint32_t msd_queries = 0;
    std::vector<SegDesc> msd_segs;         // more passes first
    std::vector<uint32_t> msd_seg_of;      // [msd segs] segment index in segs
    std::vector<uint32_t> msd_tile_seg;
    std::vector<SegChunk> msd_hist_chunks;
    std::vector<MsdSegChunk> msd_chunks;   // in arena order
    std::vector<uint32_t> seg_flag_init;   // [segs] 1: LSD passes, 0: MSD-first
    int msd_max_passes = 0;
    uint32_t msd_tiles_in_pass[16] = {};
    // workspace layout (byte offsets)
    size_t o_queries = 0, o_segs = 0, o_seg_query = 0, o_tile_seg = 0, o_chunks = 0, o_small = 0;
    size_t o_msd_segs = 0, o_msd_tile_seg = 0, o_msd_hist_chunks = 0, o_msd_chunks = 0, o_flag_init = 0;
    size_t desc_bytes = 0;
    size_t o_seg_flag = 0, o_chunk_start = 0;
    size_t o_counters = 0, o_seg_first = 0, o_arena_keys = 0, o_arena_seg = 0, o_arena_vals[VDF_BATCH_MAX_VALS] = {};
    size_t o_arena_recs = 0, rec_bytes = 0;
    size_t o_sorted_keys = 0, o_sorted_vals[VDF_BATCH_MAX_VALS] = {}, o_group_seg = 0, o_group_key = 0, o_tail = 0;
    size_t ws_bytes = 0;
    int graph_launches = 0;
};

// msd: 0 the LSD passes; 1 the MSD-first sort for large queries of 8-byte
// keys, 2 for every width (8-bit digit variants only); msd_match: the
// shared-memory finish's digit-match method.
bool plan_batch(BatchPlan& P, const vdf_batch_args& a, const BatchTuning& t, std::string& why, int msd = 0,
                int msd_match = 0);
BatchDev batch_dev_view(const BatchPlan& P, const vdf_batch_args& a, unsigned char* ws, uint32_t* err);
cudaError_t launch_batch(const BatchPlan& P, const vdf_batch_args& a, unsigned char* ws, uint32_t* err,
                         cudaStream_t s, cudaStream_t side, cudaEvent_t fork, cudaEvent_t join, Profiler* prof,
                         int* launches);
// The persistent one-CTA-per-query kernel over b.small_queries.
cudaError_t launch_small_queries(const BatchDev& b, cudaStream_t s, int sms);
cudaError_t prepare_batch_kernels();

}  // namespace vdf
