// vdf_internal.h -- host/device structures shared by the .cu files of the
// library.  Not part of the public C-ABI (that is include/vdf_capi.h).
#pragma once
#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

namespace vdf {

constexpr int kMaxKeys = 4;     // key columns per sort / group-by
constexpr int kMaxVals = 4;     // aggregated value columns per group-by launch
constexpr int kMaxGather = 8;   // columns per gather launch

// Kernel classes for the optional per-launch timing (vdf_ctx_profile).
enum KernelClass : int {
    KC_HIST = 0, KC_SCAN = 1, KC_ONESWEEP32 = 2, KC_ONESWEEP64 = 3, KC_GATHER = 4, KC_SEGREDUCE = 5,
    KC_BROADCAST = 6, KC_PACK = 7, KC_SEGSCAN = 8, KC_SEGEMIT = 9, KC_TIES = 10, KC_BATCH = 11,
    KC_CSV = 12, KC_LOCALSORT = 13, KC_FALLBACK = 14, KC_DICT = 15, KC_COUNT = 16
};

// Brackets kernel launches with CUDA events when profiling is enabled.
struct Profiler {
    virtual void begin(int cls, cudaStream_t s) = 0;
    virtual void end(int cls, cudaStream_t s) = 0;
    virtual ~Profiler() = default;
};

// ---- radix sort ------------------------------------------------------------
enum InMode : int { IN_RAW = 0, IN_GATHER = 1, IN_BUF = 2 };

constexpr int kMaxBits = 11;                  // widest radix digit compiled
constexpr int kMaxRadix = 1 << kMaxBits;
constexpr int kMaxPasses = kMaxKeys * 8;      // 8-bit digits over four 8-byte keys

struct HistCol {
    const void* data;
    int dtype;
    int passes;
    int bits;       // digit width of this column's passes
    int hist_off;   // word offset of its first pass's histogram
    int invert;
};
struct HistArgs {
    HistCol col[kMaxKeys];
    int ncols;
    int hist_words;
    uint64_t n;
    uint32_t* hist;
    const uint32_t* run_flag;  // non-null: the kernel runs only if *run_flag == 1 (the LSD fallback)
    uint32_t* run_count;       // non-null: incremented once when a conditional launch runs
};
// Histograms of every pass laid out back to back: pass g has radix[g] bins
// starting at word off[g]; the scan writes exclusive starts at the same words.
struct ScanArgs {
    const uint32_t* hist;
    uint32_t* offs;
    uint32_t off[kMaxPasses];
    uint32_t radix[kMaxPasses];
    const uint32_t* run_flag;  // non-null: the kernel runs only if *run_flag == 1 (the LSD fallback)
};

// One segment of a segmented sort: rows [row_start, row_start + rows) of the
// arena, tiles [first_tile, first_tile + ceil(rows / tile)), sorted in
// `passes` digit passes over digits first_digit .. first_digit + passes - 1
// (0 and the key's digit count for an LSD sort; the top digits for the
// MSD-first plan).
struct SegDesc {
    uint64_t row_start;
    uint32_t rows;
    uint32_t first_tile;
    uint32_t passes;
    uint32_t first_digit;
};

// Dictionary plan limits: distinct keys it takes, slots of the collection
// table (global; each CTA has a table of kDictCtaSlots in shared memory) and
// of the lookup table the pass reads.
constexpr uint32_t kDictMax = 256;
constexpr uint32_t kDictSlots = 1024;
constexpr uint32_t kDictCtaSlots = 512;
constexpr uint32_t kDictLutSlots = 512;
// One slot of a collection table: state 0 empty, 1 being written, 2 ready.
struct DictSlot {
    unsigned long long key;
    uint32_t count;
    uint32_t state;
};
// Order image -> rank among the distinct keys (rank kDictEmpty: free slot).
constexpr uint32_t kDictEmpty = 0xffffffffu;
struct DictLut {
    unsigned long long key[kDictLutSlots];
    uint32_t rank[kDictLutSlots];
};
__host__ __device__ inline uint32_t dict_hash(unsigned long long x) {
    x ^= x >> 33;
    x *= 0xff51afd7ed558ccdull;
    x ^= x >> 33;
    return (uint32_t)x;
}
struct DictArgs {
    const void* keys;         // raw key column (any row order: only the key multiset matters)
    int dtype, invert, width;
    uint64_t n;
    DictSlot* table;          // [kDictSlots], zeroed
    uint32_t* distinct;       // distinct keys merged so far
    uint32_t* overflow;       // set when there are more than kDictMax (or a wait gave up)
    uint32_t* state;          // the sort's plan word
    uint32_t fail_state;      // plan word when the dictionary does not apply (0 MSD-first, 1 LSD)
    DictLut* lut;
    uint32_t* bin_offsets;    // [256] exclusive starts of the ranks
    uint32_t* taken;          // non-null: incremented when the dictionary pass is taken
    uint32_t spin_limit;
    uint32_t* err;
};
cudaError_t dict_collect(const DictArgs& a, cudaStream_t s);
cudaError_t dict_rank(const DictArgs& a, cudaStream_t s);

struct PassArgs {
    const void* keys_in;        // raw column (IN_RAW / IN_GATHER) or ordered-key buffer
    const uint32_t* vals_in;    // row ids (IN_GATHER: current permutation; IN_BUF: buffer)
    void* keys_out;             // ordered-key buffer, or raw sorted keys (final pass; may be null)
    uint32_t* vals_out;         // row-id buffer, or the output permutation (final pass)
    const uint32_t* bin_offsets;  // [RADIX] global exclusive bin starts for this digit
    uint32_t* status;           // [tiles][RADIX] look-back words of this pass
    uint32_t* status_next;      // the other status buffer, cleared for the next pass
    uint32_t* tile_counter;     // tile ids in scheduling order
    uint32_t* err;              // error bits (vdf::ErrBits)
    uint64_t n;
    uint32_t shift;
    uint32_t status_rows;       // rows of status_next to clear
    uint32_t status_row_words;  // words per status row (the plan's widest radix)
    int dtype;
    int invert;                 // stable descending: keys bit-inverted
    int reverse;                // reference descending: output positions mirrored
    // segmented sorts only
    const uint32_t* tile_seg;   // [tiles] segment of each tile
    const SegDesc* segs;        // [segments]
    const uint32_t* seg_offs;   // [segments][seg_stride]: per pass, exclusive digit starts in the segment
    uint32_t seg_stride;        // words per segment in seg_offs (max passes x radix)
    uint32_t pass;              // digit pass index
    void* keys_final;           // where a segment's last pass writes its keys
    uint32_t* vals_final;       // ... and its row ids
    // conditional passes: with run_flag set the pass runs only when
    // *run_flag == run_when, and otherwise returns at once (the sort's plan
    // word: 0 MSD-first passes, 1 LSD passes, 2 done by the dictionary pass)
    const uint32_t* run_flag;
    uint32_t run_when;
    // dictionary pass: the digit of a key is its rank among the sort's
    // distinct keys, looked up in this table
    const DictLut* dict_lut = nullptr;
    // failure injection for tests: polls before a look-back wait gives up (0:
    // the default kSpinLimit), and a tile whose CTA publishes nothing
    uint32_t spin_limit = 0;
    uint32_t stall_tile = 0xffffffffu;
    // segmented passes only: with seg_flag set, a tile runs only when
    // (seg_flag[segment] != 0) == (seg_flag_when != 0)
    const uint32_t* seg_flag = nullptr;
    uint32_t seg_flag_when = 0;
    // tiles of the pass (0: one per CTA of the grid); a grid smaller than
    // that loops, each CTA taking the next tile id until none is left
    uint32_t ntiles = 0;
};


// Kernel-variant choice of the radix pass per key width (indices into the
// variant table in vdf_radix.cu); the autotuner's search space.
struct SortTuning {
    int variant32;
    int variant64;
    // MSD-first sort (vdf_msd.cu): 1 = used for sorts of one or two key
    // columns with at least msd_min_rows rows, 0 = never
    int msd = 0;
    uint64_t msd_min_rows = 0;
    int msd_match = 0;  // shared-memory passes: 0 = ballots, 1 = match.any
    // failure injection for tests (vdf_ctx_set_test_hooks): look-back poll
    // limit (0 = default) and a tile of the first pass that never publishes
    uint32_t spin_limit = 0;
    uint32_t stall_tile = 0xffffffffu;
    // dictionary plan (vdf_dict.cu): 1 = tried for one-key sorts with at
    // least msd_min_rows rows, 0 = never
    int dict = 0;
};
SortTuning default_sort_tuning();
bool sort_tuning_valid(const SortTuning& t);
int sort_variant_count();
bool sort_variant_info(int i, int* width, int* threads, int* items, int* bits, int* match);
bool sort_variant_uses_tma(int i);

struct SortPlan {
    uint64_t n;
    SortTuning tuning;
    int nkeys;
    int dtype[kMaxKeys], width[kMaxKeys], passes[kMaxKeys], pass_base[kMaxKeys];
    int bits[kMaxKeys], radix[kMaxKeys], hist_off[kMaxKeys];
    int total_passes, hist_words, max_radix;
    uint32_t max_tiles;
    size_t off_keys[2], off_vals[2], off_offs, off_zero, off_hist, off_counters, off_status[2];
    size_t zero_bytes;
    size_t ws_bytes;
    // MSD-first sort: msd_passes global passes over the top 8-bit digits of
    // key 0, then one CTA per chunk of whole buckets sorts the rest in shared
    // memory; the LSD passes above run only if that fails (a flag on the
    // device decides, no host round trip).
    bool msd;
    int msd_passes;
    int msd_lo_bits;           // key 0 bits ranked directly in runs (below the shared-memory passes)
    uint32_t msd_cap;          // rows a chunk may hold (kMsdCap, or kMsdWideCap)
    uint32_t msd_chunk_rows;   // nominal rows per chunk
    uint32_t msd_chunks;       // ceil(n / msd_chunk_rows)
    size_t off_msd_hist, off_msd_offs, off_msd_flag, off_chunks;
    // dictionary plan: a one-key sort whose key takes at most kDictMax
    // distinct values is one stable pass over each key's rank; the values
    // are collected on the device first, and with more of them the MSD-first
    // or LSD passes run instead (the plan word at off_msd_flag decides)
    bool dict;
    int dict_variant;          // index into the dictionary-pass kernels
    uint32_t dict_tiles;
    size_t off_dict_table, off_dict_lut, off_dict_offs, off_dict_words;
};
// MSD-first sort limits: rows one CTA sorts in shared memory, the longest
// run of equal high key bits the shared-memory finish ranks directly, and the
// most top digits that go through global passes.
constexpr uint32_t kMsdCap = 4096;
// wide chunks (one CTA of 1024 threads per SM) where they save a top digit
constexpr uint32_t kMsdWideCap = 8192;
constexpr uint32_t kMsdRunMax = 64;
constexpr int kMsdMaxPasses = 3;
constexpr uint32_t kMsdBucketRows = 1536;           // planned average bucket
constexpr uint64_t kMsdDefaultMinRows = 1u << 20;   // smaller sorts: LSD passes
struct MsdHistArgs {
    const void* keys;  // raw key 0 column
    int dtype, invert, first_digit, ndig;
    uint64_t n;
    uint32_t* hist;    // [ndig][256]
    const uint32_t* flag = nullptr;  // the plan word: the histograms run only while it is 0
};
// A chunk of a segmented MSD-first sort: nominal first row x (the segment's
// first row for its first chunk), the segment's rows [seg_start, seg_end),
// the shift that leaves its keys' top (bucket) bits, and its segment.
struct MsdSegChunk {
    uint32_t x, seg_start, seg_end, pshift, seg, pad[3];
};
struct MsdChunkArgs {
    const void* keys;  // order images sorted by their top bits
    uint64_t n;
    uint32_t chunk_rows, nchunks, pshift;
    uint32_t* chunk_start;  // [nchunks + 1]
    uint32_t* flag;
    // segmented sorts: per-chunk descriptors, and a failure flag per segment
    const MsdSegChunk* seg_chunks = nullptr;
    uint32_t* seg_flag = nullptr;
};
struct MsdLocalArgs {
    const void* keys;        // order images of key 0 sorted by their top bits
    const uint32_t* vals;    // their row ids
    const uint32_t* chunk_start;
    uint64_t n;
    const void* sec;         // raw key 1 column (null for one key)
    int sec_dtype, dtype, invert, reverse;
    uint32_t lo_bits;        // key 0 bits below the shared-memory passes
    uint32_t* flag;
    uint32_t* err;
    void* keys_out;          // raw sorted key 0 (may be null)
    uint32_t* perm_out;
    // segmented sorts: each chunk's segment; a failing chunk sets its
    // segment's flag instead of the global one
    const MsdSegChunk* seg_chunks = nullptr;
    uint32_t* seg_flag = nullptr;
};
cudaError_t msd_hist(const MsdHistArgs& a, int width, cudaStream_t s);
cudaError_t msd_scan(const uint32_t* hist, uint32_t* offs, int ndig, uint32_t cap, uint32_t* flag, cudaStream_t s);
cudaError_t msd_chunks(const MsdChunkArgs& a, int width, cudaStream_t s, uint32_t cap = kMsdCap);
cudaError_t msd_local(const MsdLocalArgs& a, int width, uint32_t nchunks, int match, cudaStream_t s,
                      uint32_t cap = kMsdCap);
// Kernel launches run_sort makes for a plan (conditional ones included).
int sort_launches(const SortPlan& p);
// Global top-digit passes of the MSD-first plan for n rows of width-byte keys
// (0: none fits).
int msd_passes_for(uint64_t n, int width, uint32_t bucket_rows = kMsdBucketRows);

SortPlan make_sort_plan(uint64_t n, const int32_t* dtypes, int nkeys, const SortTuning& tuning);
// Sorts; writes perm_out (and key0_out = raw sorted most-significant key, may
// be null).  Bounded waits that give up OR their ErrBits into *err.  With
// perm_in (a permutation of [0, n)) the rows are sorted as seen through it
// and perm_out is the composed permutation.
// msd_fallbacks (optional, device word): incremented each time an MSD-first
// plan falls back to the LSD passes.
cudaError_t run_sort(const SortPlan& p, const void* const* key_cols, int order, uint32_t* perm_out,
                     void* key0_out, unsigned char* ws, uint32_t* err, cudaStream_t s, Profiler* prof = nullptr,
                     const uint32_t* perm_in = nullptr, uint32_t* msd_fallbacks = nullptr,
                     uint32_t* dict_taken = nullptr);
cudaError_t prepare_sort_kernels();
cudaError_t prepare_msd_kernels();
// *flag |= 1 when two neighbouring elements of a sorted key column (4- or
// 8-byte elements) have the same bits.
cudaError_t flag_adjacent_ties(const void* sorted_keys, int width, uint64_t n, uint32_t* flag, cudaStream_t s,
                               Profiler* prof = nullptr);

// ---- segmented sort (many independent row ranges in one set of launches) ----
// Keys are ordered images (the batch packs them so), 8 bytes wide, or 4 when
// every segment's keys are; a 4-byte key in an 8-byte image has a zero high
// half and needs fewer passes.
struct SegChunk {      // a histogram CTA's rows: part of one segment
    uint64_t row_start;
    uint32_t rows;
    uint32_t seg;
};
struct SegSortArgs {
    uint64_t n;                   // arena rows (< 2^30)
    const void* keys;             // [n] ordered key images
    int key_width;                // 8, or 4 when every segment's keys are 4 bytes
    const SegDesc* segs;          // device [nsegs]
    uint32_t nsegs;
    const uint32_t* tile_seg;     // device [ntiles]; segments with more passes first
    uint32_t ntiles;
    const SegChunk* chunks;       // device [nchunks]
    uint32_t nchunks;
    int max_passes;
    uint32_t tiles_in_pass[16];   // launch width of pass g: tiles of segments with passes > g
    int variant;                  // index into the segmented variant table
    void* keys_out;               // [n] sorted key images (each segment in place)
    uint32_t* perm_out;           // [n] arena row ids in sorted order
    uint32_t* err;
    // conditional per segment: with seg_flag set, only the segments whose
    // flag is non-zero are sorted (their histograms, passes and outputs)
    const uint32_t* seg_flag = nullptr;
};
int seg_sort_variant_count();
bool seg_sort_variant_info(int v, int* bits, int* tile_rows);
size_t seg_sort_workspace_bytes(uint64_t n, uint32_t nsegs, uint32_t ntiles, int max_passes, int variant,
                                int key_width = 8);
cudaError_t run_seg_sort(const SegSortArgs& a, unsigned char* ws, cudaStream_t s, Profiler* prof = nullptr);

// ---- gather ----------------------------------------------------------------
struct GatherArgs {
    const uint32_t* perm;
    uint32_t* err;     // error word for out-of-range row ids (may be null)
    uint64_t n;
    int ncols;
    const void* src[kMaxGather];
    void* dst[kMaxGather];
    int width[kMaxGather];
};
// Bytes per row of the packed-record buffer a gather of ncols columns uses
// (0: gathered column by column).
size_t gather_record_bytes(int ncols);
// rec_ws: workspace of rec_ws_bytes for the packed records; the packed path
// runs only when it holds n * gather_record_bytes(ncols) bytes, otherwise the
// columns are gathered one by one.  *launches is increased by the kernels
// launched.
cudaError_t run_gather(const GatherArgs& g, cudaStream_t s, Profiler* prof = nullptr, void* rec_ws = nullptr,
                       size_t rec_ws_bytes = 0, int* launches = nullptr);
// The second half of the packed gather, for callers that wrote the records
// themselves: recs holds g.n records of gather_record_bytes(g.ncols) bytes
// (8-byte slots in column order, 4-byte values zero-extended); g.src unused.
cudaError_t run_gather_records(const GatherArgs& g, const void* recs, size_t rec_bytes, cudaStream_t s,
                               Profiler* prof = nullptr, int* launches = nullptr);

// ---- segmented reduction (group-by over sorted rows) -----------------------
// A column of rows in key order.
struct SegCol {
    const void* src;
    int dtype;
};
// Per value column outputs (device pointers, any may be null).
struct SegAggOut {
    void* sum;        // f64 (float columns) or int64 low word (integer columns)
    int64_t* sum_hi;  // high word of the 128-bit integer sum
    void* min;        // in the column's own dtype
    void* max;
    double* mean;
};
struct SegArgs {
    uint64_t n;
    int nkeys, nvals;
    SegCol key[kMaxKeys];
    SegCol val[kMaxVals];
    void* key_out[kMaxKeys];   // group key columns
    int64_t* count_out;        // rows per group
    SegAggOut agg[kMaxVals];
    uint32_t* group_start;     // first sorted row of each group (may be null)
    uint32_t* row_group;       // group index of each sorted row (may be null)
    uint64_t* n_groups;        // device word: number of groups (may be null)
    uint32_t* err;             // error word
    // tiles of the emit pass with at least this many heads (of 512 rows)
    // take the striped path, each group written by the thread of its first
    // row; 0 = kStripedMinHeads
    uint32_t striped_min_heads = 0;
};
constexpr uint32_t kStripedMinHeads = 480;
size_t segreduce_workspace_bytes(uint64_t n, int nvals);
cudaError_t prepare_segreduce_kernels();
// Three launches: tile aggregates, their scan (one CTA), then the emit pass.
// The workspace holds the tile aggregates (segreduce_workspace_bytes).
cudaError_t run_segreduce(SegArgs a, unsigned char* ws, cudaStream_t s, Profiler* prof = nullptr,
                          int* launches = nullptr);

// ---- transform output (aggregate broadcast to rows) --------------------------
cudaError_t run_broadcast(const uint32_t* row_group, uint64_t n, const void* group_vals, uint64_t n_groups,
                          int width, const uint32_t* perm, void* out, uint32_t* err, cudaStream_t s,
                          Profiler* prof = nullptr);

// ---- de-duplication and left-join row matching (vdf_unique.cu) -------------
// keep[perm[i]] = 1 where sorted row i is the first (last = 0) or last row of
// its key's run in the stable ascending sort, else 0; *count += kept rows.
// bits: unique_workspace_bytes(n) of scratch.
size_t unique_workspace_bytes(uint64_t n);
cudaError_t run_unique_mark(const void* sorted_keys, int width, const uint32_t* perm, uint64_t n, int last,
                            uint8_t* keep, unsigned long long* count, uint32_t* bits, uint32_t* err,
                            cudaStream_t s);
// Left-join matching (method 0 First, 1 Last, 2 Aligned).  The right side's
// distinct sorted keys ukeys[0 .. *n_groups), whose runs start at gstart[g],
// go into a hash table (table_ws: join_workspace_bytes(n_right)) holding the
// row of each key's first / last occurrence, or (Aligned) its run index.
size_t join_workspace_bytes(uint64_t n_right);
cudaError_t run_join_build(const void* ukeys, int width, const uint32_t* gstart, const uint64_t* n_groups,
                           const uint32_t* perm_right, uint64_t n_right, int method, void* table_ws, uint32_t* err,
                           cudaStream_t s);
// First / Last: match[i] = the table's row for left[i], or UINT32_MAX.
cudaError_t run_join_probe(const void* left, uint64_t n_left, int width, const void* table_ws, uint64_t n_right,
                           uint32_t* match, unsigned long long* matched, cudaStream_t s);
// Aligned: over the left side's stable sort (permutation, run of each sorted
// row, run starts), occurrence r of a key takes the right run's row r.
cudaError_t run_join_probe_aligned(const void* sorted_left, int width, const uint32_t* perm_left,
                                   const uint32_t* group_left, const uint32_t* gstart_left, uint64_t n_left,
                                   const void* table_ws, const uint32_t* gstart_right, const uint64_t* n_groups_right,
                                   const uint32_t* perm_right, uint64_t n_right, uint32_t* match,
                                   unsigned long long* matched, uint32_t* err, cudaStream_t s);

}  // namespace vdf
