/*
 * vdf_capi.h -- C-ABI of the B200 sort + group-by path (libvdf_b200.so).
 *
 * Plain pointers and sizes only.  Column data, permutations and outputs are
 * DEVICE pointers on the context's GPU, owned by the caller; `stream` is a
 * cudaStream_t passed as void* (NULL = the legacy default stream).  Every call
 * returns a vdf_status and never aborts or throws.  Compute calls are
 * asynchronous on `stream` unless they return a host value (n_groups_host),
 * in which case they synchronise that stream before returning, or sort by
 * several keys in the default multi-key mode (vdf_ctx_set_multikey_mode),
 * which synchronises the stream once to read one flag.
 *
 * A context owns one grow-only workspace, so calls on one context are
 * serialised on the host and must not overlap on the GPU: use one context per
 * concurrently used stream, or the *_ws variants with caller-owned workspace.
 *
 * Each entry point names the reference interface it replaces (paths relative
 * to the VisonDF project, V/ = include/vison/).  The reference's own error
 * convention (std::cerr message + early return, sort_by_mt.hpp:16-18,40-41,
 * 68-69) is restored by the C++ layer in include/vison_b200/vison.hpp.
 */
#ifndef VDF_CAPI_H
#define VDF_CAPI_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define VDF_ABI_VERSION 1u

typedef enum vdf_status {
    VDF_OK = 0,
    VDF_ERR_INVALID_ARG = 1, /* bad pointer, dtype, count or alignment            */
    VDF_ERR_OOM = 2,         /* workspace allocation failed                         */
    VDF_ERR_TIMEOUT = 3,     /* a bounded device wait gave up (look-back)           */
    VDF_ERR_DEVICE = 4,      /* CUDA runtime error                                  */
    VDF_ERR_UNSUPPORTED = 5, /* valid request outside this build's limits           */
    VDF_ERR_WORKSPACE = 6    /* caller-provided workspace too small                 */
} vdf_status;

/* Column element types.  The reference's DefaultTypes are IntT=int,
 * UIntT=unsigned int, FloatT=double (V/types/inference_type.hpp:3-8); the
 * 64-bit integer widths cover sort_integers' int64 branch
 * (V/inlines/transform/sort_by/sort_integers.inl:121-133). */
typedef enum vdf_dtype {
    VDF_I32 = 0,
    VDF_I64 = 1,
    VDF_U32 = 2,
    VDF_U64 = 3,
    VDF_F64 = 4,
    VDF_F32 = 5
} vdf_dtype;

/* Sort order.  ASC: stable ascending (ties keep row order).
 * DESC_STABLE: stable descending, the order V/INTERNALS.doc:1610-1632 shows.
 * DESC_REVERSE: the reference code's descending order, an ascending sort
 * followed by std::reverse (sort_integers.inl:225-227), so ties come out in
 * reverse row order. */
typedef enum vdf_order {
    VDF_ORDER_ASC = 0,
    VDF_ORDER_DESC_STABLE = 1,
    VDF_ORDER_DESC_REVERSE = 2
} vdf_order;

/* A device column: `data` points at n elements of `dtype`. */
typedef struct vdf_col {
    const void* data;
    int32_t dtype;
} vdf_col;

/* Group-by outputs of one value column; device arrays with room for n
 * groups (the group count is only known after the call).  Any may be NULL.
 *   sum    : double for float columns; the low 64 bits (int64 wrap-around
 *            view) of the exact 128-bit sum for integer columns
 *   sum_hi : high 64 bits of the exact integer sum (integer columns)
 *   min,max: in the column's own dtype
 *   mean   : double, sum / count (the reference divides by the frame's row
 *            count instead, V/inlines/transform/transform_group_by/
 *            create_value_col.inl:46; that is a bug and is not reproduced) */
typedef struct vdf_agg_out {
    void* sum;
    int64_t* sum_hi;
    void* min;
    void* max;
    double* mean;
} vdf_agg_out;

typedef struct vdf_ctx vdf_ctx;

/* ---- library / context --------------------------------------------------- */
uint32_t vdf_abi_version(void);
const char* vdf_status_string(vdf_status s);

/* Creates a context on `device`.  Replaces init_openmp(cores)
 * (V/vison.hpp:57-74), the reference's only runtime set-up. */
vdf_status vdf_ctx_create(int device, vdf_ctx** out);
vdf_status vdf_ctx_destroy(vdf_ctx* ctx);
/* Last error message of this context (empty string when none). */
const char* vdf_ctx_last_error(const vdf_ctx* ctx);
/* Grows the context workspace to at least `bytes` now (optional). */
vdf_status vdf_ctx_reserve(vdf_ctx* ctx, size_t bytes);
/* Synchronises `stream`, then reads and clears the device error bits that
 * bounded waits raise; returns VDF_ERR_TIMEOUT if any were set. */
vdf_status vdf_ctx_check(vdf_ctx* ctx, void* stream);
/* Number of kernels this context has launched so far (for benchmarks). */
uint64_t vdf_ctx_kernel_launches(const vdf_ctx* ctx);

/* Kernel classes for per-launch timing. */
typedef enum vdf_kernel_class {
    VDF_KC_HIST = 0,        /* all-digit histogram            */
    VDF_KC_SCAN = 1,        /* digit offset scan              */
    VDF_KC_ONESWEEP32 = 2,  /* radix pass, 4-byte keys        */
    VDF_KC_ONESWEEP64 = 3,  /* radix pass, 8-byte keys        */
    VDF_KC_GATHER = 4,      /* payload gather                 */
    VDF_KC_SEGREDUCE = 5,   /* group-by: per-tile aggregates  */
    VDF_KC_BROADCAST = 6,   /* transform broadcast            */
    VDF_KC_PACK = 7,        /* row-record packing for gathers */
    VDF_KC_SEGSCAN = 8,     /* group-by: tile prefix scan     */
    VDF_KC_SEGEMIT = 9,     /* group-by: scan + emit groups   */
    VDF_KC_TIES = 10,       /* equal-neighbour check (multi-key) */
    VDF_KC_BATCH = 11,      /* batch bookkeeping: row ids per query, group ranges, group keys */
    VDF_KC_CSV = 12,        /* CSV ingest: record split, field parse, string columns */
    VDF_KC_LOCALSORT = 13,  /* MSD-first sort: chunk search + shared-memory finish */
    VDF_KC_FALLBACK = 14,   /* MSD-first / dictionary sort: the conditional LSD kernels (return at once unless taken) */
    VDF_KC_DICT = 15        /* dictionary sort: collection of the distinct keys and their ranks */
} vdf_kernel_class;
/* When enabled, every kernel the context launches is bracketed by CUDA
 * events on its stream (no reference counterpart: the reference has no
 * tracing beyond ad-hoc std::chrono in benchmarks/readf.cpp:20-25). */
vdf_status vdf_ctx_profile(vdf_ctx* ctx, int enable);
/* Waits for the recorded events; returns the summed device time (ms) and
 * launch count of kernel class `cls` since the last reset. */
vdf_status vdf_ctx_profile_read(vdf_ctx* ctx, int cls, double* total_ms, uint64_t* launches);
vdf_status vdf_ctx_profile_reset(vdf_ctx* ctx);

/* ---- tuning (the autotuner's search space) --------------------------------- */
/* The radix pass is compiled in several variants (key width, threads per
 * CTA, keys per thread, digit bits, warp digit-match method: 0 = ballots,
 * 1 = match.any, 2 = both, alternating by item, 3 = shared-memory words
 * the lanes OR their bits into).  A context uses one variant per key width.  The reference
 * fixes its digit width at 16 bits (RADIX_KI16, radix_sorts/details/
 * constants.inl:4) and has no tuning; the digit width, tile size and match
 * method here are chosen per size class by visondf_b200/autotune.py. */
typedef struct vdf_sort_tuning {
    int32_t pass_variant32; /* variant index used for 4-byte keys */
    int32_t pass_variant64; /* variant index used for 8-byte keys */
} vdf_sort_tuning;
int vdf_sort_variant_count(void);
vdf_status vdf_sort_variant_info(int index, int32_t* key_width, int32_t* threads, int32_t* items_per_thread,
                                 int32_t* digit_bits, int32_t* match);
/* Feature bits of a variant (0 for an invalid index): bit 0 = its tiles are
 * staged in shared memory by bulk copies (cp.async.bulk behind an mbarrier,
 * the next tile's copy overlapping the current tile's ranking), on a
 * persistent grid. */
uint32_t vdf_sort_variant_flags(int index);
/* Group-by emit tuning: a 512-row tile with at least striped_min_heads group
 * starts is written by the striped path (the thread of each group's first
 * row walks and writes the group, consecutive threads writing consecutive
 * groups); others by the per-thread walk after a warp scan of aggregates.
 * 0 restores the default (480); get returns the value in use. */
vdf_status vdf_ctx_set_group_tuning(vdf_ctx* ctx, uint32_t striped_min_heads);
uint32_t vdf_ctx_get_group_tuning(vdf_ctx* ctx);
vdf_status vdf_ctx_set_sort_tuning(vdf_ctx* ctx, const vdf_sort_tuning* tuning);
vdf_status vdf_ctx_get_sort_tuning(vdf_ctx* ctx, vdf_sort_tuning* tuning);

/* How a context sorts by several keys.
 * VDF_MULTIKEY_PRIMARY_FIRST (default): sort by the most significant key
 *   alone, then check its sorted copy for equal neighbours; with none, that
 *   order already is the stable order over all keys (later keys only break
 *   ties) and the remaining keys' passes are skipped; otherwise the LSD sort
 *   over all keys follows.  The check reads one flag back: a multi-key call
 *   synchronises its stream once (not under stream capture, where the LSD
 *   sort runs).  Results are identical in both modes.
 * VDF_MULTIKEY_LSD: always the LSD sort over all keys, least-significant key
 *   first, fully asynchronous; the reference composes multi-key sorts the
 *   same way through its in/out idx (sort_by_mt.hpp:3-180 per key). */
typedef enum vdf_multikey_mode {
    VDF_MULTIKEY_LSD = 0,
    VDF_MULTIKEY_PRIMARY_FIRST = 1
} vdf_multikey_mode;
vdf_status vdf_ctx_set_multikey_mode(vdf_ctx* ctx, int mode);
int vdf_ctx_get_multikey_mode(vdf_ctx* ctx); /* -1 for a NULL context */

/* Sort strategy for sorts by one or two key columns.
 * VDF_SORT_AUTO (default, with msd_min_rows = 2^20): sorts of at least
 *   msd_min_rows rows whose key 0 is 8 bytes wide first partition the rows
 *   by the top 1-3 bytes of key 0 with global radix passes (most
 *   significant digit first) and then sort each chunk of whole partitions
 *   (<= 4096 rows) in shared memory by the rest of key 0 and key 1; where
 *   the data defeats that plan (a partition larger than a chunk, or with two
 *   keys more than 64 rows sharing key 0's high bits out of order) the LSD
 *   passes over all keys run instead, decided on the device without a host
 *   round trip.  The result is the same stable order.  Batches (vdf_batch_*)
 *   choose per query the same way (queries of 8-byte keys).  4-byte keys
 *   take the LSD passes: their four passes measured faster than the
 *   partition passes plus the shared-memory finish.
 * VDF_SORT_LSD: always the LSD passes (as the reference's radix sorts do,
 *   radix_sort_uint64_mt.inl:6-166).
 * VDF_SORT_MSD: the MSD-first plan for every key width where it fits (for
 *   tests and measurements). */
typedef enum vdf_sort_strategy {
    VDF_SORT_AUTO = 0,
    VDF_SORT_LSD = 1,
    VDF_SORT_MSD = 2
} vdf_sort_strategy;
vdf_status vdf_ctx_set_sort_strategy(vdf_ctx* ctx, int strategy, uint64_t msd_min_rows);
/* The dictionary plan (VDF_SORT_AUTO, sorts by ONE key column of at least
 * 4 x msd_min_rows rows): the key column's distinct values are collected on the
 * device first; with at most 256 of them the sort is one stable radix pass
 * over each key's rank among them (a category column: 1 pass instead of 4 or
 * 8), otherwise the MSD-first plan (8-byte keys) or the LSD passes run, as
 * decided on the device.  vdf_sort_plan_tries_dict: 1 when a sort of that
 * shape tries it (-1 for bad arguments); vdf_ctx_dict_stats: sorts of the
 * context that tried it and (reading the device counter, synchronising
 * `stream`) those that took it. */
int vdf_sort_plan_tries_dict(uint64_t n, const int32_t* key_dtypes, int nkeys, int strategy, uint64_t min_rows);
vdf_status vdf_ctx_dict_stats(vdf_ctx* ctx, void* stream, uint64_t* tried, uint64_t* taken);
vdf_status vdf_ctx_get_sort_strategy(vdf_ctx* ctx, int32_t* strategy, uint64_t* msd_min_rows);
/* The MSD-first sort's shared-memory finish.  Bit 0, digit matching of its
 * passes: 0 = one warp ballot per digit bit (default), 1 = match.any (the
 * autotuner's choice).  Bit 1: wide chunks (up to 8192 rows, one CTA of 1024
 * threads per SM) for every such sort; without it they are used only where
 * they save the third top-digit pass (between 100.7M and 201M rows). */
vdf_status vdf_ctx_set_local_sort_variant(vdf_ctx* ctx, int variant);
int vdf_ctx_get_local_sort_variant(vdf_ctx* ctx); /* -1 for a NULL context */
/* Failure injection for tests; nothing here faults the device.
 *   spin_limit : polls a look-back wait makes before it gives up, records
 *                VDF_ERR_TIMEOUT in the error bits and carries on (0: the
 *                default, about 2^20 polls, ~0.1 s)
 *   stall_tile : in the first radix pass of each later sort, the CTA that
 *                draws this tile leaves without publishing its counts, so the
 *                waits on it run out (UINT32_MAX: none); vdf_ctx_check then
 *                returns VDF_ERR_TIMEOUT and the sort's results are undefined
 *   fail_allocs: the next that many workspace allocations fail as a failed
 *                cudaMalloc would (VDF_ERR_OOM); the context stays usable
 * No counterpart in the reference. */
vdf_status vdf_ctx_set_test_hooks(vdf_ctx* ctx, uint32_t spin_limit, uint32_t stall_tile, uint32_t fail_allocs);
/* Sorts this context planned MSD-first, and how many of them fell back to
 * the LSD passes on the device (synchronises `stream`).  No counterpart in
 * the reference. */
vdf_status vdf_ctx_sort_stats(vdf_ctx* ctx, void* stream, uint64_t* msd_sorts, uint64_t* msd_fallbacks);
/* The plan a sort of n rows with these key dtypes gets under a strategy
 * (pure host function): global MSD passes (0 = LSD sort) and chunks. */
vdf_status vdf_sort_plan_info(uint64_t n, const int32_t* key_dtypes, int nkeys, int strategy, uint64_t msd_min_rows,
                              int32_t* msd_passes, uint32_t* chunks);

/* ---- workspace sizing (pure host functions) ------------------------------ */
/* Enough for every tuning; vdf_sort_argsort_ws also packs the other sorted
 * key columns into this buffer when it holds n * 16 * ceil((nkeys-1)/2)
 * bytes, else gathers them column by column. */
size_t vdf_sort_workspace_bytes(uint64_t n, const int32_t* key_dtypes, int nkeys);
size_t vdf_groupby_workspace_bytes(uint64_t n, int nvals);
/* Largest row count one call accepts (2^30 - 1 in this build). */
uint64_t vdf_max_rows(void);

/* ---- sort ----------------------------------------------------------------- */
/* Stable LSD radix argsort over nkeys key columns; keys[0] is the most
 * significant.  Writes perm_out[r] = source row of sorted row r (u32), and,
 * for each k with sorted_keys_out != NULL && sorted_keys_out[k] != NULL, the
 * raw key column k in sorted order.
 * Replaces sort_integers / sort_uintegers / sort_flt
 *   (V/inlines/transform/sort_by/sort_integers.inl:8-13 idx, col, nrow;
 *    sort_uintegers.inl:8-13; sort_flt.inl:8-13)
 * and the radix kernels they call, radix_sort_uint32[_mt] / radix_sort_uint64[_mt]
 *   (V/inlines/radix_sorts/radix_sort_uint64.inl:5-7 tkeys, idx, n;
 *    radix_sort_uint64_mt.inl:3-8), composed over several keys through the
 * idx in/out parameter (the reference has no multi-key sort entry point). */
vdf_status vdf_sort_argsort(vdf_ctx* ctx, uint64_t n, const vdf_col* keys, int nkeys, int order,
                            uint32_t* perm_out, void* const* sorted_keys_out, void* stream);
/* Same, with caller-owned workspace of at least vdf_sort_workspace_bytes(). */
vdf_status vdf_sort_argsort_ws(vdf_ctx* ctx, uint64_t n, const vdf_col* keys, int nkeys, int order,
                               uint32_t* perm_out, void* const* sorted_keys_out, void* workspace,
                               size_t workspace_bytes, void* stream);

/* ---- sort without any allocation ------------------------------------------ */
/* Largest row count vdf_sort_argsort_noalloc accepts. */
#define VDF_NOALLOC_MAX_ROWS (1u << 20)
/* The same stable argsort as vdf_sort_argsort for callers that cannot
 * allocate device memory when they sort (inside another allocator's
 * callback, under a host framework that forbids run-time allocations, or on
 * a latency-critical path that must not trigger the synchronisation
 * cudaMalloc/cudaFree can imply).  It takes no context and calls no
 * cudaMalloc, cudaFree or other allocating routine: its scratch is a fixed
 * 28 MiB device array inside the library, held on every GPU where the
 * library's module holding it is loaded (the first call on that GPU) until the
 * process exits.  The first call on a device looks up the array's device
 * address and prepares the kernels, so make it before any stream capture.
 * n above VDF_NOALLOC_MAX_ROWS returns VDF_ERR_UNSUPPORTED.  All calls on a
 * device share the one array: calls that overlap on the GPU (other streams,
 * other host threads) race and corrupt each other's results; serialise them.
 * The call is asynchronous on `stream`; device-side wait timeouts are read
 * back with vdf_sort_noalloc_error.  No counterpart in the reference: the reference's radix sort
 * always allocates its buffers (radix_sort_uint64.inl:23-24). */
vdf_status vdf_sort_argsort_noalloc(uint64_t n, const vdf_col* keys, int nkeys, int order, uint32_t* perm_out,
                                    void* const* sorted_keys_out, void* stream);
/* The device error bits of the last vdf_sort_argsort_noalloc call on the
 * current device (0 = none; bit 0: a bounded wait gave up, bit 1: an
 * out-of-range row id), copied into *host_out after `stream` has drained.
 * Allocates nothing.  No counterpart in the reference. */
vdf_status vdf_sort_noalloc_error(uint32_t* host_out, void* stream);

/* ---- gather ---------------------------------------------------------------- */
/* out[c][r] = in[c].data[perm[r]] for ncols (<= 8) columns in one launch.
 * Replaces permute_block_mt (V/inlines/transform/sort_by/permute_block_mt.inl:3-47),
 * no_inplace_permutation (V/inlines/no_inplace_permutation.inl:3-79) and the
 * per-block loop of materialize_mt (V/materialize/materialize_mt.hpp:6-55). */
vdf_status vdf_gather(vdf_ctx* ctx, uint64_t n, const uint32_t* perm, const vdf_col* in, int ncols,
                      void* const* out, void* stream);

/* ---- group-by over sorted rows -------------------------------------------- */
/* Key and value columns are already in key order (e.g. the outputs of
 * vdf_sort_argsort + vdf_gather).  Finds segment boundaries and writes, per
 * group in ascending row order: group_keys_out[k][g], count_out[g] (int64),
 * and the vdf_agg_out of each value column.  group_start_out[g] = first
 * sorted row of group g; row_group_out[r] = group of sorted row r (both
 * optional, u32).  The group count goes to *n_groups_dev (device, async)
 * and/or *n_groups_host (host; the call then synchronises `stream`).
 * Replaces the hash group-by loop of transform_group_by_onecol_mt
 * (V/transform/transform_group_by/transform_group_by_onecol_mt.hpp:182-337,
 * AddLookupOneCol / OccLookupOneCol V/inlines/transform/transform_group_by/
 * onecol_functions.inl:4-86, MergeCurMap merge_functions.inl:3-36) and the
 * multi-key variants (_sametype_mt / _difftype_mt via KeyBuildSameType /
 * KeyBuildDiffType, key_build.inl:3-110). */
vdf_status vdf_groupby_sorted(vdf_ctx* ctx, uint64_t n, const vdf_col* keys, int nkeys,
                              const vdf_col* vals, int nvals, void* const* group_keys_out,
                              int64_t* count_out, const vdf_agg_out* aggs, uint32_t* group_start_out,
                              uint32_t* row_group_out, uint64_t* n_groups_dev, uint64_t* n_groups_host,
                              void* stream);

/* ---- pivot ------------------------------------------------------------------ */
/* A string column: bytes, and n + 1 offsets (row r = bytes[offsets[r] ..
 * offsets[r + 1]), offsets[0] = 0). */
typedef struct vdf_strcol {
    const char* bytes;
    const uint64_t* offsets;
} vdf_strcol;
/* Pivot (replaces V/pivots/pivot.hpp:5-128): the sum of `value` over the
 * rows of each (col key, row key) pair, as a matrix with one column per
 * distinct col key and one row per distinct row key, both in order of first
 * appearance; a pair that never occurs is 0.  Keys compare by their bytes.
 * value: VDF_I32 / VDF_U32 / VDF_F64 (the reference's IntT, UIntT, FloatT)
 * or VDF_I64 / VDF_U64; integer sums wrap in the value type as the
 * reference's "+=" does, f64 sums are compensated (within 1e-12 relative of
 * the row-order sum).  Host memory, synchronous.  Writes *n_colkeys,
 * *n_rowkeys and each key's first row (colkey_row / rowkey_row, capacity n
 * each); then the matrix, n_colkeys x n_rowkeys values of the value dtype,
 * one output column after another (cell (c, r) at c * n_rowkeys + r), when
 * it fits in matrix_cap values, else VDF_ERR_WORKSPACE with the counts and
 * first rows written (call again with a matrix that fits).  The keys are
 * dictionary-encoded on the device (a hash table of the strings, first rows
 * by atomic minimum, ranks by a scan) and the pairs summed on the sorted
 * path (vdf_sort_groupby). */
vdf_status vdf_pivot_host(vdf_ctx* ctx, uint64_t n, vdf_strcol col_key, vdf_strcol row_key, vdf_col value,
                          uint32_t* n_colkeys, uint32_t* n_rowkeys, uint32_t* colkey_row, uint32_t* rowkey_row,
                          void* matrix, uint64_t matrix_cap);

/* ---- fused sort + payload gather + group-by --------------------------------- */
typedef struct vdf_sort_groupby_args {
    uint64_t n;
    const vdf_col* keys;      /* nkeys key columns, most significant first       */
    int32_t nkeys;
    int32_t order;            /* vdf_order                                       */
    const vdf_col* payload;   /* npayload (<= 8) payload columns                 */
    int32_t npayload;
    /* sort outputs (each may be NULL) */
    uint32_t* perm_out;            /* n row ids; NULL = internal buffer            */
    void* const* sorted_keys_out;  /* nkeys entries (entries may be NULL)          */
    void* const* payload_out;      /* npayload entries (entries may be NULL)       */
    /* group-by (groupby == 0: sort + gather only) */
    int32_t groupby;
    const int32_t* agg_cols;       /* indices into payload of the aggregated columns */
    int32_t nagg;                  /* <= 4                                           */
    void* const* group_keys_out;   /* nkeys entries (entries may be NULL)          */
    int64_t* group_count_out;
    const vdf_agg_out* aggs;       /* nagg entries                                   */
    uint32_t* group_start_out;
    uint32_t* row_group_out;
    uint64_t* n_groups_dev;
    uint64_t* n_groups_host;       /* non-NULL: the call synchronises `stream`       */
    /* optional permutation of [0, n) through which the rows are seen (a row
     * view): the sort orders rows[perm_in[i]] and perm_out is composed with it,
     * like the in/out idx of the reference's radix_sort_uint64
     * (V/inlines/radix_sorts/radix_sort_uint64.inl:5-7).  NULL = identity. */
    const uint32_t* perm_in;
} vdf_sort_groupby_args;

/* One call for the whole path: sort by the keys, gather every payload column
 * by the permutation and aggregate the chosen payload columns per group; the
 * payload gather is fused into the group-by pass.  Replaces the composition
 * sort_by_mt (V/transform/sort_by/sort_by_mt.hpp:3-180, Soft=false:
 * permute_block_mt over every type block :117-159) followed by
 * transform_group_by_mt (V/transform/transform_group_by/
 * transform_group_by_mt.hpp:12-114), in the segment layout of the "hard"
 * variant (hard/transform_group_by_onecol_hard_mt.hpp:11-372). */
vdf_status vdf_sort_groupby(vdf_ctx* ctx, const vdf_sort_groupby_args* args, void* stream);

/* The same call on HOST memory: every column, output and n_groups_host
 * pointer in `args` is a host pointer (n_groups_dev is ignored).  The inputs
 * are copied to the device, the path runs there, the outputs come back (the
 * sorted frame as n rows, the group table as n_groups rows) and the call
 * returns after synchronising `stream`.  Page-locked host buffers make the
 * copies asynchronous and fast; ordinary ones work too.  This is the entry
 * point behind the header-only dataframe layer (include/vison_b200/vison.hpp),
 * replacing the same reference calls as vdf_sort_groupby on the reference's
 * own host-resident columns (V/vison.hpp:207-212). */
vdf_status vdf_sort_groupby_host(vdf_ctx* ctx, const vdf_sort_groupby_args* args, void* stream);

/* Host-memory gather: out[c][r] = in[c].data[perm[r]] with perm, in and out
 * in host memory (synchronises `stream`).  Replaces materialize_mt
 * (V/materialize/materialize_mt.hpp:6-55) on host-resident columns. */
vdf_status vdf_gather_host(vdf_ctx* ctx, uint64_t n, const uint32_t* perm, const vdf_col* in, int ncols,
                           void* const* out, void* stream);

/* Aggregate functions of the transform-style group-by. */
typedef enum vdf_agg_fn {
    VDF_AGG_COUNT = 0, /* int64 rows in the group (GroupFunction::Occurence)        */
    VDF_AGG_SUM = 1,   /* double for float values, int64 low word of the exact sum */
    VDF_AGG_MEAN = 2,  /* double sum / count                                        */
    VDF_AGG_MIN = 3,   /* value dtype (extension: the reference has no min)         */
    VDF_AGG_MAX = 4    /* value dtype (extension: the reference has no max)         */
} vdf_agg_fn;

/* The reference's transform group-by on host memory: groups the n rows by the
 * key columns, aggregates `val` with `function`, and writes to `out` (host, n
 * elements) every row's group value in the frame's row order, as
 * transform_group_by does (V/transform/transform_group_by/
 * transform_group_by.hpp:3-113, CreateValueCol::apply create_value_col.inl:
 * 36-61).  perm_in (host, optional) is the frame's row view.  The group
 * count goes to *n_groups_host.  Synchronises `stream`. */
vdf_status vdf_transform_groupby_host(vdf_ctx* ctx, uint64_t n, const vdf_col* keys, int nkeys, vdf_col val,
                                      int32_t function, const uint32_t* perm_in, void* out, uint64_t* n_groups_host,
                                      void* stream);

/* ---- transform output --------------------------------------------------------- */
/* out[perm ? perm[r] : r] = group_vals[row_group[r]] (width 4 or 8 bytes,
 * n_groups entries in group_vals): broadcasts a per-group aggregate back to
 * every row, in sorted order or (perm != NULL) in the frame's original row
 * order.  Out-of-range group or row ids are skipped and raise the context's
 * error bits (see vdf_ctx_check).  Replaces
 * CreateValueCol::apply (V/inlines/transform/transform_group_by/
 * create_value_col.inl:36-61) and the segment fill of CreateValueColHard
 * (hard/create_value_col_hard.inl:38-59). */
vdf_status vdf_broadcast(vdf_ctx* ctx, uint64_t n, const uint32_t* row_group, const void* group_vals,
                         uint64_t n_groups, int width, const uint32_t* perm, void* out, void* stream);

/* ---- de-duplication and left-join row matching ------------------------------
 * Both run on the sorted path: a stable ascending radix sort of the key
 * column puts each key value's rows in one run in row order, so the run's
 * first (last) row is the value's first (last) occurrence.  Keys compare by
 * their raw bits (-0.0 and +0.0 differ; a NaN equals a NaN with the same
 * bits), as the reference's byte-wise hash lookups do.  The counts go to
 * *..._dev (device, async) and/or *..._host (host; the call then
 * synchronises `stream`); both are optional. */

/* keep_out[i] (u8) = 1 if row i is the first occurrence of its key
 * (keep_last = 0) or the last (keep_last = 1), else 0; the number of distinct
 * keys is the count.  Replaces the set walk of transform_unique_mt
 * (V/transform/transform_unique/transform_unique_mt.hpp:105-140), which marks
 * the same rows with mask[i] = 0 before its filter step (:173). */
vdf_status vdf_unique(vdf_ctx* ctx, uint64_t n, vdf_col key, int keep_last, uint8_t* keep_out,
                      uint64_t* n_unique_dev, uint64_t* n_unique_host, void* stream);

/* Left-join matching methods (LeftJoinMethods, V/types/supported_leftjoin_methods.inl:1-5). */
typedef enum vdf_join_method {
    VDF_JOIN_FIRST = 0,   /* the key's first right row                                  */
    VDF_JOIN_LAST = 1,    /* the key's last right row                                   */
    VDF_JOIN_ALIGNED = 2  /* the k-th left occurrence of a key takes its k-th right row */
} vdf_join_method;

/* match_out[i] (u32) = the row of the right column that left row i takes
 * under `method`, or UINT32_MAX when there is none (the key is absent, or,
 * for VDF_JOIN_ALIGNED, the right side has fewer rows of it); the number of
 * matched left rows is the count.  Both columns have the same dtype.
 * Replaces the map build and probe of transform_left_join_mt
 * (V/transform/transform_left_join/transform_left_join_mt.hpp:172-238),
 * whose match_idx holds SIZE_MAX for unmatched rows.  Aligned sorts the left
 * side as well (its rows' occurrence ranks). */
vdf_status vdf_left_join_index(vdf_ctx* ctx, uint64_t n_left, vdf_col left_key, uint64_t n_right,
                               vdf_col right_key, int method, uint32_t* match_out, uint64_t* n_matched_dev,
                               uint64_t* n_matched_host, void* stream);

/* The same two operations on HOST columns and outputs (copied through the
 * context's staging buffer; synchronise `stream`): the entry points of the
 * C++ dataframe layer (transform_unique / transform_left_join in
 * include/vison_b200/vison.hpp). */
vdf_status vdf_unique_host(vdf_ctx* ctx, uint64_t n, vdf_col key, int keep_last, uint8_t* keep_out,
                           uint64_t* n_unique, void* stream);
vdf_status vdf_left_join_index_host(vdf_ctx* ctx, uint64_t n_left, vdf_col left_key, uint64_t n_right,
                                    vdf_col right_key, int method, uint32_t* match_out, uint64_t* n_matched,
                                    void* stream);

/* ---- CSV ingest -------------------------------------------------------------
 * Parses a CSV file's bytes into device-resident columns: the reference's
 * read_csv (V/read/read_csv/read_csv.hpp:3-216, called as Dataframe::readf,
 * benchmarks/readf.cpp:21) with its single-core parser
 * (V/inlines/read/read_csv/parsers_core/parse_rows_chunk.inl:1-185) and type
 * inference (V/inlines/classify_column.inl:13-133):
 *   - the first line holds the names (header = 1) or the first data row; it
 *     ends at the first CR or LF even inside quotes (read_csv.hpp:62-69);
 *   - records end at a CR, LF or CR LF outside quotes; fields split at the
 *     delimiter outside quotes; the quote byte toggles quoting and stays in
 *     the field's text; an empty field reads "NA";
 *   - a record with another field count than the first line is an error
 *     (VDF_ERR_INVALID_ARG, "column number problem at row r"), where the
 *     reference prints "column number problem" and stops;
 *   - each column's type comes from its first 10 values: 'd' (double, the
 *     first number with a '.' decides), 's' / 'c' (a value that is not digits
 *     with at most one '.': 's' if it is longer than one byte), 'b' (all "0"
 *     or "1"), 'u' (unsigned 32-bit);
 *   - values: 'd' as fast_float::from_chars (correctly rounded; 0 when invalid
 *     or out of range), 'u' as std::from_chars into unsigned int, 'b' as
 *     std::from_chars into int != 0 (0 when invalid or out of range); strings
 *     keep their bytes (offsets + bytes, "NA" for an empty field).
 * Limits: files below 4 GiB, at most 4096 columns of which at most 64 are
 * strings (VDF_ERR_UNSUPPORTED beyond).  The table owns its device columns;
 * they come from a stream-ordered pool per device that keeps up to 8 GiB
 * cached between reads. */
typedef struct vdf_csv vdf_csv;

/* `bytes`: n bytes in device memory (16-byte aligned).  Synchronises `stream`. */
vdf_status vdf_csv_read(vdf_ctx* ctx, const void* bytes, uint64_t n, char delim, int header, char quote,
                        vdf_csv** out, void* stream);
/* The same for a file's bytes in host memory (copied to the device first). */
vdf_status vdf_csv_read_host(vdf_ctx* ctx, const void* bytes, uint64_t n, char delim, int header, char quote,
                             vdf_csv** out, void* stream);
uint64_t vdf_csv_nrow(const vdf_csv* t);
uint32_t vdf_csv_ncol(const vdf_csv* t);
/* Column name ("" without a header; "NA" for an empty header field). */
const char* vdf_csv_name(const vdf_csv* t, uint32_t col);
/* 'd' (f64), 'u' (u32), 'b' (u8 0/1), 's' or 'c' (string). */
char vdf_csv_type(const vdf_csv* t, uint32_t col);
/* Device pointer to the values (numbers) or the concatenated string bytes. */
const void* vdf_csv_values(const vdf_csv* t, uint32_t col);
/* Device pointer to nrow + 1 string offsets (NULL for numbers). */
const uint64_t* vdf_csv_offsets(const vdf_csv* t, uint32_t col);
uint64_t vdf_csv_string_bytes(const vdf_csv* t, uint32_t col);
/* Copies one column into host or device memory: values (nrow elements, or
 * the string bytes) and, for strings, the nrow + 1 offsets (either may be
 * NULL).  Synchronises `stream`. */
vdf_status vdf_csv_copy_column(vdf_ctx* ctx, const vdf_csv* t, uint32_t col, void* values, uint64_t* offsets,
                               void* stream);
/* Frees the table's columns once no work can still use them (it waits for
 * the device, as cudaFree does). */
void vdf_csv_free(vdf_csv* t);

/* ---- batched queries ------------------------------------------------------
 * Many independent sort + group-by queries (each: stable ascending sort of
 * one key column, then count/sum/min/max/mean of every value column per
 * key) planned once and run as one fixed sequence of launches.  The
 * reference runs them one call each (sort_by_mt, V/transform/sort_by/
 * sort_by_mt.hpp:3-180, then transform_group_by_onecol_mt,
 * V/transform/transform_group_by/transform_group_by_onecol_mt.hpp:14-373). */
#define VDF_BATCH_MAX_VALS 4

/* One query: n rows of one key column and nvals value columns (device
 * pointers; the value dtypes are the batch's). */
typedef struct vdf_batch_query {
    uint64_t n;
    vdf_col key;
    const void* vals[VDF_BATCH_MAX_VALS];
} vdf_batch_query;

/* Execution choices (vdf_batch_default_tuning; the Python autotuner searches
 * them).  Queries of at most small_rows rows (<= 8192) are each sorted and
 * grouped by one CTA in shared memory, with small_bits-bit digits (4 or 8);
 * the others are sorted together by the segmented radix passes of variant
 * seg_variant (vdf_batch_variant_info: digit bits, rows per tile). */
typedef struct vdf_batch_tuning {
    uint32_t small_rows;
    int32_t small_bits;
    int32_t seg_variant;
} vdf_batch_tuning;

/* Outputs are arenas of vdf_batch_rows(batch) = sum of n rows / group slots
 * (device arrays, caller-owned):
 *   perm_out[row_offset[q] + i]      i-th row (0-based within q) of q in key order
 *   group slot group_offset[q] + g   q's g-th group (ascending key), g < n_groups[q]:
 *       group_count_out[slot], aggs[j].sum/sum_hi/min/max/mean[slot]
 *       (vdf_agg_out semantics); group keys are packed in q's own key
 *       width from byte 8 * group_offset[q] of group_keys_out (8 bytes per slot)
 *   row_offset_out, group_offset_out, n_groups_out: device [nqueries]
 * A query of 0 rows has n_groups 0. */
typedef struct vdf_batch_args {
    uint32_t nqueries;
    const vdf_batch_query* queries; /* host array, copied by vdf_batch_create */
    int32_t nvals;
    int32_t val_dtypes[VDF_BATCH_MAX_VALS];
    uint32_t* perm_out;
    void* group_keys_out;     /* may be NULL */
    int64_t* group_count_out; /* may be NULL */
    vdf_agg_out aggs[VDF_BATCH_MAX_VALS];
    uint64_t* row_offset_out;
    uint64_t* group_offset_out;
    uint64_t* n_groups_out;
} vdf_batch_args;

typedef struct vdf_batch vdf_batch;

int vdf_batch_variant_count(void);
vdf_status vdf_batch_variant_info(int index, int32_t* digit_bits, int32_t* tile_rows);
vdf_status vdf_batch_default_tuning(vdf_batch_tuning* tuning);

/* Plans the batch (tuning NULL = default), sizes the context workspace for
 * it and uploads its descriptor tables; synchronous.  Writes row_offset_out
 * now.  The batch uses the context's workspace: a later call on the context
 * that needs a larger workspace invalidates it (launch then fails with
 * VDF_ERR_WORKSPACE), and its launches must not overlap other work of the
 * context on the GPU. */
vdf_status vdf_batch_create(vdf_ctx* ctx, const vdf_batch_args* args, const vdf_batch_tuning* tuning,
                            vdf_batch** out);
/* Rows (= group slots) of the batch's output arenas. */
uint64_t vdf_batch_rows(const vdf_batch* batch);
/* How the plan split the queries (any pointer may be NULL). */
vdf_status vdf_batch_info(const vdf_batch* batch, uint32_t* small_queries, uint64_t* small_rows,
                          uint32_t* large_queries, uint64_t* large_rows);
/* How the sort treats the large queries: msd_queries take the MSD-first
 * sort (top-digit passes, then chunks finished in shared memory), the other
 * lsd_queries the LSD passes.  With fallbacks non-NULL it waits for the
 * device and counts the MSD queries of the last launch whose chunks defeated
 * the plan, so that the LSD passes sorted them instead (any pointer may be
 * NULL). */
vdf_status vdf_batch_sort_info(vdf_batch* batch, uint32_t* msd_queries, uint32_t* lsd_queries,
                               uint32_t* fallbacks);
/* Enqueues the batch on `stream`: no allocation, no host synchronisation,
 * no host memory read, so it can be stream-captured.  Device-side wait
 * timeouts are reported by vdf_ctx_check. */
vdf_status vdf_batch_launch(vdf_batch* batch, void* stream);
/* The same work as one CUDA graph: captured on the first call, replayed on
 * every call (one graph launch). */
vdf_status vdf_batch_launch_graph(vdf_batch* batch, void* stream);
void vdf_batch_destroy(vdf_batch* batch);

/* ---- request loop (serving) -------------------------------------------------
 * Sort + group-by requests over device-resident columns, submitted and polled
 * by id.  A scheduler thread admits requests first-come first-served while the
 * device memory they hold (their output arenas) fits the HBM budget, and runs
 * them with continuous batching: whenever one of `slots` execution slots (a
 * context with its own stream and a workspace reserved for max_batch_rows
 * rows) is free, every admitted waiting request, up to the batch limits, joins
 * one batch (vdf_batch_*); batches of different slots overlap on the device.
 * A request's columns must stay valid until it is done; its results (device
 * pointers into its slot's output arenas, allocated once per slot) stay valid
 * until vdf_server_release, and a slot takes its next batch only when every
 * result of its previous batch has been released.
 * No counterpart in the reference (one sort_by_mt + transform_group_by call per
 * query). */
typedef struct vdf_server_config {
    int32_t device;
    uint64_t hbm_budget_bytes;  /* everything the server holds + resident_bytes */
    uint64_t resident_bytes;    /* the caller's resident columns, counted against the budget */
    uint32_t slots;             /* batches in flight (1..8) */
    uint64_t max_batch_rows;
    uint32_t max_batch_queries;
    int32_t nvals;              /* value columns per request, same dtypes for all */
    int32_t val_dtypes[VDF_BATCH_MAX_VALS];
    int32_t use_default_tuning; /* else the three fields below (vdf_batch_tuning) */
    uint32_t small_rows;
    int32_t small_bits;
    int32_t seg_variant;
    int32_t use_graph;          /* launch each batch as a captured CUDA graph */
} vdf_server_config;

typedef struct vdf_server_result {
    uint64_t n, n_groups;
    const uint32_t* perm;       /* n sorted row ids */
    const void* group_keys;     /* n_groups keys, the request's key dtype */
    const int64_t* group_count; /* n_groups */
    vdf_agg_out aggs[VDF_BATCH_MAX_VALS];
    double t_submit, t_start, t_done; /* seconds since the server was created */
} vdf_server_result;

typedef struct vdf_server_stats {
    uint64_t batches, completed, queued;
    uint64_t in_use_bytes, max_in_use_bytes, fixed_bytes;
    double host_start_seconds, host_finish_seconds; /* scheduler time spent planning/launching and reading back batches */
} vdf_server_stats;

typedef struct vdf_server vdf_server;

/* States reported by vdf_server_poll. */
#define VDF_REQ_QUEUED 0
#define VDF_REQ_RUNNING 1
#define VDF_REQ_DONE 2
#define VDF_REQ_FAILED 3

vdf_status vdf_server_default_config(vdf_server_config* cfg);
vdf_status vdf_server_create(const vdf_server_config* cfg, vdf_server** out);
/* Queues a request; VDF_ERR_OOM if it could never fit the budget,
 * VDF_ERR_UNSUPPORTED above max_batch_rows rows. */
vdf_status vdf_server_submit(vdf_server* srv, const vdf_batch_query* query, uint64_t* request_id);
/* Current state; with out, the result once done (timestamps always). */
vdf_status vdf_server_poll(vdf_server* srv, uint64_t request_id, int32_t* state, vdf_server_result* out);
/* Blocks until the request is done or failed (VDF_ERR_TIMEOUT after timeout_s). */
vdf_status vdf_server_wait(vdf_server* srv, uint64_t request_id, double timeout_s, vdf_server_result* out);
/* Gives the request's result memory back (once every request of its batch
 * is released, the batch's outputs return to the allocator). */
vdf_status vdf_server_release(vdf_server* srv, uint64_t request_id);
vdf_status vdf_server_read_stats(vdf_server* srv, vdf_server_stats* out);
/* Failure injection for tests: the next `count` batches fail with `status`
 * when they start (where = 0: planning and launch) or when they finish
 * (where = 1: reading back the results), as a real failure there would; the
 * batch's requests end VDF_REQ_FAILED with that status and later requests
 * are served as usual. */
vdf_status vdf_server_inject_failure(vdf_server* srv, int where, uint32_t count, vdf_status status);
const char* vdf_server_last_error(vdf_server* srv);
/* Stops the scheduler after the batches in flight and frees everything. */
void vdf_server_destroy(vdf_server* srv);

#ifdef __cplusplus
}
#endif

#endif /* VDF_CAPI_H */
