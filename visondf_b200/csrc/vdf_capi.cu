// vdf_capi.cu -- the extern "C" boundary declared in include/vdf_capi.h:
// argument checks, the context (device, grow-only workspace, device error
// word, launch counter) and the composition of the sort, gather and
// segmented-reduction kernels into the public operations.
#include <cstring>

#include "vdf_batch.h"
#include "vdf_ctx.h"

namespace {
using namespace vdfc;

vdf_status check_keys(vdf_ctx* c, uint64_t n, const vdf_col* keys, int nkeys) {
    if (nkeys < 1 || nkeys > vdf::kMaxKeys) return fail(c, VDF_ERR_INVALID_ARG, "nkeys must be 1..%d", vdf::kMaxKeys);
    if (!keys) return fail(c, VDF_ERR_INVALID_ARG, "keys is NULL");
    for (int k = 0; k < nkeys; ++k) {
        if (!valid_dtype(keys[k].dtype)) return fail(c, VDF_ERR_INVALID_ARG, "key %d: bad dtype %d", k, keys[k].dtype);
        if (n && !keys[k].data) return fail(c, VDF_ERR_INVALID_ARG, "key %d: NULL data", k);
    }
    return VDF_OK;
}

vdf_status check_rows(vdf_ctx* c, uint64_t n) {
    if (n > kMaxRows) return fail(c, VDF_ERR_UNSUPPORTED, "n=%llu exceeds the %llu-row limit", (unsigned long long)n,
                                  (unsigned long long)kMaxRows);
    return VDF_OK;
}

// Sorted copies of key columns 1..nkeys-1 (column 0 is written by the last
// radix pass) by gathering through the permutation.
vdf_status emit_other_keys(vdf_ctx* c, uint64_t n, const vdf_col* keys, int nkeys, const uint32_t* perm,
                           void* const* sorted_keys_out, void* rec_ws, size_t rec_ws_bytes, cudaStream_t s) {
    if (!sorted_keys_out) return VDF_OK;
    vdf::GatherArgs g{};
    g.perm = perm;
    g.err = err_word(c);
    g.n = n;
    for (int k = 1; k < nkeys; ++k) {
        if (!sorted_keys_out[k]) continue;
        g.src[g.ncols] = keys[k].data;
        g.dst[g.ncols] = sorted_keys_out[k];
        g.width[g.ncols] = vdf::dtype_width(keys[k].dtype);
        g.ncols++;
    }
    if (!g.ncols) return VDF_OK;
    int launched = 0;
    cudaError_t e = vdf::run_gather(g, s, prof_of(c), rec_ws, rec_ws_bytes, &launched);
    c->launches += launched;
    return from_cuda(c, e, "gather keys");
}

// Workspace a sort needs: the radix buffers, then (reusing them once the
// sort is done) the packed records of the other sorted key columns.
size_t sort_ws_need(const vdf::SortPlan& p, uint64_t n, int nkeys, void* const* sorted_keys_out) {
    int other = 0;
    for (int k = 1; k < nkeys; ++k) other += (sorted_keys_out && sorted_keys_out[k]) ? 1 : 0;
    return std::max(p.ws_bytes, (size_t)n * vdf::gather_record_bytes(other));
}
// ... plus, for a multi-key sort tried primary key first without a sorted
// output for that key, room for its sorted copy beside its own sort.
size_t primary_first_need(vdf_ctx* c, uint64_t n, const int32_t* dts, int nkeys, void* const* sorted_keys_out) {
    if (nkeys < 2 || c->multikey_mode != VDF_MULTIKEY_PRIMARY_FIRST || (sorted_keys_out && sorted_keys_out[0]))
        return 0;
    if (vdf::make_sort_plan(n, dts, nkeys, c->tuning).msd) return 0;
    const vdf::SortPlan p0 = vdf::make_sort_plan(n, dts, 1, c->tuning);
    return align256(p0.ws_bytes) + (size_t)n * vdf::dtype_width(dts[0]);
}

// Multi-key sorts, primary key first: sort by the most significant key alone,
// then look for equal neighbours in its sorted copy.  With none, no two rows
// share the primary key, so that order already is the stable order over all
// keys (later keys only break ties) and the sort is done; otherwise the caller
// runs the LSD sort over all keys, overwriting perm and key0.  The check reads
// one flag back, so it synchronises the stream once; under stream capture, or
// with VDF_MULTIKEY_LSD, it is skipped.  key0_out may be null, in which case
// the primary key's sorted copy goes to scratch after the sort's workspace.
// Returns VDF_OK with *done telling which case happened.
vdf_status primary_first(vdf_ctx* c, uint64_t n, const int32_t* dts, const void* const* cols, int nkeys, int order,
                         uint32_t* perm, void* key0_out, unsigned char* ws, size_t ws_bytes, cudaStream_t s,
                         const uint32_t* perm_in, bool* done) {
    *done = false;
    if (nkeys < 2 || c->multikey_mode != VDF_MULTIKEY_PRIMARY_FIRST || n < 2) return VDF_OK;
    // the MSD-first plan sorts by both keys at once without a host round trip
    if (vdf::make_sort_plan(n, dts, nkeys, c->tuning).msd) return VDF_OK;
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(s, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone) {
        cudaGetLastError();
        return VDF_OK;
    }
    const vdf::SortPlan p0 = vdf::make_sort_plan(n, dts, 1, c->tuning);
    size_t need = p0.ws_bytes;
    void* k0 = key0_out;
    if (!k0) {
        k0 = ws + align256(p0.ws_bytes);
        need = align256(p0.ws_bytes) + (size_t)n * vdf::dtype_width(dts[0]);
    }
    if (need > ws_bytes) return VDF_OK;  // no room: the LSD sort over all keys
    cudaError_t e = ctx_run_sort(c, p0, cols, order, perm, k0, ws, s, perm_in);
    if (e == cudaSuccess) e = cudaMemsetAsync(tie_word(c), 0, sizeof(uint32_t), s);
    if (e == cudaSuccess) e = vdf::flag_adjacent_ties(k0, vdf::dtype_width(dts[0]), n, tie_word(c), s, prof_of(c));
    c->launches += 1;
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(&c->host_pinned[2], tie_word(c), sizeof(uint32_t), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return from_cuda(c, e, "primary-key sort");
    *done = (static_cast<uint32_t>(c->host_pinned[2]) == 0);
    return VDF_OK;
}

vdf_status sort_impl(vdf_ctx* c, uint64_t n, const vdf_col* keys, int nkeys, int order, uint32_t* perm_out,
                     void* const* sorted_keys_out, unsigned char* ws, size_t ws_bytes, cudaStream_t s) {
    int32_t dts[vdf::kMaxKeys];
    const void* cols[vdf::kMaxKeys];
    for (int k = 0; k < nkeys; ++k) {
        dts[k] = keys[k].dtype;
        cols[k] = keys[k].data;
    }
    vdf::SortPlan p = vdf::make_sort_plan(n, dts, nkeys, c->tuning);
    if (ws_bytes < p.ws_bytes)
        return fail(c, VDF_ERR_WORKSPACE, "workspace of %zu bytes < %zu needed", ws_bytes, p.ws_bytes);
    void* key0_out = sorted_keys_out ? sorted_keys_out[0] : nullptr;
    bool done = false;
    vdf_status pst = primary_first(c, n, dts, cols, nkeys, order, perm_out, key0_out, ws, ws_bytes, s, nullptr, &done);
    if (pst != VDF_OK) return pst;
    if (!done) {
        cudaError_t e = ctx_run_sort(c, p, cols, order, perm_out, key0_out, ws, s);
        if (e != cudaSuccess) return from_cuda(c, e, "radix sort");
    }
    return emit_other_keys(c, n, keys, nkeys, perm_out, sorted_keys_out, ws, ws_bytes, s);
}

vdf_status finish_groups(vdf_ctx* c, uint64_t* n_groups_dev, uint64_t* n_groups_host, cudaStream_t s) {
    if (!n_groups_host) return VDF_OK;
    const uint64_t* src = n_groups_dev ? n_groups_dev : count_word(c);
    cudaError_t e = cudaMemcpyAsync(&c->host_pinned[0], src, sizeof(uint64_t), cudaMemcpyDeviceToHost, s);
    if (e != cudaSuccess) return from_cuda(c, e, "read group count");
    vdf_status st = drain_and_check(c, s);
    if (st != VDF_OK) return st;
    *n_groups_host = c->host_pinned[0];
    return VDF_OK;
}

std::mutex g_prep_mu;
bool g_prepared[64];

}  // namespace

extern "C" {

uint32_t vdf_abi_version(void) { return VDF_ABI_VERSION; }

const char* vdf_status_string(vdf_status s) {
    switch (s) {
    case VDF_OK: return "ok";
    case VDF_ERR_INVALID_ARG: return "invalid argument";
    case VDF_ERR_OOM: return "out of device memory";
    case VDF_ERR_TIMEOUT: return "device wait timed out";
    case VDF_ERR_DEVICE: return "CUDA error";
    case VDF_ERR_UNSUPPORTED: return "unsupported";
    case VDF_ERR_WORKSPACE: return "workspace too small";
    }
    return "unknown status";
}

uint64_t vdf_max_rows(void) { return kMaxRows; }

size_t vdf_sort_workspace_bytes(uint64_t n, const int32_t* key_dtypes, int nkeys) {
    if (!key_dtypes || nkeys < 1 || nkeys > vdf::kMaxKeys) return 0;
    for (int k = 0; k < nkeys; ++k)
        if (!valid_dtype(key_dtypes[k])) return 0;
    // the largest over every kernel-variant choice, so it fits any tuning
    size_t best = 0;
    const int nv = vdf::sort_variant_count();
    for (int a = 0; a < nv; ++a)
        for (int b = 0; b < nv; ++b)
            for (int msd = 0; msd < 2; ++msd)
                for (int dict = 0; dict < 2; ++dict) {
                    vdf::SortTuning t{a, b, msd, 0};
                    t.dict = dict;
                    if (vdf::sort_tuning_valid(t))
                        best = std::max(best, vdf::make_sort_plan(n, key_dtypes, nkeys, t).ws_bytes);
                }
    return best;
}

int vdf_sort_variant_count(void) { return vdf::sort_variant_count(); }

vdf_status vdf_sort_variant_info(int index, int32_t* key_width, int32_t* threads, int32_t* items_per_thread,
                                 int32_t* digit_bits, int32_t* match) {
    int w, t, i, b, m;
    if (!vdf::sort_variant_info(index, &w, &t, &i, &b, &m)) return VDF_ERR_INVALID_ARG;
    if (key_width) *key_width = w;
    if (threads) *threads = t;
    if (items_per_thread) *items_per_thread = i;
    if (digit_bits) *digit_bits = b;
    if (match) *match = m;
    return VDF_OK;
}

uint32_t vdf_sort_variant_flags(int index) { return vdf::sort_variant_uses_tma(index) ? 1u : 0u; }

vdf_status vdf_ctx_set_group_tuning(vdf_ctx* c, uint32_t striped_min_heads) {
    if (!c) return VDF_ERR_INVALID_ARG;
    if (striped_min_heads > 512) return fail(c, VDF_ERR_INVALID_ARG, "striped_min_heads must be 0..512");
    std::lock_guard<std::mutex> lk(c->mu);
    c->emit_min_heads = striped_min_heads;
    return VDF_OK;
}

uint32_t vdf_ctx_get_group_tuning(vdf_ctx* c) {
    if (!c) return 0;
    std::lock_guard<std::mutex> lk(c->mu);
    return c->emit_min_heads ? c->emit_min_heads : vdf::kStripedMinHeads;
}

vdf_status vdf_ctx_set_sort_tuning(vdf_ctx* c, const vdf_sort_tuning* t) {
    if (!c || !t) return VDF_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> lk(c->mu);
    vdf::SortTuning st = c->tuning;
    st.variant32 = t->pass_variant32;
    st.variant64 = t->pass_variant64;
    if (!vdf::sort_tuning_valid(st)) return fail(c, VDF_ERR_INVALID_ARG, "invalid sort tuning %d/%d", st.variant32, st.variant64);
    c->tuning = st;
    return VDF_OK;
}

vdf_status vdf_ctx_get_sort_tuning(vdf_ctx* c, vdf_sort_tuning* t) {
    if (!c || !t) return VDF_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> lk(c->mu);
    t->pass_variant32 = c->tuning.variant32;
    t->pass_variant64 = c->tuning.variant64;
    return VDF_OK;
}

vdf_status vdf_ctx_set_multikey_mode(vdf_ctx* c, int mode) {
    if (!c) return VDF_ERR_INVALID_ARG;
    if (mode != VDF_MULTIKEY_LSD && mode != VDF_MULTIKEY_PRIMARY_FIRST)
        return fail(c, VDF_ERR_INVALID_ARG, "bad multi-key mode %d", mode);
    std::lock_guard<std::mutex> lk(c->mu);
    c->multikey_mode = mode;
    return VDF_OK;
}

int vdf_ctx_get_multikey_mode(vdf_ctx* c) {
    if (!c) return -1;
    std::lock_guard<std::mutex> lk(c->mu);
    return c->multikey_mode;
}

// SortTuning::msd of a strategy: 0 LSD, 1 MSD-first for 8-byte key 0, 2 for every width
static int msd_mode_of(int strategy) {
    return strategy == VDF_SORT_MSD ? 2 : (strategy == VDF_SORT_AUTO ? 1 : 0);
}

vdf_status vdf_ctx_set_sort_strategy(vdf_ctx* c, int strategy, uint64_t msd_min_rows) {
    if (!c) return VDF_ERR_INVALID_ARG;
    if (strategy != VDF_SORT_AUTO && strategy != VDF_SORT_LSD && strategy != VDF_SORT_MSD)
        return fail(c, VDF_ERR_INVALID_ARG, "bad sort strategy %d", strategy);
    std::lock_guard<std::mutex> lk(c->mu);
    c->tuning.msd = msd_mode_of(strategy);
    c->tuning.dict = strategy == VDF_SORT_AUTO ? 1 : 0;
    c->tuning.msd_min_rows = msd_min_rows;
    return VDF_OK;
}

vdf_status vdf_ctx_set_local_sort_variant(vdf_ctx* c, int variant) {
    if (!c) return VDF_ERR_INVALID_ARG;
    if (variant < 0 || variant > 3) return fail(c, VDF_ERR_INVALID_ARG, "bad local sort variant %d", variant);
    std::lock_guard<std::mutex> lk(c->mu);
    c->tuning.msd_match = variant;
    return VDF_OK;
}

int vdf_ctx_get_local_sort_variant(vdf_ctx* c) {
    if (!c) return -1;
    std::lock_guard<std::mutex> lk(c->mu);
    return c->tuning.msd_match;
}

vdf_status vdf_ctx_set_test_hooks(vdf_ctx* c, uint32_t spin_limit, uint32_t stall_tile, uint32_t fail_allocs) {
    if (!c) return VDF_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> lk(c->mu);
    c->tuning.spin_limit = spin_limit;
    c->tuning.stall_tile = stall_tile;
    c->fail_allocs = fail_allocs;
    return VDF_OK;
}

vdf_status vdf_ctx_sort_stats(vdf_ctx* c, void* stream, uint64_t* msd_sorts, uint64_t* msd_fallbacks) {
    if (!c) return VDF_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> lk(c->mu);
    DeviceGuard g(c->device);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    cudaError_t e = cudaMemcpyAsync(&c->host_pinned[3], fallback_word(c), sizeof(uint32_t), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return from_cuda(c, e, "read sort statistics");
    if (msd_sorts) *msd_sorts = c->msd_sorts;
    if (msd_fallbacks) *msd_fallbacks = (uint32_t)c->host_pinned[3];
    return VDF_OK;
}

vdf_status vdf_ctx_get_sort_strategy(vdf_ctx* c, int32_t* strategy, uint64_t* msd_min_rows) {
    if (!c) return VDF_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> lk(c->mu);
    if (strategy) *strategy = c->tuning.msd == 2 ? VDF_SORT_MSD : (c->tuning.msd ? VDF_SORT_AUTO : VDF_SORT_LSD);
    if (msd_min_rows) *msd_min_rows = c->tuning.msd_min_rows;
    return VDF_OK;
}

vdf_status vdf_sort_plan_info(uint64_t n, const int32_t* key_dtypes, int nkeys, int strategy, uint64_t msd_min_rows,
                              int32_t* msd_passes, uint32_t* chunks) {
    if (!key_dtypes || nkeys < 1 || nkeys > vdf::kMaxKeys) return VDF_ERR_INVALID_ARG;
    for (int k = 0; k < nkeys; ++k)
        if (!valid_dtype(key_dtypes[k])) return VDF_ERR_INVALID_ARG;
    vdf::SortTuning t = vdf::default_sort_tuning();
    if (strategy != VDF_SORT_AUTO && strategy != VDF_SORT_LSD && strategy != VDF_SORT_MSD) return VDF_ERR_INVALID_ARG;
    t.msd = msd_mode_of(strategy);
    t.dict = strategy == VDF_SORT_AUTO ? 1 : 0;
    t.msd_min_rows = msd_min_rows;
    const vdf::SortPlan p = vdf::make_sort_plan(n, key_dtypes, nkeys, t);
    if (msd_passes) *msd_passes = p.msd ? p.msd_passes : 0;
    if (chunks) *chunks = p.msd ? p.msd_chunks : 0;
    return VDF_OK;
}

int vdf_sort_plan_tries_dict(uint64_t n, const int32_t* key_dtypes, int nkeys, int strategy, uint64_t min_rows) {
    if (!key_dtypes || nkeys < 1 || nkeys > vdf::kMaxKeys) return -1;
    for (int k = 0; k < nkeys; ++k)
        if (!valid_dtype(key_dtypes[k])) return -1;
    if (strategy != VDF_SORT_AUTO && strategy != VDF_SORT_LSD && strategy != VDF_SORT_MSD) return -1;
    vdf::SortTuning t = vdf::default_sort_tuning();
    t.msd = msd_mode_of(strategy);
    t.dict = strategy == VDF_SORT_AUTO ? 1 : 0;
    t.msd_min_rows = min_rows;
    return vdf::make_sort_plan(n, key_dtypes, nkeys, t).dict ? 1 : 0;
}

vdf_status vdf_ctx_dict_stats(vdf_ctx* c, void* stream, uint64_t* tried, uint64_t* taken) {
    if (!c) return VDF_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> lk(c->mu);
    DeviceGuard g(c->device);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    cudaError_t e = cudaMemcpyAsync(&c->host_pinned[5], dict_word(c), sizeof(uint32_t), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return from_cuda(c, e, "read sort statistics");
    if (tried) *tried = c->dict_sorts;
    if (taken) *taken = (uint32_t)c->host_pinned[5];
    return VDF_OK;
}

size_t vdf_groupby_workspace_bytes(uint64_t n, int nvals) {
    if (nvals < 0 || nvals > vdf::kMaxVals) return 0;
    return vdf::segreduce_workspace_bytes(n, nvals);
}

vdf_status vdf_ctx_create(int device, vdf_ctx** out) {
    if (!out) return VDF_ERR_INVALID_ARG;
    *out = nullptr;
    int count = 0;
    cudaError_t e = cudaGetDeviceCount(&count);
    if (e != cudaSuccess || count == 0) {
        cudaGetLastError();
        return VDF_ERR_DEVICE;
    }
    if (device < 0 || device >= count || device >= 64) return VDF_ERR_INVALID_ARG;
    vdf_ctx* c = new vdf_ctx();
    c->device = device;
    DeviceGuard g(device);
    {
        std::lock_guard<std::mutex> lk(g_prep_mu);
        if (!g_prepared[device]) {
            e = vdf::prepare_sort_kernels();
            if (e == cudaSuccess) e = vdf::prepare_segreduce_kernels();
            if (e == cudaSuccess) e = vdf::prepare_batch_kernels();
            if (e != cudaSuccess) {
                delete c;
                return VDF_ERR_DEVICE;
            }
            g_prepared[device] = true;
        }
    }
    if (cudaMalloc(&c->dev_small, 256) != cudaSuccess || cudaMemset(c->dev_small, 0, 256) != cudaSuccess ||
        cudaMallocHost(&c->host_pinned, 8 * sizeof(uint64_t)) != cudaSuccess) {
        cudaGetLastError();
        if (c->dev_small) cudaFree(c->dev_small);
        delete c;
        return VDF_ERR_OOM;
    }
    *out = c;
    return VDF_OK;
}

vdf_status vdf_ctx_destroy(vdf_ctx* c) {
    if (!c) return VDF_ERR_INVALID_ARG;
    {
        std::lock_guard<std::mutex> lk(c->mu);
        DeviceGuard g(c->device);
        c->prof.resolve();
        if (c->ws) cudaFree(c->ws);
        if (c->io) cudaFree(c->io);
        if (c->dev_small) cudaFree(c->dev_small);
        if (c->host_pinned) cudaFreeHost(c->host_pinned);
    }
    delete c;
    return VDF_OK;
}

const char* vdf_ctx_last_error(const vdf_ctx* c) { return c ? c->last_error.c_str() : "null context"; }

uint64_t vdf_ctx_kernel_launches(const vdf_ctx* c) { return c ? c->launches.load() : 0; }

vdf_status vdf_ctx_profile(vdf_ctx* c, int enable) {
    if (!c) return VDF_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> lk(c->mu);
    c->profiling = enable != 0;
    return VDF_OK;
}

vdf_status vdf_ctx_profile_read(vdf_ctx* c, int cls, double* total_ms, uint64_t* launches) {
    if (!c || cls < 0 || cls >= vdf::KC_COUNT) return VDF_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> lk(c->mu);
    DeviceGuard g(c->device);
    cudaError_t e = c->prof.resolve();
    if (e != cudaSuccess) return from_cuda(c, e, "profile events");
    if (total_ms) *total_ms = c->prof.total_ms[cls];
    if (launches) *launches = c->prof.count[cls];
    return VDF_OK;
}

vdf_status vdf_ctx_profile_reset(vdf_ctx* c) {
    if (!c) return VDF_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> lk(c->mu);
    DeviceGuard g(c->device);
    cudaError_t e = c->prof.resolve();
    for (int k = 0; k < vdf::KC_COUNT; ++k) {
        c->prof.total_ms[k] = 0;
        c->prof.count[k] = 0;
    }
    return from_cuda(c, e, "profile events");
}

vdf_status vdf_ctx_reserve(vdf_ctx* c, size_t bytes) {
    if (!c) return VDF_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> lk(c->mu);
    DeviceGuard g(c->device);
    return ws_ensure(c, bytes);
}

vdf_status vdf_ctx_check(vdf_ctx* c, void* stream) {
    if (!c) return VDF_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> lk(c->mu);
    DeviceGuard g(c->device);
    return drain_and_check(c, static_cast<cudaStream_t>(stream));
}

vdf_status vdf_sort_argsort_ws(vdf_ctx* c, uint64_t n, const vdf_col* keys, int nkeys, int order,
                               uint32_t* perm_out, void* const* sorted_keys_out, void* workspace,
                               size_t workspace_bytes, void* stream) {
    if (!c) return VDF_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> lk(c->mu);
    vdf_status st;
    if ((st = check_rows(c, n)) != VDF_OK) return st;
    if ((st = check_keys(c, n, keys, nkeys)) != VDF_OK) return st;
    if (order < VDF_ORDER_ASC || order > VDF_ORDER_DESC_REVERSE) return fail(c, VDF_ERR_INVALID_ARG, "bad order %d", order);
    if (n == 0) return VDF_OK;
    if (!perm_out) return fail(c, VDF_ERR_INVALID_ARG, "perm_out is NULL");
    if (!workspace) return fail(c, VDF_ERR_INVALID_ARG, "workspace is NULL");
    DeviceGuard g(c->device);
    return sort_impl(c, n, keys, nkeys, order, perm_out, sorted_keys_out, static_cast<unsigned char*>(workspace),
                     workspace_bytes, static_cast<cudaStream_t>(stream));
}

vdf_status vdf_sort_argsort(vdf_ctx* c, uint64_t n, const vdf_col* keys, int nkeys, int order, uint32_t* perm_out,
                            void* const* sorted_keys_out, void* stream) {
    if (!c) return VDF_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> lk(c->mu);
    vdf_status st;
    if ((st = check_rows(c, n)) != VDF_OK) return st;
    if ((st = check_keys(c, n, keys, nkeys)) != VDF_OK) return st;
    if (order < VDF_ORDER_ASC || order > VDF_ORDER_DESC_REVERSE) return fail(c, VDF_ERR_INVALID_ARG, "bad order %d", order);
    if (n == 0) return VDF_OK;
    if (!perm_out) return fail(c, VDF_ERR_INVALID_ARG, "perm_out is NULL");
    DeviceGuard g(c->device);
    int32_t dts[vdf::kMaxKeys];
    for (int k = 0; k < nkeys; ++k) dts[k] = keys[k].dtype;
    const size_t need = std::max(sort_ws_need(vdf::make_sort_plan(n, dts, nkeys, c->tuning), n, nkeys, sorted_keys_out),
                                 primary_first_need(c, n, dts, nkeys, sorted_keys_out));
    if ((st = ws_ensure(c, need)) != VDF_OK) return st;
    return sort_impl(c, n, keys, nkeys, order, perm_out, sorted_keys_out, c->ws, c->ws_cap,
                     static_cast<cudaStream_t>(stream));
}

vdf_status vdf_gather(vdf_ctx* c, uint64_t n, const uint32_t* perm, const vdf_col* in, int ncols, void* const* out,
                      void* stream) {
    if (!c) return VDF_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> lk(c->mu);
    vdf_status st;
    if ((st = check_rows(c, n)) != VDF_OK) return st;
    if (ncols < 0 || ncols > vdf::kMaxGather) return fail(c, VDF_ERR_INVALID_ARG, "ncols must be 0..%d", vdf::kMaxGather);
    if (n == 0 || ncols == 0) return VDF_OK;
    if (!perm || !in || !out) return fail(c, VDF_ERR_INVALID_ARG, "NULL perm, in or out");
    vdf::GatherArgs g{};
    g.perm = perm;
    g.err = err_word(c);
    g.n = n;
    g.ncols = ncols;
    for (int i = 0; i < ncols; ++i) {
        if (!valid_dtype(in[i].dtype) || !in[i].data || !out[i])
            return fail(c, VDF_ERR_INVALID_ARG, "column %d: bad dtype or NULL pointer", i);
        g.src[i] = in[i].data;
        g.dst[i] = out[i];
        g.width[i] = vdf::dtype_width(in[i].dtype);
    }
    DeviceGuard gd(c->device);
    const size_t rec = vdf::gather_record_bytes(ncols);
    if (rec && (st = ws_ensure(c, n * rec)) != VDF_OK) return st;
    int launched = 0;
    cudaError_t e = vdf::run_gather(g, static_cast<cudaStream_t>(stream), prof_of(c), rec ? c->ws : nullptr,
                                    rec ? c->ws_cap : 0, &launched);
    c->launches += launched;
    return from_cuda(c, e, "gather");
}

vdf_status vdf_groupby_sorted(vdf_ctx* c, uint64_t n, const vdf_col* keys, int nkeys, const vdf_col* vals, int nvals,
                              void* const* group_keys_out, int64_t* count_out, const vdf_agg_out* aggs,
                              uint32_t* group_start_out, uint32_t* row_group_out, uint64_t* n_groups_dev,
                              uint64_t* n_groups_host, void* stream) {
    if (!c) return VDF_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> lk(c->mu);
    vdf_status st;
    if ((st = check_rows(c, n)) != VDF_OK) return st;
    if ((st = check_keys(c, n, keys, nkeys)) != VDF_OK) return st;
    if (nvals < 0 || nvals > vdf::kMaxVals) return fail(c, VDF_ERR_INVALID_ARG, "nvals must be 0..%d", vdf::kMaxVals);
    if (nvals && (!vals || !aggs)) return fail(c, VDF_ERR_INVALID_ARG, "vals/aggs NULL with nvals > 0");
    for (int v = 0; v < nvals; ++v)
        if (!valid_dtype(vals[v].dtype) || (n && !vals[v].data))
            return fail(c, VDF_ERR_INVALID_ARG, "value %d: bad dtype or NULL data", v);
    DeviceGuard g(c->device);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    vdf::SegArgs a{};
    a.n = n;
    a.striped_min_heads = c->emit_min_heads;
    a.nkeys = nkeys;
    a.nvals = nvals;
    for (int k = 0; k < nkeys; ++k) {
        a.key[k] = vdf::SegCol{keys[k].data, keys[k].dtype};
        a.key_out[k] = group_keys_out ? group_keys_out[k] : nullptr;
    }
    for (int v = 0; v < nvals; ++v) {
        a.val[v] = vdf::SegCol{vals[v].data, vals[v].dtype};
        a.agg[v] = vdf::SegAggOut{aggs[v].sum, aggs[v].sum_hi, aggs[v].min, aggs[v].max, aggs[v].mean};
    }
    a.count_out = count_out;
    a.group_start = group_start_out;
    a.row_group = row_group_out;
    a.n_groups = n_groups_dev ? n_groups_dev : (n_groups_host ? count_word(c) : nullptr);
    a.err = err_word(c);
    if (n && (st = ws_ensure(c, vdf::segreduce_workspace_bytes(n, nvals))) != VDF_OK) return st;
    int launched = 0;
    cudaError_t e = vdf::run_segreduce(a, c->ws, s, prof_of(c), &launched);
    c->launches += launched;
    if (e != cudaSuccess) return from_cuda(c, e, "segmented reduction");
    return finish_groups(c, a.n_groups, n_groups_host, s);
}

}  // extern "C"

namespace {

// vdf_sort_groupby with the context lock already held.
vdf_status sort_groupby_locked(vdf_ctx* c, const vdf_sort_groupby_args* x, cudaStream_t stream) {
    vdf_status st;
    const uint64_t n = x->n;
    if ((st = check_rows(c, n)) != VDF_OK) return st;
    if ((st = check_keys(c, n, x->keys, x->nkeys)) != VDF_OK) return st;
    if (x->order < VDF_ORDER_ASC || x->order > VDF_ORDER_DESC_REVERSE)
        return fail(c, VDF_ERR_INVALID_ARG, "bad order %d", x->order);
    if (x->npayload < 0 || x->npayload > vdf::kMaxGather)
        return fail(c, VDF_ERR_INVALID_ARG, "npayload must be 0..%d", vdf::kMaxGather);
    if (x->npayload && !x->payload) return fail(c, VDF_ERR_INVALID_ARG, "payload is NULL");
    for (int p = 0; p < x->npayload; ++p)
        if (!valid_dtype(x->payload[p].dtype) || (n && !x->payload[p].data))
            return fail(c, VDF_ERR_INVALID_ARG, "payload %d: bad dtype or NULL data", p);
    if (x->groupby) {
        if (x->nagg < 0 || x->nagg > vdf::kMaxVals) return fail(c, VDF_ERR_INVALID_ARG, "nagg must be 0..%d", vdf::kMaxVals);
        if (x->nagg && (!x->agg_cols || !x->aggs)) return fail(c, VDF_ERR_INVALID_ARG, "agg_cols/aggs NULL");
        for (int i = 0; i < x->nagg; ++i)
            if (x->agg_cols[i] < 0 || x->agg_cols[i] >= x->npayload)
                return fail(c, VDF_ERR_INVALID_ARG, "agg_cols[%d]=%d out of range", i, x->agg_cols[i]);
    }
    DeviceGuard g(c->device);
    cudaStream_t s = stream;
    if (n == 0) {
        if (x->groupby && x->n_groups_dev) cudaMemsetAsync(x->n_groups_dev, 0, sizeof(uint64_t), s);
        if (x->groupby && x->n_groups_host) *x->n_groups_host = 0;
        return VDF_OK;
    }

    int32_t dts[vdf::kMaxKeys];
    const void* cols[vdf::kMaxKeys];
    for (int k = 0; k < x->nkeys; ++k) {
        dts[k] = x->keys[k].dtype;
        cols[k] = x->keys[k].data;
    }
    const vdf::SortPlan plan = vdf::make_sort_plan(n, dts, x->nkeys, c->tuning);
    // Sorted copies needed by the group-by that the caller did not ask for
    // live in the workspace: [perm][key 0][keys 1..][aggregated payload][tail]
    // where tail = max(sort workspace, group-by workspace).
    const bool own_perm = (x->perm_out == nullptr);
    const size_t perm_bytes = own_perm ? align256(n * 4) : 0;
    void* skey[vdf::kMaxKeys] = {};
    void* spay[vdf::kMaxGather] = {};
    size_t off = perm_bytes;
    size_t key_off[vdf::kMaxKeys] = {}, pay_off[vdf::kMaxGather] = {};
    bool key_own[vdf::kMaxKeys] = {}, pay_own[vdf::kMaxGather] = {};
    for (int k = 0; k < x->nkeys; ++k) {
        skey[k] = x->sorted_keys_out ? x->sorted_keys_out[k] : nullptr;
        if (!skey[k] && x->groupby) {
            key_own[k] = true;
            key_off[k] = off;
            off += align256(n * (size_t)vdf::dtype_width(x->keys[k].dtype));
        }
    }
    bool aggregated[vdf::kMaxGather] = {};
    if (x->groupby)
        for (int i = 0; i < x->nagg; ++i) aggregated[x->agg_cols[i]] = true;
    for (int p = 0; p < x->npayload; ++p) {
        spay[p] = x->payload_out ? x->payload_out[p] : nullptr;
        if (!spay[p] && aggregated[p]) {
            pay_own[p] = true;
            pay_off[p] = off;
            off += align256(n * (size_t)vdf::dtype_width(x->payload[p].dtype));
        }
    }
    // columns the gather will produce: requested outputs and the sorted
    // copies the group-by needs (owned buffers, assigned below)
    int ngather = 0;
    for (int k = 1; k < x->nkeys; ++k) ngather += (skey[k] || key_own[k]) ? 1 : 0;
    for (int p = 0; p < x->npayload; ++p) ngather += (spay[p] || pay_own[p]) ? 1 : 0;
    const size_t rec_bytes = (size_t)n * vdf::gather_record_bytes(std::min(ngather, vdf::kMaxGather));
    const size_t seg_bytes = x->groupby ? vdf::segreduce_workspace_bytes(n, x->nagg) : 0;
    size_t tail = std::max(std::max(plan.ws_bytes, seg_bytes), rec_bytes);
    if (x->nkeys >= 2 && c->multikey_mode == VDF_MULTIKEY_PRIMARY_FIRST && !skey[0] && !plan.msd) {
        // room for the primary key's sorted copy next to its sort's workspace
        const vdf::SortPlan p0 = vdf::make_sort_plan(n, dts, 1, c->tuning);
        tail = std::max(tail, align256(p0.ws_bytes) + (size_t)n * vdf::dtype_width(dts[0]));
    }
    if ((st = ws_ensure(c, off + tail)) != VDF_OK) return st;
    uint32_t* perm = own_perm ? reinterpret_cast<uint32_t*>(c->ws) : x->perm_out;
    for (int k = 0; k < x->nkeys; ++k)
        if (key_own[k]) skey[k] = c->ws + key_off[k];
    for (int p = 0; p < x->npayload; ++p)
        if (pay_own[p]) spay[p] = c->ws + pay_off[p];
    unsigned char* tws = c->ws + off;

    // the columns the gather produces, in record order
    struct GCol { const void* src; void* dst; int dtype; };
    std::vector<GCol> gcols;
    for (int k = 1; k < x->nkeys; ++k)
        if (skey[k]) gcols.push_back({x->keys[k].data, skey[k], x->keys[k].dtype});
    for (int p = 0; p < x->npayload; ++p)
        if (spay[p]) gcols.push_back({x->payload[p].data, spay[p], x->payload[p].dtype});
    bool done = false;
    if ((st = primary_first(c, n, dts, cols, x->nkeys, x->order, perm, skey[0], tws, c->ws_cap - off, s, x->perm_in,
                            &done)) != VDF_OK)
        return st;
    cudaError_t e = cudaSuccess;
    if (!done) {
        e = ctx_run_sort(c, plan, cols, x->order, perm, skey[0], tws, s, x->perm_in);
        if (e != cudaSuccess) return from_cuda(c, e, "radix sort");
    }

    // Gather the other key columns and the payload into sorted order, up to
    // kMaxGather columns per launch (the permutation is read once per launch).
    vdf::GatherArgs ga{};
    ga.perm = perm;
    ga.err = err_word(c);
    ga.n = n;
    auto flush = [&]() -> cudaError_t {
        if (!ga.ncols) return cudaSuccess;
        int launched = 0;
        cudaError_t ge = vdf::run_gather(ga, s, prof_of(c), tws, c->ws_cap - off, &launched);
        c->launches += launched;
        ga.ncols = 0;
        return ge;
    };
    auto add = [&](const void* src, void* dst, int dtype) -> cudaError_t {
        ga.src[ga.ncols] = src;
        ga.dst[ga.ncols] = dst;
        ga.width[ga.ncols] = vdf::dtype_width(dtype);
        if (++ga.ncols == vdf::kMaxGather) return flush();
        return cudaSuccess;
    };
    for (const GCol& gc : gcols)
        if ((e = add(gc.src, gc.dst, gc.dtype)) != cudaSuccess) return from_cuda(c, e, "gather");
    if ((e = flush()) != cudaSuccess) return from_cuda(c, e, "gather");
    if (!x->groupby) return VDF_OK;

    vdf::SegArgs a{};
    a.n = n;
    a.striped_min_heads = c->emit_min_heads;
    a.nkeys = x->nkeys;
    a.nvals = x->nagg;
    for (int k = 0; k < x->nkeys; ++k) {
        a.key[k] = vdf::SegCol{skey[k], x->keys[k].dtype};
        a.key_out[k] = x->group_keys_out ? x->group_keys_out[k] : nullptr;
    }
    for (int i = 0; i < x->nagg; ++i) {
        const int p = x->agg_cols[i];
        a.val[i] = vdf::SegCol{spay[p], x->payload[p].dtype};
        const vdf_agg_out& o = x->aggs[i];
        a.agg[i] = vdf::SegAggOut{o.sum, o.sum_hi, o.min, o.max, o.mean};
    }
    a.count_out = x->group_count_out;
    a.group_start = x->group_start_out;
    a.row_group = x->row_group_out;
    a.n_groups = x->n_groups_dev ? x->n_groups_dev : (x->n_groups_host ? count_word(c) : nullptr);
    a.err = err_word(c);
    int launched = 0;
    e = vdf::run_segreduce(a, tws, s, prof_of(c), &launched);
    c->launches += launched;
    if (e != cudaSuccess) return from_cuda(c, e, "segmented reduction");
    return finish_groups(c, a.n_groups, x->n_groups_host, s);
}

// Device copy of a host vdf_sort_groupby_args: every input is staged into the
// context's I/O buffer and every requested output gets a device slot there.
struct HostStage {
    vdf_col keys[vdf::kMaxKeys];
    vdf_col pay[vdf::kMaxGather];
    void* skeys[vdf::kMaxKeys];
    void* spay[vdf::kMaxGather];
    void* gkeys[vdf::kMaxKeys];
    vdf_agg_out aggs[vdf::kMaxVals];
    vdf_sort_groupby_args d;
};


}  // namespace

vdf_status vdfc::sort_groupby_device(vdf_ctx* c, const vdf_sort_groupby_args* x, cudaStream_t s) {
    return sort_groupby_locked(c, x, s);
}

extern "C" {

vdf_status vdf_sort_groupby(vdf_ctx* c, const vdf_sort_groupby_args* x, void* stream) {
    if (!c || !x) return VDF_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> lk(c->mu);
    return sort_groupby_locked(c, x, static_cast<cudaStream_t>(stream));
}

vdf_status vdf_sort_groupby_host(vdf_ctx* c, const vdf_sort_groupby_args* x, void* stream) {
    if (!c || !x) return VDF_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> lk(c->mu);
    vdf_status st;
    const uint64_t n = x->n;
    if ((st = check_rows(c, n)) != VDF_OK) return st;
    if ((st = check_keys(c, n, x->keys, x->nkeys)) != VDF_OK) return st;
    if (x->npayload < 0 || x->npayload > vdf::kMaxGather || (x->npayload && !x->payload))
        return fail(c, VDF_ERR_INVALID_ARG, "bad payload columns");
    for (int p = 0; p < x->npayload; ++p)
        if (!valid_dtype(x->payload[p].dtype)) return fail(c, VDF_ERR_INVALID_ARG, "payload %d: bad dtype", p);
    if (x->groupby && (x->nagg < 0 || x->nagg > vdf::kMaxVals || (x->nagg && (!x->agg_cols || !x->aggs))))
        return fail(c, VDF_ERR_INVALID_ARG, "bad aggregation list");
    for (int i = 0; x->groupby && i < x->nagg; ++i)
        if (x->agg_cols[i] < 0 || x->agg_cols[i] >= x->npayload)
            return fail(c, VDF_ERR_INVALID_ARG, "agg_cols[%d] out of range", i);
    DeviceGuard g(c->device);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (n == 0) {
        if (x->groupby && x->n_groups_host) *x->n_groups_host = 0;
        return VDF_OK;
    }
    auto kw = [&](int k) { return (size_t)vdf::dtype_width(x->keys[k].dtype); };
    auto pw = [&](int p) { return (size_t)vdf::dtype_width(x->payload[p].dtype); };
    // layout of the staging buffer
    size_t off = 0;
    auto take = [&](size_t bytes) { size_t o = off; off = align256(off + bytes); return o; };
    size_t o_keys[vdf::kMaxKeys], o_pay[vdf::kMaxGather], o_sk[vdf::kMaxKeys], o_sp[vdf::kMaxGather];
    size_t o_gk[vdf::kMaxKeys], o_agg[vdf::kMaxVals][5], o_perm = 0, o_cnt = 0, o_gs = 0, o_rg = 0, o_ng = 0;
    for (int k = 0; k < x->nkeys; ++k) o_keys[k] = take(n * kw(k));
    for (int p = 0; p < x->npayload; ++p) o_pay[p] = take(n * pw(p));
    const size_t o_pin = x->perm_in ? take(n * 4) : 0;
    if (x->perm_out) o_perm = take(n * 4);
    for (int k = 0; k < x->nkeys; ++k) o_sk[k] = (x->sorted_keys_out && x->sorted_keys_out[k]) ? take(n * kw(k)) : 0;
    for (int p = 0; p < x->npayload; ++p) o_sp[p] = (x->payload_out && x->payload_out[p]) ? take(n * pw(p)) : 0;
    if (x->groupby) {
        for (int k = 0; k < x->nkeys; ++k) o_gk[k] = (x->group_keys_out && x->group_keys_out[k]) ? take(n * kw(k)) : 0;
        if (x->group_count_out) o_cnt = take(n * 8);
        for (int i = 0; i < x->nagg; ++i) {
            const vdf_agg_out& a = x->aggs[i];
            const size_t w = pw(x->agg_cols[i]);
            o_agg[i][0] = a.sum ? take(n * 8) : 0;
            o_agg[i][1] = a.sum_hi ? take(n * 8) : 0;
            o_agg[i][2] = a.min ? take(n * w) : 0;
            o_agg[i][3] = a.max ? take(n * w) : 0;
            o_agg[i][4] = a.mean ? take(n * 8) : 0;
        }
        if (x->group_start_out) o_gs = take(n * 4);
        if (x->row_group_out) o_rg = take(n * 4);
        o_ng = take(8);
    }
    if ((st = io_ensure(c, off)) != VDF_OK) return st;
    unsigned char* io = c->io;
    auto at = [&](size_t o) -> void* { return io + o; };
    cudaError_t e = cudaSuccess;
    for (int k = 0; k < x->nkeys && e == cudaSuccess; ++k)
        e = cudaMemcpyAsync(at(o_keys[k]), x->keys[k].data, n * kw(k), cudaMemcpyHostToDevice, s);
    for (int p = 0; p < x->npayload && e == cudaSuccess; ++p)
        e = cudaMemcpyAsync(at(o_pay[p]), x->payload[p].data, n * pw(p), cudaMemcpyHostToDevice, s);
    if (x->perm_in && e == cudaSuccess) e = cudaMemcpyAsync(at(o_pin), x->perm_in, n * 4, cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) return from_cuda(c, e, "copy inputs to the device");
    HostStage h{};
    vdf_sort_groupby_args& d = h.d;
    d = *x;
    for (int k = 0; k < x->nkeys; ++k) {
        h.keys[k] = vdf_col{at(o_keys[k]), x->keys[k].dtype};
        h.skeys[k] = o_sk[k] ? at(o_sk[k]) : nullptr;
        h.gkeys[k] = (x->groupby && o_gk[k]) ? at(o_gk[k]) : nullptr;
    }
    for (int p = 0; p < x->npayload; ++p) {
        h.pay[p] = vdf_col{at(o_pay[p]), x->payload[p].dtype};
        h.spay[p] = o_sp[p] ? at(o_sp[p]) : nullptr;
    }
    d.keys = h.keys;
    d.payload = h.pay;
    d.perm_in = x->perm_in ? static_cast<const uint32_t*>(at(o_pin)) : nullptr;
    d.perm_out = x->perm_out ? static_cast<uint32_t*>(at(o_perm)) : nullptr;
    d.sorted_keys_out = x->sorted_keys_out ? h.skeys : nullptr;
    d.payload_out = x->payload_out ? h.spay : nullptr;
    uint64_t groups = 0;
    if (x->groupby) {
        for (int i = 0; i < x->nagg; ++i)
            h.aggs[i] = vdf_agg_out{o_agg[i][0] ? at(o_agg[i][0]) : nullptr,
                                    o_agg[i][1] ? static_cast<int64_t*>(at(o_agg[i][1])) : nullptr,
                                    o_agg[i][2] ? at(o_agg[i][2]) : nullptr, o_agg[i][3] ? at(o_agg[i][3]) : nullptr,
                                    o_agg[i][4] ? static_cast<double*>(at(o_agg[i][4])) : nullptr};
        d.aggs = h.aggs;
        d.group_keys_out = x->group_keys_out ? h.gkeys : nullptr;
        d.group_count_out = o_cnt ? static_cast<int64_t*>(at(o_cnt)) : nullptr;
        d.group_start_out = o_gs ? static_cast<uint32_t*>(at(o_gs)) : nullptr;
        d.row_group_out = o_rg ? static_cast<uint32_t*>(at(o_rg)) : nullptr;
        d.n_groups_dev = static_cast<uint64_t*>(at(o_ng));
        d.n_groups_host = &groups;  // synchronises once the group count is known
    }
    if ((st = sort_groupby_locked(c, &d, s)) != VDF_OK) return st;
    // results back to the host: rows (n) for the sorted frame, groups (G) for the group table
    auto down = [&](void* dst, size_t o, size_t bytes) {
        if (e == cudaSuccess && dst && bytes) e = cudaMemcpyAsync(dst, at(o), bytes, cudaMemcpyDeviceToHost, s);
    };
    down(x->perm_out, o_perm, n * 4);
    for (int k = 0; k < x->nkeys; ++k)
        if (o_sk[k]) down(x->sorted_keys_out[k], o_sk[k], n * kw(k));
    for (int p = 0; p < x->npayload; ++p)
        if (o_sp[p]) down(x->payload_out[p], o_sp[p], n * pw(p));
    if (x->groupby) {
        for (int k = 0; k < x->nkeys; ++k)
            if (o_gk[k]) down(x->group_keys_out[k], o_gk[k], groups * kw(k));
        if (o_cnt) down(x->group_count_out, o_cnt, groups * 8);
        for (int i = 0; i < x->nagg; ++i) {
            const vdf_agg_out& a = x->aggs[i];
            const size_t w = pw(x->agg_cols[i]);
            if (o_agg[i][0]) down(a.sum, o_agg[i][0], groups * 8);
            if (o_agg[i][1]) down(a.sum_hi, o_agg[i][1], groups * 8);
            if (o_agg[i][2]) down(a.min, o_agg[i][2], groups * w);
            if (o_agg[i][3]) down(a.max, o_agg[i][3], groups * w);
            if (o_agg[i][4]) down(a.mean, o_agg[i][4], groups * 8);
        }
        if (o_gs) down(x->group_start_out, o_gs, groups * 4);
        if (o_rg) down(x->row_group_out, o_rg, n * 4);
        if (x->n_groups_host) *x->n_groups_host = groups;
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return from_cuda(c, e, "copy results to the host");
    return VDF_OK;
}

vdf_status vdf_gather_host(vdf_ctx* c, uint64_t n, const uint32_t* perm, const vdf_col* in, int ncols,
                           void* const* out, void* stream) {
    if (!c) return VDF_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> lk(c->mu);
    vdf_status st;
    if ((st = check_rows(c, n)) != VDF_OK) return st;
    if (ncols < 0 || ncols > vdf::kMaxGather) return fail(c, VDF_ERR_INVALID_ARG, "ncols must be 0..%d", vdf::kMaxGather);
    if (n == 0 || ncols == 0) return VDF_OK;
    if (!perm || !in || !out) return fail(c, VDF_ERR_INVALID_ARG, "NULL perm, in or out");
    for (int i = 0; i < ncols; ++i)
        if (!valid_dtype(in[i].dtype) || !in[i].data || !out[i])
            return fail(c, VDF_ERR_INVALID_ARG, "column %d: bad dtype or NULL pointer", i);
    DeviceGuard g(c->device);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    size_t off = align256(n * 4);
    size_t o_in[vdf::kMaxGather], o_out[vdf::kMaxGather];
    for (int i = 0; i < ncols; ++i) {
        o_in[i] = off;
        off = align256(off + n * vdf::dtype_width(in[i].dtype));
        o_out[i] = off;
        off = align256(off + n * vdf::dtype_width(in[i].dtype));
    }
    if ((st = io_ensure(c, off)) != VDF_OK) return st;
    const size_t rec = vdf::gather_record_bytes(ncols);
    if (rec && (st = ws_ensure(c, n * rec)) != VDF_OK) return st;
    cudaError_t e = cudaMemcpyAsync(c->io, perm, n * 4, cudaMemcpyHostToDevice, s);
    vdf::GatherArgs ga{};
    ga.perm = reinterpret_cast<const uint32_t*>(c->io);
    ga.err = err_word(c);
    ga.n = n;
    ga.ncols = ncols;
    for (int i = 0; i < ncols && e == cudaSuccess; ++i) {
        const size_t w = (size_t)vdf::dtype_width(in[i].dtype);
        e = cudaMemcpyAsync(c->io + o_in[i], in[i].data, n * w, cudaMemcpyHostToDevice, s);
        ga.src[i] = c->io + o_in[i];
        ga.dst[i] = c->io + o_out[i];
        ga.width[i] = (int)w;
    }
    if (e != cudaSuccess) return from_cuda(c, e, "copy inputs to the device");
    int launched = 0;
    e = vdf::run_gather(ga, s, prof_of(c), rec ? c->ws : nullptr, rec ? c->ws_cap : 0, &launched);
    c->launches += launched;
    for (int i = 0; i < ncols && e == cudaSuccess; ++i)
        e = cudaMemcpyAsync(out[i], c->io + o_out[i], n * vdf::dtype_width(in[i].dtype), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return from_cuda(c, e, "gather");
    return drain_and_check(c, s);
}

vdf_status vdf_transform_groupby_host(vdf_ctx* c, uint64_t n, const vdf_col* keys, int nkeys, vdf_col val,
                                      int32_t function, const uint32_t* perm_in, void* out, uint64_t* n_groups_host,
                                      void* stream) {
    if (!c) return VDF_ERR_INVALID_ARG;
    vdf_status st;
    if (function < VDF_AGG_COUNT || function > VDF_AGG_MAX) return fail(c, VDF_ERR_INVALID_ARG, "bad function %d", function);
    if (!valid_dtype(val.dtype)) return fail(c, VDF_ERR_INVALID_ARG, "bad value dtype");
    std::lock_guard<std::mutex> lk(c->mu);
    if ((st = check_rows(c, n)) != VDF_OK) return st;
    if ((st = check_keys(c, n, keys, nkeys)) != VDF_OK) return st;
    if (n == 0) {
        if (n_groups_host) *n_groups_host = 0;
        return VDF_OK;
    }
    if (!out || (function != VDF_AGG_COUNT && !val.data)) return fail(c, VDF_ERR_INVALID_ARG, "NULL value or output");
    DeviceGuard g(c->device);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const bool is_float = (val.dtype == VDF_F64 || val.dtype == VDF_F32);
    const int vw = vdf::dtype_width(val.dtype);
    // output element width: count and sum (integer low word / double) and mean are 8 bytes
    const int ow = (function == VDF_AGG_MIN || function == VDF_AGG_MAX) ? vw : 8;
    (void)is_float;
    size_t off = 0;
    auto take = [&](size_t bytes) { size_t o = off; off = align256(off + bytes); return o; };
    size_t o_keys[vdf::kMaxKeys];
    for (int k = 0; k < nkeys; ++k) o_keys[k] = take(n * vdf::dtype_width(keys[k].dtype));
    const size_t o_val = (function != VDF_AGG_COUNT) ? take(n * vw) : 0;
    const size_t o_pin = perm_in ? take(n * 4) : 0;
    const size_t o_perm = take(n * 4), o_rg = take(n * 4), o_gv = take(n * 8), o_out = take(n * (size_t)ow);
    const size_t o_ng = take(8);
    if ((st = io_ensure(c, off)) != VDF_OK) return st;
    unsigned char* io = c->io;
    cudaError_t e = cudaSuccess;
    vdf_col dkeys[vdf::kMaxKeys];
    for (int k = 0; k < nkeys && e == cudaSuccess; ++k) {
        e = cudaMemcpyAsync(io + o_keys[k], keys[k].data, n * vdf::dtype_width(keys[k].dtype), cudaMemcpyHostToDevice, s);
        dkeys[k] = vdf_col{io + o_keys[k], keys[k].dtype};
    }
    if (o_val && e == cudaSuccess) e = cudaMemcpyAsync(io + o_val, val.data, n * vw, cudaMemcpyHostToDevice, s);
    if (perm_in && e == cudaSuccess) e = cudaMemcpyAsync(io + o_pin, perm_in, n * 4, cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) return from_cuda(c, e, "copy inputs to the device");
    vdf_col dval{o_val ? io + o_val : nullptr, val.dtype};
    vdf_agg_out agg{};
    int32_t agg_col = 0;
    vdf_sort_groupby_args d{};
    d.n = n;
    d.keys = dkeys;
    d.nkeys = nkeys;
    d.order = VDF_ORDER_ASC;
    d.perm_in = o_pin ? reinterpret_cast<const uint32_t*>(io + o_pin) : nullptr;
    d.perm_out = reinterpret_cast<uint32_t*>(io + o_perm);
    d.groupby = 1;
    d.row_group_out = reinterpret_cast<uint32_t*>(io + o_rg);
    void* gv = io + o_gv;
    if (function == VDF_AGG_COUNT) {
        d.group_count_out = static_cast<int64_t*>(gv);
    } else {
        d.payload = &dval;
        d.npayload = 1;
        d.agg_cols = &agg_col;
        d.nagg = 1;
        d.aggs = &agg;
        if (function == VDF_AGG_SUM) agg.sum = gv;
        else if (function == VDF_AGG_MEAN) agg.mean = static_cast<double*>(gv);
        else if (function == VDF_AGG_MIN) agg.min = gv;
        else agg.max = gv;
    }
    uint64_t groups = 0;
    d.n_groups_dev = reinterpret_cast<uint64_t*>(io + o_ng);
    d.n_groups_host = &groups;
    if ((st = sort_groupby_locked(c, &d, s)) != VDF_OK) return st;
    // every row receives its group's value, in the frame's row order
    e = vdf::run_broadcast(d.row_group_out, n, gv, groups, ow, d.perm_out, io + o_out, err_word(c), s, prof_of(c));
    c->launches++;
    if (e == cudaSuccess) e = cudaMemcpyAsync(out, io + o_out, n * (size_t)ow, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return from_cuda(c, e, "transform output");
    if (n_groups_host) *n_groups_host = groups;
    return drain_and_check(c, s);
}

vdf_status vdf_broadcast(vdf_ctx* c, uint64_t n, const uint32_t* row_group, const void* group_vals,
                         uint64_t n_groups, int width, const uint32_t* perm, void* out, void* stream) {
    if (!c) return VDF_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> lk(c->mu);
    vdf_status st;
    if ((st = check_rows(c, n)) != VDF_OK) return st;
    if (width != 4 && width != 8) return fail(c, VDF_ERR_INVALID_ARG, "width must be 4 or 8");
    if (n == 0) return VDF_OK;
    if (!row_group || !group_vals || !out) return fail(c, VDF_ERR_INVALID_ARG, "NULL row_group, group_vals or out");
    DeviceGuard g(c->device);
    c->launches++;
    return from_cuda(c, vdf::run_broadcast(row_group, n, group_vals, n_groups, width, perm, out, err_word(c),
                                           static_cast<cudaStream_t>(stream), prof_of(c)),
                     "broadcast");
}

// Reads a device count (u64) into *host after the stream's work.
static vdf_status read_count(vdf_ctx* c, const uint64_t* dev, uint64_t* host, cudaStream_t s, const char* what) {
    if (!host) return VDF_OK;
    cudaError_t e = cudaMemcpyAsync(&c->host_pinned[0], dev, sizeof(uint64_t), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return from_cuda(c, e, what);
    *host = c->host_pinned[0];
    return drain_and_check(c, s);
}

// vdf_unique with the context lock held
static vdf_status unique_locked(vdf_ctx* c, uint64_t n, vdf_col key, int keep_last, uint8_t* keep_out,
                                uint64_t* n_unique_dev, uint64_t* n_unique_host, void* stream) {
    vdf_status st;
    if ((st = check_rows(c, n)) != VDF_OK) return st;
    if ((st = check_keys(c, n, &key, 1)) != VDF_OK) return st;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    DeviceGuard g(c->device);
    if (n == 0) {
        if (n_unique_dev && cudaMemsetAsync(n_unique_dev, 0, sizeof(uint64_t), s) != cudaSuccess)
            return from_cuda(c, cudaGetLastError(), "clear count");
        if (n_unique_host) *n_unique_host = 0;
        return VDF_OK;
    }
    if (!keep_out) return fail(c, VDF_ERR_INVALID_ARG, "keep_out is NULL");
    const int w = vdf::dtype_width(key.dtype);
    // workspace: permutation | sorted keys | count | mark bits | the sort's own
    const size_t o_perm = 0, o_keys = align256(4 * n), o_cnt = o_keys + align256((size_t)w * n);
    const size_t o_bits = o_cnt + 256, o_sort = o_bits + align256(vdf::unique_workspace_bytes(n));
    const vdf::SortPlan plan = vdf::make_sort_plan(n, &key.dtype, 1, c->tuning);
    if ((st = ws_ensure(c, o_sort + sort_ws_need(plan, n, 1, nullptr))) != VDF_OK) return st;
    uint32_t* perm = reinterpret_cast<uint32_t*>(c->ws + o_perm);
    void* skeys = c->ws + o_keys;
    uint64_t* cnt = n_unique_dev ? n_unique_dev : reinterpret_cast<uint64_t*>(c->ws + o_cnt);
    void* const souts[1] = {skeys};
    if ((st = sort_impl(c, n, &key, 1, VDF_ORDER_ASC, perm, souts, c->ws + o_sort, c->ws_cap - o_sort, s)) != VDF_OK)
        return st;
    cudaError_t e = cudaMemsetAsync(cnt, 0, sizeof(uint64_t), s);
    if (e == cudaSuccess)
        e = vdf::run_unique_mark(skeys, w, perm, n, keep_last ? 1 : 0, keep_out,
                                 reinterpret_cast<unsigned long long*>(cnt), reinterpret_cast<uint32_t*>(c->ws + o_bits),
                                 err_word(c), s);
    c->launches += 2;
    if (e != cudaSuccess) return from_cuda(c, e, "unique");
    return read_count(c, cnt, n_unique_host, s, "read unique count");
}

// vdf_left_join_index with the context lock held
static vdf_status left_join_locked(vdf_ctx* c, uint64_t n_left, vdf_col left_key, uint64_t n_right,
                                   vdf_col right_key, int method, uint32_t* match_out, uint64_t* n_matched_dev,
                                   uint64_t* n_matched_host, void* stream) {
    vdf_status st;
    if ((st = check_rows(c, n_left)) != VDF_OK) return st;
    if ((st = check_rows(c, n_right)) != VDF_OK) return st;
    if ((st = check_keys(c, n_left, &left_key, 1)) != VDF_OK) return st;
    if ((st = check_keys(c, n_right, &right_key, 1)) != VDF_OK) return st;
    if (left_key.dtype != right_key.dtype) return fail(c, VDF_ERR_INVALID_ARG, "left and right keys differ in dtype");
    if (method < VDF_JOIN_FIRST || method > VDF_JOIN_ALIGNED) return fail(c, VDF_ERR_INVALID_ARG, "bad method %d", method);
    if (n_left && !match_out) return fail(c, VDF_ERR_INVALID_ARG, "match_out is NULL");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    DeviceGuard g(c->device);
    const int w = vdf::dtype_width(right_key.dtype);
    const uint64_t nr = n_right, nl = n_left;
    const bool aligned = method == VDF_JOIN_ALIGNED;
    // workspace: right permutation | right sorted keys | distinct keys | run
    // starts | group count | matched count | (aligned: left permutation, left
    // sorted keys, run of each sorted left row, left run starts, left group
    // count) | the sorts', the reductions' or the hash table's own
    const size_t o_perm = 0, o_sk = align256(4 * nr), o_uk = o_sk + align256((size_t)w * nr);
    const size_t o_gs = o_uk + align256((size_t)w * nr), o_ng = o_gs + align256(4 * nr), o_cnt = o_ng + 256;
    size_t o = o_cnt + 256;
    size_t o_lperm = 0, o_lsk = 0, o_lrg = 0, o_lgs = 0, o_lng = 0;
    if (aligned) {
        o_lperm = o; o += align256(4 * nl);
        o_lsk = o; o += align256((size_t)w * nl);
        o_lrg = o; o += align256(4 * nl);
        o_lgs = o; o += align256(4 * nl);
        o_lng = o; o += 256;
    }
    const size_t o_tail = o;
    size_t tail = 0;
    if (nr) {
        const vdf::SortPlan plan = vdf::make_sort_plan(nr, &right_key.dtype, 1, c->tuning);
        tail = std::max(sort_ws_need(plan, nr, 1, nullptr), vdf::segreduce_workspace_bytes(nr, 0));
        tail = std::max(tail, vdf::join_workspace_bytes(nr));
    }
    if (aligned && nl) {
        const vdf::SortPlan plan = vdf::make_sort_plan(nl, &left_key.dtype, 1, c->tuning);
        tail = std::max(tail, std::max(sort_ws_need(plan, nl, 1, nullptr), vdf::segreduce_workspace_bytes(nl, 0)));
    }
    if ((st = ws_ensure(c, o_tail + tail)) != VDF_OK) return st;
    uint64_t* cnt = n_matched_dev ? n_matched_dev : reinterpret_cast<uint64_t*>(c->ws + o_cnt);
    cudaError_t e = cudaMemsetAsync(cnt, 0, sizeof(uint64_t), s);
    if (e != cudaSuccess) return from_cuda(c, e, "clear count");
    if (nl == 0) return read_count(c, cnt, n_matched_host, s, "read match count");
    if (nr == 0) {  // nothing to match
        if ((e = cudaMemsetAsync(match_out, 0xff, 4 * nl, s)) != cudaSuccess) return from_cuda(c, e, "no match");
        return read_count(c, cnt, n_matched_host, s, "read match count");
    }
    // one side: stable sort, then its distinct keys and their run starts
    auto sort_side = [&](uint64_t n, const vdf_col& key, size_t o_p, size_t o_s, size_t o_u, size_t o_g, size_t o_n,
                         size_t o_rg) -> vdf_status {
        void* const souts[1] = {c->ws + o_s};
        vdf_status r = sort_impl(c, n, &key, 1, VDF_ORDER_ASC, reinterpret_cast<uint32_t*>(c->ws + o_p), souts,
                                 c->ws + o_tail, c->ws_cap - o_tail, s);
        if (r != VDF_OK) return r;
        vdf::SegArgs a{};
        a.n = n;
        a.striped_min_heads = c->emit_min_heads;
        a.nkeys = 1;
        a.nvals = 0;
        a.key[0] = vdf::SegCol{c->ws + o_s, key.dtype};
        a.key_out[0] = o_u ? c->ws + o_u : nullptr;
        a.group_start = reinterpret_cast<uint32_t*>(c->ws + o_g);
        a.row_group = o_rg ? reinterpret_cast<uint32_t*>(c->ws + o_rg) : nullptr;
        a.n_groups = reinterpret_cast<uint64_t*>(c->ws + o_n);
        a.err = err_word(c);
        int launched = 0;
        cudaError_t ee = vdf::run_segreduce(a, c->ws + o_tail, s, prof_of(c), &launched);
        c->launches += launched;
        return ee == cudaSuccess ? VDF_OK : from_cuda(c, ee, "distinct keys");
    };
    if ((st = sort_side(nr, right_key, o_perm, o_sk, o_uk, o_gs, o_ng, 0)) != VDF_OK) return st;
    if (aligned && (st = sort_side(nl, left_key, o_lperm, o_lsk, 0, o_lgs, o_lng, o_lrg)) != VDF_OK) return st;
    const uint32_t* perm_r = reinterpret_cast<const uint32_t*>(c->ws + o_perm);
    const uint32_t* gs_r = reinterpret_cast<const uint32_t*>(c->ws + o_gs);
    const uint64_t* ng_r = reinterpret_cast<const uint64_t*>(c->ws + o_ng);
    e = vdf::run_join_build(c->ws + o_uk, w, gs_r, ng_r, perm_r, nr, method, c->ws + o_tail, err_word(c), s);
    if (e == cudaSuccess) {
        if (aligned)
            e = vdf::run_join_probe_aligned(c->ws + o_lsk, w, reinterpret_cast<const uint32_t*>(c->ws + o_lperm),
                                            reinterpret_cast<const uint32_t*>(c->ws + o_lrg),
                                            reinterpret_cast<const uint32_t*>(c->ws + o_lgs), nl, c->ws + o_tail, gs_r,
                                            ng_r, perm_r, nr, match_out, reinterpret_cast<unsigned long long*>(cnt),
                                            err_word(c), s);
        else
            e = vdf::run_join_probe(left_key.data, nl, w, c->ws + o_tail, nr, match_out,
                                    reinterpret_cast<unsigned long long*>(cnt), s);
    }
    c->launches += 2;
    if (e != cudaSuccess) return from_cuda(c, e, "join");
    return read_count(c, cnt, n_matched_host, s, "read match count");
}

vdf_status vdf_unique(vdf_ctx* c, uint64_t n, vdf_col key, int keep_last, uint8_t* keep_out,
                      uint64_t* n_unique_dev, uint64_t* n_unique_host, void* stream) {
    if (!c) return VDF_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> lk(c->mu);
    return unique_locked(c, n, key, keep_last, keep_out, n_unique_dev, n_unique_host, stream);
}

vdf_status vdf_left_join_index(vdf_ctx* c, uint64_t n_left, vdf_col left_key, uint64_t n_right,
                               vdf_col right_key, int method, uint32_t* match_out, uint64_t* n_matched_dev,
                               uint64_t* n_matched_host, void* stream) {
    if (!c) return VDF_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> lk(c->mu);
    return left_join_locked(c, n_left, left_key, n_right, right_key, method, match_out, n_matched_dev,
                            n_matched_host, stream);
}

vdf_status vdf_unique_host(vdf_ctx* c, uint64_t n, vdf_col key, int keep_last, uint8_t* keep_out,
                           uint64_t* n_unique, void* stream) {
    if (!c) return VDF_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> lk(c->mu);
    vdf_status st;
    if ((st = check_rows(c, n)) != VDF_OK) return st;
    if (!valid_dtype(key.dtype)) return fail(c, VDF_ERR_INVALID_ARG, "bad key dtype");
    if (n && (!key.data || !keep_out)) return fail(c, VDF_ERR_INVALID_ARG, "NULL key or keep_out");
    if (n == 0) {
        if (n_unique) *n_unique = 0;
        return VDF_OK;
    }
    DeviceGuard g(c->device);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const size_t w = (size_t)vdf::dtype_width(key.dtype);
    const size_t o_key = 0, o_keep = align256(w * n);
    if ((st = io_ensure(c, o_keep + align256(n))) != VDF_OK) return st;
    cudaError_t e = cudaMemcpyAsync(c->io + o_key, key.data, w * n, cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) return from_cuda(c, e, "copy key to the device");
    uint64_t cnt = 0;
    if ((st = unique_locked(c, n, vdf_col{c->io + o_key, key.dtype}, keep_last, c->io + o_keep, nullptr, &cnt,
                            stream)) != VDF_OK)
        return st;
    e = cudaMemcpyAsync(keep_out, c->io + o_keep, n, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return from_cuda(c, e, "copy mask to the host");
    if (n_unique) *n_unique = cnt;
    return VDF_OK;
}

vdf_status vdf_left_join_index_host(vdf_ctx* c, uint64_t n_left, vdf_col left_key, uint64_t n_right,
                                    vdf_col right_key, int method, uint32_t* match_out, uint64_t* n_matched,
                                    void* stream) {
    if (!c) return VDF_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> lk(c->mu);
    vdf_status st;
    if ((st = check_rows(c, n_left)) != VDF_OK) return st;
    if ((st = check_rows(c, n_right)) != VDF_OK) return st;
    if (!valid_dtype(left_key.dtype) || left_key.dtype != right_key.dtype)
        return fail(c, VDF_ERR_INVALID_ARG, "bad or differing key dtypes");
    if ((n_left && (!left_key.data || !match_out)) || (n_right && !right_key.data))
        return fail(c, VDF_ERR_INVALID_ARG, "NULL key or match_out");
    DeviceGuard g(c->device);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const size_t w = (size_t)vdf::dtype_width(left_key.dtype);
    const size_t o_l = 0, o_r = align256(w * n_left), o_m = o_r + align256(w * n_right);
    if ((st = io_ensure(c, o_m + align256(4 * n_left))) != VDF_OK) return st;
    cudaError_t e = cudaSuccess;
    if (n_left) e = cudaMemcpyAsync(c->io + o_l, left_key.data, w * n_left, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess && n_right)
        e = cudaMemcpyAsync(c->io + o_r, right_key.data, w * n_right, cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) return from_cuda(c, e, "copy keys to the device");
    uint64_t cnt = 0;
    uint32_t* m_dev = reinterpret_cast<uint32_t*>(c->io + o_m);
    if ((st = left_join_locked(c, n_left, vdf_col{c->io + o_l, left_key.dtype}, n_right,
                               vdf_col{c->io + o_r, right_key.dtype}, method, m_dev, nullptr, &cnt, stream)) !=
        VDF_OK)
        return st;
    if (n_left) e = cudaMemcpyAsync(match_out, m_dev, 4 * n_left, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return from_cuda(c, e, "copy matches to the host");
    if (n_matched) *n_matched = cnt;
    return VDF_OK;
}

}  // extern "C"
