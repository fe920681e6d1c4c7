// vdf_server.cu -- request loop over device-resident columns (vdf_server_*).
//
// Clients submit sort + group-by requests (one key column and value columns
// that stay resident in device memory) and poll them by id.  A scheduler
// thread admits requests first-come first-served while the device memory they
// hold fits the HBM budget, and runs them with continuous batching: whenever
// one of the execution slots (each a context with its own stream and reserved
// workspace) is free, every admitted waiting request, up to the batch limits,
// joins one batch (vdf_batch_*), so requests arriving while other batches run
// are taken as soon as a slot and memory free up, and the batches of different
// slots overlap on the device.  Each slot owns output arenas for its largest
// batch, allocated once; a slot takes a new batch when its previous batch's
// results have all been released, so no batch allocates device memory.
//
// The reference has no serving layer: a host runs one sort_by_mt +
// transform_group_by_onecol_mt pair per query (sort_by_mt.hpp:3-180,
// transform_group_by_onecol_mt.hpp:14-373).
#include <chrono>
#include <atomic>
#include <condition_variable>
#include <deque>
#include <memory>
#include <thread>
#include <unordered_map>

#include "vdf_batch.h"
#include "vdf_ctx.h"

using namespace vdfc;

namespace {

enum ReqState : int32_t { RS_QUEUED = 0, RS_RUNNING = 1, RS_DONE = 2, RS_FAILED = 3 };

struct ServerBatch;

struct ServerReq {
    vdf_batch_query q{};
    uint64_t bytes = 0;
    int32_t state = RS_QUEUED;
    vdf_status status = VDF_OK;
    double t_submit = 0, t_start = 0, t_done = 0;
    std::shared_ptr<ServerBatch> batch;
    uint32_t index = 0;
};

struct ServerBatch {
    int slot = 0;
    vdf_batch* b = nullptr;
    std::vector<uint64_t> ids;
    vdf_batch_args args{};
    std::vector<vdf_batch_query> queries;
    std::vector<uint64_t> row_off, grp_off, ngroups;  // host copies once done
    cudaEvent_t done = nullptr;
    uint32_t unreleased = 0;
    uint64_t bytes = 0;
    bool finished = false;
};

uint64_t out_bytes_per_row(int nvals, const int32_t* dts) {
    uint64_t b = 4 + 8 + 8;  // permutation, group key slot, count
    for (int j = 0; j < nvals; ++j) b += (dts[j] == VDF_F64 || dts[j] == VDF_F32) ? 32 : 40;
    return b;
}

}  // namespace

// Output arenas of one slot, allocated once for max_batch_rows rows (and
// max_batch_queries queries); every batch on the slot writes into them.
struct SlotArena {
    std::vector<void*> allocs;
    uint32_t* perm = nullptr;
    void* gkeys = nullptr;
    int64_t* count = nullptr;
    vdf_agg_out aggs[VDF_BATCH_MAX_VALS] = {};
    uint64_t *row_off = nullptr, *grp_off = nullptr, *ngroups = nullptr;
    uint64_t bytes = 0;
};

struct vdf_server {
    vdf_server_config cfg{};
    int nslots = 0;
    std::vector<vdf_ctx*> ctx;
    std::vector<cudaStream_t> stream;
    std::vector<SlotArena> arena;
    std::vector<std::shared_ptr<ServerBatch>> running;  // per slot: batch in flight
    std::vector<std::shared_ptr<ServerBatch>> holding;  // per slot: finished batch with unreleased results
    double t_host_start = 0, t_host_finish = 0;         // host seconds spent starting / finishing batches
    std::mutex mu;
    std::condition_variable cv;       // wakes the scheduler (new work, releases)
    std::condition_variable done_cv;  // wakes waiters (completions)
    std::deque<uint64_t> queue;
    std::unordered_map<uint64_t, ServerReq> reqs;
    uint64_t next_id = 1;
    uint64_t fixed = 0, in_use = 0, max_in_use = 0;
    uint64_t batches = 0, completed = 0;
    bool stop = false;
    // failure injection for tests: batches left to fail at start / finish
    std::atomic<uint32_t> inject_start{0}, inject_finish{0};
    vdf_status inject_status = VDF_ERR_DEVICE;
    std::thread th;
    std::chrono::steady_clock::time_point t0;
    std::string last_error;

    double now() const { return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count(); }
};

namespace {

void free_batch_outputs(vdf_server* S, ServerBatch& B) {
    (void)S;
    if (B.b) vdf_batch_destroy(B.b);
    B.b = nullptr;
    if (B.done) cudaEventDestroy(B.done);
    B.done = nullptr;
}

// Builds and launches one batch on a free slot; called without the lock.
vdf_status start_batch(vdf_server* S, ServerBatch& B, std::string& why) {
    const vdf_server_config& c = S->cfg;
    for (uint32_t k = S->inject_start.load(); k > 0;) {
        if (S->inject_start.compare_exchange_weak(k, k - 1)) {
            why = "batch start failed (injected by a test hook)";
            return S->inject_status;
        }
    }
    cudaStream_t s = S->stream[B.slot];
    uint64_t rows = 0;
    for (const vdf_batch_query& q : B.queries) rows += q.n;
    const uint32_t nq = (uint32_t)B.queries.size();
    (void)rows;
    const SlotArena& A = S->arena[B.slot];
    vdf_batch_args& a = B.args;
    a = vdf_batch_args{};
    a.nqueries = nq;
    a.queries = B.queries.data();
    a.nvals = c.nvals;
    for (int j = 0; j < c.nvals; ++j) {
        a.val_dtypes[j] = c.val_dtypes[j];
        a.aggs[j] = A.aggs[j];
    }
    a.perm_out = A.perm;
    a.group_keys_out = A.gkeys;
    a.group_count_out = A.count;
    a.row_offset_out = A.row_off;
    a.group_offset_out = A.grp_off;
    a.n_groups_out = A.ngroups;
    cudaError_t e = cudaSuccess;
    vdf_batch_tuning t{c.small_rows, c.small_bits, c.seg_variant};
    vdf_status st = vdf_batch_create(S->ctx[B.slot], &a, c.use_default_tuning ? nullptr : &t, &B.b);
    if (st != VDF_OK) {
        why = vdf_ctx_last_error(S->ctx[B.slot]);
        return st;
    }
    st = c.use_graph ? vdf_batch_launch_graph(B.b, s) : vdf_batch_launch(B.b, s);
    if (st != VDF_OK) {
        why = vdf_ctx_last_error(S->ctx[B.slot]);
        return st;
    }
    if ((e = cudaEventCreateWithFlags(&B.done, cudaEventDisableTiming)) == cudaSuccess) e = cudaEventRecord(B.done, s);
    if (e != cudaSuccess) {
        why = cudaGetErrorString(e);
        return VDF_ERR_DEVICE;
    }
    return VDF_OK;
}

// Reads a finished batch's per-query offsets and its context's error word.
vdf_status finish_batch(vdf_server* S, ServerBatch& B, std::string& why) {
    const uint32_t nq = (uint32_t)B.queries.size();
    B.row_off.assign(nq, 0);
    B.grp_off.assign(nq, 0);
    B.ngroups.assign(nq, 0);
    cudaStream_t s = S->stream[B.slot];
    cudaError_t e = cudaSuccess;
    if (nq) {
        e = cudaMemcpyAsync(B.row_off.data(), B.args.row_offset_out, 8 * nq, cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(B.grp_off.data(), B.args.group_offset_out, 8 * nq, cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(B.ngroups.data(), B.args.n_groups_out, 8 * nq, cudaMemcpyDeviceToHost, s);
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) {
        why = cudaGetErrorString(e);
        return VDF_ERR_DEVICE;
    }
    vdf_status st = vdf_ctx_check(S->ctx[B.slot], s);  // device wait timeouts / bad indices
    if (st != VDF_OK) why = vdf_ctx_last_error(S->ctx[B.slot]);
    for (uint32_t k = S->inject_finish.load(); st == VDF_OK && k > 0;) {
        if (S->inject_finish.compare_exchange_weak(k, k - 1)) {
            why = "batch finish failed (injected by a test hook)";
            return S->inject_status;
        }
    }
    return st;
}

void scheduler(vdf_server* S) {
    DeviceGuard g(S->cfg.device);
    const uint64_t per_row = out_bytes_per_row(S->cfg.nvals, S->cfg.val_dtypes);
    std::unique_lock<std::mutex> lk(S->mu);
    while (!S->stop) {
        bool progressed = false;
        // completions
        for (int slot = 0; slot < S->nslots; ++slot) {
            std::shared_ptr<ServerBatch> B = S->running[slot];
            if (!B || cudaEventQuery(B->done) == cudaErrorNotReady) continue;
            cudaGetLastError();
            const double t_fin0 = S->now();
            lk.unlock();
            std::string why;
            vdf_status st = finish_batch(S, *B, why);
            lk.lock();
            B->finished = true;
            S->running[slot] = nullptr;
            S->holding[slot] = B;  // the slot's arenas hold its results until released
            S->t_host_finish += S->now() - t_fin0;
            const double t = S->now();
            for (uint64_t id : B->ids) {
                auto it = S->reqs.find(id);
                if (it == S->reqs.end()) continue;
                it->second.state = st == VDF_OK ? RS_DONE : RS_FAILED;
                it->second.status = st;
                it->second.t_done = t;
                S->completed++;
            }
            if (st != VDF_OK) S->last_error = why;
            progressed = true;
            S->done_cv.notify_all();
        }
        // admission: first come, first served, while memory, the batch limits
        // and a free slot allow
        for (int slot = 0; slot < S->nslots && !S->queue.empty(); ++slot) {
            if (S->running[slot] || S->holding[slot]) continue;
            auto B = std::make_shared<ServerBatch>();
            B->slot = slot;
            uint64_t rows = 0, bytes = 0;
            while (!S->queue.empty() && B->ids.size() < S->cfg.max_batch_queries) {
                ServerReq& r = S->reqs[S->queue.front()];
                if (!B->ids.empty() && rows + r.q.n > S->cfg.max_batch_rows) break;
                if (S->in_use + bytes + r.bytes > S->cfg.hbm_budget_bytes) break;
                rows += r.q.n;
                bytes += r.bytes;
                B->ids.push_back(S->queue.front());
                S->queue.pop_front();
            }
            if (B->ids.empty()) break;  // the head waits for memory to be released
            const double t = S->now();
            for (uint32_t i = 0; i < B->ids.size(); ++i) {
                ServerReq& r = S->reqs[B->ids[i]];
                r.state = RS_RUNNING;
                r.t_start = t;
                r.batch = B;
                r.index = i;
                B->queries.push_back(r.q);
            }
            B->bytes = bytes;
            B->unreleased = (uint32_t)B->ids.size();
            S->in_use += bytes;
            S->max_in_use = std::max(S->max_in_use, S->in_use);
            S->running[slot] = B;
            S->batches++;
            const double t_st0 = S->now();
            lk.unlock();
            std::string why;
            vdf_status st = start_batch(S, *B, why);
            lk.lock();
            S->t_host_start += S->now() - t_st0;
            if (st != VDF_OK) {
                S->running[slot] = nullptr;
                B->finished = true;
                for (uint64_t id : B->ids) {
                    ServerReq& r = S->reqs[id];
                    r.state = RS_FAILED;
                    r.status = st;
                    r.t_done = S->now();
                    S->completed++;
                }
                S->last_error = why;
                S->done_cv.notify_all();
            }
            progressed = true;
        }
        (void)per_row;
        if (!progressed) {
            bool busy = false;
            for (auto& b : S->running) busy = busy || (b != nullptr);
            // poll device completions often while batches run; sleep otherwise
            S->cv.wait_for(lk, busy ? std::chrono::microseconds(20) : std::chrono::milliseconds(5));
        }
    }
}

}  // namespace

extern "C" {

vdf_status vdf_server_default_config(vdf_server_config* c) {
    if (!c) return VDF_ERR_INVALID_ARG;
    *c = vdf_server_config{};
    c->device = 0;
    c->hbm_budget_bytes = 150ull * 1000 * 1000 * 1000;
    c->slots = 2;
    c->max_batch_rows = 1u << 27;
    c->max_batch_queries = 4096;
    c->nvals = 0;
    c->use_default_tuning = 1;
    vdf::BatchTuning t = vdf::default_batch_tuning();
    c->small_rows = t.small_rows;
    c->small_bits = t.small_bits;
    c->seg_variant = t.seg_variant;
    c->use_graph = 0;
    c->resident_bytes = 0;
    return VDF_OK;
}

vdf_status vdf_server_create(const vdf_server_config* cfg, vdf_server** out) {
    if (!cfg || !out) return VDF_ERR_INVALID_ARG;
    *out = nullptr;
    if (cfg->slots < 1 || cfg->slots > 8 || cfg->nvals < 0 || cfg->nvals > VDF_BATCH_MAX_VALS ||
        cfg->max_batch_rows < 1 || cfg->max_batch_rows > vdf::kMaxBatchRows || cfg->max_batch_queries < 1)
        return VDF_ERR_INVALID_ARG;
    for (int j = 0; j < cfg->nvals; ++j)
        if (!valid_dtype(cfg->val_dtypes[j])) return VDF_ERR_INVALID_ARG;
    if (!cfg->use_default_tuning) {
        vdf::BatchTuning t{cfg->small_rows, cfg->small_bits, cfg->seg_variant};
        if (!vdf::batch_tuning_valid(t)) return VDF_ERR_INVALID_ARG;
    }
    auto S = std::make_unique<vdf_server>();
    S->cfg = *cfg;
    S->nslots = (int)cfg->slots;
    S->t0 = std::chrono::steady_clock::now();
    DeviceGuard g(cfg->device);
    for (int i = 0; i < S->nslots; ++i) {
        vdf_ctx* c = nullptr;
        vdf_status st = vdf_ctx_create(cfg->device, &c);
        if (st != VDF_OK) {
            for (vdf_ctx* x : S->ctx) vdf_ctx_destroy(x);
            for (cudaStream_t x : S->stream) cudaStreamDestroy(x);
            return st;
        }
        S->ctx.push_back(c);
        cudaStream_t s = nullptr;
        if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess) {
            for (vdf_ctx* x : S->ctx) vdf_ctx_destroy(x);
            for (cudaStream_t x : S->stream) cudaStreamDestroy(x);
            return VDF_ERR_DEVICE;
        }
        S->stream.push_back(s);
        // a batch of max_batch_rows rows never regrows the slot's workspace
        vdf_batch_query q{};
        q.n = cfg->max_batch_rows;
        q.key.dtype = VDF_I64;
        q.key.data = reinterpret_cast<const void*>(16);
        for (int j = 0; j < cfg->nvals; ++j) q.vals[j] = reinterpret_cast<const void*>(16);
        vdf_batch_args a{};
        a.nqueries = 1;
        a.queries = &q;
        a.nvals = cfg->nvals;
        for (int j = 0; j < cfg->nvals; ++j) a.val_dtypes[j] = cfg->val_dtypes[j];
        vdf::BatchPlan P;
        std::string why;
        vdf::BatchTuning t = cfg->use_default_tuning ? vdf::default_batch_tuning()
                                                     : vdf::BatchTuning{cfg->small_rows, cfg->small_bits,
                                                                        cfg->seg_variant};
        if (vdf::plan_batch(P, a, t, why, c->tuning.msd, c->tuning.msd_match)) {
            // 8-byte keys need the most (a batch whose large queries all have
            // 4-byte keys packs 4-byte images); the plan's tail is the largest
            // need, plus descriptor tables for a full batch of queries: per
            // query a descriptor, its segment (twice with the MSD-first
            // tables), chunks and flags; per 1024 rows a tile entry (twice),
            // per kMsdCap / 2 rows an MSD chunk and its start
            const size_t Q = (size_t)cfg->max_batch_queries, R = (size_t)cfg->max_batch_rows;
            const size_t desc = (sizeof(vdf::BatchQuery) + 2 * sizeof(vdf::SegDesc) + 2 * sizeof(vdf::SegChunk) +
                                 sizeof(vdf::MsdSegChunk) + 32) * Q + 8 * (R / 1024 + 8) +
                                (sizeof(vdf::MsdSegChunk) + 4) * (R / (vdf::kMsdCap / 2) + 8) + 16 * 256;
            st = vdf_ctx_reserve(c, P.ws_bytes + desc + (P.ws_bytes >> 4));
            if (st != VDF_OK) {
                for (vdf_ctx* x : S->ctx) vdf_ctx_destroy(x);
                for (cudaStream_t x : S->stream) cudaStreamDestroy(x);
                return st;
            }
            S->fixed += P.ws_bytes + desc + (P.ws_bytes >> 4);
        }
    }
    // output arenas, one set per slot
    S->arena.resize(S->nslots);
    for (int i = 0; i < S->nslots; ++i) {
        SlotArena& A = S->arena[i];
        const size_t R = cfg->max_batch_rows, Q = cfg->max_batch_queries;
        bool ok = true;
        auto alloc = [&](size_t bytes) -> void* {
            void* p = nullptr;
            if (cudaMalloc(&p, bytes) != cudaSuccess) {
                cudaGetLastError();
                ok = false;
                return nullptr;
            }
            A.allocs.push_back(p);
            A.bytes += bytes;
            return p;
        };
        A.perm = static_cast<uint32_t*>(alloc(4 * R));
        A.gkeys = alloc(8 * R);
        A.count = static_cast<int64_t*>(alloc(8 * R));
        for (int j = 0; j < cfg->nvals; ++j) {
            const bool fl = (cfg->val_dtypes[j] == VDF_F64 || cfg->val_dtypes[j] == VDF_F32);
            const size_t w = (size_t)vdf::dtype_width(cfg->val_dtypes[j]);
            A.aggs[j].sum = alloc(8 * R);
            A.aggs[j].sum_hi = fl ? nullptr : static_cast<int64_t*>(alloc(8 * R));
            A.aggs[j].min = alloc(w * R);
            A.aggs[j].max = alloc(w * R);
            A.aggs[j].mean = static_cast<double*>(alloc(8 * R));
        }
        A.row_off = static_cast<uint64_t*>(alloc(8 * Q));
        A.grp_off = static_cast<uint64_t*>(alloc(8 * Q));
        A.ngroups = static_cast<uint64_t*>(alloc(8 * Q));
        S->fixed += A.bytes;
        if (!ok) {
            for (SlotArena& X : S->arena)
                for (void* p : X.allocs) cudaFree(p);
            for (vdf_ctx* x : S->ctx) vdf_ctx_destroy(x);
            for (cudaStream_t x : S->stream) cudaStreamDestroy(x);
            return VDF_ERR_OOM;
        }
    }
    S->fixed += cfg->resident_bytes;
    if (S->fixed > cfg->hbm_budget_bytes) {
        for (SlotArena& X : S->arena)
            for (void* p : X.allocs) cudaFree(p);
        for (vdf_ctx* x : S->ctx) vdf_ctx_destroy(x);
        for (cudaStream_t x : S->stream) cudaStreamDestroy(x);
        return VDF_ERR_INVALID_ARG;
    }
    S->in_use = S->fixed;
    S->max_in_use = S->fixed;
    S->running.assign(S->nslots, nullptr);
    S->holding.assign(S->nslots, nullptr);
    vdf_server* raw = S.release();
    raw->th = std::thread(scheduler, raw);
    *out = raw;
    return VDF_OK;
}

vdf_status vdf_server_submit(vdf_server* S, const vdf_batch_query* q, uint64_t* id) {
    if (!S || !q || !id) return VDF_ERR_INVALID_ARG;
    const double t = S->now();
    if (!valid_dtype(q->key.dtype) || (q->n && !q->key.data)) return VDF_ERR_INVALID_ARG;
    for (int j = 0; j < S->cfg.nvals; ++j)
        if (q->n && !q->vals[j]) return VDF_ERR_INVALID_ARG;
    if (q->n > S->cfg.max_batch_rows) return VDF_ERR_UNSUPPORTED;
    const uint64_t bytes = q->n * out_bytes_per_row(S->cfg.nvals, S->cfg.val_dtypes) + 256;
    std::lock_guard<std::mutex> lk(S->mu);
    if (S->fixed + bytes > S->cfg.hbm_budget_bytes) return VDF_ERR_OOM;  // could never be admitted
    const uint64_t rid = S->next_id++;
    ServerReq& r = S->reqs[rid];
    r.q = *q;
    r.bytes = bytes;
    r.t_submit = t;
    S->queue.push_back(rid);
    *id = rid;
    S->cv.notify_one();
    return VDF_OK;
}

static void fill_result(vdf_server* S, const ServerReq& r, vdf_server_result* out) {
    *out = vdf_server_result{};
    out->n = r.q.n;
    out->t_submit = r.t_submit;
    out->t_start = r.t_start;
    out->t_done = r.t_done;
    if (r.state != RS_DONE || !r.batch) return;
    const ServerBatch& B = *r.batch;
    const uint64_t ro = B.row_off[r.index], go = B.grp_off[r.index];
    out->n_groups = B.ngroups[r.index];
    out->perm = B.args.perm_out + ro;
    out->group_keys = static_cast<const unsigned char*>(B.args.group_keys_out) + 8 * go;
    out->group_count = B.args.group_count_out + go;
    for (int j = 0; j < S->cfg.nvals; ++j) {
        const vdf_agg_out& a = B.args.aggs[j];
        const size_t w = (size_t)vdf::dtype_width(S->cfg.val_dtypes[j]);
        vdf_agg_out& o = out->aggs[j];
        o.sum = static_cast<unsigned char*>(a.sum) + 8 * go;
        o.sum_hi = a.sum_hi ? a.sum_hi + go : nullptr;
        o.min = static_cast<unsigned char*>(a.min) + w * go;
        o.max = static_cast<unsigned char*>(a.max) + w * go;
        o.mean = a.mean + go;
    }
}

vdf_status vdf_server_poll(vdf_server* S, uint64_t id, int32_t* state, vdf_server_result* out) {
    if (!S || !state) return VDF_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> lk(S->mu);
    auto it = S->reqs.find(id);
    if (it == S->reqs.end()) return VDF_ERR_INVALID_ARG;
    *state = it->second.state;
    if (out) fill_result(S, it->second, out);
    return it->second.state == RS_FAILED ? it->second.status : VDF_OK;
}

vdf_status vdf_server_wait(vdf_server* S, uint64_t id, double timeout_s, vdf_server_result* out) {
    if (!S) return VDF_ERR_INVALID_ARG;
    std::unique_lock<std::mutex> lk(S->mu);
    auto it = S->reqs.find(id);
    if (it == S->reqs.end()) return VDF_ERR_INVALID_ARG;
    const auto deadline = std::chrono::steady_clock::now() + std::chrono::duration<double>(timeout_s);
    while (S->reqs[id].state == RS_QUEUED || S->reqs[id].state == RS_RUNNING) {
        if (S->done_cv.wait_until(lk, deadline) == std::cv_status::timeout &&
            (S->reqs[id].state == RS_QUEUED || S->reqs[id].state == RS_RUNNING))
            return VDF_ERR_TIMEOUT;
    }
    const ServerReq& r = S->reqs[id];
    if (out) fill_result(S, r, out);
    return r.state == RS_FAILED ? r.status : VDF_OK;
}

vdf_status vdf_server_release(vdf_server* S, uint64_t id) {
    if (!S) return VDF_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> lk(S->mu);
    auto it = S->reqs.find(id);
    if (it == S->reqs.end()) return VDF_ERR_INVALID_ARG;
    if (it->second.state != RS_DONE && it->second.state != RS_FAILED) return VDF_ERR_INVALID_ARG;
    std::shared_ptr<ServerBatch> B = it->second.batch;
    S->reqs.erase(it);
    if (B && --B->unreleased == 0) {
        DeviceGuard g(S->cfg.device);
        free_batch_outputs(S, *B);
        S->in_use -= B->bytes;
        if (S->holding[B->slot] == B) S->holding[B->slot] = nullptr;  // the slot's arenas are free again
        S->cv.notify_one();
    }
    return VDF_OK;
}

vdf_status vdf_server_inject_failure(vdf_server* S, int where, uint32_t count, vdf_status status) {
    if (!S || (where != 0 && where != 1) || status == VDF_OK) return VDF_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> lk(S->mu);
    S->inject_status = status;
    (where == 0 ? S->inject_start : S->inject_finish).store(count);
    return VDF_OK;
}

vdf_status vdf_server_read_stats(vdf_server* S, vdf_server_stats* out) {
    if (!S || !out) return VDF_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> lk(S->mu);
    out->batches = S->batches;
    out->completed = S->completed;
    out->queued = S->queue.size();
    out->in_use_bytes = S->in_use;
    out->max_in_use_bytes = S->max_in_use;
    out->fixed_bytes = S->fixed;
    out->host_start_seconds = S->t_host_start;
    out->host_finish_seconds = S->t_host_finish;
    return VDF_OK;
}

const char* vdf_server_last_error(vdf_server* S) {
    if (!S) return "";
    std::lock_guard<std::mutex> lk(S->mu);
    return S->last_error.c_str();
}

void vdf_server_destroy(vdf_server* S) {
    if (!S) return;
    {
        std::lock_guard<std::mutex> lk(S->mu);
        S->stop = true;
        S->cv.notify_all();
    }
    if (S->th.joinable()) S->th.join();
    DeviceGuard g(S->cfg.device);
    for (cudaStream_t s : S->stream) cudaStreamSynchronize(s);
    for (auto& kv : S->reqs)
        if (kv.second.batch && kv.second.batch->b) {
            ServerBatch& B = *kv.second.batch;
            free_batch_outputs(S, B);
        }
    for (auto& B : S->running)
        if (B) free_batch_outputs(S, *B);
    for (cudaStream_t s : S->stream) {
        cudaStreamSynchronize(s);
        cudaStreamDestroy(s);
    }
    for (SlotArena& A : S->arena)
        for (void* p : A.allocs) cudaFree(p);
    for (vdf_ctx* c : S->ctx) vdf_ctx_destroy(c);
    delete S;
}

}  // extern "C"
