// vdf_batch_small.cu -- the batch's small queries, one CTA per query.
//
// A persistent kernel: each CTA takes the next query from a device work
// counter until none is left.  A query of n <= CAP rows is sorted entirely in
// shared memory (stable LSD radix passes over its ordered key images, ranks
// from warp digit matches and per-warp counters as in the global radix pass,
// but with no look-back: the whole query is one tile), its permutation is
// written out, group heads come from one block scan, and each group is
// reduced by one warp with the same aggregate operations as the segmented
// reduction (vdf_agg.cuh), so a query gives the same groups whichever path
// runs it.  The reference's per-query equivalent is one sort_by_mt call
// (sort_by_mt.hpp:3-180) plus one transform_group_by_onecol_mt call
// (transform_group_by_onecol_mt.hpp:182-337).
#include "vdf_agg.cuh"
#include "vdf_batch.h"
#include "vdf_common.cuh"

namespace vdf {
namespace {

template <int THREADS, int ITEMS, int BITS>
struct SmallCfg {
    static constexpr int RADIX = 1 << BITS;
    static constexpr int WARPS = THREADS / 32;
    static constexpr int CAP = THREADS * ITEMS;
    static constexpr size_t KEYS = (size_t)CAP * 8;
    static constexpr size_t VALS = (size_t)CAP * 4;
    static constexpr size_t CNT = (size_t)WARPS * RADIX * 4;
    static constexpr size_t HPOS = ((size_t)(CAP + 1) * 4 + 15) / 16 * 16;
    static constexpr size_t SMEM = KEYS + VALS + CNT + HPOS + 16 + WARPS * 4;
};

// Exclusive scan of one value per thread; *total gets the sum.  Contains
// barriers: every thread of the CTA calls it.
template <int THREADS>
__device__ __forceinline__ uint32_t block_excl_scan(uint32_t v, uint32_t* wsum, uint32_t* total) {
    constexpr int WARPS = THREADS / 32;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t incl = v;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const uint32_t t = __shfl_up_sync(0xffffffffu, incl, d);
        if (lane >= d) incl += t;
    }
    __syncthreads();  // wsum may still be read from a previous call
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

template <int THREADS, int ITEMS, int BITS>
__global__ void __launch_bounds__(THREADS) k_batch_small(BatchDev b) {
    using C = SmallCfg<THREADS, ITEMS, BITS>;
    constexpr int RADIX = C::RADIX, WARPS = C::WARPS, CAP = C::CAP;
    constexpr uint32_t MASK = RADIX - 1;
    extern __shared__ __align__(16) unsigned char smem[];
    uint64_t* sk = reinterpret_cast<uint64_t*>(smem);
    uint32_t* sv = reinterpret_cast<uint32_t*>(smem + C::KEYS);
    uint32_t* wcnt = reinterpret_cast<uint32_t*>(smem + C::KEYS + C::VALS);
    uint32_t* hpos = reinterpret_cast<uint32_t*>(smem + C::KEYS + C::VALS + C::CNT);
    uint32_t* misc = reinterpret_cast<uint32_t*>(smem + C::KEYS + C::VALS + C::CNT + C::HPOS);
    uint32_t* wsum = misc + 4;

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const uint32_t lt = lanemask_lt();

    for (;;) {
        __syncthreads();  // the previous query is done with shared memory
        if (tid == 0) misc[0] = atomicAdd(b.work_counter, 1u);
        __syncthreads();
        const uint32_t qi = misc[0];
        if (qi >= b.n_small_queries) break;
        const uint32_t qid = b.small_queries[qi];
        const BatchQuery q = b.queries[qid];
        const uint32_t n = (uint32_t)q.n;
        if (q.n > (uint64_t)CAP || q.n == 0) {
            if (tid == 0 && q.n) atomicOr(b.err, ERR_BAD_INDEX);
            continue;
        }
        const int dt = q.key_dtype;
        const int kw = dtype_width(dt);
        const int passes = (kw * 8 + BITS - 1) / BITS;
        const uint32_t ia = (n + THREADS - 1) / THREADS;  // items per thread in use
        const uint64_t row0 = q.row_offset;

        // ---- keys in registers: thread items at positions (warp*ia + j)*32 + lane
        uint64_t key[ITEMS];
        uint32_t val[ITEMS];
#pragma unroll
        for (int j = 0; j < ITEMS; ++j) {
            const uint32_t pos = ((uint32_t)warp * ia + j) * 32 + lane;
            key[j] = ~0ull;
            val[j] = pos;
            if (j < (int)ia && pos < n) {
                key[j] = (kw == 4) ? (uint64_t)order32(__ldg(static_cast<const uint32_t*>(q.key) + pos), dt, false)
                                   : order64(__ldg(static_cast<const uint64_t*>(q.key) + pos), dt, false);
            }
        }

        // ---- stable LSD passes, all in shared memory ----------------------
        for (int p = 0; p < passes; ++p) {
            const uint32_t shift = (uint32_t)(p * BITS);
            for (int i = tid; i < WARPS * RADIX; i += THREADS) wcnt[i] = 0;
            __syncthreads();
            uint32_t* my = wcnt + warp * RADIX;
            uint32_t rank[ITEMS];
#pragma unroll
            for (int j = 0; j < ITEMS; ++j) {
                rank[j] = 0;
                if (j < (int)ia) {
                    const uint32_t pos = ((uint32_t)warp * ia + j) * 32 + lane;
                    const bool ok = pos < n;
                    const uint32_t d = (uint32_t)(key[j] >> shift) & MASK;
                    uint32_t peers;
                    if (BITS > 4) {
                        peers = __match_any_sync(0xffffffffu, ok ? d : (uint32_t)RADIX);
                    } else {
                        peers = __ballot_sync(0xffffffffu, ok);
                        if (!ok) peers = ~peers;
#pragma unroll
                        for (int bt = 0; bt < BITS; ++bt) {
                            const uint32_t bal = __ballot_sync(0xffffffffu, (d >> bt) & 1u);
                            peers &= ((d >> bt) & 1u) ? bal : ~bal;
                        }
                    }
                    const int leader = __ffs(peers) - 1;
                    uint32_t base = 0;
                    if (lane == leader && ok) {
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
            for (int bin = tid; bin < RADIX; bin += THREADS) {
                uint32_t run = 0;
#pragma unroll
                for (int w = 0; w < WARPS; ++w) {
                    const uint32_t c = wcnt[w * RADIX + bin];
                    wcnt[w * RADIX + bin] = run;
                    run += c;
                }
                tot = run;  // RADIX <= THREADS: one bin per thread
            }
            uint32_t all;
            const uint32_t start = block_excl_scan<THREADS>(tot, wsum, &all);
            if (tid < RADIX)
#pragma unroll
                for (int w = 0; w < WARPS; ++w) wcnt[w * RADIX + tid] += start;
            __syncthreads();
#pragma unroll
            for (int j = 0; j < ITEMS; ++j) {
                if (j < (int)ia) {
                    const uint32_t pos = ((uint32_t)warp * ia + j) * 32 + lane;
                    if (pos < n) {
                        const uint32_t d = (uint32_t)(key[j] >> shift) & MASK;
                        uint32_t r = rank[j] + my[d];
                        if (r >= n) {  // never when the counts are consistent
                            atomicOr(b.err, ERR_BAD_INDEX);
                            r = pos;
                        }
                        sk[r] = key[j];
                        sv[r] = val[j];
                    }
                }
            }
            __syncthreads();
            if (p + 1 < passes) {
#pragma unroll
                for (int j = 0; j < ITEMS; ++j) {
                    const uint32_t pos = ((uint32_t)warp * ia + j) * 32 + lane;
                    if (j < (int)ia && pos < n) {
                        key[j] = sk[pos];
                        val[j] = sv[pos];
                    }
                }
            }
        }

        // ---- permutation -------------------------------------------------
        for (uint32_t i = tid; i < n; i += THREADS) b.perm_out[row0 + i] = sv[i];

        // ---- group heads: thread t owns sorted rows [t*ia, t*ia + ia) -------
        const uint32_t r0 = (uint32_t)tid * ia;
        const uint32_t r1 = min(n, r0 + ia);
        uint32_t heads = 0;
        for (uint32_t i = r0; i < r1; ++i) heads += (i == 0 || sk[i] != sk[i - 1]) ? 1u : 0u;
        uint32_t G;
        uint32_t g = block_excl_scan<THREADS>(heads, wsum, &G);
        unsigned char* kout = static_cast<unsigned char*>(b.group_keys_out);
        for (uint32_t i = r0; i < r1; ++i) {
            if (i == 0 || sk[i] != sk[i - 1]) {
                hpos[g] = i;
                if (kout) {
                    if (kw == 4)
                        reinterpret_cast<uint32_t*>(kout + 8 * row0)[g] = unorder32((uint32_t)sk[i], dt, false);
                    else
                        reinterpret_cast<uint64_t*>(kout + 8 * row0)[g] = unorder64(sk[i], dt, false);
                }
                ++g;
            }
        }
        if (tid == 0) {
            hpos[G] = n;
            b.n_groups_out[qid] = G;
            b.group_offset_out[qid] = row0;
        }
        __syncthreads();
        if (b.group_count_out)
            for (uint32_t x = tid; x < G; x += THREADS) b.group_count_out[row0 + x] = (int64_t)(hpos[x + 1] - hpos[x]);

        // ---- aggregates: one warp per group -------------------------------
        for (int v = 0; v < b.nvals; ++v) {
            const int vdt = b.val_dtype[v];
            const int vc = vclass(vdt);
            const void* src = q.vals[v];
            const vdf_agg_out o = b.aggs[v];
            for (uint32_t x = warp; x < G; x += WARPS) {
                const uint32_t lo = hpos[x], hi = hpos[x + 1];
                uint64_t w[4] = {0, 0, 0, 0};
                bool have = false;
                for (uint32_t i = lo + lane; i < hi; i += 32) {
                    const uint64_t xv = load_val(src, vdt, sv[i]);
                    if (!have) {
                        col_init(w, xv, vc);
                        have = true;
                    } else {
                        uint64_t one[4];
                        col_init(one, xv, vc);
                        col_merge(w, one, vc);
                    }
                }
#pragma unroll
                for (int d = 16; d >= 1; d >>= 1) {
                    uint64_t other[4];
#pragma unroll
                    for (int k = 0; k < 4; ++k) other[k] = __shfl_down_sync(0xffffffffu, w[k], d);
                    const bool oh = __shfl_down_sync(0xffffffffu, have ? 1 : 0, d) != 0;
                    if (lane + d < 32 && oh) {
                        if (have) col_merge(w, other, vc);
                        else {
#pragma unroll
                            for (int k = 0; k < 4; ++k) w[k] = other[k];
                            have = true;
                        }
                    }
                }
                if (lane == 0) {
                    const uint64_t slot = row0 + x;
                    const uint32_t cnt = hi - lo;
                    if (vc == VC_FLOAT) {
                        const double s = __dadd_rn(as_f(w[0]), as_f(w[1]));
                        if (o.sum) static_cast<double*>(o.sum)[slot] = s;
                        if (o.mean) o.mean[slot] = s / (double)cnt;
                        if (vdt == F64) {
                            if (o.min) static_cast<double*>(o.min)[slot] = as_f(w[2]);
                            if (o.max) static_cast<double*>(o.max)[slot] = as_f(w[3]);
                        } else {
                            if (o.min) static_cast<float*>(o.min)[slot] = (float)as_f(w[2]);
                            if (o.max) static_cast<float*>(o.max)[slot] = (float)as_f(w[3]);
                        }
                    } else {
                        if (o.sum) static_cast<int64_t*>(o.sum)[slot] = (int64_t)w[0];
                        if (o.sum_hi) o.sum_hi[slot] = (int64_t)w[1];
                        if (o.mean) o.mean[slot] = i128_to_double(w[0], w[1], vc == VC_SINT) / (double)cnt;
                        if (dtype_width(vdt) == 4) {
                            if (o.min) static_cast<uint32_t*>(o.min)[slot] = (uint32_t)w[2];
                            if (o.max) static_cast<uint32_t*>(o.max)[slot] = (uint32_t)w[3];
                        } else {
                            if (o.min) static_cast<uint64_t*>(o.min)[slot] = w[2];
                            if (o.max) static_cast<uint64_t*>(o.max)[slot] = w[3];
                        }
                    }
                }
            }
        }
    }
}

using SmallKernel = void (*)(BatchDev);
struct SmallVariant {
    int threads, cap, bits;
    size_t smem;
    SmallKernel k;
    int blocks_per_sm;
};
template <int THREADS, int ITEMS, int BITS>
SmallVariant make_small() {
    using C = SmallCfg<THREADS, ITEMS, BITS>;
    return SmallVariant{THREADS, C::CAP, BITS, C::SMEM, k_batch_small<THREADS, ITEMS, BITS>, 0};
}
SmallVariant g_small[] = {
    make_small<256, 16, 8>(),  // up to 4096 rows
    make_small<512, 16, 8>(),  // up to 8192 rows
    make_small<256, 16, 4>(),
    make_small<512, 16, 4>(),
};
static_assert(512 * 16 == kSmallMaxRows, "widest one-CTA variant");

}  // namespace

cudaError_t prepare_batch_kernels() {
    for (SmallVariant& v : g_small) {
        cudaError_t e = cudaFuncSetAttribute(v.k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)v.smem);
        if (e != cudaSuccess) return e;
        int nb = 0;
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, v.k, v.threads, v.smem);
        if (e != cudaSuccess) return e;
        v.blocks_per_sm = nb > 0 ? nb : 1;
    }
    return cudaSuccess;
}

cudaError_t launch_small_queries(const BatchDev& b, cudaStream_t s, int sms) {
    if (b.n_small_queries == 0) return cudaSuccess;
    // the narrowest variant that holds every small query
    const int bits = b.small_bits;
    const SmallVariant* pick = nullptr;
    for (const SmallVariant& v : g_small)
        if (v.bits == bits && (uint32_t)v.cap >= b.small_cap && (!pick || v.cap < pick->cap)) pick = &v;
    if (!pick) return cudaErrorInvalidValue;
    const uint32_t grid = (uint32_t)std::min<uint64_t>((uint64_t)sms * pick->blocks_per_sm, b.n_small_queries);
    pick->k<<<grid, pick->threads, pick->smem, s>>>(b);
    return cudaGetLastError();
}

}  // namespace vdf
