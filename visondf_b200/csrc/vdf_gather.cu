// vdf_gather.cu -- payload gather by a permutation, and the group-by
// "transform" broadcast.
//
// k_gather replaces the reference's permute_block_mt
// (V/inlines/transform/sort_by/permute_block_mt.inl:3-47) and
// no_inplace_permutation (V/inlines/no_inplace_permutation.inl:3-79), which
// apply the sort's idx to every column of a type block with AVX-512 gathers.
// Here one launch serves up to kMaxGather columns of mixed width: each thread
// owns 4 consecutive output rows, reads their 4 row ids with one 16-byte load
// (the permutation is read once for all columns), issues the 4 random reads
// per column back to back, and writes each column's 4 results with 16-byte
// stores.
//
// When a workspace is supplied and two or more columns are gathered, the
// columns are first packed row-wise into records of 8-byte slots (16..64
// bytes, one streaming pass), and the gather then reads ONE record per row:
// a random read costs a full DRAM access (64 bytes on this part) however few
// bytes it uses, so gathering k columns separately costs k such accesses per
// row while the packed record costs one.
//
// k_broadcast produces the reference's transform output
// (CreateValueCol::apply, V/inlines/transform/transform_group_by/
// create_value_col.inl:36-61: v_col[i] = lookup.at(key_vec[i])): every row
// receives its group's aggregate, in sorted order or scattered back to the
// original row order through the permutation.
#include "vdf_common.cuh"
#include "vdf_internal.h"

namespace vdf {

template <bool VEC>
__global__ void __launch_bounds__(256) k_gather(GatherArgs g) {
    const uint64_t r0 = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) * 4;
    if (r0 >= g.n) return;
    if (VEC && r0 + 4 <= g.n) {
        uint4 p = ldg_stream(reinterpret_cast<const uint4*>(g.perm + r0));
        if (p.x >= g.n || p.y >= g.n || p.z >= g.n || p.w >= g.n) {  // not a permutation of [0, n)
            if (g.err) atomicOr(g.err, ERR_BAD_INDEX);
            p.x = p.x < g.n ? p.x : 0;
            p.y = p.y < g.n ? p.y : 0;
            p.z = p.z < g.n ? p.z : 0;
            p.w = p.w < g.n ? p.w : 0;
        }
#pragma unroll 1
        for (int c = 0; c < g.ncols; ++c) {
            if (g.width[c] == 8) {
                const unsigned long long* s = static_cast<const unsigned long long*>(g.src[c]);
                ulonglong2 a, b;
                a.x = ld_rand8(s + p.x);
                a.y = ld_rand8(s + p.y);
                b.x = ld_rand8(s + p.z);
                b.y = ld_rand8(s + p.w);
                ulonglong2* d = reinterpret_cast<ulonglong2*>(static_cast<unsigned long long*>(g.dst[c]) + r0);
                stg_stream(d, a);
                stg_stream(d + 1, b);
            } else {
                const uint32_t* s = static_cast<const uint32_t*>(g.src[c]);
                uint4 v;
                v.x = ld_rand4(s + p.x);
                v.y = ld_rand4(s + p.y);
                v.z = ld_rand4(s + p.z);
                v.w = ld_rand4(s + p.w);
                stg_stream(reinterpret_cast<uint4*>(static_cast<uint32_t*>(g.dst[c]) + r0), v);
            }
        }
        return;
    }
    const uint64_t r1 = r0 + 4 < g.n ? r0 + 4 : g.n;
    for (uint64_t r = r0; r < r1; ++r) {
        uint32_t p = g.perm[r];
        if (p >= g.n) {
            if (g.err) atomicOr(g.err, ERR_BAD_INDEX);
            p = 0;
        }
        for (int c = 0; c < g.ncols; ++c) {
            if (g.width[c] == 8)
                static_cast<unsigned long long*>(g.dst[c])[r] = ld_rand8(static_cast<const unsigned long long*>(g.src[c]) + p);
            else
                static_cast<uint32_t*>(g.dst[c])[r] = ld_rand4(static_cast<const uint32_t*>(g.src[c]) + p);
        }
    }
}

template <int REC>
__global__ void __launch_bounds__(256) k_pack(GatherArgs g, unsigned char* recs) {
    constexpr int SLOTS = REC / 8;
    const uint64_t r = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= g.n) return;
    unsigned long long slot[SLOTS];
#pragma unroll
    for (int c = 0; c < SLOTS; ++c) {
        slot[c] = 0;
        if (c < g.ncols)
            slot[c] = g.width[c] == 8 ? ldg_stream(static_cast<const unsigned long long*>(g.src[c]) + r)
                                      : (unsigned long long)ldg_stream(static_cast<const uint32_t*>(g.src[c]) + r);
    }
    ulonglong2* dst = reinterpret_cast<ulonglong2*>(recs + r * REC);
#pragma unroll
    for (int c = 0; c < SLOTS; c += 2) dst[c / 2] = make_ulonglong2(slot[c], slot[c + 1]);
}

// One record's 8-byte slots (records start at multiples of REC; 32- and
// 64-byte records are 32-byte aligned, 16- and 48-byte ones 16-byte aligned).
template <int REC>
__device__ __forceinline__ void load_record(const unsigned char* rec, unsigned long long (&slot)[REC / 8]) {
    if constexpr (REC % 32 == 0) {
#pragma unroll
        for (int c = 0; c < REC / 8; c += 4) {
            unsigned long long v[4];
            ld_rand32(rec + 8 * c, v);
            slot[c] = v[0];
            slot[c + 1] = v[1];
            slot[c + 2] = v[2];
            slot[c + 3] = v[3];
        }
    } else {
#pragma unroll
        for (int c = 0; c < REC / 8; c += 2) {
            const ulonglong2 v = ld_rand16(rec + 8 * c);
            slot[c] = v.x;
            slot[c + 1] = v.y;
        }
    }
}

template <int REC>
__global__ void __launch_bounds__(256) k_gather_rec(GatherArgs g, const unsigned char* recs) {
    constexpr int SLOTS = REC / 8;
    const uint64_t r = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= g.n) return;
    uint32_t p = ldg_stream(g.perm + r);
    if (p >= g.n) {  // not a permutation of [0, n)
        if (g.err) atomicOr(g.err, ERR_BAD_INDEX);
        p = 0;
    }
    unsigned long long slot[SLOTS];
    load_record<REC>(recs + (uint64_t)p * REC, slot);
#pragma unroll
    for (int c = 0; c < SLOTS; ++c) {
        if (c >= g.ncols) break;
        if (g.width[c] == 8) stg_stream(static_cast<unsigned long long*>(g.dst[c]) + r, slot[c]);
        else stg_stream(static_cast<uint32_t*>(g.dst[c]) + r, (uint32_t)slot[c]);
    }
}

// Four consecutive output rows per thread: one 16-byte load of their row ids,
// then all their record reads issued back to back (four times the random
// reads in flight per thread of k_gather_rec: the reads are latency-bound
// when the records span gigabytes), then 16/32-byte stores per column.
// Needs perm and every output column 16-byte aligned.
template <int REC>
__global__ void __launch_bounds__(256) k_gather_rec4(GatherArgs g, const unsigned char* recs) {
    constexpr int SLOTS = REC / 8;
    const uint64_t r0 = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) * 4;
    if (r0 >= g.n) return;
    if (r0 + 4 <= g.n) {
        uint4 p4 = ldg_stream(reinterpret_cast<const uint4*>(g.perm + r0));
        uint32_t p[4] = {p4.x, p4.y, p4.z, p4.w};
#pragma unroll
        for (int k = 0; k < 4; ++k)
            if (p[k] >= g.n) {  // not a permutation of [0, n)
                if (g.err) atomicOr(g.err, ERR_BAD_INDEX);
                p[k] = 0;
            }
        unsigned long long slot[4][SLOTS];
#pragma unroll
        for (int k = 0; k < 4; ++k) load_record<REC>(recs + (uint64_t)p[k] * REC, slot[k]);
#pragma unroll
        for (int c = 0; c < SLOTS; ++c) {
            if (c >= g.ncols) break;
            if (g.width[c] == 8) {
                ulonglong2* d = reinterpret_cast<ulonglong2*>(static_cast<unsigned long long*>(g.dst[c]) + r0);
                stg_stream(d, make_ulonglong2(slot[0][c], slot[1][c]));
                stg_stream(d + 1, make_ulonglong2(slot[2][c], slot[3][c]));
            } else {
                uint4 v = make_uint4((uint32_t)slot[0][c], (uint32_t)slot[1][c], (uint32_t)slot[2][c],
                                     (uint32_t)slot[3][c]);
                stg_stream(reinterpret_cast<uint4*>(static_cast<uint32_t*>(g.dst[c]) + r0), v);
            }
        }
        return;
    }
    for (uint64_t r = r0; r < g.n; ++r) {
        uint32_t p = ldg_stream(g.perm + r);
        if (p >= g.n) {
            if (g.err) atomicOr(g.err, ERR_BAD_INDEX);
            p = 0;
        }
        unsigned long long slot[SLOTS];
        load_record<REC>(recs + (uint64_t)p * REC, slot);
#pragma unroll
        for (int c = 0; c < SLOTS; ++c) {
            if (c >= g.ncols) break;
            if (g.width[c] == 8) stg_stream(static_cast<unsigned long long*>(g.dst[c]) + r, slot[c]);
            else stg_stream(static_cast<uint32_t*>(g.dst[c]) + r, (uint32_t)slot[c]);
        }
    }
}

namespace {
bool aligned16(const GatherArgs& g) {
    bool ok = (reinterpret_cast<uintptr_t>(g.perm) & 15) == 0;
    for (int c = 0; c < g.ncols; ++c) ok = ok && (reinterpret_cast<uintptr_t>(g.dst[c]) & 15) == 0;
    return ok;
}

cudaError_t launch_gather_rec(const GatherArgs& g, const unsigned char* recs, size_t rec, cudaStream_t s) {
    if (aligned16(g)) {
        const uint32_t blocks = (uint32_t)(((g.n + 3) / 4 + 255) / 256);
        switch (rec) {
        case 16: k_gather_rec4<16><<<blocks, 256, 0, s>>>(g, recs); break;
        case 32: k_gather_rec4<32><<<blocks, 256, 0, s>>>(g, recs); break;
        case 48: k_gather_rec4<48><<<blocks, 256, 0, s>>>(g, recs); break;
        default: k_gather_rec4<64><<<blocks, 256, 0, s>>>(g, recs); break;
        }
    } else {
        const uint32_t blocks = (uint32_t)((g.n + 255) / 256);
        switch (rec) {
        case 16: k_gather_rec<16><<<blocks, 256, 0, s>>>(g, recs); break;
        case 32: k_gather_rec<32><<<blocks, 256, 0, s>>>(g, recs); break;
        case 48: k_gather_rec<48><<<blocks, 256, 0, s>>>(g, recs); break;
        default: k_gather_rec<64><<<blocks, 256, 0, s>>>(g, recs); break;
        }
    }
    return cudaGetLastError();
}
}  // namespace

size_t gather_record_bytes(int ncols) {
    return (ncols >= 2 && ncols <= kMaxGather) ? (size_t)16 * ((ncols + 1) / 2) : 0;
}

cudaError_t run_gather(const GatherArgs& g, cudaStream_t s, Profiler* prof, void* rec_ws, size_t rec_ws_bytes,
                       int* launches) {
    if (g.n == 0 || g.ncols == 0) return cudaSuccess;
    const size_t rec = gather_record_bytes(g.ncols);
    if (rec_ws && rec && rec_ws_bytes / rec >= g.n) {
        unsigned char* recs = static_cast<unsigned char*>(rec_ws);
        const uint32_t blocks = (uint32_t)((g.n + 255) / 256);
        if (prof) prof->begin(KC_PACK, s);
        switch (rec) {
        case 16: k_pack<16><<<blocks, 256, 0, s>>>(g, recs); break;
        case 32: k_pack<32><<<blocks, 256, 0, s>>>(g, recs); break;
        case 48: k_pack<48><<<blocks, 256, 0, s>>>(g, recs); break;
        default: k_pack<64><<<blocks, 256, 0, s>>>(g, recs); break;
        }
        if (prof) prof->end(KC_PACK, s);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
        if (prof) prof->begin(KC_GATHER, s);
        e = launch_gather_rec(g, recs, rec, s);
        if (prof) prof->end(KC_GATHER, s);
        if (launches) *launches += 2;
        return e;
    }
    if (launches) *launches += 1;
    bool vec = (reinterpret_cast<uintptr_t>(g.perm) & 15) == 0;
    for (int c = 0; c < g.ncols; ++c) vec = vec && (reinterpret_cast<uintptr_t>(g.dst[c]) & 15) == 0;
    const uint64_t threads = (g.n + 3) / 4;
    const uint32_t blocks = (uint32_t)((threads + 255) / 256);
    if (prof) prof->begin(KC_GATHER, s);
    if (vec) k_gather<true><<<blocks, 256, 0, s>>>(g);
    else k_gather<false><<<blocks, 256, 0, s>>>(g);
    if (prof) prof->end(KC_GATHER, s);
    return cudaGetLastError();
}

cudaError_t run_gather_records(const GatherArgs& g, const void* recs, size_t rec_bytes, cudaStream_t s, Profiler* prof,
                               int* launches) {
    if (g.n == 0 || g.ncols == 0) return cudaSuccess;
    if (rec_bytes != gather_record_bytes(g.ncols)) return cudaErrorInvalidValue;
    const unsigned char* r = static_cast<const unsigned char*>(recs);
    if (prof) prof->begin(KC_GATHER, s);
    cudaError_t e = launch_gather_rec(g, r, rec_bytes, s);
    if (prof) prof->end(KC_GATHER, s);
    if (launches) *launches += 1;
    return e;
}

template <int W>
__global__ void __launch_bounds__(256) k_broadcast(const uint32_t* row_group, uint64_t n, const void* gvals,
                                                   uint64_t n_groups, const uint32_t* perm, void* out,
                                                   uint32_t* err) {
    using T = typename std::conditional<W == 8, unsigned long long, uint32_t>::type;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t r = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; r < n; r += stride) {
        const uint32_t g = row_group[r];
        const uint64_t dst = perm ? perm[r] : r;
        if (g >= n_groups || dst >= n) {
            atomicOr(err, ERR_BAD_INDEX);
            continue;
        }
        static_cast<T*>(out)[dst] = __ldcg(static_cast<const T*>(gvals) + g);
    }
}

cudaError_t run_broadcast(const uint32_t* row_group, uint64_t n, const void* group_vals, uint64_t n_groups,
                          int width, const uint32_t* perm, void* out, uint32_t* err, cudaStream_t s,
                          Profiler* prof) {
    if (n == 0) return cudaSuccess;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    uint64_t want = (n + 255) / 256;
    uint32_t blocks = (uint32_t)(want < (uint64_t)sms * 16 ? want : (uint64_t)sms * 16);
    if (prof) prof->begin(KC_BROADCAST, s);
    if (width == 8) k_broadcast<8><<<blocks, 256, 0, s>>>(row_group, n, group_vals, n_groups, perm, out, err);
    else k_broadcast<4><<<blocks, 256, 0, s>>>(row_group, n, group_vals, n_groups, perm, out, err);
    if (prof) prof->end(KC_BROADCAST, s);
    return cudaGetLastError();
}

}  // namespace vdf
