// vdf_pivot.cu -- pivot: the sum of a value column per (col key, row key)
// pair of two string columns, reshaped into a matrix with one column per
// distinct col key and one row per distinct row key, both in order of first
// appearance, as the reference's pivot (pivots/pivot.hpp:5-128) returns it.
//
// The reference walks the rows once with three hash maps (col key -> index,
// row key -> index, (col, row) -> sum).  Here each key column is first
// dictionary-encoded on the device, then the pairs go through the sorted
// group-by:
//   1. k_dict_insert  every row's string into an open-addressing table of
//                     2^k >= 2n slots (hash of the bytes, linear probing,
//                     byte-wise comparison against the slot's row); a slot
//                     keeps the smallest row of its string (atomicMin), i.e.
//                     the string's first appearance;
//   2. k_dict_flag    marks each distinct string's first row;
//   3. a three-kernel exclusive scan of the marks gives each first row its
//      rank in row order = the key's first-appearance index, which
//      k_dict_code hands to every row of the key;
//   4. the 64-bit pair code (col index << 32 | row index) is sorted with the
//      value column as payload and summed per group (the library's sort +
//      group-by: exact integer sums, compensated f64 sums);
//   5. k_pivot_scatter writes each pair's sum into its cell of the
//      zero-initialised matrix, column after column.
#include <cstdint>

#include "vdf_common.cuh"
#include "vdf_ctx.h"
#include "vdf_internal.h"

namespace vdf {
namespace {

constexpr uint32_t kEmpty = 0xffffffffu;
constexpr uint32_t kScanBlock = 2048;  // marks per block of the scan

uint32_t grid_for_rows(uint64_t n) {
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const uint64_t want = (n + 255) / 256;
    const uint64_t cap = (uint64_t)sms * 8;
    return (uint32_t)(want < cap ? (want ? want : 1) : cap);
}

__device__ __forceinline__ uint64_t str_hash(const unsigned char* s, uint64_t len) {
    uint64_t h = 1469598103934665603ull;  // FNV-1a over the bytes
    for (uint64_t i = 0; i < len; ++i) h = (h ^ s[i]) * 1099511628211ull;
    return h ^ (h >> 29);
}

__device__ __forceinline__ bool str_eq(const unsigned char* bytes, const uint64_t* offs, uint32_t a, uint32_t b) {
    const uint64_t la = offs[a + 1] - offs[a], lb = offs[b + 1] - offs[b];
    if (la != lb) return false;
    const unsigned char* pa = bytes + offs[a];
    const unsigned char* pb = bytes + offs[b];
    for (uint64_t i = 0; i < la; ++i)
        if (pa[i] != pb[i]) return false;
    return true;
}

// Each row's string into the table; slot_of_row[r] = its slot.
__global__ void __launch_bounds__(256) k_dict_insert(const unsigned char* bytes, const uint64_t* offs, uint32_t n,
                                                     uint64_t total, uint32_t* table, uint32_t mask,
                                                     uint32_t* slot_of_row, uint32_t* err) {
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += stride) {
        const uint64_t b = offs[r], e = offs[r + 1];
        if (b > e || e > total) {  // offsets must be non-decreasing and within the bytes
            atomicOr(err, ERR_BAD_INDEX);
            slot_of_row[r] = 0;
            continue;
        }
        uint32_t s = (uint32_t)str_hash(bytes + b, e - b) & mask;
        bool placed = false;
        for (uint32_t probe = 0; probe <= mask; ++probe) {  // at most every slot once
            uint32_t cur = ld_relaxed_u32(table + s);
            if (cur == kEmpty) {
                cur = atomicCAS(table + s, kEmpty, r);
                if (cur == kEmpty) {
                    placed = true;
                    break;
                }
            }
            if (str_eq(bytes, offs, cur, r)) {  // any row of the string compares the same
                atomicMin(table + s, r);
                placed = true;
                break;
            }
            s = (s + 1) & mask;
        }
        if (!placed) atomicOr(err, ERR_BAD_INDEX);  // never: the table has more slots than rows
        slot_of_row[r] = s;
    }
}

// mark[first row of each distinct string] = 1 (the marks start zeroed)
__global__ void __launch_bounds__(256) k_dict_flag(const uint32_t* table, uint32_t slots, uint32_t n,
                                                   uint32_t* mark) {
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < slots; s += stride) {
        const uint32_t r = table[s];
        if (r != kEmpty && r < n) mark[r] = 1;
    }
}

// ---- exclusive scan of the marks: per-block sums, one CTA over the sums,
//      then each block again with its offset
__global__ void __launch_bounds__(256) k_scan_sums(const uint32_t* mark, uint32_t n, uint32_t* sums) {
    const uint64_t b0 = (uint64_t)blockIdx.x * kScanBlock;
    uint32_t v = 0;
    for (uint32_t i = threadIdx.x; i < kScanBlock; i += 256)
        if (b0 + i < n) v += mark[b0 + i];
    v = __reduce_add_sync(0xffffffffu, v);
    __shared__ uint32_t w[8];
    if ((threadIdx.x & 31) == 0) w[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t t = 0;
        for (int i = 0; i < 8; ++i) t += w[i];
        sums[blockIdx.x] = t;
    }
}

__global__ void __launch_bounds__(1024) k_scan_top(uint32_t* sums, uint32_t nblocks, uint32_t* total) {
    __shared__ uint32_t wsum[32];
    __shared__ uint32_t carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (uint32_t base = 0; base < nblocks; base += 1024) {
        const uint32_t i = base + threadIdx.x;
        const uint32_t v = i < nblocks ? sums[i] : 0;
        uint32_t incl = v;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const uint32_t t = __shfl_up_sync(0xffffffffu, incl, d);
            if (lane >= d) incl += t;
        }
        if (lane == 31) wsum[warp] = incl;
        __syncthreads();
        uint32_t wb = 0, all = 0;
        for (int k = 0; k < 32; ++k) {
            wb += k < warp ? wsum[k] : 0u;
            all += wsum[k];
        }
        const uint32_t c = carry;
        if (i < nblocks) sums[i] = c + wb + incl - v;
        __syncthreads();
        if (threadIdx.x == 0) carry = c + all;
        __syncthreads();
    }
    if (threadIdx.x == 0) *total = carry;
}

// rank[r] = marks before row r (only the marked rows' ranks are used)
__global__ void __launch_bounds__(256) k_scan_apply(const uint32_t* mark, uint32_t n, const uint32_t* sums,
                                                    uint32_t* rank) {
    const uint64_t b0 = (uint64_t)blockIdx.x * kScanBlock;
    constexpr int PER = kScanBlock / 256;
    uint32_t v[PER];
    uint32_t t = 0;
#pragma unroll
    for (int j = 0; j < PER; ++j) {
        const uint64_t i = b0 + (uint64_t)threadIdx.x * PER + j;
        v[j] = i < n ? mark[i] : 0;
        t += v[j];
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t incl = t;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const uint32_t x = __shfl_up_sync(0xffffffffu, incl, d);
        if (lane >= d) incl += x;
    }
    __shared__ uint32_t wsum[8];
    if (lane == 31) wsum[warp] = incl;
    __syncthreads();
    uint32_t run = sums[blockIdx.x] + incl - t;
    for (int k = 0; k < warp; ++k) run += wsum[k];
#pragma unroll
    for (int j = 0; j < PER; ++j) {
        const uint64_t i = b0 + (uint64_t)threadIdx.x * PER + j;
        if (i < n && v[j]) rank[i] = run;
        run += v[j];
    }
}

// code[r] = first-appearance index of row r's key; first_row[index] = its first row
__global__ void __launch_bounds__(256) k_dict_code(const uint32_t* table, const uint32_t* slot_of_row,
                                                   const uint32_t* rank, uint32_t n, uint32_t slots, uint32_t* code,
                                                   uint32_t* first_row, uint32_t* err) {
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += stride) {
        const uint32_t s = slot_of_row[r];
        const uint32_t f = s < slots ? table[s] : kEmpty;
        if (f >= n) {  // never for a consistent table
            atomicOr(err, ERR_BAD_INDEX);
            code[r] = 0;
            continue;
        }
        const uint32_t c = rank[f];
        code[r] = c;
        if (f == r) first_row[c] = r;
    }
}

__global__ void __launch_bounds__(256) k_pair_code(const uint32_t* col_code, const uint32_t* row_code, uint32_t n,
                                                   unsigned long long* pair) {
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += stride)
        pair[r] = ((unsigned long long)col_code[r] << 32) | row_code[r];
}

// matrix[c * nrows + r] = the sum of pair (c, r), in the value type
__global__ void __launch_bounds__(256) k_pivot_scatter(const unsigned long long* pair, const void* sum, uint64_t g,
                                                       int dt, uint32_t ncols, uint32_t nrows, void* matrix,
                                                       uint32_t* err) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < g; i += stride) {
        const uint32_t c = (uint32_t)(pair[i] >> 32), r = (uint32_t)pair[i];
        if (c >= ncols || r >= nrows) {
            atomicOr(err, ERR_BAD_INDEX);
            continue;
        }
        const uint64_t cell = (uint64_t)c * nrows + r;
        // integer sums: the low bits of the exact sum are the value type's
        // wrapped sum; f64: the compensated sum
        const uint64_t bits = static_cast<const unsigned long long*>(sum)[i];
        if (dt == VDF_I32 || dt == VDF_U32) static_cast<uint32_t*>(matrix)[cell] = (uint32_t)bits;
        else static_cast<unsigned long long*>(matrix)[cell] = bits;
    }
}

}  // namespace
}  // namespace vdf

using namespace vdfc;

namespace {

// Dictionary codes of one string column (device pointers into the staging
// buffer); *count = distinct strings.
vdf_status encode(vdf_ctx* c, const unsigned char* bytes, const uint64_t* offs, uint64_t total, uint32_t n,
                  uint32_t* table, uint32_t slots, uint32_t* slot_of_row, uint32_t* mark, uint32_t* sums,
                  uint32_t* rank, uint32_t* code, uint32_t* first_row, uint32_t* count_dev, uint32_t* count,
                  cudaStream_t s) {
    using namespace vdf;
    const uint32_t grid = grid_for_rows(n);
    const uint32_t nblocks = (n + kScanBlock - 1) / kScanBlock;
    cudaError_t e = cudaMemsetAsync(table, 0xff, (size_t)slots * 4, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(mark, 0, (size_t)n * 4, s);
    if (e != cudaSuccess) return from_cuda(c, e, "pivot dictionary");
    k_dict_insert<<<grid, 256, 0, s>>>(bytes, offs, n, total, table, slots - 1, slot_of_row, err_word(c));
    k_dict_flag<<<grid_for_rows(slots), 256, 0, s>>>(table, slots, n, mark);
    k_scan_sums<<<nblocks, 256, 0, s>>>(mark, n, sums);
    k_scan_top<<<1, 1024, 0, s>>>(sums, nblocks, count_dev);
    k_scan_apply<<<nblocks, 256, 0, s>>>(mark, n, sums, rank);
    k_dict_code<<<grid, 256, 0, s>>>(table, slot_of_row, rank, n, slots, code, first_row, err_word(c));
    c->launches += 6;
    if ((e = cudaGetLastError()) != cudaSuccess) return from_cuda(c, e, "pivot dictionary");
    if ((e = cudaMemcpyAsync(count, count_dev, 4, cudaMemcpyDeviceToHost, s)) != cudaSuccess)
        return from_cuda(c, e, "pivot dictionary");
    return VDF_OK;
}

}  // namespace

extern "C" {

vdf_status vdf_pivot_host(vdf_ctx* c, uint64_t n, vdf_strcol col_key, vdf_strcol row_key, vdf_col value,
                          uint32_t* n_colkeys, uint32_t* n_rowkeys, uint32_t* colkey_row, uint32_t* rowkey_row,
                          void* matrix, uint64_t matrix_cap) {
    if (!c || !n_colkeys || !n_rowkeys) return VDF_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> lk(c->mu);
    *n_colkeys = *n_rowkeys = 0;
    if (n > kMaxRows) return fail(c, VDF_ERR_INVALID_ARG, "%llu rows exceed the row limit", (unsigned long long)n);
    const int dt = value.dtype;
    if (dt != VDF_I32 && dt != VDF_U32 && dt != VDF_I64 && dt != VDF_U64 && dt != VDF_F64)
        return fail(c, VDF_ERR_UNSUPPORTED, "pivot values: int32, uint32, int64, uint64 or float64 (got %d)", dt);
    if (n == 0) return VDF_OK;
    if (!col_key.bytes || !col_key.offsets || !row_key.bytes || !row_key.offsets || !value.data || !colkey_row ||
        !rowkey_row)
        return fail(c, VDF_ERR_INVALID_ARG, "NULL column or output");
    const uint32_t rows = (uint32_t)n;
    const uint64_t cbytes = col_key.offsets[n], rbytes = row_key.offsets[n];
    if (col_key.offsets[0] != 0 || row_key.offsets[0] != 0)
        return fail(c, VDF_ERR_INVALID_ARG, "string offsets must start at 0");
    uint32_t slots = 16;
    while (slots < 2 * rows + 2) slots <<= 1;
    const size_t w = (size_t)vdf::dtype_width(dt);
    const uint32_t nblocks = (rows + vdf::kScanBlock - 1) / vdf::kScanBlock;
    // staging layout
    size_t off = 0;
    auto take = [&](size_t bytes) { size_t o = off; off = align256(off + bytes); return o; };
    const size_t o_cb = take(cbytes + 1), o_co = take(8 * (n + 1)), o_rb = take(rbytes + 1), o_ro = take(8 * (n + 1));
    const size_t o_val = take(w * n), o_table = take(4 * (size_t)slots), o_slot = take(4 * n), o_mark = take(4 * n);
    const size_t o_sums = take(4 * (size_t)nblocks + 4), o_rank = take(4 * n), o_ccode = take(4 * n);
    const size_t o_rcode = take(4 * n), o_cfirst = take(4 * n), o_rfirst = take(4 * n), o_cnt = take(16);
    const size_t o_pair = take(8 * n), o_gkey = take(8 * n), o_sum = take(8 * n), o_ng = take(8);
    vdf_status st = io_ensure(c, off);
    if (st != VDF_OK) return st;
    DeviceGuard g(c->device);
    unsigned char* io = c->io;
    auto at = [&](size_t o) { return io + o; };
    auto u32 = [&](size_t o) { return reinterpret_cast<uint32_t*>(io + o); };
    cudaStream_t s = nullptr;
    cudaError_t e = cudaMemcpyAsync(at(o_cb), col_key.bytes, cbytes, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(at(o_co), col_key.offsets, 8 * (n + 1), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(at(o_rb), row_key.bytes, rbytes, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(at(o_ro), row_key.offsets, 8 * (n + 1), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(at(o_val), value.data, w * n, cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) return from_cuda(c, e, "copy pivot inputs to the device");
    uint32_t* counts = reinterpret_cast<uint32_t*>(c->host_pinned + 4);  // the key counts (pinned)
    if ((st = encode(c, at(o_cb), reinterpret_cast<const uint64_t*>(at(o_co)), cbytes, rows, u32(o_table), slots,
                     u32(o_slot), u32(o_mark), u32(o_sums), u32(o_rank), u32(o_ccode), u32(o_cfirst), u32(o_cnt),
                     &counts[0], s)) != VDF_OK)
        return st;
    if ((st = encode(c, at(o_rb), reinterpret_cast<const uint64_t*>(at(o_ro)), rbytes, rows, u32(o_table), slots,
                     u32(o_slot), u32(o_mark), u32(o_sums), u32(o_rank), u32(o_rcode), u32(o_rfirst),
                     u32(o_cnt) + 1, &counts[1], s)) != VDF_OK)
        return st;
    vdf::k_pair_code<<<vdf::grid_for_rows(rows), 256, 0, s>>>(u32(o_ccode), u32(o_rcode), rows,
                                                              reinterpret_cast<unsigned long long*>(at(o_pair)));
    c->launches += 1;
    if ((e = cudaGetLastError()) != cudaSuccess) return from_cuda(c, e, "pivot pair codes");
    // sum per pair on the sorted path
    vdf_col key{at(o_pair), VDF_U64};
    vdf_col pay{at(o_val), dt};
    int32_t agg_col = 0;
    vdf_agg_out agg{at(o_sum), nullptr, nullptr, nullptr, nullptr};
    void* gk = at(o_gkey);
    uint64_t groups = 0;
    vdf_sort_groupby_args a{};
    a.n = n;
    a.keys = &key;
    a.nkeys = 1;
    a.order = VDF_ORDER_ASC;
    a.payload = &pay;
    a.npayload = 1;
    a.groupby = 1;
    a.agg_cols = &agg_col;
    a.nagg = 1;
    a.group_keys_out = &gk;
    a.aggs = &agg;
    a.n_groups_dev = reinterpret_cast<uint64_t*>(at(o_ng));
    a.n_groups_host = &groups;  // synchronises the stream: the key counts are in too
    if ((st = sort_groupby_device(c, &a, s)) != VDF_OK) return st;
    *n_colkeys = counts[0];
    *n_rowkeys = counts[1];
    if ((st = drain_and_check(c, s)) != VDF_OK) return st;
    e = cudaMemcpyAsync(colkey_row, u32(o_cfirst), 4 * (size_t)counts[0], cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(rowkey_row, u32(o_rfirst), 4 * (size_t)counts[1], cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return from_cuda(c, e, "copy pivot keys to the host");
    const uint64_t cells = (uint64_t)counts[0] * counts[1];
    if (!matrix || cells > matrix_cap)
        return fail(c, VDF_ERR_WORKSPACE, "the pivot matrix has %llu cells, the buffer %llu",
                    (unsigned long long)cells, (unsigned long long)matrix_cap);
    // the matrix: behind the staged columns when it fits there, else in a
    // buffer of its own for this call
    const size_t o_mat = off;
    void* dmat = nullptr;
    bool own = false;
    if (o_mat + cells * w <= c->io_cap) {
        dmat = io + o_mat;
    } else if (cudaMalloc(&dmat, cells * w) == cudaSuccess) {
        own = true;
    } else {
        cudaGetLastError();
        return fail(c, VDF_ERR_OOM, "pivot matrix of %llu bytes", (unsigned long long)(cells * w));
    }
    e = cudaMemsetAsync(dmat, 0, cells * w, s);
    if (e == cudaSuccess && groups) {
        vdf::k_pivot_scatter<<<vdf::grid_for_rows(groups), 256, 0, s>>>(
            reinterpret_cast<const unsigned long long*>(io + o_gkey), io + o_sum, groups, dt, counts[0], counts[1],
            dmat, err_word(c));
        c->launches += 1;
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(matrix, dmat, cells * w, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (own) cudaFree(dmat);
    if (e != cudaSuccess) return from_cuda(c, e, "pivot matrix");
    return drain_and_check(c, s);
}

}  // extern "C"
