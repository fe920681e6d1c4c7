// vdf_csv.cu -- CSV ingest into device-resident columns: the reference's
// read_csv (V/read/read_csv/read_csv.hpp:3-216) with its single-core parser
// (V/inlines/read/read_csv/standard_parser/standard_parser.inl:1-72 ->
// parsers_core/parse_rows_chunk.inl:1-185) and type inference
// (type_inference/type_classification.inl:1-177 -> inlines/classify_column.inl).
//
// Device pipeline over the file bytes in HBM (positions are 32-bit, files
// below 4 GiB):
//   1. k_csv_count: each thread takes 64 bytes, builds bit masks of quote,
//      CR and LF bytes (SWAR zero-byte tests), the in-quote state as a prefix XOR of
//      the quote mask, and counts record terminators outside quotes (a CR, or
//      an LF not right after a CR) for both possible starting states; per
//      16 KB tile: quote parity and the two counts;
//   2. k_csv_scan: one CTA scans the tiles: in-quote state at each tile start
//      and the first record index of each tile;
//   3. k_csv_records: the same masks again, now with the known state, write
//      each record's terminator position;
//   4. the host reads the first rows back and classifies the columns
//      (classify_column's rules on the first 10 values);
//   5. k_csv_parse: one thread per record walks its fields (quote toggling,
//      delimiter splits, as parse_rows_chunk does) and converts each field by
//      its column's type (vdf_decimal.cuh); every lane of a warp works on the
//      same column at a time, so the type branch is uniform and the column
//      writes are coalesced; string fields record their start and length;
//   6. strings: an offset scan per string column, then k_csv_strings copies
//      the bytes.
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "vdf_ctx.h"
#include "vdf_decimal.cuh"

using namespace vdfc;

struct vdf_csv {
    int device = 0;
    uint64_t nrow = 0;
    uint32_t ncol = 0;
    std::vector<std::string> names;
    std::vector<char> types;
    std::vector<void*> values;        // device: f64 / u32 / u8 values, or string bytes
    std::vector<uint64_t*> offsets;   // device: nrow + 1 string offsets (strings only)
    std::vector<uint64_t> str_bytes;  // string bytes per column
    unsigned char* block = nullptr;   // numeric values + offsets + start arrays
    unsigned char* sblock = nullptr;  // string bytes
    bool pooled = false, spooled = false;  // from the stream-ordered pool (else cudaMalloc)
};

namespace {

constexpr int kThreads = 256;
constexpr int kChunk = 64;  // bytes per thread in the split passes: 16 KB tiles of kThreads threads

// Top bit of each byte of w set exactly where that byte equals the byte of
// `pat` (x = w ^ pat is zero there): adding 0x7f to the low seven bits sets
// the top bit of every byte whose low bits are nonzero and never carries
// into the next byte.
__device__ __forceinline__ uint32_t eq_bytes(uint32_t w, uint32_t pat) {
    const uint32_t x = w ^ pat;
    return ~(((x & 0x7f7f7f7fu) + 0x7f7f7f7fu) | x | 0x7f7f7f7fu);
}

__device__ __forceinline__ uint32_t nibble(uint32_t top) {
    // the top bits of the four bytes (only those set) -> four bits; the
    // products land on distinct bit positions, so no carries
    return (top * 0x00204081u) >> 28;
}

__device__ __forceinline__ uint64_t prefix_xor(uint64_t x) {
    x ^= x << 1;
    x ^= x << 2;
    x ^= x << 4;
    x ^= x << 8;
    x ^= x << 16;
    x ^= x << 32;
    return x;
}

struct Masks {
    uint64_t quote;  // quote bytes
    uint64_t term;   // record terminator candidates (CR, or LF not after CR)
    uint64_t ev;     // field end candidates: terminators and delimiters
};

// Masks of the 64 bytes at `base` restricted to [start, n).
__device__ __forceinline__ Masks chunk_masks(const uint8_t* __restrict__ buf, uint64_t n, uint64_t start,
                                             uint64_t base, uint32_t quote4, uint32_t delim4) {
    uint32_t w[16];
    if (base + kChunk <= n) {
        const uint4* p = reinterpret_cast<const uint4*>(buf + base);
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const uint4 v = __ldg(p + k);
            w[4 * k] = v.x;
            w[4 * k + 1] = v.y;
            w[4 * k + 2] = v.z;
            w[4 * k + 3] = v.w;
        }
    } else {
#pragma unroll
        for (int k = 0; k < 16; ++k) {
            uint32_t x = 0;
            for (int b = 0; b < 4; ++b) {
                const uint64_t i = base + 4 * k + b;
                if (i < n) x |= (uint32_t)__ldg(buf + i) << (8 * b);
            }
            w[k] = x;
        }
    }
    uint64_t q = 0, cr = 0, lf = 0, dl = 0;
#pragma unroll
    for (int k = 0; k < 16; ++k) {
        q |= (uint64_t)nibble(eq_bytes(w[k], quote4)) << (4 * k);
        dl |= (uint64_t)nibble(eq_bytes(w[k], delim4)) << (4 * k);
        cr |= (uint64_t)nibble(eq_bytes(w[k], 0x0d0d0d0du)) << (4 * k);
        lf |= (uint64_t)nibble(eq_bytes(w[k], 0x0a0a0a0au)) << (4 * k);
    }
    uint64_t valid = ~0ull;
    if (start > base) valid = (start - base >= 64) ? 0 : (~0ull << (start - base));
    if (n < base + 64) valid &= (n <= base) ? 0 : (~0ull >> (64 - (n - base)));
    const bool prev_cr = base > start && base - 1 < n && __ldg(buf + base - 1) == '\r';
    q &= valid;
    cr &= valid;
    lf &= valid;
    const uint64_t after_cr = (cr << 1) | (prev_cr ? 1ull : 0ull);
    Masks m;
    m.quote = q;
    m.term = cr | (lf & ~after_cr);
    m.ev = m.term | (dl & valid);
    return m;
}

__device__ __forceinline__ uint32_t lanemask_lt() {
    uint32_t m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

// Block-wide exclusive XOR of one bit per thread; also returns the total.
__device__ __forceinline__ uint32_t block_xor_excl(uint32_t bit, uint32_t* s_w, uint32_t& total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const uint32_t bal = __ballot_sync(0xffffffffu, bit);
    uint32_t pre = __popc(bal & lanemask_lt()) & 1u;
    if (lane == 0) s_w[warp] = __popc(bal) & 1u;
    __syncthreads();
    uint32_t wp = 0, tot = 0;
    for (int i = 0; i < nw; ++i) {
        if (i < warp) wp ^= s_w[i];
        tot ^= s_w[i];
    }
    __syncthreads();
    total = tot;
    return pre ^ wp;
}

// Block-wide exclusive sum of a u32 per thread; also returns the total.
__device__ __forceinline__ uint32_t block_sum_excl(uint32_t v, uint32_t* s_w, uint32_t& total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    uint32_t x = v;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, x, d);
        if (lane >= d) x += y;
    }
    if (lane == 31) s_w[warp] = x;
    __syncthreads();
    uint32_t wp = 0, tot = 0;
    for (int i = 0; i < nw; ++i) {
        if (i < warp) wp += s_w[i];
        tot += s_w[i];
    }
    __syncthreads();
    total = tot;
    return wp + x - v;
}

// Pass 1: per tile {quote parity, field ends if the tile starts outside
// quotes, field ends if it starts inside}.
__global__ void __launch_bounds__(kThreads) k_csv_count(const uint8_t* __restrict__ buf, uint64_t n, uint64_t start,
                                                        uint32_t quote4, uint32_t delim4,
                                                        uint32_t* __restrict__ tiles) {
    __shared__ uint32_t s_w[kThreads / 32];
    const uint64_t base = ((uint64_t)blockIdx.x * kThreads + threadIdx.x) * kChunk;
    const Masks m = chunk_masks(buf, n, start, base, quote4, delim4);
    const uint64_t px = prefix_xor(m.quote);  // bit i: quotes in [base, i] odd
    const uint32_t c_out = __popcll(m.ev & ~px), c_in = __popcll(m.ev & px);
    uint32_t par_total;
    const uint32_t pre = block_xor_excl(__popcll(m.quote) & 1u, s_w, par_total);
    uint32_t t0, t1;
    block_sum_excl(pre ? c_in : c_out, s_w, t0);
    block_sum_excl(pre ? c_out : c_in, s_w, t1);
    if (threadIdx.x == 0) {
        tiles[3 * blockIdx.x] = par_total;
        tiles[3 * blockIdx.x + 1] = t0;
        tiles[3 * blockIdx.x + 2] = t1;
    }
}

// Pass 2 (one CTA): tile start states and first record indices; total count.
__global__ void __launch_bounds__(1024) k_csv_scan(const uint32_t* __restrict__ tiles, uint32_t ntiles,
                                                   uint32_t* __restrict__ tile_state, uint32_t* __restrict__ tile_first,
                                                   uint32_t* __restrict__ total) {
    __shared__ uint32_t s_w[32];
    uint32_t state = 0, first = 0;
    for (uint32_t b = 0; b < ntiles; b += blockDim.x) {
        const uint32_t t = b + threadIdx.x;
        const uint32_t par = t < ntiles ? tiles[3 * t] : 0;
        uint32_t ptot;
        const uint32_t st = state ^ block_xor_excl(par, s_w, ptot);
        const uint32_t cnt = t < ntiles ? (st ? tiles[3 * t + 2] : tiles[3 * t + 1]) : 0;
        uint32_t ctot;
        const uint32_t off = first + block_sum_excl(cnt, s_w, ctot);
        if (t < ntiles) {
            tile_state[t] = st;
            tile_first[t] = off;
        }
        state ^= ptot;
        first += ctot;
    }
    if (threadIdx.x == 0) *total = first;
}

// Pass 3: write each field end's position (delimiter or record terminator
// outside quotes).  Field f belongs to record f / ncol and must end in a
// terminator exactly when f % ncol == ncol - 1; the first record that breaks
// this is the "column number problem" row.  The thread holding the last
// field end records where the bytes after it start (or ~0 after a
// delimiter: the final record then has no terminator).
__global__ void __launch_bounds__(kThreads) k_csv_fields(const uint8_t* __restrict__ buf, uint64_t n, uint64_t start,
                                                         uint32_t quote4, uint32_t delim4,
                                                         const uint32_t* __restrict__ tile_state,
                                                         const uint32_t* __restrict__ tile_first,
                                                         const uint32_t* __restrict__ total, uint32_t ncol,
                                                         uint32_t row_base, uint32_t* __restrict__ pos,
                                                         uint32_t* __restrict__ tail,
                                                         unsigned long long* __restrict__ bad_row,
                                                         uint32_t* __restrict__ err) {
    __shared__ uint32_t s_w[kThreads / 32];
    const uint64_t base = ((uint64_t)blockIdx.x * kThreads + threadIdx.x) * kChunk;
    const Masks m = chunk_masks(buf, n, start, base, quote4, delim4);
    const uint64_t px = prefix_xor(m.quote);
    uint32_t par_total;
    const uint32_t st = tile_state[blockIdx.x] ^ block_xor_excl(__popcll(m.quote) & 1u, s_w, par_total);
    uint64_t ev = m.ev & (st ? px : ~px);
    uint32_t tot;
    uint32_t off = tile_first[blockIdx.x] + block_sum_excl(__popcll(ev), s_w, tot);
    const uint32_t last = *total - 1;
    uint32_t col = ev ? off % ncol : 0;  // column of field `off`, advanced without dividing
    while (ev) {
        const int b = __ffsll((long long)ev) - 1;
        ev &= ev - 1;
        const uint32_t p = (uint32_t)(base + b);
        if (off > last) {  // cannot happen when both passes agree; never write past the array
            atomicOr(err, 8u);
            return;
        }
        pos[off] = p;
        const bool is_term = (m.term >> b) & 1;
        if (is_term != (col == ncol - 1)) atomicMin(bad_row, (unsigned long long)(off / ncol + row_base));
        col = col + 1 == ncol ? 0 : col + 1;
        if (off == last) {
            uint32_t next = 0xffffffffu;
            if (is_term) {
                next = p + 1;
                if (buf[p] == '\r' && (uint64_t)p + 1 < n && buf[p + 1] == '\n') ++next;
            }
            *tail = next;
        }
        ++off;
    }
}

// Sequential byte reader over a 16-byte window (one vector load per window).
struct Reader {
    const uint8_t* buf;
    uint64_t n;
    uint64_t wb;
    uint32_t w0, w1, w2, w3;
    __device__ __forceinline__ Reader(const uint8_t* b, uint64_t nn) : buf(b), n(nn), wb(~0ull), w0(0), w1(0), w2(0), w3(0) {}
    __device__ __forceinline__ unsigned char get(uint64_t i) {
        const uint64_t b = i & ~15ull;
        if (b != wb) {
            wb = b;
            if (b + 16 <= n) {
                const uint4 v = __ldg(reinterpret_cast<const uint4*>(buf + b));
                w0 = v.x;
                w1 = v.y;
                w2 = v.z;
                w3 = v.w;
            } else {
                uint32_t x[4] = {0, 0, 0, 0};
                for (int k = 0; k < 16; ++k)
                    if (b + k < n) x[k >> 2] |= (uint32_t)__ldg(buf + b + k) << (8 * (k & 3));
                w0 = x[0];
                w1 = x[1];
                w2 = x[2];
                w3 = x[3];
            }
        }
        const uint32_t k = (uint32_t)(i & 15);
        const uint32_t word = k < 8 ? (k < 4 ? w0 : w1) : (k < 12 ? w2 : w3);
        return (unsigned char)(word >> ((k & 3) * 8));
    }
    // The 8 bytes at i (byte i lowest), those at and past i + avail zeroed.
    __device__ __forceinline__ uint64_t get8(uint64_t i, uint32_t avail) {
        get(i);  // window holding byte i
        const uint32_t k = (uint32_t)(i & 15);
        const uint64_t lo = (uint64_t)w0 | ((uint64_t)w1 << 32), hi = (uint64_t)w2 | ((uint64_t)w3 << 32);
        uint64_t v;
        if (k == 0) v = lo;
        else if (k < 8) v = (lo >> (8 * k)) | (hi << (64 - 8 * k));
        else if (k == 8) v = hi;
        else {
            v = hi >> (8 * (k - 8));
            if (avail > 16 - k) {  // the rest is in the next window
                get(i + (16 - k));
                const uint64_t nlo = (uint64_t)w0 | ((uint64_t)w1 << 32);
                v |= nlo << (8 * (16 - k));
            }
        }
        if (avail < 8) v &= (1ull << (8 * avail)) - 1;
        return v;
    }
};

// Per-column output descriptor.
struct CsvColDev {
    uint32_t type;  // 'd', 'u', 'b', 's', 'c'
    uint32_t scol;  // string column index (strings)
    void* values;
    uint64_t* offsets;    // strings: nrow + 1 (lengths at [row + 1] before the scan)
    uint32_t* starts;     // strings: field start per row
};

struct ParseArgs {
    const uint8_t* buf;
    uint64_t n;
    uint32_t data_start;
    const uint32_t* pos;  // field end positions, ncol per record (the last may be n)
    uint32_t records;
    uint32_t row_base;    // 1 when the first line is a data row parsed separately
    uint32_t ncol;
    unsigned char delim, quote;
    const CsvColDev* cols;
    unsigned long long* bad_row;  // first record with the wrong field count
    uint32_t* err;                // device error bits (slow path overflow)
};

__device__ __noinline__ double slow_field(const uint8_t* buf, uint32_t fs, uint32_t len, uint32_t* err) {
    bool ok = true;
    const double v = vdfdec::slow_decide([=](uint32_t j) { return (unsigned char)__ldg(buf + fs + j); }, len, ok);
    if (!ok) atomicOr(err, 4u);
    return v;
}

// Converts one field [fs, fe) of column `col` into row `row`.
__device__ __forceinline__ void emit_field(const ParseArgs& a, Reader& rd, uint32_t fs, uint32_t fe, uint32_t col,
                                           uint32_t row, bool empty_is_na) {
    const CsvColDev* d = a.cols + col;
    const uint32_t type = __ldg(&d->type);
    const uint32_t len = fe - fs;
    auto at = [&](uint32_t j) { return rd.get((uint64_t)fs + j); };
    if (type == 'd') {
        vdfdec::Number num;
        if (!vdfdec::scan_number_fast(rd, fs, len, num)) num = vdfdec::scan_number(at, len);
        const vdfdec::Conv cv = vdfdec::convert(num);
        double v = cv.v;
        if (cv.ambiguous) v = slow_field(a.buf, fs, len, a.err);
        static_cast<double*>(d->values)[row] = v;
    } else if (type == 'u') {
        static_cast<uint32_t*>(d->values)[row] = vdfdec::parse_u32(at, len);
    } else if (type == 'b') {
        static_cast<uint8_t*>(d->values)[row] = vdfdec::parse_i32(at, len) != 0 ? 1 : 0;
    } else {
        // strings: an empty field reads "NA" (parse_rows_chunk.inl:80-81)
        const bool na = len == 0 && empty_is_na;
        d->offsets[row + 1] = na ? 2 : len;
        d->starts[row] = na ? 0xffffffffu : fs;
    }
}

// One thread per record; the threads of a CTA convert column c of their
// records together (the same type branch, coalesced column writes), taking
// each field's bounds from the field-end positions.
__global__ void __launch_bounds__(kThreads) k_csv_parse(ParseArgs a) {
    const uint32_t r = blockIdx.x * kThreads + threadIdx.x;
    if (r >= a.records) return;
    const uint32_t row = r + a.row_base;
    const uint32_t* fp = a.pos + (uint64_t)r * a.ncol;
    uint32_t fs = a.data_start;
    if (r > 0) {
        const uint32_t p = fp[-1];
        fs = p + 1;
        if (a.buf[p] == '\r' && (uint64_t)p + 1 < a.n && a.buf[p + 1] == '\n') ++fs;
    }
    Reader rd(a.buf, a.n);
    for (uint32_t c = 0; c < a.ncol; ++c) {
        const uint32_t fe = fp[c];
        emit_field(a, rd, fs, fe, c, row, true);
        fs = fe + 1;
    }
}

// The first line as a data row (no header): field bounds from the host, an
// empty field other than the last reads "" (read_csv.hpp:117-134).
__global__ void k_csv_first_line(ParseArgs a, const uint32_t* __restrict__ bounds) {
    const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= a.ncol) return;
    Reader rd(a.buf, a.n);
    emit_field(a, rd, bounds[2 * c], bounds[2 * c + 1], c, 0, c + 1 == a.ncol);
}

// Offsets: in-place inclusive scan of lengths at [1, nrow] per string column
// (blockIdx.y), three phases over 2048-row blocks.
constexpr int kScanRows = kThreads * 8;

struct StrCols {
    uint64_t* off[64];
};

__global__ void __launch_bounds__(kThreads) k_csv_off_partials(StrCols sc, uint64_t nrow, uint64_t* __restrict__ part,
                                                               uint32_t nblk) {
    __shared__ uint64_t s_w[kThreads / 32];
    const uint64_t* o = sc.off[blockIdx.y] + 1;
    const uint64_t b = (uint64_t)blockIdx.x * kScanRows;
    uint64_t s = 0;
    for (int k = 0; k < 8; ++k) {
        const uint64_t i = b + (uint64_t)k * kThreads + threadIdx.x;
        if (i < nrow) s += o[i];
    }
    for (int d = 16; d; d >>= 1) s += __shfl_down_sync(0xffffffffu, s, d);
    if ((threadIdx.x & 31) == 0) s_w[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint64_t t = 0;
        for (int i = 0; i < kThreads / 32; ++i) t += s_w[i];
        part[(uint64_t)blockIdx.y * nblk + blockIdx.x] = t;
    }
}

__global__ void __launch_bounds__(1024) k_csv_off_blocks(uint64_t* __restrict__ part, uint32_t nblk) {
    // one CTA per string column: exclusive scan of the block sums
    __shared__ uint64_t s_w[32];
    uint64_t* p = part + (uint64_t)blockIdx.x * nblk;
    uint64_t carry = 0;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (uint32_t b = 0; b < nblk; b += blockDim.x) {
        const uint32_t i = b + threadIdx.x;
        const uint64_t v = i < nblk ? p[i] : 0;
        uint64_t x = v;
        for (int d = 1; d < 32; d <<= 1) {
            const uint64_t y = __shfl_up_sync(0xffffffffu, x, d);
            if (lane >= d) x += y;
        }
        if (lane == 31) s_w[warp] = x;
        __syncthreads();
        uint64_t wp = 0, tot = 0;
        for (int k = 0; k < (int)(blockDim.x >> 5); ++k) {
            if (k < warp) wp += s_w[k];
            tot += s_w[k];
        }
        __syncthreads();
        if (i < nblk) p[i] = carry + wp + x - v;
        carry += tot;
    }
}

__global__ void __launch_bounds__(kThreads) k_csv_off_apply(StrCols sc, uint64_t nrow, const uint64_t* __restrict__ part,
                                                            uint32_t nblk) {
    __shared__ uint64_t s_w[kThreads / 32];
    uint64_t* o = sc.off[blockIdx.y];
    const uint64_t b = (uint64_t)blockIdx.x * kScanRows;
    uint64_t carry = part[(uint64_t)blockIdx.y * nblk + blockIdx.x];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (blockIdx.x == 0 && threadIdx.x == 0) o[0] = 0;
    for (int k = 0; k < 8; ++k) {
        const uint64_t i = b + (uint64_t)k * kThreads + threadIdx.x;
        const uint64_t v = i < nrow ? o[i + 1] : 0;
        uint64_t x = v;
        for (int d = 1; d < 32; d <<= 1) {
            const uint64_t y = __shfl_up_sync(0xffffffffu, x, d);
            if (lane >= d) x += y;
        }
        if (lane == 31) s_w[warp] = x;
        __syncthreads();
        uint64_t wp = 0, tot = 0;
        for (int j = 0; j < kThreads / 32; ++j) {
            if (j < warp) wp += s_w[j];
            tot += s_w[j];
        }
        __syncthreads();
        if (i < nrow) o[i + 1] = carry + wp + x;
        carry += tot;
    }
}

struct StrCopy {
    const uint8_t* buf;
    uint64_t nrow;
    uint32_t nstr;
    const uint64_t* off[64];
    const uint32_t* starts[64];
    uint8_t* bytes[64];
};

// One warp per 32 rows of one string column (blockIdx.y): the lanes walk the
// rows' contiguous output span byte by byte (coalesced stores) and find each
// byte's row by a binary search over the 32 row offsets held in lanes.
__global__ void __launch_bounds__(kThreads) k_csv_strings(StrCopy sc) {
    const uint32_t k = blockIdx.y;
    const int lane = threadIdx.x & 31;
    const uint64_t r0 = ((uint64_t)blockIdx.x * kThreads + threadIdx.x) & ~31ull;
    if (r0 >= sc.nrow) return;
    const uint64_t r = r0 + lane;
    const uint64_t* off = sc.off[k];
    const uint64_t o = r < sc.nrow ? off[r] : off[sc.nrow];
    const uint32_t s = r < sc.nrow ? sc.starts[k][r] : 0u;
    const uint64_t o0 = __shfl_sync(0xffffffffu, o, 0);
    const uint64_t rend = r0 + 32 < sc.nrow ? r0 + 32 : sc.nrow;
    const uint64_t span = off[rend] - o0;
    uint8_t* dst = sc.bytes[k];
    constexpr int U = 4;  // output bytes per lane per round: all U sources located, then loaded, then stored
    for (uint64_t b = 0; b < span; b += 32 * U) {  // the same trip count in every lane
        uint32_t src[U];
        bool na[U];
        uint8_t val[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const uint64_t d = b + (uint64_t)u * 32 + lane;
            const uint64_t at = o0 + (d < span ? d : span - 1);
            // largest j with off[r0 + j] <= at (lanes past the end hold the end offset)
            int j = 0;
#pragma unroll
            for (int step = 16; step; step >>= 1) {
                const uint64_t oj = __shfl_sync(0xffffffffu, o, j + step);
                if (oj <= at) j += step;
            }
            const uint64_t oj = __shfl_sync(0xffffffffu, o, j);
            const uint32_t sj = __shfl_sync(0xffffffffu, s, j);
            const uint32_t i = (uint32_t)(at - oj);
            na[u] = sj == 0xffffffffu;
            src[u] = na[u] ? i : sj + i;  // for "NA": the byte's index in "NA"
        }
#pragma unroll
        for (int u = 0; u < U; ++u)
            val[u] = na[u] ? (src[u] ? 'A' : 'N') : __ldg(sc.buf + src[u]);
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const uint64_t d = b + (uint64_t)u * 32 + lane;
            if (d < span) dst[o0 + d] = val[u];
        }
    }
}

// ---------------------------------------------------------------- host side
// Table blocks come from a stream-ordered pool per device that keeps up to
// 8 GiB cached between reads (a fresh cudaMalloc of the ~1.5 GB a 1 GB file
// needs costs about a millisecond).
cudaMemPool_t table_pool(int device) {
    static std::mutex mu;
    static cudaMemPool_t pools[64] = {};
    std::lock_guard<std::mutex> lk(mu);
    if (device < 0 || device >= 64) return nullptr;
    if (!pools[device]) {
        cudaMemPoolProps props{};
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = device;
        cudaMemPool_t p = nullptr;
        if (cudaMemPoolCreate(&p, &props) != cudaSuccess) {
            cudaGetLastError();
            return nullptr;
        }
        uint64_t keep = 8ull << 30;
        cudaMemPoolSetAttribute(p, cudaMemPoolAttrReleaseThreshold, &keep);
        pools[device] = p;
    }
    return pools[device];
}

cudaError_t table_alloc(int device, unsigned char** p, size_t bytes, cudaStream_t s, bool& pooled) {
    cudaMemPool_t pool = table_pool(device);
    pooled = pool != nullptr;
    if (!pool) return cudaMalloc(p, bytes);
    return cudaMallocFromPoolAsync(reinterpret_cast<void**>(p), bytes, pool, s);
}

// Frees a table block once no work can still use it (cudaFree's guarantee).
void table_free(unsigned char*& p, bool pooled) {
    if (!p) return;
    if (pooled) {
        cudaDeviceSynchronize();
        cudaFreeAsync(p, 0);
    } else {
        cudaFree(p);
    }
    p = nullptr;
}

// The reference's first-line pass (read_csv.hpp:58-135): splits at the
// delimiter outside quotes and stops at the first CR or LF even inside
// quotes; a CR or LF followed by LF moves the stop onto that LF, so the last
// field keeps the first of the two bytes.  Returns the stop index.
size_t first_line(const unsigned char* b, size_t n, char delim, char quote, std::vector<std::pair<size_t, size_t>>& f) {
    size_t i = 0, fs = 0;
    bool inq = false;
    for (; i < n; ++i) {
        const unsigned char c = b[i];
        if (c == '\n' || c == '\r') {
            if (i + 1 < n && b[i + 1] == '\n') ++i;
            break;
        }
        if (c == (unsigned char)quote) inq = !inq;
        else if (c == (unsigned char)delim && !inq) {
            f.push_back({fs, i});
            fs = i + 1;
        }
    }
    f.push_back({fs, i});
    return i;
}

// simd_can_be_nb (V/inlines/simd_can_be_nb.inl:1-43): non-empty, digits and
// at most one '.'.
bool can_be_nb(const std::string& s) {
    if (s.empty()) return false;
    bool dot = false;
    for (unsigned char c : s) {
        if (c == '.') {
            if (dot) return false;
            dot = true;
        } else if (c < '0' || c > '9') {
            return false;
        }
    }
    return true;
}

// classify_column's decision (V/inlines/classify_column.inl:13-133) on the
// first values of a column: a dotted number decides 'd' at once; a
// non-number longer than one byte stops the scan ('s'); other non-numbers
// make it 'c'; then all "0"/"1" -> 'b', else 'u'.  (The 'i' branch needs a
// value that is a number and starts with '-', which simd_can_be_nb never
// accepts, so it is not reachable.)
char classify(const std::vector<std::string>& v) {
    bool is_bool = true, is_nb = true, is_bufchar = true;
    const size_t k = v.size() < 10 ? v.size() : 10;
    for (size_t i = 0; i < k; ++i) {
        const std::string& s = v[i];
        if (!can_be_nb(s)) {
            is_nb = false;
            if (s.size() > 1) {
                is_bufchar = false;
                break;
            }
            continue;
        }
        if (s.find('.') != std::string::npos) return 'd';
        if (s != "0" && s != "1") is_bool = false;
    }
    if (!is_nb) return is_bufchar ? 'c' : 's';
    return is_bool ? 'b' : 'u';
}

inline unsigned grid_of(uint64_t n, unsigned per) { return (unsigned)((n + per - 1) / per); }

vdf_status csv_read_locked(vdf_ctx* c, const uint8_t* dbuf, const uint8_t* hbuf, uint64_t n, char delim, int header,
                           char quote, vdf_csv** out, cudaStream_t s) {
    vdf::Profiler* prof = prof_of(c);
    auto begin = [&]() {
        if (prof) prof->begin(vdf::KC_CSV, s);
    };
    auto end = [&]() {
        if (prof) prof->end(vdf::KC_CSV, s);
    };
    cudaError_t e;
    // ---- first line (host): names, or the first data row
    std::vector<unsigned char> head;
    const unsigned char* hb = hbuf;
    size_t hn = n;
    if (!hbuf) {
        // read until the first CR / LF (and one more byte for CR LF)
        size_t want = n < 65536 ? n : 65536;
        for (;;) {
            head.resize(want);
            e = cudaMemcpyAsync(head.data(), dbuf, want, cudaMemcpyDeviceToHost, s);
            if (e == cudaSuccess) e = cudaStreamSynchronize(s);
            if (e != cudaSuccess) return from_cuda(c, e, "read the first line");
            size_t i = 0;
            while (i < want && head[i] != '\n' && head[i] != '\r') ++i;
            if (i + 1 < want || want == n) break;
            want = (want * 4 < n) ? want * 4 : n;
        }
        hb = head.data();
        hn = head.size();
    }
    std::vector<std::pair<size_t, size_t>> f0;
    const size_t stop = first_line(hb, hn, delim, quote, f0);
    const uint32_t ncol = (uint32_t)f0.size();
    if (ncol > 4096) return fail(c, VDF_ERR_UNSUPPORTED, "%u columns (limit 4096)", ncol);
    const uint64_t data_start = stop + 1 < n ? stop + 1 : n;
    std::vector<std::string> names, first;
    for (uint32_t k = 0; k < ncol; ++k) {
        const size_t a = f0[k].first, b = f0[k].second;
        std::string v((const char*)hb + a, b - a);
        if (header) names.push_back(v.empty() ? std::string("NA") : v);
        else first.push_back((v.empty() && k + 1 == ncol) ? std::string("NA") : v);
    }
    if (!header) names.assign(ncol, std::string());  // no header: the reference keeps no names

    // ---- field ends over [data_start, n)
    const uint32_t row_base = header ? 0 : 1;
    const uint64_t nchunks = (n + kChunk - 1) / kChunk;
    const uint32_t ntiles = (uint32_t)((nchunks + kThreads - 1) / kThreads);
    const size_t o_tiles = 0, o_state = align256((size_t)12 * ntiles), o_first = o_state + align256((size_t)4 * ntiles);
    const size_t o_misc = o_first + align256((size_t)4 * ntiles), o_pos = o_misc + 256;
    vdf_status st;
    if ((st = ws_ensure(c, o_pos + 256)) != VDF_OK) return st;
    uint32_t* tiles = reinterpret_cast<uint32_t*>(c->ws + o_tiles);
    uint32_t* tstate = reinterpret_cast<uint32_t*>(c->ws + o_state);
    uint32_t* tfirst = reinterpret_cast<uint32_t*>(c->ws + o_first);
    uint32_t* misc = reinterpret_cast<uint32_t*>(c->ws + o_misc);  // [0] field ends, [1] tail
    unsigned long long* bad = reinterpret_cast<unsigned long long*>(c->ws + o_misc + 8);
    const uint32_t quote4 = 0x01010101u * (unsigned char)quote;
    const uint32_t delim4 = 0x01010101u * (unsigned char)delim;
    uint32_t nfields = 0, tail = (uint32_t)data_start;
    auto count_pass = [&]() -> vdf_status {
        begin();
        k_csv_count<<<ntiles, kThreads, 0, s>>>(dbuf, n, data_start, quote4, delim4, tiles);
        if ((e = cudaGetLastError()) != cudaSuccess) return from_cuda(c, e, "launch k_csv_count");
        k_csv_scan<<<1, 1024, 0, s>>>(tiles, ntiles, tstate, tfirst, misc);
        if ((e = cudaGetLastError()) != cudaSuccess) return from_cuda(c, e, "launch k_csv_scan");
        end();
        c->launches += 2;
        return VDF_OK;
    };
    if (ntiles && data_start < n) {
        if ((st = count_pass()) != VDF_OK) return st;
        e = cudaMemcpyAsync(&c->host_pinned[0], misc, 4, cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) return from_cuda(c, e, "field count");
        nfields = (uint32_t)(c->host_pinned[0] & 0xffffffffu);
        if (nfields > n - data_start)
            return fail(c, VDF_ERR_DEVICE, "field count %u exceeds the %llu data bytes", nfields,
                        (unsigned long long)(n - data_start));
    }
    // room for the positions (+1: a final record without terminator).
    // Growing the workspace replaces the buffer and loses the tile states and
    // offsets just computed, so the two passes run again on the new one.
    const size_t ws_need = o_pos + align256((size_t)4 * (nfields + 1));
    if (ws_need > c->ws_cap) {
        if ((st = ws_ensure(c, ws_need)) != VDF_OK) return st;
        tiles = reinterpret_cast<uint32_t*>(c->ws + o_tiles);
        tstate = reinterpret_cast<uint32_t*>(c->ws + o_state);
        tfirst = reinterpret_cast<uint32_t*>(c->ws + o_first);
        misc = reinterpret_cast<uint32_t*>(c->ws + o_misc);
        bad = reinterpret_cast<unsigned long long*>(c->ws + o_misc + 8);
        if (nfields && (st = count_pass()) != VDF_OK) return st;
    }
    uint32_t* pos = reinterpret_cast<uint32_t*>(c->ws + o_pos);
    e = cudaMemsetAsync(bad, 0xff, 8, s);
    if (e != cudaSuccess) return from_cuda(c, e, "clear the error row");
    unsigned long long bad_row = ~0ull;
    if (nfields) {
        begin();
        k_csv_fields<<<ntiles, kThreads, 0, s>>>(dbuf, n, data_start, quote4, delim4, tstate, tfirst, misc, ncol,
                                                 row_base, pos, misc + 1, bad, err_word(c));
        if ((e = cudaGetLastError()) != cudaSuccess) return from_cuda(c, e, "launch k_csv_fields");
        end();
        c->launches += 1;
        e = cudaMemcpyAsync(&c->host_pinned[0], misc + 1, 4, cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaMemcpyAsync(&c->host_pinned[2], bad, 8, cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) return from_cuda(c, e, "field tail");
        tail = (uint32_t)(c->host_pinned[0] & 0xffffffffu);
        bad_row = c->host_pinned[2];
    }
    if (tail == 0xffffffffu || tail < n) {
        // the bytes after the last terminator form one more record: its end is n
        if (nfields % ncol != ncol - 1) bad_row = std::min<unsigned long long>(bad_row, nfields / ncol + row_base);
        c->host_pinned[0] = n;
        e = cudaMemcpyAsync(pos + nfields, &c->host_pinned[0], 4, cudaMemcpyHostToDevice, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) return from_cuda(c, e, "final record");
        ++nfields;
    }
    if (bad_row != ~0ull)
        return fail(c, VDF_ERR_INVALID_ARG, "column number problem at row %llu (%u fields expected)", bad_row, ncol);
    const uint32_t records = nfields / ncol;
    const uint64_t nrow = (uint64_t)records + row_base;

    // ---- classify on the first 10 values of each column
    std::vector<std::vector<std::string>> vals(ncol);
    if (!header)
        for (uint32_t k = 0; k < ncol; ++k) vals[k].push_back(first[k]);
    const uint32_t nfirst = records < 10 ? records : 10;
    if (nfirst) {
        std::vector<uint32_t> p((size_t)nfirst * ncol);
        e = cudaMemcpyAsync(p.data(), pos, 4 * p.size(), cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) return from_cuda(c, e, "first records");
        const uint64_t span_end = (uint64_t)p.back() + 2 < n ? (uint64_t)p.back() + 2 : n;
        std::vector<unsigned char> tmp;
        const unsigned char* hb2 = hbuf;
        if (!hbuf) {
            tmp.resize(span_end);
            e = cudaMemcpyAsync(tmp.data(), dbuf, span_end, cudaMemcpyDeviceToHost, s);
            if (e == cudaSuccess) e = cudaStreamSynchronize(s);
            if (e != cudaSuccess) return from_cuda(c, e, "first records' bytes");
            hb2 = tmp.data();
        }
        uint64_t fs = data_start;
        for (uint32_t r = 0; r < nfirst; ++r)
            for (uint32_t k = 0; k < ncol; ++k) {
                const uint64_t fe = p[(size_t)r * ncol + k];
                if (vals[k].size() < 10)
                    vals[k].push_back(fe > fs ? std::string((const char*)hb2 + fs, fe - fs) : std::string("NA"));
                fs = fe + 1;
                if (k + 1 == ncol && fe < n && hb2[fe] == '\r' && fe + 1 < n && hb2[fe + 1] == '\n') ++fs;
            }
    }
    std::unique_ptr<vdf_csv> t(new vdf_csv());
    t->device = c->device;
    t->nrow = nrow;
    t->ncol = ncol;
    t->names = names;
    t->types.resize(ncol);
    t->values.assign(ncol, nullptr);
    t->offsets.assign(ncol, nullptr);
    t->str_bytes.assign(ncol, 0);
    std::vector<uint32_t> scol_of(ncol, 0), str_cols;
    for (uint32_t k = 0; k < ncol; ++k) {
        t->types[k] = classify(vals[k]);
        if (t->types[k] == 's' || t->types[k] == 'c') {
            scol_of[k] = (uint32_t)str_cols.size();
            str_cols.push_back(k);
        }
    }
    if (str_cols.size() > 64) return fail(c, VDF_ERR_UNSUPPORTED, "%zu string columns (limit 64)", str_cols.size());
    // ---- outputs: values, string offsets and starts, column descriptors
    std::vector<size_t> o_val(ncol, 0), o_off(ncol, 0), o_start(ncol, 0);
    size_t total = 0;
    for (uint32_t k = 0; k < ncol; ++k) {
        const char ty = t->types[k];
        if (ty == 'd') o_val[k] = total, total += align256(8 * nrow);
        else if (ty == 'u') o_val[k] = total, total += align256(4 * nrow);
        else if (ty == 'b') o_val[k] = total, total += align256(nrow ? nrow : 1);
        else {
            o_off[k] = total, total += align256(8 * (nrow + 1));
            o_start[k] = total, total += align256(4 * (nrow ? nrow : 1));
        }
    }
    const size_t o_desc = total;
    total += align256(sizeof(CsvColDev) * ncol);
    const size_t o_bounds = total;
    total += align256(8 * ncol);
    size_t o_part = total;
    const uint32_t nblk = (uint32_t)((nrow + kScanRows - 1) / kScanRows);
    total += align256(8 * (size_t)nblk * (str_cols.empty() ? 1 : str_cols.size()) + 8);
    e = table_alloc(c->device, &t->block, total, s, t->pooled);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return fail(c, VDF_ERR_OOM, "column allocation of %zu bytes failed", total);
    }
    std::vector<CsvColDev> desc(ncol);
    for (uint32_t k = 0; k < ncol; ++k) {
        const char ty = t->types[k];
        desc[k].type = (uint32_t)(unsigned char)ty;
        desc[k].scol = scol_of[k];
        desc[k].values = nullptr;
        desc[k].offsets = nullptr;
        desc[k].starts = nullptr;
        if (ty == 'd' || ty == 'u' || ty == 'b') {
            desc[k].values = t->block + o_val[k];
            t->values[k] = desc[k].values;
        } else {
            desc[k].offsets = reinterpret_cast<uint64_t*>(t->block + o_off[k]);
            desc[k].starts = reinterpret_cast<uint32_t*>(t->block + o_start[k]);
            t->offsets[k] = desc[k].offsets;
        }
    }
    std::vector<uint32_t> bounds(2 * ncol, 0);
    for (uint32_t k = 0; k < ncol; ++k) {
        bounds[2 * k] = (uint32_t)f0[k].first;
        bounds[2 * k + 1] = (uint32_t)f0[k].second;
    }
    CsvColDev* ddesc = reinterpret_cast<CsvColDev*>(t->block + o_desc);
    uint32_t* dbounds = reinterpret_cast<uint32_t*>(t->block + o_bounds);
    e = cudaMemcpyAsync(ddesc, desc.data(), sizeof(CsvColDev) * ncol, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dbounds, bounds.data(), 8 * ncol, cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) {
        table_free(t->block, t->pooled);
        return from_cuda(c, e, "column descriptors");
    }
    // ---- parse
    ParseArgs pa;
    pa.buf = dbuf;
    pa.n = n;
    pa.data_start = (uint32_t)data_start;
    pa.pos = pos;
    pa.records = records;
    pa.row_base = row_base;
    pa.ncol = ncol;
    pa.delim = (unsigned char)delim;
    pa.quote = (unsigned char)quote;
    pa.cols = ddesc;
    pa.bad_row = bad;
    pa.err = err_word(c);
    begin();
    if (!header) k_csv_first_line<<<grid_of(ncol, 128), 128, 0, s>>>(pa, dbounds);
    if (records) k_csv_parse<<<grid_of(records, kThreads), kThreads, 0, s>>>(pa);
    end();
    c->launches += (header ? 0 : 1) + (records ? 1 : 0);
    // ---- string offsets
    StrCols sc;
    for (size_t k = 0; k < str_cols.size(); ++k) sc.off[k] = t->offsets[str_cols[k]];
    uint64_t* part = reinterpret_cast<uint64_t*>(t->block + o_part);
    if (!str_cols.empty() && nrow) {
        const dim3 g(nblk, (unsigned)str_cols.size());
        begin();
        k_csv_off_partials<<<g, kThreads, 0, s>>>(sc, nrow, part, nblk);
        k_csv_off_blocks<<<(unsigned)str_cols.size(), 1024, 0, s>>>(part, nblk);
        k_csv_off_apply<<<g, kThreads, 0, s>>>(sc, nrow, part, nblk);
        end();
        c->launches += 3;
    } else {
        for (size_t k = 0; k < str_cols.size(); ++k) cudaMemsetAsync(t->offsets[str_cols[k]], 0, 8, s);
    }
    // string totals and the first bad record
    std::vector<uint64_t> sums(str_cols.size() + 1, 0);
    e = cudaMemcpyAsync(&sums[0], bad, 8, cudaMemcpyDeviceToHost, s);
    for (size_t k = 0; k < str_cols.size() && e == cudaSuccess; ++k)
        e = cudaMemcpyAsync(&sums[k + 1], t->offsets[str_cols[k]] + nrow, 8, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) {
        table_free(t->block, t->pooled);
        return from_cuda(c, e, "parse");
    }
    if (!str_cols.empty()) {
        size_t stotal = 0;
        std::vector<size_t> o_str(str_cols.size());
        for (size_t k = 0; k < str_cols.size(); ++k) {
            o_str[k] = stotal;
            stotal += align256(sums[k + 1] ? sums[k + 1] : 1);
            t->str_bytes[str_cols[k]] = sums[k + 1];
        }
        e = table_alloc(c->device, &t->sblock, stotal, s, t->spooled);
        if (e != cudaSuccess) {
            cudaGetLastError();
            table_free(t->block, t->pooled);
            return fail(c, VDF_ERR_OOM, "string allocation of %zu bytes failed", stotal);
        }
        StrCopy cp;
        cp.buf = dbuf;
        cp.nrow = nrow;
        cp.nstr = (uint32_t)str_cols.size();
        for (size_t k = 0; k < str_cols.size(); ++k) {
            const uint32_t col = str_cols[k];
            cp.off[k] = t->offsets[col];
            cp.starts[k] = desc[col].starts;
            cp.bytes[k] = t->sblock + o_str[k];
            t->values[col] = cp.bytes[k];
        }
        if (nrow) {
            begin();
            k_csv_strings<<<dim3(grid_of(nrow, kThreads), cp.nstr), kThreads, 0, s>>>(cp);
            end();
            c->launches += 1;
        }
    }
    e = cudaGetLastError();
    if (e != cudaSuccess) {
        vdf_csv_free(t.release());
        return from_cuda(c, e, "csv kernels");
    }
    if ((st = drain_and_check(c, s)) != VDF_OK) {
        vdf_csv_free(t.release());
        return st;
    }
    *out = t.release();
    return VDF_OK;
}

vdf_status check_csv_args(vdf_ctx* c, const void* bytes, uint64_t n, char delim, char quote, vdf_csv** out) {
    if (!out) return fail(c, VDF_ERR_INVALID_ARG, "out is NULL");
    *out = nullptr;
    if (n && !bytes) return fail(c, VDF_ERR_INVALID_ARG, "NULL bytes");
    if (n >= 0xffffffffull) return fail(c, VDF_ERR_UNSUPPORTED, "files of 4 GiB or more are not supported");
    if (delim == '\n' || delim == '\r' || quote == '\n' || quote == '\r' || delim == quote || delim == 0 || quote == 0)
        return fail(c, VDF_ERR_INVALID_ARG, "delimiter / quote must differ and not be CR, LF or NUL");
    return VDF_OK;
}

}  // namespace

vdf_status vdf_csv_read(vdf_ctx* c, const void* bytes, uint64_t n, char delim, int header, char quote, vdf_csv** out,
                        void* stream) {
    if (!c) return VDF_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> lk(c->mu);
    vdf_status st = check_csv_args(c, bytes, n, delim, quote, out);
    if (st != VDF_OK) return st;
    if (n && (reinterpret_cast<uintptr_t>(bytes) & 15))
        return fail(c, VDF_ERR_INVALID_ARG, "device bytes must be 16-byte aligned");
    DeviceGuard g(c->device);
    return csv_read_locked(c, static_cast<const uint8_t*>(bytes), nullptr, n, delim, header, quote, out,
                           static_cast<cudaStream_t>(stream));
}

vdf_status vdf_csv_read_host(vdf_ctx* c, const void* bytes, uint64_t n, char delim, int header, char quote,
                             vdf_csv** out, void* stream) {
    if (!c) return VDF_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> lk(c->mu);
    vdf_status st = check_csv_args(c, bytes, n, delim, quote, out);
    if (st != VDF_OK) return st;
    DeviceGuard g(c->device);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if ((st = io_ensure(c, align256(n ? n : 1))) != VDF_OK) return st;
    if (n) {
        cudaError_t e = cudaMemcpyAsync(c->io, bytes, n, cudaMemcpyHostToDevice, s);
        if (e != cudaSuccess) return from_cuda(c, e, "copy the file to the device");
    }
    return csv_read_locked(c, c->io, static_cast<const uint8_t*>(bytes), n, delim, header, quote, out, s);
}

uint64_t vdf_csv_nrow(const vdf_csv* t) { return t ? t->nrow : 0; }
uint32_t vdf_csv_ncol(const vdf_csv* t) { return t ? t->ncol : 0; }
const char* vdf_csv_name(const vdf_csv* t, uint32_t col) {
    return (t && col < t->ncol) ? t->names[col].c_str() : nullptr;
}
char vdf_csv_type(const vdf_csv* t, uint32_t col) { return (t && col < t->ncol) ? t->types[col] : 0; }
const void* vdf_csv_values(const vdf_csv* t, uint32_t col) { return (t && col < t->ncol) ? t->values[col] : nullptr; }
const uint64_t* vdf_csv_offsets(const vdf_csv* t, uint32_t col) {
    return (t && col < t->ncol) ? t->offsets[col] : nullptr;
}
uint64_t vdf_csv_string_bytes(const vdf_csv* t, uint32_t col) { return (t && col < t->ncol) ? t->str_bytes[col] : 0; }

vdf_status vdf_csv_copy_column(vdf_ctx* c, const vdf_csv* t, uint32_t col, void* values, uint64_t* offsets,
                               void* stream) {
    if (!c) return VDF_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> lk(c->mu);
    if (!t || col >= t->ncol) return fail(c, VDF_ERR_INVALID_ARG, "bad table or column");
    DeviceGuard g(t->device);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const char ty = t->types[col];
    const size_t w = ty == 'd' ? 8 : ty == 'u' ? 4 : 1;
    const size_t bytes = (ty == 's' || ty == 'c') ? t->str_bytes[col] : w * t->nrow;
    cudaError_t e = cudaSuccess;
    if (bytes && values) e = cudaMemcpyAsync(values, t->values[col], bytes, cudaMemcpyDefault, s);
    if (e == cudaSuccess && offsets && t->offsets[col])
        e = cudaMemcpyAsync(offsets, t->offsets[col], 8 * (t->nrow + 1), cudaMemcpyDefault, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return from_cuda(c, e, "copy a column");
    return VDF_OK;
}

void vdf_csv_free(vdf_csv* t) {
    if (!t) return;
    {
        DeviceGuard g(t->device);
        table_free(t->block, t->pooled);
        table_free(t->sblock, t->spooled);
    }
    delete t;
}
