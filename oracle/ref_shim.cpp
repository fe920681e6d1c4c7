// ref_shim.cpp -- builds the reference's OWN radix-sort kernels into
// oracle/_ref/libvdf_ref.so.  TEST INFRASTRUCTURE ONLY: used by tests/ to pin
// the oracle restatement, by tests/golden/make_golden.py to generate fixtures,
// and by bench.py's CPU-baseline / reference arm.  Never loaded by the product.
//
// Nothing here is copied from the reference: the reference's headers are
// #include'd in place from its include/vison tree (the recipe in
// oracle/Makefile passes -I<reference>/include/vison).  The reference is
// header-only and vison.hpp as a whole does not compile, so this shim includes
// only the free-function layer of the sort path:
//   inlines/warning.inl, inlines/radix_sorts/details/constants.inl,
//   inlines/radix_sorts/details/u16/get_local_u16.inl,
//   inlines/radix_sorts/details/u32/*.inl, details/u64/*.inl,
//   inlines/radix_sorts/radix_sort_uint32{,_mt}.inl, radix_sort_uint64{,_mt}.inl
// and the vendored hash map / hash used by the reference group-by:
//   external/ankerl/unordered_dense.h (v4.8.0), custom_simd_hash/simd_hash.hpp.
//
// The CSV entry point ref_csv_read() runs the reference's own record parser
// (inlines/read/read_csv/parsers_core/parse_rows_chunk.inl, its AVX2 path),
// simd_can_be_nb / has_dot and fast_float::from_chars / std::from_chars; the
// parts of read_csv that are member code of the (uncompilable) Dataframe
// class are restated: the first-line pass (read/read_csv/read_csv.hpp:58-135)
// and classify_column's decision (inlines/classify_column.inl:13-133, whose
// 'c' branch does not compile), with the per-column conversions run under
// OpenMP over columns as type_classification does (type_classification.inl:
// 15-19).  The reference's multi-core parser (standard_parser_mt.inl:30-37)
// computes every chunk's end row from the first chunk's, so only its
// single-core parser is usable.
//
// The reference group-by itself cannot compile (syntax errors in
// transform/transform_group_by/*), so ref_groupby() restates its algorithm
// (transform_group_by_onecol_mt.hpp:182-337: per-thread ankerl maps keyed by
// the raw key bytes as a string_view hashed by simd_hash, "+=" accumulation,
// then a serial merge of the per-thread maps in thread order,
// merge_functions.inl:3-36) on top of the reference's own map and hash, with
// min/max added and mean = sum / count.
#include <algorithm>
#include <array>
#include <cstdint>
#include <cstring>
#include <iostream>
#include <string>
#include <string_view>
#include <vector>
#include <omp.h>
#include <immintrin.h>

#include "inlines/warning.inl"
#include "inlines/radix_sorts/details/constants.inl"
#include "inlines/radix_sorts/details/u16/get_local_u16.inl"
#include "inlines/radix_sorts/details/u32/histogram_pass_u32_avx2.inl"
#include "inlines/radix_sorts/details/u32/histogram_pass_u32_avx2_8buckets.inl"
#include "inlines/radix_sorts/details/u32/histogram_pass_u32_avx512_16buckets.inl"
#include "inlines/radix_sorts/details/u32/scatter_pass_u32_avx512.inl"
#include "inlines/radix_sorts/details/u64/histogram_pass_u64_avx2.inl"
#include "inlines/radix_sorts/details/u64/histogram_pass_u64_avx2_8x.inl"
#include "inlines/radix_sorts/details/u64/histogram_pass_u64_avx512_16x.inl"
#include "inlines/radix_sorts/details/u64/scatter_pass_u64_avx512.inl"
#include "inlines/radix_sorts/radix_sort_uint32.inl"
#include "inlines/radix_sorts/radix_sort_uint32_mt.inl"
#include "inlines/radix_sorts/radix_sort_uint64.inl"
#include "inlines/radix_sorts/radix_sort_uint64_mt.inl"

#include "external/ankerl/unordered_dense.h"
#include "custom_simd_hash/simd_hash.hpp"

// CSV ingest: the reference's record parser, numeric-shape tests and the
// vendored fast_float (v8.1.0), compiled from the reference tree.
#include <charconv>
#include <chrono>
#include "external/fast_float/fast_float.h"
#include "inlines/simd_can_be_nb.inl"
#include "inlines/has_dot.inl"
#include "inlines/read/read_csv/parsers_core/parse_rows_chunk.inl"

namespace {

template <unsigned C, bool Simd>
void sort32(std::vector<uint32_t>& k, size_t* idx, size_t n) {
    if constexpr (C == 1) radix_sort_uint32<Simd>(k, idx, n);
    else radix_sort_uint32_mt<C, Simd>(k, idx, n);
}
template <unsigned C, bool Simd>
void sort64(std::vector<uint64_t>& k, size_t* idx, size_t n) {
    if constexpr (C == 1) radix_sort_uint64<Simd>(k, idx, n);
    else radix_sort_uint64_mt<C, Simd>(k, idx, n);
}

// CORES is a compile-time parameter in the reference; the reference's
// per-thread tables hold at most MAX_THREADS = 32 threads
// (details/constants.inl:9), so 1..32 are instantiated.
template <bool Simd, unsigned C = 1>
int dispatch32(unsigned cores, std::vector<uint32_t>& k, size_t* idx, size_t n) {
    if constexpr (C > 32) { return -1; }
    else {
        if (cores == C) { sort32<C, Simd>(k, idx, n); return 0; }
        return dispatch32<Simd, C + 1>(cores, k, idx, n);
    }
}
template <bool Simd, unsigned C = 1>
int dispatch64(unsigned cores, std::vector<uint64_t>& k, size_t* idx, size_t n) {
    if constexpr (C > 32) { return -1; }
    else {
        if (cores == C) { sort64<C, Simd>(k, idx, n); return 0; }
        return dispatch64<Simd, C + 1>(cores, k, idx, n);
    }
}

int width_of(int dt) { return (dt == 0 || dt == 2 || dt == 5) ? 4 : (dt == 1 || dt == 3 || dt == 4) ? 8 : 0; }

// sort_integers.inl:46 (tkeys = UIntT(col) ^ signbit), sort_uintegers.inl:48-74
// (copy), sort_flt.inl:123-129 (double image).
uint64_t order_key(const void* col, int dt, size_t i) {
    switch (dt) {
    case 0: return uint32_t(static_cast<const int32_t*>(col)[i]) ^ 0x80000000u;
    case 1: return uint64_t(static_cast<const int64_t*>(col)[i]) ^ 0x8000000000000000ull;
    case 2: return static_cast<const uint32_t*>(col)[i];
    case 3: return static_cast<const uint64_t*>(col)[i];
    case 4: { uint64_t b; std::memcpy(&b, static_cast<const double*>(col) + i, 8);
              uint64_t m = -(b >> 63); return b ^ (m | 0x8000000000000000ull); }
    default: return 0;
    }
}

}  // namespace

extern "C" {

// Largest thread count the reference's tables support.
int ref_max_threads(void) { return int(MAX_THREADS); }

// In-place: keys are the already-transformed unsigned keys, idx is in/out.
// simd selects the reference's Simd template argument.  Multi-threaded Simd
// variants share process-wide static histogram tables across threads
// (get_local_u16.inl:30-40), so they are refused here.
int ref_radix_u32(uint32_t* keys, uint64_t* idx, size_t n, int cores, int simd) {
    if (cores < 1 || cores > 32 || (simd && cores != 1)) return -1;
    std::vector<uint32_t> k(keys, keys + n);
    size_t* ix = reinterpret_cast<size_t*>(idx);
    int rc = simd ? dispatch32<true>(unsigned(cores), k, ix, n) : dispatch32<false>(unsigned(cores), k, ix, n);
    std::copy(k.begin(), k.end(), keys);
    return rc;
}

int ref_radix_u64(uint64_t* keys, uint64_t* idx, size_t n, int cores, int simd) {
    if (cores < 1 || cores > 32 || (simd && cores != 1)) return -1;
    std::vector<uint64_t> k(keys, keys + n);
    size_t* ix = reinterpret_cast<size_t*>(idx);
    int rc = simd ? dispatch64<true>(unsigned(cores), k, ix, n) : dispatch64<false>(unsigned(cores), k, ix, n);
    std::copy(k.begin(), k.end(), keys);
    return rc;
}

// The reference's sort path for a multi-key frame: build tkeys for the least
// significant key, radix-sort with idx = iota, then for each more significant
// key gather it through idx (tkeys[i] = key'[idx[i]]) and radix-sort again
// with idx in/out.  Payload columns are then gathered by idx
// (permute_block_mt.inl:39-41), all with `cores` OpenMP threads.
// order: 0 ascending; 2 = the reference code's descending (std::reverse).
int ref_sort_frame(const void* const* keys, const int* kdt, int nkeys, size_t n,
                   int order, int cores, uint32_t* perm_out,
                   const void* const* pay, const int* pwidth, int npay, void* const* pay_out) {
    if (nkeys < 1 || cores < 1 || cores > 32 || (order != 0 && order != 2)) return -1;
    if (n == 0) return 0;
    std::vector<size_t> idx(n);
    #pragma omp parallel for num_threads(cores)
    for (size_t i = 0; i < n; ++i) idx[i] = i;
    for (int k = nkeys - 1; k >= 0; --k) {
        int w = width_of(kdt[k]);
        if (w == 4) {
            std::vector<uint32_t> tk(n);
            #pragma omp parallel for num_threads(cores)
            for (size_t i = 0; i < n; ++i) tk[i] = uint32_t(order_key(keys[k], kdt[k], idx[i]));
            if (cores == 1) radix_sort_uint32<false>(tk, idx.data(), n);
            else if (dispatch32<false>(unsigned(cores), tk, idx.data(), n)) return -1;
        } else if (w == 8) {
            std::vector<uint64_t> tk(n);
            #pragma omp parallel for num_threads(cores)
            for (size_t i = 0; i < n; ++i) tk[i] = order_key(keys[k], kdt[k], idx[i]);
            if (cores == 1) radix_sort_uint64<false>(tk, idx.data(), n);
            else if (dispatch64<false>(unsigned(cores), tk, idx.data(), n)) return -1;
        } else {
            return -1;
        }
    }
    if (order == 2) std::reverse(idx.begin(), idx.end());
    #pragma omp parallel for num_threads(cores)
    for (size_t i = 0; i < n; ++i) perm_out[i] = uint32_t(idx[i]);
    for (int p = 0; p < npay; ++p) {
        const unsigned char* s = static_cast<const unsigned char*>(pay[p]);
        unsigned char* d = static_cast<unsigned char*>(pay_out[p]);
        size_t w = size_t(pwidth[p]);
        if (w == 8) {
            #pragma omp parallel for num_threads(cores)
            for (size_t i = 0; i < n; ++i)
                reinterpret_cast<uint64_t*>(d)[i] = reinterpret_cast<const uint64_t*>(s)[idx[i]];
        } else if (w == 4) {
            #pragma omp parallel for num_threads(cores)
            for (size_t i = 0; i < n; ++i)
                reinterpret_cast<uint32_t*>(d)[i] = reinterpret_cast<const uint32_t*>(s)[idx[i]];
        } else {
            return -1;
        }
    }
    return 0;
}

// Per-group accumulator of the restated hash group-by: count, and for each
// value column sum / min / max (float columns in double, as the reference's
// `+=` on a double map value; integer columns in __int128).
struct RefAgg {
    int64_t count = 0;
    double fsum[4] = {0, 0, 0, 0};
    double fmin[4], fmax[4];
    __int128 isum[4] = {0, 0, 0, 0};
    int64_t imin[4], imax[4];
};

// Restated reference group-by (see file header).  Keys: up to 4 columns.  A
// single key column is hashed as its raw bytes (onecol_functions.inl:77-80);
// several key columns are concatenated per row, each followed by the '\x1F'
// separator, as KeyBuildDiffType / KeyBuildSameType do (key_build.inl:3-110).
// The reference's simd_hash copies up to 16 bytes into an 8-byte local for
// keys of 9..16 bytes (simd_hash.hpp:18-22 called from :35-36), which
// overflows the stack; such composite keys are zero-padded to 17 bytes so the
// hash takes its well-defined long-key path.  Values: up to 4 columns of
// dtype i32/i64/f64.  Returns the number of groups; out_checksum receives
// sum(count) and the sum over groups of each value column's sum.
int64_t ref_groupby(const void* const* keys, const int* kdt, int nkeys,
                    const void* const* vals, const int* vdt, int nvals,
                    size_t n, int cores, double* out_checksum) {
    if (nkeys < 1 || nkeys > 4 || nvals < 0 || nvals > 4 || cores < 1) return -1;
    size_t kw = 0;
    int off[4];
    const bool composite = nkeys > 1;
    for (int k = 0; k < nkeys; ++k) {
        off[k] = int(kw);
        int w = width_of(kdt[k]);
        if (!w) return -1;
        kw += size_t(w) + (composite ? 1 : 0);
    }
    if (kw > 8 && kw <= 16) kw = 17;
    for (int v = 0; v < nvals; ++v) if (vdt[v] != 0 && vdt[v] != 1 && vdt[v] != 4) return -1;
    std::vector<unsigned char> kbuf(n * kw, 0);
    #pragma omp parallel for num_threads(cores)
    for (size_t i = 0; i < n; ++i)
        for (int k = 0; k < nkeys; ++k) {
            size_t w = size_t(width_of(kdt[k]));
            std::memcpy(&kbuf[i * kw + size_t(off[k])], static_cast<const unsigned char*>(keys[k]) + i * w, w);
            if (composite) kbuf[i * kw + size_t(off[k]) + w] = 0x1F;
        }
    using Map = ankerl::unordered_dense::map<std::string_view, RefAgg, simd_hash>;
    std::vector<Map> maps(static_cast<size_t>(cores));
    #pragma omp parallel num_threads(cores)
    {
        int t = omp_get_thread_num();
        size_t chunk = n / size_t(cores), rem = n % size_t(cores);
        size_t beg = size_t(t) * chunk + std::min<size_t>(size_t(t), rem);
        size_t end = beg + chunk + (size_t(t) < rem ? 1 : 0);
        Map& m = maps[size_t(t)];
        m.reserve((end - beg) / 4 + 16);
        for (size_t i = beg; i < end; ++i) {
            auto [it, fresh] = m.try_emplace(std::string_view(reinterpret_cast<const char*>(&kbuf[i * kw]), kw));
            RefAgg& a = it->second;
            for (int v = 0; v < nvals; ++v) {
                if (vdt[v] == 4) {
                    double x = static_cast<const double*>(vals[v])[i];
                    a.fsum[v] += x;
                    if (fresh || x < a.fmin[v]) a.fmin[v] = x;
                    if (fresh || x > a.fmax[v]) a.fmax[v] = x;
                } else {
                    int64_t x = vdt[v] == 0 ? int64_t(static_cast<const int32_t*>(vals[v])[i])
                                            : static_cast<const int64_t*>(vals[v])[i];
                    a.isum[v] += x;
                    if (fresh || x < a.imin[v]) a.imin[v] = x;
                    if (fresh || x > a.imax[v]) a.imax[v] = x;
                }
            }
            a.count++;
        }
    }
    // Serial merge in thread order (MergeCurMap, merge_functions.inl:3-36).
    Map& lookup = maps[0];
    for (int t = 1; t < cores; ++t)
        for (auto& [k, b] : maps[size_t(t)]) {
            auto [it, fresh] = lookup.try_emplace(k, b);
            if (fresh) continue;
            RefAgg& a = it->second;
            a.count += b.count;
            for (int v = 0; v < nvals; ++v) {
                a.fsum[v] += b.fsum[v];
                a.isum[v] += b.isum[v];
                if (vdt[v] == 4) { a.fmin[v] = std::min(a.fmin[v], b.fmin[v]); a.fmax[v] = std::max(a.fmax[v], b.fmax[v]); }
                else { a.imin[v] = std::min(a.imin[v], b.imin[v]); a.imax[v] = std::max(a.imax[v], b.imax[v]); }
            }
        }
    if (out_checksum) {
        double c = 0; double s[4] = {0, 0, 0, 0};
        for (auto& [k, a] : lookup) {
            c += double(a.count);
            for (int v = 0; v < nvals; ++v) s[v] += vdt[v] == 4 ? a.fsum[v] : double(a.isum[v]);
        }
        out_checksum[0] = c;
        for (int v = 0; v < nvals; ++v) out_checksum[1 + v] = s[v];
    }
    return int64_t(lookup.size());
}


// CSV: parse `n` bytes as read_csv does and write the oracle's blob layout
// (see oracle/vdf_oracle_csv.c).  `seconds` (optional): time of the parse,
// inference and conversions (not the blob).  Malformed records: the
// reference stops at the first record with fewer fields (bad_row = that
// record); a record with MORE fields indexes past its column vector, so
// callers must not pass one.
void* ref_csv_read(const char* b, size_t n, char delim, int header, char quote, int cores, size_t* blob_bytes,
                   double* seconds) {
    const auto t0 = std::chrono::steady_clock::now();
    std::string_view csv(b, n);
    std::vector<std::vector<std::string>> cols;
    std::vector<std::string> names;
    size_t i = 0, fs = 0;
    bool inq = false;
    for (; i < n; ++i) {
        const char c = b[i];
        if (c == '\n' || c == '\r') {
            if (i + 1 < n && b[i + 1] == '\n') ++i;
            break;
        }
        if (c == quote) inq = !inq;
        else if (c == delim && !inq) {
            std::string f(b + fs, i - fs);
            if (header) names.push_back(f.empty() ? "NA" : f);
            cols.emplace_back();
            if (!header) cols.back().push_back(f);
            fs = i + 1;
        }
    }
    {
        std::string f(b + fs, i - fs);
        if (header) names.push_back(f.empty() ? "NA" : f);
        cols.emplace_back();
        if (!header) cols.back().push_back(f.empty() ? std::string("NA") : f);
    }
    const unsigned ncol = unsigned(cols.size());
    const size_t start = i + 1 < n ? i + 1 : n;
    if (start < n)
        parse_rows_chunk<std::string, false>(std::string_view(b + start, n - start), cols, delim, quote, ncol, 0);
    size_t nrow = cols[0].size();
    int64_t bad = -1;
    for (auto& c : cols) nrow = std::min(nrow, c.size());
    for (auto& c : cols)
        if (c.size() != nrow) bad = int64_t(nrow);
    std::vector<char> types(ncol);
    std::vector<std::vector<double>> dv(ncol);
    std::vector<std::vector<unsigned>> uv(ncol);
    std::vector<std::vector<uint8_t>> bv(ncol);
    if (bad < 0) {
#pragma omp parallel for num_threads(cores) schedule(dynamic, 1)
        for (unsigned k = 0; k < ncol; ++k) {
            const auto& v = cols[k];
            bool is_bool = true, is_nb = true, is_bufchar = true;
            char ty = 0;
            const size_t chk = std::min<size_t>(v.size(), 10);
            for (size_t r = 0; r < chk && !ty; ++r) {
                const std::string_view s = v[r];
                if (!simd_can_be_nb(s.data(), s.size())) {
                    is_nb = false;
                    if (s.size() > 1) {
                        is_bufchar = false;
                        break;
                    }
                    continue;
                }
                if (has_dot(s)) ty = 'd';
                else if (s != "0" && s != "1") is_bool = false;
            }
            if (!ty) ty = !is_nb ? (is_bufchar ? 'c' : 's') : (is_bool ? 'b' : 'u');
            types[k] = ty;
            if (ty == 'd') {
                dv[k].reserve(nrow);
                for (const auto& el : v) {
                    double x;
                    auto [p, ec] = fast_float::from_chars(el.data(), el.data() + el.size(), x);
                    dv[k].push_back(ec == std::errc() ? x : 0.0);
                }
            } else if (ty == 'u') {
                uv[k].reserve(nrow);
                for (const auto& el : v) {
                    unsigned x;
                    auto [p, ec] = std::from_chars(el.data(), el.data() + el.size(), x);
                    uv[k].push_back(ec == std::errc() ? x : 0u);
                }
            } else if (ty == 'b') {
                bv[k].reserve(nrow);
                for (const auto& el : v) {
                    int x;
                    auto [p, ec] = std::from_chars(el.data(), el.data() + el.size(), x);
                    bv[k].push_back(ec == std::errc() ? (x != 0) : 0);
                }
            }
        }
    }
    if (seconds) seconds[0] = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    std::string blob;
    auto put = [&](const void* p, size_t k) { blob.append(static_cast<const char*>(p), k); };
    const uint64_t nrow_out = bad >= 0 ? 0 : nrow;
    const uint32_t pad = 0;
    put(&nrow_out, 8);
    put(&ncol, 4);
    put(&pad, 4);
    put(&bad, 8);
    for (unsigned k = 0; k < ncol; ++k) {
        const uint8_t ty = uint8_t(types[k] ? types[k] : 's');
        put(&ty, 1);
        const std::string nm = header ? names[k] : std::string();
        const uint32_t nl = uint32_t(nm.size());
        put(&nl, 4);
        put(nm.data(), nl);
    }
    if (nrow_out)
        for (unsigned k = 0; k < ncol; ++k) {
            const char ty = types[k];
            if (ty == 'd') put(dv[k].data(), 8 * nrow);
            else if (ty == 'u') put(uv[k].data(), 4 * nrow);
            else if (ty == 'b') put(bv[k].data(), nrow);
            else {
                uint64_t off = 0;
                put(&off, 8);
                for (size_t r = 0; r < nrow; ++r) {
                    off += cols[k][r].size();
                    put(&off, 8);
                }
                for (size_t r = 0; r < nrow; ++r) put(cols[k][r].data(), cols[k][r].size());
            }
        }
    void* out = malloc(blob.size() ? blob.size() : 1);
    if (out) memcpy(out, blob.data(), blob.size());
    if (blob_bytes) *blob_bytes = blob.size();
    return out;
}

// One-call timing of the reference path on `reps` repetitions (for the CPU
// baseline): returns the best parse + inference + conversion seconds.
double ref_csv_time(const char* b, size_t n, char delim, int header, char quote, int cores, int reps) {
    double best = 1e30;
    for (int r = 0; r < reps; ++r) {
        double s = 0;
        size_t bytes = 0;
        void* p = ref_csv_read(b, n, delim, header, quote, cores, &bytes, &s);
        free(p);
        best = std::min(best, s);
    }
    return best;
}

void ref_csv_free(void* p) { free(p); }

}  // extern "C"
