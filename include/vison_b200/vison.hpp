// vison_b200/vison.hpp -- header-only C++ dataframe layer over libvdf_b200.
//
// It keeps the reference's sort and group-by entry points (VisonDF's
// vison::Dataframe, include/vison/vison.hpp:187-616) with their template
// signatures, so code written against them compiles unchanged, while the work
// runs on the GPU through the C-ABI in vdf_capi.h:
//
//   sort_by / sort_by_mt          transform/sort_by/sort_by.hpp:3-19, sort_by_mt.hpp:3-180
//   sort_by_external[_mt]         transform/sort_by/sort_by_external_mt.hpp:3-130
//   materialize / materialize_mt  materialize/materialize_mt.hpp:3-55
//   transform_group_by[_mt]       transform/transform_group_by/transform_group_by.hpp:3-113,
//                                 transform_group_by_mt.hpp:3-114
//   transform_unique[_mt]         transform/transform_unique/transform_unique_mt.hpp:3-11
//   transform_left_join[_mt]      transform/transform_left_join/transform_left_join_mt.hpp:3-15
//                                 (methods First, Last and Aligned)
//   pivot                         pivots/pivot.hpp:5-128 (vdf_pivot_host)
//   readf                         read/read_csv/read_csv.hpp:3-216 (called as readf in
//                                 benchmarks/readf.cpp:21): the file is parsed on the GPU
//                                 (vdf_csv_read_host) into the frame's type blocks
//
// Storage follows the reference: column-major type blocks (here int_v, uint_v,
// dbl_v plus 64-bit integer blocks lint_v / luint_v, which the reference lacks:
// it has one signed width per frame, so an int32 key and an int64 value cannot
// share a frame), a per-column type char, and a lazy row view (row_view_idx +
// in_view) that Soft sorts set and materialize() applies.  String ('s'),
// one-byte string ('c') and bool ('b') columns come from readf; they are kept,
// viewed and permuted with the frame but are not sort or group-by keys here.
//
// Template parameters that tune the reference's CPU code (CORES, Simd,
// SortType, comparator factories, SimdHash, MapCol, NPerGroup) are accepted
// and ignored: the GPU path has one implementation.  Errors follow the
// reference's convention (a message on std::cerr and an early return,
// sort_by_mt.hpp:16-18,40-41,68-69).
//
// Semantics defined by this layer (documented deviations):
//   * descending sorts reproduce the reference CODE (ascending + std::reverse,
//     sort_integers.inl:225-227: ties in reverse row order); define
//     VISON_B200_STABLE_DESCENDING for the stable order INTERNALS.doc shows;
//   * a Soft sort while in view sorts the rows as currently viewed (the
//     reference re-sorts the raw column, sort_by_mt.hpp:99,111,169-176);
//   * GroupFunction::Mean is sum / group count (the reference divides by the
//     frame's row count, create_value_col.inl:46); Min and Max are added;
//   * GroupFunction::Gather calls the user function f once per group on the
//     group's values in row order (transform_group_by_alrd_mt.hpp:245-260:
//     value_col[i] = f(val_grp[grp_by[i]].v)); the groups and their values
//     come from the GPU sort + group-by with the value column as payload, f
//     runs on the host.  The element type of f's vector argument is taken
//     from a function pointer's signature (group_function_assertion.inl:3-13),
//     else it is the value column's own type.  GroupFunction::None takes the
//     same path.
#pragma once

#include <charconv>
#include <cstdint>
#include <iostream>
#include <map>
#include <memory>
#include <mutex>
#include <numeric>
#include <string>
#include <type_traits>
#include <vector>

#include "../vdf_capi.h"

namespace vison_b200 {

enum class SortType { Standard, Radix };  // supported_sorting_methods.inl:1-4 (both: the stable GPU radix sort)

// supported_group_methods.inl:1-7, plus Min and Max
enum class GroupFunction { Occurence, Sum, Mean, Gather, None, Min, Max };

// types/supported_leftjoin_methods.inl:1-5
enum class LeftJoinMethods { First, Last, Aligned };

struct DefaultTypes {  // types/inference_type.hpp:3-8 (CharT omitted: no char columns here)
    using IntT = int;
    using UIntT = unsigned int;
    using FloatT = double;
};

struct DefaultComparatorFactory {};  // types/comparator.inl:1-11; accepted, unused

// group_function_assertion.inl:22-25: the first value of the group (0 for none)
inline int default_groupfn_impl(std::vector<int>& v) { return v.empty() ? 0 : v[0]; }

// One library context per device, created on first use (the reference's
// init_openmp, vison.hpp:57-74, is likewise process-wide state).
inline vdf_ctx* context(int device = 0) {
    static std::mutex mu;
    static std::map<int, std::unique_ptr<vdf_ctx, vdf_status (*)(vdf_ctx*)>> ctxs;
    std::lock_guard<std::mutex> lk(mu);
    auto it = ctxs.find(device);
    if (it != ctxs.end()) return it->second.get();
    vdf_ctx* c = nullptr;
    if (vdf_ctx_create(device, &c) != VDF_OK) return nullptr;
    ctxs.emplace(device, std::unique_ptr<vdf_ctx, vdf_status (*)(vdf_ctx*)>(c, vdf_ctx_destroy));
    return c;
}

namespace detail {
template <typename T> constexpr int32_t dtype_of() {
    if constexpr (std::is_same_v<T, int32_t>) return VDF_I32;
    else if constexpr (std::is_same_v<T, int64_t> || (std::is_same_v<T, long> && sizeof(long) == 8)) return VDF_I64;
    else if constexpr (std::is_same_v<T, uint32_t>) return VDF_U32;
    else if constexpr (std::is_same_v<T, uint64_t> || (std::is_same_v<T, unsigned long> && sizeof(long) == 8))
        return VDF_U64;
    else if constexpr (std::is_same_v<T, double>) return VDF_F64;
    else if constexpr (std::is_same_v<T, float>) return VDF_F32;
    else return -1;
}
inline bool report(vdf_status s, const char* what) {
    if (s == VDF_OK) return true;
    vdf_ctx* c = context();
    std::cerr << what << ": " << vdf_status_string(s);
    if (c && *vdf_ctx_last_error(c)) std::cerr << " (" << vdf_ctx_last_error(c) << ")";
    std::cerr << "\n";
    return false;
}
// element type of a group function's vector argument: from a function
// pointer's or a (non-generic) lambda's signature; void when neither tells
template <typename M> struct member_arg { using type = void; };
template <typename C, typename R, typename T> struct member_arg<R (C::*)(std::vector<T>&) const> { using type = T; };
template <typename C, typename R, typename T> struct member_arg<R (C::*)(std::vector<T>&)> { using type = T; };
template <typename F, typename = void> struct group_arg { using type = void; };
template <typename R, typename T> struct group_arg<R (*)(std::vector<T>&), void> { using type = T; };
template <typename F>
struct group_arg<F, std::void_t<decltype(&F::operator())>> : member_arg<decltype(&F::operator())> {};

template <bool ASC>
constexpr int32_t order() {
#ifdef VISON_B200_STABLE_DESCENDING
    return ASC ? VDF_ORDER_ASC : VDF_ORDER_DESC_STABLE;
#else
    return ASC ? VDF_ORDER_ASC : VDF_ORDER_DESC_REVERSE;
#endif
}
}  // namespace detail

template <typename Types = DefaultTypes>
class Dataframe {
  public:
    using IntT = typename Types::IntT;
    using UIntT = typename Types::UIntT;
    using FloatT = typename Types::FloatT;
    using LIntT = int64_t;
    using LUIntT = uint64_t;

    unsigned int nrow = 0;
    unsigned int ncol = 0;
    bool in_view = false;
    std::vector<size_t> row_view_idx;

    std::vector<std::vector<IntT>> int_v;      // 'i'
    std::vector<std::vector<UIntT>> uint_v;    // 'u'
    std::vector<std::vector<FloatT>> dbl_v;    // 'd'
    std::vector<std::vector<LIntT>> lint_v;    // 'l' (extension)
    std::vector<std::vector<LUIntT>> luint_v;  // 'L' (extension)
    std::vector<std::vector<std::string>> str_v;  // 's' and 'c'
    std::vector<std::vector<uint8_t>> bool_v;     // 'b'
    std::vector<char> type_refv;               // type char of each column
    std::vector<unsigned int> slot_v;          // index of each column inside its type block
    std::vector<std::string> name_v;
    std::vector<std::string> name_v_row;       // row names (set by pivot, as in the reference)

    // ---- building and reading ------------------------------------------------
    template <typename T>
    void add_col(std::vector<T> v, std::string name = "") {
        if (ncol == 0) nrow = (unsigned int)v.size();
        if (v.size() != nrow) {
            std::cerr << "add_col: column has " << v.size() << " rows, frame has " << nrow << "\n";
            return;
        }
        if (in_view) materialize();
        char t;
        unsigned int slot;
        if constexpr (std::is_same_v<T, IntT>) { t = 'i'; slot = (unsigned)int_v.size(); int_v.push_back(std::move(v)); }
        else if constexpr (std::is_same_v<T, UIntT>) { t = 'u'; slot = (unsigned)uint_v.size(); uint_v.push_back(std::move(v)); }
        else if constexpr (std::is_same_v<T, FloatT>) { t = 'd'; slot = (unsigned)dbl_v.size(); dbl_v.push_back(std::move(v)); }
        else if constexpr (std::is_same_v<T, LIntT>) { t = 'l'; slot = (unsigned)lint_v.size(); lint_v.push_back(std::move(v)); }
        else if constexpr (std::is_same_v<T, LUIntT>) { t = 'L'; slot = (unsigned)luint_v.size(); luint_v.push_back(std::move(v)); }
        else if constexpr (std::is_same_v<T, std::string>) { t = 's'; slot = (unsigned)str_v.size(); str_v.push_back(std::move(v)); }
        else if constexpr (std::is_same_v<T, uint8_t>) { t = 'b'; slot = (unsigned)bool_v.size(); bool_v.push_back(std::move(v)); }
        else { static_assert(!sizeof(T), "unsupported column type"); }
        type_refv.push_back(t);
        slot_v.push_back(slot);
        name_v.push_back(name.empty() ? "col" + std::to_string(ncol + 1) : std::move(name));
        ++ncol;
    }

    // ---- CSV ingest --------------------------------------------------------------
    // read_csv / readf: replaces the frame with the file's columns, parsed on
    // the GPU.  strt_row / end_row other than 0 keep records [strt_row, end_row)
    // (end_row 0: to the end); CORES, WARMING, MEM_CLEAN and TrailingChar tune
    // the reference's CPU parser and are accepted and ignored.  Errors (file
    // not found, a record with another field count) go to std::cerr and leave
    // the frame empty.
    template <unsigned int strt_row = 0, unsigned int end_row = 0, unsigned int CORES = 1, bool WARMING = 0,
              bool MEM_CLEAN = 0, char TrailingChar = '0'>
    void readf(std::string& file_name, char delim = ',', bool header_name = 1, char str_context = '\'') {
        *this = Dataframe();
        std::FILE* f = std::fopen(file_name.c_str(), "rb");
        if (!f) {
            std::cerr << "Failed to open file: " << file_name << "\n";
            return;
        }
        std::vector<char> bytes;
        char chunk[1 << 16];
        size_t got;
        while ((got = std::fread(chunk, 1, sizeof chunk, f)) > 0) bytes.insert(bytes.end(), chunk, chunk + got);
        std::fclose(f);
        vdf_csv* t = nullptr;
        if (!detail::report(vdf_csv_read_host(context(), bytes.data(), bytes.size(), delim, header_name ? 1 : 0,
                                              str_context, &t, nullptr),
                            "readf"))
            return;
        const uint64_t n = vdf_csv_nrow(t);
        const uint64_t r0 = strt_row < n ? strt_row : n;
        const uint64_t r1 = (end_row == 0 || end_row > n) ? n : (end_row < r0 ? r0 : end_row);
        bool ok = true;
        for (uint32_t c = 0; c < vdf_csv_ncol(t) && ok; ++c) {
            const char ty = vdf_csv_type(t, c);
            std::string name = vdf_csv_name(t, c);
            if (ty == 'd' || ty == 'u' || ty == 'b') {
                const size_t w = ty == 'd' ? 8 : ty == 'u' ? 4 : 1;
                std::vector<unsigned char> raw(w * n);
                ok = detail::report(vdf_csv_copy_column(context(), t, c, raw.data(), nullptr, nullptr), "readf");
                auto cut = [&](auto* p, auto& block) {
                    block.emplace_back(p + r0, p + r1);
                };
                if (ty == 'd') cut(reinterpret_cast<const double*>(raw.data()), dbl_v);
                else if (ty == 'u') cut(reinterpret_cast<const uint32_t*>(raw.data()), uint_v);
                else cut(raw.data(), bool_v);
                slot_v.push_back(ty == 'd' ? (unsigned)dbl_v.size() - 1 : ty == 'u' ? (unsigned)uint_v.size() - 1
                                                                                     : (unsigned)bool_v.size() - 1);
            } else {
                std::vector<unsigned char> data(vdf_csv_string_bytes(t, c) + 1);
                std::vector<uint64_t> off(n + 1);
                ok = detail::report(vdf_csv_copy_column(context(), t, c, data.data(), off.data(), nullptr), "readf");
                std::vector<std::string> col;
                col.reserve(r1 - r0);
                for (uint64_t r = r0; r < r1; ++r)
                    col.emplace_back(reinterpret_cast<const char*>(data.data()) + off[r], off[r + 1] - off[r]);
                str_v.push_back(std::move(col));
                slot_v.push_back((unsigned)str_v.size() - 1);
            }
            type_refv.push_back(ty);
            name_v.push_back(std::move(name));
        }
        vdf_csv_free(t);
        if (!ok) {
            *this = Dataframe();
            return;
        }
        ncol = (unsigned int)type_refv.size();
        nrow = (unsigned int)(r1 - r0);
    }

    const std::vector<char>& get_typecol() const { return type_refv; }
    void reinitiate() { *this = Dataframe(); }  // vison.hpp: back to an empty frame
    unsigned int get_nrow() const { return nrow; }
    unsigned int get_ncol() const { return ncol; }

    // Column n as currently viewed (through row_view_idx when in view).
    template <typename T>
    std::vector<T> get_col(unsigned int n) const {
        const std::vector<T>* src = col_ptr<T>(n);
        if (!src) return {};
        if (!in_view) return *src;
        std::vector<T> out(nrow);
        for (unsigned int r = 0; r < nrow; ++r) out[r] = (*src)[row_view_idx[r]];
        return out;
    }

    // ---- sort ------------------------------------------------------------------
    template <bool ASC = 1, typename T = void, bool Simd = true, bool Soft = true, SortType S = SortType::Radix,
              typename Cmp = DefaultComparatorFactory>
    void sort_by(unsigned int& n) {
        sort_by_mt<ASC, 1, T, Simd, Soft, S, Cmp>(n);
    }

    template <bool ASC = 1, unsigned int CORES = 4, typename T = void, bool Simd = true, bool Soft = true,
              SortType S = SortType::Radix, typename Cmp = DefaultComparatorFactory>
    void sort_by_mt(unsigned int& n) {
        if (!Soft && in_view) {
            std::cerr << "Can't use this operation while in `view` mode, consider applying `.materialize()`\n";
            return;
        }
        if (n >= ncol) {
            std::cerr << "Column not found\n";
            return;
        }
        if (!numeric(n)) {
            std::cerr << "sort_by: string and bool columns are not sort keys on the GPU path\n";
            return;
        }
        vdf_col key = col_desc(n);
        sort_rows<ASC, Soft>(&key, 1);
    }

    // Several key columns, most significant first (no reference counterpart:
    // the reference composes single-key sorts, see sort_by_mt.hpp:169-176).
    template <bool ASC = 1, bool Soft = true>
    void sort_by_cols(const std::vector<unsigned int>& cols) {
        if (cols.empty() || cols.size() > 4) {
            std::cerr << "sort_by_cols: 1 to 4 key columns\n";
            return;
        }
        std::vector<vdf_col> keys;
        for (unsigned int c : cols) {
            if (c >= ncol) {
                std::cerr << "Column not found\n";
                return;
            }
            keys.push_back(col_desc(c));
        }
        sort_rows<ASC, Soft>(keys.data(), (int)keys.size());
    }

    template <typename T, bool ASC = true, unsigned int CORES = 4, bool Simd = true, bool Soft = true,
              SortType S = SortType::Radix, bool BoolAsU8 = true, bool IsBoolCompressed = false>
    void sort_by_external_mt(const std::vector<T>& nvec) {
        if (nvec.size() != nrow) {
            std::cerr << "sort vec must be same size as dataframe nrow\n";
            return;
        }
        if (!Soft && in_view) {
            std::cerr << "Can't use this operation while in `view` mode, consider applying `.materialize()`\n";
            return;
        }
        static_assert(detail::dtype_of<T>() >= 0, "sort_by_external: unsupported key type on the GPU path");
        // the external vector is indexed by storage row, like a frame column
        vdf_col key{nvec.data(), detail::dtype_of<T>()};
        sort_rows<ASC, Soft>(&key, 1);
    }

    template <typename T, bool ASC = true, bool Simd = true, bool Soft = true, SortType S = SortType::Radix,
              bool BoolAsU8 = true, bool IsBoolCompressed = false>
    void sort_by_external(const std::vector<T>& nvec) {
        sort_by_external_mt<T, ASC, 1, Simd, Soft, S, BoolAsU8, IsBoolCompressed>(nvec);
    }

    // ---- materialize -------------------------------------------------------------
    template <unsigned int CORES = 4, bool IsDense = true, bool MemClean = false>
    void materialize_mt() {
        if (!in_view) return;
        std::vector<uint32_t> perm(row_view_idx.begin(), row_view_idx.end());
        for (unsigned int c = 0; c < ncol; ++c) permute_col(c, perm);
        in_view = false;
        if (MemClean) std::vector<size_t>().swap(row_view_idx);
        else row_view_idx.clear();
    }

    template <bool IsDense = true, bool MemClean = false>
    void materialize() {
        materialize_mt<1, IsDense, MemClean>();
    }

    // ---- group-by (transform semantics: one new column, a value per row) ------
    template <typename TContainer = void, typename TColVal = void, GroupFunction Function = GroupFunction::Occurence,
              bool SimdHash = true, bool MapCol = false, unsigned int NPerGroup = 4,
              typename F = decltype(&default_groupfn_impl)>
    void transform_group_by(const std::vector<unsigned int>& x, const unsigned int n_col,
                            const std::string colname = "n", const F f = &default_groupfn_impl) {
        transform_group_by_mt<TContainer, TColVal, 1, Function, SimdHash, MapCol, NPerGroup, F>(x, n_col, colname, f);
    }

    template <typename TContainer = void, typename TColVal = void, unsigned int CORES = 4,
              GroupFunction Function = GroupFunction::Occurence, bool SimdHash = true, bool MapCol = false,
              unsigned int NPerGroup = 4, typename F = decltype(&default_groupfn_impl)>
    void transform_group_by_mt(const std::vector<unsigned int>& x, const unsigned int n_col,
                               const std::string colname = "n", const F f = &default_groupfn_impl) {
        (void)f;
        if constexpr (Function == GroupFunction::Gather || Function == GroupFunction::None) {
            gather_group_by(x, n_col, colname, f);
        } else {
            if (x.empty() || x.size() > 4 || n_col >= ncol) {
                std::cerr << "transform_group_by: bad key or value column\n";
                return;
            }
            std::vector<vdf_col> keys;
            for (unsigned int c : x) {
                if (c >= ncol) {
                    std::cerr << "Column not found\n";
                    return;
                }
                if (!numeric(c)) {
                    std::cerr << "transform_group_by: string and bool columns are not keys on the GPU path\n";
                    return;
                }
                keys.push_back(col_desc(c));
            }
            if (!numeric(n_col)) {
                std::cerr << "transform_group_by: string and bool columns are not value columns on the GPU path\n";
                return;
            }
            const vdf_col val = col_desc(n_col);
            int32_t fn = VDF_AGG_COUNT;
            if (Function == GroupFunction::Sum) fn = VDF_AGG_SUM;
            else if (Function == GroupFunction::Mean) fn = VDF_AGG_MEAN;
            else if (Function == GroupFunction::Min) fn = VDF_AGG_MIN;
            else if (Function == GroupFunction::Max) fn = VDF_AGG_MAX;
            std::vector<uint32_t> view;
            if (in_view) view.assign(row_view_idx.begin(), row_view_idx.end());
            const char vt = type_refv[n_col];
            const bool vfloat = (vt == 'd');
            uint64_t groups = 0;
            auto run = [&](void* out) {
                return detail::report(vdf_transform_groupby_host(context(), nrow, keys.data(), (int)keys.size(), val, fn,
                                                                 in_view ? view.data() : nullptr, out, &groups,
                                                                 nullptr),
                                      "transform_group_by");
            };
            // the new column is in storage order; when the frame is in view the
            // view applies to it like to every other column
            if (fn == VDF_AGG_COUNT) {
                std::vector<int64_t> out(nrow);
                if (!run(out.data())) return;
                add_raw(std::vector<UIntT>(out.begin(), out.end()), colname);
            } else if (fn == VDF_AGG_MEAN || (fn == VDF_AGG_SUM && vfloat)) {
                std::vector<double> out(nrow);
                if (!run(out.data())) return;
                add_raw(std::vector<FloatT>(out.begin(), out.end()), colname);
            } else if (fn == VDF_AGG_SUM) {
                std::vector<int64_t> out(nrow);  // low 64 bits of the exact sum
                if (!run(out.data())) return;
                add_like(vt, out, colname);
            } else {
                dispatch_minmax(vt, run, colname);
            }
        }
    }

    // ---- pivot --------------------------------------------------------------------
    // pivots/pivot.hpp:5-128: this frame becomes the pivot of obj -- one column
    // (named by the key) per distinct value of column n1, one row (name_v_row)
    // per distinct value of column n2, both in order of first appearance, and
    // in each cell the sum of column n3 over the rows of that pair (0 for a
    // pair that never occurs).  Keys compare as the text of their cells: the
    // strings of 's' / 'c' columns, the decimal text of numbers (the reference
    // keys on each cell's text as read).  Column n3 holds T (IntT, UIntT or
    // FloatT as in the reference, or the 64-bit integer types); integer sums
    // wrap in T like the reference's "+=", f64 sums are compensated.  The
    // rows of obj are read as viewed.
    template <typename T, bool SimdHash = true>
    void pivot(Dataframe& obj, unsigned int& n1, unsigned int& n2, unsigned int& n3) {
        (void)SimdHash;
        if (n1 >= obj.ncol || n2 >= obj.ncol || n3 >= obj.ncol) {
            std::cerr << "Column not found\n";
            return;
        }
        const std::vector<T>* vals = obj.template col_ptr<T>(n3);
        if (!vals) {
            std::cerr << "Unsupported type for pivots\n";
            return;
        }
        const unsigned int n = obj.nrow;
        auto row_of = [&](unsigned int i) -> unsigned int { return obj.in_view ? (unsigned)obj.row_view_idx[i] : i; };
        std::vector<std::string> ck = obj.cell_text(n1), rk = obj.cell_text(n2);
        std::vector<char> cb, rb;
        std::vector<uint64_t> co(n + 1, 0), ro(n + 1, 0);
        std::vector<T> v(n);
        for (unsigned int i = 0; i < n; ++i) {
            const unsigned int r = row_of(i);
            cb.insert(cb.end(), ck[r].begin(), ck[r].end());
            rb.insert(rb.end(), rk[r].begin(), rk[r].end());
            co[i + 1] = cb.size();
            ro[i + 1] = rb.size();
            v[i] = (*vals)[r];
        }
        cb.push_back(0);
        rb.push_back(0);
        uint32_t nc = 0, nr = 0;
        std::vector<uint32_t> cfirst(std::max(1u, n)), rfirst(std::max(1u, n));
        const vdf_col vc{v.data(), detail::dtype_of<T>()};
        const vdf_strcol cs{cb.data(), co.data()}, rs{rb.data(), ro.data()};
        vdf_status st = vdf_pivot_host(context(), n, cs, rs, vc, &nc, &nr, cfirst.data(), rfirst.data(), nullptr, 0);
        if (st != VDF_OK && st != VDF_ERR_WORKSPACE) {
            detail::report(st, "pivot");
            return;
        }
        std::vector<T> cells((size_t)nc * nr);
        st = vdf_pivot_host(context(), n, cs, rs, vc, &nc, &nr, cfirst.data(), rfirst.data(), cells.data(),
                            cells.size());
        if (!detail::report(st, "pivot")) return;
        Dataframe out;
        for (uint32_t c = 0; c < nc; ++c)
            out.add_col(std::vector<T>(cells.begin() + (size_t)c * nr, cells.begin() + (size_t)(c + 1) * nr),
                        ck[row_of(cfirst[c])]);
        out.nrow = nr;
        out.name_v_row.resize(nr);
        for (uint32_t r = 0; r < nr; ++r) out.name_v_row[r] = rk[row_of(rfirst[r])];
        *this = std::move(out);
    }

    // Text of every cell of column n in storage order (strings as they are,
    // integers in decimal, doubles in their shortest round-trip form, bools
    // as 0 / 1).
    std::vector<std::string> cell_text(unsigned int n) const {
        const unsigned s = slot_v[n];
        std::vector<std::string> out(nrow);
        auto num = [&](const auto& vec) {
            char buf[64];
            for (unsigned int r = 0; r < nrow; ++r) {
                auto res = std::to_chars(buf, buf + sizeof(buf), vec[r]);
                out[r].assign(buf, res.ptr);
            }
        };
        switch (type_refv[n]) {
        case 'i': num(int_v[s]); break;
        case 'u': num(uint_v[s]); break;
        case 'd': num(dbl_v[s]); break;
        case 'l': num(lint_v[s]); break;
        case 'L': num(luint_v[s]); break;
        case 'b':
            for (unsigned int r = 0; r < nrow; ++r) out[r] = bool_v[s][r] ? "1" : "0";
            break;
        default: out = str_v[s]; break;
        }
        return out;
    }

    // ---- de-duplication ------------------------------------------------------------
    // transform_unique_mt.hpp:3-11: keeps, in row order, the first (Last =
    // false) or last occurrence of each value of column n, values compared by
    // their bytes.  A frame in view is materialised first (Soft = true; with
    // Soft = false a view is an error, as in the reference).
    template <typename T = void, unsigned int CORES = 4, bool MemClean = false, bool Last = false,
              bool MapCol = false, bool Soft = true, bool SimdHash = true>
    void transform_unique_mt(unsigned int n) {
        if (in_view && !Soft) {
            std::cerr << "Can't perform this operation while in `view` mode, consider applying `.materialize()`\n";
            return;
        }
        if (n >= ncol) {
            std::cerr << "Column not found\n";
            return;
        }
        if (!numeric(n)) {
            std::cerr << "transform_unique: string and bool columns are not keys on the GPU path\n";
            return;
        }
        if (in_view) materialize();
        std::vector<uint8_t> keep(nrow);
        uint64_t distinct = 0;
        if (!detail::report(vdf_unique_host(context(), nrow, col_desc(n), Last ? 1 : 0, keep.data(), &distinct, nullptr),
                            "transform_unique"))
            return;
        std::vector<uint32_t> rows;
        rows.reserve(distinct);
        for (unsigned int r = 0; r < nrow; ++r)
            if (keep[r]) rows.push_back(r);
        keep_rows(rows);
    }
    template <typename T = void, bool MemClean = false, bool Last = false, bool MapCol = false, bool Soft = true,
              bool SimdHash = true>
    void transform_unique(unsigned int n) {
        transform_unique_mt<T, 1, MemClean, Last, MapCol, Soft, SimdHash>(n);
    }

    // ---- left join ---------------------------------------------------------------------
    // transform_left_join_mt.hpp:3-15: appends obj's columns; row i takes the
    // values of obj's first (First) or last (Last) row whose key2 equals this
    // frame's key1 at row i -- or, Aligned, the k-th such row for the key's
    // k-th occurrence here -- or the per-type default where there is none.
    template <typename T = void, unsigned int CORES = 4, bool SimdHash = true,
              LeftJoinMethods Method = LeftJoinMethods::First>
    void transform_left_join_mt(const Dataframe& obj, const unsigned int key1, const unsigned int key2,
                                const char default_chr, const std::string default_str = "NA",
                                const uint8_t default_bool = 0, const IntT default_int = 0,
                                const UIntT default_uint = 0, const FloatT default_dbl = 0) {
        (void)default_chr;
        if (in_view) {
            std::cerr << "Can't perform this operation while in`view` mode, consider applying `.materialize()`\n";
            return;
        }
        {
            if (key1 >= ncol || key2 >= obj.ncol) {
                std::cerr << "Column not found\n";
                return;
            }
            if (!numeric(key1) || !obj.numeric(key2)) {
                std::cerr << "transform_left_join: string and bool columns are not keys on the GPU path\n";
                return;
            }
            if (type_refv[key1] != obj.type_refv[key2]) {
                std::cerr << "transform_left_join: key columns differ in type\n";
                return;
            }
            Dataframe right = obj;  // obj as viewed
            if (right.in_view) right.materialize();
            std::vector<uint32_t> match(nrow);
            uint64_t matched = 0;
            if (!detail::report(vdf_left_join_index_host(context(), nrow, col_desc(key1), right.nrow,
                                                         right.col_desc(key2),
                                                         Method == LeftJoinMethods::First  ? VDF_JOIN_FIRST
                                                         : Method == LeftJoinMethods::Last ? VDF_JOIN_LAST
                                                                                           : VDF_JOIN_ALIGNED,
                                                         match.data(),
                                                         &matched, nullptr),
                                "transform_left_join"))
                return;
            for (unsigned int c = 0; c < right.ncol; ++c) {
                const unsigned s = right.slot_v[c];
                const std::string name = right.name_v[c];
                auto join = [&](const auto& src, auto dflt) {
                    using V = typename std::decay_t<decltype(src)>::value_type;
                    std::vector<V> out(nrow);
                    for (unsigned int r = 0; r < nrow; ++r) out[r] = match[r] == 0xffffffffu ? (V)dflt : src[match[r]];
                    add_col(std::move(out), name);
                };
                switch (right.type_refv[c]) {
                case 'i': join(right.int_v[s], default_int); break;
                case 'u': join(right.uint_v[s], default_uint); break;
                case 'd': join(right.dbl_v[s], default_dbl); break;
                case 'l': join(right.lint_v[s], (LIntT)default_int); break;
                case 's': case 'c': join(right.str_v[s], default_str); break;
                case 'b': join(right.bool_v[s], default_bool); break;
                default: join(right.luint_v[s], (LUIntT)default_uint); break;
                }
            }
        }
    }
    template <typename T = void, bool SimdHash = true, LeftJoinMethods Method = LeftJoinMethods::First>
    void transform_left_join(const Dataframe& obj, const unsigned int key1, const unsigned int key2,
                             const char default_chr, const std::string default_str = "NA",
                             const uint8_t default_bool = 0, const IntT default_int = 0, const UIntT default_uint = 0,
                             const FloatT default_dbl = 0) {
        transform_left_join_mt<T, 1, SimdHash, Method>(obj, key1, key2, default_chr, default_str, default_bool,
                                                       default_int, default_uint, default_dbl);
    }

  private:
    // Keeps storage rows `rows` (ascending) of every column.
    void keep_rows(const std::vector<uint32_t>& rows) {
        for (unsigned int c = 0; c < ncol; ++c) {
            const unsigned s = slot_v[c];
            auto go = [&](auto& vec) {
                using V = typename std::decay_t<decltype(vec)>::value_type;
                std::vector<V> out(rows.size());
                for (size_t i = 0; i < rows.size(); ++i) out[i] = vec[rows[i]];
                vec.swap(out);
            };
            switch (type_refv[c]) {
            case 'i': go(int_v[s]); break;
            case 'u': go(uint_v[s]); break;
            case 'd': go(dbl_v[s]); break;
            case 'l': go(lint_v[s]); break;
            case 's': case 'c': go(str_v[s]); break;
            case 'b': go(bool_v[s]); break;
            default: go(luint_v[s]); break;
            }
        }
        nrow = (unsigned int)rows.size();
        row_view_idx.clear();
        in_view = false;
    }

    template <typename T>
    const std::vector<T>* col_ptr(unsigned int n) const {
        if (n >= ncol) return nullptr;
        const unsigned s = slot_v[n];
        switch (type_refv[n]) {
        case 'i': if constexpr (std::is_same_v<T, IntT>) return &int_v[s]; break;
        case 'u': if constexpr (std::is_same_v<T, UIntT>) return &uint_v[s]; break;
        case 'd': if constexpr (std::is_same_v<T, FloatT>) return &dbl_v[s]; break;
        case 'l': if constexpr (std::is_same_v<T, LIntT>) return &lint_v[s]; break;
        case 'L': if constexpr (std::is_same_v<T, LUIntT>) return &luint_v[s]; break;
        case 's': case 'c': if constexpr (std::is_same_v<T, std::string>) return &str_v[s]; break;
        case 'b': if constexpr (std::is_same_v<T, uint8_t>) return &bool_v[s]; break;
        }
        return nullptr;
    }

    bool numeric(unsigned int n) const {
        const char t = type_refv[n];
        return t == 'i' || t == 'u' || t == 'd' || t == 'l' || t == 'L';
    }

    vdf_col col_desc(unsigned int n) const {
        const unsigned s = slot_v[n];
        switch (type_refv[n]) {
        case 'i': return vdf_col{int_v[s].data(), detail::dtype_of<IntT>()};
        case 'u': return vdf_col{uint_v[s].data(), detail::dtype_of<UIntT>()};
        case 'd': return vdf_col{dbl_v[s].data(), detail::dtype_of<FloatT>()};
        case 'l': return vdf_col{lint_v[s].data(), VDF_I64};
        default: return vdf_col{luint_v[s].data(), VDF_U64};
        }
    }

    // Gather: groups of the key columns (rows seen through the view), the
    // user function over each group's values, its result broadcast to every
    // row of the group (the new column is in storage order).
    template <typename F>
    void gather_group_by(const std::vector<unsigned int>& x, unsigned int n_col, const std::string& colname,
                         const F& f) {
        if (x.empty() || x.size() > 4 || n_col >= ncol) {
            std::cerr << "transform_group_by: bad key or value column\n";
            return;
        }
        std::vector<vdf_col> keys;
        for (unsigned int c : x) {
            if (c >= ncol) {
                std::cerr << "Column not found\n";
                return;
            }
            if (!numeric(c)) {
                std::cerr << "transform_group_by: string and bool columns are not keys on the GPU path\n";
                return;
            }
            keys.push_back(col_desc(c));
        }
        if (!numeric(n_col)) {
            std::cerr << "transform_group_by: string and bool columns are not value columns on the GPU path\n";
            return;
        }
        const unsigned s = slot_v[n_col];
        switch (type_refv[n_col]) {
        case 'i': gather_typed(keys, int_v[s], n_col, colname, f); break;
        case 'u': gather_typed(keys, uint_v[s], n_col, colname, f); break;
        case 'd': gather_typed(keys, dbl_v[s], n_col, colname, f); break;
        case 'l': gather_typed(keys, lint_v[s], n_col, colname, f); break;
        default: gather_typed(keys, luint_v[s], n_col, colname, f); break;
        }
    }

    template <typename V, typename F>
    void gather_typed(const std::vector<vdf_col>& keys, const std::vector<V>& col, unsigned int n_col,
                      const std::string& colname, const F& f) {
        using GA = typename detail::group_arg<F>::type;
        using T = std::conditional_t<std::is_void_v<GA>, V, GA>;
        if constexpr (!std::is_invocable_v<const F&, std::vector<T>&>) {
            std::cerr << "transform_group_by: the group function does not take this column's values\n";
        } else {
            gather_apply<T>(keys, col, n_col, colname, f);
        }
    }

    template <typename T, typename V, typename F>
    void gather_apply(const std::vector<vdf_col>& keys, const std::vector<V>& col, unsigned int n_col,
                      const std::string& colname, const F& f) {
        using R = std::decay_t<std::invoke_result_t<const F&, std::vector<T>&>>;
        static_assert(std::is_arithmetic_v<R>, "a group function returns a number");
        using Out = std::conditional_t<
            std::is_floating_point_v<R>, FloatT,
            std::conditional_t<std::is_signed_v<R>, std::conditional_t<(sizeof(R) > sizeof(IntT)), LIntT, IntT>,
                               std::conditional_t<(sizeof(R) > sizeof(UIntT)), LUIntT, UIntT>>>;
        std::vector<uint32_t> perm(nrow), gstart(nrow + 1);
        std::vector<V> sorted(nrow);
        std::vector<uint32_t> view;
        if (in_view) view.assign(row_view_idx.begin(), row_view_idx.end());
        const vdf_col val = col_desc(n_col);
        void* po = sorted.data();
        uint64_t groups = 0;
        vdf_sort_groupby_args a{};
        a.n = nrow;
        a.keys = keys.data();
        a.nkeys = (int32_t)keys.size();
        a.order = VDF_ORDER_ASC;
        a.payload = &val;
        a.npayload = 1;
        a.perm_out = perm.data();
        a.payload_out = &po;
        a.groupby = 1;
        a.group_start_out = gstart.data();
        a.n_groups_host = &groups;
        a.perm_in = in_view ? view.data() : nullptr;
        if (!detail::report(vdf_sort_groupby_host(context(), &a, nullptr), "transform_group_by")) return;
        (void)col;
        std::vector<Out> out(nrow);
        std::vector<T> vals;
        for (uint64_t g = 0; g < groups; ++g) {
            const uint32_t b = gstart[g], e = g + 1 < groups ? gstart[g + 1] : nrow;
            vals.clear();
            for (uint32_t p = b; p < e; ++p) vals.push_back(static_cast<T>(sorted[p]));
            const Out r = static_cast<Out>(f(vals));
            for (uint32_t p = b; p < e; ++p) out[perm[p]] = r;
        }
        add_raw(std::move(out), colname);
    }

    template <bool ASC, bool Soft>
    void sort_rows(const vdf_col* keys, int nkeys) {
        std::vector<uint32_t> perm(nrow);
        std::vector<uint32_t> view;
        if (in_view) view.assign(row_view_idx.begin(), row_view_idx.end());
        vdf_sort_groupby_args a{};
        a.n = nrow;
        a.keys = keys;
        a.nkeys = nkeys;
        a.order = detail::order<ASC>();
        a.perm_out = perm.data();
        a.perm_in = in_view ? view.data() : nullptr;
        if (!detail::report(vdf_sort_groupby_host(context(), &a, nullptr), "sort_by")) return;
        if (Soft) {
            row_view_idx.assign(perm.begin(), perm.end());
            in_view = true;
        } else {
            for (unsigned int c = 0; c < ncol; ++c) permute_col(c, perm);
        }
    }

    void permute_col(unsigned int c, const std::vector<uint32_t>& perm) {
        const unsigned s = slot_v[c];
        if (!numeric(c)) {  // strings and bools: permuted on the host
            auto host = [&](auto& vec) {
                using V = typename std::decay_t<decltype(vec)>::value_type;
                std::vector<V> out(nrow);
                for (unsigned int r = 0; r < nrow; ++r) out[r] = vec[perm[r]];
                vec.swap(out);
            };
            if (type_refv[c] == 'b') host(bool_v[s]);
            else host(str_v[s]);
            return;
        }
        vdf_col in = col_desc(c);
        auto go = [&](auto& vec) {
            using V = typename std::decay_t<decltype(vec)>::value_type;
            std::vector<V> out(nrow);
            void* o = out.data();
            if (detail::report(vdf_gather_host(context(), nrow, perm.data(), &in, 1, &o, nullptr), "materialize"))
                vec.swap(out);
        };
        switch (type_refv[c]) {
        case 'i': go(int_v[s]); break;
        case 'u': go(uint_v[s]); break;
        case 'd': go(dbl_v[s]); break;
        case 'l': go(lint_v[s]); break;
        default: go(luint_v[s]); break;
        }
    }

    // Appends a column in storage order (transform outputs are computed per
    // storage row), keeping the current view.
    template <typename T>
    void add_raw(std::vector<T> v, const std::string& name) {
        const bool keep = in_view;
        in_view = false;
        add_col(std::move(v), name);
        in_view = keep;
    }

    void add_like(char vt, const std::vector<int64_t>& v, const std::string& name) {
        switch (vt) {
        case 'i': add_raw(std::vector<IntT>(v.begin(), v.end()), name); break;
        case 'u': add_raw(std::vector<UIntT>(v.begin(), v.end()), name); break;
        case 'l': add_raw(std::vector<LIntT>(v.begin(), v.end()), name); break;
        default: add_raw(std::vector<LUIntT>(v.begin(), v.end()), name); break;
        }
    }

    template <typename Run>
    void dispatch_minmax(char vt, Run& run, const std::string& name) {
        switch (vt) {
        case 'i': { std::vector<IntT> o(nrow); if (run(o.data())) add_raw(std::move(o), name); break; }
        case 'u': { std::vector<UIntT> o(nrow); if (run(o.data())) add_raw(std::move(o), name); break; }
        case 'd': { std::vector<FloatT> o(nrow); if (run(o.data())) add_raw(std::move(o), name); break; }
        case 'l': { std::vector<LIntT> o(nrow); if (run(o.data())) add_raw(std::move(o), name); break; }
        default: { std::vector<LUIntT> o(nrow); if (run(o.data())) add_raw(std::move(o), name); break; }
        }
    }
};

}  // namespace vison_b200

#ifdef VISON_B200_AS_VISON
namespace vison = vison_b200;  // drop-in: code written against vison::Dataframe compiles unchanged
#endif
