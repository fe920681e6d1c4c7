/*
 * vdf_oracle.c -- CPU oracle for the sort + group-by path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker that the CUDA path is
 * compared against.  Only tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline leg may load it.  The product library (visondf_b200) never links,
 * loads or calls anything in this directory, and has no CPU fallback.
 *
 * It restates, in plain C, the reference's algorithm for the hot path
 * (paths relative to the reference project, V/ = include/vison/):
 *
 *   - order-preserving key transforms
 *       int32  : UIntT(x) ^ 0x80000000          V/inlines/transform/sort_by/sort_integers.inl:46,109
 *       int64  : UIntT(x) ^ 0x8000000000000000  V/inlines/transform/sort_by/sort_integers.inl:46,123
 *       uint   : identity (plain copy)          V/inlines/transform/sort_by/sort_uintegers.inl:48-74
 *       double : bits ^ (-(bits>>63) | 1<<63)   V/inlines/transform/sort_by/sort_flt.inl:123-129
 *   - stable LSD radix argsort with 16-bit digits, scalar path
 *       u32: 2 passes  V/inlines/radix_sorts/radix_sort_uint32.inl:27-97
 *       u64: 4 passes  V/inlines/radix_sorts/radix_sort_uint64.inl:21-83
 *     (histogram, exclusive scan over 65,536 buckets, stable scatter of
 *      (idx, key), then swap -- the idx array is in/out so a second sort can
 *      refine an existing permutation, which is how multi-key sorts compose)
 *   - descending order: the reference code sorts ascending then applies
 *     std::reverse (sort_integers.inl:225-227); its documentation shows a
 *     stable descending order instead (INTERNALS.doc:1610-1632).  Both are
 *     offered: ORC_DESC_STABLE and ORC_DESC_REVERSE.
 *   - payload gather dst[r] = src[idx[r]]   V/inlines/no_inplace_permutation.inl:3-79,
 *                                           V/inlines/transform/sort_by/permute_block_mt.inl:39-41
 *   - hash group-by: one map entry per distinct raw key byte string, rows
 *     visited in order, "+=" accumulation, first-appearance (insertion) order
 *     V/transform/transform_group_by/transform_group_by_onecol_mt.hpp:182-244,
 *     V/inlines/transform/transform_group_by/onecol_functions.inl:47-86.
 *     Composite keys are the concatenated key bytes (key_build.inl:3-110).
 *     Deviations (fixes, as the GPU path defines them): min and max are added
 *     (the reference has none, supported_group_methods.inl:1-7), mean is
 *     sum/count rather than sum/nrow (create_value_col.inl:46), integer sums
 *     are exact 128-bit, float sums are kept in long double with Neumaier
 *     compensation (so they are exact to ~1e-19 of sum|x|), and groups are
 *     returned in ascending key order (the hash order is kept separately).
 *   - de-duplication and left-join row matching: the reference's set / map
 *     walks over raw key bytes (orc_unique, orc_left_join, at the end of
 *     this file, with their citations).
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <math.h>

enum { ORC_I32 = 0, ORC_I64 = 1, ORC_U32 = 2, ORC_U64 = 3, ORC_F64 = 4, ORC_F32 = 5 };
enum { ORC_ASC = 0, ORC_DESC_STABLE = 1, ORC_DESC_REVERSE = 2 };

int orc_dtype_width(int dt) {
    switch (dt) {
    case ORC_I32: case ORC_U32: case ORC_F32: return 4;
    case ORC_I64: case ORC_U64: case ORC_F64: return 8;
    default: return 0;
    }
}

/* order-preserving unsigned image of element i of a column */
uint64_t orc_order_key(const void* col, int dt, size_t i) {
    switch (dt) {
    case ORC_I32: return (uint32_t)((const int32_t*)col)[i] ^ 0x80000000u;
    case ORC_I64: return (uint64_t)((const int64_t*)col)[i] ^ 0x8000000000000000ull;
    case ORC_U32: return ((const uint32_t*)col)[i];
    case ORC_U64: return ((const uint64_t*)col)[i];
    case ORC_F64: {
        uint64_t b; memcpy(&b, (const double*)col + i, 8);
        uint64_t m = (uint64_t)0 - (b >> 63);
        return b ^ (m | 0x8000000000000000ull);
    }
    case ORC_F32: {
        uint32_t b; memcpy(&b, (const float*)col + i, 4);
        uint32_t m = (uint32_t)0 - (b >> 31);
        return b ^ (m | 0x80000000u);
    }
    default: return 0;
    }
}

#define ORC_KI16 65536u

/* radix_sort_uint32.inl:27-97, scalar branch: two 16-bit passes. */
int orc_radix_u32(uint32_t* keys, uint64_t* idx, size_t n) {
    if (n == 0) return 0;
    uint64_t* count = (uint64_t*)malloc(ORC_KI16 * sizeof(uint64_t));
    uint32_t* tk = (uint32_t*)malloc(n * sizeof(uint32_t));
    uint64_t* ti = (uint64_t*)malloc(n * sizeof(uint64_t));
    if (!count || !tk || !ti) { free(count); free(tk); free(ti); return -1; }
    for (int pass = 0; pass < 2; ++pass) {
        unsigned shift = 16u * (unsigned)pass;
        memset(count, 0, ORC_KI16 * sizeof(uint64_t));
        for (size_t i = 0; i < n; ++i) count[(keys[i] >> shift) & 0xFFFFu]++;
        uint64_t sum = 0;
        for (size_t b = 0; b < ORC_KI16; ++b) { uint64_t c = count[b]; count[b] = sum; sum += c; }
        for (size_t i = 0; i < n; ++i) {
            uint32_t k = keys[i];
            uint64_t pos = count[(k >> shift) & 0xFFFFu]++;
            ti[pos] = idx[i];
            tk[pos] = k;
        }
        memcpy(keys, tk, n * sizeof(uint32_t));
        memcpy(idx, ti, n * sizeof(uint64_t));
    }
    free(count); free(tk); free(ti);
    return 0;
}

/* radix_sort_uint64.inl:21-83, scalar branch: four 16-bit passes. */
int orc_radix_u64(uint64_t* keys, uint64_t* idx, size_t n) {
    if (n == 0) return 0;
    uint64_t* count = (uint64_t*)malloc(ORC_KI16 * sizeof(uint64_t));
    uint64_t* tk = (uint64_t*)malloc(n * sizeof(uint64_t));
    uint64_t* ti = (uint64_t*)malloc(n * sizeof(uint64_t));
    if (!count || !tk || !ti) { free(count); free(tk); free(ti); return -1; }
    for (int pass = 0; pass < 4; ++pass) {
        unsigned shift = 16u * (unsigned)pass;
        memset(count, 0, ORC_KI16 * sizeof(uint64_t));
        for (size_t i = 0; i < n; ++i) count[(keys[i] >> shift) & 0xFFFFu]++;
        uint64_t sum = 0;
        for (size_t b = 0; b < ORC_KI16; ++b) { uint64_t c = count[b]; count[b] = sum; sum += c; }
        for (size_t i = 0; i < n; ++i) {
            uint64_t k = keys[i];
            uint64_t pos = count[(k >> shift) & 0xFFFFu]++;
            ti[pos] = idx[i];
            tk[pos] = k;
        }
        memcpy(keys, tk, n * sizeof(uint64_t));
        memcpy(idx, ti, n * sizeof(uint64_t));
    }
    free(count); free(tk); free(ti);
    return 0;
}

/*
 * Multi-key stable argsort.  cols[0] is the most significant key.  Keys are
 * processed least-significant first; each key column is read through the
 * current permutation (tkeys[i] = key'[P[i]]) and radix-sorted with P as the
 * in/out index, which is the composition the reference's idx parameter
 * allows (radix_sort_uint64.inl:5-7).  Returns 0, or -1 on bad input.
 */
int orc_argsort(const void* const* cols, const int* dtypes, int nkeys, size_t n,
                int order, uint32_t* perm_out) {
    if (nkeys < 1 || (order < 0 || order > 2)) return -1;
    if (n == 0) return 0;
    uint64_t* idx = (uint64_t*)malloc(n * sizeof(uint64_t));
    if (!idx) return -1;
    for (size_t i = 0; i < n; ++i) idx[i] = i;
    for (int k = nkeys - 1; k >= 0; --k) {
        int w = orc_dtype_width(dtypes[k]);
        if (w == 0) { free(idx); return -1; }
        int invert = (order == ORC_DESC_STABLE);
        if (w == 4) {
            uint32_t* tk = (uint32_t*)malloc(n * sizeof(uint32_t));
            if (!tk) { free(idx); return -1; }
            for (size_t i = 0; i < n; ++i) {
                uint32_t v = (uint32_t)orc_order_key(cols[k], dtypes[k], idx[i]);
                tk[i] = invert ? ~v : v;
            }
            int rc = orc_radix_u32(tk, idx, n);
            free(tk);
            if (rc) { free(idx); return -1; }
        } else {
            uint64_t* tk = (uint64_t*)malloc(n * sizeof(uint64_t));
            if (!tk) { free(idx); return -1; }
            for (size_t i = 0; i < n; ++i) {
                uint64_t v = orc_order_key(cols[k], dtypes[k], idx[i]);
                tk[i] = invert ? ~v : v;
            }
            int rc = orc_radix_u64(tk, idx, n);
            free(tk);
            if (rc) { free(idx); return -1; }
        }
    }
    if (order == ORC_DESC_REVERSE) {
        for (size_t i = 0; i < n; ++i) perm_out[i] = (uint32_t)idx[n - 1 - i];
    } else {
        for (size_t i = 0; i < n; ++i) perm_out[i] = (uint32_t)idx[i];
    }
    free(idx);
    return 0;
}

/* dst[r] = src[perm[r]] for one column of `width` bytes per element. */
void orc_gather(const uint32_t* perm, size_t n, const void* src, int width, void* dst) {
    const unsigned char* s = (const unsigned char*)src;
    unsigned char* d = (unsigned char*)dst;
    for (size_t r = 0; r < n; ++r)
        memcpy(d + r * (size_t)width, s + (size_t)perm[r] * (size_t)width, (size_t)width);
}

/* ------------------------------------------------------------------------ */
/* group-by                                                                  */
/* ------------------------------------------------------------------------ */

typedef struct {
    long double fsum, fcomp, fabs_sum;   /* float columns: Neumaier sum, sum |x| */
    __int128 isum;                       /* signed integer columns              */
    unsigned __int128 usum;              /* unsigned integer columns            */
    double fmin, fmax;
    int64_t imin, imax;
    uint64_t umin, umax;
} orc_acc;

static uint64_t orc_mix(uint64_t x) {
    /* 64-bit finaliser of MurmurHash3 (fmix64) */
    x ^= x >> 33; x *= 0xff51afd7ed558ccdull;
    x ^= x >> 33; x *= 0xc4ceb9fe1a85ec53ull;
    x ^= x >> 33;
    return x;
}

static uint64_t orc_row_hash(const void* const* keys, const int* kdt, int nkeys, size_t r) {
    uint64_t h = 0x9e3779b97f4a7c15ull;
    for (int k = 0; k < nkeys; ++k) h = orc_mix(h ^ orc_order_key(keys[k], kdt[k], r)) + (uint64_t)k;
    return h;
}

static int orc_row_eq(const void* const* keys, const int* kdt, int nkeys, size_t a, size_t b) {
    for (int k = 0; k < nkeys; ++k) {
        int w = orc_dtype_width(kdt[k]);
        const unsigned char* c = (const unsigned char*)keys[k];
        if (memcmp(c + a * (size_t)w, c + b * (size_t)w, (size_t)w) != 0) return 0;
    }
    return 1;
}

static const void* const* g_sort_keys;
static const int* g_sort_kdt;
static int g_sort_nkeys;
static const int64_t* g_sort_first;

static int orc_group_cmp(const void* pa, const void* pb) {
    int64_t a = g_sort_first[*(const int64_t*)pa], b = g_sort_first[*(const int64_t*)pb];
    for (int k = 0; k < g_sort_nkeys; ++k) {
        uint64_t ka = orc_order_key(g_sort_keys[k], g_sort_kdt[k], (size_t)a);
        uint64_t kb = orc_order_key(g_sort_keys[k], g_sort_kdt[k], (size_t)b);
        if (ka != kb) return ka < kb ? -1 : 1;
    }
    return 0;
}

/*
 * Hash group-by over nkeys key columns and nvals value columns of n rows.
 * Output arrays (caller-allocated, capacity n, any may be NULL):
 *   out_keys[k][g]       group key columns (raw key values)
 *   out_count[g]         rows per group
 *   out_sum[v][g]        f64 sum for float columns; int64 low word of the
 *                        exact sum for integer columns
 *   out_sum_hi[v][g]     high 64 bits of the 128-bit integer sum (int cols)
 *   out_min[v], out_max[v][g]  in the column's own type
 *   out_mean[v][g]       f64 sum/count
 *   out_abs[v][g]        f64 sum of |x| (float columns), for tolerances
 *   out_first[g]         first row of the group (the hash map's entry order)
 * Groups are written in ascending key order when sorted != 0, else in
 * first-appearance order (the reference's map order).  Returns G, or -1.
 */
int64_t orc_groupby(const void* const* keys, const int* kdt, int nkeys,
                    const void* const* vals, const int* vdt, int nvals, size_t n,
                    int sorted,
                    void* const* out_keys, int64_t* out_count,
                    void* const* out_sum, int64_t* const* out_sum_hi,
                    void* const* out_min, void* const* out_max,
                    double* const* out_mean, double* const* out_abs,
                    int64_t* out_first) {
    if (nkeys < 1 || nvals < 0) return -1;
    for (int k = 0; k < nkeys; ++k) if (orc_dtype_width(kdt[k]) == 0) return -1;
    for (int v = 0; v < nvals; ++v) if (orc_dtype_width(vdt[v]) == 0) return -1;
    if (n == 0) return 0;

    size_t cap = 16;
    while (cap < 2 * n) cap <<= 1;
    int64_t* slots = (int64_t*)malloc(cap * sizeof(int64_t));
    int64_t* first = (int64_t*)malloc(n * sizeof(int64_t));
    int64_t* count = (int64_t*)calloc(n, sizeof(int64_t));
    orc_acc* acc = (orc_acc*)calloc((size_t)(nvals ? nvals : 1) * n, sizeof(orc_acc));
    if (!slots || !first || !count || !acc) {
        free(slots); free(first); free(count); free(acc); return -1;
    }
    memset(slots, 0xff, cap * sizeof(int64_t));
    int64_t G = 0;
    for (size_t r = 0; r < n; ++r) {
        size_t s = (size_t)orc_row_hash(keys, kdt, nkeys, r) & (cap - 1);
        int64_t g;
        for (;;) {
            g = slots[s];
            if (g < 0) { g = G++; slots[s] = g; first[g] = (int64_t)r; break; }
            if (orc_row_eq(keys, kdt, nkeys, (size_t)first[g], r)) break;
            s = (s + 1) & (cap - 1);
        }
        int fresh = (count[g] == 0);
        count[g]++;
        for (int v = 0; v < nvals; ++v) {
            orc_acc* a = &acc[(size_t)v * n + (size_t)g];
            switch (vdt[v]) {
            case ORC_F64: case ORC_F32: {
                double x = vdt[v] == ORC_F64 ? ((const double*)vals[v])[r]
                                             : (double)((const float*)vals[v])[r];
                long double t = a->fsum + (long double)x;
                if (fabsl(a->fsum) >= fabsl((long double)x)) a->fcomp += (a->fsum - t) + (long double)x;
                else a->fcomp += ((long double)x - t) + a->fsum;
                a->fsum = t;
                a->fabs_sum += fabsl((long double)x);
                if (fresh || x < a->fmin) a->fmin = x;
                if (fresh || x > a->fmax) a->fmax = x;
                break;
            }
            case ORC_I32: case ORC_I64: {
                int64_t x = vdt[v] == ORC_I32 ? (int64_t)((const int32_t*)vals[v])[r]
                                              : ((const int64_t*)vals[v])[r];
                a->isum += x;
                if (fresh || x < a->imin) a->imin = x;
                if (fresh || x > a->imax) a->imax = x;
                break;
            }
            case ORC_U32: case ORC_U64: {
                uint64_t x = vdt[v] == ORC_U32 ? (uint64_t)((const uint32_t*)vals[v])[r]
                                               : ((const uint64_t*)vals[v])[r];
                a->usum += x;
                if (fresh || x < a->umin) a->umin = x;
                if (fresh || x > a->umax) a->umax = x;
                break;
            }
            }
        }
    }

    int64_t* order = (int64_t*)malloc((size_t)G * sizeof(int64_t));
    if (!order) { free(slots); free(first); free(count); free(acc); return -1; }
    for (int64_t g = 0; g < G; ++g) order[g] = g;
    if (sorted) {
        g_sort_keys = keys; g_sort_kdt = kdt; g_sort_nkeys = nkeys; g_sort_first = first;
        qsort(order, (size_t)G, sizeof(int64_t), orc_group_cmp);
    }

    for (int64_t o = 0; o < G; ++o) {
        int64_t g = order[o];
        size_t r = (size_t)first[g];
        if (out_first) out_first[o] = first[g];
        if (out_count) out_count[o] = count[g];
        if (out_keys)
            for (int k = 0; k < nkeys; ++k) {
                if (!out_keys[k]) continue;
                int w = orc_dtype_width(kdt[k]);
                memcpy((unsigned char*)out_keys[k] + (size_t)o * w,
                       (const unsigned char*)keys[k] + r * w, (size_t)w);
            }
        for (int v = 0; v < nvals; ++v) {
            orc_acc* a = &acc[(size_t)v * n + (size_t)g];
            void* os = out_sum ? out_sum[v] : NULL;
            int64_t* oh = out_sum_hi ? out_sum_hi[v] : NULL;
            void* omin = out_min ? out_min[v] : NULL;
            void* omax = out_max ? out_max[v] : NULL;
            double* om = out_mean ? out_mean[v] : NULL;
            double* oa = out_abs ? out_abs[v] : NULL;
            switch (vdt[v]) {
            case ORC_F64: case ORC_F32: {
                long double s = a->fsum + a->fcomp;
                if (os) ((double*)os)[o] = (double)s;
                if (oa) oa[o] = (double)a->fabs_sum;
                if (om) om[o] = (double)(s / (long double)count[g]);
                if (vdt[v] == ORC_F64) {
                    if (omin) ((double*)omin)[o] = a->fmin;
                    if (omax) ((double*)omax)[o] = a->fmax;
                } else {
                    if (omin) ((float*)omin)[o] = (float)a->fmin;
                    if (omax) ((float*)omax)[o] = (float)a->fmax;
                }
                break;
            }
            case ORC_I32: case ORC_I64: {
                unsigned __int128 u = (unsigned __int128)a->isum;
                if (os) ((int64_t*)os)[o] = (int64_t)(uint64_t)u;
                if (oh) oh[o] = (int64_t)(uint64_t)(u >> 64);
                if (om) om[o] = (double)((long double)a->isum / (long double)count[g]);
                if (vdt[v] == ORC_I64) {
                    if (omin) ((int64_t*)omin)[o] = a->imin;
                    if (omax) ((int64_t*)omax)[o] = a->imax;
                } else {
                    if (omin) ((int32_t*)omin)[o] = (int32_t)a->imin;
                    if (omax) ((int32_t*)omax)[o] = (int32_t)a->imax;
                }
                if (oa) oa[o] = 0.0;
                break;
            }
            case ORC_U32: case ORC_U64: {
                unsigned __int128 u = a->usum;
                if (os) ((int64_t*)os)[o] = (int64_t)(uint64_t)u;
                if (oh) oh[o] = (int64_t)(uint64_t)(u >> 64);
                if (om) om[o] = (double)((long double)a->usum / (long double)count[g]);
                if (vdt[v] == ORC_U64) {
                    if (omin) ((uint64_t*)omin)[o] = a->umin;
                    if (omax) ((uint64_t*)omax)[o] = a->umax;
                } else {
                    if (omin) ((uint32_t*)omin)[o] = (uint32_t)a->umin;
                    if (omax) ((uint32_t*)omax)[o] = (uint32_t)a->umax;
                }
                if (oa) oa[o] = 0.0;
                break;
            }
            }
        }
    }
    free(order); free(slots); free(first); free(count); free(acc);
    return G;
}

/*
 * "Transform" output of the reference group-by (CreateValueCol::apply,
 * create_value_col.inl:36-61): every row receives its group's aggregate.
 * Given the group index of each row (row_group[r]) and per-group values,
 * writes out[r] = group_vals[row_group[r]] (width bytes per element).
 */
void orc_broadcast(const int64_t* row_group, size_t n, const void* group_vals, int width, void* out) {
    for (size_t r = 0; r < n; ++r)
        memcpy((unsigned char*)out + r * (size_t)width,
               (const unsigned char*)group_vals + (size_t)row_group[r] * (size_t)width, (size_t)width);
}

/*
 * Set and map over raw key bytes, the lookup structure of the reference's
 * de-duplication and join (an ankerl set/map keyed by a string_view over the
 * element's bytes).  Open addressing with linear probing; key = the raw bits
 * zero-extended to 64, so two keys are equal exactly when their bytes are.
 */
typedef struct {
    uint64_t* key;
    int64_t* val;   /* -1: empty slot */
    size_t mask;
} orc_map;

static int orc_map_init(orc_map* m, size_t n) {
    size_t cap = 16;
    while (cap < 2 * n + 16) cap <<= 1;
    m->key = (uint64_t*)malloc(cap * sizeof(uint64_t));
    m->val = (int64_t*)malloc(cap * sizeof(int64_t));
    m->mask = cap - 1;
    if (!m->key || !m->val) { free(m->key); free(m->val); return -1; }
    for (size_t i = 0; i < cap; ++i) m->val[i] = -1;
    return 0;
}
static void orc_map_free(orc_map* m) { free(m->key); free(m->val); }
static uint64_t orc_raw_bits(const void* col, int width, size_t i) {
    return width == 8 ? ((const uint64_t*)col)[i] : (uint64_t)((const uint32_t*)col)[i];
}
/* slot of key k: the slot holding it, or the empty slot where it would go */
static size_t orc_map_slot(const orc_map* m, uint64_t k) {
    size_t s = (size_t)orc_mix(k) & m->mask;
    while (m->val[s] >= 0 && m->key[s] != k) s = (s + 1) & m->mask;
    return s;
}

/*
 * De-duplication (transform_unique_mt, V/transform/transform_unique/
 * transform_unique_mt.hpp:105-140): rows are visited in order (Last = false)
 * or in reverse (Last = true); a row whose key is not yet in the set is the
 * kept occurrence of that key and its key is inserted.  The reference records
 * the kept rows as mask[i] = 0 and then calls transform_filter_mt (:173),
 * which the reference does not define; here keep[i] = 1 marks exactly those
 * rows.
 * Returns the number of distinct keys, or -1 on allocation failure.
 */
int64_t orc_unique(const void* col, int dt, size_t n, int last, uint8_t* keep) {
    const int w = orc_dtype_width(dt);
    orc_map m;
    if (orc_map_init(&m, n)) return -1;
    int64_t distinct = 0;
    for (size_t t = 0; t < n; ++t) {
        const size_t i = last ? n - 1 - t : t;
        const uint64_t k = orc_raw_bits(col, w, i);
        const size_t s = orc_map_slot(&m, k);
        if (m.val[s] < 0) {
            m.key[s] = k;
            m.val[s] = (int64_t)i;
            keep[i] = 1;
            ++distinct;
        } else {
            keep[i] = 0;
        }
    }
    orc_map_free(&m);
    return distinct;
}

/*
 * Left-join row matching, methods First and Last (transform_left_join_mt,
 * V/transform/transform_left_join/transform_left_join_mt.hpp:172-205): the
 * right key column is loaded into a map key -> row, keeping the first row of
 * each key (try_emplace, First) or the last (assignment, Last); each left row
 * then looks its key up (:201-205): match[i] = the right row, or UINT32_MAX where the
 * key is absent (the reference's SIZE_MAX).  Keys compare by their raw bytes.
 * Method Aligned (method == 2, :206-238): the right rows of each key are kept
 * in row order with a cursor; each left row, in row order, takes the row at
 * its key's cursor and advances it, so the k-th left occurrence of a key
 * matches the k-th right occurrence, and left rows beyond the right side's
 * count of that key match nothing.
 * Returns the number of matched left rows, or -1 on allocation failure.
 */
static int64_t orc_left_join_aligned(const void* left, size_t n_left, const void* right, size_t n_right, int w,
                                     uint32_t* match) {
    orc_map m;
    if (orc_map_init(&m, n_right)) return -1;
    /* key -> slot index, then per-key row lists (CSR) and cursors */
    size_t* slot_of = (size_t*)malloc((n_right ? n_right : 1) * sizeof(size_t));
    size_t nslots = m.mask + 1;
    size_t* cnt = (size_t*)calloc(nslots + 1, sizeof(size_t));
    size_t* cur = (size_t*)calloc(nslots, sizeof(size_t));
    uint32_t* rows = (uint32_t*)malloc((n_right ? n_right : 1) * sizeof(uint32_t));
    if (!slot_of || !cnt || !cur || !rows) {
        free(slot_of); free(cnt); free(cur); free(rows); orc_map_free(&m);
        return -1;
    }
    for (size_t j = 0; j < n_right; ++j) {
        const uint64_t k = orc_raw_bits(right, w, j);
        const size_t s = orc_map_slot(&m, k);
        if (m.val[s] < 0) {
            m.key[s] = k;
            m.val[s] = (int64_t)s;
        }
        slot_of[j] = s;
        cnt[s + 1]++;
    }
    for (size_t s = 0; s < nslots; ++s) cnt[s + 1] += cnt[s];  /* list of slot s: rows[cnt[s] .. cnt[s+1]) */
    for (size_t j = 0; j < n_right; ++j) rows[cnt[slot_of[j]] + cur[slot_of[j]]++] = (uint32_t)j;
    memset(cur, 0, nslots * sizeof(size_t));
    int64_t matched = 0;
    for (size_t i = 0; i < n_left; ++i) {
        const size_t s = orc_map_slot(&m, orc_raw_bits(left, w, i));
        match[i] = 0xffffffffu;
        if (m.val[s] >= 0 && cnt[s] + cur[s] < cnt[s + 1]) {
            match[i] = rows[cnt[s] + cur[s]++];
            ++matched;
        }
    }
    free(slot_of); free(cnt); free(cur); free(rows);
    orc_map_free(&m);
    return matched;
}

int64_t orc_left_join(const void* left, size_t n_left, const void* right, size_t n_right, int dt, int last,
                      uint32_t* match) {
    const int w = orc_dtype_width(dt);
    if (last == 2) return orc_left_join_aligned(left, n_left, right, n_right, w, match);
    orc_map m;
    if (orc_map_init(&m, n_right)) return -1;
    for (size_t j = 0; j < n_right; ++j) {
        const uint64_t k = orc_raw_bits(right, w, j);
        const size_t s = orc_map_slot(&m, k);
        if (m.val[s] < 0) {
            m.key[s] = k;
            m.val[s] = (int64_t)j;
        } else if (last) {
            m.val[s] = (int64_t)j;
        }
    }
    int64_t matched = 0;
    for (size_t i = 0; i < n_left; ++i) {
        const size_t s = orc_map_slot(&m, orc_raw_bits(left, w, i));
        if (m.val[s] >= 0) {
            match[i] = (uint32_t)m.val[s];
            ++matched;
        } else {
            match[i] = 0xffffffffu;
        }
    }
    orc_map_free(&m);
    return matched;
}
