/*
 * vdf_oracle_pivot.c -- CPU oracle for the pivot (2-key sum into a matrix).
 *
 * TEST INFRASTRUCTURE ONLY.  The checker the CUDA path is compared against;
 * only tests/, __graft_entry__.smoke() and bench.py's CPU baseline leg load
 * it.  The product library never links, loads or calls anything here.
 *
 * It restates, sequentially, the reference's pivot (paths relative to the
 * reference project, V/ = include/vison/), V/pivots/pivot.hpp:5-128:
 *   - two string key columns (col key n1, row key n2) and a value column n3
 *     of type T (IntT, UIntT or FloatT);
 *   - rows visited in order: each col key and each row key gets the next
 *     index the first time it appears (idx_col / idx_row try_emplace with
 *     the map's size, :63-71), and lookup[(col key, row key)] += value in T
 *     (:72);
 *   - the result has one column per distinct col key and one row per
 *     distinct row key, both in first-appearance order, and cell
 *     [col_idx][row_idx] = the pair's sum, 0 for a pair that never occurs
 *     (:75-107); the names are the keys (:112-128).
 * Keys compare by their bytes.  Sums wrap in the value type for integers, as
 * "+=" in T does; doubles are summed in row order.  The matrix is written one
 * output column after another: cell (c, r) at c * n_rowkeys + r.  The
 * reference sizes its outer vector by the row-key count while indexing it by
 * col index (:77-85), which only works when the two counts are equal; the
 * intended [col][row] layout is what is restated here.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

enum { PV_I32 = 0, PV_I64 = 1, PV_U32 = 2, PV_U64 = 3, PV_F64 = 4 };

typedef struct {
    uint32_t* slot;  /* row of the key's first appearance + 1 (0: empty) */
    uint32_t* index; /* first-appearance index of the key */
    size_t mask;
} pv_dict;

static uint64_t pv_hash(const char* s, uint64_t len) {
    uint64_t h = 1469598103934665603ull; /* FNV-1a */
    for (uint64_t i = 0; i < len; ++i) h = (h ^ (unsigned char)s[i]) * 1099511628211ull;
    return h ^ (h >> 29);
}

static int pv_dict_init(pv_dict* d, size_t n) {
    size_t cap = 16;
    while (cap < 2 * n + 2) cap <<= 1;
    d->slot = (uint32_t*)calloc(cap, sizeof(uint32_t));
    d->index = (uint32_t*)calloc(cap, sizeof(uint32_t));
    d->mask = cap - 1;
    return d->slot && d->index ? 0 : -1;
}

static void pv_dict_free(pv_dict* d) {
    free(d->slot);
    free(d->index);
}

/* index of row r's key; a new key takes *count (then incremented) */
static uint32_t pv_dict_add(pv_dict* d, const char* bytes, const uint64_t* offs, size_t r, uint32_t* count,
                            uint32_t* first_row) {
    const char* s = bytes + offs[r];
    const uint64_t len = offs[r + 1] - offs[r];
    size_t i = (size_t)pv_hash(s, len) & d->mask;
    for (;;) {
        const uint32_t e = d->slot[i];
        if (e == 0) {
            d->slot[i] = (uint32_t)r + 1;
            d->index[i] = *count;
            first_row[*count] = (uint32_t)r;
            return (*count)++;
        }
        const size_t q = e - 1;
        if (offs[q + 1] - offs[q] == len && memcmp(bytes + offs[q], s, len) == 0) return d->index[i];
        i = (i + 1) & d->mask;
    }
}

/* Returns 0, or -1 when memory runs out or the matrix does not fit in
 * matrix_cap cells (the key counts and first rows are written either way). */
int orc_pivot(size_t n, const char* col_bytes, const uint64_t* col_offs, const char* row_bytes,
              const uint64_t* row_offs, const void* values, int dt, uint32_t* n_colkeys, uint32_t* n_rowkeys,
              uint32_t* colkey_row, uint32_t* rowkey_row, void* matrix, size_t matrix_cap) {
    pv_dict dc, dr;
    uint32_t* ci = (uint32_t*)malloc((n ? n : 1) * sizeof(uint32_t));
    uint32_t* ri = (uint32_t*)malloc((n ? n : 1) * sizeof(uint32_t));
    if (!ci || !ri || pv_dict_init(&dc, n) || pv_dict_init(&dr, n)) return -1;
    uint32_t nc = 0, nr = 0;
    for (size_t r = 0; r < n; ++r) {
        ci[r] = pv_dict_add(&dc, col_bytes, col_offs, r, &nc, colkey_row);
        ri[r] = pv_dict_add(&dr, row_bytes, row_offs, r, &nr, rowkey_row);
    }
    *n_colkeys = nc;
    *n_rowkeys = nr;
    int rc = 0;
    const size_t cells = (size_t)nc * nr;
    if (cells > matrix_cap) {
        rc = -1;
    } else {
        const int w = (dt == PV_I32 || dt == PV_U32) ? 4 : 8;
        memset(matrix, 0, cells * (size_t)w);
        for (size_t r = 0; r < n; ++r) {
            const size_t cell = (size_t)ci[r] * nr + ri[r];
            switch (dt) {
            case PV_I32: { /* wraps like int "+=" on the reference's targets */
                uint32_t* m = (uint32_t*)matrix;
                m[cell] += (uint32_t)((const int32_t*)values)[r];
                break;
            }
            case PV_U32: ((uint32_t*)matrix)[cell] += ((const uint32_t*)values)[r]; break;
            case PV_I64: {
                uint64_t* m = (uint64_t*)matrix;
                m[cell] += (uint64_t)((const int64_t*)values)[r];
                break;
            }
            case PV_U64: ((uint64_t*)matrix)[cell] += ((const uint64_t*)values)[r]; break;
            default: ((double*)matrix)[cell] += ((const double*)values)[r]; break;
            }
        }
    }
    pv_dict_free(&dc);
    pv_dict_free(&dr);
    free(ci);
    free(ri);
    return rc;
}
