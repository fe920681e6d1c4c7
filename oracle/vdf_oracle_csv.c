/*
 * vdf_oracle_csv.c -- CPU oracle for the CSV ingest (read_csv).
 *
 * TEST INFRASTRUCTURE ONLY.  The checker the CUDA path is compared against;
 * only tests/, __graft_entry__.smoke() and bench.py's CPU baseline leg load
 * it.  The product library never links, loads or calls anything here.
 *
 * It restates, in plain C and sequentially, the reference's read path
 * (paths relative to the reference project, V/ = include/vison/):
 *   - the first-line pass (V/read/read_csv/read_csv.hpp:58-135): fields split
 *     at the delimiter outside quotes; the line stops at the first CR or LF
 *     even inside quotes, and a CR or LF followed by an LF moves the stop onto
 *     that LF (the last field keeps the first byte); names: empty -> "NA";
 *     without a header the line is the first data row, where an empty field
 *     other than the last stays "" and an empty last field reads "NA";
 *     the data start one byte after the stop (:146-166);
 *   - the record parser (V/inlines/read/read_csv/parsers_core/
 *     parse_rows_chunk.inl:115-183, its scalar loop): the quote byte toggles
 *     quoting; the delimiter outside quotes ends a field; CR or LF outside
 *     quotes ends the field and the record, CR LF counting once; empty fields
 *     read "NA"; bytes after the last terminator form one more record.
 *     Deviations (as the GPU path defines them): a record whose field count
 *     differs from the first line's is an error with its row index (the
 *     reference prints "column number problem" and stops, :95-98); a final
 *     record that ends in a delimiter gets an "NA" last field (the reference
 *     emits no field for an empty tail, :172-183, leaving that column short);
 *   - the column types from the first 10 values
 *     (V/inlines/classify_column.inl:13-133, simd_can_be_nb.inl, has_dot.inl):
 *     'd', 's', 'c', 'b', 'u' ('i' is unreachable: simd_can_be_nb rejects
 *     '-', so no value both passes it and starts with '-');
 *   - the conversions: 'd' as fast_float::from_chars (v8.1.0, vendored at
 *     V/external/fast_float; not in this file: the decimal grammar is
 *     restated below and the rounding is glibc strtod's, which is correctly
 *     rounded to nearest-even like fast_float), 0 when invalid or out of
 *     range; 'u' as std::from_chars into unsigned int, 'b' as std::from_chars
 *     into int, != 0; strings keep their bytes.
 *
 * Output: one malloc'd blob (orc_csv_read), freed with orc_csv_free:
 *   u64 nrow, u32 ncol, u32 pad, i64 bad_row (-1 when none), then per column
 *   u8 type, u32 name length, name bytes; then per column its data: numbers
 *   as nrow values (f64 / u32 / u8), strings as nrow + 1 u64 offsets and the
 *   bytes.  The same layout is written by oracle/ref_shim.cpp.
 */
#include <errno.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef struct {
    uint32_t s, e;
} orc_field;

typedef struct {
    unsigned char* p;
    size_t n, cap;
} orc_buf;

static int ob_put(orc_buf* b, const void* src, size_t k) {
    if (b->n + k > b->cap) {
        size_t cap = b->cap ? b->cap : 4096;
        while (cap < b->n + k) cap *= 2;
        unsigned char* q = (unsigned char*)realloc(b->p, cap);
        if (!q) return -1;
        b->p = q;
        b->cap = cap;
    }
    if (k) memcpy(b->p + b->n, src, k);
    b->n += k;
    return 0;
}

static int is_dig(unsigned char c) { return c >= '0' && c <= '9'; }
static unsigned char low(unsigned char c) { return (c >= 'A' && c <= 'Z') ? (unsigned char)(c + 32) : c; }

/* fast_float::from_chars (chars_format::general) as the reference stores it. */
double orc_parse_double(const char* s, size_t n) {
    size_t i = 0;
    int neg = 0, seen = 0, nonzero = 0;
    if (n == 0) return 0.0;
    if (s[0] == '-') neg = 1, i = 1;
    const size_t sign_end = i;
    while (i < n && is_dig((unsigned char)s[i])) nonzero |= s[i] != '0', seen = 1, ++i;
    if (i < n && s[i] == '.') {
        ++i;
        while (i < n && is_dig((unsigned char)s[i])) nonzero |= s[i] != '0', seen = 1, ++i;
    }
    if (!seen) {
        if (n - sign_end >= 3) {
            const unsigned char a = low(s[sign_end]), b = low(s[sign_end + 1]), c = low(s[sign_end + 2]);
            if (a == 'n' && b == 'a' && c == 'n') {
                uint64_t bits = 0x7ff8000000000000ull | ((uint64_t)neg << 63);
                double d;
                memcpy(&d, &bits, 8);
                return d;
            }
            if (a == 'i' && b == 'n' && c == 'f') return neg ? -HUGE_VAL : HUGE_VAL;
        }
        return 0.0;
    }
    size_t end = i;
    if (i < n && (s[i] == 'e' || s[i] == 'E')) {
        size_t j = i + 1;
        if (j < n && (s[j] == '+' || s[j] == '-')) ++j;
        if (j < n && is_dig((unsigned char)s[j])) {
            while (j < n && is_dig((unsigned char)s[j])) ++j;
            end = j;
        }
    }
    char stack[256];
    char* tmp = end < sizeof stack ? stack : (char*)malloc(end + 1);
    if (!tmp) return 0.0;
    memcpy(tmp, s, end);
    tmp[end] = 0;
    errno = 0;
    const double v = strtod(tmp, NULL);
    if (tmp != stack) free(tmp);
    if (isinf(v)) return 0.0;          /* overflow: out of range */
    if (v == 0.0 && nonzero) return 0.0;  /* nonzero decimal rounded to zero: out of range */
    return v;
}

/* std::from_chars into unsigned int; 0 when invalid or out of range. */
uint32_t orc_parse_u32(const char* s, size_t n) {
    uint64_t v = 0;
    size_t i = 0;
    int over = 0;
    while (i < n && is_dig((unsigned char)s[i])) {
        if (!over) {
            v = v * 10 + (uint64_t)(s[i] - '0');
            if (v > 0xffffffffull) over = 1;
        }
        ++i;
    }
    return (i == 0 || over) ? 0u : (uint32_t)v;
}

/* std::from_chars into int; 0 when invalid or out of range. */
int32_t orc_parse_i32(const char* s, size_t n) {
    size_t i = 0;
    const int neg = n > 0 && s[0] == '-';
    if (neg) i = 1;
    const size_t d0 = i;
    uint64_t v = 0;
    int over = 0;
    while (i < n && is_dig((unsigned char)s[i])) {
        if (!over) {
            v = v * 10 + (uint64_t)(s[i] - '0');
            if (v > 0x80000000ull) over = 1;
        }
        ++i;
    }
    if (i == d0 || over) return 0;
    if (!neg && v > 0x7fffffffull) return 0;
    return neg ? (int32_t)(0 - v) : (int32_t)v;
}

static int can_be_nb(const char* s, size_t n) {
    int dot = 0;
    if (n == 0) return 0;
    for (size_t i = 0; i < n; ++i) {
        if (s[i] == '.') {
            if (dot) return 0;
            dot = 1;
        } else if (!is_dig((unsigned char)s[i])) {
            return 0;
        }
    }
    return 1;
}

/* classify_column on up to 10 values (pointers + lengths). */
static char classify(const char* const* v, const size_t* len, size_t k) {
    int is_bool = 1, is_nb = 1, is_bufchar = 1;
    if (k > 10) k = 10;
    for (size_t i = 0; i < k; ++i) {
        if (!can_be_nb(v[i], len[i])) {
            is_nb = 0;
            if (len[i] > 1) {
                is_bufchar = 0;
                break;
            }
            continue;
        }
        if (memchr(v[i], '.', len[i])) return 'd';
        if (!(len[i] == 1 && (v[i][0] == '0' || v[i][0] == '1'))) is_bool = 0;
    }
    if (!is_nb) return is_bufchar ? 'c' : 's';
    return is_bool ? 'b' : 'u';
}

static const char kNA[] = "NA";

void orc_csv_free(void* blob) { free(blob); }

/* Returns the blob (NULL on allocation failure); *blob_bytes its size. */
void* orc_csv_read(const char* b, size_t n, char delim, int header, char quote, size_t* blob_bytes) {
    /* first line */
    size_t i = 0, fs = 0;
    int inq = 0;
    orc_field* f0 = NULL;
    size_t nf0 = 0, cf0 = 0;
    for (;; ++i) {
        int stop = i >= n;
        if (!stop && (b[i] == '\n' || b[i] == '\r')) {
            if (i + 1 < n && b[i + 1] == '\n') ++i;
            stop = 1;
        }
        if (stop || (b[i] == delim && !inq)) {
            if (nf0 == cf0) {
                cf0 = cf0 ? 2 * cf0 : 16;
                f0 = (orc_field*)realloc(f0, cf0 * sizeof *f0);
                if (!f0) return NULL;
            }
            f0[nf0].s = (uint32_t)fs;
            f0[nf0].e = (uint32_t)(i < n ? i : n);
            ++nf0;
            fs = i + 1;
            if (stop) break;
        } else if (b[i] == quote) {
            inq = !inq;
        }
    }
    const uint32_t ncol = (uint32_t)nf0;
    const size_t data_start = i + 1 < n ? i + 1 : n;
    /* records: fields as (start, end) with end = start - 1 meaning "NA" is not
       needed: an empty field is stored as s == e and read as "NA" */
    orc_field* fl = NULL;
    size_t nfl = 0, cfl = 0;
    int64_t bad = -1;
    const uint64_t row0 = header ? 0 : 1;
    uint64_t rows = 0;
    uint32_t col = 0;
    size_t rec = data_start; /* start of the current record */
    fs = data_start;
    inq = 0;
#define PUSH_FIELD(S, E)                                                  \
    do {                                                                  \
        if (nfl == cfl) {                                                 \
            cfl = cfl ? 2 * cfl : 1024;                                   \
            fl = (orc_field*)realloc(fl, cfl * sizeof *fl);               \
            if (!fl) return NULL;                                         \
        }                                                                 \
        fl[nfl].s = (uint32_t)(S);                                        \
        fl[nfl].e = (uint32_t)(E);                                        \
        ++nfl;                                                            \
    } while (0)
    for (i = data_start; i < n && bad < 0; ++i) {
        const char c = b[i];
        if (c == quote) {
            inq = !inq;
        } else if (!inq && c == delim) {
            if (col + 1 >= ncol) {
                bad = (int64_t)(rows + row0);
                break;
            }
            PUSH_FIELD(fs, i);
            ++col;
            fs = i + 1;
        } else if (!inq && (c == '\n' || c == '\r')) {
            if (col + 1 != ncol) {
                bad = (int64_t)(rows + row0);
                break;
            }
            PUSH_FIELD(fs, i);
            col = 0;
            ++rows;
            if (c == '\r' && i + 1 < n && b[i + 1] == '\n') ++i;
            fs = i + 1;
            rec = fs;
        }
    }
    if (bad < 0 && rec < n) {
        /* the final record without terminator (its quote state carries over) */
        if (col + 1 != ncol) bad = (int64_t)(rows + row0);
        else {
            PUSH_FIELD(fs, n);
            ++rows;
        }
    }
#undef PUSH_FIELD
    const uint64_t nrow = rows + row0;
    /* the value of (row, column) */
#define VAL_PTR(R, K) \
    ((!header && (R) == 0) ? (const char*)b + f0[K].s : (const char*)b + fl[((R) - row0) * ncol + (K)].s)
    char* types = (char*)malloc(ncol ? ncol : 1);
    orc_buf ob = {0, 0, 0};
    int64_t bad_out = bad;
    uint64_t nrow_out = bad >= 0 ? 0 : nrow;
    uint32_t pad = 0;
    ob_put(&ob, &nrow_out, 8);
    ob_put(&ob, &ncol, 4);
    ob_put(&ob, &pad, 4);
    ob_put(&ob, &bad_out, 8);
    for (uint32_t k = 0; k < ncol; ++k) {
        /* first up to 10 values of column k */
        const char* v[10];
        size_t len[10];
        size_t cnt = 0;
        for (uint64_t r = 0; r < nrow && cnt < 10 && bad < 0; ++r) {
            size_t s, e;
            if (!header && r == 0) {
                s = f0[k].s;
                e = f0[k].e;
                if (s == e && k + 1 == ncol) {
                    v[cnt] = kNA, len[cnt] = 2;
                } else {
                    v[cnt] = (const char*)b + s, len[cnt] = e - s;
                }
            } else {
                const orc_field* fd = &fl[(r - row0) * ncol + k];
                s = fd->s;
                e = fd->e;
                if (s == e) v[cnt] = kNA, len[cnt] = 2;
                else v[cnt] = (const char*)b + s, len[cnt] = e - s;
            }
            ++cnt;
        }
        types[k] = classify(v, len, cnt);
        const uint8_t ty = (uint8_t)types[k];
        ob_put(&ob, &ty, 1);
        uint32_t nl;
        if (header) {
            const char* nm = (const char*)b + f0[k].s;
            nl = f0[k].e - f0[k].s;
            if (nl == 0) nm = kNA, nl = 2;
            ob_put(&ob, &nl, 4);
            ob_put(&ob, nm, nl);
        } else {
            nl = 0;
            ob_put(&ob, &nl, 4);
        }
    }
    for (uint32_t k = 0; k < ncol && nrow_out; ++k) {
        const char ty = types[k];
        if (ty == 's' || ty == 'c') {
            uint64_t off = 0;
            ob_put(&ob, &off, 8);
            for (uint64_t r = 0; r < nrow; ++r) {
                size_t s, e;
                int na;
                if (!header && r == 0) s = f0[k].s, e = f0[k].e, na = (s == e && k + 1 == ncol);
                else s = fl[(r - row0) * ncol + k].s, e = fl[(r - row0) * ncol + k].e, na = s == e;
                off += na ? 2 : e - s;
                ob_put(&ob, &off, 8);
            }
            for (uint64_t r = 0; r < nrow; ++r) {
                size_t s, e;
                int na;
                if (!header && r == 0) s = f0[k].s, e = f0[k].e, na = (s == e && k + 1 == ncol);
                else s = fl[(r - row0) * ncol + k].s, e = fl[(r - row0) * ncol + k].e, na = s == e;
                if (na) ob_put(&ob, kNA, 2);
                else ob_put(&ob, b + s, e - s);
            }
        } else {
            for (uint64_t r = 0; r < nrow; ++r) {
                size_t s, e;
                if (!header && r == 0) s = f0[k].s, e = f0[k].e;
                else s = fl[(r - row0) * ncol + k].s, e = fl[(r - row0) * ncol + k].e;
                const char* p = (const char*)b + s;
                size_t l = e - s;
                /* an empty field is "NA" (or "" in the first line), both invalid numbers */
                if (ty == 'd') {
                    const double d = orc_parse_double(p, l);
                    ob_put(&ob, &d, 8);
                } else if (ty == 'u') {
                    const uint32_t u = orc_parse_u32(p, l);
                    ob_put(&ob, &u, 4);
                } else {
                    const uint8_t x = orc_parse_i32(p, l) != 0;
                    ob_put(&ob, &x, 1);
                }
            }
        }
    }
#undef VAL_PTR
    free(types);
    free(f0);
    free(fl);
    if (blob_bytes) *blob_bytes = ob.n;
    return ob.p;
}
