// Exercises the header-only dataframe layer (include/vison_b200/vison.hpp) on
// the GPU: the reference documentation's sort_by example, Soft/Hard sorts,
// sorts while in view, materialize, sort_by_external, multi-key sorts and
// the transform group-by (Gather with user functions included) and the
// pivot, checked against plain CPU computations here.
#include <algorithm>
#include <cstdio>
#include <map>
#include <set>
#include <numeric>
#include <random>
#include <tuple>
#include <vector>

#include "vison_b200/vison.hpp"

using DF = vison_b200::Dataframe<>;
using vison_b200::LeftJoinMethods;
using vison_b200::GroupFunction;

static int failures = 0;
#define CHECK(cond)                                                                  \
    do {                                                                             \
        if (!(cond)) {                                                               \
            std::fprintf(stderr, "CHECK failed at line %d: %s\n", __LINE__, #cond); \
            ++failures;                                                              \
        }                                                                            \
    } while (0)

// V/INTERNALS.doc:1554-1632: 15 rows, sorted by column n = 2
static DF doc_frame() {
    DF df;
    std::vector<int> id(15);
    std::iota(id.begin(), id.end(), 1);
    df.add_col(id, "col1");
    df.add_col(std::vector<unsigned>{1, 6, 1, 6, 1, 6, 1, 6, 6, 1, 6, 6, 6, 1, 16}, "col2");
    df.add_col(std::vector<unsigned>{2, 7, 2, 7, 2, 7, 2, 7, 7, 2, 7, 7, 7, 2, 7}, "col3");
    df.add_col(std::vector<unsigned>{3, 8, 3, 8, 3, 8, 3, 8, 8, 3, 8, 8, 8, 3, 8}, "col4");
    return df;
}

static void test_doc_example() {
    DF df = doc_frame();
    unsigned n = 2;
    df.sort_by(n);
    CHECK(df.in_view);
    const std::vector<int> asc = {1, 3, 5, 7, 10, 14, 2, 4, 6, 8, 9, 11, 12, 13, 15};
    CHECK(df.get_col<int>(0) == asc);
    df.materialize();
    CHECK(!df.in_view);
    CHECK(df.int_v[0] == asc);
    CHECK((df.uint_v[0] == std::vector<unsigned>{1, 1, 1, 1, 1, 1, 6, 6, 6, 6, 6, 6, 6, 6, 16}));

    DF d2 = doc_frame();
    d2.sort_by<0>(n);  // the reference code: ascending, then std::reverse
    std::vector<int> rev(asc.rbegin(), asc.rend());
    CHECK(d2.get_col<int>(0) == rev);
}

static void test_hard_sort_and_view_composition() {
    std::mt19937_64 rng(5);
    const unsigned N = 200000;
    std::vector<int> a(N), b(N), id(N);
    std::vector<double> v(N);
    for (unsigned i = 0; i < N; ++i) {
        a[i] = (int)(rng() % 50) - 25;
        b[i] = (int)(rng() % 7);
        v[i] = (double)(rng() % 1000) / 8.0;
        id[i] = (int)i;
    }
    // expected: stable by (a, b)
    std::vector<unsigned> exp(N);
    std::iota(exp.begin(), exp.end(), 0u);
    std::stable_sort(exp.begin(), exp.end(), [&](unsigned x, unsigned y) { return std::tie(a[x], b[x]) < std::tie(a[y], b[y]); });

    DF df;
    df.add_col(a, "a");
    df.add_col(b, "b");
    df.add_col(v, "v");
    df.add_col(id, "id");
    // LSD composition through the view: sort by b, then (stably) by a
    unsigned nb = 1, na = 0;
    df.sort_by(nb);
    df.sort_by(na);
    std::vector<int> got = df.get_col<int>(3);
    bool ok = true;
    for (unsigned i = 0; i < N; ++i) ok &= (got[i] == (int)exp[i]);
    CHECK(ok);

    DF dh;
    dh.add_col(a, "a");
    dh.add_col(b, "b");
    dh.add_col(id, "id");
    dh.sort_by_cols<1, false>({0, 1});  // Hard: columns permuted in place
    CHECK(!dh.in_view);
    ok = true;
    for (unsigned i = 0; i < N; ++i) ok &= (dh.int_v[2][i] == (int)exp[i]);
    CHECK(ok);
}

static void test_sort_by_external() {
    DF df = doc_frame();
    std::vector<long> ext = {5, 4, 3, 2, 1, 0, -1, -2, -3, -4, -5, -6, -7, -8, -9};
    df.sort_by_external<long>(ext);
    std::vector<int> exp(15);
    for (int i = 0; i < 15; ++i) exp[i] = 15 - i;
    CHECK(df.get_col<int>(0) == exp);
}

static void test_transform_group_by() {
    std::mt19937_64 rng(11);
    const unsigned N = 100000;
    std::vector<int> k1(N), iv(N);
    std::vector<unsigned> k2(N);
    std::vector<double> dv(N);
    for (unsigned i = 0; i < N; ++i) {
        k1[i] = (int)(rng() % 97) - 40;
        k2[i] = (unsigned)(rng() % 3);
        iv[i] = (int)(rng() % 2000001) - 1000000;
        dv[i] = (double)((int64_t)(rng() % 4001) - 2000) / 16.0;  // exact sums
    }
    std::map<std::pair<int, unsigned>, std::tuple<long, long, double, int, int>> g;  // count, isum, dsum, imin, imax
    for (unsigned i = 0; i < N; ++i) {
        auto key = std::make_pair(k1[i], k2[i]);
        auto it = g.find(key);
        if (it == g.end()) g[key] = {1, iv[i], dv[i], iv[i], iv[i]};
        else {
            auto& [c, s, d, mn, mx] = it->second;
            ++c; s += iv[i]; d += dv[i]; mn = std::min(mn, iv[i]); mx = std::max(mx, iv[i]);
        }
    }
    DF df;
    df.add_col(k1, "k1");
    df.add_col(k2, "k2");
    df.add_col(iv, "iv");
    df.add_col(dv, "dv");
    df.transform_group_by<void, void, GroupFunction::Occurence>({0, 1}, 2, "n");
    df.transform_group_by<void, void, GroupFunction::Sum>({0, 1}, 2, "isum");
    df.transform_group_by<void, void, GroupFunction::Mean>({0, 1}, 3, "dmean");
    df.transform_group_by<void, void, GroupFunction::Min>({0, 1}, 2, "imin");
    df.transform_group_by<void, void, GroupFunction::Max>({0, 1}, 2, "imax");
    CHECK(df.ncol == 9);
    bool ok = true;
    for (unsigned i = 0; i < N; ++i) {
        const auto& [c, s, d, mn, mx] = g[{k1[i], k2[i]}];
        ok &= df.uint_v[1][i] == (unsigned)c;           // "n"
        ok &= df.int_v[2][i] == (int)s;                  // "isum" (fits in int here)
        ok &= df.dbl_v[1][i] == d / (double)c;           // "dmean"
        ok &= df.int_v[3][i] == mn && df.int_v[4][i] == mx;
    }
    CHECK(ok);
}

// GroupFunction::Gather: the user function over each group's values in row
// order (the rows as viewed, when the frame is in view), broadcast per row;
// checked against a std::map walk over the rows here.
static double sum_sq(std::vector<double>& v) {
    double s = 0;
    for (double x : v) s += x * x;
    return s;
}

static void test_transform_group_by_gather() {
    std::mt19937_64 rng(12);
    const unsigned N = 50000;
    std::vector<int> k(N), iv(N);
    std::vector<double> dv(N);
    for (unsigned i = 0; i < N; ++i) {
        k[i] = (int)(rng() % 97) - 40;
        iv[i] = (int)(rng() % 2000001) - 1000000;
        dv[i] = (double)((int64_t)(rng() % 4001) - 2000) / 7.0;
    }
    std::map<int, std::vector<unsigned>> rows;  // key -> rows in row order
    for (unsigned i = 0; i < N; ++i) rows[k[i]].push_back(i);
    DF df;
    df.add_col(k, "k");
    df.add_col(iv, "iv");
    df.add_col(dv, "dv");
    // the default group function (the first value) and None take the same path
    df.transform_group_by<void, void, GroupFunction::Gather>({0}, 1, "first");
    df.transform_group_by<void, void, GroupFunction::None>({0}, 1, "first2");
    df.transform_group_by<void, void, GroupFunction::Gather>({0}, 2, "ss", &sum_sq);
    df.transform_group_by<void, void, GroupFunction::Gather>(
        {0}, 1, "last", [](std::vector<int>& v) { return v.empty() ? 0 : v.back(); });
    df.transform_group_by<void, void, GroupFunction::Gather>(
        {0}, 2, "n", [](std::vector<double>& v) { return (unsigned)v.size(); });
    CHECK(df.ncol == 8);
    bool ok = true;
    for (const auto& [key, rs] : rows) {
        double ss = 0;
        for (unsigned r : rs) ss += dv[r] * dv[r];
        for (unsigned r : rs) {
            ok &= df.int_v[2][r] == iv[rs.front()];  // int_v: k, iv, first, first2, last
            ok &= df.int_v[3][r] == iv[rs.front()];
            ok &= df.dbl_v[1][r] == ss;
            ok &= df.int_v[4][r] == iv[rs.back()];
            ok &= df.uint_v[0][r] == (unsigned)rs.size();
        }
    }
    CHECK(ok);

    // in view (a Soft sort by dv): groups see their rows in view order
    DF dw;
    dw.add_col(k, "k");
    dw.add_col(iv, "iv");
    dw.add_col(dv, "dv");
    unsigned by = 2;
    dw.sort_by(by);
    CHECK(dw.in_view);
    std::vector<unsigned> view(N);
    std::iota(view.begin(), view.end(), 0u);
    std::stable_sort(view.begin(), view.end(), [&](unsigned a, unsigned b) { return dv[a] < dv[b]; });
    std::map<int, int> first_in_view;
    for (unsigned r : view) first_in_view.emplace(k[r], iv[r]);
    dw.transform_group_by<void, void, GroupFunction::Gather>({0}, 1, "first");
    CHECK(dw.in_view && dw.ncol == 4);
    dw.materialize();
    bool okv = true;
    for (unsigned p = 0; p < N; ++p) okv &= dw.int_v[2][p] == first_in_view[k[view[p]]];
    CHECK(okv);
}

// pivot: the documented example (INTERNALS.doc:1251-1296), then a random
// frame against a std::map walk in row order (first-appearance indices).
static void test_pivot() {
    DF df;
    df.add_col(std::vector<std::string>{"A", "A", "A", "B", "B", "A", "B", "B", "B", "A", "A", "B", "B", "B", "B"},
               "col5");
    df.add_col(std::vector<std::string>{"D", "D", "C", "C", "C", "D", "C", "D", "D", "C", "D", "C", "D", "C", "D"},
               "col1");
    df.add_col(std::vector<double>{3, 8, 0, 8, 3, 8, 3, 3, 8, 0, 8, 8, 0, 8, 3}, "col3");
    unsigned n1 = 0, n2 = 1, n3 = 2;
    DF p;
    p.pivot<double>(df, n1, n2, n3);
    CHECK(p.ncol == 2 && p.nrow == 2);
    CHECK((p.name_v == std::vector<std::string>{"A", "B"}));
    CHECK((p.name_v_row == std::vector<std::string>{"D", "C"}));
    CHECK((p.dbl_v[0] == std::vector<double>{27, 0}) && (p.dbl_v[1] == std::vector<double>{14, 30}));

    std::mt19937_64 rng(13);
    const unsigned N = 40000;
    std::vector<std::string> ck(N);
    std::vector<unsigned> rk(N);
    std::vector<int> v(N);
    for (unsigned i = 0; i < N; ++i) {
        ck[i] = "k" + std::string(rng() % 4, 'x') + std::to_string(rng() % 61);
        rk[i] = (unsigned)(rng() % 257);
        v[i] = (int)(rng() % 2000000001u) - 1000000000;  // sums wrap in int
    }
    DF q;
    q.add_col(ck, "ck");
    q.add_col(rk, "rk");
    q.add_col(v, "v");
    std::map<std::string, unsigned> ci, ri;
    std::vector<std::string> corder, rorder;
    std::map<std::pair<unsigned, unsigned>, uint32_t> acc;
    for (unsigned i = 0; i < N; ++i) {
        const std::string r = std::to_string(rk[i]);
        if (ci.emplace(ck[i], (unsigned)ci.size()).second) corder.push_back(ck[i]);
        if (ri.emplace(r, (unsigned)ri.size()).second) rorder.push_back(r);
        acc[{ci[ck[i]], ri[r]}] += (uint32_t)v[i];
    }
    DF pq;
    unsigned a = 0, b = 1, c = 2;
    pq.pivot<int>(q, a, b, c);
    CHECK(pq.ncol == corder.size() && pq.nrow == rorder.size());
    CHECK(pq.name_v == corder && pq.name_v_row == rorder);
    bool ok = pq.int_v.size() == corder.size();
    for (unsigned x = 0; ok && x < corder.size(); ++x)
        for (unsigned y = 0; y < rorder.size(); ++y) {
            auto it = acc.find({x, y});
            ok &= pq.int_v[x][y] == (int)(it == acc.end() ? 0u : it->second);
        }
    CHECK(ok);
}

// transform_unique: the rows kept are those a set walk keeps (first or last
// occurrence per key value, in row order), for every column of the frame.
static void test_transform_unique() {
    std::mt19937_64 rng(23);
    const unsigned N = 50000;
    std::vector<int64_t> k(N);
    std::vector<double> v(N);
    for (unsigned i = 0; i < N; ++i) {
        k[i] = (int64_t)(rng() % 7000) - 3500;
        v[i] = (double)i;
    }
    for (int last = 0; last < 2; ++last) {
        std::vector<unsigned> rows;
        std::set<int64_t> seen;
        if (!last) {
            for (unsigned i = 0; i < N; ++i)
                if (seen.insert(k[i]).second) rows.push_back(i);
        } else {
            for (unsigned i = N; i-- > 0;)
                if (seen.insert(k[i]).second) rows.push_back(i);
            std::sort(rows.begin(), rows.end());
        }
        DF df;
        df.add_col(std::vector<int64_t>(k), "k");
        df.add_col(std::vector<double>(v), "v");
        if (last) df.transform_unique<void, false, true>(0);
        else df.transform_unique(0);
        CHECK(df.nrow == rows.size());
        bool ok = df.nrow == rows.size();
        for (unsigned i = 0; ok && i < rows.size(); ++i)
            ok &= df.lint_v[0][i] == k[rows[i]] && df.dbl_v[0][i] == v[rows[i]];
        CHECK(ok);
    }
}

// transform_left_join: each left row takes the first (or last) right row with
// its key, or the defaults; the right frame's columns are appended.
static void test_transform_left_join() {
    std::mt19937_64 rng(29);
    const unsigned NL = 30000, NR = 8000;
    std::vector<int> lk(NL), rk(NR), rv(NR);
    std::vector<double> rd(NR);
    for (unsigned i = 0; i < NL; ++i) lk[i] = (int)(rng() % 6000);
    for (unsigned j = 0; j < NR; ++j) {
        rk[j] = (int)(rng() % 4000) * 2;  // even: odd left keys never match
        rv[j] = (int)j;
        rd[j] = 0.5 * j;
    }
    for (int method = 0; method < 3; ++method) {
        // expected right row per left row: first, last, or the k-th for the k-th occurrence
        std::map<int, std::vector<unsigned>> rows;
        for (unsigned j = 0; j < NR; ++j) rows[rk[j]].push_back(j);
        std::map<int, unsigned> next;
        std::vector<long> want(NL, -1);
        for (unsigned i = 0; i < NL; ++i) {
            auto it = rows.find(lk[i]);
            if (it == rows.end()) continue;
            if (method == 0) want[i] = it->second.front();
            else if (method == 1) want[i] = it->second.back();
            else if (next[lk[i]] < it->second.size()) want[i] = it->second[next[lk[i]]++];
        }
        DF left, right;
        left.add_col(std::vector<int>(lk), "lk");
        right.add_col(std::vector<int>(rk), "rk");
        right.add_col(std::vector<int>(rv), "rv");
        right.add_col(std::vector<double>(rd), "rd");
        if (method == 0) left.transform_left_join<void, true, LeftJoinMethods::First>(right, 0, 0, ' ', "NA", 0, -7, 0, -1.5);
        else if (method == 1) left.transform_left_join<void, true, LeftJoinMethods::Last>(right, 0, 0, ' ', "NA", 0, -7, 0, -1.5);
        else left.transform_left_join<void, true, LeftJoinMethods::Aligned>(right, 0, 0, ' ', "NA", 0, -7, 0, -1.5);
        CHECK(left.ncol == 4);
        bool ok = left.ncol == 4;
        for (unsigned i = 0; ok && i < NL; ++i) {
            const int ek = want[i] < 0 ? -7 : rk[want[i]];
            const int ev = want[i] < 0 ? -7 : rv[want[i]];
            const double ed = want[i] < 0 ? -1.5 : rd[want[i]];
            ok &= left.int_v[1][i] == ek && left.int_v[2][i] == ev && left.dbl_v[0][i] == ed;
        }
        CHECK(ok);
    }
}

static void test_readf() {
    // a small file with every inferred kind: 'u', 'd', 's' (quoted delimiter),
    // 'c', 'b'; CR LF line ends; an empty string field reads "NA"
    const char* text =
        "year,delay,name,code,flag\r\n"
        "2003,1.50,alpha,A,0\r\n"
        "2004,2.25,\"b, c\",B,1\r\n"
        "2005,1e3,,C,1\r\n";
    std::string path = "/tmp/vison_b200_readf_test.csv";
    std::FILE* f = std::fopen(path.c_str(), "wb");
    std::fputs(text, f);
    std::fclose(f);
    vison_b200::Dataframe df;
    df.readf<0, 0, 4, 0, 0>(path, ',', true, '"');
    CHECK(df.get_nrow() == 3 && df.get_ncol() == 5);
    CHECK((df.get_typecol() == std::vector<char>{'u', 'd', 's', 'c', 'b'}));
    // the first-line pass keeps the CR of a CR LF in the last name (read_csv.hpp:62-69)
    CHECK((df.name_v == std::vector<std::string>{"year", "delay", "name", "code", "flag\r"}));
    CHECK((df.get_col<unsigned>(0) == std::vector<unsigned>{2003, 2004, 2005}));
    CHECK((df.get_col<double>(1) == std::vector<double>{1.5, 2.25, 1000.0}));
    CHECK((df.get_col<std::string>(2) == std::vector<std::string>{"alpha", "\"b, c\"", "NA"}));
    CHECK((df.get_col<std::string>(3) == std::vector<std::string>{"A", "B", "C"}));
    CHECK((df.get_col<uint8_t>(4) == std::vector<uint8_t>{0, 1, 1}));
    // a Hard sort by the double column permutes the string columns with it
    unsigned int k = 1;
    df.sort_by<0, void, true, false>(k);
    CHECK((df.get_col<std::string>(2) == std::vector<std::string>{"NA", "\"b, c\"", "alpha"}));
    // rows [1, 2) only
    vison_b200::Dataframe part;
    part.readf<1, 2>(path, ',', true, '"');
    CHECK(part.get_nrow() == 1 && part.get_col<unsigned>(0) == std::vector<unsigned>{2004});
    std::remove(path.c_str());
}

int main() {
    test_doc_example();
    test_hard_sort_and_view_composition();
    test_sort_by_external();
    test_transform_group_by();
    test_transform_group_by_gather();
    test_pivot();
    test_transform_unique();
    test_transform_left_join();
    test_readf();
    if (failures) {
        std::fprintf(stderr, "%d checks failed\n", failures);
        return 1;
    }
    std::printf("vison_b200 C++ layer: all checks passed\n");
    return 0;
}
