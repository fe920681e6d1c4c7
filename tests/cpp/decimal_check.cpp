// Host build of the field conversions in visondf_b200/csrc/vdf_decimal.cuh
// (the same source the CSV kernels compile): reads one field per line on
// stdin, prints "<f64 bits hex> <u32> <i32> <path> <scan>" per line, path 0 =
// fast (Clinger or the product), 1 = the exact big-integer decision; scan 0 =
// the eight-bytes-at-a-time scan declined the field, 1 = it took it and gave
// exactly the general scan's result, 2 = it took it and differed.
#include <cstdio>
#include <cstring>
#include <string>

#include "vdf_decimal.cuh"

// The byte source interface the CSV parse kernel gives scan_number_fast.
struct ArrayReader {
    const char* s;
    size_t n;
    unsigned char get(uint64_t i) const { return i < n ? (unsigned char)s[i] : 0; }
    uint64_t get8(uint64_t i, uint32_t avail) const {
        uint64_t v = 0;
        for (uint32_t k = 0; k < 8 && k < avail; ++k) v |= (uint64_t)get(i + k) << (8 * k);
        return v;
    }
};

int main() {
    static char line[1 << 16];
    while (std::fgets(line, sizeof line, stdin)) {
        size_t n = std::strlen(line);
        while (n && (line[n - 1] == '\n' || line[n - 1] == '\r')) --n;
        auto at = [&](uint32_t i) { return (unsigned char)line[i]; };
        const vdfdec::Conv c = vdfdec::convert(vdfdec::scan_number(at, (uint32_t)n));
        double v = c.v;
        int path = 0;
        if (c.ambiguous) {
            bool ok = true;
            v = vdfdec::slow_decide(at, (uint32_t)n, ok);
            path = ok ? 1 : 2;
        }
        uint64_t bits;
        std::memcpy(&bits, &v, 8);
        ArrayReader rd{line, n};
        vdfdec::Number fast{};
        const vdfdec::Number slow = vdfdec::scan_number(at, (uint32_t)n);
        int scan = 0;
        if (vdfdec::scan_number_fast(rd, 0, (uint32_t)n, fast))
            scan = (fast.w == slow.w && fast.q == slow.q && fast.kind == slow.kind && fast.neg == slow.neg &&
                    fast.many == slow.many) ? 1 : 2;
        std::printf("%016llx %u %d %d %d\n", (unsigned long long)bits, vdfdec::parse_u32(at, (uint32_t)n),
                    vdfdec::parse_i32(at, (uint32_t)n), path, scan);
    }
    return 0;
}
