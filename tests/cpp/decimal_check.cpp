// Host build of the field conversions in visondf_b200/csrc/vdf_decimal.cuh
// (the same source the CSV kernels compile): reads one field per line on
// stdin, prints "<f64 bits hex> <u32> <i32> <path>" per line, path 0 = fast
// (Clinger or the product), 1 = the exact big-integer decision.
#include <cstdio>
#include <cstring>
#include <string>

#include "vdf_decimal.cuh"

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
        std::printf("%016llx %u %d %d\n", (unsigned long long)bits, vdfdec::parse_u32(at, (uint32_t)n),
                    vdfdec::parse_i32(at, (uint32_t)n), path);
    }
    return 0;
}
