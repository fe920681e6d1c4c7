// vdf_agg.cuh -- per-column group aggregates shared by the segmented
// reduction (vdf_segreduce.cu) and the one-CTA-per-query batch kernel
// (vdf_batch_small.cu), so both give identical results: canonical 64-bit
// value images, an exact 128-bit integer sum, a TwoSum-compensated f64 sum,
// and min/max in the column's order.
#pragma once
#include "vdf_common.cuh"

namespace vdf {

enum VClass : int { VC_FLOAT = 0, VC_SINT = 1, VC_UINT = 2 };
__device__ __forceinline__ int vclass(int dt) {
    return (dt == F64 || dt == F32) ? VC_FLOAT : (dt == I32 || dt == I64) ? VC_SINT : VC_UINT;
}
__device__ __forceinline__ double as_f(uint64_t b) { return __longlong_as_double((long long)b); }
__device__ __forceinline__ uint64_t as_b(double d) { return (uint64_t)__double_as_longlong(d); }

// Canonical 64-bit image of a value: double bits for float columns, the
// sign- or zero-extended integer otherwise.
__device__ __forceinline__ uint64_t load_val(const void* src, int dt, uint64_t i) {
    switch (dt) {
    case I32: return (uint64_t)(int64_t)__ldg(static_cast<const int32_t*>(src) + i);
    case U32: return (uint64_t)__ldg(static_cast<const uint32_t*>(src) + i);
    case F32: return as_b((double)__ldg(static_cast<const float*>(src) + i));
    default: return (uint64_t)__ldg(static_cast<const unsigned long long*>(src) + i);
    }
}
// Per value column accumulator words:
//   float : w0 sum, w1 compensation, w2 min, w3 max   (double bits)
//   int   : w0 sum low, w1 sum high (128-bit two's complement), w2 min, w3 max
__device__ __forceinline__ void col_init(uint64_t* w, uint64_t x, int vc) {
    w[0] = x;
    w[1] = (vc == VC_SINT && (int64_t)x < 0) ? ~0ull : 0ull;  // 0.0 for floats
    w[2] = x;
    w[3] = x;
}
__device__ __forceinline__ void col_merge(uint64_t* a, const uint64_t* b, int vc) {
    if (vc == VC_FLOAT) {
        const double x = as_f(a[0]), y = as_f(b[0]);
        const double s = __dadd_rn(x, y);
        const double bp = __dsub_rn(s, x);
        const double e = __dadd_rn(__dsub_rn(x, __dsub_rn(s, bp)), __dsub_rn(y, bp));  // TwoSum error
        a[0] = as_b(s);
        a[1] = as_b(__dadd_rn(__dadd_rn(as_f(a[1]), as_f(b[1])), e));
        a[2] = as_b(fmin(as_f(a[2]), as_f(b[2])));
        a[3] = as_b(fmax(as_f(a[3]), as_f(b[3])));
    } else {
        const uint64_t lo = a[0] + b[0];
        a[1] = a[1] + b[1] + (lo < a[0] ? 1ull : 0ull);
        a[0] = lo;
        if (vc == VC_SINT) {
            a[2] = (uint64_t)min((long long)a[2], (long long)b[2]);
            a[3] = (uint64_t)max((long long)a[3], (long long)b[3]);
        } else {
            a[2] = min((unsigned long long)a[2], (unsigned long long)b[2]);
            a[3] = max((unsigned long long)a[3], (unsigned long long)b[3]);
        }
    }
}

__device__ __forceinline__ double i128_to_double(uint64_t lo, uint64_t hi, bool is_signed) {
    if (is_signed) {
        if ((int64_t)hi == ((int64_t)lo >> 63)) return (double)(int64_t)lo;
        return ldexp((double)(int64_t)hi, 64) + (double)lo;
    }
    if (hi == 0) return (double)lo;
    return ldexp((double)hi, 64) + (double)lo;
}

}  // namespace vdf
