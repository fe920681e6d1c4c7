// Calibration program, not part of the library: times the CUDA toolkit's CUB
// radix sort (cub::DeviceRadixSort::SortPairs) on the shapes of the library's
// key sorts -- 100M random 64-bit keys with 32-bit row ids, and 100M random
// 32-bit keys with 32-bit row ids -- and prints one JSON line per shape.
// Build and run:
//   nvcc -gencode arch=compute_100a,code=sm_100a -O3 -o cub_sort_pairs cub_sort_pairs.cu && ./cub_sort_pairs
#include <cub/cub.cuh>

#include <cstdint>
#include <cstdio>
#include <random>
#include <vector>

#define CHECK(x)                                                                          \
    do {                                                                                  \
        cudaError_t e_ = (x);                                                             \
        if (e_ != cudaSuccess) {                                                          \
            std::printf("CUDA error %s at line %d\n", cudaGetErrorString(e_), __LINE__); \
            return 1;                                                                     \
        }                                                                                 \
    } while (0)

template <typename K>
int time_sort(size_t n, int reps) {
    std::vector<K> hk(n);
    std::vector<uint32_t> hv(n);
    std::mt19937_64 g(0xB200);
    for (size_t i = 0; i < n; ++i) {
        hk[i] = (K)g();
        hv[i] = (uint32_t)i;
    }
    K *kin, *kout;
    uint32_t *vin, *vout;
    CHECK(cudaMalloc(&kin, n * sizeof(K)));
    CHECK(cudaMalloc(&kout, n * sizeof(K)));
    CHECK(cudaMalloc(&vin, n * 4));
    CHECK(cudaMalloc(&vout, n * 4));
    CHECK(cudaMemcpy(kin, hk.data(), n * sizeof(K), cudaMemcpyHostToDevice));
    CHECK(cudaMemcpy(vin, hv.data(), n * 4, cudaMemcpyHostToDevice));
    size_t tmp_bytes = 0;
    CHECK(cub::DeviceRadixSort::SortPairs(nullptr, tmp_bytes, kin, kout, vin, vout, (int)n));
    void* tmp;
    CHECK(cudaMalloc(&tmp, tmp_bytes));
    cudaEvent_t a, b;
    CHECK(cudaEventCreate(&a));
    CHECK(cudaEventCreate(&b));
    float best = 1e30f, sum = 0.f;
    const int warmup = 3;
    for (int r = 0; r < warmup + reps; ++r) {
        CHECK(cudaEventRecord(a));
        CHECK(cub::DeviceRadixSort::SortPairs(tmp, tmp_bytes, kin, kout, vin, vout, (int)n));
        CHECK(cudaEventRecord(b));
        CHECK(cudaEventSynchronize(b));
        float ms = 0.f;
        CHECK(cudaEventElapsedTime(&ms, a, b));
        if (r >= warmup) {
            best = ms < best ? ms : best;
            sum += ms;
        }
    }
    CHECK(cudaMemcpy(hk.data(), kout, n * sizeof(K), cudaMemcpyDeviceToHost));
    size_t unsorted = 0;
    for (size_t i = 1; i < n; ++i) unsorted += hk[i - 1] > hk[i];
    std::printf("{\"sort\": \"cub::DeviceRadixSort::SortPairs\", \"key_bytes\": %d, \"value_bytes\": 4, \"rows\": %zu, "
                "\"best_ms\": %.4f, \"mean_ms\": %.4f, \"reps\": %d, \"unsorted_pairs\": %zu}\n",
                (int)sizeof(K), n, best, sum / reps, reps, unsorted);
    cudaFree(kin);
    cudaFree(kout);
    cudaFree(vin);
    cudaFree(vout);
    cudaFree(tmp);
    return unsorted ? 1 : 0;
}

int main() {
    const size_t n = 100000000;
    if (time_sort<uint64_t>(n, 5)) return 1;
    return time_sort<uint32_t>(n, 5);
}
