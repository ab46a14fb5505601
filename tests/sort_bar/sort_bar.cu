// Sort bar: the library's one-sweep radix sort (home-measure-privacy_b200/csrc/sort.cu)
// against cub::DeviceRadixSort::SortPairs on the same keys, at the key counts and widths
// of the training step's two sorts (the benchmark workload: 8 x 1,000,064 (view,
// Gaussian) pairs on 31-bit depth keys, about 51M key instances on 16-bit tile ids).
// TEST INFRASTRUCTURE ONLY: CUB is the timing comparator here and nothing in the library
// uses it.  Prints one JSON line per case; exits non-zero if either result is not the
// stable order of the keys.
//
//     nvcc -gencode arch=compute_100a,code=sm_100a -O3 -std=c++17 --expt-relaxed-constexpr
//          -I include -I home-measure-privacy_b200/csrc tests/sort_bar/sort_bar.cu
//          home-measure-privacy_b200/csrc/sort.cu -o sort_bar
#include <cub/device/device_radix_sort.cuh>

#include <cstdio>
#include <cstdlib>
#include <vector>

#include "internal.h"

#define CK(x)                                                                          \
    do {                                                                               \
        cudaError_t e_ = (x);                                                          \
        if (e_ != cudaSuccess) {                                                       \
            fprintf(stderr, "%s:%d %s: %s\n", __FILE__, __LINE__, #x, cudaGetErrorString(e_)); \
            exit(2);                                                                   \
        }                                                                              \
    } while (0)

static uint64_t splitmix(uint64_t& s) {
    uint64_t z = (s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

// Keys like the step's: depth float bits of depths uniform in [1, 8] with 30 % culled
// pairs at the 0x7fffffff sentinel (pairs), or tile ids uniform below `tiles`
// (instances, which arrive in depth order, so their tile ids look random).
static std::vector<uint32_t> make_keys(size_t n, bool depth, uint32_t tiles) {
    std::vector<uint32_t> k(n);
    uint64_t s = 12345;
    for (size_t i = 0; i < n; i++) {
        const uint64_t r = splitmix(s);
        if (depth) {
            if ((r & 1023) < 307) {
                k[i] = 0x7fffffffu;
            } else {
                const float d = 1.0f + 7.0f * (float)((r >> 11) & 0xffffff) / 16777216.0f;
                memcpy(&k[i], &d, 4);
            }
        } else {
            k[i] = (uint32_t)((r >> 16) % tiles);
        }
    }
    return k;
}

static bool stable_sorted(const std::vector<uint32_t>& in, const std::vector<uint32_t>& k,
                          const std::vector<uint32_t>& v) {
    for (size_t i = 0; i < k.size(); i++) {
        if (k[i] != in[v[i]]) return false;
        if (i && (k[i - 1] > k[i] || (k[i - 1] == k[i] && v[i - 1] >= v[i]))) return false;
    }
    return true;
}

int main() {
    struct Case {
        const char* name;
        size_t n;
        int bits;
        bool depth;
    } cases[] = {{"sort_pairs", 8ull * 1000064ull, 31, true}, {"sort_instances", 51000000ull, 16, false}};
    int device = 0, sms = 0;
    CK(cudaGetDevice(&device));
    CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    CK(gs::radix_prepare());
    bool ok = true;
    for (const Case& cs : cases) {
        const size_t n = cs.n;
        const std::vector<uint32_t> keys = make_keys(n, cs.depth, 35932);
        std::vector<uint32_t> iota(n);
        for (size_t i = 0; i < n; i++) iota[i] = (uint32_t)i;
        uint32_t *k0, *k1, *v0, *v1, *kin, *vin;
        CK(cudaMalloc(&k0, n * 4));
        CK(cudaMalloc(&k1, n * 4));
        CK(cudaMalloc(&v0, n * 4));
        CK(cudaMalloc(&v1, n * 4));
        CK(cudaMalloc(&kin, n * 4));
        CK(cudaMalloc(&vin, n * 4));
        CK(cudaMemcpy(kin, keys.data(), n * 4, cudaMemcpyHostToDevice));
        CK(cudaMemcpy(vin, iota.data(), n * 4, cudaMemcpyHostToDevice));
        cudaStream_t st;
        CK(cudaStreamCreate(&st));
        cudaEvent_t e0, e1;
        CK(cudaEventCreate(&e0));
        CK(cudaEventCreate(&e1));
        const int reps = 10, warm = 3;
        // ---- the library's sort
        const int parts = (int)((n + gs::radix_tile_items() - 1) / gs::radix_tile_items());
        unsigned long long* hist;
        uint32_t* totals;
        gs::SegInfo* seg;
        unsigned int* flags;
        CK(cudaMalloc(&hist, (size_t)parts * 256 * 8));
        CK(cudaMalloc(&totals, 4096 * 4));
        CK(cudaMalloc(&seg, sizeof(gs::SegInfo)));
        CK(cudaMalloc(&flags, 16));
        CK(cudaMemset(flags, 0, 16));
        gs::SegInfo h{0u, (unsigned)n};
        CK(cudaMemcpy(seg, &h, sizeof h, cudaMemcpyHostToDevice));
        gs::RadixSortArgs ra;
        memset(&ra, 0, sizeof ra);
        ra.keys = k0;
        ra.vals = v0;
        ra.keys_alt = k1;
        ra.vals_alt = v1;
        ra.iota = 1;
        ra.seg = seg;
        ra.begin_bit = 0;
        ra.end_bit = cs.bits;
        ra.hist = hist;
        ra.totals = totals;
        ra.max_parts = parts;
        ra.timeout = flags;
        ra.debug_wait = nullptr;
        ra.never_set = flags + 1;
        float ours = 0.f;
        for (int r = 0; r < warm + reps; r++) {
            CK(cudaMemcpyAsync(k0, kin, n * 4, cudaMemcpyDeviceToDevice, st));
            CK(cudaEventRecord(e0, st));
            gs::launch_radix_sort(ra, st, sms);
            CK(cudaEventRecord(e1, st));
            CK(cudaStreamSynchronize(st));
            float ms = 0.f;
            CK(cudaEventElapsedTime(&ms, e0, e1));
            if (r >= warm) ours += ms / reps;
        }
        std::vector<uint32_t> ko(n), vo(n);
        CK(cudaMemcpy(ko.data(), k0, n * 4, cudaMemcpyDeviceToHost));  // an even number of passes: back in k0
        CK(cudaMemcpy(vo.data(), v0, n * 4, cudaMemcpyDeviceToHost));
        const bool ours_ok = stable_sorted(keys, ko, vo);
        unsigned int timeout = 0;
        CK(cudaMemcpy(&timeout, flags, 4, cudaMemcpyDeviceToHost));
        // ---- CUB
        size_t temp_bytes = 0;
        CK(cub::DeviceRadixSort::SortPairs(nullptr, temp_bytes, kin, k1, vin, v1, (int)n, 0, cs.bits, st));
        void* temp;
        CK(cudaMalloc(&temp, temp_bytes));
        float cub_ms = 0.f;
        for (int r = 0; r < warm + reps; r++) {
            CK(cudaEventRecord(e0, st));
            CK(cub::DeviceRadixSort::SortPairs(temp, temp_bytes, kin, k1, vin, v1, (int)n, 0, cs.bits, st));
            CK(cudaEventRecord(e1, st));
            CK(cudaStreamSynchronize(st));
            float ms = 0.f;
            CK(cudaEventElapsedTime(&ms, e0, e1));
            if (r >= warm) cub_ms += ms / reps;
        }
        CK(cudaMemcpy(ko.data(), k1, n * 4, cudaMemcpyDeviceToHost));
        CK(cudaMemcpy(vo.data(), v1, n * 4, cudaMemcpyDeviceToHost));
        const bool cub_ok = stable_sorted(keys, ko, vo);
        const int passes = gs::radix_sort_passes(0, cs.bits);
        printf("{\"case\": \"%s\", \"n\": %zu, \"bits\": %d, \"library_ms\": %.4f, \"library_passes\": %d, "
               "\"cub_ms\": %.4f, \"library_sorted\": %s, \"cub_sorted\": %s, \"timeout\": %u}\n",
               cs.name, n, cs.bits, ours, passes, cub_ms, ours_ok ? "true" : "false", cub_ok ? "true" : "false",
               timeout);
        fflush(stdout);
        ok = ok && ours_ok && cub_ok && timeout == 0;
        CK(cudaFree(temp));
        CK(cudaFree(hist));
        CK(cudaFree(totals));
        CK(cudaFree(seg));
        CK(cudaFree(flags));
        for (uint32_t* p : {k0, k1, v0, v1, kin, vin}) CK(cudaFree(p));
        CK(cudaEventDestroy(e0));
        CK(cudaEventDestroy(e1));
        CK(cudaStreamDestroy(st));
    }
    return ok ? 0 : 1;
}
