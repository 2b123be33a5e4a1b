// Forward-NTT timing under the harness convention of the reference's
// tests/icicle_compare.cu (TEST INFRASTRUCTURE ONLY).
//
// icicle_compare.cu sets the reference's ntt_forward_optimized beside the
// closed ICICLE library.  ICICLE is not present here, so this program keeps the
// harness and puts the two builds of the same entry point side by side:
//
//   _ref/reference_harness  compiled on the reference's own sources
//   _ref/dropin_harness     compiled on the drop-in include/ntt.cuh and
//                           linked with libntt_b200.so
//
// The convention (tests/icicle_compare.cu:79-108, 136-147, 178-200):
//   * BabyBear (DEFAULT_PRIME), forward transform, in place, in-domain only:
//     ntt_init and the upload stay outside the timed loop;
//   * sizes 2^12, 2^14, 2^16 .. 2^20, or the log2 sizes given as arguments;
//   * input: std::mt19937 seeded with 0xDEADBEEF ^ N, uniform in [0, q - 1];
//   * 10 warm-up calls, then 100 timed calls, each bracketed by a
//     cudaDeviceSynchronize and timed with events on the default stream;
//   * min, median (sorted sample iters / 2) and mean, in microseconds.
//
// After timing, one forward of a fresh copy of the input is compared with
// ntt_host on the same input, so that every printed row is checked.
#include "ntt.cuh"

#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <random>
#include <vector>

namespace {

void check(cudaError_t e, int line) {
    if (e != cudaSuccess) {
        std::fprintf(stderr, "CUDA error %s at line %d\n", cudaGetErrorString(e), line);
        std::exit(1);
    }
}
#define CHK(x) check((x), __LINE__)

struct Times { double min_us, med_us, avg_us; };

template <typename F>
Times time_calls(F&& call, int warmup, int iters) {
    cudaEvent_t t0, t1;
    CHK(cudaEventCreate(&t0));
    CHK(cudaEventCreate(&t1));
    for (int i = 0; i < warmup; i++) call();
    CHK(cudaDeviceSynchronize());
    std::vector<float> ms(iters);
    for (int i = 0; i < iters; i++) {
        CHK(cudaDeviceSynchronize());
        CHK(cudaEventRecord(t0));
        call();
        CHK(cudaEventRecord(t1));
        CHK(cudaDeviceSynchronize());
        CHK(cudaEventElapsedTime(&ms[i], t0, t1));
    }
    std::sort(ms.begin(), ms.end());
    double sum = 0;
    for (float v : ms) sum += v;
    CHK(cudaEventDestroy(t0));
    CHK(cudaEventDestroy(t1));
    return {ms.front() * 1e3, ms[iters / 2] * 1e3, sum / iters * 1e3};
}

}  // namespace

int main(int argc, char** argv) {
    constexpr int kWarmup = 10, kIters = 100;
    std::vector<int> logs;
    for (int i = 1; i < argc; i++) logs.push_back(std::atoi(argv[i]));
    if (logs.empty()) logs = {12, 14, 16, 17, 18, 19, 20};

    cudaDeviceProp prop;
    CHK(cudaGetDeviceProperties(&prop, 0));
    std::printf("GPU %s (sm_%d%d, %d SMs); q = %llu; forward, in place; %d warm-up, %d timed\n",
                prop.name, prop.major, prop.minor, prop.multiProcessorCount,
                (unsigned long long)ntt::DEFAULT_PRIME, kWarmup, kIters);
    std::printf("%-10s %10s %10s %10s  %s\n", "N", "min (us)", "med (us)", "avg (us)", "vs ntt_host");

    int failures = 0;
    for (int lg : logs) {
        if (lg < 1 || lg > 27) {
            std::fprintf(stderr, "log2 size %d out of range\n", lg);
            return 1;
        }
        const uint64_t n = 1ull << lg;
        std::mt19937 rng(0xDEADBEEFu ^ static_cast<uint32_t>(n));
        std::uniform_int_distribution<uint32_t> dist(0, static_cast<uint32_t>(ntt::DEFAULT_PRIME) - 1u);
        std::vector<uint64_t> in(n);
        for (auto& v : in) v = dist(rng);

        ntt::NTTConfig* cfg = ntt::ntt_init(n, ntt::DEFAULT_PRIME);
        uint64_t* d = nullptr;
        CHK(cudaMalloc(&d, n * sizeof(uint64_t)));
        CHK(cudaMemcpy(d, in.data(), n * sizeof(uint64_t), cudaMemcpyHostToDevice));
        const Times t = time_calls([&] { ntt::ntt_forward_optimized(d, cfg); }, kWarmup, kIters);

        CHK(cudaMemcpy(d, in.data(), n * sizeof(uint64_t), cudaMemcpyHostToDevice));
        ntt::ntt_forward_optimized(d, cfg);
        std::vector<uint64_t> got(n);
        CHK(cudaMemcpy(got.data(), d, n * sizeof(uint64_t), cudaMemcpyDeviceToHost));
        std::vector<uint64_t> want = in;
        ntt::ntt_host(want, cfg->params, false);
        const bool ok = got == want;
        failures += !ok;

        CHK(cudaFree(d));
        ntt::ntt_cleanup(cfg);
        std::printf("%-10llu %10.2f %10.2f %10.2f  %s\n", (unsigned long long)n, t.min_us, t.med_us,
                    t.avg_us, ok ? "equal" : "DIFFERENT");
        std::fflush(stdout);
    }
    return failures ? 2 : 0;
}
