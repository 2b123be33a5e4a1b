// profiler.cu -- launch counter and optional per-launch CUDA-event timing.
#include <cuda_runtime.h>

#include <atomic>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/ntt_b200.h"
#include "profiler.hpp"

namespace nttb {

namespace {
struct Rec {
    const char* name;
    cudaEvent_t a, b;
};
std::atomic<uint64_t> g_launches{0};
std::atomic<bool> g_on{false};
std::mutex g_mu;
std::vector<Rec> g_recs;
std::vector<cudaEvent_t> g_pool;
thread_local const char* t_name = nullptr;
thread_local cudaEvent_t t_start = nullptr;

cudaEvent_t take_event() {
    if (!g_pool.empty()) {
        cudaEvent_t e = g_pool.back();
        g_pool.pop_back();
        return e;
    }
    cudaEvent_t e;
    cudaEventCreate(&e);
    return e;
}

struct Summary {
    std::string name;
    uint64_t launches;
    double total_ms;
};
std::vector<Summary> g_summary;
}  // namespace

void prof_begin(const char* kernel, cudaStream_t s) {
    g_launches.fetch_add(1, std::memory_order_relaxed);
    if (!g_on.load(std::memory_order_relaxed)) return;
    std::lock_guard<std::mutex> lk(g_mu);
    t_name = kernel;
    t_start = take_event();
    cudaEventRecord(t_start, s);
}

void prof_end(cudaStream_t s) {
    if (!g_on.load(std::memory_order_relaxed) || !t_start) return;
    std::lock_guard<std::mutex> lk(g_mu);
    cudaEvent_t b = take_event();
    cudaEventRecord(b, s);
    g_recs.push_back({t_name, t_start, b});
    t_start = nullptr;
}

}  // namespace nttb

using namespace nttb;

extern "C" {

int nttb_launch_count(uint64_t* out) {
    if (!out) return NTTB_ERR_INVALID_ARG;
    *out = g_launches.load();
    return NTTB_OK;
}

int nttb_profile_start(void) {
    std::lock_guard<std::mutex> lk(g_mu);
    for (auto& r : g_recs) {
        g_pool.push_back(r.a);
        g_pool.push_back(r.b);
    }
    g_recs.clear();
    g_summary.clear();
    g_on = true;
    return NTTB_OK;
}

int nttb_profile_stop(uint32_t* n_kernels) {
    g_on = false;
    std::lock_guard<std::mutex> lk(g_mu);
    std::map<std::string, Summary> acc;
    for (auto& r : g_recs) {
        if (cudaEventSynchronize(r.b) != cudaSuccess) return NTTB_ERR_CUDA;
        float ms = 0.f;
        cudaEventElapsedTime(&ms, r.a, r.b);
        auto& s = acc[r.name];
        s.name = r.name;
        s.launches++;
        s.total_ms += ms;
    }
    g_summary.clear();
    for (auto& kv : acc) g_summary.push_back(kv.second);
    if (n_kernels) *n_kernels = (uint32_t)g_summary.size();
    return NTTB_OK;
}

int nttb_profile_read(uint32_t index, char* name, uint32_t name_len, uint64_t* launches, double* total_ms) {
    std::lock_guard<std::mutex> lk(g_mu);
    if (index >= g_summary.size() || !name || name_len == 0) return NTTB_ERR_INVALID_ARG;
    std::strncpy(name, g_summary[index].name.c_str(), name_len - 1);
    name[name_len - 1] = 0;
    if (launches) *launches = g_summary[index].launches;
    if (total_ms) *total_ms = g_summary[index].total_ms;
    return NTTB_OK;
}

}  // extern "C"
