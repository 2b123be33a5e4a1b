// serve.cu -- the serving loop: polynomial products and NTTs (negacyclic by
// default) of mixed sizes and limb counts, admitted against an HBM budget and
// batched continuously.
//
// A product request is (a, b) in host memory: n_limbs rows of 2^log_n
// residues, row l reduced mod moduli[first_modulus + l]; its result a * b
// (per limb) goes to `out` in host memory.  Its device footprint is
// 2 x n_limbs x 2^log_n words (a, with the result written over it, and b).
// An NTT request is one such operand, transformed forward or inverse in
// place on the device (footprint n_limbs x 2^log_n words); both kinds share
// the queue and the batches.
//
// One worker thread owns the device side.  Device memory for requests is one
// region of (budget - resident tables and queues) bytes, carved first-fit in
// 256-byte granules.  Whenever a stream slot is free and the queue is not
// empty, the worker admits requests in arrival order while their operands fit
// in the region (and the batch stays under max_batch_requests /
// max_batch_residues), and issues the batch on the slot's stream: host ->
// device copies of every operand, ONE persistent batch launch (per product
// and limb: forward a, forward b, pointwise product, inverse; per NTT and
// limb: the transform), device -> host copies of the results, and a host callback that stamps the completion time, returns
// the memory to the region and frees the slot.  Several slots are in flight
// at once, so a batch's copies and kernels overlap with its neighbours', and
// requests that arrive while others run are admitted as soon as memory and a
// slot come free: continuous batching, not a queue drained batch by batch.
// Latency is submit -> completion callback, on the host's steady clock.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <map>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../../include/ntt_b200.h"
#include "arena.hpp"
#include "batch.hpp"
#include "engines.hpp"

namespace nttb {
namespace {

double now_s() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

enum ReqKind : uint32_t { kProduct = 0, kForward = 1, kInverse = 2 };

struct Req {
    const uint32_t* a = nullptr;
    const uint32_t* b = nullptr;  // products only
    uint32_t* out = nullptr;
    uint32_t kind = kProduct;
    uint32_t log_n = 0, limbs = 0, first = 0;
    size_t words = 0;  // per operand
    size_t off = 0;    // device offset of a; b follows
    size_t bytes() const { return (kind == kProduct ? 2 : 1) * words * 4; }
    size_t residues() const { return (kind == kProduct ? 3 : 1) * words; }  // transform work
    double t_submit = 0, t_done = 0;
    int status = NTTB_OK;
    bool done = false;
    bool device = false;  // a, b, out are device memory (copies stay in HBM)
};

}  // namespace
}  // namespace nttb

struct nttb_server;

namespace nttb {
namespace {
struct Slot {
    nttb_server* srv = nullptr;
    cudaStream_t stream = nullptr;
    BatchRunner* runner = nullptr;
    bool busy = false;
    std::vector<uint64_t> ids;
    std::vector<nttb_batch_job> jobs;
};
}  // namespace
}  // namespace nttb

struct nttb_server {
    int device = 0;
    nttb_server_config cfg{};
    nttb_batch_plan* plan = nullptr;
    uint8_t* region = nullptr;
    size_t resident = 0;
    nttb::Arena arena;
    std::mutex mu;
    std::condition_variable cv;
    std::deque<uint64_t> queue;
    std::unordered_map<uint64_t, nttb::Req> reqs;
    uint64_t next_id = 1;
    std::vector<nttb::Slot> slots;
    std::thread worker;
    bool stop = false;
    uint64_t submitted = 0, completed = 0, batches = 0, batched_requests = 0;
    std::vector<double> latencies;
};

namespace nttb {
namespace {

// Host callback at the end of a batch: no CUDA calls here.
void CUDART_CB batch_done(void* p) {
    Slot* sl = static_cast<Slot*>(p);
    nttb_server* s = sl->srv;
    std::lock_guard<std::mutex> lk(s->mu);
    const double t = now_s();
    for (uint64_t id : sl->ids) {
        Req& r = s->reqs[id];
        r.t_done = t;
        r.done = true;
        s->arena.release(r.off, r.bytes());
        s->latencies.push_back(t - r.t_submit);
        s->completed++;
    }
    sl->ids.clear();
    sl->busy = false;
    s->cv.notify_all();
}

void worker_main(nttb_server* s) {
    cudaSetDevice(s->device);
    std::unique_lock<std::mutex> lk(s->mu);
    for (;;) {
        auto free_slot = [&]() -> Slot* {
            for (Slot& sl : s->slots)
                if (!sl.busy) return &sl;
            return nullptr;
        };
        s->cv.wait(lk, [&] { return s->stop || (!s->queue.empty() && free_slot()); });
        if (s->stop) break;
        Slot* sl = free_slot();
        // admit in arrival order while memory and the batch limits allow
        std::vector<uint64_t> ids;
        size_t residues = 0;
        while (!s->queue.empty() && ids.size() < s->cfg.max_batch_requests) {
            Req& r = s->reqs[s->queue.front()];
            if (!ids.empty() && residues + r.residues() > s->cfg.max_batch_residues) break;
            size_t off = 0;
            if (!s->arena.alloc(r.bytes(), &off)) break;
            r.off = off;
            ids.push_back(s->queue.front());
            residues += r.residues();
            s->queue.pop_front();
        }
        if (ids.empty()) {  // memory is full: wait for a batch to finish
            const uint64_t c0 = s->completed;
            s->cv.wait(lk, [&] { return s->stop || s->completed != c0; });
            continue;
        }
        sl->busy = true;
        sl->ids = ids;
        sl->jobs.clear();
        std::vector<Req> work;
        for (uint64_t id : ids) {
            const Req& r = s->reqs[id];
            work.push_back(r);
            nttb_batch_job j{};
            j.data = reinterpret_cast<uint32_t*>(s->region + r.off);
            j.pointwise = r.kind == kProduct ? j.data + r.words : nullptr;
            j.log_n = r.log_n;
            j.n_limbs = r.limbs;
            j.first_modulus = r.first;
            j.flags = (r.kind == kProduct ? NTTB_BATCH_POLYMUL : r.kind == kInverse ? NTTB_BATCH_INVERSE : 0u) |
                      (s->cfg.negacyclic ? NTTB_NEGACYCLIC : 0u);
            sl->jobs.push_back(j);
        }
        s->batches++;
        s->batched_requests += ids.size();
        lk.unlock();
        // issue the batch on the slot's stream (no lock held: CUDA calls)
        bool ok = true;
        for (size_t i = 0; i < work.size() && ok; i++) {
            const size_t bytes = work[i].words * 4;
            const cudaMemcpyKind in = work[i].device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
            ok = cudaMemcpyAsync(sl->jobs[i].data, work[i].a, bytes, in, sl->stream) == cudaSuccess &&
                 (work[i].kind != kProduct ||
                  cudaMemcpyAsync(sl->jobs[i].pointwise, work[i].b, bytes, in, sl->stream) == cudaSuccess);
        }
        ok = ok && runner_run(sl->runner, sl->jobs.data(), (uint32_t)sl->jobs.size(), sl->stream) == 0;
        for (size_t i = 0; i < work.size() && ok; i++)
            ok = cudaMemcpyAsync(work[i].out, sl->jobs[i].data, work[i].words * 4,
                                 work[i].device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost,
                                 sl->stream) == cudaSuccess;
        ok = ok && cudaLaunchHostFunc(sl->stream, batch_done, sl) == cudaSuccess;
        lk.lock();
        if (!ok) {  // nothing will call back: fail the batch's requests here
            for (uint64_t id : ids) s->reqs[id].status = NTTB_ERR_CUDA;
            lk.unlock();
            cudaStreamSynchronize(sl->stream);
            batch_done(sl);
            lk.lock();
        }
    }
}

}  // namespace
}  // namespace nttb

using nttb::fail;

extern "C" {

NTTB_API int nttb_server_default_config(nttb_server_config* out) {
    if (!out) return fail(NTTB_ERR_INVALID_ARG, "nttb_server_default_config: null");
    *out = nttb_server_config{};
    out->hbm_budget_bytes = 60ull << 30;
    out->max_log_n = 17;
    out->slots = 3;
    out->max_batch_requests = 64;
    out->negacyclic = 1;
    out->max_batch_residues = 1ull << 27;
    nttb_batch_default_config(&out->batch);
    return NTTB_OK;
}

NTTB_API int nttb_server_create(const uint64_t* moduli, uint32_t n_moduli, const nttb_server_config* cfg,
                                nttb_server** out) {
    if (!cfg || !out) return fail(NTTB_ERR_INVALID_ARG, "nttb_server_create: null argument");
    if (cfg->slots < 1 || cfg->slots > 16) return fail(NTTB_ERR_INVALID_ARG, "nttb_server_create: slots in [1, 16]");
    if (cfg->max_batch_requests < 1 || cfg->max_batch_residues < 1)
        return fail(NTTB_ERR_INVALID_ARG, "nttb_server_create: batch limits must be positive");
    auto* s = new nttb_server();
    s->cfg = *cfg;
    cudaGetDevice(&s->device);
    if (int rc = nttb_batch_plan_create(moduli, n_moduli, cfg->max_log_n, cfg->negacyclic ? NTTB_NEGACYCLIC : 0,
                                        &s->plan)) {
        delete s;
        return rc;
    }
    s->resident = nttb::batch_plan_device_bytes(&s->plan->p);
    s->slots.resize(cfg->slots);
    for (nttb::Slot& sl : s->slots) {
        sl.srv = s;
        if (cudaStreamCreateWithFlags(&sl.stream, cudaStreamNonBlocking) != cudaSuccess ||
            nttb::runner_create(&s->plan->p, cfg->batch, &sl.runner)) {
            for (nttb::Slot& t : s->slots) {
                if (t.runner) nttb::runner_destroy(t.runner);
                if (t.stream) cudaStreamDestroy(t.stream);
            }
            nttb_batch_plan_destroy(s->plan);
            delete s;
            return fail(NTTB_ERR_NO_MEMORY, "nttb_server_create: stream slots");
        }
        s->resident += nttb::runner_device_bytes(sl.runner);
    }
    if (cfg->hbm_budget_bytes <= s->resident + (1u << 20)) {
        for (nttb::Slot& t : s->slots) {
            nttb::runner_destroy(t.runner);
            cudaStreamDestroy(t.stream);
        }
        nttb_batch_plan_destroy(s->plan);
        const size_t res = s->resident;
        delete s;
        return fail(NTTB_ERR_BUDGET, "nttb_server_create: budget below the resident tables and queues (%zu bytes)", res);
    }
    const size_t region = cfg->hbm_budget_bytes - s->resident;
    if (cudaMalloc(&s->region, region) != cudaSuccess) {
        for (nttb::Slot& t : s->slots) {
            nttb::runner_destroy(t.runner);
            cudaStreamDestroy(t.stream);
        }
        nttb_batch_plan_destroy(s->plan);
        delete s;
        return fail(NTTB_ERR_NO_MEMORY, "nttb_server_create: request region of %zu bytes", region);
    }
    s->arena.init(region);
    s->worker = std::thread(nttb::worker_main, s);
    *out = s;
    return NTTB_OK;
}

}  // extern "C"

namespace nttb {
namespace {

int submit_request(nttb_server* s, Req r, const char* what, uint64_t* id) {
    if (r.log_n < 1 || r.log_n > s->cfg.max_log_n)
        return fail(NTTB_ERR_INVALID_ARG, "%s: log_n %u outside [1, %u]", what, r.log_n, s->cfg.max_log_n);
    if (r.limbs == 0 || (uint64_t)r.first + r.limbs > s->plan->p.limbs.size())
        return fail(NTTB_ERR_INVALID_ARG, "%s: limbs outside the server's moduli", what);
    r.words = (size_t)r.limbs << r.log_n;
    std::lock_guard<std::mutex> lk(s->mu);
    if (round_up(r.bytes()) > s->arena.size())
        return fail(NTTB_ERR_BUDGET, "%s: %zu bytes exceed the HBM budget's request region (%zu)", what, r.bytes(),
                    s->arena.size());
    r.t_submit = now_s();
    *id = s->next_id++;
    s->reqs[*id] = r;
    s->queue.push_back(*id);
    s->submitted++;
    s->cv.notify_all();
    return NTTB_OK;
}

}  // namespace
}  // namespace nttb

extern "C" {

NTTB_API int nttb_server_submit(nttb_server* s, const uint32_t* a, const uint32_t* b, uint32_t* out, uint32_t log_n,
                                uint32_t n_limbs, uint32_t first_modulus, uint64_t* id) {
    if (!s || !a || !b || !out || !id) return fail(NTTB_ERR_INVALID_ARG, "nttb_server_submit: null argument");
    nttb::Req r;
    r.a = a;
    r.b = b;
    r.out = out;
    r.kind = nttb::kProduct;
    r.log_n = log_n;
    r.limbs = n_limbs;
    r.first = first_modulus;
    return nttb::submit_request(s, r, "nttb_server_submit", id);
}

NTTB_API int nttb_server_submit_ntt(nttb_server* s, const uint32_t* in, uint32_t* out, uint32_t log_n,
                                    uint32_t n_limbs, uint32_t first_modulus, int inverse, uint64_t* id) {
    if (!s || !in || !out || !id) return fail(NTTB_ERR_INVALID_ARG, "nttb_server_submit_ntt: null argument");
    nttb::Req r;
    r.a = in;
    r.out = out;
    r.kind = inverse ? nttb::kInverse : nttb::kForward;
    r.log_n = log_n;
    r.limbs = n_limbs;
    r.first = first_modulus;
    return nttb::submit_request(s, r, "nttb_server_submit_ntt", id);
}

NTTB_API int nttb_server_submit_device(nttb_server* s, int kind, const uint32_t* d_a, const uint32_t* d_b,
                                       uint32_t* d_out, uint32_t log_n, uint32_t n_limbs, uint32_t first_modulus,
                                       uint64_t* id) {
    static const char* what = "nttb_server_submit_device";
    if (!s || !d_a || !d_out || !id) return fail(NTTB_ERR_INVALID_ARG, "%s: null argument", what);
    if (kind < NTTB_SERVER_PRODUCT || kind > NTTB_SERVER_INVERSE)
        return fail(NTTB_ERR_INVALID_ARG, "%s: kind must be NTTB_SERVER_PRODUCT, _FORWARD or _INVERSE", what);
    if (kind == NTTB_SERVER_PRODUCT && !d_b) return fail(NTTB_ERR_INVALID_ARG, "%s: a product needs b", what);
    const void* ptrs[3] = {d_a, kind == NTTB_SERVER_PRODUCT ? (const void*)d_b : (const void*)d_a, d_out};
    for (const void* p : ptrs) {
        cudaPointerAttributes at{};
        if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
            cudaGetLastError();
            return fail(NTTB_ERR_INVALID_ARG, "%s: not a CUDA pointer", what);
        }
        if (at.type != cudaMemoryTypeDevice || at.device != s->device)
            return fail(NTTB_ERR_INVALID_ARG, "%s: operands must be device memory of the server's device %d", what,
                        s->device);
    }
    nttb::Req r;
    r.a = d_a;
    r.b = kind == NTTB_SERVER_PRODUCT ? d_b : nullptr;
    r.out = d_out;
    r.kind = kind == NTTB_SERVER_PRODUCT ? nttb::kProduct : kind == NTTB_SERVER_FORWARD ? nttb::kForward : nttb::kInverse;
    r.log_n = log_n;
    r.limbs = n_limbs;
    r.first = first_modulus;
    r.device = true;
    return nttb::submit_request(s, r, what, id);
}

NTTB_API int nttb_server_wait(nttb_server* s, uint64_t id, double timeout_s, double* latency_s) {
    if (!s) return fail(NTTB_ERR_INVALID_ARG, "nttb_server_wait: null server");
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->reqs.find(id);
    if (it == s->reqs.end()) return fail(NTTB_ERR_INVALID_ARG, "nttb_server_wait: unknown request %llu", (unsigned long long)id);
    // find() rather than operator[]: a concurrent wait on the same id may
    // collect (erase) the record while this one sleeps
    const bool done = s->cv.wait_for(lk, std::chrono::duration<double>(timeout_s), [&] {
        auto w = s->reqs.find(id);
        return w == s->reqs.end() || w->second.done;
    });
    if (!done) return fail(NTTB_ERR_TIMEOUT, "nttb_server_wait: request %llu not done", (unsigned long long)id);
    it = s->reqs.find(id);
    if (it == s->reqs.end())
        return fail(NTTB_ERR_INVALID_ARG, "nttb_server_wait: request %llu collected by another wait",
                    (unsigned long long)id);
    const nttb::Req r = it->second;
    s->reqs.erase(it);
    if (latency_s) *latency_s = r.t_done - r.t_submit;
    return r.status == NTTB_OK ? NTTB_OK : fail(r.status, "nttb_server_wait: request %llu failed", (unsigned long long)id);
}

NTTB_API int nttb_server_drain(nttb_server* s, double timeout_s) {
    if (!s) return fail(NTTB_ERR_INVALID_ARG, "nttb_server_drain: null server");
    std::unique_lock<std::mutex> lk(s->mu);
    const bool ok = s->cv.wait_for(lk, std::chrono::duration<double>(timeout_s),
                                   [&] { return s->completed == s->submitted; });
    return ok ? NTTB_OK : fail(NTTB_ERR_TIMEOUT, "nttb_server_drain: requests still pending");
}

NTTB_API int nttb_server_stats(nttb_server* s, nttb_server_stats_t* out) {
    if (!s || !out) return fail(NTTB_ERR_INVALID_ARG, "nttb_server_stats: null argument");
    std::lock_guard<std::mutex> lk(s->mu);
    out->submitted = s->submitted;
    out->completed = s->completed;
    out->queued = s->queue.size();
    out->batches = s->batches;
    out->batched_requests = s->batched_requests;
    out->bytes_in_use = s->arena.used();
    out->peak_bytes_in_use = s->arena.peak();
    out->region_bytes = s->arena.size();
    out->resident_bytes = s->resident;
    return NTTB_OK;
}

NTTB_API int nttb_server_latencies(nttb_server* s, double* out, uint64_t cap, uint64_t* count, int reset) {
    if (!s || !count) return fail(NTTB_ERR_INVALID_ARG, "nttb_server_latencies: null argument");
    std::lock_guard<std::mutex> lk(s->mu);
    *count = s->latencies.size();
    if (out)
        for (uint64_t i = 0; i < cap && i < s->latencies.size(); i++) out[i] = s->latencies[i];
    if (reset) s->latencies.clear();
    return NTTB_OK;
}

NTTB_API int nttb_server_destroy(nttb_server* s) {
    if (!s) return NTTB_OK;
    nttb_server_drain(s, 600.0);
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
        s->cv.notify_all();
    }
    s->worker.join();
    for (nttb::Slot& sl : s->slots) {
        cudaStreamSynchronize(sl.stream);
        nttb::runner_destroy(sl.runner);
        cudaStreamDestroy(sl.stream);
    }
    cudaFree(s->region);
    nttb_batch_plan_destroy(s->plan);
    delete s;
    return NTTB_OK;
}

}  // extern "C"
