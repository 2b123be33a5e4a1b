// batch.hpp -- the uneven-batch engine's host structures, shared by the C ABI
// (batch.cu) and the serving loop (serve.cu).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

#include "../../include/ntt_b200.h"
#include "plan.hpp"

namespace nttb {

// Twiddle tables of a modulus set at sizes up to 2^max_log (batch.cu).
struct BatchPlan {
    struct Mods;  // device modulus table
    uint32_t max_log = 0;
    bool negacyclic = false;
    std::vector<LimbHost> limbs;
    Mods* mods = nullptr;
    uint8_t* images = nullptr;  // DFT-64 images of the tensor-core tiles (max_log >= 13), 3 x 64 KB per modulus
    std::vector<void*> allocations;
    nttb_batch_config tuned{};
    bool have_tuned = false;
};

// Runs job lists one after another on preallocated queue and workspace
// buffers: planning on the host, upload from pinned staging and the
// persistent launch all go on the caller's stream, with no allocation unless
// a job list outgrows every earlier one.  One run per runner in flight.
struct BatchRunner;
int runner_create(BatchPlan* plan, const nttb_batch_config& cfg, BatchRunner** out);
int runner_run(BatchRunner* r, const nttb_batch_job* jobs, uint32_t n_jobs, cudaStream_t s);
void runner_destroy(BatchRunner* r);
size_t runner_device_bytes(const BatchRunner* r);
size_t batch_plan_device_bytes(const BatchPlan* plan);

}  // namespace nttb

struct nttb_batch_plan {
    nttb::BatchPlan p;
};
