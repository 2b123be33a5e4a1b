// noalloc.cu -- in-place RNS transform that allocates no device memory.
//
// For callers that cannot call cudaMalloc at transform time: code running
// inside a memory manager that owns all device memory, a real-time loop that
// must never enter the allocator (cudaMalloc can synchronize the device and
// stall every stream), or a process whose memory budget is fixed up front.
// The ordinary in-place transform stages its first pass in a workspace that
// the plan allocates on first use; this entry point stages it in a
// library-owned static device buffer instead.
//
// The buffer is a file-scope __device__ array, so every GPU that loads the
// library holds NTTB_NOALLOC_SCRATCH_BYTES of device memory until the
// process exits.  Host code cannot use the array's name as a device address;
// the first call on each device looks the address up with
// cudaGetSymbolAddress (with that device current) and caches it.  Make that
// first call before any stream capture.  The cached address is not looked up
// again: after cudaDeviceReset a process must not call this entry point
// again on that device.  The plan's device must be the current device.  All calls share the one buffer and
// it keeps the previous call's contents: the first pass writes every word
// the second pass reads, so nothing needs clearing, but two calls whose work
// overlaps on the GPU (different streams, no ordering) race on the buffer.
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>

#include "../../include/ntt_b200.h"
#include "engines.hpp"
#include "plan.hpp"

namespace nttb {

const Plan32* rns_plan_core(const nttb_rns_plan* p);

namespace {

constexpr size_t kScratchWords = NTTB_NOALLOC_SCRATCH_BYTES / sizeof(uint32_t);
__device__ __align__(256) uint32_t g_noalloc_scratch[kScratchWords];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
uint32_t* g_addr[kMaxDevices] = {};

// Device address of the static scratch on the current device (set-up on
// first use per device).  Returns nullptr and sets the error on failure.
uint32_t* scratch_address(int* status) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
        *status = fail(NTTB_ERR_CUDA, "rns_transform_noalloc: no current CUDA device");
        return nullptr;
    }
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_addr[dev]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p) {
            *status = fail(NTTB_ERR_CUDA, "rns_transform_noalloc: cudaGetSymbolAddress failed: %s",
                           cudaGetErrorString(e));
            return nullptr;
        }
        g_addr[dev] = static_cast<uint32_t*>(p);
    }
    return g_addr[dev];
}

}  // namespace
}  // namespace nttb

using namespace nttb;

extern "C" int nttb_rns_transform_noalloc(const nttb_rns_plan* plan, uint32_t* d_data, uint32_t n_polys,
                                          int inverse, void* stream) {
    const Plan32* p = rns_plan_core(plan);
    if (!p || !d_data) return fail(NTTB_ERR_INVALID_ARG, "rns_transform_noalloc: null argument");
    if (n_polys == 0) return NTTB_OK;
    if (n_polys > 65535) return fail(NTTB_ERR_INVALID_ARG, "rns_transform_noalloc: n_polys > 65535");
    if (((uintptr_t)d_data) & 15) return fail(NTTB_ERR_INVALID_ARG, "rns_transform_noalloc: pointer must be 16-byte aligned");
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess || dev != p->device)
        return fail(NTTB_ERR_INVALID_ARG,
                    "rns_transform_noalloc: the plan's device (%d) must be the current device (%d)", p->device, dev);
    // shapes that run as one pass stage nothing and are not limited
    const size_t need = scalar_transform32_ws_bytes(*p, n_polys);
    if (need > NTTB_NOALLOC_SCRATCH_BYTES)
        return fail(NTTB_ERR_INVALID_ARG,
                    "rns_transform_noalloc: batch needs %zu bytes of scratch; the static scratch holds %u bytes "
                    "(use fewer polynomials per call)",
                    need, (unsigned)NTTB_NOALLOC_SCRATCH_BYTES);
    int status = NTTB_OK;
    uint32_t* ws = scratch_address(&status);
    if (!ws) return status;
    const int rc = scalar_transform32_ws(*p, d_data, ws, n_polys, inverse != 0, (cudaStream_t)stream);
    return engine_status(rc, "rns_transform_noalloc");
}
