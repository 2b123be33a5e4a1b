// engines.hpp -- dispatch between the 31-bit engines.
#pragma once
#include <cuda_runtime.h>

#include "plan.hpp"

namespace nttb {

// Runs one batched transform of a Plan32 with the requested engine
// (NTTB_ENGINE_*).  Returns 0 on success, 1 if the engine does not serve the
// shape, 2 on a launch failure.  src/dst hold u64 words when src_u64.
int run_transform32(Plan32& p, const void* src, void* dst, bool src_u64, uint32_t n_polys, bool inverse,
                    int engine, cudaStream_t s);

// Which engine AUTO resolves to for this plan (NTTB_ENGINE_*).
int auto_engine32(const Plan32& p, bool src_u64);

// Frees engine caches attached to a plan.
void engines_release32(Plan32* p);

int fail(int code, const char* fmt, ...);

}  // namespace nttb
