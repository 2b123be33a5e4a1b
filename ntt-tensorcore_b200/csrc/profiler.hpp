// profiler.hpp -- launch accounting for every kernel the library launches.
//
// Every launch increments a counter.  While profiling is on, CUDA events are
// recorded on the launching stream before and after the launch, so that the
// per-kernel device time can be read back after a synchronize.
#pragma once
#include <cuda_runtime.h>

namespace nttb {

void prof_begin(const char* kernel, cudaStream_t s);
void prof_end(cudaStream_t s);

struct ProfScope {
    cudaStream_t s;
    ProfScope(const char* kernel, cudaStream_t st) : s(st) { prof_begin(kernel, st); }
    ~ProfScope() { prof_end(s); }
};

}  // namespace nttb
