// bounds.cuh -- range checks of the NTT_DEBUG_BOUNDS build.
//
// compute-sanitizer is not available on every machine this library runs on,
// so the kernels whose addressing is computed by hand (the INT8 cluster
// kernel's swizzled shared-memory staging and distributed-shared-memory
// piece copies, the DMMA passes' tile coordinates, the batch queue's
// tickets, units and workspace slots) can be built with their own checks:
// `python ntt-tensorcore_b200/build.py --debug-bounds` compiles every source
// with -DNTT_DEBUG_BOUNDS into ntt_b200/libntt_b200_dbg.so.  There, each
// checked index or residue that falls outside its range sets one bit of a
// per-file device word (read by nttb_bounds_errors) and the access is
// skipped, so a bad index is reported instead of touching memory it must
// not.  The release build compiles every check away.
//
// Bits (one per kind of check, shared by the kernels of a file):
//   0  global-memory index outside the operand
//   1  shared-memory offset outside the buffer it addresses
//   2  distributed-shared-memory piece: peer rank or offsets out of range
//   3  queue ticket, unit or tile index out of range
//   4  workspace slot outside the batch's ring
//   5  output residue not reduced (>= q where canonical, >= 2^32 - q lazy)
//   6  input residue >= q (the caller's data break the input contract)
#pragma once
#include <cstdint>

#ifdef NTT_DEBUG_BOUNDS
#define NTTB_DEBUG_BOUNDS 1
// Evaluates to `cond`; records `bit` in `word` when it fails.
#define NTTB_CHECK(word, bit, cond) (::nttb::bounds_check((word), (bit), (cond)))
#else
#define NTTB_DEBUG_BOUNDS 0
#define NTTB_CHECK(word, bit, cond) (true)
#endif

namespace nttb {

enum : uint32_t {
    kBoundsGlobal = 0,
    kBoundsShared = 1,
    kBoundsCluster = 2,
    kBoundsQueue = 3,
    kBoundsWorkspace = 4,
    kBoundsResidue = 5,
    kBoundsInput = 6,
};

__device__ __forceinline__ bool bounds_check(uint32_t& word, uint32_t bit, bool cond) {
    if (!cond) atomicOr(&word, 1u << bit);
    return cond;
}

}  // namespace nttb
