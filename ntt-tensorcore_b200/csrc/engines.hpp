// engines.hpp -- dispatch between the 31-bit engines.
#pragma once
#include <cuda_runtime.h>

#include <vector>

#include "plan.hpp"

namespace nttb {

// Runs one batched transform of a Plan32 with the requested engine
// (NTTB_ENGINE_*).  Returns 0 on success, 1 if the engine does not serve the
// shape, 2 on a launch failure.  src/dst hold u64 words when src_u64.
int run_transform32(Plan32& p, const void* src, void* dst, bool src_u64, uint32_t n_polys, bool inverse,
                    int engine, cudaStream_t s);

// Which engine AUTO resolves to for this plan (NTTB_ENGINE_*).
int auto_engine32(const Plan32& p, bool src_u64, uint64_t units);

// Frees engine caches attached to a plan.
void engines_release32(Plan32* p);

// The batch queue's tensor tiles as a plan engine (batch.cu): 2^13 .. 2^20.
bool tiles_serve(const Plan32& p);
int tiles_transform32(Plan32& p, const void* src, void* dst, bool u64, uint32_t n_polys, bool inverse, cudaStream_t s);
void tiles_release(Plan32* p);

int fail(int code, const char* fmt, ...);

// Byte-plane image of a 64 x 64 matrix W (mod q) as the INT8 contraction's
// B operand: 256 rows ordered (k / 32, a, k % 32) x 256 bytes, K-major SW128
// in two 128-byte K blocks (64 KB).  tc_dft_matrix(L, root, ...) returns
// W[k][j] = scale * row_twist^k * col_twist^j * root^(j k).
void tc_build_image64(uint8_t* img, const std::vector<uint64_t>& W, uint64_t q);
// Byte-plane image of a 16 x 16 matrix: 64 rows (a, k) x 64 bytes, K-major SW64 (4 KB).
void tc_build_image16(uint8_t* img, const std::vector<uint64_t>& W, uint64_t q);
std::vector<uint64_t> tc_dft_matrix(uint32_t L, uint64_t root, uint64_t q, uint64_t row_twist = 1,
                                    uint64_t col_twist = 1, uint64_t scale = 1);

}  // namespace nttb
