// tc_arith.cuh -- arithmetic of the INT8 byte-plane contraction, shared by
// the tensor-core kernels (tc_int8.cu, the batch engine's tensor tiles).
//
// A length-64 DFT of vectors x (64 residues < 2^32) is one u8 x u8 -> s32
// GEMM with K = 256 bytes: operand A holds the residues as they are (a K-major
// row of 64 little-endian words IS the row of 256 byte planes), operand B
// holds, per modulus, B[(a, k)][(j, p)] = byte a of ((256^p * 2^32 * W[k][j])
// mod q).  The four INT32 planes D[m][(a, k)] of a vector sit in one TMEM
// lane; sum_a 256^a D == 2^32 (W x)_k (mod q) is below 2^49, and one
// Montgomery REDC by 2^32 returns (W x)_k in [0, 2q).
#pragma once
#include <cstdint>

#include "tcgen05.cuh"

namespace nttb {
namespace tca {

// 32 x 32 + 64 -> 64 multiply-add (one mad.wide.u32).
__device__ __forceinline__ uint64_t mad_wide(uint32_t a, uint32_t b, uint64_t c) {
    uint64_t r;
    asm("mad.wide.u32 %0, %1, %2, %3;" : "=l"(r) : "r"(a), "r"(b), "l"(c));
    return r;
}
__device__ __forceinline__ uint32_t redc64(uint64_t v, uint32_t q, uint32_t qinv) {
    const uint32_t m = (uint32_t)v * qinv;
    return (uint32_t)(mad_wide(m, q, v) >> 32);  // [0, 2q) for v < q * 2^32
}
// Planes c_a <= 256 * 255^2 (K = 256 byte products), so c0 + 256 c1 and
// c2 + 256 c3 fit in 32 bits; v = sum_a 256^a c_a < 2^49.
__device__ __forceinline__ uint32_t combine_redc(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3, uint32_t q,
                                                 uint32_t qinv) {
    const uint32_t lo = c0 + (c1 << 8), hi = c2 + (c3 << 8);
    return redc64(mad_wide(hi, 65536u, (uint64_t)lo), q, qinv);
}
// a < 2q, b < q -> a*b*2^-32 mod q in [0, 2q)
__device__ __forceinline__ uint32_t mont_lazy(uint32_t a, uint32_t b, uint32_t q, uint32_t qinv) {
    return redc64(mad_wide(a, b, 0ull), q, qinv);
}
__device__ __forceinline__ uint32_t canon(uint32_t x, uint32_t q) { return x >= q ? x - q : x; }
// a * b mod q in [0, 2q) for any a < 2^32 and b < q, given bs = floor(b * 2^32 / q)
// (Shoup's product with a precomputed quotient): three single-width multiplies.
__device__ __forceinline__ uint32_t shoup_lazy(uint32_t a, uint32_t b, uint32_t bs, uint32_t q) {
    return a * b - __umulhi(a, bs) * q;
}

// Issues the K = 256-byte contraction (8 MMAs of K = 32, M = 128) into TMEM
// columns [tmem, tmem + N).  A and B are K-major SW128 with two 128-byte K
// blocks of `a_rows` / `b_rows` rows.  The caller commits.
__device__ __forceinline__ void issue_k256(uint32_t tmem, uint32_t a0, uint32_t a_rows, uint32_t b0, uint32_t b_rows,
                                           uint32_t N) {
    const uint32_t idesc = tc::idesc_u8(128, N);
#pragma unroll
    for (uint32_t ks = 0; ks < 8; ks++) {
        const uint32_t ka = a0 + (ks >> 2) * a_rows * 128u + (ks & 3u) * 32u;
        const uint32_t kb = b0 + (ks >> 2) * b_rows * 128u + (ks & 3u) * 32u;
        tc::mma_i8(tmem, tc::desc_k_sw128(ka), tc::desc_k_sw128(kb), idesc, ks > 0);
    }
}

// Eight outputs' four planes (a = 0..3 at columns col + 32a) of this thread's
// TMEM lane (one N = 128 output half: columns a * 32 + k % 32).
__device__ __forceinline__ void ld_planes8(uint32_t col, uint32_t (&c0)[8], uint32_t (&c1)[8], uint32_t (&c2)[8],
                                           uint32_t (&c3)[8]) {
    tc::ld_32x32b_x8(col + 0, c0);
    tc::ld_32x32b_x8(col + 32, c1);
    tc::ld_32x32b_x8(col + 64, c2);
    tc::ld_32x32b_x8(col + 96, c3);
    tc::ld_wait();
}

}  // namespace tca
}  // namespace nttb
