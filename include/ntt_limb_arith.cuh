/*
 * ntt_limb_arith.cuh -- modular arithmetic on K-limb residues with 24-bit
 * limbs (little-endian uint32 words, each < 2^24), shared by the K-limb
 * kernels in libntt_b200.so and the ntt_arbitrary.cuh drop-in header.
 *
 * The representation is the reference's DScalar<K> (include/ntt_arbitrary.cuh:
 * LIMB_BITS = 24, Montgomery radix R = 2^(24 K)).  Every function takes and
 * returns canonical values in [0, p); they are pure functions of their
 * arguments, so any two correct implementations agree bit for bit.
 */
#ifndef NTT_LIMB_ARITH_CUH
#define NTT_LIMB_ARITH_CUH

#include <stdint.h>

#if defined(__CUDACC__)
#define NTTB_LIMB_HD __host__ __device__ __forceinline__
#else
#define NTTB_LIMB_HD inline
#endif

namespace nttb_limb {

constexpr int kBits = 24;
constexpr uint32_t kMask = (1u << kBits) - 1u;

// a >= p  (both K limbs)
template <int K>
NTTB_LIMB_HD bool geq(const uint32_t* a, const uint32_t* p) {
#pragma unroll
    for (int i = K - 1; i >= 0; i--) {
        if (a[i] != p[i]) return a[i] > p[i];
    }
    return true;
}

// r = a + b mod p
template <int K>
NTTB_LIMB_HD void add_mod(uint32_t* r, const uint32_t* a, const uint32_t* b, const uint32_t* p) {
    uint32_t s[K];
    uint32_t carry = 0;
#pragma unroll
    for (int i = 0; i < K; i++) {
        const uint32_t v = a[i] + b[i] + carry;  // < 2^25 + 1
        s[i] = v & kMask;
        carry = v >> kBits;
    }
    if (carry || geq<K>(s, p)) {
        int32_t borrow = 0;
#pragma unroll
        for (int i = 0; i < K; i++) {
            const int32_t v = (int32_t)s[i] - (int32_t)p[i] - borrow;
            borrow = v < 0;
            s[i] = (uint32_t)(v + (borrow << kBits));
        }
    }
#pragma unroll
    for (int i = 0; i < K; i++) r[i] = s[i];
}

// r = a - b mod p
template <int K>
NTTB_LIMB_HD void sub_mod(uint32_t* r, const uint32_t* a, const uint32_t* b, const uint32_t* p) {
    uint32_t d[K];
    int32_t borrow = 0;
#pragma unroll
    for (int i = 0; i < K; i++) {
        const int32_t v = (int32_t)a[i] - (int32_t)b[i] - borrow;
        borrow = v < 0;
        d[i] = (uint32_t)(v + (borrow << kBits));
    }
    if (borrow) {
        uint32_t carry = 0;
#pragma unroll
        for (int i = 0; i < K; i++) {
            const uint32_t v = d[i] + p[i] + carry;
            d[i] = v & kMask;
            carry = v >> kBits;
        }
    }
#pragma unroll
    for (int i = 0; i < K; i++) r[i] = d[i];
}

// r = a * b * 2^(-24 K) mod p (word-serial Montgomery, one limb of a per
// round: t = (t + a_i b + m p) / 2^24 with m = t_0 np mod 2^24, np = -p^-1).
// Inputs in [0, p); t stays below 2p, one final subtraction.
template <int K>
NTTB_LIMB_HD void mont_mul(uint32_t* r, const uint32_t* a, const uint32_t* b, const uint32_t* p, uint32_t np) {
    uint64_t t[K + 1];
#pragma unroll
    for (int j = 0; j <= K; j++) t[j] = 0;
#pragma unroll
    for (int i = 0; i < K; i++) {
        const uint64_t ai = a[i];
        uint64_t c = 0;
#pragma unroll
        for (int j = 0; j < K; j++) {
            const uint64_t v = t[j] + ai * b[j] + c;
            t[j] = v & kMask;
            c = v >> kBits;
        }
        t[K] += c;
        const uint64_t m = ((t[0] * np) & kMask);
        c = (t[0] + m * p[0]) >> kBits;
#pragma unroll
        for (int j = 1; j < K; j++) {
            const uint64_t v = t[j] + m * p[j] + c;
            t[j - 1] = v & kMask;
            c = v >> kBits;
        }
        const uint64_t v = t[K] + c;
        t[K - 1] = v & kMask;
        t[K] = v >> kBits;
    }
    uint32_t s[K];
#pragma unroll
    for (int j = 0; j < K; j++) s[j] = (uint32_t)t[j];
    if (t[K] || geq<K>(s, p)) {
        int32_t borrow = 0;
#pragma unroll
        for (int i = 0; i < K; i++) {
            const int32_t v = (int32_t)s[i] - (int32_t)p[i] - borrow;
            borrow = v < 0;
            s[i] = (uint32_t)(v + (borrow << kBits));
        }
    }
#pragma unroll
    for (int i = 0; i < K; i++) r[i] = s[i];
}

// -p^-1 mod 2^24 for odd p (Newton iteration on the low limb).
NTTB_LIMB_HD uint32_t neg_inv24(uint32_t p0) {
    uint32_t inv = p0;  // correct to 3 bits for odd p0
    for (int i = 0; i < 5; i++) inv *= 2u - p0 * inv;
    return (0u - inv) & kMask;
}

}  // namespace nttb_limb

#endif  // NTT_LIMB_ARITH_CUH
