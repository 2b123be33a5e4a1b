// arith.cuh -- modular arithmetic shared by every kernel of the library.
//
// Residues are kept in plain (non-Montgomery) form in memory.  Twiddle
// constants are stored pre-multiplied by the Montgomery radix R, so one
// Montgomery product  mul(x, w*R)  yields  x*w mod q  directly.
//
//   M32 : q < 2^31, R = 2^32   (31-bit RNS primes, BabyBear)
//   M64 : q < 2^62, R = 2^64   (60-bit primes, the K=2 49-bit field)
//
// Both follow the same contract: inputs of mul/add/sub are canonical
// (< q), outputs are canonical.
#pragma once
#include <cstdint>

#ifndef __CUDACC__
#define __host__
#define __device__
#define __forceinline__ inline
#endif

namespace nttb {

// ---- host helpers (exact, unsigned __int128) -------------------------------
inline uint64_t h_mulmod(uint64_t a, uint64_t b, uint64_t q) {
    return (uint64_t)(((unsigned __int128)a * b) % q);
}
inline uint64_t h_powmod(uint64_t b, uint64_t e, uint64_t q) {
    uint64_t r = 1 % q;
    b %= q;
    while (e) {
        if (e & 1) r = h_mulmod(r, b, q);
        b = h_mulmod(b, b, q);
        e >>= 1;
    }
    return r;
}
inline uint64_t h_invmod(uint64_t a, uint64_t q) { return h_powmod(a, q - 2, q); }

// -q^-1 mod 2^32 / 2^64 by Newton iteration (q odd).
inline uint32_t h_neg_inv32(uint32_t q) {
    uint32_t x = q;  // correct to 3 bits for odd q
    for (int i = 0; i < 5; i++) x *= 2u - q * x;
    return 0u - x;
}
inline uint64_t h_neg_inv64(uint64_t q) {
    uint64_t x = q;
    for (int i = 0; i < 6; i++) x *= 2ull - q * x;
    return 0ull - x;
}
// x * 2^32 mod q and x * 2^64 mod q
inline uint32_t h_to_mont32(uint64_t x, uint64_t q) {
    return (uint32_t)((((unsigned __int128)(x % q)) << 32) % q);
}
inline uint64_t h_to_mont64(uint64_t x, uint64_t q) {
    return (uint64_t)((((unsigned __int128)(x % q)) << 64) % q);
}

// ---- device arithmetic ------------------------------------------------------
struct M32 {
    using elem = uint32_t;
    static constexpr bool kLazy = false;  // 4q does not fit 32 bits for 31-bit moduli
    uint32_t q, qinv;  // qinv = -q^-1 mod 2^32

    // Montgomery product: a * b * 2^-32 mod q, for a*b < q * 2^32; canonical.
    __device__ __forceinline__ uint32_t mul(uint32_t a, uint32_t b) const {
        uint64_t t = (uint64_t)a * b;
        uint32_t m = (uint32_t)t * qinv;
        uint32_t r = (uint32_t)((t + (uint64_t)m * q) >> 32);
        return r >= q ? r - q : r;
    }
    // Shoup product a * w mod q for any a and w < q, ws = floor(w * 2^32 / q); canonical.
    __device__ __forceinline__ uint32_t mul_shoup(uint32_t a, uint32_t w, uint32_t ws) const {
        const uint32_t r = a * w - __umulhi(a, ws) * q;  // in [0, 2q)
        return r >= q ? r - q : r;
    }
    __device__ __forceinline__ uint32_t add(uint32_t a, uint32_t b) const {
        uint32_t s = a + b;
        return s >= q ? s - q : s;
    }
    __device__ __forceinline__ uint32_t sub(uint32_t a, uint32_t b) const {
        uint32_t d = a - b;
        return a >= b ? d : d + q;
    }
};

struct M64 {
    using elem = uint64_t;
    // q < 2^62: values in [0, 4q) fit a word, so butterflies may run lazily
    // (D. Harvey, "Faster arithmetic for number-theoretic transforms", 2014)
    static constexpr bool kLazy = true;
    uint64_t q, qinv;  // qinv = -q^-1 mod 2^64, q < 2^62

    __device__ __forceinline__ uint64_t mul(uint64_t a, uint64_t b) const {
#ifdef __CUDA_ARCH__
        uint64_t lo = a * b, hi = __umul64hi(a, b);
        uint64_t m = lo * qinv;
        uint64_t r = hi + __umul64hi(m, q) + (lo != 0);
#else
        unsigned __int128 t = (unsigned __int128)a * b;
        uint64_t lo = (uint64_t)t, hi = (uint64_t)(t >> 64);
        uint64_t m = lo * qinv;
        uint64_t r = hi + (uint64_t)(((unsigned __int128)m * q) >> 64) + (lo != 0);
#endif
        return r >= q ? r - q : r;
    }
    // Shoup product a * w mod q for any a and w < q, ws = floor(w * 2^64 / q); canonical.
    __device__ __forceinline__ uint64_t mul_shoup(uint64_t a, uint64_t w, uint64_t ws) const {
        const uint64_t r = mul_shoup_lazy(a, w, ws);
        return r >= q ? r - q : r;
    }
    // The same product in [0, 2q).
    __device__ __forceinline__ uint64_t mul_shoup_lazy(uint64_t a, uint64_t w, uint64_t ws) const {
        return a * w - __umul64hi(a, ws) * q;
    }
    // x in [0, 4q) -> [0, 2q)
    __device__ __forceinline__ uint64_t below2q(uint64_t x) const { return x >= 2 * q ? x - 2 * q : x; }
    // x in [0, 4q) -> canonical
    __device__ __forceinline__ uint64_t canon4(uint64_t x) const {
        x = below2q(x);
        return x >= q ? x - q : x;
    }
    __device__ __forceinline__ uint64_t add(uint64_t a, uint64_t b) const {
        uint64_t s = a + b;
        return s >= q ? s - q : s;
    }
    __device__ __forceinline__ uint64_t sub(uint64_t a, uint64_t b) const {
        uint64_t d = a - b;
        return a >= b ? d : d + q;
    }
};

__host__ __device__ __forceinline__ uint32_t bitrev(uint32_t x, int bits) {
#ifdef __CUDA_ARCH__
    return bits ? (__brev(x) >> (32 - bits)) : 0u;
#else
    uint32_t r = 0;
    for (int i = 0; i < bits; i++) r |= ((x >> i) & 1u) << (bits - 1 - i);
    return r;
#endif
}

}  // namespace nttb
