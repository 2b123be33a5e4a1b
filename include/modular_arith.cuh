// modular_arith.cuh -- drop-in for the reference's include/modular_arith.cuh.
//
// Same names, field layout and results as the reference header (ModularParams
// :11-19, prime constants :21-30, device helpers :34-106, host helpers
// :110-178), implemented here independently.  The generator rule of
// find_primitive_root (smallest g >= 2 passing the {2,3,5,7} test) is kept
// identical because omega -- and therefore every transform output -- depends
// on it.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace ntt {

struct ModularParams {
    uint64_t q;          // prime modulus
    uint64_t q_twice;    // 2q
    uint64_t barrett_k;  // smallest k >= 64 with 2^(k-64) >= q (capped at 96)
    uint64_t barrett_m;  // floor(2^k / q), truncated to 64 bits
    uint64_t omega;      // primitive n-th root of unity, g^((q-1)/n)
    uint64_t omega_inv;  // omega^-1
    uint64_t n_inv;      // n^-1 mod q
};

constexpr uint64_t PRIME_32_1 = 0xFFFFFFFF00000001ULL;  // Goldilocks 2^64 - 2^32 + 1
constexpr uint64_t PRIME_30_1 = 1073479681ULL;
constexpr uint64_t PRIME_30_2 = 1073610753ULL;
constexpr uint64_t PRIME_31_1 = 2013265921ULL;           // BabyBear 15 * 2^27 + 1
constexpr uint64_t PRIME_32_2 = 4293918721ULL;
constexpr uint64_t DEFAULT_PRIME = 2013265921ULL;

// ---- device helpers (operands < q) -----------------------------------------
__device__ __forceinline__ uint64_t mod_add(uint64_t a, uint64_t b, uint64_t q) {
    uint64_t s = a + b;
    return (s >= q || s < a) ? s - q : s;
}

__device__ __forceinline__ uint64_t mod_sub(uint64_t a, uint64_t b, uint64_t q) {
    return a >= b ? a - b : a + (q - b);
}

__device__ __forceinline__ uint64_t mod_mul_naive(uint64_t a, uint64_t b, uint64_t q) {
    return (uint64_t)(((unsigned __int128)a * b) % q);
}

// a*b mod q from the Barrett constant m = floor(2^k / q), k = barrett_k.
__device__ __forceinline__ uint64_t mod_mul_barrett(uint64_t a, uint64_t b, uint64_t q, uint64_t barrett_m,
                                                    int barrett_k) {
    unsigned __int128 x = (unsigned __int128)a * b;
    uint64_t lo = (uint64_t)x, hi = (uint64_t)(x >> 64);
    unsigned __int128 t = (unsigned __int128)hi * barrett_m + (((unsigned __int128)lo * barrett_m) >> 64);
    uint64_t qt = (uint64_t)(t >> (barrett_k - 64));
    uint64_t r = lo - qt * q;
    while (r >= q) r -= q;
    return r;
}

// 32-bit Montgomery arithmetic, R = 2^32 (q odd, q < 2^31).
struct Montgomery32 {
    uint32_t q;      // modulus
    uint32_t q_inv;  // -q^-1 mod 2^32
    uint32_t r2;     // R^2 mod q

    __device__ __forceinline__ uint32_t reduce(uint64_t a) const {
        uint32_t m = (uint32_t)a * q_inv;
        uint32_t r = (uint32_t)((a + (uint64_t)m * q) >> 32);
        return r >= q ? r - q : r;
    }
    __device__ __forceinline__ uint32_t mul(uint32_t a, uint32_t b) const { return reduce((uint64_t)a * b); }
    __device__ __forceinline__ uint32_t to_montgomery(uint32_t a) const { return reduce((uint64_t)a * r2); }
    __device__ __forceinline__ uint32_t from_montgomery(uint32_t a) const { return reduce(a); }
};

// ---- host helpers ------------------------------------------------------------
inline uint64_t mod_pow(uint64_t base, uint64_t exp, uint64_t mod) {
    uint64_t r = 1 % mod;
    base %= mod;
    for (; exp; exp >>= 1) {
        if (exp & 1) r = (uint64_t)(((unsigned __int128)r * base) % mod);
        base = (uint64_t)(((unsigned __int128)base * base) % mod);
    }
    return r;
}

inline uint64_t mod_inverse(uint64_t a, uint64_t mod) { return mod_pow(a, mod - 2, mod); }

inline uint64_t find_primitive_root(uint64_t q, uint64_t n) {
    const uint64_t small[4] = {2, 3, 5, 7};
    uint64_t g = 2;
    for (;; g++) {
        bool ok = true;
        for (uint64_t p : small)
            if ((q - 1) % p == 0 && mod_pow(g, (q - 1) / p, q) == 1) { ok = false; break; }
        if (ok) break;
    }
    return mod_pow(g, (q - 1) / n, q);
}

inline ModularParams create_params(uint64_t q, uint64_t n) {
    ModularParams p;
    int k = 64;
    while ((1ULL << (k - 64)) < q && k < 96) k++;
    p.q = q;
    p.q_twice = 2 * q;
    p.barrett_k = (uint64_t)k;
    p.barrett_m = (uint64_t)(((unsigned __int128)1 << k) / q);
    p.omega = find_primitive_root(q, n);
    p.omega_inv = mod_inverse(p.omega, q);
    p.n_inv = mod_inverse(n % q, q);
    return p;
}

inline void compute_twiddle_factors(uint64_t* twiddles, uint64_t n, uint64_t omega, uint64_t q) {
    uint64_t w = 1 % q;
    for (uint64_t i = 0; i < n; i++) {
        twiddles[i] = w;
        w = (uint64_t)(((unsigned __int128)w * omega) % q);
    }
}

}  // namespace ntt
