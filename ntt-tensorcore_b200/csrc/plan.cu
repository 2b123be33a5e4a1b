// plan.cu -- host-side construction of per-modulus constants and device tables.
#include <cuda_runtime.h>

#include <cstring>
#include <type_traits>
#include <string>
#include <vector>

#include "plan.hpp"

namespace nttb {

// Smallest g >= 2 with g^((q-1)/p) != 1 for every p in {2,3,5,7} dividing
// q-1: the generator rule of include/modular_arith.cuh:130-147, kept
// identical so that omega (and hence every output) matches the reference.
uint64_t reference_generator(uint64_t q) {
    static const uint64_t small[4] = {2, 3, 5, 7};
    for (uint64_t g = 2; g < q; g++) {
        bool ok = true;
        for (uint64_t p : small)
            if ((q - 1) % p == 0 && h_powmod(g, (q - 1) / p, q) == 1) { ok = false; break; }
        if (ok) return g;
    }
    return 0;
}

static bool probably_prime(uint64_t q) {
    if (q < 2) return false;
    for (uint64_t p : {2ull, 3ull, 5ull, 7ull, 11ull, 13ull, 17ull, 19ull, 23ull, 29ull, 31ull, 37ull}) {
        if (q % p == 0) return q == p;
    }
    uint64_t d = q - 1;
    int r = 0;
    while ((d & 1) == 0) { d >>= 1; r++; }
    for (uint64_t a : {2ull, 3ull, 5ull, 7ull, 11ull, 13ull, 17ull, 19ull, 23ull, 29ull, 31ull, 37ull}) {
        uint64_t x = h_powmod(a, d, q);
        if (x == 1 || x == q - 1) continue;
        bool comp = true;
        for (int i = 1; i < r; i++) {
            x = h_mulmod(x, x, q);
            if (x == q - 1) { comp = false; break; }
        }
        if (comp) return false;
    }
    return true;
}

bool make_limb_host(uint64_t q, uint64_t n, bool need_psi, LimbHost* out, std::string* why) {
    if (q < 3 || (q & 1) == 0) { *why = "modulus must be an odd prime"; return false; }
    if (!probably_prime(q)) { *why = "modulus " + std::to_string(q) + " is not prime"; return false; }
    const uint64_t order = need_psi ? 2 * n : n;
    if ((q - 1) % order != 0) {
        *why = "modulus " + std::to_string(q) + " has no primitive " + std::to_string(order) + "-th root (q-1 not divisible)";
        return false;
    }
    LimbHost L;
    L.q = q;
    L.g = reference_generator(q);
    L.omega = h_powmod(L.g, (q - 1) / n, q);
    // The reference's generator test only screens {2,3,5,7}; require that the
    // resulting omega really has order n (it always does for the supported
    // primes because the p = 2 test makes g a non-residue).
    if (n > 1 && h_powmod(L.omega, n / 2, q) == 1) { *why = "omega is not a primitive n-th root"; return false; }
    L.omega_inv = h_invmod(L.omega, q);
    L.n_inv = h_invmod(n % q, q);
    if (need_psi) {
        L.psi = h_powmod(L.g, (q - 1) / (2 * n), q);
        L.psi_inv = h_invmod(L.psi, q);
    }
    *out = L;
    return true;
}

template <class E, class ToMont>
static void fill_powers(E* dst, uint64_t base, uint64_t start, uint64_t n, uint64_t q, ToMont tm) {
    uint64_t x = start % q;
    for (uint64_t e = 0; e < n; e++) {
        dst[e] = tm(x);
        x = h_mulmod(x, base, q);
    }
}

// Shoup pairs of the roots of each length L = 2^l <= n, level by level:
// pairs 2^(l-1) - 1 + k = (root_L^k, floor(root_L^k * 2^bits / q)), k < L/2,
// root_L = root_n^(n/L); n - 1 pairs in all.
template <class E>
static void fill_shoup_levels(E* dst, uint64_t root_n, uint32_t log_n, uint64_t q) {
    for (uint32_t l = 1; l <= log_n; l++) {
        const uint64_t step = h_powmod(root_n, 1ull << (log_n - l), q);
        E* lvl = dst + 2 * ((1ull << (l - 1)) - 1);
        uint64_t x = 1 % q;
        for (uint64_t k = 0; k < (1ull << (l - 1)); k++) {
            lvl[2 * k] = (E)x;
            if constexpr (sizeof(E) == 4) lvl[2 * k + 1] = (E)((x << 32) / q);
            else lvl[2 * k + 1] = (E)(((unsigned __int128)x << 64) / q);
            x = h_mulmod(x, step, q);
        }
    }
}

template <class A, class PlanT, class ToMont>
static int build_common(PlanT* p, uint32_t log_n, const uint64_t* moduli, uint32_t n_limbs, bool negacyclic,
                        uint64_t qmax, ToMont tm, std::string* why) {
    using E = typename A::elem;
    p->log_n = log_n;
    p->n = 1u << log_n;
    p->n_limbs = n_limbs;
    p->negacyclic = negacyclic;
    if constexpr (std::is_same<PlanT, Plan32>::value) {
        if (cudaGetDevice(&p->device) != cudaSuccess) p->device = -1;
    }
    const uint64_t n = p->n;
    if (n_limbs == 0) { *why = "no moduli"; return 1; }
    p->limbs.resize(n_limbs);
    for (uint32_t l = 0; l < n_limbs; l++) {
        if (moduli[l] >= qmax) { *why = "modulus " + std::to_string(moduli[l]) + " too large for this path"; return 1; }
        if (!make_limb_host(moduli[l], n, negacyclic, &p->limbs[l], why)) return 1;
    }
    // omega^e, omega^-e (, psi^e, n^-1 psi^-e) in Montgomery form, then the
    // level-by-level Shoup pairs of the forward and inverse roots (2n words each)
    const uint32_t tables = negacyclic ? 4 : 2;
    const size_t per_limb = (size_t)(tables + 4) * n;
    std::vector<E> host(per_limb * n_limbs);
    std::vector<LimbDev<A>> devs(n_limbs);
    E* d_tables = nullptr;
    if (cudaMalloc(&d_tables, host.size() * sizeof(E)) != cudaSuccess) { *why = "cudaMalloc failed"; return 4; }
    p->allocations.push_back(d_tables);
    for (uint32_t l = 0; l < n_limbs; l++) {
        const LimbHost& L = p->limbs[l];
        const uint64_t q = L.q;
        E* h = host.data() + per_limb * l;
        E* d = d_tables + per_limb * l;
        fill_powers(h, L.omega, 1, n, q, [&](uint64_t x) { return tm(x, q); });
        fill_powers(h + n, L.omega_inv, 1, n, q, [&](uint64_t x) { return tm(x, q); });
        LimbDev<A> dv{};
        dv.tw = d;
        dv.tw_inv = d + n;
        if (negacyclic) {
            fill_powers(h + 2 * n, L.psi, 1, n, q, [&](uint64_t x) { return tm(x, q); });
            fill_powers(h + 3 * n, L.psi_inv, L.n_inv, n, q, [&](uint64_t x) { return tm(x, q); });
            dv.psi = d + 2 * n;
            dv.psi_inv = d + 3 * n;
        }
        fill_shoup_levels(h + (size_t)tables * n, L.omega, log_n, q);
        fill_shoup_levels(h + (size_t)(tables + 2) * n, L.omega_inv, log_n, q);
        dv.tw_sh = d + (size_t)tables * n;
        dv.tw_inv_sh = d + (size_t)(tables + 2) * n;
        dv.ninv_m = (E)tm(L.n_inv, q);
        devs[l] = dv;
    }
    for (uint32_t l = 0; l < n_limbs; l++) {
        const uint64_t q = p->limbs[l].q;
        devs[l].ar.q = (E)q;
        if constexpr (sizeof(E) == 4) devs[l].ar.qinv = h_neg_inv32((uint32_t)q);
        else devs[l].ar.qinv = h_neg_inv64(q);
    }
    if (cudaMemcpy(d_tables, host.data(), host.size() * sizeof(E), cudaMemcpyHostToDevice) != cudaSuccess) {
        *why = "cudaMemcpy failed";
        return 3;
    }
    LimbDev<A>* d_limbs = nullptr;
    if (cudaMalloc(&d_limbs, devs.size() * sizeof(LimbDev<A>)) != cudaSuccess) { *why = "cudaMalloc failed"; return 4; }
    p->allocations.push_back(d_limbs);
    if (cudaMemcpy(d_limbs, devs.data(), devs.size() * sizeof(LimbDev<A>), cudaMemcpyHostToDevice) != cudaSuccess) {
        *why = "cudaMemcpy failed";
        return 3;
    }
    p->d_limbs = d_limbs;
    return 0;
}

int build_plan32(Plan32* p, uint32_t log_n, const uint64_t* moduli, uint32_t n_limbs, bool negacyclic,
                 std::string* why) {
    return build_common<M32>(p, log_n, moduli, n_limbs, negacyclic, 1ull << 31,
                             [](uint64_t x, uint64_t q) { return h_to_mont32(x, q); }, why);
}

int build_plan64(Plan64* p, uint32_t log_n, const uint64_t* moduli, uint32_t n_limbs, bool negacyclic,
                 std::string* why) {
    return build_common<M64>(p, log_n, moduli, n_limbs, negacyclic, 1ull << 62,
                             [](uint64_t x, uint64_t q) { return h_to_mont64(x, q); }, why);
}

void* plan_workspace(void** ws, size_t* ws_bytes, size_t bytes) {
    if (*ws_bytes >= bytes) return *ws;
    if (*ws) cudaFree(*ws);
    *ws = nullptr;
    *ws_bytes = 0;
    if (cudaMalloc(ws, bytes) != cudaSuccess) {
        *ws = nullptr;
        return nullptr;
    }
    *ws_bytes = bytes;
    return *ws;
}

void free_plan32(Plan32* p) {
    if (p->ws) cudaFree(p->ws);
    p->ws = nullptr;
    p->ws_bytes = 0;
    for (void* a : p->allocations) cudaFree(a);
    p->allocations.clear();
    p->d_limbs = nullptr;
}

void free_plan64(Plan64* p) {
    if (p->ws) cudaFree(p->ws);
    p->ws = nullptr;
    p->ws_bytes = 0;
    for (void* a : p->allocations) cudaFree(a);
    p->allocations.clear();
    p->d_limbs = nullptr;
}

}  // namespace nttb
