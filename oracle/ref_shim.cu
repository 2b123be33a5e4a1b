// ref_shim.cu -- extern "C" entry points onto the reference's own code.
//
// TEST INFRASTRUCTURE ONLY.  oracle/Makefile compiles this file together with
// the reference's unmodified src/ntt_basic.cu, src/ntt_four_step.cu and
// src/ntt_optimized.cu (read in place from the reference tree) into
// oracle/_ref/libntt_ref.so.  The shim adds nothing to the reference's
// arithmetic: it forwards to ntt::create_params, ntt::ntt_host and the
// reference's GPU entry points so that the tests can pin the oracle and the
// product against the reference itself, and so that bench.py can time the
// reference's CPU NTT on the host cores.
#include "ntt.cuh"
#include "ntt_arbitrary.cuh"

#include <algorithm>
#include <atomic>
#include <cstring>
#include <random>
#include <thread>
#include <vector>

extern "C" {

// create_params (include/modular_arith.cuh:153-170) + mu (src/ntt_basic.cu:226-229).
// out = {q, q_twice, barrett_k, barrett_m, omega, omega_inv, n_inv, mu}
void ref_create_params(uint64_t q, uint64_t n, uint64_t* out) {
    ntt::ModularParams p = ntt::create_params(q, n);
    out[0] = p.q; out[1] = p.q_twice; out[2] = p.barrett_k; out[3] = p.barrett_m;
    out[4] = p.omega; out[5] = p.omega_inv; out[6] = p.n_inv;
    out[7] = (uint64_t)(((unsigned __int128)1 << 64) / q);
}

// ntt::ntt_host on one polynomial (src/ntt_basic.cu:412-463).
void ref_ntt_host(uint64_t* data, uint64_t n, uint64_t q, int inverse) {
    ntt::ModularParams p = ntt::create_params(q, n);
    std::vector<uint64_t> v(data, data + n);
    ntt::ntt_host(v, p, inverse != 0);
    std::memcpy(data, v.data(), n * sizeof(uint64_t));
}

// ntt::ntt_host over a batch laid out [poly][limb][n], limb l using moduli[l],
// one (poly, limb) per task on `threads` host threads.  With negacyclic != 0
// the driver wraps ntt_host in the psi twist (x_j * psi^j before the forward,
// n^-1 psi^-j after the inverse; psi = g^((q-1)/2n) with g found the way
// find_primitive_root finds it) -- the reference has no negacyclic code, so
// the twist is driver code and the transform is the reference's.
// Returns the number of threads used.
int ref_ntt_host_batch(uint64_t* data, uint64_t n, const uint64_t* moduli, uint64_t n_limbs,
                       uint64_t n_polys, int inverse, int negacyclic, int threads) {
    if (threads <= 0) threads = (int)std::max(1u, std::thread::hardware_concurrency());
    uint64_t tasks = n_limbs * n_polys;
    std::vector<ntt::ModularParams> params(n_limbs);
    std::vector<uint64_t> psi(n_limbs), psi_inv(n_limbs);
    for (uint64_t l = 0; l < n_limbs; l++) {
        params[l] = ntt::create_params(moduli[l], n);
        if (negacyclic) {
            uint64_t q = moduli[l];
            // generator exactly as find_primitive_root searches it
            uint64_t g = 2;
            for (;; g++) {
                bool ok = true;
                for (uint64_t pr : {2ULL, 3ULL, 5ULL, 7ULL})
                    if ((q - 1) % pr == 0 && ntt::mod_pow(g, (q - 1) / pr, q) == 1) { ok = false; break; }
                if (ok) break;
            }
            psi[l] = ntt::mod_pow(g, (q - 1) / (2 * n), q);
            psi_inv[l] = ntt::mod_inverse(psi[l], q);
        }
    }
    std::atomic<uint64_t> next{0};
    auto worker = [&]() {
        std::vector<uint64_t> v(n);
        for (;;) {
            uint64_t t = next.fetch_add(1);
            if (t >= tasks) break;
            uint64_t l = t % n_limbs;
            uint64_t q = moduli[l];
            uint64_t* d = data + t * n;
            std::memcpy(v.data(), d, n * sizeof(uint64_t));
            if (negacyclic && !inverse) {
                uint64_t w = 1;
                for (uint64_t j = 0; j < n; j++) {
                    v[j] = (unsigned __int128)v[j] * w % q;
                    w = (unsigned __int128)w * psi[l] % q;
                }
            }
            ntt::ntt_host(v, params[l], inverse != 0);
            if (negacyclic && inverse) {
                uint64_t w = 1;
                for (uint64_t j = 0; j < n; j++) {
                    v[j] = (unsigned __int128)v[j] * w % q;
                    w = (unsigned __int128)w * psi_inv[l] % q;
                }
            }
            std::memcpy(d, v.data(), n * sizeof(uint64_t));
        }
    };
    std::vector<std::thread> pool;
    for (int i = 0; i < threads; i++) pool.emplace_back(worker);
    for (auto& th : pool) th.join();
    return threads;
}

// The reference tests' input generator (tests/test_ntt.cu:22-31):
// mt19937_64(seed) + uniform_int_distribution<uint64_t>(0, q-1).
void ref_random_polynomial(uint64_t* out, uint64_t n, uint64_t q, uint32_t seed) {
    std::mt19937_64 rng(seed);
    std::uniform_int_distribution<uint64_t> dist(0, q - 1);
    for (uint64_t i = 0; i < n; i++) out[i] = dist(rng);
}

// ---- reference GPU entry points (device pointers; run on a GPU box only) ----
void* ref_ntt_init(uint64_t n, uint64_t q) { return ntt::ntt_init(n, q); }
void ref_ntt_cleanup(void* cfg) { ntt::ntt_cleanup((ntt::NTTConfig*)cfg); }

// op: 0 fwd basic, 1 inv basic, 2 fwd four_step, 3 inv four_step,
//     4 fwd optimized, 5 inv optimized, 6 fwd rowmaj
void ref_ntt_run(void* cfg, uint64_t* d_data, int op) {
    auto* c = (ntt::NTTConfig*)cfg;
    switch (op) {
        case 0: ntt::ntt_forward_basic(d_data, c); break;
        case 1: ntt::ntt_inverse_basic(d_data, c); break;
        case 2: ntt::ntt_forward_four_step(d_data, c); break;
        case 3: ntt::ntt_inverse_four_step(d_data, c); break;
        case 4: ntt::ntt_forward_optimized(d_data, c); break;
        case 5: ntt::ntt_inverse_optimized(d_data, c); break;
        case 6: ntt::ntt_forward_rowmaj(d_data, c); break;
        default: break;
    }
    cudaDeviceSynchronize();
}

// The reference's optimized transforms (src/ntt_optimized.cu:515-557 forward,
// :559-600 inverse) over a batch laid out [poly][limb][n], limb l with
// cfgs[l] (one ntt_init per modulus), queued on `stream` with no
// synchronisation: ntt_forward_batch's per-polynomial loop
// (src/ntt_basic.cu:337-361) taken limb by limb, since every limb has its own
// modulus.  which: 0 forward, 1 inverse, 2 forward then inverse.
void ref_ntt_rns_optimized(void* const* cfgs, uint64_t n_limbs, uint64_t n_polys, uint64_t* d_data, int which,
                           void* stream) {
    auto s = (cudaStream_t)stream;
    for (int pass = 0; pass < 2; pass++) {
        if ((which == 0 && pass == 1) || (which == 1 && pass == 0)) continue;
        for (uint64_t p = 0; p < n_polys; p++)
            for (uint64_t l = 0; l < n_limbs; l++) {
                auto* c = (const ntt::NTTConfig*)cfgs[l];
                uint64_t* d = d_data + (p * n_limbs + l) * c->n;
                if (pass == 0) ntt::ntt_forward_optimized(d, c, s);
                else ntt::ntt_inverse_optimized(d, c, s);
            }
    }
}

}  // extern "C"

// ---- K-limb reference host code (include/ntt_arbitrary.cuh) ----
// Fills, for FieldConfig<K> and N = 2^log_n, the reference's natural-form
// input (setup_ntt's mt19937_64(seed) limbs reduced by mod_slow,
// :2698-2730) and the host_ntt_naive output (:2651-2676).  Each element is
// K uint32 limbs of 24 bits (little-endian), natural form.
template <int K>
static void klimb_case(int log_n, uint64_t seed, uint32_t* in, uint32_t* out,
                       uint32_t* prime, uint32_t* omega_n) {
    using namespace ntt_arb;
    using FC = FieldConfig<K>;
    int n = 1 << log_n;
    BigInt<K> p = FC::prime();
    BigInt<K> w = FC::omega_2pow_max();
    for (int i = 0; i < FC::MAX_LOG_N - log_n; i++) w = mod_mul<K>(w, w, p);
    std::vector<BigInt<K>> tw(n);
    tw[0] = BigInt<K>::one();
    for (int i = 1; i < n; i++) tw[i] = mod_mul<K>(tw[i - 1], w, p);
    std::mt19937_64 rng(seed);
    std::vector<BigInt<K>> data(n);
    for (int i = 0; i < n; i++) {
        BigInt<K> r;
        for (int j = 0; j < K; j++) r.limbs[j] = rng() & LIMB_MASK;
        data[i] = mod_slow<K, K>(r, p);
    }
    for (int i = 0; i < n; i++)
        for (int j = 0; j < K; j++) in[i * K + j] = (uint32_t)data[i].limbs[j];
    host_ntt_naive<K>(data, tw, p);
    for (int i = 0; i < n; i++)
        for (int j = 0; j < K; j++) out[i * K + j] = (uint32_t)data[i].limbs[j];
    for (int j = 0; j < K; j++) { prime[j] = (uint32_t)p.limbs[j]; omega_n[j] = (uint32_t)w.limbs[j]; }
}

extern "C" int ref_klimb_case(int K, int log_n, uint64_t seed, uint32_t* in, uint32_t* out,
                   uint32_t* prime, uint32_t* omega_n) {
    switch (K) {
        case 2: klimb_case<2>(log_n, seed, in, out, prime, omega_n); return 0;
        case 3: klimb_case<3>(log_n, seed, in, out, prime, omega_n); return 0;
        case 11: klimb_case<11>(log_n, seed, in, out, prime, omega_n); return 0;
        default: return 1;
    }
}

// mont_mul_big / mont_R2 / mont_np known answers (src/ntt_mma_arbitrary.cu:19-99):
// returns a*b*R^-1 mod p for FieldConfig<K>, all values as 24-bit limbs.
template <int K>
static void klimb_mont(const uint32_t* a, const uint32_t* b, uint32_t* out, uint32_t* r2, uint32_t* np) {
    using namespace ntt_arb;
    BigInt<K> p = FieldConfig<K>::prime();
    BigInt<K> x, y;
    for (int j = 0; j < K; j++) { x.limbs[j] = a[j]; y.limbs[j] = b[j]; }
    uint32_t n_p = mont_np<K>(p);
    BigInt<K> R2 = mont_R2<K>(p);
    BigInt<K> z = mont_mul_big<K>(x, y, p, n_p);
    for (int j = 0; j < K; j++) { out[j] = (uint32_t)z.limbs[j]; r2[j] = (uint32_t)R2.limbs[j]; }
    *np = n_p;
}

extern "C" int ref_klimb_mont(int K, const uint32_t* a, const uint32_t* b, uint32_t* out, uint32_t* r2, uint32_t* np) {
    switch (K) {
        case 2: klimb_mont<2>(a, b, out, r2, np); return 0;
        case 3: klimb_mont<3>(a, b, out, r2, np); return 0;
        case 11: klimb_mont<11>(a, b, out, r2, np); return 0;
        default: return 1;
    }
}

