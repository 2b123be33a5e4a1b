/*
 * ntt_arbitrary.cuh -- drop-in for the reference's header-only K-limb NTT
 * API (namespace ntt_arb, include/ntt_arbitrary.cuh of ntt-tensorcore).
 *
 * Same names, template parameters, field layouts and data formats:
 *   - BigInt<K>: K little-endian limbs of LIMB_BITS = 24 bits in uint64 words;
 *   - DScalar<K>: the device form, K uint32 words holding 24-bit limbs, in
 *     Montgomery form with R = 2^(24 K) when it lives in NTTBuffers;
 *   - FieldConfig<K> for K in {2, 3, 11}: the reference's moduli and roots;
 *   - NTTBuffers<K> / setup_ntt / teardown_ntt / run_forward_ct /
 *     run_forward_ct_tcu / host_ntt_naive / run_for_K, plus the per-stage
 *     kernels bitrev_kernel_d / ct_stage_kernel that callers launch directly.
 * The host helpers are plain big-integer code; the forward transforms run in
 * libntt_b200.so (nttb_klimb_forward, shared-memory multi-stage passes).
 * Errors: like the reference's drivers, a failed call prints a message and
 * exits.
 */
#ifndef NTT_B200_NTT_ARBITRARY_CUH
#define NTT_B200_NTT_ARBITRARY_CUH

#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <iomanip>
#include <iostream>
#include <random>
#include <string>
#include <vector>

#include "ntt_b200.h"
#include "ntt_limb_arith.cuh"

namespace ntt_arb {

constexpr int LIMB_BITS = 24;
constexpr uint64_t LIMB_BASE = 1ULL << LIMB_BITS;
constexpr uint64_t LIMB_MASK = LIMB_BASE - 1;
constexpr int TCU_LOG_INNER = 6;  // radix-64 inner size of the reference's tensor-core path
constexpr int TCU_INNER_SIZE = 1 << TCU_LOG_INNER;

// ------------------------------------------------------------- BigInt<K>
template <int K>
struct BigInt {
    uint64_t limbs[K];

    __host__ __device__ BigInt() {
        for (int i = 0; i < K; i++) limbs[i] = 0;
    }
    __host__ __device__ static BigInt zero() { return BigInt(); }
    __host__ __device__ static BigInt one() {
        BigInt r;
        r.limbs[0] = 1;
        return r;
    }
    // Low 24 K bits of v (higher bits are dropped).
    __host__ __device__ static BigInt from_u64(uint64_t v) {
        BigInt r;
        for (int i = 0; i < K; i++) {
            r.limbs[i] = v & LIMB_MASK;
            v >>= LIMB_BITS;
        }
        return r;
    }
    __host__ __device__ bool is_zero() const {
        for (int i = 0; i < K; i++)
            if (limbs[i]) return false;
        return true;
    }
    __host__ __device__ int cmp(const BigInt& o) const {
        for (int i = K - 1; i >= 0; i--) {
            if (limbs[i] != o.limbs[i]) return limbs[i] < o.limbs[i] ? -1 : 1;
        }
        return 0;
    }
};

// Hex literal (MSB first, optional 0x) -> BigInt<K>; bits beyond 24 K are dropped.
template <int K>
static inline BigInt<K> from_hex(const char* hex) {
    BigInt<K> r;
    if (hex[0] == '0' && (hex[1] == 'x' || hex[1] == 'X')) hex += 2;
    const int len = (int)std::strlen(hex);
    for (int d = 0; d < len; d++) {  // d-th digit from the right
        const char ch = hex[len - 1 - d];
        const int v = (ch >= '0' && ch <= '9') ? ch - '0'
                      : (ch >= 'a' && ch <= 'f') ? ch - 'a' + 10
                      : (ch >= 'A' && ch <= 'F') ? ch - 'A' + 10
                                                 : 0;
        for (int b = 0; b < 4; b++) {
            const int bit = 4 * d + b;
            if (((v >> b) & 1) && bit / LIMB_BITS < K) r.limbs[bit / LIMB_BITS] |= 1ULL << (bit % LIMB_BITS);
        }
    }
    return r;
}

// r = a + b; returns the carry out of the top limb.
template <int K>
__host__ __device__ inline uint64_t big_add(BigInt<K>& r, const BigInt<K>& a, const BigInt<K>& b) {
    uint64_t c = 0;
    for (int i = 0; i < K; i++) {
        const uint64_t s = a.limbs[i] + b.limbs[i] + c;
        r.limbs[i] = s & LIMB_MASK;
        c = s >> LIMB_BITS;
    }
    return c;
}
// r = a - b; returns the borrow out of the top limb.
template <int K>
__host__ __device__ inline uint64_t big_sub(BigInt<K>& r, const BigInt<K>& a, const BigInt<K>& b) {
    uint64_t borrow = 0;
    for (int i = 0; i < K; i++) {
        const uint64_t s = a.limbs[i] + LIMB_BASE - b.limbs[i] - borrow;
        r.limbs[i] = s & LIMB_MASK;
        borrow = 1 - (s >> LIMB_BITS);
    }
    return borrow;
}
// r = a * b (full 2K-limb product).
template <int K>
__host__ __device__ inline void big_mul(BigInt<2 * K>& r, const BigInt<K>& a, const BigInt<K>& b) {
    uint64_t col[2 * K];
    for (int i = 0; i < 2 * K; i++) col[i] = 0;
    uint64_t carry = 0;
    for (int c = 0; c < 2 * K; c++) {
        uint64_t acc = carry, hi = 0;
        for (int i = 0; i < K; i++) {
            const int j = c - i;
            if (j < 0 || j >= K) continue;
            acc += a.limbs[i] * b.limbs[j];  // each product < 2^48
            hi += acc >> LIMB_BITS;
            acc &= LIMB_MASK;
        }
        col[c] = acc;
        carry = hi;
    }
    for (int i = 0; i < 2 * K; i++) r.limbs[i] = col[i];
}

template <int K>
static inline BigInt<K> mod_reduce_once(const BigInt<K>& a, const BigInt<K>& p) {
    if (a.cmp(p) < 0) return a;
    BigInt<K> r;
    big_sub<K>(r, a, p);
    return r;
}
template <int K>
static inline BigInt<K> mod_add(const BigInt<K>& a, const BigInt<K>& b, const BigInt<K>& p) {
    BigInt<K> s;
    const uint64_t c = big_add<K>(s, a, b);
    if (c || s.cmp(p) >= 0) big_sub<K>(s, s, p);
    return s;
}
template <int K>
static inline BigInt<K> mod_sub(const BigInt<K>& a, const BigInt<K>& b, const BigInt<K>& p) {
    BigInt<K> d;
    if (big_sub<K>(d, a, b)) big_add<K>(d, d, p);
    return d;
}
// a (K_IN limbs) mod p (K_OUT limbs), bit by bit: r <- 2 r + bit, minus p when r >= p.
template <int K_OUT, int K_IN>
static inline BigInt<K_OUT> mod_slow(const BigInt<K_IN>& a, const BigInt<K_OUT>& p) {
    BigInt<K_OUT + 1> r, pp;
    for (int i = 0; i < K_OUT; i++) pp.limbs[i] = p.limbs[i];
    for (int bit = K_IN * LIMB_BITS - 1; bit >= 0; bit--) {
        big_add<K_OUT + 1>(r, r, r);
        r.limbs[0] |= (a.limbs[bit / LIMB_BITS] >> (bit % LIMB_BITS)) & 1;
        if (r.cmp(pp) >= 0) big_sub<K_OUT + 1>(r, r, pp);
    }
    BigInt<K_OUT> out;
    for (int i = 0; i < K_OUT; i++) out.limbs[i] = r.limbs[i];
    return out;
}
template <int K>
static inline BigInt<K> mod_mul(const BigInt<K>& a, const BigInt<K>& b, const BigInt<K>& p) {
    BigInt<2 * K> w;
    big_mul<K>(w, a, b);
    return mod_slow<K, 2 * K>(w, p);
}
template <int K>
static inline BigInt<K> mod_pow(const BigInt<K>& base, uint64_t exp, const BigInt<K>& p) {
    BigInt<K> r = mod_slow<K, 1>(BigInt<1>::one(), p), b = base;
    for (; exp; exp >>= 1) {
        if (exp & 1) r = mod_mul<K>(r, b, p);
        b = mod_mul<K>(b, b, p);
    }
    return r;
}
template <int K>
static inline BigInt<K> mod_pow_big(const BigInt<K>& base, const BigInt<K>& exp, const BigInt<K>& p) {
    BigInt<K> r = mod_slow<K, 1>(BigInt<1>::one(), p);
    for (int bit = K * LIMB_BITS - 1; bit >= 0; bit--) {
        r = mod_mul<K>(r, r, p);
        if ((exp.limbs[bit / LIMB_BITS] >> (bit % LIMB_BITS)) & 1) r = mod_mul<K>(r, base, p);
    }
    return r;
}
// a^-1 mod p for prime p (Fermat: a^(p-2)).
template <int K>
static inline BigInt<K> mod_inv(const BigInt<K>& a, const BigInt<K>& p) {
    BigInt<K> e;
    big_sub<K>(e, p, BigInt<K>::from_u64(2));
    return mod_pow_big<K>(a, e, p);
}
// -p^-1 mod 2^24.
template <int K>
static inline uint32_t mont_np(const BigInt<K>& p) {
    return nttb_limb::neg_inv24((uint32_t)p.limbs[0]);
}
// R^2 mod p, R = 2^(24 K).
template <int K>
static inline BigInt<K> mont_R2(const BigInt<K>& p) {
    BigInt<2 * K + 1> t;
    t.limbs[2 * K] = 1;  // 2^(48 K)
    return mod_slow<K, 2 * K + 1>(t, p);
}
// a b R^-1 mod p for a, b in [0, p).
template <int K>
static inline BigInt<K> mont_mul_big(const BigInt<K>& a, const BigInt<K>& b, const BigInt<K>& p, uint32_t np) {
    uint32_t aa[K], bb[K], pp[K], rr[K];
    for (int i = 0; i < K; i++) {
        aa[i] = (uint32_t)a.limbs[i];
        bb[i] = (uint32_t)b.limbs[i];
        pp[i] = (uint32_t)p.limbs[i];
    }
    nttb_limb::mont_mul<K>(rr, aa, bb, pp, np);
    BigInt<K> r;
    for (int i = 0; i < K; i++) r.limbs[i] = rr[i];
    return r;
}

// -------------------------------------------------------------- fields
// Modulus and a primitive 2^MAX_LOG_N-th root for each supported K.  The
// limbs are filled exactly as the reference does (from_u64 semantics), so
// its K = 2 modulus keeps only the low 48 bits of 281476520214529.
template <int K_>
struct FieldConfig;

template <>
struct FieldConfig<2> {
    static constexpr int K = 2;
    static constexpr int MAX_LOG_N = 12;
    static BigInt<2> prime() { return BigInt<2>::from_u64(281476520214529ULL); }
    static BigInt<2> omega_2pow_max() { return BigInt<2>::from_u64(30523202938030ULL); }
};

// Goldilocks p = 2^64 - 2^32 + 1.
template <>
struct FieldConfig<3> {
    static constexpr int K = 3;
    static constexpr int MAX_LOG_N = 24;
    static BigInt<3> prime() { return BigInt<3>::from_u64(0xFFFFFFFF00000001ULL); }
    static BigInt<3> omega_2pow_max() { return BigInt<3>::from_u64(0x86cdcc31c307e171ULL); }
};

// BN254 scalar field; its 2-adic root of order 2^28 squared down to 2^24.
template <>
struct FieldConfig<11> {
    static constexpr int K = 11;
    static constexpr int MAX_LOG_N = 24;
    static BigInt<11> prime() {
        return from_hex<11>("30644E72E131A029B85045B68181585D2833E84879B9709143E1F593F0000001");
    }
    static BigInt<11> omega_2pow_max() {
        const BigInt<11> p = prime();
        BigInt<11> w = from_hex<11>("2a3c09f0a58a7e8500e0a7eb8ef62abc402d111e41112ed49bd61b6e725b19f0");
        for (int i = 0; i < 28 - MAX_LOG_N; i++) w = mod_mul<11>(w, w, p);
        return w;
    }
};

// ---------------------------------------------------------- DScalar<K>
template <int K>
struct DScalar {
    uint32_t limbs[K];
};

template <int K>
__host__ __device__ inline DScalar<K> load_scalar(const BigInt<K>& x) {
    DScalar<K> r;
    for (int i = 0; i < K; i++) r.limbs[i] = (uint32_t)x.limbs[i];
    return r;
}
template <int K>
__host__ __device__ inline BigInt<K> store_scalar(const DScalar<K>& x) {
    BigInt<K> r;
    for (int i = 0; i < K; i++) r.limbs[i] = x.limbs[i];
    return r;
}
template <int K>
__host__ __device__ inline DScalar<K> mod_add_d(const DScalar<K>& a, const DScalar<K>& b, const DScalar<K>& p) {
    DScalar<K> r;
    nttb_limb::add_mod<K>(r.limbs, a.limbs, b.limbs, p.limbs);
    return r;
}
template <int K>
__host__ __device__ inline DScalar<K> mod_sub_d(const DScalar<K>& a, const DScalar<K>& b, const DScalar<K>& p) {
    DScalar<K> r;
    nttb_limb::sub_mod<K>(r.limbs, a.limbs, b.limbs, p.limbs);
    return r;
}
// a b R^-1 mod p (Montgomery product), host or device.
template <int K>
__host__ __device__ inline DScalar<K> mont_mul(const DScalar<K>& a, const DScalar<K>& b, const DScalar<K>& p,
                                               uint32_t np) {
    DScalar<K> r;
    nttb_limb::mont_mul<K>(r.limbs, a.limbs, b.limbs, p.limbs, np);
    return r;
}

// ------------------------------------------------------ per-stage kernels
// In-place bit reversal of n = 2^log_n elements (one thread per element).
template <int K>
__global__ void bitrev_kernel_d(DScalar<K>* data, uint32_t n, int log_n) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || log_n == 0) return;
    const uint32_t j = __brev(i) >> (32 - log_n);
    if (i < j) {
        const DScalar<K> t = data[i];
        data[i] = data[j];
        data[j] = t;
    }
}
// One radix-2 DIT stage `st` (one thread per butterfly, n / 2 threads).
template <int K>
__global__ void ct_stage_kernel(DScalar<K>* data, const DScalar<K>* tw, uint32_t n, int st, DScalar<K> prime,
                                uint32_t np) {
    const uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= n / 2) return;
    const uint32_t half = 1u << st;
    const uint32_t k = b & (half - 1), i = ((b >> st) << (st + 1)) + k;
    const DScalar<K> t = mont_mul<K>(data[i + half], tw[(size_t)k * (n >> (st + 1))], prime, np);
    const DScalar<K> u = data[i];
    data[i] = mod_add_d<K>(u, t, prime);
    data[i + half] = mod_sub_d<K>(u, t, prime);
}

// ------------------------------------------------------- forward drivers
namespace detail {
inline void check(int rc, const char* what) {
    if (rc != NTTB_OK) {
        std::cerr << what << " failed: " << nttb_last_error() << std::endl;
        std::exit(EXIT_FAILURE);
    }
}
}  // namespace detail

// Forward NTT of n = 2^log_n Montgomery-form elements in place, natural
// order in and out (the network of host_ntt_naive).
template <int K>
static inline void run_forward_ct(DScalar<K>* d_data, const DScalar<K>* d_tw, uint32_t n, int log_n, DScalar<K> prime_d,
                                  uint32_t np, cudaStream_t stream = 0) {
    detail::check(nttb_klimb_forward(K, reinterpret_cast<uint32_t*>(d_data), reinterpret_cast<const uint32_t*>(d_tw),
                                     n, (uint32_t)log_n, prime_d.limbs, np, stream),
                  "run_forward_ct");
}
// Same transform; the reference's tensor-core variant.  The radix-8 and
// inner twiddle tables are accepted for signature compatibility.
template <int K>
static inline void run_forward_ct_tcu(DScalar<K>* d_data, const DScalar<K>* d_tw, const DScalar<K>* d_tfm8,
                                      const DScalar<K>* d_hada64, uint32_t n, int log_n, DScalar<K> prime_d,
                                      uint32_t np, cudaStream_t stream = 0) {
    (void)d_tfm8;
    (void)d_hada64;
    detail::check(nttb_klimb_forward(K, reinterpret_cast<uint32_t*>(d_data), reinterpret_cast<const uint32_t*>(d_tw),
                                     n, (uint32_t)log_n, prime_d.limbs, np, stream),
                  "run_forward_ct_tcu");
}

// CPU reference (natural form): bit reversal, then radix-2 DIT stages with
// twiddle tw[k n / 2^(s+1)].
template <int K>
static inline void host_ntt_naive(std::vector<BigInt<K>>& a, const std::vector<BigInt<K>>& tw, const BigInt<K>& p) {
    const int n = (int)a.size();
    int log_n = 0;
    while ((1 << log_n) < n) log_n++;
    for (int i = 0; i < n; i++) {
        int j = 0;
        for (int b = 0; b < log_n; b++) j |= ((i >> b) & 1) << (log_n - 1 - b);
        if (i < j) std::swap(a[i], a[j]);
    }
    for (int s = 0; s < log_n; s++) {
        const int half = 1 << s, step = n >> (s + 1);
        for (int g = 0; g < n; g += 2 * half) {
            for (int k = 0; k < half; k++) {
                const BigInt<K> t = mod_mul<K>(a[g + k + half], tw[(size_t)k * step], p);
                const BigInt<K> u = a[g + k];
                a[g + k] = mod_add<K>(u, t, p);
                a[g + k + half] = mod_sub<K>(u, t, p);
            }
        }
    }
}

// ------------------------------------------------------- setup / teardown
template <int K>
struct NTTBuffers {
    int n = 0;
    int log_n = 0;
    BigInt<K> prime{};
    BigInt<K> R2{};        // R^2 mod p
    uint32_t np = 0;       // -p^-1 mod 2^24
    BigInt<K> omega_n{};
    std::vector<BigInt<K>> tw_host;    // omega_n^i, natural form
    std::vector<BigInt<K>> data_host;  // input, natural form
    DScalar<K>* d_data = nullptr;      // working buffer, Montgomery form
    DScalar<K>* d_tw = nullptr;        // omega_n^i, Montgomery form
    DScalar<K>* d_tfm8 = nullptr;      // omega_8^(i k), i, k < 8, Montgomery form
    DScalar<K>* d_hada64 = nullptr;    // omega_64^k, k < 64, Montgomery form
    DScalar<K> prime_d{};
};

namespace detail {
template <int K>
inline void upload_mont(DScalar<K>* dst, const std::vector<BigInt<K>>& src, const BigInt<K>& R2, const BigInt<K>& p,
                        uint32_t np) {
    std::vector<DScalar<K>> h(src.size());
    for (size_t i = 0; i < src.size(); i++) h[i] = load_scalar<K>(mont_mul_big<K>(src[i], R2, p, np));
    if (cudaMemcpy(dst, h.data(), h.size() * sizeof(DScalar<K>), cudaMemcpyHostToDevice) != cudaSuccess) {
        std::cerr << "ntt_arb: upload failed" << std::endl;
        std::exit(EXIT_FAILURE);
    }
}
template <int K>
inline DScalar<K>* alloc(size_t count) {
    DScalar<K>* d = nullptr;
    if (cudaMalloc(&d, count * sizeof(DScalar<K>)) != cudaSuccess) {
        std::cerr << "ntt_arb: cudaMalloc failed" << std::endl;
        std::exit(EXIT_FAILURE);
    }
    return d;
}
}  // namespace detail

// Twiddles omega_n^i and a seeded input (mt19937_64: K draws of 24 bits per
// element, reduced mod p), uploaded in Montgomery form; for n >= 64 also the
// radix-8 matrix and the 64 inner twiddles.
template <int K>
static inline NTTBuffers<K> setup_ntt(int log_n, uint64_t seed = 0xC0FFEE) {
    using FC = FieldConfig<K>;
    NTTBuffers<K> B;
    B.log_n = log_n;
    B.n = 1 << log_n;
    B.prime = FC::prime();
    B.np = mont_np<K>(B.prime);
    B.R2 = mont_R2<K>(B.prime);
    B.omega_n = FC::omega_2pow_max();
    for (int i = log_n; i < FC::MAX_LOG_N; i++) B.omega_n = mod_mul<K>(B.omega_n, B.omega_n, B.prime);
    B.tw_host.resize(B.n);
    B.tw_host[0] = BigInt<K>::one();
    for (int i = 1; i < B.n; i++) B.tw_host[i] = mod_mul<K>(B.tw_host[i - 1], B.omega_n, B.prime);
    std::mt19937_64 rng(seed);
    B.data_host.resize(B.n);
    for (int i = 0; i < B.n; i++) {
        BigInt<K> r;
        for (int j = 0; j < K; j++) r.limbs[j] = rng() & LIMB_MASK;
        B.data_host[i] = mod_slow<K, K>(r, B.prime);
    }
    B.d_data = detail::alloc<K>(B.n);
    B.d_tw = detail::alloc<K>(B.n);
    detail::upload_mont<K>(B.d_data, B.data_host, B.R2, B.prime, B.np);
    detail::upload_mont<K>(B.d_tw, B.tw_host, B.R2, B.prime, B.np);
    B.prime_d = load_scalar<K>(B.prime);
    if (B.n >= 64) {
        BigInt<K> w64 = B.omega_n;
        for (int t = B.n; t > 64; t >>= 1) w64 = mod_mul<K>(w64, w64, B.prime);
        const BigInt<K> w8 = mod_pow<K>(w64, 8, B.prime);
        std::vector<BigInt<K>> tfm(64), hada(64);
        for (int i = 0; i < 8; i++)
            for (int k = 0; k < 8; k++) tfm[i * 8 + k] = mod_pow<K>(w8, (uint64_t)(i * k), B.prime);
        hada[0] = BigInt<K>::one();
        for (int k = 1; k < 64; k++) hada[k] = mod_mul<K>(hada[k - 1], w64, B.prime);
        B.d_tfm8 = detail::alloc<K>(64);
        B.d_hada64 = detail::alloc<K>(64);
        detail::upload_mont<K>(B.d_tfm8, tfm, B.R2, B.prime, B.np);
        detail::upload_mont<K>(B.d_hada64, hada, B.R2, B.prime, B.np);
    }
    return B;
}

template <int K>
static inline void teardown_ntt(NTTBuffers<K>& B) {
    if (B.d_data) cudaFree(B.d_data);
    if (B.d_tw) cudaFree(B.d_tw);
    if (B.d_tfm8) cudaFree(B.d_tfm8);
    if (B.d_hada64) cudaFree(B.d_hada64);
    B.d_data = B.d_tw = B.d_tfm8 = B.d_hada64 = nullptr;
}

// ------------------------------------------------------------------ driver
// Times the forward transform and checks it against host_ntt_naive; returns
// 0 when every position matches (or the check is skipped).
template <int K>
static inline int run_for_K(int log_n, bool do_host_check = true) {
    using FC = FieldConfig<K>;
    if (log_n > FC::MAX_LOG_N) {
        std::cerr << "log_n=" << log_n << " exceeds MAX_LOG_N=" << FC::MAX_LOG_N << " for K=" << K << "\n";
        return 1;
    }
    NTTBuffers<K> B = setup_ntt<K>(log_n);
    std::cout << "------------------------------------------------------------\n"
              << "K=" << K << " (LIMB_BITS=" << LIMB_BITS << "), N=2^" << log_n << "=" << B.n << "\np = 0x";
    {
        bool lead = true;
        for (int i = K - 1; i >= 0; i--) {
            if (lead && B.prime.limbs[i] == 0 && i > 0) continue;
            std::cout << std::hex << std::setfill('0') << std::setw(lead ? 1 : 6) << B.prime.limbs[i];
            lead = false;
        }
        std::cout << std::dec << std::setfill(' ') << "\n";
    }
    auto run = [&]() {
        run_forward_ct_tcu<K>(B.d_data, B.d_tw, B.d_tfm8, B.d_hada64, B.n, log_n, B.prime_d, B.np);
    };
    for (int it = 0; it < 3; it++) run();
    cudaDeviceSynchronize();
    detail::upload_mont<K>(B.d_data, B.data_host, B.R2, B.prime, B.np);
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    const int iters = 20;
    cudaEventRecord(e0);
    for (int it = 0; it < iters; it++) run();
    cudaEventRecord(e1);
    cudaEventSynchronize(e1);
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    std::cout << "  NTT: " << (ms * 1000.0 / iters) << " us/iter\n";
    int mismatches = 0;
    if (do_host_check) {
        detail::upload_mont<K>(B.d_data, B.data_host, B.R2, B.prime, B.np);
        run();
        cudaDeviceSynchronize();
        std::vector<DScalar<K>> got(B.n);
        cudaMemcpy(got.data(), B.d_data, (size_t)B.n * sizeof(DScalar<K>), cudaMemcpyDeviceToHost);
        std::vector<BigInt<K>> ref = B.data_host;
        host_ntt_naive<K>(ref, B.tw_host, B.prime);
        const BigInt<K> one = BigInt<K>::one();
        for (int i = 0; i < B.n; i++) {
            const BigInt<K> v = mont_mul_big<K>(store_scalar<K>(got[i]), one, B.prime, B.np);
            if (v.cmp(ref[i]) != 0) {
                if (mismatches < 5) std::cout << "  MISMATCH @ i=" << i << "\n";
                mismatches++;
            }
        }
        if (mismatches == 0)
            std::cout << "  CORRECT (matches host reference at all " << B.n << " positions)\n";
        else
            std::cout << "  FAILED (" << mismatches << " mismatches)\n";
    } else {
        std::cout << "  (host-check skipped)\n";
    }
    teardown_ntt<K>(B);
    return mismatches ? 1 : 0;
}

}  // namespace ntt_arb

#endif  // NTT_B200_NTT_ARBITRARY_CUH
