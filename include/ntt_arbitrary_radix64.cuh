/*
 * ntt_arbitrary_radix64.cuh -- drop-in for the reference's scalar radix-64
 * K-limb comparison path (include/ntt_arbitrary_radix64.cuh of
 * ntt-tensorcore): Radix64Buffers<K>, setup_radix64_tables,
 * teardown_radix64_tables and run_forward_radix64_scalar, same signatures.
 * The transform is the same forward network as run_forward_ct (natural order
 * in and out, Montgomery form), run by libntt_b200.so; the omega_8 / omega_64
 * tables are built as the reference builds them and accepted for
 * compatibility.
 */
#ifndef NTT_B200_NTT_ARBITRARY_RADIX64_CUH
#define NTT_B200_NTT_ARBITRARY_RADIX64_CUH

#include "ntt_arbitrary.cuh"

namespace ntt_arb {

template <int K>
struct Radix64Buffers {
    DScalar<K>* d_omega8 = nullptr;   // omega_8^k, k < 8 (Montgomery form)
    DScalar<K>* d_omega64 = nullptr;  // omega_64^k, k < 64 (Montgomery form)
};

template <int K>
static inline Radix64Buffers<K> setup_radix64_tables(const NTTBuffers<K>& B) {
    Radix64Buffers<K> R;
    if (B.n < 64) return R;
    BigInt<K> w64 = B.omega_n;
    for (int t = B.n; t > 64; t >>= 1) w64 = mod_mul<K>(w64, w64, B.prime);
    const BigInt<K> w8 = mod_pow<K>(w64, 8, B.prime);
    std::vector<BigInt<K>> o8(8), o64(64);
    o8[0] = o64[0] = BigInt<K>::one();
    for (int k = 1; k < 8; k++) o8[k] = mod_mul<K>(o8[k - 1], w8, B.prime);
    for (int k = 1; k < 64; k++) o64[k] = mod_mul<K>(o64[k - 1], w64, B.prime);
    R.d_omega8 = detail::alloc<K>(8);
    R.d_omega64 = detail::alloc<K>(64);
    detail::upload_mont<K>(R.d_omega8, o8, B.R2, B.prime, B.np);
    detail::upload_mont<K>(R.d_omega64, o64, B.R2, B.prime, B.np);
    return R;
}

template <int K>
static inline void teardown_radix64_tables(Radix64Buffers<K>& R) {
    if (R.d_omega8) cudaFree(R.d_omega8);
    if (R.d_omega64) cudaFree(R.d_omega64);
    R.d_omega8 = R.d_omega64 = nullptr;
}

template <int K>
static inline void run_forward_radix64_scalar(DScalar<K>* d_data, const DScalar<K>* d_tw, const DScalar<K>* d_omega8,
                                              const DScalar<K>* d_omega64, uint32_t n, int log_n, DScalar<K> prime_d,
                                              uint32_t np, cudaStream_t stream = 0) {
    (void)d_omega8;
    (void)d_omega64;
    detail::check(nttb_klimb_forward(K, reinterpret_cast<uint32_t*>(d_data), reinterpret_cast<const uint32_t*>(d_tw),
                                     n, (uint32_t)log_n, prime_d.limbs, np, stream),
                  "run_forward_radix64_scalar");
}

}  // namespace ntt_arb

#endif  // NTT_B200_NTT_ARBITRARY_RADIX64_CUH
