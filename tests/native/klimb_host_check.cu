// Host-only checks of include/ntt_arbitrary.cuh (no GPU needed): reads
// "K log_n" then n input elements of K limbs (natural form) on stdin, and
// prints FieldConfig<K>'s prime, omega_n for that log_n, the result of
// host_ntt_naive, and whether Montgomery round trips hold for the inputs.
#include <cstdio>

#include "ntt_arbitrary.cuh"

template <int K>
static int run(int log_n) {
    using namespace ntt_arb;
    using FC = FieldConfig<K>;
    const int n = 1 << log_n;
    const BigInt<K> p = FC::prime();
    BigInt<K> w = FC::omega_2pow_max();
    for (int i = log_n; i < FC::MAX_LOG_N; i++) w = mod_mul<K>(w, w, p);
    std::vector<BigInt<K>> a(n), tw(n);
    for (int i = 0; i < n; i++)
        for (int k = 0; k < K; k++) {
            unsigned long long v;
            if (std::scanf("%llu", &v) != 1) return 2;
            a[i].limbs[k] = v;
        }
    const BigInt<K> R2 = mont_R2<K>(p);
    const uint32_t np = mont_np<K>(p);
    int mont_ok = 1;
    for (int i = 0; i < n; i++) {
        const BigInt<K> back = mont_mul_big<K>(mont_mul_big<K>(a[i], R2, p, np), BigInt<K>::one(), p, np);
        if (back.cmp(a[i]) != 0) mont_ok = 0;
        // Montgomery product against mod_mul: (a R)(b R) R^-1 = a b R
        const BigInt<K> b = a[(i + 1) % n];
        const BigInt<K> ab = mont_mul_big<K>(mont_mul_big<K>(mont_mul_big<K>(a[i], R2, p, np),
                                                              mont_mul_big<K>(b, R2, p, np), p, np),
                                             BigInt<K>::one(), p, np);
        if (ab.cmp(mod_mul<K>(a[i], b, p)) != 0) mont_ok = 0;
    }
    tw[0] = BigInt<K>::one();
    for (int i = 1; i < n; i++) tw[i] = mod_mul<K>(tw[i - 1], w, p);
    host_ntt_naive<K>(a, tw, p);
    std::printf("prime");
    for (int k = 0; k < K; k++) std::printf(" %llu", (unsigned long long)p.limbs[k]);
    std::printf("\nomega");
    for (int k = 0; k < K; k++) std::printf(" %llu", (unsigned long long)w.limbs[k]);
    std::printf("\nnp %u\nmont_ok %d\nout", np, mont_ok);
    for (int i = 0; i < n; i++)
        for (int k = 0; k < K; k++) std::printf(" %llu", (unsigned long long)a[i].limbs[k]);
    std::printf("\n");
    return 0;
}

int main() {
    int K = 0, log_n = 0;
    if (std::scanf("%d %d", &K, &log_n) != 2) return 2;
    switch (K) {
        case 2: return run<2>(log_n);
        case 3: return run<3>(log_n);
        case 11: return run<11>(log_n);
    }
    return 3;
}
