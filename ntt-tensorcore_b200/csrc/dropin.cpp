// dropin.cpp -- the reference's C++ API (include/ntt.cuh) on top of the C ABI.
//
// Each function forwards to one nttb_* entry point; on failure it prints the
// reason and exits with EXIT_FAILURE, as the reference's CUDA_CHECK does
// (src/ntt_basic.cu:13-21).
#pragma GCC visibility push(default)
#include "../../include/ntt.cuh"
#pragma GCC visibility pop

#include <cstdio>
#include <cstdlib>

#include "../../include/ntt_b200.h"

namespace {

void check(int status, const char* what) {
    if (status != NTTB_OK) {
        std::fprintf(stderr, "ntt_b200 error in %s: %s (%s)\n", what, nttb_status_string(status), nttb_last_error());
        std::exit(EXIT_FAILURE);
    }
}

void run(uint64_t* d, uint64_t batch, const ntt::NTTConfig* c, bool inverse, int engine, cudaStream_t s,
         const char* what) {
    check(nttb_u64_transform(c->plan, d, batch, inverse ? 1 : 0, engine, (void*)s), what);
}

}  // namespace

namespace ntt {

NTTConfig* ntt_init(uint64_t n, uint64_t q) {
    if (n == 0 || (n & (n - 1)) != 0) {
        std::fprintf(stderr, "ntt_init: N must be a power of 2\n");
        std::abort();
    }
    nttb_plan* plan = nullptr;
    check(nttb_plan_create(n, q, &plan), "ntt_init");
    nttb_plan_info info;
    check(nttb_plan_get_info(plan, &info), "ntt_init");
    auto* c = new NTTConfig();
    c->n = info.n;
    c->log_n = info.log_n;
    c->q = info.q;
    c->mu = info.mu;
    c->d_twiddles = info.d_twiddles;
    c->d_twiddles_inv = info.d_twiddles_inv;
    c->params.q = info.params.q;
    c->params.q_twice = info.params.q_twice;
    c->params.barrett_k = info.params.barrett_k;
    c->params.barrett_m = info.params.barrett_m;
    c->params.omega = info.params.omega;
    c->params.omega_inv = info.params.omega_inv;
    c->params.n_inv = info.params.n_inv;
    c->plan = plan;
    return c;
}

void ntt_cleanup(NTTConfig* c) {
    if (!c) return;
    nttb_plan_destroy(c->plan);
    delete c;
}

void ntt_forward_basic(uint64_t* d, const NTTConfig* c, cudaStream_t s) {
    run(d, 1, c, false, NTTB_ENGINE_SCALAR, s, "ntt_forward_basic");
}
void ntt_inverse_basic(uint64_t* d, const NTTConfig* c, cudaStream_t s) {
    run(d, 1, c, true, NTTB_ENGINE_SCALAR, s, "ntt_inverse_basic");
}
void ntt_forward_four_step(uint64_t* d, const NTTConfig* c, cudaStream_t s) {
    check(nttb_u64_four_step(c->plan, d, 0, (void*)s), "ntt_forward_four_step");
}
void ntt_inverse_four_step(uint64_t* d, const NTTConfig* c, cudaStream_t s) {
    check(nttb_u64_four_step(c->plan, d, 1, (void*)s), "ntt_inverse_four_step");
}
void ntt_forward_tlmop(uint64_t* d, const NTTConfig* c, cudaStream_t s) { ntt_forward_optimized(d, c, s); }
void ntt_inverse_tlmop(uint64_t* d, const NTTConfig* c, cudaStream_t s) { ntt_inverse_optimized(d, c, s); }
void ntt_forward_optimized(uint64_t* d, const NTTConfig* c, cudaStream_t s) {
    run(d, 1, c, false, NTTB_ENGINE_AUTO, s, "ntt_forward_optimized");
}
void ntt_inverse_optimized(uint64_t* d, const NTTConfig* c, cudaStream_t s) {
    run(d, 1, c, true, NTTB_ENGINE_AUTO, s, "ntt_inverse_optimized");
}

void ntt_forward_rowmaj(uint64_t* d, const NTTConfig* c, cudaStream_t s) {
    check(nttb_u64_rowmaj_forward(c->plan, d, (void*)s), "ntt_forward_rowmaj");
}
void rowmaj_to_pretransposed(uint64_t* dst, const uint64_t* src, int N1, int N2, cudaStream_t s) {
    check(nttb_u64_transpose(dst, src, (uint64_t)N1, (uint64_t)N2, (void*)s), "rowmaj_to_pretransposed");
}
void rowmaj_from_pretransposed(uint64_t* dst, const uint64_t* src, int N1, int N2, cudaStream_t s) {
    check(nttb_u64_transpose(dst, src, (uint64_t)N2, (uint64_t)N1, (void*)s), "rowmaj_from_pretransposed");
}

static void batch(uint64_t* d, uint64_t b, const NTTConfig* c, NTTVariant v, cudaStream_t s, bool inverse) {
    switch (v) {
        case NTTVariant::BASIC:
            run(d, b, c, inverse, NTTB_ENGINE_SCALAR, s, "ntt_batch");
            break;
        case NTTVariant::FOUR_STEP:
            for (uint64_t i = 0; i < b; i++)
                check(nttb_u64_four_step(c->plan, d + i * c->n, inverse ? 1 : 0, (void*)s), "ntt_batch");
            break;
        case NTTVariant::TLMOP:
        case NTTVariant::FULL_OPTIMIZED:
            run(d, b, c, inverse, NTTB_ENGINE_AUTO, s, "ntt_batch");
            break;
    }
}

void ntt_forward_batch(uint64_t* d, uint64_t b, const NTTConfig* c, NTTVariant v, cudaStream_t s) {
    batch(d, b, c, v, s, false);
}
void ntt_inverse_batch(uint64_t* d, uint64_t b, const NTTConfig* c, NTTVariant v, cudaStream_t s) {
    batch(d, b, c, v, s, true);
}

void poly_multiply_ntt(uint64_t* r, const uint64_t* a, const uint64_t* b, const NTTConfig* c, cudaStream_t s) {
    check(nttb_u64_pointwise_mul(c->plan, r, a, b, (void*)s), "poly_multiply_ntt");
}

void bit_reverse_permute(uint64_t* d, uint64_t n, cudaStream_t s) {
    check(nttb_u64_bit_reverse(d, n, (void*)s), "bit_reverse_permute");
}

void ntt_host(std::vector<uint64_t>& data, const ModularParams& p, bool inverse) {
    nttb_modular_params mp{p.q, p.q_twice, p.barrett_k, p.barrett_m, p.omega, p.omega_inv, p.n_inv};
    check(nttb_host_ntt(data.data(), data.size(), &mp, inverse ? 1 : 0), "ntt_host");
}

}  // namespace ntt
