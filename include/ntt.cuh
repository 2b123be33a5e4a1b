// ntt.cuh -- drop-in for the reference's include/ntt.cuh (namespace ntt).
//
// Every declaration keeps the reference's name, signature, argument meaning
// and default arguments (include/ntt.cuh:8-87); the definitions live in
// libntt_b200.so (ntt-tensorcore_b200/csrc/dropin.cpp) and run the B200
// kernels through the C ABI of ntt_b200.h.  Error behaviour follows the
// reference: a failing CUDA call prints a message and exits with
// EXIT_FAILURE, a non-power-of-two size aborts.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

#include "modular_arith.cuh"

struct nttb_plan;

namespace ntt {

struct NTTConfig {
    uint64_t n;      // transform size (power of two)
    uint64_t log_n;  // log2(n)
    uint64_t q;      // prime modulus
    uint64_t mu;     // floor(2^64 / q)

    uint64_t* d_twiddles;      // omega^k, k < n (device)
    uint64_t* d_twiddles_inv;  // omega^-k, k < n (device)

    ModularParams params;

    nttb_plan* plan;  // B200 plan behind this configuration (not in the reference)
};

enum class NTTVariant {
    BASIC,          // CUDA-core engine
    FOUR_STEP,      // the reference's four-step map
    TLMOP,          // same transform as FULL_OPTIMIZED
    FULL_OPTIMIZED  // fastest tensor-core engine for the modulus
};

NTTConfig* ntt_init(uint64_t n, uint64_t q = DEFAULT_PRIME);
void ntt_cleanup(NTTConfig* config);

void ntt_forward_basic(uint64_t* d_data, const NTTConfig* config, cudaStream_t stream = 0);
void ntt_inverse_basic(uint64_t* d_data, const NTTConfig* config, cudaStream_t stream = 0);

void ntt_forward_four_step(uint64_t* d_data, const NTTConfig* config, cudaStream_t stream = 0);
void ntt_inverse_four_step(uint64_t* d_data, const NTTConfig* config, cudaStream_t stream = 0);

void ntt_forward_tlmop(uint64_t* d_data, const NTTConfig* config, cudaStream_t stream = 0);
void ntt_inverse_tlmop(uint64_t* d_data, const NTTConfig* config, cudaStream_t stream = 0);

void ntt_forward_optimized(uint64_t* d_data, const NTTConfig* config, cudaStream_t stream = 0);
void ntt_inverse_optimized(uint64_t* d_data, const NTTConfig* config, cudaStream_t stream = 0);

void ntt_forward_rowmaj(uint64_t* d_data, const NTTConfig* config, cudaStream_t stream = 0);
void rowmaj_to_pretransposed(uint64_t* d_dst, const uint64_t* d_src, int N1, int N2, cudaStream_t stream = 0);
void rowmaj_from_pretransposed(uint64_t* d_dst, const uint64_t* d_src, int N1, int N2, cudaStream_t stream = 0);

void ntt_forward_batch(uint64_t* d_data, uint64_t batch_size, const NTTConfig* config,
                       NTTVariant variant = NTTVariant::BASIC, cudaStream_t stream = 0);
void ntt_inverse_batch(uint64_t* d_data, uint64_t batch_size, const NTTConfig* config,
                       NTTVariant variant = NTTVariant::BASIC, cudaStream_t stream = 0);

void poly_multiply_ntt(uint64_t* d_result, const uint64_t* d_a, const uint64_t* d_b, const NTTConfig* config,
                       cudaStream_t stream = 0);

void bit_reverse_permute(uint64_t* d_data, uint64_t n, cudaStream_t stream = 0);

void ntt_host(std::vector<uint64_t>& data, const ModularParams& params, bool inverse = false);

}  // namespace ntt
