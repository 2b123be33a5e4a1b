// klimb.cu -- the K-limb forward NTT (residues of K x 24-bit limbs in
// Montgomery form, the reference's DScalar<K> layout) behind
// nttb_klimb_forward.
//
// The transform is the radix-2 decimation-in-time network of the reference's
// host_ntt_naive (include/ntt_arbitrary.cuh:2651-2676) applied in the
// Montgomery domain: bit-reverse, then for stage s = 0..log_n-1 the butterfly
// (a[i], a[i + 2^s]) <- (u + t, u - t), t = a[i + 2^s] * tw[k * n / 2^(s+1)],
// k = i mod 2^s.  The network is reproduced stage for stage (not replaced by
// another DFT factorisation) because the reference's K = 2 field is not a
// field with the advertised root of unity, so only the network itself defines
// the result there.
//
// Execution: one in-place bit reversal, then "stage group" passes.  A pass
// runs r consecutive stages s0..s0+r-1 on tiles held in shared memory: a tile
// is C columns x 2^r elements, column (G, low) = { G 2^(s0+r) + j 2^s0 + low },
// C consecutive `low` values so that loads are coalesced.  The first pass
// (s0 = 0, C = 1) covers contiguous blocks; N = 2^20 with K = 3 needs two
// passes instead of the twenty radix-2 sweeps.
#include <cuda_runtime.h>

#include <cstdint>

#include "../../include/ntt_b200.h"
#include "../../include/ntt_limb_arith.cuh"
#include "engines.hpp"
#include "klimb_plan.hpp"
#include "profiler.hpp"

namespace nttb {
namespace {

template <int K>
struct Limbs {
    uint32_t l[K];
};

template <int K>
__global__ void klimb_bitrev(uint32_t* data, uint32_t n, uint32_t log_n) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || log_n == 0) return;
    const uint32_t j = __brev(i) >> (32u - log_n);
    if (i >= j) return;
    uint32_t* a = data + (size_t)i * K;
    uint32_t* b = data + (size_t)j * K;
#pragma unroll
    for (int k = 0; k < K; k++) {
        const uint32_t t = a[k];
        a[k] = b[k];
        b[k] = t;
    }
}

// In-place bit reversal by tile pairs, log_n >= 8.  With the index split as
// (a, b, c) -- a the high 4 bits, c the low 4, b the log_n - 8 middle bits --
// element (a, b, c) moves to (rev4(c), rev(b), rev4(a)).  One block takes the
// 16 x 16-element tiles of middle values b and rev(b) (b <= rev(b)): each tile
// row is 16 K contiguous words, read and written as flat word runs, and the
// permutation happens in shared memory.
__device__ __forceinline__ uint32_t rev4(uint32_t v) { return __brev(v) >> 28; }

template <int K>
__global__ void __launch_bounds__(256) klimb_bitrev_tiled(uint32_t* data, uint32_t log_n) {
    __shared__ uint32_t t0[256 * K], t1[256 * K];
    const uint32_t M = log_n - 8u, row = 16u * K;
    const uint32_t b = blockIdx.x, br = M ? (__brev(b) >> (32u - M)) : 0u;
    if (br < b) return;
    auto row_base = [&](uint32_t a, uint32_t mid) -> size_t {
        return (((size_t)a << (M + 4)) + ((size_t)mid << 4)) * K;
    };
    for (uint32_t w = threadIdx.x; w < 256u * K; w += blockDim.x) {
        const uint32_t a = w / row, off = w % row;
        t0[w] = data[row_base(a, b) + off];
        t1[w] = data[row_base(a, br) + off];
    }
    __syncthreads();
    // output row a2 of the tile stored at mid, word off = c2 K + k: element
    // (rev4(c2), rev4(a2)) of the tile loaded from the partner position
    for (uint32_t w = threadIdx.x; w < 256u * K; w += blockDim.x) {
        const uint32_t a2 = w / row, off = w % row, c2 = off / K, k = off % K;
        const uint32_t src = (rev4(c2) * 16u + rev4(a2)) * K + k;
        data[row_base(a2, br) + off] = t0[src];
        data[row_base(a2, b) + off] = t1[src];
    }
}

// Stages s0 .. s0 + r - 1 on tiles of 2^(r + logC) elements (shared memory,
// limb-major: sm[k * E + e], e = j * C + c).
// With `fused_bitrev` (one CTA holding the whole transform) the tile loads
// element i from its bit-reversed position: every load precedes the first
// store, so the permutation needs no pass of its own.
template <int K>
__global__ void __launch_bounds__(256) klimb_group(uint32_t* data, const uint32_t* tw, uint32_t log_n, uint32_t s0,
                                                   uint32_t r, uint32_t logC, Limbs<K> p, uint32_t np,
                                                   bool fused_bitrev) {
    extern __shared__ uint32_t sm[];
    // a one-warp tile (small transforms) needs only the warp's barrier
    const bool one_warp = blockDim.x <= 32;
    auto tile_sync = [&]() {
        if (one_warp) __syncwarp();
        else __syncthreads();
    };
    const uint32_t E = 1u << (r + logC), C = 1u << logC;
    const uint32_t chunks = (1u << s0) >> logC;  // column chunks per group of 2^(s0 + r)
    const uint32_t G = blockIdx.x / chunks, low0 = (blockIdx.x % chunks) << logC;
    const size_t base = ((size_t)G << (s0 + r)) + low0;
    for (uint32_t e = threadIdx.x; e < E; e += blockDim.x) {
        size_t i = base + ((size_t)(e >> logC) << s0) + (e & (C - 1));
        if (fused_bitrev) i = log_n ? (__brev((uint32_t)i) >> (32u - log_n)) : 0u;
        const uint32_t* src = data + i * K;
#pragma unroll
        for (int k = 0; k < K; k++) sm[k * E + e] = src[k];
    }
    tile_sync();
    for (uint32_t t = 0; t < r; t++) {
        const uint32_t half = 1u << t, tshift = log_n - s0 - t - 1;
        for (uint32_t bf = threadIdx.x; bf < E / 2; bf += blockDim.x) {
            const uint32_t c = bf & (C - 1), pi = bf >> logC;
            const uint32_t jlo = ((pi >> t) << (t + 1)) | (pi & (half - 1));
            const uint32_t elo = (jlo << logC) + c, ehi = elo + (half << logC);
            const uint32_t ktw = ((jlo & (half - 1)) << s0) + low0 + c;
            const uint32_t* w = tw + ((size_t)ktw << tshift) * K;
            uint32_t wv[K], u[K], v[K], x[K];
#pragma unroll
            for (int k = 0; k < K; k++) {
                wv[k] = __ldg(w + k);
                u[k] = sm[k * E + elo];
                v[k] = sm[k * E + ehi];
            }
            nttb_limb::mont_mul<K>(x, v, wv, p.l, np);
            nttb_limb::add_mod<K>(v, u, x, p.l);
            nttb_limb::sub_mod<K>(u, u, x, p.l);
#pragma unroll
            for (int k = 0; k < K; k++) {
                sm[k * E + elo] = v[k];
                sm[k * E + ehi] = u[k];
            }
        }
        tile_sync();
    }
    for (uint32_t e = threadIdx.x; e < E; e += blockDim.x) {
        const size_t i = base + ((size_t)(e >> logC) << s0) + (e & (C - 1));
        uint32_t* dst = data + i * K;
#pragma unroll
        for (int k = 0; k < K; k++) dst[k] = sm[k * E + e];
    }
}

template <int K>
int klimb_forward(uint32_t* d_data, const uint32_t* d_tw, uint32_t log_n, const uint32_t* prime, uint32_t np,
                  cudaStream_t s) {
    Limbs<K> p;
    for (int k = 0; k < K; k++) p.l[k] = prime[k];
    const uint32_t n = 1u << log_n;
    const KlimbPlan P = klimb_plan(K, log_n);
    if (P.single_tile) {
        ProfScope prof("klimb_group", s);
        const uint32_t threads = n / 2 < 256 ? (n / 2 > 0 ? n / 2 : 1) : 256;
        klimb_group<K><<<1, threads, (size_t)n * K * 4, s>>>(d_data, d_tw, log_n, 0, log_n, 0, p, np, true);
        return launch_rc();
    }
    {
        ProfScope prof("klimb_bitrev", s);
        if (log_n >= 8) klimb_bitrev_tiled<K><<<n >> 8, 256, 0, s>>>(d_data, log_n);
        else klimb_bitrev<K><<<(n + 255) / 256, 256, 0, s>>>(d_data, n, log_n);
        if (launch_rc()) return 2;
    }
    for (uint32_t i = 0; i < P.n_passes; i++) {
        const KlimbPass& ps = P.pass[i];
        const uint32_t E = 1u << (ps.r + ps.logC);
        const uint32_t threads = E / 2 < 256 ? E / 2 : 256;
        ProfScope prof("klimb_group", s);
        klimb_group<K><<<n / E, threads, (size_t)E * K * 4, s>>>(d_data, d_tw, log_n, ps.s0, ps.r, ps.logC, p, np,
                                                                  false);
        if (launch_rc()) return 2;
    }
    return 0;
}

}  // namespace
}  // namespace nttb

extern "C" {

NTTB_API int nttb_klimb_forward(uint32_t K, uint32_t* d_data, const uint32_t* d_tw, uint64_t n, uint32_t log_n,
                                const uint32_t* prime, uint32_t np, void* stream) {
    using nttb::fail;
    if (!d_data || !d_tw || !prime) return fail(NTTB_ERR_INVALID_ARG, "nttb_klimb_forward: null pointer");
    if (log_n > 24 || n != (1ull << log_n))
        return fail(NTTB_ERR_INVALID_ARG, "nttb_klimb_forward: n must be 2^log_n with log_n <= 24");
    if (K != 2 && K != 3 && K != 11)
        return fail(NTTB_ERR_UNSUPPORTED, "nttb_klimb_forward: K = %u (this build serves K = 2, 3, 11)", K);
    if ((prime[0] & 1u) == 0) return fail(NTTB_ERR_INVALID_ARG, "nttb_klimb_forward: even modulus");
    for (uint32_t k = 0; k < K; k++)
        if (prime[k] > nttb_limb::kMask) return fail(NTTB_ERR_INVALID_ARG, "nttb_klimb_forward: limb %u >= 2^24", k);
    if (np != nttb_limb::neg_inv24(prime[0]))
        return fail(NTTB_ERR_INVALID_ARG, "nttb_klimb_forward: np != -p^-1 mod 2^24");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    int rc = 0;
    switch (K) {
        case 2: rc = nttb::klimb_forward<2>(d_data, d_tw, log_n, prime, np, s); break;
        case 3: rc = nttb::klimb_forward<3>(d_data, d_tw, log_n, prime, np, s); break;
        default: rc = nttb::klimb_forward<11>(d_data, d_tw, log_n, prime, np, s); break;
    }
    return rc ? fail(NTTB_ERR_CUDA, "nttb_klimb_forward: kernel launch failed") : NTTB_OK;
}

}  // extern "C"
