// tc_int8.cu -- INT8 tensor-core (tcgen05 kind::i8) engine for 31-bit moduli.
//
// Byte-plane DFT contraction.  A length-L DFT of vectors x (L residues < 2^32)
// is one u8 x u8 -> s32 GEMM:
//   * operand A (M = 128 vectors, K = 4L bytes): the residues themselves.  A
//     K-major row of L little-endian uint32 words IS the row of 4L byte
//     planes, K index 4j + p = byte p of x_j.  No splitting is done.
//   * operand B (N = 4L rows, K = 4L bytes), precomputed per modulus:
//       B[(a, k)][(j, p)] = byte a of ((256^p * 2^32 * W[k][j]) mod q)
//   * D[m][(a, k)] = sum_{j,p} byte_p(x_j) * B[(a,k)][(j,p)]   (exact: <= 4L*255^2 < 2^31)
//   * sum_a 256^a D[m][(a, k)] == 2^32 * sum_j W[k][j] x_j  (mod q), < 2^49, and one
//     Montgomery REDC by 2^32 returns y_k = (W x)_k in [0, 2q).
// The four INT32 accumulator planes of a vector live in one TMEM lane, so one
// thread recombines them with three shifted adds -- no cross-thread exchange.
//
// N = 2^16 (64 x 64 x 16) runs as two passes; data layout [poly][limb][N]:
//   pass A: for each column b < 1024 of x viewed as [64][1024]:
//             U[d][b] = DFT64(x[.][b])[d] * t_A(b, d)
//           stored transposed (U at b*64 + d) so that each 128-column tile
//           writes one contiguous 32 KB block.
//   pass B: for each row d, Z = DFT1024(U[d][.]) as DFT64 (over stride 16,
//           twiddle t_B1) then DFT16 (contiguous); X[d + 64 k] = Z[k].  A tile
//           of 8 rows reads and writes exactly the same positions, so pass B
//           runs in place on its buffer.
// The four-step twiddles t_A, t_B1 are geometric in the output index and are
// generated in the epilogue (one Montgomery product to apply, one to advance).
// Negacyclic twists and n^-1 are folded into the B matrices and the twiddle
// ratios, so they cost nothing extra.
#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>
#include <vector>

#include "../../include/ntt_b200.h"
#include "engines.hpp"
#include "plan.hpp"
#include "profiler.hpp"
#include "tcgen05.cuh"

namespace nttb {

__device__ uint32_t g_tc_error;  // bit 0: an mbarrier wait ran out of budget

namespace {

constexpr uint32_t kMatBytes64 = 64 * 1024;  // DFT-64 byte-plane image (256 rows x 256 B)
constexpr uint32_t kMatBytes16 = 4 * 1024;   // DFT-16 byte-plane image (64 rows x 64 B)

// Device constants of one modulus for one direction.
struct TcLimb {
    uint32_t q, qinv;        // modulus, -q^-1 mod 2^32
    uint32_t one_m, pad_;    // 2^32 mod q
    const uint32_t* a_start; // pass A: t_A(b, d) = a_start[b] * a_ratio[b]^d  (Montgomery form)
    const uint32_t* a_ratio;
    const uint32_t* b_ratio; // pass B level 1: t_B1(b2, d2) = b_ratio[b2]^d2
    const uint8_t* mat_a;    // DFT-64 image for pass A
    const uint8_t* mat_b1;   // DFT-64 image for pass B level 1
    const uint8_t* mat_b2;   // DFT-16 image for pass B level 2
};

struct Int8Cache {
    uint32_t log_n = 0;
    TcLimb* d_fwd = nullptr;
    TcLimb* d_inv = nullptr;
    void* d_blob = nullptr;
};

// ---- device arithmetic ------------------------------------------------------------
__device__ __forceinline__ uint32_t redc64(uint64_t v, uint32_t q, uint32_t qinv) {
    const uint32_t m = (uint32_t)v * qinv;
    return (uint32_t)((v + (uint64_t)m * q) >> 32);  // [0, 2q) for v < q * 2^32
}
__device__ __forceinline__ uint32_t combine_redc(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3, uint32_t q,
                                                 uint32_t qinv) {
    uint64_t v = (uint64_t)c0 + ((uint64_t)c1 << 8) + ((uint64_t)c2 << 16) + ((uint64_t)c3 << 24);
    return redc64(v, q, qinv);
}
// a < 2q, b < q -> a*b*2^-32 mod q in [0, 2q)
__device__ __forceinline__ uint32_t mont_lazy(uint32_t a, uint32_t b, uint32_t q, uint32_t qinv) {
    return redc64((uint64_t)a * b, q, qinv);
}
__device__ __forceinline__ uint32_t canon(uint32_t x, uint32_t q) { return x >= q ? x - q : x; }

__device__ __forceinline__ void flag_timeout() { atomicOr(&g_tc_error, 1u); }

// Copies `bytes` (multiple of 16) from global to shared with 16-byte loads.
__device__ __forceinline__ void copy_g2s(uint8_t* s, const uint8_t* g, uint32_t bytes) {
    const uint4* src = reinterpret_cast<const uint4*>(g);
    uint4* dst = reinterpret_cast<uint4*>(s);
    for (uint32_t i = threadIdx.x; i < bytes / 16; i += blockDim.x) dst[i] = __ldg(src + i);
}

// Issues the K = 256-byte contraction (8 MMAs of K = 32) into TMEM columns
// [tmem, tmem + N) and commits to `bar`.
__device__ __forceinline__ void issue_k256(uint32_t tmem, const uint8_t* A, uint32_t a_rows, const uint8_t* B,
                                           uint32_t b_rows, uint32_t N, uint64_t* bar) {
    tc::fence_after_sync();
    const uint32_t idesc = tc::idesc_u8(128, N);
    const uint32_t a0 = tc::smem_u32(A), b0 = tc::smem_u32(B);
#pragma unroll
    for (uint32_t ks = 0; ks < 8; ks++) {
        const uint32_t ka = a0 + (ks >> 2) * a_rows * 128u + (ks & 3u) * 32u;
        const uint32_t kb = b0 + (ks >> 2) * b_rows * 128u + (ks & 3u) * 32u;
        tc::mma_i8(tmem, tc::desc_k_sw128(ka), tc::desc_k_sw128(kb), idesc, ks > 0);
    }
    tc::commit(bar);
}

// ============================================================ pass A (N = 2^16)
// One CTA: 128 consecutive columns b0.. of one (poly, limb); 128 threads.
// Input x[a*1024 + b] from `src`; output U[d][b] at (b*64 + d) in `dst`.
__global__ void __launch_bounds__(128) int8_pass_a_n16(const uint32_t* __restrict__ src, uint32_t* __restrict__ dst,
                                                       const TcLimb* __restrict__ limbs, uint32_t n_limbs) {
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    uint8_t* sA = smem;                  // 2 kblocks x 128 rows x 128 B = 32 KB
    uint8_t* sB = smem + 32768;          // 64 KB
    uint64_t* bar = reinterpret_cast<uint64_t*>(smem + 32768 + kMatBytes64);  // [0] MMA done, [1] B landed
    uint32_t* slot = reinterpret_cast<uint32_t*>(bar + 2);

    const uint32_t tid = threadIdx.x, warp = tid >> 5;
    const uint32_t limb = blockIdx.y, poly = blockIdx.z, b0 = blockIdx.x * 128u;
    const TcLimb L = limbs[limb];
    const uint64_t off = ((uint64_t)poly * n_limbs + limb) << 16;
    const uint32_t* x = src + off;
    uint32_t* out = dst + off;

    if (warp == 0) tc::tmem_alloc(slot, 256);
    if (tid == 0) {
        tc::mbar_init(bar, 1);
        tc::mbar_init(bar + 1, 1);
        tc::mbar_expect_tx(bar + 1, kMatBytes64);
#pragma unroll
        for (uint32_t i = 0; i < 4; i++) tc::bulk_g2s(sB + i * 16384u, L.mat_a + i * 16384u, 16384u, bar + 1);
    }
    // transposed load: vector m = column b0 + m, K index a (4 residues per 16-byte
    // chunk); all 64 loads are in flight before the first shared-memory store
    {
        const uint32_t* col = x + b0 + tid;
        uint32_t v[64];
#pragma unroll
        for (uint32_t a = 0; a < 64; a++) v[a] = __ldg(col + a * 1024u);
#pragma unroll
        for (uint32_t c = 0; c < 16; c++)
            *reinterpret_cast<uint4*>(sA + tc::sw128_offset(tid, 16 * c, 128)) =
                make_uint4(v[4 * c], v[4 * c + 1], v[4 * c + 2], v[4 * c + 3]);
    }
    tc::fence_proxy_async_smem();
    tc::fence_before_sync();
    __syncthreads();
    const uint32_t taddr = *slot;
    if (tid == 0) {
        if (!tc::mbar_wait_bounded(bar + 1, 0)) flag_timeout();
        issue_k256(taddr, sA, 128, sB, 256, 256, bar);
    }
    __syncwarp();
    const bool ok = tc::mbar_wait_bounded(bar, 0);
    tc::fence_after_sync();
    if (!ok) {
        if (tid == 0) flag_timeout();
    } else {
        const uint32_t q = L.q, qinv = L.qinv;
        const uint32_t b = b0 + tid;
        uint32_t tw = L.a_start[b];
        const uint32_t ratio = L.a_ratio[b];
        uint4* orow = reinterpret_cast<uint4*>(out + (uint64_t)b * 64u);
        const uint32_t lane_base = taddr + ((warp * 32u) << 16);
#pragma unroll 1
        for (uint32_t dc = 0; dc < 4; dc++) {
            uint32_t c0[16], c1[16], c2[16], c3[16];
            tc::ld_32x32b_x16(lane_base + 0 * 64 + dc * 16, c0);
            tc::ld_32x32b_x16(lane_base + 1 * 64 + dc * 16, c1);
            tc::ld_32x32b_x16(lane_base + 2 * 64 + dc * 16, c2);
            tc::ld_32x32b_x16(lane_base + 3 * 64 + dc * 16, c3);
            tc::ld_wait();
            uint32_t y[16];
#pragma unroll
            for (int i = 0; i < 16; i++) {
                const uint32_t t = combine_redc(c0[i], c1[i], c2[i], c3[i], q, qinv);
                y[i] = canon(mont_lazy(t, tw, q, qinv), q);
                tw = canon(mont_lazy(tw, ratio, q, qinv), q);
            }
#pragma unroll
            for (int i = 0; i < 4; i++)
                orow[dc * 4 + i] = make_uint4(y[4 * i], y[4 * i + 1], y[4 * i + 2], y[4 * i + 3]);
        }
    }
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 0) tc::tmem_dealloc(taddr, 256);
}

// ============================================================ pass B (N = 2^16)
// One CTA: 8 rows d0..d0+7 of U (U[d][b] at b*64 + d in `src`).  128 threads.
// Level 1: vector m = (r = m & 7, b2 = m >> 3), elements a2 at row position
// a2*16 + b2 -> DFT64 over a2, twiddle b_ratio[b2]^d2 -> A2 (SW64, rows
// d2*8 + r, K index b2).  Level 2: DFT16 over b2 -> X[d0 + r + 64*d2 + 4096*c2].
__global__ void __launch_bounds__(128) int8_pass_b_n16(const uint32_t* src, uint32_t* dst,
                                                       const TcLimb* __restrict__ limbs, uint32_t n_limbs) {
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    uint8_t* sA = smem;                          // level-1 A (32 KB), then level-2 A (32 KB, SW64)
    uint8_t* sB1 = smem + 32768;                 // 64 KB
    uint8_t* sB2 = smem + 32768 + kMatBytes64;   // 4 KB
    uint64_t* bar = reinterpret_cast<uint64_t*>(sB2 + kMatBytes16);  // [0] level 1, [1] level 2, [2] B landed
    uint32_t* slot = reinterpret_cast<uint32_t*>(bar + 3);

    const uint32_t tid = threadIdx.x, warp = tid >> 5;
    const uint32_t limb = blockIdx.y, poly = blockIdx.z, d0 = blockIdx.x * 8u;
    const TcLimb L = limbs[limb];
    const uint64_t off = ((uint64_t)poly * n_limbs + limb) << 16;
    const uint32_t* u = src + off;
    uint32_t* out = dst + off;
    const uint32_t q = L.q, qinv = L.qinv;

    if (warp == 0) tc::tmem_alloc(slot, 256);
    if (tid == 0) {
        tc::mbar_init(bar, 1);
        tc::mbar_init(bar + 1, 1);
        tc::mbar_init(bar + 2, 1);
        tc::mbar_expect_tx(bar + 2, kMatBytes64 + kMatBytes16);
#pragma unroll
        for (uint32_t i = 0; i < 4; i++) tc::bulk_g2s(sB1 + i * 16384u, L.mat_b1 + i * 16384u, 16384u, bar + 2);
        tc::bulk_g2s(sB2, L.mat_b2, kMatBytes16, bar + 2);
    }
    const uint32_t r = tid & 7u, b2 = tid >> 3;
    {
        const uint32_t* base = u + d0 + r;
        uint32_t v[64];
#pragma unroll
        for (uint32_t a2 = 0; a2 < 64; a2++) v[a2] = base[(a2 * 16u + b2) * 64u];
#pragma unroll
        for (uint32_t c = 0; c < 16; c++)
            *reinterpret_cast<uint4*>(sA + tc::sw128_offset(tid, 16 * c, 128)) =
                make_uint4(v[4 * c], v[4 * c + 1], v[4 * c + 2], v[4 * c + 3]);
    }
    tc::fence_proxy_async_smem();
    tc::fence_before_sync();
    __syncthreads();
    const uint32_t taddr = *slot;
    const uint32_t lane_base = taddr + ((warp * 32u) << 16);
    if (tid == 0) {
        if (!tc::mbar_wait_bounded(bar + 2, 0)) flag_timeout();
        issue_k256(taddr, sA, 128, sB1, 256, 256, bar);
    }
    __syncwarp();
    bool ok = tc::mbar_wait_bounded(bar, 0);
    tc::fence_after_sync();
    if (ok) {
        // level-1 epilogue -> A2 (SW64 layout, 512 rows x 64 B), overwriting level-1 A
        const uint32_t ratio = L.b_ratio[b2];
        uint32_t tw = L.one_m;
#pragma unroll 1
        for (uint32_t dc = 0; dc < 4; dc++) {
            uint32_t c0[16], c1[16], c2[16], c3[16];
            tc::ld_32x32b_x16(lane_base + 0 * 64 + dc * 16, c0);
            tc::ld_32x32b_x16(lane_base + 1 * 64 + dc * 16, c1);
            tc::ld_32x32b_x16(lane_base + 2 * 64 + dc * 16, c2);
            tc::ld_32x32b_x16(lane_base + 3 * 64 + dc * 16, c3);
            tc::ld_wait();
#pragma unroll
            for (int i = 0; i < 16; i++) {
                const uint32_t d2 = dc * 16 + i;
                const uint32_t t = combine_redc(c0[i], c1[i], c2[i], c3[i], q, qinv);
                const uint32_t y = mont_lazy(t, tw, q, qinv);  // [0, 2q): exact input for level 2
                tw = canon(mont_lazy(tw, ratio, q, qinv), q);
                *reinterpret_cast<uint32_t*>(sA + tc::sw64_offset(d2 * 8u + r, 4u * b2)) = y;
            }
        }
    } else if (tid == 0) {
        flag_timeout();
    }
    tc::fence_proxy_async_smem();
    tc::fence_before_sync();
    __syncthreads();
    if (ok && tid == 0) {
        tc::fence_after_sync();
        const uint32_t idesc = tc::idesc_u8(128, 64);
        const uint32_t a0 = tc::smem_u32(sA), bb = tc::smem_u32(sB2);
#pragma unroll
        for (uint32_t t = 0; t < 4; t++)
#pragma unroll
            for (uint32_t ks = 0; ks < 2; ks++)
                tc::mma_i8(taddr + t * 64u, tc::desc_k_sw64(a0 + t * 8192u + ks * 32u),
                           tc::desc_k_sw64(bb + ks * 32u), idesc, ks > 0);
        tc::commit(bar + 1);
    }
    __syncwarp();
    if (ok) {
        ok = tc::mbar_wait_bounded(bar + 1, 0);
        tc::fence_after_sync();
        if (!ok && tid == 0) flag_timeout();
    }
    if (ok) {
#pragma unroll 1
        for (uint32_t t = 0; t < 4; t++) {
            uint32_t c0[16], c1[16], c2[16], c3[16];
            const uint32_t col = lane_base + t * 64u;
            tc::ld_32x32b_x16(col + 0, c0);
            tc::ld_32x32b_x16(col + 16, c1);
            tc::ld_32x32b_x16(col + 32, c2);
            tc::ld_32x32b_x16(col + 48, c3);
            tc::ld_wait();
            const uint32_t row2 = t * 128u + tid;
            const uint32_t d2 = row2 >> 3, rr = row2 & 7u;
            uint32_t* o = out + d0 + rr + 64u * d2;
#pragma unroll
            for (int c = 0; c < 16; c++)
                o[4096u * c] = canon(combine_redc(c0[c], c1[c], c2[c], c3[c], q, qinv), q);
        }
    }
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 0) tc::tmem_dealloc(taddr, 256);
}

constexpr size_t kSmemA = 32768 + kMatBytes64 + 64 + 1024;
constexpr size_t kSmemB = 32768 + kMatBytes64 + kMatBytes16 + 64 + 1024;

// ---- host: tables and byte-plane images ------------------------------------------------
// Image of B[(a, k)][(j, p)] = byte a of (256^p * 2^32 * W[k][j] mod q), K-major SW128,
// 256 rows, two 128-byte K blocks.
void build_image64(uint8_t* img, const std::vector<uint64_t>& W, uint64_t q) {
    std::memset(img, 0, kMatBytes64);
    for (uint32_t k = 0; k < 64; k++)
        for (uint32_t j = 0; j < 64; j++)
            for (uint32_t p = 0; p < 4; p++) {
                const uint64_t v = h_mulmod(h_to_mont32(W[k * 64 + j], q), (1ull << (8 * p)) % q, q);
                for (uint32_t a = 0; a < 4; a++)
                    img[tc::sw128_offset(a * 64 + k, 4 * j + p, 256)] = (uint8_t)(v >> (8 * a));
            }
}
// Same for a 16-point matrix: 64 rows x 64 bytes, K-major SW64.
void build_image16(uint8_t* img, const std::vector<uint64_t>& W, uint64_t q) {
    std::memset(img, 0, kMatBytes16);
    for (uint32_t c = 0; c < 16; c++)
        for (uint32_t b = 0; b < 16; b++)
            for (uint32_t p = 0; p < 4; p++) {
                const uint64_t v = h_mulmod(h_to_mont32(W[c * 16 + b], q), (1ull << (8 * p)) % q, q);
                for (uint32_t a = 0; a < 4; a++)
                    img[tc::sw64_offset(a * 16 + c, 4 * b + p)] = (uint8_t)(v >> (8 * a));
            }
}

std::vector<uint64_t> dft_matrix(uint32_t L, uint64_t root, uint64_t q, uint64_t row_twist = 1, uint64_t col_twist = 1,
                                 uint64_t scale = 1) {
    // W[k][j] = scale * row_twist^k * col_twist^j * root^(j*k)
    std::vector<uint64_t> W((size_t)L * L);
    for (uint32_t k = 0; k < L; k++)
        for (uint32_t j = 0; j < L; j++) {
            uint64_t v = h_powmod(root, (uint64_t)j * k % (2ull * L * L), q);
            v = h_mulmod(v, h_powmod(row_twist, k, q), q);
            v = h_mulmod(v, h_powmod(col_twist, j, q), q);
            W[(size_t)k * L + j] = h_mulmod(v, scale, q);
        }
    return W;
}

int build_cache(Plan32& p, Int8Cache* c) {
    const uint32_t n = p.n, nl = p.n_limbs;
    // blob layout per limb: 4 DFT-64 images + 2 DFT-16 images + tables
    const size_t tab_words = 4 * 1024 + 2 * 16;
    const size_t per_limb = 4 * (size_t)kMatBytes64 + 2 * (size_t)kMatBytes16 + tab_words * 4;
    std::vector<uint8_t> blob(per_limb * nl);
    uint8_t* d_blob = nullptr;
    if (cudaMalloc(&d_blob, blob.size()) != cudaSuccess) return 4;
    std::vector<TcLimb> fwd(nl), inv(nl);
    for (uint32_t l = 0; l < nl; l++) {
        const LimbHost& H = p.limbs[l];
        const uint64_t q = H.q;
        uint8_t* h = blob.data() + per_limb * l;
        uint8_t* d = d_blob + per_limb * l;
        const uint64_t w = H.omega, wi = H.omega_inv;
        const uint64_t w64 = h_powmod(w, n / 64, q), w64i = h_powmod(wi, n / 64, q);
        const uint64_t w16 = h_powmod(w, n / 16, q), w16i = h_powmod(wi, n / 16, q);
        // pass A forward matrix: negacyclic folds psi^(a * n/64) on the input index
        std::vector<uint64_t> Af = p.negacyclic ? dft_matrix(64, w64, q, 1, h_powmod(H.psi, n / 64, q))
                                                : dft_matrix(64, w64, q);
        std::vector<uint64_t> Ai = dft_matrix(64, w64i, q);
        // pass B level 2 inverse: n^-1 (and psi^-(4096 c2)) folded on the output index
        std::vector<uint64_t> B2f = dft_matrix(16, w16, q);
        std::vector<uint64_t> B2i = p.negacyclic ? dft_matrix(16, w16i, q, h_powmod(H.psi_inv, 4096, q), 1, H.n_inv)
                                                 : dft_matrix(16, w16i, q, 1, 1, H.n_inv);
        build_image64(h + 0 * kMatBytes64, Af, q);
        build_image64(h + 1 * kMatBytes64, Ai, q);
        build_image64(h + 2 * kMatBytes64, dft_matrix(64, w64, q), q);  // pass B level 1 forward
        build_image64(h + 3 * kMatBytes64, Ai, q);                      // pass B level 1 inverse
        build_image16(h + 4 * kMatBytes64, B2f, q);
        build_image16(h + 4 * kMatBytes64 + kMatBytes16, B2i, q);
        uint32_t* tab = reinterpret_cast<uint32_t*>(h + 4 * kMatBytes64 + 2 * kMatBytes16);
        uint32_t* dtab = reinterpret_cast<uint32_t*>(d + 4 * kMatBytes64 + 2 * kMatBytes16);
        // pass A twiddles (b < 1024): forward start psi^b (negacyclic) or 1, ratio omega^b;
        // inverse start 1, ratio omega^-b (times psi^-1 for negacyclic)
        for (uint32_t b = 0; b < 1024; b++) {
            tab[0 * 1024 + b] = h_to_mont32(p.negacyclic ? h_powmod(H.psi, b, q) : 1, q);
            tab[1 * 1024 + b] = h_to_mont32(h_powmod(w, b, q), q);
            tab[2 * 1024 + b] = h_to_mont32(1, q);
            uint64_t ri = h_powmod(wi, b, q);
            if (p.negacyclic) ri = h_mulmod(ri, H.psi_inv, q);
            tab[3 * 1024 + b] = h_to_mont32(ri, q);
        }
        // pass B level-1 ratios (b2 < 16): omega_1024^(+-b2) (times psi^-64 for negacyclic inverse)
        for (uint32_t b2 = 0; b2 < 16; b2++) {
            tab[4096 + b2] = h_to_mont32(h_powmod(w, 64ull * b2, q), q);
            uint64_t ri = h_powmod(wi, 64ull * b2, q);
            if (p.negacyclic) ri = h_mulmod(ri, h_powmod(H.psi_inv, 64, q), q);
            tab[4096 + 16 + b2] = h_to_mont32(ri, q);
        }
        TcLimb f{}, v{};
        f.q = v.q = (uint32_t)q;
        f.qinv = v.qinv = h_neg_inv32((uint32_t)q);
        f.one_m = v.one_m = h_to_mont32(1, q);
        f.a_start = dtab;
        f.a_ratio = dtab + 1024;
        v.a_start = dtab + 2048;
        v.a_ratio = dtab + 3072;
        f.b_ratio = dtab + 4096;
        v.b_ratio = dtab + 4096 + 16;
        f.mat_a = d;
        v.mat_a = d + kMatBytes64;
        f.mat_b1 = d + 2 * kMatBytes64;
        v.mat_b1 = d + 3 * kMatBytes64;
        f.mat_b2 = d + 4 * kMatBytes64;
        v.mat_b2 = d + 4 * kMatBytes64 + kMatBytes16;
        fwd[l] = f;
        inv[l] = v;
    }
    if (cudaMemcpy(d_blob, blob.data(), blob.size(), cudaMemcpyHostToDevice) != cudaSuccess) {
        cudaFree(d_blob);
        return 3;
    }
    TcLimb* d_l = nullptr;
    if (cudaMalloc(&d_l, 2 * nl * sizeof(TcLimb)) != cudaSuccess) {
        cudaFree(d_blob);
        return 4;
    }
    cudaMemcpy(d_l, fwd.data(), nl * sizeof(TcLimb), cudaMemcpyHostToDevice);
    cudaMemcpy(d_l + nl, inv.data(), nl * sizeof(TcLimb), cudaMemcpyHostToDevice);
    c->d_fwd = d_l;
    c->d_inv = d_l + nl;
    c->d_blob = d_blob;
    c->log_n = p.log_n;
    return 0;
}

}  // namespace

bool int8_serves(const Plan32& p, bool src_u64) { return !src_u64 && p.log_n == 16; }

int int8_transform32(Plan32& p, const void* src, void* dst, bool src_u64, uint32_t n_polys, bool inverse,
                     cudaStream_t s) {
    if (!int8_serves(p, src_u64)) return 1;
    if (n_polys > 65535 || p.n_limbs > 65535) return 1;
    auto* c = reinterpret_cast<Int8Cache*>(p.engine_data[1]);
    if (!c) {
        c = new Int8Cache();
        int rc = build_cache(p, c);
        if (rc) {
            delete c;
            return 2;
        }
        p.engine_data[1] = c;
        static bool attr = false;
        if (!attr) {
            cudaFuncSetAttribute(int8_pass_a_n16, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmemA);
            cudaFuncSetAttribute(int8_pass_b_n16, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmemB);
            attr = true;
        }
    }
    const uint32_t* in = static_cast<const uint32_t*>(src);
    uint32_t* out = static_cast<uint32_t*>(dst);
    uint32_t* mid = out;
    if (src == dst) {  // pass A cannot run in place: stage it in the plan's workspace
        mid = static_cast<uint32_t*>(plan_workspace(&p.ws, &p.ws_bytes, (size_t)n_polys * p.n_limbs * p.n * 4));
        if (!mid) return 2;
    }
    const TcLimb* limbs = inverse ? c->d_inv : c->d_fwd;
    {
        ProfScope prof("int8_pass_a_n16", s);
        int8_pass_a_n16<<<dim3(8, p.n_limbs, n_polys), 128, kSmemA, s>>>(in, mid, limbs, p.n_limbs);
    }
    {
        ProfScope prof("int8_pass_b_n16", s);
        int8_pass_b_n16<<<dim3(8, p.n_limbs, n_polys), 128, kSmemB, s>>>(mid, out, limbs, p.n_limbs);
    }
    return cudaGetLastError() == cudaSuccess ? 0 : 2;
}

void int8_release(Plan32* p) {
    auto* c = reinterpret_cast<Int8Cache*>(p->engine_data[1]);
    if (!c) return;
    if (c->d_fwd) cudaFree(c->d_fwd);
    if (c->d_blob) cudaFree(c->d_blob);
    delete c;
    p->engine_data[1] = nullptr;
}

uint32_t int8_device_errors(bool clear) {
    uint32_t v = 0;
    cudaMemcpyFromSymbol(&v, g_tc_error, sizeof v);
    if (clear) {
        uint32_t z = 0;
        cudaMemcpyToSymbol(g_tc_error, &z, sizeof z);
    }
    return v;
}

}  // namespace nttb
