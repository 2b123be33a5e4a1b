// tc_wide.cu -- INT8 tensor-core (tcgen05 kind::i8) engine for the wide
// plans (moduli 2^31 <= q < 2^62, residues as uint64 words) at n = 2^20:
// the multi-limb big-prime path of the reference (run_forward_ct_tcu<K>,
// include/ntt_arbitrary.cuh:2599-2646, limb products on FP64 MMA) on byte
// planes of 64-bit words.
//
// Byte-plane contraction, eight planes.  A length-32 DFT of vectors x (32
// residues < 2^64) is one u8 x u8 -> s32 GEMM with K = 256 bytes:
//   * operand A (M = 128 vectors): the residues as they are -- a K-major row
//     of 32 little-endian uint64 words is the row of 256 byte planes, K index
//     8 j + p = byte p of x_j;
//   * operand B (N = 256 = 32 outputs x 8 planes, output-major, row 8 k + a),
//     per modulus and direction:  B[8k + a][8j + p] = byte a of
//     ((256^p * 2^64 * W[k][j]) mod q);
//   * D[m][8k + a] = sum_{j,p} byte_p(x_j) B[8k + a][8j + p] <= 256 * 255^2 < 2^24,
//     and v_k = sum_a 256^a D[m][8k + a] < 2^81 is congruent to 2^64 (W x)_k:
//     one Montgomery REDC by 2^64 returns y_k < q + 2^17.
// A thread reads the eight planes of one output with one 8-column TMEM load.
//
// n = 2^20 as the four-step 1024 x 1024 over x[j1][j2] (j = 1024 j1 + j2):
//   pass A, per column j2:  U[k1][j2] = DFT1024(x[.][j2])[k1] * w^(j2 k1)
//           (the inverse also scales by n^-1), stored transposed at j2 * 1024 + k1;
//   pass B, per k1:         X[k1 + 1024 k2] = DFT1024(U[k1][.])[k2], stored at
//           k2 * 1024 + k1, the positions it was read from.
// Both are column passes over a 1024 x 1024 row-major array.  Each column's
// DFT-1024 (element j = 32 a2 + b2) is
//   level 1: Z[k1'][b2] = DFT32_a2(x[32 a2 + b2])[k1'] * w_1024^(b2 k1')
//   level 2: Y[k1' + 32 k2'] = DFT32_b2(Z[k1'][.])[k2'].
//
// Tile: 4 consecutive columns c0 .. c0 + 3 (128 level-1 vectors: row
// m = 32 col + b2, K word a2; 128 level-2 vectors: pass A row 32 col + k1',
// pass B row 4 k1' + col, K word b2).  One CTA of 256 threads (two per SM)
// holds the unit's DFT-32 image (64 KB) and level-1 twiddles; operand A is
// loaded from global memory, the level-1 epilogue writes the level-2 operand
// over it, the level-2 epilogue stores (pass A through a staging copy of the
// four output rows and bulk stores, pass B directly in 32-byte runs).  Thread
// (warp w, lane l) reads TMEM lanes 32 (w % 4) + l and outputs 16 (w / 4)
// .. + 15 of its row.  CTAs are persistent over consecutive tiles and keep
// the image while the modulus and direction stay the same.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <mutex>
#include <vector>

#include "../../include/ntt_b200.h"
#include "arith.cuh"
#include "bounds.cuh"
#include "engines.hpp"
#include "plan.hpp"
#include "profiler.hpp"
#include "tc_arith.cuh"
#include "tcgen05.cuh"

namespace nttb {

// bit 0: a bounded wait on the tile's MMA or constant copy ran out
__device__ uint32_t g_wide_error;
// NTT_DEBUG_BOUNDS build: failed range checks (bounds.cuh bits)
__device__ uint32_t g_wide_bounds;

namespace {

constexpr uint32_t kWThreads = 256;
constexpr uint32_t kWCols = 4;                 // columns per tile
constexpr uint32_t kWLog = 20, kWN1 = 1024;    // n = 1024 x 1024
constexpr uint32_t kWTiles = kWN1 / kWCols;    // tiles per pass and unit
constexpr uint32_t kWImg = 64 * 1024;          // DFT-32 image, 256 rows x 256 bytes
constexpr uint32_t kWT1Stride = 33;            // level-1 twiddle row stride (words, padded)
constexpr uint32_t kWT1Bytes = 32 * kWT1Stride * 8 + 16 * 8;  // 8576 B (a multiple of 16)
// per (modulus, direction) constant blob
//   [0, 64K)                 DFT-32 byte-plane image
//   [64K, +kWT1Bytes)        T1[b2][k1'] = w_1024^(+-b2 k1') R, stride 33
//   then TH[1024], TL[1024]  w_n^(+-1024 i) R (* n^-1 inverse), w_n^(+-i) R
//   then RR[1024][2]         ratio w_n^(+-32 c) (plain) and floor(ratio 2^64 / q)
//   then q, qinv
constexpr uint32_t kWOffT1 = kWImg;
constexpr uint32_t kWOffTH = kWOffT1 + kWT1Bytes;
constexpr uint32_t kWOffTL = kWOffTH + 1024 * 8;
constexpr uint32_t kWOffRR = kWOffTL + 1024 * 8;
constexpr uint32_t kWOffQ = kWOffRR + 1024 * 16;
constexpr uint32_t kWBlob = kWOffQ + 16;
static_assert(kWBlob % 16 == 0 && kWOffT1 % 16 == 0 && kWOffTH % 16 == 0, "blob sections stay 16-byte aligned");
// shared memory (from a 1024-aligned base)
constexpr uint32_t kWSmA = 0;                  // operand A / staging, 32 KB
constexpr uint32_t kWSmImg = 32 * 1024;        // image, 64 KB
constexpr uint32_t kWSmT1 = kWSmImg + kWImg;   // level-1 twiddles
constexpr uint32_t kWSmBar = kWSmT1 + kWT1Bytes;
constexpr size_t kWSmem = kWSmBar + 64 + 1024;

struct WArgs {
    const uint64_t* src;    // pass input: units x 2^20 words
    uint64_t* dst;          // pass output
    const uint8_t* consts;  // per limb: forward blob, inverse blob
    uint32_t n_limbs, units, inverse, pass;  // pass 0: A, 1: B
};

__device__ __forceinline__ void werr(uint32_t bit) { atomicOr(&g_wide_error, bit); }
__device__ __forceinline__ void wwait(uint64_t* bar, uint32_t& ph) {
    if (!tc::mbar_wait_bounded(bar, ph)) werr(1u);
    ph ^= 1u;
}

// REDC by 2^64 of v = sum_a 256^a d[a] (d[a] < 2^24): y < q + 2^17, congruent to v 2^-64.
__device__ __forceinline__ uint64_t combine_redc8(const uint32_t* d, uint64_t q, uint64_t qinv) {
    const uint64_t L = tca::mad_wide(d[3], 1u << 24, tca::mad_wide(d[2], 1u << 16, tca::mad_wide(d[1], 256u, d[0])));
    const uint64_t H = tca::mad_wide(d[7], 1u << 24, tca::mad_wide(d[6], 1u << 16, tca::mad_wide(d[5], 256u, d[4])));
    // v = L + H 2^32 = lo + 2^64 hi
    const uint64_t mid = (L >> 32) + (uint64_t)(uint32_t)H;  // < 2^33
    const uint64_t lo = (uint64_t)(uint32_t)L | (mid << 32);
    const uint64_t hi = (H >> 32) + (mid >> 32);
    const uint64_t m = lo * qinv;
    return hi + __umul64hi(m, q) + (lo != 0);
}
// Montgomery product a b 2^-64 mod q for a b < q 2^64, canonical.
__device__ __forceinline__ uint64_t wmul(uint64_t a, uint64_t b, uint64_t q, uint64_t qinv) {
    const uint64_t lo = a * b, hi = __umul64hi(a, b);
    const uint64_t m = lo * qinv;
    const uint64_t r = hi + __umul64hi(m, q) + (lo != 0);
    return r >= q ? r - q : r;
}
__device__ __forceinline__ uint64_t wcanon(uint64_t x, uint64_t q) { return x >= q ? x - q : x; }

// Eight planes each of outputs k .. k + 3 of this thread's lane: TMEM columns
// 8k .. 8k + 31, one load and one wait for four outputs.
__device__ __forceinline__ void ld_planes4(uint32_t taddr, uint32_t k, uint32_t (&d)[32]) {
    tc::ld_32x32b_x32(taddr + 8u * k, d);
    tc::ld_wait();
}

template <uint32_t Pass>
__global__ void __launch_bounds__(kWThreads, 2) wide_pass(const __grid_constant__ WArgs a) {
    extern __shared__ __align__(1024) uint8_t wsm_raw[];
    __shared__ uint32_t s_taddr;
    uint8_t* base = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(wsm_raw) + 1023) & ~uintptr_t(1023));
    uint64_t* bar = reinterpret_cast<uint64_t*>(base + kWSmBar);  // [0] MMA, [1] constants
    const uint32_t tid = threadIdx.x, warp = tid >> 5, lane = tid & 31u, quarter = warp & 3u, half = warp >> 2;
    if (tid == 0) {
        tc::mbar_init(bar, 1);
        tc::mbar_init(bar + 1, 1);
    }
    if (tid < 32) tc::tmem_alloc(&s_taddr, 256);
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t taddr = s_taddr;
    const uint32_t lane_addr = taddr + ((quarter * 32u) << 16);
    const uint32_t sA = tc::smem_u32(base + kWSmA), sImg = tc::smem_u32(base + kWSmImg);
    const uint64_t* T1 = reinterpret_cast<const uint64_t*>(base + kWSmT1);
    uint32_t ph_mma = 0, ph_c = 0;
    int32_t have = -1;  // limb whose constants are in shared memory
    const uint64_t total = (uint64_t)a.units * kWTiles;
    const uint64_t per = (total + gridDim.x - 1) / gridDim.x;
    const uint64_t t0 = per * blockIdx.x, t1 = t0 + per < total ? t0 + per : total;
    for (uint64_t t = t0; t < t1; t++) {
        const uint32_t unit = (uint32_t)(t / kWTiles), tile = (uint32_t)(t % kWTiles);
        const uint32_t limb = unit % a.n_limbs, c0 = tile * kWCols;
        const uint8_t* blob = a.consts + ((size_t)limb * 2 + a.inverse) * kWBlob;
        const uint64_t q = __ldg(reinterpret_cast<const uint64_t*>(blob + kWOffQ));
        const uint64_t qinv = __ldg(reinterpret_cast<const uint64_t*>(blob + kWOffQ) + 1);
        if ((int32_t)limb != have) {  // image and level-1 twiddles of this modulus
            if (tid == 0) {
                const uint64_t pol = tc::l2_policy_evict_last();
                tc::mbar_expect_tx(bar + 1, kWImg + kWT1Bytes);
#pragma unroll
                for (uint32_t k = 0; k < 4; k++)
                    tc::bulk_g2s_hint(base + kWSmImg + k * 16384u, blob + k * 16384u, 16384u, bar + 1, pol);
                tc::bulk_g2s_hint(base + kWSmT1, blob + kWOffT1, kWT1Bytes, bar + 1, pol);
            }
            wwait(bar + 1, ph_c);
            have = (int32_t)limb;
        }
        const uint64_t* src = a.src + ((uint64_t)unit << kWLog);
        uint64_t* dst = a.dst + ((uint64_t)unit << kWLog);
        // ---- level-1 operand: row m = 32 col + b2, K word a2 <- src[(32 a2 + b2) 1024 + c0 + col]
        {
            const uint32_t col = tid & 3u, b2 = (tid >> 2) & 31u, a0 = (tid >> 7) * 16u, m = col * 32u + b2;
            const uint64_t* p = src + (size_t)(32u * a0 + b2) * kWN1 + c0 + col;
            uint64_t v[16];
#pragma unroll
            for (uint32_t i = 0; i < 16; i++) v[i] = __ldcs(p + (size_t)i * 32u * kWN1);
            if (NTTB_CHECK(g_wide_bounds, kBoundsGlobal, c0 + col < kWN1 && (32u * (a0 + 15u) + b2) < kWN1)) {
#pragma unroll
                for (uint32_t i = 0; i < 16; i += 2)
                    *reinterpret_cast<ulonglong2*>(base + kWSmA + tc::sw128_offset(m, 8u * (a0 + i), 128)) =
                        make_ulonglong2(v[i], v[i + 1]);
            }
        }
        tc::fence_proxy_async_smem();
        tc::fence_before_sync();
        __syncthreads();
        if (tid == 0) {
            tc::fence_after_sync();
            tca::issue_k256(taddr, sA, 128, sImg, 256, 256);
            tc::commit(bar);
        }
        __syncwarp();
        wwait(bar, ph_mma);
        tc::fence_after_sync();
        // ---- level-1 epilogue: row m = 32 quarter + lane (col = quarter, b2 = lane),
        // outputs k1' = 16 half + i; z = y * w_1024^(b2 k1') -> level-2 operand, K word b2
        {
            const uint32_t col = quarter, b2 = lane;
#pragma unroll 1
            for (uint32_t i0 = 0; i0 < 16; i0 += 4) {
                uint32_t d[32];
                ld_planes4(lane_addr, 16u * half + i0, d);
#pragma unroll
                for (uint32_t i = 0; i < 4; i++) {
                    const uint32_t k1 = 16u * half + i0 + i;
                    const uint64_t z = wmul(combine_redc8(d + 8 * i, q, qinv), T1[b2 * kWT1Stride + k1], q, qinv);
                    const uint32_t m2 = Pass == 0 ? col * 32u + k1 : k1 * 4u + col;
                    *reinterpret_cast<uint64_t*>(base + kWSmA + tc::sw128_offset(m2, 8u * b2, 128)) = z;
                }
            }
        }
        tc::fence_proxy_async_smem();
        tc::fence_before_sync();  // every level-1 TMEM read is done before level 2 writes TMEM
        __syncthreads();
        if (tid == 0) {
            tc::fence_after_sync();
            tca::issue_k256(taddr, sA, 128, sImg, 256, 256);
            tc::commit(bar);
        }
        __syncwarp();
        wwait(bar, ph_mma);
        tc::fence_after_sync();
        // ---- level-2 epilogue: outputs k2' = 16 half + i of row m2 = 32 quarter + lane
        if (Pass == 0) {
            // col = quarter, k1' = lane; U[c][k] (k = k1' + 32 k2') = y w_n^(c k) (n^-1): staged in
            // row col of a [4][1024] copy over operand A, then bulk-stored to row c of U
            const uint32_t col = quarter, k1 = lane, c = c0 + col;
            const uint64_t* TH = reinterpret_cast<const uint64_t*>(blob + kWOffTH);
            const uint64_t* TL = reinterpret_cast<const uint64_t*>(blob + kWOffTL);
            const uint32_t e = (c * (k1 + 512u * half)) & ((1u << kWLog) - 1u);
            uint64_t tw = wmul(__ldg(TH + (e >> 10)), __ldg(TL + (e & 1023u)), q, qinv);
            const ulonglong2 rr = __ldg(reinterpret_cast<const ulonglong2*>(blob + kWOffRR) + c);
            uint64_t* stage = reinterpret_cast<uint64_t*>(base + kWSmA) + col * kWN1;
#pragma unroll 1
            for (uint32_t i0 = 0; i0 < 16; i0 += 4) {
                uint32_t d[32];
                ld_planes4(lane_addr, 16u * half + i0, d);
                uint64_t y[4];
#pragma unroll
                for (uint32_t i = 0; i < 4; i++) y[i] = combine_redc8(d + 8 * i, q, qinv);
#pragma unroll
                for (uint32_t i = 0; i < 4; i++) {
                    const uint32_t k2 = 16u * half + i0 + i;
                    const uint64_t v = wmul(y[i], tw, q, qinv);
                    (void)NTTB_CHECK(g_wide_bounds, kBoundsResidue, v < q);
                    stage[k1 + 32u * k2] = v;
                    tw = rr.x * tw - __umul64hi(tw, rr.y) * q;  // Shoup step by w_n^(32 c): [0, 2q)
                }
            }
            tc::fence_proxy_async_smem();
            __syncthreads();
            if (tid < kWCols) {
                const uint64_t off = (uint64_t)(c0 + tid) * kWN1;
                if (NTTB_CHECK(g_wide_bounds, kBoundsGlobal, c0 + tid < kWN1)) {
                    asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;" ::"l"(dst + off),
                                 "r"(sA + tid * kWN1 * 8u), "r"(kWN1 * 8u)
                                 : "memory");
                    asm volatile("cp.async.bulk.commit_group;" ::: "memory");
                    // the staging copy is operand A of the next tile: wait until it was read
                    asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
                }
            }
        } else {
            // k1' = 8 quarter + lane / 4, col = lane % 4: X[(k1' + 32 k2') 1024 + c0 + col]
            const uint32_t k1 = 8u * quarter + (lane >> 2), col = lane & 3u;
            uint64_t* o = dst + c0 + col + (size_t)k1 * kWN1;
#pragma unroll 1
            for (uint32_t i0 = 0; i0 < 16; i0 += 4) {
                uint32_t d[32];
                ld_planes4(lane_addr, 16u * half + i0, d);
#pragma unroll
                for (uint32_t i = 0; i < 4; i++) {
                    const uint32_t k2 = 16u * half + i0 + i;
                    const uint64_t y = wcanon(combine_redc8(d + 8 * i, q, qinv), q);
                    (void)NTTB_CHECK(g_wide_bounds, kBoundsResidue, y < q);
                    if (NTTB_CHECK(g_wide_bounds, kBoundsGlobal, k1 + 32u * k2 < kWN1 && c0 + col < kWN1))
                        __stcs(o + (size_t)32u * k2 * kWN1, y);
                }
            }
        }
        tc::fence_before_sync();
        __syncthreads();
    }
    // the last bulk stores have landed before the grid completes
    if (Pass == 0 && tid < kWCols) asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");
    tc::fence_before_sync();
    __syncthreads();
    if (tid < 32) tc::tmem_dealloc(taddr, 256);
}

// ---- host ------------------------------------------------------------------------
struct WideCache {
    uint8_t* d_blob = nullptr;  // per limb: forward blob, inverse blob
};

// B[8k + a][8j + p] = byte a of (256^p 2^64 W[k][j] mod q), K-major SW128, two 128-byte K blocks.
void build_wide_image(uint8_t* img, const std::vector<uint64_t>& W, uint64_t q) {
    std::memset(img, 0, kWImg);
    for (uint32_t k = 0; k < 32; k++)
        for (uint32_t j = 0; j < 32; j++) {
            const uint64_t w = h_to_mont64(W[k * 32 + j], q);  // W 2^64 mod q
            for (uint32_t p = 0; p < 8; p++) {
                const uint64_t v = h_mulmod(w, h_powmod(256, p, q), q);
                for (uint32_t a = 0; a < 8; a++)
                    img[tc::sw128_offset(8 * k + a, 8 * j + p, 256)] = (uint8_t)(v >> (8 * a));
            }
        }
}

int build_wide(const Plan64& p, WideCache* c) {
    const uint32_t nl = p.n_limbs;
    const uint64_t n = 1ull << kWLog;
    std::vector<uint8_t> blob((size_t)kWBlob * 2 * nl);
    for (uint32_t l = 0; l < nl; l++) {
        const LimbHost& H = p.limbs[l];
        const uint64_t q = H.q;
        for (uint32_t dir = 0; dir < 2; dir++) {
            uint8_t* b = blob.data() + ((size_t)l * 2 + dir) * kWBlob;
            const uint64_t w = dir ? H.omega_inv : H.omega;  // primitive n-th root (inverse: its inverse)
            const uint64_t w32 = h_powmod(w, n / 32, q), w1024 = h_powmod(w, n / 1024, q);
            std::vector<uint64_t> W(32 * 32);
            for (uint32_t k = 0; k < 32; k++)
                for (uint32_t j = 0; j < 32; j++) W[k * 32 + j] = h_powmod(w32, (uint64_t)j * k, q);
            build_wide_image(b, W, q);
            uint64_t* T1 = reinterpret_cast<uint64_t*>(b + kWOffT1);
            for (uint32_t b2 = 0; b2 < 32; b2++)
                for (uint32_t k1 = 0; k1 < 32; k1++) T1[b2 * kWT1Stride + k1] = h_to_mont64(h_powmod(w1024, (uint64_t)b2 * k1, q), q);
            uint64_t* TH = reinterpret_cast<uint64_t*>(b + kWOffTH);
            uint64_t* TL = reinterpret_cast<uint64_t*>(b + kWOffTL);
            uint64_t* RR = reinterpret_cast<uint64_t*>(b + kWOffRR);
            const uint64_t scale = dir ? H.n_inv : 1;
            for (uint32_t i = 0; i < 1024; i++) {
                TH[i] = h_to_mont64(h_mulmod(h_powmod(w, 1024ull * i, q), scale, q), q);
                TL[i] = h_to_mont64(h_powmod(w, i, q), q);
                const uint64_t r = h_powmod(w, 32ull * i, q);
                RR[2 * i] = r;
                RR[2 * i + 1] = (uint64_t)(((unsigned __int128)r << 64) / q);
            }
            uint64_t* Q = reinterpret_cast<uint64_t*>(b + kWOffQ);
            Q[0] = q;
            Q[1] = h_neg_inv64(q);
        }
    }
    if (cudaMalloc(&c->d_blob, blob.size()) != cudaSuccess) return 4;
    if (cudaMemcpy(c->d_blob, blob.data(), blob.size(), cudaMemcpyHostToDevice) != cudaSuccess) {
        cudaFree(c->d_blob);
        c->d_blob = nullptr;
        return 3;
    }
    return 0;
}

int wide_grid() {
    static int cached[64] = {};
    int dev = 0;
    cudaGetDevice(&dev);
    if (cached[dev & 63]) return cached[dev & 63];
    // two CTAs per SM need the whole shared-memory carveout
    cudaFuncSetAttribute(wide_pass<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kWSmem);
    cudaFuncSetAttribute(wide_pass<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kWSmem);
    cudaFuncSetAttribute(wide_pass<0>, cudaFuncAttributePreferredSharedMemoryCarveout, (int)cudaSharedmemCarveoutMaxShared);
    cudaFuncSetAttribute(wide_pass<1>, cudaFuncAttributePreferredSharedMemoryCarveout, (int)cudaSharedmemCarveoutMaxShared);
    // The runtime's occupancy answer for a tcgen05 kernel is one CTA per SM;
    // count from the resources instead: TMEM holds two 256-column
    // allocations, and shared memory and registers are checked here.
    cudaFuncAttributes fa{};
    int sms = 0, smem_sm = 0, regs_sm = 0, reserved = 0;
    cudaFuncGetAttributes(&fa, wide_pass<0>);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev);
    cudaDeviceGetAttribute(&regs_sm, cudaDevAttrMaxRegistersPerMultiprocessor, dev);
    cudaDeviceGetAttribute(&reserved, cudaDevAttrReservedSharedMemoryPerBlock, dev);
    cudaGetLastError();
    const size_t per_smem = fa.sharedSizeBytes + kWSmem + (size_t)reserved;
    const size_t per_regs = (size_t)((fa.numRegs * 32 + 255) / 256 * 256) * (kWThreads / 32);
    int fit = 2;
    if (per_smem) fit = std::min<int>(fit, (int)(smem_sm / per_smem));
    if (per_regs) fit = std::min<int>(fit, (int)(regs_sm / per_regs));
    cached[dev & 63] = (fit < 1 ? 1 : fit) * (sms > 0 ? sms : 1);
    return cached[dev & 63];
}

}  // namespace

// Served: n = 2^20, cyclic, every modulus below 2^62 (the wide plans hold 2^31 <= q).
bool wide_tc_serves(const Plan64& p) { return p.log_n == kWLog && !p.negacyclic; }

int wide_tc_transform64(Plan64& p, const void* src, void* dst, uint32_t n_polys, bool inverse, cudaStream_t s) {
    if (!wide_tc_serves(p)) return 1;
    WideCache* c;
    {
        std::lock_guard<std::mutex> lock(p.engine_mu);
        c = static_cast<WideCache*>(p.engine_data);
        if (!c) {
            c = new WideCache();
            if (build_wide(p, c)) {
                delete c;
                return 2;
            }
            p.engine_data = c;
        }
    }
    const uint64_t units = (uint64_t)n_polys * p.n_limbs;
    if (units == 0) return 0;
    if (units > (1u << 20)) return 1;
    // pass A: src -> workspace (transposed); pass B: workspace -> dst (src may equal dst)
    void* ws = plan_workspace(&p.ws, &p.ws_bytes, (size_t)units << (kWLog + 3));
    if (!ws) return 2;
    const int grid = wide_grid();
    const uint64_t tiles = units * kWTiles;
    const int g = (int)(tiles < (uint64_t)grid ? tiles : (uint64_t)grid);
    WArgs a{};
    a.consts = c->d_blob;
    a.n_limbs = p.n_limbs;
    a.units = (uint32_t)units;
    a.inverse = inverse ? 1u : 0u;
    a.src = static_cast<const uint64_t*>(src);
    a.dst = static_cast<uint64_t*>(ws);
    a.pass = 0;
    {
        ProfScope prof("wide_pass_a", s);
        wide_pass<0><<<g, kWThreads, kWSmem, s>>>(a);
        if (launch_rc()) return 2;
    }
    a.src = static_cast<const uint64_t*>(ws);
    a.dst = static_cast<uint64_t*>(dst);
    a.pass = 1;
    ProfScope prof("wide_pass_b", s);
    wide_pass<1><<<g, kWThreads, kWSmem, s>>>(a);
    return launch_rc();
}

void wide_tc_release(Plan64* p) {
    auto* c = static_cast<WideCache*>(p->engine_data);
    if (!c) return;
    if (c->d_blob) cudaFree(c->d_blob);
    delete c;
    p->engine_data = nullptr;
}

uint32_t wide_device_errors(bool clear) {
    uint32_t v = 0;
    cudaMemcpyFromSymbol(&v, g_wide_error, sizeof v);
    if (clear) {
        uint32_t z = 0;
        cudaMemcpyToSymbol(g_wide_error, &z, sizeof z);
    }
    return v;
}

uint32_t wide_bounds_errors(bool clear) {
    uint32_t v = 0;
    cudaMemcpyFromSymbol(&v, g_wide_bounds, sizeof v);
    if (clear) {
        uint32_t z = 0;
        cudaMemcpyToSymbol(g_wide_bounds, &z, sizeof z);
    }
    return v;
}

}  // namespace nttb
