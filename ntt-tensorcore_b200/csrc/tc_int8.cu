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
// N = 2^16 (64 x 64 x 16) runs as two stages; data layout [poly][limb][N]:
//   stage A: for each column b < 1024 of x viewed as [64][1024]:
//              U[d][b] = DFT64(x[.][b])[d] * t_A(b, d)
//            stored transposed (U at b*64 + d): each 128-column tile writes one
//            contiguous 32 KB block.
//   stage B: for each row d, Z = DFT1024(U[d][.]) as DFT64 (over stride 16,
//            twiddle t_B1) then DFT16 (contiguous); X[d + 64 k] = Z[k].  A tile
//            of 8 rows reads and writes exactly the same positions.
// The four-step twiddles are geometric in the output index and are generated
// in the epilogue: each thread walks two interleaved chains (even and odd
// outputs, ratio^2 steps) over its 32 outputs.  Negacyclic twists and n^-1
// are folded into the B matrices and the twiddle tables.
//
// Execution: one persistent launch runs a list of stages (one transform = A, B;
// forward-then-inverse = A, B, A, B).  CTAs draw tiles from a device ticket
// counter in stage order; a tile of stage s for (poly, limb) first waits,
// with a bounded spin, until the 8 tiles of stage s-1 of the same (poly, limb)
// have signalled completion.  Tickets are claimed in order, so every awaited
// tile belongs to a CTA that is already running: no deadlock.  TMEM, the
// mbarriers and the last-used B image stay resident across a CTA's tiles.
//
// CTA shape: kWorkers workers of 256 threads (8 warps) each.  Warp w of a
// worker reads TMEM lanes 32*(w%4).. (its TMEM sub-partition) and output half
// w/4, so each of the 128 vectors of a tile is recombined by two threads.
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "../../include/ntt_b200.h"
#include "engines.hpp"
#include "plan.hpp"
#include "profiler.hpp"
#include "tcgen05.cuh"

namespace nttb {

// bit 0: an mbarrier wait ran out of budget; bit 1: a stage dependency wait did
__device__ uint32_t g_tc_error;

namespace {

constexpr uint32_t kMatBytes64 = 64 * 1024;  // DFT-64 byte-plane image (256 rows x 256 B)
constexpr uint32_t kMatBytes16 = 4 * 1024;   // DFT-16 byte-plane image (64 rows x 64 B)
constexpr uint32_t kThreads = 256;
constexpr uint32_t kTilesPerUnit = 8;        // tiles per (poly, limb) per stage
constexpr uint32_t kWorkers = 1;             // independent tile workers per CTA
// per worker: A 32 KB, B 64 KB, DFT-16 image 4 KB, generator table 2 KB, 3 mbarriers + ticket
constexpr size_t kWorkerSmem = 103 * 1024;
constexpr size_t kSmem = kWorkers * kWorkerSmem + 64 + 1024;

// Device constants of one modulus for one direction.
struct TcLimb {
    uint32_t q, qinv;        // modulus, -q^-1 mod 2^32
    uint32_t one_m, pad_;    // 2^32 mod q
    // stage A twiddle t_A(b, d) = a_st2[2b + h] * a_ratio[b]^(d - 32h), d in [32h, 32h + 32)
    const uint32_t* a_st2;   // 2048 entries (Montgomery form)
    const uint32_t* a_ratio; // 1024 entries
    // stage B level-1 twiddle t_B1(b2, d2) = b_st2[2 b2 + h] * b_ratio[b2]^(d2 - 32h)
    const uint32_t* b_st2;   // 32 entries
    const uint32_t* b_ratio; // 16 entries
    // DFT-64 images are generated in shared memory from byte-transposed tables:
    // gen[a * E + e] packs byte a of (256^p * 2^32 * T[e] mod q) for p = 0..3,
    // with W[k][j] = T[(j * m_k) mod E], m_k = k (E = 64) or 2k + 1 (E = 128).
    const uint32_t* gen_a;   // stage A
    const uint32_t* gen_b1;  // stage B level 1 (E = 64)
    uint32_t e_a, pad2_;     // stage A table length: 64 (cyclic) or 128 (negacyclic forward)
    const uint8_t* mat_b2;   // DFT-16 image for stage B level 2 (4 KB, copied as is)
};

struct Int8Cache {
    uint32_t log_n = 0;
    TcLimb* d_fwd = nullptr;
    TcLimb* d_inv = nullptr;
    void* d_blob = nullptr;
    uint32_t* d_ctr = nullptr;  // ticket + completion counters
    size_t ctr_words = 0;
};

struct StageDesc {
    const uint32_t* src;
    uint32_t* dst;
    const TcLimb* limbs;
    uint32_t kind;  // 0: stage A, 1: stage B
    uint32_t pad_;
};

struct QueueArgs {
    StageDesc st[4];
    uint32_t n_stages, n_limbs, units, total;  // units = polys x limbs; total = tiles
    uint32_t* ctr;                              // [0] ticket, [1 + s * units + u] tiles done
};

// ---- device arithmetic ------------------------------------------------------------
__device__ __forceinline__ uint32_t redc64(uint64_t v, uint32_t q, uint32_t qinv) {
    const uint32_t m = (uint32_t)v * qinv;
    return (uint32_t)((v + (uint64_t)m * q) >> 32);  // [0, 2q) for v < q * 2^32
}
__device__ __forceinline__ uint32_t combine_redc(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3, uint32_t q,
                                                 uint32_t qinv) {
    uint64_t v = (uint64_t)c1 * 256u + c0;
    v += (uint64_t)c2 * 65536u;
    v += (uint64_t)c3 * 16777216u;
    return redc64(v, q, qinv);
}
// a < 2q, b < q -> a*b*2^-32 mod q in [0, 2q)
__device__ __forceinline__ uint32_t mont_lazy(uint32_t a, uint32_t b, uint32_t q, uint32_t qinv) {
    return redc64((uint64_t)a * b, q, qinv);
}
__device__ __forceinline__ uint32_t canon(uint32_t x, uint32_t q) { return x >= q ? x - q : x; }

__device__ __forceinline__ void flag_error(uint32_t bit) { atomicOr(&g_tc_error, bit); }

// Bounded wait until *p >= target (acquire at GPU scope).
__device__ __forceinline__ bool wait_count(const uint32_t* p, uint32_t target) {
    for (uint32_t i = 0; i < (1u << 24); i++) {
        uint32_t v;
        asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
        if (v >= target) return true;
        __nanosleep(64);
    }
    return false;
}
__device__ __forceinline__ void signal_count(uint32_t* p) {
    asm volatile("red.release.gpu.global.add.u32 [%0], 1;" ::"l"(p) : "memory");
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

// The four 16-column planes (a = 0..3 at columns col + 64a) of this thread's TMEM lane.
__device__ __forceinline__ void ld_planes64(uint32_t col, uint32_t (&c0)[16], uint32_t (&c1)[16],
                                            uint32_t (&c2)[16], uint32_t (&c3)[16]) {
    tc::ld_32x32b_x16(col + 0, c0);
    tc::ld_32x32b_x16(col + 64, c1);
    tc::ld_32x32b_x16(col + 128, c2);
    tc::ld_32x32b_x16(col + 192, c3);
    tc::ld_wait();
}

// Shared state of one persistent CTA.
struct Ctx {
    uint8_t* sA;      // 32 KB operand A (stage A / level 1: SW128; level 2: SW64)
    uint8_t* sB;      // 64 KB DFT-64 image
    uint8_t* sB2;     // 4 KB DFT-16 image
    uint32_t* sTab;   // 2 KB generator table
    uint64_t* bar;    // [1] MMA (level 1), [2] MMA (level 2)
    uint32_t taddr;   // TMEM base of this worker (256 columns)
    uint32_t ph_m1, ph_m2;          // mbarrier parities
    const uint32_t* cached;         // generator table of the image currently in sB
    uint32_t tid;                   // thread index within the worker (0..255)
    uint32_t bar_id;                // named barrier of the worker
};

// Barrier over the 256 threads of one worker.
__device__ __forceinline__ void wsync(const Ctx& c) {
    asm volatile("bar.sync %0, %1;" ::"r"(c.bar_id), "r"(kThreads) : "memory");
}

// Stages the generator table (4 * E words) in shared memory.
__device__ __forceinline__ void stage_table(Ctx& c, const uint32_t* gtab, uint32_t E) {
    for (uint32_t i = c.tid; i < 4u * E; i += kThreads) c.sTab[i] = __ldg(gtab + i);
}
// Writes the 256-row x 256-byte SW128 DFT-64 image: thread t owns row
// t = (a, k); its 16-byte chunk cc holds W[k][4cc..4cc+3] byte plane a.
__device__ __forceinline__ void gen_image64(Ctx& c, uint32_t E) {
    const uint32_t t = c.tid, a = t >> 6, k = t & 63u;
    const uint32_t m = (E == 128u) ? 2u * k + 1u : k, mask = E - 1u;
    const uint32_t* ta = c.sTab + a * E;
#pragma unroll
    for (uint32_t cc = 0; cc < 16; cc++) {
        const uint32_t j = 4u * cc;
        uint4 w;
        w.x = ta[(j * m) & mask];
        w.y = ta[((j + 1u) * m) & mask];
        w.z = ta[((j + 2u) * m) & mask];
        w.w = ta[((j + 3u) * m) & mask];
        *reinterpret_cast<uint4*>(c.sB + tc::sw128_offset(t, 16u * cc, 256)) = w;
    }
}

// ---- stage A tile: 128 columns b0.. of one (poly, limb) ------------------------------
__device__ __forceinline__ void tile_a(Ctx& c, const uint32_t* x, uint32_t* out, const TcLimb& L, uint32_t b0) {
    const uint32_t tid = c.tid, warp = tid >> 5, lane = tid & 31u;
    const uint32_t quarter = warp & 3u, half = warp >> 2;
    const uint32_t b_ep = b0 + quarter * 32u + lane;
    const uint32_t q = L.q, qinv = L.qinv;
    const uint32_t ratio = L.a_ratio[b_ep];
    const uint32_t start = L.a_st2[2 * b_ep + half];
    const uint32_t* gtab = L.gen_a;
    const uint32_t E = L.e_a;
    const bool new_img = gtab != c.cached;
    if (new_img) stage_table(c, gtab, E);
    {   // transposed load: vector m = column b0 + m, rows a in [32h, 32h + 32);
        // the image is generated while the loads are in flight
        const uint32_t m = tid & 127u, h = tid >> 7;
        const uint32_t* col = x + b0 + m + (32u * h) * 1024u;
        uint32_t v[32];
#pragma unroll
        for (uint32_t a = 0; a < 32; a++) v[a] = __ldcg(col + a * 1024u);
        if (new_img) {
            wsync(c);
            gen_image64(c, E);
        }
#pragma unroll
        for (uint32_t k = 0; k < 8; k++)
            *reinterpret_cast<uint4*>(c.sA + tc::sw128_offset(m, 128u * h + 16u * k, 128)) =
                make_uint4(v[4 * k], v[4 * k + 1], v[4 * k + 2], v[4 * k + 3]);
    }
    c.cached = gtab;
    tc::fence_proxy_async_smem();
    tc::fence_before_sync();
    wsync(c);
    if (tid == 0) issue_k256(c.taddr, c.sA, 128, c.sB, 256, 256, c.bar + 1);
    __syncwarp();
    const bool ok = tc::mbar_wait_bounded(c.bar + 1, c.ph_m1);
    c.ph_m1 ^= 1u;
    tc::fence_after_sync();
    if (!ok) {
        if (lane == 0) flag_error(1u);
        return;
    }
    const uint32_t r2 = canon(mont_lazy(ratio, ratio, q, qinv), q);
    uint32_t tw_e = start;                                      // d = 32h
    uint32_t tw_o = canon(mont_lazy(tw_e, ratio, q, qinv), q);  // d = 32h + 1
    uint4* orow = reinterpret_cast<uint4*>(out + (uint64_t)b_ep * 64u + 32u * half);
    const uint32_t lane_base = c.taddr + ((quarter * 32u) << 16);
#pragma unroll 1
    for (uint32_t sub = 0; sub < 2; sub++) {
        uint32_t c0[16], c1[16], c2[16], c3[16];
        ld_planes64(lane_base + 32u * half + 16u * sub, c0, c1, c2, c3);
        uint32_t y[16];
#pragma unroll
        for (int i = 0; i < 16; i += 2) {
            const uint32_t te = combine_redc(c0[i], c1[i], c2[i], c3[i], q, qinv);
            const uint32_t to = combine_redc(c0[i + 1], c1[i + 1], c2[i + 1], c3[i + 1], q, qinv);
            y[i] = canon(mont_lazy(te, tw_e, q, qinv), q);
            y[i + 1] = canon(mont_lazy(to, tw_o, q, qinv), q);
            tw_e = canon(mont_lazy(tw_e, r2, q, qinv), q);
            tw_o = canon(mont_lazy(tw_o, r2, q, qinv), q);
        }
#pragma unroll
        for (int i = 0; i < 4; i++)
            orow[sub * 4 + i] = make_uint4(y[4 * i], y[4 * i + 1], y[4 * i + 2], y[4 * i + 3]);
    }
}

// ---- stage B tile: 8 rows d0..d0+7 of U (U[d][b] at b*64 + d) -------------------------
// Level 1: vector m = (r = m & 7, b2 = m >> 3), elements a2 at row position
// a2*16 + b2 -> DFT64 over a2, twiddle t_B1 -> A2 (SW64, rows d2*8 + r,
// K index b2).  Level 2: DFT16 over b2 -> X[d0 + r + 64*d2 + 4096*c2].
__device__ __forceinline__ void tile_b(Ctx& c, const uint32_t* u, uint32_t* out, const TcLimb& L, uint32_t d0) {
    const uint32_t tid = c.tid, warp = tid >> 5, lane = tid & 31u;
    const uint32_t quarter = warp & 3u, h = warp >> 2;
    const uint32_t mv = quarter * 32u + lane, r_ep = mv & 7u, b2_ep = mv >> 3;
    const uint32_t q = L.q, qinv = L.qinv;
    const uint32_t ratio = L.b_ratio[b2_ep];
    const uint32_t start = L.b_st2[2 * b2_ep + h];
    const uint32_t* gtab = L.gen_b1;
    const bool new_img = gtab != c.cached;
    uint4 img2;
    if (new_img) {
        stage_table(c, gtab, 64u);
        img2 = __ldg(reinterpret_cast<const uint4*>(L.mat_b2) + tid);  // 4 KB = 256 x 16 B
    }
    {
        const uint32_t m = tid & 127u, hh = tid >> 7;
        const uint32_t r = m & 7u, b2 = m >> 3;
        const uint32_t* base = u + d0 + r + ((32u * hh) * 16u + b2) * 64u;
        uint32_t v[32];
#pragma unroll
        for (uint32_t a = 0; a < 32; a++) v[a] = __ldcg(base + a * 1024u);
        if (new_img) {
            wsync(c);
            gen_image64(c, 64u);
            reinterpret_cast<uint4*>(c.sB2)[tid] = img2;
        }
#pragma unroll
        for (uint32_t k = 0; k < 8; k++)
            *reinterpret_cast<uint4*>(c.sA + tc::sw128_offset(m, 128u * hh + 16u * k, 128)) =
                make_uint4(v[4 * k], v[4 * k + 1], v[4 * k + 2], v[4 * k + 3]);
    }
    c.cached = gtab;
    tc::fence_proxy_async_smem();
    tc::fence_before_sync();
    wsync(c);
    const uint32_t lane_base = c.taddr + ((quarter * 32u) << 16);
    if (tid == 0) issue_k256(c.taddr, c.sA, 128, c.sB, 256, 256, c.bar + 1);
    __syncwarp();
    bool ok = tc::mbar_wait_bounded(c.bar + 1, c.ph_m1);
    c.ph_m1 ^= 1u;
    tc::fence_after_sync();
    if (ok) {
        // level-1 epilogue -> A2 (SW64 layout, 512 rows x 64 B), overwriting level-1 A
        const uint32_t r2 = canon(mont_lazy(ratio, ratio, q, qinv), q);
        uint32_t tw_e = start;
        uint32_t tw_o = canon(mont_lazy(tw_e, ratio, q, qinv), q);
#pragma unroll 1
        for (uint32_t sub = 0; sub < 2; sub++) {
            uint32_t c0[16], c1[16], c2[16], c3[16];
            ld_planes64(lane_base + 32u * h + 16u * sub, c0, c1, c2, c3);
#pragma unroll
            for (int i = 0; i < 16; i += 2) {
                const uint32_t d2 = 32u * h + 16u * sub + i;
                const uint32_t te = combine_redc(c0[i], c1[i], c2[i], c3[i], q, qinv);
                const uint32_t to = combine_redc(c0[i + 1], c1[i + 1], c2[i + 1], c3[i + 1], q, qinv);
                // [0, 2q) values are exact inputs for level 2
                *reinterpret_cast<uint32_t*>(c.sA + tc::sw64_offset(d2 * 8u + r_ep, 4u * b2_ep)) =
                    mont_lazy(te, tw_e, q, qinv);
                *reinterpret_cast<uint32_t*>(c.sA + tc::sw64_offset((d2 + 1u) * 8u + r_ep, 4u * b2_ep)) =
                    mont_lazy(to, tw_o, q, qinv);
                tw_e = canon(mont_lazy(tw_e, r2, q, qinv), q);
                tw_o = canon(mont_lazy(tw_o, r2, q, qinv), q);
            }
        }
    } else if (lane == 0) {
        flag_error(1u);
    }
    tc::fence_proxy_async_smem();
    tc::fence_before_sync();
    wsync(c);
    if (ok && tid == 0) {
        tc::fence_after_sync();
        const uint32_t idesc = tc::idesc_u8(128, 64);
        const uint32_t a0 = tc::smem_u32(c.sA), bb = tc::smem_u32(c.sB2);
#pragma unroll
        for (uint32_t t = 0; t < 4; t++)
#pragma unroll
            for (uint32_t ks = 0; ks < 2; ks++)
                tc::mma_i8(c.taddr + t * 64u, tc::desc_k_sw64(a0 + t * 8192u + ks * 32u),
                           tc::desc_k_sw64(bb + ks * 32u), idesc, ks > 0);
        tc::commit(c.bar + 2);
    }
    __syncwarp();
    if (!ok) return;
    ok = tc::mbar_wait_bounded(c.bar + 2, c.ph_m2);
    c.ph_m2 ^= 1u;
    tc::fence_after_sync();
    if (!ok) {
        if (lane == 0) flag_error(1u);
        return;
    }
    // level 2: warp pair h handles M-tiles 2h and 2h + 1
#pragma unroll 1
    for (uint32_t tt = 0; tt < 2; tt++) {
        const uint32_t t = 2u * h + tt;
        uint32_t c0[16], c1[16], c2[16], c3[16];
        const uint32_t col = lane_base + t * 64u;
        tc::ld_32x32b_x16(col + 0, c0);
        tc::ld_32x32b_x16(col + 16, c1);
        tc::ld_32x32b_x16(col + 32, c2);
        tc::ld_32x32b_x16(col + 48, c3);
        tc::ld_wait();
        const uint32_t row2 = t * 128u + quarter * 32u + lane;
        const uint32_t d2 = row2 >> 3, rr = row2 & 7u;
        uint32_t* o = out + d0 + rr + 64u * d2;
#pragma unroll
        for (int k = 0; k < 16; k++) o[4096u * k] = canon(combine_redc(c0[k], c1[k], c2[k], c3[k], q, qinv), q);
    }
}

// ---- persistent work-queue kernel -------------------------------------------------------
// One CTA per SM holds kWorkers independent tile workers of 256 threads each
// (own shared-memory region, TMEM column range, mbarriers, named barrier and
// ticket stream), so that tiles in different phases overlap on the SM.
__global__ void __launch_bounds__(kThreads * kWorkers, 1) int8_queue_n16(const __grid_constant__ QueueArgs args) {
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    uint8_t* base = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    const uint32_t worker = threadIdx.x / kThreads;
    uint8_t* smem = base + worker * kWorkerSmem;
    Ctx c;
    c.sA = smem;
    c.sB = smem + 32768;
    c.sB2 = smem + 32768 + kMatBytes64;
    c.sTab = reinterpret_cast<uint32_t*>(c.sB2 + kMatBytes16);
    c.bar = reinterpret_cast<uint64_t*>(c.sTab + 512);
    c.tid = threadIdx.x % kThreads;
    c.bar_id = 1 + worker;
    uint32_t* slot = reinterpret_cast<uint32_t*>(base + kWorkers * kWorkerSmem);  // CTA-wide TMEM base
    uint32_t* s_ticket = reinterpret_cast<uint32_t*>(c.bar + 3);
    const uint32_t tid = c.tid;
    if (threadIdx.x < 32) tc::tmem_alloc(slot, 256 * kWorkers);
    if (tid == 0) {
        tc::mbar_init(c.bar + 1, 1);
        tc::mbar_init(c.bar + 2, 1);
    }
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    c.taddr = *slot + worker * 256u;
    c.ph_m1 = c.ph_m2 = 0;
    c.cached = nullptr;
    for (;;) {
        if (tid == 0) *s_ticket = atomicAdd(args.ctr, 1u);
        wsync(c);
        const uint32_t t = *s_ticket;
        if (t >= args.total) break;
        const uint32_t per_stage = args.units * kTilesPerUnit;
        const uint32_t s = t / per_stage, rem = t - s * per_stage;
        const uint32_t unit = rem / kTilesPerUnit, tile = rem % kTilesPerUnit;
        const uint32_t limb = unit % args.n_limbs;
        const StageDesc& S = args.st[s];
        if (s > 0 && tid == 0 && !wait_count(args.ctr + 1 + (s - 1) * args.units + unit, kTilesPerUnit))
            flag_error(2u);
        wsync(c);
        const uint64_t off = (uint64_t)unit << 16;
        if (S.kind == 0) tile_a(c, S.src + off, S.dst + off, S.limbs[limb], tile * 128u);
        else tile_b(c, S.src + off, S.dst + off, S.limbs[limb], tile * 8u);
        __threadfence();
        tc::fence_before_sync();
        wsync(c);
        if (tid == 0) signal_count(args.ctr + 1 + s * args.units + unit);
    }
    tc::fence_before_sync();
    __syncthreads();
    if (threadIdx.x < 32) tc::tmem_dealloc(*slot, 256 * kWorkers);
}

// ---- host: tables and byte-plane images ------------------------------------------------
// The DFT-64 operand B is B[(a, k)][(j, p)] = byte a of (256^p * 2^32 * W[k][j] mod q),
// K-major SW128, 256 rows, two 128-byte K blocks; gen_image64 writes it on the device.
// Byte-transposed generator table for DFT-64 images built on the device:
// g[a*E + e] packs, for p = 0..3 (byte p), byte a of (256^p * 2^32 * root^e mod q).
void build_gen(uint32_t* g, uint64_t root, uint32_t E, uint64_t q) {
    uint64_t t = 1;
    for (uint32_t e = 0; e < E; e++) {
        uint32_t packed[4] = {0, 0, 0, 0};
        for (uint32_t p = 0; p < 4; p++) {
            const uint64_t v = h_mulmod(h_to_mont32(t, q), (1ull << (8 * p)) % q, q);
            for (uint32_t a = 0; a < 4; a++) packed[a] |= (uint32_t)((v >> (8 * a)) & 255u) << (8 * p);
        }
        for (uint32_t a = 0; a < 4; a++) g[a * E + e] = packed[a];
        t = h_mulmod(t, root, q);
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
            uint64_t v = h_powmod(root, (uint64_t)j * k, q);
            v = h_mulmod(v, h_powmod(row_twist, k, q), q);
            v = h_mulmod(v, h_powmod(col_twist, j, q), q);
            W[(size_t)k * L + j] = h_mulmod(v, scale, q);
        }
    return W;
}

// Twiddle tables of one direction: a_st2 (2048), a_ratio (1024), b_st2 (32), b_ratio (16).
constexpr size_t kTabWords = 2048 + 1024 + 32 + 16;

void fill_tables(uint32_t* t, uint64_t q, const uint64_t* start_a, const uint64_t* ratio_a, const uint64_t* ratio_b) {
    for (uint32_t b = 0; b < 1024; b++) {
        t[2 * b] = h_to_mont32(start_a[b], q);
        t[2 * b + 1] = h_to_mont32(h_mulmod(start_a[b], h_powmod(ratio_a[b], 32, q), q), q);
        t[2048 + b] = h_to_mont32(ratio_a[b], q);
    }
    for (uint32_t b2 = 0; b2 < 16; b2++) {
        t[3072 + 2 * b2] = h_to_mont32(1, q);
        t[3072 + 2 * b2 + 1] = h_to_mont32(h_powmod(ratio_b[b2], 32, q), q);
        t[3104 + b2] = h_to_mont32(ratio_b[b2], q);
    }
}

int build_cache(Plan32& p, Int8Cache* c) {
    const uint32_t n = p.n, nl = p.n_limbs;
    // blob layout per limb: 4 generator tables (512 words each: stage A / B1,
    // forward / inverse) + 2 DFT-16 images + 2 twiddle tables
    const size_t kGen = 4 * 512 * 4;
    const size_t per_limb = kGen + 2 * (size_t)kMatBytes16 + 2 * kTabWords * 4;
    std::vector<uint8_t> blob(per_limb * nl);
    uint8_t* d_blob = nullptr;
    if (cudaMalloc(&d_blob, blob.size()) != cudaSuccess) return 4;
    std::vector<TcLimb> fwd(nl), inv(nl);
    std::vector<uint64_t> st(1024), ra(1024), rb(16);
    for (uint32_t l = 0; l < nl; l++) {
        const LimbHost& H = p.limbs[l];
        const uint64_t q = H.q;
        uint8_t* h = blob.data() + per_limb * l;
        uint8_t* d = d_blob + per_limb * l;
        const uint64_t w = H.omega, wi = H.omega_inv;
        const uint64_t w64 = h_powmod(w, n / 64, q), w64i = h_powmod(wi, n / 64, q);
        const uint64_t w16 = h_powmod(w, n / 16, q), w16i = h_powmod(wi, n / 16, q);
        // stage A forward: the negacyclic twist psi^(a * n/64) on the input index
        // makes W[k][j] = psi_128^(j (2k + 1)) (table of 128 powers)
        uint32_t* gen = reinterpret_cast<uint32_t*>(h);
        const uint32_t e_af = p.negacyclic ? 128u : 64u;
        build_gen(gen + 0 * 512, p.negacyclic ? h_powmod(H.psi, n / 64, q) : w64, e_af, q);  // A forward
        build_gen(gen + 1 * 512, w64i, 64, q);                                                // A inverse
        build_gen(gen + 2 * 512, w64, 64, q);                                                 // B1 forward
        build_gen(gen + 3 * 512, w64i, 64, q);                                                // B1 inverse
        // stage B level 2 inverse: n^-1 (and psi^-(4096 c2)) folded on the output index
        std::vector<uint64_t> B2f = dft_matrix(16, w16, q);
        std::vector<uint64_t> B2i = p.negacyclic ? dft_matrix(16, w16i, q, h_powmod(H.psi_inv, 4096, q), 1, H.n_inv)
                                                 : dft_matrix(16, w16i, q, 1, 1, H.n_inv);
        build_image16(h + kGen, B2f, q);
        build_image16(h + kGen + kMatBytes16, B2i, q);
        uint32_t* tab = reinterpret_cast<uint32_t*>(h + kGen + 2 * kMatBytes16);
        uint32_t* dtab = reinterpret_cast<uint32_t*>(d + kGen + 2 * kMatBytes16);
        const uint32_t* dgen = reinterpret_cast<const uint32_t*>(d);
        // forward: t_A(b, d) = psi^b (negacyclic) * omega^(b d); t_B1(b2, d2) = omega^(64 b2 d2)
        for (uint32_t b = 0; b < 1024; b++) {
            st[b] = p.negacyclic ? h_powmod(H.psi, b, q) : 1;
            ra[b] = h_powmod(w, b, q);
        }
        for (uint32_t b2 = 0; b2 < 16; b2++) rb[b2] = h_powmod(w, 64ull * b2, q);
        fill_tables(tab, q, st.data(), ra.data(), rb.data());
        // inverse: t_A(b, d) = omega^-(b d) (* psi^-d); t_B1 = omega^-(64 b2 d2) (* psi^-(64 d2))
        for (uint32_t b = 0; b < 1024; b++) {
            st[b] = 1;
            ra[b] = h_powmod(wi, b, q);
            if (p.negacyclic) ra[b] = h_mulmod(ra[b], H.psi_inv, q);
        }
        for (uint32_t b2 = 0; b2 < 16; b2++) {
            rb[b2] = h_powmod(wi, 64ull * b2, q);
            if (p.negacyclic) rb[b2] = h_mulmod(rb[b2], h_powmod(H.psi_inv, 64, q), q);
        }
        fill_tables(tab + kTabWords, q, st.data(), ra.data(), rb.data());
        TcLimb f{}, v{};
        f.q = v.q = (uint32_t)q;
        f.qinv = v.qinv = h_neg_inv32((uint32_t)q);
        f.one_m = v.one_m = h_to_mont32(1, q);
        f.a_st2 = dtab;
        f.a_ratio = dtab + 2048;
        f.b_st2 = dtab + 3072;
        f.b_ratio = dtab + 3104;
        v.a_st2 = dtab + kTabWords;
        v.a_ratio = dtab + kTabWords + 2048;
        v.b_st2 = dtab + kTabWords + 3072;
        v.b_ratio = dtab + kTabWords + 3104;
        f.gen_a = dgen;
        f.e_a = e_af;
        v.gen_a = dgen + 512;
        v.e_a = 64;
        f.gen_b1 = dgen + 2 * 512;
        v.gen_b1 = dgen + 3 * 512;
        f.mat_b2 = d + kGen;
        v.mat_b2 = d + kGen + kMatBytes16;
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

Int8Cache* get_cache(Plan32& p) {
    auto* c = reinterpret_cast<Int8Cache*>(p.engine_data[1]);
    if (c) return c;
    c = new Int8Cache();
    if (build_cache(p, c)) {
        delete c;
        return nullptr;
    }
    p.engine_data[1] = c;
    static bool attr = false;
    if (!attr) {
        cudaFuncSetAttribute(int8_queue_n16, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmem);
        // two CTAs of ~103 KB per SM need the largest shared-memory carveout
        cudaFuncSetAttribute(int8_queue_n16, cudaFuncAttributePreferredSharedMemoryCarveout,
                             (int)cudaSharedmemCarveoutMaxShared);
        attr = true;
    }
    return c;
}

int grid_size(uint32_t total) {
    static int max_blocks = 0;
    if (!max_blocks) {
        int dev = 0, sms = 0, occ = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, int8_queue_n16, kThreads * kWorkers, kSmem);
        // launch-shape knob: CTAs per SM (clamped to the occupancy limit)
        if (const char* e = std::getenv("NTT_B200_INT8_CTAS_PER_SM")) {
            const int want = std::atoi(e);
            if (want > 0 && want < occ) occ = want;
        }
        max_blocks = sms * (occ > 0 ? occ : 1);
    }
    return (int)((uint32_t)max_blocks < total ? (uint32_t)max_blocks : total);
}

// Launches the stage list; counters live in the cache and are cleared on the stream.
int launch_queue(Int8Cache* c, QueueArgs& q, cudaStream_t s) {
    const size_t words = 1 + (size_t)q.n_stages * q.units;
    if (c->ctr_words < words) {
        if (c->d_ctr) cudaFree(c->d_ctr);
        c->d_ctr = nullptr;
        c->ctr_words = 0;
        if (cudaMalloc(&c->d_ctr, words * 4) != cudaSuccess) return 2;
        c->ctr_words = words;
    }
    q.ctr = c->d_ctr;
    q.total = q.n_stages * q.units * kTilesPerUnit;
    if (cudaMemsetAsync(c->d_ctr, 0, words * 4, s) != cudaSuccess) return 2;
    ProfScope prof(q.n_stages == 2 ? "int8_queue_n16_x2" : "int8_queue_n16_x4", s);
    int8_queue_n16<<<grid_size((q.total + kWorkers - 1) / kWorkers), kThreads * kWorkers, kSmem, s>>>(q);
    return cudaGetLastError() == cudaSuccess ? 0 : 2;
}

}  // namespace

bool int8_serves(const Plan32& p, bool src_u64) { return !src_u64 && p.log_n == 16; }

int int8_transform32(Plan32& p, const void* src, void* dst, bool src_u64, uint32_t n_polys, bool inverse,
                     cudaStream_t s) {
    if (!int8_serves(p, src_u64)) return 1;
    if ((uint64_t)n_polys * p.n_limbs > (1u << 24)) return 1;
    Int8Cache* c = get_cache(p);
    if (!c) return 2;
    const uint32_t* in = static_cast<const uint32_t*>(src);
    uint32_t* out = static_cast<uint32_t*>(dst);
    uint32_t* mid = out;
    if (src == dst) {  // stage A cannot run in place: stage it in the plan's workspace
        mid = static_cast<uint32_t*>(plan_workspace(&p.ws, &p.ws_bytes, (size_t)n_polys * p.n_limbs * p.n * 4));
        if (!mid) return 2;
    }
    const TcLimb* limbs = inverse ? c->d_inv : c->d_fwd;
    QueueArgs q{};
    q.st[0] = {in, mid, limbs, 0, 0};
    q.st[1] = {mid, out, limbs, 1, 0};
    q.n_stages = 2;
    q.n_limbs = p.n_limbs;
    q.units = n_polys * p.n_limbs;
    return launch_queue(c, q, s);
}

int int8_forward_inverse32(Plan32& p, uint32_t* data, uint32_t n_polys, cudaStream_t s) {
    if (!int8_serves(p, false)) return 1;
    if ((uint64_t)n_polys * p.n_limbs > (1u << 24)) return 1;
    Int8Cache* c = get_cache(p);
    if (!c) return 2;
    uint32_t* ws = static_cast<uint32_t*>(plan_workspace(&p.ws, &p.ws_bytes, (size_t)n_polys * p.n_limbs * p.n * 4));
    if (!ws) return 2;
    QueueArgs q{};
    q.st[0] = {data, ws, c->d_fwd, 0, 0};
    q.st[1] = {ws, data, c->d_fwd, 1, 0};
    q.st[2] = {data, ws, c->d_inv, 0, 0};
    q.st[3] = {ws, data, c->d_inv, 1, 0};
    q.n_stages = 4;
    q.n_limbs = p.n_limbs;
    q.units = n_polys * p.n_limbs;
    return launch_queue(c, q, s);
}

void int8_release(Plan32* p) {
    auto* c = reinterpret_cast<Int8Cache*>(p->engine_data[1]);
    if (!c) return;
    if (c->d_fwd) cudaFree(c->d_fwd);
    if (c->d_blob) cudaFree(c->d_blob);
    if (c->d_ctr) cudaFree(c->d_ctr);
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
