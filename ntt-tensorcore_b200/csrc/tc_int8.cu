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
// N = 2^16 (64 x 64 x 16) runs as two stages over x viewed as [64][1024]:
//   stage A: for each column b, U[d][b] = DFT64(x[.][b])[d] * t_A(b, d).
//   stage B: for each row d, Z = DFT1024(U[d][.]) as DFT64 over a2 (b = 16 a2
//            + b2, twiddle t_B1(b2, d2)) then DFT16 over b2; X[d + 64 k] = Z[k].
// The four-step twiddles are geometric in the output index and are generated
// in the epilogue: each thread walks two interleaved chains (even and odd
// outputs, ratio^2 steps) over its 32 outputs.  Negacyclic twists and n^-1
// are folded into the B matrices and the twiddle tables.  The DFT-64 images
// (rows ordered (k / 32, a, k % 32) so that each half of the outputs is one
// N = 128 MMA) are precomputed per modulus and bulk-copied into shared
// memory while the previous stage's epilogue runs.
//
// Execution: a cluster of 4 CTAs (one per SM, 512 threads = two 128-vector
// tiles each) owns one polynomial of one limb -- 256 KB, held in the
// cluster's distributed shared memory for all stages.  The unit is read from
// HBM once by stage A of the first transform and written once by stage B of
// the last.  In between, the four-step transpose is a DSMEM exchange: each
// epilogue stages its outputs in its own (now free) operand buffer, laid out
// exactly as the 1 KB pieces of the receivers' next operand buffers, and 64
// bulk copies per CTA move the pieces, each completing its bytes on the
// receiver's mbarrier.  A piece for CTA P is staged in the region that P
// itself overwrites next, so staging never races an outgoing copy.
// Forward-then-inverse runs four stages on chip.  Clusters are persistent
// over (poly, limb) units.
//
// Operand layouts (K-major, two 128-vector tiles per buffer):
//   stage A (buffer 0, SW128): row m of tile t holds column b = 128 t + beta(m)
//     (beta permutes rows so that each source CTA of the B->A exchange owns
//     whole 8-row atoms), K word a = row of x.
//   stage B level 1 (buffer 1, SW64, four 64-byte K blocks): row m' = b2 + 16 r
//     (row d = 8 t + r), K word a2 in block a2 / 16 = the source CTA.
//   stage B level 2 (in place of level 1, SW64): row r + 8 (d2 / 16) + 32 (d2 % 16),
//     K word b2.
//
// CTA layout: threads 0..511 run the epilogues, thread 512 (the last warp)
// issues the four DFT-64 MMAs of a stage and fetches the next stage's image,
// so no epilogue warp stalls behind the MMA queue.  Tile w = threadIdx.x / 256
// of CTA rank c is tile 2c + w of a stage (columns 128(2c+w).. in stage A, rows 8(2c+w).. in stage B).  Warp
// v = (threadIdx.x / 32) % 8 of a tile reads TMEM lanes 32*(v%4).. (its TMEM
// sub-partition) and output half v/4, so each vector is recombined by two
// threads.
#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "../../include/ntt_b200.h"
#include "bounds.cuh"
#include "engines.hpp"
#include "plan.hpp"
#include "profiler.hpp"
#include "tc_arith.cuh"
#include "tcgen05.cuh"

namespace nttb {

// bit 0: an mbarrier wait on a local MMA or copy ran out of budget;
// bit 1: a wait on another CTA of the cluster did
__device__ uint32_t g_tc_error;
// NTT_DEBUG_BOUNDS build: failed range checks (bounds.cuh bits)
__device__ uint32_t g_tc_bounds;

// NTT_PHASE_PROFILE build (build.py --phase-profile): clock() cycles spent
// by the epilogue warps in each phase of a stage, summed over warps (lane 0
// of each warp adds its own), plus per-CTA totals; read and cleared by
// nttb_phase_profile.  The release build compiles every probe away.
//   0 waiting for the stage's MMA   1 TMEM loads      2 gates before staging stores
//   3 part barriers + piece sends   4 level-2 MMA     5 end-of-stage barrier
//   6 whole stages                  7 CTA lifetime    8 CTA start-up   9 CTAs
__device__ unsigned long long g_phase[16];
#ifdef NTT_PHASE_PROFILE
#define PHASE_T0 uint32_t phase_t0_ = (uint32_t)clock()
#define PHASE_ADD(cat)                                                                       \
    do {                                                                                     \
        const uint32_t phase_t1_ = (uint32_t)clock();                                        \
        if ((threadIdx.x & 31u) == 0) atomicAdd(c.phase + (cat), phase_t1_ - phase_t0_);     \
        phase_t0_ = phase_t1_;                                                               \
    } while (0)
#else
#define PHASE_T0 (void)0
#define PHASE_ADD(cat) (void)0
#endif

namespace {

using namespace tca;

constexpr uint32_t kMatBytes64 = 64 * 1024;  // DFT-64 byte-plane image (256 rows x 256 B)
constexpr uint32_t kMatBytes16 = 4 * 1024;   // DFT-16 byte-plane image (64 rows x 64 B)
constexpr uint32_t kTileBytes = 32 * 1024;   // one 128-vector operand tile (SW128, 256 B rows)
constexpr uint32_t kClCtas = 4;              // CTAs per cluster
constexpr uint32_t kEpiThreads = 512;        // two tiles of 256 epilogue threads per CTA
constexpr uint32_t kClThreads = kEpiThreads + 32;  // + the warp that issues the DFT-64 MMAs and image copies
// shared memory map (offsets from a 1024-aligned base)
constexpr uint32_t kOffBuf0 = 0;                        // operand buffer 0: 2 tiles
constexpr uint32_t kOffBuf1 = 2 * kTileBytes;           // operand buffer 1: 2 tiles
constexpr uint32_t kOffImg = 4 * kTileBytes;            // DFT-64 image
constexpr uint32_t kOffImg16 = kOffImg + kMatBytes64;   // DFT-16 images: forward, inverse
constexpr uint32_t kOffTB1 = kOffImg16 + 2 * kMatBytes16;  // stage B level-1 twiddles: forward, inverse
constexpr uint32_t kTB1Stride = 68;                         // words per b2 row (64 twiddles + padding)
constexpr uint32_t kTB1Bytes = 16 * kTB1Stride * 4;         // one array of one direction: 4352 B
constexpr uint32_t kTB1Dir = 2 * kTB1Bytes;                 // a direction's twiddles t, then their quotients t'
constexpr uint32_t kOffBar = kOffTB1 + 2 * kTB1Dir;
constexpr size_t kClSmem = kOffBar + 256 + 1024;
static_assert(kClSmem <= 232448, "one CTA's dynamic shared memory (227 KB on sm_100)");
constexpr uint32_t kPiece = 1024;            // DSMEM exchange granule
constexpr uint32_t kBufBytes = 2 * kTileBytes;
// per-limb device blob: DFT-16 images (8 KB), 3 DFT-64 images, twiddle tables
constexpr uint32_t kImgSlots = 3;            // 0: stage A forward, 1: inverse (A and B), 2: stage B forward
constexpr uint32_t kBlobImg = 2 * kMatBytes16;
// twiddle table of one direction (words): a_st2[2048] a_ratio[1024] q qinv
// (pad to 16 bytes) a_step[2048] b1[16][68] b1s[16][68]; the forward table, then the
// inverse
//   stage A:  t_A(b, d) = a_st2[2b + h] * a_ratio[b]^(d - 32h),   d in [32h, 32h + 32)
//             (Montgomery form); a_step = (ratio^2 mod q, floor(ratio^2 * 2^32 / q))
//             in plain form, the Shoup operands of the twiddle chains' step
//             (every second output);
//   stage B1: b1[b2][d2] = t_B1(b2, d2) = b_ratio[b2]^d2 (plain form,
//             canonical), then b1s[b2][d2] = floor(t_B1 * 2^32 / q), the
//             operands of a Shoup product (three single-width multiplies; a
//             Montgomery product by a table entry takes more of the integer
//             multiply pipe: 1.43e12 against 1.83e12 outputs/s for this
//             epilogue's arithmetic on the whole GPU); rows b2 padded to 68
//             words so that 16-byte loads of neighbouring rows hit distinct
//             banks; bulk-copied into shared memory with the unit's
//             constants, so that the epilogue reads its twiddles instead of
//             walking chains.
constexpr uint32_t kTabAst = 0, kTabArat = 2048, kTabQ = 3072, kTabAstep = 3076, kTabB1 = 5124;
constexpr uint32_t kTabWords = kTabB1 + 2 * 16 * kTB1Stride;
static_assert((kTabB1 * 4) % 16 == 0 && (kTabWords * 4) % 16 == 0, "bulk-copied table rows stay 16-byte aligned");
constexpr uint32_t kBlobTab = kBlobImg + kImgSlots * kMatBytes64;
constexpr uint32_t kBlobBytes = kBlobTab + 2 * kTabWords * 4;
static_assert(kBlobBytes % 16 == 0, "per-limb blobs must stay 16-byte aligned");

struct Int8Cache {
    uint32_t log_n = 0;
    uint8_t* d_blob = nullptr;
    size_t per_limb = 0;
    bool negacyclic = false;
    bool lazy = false;  // every modulus below 2^31 - 2^16: unreduced twiddle chains
};

// One stage of the on-chip stage list.
struct ClStage {
    uint32_t dir;         // 0: forward, 1: inverse (twiddle table of the stage)
    uint32_t kind;        // 0: stage A (columns), 1: stage B (rows)
    uint32_t img;         // DFT-64 image slot of the stage
    uint32_t img16;       // stage B: DFT-16 image 0 (forward) or 1 (inverse)
    uint32_t pad_;
};

struct ClArgs {
    ClStage st[4];
    const void* src;        // [units][2^16] words of 4 or 8 bytes (words64)
    void* dst;              // the same layout, may equal src
    const uint8_t* consts;  // per limb: 2 DFT-16 images, 3 DFT-64 images
    uint64_t const_stride;
    uint32_t n_stages, n_limbs, units, words64;  // words64: uint64 words (residues < 2^31)
};

__device__ __forceinline__ void flag_error(uint32_t bit) { atomicOr(&g_tc_error, bit); }

// Same contraction with operand A in the stage B level-1 layout: SW64, four
// 64-byte K blocks of `a_rows` rows each.
__device__ __forceinline__ void issue_k256_a64(uint32_t tmem, uint32_t a0, uint32_t a_rows, uint32_t b0,
                                               uint32_t b_rows, uint32_t N) {
    const uint32_t idesc = tc::idesc_u8(128, N);
#pragma unroll
    for (uint32_t ks = 0; ks < 8; ks++) {
        const uint32_t ka = a0 + (ks >> 1) * a_rows * 64u + (ks & 1u) * 32u;
        const uint32_t kb = b0 + (ks >> 2) * b_rows * 128u + (ks & 3u) * 32u;
        tc::mma_i8(tmem, tc::desc_k_sw64(ka), tc::desc_k_sw128(kb), idesc, ks > 0);
    }
}

// Column offset (within a 128-column tile) held by stage A operand row m:
// bits [6][5][4:3][2:0] of m -> bits [6][3][5:4][2:0].
__device__ __forceinline__ uint32_t beta(uint32_t m) {
    return ((m >> 3) & 3u) * 16u + ((m >> 5) & 1u) * 8u + (m & 7u) + (m >> 6) * 64u;
}

// Shared state of one CTA.
struct Cl {
    uint8_t* base;
    uint32_t rank, tid, w, wt;  // CTA rank in the cluster, thread, tile, thread within tile
    uint32_t quarter, h, lane;  // TMEM sub-partition, output half, lane of this thread's warp
    uint32_t taddr;             // TMEM base (512 columns: tile w at + 256 w)
    uint64_t* bar;
#ifdef NTT_PHASE_PROFILE
    uint32_t* phase;            // shared-memory phase counters
#endif
};
// Barriers (shared memory, after the images):
//   [0, 1]  MMA of tile 0 / 1 (N = 256), issued in that order (N = 128
//           halves committed apart let half the threads start earlier, but
//           the tensor pipe runs an N = 128 MMA in the time of an N = 256 one:
//           slower overall)
//   [4, 5]  level-2 MMA of tile 0 / 1
//   [6]     per-unit constants (DFT-16 images, stage B level-1 twiddles, first DFT-64 image)
//   [7]     DFT-64 image of the next stage
//   [8, 9]  buffer 0 / 1 inbox: one arrival (the owner arming the 64 KB its
//           four senders complete)
//   [10]    unit done: one arrival per CTA of the cluster
constexpr uint32_t kBarMma = 0, kBarMma2 = 4, kBarConst = 6, kBarImg = 7, kBarIn0 = 8, kBarIn1 = 9, kBarUnit = 10;

__device__ __forceinline__ uint32_t buf_addr(const Cl& c, uint32_t which) {
    return tc::smem_u32(c.base + (which ? kOffBuf1 : kOffBuf0));
}

// Bounded waits; the phase bit is advanced by the caller.
__device__ __forceinline__ void wait_parity(uint64_t* bar, uint32_t ph) {
    if (!tc::mbar_wait_bounded(bar, ph)) flag_error(1u);
}
__device__ __forceinline__ void wait_local(uint64_t* bar, uint32_t& ph) {
    wait_parity(bar, ph);
    ph ^= 1u;
}
__device__ __forceinline__ void wait_cluster(uint64_t* bar, uint32_t& ph) {
    if (!tc::mbar_wait_cluster_bounded(bar, ph)) flag_error(2u);
    ph ^= 1u;
}
// One arrival on barrier `idx` of every CTA of the cluster (thread 0 only).
__device__ __forceinline__ void arrive_all(const Cl& c, uint32_t idx) {
    const uint32_t a = tc::smem_u32(c.bar + idx);
#pragma unroll
    for (uint32_t r = 0; r < kClCtas; r++) tc::arrive_cluster(tc::mapa(a, r));
}
// DFT-64 image `slot` of the unit's limb -> shared memory (one thread), 4 x 16 KB.
// The per-limb constants are re-read by every launch while the residues
// stream through the L2 (loaded evict-first): they are loaded evict-last.
__device__ __forceinline__ void copy_image(const Cl& c, const uint8_t* limb_blob, uint32_t slot, uint64_t* bar) {
    const uint8_t* src = limb_blob + kBlobImg + (size_t)slot * kMatBytes64;
    const uint64_t pol = tc::l2_policy_evict_last();
#pragma unroll
    for (uint32_t k = 0; k < 4; k++)
        tc::bulk_g2s_hint(c.base + kOffImg + k * 16384u, src + k * 16384u, 16384u, bar, pol);
}

// Stage A operand of tile w from HBM: row m = column b = 128(2c+w) + beta(m),
// elements a (rows of x) -> buffer 0, K-major SW128.
template <class W>
__device__ __forceinline__ void load_columns(const Cl& c, const W* x) {
    const uint32_t m = c.wt & 127u, hh = c.wt >> 7;
    const uint32_t off0 = 128u * (2u * c.rank + c.w) + beta(m) + (32u * hh) * 1024u;
    const W* col = x + off0;
    uint32_t v[32];
    const bool ok = NTTB_CHECK(g_tc_bounds, kBoundsGlobal, c.rank < kClCtas && off0 + 31u * 1024u < 65536u);
#pragma unroll
    for (uint32_t a = 0; a < 32; a++) v[a] = ok ? (uint32_t)__ldcs(col + a * 1024u) : 0u;
    uint8_t* t = c.base + kOffBuf0 + c.w * kTileBytes;
#pragma unroll
    for (uint32_t k = 0; k < 8; k++)
        *reinterpret_cast<uint4*>(t + tc::sw128_offset(m, 128u * hh + 16u * k, 128)) =
            make_uint4(v[4 * k], v[4 * k + 1], v[4 * k + 2], v[4 * k + 3]);
}

// TMEM columns of this thread's lane for its tile and output half.
__device__ __forceinline__ uint32_t lane_cols(const Cl& c) {
    return c.taddr + c.w * 256u + c.h * 128u + ((c.quarter * 32u) << 16);
}

// The epilogues run in two parts of 16 outputs.  `gate` runs between the
// first part's arithmetic and its stores: it waits until the shared memory
// the stores overwrite is no longer read by the tensor core.
//
// Twiddle chains: each step is a Shoup product, in [0, 2q) for any input
// below 2^32.  A REDC of the byte-plane sum (below 2^48) returns
// y < q + 2^16, so with every modulus below 2^31 - 2^16 the product of y and
// a twiddle in [0, 2q) stays below q * 2^32 and the Montgomery product is
// exact: the chain need not be reduced to [0, q) (Lazy).  Other moduli
// reduce every twiddle.
template <bool Lazy>
__device__ __forceinline__ uint32_t tw_norm(uint32_t t, uint32_t q) {
    return Lazy ? t : canon(t, q);
}

// Stage A epilogue: y_d * t_A(b, d) in [0, 2q) for outputs d = 32h + i,
// staged in buffer 0 for the A->B exchange.  Output d goes to CTA P = d / 16,
// tile w' = (d / 8) % 2, level-1 row m' = (b % 16) + 16 (d % 8), K word b / 16
// (K block = this CTA's rank): piece j = d % 8 of the receiver's K block
// (rows 16 j..), staged at piece slot (j / 4, 4 (j % 4) + P) of tile w'.
template <bool Lazy, class Gate, class PartDone>
__device__ __forceinline__ void epilogue_a(const Cl& c, uint32_t q, uint32_t qinv, uint32_t ratio, uint32_t start,
                                           uint2 step, Gate gate, PartDone part_done) {
    const uint32_t m = c.quarter * 32u + c.lane, b = 128u * (2u * c.rank + c.w) + beta(m);
    uint32_t tw_e = start;                                      // d = 32h
    uint32_t tw_o = tw_norm<Lazy>(mont_lazy(tw_e, ratio, q, qinv), q);  // d = 32h + 1
    const uint32_t col = lane_cols(c);
    const uint32_t bl = b & 15u, a2 = (b >> 4) & 15u;
    // SW64 offset of (row bl, K word a2) inside a 16-row piece
    const uint32_t inpiece = (bl >> 3) * 512u + (bl & 7u) * 64u + (((a2 >> 2) ^ ((bl >> 1) & 3u)) << 4) + 4u * (a2 & 3u);
#pragma unroll 1
    for (uint32_t part = 0; part < 2; part++) {
        uint32_t y[16];
#pragma unroll
        for (uint32_t sub = 0; sub < 2; sub++) {
            uint32_t c0[8], c1[8], c2[8], c3[8];
            PHASE_T0;
            ld_planes8(col + 16u * part + 8u * sub, c0, c1, c2, c3);
            PHASE_ADD(1);
#pragma unroll
            for (uint32_t i = 0; i < 8; i += 2) {
                y[8 * sub + i] = mont_lazy(combine_redc(c0[i], c1[i], c2[i], c3[i], q, qinv), tw_e, q, qinv);
                y[8 * sub + i + 1] =
                    mont_lazy(combine_redc(c0[i + 1], c1[i + 1], c2[i + 1], c3[i + 1], q, qinv), tw_o, q, qinv);
                tw_e = tw_norm<Lazy>(shoup_lazy(tw_e, step.x, step.y, q), q);
                tw_o = tw_norm<Lazy>(shoup_lazy(tw_o, step.x, step.y, q), q);
            }
        }
        if (part == 0) {
            PHASE_T0;
            gate();
            PHASE_ADD(2);
        }
        // d = 32h + 16 part + i: P = 2h + part, w' = i / 8, j = i % 8
        const uint32_t o0 = inpiece + (2u * c.h + part) * kPiece;
        uint8_t* o = c.base + kOffBuf0 + o0;
        if (NTTB_CHECK(g_tc_bounds, kBoundsShared, o0 + kTileBytes + 16384u + 3u * kPiece + 4u <= kBufBytes))
#pragma unroll
            for (uint32_t i = 0; i < 16; i++)
                *reinterpret_cast<uint32_t*>(o + (i >> 3) * kTileBytes + ((i >> 2) & 1u) * 16384u +
                                             4u * (i & 3u) * kPiece) = y[i];
        PHASE_T0;
        part_done(part);
        PHASE_ADD(3);
    }
}

// Stage B level-1 epilogue: row m' = b2 + 16 r, outputs d2 = 32h + i;
// z * t_B1(b2, d2) in [0, 2q) -> level-2 operand of the same tile (over
// level 1), SW64, row r + 8 (d2 / 16) + 32 (d2 % 16), K word b2.
template <class Gate>
__device__ __forceinline__ void epilogue_b1(const Cl& c, uint32_t q, uint32_t qinv, uint32_t dir, Gate gate) {
    const uint32_t mv = c.quarter * 32u + c.lane, b2 = mv & 15u, r = mv >> 4;
    // t_B1(b2, 32h + 16 part + i) from the shared-memory table
    const uint32_t* tb = reinterpret_cast<const uint32_t*>(c.base + kOffTB1 + dir * kTB1Dir) + b2 * kTB1Stride + 32u * c.h;
    const uint32_t* ts = tb + 16u * kTB1Stride;  // the Shoup quotients
    const uint32_t col = lane_cols(c);
    // sw64_offset(r + 8 (2h + part) + 32 i, 4 b2) = off + 512 (2h + part) + 2048 i
    const uint32_t off = r * 64u + (((b2 >> 2) ^ ((r >> 1) & 3u)) << 4) + 4u * (b2 & 3u);
#pragma unroll 1
    for (uint32_t part = 0; part < 2; part++) {
        uint32_t y[16];
#pragma unroll
        for (uint32_t sub = 0; sub < 2; sub++) {
            uint32_t c0[8], c1[8], c2[8], c3[8];
            PHASE_T0;
            ld_planes8(col + 16u * part + 8u * sub, c0, c1, c2, c3);
            PHASE_ADD(1);
#pragma unroll
            for (uint32_t g = 0; g < 2; g++) {  // four outputs per pair of 16-byte table loads
                const uint32_t o = 16u * part + 8u * sub + 4u * g;
                const uint4 t = *reinterpret_cast<const uint4*>(tb + o), u = *reinterpret_cast<const uint4*>(ts + o);
                uint32_t* ys = y + 8 * sub + 4 * g;
                const uint32_t i = 4 * g;
                ys[0] = shoup_lazy(combine_redc(c0[i], c1[i], c2[i], c3[i], q, qinv), t.x, u.x, q);
                ys[1] = shoup_lazy(combine_redc(c0[i + 1], c1[i + 1], c2[i + 1], c3[i + 1], q, qinv), t.y, u.y, q);
                ys[2] = shoup_lazy(combine_redc(c0[i + 2], c1[i + 2], c2[i + 2], c3[i + 2], q, qinv), t.z, u.z, q);
                ys[3] = shoup_lazy(combine_redc(c0[i + 3], c1[i + 3], c2[i + 3], c3[i + 3], q, qinv), t.w, u.w, q);
            }
        }
        if (part == 0) {
            PHASE_T0;
            gate();
            PHASE_ADD(2);
        }
        const uint32_t o0 = off + 512u * (2u * c.h + part);
        uint8_t* o = c.base + kOffBuf1 + c.w * kTileBytes + o0;
        if (NTTB_CHECK(g_tc_bounds, kBoundsShared, o0 + 2048u * 15u + 4u <= kTileBytes))
#pragma unroll
            for (uint32_t i = 0; i < 16; i++) *reinterpret_cast<uint32_t*>(o + 2048u * i) = y[i];
    }
}

// Stage B level-2 epilogue.  Lane row2 = 128 t2 + 32 quarter + lane
// (t2 = 2h + part) holds d2 = 16 (lane / 8) + 4 t2 + quarter, r = lane % 8,
// outputs c2: X[d + 64 d2 + 4096 c2], d = 8(2c + w) + r, in [0, 2q).  The last
// stage writes HBM (canonical); otherwise X is staged in buffer 1 for the B->A
// exchange: element (a, b) goes to CTA P = t2, tile w' = quarter / 2, row
// 32 g + 8 c + r with g = 2 (quarter % 2) + w, K word a = lane / 8 + 4 c2 --
// one word of the SW128 atom (g, K block c2 / 8), staged at piece slot
// w' * 32 + P * 8 + 2 g + c2 / 8 (in KB).
template <class Gate, class PartDone>
__device__ __forceinline__ void epilogue_b2(const Cl& c, uint32_t q, uint32_t qinv, void* gout, bool words64, Gate gate,
                                            PartDone part_done) {
    const uint32_t base = c.taddr + c.w * 256u + ((c.quarter * 32u) << 16);
    const uint32_t r = c.lane & 7u, d = 8u * (2u * c.rank + c.w) + r;
#pragma unroll 1
    for (uint32_t part = 0; part < 2; part++) {
        const uint32_t t2 = 2u * c.h + part;
        uint32_t y[16];
#pragma unroll
        for (uint32_t sub = 0; sub < 2; sub++) {
            const uint32_t col = base + t2 * 64u + 8u * sub;
            uint32_t c0[8], c1[8], c2[8], c3[8];
            PHASE_T0;
            tc::ld_32x32b_x8(col + 0, c0);
            tc::ld_32x32b_x8(col + 16, c1);
            tc::ld_32x32b_x8(col + 32, c2);
            tc::ld_32x32b_x8(col + 48, c3);
            tc::ld_wait();
            PHASE_ADD(1);
#pragma unroll
            for (uint32_t k = 0; k < 8; k++) y[8 * sub + k] = combine_redc(c0[k], c1[k], c2[k], c3[k], q, qinv);
        }
        if (gout) {
            const uint32_t d2 = 16u * (c.lane >> 3) + 4u * t2 + c.quarter;
            const uint32_t o = d + 64u * d2;
            if (!NTTB_CHECK(g_tc_bounds, kBoundsGlobal, o + 4096u * 15u < 65536u)) continue;
#if NTTB_DEBUG_BOUNDS
            for (uint32_t k = 0; k < 16; k++) NTTB_CHECK(g_tc_bounds, kBoundsResidue, canon(y[k], q) < q);
#endif
            if (words64) {
                uint64_t* g = static_cast<uint64_t*>(gout) + o;
#pragma unroll
                for (uint32_t k = 0; k < 16; k++) __stcs(g + 4096u * k, (uint64_t)canon(y[k], q));
            } else {
                uint32_t* g = static_cast<uint32_t*>(gout) + o;
#pragma unroll
                for (uint32_t k = 0; k < 16; k++) __stcs(g + 4096u * k, canon(y[k], q));
            }
        } else {
            if (part == 0) {
                PHASE_T0;
                gate();
                PHASE_ADD(2);
            }
            const uint32_t g = 2u * (c.quarter & 1u) + c.w;
            const uint32_t o0 = (c.quarter >> 1) * kTileBytes + t2 * 8u * kPiece + 2u * g * kPiece + r * 128u +
                                4u * (c.lane >> 3);
            uint8_t* o = c.base + kOffBuf1 + o0;
            if (NTTB_CHECK(g_tc_bounds, kBoundsShared, o0 + kPiece + (7u << 4) + 4u <= kBufBytes))
#pragma unroll
                for (uint32_t k = 0; k < 16; k++)
                    *reinterpret_cast<uint32_t*>(o + (k >> 3) * kPiece + (((k & 7u) ^ r) << 4)) = y[k];
            PHASE_T0;
            part_done(part);
            PHASE_ADD(3);
        }
    }
}

// The 16 piece copies of one exchange bound for CTA P (lanes 0..15 of the
// calling warp, one each), completing on barrier `bar_idx` of P.
//   A->B (kind 0): piece (w', j) from buffer 0 slot (w', j / 4, 4 (j % 4) + P)
//     to P's buffer 1, tile w', K block c, rows 16 j.. (offset 8 KB c + 1 KB j).
//   B->A (kind 1): piece (w', g, kb) from buffer 1 slot w' * 32 + P * 8 + 2 g + kb
//     to P's buffer 0, tile w', K block kb, atom 4 g + c.
__device__ __forceinline__ void send_pieces(const Cl& c, uint32_t kind, uint32_t P, uint32_t bar_idx) {
    const uint32_t t = c.lane;
    if (t >= 16) return;
    const uint32_t wp = t >> 3;
    uint32_t src, dst;
    if (kind == 0) {
        const uint32_t j = t & 7u;
        src = kOffBuf0 + wp * kTileBytes + (j >> 2) * 16384u + (4u * (j & 3u) + P) * kPiece;
        dst = kOffBuf1 + wp * kTileBytes + c.rank * 8192u + j * kPiece;
    } else {
        const uint32_t g = (t >> 1) & 3u, kb = t & 1u;
        src = kOffBuf1 + wp * kTileBytes + P * 8192u + (2u * g + kb) * kPiece;
        dst = kOffBuf0 + wp * kTileBytes + kb * 16384u + (4u * g + c.rank) * kPiece;
    }
    const uint32_t base = tc::smem_u32(c.base);
    if (!NTTB_CHECK(g_tc_bounds, kBoundsCluster,
                    P < kClCtas && src + kPiece <= kOffImg && dst + kPiece <= kOffImg && src % 16u == 0 && dst % 16u == 0))
        return;
    tc::bulk_s2cluster(tc::mapa(base + dst, P), base + src, kPiece, tc::mapa(tc::smem_u32(c.bar + bar_idx), P));
}

// ---- the cluster kernel ----------------------------------------------------------------
template <bool Lazy>
__global__ void __launch_bounds__(kClThreads, 1) int8_cluster_n16(const __grid_constant__ ClArgs args) {
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    Cl c;
#ifdef NTT_PHASE_PROFILE
    __shared__ uint32_t s_phase[16];
    const uint32_t phase_k0_ = (uint32_t)clock();
    if (threadIdx.x < 16) s_phase[threadIdx.x] = 0;
    c.phase = s_phase;
#endif
    c.base = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    c.rank = tc::cluster_rank();
    c.tid = threadIdx.x;
    c.w = (threadIdx.x >> 8) & 1u;  // the issuing warp (threads 512..) maps to tile 0; it runs no epilogue
    c.wt = threadIdx.x & 255u;
    c.lane = threadIdx.x & 31u;
    c.quarter = (c.wt >> 5) & 3u;
    c.h = c.wt >> 7;
    c.bar = reinterpret_cast<uint64_t*>(c.base + kOffBar);
    uint32_t* slot = reinterpret_cast<uint32_t*>(c.bar + 12);
    const uint32_t img_a = tc::smem_u32(c.base + kOffImg);
    const bool four = args.n_stages == 4;
    // the per-unit constants and operand: for the first unit, fetched before
    // the cluster start-up barrier
    auto fetch_consts = [&](uint32_t unit) {
        const uint8_t* limb_blob = args.consts + (unit % args.n_limbs) * args.const_stride;
        if (c.tid == 0) {
            const uint64_t pol = tc::l2_policy_evict_last();
            tc::mbar_expect_tx(c.bar + kBarConst, kBlobImg + kMatBytes64 + 2 * kTB1Dir);
            tc::bulk_g2s_hint(c.base + kOffImg16, limb_blob, kBlobImg, c.bar + kBarConst, pol);
#pragma unroll
            for (uint32_t dir = 0; dir < 2; dir++)
                tc::bulk_g2s_hint(c.base + kOffTB1 + dir * kTB1Dir, limb_blob + kBlobTab + (dir * kTabWords + kTabB1) * 4,
                                  kTB1Dir, c.bar + kBarConst, pol);
            copy_image(c, limb_blob, args.st[0].img, c.bar + kBarConst);
        }
    };
    const bool issuer = c.tid >= kEpiThreads;
    auto fetch_data = [&](uint32_t unit) {
        if (issuer) return;
        if (args.words64) load_columns(c, static_cast<const uint64_t*>(args.src) + ((uint64_t)unit << 16));
        else load_columns(c, static_cast<const uint32_t*>(args.src) + ((uint64_t)unit << 16));
    };
    // Programmatic dependent launch: the next launch on the stream may be
    // scheduled now (its CTAs set up on free SMs); nothing of it reads or
    // writes residues before this grid has completed (griddepcontrol.wait).
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    if (c.tid < 32) tc::tmem_alloc(slot, 512);
    if (c.tid == 0) {
        for (uint32_t i = 0; i <= kBarUnit; i++) tc::mbar_init(c.bar + i, i == kBarUnit ? kClCtas : 1);
        // arm the inboxes of the first unit before any peer can send
        tc::mbar_expect_tx(c.bar + kBarIn1, kBufBytes);
        if (four) tc::mbar_expect_tx(c.bar + kBarIn0, kBufBytes);
    }
    if (tc::cluster_id() < args.units) fetch_consts(tc::cluster_id());  // plan constants: no wait needed
    // the previous grid on the stream has completed and its writes are visible
    asm volatile("griddepcontrol.wait;" ::: "memory");
    if (tc::cluster_id() < args.units) fetch_data(tc::cluster_id());
    tc::fence_before_sync();
    __syncthreads();
    tc::cluster_sync();  // every CTA's barriers exist and are armed before any remote traffic
    tc::fence_after_sync();
    c.taddr = *slot;
#ifdef NTT_PHASE_PROFILE
    if (threadIdx.x == 0) atomicAdd(c.phase + 8, (uint32_t)clock() - phase_k0_);
#endif
    uint32_t ph_mma = 0, ph_mma2 = 0, ph_ld = 0, ph_img = 0, ph_in0 = 0, ph_in1 = 0, ph_unit = 0;
    uint32_t iter = 0;
    for (uint32_t unit = tc::cluster_id(); unit < args.units; unit += tc::cluster_count(), iter++) {
        const uint32_t limb = unit % args.n_limbs;
        const uint64_t off = (uint64_t)unit << 16;
        const uint8_t* limb_blob = args.consts + limb * args.const_stride;
        if (iter > 0) {
            // the previous unit is finished everywhere: peers no longer read their
            // buffers and every copy out of this CTA's buffers has landed
            wait_cluster(c.bar + kBarUnit, ph_unit);
            fetch_consts(unit);
            fetch_data(unit);
        }
        wait_local(c.bar + kBarConst, ph_ld);
        tc::fence_proxy_async_smem();
        tc::fence_before_sync();
        __syncthreads();
        bool img_pending = false;  // issuing thread: a next-stage image copy is in flight
        for (uint32_t s = 0; s < args.n_stages; s++) {
#ifdef NTT_PHASE_PROFILE
            const uint32_t phase_stage_ = (uint32_t)clock();
#endif
            const ClStage& S = args.st[s];
            const bool last = s + 1 == args.n_stages;
            const bool next_img = !last && args.st[s + 1].img != S.img;
            const uint32_t in = buf_addr(c, s & 1u);
            // this thread's twiddle inputs, loaded now so the latency hides
            // behind the operand wait and the MMA
            uint32_t q = 0, qinv = 0, ratio = 0, start = 0;
            uint2 step = make_uint2(0, 0);
            if (!issuer) {
                const uint32_t* T = reinterpret_cast<const uint32_t*>(limb_blob + kBlobTab) + S.dir * kTabWords;
                q = __ldg(T + kTabQ);
                qinv = __ldg(T + kTabQ + 1);
                if (S.kind == 0) {
                    const uint32_t b = 128u * (2u * c.rank + c.w) + beta(c.quarter * 32u + c.lane);
                    ratio = __ldg(T + kTabArat + b);
                    start = __ldg(T + kTabAst + 2 * b + c.h);
                    step = __ldg(reinterpret_cast<const uint2*>(T + kTabAstep) + b);
                }
            }
            if (issuer) {
                // the stage's operand (s > 0: 64 KB from the four CTAs) and
                // image are in shared memory: issue the four MMAs, then, once
                // they are done, fetch the next stage's image over this one
                if (s > 0) {
                    if (s & 1u) wait_cluster(c.bar + kBarIn1, ph_in1);
                    else wait_cluster(c.bar + kBarIn0, ph_in0);
                    if (s == 1 && four && c.lane == 0) tc::mbar_expect_tx(c.bar + kBarIn1, kBufBytes);  // stage 3
                }
                if (c.lane == 0) {
                    if (img_pending) wait_local(c.bar + kBarImg, ph_img);
                    img_pending = false;
                    tc::fence_after_sync();
#pragma unroll
                    for (uint32_t w = 0; w < 2; w++) {
                        if (S.kind == 0) issue_k256(c.taddr + w * 256u, in + w * kTileBytes, 128, img_a, 256, 256);
                        else issue_k256_a64(c.taddr + w * 256u, in + w * kTileBytes, 128, img_a, 256, 256);
                        tc::commit(c.bar + kBarMma + w);
                    }
                }
                __syncwarp();
                wait_parity(c.bar + kBarMma + 1, ph_mma);  // the last commit: every MMA is done
                ph_mma ^= 1u;
                if (c.lane == 0 && next_img) {
                    tc::mbar_expect_tx(c.bar + kBarImg, kMatBytes64);
                    copy_image(c, limb_blob, args.st[s + 1].img, c.bar + kBarImg);
                    img_pending = true;
                }
                __syncwarp();
                tc::fence_before_sync();
                __syncthreads();
                continue;
            }
            {
                PHASE_T0;
                wait_parity(c.bar + kBarMma + c.w, ph_mma);
                PHASE_ADD(0);
            }
            tc::fence_after_sync();
            // before the first stores: the MMAs reading the overwritten operand
            // are done (stage A stages into both tiles' operands: every MMA;
            // stage B level 1 writes over its own tile's, whose MMA this
            // thread has waited for)
            auto mma_gate = [&]() {
                if (S.kind == 0) wait_parity(c.bar + kBarMma + 1, ph_mma);
            };
            // after each part's stores: the 256 threads of output half h have
            // staged every piece for CTA 2h + part, and one warp sends them
            auto part_done = [&](uint32_t part) {
                if (last) return;
                tc::fence_proxy_async_smem();
                asm volatile("bar.sync %0, %1;" ::"r"(3u + c.h), "r"(256u) : "memory");
                if (c.w == 0 && c.quarter == 0)
                    send_pieces(c, S.kind, 2u * c.h + part, S.kind == 0 ? kBarIn1 : kBarIn0);
            };
            if (S.kind == 0) {
                epilogue_a<Lazy>(c, q, qinv, ratio, start, step, mma_gate, part_done);
                ph_mma ^= 1u;
            } else {
                epilogue_b1(c, q, qinv, S.dir, mma_gate);
                ph_mma ^= 1u;
                PHASE_T0;
                tc::fence_proxy_async_smem();
                tc::fence_before_sync();
                asm volatile("bar.sync %0, %1;" ::"r"(1u + c.w), "r"(256u) : "memory");
                if (c.wt == 0) {
                    tc::fence_after_sync();
                    const uint32_t idesc = tc::idesc_u8(128, 64);
                    const uint32_t bb = tc::smem_u32(c.base + kOffImg16 + S.img16 * kMatBytes16);
#pragma unroll
                    for (uint32_t t = 0; t < 4; t++)
#pragma unroll
                        for (uint32_t ks = 0; ks < 2; ks++)
                            tc::mma_i8(c.taddr + c.w * 256u + t * 64u,
                                       tc::desc_k_sw64(in + c.w * kTileBytes + t * 8192u + ks * 32u),
                                       tc::desc_k_sw64(bb + ks * 32u), idesc, ks > 0);
                    tc::commit(c.bar + kBarMma2 + c.w);
                }
                __syncwarp();
                wait_parity(c.bar + kBarMma2 + c.w, ph_mma2);
                PHASE_ADD(4);
                tc::fence_after_sync();
                // staging overwrites both tiles' level-2 operands
                void* gout = nullptr;
                if (last)
                    gout = args.words64 ? (void*)(static_cast<uint64_t*>(args.dst) + off)
                                        : (void*)(static_cast<uint32_t*>(args.dst) + off);
                epilogue_b2(c, q, qinv, gout, args.words64 != 0,
                            [&]() { wait_parity(c.bar + kBarMma2 + (c.w ^ 1u), ph_mma2); }, part_done);
                ph_mma2 ^= 1u;
            }
            PHASE_T0;
            tc::fence_proxy_async_smem();
            tc::fence_before_sync();
            __syncthreads();
            PHASE_ADD(5);
#ifdef NTT_PHASE_PROFILE
            if ((threadIdx.x & 31u) == 0) atomicAdd(c.phase + 6, (uint32_t)clock() - phase_stage_);
#endif
            if (last && c.tid == 0) {
                // this CTA reads its buffers no more in this unit: re-arm the
                // inboxes for the next one, then report done to every CTA
                tc::mbar_expect_tx(c.bar + kBarIn1, kBufBytes);
                if (four) tc::mbar_expect_tx(c.bar + kBarIn0, kBufBytes);
                arrive_all(c, kBarUnit);
            }
        }
    }
    // the last arrivals aimed at this CTA have landed before it exits
    if (iter > 0) wait_cluster(c.bar + kBarUnit, ph_unit);
    tc::fence_before_sync();
    __syncthreads();
    if (c.tid < 32) tc::tmem_dealloc(c.taddr, 512);
#ifdef NTT_PHASE_PROFILE
    if (threadIdx.x == 0) {
        atomicAdd(c.phase + 7, (uint32_t)clock() - phase_k0_);
        atomicAdd(c.phase + 9, 1u);
    }
    __syncthreads();
    if (threadIdx.x < 16) atomicAdd(&g_phase[threadIdx.x], (unsigned long long)c.phase[threadIdx.x]);
#endif
}

// ---- host: tables and byte-plane images ------------------------------------------------
// Byte-plane image of a 64-point matrix: B[(a, k)][(j, p)] = byte a of
// (256^p * 2^32 * W[k][j] mod q), K-major SW128, 256 rows ordered
// (k / 32, a, k % 32) so that rows 128 h.. are the four planes of outputs
// 32 h.. (one N = 128 MMA per output half).
void build_image64(uint8_t* img, const std::vector<uint64_t>& W, uint64_t q) {
    std::memset(img, 0, kMatBytes64);
    for (uint32_t k = 0; k < 64; k++)
        for (uint32_t j = 0; j < 64; j++)
            for (uint32_t p = 0; p < 4; p++) {
                const uint64_t v = h_mulmod(h_to_mont32(W[k * 64 + j], q), (1ull << (8 * p)) % q, q);
                for (uint32_t a = 0; a < 4; a++)
                    img[tc::sw128_offset((k >> 5) * 128 + a * 32 + (k & 31), 4 * j + p, 256)] = (uint8_t)(v >> (8 * a));
            }
}

// Byte-plane image of a 16-point matrix: 64 rows (a, c) x 64 bytes, K-major SW64.
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

// Twiddle table of one direction (layout above kTabWords).
void fill_tables(uint32_t* t, uint64_t q, const uint64_t* start_a, const uint64_t* ratio_a, const uint64_t* ratio_b) {
    t[kTabQ] = (uint32_t)q;
    t[kTabQ + 1] = h_neg_inv32((uint32_t)q);
    for (uint32_t b = 0; b < 1024; b++) {
        t[kTabAst + 2 * b] = h_to_mont32(start_a[b], q);
        t[kTabAst + 2 * b + 1] = h_to_mont32(h_mulmod(start_a[b], h_powmod(ratio_a[b], 32, q), q), q);
        t[kTabArat + b] = h_to_mont32(ratio_a[b], q);
        const uint64_t r2 = h_mulmod(ratio_a[b], ratio_a[b], q);
        t[kTabAstep + 2 * b] = (uint32_t)r2;
        t[kTabAstep + 2 * b + 1] = (uint32_t)((r2 << 32) / q);
    }
    for (uint32_t b2 = 0; b2 < 16; b2++)
        for (uint32_t d2 = 0; d2 < 64; d2++) {
            const uint64_t tw = h_powmod(ratio_b[b2], d2, q);
            t[kTabB1 + b2 * kTB1Stride + d2] = (uint32_t)tw;
            t[kTabB1 + (16 + b2) * kTB1Stride + d2] = (uint32_t)((tw << 32) / q);
        }
}

// DFT-64 image slots: 0 stage A forward, 1 inverse (stage A and stage B
// level 1 share it), 2 stage B level 1 forward.
int build_cache(Plan32& p, Int8Cache* c) {
    const uint32_t n = p.n, nl = p.n_limbs;
    // blob layout per limb: DFT-16 forward / inverse images, the DFT-64
    // images, then the forward and inverse twiddle tables
    const size_t per_limb = kBlobBytes;
    std::vector<uint8_t> blob(per_limb * nl);
    uint8_t* d_blob = nullptr;
    if (cudaMalloc(&d_blob, blob.size()) != cudaSuccess) return 4;
    std::vector<uint64_t> st(1024), ra(1024), rb(16);
    for (uint32_t l = 0; l < nl; l++) {
        const LimbHost& H = p.limbs[l];
        const uint64_t q = H.q;
        uint8_t* h = blob.data() + per_limb * l;
        const uint64_t w = H.omega, wi = H.omega_inv;
        const uint64_t w64 = h_powmod(w, n / 64, q), w64i = h_powmod(wi, n / 64, q);
        const uint64_t w16 = h_powmod(w, n / 16, q), w16i = h_powmod(wi, n / 16, q);
        // stage A forward: the negacyclic twist psi^(a * n/64) on the input index
        // makes W[k][j] = psi_128^(j (2k + 1)), psi_128 = psi^(n/64)
        const uint64_t p128 = h_powmod(H.psi, n / 64, q);
        build_image64(h + kBlobImg, p.negacyclic ? dft_matrix(64, h_mulmod(p128, p128, q), q, 1, p128) : dft_matrix(64, w64, q), q);
        build_image64(h + kBlobImg + kMatBytes64, dft_matrix(64, w64i, q), q);
        build_image64(h + kBlobImg + 2 * kMatBytes64, dft_matrix(64, w64, q), q);
        // stage B level 2 inverse: n^-1 (and psi^-(4096 c2)) folded on the output index
        std::vector<uint64_t> B2f = dft_matrix(16, w16, q);
        std::vector<uint64_t> B2i = p.negacyclic ? dft_matrix(16, w16i, q, h_powmod(H.psi_inv, 4096, q), 1, H.n_inv)
                                                 : dft_matrix(16, w16i, q, 1, 1, H.n_inv);
        build_image16(h, B2f, q);
        build_image16(h + kMatBytes16, B2i, q);
        uint32_t* tab = reinterpret_cast<uint32_t*>(h + kBlobTab);
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
    }
    if (cudaMemcpy(d_blob, blob.data(), blob.size(), cudaMemcpyHostToDevice) != cudaSuccess) {
        cudaFree(d_blob);
        return 3;
    }
    c->d_blob = d_blob;
    c->per_limb = per_limb;
    c->lazy = true;
    for (uint32_t l = 0; l < nl; l++) c->lazy = c->lazy && p.limbs[l].q < (1ull << 31) - (1ull << 16);
    c->negacyclic = p.negacyclic;
    c->log_n = p.log_n;
    return 0;
}

Int8Cache* get_cache(Plan32& p) {
    std::lock_guard<std::mutex> lock(p.engine_mu);
    auto* c = reinterpret_cast<Int8Cache*>(p.engine_data[1]);
    if (c) return c;
    c = new Int8Cache();
    if (build_cache(p, c)) {
        delete c;
        return nullptr;
    }
    p.engine_data[1] = c;
    return c;
}

ClStage stage(const Int8Cache* c, bool inverse, uint32_t kind) {
    ClStage s{};
    s.dir = inverse ? 1 : 0;
    s.kind = kind;
    if (kind == 0) {
        s.img = inverse ? 1 : 0;
    } else {
        // cyclic: the forward stage A and B level-1 matrices coincide (slot 0)
        s.img = inverse ? 1 : (c->negacyclic ? 2 : 0);
    }
    s.img16 = inverse ? 1 : 0;
    return s;
}

void launch_config(cudaLaunchConfig_t& cfg, cudaLaunchAttribute* attr, uint32_t clusters, cudaStream_t s) {
    std::memset(&cfg, 0, sizeof cfg);
    cfg.gridDim = dim3(kClCtas * clusters);
    cfg.blockDim = dim3(kClThreads);
    cfg.dynamicSmemBytes = kClSmem;
    cfg.stream = s;
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = kClCtas;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    attr[1].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[1].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 2;
}

// Clusters of 4 that fit on the current device at once (one CTA per SM).
// The shared-memory attribute and the answer are per device.
int max_clusters() {
    static std::atomic<int> cached[64];  // the same for both kernel instances (same resources)
    int dev = 0;
    cudaGetDevice(&dev);
    std::atomic<int>& slot = cached[dev & 63];
    if (const int c = slot.load()) return c;
    cudaFuncSetAttribute(int8_cluster_n16<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kClSmem);
    cudaFuncSetAttribute(int8_cluster_n16<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kClSmem);
    cudaLaunchConfig_t cfg;
    cudaLaunchAttribute attr[2];
    launch_config(cfg, attr, 1, 0);
    int n = 0;
    if (cudaOccupancyMaxActiveClusters(&n, int8_cluster_n16<true>, &cfg) != cudaSuccess || n < 1) {
        cudaGetLastError();
        int sms = 0;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        n = sms / (int)kClCtas / 2 > 0 ? sms / (int)kClCtas / 2 : 1;
    }
    slot.store(n);
    return n;
}

int launch_stages(Int8Cache* c, ClArgs& a, cudaStream_t s) {
    const uint32_t mc = (uint32_t)max_clusters();
    const uint32_t clusters = a.units < mc ? a.units : mc;
    a.consts = c->d_blob;
    a.const_stride = c->per_limb;
    cudaLaunchConfig_t cfg;
    cudaLaunchAttribute attr[2];
    launch_config(cfg, attr, clusters, s);
    ProfScope prof(a.n_stages == 2 ? "int8_cluster_n16_x2" : "int8_cluster_n16_x4", s);
    const cudaError_t e = c->lazy ? cudaLaunchKernelEx(&cfg, int8_cluster_n16<true>, a)
                                  : cudaLaunchKernelEx(&cfg, int8_cluster_n16<false>, a);
    return launch_rc(e);
}

}  // namespace

// DFT-64 byte-plane images for other kernels (the batch engine's tensor tiles).
void tc_build_image64(uint8_t* img, const std::vector<uint64_t>& W, uint64_t q) { build_image64(img, W, q); }
void tc_build_image16(uint8_t* img, const std::vector<uint64_t>& W, uint64_t q) { build_image16(img, W, q); }
std::vector<uint64_t> tc_dft_matrix(uint32_t L, uint64_t root, uint64_t q, uint64_t row_twist, uint64_t col_twist,
                                    uint64_t scale) {
    return dft_matrix(L, root, q, row_twist, col_twist, scale);
}

// N = 2^16, residues as uint32 or as uint64 words (the drop-in layout; read
// and written in place of the uint32 ones).
bool int8_serves(const Plan32& p, bool src_u64) {
    (void)src_u64;
    return p.log_n == 16;
}

int int8_transform32(Plan32& p, const void* src, void* dst, bool src_u64, uint32_t n_polys, bool inverse,
                     cudaStream_t s) {
    if (!int8_serves(p, src_u64)) return 1;
    if ((uint64_t)n_polys * p.n_limbs > (1u << 24)) return 1;
    Int8Cache* c = get_cache(p);
    if (!c) return 2;
    ClArgs a{};
    a.st[0] = stage(c, inverse, 0);
    a.st[1] = stage(c, inverse, 1);
    a.n_stages = 2;
    a.src = src;
    a.dst = dst;
    a.words64 = src_u64 ? 1u : 0u;
    a.n_limbs = p.n_limbs;
    a.units = n_polys * p.n_limbs;
    return launch_stages(c, a, s);
}

int int8_forward_inverse32(Plan32& p, uint32_t* data, uint32_t n_polys, cudaStream_t s) {
    if (!int8_serves(p, false)) return 1;
    if ((uint64_t)n_polys * p.n_limbs > (1u << 24)) return 1;
    Int8Cache* c = get_cache(p);
    if (!c) return 2;
    ClArgs a{};
    a.st[0] = stage(c, false, 0);
    a.st[1] = stage(c, false, 1);
    a.st[2] = stage(c, true, 0);
    a.st[3] = stage(c, true, 1);
    a.n_stages = 4;
    a.src = data;
    a.dst = data;
    a.n_limbs = p.n_limbs;
    a.units = n_polys * p.n_limbs;
    return launch_stages(c, a, s);
}

void int8_release(Plan32* p) {
    auto* c = reinterpret_cast<Int8Cache*>(p->engine_data[1]);
    if (!c) return;
    if (c->d_blob) cudaFree(c->d_blob);
    delete c;
    p->engine_data[1] = nullptr;
}

void int8_phase_profile(uint64_t* out16, bool clear) {
    unsigned long long v[16] = {};
    cudaMemcpyFromSymbol(v, g_phase, sizeof v);
    for (int i = 0; i < 16; i++) out16[i] = v[i];
    if (clear) {
        const unsigned long long z[16] = {};
        cudaMemcpyToSymbol(g_phase, z, sizeof z);
    }
}

uint32_t int8_bounds_errors(bool clear) {
    uint32_t v = 0;
    cudaMemcpyFromSymbol(&v, g_tc_bounds, sizeof v);
    if (clear) {
        uint32_t z = 0;
        cudaMemcpyToSymbol(g_tc_bounds, &z, sizeof z);
    }
    return v;
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
