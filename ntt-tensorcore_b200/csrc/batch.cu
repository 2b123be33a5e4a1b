// batch.cu -- uneven batches: polynomials of different sizes (2^1 .. 2^max_log),
// limb counts, moduli and directions transformed in ONE persistent launch.
//
// Work decomposition.  Every (polynomial, limb) transform of n = 2^L residues
// is a "unit":
//   * L <= log2(tile): one single-pass unit covers up to `rows` consecutive
//     limbs of a polynomial (one shared-memory tile, one row per limb: the
//     limb split), DIF stages, natural order in and out;
//   * larger L: a two-pass four-step unit per limb, n = N1 * N2:
//       pass A: columns b of x as [N1][N2]: U[d][b] = DFT_N1(x[.][b])[d] * w^(d b),
//               stored transposed at b N1 + d in a workspace slot;
//       pass B: columns d of the slot as [N2][N1]: X[d + N1 k] = DFT_N2, to x.
//     Pass A has N2 / va tiles, pass B N1 / vb tiles (va, vb vectors per tile).
// Negacyclic twists psi^i and the inverse's n^-1 (psi^-i) are fused into the
// first load and the last store.  This is the scalar engine's two-pass
// layout, so results are bit-identical to the per-size transforms.
//
// Polynomial products (job flag NTTB_BATCH_POLYMUL): each row group becomes
// three units -- forward(a), forward(b), and inverse(a . b), whose first load
// multiplies the two spectra (the reference's poly_multiply_ntt,
// src/ntt_basic.cu:391-409, fused between the passes).  The inverse unit
// depends on both forward units; all three run in the same launch.
//
// The device work queue.  The host lays the tiles out in one array, largest
// units first; a unit's pass B tiles are placed `lag` two-pass units after its
// pass A tiles, so CTAs rarely wait.  CTAs of the persistent grid claim tiles
// with an atomic ticket.  A pass B tile first waits (bounded spin, acquire)
// until every pass A tile of its unit has signalled; a pass A tile first waits
// until the previous user of its workspace slot has finished pass B.  Every
// awaited tile has a smaller ticket, so it belongs to a CTA that is already
// running: no deadlock.  Workspace slots form one ring per size class 2^L of
// S_L > lag slots (enough for ~1024 pass A tiles in flight), so the workspace
// is bounded by the rings, not by the size of the batch.
//
// Inside a tile, radix-2 stages run in register groups of 1, 3 or 4: one
// thread loads the 2, 8 or 16 elements that a group's stages combine,
// applies the group's butterflies in registers and stores them once -- one
// barrier and one shared-memory round trip per group.  Twiddles and twists
// come from two-level power tables (8 KB per base and modulus, L2-resident).
//
// Tuning knobs (nttb_batch_config): shared-memory tile size and CTA width
// (4096/256, 8192/256, 8192/512, 16384/512), stages per register group (3,
// 4, or 1 = stage by stage), the radix split of two-pass units (first pass 2^ceil(L/2) or
// 2^floor(L/2)), the queue lag and the CTAs per SM; nttb_batch_autotune
// times the candidates on a sample of the job mix.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <deque>
#include <string>
#include <vector>

#include "../../include/ntt_b200.h"
#include "arith.cuh"
#include "batch.hpp"
#include "bounds.cuh"
#include "engines.hpp"
#include "plan.hpp"
#include "profiler.hpp"
#include "tc_arith.cuh"
#include "tcgen05.cuh"

namespace nttb {

// bit 0: a queue dependency wait ran out of budget; bit 1: a tensor-core
// tile's wait on its MMA or image copy did
__device__ uint32_t g_batch_error;
// NTT_DEBUG_BOUNDS build: failed range checks (bounds.cuh bits)
__device__ uint32_t g_batch_bounds;

namespace {

constexpr uint32_t BF_INV = 1, BF_PRE_PSI = 2, BF_POST_TW = 4, BF_STORE_T = 8, BF_POST_SCALE = 16, BF_POST_PSI = 32,
                   BF_PRE_MUL = 64;
// UF_TC: tensor-core tiles; UF_W64: the unit's data (and its source) are
// uint64 words holding residues (tensor-tile two-pass units only)
constexpr uint32_t UF_INV = 1, UF_NEGA = 2, UF_TC = 4, UF_W64 = 8;
constexpr uint32_t kMaxRows = 32;

// Power tables: x^e R for e < 2^max_log as hi[e >> kLoBits] * lo[e & lo_mask]
// (one exact Montgomery product), 2 x 4 KB-ish per base instead of 4 MB, so
// the tables of every modulus stay resident in L2.  Bases: 0 omega (order
// 2^max_log), 1 omega^-1, 2 psi (order 2^(max_log + 1), negacyclic plans),
// 3 psi^-1.
constexpr uint32_t kLoBits = 10;
enum : uint32_t { PW_OMEGA = 0, PW_OMEGA_INV = 1, PW_PSI = 2, PW_PSI_INV = 3 };

// Per-modulus device constants at the plan's largest size 2^max_log.
struct BModulus {
    M32 ar;
    const uint32_t* pw;       // 4 bases x [hi (2^(max_log - lo_bits)) | lo (2^lo_bits)]
    uint32_t lo_bits, hi_len; // lo_bits = min(kLoBits, max_log)
    uint32_t ninv[25];        // 2^-L R mod q
    uint32_t r2;              // R^2 mod q (plain product a b = mul(mul(a, b), R^2))
};

__device__ __forceinline__ uint32_t pw(const BModulus& M, const M32& ar, uint32_t base, uint32_t e) {
    const uint32_t* t = M.pw + base * (M.hi_len + (1u << M.lo_bits));
    return ar.mul(__ldg(t + (e >> M.lo_bits)), __ldg(t + M.hi_len + (e & ((1u << M.lo_bits) - 1))));
}

struct BUnit {
    uint32_t* data;    // row 0 of the unit; row r (limb) at data + r n (uint64 words with UF_W64)
    const void* in;    // pass A reads here instead of data (same layout), or null
    uint32_t* ws;      // workspace slot (two-pass units)
    const uint32_t* pre_mul;  // inverse of a product: the input is data . pre_mul (same layout), else null
    uint32_t mod0;     // modulus index of row 0; row r uses mod0 + r
    uint32_t log_n;
    uint32_t flags;    // UF_INV | UF_NEGA
    uint32_t lg1;      // log2 of the pass A length; 0: single pass
    uint32_t rows;     // single pass: rows in the tile
    uint32_t va, vb;   // vectors per tile in pass A / pass B
    uint32_t tiles_a, tiles_b;
    int32_t prev;      // two-pass unit that held the same workspace slot before, or -1
    int32_t after[2];  // units that must be complete before this one starts, or -1
    // what pass A waits for, self-contained: counter ctr[2 + 2 prev] >= need[0],
    // ctr[after_ctr[d]] >= need[1 + d] (the last pass of unit after[d])
    uint32_t need[3];
    uint32_t after_ctr[2];
    uint32_t dis;      // tensor-tile two-pass units: first of the unit's discard-group counters
                       // (after the 1 + 2 n_units queue counters), else kNoDiscard
    uint32_t pad_[2];
};
static_assert(sizeof(BUnit) % 16 == 0, "unit records are copied in 16-byte pieces");

// Workspace lines of a two-pass unit's slot are dropped from the L2 without a
// write-back once its pass B has read them (the slot's next owner rewrites
// them; otherwise the dirty lines reach DRAM on eviction: 4 bytes per residue
// never read).  A pass B tile reads columns v0 .. v0 + V of every row of the
// slot; with V < 32 words a 128-byte line holds the columns of g = 32 / V
// consecutive tiles, so the lines are dropped by the last of each group of g
// tiles to finish reading (a counter per group), one line per row.
constexpr uint32_t kNoDiscard = 0xFFFFFFFFu;

// Job flags of the plan-transform route (tiles_transform32), which the C ABI
// refuses: kJobW64 -- data and source are uint64 words; kJobSrc -- pass A
// reads `pointwise` (the source, same layout), pass B writes data.
constexpr uint32_t kJobW64 = 1u << 30, kJobSrc = 1u << 29;
constexpr uint32_t kPublicJobFlags = NTTB_BATCH_INVERSE | NTTB_NEGACYCLIC | NTTB_BATCH_POLYMUL;
__host__ __device__ inline uint32_t discard_group(uint32_t log_n, uint32_t lg1) {
    const uint32_t V = 128u >> (log_n - lg1 - 6u);  // pass B vectors per tile row
    return V >= 32u ? 1u : 32u / V;
}

struct BTile {
    uint32_t unit;
    uint32_t pass_tile;  // pass in bit 31, tile index below
};

struct BArgs {
    const BModulus* mods;
    const BUnit* units;
    const BTile* tiles;
    uint32_t* ctr;  // [0] ticket; [1 + 2u] pass A tiles done, [2 + 2u] pass B tiles done of unit u
    const uint8_t* images;  // per modulus: DFT-64 byte-plane images (forward, inverse, negacyclic forward)
    uint32_t n_tiles, max_log;
    uint32_t n_units;       // units in the queue (range checks of the NTT_DEBUG_BOUNDS build)
    const uint32_t* ws;     // the workspace rings, ws_words words
    uint64_t ws_words;
    uint32_t n_dis;         // discard-group counters after the queue counters
};

// NTT_DEBUG_BOUNDS build: the tile's unit, its tile index and its workspace
// slot are in range (else the tile is skipped; bounds.cuh bits).
__device__ __forceinline__ bool tile_in_range(const BArgs& a, const BTile& tl) {
    if (!NTTB_CHECK(g_batch_bounds, kBoundsQueue, tl.unit < a.n_units)) return false;
    const BUnit& u = a.units[tl.unit];
    if (u.dis != kNoDiscard && (tl.pass_tile >> 31) && u.lg1 && discard_group(u.log_n, u.lg1) > 1 &&
        !NTTB_CHECK(g_batch_bounds, kBoundsQueue,
                    u.dis + (tl.pass_tile & 0x7fffffffu) / discard_group(u.log_n, u.lg1) < a.n_dis))
        return false;
    const uint32_t pass = tl.pass_tile >> 31, tile = tl.pass_tile & 0x7fffffffu;
    if (!NTTB_CHECK(g_batch_bounds, kBoundsQueue, tile < (pass ? u.tiles_b : u.tiles_a) && u.log_n <= a.max_log))
        return false;
    if (u.lg1 && !NTTB_CHECK(g_batch_bounds, kBoundsWorkspace,
                             u.ws >= a.ws && (uint64_t)(u.ws - a.ws) + (1ull << u.log_n) <= a.ws_words))
        return false;
    return true;
}

__device__ __forceinline__ bool wait_ge(const uint32_t* p, uint32_t target) {
    const uint64_t t0 = tc::globaltimer_ns();
    for (uint32_t i = 0; i < (1u << 26); i++) {  // the iteration cap backs up the clock
        uint32_t v;
        asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
        if (v >= target) return true;
        if ((i & 15) == 15 && tc::globaltimer_ns() - t0 > tc::kWaitBudgetNs) return false;
        __nanosleep(64);
    }
    return false;
}

// One tile: V vectors of length len, in shared memory.  COL mode (DIT after
// a bit-reversed load): vectors are columns vec of a [len][C] matrix; ROW
// mode (DIF, bit-reversed read at the store): vectors are rows of n words.
template <uint32_t T, uint32_t kGroup>
__device__ __forceinline__ void run_tile(const BArgs& a, const BUnit& u, uint32_t pass, uint32_t tile, uint32_t* sm,
                                         M32* s_ar) {
    const uint32_t L = u.log_n, n = 1u << L, shift = a.max_log - L;
    const bool inv = u.flags & UF_INV, nega = u.flags & UF_NEGA;
    bool row;
    uint32_t lg, V, v0, C, flags;
    const uint32_t* src;
    uint32_t* dst;
    if (u.lg1 == 0) {
        row = true;
        lg = L;
        V = u.rows;
        v0 = 0;
        C = n;
        src = u.data;
        dst = u.data;
        flags = (nega && !inv ? BF_PRE_PSI : 0u) | (inv ? (nega ? BF_POST_PSI : BF_POST_SCALE) : 0u) |
                (u.pre_mul ? BF_PRE_MUL : 0u);
    } else if (pass == 0) {
        row = false;
        lg = u.lg1;
        V = u.va;
        v0 = tile * V;
        C = n >> lg;
        src = u.data;
        dst = u.ws;
        flags = (nega && !inv ? BF_PRE_PSI : 0u) | BF_POST_TW | BF_STORE_T | (u.pre_mul ? BF_PRE_MUL : 0u);
    } else {
        row = false;
        lg = L - u.lg1;
        V = u.vb;
        v0 = tile * V;
        C = 1u << u.lg1;
        src = u.ws;
        dst = u.data;
        flags = inv ? (nega ? BF_POST_PSI : BF_POST_SCALE) : 0u;
    }
    const uint32_t len = 1u << lg, half_len = len >> 1;
    // V is a power of two for column tiles (a row tile's V is its row count);
    // every index split below is a shift or a mask
    const uint32_t lgV = row ? 0u : 31u - __clz(V);
    // row stride and in-row padding (one word every 32) keep the register
    // groups' loads and stores free of bank conflicts
    const uint32_t stride = len >= 32 ? len + (len >> 5) + 1 : len;
    const uint32_t n_mods = row ? V : 1u;
    uint32_t* t = sm;
    uint32_t* tws = sm + V * stride;  // n_mods x len / 2 root powers
    if (threadIdx.x < n_mods) s_ar[threadIdx.x] = a.mods[u.mod0 + threadIdx.x].ar;
    for (uint32_t i = threadIdx.x; i < n_mods * half_len; i += T) {
        const uint32_t r = i >> (lg - 1), k = i & (half_len - 1);
        const BModulus& M = a.mods[u.mod0 + r];
        tws[i] = pw(M, M.ar, inv ? PW_OMEGA_INV : PW_OMEGA, k << (a.max_log - lg));
    }
    __syncthreads();
    // ---- load ----
    const uint32_t total = V * len;
    for (uint32_t idx = threadIdx.x; idx < total; idx += T) {
        uint32_t v, j, elem;
        size_t pos;
        if (row) {
            v = idx >> lg;
            j = idx & (len - 1);
            pos = (size_t)v * n + j;
            elem = j;
        } else {
            v = idx & (V - 1);
            j = idx >> lgV;
            pos = (size_t)j * C + v0 + v;
            elem = (uint32_t)pos;
        }
        uint32_t x = __ldcg(src + pos);
        if (flags & BF_PRE_MUL) {
            const M32& ar = s_ar[row ? v : 0u];
            x = ar.mul(ar.mul(x, __ldcg(u.pre_mul + pos)), a.mods[u.mod0 + (row ? v : 0u)].r2);
        }
        if (flags & BF_PRE_PSI) {
            const BModulus& M = a.mods[u.mod0 + (row ? v : 0u)];
            const M32& ar = s_ar[row ? v : 0u];
            x = ar.mul(x, pw(M, ar, PW_PSI, elem << shift));
        }
        const uint32_t jj = row ? j : bitrev(j, (int)lg);
        t[v * stride + jj + (jj >> 5)] = x;
    }
    __syncthreads();
    // ---- radix-2 stages, up to kGroup at a time in registers ----
    // A group of r stages s0 .. s0+r-1 touches, for each base index with
    // zero bits [s0, s0 + r), exactly the 2^r elements base + k 2^s0; one
    // thread loads them, runs the group's butterflies (the same butterflies,
    // in the same order, as one stage at a time) and stores them back.
    constexpr uint32_t kG = 1u << kGroup;
    if (!row) {
        const M32 ar = s_ar[0];
        for (uint32_t s0 = 0; s0 < lg; s0 += kGroup) {
            const uint32_t r = lg - s0 < kGroup ? lg - s0 : kGroup, nk = 1u << r;
            const uint32_t groups = len >> r, items = V * groups;
            for (uint32_t it = threadIdx.x; it < items; it += T) {
                const uint32_t v = it & (V - 1), g = it >> lgV;
                const uint32_t low = g & ((1u << s0) - 1), base = ((g >> s0) << (s0 + r)) | low;
                uint32_t* rw = t + v * stride;
                uint32_t x[kG];
#pragma unroll
                for (uint32_t k = 0; k < kG; k++)
                    if (k < nk) {
                        const uint32_t i = base + (k << s0);
                        x[k] = rw[i + (i >> 5)];
                    }
#pragma unroll
                for (uint32_t tt = 0; tt < kGroup; tt++) {
                    if (tt >= r) break;
                    const uint32_t s = s0 + tt, half = 1u << tt;
#pragma unroll
                    for (uint32_t k = 0; k < kG; k++) {
                        if ((k & half) || k + half >= nk) continue;
                        const uint32_t p = low + ((k & (half - 1)) << s0);
                        const uint32_t y = ar.mul(x[k + half], tws[p << (lg - 1 - s)]);
                        const uint32_t u0 = x[k];
                        x[k] = ar.add(u0, y);
                        x[k + half] = ar.sub(u0, y);
                    }
                }
#pragma unroll
                for (uint32_t k = 0; k < kG; k++)
                    if (k < nk) {
                        const uint32_t i = base + (k << s0);
                        rw[i + (i >> 5)] = x[k];
                    }
            }
            __syncthreads();
        }
    } else {
        // DIF: stages from lg-1 down, groups [s_lo, s_lo + r)
        for (int s_hi = (int)lg - 1; s_hi >= 0; s_hi -= (int)kGroup) {
            const uint32_t r = (uint32_t)s_hi + 1 < kGroup ? (uint32_t)s_hi + 1 : kGroup, nk = 1u << r;
            const uint32_t s_lo = (uint32_t)s_hi + 1 - r;
            const uint32_t groups = len >> r, items = V * groups;
            for (uint32_t it = threadIdx.x; it < items; it += T) {
                const uint32_t v = it >> (lg - r), g = it & (groups - 1);
                const uint32_t low = g & ((1u << s_lo) - 1), base = ((g >> s_lo) << (s_lo + r)) | low;
                const M32 ar = s_ar[v];
                const uint32_t* tw_row = tws + v * half_len;
                uint32_t* rw = t + v * stride;
                uint32_t x[kG];
#pragma unroll
                for (uint32_t k = 0; k < kG; k++)
                    if (k < nk) {
                        const uint32_t i = base + (k << s_lo);
                        x[k] = rw[i + (i >> 5)];
                    }
#pragma unroll
                for (int tt = (int)kGroup - 1; tt >= 0; tt--) {
                    if ((uint32_t)tt >= r) continue;
                    const uint32_t s = s_lo + (uint32_t)tt, half = 1u << tt;
#pragma unroll
                    for (uint32_t k = 0; k < kG; k++) {
                        if ((k & half) || k + half >= nk) continue;
                        const uint32_t p = low + ((k & (half - 1)) << s_lo);
                        const uint32_t u0 = x[k], y = x[k + half];
                        x[k] = ar.add(u0, y);
                        x[k + half] = ar.mul(ar.sub(u0, y), tw_row[p << (lg - 1 - s)]);
                    }
                }
#pragma unroll
                for (uint32_t k = 0; k < kG; k++)
                    if (k < nk) {
                        const uint32_t i = base + (k << s_lo);
                        rw[i + (i >> 5)] = x[k];
                    }
            }
            __syncthreads();
        }
    }
    // ---- store ----
    for (uint32_t idx = threadIdx.x; idx < total; idx += T) {
        uint32_t v, k, elem;
        size_t pos;
        uint32_t x;
        if (row) {
            v = idx >> lg;
            k = idx & (len - 1);
            const uint32_t kk = bitrev(k, (int)lg);
            x = t[v * stride + kk + (kk >> 5)];
            pos = (size_t)v * n + k;
            elem = k;
        } else {
            v = idx & (V - 1);
            k = idx >> lgV;
            x = t[v * stride + k + (k >> 5)];
            const uint32_t vec = v0 + v;
            pos = (flags & BF_STORE_T) ? (size_t)vec * len + k : (size_t)k * C + vec;
            elem = (uint32_t)pos;
            if (flags & BF_POST_TW) {
                const BModulus& M = a.mods[u.mod0];
                const uint32_t e = (uint32_t)(((uint64_t)k * vec) & (n - 1));
                x = s_ar[0].mul(x, pw(M, s_ar[0], inv ? PW_OMEGA_INV : PW_OMEGA, e << shift));
            }
        }
        if (flags & (BF_POST_SCALE | BF_POST_PSI)) {
            const uint32_t r = row ? v : 0u;
            const BModulus& M = a.mods[u.mod0 + r];
            x = s_ar[r].mul(x, M.ninv[L]);
            if (flags & BF_POST_PSI) x = s_ar[r].mul(x, pw(M, s_ar[r], PW_PSI_INV, elem << shift));
        }
        dst[pos] = x;
    }
}

// Thread 0 of a tile: waits until the tile's inputs are complete (pass B:
// every pass A tile of its unit; pass A: the previous owner of its workspace
// slot and the units it depends on).  False if a wait ran out of budget.
__device__ __forceinline__ bool wait_deps(const BArgs& a, const BUnit& u, uint32_t ui, uint32_t pass) {
    bool ok = true;
    if (pass == 1) {
        ok = wait_ge(a.ctr + 1 + 2 * ui, u.tiles_a);
    } else {
        if (u.prev >= 0) ok = wait_ge(a.ctr + 2 + 2 * (uint32_t)u.prev, u.need[0]);
        for (int d = 0; d < 2; d++)
            if (u.after[d] >= 0) ok = wait_ge(a.ctr + u.after_ctr[d], u.need[1 + d]) && ok;
    }
    return ok;
}
// ---- tensor-core tiles ----------------------------------------------------------------
// A two-pass unit of 2^13 .. 2^20 residues whose pass lengths are len = 64 r'
// (r' = 1, 2, 4, 8, 16) runs its tiles on the tensor cores.  A tile is the
// pass's DFT of length len over V = 128 / r' consecutive columns (8192
// residues), with j = r' a2 + b2 and output d = k1 + 64 k2:
//   level 1: for each of the 128 vectors (column v, b2), a DFT-64 over a2 --
//            the INT8 byte-plane contraction (M = 128, N = 256, K = 256 bytes)
//            against the modulus's DFT-64 image -- times every factor that is
//            geometric in k1: the inner twiddle omega_len^(b2 k1), pass A's
//            omega_n^(col k1), the inverse's psi^-(N1 k1) and n^-1, the
//            negacyclic input twist psi^(b2 N2 + col) (its psi^(a2 n / 64)
//            part is folded into the forward image), generated as two
//            interleaved chains in the epilogue;
//   level 2: for each (column, k1), a DFT-r' over b2, times the factors that
//            depend on k2 (pass A: omega_n^(64 col k2); negacyclic inverse:
//            psi^-(64 N1 k2), which for pass B is psi_max^-(2^max_log k2 / r')
//            whatever n is, so it lives in that image's rows).
//            r' = 8, 16: a second INT8 contraction (M = 128 rows (column, k1)
//            per MMA, N = 4 r', K = 4 r' bytes, SW32 / SW64 operands) against a
//            small DFT-r' image; r' <= 4: radix 2 in registers.
// Pass A stores transposed (ws[col N1 + d]) and pass B in natural order
// (x[col + N1 d]): the CUDA-core tiles' layouts, so results are identical.
// The data of a tile crosses shared memory twice (operand A, then the level-1
// outputs over it); each image stays resident while consecutive tiles use the
// same modulus and direction.
constexpr uint32_t kTcA = 0;              // operand A: 128 rows x 256 B, SW128 (two K blocks), then level 2's
constexpr uint32_t kTcImg = 32768;        // DFT-64 image (64 KB)
constexpr uint32_t kTcImg2 = 98304;       // DFT-16 (4 KB) or DFT-8 (1 KB) image
constexpr uint32_t kTcFac = 102400;       // level-2 factors [128] and butterfly twiddles [8]
constexpr uint32_t kTcBar = kTcFac + 1024;  // mbarriers: [0] MMA commits, [1] DFT-64 image, [2] DFT-r' image
constexpr size_t kTcSmem = kTcBar + 64 + 1024;  // + alignment slack
// Per-modulus image blob: DFT-64 forward / inverse / negacyclic forward
// (64 KB each), DFT-16 forward / inverse / negacyclic inverse (4 KB each),
// DFT-8 forward / inverse / negacyclic inverse (1 KB each).
constexpr uint32_t kImgBytes = 65536;
constexpr uint32_t kImg16Off = 3 * kImgBytes, kImg8Off = kImg16Off + 3 * 4096;
constexpr uint32_t kImgPerMod = kImg8Off + 3 * 1024;

struct TcState {
    uint8_t* base;      // 1024-aligned dynamic shared memory
    uint32_t taddr;     // 256 TMEM columns
    uint32_t ph_mma, ph_img, ph_img2;
    uint32_t pend_img, pend_img2;  // an image copy in flight that no tile has waited for yet
    uint32_t img_key;   // DFT-64 image in shared memory: (modulus << 2 | variant) + 1, 0 none
    uint32_t img2_key;  // DFT-r' image: ((modulus << 2 | variant) << 1 | r' == 16) + 1, 0 none
};

__host__ __device__ constexpr uint32_t bitrev_c(uint32_t x, uint32_t bits) {
    uint32_t r = 0;
    for (uint32_t i = 0; i < bits; i++) r |= ((x >> i) & 1u) << (bits - 1 - i);
    return r;
}

__device__ __forceinline__ void tc_wait(uint64_t* bar, uint32_t ph) {
    if (!tc::mbar_wait_bounded(bar, ph)) atomicOr(&g_batch_error, 2u);
}

// Level 2 on the CUDA cores (r' <= 4): DFT-2^RL over b2 for each (column v,
// k1), canonical out.  Pass A threads walk k1 fastest (ws rows are contiguous
// in d); pass B threads walk v fastest (x rows are contiguous in the column),
// with k1 spread so that the W reads of a warp hit 32 distinct banks.
template <uint32_t RL>
__device__ __forceinline__ void tc_level2(const BUnit& u, uint32_t pass, uint32_t v0, uint32_t N1, const M32& ar,
                                          const uint32_t* W, const uint32_t* fac, bool use_fac) {
    constexpr uint32_t R = 1u << RL, lgV = 7 - RL, V = 1u << lgV, kPairs = 64u * V;
    constexpr uint32_t sh = lgV >= 5 ? 0u : 5u - lgV;
    uint32_t tw2[R > 1 ? R / 2 : 1];
#pragma unroll
    for (uint32_t j = 0; j < R / 2; j++) tw2[j] = fac[128 + j];
#pragma unroll 1
    for (uint32_t p = threadIdx.x; p < kPairs; p += 256) {
        uint32_t v, k1;
        if (pass == 0) {
            k1 = p & 63u;
            v = p >> 6;
        } else {
            v = p & (V - 1u);
            const uint32_t qq = p >> lgV;
            k1 = (qq & 32u) | ((qq & 31u) >> sh) | ((qq & ((1u << sh) - 1u)) << (5u - sh));
        }
        uint32_t x[R];
#pragma unroll
        for (uint32_t i = 0; i < R; i++) {
            const uint32_t m = bitrev_c(i, RL) * V + v;
            x[i] = tca::canon(W[m * 64u + (k1 & 32u) + ((k1 ^ m) & 31u)], ar.q);
        }
#pragma unroll
        for (uint32_t s = 0; s < RL; s++) {
            const uint32_t half = 1u << s;
#pragma unroll
            for (uint32_t k = 0; k < R; k++) {
                if (k & half) continue;
                const uint32_t j = k & (half - 1u);
                const uint32_t y = j == 0 ? x[k + half] : ar.mul(x[k + half], tw2[j << (RL - 1 - s)]);
                const uint32_t u0 = x[k];
                x[k] = ar.add(u0, y);
                x[k + half] = ar.sub(u0, y);
            }
        }
        if (pass == 0) {
            uint32_t* o = u.ws + (size_t)(v0 + v) * N1 + k1;
#pragma unroll
            for (uint32_t k2 = 0; k2 < R; k2++) o[64u * k2] = use_fac ? ar.mul(x[k2], fac[v * R + k2]) : x[k2];
        } else if (u.flags & UF_W64) {
            uint64_t* o = reinterpret_cast<uint64_t*>(u.data) + (size_t)k1 * N1 + v0 + v;
#pragma unroll
            for (uint32_t k2 = 0; k2 < R; k2++) o[(size_t)64u * k2 * N1] = use_fac ? ar.mul(x[k2], fac[k2]) : x[k2];
        } else {
            uint32_t* o = u.data + (size_t)k1 * N1 + v0 + v;
#pragma unroll
            for (uint32_t k2 = 0; k2 < R; k2++) o[(size_t)64u * k2 * N1] = use_fac ? ar.mul(x[k2], fac[k2]) : x[k2];
        }
    }
}

// Row of the level-2 operand holding (column v, k1): pass A rows run k1 within
// a column (low three bits XOR v, so that the level-1 epilogue's stores of a
// warp hit distinct banks), pass B rows run the columns within a k1.
__device__ __forceinline__ uint32_t l2_row(uint32_t pass, uint32_t v, uint32_t k1, uint32_t lgV) {
    return pass == 0 ? (v << 6) + (k1 ^ (v & 7u)) : (k1 << lgV) + v;
}
// Byte offset of (row, word b2) in the level-2 operand: SW64 (r' = 16,
// 64-byte rows) or SW32 (r' = 8, 32-byte rows).
__device__ __forceinline__ uint32_t l2_off(uint32_t row, uint32_t b2, uint32_t rl) {
    return rl == 4 ? tc::sw64_offset(row, 4u * b2) : tc::sw32_offset(row, 4u * b2);
}
// Stores the level-1 outputs k1 = k0 .. k0 + 7 (k0 a multiple of 8) of the
// thread's vector (v, b2) into the level-2 operand: the same offsets as
// l2_off(l2_row(..)), in closed form.  Pass B rows advance 512 bytes per k1
// (both swizzles); pass A rows keep the atom row (k1 & 7) ^ (v & 7).
template <uint32_t PASS, uint32_t RL>
__device__ __forceinline__ void l2_store8(uint8_t* A2, const uint32_t (&y)[8], uint32_t v, uint32_t b2, uint32_t k0) {
    if (PASS == 1) {
        uint8_t* o = A2 + l2_off(l2_row(1, v, k0, 7 - RL), b2, RL);
#pragma unroll
        for (uint32_t i = 0; i < 8; i++) *reinterpret_cast<uint32_t*>(o + 512u * i) = y[i];
    } else {
        const uint32_t v7 = v & 7u;
        uint8_t* o = A2 + (RL == 4 ? 4096u : 2048u) * v + (RL == 4 ? 512u : 256u) * (k0 >> 3) + 4u * (b2 & 3u);
#pragma unroll
        for (uint32_t i = 0; i < 8; i++) {
            const uint32_t r = i ^ v7;  // row within the 8-row atom
            const uint32_t off = RL == 4 ? 64u * r + ((((b2 >> 2) ^ (r >> 1)) & 3u) << 4)
                                         : 32u * r + ((((b2 >> 2) ^ (r >> 2)) & 1u) << 4);
            *reinterpret_cast<uint32_t*>(o + off) = y[i];
        }
    }
}

// Geometry of a tensor tile.
struct TcGeo {
    uint32_t L, n, shift, N1, lg, rl, rp, lgV, V, C, v0;
    const uint32_t* src;  // uint64 words when w64
    bool pre, mma2, inv, nega;
    bool w64;             // pass A source / pass B destination are uint64 words
    uint32_t variant, variant2, key, key2;
};
__device__ __forceinline__ TcGeo tc_geo(const BArgs& a, const BUnit& u, uint32_t pass, uint32_t tile) {
    TcGeo g;
    g.L = u.log_n;
    g.n = 1u << g.L;
    g.shift = a.max_log - g.L;
    g.inv = u.flags & UF_INV;
    g.nega = u.flags & UF_NEGA;
    g.N1 = 1u << u.lg1;
    g.lg = pass == 0 ? u.lg1 : g.L - u.lg1;  // pass length 64 r'
    g.rl = g.lg - 6;
    g.rp = 1u << g.rl;
    g.lgV = 7 - g.rl;
    g.V = 1u << g.lgV;
    g.C = pass == 0 ? g.n >> u.lg1 : g.N1;   // columns of the pass's matrix
    g.v0 = tile << g.lgV;
    g.src = pass == 0 ? static_cast<const uint32_t*>(u.in ? u.in : u.data) : u.ws;
    g.w64 = u.flags & UF_W64;
    g.pre = pass == 0 && u.pre_mul;
    g.mma2 = g.rl >= 3;  // level 2 on the tensor cores
    g.variant = g.inv ? 1u : (pass == 0 && g.nega ? 2u : 0u);
    g.variant2 = g.inv ? (pass == 1 && g.nega ? 2u : 1u) : 0u;  // DFT-r' image
    g.key = ((u.mod0 << 2) | g.variant) + 1u;
    g.key2 = g.mma2 ? ((((u.mod0 << 2) | g.variant2) << 1) | (g.rl == 4 ? 1u : 0u)) + 1u : 0u;
    return g;
}

// Image copies for a tile whose images differ from those in shared memory
// (thread 0 issues; every thread tracks the keys and the pending copies,
// which the MMA issuer waits for).
__device__ __forceinline__ void tc_images(const BArgs& a, const BUnit& u, const TcGeo& g, TcState& st) {
    uint64_t* bar = reinterpret_cast<uint64_t*>(st.base + kTcBar);
    const uint8_t* blob = a.images + (size_t)u.mod0 * kImgPerMod;
    if (g.key != st.img_key) {
        if (threadIdx.x == 0) {
            const uint8_t* img = blob + (size_t)g.variant * kImgBytes;
            tc::mbar_expect_tx(bar + 1, kImgBytes);
#pragma unroll
            for (uint32_t k = 0; k < 4; k++)
                tc::bulk_g2s(st.base + kTcImg + k * 16384u, img + k * 16384u, 16384u, bar + 1);
        }
        st.img_key = g.key;
        st.pend_img = 1;
    }
    if (g.mma2 && g.key2 != st.img2_key) {
        if (threadIdx.x == 0) {
            const uint32_t bytes = g.rl == 4 ? 4096u : 1024u;
            const uint8_t* img = blob + (g.rl == 4 ? kImg16Off : kImg8Off) + g.variant2 * bytes;
            tc::mbar_expect_tx(bar + 2, bytes);
            tc::bulk_g2s(st.base + kTcImg2, img, bytes, bar + 2);
        }
        st.img2_key = g.key2;
        st.pend_img2 = 1;
    }
}

// L2 lifetimes of a two-pass unit's traffic: every word of a tile's input is
// read once (the unit's data, or its workspace slot in pass B), so it is
// loaded evict-first; pass A's stores to the workspace are read back by
// pass B a few hundred tiles later, so they are kept (evict-last) while the
// batch's data streams past; pass B's results are stored evict-first.
__device__ __forceinline__ void st_keep(uint32_t* p, uint32_t v, uint64_t pol) {
    asm volatile("st.global.L2::cache_hint.u32 [%0], %1, %2;" ::"l"(p), "r"(v), "l"(pol) : "memory");
}

// Operand A: row m = (b2, v) = b2 V + v holds column v0 + v's elements
// j = r' a2 + b2 in K order a2; thread (m, hh) fills 16-byte chunks hh,
// hh + 2, ..  A product's inverse multiplies by the pointwise operand on the way.
// `w64`: the source rows are uint64 words (pass A of a UF_W64 unit).
__device__ __forceinline__ void tc_operand(const BUnit& u, const TcGeo& g, const M32& ar, uint8_t* A, bool w64) {
    const uint32_t mm = threadIdx.x & 127u, hh = threadIdx.x >> 7;
    const size_t off0 = (size_t)(mm >> g.lgV) * g.C + g.v0 + (mm & (g.V - 1u));
    const size_t step = (size_t)g.rp * g.C;  // between consecutive a2
    uint32_t xs[32];
    if (w64) {  // the low words (residues < q)
        const uint64_t* src = reinterpret_cast<const uint64_t*>(g.src);
#pragma unroll
        for (uint32_t j = 0; j < 8; j++)
#pragma unroll
            for (uint32_t t = 0; t < 4; t++)
                xs[4 * j + t] = (uint32_t)__ldcs(src + off0 + (size_t)(8u * j + 4u * hh + t) * step);
    } else {
#pragma unroll
        for (uint32_t j = 0; j < 8; j++)
#pragma unroll
            for (uint32_t t = 0; t < 4; t++) xs[4 * j + t] = __ldcs(g.src + off0 + (size_t)(8u * j + 4u * hh + t) * step);
    }
    if (g.pre) {
#pragma unroll
        for (uint32_t j = 0; j < 8; j++)
#pragma unroll
            for (uint32_t t = 0; t < 4; t++)
                xs[4 * j + t] = ar.mul(xs[4 * j + t], __ldcg(u.pre_mul + off0 + (size_t)(8u * j + 4u * hh + t) * step));
    }
#pragma unroll
    for (uint32_t j = 0; j < 8; j++)
        *reinterpret_cast<uint4*>(A + tc::sw128_offset(mm, 16u * (2u * j + hh), 128)) =
            make_uint4(xs[4 * j], xs[4 * j + 1], xs[4 * j + 2], xs[4 * j + 3]);
}

// Publishes a tile's completion (thread 0, after a CTA barrier that followed
// the tile's stores): release at gpu scope, cumulative over the CTA's stores.
__device__ __forceinline__ void signal_done(uint32_t* counter) {
    __threadfence();
    asm volatile("red.release.gpu.global.add.u32 [%0], 1;" ::"l"(counter) : "memory");
}

// Pass B, warp 0, after the CTA barrier that follows the tile's workspace
// loads: counts the tile into its line group; the group's last tile drops the
// group's lines (one 128-byte line per row of the slot: columns 32 gi ..
// 32 gi + 32; with V >= 32 the tile's own V / 32 lines per row).  The slot's
// next owner waits for every pass B tile of this unit before writing it.
__device__ __forceinline__ void discard_read_lines(const BArgs& a, const BUnit& u, const TcGeo& g, uint32_t tile) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t grp = g.V >= 32u ? 1u : 32u / g.V, gi = tile / grp;
    uint32_t last = 1;
    if (grp > 1) {
        // relaxed: the members' loads have returned (their values are in
        // shared memory, behind the CTA barrier) before they count in
        if (lane == 0)
            last = atomicAdd(a.ctr + 1 + 2 * a.n_units + u.dis + gi, 1u) + 1u == min(grp, u.tiles_b - gi * grp);
        last = __shfl_sync(~0u, last, 0);
    }
    if (!last) return;
    const uint32_t per_row = grp > 1 ? 1u : g.V >> 5, lines = (8192u / g.V) * per_row;
    const uint32_t* first = g.src + (grp > 1 ? 32u * gi : g.v0);
    for (uint32_t i = lane; i < lines; i += 32u)
        asm volatile("discard.global.L2 [%0], 128;" ::"l"(first + (size_t)(i / per_row) * g.C + 32u * (i % per_row))
                     : "memory");
}

__device__ __forceinline__ void run_tc_tile(const BArgs& a, const BUnit& u, uint32_t pass, uint32_t tile, TcState& st) {
    const uint32_t tid = threadIdx.x;
    const TcGeo g = tc_geo(a, u, pass, tile);
    const uint32_t L = g.L, n = g.n, shift = g.shift, N1 = g.N1, lg = g.lg, rl = g.rl, rp = g.rp, lgV = g.lgV;
    const uint32_t V = g.V, C = g.C, v0 = g.v0;
    const bool inv = g.inv, nega = g.nega, pre = g.pre, mma2 = g.mma2;
    const BModulus& M = a.mods[u.mod0];
    const M32 ar = M.ar;
    const uint32_t q = ar.q, qinv = ar.qinv;
    const uint32_t wb = inv ? PW_OMEGA_INV : PW_OMEGA;
    uint8_t* base = st.base;
    uint64_t* bar = reinterpret_cast<uint64_t*>(base + kTcBar);
    tc_images(a, u, g, st);
    // level-2 constants: factors, then (CUDA-core level 2) the DFT-r'
    // butterfly twiddles omega_r'^j.  Pass B's negacyclic factors sit in the
    // DFT-r' image when level 2 runs on the tensor cores.
    uint32_t* fac = reinterpret_cast<uint32_t*>(base + kTcFac);
    const bool use_fac = rp > 1 && (pass == 0 || (inv && nega && !mma2));
    if (use_fac) {
        if (pass == 0) {
            if (tid < 128) {
                const uint32_t fv = tid >> rl, k2 = tid & (rp - 1u);
                fac[tid] = pw(M, ar, wb, ((64u * (v0 + fv) * k2) & (n - 1u)) << shift);
            }
        } else if (tid < rp) {
            fac[tid] = pw(M, ar, PW_PSI_INV, (64u * N1 * tid) << shift);
        }
    }
    if (!mma2 && tid >= 128 && tid < 128 + rp / 2)
        fac[tid] = pw(M, ar, wb, (((n >> rl) * (tid - 128)) & (n - 1u)) << shift);
    tc_operand(u, g, ar, base + kTcA, pass == 0 && g.w64);
    tc::fence_proxy_async_smem();
    __syncthreads();
    if (tid == 0) {
        if (st.pend_img) tc_wait(bar + 1, st.ph_img);
        tc::fence_after_sync();
        tca::issue_k256(st.taddr, tc::smem_u32(base + kTcA), 128, tc::smem_u32(base + kTcImg), 256, 256);
        tc::commit(bar);
    }
    if (pass == 1 && u.dis != kNoDiscard && tid < 32) discard_read_lines(a, u, g, tile);  // during the MMA
    if (st.pend_img) {
        st.ph_img ^= 1u;
        st.pend_img = 0;
    }
    // level-1 twiddles of this thread's vector: base * ratio^k1 for k1 = 32 h ..
    const uint32_t wq = tid >> 5, quarter = wq & 3u, h = wq >> 2, lane = tid & 31u;
    const uint32_t m = quarter * 32u + lane, b2 = m >> lgV, vv = m & (V - 1u), col = v0 + vv;
    const uint32_t er = (n >> lg) * b2 + (pass == 0 ? col : 0u);  // < n
    uint32_t ratio = pw(M, ar, wb, er << shift);
    uint32_t start = pw(M, ar, wb, ((er * 32u * h) & (n - 1u)) << shift);
    if (pass == 0 && !inv && nega) start = ar.mul(start, pw(M, ar, PW_PSI, (b2 * C + col) << shift));
    if (pass == 1 && inv) {
        start = ar.mul(start, M.ninv[L]);
        if (nega) {
            ratio = ar.mul(ratio, pw(M, ar, PW_PSI_INV, N1 << shift));
            start = ar.mul(start, pw(M, ar, PW_PSI_INV, (col + 32u * h * N1) << shift));
        }
    }
    if (pre) start = ar.mul(start, M.r2);  // the product's Montgomery factor 2^-32
    __syncwarp();
    tc_wait(bar, st.ph_mma);
    st.ph_mma ^= 1u;
    tc::fence_after_sync();
    // level-1 epilogue, values in [0, 2q): the level-2 operand (row (v, k1),
    // word b2) when level 2 runs on the tensor cores, else W[m][k1] at
    // m * 64 + (k1 & 32) + ((k1 ^ m) & 31)
    {
        const uint32_t r2 = tca::canon(tca::mont_lazy(ratio, ratio, q, qinv), q);
        uint32_t tw_e = start;
        uint32_t tw_o = tca::canon(tca::mont_lazy(start, ratio, q, qinv), q);
        const uint32_t tcol = st.taddr + h * 128u + ((quarter * 32u) << 16);
        uint32_t* Wrow = reinterpret_cast<uint32_t*>(base + kTcA) + m * 64u + 32u * h;
        uint8_t* A2 = base + kTcA;
#pragma unroll 1
        for (uint32_t part = 0; part < 4; part++) {
            uint32_t c0[8], c1[8], c2[8], c3[8];
            tca::ld_planes8(tcol + 8u * part, c0, c1, c2, c3);
            uint32_t y[8];
#pragma unroll
            for (uint32_t i = 0; i < 8; i += 2) {
                y[i] = tca::mont_lazy(tca::combine_redc(c0[i], c1[i], c2[i], c3[i], q, qinv), tw_e, q, qinv);
                y[i + 1] =
                    tca::mont_lazy(tca::combine_redc(c0[i + 1], c1[i + 1], c2[i + 1], c3[i + 1], q, qinv), tw_o, q, qinv);
                tw_e = tca::canon(tca::mont_lazy(tw_e, r2, q, qinv), q);
                tw_o = tca::canon(tca::mont_lazy(tw_o, r2, q, qinv), q);
            }
            if (mma2) {
                const uint32_t k0 = 32u * h + 8u * part;
                if (pass == 0) {
                    if (rl == 4) l2_store8<0, 4>(A2, y, vv, b2, k0);
                    else l2_store8<0, 3>(A2, y, vv, b2, k0);
                } else {
                    if (rl == 4) l2_store8<1, 4>(A2, y, vv, b2, k0);
                    else l2_store8<1, 3>(A2, y, vv, b2, k0);
                }
            } else {
#pragma unroll
                for (uint32_t i = 0; i < 8; i++) Wrow[(8u * part + i) ^ lane] = y[i];
            }
        }
    }
    if (!mma2) {
        tc::fence_before_sync();
        __syncthreads();
        const uint32_t* W = reinterpret_cast<const uint32_t*>(base + kTcA);
        switch (rl) {
            case 0: tc_level2<0>(u, pass, v0, N1, ar, W, fac, use_fac); break;
            case 1: tc_level2<1>(u, pass, v0, N1, ar, W, fac, use_fac); break;
            default: tc_level2<2>(u, pass, v0, N1, ar, W, fac, use_fac); break;
        }
        return;
    }
    // level 2 on the tensor cores: M-tile t = rows 128 t .. into TMEM columns
    // t * 4 r' + a r' + k2 (the level-1 accumulators are all read by now)
    const uint32_t n_mt = 64u >> rl;  // 4 (r' = 16) or 8 (r' = 8) M-tiles of 128 rows
    tc::fence_proxy_async_smem();
    tc::fence_before_sync();
    __syncthreads();
    if (tid == 0) {
        if (st.pend_img2) tc_wait(bar + 2, st.ph_img2);
        tc::fence_after_sync();
        const uint32_t a2 = tc::smem_u32(base + kTcA), bi = tc::smem_u32(base + kTcImg2);
        const uint32_t idesc = tc::idesc_u8(128, 4u << rl);
        for (uint32_t t = 0; t < n_mt; t++) {
            if (rl == 4) {
                tc::mma_i8(st.taddr + t * 64u, tc::desc_k_sw64(a2 + t * 8192u), tc::desc_k_sw64(bi), idesc, 0);
                tc::mma_i8(st.taddr + t * 64u, tc::desc_k_sw64(a2 + t * 8192u + 32u), tc::desc_k_sw64(bi + 32u), idesc, 1);
            } else {
                tc::mma_i8(st.taddr + t * 32u, tc::desc_k_sw32(a2 + t * 4096u), tc::desc_k_sw32(bi), idesc, 0);
            }
        }
        tc::commit(bar);
    }
    if (st.pend_img2) {
        st.ph_img2 ^= 1u;
        st.pend_img2 = 0;
    }
    __syncwarp();
    tc_wait(bar, st.ph_mma);
    st.ph_mma ^= 1u;
    tc::fence_after_sync();
    // level-2 epilogue: thread (quarter, h) reads lane 32 quarter + lane of the
    // M-tiles h, h + 2, ..; 8 outputs k2 at a time (planes r' columns apart)
    const uint64_t keep = tc::l2_policy_evict_last();
#pragma unroll 1
    for (uint32_t t = h; t < n_mt; t += 2) {
        const uint32_t row = 128u * t + 32u * quarter + lane;
        uint32_t v, k1;
        if (pass == 0) {
            v = row >> 6;
            k1 = (row & 63u) ^ (v & 7u);
        } else {
            v = row & (V - 1u);
            k1 = row >> lgV;
        }
        const uint32_t tc0 = st.taddr + t * (4u << rl) + ((quarter * 32u) << 16);
#pragma unroll 1
        for (uint32_t gq = 0; gq < rp / 8; gq++) {
            uint32_t c0[8], c1[8], c2[8], c3[8];
            tc::ld_32x32b_x8(tc0 + 8u * gq, c0);
            tc::ld_32x32b_x8(tc0 + rp + 8u * gq, c1);
            tc::ld_32x32b_x8(tc0 + 2u * rp + 8u * gq, c2);
            tc::ld_32x32b_x8(tc0 + 3u * rp + 8u * gq, c3);
            tc::ld_wait();
            if (pass == 0) {
                uint32_t* o = u.ws + (size_t)(v0 + v) * N1 + k1;
#pragma unroll
                for (uint32_t i = 0; i < 8; i++) {
                    const uint32_t k2 = 8u * gq + i;
                    const uint32_t y = tca::combine_redc(c0[i], c1[i], c2[i], c3[i], q, qinv);
                    st_keep(o + 64u * k2, tca::canon(tca::mont_lazy(y, fac[v * rp + k2], q, qinv), q), keep);
                }
            } else if (g.w64) {
                uint64_t* o = reinterpret_cast<uint64_t*>(u.data) + (size_t)k1 * N1 + v0 + v;
#pragma unroll
                for (uint32_t i = 0; i < 8; i++) {
                    const uint32_t k2 = 8u * gq + i;
                    __stcs(o + (size_t)64u * k2 * N1,
                           (uint64_t)tca::canon(tca::combine_redc(c0[i], c1[i], c2[i], c3[i], q, qinv), q));
                }
            } else {
                uint32_t* o = u.data + (size_t)k1 * N1 + v0 + v;
#pragma unroll
                for (uint32_t i = 0; i < 8; i++) {
                    const uint32_t k2 = 8u * gq + i;
                    __stcs(o + (size_t)64u * k2 * N1, tca::canon(tca::combine_redc(c0[i], c1[i], c2[i], c3[i], q, qinv), q));
                }
            }
        }
    }
}

// The persistent queue with tensor-core tiles (256 threads, two CTAs per SM,
// 256 TMEM columns each); units without UF_TC run the CUDA-core tile.
template <uint32_t G>
__global__ void __launch_bounds__(256, 2) batch_queue_tc(const __grid_constant__ BArgs a) {
    extern __shared__ __align__(1024) uint8_t tc_raw[];
    __shared__ uint32_t s_ticket, s_taddr;
    __shared__ M32 s_ar[kMaxRows];
    TcState st;
    st.base = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(tc_raw) + 1023) & ~uintptr_t(1023));
    uint64_t* bar = reinterpret_cast<uint64_t*>(st.base + kTcBar);
    if (threadIdx.x == 0) {
        tc::mbar_init(bar, 1);
        tc::mbar_init(bar + 1, 1);
        tc::mbar_init(bar + 2, 1);
    }
    if (threadIdx.x < 32) tc::tmem_alloc(&s_taddr, 256);
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    st.taddr = s_taddr;
    st.ph_mma = st.ph_img = st.ph_img2 = 0;
    st.img_key = st.img2_key = 0;
    st.pend_img = st.pend_img2 = 0;
    for (;;) {
        if (threadIdx.x == 0) s_ticket = atomicAdd(a.ctr, 1u);
        __syncthreads();
        const uint32_t ticket = s_ticket;
        if (ticket >= a.n_tiles) break;
        const BTile tl = a.tiles[ticket];
#if NTTB_DEBUG_BOUNDS
        if (!tile_in_range(a, tl)) {  // uniform over the CTA: every thread read the same tile
            __syncthreads();          // s_ticket is read by every thread before it is rewritten
            continue;
        }
#endif
        const BUnit u = a.units[tl.unit];
        const uint32_t pass = tl.pass_tile >> 31, tile = tl.pass_tile & 0x7fffffffu;
        if (threadIdx.x == 0 && !wait_deps(a, u, tl.unit, pass)) atomicOr(&g_batch_error, 1u);
        __syncthreads();
        if (u.flags & UF_TC) {
            run_tc_tile(a, u, pass, tile, st);
        } else {
            run_tile<256, G>(a, u, pass, tile, reinterpret_cast<uint32_t*>(st.base), s_ar);
            st.img_key = st.img2_key = 0;  // the tile overwrote the images
        }
        tc::fence_proxy_async_smem();
        tc::fence_before_sync();
        __syncthreads();
        if (threadIdx.x == 0) signal_done(a.ctr + 1 + 2 * tl.unit + pass);
    }
    tc::fence_before_sync();
    __syncthreads();
    if (threadIdx.x < 32) tc::tmem_dealloc(st.taddr, 256);
}

template <uint32_t E, uint32_t T, uint32_t G>
// more resident CTAs for the small register groups
__global__ void __launch_bounds__(T, (G == 1 ? 1536u : G == 3 ? 768u : 512u) / T) batch_queue(const __grid_constant__ BArgs a) {
    extern __shared__ __align__(16) uint32_t sm[];
    __shared__ uint32_t s_ticket;
    __shared__ M32 s_ar[kMaxRows];
    for (;;) {
        if (threadIdx.x == 0) s_ticket = atomicAdd(a.ctr, 1u);
        __syncthreads();
        const uint32_t ticket = s_ticket;
        if (ticket >= a.n_tiles) break;
        const BTile tl = a.tiles[ticket];
#if NTTB_DEBUG_BOUNDS
        if (!tile_in_range(a, tl)) {  // uniform over the CTA: every thread read the same tile
            __syncthreads();          // s_ticket is read by every thread before it is rewritten
            continue;
        }
#endif
        const BUnit u = a.units[tl.unit];
        const uint32_t pass = tl.pass_tile >> 31, tile = tl.pass_tile & 0x7fffffffu;
        if (threadIdx.x == 0 && !wait_deps(a, u, tl.unit, pass)) atomicOr(&g_batch_error, 1u);
        __syncthreads();
        run_tile<T, G>(a, u, pass, tile, sm, s_ar);
        __syncthreads();
        if (threadIdx.x == 0) signal_done(a.ctr + 1 + 2 * tl.unit + pass);
    }
}

// ---- host ------------------------------------------------------------------------
struct Variant {
    uint32_t E, T, G, tensor;
    void (*fn)(BArgs);
};
const Variant kVariants[] = {
    {4096, 256, 1, 0, batch_queue<4096, 256, 1>},    {4096, 256, 3, 0, batch_queue<4096, 256, 3>},
    {4096, 256, 4, 0, batch_queue<4096, 256, 4>},    {8192, 256, 1, 0, batch_queue<8192, 256, 1>},
    {8192, 256, 3, 0, batch_queue<8192, 256, 3>},    {8192, 256, 4, 0, batch_queue<8192, 256, 4>},
    {8192, 512, 1, 0, batch_queue<8192, 512, 1>},    {8192, 512, 3, 0, batch_queue<8192, 512, 3>},
    {8192, 512, 4, 0, batch_queue<8192, 512, 4>},    {16384, 512, 1, 0, batch_queue<16384, 512, 1>},
    {16384, 512, 3, 0, batch_queue<16384, 512, 3>},  {16384, 512, 4, 0, batch_queue<16384, 512, 4>},
    // tensor-core tiles for the two-pass units, CUDA-core tiles of 4096 / 8192 for the rest
    {4096, 256, 1, 1, batch_queue_tc<1>},            {4096, 256, 3, 1, batch_queue_tc<3>},
    {4096, 256, 4, 1, batch_queue_tc<4>},            {8192, 256, 1, 1, batch_queue_tc<1>},
    {8192, 256, 3, 1, batch_queue_tc<3>},            {8192, 256, 4, 1, batch_queue_tc<4>},
};

const Variant* find_variant(uint32_t E, uint32_t T, uint32_t G, uint32_t tensor) {
    for (const Variant& v : kVariants)
        if (v.E == E && v.T == T && v.G == G && v.tensor == tensor) return &v;
    return nullptr;
}

// padded tile (E + E/32 + one word per vector) + root powers + slack, in bytes
size_t smem_bytes(uint32_t E) { return ((size_t)E + E / 16 + kMaxRows + E / 2) * 4 + 64; }
size_t smem_bytes(const Variant* v) { return v->tensor ? kTcSmem : smem_bytes(v->E); }

// Byte-plane image of an 8 x 8 matrix for the level-2 contraction: 32 rows
// (a, k) x 32 bytes (j, p), K-major SW32 (1 KB).
void build_image8(uint8_t* img, const std::vector<uint64_t>& W, uint64_t q) {
    std::memset(img, 0, 1024);
    for (uint32_t c = 0; c < 8; c++)
        for (uint32_t b = 0; b < 8; b++)
            for (uint32_t p = 0; p < 4; p++) {
                const uint64_t v = h_mulmod(h_to_mont32(W[c * 8 + b], q), (1ull << (8 * p)) % q, q);
                for (uint32_t a = 0; a < 4; a++) img[tc::sw32_offset(a * 8 + c, 4 * b + p)] = (uint8_t)(v >> (8 * a));
            }
}

// CTAs of a variant resident on the whole device (the persistent grid): the
// kernel asks for the largest shared-memory carveout, so that the tensor-tile
// kernel's ~100 KB CTAs fit two per SM.
int resident_ctas(const Variant* v, uint32_t ctas_per_sm) {
    const size_t smem = smem_bytes(v);
    cudaFuncSetAttribute(v->fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    cudaFuncSetAttribute(v->fn, cudaFuncAttributePreferredSharedMemoryCarveout, (int)cudaSharedmemCarveoutMaxShared);
    int dev = 0, sms = 0, occ = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, v->fn, (int)v->T, smem) != cudaSuccess) {
        cudaGetLastError();
        occ = 1;
    }
    if (v->tensor) {
        // The runtime's answer for the tcgen05 kernel is one CTA per SM; its
        // registers and shared memory fit two (and TMEM holds two 256-column
        // allocations), so count from the resources themselves.
        cudaFuncAttributes fa{};
        int smem_sm = 0, regs_sm = 0, reserved = 0;
        cudaFuncGetAttributes(&fa, v->fn);
        cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev);
        cudaDeviceGetAttribute(&regs_sm, cudaDevAttrMaxRegistersPerMultiprocessor, dev);
        cudaDeviceGetAttribute(&reserved, cudaDevAttrReservedSharedMemoryPerBlock, dev);
        const size_t per_smem = fa.sharedSizeBytes + smem + (size_t)reserved;
        const size_t per_regs = (size_t)((fa.numRegs * 32 + 255) / 256 * 256) * (v->T / 32);
        int fit = 2;  // TMEM: 512 columns per SM
        if (per_smem) fit = std::min<int>(fit, (int)(smem_sm / per_smem));
        if (per_regs) fit = std::min<int>(fit, (int)(regs_sm / per_regs));
        occ = std::max(occ, fit);
    }
    if (occ < 1) occ = 1;
    if (ctas_per_sm && (int)ctas_per_sm < occ) occ = (int)ctas_per_sm;
    return sms * occ;
}

uint32_t ilog2(uint64_t x) {
    uint32_t l = 0;
    while ((1ull << l) < x) l++;
    return l;
}

}  // namespace

struct BatchPlan::Mods {
    BModulus* d = nullptr;
};

struct Batch {
    BatchPlan* plan = nullptr;
    nttb_batch_config cfg{};
    const Variant* var = nullptr;
    BUnit* d_units = nullptr;
    BTile* d_tiles = nullptr;
    uint32_t* d_ctr = nullptr;
    uint32_t* d_ws = nullptr;
    uint32_t n_units = 0, n_tiles = 0, n_dis = 0;
    size_t ws_bytes = 0;
    int grid = 0;
    cudaGraphExec_t gexec = nullptr;
    cudaGraph_t graph = nullptr;
    cudaStream_t cap = nullptr;
};

namespace {

nttb_batch_config default_config() {
    nttb_batch_config c{};
    c.tile_elems = 4096;
    c.threads = 256;
    c.split = 1;
    c.lag = 4;
    c.ctas_per_sm = 0;
    c.group = 3;
    c.tensor = 1;
    return c;
}

int check_config(const nttb_batch_config& c) {
    if (c.tensor > 1) return fail(NTTB_ERR_INVALID_ARG, "batch config: tensor must be 0 or 1");
    if (!find_variant(c.tile_elems, c.threads, c.group, 0))
        return fail(NTTB_ERR_INVALID_ARG,
                    "batch config: tile_elems/threads must be 4096/256, 8192/256, 8192/512 or 16384/512, group 1, 3 or 4");
    if (c.split > 1) return fail(NTTB_ERR_INVALID_ARG, "batch config: split must be 0 or 1");
    if (c.lag < 1 || c.lag > 64) return fail(NTTB_ERR_INVALID_ARG, "batch config: lag must be in [1, 64]");
    return 0;
}

void free_batch(Batch* b) {
    if (b->gexec) cudaGraphExecDestroy(b->gexec);
    if (b->graph) cudaGraphDestroy(b->graph);
    if (b->cap) cudaStreamDestroy(b->cap);
    cudaFree(b->d_units);
    cudaFree(b->d_tiles);
    cudaFree(b->d_ctr);
    cudaFree(b->d_ws);
    delete b;
}

// Tensor-core tiles are used where the configuration has a tensor kernel
// (256 threads, CUDA-core tiles of 4096 or 8192 residues for the other units).
bool tensor_tiles(const nttb_batch_config& cfg) {
    return cfg.tensor && find_variant(cfg.tile_elems, cfg.threads, cfg.group, 1);
}

// Pass geometry of a unit of 2^L residues (rows: limbs per single-pass tile).
struct UnitShape {
    uint32_t lg1 = 0, per = 1, va = 0, vb = 0, tiles_a = 1, tiles_b = 0;
    bool tc = false;
};
bool unit_shape(const BatchPlan& P, const nttb_batch_config& cfg, uint32_t L, UnitShape* s) {
    const uint32_t E = cfg.tile_elems, lgE = ilog2(E), n = 1u << L;
    *s = UnitShape();
    // tensor-core two-pass units: both pass lengths 64 r', r' in 1..16
    s->tc = tensor_tiles(cfg) && P.images && L > lgE && L >= 13 && L <= 20;
    if (L <= lgE) {
        s->per = std::min<uint32_t>(E >> L, kMaxRows);
        return true;
    }
    uint32_t lg1 = cfg.split ? L / 2 : (L + 1) / 2;
    if (s->tc) {
        lg1 = std::max<uint32_t>(lg1, std::max<uint32_t>(6, L - 10));
        lg1 = std::min<uint32_t>(lg1, std::min<uint32_t>(10, L - 6));
        s->va = 128u >> (lg1 - 6);  // 8192 residues per tile: V = 128 / r' columns of length 64 r'
        s->vb = 128u >> (L - lg1 - 6);
    } else {
        if (lg1 > lgE) lg1 = lgE;
        if (L - lg1 > lgE) lg1 = L - lgE;
        if (lg1 > lgE || lg1 == 0) return false;
        s->va = std::min(E >> lg1, n >> lg1);
        s->vb = std::min(E >> (L - lg1), 1u << lg1);
    }
    s->lg1 = lg1;
    s->tiles_a = (n >> lg1) / s->va;
    s->tiles_b = (1u << lg1) / s->vb;
    return true;
}

// Workspace of the two-pass units: one ring per size class 2^L, S_L slots of
// 2^L words each: at least 16 units and more than the lag, and for a batch
// (count given) enough for ~1024 pass A tiles in flight unless the class has
// fewer units.  Runners (count null) keep 16 per class: their job lists are
// small.  A unit waits for the previous owner of its slot (same class) to
// finish its pass B.
struct WsLayout {
    uint64_t base[25] = {};  // words
    uint32_t slots[25] = {};
    uint64_t words = 0;
};
WsLayout ws_layout(const BatchPlan& P, const nttb_batch_config& cfg, const uint32_t* count) {
    WsLayout w;
    for (uint32_t L = 1; L <= P.max_log; L++) {
        UnitShape sh;
        if (!unit_shape(P, cfg, L, &sh) || !sh.lg1) continue;
        if (count && !count[L]) continue;
        uint32_t S = std::max<uint32_t>(16, cfg.lag + 2);
        if (count) S = std::min(std::max(S, (1024 + sh.tiles_a - 1) / sh.tiles_a), count[L]);
        w.base[L] = w.words;
        w.slots[L] = S;
        w.words += (uint64_t)S << L;
    }
    return w;
}

// Units, queue order and workspace ring of one batch (host work only).
// Units of phase 0 (plain jobs, forward halves of products) come first,
// largest first; phase 1 holds the inverse units of products, which depend
// on phase-0 units.  Every pass B tile deferred by the lag is flushed at the
// phase boundary, so each awaited tile precedes its waiter in the queue.
int plan_batch(const BatchPlan& P, const nttb_batch_job* jobs, uint32_t n_jobs, const nttb_batch_config& cfg,
               std::vector<BUnit>& units, std::vector<BTile>& tiles, const WsLayout* fixed, WsLayout* layout_out) {
    const uint32_t E = cfg.tile_elems;
    struct Pending {
        BUnit u;
        uint64_t work;
        uint32_t phase, id;
        int32_t after_id[2];
    };
    std::vector<Pending> list;
    // Units of one transform over rows [l0, l0 + rows) of `data`.
    auto add_units = [&](uint32_t j, uint32_t* data, const void* in, const uint32_t* pre_mul, uint32_t L,
                         uint32_t first, uint32_t n_limbs, uint32_t uf, uint32_t phase, std::vector<uint32_t>* ids,
                         const std::vector<uint32_t>* dep_a, const std::vector<uint32_t>* dep_b) -> int {
        const uint32_t n = 1u << L;
        UnitShape sh;
        if (!unit_shape(P, cfg, L, &sh))
            return fail(NTTB_ERR_INVALID_ARG, "batch job %u: log_n %u too large for tile %u", j, L, E);
        const uint32_t lg1 = sh.lg1, per = sh.per;
        const bool tcu = sh.tc;
        if ((uf & UF_W64 || in) && !(tcu && lg1))
            return fail(NTTB_ERR_UNSUPPORTED, "batch job %u: uint64 words or a separate source need tensor tiles", j);
        const size_t es = (uf & UF_W64) ? 8 : 4;  // bytes per residue of data and in
        uint32_t k = 0;
        for (uint32_t l0 = 0; l0 < n_limbs; l0 += per, k++) {
            Pending p{};
            BUnit& u = p.u;
            u.data = reinterpret_cast<uint32_t*>(reinterpret_cast<char*>(data) + (size_t)l0 * n * es);
            u.in = in ? static_cast<const char*>(in) + (size_t)l0 * n * es : nullptr;
            u.pre_mul = pre_mul ? pre_mul + (size_t)l0 * n : nullptr;
            u.mod0 = first + l0;
            u.log_n = L;
            u.flags = uf | (tcu ? UF_TC : 0u);
            u.lg1 = lg1;
            u.rows = lg1 ? 1u : std::min(per, n_limbs - l0);
            u.va = sh.va;
            u.vb = sh.vb;
            u.tiles_a = sh.tiles_a;
            u.tiles_b = sh.tiles_b;
            u.prev = -1;
            u.after[0] = u.after[1] = -1;
            p.work = (uint64_t)u.rows * n * L;
            p.phase = phase;
            p.id = (uint32_t)list.size();
            p.after_id[0] = dep_a ? (int32_t)(*dep_a)[k] : -1;
            p.after_id[1] = dep_b ? (int32_t)(*dep_b)[k] : -1;
            if (ids) ids->push_back(p.id);
            list.push_back(p);
        }
        return 0;
    };
    for (uint32_t j = 0; j < n_jobs; j++) {
        const nttb_batch_job& J = jobs[j];
        if (!J.data) return fail(NTTB_ERR_INVALID_ARG, "batch job %u: null data", j);
        if (J.log_n < 1 || J.log_n > P.max_log)
            return fail(NTTB_ERR_INVALID_ARG, "batch job %u: log_n %u outside [1, %u]", j, J.log_n, P.max_log);
        if (J.n_limbs == 0 || (uint64_t)J.first_modulus + J.n_limbs > P.limbs.size())
            return fail(NTTB_ERR_INVALID_ARG, "batch job %u: limbs [%u, %u) outside the plan's %zu moduli", j,
                        J.first_modulus, J.first_modulus + J.n_limbs, P.limbs.size());
        if ((J.flags & NTTB_NEGACYCLIC) && !P.negacyclic)
            return fail(NTTB_ERR_INVALID_ARG, "batch job %u: negacyclic job on a cyclic plan", j);
        const uint32_t nega = (J.flags & NTTB_NEGACYCLIC) ? UF_NEGA : 0u;
        const uint32_t w64 = (J.flags & kJobW64) ? UF_W64 : 0u;
        const void* in = (J.flags & kJobSrc) ? static_cast<const void*>(J.pointwise) : nullptr;
        if ((J.flags & kJobSrc) && (!in || in == J.data))
            return fail(NTTB_ERR_INVALID_ARG, "batch job %u: a separate source must be given and distinct", j);
        if ((J.flags & NTTB_BATCH_POLYMUL) && (w64 || in))
            return fail(NTTB_ERR_INVALID_ARG, "batch job %u: products take uint32 residues in place", j);
        if (J.flags & NTTB_BATCH_POLYMUL) {
            if (!J.pointwise || J.pointwise == J.data)
                return fail(NTTB_ERR_INVALID_ARG, "batch job %u: a product needs a distinct second operand", j);
            std::vector<uint32_t> fa, fb;
            if (int rc = add_units(j, J.data, nullptr, nullptr, J.log_n, J.first_modulus, J.n_limbs, nega, 0, &fa,
                                   nullptr, nullptr))
                return rc;
            if (int rc = add_units(j, const_cast<uint32_t*>(J.pointwise), nullptr, nullptr, J.log_n, J.first_modulus,
                                   J.n_limbs, nega, 0, &fb, nullptr, nullptr))
                return rc;
            if (int rc = add_units(j, J.data, nullptr, J.pointwise, J.log_n, J.first_modulus, J.n_limbs, nega | UF_INV, 1,
                                   nullptr, &fa, &fb))
                return rc;
        } else {
            const uint32_t uf = ((J.flags & NTTB_BATCH_INVERSE) ? UF_INV : 0u) | nega | w64;
            if (int rc = add_units(j, J.data, in, nullptr, J.log_n, J.first_modulus, J.n_limbs, uf, 0, nullptr, nullptr,
                                   nullptr))
                return rc;
        }
    }
    // phase by phase, largest units first
    std::stable_sort(list.begin(), list.end(), [](const Pending& x, const Pending& y) {
        return x.phase != y.phase ? x.phase < y.phase : x.work > y.work;
    });
    std::vector<int32_t> index_of(list.size());
    for (size_t i = 0; i < list.size(); i++) index_of[list[i].id] = (int32_t)i;
    uint32_t count[25] = {};
    for (const Pending& p : list)
        if (p.u.lg1) count[p.u.log_n]++;
    const WsLayout lay = fixed ? *fixed : ws_layout(P, cfg, count);
    for (uint32_t L = 1; L < 25; L++)
        if (count[L] && !lay.slots[L]) return fail(NTTB_ERR_INVALID_ARG, "batch: no workspace ring for log_n %u", L);
    const uint32_t lag = cfg.lag;
    units.clear();
    tiles.clear();
    std::vector<std::vector<int32_t>> slot_owner(25);
    for (uint32_t L = 1; L < 25; L++) slot_owner[L].assign(lay.slots[L], -1);
    uint32_t next_slot[25] = {};
    uint32_t n_dis = 0;
    std::deque<uint32_t> pend_b;
    uint32_t phase = 0;
    auto emit_b = [&](uint32_t ui) {
        for (uint32_t t = 0; t < units[ui].tiles_b; t++) tiles.push_back({ui, 0x80000000u | t});
    };
    auto flush = [&]() {
        while (!pend_b.empty()) {
            emit_b(pend_b.front());
            pend_b.pop_front();
        }
    };
    for (const Pending& p : list) {
        if (p.phase != phase) {
            flush();
            phase = p.phase;
        }
        const uint32_t ui = (uint32_t)units.size();
        BUnit u = p.u;
        for (int d = 0; d < 2; d++) {
            u.after[d] = p.after_id[d] >= 0 ? index_of[p.after_id[d]] : -1;
            if (u.after[d] >= 0) {  // complete = its last pass has signalled every tile
                const BUnit& W = units[u.after[d]];
                u.after_ctr[d] = (W.lg1 ? 2u : 1u) + 2u * (uint32_t)u.after[d];
                u.need[1 + d] = W.lg1 ? W.tiles_b : W.tiles_a;
            }
        }
        u.dis = kNoDiscard;
        if (u.lg1 && (u.flags & UF_TC)) {  // pass B rows span >= 64 words: lines never straddle two rows
            u.dis = n_dis;
            const uint32_t g = discard_group(u.log_n, u.lg1);
            if (g > 1) n_dis += (u.tiles_b + g - 1) / g;
        }
        if (u.lg1) {
            const uint32_t L = u.log_n, slot = next_slot[L]++ % lay.slots[L];
            // word offset, rebased on the workspace allocation later
            u.ws = reinterpret_cast<uint32_t*>((uintptr_t)((lay.base[L] + ((uint64_t)slot << L)) * 4u));
            u.prev = slot_owner[L][slot];
            if (u.prev >= 0) u.need[0] = units[u.prev].tiles_b;
            slot_owner[L][slot] = (int32_t)ui;
        }
        units.push_back(u);
        for (uint32_t t = 0; t < u.tiles_a; t++) tiles.push_back({ui, t});
        if (u.lg1) {
            pend_b.push_back(ui);
            while (pend_b.size() > lag) {
                emit_b(pend_b.front());
                pend_b.pop_front();
            }
        }
    }
    flush();
    if (layout_out) *layout_out = lay;
    return 0;
}

// Discard-group counters the planned units use (after the 1 + 2 units queue counters).
uint32_t discard_counters(const std::vector<BUnit>& units) {
    uint32_t n = 0;
    for (const BUnit& u : units)
        if (u.dis != kNoDiscard) {
            const uint32_t g = discard_group(u.log_n, u.lg1);
            if (g > 1) n = std::max(n, u.dis + (u.tiles_b + g - 1) / g);
        }
    return n;
}

int create_batch(BatchPlan* P, const nttb_batch_job* jobs, uint32_t n_jobs, const nttb_batch_config& cfg, Batch** out) {
    if (int rc = check_config(cfg)) return rc;
    std::vector<BUnit> units;
    std::vector<BTile> tiles;
    WsLayout lay;
    if (int rc = plan_batch(*P, jobs, n_jobs, cfg, units, tiles, nullptr, &lay)) return rc;
    if (tiles.size() >= 0x7fffffffu || units.size() >= 0x7fffffffu)
        return fail(NTTB_ERR_INVALID_ARG, "batch: too many tiles");
    Batch* b = new Batch();
    b->plan = P;
    b->cfg = cfg;
    // without tensor-core units the CUDA-core kernel runs (more CTAs per SM)
    bool any_tc = false;
    for (const BUnit& u : units) any_tc = any_tc || (u.flags & UF_TC);
    b->var = find_variant(cfg.tile_elems, cfg.threads, cfg.group, cfg.tensor && any_tc ? 1u : 0u);
    b->n_units = (uint32_t)units.size();
    b->n_tiles = (uint32_t)tiles.size();
    b->n_dis = discard_counters(units);
    b->ws_bytes = (size_t)lay.words * 4;
    bool ok = true;
    ok = ok && cudaMalloc(&b->d_units, std::max<size_t>(1, units.size()) * sizeof(BUnit)) == cudaSuccess;
    ok = ok && cudaMalloc(&b->d_tiles, std::max<size_t>(1, tiles.size()) * sizeof(BTile)) == cudaSuccess;
    ok = ok && cudaMalloc(&b->d_ctr, (1 + 2 * (size_t)units.size() + b->n_dis) * 4) == cudaSuccess;
    if (ok && b->ws_bytes) ok = cudaMalloc(&b->d_ws, b->ws_bytes) == cudaSuccess;
    if (!ok) {
        free_batch(b);
        return fail(NTTB_ERR_NO_MEMORY, "batch: device allocation failed");
    }
    for (BUnit& u : units)
        if (u.lg1) u.ws = b->d_ws + (reinterpret_cast<uintptr_t>(u.ws) / 4);
    ok = cudaMemcpy(b->d_units, units.data(), units.size() * sizeof(BUnit), cudaMemcpyHostToDevice) == cudaSuccess;
    ok = ok && cudaMemcpy(b->d_tiles, tiles.data(), tiles.size() * sizeof(BTile), cudaMemcpyHostToDevice) == cudaSuccess;
    if (!ok) {
        free_batch(b);
        return fail(NTTB_ERR_CUDA, "batch: upload failed");
    }
    b->grid = (int)std::min<uint64_t>((uint64_t)resident_ctas(b->var, cfg.ctas_per_sm), std::max<uint32_t>(1, b->n_tiles));
    *out = b;
    return 0;
}

// Counter reset + the persistent launch (no allocation, no host synchronisation).
int launch_batch(Batch* b, cudaStream_t s, bool count) {
    if (b->n_tiles == 0) return 0;
    BArgs a{};
    a.mods = b->plan->mods->d;
    a.units = b->d_units;
    a.tiles = b->d_tiles;
    a.ctr = b->d_ctr;
    a.n_tiles = b->n_tiles;
    a.max_log = b->plan->max_log;
    a.images = b->plan->images;
    a.n_units = b->n_units;
    a.ws = b->d_ws;
    a.ws_words = b->ws_bytes / 4;
    a.n_dis = b->n_dis;
    if (cudaMemsetAsync(b->d_ctr, 0, (1 + 2 * (size_t)b->n_units + b->n_dis) * 4, s) != cudaSuccess)
        return fail(NTTB_ERR_CUDA, "batch: counter reset failed");
    if (count) {
        ProfScope prof("batch_queue", s);
        b->var->fn<<<b->grid, b->var->T, smem_bytes(b->var), s>>>(a);
    } else {
        b->var->fn<<<b->grid, b->var->T, smem_bytes(b->var), s>>>(a);
    }
    return cudaGetLastError() == cudaSuccess ? 0 : fail(NTTB_ERR_CUDA, "batch: launch failed");
}

}  // namespace

// ---- runner: repeated batches without per-batch allocation -----------------------
struct BatchRunner {
    BatchPlan* plan = nullptr;
    nttb_batch_config cfg{};
    const Variant* var = nullptr;
    BUnit* d_units = nullptr;
    BTile* d_tiles = nullptr;
    uint32_t* d_ctr = nullptr;
    uint32_t* d_ws = nullptr;
    BUnit* h_units = nullptr;  // pinned staging
    BTile* h_tiles = nullptr;
    size_t cap_units = 0, cap_tiles = 0, ws_bytes = 0;
    WsLayout layout;
    int grid = 0;
    std::vector<BUnit> units;
    std::vector<BTile> tiles;
};

namespace {
void runner_free_queue(BatchRunner* r) {
    cudaFree(r->d_units);
    cudaFree(r->d_tiles);
    cudaFree(r->d_ctr);
    cudaFreeHost(r->h_units);
    cudaFreeHost(r->h_tiles);
    r->d_units = nullptr;
    r->d_tiles = nullptr;
    r->d_ctr = nullptr;
    r->h_units = nullptr;
    r->h_tiles = nullptr;
    r->cap_units = r->cap_tiles = 0;
}
int runner_reserve(BatchRunner* r, size_t units, size_t tiles) {
    if (units <= r->cap_units && tiles <= r->cap_tiles) return 0;
    const size_t cu = std::max(units, r->cap_units * 2), ct = std::max(tiles, r->cap_tiles * 2);
    runner_free_queue(r);
    bool ok = cudaMalloc(&r->d_units, cu * sizeof(BUnit)) == cudaSuccess;
    ok = ok && cudaMalloc(&r->d_tiles, ct * sizeof(BTile)) == cudaSuccess;
    ok = ok && cudaMalloc(&r->d_ctr, (1 + 2 * cu + ct) * 4) == cudaSuccess;  // discard groups <= tiles
    ok = ok && cudaMallocHost(&r->h_units, cu * sizeof(BUnit)) == cudaSuccess;
    ok = ok && cudaMallocHost(&r->h_tiles, ct * sizeof(BTile)) == cudaSuccess;
    if (!ok) {
        runner_free_queue(r);
        return fail(NTTB_ERR_NO_MEMORY, "batch runner: queue allocation failed");
    }
    r->cap_units = cu;
    r->cap_tiles = ct;
    return 0;
}
}  // namespace

int runner_create(BatchPlan* P, const nttb_batch_config& cfg, BatchRunner** out) {
    if (int rc = check_config(cfg)) return rc;
    auto* r = new BatchRunner();
    r->plan = P;
    r->cfg = cfg;
    r->var = find_variant(cfg.tile_elems, cfg.threads, cfg.group, tensor_tiles(cfg) ? 1u : 0u);
    r->layout = ws_layout(*P, cfg, nullptr);  // rings for every size class the plan allows
    r->ws_bytes = (size_t)r->layout.words * 4;
    if ((r->ws_bytes && cudaMalloc(&r->d_ws, r->ws_bytes) != cudaSuccess) || runner_reserve(r, 256, 4096)) {
        runner_destroy(r);
        return fail(NTTB_ERR_NO_MEMORY, "batch runner: allocation failed");
    }
    r->grid = resident_ctas(r->var, cfg.ctas_per_sm);
    *out = r;
    return 0;
}

void runner_destroy(BatchRunner* r) {
    if (!r) return;
    runner_free_queue(r);
    cudaFree(r->d_ws);
    delete r;
}

size_t runner_device_bytes(const BatchRunner* r) {
    return r->ws_bytes + r->cap_units * (sizeof(BUnit) + 8) + r->cap_tiles * (sizeof(BTile) + 4);
}

// Plans the jobs, uploads the queue from pinned staging and launches, all on
// `s`.  One run per runner may be in flight: the staging is reused.
int runner_run(BatchRunner* r, const nttb_batch_job* jobs, uint32_t n_jobs, cudaStream_t s) {
    if (int rc = plan_batch(*r->plan, jobs, n_jobs, r->cfg, r->units, r->tiles, &r->layout, nullptr)) return rc;
    if (r->tiles.empty()) return 0;
    if (r->units.size() > r->cap_units || r->tiles.size() > r->cap_tiles) {
        cudaStreamSynchronize(s);  // the previous run may still read the queue
        if (int rc = runner_reserve(r, r->units.size(), r->tiles.size())) return rc;
    }
    for (size_t i = 0; i < r->units.size(); i++) {
        BUnit u = r->units[i];
        if (u.lg1) u.ws = r->d_ws + (reinterpret_cast<uintptr_t>(u.ws) / 4);
        r->h_units[i] = u;
    }
    std::memcpy(r->h_tiles, r->tiles.data(), r->tiles.size() * sizeof(BTile));
    BArgs a{};
    a.mods = r->plan->mods->d;
    a.units = r->d_units;
    a.tiles = r->d_tiles;
    a.ctr = r->d_ctr;
    a.n_tiles = (uint32_t)r->tiles.size();
    a.max_log = r->plan->max_log;
    a.images = r->plan->images;
    a.n_units = (uint32_t)r->units.size();
    a.ws = r->d_ws;
    a.ws_words = r->ws_bytes / 4;
    a.n_dis = discard_counters(r->units);
    bool ok = cudaMemcpyAsync(r->d_units, r->h_units, r->units.size() * sizeof(BUnit), cudaMemcpyHostToDevice, s) ==
              cudaSuccess;
    ok = ok && cudaMemcpyAsync(r->d_tiles, r->h_tiles, r->tiles.size() * sizeof(BTile), cudaMemcpyHostToDevice, s) ==
                   cudaSuccess;
    ok = ok && cudaMemsetAsync(r->d_ctr, 0, (1 + 2 * r->units.size() + a.n_dis) * 4, s) == cudaSuccess;
    if (!ok) return fail(NTTB_ERR_CUDA, "batch runner: queue upload failed");
    const int grid = (int)std::min<size_t>((size_t)r->grid, r->tiles.size());
    ProfScope prof("batch_queue", s);
    r->var->fn<<<grid, r->var->T, smem_bytes(r->var), s>>>(a);
    return cudaGetLastError() == cudaSuccess ? 0 : fail(NTTB_ERR_CUDA, "batch runner: launch failed");
}

size_t batch_plan_device_bytes(const BatchPlan* P) {
    const uint32_t lo = std::min<uint32_t>(kLoBits, P->max_log);
    return (size_t)P->limbs.size() * 4 * 4 * (((size_t)1 << (P->max_log - lo)) + ((size_t)1 << lo)) +
           P->limbs.size() * sizeof(BModulus) + (P->images ? P->limbs.size() * (size_t)kImgPerMod : 0);
}

uint32_t batch_bounds_errors(bool clear) {
    uint32_t v = 0;
    cudaMemcpyFromSymbol(&v, g_batch_bounds, sizeof v);
    if (clear) {
        uint32_t z = 0;
        cudaMemcpyToSymbol(g_batch_bounds, &z, sizeof z);
    }
    return v;
}

uint32_t batch_device_errors(bool clear) {
    uint32_t v = 0;
    cudaMemcpyFromSymbol(&v, g_batch_error, sizeof v);
    if (clear) {
        uint32_t z = 0;
        cudaMemcpyToSymbol(g_batch_error, &z, sizeof z);
    }
    return v;
}

// ---- plan transforms on the tensor tiles (NTTB_ENGINE_TILES) -----------------------
// A transform of n_polys x n_limbs (polynomial, limb) units of 2^L residues,
// 13 <= L <= 20, as one persistent launch of the queue's tensor tiles: a
// batch plan over the plan's moduli at max_log = L (the same roots as the
// plan's, so the results are the other engines'), and one queue per
// (source, destination, count, direction, word size), built on first use and
// then replayed: a counter reset and the launch, no host work.  The queue
// reads the source in pass A and writes the destination in pass B (uint64
// words for the drop-in's layout).  kTileQueues queues are kept per plan, the
// least recently used one replaced; each owns its workspace ring (up to 16
// slots of 2^L words).  Calls that share a plan are ordered on one stream.
namespace {
constexpr size_t kTileQueues = 8;  // e.g. three staging buffers x two directions of a host stream
struct TileEntry {
    const void* src;
    void* dst;
    uint32_t n_polys;
    bool inverse, u64;
    Batch* b;
    uint64_t used;
};
struct TileCache {
    nttb_batch_plan* plan = nullptr;
    std::mutex mu;  // guards entries and clock (host threads sharing a plan)
    std::vector<TileEntry> entries;
    uint64_t clock = 0;
};
TileCache* tile_cache(Plan32& p) {
    std::lock_guard<std::mutex> lock(p.engine_mu);
    auto* c = static_cast<TileCache*>(p.engine_data[3]);
    if (c) return c;
    std::vector<uint64_t> q(p.n_limbs);
    for (uint32_t l = 0; l < p.n_limbs; l++) q[l] = p.limbs[l].q;
    nttb_batch_plan* h = nullptr;
    if (nttb_batch_plan_create(q.data(), p.n_limbs, p.log_n, p.negacyclic ? NTTB_NEGACYCLIC : 0u, &h) != NTTB_OK)
        return nullptr;
    c = new TileCache();
    c->plan = h;
    p.engine_data[3] = c;
    return c;
}
}  // namespace

bool tiles_serve(const Plan32& p) { return p.log_n >= 13 && p.log_n <= 20; }

int tiles_transform32(Plan32& p, const void* src, void* dst, bool u64, uint32_t n_polys, bool inverse,
                      cudaStream_t s) {
    if (!tiles_serve(p)) return 1;
    TileCache* c = tile_cache(p);
    if (!c) return 2;
    std::lock_guard<std::mutex> lock(c->mu);
    TileEntry* e = nullptr;
    for (TileEntry& t : c->entries)
        if (t.src == src && t.dst == dst && t.n_polys == n_polys && t.inverse == inverse && t.u64 == u64) e = &t;
    if (!e) {
        const size_t es = u64 ? 8 : 4, poly = (size_t)p.n_limbs << p.log_n;
        std::vector<nttb_batch_job> jobs(n_polys);
        for (uint32_t i = 0; i < n_polys; i++) {
            nttb_batch_job& J = jobs[i];
            J.data = reinterpret_cast<uint32_t*>(static_cast<char*>(dst) + i * poly * es);
            J.log_n = p.log_n;
            J.n_limbs = p.n_limbs;
            J.first_modulus = 0;
            J.flags = (inverse ? NTTB_BATCH_INVERSE : 0u) | (p.negacyclic ? NTTB_NEGACYCLIC : 0u) | (u64 ? kJobW64 : 0u);
            J.pointwise = nullptr;
            if (src != dst) {
                J.flags |= kJobSrc;
                J.pointwise = reinterpret_cast<uint32_t*>(const_cast<char*>(static_cast<const char*>(src) + i * poly * es));
            }
        }
        nttb_batch_config cfg = default_config();
        cfg.tensor = 1;
        Batch* b = nullptr;
        if (create_batch(&c->plan->p, jobs.data(), n_polys, cfg, &b)) return 2;
        if (c->entries.size() >= kTileQueues) {
            auto lru = std::min_element(c->entries.begin(), c->entries.end(),
                                        [](const TileEntry& x, const TileEntry& y) { return x.used < y.used; });
            cudaDeviceSynchronize();  // the evicted queue may still run, on whichever stream it was given
            free_batch(lru->b);
            c->entries.erase(lru);
        }
        c->entries.push_back({src, dst, n_polys, inverse, u64, b, 0});
        e = &c->entries.back();
    }
    e->used = ++c->clock;
    return launch_batch(e->b, s, true) ? 2 : 0;
}

void tiles_release(Plan32* p) {
    auto* c = static_cast<TileCache*>(p->engine_data[3]);
    if (!c) return;
    for (TileEntry& t : c->entries) free_batch(t.b);
    nttb_batch_plan_destroy(c->plan);
    delete c;
    p->engine_data[3] = nullptr;
}

}  // namespace nttb

using nttb::Batch;
using nttb::BatchPlan;
using nttb::fail;

struct nttb_batch {
    Batch* b;
};

// Job flags a C-ABI caller may set (the rest are the plan-transform route's).
static int check_public_flags(const nttb_batch_job* jobs, uint32_t n_jobs, const char* what) {
    for (uint32_t j = 0; j < n_jobs; j++)
        if (jobs[j].flags & ~nttb::kPublicJobFlags)
            return fail(NTTB_ERR_INVALID_ARG, "%s: job %u has unknown flag bits 0x%x", what, j,
                        jobs[j].flags & ~nttb::kPublicJobFlags);
    return NTTB_OK;
}

extern "C" {

NTTB_API int nttb_batch_plan_create(const uint64_t* moduli, uint32_t n_moduli, uint32_t max_log_n, uint32_t flags,
                                    nttb_batch_plan** out) {
    if (!moduli || !out || n_moduli == 0) return fail(NTTB_ERR_INVALID_ARG, "nttb_batch_plan_create: no moduli");
    if (max_log_n < 1 || max_log_n > 24) return fail(NTTB_ERR_INVALID_ARG, "nttb_batch_plan_create: max_log_n in [1, 24]");
    const bool nega = flags & NTTB_NEGACYCLIC;
    auto* h = new nttb_batch_plan();
    BatchPlan& P = h->p;
    P.mods = new BatchPlan::Mods();
    P.max_log = max_log_n;
    P.negacyclic = nega;
    const uint64_t N = 1ull << max_log_n;
    P.limbs.resize(n_moduli);
    for (uint32_t l = 0; l < n_moduli; l++) {
        std::string why;
        if (moduli[l] >= (1ull << 31)) {
            delete P.mods;
            delete h;
            return fail(NTTB_ERR_INVALID_ARG, "nttb_batch_plan_create: modulus %u must be < 2^31", l);
        }
        if (!nttb::make_limb_host(moduli[l], N, nega, &P.limbs[l], &why)) {
            delete P.mods;
            delete h;
            return fail(NTTB_ERR_INVALID_ARG, "nttb_batch_plan_create: %s", why.c_str());
        }
    }
    const uint32_t lo_bits = std::min<uint32_t>(nttb::kLoBits, max_log_n);
    const uint32_t hi_len = 1u << (max_log_n - lo_bits), lo_len = 1u << lo_bits;
    const size_t per_base = (size_t)hi_len + lo_len;
    std::vector<uint32_t> host(4 * per_base);
    std::vector<nttb::BModulus> mods(n_moduli);
    for (uint32_t l = 0; l < n_moduli; l++) {
        const nttb::LimbHost& H = P.limbs[l];
        const uint64_t q = H.q;
        // base^e R for e = i 2^lo_bits (hi part) and e = i (lo part)
        auto powers = [&](uint32_t* dst, uint64_t base) {
            uint64_t x = 1;
            for (uint32_t i = 0; i < lo_len; i++) {
                dst[hi_len + i] = nttb::h_to_mont32(x, q);
                x = nttb::h_mulmod(x, base, q);
            }
            const uint64_t step = x;  // base^(2^lo_bits)
            x = 1;
            for (uint32_t i = 0; i < hi_len; i++) {
                dst[i] = nttb::h_to_mont32(x, q);
                x = nttb::h_mulmod(x, step, q);
            }
        };
        powers(host.data(), H.omega);
        powers(host.data() + per_base, H.omega_inv);
        if (nega) {
            powers(host.data() + 2 * per_base, H.psi);
            powers(host.data() + 3 * per_base, H.psi_inv);
        }
        uint32_t* d = nullptr;
        if (cudaMalloc(&d, host.size() * 4) != cudaSuccess ||
            cudaMemcpy(d, host.data(), host.size() * 4, cudaMemcpyHostToDevice) != cudaSuccess) {
            if (d) cudaFree(d);
            for (void* a : P.allocations) cudaFree(a);
            delete P.mods;
            delete h;
            return fail(NTTB_ERR_NO_MEMORY, "nttb_batch_plan_create: twiddle tables");
        }
        P.allocations.push_back(d);
        nttb::BModulus& M = mods[l];
        M.ar.q = (uint32_t)q;
        M.ar.qinv = nttb::h_neg_inv32((uint32_t)q);
        M.pw = d;
        M.lo_bits = lo_bits;
        M.hi_len = hi_len;
        for (uint32_t L = 0; L < 25; L++) M.ninv[L] = nttb::h_to_mont32(nttb::h_invmod((1ull << L) % q, q), q);
        M.r2 = nttb::h_to_mont32(nttb::h_to_mont32(1, q), q);
    }
    if (max_log_n >= 13) {
        // DFT-64 images per modulus: forward (omega_64), inverse, and the
        // negacyclic forward with psi_128^j on the input index
        const size_t per = nttb::kImgPerMod;
        std::vector<uint8_t> img(per * n_moduli, 0);
        for (uint32_t l = 0; l < n_moduli; l++) {
            const nttb::LimbHost& H = P.limbs[l];
            const uint64_t q = H.q;
            const uint64_t w64 = nttb::h_powmod(H.omega, N / 64, q), w64i = nttb::h_powmod(H.omega_inv, N / 64, q);
            uint8_t* d = img.data() + per * l;
            nttb::tc_build_image64(d, nttb::tc_dft_matrix(64, w64, q), q);
            nttb::tc_build_image64(d + nttb::kImgBytes, nttb::tc_dft_matrix(64, w64i, q), q);
            if (nega)
                nttb::tc_build_image64(d + 2 * nttb::kImgBytes,
                                       nttb::tc_dft_matrix(64, w64, q, 1, nttb::h_powmod(H.psi, N / 64, q)), q);
            // DFT-16 and DFT-8 of level 2: forward, inverse, and the negacyclic
            // inverse with psi_max^-(2^max_log k2 / r') on output k2
            for (uint32_t r : {16u, 8u}) {
                const uint64_t w = nttb::h_powmod(H.omega, N / r, q), wi = nttb::h_powmod(H.omega_inv, N / r, q);
                uint8_t* o = d + (r == 16 ? nttb::kImg16Off : nttb::kImg8Off);
                const uint32_t bytes = r == 16 ? 4096 : 1024;
                auto build = r == 16 ? nttb::tc_build_image16 : nttb::build_image8;
                build(o, nttb::tc_dft_matrix(r, w, q), q);
                build(o + bytes, nttb::tc_dft_matrix(r, wi, q), q);
                if (nega) build(o + 2 * bytes, nttb::tc_dft_matrix(r, wi, q, nttb::h_powmod(H.psi_inv, N / r, q)), q);
            }
        }
        uint8_t* d = nullptr;
        if (cudaMalloc(&d, img.size()) != cudaSuccess ||
            cudaMemcpy(d, img.data(), img.size(), cudaMemcpyHostToDevice) != cudaSuccess) {
            if (d) cudaFree(d);
            for (void* a : P.allocations) cudaFree(a);
            delete P.mods;
            delete h;
            return fail(NTTB_ERR_NO_MEMORY, "nttb_batch_plan_create: DFT-64 images");
        }
        P.allocations.push_back(d);
        P.images = d;
    }
    if (cudaMalloc(&P.mods->d, mods.size() * sizeof(nttb::BModulus)) != cudaSuccess ||
        cudaMemcpy(P.mods->d, mods.data(), mods.size() * sizeof(nttb::BModulus), cudaMemcpyHostToDevice) != cudaSuccess) {
        for (void* a : P.allocations) cudaFree(a);
        delete P.mods;
        delete h;
        return fail(NTTB_ERR_NO_MEMORY, "nttb_batch_plan_create: modulus table");
    }
    P.allocations.push_back(P.mods->d);
    *out = h;
    return NTTB_OK;
}

NTTB_API int nttb_batch_plan_destroy(nttb_batch_plan* plan) {
    if (!plan) return NTTB_OK;
    for (void* a : plan->p.allocations) cudaFree(a);
    delete plan->p.mods;
    delete plan;
    return NTTB_OK;
}

NTTB_API int nttb_batch_default_config(nttb_batch_config* out) {
    if (!out) return fail(NTTB_ERR_INVALID_ARG, "nttb_batch_default_config: null");
    *out = nttb::default_config();
    return NTTB_OK;
}

NTTB_API int nttb_batch_create(nttb_batch_plan* plan, const nttb_batch_job* jobs, uint32_t n_jobs,
                               const nttb_batch_config* config, nttb_batch** out) {
    if (!plan || !out || (!jobs && n_jobs)) return fail(NTTB_ERR_INVALID_ARG, "nttb_batch_create: null argument");
    if (int rc = check_public_flags(jobs, n_jobs, "nttb_batch_create")) return rc;
    const nttb_batch_config cfg = config ? *config : plan->p.have_tuned ? plan->p.tuned : nttb::default_config();
    Batch* b = nullptr;
    if (int rc = nttb::create_batch(&plan->p, jobs, n_jobs, cfg, &b)) return rc;
    *out = new nttb_batch{b};
    return NTTB_OK;
}

NTTB_API int nttb_batch_destroy(nttb_batch* batch) {
    if (!batch) return NTTB_OK;
    nttb::free_batch(batch->b);
    delete batch;
    return NTTB_OK;
}

NTTB_API int nttb_batch_launch(nttb_batch* batch, void* stream) {
    if (!batch) return fail(NTTB_ERR_INVALID_ARG, "nttb_batch_launch: null batch");
    return nttb::launch_batch(batch->b, static_cast<cudaStream_t>(stream), true);
}

NTTB_API int nttb_batch_graph_launch(nttb_batch* batch, void* stream) {
    if (!batch) return fail(NTTB_ERR_INVALID_ARG, "nttb_batch_graph_launch: null batch");
    Batch* b = batch->b;
    if (b->n_tiles == 0) return NTTB_OK;
    if (!b->gexec) {
        if (cudaStreamCreateWithFlags(&b->cap, cudaStreamNonBlocking) != cudaSuccess)
            return fail(NTTB_ERR_CUDA, "nttb_batch_graph_launch: stream");
        if (cudaStreamBeginCapture(b->cap, cudaStreamCaptureModeThreadLocal) != cudaSuccess)
            return fail(NTTB_ERR_CUDA, "nttb_batch_graph_launch: begin capture");
        const int rc = nttb::launch_batch(b, b->cap, false);
        cudaGraph_t g = nullptr;
        const cudaError_t e = cudaStreamEndCapture(b->cap, &g);
        if (rc || e != cudaSuccess || !g) {
            if (g) cudaGraphDestroy(g);
            return fail(NTTB_ERR_CUDA, "nttb_batch_graph_launch: capture failed");
        }
        b->graph = g;
        if (cudaGraphInstantiate(&b->gexec, g, 0) != cudaSuccess) {
            b->gexec = nullptr;
            return fail(NTTB_ERR_CUDA, "nttb_batch_graph_launch: instantiate failed");
        }
    }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    nttb::ProfScope prof("batch_queue_graph", s);
    return cudaGraphLaunch(b->gexec, s) == cudaSuccess ? NTTB_OK
                                                        : fail(NTTB_ERR_CUDA, "nttb_batch_graph_launch: launch failed");
}

NTTB_API int nttb_batch_info(const nttb_batch* batch, uint64_t* units, uint64_t* tiles, uint64_t* ws_bytes,
                             nttb_batch_config* config) {
    if (!batch) return fail(NTTB_ERR_INVALID_ARG, "nttb_batch_info: null batch");
    if (units) *units = batch->b->n_units;
    if (tiles) *tiles = batch->b->n_tiles;
    if (ws_bytes) *ws_bytes = batch->b->ws_bytes;
    if (config) *config = batch->b->cfg;
    return NTTB_OK;
}

NTTB_API int nttb_batch_test_stall(nttb_batch* batch, uint32_t unit) {
    if (!batch) return fail(NTTB_ERR_INVALID_ARG, "nttb_batch_test_stall: null batch");
    Batch* b = batch->b;
    if (unit >= b->n_units) return fail(NTTB_ERR_INVALID_ARG, "nttb_batch_test_stall: unit %u of %u", unit, b->n_units);
    nttb::BUnit u{};
    if (cudaMemcpy(&u, b->d_units + unit, sizeof u, cudaMemcpyDeviceToHost) != cudaSuccess)
        return fail(NTTB_ERR_CUDA, "nttb_batch_test_stall: read");
    if (!u.lg1) return fail(NTTB_ERR_INVALID_ARG, "nttb_batch_test_stall: unit %u has a single pass", unit);
    u.tiles_a += 1;  // pass B now waits for one pass A tile more than there are
    if (cudaMemcpy(b->d_units + unit, &u, sizeof u, cudaMemcpyHostToDevice) != cudaSuccess)
        return fail(NTTB_ERR_CUDA, "nttb_batch_test_stall: write");
    return NTTB_OK;
}

NTTB_API int nttb_batch_ctas(const nttb_batch* batch, uint32_t* ctas) {
    if (!batch || !ctas) return fail(NTTB_ERR_INVALID_ARG, "nttb_batch_ctas: null argument");
    *ctas = (uint32_t)batch->b->grid;
    return NTTB_OK;
}

NTTB_API int nttb_batch_autotune(nttb_batch_plan* plan, const nttb_batch_job* jobs, uint32_t n_jobs, void* stream,
                                 nttb_batch_config* out) {
    if (!plan || !jobs || n_jobs == 0) return fail(NTTB_ERR_INVALID_ARG, "nttb_batch_autotune: no jobs");
    if (int rc = check_public_flags(jobs, n_jobs, "nttb_batch_autotune")) return rc;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    // Sample of the mix on scratch buffers (the caller's data is untouched):
    // up to two jobs per (log_n, direction, twist, product) with at most 8
    // limbs each, then further jobs until the sample holds 32 M residues, so
    // that every candidate is timed on enough work to fill the GPU.
    std::vector<nttb_batch_job> sample;
    std::vector<uint32_t> seen(64 * 8, 0);
    std::vector<char> taken(n_jobs, 0);
    size_t words = 0;
    auto take = [&](uint32_t j) {
        nttb_batch_job c = jobs[j];
        c.n_limbs = std::min<uint32_t>(c.n_limbs, 8);
        sample.push_back(c);
        words += ((size_t)c.n_limbs << c.log_n) * ((c.flags & NTTB_BATCH_POLYMUL) ? 2 : 1);
        taken[j] = 1;
    };
    for (uint32_t j = 0; j < n_jobs; j++) {
        const nttb_batch_job& J = jobs[j];
        if (J.log_n < 1 || J.log_n > plan->p.max_log) return fail(NTTB_ERR_INVALID_ARG, "nttb_batch_autotune: job %u log_n", j);
        const uint32_t key = J.log_n * 8 + ((J.flags & NTTB_BATCH_INVERSE) ? 1 : 0) + ((J.flags & NTTB_NEGACYCLIC) ? 2 : 0) +
                             ((J.flags & NTTB_BATCH_POLYMUL) ? 4 : 0);
        if (seen[key] >= 2) continue;
        seen[key]++;
        take(j);
    }
    for (uint32_t j = 0; j < n_jobs && words < (32u << 20); j++)
        if (!taken[j]) take(j);
    uint32_t* scratch = nullptr;
    if (cudaMalloc(&scratch, words * 4) != cudaSuccess) return fail(NTTB_ERR_NO_MEMORY, "nttb_batch_autotune: scratch");
    cudaMemsetAsync(scratch, 0, words * 4, s);
    size_t off = 0;
    for (nttb_batch_job& c : sample) {
        c.data = scratch + off;
        off += (size_t)c.n_limbs << c.log_n;
        if (c.flags & NTTB_BATCH_POLYMUL) {
            c.pointwise = scratch + off;
            off += (size_t)c.n_limbs << c.log_n;
        }
    }
    // {tile, threads, tensor}
    const uint32_t shapes[6][3] = {{4096, 256, 0}, {8192, 256, 0}, {8192, 512, 0}, {16384, 512, 0},
                                   {4096, 256, 1}, {8192, 256, 1}};
    const uint32_t lags[3] = {1, 4, 8}, groups[3] = {1, 3, 4};
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    float best = 1e30f;
    nttb_batch_config best_cfg = nttb::default_config();
    int rc = 0;
    for (const auto& sh : shapes)
        for (uint32_t split = 0; split < 2; split++)
            for (uint32_t lag : lags)
                for (uint32_t grp : groups) {
                    if (rc) continue;  // a failed launch ends the search
                    nttb_batch_config c = nttb::default_config();
                    c.tile_elems = sh[0];
                    c.threads = sh[1];
                    c.tensor = sh[2];
                    if (c.tensor && !plan->p.images) continue;
                    c.split = split;
                    c.lag = lag;
                    c.group = grp;
                    Batch* b = nullptr;
                    if (nttb::create_batch(&plan->p, sample.data(), (uint32_t)sample.size(), c, &b)) continue;
                    float t_min = 1e30f;
                    for (int it = 0; it < 4 && rc == 0; it++) {
                        cudaEventRecord(e0, s);
                        rc = nttb::launch_batch(b, s, false);
                        cudaEventRecord(e1, s);
                        cudaEventSynchronize(e1);
                        float ms = 0;
                        cudaEventElapsedTime(&ms, e0, e1);
                        if (it > 0) t_min = std::min(t_min, ms);  // the first run warms up
                    }
                    nttb::free_batch(b);
                    if (!rc && t_min < best) {
                        best = t_min;
                        best_cfg = c;
                    }
                }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(scratch);
    if (rc) return rc;
    plan->p.tuned = best_cfg;
    plan->p.have_tuned = true;
    if (out) *out = best_cfg;
    return NTTB_OK;
}

}  // extern "C"
