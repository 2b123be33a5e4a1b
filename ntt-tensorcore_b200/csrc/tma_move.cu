// tma_move.cu -- the HBM-bound permutations of uint64 arrays on the Tensor
// Memory Accelerator: out-of-place transpose (the reference's
// rowmaj_to_pretransposed / rowmaj_from_pretransposed and transpose helper,
// src/ntt_optimized.cu:922-936, src/ntt_four_step.cu:212-242), the in-place
// transpose of a square matrix, and the in-place bit-reversal permutation
// (bit_reverse_permute / bitrev_kernel, src/ntt_basic.cu).
//
// One persistent kernel moves 32 x 32-word tiles (8 KB) through a ring of
// shared-memory slots, one work item per slot:
//   * TMA tiled loads bring a tile into its slot with the 128-byte swizzle,
//     completing on the slot's mbarrier: two 128-byte-wide boxes for the
//     transposes, one box holding both halves of every 256-byte row segment
//     for the bit reversal (tile_off);
//   * the threads permute the tile inside the slot: whole 16-byte chunks
//     are read into registers and, after a barrier, written back to their
//     permuted places in the same swizzled layout, with lane assignments that
//     keep both sides free of bank conflicts (permute_transpose,
//     permute_bitrev);
//   * TMA tiled stores write the slot back in the same boxes, and the slot
//     is reloaded only once those stores have read it, while a third of the
//     ring's slots may still be storing.
// HBM sees only whole 256-byte row segments in both directions, and with no
// separate output buffer every slot of shared memory carries loads in flight.
// In-place jobs move tiles in pairs (a tile and the tile it is exchanged with
// are both loaded before either is stored), so no tile is read after it is
// written.
// Every mbarrier wait is bounded; a wait that runs out sets a bit read by
// nttb_device_errors.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>

#include "profiler.hpp"
#include "tcgen05.cuh"

namespace nttb {
namespace {

__device__ uint32_t g_move_error;

constexpr uint32_t kThreads = 256;
constexpr uint32_t kTileBytes = 8192;   // 32 x 32 words
constexpr uint32_t kRingBytes = 96 * 1024;  // tile slots of one CTA (two CTAs per SM)

enum Mode : int { kTranspose = 0, kSquareInPlace = 1, kBitReverse = 2 };

// Tiles per item (the in-place jobs move tile pairs), ring slots of one item
// each, and how many slots may still be read by their stores while the
// others load.
template <int MODE>
struct Ring {
    static constexpr uint32_t kTilesPerItem = MODE == kTranspose ? 1u : 2u;
    static constexpr uint32_t kBoxes = MODE == kBitReverse ? 1u : 2u;  // TMA boxes per tile (tile_off)
    static constexpr uint32_t kSlotBytes = kTilesPerItem * kTileBytes;
    static constexpr uint32_t kSlots = kRingBytes / kSlotBytes;
    static constexpr uint32_t kStoring = kSlots / 3u;
    static constexpr uint32_t kOffBar = kRingBytes;
    static constexpr uint32_t kSmemBytes = kOffBar + 8u * kSlots + 16u + 1024u;  // + abort flag, alignment slack
    static_assert(kStoring >= 1 && kStoring < kSlots, "ring split");
};

struct MoveArgs {
    uint32_t tiles_r, tiles_c;  // tile grid of the source matrix (transposes)
    uint32_t mid_bits;          // bit reversal: log2(n) - 10
    uint32_t blocked;           // item order by 16 x 16 blocks (see decode)
    uint64_t n_items;
};

// One work item: up to two tiles, each with its load and store coordinates
// in the four-dimensional view (word, half, tile, row) of the array: t = the
// tile's 256-byte column (the middle index b for the bit reversal), y = its
// first row.
struct Item {
    bool valid;
    uint32_t ntiles;
    int32_t ld_t[2], ld_y[2], st_t[2], st_y[2];
};

// Byte offset of word (r, c) of a tile in shared memory, as TMA lands it
// with the 128-byte swizzle (16-byte chunk index XOR row % 8, 128-byte rows):
//   ONE = false: two boxes {16 words, 1 half, 1 tile, 32 rows}, half h of
//     every row segment at 4096 h + 128 r;
//   ONE = true: one box {16, 2, 1, 32}, the two halves of a row segment side
//     by side in rows r' = 2 r + h.
// The transposes take two boxes, the bit reversal one: that is what measured
// fastest for each (its rows lie n / 32 words apart, and fetching both
// halves of each 256-byte segment together serves it better).
template <bool ONE>
__device__ __forceinline__ uint32_t tile_off(uint32_t r, uint32_t c) {
    const uint32_t rr = ONE ? 2u * r + (c >> 4) : r, base = ONE ? 0u : (c >> 4) * 4096u;
    return base + rr * 128u + ((((c & 15u) >> 1) ^ (rr & 7u)) << 4) + (c & 1u) * 8u;
}

__device__ __forceinline__ uint32_t rev5(uint32_t v) { return __brev(v) >> 27; }

// Item order.  The CTAs work on consecutive items at the same time, so the
// order decides how scattered the HBM accesses in flight are.  Row-major
// order over tiles reads whole rows on one side of a transpose and scatters
// 256-byte pieces on the other; with `blocked`, 256 consecutive items form a
// 16 x 16 block of tiles, so both sides move 4 KB runs.  For the bit
// reversal the same holds with the low four and the high four bits of the
// middle index b taken from the low byte of the item: b and rev(b) then both
// run over 16 consecutive tiles.
template <int MODE>
__device__ __forceinline__ Item decode(const MoveArgs& a, uint64_t t) {
    Item it;
    if (MODE == kBitReverse) {
        // element (hi, b, lo) -> (rev5(lo), rev(b), rev5(hi)): the tile at
        // middle index b is exchanged with the tile at rev(b)
        const uint32_t M = a.mid_bits, tt = (uint32_t)t;
        const uint32_t b =
            a.blocked ? (((tt >> 4) & 15u) << (M - 4u)) | ((tt >> 8) << 4) | (tt & 15u) : tt;
        const uint32_t br = a.mid_bits ? (__brev(b) >> (32 - a.mid_bits)) : 0u;
        it.valid = b <= br;
        it.ntiles = b == br ? 1u : 2u;
        it.ld_y[0] = it.ld_y[1] = it.st_y[0] = it.st_y[1] = 0;
        it.ld_t[0] = (int32_t)b;
        it.st_t[0] = (int32_t)br;
        it.ld_t[1] = (int32_t)br;
        it.st_t[1] = (int32_t)b;
        return it;
    }
    uint32_t I, J;
    if (a.blocked) {
        const uint64_t blk = t >> 8, bc = a.tiles_c >> 4;
        const uint32_t w = (uint32_t)t & 255u;
        I = (uint32_t)(blk / bc) * 16u + (w >> 4);
        J = (uint32_t)(blk % bc) * 16u + (w & 15u);
    } else {
        I = (uint32_t)(t / a.tiles_c);
        J = (uint32_t)(t % a.tiles_c);
    }
    // source tile (rows 32 I.., words 32 J..) -> destination tile (rows 32 J.., words 32 I..)
    it.ld_t[0] = (int32_t)J;
    it.ld_y[0] = (int32_t)(32u * I);
    it.st_t[0] = (int32_t)I;
    it.st_y[0] = (int32_t)(32u * J);
    if (MODE == kTranspose) {
        it.valid = true;
        it.ntiles = 1;
    } else {
        it.valid = I <= J;
        it.ntiles = I == J ? 1u : 2u;
        // the partner tile sits where tile 0 goes, and goes where tile 0 was
        it.ld_t[1] = it.st_t[0];
        it.ld_y[1] = it.st_y[0];
        it.st_t[1] = it.ld_t[0];
        it.st_y[1] = it.ld_y[0];
    }
    return it;
}

// Box {16 words, 2 / 1 halves, 1 tile, 32 rows} at half h.
__device__ __forceinline__ void tma_load(uint8_t* smem, const CUtensorMap* map, int32_t h, int32_t t, int32_t y,
                                         uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], "
        "[%6];" ::"r"(tc::smem_u32(smem)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(0), "r"(h), "r"(t), "r"(y), "r"(tc::smem_u32(bar))
        : "memory");
}

__device__ __forceinline__ void tma_store(const CUtensorMap* map, int32_t h, int32_t t, int32_t y, const uint8_t* smem) {
    asm volatile("cp.async.bulk.tensor.4d.global.shared::cta.tile.bulk_group [%0, {%1, %2, %3, %4}], [%5];" ::"l"(
                     reinterpret_cast<uint64_t>(map)),
                 "r"(0), "r"(h), "r"(t), "r"(y), "r"(tc::smem_u32(smem))
                 : "memory");
}

__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
// Waits until at most N committed store groups still read shared memory.
template <int N>
__device__ __forceinline__ void bulk_wait_read() {
    asm volatile("cp.async.bulk.wait_group.read %0;" ::"n"(N) : "memory");
}
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }

// Transpose of the item's tiles inside their slot: word (i, j) moves to
// (j, i).  Lane i, warp w reads the 16-byte chunks (row i, words 2k, 2k+1)
// for k = w and w + 8 (conflict-free: the swizzle puts the 8 rows of a
// quarter-warp in 8 different bank groups) and writes its words to column i
// of rows 2k, 2k + 1, 16 lanes filling one 128-byte row segment.
__device__ __forceinline__ void permute_transpose(uint8_t* slot, uint32_t ntiles, uint32_t lane, uint32_t warp) {
    uint4 v[2][2];
#pragma unroll
    for (uint32_t u = 0; u < 2; u++)
#pragma unroll
        for (uint32_t cc = 0; cc < 2; cc++)
            if (u < ntiles)
                v[u][cc] = *reinterpret_cast<const uint4*>(slot + u * kTileBytes + tile_off<false>(lane, 2u * (warp + 8u * cc)));
    __syncthreads();  // every word of the item is in registers: overwrite in place
#pragma unroll
    for (uint32_t u = 0; u < 2; u++)
#pragma unroll
        for (uint32_t cc = 0; cc < 2; cc++)
            if (u < ntiles) {
                const uint32_t j0 = 2u * (warp + 8u * cc);
                *reinterpret_cast<uint2*>(slot + u * kTileBytes + tile_off<false>(j0, lane)) = make_uint2(v[u][cc].x, v[u][cc].y);
                *reinterpret_cast<uint2*>(slot + u * kTileBytes + tile_off<false>(j0 + 1u, lane)) =
                    make_uint2(v[u][cc].z, v[u][cc].w);
            }
}

// Bit-reversal permutation of the item's tiles inside their slot (one-box
// layout): word (i, j) moves to (rev5(j), rev5(i)).  A thread takes the
// 16-byte chunk of words j0 = 2 kc, j0 + 1 in rows i and i + 16 (i < 16).
// Since rev5(i + 16) = rev5(i) + 1, the words (i, j) and (i + 16, j) land
// side by side in one 16-byte chunk of row rev5(j), so reads and writes are
// whole chunks.  The 8 lanes of a quarter-warp q take rows i = 4 q .. 4 q + 3
// times both halves h of chunk kk = warp (kc = 8 h + kk): their read rows
// r' = 2 i + h cover all 8 swizzle phases, and their output chunks (bits 3..1
// of i, i % 2 and h) all differ, so neither side has bank conflicts.
__device__ __forceinline__ void permute_bitrev(uint8_t* slot, uint32_t ntiles, uint32_t lane, uint32_t warp) {
    const uint32_t h = lane & 1u, i = 4u * (lane >> 3) + ((lane >> 1) & 3u);
    const uint32_t j0 = 2u * (8u * h + warp);
    const uint32_t rin0 = tile_off<true>(i, j0), rin1 = tile_off<true>(i + 16u, j0);
    const uint32_t x = rev5(i), R0 = rev5(j0);
    const uint32_t rout0 = tile_off<true>(R0, x), rout1 = tile_off<true>(R0 + 16u, x);
    uint4 a[2], b[2];
#pragma unroll
    for (uint32_t u = 0; u < 2; u++)
        if (u < ntiles) {
            a[u] = *reinterpret_cast<const uint4*>(slot + u * kTileBytes + rin0);
            b[u] = *reinterpret_cast<const uint4*>(slot + u * kTileBytes + rin1);
        }
    __syncthreads();  // every word of the item is in registers: overwrite in place
#pragma unroll
    for (uint32_t u = 0; u < 2; u++)
        if (u < ntiles) {
            *reinterpret_cast<uint4*>(slot + u * kTileBytes + rout0) = make_uint4(a[u].x, a[u].y, b[u].x, b[u].y);
            *reinterpret_cast<uint4*>(slot + u * kTileBytes + rout1) = make_uint4(a[u].z, a[u].w, b[u].z, b[u].w);
        }
}

template <int MODE>
__global__ void __launch_bounds__(kThreads) tma_move_kernel(const __grid_constant__ CUtensorMap ld_map,
                                                            const __grid_constant__ CUtensorMap st_map,
                                                            const MoveArgs a) {
    using R = Ring<MODE>;
    extern __shared__ uint8_t smem_raw[];
    uint8_t* base = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    uint64_t* full = reinterpret_cast<uint64_t*>(base + R::kOffBar);
    volatile uint32_t* abort_flag = reinterpret_cast<volatile uint32_t*>(full + R::kSlots);
    const uint32_t tid = threadIdx.x, lane = tid & 31u, warp = tid >> 5;
    if (tid == 0) {
        for (uint32_t s = 0; s < R::kSlots; s++) tc::mbar_init(full + s, 1);
        *abort_flag = 0;
    }
    __syncthreads();

    // producer (thread 0): loads of the next valid item into the next slot
    uint64_t p_item = blockIdx.x;
    uint32_t p_count = 0;
    auto produce = [&]() {
        while (p_item < a.n_items) {
            const Item it = decode<MODE>(a, p_item);
            p_item += gridDim.x;
            if (!it.valid) continue;
            const uint32_t s = p_count % R::kSlots;
            p_count++;
            tc::mbar_expect_tx(full + s, it.ntiles * kTileBytes);
            for (uint32_t u = 0; u < it.ntiles; u++)
                for (uint32_t h = 0; h < R::kBoxes; h++)
                    tma_load(base + s * R::kSlotBytes + u * kTileBytes + h * 4096u, &ld_map, (int32_t)h, it.ld_t[u],
                             it.ld_y[u], full + s);
            return;
        }
    };
    if (tid == 0)
        for (uint32_t i = 0; i < R::kSlots; i++) produce();

    uint32_t k = 0;
    for (uint64_t t = blockIdx.x; t < a.n_items; t += gridDim.x) {
        const Item it = decode<MODE>(a, t);
        if (!it.valid) continue;
        const uint32_t s = k % R::kSlots;
        uint8_t* slot = base + s * R::kSlotBytes;
        if (!tc::mbar_wait_bounded(full + s, (k / R::kSlots) & 1u)) {
            atomicOr(&g_move_error, 1u);
            *abort_flag = 1;  // the tile is not there: permute what shared memory holds, store nothing
        }
        if (MODE == kBitReverse) permute_bitrev(slot, it.ntiles, lane, warp);
        else permute_transpose(slot, it.ntiles, lane, warp);
        tc::fence_proxy_async_smem();
        __syncthreads();
        if (*abort_flag) break;
        if (tid == 0) {
            for (uint32_t u = 0; u < it.ntiles; u++)
                for (uint32_t h = 0; h < R::kBoxes; h++)
                    tma_store(&st_map, (int32_t)h, it.st_t[u], it.st_y[u], slot + u * kTileBytes + h * 4096u);
            bulk_commit();
            // the slot of item k - kStoring is free once its stores have read
            // it: load the next item there
            if (k >= R::kStoring) {
                bulk_wait_read<(int)R::kStoring>();
                produce();
            }
        }
        k++;
    }
    if (tid == 0) {
        bulk_wait_all();
        // after a wait that ran out: give the loads still in flight a bounded
        // chance to land before the shared memory is released
        if (*abort_flag)
            for (uint32_t i = k; i < p_count; i++) tc::mbar_wait_bounded(full + i % R::kSlots, (i / R::kSlots) & 1u);
    }
}

bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

// The driver's tensor-map encoder, looked up through the runtime so that the
// library does not link libcuda (it loads on hosts without a driver).
PFN_cuTensorMapEncodeTiled_v12000 encoder() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            p = nullptr;
        return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    }();
    return fn;
}

// The four-dimensional uint64 view (word, half, tile, row) of an array:
// dims[0] = 16 words of 128 bytes, dims[1] = the two halves of a 256-byte
// row segment, strides in bytes for dims 1..3; boxes of `halves` x 16 words
// x 32 rows of one tile with the 128-byte swizzle.
bool make_map(CUtensorMap* m, void* ptr, const cuuint64_t* dims, const cuuint64_t* strides, uint32_t halves) {
    const auto encode = encoder();
    if (!encode) return false;
    const cuuint32_t box[4] = {16, halves, 1, 32}, estr[4] = {1, 1, 1, 1};
    return encode(m, CU_TENSOR_MAP_DATA_TYPE_UINT64, 4, ptr, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                  CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

template <int MODE>
int launch(const CUtensorMap& ld, const CUtensorMap& st, const MoveArgs& a, cudaStream_t stream) {
    static std::atomic<uint64_t> attr_set{0};  // per template instance, one bit per device
    int dev = 0, sms = 148, per_sm = 1;
    cudaGetDevice(&dev);
    const uint64_t bit = 1ull << (dev & 63);
    if (!(attr_set.load() & bit)) {
        if (cudaFuncSetAttribute(tma_move_kernel<MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize, Ring<MODE>::kSmemBytes) !=
            cudaSuccess)
            return 2;
        attr_set.fetch_or(bit);
    }
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, tma_move_kernel<MODE>, kThreads, Ring<MODE>::kSmemBytes) !=
            cudaSuccess ||
        per_sm < 1)
        per_sm = 1;
    const uint64_t resident = (uint64_t)per_sm * (uint64_t)sms;
    const unsigned grid = (unsigned)(a.n_items < resident ? a.n_items : resident);
    if (grid == 0) return 0;
    static const char* const kName[3] = {"tma_transpose_u64", "tma_transpose_square_inplace_u64", "tma_bitrev_u64"};
    ProfScope prof(kName[MODE], stream);
    tma_move_kernel<MODE><<<grid, kThreads, Ring<MODE>::kSmemBytes, stream>>>(ld, st, a);
    return cudaPeekAtLastError() == cudaSuccess ? 0 : 2;
}

}  // namespace

// dst[c * rows + r] = src[r * cols + c].  Returns 1 when the shape or the
// alignment is not served (rows, cols multiples of 32 below 2^31, 16-byte
// aligned arrays), 2 on a CUDA error.
int tma_transpose_u64(uint64_t* dst, const uint64_t* src, uint64_t rows, uint64_t cols, cudaStream_t stream) {
    if (rows % 32 || cols % 32 || rows >= (1ull << 31) || cols >= (1ull << 31) || !aligned16(dst) || !aligned16(src))
        return 1;
    CUtensorMap ld, st;
    const cuuint64_t ld_dims[4] = {16, 2, cols / 32, rows}, ld_str[3] = {128, 256, cols * 8};
    const cuuint64_t st_dims[4] = {16, 2, rows / 32, cols}, st_str[3] = {128, 256, rows * 8};
    if (!make_map(&ld, const_cast<uint64_t*>(src), ld_dims, ld_str, 1) || !make_map(&st, dst, st_dims, st_str, 1))
        return 1;
    const uint32_t tr = (uint32_t)(rows / 32), tcn = (uint32_t)(cols / 32);
    MoveArgs a{tr, tcn, 0, (tr % 16 == 0 && tcn % 16 == 0) ? 1u : 0u, (uint64_t)tr * tcn};
    return launch<kTranspose>(ld, st, a, stream);
}

// In-place transpose of an n x n matrix (n a multiple of 32 below 2^31).
int tma_transpose_square_inplace_u64(uint64_t* d, uint64_t n, cudaStream_t stream) {
    if (n % 32 || n >= (1ull << 31) || !aligned16(d)) return 1;
    CUtensorMap map;  // loads and stores
    const cuuint64_t dims[4] = {16, 2, n / 32, n}, str[3] = {128, 256, n * 8};
    if (!make_map(&map, d, dims, str, 1)) return 1;
    const uint64_t T = n / 32;
    MoveArgs a{(uint32_t)T, (uint32_t)T, 0, T % 16 == 0 ? 1u : 0u, T * T};
    return launch<kSquareInPlace>(map, map, a, stream);
}

// In-place bit reversal of 2^log_n words, 10 <= log_n <= 40, viewed as
// [32][2^(log_n - 10)][32].
int tma_bit_reverse_u64(uint64_t* d, int log_n, cudaStream_t stream) {
    if (log_n < 10 || log_n > 40 || !aligned16(d)) return 1;
    const uint32_t M = (uint32_t)log_n - 10u;
    if (M > 31) return 1;
    CUtensorMap map;  // loads and stores
    const cuuint64_t dims[4] = {16, 2, 1ull << M, 32}, str[3] = {128, 256, (32ull << M) * 8};
    if (!make_map(&map, d, dims, str, 2)) return 1;
    MoveArgs a{0, 0, M, M >= 8 ? 1u : 0u, 1ull << M};
    return launch<kBitReverse>(map, map, a, stream);
}

uint32_t tma_move_device_errors(bool clear) {
    uint32_t v = 0;
    cudaMemcpyFromSymbol(&v, g_move_error, sizeof v);
    if (clear && v) {
        const uint32_t z = 0;
        cudaMemcpyToSymbol(g_move_error, &z, sizeof z);
    }
    return v;
}

}  // namespace nttb
