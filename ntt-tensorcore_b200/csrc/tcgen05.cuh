// tcgen05.cuh -- thin inline-PTX wrappers for the sm_100a tensor-core path:
// TMEM allocation, UMMA shared-memory / instruction descriptors,
// tcgen05.mma kind::i8, tcgen05.commit to an mbarrier, tcgen05.ld, and
// bounded mbarrier waits.  Every wait gives up after a fixed budget and
// reports it, so a kernel never spins forever.
#pragma once
#include <cstdint>

namespace nttb {
namespace tc {

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// ---- TMEM ---------------------------------------------------------------------
// One warp allocates `ncols` (power of two >= 32) TMEM columns and writes the
// base address into *slot (shared memory).
__device__ __forceinline__ void tmem_alloc(uint32_t* slot, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(slot)),
                 "r"(ncols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols));
}
__device__ __forceinline__ void fence_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// Generic-proxy shared-memory writes -> visible to the tensor core (async proxy).
__device__ __forceinline__ void fence_proxy_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// ---- mbarrier -------------------------------------------------------------------
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
// Suspend-time hint of every wait (ns): a warp whose phase is not complete
// sleeps until it completes (or this much time passes) instead of polling,
// so waiting warps take no issue slots from the warps that compute.
constexpr uint32_t kSuspendHintNs = 1000000u;
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity), "r"(kSuspendHintNs)
        : "memory");
    return ok != 0;
}
// Arms `bar` to expect `bytes` of async-proxy transfers (one arrival).
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}
// Bulk (TMA, non-tensor) copy global -> shared, completing on `bar`.
// Addresses 16-byte aligned, bytes a multiple of 16.  Local memory only.
__device__ __forceinline__ void bulk_g2s(void* smem_dst, const void* gmem_src, uint32_t bytes, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_u32(smem_dst)),
        "l"(gmem_src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}
// The same copy with an L2 eviction-priority policy (createpolicy), for
// constants that every launch re-reads while streamed operands pass through
// the L2: `policy` from l2_policy_evict_last().
__device__ __forceinline__ void bulk_g2s_hint(void* smem_dst, const void* gmem_src, uint32_t bytes, uint64_t* bar,
                                              uint64_t policy) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint [%0], [%1], %2, [%3], %4;" ::"r"(
            smem_u32(smem_dst)),
        "l"(gmem_src), "r"(bytes), "r"(smem_u32(bar)), "l"(policy)
        : "memory");
}
__device__ __forceinline__ uint64_t l2_policy_evict_last() {
    uint64_t p;
    asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
    return p;
}

// Device clock in nanoseconds (%globaltimer) and the budget of every
// bounded wait: far above any legitimate wait of these kernels (a whole
// batch takes tens of milliseconds), short enough that a wait that can never
// end gives up within a few seconds and the host sees the error.  An
// iteration cap backs up the clock.
__device__ __forceinline__ uint64_t globaltimer_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
constexpr uint64_t kWaitBudgetNs = 2000000000ull;

// Bounded wait for the phase with the given parity.  Returns false when the
// time budget runs out.  Each try_wait sleeps up to kSuspendHintNs, so the
// loop runs a few iterations per wait, not thousands.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity) {
    if (mbar_try_wait(bar, parity)) return true;
    const uint64_t t0 = globaltimer_ns();
    for (uint32_t i = 0; i < (1u << 26); i++) {
        if (mbar_try_wait(bar, parity)) return true;
        if (globaltimer_ns() - t0 > kWaitBudgetNs) return false;
    }
    return false;
}

// ---- thread-block clusters and distributed shared memory ---------------------
__device__ __forceinline__ uint32_t cluster_rank() {
    uint32_t r;
    asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
    return r;
}
__device__ __forceinline__ uint32_t cluster_id() {
    uint32_t r;
    asm volatile("mov.u32 %0, %%clusterid.x;" : "=r"(r));
    return r;
}
__device__ __forceinline__ uint32_t cluster_count() {
    uint32_t r;
    asm volatile("mov.u32 %0, %%nclusterid.x;" : "=r"(r));
    return r;
}
// Hardware barrier over every thread of every CTA in the cluster.  Used only
// where all threads reach it unconditionally (start-up), never on a data path.
__device__ __forceinline__ void cluster_sync() {
    asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}
// Shared::cluster address of the same shared-memory offset in CTA `rank`.
__device__ __forceinline__ uint32_t mapa(uint32_t local_addr, uint32_t rank) {
    uint32_t r;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(local_addr), "r"(rank));
    return r;
}
__device__ __forceinline__ void st_cluster(uint32_t addr, uint32_t v) {
    asm volatile("st.shared::cluster.u32 [%0], %1;" ::"r"(addr), "r"(v) : "memory");
}
// Arrive (release, cluster scope) on an mbarrier that may live in another CTA.
__device__ __forceinline__ void arrive_cluster(uint32_t bar_cluster_addr) {
    asm volatile("mbarrier.arrive.release.cluster.shared::cluster.b64 _, [%0];" ::"r"(bar_cluster_addr) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait_cluster(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.acquire.cluster.shared::cta.b64 p, [%1], %2, %3;\n"
        " selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity), "r"(kSuspendHintNs)
        : "memory");
    return ok != 0;
}
// Bounded wait (acquire at cluster scope) for arrivals made by other CTAs.
__device__ __forceinline__ bool mbar_wait_cluster_bounded(uint64_t* bar, uint32_t parity) {
    if (mbar_try_wait_cluster(bar, parity)) return true;
    const uint64_t t0 = globaltimer_ns();
    for (uint32_t i = 0; i < (1u << 26); i++) {
        if (mbar_try_wait_cluster(bar, parity)) return true;
        if (globaltimer_ns() - t0 > kWaitBudgetNs) return false;
    }
    return false;
}
// Bulk copy of `bytes` from this CTA's shared memory to another CTA's
// (shared::cluster addresses from mapa), completing `bytes` of transaction
// count on the destination CTA's mbarrier.  16-byte aligned, bytes % 16 == 0.
__device__ __forceinline__ void bulk_s2cluster(uint32_t dst_cluster, uint32_t src_cta, uint32_t bytes,
                                               uint32_t bar_cluster) {
    asm volatile(
        "cp.async.bulk.shared::cluster.shared::cta.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            dst_cluster),
        "r"(src_cta), "r"(bytes), "r"(bar_cluster)
        : "memory");
}
// Generic-proxy writes to (possibly remote) shared memory -> async proxy.
__device__ __forceinline__ void fence_proxy_async_cluster() {
    asm volatile("fence.proxy.async.shared::cluster;" ::: "memory");
}
__device__ __forceinline__ void fence_acq_rel_cluster() { asm volatile("fence.acq_rel.cluster;" ::: "memory"); }

// ---- descriptors -------------------------------------------------------------
// K-major operand with 128-byte swizzle: 8-row x 128-byte atoms, atoms stacked
// along M/N every 1024 bytes (SBO).  `addr` is the shared address of the
// first row's first byte for this K step (atom-aligned base + k*32 bytes).
__device__ __forceinline__ uint64_t desc_k_sw128(uint32_t addr) {
    uint64_t d = 0;
    d |= (uint64_t)((addr >> 4) & 0x3FFFu);         // start address
    d |= (uint64_t)1u << 16;                          // LBO (unused for swizzled K-major) = 16 B
    d |= (uint64_t)(1024u >> 4) << 32;                // SBO = 1024 B
    d |= (uint64_t)1u << 46;                          // descriptor version (sm_100)
    d |= (uint64_t)2u << 61;                          // SWIZZLE_128B
    return d;
}
// K-major operand with 64-byte swizzle: 8-row x 64-byte atoms, SBO = 512 B.
__device__ __forceinline__ uint64_t desc_k_sw64(uint32_t addr) {
    uint64_t d = 0;
    d |= (uint64_t)((addr >> 4) & 0x3FFFu);
    d |= (uint64_t)1u << 16;
    d |= (uint64_t)(512u >> 4) << 32;
    d |= (uint64_t)1u << 46;
    d |= (uint64_t)4u << 61;                          // SWIZZLE_64B
    return d;
}
// K-major operand with 32-byte swizzle: 8-row x 32-byte atoms, SBO = 256 B.
__device__ __forceinline__ uint64_t desc_k_sw32(uint32_t addr) {
    uint64_t d = 0;
    d |= (uint64_t)((addr >> 4) & 0x3FFFu);
    d |= (uint64_t)1u << 16;
    d |= (uint64_t)(256u >> 4) << 32;
    d |= (uint64_t)1u << 46;
    d |= (uint64_t)6u << 61;                          // SWIZZLE_32B
    return d;
}
// Instruction descriptor, kind::i8: u8 x u8 -> s32, both operands K-major.
__host__ __device__ constexpr uint32_t idesc_u8(uint32_t M, uint32_t N) {
    return (2u << 4)            // D format S32
           | (0u << 7)          // A: unsigned 8-bit
           | (0u << 10)         // B: unsigned 8-bit
           | ((N >> 3) << 17)   // N / 8
           | ((M >> 4) << 24);  // M / 16
}

// ---- MMA / commit / load --------------------------------------------------------
__device__ __forceinline__ void mma_i8(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc, uint32_t accumulate) {
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
        " tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem_d),
        "l"(da), "l"(db), "r"(idesc), "r"(accumulate));
}
__device__ __forceinline__ void commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}
// 32 lanes x 32 bits, 16 consecutive columns -> 16 registers per thread.
__device__ __forceinline__ void ld_32x32b_x16(uint32_t taddr, uint32_t (&r)[16]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
}
// 32 lanes x 32 bits, 32 consecutive columns -> 32 registers per thread.
__device__ __forceinline__ void ld_32x32b_x32(uint32_t taddr, uint32_t (&r)[32]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
}
// 32 lanes x 32 bits, 8 consecutive columns -> 8 registers per thread.
__device__ __forceinline__ void ld_32x32b_x8(uint32_t taddr, uint32_t (&r)[8]) {
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
                 : "r"(taddr));
}
__device__ __forceinline__ void ld_wait() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// ---- swizzled shared-memory addressing (matches the descriptors above) ------------
// Byte offset of (row, kbyte) inside a K-major SW128 tile whose K extent is
// split into 128-byte blocks of `rows` rows each (block-major).
__host__ __device__ __forceinline__ uint32_t sw128_offset(uint32_t row, uint32_t kbyte, uint32_t rows) {
    const uint32_t blk = kbyte >> 7, kb = kbyte & 127u;
    const uint32_t chunk = (kb >> 4) ^ (row & 7u);
    return blk * rows * 128u + (row >> 3) * 1024u + (row & 7u) * 128u + (chunk << 4) + (kb & 15u);
}
// Byte offset of (row, kbyte < 32) inside a K-major SW32 tile (16-byte chunk
// index XOR bit 2 of the row).
__host__ __device__ __forceinline__ uint32_t sw32_offset(uint32_t row, uint32_t kbyte) {
    const uint32_t chunk = ((kbyte >> 4) & 1u) ^ ((row >> 2) & 1u);
    return (row >> 3) * 256u + (row & 7u) * 32u + (chunk << 4) + (kbyte & 15u);
}
// Byte offset of (row, kbyte < 64) inside a K-major SW64 tile.
__host__ __device__ __forceinline__ uint32_t sw64_offset(uint32_t row, uint32_t kbyte) {
    const uint32_t chunk = (kbyte >> 4) ^ ((row >> 1) & 3u);
    return (row >> 3) * 512u + (row & 7u) * 64u + (chunk << 4) + (kbyte & 15u);
}

}  // namespace tc
}  // namespace nttb
