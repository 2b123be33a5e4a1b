// tc_dmma.cu -- FP64 tensor-core engine (mma.sync.aligned.m8n8k4.f64), the
// plain drop-in form.  Same two passes and global layouts as the INT8 engine
// (tc_int8.cu); only the inner DFT-64 differs.
//
// DFT-64 of one vector x[8*j1 + j0] on one warp as two radix-8 contractions:
//   T  = W8a . X          X[j1][j0] = x[8 j1 + j0]          (4 MMAs)
//   T' = T o H            H[k0][j0] = omega_64^(j0 k0) (* psi fold)
//   Y  = T' . W8b         y[k0 + 8 k1] = Y[k0][k1]          (4 MMAs)
// The second contraction consumes T' straight from the accumulator
// fragments by splitting its K dimension into even and odd columns.
//
// Exactness: the constant matrices hold V = W * 2^64 mod q split into 16-bit
// halves V = 2^16 Vh + Vl (Vh < 2^15, Vl < 2^16); with x < 2^32 every FP64
// partial sum of eight products is < 2^51, so the MMAs are exact.  Then
//   H = sum Vh x, L = sum Vl x,  2^16 H + L == 2^64 W x  (mod q)
//   y = REDC(2^16 REDC(H) + REDC(L)) == W x  (mod q),  y in [0, 2q).
#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

#include "../../include/ntt_b200.h"
#include "bounds.cuh"
#include "plan.hpp"
#include "profiler.hpp"

namespace nttb {

// NTT_DEBUG_BOUNDS build: failed range checks (bounds.cuh bits)
__device__ uint32_t g_dmma_bounds;

namespace {

// Per-modulus constants for one direction.
struct DmLimb {
    uint32_t q, qinv, one_m, pad_;
    // radix-8 matrices, V = W * 2^64 mod q split (hi, lo); [k][j] row-major
    uint32_t a_hi[3][64], a_lo[3][64];  // step-1 matrix: [0] pass A, [1] pass B level 1
    uint32_t b_hi[64], b_lo[64];        // step-2 matrix (plain radix-8 DFT)
    uint32_t hada[2][64];               // Hadamard (Montgomery form): [0] pass A, [1] pass B level 1
    uint32_t w16[8];                    // omega_16^k, k < 8 (Montgomery form), DFT-16 butterflies
    uint32_t out16[16];                 // DFT-16 output scaling (Montgomery form)
    const uint32_t* a_start;            // pass A twiddle: a_start[b] * a_pow[(b * k) mod n] * a_post[k]
    const uint32_t* a_pow;
    const uint32_t* a_post;             // 64 entries
    const uint32_t* b_tw;               // pass B level-1 twiddle: b_tw[b2 * 64 + d2]
};

struct DmCache {
    DmLimb* d_fwd = nullptr;
    DmLimb* d_inv = nullptr;
    void* d_tabs = nullptr;
};

__device__ __forceinline__ uint32_t redc64(uint64_t v, uint32_t q, uint32_t qinv) {
    const uint32_t m = (uint32_t)v * qinv;
    return (uint32_t)((v + (uint64_t)m * q) >> 32);
}
__device__ __forceinline__ uint32_t mont(uint32_t a, uint32_t b, uint32_t q, uint32_t qinv) {
    return redc64((uint64_t)a * b, q, qinv);
}
__device__ __forceinline__ uint32_t canon(uint32_t x, uint32_t q) { return x >= q ? x - q : x; }

__device__ __forceinline__ void dmma(double& d0, double& d1, double a, double b, double c0, double c1) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%4,%5};"
                 : "=d"(d0), "=d"(d1)
                 : "d"(a), "d"(b), "d"(c0), "d"(c1));
}

// y = REDC(2^16 REDC(H) + REDC(L)) for exact FP64 accumulators H, L.
__device__ __forceinline__ uint32_t recombine(double h, double l, uint32_t q, uint32_t qinv) {
    const uint32_t rh = redc64((uint64_t)h, q, qinv);
    const uint32_t rl = redc64((uint64_t)l, q, qinv);
    return redc64(((uint64_t)rh << 16) + rl, q, qinv);
}

// DFT-64 of the vector held in `row` (64 residues < 2^32, shared memory).
// Lane t returns y[k0 + 8*(2*(t%4) + e)] in out[e], k0 = t/4.
__device__ __forceinline__ void dft64_warp(const uint32_t* row, const DmLimb& L, int which, uint32_t lane,
                                           uint32_t out[2]) {
    const uint32_t q = L.q, qinv = L.qinv;
    const uint32_t r = lane >> 2, c = lane & 3;
    // step 1: A = W8a[k0][j1] (K halves j1 in {c, c+4}), B = X[j1][j0] (j1 = c or c+4, j0 = r)
    const double xb0 = (double)row[8 * c + r], xb1 = (double)row[8 * (c + 4) + r];
    const double ah0 = (double)L.a_hi[which][r * 8 + c], ah1 = (double)L.a_hi[which][r * 8 + c + 4];
    const double al0 = (double)L.a_lo[which][r * 8 + c], al1 = (double)L.a_lo[which][r * 8 + c + 4];
    double h0 = 0, h1 = 0, l0 = 0, l1 = 0;
    dmma(h0, h1, ah0, xb0, 0.0, 0.0);
    dmma(h0, h1, ah1, xb1, h0, h1);
    dmma(l0, l1, al0, xb0, 0.0, 0.0);
    dmma(l0, l1, al1, xb1, l0, l1);
    // lane holds T[k0 = r][j0 = 2c + e]; Hadamard
    const uint32_t t0 = mont(recombine(h0, l0, q, qinv), L.hada[which][r * 8 + 2 * c], q, qinv);
    const uint32_t t1 = mont(recombine(h1, l1, q, qinv), L.hada[which][r * 8 + 2 * c + 1], q, qinv);
    // step 2: A_even[k0][i] = T'[k0][2i] (= t0), A_odd = T'[k0][2i+1] (= t1);
    //         B_even[i][k1] = W8b[2i][k1], B_odd = W8b[2i+1][k1]; lane: i = c, k1 = r
    const double bh0 = (double)L.b_hi[(2 * c) * 8 + r], bh1 = (double)L.b_hi[(2 * c + 1) * 8 + r];
    const double bl0 = (double)L.b_lo[(2 * c) * 8 + r], bl1 = (double)L.b_lo[(2 * c + 1) * 8 + r];
    const double a0 = (double)t0, a1 = (double)t1;
    h0 = h1 = l0 = l1 = 0;
    dmma(h0, h1, a0, bh0, 0.0, 0.0);
    dmma(h0, h1, a1, bh1, h0, h1);
    dmma(l0, l1, a0, bl0, 0.0, 0.0);
    dmma(l0, l1, a1, bl1, l0, l1);
    out[0] = recombine(h0, l0, q, qinv);  // Y[k0 = r][k1 = 2c]
    out[1] = recombine(h1, l1, q, qinv);  // Y[k0 = r][k1 = 2c + 1]
}

constexpr uint32_t kRow = 65;  // padded row stride (words)

// ============================================================ pass A (N = 2^16)
__global__ void __launch_bounds__(128) dmma_pass_a_n16(const uint32_t* __restrict__ src, uint32_t* __restrict__ dst,
                                                       const DmLimb* __restrict__ limbs, uint32_t n_limbs) {
    __shared__ uint32_t X[128 * kRow];
    const uint32_t tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const uint32_t limb = blockIdx.y, poly = blockIdx.z, b0 = blockIdx.x * 128u;
    const DmLimb& L = limbs[limb];
    const uint64_t off = ((uint64_t)poly * n_limbs + limb) << 16;
    const uint32_t* x = src + off;
    uint32_t* out = dst + off;
    if (!NTTB_CHECK(g_dmma_bounds, kBoundsGlobal, b0 + 127u < 1024u && limb < n_limbs)) return;
    {
        uint32_t v[64];
        const uint32_t* col = x + b0 + tid;
#pragma unroll
        for (uint32_t a = 0; a < 64; a++) v[a] = __ldg(col + a * 1024u);
#pragma unroll
        for (uint32_t a = 0; a < 64; a++) X[tid * kRow + a] = v[a];
    }
    __syncthreads();
    const uint32_t q = L.q, qinv = L.qinv;
    const uint32_t k0 = (lane >> 2) + 16u * (lane & 3u), k1 = k0 + 8u;  // output indices held by this lane
    const uint32_t post0 = L.a_post[k0], post1 = L.a_post[k1];
    for (uint32_t i = 0; i < 32; i++) {
        const uint32_t m = warp * 32u + i, b = b0 + m;
        uint32_t y[2];
        dft64_warp(X + m * kRow, L, 0, lane, y);
        const uint32_t st = L.a_start[b];
        uint32_t t0 = mont(mont(L.a_pow[(b * k0) & 0xFFFFu], st, q, qinv), post0, q, qinv);
        uint32_t t1 = mont(mont(L.a_pow[(b * k1) & 0xFFFFu], st, q, qinv), post1, q, qinv);
        const uint32_t o0 = canon(mont(y[0], canon(t0, q), q, qinv), q), o1 = canon(mont(y[1], canon(t1, q), q, qinv), q);
        (void)NTTB_CHECK(g_dmma_bounds, kBoundsResidue, o0 < q && o1 < q);
        if (NTTB_CHECK(g_dmma_bounds, kBoundsGlobal, b * 64u + k1 < 65536u && k0 < 64u)) {
            out[(uint64_t)b * 64u + k0] = o0;
            out[(uint64_t)b * 64u + k1] = o1;
        }
    }
}

// ============================================================ pass B (N = 2^16)
__global__ void __launch_bounds__(128) dmma_pass_b_n16(const uint32_t* src, uint32_t* dst,
                                                       const DmLimb* __restrict__ limbs, uint32_t n_limbs) {
    __shared__ uint32_t X[512 * 17];  // level 1: 128 vectors x 65 words; then level 2: 512 rows x 17 words
    const uint32_t tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const uint32_t limb = blockIdx.y, poly = blockIdx.z, d0 = blockIdx.x * 8u;
    const DmLimb& L = limbs[limb];
    const uint64_t off = ((uint64_t)poly * n_limbs + limb) << 16;
    const uint32_t* u = src + off;
    uint32_t* out = dst + off;
    const uint32_t q = L.q, qinv = L.qinv;
    if (!NTTB_CHECK(g_dmma_bounds, kBoundsGlobal, d0 + 7u < 64u && limb < n_limbs)) return;
    {
        const uint32_t r = tid & 7u, b2 = tid >> 3;
        const uint32_t* base = u + d0 + r;
        uint32_t v[64];
#pragma unroll
        for (uint32_t a2 = 0; a2 < 64; a2++) v[a2] = base[(a2 * 16u + b2) * 64u];
#pragma unroll
        for (uint32_t a2 = 0; a2 < 64; a2++) X[tid * kRow + a2] = v[a2];
    }
    __syncthreads();
    // level 1: vector m = (r = m & 7, b2 = m >> 3); keep the 64 outputs in registers
    const uint32_t k0 = (lane >> 2) + 16u * (lane & 3u), k1 = k0 + 8u;
    uint32_t keep[32][2];
#pragma unroll
    for (uint32_t i = 0; i < 32; i++) {
        const uint32_t m = warp * 32u + i, b2 = m >> 3;
        uint32_t y[2];
        dft64_warp(X + m * kRow, L, 1, lane, y);
        keep[i][0] = mont(y[0], L.b_tw[b2 * 64u + k0], q, qinv);
        keep[i][1] = mont(y[1], L.b_tw[b2 * 64u + k1], q, qinv);
    }
    __syncthreads();
    // A2[row = d2*8 + r][b2] with a 17-word row stride
#pragma unroll
    for (uint32_t i = 0; i < 32; i++) {
        const uint32_t m = warp * 32u + i, r = m & 7u, b2 = m >> 3;
        X[(k0 * 8u + r) * 17u + b2] = keep[i][0];
        X[(k1 * 8u + r) * 17u + b2] = keep[i][1];
    }
    __syncthreads();
    // level 2: DFT-16 over b2 for each of the 512 rows (4 per thread), radix-2 DIT
    for (uint32_t row = tid; row < 512; row += 128) {
        uint32_t z[16];
#pragma unroll
        for (uint32_t i = 0; i < 16; i++) {
            const uint32_t br = ((i & 1) << 3) | ((i & 2) << 1) | ((i & 4) >> 1) | ((i & 8) >> 3);
            z[i] = canon(X[row * 17u + br], q);
        }
#pragma unroll
        for (uint32_t s = 0; s < 4; s++) {
            const uint32_t half = 1u << s;
#pragma unroll
            for (uint32_t j = 0; j < 8; j++) {
                const uint32_t p = j & (half - 1), i0 = ((j >> s) << (s + 1)) | p, i1 = i0 + half;
                const uint32_t w = L.w16[p << (3 - s)];
                const uint32_t t = canon(mont(z[i1], w, q, qinv), q);
                const uint32_t a = z[i0];
                z[i0] = canon(a + t, q);
                z[i1] = canon(a + q - t, q);
            }
        }
        const uint32_t d2 = row >> 3, r = row & 7u;
        uint32_t* o = out + d0 + r + 64u * d2;
#pragma unroll
        for (uint32_t c = 0; c < 16; c++) {
            const uint32_t v = canon(mont(z[c], L.out16[c], q, qinv), q);
            (void)NTTB_CHECK(g_dmma_bounds, kBoundsResidue, v < q);
            o[4096u * c] = v;
        }
    }
}

// ---- host ------------------------------------------------------------------------
void split_matrix(uint32_t* hi, uint32_t* lo, const std::vector<uint64_t>& W, uint64_t q) {
    for (int i = 0; i < 64; i++) {
        const uint64_t v = h_to_mont32(h_to_mont32(W[i], q), q);  // W * 2^64 mod q
        hi[i] = (uint32_t)(v >> 16);
        lo[i] = (uint32_t)(v & 0xFFFF);
    }
}

std::vector<uint64_t> mat8(uint64_t w8, uint64_t q, uint64_t col_twist = 1) {
    std::vector<uint64_t> W(64);
    for (uint32_t k = 0; k < 8; k++)
        for (uint32_t j = 0; j < 8; j++)
            W[k * 8 + j] = h_mulmod(h_powmod(w8, (uint64_t)j * k, q), h_powmod(col_twist, j, q), q);
    return W;
}

int build_dm(Plan32& p, DmCache* c) {
    const uint32_t n = p.n, nl = p.n_limbs;
    // device tables per limb and direction: a_start (1024), a_pow (n), a_post (64), b_tw (1024)
    const size_t per_dir = 1024 + (size_t)n + 64 + 1024, per_limb = 2 * per_dir;
    std::vector<uint32_t> tabs(per_limb * nl);
    uint32_t* d_tabs = nullptr;
    if (cudaMalloc(&d_tabs, tabs.size() * 4) != cudaSuccess) return 4;
    std::vector<DmLimb> fwd(nl), inv(nl);
    for (uint32_t l = 0; l < nl; l++) {
        const LimbHost& H = p.limbs[l];
        const uint64_t q = H.q;
        for (int dir = 0; dir < 2; dir++) {
            const bool iv = dir == 1;
            DmLimb D{};
            D.q = (uint32_t)q;
            D.qinv = h_neg_inv32((uint32_t)q);
            D.one_m = h_to_mont32(1, q);
            const uint64_t w = iv ? H.omega_inv : H.omega;
            const uint64_t w8 = h_powmod(w, n / 8, q), w64 = h_powmod(w, n / 64, q), w16 = h_powmod(w, n / 16, q);
            const bool nega_pre = p.negacyclic && !iv;
            // pass A step 1: negacyclic forward folds psi^(1024 j) = psi_16^j1 * psi_128^j0
            const uint64_t psi128 = nega_pre ? h_powmod(H.psi, n / 64, q) : 1;
            split_matrix(D.a_hi[0], D.a_lo[0], mat8(w8, q, h_powmod(psi128, 8, q)), q);
            split_matrix(D.a_hi[1], D.a_lo[1], mat8(w8, q), q);
            split_matrix(D.b_hi, D.b_lo, mat8(w8, q), q);
            for (uint32_t k0 = 0; k0 < 8; k0++)
                for (uint32_t j0 = 0; j0 < 8; j0++) {
                    const uint64_t hd = h_powmod(w64, (uint64_t)j0 * k0, q);
                    D.hada[0][k0 * 8 + j0] = h_to_mont32(h_mulmod(hd, h_powmod(psi128, j0, q), q), q);
                    D.hada[1][k0 * 8 + j0] = h_to_mont32(hd, q);
                }
            for (uint32_t k = 0; k < 8; k++) D.w16[k] = h_to_mont32(h_powmod(w16, k, q), q);
            for (uint32_t c2 = 0; c2 < 16; c2++) {
                uint64_t s = 1;
                if (iv) s = p.negacyclic ? h_mulmod(H.n_inv, h_powmod(H.psi_inv, 4096ull * c2, q), q) : H.n_inv;
                D.out16[c2] = h_to_mont32(s, q);
            }
            uint32_t* t = tabs.data() + per_limb * l + per_dir * dir;
            uint32_t* dt = d_tabs + per_limb * l + per_dir * dir;
            for (uint32_t b = 0; b < 1024; b++) t[b] = h_to_mont32(nega_pre ? h_powmod(H.psi, b, q) : 1, q);
            for (uint32_t e = 0; e < n; e++) t[1024 + e] = h_to_mont32(h_powmod(w, e, q), q);
            for (uint32_t k = 0; k < 64; k++)
                t[1024 + n + k] = h_to_mont32((iv && p.negacyclic) ? h_powmod(H.psi_inv, k, q) : 1, q);
            for (uint32_t b2 = 0; b2 < 16; b2++)
                for (uint32_t d2 = 0; d2 < 64; d2++) {
                    uint64_t v = h_powmod(w, 64ull * b2 * d2, q);
                    if (iv && p.negacyclic) v = h_mulmod(v, h_powmod(H.psi_inv, 64ull * d2, q), q);
                    t[1024 + n + 64 + b2 * 64 + d2] = h_to_mont32(v, q);
                }
            D.a_start = dt;
            D.a_pow = dt + 1024;
            D.a_post = dt + 1024 + n;
            D.b_tw = dt + 1024 + n + 64;
            (iv ? inv : fwd)[l] = D;
        }
    }
    if (cudaMemcpy(d_tabs, tabs.data(), tabs.size() * 4, cudaMemcpyHostToDevice) != cudaSuccess) {
        cudaFree(d_tabs);
        return 3;
    }
    DmLimb* d_l = nullptr;
    if (cudaMalloc(&d_l, 2 * nl * sizeof(DmLimb)) != cudaSuccess) {
        cudaFree(d_tabs);
        return 4;
    }
    if (cudaMemcpy(d_l, fwd.data(), nl * sizeof(DmLimb), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(d_l + nl, inv.data(), nl * sizeof(DmLimb), cudaMemcpyHostToDevice) != cudaSuccess) {
        cudaFree(d_l);
        cudaFree(d_tabs);
        return 3;
    }
    c->d_fwd = d_l;
    c->d_inv = d_l + nl;
    c->d_tabs = d_tabs;
    return 0;
}

}  // namespace

uint32_t dmma_bounds_errors(bool clear) {
    uint32_t v = 0;
    cudaMemcpyFromSymbol(&v, g_dmma_bounds, sizeof v);
    if (clear) {
        uint32_t z = 0;
        cudaMemcpyToSymbol(g_dmma_bounds, &z, sizeof z);
    }
    return v;
}

bool dmma_serves(const Plan32& p, bool src_u64) { return !src_u64 && p.log_n == 16; }

int dmma_transform32(Plan32& p, const void* src, void* dst, bool src_u64, uint32_t n_polys, bool inverse,
                     cudaStream_t s) {
    if (!dmma_serves(p, src_u64) || n_polys > 65535 || p.n_limbs > 65535) return 1;
    DmCache* c;
    {
        std::lock_guard<std::mutex> lock(p.engine_mu);
        c = reinterpret_cast<DmCache*>(p.engine_data[2]);
        if (!c) {
            c = new DmCache();
            if (build_dm(p, c)) {
                delete c;
                return 2;
            }
            p.engine_data[2] = c;
        }
    }
    const uint32_t* in = static_cast<const uint32_t*>(src);
    uint32_t* out = static_cast<uint32_t*>(dst);
    uint32_t* mid = out;
    if (src == dst) {
        mid = static_cast<uint32_t*>(plan_workspace(&p.ws, &p.ws_bytes, (size_t)n_polys * p.n_limbs * p.n * 4));
        if (!mid) return 2;
    }
    const DmLimb* limbs = inverse ? c->d_inv : c->d_fwd;
    {
        ProfScope prof("dmma_pass_a_n16", s);
        dmma_pass_a_n16<<<dim3(8, p.n_limbs, n_polys), 128, 0, s>>>(in, mid, limbs, p.n_limbs);
    }
    {
        ProfScope prof("dmma_pass_b_n16", s);
        dmma_pass_b_n16<<<dim3(8, p.n_limbs, n_polys), 128, 0, s>>>(mid, out, limbs, p.n_limbs);
    }
    return launch_rc();
}

void dmma_release(Plan32* p) {
    auto* c = reinterpret_cast<DmCache*>(p->engine_data[2]);
    if (!c) return;
    if (c->d_fwd) cudaFree(c->d_fwd);
    if (c->d_tabs) cudaFree(c->d_tabs);
    delete c;
    p->engine_data[2] = nullptr;
}

}  // namespace nttb
