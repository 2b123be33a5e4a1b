// scalar_engine.cu -- CUDA-core engine: each pass computes a batch of DFTs of
// length `len` entirely in shared memory (radix-2, DIT after a bit-reversed
// load or DIF before a bit-reversed store, whichever keeps the shared-memory
// traffic conflict-free for the pass's global access order), with the
// four-step twiddles and the negacyclic twists fused into the load/store.
//
// It serves every size and modulus width and is the engine of the 60-bit
// path; the tensor-core engines replace it for the hot 31-bit sizes.
//
// Two-pass decomposition for n = N1 * N2 (input index a*N2 + b):
//   pass A (MODE_COL):     U[d][b] = DFT_N1(x[.][b])[d] * root^(d*b)
//   pass B (MODE_ROW_NAT): X[d + N1*c] = DFT_N2(U[d][.])[c]
#include <cuda_runtime.h>

#include "plan.hpp"
#include "profiler.hpp"

namespace nttb {

namespace {

constexpr int kThreads = 256;

// Shared-memory row layout: element i of a vector at i + (i >> pad_shift)
// (one pad element per 32 words), so that the register groups' strided
// loads and stores spread over the banks; rows `tile_stride` apart.
template <class E>
__host__ __device__ constexpr uint32_t pad_shift() { return sizeof(E) == 8 ? 4u : 5u; }
template <class E>
__host__ __device__ inline uint32_t tile_stride(uint32_t L) { return L + (L >> pad_shift<E>()) + 1; }

template <class S, class A, int MODE>
__global__ void __launch_bounds__(kThreads) scalar_pass_kernel(PassArgs args, const LimbDev<A>* limbs) {
    using E = typename A::elem;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const uint32_t L = args.len, V = args.vec_per_tile, lgL = args.log_len;
    // every extent is a power of two: index splits are shifts and masks
    const uint32_t lgV = 31 - __clz(V), lgN1 = 31 - __clz(args.n1);
    const uint32_t stride = tile_stride<E>(L);
    constexpr uint32_t kPad = pad_shift<E>();
    E* t = reinterpret_cast<E*>(smem_raw);
    E* tws = t + (((size_t)V * stride + 1) & ~(size_t)1);  // pair-aligned

    const uint32_t limb = blockIdx.y, poly = blockIdx.z;
    const uint32_t v0 = blockIdx.x * V;  // first vector of this tile
    const LimbDev<A> ld = limbs[limb];
    const A ar = ld.ar;
    const uint64_t off = (uint64_t)poly * args.poly_stride + (uint64_t)limb * args.n;
    const S* src = reinterpret_cast<const S*>(args.src) + off;
    S* dst = reinterpret_cast<S*>(args.dst) + off;
    const E* tw = args.inverse ? ld.tw_inv : ld.tw;
    const uint32_t nmask = args.n - 1, N1 = args.n1, N2 = args.n2;
    const uint32_t total = V * L;
    const uint32_t flags = args.flags;

    // Shoup pairs of the length-L root: tws[2k] = root_L^k (plain form),
    // tws[2k + 1] its quotient, k < L/2; the butterflies multiply by them
    // with one high and two low products (the Montgomery product takes two
    // of each), giving the same canonical Montgomery-form results
    if (L >= 2) {  // a pass of length 1 has no butterflies (and no level 0)
        const E* sh = (args.inverse ? ld.tw_inv_sh : ld.tw_sh) + 2 * (size_t)((L >> 1) - 1);  // level lgL
        for (uint32_t k = threadIdx.x; k < L; k += blockDim.x) tws[k] = sh[k];
    }

    constexpr bool kDIT = (MODE == MODE_COL || MODE == MODE_GATHER_T);

    // Column passes with at most one vector per thread of the block keep a
    // thread on one column: its elements j (or outputs k) step by
    // kThreads / V, so the negacyclic twist psi^(j N2 + col) and the
    // four-step twiddle root^(k col) are geometric along them and are
    // generated by one product per element instead of a table gather.
    const bool chain = MODE == MODE_COL && V <= (uint32_t)kThreads;
    const uint32_t lane_v = threadIdx.x & (V - 1), step_j = (uint32_t)kThreads >> lgV;
    E psi_cur = 0, psi_step = 0;
    if (chain && (flags & F_PRE_PSI) && (threadIdx.x >> lgV) < L) {
        psi_cur = ld.psi[(uint64_t)(threadIdx.x >> lgV) * N2 + v0 + lane_v];
        const uint64_t e = (uint64_t)step_j * N2;
        psi_step = e < args.n ? ld.psi[e] : tw[0];  // tw[0] = 1 (Montgomery form)
    }
    // ---- load ----
    // Batches of kLoadBatch elements per thread: the global loads of a batch
    // are issued together, then twisted and stored to shared memory in the
    // same order (the twist chains advance per element).
    auto load_pos = [&](uint32_t idx, uint32_t& v, uint32_t& j) -> uint64_t {
        if (kDIT) { v = idx & (V - 1); j = idx >> lgV; } else { v = idx >> lgL; j = idx & (L - 1); }
        const uint32_t vec = v0 + v;
        if (MODE == MODE_COL) return (uint64_t)j * N2 + vec;
        if (MODE == MODE_ROW_NAT) return (uint64_t)vec * N2 + j;
        if (MODE == MODE_GATHER_T) {
            const uint64_t m = (uint64_t)vec * L + j;  // index into the transposed view
            return (m & (N1 - 1)) * N2 + (m >> lgN1);
        }
        return (uint64_t)vec * L + j;
    };
    constexpr uint32_t kLoadBatch = 8;
    for (uint32_t idx0 = threadIdx.x; idx0 < total; idx0 += blockDim.x * kLoadBatch) {
        S raw[kLoadBatch];
#pragma unroll
        for (uint32_t u = 0; u < kLoadBatch; u++) {
            const uint32_t idx = idx0 + u * blockDim.x;
            uint32_t v, j;
            if (idx < total) raw[u] = src[load_pos(idx, v, j)];
        }
#pragma unroll
        for (uint32_t u = 0; u < kLoadBatch; u++) {
            const uint32_t idx = idx0 + u * blockDim.x;
            if (idx >= total) break;
            uint32_t v, j;
            const uint64_t pos = load_pos(idx, v, j);
            const uint32_t vec = v0 + v;
            E x = (E)raw[u];
            if (flags & F_PRE_PSI) {
                if (chain) {
                    x = ar.mul(x, psi_cur);
                    psi_cur = ar.mul(psi_cur, psi_step);
                } else {
                    x = ar.mul(x, ld.psi[pos]);
                }
            }
            if (flags & F_PRE_TW) x = ar.mul(x, tw[((uint64_t)j * vec) & nmask]);
            const uint32_t jj = kDIT ? bitrev(j, (int)lgL) : j;
            t[(size_t)v * stride + jj + (jj >> kPad)] = x;
        }
    }
    __syncthreads();

    // ---- radix-2 stages, up to three at a time in registers ----
    // A group of r stages s0 .. s0+r-1 touches, for each base index with zero
    // bits [s0, s0 + r), exactly the 2^r elements base + k 2^s0; one thread
    // loads them, runs the group's butterflies (the same butterflies, in the
    // same order, as one stage at a time) and stores them back.
    constexpr uint32_t kG = 3, kGN = 1u << kG;
    if (kDIT) {
        for (uint32_t s0 = 0; s0 < lgL; s0 += kG) {
            const uint32_t r = lgL - s0 < kG ? lgL - s0 : kG, nk = 1u << r;
            const uint32_t items = V << (lgL - r);
            for (uint32_t it = threadIdx.x; it < items; it += blockDim.x) {
                const uint32_t v = it & (V - 1), g = it >> lgV;
                const uint32_t low = g & ((1u << s0) - 1), base = ((g >> s0) << (s0 + r)) | low;
                E* row = t + (size_t)v * stride;
                E x[kGN];
#pragma unroll
                for (uint32_t k = 0; k < kGN; k++)
                    if (k < nk) {
                        const uint32_t i = base + (k << s0);
                        x[k] = row[i + (i >> kPad)];
                    }
#pragma unroll
                for (uint32_t tt = 0; tt < kG; tt++) {
                    if (tt >= r) break;
                    const uint32_t st = s0 + tt, half = 1u << tt;
#pragma unroll
                    for (uint32_t k = 0; k < kGN; k++) {
                        if ((k & half) || k + half >= nk) continue;
                        const uint32_t p = (low + ((k & (half - 1)) << s0)) << (lgL - 1 - st);
                        if constexpr (A::kLazy) {
                            // values in [0, 4q): u0 to [0, 2q), y = w x in [0, 2q)
                            const E u0 = ar.below2q(x[k]);
                            const E y = ar.mul_shoup_lazy(x[k + half], tws[2 * p], tws[2 * p + 1]);
                            x[k] = u0 + y;
                            x[k + half] = u0 - y + 2 * ar.q;
                        } else {
                            const E y = ar.mul_shoup(x[k + half], tws[2 * p], tws[2 * p + 1]);
                            const E u0 = x[k];
                            x[k] = ar.add(u0, y);
                            x[k + half] = ar.sub(u0, y);
                        }
                    }
                }
#pragma unroll
                for (uint32_t k = 0; k < kGN; k++)
                    if (k < nk) {
                        const uint32_t i = base + (k << s0);
                        row[i + (i >> kPad)] = x[k];
                    }
            }
            __syncthreads();
        }
    } else {
        // DIF: stages from lgL-1 down, groups [s_lo, s_lo + r)
        for (int s_hi = (int)lgL - 1; s_hi >= 0; s_hi -= (int)kG) {
            const uint32_t r = (uint32_t)s_hi + 1 < kG ? (uint32_t)s_hi + 1 : kG, nk = 1u << r;
            const uint32_t s_lo = (uint32_t)s_hi + 1 - r, lgG = lgL - r;
            const uint32_t items = V << lgG;
            for (uint32_t it = threadIdx.x; it < items; it += blockDim.x) {
                const uint32_t v = it >> lgG, g = it & ((1u << lgG) - 1);
                const uint32_t low = g & ((1u << s_lo) - 1), base = ((g >> s_lo) << (s_lo + r)) | low;
                E* row = t + (size_t)v * stride;
                E x[kGN];
#pragma unroll
                for (uint32_t k = 0; k < kGN; k++)
                    if (k < nk) {
                        const uint32_t i = base + (k << s_lo);
                        x[k] = row[i + (i >> kPad)];
                    }
#pragma unroll
                for (int tt = (int)kG - 1; tt >= 0; tt--) {
                    if ((uint32_t)tt >= r) continue;
                    const uint32_t st = s_lo + (uint32_t)tt, half = 1u << tt;
#pragma unroll
                    for (uint32_t k = 0; k < kGN; k++) {
                        if ((k & half) || k + half >= nk) continue;
                        const uint32_t p = (low + ((k & (half - 1)) << s_lo)) << (lgL - 1 - st);
                        const E u0 = x[k], y = x[k + half];
                        if constexpr (A::kLazy) {
                            // values in [0, 2q)
                            x[k] = ar.below2q(u0 + y);
                            x[k + half] = ar.mul_shoup_lazy(u0 - y + 2 * ar.q, tws[2 * p], tws[2 * p + 1]);
                        } else {
                            x[k] = ar.add(u0, y);
                            x[k + half] = ar.mul_shoup(ar.sub(u0, y), tws[2 * p], tws[2 * p + 1]);
                        }
                    }
                }
#pragma unroll
                for (uint32_t k = 0; k < kGN; k++)
                    if (k < nk) {
                        const uint32_t i = base + (k << s_lo);
                        row[i + (i >> kPad)] = x[k];
                    }
            }
            __syncthreads();
        }
    }

    E tw_cur = 0, tw_step = 0;
    if (chain && (flags & F_POST_TW) && (threadIdx.x >> lgV) < L) {
        const uint64_t col = v0 + lane_v;
        tw_cur = tw[((uint64_t)(threadIdx.x >> lgV) * col) & nmask];
        tw_step = tw[((uint64_t)step_j * col) & nmask];
    }
    // ---- store ----
    for (uint32_t idx = threadIdx.x; idx < total; idx += blockDim.x) {
        uint32_t v, k;
        // row-contiguous outputs: consecutive threads take consecutive k
        if (MODE == MODE_GATHER_T || (MODE == MODE_ROW_NAT && (flags & F_STORE_T))) {
            v = idx >> lgL;
            k = idx & (L - 1);
        } else {
            v = idx & (V - 1);
            k = idx >> lgV;
        }
        const uint32_t vec = v0 + v;
        const uint32_t kk = kDIT ? k : bitrev(k, (int)lgL);
        E x = t[(size_t)v * stride + kk + (kk >> kPad)];
        if constexpr (A::kLazy) x = ar.canon4(x);  // lazy butterflies leave [0, 4q)
        uint64_t pos;
        if (MODE == MODE_COL) {
            pos = (flags & F_STORE_T) ? (uint64_t)vec * N1 + k : (uint64_t)k * N2 + vec;
            if (flags & F_POST_TW) {
                if (chain) {
                    x = ar.mul(x, tw_cur);
                    tw_cur = ar.mul(tw_cur, tw_step);
                } else {
                    x = ar.mul(x, tw[((uint64_t)k * vec) & nmask]);
                }
            }
        } else if (MODE == MODE_ROW_NAT) {
            pos = (flags & F_STORE_T) ? (uint64_t)vec * L + k : (uint64_t)vec + (uint64_t)N1 * k;
            if (flags & F_POST_TW) x = ar.mul(x, tw[((uint64_t)k * vec) & nmask]);
        } else if (MODE == MODE_GATHER_T) {
            pos = (uint64_t)vec * L + k;
        } else {
            const uint64_t m = (uint64_t)vec * L + k;
            pos = (m & (N1 - 1)) * N2 + (m >> lgN1);  // transpose n2 x n1 -> n1 x n2
        }
        if (flags & F_POST_PSI_INV) x = ar.mul(x, ld.psi_inv[pos]);
        else if (flags & F_POST_SCALE) x = ar.mul(x, ld.ninv_m);
        dst[pos] = (S)x;
    }
}

template <class S, class A>
int launch_pass(int mode, const PassArgs& a, const LimbDev<A>* d_limbs, uint32_t n_vectors,
                uint32_t n_polys, cudaStream_t s) {
    using E = typename A::elem;
    const size_t smem = ((((size_t)a.vec_per_tile * tile_stride<E>(a.len) + 1) & ~(size_t)1) + a.len + 2) * sizeof(E);
    dim3 grid(n_vectors / a.vec_per_tile, a.n_limbs, n_polys);
    if (grid.x == 0 || n_polys > 65535 || a.n_limbs > 65535) return 1;
    void (*k)(PassArgs, const LimbDev<A>*) = nullptr;
    switch (mode) {
        case MODE_COL: k = scalar_pass_kernel<S, A, MODE_COL>; break;
        case MODE_ROW_NAT: k = scalar_pass_kernel<S, A, MODE_ROW_NAT>; break;
        case MODE_GATHER_T: k = scalar_pass_kernel<S, A, MODE_GATHER_T>; break;
        default: k = scalar_pass_kernel<S, A, MODE_ROW_SCATTER_T>; break;
    }
    if (smem > 48 * 1024) cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    static const char* names[4] = {"scalar_pass_col", "scalar_pass_row", "scalar_pass_gather_t",
                                   "scalar_pass_scatter_t"};
    ProfScope prof(names[mode & 3], s);
    k<<<grid, kThreads, smem, s>>>(a, d_limbs);
    return launch_rc();
}

// Vectors per tile: as many as the shared-memory tile holds, fewer while the
// pass would have under ~1024 tiles (a single large polynomial otherwise
// leaves most SMs idle), but at least two: column passes read and write
// `V` consecutive words per row, and one word per 32-byte sector cost more
// than the extra tiles gain (one 2^20 polynomial mod the 60-bit prime:
// 15.4 -> 17.9 G coefficient-transforms/s with the floor at two).
inline uint32_t tile_vectors(uint32_t e_max, uint32_t len, uint32_t n_vectors, uint32_t units) {
    uint32_t v = e_max / len < n_vectors ? e_max / len : n_vectors;
    while (v > 2 && (uint64_t)(n_vectors / v) * units < 1024) v >>= 1;
    return v;
}

// Two-pass (or single-pass) forward/inverse over a plan.  E_max bounds the
// shared-memory tile in elements.  Two-pass layout for n = N1 * N2:
//   pass A: columns b of x as [N1][N2]: U[d][b] = DFT_N1 * root^(d*b), stored
//           transposed at b*N1 + d into `mid`;
//   pass B: columns d of `mid` as [N2][N1]: X[d + N1*k] = DFT_N2, written to
//           the same positions of `dst` -- each tile reads and writes one set
//           of positions, so pass B is safe in place.
// Pass A cannot run in place; an in-place call stages it in `ws`.
// Whether a transform runs as two passes: always above the tile size e_max;
// from 2^12 on also when there are few (polynomial, limb) units, since a
// single pass gives each unit one CTA and leaves the GPU idle (one
// polynomial of 2^12 words: one CTA for all twelve stages).
constexpr uint64_t kFewUnits = 8;
inline bool two_pass(uint32_t log_n, uint32_t e_max, uint64_t units) {
    const uint32_t n = 1u << log_n;
    return n > e_max || (log_n >= 12 && units < kFewUnits);
}

template <class S, class A>
int transform_generic(uint32_t log_n, uint32_t n_limbs, bool negacyclic, const LimbDev<A>* d_limbs,
                      const void* src, void* dst, void* ws, uint32_t n_polys, bool inverse, uint32_t e_max,
                      cudaStream_t s) {
    const uint32_t n = 1u << log_n;
    PassArgs a{};
    a.poly_stride = (uint64_t)n_limbs * n;
    a.n = n;
    a.log_n = log_n;
    a.n_limbs = n_limbs;
    a.inverse = inverse ? 1 : 0;
    uint32_t pre = (!inverse && negacyclic) ? F_PRE_PSI : 0u;
    uint32_t post = inverse ? (negacyclic ? F_POST_PSI_INV : F_POST_SCALE) : 0u;
    if (!two_pass(log_n, e_max, (uint64_t)n_limbs * n_polys)) {
        // single pass: one row of length n per (poly, limb)
        a.src = src;
        a.dst = dst;
        a.n1 = 1;
        a.n2 = n;
        a.len = n;
        a.log_len = log_n;
        a.vec_per_tile = 1;
        a.flags = pre | post;
        return launch_pass<S, A>(MODE_ROW_NAT, a, d_limbs, 1, n_polys, s);
    }
    const uint32_t lg1 = (log_n + 1) / 2, lg2 = log_n - lg1;
    const uint32_t N1 = 1u << lg1, N2 = 1u << lg2;
    if (N1 > e_max) return 1;
    void* mid = (src == dst) ? ws : dst;
    if (!mid) return 2;
    // pass A: column DFTs of length N1 + four-step twiddle, transposed store
    a.src = src;
    a.dst = mid;
    a.n1 = N1;
    a.n2 = N2;
    a.len = N1;
    a.log_len = lg1;
    a.vec_per_tile = tile_vectors(e_max, N1, N2, n_limbs * n_polys);
    a.flags = pre | F_POST_TW | F_STORE_T;
    int rc = launch_pass<S, A>(MODE_COL, a, d_limbs, N2, n_polys, s);
    if (rc) return rc;
    // pass B: DFTs of length N2 over the columns of [N2][N1], natural order
    a.src = mid;
    a.dst = dst;
    a.n1 = N2;
    a.n2 = N1;
    a.len = N2;
    a.log_len = lg2;
    a.vec_per_tile = tile_vectors(e_max, N2, N1, n_limbs * n_polys);
    a.flags = post;
    return launch_pass<S, A>(MODE_COL, a, d_limbs, N1, n_polys, s);
}

}  // namespace

int scalar_transform32(Plan32& p, const void* src, void* dst, bool src_u64, uint32_t n_polys, bool inverse,
                       cudaStream_t s) {
    void* ws = nullptr;
    if (src == dst && two_pass(p.log_n, 8192, (uint64_t)n_polys * p.n_limbs)) {
        ws = plan_workspace(&p.ws, &p.ws_bytes, (size_t)n_polys * p.n_limbs * p.n * (src_u64 ? 8 : 4));
        if (!ws) return 2;
    }
    if (src_u64)
        return transform_generic<uint64_t, M32>(p.log_n, p.n_limbs, p.negacyclic, p.d_limbs, src, dst, ws, n_polys,
                                                inverse, 8192, s);
    return transform_generic<uint32_t, M32>(p.log_n, p.n_limbs, p.negacyclic, p.d_limbs, src, dst, ws, n_polys,
                                            inverse, 8192, s);
}

int scalar_transform32_ws(const Plan32& p, uint32_t* data, void* ws, uint32_t n_polys, bool inverse,
                          cudaStream_t s) {
    return transform_generic<uint32_t, M32>(p.log_n, p.n_limbs, p.negacyclic, p.d_limbs, data, data, ws, n_polys,
                                            inverse, 8192, s);
}

size_t scalar_transform32_ws_bytes(const Plan32& p, uint32_t n_polys) {
    if (!two_pass(p.log_n, 8192, (uint64_t)n_polys * p.n_limbs)) return 0;
    return (size_t)n_polys * p.n_limbs * p.n * sizeof(uint32_t);
}

int scalar_transform64(Plan64& p, const void* src, void* dst, uint32_t n_polys, bool inverse, cudaStream_t s) {
    void* ws = nullptr;
    if (src == dst && two_pass(p.log_n, 4096, (uint64_t)n_polys * p.n_limbs)) {
        ws = plan_workspace(&p.ws, &p.ws_bytes, (size_t)n_polys * p.n_limbs * p.n * 8);
        if (!ws) return 2;
    }
    return transform_generic<uint64_t, M64>(p.log_n, p.n_limbs, p.negacyclic, p.d_limbs, src, dst, ws, n_polys,
                                            inverse, 4096, s);
}

// The RowMaj pre-transposed layout pre[b*M + a] = x[a*M + b] for n = M^2
// (the layout of rowmaj_to_pretransposed, src/ntt_optimized.cu:893-895), in
// and out, in two passes and no transpose:
//   pass A (rows of pre = columns of x): U[d][b] = DFT_M(x[.][b])[d] * root^(d*b),
//           stored at b*M + d in `mid`;
//   pass B (columns of mid): X[d + M*c] = DFT_M(U[d][.])[c], stored at d*M + c,
//           which is where pre-transposed X keeps element d + M*c.
int scalar_pretransposed32(const Plan32& p, uint64_t* data, uint64_t* mid, bool inverse, cudaStream_t s) {
    if (p.n_limbs != 1 || p.negacyclic || (p.log_n & 1u) || p.log_n < 2) return 1;
    const uint32_t lg = p.log_n / 2, M = 1u << lg, e_max = 8192;
    if (M > e_max) return 1;
    PassArgs a{};
    a.poly_stride = p.n;
    a.n = p.n;
    a.log_n = p.log_n;
    a.n_limbs = 1;
    a.inverse = inverse ? 1 : 0;
    a.n1 = M;
    a.n2 = M;
    a.len = M;
    a.log_len = lg;
    a.vec_per_tile = tile_vectors(e_max, M, M, 1);
    a.src = data;
    a.dst = mid;
    a.flags = F_POST_TW | F_STORE_T;
    int rc = launch_pass<uint64_t, M32>(MODE_ROW_NAT, a, p.d_limbs, M, 1, s);
    if (rc) return rc;
    a.src = mid;
    a.dst = data;
    a.flags = F_STORE_T | (inverse ? F_POST_SCALE : 0u);
    return launch_pass<uint64_t, M32>(MODE_COL, a, p.d_limbs, M, 1, s);
}

// The reference's four-step map (src/ntt_four_step.cu:244-392), race-free:
//   forward: column DFT-n1 + Hadamard root^(r*c)  [data -> scratch, in place layout]
//            transpose + chunked DFT-n2           [scratch -> data, one fused pass]
//   inverse: chunked DFT-n2 + transpose back      [data -> scratch]
//            Hadamard root^-(r*c) + column DFT-n1 + n^-1 [scratch -> data]
// with n1 = 2^max(6, log_n/2) capped at n, n2 = n / n1.
int scalar_four_step32(const Plan32& p, uint64_t* data, uint64_t* scratch, bool inverse, cudaStream_t s) {
    const uint32_t log_n = p.log_n, n = p.n;
    uint32_t lg1 = log_n / 2;
    if (lg1 < 6) lg1 = 6;
    if (lg1 > log_n) lg1 = log_n;
    const uint32_t lg2 = log_n - lg1, n1 = 1u << lg1, n2 = 1u << lg2;
    const uint32_t e_max = 8192;
    if (n1 > e_max || n2 > e_max) return 1;
    PassArgs a{};
    a.poly_stride = n;
    a.n = n;
    a.log_n = log_n;
    a.n_limbs = 1;
    a.n1 = n1;
    a.n2 = n2;
    a.inverse = inverse ? 1 : 0;
    int rc;
    if (!inverse) {
        a.src = data;
        a.dst = scratch;
        a.len = n1;
        a.log_len = lg1;
        a.vec_per_tile = e_max / n1 < n2 ? e_max / n1 : n2;
        a.flags = F_POST_TW;
        rc = launch_pass<uint64_t, M32>(MODE_COL, a, p.d_limbs, n2, 1, s);
        if (rc) return rc;
        a.src = scratch;
        a.dst = data;
        a.len = n2;
        a.log_len = lg2;
        a.vec_per_tile = e_max / n2 < n1 ? e_max / n2 : n1;
        a.flags = 0;
        return launch_pass<uint64_t, M32>(MODE_GATHER_T, a, p.d_limbs, n1, 1, s);
    }
    a.src = data;
    a.dst = scratch;
    a.len = n2;
    a.log_len = lg2;
    a.vec_per_tile = e_max / n2 < n1 ? e_max / n2 : n1;
    a.flags = 0;
    rc = launch_pass<uint64_t, M32>(MODE_ROW_SCATTER_T, a, p.d_limbs, n1, 1, s);
    if (rc) return rc;
    a.src = scratch;
    a.dst = data;
    a.len = n1;
    a.log_len = lg1;
    a.vec_per_tile = e_max / n1 < n2 ? e_max / n1 : n2;
    a.flags = F_PRE_TW | F_POST_SCALE;
    return launch_pass<uint64_t, M32>(MODE_COL, a, p.d_limbs, n2, 1, s);
}

}  // namespace nttb
