// capi.cu -- the extern "C" boundary of libntt_b200.so (declared in
// include/ntt_b200.h).  Host-side validation, plan ownership and dispatch to
// the engines; no arithmetic lives here beyond the small elementwise kernels.
#include <cuda_runtime.h>

#include <algorithm>

#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/ntt_b200.h"
#include "engines.hpp"
#include "plan.hpp"
#include "profiler.hpp"

namespace nttb {

static thread_local std::string g_last_error;

int fail(int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_last_error = buf;
    return code;
}

int cuda_status(const char* what) {
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail(NTTB_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
    return NTTB_OK;
}

static thread_local cudaError_t g_launch_error = cudaSuccess;

int launch_rc() {
    const cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) return 0;
    g_launch_error = e;
    return 2;
}

int launch_rc(cudaError_t e) {
    const cudaError_t last = cudaGetLastError();  // clears the sticky copy
    if (e == cudaSuccess) e = last;
    if (e == cudaSuccess) return 0;
    g_launch_error = e;
    return 2;
}

int engine_status(int rc, const char* what) {
    if (rc == 0) return cuda_status(what);
    if (rc == 1) return fail(NTTB_ERR_UNSUPPORTED, "%s: shape not served by the requested engine", what);
    cudaError_t e = g_launch_error;
    g_launch_error = cudaSuccess;
    if (e == cudaSuccess) e = cudaGetLastError();
    return fail(NTTB_ERR_CUDA, "%s: launch failed: %s", what,
                e == cudaSuccess ? "no CUDA error recorded (engine set-up failed)" : cudaGetErrorString(e));
}

uint64_t reference_generator(uint64_t q);

// ---- small elementwise kernels ---------------------------------------------
__global__ void transpose_u64_kernel(uint64_t* __restrict__ dst, const uint64_t* __restrict__ src, uint64_t rows,
                                     uint64_t cols) {
    __shared__ uint64_t tile[32][33];
    const uint64_t c0 = (uint64_t)blockIdx.x * 32, r0 = (uint64_t)blockIdx.y * 32;
    for (int i = threadIdx.y; i < 32; i += 8) {
        uint64_t r = r0 + i, c = c0 + threadIdx.x;
        if (r < rows && c < cols) tile[i][threadIdx.x] = src[r * cols + c];
    }
    __syncthreads();
    for (int i = threadIdx.y; i < 32; i += 8) {
        uint64_t c = c0 + i, r = r0 + threadIdx.x;
        if (r < rows && c < cols) dst[c * rows + r] = tile[threadIdx.x][i];
    }
}

// In-place transpose of a square matrix: each (r, c) with r < c swaps once.
__global__ void transpose_square_inplace_kernel(uint64_t* data, uint64_t n) {
    const uint64_t total = n * n;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total;
         i += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t r = i / n, c = i % n;
        if (r < c) {
            uint64_t t = data[r * n + c];
            data[r * n + c] = data[c * n + r];
            data[c * n + r] = t;
        }
    }
}

__global__ void bitrev_u64_kernel(uint64_t* data, uint64_t n, int log_n) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        uint64_t r = log_n ? (__brevll(i) >> (64 - log_n)) : 0;
        if (i < r) {
            uint64_t t = data[i];
            data[i] = data[r];
            data[r] = t;
        }
    }
}

// In-place bit reversal by tiles, log_n >= 10.  With the index split as
// (a, b, c) -- a the high 5 bits, c the low 5, b the log_n - 10 middle bits --
// element (a, b, c) moves to (rev5(c), rev(b), rev5(a)).  One block takes the
// 32 x 32 tiles of middle values b and rev(b) (b <= rev(b)), reads both with
// 256-byte rows (c contiguous), and writes each to the other's place, again
// with rows of consecutive positions.
__global__ void bitrev_tiled_u64_kernel(uint64_t* data, int log_n) {
    __shared__ uint64_t ta[32][33], tb[32][33];
    const int M = log_n - 10;
    const uint64_t n_mid = 1ull << M;
    const uint32_t x = threadIdx.x, y = threadIdx.y;  // 32 x 8 threads
    const uint32_t rx = __brev(x) >> 27;
    for (uint64_t b = blockIdx.x; b < n_mid; b += gridDim.x) {
        const uint64_t br = M ? (__brevll(b) >> (64 - M)) : 0;
        if (br < b) continue;
        for (uint32_t a = y; a < 32; a += 8) {
            ta[a][x] = data[((uint64_t)a << (M + 5)) | (b << 5) | x];
            tb[a][x] = data[((uint64_t)a << (M + 5)) | (br << 5) | x];
        }
        __syncthreads();
        for (uint32_t a2 = y; a2 < 32; a2 += 8) {  // destination high bits a2 = rev5(c), low bits x = rev5(a)
            const uint32_t c = __brev(a2) >> 27;
            data[((uint64_t)a2 << (M + 5)) | (br << 5) | x] = ta[rx][c];
            data[((uint64_t)a2 << (M + 5)) | (b << 5) | x] = tb[rx][c];
        }
        __syncthreads();
    }
}

// out = a * b mod q with one Montgomery product and one correction by R^2.
__global__ void pointwise_u64_kernel(uint64_t* out, const uint64_t* a, const uint64_t* b, uint64_t n, M64 ar,
                                     uint64_t r2) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        out[i] = ar.mul(ar.mul(a[i], b[i]), r2);
}

// Rows of 2^log_n residues, row r reduced mod limb r % n_limbs.  With
// log_n >= 2 and 16-byte aligned arrays, a thread takes four residues of one
// row per step (16-byte accesses, one limb lookup per four residues).
__global__ void pointwise_rns_kernel(uint32_t* out, const uint32_t* a, const uint32_t* b, uint32_t log_n,
                                     uint32_t n_limbs, uint64_t total, const LimbDev<M32>* limbs,
                                     const uint32_t* r2s, bool vec4) {
    const uint64_t step = (uint64_t)gridDim.x * blockDim.x;
    if (vec4) {
        const uint64_t quads = total >> 2;
        for (uint64_t qi = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; qi < quads; qi += step) {
            const uint32_t limb = (uint32_t)(((qi << 2) >> log_n) % n_limbs);
            const M32 ar = limbs[limb].ar;
            const uint32_t r2 = r2s[limb];
            const uint4 x = __ldcs(reinterpret_cast<const uint4*>(a) + qi);
            const uint4 y = __ldcs(reinterpret_cast<const uint4*>(b) + qi);
            uint4 z;
            z.x = ar.mul(ar.mul(x.x, y.x), r2);
            z.y = ar.mul(ar.mul(x.y, y.y), r2);
            z.z = ar.mul(ar.mul(x.z, y.z), r2);
            z.w = ar.mul(ar.mul(x.w, y.w), r2);
            __stcs(reinterpret_cast<uint4*>(out) + qi, z);
        }
        return;
    }
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += step) {
        const uint32_t limb = (uint32_t)((i >> log_n) % n_limbs);
        const M32 ar = limbs[limb].ar;
        out[i] = ar.mul(ar.mul(a[i], b[i]), r2s[limb]);
    }
}

static unsigned grid_for(uint64_t n) {
    uint64_t g = (n + 255) / 256;
    return (unsigned)(g > 148 * 32 ? 148 * 32 : (g ? g : 1));
}

}  // namespace nttb

using namespace nttb;

// ---- opaque handle types ------------------------------------------------------
struct nttb_plan {
    uint64_t n = 0, log_n = 0, q = 0, mu = 0;
    nttb_modular_params params{};
    uint64_t* d_twiddles = nullptr;
    uint64_t* d_twiddles_inv = nullptr;
    uint64_t* d_scratch = nullptr;  // n words: four-step / rowmaj staging
    bool wide = false;              // q >= 2^31
    Plan32 p32;
    Plan64 p64;
    M64 ar64{};
    uint64_t r2_64 = 0;
};

namespace nttb {
// Streaming of host-resident batches through one RNS plan
// (nttb_rns_stream_host): three device buffers in rotation, each batch's
// copies split in two chunks on two copy streams per direction, so that the
// host -> device copy of one batch, the transform of the previous one and the
// device -> host copy of the one before overlap.  Events order every reuse.
constexpr int kHsBufs = 3, kHsChunks = 2;  // device buffers in rotation; copy chunks (and streams) per direction
struct HostStream {
    size_t words = 0;  // capacity of each buffer
    uint32_t* dbuf[kHsBufs] = {};
    cudaStream_t in[kHsChunks] = {}, out[kHsChunks] = {};
    cudaEvent_t start = nullptr, ev_in[kHsBufs][kHsChunks] = {}, ev_c[kHsBufs] = {}, done[kHsBufs][kHsChunks] = {};
    bool used[kHsBufs] = {};
    uint32_t next = 0;  // buffer of the next batch: the rotation continues across calls
};
void host_stream_free(HostStream* h) {
    if (!h) return;
    for (int c = 0; c < kHsChunks; c++) {
        if (h->in[c]) cudaStreamSynchronize(h->in[c]);
        if (h->out[c]) cudaStreamSynchronize(h->out[c]);
    }
    for (int k = 0; k < kHsBufs; k++) {
        if (h->dbuf[k]) cudaFree(h->dbuf[k]);
        if (h->ev_c[k]) cudaEventDestroy(h->ev_c[k]);
        for (int c = 0; c < kHsChunks; c++) {
            if (h->ev_in[k][c]) cudaEventDestroy(h->ev_in[k][c]);
            if (h->done[k][c]) cudaEventDestroy(h->done[k][c]);
        }
    }
    for (int c = 0; c < kHsChunks; c++) {
        if (h->in[c]) cudaStreamDestroy(h->in[c]);
        if (h->out[c]) cudaStreamDestroy(h->out[c]);
    }
    if (h->start) cudaEventDestroy(h->start);
    delete h;
}
}  // namespace nttb

struct nttb_rns_plan {
    Plan32 p;
    uint32_t* d_r2 = nullptr;  // R^2 mod q per limb (pointwise products)
    nttb::HostStream* hs = nullptr;
};

struct nttb_wide_plan {
    Plan64 p;
};

namespace nttb {
const Plan32* rns_plan_core(const nttb_rns_plan* p) { return p ? &p->p : nullptr; }
}  // namespace nttb

extern "C" {

const char* nttb_version(void) { return "ntt_b200 0.1 (sm_100a)"; }

const char* nttb_status_string(int s) {
    switch (s) {
        case NTTB_OK: return "ok";
        case NTTB_ERR_INVALID_ARG: return "invalid argument";
        case NTTB_ERR_UNSUPPORTED: return "unsupported";
        case NTTB_ERR_CUDA: return "CUDA error";
        case NTTB_ERR_NO_MEMORY: return "out of memory";
        case NTTB_ERR_TIMEOUT: return "device wait timed out";
        case NTTB_ERR_BUDGET: return "HBM budget exceeded";
        default: return "unknown status";
    }
}

const char* nttb_last_error(void) { return g_last_error.c_str(); }

int nttb_device_errors(uint32_t* flags, int clear) {
    if (!flags) return fail(NTTB_ERR_INVALID_ARG, "device_errors: null argument");
    *flags = int8_device_errors(clear != 0) | (batch_device_errors(clear != 0) << 2) |
             (tma_move_device_errors(clear != 0) << 4) | (wide_device_errors(clear != 0) << 5);
    return cuda_status("device_errors");
}

int nttb_bounds_errors(uint32_t* flags, int* enabled, int clear) {
    if (!flags || !enabled) return fail(NTTB_ERR_INVALID_ARG, "bounds_errors: null argument");
#ifdef NTT_DEBUG_BOUNDS
    *enabled = 1;
#else
    *enabled = 0;
#endif
    *flags = int8_bounds_errors(clear != 0) | (dmma_bounds_errors(clear != 0) << 8) |
             (batch_bounds_errors(clear != 0) << 16) | (wide_bounds_errors(clear != 0) << 24);
    return cuda_status("bounds_errors");
}

int nttb_phase_profile(uint64_t* out16, int* enabled, int clear) {
    if (!out16 || !enabled) return fail(NTTB_ERR_INVALID_ARG, "phase_profile: null argument");
#ifdef NTT_PHASE_PROFILE
    *enabled = 1;
#else
    *enabled = 0;
#endif
    int8_phase_profile(out16, clear != 0);
    return cuda_status("phase_profile");
}

// A wide (64-bit modulus) transform: AUTO takes the INT8 engine where it
// serves the plan (n = 2^20, cyclic) for fewer than 8 (polynomial, limb)
// units, the CUDA-core Montgomery-64 engine otherwise.  Both spend about the
// same number of integer multiplies per residue (the 64-bit REDCs and twiddle
// products of the byte-plane epilogues match the radix-2 butterflies'); the
// INT8 engine's two passes have the shorter latency (one 2^20 polynomial:
// 82 against 95 us forward + inverse), the CUDA-core engine the higher
// throughput from 16 units on (1.01 against 1.07 ms for 16).
constexpr uint64_t kWideTcMaxUnits = 8;
static int wide_transform(Plan64& p, const void* src, void* dst, uint32_t n_polys, bool inverse, int engine,
                          cudaStream_t s) {
    if (engine == NTTB_ENGINE_AUTO)
        engine = wide_tc_serves(p) && (uint64_t)n_polys * p.n_limbs < kWideTcMaxUnits ? NTTB_ENGINE_INT8
                                                                                       : NTTB_ENGINE_SCALAR;
    if (engine == NTTB_ENGINE_INT8) return wide_tc_transform64(p, src, dst, n_polys, inverse, s);
    if (engine == NTTB_ENGINE_TILES) return 1;  // the batch queue's tiles take moduli < 2^31
    return scalar_transform64(p, src, dst, n_polys, inverse, s);  // the 31-bit engines do not serve 64-bit moduli
}

static bool pow2(uint64_t n) { return n && !(n & (n - 1)); }
// Status of a TMA tile-mover launch (0 launched, 2 CUDA error).
static int tma_status(int t, const char* what) {
    if (t == 0) return NTTB_OK;
    const int rc = cuda_status(what);
    return rc ? rc : fail(NTTB_ERR_CUDA, "%s: TMA tile launch failed", what);
}
static uint32_t ilog2(uint64_t n) { uint32_t l = 0; while ((1ull << l) < n) l++; return l; }

int nttb_create_params(uint64_t q, uint64_t n, nttb_modular_params* out) {
    if (!out || q < 3 || !pow2(n)) return fail(NTTB_ERR_INVALID_ARG, "create_params: bad q or n");
    // barrett_k / barrett_m exactly as include/modular_arith.cuh:158-162 stores them
    int k = 64;
    while ((1ULL << (k - 64)) < q && k < 96) k++;
    out->q = q;
    out->q_twice = 2 * q;
    out->barrett_k = (uint64_t)k;
    out->barrett_m = (uint64_t)(((unsigned __int128)1 << k) / q);
    uint64_t g = reference_generator(q);
    out->omega = h_powmod(g, (q - 1) / n, q);
    out->omega_inv = h_invmod(out->omega, q);
    out->n_inv = h_invmod(n % q, q);
    return NTTB_OK;
}

int nttb_find_primitive_root(uint64_t q, uint64_t n, uint64_t* omega) {
    if (!omega || q < 3 || !pow2(n)) return fail(NTTB_ERR_INVALID_ARG, "find_primitive_root: bad q or n");
    *omega = h_powmod(reference_generator(q), (q - 1) / n, q);
    return NTTB_OK;
}

int nttb_find_psi(uint64_t q, uint64_t n, uint64_t* psi) {
    if (!psi || q < 3 || !pow2(n) || (q - 1) % (2 * n)) return fail(NTTB_ERR_INVALID_ARG, "find_psi: 2n must divide q-1");
    *psi = h_powmod(reference_generator(q), (q - 1) / (2 * n), q);
    return NTTB_OK;
}

// CPU NTT (natural order): iterative decimation-in-frequency into a
// bit-reversed temporary, then an unscrambling copy; n^-1 applied for the
// inverse.  Exact with unsigned __int128 for q < 2^63.
int nttb_host_ntt(uint64_t* data, uint64_t n, const nttb_modular_params* p, int inverse) {
    if (!data || !p || !pow2(n) || p->q >= (1ull << 63)) return fail(NTTB_ERR_INVALID_ARG, "host_ntt: bad arguments");
    const uint64_t q = p->q;
    const uint64_t root = inverse ? p->omega_inv : p->omega;
    const int lg = (int)ilog2(n);
    std::vector<uint64_t> w(n / 2 + 1);
    w[0] = 1;
    for (uint64_t i = 1; i < n / 2; i++) w[i] = h_mulmod(w[i - 1], root, q);
    for (uint64_t half = n / 2; half >= 1; half >>= 1) {
        const uint64_t step = n / (2 * half);
        for (uint64_t g = 0; g < n; g += 2 * half)
            for (uint64_t j = 0; j < half; j++) {
                uint64_t u = data[g + j], v = data[g + j + half];
                uint64_t s = u + v;
                if (s >= q || s < u) s -= q;
                uint64_t d = u >= v ? u - v : u + (q - v);
                data[g + j] = s;
                data[g + j + half] = h_mulmod(d, w[j * step], q);
            }
        if (half == 1) break;
    }
    for (uint64_t i = 0; i < n; i++) {
        uint64_t r = 0;
        for (int b = 0; b < lg; b++) r |= ((i >> b) & 1ull) << (lg - 1 - b);
        if (i < r) std::swap(data[i], data[r]);
    }
    if (inverse)
        for (uint64_t i = 0; i < n; i++) data[i] = h_mulmod(data[i], p->n_inv, q);
    return NTTB_OK;
}

static bool is_prime_u64(uint64_t q) {
    LimbHost L;
    std::string why;
    return q > 2 && (q & 1) && make_limb_host(q, 1, false, &L, &why);
}

int nttb_generate_primes(uint32_t bits, uint32_t two_adicity, uint32_t count, uint64_t* out) {
    if (!out || bits < 3 || bits > 62 || two_adicity >= bits) return fail(NTTB_ERR_INVALID_ARG, "generate_primes: bad args");
    const uint64_t step = 1ull << two_adicity;
    uint64_t k = ((1ull << bits) - 1) / step;
    uint32_t found = 0;
    for (; k > 0 && found < count; k--) {
        uint64_t q = k * step + 1;
        if (q >= (1ull << bits)) continue;
        if (is_prime_u64(q)) out[found++] = q;
    }
    if (found < count) return fail(NTTB_ERR_INVALID_ARG, "generate_primes: only %u primes exist", found);
    return NTTB_OK;
}

// ---------------------------------------------------------- single-modulus plan
int nttb_plan_create(uint64_t n, uint64_t q, nttb_plan** out) {
    if (!out) return fail(NTTB_ERR_INVALID_ARG, "plan_create: null out");
    *out = nullptr;
    if (!pow2(n) || n < 2 || n > (1ull << 26)) return fail(NTTB_ERR_INVALID_ARG, "plan_create: n must be a power of two in [2, 2^26]");
    if (q >= (1ull << 62)) return fail(NTTB_ERR_UNSUPPORTED, "plan_create: q must be < 2^62");
    auto* P = new nttb_plan();
    P->n = n;
    P->log_n = ilog2(n);
    P->q = q;
    P->mu = (uint64_t)(((unsigned __int128)1 << 64) / q);
    std::string why;
    int rc;
    uint64_t qs[1] = {q};
    if (q < (1ull << 31)) {
        rc = build_plan32(&P->p32, (uint32_t)P->log_n, qs, 1, false, &why);
    } else {
        P->wide = true;
        rc = build_plan64(&P->p64, (uint32_t)P->log_n, qs, 1, false, &why);
    }
    if (rc) {
        free_plan32(&P->p32);
        free_plan64(&P->p64);
        delete P;
        return fail(rc == 4 ? NTTB_ERR_NO_MEMORY : NTTB_ERR_INVALID_ARG, "plan_create: %s", why.c_str());
    }
    nttb_create_params(q, n, &P->params);
    // the reference's twiddle tables: omega^k and omega^-k as uint64 words
    std::vector<uint64_t> tw(n), twi(n);
    tw[0] = twi[0] = 1;
    for (uint64_t i = 1; i < n; i++) {
        tw[i] = h_mulmod(tw[i - 1], P->params.omega, q);
        twi[i] = h_mulmod(twi[i - 1], P->params.omega_inv, q);
    }
    if (cudaMalloc(&P->d_twiddles, n * 8) != cudaSuccess || cudaMalloc(&P->d_twiddles_inv, n * 8) != cudaSuccess ||
        cudaMalloc(&P->d_scratch, n * 8) != cudaSuccess) {
        nttb_plan_destroy(P);
        return fail(NTTB_ERR_NO_MEMORY, "plan_create: cudaMalloc failed");
    }
    if (cudaMemcpy(P->d_twiddles, tw.data(), n * 8, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(P->d_twiddles_inv, twi.data(), n * 8, cudaMemcpyHostToDevice) != cudaSuccess) {
        nttb_plan_destroy(P);
        return fail(NTTB_ERR_CUDA, "plan_create: twiddle upload: %s", cudaGetErrorString(cudaGetLastError()));
    }
    P->ar64.q = q;
    P->ar64.qinv = h_neg_inv64(q);
    P->r2_64 = h_to_mont64(h_to_mont64(1, q), q);
    *out = P;
    return cuda_status("plan_create");
}

int nttb_plan_destroy(nttb_plan* P) {
    if (!P) return NTTB_OK;
    engines_release32(&P->p32);
    wide_tc_release(&P->p64);
    free_plan32(&P->p32);
    free_plan64(&P->p64);
    if (P->d_twiddles) cudaFree(P->d_twiddles);
    if (P->d_twiddles_inv) cudaFree(P->d_twiddles_inv);
    if (P->d_scratch) cudaFree(P->d_scratch);
    delete P;
    return NTTB_OK;
}

int nttb_plan_get_info(const nttb_plan* P, nttb_plan_info* out) {
    if (!P || !out) return fail(NTTB_ERR_INVALID_ARG, "plan_get_info: null argument");
    out->n = P->n;
    out->log_n = P->log_n;
    out->q = P->q;
    out->mu = P->mu;
    out->d_twiddles = P->d_twiddles;
    out->d_twiddles_inv = P->d_twiddles_inv;
    out->params = P->params;
    return NTTB_OK;
}

int nttb_u64_transform(const nttb_plan* P, uint64_t* d, uint64_t batch, int inverse, int engine, void* stream) {
    if (!P || !d) return fail(NTTB_ERR_INVALID_ARG, "u64_transform: null argument");
    if (batch == 0) return NTTB_OK;
    if (batch > 65535) return fail(NTTB_ERR_UNSUPPORTED, "u64_transform: batch > 65535");
    if (((uintptr_t)d) & 7) return fail(NTTB_ERR_INVALID_ARG, "u64_transform: misaligned pointer");
    cudaStream_t s = (cudaStream_t)stream;
    int rc;
    if (P->wide) {
        rc = wide_transform(const_cast<Plan64&>(P->p64), d, d, (uint32_t)batch, inverse != 0, engine, s);
    } else {
        rc = run_transform32(const_cast<Plan32&>(P->p32), d, d, true, (uint32_t)batch, inverse != 0, engine, s);
    }
    return engine_status(rc, "u64_transform");
}

int nttb_u64_four_step(const nttb_plan* P, uint64_t* d, int inverse, void* stream) {
    if (!P || !d) return fail(NTTB_ERR_INVALID_ARG, "four_step: null argument");
    if (P->wide) return fail(NTTB_ERR_UNSUPPORTED, "four_step: q must be < 2^31");
    int rc = scalar_four_step32(P->p32, d, P->d_scratch, inverse != 0, (cudaStream_t)stream);
    return engine_status(rc, "four_step");
}

int nttb_u64_transpose(uint64_t* dst, const uint64_t* src, uint64_t rows, uint64_t cols, void* stream) {
    if (!dst || !src || rows == 0 || cols == 0) return fail(NTTB_ERR_INVALID_ARG, "transpose: bad arguments");
    if (dst == src) {
        // The reference's helpers are called in place on square matrices
        // (tests/debug_rowmaj.cu:122-124); serve that race-free.
        if (rows != cols) return fail(NTTB_ERR_INVALID_ARG, "transpose: in place only for square matrices");
        const int t = tma_transpose_square_inplace_u64(dst, rows, (cudaStream_t)stream);
        if (t != 1) return tma_status(t, "transpose");
        ProfScope prof("transpose_square_inplace", (cudaStream_t)stream);
        transpose_square_inplace_kernel<<<grid_for(rows * cols), 256, 0, (cudaStream_t)stream>>>(dst, rows);
        return cuda_status("transpose");
    }
    const int t = tma_transpose_u64(dst, src, rows, cols, (cudaStream_t)stream);
    if (t != 1) return tma_status(t, "transpose");
    // shapes that are not whole 32 x 32 tiles, or unaligned arrays
    dim3 grid((unsigned)((cols + 31) / 32), (unsigned)((rows + 31) / 32));
    if (grid.y > 65535) return fail(NTTB_ERR_UNSUPPORTED, "transpose: too many rows");
    ProfScope prof("transpose_u64", (cudaStream_t)stream);
    transpose_u64_kernel<<<grid, dim3(32, 8), 0, (cudaStream_t)stream>>>(dst, src, rows, cols);
    return cuda_status("transpose");
}

int nttb_u64_rowmaj_forward(const nttb_plan* P, uint64_t* d, void* stream) {
    if (!P || !d) return fail(NTTB_ERR_INVALID_ARG, "rowmaj_forward: null argument");
    if (P->n != 4096) return nttb_u64_transform(P, d, 1, 0, NTTB_ENGINE_AUTO, stream);
    return nttb_u64_pretransposed_transform(P, d, 64, 0, stream);
}

int nttb_u64_pretransposed_transform(const nttb_plan* P, uint64_t* d, uint64_t n1, int inverse, void* stream) {
    if (!P || !d) return fail(NTTB_ERR_INVALID_ARG, "pretransposed_transform: null argument");
    if (!pow2(n1) || n1 > P->n) return fail(NTTB_ERR_INVALID_ARG, "pretransposed_transform: n1 must be a power of two <= n");
    const uint64_t n2 = P->n / n1;
    if (!P->wide && n1 == n2) {
        // square: two passes that read and write the layout directly
        const int r = scalar_pretransposed32(P->p32, d, P->d_scratch, inverse != 0, (cudaStream_t)stream);
        if (r == 0) return cuda_status("pretransposed_transform");
        if (r != 1) {
            const int st = cuda_status("pretransposed_transform");
            return st ? st : fail(NTTB_ERR_CUDA, "pretransposed_transform: launch failed");
        }
    }
    // pre[b * n1 + a] = canon[a * n2 + b]: canon is pre (n2 x n1) transposed
    int rc = nttb_u64_transpose(P->d_scratch, d, n2, n1, stream);
    if (rc) return rc;
    rc = nttb_u64_transform(P, P->d_scratch, 1, inverse, NTTB_ENGINE_AUTO, stream);
    if (rc) return rc;
    return nttb_u64_transpose(d, P->d_scratch, n1, n2, stream);
}

int nttb_u64_pointwise_mul(const nttb_plan* P, uint64_t* out, const uint64_t* a, const uint64_t* b, void* stream) {
    if (!P || !out || !a || !b) return fail(NTTB_ERR_INVALID_ARG, "pointwise_mul: null argument");
    ProfScope prof("pointwise_u64", (cudaStream_t)stream);
    pointwise_u64_kernel<<<grid_for(P->n), 256, 0, (cudaStream_t)stream>>>(out, a, b, P->n, P->ar64, P->r2_64);
    return cuda_status("pointwise_mul");
}

int nttb_u64_bit_reverse(uint64_t* d, uint64_t n, void* stream) {
    if (!d || !pow2(n)) return fail(NTTB_ERR_INVALID_ARG, "bit_reverse: n must be a power of two");
    const int log_n = (int)ilog2(n);
    if (log_n >= 10) {
        const int t = tma_bit_reverse_u64(d, log_n, (cudaStream_t)stream);
        if (t != 1) return tma_status(t, "bit_reverse");
    }
    ProfScope prof("bitrev_u64", (cudaStream_t)stream);
    if (log_n >= 10) {
        const uint64_t mids = n >> 10;
        bitrev_tiled_u64_kernel<<<(unsigned)(mids < 148 * 16 ? mids : 148 * 16), dim3(32, 8), 0, (cudaStream_t)stream>>>(
            d, log_n);
    } else {
        bitrev_u64_kernel<<<grid_for(n), 256, 0, (cudaStream_t)stream>>>(d, n, log_n);
    }
    return cuda_status("bit_reverse");
}

// ------------------------------------------------------------------ RNS plans
int nttb_rns_plan_create(uint32_t log_n, const uint64_t* moduli, uint32_t n_limbs, uint32_t flags,
                         nttb_rns_plan** out) {
    if (!out || !moduli || n_limbs == 0) return fail(NTTB_ERR_INVALID_ARG, "rns_plan_create: bad arguments");
    *out = nullptr;
    if (log_n < 1 || log_n > 24) return fail(NTTB_ERR_UNSUPPORTED, "rns_plan_create: log_n must be in [1, 24]");
    auto* P = new nttb_rns_plan();
    std::string why;
    int rc = build_plan32(&P->p, log_n, moduli, n_limbs, (flags & NTTB_NEGACYCLIC) != 0, &why);
    if (rc) {
        free_plan32(&P->p);
        delete P;
        return fail(rc == 4 ? NTTB_ERR_NO_MEMORY : NTTB_ERR_INVALID_ARG, "rns_plan_create: %s", why.c_str());
    }
    std::vector<uint32_t> r2(n_limbs);
    for (uint32_t l = 0; l < n_limbs; l++) r2[l] = h_to_mont32(h_to_mont32(1, moduli[l]), moduli[l]);
    if (cudaMalloc(&P->d_r2, n_limbs * 4) != cudaSuccess) {
        nttb_rns_plan_destroy(P);
        return fail(NTTB_ERR_NO_MEMORY, "rns_plan_create: cudaMalloc failed");
    }
    if (cudaMemcpy(P->d_r2, r2.data(), n_limbs * 4, cudaMemcpyHostToDevice) != cudaSuccess) {
        nttb_rns_plan_destroy(P);
        return fail(NTTB_ERR_CUDA, "rns_plan_create: table upload: %s", cudaGetErrorString(cudaGetLastError()));
    }
    *out = P;
    return cuda_status("rns_plan_create");
}

int nttb_rns_plan_destroy(nttb_rns_plan* P) {
    if (!P) return NTTB_OK;
    nttb::host_stream_free(P->hs);
    engines_release32(&P->p);
    free_plan32(&P->p);
    if (P->d_r2) cudaFree(P->d_r2);
    delete P;
    return NTTB_OK;
}

int nttb_rns_transform(const nttb_rns_plan* P, uint32_t* dst, const uint32_t* src, uint32_t n_polys, int inverse,
                       int engine, void* stream) {
    if (!P || !dst || !src) return fail(NTTB_ERR_INVALID_ARG, "rns_transform: null argument");
    if (n_polys == 0) return NTTB_OK;
    if ((((uintptr_t)dst) | ((uintptr_t)src)) & 15) return fail(NTTB_ERR_INVALID_ARG, "rns_transform: pointers must be 16-byte aligned");
    int rc = run_transform32(const_cast<Plan32&>(P->p), src, dst, false, n_polys, inverse != 0, engine,
                             (cudaStream_t)stream);
    return engine_status(rc, "rns_transform");
}

int nttb_rns_forward_inverse(const nttb_rns_plan* P, uint32_t* d, uint32_t n_polys, int engine, void* stream) {
    if (!P || !d) return fail(NTTB_ERR_INVALID_ARG, "rns_forward_inverse: null argument");
    if (n_polys == 0) return NTTB_OK;
    if (((uintptr_t)d) & 15) return fail(NTTB_ERR_INVALID_ARG, "rns_forward_inverse: pointer must be 16-byte aligned");
    Plan32& p = const_cast<Plan32&>(P->p);
    cudaStream_t s = (cudaStream_t)stream;
    int eng = engine == NTTB_ENGINE_AUTO ? auto_engine32(p, false, (uint64_t)n_polys * p.n_limbs) : engine;
    int rc;
    if (eng == NTTB_ENGINE_INT8) {
        rc = int8_forward_inverse32(p, d, n_polys, s);
    } else {
        rc = run_transform32(p, d, d, false, n_polys, false, eng, s);
        if (!rc) rc = run_transform32(p, d, d, false, n_polys, true, eng, s);
    }
    return engine_status(rc, "rns_forward_inverse");
}

int nttb_rns_stream_host(nttb_rns_plan* P, const uint32_t* h_src, uint32_t* h_dst, uint32_t n_polys, uint32_t n_batches,
                         int mode, int engine, void* stream) {
    if (!P || !h_src || !h_dst) return fail(NTTB_ERR_INVALID_ARG, "rns_stream_host: null argument");
    if (mode < 0 || mode > 2) return fail(NTTB_ERR_INVALID_ARG, "rns_stream_host: mode must be 0, 1 or 2");
    if (n_polys == 0 || n_batches == 0) return NTTB_OK;
    Plan32& p = P->p;
    cudaStream_t s = (cudaStream_t)stream;
    const size_t bw = (size_t)n_polys * p.n_limbs * p.n;
    const int eng = engine == NTTB_ENGINE_AUTO ? auto_engine32(p, false, (uint64_t)n_polys * p.n_limbs) : engine;
    nttb::HostStream*& H = P->hs;
    if (!H || H->words < bw) {  // (re)build the buffers, streams and events
        nttb::host_stream_free(H);
        H = new nttb::HostStream();
        bool ok = true;
        for (int k = 0; k < nttb::kHsBufs && ok; k++) {
            ok = cudaMalloc(&H->dbuf[k], bw * 4) == cudaSuccess;
            ok = ok && cudaEventCreateWithFlags(&H->ev_c[k], cudaEventDisableTiming) == cudaSuccess;
            for (int c = 0; c < nttb::kHsChunks && ok; c++) {
                ok = cudaEventCreateWithFlags(&H->ev_in[k][c], cudaEventDisableTiming) == cudaSuccess;
                ok = ok && cudaEventCreateWithFlags(&H->done[k][c], cudaEventDisableTiming) == cudaSuccess;
            }
        }
        for (int c = 0; c < nttb::kHsChunks && ok; c++) {
            ok = cudaStreamCreateWithFlags(&H->in[c], cudaStreamNonBlocking) == cudaSuccess;
            ok = ok && cudaStreamCreateWithFlags(&H->out[c], cudaStreamNonBlocking) == cudaSuccess;
        }
        ok = ok && cudaEventCreateWithFlags(&H->start, cudaEventDisableTiming) == cudaSuccess;
        if (!ok) {
            nttb::host_stream_free(H);
            H = nullptr;
            return fail(NTTB_ERR_NO_MEMORY, "rns_stream_host: buffers");
        }
        H->words = bw;
    }
    // everything after the caller's earlier work on `stream`
    cudaEventRecord(H->start, s);
    for (int c = 0; c < nttb::kHsChunks; c++) {
        cudaStreamWaitEvent(H->in[c], H->start, 0);
        cudaStreamWaitEvent(H->out[c], H->start, 0);
    }
    // chunk c of a batch: words [c chunk, min(bw, (c + 1) chunk)), 256-byte aligned
    const size_t chunk = (bw / nttb::kHsChunks + 63) & ~(size_t)63;
    auto span = [&](int c, size_t* off) {
        *off = (size_t)c * chunk;
        return *off < bw ? std::min(chunk, bw - *off) : (size_t)0;
    };
    for (uint32_t i = 0; i < n_batches; i++) {
        const int k = (int)(H->next++ % nttb::kHsBufs);
        for (int c = 0; c < nttb::kHsChunks; c++) {
            size_t off;
            const size_t len = span(c, &off);
            if (H->used[k]) cudaStreamWaitEvent(H->in[c], H->done[k][c], 0);
            if (len) cudaMemcpyAsync(H->dbuf[k] + off, h_src + i * bw + off, len * 4, cudaMemcpyHostToDevice, H->in[c]);
            cudaEventRecord(H->ev_in[k][c], H->in[c]);
            cudaStreamWaitEvent(s, H->ev_in[k][c], 0);
        }
        int rc = 0;
        if (mode == 2) {
            rc = eng == NTTB_ENGINE_INT8 ? int8_forward_inverse32(p, H->dbuf[k], n_polys, s)
                                         : run_transform32(p, H->dbuf[k], H->dbuf[k], false, n_polys, false, eng, s);
            if (!rc && eng != NTTB_ENGINE_INT8)
                rc = run_transform32(p, H->dbuf[k], H->dbuf[k], false, n_polys, true, eng, s);
        } else {
            rc = run_transform32(p, H->dbuf[k], H->dbuf[k], false, n_polys, mode == 1, eng, s);
        }
        if (rc) return engine_status(rc, "rns_stream_host");
        cudaEventRecord(H->ev_c[k], s);
        for (int c = 0; c < nttb::kHsChunks; c++) {
            size_t off;
            const size_t len = span(c, &off);
            cudaStreamWaitEvent(H->out[c], H->ev_c[k], 0);
            if (len) cudaMemcpyAsync(h_dst + i * bw + off, H->dbuf[k] + off, len * 4, cudaMemcpyDeviceToHost, H->out[c]);
            cudaEventRecord(H->done[k][c], H->out[c]);
        }
        H->used[k] = true;
    }
    // the caller's stream completes after the last copy back
    for (int k = 0; k < nttb::kHsBufs; k++)
        if (H->used[k])
            for (int c = 0; c < nttb::kHsChunks; c++) cudaStreamWaitEvent(s, H->done[k][c], 0);
    return cuda_status("rns_stream_host");
}

int nttb_rns_pointwise_mul(const nttb_rns_plan* P, uint32_t* out, const uint32_t* a, const uint32_t* b,
                           uint32_t n_polys, void* stream) {
    if (!P || !out || !a || !b) return fail(NTTB_ERR_INVALID_ARG, "rns_pointwise_mul: null argument");
    uint64_t total = (uint64_t)n_polys * P->p.n_limbs * P->p.n;
    ProfScope prof("pointwise_rns", (cudaStream_t)stream);
    const bool vec4 = P->p.log_n >= 2 && ((((uintptr_t)out) | ((uintptr_t)a) | ((uintptr_t)b)) & 15) == 0;
    pointwise_rns_kernel<<<grid_for(vec4 ? total / 4 : total), 256, 0, (cudaStream_t)stream>>>(
        out, a, b, P->p.log_n, P->p.n_limbs, total, P->p.d_limbs, P->d_r2, vec4);
    return cuda_status("rns_pointwise_mul");
}

// ---------------------------------------------------------------- wide plans
int nttb_wide_plan_create(uint32_t log_n, const uint64_t* moduli, uint32_t n_limbs, uint32_t flags,
                          nttb_wide_plan** out) {
    if (!out || !moduli || n_limbs == 0) return fail(NTTB_ERR_INVALID_ARG, "wide_plan_create: bad arguments");
    *out = nullptr;
    if (log_n < 1 || log_n > 24) return fail(NTTB_ERR_UNSUPPORTED, "wide_plan_create: log_n must be in [1, 24]");
    auto* P = new nttb_wide_plan();
    std::string why;
    int rc = build_plan64(&P->p, log_n, moduli, n_limbs, (flags & NTTB_NEGACYCLIC) != 0, &why);
    if (rc) {
        free_plan64(&P->p);
        delete P;
        return fail(rc == 4 ? NTTB_ERR_NO_MEMORY : NTTB_ERR_INVALID_ARG, "wide_plan_create: %s", why.c_str());
    }
    *out = P;
    return cuda_status("wide_plan_create");
}

int nttb_wide_plan_destroy(nttb_wide_plan* P) {
    if (!P) return NTTB_OK;
    wide_tc_release(&P->p);
    free_plan64(&P->p);
    delete P;
    return NTTB_OK;
}

int nttb_wide_transform(const nttb_wide_plan* P, uint64_t* dst, const uint64_t* src, uint32_t n_polys, int inverse,
                        void* stream) {
    return nttb_wide_transform_engine(P, dst, src, n_polys, inverse, NTTB_ENGINE_AUTO, stream);
}

int nttb_wide_transform_engine(const nttb_wide_plan* P, uint64_t* dst, const uint64_t* src, uint32_t n_polys,
                               int inverse, int engine, void* stream) {
    if (!P || !dst || !src) return fail(NTTB_ERR_INVALID_ARG, "wide_transform: null argument");
    if (engine != NTTB_ENGINE_AUTO && engine != NTTB_ENGINE_SCALAR && engine != NTTB_ENGINE_INT8)
        return fail(NTTB_ERR_INVALID_ARG, "wide_transform: engine must be AUTO, SCALAR or INT8");
    if ((((uintptr_t)dst) | ((uintptr_t)src)) & 15) return fail(NTTB_ERR_INVALID_ARG, "wide_transform: pointers must be 16-byte aligned");
    if (n_polys == 0) return NTTB_OK;
    const int rc = wide_transform(const_cast<Plan64&>(P->p), src, dst, n_polys, inverse != 0, engine,
                                  (cudaStream_t)stream);
    return engine_status(rc, "wide_transform");
}

}  // extern "C"
