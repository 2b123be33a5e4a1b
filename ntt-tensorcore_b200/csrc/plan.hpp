// plan.hpp -- host-side plan structures shared by the engines and the C-ABI.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>
#include <string>
#include <vector>

#include "arith.cuh"

namespace nttb {

// Per-limb constants handed to the kernels (one array entry per limb).
template <class A>
struct LimbDev {
    A ar;                              // modulus + Montgomery constant
    typename A::elem ninv_m;           // n^-1 * R mod q
    typename A::elem pad_;
    const typename A::elem* tw;        // omega^e * R,   e < n
    const typename A::elem* tw_inv;    // omega^-e * R,  e < n
    const typename A::elem* psi;       // psi^e * R,     e < n (negacyclic only)
    const typename A::elem* psi_inv;   // n^-1 psi^-e R, e < n (negacyclic only)
    // Shoup pairs of the radix-2 butterflies, level by level: the roots of
    // length L = 2^l sit at pairs 2^(l-1) - 1 .. 2^l - 2 (k < L/2), each pair
    // root_L^k (plain form) and floor(root_L^k * 2^bits / q) (bits = 32 or 64),
    // so a pass of length L reads one contiguous run
    const typename A::elem* tw_sh;
    const typename A::elem* tw_inv_sh;
};

// Host view of one modulus at one transform size.
struct LimbHost {
    uint64_t q = 0, g = 0, omega = 0, omega_inv = 0, psi = 0, psi_inv = 0, n_inv = 0;
};

// Fills LimbHost with the generator rule of the reference
// (include/modular_arith.cuh:130-151) plus psi = g^((q-1)/2n).
bool make_limb_host(uint64_t q, uint64_t n, bool need_psi, LimbHost* out, std::string* why);

// Transform direction / twist flags.
enum : uint32_t {
    F_PRE_PSI = 1u,       // multiply input element n by psi^n           (negacyclic forward)
    F_PRE_TW = 2u,        // multiply input (row a, col b) by root^(a*b)  (four-step inverse)
    F_POST_TW = 4u,       // multiply output (row d, col b) by root^(d*b) (four-step pass 1)
    F_POST_SCALE = 8u,    // multiply output by n^-1                      (cyclic inverse)
    F_POST_PSI_INV = 16u, // multiply output element n by n^-1 psi^-n    (negacyclic inverse)
    F_STORE_T = 32u,      // MODE_COL: store output (row k, col b) at b*N1 + k (transposed)
};

// Pass geometries of the scalar engine.
enum PassMode : int {
    MODE_COL = 0,          // vectors = columns of [N1 x N2]; out in place (row k, col b)
    MODE_ROW_NAT = 1,      // vectors = rows d; out X[d + N1*k] (natural order), or with F_STORE_T
                           // row by row at d*len + k (F_POST_TW: times root^(k*d))
    MODE_GATHER_T = 2,     // vectors = chunks of the N1 x N2 -> N2 x N1 transpose; out in place
    MODE_ROW_SCATTER_T = 3 // vectors = contiguous chunks; out through the transpose back
};

struct PassArgs {
    const void* src;
    void* dst;
    uint64_t poly_stride;  // elements between consecutive polynomials
    uint32_t n, log_n;
    uint32_t n1, n2;       // matrix view of one transform
    uint32_t len, log_len; // DFT length of this pass
    uint32_t vec_per_tile;
    uint32_t n_limbs;
    uint32_t flags;
    int inverse;
};

// A u32-residue plan (q < 2^31 for every limb).
struct Plan32 {
    uint32_t log_n = 0, n = 0, n_limbs = 0;
    bool negacyclic = false;
    std::vector<LimbHost> limbs;
    LimbDev<M32>* d_limbs = nullptr;  // device array, n_limbs entries
    std::vector<void*> allocations;   // device memory owned by the plan
    void* engine_data[4] = {nullptr, nullptr, nullptr, nullptr};  // per-engine host-side caches
    std::mutex engine_mu;             // guards the lazy construction of engine_data
    void* ws = nullptr;               // workspace for in-place multi-pass transforms
    size_t ws_bytes = 0;
    int device = -1;                  // the CUDA device holding d_limbs and the tables
};

// A u64-residue plan (q < 2^62).
struct Plan64 {
    uint32_t log_n = 0, n = 0, n_limbs = 0;
    bool negacyclic = false;
    std::vector<LimbHost> limbs;
    LimbDev<M64>* d_limbs = nullptr;
    std::vector<void*> allocations;
    void* ws = nullptr;
    size_t ws_bytes = 0;
    void* engine_data = nullptr;  // the INT8 wide engine's constants (tc_wide.cu)
    std::mutex engine_mu;         // guards their lazy construction
};

// Status of the kernel launch just made: 0, or 2 after keeping its CUDA
// error for the C-ABI's message (cudaGetLastError clears a launch error, so
// the caller could not read it again).
int launch_rc();
// The same for a launch call that returned `e` itself (cudaLaunchKernelEx).
int launch_rc(cudaError_t e);
// C-ABI status of an engine's return code: 0 -> cudaGetLastError's status,
// 1 -> NTTB_ERR_UNSUPPORTED ("<what>: shape not served"), 2 or more ->
// NTTB_ERR_CUDA with the error kept by launch_rc (or the current one).
int engine_status(int rc, const char* what);

// Returns a device workspace of at least `bytes`, growing the plan's buffer
// (an in-place multi-pass transform stages its first pass there).  Calls
// that share a plan must be ordered on one stream while they use it.
void* plan_workspace(void** ws, size_t* ws_bytes, size_t bytes);

int build_plan32(Plan32* p, uint32_t log_n, const uint64_t* moduli, uint32_t n_limbs, bool negacyclic,
                 std::string* why);
int build_plan64(Plan64* p, uint32_t log_n, const uint64_t* moduli, uint32_t n_limbs, bool negacyclic,
                 std::string* why);
void free_plan32(Plan32* p);
void free_plan64(Plan64* p);

// Scalar engine entry points (scalar_engine.cu).  Storage is u32 or u64
// words; data layout is [poly][limb][n].
int scalar_transform32(Plan32& p, const void* src, void* dst, bool src_u64, uint32_t n_polys, bool inverse,
                       cudaStream_t s);
int scalar_transform64(Plan64& p, const void* src, void* dst, uint32_t n_polys, bool inverse, cudaStream_t s);
// In-place uint32 transform staging its first pass in a caller-supplied buffer
// `ws` (n_polys * n_limbs * n words); allocates nothing.
int scalar_transform32_ws(const Plan32& p, uint32_t* data, void* ws, uint32_t n_polys, bool inverse,
                          cudaStream_t s);
// Bytes of `ws` that scalar_transform32_ws stages in for n_polys polynomials
// (0 when the shape runs as one pass and stages nothing).
size_t scalar_transform32_ws_bytes(const Plan32& p, uint32_t n_polys);

// INT8 tensor-core engine for the wide plans (tc_wide.cu): n = 2^20, cyclic,
// moduli below 2^62 on byte planes of uint64 words.  Returns 1 when the plan
// is not served; src may equal dst (the plan workspace holds the first pass).
bool wide_tc_serves(const Plan64& p);
int wide_tc_transform64(Plan64& p, const void* src, void* dst, uint32_t n_polys, bool inverse, cudaStream_t s);
void wide_tc_release(Plan64* p);
uint32_t wide_device_errors(bool clear);
uint32_t wide_bounds_errors(bool clear);

// INT8 tensor-core engine (tc_int8.cu).
bool int8_serves(const Plan32& p, bool src_u64);
int int8_transform32(Plan32& p, const void* src, void* dst, bool src_u64, uint32_t n_polys, bool inverse,
                     cudaStream_t s);
void int8_release(Plan32* p);
uint32_t int8_device_errors(bool clear);
// Failed range checks of the NTT_DEBUG_BOUNDS build (bounds.cuh bits; 0 in the
// release build), per kernel file.
uint32_t int8_bounds_errors(bool clear);
// The INT8 cluster kernel's phase counters (NTT_PHASE_PROFILE build; zeros otherwise).
void int8_phase_profile(uint64_t* out16, bool clear);
uint32_t dmma_bounds_errors(bool clear);
uint32_t batch_bounds_errors(bool clear);
// Forward then inverse, in place, in one persistent launch.
int int8_forward_inverse32(Plan32& p, uint32_t* data, uint32_t n_polys, cudaStream_t s);

// Uneven-batch queue kernel (batch.cu): its bounded-wait error bits.
uint32_t batch_device_errors(bool clear);

// TMA tile mover (tma_move.cu).  Each returns 0 on launch, 1 when the shape
// or alignment is not served (the caller uses the plain kernels), 2 on a CUDA error.
int tma_transpose_u64(uint64_t* dst, const uint64_t* src, uint64_t rows, uint64_t cols, cudaStream_t stream);
int tma_transpose_square_inplace_u64(uint64_t* d, uint64_t n, cudaStream_t stream);
int tma_bit_reverse_u64(uint64_t* d, int log_n, cudaStream_t stream);
uint32_t tma_move_device_errors(bool clear);

// FP64 DMMA tensor-core engine (tc_dmma.cu).
bool dmma_serves(const Plan32& p, bool src_u64);
int dmma_transform32(Plan32& p, const void* src, void* dst, bool src_u64, uint32_t n_polys, bool inverse,
                     cudaStream_t s);
void dmma_release(Plan32* p);
int scalar_four_step32(const Plan32& p, uint64_t* data, uint64_t* scratch, bool inverse, cudaStream_t s);
// Transform of one uint64-word polynomial in the pre-transposed layout for
// n = M^2 (in place, staged in `mid`, n words); 1 when the plan is not served.
int scalar_pretransposed32(const Plan32& p, uint64_t* data, uint64_t* mid, bool inverse, cudaStream_t s);

}  // namespace nttb
