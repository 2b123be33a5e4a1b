/*
 * ntt_b200.h -- C ABI of libntt_b200.so, the B200 (sm_100a) four-step NTT.
 *
 * Plain C: fixed-width integers, pointers and sizes, no CUDA or torch types.
 * Device pointers are device-memory addresses; `stream` is a cudaStream_t
 * passed as void* (NULL = legacy default stream).  Every entry point returns
 * an int status (NTTB_OK == 0); nttb_last_error() gives a one-line reason
 * for the last failure on the calling thread.
 *
 * Each declaration names the reference interface it replaces (paths relative
 * to the ntt-tensorcore project root).  The C++ drop-in headers in this
 * directory (ntt.cuh, modular_arith.cuh, ntt_arbitrary.cuh,
 * ntt_arbitrary_radix64.cuh) are thin wrappers over these symbols.
 */
#ifndef NTT_B200_H
#define NTT_B200_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define NTTB_API __attribute__((visibility("default")))
#else
#define NTTB_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------- status */
enum {
    NTTB_OK = 0,
    NTTB_ERR_INVALID_ARG = 1, /* size, modulus, pointer or alignment rejected */
    NTTB_ERR_UNSUPPORTED = 2, /* valid request outside what this build serves */
    NTTB_ERR_CUDA = 3,        /* a CUDA runtime call or kernel launch failed */
    NTTB_ERR_NO_MEMORY = 4,   /* a device or host allocation failed */
    NTTB_ERR_TIMEOUT = 5,     /* a bounded device-side wait ran out */
    NTTB_ERR_BUDGET = 6       /* serving admission refused: HBM budget exceeded */
};

/* Inner-DFT engines.  AUTO picks the fastest one that serves the request:
 * the INT8 tensor-core kernel at N = 2^16 from 8 (polynomial, limb) units
 * on; the batch queue's tensor tiles at N = 2^17 .. 2^20 once a call holds
 * 2^20 residues; the CUDA-core engine otherwise.  The tiles engine keeps up
 * to eight prepared queues per plan (one per source, destination, count,
 * direction), each with its own workspace ring of up to 16 x N words. */
enum {
    NTTB_ENGINE_AUTO = 0,
    NTTB_ENGINE_SCALAR = 1, /* CUDA-core radix-2 in shared memory */
    NTTB_ENGINE_DMMA = 2,   /* FP64 mma.sync m8n8k4 radix-8 contractions (the plain drop-in form) */
    NTTB_ENGINE_INT8 = 3,   /* tcgen05 kind::i8, byte-plane radix-64 contractions, INT32 in TMEM */
    NTTB_ENGINE_TILES = 4   /* the batch queue's tcgen05 tensor tiles (two-pass four-step, 2^13 .. 2^20) */
};

NTTB_API const char* nttb_version(void);
NTTB_API const char* nttb_status_string(int status);
NTTB_API const char* nttb_last_error(void);
/* Device-side error bits raised by bounded waits in the persistent kernels
 * (bit 0: an INT8-engine mbarrier wait ran out of budget, bit 1: a wait on
 * another CTA of an INT8 cluster did, bit 2: an uneven-batch queue
 * dependency wait did, bit 3: a batch tensor tile's wait on its MMA or image
 * copy did; the work item ran on regardless and its output is wrong; bit 4:
 * a TMA tile load of a transpose or bit reversal did not land, and that CTA
 * stopped storing; bit 5: a wait of the 64-bit byte-plane engine did).  Every
 * such wait gives up after about 2 s of device time.  Reads after a device
 * synchronize; clear != 0 resets them. */
NTTB_API int nttb_device_errors(uint32_t* flags, int clear);
/* Range checks of the NTT_DEBUG_BOUNDS build (ntt_b200/libntt_b200_dbg.so,
 * `python ntt-tensorcore_b200/build.py --debug-bounds`), the stand-in for a
 * memory checker: bits 0-7 the INT8 cluster kernel, 8-15 the DMMA passes,
 * 16-23 the uneven-batch queue kernels, 24-31 the 64-bit byte-plane engine
 * (nttb_wide_transform_engine); within each byte the kind of check
 * that failed (bit 0 global-memory index, 1 shared-memory offset, 2
 * distributed-shared-memory piece copy, 3 queue ticket / unit / tile index,
 * 4 workspace slot, 5 output residue not reduced).  A failed check skips
 * the access it guards.  *enabled = 1 in that build; the release build
 * compiles the checks away (enabled 0, flags 0).  Reads after a device
 * synchronize; clear != 0 resets them.  No reference counterpart (the
 * reference's debug build is nvcc -G -g, CMakeLists.txt:10). */
NTTB_API int nttb_bounds_errors(uint32_t* flags, int* enabled, int clear);

/* Phase profile of the INT8 cluster kernel, in the NTT_PHASE_PROFILE build
 * (libntt_b200_phase.so, `python ntt-tensorcore_b200/build.py
 * --phase-profile`): out[0..15] receive clock() cycles summed over the
 * epilogue warps of every launch since the last clear -- 0 waiting for the
 * stage's MMA, 1 TMEM loads, 2 gates before staging stores, 3 part barriers
 * and piece sends, 4 level-2 MMA, 5 end-of-stage barrier, 6 whole stages --
 * and per CTA: 7 lifetime, 8 start-up (including the wait for the previous
 * grid), 9 CTAs counted.  *enabled = 1 in that build; the release build
 * has no probes (enabled 0, zeros).  Read after a device synchronize;
 * clear != 0 resets the counters.  No reference counterpart. */
NTTB_API int nttb_phase_profile(uint64_t* out16, int* enabled, int clear);

/* ------------------------------------------------ modular parameters (host)
 * Field-for-field the reference's ModularParams
 * (include/modular_arith.cuh:11-19). */
typedef struct {
    uint64_t q, q_twice, barrett_k, barrett_m, omega, omega_inv, n_inv;
} nttb_modular_params;

/* Replaces create_params (include/modular_arith.cuh:153-170). */
NTTB_API int nttb_create_params(uint64_t q, uint64_t n, nttb_modular_params* out);
/* Replaces find_primitive_root (include/modular_arith.cuh:130-151). */
NTTB_API int nttb_find_primitive_root(uint64_t q, uint64_t n, uint64_t* omega);
/* psi = g^((q-1)/(2n)) with the same generator: primitive 2n-th root, psi^2 = omega. */
NTTB_API int nttb_find_psi(uint64_t q, uint64_t n, uint64_t* psi);
/* Replaces ntt_host (src/ntt_basic.cu:412-463): CPU NTT, natural order in place. */
NTTB_API int nttb_host_ntt(uint64_t* data, uint64_t n, const nttb_modular_params* params, int inverse);
/* Descending primes q < 2^bits with q == 1 mod 2^two_adicity (bits <= 62). */
NTTB_API int nttb_generate_primes(uint32_t bits, uint32_t two_adicity, uint32_t count, uint64_t* out);

/* ---------------------------------- single-modulus plan over uint64 words
 * Backs NTTConfig (include/ntt.cuh:11-24).  q < 2^31 runs the 31-bit
 * engines; 2^31 <= q < 2^62 runs the 64-bit Montgomery path. */
typedef struct nttb_plan nttb_plan;
typedef struct {
    uint64_t n, log_n, q, mu;
    uint64_t* d_twiddles;     /* omega^k, k < n (the reference's table layout) */
    uint64_t* d_twiddles_inv; /* omega^-k, k < n */
    nttb_modular_params params;
} nttb_plan_info;

/* Replaces ntt_init (src/ntt_basic.cu:217-249). */
NTTB_API int nttb_plan_create(uint64_t n, uint64_t q, nttb_plan** out);
/* Replaces ntt_cleanup (src/ntt_basic.cu:251-257). */
NTTB_API int nttb_plan_destroy(nttb_plan* plan);
NTTB_API int nttb_plan_get_info(const nttb_plan* plan, nttb_plan_info* out);

/* Natural-order cyclic NTT over `batch` contiguous polynomials of n words,
 * in place.  Replaces ntt_forward/inverse_{basic,tlmop,optimized}
 * (src/ntt_basic.cu:268-334, src/ntt_optimized.cu:515-613) and
 * ntt_forward/inverse_batch (src/ntt_basic.cu:337-389).  NTTB_ENGINE_AUTO
 * runs, for q < 2^31, the INT8 tensor-core kernel on the words directly for
 * n = 2^16 from 8 polynomials on, the batch queue's tensor tiles for
 * n = 2^17 .. 2^20 from 2^20 words per call, the CUDA-core engine otherwise
 * (residues must be below 2^32, as the reference's kernels assume them below
 * q). */
NTTB_API int nttb_u64_transform(const nttb_plan* plan, uint64_t* d_data, uint64_t batch, int inverse, int engine,
                       void* stream);
/* The reference's four-step map, in place.  Replaces
 * ntt_forward/inverse_four_step (src/ntt_four_step.cu:244-392). */
NTTB_API int nttb_u64_four_step(const nttb_plan* plan, uint64_t* d_data, int inverse, void* stream);
/* Pre-transposed forward NTT for n == 4096, plain forward otherwise.
 * Replaces ntt_forward_rowmaj (src/ntt_optimized.cu:940-965). */
NTTB_API int nttb_u64_rowmaj_forward(const nttb_plan* plan, uint64_t* d_data, void* stream);
/* The RowMaj pre-transposed layout for every n and both directions: d_data
 * holds pre[b*n1 + a] = x[a*n2 + b] (n2 = n / n1, the layout of
 * rowmaj_to_pretransposed, src/ntt_optimized.cu:893-895, 922-934) and
 * receives the transform in the same layout, in place.  n1 a power of two
 * <= n; nttb_u64_rowmaj_forward is the case n = 4096, n1 = 64, forward.
 * Square shapes (n1 * n1 == n, q < 2^31) run as two passes that read and
 * write the layout directly; others as a TMA transpose, the transform, and
 * the transpose back. */
NTTB_API int nttb_u64_pretransposed_transform(const nttb_plan* plan, uint64_t* d_data, uint64_t n1, int inverse,
                                              void* stream);
/* d_dst[c*rows + r] = d_src[r*cols + c].  Replaces rowmaj_to_pretransposed
 * (rows=N1, cols=N2) and rowmaj_from_pretransposed (rows=N2, cols=N1),
 * src/ntt_optimized.cu:922-934.  d_dst may equal d_src only for a square matrix.
 * rows and cols multiples of 32 with 16-byte aligned arrays run on TMA tiles;
 * other shapes on a plain tiled kernel. */
NTTB_API int nttb_u64_transpose(uint64_t* d_dst, const uint64_t* d_src, uint64_t rows, uint64_t cols, void* stream);
/* d_out[i] = d_a[i] * d_b[i] mod q, i < n.  Replaces poly_multiply_ntt
 * (src/ntt_basic.cu:391-409). */
NTTB_API int nttb_u64_pointwise_mul(const nttb_plan* plan, uint64_t* d_out, const uint64_t* d_a, const uint64_t* d_b,
                           void* stream);
/* In-place bit-reversal permutation.  Replaces bit_reverse_permute
 * (src/ntt_basic.cu:259-265).  From n = 2^10 on, with a 16-byte aligned
 * array, it runs on TMA tile pairs. */
NTTB_API int nttb_u64_bit_reverse(uint64_t* d_data, uint64_t n, void* stream);

/* ------------------------------------------ RNS batches of uint32 residues
 * No single reference counterpart: the reference batches only one modulus by
 * a host loop (ntt_forward_batch, src/ntt_basic.cu:337-389).  Data layout is
 * [poly][limb][n] uint32, limb l reduced mod moduli[l] (q < 2^31). */
typedef struct nttb_rns_plan nttb_rns_plan;
#define NTTB_NEGACYCLIC 1u

NTTB_API int nttb_rns_plan_create(uint32_t log_n, const uint64_t* moduli, uint32_t n_limbs, uint32_t flags,
                         nttb_rns_plan** out);
NTTB_API int nttb_rns_plan_destroy(nttb_rns_plan* plan);
/* d_dst = NTT(d_src) (forward) or NTT^-1 (inverse); d_dst may equal d_src.
 * Negacyclic plans twist by psi^j before the forward and by n^-1 psi^-j
 * after the inverse. */
NTTB_API int nttb_rns_transform(const nttb_rns_plan* plan, uint32_t* d_dst, const uint32_t* d_src, uint32_t n_polys,
                       int inverse, int engine, void* stream);
/* Forward then inverse transform of d_data in place (the round trip of the
 * reference's test_ntt_inverse, tests/test_ntt.cu:60-123, for a whole RNS
 * batch).  The INT8 engine runs both in one persistent launch with
 * per-(poly, limb) stage dependencies; other engines run two transforms. */
NTTB_API int nttb_rns_forward_inverse(const nttb_rns_plan* plan, uint32_t* d_data, uint32_t n_polys, int engine,
                                      void* stream);
/* Streams n_batches consecutive batches of n_polys polynomials from host
 * memory h_src to h_dst (batch i at offset i * n_polys * n_limbs * n words):
 * copy in, transform (mode 0 forward, 1 inverse, 2 forward then inverse),
 * copy out, with the copies of neighbouring batches overlapping the
 * transforms (three device buffers owned by the plan, two copy streams per
 * direction).  Asynchronous: `stream` completes after the last copy back;
 * h_src and h_dst must stay valid until then, and should be pinned
 * (cudaHostAlloc / cudaHostRegister) for the copies to overlap.  No reference
 * counterpart (the reference API takes device pointers only). */
NTTB_API int nttb_rns_stream_host(nttb_rns_plan* plan, const uint32_t* h_src, uint32_t* h_dst, uint32_t n_polys,
                                  uint32_t n_batches, int mode, int engine, void* stream);
/* In-place transform that allocates no device memory.  No counterpart in the
 * reference.  For callers that cannot call cudaMalloc while transforming (a
 * memory manager that owns all device memory, a loop that must never enter
 * the allocator because cudaMalloc can synchronize the device, a fixed
 * up-front memory budget).  The first pass is staged in a static device
 * buffer of NTTB_NOALLOC_SCRATCH_BYTES that every GPU loading the library
 * holds until exit.  Shapes that run in two passes (n > 8192, or n >= 4096
 * with fewer than 8 (polynomial, limb) units) stage n_polys * n_limbs * n * 4
 * bytes there, and batches needing more are rejected with
 * NTTB_ERR_INVALID_ARG; one-pass shapes stage nothing and are not limited.
 * The plan's device must be the current device (else NTTB_ERR_INVALID_ARG).
 * The first call on a device looks up the buffer's address
 * (cudaGetSymbolAddress) and keeps it: make that call before any stream
 * capture, and do not call again on a device after cudaDeviceReset.  Calls
 * share the buffer: calls whose work overlaps on the GPU race.  Runs the
 * CUDA-core engine; same results as nttb_rns_transform. */
#define NTTB_NOALLOC_SCRATCH_BYTES (8u << 20)
NTTB_API int nttb_rns_transform_noalloc(const nttb_rns_plan* plan, uint32_t* d_data, uint32_t n_polys, int inverse,
                                        void* stream);
/* d_out = d_a * d_b pointwise per limb (NTT domain). */
NTTB_API int nttb_rns_pointwise_mul(const nttb_rns_plan* plan, uint32_t* d_out, const uint32_t* d_a,
                           const uint32_t* d_b, uint32_t n_polys, void* stream);

/* ------------------------------------------- 64-bit moduli (q < 2^62)
 * The multi-limb big-prime path: residues stored as uint64 (two 32-bit
 * words).  Replaces the K-limb run_forward_ct_tcu path for primes near 2^60
 * (include/ntt_arbitrary.cuh:2599-2646) and adds the inverse it lacks. */
typedef struct nttb_wide_plan nttb_wide_plan;
NTTB_API int nttb_wide_plan_create(uint32_t log_n, const uint64_t* moduli, uint32_t n_limbs, uint32_t flags,
                          nttb_wide_plan** out);
NTTB_API int nttb_wide_plan_destroy(nttb_wide_plan* plan);
NTTB_API int nttb_wide_transform(const nttb_wide_plan* plan, uint64_t* d_dst, const uint64_t* d_src, uint32_t n_polys,
                        int inverse, void* stream);
/* The same with the engine named: NTTB_ENGINE_INT8 runs the tcgen05 kind::i8
 * byte-plane engine (eight byte planes of each uint64 word, DFT-32 x DFT-32
 * per pass of the four-step 1024 x 1024; served for n = 2^20, cyclic plans;
 * NTTB_ERR_UNSUPPORTED otherwise), NTTB_ENGINE_SCALAR the CUDA-core
 * Montgomery-64 engine, NTTB_ENGINE_AUTO (what nttb_wide_transform uses) the
 * INT8 engine where it serves the plan and the batch has fewer than 8
 * (polynomial, limb) units (it has the shorter latency; the CUDA-core engine
 * the higher throughput on larger batches).  Pointers 16-byte aligned; src may
 * equal dst.  Replaces the reference's run_forward_ct_tcu<K> for primes near
 * 2^60 (include/ntt_arbitrary.cuh:2599-2646, its limb products on FP64 MMA). */
NTTB_API int nttb_wide_transform_engine(const nttb_wide_plan* plan, uint64_t* d_dst, const uint64_t* d_src,
                                        uint32_t n_polys, int inverse, int engine, void* stream);

/* ------------------------------------------------------- uneven batches
 * No single reference counterpart (the reference transforms one size and one
 * modulus per call, ntt_forward_batch, src/ntt_basic.cu:337-389).  A batch
 * plan holds twiddle tables for up to 2^24 residues for a set of 31-bit
 * moduli; a batch is a list of jobs -- polynomials of any size 2^1 ..
 * 2^max_log_n, any number of consecutive moduli of the plan, forward or
 * inverse, cyclic or negacyclic -- run by ONE persistent launch that draws
 * (unit, pass, tile) work items from a device queue.  Results equal
 * nttb_rns_transform on each job.  Data of a job: n_limbs rows of 2^log_n
 * uint32 residues (row l reduced mod moduli[first_modulus + l]), in place. */
typedef struct nttb_batch_plan nttb_batch_plan;
typedef struct nttb_batch nttb_batch;
#define NTTB_BATCH_INVERSE 2u /* job flag; NTTB_NEGACYCLIC (1) selects the negacyclic twist */
/* Job flag: product of two polynomials.  data <- a * b (negacyclic with
 * NTTB_NEGACYCLIC, else cyclic), a = data, b = pointwise (same layout, left
 * in the NTT domain).  Forward(a), forward(b), the pointwise product and the
 * inverse run in the same launch; replaces poly_multiply_ntt
 * (src/ntt_basic.cu:391-409) between ntt_forward and ntt_inverse calls. */
#define NTTB_BATCH_POLYMUL 4u
typedef struct {
    uint32_t* data;         /* device memory, n_limbs << log_n words, transformed in place */
    uint32_t log_n;         /* 1 .. plan max_log_n */
    uint32_t n_limbs;
    uint32_t first_modulus; /* row l uses the plan's modulus first_modulus + l */
    uint32_t flags;         /* NTTB_BATCH_INVERSE | NTTB_NEGACYCLIC | NTTB_BATCH_POLYMUL */
    uint32_t* pointwise;    /* NTTB_BATCH_POLYMUL: the second operand (overwritten by its transform) */
} nttb_batch_job;
/* Tuning knobs (see nttb_batch_autotune). */
typedef struct {
    uint32_t tile_elems;  /* shared-memory tile: 4096, 8192 or 16384 residues */
    uint32_t threads;     /* CTA width: 256 (tiles 4096, 8192) or 512 (tiles 8192, 16384) */
    uint32_t split;       /* two-pass radix split: 0 first pass 2^ceil(L/2), 1 first pass 2^floor(L/2) */
    uint32_t lag;         /* two-pass units between a unit's first and second pass in the queue (1..64) */
    uint32_t ctas_per_sm; /* 0: as many as fit */
    uint32_t group;       /* radix-2 stages per register group inside a tile: 1, 3 or 4 */
    uint32_t tensor;      /* 1: two-pass units of 2^13 .. 2^20 residues (the sizes above the tile) run
                             tensor-core tiles (INT8 DFT-64 + radix-2 DFT of up to 16 points) where the
                             shape allows: threads 256 and tile_elems 4096 or 8192; otherwise ignored */
} nttb_batch_config;

/* flags: NTTB_NEGACYCLIC to allow negacyclic jobs (moduli then need 2^(max_log_n+1) | q-1). */
NTTB_API int nttb_batch_plan_create(const uint64_t* moduli, uint32_t n_moduli, uint32_t max_log_n, uint32_t flags,
                                    nttb_batch_plan** out);
NTTB_API int nttb_batch_plan_destroy(nttb_batch_plan* plan);
NTTB_API int nttb_batch_default_config(nttb_batch_config* out);
/* Times every knob combination on a sample of the jobs' mix (scratch
 * buffers; the jobs' data is not touched), keeps the fastest as the plan's
 * default for later nttb_batch_create calls and returns it. */
NTTB_API int nttb_batch_autotune(nttb_batch_plan* plan, const nttb_batch_job* jobs, uint32_t n_jobs, void* stream,
                                 nttb_batch_config* out);
/* Builds the work queue of a job list (host work + device upload; allocates
 * the queue and a workspace ring for the two-pass units).  config NULL: the
 * plan's tuned configuration, else the default. */
NTTB_API int nttb_batch_create(nttb_batch_plan* plan, const nttb_batch_job* jobs, uint32_t n_jobs,
                               const nttb_batch_config* config, nttb_batch** out);
NTTB_API int nttb_batch_destroy(nttb_batch* batch);
/* Runs the batch: a counter reset and one persistent kernel on `stream`; no
 * allocation, no host synchronisation. */
NTTB_API int nttb_batch_launch(nttb_batch* batch, void* stream);
/* Same work, replayed from a CUDA graph captured on the first call. */
NTTB_API int nttb_batch_graph_launch(nttb_batch* batch, void* stream);
NTTB_API int nttb_batch_info(const nttb_batch* batch, uint64_t* units, uint64_t* tiles, uint64_t* ws_bytes,
                             nttb_batch_config* config);
/* CTAs of the persistent launch (SMs x resident CTAs per SM, at most the tile count). */
NTTB_API int nttb_batch_ctas(const nttb_batch* batch, uint32_t* ctas);
/* Test hook for the failure path: makes the second pass of two-pass unit
 * `unit` wait for one first-pass tile more than exist, so that its bounded
 * device wait runs out (about 2 s): the launch still completes, with that
 * unit's result unreliable and bit 2 set in nttb_device_errors.  Recreate
 * the batch afterwards. */
NTTB_API int nttb_batch_test_stall(nttb_batch* batch, uint32_t unit);

/* ------------------------------------------------------------- serving
 * No reference counterpart (the reference has no request loop).  A server
 * multiplies and transforms polynomials for callers in host memory:
 *   product request = (a, b) with n_limbs rows of 2^log_n residues (row l mod
 *     moduli[first_modulus + l]), result out = a * b per limb (negacyclic
 *     unless config.negacyclic == 0), device operands 2 x n_limbs x 2^log_n words;
 *   NTT request = one such operand, result its forward or inverse transform
 *     per limb (with the negacyclic twist unless config.negacyclic == 0),
 *     device operand n_limbs x 2^log_n words.
 * Requests of both kinds share one queue and are admitted in arrival order
 * while their device operands fit in the HBM budget left after the resident
 * twiddle tables and queues, and are batched continuously: up to `slots`
 * batches are in flight on separate streams, each one persistent launch
 * (per product: forward a, forward b, product, inverse; per NTT: the
 * transform) between its copies.  a, b and out
 * must stay valid until the request completes; pinned host memory lets the
 * copies overlap.  Latency = submit -> completion, host steady clock. */
typedef struct nttb_server nttb_server;
typedef struct {
    uint64_t hbm_budget_bytes;   /* device bytes for tables, queues and request operands */
    uint32_t max_log_n;          /* largest request size */
    uint32_t slots;              /* batches in flight (streams), 1..16 */
    uint32_t max_batch_requests; /* requests per batch */
    uint32_t negacyclic;         /* 1: negacyclic products (x^n = -1), 0: cyclic */
    uint64_t max_batch_residues; /* transform residues per batch (3 per operand residue) */
    nttb_batch_config batch;     /* tiles of the batch engine */
} nttb_server_config;
typedef struct {
    uint64_t submitted, completed, queued, batches, batched_requests;
    uint64_t bytes_in_use, peak_bytes_in_use, region_bytes, resident_bytes;
} nttb_server_stats_t;

/* Defaults: 60 GB budget, 2^17, 3 slots, 64 requests and 2^27 residues per batch, negacyclic. */
NTTB_API int nttb_server_default_config(nttb_server_config* out);
NTTB_API int nttb_server_create(const uint64_t* moduli, uint32_t n_moduli, const nttb_server_config* config,
                                nttb_server** out);
/* Queues a request; NTTB_ERR_BUDGET if its operands alone exceed the request region. */
NTTB_API int nttb_server_submit(nttb_server* server, const uint32_t* a, const uint32_t* b, uint32_t* out,
                                uint32_t log_n, uint32_t n_limbs, uint32_t first_modulus, uint64_t* id);
/* Queues an NTT request: out = the forward (inverse != 0: inverse) transform of
 * `in` per limb; NTTB_ERR_BUDGET if its operand alone exceeds the request region. */
NTTB_API int nttb_server_submit_ntt(nttb_server* server, const uint32_t* in, uint32_t* out, uint32_t log_n,
                                    uint32_t n_limbs, uint32_t first_modulus, int inverse, uint64_t* id);
/* Device-resident operands: the same requests with a, b and out in device
 * memory of the server's device, for callers that keep their residues in
 * HBM between requests.  kind: NTTB_SERVER_PRODUCT (out = a * b per limb),
 * NTTB_SERVER_FORWARD / NTTB_SERVER_INVERSE (out = the transform of a per
 * limb; b ignored, may be NULL).  The operands are copied device-to-device
 * into the server's region on the batch's stream and the result
 * device-to-device into out, so nothing crosses the host link; a, b and out
 * must stay valid (and a, b unchanged) until the request completes.  Host
 * pointers, or memory of another device, are refused (NTTB_ERR_INVALID_ARG).
 * The reference's device-pointer product is poly_multiply_ntt
 * (src/ntt_basic.cu:391-409); it has no request loop. */
#define NTTB_SERVER_PRODUCT 0
#define NTTB_SERVER_FORWARD 1
#define NTTB_SERVER_INVERSE 2
NTTB_API int nttb_server_submit_device(nttb_server* server, int kind, const uint32_t* d_a, const uint32_t* d_b,
                                       uint32_t* d_out, uint32_t log_n, uint32_t n_limbs, uint32_t first_modulus,
                                       uint64_t* id);
/* Waits for one request (NTTB_ERR_TIMEOUT after timeout_s); its latency in seconds.
 * A request's record (status, latency) is kept until a wait collects it, so
 * every id should be waited for once; a second wait on it is refused. */
NTTB_API int nttb_server_wait(nttb_server* server, uint64_t id, double timeout_s, double* latency_s);
NTTB_API int nttb_server_drain(nttb_server* server, double timeout_s);
NTTB_API int nttb_server_stats(nttb_server* server, nttb_server_stats_t* out);
/* Latencies of completed requests in completion order (count = how many
 * there are; up to cap copied); reset != 0 forgets them.  They accumulate
 * (8 bytes a request) until a reset. */
NTTB_API int nttb_server_latencies(nttb_server* server, double* out, uint64_t cap, uint64_t* count, int reset);
/* Drains, then releases the server. */
NTTB_API int nttb_server_destroy(nttb_server* server);

/* ------------------------------------ K-limb residues (24-bit limbs)
 * The reference's header-only arbitrary-modulus path: elements are
 * DScalar<K> = K little-endian uint32 words, each a 24-bit limb, in
 * Montgomery form (R = 2^(24 K)), canonical in [0, p).  Forward transform in
 * place, natural order in and out: bit reversal then the radix-2 DIT network
 * of host_ntt_naive (include/ntt_arbitrary.cuh:2651-2676) with twiddle
 * d_tw[k * n / 2^(s+1)] at stage s (d_tw: n Montgomery-form powers of omega,
 * as setup_ntt builds them).  `prime` is a HOST array of K limbs, np =
 * -prime^-1 mod 2^24.  Replaces run_forward_ct, run_forward_ct_tcu
 * (include/ntt_arbitrary.cuh:2547-2646) and run_forward_radix64_scalar
 * (include/ntt_arbitrary_radix64.cuh:345-389), which compute the same
 * network.  K in {2, 3, 11} (the reference's FieldConfig set), n = 2^log_n,
 * log_n <= 24. */
NTTB_API int nttb_klimb_forward(uint32_t K, uint32_t* d_data, const uint32_t* d_tw, uint64_t n, uint32_t log_n,
                                const uint32_t* prime, uint32_t np, void* stream);

/* ------------------------------------------------------------ accounting
 * No reference counterpart (the reference times with ad-hoc cudaEvents,
 * tests/benchmark.cu:52-99).  nttb_launch_count counts every kernel launch
 * the library has issued.  Between nttb_profile_start and nttb_profile_stop
 * the library brackets each of its launches with CUDA events on the
 * launching stream; nttb_profile_stop synchronizes those events and
 * aggregates device time per kernel name, read back by index. */
NTTB_API int nttb_launch_count(uint64_t* out);
NTTB_API int nttb_profile_start(void);
NTTB_API int nttb_profile_stop(uint32_t* n_kernels);
NTTB_API int nttb_profile_read(uint32_t index, char* name, uint32_t name_len, uint64_t* launches,
                               double* total_ms);

#ifdef __cplusplus
}
#endif

#endif /* NTT_B200_H */
