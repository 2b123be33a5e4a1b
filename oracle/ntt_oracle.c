/*
 * ntt_oracle.c -- CPU oracle for the four-step NTT hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker: only tests/,
 * __graft_entry__.smoke() and bench.py's cpu_baseline leg load it.  The
 * product library never links, calls or falls back to it.
 *
 * Every function restates, in plain C with unsigned __int128 arithmetic, the
 * reference's own CPU algorithm (file:line cited per function, paths relative
 * to the ntt-tensorcore project root).  Where the reference has no CPU code
 * (negacyclic twist, RNS batches) the restatement is the textbook definition,
 * pinned by the reference's schoolbook negacyclic loop
 * (tests/test_ntt.cu:186-199).
 *
 * Parity pins: tests/test_oracle.py checks these functions against outputs of
 * the reference's ntt_host / create_params compiled from the reference sources
 * (oracle/_ref, built by oracle/Makefile) and against the committed fixtures
 * in tests/golden/.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef unsigned __int128 u128;

static uint64_t mulmod(uint64_t a, uint64_t b, uint64_t q) {
    return (uint64_t)(((u128)a * b) % q);
}

static uint64_t addmod(uint64_t a, uint64_t b, uint64_t q) {
    u128 s = (u128)a + b;
    return (uint64_t)(s >= q ? s - q : s);
}

static uint64_t submod(uint64_t a, uint64_t b, uint64_t q) {
    return a >= b ? a - b : (uint64_t)((u128)a + q - b);
}

/* Square-and-multiply; include/modular_arith.cuh:110-122 (mod_pow). */
uint64_t oracle_pow(uint64_t base, uint64_t exp, uint64_t q) {
    uint64_t r = 1 % q;
    base %= q;
    while (exp) {
        if (exp & 1) r = mulmod(r, base, q);
        base = mulmod(base, base, q);
        exp >>= 1;
    }
    return r;
}

/* Fermat inverse; include/modular_arith.cuh:124-126 (mod_inverse). */
uint64_t oracle_inv(uint64_t a, uint64_t q) { return oracle_pow(a, q - 2, q); }

/*
 * Generator search; include/modular_arith.cuh:130-147.  The reference accepts
 * the smallest g >= 2 with g^((q-1)/p) != 1 for each p in {2,3,5,7} dividing
 * q-1 (only those four small primes are tested).
 */
uint64_t oracle_generator(uint64_t q) {
    static const uint64_t small[4] = {2, 3, 5, 7};
    for (uint64_t g = 2;; g++) {
        int ok = 1;
        for (int i = 0; i < 4 && ok; i++) {
            uint64_t p = small[i];
            if ((q - 1) % p == 0 && oracle_pow(g, (q - 1) / p, q) == 1) ok = 0;
        }
        if (ok) return g;
    }
}

/* omega = g^((q-1)/n); include/modular_arith.cuh:148-151. */
uint64_t oracle_primitive_root(uint64_t q, uint64_t n) {
    return oracle_pow(oracle_generator(q), (q - 1) / n, q);
}

/* psi = g^((q-1)/(2n)), a primitive 2n-th root with psi^2 == omega.  The
 * reference has no negacyclic code; this is the definition the build uses. */
uint64_t oracle_psi(uint64_t q, uint64_t n) {
    return oracle_pow(oracle_generator(q), (q - 1) / (2 * n), q);
}

/*
 * create_params; include/modular_arith.cuh:153-170.  out[] =
 * {q, q_twice, barrett_k, barrett_m, omega, omega_inv, n_inv}.  barrett_m is
 * floor(2^k / q) truncated to 64 bits exactly as the reference stores it.
 */
void oracle_params(uint64_t q, uint64_t n, uint64_t out[7]) {
    int k = 64;
    while ((1ULL << (k - 64)) < q && k < 96) k++;
    out[0] = q;
    out[1] = 2 * q;
    out[2] = (uint64_t)k;
    out[3] = (uint64_t)(((u128)1 << k) / q);
    out[4] = oracle_primitive_root(q, n);
    out[5] = oracle_inv(out[4], q);
    out[6] = oracle_inv(n % q, q);
}

/* mu = floor(2^64 / q); src/ntt_basic.cu:226-229. */
uint64_t oracle_mu(uint64_t q) { return (uint64_t)(((u128)1 << 64) / q); }

static int ilog2(uint64_t n) { int l = 0; while ((1ULL << l) < n) l++; return l; }

void oracle_bit_reverse(uint64_t* a, uint64_t n) {
    int lg = ilog2(n);
    for (uint64_t i = 0; i < n; i++) {
        uint64_t r = 0;
        for (int b = 0; b < lg; b++) r |= ((i >> b) & 1) << (lg - 1 - b);
        if (i < r) { uint64_t t = a[i]; a[i] = a[r]; a[r] = t; }
    }
}

/*
 * Cyclic DFT X[k] = sum_j x[j] * root^(j*k) mod q, natural order in and out,
 * optionally followed by multiplication with `scale` (n^-1 for the inverse).
 * Restates ntt_host, src/ntt_basic.cu:412-463: bit-reverse, then radix-2
 * Cooley-Tukey stages with per-stage root root^(n / 2^(s+1)).
 */
void oracle_dft(uint64_t* a, uint64_t n, uint64_t q, uint64_t root, uint64_t scale) {
    oracle_bit_reverse(a, n);
    for (uint64_t half = 1; half < n; half <<= 1) {
        uint64_t ws = oracle_pow(root, n / (2 * half), q);
        for (uint64_t g = 0; g < n; g += 2 * half) {
            uint64_t w = 1;
            for (uint64_t p = 0; p < half; p++) {
                uint64_t u = a[g + p];
                uint64_t v = mulmod(a[g + p + half], w, q);
                a[g + p] = addmod(u, v, q);
                a[g + p + half] = submod(u, v, q);
                w = mulmod(w, ws, q);
            }
        }
    }
    if (scale != 1)
        for (uint64_t i = 0; i < n; i++) a[i] = mulmod(a[i], scale, q);
}

/* ntt_host(data, params, inverse); src/ntt_basic.cu:412-463. */
void oracle_ntt(uint64_t* a, uint64_t n, uint64_t q, int inverse) {
    uint64_t w = oracle_primitive_root(q, n);
    if (!inverse) {
        oracle_dft(a, n, q, w, 1);
    } else {
        oracle_dft(a, n, q, oracle_inv(w, q), oracle_inv(n % q, q));
    }
}

/* Negacyclic transform (definition; no reference code exists):
 *   forward  Y = DFT_omega(x[j] * psi^j)
 *   inverse  x[j] = n^-1 * psi^-j * DFT_omega^-1(Y)[j]                     */
void oracle_negacyclic(uint64_t* a, uint64_t n, uint64_t q, int inverse) {
    uint64_t psi = oracle_psi(q, n);
    uint64_t w = mulmod(psi, psi, q);
    if (!inverse) {
        uint64_t t = 1;
        for (uint64_t j = 0; j < n; j++) { a[j] = mulmod(a[j], t, q); t = mulmod(t, psi, q); }
        oracle_dft(a, n, q, w, 1);
    } else {
        oracle_dft(a, n, q, oracle_inv(w, q), 1);
        uint64_t pinv = oracle_inv(psi, q), t = oracle_inv(n % q, q);
        for (uint64_t j = 0; j < n; j++) { a[j] = mulmod(a[j], t, q); t = mulmod(t, pinv, q); }
    }
}

/* RNS batch: data is n_polys x n_limbs x n residues, limb i uses moduli[i]. */
void oracle_rns(uint64_t* a, uint64_t n, const uint64_t* moduli, uint64_t n_limbs,
                uint64_t n_polys, int negacyclic, int inverse) {
    for (uint64_t p = 0; p < n_polys; p++)
        for (uint64_t l = 0; l < n_limbs; l++) {
            uint64_t* v = a + (p * n_limbs + l) * n;
            if (negacyclic) oracle_negacyclic(v, n, moduli[l], inverse);
            else oracle_ntt(v, n, moduli[l], inverse);
        }
}

/* Schoolbook product mod (x^n + 1); tests/test_ntt.cu:186-199. */
void oracle_polymul_negacyclic(uint64_t* out, const uint64_t* a, const uint64_t* b,
                               uint64_t n, uint64_t q) {
    memset(out, 0, n * sizeof(uint64_t));
    for (uint64_t i = 0; i < n; i++)
        for (uint64_t j = 0; j < n; j++) {
            uint64_t p = mulmod(a[i], b[j], q);
            uint64_t k = (i + j) % n;
            out[k] = (i + j) >= n ? submod(out[k], p, q) : addmod(out[k], p, q);
        }
}

/* Pointwise product; src/ntt_basic.cu:391-409 (poly_mul_kernel). */
void oracle_pointwise(uint64_t* out, const uint64_t* a, const uint64_t* b, uint64_t n, uint64_t q) {
    for (uint64_t i = 0; i < n; i++) out[i] = mulmod(a[i], b[i], q);
}

/* Plain DFT over a stride (helper for the four-step restatement). */
static void dft_strided(uint64_t* base, uint64_t len, uint64_t stride, uint64_t q,
                        uint64_t root, uint64_t* tmp) {
    for (uint64_t i = 0; i < len; i++) tmp[i] = base[i * stride];
    oracle_dft(tmp, len, q, root, 1);
    for (uint64_t i = 0; i < len; i++) base[i * stride] = tmp[i];
}

/*
 * The reference's four-step transform, src/ntt_four_step.cu:244-314
 * (forward) and :317-392 (inverse), written without its intra-block races:
 *   n1 = 2^max(6, log_n/2) (capped at n), n2 = n / n1
 *   forward: column DFT-n1 (stride n2) with root omega^(n/n1); Hadamard
 *            data[r*n2+c] *= omega^((r*c) mod n); transpose n1 x n2 -> n2 x n1;
 *            DFT-n2 over each contiguous chunk of n2 words (root omega^(n/n2)).
 *   inverse: chunked DFT-n2 with omega^-1; transpose n2 x n1 -> n1 x n2;
 *            Hadamard with omega^-((r*c) mod n); column DFT-n1 with omega^-1;
 *            multiply by n^-1.
 * The output is the reference's (it is not the natural-order DFT).
 */
void oracle_four_step(uint64_t* a, uint64_t n, uint64_t q, int inverse) {
    int log_n = ilog2(n);
    int log_n1 = log_n / 2;
    if (log_n1 < 6) log_n1 = 6;
    if (log_n1 > log_n) log_n1 = log_n;
    uint64_t n1 = 1ULL << log_n1, n2 = n / n1;
    uint64_t w = oracle_primitive_root(q, n);
    if (inverse) w = oracle_inv(w, q);
    uint64_t w1 = oracle_pow(w, n / n1, q), w2 = oracle_pow(w, n / n2, q);
    uint64_t* tmp = (uint64_t*)malloc(n * sizeof(uint64_t));
    uint64_t* t2 = (uint64_t*)malloc(n * sizeof(uint64_t));
    if (!inverse) {
        for (uint64_t c = 0; c < n2; c++) dft_strided(a + c, n1, n2, q, w1, tmp);
        for (uint64_t i = 0; i < n; i++) a[i] = mulmod(a[i], oracle_pow(w, ((i / n2) * (i % n2)) % n, q), q);
        for (uint64_t r = 0; r < n1; r++)
            for (uint64_t c = 0; c < n2; c++) t2[c * n1 + r] = a[r * n2 + c];
        memcpy(a, t2, n * sizeof(uint64_t));
        for (uint64_t p = 0; p < n1; p++) dft_strided(a + p * n2, n2, 1, q, w2, tmp);
    } else {
        for (uint64_t p = 0; p < n1; p++) dft_strided(a + p * n2, n2, 1, q, w2, tmp);
        for (uint64_t r = 0; r < n2; r++)
            for (uint64_t c = 0; c < n1; c++) t2[c * n2 + r] = a[r * n1 + c];
        memcpy(a, t2, n * sizeof(uint64_t));
        for (uint64_t i = 0; i < n; i++) a[i] = mulmod(a[i], oracle_pow(w, ((i / n2) * (i % n2)) % n, q), q);
        for (uint64_t c = 0; c < n2; c++) dft_strided(a + c, n1, n2, q, w1, tmp);
        uint64_t ninv = oracle_inv(n % q, q);
        for (uint64_t i = 0; i < n; i++) a[i] = mulmod(a[i], ninv, q);
    }
    free(tmp);
    free(t2);
}

/*
 * RowMaj layout helpers; src/ntt_optimized.cu:896-934:
 *   pre[beta * n1 + alpha] = canon[alpha * n2 + beta].
 */
void oracle_to_pretransposed(uint64_t* dst, const uint64_t* src, uint64_t n1, uint64_t n2) {
    for (uint64_t al = 0; al < n1; al++)
        for (uint64_t be = 0; be < n2; be++) dst[be * n1 + al] = src[al * n2 + be];
}

void oracle_from_pretransposed(uint64_t* dst, const uint64_t* src, uint64_t n1, uint64_t n2) {
    for (uint64_t al = 0; al < n1; al++)
        for (uint64_t be = 0; be < n2; be++) dst[al * n2 + be] = src[be * n1 + al];
}

/*
 * ntt_forward_rowmaj, src/ntt_optimized.cu:940-965 (kernels :650-890).  For
 * n == 4096 (n1 = n2 = 64) the buffer holds the pre-transposed input and
 * receives the pre-transposed forward DFT; other sizes run the plain forward
 * transform on the buffer as given (:944-948).
 */
void oracle_rowmaj_forward(uint64_t* a, uint64_t n, uint64_t q) {
    if (n != 4096) { oracle_ntt(a, n, q, 0); return; }
    uint64_t* c = (uint64_t*)malloc(n * sizeof(uint64_t));
    oracle_from_pretransposed(c, a, 64, 64);
    oracle_ntt(c, n, q, 0);
    oracle_to_pretransposed(a, c, 64, 64);
    free(c);
}
