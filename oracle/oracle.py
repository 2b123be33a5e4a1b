"""ctypes loader for the CPU oracle (TEST INFRASTRUCTURE ONLY).

Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline / reference
legs import this module.  The product package never does.

Two libraries:
  * ``liboracle.so`` -- the C restatement in ``ntt_oracle.c``;
  * ``_ref/libntt_ref.so`` -- the reference's own CPU (and GPU) NTT compiled
    from the reference sources by ``oracle/Makefile`` (optional: absent when
    the reference tree was not available at build time).
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_u64p = ctypes.POINTER(ctypes.c_uint64)
_u32p = ctypes.POINTER(ctypes.c_uint32)


def _p64(a):
    assert a.dtype == np.uint64 and a.flags.c_contiguous
    return a.ctypes.data_as(_u64p)


def _p32(a):
    assert a.dtype == np.uint32 and a.flags.c_contiguous
    return a.ctypes.data_as(_u32p)


_lib = None
_ref = None


def lib():
    global _lib
    if _lib is None:
        path = os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            raise RuntimeError("oracle not built: run `make -C oracle`")
        L = ctypes.CDLL(path)
        u64 = ctypes.c_uint64
        L.oracle_pow.restype = u64
        L.oracle_pow.argtypes = [u64, u64, u64]
        L.oracle_inv.restype = u64
        L.oracle_inv.argtypes = [u64, u64]
        L.oracle_generator.restype = u64
        L.oracle_generator.argtypes = [u64]
        L.oracle_primitive_root.restype = u64
        L.oracle_primitive_root.argtypes = [u64, u64]
        L.oracle_psi.restype = u64
        L.oracle_psi.argtypes = [u64, u64]
        L.oracle_mu.restype = u64
        L.oracle_mu.argtypes = [u64]
        L.oracle_params.argtypes = [u64, u64, _u64p]
        L.oracle_ntt.argtypes = [_u64p, u64, u64, ctypes.c_int]
        L.oracle_negacyclic.argtypes = [_u64p, u64, u64, ctypes.c_int]
        L.oracle_rns.argtypes = [_u64p, u64, _u64p, u64, u64, ctypes.c_int, ctypes.c_int]
        L.oracle_polymul_negacyclic.argtypes = [_u64p, _u64p, _u64p, u64, u64]
        L.oracle_pointwise.argtypes = [_u64p, _u64p, _u64p, u64, u64]
        L.oracle_four_step.argtypes = [_u64p, u64, u64, ctypes.c_int]
        L.oracle_rowmaj_forward.argtypes = [_u64p, u64, u64]
        L.oracle_to_pretransposed.argtypes = [_u64p, _u64p, u64, u64]
        L.oracle_from_pretransposed.argtypes = [_u64p, _u64p, u64, u64]
        L.oracle_bit_reverse.argtypes = [_u64p, u64]
        _lib = L
    return _lib


def ref():
    """The reference's own code, or None when it was not built."""
    global _ref
    if _ref is None:
        path = os.path.join(HERE, "_ref", "libntt_ref.so")
        if not os.path.exists(path):
            return None
        R = ctypes.CDLL(path)
        u64 = ctypes.c_uint64
        R.ref_create_params.argtypes = [u64, u64, _u64p]
        R.ref_ntt_host.argtypes = [_u64p, u64, u64, ctypes.c_int]
        R.ref_ntt_host_batch.restype = ctypes.c_int
        R.ref_ntt_host_batch.argtypes = [_u64p, u64, _u64p, u64, u64, ctypes.c_int, ctypes.c_int, ctypes.c_int]
        R.ref_random_polynomial.argtypes = [_u64p, u64, u64, ctypes.c_uint32]
        R.ref_ntt_init.restype = ctypes.c_void_p
        R.ref_ntt_init.argtypes = [u64, u64]
        R.ref_ntt_cleanup.argtypes = [ctypes.c_void_p]
        R.ref_ntt_run.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int]
        if hasattr(R, "ref_ntt_rns_optimized"):  # absent from libraries built before it existed
            R.ref_ntt_rns_optimized.argtypes = [ctypes.POINTER(ctypes.c_void_p), u64, u64, ctypes.c_void_p,
                                                ctypes.c_int, ctypes.c_void_p]
        R.ref_klimb_case.restype = ctypes.c_int
        R.ref_klimb_case.argtypes = [ctypes.c_int, ctypes.c_int, u64, _u32p, _u32p, _u32p, _u32p]
        R.ref_klimb_mont.restype = ctypes.c_int
        R.ref_klimb_mont.argtypes = [ctypes.c_int, _u32p, _u32p, _u32p, _u32p, _u32p]
        _ref = R
    return _ref


# ---------------------------------------------------------------- oracle API
def params(q, n):
    out = np.zeros(7, dtype=np.uint64)
    lib().oracle_params(q, n, _p64(out))
    return [int(x) for x in out]


def generator(q):
    return int(lib().oracle_generator(q))


def primitive_root(q, n):
    return int(lib().oracle_primitive_root(q, n))


def psi(q, n):
    return int(lib().oracle_psi(q, n))


def ntt(x, q, inverse=False):
    a = np.ascontiguousarray(x, dtype=np.uint64).copy()
    lib().oracle_ntt(_p64(a), a.size, q, int(inverse))
    return a


def negacyclic(x, q, inverse=False):
    a = np.ascontiguousarray(x, dtype=np.uint64).copy()
    lib().oracle_negacyclic(_p64(a), a.size, q, int(inverse))
    return a


def rns(x, moduli, negacyclic=False, inverse=False):
    """x: array shaped (n_polys, n_limbs, n) or (n_limbs, n)."""
    a = np.ascontiguousarray(x, dtype=np.uint64).copy()
    m = np.ascontiguousarray(moduli, dtype=np.uint64)
    n = a.shape[-1]
    n_limbs = m.size
    n_polys = a.size // (n * n_limbs)
    lib().oracle_rns(_p64(a), n, _p64(m), n_limbs, n_polys, int(negacyclic), int(inverse))
    return a


def polymul_negacyclic(a, b, q):
    a = np.ascontiguousarray(a, dtype=np.uint64)
    b = np.ascontiguousarray(b, dtype=np.uint64)
    out = np.zeros_like(a)
    lib().oracle_polymul_negacyclic(_p64(out), _p64(a), _p64(b), a.size, q)
    return out


def pointwise(a, b, q):
    a = np.ascontiguousarray(a, dtype=np.uint64)
    b = np.ascontiguousarray(b, dtype=np.uint64)
    out = np.zeros_like(a)
    lib().oracle_pointwise(_p64(out), _p64(a), _p64(b), a.size, q)
    return out


def four_step(x, q, inverse=False):
    a = np.ascontiguousarray(x, dtype=np.uint64).copy()
    lib().oracle_four_step(_p64(a), a.size, q, int(inverse))
    return a


def rowmaj_forward(x, q):
    a = np.ascontiguousarray(x, dtype=np.uint64).copy()
    lib().oracle_rowmaj_forward(_p64(a), a.size, q)
    return a


def to_pretransposed(x, n1, n2):
    a = np.ascontiguousarray(x, dtype=np.uint64)
    out = np.zeros_like(a)
    lib().oracle_to_pretransposed(_p64(out), _p64(a), n1, n2)
    return out


def from_pretransposed(x, n1, n2):
    a = np.ascontiguousarray(x, dtype=np.uint64)
    out = np.zeros_like(a)
    lib().oracle_from_pretransposed(_p64(out), _p64(a), n1, n2)
    return out


def bit_reverse(x):
    a = np.ascontiguousarray(x, dtype=np.uint64).copy()
    lib().oracle_bit_reverse(_p64(a), a.size)
    return a


# ------------------------------------------------------ reference CPU (pins)
def ref_params(q, n):
    R = ref()
    out = np.zeros(8, dtype=np.uint64)
    R.ref_create_params(q, n, _p64(out))
    return [int(x) for x in out]


def ref_ntt_host(x, q, inverse=False):
    R = ref()
    a = np.ascontiguousarray(x, dtype=np.uint64).copy()
    R.ref_ntt_host(_p64(a), a.size, q, int(inverse))
    return a


def ref_random_polynomial(n, q, seed=42):
    R = ref()
    out = np.zeros(n, dtype=np.uint64)
    R.ref_random_polynomial(_p64(out), n, q, seed)
    return out


def ref_host_batch(x, moduli, inverse=False, negacyclic=False, threads=0):
    """Reference ntt_host over a [poly][limb][n] batch on host threads (in place).
    Returns the thread count used."""
    R = ref()
    assert x.dtype == np.uint64 and x.flags.c_contiguous
    m = np.ascontiguousarray(moduli, dtype=np.uint64)
    n = x.shape[-1]
    n_polys = x.size // (n * m.size)
    return R.ref_ntt_host_batch(_p64(x), n, _p64(m), m.size, n_polys, int(inverse), int(negacyclic), threads)


def ref_klimb_case(K, log_n, seed=0xC0FFEE):
    R = ref()
    n = 1 << log_n
    inp = np.zeros(n * K, dtype=np.uint32)
    out = np.zeros(n * K, dtype=np.uint32)
    prime = np.zeros(K, dtype=np.uint32)
    omega = np.zeros(K, dtype=np.uint32)
    rc = R.ref_klimb_case(K, log_n, seed, _p32(inp), _p32(out), _p32(prime), _p32(omega))
    assert rc == 0
    return inp.reshape(n, K), out.reshape(n, K), prime, omega


def limbs_to_int(limbs, bits=24):
    return sum(int(v) << (bits * i) for i, v in enumerate(limbs))


def int_to_limbs(x, K, bits=24):
    return [(x >> (bits * i)) & ((1 << bits) - 1) for i in range(K)]


def host_ntt_naive(xs, omega, p):
    """Pure-Python restatement of host_ntt_naive (include/ntt_arbitrary.cuh:2651-2676):
    bit-reverse, then radix-2 DIT stages with twiddle tw[k * (n / m)], tw[i] = omega^i mod p.
    Exact for any omega (the K=2 field's omega is not a root of unity mod its truncated prime,
    so only this exact network reproduces the reference there).  Small n only."""
    a = [int(x) % p if False else int(x) for x in xs]
    n = len(a)
    lg = n.bit_length() - 1
    tw = [1] * n
    for i in range(1, n):
        tw[i] = tw[i - 1] * omega % p
    for i in range(n):
        j = int(format(i, "0%db" % lg)[::-1], 2) if lg else 0
        if i < j:
            a[i], a[j] = a[j], a[i]
    m = 2
    while m <= n:
        half = m // 2
        stride = n // m
        for g in range(0, n, m):
            for k in range(half):
                w = tw[(k * stride) % n]
                t = a[g + k + half] * w % p
                u = a[g + k]
                a[g + k] = (u + t) % p
                a[g + k + half] = (u - t) % p
        m *= 2
    return a
