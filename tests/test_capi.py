"""CPU: the C-ABI library loads, exports every declared symbol, and its host
math matches the oracle.  No device work is issued here."""
import ctypes
import os
import subprocess

import numpy as np
import pytest

from conftest import BABYBEAR, Q60, ROOT
from oracle import oracle as O
import ntt_b200 as nb


def test_library_exports_every_header_symbol():
    L = nb.lib()
    syms = nb.header_symbols()
    assert len(syms) >= 24
    missing = [s for s in syms if not hasattr(L, s)]
    assert not missing, missing


def test_debug_bounds_library_exports_every_header_symbol():
    """The NTT_DEBUG_BOUNDS build exports the same C ABI; the release build
    reports its range checks as compiled away."""
    dbg = os.path.join(os.path.dirname(nb.LIB_PATH), "libntt_b200_dbg.so")
    assert os.path.exists(dbg), "run `python ntt-tensorcore_b200/build.py --debug-bounds`"
    D = ctypes.CDLL(dbg)
    missing = [s for s in nb.header_symbols() if not hasattr(D, s)]
    assert not missing, missing
    out = subprocess.run(["nm", "-D", "--defined-only", dbg], capture_output=True, text=True).stdout
    assert "g_tc_bounds" not in out  # device words stay internal
    f, e = ctypes.c_uint32(7), ctypes.c_int(7)
    assert nb.lib().nttb_bounds_errors(None, None, 0) == 1
    import torch
    if not torch.cuda.is_available():  # the symbol lookups need a device; the flag does not
        return
    assert nb.lib().nttb_bounds_errors(ctypes.byref(f), ctypes.byref(e), 0) == 0 and e.value == 0


def test_phase_profile_library_exports_every_header_symbol():
    """The NTT_PHASE_PROFILE build exports the same C ABI; null arguments are
    refused in both builds without touching a device."""
    ph = os.path.join(os.path.dirname(nb.LIB_PATH), "libntt_b200_phase.so")
    assert os.path.exists(ph), "run `python ntt-tensorcore_b200/build.py --phase-profile`"
    P = ctypes.CDLL(ph)
    missing = [s for s in nb.header_symbols() if not hasattr(P, s)]
    assert not missing, missing
    P.nttb_phase_profile.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int]
    assert P.nttb_phase_profile(None, None, 0) == 1
    assert nb.lib().nttb_phase_profile(None, None, 0) == 1


def test_library_exports_dropin_cpp_api():
    out = subprocess.run(["nm", "-DC", "--defined-only", nb.LIB_PATH], capture_output=True, text=True).stdout
    for name in ["ntt::ntt_init", "ntt::ntt_cleanup", "ntt::ntt_forward_basic", "ntt::ntt_inverse_basic",
                 "ntt::ntt_forward_four_step", "ntt::ntt_inverse_four_step", "ntt::ntt_forward_tlmop",
                 "ntt::ntt_inverse_tlmop", "ntt::ntt_forward_optimized", "ntt::ntt_inverse_optimized",
                 "ntt::ntt_forward_rowmaj", "ntt::rowmaj_to_pretransposed", "ntt::rowmaj_from_pretransposed",
                 "ntt::ntt_forward_batch", "ntt::ntt_inverse_batch", "ntt::poly_multiply_ntt",
                 "ntt::bit_reverse_permute", "ntt::ntt_host"]:
        assert name + "(" in out, name


def test_version_and_status_strings():
    assert "sm_100a" in nb.version()
    assert nb.lib().nttb_status_string(0) == b"ok"


@pytest.mark.parametrize("q,n", [(BABYBEAR, 1 << 16), (BABYBEAR, 2), (1073479681, 1 << 20), (Q60, 1 << 20),
                                 (4293918721, 1 << 12), (2147352577, 1 << 17)])
def test_create_params_matches_oracle(q, n):
    keys = ["q", "q_twice", "barrett_k", "barrett_m", "omega", "omega_inv", "n_inv"]
    assert nb.create_params(q, n) == dict(zip(keys, O.params(q, n)))
    assert nb.find_primitive_root(q, n) == O.primitive_root(q, n)


def test_psi_squares_to_omega():
    for q in (BABYBEAR, 2147352577, Q60):
        n = 1 << 12
        psi = nb.find_psi(q, n)
        assert psi == O.psi(q, n)
        assert pow(psi, 2, q) == nb.find_primitive_root(q, n)
        assert pow(psi, n, q) == q - 1


@pytest.mark.parametrize("lg", [0, 1, 2, 6, 10, 12])
def test_host_ntt_matches_oracle(lg):
    rng = np.random.default_rng(lg)
    for q in (BABYBEAR, Q60):
        x = rng.integers(0, q, 1 << lg, dtype=np.uint64)
        for inv in (False, True):
            y = x.copy()
            nb.host_ntt(y, q, inv)
            assert (y == O.ntt(x, q, inv)).all()


def test_generate_primes():
    ps = nb.generate_primes(31, 17, 24)
    assert len(set(ps)) == 24 and all(p < 2 ** 31 and (p - 1) % (1 << 17) == 0 for p in ps)
    assert ps == sorted(ps, reverse=True)
    for p in ps[:4]:
        assert pow(3, p - 1, p) == 1


def test_invalid_arguments_rejected_without_device():
    h = ctypes.c_void_p()
    L = nb.lib()
    assert L.nttb_plan_create(1000, BABYBEAR, ctypes.byref(h)) == 1      # not a power of two
    assert b"power of two" in L.nttb_last_error()
    assert L.nttb_plan_create(1 << 10, 1 << 62, ctypes.byref(h)) == 2    # modulus too wide
    assert L.nttb_rns_plan_create(30, None, 0, 0, ctypes.byref(h)) == 1  # no moduli
    assert L.nttb_u64_transform(None, None, 1, 0, 0, None) == 1
    assert L.nttb_rns_transform(None, None, None, 1, 0, 0, None) == 1
    rid = ctypes.c_uint64()
    assert L.nttb_u64_pretransposed_transform(None, None, 64, 0, None) == 1
    assert L.nttb_server_submit_ntt(None, None, None, 10, 1, 0, 0, ctypes.byref(rid)) == 1
    assert L.nttb_server_submit_device(None, 0, None, None, None, 10, 1, 0, ctypes.byref(rid)) == 1
    assert b"null" in L.nttb_last_error()
    assert L.nttb_u64_transpose(None, None, 32, 32, None) == 1
    assert L.nttb_u64_bit_reverse(None, 1024, None) == 1
    p = (ctypes.c_uint32 * 5)(*([1] * 5))
    buf = ctypes.c_void_p(16)  # never dereferenced: K = 5 is refused first
    assert L.nttb_klimb_forward(5, buf, buf, 1 << 10, 10, p, 1, None) == 2  # K not served
    assert b"K = 5" in L.nttb_last_error()


def test_dropin_headers_compile_reference_test_programs(tmp_path):
    """The reference's own test sources compile against include/ntt.cuh (drop-in)."""
    # the reference checkout: $REF, else where the oracle build found it
    root = os.environ.get("REF", "")
    rec = os.path.join(ROOT, "oracle", "_ref", "ref_root.txt")
    if not root and os.path.exists(rec):
        root = open(rec).read().strip()
    ref = os.path.join(root, "tests", "test_ntt.cu")
    if not root or not os.path.exists(ref):
        pytest.skip("reference tree not present")
    out = str(tmp_path / "dropin_compile_check.o")
    r = subprocess.run(["/usr/local/cuda/bin/nvcc", "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a",
                        "-I" + os.path.join(ROOT, "include"), "-c", ref, "-o", out],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


def test_harness_program_compiles_against_dropin_headers(tmp_path):
    """oracle/harness_compare.cu needs only the drop-in's include/ntt.cuh."""
    src = os.path.join(ROOT, "oracle", "harness_compare.cu")
    out = str(tmp_path / "harness_compile_check.o")
    r = subprocess.run(["/usr/local/cuda/bin/nvcc", "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a",
                        "-I" + os.path.join(ROOT, "include"), "-c", src, "-o", out],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


def test_device_paths_fail_loudly_without_a_gpu():
    """With no usable CUDA device the product path raises: plans need device
    memory and there is no host fallback for any transform."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is visible")
    qs = nb.generate_primes(31, 17, 2)
    with pytest.raises(nb.NTTError):
        nb.RnsPlan(16, qs, negacyclic=True)
    with pytest.raises(nb.NTTError):
        nb.Plan(1 << 12, BABYBEAR)
