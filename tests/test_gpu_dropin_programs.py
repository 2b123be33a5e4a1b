"""GPU: the reference's own test programs, compiled unmodified against the
drop-in headers (include/ntt.cuh) and linked with libntt_b200.so, pass.
Built by `make -C oracle dropin` (needs the reference tree at build time)."""
import os
import subprocess

import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu

BIN = os.path.join(ROOT, "oracle", "_ref")


def run(name, timeout=600):
    path = os.path.join(BIN, "dropin_" + name)
    if not os.path.exists(path):
        pytest.skip("drop-in program %s not built" % name)
    r = subprocess.run([path], capture_output=True, text=True, timeout=timeout)
    return r.returncode, r.stdout + r.stderr


def test_reference_test_ntt_suite():
    rc, out = run("test_ntt")
    assert rc == 0, out[-3000:]
    assert "Passed: 25 / 25" in out, out[-3000:]


def test_reference_test_inner_ntt():
    rc, out = run("test_inner_ntt")
    assert rc == 0, out[-2000:]
    assert "Forward NTT: PASSED" in out and "Roundtrip: PASSED" in out


def test_reference_debug_inner():
    rc, out = run("debug_inner")
    assert rc == 0, out[-2000:]
    for n in (64, 128, 4096):
        assert "Direct matches: %d / %d" % (n, n) in out, out[-2000:]


def test_reference_debug_rowmaj():
    rc, out = run("debug_rowmaj")
    assert rc == 0, out[-2000:]
    assert "Optimized vs host: 4096 / 4096  PASS" in out
    assert "RowMaj    vs host: 4096 / 4096  PASS" in out


def test_reference_ntt_mma_arbitrary_driver():
    """src/ntt_mma_arbitrary.cu (the K-limb driver) against ntt_arbitrary.cuh:
    Montgomery self tests for K = 2, 3, 11 and the forward NTT checked against
    host_ntt_naive at every size of its default sweep."""
    rc, out = run("ntt_mma_arbitrary", timeout=1200)
    assert rc == 0, out[-3000:]
    assert out.count("mont round-trip + mult OK") == 3, out[-3000:]
    assert out.count("device mont_mul == host mont_mul OK") == 3, out[-3000:]
    assert out.count("0 mismatches  OK") == 3, out[-3000:]
    assert out.count("CORRECT (matches host reference") == 7, out[-3000:]
    assert "MISMATCH" not in out and "FAIL" not in out, out[-3000:]


def test_reference_timing_compare_runs():
    """tests/timing_compare.cu builds against the drop-in (including its direct
    launches of bitrev_kernel_d / ct_stage_kernel) and runs its K = 2 and
    K = 11 sweeps to completion."""
    path = os.path.join(BIN, "dropin_timing_compare")
    if not os.path.exists(path):
        pytest.skip("drop-in program timing_compare not built")
    r = subprocess.run([path, "6", "8", "10", "12"], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, (r.stdout + r.stderr)[-3000:]
    assert "LEGEND" in r.stdout


def test_icicle_harness_forward_matches_host():
    """oracle/harness_compare.cu (the timing convention of the reference's
    tests/icicle_compare.cu) on the drop-in: every timed size's forward equals
    ntt_host on the same seeded input."""
    rc, out = run("harness")
    assert rc == 0, out[-2000:]
    assert out.count("equal") == 7 and "DIFFERENT" not in out, out[-2000:]
