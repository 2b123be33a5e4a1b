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
