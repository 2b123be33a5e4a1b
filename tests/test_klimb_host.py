"""The K-limb drop-in header's host arithmetic (include/ntt_arbitrary.cuh)
against the reference: FieldConfig moduli / roots, Montgomery round trips,
and host_ntt_naive on the reference-generated K-limb fixture
(tests/golden/klimb.npz, made by the reference's own host_ntt_naive).
Host-only: the helper is compiled with nvcc and runs without a GPU."""
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT, golden

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")


@pytest.fixture(scope="module")
def helper(tmp_path_factory):
    if not os.path.exists(NVCC):
        pytest.skip("nvcc not available")
    exe = str(tmp_path_factory.mktemp("klimb") / "klimb_host_check")
    subprocess.run([NVCC, "-O1", "-std=c++17", "-w", "-I" + os.path.join(ROOT, "include"),
                    "-o", exe, os.path.join(ROOT, "tests", "native", "klimb_host_check.cu")],
                   check=True, capture_output=True)
    return exe


@pytest.mark.parametrize("K", [2, 3, 11])
def test_header_host_ntt_matches_reference_fixture(helper, K):
    g = golden("klimb.npz")
    inp, out = g["in_K%d" % K], g["out_K%d" % K]
    n = inp.shape[0]
    log_n = n.bit_length() - 1
    text = "%d %d\n" % (K, log_n) + " ".join(str(int(v)) for v in inp.reshape(-1))
    r = subprocess.run([helper], input=text, capture_output=True, text=True, check=True)
    lines = dict(l.split(" ", 1) for l in r.stdout.strip().splitlines())
    assert [int(v) for v in lines["prime"].split()] == [int(v) for v in g["prime_K%d" % K]]
    assert [int(v) for v in lines["omega"].split()] == [int(v) for v in g["omega_K%d" % K]]
    assert lines["mont_ok"].strip() == "1"
    got = np.array([int(v) for v in lines["out"].split()], dtype=np.uint64).reshape(n, K)
    assert (got == out.astype(np.uint64)).all()
