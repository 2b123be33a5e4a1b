"""Generates tests/golden/*.npz from the reference's own CPU code.

Run in a container that has the reference tree (it builds oracle/_ref via
`make -C oracle`):  python tests/golden/make_golden.py

Fixtures (all uint64 unless noted):
  babybear_seed42.npz   reference random_polynomial(n, q, seed=42) inputs
                        (tests/test_ntt.cu:22-31) with ntt_host forward and
                        inverse outputs for n in 64..4096
  babybear_iplus1.npz   x[i] = i + 1 (tests/debug_inner.cu:17-20) forward
                        outputs for n in {64, 128, 4096}
  params.npz            create_params for several (q, n)
  q60.npz               60-bit prime q = 1152921504577486849, n = 1024,
                        ntt_host forward/inverse
  klimb.npz             K-limb (K = 2, 3, 11) natural-form inputs and
                        host_ntt_naive outputs (uint32 24-bit limbs),
                        include/ntt_arbitrary.cuh:2651-2730, seed 0xC0FFEE
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
from oracle import oracle as O  # noqa: E402

BABYBEAR = 2013265921
Q60 = 1152921504577486849


def main():
    assert O.ref() is not None, "oracle/_ref/libntt_ref.so missing (needs the reference tree)"
    out = {}
    for lg in (6, 8, 10, 12):
        n = 1 << lg
        x = O.ref_random_polynomial(n, BABYBEAR, 42)
        out["in_%d" % n] = x
        out["fwd_%d" % n] = O.ref_ntt_host(x, BABYBEAR, False)
        out["inv_%d" % n] = O.ref_ntt_host(x, BABYBEAR, True)
    np.savez_compressed(os.path.join(HERE, "babybear_seed42.npz"), **out)

    out = {}
    for n in (64, 128, 4096):
        x = np.arange(1, n + 1, dtype=np.uint64)
        out["fwd_%d" % n] = O.ref_ntt_host(x, BABYBEAR, False)
    np.savez_compressed(os.path.join(HERE, "babybear_iplus1.npz"), **out)

    cases = [(BABYBEAR, 1 << 16), (BABYBEAR, 64), (1073479681, 1 << 20), (1073610753, 1 << 10),
             (4293918721, 1 << 12), (Q60, 1 << 20), (2147352577, 1 << 17)]
    rows = np.array([O.ref_params(q, n) for q, n in cases], dtype=np.uint64)
    np.savez_compressed(os.path.join(HERE, "params.npz"), cases=np.array(cases, dtype=np.uint64), params=rows)

    n = 1024
    x = O.ref_random_polynomial(n, Q60, 7)
    np.savez_compressed(os.path.join(HERE, "q60.npz"), q=np.uint64(Q60), inp=x,
                        fwd=O.ref_ntt_host(x, Q60, False), inv=O.ref_ntt_host(x, Q60, True))

    out = {}
    for K, lg in ((2, 8), (3, 8), (11, 6)):
        inp, res, prime, omega = O.ref_klimb_case(K, lg, 0xC0FFEE)
        out["in_K%d" % K] = inp
        out["out_K%d" % K] = res
        out["prime_K%d" % K] = prime
        out["omega_K%d" % K] = omega
    np.savez_compressed(os.path.join(HERE, "klimb.npz"), **out)
    print("wrote fixtures to", HERE)


if __name__ == "__main__":
    main()
