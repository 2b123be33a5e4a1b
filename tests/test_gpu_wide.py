"""GPU: the INT8 byte-plane engine for 64-bit moduli (tc_wide.cu) -- the
60-bit prime at n = 2^20 and other wide moduli -- against the oracle, the
reference's own ntt_host (oracle/_ref) and the CUDA-core Montgomery-64
engine, bit for bit."""
import numpy as np
import pytest

from conftest import Q60, to_dev, to_host
from oracle import oracle as O
import ntt_b200 as nb

pytestmark = pytest.mark.gpu

LG = 20
N = 1 << LG


def rand(q, count, seed):
    return np.random.default_rng(seed).integers(0, q, (count, N), dtype=np.uint64)


@pytest.mark.parametrize("inverse", [False, True])
def test_int8_wide_q60_vs_oracle_and_reference(torch_cuda, inverse):
    x = rand(Q60, 1, 60 + inverse)[0]
    plan = nb.WidePlan(LG, [Q60])
    d = to_dev(torch_cuda, x)
    out = torch_cuda.empty_like(d)
    plan.transform(out, d, 1, inverse=inverse, engine="int8")
    torch_cuda.cuda.synchronize()
    got = to_host(out, np.uint64)
    assert (got == O.ntt(x, Q60, inverse=inverse)).all()
    if O.ref() is not None:  # the reference's CPU NTT (unsigned __int128), compiled from its sources
        assert (got == O.ref_ntt_host(x, Q60, inverse=inverse)).all()
    assert (to_host(d, np.uint64) == x).all()  # out of place: the input is left alone
    assert nb.device_errors() == 0


def test_int8_wide_matches_scalar_on_batches(torch_cuda):
    """Three polynomials x three moduli (two near 2^62, a 60-bit and a
    33-bit one), both directions, in place, against the CUDA-core engine."""
    qs = nb.generate_primes(62, 21, 2) + [Q60] + nb.generate_primes(33, 21, 1)
    plan = nb.WidePlan(LG, qs)
    x = np.stack([rand(q, 3, 7 + i) for i, q in enumerate(qs)], axis=1)  # [poly][limb][n]
    for inverse in (False, True):
        a, b = to_dev(torch_cuda, x.reshape(-1)), to_dev(torch_cuda, x.reshape(-1))
        plan.transform(a, a, 3, inverse=inverse, engine="int8")
        plan.transform(b, b, 3, inverse=inverse, engine="scalar")
        torch_cuda.cuda.synchronize()
        assert torch_cuda.equal(a, b), inverse
        got = to_host(a, np.uint64).reshape(x.shape)
        for l, q in ((0, qs[0]), (3, qs[3])):
            assert (got[1, l] == O.ntt(x[1, l], q, inverse=inverse)).all()
    assert nb.device_errors() == 0


def test_int8_wide_round_trip_and_extreme_residues(torch_cuda):
    """inverse(forward(x)) == x, with rows of q - 1 (every byte plane near
    its maximum), zeros and ones beside random rows."""
    q = Q60
    x = rand(q, 4, 3)
    x[0] = q - 1
    x[1] = 0
    x[2] = 1
    plan = nb.WidePlan(LG, [q])
    d = to_dev(torch_cuda, x.reshape(-1))
    plan.transform(d, d, 4, engine="int8")
    torch_cuda.cuda.synchronize()
    f = to_host(d, np.uint64).reshape(x.shape)
    for r in range(3):
        assert (f[r] == O.ntt(x[r], q)).all(), r
    plan.transform(d, d, 4, inverse=True, engine="int8")
    torch_cuda.cuda.synchronize()
    assert (to_host(d, np.uint64).reshape(x.shape) == x).all()


def test_dropin_u64_transform_runs_the_wide_engine(torch_cuda):
    """The drop-in single-modulus plan (NTTConfig) with the 60-bit prime at
    2^20: AUTO takes the INT8 engine and gives the oracle's transform."""
    x = rand(Q60, 1, 11)[0]
    plan = nb.Plan(N, Q60)
    d = to_dev(torch_cuda, x)
    nb.profile_start()
    plan.transform(d)
    prof = nb.profile_stop()
    torch_cuda.cuda.synchronize()
    assert (to_host(d, np.uint64) == O.ntt(x, Q60)).all()
    assert "wide_pass_a" in prof and "wide_pass_b" in prof


def test_int8_wide_refuses_what_it_does_not_serve(torch_cuda):
    nega = nb.WidePlan(LG, [Q60], negacyclic=True)
    small = nb.WidePlan(18, [Q60])
    d = to_dev(torch_cuda, rand(Q60, 1, 1)[0])
    for plan in (nega, small):
        with pytest.raises(nb.NTTError) as e:
            plan.transform(d, d, 1, engine="int8")
        assert e.value.status == nb.ERR_UNSUPPORTED
    x = rand(Q60, 1, 2)[0][: 1 << 18]
    s = to_dev(torch_cuda, x)
    small.transform(s, s, 1)  # AUTO: the CUDA-core engine
    torch_cuda.cuda.synchronize()
    assert (to_host(s, np.uint64) == O.ntt(x, Q60)).all()
