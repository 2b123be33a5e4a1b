"""GPU parity of the K-limb forward NTT (nttb_klimb_forward, the engine behind
the ntt_arbitrary.cuh drop-in) against the reference's own outputs
(tests/golden/klimb.npz) and the host_ntt_naive network restated in Python,
for the reference's three fields K = 2, 3, 11.  Zero mismatches allowed."""
import numpy as np
import pytest

from conftest import golden, to_dev, to_host
from oracle import oracle as O
import ntt_b200 as nb

pytestmark = pytest.mark.gpu


def field(g, K):
    return O.limbs_to_int(g["prime_K%d" % K]), O.limbs_to_int(g["omega_K%d" % K])


def run_klimb(torch, K, xs, omega, p):
    """Natural-form ints in -> natural-form ints out through the device path
    (Montgomery form R = 2^(24 K) on the device; p is odd, so R is invertible)."""
    n = len(xs)
    log_n = n.bit_length() - 1
    R = 1 << (24 * K)
    tw, t = [], R % p
    for _ in range(n):
        tw.append(t)
        t = t * omega % p
    data = np.array([O.int_to_limbs(x * R % p, K) for x in xs], dtype=np.uint32).reshape(-1)
    twl = np.array([O.int_to_limbs(v, K) for v in tw], dtype=np.uint32).reshape(-1)
    d, dt = to_dev(torch, data), to_dev(torch, twl)
    limbs = O.int_to_limbs(p, K)
    nb.klimb_forward(K, d, dt, log_n, limbs, nb.klimb_neg_inv24(limbs[0]))
    torch.cuda.synchronize()
    out = to_host(d, np.uint32).reshape(n, K)
    rinv = pow(R, -1, p)
    return [O.limbs_to_int(row) * rinv % p for row in out]


@pytest.mark.parametrize("K", [2, 3, 11])
def test_klimb_vs_reference_fixture(torch_cuda, K):
    g = golden("klimb.npz")
    p, omega = field(g, K)
    xs = [O.limbs_to_int(r) for r in g["in_K%d" % K]]
    want = [O.limbs_to_int(r) for r in g["out_K%d" % K]]
    assert run_klimb(torch_cuda, K, xs, omega, p) == want


@pytest.mark.parametrize("K,log_n", [(2, 1), (2, 6), (2, 10), (2, 11), (2, 12), (3, 10), (3, 13), (11, 8),
                                     (11, 9), (11, 12)])
def test_klimb_vs_naive_network(torch_cuda, K, log_n):
    """Against the network: one fused tile (K <= 3 up to 2^10, K = 11 up to
    2^8) and the multi-pass sizes above, whose tiles shrink until a pass has
    enough CTAs."""
    g = golden("klimb.npz")
    # the fixture's omega as the twiddle base: the network is defined for
    # any omega (a DFT only when omega has order 2^log_n)
    p, omega = field(g, K)
    rng = np.random.default_rng(K * 100 + log_n)
    xs = [int(v) % p for v in rng.integers(0, 2 ** 62, 1 << log_n, dtype=np.uint64)]
    got = run_klimb(torch_cuda, K, xs, omega, p)
    assert got == O.host_ntt_naive(xs, omega, p)


def test_klimb_goldilocks_2_20_spot(torch_cuda):
    """N = 2^20 Goldilocks (K = 3): three device passes; a true DFT there, so
    check X[k] = sum_i x_i omega^(i k) at a few k."""
    p = 0xFFFFFFFF00000001
    w24 = 0x86cdcc31c307e171
    omega = pow(w24, 1 << 4, p)  # 2^20-th root
    n = 1 << 20
    rng = np.random.default_rng(20)
    xs = [int(v) % p for v in rng.integers(0, 2 ** 63, n, dtype=np.uint64)]
    got = run_klimb(torch_cuda, 3, xs, omega, p)
    for k in (0, 1, 12345, n - 1):
        wk = pow(omega, k, p)
        acc, t = 0, 1
        for x in xs:
            acc += x * t
            t = t * wk % p
        assert got[k] == acc % p


def test_klimb_rejects_bad_arguments(torch_cuda):
    d = torch_cuda.zeros(64 * 3, dtype=torch_cuda.int32, device="cuda")
    with pytest.raises(nb.NTTError):
        nb.klimb_forward(5, d, d, 6, [1] * 5, 0)  # K outside {2, 3, 11}
    with pytest.raises(nb.NTTError):
        nb.klimb_forward(3, d, d, 6, [1, 0, 0], 12345)  # wrong np
