"""CPU: the oracle pinned against the reference's own CPU code and fixtures."""
import numpy as np
import pytest

from conftest import BABYBEAR, Q60, golden
from oracle import oracle as O

HAVE_REF = O.ref() is not None


def test_params_fixture():
    g = golden("params.npz")
    for (q, n), row in zip(g["cases"], g["params"]):
        assert O.params(int(q), int(n)) == [int(x) for x in row[:7]]
        assert O.lib().oracle_mu(int(q)) == int(row[7])


def test_known_answers():
    # values recorded from the reference's create_params (BabyBear, 2^16) and the 60-bit prime
    assert O.generator(BABYBEAR) == 31
    assert O.primitive_root(BABYBEAR, 1 << 16) == 1421947380
    assert O.params(BABYBEAR, 1 << 16)[6] == 2013235201
    assert O.primitive_root(Q60, 1 << 20) == 459211391583378785


@pytest.mark.parametrize("n", [64, 256, 1024, 4096])
def test_ntt_host_fixture(n):
    g = golden("babybear_seed42.npz")
    x = g["in_%d" % n]
    assert (O.ntt(x, BABYBEAR) == g["fwd_%d" % n]).all()
    assert (O.ntt(x, BABYBEAR, True) == g["inv_%d" % n]).all()


@pytest.mark.parametrize("n", [64, 128, 4096])
def test_iplus1_fixture(n):
    g = golden("babybear_iplus1.npz")
    x = np.arange(1, n + 1, dtype=np.uint64)
    assert (O.ntt(x, BABYBEAR) == g["fwd_%d" % n]).all()


def test_q60_fixture():
    g = golden("q60.npz")
    q = int(g["q"])
    assert (O.ntt(g["inp"], q) == g["fwd"]).all()
    assert (O.ntt(g["inp"], q, True) == g["inv"]).all()


def test_negacyclic_vs_schoolbook():
    rng = np.random.default_rng(3)
    for q in (BABYBEAR, 2147352577):
        for n in (2, 16, 128):
            a = rng.integers(0, q, n, dtype=np.uint64)
            b = rng.integers(0, q, n, dtype=np.uint64)
            c = O.negacyclic(O.pointwise(O.negacyclic(a, q), O.negacyclic(b, q), q), q, True)
            assert (c == O.polymul_negacyclic(a, b, q)).all()


def test_four_step_roundtrip_and_shape():
    rng = np.random.default_rng(5)
    for n in (4096, 8192, 16384):
        x = rng.integers(0, BABYBEAR, n, dtype=np.uint64)
        y = O.four_step(x, BABYBEAR)
        assert (O.four_step(y, BABYBEAR, True) == x).all()
    # the reference's four-step map is not the DFT (its row step runs over the transposed axis)
    x = rng.integers(0, BABYBEAR, 4096, dtype=np.uint64)
    assert not (O.four_step(x, BABYBEAR) == O.ntt(x, BABYBEAR)).all()


def test_rowmaj_is_pretransposed_dft():
    rng = np.random.default_rng(6)
    x = rng.integers(0, BABYBEAR, 4096, dtype=np.uint64)
    pre = O.to_pretransposed(x, 64, 64)
    assert (O.from_pretransposed(O.rowmaj_forward(pre, BABYBEAR), 64, 64) == O.ntt(x, BABYBEAR)).all()


@pytest.mark.skipif(not HAVE_REF, reason="reference library not built")
def test_oracle_vs_reference_cpu_random():
    rng = np.random.default_rng(11)
    for q in (BABYBEAR, 1073479681, 4293918721, Q60):
        for lg in (1, 3, 9, 11):
            x = rng.integers(0, q, 1 << lg, dtype=np.uint64)
            for inv in (False, True):
                assert (O.ntt(x, q, inv) == O.ref_ntt_host(x, q, inv)).all()


@pytest.mark.skipif(not HAVE_REF, reason="reference library not built")
def test_oracle_vs_reference_cpu_smallest_sizes():
    """n = 1, 2, 4: the reference's ntt_host (src/ntt_basic.cu:412-463) and the
    restatement agree at the edge of the size range, including n = 1
    (omega = 1, identity forward and inverse)."""
    rng = np.random.default_rng(13)
    for q in (BABYBEAR, Q60):
        for lg in (0, 1, 2):
            x = rng.integers(0, q, 1 << lg, dtype=np.uint64)
            for inv in (False, True):
                assert (O.ntt(x, q, inv) == O.ref_ntt_host(x, q, inv)).all()
        x = rng.integers(0, q, 1, dtype=np.uint64)
        assert (O.ntt(x, q, False) == x).all() and (O.ntt(x, q, True) == x).all()


@pytest.mark.skipif(not HAVE_REF, reason="reference library not built")
def test_reference_batch_driver_negacyclic():
    rng = np.random.default_rng(12)
    from conftest import GOLDEN  # noqa: F401
    moduli = [2147352577, 2146959361, 2146041857]
    x = np.stack([rng.integers(0, q, 256, dtype=np.uint64) for q in moduli])
    y = x.copy()
    O.ref_host_batch(y, moduli, inverse=False, negacyclic=True, threads=2)
    assert (y == O.rns(x, moduli, negacyclic=True)).all()
    O.ref_host_batch(y, moduli, inverse=True, negacyclic=True, threads=2)
    assert (y == x).all()


def test_klimb_fixture_matches_naive_network():
    """The K-limb fixtures equal the restated host_ntt_naive network for every K."""
    g = golden("klimb.npz")
    for K in (2, 3, 11):
        inp, out = g["in_K%d" % K], g["out_K%d" % K]
        p = O.limbs_to_int(g["prime_K%d" % K])
        w = O.limbs_to_int(g["omega_K%d" % K])
        ys = O.host_ntt_naive([O.limbs_to_int(r) for r in inp], w, p)
        assert ys == [O.limbs_to_int(r) for r in out]


def test_klimb_fixture_is_dft_for_true_roots():
    """K=3 (Goldilocks) and K=11 (BN254): host_ntt_naive is the DFT with omega_n.
    K=2: the reference packs its 49-bit prime into 2 x 24-bit limbs, which truncates it to
    92 * 2^24 + 1; omega is then not a root of unity and the network is not a DFT."""
    g = golden("klimb.npz")
    assert O.limbs_to_int(g["prime_K2"]) == 92 * 2 ** 24 + 1
    for K in (3, 11):
        inp, out = g["in_K%d" % K], g["out_K%d" % K]
        p = O.limbs_to_int(g["prime_K%d" % K])
        w = O.limbs_to_int(g["omega_K%d" % K])
        n = inp.shape[0]
        xs = [O.limbs_to_int(r) for r in inp]
        ys = [O.limbs_to_int(r) for r in out]
        for k in (0, 1, n // 2 + 3, n - 1):
            wk = pow(w, k, p)
            acc, t = 0, 1
            for j in range(n):
                acc = (acc + xs[j] * t) % p
                t = t * wk % p
            assert acc == ys[k]
