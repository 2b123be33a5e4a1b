"""GPU parity of the batched RNS path (uint32 residues, many moduli, cyclic and
negacyclic) for every engine, against the oracle.  Zero mismatches allowed."""
import numpy as np
import pytest

from conftest import to_dev, to_host
from oracle import oracle as O
import ntt_b200 as nb

pytestmark = pytest.mark.gpu

PRIMES17 = nb.generate_primes(31, 17, 24)  # q == 1 mod 2^17 (config: 24 limbs, N = 2^16 negacyclic)
PRIMES21 = nb.generate_primes(31, 21, 8)


def engines():
    return ["scalar", "int8", "dmma", "tiles", "auto"]


def serves(engine, lg):
    """The INT8 cluster and DMMA engines serve N = 2^16, the batch queue's
    tensor tiles 2^13 .. 2^20; AUTO falls back elsewhere."""
    if engine == "tiles":
        return 13 <= lg <= 20
    return engine not in ("int8", "dmma") or lg == 16


def rand_batch(n_polys, moduli, n, seed):
    rng = np.random.default_rng(seed)
    x = np.empty((n_polys, len(moduli), n), dtype=np.uint32)
    for l, q in enumerate(moduli):
        x[:, l, :] = rng.integers(0, q, (n_polys, n), dtype=np.uint64).astype(np.uint32)
    return x


def run(torch, plan, x, inverse, engine, out_of_place=False):
    d = to_dev(torch, x.reshape(-1))
    dst = torch.empty_like(d) if out_of_place else d
    plan.transform(dst, d, x.shape[0], inverse=inverse, engine=engine)
    torch.cuda.synchronize()
    return to_host(dst, np.uint32).reshape(x.shape)


@pytest.mark.parametrize("engine,lg", [(e, lg) for e in engines() for lg in (1, 4, 6, 10, 12, 13, 16, 17, 18, 20)
                                       if serves(e, lg) and (lg < 18 or e in ("tiles", "auto"))])
@pytest.mark.parametrize("negacyclic", [False, True])
def test_rns_vs_oracle(torch_cuda, engine, negacyclic, lg):
    moduli = nb.generate_primes(31, max(17, lg + 1), 3)
    x = rand_batch(2, moduli, 1 << lg, lg)
    plan = nb.RnsPlan(lg, moduli, negacyclic=negacyclic)
    y = run(torch_cuda, plan, x, False, engine)
    ref = O.rns(x.astype(np.uint64), moduli, negacyclic=negacyclic)
    assert (y.astype(np.uint64) == ref).all(), int((y.astype(np.uint64) != ref).sum())
    z = run(torch_cuda, plan, y, True, engine, out_of_place=True)
    assert (z == x).all()
    refi = O.rns(x.astype(np.uint64), moduli, negacyclic=negacyclic, inverse=True)
    assert (run(torch_cuda, plan, x, True, engine).astype(np.uint64) == refi).all()
    assert nb.device_errors() == 0


@pytest.mark.parametrize("engine", engines())
def test_config_rns_negacyclic_full_size(torch_cuda, engine):
    """24 limbs x 2^16 negacyclic: every limb of the forward checked against the
    oracle, and the whole batch's round trip exact."""
    lg = 16
    x = rand_batch(1, PRIMES17, 1 << lg, 2024)
    plan = nb.RnsPlan(lg, PRIMES17, negacyclic=True)
    y = run(torch_cuda, plan, x, False, engine)
    ref = O.rns(x.astype(np.uint64), PRIMES17, negacyclic=True)
    assert (y.astype(np.uint64) == ref).all(), [l for l in range(24) if (y[0, l] != ref[0, l]).any()]
    z = run(torch_cuda, plan, y, True, engine)
    assert (z == x).all()


@pytest.mark.parametrize("engine", engines())
@pytest.mark.parametrize("n_polys", [1, 3])
def test_forward_inverse_one_call(torch_cuda, engine, n_polys):
    """nttb_rns_forward_inverse (one persistent launch on the INT8 engine):
    exact round trip over several polynomials, and the forward half equals a
    separate forward transform (checked through a second buffer)."""
    lg = 16
    x = rand_batch(n_polys, PRIMES17[:5], 1 << lg, 40 + n_polys)
    plan = nb.RnsPlan(lg, PRIMES17[:5], negacyclic=True)
    d = to_dev(torch_cuda, x.reshape(-1))
    plan.forward_inverse(d, n_polys, engine=engine)
    torch_cuda.cuda.synchronize()
    assert (to_host(d, np.uint32).reshape(x.shape) == x).all()
    assert nb.device_errors() == 0
    y = run(torch_cuda, plan, x, False, engine)
    ref = O.rns(x.astype(np.uint64), PRIMES17[:5], negacyclic=True)
    assert (y.astype(np.uint64) == ref).all()


@pytest.mark.parametrize("engine", ["int8", "dmma"])
def test_many_units_per_launch(torch_cuda, engine):
    """3 polynomials x 24 limbs = 72 (poly, limb) units: more units than the
    INT8 engine runs at once, so its persistent clusters each take several
    units in turn.  Every limb of every polynomial is checked."""
    lg, n_polys = 16, 3
    x = rand_batch(n_polys, PRIMES17, 1 << lg, 72)
    plan = nb.RnsPlan(lg, PRIMES17, negacyclic=True)
    y = run(torch_cuda, plan, x, False, engine, out_of_place=True)
    ref = O.rns(x.astype(np.uint64), PRIMES17, negacyclic=True)
    assert (y.astype(np.uint64) == ref).all(), int((y.astype(np.uint64) != ref).sum())
    d = to_dev(torch_cuda, x.reshape(-1))
    plan.forward_inverse(d, n_polys, engine=engine)
    torch_cuda.cuda.synchronize()
    assert (to_host(d, np.uint32).reshape(x.shape) == x).all()
    assert nb.device_errors() == 0


@pytest.mark.parametrize("engine", ["scalar", "auto"])
def test_large_n_roundtrip_and_spotcheck(torch_cuda, engine):
    lg = 20
    moduli = PRIMES21[:2]
    x = rand_batch(1, moduli, 1 << lg, 77)
    plan = nb.RnsPlan(lg, moduli, negacyclic=False)
    y = run(torch_cuda, plan, x, False, engine)
    assert (y[0, 1].astype(np.uint64) == O.ntt(x[0, 1].astype(np.uint64), moduli[1])).all()
    assert (run(torch_cuda, plan, y, True, engine) == x).all()


def test_edge_values(torch_cuda):
    """All-zero, all-(q-1) and one-hot inputs."""
    lg, moduli = 12, PRIMES17[:2]
    n = 1 << lg
    plan = nb.RnsPlan(lg, moduli, negacyclic=True)
    cases = [np.zeros((1, 2, n), np.uint32),
             np.stack([np.full(n, q - 1, np.uint32) for q in moduli])[None],
             np.zeros((1, 2, n), np.uint32)]
    cases[2][0, :, 5] = 1
    for x in cases:
        y = run(torch_cuda, plan, x, False, "auto")
        assert (y.astype(np.uint64) == O.rns(x.astype(np.uint64), moduli, negacyclic=True)).all()


def test_negacyclic_polymul_vs_schoolbook(torch_cuda):
    lg, moduli = 8, PRIMES17[:2]
    n = 1 << lg
    a, b = rand_batch(1, moduli, n, 1), rand_batch(1, moduli, n, 2)
    plan = nb.RnsPlan(lg, moduli, negacyclic=True)
    da, db = to_dev(torch_cuda, a.reshape(-1)), to_dev(torch_cuda, b.reshape(-1))
    plan.transform(da, da, 1)
    plan.transform(db, db, 1)
    out = torch_cuda.empty_like(da)
    plan.pointwise_mul(out, da, db, 1)
    plan.transform(out, out, 1, inverse=True)
    torch_cuda.cuda.synchronize()
    got = to_host(out, np.uint32).reshape(1, 2, n)
    for l, q in enumerate(moduli):
        ref = O.polymul_negacyclic(a[0, l].astype(np.uint64), b[0, l].astype(np.uint64), q)
        assert (got[0, l].astype(np.uint64) == ref).all()


def test_wide_plan_q60(torch_cuda):
    from conftest import Q60
    lg = 20
    x = np.random.default_rng(60).integers(0, Q60, 1 << lg, dtype=np.uint64)
    plan = nb.WidePlan(lg, [Q60])
    d = to_dev(torch_cuda, x)
    plan.transform(d, d, 1)
    torch_cuda.cuda.synchronize()
    y = to_host(d, np.uint64)
    assert (y == O.ntt(x, Q60)).all()
    plan.transform(d, d, 1, inverse=True)
    torch_cuda.cuda.synchronize()
    assert (to_host(d, np.uint64) == x).all()


def test_launch_accounting(torch_cuda):
    lg, moduli = 16, PRIMES17[:4]
    plan = nb.RnsPlan(lg, moduli, negacyclic=True)
    x = rand_batch(1, moduli, 1 << lg, 3)
    d = to_dev(torch_cuda, x.reshape(-1))
    c0 = nb.launch_count()
    nb.profile_start()
    plan.transform(d, d, 1)
    prof = nb.profile_stop()
    assert nb.launch_count() > c0
    assert sum(v[0] for v in prof.values()) == nb.launch_count() - c0
    assert all(v[1] > 0 for v in prof.values())


@pytest.mark.parametrize("lg,polys,offset", [(10, 5, 0), (10, 3, 1), (1, 4, 0), (12, 2, 3)])
def test_pointwise_mul_rows_and_alignment(torch_cuda, lg, polys, offset):
    """The pointwise product row by row (row r mod limb r % n_limbs) against
    numpy, on 16-byte aligned arrays (four residues per access) and on arrays
    offset by a few words (one residue per access)."""
    moduli = PRIMES17[:3]
    n = 1 << lg
    plan = nb.RnsPlan(lg, moduli, negacyclic=False)
    a, b = rand_batch(polys, moduli, n, 5), rand_batch(polys, moduli, n, 6)
    words = polys * len(moduli) * n
    big = torch_cuda.zeros(3 * (words + 8), dtype=torch_cuda.int32, device="cuda")
    da = big[offset:offset + words]
    db = big[words + 8 + offset:2 * words + 8 + offset]
    out = big[2 * words + 16 + offset:3 * words + 16 + offset]
    da.copy_(to_dev(torch_cuda, a.reshape(-1)))
    db.copy_(to_dev(torch_cuda, b.reshape(-1)))
    plan.pointwise_mul(out, da, db, polys)
    torch_cuda.cuda.synchronize()
    got = to_host(out, np.uint32).reshape(polys, len(moduli), n).astype(np.uint64)
    q = np.array(moduli, dtype=np.uint64)[None, :, None]
    want = (a.astype(np.uint64) * b.astype(np.uint64)) % q
    assert (got == want).all()


def test_int8_plan_on_two_streams(torch_cuda):
    """One plan, launches alternating over two streams on independent
    batches (the INT8 path keeps no per-plan workspace, so they may run at
    the same time): every forward equals the oracle."""
    torch = torch_cuda
    qs = PRIMES17[:8]
    plan = nb.RnsPlan(16, qs, negacyclic=True)
    xs = [rand_batch(1, qs, 1 << 16, 900 + i) for i in range(6)]
    ds = [to_dev(torch, x.reshape(-1)) for x in xs]
    outs = [torch.empty_like(d) for d in ds]
    streams = [torch.cuda.Stream(), torch.cuda.Stream()]
    for i in range(6):
        plan.transform(outs[i], ds[i], 1, engine="int8", stream=streams[i & 1])
    torch.cuda.synchronize()
    for i in range(6):
        want = O.rns(xs[i].astype(np.uint64), qs, negacyclic=True)
        assert (to_host(outs[i], np.uint32).reshape(xs[i].shape).astype(np.uint64) == want).all(), i
    assert nb.device_errors() == 0
