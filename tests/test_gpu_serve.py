"""GPU: the serving loop (nttb_server_*) -- polynomial products and NTTs of
mixed sizes admitted against an HBM budget and batched continuously.  Every
result equals the oracle's product or transform, and a request gives the
same result alone and in a mix of concurrent requests."""
import numpy as np
import pytest

from oracle import oracle as O
import ntt_b200 as nb

pytestmark = pytest.mark.gpu

PRIMES = nb.generate_primes(31, 18, 8)  # negacyclic up to 2^17


def product(a, b, moduli, nega):
    fa = O.rns(a[None].astype(np.uint64), moduli, negacyclic=nega)[0]
    fb = O.rns(b[None].astype(np.uint64), moduli, negacyclic=nega)[0]
    q = np.array(moduli, dtype=np.uint64)[:, None]
    return O.rns(((fa * fb) % q)[None], moduli, negacyclic=nega, inverse=True)[0].astype(np.uint32)


def request(rng, log_range, limb_range):
    lg = int(rng.integers(log_range[0], log_range[1] + 1))
    limbs = int(rng.integers(limb_range[0], limb_range[1] + 1))
    first = int(rng.integers(0, len(PRIMES) - limbs + 1))
    mods = PRIMES[first:first + limbs]
    a = np.stack([rng.integers(0, q, 1 << lg, dtype=np.uint64) for q in mods]).astype(np.uint32)
    b = np.stack([rng.integers(0, q, 1 << lg, dtype=np.uint64) for q in mods]).astype(np.uint32)
    return a, b, lg, limbs, first


def test_server_products_vs_oracle(torch_cuda):
    rng = np.random.default_rng(1)
    srv = nb.Server(PRIMES, hbm_budget_bytes=64 << 20, max_log_n=14, slots=3, max_batch_requests=8)
    reqs = [request(rng, (3, 14), (1, 4)) for _ in range(30)]
    outs = [np.zeros_like(r[0]) for r in reqs]
    ids = [srv.submit(r[0], r[1], o, r[2], r[3], r[4]) for r, o in zip(reqs, outs)]
    lats = [srv.wait(i) for i in ids]
    assert all(l > 0 for l in lats)
    for (a, b, lg, limbs, first), o in zip(reqs, outs):
        assert (o == product(a, b, PRIMES[first:first + limbs], True)).all(), (lg, limbs)
    st = srv.stats()
    assert st["completed"] == 30 and st["bytes_in_use"] == 0 and st["batches"] >= 4
    assert len(srv.latencies()) == 30
    for (a, b, lg, limbs, first), o in zip(reqs, outs):  # small products against the schoolbook
        if lg <= 7:
            for l in range(limbs):
                ref = O.polymul_negacyclic(a[l].astype(np.uint64), b[l].astype(np.uint64), PRIMES[first + l])
                assert (o[l].astype(np.uint64) == ref).all()
    srv.close()
    assert nb.device_errors() == 0


def test_server_same_result_alone_and_in_mix(torch_cuda):
    rng = np.random.default_rng(2)
    srv = nb.Server(PRIMES, hbm_budget_bytes=96 << 20, max_log_n=16, slots=3, max_batch_requests=16)
    a, b, lg, limbs, first = request(rng, (13, 13), (3, 3))
    alone = np.zeros_like(a)
    srv.wait(srv.submit(a, b, alone, lg, limbs, first))
    others = [request(rng, (4, 16), (1, 6)) for _ in range(40)]
    outs = [np.zeros_like(r[0]) for r in others]
    mixed = np.zeros_like(a)
    ids = []
    for k, (r, o) in enumerate(zip(others, outs)):
        ids.append(srv.submit(r[0], r[1], o, r[2], r[3], r[4]))
        if k == 20:
            mine = srv.submit(a, b, mixed, lg, limbs, first)
    srv.drain()
    for i in ids + [mine]:
        srv.wait(i)
    assert (alone == mixed).all()
    assert (alone == product(a, b, PRIMES[first:first + limbs], True)).all()
    for r, o in zip(others, outs):
        assert (o == product(r[0], r[1], PRIMES[r[4]:r[4] + r[3]], True)).all()
    srv.close()


def test_server_ntt_requests_in_the_mix(torch_cuda):
    """Forward and inverse NTT requests share the queue and the batches with
    products: each equals the oracle's negacyclic transform per limb, and an
    NTT request gives the same result alone and in the mix."""
    rng = np.random.default_rng(5)
    srv = nb.Server(PRIMES, hbm_budget_bytes=96 << 20, max_log_n=16, slots=3, max_batch_requests=16)
    x, _, lg, limbs, first = request(rng, (12, 12), (3, 3))
    alone = np.zeros_like(x)
    srv.wait(srv.submit_ntt(x, alone, lg, limbs, first))
    mods = PRIMES[first:first + limbs]
    assert (alone == O.rns(x[None].astype(np.uint64), mods, negacyclic=True)[0].astype(np.uint32)).all()
    jobs = []
    for k in range(36):
        a, b, lgk, lk, fk = request(rng, (4, 16), (1, 5))
        out = np.zeros_like(a)
        if k % 3 == 0:
            jobs.append(("product", a, b, lgk, lk, fk, out, srv.submit(a, b, out, lgk, lk, fk)))
        else:
            inv = k % 3 == 2
            jobs.append(("inverse" if inv else "forward", a, None, lgk, lk, fk, out,
                         srv.submit_ntt(a, out, lgk, lk, fk, inverse=inv)))
        if k == 17:
            mixed = np.zeros_like(x)
            mine = srv.submit_ntt(x, mixed, lg, limbs, first)
    srv.drain()
    for j in jobs:
        srv.wait(j[-1])
    srv.wait(mine)
    assert (mixed == alone).all()
    for kind, a, b, lgk, lk, fk, out, _ in jobs:
        m = PRIMES[fk:fk + lk]
        if kind == "product":
            want = product(a, b, m, True)
        else:
            want = O.rns(a[None].astype(np.uint64), m, negacyclic=True, inverse=kind == "inverse")[0].astype(np.uint32)
        assert (out == want).all(), (kind, lgk, lk)
    st = srv.stats()
    assert st["completed"] == 38 and st["bytes_in_use"] == 0
    srv.close()
    assert nb.device_errors() == 0


def test_server_admission_under_budget(torch_cuda):
    """A budget that holds only a few requests at a time: the rest wait for
    memory, and everything completes correctly."""
    rng = np.random.default_rng(3)
    probe = nb.Server(PRIMES, hbm_budget_bytes=64 << 20, max_log_n=12, slots=2)
    resident = probe.stats()["resident_bytes"]
    probe.close()
    per = 2 * 4 * (1 << 12) * 4  # 4 limbs of 2^12, two operands
    srv = nb.Server(PRIMES, hbm_budget_bytes=resident + (2 << 20) + 3 * per, max_log_n=12, slots=2)
    st = srv.stats()
    assert st["region_bytes"] < 4 * per + (2 << 20) + 4096
    reqs = [request(rng, (12, 12), (4, 4)) for _ in range(24)]
    outs = [np.zeros_like(r[0]) for r in reqs]
    ids = [srv.submit(r[0], r[1], o, r[2], r[3], r[4]) for r, o in zip(reqs, outs)]
    srv.drain()
    for i in ids:
        srv.wait(i)
    for r, o in zip(reqs, outs):
        assert (o == product(r[0], r[1], PRIMES[r[4]:r[4] + r[3]], True)).all()
    st = srv.stats()
    assert st["peak_bytes_in_use"] <= st["region_bytes"]
    srv.close()


def test_server_refuses_oversized_and_bad_requests(torch_cuda):
    probe = nb.Server(PRIMES, hbm_budget_bytes=256 << 20, max_log_n=16, slots=1)
    resident = probe.stats()["resident_bytes"]
    probe.close()
    srv = nb.Server(PRIMES, hbm_budget_bytes=resident + (3 << 20), max_log_n=16, slots=1)
    big = np.zeros((8, 1 << 16), dtype=np.uint32)  # 4 MB of operands > the 2-3 MB request region
    with pytest.raises(nb.NTTError) as e:
        srv.submit(big, big.copy(), big.copy(), 16, 8, 0)
    assert e.value.status == nb.ERR_BUDGET
    with pytest.raises(nb.NTTError):
        srv.submit(big, big, big, 17, 1, 0)  # log_n above the server's
    with pytest.raises(nb.NTTError):
        srv.submit(big, big, big, 10, 4, 6)  # moduli 6..9 of 8
    with pytest.raises(nb.NTTError) as e:  # a budget below the resident tables
        nb.Server(PRIMES, hbm_budget_bytes=resident // 2, max_log_n=16, slots=1)
    assert e.value.status == nb.ERR_BUDGET
    srv.close()


def test_server_cyclic_products(torch_cuda):
    rng = np.random.default_rng(4)
    srv = nb.Server(PRIMES, hbm_budget_bytes=64 << 20, max_log_n=13, slots=2, negacyclic=0)
    reqs = [request(rng, (2, 13), (1, 3)) for _ in range(12)]
    outs = [np.zeros_like(r[0]) for r in reqs]
    for i in [srv.submit(r[0], r[1], o, r[2], r[3], r[4]) for r, o in zip(reqs, outs)]:
        srv.wait(i)
    for r, o in zip(reqs, outs):
        assert (o == product(r[0], r[1], PRIMES[r[4]:r[4] + r[3]], False)).all()
    # cyclic NTT requests, the smallest size and the largest the server takes
    for lg, inv in ((1, False), (13, False), (13, True), (7, True)):
        x, _, lgx, limbs, first = request(rng, (lg, lg), (2, 2))
        out = np.zeros_like(x)
        srv.wait(srv.submit_ntt(x, out, lgx, limbs, first, inverse=inv))
        want = O.rns(x[None].astype(np.uint64), PRIMES[first:first + limbs], negacyclic=False, inverse=inv)[0]
        assert (out == want.astype(np.uint32)).all(), (lg, inv)
    srv.close()


def test_server_device_resident_requests(torch_cuda):
    """Requests whose operands and result stay in device memory
    (nttb_server_submit_device): products and forward / inverse NTTs equal
    the oracle, a device product gives the same result alone and in a mix
    with host-memory requests, and host pointers are refused."""
    torch = torch_cuda
    rng = np.random.default_rng(9)
    srv = nb.Server(PRIMES, hbm_budget_bytes=96 << 20, max_log_n=16, slots=3, max_batch_requests=16)
    dev = lambda x: torch.from_numpy(np.ascontiguousarray(x).view(np.int32)).cuda()
    host = lambda t: t.cpu().numpy().view(np.uint32)
    a, b, lg, limbs, first = request(rng, (14, 14), (3, 3))
    da, db = dev(a), dev(b)
    alone = torch.zeros_like(da)
    srv.wait(srv.submit_device("mul", da, db, alone, lg, limbs, first))
    want = product(a, b, PRIMES[first:first + limbs], True)
    assert (host(alone).reshape(a.shape) == want).all()
    jobs, mine = [], None
    for k in range(30):
        x, y, lgk, lk, fk = request(rng, (4, 16), (1, 5))
        if k % 2:  # host-memory product
            out = np.zeros_like(x)
            jobs.append(("host", x, y, lgk, lk, fk, out, srv.submit(x, y, out, lgk, lk, fk)))
        else:  # device-resident forward / inverse NTT
            inv = k % 4 == 2
            dx, dout = dev(x), torch.zeros(x.size, dtype=torch.int32, device="cuda")
            jobs.append(("inverse" if inv else "forward", x, dx, lgk, lk, fk, dout,
                         srv.submit_device("inverse" if inv else "forward", dx, None, dout, lgk, lk, fk)))
        if k == 15:
            mixed = torch.zeros_like(da)
            mine = srv.submit_device("mul", da, db, mixed, lg, limbs, first)
    srv.drain()
    for j in jobs:
        srv.wait(j[-1])
    srv.wait(mine)
    assert torch.equal(mixed, alone)
    assert (host(da).reshape(a.shape) == a).all() and (host(db).reshape(b.shape) == b).all()  # inputs untouched
    for kind, x, y, lgk, lk, fk, out, _ in jobs:
        m = PRIMES[fk:fk + lk]
        if kind == "host":
            assert (out == product(x, y, m, True)).all()
        else:
            w = O.rns(x[None].astype(np.uint64), m, negacyclic=True, inverse=kind == "inverse")[0].astype(np.uint32)
            assert (host(out).reshape(x.shape) == w).all(), (kind, lgk, lk)
    with pytest.raises(nb.NTTError):  # host memory is not a device operand
        srv.submit_device("forward", torch.from_numpy(a.view(np.int32)), None, da, lg, limbs, first)
    srv.close()
    assert nb.device_errors() == 0
