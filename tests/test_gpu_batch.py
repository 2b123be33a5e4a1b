"""GPU parity of uneven batches (nttb_batch_*: one persistent launch over a
device work queue) against the oracle, job by job: every job's output equals
the oracle's RNS transform of that job (same moduli, direction and twist).
Zero mismatches allowed."""
import numpy as np
import pytest

from conftest import to_dev, to_host
from oracle import oracle as O
import ntt_b200 as nb

pytestmark = pytest.mark.gpu

PRIMES = nb.generate_primes(31, 21, 12)  # q == 1 mod 2^21: negacyclic up to 2^20

CONFIGS = [
    None,  # the default
    {"tile_elems": 4096, "threads": 256, "split": 1, "lag": 1, "group": 4},
    {"tile_elems": 8192, "threads": 512, "split": 0, "lag": 3, "group": 3},
    {"tile_elems": 8192, "threads": 256, "split": 1, "lag": 2, "group": 4},
    {"tile_elems": 16384, "threads": 512, "split": 1, "lag": 4, "ctas_per_sm": 1, "group": 4},
    {"tile_elems": 4096, "threads": 256, "split": 0, "lag": 2, "group": 3, "tensor": 1},
    {"tile_elems": 8192, "threads": 256, "split": 1, "lag": 1, "group": 1, "tensor": 1},
]

TENSOR = [
    {"tile_elems": 4096, "threads": 256, "split": 0, "lag": 2, "group": 3, "tensor": 1},
    {"tile_elems": 4096, "threads": 256, "split": 1, "lag": 4, "group": 4, "tensor": 1},
    {"tile_elems": 8192, "threads": 256, "split": 0, "lag": 1, "group": 1, "tensor": 1},
]


def make_jobs(torch, rng, n_jobs, log_range, limb_range, n_moduli, nega_ok=True):
    """Random job list: (host array, device tensor, log_n, limbs, first, inverse, nega)."""
    jobs = []
    for _ in range(n_jobs):
        lg = int(rng.integers(log_range[0], log_range[1] + 1))
        limbs = int(rng.integers(limb_range[0], limb_range[1] + 1))
        first = int(rng.integers(0, n_moduli - limbs + 1))
        inv = bool(rng.integers(0, 2))
        nega = nega_ok and bool(rng.integers(0, 2))
        x = np.empty((limbs, 1 << lg), dtype=np.uint32)
        for l in range(limbs):
            x[l] = rng.integers(0, PRIMES[first + l], 1 << lg, dtype=np.uint64).astype(np.uint32)
        jobs.append([x, to_dev(torch, x.reshape(-1)), lg, limbs, first, inv, nega])
    return jobs


def spec(jobs):
    return [(j[1], j[2], j[3], j[4], j[5], j[6]) for j in jobs]


def expect(job):
    x, _, lg, limbs, first, inv, nega = job
    return O.rns(x[None].astype(np.uint64), PRIMES[first:first + limbs], negacyclic=nega, inverse=inv)[0]


def check(torch, jobs):
    torch.cuda.synchronize()
    for j in jobs:
        got = to_host(j[1], np.uint32).reshape(j[0].shape).astype(np.uint64)
        want = expect(j)
        assert (got == want).all(), (j[2:], int((got != want).sum()))
    assert nb.device_errors() == 0


@pytest.mark.parametrize("config", CONFIGS)
def test_batch_mixed_small_sizes(torch_cuda, config):
    """2^1 .. 2^15 (single-pass tiles with several limbs per tile, and
    two-pass units for the sizes above the tile), both directions and twists."""
    rng = np.random.default_rng(7)
    plan = nb.BatchPlan(PRIMES, 15, negacyclic=True)
    jobs = make_jobs(torch_cuda, rng, 40, (1, 15), (1, 4), len(PRIMES))
    b = plan.batch(spec(jobs), config)
    b.launch()
    check(torch_cuda, jobs)


def test_batch_large_sizes(torch_cuda):
    """2^16 .. 2^20 two-pass units sharing the workspace ring."""
    rng = np.random.default_rng(20)
    plan = nb.BatchPlan(PRIMES, 20, negacyclic=True)
    jobs = make_jobs(torch_cuda, rng, 10, (16, 20), (1, 2), len(PRIMES))
    b = plan.batch(spec(jobs), {"tile_elems": 4096, "threads": 256, "split": 0, "lag": 1})
    info = b.info()
    assert info["units"] == sum(j[3] for j in jobs)
    b.launch()
    check(torch_cuda, jobs)


def test_batch_cyclic_plan(torch_cuda):
    rng = np.random.default_rng(3)
    plan = nb.BatchPlan(PRIMES[:6], 17, negacyclic=False)
    jobs = make_jobs(torch_cuda, rng, 16, (2, 17), (1, 3), 6, nega_ok=False)
    plan.batch(spec(jobs)).launch()
    check(torch_cuda, jobs)


def test_batch_graph_replay(torch_cuda):
    """The CUDA-graph replay gives the launch's results, on two replays."""
    rng = np.random.default_rng(11)
    plan = nb.BatchPlan(PRIMES, 18, negacyclic=True)
    jobs = make_jobs(torch_cuda, rng, 12, (6, 18), (1, 3), len(PRIMES))
    b = plan.batch(spec(jobs))
    for rep in range(2):
        for j in jobs:  # fresh input in the same buffers
            j[1].copy_(to_dev(torch_cuda, j[0].reshape(-1)))
        b.graph_launch()
        check(torch_cuda, jobs)


def test_batch_round_trip_uneven(torch_cuda):
    """A reduced config-4 mix (log2 N in 12..20, 1..3 limbs): a forward batch
    then an inverse batch over the same buffers returns the input."""
    rng = np.random.default_rng(4)
    plan = nb.BatchPlan(PRIMES, 20, negacyclic=True)
    jobs = make_jobs(torch_cuda, rng, 24, (12, 20), (1, 3), len(PRIMES))
    fwd = [(j[1], j[2], j[3], j[4], False, j[6]) for j in jobs]
    inv = [(j[1], j[2], j[3], j[4], True, j[6]) for j in jobs]
    plan.batch(fwd).launch()
    plan.batch(inv).launch()
    torch_cuda.cuda.synchronize()
    for j in jobs:
        assert (to_host(j[1], np.uint32).reshape(j[0].shape) == j[0]).all()
    assert nb.device_errors() == 0


def test_batch_autotune(torch_cuda):
    rng = np.random.default_rng(5)
    plan = nb.BatchPlan(PRIMES, 16, negacyclic=True)
    jobs = make_jobs(torch_cuda, rng, 20, (8, 16), (1, 3), len(PRIMES))
    before = [to_host(j[1], np.uint32).copy() for j in jobs]
    cfg = plan.autotune(spec(jobs))
    assert cfg["tile_elems"] in (4096, 8192, 16384) and cfg["split"] in (0, 1) and cfg["lag"] >= 1
    assert cfg["group"] in (1, 3, 4)
    for j, b0 in zip(jobs, before):  # autotuning leaves the jobs' data alone
        assert (to_host(j[1], np.uint32) == b0).all()
    b = plan.batch(spec(jobs))
    assert b.info()["config"] == cfg
    b.launch()
    check(torch_cuda, jobs)


def test_batch_rejects_bad_jobs(torch_cuda):
    plan = nb.BatchPlan(PRIMES[:4], 12, negacyclic=False)
    d = torch_cuda.zeros(1 << 14, dtype=torch_cuda.int32, device="cuda")
    with pytest.raises(nb.NTTError):
        plan.batch([(d, 13, 1, 0, False, False)])  # log_n above the plan
    with pytest.raises(nb.NTTError):
        plan.batch([(d, 10, 3, 2, False, False)])  # moduli 2..4 of 4
    with pytest.raises(nb.NTTError):
        plan.batch([(d, 10, 1, 0, False, True)])  # negacyclic job, cyclic plan
    with pytest.raises(nb.NTTError):
        plan.batch([(d, 10, 1, 0, False, False)], {"tile_elems": 2048})
    # flag bits other than inverse / negacyclic / product are refused at the C ABI
    import ctypes
    arr = (nb.BatchJob * 1)()
    arr[0] = nb.BatchJob(d.data_ptr(), 10, 1, 0, 1 << 30, None)
    h = ctypes.c_void_p()
    assert nb.lib().nttb_batch_create(plan._h, arr, 1, None, ctypes.byref(h)) == nb.ERR_INVALID_ARG
    # an empty job list is a batch that launches nothing
    b = plan.batch([])
    b.launch()
    torch_cuda.cuda.synchronize()
    b.close()
    assert nb.device_errors() == 0


def expect_product(a, b, moduli, nega):
    """inverse(forward(a) . forward(b)) per limb through the oracle."""
    fa = O.rns(a[None].astype(np.uint64), moduli, negacyclic=nega)[0]
    fb = O.rns(b[None].astype(np.uint64), moduli, negacyclic=nega)[0]
    q = np.array(moduli, dtype=np.uint64)[:, None]
    return O.rns(((fa * fb) % q)[None], moduli, negacyclic=nega, inverse=True)[0]


@pytest.mark.parametrize("nega", [True, False])
def test_batch_polymul_fused(torch_cuda, nega):
    """Products (forward a, forward b, pointwise, inverse in one launch) of
    sizes 2^3 .. 2^17 mixed with plain transforms in the same batch."""
    rng = np.random.default_rng(17 + nega)
    plan = nb.BatchPlan(PRIMES, 17, negacyclic=nega)
    plain = make_jobs(torch_cuda, rng, 8, (3, 17), (1, 3), len(PRIMES), nega_ok=nega)
    prods = []
    for _ in range(14):
        lg = int(rng.integers(3, 18))
        limbs = int(rng.integers(1, 4))
        first = int(rng.integers(0, len(PRIMES) - limbs + 1))
        mods = PRIMES[first:first + limbs]
        a = np.stack([rng.integers(0, q, 1 << lg, dtype=np.uint64) for q in mods]).astype(np.uint32)
        b = np.stack([rng.integers(0, q, 1 << lg, dtype=np.uint64) for q in mods]).astype(np.uint32)
        prods.append((a, b, to_dev(torch_cuda, a.reshape(-1)), to_dev(torch_cuda, b.reshape(-1)), lg, limbs, first))
    jobs = spec(plain) + [(p[2], p[4], p[5], p[6], "mul", nega, p[3]) for p in prods]
    plan.batch(jobs).launch()
    check(torch_cuda, plain)
    for a, b, da, db, lg, limbs, first in prods:
        got = to_host(da, np.uint32).reshape(a.shape).astype(np.uint64)
        want = expect_product(a, b, PRIMES[first:first + limbs], nega)
        assert (got == want).all(), (lg, limbs, int((got != want).sum()))
        if nega and lg <= 8:  # against the schoolbook product itself
            for l in range(limbs):
                ref = O.polymul_negacyclic(a[l].astype(np.uint64), b[l].astype(np.uint64), PRIMES[first + l])
                assert (got[l] == ref).all()


@pytest.mark.parametrize("config", TENSOR)
def test_batch_tensor_tiles_every_size(torch_cuda, config):
    """Tensor-core tiles (INT8 DFT-64 + DFT-r' on the CUDA cores) for every
    two-pass size 2^13 .. 2^20, both directions and twists, in one launch with
    CUDA-core units of the smaller sizes."""
    rng = np.random.default_rng(31 + config["split"])
    plan = nb.BatchPlan(PRIMES, 20, negacyclic=True)
    jobs = []
    for lg in range(13, 21):
        for inv in (False, True):
            for nega in (False, True):
                limbs = 1 if lg >= 18 else 2
                first = int(rng.integers(0, len(PRIMES) - limbs + 1))
                x = np.stack([rng.integers(0, PRIMES[first + l], 1 << lg, dtype=np.uint64)
                              for l in range(limbs)]).astype(np.uint32)
                jobs.append([x, to_dev(torch_cuda, x.reshape(-1)), lg, limbs, first, inv, nega])
    jobs += make_jobs(torch_cuda, rng, 12, (1, 12), (1, 3), len(PRIMES))
    b = plan.batch(spec(jobs), config)
    assert b.info()["config"]["tensor"] == 1
    b.launch()
    check(torch_cuda, jobs)


def test_batch_tensor_round_trip_and_graph(torch_cuda):
    """Forward then inverse batches on tensor tiles return the input; a graph
    replay gives the launch's results."""
    rng = np.random.default_rng(41)
    plan = nb.BatchPlan(PRIMES, 20, negacyclic=True)
    cfg = TENSOR[0]
    jobs = make_jobs(torch_cuda, rng, 16, (12, 20), (1, 3), len(PRIMES))
    fwd = [(j[1], j[2], j[3], j[4], False, j[6]) for j in jobs]
    inv = [(j[1], j[2], j[3], j[4], True, j[6]) for j in jobs]
    bf, bi = plan.batch(fwd, cfg), plan.batch(inv, cfg)
    for rep in range(2):
        if rep:
            bf.graph_launch()
            bi.graph_launch()
        else:
            bf.launch()
            bi.launch()
        torch_cuda.cuda.synchronize()
        for j in jobs:
            assert (to_host(j[1], np.uint32).reshape(j[0].shape) == j[0]).all(), j[2:]
    assert nb.device_errors() == 0


@pytest.mark.parametrize("nega", [True, False])
def test_batch_tensor_polymul(torch_cuda, nega):
    """Products whose transforms run on tensor tiles (2^13 .. 2^17) next to
    small CUDA-core products, one launch."""
    rng = np.random.default_rng(51 + nega)
    plan = nb.BatchPlan(PRIMES, 17, negacyclic=nega)
    prods = []
    for lg in [4, 9, 12, 13, 14, 15, 16, 17, 13, 16]:
        limbs = int(rng.integers(1, 4))
        first = int(rng.integers(0, len(PRIMES) - limbs + 1))
        mods = PRIMES[first:first + limbs]
        a = np.stack([rng.integers(0, q, 1 << lg, dtype=np.uint64) for q in mods]).astype(np.uint32)
        b = np.stack([rng.integers(0, q, 1 << lg, dtype=np.uint64) for q in mods]).astype(np.uint32)
        prods.append((a, b, to_dev(torch_cuda, a.reshape(-1)), to_dev(torch_cuda, b.reshape(-1)), lg, limbs, first))
    jobs = [(p[2], p[4], p[5], p[6], "mul", nega, p[3]) for p in prods]
    plan.batch(jobs, TENSOR[1]).launch()
    torch_cuda.cuda.synchronize()
    for a, b, da, db, lg, limbs, first in prods:
        got = to_host(da, np.uint32).reshape(a.shape).astype(np.uint64)
        want = expect_product(a, b, PRIMES[first:first + limbs], nega)
        assert (got == want).all(), (lg, limbs, int((got != want).sum()))
    assert nb.device_errors() == 0


def test_batch_tensor_flag_where_the_shape_allows(torch_cuda):
    """tensor = 1 with a 512-thread shape runs the CUDA-core tiles (same
    results); tensor = 2 is refused."""
    rng = np.random.default_rng(61)
    plan = nb.BatchPlan(PRIMES[:4], 16, negacyclic=True)
    jobs = make_jobs(torch_cuda, rng, 6, (13, 16), (1, 2), 4)
    b = plan.batch(spec(jobs), {"tile_elems": 8192, "threads": 512, "tensor": 1})
    b.launch()
    check(torch_cuda, jobs)
    with pytest.raises(nb.NTTError):
        plan.batch(spec(jobs), {"tensor": 2})


def test_batch_wait_timeout_is_reported_and_recoverable(torch_cuda):
    """Failure path without a GPU fault: a planted unsatisfiable dependency
    (the test hook raises the first-pass tile count that one unit's second
    pass waits for) makes that bounded device wait run out; the launch
    completes, nttb_device_errors reports it, the units of other sizes are
    still exact, and the context stays usable for a fresh batch."""
    import time
    rng = np.random.default_rng(81)
    plan = nb.BatchPlan(PRIMES[:4], 16, negacyclic=True)
    assert nb.device_errors() == 0
    for config in (TENSOR[0], {"tile_elems": 4096, "threads": 256, "tensor": 0}):
        jobs = make_jobs(torch_cuda, rng, 4, (14, 16), (1, 1), 4)
        b = plan.batch(spec(jobs), config)
        b.test_stall(0)  # units run largest first: unit 0 belongs to the largest job
        t = time.time()
        b.launch()
        torch_cuda.cuda.synchronize()
        assert time.time() - t < 30
        flags = nb.device_errors()
        assert flags & 4, flags
        largest = max(j[2] for j in jobs)
        for j in jobs:
            if j[2] == largest:
                continue  # the stalled unit, or one of its size
            got = to_host(j[1], np.uint32).reshape(j[0].shape).astype(np.uint64)
            assert (got == expect(j)).all()
        b.close()
    fresh = make_jobs(torch_cuda, rng, 6, (8, 16), (1, 2), 4)
    plan.batch(spec(fresh)).launch()
    check(torch_cuda, fresh)


PRIMES32 = nb.generate_primes(31, 21, 32)


@pytest.mark.parametrize("config", [None, TENSOR[0]])
def test_batch_config4_shaped_mix_wraps_the_rings(torch_cuda, config):
    """The uneven-batch workload's shape at reduced size: 128 polynomials,
    log2 N uniform in 12..20, 1..32 limbs over 32 moduli, mixed directions
    (1.8 GB).  The 2^17 .. 2^20 classes hold many more units than their
    workspace rings have slots (217 units of 2^20 against 16 slots), so the
    rings wrap many times and pass A tiles wait for their slot's previous
    owner.  Checked job by job (limbs first, middle and last of every job
    against the oracle) and as a whole (the batch with every direction
    flipped returns the inputs word for word)."""
    from concurrent.futures import ThreadPoolExecutor
    torch = torch_cuda
    rng = np.random.default_rng(8)
    lgs, limbss = rng.integers(12, 21, 128), rng.integers(1, 33, 128)
    invs = rng.integers(0, 2, 128).astype(bool)
    words = int(sum(int(b) << int(a) for a, b in zip(lgs, limbss)))
    buf = torch.empty(words, dtype=torch.int32, device="cuda")
    qt = torch.tensor(PRIMES32, dtype=torch.int64, device="cuda")
    gen = torch.Generator(device="cuda")
    gen.manual_seed(8)
    jobs, off = [], 0
    for lg, limbs, inv in zip(lgs, limbss, invs):
        lg, limbs = int(lg), int(limbs)
        view = buf[off:off + (limbs << lg)].view(limbs, 1 << lg)
        r = torch.randint(0, 1 << 31, (limbs, 1 << lg), generator=gen, device="cuda", dtype=torch.int64)
        view.copy_((r % qt[:limbs, None]).to(torch.int32))
        jobs.append((view, lg, limbs, 0, bool(inv), False))
        off += limbs << lg
    buf0 = buf.clone()
    plan = nb.BatchPlan(PRIMES32, 20)
    b = plan.batch(jobs, config)
    assert b.info()["ws_bytes"] < 4 * words  # the rings are smaller than the batch: they wrap
    b.launch()
    torch.cuda.synchronize()
    assert nb.device_errors() == 0
    rows = [(i, l) for i, j in enumerate(jobs) for l in sorted({0, j[2] // 2, j[2] - 1})]

    def one(row):
        i, l = row
        view, lg, limbs, _, inv, _ = jobs[i]
        start = view.storage_offset() - buf.storage_offset() + (l << lg)
        x = to_host(buf0[start:start + (1 << lg)], np.uint32).astype(np.uint64)
        want = O.rns(x[None, None], [PRIMES32[l]], inverse=inv)[0, 0]
        got = to_host(view[l], np.uint32).astype(np.uint64)
        return int((got != want).sum())

    with ThreadPoolExecutor(max_workers=16) as ex:  # the oracle's ctypes calls release the GIL
        bad = list(ex.map(one, rows))
    assert sum(bad) == 0, [(jobs[r[0]][1:5], r[1], n) for r, n in zip(rows, bad) if n][:8]
    b.close()
    flipped = [(v, lg, limbs, first, not inv, nega) for v, lg, limbs, first, inv, nega in jobs]
    plan.batch(flipped, config).launch()
    torch.cuda.synchronize()
    assert nb.device_errors() == 0
    assert torch.equal(buf, buf0)
