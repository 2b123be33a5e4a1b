"""GPU parity of the uint64-word drop-in path (the reference's include/ntt.cuh
entry points) against the oracle, the golden fixtures and the reference's own
GPU kernels.  Tolerance: zero mismatches (exact integer arithmetic)."""
import numpy as np
import pytest

from conftest import BABYBEAR, Q60, golden, to_dev, to_host
from oracle import oracle as O
import ntt_b200 as nb

pytestmark = pytest.mark.gpu

ENGINES = ["scalar", "auto"]


def rand(n, q, seed):
    return np.random.default_rng(seed).integers(0, q, n, dtype=np.uint64)


def run_u64(torch, plan, x, inverse=False, engine="auto", batch=1):
    d = to_dev(torch, x)
    plan.transform(d, batch=batch, inverse=inverse, engine=engine)
    torch.cuda.synchronize()
    return to_host(d, np.uint64)


@pytest.mark.parametrize("engine", ENGINES)
@pytest.mark.parametrize("lg", [1, 2, 5, 6, 7, 10, 12, 13, 14, 16, 17, 20])
def test_forward_inverse_vs_oracle(torch_cuda, engine, lg):
    n = 1 << lg
    x = rand(n, BABYBEAR, lg)
    plan = nb.Plan(n, BABYBEAR)
    y = run_u64(torch_cuda, plan, x, False, engine)
    ref = O.ntt(x, BABYBEAR)
    assert (y == ref).all(), "forward mismatches: %d" % int((y != ref).sum())
    z = run_u64(torch_cuda, plan, y, True, engine)
    assert (z == x).all()
    if lg <= 16:
        assert (run_u64(torch_cuda, plan, x, True, engine) == O.ntt(x, BABYBEAR, True)).all()


@pytest.mark.parametrize("batch", [1, 3, 8, 24])
@pytest.mark.parametrize("q", [BABYBEAR, 2147352577])
def test_int8_engine_on_uint64_words(torch_cuda, batch, q):
    """The INT8 tensor-core engine serves the drop-in uint64-word layout at
    N = 2^16 (read and written as 8-byte words, in place): forward and
    inverse equal the oracle for every polynomial of the batch."""
    n = 1 << 16
    x = np.stack([rand(n, q, 700 + i) for i in range(batch)])
    plan = nb.Plan(n, q)
    y = run_u64(torch_cuda, plan, x.reshape(-1), False, "int8", batch).reshape(batch, n)
    for i in range(batch):
        assert (y[i] == O.ntt(x[i], q)).all(), "poly %d" % i
    z = run_u64(torch_cuda, plan, y.reshape(-1), True, "int8", batch).reshape(batch, n)
    assert (z == x).all()
    assert nb.device_errors() == 0


def test_auto_engine_for_uint64_batches(torch_cuda):
    """AUTO takes the INT8 kernel for uint64 batches of 8 or more polynomials
    at N = 2^16 and the CUDA-core engine for fewer; both bit-exact."""
    n = 1 << 16
    plan = nb.Plan(n, BABYBEAR)
    for batch, kernel in ((8, "int8_cluster_n16_x2"), (2, "scalar_pass_col")):
        x = np.stack([rand(n, BABYBEAR, 900 + i) for i in range(batch)])
        d = to_dev(torch_cuda, x.reshape(-1))
        nb.profile_start()
        plan.transform(d, batch=batch)
        torch_cuda.cuda.synchronize()
        ran = nb.profile_stop()
        assert kernel in ran, (batch, ran)
        y = to_host(d, np.uint64).reshape(batch, n)
        for i in range(batch):
            assert (y[i] == O.ntt(x[i], BABYBEAR)).all()


@pytest.mark.parametrize("lg", [13, 15, 17, 18, 19, 20])
@pytest.mark.parametrize("batch", [1, 3])
def test_tiles_engine_on_uint64_words(torch_cuda, lg, batch):
    """The batch queue's tensor tiles as a plan engine (NTTB_ENGINE_TILES) on
    the drop-in uint64-word layout, in place: pass A reads the words, pass B
    writes them back.  Forward and inverse equal the oracle for every
    polynomial; the high words of the results are zero."""
    n = 1 << lg
    x = np.stack([rand(n, BABYBEAR, 1300 + 7 * lg + i) for i in range(batch)])
    plan = nb.Plan(n, BABYBEAR)
    y = run_u64(torch_cuda, plan, x.reshape(-1), False, "tiles", batch).reshape(batch, n)
    for i in range(batch):
        assert (y[i] == O.ntt(x[i], BABYBEAR)).all(), "poly %d" % i
    z = run_u64(torch_cuda, plan, y.reshape(-1), True, "tiles", batch).reshape(batch, n)
    assert (z == x).all()
    assert nb.device_errors() == 0


def test_tiles_engine_queue_cache(torch_cuda):
    """A plan keeps eight tile queues (one per source / destination / count /
    direction): ten buffers in turn, twice over, replace queues in LRU order;
    every call is exact."""
    lg, n = 18, 1 << 18
    plan = nb.Plan(n, BABYBEAR)
    xs = [rand(n, BABYBEAR, 1400 + i) for i in range(10)]
    ds = [to_dev(torch_cuda, x) for x in xs]
    for rnd in range(2):
        for i, d in enumerate(ds):
            plan.transform(d, inverse=bool(rnd), engine="tiles")
    torch_cuda.cuda.synchronize()
    for x, d in zip(xs, ds):
        assert (to_host(d, np.uint64) == x).all()
    assert nb.device_errors() == 0


def test_auto_engine_takes_tiles(torch_cuda):
    """AUTO sends calls of 2^17 .. 2^20 residues per polynomial that hold at
    least 2^20 residues to the tensor tiles (one launch of the batch queue),
    smaller calls to the CUDA-core engine; both exact."""
    for lg, batch, kernel in ((20, 1, "batch_queue"), (18, 4, "batch_queue"), (19, 1, "scalar_pass_col"),
                              (17, 2, "scalar_pass_col")):
        n = 1 << lg
        x = np.stack([rand(n, BABYBEAR, 1500 + lg + i) for i in range(batch)])
        plan = nb.Plan(n, BABYBEAR)
        d = to_dev(torch_cuda, x.reshape(-1))
        nb.profile_start()
        plan.transform(d, batch=batch)
        torch_cuda.cuda.synchronize()
        ran = nb.profile_stop()
        assert kernel in ran, (lg, batch, ran)
        y = to_host(d, np.uint64).reshape(batch, n)
        for i in range(batch):
            assert (y[i] == O.ntt(x[i], BABYBEAR)).all()


@pytest.mark.parametrize("n", [64, 256, 1024, 4096])
def test_golden_seed42(torch_cuda, n):
    g = golden("babybear_seed42.npz")
    plan = nb.Plan(n, BABYBEAR)
    assert (run_u64(torch_cuda, plan, g["in_%d" % n]) == g["fwd_%d" % n]).all()
    assert (run_u64(torch_cuda, plan, g["in_%d" % n], True) == g["inv_%d" % n]).all()


@pytest.mark.parametrize("n", [64, 128, 4096])
def test_golden_iplus1(torch_cuda, n):
    g = golden("babybear_iplus1.npz")
    plan = nb.Plan(n, BABYBEAR)
    assert (run_u64(torch_cuda, plan, np.arange(1, n + 1, dtype=np.uint64)) == g["fwd_%d" % n]).all()


def test_composite_modulus_rejected():
    """The reference's PRIME_30_2 = 1073610753 (include/modular_arith.cuh:26) is 3 * 10837 * 33023;
    plans refuse composite moduli instead of computing a non-invertible map."""
    with pytest.raises(nb.NTTError) as e:
        nb.Plan(1 << 10, 1073610753)
    assert "not prime" in str(e.value)


@pytest.mark.parametrize("q", [1073479681, 2146959361, 2147352577])
def test_other_31bit_primes(torch_cuda, q):
    for lg in (4, 11, 15):
        n = 1 << lg
        x = rand(n, q, lg + 100)
        plan = nb.Plan(n, q)
        assert (run_u64(torch_cuda, plan, x) == O.ntt(x, q)).all()


def test_batch_matches_per_poly(torch_cuda):
    n, b = 1 << 12, 7
    x = np.stack([rand(n, BABYBEAR, 300 + i) for i in range(b)])
    plan = nb.Plan(n, BABYBEAR)
    y = run_u64(torch_cuda, plan, x.reshape(-1), batch=b).reshape(b, n)
    for i in range(b):
        assert (y[i] == O.ntt(x[i], BABYBEAR)).all()


def test_wide_modulus_through_u64_plan(torch_cuda):
    g = golden("q60.npz")
    q = int(g["q"])
    plan = nb.Plan(1024, q)
    assert (run_u64(torch_cuda, plan, g["inp"]) == g["fwd"]).all()
    assert (run_u64(torch_cuda, plan, g["inp"], True) == g["inv"]).all()
    plan2 = nb.Plan(1 << 12, 4293918721)  # 32-bit modulus (>= 2^31) runs the 64-bit path
    x = rand(1 << 12, 4293918721, 9)
    assert (run_u64(torch_cuda, plan2, x) == O.ntt(x, 4293918721)).all()


@pytest.mark.parametrize("n", [64, 128, 4096, 8192, 16384, 1 << 16])
def test_four_step_matches_reference_map(torch_cuda, n):
    """n = 64 makes the second pass of length 1 (n1 = 64, n2 = 1)."""
    x = rand(n, BABYBEAR, n)
    plan = nb.Plan(n, BABYBEAR)
    d = to_dev(torch_cuda, x)
    plan.four_step(d)
    torch_cuda.cuda.synchronize()
    y = to_host(d, np.uint64)
    assert (y == O.four_step(x, BABYBEAR)).all()
    plan.four_step(d, inverse=True)
    torch_cuda.cuda.synchronize()
    assert (to_host(d, np.uint64) == x).all()


def test_rowmaj_forward(torch_cuda):
    n = 4096
    x = rand(n, BABYBEAR, 77)
    pre = O.to_pretransposed(x, 64, 64)
    plan = nb.Plan(n, BABYBEAR)
    d = to_dev(torch_cuda, pre)
    plan.rowmaj_forward(d)
    torch_cuda.cuda.synchronize()
    assert (to_host(d, np.uint64) == O.rowmaj_forward(pre, BABYBEAR)).all()
    # other sizes: plain forward on the buffer as given (src/ntt_optimized.cu:944-948)
    plan2 = nb.Plan(1024, BABYBEAR)
    x2 = rand(1024, BABYBEAR, 78)
    d2 = to_dev(torch_cuda, x2)
    plan2.rowmaj_forward(d2)
    torch_cuda.cuda.synchronize()
    assert (to_host(d2, np.uint64) == O.ntt(x2, BABYBEAR)).all()


@pytest.mark.parametrize("lg,n1", [(10, 32), (12, 64), (12, 16), (16, 256), (16, 64), (20, 1024), (13, 8192),
                                   (6, 1)])
def test_pretransposed_transform_every_size(torch_cuda, lg, n1):
    """The RowMaj pre-transposed layout pre[b*n1 + a] = x[a*n2 + b] for every
    n: forward gives the pre-transposed forward transform, inverse returns the
    input; n = 4096, n1 = 64 forward is ntt_forward_rowmaj."""
    n = 1 << lg
    n2 = n // n1
    x = rand(n, BABYBEAR, lg * 31 + n1)
    plan = nb.Plan(n, BABYBEAR)
    d = to_dev(torch_cuda, O.to_pretransposed(x, n1, n2))
    plan.pretransposed_transform(d, n1)
    torch_cuda.cuda.synchronize()
    assert (to_host(d, np.uint64) == O.to_pretransposed(O.ntt(x, BABYBEAR), n1, n2)).all()
    plan.pretransposed_transform(d, n1, inverse=True)
    torch_cuda.cuda.synchronize()
    assert (to_host(d, np.uint64) == O.to_pretransposed(x, n1, n2)).all()
    if n == 4096 and n1 == 64:
        d2 = to_dev(torch_cuda, O.to_pretransposed(x, 64, 64))
        plan.rowmaj_forward(d2)
        torch_cuda.cuda.synchronize()
        assert (to_host(d2, np.uint64) == O.rowmaj_forward(O.to_pretransposed(x, 64, 64), BABYBEAR)).all()


@pytest.mark.parametrize("n1", [64, 16])
def test_pretransposed_transform_60bit_prime(torch_cuda, n1):
    """The 64-bit Montgomery plan takes the transpose route for every shape."""
    g = golden("q60.npz")
    q = int(g["q"])
    n = 1 << 12
    x = rand(n, q, 60 + n1)
    plan = nb.Plan(n, q)
    d = to_dev(torch_cuda, O.to_pretransposed(x, n1, n // n1))
    plan.pretransposed_transform(d, n1)
    torch_cuda.cuda.synchronize()
    assert (to_host(d, np.uint64) == O.to_pretransposed(O.ntt(x, q), n1, n // n1)).all()
    plan.pretransposed_transform(d, n1, inverse=True)
    torch_cuda.cuda.synchronize()
    assert (to_host(d, np.uint64) == O.to_pretransposed(x, n1, n // n1)).all()


@pytest.mark.parametrize("rows,cols", [(32, 1 << 20), (1 << 20, 32), (64, 1 << 18)])
def test_transpose_tall_and_wide(torch_cuda, rows, cols):
    """One row or one column of TMA tiles across 2^20 words."""
    x = np.random.default_rng(rows + cols).integers(0, 1 << 63, rows * cols, dtype=np.uint64)
    src = to_dev(torch_cuda, x)
    dst = torch_cuda.empty_like(src)
    nb.transpose_u64(dst, src, rows, cols)
    torch_cuda.cuda.synchronize()
    assert (to_host(dst, np.uint64) == x.reshape(rows, cols).T.reshape(-1)).all()
    assert nb.device_errors() == 0


def test_pretransposed_square_runs_without_transposes(torch_cuda):
    """n = M^2, n1 = M: two scalar passes read and write the layout directly
    (no transpose kernel runs); the result is the pre-transposed transform."""
    n, m = 1 << 16, 256
    x = rand(n, BABYBEAR, 4242)
    plan = nb.Plan(n, BABYBEAR)
    d = to_dev(torch_cuda, O.to_pretransposed(x, m, m))
    nb.profile_start()
    plan.pretransposed_transform(d, m)
    torch_cuda.cuda.synchronize()
    ran = nb.profile_stop()
    assert not any("transpose" in k for k in ran), ran
    assert sum(v[0] for k, v in ran.items() if k.startswith("scalar_pass")) == 2, ran
    assert (to_host(d, np.uint64) == O.to_pretransposed(O.ntt(x, BABYBEAR), m, m)).all()


def test_pretransposed_transform_rejects_bad_n1(torch_cuda):
    plan = nb.Plan(1 << 10, BABYBEAR)
    d = to_dev(torch_cuda, rand(1 << 10, BABYBEAR, 1))
    for bad in (3, 1 << 11, 0):
        with pytest.raises(nb.NTTError) as e:
            plan.pretransposed_transform(d, bad)
        assert "n1" in str(e.value)


def test_transpose_helpers(torch_cuda):
    x = rand(64 * 128, BABYBEAR, 5)
    src = to_dev(torch_cuda, x)
    dst = torch_cuda.empty_like(src)
    nb.transpose_u64(dst, src, 64, 128)  # rowmaj_to_pretransposed(N1=64, N2=128)
    torch_cuda.cuda.synchronize()
    assert (to_host(dst, np.uint64) == O.to_pretransposed(x, 64, 128)).all()
    back = torch_cuda.empty_like(src)
    nb.transpose_u64(back, dst, 128, 64)  # rowmaj_from_pretransposed(N1=64, N2=128)
    torch_cuda.cuda.synchronize()
    assert (to_host(back, np.uint64) == x).all()


@pytest.mark.parametrize("rows,cols", [(32, 32), (64, 128), (128, 64), (96, 4096), (4096, 96), (2048, 2048),
                                       (33, 64), (64, 48), (1, 1000), (7, 3)])
def test_transpose_every_shape(torch_cuda, rows, cols):
    """Out-of-place transpose: TMA tiles where rows and cols are multiples of
    32, the plain tiled kernel otherwise; both against numpy."""
    x = np.random.default_rng(rows * 7919 + cols).integers(0, 1 << 63, rows * cols, dtype=np.uint64)
    src = to_dev(torch_cuda, x)
    dst = torch_cuda.full_like(src, -1)
    nb.transpose_u64(dst, src, rows, cols)
    torch_cuda.cuda.synchronize()
    assert (to_host(dst, np.uint64) == x.reshape(rows, cols).T.reshape(-1)).all()
    assert nb.device_errors() == 0


def test_transpose_unaligned_arrays(torch_cuda):
    """Arrays that start 8 bytes past a 16-byte boundary take the plain kernel."""
    rows, cols = 64, 96
    x = np.random.default_rng(11).integers(0, 1 << 63, rows * cols, dtype=np.uint64)
    src_buf = to_dev(torch_cuda, np.concatenate([np.zeros(1, np.uint64), x]))
    dst_buf = torch_cuda.zeros(rows * cols + 1, dtype=torch_cuda.int64, device="cuda")
    src, dst = src_buf[1:], dst_buf[1:]
    assert src.data_ptr() % 16 == 8 and dst.data_ptr() % 16 == 8
    nb.transpose_u64(dst, src, rows, cols)
    torch_cuda.cuda.synchronize()
    assert (to_host(dst, np.uint64) == x.reshape(rows, cols).T.reshape(-1)).all()
    assert int(dst_buf[0].item()) == 0


def test_tma_paths_are_the_ones_that_run(torch_cuda):
    """Whole tiles on 16-byte aligned arrays launch the TMA tile kernels (the
    profiler names the kernel that ran); ragged shapes the plain ones."""
    x = to_dev(torch_cuda, np.arange(64 * 64, dtype=np.uint64))
    y = torch_cuda.empty_like(x)
    nb.profile_start()
    nb.transpose_u64(y, x, 64, 64)
    nb.transpose_u64(x, x, 64, 64)
    nb.bit_reverse_u64(x, 64 * 64)
    nb.transpose_u64(y[:40 * 40], x[:40 * 40], 40, 40)
    torch_cuda.cuda.synchronize()
    ran = nb.profile_stop()
    for name in ("tma_transpose_u64", "tma_transpose_square_inplace_u64", "tma_bitrev_u64", "transpose_u64"):
        assert ran.get(name, (0, 0))[0] == 1, (name, ran)


@pytest.mark.parametrize("n", [32, 64, 96, 1024, 4096, 40, 1])
def test_transpose_square_in_place(torch_cuda, n):
    """In-place transpose of a square matrix: TMA tile pairs for multiples of
    32, the element-pair kernel otherwise."""
    x = np.random.default_rng(n).integers(0, 1 << 63, n * n, dtype=np.uint64)
    d = to_dev(torch_cuda, x)
    nb.transpose_u64(d, d, n, n)
    torch_cuda.cuda.synchronize()
    assert (to_host(d, np.uint64) == x.reshape(n, n).T.reshape(-1)).all()
    assert nb.device_errors() == 0


@pytest.mark.parametrize("lg", [10, 12, 16, 22, 24])
def test_bit_reverse_tma_and_unaligned(torch_cuda, lg):
    """Bit reversal from 2^10 on runs on TMA tile pairs; the same array 8 bytes
    off a 16-byte boundary takes the plain tiled kernel; both match the oracle."""
    n = 1 << lg
    x = np.random.default_rng(lg + 100).integers(0, 1 << 63, n, dtype=np.uint64)
    want = O.bit_reverse(x)
    d = to_dev(torch_cuda, x)
    nb.bit_reverse_u64(d, n)
    torch_cuda.cuda.synchronize()
    assert (to_host(d, np.uint64) == want).all()
    buf = to_dev(torch_cuda, np.concatenate([np.zeros(1, np.uint64), x]))
    nb.bit_reverse_u64(buf[1:], n)
    torch_cuda.cuda.synchronize()
    assert (to_host(buf[1:], np.uint64) == want).all()
    assert nb.device_errors() == 0


def test_pointwise_and_bitrev(torch_cuda):
    n = 1 << 12
    for q in (BABYBEAR, Q60):
        a, b = rand(n, q, 1), rand(n, q, 2)
        plan = nb.Plan(n, q)
        da, db = to_dev(torch_cuda, a), to_dev(torch_cuda, b)
        out = torch_cuda.empty_like(da)
        plan.pointwise_mul(out, da, db)
        torch_cuda.cuda.synchronize()
        assert (to_host(out, np.uint64) == O.pointwise(a, b, q)).all()
    nb.bit_reverse_u64(da, n)
    torch_cuda.cuda.synchronize()
    assert (to_host(da, np.uint64) == O.bit_reverse(a)).all()


def test_negacyclic_polymul_through_dropin_ops(torch_cuda):
    """Cyclic drop-in ops compose to a cyclic convolution (the reference's
    test_polynomial_multiplication is negacyclic and skipped; see RNS tests)."""
    n, q = 256, BABYBEAR
    a, b = rand(n, q, 11), rand(n, q, 12)
    plan = nb.Plan(n, q)
    da, db = to_dev(torch_cuda, a), to_dev(torch_cuda, b)
    plan.transform(da)
    plan.transform(db)
    out = torch_cuda.empty_like(da)
    plan.pointwise_mul(out, da, db)
    plan.transform(out, inverse=True)
    torch_cuda.cuda.synchronize()
    cyc = np.zeros(n, dtype=object)
    for i in range(n):
        cyc[(i + np.arange(n)) % n] += int(a[i]) * b.astype(object)
    assert (to_host(out, np.uint64) == np.array([int(v) % q for v in cyc], dtype=np.uint64)).all()


@pytest.mark.skipif(O.ref() is None, reason="reference library not built")
@pytest.mark.parametrize("n,op", [(4096, 4), (1 << 16, 4), (4096, 5), (1 << 16, 5), (1024, 0), (1024, 1),
                                  (4096, 2), (4096, 3)])
def test_vs_reference_gpu_kernels(torch_cuda, n, op):
    """Same bytes in, same bytes out as the reference's own kernels (compiled for sm_100a).
    op: 0/1 basic fwd/inv, 2/3 four-step fwd/inv (n=4096: the reference's race-free size),
    4/5 optimized fwd/inv."""
    R = O.ref()
    x = O.ref_random_polynomial(n, BABYBEAR, 42)
    cfg = R.ref_ntt_init(n, BABYBEAR)
    d_ref = to_dev(torch_cuda, x)
    R.ref_ntt_run(cfg, d_ref.data_ptr(), op)
    torch_cuda.cuda.synchronize()
    R.ref_ntt_cleanup(cfg)
    plan = nb.Plan(n, BABYBEAR)
    d = to_dev(torch_cuda, x)
    if op in (2, 3):
        plan.four_step(d, inverse=(op == 3))
    else:
        plan.transform(d, inverse=(op % 2 == 1), engine="scalar" if op < 2 else "auto")
    torch_cuda.cuda.synchronize()
    assert (to_host(d, np.uint64) == to_host(d_ref, np.uint64)).all()


@pytest.mark.skipif(O.ref() is None or not hasattr(O.ref(), "ref_ntt_rns_optimized"),
                    reason="reference library not built")
def test_reference_optimized_on_rns_moduli(torch_cuda):
    """The reference's ntt_forward_optimized / ntt_inverse_optimized over the
    24 distinct 31-bit moduli of the RNS batch (one ntt_init per modulus,
    queued on one stream, no synchronisation inside) give the same bytes as
    this library's uint64 transform per limb, and the round trip returns the input."""
    import ctypes
    R = O.ref()
    n, limbs = 1 << 16, 24
    qs = nb.generate_primes(31, 17, limbs)
    x = np.stack([rand(n, int(q), 500 + l) for l, q in enumerate(qs)])
    cfgs = (ctypes.c_void_p * limbs)(*[R.ref_ntt_init(n, int(q)) for q in qs])
    stream = torch_cuda.cuda.Stream()
    try:
        d = to_dev(torch_cuda, x.reshape(-1))
        R.ref_ntt_rns_optimized(cfgs, limbs, 1, ctypes.c_void_p(d.data_ptr()), 0, stream.cuda_stream)
        torch_cuda.cuda.synchronize()
        fwd = to_host(d, np.uint64).reshape(limbs, n)
        R.ref_ntt_rns_optimized(cfgs, limbs, 1, ctypes.c_void_p(d.data_ptr()), 1, stream.cuda_stream)
        torch_cuda.cuda.synchronize()
        assert (to_host(d, np.uint64).reshape(limbs, n) == x).all()
    finally:
        for c in cfgs:
            R.ref_ntt_cleanup(c)
    for l, q in enumerate(qs):
        ours = run_u64(torch_cuda, nb.Plan(n, int(q)), x[l])
        assert (ours == fwd[l]).all(), "limb %d (q=%d) mismatches: %d" % (l, q, int((ours != fwd[l]).sum()))


@pytest.mark.parametrize("lg", [1, 5, 9, 10, 11, 14, 20])
def test_bit_reverse_every_path(torch_cuda, lg):
    """In-place bit reversal: the element-wise kernel below 2^10, the tiled one
    (32 x 32 tiles swapped through shared memory) from 2^10 on."""
    n = 1 << lg
    x = np.random.default_rng(lg).integers(0, 1 << 62, n, dtype=np.uint64)
    d = to_dev(torch_cuda, x)
    nb.bit_reverse_u64(d, n)
    torch_cuda.cuda.synchronize()
    assert (to_host(d, np.uint64) == O.bit_reverse(x)).all()
