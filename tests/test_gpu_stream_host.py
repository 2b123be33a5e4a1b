"""GPU: nttb_rns_stream_host -- batches in host memory streamed through the
GPU (copies overlapping the transforms) give, batch by batch, the oracle's
transforms and round trips; the copies of neighbouring batches do not mix."""
import numpy as np
import pytest

from oracle import oracle as O
import ntt_b200 as nb

pytestmark = pytest.mark.gpu


def host_batches(torch, rng, qs, lg, n_polys, n_batches):
    x = np.stack([np.stack([rng.integers(0, q, 1 << lg, dtype=np.uint64) for q in qs]) for _ in range(n_batches * n_polys)])
    x = x.astype(np.uint32)
    t = torch.from_numpy(x.reshape(-1).view(np.int32)).pin_memory()
    return x, t


@pytest.mark.parametrize("mode", ["forward", "inverse", "forward_inverse"])
def test_stream_host_vs_oracle(torch_cuda, mode):
    torch = torch_cuda
    rng = np.random.default_rng(71)
    qs = nb.generate_primes(31, 17, 3)
    plan = nb.RnsPlan(16, qs, negacyclic=True)
    x, h_in = host_batches(torch, rng, qs, 16, 2, 5)  # 5 batches of 2 polys, distinct data
    h_out = torch.empty_like(h_in).pin_memory()
    s = torch.cuda.Stream()
    plan.stream_host(h_in, h_out, 2, 5, mode=mode, stream=s)
    s.synchronize()
    got = h_out.numpy().view(np.uint32).reshape(x.shape)
    if mode == "forward_inverse":
        assert (got == x).all()
    else:
        want = O.rns(x.astype(np.uint64), qs, negacyclic=True, inverse=(mode == "inverse"))
        assert (got.astype(np.uint64) == want).all()
    assert nb.device_errors() == 0


@pytest.mark.parametrize("lg,engine", [(16, "dmma"), (12, "scalar"), (5, "scalar"), (16, "int8")])
def test_stream_host_engines_and_small_batches(torch_cuda, lg, engine):
    """Other sizes and engines, one polynomial per batch (a 2^5 batch is
    smaller than one copy chunk), several calls on the same plan."""
    torch = torch_cuda
    rng = np.random.default_rng(72 + lg)
    qs = nb.generate_primes(31, 17, 2)
    plan = nb.RnsPlan(lg, qs, negacyclic=False)
    for n_batches in (1, 4, 7):
        x, h_in = host_batches(torch, rng, qs, lg, 1, n_batches)
        h_out = torch.empty_like(h_in).pin_memory()
        plan.stream_host(h_in, h_out, 1, n_batches, mode="forward", engine=engine)
        torch.cuda.synchronize()
        want = O.rns(x.astype(np.uint64), qs, negacyclic=False)
        assert (h_out.numpy().view(np.uint32).reshape(x.shape).astype(np.uint64) == want).all(), n_batches


@pytest.mark.parametrize("mode", ["forward", "forward_inverse"])
def test_stream_host_on_tensor_tiles(torch_cuda, mode):
    """2^20 residues per batch route AUTO to the batch queue's tensor tiles:
    each of the three staging buffers gets its own prepared queue, and five
    batches in a row still give the oracle's transforms and round trips."""
    torch = torch_cuda
    rng = np.random.default_rng(73)
    qs = nb.generate_primes(31, 21, 2)
    plan = nb.RnsPlan(19, qs, negacyclic=True)  # 1 poly x 2 limbs x 2^19 = 2^20 residues
    x, h_in = host_batches(torch, rng, qs, 19, 1, 5)
    h_out = torch.empty_like(h_in).pin_memory()
    nb.profile_start()
    plan.stream_host(h_in, h_out, 1, 5, mode=mode)
    torch.cuda.synchronize()
    assert "batch_queue" in nb.profile_stop()
    got = h_out.numpy().view(np.uint32).reshape(x.shape)
    if mode == "forward_inverse":
        assert (got == x).all()
    else:
        want = O.rns(x.astype(np.uint64), qs, negacyclic=True)
        assert (got.astype(np.uint64) == want).all()
    assert nb.device_errors() == 0


def test_stream_host_rejects(torch_cuda):
    qs = nb.generate_primes(31, 17, 1)
    plan = nb.RnsPlan(12, qs)
    buf = np.zeros(1 << 12, dtype=np.uint32)
    with pytest.raises(nb.NTTError):
        plan.stream_host(buf, buf, 1, 1, mode="forward", engine="int8")  # the INT8 engine serves 2^16 only
