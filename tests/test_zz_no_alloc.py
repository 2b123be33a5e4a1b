"""GPU: the allocation-free in-place transform (nttb_rns_transform_noalloc).

Some callers cannot call cudaMalloc while they transform: a memory manager
that owns every byte of device memory, a loop that must never enter the
allocator (cudaMalloc can synchronize the whole device), or a process with a
fixed up-front budget.  For them the library stages the first pass in a static
device buffer instead of a plan workspace.  This file checks that entry point
through the C ABI against the ordinary entry point (nttb_rns_transform) on two
calls in a row, exact to the last bit (the tolerance of every test here), and
that oversized batches are refused.  It is collected last so that a run that
stops at the first failure has run every other test first; it also passes
alone in a fresh process (where its first call does the per-device set-up).
"""
import ctypes

import numpy as np
import pytest

from conftest import to_dev, to_host
import ntt_b200 as nb

pytestmark = pytest.mark.gpu

SCRATCH_BYTES = 8 << 20


def batch(moduli, n, n_polys, seed):
    rng = np.random.default_rng(seed)
    x = np.empty((n_polys, len(moduli), n), dtype=np.uint32)
    for l, q in enumerate(moduli):
        x[:, l, :] = rng.integers(0, q, (n_polys, n), dtype=np.uint64).astype(np.uint32)
    return x


def regular(torch, plan, x, inverse):
    d = to_dev(torch, x.reshape(-1))
    plan.transform(d, d, x.shape[0], inverse=inverse)
    torch.cuda.synchronize()
    return to_host(d, np.uint32).reshape(x.shape)


def noalloc(torch, plan, x, inverse):
    d = to_dev(torch, x.reshape(-1))
    rc = nb.lib().nttb_rns_transform_noalloc(plan._h, d.data_ptr(), x.shape[0], int(inverse), None)
    assert rc == 0, nb.lib().nttb_last_error()
    torch.cuda.synchronize()
    return to_host(d, np.uint32).reshape(x.shape)


def test_noalloc_matches_regular_entry_point_twice(torch_cuda):
    # 24 limbs x 2^16 (6 MiB of staging) negacyclic: the bench configuration
    moduli = nb.generate_primes(31, 17, 24)
    plan = nb.RnsPlan(16, moduli, negacyclic=True)
    x1 = batch(moduli, 1 << 16, 1, 1)
    x2 = batch(moduli, 1 << 16, 1, 2)
    y1 = noalloc(torch_cuda, plan, x1, False)       # first call (per-device set-up)
    assert (y1 == regular(torch_cuda, plan, x1, False)).all()
    y2 = noalloc(torch_cuda, plan, x2, False)       # second call reuses the buffer
    assert (y2 == regular(torch_cuda, plan, x2, False)).all()
    z = noalloc(torch_cuda, plan, y2, True)
    assert (z == regular(torch_cuda, plan, y2, True)).all()
    assert (z == x2).all()


def test_noalloc_smaller_and_cyclic(torch_cuda):
    moduli = nb.generate_primes(31, 21, 3)
    plan = nb.RnsPlan(20, moduli, negacyclic=False)   # 3 x 2^20 words = 12 MiB > scratch: one poly of 2 limbs fits
    small = nb.RnsPlan(20, moduli[:2], negacyclic=False)
    x = batch(moduli[:2], 1 << 20, 1, 3)
    for _ in range(2):
        assert (noalloc(torch_cuda, small, x, False) == regular(torch_cuda, small, x, False)).all()
    big = batch(moduli, 1 << 20, 1, 4)
    d = to_dev(torch_cuda, big.reshape(-1))
    rc = nb.lib().nttb_rns_transform_noalloc(plan._h, d.data_ptr(), 1, 0, None)
    assert rc == 1
    assert b"static scratch holds" in nb.lib().nttb_last_error()


def test_noalloc_rejects_oversized_batch(torch_cuda):
    moduli = nb.generate_primes(31, 17, 24)
    plan = nb.RnsPlan(16, moduli, negacyclic=True)
    x = batch(moduli, 1 << 16, 2, 5)  # 12 MiB of staging
    assert x.nbytes > SCRATCH_BYTES
    d = to_dev(torch_cuda, x.reshape(-1))
    rc = nb.lib().nttb_rns_transform_noalloc(plan._h, d.data_ptr(), 2, 0, None)
    assert rc == 1
    assert b"static scratch holds" in nb.lib().nttb_last_error()
    before = to_host(d, np.uint32)
    assert (before == x.reshape(-1)).all()  # refused before touching the data


def test_noalloc_wrapper_on_a_side_stream(torch_cuda):
    # the Python wrapper (RnsPlan.transform_noalloc) on a non-default stream,
    # two calls in a row, against the ordinary entry point
    moduli = nb.generate_primes(31, 17, 4)
    plan = nb.RnsPlan(16, moduli, negacyclic=True)
    side = torch_cuda.cuda.Stream()
    for seed in (6, 7):
        x = batch(moduli, 1 << 16, 1, seed)
        d = to_dev(torch_cuda, x.reshape(-1))
        torch_cuda.cuda.synchronize()
        plan.transform_noalloc(d, 1, inverse=False, stream=side)
        side.synchronize()
        assert (to_host(d, np.uint32).reshape(x.shape) == regular(torch_cuda, plan, x, False)).all()


def test_noalloc_one_pass_shapes_are_not_limited(torch_cuda):
    # 2^10 words x 24 limbs x 400 polynomials = 37.5 MiB: a one-pass shape
    # stages nothing, so the scratch limit does not apply
    moduli = nb.generate_primes(31, 17, 24)
    plan = nb.RnsPlan(10, moduli, negacyclic=True)
    x = batch(moduli, 1 << 10, 400, 8)
    assert x.nbytes > SCRATCH_BYTES
    assert (noalloc(torch_cuda, plan, x, False) == regular(torch_cuda, plan, x, False)).all()
