"""GPU: the NTT_DEBUG_BOUNDS build (ntt_b200/libntt_b200_dbg.so), the
stand-in for a memory checker.  Every hand-computed index of the INT8
cluster kernel (column loads, swizzled shared-memory staging, the
distributed-shared-memory piece copies, the final stores), of the DMMA
passes, of the uneven-batch queue (tickets, units, tiles, workspace slots)
and of the 64-bit byte-plane engine is range-checked there, and every output
residue is checked to be reduced.  Small cases of each run in a fresh
process on that library: the results equal the oracle's and no check fails."""
import json
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CASES = r'''
import json, sys
import numpy as np
import torch
sys.path[:0] = [ROOT, ROOT + "/ntt-tensorcore_b200"]
import ntt_b200 as nb
from oracle import oracle as O
assert nb.LIB_PATH.endswith("libntt_b200_dbg.so")
out = {}
rng = np.random.default_rng(3)
qs = nb.generate_primes(31, 17, 4)
x = np.stack([rng.integers(0, q, 1 << 16, dtype=np.uint64) for q in qs]).astype(np.uint32)
want = O.rns(x[None].astype(np.uint64), qs, negacyclic=True)[0]
plan = nb.RnsPlan(16, qs, negacyclic=True)
for eng in ("int8", "dmma"):
    d = torch.from_numpy(x.reshape(-1).view(np.int32)).cuda()
    o = torch.empty_like(d)
    plan.transform(o, d, 1, engine=eng)
    plan.forward_inverse(d, 1, engine=eng)
    torch.cuda.synchronize()
    out[eng] = bool((o.cpu().numpy().view(np.uint32).reshape(x.shape).astype(np.uint64) == want).all()) and \
        bool((d.cpu().numpy().view(np.uint32).reshape(x.shape) == x).all())
bq = nb.generate_primes(31, 21, 6)
bp = nb.BatchPlan(bq, 17, negacyclic=True)
jobs, hosts = [], []
for lg, limbs, inv, nega in ((5, 2, False, True), (11, 3, True, False), (13, 2, False, True), (14, 1, True, True),
                             (17, 2, False, False), (16, 3, True, True)):
    h = np.stack([rng.integers(0, q, 1 << lg, dtype=np.uint64) for q in bq[:limbs]]).astype(np.uint32)
    jobs.append((torch.from_numpy(h.reshape(-1).view(np.int32)).cuda(), lg, limbs, 0, inv, nega))
    hosts.append(h)
for cfg in ({"tensor": 1}, {"tensor": 0}):
    ds = [j[0].clone() for j in jobs]
    bp.batch([(d,) + j[1:] for d, j in zip(ds, jobs)], cfg).launch()
    torch.cuda.synchronize()
    ok = True
    for d, j, h in zip(ds, jobs, hosts):
        w = O.rns(h[None].astype(np.uint64), bq[:j[2]], negacyclic=j[5], inverse=j[4])[0]
        ok = ok and bool((d.cpu().numpy().view(np.uint32).reshape(h.shape).astype(np.uint64) == w).all())
    out["batch_tensor%d" % cfg["tensor"]] = ok
q60 = 1152921504577486849
x60 = rng.integers(0, q60, 1 << 20, dtype=np.uint64)
wp = nb.WidePlan(20, [q60])
d = torch.from_numpy(x60.view(np.int64)).cuda()
o = torch.empty_like(d)
wp.transform(o, d, 1, engine="int8")
torch.cuda.synchronize()
out["wide"] = bool((o.cpu().numpy().view(np.uint64) == O.ntt(x60, q60)).all())
enabled, flags = nb.bounds_errors()
out.update(enabled=enabled, flags=flags, device_errors=nb.device_errors())
print(json.dumps(out))
'''


def test_debug_bounds_build_runs_every_engine_clean(torch_cuda):
    lib = os.path.join(ROOT, "ntt-tensorcore_b200", "ntt_b200", "libntt_b200_dbg.so")
    assert os.path.exists(lib), "build it with `python ntt-tensorcore_b200/build.py --debug-bounds`"
    env = dict(os.environ, NTT_B200_LIB="dbg")
    r = subprocess.run([sys.executable, "-c", "ROOT = %r\n" % ROOT + CASES], env=env, capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stderr[-3000:]
    got = json.loads(r.stdout.strip().splitlines()[-1])
    assert got == {"int8": True, "dmma": True, "batch_tensor1": True, "batch_tensor0": True, "wide": True,
                   "enabled": True, "flags": 0, "device_errors": 0}, got
