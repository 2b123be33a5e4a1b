"""GPU: the NTT_PHASE_PROFILE build (ntt_b200/libntt_b200_phase.so) of the
INT8 cluster kernel.  Its phase counters must not change a result: the
24-limb 2^16 negacyclic step runs in a fresh process on that library, the
forward equals the oracle, forward + inverse returns the input, and every
counter the profile case reports has been advanced."""
import json
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CASE = r'''
import json, sys
import numpy as np
import torch
sys.path[:0] = [ROOT, ROOT + "/ntt-tensorcore_b200"]
import ntt_b200 as nb
from oracle import oracle as O
assert nb.LIB_PATH.endswith("libntt_b200_phase.so")
rng = np.random.default_rng(5)
qs = nb.generate_primes(31, 17, 24)
x = np.stack([rng.integers(0, q, 1 << 16, dtype=np.uint64) for q in qs]).astype(np.uint32)
plan = nb.RnsPlan(16, qs, negacyclic=True)
d = torch.from_numpy(x.reshape(-1).view(np.int32)).cuda()
o = torch.empty_like(d)
nb.phase_profile(clear=True)
plan.transform(o, d, 1, engine="int8")
plan.forward_inverse(d, 1, engine="int8")
torch.cuda.synchronize()
enabled, ph = nb.phase_profile(clear=True)
want = O.rns(x[None].astype(np.uint64), qs, negacyclic=True)[0]
fwd = bool((o.cpu().numpy().view(np.uint32).reshape(x.shape).astype(np.uint64) == want).all())
rt = bool((d.cpu().numpy().view(np.uint32).reshape(x.shape) == x).all())
print(json.dumps({"enabled": enabled, "phases": ph, "fwd": fwd, "round_trip": rt, "errors": nb.device_errors()}))
'''


def test_phase_profile_build_is_exact_and_counts():
    env = dict(os.environ, NTT_B200_LIB="phase")
    r = subprocess.run([sys.executable, "-c", "ROOT = %r\n" % ROOT + CASE], capture_output=True, text=True,
                       env=env, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    out = json.loads(r.stdout.strip().splitlines()[-1])
    assert out["enabled"] and out["fwd"] and out["round_trip"] and out["errors"] == 0, out
    ph = out["phases"]
    assert ph["ctas"] == 2 * 96  # two launches of 24 four-CTA clusters
    for k in ("mma_wait", "tmem_load", "part_sync_send", "level2_mma", "stages", "cta_lifetime"):
        assert ph[k] > 0, (k, ph)
    assert ph["stages"] > ph["mma_wait"] + ph["tmem_load"]
