"""The multi-rank host logic of bench.py on CPU: two gloo ranks on 127.0.0.1.

bench.py runs one process per GPU (torchrun); its timings are the max over
ranks, replica throughputs the sum, and the reference arm runs on rank 0
alone.  No GPU is involved: with none visible the process group is gloo."""
import json
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _reduce_worker(rank, world, port, out_dir):
    import datetime

    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    got = {
        "max": bench.reduce_over_ranks(1.5 + rank, world, "max"),
        "sum": bench.reduce_over_ranks(1.5 + rank, world, "sum"),
    }
    bench.rank_barrier(world)
    with open(os.path.join(out_dir, "rank%d.json" % rank), "w") as f:
        json.dump(got, f)
    dist.destroy_process_group()


def test_reduce_over_ranks_two_gloo_ranks(tmp_path):
    import torch.multiprocessing as mp

    mp.start_processes(_reduce_worker, args=(2, free_port(), str(tmp_path)), nprocs=2, start_method="spawn")
    for rank in (0, 1):
        got = json.load(open(tmp_path / ("rank%d.json" % rank)))
        assert got == {"max": 2.5, "sum": 4.0}


def test_reduce_over_ranks_single_rank_is_identity():
    sys.path.insert(0, ROOT)
    import bench

    assert bench.reduce_over_ranks(3.25, 1) == 3.25
    bench.rank_barrier(1)  # no process group: a no-op


@pytest.mark.skipif(not os.path.exists(os.path.join(ROOT, "oracle", "_ref", "libntt_ref.so"))
                    and not os.path.exists(os.path.join(ROOT, "oracle", "liboracle.so")),
                    reason="oracle not built")
def test_reference_arm_under_torchrun_two_ranks():
    """`bench.py --impl reference` launched the way the driver launches N > 1:
    rank 0 alone runs the reference and prints one JSON line; both ranks exit 0."""
    env = dict(os.environ, CUDA_VISIBLE_DEVICES="")
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes", "1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(free_port()),
           os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2", "--steps", "1", "--warmup", "0"]
    r = subprocess.run(cmd, cwd=ROOT, env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-3000:]
    lines = [json.loads(l) for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, r.stdout
    line = lines[0]
    assert line["impl"] == "reference" and line["n_gpus"] == 2
    assert line["value"] > 0 and line["cpu_baseline"]["cores"] >= 1
    assert "reference_gpu" not in line  # no GPU visible
    assert line["config"] == __import__("bench").headline_config(2)  # the same config as the measured arm
    assert line["ms_per_step"] > 0


def test_reference_arm_does_not_load_the_library():
    """The reference arm computes its moduli in pure Python: running it loads
    no libntt_b200.so (only the oracle's libraries)."""
    env = dict(os.environ, CUDA_VISIBLE_DEVICES="")
    code = ("import sys, json; sys.argv = ['bench.py', '--impl', 'reference', '--steps', '1', '--warmup', '0'];"
            "sys.path.insert(0, %r); import bench; bench.main();"
            "maps = open('/proc/self/maps').read();"
            "print(json.dumps({'dropin_loaded': 'libntt_b200' in maps}))" % ROOT)
    r = subprocess.run([sys.executable, "-c", code], cwd=ROOT, env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-3000:]
    last = json.loads(r.stdout.strip().splitlines()[-1])
    assert last == {"dropin_loaded": False}


def test_workload_primes_match_the_library():
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "ntt-tensorcore_b200"))
    import bench
    import ntt_b200 as nb

    for bits, adic, count in ((31, 17, 24), (31, 21, 32), (31, 18, 48), (62, 21, 3)):
        assert bench.workload_primes(bits, adic, count) == nb.generate_primes(bits, adic, count)
