#!/usr/bin/env python
"""NTT throughput on B200: the 24-limb RNS negacyclic batch.

Workload (one step): 24 distinct 31-bit primes q == 1 mod 2^17, N = 2^16 per
limb, uint32 residues uniform in [0, q); a negacyclic forward NTT over the
whole batch followed by the inverse, through the C ABI (nttb_rns_transform).
`value` counts coefficient-transforms per second over all ranks
(2 transforms x 24 limbs x 2^16 coefficients per step and GPU).

Inputs rotate through a pool of batches larger than twice the 126 MB L2, so
no step finds its input in L2.  Multi-GPU runs are independent replicas
(the path shards by limb and polynomial with no exchange); the timing is the
max over ranks.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--engine auto|int8|dmma|scalar]
"""
import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "ntt-tensorcore_b200"))
sys.path.insert(0, ROOT)

LOG_N = 16
N_LIMBS = 24
TWO_ADICITY = 17
L2_BYTES = 126 * 2 ** 20
METRIC = "NTT coeffs/s + HBM GB/s, INT8-limb vs FP64-DMMA (bit-exact); serve p50/p99"
UNIT = "coeff-transforms/s"
WORKLOAD = "rns_negacyclic_24x2^16_fwd+inv"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--engine", default="auto", choices=["auto", "int8", "dmma", "scalar"])
    ap.add_argument("--workload", default="rns", choices=["rns", "uneven", "serve", "q60", "aux"],
                    help="rns: the 24-limb 2^16 negacyclic batch (headline); uneven: 512 polynomials of "
                         "2^12..2^20 residues, 1..32 limbs, mixed directions, one persistent launch; "
                         "serve: Poisson stream of negacyclic products under a 60 GB budget, p50/p99; "
                         "q60: the 60-bit prime at N = 2^20, cyclic forward + inverse; aux: the helper "
                         "kernels (transposes, bit reversal, pointwise products) against the HBM roofline")
    ap.add_argument("--serve-seconds", type=float, default=3.0, help="seconds per load level (serve)")
    ap.add_argument("--profile-case", choices=["int8", "int8_phases", "dmma", "batch", "batch_tc", "q60", "move", "klimb"],
                    default=None,
                    help="run one small profiling case and exit (the workloads the profiles/ captures use)")
    ap.add_argument("--no-compare", action="store_true", help="skip the per-engine comparison lines")
    ap.add_argument("--no-secondary", action="store_true",
                    help="skip the secondary workloads (q60, uneven, serve) that a single-GPU default run "
                         "measures after the headline and reports under `secondary`")
    ap.add_argument("--quick", action="store_true",
                    help="warm-up + timed steps only (no clock soak, e2e, comparisons or CPU leg): "
                         "the short run used under ncu")
    return ap.parse_args()


def dist_setup(args):
    """One process per GPU (torchrun): NCCL on GPUs, gloo where none is visible
    (the host-side logic of the multi-rank path runs on CPU that way)."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        backend = "nccl" if torch.cuda.is_available() else "gloo"
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
    return world, rank, local


def reduce_over_ranks(x, world, op="max"):
    """max (times, latencies) or sum (replica throughput) of a per-rank number
    over all ranks.  Every rank calls it, in the same order."""
    if world <= 1:
        return x
    import torch
    import torch.distributed as dist
    dev = torch.device("cuda", torch.cuda.current_device()) if torch.cuda.is_available() else torch.device("cpu")
    t = torch.tensor([float(x)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX if op == "max" else dist.ReduceOp.SUM)
    return float(t.item())


def rank_barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def _is_prime(n):
    """Deterministic Miller-Rabin for n < 2^64 (the first twelve prime bases)."""
    if n < 2:
        return False
    small = (2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37)
    for p in small:
        if n % p == 0:
            return n == p
    d, r = n - 1, 0
    while d % 2 == 0:
        d //= 2
        r += 1
    for a in small:
        x = pow(a, d, n)
        if x in (1, n - 1):
            continue
        for _ in range(r - 1):
            x = x * x % n
            if x == n - 1:
                break
        else:
            return False
    return True


def workload_primes(bits, two_adicity, count):
    """The workload's moduli: the `count` largest primes q < 2^bits with
    q == 1 mod 2^two_adicity, in descending order (the rule of the library's
    nttb_generate_primes, restated here so that the reference arm computes its
    moduli without loading the library)."""
    step = 1 << two_adicity
    out, k = [], ((1 << bits) - 1) // step
    while k > 0 and len(out) < count:
        q = k * step + 1
        if q < (1 << bits) and _is_prime(q):
            out.append(q)
        k -= 1
    if len(out) < count:
        raise ValueError("only %d primes exist" % len(out))
    return out


def moduli():
    return workload_primes(31, TWO_ADICITY, N_LIMBS)


def headline_config(world):
    """The workload description shared by both arms' JSON lines."""
    batch_bytes = N_LIMBS * (1 << LOG_N) * 4
    pool_n = max(8, int(np.ceil(2.4 * L2_BYTES / batch_bytes)))
    return {"workload": WORKLOAD, "n": 1 << LOG_N, "limbs": N_LIMBS, "moduli": "31-bit, q == 1 mod 2^17",
            "negacyclic": True, "transforms_per_step": 2,
            "l2": "inputs rotate through %d batches (%d MB of uint32 residues) > 2x L2" % (pool_n, pool_n * batch_bytes >> 20),
            "parallelism": "replicas x%d" % world}


def load_peaks():
    """(peaks dict, source) from MEASURED_PEAKS.json, else the fallback figures."""
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            peaks = json.load(f)
        if "hbm_gbs" in peaks:
            return peaks, "measured (MEASURED_PEAKS.json hbm_gbs)"
    except (OSError, ValueError):
        pass
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}, "fallback (6650 GB/s: no MEASURED_PEAKS.json on this host)"


def make_batch(qs, seed):
    rng = np.random.default_rng(seed)
    x = np.empty((N_LIMBS, 1 << LOG_N), dtype=np.uint32)
    for l, q in enumerate(qs):
        x[l] = rng.integers(0, q, 1 << LOG_N, dtype=np.uint64).astype(np.uint32)
    return x


# ------------------------------------------------------------------ clocks
class ClockSampler:
    """nvidia-smi sampling of SM clock and throttle reasons while running."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index):
        self.dev = device_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.dev), "--query-gpu=" + self.FIELDS, "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except FileNotFoundError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sms, maxes, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sms.append(float(parts[1]))
                maxes.append(float(parts[2]))
            except ValueError:
                continue
            for name, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sms) if sms else None,
                "sm_max_mhz": max(maxes) if maxes else None,
                "samples": len(sms),
                "reasons": sorted(reasons)}


# ------------------------------------------------------------- reference arm
def cpu_reference(qs, steps, warmup, threads=0):
    """The reference's ntt_host (oracle/_ref, compiled from the reference
    sources) over the same batch on all host threads; one step = the full
    batch forward + inverse with the driver's psi twist."""
    from oracle import oracle as O
    kind = "reference" if O.ref() is not None else "port"
    x = make_batch(qs, 1).astype(np.uint64)
    coeffs = 2 * N_LIMBS * (1 << LOG_N)

    def one():
        y = x.copy()
        if kind == "reference":
            used = O.ref_host_batch(y, qs, inverse=False, negacyclic=True, threads=threads)
            O.ref_host_batch(y, qs, inverse=True, negacyclic=True, threads=threads)
        else:
            y = O.rns(y, qs, negacyclic=True)
            y = O.rns(y, qs, negacyclic=True, inverse=True)
            used = 1
        return used, y

    for _ in range(warmup):
        one()
    t0 = time.perf_counter()
    for _ in range(steps):
        used, y = one()
    dt = time.perf_counter() - t0
    assert (y == x).all(), "reference round trip failed"
    return {"value": coeffs * steps / dt, "unit": UNIT, "cores": used, "kind": kind,
            "sample": "%d x (24 limbs x 2^16 negacyclic forward+inverse)" % steps, "seconds": dt}


def reference_gpu_bar(qs, steps, warmup, device=0):
    """The reference's own GPU kernels on the same workload: ntt_init per
    modulus, then ntt_forward_optimized + ntt_inverse_optimized on every limb
    (oracle/_ref, the reference sources compiled unmodified for sm_100a), in
    the reference's uint64 words, queued on one stream and timed with CUDA
    events.  The reference has no negacyclic code, so this is the cyclic
    transform: the same data volume with the psi twist left out.  The
    forward is checked against the reference's ntt_host on the same batch."""
    import torch
    from oracle import oracle as O
    R = O.ref()
    if R is None or not hasattr(R, "ref_ntt_rns_optimized"):
        return {"unavailable": "reference library oracle/_ref/libntt_ref.so not built (or built without "
                               "ref_ntt_rns_optimized; rerun __graft_entry__.build())"}
    torch.cuda.set_device(device)
    dev = torch.device("cuda", device)
    stream = torch.cuda.Stream(device=dev)
    n = 1 << LOG_N
    cfgs = (ctypes.c_void_p * N_LIMBS)(*[R.ref_ntt_init(n, int(q)) for q in qs])
    try:
        batch_bytes = N_LIMBS * n * 8
        pool_n = max(8, int(np.ceil(2.4 * L2_BYTES / batch_bytes)))
        host = [make_batch(qs, 2000 + i).astype(np.uint64) for i in range(4)]
        pool = torch.empty((pool_n, N_LIMBS * n), dtype=torch.int64, device=dev)
        for i in range(pool_n):
            pool[i].copy_(torch.from_numpy(host[i % 4].reshape(-1).view(np.int64)))
        torch.cuda.synchronize()

        def run(buf, which):
            R.ref_ntt_rns_optimized(cfgs, N_LIMBS, 1, ctypes.c_void_p(buf.data_ptr()), which, stream.cuda_stream)

        # parity: the forward of one batch against ntt_host on the host
        probe = pool[0].clone()
        run(probe, 0)
        torch.cuda.synchronize()
        want = host[0].copy()
        O.ref_host_batch(want, qs, inverse=False, negacyclic=False)
        forward_ok = bool((probe.cpu().numpy().view(np.uint64) == want.reshape(-1)).all())
        del probe
        for i in range(max(3, warmup)):
            run(pool[i % pool_n], 2)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for i in range(steps):
            run(pool[i % pool_n], 2)
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        round_trip_ok = all((pool[i].cpu().numpy().view(np.uint64) == host[i % 4].reshape(-1)).all()
                            for i in range(min(pool_n, 4)))
    finally:
        for c in cfgs:
            R.ref_ntt_cleanup(c)
    coeffs = 2 * N_LIMBS * n
    log_inner = 6
    launches = N_LIMBS * (2 * (1 + LOG_N % log_inner + LOG_N // log_inner) + 1)
    return {"value": coeffs * steps / (ms / 1e3), "unit": UNIT, "ms_per_step": ms / steps, "steps": steps,
            "kernels": "ntt_forward_optimized + ntt_inverse_optimized per limb (cyclic; uint64 words)",
            "launches_per_step": launches, "forward_matches_ntt_host": forward_ok,
            "round_trip_ok": bool(round_trip_ok), "l2": "pool of %d batches (%.0f MB) > L2" %
            (pool_n, pool_n * batch_bytes / 1e6)}


def bounded_cpu_baseline(qs, budget_s=10.0):
    """cpu_baseline: the reference CPU NTT on a bounded sample (~budget_s of wall time)."""
    probe = cpu_reference(qs, 1, 0)
    steps = max(1, int(budget_s / max(probe["seconds"], 1e-3)))
    steps = min(steps, 200)
    r = cpu_reference(qs, steps, 0)
    r.pop("seconds")
    return r


# ---------------------------------------------------------------- our arm
def run_ours(args, world, rank, local):
    import torch
    import ntt_b200 as nb

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    stream = torch.cuda.Stream(device=dev)
    qs = moduli()
    plan = nb.RnsPlan(LOG_N, qs, negacyclic=True)
    batch_bytes = N_LIMBS * (1 << LOG_N) * 4
    pool_n = max(8, int(np.ceil(2.4 * L2_BYTES / batch_bytes)))
    host = [make_batch(qs, 1000 + i) for i in range(4)]
    pool = torch.empty((pool_n, N_LIMBS << LOG_N), dtype=torch.int32, device=dev)
    for i in range(pool_n):
        pool[i].copy_(torch.from_numpy(host[i % 4].reshape(-1).view(np.int32)))
    torch.cuda.synchronize()
    coeffs_per_step = 2 * N_LIMBS * (1 << LOG_N)

    def step(i, engine):
        buf = pool[i % pool_n]
        plan.forward_inverse(buf, 1, engine=engine, stream=stream)

    def barrier():
        if world > 1:
            import torch.distributed as dist
            dist.barrier()

    def timed(engine, steps):
        barrier()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        c0 = nb.launch_count()
        e0.record(stream)
        for i in range(steps):
            step(i, engine)
        e1.record(stream)
        torch.cuda.synchronize()
        launches = nb.launch_count() - c0
        ms = reduce_over_ranks(e0.elapsed_time(e1), world)
        barrier()
        return ms, launches

    engine = args.engine
    # warm-up (also brings the clocks up before the sampled region)
    for i in range(max(3, args.warmup)):
        step(i, engine)
    torch.cuda.synchronize()
    if args.quick:
        ms, launches = timed(engine, args.steps)
        return {"metric": METRIC, "value": world * coeffs_per_step * args.steps / (ms / 1e3), "unit": UNIT,
                "n_gpus": world, "steps": args.steps, "ms_per_step": ms / args.steps, "quick": True,
                "config": headline_config(world), "engine": engine, "gpu_launches": launches}, qs
    clocks = ClockSampler(local)
    clocks.start()
    t_end = time.time() + 1.0
    i = 0
    while time.time() < t_end:  # ~1 s of load so the sampler sees the clocks under load
        step(i, engine)
        i += 1
        if i % 50 == 0:
            torch.cuda.synchronize()
    ms, launches = timed(engine, args.steps)
    clk = clocks.stop()
    # round trip leaves every buffer unchanged: check the data is intact
    for i in range(min(pool_n, 4)):
        got = pool[i].cpu().numpy().view(np.uint32)
        assert (got == host[i % 4].reshape(-1)).all(), "round trip mismatch in buffer %d" % i
    value = world * coeffs_per_step * args.steps / (ms / 1e3)

    # per-kernel device time over the same steps (events around each library launch)
    nb.profile_start()
    for i in range(args.steps):
        step(i, engine)
    torch.cuda.synchronize()
    prof = nb.profile_stop()
    top = max(prof.items(), key=lambda kv: kv[1][1])
    k_name, (k_launches, k_ms) = top
    # Events around each launch add their own overhead, so the per-launch
    # sums run longer than the back-to-back timed loop.  The dominant
    # kernel's time is its SHARE of the event sums applied to the timed loop's
    # device time (with one kernel per step: exactly ms_per_step).
    ev_total_ms = sum(v[1] for v in prof.values())
    k_share = k_ms / ev_total_ms
    # (the profiled loop runs the same steps as the timed one)
    k_avg_s = ms * k_share / k_launches / 1e3
    # algorithmic bytes: 8 B per coefficient per transform (4 B read + 4 B
    # write of a uint32 residue).  The fused queue kernel runs two transforms
    # (x4 = forward + inverse, 4 stages) or one (x2); a single-pass kernel
    # moves the batch once.
    coeffs_per_launch = N_LIMBS * (1 << LOG_N)
    transforms = 2 if k_name.endswith("_x4") else 1
    alg_bytes = 8 * coeffs_per_launch * transforms
    peaks, peak_source = load_peaks()
    peak = peaks["hbm_gbs"]
    achieved = alg_bytes / k_avg_s / 1e9
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tpath):
        with open(tpath) as f:
            traffic = json.load(f).get(k_name)

    # end to end through the C ABI with host buffers: every step copies its
    # batch host->device from pinned memory, runs forward + inverse and copies
    # the result back -- nttb_rns_stream_host, which overlaps the copies of
    # neighbouring steps with the transforms (three device buffers, chunked
    # copies on two streams per direction).
    e_steps = max(3, min(args.steps, 30))
    h_in = torch.from_numpy(np.tile(host[0].reshape(-1), e_steps).view(np.int32)).pin_memory()
    h_out = torch.empty_like(h_in).pin_memory()
    # a first pass over the pinned buffers (device buffers, streams, and the
    # first DMA to every host page) before the timed pass
    plan.stream_host(h_in, h_out, 1, e_steps, mode="forward_inverse", engine=engine, stream=stream)
    torch.cuda.synchronize()
    barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    plan.stream_host(h_in, h_out, 1, e_steps, mode="forward_inverse", engine=engine, stream=stream)
    e1.record(stream)
    torch.cuda.synchronize()
    e_ms = reduce_over_ranks(e0.elapsed_time(e1), world)
    assert (h_out.numpy().view(np.uint32) == h_in.numpy().view(np.uint32)).all(), "e2e round trip mismatch"
    e2e = {"value": world * coeffs_per_step * e_steps / (e_ms / 1e3), "unit": UNIT,
           "h2d_bytes_per_step": batch_bytes, "d2h_bytes_per_step": batch_bytes,
           "api": "nttb_rns_stream_host (pinned host buffers, %d steps)" % e_steps}

    # engine comparison on the same workload (information; the headline is `engine`)
    compare = {}
    if not args.no_compare:
        for eng in ("int8", "dmma", "scalar"):
            if eng == engine:
                continue
            try:
                step(0, eng)
                torch.cuda.synchronize()
            except nb.NTTError:
                compare[eng] = None
                continue
            for i in range(3):
                step(i, eng)
            m, _ = timed(eng, max(10, args.steps // 2))
            compare[eng] = world * coeffs_per_step * max(10, args.steps // 2) / (m / 1e3)

    # information, not the headline: the same steps spread over two streams
    # (independent batches), so that a second launch can take the SMs the
    # first leaves idle (24 four-CTA clusters occupy 96 of the 148)
    two_streams = None
    if not args.no_compare:
        streams = [torch.cuda.Stream(device=dev), torch.cuda.Stream(device=dev)]
        for i in range(4):
            plan.forward_inverse(pool[i % pool_n], 1, engine=engine, stream=streams[i & 1])
        barrier()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for st in streams:
            st.wait_event(e0)
        for i in range(args.steps):
            plan.forward_inverse(pool[i % pool_n], 1, engine=engine, stream=streams[i & 1])
        for st in streams:
            stream.wait_stream(st)
        e1.record(stream)
        torch.cuda.synchronize()
        ms2 = reduce_over_ranks(e0.elapsed_time(e1), world)
        barrier()
        for i in range(min(pool_n, 4)):  # the concurrent round trips left every buffer intact
            got = pool[i].cpu().numpy().view(np.uint32)
            assert (got == host[i % 4].reshape(-1)).all(), "two-stream round trip mismatch in buffer %d" % i
        two_streams = {"value": world * coeffs_per_step * args.steps / (ms2 / 1e3), "unit": UNIT,
                       "ms_per_step": ms2 / args.steps,
                       "note": "steps alternate over two streams (each on its own batch); information only"}

    result = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u32", "data": "synthetic: seeded uniform residues",
        "config": headline_config(world), "engine": engine,
        "roofline": {"bound": "hbm", "kernel": k_name, "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": traffic,
                     "peak_source": peak_source,
                     "kernel_avg_us": k_avg_s * 1e6, "kernel_share": k_share,
                     "kernel_timing": "share of per-launch event time x the timed loop's device time",
                     "alg_bytes_per_launch": alg_bytes},
        "kernels": {k: {"launches": v[0], "total_ms": v[1]} for k, v in prof.items()},
        "e2e": e2e, "gpu_launches": launches, "clocks": clk,
        "engines_coeffs_per_s": dict(compare, **{engine: value}),
        "two_streams": two_streams,
    }
    return result, qs


# --------------------------------------------- reference CPU path beside
def cpu_sample(jobs, moduli, budget_s=10.0):
    """The reference's ntt_host (oracle/_ref) on all host threads over a
    bounded sample of a job mix: jobs = (log_n, limbs, inverse, negacyclic,
    product) tuples taken in order until ~budget_s of work.  Products are
    forward a, forward b, pointwise, inverse (3 transforms per residue)."""
    from oracle import oracle as O
    if O.ref() is None:
        return {"unavailable": "reference library oracle/_ref not built"}
    rng = np.random.default_rng(11)
    done, coeffs, used, t0 = 0, 0, 1, time.perf_counter()
    for lg, limbs, inv, nega, prod in jobs:
        qs = moduli[:limbs]
        q = np.array(qs, dtype=np.uint64)[:, None]
        x = (rng.integers(0, 1 << 62, (1, limbs, 1 << lg), dtype=np.uint64) % q).copy()
        if prod:
            y = (rng.integers(0, 1 << 62, (1, limbs, 1 << lg), dtype=np.uint64) % q).copy()
            used = O.ref_host_batch(x, qs, negacyclic=nega)
            O.ref_host_batch(y, qs, negacyclic=nega)
            x = np.ascontiguousarray((x * y) % q[None])  # residues < 2^31: the product fits
            O.ref_host_batch(x, qs, inverse=True, negacyclic=nega)
            coeffs += 3 * limbs << lg
        else:
            used = O.ref_host_batch(x, qs, inverse=inv, negacyclic=nega)
            coeffs += limbs << lg
        done += 1
        if time.perf_counter() - t0 > budget_s:
            break
    dt = time.perf_counter() - t0
    return {"value": coeffs / dt, "unit": UNIT, "cores": used, "kind": "reference",
            "sample": "%d jobs of the mix (ntt_host per (poly, limb), all host threads)" % done}


# ------------------------------------------------------- uneven workload
UNEVEN_JOBS = 512
UNEVEN_WORKLOAD = "uneven_512polys_logN12-20_limbs1-32_mixed_dir"


def uneven_jobs(seed=4):
    """Job shapes: log2 N ~ U{12..20}, limbs ~ U{1..32}, 50% forward / 50% inverse."""
    rng = np.random.default_rng(seed)
    lg = rng.integers(12, 21, UNEVEN_JOBS)
    limbs = rng.integers(1, 33, UNEVEN_JOBS)
    inv = rng.integers(0, 2, UNEVEN_JOBS)
    return [(int(a), int(b), bool(c)) for a, b, c in zip(lg, limbs, inv)]


def uneven_sample(shapes):
    """(job index, limb) rows checked against the oracle: the first job of
    every (log2 N, direction) class and of every limb-count bucket (1-8,
    9-16, 17-24, 25-32), limbs first, middle and last of each."""
    picked, seen = [], set()
    for i, (lg, limbs, inv) in enumerate(shapes):
        for key in (("class", lg, inv), ("bucket", (limbs - 1) // 8)):
            if key not in seen:
                seen.add(key)
                if i not in picked:
                    picked.append(i)
    return [(i, l) for i in picked for l in sorted({0, shapes[i][1] // 2, shapes[i][1] - 1})]


def uneven_check(torch, nb, plan, jobs, shapes, qs, buf, buf0, config, stream):
    """Bit-exact check of the full-size batch: restore the inputs, launch the
    batch once, compare the sampled rows with the oracle's transforms; then
    launch the batch with every direction flipped and require the inputs
    back, word for word."""
    from concurrent.futures import ThreadPoolExecutor
    from oracle import oracle as O
    buf.copy_(buf0)
    b = plan.batch(jobs, config)
    b.launch(stream)
    torch.cuda.synchronize()
    errors = nb.device_errors()
    rows = uneven_sample(shapes)

    def one(row):
        i, l = row
        view = jobs[i][0]
        got = view[l].cpu().numpy().view(np.uint32).astype(np.uint64)
        x = buf0[view.storage_offset() - buf.storage_offset():][:view.numel()].view(view.shape)[l]
        want = O.rns(x.cpu().numpy().view(np.uint32).astype(np.uint64)[None, None], [qs[l]],
                     inverse=shapes[i][2])[0, 0]
        return bool((got == want).all())

    with ThreadPoolExecutor(max_workers=max(1, min(16, os.cpu_count() or 1))) as ex:  # ctypes drops the GIL
        ok = list(ex.map(one, rows))
    b.close()
    flipped = [(v, lg, limbs, first, not inv, nega) for v, lg, limbs, first, inv, nega in jobs]
    b2 = plan.batch(flipped, config)
    b2.launch(stream)
    torch.cuda.synchronize()
    errors |= nb.device_errors()
    round_trip = bool(torch.equal(buf, buf0))
    b2.close()
    res = {"rows_checked": len(rows), "rows_exact": int(sum(ok)),
           "jobs_sampled": len({i for i, _ in rows}), "round_trip_exact": round_trip,
           "words_round_trip": int(buf.numel()), "device_errors": int(errors)}
    assert all(ok) and round_trip and errors == 0, "uneven batch parity failed: %s" % res
    return res


def run_uneven(args, world, rank, local):
    import torch
    import ntt_b200 as nb

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    stream = torch.cuda.Stream(device=dev)
    qs = nb.generate_primes(31, 21, 32)
    shapes = uneven_jobs()
    words = sum(b << a for a, b, _ in shapes)
    buf = torch.empty(words, dtype=torch.int32, device=dev)
    qt = torch.tensor([int(q) for q in qs], dtype=torch.int64, device=dev)
    gen = torch.Generator(device=dev)
    gen.manual_seed(4 + rank)
    jobs, off = [], 0
    for lg, limbs, inv in shapes:
        n = 1 << lg
        view = buf[off:off + limbs * n].view(limbs, n)
        r = torch.randint(0, 1 << 31, (limbs, n), generator=gen, device=dev, dtype=torch.int64)
        view.copy_((r % qt[:limbs, None]).to(torch.int32))
        jobs.append((view, lg, limbs, 0, inv, False))
        off += limbs * n
    buf0 = buf.clone()  # the inputs, for the parity check after the timed steps
    torch.cuda.synchronize()
    coeffs = words  # one transform per residue per launch
    plan = nb.BatchPlan(qs, 20)
    tuned = plan.autotune(jobs, stream=stream)
    batch = plan.batch(jobs)
    info = batch.info()
    for _ in range(max(3, args.warmup)):
        batch.launch(stream)
    torch.cuda.synchronize()
    assert nb.device_errors() == 0

    def timed(fn, steps):
        rank_barrier(world)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        c0 = nb.launch_count()
        e0.record(stream)
        for _ in range(steps):
            fn(stream)
        e1.record(stream)
        torch.cuda.synchronize()
        return reduce_over_ranks(e0.elapsed_time(e1), world), nb.launch_count() - c0

    clocks = ClockSampler(local)
    clocks.start()
    t_end = time.time() + 1.0
    while time.time() < t_end:
        batch.launch(stream)
        torch.cuda.synchronize()
    ms, launches = timed(batch.launch, args.steps)
    clk = clocks.stop()
    batch.graph_launch(stream)
    g_ms, _ = timed(batch.graph_launch, args.steps)
    value = world * coeffs * args.steps / (ms / 1e3)
    peaks, peak_source = load_peaks()
    peak = peaks["hbm_gbs"]
    avg_s = ms / args.steps / 1e3
    alg_bytes = 8 * coeffs
    # units of two passes move each residue twice (through the workspace ring)
    two_pass = sum(b << a for a, b, _ in shapes if a > {4096: 12, 8192: 13, 16384: 14}[info["config"]["tile_elems"]])
    model_bytes = 8 * (coeffs - two_pass) + 16 * two_pass
    traffic, traffic_src = None, None
    try:
        with open(os.path.join(ROOT, "profiles", "traffic.json")) as f:
            bpr = json.load(f).get("batch_queue_tc_bytes_per_residue")
        if bpr and info["config"].get("tensor"):
            traffic = bpr * coeffs
            traffic_src = "ncu DRAM bytes per residue of a 150 M-residue capture, scaled to this launch's residues"
    except OSError:
        pass
    result = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u32", "data": "synthetic: seeded uniform residues (generated on the device)",
        "config": {"workload": UNEVEN_WORKLOAD, "polys": UNEVEN_JOBS, "limbs_total": sum(b for _, b, _ in shapes),
                   "residues": coeffs, "bytes": 4 * coeffs, "moduli": "32 x 31-bit, q == 1 mod 2^21",
                   "negacyclic": False, "units": info["units"], "tiles": info["tiles"],
                   "workspace_bytes": info["ws_bytes"], "tuned": tuned, "l2": "inputs 7.9 GB >> L2",
                   "parallelism": "replicas x%d" % world},
        "graph_replay": {"value": world * coeffs * args.steps / (g_ms / 1e3), "ms_per_step": g_ms / args.steps},
        "roofline": {"bound": "hbm", "kernel": "batch_queue_tc" if info["config"].get("tensor") else "batch_queue",
                     "achieved": alg_bytes / avg_s / 1e9, "peak": peak,
                     "unit": "GB/s", "frac": alg_bytes / avg_s / 1e9 / peak, "traffic": traffic,
                     "traffic_source": traffic_src,
                     "model_bytes_per_launch": model_bytes, "model_frac": model_bytes / avg_s / 1e9 / peak,
                     "alg_bytes_per_launch": alg_bytes,
                     "peak_source": peak_source},
        "gpu_launches": launches, "clocks": clk, "e2e": None,
    }
    batch.close()
    result["parity"] = uneven_check(torch, nb, plan, jobs, shapes, qs, buf, buf0, tuned, stream)
    plan.close()
    if rank == 0 and world == 1:
        result["cpu_baseline"] = cpu_sample([(a, min(b, 8), c, False, False) for a, b, c in shapes], qs)
    return result


# --------------------------------------------------------- serving workload
SERVE_WORKLOAD = "serve_negacyclic_polymul_logN12-17_limbs4-48_60GB"


def run_serve(args, world, rank, local):
    """Closed loop at saturation (at most `outstanding` requests in flight)
    for the peak rate, then open-loop Poisson arrivals at 25/50/80/100% of
    it; latency = submit -> completion per request."""
    import threading
    import torch
    import ntt_b200 as nb

    torch.cuda.set_device(local)
    qs = nb.generate_primes(31, 18, 48)
    rng = np.random.default_rng(5 + rank)
    pool_n, outstanding = 96, 64
    pool = []
    for _ in range(pool_n):
        lg = int(rng.integers(12, 18))
        limbs = int(rng.integers(4, 49))
        first = int(rng.integers(0, 48 - limbs + 1))
        mods = np.array(qs[first:first + limbs], dtype=np.uint64)[:, None]
        a = torch.from_numpy((rng.integers(0, 1 << 62, (limbs, 1 << lg), dtype=np.uint64) % mods)
                             .astype(np.uint32).view(np.int32)).pin_memory()
        b = torch.from_numpy((rng.integers(0, 1 << 62, (limbs, 1 << lg), dtype=np.uint64) % mods)
                             .astype(np.uint32).view(np.int32)).pin_memory()
        pool.append((a, b, lg, limbs, first))
    # Results go to per-entry output buffers (the inputs stay unchanged).
    # Every CHECK_EVERY-th pool entry is a check entry: each of its requests
    # writes into a slot of its own ring, and the slot's limbs 0 and last are
    # compared with the oracle's negacyclic product (forward a, forward b,
    # pointwise, inverse) before the slot is reused and at the end of every
    # phase.  That checks every CHECK_EVERY-th product of the stream.
    CHECK_EVERY, RING = 8, 12
    outs = [torch.empty_like(a).pin_memory() for a, _, _, _, _ in pool]
    from oracle import oracle as O

    def oracle_product(a, b, lg, limbs, first, l):
        q = qs[first + l]
        x = a.numpy().view(np.uint32).reshape(limbs, 1 << lg)[l].astype(np.uint64)
        y = b.numpy().view(np.uint32).reshape(limbs, 1 << lg)[l].astype(np.uint64)
        fa, fb = O.negacyclic(x, q), O.negacyclic(y, q)
        return O.negacyclic(fa * fb % np.uint64(q), q, inverse=True).astype(np.uint32)

    expect, rings = {}, {}
    for e in range(0, pool_n, CHECK_EVERY):
        a, b, lg, limbs, first = pool[e]
        expect[e] = {l: oracle_product(a, b, lg, limbs, first, l) for l in sorted({0, limbs - 1})}
        rings[e] = {"bufs": [torch.empty_like(a).pin_memory() for _ in range(RING)], "pending": [None] * RING,
                    "next": 0}
    checks = {"products_checked": 0, "mismatches": 0}

    # The same pool resident on the device, for requests whose operands and
    # results stay in HBM (nttb_server_submit_device).
    dpool = [(a.cuda(), b.cuda(), lg, limbs, first) for a, b, lg, limbs, first in pool]
    douts = [torch.empty_like(d[0]) for d in dpool]
    drings = {e: {"bufs": [torch.empty_like(dpool[e][0]) for _ in range(RING)], "pending": [None] * RING, "next": 0}
              for e in rings}
    modes = {"host": {"pool": pool, "outs": outs, "rings": rings},
             "device": {"pool": dpool, "outs": douts, "rings": drings}}
    cur = modes["host"]

    def verify(e, slot):
        a, b, lg, limbs, first = pool[e]
        buf = cur["rings"][e]["bufs"][slot].view(limbs, 1 << lg)
        checks["products_checked"] += 1
        for l, want in expect[e].items():
            if not (buf[l].cpu().numpy().view(np.uint32) == want).all():
                checks["mismatches"] += 1
                break
        cur["rings"][e]["pending"][slot] = None
    # tile configuration tuned on this request mix
    tplan = nb.BatchPlan(qs, 17, negacyclic=True)
    sample = []
    for a, b, lg, limbs, first in pool[:24]:
        da, db = a.cuda(), b.cuda()
        sample.append((da, lg, limbs, first, "mul", True, db))
    tuned = tplan.autotune(sample)
    del sample
    tplan.close()
    budget = 60 << 30
    srv = nb.Server(qs, hbm_budget_bytes=budget, max_log_n=17, slots=3, max_batch_requests=64,
                    max_batch_residues=1 << 27, batch=tuned)
    coeffs = [3 * limbs << lg for _, _, lg, limbs, _ in pool]  # transforms per request

    def phase(rate, seconds):
        """rate None: closed loop; else Poisson arrivals at `rate` requests/s."""
        srv.latencies(reset=True)
        ids, done = [], [0]
        lock = threading.Condition()
        stop = [False]

        def reaper():
            k = 0
            while True:
                with lock:
                    while k >= len(ids) and not stop[0]:
                        lock.wait(0.05)
                    if k >= len(ids) and stop[0]:
                        return
                    rid = ids[k]
                srv.wait(rid, 120.0)
                k += 1
                with lock:
                    done[0] = k
                    lock.notify_all()

        th = threading.Thread(target=reaper)
        th.start()
        t0 = time.perf_counter()
        nxt, i, work = t0, 0, 0
        arr = np.random.default_rng(99)
        while time.perf_counter() - t0 < seconds:
            if rate is None:
                with lock:
                    while len(ids) - done[0] >= outstanding:
                        lock.wait(0.01)
            else:
                nxt += arr.exponential(1.0 / rate)
                dt = nxt - time.perf_counter()
                if dt > 0:
                    time.sleep(dt)
            e = i % pool_n
            a, b, lg, limbs, first = cur["pool"][e]
            out = cur["outs"][e]
            if e in rings:  # a check request: its own output slot
                r = cur["rings"][e]
                slot = r["next"]
                r["next"] = (slot + 1) % RING
                if r["pending"][slot] is not None:  # the slot's last request: done, then checked
                    with lock:
                        while done[0] <= r["pending"][slot]:
                            lock.wait(0.01)
                    verify(e, slot)
                out = r["bufs"][slot]
            if cur is modes["host"]:
                rid = srv.submit(a, b, out, lg, limbs, first)
            else:
                rid = srv.submit_device("mul", a, b, out, lg, limbs, first)
            work += coeffs[e]
            with lock:
                ids.append(rid)
                lock.notify_all()
            if e in rings:
                cur["rings"][e]["pending"][slot] = len(ids) - 1
            i += 1
        t_sub = time.perf_counter() - t0
        with lock:
            stop[0] = True
            lock.notify_all()
        th.join()
        t_all = time.perf_counter() - t0
        for e, r in cur["rings"].items():  # every request has completed: check the slots left
            for slot in range(RING):
                if r["pending"][slot] is not None:
                    verify(e, slot)
        lat = np.sort(srv.latencies(reset=True)) * 1e3
        return {"offered_rps": None if rate is None else rate, "requests": i,
                "achieved_rps": i / t_all, "coeffs_per_s": work / t_all, "submit_s": t_sub,
                "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
                "mean_ms": float(lat.mean())}

    def over_ranks(r):
        # replicas: rates add up, latencies are the worst rank's
        if world <= 1:
            return r
        out = dict(r)
        for k in ("requests", "achieved_rps", "coeffs_per_s"):
            out[k] = reduce_over_ranks(r[k], world, "sum")
        for k in ("p50_ms", "p99_ms", "mean_ms", "submit_s"):
            out[k] = reduce_over_ranks(r[k], world, "max")
        if r["offered_rps"] is not None:
            out["offered_rps"] = reduce_over_ranks(r["offered_rps"], world, "sum")
        return out

    def load_levels():
        phase(None, 1.0)  # warm-up
        sat = phase(None, args.serve_seconds)
        peak = sat["achieved_rps"]  # this rank's saturated rate sets its own load levels
        levels = {}
        for frac in (0.25, 0.5, 0.8, 1.0):
            levels["%d%%" % int(frac * 100)] = over_ranks(phase(frac * peak, args.serve_seconds))
        return over_ranks(sat), levels

    sat, levels = load_levels()  # operands and results in pinned host memory
    cur = modes["device"]
    dsat, dlevels = load_levels()  # operands and results resident in HBM
    st = srv.stats()
    srv.close()
    assert checks["mismatches"] == 0, "serving products differ from the oracle: %s" % checks
    cpu = cpu_sample([(lg, limbs, False, True, True) for _, _, lg, limbs, _ in pool], qs) if rank == 0 else None
    return {
        "metric": METRIC, "value": sat["coeffs_per_s"], "unit": UNIT, "n_gpus": world, "steps": sat["requests"],
        "warmup": 1, "ms_per_step": 1e3 / sat["achieved_rps"], "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u32", "data": "synthetic: seeded uniform residues, pinned host buffers",
        "config": {"workload": SERVE_WORKLOAD, "n": "2^12..2^17", "limbs": "4..48", "moduli": "48 x 31-bit",
                   "budget_bytes": budget, "slots": 3, "max_batch_requests": 64, "tuned": tuned,
                   "closed_loop_outstanding": outstanding, "parallelism": "replicas x%d" % world},
        "parity": dict(checks, rule="every %d-th product of the stream (one pool entry in %d), limbs 0 and last, "
                                    "vs the oracle's negacyclic product" % (CHECK_EVERY, CHECK_EVERY)),
        "serve_device_resident": {"saturated": dsat, "load_levels": dlevels,
                                  "api": "nttb_server_submit_device (operands and results in device memory)"},
        "serve": {"saturated": sat, "load_levels": levels, "batches": st["batches"],
                  "mean_batch_requests": st["batched_requests"] / max(1, st["batches"]),
                  "peak_region_bytes_in_use": st["peak_bytes_in_use"], "resident_bytes": st["resident_bytes"]},
        "e2e": {"value": sat["coeffs_per_s"], "unit": UNIT, "note": "host buffers in, host buffers out"},
        "cpu_baseline": cpu,
    }


# ------------------------------------------------------------ 60-bit prime
Q60 = 1152921504577486849  # largest 60-bit prime == 1 mod 2^21
Q60_WORKLOAD = "q60_2^20_cyclic_fwd+inv"


def run_q60(args, world, rank, local):
    """One 2^20 polynomial mod the 60-bit prime per step (forward + inverse),
    residues as uint64; also a batch of 16 polynomials per launch."""
    import torch
    import ntt_b200 as nb

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    stream = torch.cuda.Stream(device=dev)
    lg = 20
    plan = nb.WidePlan(lg, [Q60])
    rng = np.random.default_rng(60)
    host = rng.integers(0, Q60, 1 << lg, dtype=np.uint64)
    pool_n = 40  # 40 x 8 MB > 2x L2
    pool = torch.from_numpy(host.view(np.int64)).to(dev).repeat(pool_n, 1)

    def timed(fn, steps):
        rank_barrier(world)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        c0 = nb.launch_count()
        e0.record(stream)
        for i in range(steps):
            fn(i)
        e1.record(stream)
        torch.cuda.synchronize()
        return reduce_over_ranks(e0.elapsed_time(e1), world), nb.launch_count() - c0

    engine = "auto" if args.engine == "auto" else ("int8" if args.engine == "int8" else "scalar")

    def one(i, eng=None):
        buf = pool[i % pool_n]
        plan.transform(buf, buf, 1, engine=eng or engine, stream=stream)
        plan.transform(buf, buf, 1, inverse=True, engine=eng or engine, stream=stream)

    def sixteen(i, eng=None):
        b = pool[(16 * i) % 32:(16 * i) % 32 + 16]
        plan.transform(b, b, 16, engine=eng or engine, stream=stream)
        plan.transform(b, b, 16, inverse=True, engine=eng or engine, stream=stream)

    for i in range(max(3, args.warmup)):
        one(i)
        sixteen(i)
    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.5)
    ms, launches = timed(one, args.steps)
    ms16, _ = timed(sixteen, max(3, args.steps // 8))
    # the CUDA-core Montgomery-64 engine on the same polynomial (comparison)
    for i in range(3):
        one(i, "scalar")
    ms_sc, _ = timed(lambda i: one(i, "scalar"), max(10, args.steps // 4))
    b16 = {}
    for eng in ("int8", "scalar"):  # 16 polynomials per launch on each engine
        sixteen(0, eng)
        b16[eng], _ = timed(lambda i: sixteen(i, eng), max(3, args.steps // 8))
    # per-kernel device time: each pass kernel's share of the event-timed launches
    nb.profile_start()
    for i in range(args.steps):
        one(i)
    torch.cuda.synchronize()
    prof = nb.profile_stop()
    clk = clocks.stop()
    got = pool[0].cpu().numpy().view(np.uint64)
    assert (got == host).all(), "q60 round trip failed"
    coeffs = 2 << lg
    value = world * coeffs * args.steps / (ms / 1e3)
    peaks, peak_source = load_peaks()
    peak = peaks["hbm_gbs"]
    achieved = 16 * coeffs / (ms / args.steps / 1e3) / 1e9  # 8 B read + 8 B write per residue per transform
    cpu = None
    try:
        from oracle import oracle as O
        if O.ref() is not None and rank == 0 and world == 1:
            # the reference's ntt_host (__int128) on all host threads: one
            # 2^20 polynomial per thread, forward then inverse
            threads = max(1, os.cpu_count() or 1)
            x = np.tile(host, (threads, 1)).reshape(threads, 1, 1 << lg).copy()
            t0 = time.perf_counter()
            used = O.ref_host_batch(x, [Q60], inverse=False, threads=threads)
            O.ref_host_batch(x, [Q60], inverse=True, threads=threads)
            dt = time.perf_counter() - t0
            assert (x[0, 0] == host).all(), "reference round trip failed"
            cpu = {"value": threads * coeffs / dt, "unit": UNIT, "cores": used, "kind": "reference",
                   "sample": "%d x 2^20 forward + inverse, one polynomial per thread (ntt_host, __int128)" % threads}
    except Exception as e:  # reference library missing on this host
        cpu = {"unavailable": str(e)[:200]}
    return {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "u64", "data": "synthetic: seeded uniform residues",
        "config": {"workload": Q60_WORKLOAD, "n": 1 << lg, "q": Q60, "l2": "rotating 40 x 8 MB", "parallelism": "replicas x%d" % world},
        "engine": engine,
        "batch16": dict({"value": world * 16 * coeffs * max(3, args.steps // 8) / (ms16 / 1e3),
                          "ms_per_step": ms16 / max(3, args.steps // 8)},
                         **{eng + "_ms_per_step": m / max(3, args.steps // 8) for eng, m in b16.items()}),
        "engines_coeffs_per_s": {engine: value,
                                 "scalar": world * coeffs * max(10, args.steps // 4) / (ms_sc / 1e3)},
        "kernels": {k: {"launches": v[0], "total_ms": v[1]} for k, v in prof.items()},
        "roofline": {"bound": "hbm", "kernel": ", ".join(sorted(prof)), "achieved": achieved, "peak": peak,
                     "unit": "GB/s", "frac": achieved / peak, "traffic": None, "peak_source": peak_source,
                     "alg_bytes_per_step": 16 * coeffs,
                     "note": "16 B per residue per transform over the step's device time"},
        "cpu_baseline": cpu, "gpu_launches": launches, "clocks": clk, "e2e": None,
    }


# ----------------------------------------------------- small profiling cases
# ------------------------------------------------------ memory-bound helpers
def run_aux(args, world, rank, local):
    """The library's HBM-bound helper passes on inputs far larger than L2,
    against the measured copy peak: the RNS pointwise product (12 B per
    residue), the u64 transpose out of place and in place, and the in-place
    bit reversal (16 B per word each; the last three on TMA tiles)."""
    import torch
    import ntt_b200 as nb

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    stream = torch.cuda.Stream(device=dev)
    peaks, peak_source = load_peaks()
    peak = peaks["hbm_gbs"]

    def timed(fn, steps):
        # seconds per launch on the slowest rank (the figures are per GPU)
        for _ in range(3):
            fn()
        rank_barrier(world)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return reduce_over_ranks(e0.elapsed_time(e1) / steps / 1e3, world)

    out = {}
    qs = nb.generate_primes(31, TWO_ADICITY, N_LIMBS)
    plan = nb.RnsPlan(LOG_N, qs, negacyclic=True)
    polys = 64  # 64 x 24 x 2^16 residues = 402 MB per operand
    words = polys * N_LIMBS << LOG_N
    a = torch.randint(0, 1 << 30, (words,), dtype=torch.int32, device=dev)
    b = torch.randint(0, 1 << 30, (words,), dtype=torch.int32, device=dev)
    c = torch.empty_like(a)
    t = timed(lambda: plan.pointwise_mul(c, a, b, polys, stream=stream), args.steps)
    out["rns_pointwise_mul"] = {"bytes": 12 * words, "s": t, "gbs": 12 * words / t / 1e9}
    del a, b, c
    n = 1 << 13
    x = torch.randint(0, 1 << 62, (n * n,), dtype=torch.int64, device=dev)
    y = torch.empty_like(x)
    t = timed(lambda: nb.transpose_u64(y, x, n, n, stream=stream), args.steps)
    out["u64_transpose_8192x8192"] = {"bytes": 16 * n * n, "s": t, "gbs": 16 * n * n / t / 1e9}
    t = timed(lambda: nb.transpose_u64(x, x, n, n, stream=stream), args.steps)
    out["u64_transpose_in_place_8192x8192"] = {"bytes": 16 * n * n, "s": t, "gbs": 16 * n * n / t / 1e9}
    t = timed(lambda: nb.bit_reverse_u64(x, n * n, stream=stream), args.steps)
    out["u64_bit_reverse_2^26"] = {"bytes": 16 * n * n, "s": t, "gbs": 16 * n * n / t / 1e9}
    for v in out.values():
        v["frac"] = v["gbs"] / peak
    return {"metric": "HBM GB/s of the memory-bound helper passes", "unit": "GB/s", "peak": peak,
            "peak_source": peak_source,
            "kernels": out, "n_gpus": world, "steps": args.steps}


def profile_case(name):
    """Small, self-checking cases for ncu captures (a few launches, < 1 GB):
    int8 / dmma: forward+inverse of the 24-limb 2^16 negacyclic batch, four
    launches; batch: a ~600 MB uneven batch (log2 N 12..20, 1..8 limbs, mixed
    directions) launched twice; batch_tc: the same with log2 N 17..20 on
    tensor-core tiles; q60: forward + inverse of one 2^20 polynomial mod the
    60-bit prime, four times; move: the TMA tile kernels on 4096 x 4096
    words (transpose, in-place transpose, bit reversal), one launch each;
    klimb: the K-limb forward NTT over the BN254 field (K = 11) at 2^14,
    three times (its field from the committed fixture); int8_phases: the
    int8 case's step 100 times on the NTT_PHASE_PROFILE build
    (NTT_B200_LIB=phase), printing where the epilogue warps spend a step."""
    import torch
    import ntt_b200 as nb
    if name == "int8_phases":
        qs = nb.generate_primes(31, TWO_ADICITY, N_LIMBS)
        plan = nb.RnsPlan(LOG_N, qs, negacyclic=True)
        x = make_batch(qs, 7)
        d = torch.from_numpy(x.reshape(-1).view(np.int32)).cuda()
        for _ in range(10):
            plan.forward_inverse(d, 1, engine="int8")
        torch.cuda.synchronize()
        enabled, _ = nb.phase_profile(clear=True)
        if not enabled:
            sys.exit("int8_phases: load the NTT_PHASE_PROFILE build (NTT_B200_LIB=phase)")
        steps = 100
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(steps):
            plan.forward_inverse(d, 1, engine="int8")
        e1.record()
        torch.cuda.synchronize()
        _, ph = nb.phase_profile(clear=True)
        assert (d.cpu().numpy().view(np.uint32).reshape(x.shape) == x).all()
        mhz = float(subprocess.run(["nvidia-smi", "--query-gpu=clocks.sm", "--format=csv,noheader,nounits", "-i", "0"],
                                   capture_output=True, text=True).stdout.split()[0])
        ctas = ph.pop("ctas")
        warps = ctas * 16  # epilogue warps
        out = {k: round(v / warps / mhz, 3) for k, v in ph.items() if not k.startswith("cta_")}
        out.update({k: round(v / ctas / mhz, 3) for k, v in ph.items() if k.startswith("cta_")})
        out["us_per_step_events"] = round(e0.elapsed_time(e1) / steps * 1e3, 3)
        out["note"] = ("us per launch: epilogue-warp phases summed over the four stages (mean over warps), "
                       "CTA lifetime and start-up per CTA; clock %d MHz" % mhz)
        print(json.dumps(out))
        return
    if name == "klimb":
        # BN254 (K = 11 limbs of 24 bits), Montgomery form R = 2^264.  The
        # twiddles are powers of the fixture's omega: the network does the same
        # arithmetic for any base, and this case is timed, not checked.
        K, lg = 11, 14
        g = np.load(os.path.join(ROOT, "tests", "golden", "klimb.npz"))
        to_int = lambda limbs: sum(int(v) << (24 * i) for i, v in enumerate(limbs))
        to_limbs = lambda x: [(x >> (24 * i)) & 0xFFFFFF for i in range(K)]
        p, w = to_int(g["prime_K11"]), to_int(g["omega_K11"])
        R = 1 << (24 * K)
        n = 1 << lg
        tw, t = [], R % p
        for _ in range(n):
            tw.append(to_limbs(t))
            t = t * w % p
        rng = np.random.default_rng(11)
        xs = [to_limbs(int(v) % p * R % p) for v in rng.integers(0, 2 ** 62, n, dtype=np.uint64)]
        d = torch.from_numpy(np.array(xs, dtype=np.uint32).reshape(-1).view(np.int32)).cuda()
        dt = torch.from_numpy(np.array(tw, dtype=np.uint32).reshape(-1).view(np.int32)).cuda()
        limbs = to_limbs(p)
        for _ in range(3):
            nb.klimb_forward(K, d, dt, lg, limbs, nb.klimb_neg_inv24(limbs[0]))
        torch.cuda.synchronize()
        return
    if name == "move":
        # TMA tile kernels: 4096 x 4096 words (128 MB) transposed out of place,
        # then in place, then bit-reversed in place; checked against numpy
        n = 4096
        x = np.random.default_rng(5).integers(0, 1 << 63, n * n, dtype=np.uint64)
        src = torch.from_numpy(x.view(np.int64)).cuda()
        dst = torch.empty_like(src)
        nb.transpose_u64(dst, src, n, n)
        nb.transpose_u64(dst, dst, n, n)
        nb.bit_reverse_u64(dst, n * n)
        torch.cuda.synchronize()
        got = dst.cpu().numpy().view(np.uint64)
        idx = np.arange(n * n, dtype=np.uint64)
        rev = np.zeros_like(idx)
        for b in range(24):
            rev |= ((idx >> np.uint64(b)) & np.uint64(1)) << np.uint64(23 - b)
        assert (got == x[rev]).all()
        assert nb.device_errors() == 0
        return
    if name == "q60":
        plan = nb.WidePlan(20, [Q60])
        x = np.random.default_rng(3).integers(0, Q60, 1 << 20, dtype=np.uint64)
        d = torch.from_numpy(x.view(np.int64)).cuda()
        for _ in range(4):
            plan.transform(d, d, 1)
            plan.transform(d, d, 1, inverse=True)
        torch.cuda.synchronize()
        assert (d.cpu().numpy().view(np.uint64) == x).all()
    elif name in ("int8", "dmma"):
        qs = nb.generate_primes(31, TWO_ADICITY, N_LIMBS)
        plan = nb.RnsPlan(LOG_N, qs, negacyclic=True)
        x = make_batch(qs, 7)
        d = torch.from_numpy(x.reshape(-1).view(np.int32)).cuda()
        for _ in range(4):
            plan.forward_inverse(d, 1, engine=name)
        torch.cuda.synchronize()
        assert (d.cpu().numpy().view(np.uint32).reshape(x.shape) == x).all()
    else:
        qs = nb.generate_primes(31, 21, 8)
        rng = np.random.default_rng(1)
        jobs, bufs, words = [], [], 0
        lo = 17 if name == "batch_tc" else 12
        while words < 150_000_000:
            lg, limbs = int(rng.integers(lo, 21)), int(rng.integers(1, 9))
            t = torch.randint(0, 1 << 30, (limbs << lg,), dtype=torch.int32, device="cuda") % int(min(qs))
            bufs.append(t)
            words += limbs << lg
            jobs.append((t, lg, limbs, 0, bool(rng.integers(0, 2)), False))
        plan = nb.BatchPlan(qs, 20)
        cfg = {"tile_elems": 4096, "threads": 256, "split": 1, "lag": 4, "group": 3}
        if name == "batch_tc":
            cfg.update(split=0, tensor=1)
        b = plan.batch(jobs, cfg)
        b.launch()
        b.launch()
        torch.cuda.synchronize()
        assert nb.device_errors() == 0
    print("profile case %s ok" % name)


def secondary_workloads(args, world, rank, local):
    """The other configurations, measured in the same single-GPU run after the
    headline (each one's own checks run too: round trips, the uneven batch's
    oracle rows and round trip, the serving stream's oracle products).  A
    summary of each JSON line; a failure is recorded, not raised."""
    import copy
    out = {}
    for name, fn, steps in (("q60", run_q60, 50), ("uneven", run_uneven, 5), ("serve", run_serve, 0)):
        a = copy.copy(args)
        a.steps, a.warmup, a.serve_seconds = (steps or args.steps), 3, 1.5
        t0 = time.time()
        try:
            r = fn(a, world, rank, local)
        except Exception as e:  # reported beside the headline, which stands on its own
            out[name] = {"error": "%s: %s" % (type(e).__name__, str(e)[:300])}
            continue
        keep = {k: r[k] for k in ("workload", "value", "unit", "ms_per_step", "steps", "engine", "batch16",
                                  "engines_coeffs_per_s", "parity", "roofline", "graph_replay") if k in r}
        keep["config"] = r.get("config", {}).get("workload")
        if "serve" in r:
            keep["serve"] = {"saturated_rps": r["serve"]["saturated"]["achieved_rps"],
                             "p50_p99_ms": {k: [v["p50_ms"], v["p99_ms"]] for k, v in r["serve"]["load_levels"].items()}}
            d = r["serve_device_resident"]
            keep["serve_device_resident"] = {"saturated_rps": d["saturated"]["achieved_rps"],
                                             "p50_p99_ms": {k: [v["p50_ms"], v["p99_ms"]] for k, v in d["load_levels"].items()}}
        if r.get("cpu_baseline"):
            keep["cpu_baseline"] = r["cpu_baseline"]
        keep["wall_s"] = round(time.time() - t0, 1)
        out[name] = keep
    return out


def main():
    args = parse()
    if args.profile_case:
        profile_case(args.profile_case)
        return
    world, rank, local = dist_setup(args)
    if args.workload in ("uneven", "serve", "q60", "aux") and args.impl == "ours":
        fn = {"uneven": run_uneven, "serve": run_serve, "q60": run_q60, "aux": run_aux}[args.workload]
        r = fn(args, world, rank, local)
        if rank == 0:
            print(json.dumps(r))
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return
    if args.impl == "reference":
        if rank != 0:  # rank 0 alone runs the reference; no collective is issued on this arm
            if world > 1:
                import torch.distributed as dist
                dist.destroy_process_group()
            return
        qs = moduli()
        r = cpu_reference(qs, args.steps, args.warmup)
        line = {"impl": "reference", "metric": METRIC, "value": r["value"], "unit": UNIT, "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": r["seconds"] / args.steps * 1e3,
                "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "u64", "data": "synthetic: seeded uniform residues",
                "config": headline_config(world),
                "engine": "the reference's ntt_host (CPU), all host threads",
                "cpu_baseline": {"value": r["value"], "unit": UNIT, "cores": r["cores"], "kind": r["kind"],
                                 "sample": r["sample"]},
                "e2e": {"value": r["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        import torch
        if torch.cuda.is_available():
            # the reference's own GPU kernels on the same batch (reported beside the CPU arm)
            line["reference_gpu"] = reference_gpu_bar(qs, args.steps, args.warmup, local)
        print(json.dumps(line))
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return
    result, qs = run_ours(args, world, rank, local)
    if rank == 0 and world == 1 and not args.quick:
        result["cpu_baseline"] = bounded_cpu_baseline(qs)
        if not args.no_secondary:
            result["secondary"] = secondary_workloads(args, world, rank, local)
    if rank == 0:
        print(json.dumps(result))
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
