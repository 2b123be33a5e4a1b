"""Builds libntt_b200.so (in-tree) from csrc/*.cu and csrc/*.cpp with nvcc for sm_100a.

Usage: python ntt-tensorcore_b200/build.py [--force] [--debug-bounds | --phase-profile]
Objects go to ntt-tensorcore_b200/_build/, the library to
ntt-tensorcore_b200/ntt_b200/libntt_b200.so.  Rebuilds only what changed
(by modification time, headers included).  --debug-bounds builds the
range-checked variant (-DNTT_DEBUG_BOUNDS, csrc/bounds.cuh) into _build_dbg/
and ntt_b200/libntt_b200_dbg.so instead; --phase-profile builds the INT8
cluster kernel with its phase counters (-DNTT_PHASE_PROFILE, read by
nttb_phase_profile) into _build_phase/ and ntt_b200/libntt_b200_phase.so.
"""
import concurrent.futures as cf
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "ntt_b200", "libntt_b200.so")
BUILD_DBG = os.path.join(HERE, "_build_dbg")
LIB_DBG = os.path.join(HERE, "ntt_b200", "libntt_b200_dbg.so")
BUILD_PHASE = os.path.join(HERE, "_build_phase")
LIB_PHASE = os.path.join(HERE, "ntt_b200", "libntt_b200_phase.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
         "-I" + os.path.join(ROOT, "include"), "-I" + CSRC, "--expt-relaxed-constexpr"]


def _headers():
    hs = glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.hpp"))
    hs += glob.glob(os.path.join(ROOT, "include", "*.h")) + glob.glob(os.path.join(ROOT, "include", "*.cuh"))
    return max((os.path.getmtime(h) for h in hs), default=0)


def _compile(src, obj, extra=()):
    cmd = [NVCC] + ARCH + FLAGS + list(extra) + ["-c", src, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("nvcc failed for %s:\n%s%s" % (src, r.stdout, r.stderr))
    return obj


def build(force=False, verbose=False, debug_bounds=False, phase_profile=False):
    if debug_bounds:
        build_dir, lib, extra = BUILD_DBG, LIB_DBG, ["-DNTT_DEBUG_BOUNDS"]
    elif phase_profile:
        build_dir, lib, extra = BUILD_PHASE, LIB_PHASE, ["-DNTT_PHASE_PROFILE"]
    else:
        build_dir, lib, extra = BUILD, LIB, []
    os.makedirs(build_dir, exist_ok=True)
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cpp")))
    hdr_time = _headers()
    jobs = []
    objs = []
    for s in srcs:
        o = os.path.join(build_dir, os.path.basename(s) + ".o")
        objs.append(o)
        if force or not os.path.exists(o) or os.path.getmtime(o) < max(os.path.getmtime(s), hdr_time):
            jobs.append((s, o))
    if jobs:
        with cf.ThreadPoolExecutor(max_workers=min(8, len(jobs))) as ex:
            for f in [ex.submit(_compile, s, o, extra) for s, o in jobs]:
                f.result()
    if jobs or not os.path.exists(lib):
        cmd = [NVCC] + ARCH + ["-shared", "-o", lib] + objs + ["-lcudart", "-lcuda"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("link failed:\n%s%s" % (r.stdout, r.stderr))
    if verbose:
        print("built", lib, "(%d objects recompiled)" % len(jobs))
    return lib


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True, debug_bounds="--debug-bounds" in sys.argv,
          phase_profile="--phase-profile" in sys.argv)
