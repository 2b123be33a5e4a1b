"""CPU: host-side C++ of the library checked by small g++ programs:
the serving loop's first-fit device-region allocator
(ntt-tensorcore_b200/csrc/arena.hpp) against a granule bitmap, and the K-limb
pass plan (ntt-tensorcore_b200/csrc/klimb_plan.hpp) against its launch limits."""
import os
import subprocess

import pytest

from conftest import ROOT


@pytest.mark.parametrize("prog", ["arena_check", "klimb_plan_check"])
def test_host_logic(prog, tmp_path):
    exe = str(tmp_path / prog)
    r = subprocess.run(["g++", "-std=c++17", "-O1", "-Wall", "-Werror",
                        "-I" + os.path.join(ROOT, "ntt-tensorcore_b200", "csrc"),
                        os.path.join(ROOT, "tests", prog + ".cpp"), "-o", exe],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    r = subprocess.run([exe], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0 and r.stdout.strip() == "ok", r.stdout[-2000:]
