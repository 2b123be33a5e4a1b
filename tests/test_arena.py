"""CPU: the serving loop's first-fit device-region allocator
(ntt-tensorcore_b200/csrc/arena.hpp), checked by tests/arena_check.cpp against
a granule bitmap."""
import os
import subprocess

from conftest import ROOT


def test_arena_first_fit_against_bitmap(tmp_path):
    exe = str(tmp_path / "arena_check")
    r = subprocess.run(["g++", "-std=c++17", "-O1", "-Wall", "-Werror",
                        "-I" + os.path.join(ROOT, "ntt-tensorcore_b200", "csrc"),
                        os.path.join(ROOT, "tests", "arena_check.cpp"), "-o", exe],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    r = subprocess.run([exe], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0 and r.stdout.strip() == "ok", r.stdout[-2000:]
