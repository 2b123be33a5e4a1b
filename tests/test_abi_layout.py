"""CPU: the ctypes mirror of the C ABI (ntt_b200/__init__.py) agrees with
include/ntt_b200.h: every struct has the same size and field offsets as the
C compiler gives it, and every bound function declares as many arguments as
its C prototype."""
import ctypes
import os
import re
import subprocess

from conftest import ROOT
import ntt_b200 as nb

HEADER = os.path.join(ROOT, "include", "ntt_b200.h")

STRUCTS = [
    ("nttb_modular_params", nb._Params),
    ("nttb_plan_info", nb._PlanInfo),
    ("nttb_batch_job", nb.BatchJob),
    ("nttb_batch_config", nb.BatchConfig),
    ("nttb_server_config", nb.ServerConfig),
    ("nttb_server_stats_t", nb.ServerStats),
]


def test_struct_layouts_match_the_c_compiler(tmp_path):
    lines = ['#include <stddef.h>', '#include <stdio.h>', '#include "ntt_b200.h"', "int main(void) {"]
    for cname, cls in STRUCTS:
        lines.append('printf("%s %%zu\\n", sizeof(%s));' % (cname, cname))
        for f, _ in cls._fields_:
            lines.append('printf("%s.%s %%zu\\n", offsetof(%s, %s));' % (cname, f, cname, f))
    lines += ["return 0;", "}"]
    src, exe = tmp_path / "layout.c", str(tmp_path / "layout")
    src.write_text("\n".join(lines) + "\n")
    r = subprocess.run(["gcc", "-std=c11", "-Wall", "-Werror", "-I" + os.path.join(ROOT, "include"), str(src),
                        "-o", exe], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    c = dict(line.split() for line in subprocess.run([exe], capture_output=True, text=True).stdout.splitlines())
    for cname, cls in STRUCTS:
        assert int(c[cname]) == ctypes.sizeof(cls), cname
        for f, _ in cls._fields_:
            assert int(c["%s.%s" % (cname, f)]) == getattr(cls, f).offset, (cname, f)


def _prototypes():
    text = re.sub(r"/\*.*?\*/", " ", open(HEADER).read(), flags=re.S)
    out = {}
    for m in re.finditer(r"NTTB_API\s+[\w\s\*]+?\b(nttb_\w+)\s*\(([^;]*?)\)\s*;", text):
        params = m.group(2).strip()
        out[m.group(1)] = 0 if params in ("", "void") else params.count(",") + 1
    return out


def test_bound_functions_match_prototype_arity():
    protos = _prototypes()
    assert len(protos) == len(nb.header_symbols())
    L = nb.lib()
    checked = 0
    for name, arity in protos.items():
        fn = getattr(L, name)
        if fn.argtypes is None:
            continue
        assert len(fn.argtypes) == arity, (name, len(fn.argtypes), arity)
        checked += 1
    assert checked >= 40
