"""The ctypes mirrors of the C ABI's structs (phasecon_b200/mbir.py, pcmbir.py)
against include/mbirgpu.h: every struct's size and every field's offset, as
the C compiler lays them out. A field added on one side only would shift the
others silently; this catches it on the CPU."""
import ctypes as C
import os
import subprocess

from phasecon_b200 import mbir as M
from phasecon_b200 import pcmbir as PC

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

PAIRS = [
    (M.Options, "mbirgpu_options"),
    (M.ProblemStruct, "mbirgpu_problem"),
    (M.SessionInfo, "mbirgpu_session_info"),
    (M.IterStats, "mbirgpu_iter_stats"),
    (M.BatchStats, "mbirgpu_batch_stats"),
    (PC.PcProblemStruct, "mbirgpu_pc_problem"),
    (PC.PcOptions, "mbirgpu_pc_options"),
    (PC.PcStats, "mbirgpu_pc_stats"),
    (PC.SimOptions, "mbirgpu_pc_sim_options"),
]


def c_layout(tmp_path):
    lines = ['#include <stddef.h>', '#include <stdio.h>', '#include "mbirgpu.h"', "int main(void) {"]
    for cls, cname in PAIRS:
        lines.append(f'    printf("{cname} sizeof %zu\\n", sizeof({cname}));')
        for f in cls._fields_:
            lines.append(f'    printf("{cname} {f[0]} %zu\\n", offsetof({cname}, {f[0]}));')
    lines += ["    return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c11", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout
    got = {}
    for line in out.splitlines():
        cname, field, value = line.split()
        got[(cname, field)] = int(value)
    return got


def test_ctypes_structs_match_the_c_header(tmp_path):
    got = c_layout(tmp_path)
    for cls, cname in PAIRS:
        assert C.sizeof(cls) == got[(cname, "sizeof")], cname
        for f in cls._fields_:
            assert getattr(cls, f[0]).offset == got[(cname, f[0])], (cname, f[0])
