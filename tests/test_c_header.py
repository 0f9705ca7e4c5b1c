"""include/mbirgpu.h is the drop-in boundary for C callers: it must compile as
plain C (C11, warnings as errors) and every function it declares must link
against libmbirgpu.so from a C program (CPU only: the program takes the
functions' addresses and exits without calling any of them)."""
import os
import shutil
import subprocess

import pytest

from test_abi import ROOT, header_functions

import phasecon_b200 as pc

CUDA_LIB = "/usr/local/cuda/lib64"


@pytest.mark.skipif(shutil.which("gcc") is None, reason="no C compiler")
def test_header_compiles_as_c_and_links(tmp_path):
    if not os.path.exists(pc.LIB_PATH):
        from phasecon_b200 import build
        build.build()
    names = header_functions()
    src = tmp_path / "use_header.c"
    src.write_text(
        "#include <stdio.h>\n#include \"mbirgpu.h\"\n"
        "typedef void (*fn_t)(void);\n"
        "static const fn_t fns[] = {\n" + "".join(f"    (fn_t){n},\n" for n in names) + "};\n"
        "int main(void)\n{\n"
        "    size_t n = 0;\n"
        "    for (size_t i = 0; i < sizeof(fns) / sizeof(fns[0]); i++) n += fns[i] != NULL;\n"
        "    printf(\"%zu\\n\", n);\n"
        "    return 0;\n}\n")
    exe = tmp_path / "use_header"
    lib_dir = os.path.dirname(pc.LIB_PATH)
    cmd = ["gcc", "-std=c11", "-Wall", "-Wextra", "-Werror", "-I", os.path.join(ROOT, "include"), str(src),
           "-o", str(exe), "-L", lib_dir, "-lmbirgpu", "-Wl,--allow-shlib-undefined", f"-Wl,-rpath,{lib_dir}"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    env = dict(os.environ, LD_LIBRARY_PATH=os.pathsep.join([lib_dir, CUDA_LIB, os.environ.get("LD_LIBRARY_PATH", "")]))
    r = subprocess.run([str(exe)], capture_output=True, text=True, env=env)
    if r.returncode != 0 and "libcudart" in r.stderr:
        pytest.skip("the CUDA runtime library is not on the loader path: " + r.stderr.strip())
    assert r.returncode == 0, r.stderr
    assert int(r.stdout) == len(names)
