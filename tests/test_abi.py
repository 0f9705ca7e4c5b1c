"""The C-ABI library loads and exports every symbol include/mbirgpu.h declares (CPU only)."""
import ctypes
import os
import re

import pytest

import phasecon_b200 as pc

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    txt = open(os.path.join(ROOT, "include", "mbirgpu.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b([A-Za-z_]\w*)\s*\(", txt)) - {"if", "sizeof"})


def test_library_exports_every_declared_symbol():
    if not os.path.exists(pc.LIB_PATH):
        from phasecon_b200 import build
        build.build()
    lib = ctypes.CDLL(pc.LIB_PATH)
    declared = header_functions()
    assert "reconstruct" in declared
    missing = [f for f in declared if not hasattr(lib, f)]
    assert not missing, missing
    assert sorted(declared) == sorted(pc.EXPORTS)


def test_options_roundtrip_and_validation():
    o = pc.default_options()
    assert o.mrf_p == 1.2 and o.mrf_q == 2.0 and o.alpha == 1.5 and o.max_iterations == 1000
    saved = pc.get_options()
    try:
        pc.set_options(mrf_p=1.1, sv_size=4)
        assert pc.get_options().mrf_p == 1.1
        with pytest.raises(pc.MbirError):
            pc.set_options(mrf_p=0.5)
        with pytest.raises(pc.MbirError):
            pc.set_options(sv_size=99)
    finally:
        pc.lib().mbirgpu_set_options(ctypes.byref(saved))


def test_missing_library_fails_loudly(monkeypatch, tmp_path):
    from phasecon_b200 import mbir
    monkeypatch.setattr(mbir, "_lib", None)
    monkeypatch.setattr(mbir, "LIB_PATH", str(tmp_path / "absent.so"))
    with pytest.raises(mbir.MbirError):
        mbir.lib()
