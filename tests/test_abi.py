"""The C-ABI library loads and exports every symbol the header declares
(CPU only: no compute calls without a GPU)."""
import ctypes
import os
import subprocess

import pytest

from simuse_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_library_built_and_loads():
    assert os.path.exists(_lib.library_path), "run `make -C dioma-core_b200`"
    L = _lib.lib()
    assert L.sg_abi_version() == 1


def test_every_declared_symbol_is_exported():
    declared = _lib.declared_symbols()
    assert len(declared) >= 40
    L = ctypes.CDLL(_lib.library_path)
    missing = [s for s in declared if not hasattr(L, s)]
    assert not missing, missing
    # and the Python binding covers every declared entry point
    assert set(declared) <= set(_lib.SIGNATURES), set(declared) - set(_lib.SIGNATURES)


def test_exports_are_plain_c():
    out = subprocess.run(["nm", "-D", "--defined-only", _lib.library_path], capture_output=True, text=True).stdout
    names = {ln.split()[-1] for ln in out.splitlines() if " T " in ln}
    for s in _lib.declared_symbols():
        assert s in names, s


def test_null_handle_is_an_error_not_a_crash():
    L = _lib.lib()
    assert L.sg_step(None, 1) == -1
    assert L.sg_build(None) == -1
    assert "null" in _lib.last_error()


def test_product_path_has_no_oracle_dependency():
    # the product never links or imports the CPU oracle
    out = subprocess.run(["ldd", _lib.library_path], capture_output=True, text=True).stdout
    assert "oracle" not in out
    pkg = os.path.join(ROOT, "dioma-core_b200", "simuse_b200")
    import re
    for f in os.listdir(pkg):
        if f.endswith(".py"):
            src = open(os.path.join(pkg, f)).read()
            assert not re.search(r"^\s*(import|from)\s+oracle", src, re.M), f
