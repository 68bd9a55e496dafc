"""The C-ABI library loads without a GPU and exports every function include/lcs_gpu.h declares."""
import ctypes
import os
import re

from luisacomputesimulator_b200 import _capi, build

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = []
    for h in sorted(os.listdir(os.path.join(ROOT, "include"))):
        if h.endswith(".h"):
            src = open(os.path.join(ROOT, "include", h)).read()
            src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
            names += re.findall(r"^\s*(?:const\s+)?[A-Za-z_][\w\s\*]*?\b(lcs_\w+)\s*\(", src, flags=re.M)
    return sorted(set(names))


def test_header_declares_functions():
    assert len(declared_functions()) >= 25


def test_library_exports_every_declared_symbol():
    build.build()
    lib = ctypes.CDLL(_capi.LIB_PATH)
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_binding_covers_every_declared_symbol():
    assert set(declared_functions()) <= set(_capi.SIGNATURES)


def test_version_string_without_gpu():
    lib = _capi.load()
    assert lib.lcs_version().decode().startswith("lcs_b200")
