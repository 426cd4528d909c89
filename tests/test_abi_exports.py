"""The C-ABI library loads without a GPU and exports every symbol include/pe_b200.h declares."""
import ctypes
import os
import re

import pytest

from pe_b200 import _abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "pe_b200.h")


def declared_symbols():
    txt = open(HEADER).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(pe_b200_\w+)\s*\(", txt)))


def test_header_and_binding_agree():
    assert declared_symbols() == sorted(_abi.EXPORTS)


def test_library_exports_all_symbols():
    if not os.path.exists(_abi.LIB_PATH):
        from pe_b200 import build
        build.build()
    lib = ctypes.CDLL(_abi.LIB_PATH)
    missing = [s for s in declared_symbols() if not hasattr(lib, s)]
    assert not missing, missing


def test_default_params_without_gpu():
    p = _abi.default_params()
    assert p.max_iterations == 100 and abs(p.erp - 0.7) < 1e-15 and p.damping == 1.0
