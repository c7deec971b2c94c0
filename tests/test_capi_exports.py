"""CPU test: the C-ABI library loads and exports every symbol include/*.h declares."""
import glob
import os
import re

import pytest

from cpw2000_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = []
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"^\s*(?:const\s+)?[A-Za-z_][A-Za-z0-9_]*\s*\**\s*([A-Za-z_][A-Za-z0-9_]*)\s*\(",
                             text, flags=re.M):
            names.append(m.group(1))
    return sorted(set(names))


def test_header_declares_entry_points():
    names = declared_functions()
    assert "cpw_b200_hk_psi_c16" in names and "hk_psi_c16_" in names
    assert len(names) >= 15


def test_library_exports_every_declared_symbol():
    if not _lib.LIB_PATH.exists():
        pytest.fail("libcpwb200.so is not built (run python -m cpw2000_b200.build)")
    L = _lib.lib()
    missing = [n for n in declared_functions() if not hasattr(L, n)]
    assert not missing, f"missing exports: {missing}"
    # the ctypes signature table covers the header too
    assert set(declared_functions()) <= set(_lib.SIGNATURES)
    assert L.cpw_b200_version() >= 10000
