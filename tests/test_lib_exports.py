"""The C-ABI library loads and exports every entry point include/*.h declares
(no GPU needed: nothing is called)."""
import ctypes
import glob
import os
import re

from conftest import ROOT
from swinmd_b200 import _lib


def declared_symbols():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"\b(smd_[a-z0-9_]+)\s*\(", text):
            names.add(m.group(1))
    return names


def test_library_exports_all_declared_symbols():
    from swinmd_b200 import build
    build.build()
    lib = ctypes.CDLL(_lib.LIB_PATH)
    names = declared_symbols()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_binding_covers_declarations():
    assert declared_symbols() <= set(_lib.SIGNATURES)
