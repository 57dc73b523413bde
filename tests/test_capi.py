"""The C-ABI library loads without a GPU and exports every function that
include/matvans.h declares."""
import ctypes
import os
import re

from conftest import ROOT
from matvans_b200 import _lib


def declared_functions():
    src = open(os.path.join(ROOT, "include", "matvans.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    names = re.findall(r"\b([A-Za-z_][A-Za-z0-9_]*)\s*\(", src)
    skip = {"if", "for", "while", "return", "sizeof", "defined"}
    return sorted({n for n in names if n not in skip and (n.startswith("mv_") or n.startswith("mat_vec_mul_coalesced"))})


def test_library_exports_every_declared_symbol():
    L = ctypes.CDLL(_lib.LIB_PATH)
    decl = declared_functions()
    assert len(decl) >= 20
    missing = [n for n in decl if not hasattr(L, n)]
    assert not missing, missing
    assert sorted(_lib.EXPORTS) == decl


def test_version_and_error_string():
    L = _lib.lib()
    assert b"sm_100a" in L.mv_version()
    rc = L.mv_awr_encode(None, 0, 0, 0, ctypes.byref(ctypes.c_void_p()))
    assert rc == 1
    assert b"bad arguments" in L.mv_last_error()
