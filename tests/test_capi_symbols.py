"""The C-ABI library loads on a machine without a GPU and exports every
function include/bdlu.h declares (no compute calls)."""
import ctypes
import os
import re

import blockdaglu as bd

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    text = open(os.path.join(ROOT, "include", "bdlu.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(bdlu_[a-z0-9_]+)\s*\(", text)))


def test_every_declared_symbol_is_exported():
    lib = ctypes.CDLL(bd.LIB_PATH)
    names = declared_symbols()
    assert len(names) > 30
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_handle_lifecycle_without_device():
    s = bd.Solver()
    assert s.n() == 0
    assert s.selected_mode() == "BLOCK"
    del s
