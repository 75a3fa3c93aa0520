"""The C-ABI library loads without a GPU and exports every symbol that
include/curc_b200.h declares."""
import ctypes
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    syms = set()
    for fn in os.listdir(os.path.join(ROOT, "include")):
        if fn.endswith(".h"):
            text = open(os.path.join(ROOT, "include", fn)).read()
            text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
            syms |= set(re.findall(r"\b(curc_[a-z0-9_]+)\s*\(", text))
    return syms


def test_header_symbols_exported():
    from curc_b200 import LIB_PATH
    lib = ctypes.CDLL(LIB_PATH)
    syms = declared_symbols()
    assert len(syms) >= 6
    missing = [s for s in sorted(syms) if not hasattr(lib, s)]
    assert not missing, missing


def test_create_without_gpu_fails_cleanly():
    import torch
    if torch.cuda.is_available():
        return
    from curc_b200 import Context, CurcError
    try:
        Context(0)
    except CurcError as e:
        assert "curc_ctx_create" in str(e)
    else:
        raise AssertionError("context creation should fail without a GPU")
