"""CPU checks of the C-ABI library: it loads, exports every declared entry point,
and the ctypes mirrors of the IR structs match the header's layout."""
import ctypes as C
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "dogqc_b200.h")


def declared_functions():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"^\s*(?:int|void|const char\*)\s+(dq_\w+)\s*\(", text, re.M)))


def test_library_exports_every_declared_symbol():
    from dogqc_b200 import _lib
    lib = _lib.lib()
    names = declared_functions()
    assert "dq_plan_execute" in names and len(names) >= 15
    for n in names:
        assert hasattr(lib, n), n
    assert lib.dq_version() == _lib.ABI_VERSION


def test_struct_layout():
    from dogqc_b200 import _lib
    _lib.check_layout()
    assert C.sizeof(_lib.dq_op) == 40


def test_init_without_gpu_fails_cleanly():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from dogqc_b200 import _lib
    from dogqc_b200.engine import Engine
    with pytest.raises(_lib.DqError):
        Engine(0)
