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


@pytest.mark.parametrize("field,value,needle", [
    ("max_groups", 0, b"max_groups"),
    ("max_groups", None, b"max_groups"),   # DQ_NOALLOC_MAX_GROUPS + 1
    ("out_ngroups", 0, b"null argument"),
    ("build_key", 0, b"null argument"),
    ("build_rows", -1, b"negative"),
])
def test_noalloc_rejects_bad_arguments_before_any_device_work(field, value, needle):
    """Argument checks of the allocation-free join run on the host before any
    device call, so they hold without a GPU."""
    from dogqc_b200 import _lib as L
    lib = L.lib()
    a = L.dq_join_agg_args()
    a.build_key = a.build_filter = a.build_group = 16
    a.out_group = a.out_sum = a.out_count = a.out_ngroups = 16
    a.build_rows, a.probe_rows, a.max_groups = 8, 0, 16
    setattr(a, field, L.NOALLOC_MAX_GROUPS + 1 if value is None else value)
    assert lib.dq_join_agg_noalloc(C.byref(a), None) == L.ERR_INVALID
    assert needle in lib.dq_last_error(None)
