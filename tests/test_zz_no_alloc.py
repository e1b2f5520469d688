"""The allocation-free join entry point against the regular plan path.

``dq_join_agg_noalloc`` exists for callers that cannot allocate device memory
themselves (a host program that owns every device allocation through its own
pool, a plugin whose allocator must see every byte, a path where cudaMalloc
would synchronise the device): its hash and group tables live in a fixed-size
device array inside the library.  This test runs the FK-PK join + grouped
SUM/COUNT through that entry point twice in a row (the second call must start
from a cleared array) and compares both results with ``dq_plan_execute`` on the
same plan, bit for bit after a canonical sort.  The device buffers here are
the caller's (allocated by the test through torch), as the entry point expects.

The file name makes pytest collect it last, so a run that stops at the first
failure has run every other test before this one.
"""
import ctypes as C

import numpy as np
import pytest

from canonical import canonical_rows

pytestmark = pytest.mark.gpu


def _plan_result(db):
    from dogqc_b200 import workloads
    from dogqc_b200.engine import Engine
    from dogqc_b200.relational import RelationalAlgebra
    alg = RelationalAlgebra(db)
    plan, cfg = workloads.build("c1", alg)
    plan = alg.resolveAlgebraPlan(plan, cfg)
    e = Engine(0)
    try:
        e.register_database(db)
        p = e.prepare(plan)
        res = p.execute()
        p.free()
    finally:
        e.close()
    assert res.names == ["d_nation", "sum_measure", "cnt"]
    return canonical_rows(res.rows())


def _noalloc_call(lib, dev, max_groups):
    import torch
    from dogqc_b200 import _lib as L
    out_group = torch.zeros(max_groups, dtype=torch.int32, device="cuda")
    out_sum = torch.zeros(max_groups, dtype=torch.int64, device="cuda")
    out_count = torch.zeros(max_groups, dtype=torch.int32, device="cuda")
    out_n = torch.full((1,), -7, dtype=torch.int64, device="cuda")
    a = L.dq_join_agg_args()
    a.build_key, a.build_filter, a.build_group = dev["d_key"], dev["d_segment"], dev["d_nation"]
    a.filter_value = 1
    a.build_rows = dev["build_rows"]
    a.probe_key, a.probe_value = dev["f_fk"], dev["f_measure"]
    a.probe_rows = dev["probe_rows"]
    a.out_group, a.out_sum, a.out_count = out_group.data_ptr(), out_sum.data_ptr(), out_count.data_ptr()
    a.out_ngroups = out_n.data_ptr()
    a.max_groups = max_groups
    torch.cuda.synchronize()
    L.check(lib.dq_join_agg_noalloc(C.byref(a), None))
    torch.cuda.synchronize()
    return int(out_n.item()), out_group, out_sum, out_count


def _noalloc_result(lib, dev, max_groups):
    n, out_group, out_sum, out_count = _noalloc_call(lib, dev, max_groups)
    assert n >= 0
    g = out_group[:n].cpu().numpy()
    s = out_sum[:n].cpu().numpy().view(np.uint64)
    c = out_count[:n].cpu().numpy()
    return canonical_rows(zip(g.tolist(), s.tolist(), c.tolist()))


def _device_columns(db):
    import torch
    dim, fact = db["dim"], db["fact"]
    keep = {}
    dev = {}
    for t in (dim, fact):
        for name, col in t.columns.items():
            arr = np.ascontiguousarray(col)
            tt = torch.from_numpy(arr.view(np.uint8).copy()).cuda()
            keep[name] = tt
            dev[name] = tt.data_ptr()
    dev["build_rows"], dev["probe_rows"] = dim.size, fact.size
    return keep, dev


def test_noalloc_join_matches_plan_execute_twice():
    from dogqc_b200 import _lib as L
    from dogqc_b200 import workloads
    db = workloads.gen_c1(0.01)
    want = _plan_result(db)
    keep, dev = _device_columns(db)
    lib = L.lib()
    first = _noalloc_result(lib, dev, 64)
    second = _noalloc_result(lib, dev, 64)
    assert first == want
    assert second == want
    del keep


def test_noalloc_reports_groups_that_do_not_fit():
    """25 nations into an output of 4 groups: -1, and the next call with room
    for all groups gives the full result again."""
    from dogqc_b200 import _lib as L
    from dogqc_b200 import workloads
    db = workloads.gen_c1(0.01)
    want = _plan_result(db)
    keep, dev = _device_columns(db)
    lib = L.lib()
    n, _, _, _ = _noalloc_call(lib, dev, 4)
    assert n == -1
    assert _noalloc_result(lib, dev, 64) == want
    del keep


def test_noalloc_rejects_oversized_build():
    from dogqc_b200 import _lib as L
    lib = L.lib()
    a = L.dq_join_agg_args()
    a.build_key = a.build_filter = a.build_group = 1
    a.out_group = a.out_sum = a.out_count = a.out_ngroups = 1
    a.build_rows = L.NOALLOC_MAX_BUILD_ROWS + 1
    a.max_groups = 16
    status = lib.dq_join_agg_noalloc(C.byref(a), None)
    assert status == L.ERR_INVALID
    assert b"exceeds" in lib.dq_last_error(None)
