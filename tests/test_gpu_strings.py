"""String group keys and string result columns on the GPU, against the oracle.

A scanned string travels as a 64-bit reference (its plan string source and
row); group keys of string type hash and compare the bytes behind the
references, and string result columns are gathered into offsets and a heap on
the device after the run.  Cases: grouping by two variable-length strings
(Q12 shape), a projection carrying strings, fixed-width strings, tables that
came in as text, strings carried from a join's build side (Q10 shape), and
the paths that do not take string results (batches,
served requests, the prebuilt kernels) refusing them."""
import numpy as np
import pytest

from canonical import canonical_rows
from evaluator import run_plan
from helpers import make_case

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def engine():
    from dogqc_b200.engine import Engine
    e = Engine(0)
    yield e
    e.close()


def run(engine, db, plan):
    engine.register_database(db, force=True)
    p = engine.prepare(plan)
    try:
        return p.execute()
    finally:
        p.free()


@pytest.mark.parametrize("workload,scale", [("c9", 0.002), ("c9", 0.1), ("c9p", 0.002), ("c9p", 0.1),
                                            ("c10", 0.02), ("c10", 1.0), ("c10p", 0.02), ("c10p", 1.0)])
def test_string_keys_and_results_match_oracle(engine, workload, scale):
    db, alg, plan = make_case({"workload": workload, "scale": scale})
    names, want = run_plan(db, plan)
    res = run(engine, db, plan)
    assert res.names == names
    got = canonical_rows(res.rows())
    assert got == canonical_rows(want)
    assert all(isinstance(r[1 if workload == "c9p" else 0], bytes) for r in got)


def test_fixed_width_string_keys(engine):
    """Strings of one width (read without offsets) as group keys and outputs."""
    from dogqc_b200.database import Database, StringColumn, Table
    db, alg, plan = make_case({"workload": "c9", "scale": 0.01})
    t = db.tables["lineitem"]
    cols = dict(t.columns)
    codes = np.array([list(b"%-4s" % m[:4]) for m in (t.columns["l_shipmode"].get(i) for i in range(t.size))],
                     dtype=np.uint8)
    cols["l_shipmode"] = StringColumn.fixed(codes)
    db2 = Database([Table("lineitem", cols, t.types)])
    assert db2.tables["lineitem"].columns["l_shipmode"].width == 4
    names, want = run_plan(db2, plan)
    assert canonical_rows(run(engine, db2, plan).rows()) == canonical_rows(want)


def test_imported_text_string_keys(engine):
    """The same grouping over a table that came in as .tbl text."""
    from dogqc_b200 import importer
    from tbl_text import table_text
    db, alg, plan = make_case({"workload": "c9", "scale": 0.01})
    t = db.tables["lineitem"]
    from dogqc_b200.engine import Engine
    e = Engine(0)
    try:
        assert importer.load_table(e, t.schema_entry(), table_text(t)) == t.size
        p = e.prepare(plan)
        try:
            got = canonical_rows(p.execute().rows())
        finally:
            p.free()
    finally:
        e.close()
    assert got == canonical_rows(run_plan(db, plan)[1])


def test_paths_without_string_results_refuse_them(engine):
    from dogqc_b200 import _lib as L
    from dogqc_b200.engine import Engine
    from dogqc_b200.lowering import Lowering
    db, alg, plan = make_case({"workload": "c9", "scale": 0.002})
    engine.register_database(db, force=True)
    lw = Lowering(plan)
    with pytest.raises(L.DqError) as e:
        engine.prepare_batch([lw, Lowering(plan)])
    assert e.value.status == L.ERR_UNSUPPORTED
    prebuilt = Engine(0, flags=L.CFG_NO_JIT)
    try:
        prebuilt.register_database(db)
        with pytest.raises(L.DqError) as e:
            prebuilt.prepare(plan)
        assert e.value.status == L.ERR_UNSUPPORTED
    finally:
        prebuilt.close()
    from dogqc_b200 import serve
    srv = serve.Server(engine, slots=2)
    try:
        with pytest.raises(L.DqError) as e:
            srv.submit(lw)
        assert e.value.status == L.ERR_UNSUPPORTED
    finally:
        srv.stop()
