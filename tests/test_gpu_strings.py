"""Strings on the GPU, against the oracle.

A scanned string travels as a 64-bit reference (its plan string source, a
substring window and its row); join keys and group keys of string type hash
and compare the bytes behind the references, and string result columns are
gathered into offsets and a heap on the device after the run.  Cases: grouping
by two variable-length strings (Q12 shape), a projection carrying strings,
fixed-width strings, tables that came in as text, strings carried from a
join's build side (Q10 shape), string predicates before and after a join with
string group keys of an aggregation over an aggregation (Q16 shape), joins on
string keys (unique, multimatch, semi, anti, semi with a condition, a build
side repeating its keys), substrings in IN lists, as map results and group
keys (Q22 shape), substring windows at and past the string's ends, and the
prebuilt kernels refusing string references."""
import numpy as np
import pytest

from canonical import canonical_rows
from evaluator import run_plan
from helpers import make_case
import string_cases

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


STRING_WORKLOADS = [
    ("c14", {}, 0.05), ("c14", {"late_filter": True}, 0.05), ("c14", {}, 1.0), ("c14", {"late_filter": True}, 1.0),
    ("c15", {"variant": "unique"}, 0.05), ("c15", {"variant": "multi"}, 0.05), ("c15", {"variant": "semi"}, 0.05),
    ("c15", {"variant": "anti"}, 0.05), ("c15", {"variant": "exists"}, 0.05), ("c15", {"variant": "dup"}, 0.05),
    ("c15", {"variant": "unique"}, 1.0), ("c15", {"variant": "semi"}, 1.0), ("c15", {"variant": "dup"}, 0.2),
    ("c15", {"variant": "exists"}, 0.2), ("c16", {}, 0.05), ("c16", {}, 1.0)]


@pytest.mark.parametrize("workload,plan_kw,scale", STRING_WORKLOADS)
def test_string_joins_predicates_and_substrings_match_oracle(engine, workload, plan_kw, scale):
    db, alg, plan = make_case({"workload": workload, "scale": scale, "plan_kw": plan_kw})
    names, want = run_plan(db, plan)
    res = run(engine, db, plan)
    assert res.names == names
    assert canonical_rows(res.rows()) == canonical_rows(want)


@pytest.mark.parametrize("window,nested", string_cases.WINDOWS)
def test_substring_windows_match_oracle(engine, window, nested):
    db = string_cases.edge_db()
    plan = string_cases.substring_plan(db, window, nested)
    assert canonical_rows(run(engine, db, plan).rows()) == canonical_rows(run_plan(db, plan)[1])


@pytest.mark.parametrize("make", [string_cases.equal_strings_plan, string_cases.like_joined_plan])
def test_string_comparisons_through_joins_match_oracle(engine, make):
    db = string_cases.edge_db()
    plan = make(db)
    assert canonical_rows(run(engine, db, plan).rows()) == canonical_rows(run_plan(db, plan)[1])


@pytest.mark.parametrize("kind", ["group", "unique", "multi", "semi", "anti"])
def test_long_string_keys_match_oracle(engine, kind):
    """Keys of up to 300 bytes: hashed (and, after a multimatch expansion,
    compared) by whole warps, a word or a byte per lane, giving the values a
    lane computes alone for the short ones."""
    db = string_cases.long_db()
    plan = string_cases.long_key_plan(db, kind)
    assert canonical_rows(run(engine, db, plan).rows()) == canonical_rows(run_plan(db, plan)[1])


@pytest.mark.parametrize("pattern", ["%#1%", "%ABC%xyz%", "%!\"#%#4%", "%pqrs%PQRS%#%", "%~!%", "%abc%abc%abc%abc%",
                                     "%a%b%c%d%e%f%g%h%", "%a%b%c%d%e%f%g%h%i%", "%AB_D%", "A%", "%#59", "%",
                                     "%%", "%#%%1%", "%~", "%}~!\"#$%&'()*+,-./0123456789:;<=>?@ABCDEFG%"])
def test_like_on_long_strings_matches_oracle(engine, pattern):
    """Strings of up to 300 bytes: patterns '%L1%...%Ln%' find their literals
    one after another, eight bytes a step; patterns with '_', an empty literal
    or a missing leading or trailing '%' run the reference matcher's algorithm.
    Both give its answers."""
    import dogqc_b200.scalar as scal
    from dogqc_b200.relational import RelationalAlgebra
    from dogqc_b200.types import Type
    db = string_cases.long_db()
    alg = RelationalAlgebra(db)
    sel = alg.selection(scal.LikeExpr(scal.AttrExpr("fk"), scal.ConstExpr(pattern, Type.STRING)), alg.scan("f"))
    plan = alg.resolveAlgebraPlan(alg.projection(["fv", "fk"], sel), {})
    want = canonical_rows(run_plan(db, plan)[1])
    assert canonical_rows(run(engine, db, plan).rows()) == want


@pytest.mark.parametrize("pattern", ["%ABCDEFGHIJKLMNOP%", "xxxxxxxxxxxxxxxxxxxx%", "%JKLMNOPQRSTUVWXYZABC%",
                                     "hello world%"])
def test_long_like_patterns_match_oracle(engine, pattern):
    """Patterns of 16 bytes and more (held on the heap by the host string
    that keeps them, not inline) survive the pipeline's re-derivation at run
    time."""
    import dogqc_b200.scalar as scal
    from dogqc_b200.relational import RelationalAlgebra
    from dogqc_b200.types import Type
    db = string_cases.edge_db(2000)
    alg = RelationalAlgebra(db)
    sel = alg.selection(scal.LikeExpr(scal.AttrExpr("s"), scal.ConstExpr(pattern, Type.STRING)), alg.scan("t"))
    plan = alg.resolveAlgebraPlan(alg.projection(["k", "s"], sel), {})
    want = canonical_rows(run_plan(db, plan)[1])
    assert want and canonical_rows(run(engine, db, plan).rows()) == want


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


def test_prebuilt_kernels_refuse_string_references(engine):
    """The prebuilt kernels read strings in place only: plans whose strings
    travel as references (group keys, results, join keys, substrings) are
    refused there; batches and served requests take them (test_gpu_batch,
    test_gpu_serve)."""
    from dogqc_b200 import _lib as L
    from dogqc_b200.engine import Engine
    prebuilt = Engine(0, flags=L.CFG_NO_JIT)
    try:
        for case in ({"workload": "c9", "scale": 0.002}, {"workload": "c16", "scale": 0.002},
                     {"workload": "c15", "scale": 0.002, "plan_kw": {"variant": "unique"}}):
            db, alg, plan = make_case(case)
            prebuilt.register_database(db, force=True)
            with pytest.raises(L.DqError) as e:
                prebuilt.prepare(plan)
            assert e.value.status == L.ERR_UNSUPPORTED
    finally:
        prebuilt.close()
