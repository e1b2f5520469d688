"""Strings without a GPU: how the lowering expresses substrings, comparisons of
two strings and string join keys in the plan IR, what it refuses, and the C++
evaluator of that IR against the oracle on the substring and comparison edge
cases (windows before, at and past a string's ends, nested windows, strings
carried through unique and multimatch joins)."""
import pytest

import dogqc_b200.scalar as scal
from canonical import canonical_rows
from dogqc_b200 import _lib as L
from dogqc_b200.lowering import Lowering, Unsupported
from dogqc_b200.relational import RelationalAlgebra, Reduction
from dogqc_b200.types import Type
from evaluator import run_plan
from helpers import make_case
import string_cases


def ops_of(plan):
    return [o for p in Lowering(plan).pipes for o in p.ops]


def test_substring_is_one_op_on_the_reference():
    db = string_cases.edge_db(200)
    ops = ops_of(string_cases.substring_plan(db, (3, 20), (2, 5)))
    subs = [o for o in ops if o["kind"] == L.OP_SUBSTR]
    assert len(subs) == 2
    assert [(o["imm"] & 0xffffffff, o["imm"] >> 32) for o in subs] == [(3, 20), (2, 5)]
    assert any(o["kind"] == L.OP_STRREF for o in ops)


def test_two_string_equality_uses_the_two_slot_form():
    db = string_cases.edge_db(200)
    ops = ops_of(string_cases.equal_strings_plan(db))
    eqs = [o for o in ops if o["kind"] == L.OP_STREQ]
    assert sum(o["res"] == -1 for o in eqs) == 2 and sum(o["res"] >= 0 for o in eqs) == 1


@pytest.mark.parametrize("variant,kind", [("unique", L.RES_UNIQUE), ("multi", L.RES_MULTI), ("semi", L.RES_UNIQUE),
                                          ("exists", L.RES_MULTI)])
def test_string_join_keys_are_string_typed_tables(variant, kind):
    db, alg, plan = make_case({"workload": "c15", "scale": 0.001, "plan_kw": {"variant": variant}})
    lw = Lowering(plan)
    tables = [r for r in lw.res if r.kind in (L.RES_UNIQUE, L.RES_MULTI)]
    assert [r.kind for r in tables] == [kind] and tables[0].key_ctype == ["str"]


def _plan_with(db, expr_of):
    alg = RelationalAlgebra(db)
    m = alg.map("x", expr_of(), alg.scan("t"))
    agg = alg.aggregation(["x"], [(Reduction.COUNT, "", "cnt")], m)
    return alg.resolveAlgebraPlan(agg, {})


@pytest.mark.parametrize("expr_of", [
    lambda: scal.SubstringExpr(scal.AttrExpr("s"), scal.ConstExpr("250", Type.INT), scal.ConstExpr("10", Type.INT)),
    lambda: scal.SubstringExpr(scal.AttrExpr("s"), scal.AttrExpr("k"), scal.ConstExpr("2", Type.INT)),
])
def test_substrings_the_reference_layout_cannot_hold_are_refused(expr_of):
    db = string_cases.edge_db(100)
    with pytest.raises(Unsupported):
        Lowering(_plan_with(db, expr_of))


def test_ordering_strings_is_refused():
    db = string_cases.edge_db(100)
    alg = RelationalAlgebra(db)
    sel = alg.selection(scal.SmallerExpr(scal.AttrExpr("s"), scal.AttrExpr("t")), alg.scan("t"))
    plan = alg.resolveAlgebraPlan(alg.aggregation([], [(Reduction.COUNT, "", "c")], sel), {})
    with pytest.raises(Unsupported):
        Lowering(plan)


@pytest.mark.parametrize("window,nested", string_cases.WINDOWS)
def test_cpu_evaluator_substrings_match_oracle(window, nested):
    import cpu_eval
    db = string_cases.edge_db()
    plan = string_cases.substring_plan(db, window, nested)
    assert canonical_rows(cpu_eval.Prepared(db, plan, 3).run()[1]) == canonical_rows(run_plan(db, plan)[1])


@pytest.mark.parametrize("make", [string_cases.equal_strings_plan, string_cases.like_joined_plan])
def test_cpu_evaluator_string_comparisons_match_oracle(make):
    import cpu_eval
    db = string_cases.edge_db()
    plan = make(db)
    assert canonical_rows(cpu_eval.Prepared(db, plan, 3).run()[1]) == canonical_rows(run_plan(db, plan)[1])


@pytest.mark.parametrize("variant", ["unique", "multi", "semi", "anti", "exists", "dup"])
def test_cpu_evaluator_string_join_keys_match_oracle(variant):
    import cpu_eval
    db, alg, plan = make_case({"workload": "c15", "scale": 0.02, "plan_kw": {"variant": variant}})
    assert canonical_rows(cpu_eval.Prepared(db, plan, 4).run()[1]) == canonical_rows(run_plan(db, plan)[1])


@pytest.mark.parametrize("kind", ["group", "unique", "multi", "semi", "anti"])
def test_cpu_evaluator_long_string_keys_match_oracle(kind):
    import cpu_eval
    db = string_cases.long_db()
    plan = string_cases.long_key_plan(db, kind)
    assert canonical_rows(cpu_eval.Prepared(db, plan, 3).run()[1]) == canonical_rows(run_plan(db, plan)[1])


def test_string_column_reads_as_bytes():
    """A string result column stays a heap and offsets; reading it gives the
    rows' bytes (by index, negative too, by iteration and as a list)."""
    import numpy as np
    from dogqc_b200.database import StringColumn
    from dogqc_b200.engine import Result
    words = [b"", b"a", b"hello world", b"x" * 40, b"AB-12"]
    col = StringColumn.from_list(words)
    assert len(col) == 5
    assert col.tolist() == words
    assert list(col) == words
    assert [col[i] for i in range(5)] == words
    assert col[-1] == b"AB-12" and col[-5] == b""
    with pytest.raises(IndexError):
        col[5]
    with pytest.raises(IndexError):
        col[-6]
    res = Result(["s", "k"], [L.STR, L.I32], [col, np.arange(5, dtype=np.int32)], 5)
    assert res.rows() == list(zip(words, range(5)))
    assert "hello world" in res.format_sample()
