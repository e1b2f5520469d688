"""Semi and anti joins on the device against the CPU oracle.

The reference's own generated pipelines pin the cases in tests/golden
(``ref_c11*``, ``ref_c12*``, ``ref_c13*``, checked by test_gpu_parity); these
tests add sizes and plan variants the fixtures do not cover: EXISTS without a
condition on a unique key table (Q4 shape, NOT EXISTS of Q22), EXISTS and NOT
EXISTS with a condition walked over a multimap (Q21 shape) with the hint
``multimatch`` either way, an empty build side (every probe row rejected for
EXISTS, kept for NOT EXISTS), and the join behind a lane refill.
"""
import pytest

from canonical import canonical_rows
from evaluator import run_plan

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def engine():
    from dogqc_b200.engine import Engine
    e = Engine(0)
    yield e
    e.close()


def _check(engine, name, scale, plan_kw=None, gen_kw=None):
    from dogqc_b200 import workloads
    from dogqc_b200.relational import RelationalAlgebra
    db = workloads.GENERATORS[name](scale, **(gen_kw or {}))
    alg = RelationalAlgebra(db)
    plan, cfg = workloads.build(name, alg, **(plan_kw or {}))
    plan = alg.resolveAlgebraPlan(plan, cfg)
    engine.register_database(db, force=True)
    p = engine.prepare(plan)
    try:
        first = p.execute()
        again = p.execute()   # the second run replays the captured graph
    finally:
        p.free()
    names, rows = run_plan(db, plan)
    assert first.names == names
    want = canonical_rows(rows)
    assert canonical_rows(first.rows()) == want
    assert canonical_rows(again.rows()) == want
    return len(rows)


@pytest.mark.parametrize("scale", [0.0001, 0.003, 0.05])
def test_exists_without_condition(engine, scale):
    assert _check(engine, "c11", scale) >= 0


@pytest.mark.parametrize("scale", [0.0001, 0.003, 0.05])
@pytest.mark.parametrize("multimatch", [True, False])
def test_exists_and_not_exists_with_conditions(engine, scale, multimatch):
    _check(engine, "c12", scale, plan_kw={"multimatch": multimatch})


@pytest.mark.parametrize("scale", [0.01, 0.2])
@pytest.mark.parametrize("multimatch", [True, False])
def test_not_exists_without_condition(engine, scale, multimatch):
    assert _check(engine, "c13", scale, plan_kw={"multimatch": multimatch}) > 0


def test_empty_build_side(engine):
    """No late line item: EXISTS rejects every order; NOT EXISTS over an empty
    build side keeps every customer."""
    assert _check(engine, "c11", 0.01, plan_kw={"late_slack": 100}) == 0
    assert _check(engine, "c13", 0.01, plan_kw={"flag_cut": 1000}) == 25
