"""Device parity: the CUDA engine against the reference's golden results and the oracle.

Every result set is compared bit-exactly after a canonical sort: against the rows
the reference's own generated pipeline produced (tests/golden, small cases and
edge cases), against its checksums at the full workload sizes, and against the
CPU oracle for cases the fixtures do not cover (tile boundaries, deferred
expansion ranges, hash-table growth, output growth, plain-load staging).
"""
import numpy as np
import pytest

from canonical import canonical_checksum, canonical_rows
from evaluator import run_plan
from helpers import golden, golden_cases, make_case, reference_rows, result_checksum

pytestmark = pytest.mark.gpu

SMALL = [c for c in golden_cases() if golden(c)["spec"]["scale"] < 0.1]
FULL = ["c0", "c1", "c2", "c3", "c5", "c7", "c8", "c11", "c12", "c13", "c14", "c15_m", "c16", "c17", "c18", "c19"]


@pytest.fixture(scope="module")
def engine():
    from dogqc_b200.engine import Engine
    e = Engine(0)
    yield e
    e.close()


def run_engine(engine, db, plan, options=None):
    engine.register_database(db, force=True)
    p = engine.prepare(plan, options)
    try:
        return p.execute(), p.timing()
    finally:
        p.free()


@pytest.mark.parametrize("case", SMALL)
def test_small_cases_match_reference(engine, case):
    g = golden(case)
    db, alg, plan = make_case(g["spec"])
    res, _ = run_engine(engine, db, plan)
    assert res.names == g["columns"]
    assert reference_rows(res.rows(), g["spec"]) == g["rows"]


@pytest.mark.parametrize("case", FULL)
def test_full_size_matches_reference(engine, case):
    g = golden(case)
    db, alg, plan = make_case(g["spec"])
    res, t = run_engine(engine, db, plan)
    assert res.nrows == g["nrows"]
    assert result_checksum(res.rows(), g["spec"]) == g["checksum"]
    assert t["kernel_launches"] >= len(t["pipeline_ms"])


def _plan(name, scale, gen_kw=None, plan_kw=None):
    from dogqc_b200 import workloads
    from dogqc_b200.relational import RelationalAlgebra
    db = workloads.GENERATORS[name](scale, **(gen_kw or {}))
    alg = RelationalAlgebra(db)
    plan, cfg = workloads.build(name, alg, **(plan_kw or {}))
    return db, alg.resolveAlgebraPlan(plan, cfg)


@pytest.mark.parametrize("rows", [1, 15, 1023, 1024, 1025, 3000])
def test_tile_boundaries(engine, rows):
    scale = rows / 6_000_000
    db, plan = _plan("c0", scale)
    res, _ = run_engine(engine, db, plan)
    assert canonical_rows(res.rows()) == canonical_rows(run_plan(db, plan)[1])


def test_deferred_expansion_matches_oracle():
    """Force wide expansion ranges into the cross-CTA deferral path."""
    from dogqc_b200.engine import Engine
    e = Engine(0, defer_threshold=64)
    try:
        db, plan = _plan("c2", 0.002)
        res, _ = run_engine(e, db, plan)
        assert canonical_rows(res.rows()) == canonical_rows(run_plan(db, plan)[1])
    finally:
        e.close()


def test_plain_staging_matches_tma(engine):
    from dogqc_b200 import _lib as L
    from dogqc_b200.engine import Engine
    db, plan = _plan("c3", 0.001)
    want = canonical_rows(run_plan(db, plan)[1])
    e = Engine(0, flags=L.CFG_NO_TMA)
    try:
        res, _ = run_engine(e, db, plan)
    finally:
        e.close()
    assert canonical_rows(res.rows()) == want
    res2, _ = run_engine(engine, db, plan)
    assert canonical_rows(res2.rows()) == want


def test_hash_table_growth(engine):
    """Estimates far below the real sizes: tables are grown and the plan re-run."""
    from dogqc_b200 import workloads
    from dogqc_b200.relational import RelationalAlgebra
    db = workloads.gen_c3(0.001)
    alg = RelationalAlgebra(db)
    plan, cfg = workloads.build("c3", alg)
    for k in cfg:
        cfg[k] = {kk: (0.0001 if kk == "selectivity" else (3 if kk == "numgroups" else v))
                  for kk, v in cfg[k].items()}
    plan = alg.resolveAlgebraPlan(plan, cfg)
    res, _ = run_engine(engine, db, plan)
    assert canonical_rows(res.rows()) == canonical_rows(run_plan(db, plan)[1])


def test_tile_sizes(engine):
    from dogqc_b200.engine import Engine
    db, plan = _plan("c2", 0.001)
    want = canonical_rows(run_plan(db, plan)[1])
    for tile in (256, 2048):
        e = Engine(0, tile_rows=tile)
        try:
            res, _ = run_engine(e, db, plan)
        finally:
            e.close()
        assert canonical_rows(res.rows()) == want, tile


def test_repeated_execution_is_stable(engine):
    db, plan = _plan("c1", 0.01)
    engine.register_database(db, force=True)
    p = engine.prepare(plan)
    try:
        first = canonical_rows(p.execute().rows())
        for _ in range(3):
            assert canonical_rows(p.execute().rows()) == first
    finally:
        p.free()
    assert first == canonical_rows(run_plan(db, plan)[1])


def test_backend_drop_in(engine):
    """The reference's driver sequence: translate -> gencode -> compile -> execute."""
    from dogqc_b200.backend import Backend
    from dogqc_b200 import workloads
    from dogqc_b200.relational import RelationalAlgebra
    db = workloads.gen_c0(0.001)
    alg = RelationalAlgebra(db)
    plan, cfg = workloads.build("c0", alg)
    plan = alg.resolveAlgebraPlan(plan, cfg)
    b = Backend(alg, engine=engine)
    b.gencode(alg.translateToCompilerPlan(plan, b))
    b.compile("c0")
    res = b.execute(quiet=True)
    assert canonical_checksum(res.rows()) == golden("c0_s")["checksum"]


@pytest.mark.parametrize("name,scale", [("c0", 0.001), ("c1", 0.001), ("c3", 0.0002)])
def test_tile_kernel_matches_row_kernel(engine, name, scale):
    """Pipelines without expansion can run on the row kernel; it must give
    the same results as the default tile kernel."""
    from dogqc_b200 import _lib as L
    from dogqc_b200.engine import Engine
    db, plan = _plan(name, scale)
    want = canonical_rows(run_plan(db, plan)[1])
    e = Engine(0, flags=L.CFG_ROW_KERNEL)
    try:
        res, _ = run_engine(e, db, plan)
    finally:
        e.close()
    assert canonical_rows(res.rows()) == want
    res2, _ = run_engine(engine, db, plan)
    assert canonical_rows(res2.rows()) == want
