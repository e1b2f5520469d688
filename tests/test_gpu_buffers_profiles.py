"""setBuffers and setProfilers of the drop-in Backend on the device.

setBuffers places the lane refill where the reference's CudaCompiler places its
LaneRefill; the run the reference made with its refill after c0's selection
(tests/golden/ref_c0_lr.json) pins the result.  setProfilers counts, per
profiled operator, warp steps by active lanes where the operator hands its
rows on; summed over the histogram, active lanes are exactly the rows that
reach that point (checked against the CPU oracle: scanned rows, rows through a
selection, matched probe rows, join pairs)."""
import numpy as np
import pytest

from canonical import canonical_rows
from evaluator import run_plan
from helpers import golden, make_case, reference_rows

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def engine():
    from dogqc_b200.engine import Engine
    e = Engine(0)
    yield e
    e.close()


def _nodes(root, kind):
    out, stack = [], [root]
    while stack:
        n = stack.pop()
        if type(n).__name__ == kind:
            out.append(n)
        stack.extend(getattr(n, "inputs", ()))
    return out


def _backend(engine, alg, plan, buffers=None, profilers=None):
    from dogqc_b200.backend import Backend
    b = Backend(alg, engine=engine)
    if buffers is not None:
        b.setBuffers(buffers)
    if profilers:
        b.setProfilers(profilers)
    b.gencode(alg.translateToCompilerPlan(plan, b))
    b.compile("q")
    return b


def test_set_buffers_matches_the_references_refill_run(engine):
    g = golden("c0_lr")
    db, alg, plan = make_case(g["spec"])
    engine.register_database(db, force=True)
    b = _backend(engine, alg, plan, buffers=[alg.selectionNodes[0].opId])
    assert "refill buffer" in b.plan.source(0)
    res = b.execute(quiet=True)
    assert reference_rows(res.rows(), g["spec"]) == g["rows"]


def _active(counts):
    return sum(i * c for i, c in enumerate(counts))


def test_profiles_count_the_rows_through_scan_and_selection(engine):
    from dogqc_b200 import workloads as W
    from dogqc_b200.relational import RelationalAlgebra
    db = W.gen_c0(0.01)
    alg = RelationalAlgebra(db)
    plan, cfg = W.build("c0", alg)
    plan = alg.resolveAlgebraPlan(plan, cfg)
    scan = _nodes(plan[0], "Scan")[0]
    sel = alg.selectionNodes[0]
    engine.register_database(db, force=True)
    b = _backend(engine, alg, plan, profilers=[scan.opId, sel.opId])
    res = b.execute(quiet=True)
    prof = b.profiles()
    n = db["lineitem"].size
    cutoff = W.EPOCH_1992 + W.DATE_RANGE - 1 - 90
    passing = int(np.count_nonzero(db["lineitem"].columns["l_shipdate"] <= cutoff))
    assert _active(prof[scan.opId]) == n
    assert _active(prof[sel.opId]) == passing
    assert canonical_rows(res.rows()) == canonical_rows(run_plan(db, plan)[1])
    # a second run reports that run's counts only
    b.execute(quiet=True)
    assert _active(b.profiles()[scan.opId]) == n


@pytest.mark.parametrize("name,scale", [("c1", 0.01), ("c2", 0.0005)])
def test_profiles_count_matched_rows_and_pairs(engine, name, scale):
    from dogqc_b200 import workloads as W
    from dogqc_b200.relational import RelationalAlgebra
    db = W.GENERATORS[name](scale)
    alg = RelationalAlgebra(db)
    plan, cfg = W.build(name, alg)
    plan = alg.resolveAlgebraPlan(plan, cfg)
    join = _nodes(plan[0], "EquiJoin")[0]
    engine.register_database(db, force=True)
    b = _backend(engine, alg, plan, profilers=[join.opId])
    b.execute(quiet=True)
    got = _active(b.profiles()[join.opId])
    # the rows the join hands on: a count over the join alone, from the oracle
    from dogqc_b200.relational import Reduction
    alg2 = RelationalAlgebra(db)
    import dogqc_b200.scalar as scal  # noqa: F401
    plan2, cfg2 = W.build(name, alg2)
    j2 = _nodes(plan2, "EquiJoin")[0]
    cnt = alg2.aggregation([], [(Reduction.COUNT, "", "n")], j2)
    cfg2 = dict(cfg2)
    plan2 = alg2.resolveAlgebraPlan(cnt, cfg2)
    want = run_plan(db, plan2)[1][0][0]
    assert got == want
