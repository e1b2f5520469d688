"""The multithreaded C++ evaluator of the plan IR (oracle/cpu_eval.cpp), the
timed CPU baseline, pinned on the reference's own results: every small golden
case row for row and the full-size cases that evaluate in seconds by their
checksums, with one and with several threads (morsel order and merges must not
change a result)."""
import pytest

from canonical import canonical_checksum
from helpers import golden, golden_cases, make_case, reference_rows, result_checksum

SMALL = [c for c in golden_cases() if golden(c)["spec"]["scale"] < 0.1]
FULL = ["c0", "c1", "c5", "c7", "c8", "c11", "c13", "c14", "c15_m", "c16", "c17", "c18", "c19"]


def _run(case, threads):
    import cpu_eval
    g = golden(case)
    db, alg, plan = make_case(g["spec"])
    names, rows, _ = cpu_eval.Prepared(db, plan, threads=threads).run()
    return g, names, rows


@pytest.mark.parametrize("threads", [1, 4])
@pytest.mark.parametrize("case", SMALL)
def test_small_cases_match_reference(case, threads):
    g, names, rows = _run(case, threads)
    assert names == g["columns"]
    assert reference_rows(rows, g["spec"]) == g["rows"]


@pytest.mark.parametrize("case", FULL)
def test_full_size_matches_reference(case):
    g, names, rows = _run(case, 4)
    assert len(rows) == g["nrows"]
    assert result_checksum(rows, g["spec"]) == g["checksum"]


def test_evaluates_the_ir_the_device_prepares():
    """The evaluator reads the descriptors Lowering.ir() builds (the IR the
    device engine prepares), not the operator tree."""
    import cpu_eval
    from dogqc_b200 import workloads
    from dogqc_b200.relational import RelationalAlgebra
    db = workloads.gen_c1(0.001)
    alg = RelationalAlgebra(db)
    plan, cfg = workloads.build("c1", alg)
    plan = alg.resolveAlgebraPlan(plan, cfg)
    p = cpu_eval.Prepared(db, plan, threads=2)
    assert p.desc.npipes == len(p.lowering.pipes)
    names, rows, seconds = p.run()
    assert names == ["d_nation", "sum_measure", "cnt"] and len(rows) == 25 and seconds > 0
