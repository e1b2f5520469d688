"""Host-side lowering of every workload plan into the pipeline IR (no GPU)."""
import pytest

from dogqc_b200 import _lib as L
from dogqc_b200 import workloads
from dogqc_b200.lowering import Lowering, Unsupported, common_type
from dogqc_b200.relational import RelationalAlgebra

SCALES = {"c0": 0.001, "c1": 0.001, "c2": 0.0005, "c3": 0.0002}


@pytest.mark.parametrize("name", sorted(SCALES))
def test_workload_lowers(name):
    db = workloads.GENERATORS[name](SCALES[name])
    alg = RelationalAlgebra(db)
    plan, cfg = workloads.build(name, alg)
    plan = alg.resolveAlgebraPlan(plan, cfg)
    lw = Lowering(plan)
    desc, keep = lw.ir()
    assert desc.npipes == len(lw.pipes) >= 2
    for p in lw.pipes:
        assert p.ops[-1]["kind"] >= L.OP_AGG
    sinks = [p.ops[-1]["kind"] for p in lw.pipes]
    if name == "c2":
        assert sinks[:2] == [L.OP_MM_COUNT, L.OP_MM_SCATTER]
        assert any(o["kind"] == L.OP_EXPAND for o in lw.pipes[2].ops)
    if name == "c1":
        assert sinks == [L.OP_BUILD, L.OP_AGG, L.OP_EMIT]
    assert lw.result_names


def test_c_conversions():
    assert common_type("i8", "i8") == "i32"
    assert common_type("i32", "u32") == "u32"
    assert common_type("u32", "i64") == "i64"
    assert common_type("i32", "u64") == "u64"


def test_float_constants_rejected():
    import dogqc_b200.scalar as scal
    from dogqc_b200.types import Type
    db = workloads.gen_c0(0.0001)
    alg = RelationalAlgebra(db)
    plan = alg.map("x", scal.MulExpr(scal.AttrExpr("l_extendedprice"), scal.ConstExpr("0.5", Type.FLOAT)),
                   alg.scan("lineitem"))
    plan = alg.resolveAlgebraPlan(plan, {})
    with pytest.raises(Unsupported):
        Lowering(plan)


def _reference_front_end():
    import os
    import sys
    ref = os.environ.get("DOGQC_REFERENCE", "/root/reference")
    if not os.path.isdir(os.path.join(ref, "dogqc")):
        pytest.skip("reference source tree not present")
    sys.path.insert(0, ref)
    try:
        import dogqc.scalarAlgebra as rscal
        from dogqc.relationalAlgebra import RelationalAlgebra as RAlg, Reduction as RRed
        from dogqc.types import Type as RType
    finally:
        sys.path.remove(ref)
    return rscal, RAlg, RRed, RType


def _fingerprint(roots):
    """Operator ids, kinds, outputs (attribute ids, names, types, in order),
    estimates and hints of every node, walked in translation order."""
    out = []

    def walk(n):
        kids = [getattr(n, k) for k in ("child", "leftChild", "rightChild") if hasattr(n, k)]
        for k in kids:
            walk(k)
        rel = [(i, a.name, a.dataType.name, a.lastUse, tuple(a.identifiers)) for i, a in n.outRelation.items()]
        extra = tuple((k, str(getattr(n, k))) for k in ("multimatch", "htSizeFactor", "numgroups", "selectivity")
                      if hasattr(n, k))
        out.append((type(n).__name__, n.opId, n.tupleNum, tuple(rel), extra))

    for r in roots:
        walk(r)
    return out


@pytest.mark.parametrize("name", ["c0", "c1", "c2", "c3", "c5", "c7", "c8", "c9", "c9p", "c10", "c10p"])
def test_reference_front_end_trees_lower(name):
    """Trees built by the reference's own classes and by this package's front
    end agree node for node (ids, outputs in order, estimates, hints) and
    lower to the same IR."""
    import types as pytypes
    rscal, RAlg, RRed, RType = _reference_front_end()
    db = workloads.GENERATORS[name](0.001)
    schema = {}
    for t, e in db.schema.items():
        e = dict(e)
        e["attributes"] = type(e["attributes"])((a, RType[ty.name]) for a, ty in e["attributes"].items())
        schema[t] = e
    alg = RAlg(pytypes.SimpleNamespace(schema=schema))
    plan, cfg = workloads.PLANS[name](alg, rscal, RType, RRed)
    plan = alg.resolveAlgebraPlan(plan, cfg)
    ours = RelationalAlgebra(db)
    p2, c2 = workloads.build(name, ours)
    p2 = ours.resolveAlgebraPlan(p2, c2)
    assert _fingerprint(plan) == _fingerprint(p2)
    a, b = Lowering(plan), Lowering(p2)
    assert a.describe() == b.describe()


def _lowered(name, scale=0.001):
    db = workloads.GENERATORS[name](scale)
    alg = RelationalAlgebra(db)
    plan, cfg = workloads.build(name, alg)
    return Lowering(alg.resolveAlgebraPlan(plan, cfg))


def test_inner_join_build_key_read_from_probe_side():
    """C3 groups by its first dimension's key: above the inner join that key
    equals the fact row's foreign key (same type), so the join table keeps no
    payload and the aggregation reads the fact column."""
    lw = _lowered("c3", 0.0002)
    fact = lw.pipes[3]
    probes = [o for o in fact.ops if o["kind"] == L.OP_PROBE]
    assert len(probes) == 3
    assert all(len(lw.res[o["res"]].pay_ctype) == 0 for o in probes)
    agg = fact.ops[-1]
    assert agg["kind"] == L.OP_AGG
    key = fact.lists[agg["list"]]
    assert fact.slots[key]["kind"] == L.SLOT_COL
    assert fact.cols[fact.slots[key]["src"]] == "f_fk1"


def test_costly_multimap_build_side_is_staged_once():
    """Q13: the orders behind the outer join pass a NOT LIKE on their
    comments.  One pipeline evaluates it and writes the surviving rows' keys
    and payload to a temp table; the multimap's count and scatter passes scan
    that table instead of the comments."""
    lw = _lowered("c17")
    sinks = [p.ops[-1]["kind"] for p in lw.pipes]
    assert sinks[:3] == [L.OP_EMIT, L.OP_MM_COUNT, L.OP_MM_SCATTER]
    stage = lw.pipes[0].ops[-1]["res"]
    assert lw.res[stage].kind == L.RES_OUTPUT
    assert [p.source_kind for p in lw.pipes[1:3]] == [L.SRC_OUTPUT, L.SRC_OUTPUT]
    assert all(p.source_res == stage for p in lw.pipes[1:3])
    assert any(o["kind"] == L.OP_LIKE for o in lw.pipes[0].ops)
    assert not any(o["kind"] == L.OP_LIKE for p in lw.pipes[1:3] for o in p.ops)


def test_plain_multimap_build_side_is_scanned_per_pass():
    """C2's build side is a plain scan: both passes read the table."""
    lw = _lowered("c2", 0.0005)
    assert [p.ops[-1]["kind"] for p in lw.pipes[:2]] == [L.OP_MM_COUNT, L.OP_MM_SCATTER]
    assert [p.source_kind for p in lw.pipes[:2]] == [L.SRC_TABLE, L.SRC_TABLE]
