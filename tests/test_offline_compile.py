"""CPU checks of the kernel generator: with DQ_CFG_OFFLINE a context needs no
device, and preparing a plan generates and compiles (NVRTC, sm_100a) every
pipeline's kernel.  Every workload shape compiles without register spills,
under the default launch shape and under the tunings the autotuner searches (a
kernel that spills is recompiled with a minimum of one block per SM in its
launch bounds)."""
import re

import pytest

from dogqc_b200 import _lib as L
from dogqc_b200 import workloads as W
from dogqc_b200.engine import Engine
from dogqc_b200.relational import RelationalAlgebra

SCALE = 0.001


@pytest.fixture(scope="module")
def engine():
    e = Engine(0, flags=L.CFG_OFFLINE)
    yield e
    e.close()


def resolved(engine, name):
    db = W.GENERATORS[name](SCALE)
    alg = RelationalAlgebra(db)
    plan, cfg = W.build(name, alg)
    engine.register_database(db)
    return alg.resolveAlgebraPlan(plan, cfg)


def check_sources(plan, max_spill=0):
    n = len(plan.lowering.pipes)
    assert n >= 1
    for i in range(n):
        src = plan.source(i)
        assert "dq_main" in src, i
        assert "#include" in src
        regs = [int(r) for r in re.findall(r"Used (\d+) registers", src)]
        assert regs and max(regs) <= 128, (i, regs)
        spills = [int(b) for b in re.findall(r"(\d+) bytes spill stores", src)]
        assert spills and max(spills) <= max_spill, (i, spills)


@pytest.mark.parametrize("name", ["c0", "c1", "c2", "c3", "c5", "c7", "c8", "c9", "c9p", "c10", "c10p", "c14", "c15",
                                  "c16", "c17", "c18", "c19"])
def test_every_workload_compiles_offline(engine, name):
    plan = engine.prepare(resolved(engine, name))
    check_sources(plan)
    with pytest.raises(L.DqError):
        plan.execute()


@pytest.mark.parametrize("tuning", [
    {"rows_per_thread": 1, "block_threads": 128},
    {"rows_per_thread": 2, "block_threads": 512, "refill": -1},
    {"rows_per_thread": 4, "block_threads": 256, "unique_slots_pct": 400, "multi_buckets_pct": 50},
    {"rows_per_thread": 2, "block_threads": 256, "ctas_per_sm": 4},
])
@pytest.mark.parametrize("name", ["c1", "c2"])
def test_tuned_launch_shapes_compile(engine, name, tuning):
    plan = engine.prepare(resolved(engine, name), tuning=tuning)
    check_sources(plan)


@pytest.mark.parametrize("shape", ["c0", "c1", "c2", "c3"])
def test_batches_compile_offline(engine, shape):
    """A batch's many-instance kernels (the expansion's deferral and its
    grouped heavy kernel included) compile without a device."""
    from dogqc_b200 import batch
    insts = batch.make_instances(shape, 3, lo=1 << 10, hi=1 << 12)
    batch.register(engine, insts)
    b = batch.prepare_batch(engine, insts, tuning={"rows_per_thread": 2})
    with pytest.raises(L.DqError):
        b.execute()


@pytest.mark.parametrize("name", ["c11", "c12", "c13"])
def test_semi_anti_joins_compile_offline(engine, name):
    plan = engine.prepare(resolved(engine, name))
    check_sources(plan)


def test_conditioned_semi_join_refused_on_prebuilt_kernels():
    """EXISTS with a condition has a generated form only."""
    e = Engine(0, flags=L.CFG_OFFLINE | L.CFG_NO_JIT)
    try:
        with pytest.raises(L.DqError) as err:
            e.prepare(resolved(e, "c12"))
        assert err.value.status == L.ERR_UNSUPPORTED
    finally:
        e.close()


def test_set_buffers_places_the_refill_where_the_reference_does(engine):
    """Without setBuffers the c0 filter (96% pass) gets no refill; with the
    selection's id the generated kernel refills after it, as the reference's
    LaneRefill does (ref_c0_lr pins its results)."""
    from dogqc_b200.backend import Backend
    db = W.GENERATORS["c0"](SCALE)
    engine.register_database(db)
    srcs = []
    for positions in (None, "selection"):
        alg = RelationalAlgebra(db)
        plan, cfg = W.build("c0", alg)
        plan = alg.resolveAlgebraPlan(plan, cfg)
        b = Backend(alg, engine=engine)
        if positions:
            b.setBuffers([alg.selectionNodes[0].opId])
        b.gencode(alg.translateToCompilerPlan(plan, b))
        b.compile("c0")
        srcs.append(b.plan.source(0))
    assert "refill buffer" not in srcs[0]
    assert "refill buffer" in srcs[1]


def test_refill_threshold_knob(engine):
    p = engine.prepare(resolved(engine, "c1"), tuning={"refill_threshold": 28})
    assert "while (wn >= 28" in p.source(1)
    p = engine.prepare(resolved(engine, "c1"))
    assert "while (wn >= 32" in p.source(1)


def test_tuning_cache_on_disk(tmp_path, monkeypatch):
    from dogqc_b200 import autotune
    monkeypatch.setenv("DOGQC_B200_TUNING_CACHE", str(tmp_path / "t.json"))
    monkeypatch.setattr(autotune, "_cache", {})
    got = autotune._tuned("plan|x", None, lambda: ({"rows_per_thread": 2, "refill_threshold": 28}, 0.5, [1, 2]))
    assert got[0]["refill_threshold"] == 28
    monkeypatch.setattr(autotune, "_cache", {})

    def again():
        raise AssertionError("searched although the file holds the result")
    got = autotune._tuned("plan|x", None, again)
    assert got[0] == {"rows_per_thread": 2, "refill_threshold": 28} and got[1] == 0.5


def test_replayed_runs_overlap_independent_pipelines(engine):
    """A replayed run waits only where pipelines share a table.  C3: the three
    dimension builds share none and may run side by side; the fact pipeline
    waits for all three, the result scan for the fact pipeline.  Q13 (C17):
    the staged build side, then the multimap's count and scatter passes over
    it, the probe after both passes, its aggregation's scan, and a fused
    result scan (it runs in its predecessor's kernel) with none."""
    plan = engine.prepare(resolved(engine, "c3"))
    assert [plan.dependencies(i) for i in range(5)] == [[], [], [], [0, 1, 2], [3]]
    plan = engine.prepare(resolved(engine, "c17"))
    assert [plan.dependencies(i) for i in range(6)] == [[], [0], [0, 1], [1, 2], [3], []]
    plan = engine.prepare(resolved(engine, "c1"))
    assert [plan.dependencies(i) for i in range(3)] == [[], [0], []]
    with pytest.raises(L.DqError):
        plan.dependencies(3)


@pytest.mark.parametrize("pattern,search", [("%#1%", True), ("%ABC%xyz%", True), ("%a%b%c%d%e%f%g%h%i%", True),
                                            ("%", False), ("%%", False), ("%a%%b%", False), ("A%", False),
                                            ("%#59", False), ("%AB_D%", False), ("abc", False)])
def test_like_patterns_of_percent_separated_literals_compile_to_searches(engine, pattern, search):
    """'%L1%...%Ln%' (no '_', no empty literal) becomes one literal search
    after another (like_find); every other pattern runs the reference
    matcher's algorithm (like_match)."""
    import string_cases
    import dogqc_b200.scalar as scal
    from dogqc_b200.types import Type
    db = string_cases.long_db(200)
    engine.register_database(db, force=True)
    alg = RelationalAlgebra(db)
    sel = alg.selection(scal.LikeExpr(scal.AttrExpr("fk"), scal.ConstExpr(pattern, Type.STRING)), alg.scan("f"))
    plan = engine.prepare(alg.resolveAlgebraPlan(alg.projection(["fv", "fk"], sel), {}))
    src = plan.source(0)
    body = src[src.index("dq_main"):]
    assert ("like_find(" in body) == search
    assert ("like_match(" in body) == (not search)
