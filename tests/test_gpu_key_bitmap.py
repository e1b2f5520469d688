"""Key-domain tables on the GPU against the CPU oracle.

A unique join table with one integer key, built straight from a column whose
values span few keys (measured on the device when the plan is prepared),
needs no hashing: without a payload it is a bit per key, probed in shared
memory up to 2^18 keys and in place above (C3 at scale 0.3: 300,000 keys of
the first dimension); with one payload of at most 32 bits and at most four
keys per build row it is a word per key, one load a probe.  Cases: the C3 star
join's three dimensions (inner joins whose build key, the one attribute read
above them, is read from the probe side), semi and anti filters (Q4 / Q22
shapes), the C1 dimension (the nation as payload), and a table whose keys move
out of the measured domain after preparation: the build reports it, and the
plan re-runs with a hash table and stays exact.
"""
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


def _bitmap_pipelines(p):
    return [i for i in range(len(p.lowering.pipes)) if ".bmin" in p.source(i)]


@pytest.mark.parametrize("workload,scale", [("c3", 0.05), ("c3", 0.3), ("c11", 0.05), ("c13", 0.05), ("c1", 0.05),
                                            ("c1", 1.0)])
def test_bitmap_probes_match_oracle(engine, workload, scale):
    db, alg, plan = make_case({"workload": workload, "scale": scale})
    engine.register_database(db, force=True)
    p = engine.prepare(plan)
    try:
        assert _bitmap_pipelines(p)
        want = canonical_rows(run_plan(db, plan)[1])
        assert canonical_rows(p.execute().rows()) == want
        assert canonical_rows(p.execute().rows()) == want   # replayed graph, bits cleared
    finally:
        p.free()


def test_keys_leaving_the_domain_fall_back_to_a_hash_table(engine):
    """Every order key moves up by 10^7 after preparation (on both sides, so
    the join's answer is unchanged): the bitmap's build meets keys outside its
    range, and the run is repeated with a hash table."""
    from dogqc_b200.database import Database, Table
    db, alg, plan = make_case({"workload": "c11", "scale": 0.02})
    engine.register_database(db, force=True)
    p = engine.prepare(plan)
    try:
        assert _bitmap_pipelines(p)
        want = canonical_rows(run_plan(db, plan)[1])
        assert canonical_rows(p.execute().rows()) == want
        moved = []
        for t in db.tables.values():
            cols = dict(t.columns)
            for name in cols:
                if name.endswith("orderkey"):
                    cols[name] = (np.asarray(cols[name]).astype(np.int64) + 10_000_000).astype(np.int32)
            moved.append(Table(t.name, cols, t.types))
        db2 = Database(moved)
        for t in moved:
            engine.update_table(t)
        assert canonical_rows(p.execute().rows()) == canonical_rows(run_plan(db2, plan)[1]) == want
        assert not _bitmap_pipelines(p)
    finally:
        p.free()
