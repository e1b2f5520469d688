"""Batched form on the GPU: every instance of a batch gives the oracle's result
and the same result as the instance run alone."""
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


def _instances(shape, n, lo, hi):
    from dogqc_b200 import batch
    return [batch.Instance(shape, i, rows) for i, rows in enumerate(batch.instance_sizes(n, lo, hi))]


def _check(engine, insts, tuning=None):
    from dogqc_b200 import batch
    batch.register(engine, insts)
    b = batch.prepare_batch(engine, insts, tuning)
    try:
        for _ in range(2):  # a repeated execute must reset every instance's tables
            got = b.execute()
            for inst, res in zip(insts, got):
                want = canonical_rows(run_plan(inst.base_db, inst.plan)[1])
                assert canonical_rows(res.rows()) == want, (inst.shape, inst.index, inst.rows)
        t = b.timing()
        assert t["total_ms"] > 0 and t["kernel_launches"] >= 3
    finally:
        b.free()


@pytest.mark.parametrize("shape,n,lo,hi", [("c2", 12, 1 << 10, 1 << 14), ("c1", 6, 1 << 10, 1 << 15),
                                            ("c0", 5, 1 << 10, 1 << 15), ("c3", 3, 1 << 12, 1 << 15)])
def test_batch_matches_oracle(engine, shape, n, lo, hi):
    _check(engine, _instances(shape, n, lo, hi))


@pytest.mark.parametrize("shape,n,lo,hi", [("c9", 5, 1 << 10, 1 << 15), ("c14", 4, 1 << 12, 1 << 15),
                                            ("c16", 4, 1 << 11, 1 << 15)])
def test_batch_with_strings_matches_oracle(engine, shape, n, lo, hi):
    """String group keys and result columns (c9), string predicates, string
    keys of an aggregation over an aggregation (c14) and substrings (c16):
    each instance's references resolve against its own tables."""
    _check(engine, _instances(shape, n, lo, hi))


@pytest.mark.parametrize("tuning", [{"rows_per_thread": 1}, {"rows_per_thread": 4, "block_threads": 128},
                                    {"block_threads": 512, "refill": -1}, {"multi_buckets_pct": 50},
                                    {"unique_slots_pct": 400}])
def test_batch_tunings(engine, tuning):
    _check(engine, _instances("c2", 6, 1 << 10, 1 << 13) + [], tuning)
    _check(engine, _instances("c1", 4, 1 << 10, 1 << 13), tuning)


def test_batch_regrows_small_tables(engine):
    """Join tables a quarter of the plan's estimate overflow; the batch grows
    them, rebuilds its graph and runs again."""
    _check(engine, _instances("c1", 4, 1 << 12, 1 << 14), {"unique_slots_pct": 25})


def test_batch_equals_one_by_one(engine):
    from dogqc_b200 import batch
    insts = _instances("c2", 8, 1 << 10, 1 << 14)
    batch.register(engine, insts)
    b = batch.prepare_batch(engine, insts)
    plans = batch.prepare_one_by_one(engine, insts)
    try:
        got = b.execute()
        for p, res in zip(plans, got):
            assert canonical_rows(p.execute().rows()) == canonical_rows(res.rows())
    finally:
        b.free()
        for p in plans:
            p.free()


def test_tuned_plan_matches(engine):
    from dogqc_b200 import batch
    inst = _instances("c1", 1, 1 << 14, 1 << 14)[0]
    batch.register(engine, [inst])
    want = canonical_rows(run_plan(inst.base_db, inst.plan)[1])
    for tuning in ({"rows_per_thread": 1}, {"rows_per_thread": 2, "refill": -1}, {"unique_slots_pct": 400}):
        p = engine.prepare(inst.lowering, tuning=tuning)
        try:
            assert canonical_rows(p.execute().rows()) == want
        finally:
            p.free()
