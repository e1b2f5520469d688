"""Served form on the GPU: results are the same alone and in a concurrent mix,
admission by memory, statistics."""
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


@pytest.fixture(scope="module")
def queries(engine):
    from dogqc_b200 import serve
    qs = serve.make_queries(sizes=(0.0005, 0.004))
    serve.register(engine, qs)
    return qs


def test_results_same_alone_and_in_mix(engine, queries):
    from dogqc_b200 import serve
    want = [canonical_rows(run_plan(q.base_db, q.plan)[1]) for q in queries]
    alone = []
    for q in queries:
        p = engine.prepare(q.lowering)
        try:
            alone.append(canonical_rows(p.execute().rows()))
        finally:
            p.free()
    assert alone == want
    srv = serve.Server(engine, slots=6)
    try:
        sched = serve.arrivals(48, None, queries, seed=7)   # all at once: maximal overlap
        results, infos, wall, errors = serve.mixed_stream(srv, queries, sched)
        assert not errors
        for (at, qi), res in zip(sched, results):
            assert canonical_rows(res.rows()) == want[qi]
        st = srv.stats()
        assert st["completed"] == 48 and st["failed"] == 0
        assert st["p99_ms"] >= st["p50_ms"] > 0
        assert all(i["total_ms"] >= i["queue_ms"] for i in infos)
    finally:
        srv.stop()


def test_poisson_arrivals(engine, queries):
    from dogqc_b200 import serve
    srv = serve.Server(engine, slots=4)
    try:
        sched = serve.arrivals(30, 2000.0, queries, seed=11)
        results, infos, wall, errors = serve.mixed_stream(srv, queries, sched)
        assert not errors and len(results) == 30
        assert srv.stats()["completed"] == 30
    finally:
        srv.stop()


def test_admission_rejects_oversized_request(engine, queries):
    from dogqc_b200 import _lib as L, serve
    srv = serve.Server(engine, slots=2, memory_budget=64 << 10)
    try:
        t = srv.submit(queries[-1].lowering)
        with pytest.raises(L.DqError) as ei:
            srv.wait(t)
        assert ei.value.status == L.ERR_ADMISSION
    finally:
        srv.stop()


def test_tight_budget_evicts_and_completes(engine, queries):
    """A budget that holds about one plan: requests wait for memory, idle plans
    are freed, every request still completes with the right result."""
    from dogqc_b200 import serve
    want = {i: canonical_rows(run_plan(q.base_db, q.plan)[1]) for i, q in enumerate(queries)}
    srv = serve.Server(engine, slots=4)
    try:  # the device bytes of every query's plan
        sched = [(0.0, i) for i in range(len(queries))]
        _, infos, _, errors = serve.mixed_stream(srv, queries, sched)
        assert not errors
        need = max(i["bytes"] for i in infos)
    finally:
        srv.stop()
    budget = need + need // 2
    srv = serve.Server(engine, slots=4, memory_budget=budget)
    try:
        sched = serve.arrivals(16, None, queries, seed=3)
        results, infos, wall, errors = serve.mixed_stream(srv, queries, sched)
        assert not errors
        for (at, qi), res in zip(sched, results):
            assert canonical_rows(res.rows()) == want[qi]
        assert srv.stats()["memory_peak"] <= budget
    finally:
        srv.stop()


@pytest.mark.parametrize("batch_max", [8, 1])
def test_continuous_batching_results(engine, queries, batch_max):
    """Requests of one shape waiting together run as one many-instance launch
    (batch_max > 1); every request's result still equals the oracle's."""
    from dogqc_b200 import serve
    want = [canonical_rows(run_plan(q.base_db, q.plan)[1]) for q in queries]
    srv = serve.Server(engine, slots=2, batch_max=batch_max)
    try:
        serve.warm(srv, queries, 2, rounds=1)          # every request shape prepared
        sched = serve.arrivals(96, None, queries, seed=13)
        results, infos, wall, errors = serve.mixed_stream(srv, queries, sched)
        assert not errors
        for (at, qi), res in zip(sched, results):
            assert canonical_rows(res.rows()) == want[qi]
        st = srv.stats()
        if batch_max > 1:
            assert st["batches"] > 0 and st["batched"] >= 2 * st["batches"]
        else:
            assert st["batches"] == 0
    finally:
        srv.stop()


def test_large_request_same_alone_and_in_mix(engine, queries):
    """A large request (the c3 shape at half its configuration: 30,000,000
    fact rows, ~500,000 groups) gives the same rows alone and while small
    requests run beside it, and the C++ evaluator of the plan agrees."""
    import cpu_eval
    from dogqc_b200 import serve
    from dogqc_b200.batch import Instance
    big = Instance("c3", 990, 30_000_000)
    engine.register_database(big.db)
    p = engine.prepare(big.lowering)
    try:
        alone = canonical_rows(p.execute().rows())
    finally:
        p.free()
    assert canonical_rows(cpu_eval.run_plan(big.base_db, big.plan)[1]) == alone
    small = {}
    for i, q in enumerate(queries):
        ps = engine.prepare(q.lowering)
        try:
            small[i] = canonical_rows(ps.execute().rows())
        finally:
            ps.free()
    qs = list(queries) + [big]
    sched = serve.arrivals(24, None, queries, seed=13)
    sched = sched[:8] + [(0.0, len(qs) - 1)] + sched[8:]
    srv = serve.Server(engine, slots=4)
    try:
        results, infos, wall, errors = serve.mixed_stream(srv, qs, sched)
        assert not errors
        for (at, qi), res in zip(sched, results):
            assert canonical_rows(res.rows()) == (alone if qi == len(qs) - 1 else small[qi])
    finally:
        srv.stop()


def test_unseen_shape_compiles_in_the_submitter(engine, queries):
    """A request of a shape the server has not seen compiles its kernels in
    the submitting thread (dq_server_submit), so the request loop serves the
    others meanwhile; its result is right."""
    from dogqc_b200 import serve
    from dogqc_b200 import workloads
    from dogqc_b200.database import Database, Table
    from dogqc_b200.lowering import Lowering
    from dogqc_b200.relational import RelationalAlgebra
    db = workloads.gen_c11(0.01)
    alg = RelationalAlgebra(db)
    plan, cfg = workloads.build("c11", alg)
    plan = alg.resolveAlgebraPlan(plan, cfg)
    low = Lowering(plan)
    for p in low.pipes:
        if p.table:
            p.table = p.table + "@unseen"
    engine.register_database(Database([Table(t.name + "@unseen", t.columns, t.types) for t in db.tables.values()]))
    srv = serve.Server(engine, slots=2)
    try:
        t = srv.submit(low)
        res, info = srv.wait(t)
        assert canonical_rows(res.rows()) == canonical_rows(run_plan(db, plan)[1])
    finally:
        srv.stop()


def test_string_requests_alone_and_batched(engine):
    """Requests with string group keys, predicates, substrings and string
    result columns, alone and as continuous batches: their results are the
    oracle's, strings gathered per request."""
    from dogqc_b200 import serve
    qs = serve.make_queries(shapes=("c9", "c14", "c16"), sizes=(0.0005, 0.002, 0.01))
    serve.register(engine, qs)
    want = [canonical_rows(run_plan(q.base_db, q.plan)[1]) for q in qs]
    for batch_max in (8, 1):
        srv = serve.Server(engine, slots=2, batch_max=batch_max)
        try:
            serve.warm(srv, qs, 2, rounds=1)
            sched = serve.arrivals(48, None, qs, seed=21)
            results, infos, wall, errors = serve.mixed_stream(srv, qs, sched)
            assert not errors
            for (at, qi), res in zip(sched, results):
                assert canonical_rows(res.rows()) == want[qi]
            if batch_max > 1:
                assert srv.stats()["batches"] > 0
        finally:
            srv.stop()
