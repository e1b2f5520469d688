"""Served form: a request loop over resident tables (dq_server_*), and the
mixed query stream it is measured on.

``Server`` wraps the C ABI's server: ``submit`` hands it a lowered plan (the IR
is copied), ``wait`` returns the result with the request's queue, run and total
times.  ``mixed_stream`` replays a Poisson arrival process of queries drawn
from the workload shapes c0-c3 at several table sizes (tables preloaded and
resident), ``one_at_a_time`` runs the same requests as plain plans, one after
the other, for comparison.
"""
import ctypes as C
import math
import threading
import time

import numpy as np

from dogqc_b200 import _lib as L
from dogqc_b200.batch import FULL_ROWS, Instance
from dogqc_b200.engine import _take_result


class Server(object):
    def __init__(self, engine, slots=4, memory_budget=0, pool_per_query=0, batch_max=0, batch_rows_max=0):
        """``batch_max``: requests of one shape run as one launch (0: 16, 1:
        every request alone); ``batch_rows_max``: requests scanning more input
        rows run alone (0: 2^18); ``pool_per_query`` 0: twice ``slots``."""
        self.engine = engine
        cfg = L.dq_server_config()
        cfg.slots = slots
        cfg.memory_budget = int(memory_budget)
        cfg.pool_per_query = pool_per_query
        cfg.batch_max = batch_max
        cfg.batch_rows_max = batch_rows_max
        h = C.c_void_p()
        L.check(L.lib().dq_server_start(engine.ctx, C.byref(cfg), C.byref(h)), engine.ctx)
        self.handle = h
        self._names = {}
        self._lock = threading.Lock()

    def submit(self, lowering):
        desc, keep = lowering.ir()
        t = C.c_uint64()
        L.check(L.lib().dq_server_submit(self.handle, C.byref(desc), C.byref(t)), self.engine.ctx)
        with self._lock:
            self._names[t.value] = lowering.result_names
        return t.value

    def wait(self, ticket):
        """(Result, info dict); raises DqError when the request failed."""
        res = C.c_void_p()
        info = L.dq_request_info()
        st = L.lib().dq_server_wait(self.handle, ticket, C.byref(res), C.byref(info))
        with self._lock:
            names = self._names.pop(ticket, [])
        d = {"queue_ms": info.queue_ms, "run_ms": info.run_ms, "total_ms": info.total_ms, "bytes": info.bytes,
             "status": info.status, "kernel_launches": info.kernel_launches}
        if st != L.OK:
            L.check(st, self.engine.ctx)
        return _take_result(res, names), d

    def stats(self):
        s = L.dq_server_stats()
        L.check(L.lib().dq_server_stats_get(self.handle, C.byref(s)))
        return {f: getattr(s, f) for f, _ in L.dq_server_stats._fields_}

    def stop(self):
        if self.handle:
            L.lib().dq_server_stop(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.stop()
        except Exception:
            pass


# ------------------------------------------------------------ mixed stream --

def make_queries(shapes=("c0", "c1", "c2", "c3"), sizes=(0.01, 0.1, 1.0), max_rows=None):
    """One query per (shape, size): the shape's plan over its own seeded tables
    at ``size`` x the configuration's rows (tables named ``<table>@<n>``)."""
    out = []
    for si, shape in enumerate(shapes):
        for zi, size in enumerate(sizes):
            rows = int(round(FULL_ROWS[shape] * size))
            if max_rows:
                rows = min(rows, max_rows)
            out.append(Instance(shape, 100 * si + zi, max(rows, 1024)))
    return out


def c4_sizes(per_shape=6, lo=0.01, hi=5.0, seed=20261203 + 4):
    """Table sizes of the served configuration, as fractions of the shapes'
    full configurations: per shape, `per_shape` - 1 sizes drawn log-uniform in
    [lo, hi] (seeded) and the largest size itself."""
    r = np.random.Generator(np.random.Philox(seed))
    out = {}
    for shape in ("c0", "c1", "c2", "c3"):
        draws = np.exp(r.uniform(math.log(lo), math.log(hi), per_shape - 1))
        out[shape] = sorted([float(x) for x in draws] + [hi])
    return out


def make_c4_queries(per_shape=6, lo=0.01, hi=5.0):
    """The served configuration's queries: each shape of c0-c3 at its
    `c4_sizes`, on its own seeded tables (the largest, 5x c3: 300,000,000 fact
    rows)."""
    out = []
    for si, (shape, sizes) in enumerate(sorted(c4_sizes(per_shape, lo, hi).items())):
        for zi, size in enumerate(sizes):
            out.append(Instance(shape, 100 * si + zi, max(int(round(FULL_ROWS[shape] * size)), 1024)))
    return out


def register(engine, queries):
    for q in queries:
        engine.register_database(q.db)


def arrivals(n, rate_qps, queries, seed=12345):
    """``n`` (time offset in s, query index) pairs: Poisson arrivals at
    ``rate_qps`` (None: all at once), queries drawn uniformly."""
    r = np.random.Generator(np.random.Philox(seed))
    if rate_qps:
        t = np.cumsum(r.exponential(1.0 / rate_qps, n))
    else:
        t = np.zeros(n)
    return list(zip(t.tolist(), r.integers(0, len(queries), n).tolist()))


def mixed_stream(server, queries, schedule):
    """Submits the schedule's requests at their arrival times from one thread
    and collects them on another; returns (results by request, infos, wall s)."""
    tickets = [None] * len(schedule)
    ready = threading.Semaphore(0)
    results, infos = [None] * len(schedule), [None] * len(schedule)
    errors = []

    def collect():
        for i in range(len(schedule)):
            ready.acquire()
            try:
                results[i], infos[i] = server.wait(tickets[i])
            except Exception as ex:  # recorded, the caller decides
                errors.append((i, str(ex)))

    th = threading.Thread(target=collect)
    th.start()
    t0 = time.perf_counter()
    for i, (at, qi) in enumerate(schedule):
        delay = t0 + at - time.perf_counter()
        if delay > 0:
            time.sleep(delay)
        tickets[i] = server.submit(queries[qi].lowering)
        ready.release()
    th.join()
    wall = time.perf_counter() - t0
    return results, infos, wall, errors


def replay(server, queries, schedule):
    """The schedule through the server from native code (dq_server_replay):
    no Python per request.  Returns (per-request info dicts, wall seconds)."""
    irs = [q.lowering.ir() for q in queries]
    arr = (L.dq_plan_desc * len(irs))(*[d for d, _ in irs])
    n = len(schedule)
    at = (C.c_double * max(n, 1))(*[1e3 * t for t, _ in schedule])
    qi = (C.c_int32 * max(n, 1))(*[q for _, q in schedule])
    infos = (L.dq_request_info * max(n, 1))()
    t0 = time.perf_counter()
    L.check(L.lib().dq_server_replay(server.handle, len(irs), arr, n, at, qi, infos), server.engine.ctx)
    wall = time.perf_counter() - t0
    out = [{"queue_ms": i.queue_ms, "run_ms": i.run_ms, "total_ms": i.total_ms, "bytes": i.bytes}
           for i in list(infos)[:n]]
    return out, wall


def warm(server, queries, slots, rounds=2):
    """Prepares what a served stream needs before it is timed: every query's
    plan pool (its first request prepares the whole pool and compiles the
    batch kernels of its shape), then bursts of all queries at once, so the
    slots' batch buffers have grown to the sizes the stream's batches take."""
    sched = [(0.0, qi) for qi in range(len(queries)) for _ in range(slots)]
    for _ in range(rounds):
        replay(server, queries, sched)
    burst = [(0.0, qi) for _ in range(16 * slots) for qi in range(len(queries))]
    for _ in range(rounds):
        replay(server, queries, burst)


def sequence(engine, queries, schedule, plans=None):
    """The schedule's requests as plain plans executed one after the other from
    native code (dq_plan_run_sequence).  Returns (per-request ms, wall s, plans)."""
    plans = plans or {}
    for _, qi in schedule:
        if qi not in plans:
            plans[qi] = engine.prepare(queries[qi].lowering)
    keys = sorted(plans)
    index = {k: i for i, k in enumerate(keys)}
    handles = (C.c_void_p * len(keys))(*[plans[k].handle.value for k in keys])
    n = len(schedule)
    order = (C.c_int32 * max(n, 1))(*[index[q] for _, q in schedule])
    ms = (C.c_double * max(n, 1))()
    t0 = time.perf_counter()
    L.check(L.lib().dq_plan_run_sequence(handles, len(keys), n, order, ms), engine.ctx)
    wall = time.perf_counter() - t0
    return list(ms)[:n], wall, plans


def one_at_a_time(engine, queries, schedule, plans=None):
    """The same requests as plain plans, executed one after the other (each
    plan prepared once); returns (results, per-request seconds, wall s)."""
    plans = plans or {}
    for _, qi in schedule:
        if qi not in plans:
            plans[qi] = engine.prepare(queries[qi].lowering)
    results, times = [], []
    t0 = time.perf_counter()
    for _, qi in schedule:
        s = time.perf_counter()
        results.append(plans[qi].execute())
        times.append(time.perf_counter() - s)
    return results, times, time.perf_counter() - t0, plans


def percentile(xs, q):
    xs = sorted(xs)
    if not xs:
        return float("nan")
    return xs[min(len(xs) - 1, int(math.floor(q * (len(xs) - 1) + 0.5)))]
