"""Autotuner for launch shape and table sizing (dq_tuning).

The reference fixes these choices in its generator: grid 920-1024 CTAs of 128
threads (dogqc/kernel.py:10-11), hash tables at twice the estimated rows
(dogqc/hashJoins.py:43) and a lane-refill threshold of 28 of 32 lanes
(dogqc/cudaDivergenceBuffer.py:15).  Here they are measured: a coordinate
search over the knobs below, each candidate prepared (its kernels generated and
compiled, its tables sized) and timed on the device with CUDA events, the
fastest kept.  Results are cached per plan shape for the life of the process.

Knobs (the dq_tuning fields):
  rows_per_thread    consecutive rows one thread loads and processes per step
  block_threads      threads per CTA of the generated kernels
  refill             -1 turns the plan's lane refill off
  unique_slots_pct   join-table slots as % of the plan's estimate (load factor;
                     0 is the backend's size-dependent default)
  multi_buckets_pct  multimap buckets as % of the plan's estimate
"""
import hashlib

import numpy as np

KNOBS = [
    ("rows_per_thread", [1, 2, 4]),
    ("block_threads", [128, 256, 512]),
    ("refill", [0, -1]),
    ("unique_slots_pct", [0, 200, 400, 800]),
    ("multi_buckets_pct", [100, 50, 25, 200]),
]

_cache = {}


def shape_key(lowering):
    """A key for a plan's shape (its pipelines and ops; not its sizes or tables)."""
    h = hashlib.sha1()
    for p in lowering.pipes:
        h.update(repr((p.source_kind, p.cols, [dict((k, o[k]) for k in sorted(o) if k != "imm") for o in p.ops],
                       p.lists)).encode())
    return h.hexdigest()


def coordinate_search(measure, knobs=KNOBS, base=None):
    """Tries each knob's values in turn with the others at the best so far.
    ``measure(tuning_dict) -> seconds`` (None when the candidate failed).
    Returns (best tuning, its time, [(tuning, time), ...])."""
    best = dict(base or {})
    best_t = measure(best)
    log = [(dict(best), best_t)]
    for knob, values in knobs:
        for v in values:
            if best.get(knob, 0) == v:
                continue
            cand = dict(best)
            cand[knob] = v
            t = measure(cand)
            log.append((cand, t))
            if t is not None and (best_t is None or t < best_t):
                best, best_t = cand, t
    return best, best_t, log


def batch_measure(engine, lowerings, reps=3, warmup=1):
    """Median device time of a batch prepared with the candidate tuning."""
    def measure(tuning):
        try:
            b = engine.prepare_batch(lowerings, tuning)
        except Exception:
            return None
        try:
            for _ in range(warmup):
                b.execute()
            ts = []
            for _ in range(reps):
                b.execute()
                ts.append(b.timing()["total_ms"])
            return float(np.median(ts)) / 1e3
        finally:
            b.free()
    return measure


def plan_measure(engine, lowering, reps=3, warmup=1):
    """Median device time of a plan prepared with the candidate tuning."""
    def measure(tuning):
        try:
            p = engine.prepare(lowering, tuning=tuning)
        except Exception:
            return None
        try:
            for _ in range(warmup):
                p.execute()
            ts = []
            for _ in range(reps):
                p.execute()
                ts.append(p.timing()["total_ms"])
            return float(np.median(ts)) / 1e3
        finally:
            p.free()
    return measure


def tune_batch(engine, lowerings, knobs=KNOBS, reps=3):
    key = ("batch", shape_key(lowerings[0]), len(lowerings))
    if key not in _cache:
        _cache[key] = coordinate_search(batch_measure(engine, lowerings, reps), knobs)
    return _cache[key]


def tune_plan(engine, lowering, knobs=KNOBS, reps=3):
    key = ("plan", shape_key(lowering))
    if key not in _cache:
        _cache[key] = coordinate_search(plan_measure(engine, lowering, reps), knobs)
    return _cache[key]
