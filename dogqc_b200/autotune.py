"""Autotuner for launch shape, table sizing and divergence handling (dq_tuning).

The reference fixes these choices in its generator: grid 920-1024 CTAs of 128
threads (dogqc/kernel.py:10-11), hash tables at twice the estimated rows
(dogqc/hashJoins.py:43) and a lane-refill threshold of 28 of 32 lanes
(dogqc/cudaDivergenceBuffer.py:15, 216).  Here they are measured: a coordinate
search over the knobs below, each candidate prepared (its kernels generated and
compiled, its tables sized) and timed on the device with CUDA events, the
fastest kept.  Results are cached per plan shape, in the process and in a JSON
file (``DOGQC_B200_TUNING_CACHE``, default ``~/.cache/dogqc_b200/tuning.json``)
keyed by the plan shape, the device name and the library's ABI version, so a
later process starts from the tuned values.

Knobs (the dq_tuning fields):
  rows_per_thread    consecutive rows one thread loads and processes per step
  block_threads      threads per CTA of the generated kernels
  refill             -1 turns the plan's lane refill off
  refill_threshold   buffered rows that make a warp process them (the
                     reference's 28 of 32; 0: 32, full warps only)
  defer_threshold    expansion ranges longer than this are deferred and
                     grouped (the expansion granularity; 0: adaptive)
  unique_slots_pct   join-table slots as % of the plan's estimate (load factor;
                     0 is the backend's size-dependent default)
  multi_buckets_pct  multimap buckets as % of the plan's estimate
"""
import hashlib
import json
import os

import numpy as np

KNOBS = [
    ("rows_per_thread", [1, 2, 4]),
    ("block_threads", [128, 256, 512]),
    ("refill", [0, -1]),
    ("refill_threshold", [0, 28, 24, 16]),
    ("defer_threshold", [0, 8, 32, 128, 512]),
    ("unique_slots_pct", [0, 200, 400, 800]),
    ("multi_buckets_pct", [100, 50, 25, 200]),
    ("ctas_per_sm", [0, 3, 4, 2]),
]

_cache = {}


def cache_path():
    return os.environ.get("DOGQC_B200_TUNING_CACHE",
                          os.path.join(os.path.expanduser("~"), ".cache", "dogqc_b200", "tuning.json"))


def _disk_load():
    try:
        with open(cache_path()) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def _disk_store(key, tuning, seconds):
    """Adds one entry (atomic rename; a concurrent writer loses at worst its own entry)."""
    path = cache_path()
    data = _disk_load()
    data[key] = {"tuning": tuning, "seconds": seconds}
    try:
        os.makedirs(os.path.dirname(path), exist_ok=True)
        tmp = "%s.%d.tmp" % (path, os.getpid())
        with open(tmp, "w") as f:
            json.dump(data, f, indent=1, sort_keys=True)
        os.replace(tmp, path)
    except OSError:
        pass


def _device_tag(engine):
    try:
        import torch
        name = torch.cuda.get_device_name(getattr(engine, "device", 0))
    except Exception:
        name = "device"
    from dogqc_b200 import _lib
    return "%s|abi%d" % (name, _lib.ABI_VERSION)


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


def plan_measure(engine, lowering, reps=3, warmup=1, between=None):
    """Median device time of a plan prepared with the candidate tuning;
    ``between()`` runs before every execution (an L2 flush, so that inputs
    that would fit L2 are read from HBM as in a timed run)."""
    def measure(tuning):
        try:
            p = engine.prepare(lowering, tuning=tuning)
        except Exception:
            return None
        try:
            for _ in range(warmup):
                if between:
                    between()
                p.execute()
            ts = []
            for _ in range(reps):
                if between:
                    between()
                p.execute()
                ts.append(p.timing()["total_ms"])
            return float(np.median(ts)) / 1e3
        finally:
            p.free()
    return measure


def relevant_knobs(lowering, knobs=KNOBS):
    """The knobs that can change a plan's kernels: table sizing only with
    such tables, expansion deferral only with an expansion."""
    kinds = {r.kind for r in lowering.res}
    from dogqc_b200 import _lib as L
    ops = {o["kind"] for p in lowering.pipes for o in p.ops}
    out = []
    for knob, values in knobs:
        if knob == "unique_slots_pct" and L.RES_UNIQUE not in kinds:
            continue
        if knob == "multi_buckets_pct" and L.RES_MULTI not in kinds:
            continue
        if knob == "defer_threshold" and L.OP_EXPAND not in ops:
            continue
        out.append((knob, values))
    return out


def _tuned(key, engine, search):
    """(best tuning, its seconds, search log): from this process's cache, the
    file cache (no log: not searched here), or a new search that is stored."""
    if key in _cache:
        return _cache[key]
    disk_key = "%s|%s" % (key, _device_tag(engine))
    hit = _disk_load().get(disk_key)
    if hit is not None:
        _cache[key] = (hit["tuning"], hit["seconds"], [])
        return _cache[key]
    best, t, log = search()
    _cache[key] = (best, t, log)
    if t is not None:
        _disk_store(disk_key, best, t)
    return _cache[key]


def tune_batch(engine, lowerings, knobs=KNOBS, reps=3):
    key = "batch|%s|%d" % (shape_key(lowerings[0]), len(lowerings))
    return _tuned(key, engine, lambda: coordinate_search(batch_measure(engine, lowerings, reps), knobs))


def tune_plan(engine, lowering, knobs=None, reps=3, between=None):
    key = "plan|%s" % shape_key(lowering)
    knobs = relevant_knobs(lowering) if knobs is None else knobs
    return _tuned(key, engine, lambda: coordinate_search(plan_measure(engine, lowering, reps, between=between), knobs))
