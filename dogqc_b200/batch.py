"""Batched form: many independent instances of one plan shape in one launch.

An instance is a workload shape (c0..c3, or the string shapes c9, c14, c16) at
its own size, on its own tables.
Its tables are registered under instance names (``<table>@<i>``) and its lowered
plan is rewritten to scan them, so every instance has the same pipelines and
ops and the C ABI's batch (dq_batch_*) runs them all through one generated
kernel per pipeline under one CUDA graph (dogqc_b200.engine.Batch).

The configuration this follows: the divergent-expansion workload (multimap
build + probe + filter chain + aggregate) as 256 independent instances whose
row counts are log-uniform between 2^10 and 2^20.
"""
import math

import numpy as np

from dogqc_b200 import workloads
from dogqc_b200.database import Database, Table
from dogqc_b200.lowering import Lowering
from dogqc_b200.relational import RelationalAlgebra

# rows of the largest table of each shape at scale 1 (instance sizes scale it);
# c9, c14 and c16 carry strings (group keys, predicates, substrings, results)
FULL_ROWS = {"c0": 6_000_000, "c1": 6_000_000, "c2": 16_777_216, "c3": 60_000_000, "c9": 6_000_000,
             "c14": 800_000, "c16": 1_500_000}
SEED = workloads.BASE_SEED + 7000


def instance_sizes(n, lo=1 << 10, hi=1 << 20, seed=SEED):
    """``n`` row counts log-uniform in [lo, hi] (seeded)."""
    r = np.random.Generator(np.random.Philox(seed))
    return [int(round(math.exp(x))) for x in r.uniform(math.log(lo), math.log(hi), n)]


class Instance(object):
    """One instance: its database (tables under instance names), its resolved
    plan (on the original names) and its lowering (scanning the instance names)."""

    def __init__(self, shape, index, rows, seed=None):
        self.shape = shape
        self.index = index
        self.rows = rows
        self.suffix = "@%d" % index
        scale = rows / float(FULL_ROWS[shape])
        base = workloads.GENERATORS[shape](scale, seed=seed if seed is not None else SEED + 1 + index)
        self.base_db = base
        alg = RelationalAlgebra(base)
        plan, cfg = workloads.build(shape, alg, scale=scale)
        self.plan = alg.resolveAlgebraPlan(plan, cfg)
        self.lowering = Lowering(self.plan)
        for p in self.lowering.pipes:
            if p.table:
                p.table = p.table + self.suffix
        self.db = Database([Table(t.name + self.suffix, t.columns, t.types) for t in base.tables.values()])

    @property
    def input_rows(self):
        return sum(t.size for t in self.base_db.tables.values())


def make_instances(shape="c2", n=256, lo=1 << 10, hi=1 << 20, seed=SEED):
    return [Instance(shape, i, rows) for i, rows in enumerate(instance_sizes(n, lo, hi, seed))]


def register(engine, instances):
    for inst in instances:
        engine.register_database(inst.db)


def prepare_batch(engine, instances, tuning=None):
    return engine.prepare_batch([inst.lowering for inst in instances], tuning)


def prepare_one_by_one(engine, instances, tuning=None):
    """The reference point of the batched form: every instance as its own plan."""
    return [engine.prepare(inst.lowering, tuning=tuning) for inst in instances]
