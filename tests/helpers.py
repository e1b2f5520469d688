"""Shared test helpers: golden fixtures and plan construction."""
import json
import os

from dogqc_b200 import workloads
from dogqc_b200.relational import RelationalAlgebra

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def golden(case):
    with open(os.path.join(GOLDEN, "ref_%s.json" % case)) as f:
        return json.load(f)


def golden_cases():
    return sorted(f[4:-5] for f in os.listdir(GOLDEN) if f.startswith("ref_") and f.endswith(".json"))


def make_case(spec):
    """Database and resolved plan (this package's front end) for a golden case spec."""
    db = workloads.GENERATORS[spec["workload"]](spec["scale"], **spec.get("gen_kw", {}))
    alg = RelationalAlgebra(db)
    plan, cfg = workloads.build(spec["workload"], alg, **spec.get("plan_kw", {}))
    plan = alg.resolveAlgebraPlan(plan, cfg)
    return db, alg, plan


def reference_rows(rows, spec):
    """Rows as a golden fixture holds them: sorted lists, and the string
    columns (``spec["str_cols"]``) as the reference's result file shows them,
    right-aligned in 10 characters and cut to 10 (oracle/mmdb.py)."""
    from mmdb import render_string
    sc = set(spec.get("str_cols", ()))
    return sorted([render_string(v) if j in sc else int(v) for j, v in enumerate(r)] for r in rows)



def result_checksum(rows, spec):
    """Checksum of result rows as the fixtures hold it: string columns as the
    reference's result file shows them."""
    from canonical import canonical_checksum
    if spec.get("str_cols"):
        return canonical_checksum(reference_rows(rows, spec))
    return canonical_checksum(rows)
