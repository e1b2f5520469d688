"""Cases on which the reference's own generated pipeline pins the oracle.

Test infrastructure (oracle side): nothing in the product imports this module.

Each case names a workload (``dogqc_b200.workloads``), a scale, plan-builder
keyword arguments and reference-compiler knobs.  ``ref_harness.py`` turns every
case into a reference-generated ``.cu`` compiled for sm_100a; ``ref_run.py`` runs
those binaries on a GPU host over tables generated from the same seeds, and
``tests/golden/make_golden.py`` converts their outputs into committed fixtures.
"""

CASES = {
    # small cases: full result sets are committed as fixtures
    "c0_s": dict(workload="c0", scale=0.001),
    "c1_s": dict(workload="c1", scale=0.001),
    "c2_s": dict(workload="c2", scale=0.0005, pushdown=False),
    "c2_s_pd": dict(workload="c2", scale=0.0005, pushdown=True),
    "c3_s": dict(workload="c3", scale=0.0002),
    "c0_lr": dict(workload="c0", scale=0.001, buffers="selection"),
    # edge cases
    "c0_empty": dict(workload="c0", scale=0.001, plan_kw=dict(cutoff=0)),
    "c1_nomatch": dict(workload="c1", scale=0.001, plan_kw=dict(segment=9)),
    "c2_nomatch": dict(workload="c2", scale=0.0005, gen_kw=dict(probe_lo=51)),
    # left outer join (customers without orders count 0), two aggregations
    "c5_s": dict(workload="c5", scale=0.01),
    "c5": dict(workload="c5", scale=1.0),
    # nested-loop join with a one-row aggregate (Q22 shape)
    "c7_s": dict(workload="c7", scale=0.01),
    "c7": dict(workload="c7", scale=1.0),
    # two plan roots: a temp table written by the first, scanned by the second
    "c8_s": dict(workload="c8", scale=0.01),
    "c9_s": dict(workload="c9", scale=0.002, str_cols=[0, 1], plan_kw={"groups_hint": 256}),
    "c9p_s": dict(workload="c9p", scale=0.002, str_cols=[1]),
    "c10_s": dict(workload="c10", scale=0.02, str_cols=[0]),
    "c10p_s": dict(workload="c10p", scale=0.02, str_cols=[0]),
    "c8": dict(workload="c8", scale=1.0),
    # semi and anti joins: EXISTS without a condition on the reference's filter
    # table (Q4 shape), EXISTS / NOT EXISTS with a condition on its multimatch
    # table and on its filter table (Q21 shape), NOT EXISTS alone (Q22's);
    # an empty build side rejects every probe row
    "c11_s": dict(workload="c11", scale=0.01),
    "c11": dict(workload="c11", scale=1.0),
    "c11_none": dict(workload="c11", scale=0.01, plan_kw=dict(late_slack=100)),
    "c12_s": dict(workload="c12", scale=0.01),
    "c12": dict(workload="c12", scale=1.0),
    "c13_s": dict(workload="c13", scale=0.05),
    "c13_mm": dict(workload="c13", scale=0.05, plan_kw=dict(multimatch=True)),
    "c13": dict(workload="c13", scale=1.0),
    # strings beyond the scan: Q16 (string predicates before / after the join,
    # string group keys of an aggregation over an aggregation), joins on string
    # keys (unique, multimatch, semi, anti, semi with a condition), Q22
    # (substrings in an IN list, as a map result and a group key)
    "c14_s": dict(workload="c14", scale=0.05, str_cols=[0, 1]),
    "c14_late_s": dict(workload="c14", scale=0.05, str_cols=[0, 1], plan_kw=dict(late_filter=True)),
    "c14": dict(workload="c14", scale=1.0, str_cols=[0, 1]),
    "c15_u_s": dict(workload="c15", scale=0.02, plan_kw=dict(variant="unique")),
    "c15_m_s": dict(workload="c15", scale=0.02, plan_kw=dict(variant="multi")),
    "c15_semi_s": dict(workload="c15", scale=0.02, str_cols=[0], plan_kw=dict(variant="semi")),
    "c15_anti_s": dict(workload="c15", scale=0.02, str_cols=[0], plan_kw=dict(variant="anti")),
    "c15_x_s": dict(workload="c15", scale=0.02, str_cols=[0], plan_kw=dict(variant="exists")),
    # the reference's filter table stores every repeat of a build key in a slot
    # of its own, so an insert walks all earlier repeats: kept small
    "c15_dup_s": dict(workload="c15", scale=0.005, plan_kw=dict(variant="dup")),
    "c15_m": dict(workload="c15", scale=1.0, plan_kw=dict(variant="multi")),
    "c16_s": dict(workload="c16", scale=0.05, str_cols=[0]),
    "c16": dict(workload="c16", scale=1.0, str_cols=[0]),
    # TPC-H Q13 (NOT LIKE on variable-length comments under an outer join),
    # Q20 (LIKE prefix, string equality on the nation, a two-attribute unique
    # table built from an aggregation, string results) and Q2 (LIKE suffix,
    # MIN joined back, eight result columns of which six are strings)
    "c17_s": dict(workload="c17", scale=0.01),
    "c17": dict(workload="c17", scale=1.0),
    "c18_s": dict(workload="c18", scale=0.05, str_cols=[0, 1]),
    "c18": dict(workload="c18", scale=1.0, str_cols=[0, 1]),
    "c19_s": dict(workload="c19", scale=0.05, str_cols=[1, 2, 4, 5, 6, 7]),
    "c19": dict(workload="c19", scale=1.0, str_cols=[1, 2, 4, 5, 6, 7]),
    # full sizes: row counts, checksums and (small) full results are committed
    "c0": dict(workload="c0", scale=1.0),
    "c1": dict(workload="c1", scale=1.0),
    "c2": dict(workload="c2", scale=1.0, pushdown=True),
    "c3": dict(workload="c3", scale=1.0),
}
