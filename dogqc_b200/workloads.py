"""Seeded synthetic workloads: tables, plans and plan configs.

Four pipeline shapes, sized at ``scale=1.0`` as follows:

* ``c0`` scan-filter-aggregate over one 6,000,000-row table (TPC-H Q1 shape):
  filter ``shipdate <= max-90``, group by two char flags (6 groups), exact
  64-bit sums of quantity, price, ``price*(100-disc)`` and
  ``price*(100-disc)*(100+tax)``, a count, and averages derived from them.
* ``c1`` FK-PK hash join + aggregate: a 1,500,000-row dimension (unique keys,
  a permutation of 1..1.5M) filtered on ``segment == 1`` (20%), probed by a
  6,000,000-row fact table, grouped by ``nation`` (25 groups).
* ``c2`` divergent expansion: a 10,000,000-row multimap build side with Zipf(1.0)
  keys over 100,000 values, probed by 16,777,216 uniform keys over 200,000
  values (about half miss), followed by 4 filters (90/50/10/1%) on build-side
  columns, then a count and a 64-bit sum.
* ``c3`` three-way star join: 60,000,000 fact rows against dimensions of
  1,500,000 / 200,000 / 10,000 rows with 50% / ~20% (``LIKE '%word%'``
  disjunction on a 25-byte string) / 100% filters, grouped by the 1.5M-key
  dimension.

TPC-H data is not available here; these seeded tables have TPC-H-like shapes,
value ranges and distributions.  Each generator is deterministic in its seed
(numpy ``Philox``), so the device engine, the CPU oracle and the reference's own
generated pipeline all see identical bytes.

Plan builders take the algebra object and the scalar/type/reduction namespaces
as arguments, so the same function builds the plan with this package's front end
or with the reference's (``oracle/ref_harness.py``).
"""
import math
from collections import namedtuple

import numpy as np

from dogqc_b200.database import Database, StringColumn, Table
from dogqc_b200.types import Type

BASE_SEED = 20261203
EPOCH_1992 = 8035          # 1992-01-01 as days since 1970-01-01
DATE_RANGE = 2557          # 1992-01-01 .. 1998-12-31

Workload = namedtuple("Workload", "name db build_plan description")


def _rng(seed):
    return np.random.Generator(np.random.Philox(seed))


def _n(base, scale, minimum=1):
    return max(minimum, int(round(base * scale)))


# ---------------------------------------------------------------- c0 ----------

def gen_c0(scale=1.0, seed=BASE_SEED + 0):
    n = _n(6_000_000, scale)
    r = _rng(seed)
    cols = {
        "l_quantity": r.integers(1, 51, n, dtype=np.int32),
        "l_extendedprice": r.integers(90_000, 10_500_001, n, dtype=np.int64).astype(np.uint64),
        "l_discount": r.integers(0, 11, n, dtype=np.int32),
        "l_tax": r.integers(0, 9, n, dtype=np.int32),
        "l_shipdate": (EPOCH_1992 + r.integers(0, DATE_RANGE, n)).astype(np.uint32),
        "l_returnflag": np.frombuffer(b"ANR", dtype=np.int8)[r.integers(0, 3, n)],
        "l_linestatus": np.frombuffer(b"FO", dtype=np.int8)[r.integers(0, 2, n)],
    }
    types = {"l_quantity": Type.INT, "l_extendedprice": Type.FLOAT, "l_discount": Type.INT,
             "l_tax": Type.INT, "l_shipdate": Type.DATE, "l_returnflag": Type.CHAR,
             "l_linestatus": Type.CHAR}
    return Database([Table("lineitem", cols, types)])


def plan_c0(alg, scal, Type, Reduction, cutoff=EPOCH_1992 + DATE_RANGE - 1 - 90):
    sel = alg.selection(
        scal.SmallerEqualExpr(scal.AttrExpr("l_shipdate"), scal.ConstExpr(str(cutoff), Type.DATE)),
        alg.scan("lineitem"))
    disc = alg.map("disc_price",
                   scal.MulExpr(scal.AttrExpr("l_extendedprice"),
                                scal.SubExpr(scal.ConstExpr("100", Type.INT), scal.AttrExpr("l_discount"))),
                   sel)
    charge = alg.map("charge",
                     scal.MulExpr(scal.AttrExpr("disc_price"),
                                  scal.AddExpr(scal.ConstExpr("100", Type.INT), scal.AttrExpr("l_tax"))),
                     disc)
    agg = alg.aggregation(
        ["l_returnflag", "l_linestatus"],
        [(Reduction.SUM, "l_quantity", "sum_qty"),
         (Reduction.SUM, "l_extendedprice", "sum_base_price"),
         (Reduction.SUM, "disc_price", "sum_disc_price"),
         (Reduction.SUM, "charge", "sum_charge"),
         (Reduction.AVG, "l_quantity", "avg_qty"),
         (Reduction.AVG, "l_extendedprice", "avg_price"),
         (Reduction.AVG, "l_discount", "avg_disc"),
         (Reduction.COUNT, "", "count_order")],
        charge)
    cfg = {sel.opId: {"selectivity": (cutoff - EPOCH_1992 + 1) / DATE_RANGE},
           agg.opId: {"numgroups": 6}}
    return agg, cfg


# ---------------------------------------------------------------- c1 ----------

def gen_c1(scale=1.0, seed=BASE_SEED + 1):
    nd = _n(1_500_000, scale)
    nf = _n(6_000_000, scale)
    r = _rng(seed)
    dim = {
        "d_key": (r.permutation(nd) + 1).astype(np.int32),
        "d_segment": r.integers(0, 5, nd, dtype=np.int32),
        "d_nation": r.integers(0, 25, nd, dtype=np.int32),
    }
    fact = {
        "f_fk": r.integers(1, nd + 1, nf, dtype=np.int32),
        "f_measure": r.integers(1_000, 10_000_001, nf, dtype=np.int64).astype(np.uint64),
    }
    return Database([
        Table("dim", dim, {"d_key": Type.INT, "d_segment": Type.INT, "d_nation": Type.INT}),
        Table("fact", fact, {"f_fk": Type.INT, "f_measure": Type.FLOAT}),
    ])


def plan_c1(alg, scal, Type, Reduction, segment=1):
    sel = alg.selection(scal.EqualsExpr(scal.AttrExpr("d_segment"), scal.ConstExpr(str(segment), Type.INT)),
                        alg.scan("dim"))
    join = alg.join(("d_key", "f_fk"), sel, alg.scan("fact"))
    agg = alg.aggregation(["d_nation"],
                          [(Reduction.SUM, "f_measure", "sum_measure"),
                           (Reduction.COUNT, "", "cnt")],
                          join)
    cfg = {sel.opId: {"selectivity": 0.2},
           join.opId: {"multimatch": False, "selectivity": 0.2},
           agg.opId: {"numgroups": 25}}
    return agg, cfg


# ---------------------------------------------------------------- c2 ----------

def zipf_keys(r, n, distinct, s=1.0):
    """``n`` keys in ``1..distinct`` with P(rank k) ~ 1/k^s and permuted labels.

    Follows the construction of the reference's join-data generator
    (query/datagen/zipfdist.c:295-355): a cumulative distribution over ranks,
    a uniform draw mapped through it, and a random permutation from ranks to key
    labels.
    """
    ranks = np.arange(1, distinct + 1, dtype=np.float64)
    p = 1.0 / np.power(ranks, s)
    cdf = np.cumsum(p)
    cdf /= cdf[-1]
    labels = (r.permutation(distinct) + 1).astype(np.int32)
    u = r.random(n)
    idx = np.searchsorted(cdf, u, side="left")
    np.minimum(idx, distinct - 1, out=idx)
    return labels[idx]


def gen_c2(scale=1.0, seed=BASE_SEED + 2, distinct=None, probe_range=None, probe_lo=1):
    nb = _n(10_000_000, scale)
    npr = _n(16_777_216, scale)
    distinct = distinct or _n(100_000, scale, 16)
    probe_range = probe_range or 2 * distinct
    r = _rng(seed)
    build = {"r_key": zipf_keys(r, nb, distinct)}
    for i in range(1, 5):
        build["r_f%d" % i] = r.integers(0, 100, nb, dtype=np.int32)
    build["r_measure"] = r.integers(1, 1_000_001, nb, dtype=np.int64).astype(np.uint64)
    probe = {"s_key": r.integers(probe_lo, probe_lo + probe_range, npr, dtype=np.int32)}
    btypes = {"r_key": Type.INT, "r_f1": Type.INT, "r_f2": Type.INT, "r_f3": Type.INT,
              "r_f4": Type.INT, "r_measure": Type.FLOAT}
    return Database([Table("r_build", build, btypes),
                     Table("s_probe", probe, {"s_key": Type.INT})])


C2_THRESHOLDS = (90, 50, 10, 1)


def plan_c2(alg, scal, Type, Reduction, thresholds=C2_THRESHOLDS):
    join = alg.join(("r_key", "s_key"), alg.scan("r_build"), alg.scan("s_probe"))
    node = join
    cfg = {join.opId: {"selectivity": 50.0}}
    for i, t in enumerate(thresholds, start=1):
        node = alg.selection(scal.SmallerExpr(scal.AttrExpr("r_f%d" % i), scal.ConstExpr(str(t), Type.INT)),
                             node)
        cfg[node.opId] = {"selectivity": t / 100.0}
    agg = alg.aggregation([], [(Reduction.COUNT, "", "cnt"),
                               (Reduction.SUM, "r_measure", "sum_measure")], node)
    return agg, cfg


# ---------------------------------------------------------------- c3 ----------

def vocabulary(seed=BASE_SEED + 3, size=90, length=4):
    """``size`` distinct lowercase words of ``length`` letters (seeded)."""
    r = _rng(seed + 1000)
    words = []
    seen = set()
    letters = np.frombuffer(b"abcdefghijklmnopqrstuvwxyz", dtype=np.uint8)
    while len(words) < size:
        w = bytes(letters[r.integers(0, 26, length)])
        if w not in seen:
            seen.add(w)
            words.append(w)
    return words


C3_WIDTH = 25


def gen_c3(scale=1.0, seed=BASE_SEED + 3):
    n1 = _n(1_500_000, scale)
    n2 = _n(200_000, scale)
    n3 = _n(10_000, scale)
    nf = _n(60_000_000, scale)
    r = _rng(seed)
    vocab = np.array([list(w) for w in vocabulary(seed)], dtype=np.uint8)   # 90 x 4
    d1 = {"d1_key": (r.permutation(n1) + 1).astype(np.int32),
          "d1_attr": r.integers(0, 100, n1, dtype=np.int32)}
    pick = r.integers(0, len(vocab), (n2, 5))
    text = np.full((n2, C3_WIDTH), ord(" "), dtype=np.uint8)
    for j in range(5):
        text[:, 5 * j:5 * j + 4] = vocab[pick[:, j]]
    d2 = {"d2_key": (r.permutation(n2) + 1).astype(np.int32),
          "d2_text": StringColumn.fixed(text)}
    d3 = {"d3_key": (r.permutation(n3) + 1).astype(np.int32),
          "d3_attr": r.integers(0, 100, n3, dtype=np.int32)}
    fact = {"f_fk1": r.integers(1, n1 + 1, nf, dtype=np.int32),
            "f_fk2": r.integers(1, n2 + 1, nf, dtype=np.int32),
            "f_fk3": r.integers(1, n3 + 1, nf, dtype=np.int32),
            "f_price": r.integers(90_000, 10_500_001, nf, dtype=np.int64).astype(np.uint64),
            "f_disc": r.integers(0, 11, nf, dtype=np.int32)}
    return Database([
        Table("dim1", d1, {"d1_key": Type.INT, "d1_attr": Type.INT}),
        Table("dim2", d2, {"d2_key": Type.INT, "d2_text": Type.STRING}),
        Table("dim3", d3, {"d3_key": Type.INT, "d3_attr": Type.INT}),
        Table("fact", fact, {"f_fk1": Type.INT, "f_fk2": Type.INT, "f_fk3": Type.INT,
                             "f_price": Type.FLOAT, "f_disc": Type.INT}),
    ])


def c3_patterns(seed=BASE_SEED + 3, nwords=4):
    """The LIKE patterns: ``nwords`` vocabulary words; 4 words give
    P(match) = 1 - (86/90)^5 ~= 20.3% for 5-word strings."""
    words = vocabulary(seed)
    return ["%" + w.decode() + "%" for w in words[:nwords]]


def plan_c3(alg, scal, Type, Reduction, patterns=None, d1_cut=50, d3_cut=100, numgroups=1_000_000):
    patterns = patterns or c3_patterns()
    s1 = alg.selection(scal.SmallerExpr(scal.AttrExpr("d1_attr"), scal.ConstExpr(str(d1_cut), Type.INT)),
                       alg.scan("dim1"))
    like = scal.LikeExpr(scal.AttrExpr("d2_text"), scal.ConstExpr(patterns[0], Type.STRING))
    for p in patterns[1:]:
        like = scal.OrExpr(like, scal.LikeExpr(scal.AttrExpr("d2_text"), scal.ConstExpr(p, Type.STRING)))
    s2 = alg.selection(like, alg.scan("dim2"))
    s3 = alg.selection(scal.SmallerExpr(scal.AttrExpr("d3_attr"), scal.ConstExpr(str(d3_cut), Type.INT)),
                       alg.scan("dim3"))
    j3 = alg.join(("d3_key", "f_fk3"), s3, alg.scan("fact"))
    j2 = alg.join(("d2_key", "f_fk2"), s2, j3)
    j1 = alg.join(("d1_key", "f_fk1"), s1, j2)
    m = alg.map("disc_price",
                scal.MulExpr(scal.AttrExpr("f_price"),
                             scal.SubExpr(scal.ConstExpr("100", Type.INT), scal.AttrExpr("f_disc"))),
                j1)
    agg = alg.aggregation(["d1_key"],
                          [(Reduction.SUM, "f_price", "sum_price"),
                           (Reduction.SUM, "disc_price", "sum_disc_price"),
                           (Reduction.COUNT, "", "cnt")],
                          m)
    sel_like = 1.0 - (1.0 - len(patterns) / 90.0) ** 5
    cfg = {s1.opId: {"selectivity": d1_cut / 100.0},
           s2.opId: {"selectivity": sel_like},
           s3.opId: {"selectivity": d3_cut / 100.0},
           j3.opId: {"multimatch": False, "selectivity": 1.0},
           j2.opId: {"multimatch": False, "selectivity": sel_like},
           # a join's selectivity scales its larger input: the rows reaching j1
           j1.opId: {"multimatch": False, "selectivity": d1_cut / 100.0},
           agg.opId: {"numgroups": numgroups}}
    return agg, cfg


# ---------------------------------------------------------------- c5 ----------

def gen_c5(scale=1.0, seed=BASE_SEED + 5):
    """Customers and their orders (TPC-H Q13 shape): customer keys a
    permutation of 1..n; every order belongs to a customer whose key is not a
    multiple of 3, so a third of the customers have no orders."""
    nc = _n(150_000, scale, 16)
    no = _n(1_500_000, scale, 16)
    r = _rng(seed)
    cust = {"c_custkey": (r.permutation(nc) + 1).astype(np.int32),
            "c_nation": r.integers(0, 25, nc, dtype=np.int32)}
    with_orders = np.arange(1, nc + 1, dtype=np.int32)
    with_orders = with_orders[with_orders % 3 != 0]
    orders = {"o_orderkey": (r.permutation(no) + 1).astype(np.int32),
              "o_custkey": with_orders[r.integers(0, len(with_orders), no)],
              "o_flag": r.integers(0, 100, no, dtype=np.int32)}
    cust["c_acctbal"] = r.integers(0, 10_000, nc, dtype=np.int32)   # drawn last: earlier columns unchanged
    return Database([Table("customer", cust, {"c_custkey": Type.INT, "c_nation": Type.INT, "c_acctbal": Type.INT}),
                     Table("orders", orders, {"o_orderkey": Type.INT, "o_custkey": Type.INT, "o_flag": Type.INT})])


def plan_c5(alg, scal, Type, Reduction, flag_cut=2, numgroups=150_000):
    """Customers left outer join their (filtered) orders, the number of orders
    per customer (COUNT of a build attribute: null rows count 0), then the
    number of customers per order count (Q13's two aggregations)."""
    ords = alg.selection(scal.LargerEqualExpr(scal.AttrExpr("o_flag"), scal.ConstExpr(str(flag_cut), Type.INT)),
                         alg.scan("orders"))
    j = alg.outerjoin(("o_custkey", "c_custkey"), None, ords, alg.scan("customer"))
    per_cust = alg.aggregation(["c_custkey"], [(Reduction.COUNT, "o_orderkey", "c_count")], j)
    dist = alg.aggregation(["c_count"], [(Reduction.COUNT, "", "custdist")], per_cust)
    cfg = {ords.opId: {"selectivity": (100 - flag_cut) / 100.0},
           j.opId: {"multimatch": True},
           per_cust.opId: {"numgroups": numgroups},
           dist.opId: {"numgroups": 64}}
    return dist, cfg


def plan_c7(alg, scal, Type, Reduction):
    """Customers whose balance exceeds the average balance (TPC-H Q22 shape):
    the one-row average, nested-loop joined to every customer with the
    comparison as the join condition, then counts and sums per nation."""
    avg = alg.aggregation([], [(Reduction.AVG, "c_acctbal", "avg_bal")], alg.scan("customer"))
    cj = alg.crossjoin(scal.LargerExpr(scal.AttrExpr("c_acctbal"), scal.AttrExpr("avg_bal")), avg,
                       alg.scan("customer"))
    agg = alg.aggregation(["c_nation"], [(Reduction.COUNT, "", "numcust"), (Reduction.SUM, "c_acctbal", "totbal")],
                          cj)
    cfg = {cj.opId: {"selectivity": 0.5}, agg.opId: {"numgroups": 25}}
    return agg, cfg


def plan_c8(alg, scal, Type, Reduction, flag_cut=50, nation_cut=5):
    """Two plan roots over a temp table (TPC-H Q15 shape): the first
    materialises orders per customer (the filtered orders grouped by
    customer), the second scans it, joins the customers of some nations
    (unique keys) and counts customers per order count."""
    ords = alg.selection(scal.SmallerExpr(scal.AttrExpr("o_flag"), scal.ConstExpr(str(flag_cut), Type.INT)),
                         alg.scan("orders"))
    per = alg.aggregation(["o_custkey"], [(Reduction.COUNT, "", "n_orders")], ords)
    tmp = alg.createtemp("cust_orders", per)
    cust = alg.selection(scal.SmallerExpr(scal.AttrExpr("c_nation"), scal.ConstExpr(str(nation_cut), Type.INT)),
                         alg.scan("customer"))
    j = alg.join(("o_custkey", "c_custkey"), alg.scan("cust_orders"), cust)
    dist = alg.aggregation(["n_orders"], [(Reduction.COUNT, "", "customers")], j)
    cfg = {ords.opId: {"selectivity": flag_cut / 100.0},
           per.opId: {"numgroups": 100_000},
           cust.opId: {"selectivity": nation_cut / 25.0},
           j.opId: {"multimatch": False},
           dist.opId: {"numgroups": 64}}
    return [tmp, dist], cfg


C9_MODES = [b"REG AIR", b"AIR", b"RAIL", b"SHIP", b"TRUCK", b"MAIL", b"FOB"]
C9_INSTRUCT = [b"DELIVER IN PERSON", b"COLLECT COD", b"NONE", b"TAKE BACK RETURN"]


def gen_c9(scale=1.0, seed=BASE_SEED + 9):
    """Q12-shaped: lineitem with variable-length string attributes (ship mode,
    ship instruction), a key, a measure and a receipt date."""
    n = _n(6_000_000, scale)
    r = _rng(seed)
    mode = r.integers(0, len(C9_MODES), n)
    instr = r.integers(0, len(C9_INSTRUCT), n)
    cols = {
        "l_orderkey": r.integers(1, 6_000_000, n, dtype=np.int32),
        "l_extendedprice": r.integers(90_000, 10_500_001, n, dtype=np.int64).astype(np.uint64),
        "l_receiptdate": (EPOCH_1992 + r.integers(0, DATE_RANGE, n)).astype(np.uint32),
        "l_shipmode": StringColumn.from_list([C9_MODES[i] for i in mode]),
        "l_shipinstruct": StringColumn.from_list([C9_INSTRUCT[i] for i in instr]),
    }
    types = {"l_orderkey": Type.INT, "l_extendedprice": Type.FLOAT, "l_receiptdate": Type.DATE,
             "l_shipmode": Type.STRING, "l_shipinstruct": Type.STRING}
    return Database([Table("lineitem", cols, types)])


def plan_c9(alg, scal, Type, Reduction, cutoff=EPOCH_1992 + DATE_RANGE // 2, groups_hint=None):
    """Rows received before the cutoff, per (ship mode, ship instruction):
    count and revenue -- grouping by two strings, both in the result."""
    sel = alg.selection(
        scal.SmallerExpr(scal.AttrExpr("l_receiptdate"), scal.ConstExpr(str(cutoff), Type.DATE)),
        alg.scan("lineitem"))
    agg = alg.aggregation(
        ["l_shipmode", "l_shipinstruct"],
        [(Reduction.COUNT, "", "line_count"), (Reduction.SUM, "l_extendedprice", "revenue")],
        sel)
    cfg = {sel.opId: {"selectivity": 0.5},
           agg.opId: {"numgroups": groups_hint or len(C9_MODES) * len(C9_INSTRUCT)}}
    return agg, cfg


def plan_c9p(alg, scal, Type, Reduction, key_cut=20_000):
    """A projection carrying strings: the rows with a small order key, their
    key and ship mode."""
    sel = alg.selection(
        scal.SmallerExpr(scal.AttrExpr("l_orderkey"), scal.ConstExpr(str(key_cut), Type.INT)),
        alg.scan("lineitem"))
    proj = alg.projection(["l_orderkey", "l_shipmode"], sel)
    return proj, {sel.opId: {"selectivity": key_cut / 6_000_000}}


C10_SEGMENTS = [b"AUTOMOBILE", b"BUILDING", b"FURNITURE", b"HOUSEHOLD", b"MACHINERY"]


def gen_c10(scale=1.0, seed=BASE_SEED + 10):
    """Q10-shaped: customers with a name and a market segment (strings) and
    their orders."""
    nc = _n(150_000, scale)
    no = _n(1_500_000, scale)
    r = _rng(seed)
    seg = r.integers(0, len(C10_SEGMENTS), nc)
    cust = {"c_custkey": (r.permutation(nc) + 1).astype(np.int32),
            "c_name": StringColumn.from_list([b"Customer#%09d" % (i + 1) for i in range(nc)]),
            "c_mktsegment": StringColumn.from_list([C10_SEGMENTS[i] for i in seg])}
    orders = {"o_custkey": r.integers(1, nc + 1, no, dtype=np.int32),
              "o_totalprice": r.integers(90_000, 50_000_000, no, dtype=np.int64).astype(np.uint64)}
    return Database([
        Table("customer", cust, {"c_custkey": Type.INT, "c_name": Type.STRING, "c_mktsegment": Type.STRING}),
        Table("orders", orders, {"o_custkey": Type.INT, "o_totalprice": Type.FLOAT})])


def plan_c10(alg, scal, Type, Reduction):
    """Orders joined to their customer (unique build), revenue and count per
    market segment: the group key is a string carried from the build side."""
    join = alg.join(("c_custkey", "o_custkey"), alg.scan("customer"), alg.scan("orders"))
    agg = alg.aggregation(["c_mktsegment"],
                          [(Reduction.SUM, "o_totalprice", "revenue"), (Reduction.COUNT, "", "cnt")], join)
    return agg, {join.opId: {"multimatch": False, "selectivity": 1.0},
                 agg.opId: {"numgroups": len(C10_SEGMENTS)}}


def plan_c10p(alg, scal, Type, Reduction, price_cut=200_000):
    """The customer name of every cheap order: a string result from the build side."""
    sel = alg.selection(scal.SmallerExpr(scal.AttrExpr("o_totalprice"), scal.ConstExpr(str(price_cut), Type.INT)),
                        alg.scan("orders"))
    join = alg.join(("c_custkey", "o_custkey"), alg.scan("customer"), sel)
    proj = alg.projection(["c_name", "o_totalprice"], join)
    return proj, {sel.opId: {"selectivity": 0.005}, join.opId: {"multimatch": False, "selectivity": 1.0}}


# ------------------------------------------------------- c11 .. c13 -------------
# Semi and anti joins: orders and their line items (TPC-H Q4 / Q21 shapes) and
# customers without orders (the NOT EXISTS of Q22).

def gen_c11(scale=1.0, seed=BASE_SEED + 11):
    """Orders (keys a permutation of 1..n, a date, a status flag, a priority)
    and line items (about four per order; orders whose key is a multiple of 7
    have none), with a supplier, a commit and a receipt date; a line is late
    (receipt after commit) about half the time."""
    no = _n(1_500_000, scale, 64)
    nl = _n(6_000_000, scale, 256)
    ns = _n(10_000, scale, 16)
    r = _rng(seed)
    okeys = (r.permutation(no) + 1).astype(np.int32)
    orders = {"o_orderkey": okeys,
              "o_orderdate": (EPOCH_1992 + r.integers(0, DATE_RANGE, no)).astype(np.int32),
              "o_orderstatus": np.frombuffer(b"FOP", dtype=np.int8)[r.integers(0, 3, no)],
              "o_orderpriority": r.integers(1, 6, no, dtype=np.int32)}
    with_lines = np.arange(1, no + 1, dtype=np.int32)
    with_lines = with_lines[with_lines % 7 != 0]
    commit = (EPOCH_1992 + r.integers(0, DATE_RANGE, nl)).astype(np.int32)
    lines = {"l_orderkey": with_lines[r.integers(0, len(with_lines), nl)],
             "l_suppkey": r.integers(1, ns + 1, nl, dtype=np.int32),
             "l_commitdate": commit,
             "l_receiptdate": (commit + r.integers(-30, 31, nl)).astype(np.int32)}
    return Database([Table("orders", orders, {"o_orderkey": Type.INT, "o_orderdate": Type.INT,
                                              "o_orderstatus": Type.CHAR, "o_orderpriority": Type.INT}),
                     Table("lineitem", lines, {"l_orderkey": Type.INT, "l_suppkey": Type.INT,
                                               "l_commitdate": Type.INT, "l_receiptdate": Type.INT})])


def plan_c11(alg, scal, Type, Reduction, start=EPOCH_1992 + 546, days=92, late_slack=0):
    """Q4 shape: orders of one quarter that have at least one late line item
    (EXISTS, a semi join on the order key with no further condition, on a
    unique filter table), counted per priority.  ``late_slack`` > 60 leaves no
    late line: the semi join then rejects every order."""
    late = alg.selection(scal.SmallerExpr(scal.AddExpr(scal.AttrExpr("l_commitdate"),
                                                       scal.ConstExpr(str(late_slack), Type.INT)),
                                          scal.AttrExpr("l_receiptdate")),
                         alg.scan("lineitem"))
    ords = alg.selection(scal.AndExpr(scal.LargerEqualExpr(scal.AttrExpr("o_orderdate"),
                                                           scal.ConstExpr(str(start), Type.INT)),
                                      scal.SmallerExpr(scal.AttrExpr("o_orderdate"),
                                                       scal.ConstExpr(str(start + days), Type.INT))),
                         alg.scan("orders"))
    sj = alg.semijoin(("l_orderkey", "o_orderkey"), None, late, ords)
    agg = alg.aggregation(["o_orderpriority"], [(Reduction.COUNT, "", "order_count")], sj)
    cfg = {late.opId: {"selectivity": 0.5},
           ords.opId: {"selectivity": days / float(DATE_RANGE)},
           sj.opId: {"multimatch": False, "htSizeFactor": 0.5},
           agg.opId: {"numgroups": 100}}
    return agg, cfg


def plan_c12(alg, scal, Type, Reduction, multimatch=True):
    """Q21 shape: late line items (l1) of orders with status 'F' for which
    another supplier has a line of the same order (EXISTS l2 with
    l2.suppkey <> l1.suppkey, a semi join with a condition) and no other
    supplier's line of the order is late (NOT EXISTS l3 ..., an anti join
    with a condition); waiting lines counted per supplier.  The conditions
    compare a build-side and a probe-side attribute for every key match."""
    l1 = alg.selection(scal.LargerExpr(scal.AttrExpr("l1.l_receiptdate"), scal.AttrExpr("l1.l_commitdate")),
                       alg.scan("lineitem", "l1"))
    ords = alg.selection(scal.EqualsExpr(scal.AttrExpr("o_orderstatus"), scal.ConstExpr("F", Type.CHAR)),
                         alg.scan("orders"))
    j = alg.join(("o_orderkey", "l1.l_orderkey"), ords, l1)
    l3 = alg.selection(scal.LargerExpr(scal.AttrExpr("l3.l_receiptdate"), scal.AttrExpr("l3.l_commitdate")),
                       alg.scan("lineitem", "l3"))
    aj = alg.antijoin(("l3.l_orderkey", "l1.l_orderkey"),
                      scal.NotExpr(scal.EqualsExpr(scal.AttrExpr("l3.l_suppkey"), scal.AttrExpr("l1.l_suppkey"))),
                      l3, j)
    sj = alg.semijoin(("l2.l_orderkey", "l1.l_orderkey"),
                      scal.NotExpr(scal.EqualsExpr(scal.AttrExpr("l2.l_suppkey"), scal.AttrExpr("l1.l_suppkey"))),
                      alg.scan("lineitem", "l2"), aj)
    agg = alg.aggregation(["l1.l_suppkey"], [(Reduction.COUNT, "", "numwait")], sj)
    cfg = {l1.opId: {"selectivity": 0.5},
           ords.opId: {"selectivity": 0.33},
           j.opId: {"multimatch": False, "selectivity": 0.33},
           l3.opId: {"selectivity": 0.5},
           aj.opId: {"multimatch": multimatch, "htSizeFactor": 1.0, "selectivity": 0.1},
           sj.opId: {"multimatch": multimatch, "htSizeFactor": 0.5, "selectivity": 0.1},
           agg.opId: {"numgroups": 20_000}}
    return agg, cfg


def plan_c13(alg, scal, Type, Reduction, multimatch=False, flag_cut=0):
    """NOT EXISTS without a further condition (the anti join of TPC-H Q22):
    customers with no order whose flag is at least ``flag_cut``, counted and
    their balances summed per nation."""
    ords = alg.selection(scal.LargerEqualExpr(scal.AttrExpr("o_flag"), scal.ConstExpr(str(flag_cut), Type.INT)),
                         alg.scan("orders"))
    aj = alg.antijoin(("o_custkey", "c_custkey"), None, ords, alg.scan("customer"))
    agg = alg.aggregation(["c_nation"], [(Reduction.COUNT, "", "numcust"), (Reduction.SUM, "c_acctbal", "totacctbal")],
                          aj)
    cfg = {ords.opId: {"selectivity": (100 - flag_cut) / 100.0},
           aj.opId: {"multimatch": multimatch, "selectivity": 0.33},
           agg.opId: {"numgroups": 25}}
    return agg, cfg


# ------------------------------------------------------- c14 .. c16 -------------
# Strings beyond the scan: predicates on strings carried through a join and
# group keys of strings from aggregation tables (TPC-H Q16 shape), joins on
# string keys (unique, multimatch, semi and anti), and substrings as map
# results, IN lists and group keys (TPC-H Q22 shape).

C14_TYPE1 = [b"STANDARD", b"SMALL", b"MEDIUM", b"LARGE", b"ECONOMY", b"PROMO"]
C14_TYPE2 = [b"ANODIZED", b"BURNISHED", b"PLATED", b"POLISHED", b"BRUSHED"]
C14_TYPE3 = [b"TIN", b"NICKEL", b"BRASS", b"STEEL", b"COPPER"]
C14_WORDS = [b"carefully", b"final", b"deposits", b"sleep", b"furiously", b"regular", b"accounts", b"haggle",
             b"quickly", b"ironic", b"packages", b"among", b"the", b"blithely", b"pending", b"requests", b"wake",
             b"slyly", b"express", b"theodolites", b"above", b"bold", b"foxes", b"instructions", b"nag"]
C14_SIZES = [49, 14, 23, 45, 19, 3, 36, 9]


def _comments(r, n, plant=None, plant_rate=0.0):
    """n variable-length comments of 3..12 words; with ``plant`` (a pair of
    words) about ``plant_rate`` of them hold the first word, later the second."""
    nw = r.integers(3, 13, n)
    words = r.integers(0, len(C14_WORDS), int(nw.sum()))
    planted = r.random(n) < plant_rate if plant else np.zeros(n, bool)
    out, k = [], 0
    for i in range(n):
        w = [C14_WORDS[j] for j in words[k:k + nw[i]]]
        k += nw[i]
        if planted[i]:
            w.insert(1, plant[0])
            w.insert(len(w), plant[1])
        out.append(b" ".join(w))
    return StringColumn.from_list(out)


def gen_c14(scale=1.0, seed=BASE_SEED + 14):
    """Q16-shaped: parts with a brand ("Brand#MN"), a three-word type and a
    size, four supplier rows per part, and suppliers with comments (1% of them
    hold "Customer ... Complaints")."""
    np_ = _n(200_000, scale, 64)
    ns = _n(10_000, scale, 16)
    r = _rng(seed)
    pk = (r.permutation(np_) + 1).astype(np.int32)
    brand = r.integers(1, 6, (np_, 2))
    t = r.integers(0, [len(C14_TYPE1), len(C14_TYPE2), len(C14_TYPE3)], (np_, 3))
    part = {"p_partkey": pk,
            "p_brand": StringColumn.from_list([b"Brand#%d%d" % (a, b) for a, b in brand]),
            "p_type": StringColumn.from_list([b" ".join((C14_TYPE1[a], C14_TYPE2[b], C14_TYPE3[c])) for a, b, c in t]),
            "p_size": r.integers(1, 51, np_, dtype=np.int32)}
    base = np.repeat(np.arange(1, np_ + 1, dtype=np.int64), 4)
    i = np.tile(np.arange(4, dtype=np.int64), np_)
    partsupp = {"ps_partkey": base.astype(np.int32),
                "ps_suppkey": ((base + i * (ns // 4 + (base - 1) // ns)) % ns + 1).astype(np.int32)}
    supplier = {"s_suppkey": (r.permutation(ns) + 1).astype(np.int32),
                "s_comment": _comments(r, ns, (b"Customer", b"Complaints"), 0.01)}
    return Database([
        Table("part", part, {"p_partkey": Type.INT, "p_brand": Type.STRING, "p_type": Type.STRING, "p_size": Type.INT}),
        Table("partsupp", partsupp, {"ps_partkey": Type.INT, "ps_suppkey": Type.INT}),
        Table("supplier", supplier, {"s_suppkey": Type.INT, "s_comment": Type.STRING})])


def plan_c14(alg, scal, Type, Reduction, late_filter=False):
    """TPC-H Q16: the parts not of one brand, not of a type prefix and of eight
    sizes, joined to their supplier rows, without the suppliers with complaints
    (an anti join), counted per supplier and then per (brand, type, size).
    With ``late_filter`` the brand and type predicates run above the join, on
    the strings the join carries from its build side."""
    brand_ok = scal.NotExpr(scal.EqualsExpr(scal.AttrExpr("p_brand"), scal.ConstExpr("Brand#45", Type.STRING)))
    type_ok = scal.NotExpr(scal.LikeExpr(scal.AttrExpr("p_type"), scal.ConstExpr("MEDIUM POLISHED%", Type.STRING)))
    sizes = scal.InExpr(scal.AttrExpr("p_size"), [scal.ConstExpr(str(v), Type.INT) for v in C14_SIZES])
    complaints = alg.selection(
        scal.LikeExpr(scal.AttrExpr("s_comment"), scal.ConstExpr("%Customer%Complaints%", Type.STRING)),
        alg.scan("supplier"))
    if late_filter:
        parts = alg.selection(sizes, alg.scan("part"))
        join = alg.join(("p_partkey", "ps_partkey"), parts, alg.scan("partsupp"))
        late = alg.selection(scal.AndExpr(brand_ok, type_ok), join)
        top = late
    else:
        parts = alg.selection(scal.AndExpr(scal.AndExpr(brand_ok, type_ok), sizes), alg.scan("part"))
        join = alg.join(("p_partkey", "ps_partkey"), parts, alg.scan("partsupp"))
        late = None
        top = join
    anti = alg.antijoin(("ps_suppkey", "s_suppkey"), None, complaints, top)
    per_supp = alg.aggregation(["p_brand", "p_type", "p_size", "ps_suppkey"],
                               [(Reduction.COUNT, "", "supp_count_resolvedistinct")], anti)
    agg = alg.aggregation(["p_brand", "p_type", "p_size"], [(Reduction.COUNT, "", "supp_count")], per_supp)
    proj = alg.projection(["p_brand", "p_type", "p_size", "supp_count"], agg)
    cfg = {parts.opId: {"selectivity": 0.15}, complaints.opId: {"selectivity": 0.01},
           join.opId: {"multimatch": False},
           per_supp.opId: {"numgroups": 120_000}, agg.opId: {"numgroups": 20_000}}
    if late is not None:
        cfg[late.opId] = {"selectivity": 0.8}
    return proj, cfg


C15_NATIONS = [b"ALGERIA", b"ARGENTINA", b"BRAZIL", b"CANADA", b"EGYPT", b"ETHIOPIA", b"FRANCE", b"GERMANY",
               b"INDIA", b"INDONESIA", b"IRAN", b"IRAQ", b"JAPAN", b"JORDAN", b"KENYA", b"MOROCCO",
               b"MOZAMBIQUE", b"PERU", b"CHINA", b"ROMANIA", b"SAUDI ARABIA", b"VIETNAM", b"RUSSIA",
               b"UNITED KINGDOM", b"UNITED STATES"]
C15_MODES = [b"REG AIR", b"AIR", b"RAIL", b"SHIP", b"TRUCK", b"MAIL", b"FOB"]


def gen_c15(scale=1.0, seed=BASE_SEED + 15):
    """Joins on strings: nations keyed by name (25, with a region), suppliers
    naming their nation (1% name one that is not in the table), shipping modes
    with one to three carriers each (a string key with duplicates) and line
    items naming their mode (one mode of eight is not in the table)."""
    ns = _n(100_000, scale, 64)
    nl = _n(6_000_000, scale, 256)
    r = _rng(seed)
    nation = {"n_name": StringColumn.from_list(C15_NATIONS),
              "n_regionkey": (np.arange(len(C15_NATIONS)) % 5).astype(np.int32)}
    names = C15_NATIONS + [b"ATLANTIS"]
    pick = np.where(r.random(ns) < 0.01, len(C15_NATIONS), r.integers(0, len(C15_NATIONS), ns))
    supplier = {"s_suppkey": (r.permutation(ns) + 1).astype(np.int32),
                "s_nation": StringColumn.from_list([names[i] for i in pick]),
                "s_acctbal": r.integers(0, 1_000_000, ns, dtype=np.int32)}
    reps = r.integers(1, 4, len(C15_MODES))
    modes = {"m_mode": StringColumn.from_list([m for m, k in zip(C15_MODES, reps) for _ in range(k)]),
             "m_carrier": np.arange(int(reps.sum()), dtype=np.int32) + 1,
             "m_maxqty": r.integers(10, 51, int(reps.sum()), dtype=np.int32)}
    lmodes = C15_MODES + [b"BARGE"]
    lineitem = {"l_shipmode": StringColumn.from_list([lmodes[i] for i in r.integers(0, len(lmodes), nl)]),
                "l_quantity": r.integers(1, 51, nl, dtype=np.int32)}
    return Database([
        Table("nation", nation, {"n_name": Type.STRING, "n_regionkey": Type.INT}),
        Table("supplier", supplier, {"s_suppkey": Type.INT, "s_nation": Type.STRING, "s_acctbal": Type.INT}),
        Table("modes", modes, {"m_mode": Type.STRING, "m_carrier": Type.INT, "m_maxqty": Type.INT}),
        Table("lineitem", lineitem, {"l_shipmode": Type.STRING, "l_quantity": Type.INT})])


def plan_c15(alg, scal, Type, Reduction, variant="unique", region_cut=3):
    """One join on a string key.

    * ``unique``: suppliers joined to their nation by name (a unique table of
      the nation names), count and balance per region;
    * ``multi``: line items joined to every carrier of their shipping mode (a
      multimap keyed by the mode), count and quantity per carrier;
    * ``semi`` / ``anti``: the suppliers whose nation is (not) among the
      nations of the first regions, counted per nation name;
    * ``exists``: the line items of a mode with a carrier that takes their
      quantity (a semi join with a further condition on a string key), count
      and quantity per mode;
    * ``dup``: the carriers whose mode some line item ships by (a semi join
      whose build side repeats each of its eight keys many times)."""
    if variant == "dup":
        j = alg.semijoin(("l_shipmode", "m_mode"), None, alg.scan("lineitem"), alg.scan("modes"))
        agg = alg.aggregation(["m_carrier"], [(Reduction.COUNT, "", "carriers"),
                                              (Reduction.SUM, "m_maxqty", "maxqty")], j)
        return agg, {agg.opId: {"numgroups": 32}}
    if variant == "unique":
        j = alg.join(("n_name", "s_nation"), alg.scan("nation"), alg.scan("supplier"))
        agg = alg.aggregation(["n_regionkey"], [(Reduction.COUNT, "", "suppliers"),
                                                (Reduction.SUM, "s_acctbal", "balance")], j)
        return agg, {j.opId: {"multimatch": False}, agg.opId: {"numgroups": 5}}
    if variant == "multi":
        j = alg.join(("m_mode", "l_shipmode"), alg.scan("modes"), alg.scan("lineitem"))
        agg = alg.aggregation(["m_carrier"], [(Reduction.COUNT, "", "lines"),
                                              (Reduction.SUM, "l_quantity", "quantity")], j)
        return agg, {j.opId: {"multimatch": True}, agg.opId: {"numgroups": 32}}
    if variant in ("semi", "anti"):
        nat = alg.selection(scal.SmallerExpr(scal.AttrExpr("n_regionkey"), scal.ConstExpr(str(region_cut), Type.INT)),
                            alg.scan("nation"))
        make = alg.semijoin if variant == "semi" else alg.antijoin
        j = make(("n_name", "s_nation"), None, nat, alg.scan("supplier"))
        agg = alg.aggregation(["s_nation"], [(Reduction.COUNT, "", "suppliers")], j)
        return agg, {nat.opId: {"selectivity": region_cut / 5.0}, agg.opId: {"numgroups": 32}}
    cond = scal.LargerEqualExpr(scal.AttrExpr("m_maxqty"), scal.AttrExpr("l_quantity"))
    j = alg.semijoin(("m_mode", "l_shipmode"), cond, alg.scan("modes"), alg.scan("lineitem"))
    agg = alg.aggregation(["l_shipmode"], [(Reduction.COUNT, "", "lines"),
                                           (Reduction.SUM, "l_quantity", "quantity")], j)
    return agg, {j.opId: {"multimatch": True}, agg.opId: {"numgroups": 16}}


C16_CODES = ["13", "31", "23", "29", "30", "18", "17"]


def gen_c16(scale=1.0, seed=BASE_SEED + 16):
    """Q22-shaped: customers with a phone number "CC-AAA-BBB-CCCC" (country
    codes 10..34), an account balance (5% zero) and orders (every customer
    whose key is a multiple of 3 has none)."""
    nc = _n(150_000, scale, 64)
    no = _n(1_500_000, scale, 64)
    r = _rng(seed)
    cc = r.integers(10, 35, nc)
    rest = r.integers(0, [1000, 1000, 10000], (nc, 3))
    cust = {"c_custkey": (r.permutation(nc) + 1).astype(np.int32),
            "c_phone": StringColumn.from_list([b"%02d-%03d-%03d-%04d" % (c, a, b, d)
                                               for c, (a, b, d) in zip(cc, rest)]),
            "c_acctbal": np.where(r.random(nc) < 0.05, 0, r.integers(1, 1_000_000, nc)).astype(np.int32)}
    with_orders = np.arange(1, nc + 1, dtype=np.int32)
    with_orders = with_orders[with_orders % 3 != 0]
    orders = {"o_custkey": with_orders[r.integers(0, len(with_orders), no)]}
    return Database([
        Table("customer", cust, {"c_custkey": Type.INT, "c_phone": Type.STRING, "c_acctbal": Type.INT}),
        Table("orders", orders, {"o_custkey": Type.INT})])


def plan_c16(alg, scal, Type, Reduction):
    """TPC-H Q22: the customers of seven country codes (the phone number's
    first two characters) with a balance above those codes' average positive
    balance and no orders, counted and summed per country code (a substring as
    a map result and group key)."""
    def code(alias):
        return scal.SubstringExpr(scal.AttrExpr(alias + ".c_phone"), scal.ConstExpr("1", Type.INT),
                                  scal.ConstExpr("2", Type.INT))

    def in_codes(alias):
        return scal.InExpr(code(alias), [scal.ConstExpr(c, Type.STRING) for c in C16_CODES])

    c1 = alg.selection(scal.AndExpr(scal.LargerExpr(scal.AttrExpr("c1.c_acctbal"), scal.ConstExpr("0", Type.INT)),
                                    in_codes("c1")), alg.scan("customer", "c1"))
    avg = alg.aggregation([], [(Reduction.AVG, "c1.c_acctbal", "avg")], c1)
    c2 = alg.selection(in_codes("c2"), alg.scan("customer", "c2"))
    cj = alg.crossjoin(scal.LargerExpr(scal.AttrExpr("c2.c_acctbal"), scal.AttrExpr("avg")), avg, c2)
    anti = alg.antijoin([("o_custkey", "c_custkey")], None, alg.scan("orders"), cj)
    m = alg.map("cntrycode", code("c2"), anti)
    agg = alg.aggregation(["cntrycode"], [(Reduction.COUNT, "", "numcust"),
                                          (Reduction.SUM, "c_acctbal", "totacctbal")], m)
    cfg = {c1.opId: {"selectivity": 0.27}, c2.opId: {"selectivity": 0.28}, cj.opId: {"selectivity": 0.5},
           anti.opId: {"multimatch": False}, agg.opId: {"numgroups": 7}}
    return agg, cfg


# ------------------------------------------------------- c17 .. c19 -------------
# TPC-H Q13, Q20 and Q2 over one TPC-H-like schema with its strings (names,
# addresses, phone numbers, comments, part names and types).

TPCH_REGIONS = [b"AFRICA", b"AMERICA", b"ASIA", b"EUROPE", b"MIDDLE EAST"]
TPCH_COLORS = [b"almond", b"antique", b"aquamarine", b"azure", b"beige", b"bisque", b"black", b"blanched",
               b"blue", b"blush", b"brown", b"burlywood", b"chartreuse", b"chiffon", b"chocolate", b"coral",
               b"cornflower", b"cornsilk", b"cream", b"cyan", b"dark", b"deep", b"dim", b"dodger", b"drab",
               b"firebrick", b"floral", b"forest", b"frosted", b"gainsboro", b"ghost", b"goldenrod", b"green",
               b"grey", b"honeydew", b"hot", b"indian", b"ivory", b"khaki", b"lace", b"lavender", b"lawn",
               b"lemon", b"light", b"lime", b"linen", b"magenta", b"maroon", b"medium", b"metallic"]
ALNUM = np.frombuffer(b"abcdefghijklmnopqrstuvwxyzABCDEFGHIJKLMNOPQRSTUVWXYZ0123456789 ,.", dtype=np.uint8)


def _text(r, n, lo, hi):
    """n strings of lo..hi random characters (addresses)."""
    lens = r.integers(lo, hi + 1, n)
    chars = ALNUM[r.integers(0, len(ALNUM), int(lens.sum()))]
    offsets = np.zeros(n + 1, dtype=np.uint64)
    np.cumsum(lens, out=offsets[1:])
    return StringColumn(chars, offsets, 0)


def gen_tpch(scale=1.0, seed=BASE_SEED + 17):
    """TPC-H-like tables at scale factor ``scale`` (lineitem 6,000,000 rows at
    1.0): region, nation, supplier, customer, part, partsupp (four suppliers a
    part), orders (a third of the customers have none; 1% of the comments hold
    "special ... requests") and lineitem (lines of the partsupp pairs)."""
    ns = _n(10_000, scale, 16)
    nc = _n(150_000, scale, 16)
    np_ = _n(200_000, scale, 16)
    no = _n(1_500_000, scale, 16)
    nl = _n(6_000_000, scale, 64)
    r = _rng(seed)
    region = {"r_regionkey": np.arange(5, dtype=np.int32), "r_name": StringColumn.from_list(TPCH_REGIONS)}
    nation = {"n_nationkey": np.arange(25, dtype=np.int32), "n_name": StringColumn.from_list(C15_NATIONS),
              "n_regionkey": (np.arange(25) % 5).astype(np.int32)}
    supplier = {"s_suppkey": np.arange(1, ns + 1, dtype=np.int32),
                "s_name": StringColumn.from_list([b"Supplier#%09d" % (i + 1) for i in range(ns)]),
                "s_address": _text(r, ns, 10, 40),
                "s_nationkey": r.integers(0, 25, ns, dtype=np.int32),
                "s_phone": StringColumn.from_list([b"%02d-%03d-%03d-%04d" % (10 + a, b, c, d) for a, b, c, d in
                                                   r.integers(0, [25, 1000, 1000, 10000], (ns, 4))]),
                "s_acctbal": r.integers(0, 1_100_000, ns, dtype=np.int64).astype(np.uint64),
                "s_comment": _comments(r, ns)}
    customer = {"c_custkey": np.arange(1, nc + 1, dtype=np.int32)}
    names = r.integers(0, len(TPCH_COLORS), (np_, 5))
    t = r.integers(0, [len(C14_TYPE1), len(C14_TYPE2), len(C14_TYPE3)], (np_, 3))
    part = {"p_partkey": np.arange(1, np_ + 1, dtype=np.int32),
            "p_name": StringColumn.from_list([b" ".join(TPCH_COLORS[j] for j in row) for row in names]),
            "p_mfgr": StringColumn.from_list([b"Manufacturer#%d" % m for m in r.integers(1, 6, np_)]),
            "p_type": StringColumn.from_list([b" ".join((C14_TYPE1[a], C14_TYPE2[b], C14_TYPE3[c])) for a, b, c in t]),
            "p_size": r.integers(1, 51, np_, dtype=np.int32)}
    pk = np.repeat(np.arange(1, np_ + 1, dtype=np.int64), 4)
    i = np.tile(np.arange(4, dtype=np.int64), np_)
    partsupp = {"ps_partkey": pk.astype(np.int32),
                "ps_suppkey": ((pk + i * (ns // 4 + (pk - 1) // ns)) % ns + 1).astype(np.int32),
                "ps_availqty": r.integers(1, 10_000, 4 * np_, dtype=np.int32),
                "ps_supplycost": r.integers(100, 100_001, 4 * np_, dtype=np.int64).astype(np.uint64)}
    with_orders = np.arange(1, nc + 1, dtype=np.int32)
    with_orders = with_orders[with_orders % 3 != 0]
    orders = {"o_orderkey": np.arange(1, no + 1, dtype=np.int32),
              "o_custkey": with_orders[r.integers(0, len(with_orders), no)],
              "o_comment": _comments(r, no, (b"special", b"requests"), 0.01)}
    ps = r.integers(0, 4 * np_, nl)
    lineitem = {"l_partkey": partsupp["ps_partkey"][ps], "l_suppkey": partsupp["ps_suppkey"][ps],
                "l_quantity": r.integers(1, 51, nl, dtype=np.int32),
                "l_shipdate": (EPOCH_1992 + r.integers(0, DATE_RANGE, nl)).astype(np.int32)}
    I, S, F, D = Type.INT, Type.STRING, Type.FLOAT, Type.DATE
    return Database([
        Table("region", region, {"r_regionkey": I, "r_name": S}),
        Table("nation", nation, {"n_nationkey": I, "n_name": S, "n_regionkey": I}),
        Table("supplier", supplier, {"s_suppkey": I, "s_name": S, "s_address": S, "s_nationkey": I, "s_phone": S,
                                     "s_acctbal": F, "s_comment": S}),
        Table("customer", customer, {"c_custkey": I}),
        Table("part", part, {"p_partkey": I, "p_name": S, "p_mfgr": S, "p_type": S, "p_size": I}),
        Table("partsupp", partsupp, {"ps_partkey": I, "ps_suppkey": I, "ps_availqty": I, "ps_supplycost": F}),
        Table("orders", orders, {"o_orderkey": I, "o_custkey": I, "o_comment": S}),
        Table("lineitem", lineitem, {"l_partkey": I, "l_suppkey": I, "l_quantity": I, "l_shipdate": I})])


def plan_c17(alg, scal, Type, Reduction, numgroups=150_000):
    """TPC-H Q13: customers left outer join their orders whose comment does
    not mention special requests (NOT LIKE '%special%requests%' on
    variable-length comments), orders per customer, then customers per order
    count."""
    ords = alg.selection(scal.NotExpr(scal.LikeExpr(scal.AttrExpr("o_comment"),
                                                    scal.ConstExpr("%special%requests%", Type.STRING))),
                         alg.scan("orders"))
    j = alg.outerjoin([("c_custkey", "o_custkey")], None, ords, alg.scan("customer"))
    per = alg.aggregation(["c_custkey"], [(Reduction.COUNT, "o_orderkey", "c_count")], j)
    dist = alg.aggregation(["c_count"], [(Reduction.COUNT, "", "custdist")], per)
    return dist, {ords.opId: {"selectivity": 0.99}, j.opId: {"multimatch": True},
                  per.opId: {"numgroups": numgroups}, dist.opId: {"numgroups": 64}}


def plan_c18(alg, scal, Type, Reduction, start=EPOCH_1992 + 731, nation="CANADA", prefix="forest%"):
    """TPC-H Q20: suppliers of one nation (n_name = constant, joined by key)
    holding a part whose name starts with a word (LIKE 'forest%') in excess:
    twice the available quantity above the quantity the supplier shipped of
    that part in one year (a unique table keyed by two attributes, built from
    an aggregation); their names and addresses."""
    forest = alg.selection(scal.LikeExpr(scal.AttrExpr("p_name"), scal.ConstExpr(prefix, Type.STRING)),
                           alg.scan("part"))
    ps = alg.semijoin(("ps_partkey", "p_partkey"), None, forest, alg.scan("partsupp"))
    year = alg.selection(scal.AndExpr(
        scal.LargerEqualExpr(scal.AttrExpr("l_shipdate"), scal.ConstExpr(str(start), Type.DATE)),
        scal.SmallerExpr(scal.AttrExpr("l_shipdate"), scal.ConstExpr(str(start + 365), Type.DATE))),
        alg.scan("lineitem"))
    shipped = alg.aggregation(["l_partkey", "l_suppkey"], [(Reduction.SUM, "l_quantity", "sum_qty")], year)
    j = alg.join([("l_partkey", "ps_partkey"), ("l_suppkey", "ps_suppkey")], shipped, ps)
    excess = alg.selection(scal.LargerExpr(scal.MulExpr(scal.ConstExpr("2", Type.INT), scal.AttrExpr("ps_availqty")),
                                           scal.AttrExpr("sum_qty")), j)
    nat = alg.selection(scal.EqualsExpr(scal.AttrExpr("n_name"), scal.ConstExpr(nation, Type.STRING)),
                        alg.scan("nation"))
    supp = alg.join(("s_nationkey", "n_nationkey"), nat, alg.scan("supplier"))
    semi = alg.semijoin(("s_suppkey", "ps_suppkey"), None, excess, supp)
    proj = alg.projection(["s_name", "s_address"], semi)
    cfg = {forest.opId: {"selectivity": 0.1}, year.opId: {"selectivity": 0.15},
           shipped.opId: {"numgroups": 800_000}, j.opId: {"multimatch": False, "selectivity": 0.08},
           excess.opId: {"selectivity": 0.5}, nat.opId: {"selectivity": 0.04}, supp.opId: {"multimatch": False}}
    return proj, cfg


def plan_c19(alg, scal, Type, Reduction, region="EUROPE", size=15, suffix="%BRASS"):
    """TPC-H Q2: the parts of one size and type suffix (LIKE '%BRASS') with
    the supplier of one region (r_name = constant) offering the minimum supply
    cost (an aggregation's MIN joined back, equality of two attributes), with
    the supplier's and nation's strings in the result."""
    def europe(sup_alias):
        reg = alg.selection(scal.EqualsExpr(scal.AttrExpr("r_name"), scal.ConstExpr(region, Type.STRING)),
                            alg.scan("region"))
        nat = alg.join(("r_regionkey", "n_regionkey"), reg, alg.scan("nation"))
        return alg.join(("s_nationkey", "n_nationkey"), nat, alg.scan("supplier", sup_alias))

    def parts(alias):
        pref = (alias + ".") if alias else ""
        return alg.selection(scal.AndExpr(
            scal.LikeExpr(scal.AttrExpr(pref + "p_type"), scal.ConstExpr(suffix, Type.STRING)),
            scal.EqualsExpr(scal.AttrExpr(pref + "p_size"), scal.ConstExpr(str(size), Type.INT))),
            alg.scan("part", alias) if alias else alg.scan("part"))

    early = alg.semijoin(("ps_partkey", "earlyp.p_partkey"), None, parts("earlyp"), alg.scan("partsupp", "ps1"))
    cost = alg.join(("s_suppkey", "ps_suppkey"), europe(None), early)
    mins = alg.aggregation(["ps_partkey"], [(Reduction.MIN, "ps_supplycost", "min_supplycost")], cost)
    withp = alg.join(("p_partkey", "ps_partkey"), mins, parts(None))
    best = alg.join([("ps2.ps_partkey", "ps1.ps_partkey")], withp, alg.scan("partsupp", "ps2"))
    best = alg.selection(scal.EqualsExpr(scal.AttrExpr("min_supplycost"), scal.AttrExpr("ps2.ps_supplycost")), best)
    out = alg.join(("s2.s_suppkey", "ps2.ps_suppkey"), europe("s2"), best)
    proj = alg.projection(["s_acctbal", "s_name", "n_name", "p_partkey", "p_mfgr", "s_address", "s_phone",
                           "s_comment"], out)
    return proj, {mins.opId: {"numgroups": 4_000}}


GENERATORS = {"c0": gen_c0, "c1": gen_c1, "c2": gen_c2, "c3": gen_c3, "c5": gen_c5, "c7": gen_c5, "c8": gen_c5,
              "c9": gen_c9, "c9p": gen_c9, "c10": gen_c10, "c10p": gen_c10, "c11": gen_c11, "c12": gen_c11,
              "c13": gen_c5, "c14": gen_c14, "c15": gen_c15, "c16": gen_c16, "c17": gen_tpch, "c18": gen_tpch,
              "c19": gen_tpch}
PLANS = {"c0": plan_c0, "c1": plan_c1, "c2": plan_c2, "c3": plan_c3, "c5": plan_c5, "c7": plan_c7,
         "c8": plan_c8, "c9": plan_c9, "c9p": plan_c9p, "c10": plan_c10, "c10p": plan_c10p, "c11": plan_c11,
         "c12": plan_c12, "c13": plan_c13, "c14": plan_c14, "c15": plan_c15, "c16": plan_c16, "c17": plan_c17,
         "c18": plan_c18, "c19": plan_c19}


def build(name, alg, scale=1.0, **kw):
    """Build workload ``name``'s plan with this package's front end.  The
    cardinality hints follow ``scale`` (c3's group count: one million at full
    size), as an optimizer's estimate from the tables would."""
    import dogqc_b200.scalar as scal
    from dogqc_b200.relational import Reduction
    if name == "c3" and "numgroups" not in kw:
        kw["numgroups"] = max(1024, int(round(1_000_000 * scale)))
    if name == "c5" and "numgroups" not in kw:
        kw["numgroups"] = max(1024, int(round(150_000 * scale)))
    return PLANS[name](alg, scal, Type, Reduction, **kw)


def algorithmic_bytes(db, tables):
    """Bytes of the named tables' columns at stored width."""
    return sum(db[t].nbytes for t in tables)
