"""Small string tables and plans for the substring and string-comparison edge
cases: empty, one-byte and 286-byte strings, substring windows that start
before the string, end past it, lie wholly past it or have no length, nested
substrings, equality of two string columns, of a scanned string and one a join
carries, and a substring of a joined string as a group key; long strings (up
to 300 bytes, hashed and compared by whole warps) as group and join keys."""
import numpy as np

import dogqc_b200.scalar as scal
from dogqc_b200.database import Database, StringColumn, Table
from dogqc_b200.relational import RelationalAlgebra, Reduction
from dogqc_b200.types import Type

WORDS = [b"", b"a", b"ab", b"abc", b"hello world", b"hello", b"x" * 40, bytes(range(65, 91)) * 11,
         b"AB-12", b"13-555", b"31-1", b"1", b"ab-xyz"]

# (from, for) of SUBSTRING(s, from, for), optionally nested: (outer, inner)
WINDOWS = [((1, 2), None), ((3, 4), None), ((0, 3), None), ((-2, 5), None), ((5, 0), None), ((20, 3), None),
           ((1, 255), None), ((250, 5), None), ((2, -1), None), ((3, 20), (2, 5)), ((1, 4), (3, 9))]


def edge_db(n=5000, seed=7):
    r = np.random.Generator(np.random.Philox(seed))
    pick = lambda: StringColumn.from_list([WORDS[i] for i in r.integers(0, len(WORDS), n)])  # noqa: E731
    t = {"k": r.integers(0, 50, n, dtype=np.int32), "s": pick(), "t": pick()}
    d = {"dk": (r.permutation(50)).astype(np.int32),
         "ds": StringColumn.from_list([WORDS[i] for i in r.integers(0, len(WORDS), 50)])}
    return Database([Table("t", t, {"k": Type.INT, "s": Type.STRING, "t": Type.STRING}),
                     Table("d", d, {"dk": Type.INT, "ds": Type.STRING})])


def _const(v):
    return scal.ConstExpr(str(v), Type.INT)


def _resolve(db, build):
    alg = RelationalAlgebra(db)
    plan, cfg = build(alg)
    return alg.resolveAlgebraPlan(plan, cfg)


def substring_plan(db, window, nested=None):
    """Rows per SUBSTRING(s, from, for) (nested: of that, again), with the
    substring as the map result, group key and output column."""
    def build(alg):
        x = scal.SubstringExpr(scal.AttrExpr("s"), _const(window[0]), _const(window[1]))
        if nested:
            x = scal.SubstringExpr(x, _const(nested[0]), _const(nested[1]))
        m = alg.map("x", x, alg.scan("t"))
        agg = alg.aggregation(["x"], [(Reduction.COUNT, "", "cnt"), (Reduction.SUM, "k", "ks")], m)
        return agg, {agg.opId: {"numgroups": 64}}
    return _resolve(db, build)


def equal_strings_plan(db):
    """Rows whose two string columns are equal, or whose string equals the one
    the join carries from its build side, or whose second string starts with
    "ab"; counted per the first three bytes of the joined string."""
    def build(alg):
        j = alg.join(("dk", "k"), alg.scan("d"), alg.scan("t"))
        cond = scal.OrExpr(
            scal.OrExpr(scal.EqualsExpr(scal.AttrExpr("s"), scal.AttrExpr("t")),
                        scal.EqualsExpr(scal.AttrExpr("s"), scal.AttrExpr("ds"))),
            scal.EqualsExpr(scal.SubstringExpr(scal.AttrExpr("t"), _const(1), _const(2)),
                            scal.ConstExpr("ab", Type.STRING)))
        sel = alg.selection(cond, j)
        m = alg.map("d3", scal.SubstringExpr(scal.AttrExpr("ds"), _const(1), _const(3)), sel)
        agg = alg.aggregation(["d3"], [(Reduction.COUNT, "", "cnt")], m)
        return agg, {j.opId: {"multimatch": False}, sel.opId: {"selectivity": 0.3}, agg.opId: {"numgroups": 16}}
    return _resolve(db, build)


def like_joined_plan(db):
    """LIKE on a string carried through a multimatch join (a gathered
    reference one level down)."""
    def build(alg):
        j = alg.join(("k", "dk"), alg.scan("t"), alg.scan("d"))
        sel = alg.selection(scal.LikeExpr(scal.AttrExpr("s"), scal.ConstExpr("%l%o%", Type.STRING)), j)
        agg = alg.aggregation(["ds"], [(Reduction.COUNT, "", "cnt")], sel)
        return agg, {j.opId: {"multimatch": True}, sel.opId: {"selectivity": 0.2}, agg.opId: {"numgroups": 16}}
    return _resolve(db, build)


def long_db(n=4000, distinct=60, seed=11):
    """Strings of 0 to 300 bytes (``distinct`` of them, many sharing long
    prefixes) as keys: a fact table naming them, a dimension with each once
    and a multimap side with each one to three times."""
    r = np.random.Generator(np.random.Philox(seed))
    base = bytes(range(33, 127)) * 4
    words = [base[:int(x)] + b"#%d" % i for i, x in enumerate(r.integers(0, 297, distinct))]
    words[0] = b""
    f = {"fk": StringColumn.from_list([words[i] for i in r.integers(0, distinct, n)]),
         "fv": r.integers(0, 1000, n, dtype=np.int32)}
    dim = {"dk": StringColumn.from_list(words[1:]), "dv": np.arange(1, distinct, dtype=np.int32)}
    reps = r.integers(1, 4, distinct)
    mm = {"mk": StringColumn.from_list([w for w, k in zip(words, reps) for _ in range(k)]),
          "mv": np.arange(int(reps.sum()), dtype=np.int32)}
    return Database([Table("f", f, {"fk": Type.STRING, "fv": Type.INT}),
                     Table("dim", dim, {"dk": Type.STRING, "dv": Type.INT}),
                     Table("mm", mm, {"mk": Type.STRING, "mv": Type.INT})])


def long_key_plan(db, kind):
    """``group``: count and sum per long string; ``unique`` / ``multi``: the
    fact rows joined to the dimension / multimap by the long string;
    ``semi`` / ``anti``: the fact rows whose string the dimension holds (not)."""
    def build(alg):
        if kind == "group":
            agg = alg.aggregation(["fk"], [(Reduction.COUNT, "", "c"), (Reduction.SUM, "fv", "s")], alg.scan("f"))
            return agg, {agg.opId: {"numgroups": 64}}
        if kind in ("unique", "multi"):
            build_side, key = ("dim", "dk") if kind == "unique" else ("mm", "mk")
            j = alg.join((key, "fk"), alg.scan(build_side), alg.scan("f"))
            agg = alg.aggregation(["dv" if kind == "unique" else "mv"], [(Reduction.COUNT, "", "c"),
                                                                         (Reduction.SUM, "fv", "s")], j)
            return agg, {j.opId: {"multimatch": kind == "multi"}, agg.opId: {"numgroups": 256}}
        make = alg.semijoin if kind == "semi" else alg.antijoin
        j = make(("dk", "fk"), None, alg.scan("dim"), alg.scan("f"))
        agg = alg.aggregation(["fk"], [(Reduction.COUNT, "", "c")], j)
        return agg, {agg.opId: {"numgroups": 64}}
    return _resolve(db, build)
