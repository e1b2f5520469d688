"""Lowering of a resolved DogQC plan into the backend's pipeline IR.

The reference turns the operator tree into CUDA source with a produce/consume
walk (dogqc/cudaTranslator.py:31-89, translatorBase.py:6-63): a scan opens a
kernel, each operator appends code, a hash-join build or an aggregation closes
the kernel, and the parent continues in a new one.  This module does the same
walk but emits the IR of include/dogqc_b200.h: for every pipeline a source, the
slots (typed values per row), an operator list and one sink, plus the hash
tables and outputs the pipelines share.  The kernels that execute the IR are
hand-written (dogqc_b200/csrc/dq_kernels.cu); nothing here generates code.

Pipeline breaking follows the reference:

* Scan -> new pipeline over the table (only columns that are read are staged);
* Selection -> FILTER on the lowered condition (translator :353-366);
* Map -> expression ops whose result is converted to the attribute's C type
  (:402-422);
* EquiJoin -> the build child is produced first into a BUILD sink (unique hash
  table, ``multimatch=False``, hashJoins.py:95-109) or into a multimap built by
  a count pass, a bucket scan and a scatter pass over the same build pipeline
  (hashJoins.py:214-240, codegen.py:60-66); the probe child then continues with
  PROBE or EXPAND (hashJoins.py:113-153, 465-681);
* Aggregation -> AGG sink, then a new pipeline scanning the aggregation table,
  computing AVG = SUM / (ULL)COUNT (cudaTranslator.py:431-525);
* Materialize -> EMIT sink into an output (result or temp table, :582-616).

Expression typing follows C: char promotes to int, the usual arithmetic
conversions pick int / unsigned / long / unsigned long long, comparisons yield
int, and a map's value is converted to its attribute's C type
(codegen.py:37-45: INT->int, DATE->unsigned, CHAR->char, FLOAT/DOUBLE->ULL).
"""
import ctypes as C

from dogqc_b200 import _lib as L


class Unsupported(NotImplementedError):
    """The plan uses an operator or expression this backend does not execute."""


LANG = {"INT": "i32", "DATE": "u32", "CHAR": "i8", "FLOAT": "u64", "DOUBLE": "u64", "STRING": "str"}
CT = {"i8": L.I8, "i32": L.I32, "u32": L.U32, "i64": L.I64, "u64": L.U64, "str": L.STR}
NP_DTYPE = {L.I8: "int8", L.I32: "int32", L.U32: "uint32", L.I64: "int64", L.U64: "uint64"}


class _Op(dict):
    """One IR op (its fields), plus the plan's estimate of the fraction of rows
    that pass it (filters and probes) and the id of the algebra operator it
    came from, which place the lane refill."""
    sel = 1.0
    origin = None


# A filter or probe whose estimated pass fraction is at most this refills the
# lanes of the generated kernel before the rest of the pipeline.
REFILL_SELECTIVITY = 0.5
L2_TABLE_BYTES = 48 << 20   # join tables the runtime gives 4x slots (they stay in L2)
NARROW = ("i8", "i32", "u32")


def refill_point(ops, buffers=None):
    """The ``compact`` field of dq_pipeline: 1 + the index of the level-0
    filter or probe after which the lanes are refilled, or 0.

    ``buffers`` (``Backend.setBuffers``): the operator ids the reference wraps
    in its ``LaneRefill`` (dogqc/cudaTranslator.py:84-86) -- the refill goes
    after the filter of such a selection or the probe of such a join, the first
    of them in the pipeline; a pipeline with none has no refill, as in the
    reference.  Without positions: after the first filter or probe estimated to
    pass at most REFILL_SELECTIVITY of its rows."""
    for k, o in enumerate(ops):
        if o["kind"] == L.OP_EXPAND:
            break
        if o["kind"] not in (L.OP_FILTER, L.OP_PROBE):
            continue
        if buffers is not None:
            if getattr(o, "origin", None) in buffers:
                return k + 1
        elif getattr(o, "sel", 1.0) <= REFILL_SELECTIVITY:
            return k + 1
    return 0


def _tname(t):
    return t.name if hasattr(t, "name") else str(t)


def lang_type(relational_type):
    n = _tname(relational_type)
    if n not in LANG:
        raise Unsupported("no C type for attribute type %s" % n)
    return LANG[n]


def _promote(t):
    return "i32" if t == "i8" else t


def common_type(a, b):
    a, b = _promote(a), _promote(b)
    if "u64" in (a, b):
        return "u64"
    if "i64" in (a, b):
        return "i64"
    if "u32" in (a, b):
        return "u32"
    return "i32"


def _wrap(v, t):
    """Two's-complement value of v in C type t, as a Python int (signed for i*)."""
    bits = {"i8": 8, "i32": 32, "u32": 32, "i64": 64, "u64": 64}[t]
    v &= (1 << bits) - 1
    if t.startswith("i") and v >= 1 << (bits - 1):
        v -= 1 << bits
    return v


def _imm64(v):
    """Immediate as the int64 bit pattern the device reads."""
    v &= (1 << 64) - 1
    return v - (1 << 64) if v >= 1 << 63 else v


class Imm(object):
    def __init__(self, value, ctype):
        self.value = value
        self.ctype = ctype


class Pattern(object):
    def __init__(self, data):
        self.data = data


class Res(object):
    def __init__(self, kind, **kw):
        self.kind = kind
        self.nkeys = kw.get("nkeys", 0)
        self.key_ctype = kw.get("key_ctype", [])
        self.pay_ctype = kw.get("pay_ctype", [])
        self.agg_red = kw.get("agg_red", [])
        self.capacity = int(kw.get("capacity", 1024))
        self.group_hint = int(kw.get("group_hint", 0))
        self.name = kw.get("name")
        self.columns = kw.get("columns", [])


def _costly_rows(node):
    """Whether producing ``node``'s rows does costly per-row work: a join, or
    a LIKE or SUBSTRING in a selection or map."""
    def costly_expr(e):
        if e is None:
            return False
        if type(e).__name__ in ("LikeExpr", "SubstringExpr"):
            return True
        return any(costly_expr(getattr(e, a, None)) for a in ("leftChild", "rightChild", "child"))
    k = type(node).__name__
    if k in ("EquiJoin", "CrossJoin", "Aggregation"):
        return True
    if k == "Selection" and costly_expr(node.condition):
        return True
    if k == "Map" and costly_expr(node.expression):
        return True
    child = getattr(node, "child", None)
    return child is not None and _costly_rows(child)


class Pipe(object):
    """One pipeline under construction."""

    def __init__(self, source_kind, table=None, source_res=-1):
        self.source_kind = source_kind
        self.table = table
        self.source_res = source_res
        self.cols = []          # source columns (names or output indices)
        self.slots = []         # dicts: kind, level, ctype, src, res
        self.ops = []           # dicts
        self.lists = []
        self.patterns = []
        self.att = {}           # attribute id -> slot index
        self.level = 0
        self.lazy = {}          # attribute id -> callable creating its slot
        self.strref = {}        # string column slot -> register holding its reference

    def slot(self, kind, level, ctype, src=0, res=-1):
        self.slots.append(dict(kind=kind, level=level, ctype=ctype, src=src, res=res))
        if len(self.slots) > L.MAX_SLOTS:
            raise Unsupported("pipeline needs more than %d slots" % L.MAX_SLOTS)
        return len(self.slots) - 1

    def reg(self, ctype):
        return self.slot(L.SLOT_REG, self.level, ctype)

    def col(self, name):
        if name not in self.cols:
            self.cols.append(name)
        return self.cols.index(name)

    def op(self, kind, **kw):
        d = _Op(kind=kind, sub=0, dst=-1, a=-1, b=-1, c=-1, ctype=0, flags=0, res=-1,
                list=0, nlist=0, list2=0, nlist2=0, imm=0)
        d.update(kw)
        self.ops.append(d)
        if len(self.ops) > L.MAX_OPS:
            raise Unsupported("pipeline needs more than %d ops" % L.MAX_OPS)
        return d

    def list_(self, items):
        start = len(self.lists)
        self.lists.extend(items)
        if len(self.lists) > L.MAX_LIST:
            raise Unsupported("pipeline lists exceed %d entries" % L.MAX_LIST)
        return start, len(items)

    def pattern(self, data):
        if data in self.patterns:
            return self.patterns.index(data)
        self.patterns.append(data)
        if len(self.patterns) > L.MAX_PATTERNS:
            raise Unsupported("more than %d string constants in a pipeline" % L.MAX_PATTERNS)
        return len(self.patterns) - 1

    def attr_slot(self, attr):
        if attr.id not in self.att:
            if attr.id in self.lazy:
                self.att[attr.id] = self.lazy.pop(attr.id)()
            else:
                raise Unsupported("attribute %s (%d) is not available in this pipeline" % (attr.name, attr.id))
        return self.att[attr.id]

    def value_slot(self, attr):
        """The slot of ``attr`` as a value (see ``ref_of``)."""
        return self.ref_of(self.attr_slot(attr))

    def ref_of(self, s):
        """Slot ``s`` as a value: a scanned string becomes its 64-bit reference
        (plan string source, substring window, row), computed first thing in
        the pipeline so refill and expansion carry it like any other value."""
        if self.slots[s]["kind"] != L.SLOT_STR:
            return s
        if s not in self.strref:
            r = self.slot(L.SLOT_REG, 0, "str")
            self.op(L.OP_STRREF, dst=r, a=s, ctype=L.STR)
            self.ops.insert(0, self.ops.pop())
            self.strref[s] = r
        return self.strref[s]

    def clone_for_rebuild(self):
        """Fresh copy of the source part (used to run a build pipeline twice)."""
        return Pipe(self.source_kind, self.table, self.source_res)


class Lowering(object):
    """Lowers resolved plan roots; ``ir()`` returns the ctypes plan description."""

    def __init__(self, plan, options=None):
        self.roots = plan if isinstance(plan, list) else [plan]
        self.options = dict(options or {})
        self.res = []
        self.pipes = []
        self.result_res = -1
        self.result_names = []
        self.result_types = []
        self.temp = {}
        self.parent = {}
        self.joins = {}   # id(EquiJoin node) -> build information
        self.profile_points = []   # operator ids with a lane-activity profile, by point
        for r in self.roots:
            self._link(r, None)
        for r in self.roots:
            self.produce(r)
        if self.result_res < 0:
            raise Unsupported("plan has no result materialisation")

    # -- tree helpers ------------------------------------------------------------
    def _link(self, node, parent):
        self.parent[id(node)] = parent
        for ch in self._children(node):
            self._link(ch, node)

    @staticmethod
    def _children(node):
        k = type(node).__name__
        if k in ("Selection", "Map", "Aggregation", "Projection", "Materialize"):
            return [node.child]
        if k in ("EquiJoin", "CrossJoin"):
            return [node.leftChild, node.rightChild]
        return []

    def new_res(self, res):
        self.res.append(res)
        return len(self.res) - 1

    # -- produce / consume -------------------------------------------------------
    def produce(self, node):
        k = type(node).__name__
        if k == "Scan":
            self.scan(node)
        elif k in ("Selection", "Map", "Projection", "Materialize", "Aggregation"):
            self.produce(node.child)
        elif k == "EquiJoin":
            self.produce_join(node)
        elif k == "CrossJoin":
            self.produce_cross(node)
        else:
            raise Unsupported("operator %s" % k)

    def produce_cross(self, node):
        """Nested-loop join (cudaTranslator.py:369-397: the inner side, the left
        child, materialised; every outer row loops over all of it with the
        condition as the filter).  Lowered as a multimap without keys: one
        bucket holds every inner row, the outer rows' expansion walks it, the
        condition filters the pairs.  Outer rows share the one range, so the
        grouped deferral reads each chunk of the inner rows once for all."""
        if self.joins.get(id(node), {}).get("built"):
            self.produce(node.rightChild)
            return
        atts = list(node.leftChild.outRelation.values())
        payload = [lang_type(a.dataType) for a in atts]
        if any(t == "str" for t in payload):
            raise Unsupported("string attributes in nested-loop join inputs")
        if len(payload) > L.MAX_PAY:
            raise Unsupported("more than %d payload attributes" % L.MAX_PAY)
        rid = self.new_res(Res(L.RES_MULTI, nkeys=0, key_ctype=[], pay_ctype=payload, capacity=1))
        info = dict(res=rid, unique=False, bk=[], pk=[], build_atts=atts, passes=["count", "scatter"], cross=True)
        self.joins[id(node)] = info
        for p in info["passes"]:
            info["pass"] = p
            self.produce(node.leftChild)
        info["built"] = True
        self.produce(node.rightChild)

    def consume(self, node, child, pipe):
        """Continue ``pipe`` (which delivers ``child``'s rows) at ``node``."""
        k = type(node).__name__
        if k == "Selection":
            self.filter(pipe, node.condition, getattr(node, "selectivity", 1.0), origin=node.opId)
            self.consume_parent(node, pipe)
        elif k == "Map":
            v = self.expr(pipe, node.expression)
            want = lang_type(node.mapAttr.dataType)
            pipe.att[node.mapAttr.id] = self.materialize_value(pipe, v, want)
            self.consume_parent(node, pipe)
        elif k == "Projection":
            self.consume_parent(node, pipe)
        elif k == "EquiJoin":
            if child is node.leftChild:
                self.join_build_sink(node, pipe)
            else:
                self.join_probe(node, pipe)
                self.consume_parent(node, pipe)
        elif k == "CrossJoin":
            if child is node.leftChild:
                self.join_build_sink(node, pipe)
            else:
                self.join_probe(node, pipe)
                self.filter(pipe, node.condition, getattr(node, "selectivity", 1.0), origin=node.opId)
                self.consume_parent(node, pipe)
        elif k == "Aggregation":
            self.aggregate(node, pipe)
        elif k == "Materialize":
            self.materialize(node, pipe)
        else:
            raise Unsupported("operator %s" % k)

    def consume_parent(self, node, pipe):
        if node.opId in self.options.get("profilers", ()):
            # the reference's LaneActivityProfiler sits between the operator
            # and its parent (dogqc/cudaTranslator.py:87-88): count the lanes
            # still active as the operator hands its rows on
            if node.opId not in self.profile_points:
                self.profile_points.append(node.opId)
            pipe.op(L.OP_PROFILE, res=self.profile_points.index(node.opId))
        parent = self.parent[id(node)]
        if parent is None:
            raise Unsupported("plan root %s is not a materialisation" % type(node).__name__)
        self.consume(parent, node, pipe)

    # -- scans -------------------------------------------------------------------
    def scan(self, node):
        if node.isTempScan:
            rid = self.temp[node.table["name"]]
            r = self.res[rid]
            pipe = Pipe(L.SRC_OUTPUT, source_res=rid)
            for id, a in node.outRelation.items():
                j = r.columns.index(a.sourceId)
                pipe.lazy[id] = self._lazy_col(pipe, str(j), r.pay_ctype[j])
        else:
            pipe = Pipe(L.SRC_TABLE, table=node.table["name"])
            for id, a in node.outRelation.items():
                pipe.lazy[id] = self._lazy_col(pipe, a.name, lang_type(a.dataType))
        self._scan_node = node
        self.consume_parent(node, pipe)

    @staticmethod
    def _lazy_col(pipe, name, ctype):
        def make():
            c = pipe.col(name)
            if ctype == "str":
                return pipe.slot(L.SLOT_STR, 0, "str", src=c)
            return pipe.slot(L.SLOT_COL, 0, ctype, src=c)
        return make

    # -- expressions -------------------------------------------------------------
    def const(self, e):
        t = _tname(e.type)
        tok = e.token
        if t == "STRING":
            return Pattern(tok.encode() if isinstance(tok, str) else bytes(tok))
        if t == "CHAR":
            return Imm(_wrap(ord(tok[0]), "i8"), "i8")
        if t == "FLOAT":
            raise Unsupported("FLOAT constants are not exact (the reference emits (float)%s); use INT" % tok)
        try:
            v = int(tok)
        except ValueError:
            raise Unsupported("non-integer constant %r is not exact" % tok)
        return Imm(v, "i32" if -(1 << 31) <= v < (1 << 31) else "i64")

    def ctype_of(self, pipe, v):
        if isinstance(v, Imm):
            return v.ctype
        if isinstance(v, Pattern):
            return "strconst"
        return pipe.slots[v]["ctype"]

    def materialize_value(self, pipe, v, ctype):
        """A slot holding v converted to ctype (a string as its reference)."""
        if isinstance(v, Pattern):
            raise Unsupported("string constants as map results")
        if not isinstance(v, Imm) and pipe.slots[v]["ctype"] == ctype:
            return pipe.ref_of(v) if ctype == "str" else v
        if ctype == "str" or (not isinstance(v, Imm) and pipe.slots[v]["ctype"] == "str"):
            raise Unsupported("conversions between strings and numbers")
        d = pipe.reg(ctype)
        if isinstance(v, Imm):
            pipe.op(L.OP_CAST, dst=d, ctype=CT[ctype], flags=L.OPF_A_IMM, imm=_imm64(_wrap(v.value, ctype)))
        else:
            pipe.op(L.OP_CAST, dst=d, a=v, ctype=CT[ctype])
        return d

    def binary_operands(self, pipe, a, b, t):
        """Operand fields for an op computing in t; at most one immediate."""
        kw = {}
        if isinstance(a, Imm) and isinstance(b, Imm):
            a = self.materialize_value(pipe, a, t)
        if isinstance(a, Imm):
            kw.update(flags=L.OPF_A_IMM, imm=_imm64(_wrap(a.value, t)), b=b)
        elif isinstance(b, Imm):
            kw.update(flags=L.OPF_B_IMM, imm=_imm64(_wrap(b.value, t)), a=a)
        else:
            kw.update(a=a, b=b)
        return kw

    ARITH = {"AddExpr": L.ADD, "SubExpr": L.SUB, "MulExpr": L.MUL, "DivExpr": L.DIV}
    CMPS = {"EqualsExpr": L.EQ, "SmallerExpr": L.LT, "SmallerEqualExpr": L.LE,
            "LargerExpr": L.GT, "LargerEqualExpr": L.GE}

    def expr(self, pipe, e):
        """Lower scalar expression e; returns a slot index, Imm or Pattern."""
        k = type(e).__name__
        if k == "AttrExpr":
            return pipe.attr_slot(e.attr)
        if k == "ConstExpr":
            return self.const(e)
        if k in self.ARITH:
            a = self.expr(pipe, e.leftChild)
            b = self.expr(pipe, e.rightChild)
            t = common_type(self.ctype_of(pipe, a), self.ctype_of(pipe, b))
            d = pipe.reg(t)
            pipe.op(L.OP_ARITH, sub=self.ARITH[k], dst=d, ctype=CT[t], **self.binary_operands(pipe, a, b, t))
            return d
        if k in self.CMPS:
            a = self.expr(pipe, e.leftChild)
            b = self.expr(pipe, e.rightChild)
            ta, tb = self.ctype_of(pipe, a), self.ctype_of(pipe, b)
            if "str" in (ta, tb) or "strconst" in (ta, tb):
                # the reference's stringEquals (util.cuh:86-102, scalarAlgebra.py:167-188);
                # it has no ordering of strings
                if k != "EqualsExpr":
                    raise Unsupported("ordering comparisons on strings")
                if ta == "strconst":
                    a, b = b, a
                    ta, tb = tb, ta
                if ta == "strconst":
                    return Imm(int(a.data == b.data), "i32")
                if ta != "str" or tb not in ("str", "strconst"):
                    raise Unsupported("comparisons of strings with numbers")
                d = pipe.reg("i32")
                if tb == "strconst":
                    pipe.op(L.OP_STREQ, dst=d, a=self.str_operand(pipe, a), res=pipe.pattern(b.data))
                else:
                    pipe.op(L.OP_STREQ, dst=d, a=self.str_operand(pipe, a), b=self.str_operand(pipe, b), res=-1)
                return d
            t = common_type(ta, tb)
            d = pipe.reg("i32")
            pipe.op(L.OP_CMP, sub=self.CMPS[k], dst=d, ctype=CT[t], **self.binary_operands(pipe, a, b, t))
            return d
        if k in ("AndExpr", "OrExpr"):
            a = self.as_slot(pipe, self.expr(pipe, e.leftChild))
            b = self.as_slot(pipe, self.expr(pipe, e.rightChild))
            d = pipe.reg("i32")
            pipe.op(L.OP_LOGIC, sub=L.AND if k == "AndExpr" else L.OR, dst=d, a=a, b=b)
            return d
        if k == "NotExpr":
            a = self.as_slot(pipe, self.expr(pipe, e.child))
            d = pipe.reg("i32")
            pipe.op(L.OP_LOGIC, sub=L.NOT, dst=d, a=a)
            return d
        if k == "LikeExpr":
            s = self.expr(pipe, e.leftChild)
            p = self.expr(pipe, e.rightChild)
            if not isinstance(p, Pattern) or isinstance(s, (Imm, Pattern)) or self.ctype_of(pipe, s) != "str":
                raise Unsupported("LIKE needs a string value and a constant pattern")
            d = pipe.reg("i32")
            pipe.op(L.OP_LIKE, dst=d, a=self.str_operand(pipe, s), res=pipe.pattern(p.data))
            return d
        if k == "SubstringExpr":
            return self.substring(pipe, e)
        if k == "ExtractExpr":
            a = self.expr(pipe, e.child)
            t = common_type(self.ctype_of(pipe, a), "i32")
            ext = _tname(e.extract)
            if ext == "YEAR":
                steps = [(L.DIV, 10000)]
            elif ext == "DAY":
                steps = [(L.MOD, 100)]
            else:
                steps = [(L.DIV, 100), (L.MOD, 100)]
            for sub, c in steps:
                d = pipe.reg(t)
                pipe.op(L.OP_ARITH, sub=sub, dst=d, ctype=CT[t], **self.binary_operands(pipe, a, Imm(c, "i32"), t))
                a = d
            return a
        if k == "CaseExpr":
            d = pipe.reg("u64")
            if e.exprElse is not None:
                ev = self.expr(pipe, e.exprElse)
                self._cast_into(pipe, d, ev, "u64")
            else:
                pipe.op(L.OP_CAST, dst=d, ctype=CT["u64"], flags=L.OPF_A_IMM, imm=0)
            for w, th in reversed(e.exprListWhenThen):
                c = self.as_slot(pipe, self.expr(pipe, w))
                tv = self.expr(pipe, th)
                kw = dict(dst=d, a=c, c=d, ctype=CT["u64"])
                if isinstance(tv, Imm):
                    kw.update(flags=L.OPF_B_IMM, imm=_imm64(_wrap(tv.value, "u64")))
                else:
                    kw.update(b=tv)
                pipe.op(L.OP_SELECT, **kw)
            return d
        raise Unsupported("scalar expression %s" % k)

    @staticmethod
    def str_operand(pipe, s):
        """A string operand: a scanned column is read in place at level 0; below
        an expansion its reference is used, a value that deferred expansion
        ranges carry like any other."""
        return pipe.ref_of(s) if pipe.level > 0 else s

    def substring(self, pipe, e):
        """SUBSTRING(s, from, for) with constant bounds (the reference's
        stringSubstring, util.cuh:132-142): a reference to the same bytes with a
        window; nested substrings narrow it.  The window ends within the
        string's first 255 bytes."""
        s = self.expr(pipe, e.exprString)
        f = self.expr(pipe, e.exprFrom)
        n = self.expr(pipe, e.exprFor)
        if isinstance(s, (Imm, Pattern)) or self.ctype_of(pipe, s) != "str":
            raise Unsupported("SUBSTRING of a string constant")
        if not isinstance(f, Imm) or not isinstance(n, Imm):
            raise Unsupported("SUBSTRING bounds that are not constants")
        fv, nv = _wrap(f.value, "i32"), _wrap(n.value, "i32")
        if fv - 1 > 255 or fv - 1 + nv > 255:
            raise Unsupported("SUBSTRING windows ending past byte 255")
        d = pipe.reg("str")
        pipe.op(L.OP_SUBSTR, dst=d, a=pipe.ref_of(s), ctype=L.STR,
                imm=_imm64((fv & 0xffffffff) | ((nv & 0xffffffff) << 32)))
        return d

    def _cast_into(self, pipe, d, v, t):
        if isinstance(v, Imm):
            pipe.op(L.OP_CAST, dst=d, ctype=CT[t], flags=L.OPF_A_IMM, imm=_imm64(_wrap(v.value, t)))
        else:
            pipe.op(L.OP_CAST, dst=d, a=v, ctype=CT[t])

    def as_slot(self, pipe, v):
        if isinstance(v, Imm):
            return self.materialize_value(pipe, v, _promote(v.ctype))
        if isinstance(v, Pattern):
            raise Unsupported("string constant used as a value")
        return v

    def filter(self, pipe, condition, selectivity=1.0, origin=None):
        v = self.expr(pipe, condition)
        if isinstance(v, Imm):
            if v.value != 0:
                return
            v = self.materialize_value(pipe, v, "i32")
        op = pipe.op(L.OP_FILTER, a=v)
        op.sel = selectivity
        op.origin = origin

    # -- joins -------------------------------------------------------------------
    def produce_join(self, node):
        if self.joins.get(id(node), {}).get("built"):
            # a second pass over an enclosing build pipeline: this join's own
            # table exists already, only its probe side is produced again
            self.produce(node.rightChild)
            return
        jt = _tname(node.joinType)
        if jt == "OUTER":
            # The reference's outer join runs on its multimatch table only and
            # yields the inner join's rows: an unmatched probe row's extra
            # iteration repeats the key check on a foreign payload row and drops
            # it (hashJoins.py:473-530, include/hashing.cuh:189-199); its unique
            # table rejects the join type (hashJoins.py:95-109).
            if not getattr(node, "multimatch", True):
                raise Unsupported("outer joins on unique keys (the reference's unique hash table rejects them)")
            jt = "INNER"
        semi = jt in ("SEMI", "ANTI")
        if node.conditions is not None and not semi:
            # the reference evaluates a join's further conditions only in its
            # semi and anti probes (hashJoins.py:203-204, 264-265)
            raise Unsupported("inner and outer joins with further conditions (the reference does not evaluate them)")
        bk = list(node.buildKeyAttributes.values())
        pk = list(node.probeKeyAttributes.values())
        if len(bk) > L.MAX_KEYS:
            raise Unsupported("more than %d join keys" % L.MAX_KEYS)
        key_types = []
        for b, p in zip(bk, pk):
            tb, tp = lang_type(b.dataType), lang_type(p.dataType)
            if "str" in (tb, tp):
                # string keys: references, hashed and compared by their bytes
                # (the reference's stringHash / stringEquals, hashTableUtil.py:15-35)
                if tb != tp:
                    raise Unsupported("join keys comparing a string with a number")
                key_types.append("str")
            else:
                key_types.append(common_type(tb, tp))
        build_atts = list(node.leftChild.outRelation.values())
        # A semi or anti join asks whether a build row with equal keys exists;
        # without a further condition only the keys matter (a unique table of
        # keys, the reference's filter table, hashJoins.py:159-211).  With a
        # condition every build row of the key may decide, so the build side
        # becomes a multimap of its keys and the attributes the condition reads,
        # walked per probe row until a row satisfies it (the reference's
        # multimatch semi/anti probe, hashJoins.py:244-272).
        unique = (not getattr(node, "multimatch", True) or semi) and node.conditions is None
        est = max(int(node.leftChild.tupleNum), 1)
        cap = max(int(est * float(getattr(node, "htSizeFactor", 2.0))), 16)
        if semi and node.conditions is None:
            build_atts = []
        if unique:
            packed = "str" not in key_types and (
                len(bk) == 1 or (len(bk) == 2 and all(t in ("i8", "i32", "u32") for t in key_types)))
            alias = {}
            if packed:
                # the packed tag is the exact key: build keys that no operator above
                # the join reads need not be stored in the payload, and above an
                # inner join a build key equals its probe key, so one of the same
                # type is read from the probe side
                for b, p in zip(bk, pk):
                    if jt == "INNER" and b.dataType == p.dataType and lang_type(b.dataType) == lang_type(p.dataType):
                        alias[b.id] = p
                build_atts = [a for a in build_atts
                              if not (a in bk and (a.lastUse <= node.opId or a.id in alias))]
            payload = [lang_type(a.dataType) for a in build_atts]
            rid = self.new_res(Res(L.RES_UNIQUE, nkeys=len(bk), key_ctype=key_types, pay_ctype=payload,
                                   capacity=cap))
            info = dict(res=rid, unique=True, bk=bk, pk=pk, build_atts=build_atts, passes=["build"], alias=alias)
        else:
            keys_in_payload = [build_atts.index(b) if b in build_atts else -1 for b in bk]
            atts = list(build_atts)
            for i, b in enumerate(bk):
                if keys_in_payload[i] < 0:
                    atts.append(b)
            payload = [lang_type(a.dataType) for a in atts]
            if len(payload) > L.MAX_PAY:
                raise Unsupported("more than %d payload attributes" % L.MAX_PAY)
            rid = self.new_res(Res(L.RES_MULTI, nkeys=len(bk), key_ctype=key_types, pay_ctype=payload,
                                   capacity=cap))
            info = dict(res=rid, unique=False, bk=bk, pk=pk, build_atts=atts, passes=["count", "scatter"],
                        exists=semi)
            if "str" not in payload and _costly_rows(node.leftChild):
                # the multimap's two passes would each redo the build side's
                # costly per-row work (string predicates, joins): one pass
                # writes its rows' keys and payload to a temp table that the
                # count and scatter passes scan instead
                info["stage"] = self.new_res(Res(L.RES_OUTPUT, pay_ctype=payload, capacity=max(est, 1024),
                                                 columns=[a.id for a in atts]))
        self.joins[id(node)] = info
        if "stage" in info:
            info["pass"] = "stage"
            self.produce(node.leftChild)
            for p in info["passes"]:
                info["pass"] = p
                pipe = Pipe(L.SRC_OUTPUT, source_res=info["stage"])
                for j, a in enumerate(info["build_atts"]):
                    pipe.lazy[a.id] = self._lazy_col(pipe, str(j), lang_type(a.dataType))
                self.join_build_sink(node, pipe)
        else:
            for p in info["passes"]:
                info["pass"] = p
                self.produce(node.leftChild)
        info["built"] = True
        self.produce(node.rightChild)

    def join_build_sink(self, node, pipe):
        info = self.joins[id(node)]
        if info.get("pass") == "stage":
            sl, sn = pipe.list_([pipe.value_slot(a) for a in info["build_atts"]])
            pipe.op(L.OP_EMIT, res=info["stage"], list=sl, nlist=sn)
            self.finish(pipe)
            return
        keys = [pipe.value_slot(a) for a in info["bk"]]
        kl, kn = pipe.list_(keys)
        if info["unique"]:
            pl, pn = pipe.list_([pipe.value_slot(a) for a in info["build_atts"]])
            pipe.op(L.OP_BUILD, res=info["res"], list=kl, nlist=kn, list2=pl, nlist2=pn)
        elif info["pass"] == "count":
            pipe.op(L.OP_MM_COUNT, res=info["res"], list=kl, nlist=kn)
        else:
            pl, pn = pipe.list_([pipe.value_slot(a) for a in info["build_atts"]])
            pipe.op(L.OP_MM_SCATTER, res=info["res"], list=kl, nlist=kn, list2=pl, nlist2=pn)
        self.finish(pipe)

    def join_probe(self, node, pipe):
        info = self.joins[id(node)]
        jt = _tname(node.joinType)
        keys = [pipe.value_slot(a) for a in info["pk"]]
        kl, kn = pipe.list_(keys)
        if info["unique"]:
            dsts = []
            for a in info["build_atts"]:
                s = pipe.reg(lang_type(a.dataType))
                pipe.att[a.id] = s
                dsts.append(s)
            for b, ks in zip(info["bk"], keys):
                if b.id in info["alias"]:
                    pipe.att[b.id] = ks
            pl, pn = pipe.list_(dsts)
            sub = {"INNER": L.JOIN_INNER, "SEMI": L.JOIN_SEMI, "ANTI": L.JOIN_ANTI}[jt]
            op = pipe.op(L.OP_PROBE, sub=sub, res=info["res"], list=kl, nlist=kn, list2=pl, nlist2=pn)
            op.origin = node.opId
            # fraction of probe rows that find a match (the plan's estimate)
            probe_rows = max(getattr(node.rightChild, "tupleNum", 0), 1)
            op.sel = min(1.0, getattr(node, "tupleNum", probe_rows) / float(probe_rows))
        elif info.get("exists"):
            self.exists_probe(node, pipe, info, jt, kl, kn)
        else:
            if pipe.level + 1 >= L.MAX_LEVELS:
                raise Unsupported("more than %d nested multimatch joins in one pipeline" % (L.MAX_LEVELS - 1))
            lv = pipe.level + 1
            gathers = []
            for j, a in enumerate(info["build_atts"]):
                s = pipe.slot(L.SLOT_GATHER, lv, lang_type(a.dataType), src=j, res=info["res"])
                pipe.att[a.id] = s
                gathers.append(s)
            bkeys = [gathers[info["build_atts"].index(b)] for b in info["bk"]]
            bl, bn = pipe.list_(bkeys)
            pipe.op(L.OP_EXPAND, res=info["res"], list=kl, nlist=kn, list2=bl, nlist2=bn)
            pipe.level = lv

    def exists_probe(self, node, pipe, info, jt, kl, kn):
        """Semi/anti join with a condition: an EXISTS op walks the probe row's
        key range of the multimap; for each build row with equal keys the
        condition's ops (the count that follow it, on the build row's gathered
        attributes one level down) decide; the first build row that satisfies
        the condition ends the walk.  The row stays (SEMI) or goes (ANTI)
        depending on whether one did.  The build attributes are visible to the
        condition only."""
        if pipe.level + 1 >= L.MAX_LEVELS:
            raise Unsupported("more than %d nested multimatch joins in one pipeline" % (L.MAX_LEVELS - 1))
        lv = pipe.level + 1
        gathers = []
        for j, a in enumerate(info["build_atts"]):
            gathers.append(pipe.slot(L.SLOT_GATHER, lv, lang_type(a.dataType), src=j, res=info["res"]))
        bkeys = [gathers[info["build_atts"].index(b)] for b in info["bk"]]
        bl, bn = pipe.list_(bkeys)
        sub = L.JOIN_SEMI if jt == "SEMI" else L.JOIN_ANTI
        op = pipe.op(L.OP_EXISTS, sub=sub, res=info["res"], list=kl, nlist=kn, list2=bl, nlist2=bn)
        probe_rows = max(getattr(node.rightChild, "tupleNum", 0), 1)
        op.sel = min(1.0, getattr(node, "tupleNum", probe_rows) / float(probe_rows))
        first = len(pipe.ops)
        saved_level = pipe.level
        saved = {a.id: pipe.att.get(a.id) for a in info["build_atts"]}
        pipe.level = lv
        for a, g in zip(info["build_atts"], gathers):
            pipe.att[a.id] = g
        try:
            v = self.expr(pipe, node.conditions)
            v = self.as_slot(pipe, v)
        finally:
            pipe.level = saved_level
            for aid, old in saved.items():
                if old is None:
                    pipe.att.pop(aid, None)
                else:
                    pipe.att[aid] = old
        for o in pipe.ops[first:]:
            if o["kind"] not in (L.OP_ARITH, L.OP_CMP, L.OP_LOGIC, L.OP_CAST, L.OP_SELECT):
                raise Unsupported("semi/anti join conditions of this form (%d)" % o["kind"])
        op["a"] = v
        op["imm"] = len(pipe.ops) - first

    # -- aggregation -------------------------------------------------------------
    RED = {"SUM": L.RED_SUM, "AVG": L.RED_SUM, "COUNT": L.RED_COUNT, "MIN": L.RED_MIN, "MAX": L.RED_MAX}

    def aggregate(self, node, pipe):
        groups = list(node.groupAttributes.values())
        if len(groups) > L.MAX_KEYS:
            raise Unsupported("more than %d grouping attributes" % L.MAX_KEYS)
        gtypes = [lang_type(g.dataType) for g in groups]
        # string group keys: their references, hashed and compared by their bytes
        aggs = [(id, inId, _tname(red)) for id, (inId, red) in node.aggregateTuples.items()]
        # one accumulator per distinct (reduction, input): an AVG shares the SUM
        # of its input with a SUM aggregate of the same attribute and divides by
        # the COUNT (one is added when the query has none)
        accs, acc_of = [], {}
        for id, inId, red in aggs:
            key = ("COUNT", None) if red == "COUNT" else (self.RED[red], inId)
            if key not in acc_of:
                acc_of[key] = len(accs)
                accs.append(key)
            acc_of[id] = acc_of[key]
        if any(r == "AVG" for _, _, r in aggs) and ("COUNT", None) not in acc_of:
            acc_of[("COUNT", None)] = len(accs)
            accs.append(("COUNT", None))
        if len(accs) > L.MAX_AGGS:
            raise Unsupported("more than %d aggregates" % L.MAX_AGGS)
        numgroups = max(int(getattr(node, "numgroups", 1)), 1)
        cap = max(2 * numgroups, 1024) if groups else 1
        reds = [L.RED_COUNT if k[0] == "COUNT" else k[0] for k in accs]
        rid = self.new_res(Res(L.RES_AGG, nkeys=len(groups), key_ctype=gtypes,
                               agg_red=reds, capacity=cap, group_hint=numgroups))
        kl, kn = pipe.list_([pipe.value_slot(g) for g in groups])
        inputs = []
        for red, inId in accs:
            if red == "COUNT":
                inputs.append(-1)
            else:
                a = node.aggregateInAttributes[inId]
                if lang_type(a.dataType) == "str":
                    raise Unsupported("aggregating strings")
                inputs.append(pipe.attr_slot(a))
        il, inn = pipe.list_(inputs)
        pipe.op(L.OP_AGG, res=rid, list=kl, nlist=kn, list2=il, nlist2=inn)
        self.finish(pipe)
        # the aggregation table becomes the source of the next pipeline
        out = Pipe(L.SRC_AGG, source_res=rid)
        for j, g in enumerate(groups):
            out.att[g.id] = out.slot(L.SLOT_AGGKEY, 0, gtypes[j], src=j, res=rid)
        acc_slot = [out.slot(L.SLOT_AGGVAL, 0, "i32" if red == "COUNT" else "u64", src=j, res=rid)
                    for j, (red, _) in enumerate(accs)]
        count_slot = acc_slot[acc_of[("COUNT", None)]] if ("COUNT", None) in acc_of else None
        for id, inId, red in aggs:
            if red == "AVG":
                d = out.reg("u64")
                out.op(L.OP_ARITH, sub=L.DIV, dst=d, a=acc_slot[acc_of[id]], b=count_slot, ctype=L.U64)
                out.att[id] = d
            else:
                out.att[id] = acc_slot[acc_of[id]]
        self.consume_parent(node, out)

    # -- materialisation ---------------------------------------------------------
    def materialize(self, node, pipe):
        atts = list(node.outRelation.values())
        types = [lang_type(a.dataType) for a in atts]
        temp = _tname(node.matType) == "TEMPTABLE"
        if "str" in types and temp:
            raise Unsupported("string attributes in temp tables")
        cap = max(int(getattr(node, "tupleNum", 0)), 1024)
        if type(node.child).__name__ == "Aggregation":
            cap = max(cap, self.res[pipe.source_res].capacity + 1)
        rid = self.new_res(Res(L.RES_OUTPUT, pay_ctype=types, capacity=cap,
                               name=node.table["name"] if temp else None,
                               columns=[a.id for a in atts]))
        sl, sn = pipe.list_([pipe.value_slot(a) for a in atts])
        pipe.op(L.OP_EMIT, res=rid, list=sl, nlist=sn)
        self.finish(pipe)
        if temp:
            self.temp[node.table["name"]] = rid
        else:
            self.result_res = rid
            self.result_names = [a.name for a in atts]
            self.result_types = [CT[t] for t in types]

    def finish(self, pipe):
        self.reorder_probes(pipe)
        self.pipes.append(pipe)

    def probe_cost(self, op):
        """Relative cost of one probe of a join table: 1 for a table that stays
        L2-resident (the runtime's 4x slots fit L2_TABLE_BYTES), 2 otherwise."""
        r = self.res[op["res"]]
        packed = "str" not in r.key_ctype and (r.nkeys <= 1 or (r.nkeys == 2 and all(t in NARROW for t in r.key_ctype)))
        words = 1 + len(r.pay_ctype) + (0 if packed else r.nkeys)
        return 1.0 if r.capacity * 4 * words * 8 <= L2_TABLE_BYTES else 2.0

    def reorder_probes(self, pipe):
        """Consecutive unique-key probes whose keys none of them produces are
        independent filters (inner, semi or anti; results do not depend on
        their order): ordered by cost / (1 - estimated pass rate), the cheap,
        selective ones first, so later probes see fewer rows.  The reference
        probes in plan order."""
        ops = pipe.ops
        i = 0
        while i < len(ops):
            if ops[i]["kind"] != L.OP_PROBE:
                i += 1
                continue
            j = i
            while j < len(ops) and ops[j]["kind"] == L.OP_PROBE:
                j += 1
            run = ops[i:j]
            if len(run) > 1:
                written = set()
                for o in run:
                    written.update(pipe.lists[o["list2"]:o["list2"] + o["nlist2"]])
                if all(not set(pipe.lists[o["list"]:o["list"] + o["nlist"]]) & written for o in run):
                    def rank(o):
                        sel = getattr(o, "sel", 1.0)
                        return self.probe_cost(o) / (1.0 - sel) if sel < 1.0 else float("inf")
                    ops[i:j] = sorted(run, key=rank)
            i = j

    # -- IR ----------------------------------------------------------------------
    def ir(self):
        """ctypes ``dq_plan_desc`` plus the objects that keep its memory alive."""
        keep = []
        res_arr = (L.dq_resource * max(len(self.res), 1))()
        for i, r in enumerate(self.res):
            d = res_arr[i]
            d.kind = r.kind
            d.nkeys = r.nkeys
            for j, t in enumerate(r.key_ctype):
                d.key_ctype[j] = CT[t]
            d.npay = len(r.pay_ctype)
            for j, t in enumerate(r.pay_ctype):
                d.pay_ctype[j] = CT[t] if isinstance(t, str) else t
            d.naggs = len(r.agg_red)
            for j, red in enumerate(r.agg_red):
                d.agg_red[j] = red
            d.capacity = r.capacity
            d.group_hint = r.group_hint
            if r.name:
                b = r.name.encode()
                keep.append(b)
                d.name = b
        pipe_arr = (L.dq_pipeline * len(self.pipes))()
        for i, p in enumerate(self.pipes):
            d = pipe_arr[i]
            d.source_kind = p.source_kind
            d.source_res = p.source_res
            if p.table:
                b = p.table.encode()
                keep.append(b)
                d.table = b
            if len(p.cols) > L.MAX_COLS:
                raise Unsupported("pipeline reads more than %d columns" % L.MAX_COLS)
            d.ncols = len(p.cols)
            for j, c in enumerate(p.cols):
                b = c.encode()
                keep.append(b)
                d.cols[j] = b
            d.nslots = len(p.slots)
            for j, s in enumerate(p.slots):
                ds = d.slots[j]
                ds.kind, ds.level, ds.ctype = s["kind"], s["level"], CT[s["ctype"]]
                ds.src, ds.res = s["src"], s["res"]
            d.nops = len(p.ops)
            for j, o in enumerate(p.ops):
                do = d.ops[j]
                for f in ("kind", "sub", "dst", "a", "b", "c", "ctype", "flags", "res", "list", "nlist",
                          "list2", "nlist2", "imm"):
                    setattr(do, f, o[f])
            d.nlist = len(p.lists)
            for j, v in enumerate(p.lists):
                d.lists[j] = v
            d.npatterns = len(p.patterns)
            for j, pat in enumerate(p.patterns):
                keep.append(pat)
                d.patterns[j] = pat
            d.compact = refill_point(p.ops, self.options.get("buffers"))
        desc = L.dq_plan_desc()
        desc.abi_version = L.ABI_VERSION
        desc.nres = len(self.res)
        desc.res = res_arr
        desc.npipes = len(self.pipes)
        desc.pipes = pipe_arr
        desc.result_res = self.result_res
        keep += [res_arr, pipe_arr]
        return desc, keep

    def describe(self):
        """Readable summary of the lowered plan (for logs and tests)."""
        lines = []
        for i, r in enumerate(self.res):
            lines.append("res %d kind=%d keys=%s pay=%s aggs=%s cap=%d" % (
                i, r.kind, r.key_ctype, r.pay_ctype, r.agg_red, r.capacity))
        for i, p in enumerate(self.pipes):
            lines.append("pipe %d src=%d table=%s cols=%s slots=%d ops=%s" % (
                i, p.source_kind, p.table, p.cols, len(p.slots), [o["kind"] for o in p.ops]))
        return "\n".join(lines)
