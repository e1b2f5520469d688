"""CPU oracle: a numpy restatement of the reference's plan semantics.

TEST INFRASTRUCTURE.  Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU
baseline leg of ``bench.py`` may import this module, and only as the checker or
the timed CPU baseline; the product path never calls it.

It evaluates a *resolved* plan tree (this package's front end or the reference's
own ``dogqc.relationalAlgebra`` classes; dispatch is by class name) over a
``dogqc_b200.database.Database`` and returns the result table.  It is written
from the operator semantics, not from the reference's generated code:

* Selection keeps rows whose condition is non-zero (cudaTranslator.py:353-366).
* Map stores the expression, evaluated with C++ integer semantics (integer
  promotion, usual arithmetic conversions, two's-complement wrap-around), into
  a register of the attribute's C type (codegen.py:37-45, cudaTranslator.py:402-422).
* Inner equi-join returns every (build, probe) pair with equal keys
  (hashJoins.py:465-534); with ``multimatch=False`` one build row per probe row
  (hashJoins.py:113-153 stops at the first match; the first build row in build
  order is taken here).  Semi/anti keep probe rows with / without a match that
  also satisfies the extra conditions (hashJoins.py:183-211, 244-276).
* Aggregation (cudaTranslator.py:431-525, hashTableUtil.py:118-137): SUM/AVG/MIN/MAX
  accumulate ``(unsigned long long)value`` (wrapping sum, unsigned min/max with
  initial values ULLONG_MAX / 0), COUNT is a wrapping ``int``, AVG = sum / count
  in ``unsigned long long``; without grouping exactly one row is produced.
* LIKE follows the reference's matcher (util.cuh:144-199) including its quirks.

Large inputs are streamed in chunks so that joins with large fan-out (hundreds
of millions of pairs) run in bounded memory.
"""
import numpy as np

CHUNK = 1 << 22
PAIR_CHUNK = 1 << 24

# --------------------------------------------------------------------- types --

# C value types: i8 (char), i32 (int), u32 (unsigned), i64 (long), u64 (ULL)
NP = {"i8": np.int8, "i32": np.int32, "u32": np.uint32, "i64": np.int64, "u64": np.uint64}

LANG = {"INT": "i32", "DATE": "u32", "CHAR": "i8", "FLOAT": "u64", "DOUBLE": "u64"}


def tname(t):
    return t.name if hasattr(t, "name") else str(t)


def lang_type(relational_type):
    n = tname(relational_type)
    if n == "STRING":
        return "str"
    if n not in LANG:
        raise NotImplementedError("no C type for %s" % n)
    return LANG[n]


def promote(t):
    return "i32" if t == "i8" else t


def common(a, b):
    a, b = promote(a), promote(b)
    if "u64" in (a, b):
        return "u64"
    if "i64" in (a, b):
        return "i64"
    if "u32" in (a, b):
        return "u32"
    return "i32"


def conv(v, t):
    return np.asarray(v).astype(NP[t], copy=False)


class Strs(object):
    """String values as (heap, start, end) triples."""

    def __init__(self, heap, start, end):
        self.heap = heap
        self.start = np.asarray(start, dtype=np.int64)
        self.end = np.asarray(end, dtype=np.int64)

    def __len__(self):
        return len(self.start)

    def take(self, idx):
        return Strs(self.heap, self.start[idx], self.end[idx])

    def get(self, i):
        return bytes(self.heap[self.start[i]:self.end[i]])

    def fixed_matrix(self):
        lens = self.end - self.start
        if len(lens) == 0 or not np.all(lens == lens[0]):
            return None
        L = int(lens[0])
        return self.heap[self.start[:, None] + np.arange(L)[None, :]]


def concat_values(parts):
    if isinstance(parts[0], Strs):
        return Strs(parts[0].heap, np.concatenate([p.start for p in parts]),
                    np.concatenate([p.end for p in parts]))
    return np.concatenate(parts)


def take(col, idx):
    return col.take(idx) if isinstance(col, Strs) else col[idx]


# ---------------------------------------------------------------------- LIKE --

def like_check(s, p):
    """The reference's LIKE matcher (util.cuh:144-199) restated over bytes.

    Wildcards ``%`` and ``_``; prefix and suffix are matched first, then the
    infixes left to right.  Reads one past the end of the string or pattern read
    a zero byte, as the reference's NUL-terminated constant does.
    """
    ls, lp = len(s), len(p)

    def S(i):
        return s[i] if 0 <= i < ls else 0

    def P(i):
        return p[i] if 0 <= i < lp else 0

    def cmp(c, l):
        return c == l or l == 0x5F

    PCT = 0x25
    l_in_start, l_in_end = 0, lp
    s_in_start, s_in_end = 0, ls
    l_pos = 0
    if P(0) != PCT:
        s_pos, l_pos = 0, 0
        while l_pos < lp and s_pos < ls and P(l_pos) != PCT:
            if not cmp(S(s_pos), P(l_pos)):
                return False
            l_pos += 1
            s_pos += 1
        l_in_start, s_in_start = l_pos, s_pos
    if P(lp - 1) != PCT:
        s_pos, l_pos = ls - 1, lp - 1
        while l_pos >= 0 and s_pos >= 0 and P(l_pos) != PCT:
            if not cmp(S(s_pos), P(l_pos)):
                return False
            l_pos -= 1
            s_pos -= 1
        l_in_end, s_in_end = l_pos, s_pos + 1
    if l_in_start < l_in_end:
        l_pos = l_in_start + 1
        s_pos = s_in_start
        while s_pos < s_in_end and l_pos < l_in_end:
            l_tr, s_tr = l_pos, s_pos
            while cmp(S(s_tr), P(l_tr)) and s_tr < s_in_end:
                l_tr += 1
                if P(l_tr) == PCT:
                    l_tr += 1
                    l_pos = l_tr
                    s_pos = s_tr
                    break
                s_tr += 1
            s_pos += 1
    return l_pos >= l_in_end


def like_column(strs, pattern):
    pat = pattern.encode() if isinstance(pattern, str) else bytes(pattern)
    lit = pat[1:-1]
    simple = (len(pat) >= 3 and pat[0] == 0x25 and pat[-1] == 0x25
              and b"%" not in lit and b"_" not in lit)
    mat = strs.fixed_matrix() if simple else None
    if mat is not None:
        n, L = mat.shape
        k = len(lit)
        out = np.zeros(n, dtype=bool)
        lit_a = np.frombuffer(lit, dtype=np.uint8)
        for off in range(0, L - k + 1):
            out |= np.all(mat[:, off:off + k] == lit_a[None, :], axis=1)
        return out
    return np.array([like_check(strs.get(i), pat) for i in range(len(strs))], dtype=bool)


# --------------------------------------------------------------- expressions --

def const_value(e):
    t = tname(e.type)
    tok = e.token
    if t == "STRING":
        return tok.encode() if isinstance(tok, str) else bytes(tok), "strconst"
    if t == "CHAR":
        return np.int8(ord(tok[0])), "i8"
    if t == "FLOAT":
        raise NotImplementedError("FLOAT constants are not exact; use INT constants")
    try:
        v = int(tok)
    except ValueError:
        raise NotImplementedError("non-integer constant %r is not exact" % tok)
    if -(1 << 31) <= v < (1 << 31):
        return np.int32(v), "i32"
    return np.int64(v), "i64"


def c_div(a, b, t):
    a = conv(a, t)
    b = conv(b, t)
    zero = b == 0
    bs = np.where(zero, 1, b).astype(NP[t])
    if t.startswith("u"):
        q = a // bs
    else:
        q = np.abs(a.astype(np.int64)) // np.abs(bs.astype(np.int64))
        q = np.where((a < 0) != (bs < 0), -q, q).astype(NP[t])
    return np.where(zero, 0, q).astype(NP[t])


def c_mod(a, b, t):
    q = c_div(a, b, t)
    a = conv(a, t)
    b = conv(b, t)
    r = (a - q * b).astype(NP[t])
    return np.where(b == 0, 0, r).astype(NP[t])


CMP = {"EqualsExpr": np.equal, "SmallerExpr": np.less, "SmallerEqualExpr": np.less_equal,
       "LargerExpr": np.greater, "LargerEqualExpr": np.greater_equal}


def evaluate(e, frame, n):
    """Value of scalar expression ``e`` over ``frame``: (array-or-Strs, C type)."""
    k = type(e).__name__
    if k == "AttrExpr":
        col = frame[e.attr.id]
        if isinstance(col, Strs):
            return col, "str"
        return col, lang_type(e.attr.dataType)
    if k == "ConstExpr":
        v, t = const_value(e)
        if t == "strconst":
            return v, t
        return np.full(n, v, dtype=NP[t]), t
    if k in ("AddExpr", "SubExpr", "MulExpr", "DivExpr"):
        a, ta = evaluate(e.leftChild, frame, n)
        b, tb = evaluate(e.rightChild, frame, n)
        t = common(ta, tb)
        with np.errstate(over="ignore"):
            if k == "AddExpr":
                return (conv(a, t) + conv(b, t)).astype(NP[t]), t
            if k == "SubExpr":
                return (conv(a, t) - conv(b, t)).astype(NP[t]), t
            if k == "MulExpr":
                return (conv(a, t) * conv(b, t)).astype(NP[t]), t
            return c_div(a, b, t), t
    if k in CMP:
        a, ta = evaluate(e.leftChild, frame, n)
        b, tb = evaluate(e.rightChild, frame, n)
        if ta in ("str", "strconst") or tb in ("str", "strconst"):
            if k != "EqualsExpr":
                raise NotImplementedError("ordering comparison on strings")
            return string_equals(a, ta, b, tb, n).astype(np.int32), "i32"
        t = common(ta, tb)
        return CMP[k](conv(a, t), conv(b, t)).astype(np.int32), "i32"
    if k == "AndExpr":
        a, _ = evaluate(e.leftChild, frame, n)
        b, _ = evaluate(e.rightChild, frame, n)
        return ((a != 0) & (b != 0)).astype(np.int32), "i32"
    if k == "OrExpr":
        a, _ = evaluate(e.leftChild, frame, n)
        b, _ = evaluate(e.rightChild, frame, n)
        return ((a != 0) | (b != 0)).astype(np.int32), "i32"
    if k == "NotExpr":
        a, _ = evaluate(e.child, frame, n)
        return (a == 0).astype(np.int32), "i32"
    if k == "LikeExpr":
        s, ts = evaluate(e.leftChild, frame, n)
        p, tp = evaluate(e.rightChild, frame, n)
        if ts != "str" or tp != "strconst":
            raise NotImplementedError("LIKE needs a string attribute and a constant pattern")
        return like_column(s, p).astype(np.int32), "i32"
    if k == "ExtractExpr":
        a, ta = evaluate(e.child, frame, n)
        t = common(ta, "i32")
        ext = tname(e.extract)
        if ext == "YEAR":
            return c_div(a, np.int32(10000), t), t
        if ext == "DAY":
            return c_mod(a, np.int32(100), t), t
        return c_mod(c_div(a, np.int32(100), t), np.int32(100), t), t
    if k == "CaseExpr":
        out = np.zeros(n, dtype=np.uint64)
        done = np.zeros(n, dtype=bool)
        for w, th in e.exprListWhenThen:
            c, _ = evaluate(w, frame, n)
            v, _ = evaluate(th, frame, n)
            hit = (c != 0) & ~done
            out = np.where(hit, conv(v, "u64"), out)
            done |= hit
        if e.exprElse is not None:
            v, _ = evaluate(e.exprElse, frame, n)
            out = np.where(done, out, conv(v, "u64"))
        return out, "u64"
    if k == "SubstringExpr":
        s, ts = evaluate(e.exprString, frame, n)
        f, _ = evaluate(e.exprFrom, frame, n)
        c, _ = evaluate(e.exprFor, frame, n)
        start = s.start + f.astype(np.int64) - 1
        end = start + c.astype(np.int64)
        start = np.maximum(start, s.start)
        end = np.minimum(end, s.end)
        # a window that starts past the string's end (or a negative length)
        # gives the reference a string of negative length, equal to nothing
        # and hashed over no bytes; here it is the empty string
        start = np.minimum(start, s.end)
        end = np.maximum(end, start)
        return Strs(s.heap, start, end), "str"
    raise NotImplementedError("scalar expression %s" % k)


def string_equals(a, ta, b, tb, n):
    if ta == "strconst" and tb == "strconst":
        return np.full(n, a == b)
    if ta == "strconst":
        a, ta, b, tb = b, tb, a, ta
    if tb == "strconst":
        lens = a.end - a.start
        out = lens == len(b)
        idx = np.nonzero(out)[0]
        if len(b) and len(idx):
            lit = np.frombuffer(b, dtype=np.uint8)
            mat = a.heap[a.start[idx][:, None] + np.arange(len(b))[None, :]]
            out[idx] = np.all(mat == lit[None, :], axis=1)
        return out
    return np.array([a.get(i) == b.get(i) for i in range(n)], dtype=bool)


# ------------------------------------------------------------------- frames --

class Frame(object):
    def __init__(self, cols, n):
        self.cols = cols
        self.n = n

    def __getitem__(self, k):
        return self.cols[k]

    def take(self, idx):
        return Frame({k: take(v, idx) for k, v in self.cols.items()}, len(idx))


def concat_frames(frames, ids):
    frames = [f for f in frames if f.n]
    if not frames:
        return None
    return Frame({i: concat_values([f.cols[i] for f in frames]) for i in ids}, sum(f.n for f in frames))


def store(values, ctype, target):
    """Assign a computed C value to a register of C type ``target``."""
    if target == "str":
        return values
    return conv(values, target)


class Oracle(object):
    """Evaluates resolved plans.  ``run(plan)`` returns ``(names, rows)``."""

    def __init__(self, db):
        self.db = db
        self.temps = {}
        self._string_ids = {}

    def run(self, plan):
        out = None
        for root in plan if isinstance(plan, list) else [plan]:
            out = self.materialize(root)
        return out

    # -- streaming ------------------------------------------------------------
    def stream(self, node):
        k = type(node).__name__
        if k == "Scan":
            yield from self.scan(node)
        elif k == "Selection":
            for f in self.stream(node.child):
                c, _ = evaluate(node.condition, f, f.n)
                keep = np.nonzero(c != 0)[0]
                yield f.take(keep)
        elif k == "Map":
            for f in self.stream(node.child):
                v, t = evaluate(node.expression, f, f.n)
                f.cols[node.mapAttr.id] = store(v, t, lang_type(node.mapAttr.dataType))
                yield f
        elif k == "Projection":
            yield from self.stream(node.child)
        elif k == "EquiJoin":
            yield from self.equijoin(node)
        elif k == "CrossJoin":
            yield from self.crossjoin(node)
        elif k == "Aggregation":
            yield self.aggregate(node)
        elif k == "Materialize":
            yield from self.stream(node.child)
        else:
            raise NotImplementedError(k)

    def scan(self, node):
        if node.isTempScan:
            src = self.temps[node.table["name"]]
            cols = {id: src[a.sourceId] for id, a in node.outRelation.items()}
            n = len(next(iter(src.values()))) if src else 0
            yield Frame(cols, n)
            return
        table = self.db[node.table["name"]]
        n = table.size
        needed = {}
        for id, a in node.outRelation.items():
            needed[id] = table.columns[a.name]
        for lo in range(0, max(n, 1), CHUNK):
            hi = min(n, lo + CHUNK)
            cols = {}
            for id, col in needed.items():
                if hasattr(col, "offsets"):
                    off = col.offsets.astype(np.int64)
                    cols[id] = Strs(col.chars, off[lo:hi], off[lo + 1:hi + 1])
                else:
                    cols[id] = col[lo:hi]
            yield Frame(cols, hi - lo)

    def collect(self, node):
        ids = list(node.outRelation.keys())
        frames = list(self.stream(node))
        f = concat_frames(frames, ids)
        if f is None:
            f = Frame({i: np.zeros(0, dtype=np.uint64) for i in ids}, 0)
            for i, a in node.outRelation.items():
                lt = lang_type(a.dataType)
                f.cols[i] = Strs(np.zeros(0, np.uint8), [], []) if lt == "str" else np.zeros(0, NP[lt])
        return f

    # -- joins ----------------------------------------------------------------
    def _keys(self, frame, atts_a, atts_b):
        """Keys of frame for attributes ``atts_a`` compared against ``atts_b``.
        A string key becomes the number of its bytes in a dictionary shared
        by both sides of every join (the reference hashes and compares the
        bytes, hashTableUtil.py:15-35)."""
        cols = []
        for a, b in zip(atts_a, atts_b):
            ta, tb = lang_type(a.dataType), lang_type(b.dataType)
            v = frame[a.id]
            if ta == "str" or tb == "str":
                if ta != tb:
                    raise NotImplementedError("join keys comparing a string with a number")
                cols.append(self._string_key_ids(v))
                continue
            cols.append(conv(v, common(ta, tb)).astype(np.uint64).view(np.int64))
        return cols

    def _string_key_ids(self, v):
        """Dictionary numbers of the strings of ``v``: the distinct byte strings
        are found over a zero-padded matrix (with the length as a last column),
        then numbered through the shared dictionary."""
        n = len(v)
        if n == 0:
            return np.zeros(0, dtype=np.int64)
        lens = v.end - v.start
        width = int(lens.max())
        pos = v.start[:, None] + np.arange(max(width, 1))[None, :]
        inside = np.arange(max(width, 1))[None, :] < lens[:, None]
        mat = np.where(inside, v.heap[np.minimum(pos, max(len(v.heap) - 1, 0))] if len(v.heap) else 0, 0)
        mat = np.concatenate([mat.astype(np.int64), lens[:, None].astype(np.int64)], axis=1)
        uniq, inv = np.unique(mat, axis=0, return_inverse=True)
        ids = self._string_ids
        local = np.array([ids.setdefault(bytes(u[:u[-1]].astype(np.uint8)), len(ids)) for u in uniq], dtype=np.int64)
        return local[inv.reshape(-1)]

    def equijoin(self, node):
        jt = tname(node.joinType)
        if jt == "OUTER":
            # The reference runs an outer join only on its multimatch hash table
            # (its unique table rejects the join type, hashJoins.py:95-109).
            # After a probe row's matches, the generated loop gives an unmatched
            # row one more iteration (hashJoins.py:524-530), but that iteration
            # runs the key check again on the payload at the row's offset
            # (hashJoins.py:505-510; hashProbeMulti leaves the offset at 0 or at
            # the range end, include/hashing.cuh:189-199), which fails: unmatched
            # rows are dropped, matched rows have no nulls.  The result is the
            # inner join's.
            if not getattr(node, "multimatch", True):
                raise NotImplementedError("outer join on a unique hash table")
            jt = "INNER"
        if jt not in ("INNER", "SEMI", "ANTI"):
            raise NotImplementedError("join type %s" % jt)
        bk = list(node.buildKeyAttributes.values())
        pk = list(node.probeKeyAttributes.values())
        build = self.collect(node.leftChild)
        bkeys = self._keys(build, bk, pk)
        for probe in self.stream(node.rightChild):
            pkeys = self._keys(probe, pk, bk)
            yield from self._join_chunk(node, jt, build, bkeys, probe, pkeys)

    def _join_chunk(self, node, jt, build, bkeys, probe, pkeys):
        if len(bkeys) == 1:
            bkey, pkey = bkeys[0], pkeys[0]
        else:
            allk = np.stack([np.concatenate([b, p]) for b, p in zip(bkeys, pkeys)], axis=1)
            _, inv = np.unique(allk, axis=0, return_inverse=True)
            inv = inv.reshape(-1)
            bkey, pkey = inv[:build.n], inv[build.n:]
        order = np.argsort(bkey, kind="stable")
        sk = bkey[order]
        lo = np.searchsorted(sk, pkey, "left")
        hi = np.searchsorted(sk, pkey, "right")
        cnt = (hi - lo).astype(np.int64)
        multi = bool(getattr(node, "multimatch", True))
        if jt == "INNER" and not multi:
            cnt = np.minimum(cnt, 1)
        if jt in ("SEMI", "ANTI") and node.conditions is None:
            keep = (cnt > 0) if jt == "SEMI" else (cnt == 0)
            yield probe.take(np.nonzero(keep)[0])
            return
        # expand pairs in bounded chunks of probe rows
        csum = np.cumsum(cnt)
        start = 0
        found = np.zeros(probe.n, dtype=bool)
        while start < probe.n:
            base = csum[start - 1] if start else 0
            stop = int(np.searchsorted(csum, base + PAIR_CHUNK, "right"))
            stop = max(stop, start + 1)
            stop = min(stop, probe.n)
            c = cnt[start:stop]
            total = int(c.sum())
            if total:
                pidx = np.repeat(np.arange(start, stop), c)
                first = np.repeat(np.cumsum(c) - c, c)
                bpos = lo[pidx] + (np.arange(total) - first)
                bidx = order[bpos]
                cols = {}
                for id in build.cols:
                    cols[id] = take(build.cols[id], bidx)
                for id in probe.cols:
                    cols[id] = take(probe.cols[id], pidx)
                pairs = Frame(cols, total)
                if jt == "INNER":
                    if node.conditions is not None:
                        cv, _ = evaluate(node.conditions, pairs, total)
                        pairs = pairs.take(np.nonzero(cv != 0)[0])
                    yield pairs
                else:
                    cv, _ = evaluate(node.conditions, pairs, total)
                    found[pidx[cv != 0]] = True
            start = stop
        if jt in ("SEMI", "ANTI"):
            keep = found if jt == "SEMI" else ~found
            yield probe.take(np.nonzero(keep)[0])

    def crossjoin(self, node):
        """Nested-loop join: every (inner, outer) pair that satisfies the
        condition; the inner side is the left child, materialised, the outer
        side streams (cudaTranslator.py:369-397)."""
        left = self.collect(node.leftChild)
        for right in self.stream(node.rightChild):
            total = left.n * right.n
            if total == 0:
                continue
            lidx = np.tile(np.arange(left.n), right.n)
            ridx = np.repeat(np.arange(right.n), left.n)
            cols = {id: take(v, lidx) for id, v in left.cols.items()}
            cols.update({id: take(v, ridx) for id, v in right.cols.items()})
            f = Frame(cols, total)
            cv, _ = evaluate(node.condition, f, total)
            yield f.take(np.nonzero(cv != 0)[0])

    # -- aggregation ----------------------------------------------------------
    def aggregate(self, node):
        groups = list(node.groupAttributes.values())
        aggs = [(id, inId, tname(red)) for id, (inId, red) in node.aggregateTuples.items()]
        partial_keys, partial_vals = [], []
        # string keys: each distinct byte string gets a code (first seen, first code)
        codes, strs_of = {}, []

        def key_values(g, v):
            if lang_type(g.dataType) != "str":
                return conv(v, lang_type(g.dataType))
            out = np.empty(len(v), np.int64)
            for i in range(len(v)):
                b = v.get(i)
                if b not in codes:
                    codes[b] = len(strs_of)
                    strs_of.append(b)
                out[i] = codes[b]
            return out
        for f in self.stream(node.child):
            if f.n == 0:
                continue
            keys = [key_values(g, f[g.id]) for g in groups]
            if groups:
                stacked = np.stack([k.astype(np.int64) for k in keys], axis=1)
                uniq, inv = np.unique(stacked, axis=0, return_inverse=True)
                inv = inv.reshape(-1)
            else:
                uniq, inv = np.zeros((1, 0), np.int64), np.zeros(f.n, np.int64)
            order = np.argsort(inv, kind="stable")
            bounds = np.concatenate([[0], np.nonzero(np.diff(inv[order]))[0] + 1])
            vals = {}
            for id, inId, red in aggs:
                if red == "COUNT":
                    vals[id] = np.add.reduceat(np.ones(f.n, np.int64)[order], bounds)
                    continue
                v = conv(f[inId], "u64")[order]
                if red in ("SUM", "AVG"):
                    vals[id] = np.add.reduceat(v, bounds).astype(np.uint64)
                elif red == "MIN":
                    vals[id] = np.minimum.reduceat(v, bounds)
                elif red == "MAX":
                    vals[id] = np.maximum.reduceat(v, bounds)
            partial_keys.append(uniq)
            partial_vals.append(vals)
        cols = {}
        if partial_keys:
            allk = np.concatenate(partial_keys, axis=0)
            if groups:
                uniq, inv = np.unique(allk, axis=0, return_inverse=True)
                inv = inv.reshape(-1)
            else:
                uniq, inv = np.zeros((1, 0), np.int64), np.zeros(len(allk), np.int64)
            order = np.argsort(inv, kind="stable")
            bounds = np.concatenate([[0], np.nonzero(np.diff(inv[order]))[0] + 1])
            ng = len(uniq)
            for id, inId, red in aggs:
                v = np.concatenate([p[id] for p in partial_vals])[order]
                if red == "COUNT":
                    cols[id] = np.add.reduceat(v, bounds).astype(np.int64).astype(np.int32)
                elif red in ("SUM", "AVG"):
                    cols[id] = np.add.reduceat(v, bounds).astype(np.uint64)
                elif red == "MIN":
                    cols[id] = np.minimum.reduceat(v, bounds)
                else:
                    cols[id] = np.maximum.reduceat(v, bounds)
        else:
            ng = 0 if groups else 1
            uniq = np.zeros((ng, len(groups)), np.int64)
            for id, inId, red in aggs:
                if red == "COUNT":
                    cols[id] = np.zeros(ng, np.int32)
                elif red == "MIN":
                    cols[id] = np.full(ng, np.iinfo(np.uint64).max, np.uint64)
                else:
                    cols[id] = np.zeros(ng, np.uint64)
        for j, g in enumerate(groups):
            if lang_type(g.dataType) == "str":
                vals = [strs_of[int(c)] for c in uniq[:, j]]
                heap = np.frombuffer(b"".join(vals), np.uint8) if vals else np.zeros(0, np.uint8)
                ends = np.cumsum([len(b) for b in vals]).astype(np.int64) if vals else np.zeros(0, np.int64)
                cols[g.id] = Strs(heap, ends - np.array([len(b) for b in vals], np.int64), ends)
            else:
                cols[g.id] = uniq[:, j].astype(NP[lang_type(g.dataType)])
        count_id = node.countAttr.id if hasattr(node, "countAttr") else None
        for id in node.avgAggregates:
            cnt = cols[count_id].astype(np.int64).astype(np.uint64)
            cols[id] = np.where(cnt == 0, 0, cols[id] // np.where(cnt == 0, 1, cnt)).astype(np.uint64)
        return Frame(cols, ng)

    # -- materialization ------------------------------------------------------
    def materialize(self, node):
        f = self.collect(node.child) if type(node).__name__ == "Materialize" else self.collect(node)
        out = node.outRelation
        if type(node).__name__ == "Materialize" and tname(node.matType) == "TEMPTABLE":
            self.temps[node.table["name"]] = {id: f[id] for id in out}
            return None
        names = [a.name for a in out.values()]
        columns = []
        for id, a in out.items():
            v = f[id]
            if isinstance(v, Strs):
                columns.append([v.get(i) for i in range(len(v))])
            else:
                columns.append(v)
        rows = list(zip(*[c.tolist() if hasattr(c, "tolist") else c for c in columns])) if f.n else []
        return names, rows


def run_plan(db, plan):
    """Evaluate a resolved plan; returns (column names, list of row tuples)."""
    return Oracle(db).run(plan)
