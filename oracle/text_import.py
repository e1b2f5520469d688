"""CPU oracle of the text import: a Python restatement of how the reference
loads a ``.tbl`` file.

TEST INFRASTRUCTURE.  Only ``tests/`` and the CPU baseline leg of ``bench.py``
may import this module, and only as the checker or the timed CPU baseline; the
product path never calls it.

The reference's importer (dogqc/dbio.py:117-253) reads each line with the CSV
reader it vendors (dogqc/include/csv.h, ``io::CSVReader<n + 1,
io::trim_chars<' '>, io::no_quote_escape<'|'>>``, dbio.py:97) and parses:

* lines end at '\\n'; a '\\r' before it is dropped (csv.h:478-480); a last line
  without '\\n' counts (csv.h:471-475);
* a line is split at every delimiter into exactly ``n + 1`` columns, the last
  one (after the terminal delimiter) read into an unused ``char*``; fewer or
  more columns are errors (csv.h:846-866);
* each column is trimmed of spaces (csv.h:673-692);
* INT: ``parse_signed_integer`` into ``int`` with overflow an error
  (csv.h:945-995); an empty column is 0;
* CHAR: exactly one byte (csv.h:920-928);
* FLOAT: ``parse_float`` into ``float`` (the importer's decimal type is FP32,
  dbio.py:142), each step rounded to binary32 (csv.h:1008-1069);
* DATE: the schema's ``toDate`` over bytes 0-3, 5-6, 8-9
  (query/schema/tpch.py:9-20), stored as ``unsigned`` (codegen.py:39);
* STRING: the trimmed bytes, into offsets and a heap (dbio.py:226-251).

``parse`` returns the columns, or raises ``TextImportError`` for the first bad
line.  Kinds follow the library's ``dq_text_kind`` numbering; DECIMAL (exact
fixed point, the library's own kind) is the float grammar without exponent,
scaled by 10^scale with further digits dropped.
"""
import numpy as np

INT, DATE, CHAR, DECIMAL, STRING, SKIP, FLOAT = 1, 2, 3, 4, 5, 6, 7
TOO_FEW, TOO_MANY, NO_DIGIT, OVERFLOW, NOT_CHAR, SHORT_DATE, EXPONENT = 1, 2, 3, 4, 5, 6, 7
I32_MIN, I32_MAX, I64_MAX = -2 ** 31, 2 ** 31 - 1, 2 ** 63 - 1


class TextImportError(ValueError):
    def __init__(self, line, field, reason):
        ValueError.__init__(self, "line %d field %d: reason %d" % (line, field, reason))
        self.line, self.field, self.reason = line, field, reason


class _Bad(Exception):
    def __init__(self, reason):
        Exception.__init__(self, reason)
        self.reason = reason


def lines_of(text):
    """The lines of ``text`` (bytes) as the reference's line reader yields them."""
    if not text:
        return []
    parts = text.split(b"\n")
    if parts[-1] == b"":
        parts.pop()
    return [p[:-1] if p.endswith(b"\r") else p for p in parts]


def _int(s):
    """csv.h parse_signed_integer for int, throw_on_overflow."""
    neg = s[:1] == b"-"
    if s[:1] in (b"-", b"+"):
        s = s[1:]
    x = 0
    for c in s:
        if not 48 <= c <= 57:
            raise _Bad(NO_DIGIT)
        y = c - 48
        if neg:
            # C++ integer division truncates toward zero
            if x < -((-(I32_MIN + y)) // 10):
                raise _Bad(OVERFLOW)
            x = 10 * x - y
        else:
            if x > (I32_MAX - y) // 10:
                raise _Bad(OVERFLOW)
            x = 10 * x + y
    return x


def _float32(s):
    """csv.h parse_float for float: the IEEE binary32 bits it produces.
    Exponents beyond four digits are rejected, as the library does."""
    with np.errstate(over="ignore", under="ignore"):
        return _float32_steps(s)


def _float32_steps(s):
    f32 = np.float32
    neg = False
    i = 0
    if s[:1] in (b"-", b"+"):
        neg = s[:1] == b"-"
        i = 1
    x = f32(0)
    while i < len(s) and 48 <= s[i] <= 57:
        x = f32(f32(x * f32(10)) + f32(s[i] - 48))
        i += 1
    if i < len(s) and s[i] in b".,":
        i += 1
        pos = f32(1)
        while i < len(s) and 48 <= s[i] <= 57:
            pos = f32(pos / f32(10))
            x = f32(x + f32(f32(s[i] - 48) * pos))
            i += 1
    if i < len(s) and s[i] in b"eE":
        rest = s[i + 1:]
        eneg = rest[:1] == b"-"
        if rest[:1] in (b"-", b"+"):
            rest = rest[1:]
        e = 0
        for c in rest:
            if not 48 <= c <= 57:
                raise _Bad(NO_DIGIT)
            e = e * 10 + c - 48
            if e > 9999:
                raise _Bad(EXPONENT)
        if eneg:
            e = -e
        if e != 0:
            base = f32(0.1) if e < 0 else f32(10)
            e = abs(e)
            while e != 1:
                if e & 1 == 0:
                    base = f32(base * base)
                    e >>= 1
                else:
                    x = f32(x * base)
                    e -= 1
            x = f32(x * base)
    elif i != len(s):
        raise _Bad(NO_DIGIT)
    if neg:
        x = f32(-x)
    return int(np.array([x], np.float32).view(np.uint32)[0])


def _decimal(s, scale):
    neg = s[:1] == b"-"
    if s[:1] in (b"-", b"+"):
        s = s[1:]
    m, fd, frac = 0, 0, False
    for c in s:
        if c in b".," and not frac:
            frac = True
            continue
        if c in b"eE":
            raise _Bad(EXPONENT)
        if not 48 <= c <= 57:
            raise _Bad(NO_DIGIT)
        if frac:
            if fd >= scale:
                continue
            fd += 1
        m = 10 * m + c - 48
        if m > I64_MAX:
            raise _Bad(OVERFLOW)
    m *= 10 ** (scale - fd)
    if m > I64_MAX:
        raise _Bad(OVERFLOW)
    return -m if neg else m


def _date(s):
    if len(s) < 10:
        raise _Bad(SHORT_DATE)
    w = (10000000, 1000000, 100000, 10000, 0, 1000, 100, 0, 10, 1)
    return sum((s[k] - 48) * w[k] for k in range(10)) & 0xFFFFFFFF


def parse(text, fields, delim=b"|"):
    """{column: values} for ``fields`` [(name, kind[, scale])]; FLOAT values are
    the uint32 bits, CHAR values signed bytes, STRING values bytes."""
    out = {f[0]: [] for f in fields if f[1] != SKIP}
    n = len(fields)
    for ln, line in enumerate(lines_of(text)):
        cols = line.split(delim)
        # the line is split before any value is parsed (csv.h:846-866)
        if len(cols) < n + 1:
            raise TextImportError(ln + 1, len(cols) - 1, TOO_FEW)
        if len(cols) > n + 1:
            raise TextImportError(ln + 1, n, TOO_MANY)
        for f, fd in enumerate(fields):
            s = cols[f].strip(b" ")
            kind = fd[1]
            try:
                if kind == INT:
                    v = _int(s)
                elif kind == FLOAT:
                    v = _float32(s)
                elif kind == DECIMAL:
                    v = _decimal(s, fd[2] if len(fd) > 2 else 0)
                elif kind == DATE:
                    v = _date(s)
                elif kind == CHAR:
                    if len(s) != 1:
                        raise _Bad(NOT_CHAR)
                    v = s[0] - 256 if s[0] > 127 else s[0]
                elif kind == STRING:
                    v = s
                else:
                    continue
            except _Bad as b:
                raise TextImportError(ln + 1, f, b.reason)
            out[fd[0]].append(v)
    return out
