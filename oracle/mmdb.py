"""Reference column-file format and result-file parser (test infrastructure).

Only the oracle recipe uses this module; the product never reads or writes these
files.

Column files: the reference's generated ``main()`` maps ``mmdb/<table>_<attr>``
with ``map_memory_file`` (dogqc/include/mappedmalloc.h:69-82): an 8-byte
little-endian total mapping size, then the raw array.  Strings are two files,
``<table>_<attr>_offset`` (``size_t[n+1]``) and ``<table>_<attr>_char``
(dogqc/cudaTranslator.py:138-166, 263-269).

Result file: ``queryresult.csv`` as written by the reference's
``MaterializeTranslator.consumePrintToFile`` (dogqc/cudaTranslator.py:645-668):
a header of ``name, `` items, then one line per row with every value followed by
two spaces (``%8i``, ``%10llu``, ``%10i`` or ``%c``; dogqc/cudalang.py:124-131).
"""
import os

import numpy as np

from dogqc_b200.database import StringColumn


def _write(path, arr):
    data = np.ascontiguousarray(arr).tobytes()
    with open(path, "wb") as f:
        f.write(np.uint64(8 + len(data) + 1).tobytes())
        f.write(data)
        f.write(b"\0")


def write_mmdb(db, path):
    os.makedirs(path, exist_ok=True)
    for tname, table in db.tables.items():
        for attr, col in table.columns.items():
            base = os.path.join(path, "%s_%s" % (tname, attr))
            if isinstance(col, StringColumn):
                _write(base + "_offset", col.offsets.astype(np.uint64))
                _write(base + "_char", col.chars)
            else:
                _write(base, col)


STRING_FIELD = 10  # stringPrint's default width (dogqc/include/util.h:18-30)


def render_string(b):
    """A string as the reference's result file shows it: right-aligned in 10
    characters, cut to its first 10 (stringPrint, dogqc/include/util.h:18-30)."""
    s = b.decode("latin-1") if isinstance(b, (bytes, bytearray)) else b
    return (" " * max(0, STRING_FIELD - len(s)) + s)[:STRING_FIELD]


def _parse_typed(line, ncols, str_cols):
    """One result line whose string columns are fixed 10-character fields with
    no separator after them; every other value is followed by two spaces."""
    row, i = [], 0
    for j in range(ncols):
        if j in str_cols:
            row.append(line[i:i + STRING_FIELD])
            i += STRING_FIELD
            continue
        while i < len(line) and line[i] == " ":
            i += 1
        k = i
        while k < len(line) and line[k] != " ":
            k += 1
        t = line[i:k]
        row.append(ord(t) if len(t) == 1 and not t.isdigit() and t != "-" else int(t))
        i = k + 2
    return tuple(row)


def parse_result(path, str_cols=()):
    """Return (column names, list of row tuples) from a reference result file:
    ints, and for the columns in ``str_cols`` the 10-character string fields."""
    with open(path, "rb") as f:
        lines = f.read().decode("latin-1").split("\n")
    names = [n.strip() for n in lines[0].split(",") if n.strip()]
    rows = []
    for line in lines[1:]:
        if not line.strip():
            continue
        if str_cols:
            rows.append(_parse_typed(line, len(names), set(str_cols)))
            continue
        toks = line.split()
        if len(toks) != len(names):
            raise ValueError("malformed result line %r for columns %s" % (line, names))
        row = []
        for t in toks:
            if len(t) == 1 and not t.isdigit() and t != "-":
                row.append(ord(t))
            else:
                row.append(int(t))
        rows.append(tuple(row))
    return names, rows
