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


def parse_result(path):
    """Return (column names, list of row tuples of ints) from a reference result file."""
    with open(path, "rb") as f:
        lines = f.read().decode("latin-1").split("\n")
    names = [n.strip() for n in lines[0].split(",") if n.strip()]
    rows = []
    for line in lines[1:]:
        if not line.strip():
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
