"""Writing tables as ``.tbl`` text (test helper): the inverse of the import for
the engine's column types, so a generated database can go through the text
path and be compared with itself.

INT -> decimal integer; DATE (u32) -> eight digits as ``DDDD-DD-DD`` (the
reference's toDate reads the digits back at those positions); CHAR -> the
byte; FLOAT (u64 fixed point, two decimals) -> ``int.cc``; STRING -> the bytes.
Every field is followed by ``|``, as in dbgen's output.
"""
import numpy as np


def _type_name(t):
    return getattr(t, "name", t)


def column_text(col, type_name):
    """The text of every value of one column (list of bytes)."""
    if type_name == "STRING":
        return [col.get(i) for i in range(len(col))]
    a = np.asarray(col)
    if type_name == "INT":
        return [b"%d" % v for v in a.tolist()]
    if type_name == "DATE":
        out = []
        for v in a.tolist():
            d = b"%08d" % v
            out.append(d[:4] + b"-" + d[4:6] + b"-" + d[6:])
        return out
    if type_name == "CHAR":
        return [bytes([v & 0xFF]) for v in a.tolist()]
    if type_name in ("FLOAT", "DOUBLE"):
        return [b"%d.%02d" % (v // 100, v % 100) for v in a.tolist()]
    raise ValueError(type_name)


def table_text(table):
    cols = [column_text(table.columns[name], _type_name(t)) for name, t in table.types.items()]
    return b"".join(b"|".join(vals) + b"|\n" for vals in zip(*cols))

