"""Reader for the reference's memory-mapped column files.

The reference imports ``.tbl`` files once into ``<dbpath>/<table>_<attr>`` files
(dogqc/dbio.py:117-253) that its generated programs map with
``map_memory_file`` (dogqc/include/mappedmalloc.h:69-82): an 8-byte header,
then the raw array; strings are ``<table>_<attr>_offset`` (``size_t[n+1]``) and
``<table>_<attr>_char``.  ``load_mmdb`` maps those files into a ``Database`` so
a plan built against the reference's accessor runs on this backend unchanged.
"""
import os

import numpy as np

from dogqc_b200.database import STORAGE_DTYPE, Database, StringColumn, Table
from dogqc_b200.types import Type


def _map(path, dtype, count):
    return np.memmap(path, dtype=dtype, mode="r", offset=8, shape=(count,))


def load_mmdb(schema, dbpath):
    db = Database()
    for name, entry in schema.items():
        if not isinstance(entry, dict) or "attributes" not in entry:
            continue
        n = int(entry["size"])
        cols, types = {}, {}
        for attr, t in entry["attributes"].items():
            tn = t.name if hasattr(t, "name") else str(t)
            typ = Type[tn]
            base = os.path.join(dbpath, "%s_%s" % (name, attr))
            if typ == Type.STRING:
                off = np.array(_map(base + "_offset", np.uint64, n + 1))
                chars = np.array(_map(base + "_char", np.uint8, int(off[-1]) if n else 0))
                lens = np.diff(off)
                width = int(lens[0]) if n and np.all(lens == lens[0]) else 0
                cols[attr] = StringColumn(chars, off, width)
            else:
                cols[attr] = np.array(_map(base, STORAGE_DTYPE[typ], n))
            types[attr] = typ
        db.add(Table(name, cols, types))
    return db
