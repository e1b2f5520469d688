"""The storage boundary: tables from ``.tbl`` text or from the reference's
database directories, into device-resident tables.

* Text: the counterpart of the reference's ``Importer`` (dogqc/dbio.py:117-253),
  which generates and compiles a C++ program per schema to parse the files on
  the host and write one memory-mapped file per column.  Here each file's bytes
  go to the device once and are parsed there (``dq_table_import_text``).
* Column files: a directory the reference's importer wrote (``dbAccess``,
  dbio.py:13-27) -- one file per column, ``<table>_<attribute>`` (strings:
  ``_offset`` with ``size_t`` offsets and ``_char`` with the bytes), each an
  8-byte size header, the values and a trailing zero byte
  (dogqc/include/mappedmalloc.h:11-60), and ``dbschema.pickle`` with the
  schema and table sizes (dbio.py:53-65) -- read on the host and registered.

A schema is the reference's dictionary layout (query/schema/tpch.py):
``{"dateformat": ..., "<table>": {"name": ..., "attributes": OrderedDict(
(attribute, Type))}}`` -- types are matched by name (INT, DATE, CHAR, FLOAT,
DOUBLE, STRING), so the reference's ``Type`` enum or plain strings both work.
"""
import os
import pickle
from collections import OrderedDict

import numpy as np

from dogqc_b200 import _lib as L
from dogqc_b200.types import Type

KIND = {"INT": L.TEXT_INT, "DATE": L.TEXT_DATE, "CHAR": L.TEXT_CHAR, "STRING": L.TEXT_STRING}


def _type_name(t):
    return getattr(t, "name", t)


def fields_for(table_schema, floats="decimal", scale=2):
    """The field list of one table: FLOAT/DOUBLE become exact decimals scaled by
    ``10**scale`` (the engine's fixed-point FLOAT columns), or with
    ``floats="binary32"`` the float bits the reference's importer stores."""
    out = []
    for attr, t in table_schema["attributes"].items():
        name = _type_name(t)
        if name in ("FLOAT", "DOUBLE"):
            out.append((attr, L.TEXT_DECIMAL, scale) if floats == "decimal" else (attr, L.TEXT_FLOAT))
        elif name in KIND:
            out.append((attr, KIND[name]))
        else:
            raise ValueError("attribute %s has no text import for type %r" % (attr, t))
    return out


def load_table(engine, table_schema, text, floats="decimal", scale=2, delim="|"):
    """Import one table's text; sets ``table_schema["size"]`` and returns it."""
    n = engine.import_text(table_schema["name"], text, fields_for(table_schema, floats, scale), delim)
    table_schema["size"] = n
    return n


def load_database(engine, schema, csvpath, floats="decimal", scale=2, delim="|"):
    """Every table of ``schema`` from ``<csvpath>/<table>.tbl`` (dbio.py:140-149:
    ``loadDatabase``; table sizes as ``retrieveTableSizes``, dbio.py:124-138).
    Returns {table: rows}."""
    sizes = {}
    for key, table in schema.items():
        if key == "dateformat":
            continue
        path = os.path.join(csvpath, table["name"] + ".tbl")
        with open(path, "rb") as fh:
            text = fh.read()
        sizes[table["name"]] = load_table(engine, table, text, floats, scale, delim)
    return sizes


class _SchemaUnpickler(pickle.Unpickler):
    """Only the classes a schema pickle holds: the ordered attribute maps and
    the type enumeration (the reference's ``dogqc.types.Type`` maps to this
    package's, whose members have the same values)."""

    def find_class(self, module, name):
        if (module, name) == ("collections", "OrderedDict"):
            return OrderedDict
        if name == "Type" and module in ("dogqc.types", "dogqc_b200.types"):
            return Type
        raise pickle.UnpicklingError("a schema pickle does not hold %s.%s" % (module, name))


def read_schema(dbpath):
    """The schema a database directory was written with (``dbschema.pickle``)."""
    with open(os.path.join(dbpath, "dbschema.pickle"), "rb") as fh:
        return _SchemaUnpickler(fh).load()


# element types of the column files, as the reference's importer writes them
# (its code generator maps FLOAT/DOUBLE to float, dbio.py:142, codegen.py:37-45)
FILE_DTYPE = {"INT": np.int32, "DATE": np.uint32, "CHAR": np.int8, "FLOAT": np.float32, "DOUBLE": np.float32}


def _column_file(path, dtype, n):
    """The first ``n`` values of one column file (after its 8-byte header)."""
    a = np.fromfile(path, dtype=np.uint8, offset=8)
    size = np.dtype(dtype).itemsize
    if len(a) < n * size:
        raise ValueError("%s holds %d bytes, %d values of %d bytes expected" % (path, len(a), n, size))
    return a[:n * size].view(dtype).copy()


def read_mmdb(dbpath, schema=None, floats="decimal", scale=2):
    """A ``Database`` from a directory the reference's importer wrote.

    FLOAT/DOUBLE files hold binary32 values: ``floats="decimal"`` rounds them to
    the engine's fixed point (``round(value * 10**scale)``, two's complement in
    the 64-bit column), ``floats="bits"`` keeps their IEEE bits in an INT
    column."""
    from dogqc_b200.database import Database, StringColumn, Table
    schema = schema or read_schema(dbpath)
    tables = []
    for key, t in schema.items():
        if not isinstance(t, dict) or "attributes" not in t:
            continue
        name, n = t["name"], int(t["size"])
        cols, types = OrderedDict(), OrderedDict()
        for attr, ty in t["attributes"].items():
            tn = _type_name(ty)
            path = os.path.join(dbpath, "%s_%s" % (name, attr))
            if tn == "STRING":
                offs = _column_file(path + "_offset", np.uint64, n + 1)
                chars = np.fromfile(path + "_char", dtype=np.uint8, offset=8)[:int(offs[-1]) if n else 0]
                lens = np.diff(offs)
                width = int(lens[0]) if n and np.all(lens == lens[0]) else 0  # fixed width: read without offsets
                cols[attr] = StringColumn(chars, offs, width)
                types[attr] = Type.STRING
            elif tn in ("FLOAT", "DOUBLE"):
                v = _column_file(path, np.float32, n)
                if floats == "bits":
                    cols[attr], types[attr] = v.view(np.int32).copy(), Type.INT
                else:
                    cols[attr] = np.rint(v.astype(np.float64) * 10.0 ** scale).astype(np.int64).view(np.uint64)
                    types[attr] = Type.FLOAT
            elif tn in FILE_DTYPE:
                cols[attr], types[attr] = _column_file(path, FILE_DTYPE[tn], n), Type[tn]
            else:
                raise ValueError("attribute %s.%s has type %r" % (name, attr, ty))
        tables.append(Table(name, cols, types))
    return Database(tables)


def load_mmdb(engine, dbpath, floats="decimal", scale=2):
    """Every table of a reference database directory onto the device.
    Returns {table: rows}."""
    db = read_mmdb(dbpath, floats=floats, scale=scale)
    engine.register_database(db, force=True)
    return {name: t.size for name, t in db.tables.items()}
