"""Loading ``.tbl`` text into device tables: the counterpart of the
reference's ``Importer`` (dogqc/dbio.py:117-253), which generates and compiles
a C++ program per schema to parse the files on the host and write one
memory-mapped file per column.  Here each file's bytes go to the device once
and are parsed there (``dq_table_import_text``); the columns stay resident in
HBM for the plans that scan them.

A schema is the reference's dictionary layout (query/schema/tpch.py):
``{"dateformat": ..., "<table>": {"name": ..., "attributes": OrderedDict(
(attribute, Type))}}`` -- types are matched by name (INT, DATE, CHAR, FLOAT,
DOUBLE, STRING), so the reference's ``Type`` enum or plain strings both work.
"""
import os

from dogqc_b200 import _lib as L

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
