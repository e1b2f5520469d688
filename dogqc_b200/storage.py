"""Reader for the reference's memory-mapped column files.

The reference imports ``.tbl`` files once into ``<dbpath>/<table>_<attr>`` files
(dogqc/dbio.py:117-253) that its generated programs map with
``map_memory_file`` (dogqc/include/mappedmalloc.h:69-82): an 8-byte header,
then the raw array; strings are ``<table>_<attr>_offset`` (``size_t[n+1]``) and
``<table>_<attr>_char``; FLOAT/DOUBLE columns hold binary32 values (the
importer's decimal type, dbio.py:142).  ``load_mmdb`` reads those files into a
``Database`` so a plan built against the reference's accessor runs on this
backend unchanged (the reading itself is ``dogqc_b200.importer.read_mmdb``).
"""
from dogqc_b200.importer import read_mmdb


def load_mmdb(schema, dbpath, floats="decimal", scale=2):
    return read_mmdb(dbpath, schema=schema, floats=floats, scale=scale)
