"""Pin the text importer on the reference's own one (test infrastructure).

The reference loads ``<table>.tbl`` files (``|``-separated fields, a terminal
``|`` on every line) through generated C++ compiled with g++
(dogqc/dbio.py:117-253: ``Importer.loadDatabase``): integers as ``int``,
dates through the schema's ``toDate`` (``YYYY-MM-DD`` -> ``YYYYMMDD``), chars as
one byte, decimals as ``float`` (the importer's code generator is FP32,
dbio.py:142), strings as ``size_t`` offsets plus a char heap; every column goes
to a file ``<table>_<attr>`` (``_offset``/``_char`` for strings) with an 8-byte
size header (dogqc/include/mappedmalloc.h).

This script writes a seeded table as ``.tbl`` text, runs the reference importer
on it here (it needs only g++ and the reference's headers, no GPU), reads the
column files back and stores text and values in ``tests/golden/import_ref.json``.
It also keeps the reference's database directory for the first 200 lines
(column files and ``dbschema.pickle``) as ``tests/golden/mmdb_ref/``, the
fixture of the column-file reader; the pickle's ``dateformat`` entry (the
schema's date parser as C source) is dropped so that no reference code is
committed.

Usage: ``python oracle/ref_import.py`` (reads the reference at
$DOGQC_REFERENCE, default /root/reference).
"""
import json
import os
import shutil
import subprocess
import sys
import tempfile
from collections import OrderedDict

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
REF = os.environ.get("DOGQC_REFERENCE", "/root/reference")
OUT = os.path.join(REPO, "tests", "golden", "import_ref.json")
MMDB_OUT = os.path.join(REPO, "tests", "golden", "mmdb_ref")
MMDB_ROWS = 200


def make_text(n=3000, seed=20261203 + 9):
    """``n`` rows: int key, date, char flag, 2-decimal amount, string comment."""
    r = np.random.Generator(np.random.Philox(seed))
    words = ["alpha", "beta", "gamma", "delta", "kappa", "omega", "sigma", "theta", "quick", "brown"]
    lines = []
    days_in = [31, 28, 31, 30, 31, 30, 31, 31, 30, 31, 30, 31]
    for i in range(n):
        k = int(r.integers(-50_000, 1_000_000))
        y = int(r.integers(1992, 1999))
        m = int(r.integers(1, 13))
        d = int(r.integers(1, days_in[m - 1] + 1))
        c = "AFNOR"[int(r.integers(0, 5))]
        cents = int(r.integers(0, 5_000_000))          # up to 49,999.99: exact in a float
        f = "%d.%02d" % (cents // 100, cents % 100)
        s = " ".join(words[int(j)] for j in r.integers(0, len(words), int(r.integers(0, 6))))
        lines.append("%d|%04d-%02d-%02d|%s|%s|%s|" % (k, y, m, d, c, f, s))
    return "\n".join(lines) + "\n"


def _read(path, dtype):
    """The array after the 8-byte size header (whole elements; the mapping may
    end with padding)."""
    with open(path, "rb") as fh:
        data = fh.read()[8:]
    size = np.dtype(dtype).itemsize
    return np.frombuffer(data[:len(data) // size * size], dtype=dtype)


def main():
    sys.path.insert(0, REF)
    from dogqc import dbio
    from dogqc.types import Type
    from query.schema.tpch import tpchSchema   # the reference's toDate (imported, not copied)
    text = make_text()
    schema = {"dateformat": tpchSchema["dateformat"],
              "imp": {"name": "imp", "size": 0, "numColumns": 5,
                      "attributes": OrderedDict([("k", Type.INT), ("d", Type.DATE), ("c", Type.CHAR),
                                                 ("f", Type.FLOAT), ("s", Type.STRING)])}}
    work = tempfile.mkdtemp(prefix="dq_import_")
    cwd = os.getcwd()
    try:
        csv = os.path.join(work, "csv")
        db = os.path.join(work, "mmdb")
        os.makedirs(csv)
        with open(os.path.join(csv, "imp.tbl"), "w") as fh:
            fh.write(text)
        src = os.path.join(work, "src")
        os.makedirs(src)
        os.symlink(os.path.join(REF, "dogqc"), os.path.join(work, "dogqc"))
        os.chdir(src)
        dbio.dbAccess(schema, db, csv, doReload=True)
        n = text.count("\n")
        vals = {"k": _read(os.path.join(db, "imp_k"), np.int32)[:n].tolist(),
                "d": _read(os.path.join(db, "imp_d"), np.int32)[:n].tolist(),
                "c": _read(os.path.join(db, "imp_c"), np.int8)[:n].tolist(),
                "f": [float(x) for x in _read(os.path.join(db, "imp_f"), np.float32)[:n]]}
        off = _read(os.path.join(db, "imp_s_offset"), np.uint64)[:n + 1]
        chars = _read(os.path.join(db, "imp_s_char"), np.uint8)
        vals["s"] = [bytes(chars[off[i]:off[i + 1]]).decode() for i in range(n)]
    finally:
        os.chdir(cwd)
        shutil.rmtree(work, ignore_errors=True)
    with open(OUT, "w") as fh:
        json.dump({"text": text, "rows": n, "columns": vals}, fh, separators=(",", ":"))
        fh.write("\n")
    print("wrote", OUT, n, "rows")
    # the reference's generator keeps state between imports: the second one runs in its own process
    subprocess.run([sys.executable, os.path.abspath(__file__), "--mmdb"], check=True)


def write_mmdb_fixture():
    """The reference's database directory for the first 200 lines of the text."""
    sys.path.insert(0, REF)
    from dogqc import dbio
    from dogqc.types import Type
    from query.schema.tpch import tpchSchema
    small = "".join(make_text().splitlines(True)[:MMDB_ROWS])
    schema = {"dateformat": tpchSchema["dateformat"],
              "imp": {"name": "imp", "size": 0, "numColumns": 5,
                      "attributes": OrderedDict([("k", Type.INT), ("d", Type.DATE), ("c", Type.CHAR),
                                                 ("f", Type.FLOAT), ("s", Type.STRING)])}}
    work = tempfile.mkdtemp(prefix="dq_mmdb_")
    cwd = os.getcwd()
    try:
        csv = os.path.join(work, "csv")
        db = os.path.join(work, "mmdb")
        os.makedirs(csv)
        with open(os.path.join(csv, "imp.tbl"), "w") as fh:
            fh.write(small)
        src = os.path.join(work, "src")
        os.makedirs(src)
        os.symlink(os.path.join(REF, "dogqc"), os.path.join(work, "dogqc"))
        os.chdir(src)
        dbio.dbAccess(schema, db, csv, doReload=True)
        shutil.rmtree(MMDB_OUT, ignore_errors=True)
        os.makedirs(MMDB_OUT)
        for f in sorted(os.listdir(db)):
            shutil.copy2(os.path.join(db, f), os.path.join(MMDB_OUT, f))
        # the schema pickle carries the schema's date parser as C source: drop that entry
        import pickle
        spath = os.path.join(MMDB_OUT, "dbschema.pickle")
        with open(spath, "rb") as fh:
            sch = pickle.load(fh)
        sch.pop("dateformat", None)
        with open(spath, "wb") as fh:
            pickle.dump(sch, fh, protocol=pickle.HIGHEST_PROTOCOL)
    finally:
        os.chdir(cwd)
        shutil.rmtree(work, ignore_errors=True)
    print("wrote", MMDB_OUT)


if __name__ == "__main__":
    if "--mmdb" in sys.argv:
        write_mmdb_fixture()
    else:
        main()
