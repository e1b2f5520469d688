"""Text import on the GPU (dq_table_import_text) against the reference's own
importer output and the CPU oracle of it (oracle/text_import.py), bit for bit:
every column read back through dq_table_column_read.  Then queries over tables
that came in as text give the reference's results."""
import json
import os
import re

import numpy as np
import pytest

import text_import as T
from canonical import canonical_rows
from evaluator import run_plan
from helpers import golden, make_case
from tbl_text import table_text

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "import_ref.json")
REASON = {T.TOO_FEW: "fewer delimiters than fields", T.TOO_MANY: "more delimiters than fields",
          T.NO_DIGIT: "not a number", T.OVERFLOW: "number out of range", T.NOT_CHAR: "not a single character",
          T.SHORT_DATE: "date shorter than 10 bytes", T.EXPONENT: "exponent not accepted"}


@pytest.fixture(scope="module")
def engine():
    from dogqc_b200.engine import Engine
    e = Engine(0)
    yield e
    e.close()


def ctype_of(kind):
    from dogqc_b200 import _lib as L
    return {T.INT: L.I32, T.DATE: L.U32, T.CHAR: L.I8, T.DECIMAL: L.I64, T.FLOAT: L.U32, T.STRING: L.STR}[kind]


def read_all(engine, name, fields):
    from dogqc_b200 import _lib as L
    out = {}
    for fd in fields:
        if fd[1] == T.SKIP:
            continue
        ct = ctype_of(fd[1])
        if ct == L.STR:
            chars, offs = engine.read_column(name, fd[0], ct)
            b = chars.tobytes()
            out[fd[0]] = [b[int(offs[i]):int(offs[i + 1])] for i in range(len(offs) - 1)]
        else:
            out[fd[0]] = engine.read_column(name, fd[0], ct).astype(np.int64).tolist()
    return out


def check_same(engine, text, fields, delim=b"|"):
    n = engine.import_text("t_imp", text, fields, delim.decode())
    want = T.parse(text, fields, delim)
    got = read_all(engine, "t_imp", fields)
    assert n == len(T.lines_of(text))
    assert got == want
    return n


def test_golden_matches_reference_importer(engine):
    with open(GOLDEN) as fh:
        g = json.load(fh)
    fields = [("k", T.INT), ("d", T.DATE), ("c", T.CHAR), ("f", T.FLOAT), ("s", T.STRING)]
    n = engine.import_text("imp", g["text"].encode(), fields)
    assert n == g["rows"] == 3000
    got = read_all(engine, "imp", fields)
    cols = g["columns"]
    assert got["k"] == cols["k"]
    assert got["d"] == cols["d"]
    assert got["c"] == cols["c"]
    assert got["f"] == np.array(cols["f"], np.float32).view(np.uint32).tolist()   # bit-exact floats
    assert [s.decode() for s in got["s"]] == cols["s"]
    t = engine.import_timing()
    assert t["kernel_launches"] == 6 and t["parse_ms"] > 0


def test_device_text_and_decimals(engine):
    import torch
    with open(GOLDEN) as fh:
        text = json.load(fh)["text"].encode()
    fields = [("k", T.INT), (None, T.SKIP), ("c", T.CHAR), ("f", T.DECIMAL, 2), ("s", T.STRING)]
    dev = torch.frombuffer(bytearray(text), dtype=torch.uint8).cuda()
    assert engine.import_text("imp_dev", dev, fields) == 3000
    assert read_all(engine, "imp_dev", fields) == T.parse(text, fields)


EDGE = [
    # (text, fields)
    (b"", [("a", T.INT)]),
    (b"7|", [("a", T.INT)]),                                        # no final newline
    (b"1 | 2|\r\n  -3|+4|tail\n-|  |\n", [("a", T.INT), ("b", T.INT)]),
    (b"2147483647|-2147483648|\n0|-0|\n", [("a", T.INT), ("b", T.INT)]),
    (b"12.345| A |1998-12-01|\n-0.5|b|1992-01-02xyz|\n7|c|0000-00-00|\n,5|d|1234567890|\n",
     [("p", T.DECIMAL, 2), ("c", T.CHAR), ("d", T.DATE)]),
    (b"1.5|\n-2,25|\n3e2|\n.5|\n-|\n1e-3|\n123456789.987654321|\n1e38|\n1e39|\n1e-45|\n7E+2|\n|\n",
     [("f", T.FLOAT)]),
    (b"|x|\n  |  yy  |\nabc def|z|\n", [("s", T.STRING), ("t", T.STRING)]),
    (b"a;1;\nb;2;\n", [("s", T.STRING), ("n", T.INT)]),             # another delimiter
    (b"9223372036854775807|\n-9223372036854775807|\n", [("p", T.DECIMAL, 0)]),
]


@pytest.mark.parametrize("i", range(len(EDGE)))
def test_edge_cases_match_oracle(engine, i):
    text, fields = EDGE[i]
    delim = b";" if b";" in text else b"|"
    check_same(engine, text, fields, delim)


BAD = [
    (b"1|\n2\n", [("a", T.INT)]),
    (b"1|2|\n", [("a", T.INT)]),
    (b"1|\n1 2|\n", [("a", T.INT)]),
    (b"1|\n2|\n2147483648|\n", [("a", T.INT)]),
    (b"1|\n\n", [("a", T.INT)]),
    (b"x|\n", [("a", T.INT), ("b", T.INT)]),
    (b"1|ab|\n", [("a", T.INT), ("c", T.CHAR)]),
    (b"1||\n", [("a", T.INT), ("c", T.CHAR)]),
    (b"98-12-01|\n", [("d", T.DATE)]),
    (b"1e5|\n", [("p", T.DECIMAL, 2)]),
    (b"1.5.|\n", [("f", T.FLOAT)]),
    (b"1e99999|\n", [("f", T.FLOAT)]),
    (b"99999999999999999999|\n", [("p", T.DECIMAL, 2)]),
]


@pytest.mark.parametrize("i", range(len(BAD)))
def test_malformed_rows_name_their_line(engine, i):
    from dogqc_b200._lib import DqError
    text, fields = BAD[i]
    with pytest.raises(T.TextImportError) as want:
        T.parse(text, fields)
    with pytest.raises(DqError) as got:
        engine.import_text("t_bad", text, fields)
    msg = str(got.value)
    assert re.search(r"line (\d+)", msg).group(1) == str(want.value.line), msg
    assert REASON[want.value.reason] in msg, msg
    if want.value.field < len(fields):
        assert "field %d " % (want.value.field + 1) in msg, msg


def _random_text(n, seed):
    r = np.random.Generator(np.random.Philox(seed))
    words = [b"alpha", b"beta", b"gamma", b"delta", b"kappa", b"omega", b"sigma", b"theta"]
    lines = []
    for i in range(n):
        k = int(r.integers(-2 ** 31, 2 ** 31))
        cents = int(r.integers(-10 ** 12, 10 ** 12))
        frac = b"%d.%02d" % (abs(cents) // 100, abs(cents) % 100)
        frac = (b"-" if cents < 0 else b"") + frac
        m = int(r.integers(0, 40))
        if i % 5000 == 17:
            m = int(r.integers(3000, 6000))          # a line longer than a 16 KB tile
        s = b" ".join(words[int(j)] for j in r.integers(0, len(words), m))
        c = bytes([int(r.integers(33, 127))])
        if c == b"|":
            c = b"!"
        pad = b" " * int(r.integers(0, 3))
        end = b"\r\n" if i % 7 == 3 else b"\n"
        lines.append(b"%s%d%s|%s|%s|%s|%s|%s|" % (pad, k, pad, frac, c, s, frac, b"1998-%02d-%02d" % (i % 12 + 1, i % 28 + 1)) + end)
    return b"".join(lines)


def test_random_text_across_tiles(engine):
    import torch
    text = _random_text(60_000, 11)
    assert len(text) > 20 * 16384
    fields = [("k", T.INT), ("p", T.DECIMAL, 2), ("c", T.CHAR), ("s", T.STRING), ("f", T.FLOAT), ("d", T.DATE)]
    check_same(engine, text, fields)
    want = T.parse(text, fields)
    # device text: read in place (aligned) and copied (a view one byte in)
    buf = torch.zeros(len(text) + 1, dtype=torch.uint8)
    buf[1:] = torch.frombuffer(bytearray(text), dtype=torch.uint8)
    dev = buf.cuda()
    for view in (dev[1:].clone(), dev[1:]):
        assert engine.import_text("t_dev", view, fields) == 60_000
        assert read_all(engine, "t_dev", fields) == want


def test_fast_path_boundaries(engine):
    """Values around the 16-byte window, the int32 range and 18 decimal digits,
    at every alignment of the field within a 16-byte chunk."""
    ints = [b"0", b"-0", b"+7", b"-", b"+", b"2147483647", b"-2147483648", b"2147483648", b"-2147483649",
            b"0000000000000001", b"00000000000000001", b"-000000000000042", b" 5", b"5 ", b"1 2"]
    decs = [b"0.04", b"12345678901234.5", b"1234567890123456", b"123456789012345.6789", b".5", b"-.", b"7.",
            b"99999999999999.99", b"999999999999999.9", b"1,25", b" 3.1", b"3.1 "]
    dates = [b"1998-12-01", b"1998-12-01T00:00", b"1998-12-01T00:00:0", b" 1998-12-01", b"1998-12-01 "]
    lines = []
    for pad in range(16):
        for v in ints:
            for d in decs:
                lines.append(b"%s|%s|%s|%s|\n" % (b"x" * pad, v, d, dates[(pad + len(v)) % len(dates)]))
    text = b"".join(lines)
    fields = [("s", T.STRING), ("k", T.INT), ("p", T.DECIMAL, 2), ("d", T.DATE)]
    # rows whose value is out of range fail the whole import: check those one line at a time
    good = []
    for ln in lines:
        try:
            T.parse(ln, fields)
            good.append(ln)
        except T.TextImportError:
            with pytest.raises(Exception):
                engine.import_text("t_fast", ln, fields)
    check_same(engine, b"".join(good), fields)


def test_reimport_reuses_and_failure_drops(engine):
    """A table replaced by a new import of the same name: smaller, larger, then
    a failing import (which leaves no table of that name)."""
    from dogqc_b200._lib import DqError
    fields = [("k", T.INT), ("s", T.STRING), ("d", T.DATE)]
    big = _random_text(3000, 5)
    big_fields = [("k", T.INT), ("p", T.DECIMAL, 2), ("c", T.CHAR), ("s", T.STRING), ("f", T.FLOAT), ("d", T.DATE)]
    small = b"".join(b"%d|%s|1998-01-%02d|\n" % (i, b"ab" * (i % 7), i % 28 + 1) for i in range(500))
    for text, fl in ((big, big_fields), (small, fields), (big, big_fields), (big, big_fields)):
        n = engine.import_text("t_re", text, fl)
        assert n == len(T.lines_of(text))
        assert read_all(engine, "t_re", fl) == T.parse(text, fl)
    with pytest.raises(DqError):
        engine.import_text("t_re", small + b"x|y|z|\n", fields)
    with pytest.raises(DqError):
        engine.read_column("t_re", "k", ctype_of(T.INT))


def test_mmdb_directory_and_text_agree(engine):
    """The reference importer's column files loaded onto the device, and the
    same lines imported as text: equal columns."""
    from dogqc_b200 import _lib as L
    from dogqc_b200 import importer
    mmdb = os.path.join(os.path.dirname(GOLDEN), "mmdb_ref")
    e = engine
    sizes = importer.load_mmdb(e, mmdb)
    assert sizes == {"imp": 200}
    with open(GOLDEN) as fh:
        g = json.load(fh)
    text = "".join(g["text"].splitlines(True)[:200]).encode()
    fields = [("k", T.INT), ("d", T.DATE), ("c", T.CHAR), ("f", T.DECIMAL, 2), ("s", T.STRING)]
    e.import_text("imp_txt", text, fields)
    for name, kind in (("k", T.INT), ("d", T.DATE), ("c", T.CHAR)):
        assert e.read_column("imp", name, ctype_of(kind)).tolist() == e.read_column("imp_txt", name, ctype_of(kind)).tolist()
    assert e.read_column("imp", "f", L.U64).view(np.int64).tolist() == e.read_column("imp_txt", "f", L.I64).tolist()
    a, b = e.read_column("imp", "s", L.STR), e.read_column("imp_txt", "s", L.STR)
    assert a[0].tobytes() == b[0].tobytes() and a[1].tolist() == b[1].tolist()


def _import_database(engine, db):
    from dogqc_b200 import importer
    for name, t in db.tables.items():
        n = importer.load_table(engine, t.schema_entry(), table_text(t))
        assert n == t.size


def test_query_on_imported_tables_matches_reference():
    """c0 at the golden case's size, its table loaded as text: the reference's rows."""
    from dogqc_b200.engine import Engine
    g = golden("c0_s")
    db, alg, plan = make_case(g["spec"])
    e = Engine(0)
    try:
        _import_database(e, db)
        p = e.prepare(plan)
        try:
            res = p.execute()
        finally:
            p.free()
    finally:
        e.close()
    assert res.names == g["columns"]
    assert [list(r) for r in canonical_rows(res.rows())] == g["rows"]


def test_query_on_imported_strings_matches_oracle():
    """c3 (LIKE over a string dimension): text import trims the strings as the
    reference's importer does, so the oracle runs on the trimmed table."""
    from dogqc_b200.database import Database, StringColumn, Table
    from dogqc_b200.engine import Engine
    g = golden("c3_s")
    db, alg, plan = make_case(g["spec"])
    tables = []
    for name, t in db.tables.items():
        cols = dict(t.columns)
        for a, c in cols.items():
            if isinstance(c, StringColumn):
                cols[a] = StringColumn.from_list([c.get(i).strip(b" ") for i in range(len(c))])
        tables.append(Table(name, cols, t.types))
    trimmed = Database(tables)
    want = canonical_rows(run_plan(trimmed, plan)[1])
    e = Engine(0)
    try:
        _import_database(e, db)
        p = e.prepare(plan)
        try:
            got = canonical_rows(p.execute().rows())
        finally:
            p.free()
    finally:
        e.close()
    assert got == want
