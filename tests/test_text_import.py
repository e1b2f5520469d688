"""Text import, host side: the CPU oracle of the reference's importer pinned on
the reference's own output (tests/golden/import_ref.json, written by
oracle/ref_import.py from the reference's generated importer), its edge cases
as the reference's CSV reader defines them, and the schema -> field mapping."""
import json
import os

import numpy as np
import pytest

import text_import as T
from tbl_text import table_text

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "import_ref.json")
FIELDS = [("k", T.INT), ("d", T.DATE), ("c", T.CHAR), ("f", T.FLOAT), ("s", T.STRING)]


def golden():
    with open(GOLDEN) as fh:
        return json.load(fh)


def test_oracle_matches_reference_importer():
    g = golden()
    out = T.parse(g["text"].encode(), FIELDS)
    cols = g["columns"]
    assert len(out["k"]) == g["rows"] == 3000
    assert out["k"] == cols["k"]
    assert out["d"] == cols["d"]
    assert out["c"] == cols["c"]
    assert out["f"] == np.array(cols["f"], np.float32).view(np.uint32).tolist()
    assert [s.decode() for s in out["s"]] == cols["s"]


def test_reference_float_is_not_the_nearest_float():
    """The reference accumulates digit by digit in float; on many rows that is
    not the correctly rounded value, so only a step-by-step parse matches."""
    g = golden()
    ref = np.array(g["columns"]["f"], np.float32)
    nearest = np.array([float(l.split("|")[3]) for l in g["text"].splitlines()], np.float32)
    assert (ref != nearest).sum() > 100


def test_lines_and_trimming():
    text = b"1 | 2|\r\n  -3|+4|tail\n-|  |"
    out = T.parse(text, [("a", T.INT), ("b", T.INT)])
    assert out == {"a": [1, -3, 0], "b": [2, 4, 0]}
    assert T.parse(b"", [("a", T.INT)]) == {"a": []}


@pytest.mark.parametrize("text,line,field,reason", [
    (b"1|\n2\n", 2, 0, T.TOO_FEW),
    (b"1|2|\n", 1, 1, T.TOO_MANY),
    (b"1 2|\n", 1, 0, T.NO_DIGIT),
    (b"2147483648|\n", 1, 0, T.OVERFLOW),
    (b"1|\n\n", 2, 0, T.TOO_FEW),          # an empty line
])
def test_int_errors(text, line, field, reason):
    with pytest.raises(T.TextImportError) as e:
        T.parse(text, [("a", T.INT)])
    assert (e.value.line, e.value.field, e.value.reason) == (line, field, reason)


def test_int_limits():
    out = T.parse(b"2147483647|\n-2147483648|\n", [("a", T.INT)])
    assert out["a"] == [2147483647, -2147483648]
    with pytest.raises(T.TextImportError):
        T.parse(b"-2147483649|\n", [("a", T.INT)])


def test_shape_errors_come_before_value_errors():
    # csv.h splits the whole line before parsing any column
    with pytest.raises(T.TextImportError) as e:
        T.parse(b"x|\n", [("a", T.INT), ("b", T.INT)])
    assert e.value.reason == T.TOO_FEW and e.value.field == 1


def test_decimal_char_date():
    f = [("p", T.DECIMAL, 2), ("c", T.CHAR), ("d", T.DATE)]
    out = T.parse(b"12.345| A |1998-12-01|\n-0.5|b|1992-01-02xyz|\n7|c|0000-00-00|\n", f)
    assert out["p"] == [1234, -50, 700]
    assert out["c"] == [65, 98, 99]
    assert out["d"] == [19981201, 19920102, 0]
    for bad in (b"1e5|a|1998-12-01|\n", b"1|ab|1998-12-01|\n", b"1|a|98-12-01|\n"):
        with pytest.raises(T.TextImportError):
            T.parse(bad, f)


def test_float_grammar():
    vals = T.parse(b"1.5|\n-2,25|\n3e2|\n.5|\n-|\n1e-3|\n", [("f", T.FLOAT)])["f"]
    got = np.array(vals, np.uint32).view(np.float32).tolist()
    assert got[:5] == [1.5, -2.25, 300.0, 0.5, -0.0]
    assert abs(got[5] - 1e-3) < 1e-9


def test_table_text_round_trip_through_oracle():
    """The writer the GPU tests use produces text whose parse is the table."""
    from dogqc_b200 import workloads
    db = workloads.GENERATORS["c0"](0.0005)
    t = db.tables["lineitem"]
    kinds = {"INT": T.INT, "DATE": T.DATE, "CHAR": T.CHAR}
    fields = [(a, kinds[getattr(ty, "name", ty)]) if getattr(ty, "name", ty) in kinds else (a, T.DECIMAL, 2)
              for a, ty in t.types.items()]
    out = T.parse(table_text(t), fields)
    for a, _ in t.types.items():
        want = np.asarray(t.columns[a]).astype(np.int64).tolist()
        assert out[a] == want, a


def test_importer_field_mapping():
    from collections import OrderedDict
    from dogqc_b200 import _lib as L
    from dogqc_b200 import importer
    from dogqc_b200.types import Type
    sch = {"name": "t", "attributes": OrderedDict([("a", Type.INT), ("b", Type.DATE), ("c", Type.CHAR),
                                                   ("d", Type.FLOAT), ("e", Type.STRING)])}
    assert importer.fields_for(sch) == [("a", L.TEXT_INT), ("b", L.TEXT_DATE), ("c", L.TEXT_CHAR),
                                        ("d", L.TEXT_DECIMAL, 2), ("e", L.TEXT_STRING)]
    assert importer.fields_for(sch, floats="binary32")[3] == ("d", L.TEXT_FLOAT)
    assert [k for k in (T.INT, T.DATE, T.CHAR, T.DECIMAL, T.STRING, T.SKIP, T.FLOAT)] == \
        [L.TEXT_INT, L.TEXT_DATE, L.TEXT_CHAR, L.TEXT_DECIMAL, L.TEXT_STRING, L.TEXT_SKIP, L.TEXT_FLOAT]


MMDB = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "mmdb_ref")


def test_mmdb_reader_matches_reference_directory():
    """The reference importer's own column files (first 200 lines of the golden
    text) read back: the same values its reader maps."""
    from dogqc_b200 import importer
    g = golden()
    cols = g["columns"]
    db = importer.read_mmdb(MMDB)
    t = db.tables["imp"]
    assert t.size == 200
    assert t.columns["k"].tolist() == cols["k"][:200]
    assert t.columns["d"].tolist() == cols["d"][:200]
    assert t.columns["c"].tolist() == cols["c"][:200]
    assert [t.columns["s"].get(i).decode() for i in range(200)] == cols["s"][:200]
    text = "".join(g["text"].splitlines(True)[:200]).encode()
    skip = (None, T.SKIP)
    exact = T.parse(text, [skip, skip, skip, ("f", T.DECIMAL, 2), skip])["f"]
    assert t.columns["f"].view(np.int64).tolist() == exact          # binary32 rounded back to cents
    # the backend's path to a reference accessor's files (schema given, not read)
    same = importer.read_mmdb(MMDB, schema=importer.read_schema(MMDB)).tables["imp"]
    assert all(np.array_equal(np.asarray(same.columns[a] if a != "s" else same.columns[a].chars),
                              np.asarray(t.columns[a] if a != "s" else t.columns[a].chars)) for a in "kdcfs")
    bits = importer.read_mmdb(MMDB, floats="bits").tables["imp"].columns["f"]
    assert bits.view(np.float32).tolist() == np.array(cols["f"][:200], np.float32).tolist()


def test_schema_unpickler_refuses_other_classes(tmp_path):
    import pickle
    from dogqc_b200 import importer

    class Evil(object):
        def __reduce__(self):
            return (os.getcwd, ())
    d = tmp_path / "db"
    d.mkdir()
    (d / "dbschema.pickle").write_bytes(pickle.dumps({"t": Evil()}))
    with pytest.raises(pickle.UnpicklingError):
        importer.read_schema(str(d))
