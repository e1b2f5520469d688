"""The CPU oracle against the reference's own generated pipeline.

The fixtures in tests/golden/ were produced by running the reference's generated
CUDA code (compiled for sm_100a, exact ULL decimals) over the same seeded tables;
tests/golden/make_golden.py documents the recipe.  These tests pin the oracle:
the device engine is later checked against the oracle and the same fixtures.
"""
import pytest

from canonical import canonical_checksum, canonical_rows
from evaluator import run_plan
from helpers import golden, golden_cases, make_case, reference_rows, result_checksum

SMALL = [c for c in golden_cases() if golden(c)["spec"]["scale"] < 0.1]
FULL_FAST = ["c0", "c1", "c5", "c7", "c8", "c11", "c12", "c13", "c14", "c16", "c18", "c19"]


@pytest.mark.parametrize("case", SMALL)
def test_oracle_matches_reference_small(case):
    g = golden(case)
    db, alg, plan = make_case(g["spec"])
    names, rows = run_plan(db, plan)
    assert names == g["columns"]
    assert len(rows) == g["nrows"]
    assert canonical_checksum(reference_rows(rows, g["spec"])) == g["checksum"]
    assert reference_rows(rows, g["spec"]) == g["rows"]


@pytest.mark.parametrize("case", FULL_FAST)
def test_oracle_matches_reference_full(case):
    g = golden(case)
    db, alg, plan = make_case(g["spec"])
    names, rows = run_plan(db, plan)
    assert len(rows) == g["nrows"]
    assert result_checksum(rows, g["spec"]) == g["checksum"]


def test_like_matcher_quirks():
    from evaluator import like_check
    assert like_check(b"abcd efgh", b"%efg%")
    assert not like_check(b"abcd efgh", b"%xyz%")
    assert like_check(b"abc", b"a_c")
    assert like_check(b"abcx", b"abc%")
    assert like_check(b"xabc", b"%abc")
    assert not like_check(b"", b"%a%")
    # the reference's matcher checks no total length without a '%' (util.cuh:144-199)
    assert like_check(b"abcabc", b"abc")
