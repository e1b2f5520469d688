"""Canonical form of a result set (test infrastructure).

Results are compared as multisets: rows (tuples of Python ints; chars as their
byte value) are sorted lexicographically and hashed.  Row order and column
widths do not enter the checksum.
"""
import hashlib


def _canon(v):
    if isinstance(v, (bytes, bytearray)):
        return bytes(v)
    return v if isinstance(v, str) else int(v)


def canonical_rows(rows):
    """Rows as sorted tuples: integers, and strings as bytes."""
    return sorted(tuple(_canon(v) for v in r) for r in rows)


def canonical_checksum(rows):
    h = hashlib.sha256()
    for r in canonical_rows(rows):
        h.update((",".join(str(v) for v in r) + "\n").encode())
    return h.hexdigest()
