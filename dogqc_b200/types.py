"""Relational data types of the plan front end.

Mirrors the type enumeration of the reference front end (dogqc/types.py:3-10) with
the same member names and values, so plan scripts written for the reference load
unchanged.
"""
from enum import Enum


class Type(Enum):
    INT = 1
    FLOAT = 2
    DOUBLE = 3
    CHAR = 4
    STRING = 5
    DATE = 6
    BOOLEAN = 7


class CType(object):
    """Names of the decimal representations a backend may be asked for.

    The reference passes one of these as ``decimalRepr`` (dogqc/cudalang.py:111-122,
    dogqc/codegen.py:37-45).  This backend always computes FLOAT/DOUBLE attributes
    as exact 64-bit integers with the wrap-around semantics of ``unsigned long
    long``; ``ULL`` is the matching reference mode and the other names are accepted
    and mapped to it.
    """
    INT = "int"
    UINT = "unsigned"
    UINT64 = "uint64_t"
    FP32 = "float"
    FP64 = "double"
    CHAR = "char"
    SIZE = "size_t"
    ULL = "unsigned long long"
    STR_TYPE = "str_t"
