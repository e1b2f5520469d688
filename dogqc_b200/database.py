"""Host-side table catalogue.

A ``Database`` holds named tables of host columns plus the schema dictionary the
plan front end reads (``database.schema``; the reference's accessor exposes the
same shape, dogqc/dbio.py:13-27 and query/schema/tpch.py): per table
``{"name", "size", "numColumns", "attributes": OrderedDict(name -> Type),
"charSizes": {name: bytes}}``.

Column storage follows the reference's C representation of each type
(dogqc/codegen.py:37-45) so values round-trip bit for bit:

=========  ===================  =====================================
Type       numpy dtype          reference C type
=========  ===================  =====================================
INT        int32                int
DATE       uint32               unsigned
CHAR       int8                 char
FLOAT      uint64               unsigned long long (exact decimals)
DOUBLE     uint64               unsigned long long
STRING     ``StringColumn``     size_t offsets[n+1] + char heap
=========  ===================  =====================================
"""
from collections import OrderedDict

import numpy as np

from dogqc_b200.types import Type

STORAGE_DTYPE = {
    Type.INT: np.int32,
    Type.DATE: np.uint32,
    Type.CHAR: np.int8,
    Type.FLOAT: np.uint64,
    Type.DOUBLE: np.uint64,
}


class StringColumn(object):
    """Strings as a char heap plus ``n+1`` byte offsets.

    ``width`` is set when every string has the same length; the device then reads
    string ``i`` at ``chars[i*width:(i+1)*width]`` without the offsets.
    """

    def __init__(self, chars, offsets, width=0):
        self.chars = np.ascontiguousarray(chars, dtype=np.uint8)
        self.offsets = np.ascontiguousarray(offsets, dtype=np.uint64)
        self.width = int(width)

    @staticmethod
    def fixed(matrix):
        m = np.ascontiguousarray(matrix, dtype=np.uint8)
        n, w = m.shape
        offsets = np.arange(n + 1, dtype=np.uint64) * np.uint64(w)
        return StringColumn(m.reshape(-1), offsets, w)

    @staticmethod
    def from_list(strings):
        enc = [s.encode() if isinstance(s, str) else bytes(s) for s in strings]
        lens = np.array([len(s) for s in enc], dtype=np.uint64)
        offsets = np.zeros(len(enc) + 1, dtype=np.uint64)
        np.cumsum(lens, out=offsets[1:])
        chars = np.frombuffer(b"".join(enc), dtype=np.uint8) if enc else np.zeros(0, np.uint8)
        width = int(lens[0]) if len(enc) and np.all(lens == lens[0]) else 0
        return StringColumn(chars.copy(), offsets, width)

    def __len__(self):
        return len(self.offsets) - 1

    def get(self, i):
        return bytes(self.chars[int(self.offsets[i]):int(self.offsets[i + 1])])

    def __getitem__(self, i):
        if not -len(self) <= i < len(self):
            raise IndexError(i)
        return self.get(i % len(self))

    def __iter__(self):
        return iter(self.tolist())

    def tolist(self):
        heap, offs = self.chars.tobytes(), self.offsets.tolist()
        return [heap[offs[i]:offs[i + 1]] for i in range(len(offs) - 1)]

    def take(self, idx):
        idx = np.asarray(idx, dtype=np.int64)
        return [self.get(i) for i in idx]

    @property
    def nbytes(self):
        return self.chars.nbytes + self.offsets.nbytes


class Table(object):
    def __init__(self, name, columns, types):
        self.name = name
        self.columns = OrderedDict(columns)
        self.types = OrderedDict(types)
        sizes = {len(c) for c in self.columns.values()}
        if len(sizes) > 1:
            raise ValueError("table %s has columns of different lengths %s" % (name, sizes))
        self.size = sizes.pop() if sizes else 0
        for attr, col in self.columns.items():
            t = self.types[attr]
            if t == Type.STRING:
                if not isinstance(col, StringColumn):
                    raise TypeError("STRING attribute %s.%s needs a StringColumn" % (name, attr))
            else:
                want = STORAGE_DTYPE[t]
                if col.dtype != want:
                    self.columns[attr] = np.ascontiguousarray(col, dtype=want)

    def schema_entry(self):
        return {
            "name": self.name,
            "size": self.size,
            "numColumns": len(self.columns),
            "attributes": OrderedDict(self.types),
            "charSizes": {a: int(len(c.chars)) for a, c in self.columns.items()
                          if isinstance(c, StringColumn)},
        }

    @property
    def nbytes(self):
        return sum(c.nbytes for c in self.columns.values())


class Database(object):
    def __init__(self, tables=()):
        self.tables = OrderedDict()
        self.schema = {}
        for t in tables:
            self.add(t)

    def add(self, table):
        self.tables[table.name] = table
        self.schema[table.name] = table.schema_entry()
        return table

    def __getitem__(self, name):
        return self.tables[name]
