"""Multithreaded C++ evaluation of a lowered plan on the host's cores.

Test infrastructure and the timed CPU baseline: the tests pin it against the
reference's golden fixtures, and the bench times it beside the device engine
(its ``cpu_baseline`` leg and ``--impl reference`` arm).  The product never
loads it.  ``oracle/cpu_eval.cpp`` evaluates the same plan IR the device
engine prepares (``Lowering(plan).ir()``), row at a time over morsels taken by
worker threads; ``build()`` compiles it with g++ into ``oracle/_build``.
"""
import ctypes as C
import os
import subprocess
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "cpu_eval.cpp")
OUT = os.path.join(HERE, "_build", "libdq_cpu.so")

_lib = None


def build(force=False):
    """Compiles the evaluator (g++ -O3, portable code: the library travels to
    other hosts) when its source is newer than the library."""
    if not force and os.path.exists(OUT) and os.path.getmtime(OUT) >= max(
            os.path.getmtime(SRC), os.path.getmtime(os.path.join(HERE, "..", "include", "dogqc_b200.h"))):
        return OUT
    os.makedirs(os.path.dirname(OUT), exist_ok=True)
    tmp = OUT + ".tmp"
    cmd = ["g++", "-O3", "-std=c++17", "-fPIC", "-shared", "-pthread", "-o", tmp, SRC]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("g++ failed:\n" + r.stderr[-4000:])
    os.replace(tmp, OUT)
    return OUT


class dqcpu_table(C.Structure):
    _fields_ = [("name", C.c_char_p), ("ncols", C.c_int32), ("cols", C.c_void_p), ("nrows", C.c_int64)]


def lib():
    global _lib
    if _lib is None:
        _lib = C.CDLL(build())
        _lib.dqcpu_run.argtypes = [C.c_void_p, C.c_int32, C.c_void_p, C.c_int32, C.POINTER(C.c_void_p)]
        _lib.dqcpu_last_error.restype = C.c_char_p
        _lib.dqcpu_result_shape.argtypes = [C.c_void_p, C.POINTER(C.c_int64), C.POINTER(C.c_int32)]
        _lib.dqcpu_result_column.argtypes = [C.c_void_p, C.c_int32, C.POINTER(C.c_int32), C.POINTER(C.c_void_p),
                                             C.POINTER(C.c_void_p), C.POINTER(C.c_uint64)]
        _lib.dqcpu_result_free.argtypes = [C.c_void_p]
    return _lib


def default_threads():
    return len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else (os.cpu_count() or 1)


class Prepared(object):
    """A plan lowered once, with the host tables it scans, ready to run."""

    def __init__(self, db, plan, threads=None):
        from dogqc_b200.engine import Engine
        from dogqc_b200.lowering import Lowering
        self.lowering = Lowering(plan)
        self.desc, self._keep = self.lowering.ir()
        self.names = self.lowering.result_names
        read = {p.table for p in self.lowering.pipes if p.table}
        tabs = []
        self._cols = []
        for name, table in db.tables.items():
            if name not in read:
                continue
            arr, n, keep = Engine._columns(table)
            self._cols.append((arr, keep))
            b = name.encode()
            self._cols.append(b)
            tabs.append(dqcpu_table(b, n, C.cast(arr, C.c_void_p), table.size))
        self.tables = (dqcpu_table * max(len(tabs), 1))(*tabs)
        self.ntables = len(tabs)
        self.threads = threads or default_threads()

    def run(self):
        """(column names, rows as tuples, seconds of the evaluation)."""
        L = lib()
        out = C.c_void_p()
        t0 = time.perf_counter()
        st = L.dqcpu_run(C.addressof(self.desc), self.ntables, C.cast(self.tables, C.c_void_p), self.threads,
                         C.byref(out))
        dt = time.perf_counter() - t0
        if st != 0:
            raise RuntimeError("CPU evaluation failed: %s" % L.dqcpu_last_error().decode())
        try:
            return self.names, _rows(L, out), dt
        finally:
            L.dqcpu_result_free(out)


_NP = {1: np.int8, 2: np.int32, 3: np.uint32, 4: np.int64, 5: np.uint64}


def _rows(L, res):
    n, nc = C.c_int64(), C.c_int32()
    L.dqcpu_result_shape(res, C.byref(n), C.byref(nc))
    cols = []
    for j in range(nc.value):
        t, vals, heap, nch = C.c_int32(), C.c_void_p(), C.c_void_p(), C.c_uint64()
        L.dqcpu_result_column(res, j, C.byref(t), C.byref(vals), C.byref(heap), C.byref(nch))
        if t.value == 6:
            offs = np.ctypeslib.as_array((C.c_uint64 * (n.value + 1)).from_address(vals.value)).copy()
            data = C.string_at(heap.value, nch.value) if nch.value else b""
            cols.append([data[int(offs[i]):int(offs[i + 1])] for i in range(n.value)])
        else:
            if n.value:
                v = np.ctypeslib.as_array((C.c_uint64 * n.value).from_address(vals.value)).copy()
            else:
                v = np.zeros(0, dtype=np.uint64)
            cols.append(v.astype(_NP[t.value]).tolist())
    return list(zip(*cols)) if n.value else []


def run_plan(db, plan, threads=None):
    """(names, rows) of a resolved plan, like the numpy oracle's run_plan."""
    names, rows, _ = Prepared(db, plan, threads).run()
    return names, rows
