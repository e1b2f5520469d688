"""Python handle on the CUDA engine (``libdogqc_b200.so``).

``Engine`` owns one ``dq_ctx`` (one device, one stream), registers tables and
prepares plans; ``Plan.execute`` runs a plan and returns a ``Result`` of numpy
columns.  Everything here goes through the C ABI; there is no CPU path.
"""
import ctypes as C

import numpy as np

from dogqc_b200 import _lib as L
from dogqc_b200.database import StringColumn
from dogqc_b200.lowering import NP_DTYPE, Lowering, lang_type


class Result(object):
    """A materialised result: column names, C types and columns (numpy arrays;
    strings as a StringColumn, whose rows become bytes on demand)."""

    def __init__(self, names, ctypes_, columns, nrows):
        self.names = list(names)
        self.ctypes = list(ctypes_)
        self.columns = columns
        self.nrows = int(nrows)

    def rows(self):
        if self.nrows == 0:
            return []
        return list(zip(*[c.tolist() for c in self.columns]))

    def column(self, name):
        return self.columns[self.names.index(name)]

    def format_sample(self, limit=10):
        """The reference's console summary (cudaTranslator.py:607-643)."""
        out = ["", "Result: %i tuples" % self.nrows]
        for i in range(min(limit, self.nrows)):
            parts = []
            for n, t, c in zip(self.names, self.ctypes, self.columns):
                v = c[i]
                if t == L.STR:
                    s = v.decode(errors="replace")
                elif t == L.I8:
                    s = chr(int(v) & 0xFF)
                elif t == L.U64:
                    s = "%10d" % int(v)
                elif t == L.U32:
                    s = "%10d" % int(v)
                else:
                    s = "%8d" % int(v)
                parts.append("%s: %s" % (n, s))
            out.append("  ".join(parts) + "  ")
        if self.nrows > limit:
            out.append("[...]")
        return "\n".join(out) + "\n"


def _take_result(res, names):
    """Copies a dq_result into a Result and frees it."""
    lib = L.lib()
    try:
        n = C.c_int64()
        nc = C.c_int32()
        L.check(lib.dq_result_rows(res, C.byref(n)))
        L.check(lib.dq_result_ncols(res, C.byref(nc)))
        cols, types = [], []
        for j in range(nc.value):
            t = C.c_int32()
            ptr = C.c_void_p()
            L.check(lib.dq_result_column(res, j, C.byref(t), C.byref(ptr)))
            if t.value == L.STR:  # offsets into a heap, kept as a StringColumn (bytes per row on demand)
                offs = np.frombuffer((C.c_uint8 * ((n.value + 1) * 8)).from_address(ptr.value), np.uint64).copy()
                hp, nch = C.c_void_p(), C.c_uint64()
                L.check(lib.dq_result_string_heap(res, j, C.byref(hp), C.byref(nch)))
                heap = C.string_at(hp.value, nch.value) if nch.value else b""
                cols.append(StringColumn(np.frombuffer(heap, dtype=np.uint8), offs))
                types.append(t.value)
                continue
            dt = np.dtype(NP_DTYPE[t.value])
            if n.value:
                buf = (C.c_uint8 * (n.value * dt.itemsize)).from_address(ptr.value)
                cols.append(np.frombuffer(buf, dtype=dt).copy())
            else:
                cols.append(np.zeros(0, dtype=dt))
            types.append(t.value)
    finally:
        lib.dq_result_free(res)
    return Result(names, types, cols, n.value)


def make_tuning(tuning):
    """A dq_tuning from a dict (keys are the struct's fields) or None."""
    if tuning is None:
        return None
    if isinstance(tuning, L.dq_tuning):
        return tuning
    t = L.dq_tuning()
    for k, v in dict(tuning).items():
        setattr(t, k, int(v))
    return t


class Plan(object):
    def __init__(self, engine, lowering, tuning=None):
        self.engine = engine
        self.lowering = lowering
        desc, keep = lowering.ir()
        handle = C.c_void_p()
        t = make_tuning(tuning)
        if t is None:
            L.check(L.lib().dq_plan_prepare(engine.ctx, C.byref(desc), C.byref(handle)), engine.ctx)
        else:
            L.check(L.lib().dq_plan_prepare_tuned(engine.ctx, C.byref(desc), C.byref(t), C.byref(handle)), engine.ctx)
        self.handle = handle

    def execute(self, stream=None):
        res = C.c_void_p()
        L.check(L.lib().dq_plan_execute(self.handle, stream, C.byref(res)), self.engine.ctx)
        return _take_result(res, self.lowering.result_names)

    def source(self, pipe):
        """Generated CUDA source of pipeline ``pipe`` with the compiler's
        register report (None when the pipeline runs on a prebuilt kernel)."""
        lib = L.lib()
        n = C.c_int64()
        st = lib.dq_plan_source(self.handle, pipe, None, 0, C.byref(n))
        if st == L.ERR_NOT_FOUND:
            return None
        L.check(st, self.engine.ctx)
        buf = C.create_string_buffer(n.value + 1)
        L.check(lib.dq_plan_source(self.handle, pipe, buf, n.value + 1, C.byref(n)), self.engine.ctx)
        return buf.value.decode()

    def dependencies(self, pipe):
        """The earlier pipelines ``pipe`` waits for in a replayed run (the
        others may run beside it)."""
        out = (C.c_int32 * len(self.lowering.pipes))()
        n = C.c_int32()
        L.check(L.lib().dq_plan_dependencies(self.handle, pipe, out, len(out), C.byref(n)), self.engine.ctx)
        return list(out[:n.value])

    def profile(self, point):
        """Lane-activity histogram of profile point ``point`` in the last
        execute: 33 counts, warp steps with 0..32 active lanes."""
        counts = (C.c_uint64 * 33)()
        L.check(L.lib().dq_plan_profile(self.handle, point, counts), self.engine.ctx)
        return list(counts)

    def timing(self):
        t = L.dq_plan_timing()
        L.check(L.lib().dq_plan_timing_get(self.handle, C.byref(t)))
        return {"total_ms": t.total_ms, "max_pipeline_ms": t.max_pipeline_ms,
                "max_pipeline": t.max_pipeline, "kernel_launches": t.kernel_launches,
                "pipeline_ms": [t.pipeline_ms[i] for i in range(len(self.lowering.pipes))]}

    def free(self):
        if self.handle:
            L.lib().dq_plan_free(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


class Batch(object):
    """Many instances of one plan shape executed together (dq_batch_*): one
    generated kernel per pipeline over all instances, under one CUDA graph.
    ``lowerings`` are the instances' lowered plans, each naming its own tables."""

    def __init__(self, engine, lowerings, tuning=None):
        self.engine = engine
        self.lowerings = list(lowerings)
        irs = [lw.ir() for lw in self.lowerings]
        self._keep = irs
        arr = (L.dq_plan_desc * len(irs))(*[d for d, _ in irs])
        self._arr = arr
        handle = C.c_void_p()
        t = make_tuning(tuning)
        L.check(L.lib().dq_batch_prepare(engine.ctx, len(irs), arr, C.byref(t) if t is not None else None,
                                         C.byref(handle)), engine.ctx)
        self.handle = handle

    def __len__(self):
        return len(self.lowerings)

    def execute(self, stream=None):
        n = len(self.lowerings)
        out = (C.c_void_p * n)()
        L.check(L.lib().dq_batch_execute(self.handle, stream, out), self.engine.ctx)
        return [_take_result(C.c_void_p(out[i]), self.lowerings[i].result_names) for i in range(n)]

    def profile(self, point):
        """Lane-activity histogram of profile point ``point`` in the last
        execute: 33 counts, warp steps with 0..32 active lanes."""
        counts = (C.c_uint64 * 33)()
        L.check(L.lib().dq_plan_profile(self.handle, point, counts), self.engine.ctx)
        return list(counts)

    def timing(self):
        t = L.dq_plan_timing()
        L.check(L.lib().dq_batch_timing_get(self.handle, C.byref(t)))
        return {"total_ms": t.total_ms, "kernel_launches": t.kernel_launches}

    def free(self):
        if self.handle:
            L.lib().dq_batch_free(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


class Engine(object):
    """One device context.  ``register_database`` uploads host tables once."""

    def __init__(self, device=0, tile_rows=0, ctas_per_sm=0, flags=0, defer_threshold=0):
        cfg = L.dq_config()
        cfg.abi_version = L.ABI_VERSION
        cfg.device = device
        cfg.tile_rows = tile_rows
        cfg.ctas_per_sm = ctas_per_sm
        cfg.flags = flags
        cfg.defer_threshold = defer_threshold
        handle = C.c_void_p()
        L.check(L.lib().dq_init(C.byref(cfg), C.byref(handle)))
        self.ctx = handle
        self.device = device
        self.registered = {}

    @staticmethod
    def _columns(table):
        cols, keep = [], []
        for name, col in table.columns.items():
            c = L.dq_column()
            nb = name.encode()
            keep.append(nb)
            c.name = nb
            t = lang_type(table.types[name])
            c.ctype = {"i8": L.I8, "i32": L.I32, "u32": L.U32, "u64": L.U64, "str": L.STR}[t]
            if isinstance(col, StringColumn):
                keep += [col.chars, col.offsets]
                c.width = col.width
                c.data = col.chars.ctypes.data if len(col.chars) else None
                c.offsets = col.offsets.ctypes.data
                c.nchars = len(col.chars)
            else:
                arr = np.ascontiguousarray(col)
                keep.append(arr)
                c.data = arr.ctypes.data if len(arr) else None
            cols.append(c)
        arr = (L.dq_column * max(len(cols), 1))(*cols)
        return arr, len(cols), keep

    def register_table(self, table):
        arr, n, keep = self._columns(table)
        L.check(L.lib().dq_table_register(self.ctx, table.name.encode(), n, arr, table.size, 0), self.ctx)
        self.registered[table.name] = table

    def register_database(self, db, force=False):
        for name, table in db.tables.items():
            if force or self.registered.get(name) is not table:
                self.register_table(table)

    def update_table(self, table, stream=None):
        """Copy new host values of a registered table's columns to the device."""
        arr, n, keep = self._columns(table)
        L.check(L.lib().dq_table_update(self.ctx, table.name.encode(), n, arr, table.size, stream), self.ctx)

    def import_text(self, name, text, fields, delim="|"):
        """Parse ``.tbl`` text on the device into the table ``name``.

        ``text``: bytes, or a device tensor of uint8 (``data_ptr`` is read);
        ``fields``: (column name, kind[, scale]) per field, kind one of
        ``L.TEXT_*`` (``None`` name for ``TEXT_SKIP``).  Returns the rows."""
        arr = (L.dq_text_field * max(len(fields), 1))()
        keep = []
        for i, fd in enumerate(fields):
            nm = fd[0].encode() if fd[0] else None
            keep.append(nm)
            arr[i].name = nm
            arr[i].kind = fd[1]
            arr[i].scale = fd[2] if len(fd) > 2 else 0
        if hasattr(text, "data_ptr"):
            ptr, nbytes = text.data_ptr(), int(text.numel())
        else:
            buf = C.create_string_buffer(bytes(text), len(text))
            keep.append(buf)
            ptr, nbytes = C.addressof(buf), len(text)
        nrows = C.c_int64()
        L.check(L.lib().dq_table_import_text(self.ctx, name.encode(), ptr, nbytes, delim.encode(), len(fields),
                                             arr, C.byref(nrows)), self.ctx)
        self.registered.pop(name, None)
        return nrows.value

    def import_timing(self):
        """Phase times of the last ``import_text`` (dict; device ms from CUDA
        events, ``call_ms`` the host time of the whole call)."""
        t = L.dq_import_timing()
        L.check(L.lib().dq_table_import_timing_get(self.ctx, C.byref(t)), self.ctx)
        return {name: getattr(t, name) for name, _ in t._fields_}

    def read_column(self, table, column, ctype=None):
        """A registered column copied back to the host: a numpy array of the
        column's type ``ctype`` (``L.I8``, ``L.I32``, ``L.U32``, ``L.I64``,
        ``L.U64``), or for ``L.STR`` the pair (heap bytes, uint64 offsets)."""
        nrows = C.c_int64()
        L.check(L.lib().dq_table_rows(self.ctx, table.encode(), C.byref(nrows)), self.ctx)
        n = nrows.value
        if ctype == L.STR:
            nch = C.c_uint64()
            L.check(L.lib().dq_table_column_read(self.ctx, table.encode(), column.encode(), None, 0, None,
                                                 C.byref(nch)), self.ctx)
            chars = np.zeros(max(nch.value, 1), np.uint8)
            offs = np.zeros(n + 1, np.uint64)
            L.check(L.lib().dq_table_column_read(self.ctx, table.encode(), column.encode(), chars.ctypes.data,
                                                 chars.nbytes, offs.ctypes.data, C.byref(nch)), self.ctx)
            return chars[:nch.value], offs
        out = np.zeros(max(n, 1), NP_DTYPE[ctype])
        L.check(L.lib().dq_table_column_read(self.ctx, table.encode(), column.encode(), out.ctypes.data,
                                             out.nbytes, None, None), self.ctx)
        return out[:n]

    def prepare(self, plan, options=None, tuning=None):
        """``tuning``: dq_tuning fields as a dict (see dogqc_b200.autotune)."""
        lowering = plan if isinstance(plan, Lowering) else Lowering(plan, options)
        return Plan(self, lowering, tuning)

    def prepare_batch(self, lowerings, tuning=None):
        return Batch(self, lowerings, tuning)

    def close(self):
        if self.ctx:
            L.lib().dq_shutdown(self.ctx)
            self.ctx = None


_default = {}


def default_engine(device=0):
    if device not in _default:
        _default[device] = Engine(device)
    return _default[device]
