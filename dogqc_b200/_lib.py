"""ctypes binding of ``libdogqc_b200.so`` (declarations in include/dogqc_b200.h).

The structures below mirror the header field by field; ``check_layout`` compares
their sizes with the values the header implies.  Loading fails loudly when the
library is missing: there is no fallback implementation.
"""
import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libdogqc_b200.so")

ABI_VERSION = 1
MAX_COLS, MAX_SLOTS, MAX_OPS, MAX_LIST = 16, 64, 48, 192
MAX_KEYS, MAX_PAY, MAX_AGGS, MAX_LEVELS, MAX_PATTERNS = 4, 16, 16, 3, 8

# dq_status
OK, ERR_INVALID, ERR_CUDA, ERR_OOM, ERR_HT_FULL, ERR_TIMEOUT = 0, -1, -2, -3, -4, -5
ERR_BAD_IR, ERR_ADMISSION, ERR_NOT_FOUND, ERR_OVERFLOW, ERR_UNSUPPORTED = -6, -7, -8, -9, -10
STATUS_NAMES = {0: "OK", -1: "INVALID", -2: "CUDA", -3: "OOM", -4: "HT_FULL", -5: "TIMEOUT",
                -6: "BAD_IR", -7: "ADMISSION", -8: "NOT_FOUND", -9: "OVERFLOW", -10: "UNSUPPORTED"}

# dq_ctype
I8, I32, U32, I64, U64, STR = 1, 2, 3, 4, 5, 6
CTYPE_NAMES = {"i8": I8, "i32": I32, "u32": U32, "i64": I64, "u64": U64, "str": STR}
WIDTH = {I8: 1, I32: 4, U32: 4, I64: 8, U64: 8}

# dq_slot_kind
SLOT_COL, SLOT_REG, SLOT_GATHER, SLOT_AGGKEY, SLOT_AGGVAL, SLOT_STR = 1, 2, 3, 4, 5, 6
# dq_op_kind
OP_ARITH, OP_CMP, OP_LOGIC, OP_CAST, OP_SELECT, OP_LIKE, OP_STREQ, OP_STRREF = 1, 2, 3, 4, 5, 6, 7, 8
OP_PROFILE, OP_FILTER, OP_PROBE, OP_EXPAND, OP_EXISTS, OP_SUBSTR = 9, 10, 11, 12, 13, 14
OP_AGG, OP_BUILD, OP_MM_COUNT, OP_MM_SCATTER, OP_EMIT = 20, 21, 22, 23, 24
ADD, SUB, MUL, DIV, MOD = 1, 2, 3, 4, 5
EQ, NE, LT, LE, GT, GE = 1, 2, 3, 4, 5, 6
AND, OR, NOT = 1, 2, 3
JOIN_INNER, JOIN_SEMI, JOIN_ANTI = 1, 2, 3
RED_SUM, RED_COUNT, RED_MIN, RED_MAX = 1, 2, 3, 4
OPF_B_IMM, OPF_A_IMM = 1, 2
RES_UNIQUE, RES_MULTI, RES_AGG, RES_OUTPUT = 1, 2, 3, 4
SRC_TABLE, SRC_OUTPUT, SRC_AGG = 1, 2, 3
TABLE_DEVICE_DATA = 1
CFG_NO_TMA, CFG_NO_GRAPH, CFG_ROW_KERNEL, CFG_NO_JIT, CFG_OFFLINE = 1, 2, 4, 8, 16


class dq_config(C.Structure):
    _fields_ = [("abi_version", C.c_int32), ("device", C.c_int32), ("memory_budget", C.c_uint64),
                ("block_threads", C.c_int32), ("tile_rows", C.c_int32), ("ctas_per_sm", C.c_int32),
                ("flags", C.c_int32), ("defer_threshold", C.c_int32), ("reserved", C.c_int32)]


class dq_column(C.Structure):
    _fields_ = [("name", C.c_char_p), ("ctype", C.c_int32), ("width", C.c_int32), ("data", C.c_void_p),
                ("offsets", C.c_void_p), ("nchars", C.c_uint64)]


TEXT_INT, TEXT_DATE, TEXT_CHAR, TEXT_DECIMAL, TEXT_STRING, TEXT_SKIP, TEXT_FLOAT = 1, 2, 3, 4, 5, 6, 7


class dq_text_field(C.Structure):
    _fields_ = [("name", C.c_char_p), ("kind", C.c_int32), ("scale", C.c_int32)]


class dq_import_timing(C.Structure):
    _fields_ = [("copy_ms", C.c_double), ("newline_ms", C.c_double), ("line_end_ms", C.c_double),
                ("parse_ms", C.c_double), ("string_ms", C.c_double), ("call_ms", C.c_double),
                ("span_ms", C.c_double),
                ("kernel_launches", C.c_int64), ("nbytes", C.c_uint64)]


class dq_slot(C.Structure):
    _fields_ = [("kind", C.c_int8), ("level", C.c_int8), ("ctype", C.c_int8), ("pad", C.c_int8),
                ("src", C.c_int16), ("res", C.c_int16)]


class dq_op(C.Structure):
    _fields_ = [("kind", C.c_int16), ("sub", C.c_int16), ("dst", C.c_int16), ("a", C.c_int16),
                ("b", C.c_int16), ("c", C.c_int16), ("ctype", C.c_int8), ("flags", C.c_int8),
                ("res", C.c_int16), ("list", C.c_int16), ("nlist", C.c_int16), ("list2", C.c_int16),
                ("nlist2", C.c_int16), ("pad", C.c_int16), ("imm", C.c_int64)]


class dq_resource(C.Structure):
    _fields_ = [("kind", C.c_int32), ("nkeys", C.c_int32), ("key_ctype", C.c_int8 * MAX_KEYS),
                ("npay", C.c_int32), ("pay_ctype", C.c_int8 * MAX_PAY), ("naggs", C.c_int32),
                ("agg_red", C.c_int8 * MAX_AGGS), ("capacity", C.c_int64), ("group_hint", C.c_int64),
                ("name", C.c_char_p)]


class dq_pipeline(C.Structure):
    _fields_ = [("source_kind", C.c_int32), ("source_res", C.c_int32), ("table", C.c_char_p),
                ("ncols", C.c_int32), ("cols", C.c_char_p * MAX_COLS), ("nslots", C.c_int32),
                ("slots", dq_slot * MAX_SLOTS), ("nops", C.c_int32), ("ops", dq_op * MAX_OPS),
                ("nlist", C.c_int32), ("lists", C.c_int16 * MAX_LIST), ("npatterns", C.c_int32),
                ("patterns", C.c_char_p * MAX_PATTERNS), ("compact", C.c_int32)]


class dq_plan_desc(C.Structure):
    _fields_ = [("abi_version", C.c_int32), ("nres", C.c_int32), ("res", C.POINTER(dq_resource)),
                ("npipes", C.c_int32), ("pipes", C.POINTER(dq_pipeline)), ("result_res", C.c_int32)]


class dq_plan_timing(C.Structure):
    _fields_ = [("total_ms", C.c_double), ("max_pipeline_ms", C.c_double), ("max_pipeline", C.c_int32),
                ("kernel_launches", C.c_int32), ("pipeline_ms", C.c_double * MAX_OPS)]


class dq_tuning(C.Structure):
    _fields_ = [("rows_per_thread", C.c_int32), ("block_threads", C.c_int32), ("refill", C.c_int32),
                ("unique_slots_pct", C.c_int32), ("multi_buckets_pct", C.c_int32), ("refill_threshold", C.c_int32),
                ("defer_threshold", C.c_int32), ("ctas_per_sm", C.c_int32)]


class dq_server_config(C.Structure):
    _fields_ = [("slots", C.c_int32), ("pool_per_query", C.c_int32), ("memory_budget", C.c_uint64),
                ("batch_max", C.c_int32), ("batch_rows_max", C.c_int32), ("reserved", C.c_int32 * 2)]


class dq_request_info(C.Structure):
    _fields_ = [("queue_ms", C.c_double), ("run_ms", C.c_double), ("total_ms", C.c_double), ("bytes", C.c_uint64),
                ("status", C.c_int32), ("kernel_launches", C.c_int32)]


class dq_server_stats(C.Structure):
    _fields_ = [("submitted", C.c_uint64), ("completed", C.c_uint64), ("failed", C.c_uint64),
                ("memory_in_use", C.c_uint64), ("memory_peak", C.c_uint64), ("p50_ms", C.c_double),
                ("p99_ms", C.c_double), ("mean_ms", C.c_double), ("span_ms", C.c_double),
                ("batches", C.c_uint64), ("batched", C.c_uint64)]


NOALLOC_MAX_BUILD_ROWS = 262144
NOALLOC_MAX_GROUPS = 4096


class dq_join_agg_args(C.Structure):
    _fields_ = [("build_key", C.c_void_p), ("build_filter", C.c_void_p), ("filter_value", C.c_int32),
                ("build_group", C.c_void_p), ("build_rows", C.c_int64), ("probe_key", C.c_void_p),
                ("probe_value", C.c_void_p), ("probe_rows", C.c_int64), ("out_group", C.c_void_p),
                ("out_sum", C.c_void_p), ("out_count", C.c_void_p), ("out_ngroups", C.c_void_p),
                ("max_groups", C.c_int32)]


def check_layout():
    """Sizes the C compiler gives these structs on x86-64 (LP64)."""
    expect = {dq_config: 40, dq_column: 40, dq_slot: 8, dq_op: 40, dq_resource: 80, dq_join_agg_args: 104,
              dq_tuning: 32, dq_server_config: 32, dq_request_info: 40, dq_server_stats: 88,
              dq_text_field: 16, dq_import_timing: 72}
    for t, n in expect.items():
        if C.sizeof(t) != n:
            raise AssertionError("%s is %d bytes, header implies %d" % (t.__name__, C.sizeof(t), n))


class DqError(RuntimeError):
    def __init__(self, status, message):
        RuntimeError.__init__(self, "%s (%d): %s" % (STATUS_NAMES.get(status, "?"), status, message))
        self.status = status


_lib = None

EXPORTS = {
    "dq_version": (C.c_int, []),
    "dq_last_error": (C.c_char_p, [C.c_void_p]),
    "dq_init": (C.c_int, [C.POINTER(dq_config), C.POINTER(C.c_void_p)]),
    "dq_shutdown": (None, [C.c_void_p]),
    "dq_table_register": (C.c_int, [C.c_void_p, C.c_char_p, C.c_int32, C.POINTER(dq_column), C.c_int64, C.c_int32]),
    "dq_table_update": (C.c_int, [C.c_void_p, C.c_char_p, C.c_int32, C.POINTER(dq_column), C.c_int64, C.c_void_p]),
    "dq_table_drop": (C.c_int, [C.c_void_p, C.c_char_p]),
    "dq_table_rows": (C.c_int, [C.c_void_p, C.c_char_p, C.POINTER(C.c_int64)]),
    "dq_table_import_text": (C.c_int, [C.c_void_p, C.c_char_p, C.c_void_p, C.c_uint64, C.c_char, C.c_int32,
                                       C.POINTER(dq_text_field), C.POINTER(C.c_int64)]),
    "dq_table_import_timing_get": (C.c_int, [C.c_void_p, C.POINTER(dq_import_timing)]),
    "dq_table_column_read": (C.c_int, [C.c_void_p, C.c_char_p, C.c_char_p, C.c_void_p, C.c_uint64,
                                       C.c_void_p, C.POINTER(C.c_uint64)]),
    "dq_plan_prepare": (C.c_int, [C.c_void_p, C.POINTER(dq_plan_desc), C.POINTER(C.c_void_p)]),
    "dq_plan_execute": (C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(C.c_void_p)]),
    "dq_plan_free": (None, [C.c_void_p]),
    "dq_plan_source": (C.c_int, [C.c_void_p, C.c_int32, C.c_char_p, C.c_int64, C.POINTER(C.c_int64)]),
    "dq_plan_dependencies": (C.c_int, [C.c_void_p, C.c_int32, C.POINTER(C.c_int32), C.c_int32,
                                       C.POINTER(C.c_int32)]),
    "dq_plan_profile": (C.c_int, [C.c_void_p, C.c_int32, C.POINTER(C.c_uint64)]),
    "dq_plan_timing_get": (C.c_int, [C.c_void_p, C.POINTER(dq_plan_timing)]),
    "dq_result_rows": (C.c_int, [C.c_void_p, C.POINTER(C.c_int64)]),
    "dq_result_ncols": (C.c_int, [C.c_void_p, C.POINTER(C.c_int32)]),
    "dq_result_column": (C.c_int, [C.c_void_p, C.c_int32, C.POINTER(C.c_int32), C.POINTER(C.c_void_p)]),
    "dq_result_string_heap": (C.c_int, [C.c_void_p, C.c_int32, C.POINTER(C.c_void_p), C.POINTER(C.c_uint64)]),
    "dq_result_free": (None, [C.c_void_p]),
    "dq_join_agg_noalloc": (C.c_int, [C.POINTER(dq_join_agg_args), C.c_void_p]),
    "dq_plan_prepare_tuned": (C.c_int, [C.c_void_p, C.POINTER(dq_plan_desc), C.POINTER(dq_tuning),
                                        C.POINTER(C.c_void_p)]),
    "dq_batch_prepare": (C.c_int, [C.c_void_p, C.c_int32, C.POINTER(dq_plan_desc), C.POINTER(dq_tuning),
                                   C.POINTER(C.c_void_p)]),
    "dq_batch_execute": (C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(C.c_void_p)]),
    "dq_batch_timing_get": (C.c_int, [C.c_void_p, C.POINTER(dq_plan_timing)]),
    "dq_batch_size": (C.c_int, [C.c_void_p, C.POINTER(C.c_int32)]),
    "dq_batch_free": (None, [C.c_void_p]),
    "dq_server_start": (C.c_int, [C.c_void_p, C.POINTER(dq_server_config), C.POINTER(C.c_void_p)]),
    "dq_server_submit": (C.c_int, [C.c_void_p, C.POINTER(dq_plan_desc), C.POINTER(C.c_uint64)]),
    "dq_server_wait": (C.c_int, [C.c_void_p, C.c_uint64, C.POINTER(C.c_void_p), C.POINTER(dq_request_info)]),
    "dq_server_stats_get": (C.c_int, [C.c_void_p, C.POINTER(dq_server_stats)]),
    "dq_server_stop": (None, [C.c_void_p]),
    "dq_server_replay": (C.c_int, [C.c_void_p, C.c_int32, C.POINTER(dq_plan_desc), C.c_int64,
                                   C.POINTER(C.c_double), C.POINTER(C.c_int32), C.POINTER(dq_request_info)]),
    "dq_plan_run_sequence": (C.c_int, [C.POINTER(C.c_void_p), C.c_int32, C.c_int64, C.POINTER(C.c_int32),
                                       C.POINTER(C.c_double)]),
}


def lib():
    """The loaded library (raises if it was not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError("libdogqc_b200.so is not built (run python -m dogqc_b200.build)")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in EXPORTS.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        check_layout()
        _lib = L
    return _lib


def check(status, ctx=None):
    if status != OK:
        msg = lib().dq_last_error(ctx)
        raise DqError(status, msg.decode() if msg else "")
