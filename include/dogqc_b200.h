/*
 * dogqc_b200 — C ABI of the B200 execution backend for DogQC relational plans.
 *
 * The reference has no runtime library: its Python translator emits one CUDA
 * source file per query whose generated main() maps column files, allocates
 * device memory, launches the pipeline kernels and prints the result
 * (dogqc/codegen.py:121-159, dogqc/cudaTranslator.py:31-101).  This header is the
 * boundary that replaces that generated host program.  A caller (the Python
 * Backend in dogqc_b200/backend.py, or any FFI binding) registers device-resident
 * tables, hands a lowered plan (the IR below) to dq_plan_prepare, runs it with
 * dq_plan_execute and reads result columns.  Every entry point returns a status
 * (0 = OK, negative dq_status on error, message in dq_last_error); nothing calls
 * exit() or prints, unlike the reference's ERROR macro (dogqc/include/util.h:1-5)
 * and device printf on full hash tables (dogqc/include/hashing.cuh:96,117,267).
 *
 * Plain C types only: no CUDA or torch types appear in the signatures (streams
 * are passed as void*).
 */
#ifndef DOGQC_B200_H
#define DOGQC_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define DQ_ABI_VERSION 1

/* ---------------------------------------------------------------- status -- */
typedef enum {
    DQ_OK = 0,
    DQ_ERR_INVALID = -1,     /* bad argument                                   */
    DQ_ERR_CUDA = -2,        /* CUDA runtime error                             */
    DQ_ERR_OOM = -3,         /* device allocation failed                       */
    DQ_ERR_HT_FULL = -4,     /* a hash table stayed full after resizing        */
    DQ_ERR_TIMEOUT = -5,     /* a bounded device wait gave up                  */
    DQ_ERR_BAD_IR = -6,      /* plan IR failed validation                      */
    DQ_ERR_ADMISSION = -7,   /* serving: query rejected by the memory budget   */
    DQ_ERR_NOT_FOUND = -8,   /* unknown table / column / ticket                */
    DQ_ERR_OVERFLOW = -9,    /* an output stayed larger than its allocation    */
    DQ_ERR_UNSUPPORTED = -10 /* plan uses a feature this build does not have   */
} dq_status;

/* C value types of columns and plan values.  They mirror the reference's type
 * map (dogqc/codegen.py:37-45) with decimals in exact 64-bit integers:
 * INT -> I32, DATE -> U32, CHAR -> I8, FLOAT/DOUBLE -> U64, STRING -> STR.    */
typedef enum {
    DQ_I8 = 1, DQ_I32 = 2, DQ_U32 = 3, DQ_I64 = 4, DQ_U64 = 5, DQ_STR = 6
} dq_ctype;

typedef struct dq_ctx dq_ctx;
typedef struct dq_plan dq_plan;
typedef struct dq_result dq_result;
typedef struct dq_batch dq_batch;

typedef struct {
    int32_t abi_version;        /* DQ_ABI_VERSION                               */
    int32_t device;             /* CUDA device ordinal                          */
    uint64_t memory_budget;     /* bytes the context may hold (0 = no limit)    */
    int32_t block_threads;      /* pipeline kernel block size (0 = default 256) */
    int32_t tile_rows;          /* rows per tile (0 = default)                  */
    int32_t ctas_per_sm;        /* persistent CTAs per SM (0 = default)         */
    int32_t flags;              /* DQ_CFG_* bits                                */
    int32_t defer_threshold;    /* expansion ranges longer than this many pairs */
                                /* are split across CTAs (0 = 8 tiles)          */
    int32_t reserved;
} dq_config;

#define DQ_CFG_NO_TMA      1    /* stage tiles with plain loads instead of TMA */
#define DQ_CFG_NO_GRAPH    2    /* do not capture CUDA graphs                  */
#define DQ_CFG_ROW_KERNEL  4    /* run pipelines without a multimap expansion  */
                                /* on the row-at-a-time kernel                 */
#define DQ_CFG_NO_JIT      8    /* run every pipeline on the prebuilt tile      */
                                /* kernel instead of a generated one           */
#define DQ_CFG_OFFLINE     16   /* no device: tables are metadata only, plans   */
                                /* are lowered and their kernels compiled but  */
                                /* cannot execute (ahead-of-time checking)     */

/* ------------------------------------------------------------- contexts -- */
int dq_init(const dq_config* cfg, dq_ctx** out);
void dq_shutdown(dq_ctx* ctx);
const char* dq_last_error(dq_ctx* ctx);      /* NULL ctx: last init error      */
int dq_version(void);

/* --------------------------------------------------------------- tables -- */
/* One column to register.  Fixed-width types: `data` holds nrows values.
 * Strings: `data` is the char heap of `nchars` bytes and `offsets` holds
 * nrows+1 byte offsets (the reference's size_t offsets + char heap,
 * dogqc/cudaTranslator.py:263-269); with `width` > 0 every string has that
 * length and `offsets` may be NULL.                                          */
typedef struct {
    const char* name;
    int32_t ctype;              /* dq_ctype                                     */
    int32_t width;              /* string width for fixed-width strings, else 0 */
    const void* data;
    const uint64_t* offsets;
    uint64_t nchars;
} dq_column;

#define DQ_TABLE_DEVICE_DATA 1  /* pointers are device memory (else host)      */

/* Copies the columns into library-owned, padded device memory (replacing a
 * table of the same name).                                                   */
int dq_table_register(dq_ctx* ctx, const char* name, int32_t ncols, const dq_column* cols,
                      int64_t nrows, int32_t flags);
/* Overwrites the values of an existing table's columns with the same types and
 * row count from host memory (pinned memory gives full copy bandwidth).  The
 * copies are queued on `stream` (NULL: the context stream).                  */
int dq_table_update(dq_ctx* ctx, const char* name, int32_t ncols, const dq_column* cols,
                    int64_t nrows, void* stream);
int dq_table_drop(dq_ctx* ctx, const char* name);
int dq_table_rows(dq_ctx* ctx, const char* name, int64_t* nrows);

/* ------------------------------------------------------------- import -- */
/* A table from text in the reference's .tbl layout (replaces the generated
 * C++ importer of dogqc/dbio.py:117-253 and the CSV reader it drives,
 * dogqc/include/csv.h).  Lines end at '\n' (a '\r' before it is dropped; a
 * last line without '\n' counts); every line holds exactly `nfields`
 * delimiters, each field followed by one, and the text after the last one is
 * ignored; spaces around a field are trimmed.  The text is copied to the
 * device and parsed there: line ends from a per-tile newline count and its
 * prefix sum, one thread per row for the fields, string heaps from a prefix
 * sum of the lengths.  Kinds and column types:
 *   INT     -> DQ_I32, [+-]digits (empty: 0), overflow is an error;
 *   DATE    -> DQ_U32, the schema's toDate of a field of at least 10 bytes
 *              ('YYYY-MM-DD' -> YYYYMMDD, query/schema/tpch.py:9-20);
 *   CHAR    -> DQ_I8, a field of exactly one byte;
 *   DECIMAL -> DQ_I64 exact, scaled by 10^scale ([+-]digits[.digits]; digits
 *              beyond `scale` are dropped), the engine's FLOAT representation;
 *   FLOAT   -> DQ_U32 holding the IEEE binary32 bits the reference's importer
 *              stores (its float parse, step by step, rounded the same way);
 *   STRING  -> DQ_STR (offsets + heap);  SKIP: not stored.
 * A malformed row fails the call with DQ_ERR_INVALID naming its line.
 * *nrows: the rows imported.                                                 */
typedef enum {
    DQ_TEXT_INT = 1, DQ_TEXT_DATE = 2, DQ_TEXT_CHAR = 3, DQ_TEXT_DECIMAL = 4, DQ_TEXT_STRING = 5, DQ_TEXT_SKIP = 6,
    DQ_TEXT_FLOAT = 7
} dq_text_kind;
typedef struct {
    const char* name;                /* column name (ignored for DQ_TEXT_SKIP)   */
    int32_t kind;                    /* dq_text_kind                             */
    int32_t scale;                   /* DQ_TEXT_DECIMAL: digits after the point  */
} dq_text_field;
int dq_table_import_text(dq_ctx* ctx, const char* name, const char* text, uint64_t nbytes, char delim,
                         int32_t nfields, const dq_text_field* fields, int64_t* nrows);
/* Copies a registered column back to the host: fixed width -> `data`
 * (nrows values, `data_bytes` at most); strings -> the heap into `data`
 * (*nchars bytes) and nrows+1 offsets into `offsets` (may be NULL to query
 * *nchars first).                                                           */
int dq_table_column_read(dq_ctx* ctx, const char* table, const char* column, void* data, uint64_t data_bytes,
                         uint64_t* offsets, uint64_t* nchars);
/* Device time of the last import's phases (CUDA events on the context
 * stream) and the host time of the whole call.                              */
typedef struct {
    double copy_ms;                  /* text into the padded device buffer      */
    double newline_ms;               /* newline count per tile + its prefix sum */
    double line_end_ms;              /* line end positions                      */
    double parse_ms;                 /* fields, one thread per row + string sums*/
    double string_ms;                /* string offsets and heaps                */
    double call_ms;                  /* host wall time of the call              */
    double span_ms;                  /* device timeline from the first phase to */
                                     /* the last, host waits between included   */
    int64_t kernel_launches;
    uint64_t nbytes;
} dq_import_timing;
int dq_table_import_timing_get(dq_ctx* ctx, dq_import_timing* out);

/* ------------------------------------------------------------------ IR -- */
/* A plan is a list of resources (hash tables, aggregation tables, outputs)
 * and pipelines.  Each pipeline streams one source in tiles through a list of
 * operators that read and write slots (values per row), ending in one sink.
 * The Python Backend (dogqc_b200/lowering.py) produces this from the
 * reference's resolved operator tree; the produce/consume translators it
 * replaces are dogqc/cudaTranslator.py:333-668 and dogqc/hashJoins.py:12-681. */

#define DQ_MAX_COLS    16
#define DQ_MAX_SLOTS   64
#define DQ_MAX_OPS     48
#define DQ_MAX_LIST   192
#define DQ_MAX_KEYS     4
#define DQ_MAX_PAY     16
#define DQ_MAX_AGGS    16
#define DQ_MAX_LEVELS   3
#define DQ_MAX_PATTERNS 8

typedef enum {
    DQ_SLOT_COL = 1,     /* source column, staged per tile (level 0)           */
    DQ_SLOT_REG = 2,     /* computed value                                     */
    DQ_SLOT_GATHER = 3,  /* multimap payload column at an expansion level      */
    DQ_SLOT_AGGKEY = 4,  /* aggregation-table key (agg-scan source)            */
    DQ_SLOT_AGGVAL = 5,  /* aggregation-table accumulator (agg-scan source)    */
    DQ_SLOT_STR = 6      /* string source column (read in place)               */
} dq_slot_kind;

typedef struct {
    int8_t kind;         /* dq_slot_kind                                        */
    int8_t level;        /* expansion level the value lives on                  */
    int8_t ctype;        /* dq_ctype                                            */
    int8_t pad;
    int16_t src;         /* COL/STR: pipeline column; GATHER: payload column;   */
                         /* AGGKEY: key index; AGGVAL: aggregate index          */
    int16_t res;         /* resource for GATHER/AGGKEY/AGGVAL                   */
} dq_slot;

typedef enum {
    DQ_OP_ARITH = 1,     /* sub: dq_arith; dst = a (op) b in ctype             */
    DQ_OP_CMP = 2,       /* sub: dq_cmp;   dst = (a cmp b) in ctype, as I32     */
    DQ_OP_LOGIC = 3,     /* sub: dq_logic                                      */
    DQ_OP_CAST = 4,      /* dst = (dst type) a                                 */
    DQ_OP_SELECT = 5,    /* dst = a ? b : c (CASE arm)                         */
    DQ_OP_LIKE = 6,      /* dst = a LIKE pattern[res]; a is a string column    */
                         /* slot or a slot holding a string reference          */
    DQ_OP_STREQ = 7,     /* dst = a == pattern[res] (string constant); with    */
                         /* res = -1, dst = a == b (two string values)         */
    DQ_OP_STRREF = 8,    /* dst = reference to string slot a's value: the     */
                         /* plan's string source, a substring window and the  */
                         /* row in one 64-bit value that join keys, payloads,  */
                         /* group keys and output columns carry               */
    DQ_OP_PROFILE = 9,   /* lane-activity counter `res`: each warp step that   */
                         /* passes adds 1 to bin (active lanes, 0..32) of the  */
                         /* point's histogram (dq_plan_profile)                */
    DQ_OP_FILTER = 10,   /* keep rows with a != 0                              */
    DQ_OP_SUBSTR = 14,   /* dst = SUBSTRING(a FROM f FOR n) of reference a:    */
                         /* f = (int32_t)imm, n = (int32_t)(imm >> 32); the    */
                         /* window (f - 1 .. f - 1 + n, clamped to the string) */
                         /* must end within the string's first 255 bytes       */
    DQ_OP_PROBE = 11,    /* unique-HT probe (res); sub: dq_join                */
    DQ_OP_EXPAND = 12,   /* multimap probe (res) opening level+1               */
    DQ_OP_EXISTS = 13,   /* semi/anti probe of a multimap (res); sub: dq_join  */
                         /* (SEMI or ANTI).  list: probe keys; list2: the      */
                         /* build keys' GATHER slots one level down; the `imm` */
                         /* ops that follow compute slot `a` (the condition)   */
                         /* from gathered and current values.  The row's key   */
                         /* range is walked until a build row has equal keys   */
                         /* and a != 0; SEMI keeps the row if one did, ANTI if */
                         /* none did; the pipeline continues on this level     */
    DQ_OP_AGG = 20,      /* sink: aggregate into res                           */
    DQ_OP_BUILD = 21,    /* sink: insert into unique HT res                    */
    DQ_OP_MM_COUNT = 22, /* sink: multimap bucket counts                       */
    DQ_OP_MM_SCATTER = 23, /* sink: multimap payload scatter                   */
    DQ_OP_EMIT = 24      /* sink: append rows to output res                    */
} dq_op_kind;

typedef enum { DQ_ADD = 1, DQ_SUB = 2, DQ_MUL = 3, DQ_DIV = 4, DQ_MOD = 5 } dq_arith;
typedef enum { DQ_EQ = 1, DQ_NE = 2, DQ_LT = 3, DQ_LE = 4, DQ_GT = 5, DQ_GE = 6 } dq_cmp;
typedef enum { DQ_AND = 1, DQ_OR = 2, DQ_NOT = 3 } dq_logic;
typedef enum { DQ_JOIN_INNER = 1, DQ_JOIN_SEMI = 2, DQ_JOIN_ANTI = 3 } dq_join;
typedef enum { DQ_RED_SUM = 1, DQ_RED_COUNT = 2, DQ_RED_MIN = 3, DQ_RED_MAX = 4 } dq_reduction;

#define DQ_OPF_B_IMM 1   /* operand b is `imm` (in the op's ctype)              */
#define DQ_OPF_A_IMM 2   /* operand a is `imm`                                  */

typedef struct {
    int16_t kind;        /* dq_op_kind                                          */
    int16_t sub;         /* dq_arith / dq_cmp / dq_logic / dq_join              */
    int16_t dst, a, b, c;/* slot indices (-1 if unused)                         */
    int8_t ctype;        /* computation type                                    */
    int8_t flags;        /* DQ_OPF_*                                            */
    int16_t res;         /* resource or pattern index                           */
    int16_t list, nlist; /* keys (probe/build/agg) or emitted slots             */
    int16_t list2, nlist2; /* payload destinations / sources, agg inputs      */
    int16_t pad;
    int64_t imm;
} dq_op;

typedef enum {
    DQ_RES_UNIQUE = 1,   /* unique join hash table (multimatch = False)        */
    DQ_RES_MULTI = 2,    /* multimap: bucket counts/offsets + payload columns  */
    DQ_RES_AGG = 3,      /* aggregation table                                  */
    DQ_RES_OUTPUT = 4    /* materialised rows (result or temp table)           */
} dq_res_kind;

typedef struct {
    int32_t kind;                    /* dq_res_kind                             */
    int32_t nkeys;
    int8_t key_ctype[DQ_MAX_KEYS];
    int32_t npay;                    /* UNIQUE/MULTI payload; OUTPUT columns    */
    int8_t pay_ctype[DQ_MAX_PAY];
    int32_t naggs;
    int8_t agg_red[DQ_MAX_AGGS];     /* dq_reduction                            */
    int64_t capacity;                /* slots / buckets / rows (from estimates) */
    int64_t group_hint;              /* AGG: estimated groups                   */
    const char* name;                /* OUTPUT: temp-table name or NULL         */
} dq_resource;

typedef enum {
    DQ_SRC_TABLE = 1,    /* registered table                                    */
    DQ_SRC_OUTPUT = 2,   /* rows of an OUTPUT resource (temp table)             */
    DQ_SRC_AGG = 3       /* occupied slots of an AGG resource                   */
} dq_source_kind;

typedef struct {
    int32_t source_kind;             /* dq_source_kind                          */
    int32_t source_res;              /* OUTPUT / AGG resource                   */
    const char* table;               /* DQ_SRC_TABLE                            */
    int32_t ncols;
    const char* cols[DQ_MAX_COLS];   /* TABLE: column names; OUTPUT: indices as */
                                     /* decimal strings                         */
    int32_t nslots;
    dq_slot slots[DQ_MAX_SLOTS];
    int32_t nops;
    dq_op ops[DQ_MAX_OPS];
    int32_t nlist;
    int16_t lists[DQ_MAX_LIST];
    int32_t npatterns;
    const char* patterns[DQ_MAX_PATTERNS];  /* LIKE patterns / string constants */
    int32_t compact;                 /* k > 0: generated kernels refill lanes   */
                                     /* after op k-1 (a selective filter or    */
                                     /* probe); 0: no refill.  The tile kernel */
                                     /* compacts after every filter and probe. */
} dq_pipeline;

typedef struct {
    int32_t abi_version;
    int32_t nres;
    const dq_resource* res;
    int32_t npipes;
    const dq_pipeline* pipes;        /* executed in order                       */
    int32_t result_res;              /* OUTPUT resource returned as the result  */
} dq_plan_desc;

/* -------------------------------------------------------------- plans -- */
/* Validates the IR, lays out the plan's tables and, unless DQ_CFG_NO_JIT or
 * DQ_CFG_ROW_KERNEL is set, generates one CUDA kernel per pipeline and
 * compiles it for sm_100a (NVRTC, in process; cached by source text).  This is
 * the step where the reference writes and compiles its query source
 * (dogqc/cudaTranslator.py:31-101, dogqc/code.py:4-26).                      */
int dq_plan_prepare(dq_ctx* ctx, const dq_plan_desc* desc, dq_plan** out);
/* Generated CUDA source of pipeline `pipe` followed by the compiler's
 * register report, NUL-terminated into buf (at most cap bytes); *len is the
 * full length.  DQ_ERR_NOT_FOUND when the pipeline runs on a prebuilt kernel.
 * A small scan of an aggregation table that follows the pipeline filling it
 * runs in the last CTA of that pipeline's kernel (no launch of its own): its
 * source is that kernel's, where it is the function dq_tail.
 * The counterpart of the reference's generated query file.                 */
int dq_plan_source(dq_plan* plan, int32_t pipe, char* buf, int64_t cap, int64_t* len);
/* The earlier pipelines pipeline `pipe` waits for when a run is replayed as a
 * CUDA graph: those that write a table it reads or writes, or read a table it
 * writes (a scanned temp or aggregation table counts as written).  The others
 * may run beside it, on other streams of the graph.  At most cap indices into
 * out, ascending; *n is their count.  A result scan fused into the kernel of
 * the pipeline before it has none (it runs in that kernel).  No device work:
 * offline contexts answer too.                                              */
int dq_plan_dependencies(dq_plan* plan, int32_t pipe, int32_t* out, int32_t cap, int32_t* n);
/* Runs every pipeline in order on `stream` (NULL: the context stream) and
 * returns a new result.  Resources start every run empty.  After a
 * successful run the same launches are captured as a CUDA graph and replayed
 * by later executes while the plan's tables and launch shapes stay the same
 * (DQ_CFG_NO_GRAPH: never); an aggregation table that one pipeline alone
 * scans is reset by that scan, so the next run needs no initialising kernel. */
int dq_plan_execute(dq_plan* plan, void* stream, dq_result** out);
void dq_plan_free(dq_plan* plan);
/* Lane-activity histogram of profile point `point` (DQ_OP_PROFILE res) over
 * the last execute: counts[i] = warp steps that reached the point with i of
 * their 32 lanes active (33 bins).  The reference's LaneActivityProfiler,
 * placed by CudaCompiler.setProfilers (dogqc/cudaLaneActivityProfile.py:10-35,
 * dogqc/cudaTranslator.py:65-89).  DQ_ERR_NOT_FOUND: no such point.         */
int dq_plan_profile(dq_plan* plan, int32_t point, uint64_t* counts);

/* Device time of the last execute (CUDA events on the launching stream):
 * total, and the longest pipeline kernel with its index.  Once a plan has run
 * successfully, dq_plan_execute replays its launches from a captured CUDA
 * graph (unless the context has DQ_CFG_NO_GRAPH); a replayed run reports the
 * total only (pipeline_ms zero, max_pipeline -1).                           */
typedef struct {
    double total_ms;
    double max_pipeline_ms;
    int32_t max_pipeline;
    int32_t kernel_launches;         /* kernels launched by the last execute    */
    double pipeline_ms[DQ_MAX_OPS];
} dq_plan_timing;
int dq_plan_timing_get(dq_plan* plan, dq_plan_timing* out);

/* ------------------------------------------------------------- tuning -- */
/* Launch-shape and table-sizing choices an autotuner sets (0: the backend's
 * default).  The reference fixes these in its generator (grid 920-1024 x 128,
 * dogqc/kernel.py:10-11; htSizeFactor 2.0, dogqc/hashJoins.py:43; lane-refill
 * threshold 28 of 32, dogqc/cudaDivergenceBuffer.py:15).                     */
typedef struct {
    int32_t rows_per_thread;         /* 1, 2 or 4 consecutive rows per thread   */
    int32_t block_threads;           /* 128, 256 or 512 (batched kernels)       */
    int32_t refill;                  /* -1: no lane refill; 0: the plan's own   */
    int32_t unique_slots_pct;        /* join-table slots, % of the plan's       */
                                     /* capacity (default 400 for tables of     */
                                     /* up to 48 MB there, else 200)            */
    int32_t multi_buckets_pct;       /* multimap buckets, % (default 100)       */
    int32_t refill_threshold;        /* lane refill: buffered rows that make a  */
                                     /* warp process them, 1..32 (default 32;   */
                                     /* the reference's 0.9 x 32 = 28)          */
    int32_t defer_threshold;         /* expansion ranges longer than this are   */
                                     /* deferred (0: adaptive, 128 or 8)        */
    int32_t ctas_per_sm;             /* resident CTAs per SM of each generated  */
                                     /* pipeline kernel (0: as many as fit);    */
                                     /* 1..8 also bound its registers so that   */
                                     /* they fit (unless that spills)           */
} dq_tuning;
int dq_plan_prepare_tuned(dq_ctx* ctx, const dq_plan_desc* desc, const dq_tuning* tuning, dq_plan** out);

/* ------------------------------------------------------------ batches -- */
/* Many instances of one plan shape (same pipelines and ops; own tables and
 * capacities), such as the partitions of a workload or many small queries,
 * run together: one generated kernel per pipeline walks the row blocks of all
 * instances, one launch resets all their tables, one segmented scan builds all
 * their multimaps, and the whole run (resets, pipelines, scans, result pack
 * and the device-to-host copy) is a captured CUDA graph replayed per execute.
 * No counterpart in the reference, which launches every query separately.  */
int dq_batch_prepare(dq_ctx* ctx, int32_t ninst, const dq_plan_desc* descs, const dq_tuning* tuning,
                     dq_batch** out);
/* results: ninst new results, one per instance, in instance order           */
int dq_batch_execute(dq_batch* batch, void* stream, dq_result** results);
int dq_batch_timing_get(dq_batch* batch, dq_plan_timing* out);  /* total_ms: the graph */
int dq_batch_size(dq_batch* batch, int32_t* ninst);
void dq_batch_free(dq_batch* batch);

/* ------------------------------------------------------------ serving -- */
/* A request loop on its own thread over one context's resident tables.  A
 * request is a plan IR; the server keeps prepared plans pooled per distinct
 * request (tables, built hash tables and compiled kernels stay resident),
 * admits the oldest waiting request when one of `slots` CUDA streams is free
 * and its estimated table and intermediate bytes fit `memory_budget` beside
 * the plans already held (idle pooled plans are freed to make room; a request
 * larger than the whole budget fails with DQ_ERR_ADMISSION), and enqueues it
 * without waiting, so that requests arriving while others run are admitted as
 * slots and memory free up and their kernels overlap on the device.
 * Continuous batching: when a slot frees up, waiting requests of the oldest
 * request's shape (the same pipelines and ops, any tables and sizes) that have
 * an idle pooled plan run together as one many-instance launch on that slot,
 * each on its own plan and tables (the batch kernels of dq_batch_*).  No
 * counterpart in the reference, which runs one query per process.          */
typedef struct dq_server dq_server;
typedef struct {
    int32_t slots;                   /* batches in flight (streams); 0: 8       */
    int32_t pool_per_query;          /* plans kept per request; 0: twice slots  */
    uint64_t memory_budget;          /* bytes; 0: 150 GB                         */
    int32_t batch_max;               /* requests per launch; 0: 16, 1: alone    */
    int32_t batch_rows_max;          /* requests scanning more input rows than  */
                                     /* this run alone (their plain plan's      */
                                     /* graph); 0: 2^18                         */
    int32_t reserved[2];
} dq_server_config;
typedef struct {
    double queue_ms;                 /* submitted -> dispatched to a stream      */
    double run_ms;                   /* dispatched -> result read                */
    double total_ms;                 /* submitted -> result ready                */
    uint64_t bytes;                  /* device bytes of the plan that ran it     */
    int32_t status;                  /* dq_status of the request                 */
    int32_t kernel_launches;
} dq_request_info;
typedef struct {
    uint64_t submitted, completed, failed;
    uint64_t memory_in_use, memory_peak;   /* bytes of pooled plans              */
    double p50_ms, p99_ms, mean_ms;        /* total latency of completed requests */
    double span_ms;                        /* first submit -> last completion    */
    uint64_t batches;                      /* launches that ran several requests */
    uint64_t batched;                      /* requests that ran in them          */
} dq_server_stats;
int dq_server_start(dq_ctx* ctx, const dq_server_config* cfg, dq_server** out);
/* Copies the IR; the tables it names must stay registered until the request
 * completes.                                                               */
int dq_server_submit(dq_server* server, const dq_plan_desc* desc, uint64_t* ticket);
/* Blocks until the request completes; returns its status; *out: its result. */
int dq_server_wait(dq_server* server, uint64_t ticket, dq_result** out, dq_request_info* info);
int dq_server_stats_get(dq_server* server, dq_server_stats* out);
/* Measurement driver: submits request i (query `query_of[i]` of `queries`)
 * at `arrival_ms[i]` after the call starts, from the calling thread, then
 * waits for all of them; infos[i] receives each request's times (results are
 * discarded).  Returns the first failed request's status, else DQ_OK.      */
int dq_server_replay(dq_server* server, int32_t nq, const dq_plan_desc* queries, int64_t nreq,
                     const double* arrival_ms, const int32_t* query_of, dq_request_info* infos);
/* The one-at-a-time reference point: executes plans[plan_of[i]] for every i
 * in order, each to completion (result read and freed); ms_out[i]: its time. */
int dq_plan_run_sequence(dq_plan* const* plans, int32_t nplans, int64_t nreq, const int32_t* plan_of,
                         double* ms_out);
/* Finishes the waiting and running requests, then frees the server.        */
void dq_server_stop(dq_server* server);

/* ------------------------------------------------------------ results -- */
int dq_result_rows(dq_result* r, int64_t* nrows);
int dq_result_ncols(dq_result* r, int32_t* ncols);
/* Host pointer to column `col` (nrows values of its C type; strings as
 * nrows (start,end) byte offsets into `dq_result_heap`).                      */
int dq_result_column(dq_result* r, int32_t col, int32_t* ctype, const void** data);
/* A DQ_STR result column: dq_result_column gives nrows+1 uint64 offsets into
 * this heap of `*nchars` bytes.                                              */
int dq_result_string_heap(dq_result* r, int32_t col, const void** chars, uint64_t* nchars);
void dq_result_free(dq_result* r);

/* ------------------------------------------------- allocation-free join -- */
/* No counterpart in the reference (whose generated programs allocate every
 * buffer with cudaMalloc).  For callers that cannot allocate device memory
 * themselves -- code inside a host program that owns all device memory through
 * its own pool, plugins whose allocator must account for every byte, paths on
 * which cudaMalloc/cudaFree would synchronise the device -- this entry point
 * runs the FK-PK join + grouped SUM/COUNT plan
 *     aggregation([group], [SUM(value), COUNT])(
 *       join(build.key = probe.key, selection(build.filter == filter_value, build), probe))
 * with no allocation at all: its hash table and group table live in one
 * statically sized device array (about 8.2 MB) that every GPU loading this
 * library holds until the process exits.  The caller passes device pointers for
 * all inputs and outputs and the stream to launch on.
 *   - Limits: build_rows <= DQ_NOALLOC_MAX_BUILD_ROWS, max_groups <=
 *     DQ_NOALLOC_MAX_GROUPS; larger requests return DQ_ERR_INVALID with a
 *     message in dq_last_error(NULL).
 *   - out_group/out_sum/out_count must hold max_groups entries; *out_ngroups
 *     receives the number of groups, or -1 when they did not fit.
 *   - The first call on a device looks up the array's device address
 *     (cudaGetSymbolAddress) with that device current; make that first call
 *     before any stream capture.  The address is kept for the life of the
 *     process: after cudaDeviceReset (or anything else that replaces the
 *     device's primary context) this entry point must not be called again.
 *   - A launch failure returns DQ_ERR_CUDA; an error the caller left pending
 *     on the thread is neither reported nor cleared.
 *   - Every call reuses the same array and clears what must start empty, so
 *     calls whose work overlaps on the GPU (different streams or threads)
 *     race; serialise them.
 *   - Runs on the calling thread's current device.  Returns without
 *     synchronising; results are ready when the stream reaches them.       */
#define DQ_NOALLOC_MAX_BUILD_ROWS 262144
#define DQ_NOALLOC_MAX_GROUPS 4096

typedef struct {
    const int32_t* build_key;       /* unique join keys of the build side       */
    const int32_t* build_filter;    /* rows with build_filter == filter_value   */
    int32_t filter_value;
    const int32_t* build_group;     /* grouping value carried to the output     */
    int64_t build_rows;
    const int32_t* probe_key;       /* foreign keys of the probe side           */
    const uint64_t* probe_value;    /* summed per group                         */
    int64_t probe_rows;
    int32_t* out_group;
    uint64_t* out_sum;
    int32_t* out_count;
    int64_t* out_ngroups;
    int32_t max_groups;
} dq_join_agg_args;

int dq_join_agg_noalloc(const dq_join_agg_args* args, void* stream);

#ifdef __cplusplus
}
#endif
#endif
