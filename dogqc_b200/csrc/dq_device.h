// Device-side descriptors of one pipeline launch, filled by the host runtime
// (dq_runtime.cu) from the public IR (include/dogqc_b200.h) and passed to the
// pipeline kernel as one __grid_constant__ parameter.
#pragma once
#include <stdint.h>
#include "../../include/dogqc_b200.h"

namespace dq {

constexpr int kThreads = 256;          // pipeline kernel block size
constexpr int kMaxStages = 4;          // tile staging depth
constexpr int kMaxRes = 16;            // resources of a plan (every pipeline sees them all)
constexpr int kMaxStr = 8;             // string columns per pipeline
constexpr int kMaxStash = 24;          // values carried by one heavy work item
constexpr uint64_t kEmpty = ~0ull;     // empty tag of every hash table

// status bits written by device code
enum : int32_t {
  kErrHtFull = 1,
  kErrTimeout = 2,
  kErrOverflow = 4,
  kErrBadOp = 8,
  kErrKeyRange = 16,     // a key outside a key-domain bitmap's range: the host
                         // turns the table back into a hash table and re-runs
  kInfoHeavyFull = 32,   // informational: deferred expansion items exceeded their
                         // capacity; the rest ran in place (results stay exact)
};
constexpr int32_t kInfoMask = kInfoHeavyFull;

struct DevCol {           // staged fixed-width column
  const uint8_t* ptr;
  int32_t width;
  int32_t smem_off;       // offset inside one stage buffer
};

struct DevStr {           // string column, read in place
  const uint8_t* chars;
  const uint64_t* offsets;
  int32_t width;          // > 0: fixed-width strings
  int32_t sid;            // its index in the plan's string sources (string references)
};

// A string value carried as a 64-bit reference (group keys, join payloads and
// output columns hold these; the bytes stay in place): the plan's string source
// (bits 63..52), a substring flag (bit 51) with the substring's first and end
// byte offsets in the string (bits 50..43 and 42..35) and the row (bits 34..0).
constexpr int kStrRefShift = 52;
constexpr uint64_t kStrRefSub = 1ull << 51;
constexpr int kStrRefStartShift = 43;
constexpr int kStrRefEndShift = 35;
constexpr uint64_t kStrRefRow = (1ull << kStrRefEndShift) - 1;
constexpr int kStrRefMaxSources = 1 << 12;
constexpr int kStrRefMaxOffset = 255;

#ifdef __CUDACC__
// The bytes a reference names: its source's row, cut to the substring window
// when the flag is set (offsets past the string's end give the empty string).
__device__ __forceinline__ void str_ref_bytes(const DevStr* src, uint64_t ref, const uint8_t*& p, int& n) {
  const DevStr& d = src[ref >> kStrRefShift];
  const uint64_t row = ref & kStrRefRow;
  if (d.width > 0) {
    p = d.chars + row * (uint64_t)d.width;
    n = d.width;
  } else {
    p = d.chars + d.offsets[row];
    n = (int)(d.offsets[row + 1] - d.offsets[row]);
  }
  if (ref & kStrRefSub) {
    int st = (int)((ref >> kStrRefStartShift) & 0xff), en = (int)((ref >> kStrRefEndShift) & 0xff);
    st = st < n ? st : n;
    en = en < n ? en : n;
    if (en < st) en = st;
    p += st;
    n = en - st;
  }
}
#endif

struct DevSlot {
  int8_t kind, level, ctype, width;
  int16_t src, res;
  int32_t smem_off;       // REG: offset inside the level's register area
  int32_t stash;          // index in a heavy item's stash (-1: not carried)
};

struct DevRes {
  int32_t kind;           // dq_res_kind
  int32_t nkeys;
  int8_t key_ctype[DQ_MAX_KEYS];
  int32_t packed;         // keys packed into the 64-bit tag
  int32_t compact;        // UNIQUE, one key and one payload of at most 32 bits
                          // each: a slot is one word, key << 32 | payload
                          // (~0 empty); the all-ones key lives at slot cap
                          // (0 when present) with its payload at cap + 1
  int32_t words;          // 64-bit words per slot (tag + keys + payload/aggs)
  int32_t key_word;       // first key word (hashed keys only)
  int32_t val_word;       // first payload / accumulator word
  uint64_t cap;           // slots (UNIQUE/AGG), buckets (MULTI), rows (OUTPUT)
  uint64_t* slots;        // UNIQUE/AGG: cap+1 slots (last = tag ~0 key)
  uint32_t* counts;       // MULTI
  uint32_t* offsets;      // MULTI (cap+1)
  int32_t npay;
  int32_t naggs;
  int8_t pay_ctype[DQ_MAX_PAY];
  int8_t pay_width[DQ_MAX_PAY];
  int8_t agg_red[DQ_MAX_AGGS];
  uint8_t* pay[DQ_MAX_PAY];   // MULTI payload columns / OUTPUT columns
  uint64_t* cursor;       // OUTPUT row cursor
  int32_t smem_slots;     // AGG: CTA-local table slots (0: global only)
  int32_t smem_off;       // AGG: offset of the CTA-local table
  int32_t bitmap;         // UNIQUE over a small key domain [bmin, bmin + brange):
                          // 1: no payload, slots hold one bit per key;
                          // 2: one 32-bit payload, slots hold a word per key,
                          //    (1 << 32) | payload, 0 when the key is absent
  int64_t bmin;
  uint64_t brange;
};

struct DevHeavy {         // deferred wide expansion ranges
  uint64_t* items;        // cap * words
  uint32_t* count;
  uint64_t* unit_prefix;  // work-unit prefix over items (heavy mode)
  uint32_t cap;
  int32_t words;          // 2 + number of stashed values
  int32_t nstash;
  int32_t op;             // index of the EXPAND op the items belong to
  uint64_t threshold;     // ranges longer than this are deferred
  // grouped mode (generated kernels): items whose probe rows matched the same
  // range form a group, and a warp gathers a chunk of the range once for all
  // of the group's items
  int32_t grouped;
  uint32_t gcap;          // group table slots
  uint64_t* gkey;         // (instance << 32) | range offset; kEmpty: free.  A
                          // range's offset identifies it within its instance
                          // (plain plans: instance 0; batches: shared buffers)
  uint32_t* glen;         // range length of a claimed group slot
  uint32_t* gcnt;         // items per group slot, then its scatter cursor
  uint32_t* glist;        // claimed group slots, in claim order
  uint32_t* ngroups;
  uint32_t* gstart;       // item prefix over glist (ngroups + 1 entries)
  uint64_t* sorted;       // the items' stashed values, grouped (cap * nstash)
};

constexpr int kGroupRows = 32;    // range rows per grouped work unit (a warp)
constexpr int kGroupItems = 64;   // items per grouped work unit
constexpr int kGroupThreshold = 128;   // grouped mode: ranges longer than this are deferred
constexpr int kGroupThresholdLow = 8;  // ... once a run showed several probe rows per range
constexpr int kBatchGroupThreshold = 128;  // the same in batches (their item buffers do not grow)

constexpr int kHotSlots = 512;         // CTA-local hot multimap buckets (generated kernels)
constexpr int kHotProbe = 4;           // probe window in that table
constexpr uint32_t kEmpty32 = 0xffffffffu;

struct DevPipe {
  int64_t nrows;
  const uint64_t* nrows_dev;   // row count produced on the device (temp tables)
  int32_t source_kind;         // dq_source_kind
  int32_t source_res;
  int32_t tile;                // rows per tile (multiple of 16)
  int32_t nstage;
  int32_t stage_bytes;
  int32_t exp_cap;             // rows per expansion chunk
  int32_t use_tma;
  int32_t mode;                // 0: tiles, 1: heavy work units
  int32_t clear_src;           // DQ_SRC_AGG: reset every slot read to its initial
                               // state (the table's only scan; the next run then
                               // needs no initialising kernel)
  int32_t ncols;
  DevCol cols[DQ_MAX_COLS];
  int32_t nstr;
  DevStr strs[kMaxStr];
  int32_t nslots;
  DevSlot slots[DQ_MAX_SLOTS];
  int32_t nops;
  dq_op ops[DQ_MAX_OPS];
  int16_t lists[DQ_MAX_LIST];
  int32_t nres;
  DevRes res[kMaxRes];
  const uint8_t* patterns;     // concatenated LIKE patterns / string constants
  int32_t pat_off[DQ_MAX_PATTERNS + 1];
  DevHeavy heavy;
  // shared-memory layout (bytes)
  int32_t off_stage;
  int32_t off_reg[DQ_MAX_LEVELS];
  int32_t off_sel[DQ_MAX_LEVELS];
  int32_t off_par[DQ_MAX_LEVELS];
  int32_t off_match[DQ_MAX_LEVELS];
  int32_t off_exp;             // expansion bookkeeping (off, cnt, pos) per parent level
  int32_t off_flags;           // per-row probe results
  int32_t off_stash;
  int32_t smem_bytes;
  const DevStr* strsrc;        // the plan's string sources (string references)
  int32_t nstrsrc;
  int32_t* status;
  uint32_t* tile_counter;      // dynamic tile scheduler; [1]: CTAs done (fused tail)
  const DevPipe* tail;         // the next pipeline's descriptor when this kernel's
                               // last CTA runs it (a scan of this pipeline's small
                               // aggregation table into the result)
  uint64_t* scratch_ll;        // misc device counters
  uint64_t* profile;           // lane-activity histograms, 33 bins a profile point
};

// ---------------------------------------------------------------- batches --
// A batch runs many instances of one plan shape: these descriptors let one
// launch reset, scan or pack the per-instance buffers of all instances.

struct BatchReset {       // one buffer to reset before a batch run
  void* ptr;
  uint64_t n;             // 64-bit words (kind 0), 32-bit words (kind 1), slots (kind 2)
  uint64_t value;         // kinds 0 and 1
  uint64_t reds;          // kind 2: 4 bits of dq_red_kind per aggregate
  int32_t kind;           // 0: fill u64, 1: fill u32, 2: aggregation table
  int32_t words;          // kind 2: words per slot
  int32_t val_word;       // kind 2: first accumulator word
  int32_t naggs;          // kind 2
};

struct BatchScanSeg {     // one multimap's bucket counts -> offsets
  uint32_t* counts;
  uint32_t* offsets;
  uint64_t n;             // buckets
  uint64_t block0;        // first scan block of this segment
  uint64_t nblocks;
};

struct BatchPack {        // one output column of one instance
  const uint8_t* src;
  const uint64_t* cursor; // rows emitted (may exceed cap on overflow)
  uint64_t cap;
  uint64_t dst;           // byte offset in the packed buffer
  uint64_t* rows_out;     // where the kernel records min(cursor, cap)
  int32_t width;
  int32_t pad;
};

// ------------------------------------------------------------ text import --
constexpr int kImpTile = 16384;       // text bytes per CTA in the newline passes (64 a thread)
constexpr int kImpRows = 256;         // rows per CTA in the parse and string passes
constexpr int kImpMaxFields = 64;

// Field kinds (dq_text_kind) and the reasons a row is rejected.
enum : int32_t { kTxtInt = 1, kTxtDate = 2, kTxtChar = 3, kTxtDecimal = 4, kTxtString = 5, kTxtSkip = 6,
                 kTxtFloat = 7 };
enum : int32_t { kImpTooFew = 1, kImpTooMany = 2, kImpNoDigit = 3, kImpOverflow = 4, kImpNotChar = 5,
                 kImpShortDate = 6, kImpExponent = 7 };

struct ImpField {
  int32_t kind;
  int32_t scale;          // decimal digits kept after the point
  void* out;              // fixed-width column (nrows values)
  int32_t str;            // string ordinal (kTxtString)
  int32_t pad;
};

// The text as whole tiles: bytes [0, nmain) at `main`, the rest (one
// zero-padded tile at most) at `tail`.
struct ImpText {
  const uint8_t* main;
  const uint8_t* tail;
  uint64_t nmain;         // a multiple of kImpTile
};

struct ImpArgs {
  ImpText text;
  uint64_t nbytes;
  uint64_t nlines;        // newlines in the text
  uint64_t nrows;         // nlines, plus one for a last line without a newline
  const uint64_t* line_end;
  uint64_t* err;          // min over bad rows of row << 16 | field << 8 | reason
  uint64_t* spos;         // [nstr][nrows] first byte of each string
  uint32_t* slen;         // [nstr][nrows] its length
  uint64_t* bsum;         // [nstr][nblocks + 1] string bytes per parse block
  uint64_t* boff;         // the same, exclusive prefix sums (total last)
  uint64_t nblocks;
  int32_t nfields;
  int32_t nstr;
  uint32_t delim;
  int32_t pad;
  ImpField f[kImpMaxFields];
  uint64_t* soff[kImpMaxFields];  // string offsets (nrows + 1), by string ordinal
  uint8_t* sheap[kImpMaxFields];  // string heaps
};

}  // namespace dq
