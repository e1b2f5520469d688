// Multithreaded CPU evaluation of a lowered plan: the plan IR of
// include/dogqc_b200.h (the same descriptors the device engine prepares) run
// over host tables on the host's cores.
//
// Test infrastructure and the timed CPU baseline, not part of the product: only
// the tests and the bench's CPU legs load it.  It restates, row at a time, the
// operator semantics the reference's generated pipelines have
// (dogqc/cudaTranslator.py:333-668, dogqc/hashJoins.py:95-681): selections,
// maps with C arithmetic on 64-bit canonical values, unique-key joins (inner,
// semi, anti), multimatch joins walked per probe row, semi/anti joins with a
// condition, hash aggregation (SUM/COUNT/MIN/MAX; AVG is an op on the
// aggregates), materialised results and temp tables, LIKE with the reference
// matcher's rules (dogqc/include/util.cuh:144-199) and string values.
//
// Execution: pipelines in plan order; each pipeline's source rows are split
// into morsels of 16,384 rows taken by `threads` worker threads; every thread
// evaluates the ops of a row in order (an expansion recurses into the ops after
// it once per matching build row) and feeds the sink of its own (a local
// aggregation table, local build rows, local output rows).  After the pipeline
// the local sinks are merged: build rows become a unique table or a multimap
// (rows grouped by key), aggregation tables merge by partitions of the key hash
// (one partition per thread), output rows are concatenated.
#include <malloc.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstdint>
#include <cstring>
#include <exception>
#include <memory>
#include <stdexcept>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../include/dogqc_b200.h"

namespace {

thread_local std::string g_error;

struct Fail : std::runtime_error {
  explicit Fail(const std::string& m) : std::runtime_error(m) {}
};

// ------------------------------------------------------------------ values --

uint64_t canon(uint64_t v, int t) {
  switch (t) {
    case DQ_I8: return (uint64_t)(int64_t)(int8_t)v;
    case DQ_I32: return (uint64_t)(int64_t)(int32_t)v;
    case DQ_U32: return (uint64_t)(uint32_t)v;
    default: return v;
  }
}

bool is_signed(int t) { return t == DQ_I8 || t == DQ_I32 || t == DQ_I64; }

int width_of(int t) {
  switch (t) {
    case DQ_I8: return 1;
    case DQ_I32:
    case DQ_U32: return 4;
    default: return 8;
  }
}

uint64_t truncate(uint64_t v, int w) { return w >= 8 ? v : v & ((1ull << (8 * w)) - 1); }

uint64_t arith(int sub, int t, uint64_t a, uint64_t b) {
  a = canon(a, t);
  b = canon(b, t);
  uint64_t r = 0;
  switch (sub) {
    case DQ_ADD: r = a + b; break;
    case DQ_SUB: r = a - b; break;
    case DQ_MUL: r = a * b; break;
    case DQ_DIV:
    case DQ_MOD: {
      if (b == 0) return 0;  // undefined in C; 0 here, as on the device
      const bool div = sub == DQ_DIV;
      if (t == DQ_I32) {
        const int32_t x = (int32_t)a, y = (int32_t)b;
        if (y == -1) r = div ? (uint64_t)(uint32_t)(0u - (uint32_t)x) : 0;
        else r = (uint64_t)(uint32_t)(div ? x / y : x % y);
      } else if (t == DQ_U32) {
        const uint32_t x = (uint32_t)a, y = (uint32_t)b;
        r = div ? x / y : x % y;
      } else if (t == DQ_I64) {
        const int64_t x = (int64_t)a, y = (int64_t)b;
        if (y == -1) r = div ? 0ull - a : 0;
        else r = (uint64_t)(div ? x / y : x % y);
      } else {
        r = div ? a / b : a % b;
      }
      break;
    }
    default: break;
  }
  return canon(r, t);
}

// LIKE as the reference matcher decides it: prefix, then suffix, then the
// infixes left to right; '_' matches any byte; reads past either end see 0.
bool like_match(const uint8_t* s, int ls, const uint8_t* p, int lp) {
  auto S = [&](int i) -> int { return (i >= 0 && i < ls) ? s[i] : 0; };
  auto P = [&](int i) -> int { return (i >= 0 && i < lp) ? p[i] : 0; };
  auto same = [](int c, int l) { return c == l || l == '_'; };
  int lo = 0, hi = lp, slo = 0, shi = ls, lpos = 0;
  if (P(0) != '%') {
    int spos = 0;
    lpos = 0;
    while (lpos < lp && spos < ls && P(lpos) != '%') {
      if (!same(S(spos), P(lpos))) return false;
      ++lpos;
      ++spos;
    }
    lo = lpos;
    slo = spos;
  }
  if (P(lp - 1) != '%') {
    int spos = ls - 1;
    lpos = lp - 1;
    while (lpos >= 0 && spos >= 0 && P(lpos) != '%') {
      if (!same(S(spos), P(lpos))) return false;
      --lpos;
      --spos;
    }
    hi = lpos;
    shi = spos + 1;
  }
  if (lo < hi) {
    lpos = lo + 1;
    int spos = slo;
    while (spos < shi && lpos < hi) {
      int lt = lpos, st = spos;
      while (same(S(st), P(lt)) && st < shi) {
        ++lt;
        if (P(lt) == '%') {
          ++lt;
          lpos = lt;
          spos = st;
          break;
        }
        ++st;
      }
      ++spos;
    }
  }
  return lpos >= hi;
}

uint64_t mix(uint64_t k) {
  k ^= k >> 33;
  k *= 0xff51afd7ed558ccdull;
  k ^= k >> 33;
  k *= 0xc4ceb9fe1a85ec53ull;
  k ^= k >> 33;
  return k;
}

uint64_t hash_bytes(const uint8_t* p, int n) {
  uint64_t h = 0xcbf29ce484222325ull;
  for (int i = 0; i < n; ++i) h = (h ^ p[i]) * 0x100000001b3ull;
  return mix(h);
}

// ---------------------------------------------------------------- tables --

struct Column {
  int ctype = 0;
  int width = 0;                 // fixed-width strings
  const uint8_t* data = nullptr;
  const uint64_t* offsets = nullptr;
};

struct Table {
  int64_t nrows = 0;
  std::unordered_map<std::string, Column> cols;
};

// A string value is a reference: its string source (a column of a table,
// bits 63..52), a substring flag (bit 51) with the window's first and end byte
// offsets (bits 50..43, 42..35) and its row (bits 34..0), the device's layout.
constexpr int kRefShift = 52;
constexpr uint64_t kRefSub = 1ull << 51;
constexpr int kRefStartShift = 43;
constexpr int kRefEndShift = 35;
constexpr uint64_t kRefRow = (1ull << kRefEndShift) - 1;

struct Strings {
  std::vector<const Column*> src;
  void at(uint64_t ref, const uint8_t*& p, int& n) const {
    const Column& c = *src[ref >> kRefShift];
    const uint64_t row = ref & kRefRow;
    if (c.width > 0) {
      p = c.data + row * (uint64_t)c.width;
      n = c.width;
    } else {
      p = c.data + c.offsets[row];
      n = (int)(c.offsets[row + 1] - c.offsets[row]);
    }
    if (ref & kRefSub) {
      const int st = std::min((int)((ref >> kRefStartShift) & 0xff), n);
      const int en = std::max(std::min((int)((ref >> kRefEndShift) & 0xff), n), st);
      p += st;
      n = en - st;
    }
  }
};

// SUBSTRING(s, from, len) as a window on the reference: the first byte from - 1,
// len bytes, within the parent window (the reference's stringSubstring,
// include/util.cuh:132-142); a window past the string's end is empty.
uint64_t substring_ref(uint64_t ref, int from, int len) {
  int s0 = 0, e0 = 1 << 30;
  if (ref & kRefSub) {
    s0 = (int)((ref >> kRefStartShift) & 0xff);
    e0 = (int)((ref >> kRefEndShift) & 0xff);
  }
  int st = s0 + from - 1;
  int en = st + len;
  st = std::max(st, s0);
  en = std::min(en, e0);
  st = std::min(std::max(st, 0), 255);
  en = std::min(std::max(en, st), 255);
  return (ref & ((~0ull << kRefShift) | kRefRow)) | kRefSub | ((uint64_t)st << kRefStartShift) |
         ((uint64_t)en << kRefEndShift);
}

// ------------------------------------------------------------ resources --

struct Rows {        // build rows or output rows: `width` words a row
  int width = 0;
  std::vector<uint64_t> v;
  int64_t n() const { return width ? (int64_t)(v.size() / width) : 0; }
};

struct KeyHash {
  const dq_resource* r = nullptr;
  const Strings* strs = nullptr;
  uint64_t operator()(const uint64_t* k) const {
    uint64_t h = 0x9e3779b97f4a7c15ull;
    for (int i = 0; i < r->nkeys; ++i) {
      uint64_t v = k[i];
      if (r->key_ctype[i] == DQ_STR) {
        const uint8_t* p;
        int n;
        strs->at(v, p, n);
        v = hash_bytes(p, n);
      }
      h = mix(h ^ v) + 0x632be59bd9b4e019ull * (uint64_t)(i + 1);
    }
    return mix(h);
  }
  bool eq(const uint64_t* a, const uint64_t* b) const {
    for (int i = 0; i < r->nkeys; ++i) {
      if (a[i] == b[i]) continue;
      if (r->key_ctype[i] != DQ_STR) return false;
      const uint8_t *pa, *pb;
      int na, nb;
      strs->at(a[i], pa, na);
      strs->at(b[i], pb, nb);
      if (na != nb || memcmp(pa, pb, (size_t)na) != 0) return false;
    }
    return true;
  }
  // A total order of keys that agrees with eq (strings by their bytes).
  int cmp(const uint64_t* a, const uint64_t* b) const {
    for (int i = 0; i < r->nkeys; ++i) {
      if (a[i] == b[i]) continue;
      if (r->key_ctype[i] != DQ_STR) return a[i] < b[i] ? -1 : 1;
      const uint8_t *pa, *pb;
      int na, nb;
      strs->at(a[i], pa, na);
      strs->at(b[i], pb, nb);
      const int c = memcmp(pa, pb, (size_t)std::min(na, nb));
      if (c != 0) return c;
      if (na != nb) return na < nb ? -1 : 1;
    }
    return 0;
  }
};

// Open-addressing index over rows with key words at the front of each row.
struct KeyIndex {
  std::vector<int64_t> slot;     // row index or -1
  uint64_t mask = 0;
  void build(const Rows& rows, int nkeys, const KeyHash& kh, bool first_wins) {
    const int64_t n = rows.n();
    uint64_t cap = 16;
    while (cap < (uint64_t)n * 2) cap <<= 1;
    slot.assign(cap, -1);
    mask = cap - 1;
    for (int64_t i = 0; i < n; ++i) {
      const uint64_t* k = &rows.v[(size_t)i * rows.width];
      uint64_t h = kh(k) & mask;
      for (;;) {
        const int64_t s = slot[h];
        if (s < 0) {
          slot[h] = i;
          break;
        }
        if (first_wins && kh.eq(&rows.v[(size_t)s * rows.width], k)) break;
        h = (h + 1) & mask;
      }
      (void)nkeys;
    }
  }
  int64_t find(const Rows& rows, const uint64_t* k, const KeyHash& kh) const {
    if (slot.empty()) return -1;
    uint64_t h = kh(k) & mask;
    for (;;) {
      const int64_t s = slot[h];
      if (s < 0) return -1;
      if (kh.eq(&rows.v[(size_t)s * rows.width], k)) return s;
      h = (h + 1) & mask;
    }
  }
};

// Unique join table: open addressing with each slot holding its row (a used
// marker, the key words, the payload words) inline, so a probe touches one
// slot.  The first row inserted for a key wins.
struct UniqueTable {
  int W = 0;                     // words a row (keys + payload)
  int nk = 0;
  std::vector<uint64_t> slots;   // (1 + W) words a slot; word 0: 1 if used
  uint64_t mask = 0;
  const KeyHash* keq = nullptr;  // key equality (string keys by their bytes)
  void build(const Rows& rows, int nkeys, const KeyHash& kh) {
    W = rows.width;
    nk = nkeys;
    keq = &kh;
    uint64_t cap = 16;
    while (cap < (uint64_t)rows.n() * 2) cap <<= 1;
    mask = cap - 1;
    slots.assign(cap * (uint64_t)(W + 1), 0);
    for (int64_t i = 0; i < rows.n(); ++i) {
      const uint64_t* row = &rows.v[(size_t)i * W];
      uint64_t h = kh(row) & mask;
      for (;;) {
        uint64_t* sl = &slots[h * (W + 1)];
        if (!sl[0]) {
          sl[0] = 1;
          std::copy(row, row + W, sl + 1);
          break;
        }
        if (kh.eq(row, sl + 1)) break;
        h = (h + 1) & mask;
      }
    }
  }
  // The matching row's words, or nullptr.
  const uint64_t* find(const uint64_t* k, uint64_t hash) const {
    if (slots.empty()) return nullptr;
    uint64_t h = hash & mask;
    for (;;) {
      const uint64_t* sl = &slots[h * (W + 1)];
      if (!sl[0]) return nullptr;
      if (keq->eq(k, sl + 1)) return sl + 1;
      h = (h + 1) & mask;
    }
  }
};

// Aggregation table: groups of key words and accumulators.
struct AggTable {
  const dq_resource* r = nullptr;
  KeyHash kh;
  int width = 0;                 // nkeys + naggs
  std::vector<uint64_t> rows;    // groups
  std::vector<uint64_t> hashes;
  std::vector<int64_t> slot;
  uint64_t mask = 0;
  void init(const dq_resource* res, const Strings* s, uint64_t cap_hint) {
    r = res;
    kh.r = res;
    kh.strs = s;
    width = res->nkeys + res->naggs;
    uint64_t cap = 64;
    while (cap < cap_hint * 2) cap <<= 1;
    slot.assign(cap, -1);
    mask = cap - 1;
    rows.clear();
    hashes.clear();
  }
  int64_t n() const { return width ? (int64_t)(rows.size() / width) : 0; }
  void grow() {
    const uint64_t cap = (mask + 1) * 2;
    slot.assign(cap, -1);
    mask = cap - 1;
    for (int64_t g = 0; g < n(); ++g) {
      uint64_t h = hashes[g] & mask;
      while (slot[h] >= 0) h = (h + 1) & mask;
      slot[h] = g;
    }
  }
  uint64_t* group(const uint64_t* k, uint64_t hash) { return &rows[(size_t)group_index(k, hash) * width]; }
  // Index of the group of key k (claimed if new).
  int64_t group_index(const uint64_t* k, uint64_t hash) {
    uint64_t h = hash & mask;
    for (;;) {
      const int64_t s = slot[h];
      if (s < 0) break;
      if (hashes[s] == hash && kh.eq(&rows[(size_t)s * width], k)) return s;
      h = (h + 1) & mask;
    }
    const int64_t g = n();
    rows.resize(rows.size() + width);
    uint64_t* row = &rows[(size_t)g * width];
    for (int i = 0; i < r->nkeys; ++i) row[i] = k[i];
    for (int j = 0; j < r->naggs; ++j) row[r->nkeys + j] = r->agg_red[j] == DQ_RED_MIN ? ~0ull : 0ull;
    hashes.push_back(hash);
    slot[h] = g;
    if ((uint64_t)n() * 2 > mask) grow();
    return g;
  }
};

void combine(int red, uint64_t& acc, uint64_t v) {
  switch (red) {
    case DQ_RED_MIN: acc = v < acc ? v : acc; break;
    case DQ_RED_MAX: acc = v > acc ? v : acc; break;
    default: acc += v; break;
  }
}

struct Resource {
  const dq_resource* d = nullptr;
  // UNIQUE (key words, then payload) and MULTI (rows grouped by key: key
  // words, then payload) build rows; OUTPUT rows (one word a column)
  Rows rows;
  UniqueTable unique;                  // UNIQUE
  KeyIndex index;                      // MULTI: key -> first row of its run
  std::vector<int64_t> run_len;        // MULTI: rows in the run starting at each row
  AggTable agg;                        // AGG (merged)
};

// ------------------------------------------------------------ execution --

struct Plan;

constexpr int kBatch = 1024;   // rows a batch (values of a slot are one array)

// One batch of rows at one expansion level: every slot's values, the active
// rows, each row's source row (string ops read the source row) and, below
// level 0, each row's row in the level above.
struct Level {
  std::vector<uint64_t> v;
  std::vector<uint32_t> sel;
  int nsel = 0;
  std::vector<int64_t> srow;
  std::vector<uint32_t> parent;
  uint64_t* slot(int s) { return &v[(size_t)s * kBatch]; }
  const uint64_t* slot(int s) const { return &v[(size_t)s * kBatch]; }
  void init(int nslots) {
    v.assign((size_t)std::max(nslots, 1) * kBatch, 0);
    sel.assign(kBatch, 0);
    srow.assign(kBatch, 0);
    parent.assign(kBatch, 0);
    nsel = 0;
  }
};

struct Worker {        // one thread's state for one pipeline
  Level lv[DQ_MAX_LEVELS];
  AggTable agg;
  Rows out;            // BUILD / MM_SCATTER / EMIT rows
  std::vector<uint64_t> keys, hashes;
  std::vector<const uint64_t*> hits;
  std::vector<int64_t> gidx;
};

template <int T>
inline uint64_t cn(uint64_t v) {
  if (T == DQ_I8) return (uint64_t)(int64_t)(int8_t)v;
  if (T == DQ_I32) return (uint64_t)(int64_t)(int32_t)v;
  if (T == DQ_U32) return (uint64_t)(uint32_t)v;
  return v;
}

// d[i] = canon_T(f(canon_T(a[i]), canon_T(b[i]))) over the active rows; a or b
// null: the immediate.
template <int T, class F>
void bin_loop(const uint32_t* sel, int n, uint64_t* d, const uint64_t* a, uint64_t ai, const uint64_t* b, uint64_t bi,
              F f) {
  if (a && b) {
    for (int j = 0; j < n; ++j) {
      const uint32_t i = sel[j];
      d[i] = cn<T>(f(cn<T>(a[i]), cn<T>(b[i])));
    }
  } else if (a) {
    const uint64_t y = cn<T>(bi);
    for (int j = 0; j < n; ++j) {
      const uint32_t i = sel[j];
      d[i] = cn<T>(f(cn<T>(a[i]), y));
    }
  } else {
    const uint64_t x = cn<T>(ai);
    for (int j = 0; j < n; ++j) {
      const uint32_t i = sel[j];
      d[i] = cn<T>(f(x, b ? cn<T>(b[i]) : cn<T>(bi)));
    }
  }
}

template <int T>
void arith_loop(int sub, const uint32_t* sel, int n, uint64_t* d, const uint64_t* a, uint64_t ai, const uint64_t* b,
                uint64_t bi) {
  switch (sub) {
    case DQ_ADD: bin_loop<T>(sel, n, d, a, ai, b, bi, [](uint64_t x, uint64_t y) { return x + y; }); break;
    case DQ_SUB: bin_loop<T>(sel, n, d, a, ai, b, bi, [](uint64_t x, uint64_t y) { return x - y; }); break;
    case DQ_MUL: bin_loop<T>(sel, n, d, a, ai, b, bi, [](uint64_t x, uint64_t y) { return x * y; }); break;
    default:
      bin_loop<T>(sel, n, d, a, ai, b, bi, [sub](uint64_t x, uint64_t y) { return arith(sub, T, x, y); });
      break;
  }
}

template <int T>
void cmp_loop(int sub, const uint32_t* sel, int n, uint64_t* d, const uint64_t* a, uint64_t ai, const uint64_t* b,
              uint64_t bi) {
  constexpr bool sg = T == DQ_I8 || T == DQ_I32 || T == DQ_I64;
  auto lt = [](uint64_t x, uint64_t y) -> uint64_t { return sg ? (int64_t)x < (int64_t)y : x < y; };
  switch (sub) {
    case DQ_EQ: bin_loop<T>(sel, n, d, a, ai, b, bi, [](uint64_t x, uint64_t y) -> uint64_t { return x == y; }); break;
    case DQ_NE: bin_loop<T>(sel, n, d, a, ai, b, bi, [](uint64_t x, uint64_t y) -> uint64_t { return x != y; }); break;
    case DQ_LT: bin_loop<T>(sel, n, d, a, ai, b, bi, [&](uint64_t x, uint64_t y) { return lt(x, y); }); break;
    case DQ_LE: bin_loop<T>(sel, n, d, a, ai, b, bi, [&](uint64_t x, uint64_t y) -> uint64_t { return !lt(y, x); }); break;
    case DQ_GT: bin_loop<T>(sel, n, d, a, ai, b, bi, [&](uint64_t x, uint64_t y) { return lt(y, x); }); break;
    default: bin_loop<T>(sel, n, d, a, ai, b, bi, [&](uint64_t x, uint64_t y) -> uint64_t { return !lt(x, y); }); break;
  }
}

template <template <int> class K, class... A>
void by_type(int t, A... args) {
  switch (t) {
    case DQ_I8: K<DQ_I8>::run(args...); break;
    case DQ_I32: K<DQ_I32>::run(args...); break;
    case DQ_U32: K<DQ_U32>::run(args...); break;
    case DQ_I64: K<DQ_I64>::run(args...); break;
    default: K<DQ_U64>::run(args...); break;
  }
}
template <int T>
struct ArithK {
  static void run(int sub, const uint32_t* sel, int n, uint64_t* d, const uint64_t* a, uint64_t ai, const uint64_t* b,
                  uint64_t bi) {
    arith_loop<T>(sub, sel, n, d, a, ai, b, bi);
  }
};
template <int T>
struct CmpK {
  static void run(int sub, const uint32_t* sel, int n, uint64_t* d, const uint64_t* a, uint64_t ai, const uint64_t* b,
                  uint64_t bi) {
    cmp_loop<T>(sub, sel, n, d, a, ai, b, bi);
  }
};

struct Pipeline {
  const dq_pipeline* d = nullptr;
  const Table* table = nullptr;        // DQ_SRC_TABLE
  std::vector<const Column*> cols;     // per pipeline column (table sources)
  std::vector<int> sid;                // string source of STR slots
  std::vector<std::string> patterns;
};

struct Plan {
  const dq_plan_desc* d = nullptr;
  std::vector<Resource> res;
  std::vector<Pipeline> pipes;
  Strings strs;
  int threads = 1;

  // d = canon(d, t) over the active rows (the slot's own type after an op's).
  static void recast(const Level& L, uint64_t* d, int t) {
    if (t == DQ_I64 || t == DQ_U64 || t == DQ_STR) return;
    for (int j = 0; j < L.nsel; ++j) d[L.sel[j]] = canon(d[L.sel[j]], t);
  }

  void scalar(const Pipeline& p, const dq_op& op, Level& L) const {
    const dq_pipeline& d = *p.d;
    uint64_t* dst = L.slot(op.dst);
    const int dt = d.slots[op.dst].ctype;
    const uint32_t* sel = L.sel.data();
    const int n = L.nsel;
    const uint64_t* a = (op.flags & DQ_OPF_A_IMM) || op.a < 0 ? nullptr : L.slot(op.a);
    const uint64_t* b = (op.flags & DQ_OPF_B_IMM) || op.b < 0 ? nullptr : L.slot(op.b);
    const uint64_t ai = (uint64_t)op.imm, bi = (uint64_t)op.imm;
    switch (op.kind) {
      case DQ_OP_ARITH:
        by_type<ArithK>(op.ctype, (int)op.sub, sel, n, dst, a, ai, b, bi);
        if (dt != op.ctype) recast(L, dst, dt);
        break;
      case DQ_OP_CMP:
        by_type<CmpK>(op.ctype, (int)op.sub, sel, n, dst, a, ai, b, bi);
        break;
      case DQ_OP_LOGIC: {
        const uint64_t* x = L.slot(op.a);
        if (op.sub == DQ_NOT) {
          for (int j = 0; j < n; ++j) dst[sel[j]] = x[sel[j]] == 0;
        } else {
          const uint64_t* y = L.slot(op.b);
          if (op.sub == DQ_AND)
            for (int j = 0; j < n; ++j) dst[sel[j]] = x[sel[j]] != 0 && y[sel[j]] != 0;
          else
            for (int j = 0; j < n; ++j) dst[sel[j]] = x[sel[j]] != 0 || y[sel[j]] != 0;
        }
        break;
      }
      case DQ_OP_CAST:
        for (int j = 0; j < n; ++j) {
          const uint32_t i = sel[j];
          dst[i] = canon(canon(a ? a[i] : ai, op.ctype), dt);
        }
        break;
      case DQ_OP_SELECT: {
        const uint64_t* c = L.slot(op.a);
        const uint64_t* prev = L.slot(op.c >= 0 ? op.c : op.dst);
        for (int j = 0; j < n; ++j) {
          const uint32_t i = sel[j];
          dst[i] = canon(canon(c[i] ? (b ? b[i] : bi) : prev[i], op.ctype), dt);
        }
        break;
      }
      default: throw Fail("not a scalar op");
    }
  }

  // Keys of the active rows, canonical in the resource's key types (nk words
  // a row, row j of the selection at keys[j * nk]).
  void keys(const Pipeline& p, const dq_resource& r, const Level& L, int list, int n, std::vector<uint64_t>& out) const {
    const int stride = std::max(n, 1);
    out.assign((size_t)L.nsel * stride, 0);
    for (int i = 0; i < n; ++i) {
      const uint64_t* src = L.slot(p.d->lists[list + i]);
      const int t = r.key_ctype[i];
      for (int j = 0; j < L.nsel; ++j) out[(size_t)j * stride + i] = canon(src[L.sel[j]], t);
    }
  }

  void keep_where(Level& L, const std::vector<uint8_t>& keep) const {
    int m = 0;
    for (int j = 0; j < L.nsel; ++j)
      if (keep[j]) L.sel[m++] = L.sel[j];
    L.nsel = m;
  }

  // The rows of multimap `r` matching each active row (runs of equal keys):
  // child rows at `C` are (parent row, match) pairs, emitted batch by batch to
  // `flush`, with the build row's gathered slots and the live slots of the
  // level above copied in.
  template <class Flush>
  void pairs(const Pipeline& p, const dq_op& op, int level, Level& L, Level& C, Worker& w, Flush flush) const {
    (void)w;
    const dq_pipeline& d = *p.d;
    const Resource& r = res[op.res];
    std::vector<uint64_t> pk;   // this op's own keys: the ops run on each child batch use the worker's
    keys(p, *r.d, L, op.list, op.nlist, pk);
    const int nk = std::max((int)op.nlist, 1);
    const int W = r.rows.width;
    std::vector<int> gath, copy;
    for (int s = 0; s < d.nslots; ++s) {
      const dq_slot& sl = d.slots[s];
      if (sl.kind == DQ_SLOT_STR) continue;
      if (sl.kind == DQ_SLOT_GATHER && sl.level == level + 1 && sl.res == op.res) gath.push_back(s);
      else if (sl.level <= level) copy.push_back(s);
    }
    std::vector<int64_t> match((size_t)kBatch);
    auto emit = [&]() {
      const int n = C.nsel;
      for (int s : copy) {
        const uint64_t* src = L.slot(s);
        uint64_t* dst = C.slot(s);
        for (int c = 0; c < n; ++c) dst[c] = src[C.parent[c]];
      }
      for (int s : gath) {
        const dq_slot& sl = d.slots[s];
        const int off = r.d->nkeys + sl.src;
        const int wd = width_of(r.d->pay_ctype[sl.src]);
        uint64_t* dst = C.slot(s);
        const uint64_t* rows = r.rows.v.data();
        for (int c = 0; c < n; ++c) dst[c] = canon(truncate(rows[(size_t)match[c] * W + off], wd), sl.ctype);
      }
      for (int c = 0; c < n; ++c) C.srow[c] = L.srow[C.parent[c]];
      flush(C);
      C.nsel = 0;
    };
    C.nsel = 0;
    for (int j = 0; j < L.nsel; ++j) {
      const uint32_t i = L.sel[j];
      const int64_t first = r.index.find(r.rows, &pk[(size_t)j * nk], r.agg.kh);
      if (first < 0) continue;
      const int64_t end = first + r.run_len[first];
      for (int64_t m = first; m < end; ++m) {
        if (C.nsel == kBatch) emit();
        const int c = C.nsel++;
        C.sel[c] = (uint32_t)c;
        C.parent[c] = i;
        match[c] = m;
      }
    }
    if (C.nsel) emit();
  }

  // The reference of string slot s for row i: a string column's value is its
  // source row's, anything else holds a reference already.
  uint64_t str_value(const Pipeline& p, const Level& L, int s, uint32_t i) const {
    if (p.d->slots[s].kind == DQ_SLOT_STR) return ((uint64_t)p.sid[s] << kRefShift) | (uint64_t)L.srow[i];
    return L.slot(s)[i];
  }

  // Ops k.. over the active rows of batch L at `level`.
  void eval(const Pipeline& p, int k, int level, Worker& w) const {
    const dq_pipeline& d = *p.d;
    Level& L = w.lv[level];
    for (; k < d.nops && L.nsel > 0; ++k) {
      const dq_op& op = d.ops[k];
      switch (op.kind) {
        case DQ_OP_ARITH:
        case DQ_OP_CMP:
        case DQ_OP_LOGIC:
        case DQ_OP_CAST:
        case DQ_OP_SELECT:
          scalar(p, op, L);
          break;
        case DQ_OP_LIKE:
        case DQ_OP_STREQ: {
          uint64_t* dst = L.slot(op.dst);
          const bool two = op.kind == DQ_OP_STREQ && op.res < 0;
          static const std::string none;
          const std::string& pat = two ? none : p.patterns[op.res];
          for (int j = 0; j < L.nsel; ++j) {
            const uint32_t i = L.sel[j];
            const uint8_t* s;
            int n;
            strs.at(str_value(p, L, op.a, i), s, n);
            if (two) {
              const uint8_t* t;
              int m;
              strs.at(str_value(p, L, op.b, i), t, m);
              dst[i] = n == m && memcmp(s, t, (size_t)n) == 0;
            } else {
              dst[i] = op.kind == DQ_OP_LIKE
                           ? like_match(s, n, reinterpret_cast<const uint8_t*>(pat.data()), (int)pat.size())
                           : (n == (int)pat.size() && memcmp(s, pat.data(), (size_t)n) == 0);
            }
          }
          break;
        }
        case DQ_OP_SUBSTR: {
          uint64_t* dst = L.slot(op.dst);
          const uint64_t* a = L.slot(op.a);
          const int from = (int32_t)(uint32_t)op.imm, len = (int32_t)(uint32_t)((uint64_t)op.imm >> 32);
          for (int j = 0; j < L.nsel; ++j) dst[L.sel[j]] = substring_ref(a[L.sel[j]], from, len);
          break;
        }
        case DQ_OP_STRREF: {
          uint64_t* dst = L.slot(op.dst);
          const uint64_t base = (uint64_t)p.sid[op.a] << kRefShift;
          for (int j = 0; j < L.nsel; ++j) dst[L.sel[j]] = base | (uint64_t)L.srow[L.sel[j]];
          break;
        }
        case DQ_OP_PROFILE:  // lane-activity counters are a device measurement
          break;
        case DQ_OP_FILTER: {
          const uint64_t* x = L.slot(op.a);
          int m = 0;
          for (int j = 0; j < L.nsel; ++j)
            if (x[L.sel[j]] != 0) L.sel[m++] = L.sel[j];
          L.nsel = m;
          break;
        }
        case DQ_OP_PROBE: {
          const Resource& r = res[op.res];
          const int nk = std::max((int)op.nlist, 1);
          keys(p, *r.d, L, op.list, op.nlist, w.keys);
          w.hashes.resize(L.nsel);
          w.hits.resize(L.nsel);
          for (int j = 0; j < L.nsel; ++j) {
            w.hashes[j] = r.agg.kh(&w.keys[(size_t)j * nk]);
            if (!r.unique.slots.empty())
              __builtin_prefetch(&r.unique.slots[(w.hashes[j] & r.unique.mask) * (uint64_t)(r.unique.W + 1)]);
          }
          for (int j = 0; j < L.nsel; ++j) w.hits[j] = r.unique.find(&w.keys[(size_t)j * nk], w.hashes[j]);
          int m = 0;
          for (int j = 0; j < L.nsel; ++j) {
            const uint64_t* hit = w.hits[j];
            const uint32_t i = L.sel[j];
            if ((op.sub == DQ_JOIN_ANTI) == (hit != nullptr)) continue;
            if (op.sub == DQ_JOIN_INNER)
              for (int q = 0; q < op.nlist2; ++q) {
                const int dst = d.lists[op.list2 + q];
                if (dst >= 0) L.slot(dst)[i] = canon(canon(hit[r.d->nkeys + q], r.d->pay_ctype[q]), d.slots[dst].ctype);
              }
            L.sel[m++] = i;
          }
          L.nsel = m;
          break;
        }
        case DQ_OP_EXPAND: {
          Level& C = w.lv[level + 1];
          pairs(p, op, level, L, C, w, [&](Level&) { eval(p, k + 1, level + 1, w); });
          return;
        }
        case DQ_OP_EXISTS: {
          Level& C = w.lv[level + 1];
          std::vector<uint8_t> found((size_t)kBatch, 0);
          pairs(p, op, level, L, C, w, [&](Level& c) {
            for (int j = k + 1; j <= k + (int)op.imm; ++j) scalar(p, d.ops[j], c);
            const uint64_t* cond = op.imm > 0 ? c.slot(op.a) : nullptr;
            for (int j = 0; j < c.nsel; ++j) {
              const uint32_t i = c.sel[j];
              if (!cond || cond[i] != 0) found[c.parent[i]] = 1;
            }
          });
          const bool semi = op.sub == DQ_JOIN_SEMI;
          int m = 0;
          for (int j = 0; j < L.nsel; ++j)
            if ((found[L.sel[j]] != 0) == semi) L.sel[m++] = L.sel[j];
          L.nsel = m;
          k += (int)op.imm;
          break;
        }
        case DQ_OP_AGG: {
          const dq_resource& r = *res[op.res].d;
          keys(p, r, L, op.list, op.nlist, w.keys);
          const int nk = std::max((int)op.nlist, 1);
          w.gidx.resize(L.nsel);
          for (int j = 0; j < L.nsel; ++j) {
            const uint64_t* kk = &w.keys[(size_t)j * nk];
            w.gidx[j] = w.agg.group_index(kk, w.agg.kh(kk));
          }
          uint64_t* rows = w.agg.rows.data();
          const int gw = w.agg.width;
          for (int q = 0; q < op.nlist2; ++q) {
            const int s = d.lists[op.list2 + q];
            const int red = r.agg_red[q];
            const int off = r.nkeys + q;
            if (red == DQ_RED_COUNT || s < 0) {
              for (int j = 0; j < L.nsel; ++j) rows[(size_t)w.gidx[j] * gw + off] += 1;
            } else {
              const uint64_t* x = L.slot(s);
              for (int j = 0; j < L.nsel; ++j) combine(red, rows[(size_t)w.gidx[j] * gw + off], x[L.sel[j]]);
            }
          }
          return;
        }
        case DQ_OP_BUILD:
        case DQ_OP_MM_SCATTER: {
          const dq_resource& r = *res[op.res].d;
          keys(p, r, L, op.list, op.nlist, w.keys);
          for (int j = 0; j < L.nsel; ++j) {
            for (int q = 0; q < op.nlist; ++q) w.out.v.push_back(w.keys[(size_t)j * std::max((int)op.nlist, 1) + q]);
            for (int q = 0; q < op.nlist2; ++q)
              w.out.v.push_back(truncate(L.slot(d.lists[op.list2 + q])[L.sel[j]], width_of(r.pay_ctype[q])));
          }
          return;
        }
        case DQ_OP_MM_COUNT:
          return;  // the scatter pass collects the rows
        case DQ_OP_EMIT:
          for (int j = 0; j < L.nsel; ++j)
            for (int q = 0; q < op.nlist; ++q) w.out.v.push_back(L.slot(d.lists[op.list + q])[L.sel[j]]);
          return;
        default:
          throw Fail("op kind " + std::to_string(op.kind) + " is not evaluated here");
      }
    }
  }

  int64_t source_rows(const Pipeline& p) const {
    switch (p.d->source_kind) {
      case DQ_SRC_TABLE: return p.table->nrows;
      case DQ_SRC_OUTPUT: return res[p.d->source_res].rows.n();
      default: {
        const Resource& r = res[p.d->source_res];
        return r.d->nkeys == 0 ? 1 : r.agg.n();
      }
    }
  }

  void run_pipeline(const Pipeline& p) {
    const dq_pipeline& d = *p.d;
    const dq_op& sink = d.ops[d.nops - 1];
    const int64_t nrows = source_rows(p);
    std::vector<Worker> workers(threads);
    for (auto& w : workers) {
      for (auto& L : w.lv) L.init(d.nslots);
      if (sink.kind == DQ_OP_AGG) w.agg.init(res[sink.res].d, &strs, 1024);
      if (sink.kind == DQ_OP_BUILD || sink.kind == DQ_OP_MM_SCATTER) w.out.width = sink.nlist + sink.nlist2;
      if (sink.kind == DQ_OP_EMIT) w.out.width = sink.nlist;
    }
    const int64_t morsel = 16 * kBatch;
    std::atomic<int64_t> next{0};
    parallel(threads, [&](int t) {
      Worker& w = workers[t];
      Level& L = w.lv[0];
      for (;;) {
        const int64_t lo = next.fetch_add(morsel);
        if (lo >= nrows) break;
        const int64_t hi = std::min(nrows, lo + morsel);
        for (int64_t b = lo; b < hi; b += kBatch) {
          const int n = (int)std::min<int64_t>(kBatch, hi - b);
          load_batch(p, b, n, L);
          eval(p, 0, 0, w);
        }
      }
    });
    merge(p, sink, workers);
  }

  // Level-0 values of source rows b .. b+n-1 into L (all rows active).
  void load_batch(const Pipeline& p, int64_t b, int n, Level& L) const {
    const dq_pipeline& d = *p.d;
    L.nsel = n;
    for (int j = 0; j < n; ++j) {
      L.sel[j] = (uint32_t)j;
      L.srow[j] = b + j;
    }
    for (int s = 0; s < d.nslots; ++s) {
      const dq_slot& sl = d.slots[s];
      uint64_t* dst = L.slot(s);
      if (sl.kind == DQ_SLOT_COL) {
        if (d.source_kind == DQ_SRC_TABLE) {
          const Column& c = *p.cols[sl.src];
          switch (width_of(c.ctype)) {
            case 1:
              for (int j = 0; j < n; ++j) dst[j] = canon(c.data[b + j], sl.ctype);
              break;
            case 4: {
              const uint32_t* x = reinterpret_cast<const uint32_t*>(c.data) + b;
              if (sl.ctype == DQ_I32)
                for (int j = 0; j < n; ++j) dst[j] = (uint64_t)(int64_t)(int32_t)x[j];
              else
                for (int j = 0; j < n; ++j) dst[j] = canon(x[j], sl.ctype);
              break;
            }
            default: {
              const uint64_t* x = reinterpret_cast<const uint64_t*>(c.data) + b;
              for (int j = 0; j < n; ++j) dst[j] = canon(x[j], sl.ctype);
              break;
            }
          }
        } else {
          const Resource& r = res[d.source_res];
          const int col = atoi(d.cols[sl.src]);
          const int wd = width_of(r.d->pay_ctype[col]);
          for (int j = 0; j < n; ++j)
            dst[j] = canon(truncate(r.rows.v[(size_t)(b + j) * r.rows.width + col], wd), sl.ctype);
        }
      } else if (sl.kind == DQ_SLOT_AGGKEY || sl.kind == DQ_SLOT_AGGVAL) {
        const Resource& r = res[sl.res];
        for (int j = 0; j < n; ++j) {
          if (r.agg.n() == 0) {  // no group yet: a table without keys still has its one row
            dst[j] = sl.kind == DQ_SLOT_AGGVAL && r.d->agg_red[sl.src] == DQ_RED_MIN ? canon(~0ull, sl.ctype) : 0;
            continue;
          }
          const uint64_t* g = &r.agg.rows[(size_t)(b + j) * r.agg.width];
          dst[j] = canon(sl.kind == DQ_SLOT_AGGKEY ? g[sl.src] : g[r.d->nkeys + sl.src], sl.ctype);
        }
      }
    }
  }

  // Multimap: the build rows grouped by key (a run of rows per key) and an
  // index from each key to its run.  Rows are partitioned by their key hash
  // (one partition per thread, in parallel), each partition is sorted by
  // (hash, key words) in parallel, and runs of equal keys are indexed.
  void group_rows(Resource& r, std::vector<Worker>& workers) {
    const bool trace = getenv("DQCPU_TRACE") != nullptr;
    auto t0 = std::chrono::steady_clock::now();
    auto mark = [&](const char* what) {
      if (!trace) return;
      const auto t1 = std::chrono::steady_clock::now();
      fprintf(stderr, "  group_rows %s: %.3f ms\n", what, std::chrono::duration<double, std::milli>(t1 - t0).count());
      t0 = t1;
    };
    const int W = r.rows.width;
    const int nk = r.d->nkeys;
    const KeyHash& kh = r.agg.kh;   // string keys compare by their bytes
    const int P = threads;
    const int nw = (int)workers.size();
    std::vector<std::vector<uint64_t>> hashes(nw);
    std::vector<int64_t> cnt((size_t)nw * P, 0);
    parallel(nw, [&](int w) {
      const Rows& o = workers[w].out;
      hashes[w].resize((size_t)o.n());
      for (int64_t i = 0; i < o.n(); ++i) {
        const uint64_t h = r.agg.kh(&o.v[(size_t)i * W]);
        hashes[w][i] = h;
        ++cnt[(size_t)w * P + (int)((h >> 40) % (uint64_t)P)];
      }
    });
    mark("hash");
    std::vector<int64_t> off((size_t)nw * P, 0), pstart(P + 1, 0);
    int64_t total = 0;
    for (int q = 0; q < P; ++q) {
      pstart[q] = total;
      for (int w = 0; w < nw; ++w) {
        off[(size_t)w * P + q] = total;
        total += cnt[(size_t)w * P + q];
      }
    }
    pstart[P] = total;
    std::vector<uint64_t> part((size_t)total * W), phash((size_t)total);
    parallel(nw, [&](int w) {
      const Rows& o = workers[w].out;
      std::vector<int64_t> pos(off.begin() + (size_t)w * P, off.begin() + (size_t)(w + 1) * P);
      for (int64_t i = 0; i < o.n(); ++i) {
        const uint64_t h = hashes[w][i];
        const int64_t d = pos[(int)((h >> 40) % (uint64_t)P)]++;
        std::copy(&o.v[(size_t)i * W], &o.v[(size_t)(i + 1) * W], &part[(size_t)d * W]);
        phash[d] = h;
      }
    });
    mark("partition");
    Rows sorted;
    sorted.width = W;
    sorted.v.resize(part.size());
    std::vector<int64_t> run((size_t)total, 0);
    parallel(P, [&](int q) {
      const int64_t lo = pstart[q], hi = pstart[q + 1];
      // sort (hash, row) pairs; rows with equal hashes but different keys
      // (rare) are then ordered by their keys
      std::vector<std::pair<uint64_t, int64_t>> idx((size_t)(hi - lo));
      for (int64_t i = lo; i < hi; ++i) idx[i - lo] = {phash[i], i};
      std::sort(idx.begin(), idx.end());
      auto key_less = [&](const std::pair<uint64_t, int64_t>& a, const std::pair<uint64_t, int64_t>& b) {
        const int c = kh.cmp(&part[(size_t)a.second * W], &part[(size_t)b.second * W]);
        return c != 0 ? c < 0 : a.second < b.second;
      };
      for (size_t a = 0; a < idx.size();) {
        size_t b = a + 1;
        while (b < idx.size() && idx[b].first == idx[a].first) ++b;
        bool mixed = false;
        for (size_t c = a + 1; c < b && !mixed; ++c)
          mixed = !kh.eq(&part[(size_t)idx[c].second * W], &part[(size_t)idx[a].second * W]);
        if (mixed) std::sort(idx.begin() + a, idx.begin() + b, key_less);
        a = b;
      }
      int64_t start = lo;
      for (int64_t i = lo; i < hi; ++i) {
        const int64_t src = idx[i - lo].second;
        std::copy(&part[(size_t)src * W], &part[(size_t)(src + 1) * W], &sorted.v[(size_t)i * W]);
        if (i > lo && !kh.eq(&sorted.v[(size_t)i * W], &sorted.v[(size_t)(i - 1) * W])) {
          run[start] = i - start;
          start = i;
        }
      }
      if (hi > lo) run[start] = hi - start;
    });
    mark("sort");
    r.rows = std::move(sorted);
    r.run_len = std::move(run);
    std::vector<int64_t> starts;
    for (int64_t q = 0; q < total; q += std::max<int64_t>(r.run_len[q], 1)) starts.push_back(q);
    uint64_t cap = 16;
    while (cap < starts.size() * 2) cap <<= 1;
    r.index.slot.assign(cap, -1);
    r.index.mask = cap - 1;
    for (int64_t q : starts) {
      uint64_t h = r.agg.kh(&r.rows.v[(size_t)q * W]) & r.index.mask;
      while (r.index.slot[h] >= 0) h = (h + 1) & r.index.mask;
      r.index.slot[h] = q;
    }
    mark("index");
  }

  template <class F>
  static void parallel(int n, F f) {
    std::vector<std::exception_ptr> errs(n);
    auto body = [&](int i) {
      try {
        f(i);
      } catch (...) {
        errs[i] = std::current_exception();
      }
    };
    std::vector<std::thread> pool;
    for (int i = 1; i < n; ++i) pool.emplace_back(body, i);
    if (n > 0) body(0);
    for (auto& t : pool) t.join();
    for (auto& e : errs)
      if (e) std::rethrow_exception(e);
  }

  void merge(const Pipeline& p, const dq_op& sink, std::vector<Worker>& workers) {
    Resource& r = res[sink.res];
    switch (sink.kind) {
      case DQ_OP_AGG: {
        // partitions of the key hash, one per thread, merged in parallel
        const int P = threads;
        std::vector<AggTable> part(P);
        auto body = [&](int q) {
          AggTable& t = part[q];
          t.init(r.d, &strs, 1024);
          for (auto& w : workers)
            for (int64_t g = 0; g < w.agg.n(); ++g) {
              const uint64_t h = w.agg.hashes[g];
              if ((int)((h >> 40) % (uint64_t)P) != q) continue;
              const uint64_t* src = &w.agg.rows[(size_t)g * w.agg.width];
              uint64_t* dst = t.group(src, h);
              for (int j = 0; j < r.d->naggs; ++j) combine(r.d->agg_red[j], dst[r.d->nkeys + j], src[r.d->nkeys + j]);
            }
        };
        std::vector<std::thread> pool;
        for (int q = 1; q < P; ++q) pool.emplace_back(body, q);
        body(0);
        for (auto& th : pool) th.join();
        AggTable& all = r.agg;
        uint64_t total = 0;
        for (auto& t : part) total += (uint64_t)t.n();
        all.init(r.d, &strs, total);
        for (auto& t : part)
          for (int64_t g = 0; g < t.n(); ++g) {
            const uint64_t* src = &t.rows[(size_t)g * t.width];
            uint64_t* dst = all.group(src, t.hashes[g]);
            for (int j = 0; j < r.d->naggs; ++j) dst[r.d->nkeys + j] = src[r.d->nkeys + j];
          }
        break;
      }
      case DQ_OP_BUILD:
      case DQ_OP_MM_SCATTER: {
        r.rows.width = sink.nlist + sink.nlist2;
        r.rows.v.clear();
        for (auto& w : workers) r.rows.v.insert(r.rows.v.end(), w.out.v.begin(), w.out.v.end());
        r.agg.kh.r = r.d;
        r.agg.kh.strs = &strs;
        if (sink.kind == DQ_OP_BUILD) {
          r.unique.build(r.rows, r.d->nkeys, r.agg.kh);
          r.rows.v.clear();
          r.rows.v.shrink_to_fit();
        } else {
          group_rows(r, workers);
        }
        break;
      }
      case DQ_OP_EMIT: {
        Rows& o = r.rows;
        o.width = sink.nlist;
        for (auto& w : workers) o.v.insert(o.v.end(), w.out.v.begin(), w.out.v.end());
        break;
      }
      default:
        break;
    }
    (void)p;
  }
};

struct Result {
  int64_t nrows = 0;
  std::vector<int32_t> ctypes;
  std::vector<std::vector<uint64_t>> cols;     // values, or nrows+1 offsets for strings
  std::vector<std::vector<uint8_t>> heaps;
};

}  // namespace

extern "C" {

typedef struct {
  const char* name;
  int32_t ncols;
  const dq_column* cols;
  int64_t nrows;
} dqcpu_table;

const char* dqcpu_last_error(void) { return g_error.c_str(); }

// Freed memory stays with the process (no trimming, large blocks from the
// heap rather than fresh mappings), so that repeated runs reuse pages instead
// of faulting in new ones: first touches of fresh pages otherwise dominate
// the grouping of large build sides on some hosts.
__attribute__((constructor)) static void keep_freed_memory() {
  mallopt(M_MMAP_THRESHOLD, 1 << 30);
  mallopt(M_TRIM_THRESHOLD, -1);
}

int dqcpu_run(const dq_plan_desc* desc, int32_t ntables, const dqcpu_table* tables, int32_t threads, void** out) {
  try {
    if (!desc || !out || ntables < 0 || (ntables && !tables)) throw Fail("bad arguments");
    *out = nullptr;
    std::unordered_map<std::string, Table> db;
    for (int i = 0; i < ntables; ++i) {
      Table& t = db[tables[i].name];
      t.nrows = tables[i].nrows;
      for (int c = 0; c < tables[i].ncols; ++c) {
        const dq_column& dc = tables[i].cols[c];
        Column& col = t.cols[dc.name];
        col.ctype = dc.ctype;
        col.width = dc.width;
        col.data = static_cast<const uint8_t*>(dc.data);
        col.offsets = dc.offsets;
      }
    }
    Plan plan;
    plan.d = desc;
    plan.threads = threads > 0 ? threads : (int)std::max(1u, std::thread::hardware_concurrency());
    plan.res.resize(desc->nres);
    for (int i = 0; i < desc->nres; ++i) {
      plan.res[i].d = &desc->res[i];
      plan.res[i].agg.init(&desc->res[i], &plan.strs, 64);
    }
    std::unordered_map<const Column*, int> sid_of;
    plan.pipes.resize(desc->npipes);
    for (int i = 0; i < desc->npipes; ++i) {
      Pipeline& p = plan.pipes[i];
      p.d = &desc->pipes[i];
      if (p.d->source_kind == DQ_SRC_TABLE) {
        auto it = db.find(p.d->table ? p.d->table : "");
        if (it == db.end()) throw Fail(std::string("unknown table ") + (p.d->table ? p.d->table : "?"));
        p.table = &it->second;
        for (int c = 0; c < p.d->ncols; ++c) {
          auto ci = p.table->cols.find(p.d->cols[c]);
          if (ci == p.table->cols.end()) throw Fail(std::string("unknown column ") + p.d->cols[c]);
          p.cols.push_back(&ci->second);
        }
      }
      p.sid.assign(p.d->nslots, 0);
      for (int s = 0; s < p.d->nslots; ++s)
        if (p.d->slots[s].kind == DQ_SLOT_STR) {
          const Column* c = p.cols.at(p.d->slots[s].src);
          auto f = sid_of.find(c);
          if (f == sid_of.end()) {
            f = sid_of.emplace(c, (int)plan.strs.src.size()).first;
            plan.strs.src.push_back(c);
          }
          p.sid[s] = f->second;
        }
      for (int q = 0; q < p.d->npatterns; ++q) p.patterns.emplace_back(p.d->patterns[q] ? p.d->patterns[q] : "");
    }
    const bool trace = getenv("DQCPU_TRACE") != nullptr;
    for (auto& p : plan.pipes) {
      const auto t0 = std::chrono::steady_clock::now();
      plan.run_pipeline(p);
      if (trace)
        fprintf(stderr, "pipeline %d: %.3f ms\n", (int)(&p - plan.pipes.data()),
                std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count());
    }

    // the result: the OUTPUT resource's rows, strings resolved
    const Resource& o = plan.res.at(desc->result_res);
    std::unique_ptr<Result> res(new Result());
    res->nrows = o.rows.n();
    const int nc = o.d->npay;
    res->cols.resize(nc);
    res->heaps.resize(nc);
    for (int j = 0; j < nc; ++j) {
      const int t = o.d->pay_ctype[j];
      res->ctypes.push_back(t);
      auto& col = res->cols[j];
      if (t == DQ_STR) {
        col.push_back(0);
        for (int64_t r = 0; r < res->nrows; ++r) {
          const uint8_t* s;
          int n;
          plan.strs.at(o.rows.v[(size_t)r * o.rows.width + j], s, n);
          res->heaps[j].insert(res->heaps[j].end(), s, s + n);
          col.push_back(res->heaps[j].size());
        }
      } else {
        col.resize((size_t)res->nrows);
        for (int64_t r = 0; r < res->nrows; ++r)
          col[r] = canon(truncate(o.rows.v[(size_t)r * o.rows.width + j], width_of(t)), t);
      }
    }
    *out = res.release();
    return DQ_OK;
  } catch (const std::exception& e) {
    g_error = e.what();
    return DQ_ERR_UNSUPPORTED;
  }
}

int dqcpu_result_shape(void* r, int64_t* nrows, int32_t* ncols) {
  Result* res = static_cast<Result*>(r);
  *nrows = res->nrows;
  *ncols = (int32_t)res->ctypes.size();
  return DQ_OK;
}

// Column j: its type, its values (canonical 64-bit words) or, for strings,
// nrows+1 offsets into the heap.
int dqcpu_result_column(void* r, int32_t j, int32_t* ctype, const uint64_t** values, const uint8_t** heap,
                        uint64_t* nchars) {
  Result* res = static_cast<Result*>(r);
  if (j < 0 || j >= (int32_t)res->ctypes.size()) return DQ_ERR_INVALID;
  *ctype = res->ctypes[j];
  *values = res->cols[j].data();
  *heap = res->heaps[j].data();
  *nchars = res->heaps[j].size();
  return DQ_OK;
}

void dqcpu_result_free(void* r) { delete static_cast<Result*>(r); }

}  // extern "C"
