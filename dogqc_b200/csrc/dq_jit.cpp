// Per-pipeline kernel generator and NVRTC compiler (host code).
//
// A generated pipeline kernel processes one row per lane and keeps every
// value in registers: the ops of the pipeline become straight-line code, so
// the per-row cost is the work of the ops themselves, not the interpretation
// of an op list.  The structure of every kernel:
//
//   * a grid-stride loop over the source, `rows_per_thread` rows per thread
//     per step (row = base + u * 256 + thread), with the staged columns of all
//     of them loaded before any is processed (coalesced, independent loads);
//   * filters and probes clear a lane's `act` flag; when no lane of a warp is
//     active the warp skips to its next row;
//   * a multimap probe (EXPAND) is distributed over the warp, the reference's
//     warp-level push-down expansion (dogqc/hashJoins.py:599-681): the lanes'
//     match ranges are scanned, then the warp walks the concatenated
//     (row, match) pairs 32 at a time, each lane taking one pair and the
//     parent row's values by shuffle.  Ranges longer than a threshold are
//     handed to a second kernel in which whole CTAs split them;
//   * aggregation is pre-combined where the group count allows: in registers
//     for a single group, in a CTA-local shared-memory table whose
//     accumulators are replicated 16 ways (lane % 16) so that lanes of one warp
//     do not collide on hot groups, and in the global table otherwise;
//   * emits reserve output rows once per warp (ballot + one atomic).
//
// Table layouts, hashing and value semantics are the shared helpers of
// dq_common.cuh, embedded with the other device headers as in-memory headers.
#include "dq_jit.h"

#include <dlfcn.h>
#include <nvrtc.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <vector>

#include "dq_jit_embed.inc"  // kEmbedCount, kEmbedNames[], kEmbedText[] (written by build.py)

namespace dq {
namespace jit {
namespace {

constexpr int kStripedMax = 12 * 1024;      // shared memory a replicated CTA-local aggregation table may take
constexpr int kBlock = kThreads;
constexpr int kWarpBuf = 64;                // rows one warp's divergence buffer holds
constexpr int kStrSlotWords = 6;            // a CTA-local group slot's string: location, length, 4 words

const char* ct_name(int t) {
  switch (t) {
    case DQ_I8: return "DQ_I8";
    case DQ_I32: return "DQ_I32";
    case DQ_U32: return "DQ_U32";
    case DQ_I64: return "DQ_I64";
    default: return "DQ_U64";
  }
}

const char* red_name(int r) {
  switch (r) {
    case DQ_RED_SUM: return "DQ_RED_SUM";
    case DQ_RED_COUNT: return "DQ_RED_COUNT";
    case DQ_RED_MIN: return "DQ_RED_MIN";
    default: return "DQ_RED_MAX";
  }
}

const char* arith_name(int s) {
  switch (s) {
    case DQ_ADD: return "DQ_ADD";
    case DQ_SUB: return "DQ_SUB";
    case DQ_MUL: return "DQ_MUL";
    case DQ_DIV: return "DQ_DIV";
    default: return "DQ_MOD";
  }
}

const char* cmp_name(int s) {
  switch (s) {
    case DQ_EQ: return "DQ_EQ";
    case DQ_NE: return "DQ_NE";
    case DQ_LT: return "DQ_LT";
    case DQ_LE: return "DQ_LE";
    case DQ_GT: return "DQ_GT";
    default: return "DQ_GE";
  }
}

const char* uint_type(int w) {
  switch (w) {
    case 1: return "uint8_t";
    case 2: return "uint16_t";
    case 4: return "uint32_t";
    default: return "uint64_t";
  }
}

std::string lit(uint64_t v) {
  char b[40];
  snprintf(b, sizeof b, "0x%llxull", (unsigned long long)v);
  return b;
}

std::string num(long long v) { return std::to_string(v); }

// Slots an op reads (same rule as the runtime's validation).
void op_reads(const DevPipe& P, const dq_op& op, std::vector<int>& out) {
  auto add = [&](int s) {
    if (s >= 0) out.push_back(s);
  };
  auto add_list = [&](int list, int n) {
    for (int i = 0; i < n; ++i) add(P.lists[list + i]);
  };
  switch (op.kind) {
    case DQ_OP_ARITH:
    case DQ_OP_CMP:
    case DQ_OP_CAST:
      if (!(op.flags & DQ_OPF_A_IMM)) add(op.a);
      if (op.kind != DQ_OP_CAST && !(op.flags & DQ_OPF_B_IMM)) add(op.b);
      break;
    case DQ_OP_LOGIC:
      add(op.a);
      if (op.sub != DQ_NOT) add(op.b);
      break;
    case DQ_OP_SELECT:
      add(op.a);
      if (!(op.flags & DQ_OPF_B_IMM)) add(op.b);
      add(op.c >= 0 ? op.c : op.dst);
      break;
    case DQ_OP_STREQ:
      add(op.a);
      if (op.res < 0) add(op.b);
      break;
    case DQ_OP_LIKE:
    case DQ_OP_STRREF:
    case DQ_OP_SUBSTR:
    case DQ_OP_FILTER:
      add(op.a);
      break;
    case DQ_OP_PROBE:
    case DQ_OP_EXISTS:
    case DQ_OP_EXPAND:
    case DQ_OP_MM_COUNT:
      add_list(op.list, op.nlist);
      if (op.kind == DQ_OP_EXPAND) add_list(op.list2, op.nlist2);
      break;
    case DQ_OP_AGG:
    case DQ_OP_BUILD:
    case DQ_OP_MM_SCATTER:
      add_list(op.list, op.nlist);
      add_list(op.list2, op.nlist2);
      break;
    case DQ_OP_EMIT:
      add_list(op.list, op.nlist);
      break;
  }
}

enum AggMode { AGG_NONE, AGG_REGS, AGG_STRIPED, AGG_LOCAL, AGG_GLOBAL };

struct Gen {
  const DevPipe& P;
  int expand_op;
  std::string o;
  int ind = 0;
  int uid = 0;
  std::vector<std::string> var;  // slot -> C variable holding its canonical value
  std::string row;               // level-0 row index of the current lane
  AggMode agg = AGG_NONE;
  int agg_res = -1;
  int ns = 0;                    // local table slots (without the all-ones slot)
  int copies = 1;
  int U = 1;
  int smem = 0;
  std::string pay_reg;           // probe payload already loaded with its tag
  std::vector<int> prefetch;     // probes whose first slot pair is loaded early
  std::map<int, std::string> pending;  // gathered slots not loaded yet -> match index
  int min_blocks = 0;            // __launch_bounds__ minimum CTAs per SM (0: none)
  int refill = -1;               // op after which lanes are refilled (-1: none)
  int refill_threshold = 32;     // buffered rows that make the warp process them
  int nbuf = 0;                  // values per row in the warp buffers
  int buf_off = 0;               // shared-memory offset of the warp buffers
  int hot = 0;                   // multimap sink through the CTA's hot-bucket table:
                                 // 1 count (flushed at the end), 2 scatter (per step)
  int hot_off = 0;               // shared-memory offset of that table
  std::string inst_expr = "0u";  // the instance a deferred item belongs to (batches)
  std::string ldfn = "__ldcs";   // load function of streamed source columns
  std::vector<std::pair<int, int>> bitmaps;  // key-domain bitmaps probed: (resource, smem offset)
  const std::string* patterns = nullptr;     // host copy of the pattern bytes (P.pat_off into it)
  std::vector<std::string> str_ptr, str_len;  // located string keys of the last str_key_hashes
  std::vector<std::string> str_words;         // and their words (strings of at most kStrCoopMin bytes)
  bool single_cta = false;       // the tail function: one CTA scans the whole source
  bool tail_call = false;        // the main kernel's last CTA calls dq_tail
  int block = kBlock;            // threads per CTA
  bool batched = false;          // kernel over many instances of the plan
  // whether the current step is the lane's last (the refill buffer drains then)
  std::string last_step = "base + (int64_t)gridDim.x * span >= nrows";

  Gen(const DevPipe& p, int e) : P(p), expand_op(e), var(p.nslots) {}

  static bool narrow(int t) { return t == DQ_I8 || t == DQ_I32 || t == DQ_U32; }

  // Tag of a packed-key table (the value key_tag computes), from a slot list.
  std::string packed_tag(int r, int list, int n) {
    const DevRes& R = P.res[r];
    std::string t = fresh("tg");
    auto key = [&](int i) { return "canon(" + V(P.lists[list + i]) + ", " + ct_name(R.key_ctype[i]) + ")"; };
    if (n == 0) L("const uint64_t " + t + " = 0ull;");
    else if (n == 1 && !narrow(R.key_ctype[0])) L("const uint64_t " + t + " = " + key(0) + ";");
    else if (n == 1) L("const uint64_t " + t + " = (uint64_t)(uint32_t)" + key(0) + ";");
    else L("const uint64_t " + t + " = (uint64_t)(uint32_t)" + key(0) + " | ((uint64_t)(uint32_t)" + key(1) + " << 32);");
    return t;
  }

  // Whether a packed tag can equal the empty marker (all ones).
  bool tag_can_be_empty(int r) const {
    const DevRes& R = P.res[r];
    return !(R.nkeys == 1 && narrow(R.key_ctype[0])) && R.nkeys > 0;
  }

  // Declares `int64_t g_`: the global aggregation slot of packed tag `tag`
  // (agg_slot_global's packed-key claim, inline: find the tag or claim an empty
  // slot with a compare-and-swap; the all-ones key has its own slot).  Inline
  // because a call needs an ABI stack frame in the calling kernel.
  void packed_claim(int r, const std::string& tag) {
    const DevRes& R = P.res[r];
    const std::string W = num(R.words);
    L("int64_t g_ = -1;");
    L("{");
    ++ind;
    L("uint64_t* const gs_ = " + res(r) + ".slots;");
    L("const uint32_t gc_ = (uint32_t)" + res(r) + ".cap;");
    if (tag_can_be_empty(r)) {
      L("if (" + tag + " == kEmpty) {");
      L("  atomicCAS((unsigned long long*)(gs_ + (uint64_t)gc_ * " + W + "), kEmpty, 0ull);");
      L("  g_ = (int64_t)gc_;");
      L("} else {");
      ++ind;
    }
    L("uint32_t i_ = slot_of(" + tag + ", gc_);");
    L("for (uint32_t n_ = 0; n_ < gc_; ++n_) {");
    ++ind;
    L("uint64_t* const s_ = gs_ + (uint64_t)i_ * " + W + ";");
    L("const uint64_t t_ = *(volatile uint64_t*)s_;");
    L("if (t_ == " + tag + ") { g_ = (int64_t)i_; break; }");
    L("if (t_ == kEmpty) {");
    L("  const uint64_t o_ = atomicCAS((unsigned long long*)s_, kEmpty, " + tag + ");");
    L("  if (o_ == kEmpty || o_ == " + tag + ") { g_ = (int64_t)i_; break; }");
    L("}");
    L("i_ = (i_ + 1u == gc_) ? 0u : i_ + 1u;");
    --ind;
    L("}");
    L("if (g_ < 0) set_status(P, kErrHtFull);");
    if (tag_can_be_empty(r)) {
      --ind;
      L("}");
    }
    --ind;
    L("}");
  }

  void L(const std::string& s) {
    o.append((size_t)ind * 2, ' ');
    o += s;
    o += '\n';
  }
  std::string fresh(const char* b) { return std::string(b) + num(uid++); }
  const DevSlot& slot(int s) const { return P.slots[s]; }
  std::string V(int s) const {
    if (s < 0 || s >= P.nslots || var[s].empty()) throw Error("generated code reads an undefined slot " + num(s));
    return var[s];
  }
  std::string res(int r) const { return "P.res[" + num(r) + "]"; }
  std::string operand(const dq_op& op, int which) const {
    if (which == 0) return (op.flags & DQ_OPF_A_IMM) ? lit((uint64_t)op.imm) : V(op.a);
    return (op.flags & DQ_OPF_B_IMM) ? lit((uint64_t)op.imm) : V(op.b);
  }
  std::string assign(int dst, const std::string& expr, int op_ctype) const {
    return V(dst) + " = canon(canon(" + expr + ", " + ct_name(op_ctype) + "), " + ct_name(slot(dst).ctype) + ");";
  }

  // keys of a resource from a slot list, canonicalised to the key types
  // Declares nothing; sets p/n to the bytes of string slot s (a string
  // column read at `row`, or a reference held in a value).
  void str_bytes(int s, const std::string& row, const std::string& p, const std::string& n) {
    const DevSlot& sl = slot(s);
    if (sl.ctype != DQ_STR) throw Error("string op on a non-string slot");
    if (sl.kind == DQ_SLOT_STR) L("str_at(P.strs[" + num(sl.src) + "], " + row + ", " + p + ", " + n + ");");
    else L(locate_ref(s, p, n) + ";");
  }

  // The pipeline string a reference slot holds when one STRREF op writes it
  // (no window; its source known here), else -1.
  int ref_source(int s) const {
    int src = -1, writers = 0;
    for (int k = 0; k < P.nops; ++k) {
      const dq_op& op = P.ops[k];
      if (op.dst != s) continue;
      ++writers;
      if (op.kind == DQ_OP_STRREF && slot(op.a).kind == DQ_SLOT_STR) src = slot(op.a).src;
    }
    return writers == 1 ? src : -1;
  }

  // Locating the bytes behind reference slot s: straight from the pipeline's
  // string column when its source is known, else through the plan's sources.
  std::string locate_ref(int s, const std::string& p, const std::string& n) const {
    const int src = ref_source(s);
    if (src >= 0)
      return "str_at(P.strs[" + num(src) + "], (int64_t)(" + V(s) + " & kStrRefRow), " + p + ", " + n + ")";
    return "str_ref_at(P, " + V(s) + ", " + p + ", " + n + ")";
  }

  // Bucket of a multimap key held in array kk (string keys: their hashes in sh).
  std::string bucket(const dq_op& op, int r, const std::string& kk, const std::string& sh) {
    if (has_str_key(P.res[r]))
      return "bucket_of_strh(" + res(r) + ", " + kk + ", " + sh + ", " + num(op.nlist) + ", (uint32_t)" + res(r) +
             ".cap)";
    return "bucket_of(" + kk + ", " + num(op.nlist) + ", (uint32_t)" + res(r) + ".cap)";
  }

  // Hashes of the string values among a key list, computed by the whole warp
  // where its lanes have not branched (long strings cooperatively, a word per
  // lane); the array's other entries stay 0.  Empty when resource r has no
  // string keys.
  // The bytes behind each string key are located once (str_ptr / str_len
  // name them, per key index) for the comparisons that follow.  All keys are
  // located first and the short ones hashed by their lanes with independent
  // loads, so the loads of several keys overlap; long ones go to the warp.
  std::string str_key_hashes(int r, int list, int n, const std::string& act) {
    str_ptr.assign((size_t)std::max(n, 0), std::string());
    str_len.assign((size_t)std::max(n, 0), std::string());
    str_words.assign((size_t)std::max(n, 0), std::string());
    if (!has_str_key(P.res[r])) return std::string();
    const std::string h = fresh("sh");
    L("uint64_t " + h + "[" + num(std::max(n, 1)) + "] = {};");
    for (int i = 0; i < n; ++i)
      if (P.res[r].key_ctype[i] == DQ_STR) {
        const std::string sp = fresh("skp"), sn = fresh("skn");
        L("const uint8_t* " + sp + " = nullptr;");
        L("int " + sn + " = 0;");
        L("if (" + act + ") " + locate_ref(P.lists[list + i], sp, sn) + ";");
        str_ptr[(size_t)i] = sp;
        str_len[(size_t)i] = sn;
      }
    for (int i = 0; i < n; ++i)
      if (P.res[r].key_ctype[i] == DQ_STR) {
        const std::string w = fresh("skw");
        L("uint64_t " + w + "[kStrShortWords] = {};");
        L("if (" + act + " && " + str_len[(size_t)i] + " <= kStrCoopMin) {");
        L("  str_words_short(" + str_ptr[(size_t)i] + ", " + str_len[(size_t)i] + ", " + w + ");");
        L("  " + h + "[" + num(i) + "] = str_hash_words(" + w + ", " + str_len[(size_t)i] + ");");
        L("}");
        str_words[(size_t)i] = w;
      }
    for (int i = 0; i < n; ++i)
      if (P.res[r].key_ctype[i] == DQ_STR) {
        const std::string wide = "(" + act + " && " + str_len[(size_t)i] + " > kStrCoopMin)";
        L("if (__any_sync(kFull, " + wide + ")) " + h + "[" + num(i) + "] = str_hash_wide(" + wide + ", " +
          str_ptr[(size_t)i] + ", " + str_len[(size_t)i] + ", " + h + "[" + num(i) + "]);");
      }
    return h;
  }

  // CTA-local group slot of a key with strings: linear probing over ns slots
  // of ltags; a claim publishes the key values (lkeys, for the flush) and,
  // per string, its location, length and words (lstr: kStrSlotWords words)
  // before the tag.  A row whose tag matches compares lengths and words (a
  // string of at most kStrCoopMin bytes) or its bytes with the slot string's
  // (a longer one), without locating the slot's string again.  s_ stays -1
  // when the table is full or a claim stays unpublished past the wait limit
  // (the caller aggregates into the global table).
  void local_str_slot(int r, const std::string& k) {
    const DevRes& R = P.res[r];
    const std::string NK = num(R.nkeys), NS = num(ns), NSTR = num(nstr_keys(R));
    L("int s_ = -1;");
    L("{");
    ++ind;
    L("uint32_t i_ = slot_of(tag_, " + NS + "u);");
    L("for (int n_ = 0; n_ < " + NS + "; ++n_) {");
    ++ind;
    L("uint64_t t_ = ((volatile uint64_t*)ltags)[i_];");
    L("if (t_ == kEmpty) {");
    ++ind;
    L("const uint64_t o_ = s_cas64(saddr(&ltags[i_]), kEmpty, kBusy);");
    L("if (o_ == kEmpty) {");
    ++ind;
    for (int q = 0, j = 0; q < R.nkeys; ++q) {
      L("((volatile uint64_t*)lkeys)[i_ * " + NK + " + " + num(q) + "] = " + k + "[" + num(q) + "];");
      if (R.key_ctype[q] != DQ_STR) continue;
      const std::string at = "((volatile uint64_t*)lstr)[(i_ * " + NSTR + " + " + num(j) + ") * " + num(kStrSlotWords);
      L(at + "] = (uint64_t)" + str_ptr[(size_t)q] + ";");
      L(at + " + 1] = (uint64_t)" + str_len[(size_t)q] + ";");
      for (int w = 0; w < kStrSlotWords - 2; ++w)
        L(at + " + " + num(2 + w) + "] = " + str_words[(size_t)q] + "[" + num(w) + "];");
      ++j;
    }
    L("__threadfence_block();");
    L("((volatile uint64_t*)ltags)[i_] = tag_;");
    L("s_ = (int)i_;");
    L("break;");
    --ind;
    L("}");
    L("t_ = o_;");
    --ind;
    L("}");
    L("for (long long w_ = 0; t_ == kBusy && w_ < kSpinLimit; ++w_) t_ = ((volatile uint64_t*)ltags)[i_];");
    L("if (t_ == kBusy) break;");
    L("if (t_ == tag_) {");
    ++ind;
    L("__threadfence_block();");
    std::string eq;
    for (int q = 0, j = 0; q < R.nkeys; ++q) {
      if (!eq.empty()) eq += " && ";
      if (R.key_ctype[q] != DQ_STR) {
        eq += "((volatile uint64_t*)lkeys)[i_ * " + NK + " + " + num(q) + "] == " + k + "[" + num(q) + "]";
        continue;
      }
      const std::string at = "((volatile uint64_t*)lstr)[(i_ * " + NSTR + " + " + num(j) + ") * " + num(kStrSlotWords);
      const std::string& n = str_len[(size_t)q];
      std::string words;
      for (int w = 0; w < kStrSlotWords - 2; ++w)
        words += (w ? " && " : "") + at + " + " + num(2 + w) + "] == " + str_words[(size_t)q] + "[" + num(w) + "]";
      eq += "(int)" + at + " + 1] == " + n + " && (" + n + " <= kStrCoopMin ? (" + words +
            ") : str_eq((const uint8_t*)" + at + "], " + n + ", " + str_ptr[(size_t)q] + ", " + n + "))";
      ++j;
    }
    L("if (" + eq + ") {");
    L("  s_ = (int)i_;");
    L("  break;");
    L("}");
    --ind;
    L("}");
    L("i_ = i_ + 1 == " + NS + "u ? 0u : i_ + 1;");
    --ind;
    L("}");
    --ind;
    L("}");
  }

  static int nstr_keys(const DevRes& R) {
    int n = 0;
    for (int q = 0; q < R.nkeys; ++q) n += R.key_ctype[q] == DQ_STR;
    return n;
  }

  // Equality of a probe key slot and a build key slot of resource r's key q.
  std::string key_eq(int r, int q, int a, int b) {
    const int t = P.res[r].key_ctype[q];
    if (t == DQ_STR) return "str_ref_eq(P, " + V(a) + ", " + V(b) + ")";
    return "canon(" + V(a) + ", " + ct_name(t) + ") == canon(" + V(b) + ", " + ct_name(t) + ")";
  }

  std::string keys(const dq_op& op, int r, int list, int n) {
    std::string k = fresh("kk");
    L("uint64_t " + k + "[" + num(std::max(n, 1)) + "];");
    for (int i = 0; i < n; ++i)
      L(k + "[" + num(i) + "] = canon(" + V(P.lists[list + i]) + ", " + ct_name(P.res[r].key_ctype[i]) + ");");
    (void)op;
    return k;
  }

  void declare_regs(int level) {
    for (int s = 0; s < P.nslots; ++s)
      if (slot(s).kind == DQ_SLOT_REG && slot(s).level == level) {
        var[s] = "v" + num(s);
        L("uint64_t " + var[s] + " = 0;");
      }
  }

  void skip_if_idle(const std::string& act, const std::string& exit) {
    L("if (!__any_sync(kFull, " + act + ")) " + exit);
  }

  // ---------------------------------------------------------------- ops --
  // One ARITH / CMP / LOGIC / CAST / SELECT op (straight-line C).
  void scalar_op(const dq_op& op) {
    switch (op.kind) {
      case DQ_OP_ARITH:
        L(assign(op.dst, std::string("arith(") + arith_name(op.sub) + ", " + ct_name(op.ctype) + ", " +
                             operand(op, 0) + ", " + operand(op, 1) + ")", op.ctype));
        break;
      case DQ_OP_CMP:
        L(assign(op.dst, std::string("(uint64_t)compare(") + cmp_name(op.sub) + ", " + ct_name(op.ctype) + ", " +
                             operand(op, 0) + ", " + operand(op, 1) + ")", DQ_U64));
        break;
      case DQ_OP_LOGIC:
        if (op.sub == DQ_NOT) L(assign(op.dst, "(uint64_t)(" + V(op.a) + " == 0ull)", DQ_U64));
        else
          L(assign(op.dst, "(uint64_t)(" + V(op.a) + (op.sub == DQ_AND ? " != 0ull && " : " != 0ull || ") +
                               V(op.b) + " != 0ull)", DQ_U64));
        break;
      case DQ_OP_CAST:
        L(assign(op.dst, operand(op, 0), op.ctype));
        break;
      case DQ_OP_SELECT: {
        std::string prev = V(op.c >= 0 ? op.c : op.dst);
        L(assign(op.dst, "(" + V(op.a) + " ? " + operand(op, 1) + " : " + prev + ")", op.ctype));
        break;
      }
      default:
        throw Error("op kind " + num(op.kind) + " is not a scalar op");
    }
  }

  void ops_from(int k, int level, const std::string& act, const std::string& exit) {
    for (; k < P.nops; ++k) {
      const dq_op& op = P.ops[k];
      if (!pending.empty()) {
        std::vector<int> reads;
        op_reads(P, op, reads);
        if (op.kind == DQ_OP_EXPAND) {
          std::vector<int> live = live_after(k, level);
          reads.insert(reads.end(), live.begin(), live.end());
        }
        materialize(reads, act);
      }
      switch (op.kind) {
        case DQ_OP_ARITH:
        case DQ_OP_CMP:
        case DQ_OP_LOGIC:
        case DQ_OP_CAST:
        case DQ_OP_SELECT:
          scalar_op(op);
          break;
        case DQ_OP_LIKE: {
          // a pattern '%L1%...%Ln%' (no '_', no empty literal) finds its
          // literals one after another, eight bytes a step; others run the
          // reference matcher's algorithm (like_match)
          std::vector<std::pair<int, int>> lits;  // (offset in the pattern buffer, length)
          bool simple = false;
          if (patterns) {
            const int o = P.pat_off[op.res], lp = P.pat_off[op.res + 1] - o;
            const std::string pat = patterns->substr((size_t)o, (size_t)lp);
            simple = lp >= 3 && pat.front() == '%' && pat.back() == '%' && pat.find('_') == std::string::npos;
            for (int i = 1, start = 1; simple && i < lp; ++i)
              if (pat[(size_t)i] == '%') {
                if (i == start) simple = false;
                else lits.emplace_back(o + start, i - start);
                start = i + 1;
              }
          }
          L(V(op.dst) + " = 0;");
          L("if (" + act + ") {");
          ++ind;
          L("const uint8_t* sp_; int sn_;");
          str_bytes(op.a, row, "sp_", "sn_");
          if (simple) {
            L("int lp_ = 0;");
            std::string cond;
            for (auto& l : lits)
              cond += (cond.empty() ? "" : " && ") + std::string("like_find(sp_, sn_, lp_, P.patterns + ") + num(l.first) +
                      ", " + num(l.second) + ")";
            L(V(op.dst) + " = (uint64_t)(" + cond + ");");
          } else {
            L(V(op.dst) + " = (uint64_t)like_match(sp_, sn_, P.patterns + P.pat_off[" + num(op.res) + "], P.pat_off[" +
              num(op.res + 1) + "] - P.pat_off[" + num(op.res) + "]);");
          }
          --ind;
          L("}");
          break;
        }
        case DQ_OP_STREQ: {
          L(V(op.dst) + " = 0;");
          L("if (" + act + ") {");
          ++ind;
          L("const uint8_t* sp_; int sn_;");
          str_bytes(op.a, row, "sp_", "sn_");
          if (op.kind == DQ_OP_STREQ && op.res < 0) {
            L("const uint8_t* sq_; int sm_;");
            str_bytes(op.b, row, "sq_", "sm_");
            L(V(op.dst) + " = (uint64_t)str_eq(sp_, sn_, sq_, sm_);");
          } else {
            std::string pat = "P.patterns + P.pat_off[" + num(op.res) + "]";
            std::string plen = "P.pat_off[" + num(op.res + 1) + "] - P.pat_off[" + num(op.res) + "]";
            L(V(op.dst) + std::string(" = (uint64_t)") + (op.kind == DQ_OP_LIKE ? "like_match" : "str_eq") +
              "(sp_, sn_, " + pat + ", " + plen + ");");
          }
          --ind;
          L("}");
          break;
        }
        case DQ_OP_SUBSTR: {
          if (slot(op.a).ctype != DQ_STR || slot(op.a).kind == DQ_SLOT_STR)
            throw Error("SUBSTR reads a string reference");
          L(V(op.dst) + " = str_ref_substring(" + V(op.a) + ", " + num((int32_t)(uint32_t)op.imm) + ", " +
            num((int32_t)(uint32_t)((uint64_t)op.imm >> 32)) + ");");
          break;
        }
        case DQ_OP_STRREF: {  // the string's plan-wide reference: source, no window, row
          const DevSlot& sl = slot(op.a);
          if (sl.kind != DQ_SLOT_STR) throw Error("string reference of a non-string slot");
          L(V(op.dst) + " = ((uint64_t)(uint32_t)P.strs[" + num(sl.src) + "].sid << kStrRefShift) | (uint64_t)" + row +
            ";");
          break;
        }
        case DQ_OP_PROFILE:
          L("{");
          L("  const unsigned pm_ = __ballot_sync(kFull, " + act + ");");
          L("  if (lane == 0) atomicAdd((unsigned long long*)(P.profile + " + num(op.res * 33) + " + __popc(pm_)), 1ull);");
          L("}");
          break;
        case DQ_OP_FILTER:
          L(act + " = " + act + " && (" + V(op.a) + " != 0ull);");
          skip_if_idle(act, exit);
          if (k == refill && level == 0) {
            refill_lanes(k, act);
            return;
          }
          break;
        case DQ_OP_PROBE:
          probe(k, act);
          skip_if_idle(act, exit);
          if (k == refill && level == 0) {
            refill_lanes(k, act);
            return;
          }
          break;
        case DQ_OP_EXISTS:
          exists(k, level, act);
          k += (int)op.imm;  // the condition's ops ran inside the walk
          skip_if_idle(act, exit);
          break;
        case DQ_OP_EXPAND:
          expand(k, level, act);
          return;
        case DQ_OP_AGG:
          sink_agg(op, act);
          return;
        case DQ_OP_BUILD:
          sink_build(op, act);
          return;
        case DQ_OP_MM_COUNT:
        case DQ_OP_MM_SCATTER:
          sink_mm(op, act);
          return;
        case DQ_OP_EMIT:
          sink_emit(op, act);
          return;
        default:
          throw Error("op kind " + num(op.kind) + " has no generated form");
      }
    }
  }

  bool is_prefetched(int k) const {
    return std::find(prefetch.begin(), prefetch.end(), k) != prefetch.end();
  }

  // Probes whose first slot pair is loaded together with the row's columns:
  // packed-key join tables of at most two words, probed at level 0 before the
  // lane refill, with keys read straight from source columns.
  void choose_prefetch() {
    prefetch.clear();
    if (P.source_kind == DQ_SRC_AGG) return;
    for (int k = 0; k < P.nops; ++k) {
      const dq_op& op = P.ops[k];
      if (op.kind == DQ_OP_EXPAND || (refill >= 0 && k > refill)) break;
      if (op.kind != DQ_OP_PROBE) continue;
      const DevRes& R = P.res[op.res];
      if (R.bitmap == 1) continue;
      if (R.bitmap != 2 && (!R.packed || R.nkeys == 0 || R.words > 2 || tag_can_be_empty(op.res))) continue;
      bool cols = true;
      for (int i = 0; i < op.nlist; ++i) cols &= slot(P.lists[op.list + i]).kind == DQ_SLOT_COL;
      if (cols) prefetch.push_back(k);
    }
  }

  // Issues the first pair loads of the prefetched probes for row u (inside
  // the column-load loop, where c<col>[u] and in_ are defined).
  void prefetch_loads() {
    for (int k : prefetch) {
      const dq_op& op = P.ops[k];
      const int r = op.res;
      const DevRes& R = P.res[r];
      std::string key[2];
      for (int i = 0; i < op.nlist && i < 2; ++i) {
        const DevSlot& sl = slot(P.lists[op.list + i]);
        key[i] = "canon(canon(c" + num(sl.src) + "[u], " + ct_name(sl.ctype) + "), " + ct_name(R.key_ctype[i]) + ")";
      }
      std::string tag = op.nlist == 1 ? (narrow(R.key_ctype[0]) ? "(uint64_t)(uint32_t)" + key[0] : key[0])
                                      : "(uint64_t)(uint32_t)" + key[0] + " | ((uint64_t)(uint32_t)" + key[1] + " << 32)";
      L("{");
      ++ind;
      L("const uint64_t* const ht_ = " + res(r) + ".slots;");
      const std::string K = num(k);
      if (R.bitmap == 2) {
        // the key's word of a dense table
        L("const uint64_t o_ = (uint64_t)" + key[0] + " - (uint64_t)" + res(r) + ".bmin;");
        L("pw" + K + "_0[u] = in_ && o_ < " + res(r) + ".brange ? __ldg(reinterpret_cast<const unsigned long long*>(ht_) + o_) : 0ull;");
        --ind;
        L("}");
        continue;
      }
      if (R.compact) {
        // compact slots: the aligned 16-byte pair of the home slot
        L("const uint32_t p_ = slot_of(" + tag + ", (uint32_t)" + res(r) + ".cap) & ~1u;");
        L("if (in_) {");
        L("  ld_nc_16B(ht_ + (uint64_t)p_, pw" + K + "_0[u], pw" + K + "_1[u]);");
        L("} else {");
        L("  pw" + K + "_0[u] = pw" + K + "_1[u] = kEmpty;");
        L("}");
      } else {
        L("const uint32_t p_ = slot_of(" + tag + ", (uint32_t)" + res(r) + ".cap) & ~" + num(4 / R.words - 1) + "u;");
        L("if (in_) {");
        L("  ld_nc_32B(ht_ + (uint64_t)p_ * " + num(R.words) + ", pw" + K + "_0[u], pw" + K + "_1[u], pw" + K + "_2[u], pw" +
          K + "_3[u]);");
        L("} else {");
        L("  pw" + K + "_0[u] = pw" + K + "_1[u] = pw" + K + "_2[u] = pw" + K + "_3[u] = kEmpty;");
        L("}");
      }
      --ind;
      L("}");
    }
  }

  void probe(int k, const std::string& act) {
    const dq_op& op = P.ops[k];
    const int r = op.res;
    const DevRes& R = P.res[r];
    std::string s = fresh("ps");
    if (R.bitmap == 2) {
      // a payload word per key of the build column's domain
      const std::string key = "canon(" + V(P.lists[op.list]) + ", " + ct_name(R.key_ctype[0]) + ")";
      const bool with_pay = op.sub == DQ_JOIN_INNER && op.nlist2 > 0 && P.lists[op.list2] >= 0;
      L("int64_t " + s + " = -1;");
      L("if (" + act + ") {");
      ++ind;
      if (is_prefetched(k)) {
        L("const uint64_t w_ = pw" + num(k) + "_0[u];");
      } else {
        L("const uint64_t o_ = (uint64_t)" + key + " - (uint64_t)" + res(r) + ".bmin;");
        L("const uint64_t w_ = o_ < " + res(r) + ".brange ? __ldg(reinterpret_cast<const unsigned long long*>(" + res(r) +
          ".slots) + o_) : 0ull;");
      }
      L("if (w_) {");
      L("  " + s + " = 0;");
      if (with_pay) {
        const int d = P.lists[op.list2];
        L("  " + V(d) + " = canon(canon((uint64_t)(uint32_t)w_, " + ct_name(R.pay_ctype[0]) + "), " +
          ct_name(slot(d).ctype) + ");");
      }
      L("}");
      --ind;
      L("}");
      if (op.sub == DQ_JOIN_ANTI) L(act + " = " + act + " && " + s + " < 0;");
      else L(act + " = " + act + " && " + s + " >= 0;");
      return;
    }
    if (R.bitmap) {
      // a bit per key of the build column's domain
      const std::string key = "canon(" + V(P.lists[op.list]) + ", " + ct_name(R.key_ctype[0]) + ")";
      L("int64_t " + s + " = -1;");
      L("if (" + act + ") {");
      L("  const uint64_t o_ = (uint64_t)" + key + " - (uint64_t)" + res(r) + ".bmin;");
      L("  if (o_ < " + res(r) + ".brange && ((" + bitmap_words(r) + "[o_ >> 5] >> (o_ & 31u)) & 1u)) " + s + " = 0;");
      L("}");
      if (op.sub == DQ_JOIN_ANTI) L(act + " = " + act + " && " + s + " < 0;");
      else L(act + " = " + act + " && " + s + " >= 0;");
      return;
    }
    const std::string sh = str_key_hashes(r, op.list, op.nlist, act);
    L("int64_t " + s + " = -1;");
    L("if (" + act + ") {");
    ++ind;
    if (R.packed && R.nkeys > 0) {
      // packed keys: the tag is the key; linear probing with a 32-bit index
      const std::string tg = packed_tag(r, op.list, op.nlist);
      const std::string W = num(R.words);
      const bool ext = tag_can_be_empty(r);
      L("const uint64_t* const ht_ = " + res(r) + ".slots;");
      L("const uint32_t hc_ = (uint32_t)" + res(r) + ".cap;");
      if ((R.words == 2 || R.compact) && op.sub == DQ_JOIN_INNER && op.nlist2 > 0 && P.lists[op.list2] >= 0)
        L("uint64_t pv_ = 0;");
      if (R.compact) {
        // one word a slot: key << 32 | payload, read in aligned 16-byte pairs
        // (the slot count is even).  The walk compares the keys (high words);
        // an empty slot's key is all ones, a key the table never holds.
        const bool pf = is_prefetched(k);
        const bool with_pay = op.sub == DQ_JOIN_INNER && op.nlist2 > 0 && P.lists[op.list2] >= 0;
        L("const uint32_t k_ = (uint32_t)" + tg + ";");
        L("if (k_ == 0xffffffffu) {");
        L("  if (ht_[(uint64_t)hc_] == 0ull) { " + s + " = (int64_t)hc_;" + (with_pay ? " pv_ = ht_[(uint64_t)hc_ + 1];" : "") +
          " }");
        L("} else {");
        ++ind;
        L("uint32_t p_ = slot_of(" + tg + ", hc_);");
        L("uint32_t f_ = p_ & 1u;");
        L("p_ -= f_;");
        if (pf) {
          L("uint64_t w0_ = pw" + num(k) + "_0[u], w1_ = pw" + num(k) + "_1[u];");
        } else {
          L("uint64_t w0_, w1_;");
          L("ld_nc_16B(ht_ + (uint64_t)p_, w0_, w1_);");
        }
        L("for (uint32_t n_ = 0;;) {");
        ++ind;
        L("if ((uint32_t)(w0_ >> 32) == k_) { " + s + " = (int64_t)p_;" + (with_pay ? " pv_ = w0_;" : "") + " break; }");
        L("if ((uint32_t)(w1_ >> 32) == k_) { " + s + " = (int64_t)p_ + 1;" + (with_pay ? " pv_ = w1_;" : "") + " break; }");
        L("if ((f_ == 0u && w0_ == kEmpty) || w1_ == kEmpty) break;");
        L("f_ = 0u;");
        L("p_ = (p_ + 2u == hc_) ? 0u : p_ + 2u;");
        L("n_ += 2u;");
        L("if (n_ >= hc_) break;");
        L("ld_nc_16B(ht_ + (uint64_t)p_, w0_, w1_);");
        --ind;
        L("}");
        --ind;
        L("}");
        if (with_pay) {
          const int d = P.lists[op.list2];
          L("if (" + s + " >= 0) " + V(d) + " = canon(canon((uint64_t)(uint32_t)pv_, " + ct_name(R.pay_ctype[0]) + "), " +
            ct_name(slot(d).ctype) + ");");
        }
        --ind;
        L("}");
        if (op.sub == DQ_JOIN_ANTI) L(act + " = " + act + " && " + s + " < 0;");
        else L(act + " = " + act + " && " + s + " >= 0;");
        return;
      }
      if (ext) {
        L("if (" + tg + " == kEmpty) {");
        L("  if (ht_[(uint64_t)hc_ * " + W + "] == 0ull) " + s + " = (int64_t)hc_;");
        L("} else {");
        ++ind;
      }
      if (R.words <= 2) {
        // aligned 32-byte groups (two slots with a payload word, four tags
        // otherwise; the slot count divides by 4) read in one load.  Slots of
        // the first group before the home slot can only match, not end the
        // walk.  A prefetched probe takes its first group from the load issued
        // with the row's columns.
        const bool pf = is_prefetched(k);
        const int G = 4 / R.words;
        const std::string Gs = num(G);
        const bool with_pay = R.words == 2 && op.sub == DQ_JOIN_INNER && op.nlist2 > 0 && P.lists[op.list2] >= 0;
        L("uint32_t p_ = slot_of(" + tg + ", hc_);");
        L("uint32_t f_ = p_ & " + num(G - 1) + "u;");
        L("p_ -= f_;");
        if (pf) {
          L("uint64_t w0_ = pw" + num(k) + "_0[u], w1_ = pw" + num(k) + "_1[u], w2_ = pw" + num(k) + "_2[u], w3_ = pw" +
            num(k) + "_3[u];");
        } else {
          L("uint64_t w0_, w1_, w2_, w3_;");
          L("ld_nc_32B(ht_ + (uint64_t)p_ * " + W + ", w0_, w1_, w2_, w3_);");
        }
        L("for (uint32_t n_ = 0;;) {");
        ++ind;
        if (R.words == 2) {
          L("if (w0_ == " + tg + ") { " + s + " = (int64_t)p_;" + (with_pay ? " pv_ = w1_;" : "") + " break; }");
          L("if (w2_ == " + tg + ") { " + s + " = (int64_t)p_ + 1;" + (with_pay ? " pv_ = w3_;" : "") + " break; }");
          L("if ((f_ == 0u && w0_ == kEmpty) || w2_ == kEmpty) break;");
        } else {
          L("if (w0_ == " + tg + ") { " + s + " = (int64_t)p_; break; }");
          L("if (w1_ == " + tg + ") { " + s + " = (int64_t)p_ + 1; break; }");
          L("if (w2_ == " + tg + ") { " + s + " = (int64_t)p_ + 2; break; }");
          L("if (w3_ == " + tg + ") { " + s + " = (int64_t)p_ + 3; break; }");
          L("if ((f_ == 0u && w0_ == kEmpty) || (f_ <= 1u && w1_ == kEmpty) || (f_ <= 2u && w2_ == kEmpty) || "
            "w3_ == kEmpty) break;");
        }
        L("f_ = 0u;");
        L("p_ = (p_ + " + Gs + "u == hc_) ? 0u : p_ + " + Gs + "u;");
        L("n_ += " + Gs + "u;");
        L("if (n_ >= hc_) break;");
        L("ld_nc_32B(ht_ + (uint64_t)p_ * " + W + ", w0_, w1_, w2_, w3_);");
        --ind;
        L("}");
        if (with_pay) pay_reg = "pv_";
      } else {
        L("uint32_t i_ = slot_of(" + tg + ", hc_);");
        L("for (uint32_t n_ = 0; n_ < hc_; ++n_) {");
        L("  const uint64_t t_ = ht_[(uint64_t)i_ * " + W + "];");
        L("  if (t_ == " + tg + ") { " + s + " = (int64_t)i_; break; }");
        L("  if (t_ == kEmpty) break;");
        L("  i_ = (i_ + 1u == hc_) ? 0u : i_ + 1u;");
        L("}");
      }
      if (ext) {
        --ind;
        L("}");
      }
    } else {
      std::string k = keys(op, r, op.list, op.nlist);
      if (has_str_key(R))
        L(s + " = unique_find_str(P, " + res(r) + ", key_tag_strh(" + res(r) + ", " + k + ", " + sh + "), " + k + ");");
      else
        L(s + " = unique_find(" + res(r) + ", key_tag(" + res(r) + ", " + k + "), " + k + ");");
    }
    if (!pay_reg.empty()) {
      // the payload came with the tag (the all-ones key's slot is read here)
      int d = P.lists[op.list2];
      L("if (" + s + " >= 0) " + V(d) + " = canon(" + s + " == (int64_t)hc_ ? ht_[(uint64_t)hc_ * 2 + 1] : pv_, " +
        ct_name(slot(d).ctype) + ");");
      pay_reg.clear();
    } else if (op.sub == DQ_JOIN_INNER && op.nlist2 > 0) {
      L("if (" + s + " >= 0) {");
      ++ind;
      L("const uint64_t* pay_ = " + res(r) + ".slots + (uint64_t)" + s + " * " + num(R.words) + " + " +
        num(R.val_word) + ";");
      for (int j = 0; j < op.nlist2; ++j) {
        int d = P.lists[op.list2 + j];
        if (d >= 0) L(V(d) + " = canon(pay_[" + num(j) + "], " + ct_name(slot(d).ctype) + ");");
      }
      --ind;
      L("}");
    }
    --ind;
    L("}");
    if (op.sub == DQ_JOIN_ANTI) L(act + " = " + act + " && " + s + " < 0;");
    else L(act + " = " + act + " && " + s + " >= 0;");
  }

  // live values of parent levels that ops k.. read
  std::vector<int> live_after(int k, int level) {
    std::vector<int> reads;
    for (int j = k; j < P.nops; ++j) op_reads(P, P.ops[j], reads);
    std::vector<int> live;
    for (int s : reads) {
      if (slot(s).level > level || slot(s).kind == DQ_SLOT_STR) continue;
      if (std::find(live.begin(), live.end(), s) == live.end()) live.push_back(s);
    }
    std::sort(live.begin(), live.end());
    return live;
  }

  bool reads_strings_after(int k) {
    std::vector<int> reads;
    for (int j = k; j < P.nops; ++j) op_reads(P, P.ops[j], reads);
    for (int s : reads)
      if (slot(s).kind == DQ_SLOT_STR) return true;
    return false;
  }

  // gathers of level `lv` (the key columns first), key check, rest of the ops
  // Loads a gathered multimap payload value of match `m` for the active lanes.
  void gather(int s, const std::string& act, const std::string& m) {
    const DevSlot& g = slot(s);
    var[s] = "v" + num(s) + "_" + num(uid++);
    L("const uint64_t " + var[s] + " = " + act + " ? canon(ldg_w(" + res(g.res) + ".pay[" + num(g.src) +
      "] + (uint64_t)" + m + " * " + num(g.width) + ", " + num(g.width) + "), " + ct_name(g.ctype) + ") : 0ull;");
  }

  // Gathers the pending payload values the given slots need (lanes that a
  // filter has dropped since the expansion do not load them).
  void materialize(const std::vector<int>& slots, const std::string& act) {
    for (int s : slots) {
      auto it = pending.find(s);
      if (it == pending.end()) continue;
      const std::string m = it->second;
      pending.erase(it);
      gather(s, act, m);
    }
  }

  // Gathers of level `lv`, all issued together (one round trip per chunk of
  // pairs: the hot buckets of a skewed build side are L2-resident, so the
  // latency of dependent loads, not their bytes, bounds the expansion), key
  // check, rest of the ops.  The `pending` mechanism (load at first read)
  // stays available for slots a generator variant wants to defer.
  void pairs(int k, int lv, const std::string& a, const std::string& m, const std::string& exit) {
    gather_level(k, lv, a, m);
    match_ops(k, lv, a, exit);
  }

  // The payload values of level `lv` for match `m` (the key columns first).
  void gather_level(int k, int lv, const std::string& a, const std::string& m) {
    const dq_op& op = P.ops[k];
    for (int q = 0; q < op.nlist2; ++q) {
      int s = P.lists[op.list2 + q];
      if (s >= 0 && slot(s).kind == DQ_SLOT_GATHER && slot(s).level == lv && var[s].empty()) gather(s, a, m);
    }
    for (int s = 0; s < P.nslots; ++s)
      if (slot(s).kind == DQ_SLOT_GATHER && slot(s).level == lv && var[s].empty()) gather(s, a, m);
  }

  // Key check of a pair whose payload is gathered, then the ops after the
  // expansion.
  void match_ops(int k, int lv, const std::string& a, const std::string& exit) {
    const dq_op& op = P.ops[k];
    declare_regs(lv);
    for (int q = 0; q < op.nlist; ++q) {
      const int x = P.lists[op.list + q], y = P.lists[op.list2 + q];
      if (P.res[op.res].key_ctype[q] == DQ_STR)  // long strings compared by the whole warp
        L(a + " = str_ref_eq_warp(P, " + a + ", " + V(x) + ", " + V(y) + ");");
      else
        L(a + " = " + a + " && " + key_eq(op.res, q, x, y) + ";");
    }
    skip_if_idle(a, exit);
    ops_from(k + 1, lv, a, exit);
  }

  // Semi/anti join with a condition (the reference's multimatch semi/anti
  // probe, dogqc/hashJoins.py:244-272): each lane walks its row's key range
  // of the multimap; a build row counts when its keys equal the row's and the
  // condition (ops k+1 .. k+imm, one level down, on the build row's gathered
  // values and the row's own) holds; the first such row ends the walk.
  void exists(int k, int level, const std::string& act) {
    const dq_op& op = P.ops[k];
    const int r = op.res;
    const int lv = level + 1;
    const std::string id = num(uid++);
    const std::string fm = "xf" + id, m = "xm" + id, me = "xe" + id;
    const std::string sh = str_key_hashes(r, op.list, op.nlist, act);
    L("bool " + fm + " = false;");
    L("if (" + act + ") {");
    ++ind;
    std::string kk = keys(op, r, op.list, op.nlist);
    L("const uint32_t b_ = " + bucket(op, r, kk, sh) + ";");
    L("const uint32_t xc_ = " + res(r) + ".counts[b_];");
    L("uint32_t " + m + " = xc_ ? " + res(r) + ".offsets[b_] : 0u;");
    L("const uint32_t " + me + " = " + m + " + xc_;");
    L("for (; " + m + " < " + me + "; ++" + m + ") {");
    ++ind;
    const std::vector<std::string> saved = var;
    for (int s2 = 0; s2 < P.nslots; ++s2)
      if (slot(s2).kind == DQ_SLOT_GATHER && slot(s2).level == lv && slot(s2).res == r) gather(s2, "true", m);
    std::string eq = "true";
    for (int q = 0; q < op.nlist; ++q) eq += " && " + key_eq(r, q, P.lists[op.list + q], P.lists[op.list2 + q]);
    L("if (!(" + eq + ")) continue;");
    if (op.imm > 0) {
      declare_regs(lv);
      for (int j = k + 1; j <= k + (int)op.imm; ++j) scalar_op(P.ops[j]);
      L("if (" + V(op.a) + " == 0ull) continue;");
    }
    L(fm + " = true;");
    L("break;");
    var = saved;  // the build row's values end with the walk
    --ind;
    L("}");
    --ind;
    L("}");
    L(act + " = " + act + " && " + (op.sub == DQ_JOIN_ANTI ? "!" : "") + fm + ";");
  }

  void expand(int k, int level, const std::string& act) {
    const dq_op& op = P.ops[k];
    const int r = op.res;
    const std::string id = num(uid++);
    const std::string eo = "eo" + id, ec = "ec" + id, ei = "ei" + id, et = "et" + id, eb = "eb" + id,
                      q = "eq" + id, sl = "es" + id, m = "em" + id, a = "ea" + id;
    L("{");
    ++ind;
    const std::string sh = str_key_hashes(r, op.list, op.nlist, act);
    L("uint32_t " + eo + " = 0u, " + ec + " = 0u;");
    L("if (" + act + ") {");
    ++ind;
    std::string kk = keys(op, r, op.list, op.nlist);
    L("const uint32_t b_ = " + bucket(op, r, kk, sh) + ";");
    L(ec + " = " + res(r) + ".counts[b_];");
    L(eo + " = " + ec + " ? " + res(r) + ".offsets[b_] : 0u;");
    --ind;
    L("}");
    if (k == expand_op && level == 0) {
      // deferral of long ranges: one atomic per warp reserves the item slots
      L("{");
      ++ind;
      L("const bool dw_ = " + ec + " > P.heavy.threshold;");
      L("const unsigned dm_ = __ballot_sync(kFull, dw_);");
      L("if (dm_) {");
      ++ind;
      L("const int dl_ = __ffs(dm_) - 1;");
      L("uint32_t db_ = 0u;");
      L("if (lane == dl_) db_ = atomicAdd(P.heavy.count, (uint32_t)__popc(dm_));");
      L("db_ = __shfl_sync(kFull, db_, dl_);");
      L("const uint32_t hs_ = db_ + (uint32_t)__popc(dm_ & ((1u << lane) - 1u));");
      L("if (dw_ && hs_ < P.heavy.cap) {");
      ++ind;
      L("uint64_t* it_ = P.heavy.items + (size_t)hs_ * P.heavy.words;");
      if (P.heavy.grouped) {
        // the item joins the group of its range (claimed on first sight); an
        // item whose claim fails is expanded here and carries kEmpty
        L("const uint64_t gk_ = ((uint64_t)" + inst_expr + " << 32) | " + eo + ";");
        L("uint32_t g_ = slot_of(gk_, P.heavy.gcap);");
        L("uint64_t gid_ = kEmpty;");
        L("for (uint32_t n_ = 0; n_ < P.heavy.gcap; ++n_) {");
        L("  const uint64_t t_ = *(volatile uint64_t*)(P.heavy.gkey + g_);");
        L("  if (t_ == gk_) { gid_ = g_; break; }");
        L("  if (t_ == kEmpty) {");
        L("    const uint64_t o_ = atomicCAS((unsigned long long*)(P.heavy.gkey + g_), kEmpty, gk_);");
        L("    if (o_ == kEmpty) {");
        L("      P.heavy.glen[g_] = " + ec + ";");
        L("      P.heavy.glist[atomicAdd(P.heavy.ngroups, 1u)] = g_;");
        L("      gid_ = g_;");
        L("      break;");
        L("    }");
        L("    if (o_ == gk_) { gid_ = g_; break; }");
        L("  }");
        L("  g_ = (g_ + 1u == P.heavy.gcap) ? 0u : g_ + 1u;");
        L("}");
        L("it_[0] = gid_;");
        L("if (gid_ != kEmpty) {");
        ++ind;
        L("atomicAdd(P.heavy.gcnt + gid_, 1u);");
      } else {
        L("it_[0] = " + eo + ";");
        L("it_[1] = " + ec + ";");
      }
      for (int s = 0; s < P.nslots; ++s)
        if (slot(s).stash >= 0) L("it_[" + num(2 + slot(s).stash) + "] = " + V(s) + ";");
      L(ec + " = 0u;");
      if (P.heavy.grouped) {
        --ind;
        L("}");
      }
      --ind;
      L("}");
      --ind;
      L("}");
      --ind;
      L("}");
    }
    L("uint32_t " + ei + " = " + ec + ";");
    L("#pragma unroll");
    L("for (int d_ = 1; d_ < 32; d_ <<= 1) {");
    L("  const uint32_t t_ = __shfl_up_sync(kFull, " + ei + ", d_);");
    L("  if (lane >= d_) " + ei + " += t_;");
    L("}");
    L("const uint32_t " + et + " = __shfl_sync(kFull, " + ei + ", 31);");
    L("for (uint32_t " + eb + " = 0; " + eb + " < " + et + "; " + eb + " += 32u) {");
    ++ind;
    L("const uint32_t " + q + " = " + eb + " + (uint32_t)lane;");
    L("int " + sl + " = 0;");
    L("#pragma unroll");
    L("for (int s_ = 16; s_ > 0; s_ >>= 1)");
    L("  if (__shfl_sync(kFull, " + ei + ", " + sl + " + s_ - 1) <= " + q + ") " + sl + " += s_;");
    L("const uint32_t " + m + " = __shfl_sync(kFull, " + eo + ", " + sl + ") + (" + q + " - (__shfl_sync(kFull, " +
      ei + ", " + sl + ") - __shfl_sync(kFull, " + ec + ", " + sl + ")));");
    L("bool " + a + " = " + q + " < " + et + ";");
    for (int s : live_after(k, level)) {
      std::string nv = "v" + num(s) + "_" + num(uid++);
      L("uint64_t " + nv + " = shfl64(" + V(s) + ", " + sl + ");");
      var[s] = nv;
    }
    if (reads_strings_after(k + 1)) {
      std::string nr = fresh("row");
      L("const int64_t " + nr + " = (int64_t)shfl64((uint64_t)" + row + ", " + sl + ");");
      row = nr;
    }
    pairs(k, level + 1, a, m, "continue;");
    --ind;
    L("}");
    --ind;
    L("}");
  }

  // ---------------------------------------------------------------- sinks --
  static bool has_str_key(const DevRes& R) {
    for (int i = 0; i < R.nkeys; ++i)
      if (R.key_ctype[i] == DQ_STR) return true;
    return false;
  }

  void sink_agg(const dq_op& op, const std::string& act) {
    const int r = op.res;
    const DevRes& R = P.res[r];
    std::vector<std::string> vals;
    for (int j = 0; j < R.naggs; ++j) {
      int src = P.lists[op.list2 + j];
      vals.push_back(R.agg_red[j] == DQ_RED_COUNT || src < 0 ? std::string("1ull") : V(src));
    }
    if (agg == AGG_REGS) {
      L("if (" + act + ") {");
      for (int j = 0; j < R.naggs; ++j)
        L("  acc" + num(j) + " = red_combine(" + red_name(R.agg_red[j]) + ", acc" + num(j) + ", " + vals[j] + ");");
      L("}");
      return;
    }
    const std::string sh = str_key_hashes(r, op.list, op.nlist, act);
    L("if (" + act + ") {");
    ++ind;
    std::string k = keys(op, r, op.list, op.nlist);
    if (R.packed) L("const uint64_t tag_ = " + packed_tag(r, op.list, op.nlist) + ";");
    else if (has_str_key(R)) {
      // key_tag_strh unrolled over the resource's keys
      L("uint64_t th_ = 0x9e3779b97f4a7c15ull;");
      for (int q = 0; q < R.nkeys; ++q)
        L("th_ = fmix64(th_ ^ " + (R.key_ctype[q] == DQ_STR ? sh : k) + "[" + num(q) + "]) + 0x632be59bd9b4e019ull * " +
          num(q + 1) + "ull;");
      L("const uint64_t tag_ = fmix64(th_) & 0x7fffffffffffffffull;");
    } else {
      L("const uint64_t tag_ = key_tag(" + res(r) + ", " + k + ");");
    }
    auto global = [&]() {
      if (R.packed) {
        packed_claim(r, "tag_");
      } else {
        L("const int64_t g_ = agg_slot_global(P, " + res(r) + ", tag_, " + k + ");");
      }
      L("if (g_ >= 0) {");
      ++ind;
      L("uint64_t* a_ = " + res(r) + ".slots + (uint64_t)g_ * " + num(R.words) + " + " + num(R.val_word) + ";");
      for (int j = 0; j < R.naggs; ++j)
        L("accumulate(a_ + " + num(j) + ", " + red_name(R.agg_red[j]) + ", " + vals[j] + ");");
      --ind;
      L("}");
    };
    if (agg == AGG_GLOBAL) {
      global();
    } else {
      if (R.packed) L("const int s_ = local_group_slot(ltags, " + num(ns) + ", tag_, " + num(R.nkeys) + ");");
      else if (has_str_key(R)) local_str_slot(r, k);
      else L("const int s_ = local_group_slot_keys(P, " + res(r) + ", ltags, lkeys, " + num(ns) + ", tag_, " + k + ");");
      L("if (s_ >= 0) {");
      ++ind;
      for (int j = 0; j < R.naggs; ++j) {
        std::string idx = agg == AGG_STRIPED
                              ? "((s_ * " + num(R.naggs) + " + " + num(j) + ") * " + num(copies) + " + (lane & " +
                                    num(copies - 1) + "))"
                              : "(s_ * " + num(R.naggs) + " + " + num(j) + ")";
        L("s_merge(saddr(lacc + " + idx + "), " + red_name(R.agg_red[j]) + ", " + vals[j] + ");");
      }
      --ind;
      L("} else {");
      ++ind;
      global();
      --ind;
      L("}");
    }
    --ind;
    L("}");
  }

  void sink_build(const dq_op& op, const std::string& act) {
    const int r = op.res;
    const DevRes& R = P.res[r];
    if (R.bitmap) {
      // keys outside the domain measured at preparation: the table's data
      // changed; the host re-runs the plan with a hash table
      const std::string key = "canon(" + V(P.lists[op.list]) + ", " + ct_name(R.key_ctype[0]) + ")";
      L("if (" + act + ") {");
      L("  const uint64_t o_ = (uint64_t)" + key + " - (uint64_t)" + res(r) + ".bmin;");
      if (R.bitmap == 2) {
        // one row of a key wins (an 8-byte store is atomic), as one claim
        // wins in the hash table; a store needs no round trip to L2
        const std::string pay = op.nlist2 > 0 ? "(uint64_t)(uint32_t)" + V(P.lists[op.list2]) : "0ull";
        L("  if (o_ < " + res(r) + ".brange) reinterpret_cast<unsigned long long*>(" + res(r) +
          ".slots)[o_] = (1ull << 32) | " + pay + ";");
      } else {
        L("  if (o_ < " + res(r) + ".brange) atomicOr(reinterpret_cast<unsigned int*>(" + res(r) +
          ".slots) + (o_ >> 5), 1u << (o_ & 31u));");
      }
      L("  else set_status(P, kErrKeyRange);");
      L("}");
      return;
    }
    const std::string sh = str_key_hashes(r, op.list, op.nlist, act);
    L("if (" + act + ") {");
    ++ind;
    if (R.compact) {
      const std::string key = "canon(" + V(P.lists[op.list]) + ", " + ct_name(R.key_ctype[0]) + ")";
      const std::string pay = op.nlist2 > 0 ? "(uint32_t)" + V(P.lists[op.list2]) : "0u";
      L("unique_insert_compact(P, " + res(r) + ", (uint32_t)" + key + ", " + pay + ");");
      --ind;
      L("}");
      return;
    }
    std::string k = keys(op, r, op.list, op.nlist);
    if (has_str_key(R))
      L("const int64_t s_ = unique_insert_str(P, " + res(r) + ", key_tag_strh(" + res(r) + ", " + k + ", " + sh + "), " + k +
        ");");
    else
      L("const int64_t s_ = unique_insert(P, " + res(r) + ", key_tag(" + res(r) + ", " + k + "), " + k + ");");
    if (op.nlist2 > 0) {
      L("if (s_ >= 0) {");
      ++ind;
      L("uint64_t* pay_ = " + res(r) + ".slots + (uint64_t)s_ * " + num(R.words) + " + " + num(R.val_word) + ";");
      for (int j = 0; j < op.nlist2; ++j) L("pay_[" + num(j) + "] = " + V(P.lists[op.list2 + j]) + ";");
      --ind;
      L("}");
    }
    --ind;
    L("}");
  }

  void sink_mm(const dq_op& op, const std::string& act) {
    // lanes of a warp that hit the same bucket (the hot keys of a skewed build
    // side) take one atomic per bucket: the lowest such lane adds the group's
    // size, the others their rank within the group
    const int r = op.res;
    const DevRes& R = P.res[r];
    const std::string sh = str_key_hashes(r, op.list, op.nlist, act);
    L("uint32_t b_ = 0xffffffffu;");
    L("if (" + act + ") {");
    ++ind;
    std::string k = keys(op, r, op.list, op.nlist);
    L("b_ = " + bucket(op, r, k, sh) + ";");
    --ind;
    L("}");
    L("const unsigned peers_ = __match_any_sync(kFull, b_);");
    L("if (" + act + ") {");
    ++ind;
    L("const int lead_ = __ffs(peers_) - 1;");
    if (hot == 1) {
      L("if (lane == lead_) {");
      L("  const int hs_ = hot_slot(hk_, b_);");
      L("  if (hs_ >= 0) atomicAdd(&hc_[hs_], (uint32_t)__popc(peers_));");
      L("  else atomicAdd(&" + res(r) + ".counts[b_], (uint32_t)__popc(peers_));");
      L("}");
    } else if (hot == 2) {
      // the bucket's offset does not depend on the claim: load it first
      L("const uint32_t ob_ = " + res(r) + ".offsets[b_];");
      L("int hs_ = -1;");
      L("uint32_t at_ = 0;");
      L("if (lane == lead_) {");
      L("  hs_ = hot_slot(hk_, b_);");
      L("  at_ = atomicAdd(hs_ >= 0 ? &hc_[hs_] : &" + res(r) + ".counts[b_], (uint32_t)__popc(peers_));");
      L("}");
      L("hs_ = __shfl_sync(peers_, hs_, lead_);");
      L("at_ = __shfl_sync(peers_, at_, lead_) + (uint32_t)__popc(peers_ & ((1u << lane) - 1u));");
      L("if (hs_ >= 0) {");
      ++ind;
      L("hs_u[u] = hs_;");
      L("hr_u[u] = ob_ + at_;");
      for (int j = 0; j < op.nlist2; ++j)
        if (hot_value(op, j, "u").empty()) L("hv" + num(j) + "_u[u] = " + V(P.lists[op.list2 + j]) + ";");
      --ind;
      L("} else {");
      ++ind;
      L("const uint32_t pos_ = ob_ + at_;");
      for (int j = 0; j < op.nlist2; ++j) {
        int w = R.pay_width[j];
        L("st(" + res(r) + ".pay[" + num(j) + "] + (size_t)pos_ * " + num(w) + ", " + num(w) + ", " +
          V(P.lists[op.list2 + j]) + ");");
      }
      --ind;
      L("}");
    } else if (op.kind == DQ_OP_MM_COUNT) {
      L("if (lane == lead_) atomicAdd(&" + res(r) + ".counts[b_], (uint32_t)__popc(peers_));");
    } else {
      L("uint32_t at_ = 0;");
      L("if (lane == lead_) at_ = atomicAdd(&" + res(r) + ".counts[b_], (uint32_t)__popc(peers_));");
      L("at_ = __shfl_sync(peers_, at_, lead_);");
      L("const uint32_t pos_ = " + res(r) + ".offsets[b_] + at_ + (uint32_t)__popc(peers_ & ((1u << lane) - 1u));");
      for (int j = 0; j < op.nlist2; ++j) {
        int w = R.pay_width[j];
        L("st(" + res(r) + ".pay[" + num(j) + "] + (size_t)pos_ * " + num(w) + ", " + num(w) + ", " +
          V(P.lists[op.list2 + j]) + ");");
      }
    }
    --ind;
    L("}");
  }

  void sink_emit(const dq_op& op, const std::string& act) {
    const int r = op.res;
    const DevRes& R = P.res[r];
    L("{");
    ++ind;
    L("const unsigned am_ = __ballot_sync(kFull, " + act + ");");
    L("if (am_) {");
    ++ind;
    L("const int ld_ = __ffs(am_) - 1;");
    L("unsigned long long b_ = 0;");
    L("if (lane == ld_) b_ = atomicAdd((unsigned long long*)" + res(r) + ".cursor, (unsigned long long)__popc(am_));");
    L("b_ = __shfl_sync(kFull, b_, ld_);");
    L("if (" + act + ") {");
    ++ind;
    L("const uint64_t pos_ = b_ + __popc(am_ & ((1u << lane) - 1u));");
    L("if (pos_ >= " + res(r) + ".cap) {");
    L("  set_status(P, kErrOverflow);");
    L("} else {");
    ++ind;
    for (int j = 0; j < op.nlist; ++j) {
      int w = R.pay_width[j];
      L("st(" + res(r) + ".pay[" + num(j) + "] + pos_ * " + num(w) + ", " + num(w) + ", " + V(P.lists[op.list + j]) +
        ");");
    }
    --ind;
    L("}");
    --ind;
    L("}");
    --ind;
    L("}");
    --ind;
    L("}");
  }

  // --------------------------------------------------------- aggregation --
  void choose_agg() {
    const dq_op& sink = P.ops[P.nops - 1];
    if (sink.kind != DQ_OP_AGG) return;
    agg_res = sink.res;
    const DevRes& R = P.res[agg_res];
    if (R.nkeys == 0) {
      agg = AGG_REGS;
      return;
    }
    ns = R.smem_slots;
    if (ns <= 0 || (!R.packed && !has_str_key(R)) || batched) {  // a batched kernel's items change instance
      agg = AGG_GLOBAL;
      ns = 0;
      return;
    }
    // replicate the accumulators per lane (32 copies: lanes of a warp never
    // collide), per half-warp (16) or per eighth (8, 4) when the table stays
    // within kStripedMax, else one copy.  A large table costs more than the
    // collisions it avoids: shared memory taken from the SM's L1 leaves fewer
    // lines for the loads in flight (a 33 KB table made the C1 probe kernel
    // twice as slow at five CTAs per SM as an 8.8 KB one), and even without
    // probes 32 copies of C0's table (26 KB) ran 8 % slower than 8 (6.5 KB)
    // hashed keys: their values too, and each string's location
    const int tags = (ns + 1) * 8 + (R.packed ? 0 : ns * (R.nkeys + kStrSlotWords * nstr_keys(R)) * 8);
    agg = AGG_LOCAL;
    copies = 1;
    for (int c : {32, 16, 8, 4})
      if (tags + (ns + 1) * R.naggs * 8 * c <= kStripedMax) {
        agg = AGG_STRIPED;
        copies = c;
        break;
      }
    smem = tags + (ns + 1) * R.naggs * 8 * copies;
  }

  // Lane refill after op `k`: only when later ops do enough per-row work to
  // pay for buffering the live values.
  void choose_refill(int k) {
    refill = -1;
    if (k < 0 || k >= P.nops || P.source_kind == DQ_SRC_AGG) return;
    const dq_op& op = P.ops[k];
    if (op.kind != DQ_OP_FILTER && op.kind != DQ_OP_PROBE) return;
    for (int j = 0; j < k; ++j)
      if (P.ops[j].kind == DQ_OP_EXPAND) return;
    bool heavy = false;
    for (int j = k + 1; j < P.nops; ++j) {
      const int kind = P.ops[j].kind;
      heavy |= kind == DQ_OP_PROBE || kind == DQ_OP_EXPAND || kind == DQ_OP_EXISTS || kind == DQ_OP_LIKE ||
               kind == DQ_OP_STREQ || kind == DQ_OP_SUBSTR ||
               kind == DQ_OP_BUILD || kind == DQ_OP_MM_COUNT || kind == DQ_OP_MM_SCATTER || kind == DQ_OP_EMIT ||
               (kind == DQ_OP_AGG && agg != AGG_REGS);
    }
    if (!heavy) return;
    refill = k;
    nbuf = (int)live_after(k + 1, 0).size() + (reads_strings_after(k + 1) ? 1 : 0);
    if (nbuf == 0) nbuf = 1;
    buf_off = (smem + 15) / 16 * 16;
    smem = buf_off + (block / 32) * kWarpBuf * nbuf * 8;
  }

  // Multimap sinks of a skewed build side meet on a few buckets: a CTA-local
  // table of buckets takes their counts (count pass) or ranks (scatter pass),
  // so a hot bucket sees one global atomic per CTA (count) or per CTA and row
  // step (scatter) instead of one per warp.  The scatter pass reserves ranges
  // at the end of every row step behind block barriers, so it needs straight
  // row steps: no lane refill, no expansion.
  void choose_hot() {
    hot = 0;
    if (batched || P.nops == 0) return;
    const int kind = P.ops[P.nops - 1].kind;
    if (kind != DQ_OP_MM_COUNT && kind != DQ_OP_MM_SCATTER) return;
    for (int j = 0; j < P.nops; ++j)
      if (P.ops[j].kind == DQ_OP_EXPAND) return;
    if (kind == DQ_OP_MM_SCATTER && refill >= 0) return;
    hot = kind == DQ_OP_MM_COUNT ? 1 : 2;
    hot_off = (smem + 15) / 16 * 16;
    smem = hot_off + kHotSlots * 12;
  }

  void hot_init() {
    if (!hot) return;
    L("uint32_t* const hk_ = reinterpret_cast<uint32_t*>(smem + " + num(hot_off) + ");  // hot buckets");
    L("uint32_t* const hc_ = hk_ + " + num(kHotSlots) + ";  // their counts (of this step when scattering)");
    L("uint32_t* const hb_ = hc_ + " + num(kHotSlots) + ";  // their reserved range starts");
    L("(void)hb_;");
    L("for (int i = tid; i < " + num(kHotSlots) + "; i += " + num(block) + ") {");
    L("  hk_[i] = kEmpty32;");
    L("  hc_[i] = 0u;");
    L("}");
    L("__syncthreads();");
  }

  // Scatter pass: per-row state of the table rows of the current step.
  void hot_step_begin() {
    if (hot != 2) return;
    const dq_op& op = P.ops[P.nops - 1];
    L("int hs_u[" + num(U) + "];");
    L("uint32_t hr_u[" + num(U) + "];  // bucket offset + rank in the step");
    for (int j = 0; j < op.nlist2; ++j)
      if (hot_value(op, j, "u").empty()) L("uint64_t hv" + num(j) + "_u[" + num(U) + "];");
    L("#pragma unroll");
    L("for (int u = 0; u < " + num(U) + "; ++u) hs_u[u] = -1;");
  }

  // Payload value j of a deferred table row in the scatter's last phase: a
  // source column value is still in the step's column registers; anything else
  // was kept in hv<j>_u (empty result).
  std::string hot_value(const dq_op& op, int j, const std::string& u) {
    const int s = P.lists[op.list2 + j];
    if (s >= 0 && slot(s).kind == DQ_SLOT_COL)
      return "canon(c" + num(slot(s).src) + "[" + u + "], " + ct_name(slot(s).ctype) + ")";
    return std::string();
  }

  // Scatter pass: one global range per hot bucket of the step, then the
  // table rows' payload at range start + rank.
  void hot_step_end() {
    if (hot != 2) return;
    const dq_op& op = P.ops[P.nops - 1];
    const int r = op.res;
    const DevRes& R = P.res[r];
    L("__syncthreads();");
    L("for (int i = tid; i < " + num(kHotSlots) + "; i += " + num(block) + ") {");
    L("  const uint32_t c_ = hc_[i];");
    L("  if (c_) {");
    L("    hb_[i] = atomicAdd(&" + res(r) + ".counts[hk_[i]], c_);");
    L("    hc_[i] = 0u;");
    L("  }");
    L("}");
    L("__syncthreads();");
    L("#pragma unroll");
    L("for (int u = 0; u < " + num(U) + "; ++u) {");
    ++ind;
    L("if (hs_u[u] >= 0) {");
    ++ind;
    L("const uint32_t pos_ = hb_[hs_u[u]] + hr_u[u];");
    for (int j = 0; j < op.nlist2; ++j) {
      int w = R.pay_width[j];
      std::string v = hot_value(op, j, "u");
      if (v.empty()) v = "hv" + num(j) + "_u[u]";
      L("st(" + res(r) + ".pay[" + num(j) + "] + (size_t)pos_ * " + num(w) + ", " + num(w) + ", " + v + ");");
    }
    --ind;
    L("}");
    --ind;
    L("}");
  }

  // Count pass: the table's counts go to the global ones once per CTA.
  void hot_flush() {
    if (hot != 1) return;
    const int r = P.ops[P.nops - 1].res;
    L("__syncthreads();");
    L("for (int i = tid; i < " + num(kHotSlots) + "; i += " + num(block) + ") {");
    L("  const uint32_t c_ = hc_[i];");
    L("  if (c_) atomicAdd(&" + res(r) + ".counts[hk_[i]], c_);");
    L("}");
  }

  // Appends the active lanes' live values to the warp's buffer, then drains
  // it 32 rows at a time (and the remainder after the warp's last rows)
  // through ops k+1.. with every lane busy.  Called inside the row body's
  // do-while, which it closes and reopens.
  void refill_lanes(int k, const std::string& act) {
    std::vector<int> live = live_after(k + 1, 0);
    const bool need_row = reads_strings_after(k + 1);
    const std::string B = num(kWarpBuf);
    L("{");
    ++ind;
    L("const unsigned bm_ = __ballot_sync(kFull, " + act + ");");
    L("if (" + act + ") {");
    ++ind;
    L("const int p_ = wn + __popc(bm_ & ((1u << lane) - 1u));");
    int j = 0;
    for (int s : live) L("wb[" + num(j++ * kWarpBuf) + " + p_] = " + V(s) + ";");
    if (need_row) L("wb[" + num(j * kWarpBuf) + " + p_] = (uint64_t)" + row + ";");
    --ind;
    L("}");
    L("wn += __popc(bm_);");
    --ind;
    L("}");
    --ind;
    L("} while (0);");
    L("__syncwarp();");
    L("const bool last_ = " + last_step + " && u == " + num(U - 1) + ";");
    L("while (wn >= " + num(refill_threshold) + " || (last_ && wn > 0)) {");
    ++ind;
    L("bool ra = lane < wn;");
    j = 0;
    for (int s : live) {
      std::string nv = "b" + num(s) + "_" + num(uid++);
      L("uint64_t " + nv + " = wb[" + num(j++ * kWarpBuf) + " + lane];");
      var[s] = nv;
    }
    if (need_row) {
      row = fresh("brow");
      L("const int64_t " + row + " = (int64_t)wb[" + num(j * kWarpBuf) + " + lane];");
    }
    L("__syncwarp();");
    L("if (lane + 32 < wn) {");
    for (int q = 0; q < nbuf; ++q)
      L("  wb[" + num(q * kWarpBuf) + " + lane] = wb[" + num(q * kWarpBuf) + " + lane + 32];");
    L("}");
    L("__syncwarp();");
    L("wn = wn > 32 ? wn - 32 : 0;");
    L("do {");
    ++ind;
    ops_from(k + 1, 0, "ra", "break;");
    --ind;
    L("} while (0);");
    --ind;
    L("}");
    L("do {");
    ++ind;
    (void)B;
  }

  uint64_t min_mask() const {
    const DevRes& R = P.res[agg_res];
    uint64_t mask = 0;
    for (int j = 0; j < R.naggs; ++j)
      if (R.agg_red[j] == DQ_RED_MIN) mask |= 1ull << j;
    return mask;
  }

  void agg_init() {
    if (agg == AGG_NONE || agg == AGG_GLOBAL) return;
    const DevRes& R = P.res[agg_res];
    if (agg == AGG_REGS) {
      for (int j = 0; j < R.naggs; ++j)
        L("uint64_t acc" + num(j) + " = red_init(" + red_name(R.agg_red[j]) + ");");
      return;
    }
    L("uint64_t* ltags = reinterpret_cast<uint64_t*>(smem);");
    if (R.packed) {
      L("uint64_t* lacc = ltags + " + num(ns + 1) + ";");
    } else {
      L("uint64_t* lkeys = ltags + " + num(ns + 1) + ";");
      if (has_str_key(R)) {
        L("uint64_t* lstr = lkeys + " + num(ns * R.nkeys) + ";");
        L("uint64_t* lacc = lstr + " + num(ns * kStrSlotWords * nstr_keys(R)) + ";");
      } else {
        L("uint64_t* lacc = lkeys + " + num(ns * R.nkeys) + ";");
      }
    }
    L("for (int i = tid; i <= " + num(ns) + "; i += " + num(block) + ") ltags[i] = kEmpty;");
    L("for (int i = tid; i < " + num((ns + 1) * R.naggs * copies) + "; i += " + num(block) + ")");
    L("  lacc[i] = ((" + lit(min_mask()) + " >> ((i / " + num(copies) + ") % " + num(R.naggs) +
      ")) & 1ull) ? ~0ull : 0ull;");
    L("__syncthreads();");
  }

  void agg_flush() {
    if (agg == AGG_NONE || agg == AGG_GLOBAL) return;
    const DevRes& R = P.res[agg_res];
    const std::string rr = res(agg_res);
    if (agg == AGG_REGS) {
      for (int j = 0; j < R.naggs; ++j) {
        L("{");
        L("  const uint64_t w_ = warp_reduce_all(" + std::string(red_name(R.agg_red[j])) + ", acc" + num(j) + ");");
        L("  if (lane == 0) accumulate(" + rr + ".slots + " + num(R.val_word + j) + ", " + red_name(R.agg_red[j]) +
          ", w_);");
        L("}");
      }
      return;
    }
    uint64_t packed_reds = 0;
    for (int j = 0; j < R.naggs; ++j) packed_reds |= (uint64_t)(R.agg_red[j] & 15) << (4 * j);
    L("__syncthreads();");
    L("for (int i = tid; i < " + num((ns + 1) * R.naggs) + "; i += " + num(block) + ") {");
    ++ind;
    L("const int s_ = i / " + num(R.naggs) + ", j_ = i % " + num(R.naggs) + ";");
    L("uint64_t tg_ = ltags[s_];");
    L("if (tg_ == kEmpty) continue;");
    L("if (s_ == " + num(ns) + ") tg_ = kEmpty;  // the all-ones key");
    L("const int red_ = (int)((" + lit(packed_reds) + " >> (4 * j_)) & 15ull);");
    L("uint64_t v_ = lacc[i * " + num(copies) + "];");
    if (copies > 1) L("for (int c_ = 1; c_ < " + num(copies) + "; ++c_) v_ = red_combine(red_, v_, lacc[i * " +
                      num(copies) + " + c_]);");
    if (R.packed) packed_claim(agg_res, "tg_");
    else L("const int64_t g_ = agg_slot_global(P, " + rr + ", tg_, lkeys + s_ * " + num(R.nkeys) + ");");
    L("if (g_ >= 0) accumulate(" + rr + ".slots + (uint64_t)g_ * " + num(R.words) + " + " + num(R.val_word) +
      " + j_, red_, v_);");
    --ind;
    L("}");
  }

  void prologue(const char* name) {
    L(std::string("extern \"C\" __global__ void __launch_bounds__(") + num(block) +
      (min_blocks > 0 ? ", " + num(min_blocks) : std::string()) + ") " + name + "(const __grid_constant__ DevPipe P) {");
    ++ind;
    L("extern __shared__ __align__(16) uint8_t smem[];");
    L("if (*(volatile int32_t*)P.status & (kErrHtFull | kErrTimeout)) return;");
    L("const int tid = threadIdx.x, lane = tid & 31;");
    L("(void)smem;");
    L("(void)lane;");
    agg_init();
    bitmap_init();
  }

  // The key-domain bitmaps of at most 32 KB this kernel probes, one word per
  // thread into shared memory (a probe is then a bank access, not an L2
  // access); larger ones are probed in place.
  void choose_bitmaps() {
    bitmaps.clear();
    if (batched) return;  // a batched kernel's items change instance: its probes read the bits in place
    for (int k = 0; k < P.nops; ++k) {
      const dq_op& op = P.ops[k];
      if (op.kind != DQ_OP_PROBE || P.res[op.res].bitmap != 1 || P.res[op.res].cap > 8192) continue;
      bool seen = false;
      for (auto& b : bitmaps) seen |= b.first == op.res;
      if (seen) continue;
      const int off = (smem + 15) / 16 * 16;
      bitmaps.emplace_back(op.res, off);
      smem = off + (int)P.res[op.res].cap * 4;
    }
  }

  void bitmap_init() {
    for (auto& b : bitmaps) {
      L("{");
      L("  const uint32_t* g_ = reinterpret_cast<const uint32_t*>(" + res(b.first) + ".slots);");
      L("  uint32_t* s_ = reinterpret_cast<uint32_t*>(smem + " + num(b.second) + ");");
      L("  for (uint32_t i = tid; i < (uint32_t)" + res(b.first) + ".cap; i += " + num(block) + "u) s_[i] = __ldcg(g_ + i);");
      L("}");
    }
    if (!bitmaps.empty()) L("__syncthreads();");
  }

  // Bits of resource r as the probe reads them: shared memory or in place.
  std::string bitmap_words(int r) const {
    for (auto& b : bitmaps)
      if (b.first == r) return "reinterpret_cast<const uint32_t*>(smem + " + num(b.second) + ")";
    return "reinterpret_cast<const uint32_t*>(" + res(r) + ".slots)";
  }

  // A word of the aggregation table the pipeline scans.  The fused tail reads
  // it past L1 (__ldcg): the other CTAs' atomics wrote it at L2.
  std::string src_ld(const std::string& ptr) const {
    return single_cta ? "__ldcg(reinterpret_cast<const unsigned long long*>(" + ptr + "))" : "*(" + ptr + ")";
  }

  void epilogue() {
    agg_flush();
    if (tail_call) {
      // every CTA's aggregates are merged (its atomics fenced) before it
      // counts itself done; the last one scans the table into the result
      L("{");
      L("  __shared__ int dq_last_;");
      L("  __threadfence();");
      L("  __syncthreads();");
      L("  if (tid == 0) dq_last_ = atomicAdd(P.tile_counter + 1, 1u) == gridDim.x - 1u;");
      L("  __syncthreads();");
      L("  if (dq_last_) {");
      L("    __threadfence();");
      L("    dq_tail(*P.tail);");
      L("  }");
      L("}");
    }
    --ind;
    L("}");
  }

  // The next pipeline as a device function one CTA runs over its whole source
  // (the fused tail): the row loop of dq_main without the grid stride.
  void tail_function() {
    L("__device__ __noinline__ void dq_tail(const DevPipe& P) {");
    ++ind;
    L("if (*(volatile int32_t*)P.status & (kErrHtFull | kErrTimeout)) return;");
    L("const int tid = threadIdx.x, lane = tid & 31;");
    L("(void)lane;");
    L("const int64_t nrows = source_rows(P);");
    L("const int64_t span = (int64_t)blockDim.x * " + num(U) + ";");
    L("for (int64_t base = 0; base < nrows; base += span) {");
    ++ind;
    row_loop();
    --ind;
    L("}");
    --ind;
    L("}");
    L("");
  }

  // <dst><col>[0..U) for the thread's U consecutive rows of the step starting
  // at `base_expr`: whole rows of every column in vector loads when the step
  // is complete (columns are 256-byte aligned), else per row.  Source columns
  // are streamed once: evict-first loads keep the join tables resident in L2.
  void col_loads(const std::vector<int>& cols, const std::string& dst, const std::string& base_expr) {
    L("{");
    ++ind;
    L("const int64_t r0_ = " + base_expr + " + (int64_t)tid * " + num(U) + ";");
    L("if (r0_ + " + num(U) + " <= nrows) {");
    ++ind;
    for (int c : cols) vector_load(c, dst);
    --ind;
    L("} else {");
    ++ind;
    L("#pragma unroll");
    L("for (int u = 0; u < " + num(U) + "; ++u) {");
    L("  const bool in_ = r0_ + u < nrows;");
    for (int c : cols) {
      int w = P.cols[c].width;
      L("  " + dst + num(c) + "[u] = in_ ? (uint64_t)" + ldfn + "(reinterpret_cast<const " + uint_type(w) + "*>(P.cols[" +
        num(c) + "].ptr) + r0_ + u) : 0ull;");
    }
    L("}");
    --ind;
    L("}");
    --ind;
    L("}");
  }

  // <dst><col>[0..U) from U consecutive rows starting at r0_ (in bounds): loads
  // of up to 16 bytes, split into the column's values.
  void vector_load(int c, const std::string& dst) {
    const int w = P.cols[c].width;
    const int total = U * w;
    const int chunk = std::min(16, total);
    const int n = total / chunk;
    const char* T = chunk == 16 ? "uint4" : chunk == 8 ? "uint2" : uint_type(chunk);
    const std::string base_ptr = "reinterpret_cast<const " + std::string(T) + "*>(P.cols[" + num(c) + "].ptr + r0_ * " +
                                 num(w) + ")";
    std::vector<std::string> words;  // 32-bit words of the loaded bytes (or narrower chunks)
    for (int q = 0; q < n; ++q) {
      std::string x = "x" + num(c) + "_" + num(q);
      L("const " + std::string(T) + " " + x + " = " + ldfn + "(" + base_ptr + " + " + num(q) + ");");
      if (chunk == 16) {
        for (const char* f : {".x", ".y", ".z", ".w"}) words.push_back(x + f);
      } else if (chunk == 8) {
        words.push_back(x + ".x");
        words.push_back(x + ".y");
      } else {
        words.push_back("(uint32_t)" + x);
      }
    }
    for (int u = 0; u < U; ++u) {
      std::string v;
      const int byte = u * w;
      if (w == 8) v = "((uint64_t)" + words[byte / 4] + " | ((uint64_t)" + words[byte / 4 + 1] + " << 32))";
      else if (w == 4) v = "(uint64_t)" + words[byte / 4];
      else if (chunk < 4) v = "(uint64_t)((" + words[0] + " >> " + num(8 * byte) + ") & " + (w == 2 ? "0xffffu" : "0xffu") + ")";
      else v = "(uint64_t)((" + words[byte / 4] + " >> " + num(8 * (byte % 4)) + ") & " + (w == 2 ? "0xffffu" : "0xffu") + ")";
      L(dst + num(c) + "[" + num(u) + "] = " + v + ";");
    }
  }

  // ----------------------------------------------------------- kernels --
  void main_kernel() {
    prologue("dq_main");
    hot_init();
    std::vector<int> cols = source_cols();
    L("const int64_t nrows = source_rows(P);");
    L("const int64_t span = " + num((long long)block * U) + ";");
    if (refill >= 0) {
      L("uint64_t* const wb = reinterpret_cast<uint64_t*>(smem + " + num(buf_off) + ") + (tid >> 5) * " +
        num(kWarpBuf * nbuf) + ";  // this warp's refill buffer");
      L("int wn = 0;  // rows in it");
    }
    for (int c : cols) L("uint64_t c" + num(c) + "[" + num(U) + "];");
    if (!cols.empty()) col_loads(cols, "c", "(int64_t)blockIdx.x * span");
    L("for (int64_t base = (int64_t)blockIdx.x * span; base < nrows; base += (int64_t)gridDim.x * span) {");
    ++ind;
    for (int k : prefetch) {
      const DevRes& Rk = P.res[P.ops[k].res];
      const int nq = Rk.bitmap == 2 ? 1 : Rk.compact ? 2 : 4;
      for (int q = 0; q < nq; ++q) L("uint64_t pw" + num(k) + "_" + num(q) + "[" + num(U) + "];");
    }
    if (!cols.empty()) {
      // the columns of the next step are loaded before this step's rows are
      // processed, so their DRAM latency overlaps the probes of this step
      for (int c : cols) L("uint64_t n" + num(c) + "[" + num(U) + "];");
      col_loads(cols, "n", "base + (int64_t)gridDim.x * span");
      if (!prefetch.empty()) {
        L("#pragma unroll");
        L("for (int u = 0; u < " + num(U) + "; ++u) {");
        ++ind;
        L("const bool in_ = base + (int64_t)tid * " + num(U) + " + u < nrows;");
        prefetch_loads();
        --ind;
        L("}");
      }
    }
    hot_step_begin();
    row_loop();
    hot_step_end();
    if (!cols.empty()) {
      L("#pragma unroll");
      L("for (int u = 0; u < " + num(U) + "; ++u) {");
      for (int c : cols) L("  c" + num(c) + "[u] = n" + num(c) + "[u];");
      L("}");
    }
    --ind;
    L("}");
    hot_flush();
    epilogue();
  }

  std::vector<int> source_cols() const {
    std::vector<int> cols;  // staged columns read by COL slots
    for (int s = 0; s < P.nslots; ++s)
      if (slot(s).kind == DQ_SLOT_COL && std::find(cols.begin(), cols.end(), slot(s).src) == cols.end())
        cols.push_back(slot(s).src);
    return cols;
  }

  // The U rows of the thread in the current step: slot values, then the ops.
  // Expects base, nrows, c<col>[u] (and the prefetched probe groups) in scope.
  void row_loop() {
    const bool agg_src = P.source_kind == DQ_SRC_AGG;
    L("#pragma unroll");
    L("for (int u = 0; u < " + num(U) + "; ++u) {");
    ++ind;
    L("const int64_t row = base + (int64_t)tid * " + num(U) + " + u;");
    L("bool act = row < nrows;");
    row = "row";
    if (agg_src) {
      const int sr = P.source_res;
      const DevRes& R = P.res[sr];
      if (R.nkeys > 0)
        L("if (act) act = " + src_ld(res(sr) + ".slots + (uint64_t)row * " + num(R.words)) + " != kEmpty;");
    }
    for (int s = 0; s < P.nslots; ++s) {
      const DevSlot& sl = slot(s);
      if (sl.kind == DQ_SLOT_COL) {
        var[s] = "v" + num(s);
        L("const uint64_t " + var[s] + " = canon(c" + num(sl.src) + "[u], " + ct_name(sl.ctype) + ");");
      } else if (sl.kind == DQ_SLOT_AGGKEY || sl.kind == DQ_SLOT_AGGVAL) {
        const DevRes& R = P.res[sl.res];
        var[s] = "v" + num(s);
        L("uint64_t " + var[s] + " = 0;");
        L("if (row < nrows) {");
        ++ind;
        L("const uint64_t* as_ = " + res(sl.res) + ".slots + (uint64_t)row * " + num(R.words) + ";");
        if (sl.kind == DQ_SLOT_AGGVAL) {
          L(var[s] + " = canon(" + src_ld("as_ + " + num(R.val_word + sl.src)) + ", " + ct_name(sl.ctype) + ");");
        } else if (R.packed) {
          L("const uint64_t t_ = (uint64_t)row == " + res(sl.res) + ".cap ? kEmpty : " + src_ld("as_") + ";");
          bool wide = R.nkeys == 1 && (R.key_ctype[0] == DQ_I64 || R.key_ctype[0] == DQ_U64);
          L(var[s] + " = canon(" + (wide ? std::string("t_") : "(t_ >> " + num(32 * sl.src) + ") & 0xffffffffull") +
            ", " + ct_name(sl.ctype) + ");");
        } else {
          L(var[s] + " = canon(" + src_ld("as_ + " + num(R.key_word + sl.src)) + ", " + ct_name(sl.ctype) + ");");
        }
        --ind;
        L("}");
      }
    }
    if (agg_src) {
      // the table's only scan puts back each slot it read (tag and keys empty,
      // accumulators at their initial values) when the runtime asks for it
      const int sr = P.source_res;
      const DevRes& R = P.res[sr];
      L("if (P.clear_src && " + std::string(R.nkeys > 0 ? "act" : "row < nrows") + ") {");
      ++ind;
      L("uint64_t* const cs_ = " + res(sr) + ".slots + (uint64_t)row * " + num(R.words) + ";");
      for (int w = 0; w < R.words; ++w) {
        const bool acc = w >= R.val_word && w < R.val_word + R.naggs;
        L("cs_[" + num(w) + "] = " + (acc ? std::string("red_init(") + red_name(R.agg_red[w - R.val_word]) + ")" : "kEmpty") +
          ";");
      }
      --ind;
      L("}");
    }
    declare_regs(0);
    L("do {");
    ++ind;
    ops_from(0, 0, "act", "break;");
    --ind;
    L("} while (0);");
    --ind;
    L("}");
  }

  // Many instances of the plan (same shape, own tables) in one launch: the
  // work items are the row blocks of all instances (prefix bprefix over the
  // instances); a CTA takes items grid-stride, binds the item's instance
  // descriptor, drains its lane-refill buffer and flushes its aggregates at the
  // end of every item.
  void batch_kernel() {
    L(std::string("extern \"C\" __global__ void __launch_bounds__(") + num(block) +
      (min_blocks > 0 ? ", " + num(min_blocks) : std::string()) +
      ") dq_batch_main(const DevPipe* __restrict__ Ps, const int64_t* __restrict__ bprefix, int ninst) {");
    ++ind;
    L("extern __shared__ __align__(16) uint8_t smem[];");
    L("if (*(volatile int32_t*)Ps[0].status & (kErrHtFull | kErrTimeout)) return;");
    L("const int tid = threadIdx.x, lane = tid & 31;");
    L("(void)smem;");
    L("(void)lane;");
    L("const int64_t span = " + num((long long)block * U) + ";");
    if (refill >= 0) {
      L("uint64_t* const wb = reinterpret_cast<uint64_t*>(smem + " + num(buf_off) + ") + (tid >> 5) * " +
        num(kWarpBuf * nbuf) + ";  // this warp's refill buffer");
      L("int wn = 0;  // rows in it");
    }
    L("const int64_t total = bprefix[ninst];");
    L("for (int64_t blk = blockIdx.x; blk < total; blk += gridDim.x) {");
    ++ind;
    L("int lo = 0, hi = ninst;");
    L("while (hi - lo > 1) {");
    L("  const int mid = (lo + hi) >> 1;");
    L("  if (bprefix[mid] <= blk) lo = mid; else hi = mid;");
    L("}");
    L("const DevPipe& P = Ps[lo];");
    L("const int64_t nrows = source_rows(P);");
    L("const int64_t base = (blk - bprefix[lo]) * span;");
    inst_expr = "(uint32_t)lo";
    agg_init();
    std::vector<int> cols = source_cols();
    for (int c : cols) L("uint64_t c" + num(c) + "[" + num(U) + "];");
    for (int k : prefetch)
      for (int q = 0; q < (P.res[P.ops[k].res].bitmap == 2 ? 1 : P.res[P.ops[k].res].compact ? 2 : 4); ++q)
        L("uint64_t pw" + num(k) + "_" + num(q) + "[" + num(U) + "];");
    if (!cols.empty()) {
      col_loads(cols, "c", "base");
      if (!prefetch.empty()) {
        L("#pragma unroll");
        L("for (int u = 0; u < " + num(U) + "; ++u) {");
        ++ind;
        L("const bool in_ = base + (int64_t)tid * " + num(U) + " + u < nrows;");
        prefetch_loads();
        --ind;
        L("}");
      }
    }
    last_step = "true";
    row_loop();
    agg_flush();
    --ind;
    L("}");
    --ind;
    L("}");
  }

  // Deferred items grouped by range: a warp's work unit is 32 rows of one
  // group's range and up to kGroupItems of its items.  The rows' payload is
  // gathered once; the items' carried values come 32 at a time in one load and
  // are broadcast by shuffle, and every (item, row) pair runs the key check
  // and the ops after the expansion.
  void heavy_grouped_kernel() {
    std::fill(var.begin(), var.end(), std::string());
    pending.clear();
    if (batched) {
      // the instances share the deferral buffers; a unit binds its instance
      L(std::string("extern \"C\" __global__ void __launch_bounds__(") + num(block) +
        ") dq_batch_heavy(const DevPipe* __restrict__ Ps, int ninst) {");
      ++ind;
      L("extern __shared__ __align__(16) uint8_t smem[];");
      L("if (*(volatile int32_t*)Ps[0].status & (kErrHtFull | kErrTimeout)) return;");
      L("const int tid = threadIdx.x, lane = tid & 31;");
      L("(void)smem;");
      L("(void)tid;");
      L("(void)ninst;");
      L("const DevHeavy& H = Ps[0].heavy;");
      L("uint32_t* const units_taken = Ps[0].tile_counter;");
    } else {
      prologue("dq_heavy");
      L("const DevHeavy& H = P.heavy;");
      L("uint32_t* const units_taken = P.tile_counter;");
    }
    L("const uint32_t ng = *H.ngroups < H.gcap ? *H.ngroups : H.gcap;");
    L("const uint64_t units = H.unit_prefix[ng];");
    L("const int ns = H.nstash;");
    L("(void)ns;");
    // the warp's current group and its unit range stay in registers: the
    // units of a long range come to the same warp in runs
    L("uint32_t lo = 0;");
    L("uint64_t ulo = 1, uhi = 0;");
    L("for (;;) {");
    ++ind;
    L("uint32_t unit = 0;");
    L("if (lane == 0) unit = atomicAdd(units_taken, 1u);");
    L("unit = __shfl_sync(kFull, unit, 0);");
    L("if ((uint64_t)unit >= units) break;");
    L("if ((uint64_t)unit < ulo || (uint64_t)unit >= uhi) {");
    ++ind;
    // 32-ary search of the unit prefix: every round the lanes read 32 evenly
    // spaced entries of [a, b) and keep the segment that holds the unit
    L("uint32_t a = 0, b = ng;");
    L("while (b - a > 1u) {");
    L("  const uint32_t st_ = (b - a + 31u) / 32u;");
    L("  const uint32_t ix_ = a + (uint32_t)lane * st_;");
    L("  const bool le_ = ix_ < b && H.unit_prefix[ix_] <= (uint64_t)unit;");
    L("  const unsigned m_ = __ballot_sync(kFull, le_);");
    L("  a = a + (uint32_t)(31 - __clz(m_)) * st_;");
    L("  b = b < a + st_ ? b : a + st_;");
    L("}");
    L("lo = a;");
    L("ulo = H.unit_prefix[lo];");
    L("uhi = H.unit_prefix[lo + 1];");
    --ind;
    L("}");
    L("const uint32_t gs = H.glist[lo];");
    L("const uint64_t gk = H.gkey[gs];");
    L("const uint32_t len = H.glen[gs];");
    L("const uint32_t i0 = H.gstart[lo], ni = H.gstart[lo + 1] - i0;");
    if (batched) {
      // aggregates go to the unit's own instance: accumulated per unit
      L("const DevPipe& P = Ps[(uint32_t)(gk >> 32)];");
      agg_init();
    }
    L("const uint32_t local = (uint32_t)((uint64_t)unit - ulo);");
    L("const uint32_t rch = (len + " + num(kGroupRows - 1) + "u) / " + num(kGroupRows) + "u;");
    L("const uint32_t q = (local % rch) * " + num(kGroupRows) + "u + (uint32_t)lane;");
    L("const bool a0 = q < len;");
    L("const uint32_t m = (uint32_t)gk + q;");
    L("const uint32_t ib = (local / rch) * " + num(kGroupItems) + "u;");
    L("const uint32_t ie = ni < ib + " + num(kGroupItems) + "u ? ni : ib + " + num(kGroupItems) + "u;");
    row = "";
    gather_level(expand_op, 1, "a0", "m");
    L("for (uint32_t ix = ib; ix < ie; ix += 32u) {");
    ++ind;
    std::vector<std::pair<int, std::string>> carried;
    for (int s = 0; s < P.nslots; ++s)
      if (slot(s).stash >= 0) {
        const std::string hl = "hl" + num(s);
        L("const uint64_t " + hl + " = ix + lane < ie ? H.sorted[(size_t)(i0 + ix + lane) * ns + " +
          num(slot(s).stash) + "] : 0ull;");
        carried.emplace_back(s, hl);
      }
    L("const int nt = (int)(ie - ix < 32u ? ie - ix : 32u);");
    L("for (int t = 0; t < nt; ++t) {");
    ++ind;
    for (auto& c : carried) {
      var[c.first] = "h" + num(c.first);
      L("const uint64_t " + var[c.first] + " = shfl64(" + c.second + ", t);");
    }
    L("bool a = a0;");
    match_ops(expand_op, 1, "a", "continue;");
    --ind;
    L("}");
    --ind;
    L("}");
    if (batched) agg_flush();
    --ind;
    L("}");
    if (batched) {
      --ind;
      L("}");
    } else {
      epilogue();
    }
  }

  void heavy_kernel() {
    if (P.heavy.grouped) {
      heavy_grouped_kernel();
      return;
    }
    std::fill(var.begin(), var.end(), std::string());
    pending.clear();
    prologue("dq_heavy");
    L("__shared__ uint32_t s_unit;");
    L("const uint32_t nitems = *P.heavy.count < P.heavy.cap ? *P.heavy.count : P.heavy.cap;");
    L("const uint64_t units = P.heavy.unit_prefix[nitems];");
    L("for (;;) {");
    ++ind;
    L("if (tid == 0) s_unit = atomicAdd(P.tile_counter, 1u);");
    L("__syncthreads();");
    L("const uint64_t unit = s_unit;");
    L("__syncthreads();");
    L("if (unit >= units) break;");
    L("int lo = 0, hi = (int)nitems;");
    L("while (lo < hi) {");
    L("  const int mid = (lo + hi) >> 1;");
    L("  if (P.heavy.unit_prefix[mid + 1] <= unit) lo = mid + 1; else hi = mid;");
    L("}");
    L("const uint64_t* it = P.heavy.items + (size_t)lo * P.heavy.words;");
    L("const uint64_t chunk = unit - P.heavy.unit_prefix[lo];");
    L("const uint64_t off = it[0] + chunk * (uint64_t)P.exp_cap;");
    L("const uint64_t rem = it[1] - chunk * (uint64_t)P.exp_cap;");
    L("const uint32_t len = (uint32_t)(rem < (uint64_t)P.exp_cap ? rem : (uint64_t)P.exp_cap);");
    for (int s = 0; s < P.nslots; ++s)
      if (slot(s).stash >= 0) {
        var[s] = "h" + num(s);
        L("const uint64_t " + var[s] + " = it[" + num(2 + slot(s).stash) + "];");
      }
    L("for (uint32_t pb = 0; pb < len; pb += " + num(block) + "u) {");
    ++ind;
    L("const uint32_t q = pb + (uint32_t)tid;");
    L("bool a = q < len;");
    L("const uint32_t m = (uint32_t)off + q;");
    row = "";
    pairs(expand_op, 1, "a", "m", "continue;");
    --ind;
    L("}");
    --ind;
    L("}");
    epilogue();
  }
};

}  // namespace

Program generate(const DevPipe& P, int expand_op, int refill_op, const Tuning& t, const DevPipe* tail,
                 const std::string* patterns) {
  Gen g(P, expand_op);
  g.patterns = patterns;
  g.batched = t.batched;
  if (t.block == 128 || t.block == 256 || t.block == 512) g.block = t.block;
  if (t.min_blocks > 0 && t.min_blocks * g.block <= 2048) g.min_blocks = t.min_blocks;
  bool has_expand = false;
  for (int i = 0; i < P.nops; ++i) has_expand |= P.ops[i].kind == DQ_OP_EXPAND;
  g.U = (has_expand || P.source_kind == DQ_SRC_AGG) ? 1 : 4;
  // tuning knobs: rows per thread and step (1, 2 or 4), minimum resident CTAs per SM
  const int rows = t.rows_per_thread;
  if (rows > 0 && !has_expand && P.source_kind != DQ_SRC_AGG) g.U = rows >= 4 ? 4 : rows >= 2 ? 2 : 1;
  if (t.refill < 0) refill_op = -1;
  if (t.refill_threshold >= 1 && t.refill_threshold <= 32) g.refill_threshold = t.refill_threshold;
  g.choose_agg();
  g.choose_refill(refill_op);
  g.choose_hot();
  g.choose_prefetch();
  g.choose_bitmaps();
  if (g.U == 4 && rows <= 0) {
    // four rows per thread keep enough loads in flight for narrow pipelines;
    // wide ones (many columns or several early probes) run out of registers
    std::vector<int> cols;
    for (int s = 0; s < P.nslots; ++s)
      if (P.slots[s].kind == DQ_SLOT_COL && std::find(cols.begin(), cols.end(), P.slots[s].src) == cols.end())
        cols.push_back(P.slots[s].src);
    if (cols.size() > 3 || g.prefetch.size() > 1) g.U = 2;
  }
  g.o = "// generated pipeline kernel (dogqc_b200)\n#include \"dq_common.cuh\"\nusing namespace dq;\n\n";
  if (tail && !t.batched && expand_op < 0) {
    Gen tg(*tail, -1);
    tg.single_cta = true;
    tg.U = 1;
    tg.choose_agg();
    tg.choose_refill(-1);
    if (tg.agg != AGG_NONE || tg.smem > 0) throw Error("a fused tail takes no shared memory");
    tg.tail_function();
    g.o += tg.o;
    g.tail_call = true;
  }
  Program prog;
  prog.block = g.block;
  if (t.batched) {
    g.batch_kernel();
    if (expand_op >= 0) {
      g.o += "\n";
      g.heavy_kernel();
      prog.heavy = true;
    }
    prog.source = g.o;
    prog.smem_bytes = g.smem;
    prog.rows_per_thread = g.U;
    prog.batched = true;
    return prog;
  }
  g.main_kernel();
  if (expand_op >= 0) {
    g.o += "\n";
    g.heavy_kernel();
    prog.heavy = true;
  }
  prog.source = g.o;
  prog.smem_bytes = g.smem;
  prog.rows_per_thread = g.U;
  return prog;
}

// ------------------------------------------------------------- compiler --

namespace {

struct Entry {
  std::vector<char> cubin;
  std::string log;
  cudaLibrary_t lib = nullptr;
  cudaKernel_t main = nullptr, heavy = nullptr;
};

std::mutex g_mu;
std::map<std::string, std::unique_ptr<Entry>> g_cache;

const char* kStdint =
    "#pragma once\n"
    "typedef signed char int8_t; typedef short int16_t; typedef int int32_t; typedef long long int64_t;\n"
    "typedef unsigned char uint8_t; typedef unsigned short uint16_t; typedef unsigned int uint32_t;\n"
    "typedef unsigned long long uint64_t;\n";
const char* kStddef = "#pragma once\ntypedef unsigned long size_t; typedef long ptrdiff_t;\n";

// The NVRTC that compiles generated kernels.  An application may have loaded
// an older NVRTC into the process before this library (PyTorch loads its own);
// the CUDA toolkit's library, when newer, is opened privately beside it (local
// symbols, its own bindings first), since 256-bit loads for sm_100a need 12.9.
struct NvrtcApi {
  nvrtcResult (*version)(int*, int*);
  nvrtcResult (*create)(nvrtcProgram*, const char*, const char*, int, const char* const*, const char* const*);
  nvrtcResult (*compile)(nvrtcProgram, int, const char* const*);
  nvrtcResult (*log_size)(nvrtcProgram, size_t*);
  nvrtcResult (*log)(nvrtcProgram, char*);
  nvrtcResult (*cubin_size)(nvrtcProgram, size_t*);
  nvrtcResult (*cubin)(nvrtcProgram, char*);
  nvrtcResult (*destroy)(nvrtcProgram*);
  const char* (*error)(nvrtcResult);
};

bool open_nvrtc(const std::string& path, NvrtcApi& a) {
  void* h = dlopen(path.c_str(), RTLD_NOW | RTLD_LOCAL | RTLD_DEEPBIND);
  if (!h) return false;
  auto sym = [&](const char* n) { return dlsym(h, n); };
  a.version = reinterpret_cast<decltype(a.version)>(sym("nvrtcVersion"));
  a.create = reinterpret_cast<decltype(a.create)>(sym("nvrtcCreateProgram"));
  a.compile = reinterpret_cast<decltype(a.compile)>(sym("nvrtcCompileProgram"));
  a.log_size = reinterpret_cast<decltype(a.log_size)>(sym("nvrtcGetProgramLogSize"));
  a.log = reinterpret_cast<decltype(a.log)>(sym("nvrtcGetProgramLog"));
  a.cubin_size = reinterpret_cast<decltype(a.cubin_size)>(sym("nvrtcGetCUBINSize"));
  a.cubin = reinterpret_cast<decltype(a.cubin)>(sym("nvrtcGetCUBIN"));
  a.destroy = reinterpret_cast<decltype(a.destroy)>(sym("nvrtcDestroyProgram"));
  a.error = reinterpret_cast<decltype(a.error)>(sym("nvrtcGetErrorString"));
  if (a.version && a.create && a.compile && a.log_size && a.log && a.cubin_size && a.cubin && a.destroy && a.error)
    return true;
  dlclose(h);
  return false;
}

const NvrtcApi& nvrtc() {
  static const NvrtcApi api = [] {
    NvrtcApi linked = {&nvrtcVersion, &nvrtcCreateProgram, &nvrtcCompileProgram, &nvrtcGetProgramLogSize,
                       &nvrtcGetProgramLog, &nvrtcGetCUBINSize, &nvrtcGetCUBIN, &nvrtcDestroyProgram,
                       &nvrtcGetErrorString};
    int maj = 0, min = 0;
    linked.version(&maj, &min);
    std::vector<std::string> roots;
    for (const char* e : {"DQ_CUDA_HOME", "CUDA_HOME", "CUDA_PATH"})
      if (const char* v = getenv(e)) roots.push_back(v);
    roots.push_back("/usr/local/cuda");
    for (const std::string& r : roots) {
      NvrtcApi a;
      if (!open_nvrtc(r + "/lib64/libnvrtc.so.12", a) && !open_nvrtc(r + "/lib64/libnvrtc.so", a)) continue;
      int M = 0, m = 0;
      if (a.version(&M, &m) == NVRTC_SUCCESS && (M > maj || (M == maj && m > min))) return a;
    }
    return linked;
  }();
  return api;
}

void nvrtc_check(nvrtcResult r, const char* what) {
  if (r != NVRTC_SUCCESS) throw Error(std::string(what) + ": " + nvrtc().error(r));
}

// One NVRTC compilation of `src`; false (log kept) when it does not compile.
bool compile_once(const std::string& src, bool ld256, std::string& log, std::vector<char>& cubin) {
  std::vector<const char*> hdrs, names;
  for (int i = 0; i < kEmbedCount; ++i) {
    hdrs.push_back(kEmbedText[i]);
    names.push_back(kEmbedNames[i]);
  }
  hdrs.push_back(kStdint);
  names.push_back("stdint.h");
  hdrs.push_back(kStddef);
  names.push_back("stddef.h");
  nvrtcProgram prog;
  nvrtc_check(nvrtc().create(&prog, src.c_str(), "dq_pipeline.cu", (int)hdrs.size(), hdrs.data(), names.data()),
              "nvrtcCreateProgram");
  const char* opts[] = {"--gpu-architecture=sm_100a", "-std=c++17", "-default-device", "-lineinfo",
                        "--ptxas-options=-v", ld256 ? "-DDQ_LD256=1" : "-DDQ_LD256=0"};
  nvrtcResult r = nvrtc().compile(prog, (int)(sizeof(opts) / sizeof(opts[0])), opts);
  size_t n = 0;
  nvrtc().log_size(prog, &n);
  log.assign(n, '\0');
  if (n) nvrtc().log(prog, &log[0]);
  while (!log.empty() && log.back() == '\0') log.pop_back();
  if (r != NVRTC_SUCCESS) {
    nvrtc().destroy(&prog);
    return false;
  }
  size_t cb = 0;
  nvrtc_check(nvrtc().cubin_size(prog, &cb), "nvrtcGetCUBINSize");
  cubin.resize(cb);
  nvrtc_check(nvrtc().cubin(prog, cubin.data()), "nvrtcGetCUBIN");
  nvrtc().destroy(&prog);
  return true;
}

// The generated lines around the first line a compiler message names.
std::string source_excerpt(const std::string& src, const std::string& log) {
  const std::string tag = "dq_pipeline.cu(";
  const size_t at = log.find(tag);
  if (at == std::string::npos) return std::string();
  const int line = atoi(log.c_str() + at + tag.size());
  std::string out = "\ngenerated source near line " + std::to_string(line) + ":\n";
  int n = 1;
  size_t pos = 0;
  while (pos < src.size()) {
    size_t end = src.find('\n', pos);
    if (end == std::string::npos) end = src.size();
    if (n >= line - 6 && n <= line + 3) out += std::to_string(n) + ": " + src.substr(pos, end - pos) + "\n";
    pos = end + 1;
    ++n;
  }
  return out;
}

// Whether a ptxas report shows register spills in any function.
bool spills(const std::string& log) {
  const std::string tag = " bytes spill stores";
  for (size_t i = log.find(tag); i != std::string::npos; i = log.find(tag, i + 1)) {
    size_t b = i;
    while (b > 0 && log[b - 1] >= '0' && log[b - 1] <= '9') --b;
    if (b < i && std::stoll(log.substr(b, i - b)) > 0) return true;
  }
  return false;
}

// The source with every `__launch_bounds__(N)` or `__launch_bounds__(N, M)`
// made `__launch_bounds__(N, 1)`.
std::string one_block_bounds(const std::string& src) {
  std::string out;
  const std::string tag = "__launch_bounds__(";
  size_t pos = 0;
  for (size_t i = src.find(tag); i != std::string::npos; i = src.find(tag, pos)) {
    const size_t close = src.find(')', i);
    const size_t comma = src.find(',', i);
    out += src.substr(pos, (comma < close ? comma : close) - pos);
    out += ", 1";
    pos = close;
  }
  return out + src.substr(pos);
}

void build(Entry& e, const std::string& src) {
  // the NVRTC the process resolved (an application may have loaded an older
  // one first): 256-bit loads for sm_100a need 12.9
  int major = 0, minor = 0;
  nvrtc().version(&major, &minor);
  const bool ld256 = major > 12 || (major == 12 && minor >= 9);
  bool ok = compile_once(src, ld256, e.log, e.cubin);
  // With a block size alone in the launch bounds, ptxas may aim at more
  // resident blocks than the kernel's registers allow and spill; a minimum of
  // one block lets it keep the values in registers.  Kept when spill-free.
  if (ok && spills(e.log)) {
    std::string log2;
    std::vector<char> cubin2;
    if (compile_once(one_block_bounds(src), ld256, log2, cubin2) && !spills(log2)) {
      e.log = "launch bounds with a minimum of one block per SM (spill-free)\n" + log2;
      e.cubin.swap(cubin2);
    }
  }
  e.log = "NVRTC " + std::to_string(major) + "." + std::to_string(minor) + "\n" + e.log;
  if (!ok) throw Error("generated pipeline kernel failed to compile:\n" + e.log + source_excerpt(src, e.log));
}

}  // namespace

Kernels compile(const Program& prog, bool load) {
  // the cache is looked up and filled under the lock, the compiler runs
  // outside it: a thread compiling a new shape does not hold up threads whose
  // kernels are cached already (a server's request loop)
  Entry* found = nullptr;
  {
    std::lock_guard<std::mutex> lk(g_mu);
    auto it = g_cache.find(prog.source);
    if (it != g_cache.end()) found = it->second.get();
  }
  if (!found) {
    std::unique_ptr<Entry> built(new Entry());
    build(*built, prog.source);
    std::lock_guard<std::mutex> lk(g_mu);
    std::unique_ptr<Entry>& slot = g_cache[prog.source];
    if (!slot) slot = std::move(built);  // else another thread built it first
    found = slot.get();
  }
  std::lock_guard<std::mutex> lk(g_mu);
  Entry& e = *found;
  if (load && !e.lib) {
    cudaError_t err = cudaLibraryLoadData(&e.lib, e.cubin.data(), nullptr, nullptr, 0, nullptr, nullptr, 0);
    if (err != cudaSuccess) {
      e.lib = nullptr;
      throw Error(std::string("loading a generated pipeline kernel: ") + cudaGetErrorString(err));
    }
    err = cudaLibraryGetKernel(&e.main, e.lib, prog.batched ? "dq_batch_main" : "dq_main");
    if (err == cudaSuccess && prog.heavy)
      err = cudaLibraryGetKernel(&e.heavy, e.lib, prog.batched ? "dq_batch_heavy" : "dq_heavy");
    if (err != cudaSuccess) throw Error(std::string("generated kernel entry: ") + cudaGetErrorString(err));
  }
  Kernels k;
  k.main = e.main;
  k.heavy = e.heavy;
  k.log = e.log;
  return k;
}

}  // namespace jit
}  // namespace dq
