// Host runtime behind the C ABI (include/dogqc_b200.h).
//
// It owns device memory for registered tables and for every plan's resources,
// turns the plan IR into pipeline launch descriptors (shared-memory layout,
// resource layouts, tile sizes, persistent grid size), and executes a plan as
// a stream-ordered sequence of launches.  Where the reference's generated
// main() re-allocates, copies and frees everything per query and times launches
// with std::clock (dogqc/codegen.py:121-159, dogqc/code.py:4-26), this runtime
// keeps tables and hash tables resident, resets them with memsets, and times
// launches with CUDA events on the launching stream.
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <chrono>
#include <condition_variable>
#include <cstdio>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <thread>
#include <unordered_map>
#include <unordered_set>
#include <vector>

#include "../../include/dogqc_b200.h"
#include "dq_device.h"
#include "dq_jit.h"

namespace dq {
cudaError_t launch_pipeline(const DevPipe& P, int grid, cudaStream_t stream);
int pipeline_occupancy(int smem_bytes);
cudaError_t launch_row(const DevPipe& P, int grid, cudaStream_t stream);
int row_occupancy(int smem_bytes);
cudaError_t launch_agg_init(uint64_t* slots, uint64_t nslots, int words, int val_word, int naggs,
                            const int8_t* reds, cudaStream_t stream);
size_t mm_scan_scratch_words(uint64_t n);
cudaError_t launch_mm_scan(uint32_t* counts, uint32_t* offsets, uint64_t n, uint32_t* partials,
                           cudaStream_t stream, int* launches);
cudaError_t launch_heavy_prefix(const DevHeavy& H, uint64_t exp_cap, int32_t* status, cudaStream_t stream);
cudaError_t launch_heavy_group(const DevHeavy& H, int32_t* status, int sms, cudaStream_t stream);
size_t batch_scan_blocks(uint64_t n);
cudaError_t launch_batch_reset(const BatchReset* ops, int nops, int sms, cudaStream_t stream);
cudaError_t launch_batch_scan(const BatchScanSeg* segs, int nseg, uint64_t total_blocks, uint32_t* partials,
                              cudaStream_t stream);
cudaError_t launch_batch_pack(const BatchPack* ops, int nops, uint8_t* dst, int sms, cudaStream_t stream);
cudaError_t launch_import_lines(const ImpText& T, uint64_t ntiles, uint64_t* tile_cnt, uint64_t* tile_off,
                                cudaStream_t st);
cudaError_t launch_import_line_ends(const ImpText& T, uint64_t ntiles, const uint64_t* tile_off, uint64_t* line_end,
                                    cudaStream_t st);
cudaError_t launch_import_parse(const ImpArgs& A, cudaStream_t st);
cudaError_t launch_str_ref_offsets(const uint64_t* refs, uint64_t n, const DevStr* src, uint64_t* lens,
                                   uint64_t* offs, int sms, cudaStream_t st);
cudaError_t launch_str_ref_copy(const uint64_t* refs, uint64_t n, const DevStr* src, const uint64_t* offs,
                                uint8_t* heap, int sms, cudaStream_t st);
cudaError_t launch_import_strings(const ImpArgs& A, cudaStream_t st);
cudaError_t launch_col_minmax(const uint8_t* col, uint64_t n, int width, bool is_signed, long long* out, int sms,
                              cudaStream_t st);
}  // namespace dq

using namespace dq;

namespace {

std::string g_init_error;

}  // namespace

namespace dq_internal {
// Error text for entry points without a context (read with dq_last_error(NULL)).
void set_global_error(const std::string& msg) { g_init_error = msg; }
}  // namespace dq_internal

namespace {

struct DqError : std::runtime_error {
  int code;
  DqError(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

#define DQ_CUDA(expr)                                                                        \
  do {                                                                                       \
    cudaError_t _e = (expr);                                                                 \
    if (_e != cudaSuccess)                                                                   \
      throw DqError(_e == cudaErrorMemoryAllocation ? DQ_ERR_OOM : DQ_ERR_CUDA,              \
                    std::string(#expr) + ": " + cudaGetErrorString(_e));                     \
  } while (0)

int ctype_width(int t) {
  switch (t) {
    case DQ_I8: return 1;
    case DQ_I32:
    case DQ_U32: return 4;
    case DQ_I64:
    case DQ_U64:
    case DQ_STR: return 8;  // as a value, a string is a 64-bit reference (source, window, row)
    default: return 0;
  }
}

uint64_t align_up(uint64_t x, uint64_t a) { return (x + a - 1) / a * a; }

// Set while an offline context (DQ_CFG_OFFLINE) registers tables or prepares
// plans: buffers then record their size but take no device memory.
thread_local bool t_offline = false;

struct OfflineScope {
  bool prev;
  explicit OfflineScope(bool on) : prev(t_offline) { t_offline = on; }
  ~OfflineScope() { t_offline = prev; }
};

// Generation only: with a list set, preparing a plan (under an OfflineScope)
// appends each pipeline's generated program to it instead of compiling it.
thread_local std::vector<jit::Program>* t_collect = nullptr;

struct CollectScope {
  std::vector<jit::Program>* prev;
  explicit CollectScope(std::vector<jit::Program>* to) : prev(t_collect) { t_collect = to; }
  ~CollectScope() { t_collect = prev; }
};

// Device buffer with 256 bytes of tail padding: tile copies round their size up
// to 16 bytes and may read past the last row.
struct DevBuf {
  void* ptr = nullptr;
  size_t bytes = 0;
  std::shared_ptr<DevBuf> slab;  // set for a view into a larger buffer (freed with the last view)
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  ~DevBuf() { release(); }
  void alloc(size_t b) {
    release();
    bytes = b;
    if (t_offline) return;
    DQ_CUDA(cudaMalloc(&ptr, align_up(b, 256) + 256));
  }
  // Grows (never shrinks) a reusable buffer.
  void reserve(size_t b) {
    if (!ptr || bytes < b) alloc(b);
  }
  void release() {
    if (ptr && !slab) cudaFree(ptr);
    slab.reset();
    ptr = nullptr;
    bytes = 0;
  }
  // Bytes a view of `b` bytes takes in a slab (the same padding as alloc).
  static size_t span_of(size_t b) { return align_up(b, 256) + 256; }
  static std::shared_ptr<DevBuf> view(const std::shared_ptr<DevBuf>& slab, size_t off, size_t b) {
    auto v = std::make_shared<DevBuf>();
    v->slab = slab;
    v->ptr = static_cast<uint8_t*>(slab->ptr) + off;
    v->bytes = b;
    return v;
  }
  template <class T>
  T* as() const { return reinterpret_cast<T*>(ptr); }
};

struct ColRec {
  std::string name;
  int ctype = 0;
  int width = 0;       // bytes per value, or string width for fixed strings
  uint64_t nchars = 0;
  std::shared_ptr<DevBuf> data;
  std::shared_ptr<DevBuf> offsets;
};

struct TableRec {
  int64_t nrows = 0;
  std::vector<ColRec> cols;
  const ColRec* find(const char* n) const {
    for (auto& c : cols)
      if (c.name == n) return &c;
    return nullptr;
  }
};

}  // namespace

struct dq_ctx {
  dq_config cfg{};
  int device = 0;
  bool offline = false;     // DQ_CFG_OFFLINE: no device, plans are compiled only
  int sms = 148;
  cudaStream_t stream = nullptr;
  std::string error;
  std::mutex mu;
  std::map<std::string, TableRec> tables;
  dq_import_timing last_import{};
  struct {  // text import scratch, kept for the next import
    DevBuf text, tail, tcnt, toff, lend, err, spos, slen, bsum, boff;
  } imp;
};

struct ResRec {
  dq_resource desc{};
  std::string name;
  DevRes dev{};
  DevBuf slots, counts, offsets, scan_scratch;
  std::vector<std::unique_ptr<DevBuf>> pay;
  uint64_t pay_rows = 0;
  int pct = 100;            // UNIQUE: slots as a percentage of the plan's capacity
  int index = 0;            // position in the plan's resources
  bool agg_clean = false;   // AGG: every slot is in its initial state (the last
                            // run's scan reset what it read)
  int bitmap = 0;           // UNIQUE: a bit (1) or a payload word (2) per key of the
  int64_t bmin = 0;         //   build column's domain [bmin, bmin + brange), no hash table
  uint64_t brange = 0;
  bool no_bitmap = false;   // a run met a key outside the domain: hash table from then on
};

constexpr uint64_t kL2TableBytes = 48ull << 20;  // join tables up to this size get extra slack

struct PipeRec {
  dq_pipeline desc{};
  std::vector<std::string> col_names;
  std::vector<std::string> patterns;
  DevPipe dev{};
  int grid = 1;             // CTAs of a tile launch (at most one per tile)
  int grid_full = 1;        // persistent grid (SMs x resident CTAs)
  bool row = false;         // runs on the row kernel
  bool jit = false;         // runs on its generated kernel
  jit::Program prog;        // generated source and launch shape
  jit::Kernels kernels;
  int expand_op = -1;       // level-0 expansion op with deferral
  uint64_t heavy_cap = 0;   // deferred-item capacity grown after an overflow (0: default)
  uint64_t heavy_threshold = 0;       // adapted deferral threshold (0: the default)
  uint32_t* heavy_stats = nullptr;    // pinned: items and groups of the last run
  ~PipeRec() {
    if (heavy_stats) cudaFreeHost(heavy_stats);
  }
  DevBuf pattern_buf, heavy_items, heavy_count, heavy_prefix;
  std::string pattern_text;  // the concatenated patterns pattern_buf holds (P.pat_off into it)
  DevBuf heavy_gkey, heavy_glen, heavy_gcnt, heavy_glist, heavy_gstart, heavy_sorted;  // grouped deferral
  bool clears_source = false;  // scans an aggregation table that no other pipeline
                               // reads, and may reset its slots as it reads them
  bool mm_count = false;    // sink is a multimap count: bucket scan follows
  int mm_res = -1;
  int staged_cols = 0;
  int tail = -1;            // the pipeline this kernel's last CTA runs (fused tail)
  int fused_into = -1;      // runs inside that pipeline's kernel, not launched
  DevBuf tail_buf;          // device copy of the fused tail's descriptor
};

struct dq_result {
  int64_t nrows = 0;
  std::vector<int> ctypes;
  std::vector<std::vector<uint8_t>> cols;   // DQ_STR: nrows + 1 uint64 offsets into heaps[j]
  std::vector<std::vector<uint8_t>> heaps;
};

// How a plan is laid out: standalone (the default) or as one instance of a
// batch, with the join-table sizing an autotuner may change.
struct PlanOpts {
  bool batch_member = false;  // no standalone kernels, no deferred expansion
  int unique_pct = 0;         // join-table slots, % of the plan's capacity (0: by size)
  int multi_pct = 100;        // multimap buckets, % of the plan's capacity
  int defer_threshold = 0;    // expansion ranges longer than this are deferred (0: adaptive)
  int ctas_per_sm = 0;        // resident CTAs per SM of pipeline kernels (0: occupancy)
  jit::Tuning tuning;
};

struct dq_plan {
  dq_ctx* ctx = nullptr;
  PlanOpts opts;
  std::vector<std::unique_ptr<ResRec>> res;
  std::vector<std::unique_ptr<PipeRec>> pipes;
  int result_res = -1;
  // The words every run starts from zero, in one buffer so that one memset
  // clears them: the status word (8 bytes), two tile counters per pipeline,
  // then one row cursor per resource (used by OUTPUT resources), then the
  // lane-activity histograms of the plan's profile points (33 bins each).
  DevBuf status;
  uint32_t* counters = nullptr;
  uint64_t* cursors = nullptr;
  uint64_t* profile = nullptr;
  int nprofile = 0;
  dq_plan_timing timing{};
  std::vector<cudaEvent_t> events;
  std::vector<DevStr> str_src;  // string columns the pipelines read: string references index these
  DevBuf str_src_dev;
  // Steady state of dq_plan_execute: once a run succeeded, the run's launches
  // are captured as a CUDA graph and replayed while nothing they depend on
  // changes (the signature: every pipeline's descriptor and launch shape and
  // which aggregation tables start clean).  A failed run drops the graph.
  int32_t* host_status = nullptr;   // pinned
  cudaEvent_t graph_ev[2] = {nullptr, nullptr};  // around a graph launch (the
                                    // events inside a graph give no times)
  bool steady = false;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t graph_exec = nullptr;
  std::string graph_sig;
  int graph_launches = 0;
  // Side streams a captured run forks its independent pipelines onto (the
  // graph then holds them as parallel branches), and the fork event.
  std::vector<cudaStream_t> lanes;
  cudaEvent_t fork_ev = nullptr;
  void drop_graph() {
    if (graph_exec) cudaGraphExecDestroy(graph_exec);
    if (graph) cudaGraphDestroy(graph);
    graph_exec = nullptr;
    graph = nullptr;
    graph_sig.clear();
  }
  ~dq_plan() {
    drop_graph();
    if (host_status) cudaFreeHost(host_status);
    for (auto e : graph_ev)
      if (e) cudaEventDestroy(e);
    for (auto l : lanes) cudaStreamDestroy(l);
    if (fork_ev) cudaEventDestroy(fork_ev);
  }
};

// One pipeline of a batch: a generated kernel over all instances.
struct BatchStage {
  jit::Program prog;
  jit::Kernels kernels;
  DevBuf descs;             // the instances' launch descriptors (DevPipe[ninst])
  DevBuf bprefix;           // row blocks of the instances before each (int64[ninst + 1])
  int grid = 1;
  bool mm_scan = false;     // a multimap count: the bucket scan of every instance follows
  DevBuf segs, partials;
  int nsegs = 0;
  uint64_t scan_blocks = 0;
  // deferred expansion shared by the instances (grouped by instance and range)
  DevHeavy heavy{};
  DevBuf h_items, h_count, h_prefix, h_gkey, h_glen, h_gcnt, h_glist, h_gstart, h_sorted, h_units;
  int heavy_grid = 0;
};

struct dq_batch {
  dq_ctx* ctx = nullptr;
  int ninst = 0;
  std::vector<std::unique_ptr<dq_plan>> inst;
  std::vector<std::unique_ptr<BatchStage>> stages;
  DevBuf status, resets, packs, packed, rows;
  int nresets = 0, npacks = 0;
  size_t packed_bytes = 0;
  std::vector<std::vector<uint64_t>> col_off;   // [instance][column] offset in the packed buffer
  uint64_t heavy_cap = 0;                       // deferred items, grown after an overflow
  uint8_t* host = nullptr;                      // pinned: packed columns, rows per instance, status
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  dq_plan_timing timing{};
  int launches = 0;
  jit::Tuning tuning;
  ~dq_batch() {
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    if (host) cudaFreeHost(host);
    if (ev0) cudaEventDestroy(ev0);
    if (ev1) cudaEventDestroy(ev1);
  }
};

namespace {

int fail(dq_ctx* ctx, int code, const std::string& msg) {
  if (ctx) ctx->error = msg;
  else g_init_error = msg;
  return code;
}

template <class F>
int guarded(dq_ctx* ctx, F f) {
  try {
    return f();
  } catch (const DqError& e) {
    return fail(ctx, e.code, e.what());
  } catch (const jit::Error& e) {
    return fail(ctx, DQ_ERR_CUDA, e.what());
  } catch (const std::bad_alloc&) {
    return fail(ctx, DQ_ERR_OOM, "host allocation failed");
  } catch (const std::exception& e) {
    return fail(ctx, DQ_ERR_INVALID, e.what());
  }
}

void upload_column(dq_ctx* ctx, ColRec& rec, const dq_column& c, int64_t nrows, bool device_src,
                   cudaStream_t stream) {
  cudaMemcpyKind kind = device_src ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
  if (ctx->offline) {  // sizes only
    if (!rec.data) rec.data = std::make_shared<DevBuf>();
    if (c.ctype == DQ_STR && c.width <= 0 && !rec.offsets) rec.offsets = std::make_shared<DevBuf>();
    return;
  }
  if (c.ctype == DQ_STR) {
    uint64_t nchars = c.width > 0 ? (uint64_t)c.width * nrows : c.nchars;
    if (!rec.data) rec.data = std::make_shared<DevBuf>();
    if (rec.data->bytes != nchars || !rec.data->ptr) rec.data->alloc(nchars);
    if (nchars) DQ_CUDA(cudaMemcpyAsync(rec.data->ptr, c.data, nchars, kind, stream));
    rec.nchars = nchars;
    if (c.width <= 0) {
      if (!c.offsets) throw DqError(DQ_ERR_INVALID, "variable-width string column " + rec.name + " needs offsets");
      if (!rec.offsets) rec.offsets = std::make_shared<DevBuf>();
      size_t ob = (size_t)(nrows + 1) * 8;
      if (rec.offsets->bytes != ob || !rec.offsets->ptr) rec.offsets->alloc(ob);
      DQ_CUDA(cudaMemcpyAsync(rec.offsets->ptr, c.offsets, ob, kind, stream));
    }
  } else {
    size_t b = (size_t)nrows * ctype_width(c.ctype);
    if (!rec.data) rec.data = std::make_shared<DevBuf>();
    if (rec.data->bytes != b || !rec.data->ptr) rec.data->alloc(b);
    if (b) DQ_CUDA(cudaMemcpyAsync(rec.data->ptr, c.data, b, kind, stream));
  }
}

bool keys_packed(int nkeys, const int8_t* kt) {
  for (int i = 0; i < nkeys; ++i)
    if (kt[i] == DQ_STR) return false;  // string keys hash and compare their bytes
  if (nkeys == 0) return true;
  if (nkeys == 1) return true;
  if (nkeys == 2) return ctype_width(kt[0]) <= 4 && ctype_width(kt[1]) <= 4;
  return false;
}

// ------------------------------------------------------------- resources --

void setup_resource(dq_plan* plan, ResRec& r, int64_t build_rows_bound) {
  const dq_resource& d = r.desc;
  DevRes& R = r.dev;
  memset(&R, 0, sizeof(R));
  r.agg_clean = false;
  R.kind = d.kind;
  R.nkeys = d.nkeys;
  for (int i = 0; i < DQ_MAX_KEYS; ++i) R.key_ctype[i] = d.key_ctype[i];
  R.npay = d.npay;
  R.naggs = d.naggs;
  for (int i = 0; i < DQ_MAX_PAY; ++i) {
    R.pay_ctype[i] = d.pay_ctype[i];
    R.pay_width[i] = (int8_t)ctype_width(d.pay_ctype[i]);
  }
  for (int i = 0; i < DQ_MAX_AGGS; ++i) R.agg_red[i] = d.agg_red[i];
  if (d.nkeys < 0 || d.nkeys > DQ_MAX_KEYS || d.npay < 0 || d.npay > DQ_MAX_PAY || d.naggs < 0 ||
      d.naggs > DQ_MAX_AGGS)
    throw DqError(DQ_ERR_BAD_IR, "resource sizes out of range");
  uint64_t cap = (uint64_t)std::max<int64_t>(d.capacity, 1);
  if (d.kind == DQ_RES_UNIQUE && r.bitmap && !r.no_bitmap) {
    // one bit (no payload) or one word (a payload) per key of the build
    // column's domain, cleared every run; cap counts 32- or 64-bit words
    R.bitmap = r.bitmap;
    R.bmin = r.bmin;
    R.brange = r.brange;
    R.cap = r.bitmap == 1 ? (r.brange + 31) / 32 : r.brange;
    R.words = 0;
    r.slots.alloc(R.cap * (r.bitmap == 1 ? 4 : 8) + 16);
    R.slots = r.slots.as<uint64_t>();
    return;
  }
  switch (d.kind) {
    case DQ_RES_UNIQUE:
    case DQ_RES_AGG: {
      R.packed = keys_packed(d.nkeys, d.key_ctype);
      R.key_word = 1;
      R.val_word = 1 + (R.packed ? 0 : d.nkeys);
      R.words = R.val_word + (d.kind == DQ_RES_UNIQUE ? d.npay : d.naggs);
      // a join table whose one key and one payload fit 32 bits each keeps both
      // in one word (generated kernels; the prebuilt ones read wide slots)
      if (d.kind == DQ_RES_UNIQUE && R.packed && d.nkeys == 1 && ctype_width(d.key_ctype[0]) <= 4 && d.npay == 1 &&
          d.pay_ctype[0] != DQ_STR && ctype_width(d.pay_ctype[0]) <= 4 &&
          !(plan->ctx->cfg.flags & (DQ_CFG_NO_JIT | DQ_CFG_ROW_KERNEL))) {
        R.compact = 1;
        R.words = 1;
        R.val_word = 0;
      }
      // join tables get more slots than the plan asks for: most probes of a
      // selective join miss, a miss walks to the next empty slot, and a walk
      // past the first 32-byte slot group is a second dependent load.  Four
      // times (a load factor of at most 1/8 with the reference's default size
      // factor 2) while the table stays small enough to live in L2 beside the
      // probe's input stream, else twice.  A slot count divisible by 4 lets
      // probes read aligned 32-byte slot groups.
      if (d.kind == DQ_RES_UNIQUE) {
        r.pct = plan->opts.unique_pct > 0 ? std::max(plan->opts.unique_pct, 25)
                : cap * 4 * (uint64_t)R.words * 8 <= kL2TableBytes ? 400 : 200;
        cap = (cap * (uint64_t)r.pct / 100 + 3) & ~3ull;
      }
      cap = std::max<uint64_t>(cap, 16);
      if (cap >= 0xffffffffull) throw DqError(DQ_ERR_UNSUPPORTED, "hash tables hold fewer than 2^32 slots");
      R.cap = cap;
      r.slots.alloc((cap + 1 + (R.compact ? 1 : 0)) * R.words * 8);
      R.slots = r.slots.as<uint64_t>();
      bool str_keys = false;
      for (int i = 0; i < d.nkeys; ++i) str_keys |= d.key_ctype[i] == DQ_STR;
      if (d.kind == DQ_RES_AGG && (R.packed || str_keys)) {
        // CTA-local table (generated kernels only for string keys: they store the keys too)
        uint64_t want = std::max<int64_t>(d.group_hint, 1) * 2;
        uint64_t ns = 16;
        while (ns < want) ns <<= 1;
        uint64_t bytes = (ns + 1) * (1 + d.naggs) * 8 + (str_keys ? ns * d.nkeys * 8 : 0);
        if (d.nkeys == 0) ns = 1, bytes = 2 * (1 + d.naggs) * 8;
        R.smem_slots = bytes <= 24 * 1024 ? (int)ns : 0;
      }
      break;
    }
    case DQ_RES_MULTI: {
      cap = std::max<uint64_t>(1, cap * (uint64_t)std::max(plan->opts.multi_pct, 10) / 100);
      if (cap >= 0xffffffffull) throw DqError(DQ_ERR_UNSUPPORTED, "multimaps hold fewer than 2^32 buckets");
      R.cap = cap;
      r.counts.alloc(cap * 4);
      r.offsets.alloc((cap + 1) * 4);
      R.counts = r.counts.as<uint32_t>();
      R.offsets = r.offsets.as<uint32_t>();
      r.scan_scratch.alloc(mm_scan_scratch_words(cap) * 4);
      r.pay_rows = (uint64_t)std::max<int64_t>(build_rows_bound, 1);
      r.pay.clear();
      for (int j = 0; j < d.npay; ++j) {
        r.pay.emplace_back(new DevBuf());
        r.pay.back()->alloc(r.pay_rows * ctype_width(d.pay_ctype[j]));
        R.pay[j] = r.pay.back()->as<uint8_t>();
      }
      break;
    }
    case DQ_RES_OUTPUT: {
      R.cap = cap;
      R.cursor = plan->cursors ? plan->cursors + r.index : nullptr;
      r.pay.clear();
      for (int j = 0; j < d.npay; ++j) {
        r.pay.emplace_back(new DevBuf());  // a string column holds references (8 bytes a row)
        r.pay.back()->alloc(cap * ctype_width(d.pay_ctype[j]));
        R.pay[j] = r.pay.back()->as<uint8_t>();
      }
      break;
    }
    default:
      throw DqError(DQ_ERR_BAD_IR, "unknown resource kind");
  }
}

// ------------------------------------------------------------- pipelines --

void slot_reads(const dq_pipeline& d, const dq_op& op, std::vector<int>& out) {
  auto add = [&](int s) {
    if (s >= 0) out.push_back(s);
  };
  auto add_list = [&](int list, int n) {
    for (int i = 0; i < n; ++i) add(d.lists[list + i]);
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

void validate_pipeline(const dq_pipeline& d, int nres) {
  if (d.nslots < 0 || d.nslots > DQ_MAX_SLOTS || d.nops <= 0 || d.nops > DQ_MAX_OPS || d.nlist < 0 ||
      d.nlist > DQ_MAX_LIST || d.ncols < 0 || d.ncols > DQ_MAX_COLS || d.npatterns < 0 ||
      d.npatterns > DQ_MAX_PATTERNS)
    throw DqError(DQ_ERR_BAD_IR, "pipeline sizes out of range");
  auto slot_ok = [&](int s) { return s >= -1 && s < d.nslots; };
  for (int i = 0; i < d.nops; ++i) {
    const dq_op& op = d.ops[i];
    if (!slot_ok(op.dst) || !slot_ok(op.a) || !slot_ok(op.b) || !slot_ok(op.c))
      throw DqError(DQ_ERR_BAD_IR, "op slot out of range");
    if (op.nlist < 0 || op.nlist2 < 0 || op.list < 0 || op.list2 < 0 || op.list + op.nlist > d.nlist ||
        op.list2 + op.nlist2 > d.nlist)
      throw DqError(DQ_ERR_BAD_IR, "op list out of range");
    bool sink = op.kind >= DQ_OP_AGG;
    if (sink != (i == d.nops - 1)) throw DqError(DQ_ERR_BAD_IR, "the sink must be the last op");
    if ((op.kind == DQ_OP_PROBE || op.kind == DQ_OP_EXPAND || op.kind == DQ_OP_EXISTS || sink) &&
        (op.res < 0 || op.res >= nres))
      throw DqError(DQ_ERR_BAD_IR, "op resource out of range");
    if (op.kind == DQ_OP_EXISTS) {
      // the condition's ops follow it and are plain scalar ops
      if (op.imm < 0 || i + op.imm >= d.nops - 1 || (op.imm > 0 && op.a < 0) ||
          (op.sub != DQ_JOIN_SEMI && op.sub != DQ_JOIN_ANTI) || op.nlist != op.nlist2)
        throw DqError(DQ_ERR_BAD_IR, "malformed EXISTS op");
      for (int64_t j = i + 1; j <= i + op.imm; ++j) {
        const int kj = d.ops[j].kind;
        if (kj != DQ_OP_ARITH && kj != DQ_OP_CMP && kj != DQ_OP_LOGIC && kj != DQ_OP_CAST && kj != DQ_OP_SELECT)
          throw DqError(DQ_ERR_BAD_IR, "an EXISTS condition holds scalar ops only");
      }
    }
    const bool two_strings = op.kind == DQ_OP_STREQ && op.res == -1;
    if ((op.kind == DQ_OP_LIKE || op.kind == DQ_OP_STREQ) && !two_strings && (op.res < 0 || op.res >= d.npatterns))
      throw DqError(DQ_ERR_BAD_IR, "pattern index out of range");
    auto is_str = [&](int s) { return s >= 0 && d.slots[s].ctype == DQ_STR; };
    if ((op.kind == DQ_OP_LIKE || op.kind == DQ_OP_STREQ) && (!is_str(op.a) || (two_strings && !is_str(op.b))))
      throw DqError(DQ_ERR_BAD_IR, "string comparison of a non-string slot");
    if (op.kind == DQ_OP_SUBSTR) {
      const int32_t from = (int32_t)(uint32_t)op.imm, len = (int32_t)(uint32_t)((uint64_t)op.imm >> 32);
      if (!is_str(op.a) || d.slots[op.a].kind == DQ_SLOT_STR || op.dst < 0 || d.slots[op.dst].ctype != DQ_STR)
        throw DqError(DQ_ERR_BAD_IR, "SUBSTR takes and gives string references");
      if ((int64_t)from - 1 + (int64_t)len > 255 || (int64_t)from - 1 > 255)
        throw DqError(DQ_ERR_UNSUPPORTED, "substring windows end within the first 255 bytes of a string");
    }
    if (op.nlist > DQ_MAX_KEYS && (op.kind == DQ_OP_PROBE || op.kind == DQ_OP_EXPAND || op.kind == DQ_OP_EXISTS ||
                                    op.kind == DQ_OP_BUILD ||
                                    op.kind == DQ_OP_AGG || op.kind == DQ_OP_MM_COUNT || op.kind == DQ_OP_MM_SCATTER))
      throw DqError(DQ_ERR_BAD_IR, "too many keys");
  }
  for (int i = 0; i < d.nlist; ++i)
    if (!slot_ok(d.lists[i])) throw DqError(DQ_ERR_BAD_IR, "list entry out of range");
  for (int s = 0; s < d.nslots; ++s) {
    const dq_slot& sl = d.slots[s];
    if (sl.level < 0 || sl.level >= DQ_MAX_LEVELS) throw DqError(DQ_ERR_BAD_IR, "slot level out of range");
    if (sl.ctype < DQ_I8 || sl.ctype > DQ_STR) throw DqError(DQ_ERR_BAD_IR, "slot type out of range");
    if ((sl.kind == DQ_SLOT_COL || sl.kind == DQ_SLOT_STR) && (sl.src < 0 || sl.src >= d.ncols))
      throw DqError(DQ_ERR_BAD_IR, "slot column out of range");
    if ((sl.kind == DQ_SLOT_GATHER || sl.kind == DQ_SLOT_AGGKEY || sl.kind == DQ_SLOT_AGGVAL) &&
        (sl.res < 0 || sl.res >= nres))
      throw DqError(DQ_ERR_BAD_IR, "slot resource out of range");
  }
}

void setup_pipeline(dq_plan* plan, PipeRec& p) {
  dq_ctx* ctx = plan->ctx;
  const dq_pipeline& d = p.desc;
  DevPipe& P = p.dev;
  memset(&P, 0, sizeof(P));
  validate_pipeline(d, (int)plan->res.size());

  const int tile = ctx->cfg.tile_rows > 0 ? ctx->cfg.tile_rows : 1024;
  if (tile % 16 || tile > kThreads * 8 || tile < 32) throw DqError(DQ_ERR_INVALID, "tile_rows must be a multiple of 16 in [32, 2048]");
  P.tile = tile;
  P.exp_cap = tile;
  P.use_tma = !(ctx->cfg.flags & DQ_CFG_NO_TMA);
  P.source_kind = d.source_kind;
  P.source_res = d.source_res;
  P.status = plan->status.as<int32_t>();
  P.profile = plan->profile;

  // resources: the pipeline sees the plan's resources under the same indices
  if (plan->res.size() > (size_t)kMaxRes) throw DqError(DQ_ERR_UNSUPPORTED, "more than " + std::to_string(kMaxRes) + " resources in a plan");
  P.nres = (int)plan->res.size();
  for (size_t i = 0; i < plan->res.size(); ++i) P.res[i] = plan->res[i]->dev;

  // source columns
  std::vector<int> col_map(d.ncols, -1);  // pipeline column -> staged / string index
  const TableRec* table = nullptr;
  if (d.source_kind == DQ_SRC_TABLE) {
    auto it = ctx->tables.find(d.table ? d.table : "");
    if (it == ctx->tables.end()) throw DqError(DQ_ERR_NOT_FOUND, std::string("unknown table ") + (d.table ? d.table : "(null)"));
    table = &it->second;
    P.nrows = table->nrows;
  } else if (d.source_kind == DQ_SRC_OUTPUT) {
    if (d.source_res < 0 || d.source_res >= (int)plan->res.size() || plan->res[d.source_res]->desc.kind != DQ_RES_OUTPUT)
      throw DqError(DQ_ERR_BAD_IR, "bad temp-table source");
    P.nrows_dev = plan->res[d.source_res]->dev.cursor;
  } else if (d.source_kind == DQ_SRC_AGG) {
    if (d.source_res < 0 || d.source_res >= (int)plan->res.size() || plan->res[d.source_res]->desc.kind != DQ_RES_AGG)
      throw DqError(DQ_ERR_BAD_IR, "bad aggregation source");
    const DevRes& ar = plan->res[d.source_res]->dev;
    P.nrows = ar.nkeys == 0 ? 1 : (int64_t)ar.cap + 1;  // no grouping: exactly one row
  } else {
    throw DqError(DQ_ERR_BAD_IR, "bad source kind");
  }
  int off = 0;
  for (int i = 0; i < d.ncols; ++i) {
    const char* cname = d.cols[i];
    if (d.source_kind == DQ_SRC_TABLE) {
      const ColRec* c = table->find(cname ? cname : "");
      if (!c) throw DqError(DQ_ERR_NOT_FOUND, std::string("unknown column ") + (cname ? cname : "(null)"));
      if (c->ctype == DQ_STR) {
        if (P.nstr >= kMaxStr) throw DqError(DQ_ERR_UNSUPPORTED, "too many string columns");
        DevStr& s = P.strs[P.nstr];
        s.chars = c->data->as<uint8_t>();
        s.offsets = c->offsets ? c->offsets->as<uint64_t>() : nullptr;
        s.width = c->width;
        s.sid = -1;
        for (size_t k = 0; k < plan->str_src.size(); ++k)
          if (plan->str_src[k].chars == s.chars && plan->str_src[k].offsets == s.offsets) s.sid = (int32_t)k;
        if (s.sid < 0) {
          if (plan->str_src.size() >= (size_t)kStrRefMaxSources)
            throw DqError(DQ_ERR_UNSUPPORTED, "a plan reads at most 4096 string columns");
          s.sid = (int32_t)plan->str_src.size();
          plan->str_src.push_back(s);
        }
        col_map[i] = P.nstr++;
      } else {
        DevCol& dc = P.cols[P.ncols];
        dc.ptr = c->data->as<uint8_t>();
        dc.width = ctype_width(c->ctype);
        dc.smem_off = off;
        off += (int)align_up((uint64_t)tile * dc.width, 16);
        col_map[i] = P.ncols++;
      }
    } else if (d.source_kind == DQ_SRC_OUTPUT) {
      int j = atoi(cname ? cname : "-1");
      const ResRec& o = *plan->res[d.source_res];
      if (j < 0 || j >= o.desc.npay) throw DqError(DQ_ERR_BAD_IR, "bad temp-table column");
      DevCol& dc = P.cols[P.ncols];
      dc.ptr = o.dev.pay[j];
      dc.width = ctype_width(o.desc.pay_ctype[j]);
      dc.smem_off = off;
      off += (int)align_up((uint64_t)tile * dc.width, 16);
      col_map[i] = P.ncols++;
    }
  }
  P.stage_bytes = off;
  p.staged_cols = P.ncols;

  // slots and register areas
  int reg_bytes[DQ_MAX_LEVELS] = {0, 0, 0};
  int nlevels = 1;
  P.nslots = d.nslots;
  for (int s = 0; s < d.nslots; ++s) {
    const dq_slot& sl = d.slots[s];
    DevSlot& ds = P.slots[s];
    ds.kind = sl.kind;
    ds.level = sl.level;
    ds.ctype = sl.ctype;
    ds.src = sl.src;
    ds.res = sl.res;
    ds.stash = -1;
    nlevels = std::max(nlevels, (int)sl.level + 1);
    switch (sl.kind) {
      case DQ_SLOT_COL:
        if (col_map[sl.src] < 0 || d.source_kind == DQ_SRC_AGG) throw DqError(DQ_ERR_BAD_IR, "COL slot on a non-staged column");
        ds.src = (int16_t)col_map[sl.src];
        ds.width = (int8_t)P.cols[ds.src].width;
        break;
      case DQ_SLOT_STR:
        if (col_map[sl.src] < 0) throw DqError(DQ_ERR_BAD_IR, "STR slot on a bad column");
        ds.src = (int16_t)col_map[sl.src];
        ds.width = 0;
        break;
      case DQ_SLOT_REG:
        ds.width = (int8_t)ctype_width(sl.ctype);
        if (!ds.width) throw DqError(DQ_ERR_UNSUPPORTED, "string registers");
        ds.smem_off = reg_bytes[sl.level];
        reg_bytes[sl.level] += (int)align_up((uint64_t)tile * ds.width, 16);
        break;
      case DQ_SLOT_GATHER: {
        const ResRec& r = *plan->res[sl.res];
        if (r.desc.kind != DQ_RES_MULTI || sl.src < 0 || sl.src >= r.desc.npay) throw DqError(DQ_ERR_BAD_IR, "bad GATHER slot");
        if (sl.level < 1) throw DqError(DQ_ERR_BAD_IR, "GATHER slot on level 0");
        ds.width = (int8_t)ctype_width(r.desc.pay_ctype[sl.src]);
        break;
      }
      case DQ_SLOT_AGGKEY:
      case DQ_SLOT_AGGVAL:
        if (d.source_kind != DQ_SRC_AGG || sl.res != d.source_res) throw DqError(DQ_ERR_BAD_IR, "aggregation slot outside its scan");
        ds.width = 8;
        break;
      default:
        throw DqError(DQ_ERR_BAD_IR, "bad slot kind");
    }
  }
  // ops, lists, patterns (d.patterns point into p.patterns, which outlives
  // every re-derivation of the pipeline)
  P.nops = d.nops;
  for (int i = 0; i < d.nops; ++i) P.ops[i] = d.ops[i];
  for (int i = 0; i < d.nlist; ++i) P.lists[i] = d.lists[i];
  std::string& cat = p.pattern_text;
  cat.clear();
  for (int i = 0; i < d.npatterns; ++i) {
    P.pat_off[i] = (int32_t)cat.size();
    cat += d.patterns[i] ? d.patterns[i] : "";
  }
  P.pat_off[d.npatterns] = (int32_t)cat.size();
  if (!cat.empty()) {
    p.pattern_buf.alloc(cat.size());
    if (!ctx->offline && !t_offline) DQ_CUDA(cudaMemcpy(p.pattern_buf.ptr, cat.data(), cat.size(), cudaMemcpyHostToDevice));
    P.patterns = p.pattern_buf.as<uint8_t>();
  }
  const dq_op& sink = d.ops[d.nops - 1];
  p.mm_count = sink.kind == DQ_OP_MM_COUNT;
  p.mm_res = p.mm_count ? sink.res : -1;
  for (int i = 0; i < d.nops; ++i)
    if (d.ops[i].kind == DQ_OP_EXPAND) nlevels = std::max(nlevels, 2);

  // deferred wide expansion ranges for the first level-0 expansion
  p.expand_op = -1;
  for (int i = 0; i < d.nops; ++i) {
    const dq_op& op = d.ops[i];
    if (op.kind != DQ_OP_EXPAND) continue;
    bool level0 = true;
    for (int q = 0; q < op.nlist; ++q) level0 &= d.slots[d.lists[op.list + q]].level == 0;
    if (!level0) break;
    std::vector<int> reads;
    for (int j = i; j < d.nops; ++j) slot_reads(d, d.ops[j], reads);
    std::vector<int> stash;
    bool ok = true;
    for (int s : reads) {
      if (d.slots[s].level != 0) continue;
      if (d.slots[s].kind == DQ_SLOT_STR) ok = false;
      if (std::find(stash.begin(), stash.end(), s) == stash.end()) stash.push_back(s);
    }
    if (!ok || (int)stash.size() > kMaxStash) break;
    for (size_t q = 0; q < stash.size(); ++q) P.slots[stash[q]].stash = (int)q;
    p.expand_op = i;
    DevHeavy& H = P.heavy;
    H.nstash = (int)stash.size();
    H.words = 2 + H.nstash;
    int64_t rows = P.nrows_dev ? 1 << 20 : P.nrows;
    H.cap = (uint32_t)std::min<int64_t>(std::max<int64_t>(rows, 1),
                                        std::max<int64_t>(1 << 20, (int64_t)p.heavy_cap));
    H.op = i;
    // generated kernels group the deferred items by range, so shorter ranges
    // pay off there: a range is gathered once per 32-row chunk for all probe
    // rows that matched it
    H.grouped = plan->opts.batch_member || !(ctx->cfg.flags & (DQ_CFG_NO_JIT | DQ_CFG_ROW_KERNEL)) ? 1 : 0;
    const uint64_t dflt = H.grouped ? (p.heavy_threshold ? p.heavy_threshold : (uint64_t)kGroupThreshold)
                                    : (uint64_t)tile * 8;
    H.threshold = ctx->cfg.defer_threshold > 0    ? (uint64_t)ctx->cfg.defer_threshold
                  : plan->opts.defer_threshold > 0 ? (uint64_t)plan->opts.defer_threshold
                                                   : dflt;
    if (H.grouped && !p.heavy_stats && !ctx->offline && !t_offline && !plan->opts.batch_member)
      DQ_CUDA(cudaMallocHost((void**)&p.heavy_stats, 8));
    if (plan->opts.batch_member) break;  // the batch holds the buffers, shared by its instances
    p.heavy_items.alloc((size_t)H.cap * H.words * 8);
    p.heavy_count.alloc(8);  // item count, group count
    size_t nprefix = (size_t)H.cap + 1;
    if (H.grouped) {
      // distinct ranges longer than the threshold: at most rows / (threshold + 1)
      const uint64_t rows_bound = std::max<uint64_t>(plan->res[op.res]->pay_rows, 1);
      const uint64_t groups = std::min<uint64_t>(H.cap, rows_bound / (H.threshold + 1) + 1);
      H.gcap = (uint32_t)std::max<uint64_t>(64, 2 * groups);
      p.heavy_gkey.alloc((size_t)H.gcap * 8);
      p.heavy_glen.alloc((size_t)H.gcap * 4);
      p.heavy_gcnt.alloc((size_t)H.gcap * 4);
      p.heavy_glist.alloc((size_t)H.gcap * 4);
      p.heavy_gstart.alloc(((size_t)H.gcap + 1) * 4);
      p.heavy_sorted.alloc((size_t)H.cap * std::max(H.nstash, 1) * 8);
      H.gkey = p.heavy_gkey.as<uint64_t>();
      H.glen = p.heavy_glen.as<uint32_t>();
      H.gcnt = p.heavy_gcnt.as<uint32_t>();
      H.glist = p.heavy_glist.as<uint32_t>();
      H.ngroups = p.heavy_count.as<uint32_t>() + 1;
      H.gstart = p.heavy_gstart.as<uint32_t>();
      H.sorted = p.heavy_sorted.as<uint64_t>();
      nprefix = std::max<size_t>(nprefix, (size_t)H.gcap + 1);
    }
    p.heavy_prefix.alloc(nprefix * 8);
    H.items = p.heavy_items.as<uint64_t>();
    H.count = p.heavy_count.as<uint32_t>();
    H.unit_prefix = p.heavy_prefix.as<uint64_t>();
    break;
  }

  // row kernel (on request) for pipelines without a multimap expansion
  p.row = (ctx->cfg.flags & DQ_CFG_ROW_KERNEL) != 0;
  for (int i = 0; i < d.nops; ++i)
    if (d.ops[i].kind == DQ_OP_EXPAND) p.row = false;

  // shared-memory layout
  int base = 0;
  auto take = [&](int bytes) {
    int o = base;
    base += (int)align_up(bytes, 16);
    return o;
  };
  P.nstage = p.staged_cols ? 3 : 1;
  for (int l = 0; l < DQ_MAX_LEVELS; ++l) P.off_reg[l] = P.off_sel[l] = P.off_par[l] = P.off_match[l] = 0;
  if (p.row) {
    // the launch descriptor first (the row kernel copies it there), then one
    // 8-byte register per thread for every computed value
    base = (int)align_up(sizeof(DevPipe), 16);
    int nreg = 0;
    for (int s = 0; s < P.nslots; ++s)
      if (P.slots[s].kind == DQ_SLOT_REG) P.slots[s].smem_off = nreg++;
    P.off_reg[0] = take(std::max(nreg, 1) * kThreads * 8);
  } else {
    for (int l = 0; l < nlevels; ++l) {
      P.off_reg[l] = take(reg_bytes[l]);
      P.off_sel[l] = take(tile * 2);
      if (l > 0) {
        P.off_par[l] = take(tile * 2);
        P.off_match[l] = take(tile * 4);
      }
    }
    P.off_exp = take(std::max(1, nlevels - 1) * 3 * tile * 4);
    P.off_flags = take(tile);
    P.off_stash = take(kMaxStash * 8);
  }
  for (int r = 0; r < P.nres; ++r) {
    DevRes& R = P.res[r];
    if (R.kind == DQ_RES_AGG && R.smem_slots > 0) {
      bool used = sink.kind == DQ_OP_AGG && sink.res == r;
      if (used) R.smem_off = take((R.smem_slots + 1) * (1 + R.naggs) * 8);
      else R.smem_slots = 0;
    } else if (R.kind == DQ_RES_AGG) {
      R.smem_slots = 0;
    }
  }
  const int fixed = base;
  const int max_smem = 227 * 1024 - 2048;
  while (P.nstage > 1 && fixed + P.nstage * P.stage_bytes > max_smem) --P.nstage;
  if (fixed + P.nstage * P.stage_bytes > max_smem)
    throw DqError(DQ_ERR_UNSUPPORTED, "pipeline needs more shared memory than a CTA has; lower tile_rows");
  P.off_stage = fixed;
  P.smem_bytes = fixed + P.nstage * P.stage_bytes;

  // generated kernel (default), else the prebuilt tile or row kernel
  p.jit = !(ctx->cfg.flags & (DQ_CFG_NO_JIT | DQ_CFG_ROW_KERNEL)) && !plan->opts.batch_member;
  for (int i = 0; i < d.nops; ++i)
    if ((d.ops[i].kind == DQ_OP_EXISTS || d.ops[i].kind == DQ_OP_PROFILE) && !p.jit && !plan->opts.batch_member)
      throw DqError(DQ_ERR_UNSUPPORTED, "semi/anti joins with conditions and lane-activity profiles run on "
                                        "generated kernels only (not DQ_CFG_NO_JIT / DQ_CFG_ROW_KERNEL)");
  if (!p.jit && !plan->opts.batch_member)
    for (int k = 0; k < p.desc.nops; ++k) {
      const dq_op& op = p.desc.ops[k];
      // the prebuilt kernels read strings in place only: references (string
      // keys, payloads, results, substrings) need generated kernels
      const bool refs = op.kind == DQ_OP_STRREF || op.kind == DQ_OP_SUBSTR ||
                        ((op.kind == DQ_OP_LIKE || op.kind == DQ_OP_STREQ) &&
                         (op.res < 0 || p.desc.slots[op.a].kind != DQ_SLOT_STR));
      if (refs)
        throw DqError(DQ_ERR_UNSUPPORTED, "string join keys, string group keys, substrings and string result columns "
                                          "run on generated kernels only (not DQ_CFG_NO_JIT / DQ_CFG_ROW_KERNEL)");
    }
  int occ = 1;
  int64_t rows_per_cta = tile;
  if (plan->opts.batch_member) {
    // the batch launches its own many-instance kernels
  } else if (p.jit && p.fused_into >= 0) {
    // runs inside the kernel of pipeline `fused_into`: no kernel of its own
  } else if (p.jit) {
    const DevPipe* tail = p.tail >= 0 && p.expand_op < 0 ? &plan->pipes[p.tail]->dev : nullptr;
    if (p.tail >= 0 && !tail) throw DqError(DQ_ERR_BAD_IR, "a pipeline with deferred expansion cannot run a fused tail");
    p.prog = jit::generate(P, p.expand_op, d.compact - 1, plan->opts.tuning, tail, &p.pattern_text);
    if (t_collect) t_collect->push_back(p.prog);
    else p.kernels = jit::compile(p.prog, !ctx->offline);
    rows_per_cta = (int64_t)p.prog.block * p.prog.rows_per_thread;
    if (!ctx->offline && !t_offline) {
      const void* fn = (const void*)p.kernels.main;
      DQ_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, p.prog.smem_bytes));
      DQ_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, fn, p.prog.block, p.prog.smem_bytes));
      if (p.kernels.heavy)
        DQ_CUDA(cudaFuncSetAttribute((const void*)p.kernels.heavy, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     p.prog.smem_bytes));
    }
  } else if (!ctx->offline) {
    occ = p.row ? row_occupancy(P.smem_bytes) : pipeline_occupancy(P.smem_bytes);
  }
  if (occ < 1) throw DqError(DQ_ERR_UNSUPPORTED, "pipeline kernel cannot be resident with this shared memory");
  const int asked = plan->opts.ctas_per_sm > 0 ? plan->opts.ctas_per_sm : ctx->cfg.ctas_per_sm;
  int want = asked > 0 ? std::min(asked, occ) : occ;
  p.grid_full = ctx->sms * want;
  p.grid = p.grid_full;
  if (!P.nrows_dev) {  // no more CTAs than row blocks
    int64_t blocks = (P.nrows + rows_per_cta - 1) / rows_per_cta;
    p.grid = (int)std::max<int64_t>(1, std::min<int64_t>(p.grid_full, blocks));
  }
}

cudaError_t launch_generated(cudaKernel_t k, const DevPipe& P, int grid, int block, int smem, cudaStream_t st) {
  void* args[] = {(void*)&P};
  return cudaLaunchKernel((const void*)k, dim3(grid), dim3(block), args, (size_t)smem, st);
}

void free_events(dq_plan* plan) {
  for (auto e : plan->events) cudaEventDestroy(e);
  plan->events.clear();
}

// Resources pipeline i's kernel reads and writes, its fused tail's included.
// A scanned temp table or aggregation table counts as written as well (a scan
// may reset the slots it reads).
void pipe_access(const dq_plan* plan, size_t i, std::vector<int>& rd, std::vector<int>& wr) {
  rd.clear();
  wr.clear();
  for (size_t j = 0; j < plan->pipes.size(); ++j) {
    const PipeRec& p = *plan->pipes[j];
    if (j != i && p.fused_into != (int)i) continue;
    const dq_pipeline& d = p.desc;
    if (d.source_kind == DQ_SRC_OUTPUT || d.source_kind == DQ_SRC_AGG) {
      rd.push_back(d.source_res);
      wr.push_back(d.source_res);
    }
    for (int k = 0; k < d.nops && k < DQ_MAX_OPS; ++k) {
      const dq_op& op = d.ops[k];
      switch (op.kind) {
        case DQ_OP_PROBE:
        case DQ_OP_EXPAND:
        case DQ_OP_EXISTS:
          rd.push_back(op.res);
          break;
        case DQ_OP_AGG:
        case DQ_OP_BUILD:
        case DQ_OP_MM_COUNT:
        case DQ_OP_MM_SCATTER:
        case DQ_OP_EMIT:
          wr.push_back(op.res);
          break;
        default:
          break;
      }
    }
  }
}

// For each launched pipeline, the earlier launched pipelines it must follow:
// those that write a resource it reads or writes, or read one it writes.
std::vector<std::vector<int>> pipe_deps(const dq_plan* plan) {
  const size_t np = plan->pipes.size();
  std::vector<std::vector<int>> rd(np), wr(np), deps(np);
  for (size_t i = 0; i < np; ++i) pipe_access(plan, i, rd[i], wr[i]);
  auto meets = [](const std::vector<int>& a, const std::vector<int>& b) {
    for (int x : a)
      for (int y : b)
        if (x == y) return true;
    return false;
  };
  for (size_t j = 0; j < np; ++j) {
    if (plan->pipes[j]->fused_into >= 0) continue;
    for (size_t i = 0; i < j; ++i) {
      if (plan->pipes[i]->fused_into >= 0) continue;
      if (meets(wr[i], rd[j]) || meets(wr[i], wr[j]) || meets(rd[i], wr[j])) deps[j].push_back((int)i);
    }
  }
  return deps;
}

// Enqueues one execution of all pipelines on `st`, ending with the copy of the
// device status word to `host_status`; returns the kernels launched.
// `dag` (a captured run): a pipeline that follows no unfinished pipeline of
// `st` starts on a side stream, so independent pipelines become parallel
// branches of the graph; each waits for the pipelines it depends on.
//
// `fast` (dq_plan_execute, where the caller reads the status after every run):
// an aggregation table that exactly one later pipeline scans is reset by that
// scan (each thread puts back the slots it read), so the next run needs no
// initialising kernel; run_once records which tables a successful run left
// clean.  Captured runs (served requests) always initialise, since a graph
// replays the same launches whatever the previous replay left.
constexpr int kLanes = 4;  // streams a captured run spreads its pipelines over

// The side streams and fork event of a captured run (made before the capture).
void ensure_lanes(dq_plan* plan) {
  while ((int)plan->lanes.size() < kLanes - 1) {
    cudaStream_t l;
    DQ_CUDA(cudaStreamCreateWithFlags(&l, cudaStreamNonBlocking));
    plan->lanes.push_back(l);
  }
  if (!plan->fork_ev) DQ_CUDA(cudaEventCreateWithFlags(&plan->fork_ev, cudaEventDisableTiming));
}

int enqueue_run(dq_plan* plan, cudaStream_t st, int32_t* host_status, bool fast = false, bool dag = false) {
  int launches = 0;
  const size_t np = plan->pipes.size();
  std::vector<std::vector<int>> deps;
  std::vector<int> lane_of(np, 0), lane_last(kLanes, -1);
  std::vector<bool> lane_forked(kLanes, false);
  bool forks = false;
  if (dag) {
    if ((int)plan->lanes.size() < kLanes - 1 || !plan->fork_ev) throw DqError(DQ_ERR_INVALID, "side streams missing");
    deps = pipe_deps(plan);
    // lanes: a fused tail runs with its kernel, a pipeline with dependencies
    // continues the chain of the latest one, the others take the least
    // recently used lane
    std::vector<int> last(kLanes, -1);
    for (size_t i = 0; i < np; ++i) {
      const PipeRec& p = *plan->pipes[i];
      int lane = 0;
      if (p.fused_into >= 0) {
        lane = lane_of[(size_t)p.fused_into];
      } else if (!deps[i].empty()) {
        lane = lane_of[(size_t)deps[i].back()];
      } else {
        for (int l = 1; l < kLanes; ++l)
          if (last[(size_t)l] < last[(size_t)lane]) lane = l;
      }
      lane_of[i] = lane;
      last[(size_t)lane] = (int)i;
      forks |= lane != 0;
    }
    dag = forks;
  }
  auto lane_stream = [&](int l) { return l == 0 ? st : plan->lanes[(size_t)l - 1]; };
  if (plan->events.size() != 2 * np + 2) {
    free_events(plan);
    for (size_t i = 0; i < 2 * np + 2; ++i) {
      cudaEvent_t e;
      DQ_CUDA(cudaEventCreate(&e));
      plan->events.push_back(e);
    }
  }
  DQ_CUDA(cudaEventRecord(plan->events[0], st));
  // status, tile counters and output cursors: one buffer, one memset
  DQ_CUDA(cudaMemsetAsync(plan->status.ptr, 0, plan->status.bytes, st));
  for (auto& rp : plan->res) {
    ResRec& r = *rp;
    switch (r.desc.kind) {
      case DQ_RES_UNIQUE:
        DQ_CUDA(cudaMemsetAsync(r.slots.ptr, r.dev.bitmap ? 0 : 0xff, r.slots.bytes, st));
        break;
      case DQ_RES_AGG:
        if (!(fast && r.agg_clean)) {
          DQ_CUDA(launch_agg_init(r.dev.slots, r.dev.cap + 1, r.dev.words, r.dev.val_word, r.dev.naggs, r.dev.agg_red, st));
          ++launches;
        }
        r.agg_clean = false;
        break;
      case DQ_RES_MULTI:
        DQ_CUDA(cudaMemsetAsync(r.counts.ptr, 0, r.counts.bytes, st));
        break;
      default:
        break;
    }
  }
  if (dag) DQ_CUDA(cudaEventRecord(plan->fork_ev, st));
  const cudaStream_t origin = st;
  uint32_t* counters = plan->counters;
  for (size_t i = 0; i < np; ++i) {
    PipeRec& p = *plan->pipes[i];
    p.dev.tile_counter = counters + 2 * i;
    p.dev.clear_src = fast && p.clears_source ? 1 : 0;
    if (dag) {
      const int lane = lane_of[i];
      st = lane_stream(lane);
      if (lane && !lane_forked[(size_t)lane]) {
        DQ_CUDA(cudaStreamWaitEvent(st, plan->fork_ev, 0));
        lane_forked[(size_t)lane] = true;
      }
      if (p.fused_into < 0)
        for (int d : deps[i])
          if (lane_of[(size_t)d] != lane) DQ_CUDA(cudaStreamWaitEvent(st, plan->events[2 + 2 * (size_t)d], 0));
      lane_last[(size_t)lane] = (int)i;
    }
    DQ_CUDA(cudaEventRecord(plan->events[1 + 2 * i], st));
    if (p.expand_op >= 0) {
      DQ_CUDA(cudaMemsetAsync(p.heavy_count.ptr, 0, 8, st));
      if (p.dev.heavy.grouped) {
        DQ_CUDA(cudaMemsetAsync(p.heavy_gkey.ptr, 0xff, p.heavy_gkey.bytes, st));
        DQ_CUDA(cudaMemsetAsync(p.heavy_gcnt.ptr, 0, p.heavy_gcnt.bytes, st));
      }
    }
    if (p.fused_into >= 0) {
      // ran in the last CTA of pipeline fused_into's kernel
    } else if (p.jit) {
      DQ_CUDA(launch_generated(p.kernels.main, p.dev, p.grid, p.prog.block, p.prog.smem_bytes, st));
      ++launches;
    } else {
      DQ_CUDA(p.row ? launch_row(p.dev, p.grid, st) : launch_pipeline(p.dev, p.grid, st));
      ++launches;
    }
    if (p.expand_op >= 0) {
      if (p.dev.heavy.grouped) {
        DQ_CUDA(launch_heavy_group(p.dev.heavy, p.dev.status, plan->ctx->sms, st));
        launches += 2;  // units, prefix and scatter, in place of the item prefix
      } else {
        DQ_CUDA(launch_heavy_prefix(p.dev.heavy, (uint64_t)p.dev.exp_cap, p.dev.status, st));
      }
      DevPipe H = p.dev;
      H.mode = 1;
      H.tile_counter = counters + 2 * i + 1;
      if (p.jit) DQ_CUDA(launch_generated(p.kernels.heavy, H, p.grid_full, p.prog.block, p.prog.smem_bytes, st));
      else DQ_CUDA(launch_pipeline(H, p.grid_full, st));
      launches += 2;
      if (p.heavy_stats) DQ_CUDA(cudaMemcpyAsync(p.heavy_stats, p.heavy_count.ptr, 8, cudaMemcpyDeviceToHost, st));
    }
    if (p.mm_count) {
      ResRec& r = *plan->res[p.mm_res];
      DQ_CUDA(launch_mm_scan(r.dev.counts, r.dev.offsets, r.dev.cap, r.scan_scratch.as<uint32_t>(), st, &launches));
    }
    DQ_CUDA(cudaEventRecord(plan->events[2 + 2 * i], st));
  }
  st = origin;
  if (dag)
    for (int l = 1; l < kLanes; ++l)
      if (lane_last[(size_t)l] >= 0) DQ_CUDA(cudaStreamWaitEvent(st, plan->events[2 + 2 * (size_t)lane_last[(size_t)l]], 0));
  DQ_CUDA(cudaEventRecord(plan->events[2 * np + 1], st));
  DQ_CUDA(cudaMemcpyAsync(host_status, plan->status.ptr, 4, cudaMemcpyDeviceToHost, st));
  return launches;
}

// Device times of the last completed execution (its events have completed).
void collect_timing(dq_plan* plan, int launches) {
  const size_t np = plan->pipes.size();
  float ms = 0;
  dq_plan_timing& T = plan->timing;
  memset(&T, 0, sizeof(T));
  cudaEventElapsedTime(&ms, plan->events[0], plan->events[2 * np + 1]);
  T.total_ms = ms;
  T.max_pipeline = -1;
  for (size_t i = 0; i < np && i < (size_t)DQ_MAX_OPS; ++i) {
    cudaEventElapsedTime(&ms, plan->events[1 + 2 * i], plan->events[2 + 2 * i]);
    T.pipeline_ms[i] = ms;
    if (ms > T.max_pipeline_ms) {
      T.max_pipeline_ms = ms;
      T.max_pipeline = (int)i;
    }
  }
  T.kernel_launches = launches;
}

// One execution of all pipelines; returns the device status word.
// What a captured run depends on besides the plan's fixed buffers.
std::string graph_signature(const dq_plan* plan) {
  std::string sig;
  for (const auto& pp : plan->pipes) {
    const PipeRec& p = *pp;
    DevPipe d = p.dev;
    d.clear_src = p.clears_source ? 1 : 0;  // as enqueue_run sets them in fast mode
    sig.append(reinterpret_cast<const char*>(&d), sizeof(d));
    const int shape[4] = {p.grid, p.grid_full, p.prog.block, p.prog.smem_bytes};
    sig.append(reinterpret_cast<const char*>(shape), sizeof(shape));
  }
  for (const auto& rp : plan->res) {
    sig.push_back(rp->agg_clean ? 1 : 0);
    const void* bufs[3] = {rp->slots.ptr, rp->counts.ptr, rp->dev.cursor};
    sig.append(reinterpret_cast<const char*>(bufs), sizeof(bufs));
  }
  const cudaEvent_t* ev = plan->events.data();
  sig.append(reinterpret_cast<const char*>(ev), plan->events.size() * sizeof(cudaEvent_t));
  return sig;
}

// One execution of all pipelines; returns the device status word.  After a
// successful run the same launches replay from a captured graph (unless the
// context has DQ_CFG_NO_GRAPH).
int run_once(dq_plan* plan, cudaStream_t st) {
  if (!plan->host_status) DQ_CUDA(cudaMallocHost((void**)&plan->host_status, sizeof(int32_t)));
  *plan->host_status = 0;
  int launches = 0;
  bool graphs = !(plan->ctx->cfg.flags & DQ_CFG_NO_GRAPH) && plan->steady;
  if (graphs) {
    std::string sig = graph_signature(plan);
    if (plan->graph_exec && sig != plan->graph_sig) plan->drop_graph();
    if (!plan->graph_exec) ensure_lanes(plan);
    // a stream that cannot be captured (the legacy default stream) runs the launches directly
    if (!plan->graph_exec && cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
      cudaGetLastError();
      graphs = false;
    }
  }
  if (graphs) {
    if (!plan->graph_exec) {
      cudaGraph_t g = nullptr;
      try {
        plan->graph_launches = enqueue_run(plan, st, plan->host_status, true, true);
      } catch (...) {
        cudaStreamEndCapture(st, &g);
        if (g) cudaGraphDestroy(g);
        throw;
      }
      DQ_CUDA(cudaStreamEndCapture(st, &g));
      plan->graph = g;
      DQ_CUDA(cudaGraphInstantiate(&plan->graph_exec, plan->graph, 0));
      plan->graph_sig = graph_signature(plan);
    }
    for (auto& e : plan->graph_ev)
      if (!e) DQ_CUDA(cudaEventCreate(&e));
    DQ_CUDA(cudaEventRecord(plan->graph_ev[0], st));
    DQ_CUDA(cudaGraphLaunch(plan->graph_exec, st));
    DQ_CUDA(cudaEventRecord(plan->graph_ev[1], st));
    launches = plan->graph_launches;
  } else {
    launches = enqueue_run(plan, st, plan->host_status, true);
  }
  DQ_CUDA(cudaStreamSynchronize(st));
  const int32_t status = *plan->host_status;
  if (graphs) {
    // the whole run from the events around the launch; no per-pipeline times
    float ms = 0;
    memset(&plan->timing, 0, sizeof(plan->timing));
    cudaEventElapsedTime(&ms, plan->graph_ev[0], plan->graph_ev[1]);
    plan->timing.total_ms = ms;
    plan->timing.max_pipeline = -1;
    plan->timing.kernel_launches = launches;
  } else {
    collect_timing(plan, launches);
  }
  if ((status & ~kInfoMask) == 0) {
    // a completed run whose scans reset their aggregation tables leaves them clean
    for (auto& pp : plan->pipes)
      if (pp->clears_source) plan->res[pp->desc.source_res]->agg_clean = true;
    plan->steady = true;
  } else {
    plan->steady = false;
    plan->drop_graph();
  }
  return status;
}

// A result's string column: the n references a run left in device memory,
// gathered on the device through the plan's string sources into nrows + 1
// offsets and a heap, then copied to the host.
void gather_string_column(const dq_plan* plan, const uint64_t* refs, uint64_t n, cudaStream_t st,
                          std::vector<uint8_t>& offsets, std::vector<uint8_t>& heap_out) {
  DevBuf lens, offs, heap;
  lens.alloc(std::max<uint64_t>(n, 1) * 8);
  offs.alloc((n + 1) * 8);
  DQ_CUDA(launch_str_ref_offsets(refs, n, plan->str_src_dev.as<DevStr>(), lens.as<uint64_t>(), offs.as<uint64_t>(),
                                 plan->ctx->sms, st));
  offsets.resize((size_t)(n + 1) * 8);
  DQ_CUDA(cudaMemcpyAsync(offsets.data(), offs.ptr, (n + 1) * 8, cudaMemcpyDeviceToHost, st));
  DQ_CUDA(cudaStreamSynchronize(st));
  uint64_t total = 0;
  memcpy(&total, offsets.data() + n * 8, 8);
  heap.alloc(std::max<uint64_t>(total, 1));
  DQ_CUDA(launch_str_ref_copy(refs, n, plan->str_src_dev.as<DevStr>(), offs.as<uint64_t>(), heap.as<uint8_t>(),
                              plan->ctx->sms, st));
  heap_out.resize(total);
  if (total) DQ_CUDA(cudaMemcpyAsync(heap_out.data(), heap.ptr, total, cudaMemcpyDeviceToHost, st));
  DQ_CUDA(cudaStreamSynchronize(st));
}

// Result columns of a plan's OUTPUT resource whose n rows were copied to the
// host at `packed` + col_off[j] (fixed-width columns); string columns are
// gathered from the device references instead.
dq_result* packed_result(const dq_plan* plan, const uint8_t* packed, const std::vector<uint64_t>& col_off, uint64_t n,
                         cudaStream_t st) {
  const ResRec& o = *plan->res[plan->result_res];
  std::unique_ptr<dq_result> res(new dq_result());
  res->nrows = (int64_t)n;
  res->heaps.resize(o.desc.npay);
  for (int j = 0; j < o.desc.npay; ++j) {
    const int w = ctype_width(o.desc.pay_ctype[j]);
    res->ctypes.push_back(o.desc.pay_ctype[j]);
    if (o.desc.pay_ctype[j] == DQ_STR) {
      res->cols.emplace_back();
      gather_string_column(plan, reinterpret_cast<const uint64_t*>(o.dev.pay[j]), n, st, res->cols.back(),
                           res->heaps[j]);
      continue;
    }
    const uint8_t* src = packed + col_off[j];
    res->cols.emplace_back(src, src + (size_t)n * w);
  }
  return res.release();
}

// Copies a completed execution's result (OUTPUT resource) to the host.
dq_result* read_result(dq_plan* plan, cudaStream_t st) {
  ResRec& o = *plan->res[plan->result_res];
  uint64_t n = 0;
  DQ_CUDA(cudaMemcpyAsync(&n, o.dev.cursor, 8, cudaMemcpyDeviceToHost, st));
  DQ_CUDA(cudaStreamSynchronize(st));
  if (n > o.dev.cap) n = o.dev.cap;
  std::unique_ptr<dq_result> res(new dq_result());
  res->nrows = (int64_t)n;
  res->heaps.resize(o.desc.npay);
  for (int j = 0; j < o.desc.npay; ++j) {
    int w = ctype_width(o.desc.pay_ctype[j]);
    res->ctypes.push_back(o.desc.pay_ctype[j]);
    if (o.desc.pay_ctype[j] == DQ_STR) {
      res->cols.emplace_back();
      gather_string_column(plan, reinterpret_cast<const uint64_t*>(o.dev.pay[j]), n, st, res->cols.back(),
                           res->heaps[j]);
      continue;
    }
    res->cols.emplace_back((size_t)n * w);
    if (n) DQ_CUDA(cudaMemcpyAsync(res->cols.back().data(), o.dev.pay[j], (size_t)n * w, cudaMemcpyDeviceToHost, st));
  }
  DQ_CUDA(cudaStreamSynchronize(st));
  return res.release();
}

// Device bytes a plan holds (its tables, intermediates and scratch).
uint64_t plan_bytes(const dq_plan* plan) {
  uint64_t b = plan->status.bytes;
  for (auto& rp : plan->res) {
    const ResRec& r = *rp;
    b += r.slots.bytes + r.counts.bytes + r.offsets.bytes + r.scan_scratch.bytes;
    for (auto& p : r.pay) b += p->bytes;
  }
  for (auto& pp : plan->pipes) {
    b += pp->pattern_buf.bytes + pp->heavy_items.bytes + pp->heavy_count.bytes + pp->heavy_prefix.bytes;
    b += pp->heavy_gkey.bytes + pp->heavy_glen.bytes + pp->heavy_gcnt.bytes + pp->heavy_glist.bytes +
         pp->heavy_gstart.bytes + pp->heavy_sorted.bytes;
  }
  return b;
}

// Re-derives every pipeline's copy of the resource descriptors.
// Ordering: the string-source table is rewritten in place with a synchronous
// copy.  Every caller runs when none of the plan's work is in flight: at
// preparation, or when growing tables after a run whose stream the caller has
// synchronised (dq_plan_execute's run_once, a batch execute, a completed server
// slot).  Growing also frees the old device buffers, and cudaFree waits for the
// device as well.
void refresh_pipelines(dq_plan* plan) {
  plan->str_src.clear();
  // last pipeline first: a fused tail's descriptor is laid out before the
  // kernel that runs it is generated
  for (size_t i = plan->pipes.size(); i-- > 0;) setup_pipeline(plan, *plan->pipes[i]);
  // the string sources every pipeline may resolve references against
  const size_t n = plan->str_src.size();
  if (plan->str_src_dev.bytes != std::max<size_t>(n, 1) * sizeof(DevStr) || (!plan->str_src_dev.ptr && !t_offline))
    plan->str_src_dev.alloc(std::max<size_t>(n, 1) * sizeof(DevStr));
  if (n && !plan->ctx->offline && !t_offline)
    DQ_CUDA(cudaMemcpy(plan->str_src_dev.ptr, plan->str_src.data(), n * sizeof(DevStr), cudaMemcpyHostToDevice));
  for (auto& pp : plan->pipes) {
    pp->dev.strsrc = plan->str_src_dev.as<DevStr>();
    pp->dev.nstrsrc = (int32_t)n;
  }
  // fused tails: their descriptors where the kernels that run them read them
  // (they always reset the aggregation table they scan: they are its only scan)
  for (size_t i = 0; i < plan->pipes.size(); ++i) {
    PipeRec& p = *plan->pipes[i];
    if (p.tail < 0) continue;
    PipeRec& t = *plan->pipes[p.tail];
    t.dev.clear_src = 1;
    t.dev.tile_counter = plan->counters + 2 * p.tail;
    if (!p.tail_buf.ptr || p.tail_buf.bytes != sizeof(DevPipe)) p.tail_buf.alloc(sizeof(DevPipe));
    if (!plan->ctx->offline && !t_offline)
      DQ_CUDA(cudaMemcpy(p.tail_buf.ptr, &t.dev, sizeof(DevPipe), cudaMemcpyHostToDevice));
    p.dev.tail = p.tail_buf.as<DevPipe>();
  }
}

// Whether pipeline k's kernel can run pipeline k + 1 in its last CTA: k
// aggregates into a table of at most kTailSlots slots that k + 1 alone scans,
// with scalar ops and filters into an emit sink, and k defers no expansion.
// One CTA scans the table: at 40,000 slots (the Q16- and Q21-shaped results)
// that took 0.08-0.18 ms, far more than the launch it saves.
constexpr uint64_t kTailSlots = 8192;
bool fusable_tail(const dq_plan_desc* desc, const std::vector<std::unique_ptr<ResRec>>& res, int k) {
  const dq_pipeline& a = desc->pipes[k];
  const dq_pipeline& b = desc->pipes[k + 1];
  if (a.nops <= 0 || b.nops <= 0) return false;
  const dq_op& sink = a.ops[a.nops - 1];
  if (sink.kind != DQ_OP_AGG || b.source_kind != DQ_SRC_AGG || b.source_res != sink.res) return false;
  if (sink.res < 0 || sink.res >= (int)res.size() || res[sink.res]->dev.cap + 1 > kTailSlots) return false;
  for (int i = 0; i < a.nops; ++i)
    if (a.ops[i].kind == DQ_OP_EXPAND) return false;
  for (int i = 0; i < b.nops; ++i) {
    const int kd = b.ops[i].kind;
    const bool ok = kd == DQ_OP_ARITH || kd == DQ_OP_CMP || kd == DQ_OP_LOGIC || kd == DQ_OP_CAST ||
                    kd == DQ_OP_SELECT || kd == DQ_OP_FILTER || (kd == DQ_OP_EMIT && i == b.nops - 1);
    if (!ok) return false;
  }
  for (int i = 0; i < desc->npipes; ++i)
    if (i != k + 1 && desc->pipes[i].source_kind == DQ_SRC_AGG && desc->pipes[i].source_res == sink.res) return false;
  return true;
}

// Unique tables over a small key domain need no hashing: one key, read
// straight from a column of a registered table by the one pipeline that builds
// the table, whose smallest and largest values (measured on the device at
// preparation) span few keys.
// - No payload: a bit per key, for at most kBitmapKeys keys, or at most
//   kDenseKeys keys and at most 64 per row of the build table.  A probe is one
//   bit test (in shared memory for the generated kernels when the bits fit
//   kBitmapKeys, else a 4-byte load of a table of at most 2 MB).
// - One payload of at most 32 bits, at most kDenseKeys keys and at most four
//   per row of the build table: a word per key.  A probe is one 8-byte load.
constexpr uint64_t kBitmapKeys = 1ull << 18;  // 32 KB of bits
constexpr uint64_t kDenseKeys = 1ull << 24;   // 128 MB of words, 2 MB of bits

void choose_bitmap(dq_ctx* ctx, const dq_plan_desc* desc, int i, ResRec& r) {
  const dq_resource& d = desc->res[i];
  if (d.kind != DQ_RES_UNIQUE || d.nkeys != 1 || d.npay > 1 || r.no_bitmap) return;
  if (d.npay == 1 && (d.pay_ctype[0] == DQ_STR || ctype_width(d.pay_ctype[0]) > 4)) return;
  const int kt = d.key_ctype[0];
  if (kt != DQ_I8 && kt != DQ_I32 && kt != DQ_U32 && kt != DQ_I64) return;
  const dq_pipeline* build = nullptr;
  for (int p = 0; p < desc->npipes; ++p) {
    const dq_pipeline& pd = desc->pipes[p];
    if (pd.nops <= 0 || pd.nops > DQ_MAX_OPS) return;
    for (int k = 0; k < pd.nops; ++k) {
      const dq_op& op = pd.ops[k];
      // ops whose `res` names a resource (LIKE, STREQ and PROFILE use it otherwise)
      const bool uses_res = op.kind == DQ_OP_PROBE || op.kind == DQ_OP_EXPAND || op.kind == DQ_OP_EXISTS ||
                            op.kind >= DQ_OP_AGG;
      if (!uses_res || op.res != i) continue;
      if (op.kind == DQ_OP_BUILD && k == pd.nops - 1) {
        if (build) return;
        build = &pd;
      } else if (op.kind != DQ_OP_PROBE || op.nlist != 1) {
        return;
      }
    }
  }
  if (!build || build->source_kind != DQ_SRC_TABLE || !build->table) return;
  const dq_op& sink = build->ops[build->nops - 1];
  if (sink.nlist != 1 || sink.nlist2 != d.npay || sink.list < 0 || sink.list >= build->nlist) return;
  const int ks = build->lists[sink.list];
  if (ks < 0 || ks >= build->nslots || build->slots[ks].kind != DQ_SLOT_COL) return;
  const int ci = build->slots[ks].src;
  if (ci < 0 || ci >= build->ncols || !build->cols[ci]) return;
  auto t = ctx->tables.find(build->table);
  if (t == ctx->tables.end() || t->second.nrows <= 0) return;
  const ColRec* c = t->second.find(build->cols[ci]);
  // the key is the column's value unchanged: same type in the slot and the table
  if (!c || c->ctype != kt || build->slots[ks].ctype != kt || !c->data || !c->data->ptr) return;
  DevBuf mm;
  mm.alloc(16);
  const long long init[2] = {LLONG_MAX, LLONG_MIN};
  DQ_CUDA(cudaMemcpy(mm.ptr, init, 16, cudaMemcpyHostToDevice));
  DQ_CUDA(launch_col_minmax(c->data->as<uint8_t>(), (uint64_t)t->second.nrows, ctype_width(c->ctype),
                            kt != DQ_U32, mm.as<long long>(), ctx->sms, ctx->stream));
  long long got[2];
  DQ_CUDA(cudaMemcpyAsync(got, mm.ptr, 16, cudaMemcpyDeviceToHost, ctx->stream));
  DQ_CUDA(cudaStreamSynchronize(ctx->stream));
  if (got[0] > got[1]) return;
  const uint64_t span = (uint64_t)got[1] - (uint64_t)got[0] + 1;  // 0: all 2^64 values
  const uint64_t rows = (uint64_t)t->second.nrows;
  if (span == 0 || span > kDenseKeys || (d.npay == 0 ? span > kBitmapKeys && span > 64 * rows : span > 4 * rows))
    return;
  r.bitmap = d.npay == 0 ? 1 : 2;
  r.bmin = got[0];
  r.brange = span;
}

// Lays out a plan's resources and pipelines (the caller holds the context lock
// and has made the device current).
std::unique_ptr<dq_plan> make_plan(dq_ctx* ctx, const dq_plan_desc* desc, const PlanOpts& opts) {
  if (desc->abi_version != DQ_ABI_VERSION) throw DqError(DQ_ERR_BAD_IR, "IR version mismatch");
  if (desc->nres < 0 || desc->npipes <= 0 || (desc->nres && !desc->res) || !desc->pipes)
    throw DqError(DQ_ERR_BAD_IR, "empty plan");
  std::unique_ptr<dq_plan> plan(new dq_plan());
  plan->ctx = ctx;
  plan->opts = opts;
  for (int i = 0; i < desc->npipes; ++i)
    for (int k = 0; k < desc->pipes[i].nops && k < DQ_MAX_OPS; ++k)
      if (desc->pipes[i].ops[k].kind == DQ_OP_PROFILE) {
        const int r = desc->pipes[i].ops[k].res;
        if (r < 0 || r >= 1024) throw DqError(DQ_ERR_BAD_IR, "profile point out of range");
        plan->nprofile = std::max(plan->nprofile, r + 1);
      }
  const size_t ctrl = 8 + 8 * (size_t)desc->npipes + 8 * (size_t)std::max(desc->nres, 0);
  plan->status.alloc(ctrl + 33 * 8 * (size_t)plan->nprofile);
  if (plan->status.ptr) {
    plan->counters = reinterpret_cast<uint32_t*>(plan->status.as<uint8_t>() + 8);
    plan->cursors = reinterpret_cast<uint64_t*>(plan->status.as<uint8_t>() + 8 + 8 * (size_t)desc->npipes);
    if (plan->nprofile) plan->profile = reinterpret_cast<uint64_t*>(plan->status.as<uint8_t>() + ctrl);
  }
  // row bound for multimap payloads: rows of the source of the pipeline that scatters into it
  std::vector<int64_t> bound(desc->nres, 1);
  for (int i = 0; i < desc->npipes; ++i) {
    const dq_pipeline& d = desc->pipes[i];
    if (d.nops <= 0 || d.nops > DQ_MAX_OPS) throw DqError(DQ_ERR_BAD_IR, "bad op count");
    const dq_op& sink = d.ops[d.nops - 1];
    if ((sink.kind == DQ_OP_MM_SCATTER || sink.kind == DQ_OP_MM_COUNT) && sink.res >= 0 && sink.res < desc->nres) {
      int64_t rows = 1 << 20;
      if (d.source_kind == DQ_SRC_TABLE && d.table) {
        auto it = ctx->tables.find(d.table);
        if (it != ctx->tables.end()) rows = it->second.nrows;
      } else if (d.source_kind == DQ_SRC_OUTPUT && d.source_res >= 0 && d.source_res < desc->nres) {
        rows = desc->res[d.source_res].capacity;
      }
      bound[sink.res] = std::max(bound[sink.res], rows);
    }
  }
  for (int i = 0; i < desc->nres; ++i) {
    std::unique_ptr<ResRec> r(new ResRec());
    r->index = i;
    r->desc = desc->res[i];
    r->name = desc->res[i].name ? desc->res[i].name : "";
    r->desc.name = nullptr;
    if (!(ctx->cfg.flags & (DQ_CFG_NO_JIT | DQ_CFG_ROW_KERNEL)) && !ctx->offline && !t_offline)
      choose_bitmap(ctx, desc, i, *r);
    setup_resource(plan.get(), *r, bound[i]);
    plan->res.push_back(std::move(r));
  }
  for (int i = 0; i < desc->npipes; ++i) {
    std::unique_ptr<PipeRec> p(new PipeRec());
    p->desc = desc->pipes[i];
    // keep string arguments alive
    for (int c = 0; c < p->desc.ncols; ++c) p->col_names.push_back(p->desc.cols[c] ? p->desc.cols[c] : "");
    for (int c = 0; c < p->desc.ncols; ++c) p->desc.cols[c] = p->col_names[c].c_str();
    p->desc.table = nullptr;
    std::string tname = desc->pipes[i].table ? desc->pipes[i].table : "";
    p->col_names.push_back(tname);
    p->desc.table = p->col_names.back().c_str();
    for (int c = 0; c < p->desc.npatterns; ++c) p->patterns.push_back(p->desc.patterns[c] ? p->desc.patterns[c] : "");
    for (int c = 0; c < p->desc.npatterns; ++c) p->desc.patterns[c] = p->patterns[c].c_str();
    plan->pipes.push_back(std::move(p));
  }
  // the col_names vector may have reallocated: re-point
  for (auto& p : plan->pipes) {
    for (int c = 0; c < p->desc.ncols; ++c) p->desc.cols[c] = p->col_names[c].c_str();
    p->desc.table = p->col_names.back().c_str();
    for (int c = 0; c < p->desc.npatterns; ++c) p->desc.patterns[c] = p->patterns[c].c_str();
  }
  // the last CTA of an aggregating kernel runs the small scan that follows it
  const bool generated = !(ctx->cfg.flags & (DQ_CFG_NO_JIT | DQ_CFG_ROW_KERNEL)) && !opts.batch_member;
  if (generated)
    for (int k = 0; k + 1 < desc->npipes; ++k)
      if (plan->pipes[k]->fused_into < 0 && fusable_tail(desc, plan->res, k)) {
        plan->pipes[k]->tail = k + 1;
        plan->pipes[k + 1]->fused_into = k;
      }
  refresh_pipelines(plan.get());
  // an aggregation table that one generated pipeline alone scans is reset by that scan
  std::vector<int> scans(desc->nres, 0);
  for (auto& p : plan->pipes)
    if (p->desc.source_kind == DQ_SRC_AGG && p->desc.source_res >= 0 && p->desc.source_res < desc->nres)
      ++scans[p->desc.source_res];
  for (auto& p : plan->pipes)
    p->clears_source = p->jit && p->desc.source_kind == DQ_SRC_AGG && p->desc.source_res >= 0 &&
                       p->desc.source_res < desc->nres && scans[p->desc.source_res] == 1;
  plan->result_res = desc->result_res;
  if (plan->result_res < 0 || plan->result_res >= desc->nres || plan->res[plan->result_res]->desc.kind != DQ_RES_OUTPUT)
    throw DqError(DQ_ERR_BAD_IR, "result must be an OUTPUT resource");
  return plan;
}

// Grows the tables a failed run overflowed (device status bits) and re-derives
// the pipelines' descriptors.
void grow_plan(dq_plan* plan, int status) {
  for (auto& rp : plan->res) {
    ResRec& r = *rp;
    if ((status & kErrKeyRange) && r.bitmap && !r.no_bitmap) {
      // the table's data changed since preparation: a hash table from now on
      r.no_bitmap = true;
      setup_resource(plan, r, 1);
      continue;
    }
    if ((status & kErrHtFull) && (r.desc.kind == DQ_RES_UNIQUE || r.desc.kind == DQ_RES_AGG)) {
      // four times the slots (join tables are sized at unique_pct of the capacity)
      const int64_t pct = r.desc.kind == DQ_RES_UNIQUE ? r.pct : 100;
      r.desc.capacity = (int64_t)r.dev.cap * 4 * 100 / pct;
      setup_resource(plan, r, 1);
    }
    if ((status & kErrOverflow) && r.desc.kind == DQ_RES_OUTPUT) {
      uint64_t need = 0;
      DQ_CUDA(cudaMemcpy(&need, r.dev.cursor, 8, cudaMemcpyDeviceToHost));
      if (need > r.dev.cap) {
        r.desc.capacity = (int64_t)need;
        setup_resource(plan, r, 1);
      }
    }
  }
  refresh_pipelines(plan);
}

// After a run whose deferred expansion items overflowed (kInfoHeavyFull; its
// results are exact, the overflowing rows were expanded in place, which is
// slow for long ranges): twice the items the run wanted, for the runs that
// follow.  Returns whether the plan's buffers moved.
bool grow_heavy(dq_plan* plan) {
  bool moved = false;
  for (auto& pp : plan->pipes) {
    PipeRec& p = *pp;
    if (p.expand_op < 0) continue;
    uint32_t n = 0;
    DQ_CUDA(cudaMemcpy(&n, p.heavy_count.ptr, 4, cudaMemcpyDeviceToHost));
    if (n > p.dev.heavy.cap) {
      p.heavy_cap = std::min<uint64_t>(2ull * n, 0xffffffffull);
      moved = true;
    }
  }
  if (moved) refresh_pipelines(plan);
  return moved;
}

// Deferral pays when several probe rows match the same range (its chunks are
// gathered once for all of them); with one probe row per range it only adds
// passes.  After a completed run: items per group of 4 or more lower a plan's
// threshold to kGroupThresholdLow for the runs that follow, fewer than 2 raise
// it back (the runs' results do not depend on it).
void adapt_threshold(dq_plan* plan) {
  if (plan->ctx->cfg.defer_threshold > 0 || plan->opts.defer_threshold > 0) return;
  for (auto& pp : plan->pipes) {
    PipeRec& p = *pp;
    if (p.expand_op < 0 || !p.heavy_stats || !p.dev.heavy.grouped) continue;
    const uint64_t items = std::min<uint64_t>(p.heavy_stats[0], p.dev.heavy.cap), groups = p.heavy_stats[1];
    if (groups == 0) continue;
    uint64_t t = p.dev.heavy.threshold;
    if (items >= 4 * groups) t = kGroupThresholdLow;
    else if (items < 2 * groups) t = kGroupThreshold;
    p.heavy_threshold = t;
    p.dev.heavy.threshold = t;
  }
}

void throw_status(int status) {
  throw DqError(status & kErrTimeout ? DQ_ERR_TIMEOUT
                : status & kErrHtFull ? DQ_ERR_HT_FULL
                : status & kErrOverflow ? DQ_ERR_OVERFLOW : DQ_ERR_BAD_IR,
                "device status " + std::to_string(status));
}

jit::Tuning tuning_of(const dq_tuning* t) {
  jit::Tuning j;
  if (t) {
    j.rows_per_thread = t->rows_per_thread;
    j.block = t->block_threads;
    j.refill = t->refill;
    j.refill_threshold = t->refill_threshold;
    // resident CTAs asked for: the kernels' register budget must let them fit
    if (t->ctas_per_sm > 0 && t->ctas_per_sm <= 8) j.min_blocks = t->ctas_per_sm;
  }
  return j;
}

PlanOpts opts_of(const dq_tuning* t) {
  PlanOpts o;
  o.tuning = tuning_of(t);
  if (t && t->unique_slots_pct > 0) o.unique_pct = t->unique_slots_pct;
  if (t && t->multi_buckets_pct > 0) o.multi_pct = t->multi_buckets_pct;
  if (t && t->defer_threshold > 0) o.defer_threshold = t->defer_threshold;
  if (t && t->ctas_per_sm > 0) o.ctas_per_sm = t->ctas_per_sm;
  return o;
}

// ---------------------------------------------------------------- batches --

template <class T>
void upload(DevBuf& buf, const std::vector<T>& v) {
  buf.alloc(std::max<size_t>(v.size(), 1) * sizeof(T));
  if (!v.empty()) DQ_CUDA(cudaMemcpy(buf.ptr, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice));
}

// (Re)builds the batch's kernels, descriptors and CUDA graph from its
// instance plans (after preparation and after tables grew).
// Deferred-expansion buffers of batch stage `p`, shared by all instances: items
// of any instance, grouped by (instance, range).  Sized by the instances'
// probe rows (at most 2^20 items, or what an overflow asked for) and their
// build rows.
void setup_batch_heavy(dq_batch* b, size_t p, BatchStage& S) {
  const PipeRec& p0 = *b->inst[0]->pipes[p];
  DevHeavy H = p0.dev.heavy;
  int64_t rows = 0;
  uint64_t build_rows = 0;
  for (int i = 0; i < b->ninst; ++i) {
    const dq_plan& pl = *b->inst[i];
    const PipeRec& pi = *pl.pipes[p];
    rows += pi.dev.nrows_dev ? (int64_t)pl.res[pi.dev.source_res]->dev.cap : pi.dev.nrows;
    build_rows += std::max<uint64_t>(pl.res[pi.desc.ops[pi.expand_op].res]->pay_rows, 1);
  }
  H.grouped = 1;
  H.cap = (uint32_t)std::min<int64_t>(std::max<int64_t>(rows, 1),
                                      std::max<int64_t>(1 << 20, (int64_t)b->heavy_cap));
  const uint64_t groups = std::min<uint64_t>(
      H.cap, build_rows / ((b->inst[0]->opts.defer_threshold > 0 ? H.threshold
                                                                   : std::max<uint64_t>(H.threshold, kBatchGroupThreshold)) +
                           1) +
                 (uint64_t)b->ninst);
  H.gcap = (uint32_t)std::min<uint64_t>(std::max<uint64_t>(64, 2 * groups), 0xfffffff0ull);
  S.h_items.alloc((size_t)H.cap * H.words * 8);
  S.h_count.alloc(8);
  S.h_units.alloc(4);
  S.h_gkey.alloc((size_t)H.gcap * 8);
  S.h_glen.alloc((size_t)H.gcap * 4);
  S.h_gcnt.alloc((size_t)H.gcap * 4);
  S.h_glist.alloc((size_t)H.gcap * 4);
  S.h_gstart.alloc(((size_t)H.gcap + 1) * 4);
  S.h_sorted.alloc((size_t)H.cap * std::max(H.nstash, 1) * 8);
  S.h_prefix.alloc((std::max<size_t>(H.cap, H.gcap) + 1) * 8);
  H.items = S.h_items.as<uint64_t>();
  H.count = S.h_count.as<uint32_t>();
  H.ngroups = S.h_count.as<uint32_t>() + 1;
  H.unit_prefix = S.h_prefix.as<uint64_t>();
  H.gkey = S.h_gkey.as<uint64_t>();
  H.glen = S.h_glen.as<uint32_t>();
  H.gcnt = S.h_gcnt.as<uint32_t>();
  H.glist = S.h_glist.as<uint32_t>();
  H.gstart = S.h_gstart.as<uint32_t>();
  H.sorted = S.h_sorted.as<uint64_t>();
  S.heavy = H;
}

void build_batch(dq_batch* b, const jit::Tuning& tuning, cudaStream_t st) {
  dq_ctx* ctx = b->ctx;
  const dq_plan& first = *b->inst[0];
  const size_t np = first.pipes.size();
  b->stages.clear();
  b->launches = 0;
  for (size_t p = 0; p < np; ++p) {
    b->stages.emplace_back(new BatchStage());
    BatchStage& S = *b->stages[p];
    jit::Tuning t = tuning;
    t.batched = true;
    const PipeRec& p0 = *first.pipes[p];
    S.prog = jit::generate(p0.dev, p0.expand_op, p0.desc.compact - 1, t);
    for (int i = 1; i < b->ninst; ++i) {
      const PipeRec& pi = *b->inst[i]->pipes[p];
      if (pi.expand_op != p0.expand_op ||
          jit::generate(pi.dev, pi.expand_op, pi.desc.compact - 1, t).source != S.prog.source)
        throw DqError(DQ_ERR_BAD_IR, "batch instance " + std::to_string(i) + " differs in shape from instance 0");
    }
    S.kernels = jit::compile(S.prog, !ctx->offline);
    if (ctx->offline) continue;
    if (p0.expand_op >= 0) setup_batch_heavy(b, p, S);
    std::vector<DevPipe> descs(b->ninst);
    std::vector<int64_t> prefix(b->ninst + 1, 0);
    const int64_t span = (int64_t)S.prog.block * S.prog.rows_per_thread;
    for (int i = 0; i < b->ninst; ++i) {
      const dq_plan& pl = *b->inst[i];
      descs[i] = pl.pipes[p]->dev;
      descs[i].status = b->status.as<int32_t>();
      if (p0.expand_op >= 0) {
        const uint64_t threshold = pl.opts.defer_threshold > 0
                                       ? (uint64_t)pl.opts.defer_threshold
                                       : std::max<uint64_t>(descs[i].heavy.threshold, kBatchGroupThreshold);
        descs[i].heavy = S.heavy;
        descs[i].heavy.threshold = threshold;
        descs[i].tile_counter = S.h_units.as<uint32_t>();
      }
      int64_t rows = descs[i].nrows;
      if (descs[i].nrows_dev) rows = (int64_t)pl.res[descs[i].source_res]->dev.cap;  // temp table: its capacity
      prefix[i + 1] = prefix[i] + (rows + span - 1) / span;
    }
    upload(S.descs, descs);
    upload(S.bprefix, prefix);
    const void* fn = (const void*)S.kernels.main;
    DQ_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, S.prog.smem_bytes));
    int occ = 0;
    DQ_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, fn, S.prog.block, S.prog.smem_bytes));
    if (occ < 1) throw DqError(DQ_ERR_UNSUPPORTED, "batched pipeline kernel cannot be resident");
    S.grid = (int)std::max<int64_t>(1, std::min<int64_t>((int64_t)ctx->sms * occ, prefix[b->ninst]));
    if (S.kernels.heavy) {
      const void* hf = (const void*)S.kernels.heavy;
      DQ_CUDA(cudaFuncSetAttribute(hf, cudaFuncAttributeMaxDynamicSharedMemorySize, S.prog.smem_bytes));
      int hocc = 0;
      DQ_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&hocc, hf, S.prog.block, S.prog.smem_bytes));
      S.heavy_grid = ctx->sms * std::max(hocc, 1);
    }
    S.mm_scan = p0.mm_count;
    if (S.mm_scan) {
      std::vector<BatchScanSeg> segs(b->ninst);
      uint64_t blocks = 0;
      for (int i = 0; i < b->ninst; ++i) {
        const DevRes& R = b->inst[i]->res[p0.mm_res]->dev;
        segs[i].counts = R.counts;
        segs[i].offsets = R.offsets;
        segs[i].n = R.cap;
        segs[i].block0 = blocks;
        segs[i].nblocks = batch_scan_blocks(R.cap);
        blocks += segs[i].nblocks;
      }
      upload(S.segs, segs);
      S.partials.alloc(std::max<uint64_t>(blocks, 1) * 4);
      S.nsegs = b->ninst;
      S.scan_blocks = blocks;
    }
  }
  if (ctx->offline) return;
  // resets of every instance's tables, in one launch
  std::vector<BatchReset> resets;
  for (int i = 0; i < b->ninst; ++i)
    for (auto& rp : b->inst[i]->res) {
      const ResRec& r = *rp;
      BatchReset op{};
      switch (r.desc.kind) {
        case DQ_RES_UNIQUE:
          if (r.dev.bitmap) op.ptr = r.dev.slots, op.n = r.dev.bitmap == 1 ? (r.dev.cap * 4 + 7) / 8 : r.dev.cap,
                            op.value = 0, op.kind = 0;
          else op.ptr = r.dev.slots, op.n = (r.dev.cap + 1) * r.dev.words, op.value = kEmpty, op.kind = 0;
          break;
        case DQ_RES_AGG:
          op.ptr = r.dev.slots, op.n = r.dev.cap + 1, op.kind = 2, op.words = r.dev.words;
          op.val_word = r.dev.val_word, op.naggs = r.dev.naggs;
          for (int j = 0; j < r.dev.naggs && j < 16; ++j) op.reds |= (uint64_t)(r.dev.agg_red[j] & 15) << (4 * j);
          break;
        case DQ_RES_MULTI:
          op.ptr = r.dev.counts, op.n = r.dev.cap, op.value = 0, op.kind = 1;
          break;
        case DQ_RES_OUTPUT:
          op.ptr = r.dev.cursor, op.n = 1, op.value = 0, op.kind = 0;
          break;
      }
      resets.push_back(op);
    }
  upload(b->resets, resets);
  b->nresets = (int)resets.size();
  // results: every instance's output columns packed into one buffer
  std::vector<BatchPack> packs;
  b->col_off.assign(b->ninst, std::vector<uint64_t>());
  uint64_t off = 0;
  b->rows.alloc((size_t)b->ninst * 8);
  for (int i = 0; i < b->ninst; ++i) {
    const ResRec& o = *b->inst[i]->res[b->inst[i]->result_res];
    for (int j = 0; j < o.desc.npay; ++j) {
      BatchPack pk{};
      pk.src = o.dev.pay[j];
      pk.cursor = o.dev.cursor;
      pk.cap = o.dev.cap;
      pk.width = ctype_width(o.desc.pay_ctype[j]);
      pk.dst = off;
      pk.rows_out = j == 0 ? b->rows.as<uint64_t>() + i : nullptr;
      b->col_off[i].push_back(off);
      off += align_up(o.dev.cap * (uint64_t)pk.width, 16);
      packs.push_back(pk);
    }
    if (o.desc.npay == 0) throw DqError(DQ_ERR_BAD_IR, "batch results need at least one column");
  }
  upload(b->packs, packs);
  b->npacks = (int)packs.size();
  b->packed_bytes = std::max<uint64_t>(off, 16);
  b->packed.alloc(b->packed_bytes);
  if (b->host) cudaFreeHost(b->host);
  b->host = nullptr;
  DQ_CUDA(cudaMallocHost((void**)&b->host, b->packed_bytes + (size_t)b->ninst * 8 + 16));
  // the whole run as one CUDA graph
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  b->exec = nullptr;
  b->graph = nullptr;
  DQ_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
  cudaError_t err = cudaSuccess;
  auto rec = [&](cudaError_t e) {
    if (err == cudaSuccess && e != cudaSuccess) err = e;
  };
  rec(cudaMemsetAsync(b->status.ptr, 0, 4, st));
  rec(launch_batch_reset(b->resets.as<BatchReset>(), b->nresets, ctx->sms, st));
  int launches = 1;
  for (auto& Sp : b->stages) {
    BatchStage& S = *Sp;
    const DevPipe* d = S.descs.as<DevPipe>();
    const int64_t* pre = S.bprefix.as<int64_t>();
    int n = b->ninst;
    void* args[] = {(void*)&d, (void*)&pre, (void*)&n};
    if (S.kernels.heavy) {
      rec(cudaMemsetAsync(S.h_count.ptr, 0, S.h_count.bytes, st));
      rec(cudaMemsetAsync(S.h_units.ptr, 0, S.h_units.bytes, st));
      rec(cudaMemsetAsync(S.h_gkey.ptr, 0xff, S.h_gkey.bytes, st));
      rec(cudaMemsetAsync(S.h_gcnt.ptr, 0, S.h_gcnt.bytes, st));
    }
    rec(cudaLaunchKernel((const void*)S.kernels.main, dim3(S.grid), dim3(S.prog.block), args,
                         (size_t)S.prog.smem_bytes, st));
    ++launches;
    if (S.kernels.heavy) {
      rec(launch_heavy_group(S.heavy, b->status.as<int32_t>(), ctx->sms, st));
      void* hargs[] = {(void*)&d, (void*)&n};
      rec(cudaLaunchKernel((const void*)S.kernels.heavy, dim3(S.heavy_grid), dim3(S.prog.block), hargs,
                           (size_t)S.prog.smem_bytes, st));
      launches += 4;
    }
    if (S.mm_scan) {
      rec(launch_batch_scan(S.segs.as<BatchScanSeg>(), S.nsegs, S.scan_blocks, S.partials.as<uint32_t>(), st));
      launches += 3;
    }
  }
  rec(launch_batch_pack(b->packs.as<BatchPack>(), b->npacks, b->packed.as<uint8_t>(), ctx->sms, st));
  ++launches;
  rec(cudaMemcpyAsync(b->host, b->packed.ptr, b->packed_bytes, cudaMemcpyDeviceToHost, st));
  rec(cudaMemcpyAsync(b->host + b->packed_bytes, b->rows.ptr, (size_t)b->ninst * 8, cudaMemcpyDeviceToHost, st));
  rec(cudaMemcpyAsync(b->host + b->packed_bytes + (size_t)b->ninst * 8, b->status.ptr, 4, cudaMemcpyDeviceToHost, st));
  cudaGraph_t g = nullptr;
  cudaError_t end = cudaStreamEndCapture(st, &g);
  DQ_CUDA(err);
  DQ_CUDA(end);
  b->graph = g;
  DQ_CUDA(cudaGraphInstantiate(&b->exec, b->graph, 0));
  b->launches = launches;
}

}  // namespace

// ====================================================================== ABI ==

extern "C" {

int dq_version(void) { return DQ_ABI_VERSION; }

const char* dq_last_error(dq_ctx* ctx) { return ctx ? ctx->error.c_str() : g_init_error.c_str(); }

int dq_init(const dq_config* cfg, dq_ctx** out) {
  if (!out) return fail(nullptr, DQ_ERR_INVALID, "null output");
  *out = nullptr;
  return guarded(nullptr, [&]() {
    std::unique_ptr<dq_ctx> ctx(new dq_ctx());
    if (cfg) {
      if (cfg->abi_version != DQ_ABI_VERSION) throw DqError(DQ_ERR_INVALID, "ABI version mismatch");
      ctx->cfg = *cfg;
    }
    ctx->device = ctx->cfg.device;
    if (ctx->cfg.flags & DQ_CFG_OFFLINE) {
      ctx->offline = true;  // 148 SMs assumed for launch shapes; nothing touches a device
      *out = ctx.release();
      return (int)DQ_OK;
    }
    int n = 0;
    DQ_CUDA(cudaGetDeviceCount(&n));
    if (ctx->device < 0 || ctx->device >= n) throw DqError(DQ_ERR_INVALID, "no such CUDA device");
    DQ_CUDA(cudaSetDevice(ctx->device));
    DQ_CUDA(cudaDeviceGetAttribute(&ctx->sms, cudaDevAttrMultiProcessorCount, ctx->device));
    DQ_CUDA(cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking));
    *out = ctx.release();
    return (int)DQ_OK;
  });
}

void dq_shutdown(dq_ctx* ctx) {
  if (!ctx) return;
  if (ctx->offline) {
    delete ctx;
    return;
  }
  cudaSetDevice(ctx->device);
  ctx->tables.clear();
  if (ctx->stream) cudaStreamDestroy(ctx->stream);
  delete ctx;
}

int dq_table_register(dq_ctx* ctx, const char* name, int32_t ncols, const dq_column* cols, int64_t nrows,
                      int32_t flags) {
  if (!ctx || !name || (ncols > 0 && !cols) || nrows < 0 || ncols < 0) return fail(ctx, DQ_ERR_INVALID, "bad table arguments");
  return guarded(ctx, [&]() {
    std::lock_guard<std::mutex> lk(ctx->mu);
    OfflineScope offline(ctx->offline);
    if (!ctx->offline) DQ_CUDA(cudaSetDevice(ctx->device));
    TableRec t;
    t.nrows = nrows;
    for (int i = 0; i < ncols; ++i) {
      const dq_column& c = cols[i];
      if (!c.name || c.ctype < DQ_I8 || c.ctype > DQ_STR) throw DqError(DQ_ERR_INVALID, "bad column descriptor");
      if (nrows > 0 && !c.data) throw DqError(DQ_ERR_INVALID, std::string("column ") + c.name + " has no data");
      ColRec rec;
      rec.name = c.name;
      rec.ctype = c.ctype;
      rec.width = c.ctype == DQ_STR ? c.width : ctype_width(c.ctype);
      upload_column(ctx, rec, c, nrows, flags & DQ_TABLE_DEVICE_DATA, ctx->stream);
      t.cols.push_back(std::move(rec));
    }
    if (!ctx->offline) DQ_CUDA(cudaStreamSynchronize(ctx->stream));
    ctx->tables[name] = std::move(t);
    return (int)DQ_OK;
  });
}

int dq_table_update(dq_ctx* ctx, const char* name, int32_t ncols, const dq_column* cols, int64_t nrows,
                    void* stream) {
  if (!ctx || !name || !cols) return fail(ctx, DQ_ERR_INVALID, "bad table arguments");
  return guarded(ctx, [&]() {
    auto it = ctx->tables.find(name);
    if (it == ctx->tables.end()) throw DqError(DQ_ERR_NOT_FOUND, std::string("unknown table ") + name);
    TableRec& t = it->second;
    if (t.nrows != nrows) throw DqError(DQ_ERR_INVALID, "row count differs from the registered table");
    cudaStream_t st = stream ? (cudaStream_t)stream : ctx->stream;
    for (int i = 0; i < ncols; ++i) {
      ColRec* rec = nullptr;
      for (auto& c : t.cols)
        if (c.name == cols[i].name) rec = &c;
      if (!rec || rec->ctype != cols[i].ctype) throw DqError(DQ_ERR_INVALID, std::string("column mismatch ") + cols[i].name);
      if (rec->ctype == DQ_STR) throw DqError(DQ_ERR_UNSUPPORTED, "updating string columns");
      DQ_CUDA(cudaMemcpyAsync(rec->data->ptr, cols[i].data, (size_t)nrows * ctype_width(rec->ctype),
                              cudaMemcpyHostToDevice, st));
    }
    return (int)DQ_OK;
  });
}

int dq_table_drop(dq_ctx* ctx, const char* name) {
  if (!ctx || !name) return fail(ctx, DQ_ERR_INVALID, "bad arguments");
  std::lock_guard<std::mutex> lk(ctx->mu);
  if (!ctx->tables.erase(name)) return fail(ctx, DQ_ERR_NOT_FOUND, std::string("unknown table ") + name);
  return DQ_OK;
}

int dq_table_rows(dq_ctx* ctx, const char* name, int64_t* nrows) {
  if (!ctx || !name || !nrows) return fail(ctx, DQ_ERR_INVALID, "bad arguments");
  auto it = ctx->tables.find(name);
  if (it == ctx->tables.end()) return fail(ctx, DQ_ERR_NOT_FOUND, std::string("unknown table ") + name);
  *nrows = it->second.nrows;
  return DQ_OK;
}

// ---------------------------------------------------------------- import --

namespace {

const char* import_reason(int why) {
  switch (why) {
    case kImpTooFew: return "fewer delimiters than fields";
    case kImpTooMany: return "more delimiters than fields";
    case kImpNoDigit: return "not a number";
    case kImpOverflow: return "number out of range";
    case kImpNotChar: return "not a single character";
    case kImpShortDate: return "date shorter than 10 bytes";
    case kImpExponent: return "exponent not accepted";
    default: return "malformed";
  }
}

int text_ctype(int kind) {
  switch (kind) {
    case kTxtInt: return DQ_I32;
    case kTxtDate: return DQ_U32;
    case kTxtChar: return DQ_I8;
    case kTxtDecimal: return DQ_I64;
    case kTxtFloat: return DQ_U32;
    case kTxtString: return DQ_STR;
    default: return 0;
  }
}

}  // namespace

int dq_table_import_text(dq_ctx* ctx, const char* name, const char* text, uint64_t nbytes, char delim,
                         int32_t nfields, const dq_text_field* fields, int64_t* nrows_out) {
  if (!ctx || !name || (nbytes && !text) || nfields <= 0 || !fields || !nrows_out)
    return fail(ctx, DQ_ERR_INVALID, "bad import arguments");
  if (nfields > kImpMaxFields) return fail(ctx, DQ_ERR_UNSUPPORTED, "more than 64 fields a line");
  if (delim == '\n' || delim == '\r' || delim == '\0') return fail(ctx, DQ_ERR_INVALID, "bad delimiter");
  return guarded(ctx, [&]() {
    if (ctx->offline) throw DqError(DQ_ERR_UNSUPPORTED, "an offline context cannot import");
    for (int f = 0; f < nfields; ++f) {
      const dq_text_field& F = fields[f];
      if (F.kind < kTxtInt || F.kind > kTxtFloat) throw DqError(DQ_ERR_INVALID, "bad field kind");
      if (F.kind == kTxtSkip) continue;
      if (!F.name || !*F.name) throw DqError(DQ_ERR_INVALID, "field without a name");
      if (F.kind == kTxtDecimal && (F.scale < 0 || F.scale > 18)) throw DqError(DQ_ERR_INVALID, "decimal scale not in 0..18");
      for (int g = 0; g < f; ++g)
        if (fields[g].kind != kTxtSkip && !strcmp(fields[g].name, F.name))
          throw DqError(DQ_ERR_INVALID, std::string("duplicate column ") + F.name);
    }
    std::lock_guard<std::mutex> lk(ctx->mu);
    DQ_CUDA(cudaSetDevice(ctx->device));
    cudaStream_t st = ctx->stream;
    const auto t_call = std::chrono::steady_clock::now();
    struct Events {
      cudaEvent_t e[9] = {};
      ~Events() {
        for (auto& x : e)
          if (x) cudaEventDestroy(x);
      }
    } ev;
    for (auto& x : ev.e) DQ_CUDA(cudaEventCreate(&x));
    dq_import_timing tm{};
    tm.nbytes = nbytes;
    auto& S = ctx->imp;
    DQ_CUDA(cudaEventRecord(ev.e[0], st));
    // The text as whole 16 KB tiles: text in this device's memory at a 16-byte
    // boundary is read where it lies, its last partial tile from a zero-padded
    // copy; other text is copied into a padded buffer.
    const uint64_t ntiles = std::max<uint64_t>(1, (nbytes + kImpTile - 1) / kImpTile);
    cudaPointerAttributes pa{};
    const bool on_device = nbytes && cudaPointerGetAttributes(&pa, text) == cudaSuccess &&
                           pa.type == cudaMemoryTypeDevice && pa.device == ctx->device;
    cudaGetLastError();
    const bool in_place = on_device && ((uintptr_t)text & 15) == 0;
    const uint8_t* main_text;
    uint64_t nmain;  // bytes read from main_text: whole tiles
    S.tail.reserve(kImpTile);
    if (in_place) {
      nmain = nbytes / kImpTile * kImpTile;
      main_text = reinterpret_cast<const uint8_t*>(text);
      DQ_CUDA(cudaMemsetAsync(S.tail.ptr, 0, kImpTile + 256, st));
      if (nbytes > nmain)
        DQ_CUDA(cudaMemcpyAsync(S.tail.ptr, text + nmain, nbytes - nmain, cudaMemcpyDeviceToDevice, st));
    } else {
      nmain = ntiles * kImpTile;
      S.text.reserve(nmain);
      main_text = S.text.as<uint8_t>();
      if (nbytes) DQ_CUDA(cudaMemcpyAsync(S.text.ptr, text, nbytes, on_device ? cudaMemcpyDeviceToDevice
                                                                              : cudaMemcpyHostToDevice, st));
      DQ_CUDA(cudaMemsetAsync(S.text.as<uint8_t>() + nbytes, 0, nmain - nbytes + 256, st));
    }
    S.tcnt.reserve((ntiles + 1) * 8);
    S.toff.reserve((ntiles + 1) * 8);
    ImpText T{main_text, S.tail.as<uint8_t>(), nmain};
    DQ_CUDA(cudaEventRecord(ev.e[1], st));
    DQ_CUDA(launch_import_lines(T, ntiles, S.tcnt.as<uint64_t>(), S.toff.as<uint64_t>(), st));
    DQ_CUDA(cudaEventRecord(ev.e[2], st));
    tm.kernel_launches += 2;
    uint64_t nlines = 0;
    uint8_t last = '\n';
    DQ_CUDA(cudaMemcpyAsync(&nlines, S.toff.as<uint64_t>() + ntiles, 8, cudaMemcpyDeviceToHost, st));
    if (nbytes && on_device) DQ_CUDA(cudaMemcpyAsync(&last, text + nbytes - 1, 1, cudaMemcpyDeviceToHost, st));
    if (nbytes && !on_device) last = (uint8_t)text[nbytes - 1];
    DQ_CUDA(cudaStreamSynchronize(st));
    const uint64_t nrows = nlines + (nbytes && last != '\n' ? 1 : 0);
    S.lend.reserve(std::max<uint64_t>(nlines, 1) * 8);
    DQ_CUDA(cudaEventRecord(ev.e[3], st));
    if (nlines) DQ_CUDA(launch_import_line_ends(T, ntiles, S.toff.as<uint64_t>(), S.lend.as<uint64_t>(), st));
    tm.kernel_launches += nlines ? 1 : 0;
    DQ_CUDA(cudaEventRecord(ev.e[4], st));

    ImpArgs A{};
    A.text = T;
    A.nbytes = nbytes;
    A.nlines = nlines;
    A.nrows = nrows;
    A.line_end = S.lend.as<uint64_t>();
    A.nblocks = (nrows + kImpRows - 1) / kImpRows;
    A.nfields = nfields;
    A.delim = (uint8_t)delim;
    // The fixed-width columns and the string offsets of the new table: one
    // slab; the string heaps: a second one.  A table of the same name that is
    // being replaced lends its slabs when they are large enough (a repeated
    // load allocates nothing); if this import then fails, that table is gone.
    std::shared_ptr<DevBuf> old_fixed, old_heap;
    auto old = ctx->tables.find(name);
    if (old != ctx->tables.end()) {
      for (auto& c : old->second.cols) {
        if (c.ctype == DQ_STR) {
          if (c.offsets && c.offsets->slab) old_fixed = c.offsets->slab;
          if (c.data && c.data->slab) old_heap = c.data->slab;
        } else if (c.data && c.data->slab) {
          old_fixed = c.data->slab;
        }
      }
    }
    bool reused = false;
    struct DropOnFail {  // a failed import that wrote into the old table's slab removes that table
      dq_ctx* c;
      const char* n;
      const bool& reused;
      bool done;
      ~DropOnFail() {
        if (!done && reused) c->tables.erase(n);
      }
    } guard{ctx, name, reused, false};
    TableRec t;
    t.nrows = (int64_t)nrows;
    std::vector<int> str_col;  // string ordinal -> column index in t.cols
    size_t slab_bytes = 0;
    for (int f = 0; f < nfields; ++f) {
      const int k = fields[f].kind;
      if (k == kTxtSkip) continue;
      slab_bytes += DevBuf::span_of(k == kTxtString ? (nrows + 1) * 8 : nrows * ctype_width(text_ctype(k)));
    }
    std::shared_ptr<DevBuf> slab;
    if (old_fixed && old_fixed->bytes >= slab_bytes) {
      slab = old_fixed;
      reused = true;
    } else {
      slab = std::make_shared<DevBuf>();
      slab->alloc(slab_bytes);
    }
    size_t at = 0;
    for (int f = 0; f < nfields; ++f) {
      const dq_text_field& F = fields[f];
      ImpField& G = A.f[f];
      G.kind = F.kind;
      G.scale = F.scale;
      if (F.kind == kTxtSkip) continue;
      ColRec rec;
      rec.name = F.name;
      rec.ctype = text_ctype(F.kind);
      if (F.kind == kTxtString) {
        rec.width = 0;
        rec.offsets = DevBuf::view(slab, at, (nrows + 1) * 8);
        at += DevBuf::span_of((nrows + 1) * 8);
        G.str = A.nstr++;
        str_col.push_back((int)t.cols.size());
      } else {
        rec.width = ctype_width(rec.ctype);
        rec.data = DevBuf::view(slab, at, nrows * rec.width);
        at += DevBuf::span_of(nrows * rec.width);
        G.out = rec.data->ptr;
      }
      t.cols.push_back(std::move(rec));
    }
    S.err.reserve(8);
    DQ_CUDA(cudaMemsetAsync(S.err.ptr, 0xff, 8, st));
    A.err = S.err.as<uint64_t>();
    if (A.nstr) {
      S.spos.reserve((uint64_t)A.nstr * std::max<uint64_t>(nrows, 1) * 8);
      S.slen.reserve((uint64_t)A.nstr * std::max<uint64_t>(nrows, 1) * 4);
      S.bsum.reserve((uint64_t)A.nstr * (A.nblocks + 1) * 8);
      S.boff.reserve((uint64_t)A.nstr * (A.nblocks + 1) * 8);
      A.spos = S.spos.as<uint64_t>();
      A.slen = S.slen.as<uint32_t>();
      A.bsum = S.bsum.as<uint64_t>();
      A.boff = S.boff.as<uint64_t>();
      if (nrows == 0) DQ_CUDA(cudaMemsetAsync(S.boff.ptr, 0, (uint64_t)A.nstr * 8, st));
    }
    DQ_CUDA(cudaEventRecord(ev.e[8], st));
    DQ_CUDA(launch_import_parse(A, st));
    DQ_CUDA(cudaEventRecord(ev.e[5], st));
    tm.kernel_launches += nrows ? 1 + (A.nstr ? 1 : 0) : 0;
    std::vector<uint64_t> totals(A.nstr, 0);
    uint64_t bad = ~0ull;
    DQ_CUDA(cudaMemcpyAsync(&bad, S.err.ptr, 8, cudaMemcpyDeviceToHost, st));
    for (int j = 0; j < A.nstr; ++j)
      DQ_CUDA(cudaMemcpyAsync(&totals[j], A.boff + (uint64_t)j * (A.nblocks + 1) + A.nblocks, 8,
                              cudaMemcpyDeviceToHost, st));
    DQ_CUDA(cudaStreamSynchronize(st));
    if (bad != ~0ull) {
      const uint64_t row = bad >> 16;
      const int field = (int)((bad >> 8) & 0xff), why = (int)(bad & 0xff);
      std::string where = field < nfields ? std::string(" field ") + std::to_string(field + 1) +
                                                (fields[field].kind != kTxtSkip ? std::string(" (") + fields[field].name + ")" : "")
                                          : std::string();
      throw DqError(DQ_ERR_INVALID, std::string("import of ") + name + ": line " + std::to_string(row + 1) + where +
                                        ": " + import_reason(why));
    }
    // the string heaps: a second slab
    size_t heap_bytes = 0;
    for (int j = 0; j < A.nstr; ++j) heap_bytes += DevBuf::span_of(totals[j]);
    std::shared_ptr<DevBuf> heaps;
    if (old_heap && old_heap->bytes >= heap_bytes) {
      heaps = old_heap;
    } else {
      heaps = std::make_shared<DevBuf>();
      if (A.nstr) heaps->alloc(heap_bytes);
    }
    at = 0;
    for (int j = 0; j < A.nstr; ++j) {
      ColRec& c = t.cols[str_col[j]];
      c.nchars = totals[j];
      c.data = DevBuf::view(heaps, at, totals[j]);
      at += DevBuf::span_of(totals[j]);
      A.sheap[j] = c.data->as<uint8_t>();
      A.soff[j] = c.offsets->as<uint64_t>();
      if (nrows == 0) DQ_CUDA(cudaMemsetAsync(c.offsets->ptr, 0, 8, st));
    }
    DQ_CUDA(cudaEventRecord(ev.e[6], st));
    DQ_CUDA(launch_import_strings(A, st));
    DQ_CUDA(cudaEventRecord(ev.e[7], st));
    tm.kernel_launches += nrows && A.nstr ? 1 : 0;
    DQ_CUDA(cudaStreamSynchronize(st));
    ctx->tables[name] = std::move(t);
    guard.done = true;
    *nrows_out = (int64_t)nrows;
    float ms = 0;
    auto span = [&](int a, int b) {
      DQ_CUDA(cudaEventElapsedTime(&ms, ev.e[a], ev.e[b]));
      return (double)ms;
    };
    tm.copy_ms = span(0, 1);
    tm.newline_ms = span(1, 2);
    tm.line_end_ms = span(3, 4);
    tm.parse_ms = span(8, 5);
    tm.string_ms = span(6, 7);
    tm.span_ms = span(0, 7);
    tm.call_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_call).count();
    ctx->last_import = tm;
    return (int)DQ_OK;
  });
}

int dq_table_import_timing_get(dq_ctx* ctx, dq_import_timing* out) {
  if (!ctx || !out) return fail(ctx, DQ_ERR_INVALID, "bad arguments");
  std::lock_guard<std::mutex> lk(ctx->mu);
  *out = ctx->last_import;
  return DQ_OK;
}

int dq_table_column_read(dq_ctx* ctx, const char* table, const char* column, void* data, uint64_t data_bytes,
                         uint64_t* offsets, uint64_t* nchars) {
  if (!ctx || !table || !column) return fail(ctx, DQ_ERR_INVALID, "bad arguments");
  return guarded(ctx, [&]() {
    if (ctx->offline) throw DqError(DQ_ERR_UNSUPPORTED, "an offline context holds no column data");
    std::lock_guard<std::mutex> lk(ctx->mu);
    auto it = ctx->tables.find(table);
    if (it == ctx->tables.end()) throw DqError(DQ_ERR_NOT_FOUND, std::string("unknown table ") + table);
    const ColRec* c = it->second.find(column);
    if (!c) throw DqError(DQ_ERR_NOT_FOUND, std::string("unknown column ") + column);
    const uint64_t nrows = (uint64_t)it->second.nrows;
    DQ_CUDA(cudaSetDevice(ctx->device));
    cudaStream_t st = ctx->stream;
    if (c->ctype == DQ_STR) {
      if (nchars) *nchars = c->nchars;
      if (data) {
        if (data_bytes < c->nchars) throw DqError(DQ_ERR_INVALID, "buffer smaller than the string heap");
        if (c->nchars) DQ_CUDA(cudaMemcpyAsync(data, c->data->ptr, c->nchars, cudaMemcpyDeviceToHost, st));
      }
      if (offsets) {
        if (c->width > 0) {
          for (uint64_t i = 0; i <= nrows; ++i) offsets[i] = i * (uint64_t)c->width;
        } else {
          DQ_CUDA(cudaMemcpyAsync(offsets, c->offsets->ptr, (nrows + 1) * 8, cudaMemcpyDeviceToHost, st));
        }
      }
    } else {
      const uint64_t b = nrows * (uint64_t)ctype_width(c->ctype);
      if (!data || data_bytes < b) throw DqError(DQ_ERR_INVALID, "buffer smaller than the column");
      if (b) DQ_CUDA(cudaMemcpyAsync(data, c->data->ptr, b, cudaMemcpyDeviceToHost, st));
    }
    DQ_CUDA(cudaStreamSynchronize(st));
    return (int)DQ_OK;
  });
}

int dq_plan_prepare(dq_ctx* ctx, const dq_plan_desc* desc, dq_plan** out) {
  if (!ctx || !desc || !out) return fail(ctx, DQ_ERR_INVALID, "bad arguments");
  *out = nullptr;
  return guarded(ctx, [&]() {
    if (desc->abi_version != DQ_ABI_VERSION) throw DqError(DQ_ERR_BAD_IR, "IR version mismatch");
    if (desc->nres < 0 || desc->npipes <= 0 || (desc->nres && !desc->res) || !desc->pipes)
      throw DqError(DQ_ERR_BAD_IR, "empty plan");
    std::lock_guard<std::mutex> lk(ctx->mu);
    OfflineScope offline(ctx->offline);
    if (!ctx->offline) DQ_CUDA(cudaSetDevice(ctx->device));
    std::unique_ptr<dq_plan> plan = make_plan(ctx, desc, PlanOpts());
    *out = plan.release();
    return (int)DQ_OK;
  });
}

int dq_plan_execute(dq_plan* plan, void* stream, dq_result** out) {
  if (!plan || !out) return DQ_ERR_INVALID;
  dq_ctx* ctx = plan->ctx;
  *out = nullptr;
  return guarded(ctx, [&]() {
    if (ctx->offline) throw DqError(DQ_ERR_UNSUPPORTED, "an offline context compiles plans but cannot execute them");
    std::lock_guard<std::mutex> lk(ctx->mu);
    DQ_CUDA(cudaSetDevice(ctx->device));
    cudaStream_t st = stream ? (cudaStream_t)stream : ctx->stream;
    int status = 0;
    for (int attempt = 0;; ++attempt) {
      status = run_once(plan, st);
      if (status & kInfoMask) {
        if (status & kInfoHeavyFull) grow_heavy(plan);
        status &= ~kInfoMask;
      }
      if (status == 0) {
        adapt_threshold(plan);
        break;
      }
      if (attempt >= 8 || (status & (kErrTimeout | kErrBadOp)))
        throw DqError(status & kErrTimeout ? DQ_ERR_TIMEOUT
                      : status & kErrHtFull ? DQ_ERR_HT_FULL
                      : status & kErrOverflow ? DQ_ERR_OVERFLOW : DQ_ERR_BAD_IR,
                      "device status " + std::to_string(status));
      // grow what overflowed and run again (the results of a failed run are discarded)
      grow_plan(plan, status);
    }
    *out = read_result(plan, st);
    return (int)DQ_OK;
  });
}

void dq_plan_free(dq_plan* plan) {
  if (!plan) return;
  if (plan->ctx->offline) {
    delete plan;
    return;
  }
  cudaSetDevice(plan->ctx->device);
  free_events(plan);
  delete plan;
}

int dq_plan_profile(dq_plan* plan, int32_t point, uint64_t* counts) {
  if (!plan || !counts) return DQ_ERR_INVALID;
  if (point < 0 || point >= plan->nprofile) return fail(plan->ctx, DQ_ERR_NOT_FOUND, "no such profile point");
  return guarded(plan->ctx, [&]() {
    if (plan->ctx->offline) throw DqError(DQ_ERR_UNSUPPORTED, "an offline context has no profiles");
    std::lock_guard<std::mutex> lk(plan->ctx->mu);
    DQ_CUDA(cudaSetDevice(plan->ctx->device));
    DQ_CUDA(cudaMemcpy(counts, plan->profile + (size_t)point * 33, 33 * 8, cudaMemcpyDeviceToHost));
    return (int)DQ_OK;
  });
}

int dq_plan_source(dq_plan* plan, int32_t pipe, char* buf, int64_t cap, int64_t* len) {
  if (!plan || !len || cap < 0 || (cap > 0 && !buf)) return DQ_ERR_INVALID;
  if (pipe < 0 || pipe >= (int32_t)plan->pipes.size()) return fail(plan->ctx, DQ_ERR_INVALID, "no such pipeline");
  const PipeRec* pp = plan->pipes[pipe].get();
  std::string text;
  if (pp->fused_into >= 0) {
    // a fused tail: the kernel that runs it (its code is dq_tail there)
    text = "// pipeline " + std::to_string(pipe) + " runs as dq_tail in the last CTA of pipeline " +
           std::to_string(pp->fused_into) + "'s kernel\n";
    pp = plan->pipes[pp->fused_into].get();
  }
  const PipeRec& p = *pp;
  if (!p.jit) return fail(plan->ctx, DQ_ERR_NOT_FOUND, "pipeline runs on a prebuilt kernel");
  text += p.prog.source;
  if (!p.kernels.log.empty()) text += "\n/* compiler report:\n" + p.kernels.log + "\n*/\n";
  *len = (int64_t)text.size();
  if (cap > 0) {
    size_t n = std::min<size_t>((size_t)cap - 1, text.size());
    memcpy(buf, text.data(), n);
    buf[n] = '\0';
  }
  return DQ_OK;
}

int dq_plan_dependencies(dq_plan* plan, int32_t pipe, int32_t* out, int32_t cap, int32_t* n) {
  if (!plan || !n || cap < 0 || (cap > 0 && !out)) return DQ_ERR_INVALID;
  if (pipe < 0 || pipe >= (int32_t)plan->pipes.size()) return fail(plan->ctx, DQ_ERR_INVALID, "no such pipeline");
  const std::vector<std::vector<int>> deps = pipe_deps(plan);
  const std::vector<int>& d = deps[(size_t)pipe];
  *n = (int32_t)d.size();
  for (int32_t i = 0; i < cap && i < *n; ++i) out[i] = d[(size_t)i];
  return DQ_OK;
}

int dq_plan_timing_get(dq_plan* plan, dq_plan_timing* out) {
  if (!plan || !out) return DQ_ERR_INVALID;
  *out = plan->timing;
  return DQ_OK;
}

int dq_result_rows(dq_result* r, int64_t* nrows) {
  if (!r || !nrows) return DQ_ERR_INVALID;
  *nrows = r->nrows;
  return DQ_OK;
}

int dq_result_ncols(dq_result* r, int32_t* ncols) {
  if (!r || !ncols) return DQ_ERR_INVALID;
  *ncols = (int32_t)r->cols.size();
  return DQ_OK;
}

int dq_result_column(dq_result* r, int32_t col, int32_t* ctype, const void** data) {
  if (!r || col < 0 || col >= (int32_t)r->cols.size() || !ctype || !data) return DQ_ERR_INVALID;
  *ctype = r->ctypes[col];
  *data = r->cols[col].data();
  return DQ_OK;
}

int dq_result_string_heap(dq_result* r, int32_t col, const void** chars, uint64_t* nchars) {
  if (!r || col < 0 || col >= (int32_t)r->cols.size() || !chars || !nchars) return DQ_ERR_INVALID;
  if (r->ctypes[col] != DQ_STR) return DQ_ERR_INVALID;
  *chars = r->heaps[col].data();
  *nchars = r->heaps[col].size();
  return DQ_OK;
}

void dq_result_free(dq_result* r) { delete r; }

int dq_plan_prepare_tuned(dq_ctx* ctx, const dq_plan_desc* desc, const dq_tuning* tuning, dq_plan** out) {
  if (!ctx || !desc || !out) return fail(ctx, DQ_ERR_INVALID, "bad arguments");
  *out = nullptr;
  return guarded(ctx, [&]() {
    std::lock_guard<std::mutex> lk(ctx->mu);
    OfflineScope offline(ctx->offline);
    if (!ctx->offline) DQ_CUDA(cudaSetDevice(ctx->device));
    *out = make_plan(ctx, desc, opts_of(tuning)).release();
    return (int)DQ_OK;
  });
}

// --------------------------------------------------------------- batches --

int dq_batch_prepare(dq_ctx* ctx, int32_t ninst, const dq_plan_desc* descs, const dq_tuning* tuning, dq_batch** out) {
  if (!ctx || !descs || !out || ninst <= 0) return fail(ctx, DQ_ERR_INVALID, "bad arguments");
  *out = nullptr;
  return guarded(ctx, [&]() {
    std::lock_guard<std::mutex> lk(ctx->mu);
    OfflineScope offline(ctx->offline);  // offline: the batch's kernels are compiled only
    if (!ctx->offline) DQ_CUDA(cudaSetDevice(ctx->device));
    std::unique_ptr<dq_batch> b(new dq_batch());
    b->ctx = ctx;
    b->ninst = ninst;
    b->tuning = tuning_of(tuning);
    PlanOpts o = opts_of(tuning);
    o.batch_member = true;
    for (int i = 0; i < ninst; ++i) {
      b->inst.push_back(make_plan(ctx, &descs[i], o));
      if (b->inst[i]->pipes.size() != b->inst[0]->pipes.size() || b->inst[i]->res.size() != b->inst[0]->res.size())
        throw DqError(DQ_ERR_BAD_IR, "batch instance " + std::to_string(i) + " differs in shape from instance 0");
    }
    b->status.alloc(4);
    if (!ctx->offline) {
      DQ_CUDA(cudaEventCreate(&b->ev0));
      DQ_CUDA(cudaEventCreate(&b->ev1));
    }
    build_batch(b.get(), b->tuning, ctx->stream);
    *out = b.release();
    return (int)DQ_OK;
  });
}

int dq_batch_execute(dq_batch* b, void* stream, dq_result** results) {
  if (!b || !results) return DQ_ERR_INVALID;
  dq_ctx* ctx = b->ctx;
  return guarded(ctx, [&]() {
    if (ctx->offline) throw DqError(DQ_ERR_UNSUPPORTED, "an offline context compiles batches but cannot execute them");
    std::lock_guard<std::mutex> lk(ctx->mu);
    DQ_CUDA(cudaSetDevice(ctx->device));
    cudaStream_t st = stream ? (cudaStream_t)stream : ctx->stream;
    int32_t status = 0;
    for (int attempt = 0;; ++attempt) {
      DQ_CUDA(cudaEventRecord(b->ev0, st));
      DQ_CUDA(cudaGraphLaunch(b->exec, st));
      DQ_CUDA(cudaEventRecord(b->ev1, st));
      DQ_CUDA(cudaStreamSynchronize(st));
      memcpy(&status, b->host + b->packed_bytes + (size_t)b->ninst * 8, 4);
      if (status & kInfoHeavyFull) {
        // this run's results stand; later runs get twice the deferred items
        uint64_t want = 0;
        for (auto& Sp : b->stages)
          if (Sp->kernels.heavy) {
            uint32_t n = 0;
            DQ_CUDA(cudaMemcpy(&n, Sp->h_count.ptr, 4, cudaMemcpyDeviceToHost));
            want = std::max<uint64_t>(want, 2ull * n);
          }
        b->heavy_cap = std::min<uint64_t>(std::max(want, 2 * std::max<uint64_t>(b->heavy_cap, 1 << 20)),
                                          0xffffffffull);
        status &= ~kInfoMask;
        if (status == 0) build_batch(b, b->tuning, st);
      }
      status &= ~kInfoMask;
      if (status == 0) break;
      if (attempt >= 8 || (status & (kErrTimeout | kErrBadOp))) throw_status(status);
      for (auto& pl : b->inst) grow_plan(pl.get(), status);
      build_batch(b, b->tuning, st);
    }
    float ms = 0;
    cudaEventElapsedTime(&ms, b->ev0, b->ev1);
    memset(&b->timing, 0, sizeof(b->timing));
    b->timing.total_ms = ms;
    b->timing.max_pipeline = -1;
    b->timing.kernel_launches = b->launches;
    const uint64_t* rows = reinterpret_cast<const uint64_t*>(b->host + b->packed_bytes);
    for (int i = 0; i < b->ninst; ++i) results[i] = nullptr;
    try {
      for (int i = 0; i < b->ninst; ++i) results[i] = packed_result(b->inst[i].get(), b->host, b->col_off[i], rows[i], st);
    } catch (...) {
      for (int i = 0; i < b->ninst; ++i) {
        delete results[i];
        results[i] = nullptr;
      }
      throw;
    }
    return (int)DQ_OK;
  });
}

int dq_batch_timing_get(dq_batch* b, dq_plan_timing* out) {
  if (!b || !out) return DQ_ERR_INVALID;
  *out = b->timing;
  return DQ_OK;
}

int dq_batch_size(dq_batch* b, int32_t* ninst) {
  if (!b || !ninst) return DQ_ERR_INVALID;
  *ninst = b->ninst;
  return DQ_OK;
}

void dq_batch_free(dq_batch* b) {
  if (!b) return;
  cudaSetDevice(b->ctx->device);
  delete b;
}

}  // extern "C"

// ================================================================= serving ==
//
// A request loop on its own thread.  Requests carry a plan IR over registered
// (resident) tables; the loop keeps prepared plans pooled per distinct request,
// so a repeated query reuses its tables and compiled kernels.  It admits the
// oldest waiting request when a device slot (a CUDA stream) is free and the
// request's estimated table and intermediate bytes fit the memory budget next
// to the plans already held (idle pooled plans are freed first to make room),
// enqueues the request's pipelines on that stream without waiting, and turns
// completed slots into results.  Requests that arrive while others run are
// admitted as soon as a slot and memory free up, and their kernels overlap on
// the device with the running ones.

namespace {

double now_ms() {
  return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

// A deep copy of a request's IR (the caller's arrays and strings may go away
// after submit) and the key that identifies the query.
struct DescCopy {
  std::vector<dq_resource> res;
  std::vector<dq_pipeline> pipes;
  std::deque<std::string> strs;
  dq_plan_desc d{};
  std::string key;
  uint64_t rows = 0;                // input rows of the tables it scans (set at submit)
  const char* keep(const char* s) {
    if (!s) return nullptr;
    strs.emplace_back(s);
    return strs.back().c_str();
  }
};

std::shared_ptr<DescCopy> copy_desc(const dq_plan_desc* in) {
  if (!in || in->abi_version != DQ_ABI_VERSION || in->npipes <= 0 || !in->pipes || in->nres < 0 ||
      (in->nres > 0 && !in->res))
    throw DqError(DQ_ERR_BAD_IR, "bad plan descriptor");
  std::shared_ptr<DescCopy> c(new DescCopy());
  c->res.assign(in->res, in->res + in->nres);
  c->pipes.assign(in->pipes, in->pipes + in->npipes);
  std::string key;
  for (auto& r : c->res) {
    dq_resource z = r;
    z.name = nullptr;
    key.append(reinterpret_cast<const char*>(&z), sizeof(z));
    r.name = c->keep(r.name);
  }
  for (auto& p : c->pipes) {
    if (p.ncols < 0 || p.ncols > DQ_MAX_COLS || p.npatterns < 0 || p.npatterns > DQ_MAX_PATTERNS)
      throw DqError(DQ_ERR_BAD_IR, "pipeline sizes out of range");
    dq_pipeline z = p;
    z.table = nullptr;
    for (int j = 0; j < DQ_MAX_COLS; ++j) z.cols[j] = nullptr;
    for (int j = 0; j < DQ_MAX_PATTERNS; ++j) z.patterns[j] = nullptr;
    key.append(reinterpret_cast<const char*>(&z), sizeof(z));
    p.table = c->keep(p.table);
    key += p.table ? p.table : "";
    key.push_back('\0');
    for (int j = 0; j < p.ncols; ++j) {
      p.cols[j] = c->keep(p.cols[j]);
      key += p.cols[j] ? p.cols[j] : "";
      key.push_back('\0');
    }
    for (int j = 0; j < p.npatterns; ++j) {
      p.patterns[j] = c->keep(p.patterns[j]);
      key += p.patterns[j] ? p.patterns[j] : "";
      key.push_back('\0');
    }
  }
  c->d = *in;
  c->d.res = c->res.data();
  c->d.pipes = c->pipes.data();
  c->key = std::move(key);
  return c;
}

// Device bytes a request's plan will hold, from its IR (before preparing it).
// Rows of the registered tables a plan scans (each table once).
uint64_t scanned_rows(dq_ctx* ctx, const dq_plan_desc& d) {
  std::unordered_set<std::string> seen;
  uint64_t rows = 0;
  for (int i = 0; i < d.npipes; ++i) {
    const dq_pipeline& p = d.pipes[i];
    if (p.source_kind != DQ_SRC_TABLE || !p.table || !seen.insert(p.table).second) continue;
    auto it = ctx->tables.find(p.table);
    if (it != ctx->tables.end()) rows += (uint64_t)std::max<int64_t>(it->second.nrows, 0);
  }
  return rows;
}

uint64_t estimate_bytes(dq_ctx* ctx, const dq_plan_desc& d) {
  uint64_t b = 4096;
  std::vector<uint64_t> multi_rows(std::max(d.nres, 0), 0);
  for (int i = 0; i < d.nres; ++i) {
    const dq_resource& r = d.res[i];
    const uint64_t cap = (uint64_t)std::max<int64_t>(r.capacity, 16);
    const bool packed = keys_packed(r.nkeys, r.key_ctype);
    const uint64_t keyw = packed ? 0 : r.nkeys;
    uint64_t widths = 0;
    for (int j = 0; j < r.npay && j < DQ_MAX_PAY; ++j) widths += ctype_width(r.pay_ctype[j]);
    switch (r.kind) {
      case DQ_RES_UNIQUE: {  // the sizing of setup_resource: 4x while that fits kL2TableBytes, else 2x
        const uint64_t words = 1 + keyw + r.npay;
        const uint64_t slots = cap * 4 * words * 8 <= kL2TableBytes ? 4 * cap : 2 * cap;
        b += (slots + 4) * words * 8;
        break;
      }
      case DQ_RES_AGG: b += (cap + 1) * (1 + keyw + r.naggs) * 8; break;
      case DQ_RES_MULTI: {
        uint64_t rows = cap;
        for (int p = 0; p < d.npipes; ++p) {
          const dq_pipeline& pp = d.pipes[p];
          const dq_op& sink = pp.ops[std::max(pp.nops - 1, 0)];
          if (sink.kind == DQ_OP_MM_SCATTER && sink.res == i && pp.table) {
            auto it = ctx->tables.find(pp.table);
            if (it != ctx->tables.end()) rows = (uint64_t)it->second.nrows;
          }
        }
        b += cap * 8 + rows * widths + 256;
        multi_rows[i] = rows;
        break;
      }
      case DQ_RES_OUTPUT: b += cap * widths + 256; break;
    }
  }
  // deferred-expansion buffers of a pipeline that expands at level 0 (the
  // sizing of setup_pipeline: items, their grouped copy, prefixes, group table)
  for (int p = 0; p < d.npipes; ++p) {
    const dq_pipeline& pp = d.pipes[p];
    for (int k = 0; k < pp.nops; ++k) {
      const dq_op& op = pp.ops[k];
      if (op.kind != DQ_OP_EXPAND) continue;
      std::vector<int> reads;
      for (int j = k; j < pp.nops; ++j) slot_reads(pp, pp.ops[j], reads);
      std::sort(reads.begin(), reads.end());
      reads.erase(std::unique(reads.begin(), reads.end()), reads.end());
      uint64_t stash = 0;
      for (int sl : reads) stash += pp.slots[sl].level == 0 ? 1 : 0;
      if (stash > (uint64_t)kMaxStash) break;
      uint64_t rows = 1 << 20;
      if (pp.table) {
        auto it = ctx->tables.find(pp.table);
        if (it != ctx->tables.end()) rows = std::min<uint64_t>(rows, std::max<int64_t>(it->second.nrows, 1));
      }
      const uint64_t built = op.res >= 0 && op.res < d.nres ? std::max<uint64_t>(multi_rows[op.res], 1) : rows;
      const uint64_t gcap = std::max<uint64_t>(64, 2 * std::min<uint64_t>(rows, built / (kGroupThreshold + 1) + 1));
      b += rows * (2 + stash) * 8 + rows * std::max<uint64_t>(stash, 1) * 8 + (std::max(rows, gcap) + 1) * 8 +
           gcap * 24 + 4096;
      break;
    }
  }
  return b;
}

struct SrvReq {
  uint64_t id = 0;
  std::shared_ptr<DescCopy> desc;
  uint64_t est = 0;
  double t_submit = 0, t_dispatch = 0, t_done = 0;
  dq_result* result = nullptr;
  int status = DQ_OK;
  std::string error;
  bool done = false;
  int attempts = 0;                 // executions after tables grew
  bool solo = false;                // runs alone (a batch it was in overflowed)
  dq_request_info info{};
};

// Outputs up to this size are copied back inside a pooled plan's CUDA graph
// (at full capacity, into pinned memory); larger ones are read after the run.
constexpr uint64_t kGraphOutMax = 16ull << 20;

struct PoolEntry {
  std::unique_ptr<dq_plan> plan;
  uint64_t bytes = 0;
  bool busy = false;
  int32_t* host_status = nullptr;   // pinned
  // the whole run (resets, pipelines, status, row count and result columns
  // copied back) as one graph: one launch per request
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  uint8_t* host_out = nullptr;      // pinned: row count, then the columns
  std::vector<uint64_t> col_off;
  int launches = 0;
  bool no_graph = false;
  bool count_only = false;          // results too large to copy whole: the graph copies the
                                    // row count, the rows follow after completion
  void drop_graph() {
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    if (host_out) cudaFreeHost(host_out);
    exec = nullptr;
    graph = nullptr;
    host_out = nullptr;
  }
  ~PoolEntry() {
    drop_graph();
    if (host_status) cudaFreeHost(host_status);
  }
};

// Captures a pooled plan's run and result copies into a graph (outputs whose
// capacity exceeds kGraphOutMax: the row count only, the rows follow).
void srv_build_graph(PoolEntry* pe, cudaStream_t st) {
  pe->drop_graph();
  dq_plan* plan = pe->plan.get();
  const ResRec& o = *plan->res[plan->result_res];
  uint64_t bytes = 16;
  pe->col_off.clear();
  for (int j = 0; j < o.desc.npay; ++j) {
    pe->col_off.push_back(bytes);
    bytes = align_up(bytes + o.dev.cap * (uint64_t)ctype_width(o.desc.pay_ctype[j]), 16);
  }
  pe->count_only = bytes > kGraphOutMax;
  if (pe->count_only) bytes = 16;
  DQ_CUDA(cudaMallocHost((void**)&pe->host_out, bytes));
  DQ_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
  cudaError_t err = cudaSuccess;
  try {
    pe->launches = enqueue_run(plan, st, pe->host_status);
  } catch (const DqError&) {
    err = cudaErrorUnknown;
  }
  auto rec = [&](cudaError_t e) {
    if (err == cudaSuccess && e != cudaSuccess) err = e;
  };
  rec(cudaMemcpyAsync(pe->host_out, o.dev.cursor, 8, cudaMemcpyDeviceToHost, st));
  if (!pe->count_only)
    for (int j = 0; j < o.desc.npay; ++j)
      rec(cudaMemcpyAsync(pe->host_out + pe->col_off[j], o.dev.pay[j],
                          o.dev.cap * (uint64_t)ctype_width(o.desc.pay_ctype[j]), cudaMemcpyDeviceToHost, st));
  cudaGraph_t g = nullptr;
  const cudaError_t end = cudaStreamEndCapture(st, &g);
  pe->graph = g;
  DQ_CUDA(err);
  DQ_CUDA(end);
  DQ_CUDA(cudaGraphInstantiate(&pe->exec, pe->graph, 0));
  DQ_CUDA(cudaGraphUpload(pe->exec, st));  // not at the first request's launch
}

dq_result* srv_graph_result(PoolEntry* pe, cudaStream_t st) {
  const ResRec& o = *pe->plan->res[pe->plan->result_res];
  uint64_t n = 0;
  memcpy(&n, pe->host_out, 8);
  if (n > o.dev.cap) n = o.dev.cap;
  if (!pe->count_only) return packed_result(pe->plan.get(), pe->host_out, pe->col_off, n, st);
  std::unique_ptr<dq_result> res(new dq_result());
  res->nrows = (int64_t)n;
  res->heaps.resize(o.desc.npay);
  for (int j = 0; j < o.desc.npay; ++j) {
    const int w = ctype_width(o.desc.pay_ctype[j]);
    res->ctypes.push_back(o.desc.pay_ctype[j]);
    if (o.desc.pay_ctype[j] == DQ_STR) {
      res->cols.emplace_back();
      gather_string_column(pe->plan.get(), reinterpret_cast<const uint64_t*>(o.dev.pay[j]), n, st, res->cols.back(),
                           res->heaps[j]);
    } else {
      res->cols.emplace_back((size_t)n * w);
      if (n) DQ_CUDA(cudaMemcpyAsync(res->cols.back().data(), o.dev.pay[j], (size_t)n * w, cudaMemcpyDeviceToHost, st));
    }
  }
  if (n) DQ_CUDA(cudaStreamSynchronize(st));
  return res.release();
}

// ------------------------------------------------------ continuous batching --
// Waiting requests of one shape (the same generated batch kernels: same
// pipelines and ops, any tables and sizes) run as one many-instance launch on
// one slot, each on its own pooled plan: the batch kernels and helpers of
// dq_batch_* over descriptors assembled per dispatch.

struct SrvShape {                   // the batch kernels of one request shape
  struct Stage {
    jit::Program prog;
    jit::Kernels kernels;
    int occ = 1, hocc = 1;          // resident CTAs per SM (main, heavy kernel)
    bool mm_scan = false;           // a multimap count: the bucket scans follow
    int mm_res = -1;
    int expand_op = -1;             // deferred expansion (heavy kernel)
  };
  std::vector<Stage> stages;
  // the largest per-member needs seen: a slot's scratch is sized for a full
  // batch of such members, so it grows while the shape's mix is first seen
  // (growing frees device memory, which synchronises the device), not later
  uint64_t member_out = 0, member_rows = 0, member_build = 0;
};

void grow(DevBuf& b, size_t n) {
  if (b.bytes < n) b.alloc(n + n / 2);
}

struct HeavyBufs {                  // a slot's shared deferral buffers of one stage
  DevBuf items, count, units, gkey, glen, gcnt, glist, gstart, sorted, prefix;
  DevHeavy bind(const DevHeavy& proto, uint32_t cap, uint32_t gcap) {
    DevHeavy H = proto;
    H.grouped = 1;
    H.cap = cap;
    H.gcap = gcap;
    grow(items, (size_t)cap * H.words * 8);
    grow(count, 8);
    grow(units, 4);
    grow(gkey, (size_t)gcap * 8);
    grow(glen, (size_t)gcap * 4);
    grow(gcnt, (size_t)gcap * 4);
    grow(glist, (size_t)gcap * 4);
    grow(gstart, ((size_t)gcap + 1) * 4);
    grow(sorted, (size_t)cap * std::max(H.nstash, 1) * 8);
    grow(prefix, (std::max<size_t>(cap, gcap) + 1) * 8);
    H.items = items.as<uint64_t>();
    H.count = count.as<uint32_t>();
    H.ngroups = count.as<uint32_t>() + 1;
    H.unit_prefix = prefix.as<uint64_t>();
    H.gkey = gkey.as<uint64_t>();
    H.glen = glen.as<uint32_t>();
    H.gcnt = gcnt.as<uint32_t>();
    H.glist = glist.as<uint32_t>();
    H.gstart = gstart.as<uint32_t>();
    H.sorted = sorted.as<uint64_t>();
    return H;
  }
};

struct SrvBatch {                   // a slot's batch in flight and its scratch
  std::vector<std::pair<SrvReq*, PoolEntry*>> members;
  DevBuf params, packed, rows, status, partials;
  uint8_t* host_params = nullptr;   // pinned staging of the descriptors
  size_t host_params_cap = 0;
  uint8_t* host_out = nullptr;      // pinned: packed columns, rows per member, status
  size_t host_out_cap = 0;
  std::vector<std::unique_ptr<HeavyBufs>> heavy;
  std::vector<std::vector<uint64_t>> col_off;
  size_t packed_bytes = 0;
  int launches = 0;
  ~SrvBatch() {
    if (host_params) cudaFreeHost(host_params);
    if (host_out) cudaFreeHost(host_out);
  }
};

struct SrvSlot {
  cudaStream_t st = nullptr;
  cudaEvent_t done = nullptr;
  SrvReq* req = nullptr;            // a request alone, or
  PoolEntry* pe = nullptr;
  std::unique_ptr<SrvBatch> batch;  // a batch (members non-empty)
  int launches = 0;
  bool busy() const { return req || (batch && !batch->members.empty()); }
};

}  // namespace

struct dq_server {
  dq_ctx* ctx = nullptr;
  dq_server_config cfg{};
  std::mutex mu;                    // requests, pending queue, statistics
  std::condition_variable cv;
  std::deque<SrvReq*> pending;
  std::unordered_map<uint64_t, std::unique_ptr<SrvReq>> reqs;
  uint64_t next_id = 1;
  // owned by the worker thread
  std::unordered_map<std::string, std::vector<std::unique_ptr<PoolEntry>>> pool;
  std::unordered_map<std::string, SrvShape*> shape_of;   // request key -> its batch shape (null: alone)
  std::unordered_map<std::string, std::unique_ptr<SrvShape>> shapes;
  uint64_t batches = 0, batched = 0;
  std::vector<SrvSlot> slots;
  cudaStream_t prep = nullptr;      // captures and uploads of pooled plans' graphs
  uint64_t mem = 0;
  std::unordered_set<std::string> compiled;  // request keys whose kernels a submitter compiled (under ctx->mu)
  // statistics (under mu)
  uint64_t submitted = 0, completed = 0, failed = 0, mem_peak = 0, mem_now = 0;
  std::vector<double> lat;
  double t_first = 0, t_last = 0;
  bool stop = false;
  std::thread worker;
};

namespace {

void srv_finish(dq_server* s, SrvReq* r, int status, const std::string& err, dq_result* res) {
  std::lock_guard<std::mutex> lk(s->mu);
  r->status = status;
  r->error = err;
  r->result = res;
  r->t_done = now_ms();
  r->done = true;
  r->info.status = status;
  r->info.total_ms = r->t_done - r->t_submit;
  r->info.queue_ms = r->t_dispatch > 0 ? r->t_dispatch - r->t_submit : r->info.total_ms;
  r->info.run_ms = r->t_dispatch > 0 ? r->t_done - r->t_dispatch : 0;
  if (status == DQ_OK) {
    ++s->completed;
    s->lat.push_back(r->info.total_ms);
  } else {
    ++s->failed;
  }
  s->t_last = r->t_done;
  s->mem_now = s->mem;
  s->mem_peak = std::max(s->mem_peak, s->mem);
  s->cv.notify_all();
}

// Frees idle pooled plans (other than those of `keep`) until `need` more bytes
// fit the budget; returns whether they fit.
bool srv_make_room(dq_server* s, uint64_t need, const std::string& keep) {
  for (auto& kv : s->pool) {
    if (s->mem + need <= s->cfg.memory_budget) break;
    if (kv.first == keep) continue;
    auto& v = kv.second;
    for (size_t i = 0; i < v.size() && s->mem + need > s->cfg.memory_budget;) {
      if (!v[i]->busy) {
        s->mem -= v[i]->bytes;
        v.erase(v.begin() + i);
      } else {
        ++i;
      }
    }
  }
  return s->mem + need <= s->cfg.memory_budget;
}

// A prepared plan for the request: an idle one of the same query, else a new
// one if the budget allows.  nullptr: wait; throws: the request fails.
// The batch shape of a prepared plan: its pipelines' many-instance kernels
// (generated, compiled on first sight of the shape), or null when the plan
// runs alone (a prebuilt kernel, or a result too large for the packed copy).
SrvShape* srv_shape(dq_server* s, dq_plan* plan) {
  if (s->cfg.batch_max <= 1) return nullptr;
  for (auto& pp : plan->pipes)
    if (!pp->jit) return nullptr;
  const ResRec& o = *plan->res[plan->result_res];
  if (o.desc.npay == 0) return nullptr;
  uint64_t out = 0;
  for (int j = 0; j < o.desc.npay; ++j) out += o.dev.cap * (uint64_t)ctype_width(o.desc.pay_ctype[j]);
  if (out > kGraphOutMax) return nullptr;
  std::vector<jit::Program> progs;
  std::string key;
  for (auto& pp : plan->pipes) {
    jit::Tuning t = plan->opts.tuning;
    t.batched = true;
    progs.push_back(jit::generate(pp->dev, pp->expand_op, pp->desc.compact - 1, t));
    key += progs.back().source;
    key.push_back('\1');
  }
  auto it = s->shapes.find(key);
  if (it != s->shapes.end()) return it->second.get();
  std::unique_ptr<SrvShape> sh(new SrvShape());
  for (size_t p = 0; p < progs.size(); ++p) {
    SrvShape::Stage st;
    st.prog = progs[p];
    st.kernels = jit::compile(st.prog, true);
    const void* fn = (const void*)st.kernels.main;
    DQ_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, st.prog.smem_bytes));
    DQ_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&st.occ, fn, st.prog.block, st.prog.smem_bytes));
    if (st.kernels.heavy) {
      const void* hf = (const void*)st.kernels.heavy;
      DQ_CUDA(cudaFuncSetAttribute(hf, cudaFuncAttributeMaxDynamicSharedMemorySize, st.prog.smem_bytes));
      DQ_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&st.hocc, hf, st.prog.block, st.prog.smem_bytes));
    }
    if (st.occ < 1 || (st.kernels.heavy && st.hocc < 1)) return nullptr;
    st.mm_scan = plan->pipes[p]->mm_count;
    st.mm_res = plan->pipes[p]->mm_res;
    st.expand_op = plan->pipes[p]->expand_op;
    sh->stages.push_back(st);
  }
  SrvShape* raw = sh.get();
  s->shapes[key] = std::move(sh);
  return raw;
}

// Appends `n` bytes of `src` to a parameter blob at a 256-byte boundary; returns the offset.
size_t blob_put(std::vector<uint8_t>& blob, const void* src, size_t n) {
  const size_t off = align_up(blob.size(), 256);
  blob.resize(off + n);
  if (n) memcpy(blob.data() + off, src, n);
  return off;
}

// One launch sequence for the batch's members on the slot's stream: resets of
// all members' tables, every stage's many-instance kernel (with its shared
// deferral and bucket scans), a pack of all results, one copy back.
void srv_dispatch_batch(dq_server* s, SrvSlot& slot, SrvShape* sh) {
  SrvBatch& B = *slot.batch;
  dq_ctx* ctx = s->ctx;
  cudaStream_t st = slot.st;
  const int K = (int)B.members.size();
  {
    std::lock_guard<std::mutex> lk(s->mu);
    const double t = now_ms();
    for (auto& m : B.members) {
      m.first->t_dispatch = t;
      m.first->info.bytes = m.second->bytes;
    }
  }
  const uint64_t full = (uint64_t)std::max(s->cfg.batch_max, K);
  grow(B.status, 4);
  grow(B.rows, (size_t)full * 8);
  while (B.heavy.size() < sh->stages.size()) B.heavy.emplace_back(new HeavyBufs());
  std::vector<uint8_t> blob;
  struct StageArgs {
    size_t descs = 0, bprefix = 0, segs = 0;
    uint64_t blocks = 0, scan_blocks = 0;
    int grid = 1;
    DevHeavy heavy{};
  };
  std::vector<StageArgs> sa(sh->stages.size());
  uint64_t max_scan_blocks = 0;
  for (size_t p = 0; p < sh->stages.size(); ++p) {
    const SrvShape::Stage& S = sh->stages[p];
    std::vector<DevPipe> descs(K);
    std::vector<int64_t> prefix(K + 1, 0);
    const int64_t span = (int64_t)S.prog.block * S.prog.rows_per_thread;
    int64_t rows_all = 0;
    uint64_t build_rows = 0;
    for (int i = 0; i < K; ++i) {
      const dq_plan& pl = *B.members[i].second->plan;
      const PipeRec& pi = *pl.pipes[p];
      descs[i] = pi.dev;
      descs[i].status = B.status.as<int32_t>();
      const int64_t rows = pi.dev.nrows_dev ? (int64_t)pl.res[pi.dev.source_res]->dev.cap : pi.dev.nrows;
      prefix[i + 1] = prefix[i] + (rows + span - 1) / span;
      rows_all += rows;
      if (S.expand_op >= 0) {
        const uint64_t b = std::max<uint64_t>(pl.res[pi.desc.ops[S.expand_op].res]->pay_rows, 1);
        build_rows += b;
        sh->member_rows = std::max<uint64_t>(sh->member_rows, (uint64_t)std::max<int64_t>(rows, 1));
        sh->member_build = std::max(sh->member_build, b);
      }
    }
    if (S.expand_op >= 0) {
      const DevHeavy& proto = B.members[0].second->plan->pipes[p]->dev.heavy;
      auto sizes = [&](uint64_t rows, uint64_t build, uint64_t k, uint32_t& cap, uint32_t& gcap) {
        cap = (uint32_t)std::min<uint64_t>(std::max<uint64_t>(rows, 1), 1 << 20);
        const uint64_t groups =
            std::min<uint64_t>(cap, build / (std::max<uint64_t>(proto.threshold, kBatchGroupThreshold) + 1) + k);
        gcap = (uint32_t)std::min<uint64_t>(std::max<uint64_t>(64, 2 * groups), 0xfffffff0ull);
      };
      uint32_t cap, gcap, cap_full, gcap_full;
      sizes((uint64_t)rows_all, build_rows, (uint64_t)K, cap, gcap);
      sizes(full * sh->member_rows, full * sh->member_build, full, cap_full, gcap_full);
      B.heavy[p]->bind(proto, std::max(cap, cap_full), std::max(gcap, gcap_full));  // capacity for a full batch
      sa[p].heavy = B.heavy[p]->bind(proto, cap, gcap);
      for (int i = 0; i < K; ++i) {
        const uint64_t threshold = std::max<uint64_t>(descs[i].heavy.threshold, kBatchGroupThreshold);
        descs[i].heavy = sa[p].heavy;
        descs[i].heavy.threshold = threshold;
        descs[i].tile_counter = B.heavy[p]->units.as<uint32_t>();
      }
    }
    sa[p].blocks = (uint64_t)prefix[K];
    sa[p].grid = (int)std::max<int64_t>(1, std::min<int64_t>((int64_t)ctx->sms * S.occ, prefix[K]));
    sa[p].descs = blob_put(blob, descs.data(), descs.size() * sizeof(DevPipe));
    sa[p].bprefix = blob_put(blob, prefix.data(), prefix.size() * sizeof(int64_t));
    if (S.mm_scan) {
      std::vector<BatchScanSeg> segs(K);
      uint64_t blocks = 0;
      for (int i = 0; i < K; ++i) {
        const DevRes& R = B.members[i].second->plan->res[S.mm_res]->dev;
        segs[i].counts = R.counts;
        segs[i].offsets = R.offsets;
        segs[i].n = R.cap;
        segs[i].block0 = blocks;
        segs[i].nblocks = batch_scan_blocks(R.cap);
        blocks += segs[i].nblocks;
      }
      sa[p].segs = blob_put(blob, segs.data(), segs.size() * sizeof(BatchScanSeg));
      sa[p].scan_blocks = blocks;
      max_scan_blocks = std::max(max_scan_blocks, blocks);
    }
  }
  // resets and the result pack of every member
  std::vector<BatchReset> resets;
  std::vector<BatchPack> packs;
  B.col_off.assign(K, std::vector<uint64_t>());
  uint64_t off = 0;
  for (int i = 0; i < K; ++i) {
    const dq_plan& pl = *B.members[i].second->plan;
    for (auto& rp : pl.res) {
      const ResRec& r = *rp;
      BatchReset op{};
      switch (r.desc.kind) {
        case DQ_RES_UNIQUE:
          if (r.dev.bitmap) op.ptr = r.dev.slots, op.n = r.dev.bitmap == 1 ? (r.dev.cap * 4 + 7) / 8 : r.dev.cap,
                            op.value = 0, op.kind = 0;
          else op.ptr = r.dev.slots, op.n = (r.dev.cap + 1) * r.dev.words, op.value = kEmpty, op.kind = 0;
          break;
        case DQ_RES_AGG:
          op.ptr = r.dev.slots, op.n = r.dev.cap + 1, op.kind = 2, op.words = r.dev.words;
          op.val_word = r.dev.val_word, op.naggs = r.dev.naggs;
          for (int j = 0; j < r.dev.naggs && j < 16; ++j) op.reds |= (uint64_t)(r.dev.agg_red[j] & 15) << (4 * j);
          break;
        case DQ_RES_MULTI:
          op.ptr = r.dev.counts, op.n = r.dev.cap, op.value = 0, op.kind = 1;
          break;
        case DQ_RES_OUTPUT:
          op.ptr = r.dev.cursor, op.n = 1, op.value = 0, op.kind = 0;
          break;
      }
      resets.push_back(op);
    }
    const ResRec& o = *pl.res[pl.result_res];
    const uint64_t off0 = off;
    for (int j = 0; j < o.desc.npay; ++j) {
      BatchPack pk{};
      pk.src = o.dev.pay[j];
      pk.cursor = o.dev.cursor;
      pk.cap = o.dev.cap;
      pk.width = ctype_width(o.desc.pay_ctype[j]);
      pk.dst = off;
      pk.rows_out = j == 0 ? B.rows.as<uint64_t>() + i : nullptr;
      B.col_off[i].push_back(off);
      off += align_up(o.dev.cap * (uint64_t)pk.width, 16);
      packs.push_back(pk);
    }
    sh->member_out = std::max(sh->member_out, off - off0);
  }
  const size_t resets_off = blob_put(blob, resets.data(), resets.size() * sizeof(BatchReset));
  const size_t packs_off = blob_put(blob, packs.data(), packs.size() * sizeof(BatchPack));
  B.packed_bytes = std::max<uint64_t>(off, 16);
  const uint64_t packed_full = std::max<uint64_t>(B.packed_bytes, full * sh->member_out);
  const size_t blob_full = std::max<size_t>(blob.size(), (size_t)(blob.size() * full / (uint64_t)K) + 4096);
  grow(B.packed, packed_full);
  grow(B.partials, std::max<uint64_t>(max_scan_blocks, 1) * 4 * full / (uint64_t)K);
  const size_t out_need = packed_full + (size_t)full * 8 + 16;
  if (B.host_out_cap < B.packed_bytes + (size_t)K * 8 + 16) {
    if (B.host_out) cudaFreeHost(B.host_out);
    B.host_out = nullptr;
    B.host_out_cap = out_need + out_need / 2;
    DQ_CUDA(cudaMallocHost((void**)&B.host_out, B.host_out_cap));
  }
  if (B.host_params_cap < blob.size()) {
    if (B.host_params) cudaFreeHost(B.host_params);
    B.host_params = nullptr;
    B.host_params_cap = blob_full + blob_full / 2;
    DQ_CUDA(cudaMallocHost((void**)&B.host_params, B.host_params_cap));
  }
  grow(B.params, blob_full);
  memcpy(B.host_params, blob.data(), blob.size());
  uint8_t* dev = B.params.as<uint8_t>();
  int launches = 0;
  DQ_CUDA(cudaMemcpyAsync(dev, B.host_params, blob.size(), cudaMemcpyHostToDevice, st));
  DQ_CUDA(cudaMemsetAsync(B.status.ptr, 0, 4, st));
  DQ_CUDA(launch_batch_reset(reinterpret_cast<const BatchReset*>(dev + resets_off), (int)resets.size(), ctx->sms, st));
  ++launches;
  for (size_t p = 0; p < sh->stages.size(); ++p) {
    const SrvShape::Stage& S = sh->stages[p];
    const DevPipe* d = reinterpret_cast<const DevPipe*>(dev + sa[p].descs);
    const int64_t* pre = reinterpret_cast<const int64_t*>(dev + sa[p].bprefix);
    int n = K;
    if (S.expand_op >= 0) {
      HeavyBufs& hb = *B.heavy[p];
      DQ_CUDA(cudaMemsetAsync(hb.count.ptr, 0, 8, st));
      DQ_CUDA(cudaMemsetAsync(hb.units.ptr, 0, 4, st));
      DQ_CUDA(cudaMemsetAsync(hb.gkey.ptr, 0xff, (size_t)sa[p].heavy.gcap * 8, st));
      DQ_CUDA(cudaMemsetAsync(hb.gcnt.ptr, 0, (size_t)sa[p].heavy.gcap * 4, st));
    }
    void* args[] = {(void*)&d, (void*)&pre, (void*)&n};
    DQ_CUDA(cudaLaunchKernel((const void*)S.kernels.main, dim3(sa[p].grid), dim3(S.prog.block), args,
                             (size_t)S.prog.smem_bytes, st));
    ++launches;
    if (S.expand_op >= 0) {
      DQ_CUDA(launch_heavy_group(sa[p].heavy, B.status.as<int32_t>(), ctx->sms, st));
      void* hargs[] = {(void*)&d, (void*)&n};
      DQ_CUDA(cudaLaunchKernel((const void*)S.kernels.heavy, dim3(ctx->sms * S.hocc), dim3(S.prog.block), hargs,
                               (size_t)S.prog.smem_bytes, st));
      launches += 4;
    }
    if (S.mm_scan) {
      DQ_CUDA(launch_batch_scan(reinterpret_cast<const BatchScanSeg*>(dev + sa[p].segs), K, sa[p].scan_blocks,
                                B.partials.as<uint32_t>(), st));
      launches += 3;
    }
  }
  DQ_CUDA(launch_batch_pack(reinterpret_cast<const BatchPack*>(dev + packs_off), (int)packs.size(),
                            B.packed.as<uint8_t>(), ctx->sms, st));
  ++launches;
  DQ_CUDA(cudaMemcpyAsync(B.host_out, B.packed.ptr, B.packed_bytes, cudaMemcpyDeviceToHost, st));
  DQ_CUDA(cudaMemcpyAsync(B.host_out + B.packed_bytes, B.rows.ptr, (size_t)K * 8, cudaMemcpyDeviceToHost, st));
  DQ_CUDA(cudaMemcpyAsync(B.host_out + B.packed_bytes + (size_t)K * 8, B.status.ptr, 4, cudaMemcpyDeviceToHost, st));
  DQ_CUDA(cudaEventRecord(slot.done, st));
  B.launches = launches;
  std::lock_guard<std::mutex> lk(s->mu);
  ++s->batches;
  s->batched += (uint64_t)K;
}

void srv_finish(dq_server* s, SrvReq* r, int status, const std::string& err, dq_result* res);
void srv_release(dq_server* s, SrvReq* r, PoolEntry* pe);

// A completed batch: every member's result, or (a member's table overflowed)
// every member back to the front of the queue to run alone, where tables grow.
void srv_complete_batch(dq_server* s, SrvSlot& slot) {
  SrvBatch& B = *slot.batch;
  const int K = (int)B.members.size();
  int32_t status = 0;
  memcpy(&status, B.host_out + B.packed_bytes + (size_t)K * 8, 4);
  status &= ~kInfoMask;
  std::vector<std::pair<SrvReq*, PoolEntry*>> members;
  members.swap(B.members);
  if (status != 0) {
    for (auto& m : members) srv_release(s, m.first, m.second);
    std::lock_guard<std::mutex> lk(s->mu);
    for (auto it = members.rbegin(); it != members.rend(); ++it) {
      it->first->solo = true;
      it->first->t_dispatch = 0;
      s->pending.push_front(it->first);
    }
    return;
  }
  const uint64_t* rows = reinterpret_cast<const uint64_t*>(B.host_out + B.packed_bytes);
  for (int i = 0; i < K; ++i) {
    SrvReq* r = members[i].first;
    PoolEntry* pe = members[i].second;
    dq_result* res = nullptr;
    try {
      res = packed_result(pe->plan.get(), B.host_out, B.col_off[i], rows[i], slot.st);
    } catch (const DqError& e) {
      srv_release(s, r, pe);
      srv_finish(s, r, e.code, e.what(), nullptr);
      continue;
    }
    r->info.kernel_launches += B.launches;
    srv_release(s, r, pe);
    srv_finish(s, r, DQ_OK, "", res);
  }
}

// Waiting requests of the shape of the oldest one that have an idle pooled
// plan, up to batch_max, taken out of the queue (none when the oldest
// request runs alone or its shape is not known yet).
std::vector<std::pair<SrvReq*, PoolEntry*>> srv_take_batch(dq_server* s, SrvShape** shape) {
  std::vector<std::pair<SrvReq*, PoolEntry*>> out;
  std::lock_guard<std::mutex> lk(s->mu);
  if (s->pending.empty() || s->cfg.batch_max <= 1) return out;
  // large requests run alone: the many-instance kernels pay off for requests
  // whose launches, not their rows, dominate (their aggregates go to global
  // tables, without a plain kernel's CTA-local pre-aggregation)
  const uint64_t rows_max = s->cfg.batch_rows_max > 0 ? (uint64_t)s->cfg.batch_rows_max : (1ull << 18);
  SrvReq* head = s->pending.front();
  if (head->solo || head->desc->rows > rows_max) return out;
  auto sit = s->shape_of.find(head->desc->key);
  if (sit == s->shape_of.end() || !sit->second) return out;
  SrvShape* sh = sit->second;
  size_t seen = 0;
  for (auto it = s->pending.begin(); it != s->pending.end() && (int)out.size() < s->cfg.batch_max && seen < 1024;
       ++seen) {
    SrvReq* r = *it;
    auto q = s->shape_of.find(r->desc->key);
    PoolEntry* pe = nullptr;
    if (!r->solo && r->desc->rows <= rows_max && q != s->shape_of.end() && q->second == sh) {
      auto& v = s->pool[r->desc->key];
      for (auto& e : v)
        if (!e->busy) {
          pe = e.get();
          break;
        }
    }
    if (!pe) {
      ++it;
      continue;
    }
    pe->busy = true;
    out.emplace_back(r, pe);
    it = s->pending.erase(it);
  }
  *shape = sh;
  return out;
}

PoolEntry* srv_acquire(dq_server* s, SrvReq* r) {
  auto& v = s->pool[r->desc->key];
  for (auto& e : v)
    if (!e->busy) {
      e->busy = true;
      return e.get();
    }
  // a full pool waits for one of its plans (preparing more on the loop stalls
  // every slot, and the surplus would be freed later with a device sync)
  if (!v.empty() && v.size() >= (size_t)std::max(s->cfg.pool_per_query, 1)) return nullptr;
  // the bytes of a plan of this request when one exists, else the estimate
  const uint64_t need = v.empty() ? r->est : std::max(r->est, v.front()->bytes);
  if (!srv_make_room(s, need, r->desc->key)) {
    bool any_busy = false;
    for (auto& kv : s->pool)
      for (auto& e : kv.second) any_busy |= e->busy;
    if (!any_busy) throw DqError(DQ_ERR_ADMISSION, "request needs more device memory than the server's budget");
    return nullptr;
  }
  auto prepare = [&]() {
    std::unique_ptr<PoolEntry> e(new PoolEntry());
    e->plan = make_plan(s->ctx, &r->desc->d, PlanOpts());
    e->bytes = plan_bytes(e->plan.get());
    DQ_CUDA(cudaMallocHost((void**)&e->host_status, 4));
    s->mem += e->bytes;
    v.push_back(std::move(e));
    return v.back().get();
  };
  const bool first = v.empty();
  PoolEntry* got = prepare();
  got->busy = true;
  if (first && !s->shape_of.count(r->desc->key)) s->shape_of[r->desc->key] = srv_shape(s, got->plan.get());
  // the rest of the request's pool (graphs captured), while this request pays
  // for preparing one: concurrent copies of it later find a prepared plan
  // instead of stalling the loop to prepare and capture one
  const size_t want = (size_t)std::max(s->cfg.pool_per_query, 1);
  while (v.size() < want && s->mem + std::max(r->est, got->bytes) <= s->cfg.memory_budget) {  // never evicts
    PoolEntry* extra = prepare();
    srv_build_graph(extra, s->prep);
  }
  if (v.size() > 1) DQ_CUDA(cudaStreamSynchronize(s->prep));
  return got;
}

void srv_release(dq_server* s, SrvReq* r, PoolEntry* pe) {
  pe->busy = false;
  auto& v = s->pool[r->desc->key];
  int idle = 0;
  for (auto& e : v) idle += !e->busy;
  if (idle > s->cfg.pool_per_query)
    for (size_t i = 0; i < v.size(); ++i)
      if (v[i].get() == pe) {
        s->mem -= pe->bytes;
        v.erase(v.begin() + i);
        break;
      }
}

void srv_dispatch(dq_server* s, SrvSlot& slot, SrvReq* r, PoolEntry* pe) {
  slot.req = r;
  slot.pe = pe;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    r->t_dispatch = now_ms();
    r->info.bytes = pe->bytes;
  }
  if (!pe->exec && !pe->no_graph) srv_build_graph(pe, slot.st);
  if (pe->exec) {
    DQ_CUDA(cudaGraphLaunch(pe->exec, slot.st));
    slot.launches = pe->launches;
  } else {
    slot.launches = enqueue_run(pe->plan.get(), slot.st, pe->host_status);
  }
  DQ_CUDA(cudaEventRecord(slot.done, slot.st));
}

// A slot whose event completed: its result, or a re-run after growing the
// tables that overflowed.
void srv_complete(dq_server* s, SrvSlot& slot) {
  SrvReq* r = slot.req;
  PoolEntry* pe = slot.pe;
  int32_t status = *pe->host_status;
  bool regrow_heavy = false;
  if (status & kInfoMask) {
    regrow_heavy = (status & kInfoHeavyFull) != 0;
    status &= ~kInfoMask;
  }
  if (status != 0 && !(status & (kErrTimeout | kErrBadOp)) && r->attempts < 8) {
    ++r->attempts;
    const uint64_t before = pe->bytes;
    grow_plan(pe->plan.get(), status);
    pe->bytes = plan_bytes(pe->plan.get());
    s->mem = s->mem - before + pe->bytes;
    r->info.kernel_launches += slot.launches;
    pe->drop_graph();  // the tables moved: capture again
    pe->no_graph = false;
    srv_build_graph(pe, slot.st);
    if (pe->exec) {
      DQ_CUDA(cudaGraphLaunch(pe->exec, slot.st));
      slot.launches = pe->launches;
    } else {
      slot.launches = enqueue_run(pe->plan.get(), slot.st, pe->host_status);
    }
    DQ_CUDA(cudaEventRecord(slot.done, slot.st));
    return;
  }
  slot.req = nullptr;
  slot.pe = nullptr;
  if (status != 0) {
    srv_release(s, r, pe);
    srv_finish(s, r, status & kErrTimeout ? DQ_ERR_TIMEOUT : DQ_ERR_BAD_IR, "device status " + std::to_string(status),
               nullptr);
    return;
  }
  r->info.kernel_launches += slot.launches;
  dq_result* res;
  if (pe->exec) {
    res = srv_graph_result(pe, slot.st);
  } else {
    collect_timing(pe->plan.get(), slot.launches);
    res = read_result(pe->plan.get(), slot.st);
  }
  if (regrow_heavy) {
    // the result stands; later runs get the larger item capacity
    const uint64_t before = pe->bytes;
    if (grow_heavy(pe->plan.get())) {
      pe->bytes = plan_bytes(pe->plan.get());
      s->mem = s->mem - before + pe->bytes;
      pe->drop_graph();
      pe->no_graph = false;
      srv_build_graph(pe, slot.st);
    }
  }
  srv_release(s, r, pe);
  srv_finish(s, r, DQ_OK, "", res);
}

void srv_loop(dq_server* s) {
  cudaSetDevice(s->ctx->device);
  for (;;) {
    bool busy = false, progressed = false;
    {
      std::lock_guard<std::mutex> lk(s->ctx->mu);
      // completions
      for (auto& slot : s->slots) {
        if (!slot.busy()) continue;
        busy = true;
        const cudaError_t q = cudaEventQuery(slot.done);
        if (q == cudaErrorNotReady) continue;
        progressed = true;
        if (!slot.req) {  // a batch
          if (q == cudaSuccess) {
            srv_complete_batch(s, slot);
          } else {
            std::vector<std::pair<SrvReq*, PoolEntry*>> members;
            members.swap(slot.batch->members);
            for (auto& m : members) {
              srv_release(s, m.first, m.second);
              srv_finish(s, m.first, DQ_ERR_CUDA, std::string("batch execution: ") + cudaGetErrorString(q), nullptr);
            }
          }
          continue;
        }
        SrvReq* r = slot.req;
        try {
          if (q != cudaSuccess) throw DqError(DQ_ERR_CUDA, std::string("request execution: ") + cudaGetErrorString(q));
          srv_complete(s, slot);
        } catch (const DqError& e) {
          if (slot.pe) srv_release(s, r, slot.pe);
          slot.req = nullptr;
          slot.pe = nullptr;
          srv_finish(s, r, e.code, e.what(), nullptr);
        } catch (const std::exception& e) {
          if (slot.pe) srv_release(s, r, slot.pe);
          slot.req = nullptr;
          slot.pe = nullptr;
          srv_finish(s, r, DQ_ERR_CUDA, e.what(), nullptr);
        }
      }
      // admissions, oldest first, while a slot and memory are free: the oldest
      // request with the waiting requests of its shape as one batch when there
      // are several, else alone
      for (auto& slot : s->slots) {
        if (slot.busy()) continue;
        {
          SrvShape* sh = nullptr;
          std::vector<std::pair<SrvReq*, PoolEntry*>> take = srv_take_batch(s, &sh);
          if (take.size() >= 2) {
            if (!slot.batch) slot.batch.reset(new SrvBatch());
            slot.batch->members = take;
            try {
              srv_dispatch_batch(s, slot, sh);
            } catch (const std::exception& e) {
              std::vector<std::pair<SrvReq*, PoolEntry*>> members;
              members.swap(slot.batch->members);
              for (auto& m : members) {
                srv_release(s, m.first, m.second);
                const DqError* de = dynamic_cast<const DqError*>(&e);
                srv_finish(s, m.first, de ? de->code : DQ_ERR_CUDA, e.what(), nullptr);
              }
            }
            progressed = true;
            busy = true;
            continue;
          }
          if (take.size() == 1) {  // alone, on the plan it took
            try {
              srv_dispatch(s, slot, take[0].first, take[0].second);
            } catch (const std::exception& e) {
              srv_release(s, take[0].first, take[0].second);
              slot.req = nullptr;
              slot.pe = nullptr;
              const DqError* de = dynamic_cast<const DqError*>(&e);
              srv_finish(s, take[0].first, de ? de->code : DQ_ERR_CUDA, e.what(), nullptr);
            }
            progressed = true;
            busy = true;
            continue;
          }
        }
        SrvReq* r = nullptr;
        {
          std::lock_guard<std::mutex> lk2(s->mu);
          if (s->pending.empty()) break;
          r = s->pending.front();
        }
        PoolEntry* pe = nullptr;
        try {
          pe = srv_acquire(s, r);
          if (!pe) break;
          {
            std::lock_guard<std::mutex> lk2(s->mu);
            s->pending.pop_front();
            s->mem_peak = std::max(s->mem_peak, s->mem);
            s->mem_now = s->mem;
          }
          srv_dispatch(s, slot, r, pe);
        } catch (const DqError& e) {
          {
            std::lock_guard<std::mutex> lk2(s->mu);
            if (!s->pending.empty() && s->pending.front() == r) s->pending.pop_front();
          }
          if (pe) srv_release(s, r, pe);
          slot.req = nullptr;
          slot.pe = nullptr;
          srv_finish(s, r, e.code, e.what(), nullptr);
        } catch (const std::exception& e) {
          {
            std::lock_guard<std::mutex> lk2(s->mu);
            if (!s->pending.empty() && s->pending.front() == r) s->pending.pop_front();
          }
          if (pe) srv_release(s, r, pe);
          slot.req = nullptr;
          slot.pe = nullptr;
          srv_finish(s, r, DQ_ERR_CUDA, e.what(), nullptr);
        }
        progressed = true;
        busy = true;
      }
    }
    if (progressed) continue;
    if (busy) {
      std::this_thread::sleep_for(std::chrono::microseconds(4));
      continue;
    }
    std::unique_lock<std::mutex> lk(s->mu);
    if (s->stop && s->pending.empty()) break;
    if (s->pending.empty()) s->cv.wait_for(lk, std::chrono::milliseconds(2));
  }
}

}  // namespace

extern "C" {

int dq_server_start(dq_ctx* ctx, const dq_server_config* cfg, dq_server** out) {
  if (!ctx || !out) return fail(ctx, DQ_ERR_INVALID, "bad arguments");
  *out = nullptr;
  return guarded(ctx, [&]() {
    if (ctx->offline) throw DqError(DQ_ERR_UNSUPPORTED, "an offline context cannot serve");
    std::unique_ptr<dq_server> s(new dq_server());
    s->ctx = ctx;
    if (cfg) s->cfg = *cfg;
    if (s->cfg.slots <= 0) s->cfg.slots = 8;
    if (s->cfg.slots > 64) s->cfg.slots = 64;
    // no plan churn (freeing synchronises the device); batches take several plans of a request
    if (s->cfg.pool_per_query <= 0) s->cfg.pool_per_query = 2 * s->cfg.slots;
    if (s->cfg.batch_max <= 0) s->cfg.batch_max = 16;
    if (s->cfg.memory_budget == 0) s->cfg.memory_budget = 150ull << 30;
    {
      std::lock_guard<std::mutex> lk(ctx->mu);
      DQ_CUDA(cudaSetDevice(ctx->device));
      s->slots.resize(s->cfg.slots);
      for (auto& slot : s->slots) {
        DQ_CUDA(cudaStreamCreateWithFlags(&slot.st, cudaStreamNonBlocking));
        DQ_CUDA(cudaEventCreateWithFlags(&slot.done, cudaEventDisableTiming));
      }
      DQ_CUDA(cudaStreamCreateWithFlags(&s->prep, cudaStreamNonBlocking));
    }
    dq_server* raw = s.get();
    s->worker = std::thread(srv_loop, raw);
    *out = s.release();
    return (int)DQ_OK;
  });
}

}  // extern "C"

namespace {

uint64_t srv_submit(dq_server* s, const std::shared_ptr<DescCopy>& desc, uint64_t est) {
  std::unique_ptr<SrvReq> r(new SrvReq());
  r->desc = desc;
  r->est = est;
  std::lock_guard<std::mutex> lk(s->mu);
  if (s->stop) throw DqError(DQ_ERR_INVALID, "server is stopping");
  r->id = s->next_id++;
  r->t_submit = now_ms();
  if (s->submitted == 0) s->t_first = r->t_submit;
  ++s->submitted;
  const uint64_t id = r->id;
  s->pending.push_back(r.get());
  s->reqs[id] = std::move(r);
  s->cv.notify_all();
  return id;
}

// Waits for a request; returns its status, fills *out and *info.
int srv_wait(dq_server* s, uint64_t ticket, dq_result** out, dq_request_info* info) {
  std::unique_lock<std::mutex> lk(s->mu);
  auto it = s->reqs.find(ticket);
  if (it == s->reqs.end()) return fail(s->ctx, DQ_ERR_NOT_FOUND, "unknown ticket");
  SrvReq* r = it->second.get();
  s->cv.wait(lk, [&]() { return r->done; });
  const int status = r->status;
  if (info) *info = r->info;
  *out = r->result;
  if (status != DQ_OK) s->ctx->error = r->error;
  s->reqs.erase(it);
  return status;
}

// A request of a shape this server has not seen: its kernels (the plan's and
// the many-instance ones its batches use) are generated under the context lock
// with no device work, then compiled in the submitting thread without any lock
// held.  The request loop's preparation of it then finds them in the compiled
// kernel cache instead of compiling on the loop, where it would hold up every
// request in flight.
void precompile(dq_server* s, const DescCopy& d) {
  std::vector<jit::Program> progs;
  {
    std::lock_guard<std::mutex> lk(s->ctx->mu);
    if (!s->compiled.insert(d.key).second) return;
    try {
      OfflineScope off(true);
      CollectScope cs(&progs);
      std::unique_ptr<dq_plan> plan = make_plan(s->ctx, &d.d, PlanOpts());
      if (s->cfg.batch_max != 1)
        for (auto& pp : plan->pipes) {
          if (!pp->jit) continue;
          jit::Tuning t = plan->opts.tuning;
          t.batched = true;
          progs.push_back(jit::generate(pp->dev, pp->expand_op, pp->desc.compact - 1, t));
        }
    } catch (const std::exception&) {
      return;  // the loop's own preparation reports what is wrong with the request
    }
  }
  for (auto& pr : progs) {
    try {
      jit::compile(pr, false);
    } catch (const std::exception&) {
    }
  }
}

}  // namespace

extern "C" {

int dq_server_submit(dq_server* s, const dq_plan_desc* desc, uint64_t* ticket) {
  if (!s || !desc || !ticket) return DQ_ERR_INVALID;
  return guarded(s->ctx, [&]() {
    std::shared_ptr<DescCopy> d = copy_desc(desc);
    precompile(s, *d);
    uint64_t est;
    {
      std::lock_guard<std::mutex> lk(s->ctx->mu);
      est = estimate_bytes(s->ctx, d->d);
      d->rows = scanned_rows(s->ctx, d->d);
    }
    *ticket = srv_submit(s, d, est);
    return (int)DQ_OK;
  });
}

int dq_server_replay(dq_server* s, int32_t nq, const dq_plan_desc* queries, int64_t nreq, const double* arrival_ms,
                     const int32_t* query_of, dq_request_info* infos) {
  if (!s || nq <= 0 || !queries || nreq < 0 || (nreq > 0 && (!arrival_ms || !query_of || !infos)))
    return DQ_ERR_INVALID;
  return guarded(s->ctx, [&]() {
    std::vector<std::shared_ptr<DescCopy>> descs;
    std::vector<uint64_t> est;
    for (int q = 0; q < nq; ++q) descs.push_back(copy_desc(&queries[q]));
    // the driver holds every query before the first arrival: unseen shapes are
    // compiled now, as their submitters would have compiled them
    for (auto& d : descs) precompile(s, *d);
    {
      std::lock_guard<std::mutex> lk(s->ctx->mu);
      for (auto& d : descs) {
        est.push_back(estimate_bytes(s->ctx, d->d));
        d->rows = scanned_rows(s->ctx, d->d);
      }
    }
    for (int64_t i = 0; i < nreq; ++i)
      if (query_of[i] < 0 || query_of[i] >= nq) throw DqError(DQ_ERR_INVALID, "request names no query");
    std::vector<uint64_t> tickets((size_t)nreq);
    const double t0 = now_ms();
    for (int64_t i = 0; i < nreq; ++i) {
      const double target = t0 + arrival_ms[i];
      for (double t = now_ms(); t < target; t = now_ms()) {
        if (target - t > 0.3) std::this_thread::sleep_for(std::chrono::microseconds((int64_t)((target - t - 0.2) * 1e3)));
      }
      tickets[i] = srv_submit(s, descs[query_of[i]], est[query_of[i]]);
    }
    int first_error = DQ_OK;
    for (int64_t i = 0; i < nreq; ++i) {
      dq_result* res = nullptr;
      const int st = srv_wait(s, tickets[i], &res, &infos[i]);
      if (res) delete res;
      if (st != DQ_OK && first_error == DQ_OK) first_error = st;
    }
    return first_error;
  });
}

int dq_plan_run_sequence(dq_plan* const* plans, int32_t nplans, int64_t nreq, const int32_t* plan_of, double* ms_out) {
  if (!plans || nplans <= 0 || nreq < 0 || (nreq > 0 && (!plan_of || !ms_out))) return DQ_ERR_INVALID;
  for (int64_t i = 0; i < nreq; ++i) {
    if (plan_of[i] < 0 || plan_of[i] >= nplans || !plans[plan_of[i]]) return DQ_ERR_INVALID;
    const double t = now_ms();
    dq_result* res = nullptr;
    const int st = dq_plan_execute(plans[plan_of[i]], nullptr, &res);
    if (st != DQ_OK) return st;
    dq_result_free(res);
    ms_out[i] = now_ms() - t;
  }
  return DQ_OK;
}

int dq_server_wait(dq_server* s, uint64_t ticket, dq_result** out, dq_request_info* info) {
  if (!s || !out) return DQ_ERR_INVALID;
  *out = nullptr;
  return srv_wait(s, ticket, out, info);
}

int dq_server_stats_get(dq_server* s, dq_server_stats* out) {
  if (!s || !out) return DQ_ERR_INVALID;
  std::lock_guard<std::mutex> lk(s->mu);
  memset(out, 0, sizeof(*out));
  out->submitted = s->submitted;
  out->completed = s->completed;
  out->failed = s->failed;
  out->memory_in_use = s->mem_now;
  out->memory_peak = s->mem_peak;
  if (!s->lat.empty()) {
    std::vector<double> v = s->lat;
    std::sort(v.begin(), v.end());
    auto pct = [&](double q) { return v[std::min(v.size() - 1, (size_t)(q * (v.size() - 1) + 0.5))]; };
    out->p50_ms = pct(0.50);
    out->p99_ms = pct(0.99);
    double sum = 0;
    for (double x : v) sum += x;
    out->mean_ms = sum / v.size();
  }
  out->span_ms = s->t_last > s->t_first ? s->t_last - s->t_first : 0;
  out->batches = s->batches;
  out->batched = s->batched;
  return DQ_OK;
}

void dq_server_stop(dq_server* s) {
  if (!s) return;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stop = true;
    s->cv.notify_all();
  }
  if (s->worker.joinable()) s->worker.join();
  {
    std::lock_guard<std::mutex> lk(s->ctx->mu);
    cudaSetDevice(s->ctx->device);
    for (auto& slot : s->slots) {
      if (slot.st) cudaStreamSynchronize(slot.st);
    }
    if (s->prep) cudaStreamSynchronize(s->prep);
    s->pool.clear();
    for (auto& slot : s->slots) {
      if (slot.done) cudaEventDestroy(slot.done);
      if (slot.st) cudaStreamDestroy(slot.st);
    }
    if (s->prep) cudaStreamDestroy(s->prep);
  }
  for (auto& kv : s->reqs)
    if (kv.second->result) delete kv.second->result;
  delete s;
}

}  // extern "C"
