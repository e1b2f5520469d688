// Pipeline kernels of the B200 backend (sm_100a).
//
// One persistent kernel executes one pipeline of a plan: it streams the source
// in tiles of `tile` rows, staged from HBM into shared memory with TMA bulk
// copies (cp.async.bulk + mbarrier, multi-stage), and runs the pipeline's
// operator list over each tile column-wise:
//
//   * expression ops evaluate for every selected row and write a register slot;
//   * filters and probes keep a subset of rows: the tile's selection vector is
//     compacted block-wide (warp ballot/popc + one scan), so every later op
//     runs on full warps.  This is the lane-refill idea of the reference
//     (dogqc/cudaDivergenceBuffer.py:11-283) applied at tile granularity;
//   * a multimap probe opens an expansion level: the (row, match) pairs of the
//     tile are produced in chunks of `tile` pairs and the rest of the pipeline
//     runs once per chunk.  This generalises the reference's warp-level
//     push-down expansion (dogqc/hashJoins.py:599-681) to the whole CTA; ranges
//     longer than a threshold are deferred to a second launch in which all CTAs
//     split them (the skewed heads of Zipf build sides);
//   * the sink (aggregate / build / emit) ends the list.
//
// Values, hashing and table probing are shared with the generated pipeline
// kernels (dq_common.cuh).
#include <cuda_runtime.h>
#include <stdint.h>

#include "dq_common.cuh"

namespace dq {

constexpr int kWarps = kThreads / 32;
constexpr int kMaxItems = 8;                 // tile <= kThreads * kMaxItems

// ------------------------------------------------------------ CTA state --

struct Cta {
  uint8_t* smem;
  const uint8_t* stage;                 // staged columns of the current tile
  int64_t tile_start;                   // first source row of the tile
  int heavy;                            // executing deferred expansion units
  uint8_t* reg[DQ_MAX_LEVELS];
  uint16_t* sel[DQ_MAX_LEVELS];
  uint16_t* par[DQ_MAX_LEVELS];
  uint32_t* match[DQ_MAX_LEVELS];
  uint32_t* eoff[DQ_MAX_LEVELS];        // expansion bookkeeping per parent level
  uint32_t* ecnt[DQ_MAX_LEVELS];
  uint32_t* epos[DQ_MAX_LEVELS];
  uint8_t* flags;                       // per-row probe results
  uint64_t* stash;
};

__shared__ int32_t s_scan[kMaxItems * kWarps + 64];
__shared__ uint64_t s_bcast[8];

__device__ __forceinline__ int slot_row(const Cta& c, int slot_level, int level, int row) {
  for (int l = level; l > slot_level; --l) row = c.par[l][row];
  return row;
}

__device__ __forceinline__ const DevStr& str_of(const DevPipe& P, int s) { return P.strs[P.slots[s].src]; }

__device__ __forceinline__ void read_str(const DevPipe& P, const Cta& c, int s, int level, int row,
                                         const uint8_t*& ptr, int& len) {
  const DevSlot& sl = P.slots[s];
  int r = slot_row(c, sl.level, level, row);
  str_at(P.strs[sl.src], c.tile_start + r, ptr, len);
}

__device__ __forceinline__ uint64_t read_slot(const DevPipe& P, const Cta& c, int s, int level, int row) {
  const DevSlot& sl = P.slots[s];
  if (c.heavy && sl.level == 0) return c.stash[sl.stash];
  int r = slot_row(c, sl.level, level, row);
  uint64_t raw;
  switch (sl.kind) {
    case DQ_SLOT_COL:
      raw = ld(c.stage + P.cols[sl.src].smem_off + (size_t)r * sl.width, sl.width);
      break;
    case DQ_SLOT_REG:
      raw = ld(c.reg[sl.level] + sl.smem_off + (size_t)r * sl.width, sl.width);
      break;
    case DQ_SLOT_GATHER: {
      uint32_t m = c.match[sl.level][r];
      raw = ld(P.res[sl.res].pay[sl.src] + (size_t)m * sl.width, sl.width);
      break;
    }
    case DQ_SLOT_AGGKEY: {
      const DevRes& R = P.res[sl.res];
      uint64_t idx = (uint64_t)(c.tile_start + r);
      const uint64_t* slot = R.slots + idx * R.words;
      if (R.packed) {
        uint64_t tag = slot[0];
        if (idx == R.cap) tag = kEmpty;  // the slot reserved for the all-ones key
        raw = (R.nkeys == 1 && (R.key_ctype[0] == DQ_I64 || R.key_ctype[0] == DQ_U64))
                  ? tag : (tag >> (32 * sl.src)) & 0xffffffffull;
      } else {
        raw = slot[R.key_word + sl.src];
      }
      break;
    }
    case DQ_SLOT_AGGVAL: {
      const DevRes& R = P.res[sl.res];
      uint64_t idx = (uint64_t)(c.tile_start + r);
      raw = R.slots[idx * R.words + R.val_word + sl.src];
      break;
    }
    default:
      raw = 0;
  }
  return canon(raw, sl.ctype);
}

__device__ __forceinline__ void write_reg(const DevPipe& P, const Cta& c, int s, int row, uint64_t v) {
  const DevSlot& sl = P.slots[s];
  st(c.reg[sl.level] + sl.smem_off + (size_t)row * sl.width, sl.width, canon(v, sl.ctype));
}

// ------------------------------------------------------------ compaction --

// Keeps the selection entries whose predicate holds; order preserving.
// Element i of the selection is handled by thread (i % kThreads); all threads
// must call this with the same n.
template <class Keep>
__device__ int compact(uint16_t* sel, int n, Keep keep) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int items = (n + kThreads - 1) / kThreads;
  uint16_t v[kMaxItems];
  uint32_t bal[kMaxItems];
  bool kp[kMaxItems];
#pragma unroll
  for (int k = 0; k < kMaxItems; ++k) {
    kp[k] = false;
    bal[k] = 0;
    v[k] = 0;
    if (k < items) {
      int i = tid + k * kThreads;
      if (i < n) {
        v[k] = sel[i];
        kp[k] = keep(v[k]);
      }
      bal[k] = __ballot_sync(0xffffffffu, kp[k]);
      if (lane == 0) s_scan[k * kWarps + warp] = __popc(bal[k]);
    }
  }
  __syncthreads();
  if (warp == 0) {
    const int total_n = items * kWarps;
    int carry = 0;
    for (int base = 0; base < total_n; base += 32) {
      int x = (base + lane < total_n) ? s_scan[base + lane] : 0;
      int incl = x;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        int y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += y;
      }
      if (base + lane < total_n) s_scan[base + lane] = carry + incl - x;
      carry += __shfl_sync(0xffffffffu, incl, 31);
    }
    if (lane == 0) s_scan[kMaxItems * kWarps] = carry;
  }
  __syncthreads();
  const uint32_t lt = (1u << lane) - 1u;
#pragma unroll
  for (int k = 0; k < kMaxItems; ++k)
    if (k < items && kp[k]) sel[s_scan[k * kWarps + warp] + __popc(bal[k] & lt)] = v[k];
  int total = s_scan[kMaxItems * kWarps];
  __syncthreads();
  return total;
}

// Exclusive block scan of one value per thread; returns the total.
__device__ uint32_t block_exclusive_scan(uint32_t x, uint32_t& excl) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  uint32_t incl = x;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += y;
  }
  if (lane == 31) s_scan[warp] = (int32_t)incl;
  __syncthreads();
  if (warp == 0) {
    uint32_t w = lane < kWarps ? (uint32_t)s_scan[lane] : 0;
    uint32_t wi = w;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      uint32_t y = __shfl_up_sync(0xffffffffu, wi, o);
      if (lane >= o) wi += y;
    }
    if (lane < kWarps) s_scan[32 + lane] = (int32_t)(wi - w);
    if (lane == kWarps - 1) s_scan[63] = (int32_t)wi;
  }
  __syncthreads();
  excl = (uint32_t)s_scan[32 + warp] + incl - x;
  uint32_t total = (uint32_t)s_scan[63];
  __syncthreads();
  return total;
}

// ------------------------------------------------------------- hashing --

__device__ __forceinline__ void key_values(const DevPipe& P, const Cta& c, const DevRes& R, int list,
                                           int nlist, int level, int row, uint64_t* k) {
  for (int i = 0; i < nlist; ++i) k[i] = canon(read_slot(P, c, P.lists[list + i], level, row), R.key_ctype[i]);
}

// CTA-local aggregation table in shared memory: (ns+1) tags then accumulators.
struct LocalAgg {
  uint64_t* tags;
  uint64_t* acc;
  int ns;
};

__device__ __forceinline__ LocalAgg local_agg(const DevPipe& P, const Cta& c, const DevRes& R) {
  LocalAgg a;
  a.ns = R.smem_slots;
  a.tags = reinterpret_cast<uint64_t*>(c.smem + R.smem_off);
  a.acc = a.tags + (a.ns + 1);
  return a;
}

__device__ int local_slot(const LocalAgg& a, uint64_t tag, int nkeys) {
  if (nkeys == 0) {
    a.tags[0] = 0;  // mark the single group present
    return 0;
  }
  if (tag == kEmpty) {
    atomicCAS((unsigned long long*)&a.tags[a.ns], kEmpty, 0ull);
    return a.ns;
  }
  uint32_t idx = slot_of(tag, (uint32_t)a.ns);
  for (int n = 0; n < a.ns; ++n) {
    uint64_t t = *(volatile uint64_t*)&a.tags[idx];
    if (t == tag) return (int)idx;
    if (t == kEmpty) {
      uint64_t old = atomicCAS((unsigned long long*)&a.tags[idx], kEmpty, tag);
      if (old == kEmpty || old == tag) return (int)idx;
    }
    idx = (idx + 1 == (uint32_t)a.ns) ? 0 : idx + 1;
  }
  return -1;
}

// ---------------------------------------------------------------- ops --

struct Level {
  int level;   // current expansion level
  int n;       // selected rows at this level
};

__device__ void op_expr(const DevPipe& P, const Cta& c, const dq_op& op, const Level& L) {
  const uint16_t* sel = c.sel[L.level];
  for (int i = threadIdx.x; i < L.n; i += kThreads) {
    int row = sel[i];
    uint64_t r = 0;
    switch (op.kind) {
      case DQ_OP_ARITH: {
        uint64_t a = (op.flags & DQ_OPF_A_IMM) ? (uint64_t)op.imm : read_slot(P, c, op.a, L.level, row);
        uint64_t b = (op.flags & DQ_OPF_B_IMM) ? (uint64_t)op.imm : read_slot(P, c, op.b, L.level, row);
        r = arith(op.sub, op.ctype, a, b);
        break;
      }
      case DQ_OP_CMP: {
        uint64_t a = (op.flags & DQ_OPF_A_IMM) ? (uint64_t)op.imm : read_slot(P, c, op.a, L.level, row);
        uint64_t b = (op.flags & DQ_OPF_B_IMM) ? (uint64_t)op.imm : read_slot(P, c, op.b, L.level, row);
        r = compare(op.sub, op.ctype, a, b);
        break;
      }
      case DQ_OP_LOGIC: {
        uint64_t a = read_slot(P, c, op.a, L.level, row);
        if (op.sub == DQ_NOT) {
          r = a == 0;
        } else {
          uint64_t b = read_slot(P, c, op.b, L.level, row);
          r = op.sub == DQ_AND ? (a != 0 && b != 0) : (a != 0 || b != 0);
        }
        break;
      }
      case DQ_OP_CAST:
        r = canon((op.flags & DQ_OPF_A_IMM) ? (uint64_t)op.imm : read_slot(P, c, op.a, L.level, row), op.ctype);
        break;
      case DQ_OP_SELECT: {
        uint64_t cond = read_slot(P, c, op.a, L.level, row);
        if (cond) r = (op.flags & DQ_OPF_B_IMM) ? (uint64_t)op.imm : read_slot(P, c, op.b, L.level, row);
        else r = op.c >= 0 ? read_slot(P, c, op.c, L.level, row) : read_slot(P, c, op.dst, L.level, row);
        r = canon(r, op.ctype);
        break;
      }
      case DQ_OP_LIKE:
      case DQ_OP_STREQ: {
        const uint8_t* s;
        int ls;
        read_str(P, c, op.a, L.level, row, s, ls);
        const uint8_t* p = P.patterns + P.pat_off[op.res];
        int lp = P.pat_off[op.res + 1] - P.pat_off[op.res];
        if (op.kind == DQ_OP_LIKE) {
          r = like_match(s, ls, p, lp);
        } else {
          bool eq = ls == lp;
          for (int j = 0; eq && j < ls; ++j) eq = s[j] == p[j];
          r = eq;
        }
        break;
      }
    }
    write_reg(P, c, op.dst, row, r);
  }
}

// Unique-table probe: payload copied into register slots, then compaction.
__device__ int op_probe(const DevPipe& P, const Cta& c, const dq_op& op, const Level& L) {
  const DevRes& R = P.res[op.res];
  const uint16_t* sel = c.sel[L.level];
  uint8_t* found = c.flags;
  for (int i = threadIdx.x; i < L.n; i += kThreads) {
    int row = sel[i];
    uint64_t k[DQ_MAX_KEYS];
    key_values(P, c, R, op.list, op.nlist, L.level, row, k);
    uint64_t tag = key_tag(R, k);
    int64_t s = unique_find(R, tag, k);
    found[row] = s >= 0;
    if (s >= 0 && op.sub == DQ_JOIN_INNER) {
      const uint64_t* pay = R.slots + (uint64_t)s * R.words + R.val_word;
      for (int j = 0; j < op.nlist2; ++j) {
        int d = P.lists[op.list2 + j];
        if (d >= 0) write_reg(P, c, d, row, pay[j]);
      }
    }
  }
  __syncthreads();
  const bool anti = op.sub == DQ_JOIN_ANTI;
  return compact(c.sel[L.level], L.n, [&](int row) { return anti ? found[row] == 0 : found[row] != 0; });
}

__device__ void op_build(const DevPipe& P, const Cta& c, const dq_op& op, const Level& L) {
  const DevRes& R = P.res[op.res];
  const uint16_t* sel = c.sel[L.level];
  for (int i = threadIdx.x; i < L.n; i += kThreads) {
    int row = sel[i];
    uint64_t k[DQ_MAX_KEYS];
    key_values(P, c, R, op.list, op.nlist, L.level, row, k);
    int64_t s = unique_insert(P, R, key_tag(R, k), k);
    if (s >= 0) {
      uint64_t* pay = R.slots + (uint64_t)s * R.words + R.val_word;
      for (int j = 0; j < op.nlist2; ++j) pay[j] = read_slot(P, c, P.lists[op.list2 + j], L.level, row);
    }
  }
}

__device__ void op_mm(const DevPipe& P, const Cta& c, const dq_op& op, const Level& L) {
  const DevRes& R = P.res[op.res];
  const uint16_t* sel = c.sel[L.level];
  for (int i = threadIdx.x; i < L.n; i += kThreads) {
    int row = sel[i];
    uint64_t k[DQ_MAX_KEYS];
    key_values(P, c, R, op.list, op.nlist, L.level, row, k);
    uint64_t b = bucket_of(k, op.nlist, (uint32_t)R.cap);
    if (op.kind == DQ_OP_MM_COUNT) {
      atomicAdd(&R.counts[b], 1u);
    } else {
      uint32_t pos = R.offsets[b] + atomicAdd(&R.counts[b], 1u);
      for (int j = 0; j < op.nlist2; ++j)
        st(R.pay[j] + (size_t)pos * R.pay_width[j], R.pay_width[j],
           read_slot(P, c, P.lists[op.list2 + j], L.level, row));
    }
  }
}

__device__ void op_agg(const DevPipe& P, const Cta& c, const dq_op& op, const Level& L) {
  const DevRes& R = P.res[op.res];
  const uint16_t* sel = c.sel[L.level];
  const bool local = R.smem_slots > 0;
  LocalAgg la;
  if (local) la = local_agg(P, c, R);
  for (int i = threadIdx.x; i < L.n; i += kThreads) {
    int row = sel[i];
    uint64_t k[DQ_MAX_KEYS];
    key_values(P, c, R, op.list, op.nlist, L.level, row, k);
    uint64_t tag = key_tag(R, k);
    uint64_t* acc = nullptr;
    if (local) {
      int s = local_slot(la, tag, R.nkeys);
      if (s >= 0) acc = la.acc + (size_t)s * R.naggs;
    }
    if (!acc) {
      int64_t g = agg_slot_global(P, R, tag, k);
      if (g < 0) continue;
      acc = R.slots + (uint64_t)g * R.words + R.val_word;
    }
    for (int j = 0; j < R.naggs; ++j) {
      int src = P.lists[op.list2 + j];
      uint64_t v = src >= 0 ? read_slot(P, c, src, L.level, row) : 1;
      accumulate(acc + j, R.agg_red[j], v);
    }
  }
}

__device__ void op_emit(const DevPipe& P, const Cta& c, const dq_op& op, const Level& L) {
  const DevRes& R = P.res[op.res];
  const uint16_t* sel = c.sel[L.level];
  if (threadIdx.x == 0) s_bcast[0] = L.n ? atomicAdd((unsigned long long*)R.cursor, (unsigned long long)L.n) : 0;
  __syncthreads();
  uint64_t base = s_bcast[0];
  __syncthreads();
  if (base + L.n > R.cap) set_status(P, kErrOverflow);
  for (int i = threadIdx.x; i < L.n; i += kThreads) {
    uint64_t pos = base + i;
    if (pos >= R.cap) break;
    int row = sel[i];
    for (int j = 0; j < op.nlist; ++j)
      st(R.pay[j] + pos * R.pay_width[j], R.pay_width[j], read_slot(P, c, P.lists[op.list + j], L.level, row));
  }
}

// ------------------------------------------------------------ expansion --

struct Frame {
  int op;          // EXPAND op index
  int level;       // parent level
  int pn;          // selected parent rows
  uint32_t total;  // pairs of the parent selection
  uint32_t next;   // first pair of the next chunk
};

// Sets up an expansion over the selected rows of level L: ranges, deferral of
// wide ranges, and the exclusive scan of range lengths.  Returns total pairs.
__device__ uint32_t expand_setup(const DevPipe& P, const Cta& c, const dq_op& op, const Level& L) {
  const DevRes& R = P.res[op.res];
  const uint16_t* sel = c.sel[L.level];
  const int tid = threadIdx.x;
  const bool defer = L.level == 0 && P.heavy.cap > 0 && !c.heavy;
  // each thread owns a contiguous run of selection entries
  const int per = (L.n + kThreads - 1) / kThreads;
  const int i0 = min(tid * per, L.n), i1 = min(i0 + per, L.n);
  uint32_t* eoff = c.eoff[L.level];
  uint32_t* ecnt = c.ecnt[L.level];
  uint32_t* epos = c.epos[L.level];
  uint32_t local = 0;
  for (int i = i0; i < i1; ++i) {
    int row = sel[i];
    uint64_t k[DQ_MAX_KEYS];
    key_values(P, c, R, op.list, op.nlist, L.level, row, k);
    uint64_t b = bucket_of(k, op.nlist, (uint32_t)R.cap);
    uint32_t cnt = R.counts[b];
    uint32_t off = cnt ? R.offsets[b] : 0;
    if (defer && cnt > P.heavy.threshold) {
      uint32_t slot = atomicAdd(P.heavy.count, 1u);
      if (slot < P.heavy.cap) {
        uint64_t* it = P.heavy.items + (size_t)slot * P.heavy.words;
        it[0] = off;
        it[1] = cnt;
        int j = 0;
        for (int s = 0; s < P.nslots && j < P.heavy.nstash; ++s)
          if (P.slots[s].stash >= 0) it[2 + P.slots[s].stash] = read_slot(P, c, s, 0, row), ++j;
        cnt = 0;
      }
    }
    eoff[i] = off;
    ecnt[i] = cnt;
    local += cnt;
  }
  uint32_t excl;
  uint32_t total = block_exclusive_scan(local, excl);
  for (int i = i0; i < i1; ++i) {
    epos[i] = excl;
    excl += ecnt[i];
  }
  __syncthreads();
  return total;
}

// Produces pairs [base, base+n) of the expansion as level L+1 rows, checks the
// build keys, and returns the number of matching rows.
__device__ int expand_chunk(const DevPipe& P, const Cta& c, const dq_op& op, int parent_level, int parent_n,
                            uint32_t base, int n) {
  const int tid = threadIdx.x;
  const int lv = parent_level + 1;
  const uint16_t* psel = c.sel[parent_level];
  const int per = (n + kThreads - 1) / kThreads;
  const int j0 = min(tid * per, n), j1 = min(j0 + per, n);
  const uint32_t* eoff = c.eoff[parent_level];
  const uint32_t* ecnt = c.ecnt[parent_level];
  const uint32_t* epos = c.epos[parent_level];
  if (j0 < j1) {
    uint32_t g = base + j0;
    // last parent whose first pair is <= g
    int lo = 0, hi = parent_n;
    while (lo < hi) {
      int mid = (lo + hi) >> 1;
      if (epos[mid] <= g) lo = mid + 1;
      else hi = mid;
    }
    int i = lo - 1;
    for (int j = j0; j < j1; ++j, ++g) {
      while (g >= epos[i] + ecnt[i]) ++i;
      c.par[lv][j] = psel[i];
      c.match[lv][j] = eoff[i] + (g - epos[i]);
      c.sel[lv][j] = (uint16_t)j;
    }
  }
  __syncthreads();
  // key check: build keys are payload columns gathered at the new level
  return compact(c.sel[lv], n, [&](int row) {
    bool eq = true;
    for (int q = 0; q < op.nlist; ++q) {
      uint64_t pk = read_slot(P, c, P.lists[op.list + q], lv, row);
      uint64_t bk = read_slot(P, c, P.lists[op.list2 + q], lv, row);
      int t = P.res[op.res].key_ctype[q];
      eq &= canon(pk, t) == canon(bk, t);
    }
    return eq;
  });
}

// Runs ops [start, nops) over the current selection; handles expansion frames.
__device__ void run_ops(const DevPipe& P, Cta& c, int start, Level L) {
  Frame fr[DQ_MAX_LEVELS];
  int depth = 0;
  int k = start;
  while (true) {
    if (k >= P.nops) {
      // resume the innermost expansion that still has chunks
      bool resumed = false;
      while (depth > 0) {
        Frame& f = fr[depth - 1];
        if (f.next < f.total) {
          uint32_t n = min((uint32_t)P.exp_cap, f.total - f.next);
          int got = expand_chunk(P, c, P.ops[f.op], f.level, f.pn, f.next, (int)n);
          f.next += n;
          L.level = f.level + 1;
          L.n = got;
          k = f.op + 1;
          resumed = true;
          break;
        }
        --depth;
      }
      if (!resumed) return;
      continue;
    }
    const dq_op& op = P.ops[k];
    switch (op.kind) {
      case DQ_OP_ARITH:
      case DQ_OP_CMP:
      case DQ_OP_LOGIC:
      case DQ_OP_CAST:
      case DQ_OP_SELECT:
      case DQ_OP_LIKE:
      case DQ_OP_STREQ:
        op_expr(P, c, op, L);
        __syncthreads();
        ++k;
        break;
      case DQ_OP_FILTER: {
        L.n = compact(c.sel[L.level], L.n,
                      [&](int row) { return read_slot(P, c, op.a, L.level, row) != 0; });
        ++k;
        break;
      }
      case DQ_OP_PROBE:
        L.n = op_probe(P, c, op, L);
        ++k;
        break;
      case DQ_OP_EXPAND: {
        if (L.level + 1 >= DQ_MAX_LEVELS) {
          set_status(P, kErrBadOp);
          return;
        }
        uint32_t total;
        if (c.heavy && L.level == 0) {
          total = c.ecnt[0][0];  // prepared by the heavy-unit loop
        } else {
          total = expand_setup(P, c, op, L);
        }
        fr[depth].op = k;
        fr[depth].level = L.level;
        fr[depth].pn = L.n;
        fr[depth].total = total;
        fr[depth].next = 0;
        ++depth;
        k = P.nops;  // the resume logic produces the first chunk
        break;
      }
      case DQ_OP_AGG:
        op_agg(P, c, op, L);
        __syncthreads();
        k = P.nops;
        break;
      case DQ_OP_BUILD:
        op_build(P, c, op, L);
        __syncthreads();
        k = P.nops;
        break;
      case DQ_OP_MM_COUNT:
      case DQ_OP_MM_SCATTER:
        op_mm(P, c, op, L);
        __syncthreads();
        k = P.nops;
        break;
      case DQ_OP_EMIT:
        op_emit(P, c, op, L);
        __syncthreads();
        k = P.nops;
        break;
      default:
        set_status(P, kErrBadOp);
        return;
    }
  }
}

// ------------------------------------------------------------- staging --

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
               : "memory");
}

__device__ __forceinline__ void tma_load_1d(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_addr(dst)),
      "l"(src), "r"(bytes), "r"(smem_addr(bar))
      : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t phase) {
  uint32_t done;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(done)
      : "r"(smem_addr(bar)), "r"(phase)
      : "memory");
  return done != 0;
}

// Bounded wait; on exhaustion flags a timeout (the data is then not used).
__device__ __forceinline__ bool mbar_wait(const DevPipe& P, uint64_t* bar, uint32_t phase) {
  for (long long i = 0; i < (1ll << 24); ++i)
    if (mbar_try_wait(bar, phase)) return true;
  set_status(P, kErrTimeout);
  return false;
}

// Issues the copies of tile `t` into stage buffer `dst` (thread 0 only).
__device__ void stage_issue(const DevPipe& P, uint8_t* dst, int64_t t, int64_t nrows, uint64_t* bar) {
  const int64_t start = t * P.tile;
  const int64_t rows = min((int64_t)P.tile, nrows - start);
  uint32_t total = 0;
  for (int i = 0; i < P.ncols; ++i) total += (uint32_t)((rows * P.cols[i].width + 15) & ~15ll);
  mbar_expect_tx(bar, total);
  for (int i = 0; i < P.ncols; ++i) {
    const DevCol& col = P.cols[i];
    uint32_t bytes = (uint32_t)((rows * col.width + 15) & ~15ll);
    tma_load_1d(dst + col.smem_off, col.ptr + start * col.width, bytes, bar);
  }
}

// Plain cooperative copy of a tile (used when TMA staging is disabled).
__device__ void stage_plain(const DevPipe& P, uint8_t* dst, int64_t t, int64_t nrows) {
  const int64_t start = t * P.tile;
  const int64_t rows = min((int64_t)P.tile, nrows - start);
  for (int i = 0; i < P.ncols; ++i) {
    const DevCol& col = P.cols[i];
    int64_t bytes = (rows * col.width + 15) & ~15ll;
    const uint4* s = reinterpret_cast<const uint4*>(col.ptr + start * col.width);
    uint4* d = reinterpret_cast<uint4*>(dst + col.smem_off);
    for (int64_t j = threadIdx.x; j < bytes / 16; j += kThreads) d[j] = s[j];
  }
}

// ----------------------------------------------------------- the kernel --

__device__ void init_cta(const DevPipe& P, Cta& c, uint8_t* smem) {
  c.smem = smem;
  c.heavy = P.mode == 1;
  for (int l = 0; l < DQ_MAX_LEVELS; ++l) {
    c.reg[l] = smem + P.off_reg[l];
    c.sel[l] = reinterpret_cast<uint16_t*>(smem + P.off_sel[l]);
    c.par[l] = reinterpret_cast<uint16_t*>(smem + P.off_par[l]);
    c.match[l] = reinterpret_cast<uint32_t*>(smem + P.off_match[l]);
  }
  for (int l = 0; l < DQ_MAX_LEVELS; ++l) {
    c.eoff[l] = reinterpret_cast<uint32_t*>(smem + P.off_exp) + (size_t)l * 3 * P.tile;
    c.ecnt[l] = c.eoff[l] + P.tile;
    c.epos[l] = c.ecnt[l] + P.tile;
  }
  c.flags = smem + P.off_flags;
  c.stash = reinterpret_cast<uint64_t*>(smem + P.off_stash);
  c.stage = smem + P.off_stage;
  c.tile_start = 0;
  // CTA-local aggregation tables
  for (int r = 0; r < P.nres; ++r) {
    const DevRes& R = P.res[r];
    if (R.kind == DQ_RES_AGG && R.smem_slots > 0) {
      LocalAgg a = local_agg(P, c, R);
      for (int i = threadIdx.x; i <= a.ns; i += kThreads) a.tags[i] = kEmpty;
      for (int i = threadIdx.x; i < (a.ns + 1) * R.naggs; i += kThreads) a.acc[i] = red_init(R.agg_red[i % R.naggs]);
    }
  }
  __syncthreads();
}

__device__ void flush_local_aggs(const DevPipe& P, Cta& c) {
  __syncthreads();
  for (int r = 0; r < P.nres; ++r) {
    const DevRes& R = P.res[r];
    if (R.kind != DQ_RES_AGG || R.smem_slots <= 0) continue;
    LocalAgg a = local_agg(P, c, R);
    for (int i = threadIdx.x; i <= a.ns; i += kThreads) {
      uint64_t tag = a.tags[i];
      if (tag == kEmpty) continue;
      if (i == a.ns) tag = kEmpty;  // the all-ones key
      int64_t g = R.nkeys == 0 ? 0 : agg_slot_global(P, R, tag, nullptr);
      if (g < 0) continue;
      uint64_t* acc = R.slots + (uint64_t)g * R.words + R.val_word;
      for (int j = 0; j < R.naggs; ++j) {
        uint64_t v = a.acc[(size_t)i * R.naggs + j];
        int red = R.agg_red[j];
        if (red == DQ_RED_COUNT) atomicAdd((unsigned long long*)(acc + j), v);
        else accumulate(acc + j, red, v);
      }
    }
  }
}

__global__ void __launch_bounds__(kThreads, 2) pipeline_kernel(const __grid_constant__ DevPipe P) {
  extern __shared__ __align__(128) uint8_t smem[];
  __shared__ __align__(8) uint64_t s_mbar[kMaxStages];
  __shared__ int64_t s_tile[kMaxStages];
  // an earlier pipeline of this run overflowed a table: the host re-runs the
  // plan with larger tables, so skip the work (probing a full table is slow)
  if (*(volatile int32_t*)P.status & (kErrHtFull | kErrTimeout)) return;
  Cta c;
  init_cta(P, c, smem);
  const int tid = threadIdx.x;

  if (P.mode == 1) {
    // deferred expansion ranges: work units of exp_cap pairs
    const uint32_t nitems = min(*P.heavy.count, P.heavy.cap);
    const uint64_t units = P.heavy.unit_prefix[nitems];
    const dq_op& op = P.ops[P.heavy.op];
    while (true) {
      if (tid == 0) s_bcast[1] = atomicAdd(P.tile_counter, 1u);
      __syncthreads();
      uint64_t u = s_bcast[1];
      __syncthreads();
      if (u >= units) break;
      int lo = 0, hi = (int)nitems;
      while (lo < hi) {
        int mid = (lo + hi) >> 1;
        if (P.heavy.unit_prefix[mid + 1] <= u) lo = mid + 1;
        else hi = mid;
      }
      const uint64_t* it = P.heavy.items + (size_t)lo * P.heavy.words;
      uint64_t chunk = u - P.heavy.unit_prefix[lo];
      uint64_t off = it[0] + chunk * P.exp_cap;
      uint64_t len = min((uint64_t)P.exp_cap, it[1] - chunk * P.exp_cap);
      for (int s = tid; s < P.heavy.nstash; s += kThreads) c.stash[s] = it[2 + s];
      if (tid == 0) {
        c.sel[0][0] = 0;
        c.eoff[0][0] = (uint32_t)off;
        c.ecnt[0][0] = (uint32_t)len;
        c.epos[0][0] = 0;
      }
      __syncthreads();
      Level L{0, 1};
      run_ops(P, c, P.heavy.op, L);
      (void)op;
      __syncthreads();
    }
    flush_local_aggs(P, c);
    return;
  }

  const int64_t nrows = source_rows(P);
  const int64_t ntiles = (nrows + P.tile - 1) / P.tile;
  const bool staged = P.ncols > 0;
  const bool tma = staged && P.use_tma;

  if (tma) {
    if (tid == 0) {
      for (int s = 0; s < P.nstage; ++s) mbar_init(&s_mbar[s], 1);
      asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
      for (int s = 0; s < P.nstage; ++s) {
        int64_t t = atomicAdd(P.tile_counter, 1u);
        s_tile[s] = t;
        if (t < ntiles) stage_issue(P, smem + P.off_stage + s * P.stage_bytes, t, nrows, &s_mbar[s]);
      }
    }
    __syncthreads();
  }

  uint32_t phase_bits = 0;
  for (int64_t iter = 0;; ++iter) {
    const int s = tma ? (int)(iter % P.nstage) : 0;
    int64_t t;
    if (tma) {
      t = s_tile[s];
    } else {
      if (tid == 0) s_bcast[1] = atomicAdd(P.tile_counter, 1u);
      __syncthreads();
      t = (int64_t)s_bcast[1];
      __syncthreads();
    }
    if (t >= ntiles) break;
    c.stage = smem + P.off_stage + s * P.stage_bytes;
    c.tile_start = t * P.tile;
    const int rows = (int)min((int64_t)P.tile, nrows - c.tile_start);
    if (tma) {
      mbar_wait(P, &s_mbar[s], (phase_bits >> s) & 1u);
      phase_bits ^= 1u << s;
    } else if (staged) {
      stage_plain(P, smem + P.off_stage, t, nrows);
      __syncthreads();
    }
    // initial selection: every row of the tile (occupied slots for AGG sources)
    for (int i = tid; i < rows; i += kThreads) c.sel[0][i] = (uint16_t)i;
    __syncthreads();
    Level L{0, rows};
    if (P.source_kind == DQ_SRC_AGG && P.res[P.source_res].nkeys > 0) {
      const DevRes& R = P.res[P.source_res];
      L.n = compact(c.sel[0], rows, [&](int row) {
        return R.slots[(uint64_t)(c.tile_start + row) * R.words] != kEmpty;
      });
    }
    run_ops(P, c, 0, L);
    __syncthreads();
    if (tma && tid == 0) {
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      int64_t nt = atomicAdd(P.tile_counter, 1u);
      s_tile[s] = nt;
      if (nt < ntiles) stage_issue(P, smem + P.off_stage + s * P.stage_bytes, nt, nrows, &s_mbar[s]);
    }
    __syncthreads();
  }
  flush_local_aggs(P, c);
}

// ------------------------------------------------------ row-at-a-time kernel --
//
// Pipelines without a multimap expansion run row-at-a-time: each warp carries
// 32 rows of a staged tile through the whole operator list, with one active
// flag per lane, and leaves as soon as no lane of the warp is active.  There is
// no per-operator barrier, compaction or shared-memory slot traffic for
// columns: staged columns are read in place, computed values live in a
// per-thread shared-memory register area.  Tiles are staged exactly as for the
// tile kernel (bulk copies on an mbarrier, three tiles ahead).

struct Row {
  const DevPipe* P;
  const uint8_t* stage;   // staged columns of the tile
  uint64_t* regs;         // register area: value of register r of this thread at regs[r * kThreads]
  int64_t tile_start;
  int row;                // row within the tile
};

__device__ __forceinline__ uint64_t rget(const Row& x, int s) {
  const DevPipe& P = *x.P;
  const DevSlot& sl = P.slots[s];
  switch (sl.kind) {
    case DQ_SLOT_COL:
      return canon(ld(x.stage + P.cols[sl.src].smem_off + (size_t)x.row * sl.width, sl.width), sl.ctype);
    case DQ_SLOT_REG:
      return x.regs[(size_t)sl.smem_off * kThreads];
    case DQ_SLOT_AGGKEY: {
      const DevRes& R = P.res[sl.res];
      uint64_t idx = (uint64_t)(x.tile_start + x.row);
      const uint64_t* slot = R.slots + idx * R.words;
      uint64_t raw;
      if (R.packed) {
        uint64_t tag = slot[0];
        if (idx == R.cap) tag = kEmpty;
        raw = (R.nkeys == 1 && (R.key_ctype[0] == DQ_I64 || R.key_ctype[0] == DQ_U64))
                  ? tag : (tag >> (32 * sl.src)) & 0xffffffffull;
      } else {
        raw = slot[R.key_word + sl.src];
      }
      return canon(raw, sl.ctype);
    }
    case DQ_SLOT_AGGVAL: {
      const DevRes& R = P.res[sl.res];
      uint64_t idx = (uint64_t)(x.tile_start + x.row);
      return canon(R.slots[idx * R.words + R.val_word + sl.src], sl.ctype);
    }
    default:
      return 0;
  }
}

__device__ __forceinline__ void rput(const Row& x, int s, uint64_t v) {
  const DevSlot& sl = x.P->slots[s];
  x.regs[(size_t)sl.smem_off * kThreads] = canon(v, sl.ctype);
}

__device__ __forceinline__ void rstr(const Row& x, int s, const uint8_t*& ptr, int& len) {
  const DevPipe& P = *x.P;
  str_at(P.strs[P.slots[s].src], x.tile_start + x.row, ptr, len);
}

__device__ __forceinline__ uint64_t rop(const Row& x, const dq_op& op, int which) {
  if (which == 0) return (op.flags & DQ_OPF_A_IMM) ? (uint64_t)op.imm : rget(x, op.a);
  return (op.flags & DQ_OPF_B_IMM) ? (uint64_t)op.imm : rget(x, op.b);
}

__device__ __forceinline__ void rkeys(const Row& x, const DevRes& R, int list, int n, uint64_t* k) {
  const DevPipe& P = *x.P;
  for (int i = 0; i < n; ++i) k[i] = canon(rget(x, P.lists[list + i]), R.key_ctype[i]);
}

__device__ void row_agg(const Row& x, const dq_op& op, bool act, uint8_t* smem) {
  const DevPipe& P = *x.P;
  const DevRes& R = P.res[op.res];
  const int naggs = R.naggs;
  uint64_t k[DQ_MAX_KEYS];
  uint64_t tag = 0;
  if (act) {
    rkeys(x, R, op.list, op.nlist, k);
    tag = key_tag(R, k);
  }
  const bool local = R.smem_slots > 0;
  uint64_t* tags = local ? reinterpret_cast<uint64_t*>(smem + R.smem_off) : nullptr;
  const int ns = R.smem_slots;
  uint64_t* acc_base = local ? tags + (ns + 1) : nullptr;
  const unsigned active = __ballot_sync(0xffffffffu, act);
  const int lane = threadIdx.x & 31;
  if (local && __popc(active) >= 12) {
    // many rows, few groups: pre-aggregate the warp's rows per distinct key and
    // merge each group once
    unsigned todo = active;
    while (todo) {
      const int leader = __ffs(todo) - 1;
      const uint64_t lt = __shfl_sync(0xffffffffu, tag, leader);
      const bool in = act && tag == lt;
      const unsigned grp = __ballot_sync(0xffffffffu, in);
      int s = -1;
      if (lane == leader) s = local_group_slot(tags, ns, lt, R.nkeys);
      s = __shfl_sync(0xffffffffu, s, leader);
      int64_t g = -1;
      if (s < 0 && lane == leader) g = agg_slot_global(P, R, lt, k);
      for (int j = 0; j < naggs; ++j) {
        const int src = P.lists[op.list2 + j];
        const uint64_t v = (in && src >= 0) ? rget(x, src) : 1;
        const uint64_t r = warp_reduce(R.agg_red[j], in, v, grp);
        if (lane == leader) {
          if (s >= 0) s_merge(saddr(acc_base + (size_t)s * naggs + j), R.agg_red[j], r);
          else if (g >= 0) accumulate(R.slots + (uint64_t)g * R.words + R.val_word + j, R.agg_red[j], r);
        }
      }
      todo &= ~grp;
    }
    return;
  }
  if (!act) return;
  if (local) {
    int s = local_group_slot(tags, ns, tag, R.nkeys);
    if (s >= 0) {
      for (int j = 0; j < naggs; ++j) {
        const int src = P.lists[op.list2 + j];
        s_merge(saddr(acc_base + (size_t)s * naggs + j), R.agg_red[j], src >= 0 ? rget(x, src) : 1);
      }
      return;
    }
  }
  int64_t g = agg_slot_global(P, R, tag, k);
  if (g < 0) return;
  uint64_t* acc = R.slots + (uint64_t)g * R.words + R.val_word;
  for (int j = 0; j < naggs; ++j) {
    const int src = P.lists[op.list2 + j];
    accumulate(acc + j, R.agg_red[j], src >= 0 ? rget(x, src) : 1);
  }
}

__device__ void row_emit(const Row& x, const dq_op& op, bool act) {
  const DevPipe& P = *x.P;
  const DevRes& R = P.res[op.res];
  const unsigned active = __ballot_sync(0xffffffffu, act);
  if (!active) return;
  const int lane = threadIdx.x & 31;
  const int leader = __ffs(active) - 1;
  unsigned long long base = 0;
  if (lane == leader) base = atomicAdd((unsigned long long*)R.cursor, (unsigned long long)__popc(active));
  base = __shfl_sync(0xffffffffu, base, leader);
  if (!act) return;
  const uint64_t pos = base + __popc(active & ((1u << lane) - 1u));
  if (pos >= R.cap) {
    set_status(P, kErrOverflow);
    return;
  }
  for (int j = 0; j < op.nlist; ++j) st(R.pay[j] + pos * R.pay_width[j], R.pay_width[j], rget(x, P.lists[op.list + j]));
}

// Runs the operator list for the calling warp's 32 rows.
__device__ void row_ops(Row& x, bool act, uint8_t* smem) {
  const DevPipe& P = *x.P;
  for (int k = 0; k < P.nops; ++k) {
    if (!__any_sync(0xffffffffu, act)) return;
    const dq_op& op = P.ops[k];
    switch (op.kind) {
      case DQ_OP_ARITH:
        if (act) rput(x, op.dst, arith(op.sub, op.ctype, rop(x, op, 0), rop(x, op, 1)));
        break;
      case DQ_OP_CMP:
        if (act) rput(x, op.dst, compare(op.sub, op.ctype, rop(x, op, 0), rop(x, op, 1)));
        break;
      case DQ_OP_LOGIC:
        if (act) {
          uint64_t a = rget(x, op.a);
          uint64_t r;
          if (op.sub == DQ_NOT) r = a == 0;
          else if (op.sub == DQ_AND) r = a != 0 && rget(x, op.b) != 0;
          else r = a != 0 || rget(x, op.b) != 0;
          rput(x, op.dst, r);
        }
        break;
      case DQ_OP_CAST:
        if (act) rput(x, op.dst, canon(rop(x, op, 0), op.ctype));
        break;
      case DQ_OP_SELECT:
        if (act) {
          uint64_t r = rget(x, op.a) ? rop(x, op, 1) : rget(x, op.c >= 0 ? op.c : op.dst);
          rput(x, op.dst, canon(r, op.ctype));
        }
        break;
      case DQ_OP_LIKE:
      case DQ_OP_STREQ:
        if (act) {
          const uint8_t* s;
          int ls;
          rstr(x, op.a, s, ls);
          const uint8_t* p = P.patterns + P.pat_off[op.res];
          const int lp = P.pat_off[op.res + 1] - P.pat_off[op.res];
          bool r;
          if (op.kind == DQ_OP_LIKE) {
            r = like_match(s, ls, p, lp);
          } else {
            r = ls == lp;
            for (int j = 0; r && j < ls; ++j) r = s[j] == p[j];
          }
          rput(x, op.dst, r);
        }
        break;
      case DQ_OP_FILTER:
        if (act) act = rget(x, op.a) != 0;
        break;
      case DQ_OP_PROBE:
        if (act) {
          const DevRes& R = P.res[op.res];
          uint64_t kv[DQ_MAX_KEYS];
          rkeys(x, R, op.list, op.nlist, kv);
          int64_t s = unique_find(R, key_tag(R, kv), kv);
          if (op.sub == DQ_JOIN_ANTI) {
            act = s < 0;
          } else {
            act = s >= 0;
            if (act && op.sub == DQ_JOIN_INNER) {
              const uint64_t* pay = R.slots + (uint64_t)s * R.words + R.val_word;
              for (int j = 0; j < op.nlist2; ++j) {
                int d = P.lists[op.list2 + j];
                if (d >= 0) rput(x, d, pay[j]);
              }
            }
          }
        }
        break;
      case DQ_OP_AGG:
        row_agg(x, op, act, smem);
        return;
      case DQ_OP_BUILD:
        if (act) {
          const DevRes& R = P.res[op.res];
          uint64_t kv[DQ_MAX_KEYS];
          rkeys(x, R, op.list, op.nlist, kv);
          int64_t s = unique_insert(P, R, key_tag(R, kv), kv);
          if (s >= 0) {
            uint64_t* pay = R.slots + (uint64_t)s * R.words + R.val_word;
            for (int j = 0; j < op.nlist2; ++j) pay[j] = rget(x, P.lists[op.list2 + j]);
          }
        }
        return;
      case DQ_OP_MM_COUNT:
      case DQ_OP_MM_SCATTER:
        if (act) {
          const DevRes& R = P.res[op.res];
          uint64_t kv[DQ_MAX_KEYS];
          rkeys(x, R, op.list, op.nlist, kv);
          uint64_t b = bucket_of(kv, op.nlist, (uint32_t)R.cap);
          if (op.kind == DQ_OP_MM_COUNT) {
            atomicAdd(&R.counts[b], 1u);
          } else {
            uint32_t pos = R.offsets[b] + atomicAdd(&R.counts[b], 1u);
            for (int j = 0; j < op.nlist2; ++j)
              st(R.pay[j] + (size_t)pos * R.pay_width[j], R.pay_width[j], rget(x, P.lists[op.list2 + j]));
          }
        }
        return;
      case DQ_OP_EMIT:
        row_emit(x, op, act);
        return;
      default:
        if (act) set_status(P, kErrBadOp);
        return;
    }
  }
}

__global__ void __launch_bounds__(kThreads, 3) row_kernel(const __grid_constant__ DevPipe Pk) {
  extern __shared__ __align__(128) uint8_t smem[];
  __shared__ __align__(8) uint64_t s_mbar[kMaxStages];
  if (*(volatile int32_t*)Pk.status & (kErrHtFull | kErrTimeout)) return;
  // the descriptor is indexed with runtime values in every operator: keep it in
  // shared memory rather than reading the parameter space through pointers
  {
    const uint4* src = reinterpret_cast<const uint4*>(&Pk);
    uint4* dst = reinterpret_cast<uint4*>(smem);
    for (int i = threadIdx.x; i < (int)(sizeof(DevPipe) / 16); i += kThreads) dst[i] = src[i];
  }
  __syncthreads();
  const DevPipe& P = *reinterpret_cast<const DevPipe*>(smem);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  // CTA-local aggregation tables
  for (int r = 0; r < P.nres; ++r) {
    const DevRes& R = P.res[r];
    if (R.kind == DQ_RES_AGG && R.smem_slots > 0) {
      uint64_t* tags = reinterpret_cast<uint64_t*>(smem + R.smem_off);
      uint64_t* acc = tags + (R.smem_slots + 1);
      for (int i = tid; i <= R.smem_slots; i += kThreads) tags[i] = kEmpty;
      for (int i = tid; i < (R.smem_slots + 1) * R.naggs; i += kThreads) acc[i] = red_init(R.agg_red[i % R.naggs]);
    }
  }
  Row x;
  x.P = &P;
  x.regs = reinterpret_cast<uint64_t*>(smem + P.off_reg[0]) + tid;
  const int64_t nrows = source_rows(P);
  const int64_t ntiles = (nrows + P.tile - 1) / P.tile;
  const bool staged = P.ncols > 0;
  const bool tma = staged && P.use_tma;
  const int64_t first = blockIdx.x, stride = gridDim.x;
  if (tma && tid == 0) {
    for (int s = 0; s < P.nstage; ++s) mbar_init(&s_mbar[s], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    for (int s = 0; s < P.nstage; ++s) {
      int64_t t = first + s * stride;
      if (t < ntiles) stage_issue(P, smem + P.off_stage + s * P.stage_bytes, t, nrows, &s_mbar[s]);
    }
  }
  __syncthreads();
  const bool agg_src = P.source_kind == DQ_SRC_AGG && P.res[P.source_res].nkeys > 0;
  uint32_t phase_bits = 0;
  for (int64_t k = 0;; ++k) {
    const int64_t t = first + k * stride;
    if (t >= ntiles) break;
    const int s = tma ? (int)(k % P.nstage) : 0;
    x.stage = smem + P.off_stage + s * P.stage_bytes;
    x.tile_start = t * P.tile;
    const int rows = (int)min((int64_t)P.tile, nrows - x.tile_start);
    if (tma) {
      mbar_wait(P, &s_mbar[s], (phase_bits >> s) & 1u);
      phase_bits ^= 1u << s;
    } else if (staged) {
      stage_plain(P, smem + P.off_stage, t, nrows);
      __syncthreads();
    }
    for (int base = warp * 32; base < rows; base += kThreads) {
      x.row = base + lane;
      bool act = x.row < rows;
      if (act && agg_src) {
        const DevRes& R = P.res[P.source_res];
        act = R.slots[(uint64_t)(x.tile_start + x.row) * R.words] != kEmpty;
      }
      row_ops(x, act, smem);
    }
    __syncthreads();
    if (tma && tid == 0) {
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      int64_t nt = first + (k + P.nstage) * stride;
      if (nt < ntiles) stage_issue(P, smem + P.off_stage + s * P.stage_bytes, nt, nrows, &s_mbar[s]);
    }
  }
  // merge the CTA-local aggregation tables
  __syncthreads();
  for (int r = 0; r < P.nres; ++r) {
    const DevRes& R = P.res[r];
    if (R.kind != DQ_RES_AGG || R.smem_slots <= 0) continue;
    const uint64_t* tags = reinterpret_cast<const uint64_t*>(smem + R.smem_off);
    const uint64_t* acc = tags + (R.smem_slots + 1);
    for (int i = tid; i <= R.smem_slots; i += kThreads) {
      uint64_t tag = tags[i];
      if (tag == kEmpty) continue;
      if (i == R.smem_slots) tag = kEmpty;
      int64_t g = R.nkeys == 0 ? 0 : agg_slot_global(P, R, tag, nullptr);
      if (g < 0) continue;
      uint64_t* dst = R.slots + (uint64_t)g * R.words + R.val_word;
      for (int j = 0; j < R.naggs; ++j) accumulate(dst + j, R.agg_red[j], acc[(size_t)i * R.naggs + j]);
    }
  }
}

// ------------------------------------------------------- helper kernels --

// Fills aggregation tables: tags empty, accumulators at their initial values.
__global__ void agg_init_kernel(uint64_t* slots, uint64_t nslots, int words, int val_word, int naggs,
                                uint64_t red_packed) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < nslots * words;
       i += (uint64_t)gridDim.x * blockDim.x) {
    uint64_t w = i % words;
    uint64_t v = kEmpty;
    if ((int)w >= val_word && (int)w < val_word + naggs) {
      int red = (int)((red_packed >> (4 * (w - val_word))) & 15);
      v = red_init(red);
    }
    slots[i] = v;
  }
}

// Multimap bucket offsets: exclusive scan of counts in three passes.
constexpr int kScanItems = 16;
constexpr int kScanChunk = kThreads * kScanItems;

__global__ void mm_scan_partials(const uint32_t* counts, uint64_t n, uint32_t* partials) {
  uint64_t base = (uint64_t)blockIdx.x * kScanChunk;
  uint32_t sum = 0;
  for (int k = 0; k < kScanItems; ++k) {
    uint64_t i = base + (uint64_t)k * kThreads + threadIdx.x;
    if (i < n) sum += counts[i];
  }
  uint32_t excl;
  uint32_t total = block_exclusive_scan(sum, excl);
  if (threadIdx.x == 0) partials[blockIdx.x] = total;
}

// Exclusive scan of the block partials (one block; 8 consecutive partials a
// thread per round).
__global__ void mm_scan_top(uint32_t* partials, int nblocks) {
  constexpr int kPer = 8;
  uint32_t carry = 0;
  for (int base = 0; base < nblocks; base += kThreads * kPer) {
    const int i0 = base + threadIdx.x * kPer;
    uint32_t v[kPer];
    uint32_t sum = 0;
#pragma unroll
    for (int k = 0; k < kPer; ++k) {
      v[k] = i0 + k < nblocks ? partials[i0 + k] : 0u;
      sum += v[k];
    }
    uint32_t excl;
    const uint32_t total = block_exclusive_scan(sum, excl);
    uint32_t run = carry + excl;
#pragma unroll
    for (int k = 0; k < kPer; ++k) {
      if (i0 + k < nblocks) partials[i0 + k] = run;
      run += v[k];
    }
    carry += total;
  }
}

// Offsets of one chunk of buckets (kScanItems consecutive counts a thread, in
// 16-byte vectors when the chunk is whole) and the counts reset to zero for the
// scatter pass that follows.
__global__ void mm_scan_final(uint32_t* counts, uint32_t* offsets, uint64_t n, const uint32_t* partials) {
  static_assert(kScanItems % 4 == 0, "vector path");
  const uint64_t i0 = (uint64_t)blockIdx.x * kScanChunk + (uint64_t)threadIdx.x * kScanItems;
  const bool whole = i0 + kScanItems <= n;
  uint32_t v[kScanItems];
  uint32_t sum = 0;
  if (whole) {
#pragma unroll
    for (int k = 0; k < kScanItems; k += 4) {
      const uint4 x = *reinterpret_cast<const uint4*>(counts + i0 + k);
      v[k] = x.x;
      v[k + 1] = x.y;
      v[k + 2] = x.z;
      v[k + 3] = x.w;
    }
  } else {
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) v[k] = (i0 + k < n) ? counts[i0 + k] : 0;
  }
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) sum += v[k];
  uint32_t excl;
  block_exclusive_scan(sum, excl);
  uint32_t run = partials[blockIdx.x] + excl;
  if (whole) {
#pragma unroll
    for (int k = 0; k < kScanItems; k += 4) {
      uint4 o;
      o.x = run;
      run += v[k];
      o.y = run;
      run += v[k + 1];
      o.z = run;
      run += v[k + 2];
      o.w = run;
      run += v[k + 3];
      *reinterpret_cast<uint4*>(offsets + i0 + k) = o;
      *reinterpret_cast<uint4*>(counts + i0 + k) = make_uint4(0u, 0u, 0u, 0u);
    }
  } else {
    for (int k = 0; k < kScanItems; ++k) {
      if (i0 + k < n) {
        offsets[i0 + k] = run;
        counts[i0 + k] = 0;
      }
      run += v[k];
    }
  }
}

// Work-unit prefix over deferred expansion items (one block).
__global__ void heavy_prefix_kernel(const uint64_t* items, const uint32_t* count, uint32_t cap, int words,
                                    uint64_t exp_cap, uint64_t* prefix, int32_t* status) {
  const uint32_t n = min(*count, cap);
  if (threadIdx.x == 0 && *count > cap) atomicOr(status, kInfoHeavyFull);
  uint64_t carry = 0;
  for (uint32_t base = 0; base < n || base == 0; base += kThreads) {
    uint32_t i = base + threadIdx.x;
    uint32_t u = i < n ? (uint32_t)((items[(size_t)i * words + 1] + exp_cap - 1) / exp_cap) : 0;
    uint32_t excl;
    uint32_t total = block_exclusive_scan(u, excl);
    if (i < n) prefix[i] = carry + excl;
    carry += total;
    if (base + kThreads >= n) break;
  }
  if (threadIdx.x == 0) prefix[n] = carry;
}

// Exclusive block scan of one 64-bit value per thread; returns the total.
__device__ uint64_t block_exclusive_scan64(uint64_t x, uint64_t& excl) {
  __shared__ uint64_t s_w[kThreads / 32 + 1];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  uint64_t incl = x;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint64_t y = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += y;
  }
  if (lane == 31) s_w[warp] = incl;
  __syncthreads();
  if (tid == 0) {
    uint64_t run = 0;
    for (int w = 0; w < kThreads / 32; ++w) {
      const uint64_t v = s_w[w];
      s_w[w] = run;
      run += v;
    }
    s_w[kThreads / 32] = run;
  }
  __syncthreads();
  excl = s_w[warp] + incl - x;
  const uint64_t total = s_w[kThreads / 32];
  __syncthreads();
  return total;
}

// Grouped deferred expansion, step 1 (all CTAs): per claimed group, its item
// count and its work units (a group of `len` range rows and `cnt` items is
// ceil(len / kGroupRows) x ceil(cnt / kGroupItems) units), written in place of
// the two prefixes that step 2 computes.
__global__ void heavy_group_units_kernel(DevHeavy H, int32_t* status) {
  const uint32_t n = min(*H.ngroups, H.gcap);
  if (blockIdx.x == 0 && threadIdx.x == 0 && *H.count > H.cap) atomicOr(status, kInfoHeavyFull);
  const uint32_t stride = gridDim.x * blockDim.x;
  for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += stride) {
    const uint32_t g = H.glist[j];
    const uint64_t len = H.glen[g];
    const uint32_t cnt = H.gcnt[g];
    H.gstart[j] = cnt;
    H.unit_prefix[j] = ((len + kGroupRows - 1) / kGroupRows) * (uint64_t)((cnt + kGroupItems - 1) / kGroupItems);
  }
}

// Grouped deferred expansion, step 2 (one block, 8 consecutive groups a
// thread per round): exclusive prefixes of the items (each group's first
// position in `sorted`, also its scatter cursor) and of the work units.
// Totals of 2^32 units or more are refused (the unit counter is 32-bit): the
// pipeline then reports kErrBadOp instead of running them.
__global__ void heavy_group_prefix_kernel(DevHeavy H, int32_t* status) {
  constexpr int kPer = 8;
  const uint32_t n = min(*H.ngroups, H.gcap);
  uint64_t ucarry = 0;
  uint32_t icarry = 0;
  for (uint32_t base = 0; base < n; base += kThreads * kPer) {
    const uint32_t j0 = base + threadIdx.x * kPer;
    uint32_t cnt[kPer];
    uint64_t units[kPer];
    uint32_t csum = 0;
    uint64_t usum = 0;
#pragma unroll
    for (int k = 0; k < kPer; ++k) {
      const bool in = j0 + k < n;
      cnt[k] = in ? H.gstart[j0 + k] : 0u;
      units[k] = in ? H.unit_prefix[j0 + k] : 0ull;
      csum += cnt[k];
      usum += units[k];
    }
    uint32_t iexcl;
    const uint32_t itot = block_exclusive_scan(csum, iexcl);
    uint64_t uexcl;
    const uint64_t utot = block_exclusive_scan64(usum, uexcl);
    uint32_t irun = icarry + iexcl;
    uint64_t urun = ucarry + uexcl;
#pragma unroll
    for (int k = 0; k < kPer; ++k) {
      if (j0 + k < n) {
        H.gstart[j0 + k] = irun;
        H.gcnt[H.glist[j0 + k]] = irun;
        H.unit_prefix[j0 + k] = urun;
      }
      irun += cnt[k];
      urun += units[k];
    }
    icarry += itot;
    ucarry += utot;
  }
  if (threadIdx.x == 0) {
    H.gstart[n] = icarry;
    if (ucarry >= (1ull << 32)) {
      atomicOr(status, kErrBadOp);
      ucarry = 0;
    }
    H.unit_prefix[n] = ucarry;
  }
}

// Grouped deferred expansion, step 2: every item's stashed values move to its
// group's next position in `sorted` (items whose group claim failed were not
// deferred and carry kEmpty as their group).
__global__ void heavy_group_scatter_kernel(DevHeavy H) {
  const uint32_t n = min(*H.count, H.cap);
  const uint32_t stride = gridDim.x * blockDim.x;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    const uint64_t* it = H.items + (size_t)i * H.words;
    const uint64_t g = it[0];
    if (g == kEmpty) continue;
    const uint32_t pos = atomicAdd(H.gcnt + g, 1u);
    for (int s = 0; s < H.nstash; ++s) H.sorted[(size_t)pos * H.nstash + s] = it[2 + s];
  }
}

// ------------------------------------------------------- batch helpers --

// Resets every per-instance buffer of a batch in one launch; each CTA walks
// all descriptors (starting at a rotated one) and strides over its share.
__global__ void batch_reset_kernel(const BatchReset* ops, int nops) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (int k = 0; k < nops; ++k) {
    const int o = (int)((blockIdx.x + (unsigned)k) % (unsigned)nops);
    const BatchReset op = ops[o];
    const uint64_t start = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (op.kind == 0) {
      uint64_t* p = reinterpret_cast<uint64_t*>(op.ptr);
      for (uint64_t i = start; i < op.n; i += stride) p[i] = op.value;
    } else if (op.kind == 1) {
      uint32_t* p = reinterpret_cast<uint32_t*>(op.ptr);
      for (uint64_t i = start; i < op.n; i += stride) p[i] = (uint32_t)op.value;
    } else {
      uint64_t* p = reinterpret_cast<uint64_t*>(op.ptr);
      const uint64_t total = op.n * (uint64_t)op.words;
      for (uint64_t i = start; i < total; i += stride) {
        const int w = (int)(i % (uint64_t)op.words);
        uint64_t v = kEmpty;
        if (w >= op.val_word && w < op.val_word + op.naggs) v = red_init((int)((op.reds >> (4 * (w - op.val_word))) & 15));
        p[i] = v;
      }
    }
  }
}

__device__ __forceinline__ int batch_seg_of(const BatchScanSeg* segs, int nseg, uint64_t block) {
  int lo = 0, hi = nseg;
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (segs[mid].block0 <= block) lo = mid;
    else hi = mid;
  }
  return lo;
}

// Segmented form of the three-pass multimap bucket scan: scan block b belongs to
// the segment (multimap of one instance) whose block range holds b.
__global__ void batch_scan_partials(const BatchScanSeg* segs, int nseg, uint32_t* partials) {
  const uint64_t b = blockIdx.x;
  const BatchScanSeg s = segs[batch_seg_of(segs, nseg, b)];
  const uint64_t base = (b - s.block0) * kScanChunk;
  uint32_t sum = 0;
  for (int k = 0; k < kScanItems; ++k) {
    const uint64_t i = base + (uint64_t)k * kThreads + threadIdx.x;
    if (i < s.n) sum += s.counts[i];
  }
  uint32_t excl;
  const uint32_t total = block_exclusive_scan(sum, excl);
  if (threadIdx.x == 0) partials[b] = total;
}

__global__ void batch_scan_top(const BatchScanSeg* segs, uint32_t* partials) {
  const BatchScanSeg s = segs[blockIdx.x];
  uint32_t carry = 0;
  for (uint64_t base = 0; base < s.nblocks; base += kThreads) {
    const uint64_t i = base + threadIdx.x;
    const uint32_t x = i < s.nblocks ? partials[s.block0 + i] : 0;
    uint32_t excl;
    const uint32_t total = block_exclusive_scan(x, excl);
    if (i < s.nblocks) partials[s.block0 + i] = carry + excl;
    carry += total;
  }
}

__global__ void batch_scan_final(const BatchScanSeg* segs, int nseg, const uint32_t* partials) {
  const uint64_t b = blockIdx.x;
  const BatchScanSeg s = segs[batch_seg_of(segs, nseg, b)];
  const uint64_t i0 = (b - s.block0) * kScanChunk + (uint64_t)threadIdx.x * kScanItems;
  uint32_t v[kScanItems];
  uint32_t sum = 0;
  for (int k = 0; k < kScanItems; ++k) {
    v[k] = (i0 + k < s.n) ? s.counts[i0 + k] : 0;
    sum += v[k];
  }
  uint32_t excl;
  block_exclusive_scan(sum, excl);
  uint32_t run = partials[b] + excl;
  for (int k = 0; k < kScanItems; ++k) {
    if (i0 + k < s.n) {
      s.offsets[i0 + k] = run;
      s.counts[i0 + k] = 0;
    }
    run += v[k];
  }
}

// Copies every instance's output columns (the rows emitted, at most the
// capacity) into one buffer that a single device-to-host copy returns.
__global__ void batch_pack_kernel(const BatchPack* ops, int nops, uint8_t* dst) {
  for (int o = blockIdx.x; o < nops; o += gridDim.x) {
    const BatchPack op = ops[o];
    uint64_t n = *op.cursor;
    if (n > op.cap) n = op.cap;
    const uint64_t bytes = n * (uint64_t)op.width;
    for (uint64_t i = threadIdx.x; i < bytes; i += blockDim.x) dst[op.dst + i] = op.src[i];
    if (threadIdx.x == 0 && op.rows_out) *op.rows_out = n;
  }
}

}  // namespace dq

// ------------------------------------------------------ host-side launchers --

namespace dq {

cudaError_t launch_pipeline(const DevPipe& P, int grid, cudaStream_t stream) {
  cudaError_t e = cudaFuncSetAttribute(pipeline_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, P.smem_bytes);
  if (e != cudaSuccess) return e;
  pipeline_kernel<<<grid, kThreads, P.smem_bytes, stream>>>(P);
  return cudaGetLastError();
}

cudaError_t launch_row(const DevPipe& P, int grid, cudaStream_t stream) {
  cudaError_t e = cudaFuncSetAttribute(row_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, P.smem_bytes);
  if (e != cudaSuccess) return e;
  row_kernel<<<grid, kThreads, P.smem_bytes, stream>>>(P);
  return cudaGetLastError();
}

int row_occupancy(int smem_bytes) {
  int blocks = 0;
  if (cudaFuncSetAttribute(row_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_bytes) != cudaSuccess)
    return 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, row_kernel, kThreads, smem_bytes);
  return blocks;
}

int pipeline_occupancy(int smem_bytes) {
  int blocks = 0;
  cudaFuncSetAttribute(pipeline_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_bytes);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, pipeline_kernel, kThreads, smem_bytes);
  return blocks;
}

cudaError_t launch_agg_init(uint64_t* slots, uint64_t nslots, int words, int val_word, int naggs,
                            const int8_t* reds, cudaStream_t stream) {
  uint64_t packed = 0;
  for (int j = 0; j < naggs && j < 16; ++j) packed |= (uint64_t)(reds[j] & 15) << (4 * j);
  uint64_t total = nslots * words;
  uint64_t want = (total + 255) / 256;
  int grid = (int)(want < 148ull * 16 ? want : 148ull * 16);
  if (grid < 1) grid = 1;
  agg_init_kernel<<<grid, 256, 0, stream>>>(slots, nslots, words, val_word, naggs, packed);
  return cudaGetLastError();
}

size_t mm_scan_scratch_words(uint64_t n) { return (n + kScanChunk - 1) / kScanChunk + 1; }

cudaError_t launch_mm_scan(uint32_t* counts, uint32_t* offsets, uint64_t n, uint32_t* partials,
                           cudaStream_t stream, int* launches) {
  int nblocks = (int)((n + kScanChunk - 1) / kScanChunk);
  if (nblocks < 1) nblocks = 1;
  mm_scan_partials<<<nblocks, kThreads, 0, stream>>>(counts, n, partials);
  mm_scan_top<<<1, kThreads, 0, stream>>>(partials, nblocks);
  mm_scan_final<<<nblocks, kThreads, 0, stream>>>(counts, offsets, n, partials);
  *launches += 3;
  return cudaGetLastError();
}

size_t batch_scan_blocks(uint64_t n) { return (size_t)((n + kScanChunk - 1) / kScanChunk); }

cudaError_t launch_batch_reset(const BatchReset* ops, int nops, int sms, cudaStream_t stream) {
  if (nops <= 0) return cudaSuccess;
  batch_reset_kernel<<<sms * 4, 256, 0, stream>>>(ops, nops);
  return cudaGetLastError();
}

cudaError_t launch_batch_scan(const BatchScanSeg* segs, int nseg, uint64_t total_blocks, uint32_t* partials,
                              cudaStream_t stream) {
  if (nseg <= 0 || total_blocks == 0) return cudaSuccess;
  batch_scan_partials<<<(unsigned)total_blocks, kThreads, 0, stream>>>(segs, nseg, partials);
  batch_scan_top<<<nseg, kThreads, 0, stream>>>(segs, partials);
  batch_scan_final<<<(unsigned)total_blocks, kThreads, 0, stream>>>(segs, nseg, partials);
  return cudaGetLastError();
}

cudaError_t launch_batch_pack(const BatchPack* ops, int nops, uint8_t* dst, int sms, cudaStream_t stream) {
  if (nops <= 0) return cudaSuccess;
  batch_pack_kernel<<<sms * 2, 256, 0, stream>>>(ops, nops, dst);
  return cudaGetLastError();
}

cudaError_t launch_heavy_prefix(const DevHeavy& H, uint64_t exp_cap, int32_t* status, cudaStream_t stream) {
  heavy_prefix_kernel<<<1, kThreads, 0, stream>>>(H.items, H.count, H.cap, H.words, exp_cap, H.unit_prefix, status);
  return cudaGetLastError();
}

cudaError_t launch_heavy_group(const DevHeavy& H, int32_t* status, int sms, cudaStream_t stream) {
  heavy_group_units_kernel<<<sms, 256, 0, stream>>>(H, status);
  heavy_group_prefix_kernel<<<1, kThreads, 0, stream>>>(H, status);
  heavy_group_scatter_kernel<<<sms * 2, 256, 0, stream>>>(H);
  return cudaGetLastError();
}

}  // namespace dq
