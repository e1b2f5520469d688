// Device helpers shared by the prebuilt pipeline kernels (dq_kernels.cu) and
// the per-pipeline kernels generated at plan preparation (dq_jit.cu compiles
// them with NVRTC and embeds this file as an in-memory header).  Keeping one
// copy of the value semantics, hashing and table probing makes every kernel
// of a plan agree on table layouts and results.
//
// Values are carried as canonical 64-bit words: sign-extended for signed C
// types, zero-extended for unsigned ones, and every operation computes in the C
// type the lowering assigned (usual arithmetic conversions, wrap-around).
#pragma once
#include "dq_device.h"

namespace dq {

constexpr long long kSpinLimit = 1ll << 28;  // bound of every device wait
constexpr uint64_t kBusy = ~0ull - 1;        // aggregation slot being claimed
constexpr unsigned kFull = 0xffffffffu;

// ------------------------------------------------------------------ values --

__device__ __forceinline__ uint64_t canon(uint64_t v, int t) {
  switch (t) {
    case DQ_I8: return (uint64_t)(int64_t)(int8_t)v;
    case DQ_I32: return (uint64_t)(int64_t)(int32_t)v;
    case DQ_U32: return (uint64_t)(uint32_t)v;
    default: return v;
  }
}

__device__ __forceinline__ bool is_signed(int t) { return t == DQ_I8 || t == DQ_I32 || t == DQ_I64; }

__device__ __forceinline__ uint64_t ld(const uint8_t* p, int w) {
  switch (w) {
    case 1: return *p;
    case 2: return *reinterpret_cast<const uint16_t*>(p);
    case 4: return *reinterpret_cast<const uint32_t*>(p);
    default: return *reinterpret_cast<const uint64_t*>(p);
  }
}

__device__ __forceinline__ void st(uint8_t* p, int w, uint64_t v) {
  switch (w) {
    case 1: *p = (uint8_t)v; break;
    case 2: *reinterpret_cast<uint16_t*>(p) = (uint16_t)v; break;
    case 4: *reinterpret_cast<uint32_t*>(p) = (uint32_t)v; break;
    default: *reinterpret_cast<uint64_t*>(p) = v; break;
  }
}

template <class T>
__device__ __forceinline__ T ld_plain(const T* p) { return *p; }

// Read-only (non-coherent) load of a w-byte value: for data a kernel does not
// write, such as a multimap payload during the probe.
__device__ __forceinline__ uint64_t ldg_w(const uint8_t* p, int w) {
  switch (w) {
    case 1: return __ldg(p);
    case 2: return __ldg(reinterpret_cast<const uint16_t*>(p));
    case 4: return __ldg(reinterpret_cast<const uint32_t*>(p));
    default: return __ldg(reinterpret_cast<const unsigned long long*>(p));
  }
}

// 32 read-only bytes (four 64-bit words; p 32-byte aligned): one 256-bit load
// where the compiler accepts it (CUDA 12.9 and later for sm_100a, signalled by
// DQ_LD256), else two 128-bit loads of the same sector.
__device__ __forceinline__ void ld_nc_32B(const uint64_t* p, uint64_t& a, uint64_t& b, uint64_t& c, uint64_t& d) {
#if defined(DQ_LD256) && DQ_LD256
  asm volatile("ld.global.nc.v4.u64 {%0, %1, %2, %3}, [%4];" : "=l"(a), "=l"(b), "=l"(c), "=l"(d) : "l"(p));
#else
  const ulonglong2 x = __ldg(reinterpret_cast<const ulonglong2*>(p));
  const ulonglong2 y = __ldg(reinterpret_cast<const ulonglong2*>(p) + 1);
  a = x.x;
  b = x.y;
  c = y.x;
  d = y.y;
#endif
}

// 16 read-only bytes (two 64-bit words; p 16-byte aligned).
__device__ __forceinline__ void ld_nc_16B(const uint64_t* p, uint64_t& a, uint64_t& b) {
  const ulonglong2 x = __ldg(reinterpret_cast<const ulonglong2*>(p));
  a = x.x;
  b = x.y;
}

// MurmurHash3 64-bit finaliser (Appleby), used for every hash table.
__device__ __forceinline__ uint64_t fmix64(uint64_t k) {
  k ^= k >> 33;
  k *= 0xff51afd7ed558ccdull;
  k ^= k >> 33;
  k *= 0xc4ceb9fe1a85ec53ull;
  k ^= k >> 33;
  return k;
}

// Maps a 64-bit hash onto [0, cap) without a division (multiply-high range
// reduction).
__device__ __forceinline__ uint64_t reduce_range(uint64_t h, uint64_t cap) { return __umul64hi(h, cap); }

// Home slot of a 64-bit tag in a table of `cap` slots (cap < 2^32): the high
// word of a multiplicative (Fibonacci) hash, range-reduced by a multiply-high.
// Every hash table of a plan places keys with this function.
__device__ __forceinline__ uint32_t slot_of(uint64_t tag, uint32_t cap) {
  const uint32_t h = (uint32_t)((tag * 0x9e3779b97f4a7c15ull) >> 32);
  return __umulhi(h, cap);
}

// Bucket of a multimap key (n key values) among `cap` buckets.
__device__ __forceinline__ uint32_t bucket_of(const uint64_t* k, int n, uint32_t cap) {
  uint64_t h = n > 0 ? k[0] : 0;
  for (int i = 1; i < n; ++i) h = (h ^ (h >> 29)) * 0xbf58476d1ce4e5b9ull + k[i];
  return slot_of(h, cap);
}

__device__ __forceinline__ uint64_t arith(int sub, int t, uint64_t a, uint64_t b) {
  a = canon(a, t);
  b = canon(b, t);
  uint64_t r = 0;
  switch (sub) {
    case DQ_ADD: r = a + b; break;
    case DQ_SUB: r = a - b; break;
    case DQ_MUL: r = a * b; break;
    case DQ_DIV:
    case DQ_MOD: {
      if (b == 0) return 0;  // undefined in C; defined as 0 here
      bool div = sub == DQ_DIV;
      if (t == DQ_I32) {
        int32_t x = (int32_t)a, y = (int32_t)b;
        if (y == -1) r = div ? (uint64_t)(uint32_t)(0u - (uint32_t)x) : 0;
        else r = (uint64_t)(uint32_t)(div ? x / y : x % y);
      } else if (t == DQ_U32) {
        uint32_t x = (uint32_t)a, y = (uint32_t)b;
        r = div ? x / y : x % y;
      } else if (t == DQ_I64) {
        int64_t x = (int64_t)a, y = (int64_t)b;
        if (y == -1) r = div ? 0ull - a : 0;
        else r = (uint64_t)(div ? x / y : x % y);
      } else {
        r = div ? a / b : a % b;
      }
      break;
    }
  }
  return canon(r, t);
}

__device__ __forceinline__ bool compare(int sub, int t, uint64_t a, uint64_t b) {
  a = canon(a, t);
  b = canon(b, t);
  if (is_signed(t)) {
    int64_t x = (int64_t)a, y = (int64_t)b;
    switch (sub) {
      case DQ_EQ: return x == y;
      case DQ_NE: return x != y;
      case DQ_LT: return x < y;
      case DQ_LE: return x <= y;
      case DQ_GT: return x > y;
      default: return x >= y;
    }
  }
  switch (sub) {
    case DQ_EQ: return a == b;
    case DQ_NE: return a != b;
    case DQ_LT: return a < b;
    case DQ_LE: return a <= b;
    case DQ_GT: return a > b;
    default: return a >= b;
  }
}

// LIKE with the reference matcher's exact semantics (util.cuh:144-199):
// prefix, then suffix, then infixes left to right; '_' matches any byte; reads
// one past the end of the string or pattern see a zero byte.
__device__ __noinline__ bool like_match(const uint8_t* s, int ls, const uint8_t* p, int lp) {
  auto S = [&](int i) -> int { return (i >= 0 && i < ls) ? s[i] : 0; };
  auto P = [&](int i) -> int { return (i >= 0 && i < lp) ? p[i] : 0; };
  auto cmp = [](int c, int l) { return c == l || l == '_'; };
  int l_in_start = 0, l_in_end = lp, s_in_start = 0, s_in_end = ls, l_pos = 0;
  if (P(0) != '%') {
    int s_pos = 0;
    l_pos = 0;
    while (l_pos < lp && s_pos < ls && P(l_pos) != '%') {
      if (!cmp(S(s_pos), P(l_pos))) return false;
      ++l_pos;
      ++s_pos;
    }
    l_in_start = l_pos;
    s_in_start = s_pos;
  }
  if (P(lp - 1) != '%') {
    int s_pos = ls - 1;
    l_pos = lp - 1;
    while (l_pos >= 0 && s_pos >= 0 && P(l_pos) != '%') {
      if (!cmp(S(s_pos), P(l_pos))) return false;
      --l_pos;
      --s_pos;
    }
    l_in_end = l_pos;
    s_in_end = s_pos + 1;
  }
  if (l_in_start < l_in_end) {
    l_pos = l_in_start + 1;
    int s_pos = s_in_start;
    while (s_pos < s_in_end && l_pos < l_in_end) {
      int l_tr = l_pos, s_tr = s_pos;
      while (cmp(S(s_tr), P(l_tr)) && s_tr < s_in_end) {
        ++l_tr;
        if (P(l_tr) == '%') {
          ++l_tr;
          l_pos = l_tr;
          s_pos = s_tr;
          break;
        }
        ++s_tr;
      }
      ++s_pos;
    }
  }
  return l_pos >= l_in_end;
}

// Prefetches into L1 the 128-byte lines (at most four) that n bytes at p
// cover: a warp that works through its lanes' long strings one after another
// then waits for their memory once, not once per string.  The lines lie in the
// string's own allocation (heaps start 256-byte aligned).
__device__ __forceinline__ void prefetch_bytes(const uint8_t* p, int n) {
  const unsigned long long a = (unsigned long long)p & ~127ull, e = (unsigned long long)p + (unsigned long long)n;
  for (int i = 0; i < 4 && a + 128ull * (unsigned long long)i < e; ++i)
    asm volatile("prefetch.global.L1 [%0];" ::"l"(a + 128ull * (unsigned long long)i));
}

// Bytes p[0, m) (1 <= m <= 8) as a little-endian word, zero above byte m:
// one or two loads of the aligned words that hold them, shifted together.
// Every such word holds at least one of the bytes, so it lies in the same
// allocation (string heaps start 256-byte aligned and are padded at the end).
__device__ __forceinline__ uint64_t load_bytes(const uint8_t* p, int m) {
  const unsigned long long at = (unsigned long long)p;
  const unsigned long long* a = reinterpret_cast<const unsigned long long*>(at & ~7ull);
  const int sh = (int)(at & 7);
  uint64_t w = __ldg(a) >> (8 * sh);
  if (sh + m > 8) w |= __ldg(a + 1) << (64 - 8 * sh);
  return m >= 8 ? w : (w & ((1ull << (8 * m)) - 1));
}

// First index in [from, to) of byte c in s, or -1.  Tests eight bytes at a
// time in the aligned words that cover the range (a zero-byte test on
// w ^ c repeated, Mycroft's method); bytes before `from` are set to 0xff first
// so that no borrow from them can flag a later byte.  String heaps start
// 256-byte aligned and are padded at the end, so every such word lies in the
// heap's allocation.
__device__ __forceinline__ int find_byte(const uint8_t* s, int from, int to, uint8_t c) {
  if (from >= to) return -1;
  const unsigned long long ones = 0x0101010101010101ull, pat = ones * c;
  const unsigned long long first = (unsigned long long)(s + from), end = (unsigned long long)(s + to);
  unsigned long long a = first & ~7ull;
  int skip = (int)(first - a);
  for (; a < end; a += 8, skip = 0) {
    unsigned long long t = __ldg(reinterpret_cast<const unsigned long long*>(a)) ^ pat;
    if (skip) t |= (1ull << (8 * skip)) - 1;
    const unsigned long long z = (t - ones) & ~t & 0x8080808080808080ull;
    if (z) {
      const int i = (int)(a - (unsigned long long)s) + (__ffsll((long long)z) - 1) / 8;
      return i < to ? i : -1;
    }
  }
  return -1;
}

// One literal of a LIKE pattern '%L1%...%Ln%': its leftmost occurrence in
// s[pos, n); on success pos moves past it.  For such patterns (no '_', no
// empty literal) like_match's outcome is that of finding L1, ..., Ln this way
// one after another.
__device__ __forceinline__ bool like_find(const uint8_t* s, int n, int& pos, const uint8_t* L, int m) {
  while (pos + m <= n) {
    const int c = find_byte(s, pos, n - m + 1, L[0]);
    if (c < 0) return false;
    int j = 1;
    while (j < m && s[c + j] == L[j]) ++j;
    if (j == m) {
      pos = c + m;
      return true;
    }
    pos = c + 1;
  }
  return false;
}

// String value of row g of a string column.
__device__ __forceinline__ void str_at(const DevStr& d, int64_t g, const uint8_t*& ptr, int& len) {
  if (d.width > 0) {
    ptr = d.chars + g * d.width;
    len = d.width;
  } else {
    uint64_t a = d.offsets[g], b = d.offsets[g + 1];
    ptr = d.chars + a;
    len = (int)(b - a);
  }
}

__device__ __forceinline__ bool str_eq(const uint8_t* s, int ls, const uint8_t* p, int lp) {
  if (ls != lp) return false;
  for (int b = 0; b < ls; b += 8) {
    const int m = ls - b < 8 ? ls - b : 8;
    if (load_bytes(s + b, m) != load_bytes(p + b, m)) return false;
  }
  return true;
}

// ------------------------------------------------------------ pipelines --

__device__ __forceinline__ void set_status(const DevPipe& P, int32_t bits) { atomicOr(P.status, bits); }

// Rows of the pipeline's source.  A temp table's row count is its cursor,
// which an overflowing emit may have advanced past the capacity: the rows
// beyond it were never written (the plan is re-run with a larger table).
__device__ __forceinline__ int64_t source_rows(const DevPipe& P) {
  if (!P.nrows_dev) return P.nrows;
  uint64_t n = *P.nrows_dev;
  if (P.source_res >= 0 && n > P.res[P.source_res].cap) n = P.res[P.source_res].cap;
  return (int64_t)n;
}

// ------------------------------------------------------------- hashing --

// Packed tag (exact key) or 63-bit hash tag for wide keys.
__device__ __forceinline__ uint64_t key_tag(const DevRes& R, const uint64_t* k) {
  if (R.packed) {
    if (R.nkeys == 0) return 0;
    if (R.nkeys == 1 && (R.key_ctype[0] == DQ_I64 || R.key_ctype[0] == DQ_U64)) return k[0];
    uint64_t t = (uint32_t)k[0];
    if (R.nkeys > 1) t |= (uint64_t)(uint32_t)k[1] << 32;
    return t;
  }
  uint64_t h = 0x9e3779b97f4a7c15ull;
  for (int i = 0; i < R.nkeys; ++i) h = fmix64(h ^ k[i]) + 0x632be59bd9b4e019ull * (i + 1);
  return fmix64(h) & 0x7fffffffffffffffull;
}

// String references (source, substring window, row): the bytes behind them,
// their hash and equality.  Join and group keys of string type hash and
// compare the bytes, so two rows with equal strings meet whatever rows they
// came from.
__device__ __forceinline__ void str_ref_at(const DevPipe& P, uint64_t ref, const uint8_t*& ptr, int& len) {
  str_ref_bytes(P.strsrc, ref, ptr, len);
}

// SUBSTRING(s, from, for) of a reference, the reference's stringSubstring
// (include/util.cuh:132-142): first byte from - 1, `for` bytes, the window
// clamped to the string (a window past its end is empty).  Offsets are within
// the string's first kStrRefMaxOffset bytes (the lowering checks constants).
__device__ __forceinline__ uint64_t str_ref_substring(uint64_t ref, int from, int len) {
  int s0 = 0, e0 = 1 << 30;
  if (ref & kStrRefSub) {
    s0 = (int)((ref >> kStrRefStartShift) & 0xff);
    e0 = (int)((ref >> kStrRefEndShift) & 0xff);
  }
  int st = s0 + from - 1;
  int en = st + len;
  if (st < s0) st = s0;
  if (en > e0) en = e0;
  st = st < 0 ? 0 : (st > kStrRefMaxOffset ? kStrRefMaxOffset : st);
  en = en < st ? st : (en > kStrRefMaxOffset ? kStrRefMaxOffset : en);
  return (ref & ~((1ull << kStrRefShift) - 1 - kStrRefRow)) | kStrRefSub | ((uint64_t)st << kStrRefStartShift) |
         ((uint64_t)en << kStrRefEndShift);
}

// String hash: the string's 8-byte little-endian words (the last one
// zero-padded), each offset by an index constant and multiplied by an odd
// index-dependent constant (a multilinear hash), summed, and the sum mixed
// with the length.  A sum of independent word terms lets a warp hash one
// string a word per lane (str_hash_wide) and reach the value one lane
// computes alone, so either may hash the keys of one table.
__device__ __forceinline__ uint64_t str_word(const uint8_t* p, int n, int i) {
  const int b = 8 * i;
  return load_bytes(p + b, n - b < 8 ? n - b : 8);
}

__device__ __forceinline__ uint64_t str_word_term(uint64_t w, int i) {
  return (w + 0x632be59bd9b4e019ull * (uint64_t)(i + 1)) * (0x9e3779b97f4a7c15ull * (uint64_t)(2 * i + 1));
}

__device__ __forceinline__ uint64_t str_hash_final(uint64_t sum, int n) {
  return fmix64(sum + (uint64_t)n * 0xc2b2ae3d27d4eb4full);
}

__device__ __forceinline__ uint64_t str_hash(const uint8_t* p, int n) {
  uint64_t sum = 0;
  for (int i = 0; 8 * i < n; ++i) sum += str_word_term(str_word(p, n, i), i);
  return str_hash_final(sum, n);
}

__device__ __forceinline__ uint64_t str_ref_hash(const DevPipe& P, uint64_t ref) {
  const uint8_t* p;
  int n;
  str_ref_at(P, ref, p, n);
  return str_hash(p, n);
}

__device__ __forceinline__ bool str_ref_eq(const DevPipe& P, uint64_t a, uint64_t b) {
  if (a == b) return true;
  const uint8_t *pa, *pb;
  int na, nb;
  str_ref_at(P, a, pa, na);
  str_ref_at(P, b, pb, nb);
  return str_eq(pa, na, pb, nb);
}

constexpr int kStrCoopMin = 32;  // strings longer than this are hashed and compared by the whole warp

__device__ __forceinline__ uint64_t warp_sum64(uint64_t v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
  return v;
}

// The words of a string of at most kStrCoopMin bytes, loaded independently
// of one another (zero past the end), and its str_hash from them.  Two such
// strings are equal exactly when their lengths and words are.
constexpr int kStrShortWords = kStrCoopMin / 8;

__device__ __forceinline__ void str_words_short(const uint8_t* p, int n, uint64_t* w) {
#pragma unroll
  for (int i = 0; i < kStrShortWords; ++i) w[i] = 8 * i < n ? load_bytes(p + 8 * i, n - 8 * i < 8 ? n - 8 * i : 8) : 0ull;
}

__device__ __forceinline__ uint64_t str_hash_words(const uint64_t* w, int n) {
  uint64_t sum = 0;
#pragma unroll
  for (int i = 0; i < kStrShortWords; ++i)
    if (8 * i < n) sum += str_word_term(w[i], i);
  return str_hash_final(sum, n);
}

// The warp's strings longer than kStrCoopMin bytes (lanes with `wide` set)
// hashed one after another by all 32 lanes, a word per lane with coalesced
// reads (the reference's push-down string hash, include/hashing.cuh:39-62);
// each gets str_hash's value, and the other lanes keep h.  Called by every
// lane of the warp, before its lanes branch.
__device__ __noinline__ uint64_t str_hash_wide(bool wide, const uint8_t* p, int n, uint64_t h) {
  const int lane = (int)(threadIdx.x & 31);
  if (wide) prefetch_bytes(p, n);
  unsigned todo = __ballot_sync(kFull, wide);
  while (todo) {
    const int src = __ffs(todo) - 1;
    todo &= todo - 1;
    const uint8_t* q = reinterpret_cast<const uint8_t*>(__shfl_sync(kFull, (unsigned long long)p, src));
    const int m = __shfl_sync(kFull, n, src);
    uint64_t part = 0;
    for (int i = lane; 8 * i < m; i += 32) part += str_word_term(str_word(q, m, i), i);
    part = warp_sum64(part);
    if (lane == src) h = str_hash_final(part, m);
  }
  return h;
}

// Equality of two active lanes' string references, called by every lane of
// the warp (the reference's stringEqualsPushdown, include/util.cuh:104-130):
// pairs of equal length longer than kStrCoopMin bytes are compared by all 32
// lanes a byte each, the shorter ones by their own lane.
__device__ __noinline__ bool str_ref_eq_warp(const DevPipe& P, bool active, uint64_t a, uint64_t b) {
  const uint8_t *pa = nullptr, *pb = nullptr;
  int na = 0, nb = 0;
  if (active && a != b) {
    str_ref_at(P, a, pa, na);
    str_ref_at(P, b, pb, nb);
  }
  const bool wide = active && a != b && na == nb && na > kStrCoopMin;
  if (wide) {
    prefetch_bytes(pa, na);
    prefetch_bytes(pb, nb);
  }
  bool eq = active && (a == b || (!wide && str_eq(pa, na, pb, nb)));
  const int lane = (int)(threadIdx.x & 31);
  unsigned todo = __ballot_sync(kFull, wide);
  while (todo) {
    const int src = __ffs(todo) - 1;
    todo &= todo - 1;
    const uint8_t* x = reinterpret_cast<const uint8_t*>(__shfl_sync(kFull, (unsigned long long)pa, src));
    const uint8_t* y = reinterpret_cast<const uint8_t*>(__shfl_sync(kFull, (unsigned long long)pb, src));
    const int m = __shfl_sync(kFull, na, src);
    bool same = true;
    for (int j = lane; j < m; j += 32) same &= x[j] == y[j];
    same = __all_sync(kFull, same);
    if (lane == src) eq = same;
  }
  return eq;
}

// Hash tag of wide keys some of which are string references, given the
// strings' hashes `sh` (entries of non-string keys unused).
__device__ __forceinline__ uint64_t key_tag_strh(const DevRes& R, const uint64_t* k, const uint64_t* sh) {
  uint64_t h = 0x9e3779b97f4a7c15ull;
  for (int i = 0; i < R.nkeys; ++i) {
    const uint64_t v = R.key_ctype[i] == DQ_STR ? sh[i] : k[i];
    h = fmix64(h ^ v) + 0x632be59bd9b4e019ull * (i + 1);
  }
  return fmix64(h) & 0x7fffffffffffffffull;
}

__device__ __forceinline__ uint64_t key_tag_str(const DevPipe& P, const DevRes& R, const uint64_t* k) {
  uint64_t sh[DQ_MAX_KEYS];
  for (int i = 0; i < R.nkeys; ++i) sh[i] = R.key_ctype[i] == DQ_STR ? str_ref_hash(P, k[i]) : 0ull;
  return key_tag_strh(R, k, sh);
}

// Bucket of a multimap key some of whose values are string references: their
// bytes' hashes `sh` stand in for them (bucket_of otherwise).
__device__ __forceinline__ uint32_t bucket_of_strh(const DevRes& R, const uint64_t* k, const uint64_t* sh, int n,
                                                   uint32_t cap) {
  uint64_t h = 0;
  for (int i = 0; i < n; ++i) {
    const uint64_t v = R.key_ctype[i] == DQ_STR ? sh[i] : k[i];
    h = i == 0 ? v : (h ^ (h >> 29)) * 0xbf58476d1ce4e5b9ull + v;
  }
  return slot_of(h, cap);
}

// Key equality of a stored key word and a probe key word of ctype t.
__device__ __forceinline__ bool key_word_eq(const DevPipe& P, int t, uint64_t a, uint64_t b) {
  return t == DQ_STR ? str_ref_eq(P, a, b) : a == b;
}

// Unique join table: returns slot index or -1.
__device__ __forceinline__ int64_t unique_find(const DevRes& R, uint64_t tag, const uint64_t* k) {
  if (R.packed && tag == kEmpty) return R.slots[R.cap * R.words] == 0 ? (int64_t)R.cap : -1;
  uint64_t idx = slot_of(tag, (uint32_t)R.cap);
  for (uint64_t n = 0; n < R.cap; ++n) {
    const uint64_t* s = R.slots + idx * R.words;
    uint64_t t = s[0];
    if (t == kEmpty) return -1;
    if (t == tag) {
      bool eq = true;
      if (!R.packed)
        for (int i = 0; i < R.nkeys; ++i) eq &= s[R.key_word + i] == k[i];
      if (eq) return (int64_t)idx;
    }
    idx = (idx + 1 == R.cap) ? 0 : idx + 1;
  }
  return -1;
}

// Unique join table with string keys (tags are byte hashes): the keys of a
// slot with the probe's tag are compared by their bytes.
__device__ __forceinline__ int64_t unique_find_str(const DevPipe& P, const DevRes& R, uint64_t tag,
                                                   const uint64_t* k) {
  uint64_t idx = slot_of(tag, (uint32_t)R.cap);
  for (uint64_t n = 0; n < R.cap; ++n) {
    const uint64_t* s = R.slots + idx * R.words;
    const uint64_t t = s[0];
    if (t == kEmpty) return -1;
    if (t == tag) {
      bool eq = true;
      for (int i = 0; i < R.nkeys && eq; ++i) eq = key_word_eq(P, R.key_ctype[i], s[R.key_word + i], k[i]);
      if (eq) return (int64_t)idx;
    }
    idx = (idx + 1 == R.cap) ? 0 : idx + 1;
  }
  return -1;
}

// Inserts string keys: a slot is claimed with a busy marker, its keys written,
// then its tag published, so an insert of equal bytes (another row holding the
// same string) finds the keys and stops there: each distinct key takes one
// slot, however often the build side repeats it.  Returns the claimed slot,
// or -1 when the key was present (the first insert wins) or the table is full.
__device__ __forceinline__ int64_t unique_insert_str(const DevPipe& P, const DevRes& R, uint64_t tag,
                                                     const uint64_t* k) {
  uint64_t idx = slot_of(tag, (uint32_t)R.cap);
  for (uint64_t n = 0; n < R.cap; ++n) {
    uint64_t* s = R.slots + idx * R.words;
    uint64_t t = *(volatile uint64_t*)s;
    if (t == kEmpty) {
      const uint64_t old = atomicCAS((unsigned long long*)s, kEmpty, kBusy);
      if (old == kEmpty) {
        for (int i = 0; i < R.nkeys; ++i) s[R.key_word + i] = k[i];
        __threadfence();
        atomicExch((unsigned long long*)s, tag);
        return (int64_t)idx;
      }
      t = old;
    }
    long long spins = 0;
    while (t == kBusy && spins < kSpinLimit) {
      t = *(volatile uint64_t*)s;
      ++spins;
    }
    if (t == kBusy) {
      set_status(P, kErrTimeout);
      return -1;
    }
    if (t == tag) {
      __threadfence();
      bool eq = true;
      for (int i = 0; i < R.nkeys && eq; ++i)
        eq = key_word_eq(P, R.key_ctype[i], ((volatile uint64_t*)s)[R.key_word + i], k[i]);
      if (eq) return -1;
    }
    idx = (idx + 1 == R.cap) ? 0 : idx + 1;
  }
  set_status(P, kErrHtFull);
  return -1;
}

// Inserts the key; returns the slot to write the payload to, or -1 if the key
// was present already (first insert wins) or the table is full.
__device__ __forceinline__ int64_t unique_insert(const DevPipe& P, const DevRes& R, uint64_t tag,
                                                 const uint64_t* k) {
  if (R.packed && tag == kEmpty) {
    uint64_t old = atomicCAS((unsigned long long*)(R.slots + R.cap * R.words), kEmpty, 0ull);
    return old == kEmpty ? (int64_t)R.cap : -1;
  }
  uint64_t idx = slot_of(tag, (uint32_t)R.cap);
  for (uint64_t n = 0; n < R.cap; ++n) {
    uint64_t* s = R.slots + idx * R.words;
    uint64_t old = atomicCAS((unsigned long long*)s, kEmpty, tag);
    if (old == kEmpty) {
      if (!R.packed)
        for (int i = 0; i < R.nkeys; ++i) s[R.key_word + i] = k[i];
      return (int64_t)idx;
    }
    if (old == tag && R.packed) return -1;
    idx = (idx + 1 == R.cap) ? 0 : idx + 1;
  }
  set_status(P, kErrHtFull);
  return -1;
}

// Compact unique table (R.compact): inserts key k32 with its 32-bit payload,
// one compare-and-swap of the whole word.  The first insert of a key wins.
// The all-ones key cannot share the empty marker's word and is kept at slot
// cap (0 when present), its payload at cap + 1.
__device__ __forceinline__ void unique_insert_compact(const DevPipe& P, const DevRes& R, uint32_t k32, uint32_t pay) {
  uint64_t* const ht = R.slots;
  const uint32_t cap = (uint32_t)R.cap;
  if (k32 == 0xffffffffu) {
    if (atomicCAS((unsigned long long*)(ht + cap), kEmpty, 0ull) == kEmpty) ht[(uint64_t)cap + 1] = pay;
    return;
  }
  const uint64_t w = ((uint64_t)k32 << 32) | pay;
  uint32_t idx = slot_of((uint64_t)k32, cap);
  for (uint32_t n = 0; n < cap; ++n) {
    const uint64_t old = atomicCAS((unsigned long long*)(ht + idx), kEmpty, w);
    if (old == kEmpty || (uint32_t)(old >> 32) == k32) return;
    idx = (idx + 1u == cap) ? 0u : idx + 1u;
  }
  set_status(P, kErrHtFull);
}

// Aggregation table (global): find or claim the group's slot.
__device__ __noinline__ int64_t agg_slot_global(const DevPipe& P, const DevRes& R, uint64_t tag,
                                                const uint64_t* k) {
  if (R.nkeys == 0) return 0;  // one group, always at slot 0
  if (R.packed) {
    if (tag == kEmpty) {
      atomicCAS((unsigned long long*)(R.slots + R.cap * R.words), kEmpty, 0ull);
      return (int64_t)R.cap;
    }
    uint64_t idx = slot_of(tag, (uint32_t)R.cap);
    for (uint64_t n = 0; n < R.cap; ++n) {
      uint64_t* s = R.slots + idx * R.words;
      uint64_t t = *(volatile uint64_t*)s;
      if (t == tag) return (int64_t)idx;
      if (t == kEmpty) {
        uint64_t old = atomicCAS((unsigned long long*)s, kEmpty, tag);
        if (old == kEmpty || old == tag) return (int64_t)idx;
      }
      idx = (idx + 1 == R.cap) ? 0 : idx + 1;
    }
    set_status(P, kErrHtFull);
    return -1;
  }
  // wide keys: claim with a busy marker, publish keys, then the tag
  uint64_t idx = slot_of(tag, (uint32_t)R.cap);
  for (uint64_t n = 0; n < R.cap; ++n) {
    uint64_t* s = R.slots + idx * R.words;
    uint64_t t = *(volatile uint64_t*)s;
    if (t == kEmpty) {
      uint64_t old = atomicCAS((unsigned long long*)s, kEmpty, kBusy);
      if (old == kEmpty) {
        for (int i = 0; i < R.nkeys; ++i) s[R.key_word + i] = k[i];
        __threadfence();
        atomicExch((unsigned long long*)s, tag);
        return (int64_t)idx;
      }
      t = old;
    }
    long long spins = 0;
    while (t == kBusy && spins < kSpinLimit) {
      t = *(volatile uint64_t*)s;
      ++spins;
    }
    if (t == kBusy) {
      set_status(P, kErrTimeout);
      return -1;
    }
    if (t == tag) {
      __threadfence();
      bool eq = true;
      for (int i = 0; i < R.nkeys; ++i) {
        const uint64_t a = ((volatile uint64_t*)s)[R.key_word + i];
        eq &= R.key_ctype[i] == DQ_STR ? str_ref_eq(P, a, k[i]) : a == k[i];
      }
      if (eq) return (int64_t)idx;
    }
    idx = (idx + 1 == R.cap) ? 0 : idx + 1;
  }
  set_status(P, kErrHtFull);
  return -1;
}

// Merges v into a global accumulator.  COUNT accumulators add v (1 per row,
// or a partial count when a CTA-local table is merged).
__device__ __forceinline__ void accumulate(uint64_t* acc, int red, uint64_t v) {
  switch (red) {
    case DQ_RED_SUM: atomicAdd((unsigned long long*)acc, v); break;
    case DQ_RED_COUNT: atomicAdd((unsigned long long*)acc, v); break;
    case DQ_RED_MIN: atomicMin((unsigned long long*)acc, v); break;
    case DQ_RED_MAX: atomicMax((unsigned long long*)acc, v); break;
  }
}

__device__ __forceinline__ uint64_t red_init(int red) { return red == DQ_RED_MIN ? ~0ull : 0ull; }

// Combines two partial aggregates (on the canonical 64-bit words).
__device__ __forceinline__ uint64_t red_combine(int red, uint64_t a, uint64_t b) {
  switch (red) {
    case DQ_RED_MIN: return a < b ? a : b;
    case DQ_RED_MAX: return a > b ? a : b;
    default: return a + b;
  }
}

// ------------------------------------------------------- shared memory --

__device__ __forceinline__ uint32_t saddr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ uint64_t s_cas64(uint32_t a, uint64_t cmp, uint64_t val) {
  uint64_t old;
  asm volatile("atom.shared.cas.b64 %0, [%1], %2, %3;" : "=l"(old) : "r"(a), "l"(cmp), "l"(val) : "memory");
  return old;
}

// A 64-bit shared-memory sum kept as two 32-bit words: a 32-bit atomic add of
// the low word returns the old word, whose wrap-around carries into the high
// word together with the value's high part (exact mod 2^64 once all adds are
// done).  64-bit shared-memory atomics run at about a third of the 32-bit rate
// on sm_100a, and most summed values have a zero high word.
__device__ __forceinline__ void s_add64(uint32_t a, uint64_t v) {
  const uint32_t lo = (uint32_t)v;
  uint32_t old;
  asm volatile("atom.shared.add.u32 %0, [%1], %2;" : "=r"(old) : "r"(a), "r"(lo) : "memory");
  const uint32_t hi = (uint32_t)(v >> 32) + (old + lo < old ? 1u : 0u);
  if (hi) asm volatile("red.shared.add.u32 [%0], %1;" ::"r"(a + 4), "r"(hi) : "memory");
}

__device__ __forceinline__ void s_merge(uint32_t a, int red, uint64_t v) {
  switch (red) {
    case DQ_RED_SUM:
    case DQ_RED_COUNT: s_add64(a, v); break;
    case DQ_RED_MIN: asm volatile("red.shared.min.u64 [%0], %1;" ::"r"(a), "l"(v) : "memory"); break;
    case DQ_RED_MAX: asm volatile("red.shared.max.u64 [%0], %1;" ::"r"(a), "l"(v) : "memory"); break;
  }
}

// Exact reduction of one aggregate over the lanes in `in` (all 32 lanes call
// it).  64-bit sums are split into 22-bit limbs so the 32-bit warp reductions
// cannot overflow; min/max reduce the high words, then the low words of the
// lanes holding the extreme high word.
__device__ __forceinline__ uint64_t warp_reduce(int red, bool in, uint64_t v, unsigned grp) {
  switch (red) {
    case DQ_RED_COUNT:
      return (uint64_t)__popc(grp);
    case DQ_RED_SUM: {
      uint32_t l0 = __reduce_add_sync(kFull, in ? (uint32_t)(v & 0x3fffff) : 0u);
      uint32_t l1 = __reduce_add_sync(kFull, in ? (uint32_t)((v >> 22) & 0x3fffff) : 0u);
      uint32_t l2 = __reduce_add_sync(kFull, in ? (uint32_t)(v >> 44) : 0u);
      return (uint64_t)l0 + ((uint64_t)l1 << 22) + ((uint64_t)l2 << 44);
    }
    case DQ_RED_MIN: {
      uint32_t hi = __reduce_min_sync(kFull, in ? (uint32_t)(v >> 32) : 0xffffffffu);
      uint32_t lo = __reduce_min_sync(kFull, (in && (uint32_t)(v >> 32) == hi) ? (uint32_t)v : 0xffffffffu);
      return ((uint64_t)hi << 32) | lo;
    }
    default: {
      uint32_t hi = __reduce_max_sync(kFull, in ? (uint32_t)(v >> 32) : 0u);
      uint32_t lo = __reduce_max_sync(kFull, (in && (uint32_t)(v >> 32) == hi) ? (uint32_t)v : 0u);
      return ((uint64_t)hi << 32) | lo;
    }
  }
}

// Warp reduction of a partial aggregate every lane holds (all lanes take part).
__device__ __forceinline__ uint64_t warp_reduce_all(int red, uint64_t v) {
  if (red == DQ_RED_COUNT) red = DQ_RED_SUM;
  return warp_reduce(red, true, v, kFull);
}

// CTA-local aggregation table through shared-memory atomics: ns slots plus
// one for the all-ones packed key; returns the slot or -1 when full.
__device__ __forceinline__ int local_group_slot(uint64_t* tags, int ns, uint64_t tag, int nkeys) {
  if (nkeys == 0) {
    tags[0] = 0;
    return 0;
  }
  if (tag == kEmpty) {
    s_cas64(saddr(&tags[ns]), kEmpty, 0ull);
    return ns;
  }
  uint32_t idx = slot_of(tag, (uint32_t)ns);
  for (int n = 0; n < ns; ++n) {
    uint64_t t = ((volatile uint64_t*)tags)[idx];
    if (t == tag) return (int)idx;
    if (t == kEmpty) {
      uint64_t old = s_cas64(saddr(&tags[idx]), kEmpty, tag);
      if (old == kEmpty || old == tag) return (int)idx;
    }
    idx = (idx + 1 == (uint32_t)ns) ? 0 : idx + 1;
  }
  return -1;
}

// CTA-local group table for hashed keys that include strings: tags, then the
// keys (string references) of each slot.  A claim publishes the keys before
// the tag; a match compares the keys (strings by their bytes).  -1 when the
// table is full or a claim stays unpublished past the wait limit: the caller
// then aggregates into the global table, whose flush merges by key.
__device__ __forceinline__ int local_group_slot_keys(const DevPipe& P, const DevRes& R, uint64_t* tags, uint64_t* keys,
                                                     int ns, uint64_t tag, const uint64_t* k) {
  uint32_t idx = slot_of(tag, (uint32_t)ns);
  for (int n = 0; n < ns; ++n) {
    uint64_t t = ((volatile uint64_t*)tags)[idx];
    if (t == kEmpty) {
      const uint64_t old = s_cas64(saddr(&tags[idx]), kEmpty, kBusy);
      if (old == kEmpty) {
        for (int i = 0; i < R.nkeys; ++i) ((volatile uint64_t*)keys)[idx * R.nkeys + i] = k[i];
        __threadfence_block();
        ((volatile uint64_t*)tags)[idx] = tag;
        return (int)idx;
      }
      t = old;
    }
    long long spins = 0;
    while (t == kBusy && spins < kSpinLimit) {
      t = ((volatile uint64_t*)tags)[idx];
      ++spins;
    }
    if (t == kBusy) return -1;
    if (t == tag) {
      __threadfence_block();
      bool eq = true;
      for (int i = 0; i < R.nkeys; ++i) {
        const uint64_t a = ((volatile uint64_t*)keys)[idx * R.nkeys + i];
        eq &= R.key_ctype[i] == DQ_STR ? str_ref_eq(P, a, k[i]) : a == k[i];
      }
      if (eq) return (int)idx;
    }
    idx = (idx + 1 == (uint32_t)ns) ? 0 : idx + 1;
  }
  return -1;
}

// CTA-local table of multimap buckets (the hot buckets of a skewed build side
// land in it first): kHotSlots bucket ids, kEmpty32 when free.  Returns the
// bucket's slot, claiming a free one in its window of kHotProbe slots, or -1.

__device__ __forceinline__ int hot_slot(uint32_t* keys, uint32_t b) {
  uint32_t idx = __umulhi(b * 0x9E3779B1u, (uint32_t)kHotSlots);
  for (int n = 0; n < kHotProbe; ++n) {
    const uint32_t k = ((volatile uint32_t*)keys)[idx];
    if (k == b) return (int)idx;
    if (k == kEmpty32) {
      const uint32_t old = atomicCAS(&keys[idx], kEmpty32, b);
      if (old == kEmpty32 || old == b) return (int)idx;
    }
    idx = (idx + 1) & (uint32_t)(kHotSlots - 1);
  }
  return -1;
}

__device__ __forceinline__ uint64_t shfl64(uint64_t v, int src) {
  uint32_t lo = __shfl_sync(kFull, (uint32_t)v, src);
  uint32_t hi = __shfl_sync(kFull, (uint32_t)(v >> 32), src);
  return ((uint64_t)hi << 32) | lo;
}

}  // namespace dq
