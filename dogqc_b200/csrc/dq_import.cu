// Text import kernels (sm_100a): a table in the reference's .tbl layout parsed
// on the device.
//
// The reference loads text on the host with generated C++ (dogqc/dbio.py:
// 117-253) around a CSV reader (dogqc/include/csv.h): one row per line, fields
// split at the delimiter, spaces trimmed, integers and floats parsed digit by
// digit, dates through the schema's toDate (query/schema/tpch.py:9-20), and a
// second pass over the file to fill the string heaps.  Here the whole text sits
// in HBM and four passes run over it:
//
//   1. count:   each CTA counts the newlines of a 16 KB tile (64 bytes a
//               thread, four 16-byte loads, a SIMD byte compare per word);
//   2. scan:    one CTA turns the tile counts into each tile's first line;
//   3. lines:   each CTA writes the byte positions of its newlines in order
//               (a block scan over the threads' counts places them);
//   4. parse:   one thread per row walks its line in 16-byte chunks held in
//               registers: delimiters are found with a byte-compare mask,
//               numbers are parsed as they stream past, strings are recorded
//               as (first byte, length);
//   5. strings: a prefix sum of the lengths (per-CTA sums from the parse pass,
//               then one CTA per column) gives the offsets, and each warp
//               copies the bytes of its 32 rows, coalesced on both sides.
//
// Every pass is a read of the text at most once from HBM (the parse pass
// reads each chunk through L1); the algorithmic traffic is the text, the line
// ends, and the columns written.
#include <cuda_runtime.h>
#include <stdint.h>

#include <climits>

#include "dq_device.h"

namespace dq {
namespace {

constexpr int kImpThreads = 256;
constexpr int kImpPerThread = kImpTile / kImpThreads;  // 64 bytes: four 16-byte chunks
constexpr int kScanThreads = 1024;
constexpr int kScanItems = 8;

// Bit 8k+7 set exactly for the zero bytes k of x: a byte's low seven bits plus
// 0x7F reach bit 7 unless they are all zero, and its own bit 7 rules out the
// rest; no carry leaves a byte (the classic exact zero-byte test).  XOR with a
// repeated byte first to find that byte.
__device__ __forceinline__ uint32_t zero_bytes(uint32_t x) {
  return ~(((x & 0x7F7F7F7Fu) + 0x7F7F7F7Fu) | x | 0x7F7F7F7Fu);
}

// Zero-byte flags of a word (bits 7, 15, 23, 31) as a nibble (byte k -> bit
// k): the flags move to bits 24..27 by one multiply whose partial products do
// not overlap.  Four nibbles make a 16-byte chunk's mask.
__device__ __forceinline__ uint32_t nibble_of(uint32_t z) { return (((z >> 7) & 0x01010101u) * 0x01020408u) >> 24; }
__device__ __forceinline__ uint32_t newline_mask16(const uint4& v) {
  return nibble_of(zero_bytes(v.x ^ 0x0a0a0a0au)) | (nibble_of(zero_bytes(v.y ^ 0x0a0a0a0au)) << 4) |
         (nibble_of(zero_bytes(v.z ^ 0x0a0a0a0au)) << 8) | (nibble_of(zero_bytes(v.w ^ 0x0a0a0a0au)) << 12);
}

__device__ __forceinline__ uint4 ld_chunk(const uint8_t* p) {
  return __ldg(reinterpret_cast<const uint4*>(p));
}

// Byte `i` of the text lives in the main part or in the padded tail tile.
__device__ __forceinline__ const uint8_t* text_at(const ImpText& T, uint64_t i) {
  return i < T.nmain ? T.main + i : T.tail + (i - T.nmain);
}

// Exclusive block scan of one value per thread (any power-of-two block up to
// 1024); returns the total.
template <int kBlock, class T>
__device__ T block_scan(T x, T& excl) {
  constexpr int kW = kBlock / 32;
  __shared__ T s_w[kW + 1];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  T incl = x;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const T y = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += y;
  }
  if (lane == 31) s_w[warp] = incl;
  __syncthreads();
  if (warp == 0) {
    T v = lane < kW ? s_w[lane] : T(0);
    T vi = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const T y = __shfl_up_sync(0xffffffffu, vi, o);
      if (lane >= o) vi += y;
    }
    if (lane < kW) s_w[lane] = vi - v;
    if (lane == kW - 1) s_w[kW] = vi;
  }
  __syncthreads();
  excl = s_w[warp] + incl - x;
  const T total = s_w[kW];
  __syncthreads();
  return total;
}

// ------------------------------------------------------------ newlines --

__global__ void __launch_bounds__(kImpThreads) imp_count_kernel(const ImpText T, uint64_t* tile_cnt) {
  const uint8_t* p = text_at(T, (uint64_t)blockIdx.x * kImpTile) + threadIdx.x * kImpPerThread;
  uint32_t n = 0;
#pragma unroll
  for (int k = 0; k < kImpPerThread / 16; ++k) {
    const uint4 v = ld_chunk(p + 16 * k);
    n += __popc(zero_bytes(v.x ^ 0x0a0a0a0au)) + __popc(zero_bytes(v.y ^ 0x0a0a0a0au)) +
         __popc(zero_bytes(v.z ^ 0x0a0a0a0au)) + __popc(zero_bytes(v.w ^ 0x0a0a0a0au));
  }
  uint32_t excl;
  const uint32_t total = block_scan<kImpThreads>(n, excl);
  if (threadIdx.x == 0) tile_cnt[blockIdx.x] = total;
}

__global__ void __launch_bounds__(kImpThreads) imp_lines_kernel(const ImpText T, const uint64_t* tile_off,
                                                                uint64_t* line_end) {
  const uint64_t first = (uint64_t)blockIdx.x * kImpTile + threadIdx.x * kImpPerThread;
  const uint8_t* p = text_at(T, (uint64_t)blockIdx.x * kImpTile) + threadIdx.x * kImpPerThread;
  uint32_t m[kImpPerThread / 16];  // per 16-byte chunk: bit k for a newline at byte k
  uint32_t n = 0;
#pragma unroll
  for (int k = 0; k < kImpPerThread / 16; ++k) {
    m[k] = newline_mask16(ld_chunk(p + 16 * k));
    n += __popc(m[k]);
  }
  uint32_t excl;
  block_scan<kImpThreads>(n, excl);
  uint64_t at = tile_off[blockIdx.x] + excl;
#pragma unroll
  for (int k = 0; k < kImpPerThread / 16; ++k) {
    uint32_t b = m[k];
    while (b) {
      line_end[at++] = first + 16 * k + (__ffs(b) - 1);
      b &= b - 1;
    }
  }
}

// One CTA per segment: out[i] = in[0] + ... + in[i - 1], out[n] = the total.
__global__ void __launch_bounds__(kScanThreads) imp_scan_kernel(const uint64_t* in, uint64_t* out, uint64_t n,
                                                                uint64_t stride) {
  in += blockIdx.x * stride;
  out += blockIdx.x * stride;
  uint64_t carry = 0;
  for (uint64_t base = 0; base < n; base += (uint64_t)kScanThreads * kScanItems) {
    const uint64_t i0 = base + (uint64_t)threadIdx.x * kScanItems;
    uint64_t v[kScanItems], s = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
      v[k] = i0 + k < n ? in[i0 + k] : 0;
      s += v[k];
    }
    uint64_t excl;
    const uint64_t total = block_scan<kScanThreads>(s, excl);
    uint64_t run = carry + excl;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
      if (i0 + k < n) out[i0 + k] = run;
      run += v[k];
    }
    carry += total;
  }
  if (threadIdx.x == 0) out[n] = carry;
}

// ---------------------------------------------------------------- parse --

// A thread's view of its line: the 16-byte chunk last loaded, in registers,
// with the mask of its delimiter bytes (computed once per chunk: the fields
// of a line share its chunks).
struct LineReader {
  ImpText text;
  uint32_t pat;           // the delimiter in every byte
  uint64_t base = ~0ull;
  uint4 v;
  uint32_t dm = 0;        // bit k: byte k of the chunk is the delimiter

  __device__ __forceinline__ void fetch(uint64_t i) {
    const uint64_t b = i & ~15ull;
    if (b != base) {
      v = ld_chunk(text_at(text, b));
      base = b;
      dm = nibble_of(zero_bytes(v.x ^ pat)) | (nibble_of(zero_bytes(v.y ^ pat)) << 4) |
           (nibble_of(zero_bytes(v.z ^ pat)) << 8) | (nibble_of(zero_bytes(v.w ^ pat)) << 12);
    }
  }
  // First byte equal to the delimiter in [i, end); `end` if there is none.
  __device__ __forceinline__ uint64_t find(uint64_t i, uint64_t end) {
    while (i < end) {
      fetch(i);
      const uint32_t m = dm >> (i & 15);
      if (m) {
        const uint64_t q = i + (__ffs(m) - 1);
        return q < end ? q : end;
      }
      i = base + 16;
    }
    return end;
  }
};

// One byte of the text (trimming and the line's last byte: a load that hits
// L1, without disturbing the reader's chunk).
__device__ __forceinline__ uint32_t byte_at(const ImpText& T, uint64_t i) { return __ldg(text_at(T, i)); }

// Field [i, q) of a line ending at `end`, with the spaces around it trimmed
// to [cs, ce).  Returns a reason code, 0 when the delimiter was found.
__device__ __forceinline__ int32_t field_bounds(LineReader& rd, uint64_t i, uint64_t end, uint64_t& q,
                                                uint64_t& cs, uint64_t& ce) {
  q = rd.find(i, end);
  if (q >= end) return kImpTooFew;
  cs = i;
  ce = q;
  while (cs < ce && byte_at(rd.text, cs) == ' ') ++cs;
  while (ce > cs && byte_at(rd.text, ce - 1) == ' ') --ce;
  return 0;
}

// ---------------------------------------------------------- date window --
// A date field of 10 to 16 bytes with no spaces around it is read from a
// 16-byte window in registers; anything else goes to the byte-at-a-time path
// below, which gives the same value or the exact reason.  (Numbers stay on the
// byte-at-a-time parsers: on fields of a few digits a window, a digit check
// and a SWAR conversion cost more than one pass over the bytes.)

// Bytes [i, i + 16) of the text as two little-endian halves (w0: bytes 0-7),
// from the chunk holding i and the next one (both lie in the padded text).
// Branch-free: the word offset selects in two steps, the byte offset is one
// byte permute per word.
struct Window {
  uint64_t w0, w1;
};

__device__ __forceinline__ Window load_window(const ImpText& T, uint64_t i) {
  const uint64_t b = i & ~15ull;
  const uint32_t sh = (uint32_t)i & 15u;
  const uint4 a = ld_chunk(text_at(T, b));
  const uint4 c = ld_chunk(text_at(T, b + 16));
  const bool s1 = sh & 4u, s2 = sh & 8u;
  // z[j] = x[j + (sh>>2 & 1)], then y[k] = z[k + 2 * (sh>>3 & 1)] over x = a.x .. c.w
  const uint32_t z0 = s1 ? a.y : a.x, z1 = s1 ? a.z : a.y, z2 = s1 ? a.w : a.z, z3 = s1 ? c.x : a.w,
                 z4 = s1 ? c.y : c.x, z5 = s1 ? c.z : c.y, z6 = s1 ? c.w : c.z;
  const uint32_t y0 = s2 ? z2 : z0, y1 = s2 ? z3 : z1, y2 = s2 ? z4 : z2, y3 = s2 ? z5 : z3, y4 = s2 ? z6 : z4;
  const uint32_t sel = 0x3210u + 0x1111u * (sh & 3u);
  Window W;
  W.w0 = ((uint64_t)__byte_perm(y1, y2, sel) << 32) | __byte_perm(y0, y1, sel);
  W.w1 = ((uint64_t)__byte_perm(y3, y4, sel) << 32) | __byte_perm(y2, y3, sel);
  return W;
}

__device__ __forceinline__ uint32_t win_byte(const Window& W, uint32_t k) {
  return (uint32_t)((k < 8 ? W.w0 >> (8 * k) : W.w1 >> (8 * (k - 8))) & 0xffu);
}

// DATE from the untrimmed field [i, q) of 10 to 16 bytes without spaces
// around it (query/schema/tpch.py:9-20 over bytes 0-3, 5-6, 8-9).
__device__ __forceinline__ bool fast_date(const ImpText& T, uint64_t i, uint64_t q, uint32_t& out) {
  const uint32_t n = (uint32_t)(q - i);
  if (n < 10 || n > 16) return false;
  const Window W = load_window(T, i);
  if ((W.w0 & 0xffu) == ' ' || win_byte(W, n - 1) == ' ') return false;
  const uint32_t a = (uint32_t)W.w0, b = (uint32_t)(W.w0 >> 32), c = (uint32_t)W.w1;
  out = ((a & 0xffu) - 48u) * 10000000u + (((a >> 8) & 0xffu) - 48u) * 1000000u +
        (((a >> 16) & 0xffu) - 48u) * 100000u + ((a >> 24) - 48u) * 10000u +
        (((b >> 8) & 0xffu) - 48u) * 1000u + (((b >> 16) & 0xffu) - 48u) * 100u +
        ((c & 0xffu) - 48u) * 10u + (((c >> 8) & 0xffu) - 48u);
  return true;
}

// The bytes of a field in order: one aligned 4-byte load per four bytes, then
// shifts (the padded text holds every word a line touches).
struct ByteStream {
  const ImpText& T;
  uint64_t pos;
  uint32_t w = 0, left = 0;
  __device__ __forceinline__ ByteStream(const ImpText& t, uint64_t i) : T(t), pos(i) {}
  __device__ __forceinline__ uint32_t next() {
    if (left == 0) {
      const uint32_t sh = (uint32_t)pos & 3u;
      w = __ldg(reinterpret_cast<const uint32_t*>(text_at(T, pos - sh))) >> (8 * sh);
      left = 4 - sh;
    }
    const uint32_t c = w & 0xffu;
    w >>= 8;
    --left;
    ++pos;
    return c;
  }
};

// csv.h parse_signed_integer for int, throw_on_overflow (csv.h:945-995), on
// the trimmed field: the magnitude is checked against the bound after every
// digit, which is the reference's test (x > (max - y) / 10 is 10x + y > max),
// so an overflow is reported at the same digit.
__device__ int32_t parse_int(const ImpText& T, uint64_t& i, uint64_t end, uint32_t delim, int32_t& out) {
  ByteStream bs(T, i);
  int state = 0;  // 0: before the value, 1: in it, 2: trailing spaces
  uint64_t lim = 2147483647ull, u = 0;
  bool neg = false;
  for (;; ++i) {
    if (i >= end) return kImpTooFew;
    const uint32_t c = bs.next();
    if (c == delim) break;
    if (c == ' ') {
      if (state == 1) state = 2;
      continue;
    }
    if (state == 2) return kImpNoDigit;  // a space inside the value
    if (state == 0) {
      state = 1;
      if (c == '-') {
        neg = true;
        lim = 2147483648ull;
        continue;
      }
      if (c == '+') continue;
    }
    const uint32_t y = c - '0';
    if (y > 9) return kImpNoDigit;
    u = u * 10 + y;
    if (u > lim) return kImpOverflow;
  }
  out = neg ? (int32_t)(0u - (uint32_t)u) : (int32_t)u;
  return 0;
}

// Exact fixed point: [+-]digits[(.|,)digits] scaled by 10^scale, digits past
// `scale` dropped (the grammar of csv.h parse_float without the exponent).
__device__ int32_t parse_decimal(const ImpText& T, uint64_t& i, uint64_t end, uint32_t delim, int scale,
                                 int64_t& out) {
  ByteStream bs(T, i);
  int state = 0;  // 0: before, 1: integer digits, 3: fraction digits, 2: trailing spaces
  bool neg = false;
  uint64_t m = 0;
  int fd = 0;
  constexpr uint64_t kMax = (uint64_t)INT64_MAX, kTenth = kMax / 10, kLast = kMax % 10;
  for (;; ++i) {
    if (i >= end) return kImpTooFew;
    const uint32_t c = bs.next();
    if (c == delim) break;
    if (c == ' ') {
      if (state != 0) state = 2;
      continue;
    }
    if (state == 2) return kImpNoDigit;
    if (state == 0) {
      state = 1;
      if (c == '-' || c == '+') {
        neg = c == '-';
        continue;
      }
    }
    if ((c == '.' || c == ',') && state == 1) {
      state = 3;
      continue;
    }
    if (c == 'e' || c == 'E') return kImpExponent;
    const uint32_t y = c - '0';
    if (y > 9) return kImpNoDigit;
    if (state == 3) {
      if (fd >= scale) continue;
      ++fd;
    }
    if (m > kTenth || (m == kTenth && y > kLast)) return kImpOverflow;
    m = 10 * m + y;
  }
  for (; fd < scale; ++fd) {
    if (m > kTenth) return kImpOverflow;
    m *= 10;
  }
  out = neg ? -(int64_t)m : (int64_t)m;
  return 0;
}

// csv.h parse_float for float (csv.h:1008-1069), step for step: every product,
// quotient and sum rounded to binary32 on its own (the reference's host code
// is compiled without contraction), the sign applied last.  Exponents beyond
// four digits are rejected (the reference saturates them and, for the most
// negative one, does not terminate).
__device__ int32_t parse_float(const ImpText& T, uint64_t& i, uint64_t end, uint32_t delim, uint32_t& out) {
  ByteStream bs(T, i);
  int state = 0;  // 0: before, 1: integer digits, 3: fraction digits, 4: exponent, 2: trailing spaces
  bool neg = false, eneg = false, esign = false;
  float x = 0.f, pos = 1.f;
  int e = 0;
  for (;; ++i) {
    if (i >= end) return kImpTooFew;
    const uint32_t c = bs.next();
    if (c == delim) break;
    if (c == ' ') {
      if (state != 0) state = 2;
      continue;
    }
    if (state == 2) return kImpNoDigit;
    if (state == 0) {
      state = 1;
      if (c == '-' || c == '+') {
        neg = c == '-';
        continue;
      }
    }
    if (state == 4) {
      if (!esign && e == 0 && (c == '-' || c == '+')) {  // the exponent's own sign, first
        esign = true;
        eneg = c == '-';
        continue;
      }
      esign = true;
      if (c < '0' || c > '9') return kImpNoDigit;
      e = e * 10 + (int)(c - '0');
      if (e > 9999) return kImpExponent;
      continue;
    }
    if ((c == '.' || c == ',') && state == 1) {
      state = 3;
      continue;
    }
    if (c == 'e' || c == 'E') {
      state = 4;
      continue;
    }
    if (c < '0' || c > '9') return kImpNoDigit;
    const float y = (float)(int)(c - '0');
    if (state == 1) {
      x = __fadd_rn(__fmul_rn(x, 10.f), y);
    } else {
      pos = __fdiv_rn(pos, 10.f);
      x = __fadd_rn(x, __fmul_rn(y, pos));
    }
  }
  if (eneg) e = -e;
  if (e != 0) {
    float b = e < 0 ? 0.1f : 10.f;
    if (e < 0) e = -e;
    while (e != 1) {
      if ((e & 1) == 0) {
        b = __fmul_rn(b, b);
        e >>= 1;
      } else {
        x = __fmul_rn(x, b);
        --e;
      }
    }
    x = __fmul_rn(x, b);
  }
  if (neg) x = -x;
  out = __float_as_uint(x);
  return 0;
}

__global__ void __launch_bounds__(kImpRows, 6) imp_parse_kernel(const ImpArgs A) {
  const uint64_t r = (uint64_t)blockIdx.x * kImpRows + threadIdx.x;
  const bool live = r < A.nrows;
  const uint32_t delim = A.delim;
  LineReader rd{A.text, delim * 0x01010101u};
  uint64_t pos = 0, end = 0;
  int32_t bad = 0, bad_field = 0;
  bool shape_bad = false;  // the line has too few delimiters: that outranks a bad value
  if (live) {
    pos = r ? A.line_end[r - 1] + 1 : 0;
    end = r < A.nlines ? A.line_end[r] : A.nbytes;
    if (end > pos && byte_at(A.text, end - 1) == '\r') --end;  // csv.h:479, Windows line breaks
  }
  for (int f = 0; f < A.nfields; ++f) {
    if (!live || shape_bad) continue;
    if (bad) {  // after a bad value only the delimiters are checked (csv.h splits the line first)
      const uint64_t q = rd.find(pos, end);
      if (q >= end) {
        bad = kImpTooFew;
        bad_field = f;
        shape_bad = true;
      }
      pos = q + 1;
      continue;
    }
    const ImpField F = A.f[f];
    uint64_t q = pos, cs = 0, ce = 0;
    int32_t why = 0;
    switch (F.kind) {
      case kTxtInt: {
        int32_t v = 0;
        why = parse_int(A.text, q, end, delim, v);
        if (!why) static_cast<int32_t*>(F.out)[r] = v;
        break;
      }
      case kTxtDecimal: {
        int64_t v = 0;
        why = parse_decimal(A.text, q, end, delim, F.scale, v);
        if (!why) static_cast<int64_t*>(F.out)[r] = v;
        break;
      }
      case kTxtFloat: {
        uint32_t v = 0;
        why = parse_float(A.text, q, end, delim, v);
        if (!why) static_cast<uint32_t*>(F.out)[r] = v;
        break;
      }
      case kTxtDate: {
        uint32_t v = 0;
        const uint64_t d = rd.find(pos, end);
        if (d < end && fast_date(A.text, pos, d, v)) {
          q = d;
          static_cast<uint32_t*>(F.out)[r] = v;
          break;
        }
        why = field_bounds(rd, pos, end, q, cs, ce);
        if (!why && ce - cs < 10) why = kImpShortDate;
        if (!why) {
          // toDate: digits at 0-3, 5-6, 8-9 weighted 10^7 .. 10^0 (query/schema/tpch.py:9-20)
          constexpr uint32_t kW[10] = {10000000u, 1000000u, 100000u, 10000u, 0u, 1000u, 100u, 0u, 10u, 1u};
          uint32_t d = 0;
#pragma unroll
          for (int k = 0; k < 10; ++k)
            if (kW[k]) d += (byte_at(A.text, cs + k) - 48u) * kW[k];
          static_cast<uint32_t*>(F.out)[r] = d;
        }
        break;
      }
      case kTxtChar: {
        why = field_bounds(rd, pos, end, q, cs, ce);
        if (!why && ce - cs != 1) why = kImpNotChar;  // csv.h:920-928
        if (!why) static_cast<int8_t*>(F.out)[r] = (int8_t)byte_at(A.text, cs);
        break;
      }
      case kTxtString: {
        why = field_bounds(rd, pos, end, q, cs, ce);
        if (!why) {
          A.spos[(uint64_t)F.str * A.nrows + r] = cs;
          A.slen[(uint64_t)F.str * A.nrows + r] = (uint32_t)(ce - cs);
        }
        break;
      }
      default: {  // kTxtSkip
        q = rd.find(pos, end);
        if (q >= end) why = kImpTooFew;
        break;
      }
    }
    if (why && why != kImpTooFew) {
      q = rd.find(q, end);  // the field's own delimiter, past the bad byte
      if (q >= end) why = kImpTooFew;
    }
    if (why) {
      bad = why;
      bad_field = f;
      shape_bad = why == kImpTooFew;
    }
    pos = q + 1;
  }
  if (live && !shape_bad && rd.find(pos, end) < end) {  // csv.h:864-866: one delimiter too many
    bad = kImpTooMany;
    bad_field = A.nfields;
  }
  if (bad) atomicMin(reinterpret_cast<unsigned long long*>(A.err),
                     (unsigned long long)(r << 16 | (uint64_t)bad_field << 8 | (uint64_t)bad));
  // string bytes of this CTA, per string column
  for (int j = 0; j < A.nstr; ++j) {
    uint64_t len = live && !bad ? A.slen[(uint64_t)j * A.nrows + r] : 0;
    if (live && bad) A.slen[(uint64_t)j * A.nrows + r] = 0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) len += __shfl_xor_sync(0xffffffffu, len, o);
    __shared__ uint64_t s_sum[kImpRows / 32];
    if ((threadIdx.x & 31) == 0) s_sum[threadIdx.x >> 5] = len;
    __syncthreads();
    if (threadIdx.x == 0) {
      uint64_t t = 0;
      for (int w = 0; w < kImpRows / 32; ++w) t += s_sum[w];
      A.bsum[(uint64_t)j * (A.nblocks + 1) + blockIdx.x] = t;
    }
    __syncthreads();
  }
}

// Offsets from the per-CTA prefix sums, then each warp copies the bytes of
// its 32 rows, which are contiguous in the heap: lane k moves bytes k, k + 32,
// ... of that run, finding the row of its byte by a binary search over the
// rows' starts (shuffles), so every lane moves a byte on every step.  One CTA
// does every string column of its rows, so their lines are read from HBM once.
__global__ void __launch_bounds__(kImpRows) imp_strings_kernel(const ImpArgs A) {
  const uint64_t r = (uint64_t)blockIdx.x * kImpRows + threadIdx.x;
  const bool live = r < A.nrows;
  const int lane = threadIdx.x & 31;
  for (int j = 0; j < A.nstr; ++j) {
    const uint64_t len = live ? A.slen[(uint64_t)j * A.nrows + r] : 0;
    const uint64_t src = live ? A.spos[(uint64_t)j * A.nrows + r] : 0;
    uint64_t excl;
    block_scan<kImpRows>(len, excl);
    const uint64_t off = A.boff[(uint64_t)j * (A.nblocks + 1) + blockIdx.x] + excl;
    uint64_t* offs = A.soff[j];
    if (live) {
      offs[r] = off;
      if (r + 1 == A.nrows) offs[r + 1] = off + len;
    }
    uint64_t wincl = len;  // warp-relative run of the rows' bytes
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint64_t y = __shfl_up_sync(0xffffffffu, wincl, o);
      if (lane >= o) wincl += y;
    }
    const uint64_t wstart = wincl - len;
    const uint64_t wtotal = __shfl_sync(0xffffffffu, wincl, 31);
    uint8_t* dst = A.sheap[j] + __shfl_sync(0xffffffffu, off, 0);
    // The rows of a warp are consecutive lines: with the run and the lines'
    // span below 4 GB (always, short of multi-GB lines) the search works on
    // 32-bit values, one shuffle a step.
    const uint64_t src0 = __shfl_sync(0xffffffffu, src, 0);
    const bool narrow = __all_sync(0xffffffffu, wincl < (1ull << 32) && (len == 0 || src - src0 < (1ull << 32)));
    if (narrow) {
      const uint32_t ws32 = (uint32_t)wstart, wt32 = (uint32_t)wtotal;
      const uint32_t rel = len ? (uint32_t)(src - src0) - ws32 : 0u;  // source offset minus run offset
      for (uint32_t b0 = 0; b0 < wt32; b0 += 32) {
        const uint32_t b = b0 + lane;
        int row = 0;
#pragma unroll
        for (int step = 16; step > 0; step >>= 1) {
          const uint32_t st = __shfl_sync(0xffffffffu, ws32, row + step);
          if (st <= b) row += step;
        }
        const uint32_t d = __shfl_sync(0xffffffffu, rel, row);
        if (b < wt32) dst[b] = *text_at(A.text, src0 + (uint32_t)(b + d));
      }
    } else {
      for (uint64_t b0 = 0; b0 < wtotal; b0 += 32) {
        const uint64_t b = b0 + lane;
        int row = 0;
#pragma unroll
        for (int step = 16; step > 0; step >>= 1) {
          const uint64_t st = __shfl_sync(0xffffffffu, wstart, row + step);
          if (st <= b) row += step;
        }
        const uint64_t rs = __shfl_sync(0xffffffffu, wstart, row);
        const uint64_t rsrc = __shfl_sync(0xffffffffu, src, row);
        if (b < wtotal) dst[b] = *text_at(A.text, rsrc + (b - rs));
      }
    }
  }
}

// ------------------------------------------------------- string results --
// Result columns of string type hold references (source, substring window, row); these
// turn them into offsets and a heap: the lengths, their prefix sum (the scan
// above), then one warp per row copies its bytes.

__global__ void str_ref_len_kernel(const uint64_t* refs, uint64_t n, const DevStr* src, uint64_t* lens) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint8_t* p;
    int n;
    str_ref_bytes(src, refs[i], p, n);
    lens[i] = (uint64_t)n;
  }
}

__global__ void str_ref_copy_kernel(const uint64_t* refs, uint64_t n, const DevStr* src, const uint64_t* offs,
                                    uint8_t* heap) {
  const int lane = threadIdx.x & 31;
  const uint64_t warps = (uint64_t)gridDim.x * (blockDim.x / 32);
  for (uint64_t i = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) / 32; i < n; i += warps) {
    const uint8_t* from;
    int n;
    str_ref_bytes(src, refs[i], from, n);
    const uint64_t len = offs[i + 1] - offs[i];
    for (uint64_t b = lane; b < len; b += 32) heap[offs[i] + b] = from[b];
  }
}

}  // namespace

cudaError_t launch_str_ref_offsets(const uint64_t* refs, uint64_t n, const DevStr* src, uint64_t* lens,
                                   uint64_t* offs, int sms, cudaStream_t st) {
  if (n) str_ref_len_kernel<<<sms * 4, 256, 0, st>>>(refs, n, src, lens);
  imp_scan_kernel<<<1, kScanThreads, 0, st>>>(lens, offs, n, 0);
  return cudaGetLastError();
}

cudaError_t launch_str_ref_copy(const uint64_t* refs, uint64_t n, const DevStr* src, const uint64_t* offs,
                                uint8_t* heap, int sms, cudaStream_t st) {
  if (n) str_ref_copy_kernel<<<sms * 8, 256, 0, st>>>(refs, n, src, offs, heap);
  return cudaGetLastError();
}

cudaError_t launch_import_lines(const ImpText& T, uint64_t ntiles, uint64_t* tile_cnt, uint64_t* tile_off,
                                cudaStream_t st) {
  imp_count_kernel<<<(unsigned)ntiles, kImpThreads, 0, st>>>(T, tile_cnt);
  imp_scan_kernel<<<1, kScanThreads, 0, st>>>(tile_cnt, tile_off, ntiles, 0);
  return cudaGetLastError();
}

cudaError_t launch_import_line_ends(const ImpText& T, uint64_t ntiles, const uint64_t* tile_off, uint64_t* line_end,
                                    cudaStream_t st) {
  imp_lines_kernel<<<(unsigned)ntiles, kImpThreads, 0, st>>>(T, tile_off, line_end);
  return cudaGetLastError();
}

cudaError_t launch_import_parse(const ImpArgs& A, cudaStream_t st) {
  if (A.nrows == 0) return cudaSuccess;
  imp_parse_kernel<<<(unsigned)A.nblocks, kImpRows, 0, st>>>(A);
  if (A.nstr > 0) imp_scan_kernel<<<A.nstr, kScanThreads, 0, st>>>(A.bsum, A.boff, A.nblocks, A.nblocks + 1);
  return cudaGetLastError();
}

// Smallest and largest value of an integer column (`width` bytes a value,
// sign-extended when `is_signed`) into out[0], out[1] (initialised by the caller
// to INT64_MAX, INT64_MIN).
__global__ void col_minmax_kernel(const uint8_t* col, uint64_t n, int width, int is_signed, long long* out) {
  long long lo = LLONG_MAX, hi = LLONG_MIN;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    long long v;
    if (width == 1) v = is_signed ? (long long)(int8_t)col[i] : (long long)col[i];
    else if (width == 4) {
      const uint32_t u = reinterpret_cast<const uint32_t*>(col)[i];
      v = is_signed ? (long long)(int32_t)u : (long long)u;
    } else {
      v = (long long)reinterpret_cast<const uint64_t*>(col)[i];
    }
    lo = v < lo ? v : lo;
    hi = v > hi ? v : hi;
  }
  for (int o = 16; o > 0; o >>= 1) {
    const long long a = __shfl_xor_sync(0xffffffffu, lo, o), b = __shfl_xor_sync(0xffffffffu, hi, o);
    lo = a < lo ? a : lo;
    hi = b > hi ? b : hi;
  }
  if ((threadIdx.x & 31) == 0) {
    atomicMin(out, lo);
    atomicMax(out + 1, hi);
  }
}

cudaError_t launch_col_minmax(const uint8_t* col, uint64_t n, int width, bool is_signed, long long* out, int sms,
                              cudaStream_t st) {
  if (n) col_minmax_kernel<<<sms * 4, 256, 0, st>>>(col, n, width, is_signed ? 1 : 0, out);
  return cudaGetLastError();
}

cudaError_t launch_import_strings(const ImpArgs& A, cudaStream_t st) {
  if (A.nrows == 0 || A.nstr == 0) return cudaSuccess;
  imp_strings_kernel<<<(unsigned)A.nblocks, kImpRows, 0, st>>>(A);
  return cudaGetLastError();
}

}  // namespace dq
