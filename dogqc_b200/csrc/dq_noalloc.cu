// FK-PK hash join + grouped SUM/COUNT that allocates no device memory.
//
// Some callers cannot allocate device memory on their own: code running inside
// a host application that owns every device allocation through its own pool,
// plugins loaded into processes whose allocator must account for all memory,
// or callers on a path where cudaMalloc would synchronise the device.  For them
// this file keeps the scratch of the join (hash table, group table, counters)
// in one statically sized device array that exists once per device for the
// lifetime of the process; the caller passes only inputs and outputs.
//
// The computation is the plan shape
//   aggregation([group], [SUM(value), COUNT]) (
//     join(build.key = probe.key, selection(build.filter == v, build), probe))
// with the engine's semantics: unique build keys (the first inserted row wins
// for duplicates), SUM as a wrapping 64-bit unsigned sum, COUNT as a 32-bit
// count.
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "../../include/dogqc_b200.h"

namespace dq_internal {
void set_global_error(const std::string& msg);
}

namespace {

constexpr uint64_t kEmptyTag = ~0ull;
constexpr uint64_t kSlots = 2ull * DQ_NOALLOC_MAX_BUILD_ROWS;   // hash-table slots (load <= 1/2)
constexpr int kGroupSlots = 2 * DQ_NOALLOC_MAX_GROUPS;          // group-table slots
constexpr int kThreads = 256;

struct Scratch {
  unsigned long long ht[2 * kSlots];         // per slot: packed key tag, group
  unsigned long long gtag[kGroupSlots];      // packed group key or empty
  unsigned long long gsum[kGroupSlots];
  unsigned long long gcnt[kGroupSlots];
  unsigned long long ngroups;                // groups written by the last call
  unsigned long long overflow;               // groups beyond the table
};

// The scratch.  Host code must not pass this symbol to a kernel: on the host it
// names a stand-in, not device memory.  Its device address comes from
// cudaGetSymbolAddress, once per device (scratch_on_device below).
static __device__ __align__(256) Scratch g_scratch;

__device__ __forceinline__ uint64_t mix(uint64_t k) {
  k ^= k >> 33;
  k *= 0xff51afd7ed558ccdull;
  k ^= k >> 33;
  k *= 0xc4ceb9fe1a85ec53ull;
  k ^= k >> 33;
  return k;
}

__global__ void clear_kernel(Scratch* s) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < kSlots; i += stride)
    s->ht[2 * i] = kEmptyTag;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < (uint64_t)kGroupSlots; i += stride) {
    s->gtag[i] = kEmptyTag;
    s->gsum[i] = 0;
    s->gcnt[i] = 0;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    s->ngroups = 0;
    s->overflow = 0;
  }
}

__global__ void build_kernel(Scratch* s, const int32_t* key, const int32_t* filter, int32_t value,
                             const int32_t* group, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    if (filter[i] != value) continue;
    const uint64_t tag = (uint32_t)key[i];
    uint64_t j = __umul64hi(mix(tag), kSlots);
    for (uint64_t q = 0; q < kSlots; ++q) {
      unsigned long long old = atomicCAS(&s->ht[2 * j], kEmptyTag, tag);
      if (old == kEmptyTag) {
        s->ht[2 * j + 1] = (uint32_t)group[i];
        break;
      }
      if (old == tag) break;  // duplicate key: the first row wins
      j = (j + 1 == kSlots) ? 0 : j + 1;
    }
  }
}

__device__ int group_slot(Scratch* s, uint64_t g) {
  uint32_t j = (uint32_t)__umul64hi(mix(g), (uint64_t)kGroupSlots);
  for (int q = 0; q < kGroupSlots; ++q) {
    unsigned long long t = ((volatile unsigned long long*)s->gtag)[j];
    if (t == g) return (int)j;
    if (t == kEmptyTag) {
      unsigned long long old = atomicCAS(&s->gtag[j], kEmptyTag, g);
      if (old == kEmptyTag || old == g) return (int)j;
    }
    j = (j + 1 == (uint32_t)kGroupSlots) ? 0 : j + 1;
  }
  return -1;
}

__global__ void probe_kernel(Scratch* s, const int32_t* key, const uint64_t* value, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const uint64_t tag = (uint32_t)key[i];
    uint64_t j = __umul64hi(mix(tag), kSlots);
    for (uint64_t q = 0; q < kSlots; ++q) {
      const uint64_t t = s->ht[2 * j];
      if (t == kEmptyTag) break;
      if (t == tag) {
        int g = group_slot(s, s->ht[2 * j + 1]);
        if (g < 0) {
          atomicAdd(&s->overflow, 1ull);
        } else {
          atomicAdd(&s->gsum[g], (unsigned long long)value[i]);
          atomicAdd(&s->gcnt[g], 1ull);
        }
        break;
      }
      j = (j + 1 == kSlots) ? 0 : j + 1;
    }
  }
}

__global__ void output_kernel(Scratch* s, int32_t* out_group, uint64_t* out_sum, int32_t* out_count,
                              int32_t max_groups) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < kGroupSlots; i += gridDim.x * blockDim.x) {
    if (s->gtag[i] == kEmptyTag) continue;
    unsigned long long pos = atomicAdd(&s->ngroups, 1ull);
    if (pos < (unsigned long long)max_groups) {
      out_group[pos] = (int32_t)(uint32_t)s->gtag[i];
      out_sum[pos] = s->gsum[i];
      out_count[pos] = (int32_t)(uint32_t)s->gcnt[i];
    }
  }
}

__global__ void finish_kernel(const Scratch* s, int64_t* out_ngroups, int32_t max_groups) {
  // -1 reports groups that did not fit the caller's output or the group table
  *out_ngroups = (s->overflow || s->ngroups > (unsigned long long)max_groups) ? -1 : (int64_t)s->ngroups;
}

std::mutex g_mu;
Scratch* g_addr[64];

// Device address of the scratch on the current device, looked up once per device.
int scratch_on_device(Scratch** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess || dev < 0 || dev >= 64) {
    dq_internal::set_global_error("dq_join_agg_noalloc: no usable current device");
    return DQ_ERR_CUDA;
  }
  std::lock_guard<std::mutex> lk(g_mu);
  if (!g_addr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_scratch);
    if (e != cudaSuccess || !p) {
      dq_internal::set_global_error(std::string("dq_join_agg_noalloc: cudaGetSymbolAddress failed: ") +
                                    cudaGetErrorString(e));
      return DQ_ERR_CUDA;
    }
    g_addr[dev] = static_cast<Scratch*>(p);
  }
  *out = g_addr[dev];
  return DQ_OK;
}

}  // namespace

extern "C" int dq_join_agg_noalloc(const dq_join_agg_args* a, void* stream) {
  if (!a || !a->build_key || !a->build_filter || !a->build_group || !a->out_group || !a->out_sum ||
      !a->out_count || !a->out_ngroups || (a->probe_rows > 0 && (!a->probe_key || !a->probe_value))) {
    dq_internal::set_global_error("dq_join_agg_noalloc: null argument");
    return DQ_ERR_INVALID;
  }
  if (a->build_rows < 0 || a->probe_rows < 0) {
    dq_internal::set_global_error("dq_join_agg_noalloc: negative row count");
    return DQ_ERR_INVALID;
  }
  if (a->build_rows > DQ_NOALLOC_MAX_BUILD_ROWS) {
    dq_internal::set_global_error("dq_join_agg_noalloc: build_rows " + std::to_string(a->build_rows) +
                                  " exceeds the fixed maximum of " +
                                  std::to_string(DQ_NOALLOC_MAX_BUILD_ROWS) + " rows");
    return DQ_ERR_INVALID;
  }
  if (a->max_groups <= 0 || a->max_groups > DQ_NOALLOC_MAX_GROUPS) {
    dq_internal::set_global_error("dq_join_agg_noalloc: max_groups must be in [1, " +
                                  std::to_string(DQ_NOALLOC_MAX_GROUPS) + "]");
    return DQ_ERR_INVALID;
  }
  Scratch* s = nullptr;
  int st = scratch_on_device(&s);
  if (st != DQ_OK) return st;
  cudaStream_t cs = static_cast<cudaStream_t>(stream);
  // Each launch's own status comes back from cudaLaunchKernel, so an error left
  // pending by the caller's earlier runtime calls is neither reported as ours
  // nor cleared.
  const char* failed = nullptr;
  cudaError_t e = cudaSuccess;
  auto launch = [&](const void* fn, int grid, void** args, const char* what) {
    if (failed) return;
    e = cudaLaunchKernel(fn, dim3(grid), dim3(kThreads), args, 0, cs);
    if (e != cudaSuccess) failed = what;
  };
  {
    void* args[] = {&s};
    launch((const void*)clear_kernel, 512, args, "clear");
  }
  if (a->build_rows > 0) {
    const int64_t blocks = (a->build_rows + kThreads - 1) / kThreads;
    const int32_t* bk = a->build_key;
    const int32_t* bf = a->build_filter;
    int32_t fv = a->filter_value;
    const int32_t* bg = a->build_group;
    int64_t bn = a->build_rows;
    void* args[] = {&s, &bk, &bf, &fv, &bg, &bn};
    launch((const void*)build_kernel, (int)(blocks < 2048 ? blocks : 2048), args, "build");
  }
  if (a->probe_rows > 0) {
    const int64_t blocks = (a->probe_rows + kThreads - 1) / kThreads;
    const int32_t* pk = a->probe_key;
    const uint64_t* pv = a->probe_value;
    int64_t pn = a->probe_rows;
    void* args[] = {&s, &pk, &pv, &pn};
    launch((const void*)probe_kernel, (int)(blocks < 4096 ? blocks : 4096), args, "probe");
  }
  {
    int32_t* og = a->out_group;
    uint64_t* os = a->out_sum;
    int32_t* oc = a->out_count;
    int32_t mg = a->max_groups;
    void* args[] = {&s, &og, &os, &oc, &mg};
    launch((const void*)output_kernel, (kGroupSlots + kThreads - 1) / kThreads, args, "output");
  }
  {
    const Scratch* cs_ = s;
    int64_t* on = a->out_ngroups;
    int32_t mg = a->max_groups;
    void* args[] = {&cs_, &on, &mg};
    if (!failed) {
      e = cudaLaunchKernel((const void*)finish_kernel, dim3(1), dim3(1), args, 0, cs);
      if (e != cudaSuccess) failed = "finish";
    }
  }
  if (failed) {
    dq_internal::set_global_error(std::string("dq_join_agg_noalloc: ") + failed + " kernel launch failed: " +
                                  cudaGetErrorString(e));
    return DQ_ERR_CUDA;
  }
  return DQ_OK;
}
