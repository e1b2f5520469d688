// Per-pipeline kernels generated at plan preparation (host side).
//
// The reference compiles every query: its translator writes one CUDA source per
// query and runs nvcc on it (dogqc/cudaTranslator.py, dogqc/codegen.py,
// dogqc/code.py).  This backend does the same per pipeline of the lowered plan,
// in process: dq_jit.cu turns a pipeline descriptor into straight-line CUDA
// (values in registers, one row per lane, warp-cooperative expansion and
// aggregation), compiles it with NVRTC for sm_100a and loads the cubin with
// the runtime's library API.  Compiled programs are cached by source text, so
// re-preparing a plan or growing its tables does not recompile.
#pragma once
#include <cuda_runtime.h>

#include <stdexcept>
#include <string>

#include "dq_device.h"

namespace dq {
namespace jit {

struct Error : std::runtime_error {
  explicit Error(const std::string& m) : std::runtime_error(m) {}
};

struct Program {
  std::string source;
  int smem_bytes = 0;        // dynamic shared memory of both kernels
  int rows_per_thread = 1;   // rows one thread takes per grid-stride step
  int block = kThreads;      // threads per CTA
  bool heavy = false;        // second kernel for deferred expansion ranges
  bool batched = false;      // one kernel `dq_batch_main` over many instances
};

struct Kernels {
  cudaKernel_t main = nullptr;
  cudaKernel_t heavy = nullptr;
  std::string log;           // compiler log (register and spill report)
};

// Launch-shape choices an autotuner may override (0 / default: the
// generator's own choice).
struct Tuning {
  bool batched = false;      // generate the many-instance kernel
  int rows_per_thread = 0;   // 1, 2 or 4
  int block = 0;             // 128, 256 or 512 threads per CTA
  int refill = 0;            // -1: no lane refill; 0: the plan's refill point
  int refill_threshold = 0;  // buffered rows that make a warp process them (0: 32)
  int min_blocks = 0;        // CTAs per SM the launch bounds ask registers for (0: none)
};

// Source of the kernels for one pipeline.  `P` is the launch descriptor the
// runtime filled (resource layouts, slots with their staged-column indices,
// stash indices); `expand_op` is the expansion whose wide ranges are deferred
// to the second kernel (-1: none); `refill_op` is the selective filter or
// probe after which the warps refill their lanes from a buffer (-1: none).
// With `tail` (the next pipeline: a scan of this pipeline's aggregation table
// with scalar ops and an emit sink), the kernel's last CTA runs that pipeline
// after every CTA has merged its aggregates, and the tail needs no launch.
// `patterns`: the host copy of the bytes P.patterns points to (the LIKE
// patterns and string constants, P.pat_off into them); with it, a LIKE
// pattern of '%'-separated literals compiles into a search for each literal.
Program generate(const DevPipe& P, int expand_op, int refill_op, const Tuning& t = Tuning(),
                 const DevPipe* tail = nullptr, const std::string* patterns = nullptr);

// Compiles the program (cached by source text) and, with `load`, loads it.
Kernels compile(const Program& prog, bool load);

}  // namespace jit
}  // namespace dq
