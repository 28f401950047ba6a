// Internal helpers shared by the host and CUDA translation units.
#pragma once
#include <stdint.h>
#include <stdarg.h>
#include <vector>
#include <atomic>
#include <nvtx3/nvToolsExt.h>
#include "../../include/enterprise_b200.h"

namespace ent {

// NVTX range over a host entry point, so a timeline profiler shows which
// call issued which kernels (header-only NVTX v3: a no-op without a tool).
struct NvtxRange {
  explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
  ~NvtxRange() { nvtxRangePop(); }
  NvtxRange(const NvtxRange&) = delete;
  NvtxRange& operator=(const NvtxRange&) = delete;
};

// Records a thread-local error message and returns `code` so call sites can
// write `return fail(ENT_ERR_IO, "...")`.
int fail(int code, const char* fmt, ...) __attribute__((format(printf, 2, 3)));
void clear_error();

// Kernels launched by this library (host-side count, includes the kernels a
// device-driven level loop runs, reported back by the loop).
extern std::atomic<int64_t> g_kernel_launches;

}  // namespace ent

// Host-resident CSR. Offsets are int64 (E may exceed 2^31); ids int32.
struct ent_csr {
  int64_t V = 0;
  int64_t E = 0;
  std::vector<int64_t> off;  // V+1
  std::vector<int32_t> adj;  // E
};
