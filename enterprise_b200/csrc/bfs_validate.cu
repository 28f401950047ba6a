// Graph500-style validation of a traversal's result on the GPU.
//
// The reference checks one random vertex per source on the host (validate(),
// validate.h:34-103: its depth is one more than some neighbour's and no
// neighbour is two levels shallower). This file checks every vertex and edge
// with two certificates, rule for rule the ones the CPU oracle states:
//  * depth certificate (codes as oracle_check_depths):
//      -1 depth[src] != 0;  for each vertex v in ascending order:
//      -2 depth[v] < -1;  -3 depth[v] == 0 and v != src;  then its row in CSR
//      order, at the first edge (v, u) that breaks a rule: -4 exactly one of
//      v, u reached, -5 both reached with depths more than one apart; then
//      -6 a reached v > 0 deep with no neighbour one level up;
//  * parent certificate (codes as oracle_check_parents):
//      -1 parent[src] != src or depth[src] != 0; for each v != src in
//      ascending order: -2 unreached v with a parent, -3 parent out of range,
//      -4 depth[parent] != depth[v] - 1, -5 (parent, v) is not an edge.
// Every vertex's first broken rule is computed independently; the smallest
// such vertex wins (atomicMin on vertex << 8 | rule), so the answer is the
// oracle's (rule, vertex) exactly, whatever the launch order.
#include <cub/cub.cuh>

#include "dev_common.cuh"
#include "dev_graph.h"

namespace ent {
namespace {

constexpr int VT = 256;

__device__ __forceinline__ void report(unsigned long long* slot, int64_t v, int code) {
  atomicMin(slot, ((unsigned long long)v << 8) | (unsigned)(-code));
}

// One warp per vertex; lanes walk the row 32 edges at a time in CSR order.
__global__ void __launch_bounds__(VT) k_val_depth(const int64_t* __restrict__ off, const int32_t* __restrict__ adj,
                                                  int64_t V, int32_t src, const int32_t* __restrict__ depth,
                                                  unsigned long long* slot) {
  const int lane = threadIdx.x & 31;
  const int64_t gw = (blockIdx.x * (int64_t)VT + threadIdx.x) >> 5, nw = ((int64_t)gridDim.x * VT) >> 5;
  for (int64_t v = gw; v < V; v += nw) {
    const int dv = depth[v];
    int code = 0;
    if (dv < -1) code = -2;
    else if (dv == 0 && v != src) code = -3;
    if (!code) {
      const int64_t b = off[v], e = off[v + 1];
      bool has_parent = false;
      for (int64_t k0 = b; k0 < e && !code; k0 += 32) {
        const int64_t k = k0 + lane;
        int c = 0;
        if (k < e) {
          const int du = depth[adj[k]];
          if ((du == -1) != (dv == -1)) c = -4;
          else if (dv != -1 && (du > dv + 1 || du < dv - 1)) c = -5;
          if (dv > 0 && du == dv - 1) has_parent = true;
        }
        const unsigned bad = __ballot_sync(FULL, c != 0);
        if (bad) code = __shfl_sync(FULL, c, __ffs(bad) - 1);  // the first broken edge in row order
      }
      has_parent = __any_sync(FULL, has_parent);
      if (!code && dv > 0 && !has_parent) code = -6;
    }
    if (code && lane == 0) report(slot, v, code);
  }
}

__device__ __forceinline__ bool row_has(const int64_t* off, const int32_t* rows, int32_t p, int32_t v) {
  int64_t lo = off[p], hi = off[p + 1];  // rows sorted ascending
  while (lo < hi) {
    const int64_t mid = (lo + hi) >> 1;
    const int32_t x = rows[mid];
    if (x == v) return true;
    if (x < v) lo = mid + 1;
    else hi = mid;
  }
  return false;
}

__global__ void __launch_bounds__(VT) k_val_parent(const int64_t* __restrict__ off,
                                                   const int32_t* __restrict__ rows_sorted, int64_t V, int32_t src,
                                                   const int32_t* __restrict__ depth,
                                                   const int32_t* __restrict__ parent, unsigned long long* slot) {
  for (int64_t v = blockIdx.x * (int64_t)VT + threadIdx.x; v < V; v += (int64_t)gridDim.x * VT) {
    if (v == src) continue;
    const int dv = depth[v], p = parent[v];
    int code = 0;
    if (dv == -1) {
      if (p != -1) code = -2;
    } else if (p < 0 || p >= V) {
      code = -3;
    } else if (depth[p] != dv - 1) {
      code = -4;
    } else if (!row_has(off, rows_sorted, p, (int32_t)v)) {
      code = -5;
    }
    if (code) report(slot, v, code);
  }
}

__global__ void k_rows_unsorted(const int64_t* __restrict__ off, const int32_t* __restrict__ adj, int64_t V,
                                unsigned long long* n_bad) {
  for (int64_t v = blockIdx.x * (int64_t)VT + threadIdx.x; v < V; v += (int64_t)gridDim.x * VT)
    for (int64_t k = off[v] + 1; k < off[v + 1]; ++k)
      if (adj[k - 1] > adj[k]) {
        atomicAdd(n_bad, 1ull);
        break;
      }
}

__global__ void k_val_src(int32_t src, const int32_t* depth, const int32_t* parent, unsigned long long* slots) {
  if (blockIdx.x || threadIdx.x) return;
  if (depth[src] != 0) slots[0] = ((unsigned long long)src << 8) | 1u;
  if (parent && (parent[src] != src || depth[src] != 0)) slots[1] = ((unsigned long long)src << 8) | 1u;
}

void decode(unsigned long long key, int32_t* code, int64_t* bad) {
  if (key == ~0ull) {
    *code = 0;
    *bad = -1;
  } else {
    *code = -(int32_t)(key & 0xff);
    *bad = (int64_t)(key >> 8);
  }
}

}  // namespace
}  // namespace ent

using namespace ent;

extern "C" int ent_validate(ent_graph* g, int32_t src, const int32_t* depth_dev, const int32_t* parent_dev,
                            int32_t* depth_code, int64_t* depth_bad, int32_t* parent_code, int64_t* parent_bad) {
  ent::NvtxRange nvtx_range("ent_validate");
  clear_error();
  if (!g || !depth_dev || !depth_code || !depth_bad) return fail(ENT_ERR_INVALID_ARG, "null argument");
  if (parent_dev && (!parent_code || !parent_bad)) return fail(ENT_ERR_INVALID_ARG, "null parent result");
  if (src < 0 || src >= g->V) return fail(ENT_ERR_INVALID_ARG, "source %d out of range", src);
  std::lock_guard<std::mutex> lk(g->mu);
  DeviceGuard dg(g->device);
  cudaStream_t s = g->stream;
  const int64_t V = g->V, E = g->E;
  unsigned long long* slots = nullptr;  // [0] depth certificate, [1] parent certificate, [2] unsorted rows
  int32_t* sorted = nullptr;
  void* tmp = nullptr;
  int rc = ENT_OK;
  unsigned long long h[3] = {~0ull, ~0ull, 0ull};
  const int grid = g->num_sms * 8;
  cudaError_t e = cudaMallocAsync(&slots, sizeof(h), s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(slots, h, sizeof(h), cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) {
    k_val_depth<<<grid, VT, 0, s>>>(g->off, g->adj, V, src, depth_dev, slots);
    g_kernel_launches++;
    e = cudaGetLastError();
  }
  const int32_t* rows = g->adj;
  if (e == cudaSuccess && parent_dev) {
    // binary search needs sorted rows: check, and sort a copy if a caller's
    // CSR came with unsorted rows
    k_rows_unsorted<<<grid, VT, 0, s>>>(g->off, g->adj, V, slots + 2);
    g_kernel_launches++;
    e = cudaMemcpyAsync(h + 2, slots + 2, sizeof(unsigned long long), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e == cudaSuccess && h[2] != 0) {
      if (E > 0x7fffffffll) {
        rc = fail(ENT_ERR_UNSUPPORTED, "parent validation of unsorted rows needs E < 2^31");
      } else {
        size_t tmp_bytes = 0;
        e = cudaMallocAsync(&sorted, sizeof(int32_t) * E, s);
        if (e == cudaSuccess)
          e = cub::DeviceSegmentedSort::SortKeys(nullptr, tmp_bytes, g->adj, sorted, (int)E, (int)V, g->off,
                                                 g->off + 1, s);
        if (e == cudaSuccess) e = cudaMallocAsync(&tmp, tmp_bytes, s);
        if (e == cudaSuccess)
          e = cub::DeviceSegmentedSort::SortKeys(tmp, tmp_bytes, g->adj, sorted, (int)E, (int)V, g->off,
                                                 g->off + 1, s);
        rows = sorted;
      }
    }
    if (e == cudaSuccess && rc == ENT_OK) {
      k_val_parent<<<grid, VT, 0, s>>>(g->off, rows, V, src, depth_dev, parent_dev, slots + 1);
      g_kernel_launches++;
      e = cudaGetLastError();
    }
  }
  if (e == cudaSuccess && rc == ENT_OK) {
    k_val_src<<<1, 32, 0, s>>>(src, depth_dev, parent_dev, slots);
    g_kernel_launches++;
    e = cudaGetLastError();
  }
  if (e == cudaSuccess && rc == ENT_OK) e = cudaMemcpyAsync(h, slots, sizeof(h), cudaMemcpyDeviceToHost, s);
  if (slots) cudaFreeAsync(slots, s);
  if (sorted) cudaFreeAsync(sorted, s);
  if (tmp) cudaFreeAsync(tmp, s);
  cudaError_t e2 = cudaStreamSynchronize(s);
  if (rc != ENT_OK) return rc;
  if (e != cudaSuccess || e2 != cudaSuccess)
    return fail(ENT_ERR_CUDA, "validation failed: %s", cudaGetErrorString(e != cudaSuccess ? e : e2));
  // the parent certificate's key for the src rule sits in slot 1 with the
  // others; slot 0 likewise for the depth certificate (src is checked first
  // by the oracle: the src rule wins over any vertex)
  decode(h[0], depth_code, depth_bad);
  if (parent_dev) decode(h[1], parent_code, parent_bad);
  return ENT_OK;
}
