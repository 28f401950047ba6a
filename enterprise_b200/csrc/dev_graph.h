// Device-resident graph handle and the traversal workspaces hanging off it.
#pragma once
#include <cuda_runtime.h>
#include <mutex>
#include <stdint.h>
#include "ent_internal.h"

namespace ent {
struct BfsWorkspace;    // single-source direction-optimising traversal
struct BatchWorkspace;  // bitwise multi-source traversal
struct DeepLanes;       // concurrent single-source traversals of a batch on a deep graph
void destroy_bfs_workspace(BfsWorkspace* w);
void destroy_batch_workspace(BatchWorkspace* w);
void destroy_deep_lanes(DeepLanes* l);
}  // namespace ent

// Device memory layout of one graph (all on `device`):
//   off  int64[V+1]   row offsets (reference strt_pos + adj_card, allocator.cuh:107-114)
//   adj  int32[E]     column ids, rows ascending (reference adj_list, allocator.cuh:116-120)
//   deg  int32[V]     degrees, read by the classifier (reference adj_card)
//   active uint32[V/32] bit v set iff deg(v) > 0 (bottom-up skips isolated vertices)
//   trav int32[E]     the rows of adj re-ordered by descending neighbour degree
//                     (ties by id): the traversal's adjacency. A bottom-up check
//                     then meets the likeliest parent, a hub, first. Equal to
//                     adj when E >= 2^31 (no re-ordering).
//   lead int4[V]      first 4 entries of each trav row (the highest-degree
//                     neighbours), -1 past the row's end: a bottom-up sweep
//                     reads them coalesced instead of a random row sector per
//                     vertex, and most light vertices need nothing else.
struct ent_graph {
  int device = 0;
  int num_sms = 0;
  int64_t V = 0, E = 0;
  int64_t* off = nullptr;
  int32_t* adj = nullptr;
  int32_t* deg = nullptr;
  uint32_t* active = nullptr;
  int32_t* trav = nullptr;
  int4* lead = nullptr;
  cudaStream_t stream = nullptr;
  ent_bfs_opts opts;
  std::mutex mu;
  ent::BfsWorkspace* ws = nullptr;
  ent::BatchWorkspace* bws = nullptr;
  ent::DeepLanes* lanes = nullptr;
  int32_t probe_levels = -1;  // depth of the graph as probed by its first auto-mode batch (-1: not yet)
  void* stage = nullptr;      // device rows of batches whose results go to host memory
  size_t stage_cap = 0;
};

namespace ent {

// RAII device guard: switches to `dev`, restores the previous device.
struct DeviceGuard {
  int prev = -1;
  explicit DeviceGuard(int dev) {
    cudaGetDevice(&prev);
    if (prev != dev) cudaSetDevice(dev);
  }
  ~DeviceGuard() {
    int cur;
    cudaGetDevice(&cur);
    if (prev >= 0 && cur != prev) cudaSetDevice(prev);
  }
};

#define ENT_CUDA(call)                                                                      \
  do {                                                                                      \
    cudaError_t _e = (call);                                                                \
    if (_e != cudaSuccess)                                                                  \
      return ::ent::fail(_e == cudaErrorMemoryAllocation ? ENT_ERR_OOM : ENT_ERR_CUDA,      \
                         "%s failed: %s (%s:%d)", #call, cudaGetErrorString(_e), __FILE__, \
                         __LINE__);                                                         \
  } while (0)

int graph_alloc(ent_graph* g, int64_t V, int64_t E);
int graph_finish(ent_graph* g);  // computes deg, creates stream
int run_bfs_single(ent_graph* g, int32_t src, int32_t* depth_dev, int32_t* parent_dev, cudaStream_t stream,
                   ent_stats* stats);
int run_bfs_batch(ent_graph* g, const int32_t* src, int32_t n_src, int32_t* depth_dev, cudaStream_t stream,
                  ent_stats* stats, bool bytes = false);
// Depth (levels) of g seen from the given candidate sources: single-source
// traversals from up to three of them (the deepest answer wins; a source that
// reaches a quarter of the graph ends the search). Synchronous, on g->stream;
// the caller holds g->mu.
int probe_graph_levels(ent_graph* g, const int32_t* src, int32_t n_src, int32_t* levels);
// A batch on a deep graph as concurrent single-source traversals, one per
// lane; rows as run_bfs_batch writes them (int32, or bytes with 255 for
// unreached). Ordered after and before `stream` like a launch on it; stats
// (n_src entries) synchronise. The caller holds g->mu.
int run_bfs_deep(ent_graph* g, const int32_t* src, int32_t n_src, void* depth_dev, bool bytes, cudaStream_t stream,
                 ent_stats* stats);

}  // namespace ent
