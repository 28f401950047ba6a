/*
 * bfs_gpu_opt.cuh — source-compatible replacement for the reference's entry
 * point header (bfs_gpu_opt.cuh:293-447).
 *
 * Keeps
 *     template<typename vertex_t, typename index_t>
 *     int bfs_gpu_coalescing_mem(vertex_t* src_list, index_t* beg_pos,
 *                                vertex_t* csr, index_t vert_count,
 *                                index_t edge_count, index_t gpu_id);
 * with the same meaning: upload the CSR to GPU gpu_id, run one BFS from each
 * of the first 64 entries of src_list and print the reference's per-source
 * block and "Final Average TEPS (Billion)" line (bfs_gpu_opt.cuh:372-445).
 * The body forwards to the C ABI in enterprise_b200.h. Differences, by design:
 *  - errors return non-zero instead of exit() (reference comm.h:34-45);
 *  - the validation line reports the real outcome of a complete depth
 *    certificate computed on the GPU over every vertex and edge (ent_validate;
 *    the reference spot-checks one random vertex, validate.h:34-103, and
 *    prints CORRECT on both branches, bfs_gpu_opt.cuh:424-426);
 *  - time is the traversal's CUDA-event time (the reference used gettimeofday
 *    around a host-driven loop, bfs_gpu_opt.cuh:381-411).
 * Plain C++: include it from a .cpp or .cu file and link libenterprise_b200.
 */
#ifndef ENTERPRISE_B200_BFS_GPU_OPT_CUH
#define ENTERPRISE_B200_BFS_GPU_OPT_CUH

#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <vector>
#include "enterprise_b200.h"

namespace ent_compat {

struct RunOptions {
  int n_sources = 64;          /* the reference hard-codes 64 (bfs_gpu_opt.cuh:370) */
  const ent_bfs_opts* opts = nullptr;
  FILE* json = nullptr;        /* optional machine-readable per-source lines */
  int batch = 0;               /* > 0: run the sources as bitwise batches of up to this many
                                  (ent_bfs_batch, one launch per batch); each source's time
                                  line shows its batch's time divided by the batch's sources */
  int64_t cpu_bytes = 0;       /* host bytes the caller holds for the graph, printed as the
                                  reference's "CPU alloc space" line (allocator.cuh:150) */
};

/* The reference's per-source output block (bfs_gpu_opt.cuh:372-431) and its
 * closing lines, shared by both runners. `check` is called only for sources
 * whose traversal has more than 2 levels, as the reference validates only
 * those; it returns 0 when the depths pass, else the broken rule. */
struct Report {
  const RunOptions& ro;
  double average_teps = 0.0, inv_sum = 0.0;
  int64_t validate_count = 0;
  int failures = 0;
  explicit Report(const RunOptions& r) : ro(r) {}
  template <class Check>
  void source(int i, int32_t src, const ent_stats& st, double tm, Check check) {
    printf("Test %d\n", i + 1);
    printf("Started from: %d\n", src);
    if (st.levels > 2) {
      ++validate_count;
      const int ret = check();
      if (ret != 0) ++failures;
      printf("\nBFS result validation: %s\n", ret == 0 ? "CORRECT" : "WRONG");
      const double curr_teps = (double)st.traversed_edges / (1e9 * tm);
      average_teps = (curr_teps + average_teps * (validate_count - 1)) / validate_count;
      inv_sum += 1.0 / curr_teps;
      printf("Traversed vertices: %lld\t\t\tTraversed edges: %lld\n", (long long)st.reached_vertices,
             (long long)st.traversed_edges);
      printf("Traversed time(s) :%g\t\tCurrent TEPS (Billion): %g\n", tm, curr_teps);
      printf("Average TEPS (Billion): %g\n", average_teps);
      if (ro.json)
        fprintf(ro.json,
                "{\"source\": %d, \"levels\": %d, \"td_levels\": %d, \"bu_levels\": %d, \"reached\": %lld, "
                "\"edges\": %lld, \"ms\": %.6f, \"gteps\": %.6f, \"check\": %d, \"batched\": %s}\n",
                src, st.levels, st.td_levels, st.bu_levels, (long long)st.reached_vertices,
                (long long)st.traversed_edges, tm * 1e3, curr_teps, ret, ro.batch > 0 ? "true" : "false");
    } else {
      printf("Traverse depth is %d\n", st.levels);
    }
    printf("\n====================================\n");
  }
  int finish() {
    printf("Final Average TEPS (Billion): %g\n", average_teps);
    if (validate_count) printf("Harmonic Mean TEPS (Billion): %g\n", validate_count / inv_sum);
    return failures ? 2 : 0;
  }
};

/* Host CSR in hand (the reference's setting): upload it, then run as
 * run_loaded does. */
inline int run_loaded(ent_graph* g, const int32_t* src_list, const RunOptions& ro);
inline int run(const int32_t* src_list, const int64_t* beg_pos, const int32_t* csr, int64_t vert_count,
               int64_t edge_count, int gpu_id, const RunOptions& ro) {
  ent_graph* g = nullptr;
  if (ent_graph_create(beg_pos, csr, vert_count, edge_count, gpu_id, &g) != ENT_OK) {
    printf("Graph upload failed: %s\n", ent_last_error());
    return 1;
  }
  const int rc = run_loaded(g, src_list, ro);
  ent_graph_destroy(g);
  return rc;
}

/* Graph already on the GPU (ent_graph_load): traverse into device buffers
 * and validate every result completely on the GPU (ent_validate: the depth
 * certificate over every vertex and edge), so no host copy of the CSR or of
 * the depths is needed. The caller keeps ownership of g. */
inline int run_loaded(ent_graph* g, const int32_t* src_list, const RunOptions& ro) {
  if (ro.opts && ent_graph_set_opts(g, ro.opts) != ENT_OK) {
    printf("Bad options: %s\n", ent_last_error());
    return 1;
  }
  const int64_t V = ent_graph_vert_count(g);
  const int width = ro.batch > 0 ? ro.batch : 1;
  void* buf = nullptr;
  if (ent_device_alloc(ent_graph_device(g), sizeof(int32_t) * (size_t)V * (size_t)width, &buf) != ENT_OK) {
    printf("Device buffer failed: %s\n", ent_last_error());
    return 1;
  }
  int32_t* rows = static_cast<int32_t*>(buf);
  /* the reference's allocation lines (allocator.cuh:149-150), then its banner */
  printf("GPU alloc space: %lld bytes\n",
         (long long)(ent_graph_device_bytes(g) + (int64_t)sizeof(int32_t) * V * width));
  printf("CPU alloc space: %lld bytes\n", (long long)ro.cpu_bytes);
  printf("In gpu bfs\n");
  Report rep(ro);
  int rc = 0;
  const auto certify = [&](int32_t src, const int32_t* depth_dev) {
    int32_t dc = 0, pc = 0;
    int64_t db = -1, pb = -1;
    if (ent_validate(g, src, depth_dev, nullptr, &dc, &db, &pc, &pb) != ENT_OK) return -100;
    return (int)dc;
  };
  for (int first = 0; first < ro.n_sources && rc == 0; first += width) {
    const int k = ro.n_sources - first < width ? ro.n_sources - first : width;
    std::vector<ent_stats> st((size_t)k);
    const int e = ro.batch > 0 ? ent_bfs_batch_device(g, src_list + first, k, rows, nullptr, st.data())
                               : ent_bfs_device(g, src_list[first], rows, nullptr, nullptr, st.data());
    if (e != ENT_OK) {
      printf("BFS failed: %s\n", ent_last_error());
      rc = 1;
      break;
    }
    const double tm = st[0].device_ms * 1e-3 / k;
    for (int j = 0; j < k; ++j) {
      const int32_t* row = rows + (size_t)j * (size_t)V;
      rep.source(first + j, src_list[first + j], st[j], tm, [&] { return certify(src_list[first + j], row); });
    }
  }
  ent_device_free(buf);
  return rc ? rc : rep.finish();
}

}  // namespace ent_compat

template <typename vertex_t, typename index_t>
int bfs_gpu_coalescing_mem(vertex_t* src_list, index_t* beg_pos, vertex_t* csr, index_t vert_count,
                           index_t edge_count, index_t gpu_id) {
  std::vector<int64_t> off((size_t)vert_count + 1);
  for (int64_t i = 0; i <= (int64_t)vert_count; ++i) off[i] = (int64_t)beg_pos[i];
  std::vector<int32_t> adj((size_t)edge_count);
  for (int64_t i = 0; i < (int64_t)edge_count; ++i) adj[i] = (int32_t)csr[i];
  std::vector<int32_t> src(64);
  for (int i = 0; i < 64; ++i) src[i] = (int32_t)src_list[i];
  ent_compat::RunOptions ro;
  ro.cpu_bytes = (int64_t)(sizeof(int64_t) * off.size() + sizeof(int32_t) * adj.size() + sizeof(int32_t) * src.size());
  return ent_compat::run(src.data(), off.data(), adj.data(), (int64_t)vert_count, (int64_t)edge_count,
                         (int)gpu_id, ro);
}

#endif
