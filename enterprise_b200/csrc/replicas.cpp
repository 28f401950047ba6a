// Source sharding over replicas of one graph on several GPUs of a node.
//
// No reference counterpart: the reference drives one GPU (bfs_gpu_opt.cuh:305
// cudaSetDevice(gpu_id), main.cu:49 gpu_id = 0). Sources are independent, so
// a many-source request spreads over replicas of the graph with no exchange on
// the data path: the source list is cut into contiguous chunks of at most
// max_batch sources (ent_replicas_plan), one host thread per replica takes the
// next unclaimed chunk, runs it as one bitwise batch on its own GPU and copies
// the chunk's depth rows into the caller's buffer at the chunk's own rows, so
// the result is in input order whichever replica ran which chunk. Every kernel
// reads only its own GPU's replica; no peer memory is touched.
#include <algorithm>
#include <atomic>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "dev_graph.h"

struct ent_replicas {
  std::vector<ent_graph*> graphs;  // borrowed, one per replica
  int32_t max_batch = 1024;
  std::vector<int64_t> ran;        // sources each replica ran in the last call
};

namespace {

// Contiguous chunks of at most max_batch sources, and at least one per replica
// while there are sources to give: chunk = min(max_batch, ceil(n / replicas)).
int32_t plan_chunk(int32_t n_src, int32_t n_rep, int32_t max_batch) {
  const int32_t even = (n_src + n_rep - 1) / n_rep;
  return std::max<int32_t>(1, std::min<int32_t>(max_batch, even));
}

int run_chunks(ent_replicas* r, const int32_t* src, int32_t n_src, void* depth_out, bool bytes, ent_stats* stats) {
  const int32_t n_rep = (int32_t)r->graphs.size();
  const int32_t chunk = plan_chunk(n_src, n_rep, r->max_batch);
  const int32_t n_chunks = (n_src + chunk - 1) / chunk;
  const int64_t V = r->graphs[0]->V;
  const size_t row_bytes = (bytes ? 1 : sizeof(int32_t)) * (size_t)V;
  std::atomic<int32_t> next{0};
  std::mutex mu;
  int first_rc = ENT_OK;
  std::string first_msg;
  std::vector<int64_t> ran(n_rep, 0);
  auto worker = [&](int k) {
    ent_graph* g = r->graphs[k];
    for (;;) {
      {
        std::lock_guard<std::mutex> lk(mu);
        if (first_rc != ENT_OK) return;  // stop handing out work after a failure
      }
      const int32_t c = next.fetch_add(1);
      if (c >= n_chunks) return;
      const int32_t b = c * chunk, n = std::min<int32_t>(chunk, n_src - b);
      char* out = depth_out ? static_cast<char*>(depth_out) + (size_t)b * row_bytes : nullptr;
      ent_stats* st = stats ? stats + b : nullptr;
      const int rc = bytes ? ent_bfs_batch_u8(g, src + b, n, reinterpret_cast<uint8_t*>(out), st)
                           : ent_bfs_batch(g, src + b, n, reinterpret_cast<int32_t*>(out), st);
      if (rc != ENT_OK) {
        std::lock_guard<std::mutex> lk(mu);
        if (first_rc == ENT_OK) {
          first_rc = rc;
          first_msg = ent_last_error();
        }
        return;
      }
      ran[k] += n;
    }
  };
  std::vector<std::thread> th;
  for (int k = 1; k < n_rep; ++k) th.emplace_back(worker, k);
  worker(0);
  for (std::thread& t : th) t.join();
  r->ran = ran;
  if (first_rc != ENT_OK) return ent::fail(first_rc, "%s", first_msg.c_str());
  return ENT_OK;
}

}  // namespace

extern "C" {

int ent_replicas_plan(int32_t n_src, int32_t n_replicas, int32_t max_batch, int32_t* chunk_begin,
                      int32_t* n_chunks) {
  ent::clear_error();
  if (n_src < 0 || n_replicas < 1 || max_batch < 1 || !n_chunks)
    return ent::fail(ENT_ERR_INVALID_ARG, "bad arguments");
  const int32_t chunk = plan_chunk(n_src, n_replicas, max_batch);
  const int32_t n = (n_src + chunk - 1) / chunk;
  if (chunk_begin)
    for (int32_t c = 0; c <= n; ++c) chunk_begin[c] = std::min<int32_t>(c * chunk, n_src);
  *n_chunks = n;
  return ENT_OK;
}

int ent_replicas_create(ent_graph* const* graphs, int32_t n_replicas, ent_replicas** out) {
  ent::NvtxRange nvtx_range("ent_replicas_create");
  ent::clear_error();
  if (!graphs || n_replicas < 1 || !out) return ent::fail(ENT_ERR_INVALID_ARG, "bad arguments");
  *out = nullptr;
  for (int32_t k = 0; k < n_replicas; ++k) {
    if (!graphs[k]) return ent::fail(ENT_ERR_INVALID_ARG, "replica %d is null", k);
    if (graphs[k]->V != graphs[0]->V || graphs[k]->E != graphs[0]->E)
      return ent::fail(ENT_ERR_INVALID_ARG, "replica %d is not the same graph (V or E differ)", k);
    for (int32_t j = 0; j < k; ++j)
      if (graphs[j] == graphs[k]) return ent::fail(ENT_ERR_INVALID_ARG, "replica %d listed twice", k);
  }
  ent_replicas* r = new ent_replicas();
  r->graphs.assign(graphs, graphs + n_replicas);
  r->ran.assign(n_replicas, 0);
  *out = r;
  return ENT_OK;
}

int ent_replicas_set_max_batch(ent_replicas* r, int32_t max_batch) {
  ent::clear_error();
  if (!r || max_batch < 1 || max_batch > 2048) return ent::fail(ENT_ERR_INVALID_ARG, "max_batch must be 1..2048");
  r->max_batch = max_batch;
  return ENT_OK;
}

int ent_replicas_bfs_batch(ent_replicas* r, const int32_t* src, int32_t n_src, int32_t* depth_out,
                           ent_stats* stats) {
  ent::NvtxRange nvtx_range("ent_replicas_bfs_batch");
  ent::clear_error();
  if (!r || !src || n_src < 1) return ent::fail(ENT_ERR_INVALID_ARG, "bad arguments");
  for (int32_t i = 0; i < n_src; ++i)
    if (src[i] < 0 || src[i] >= r->graphs[0]->V) return ent::fail(ENT_ERR_INVALID_ARG, "source %d out of range", src[i]);
  return run_chunks(r, src, n_src, depth_out, false, stats);
}

int ent_replicas_bfs_batch_u8(ent_replicas* r, const int32_t* src, int32_t n_src, uint8_t* depth_out,
                              ent_stats* stats) {
  ent::NvtxRange nvtx_range("ent_replicas_bfs_batch_u8");
  ent::clear_error();
  if (!r || !src || n_src < 1) return ent::fail(ENT_ERR_INVALID_ARG, "bad arguments");
  for (int32_t i = 0; i < n_src; ++i)
    if (src[i] < 0 || src[i] >= r->graphs[0]->V) return ent::fail(ENT_ERR_INVALID_ARG, "source %d out of range", src[i]);
  return run_chunks(r, src, n_src, depth_out, true, stats);
}

int ent_replicas_sources_run(const ent_replicas* r, int64_t* per_replica) {
  ent::clear_error();
  if (!r || !per_replica) return ent::fail(ENT_ERR_INVALID_ARG, "bad arguments");
  for (size_t k = 0; k < r->ran.size(); ++k) per_replica[k] = r->ran[k];
  return ENT_OK;
}

int ent_replicas_destroy(ent_replicas* r) {
  delete r;
  return ENT_OK;
}

}  // extern "C"
