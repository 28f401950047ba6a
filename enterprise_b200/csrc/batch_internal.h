// Internal interface of the traversals used by the serving loop.
#pragma once
#include <cuda_runtime.h>
#include "dev_graph.h"

namespace ent {
// Sources that join a running bitwise batch at its next level boundary. Lives
// in mapped, page-locked host memory: the host fills the entries, then bumps
// seq (release); the batch's level finisher, seeing seq != taken at a level no
// deeper than `limit`, adds the entries to that level's frontier and stores
// taken = seq (release). A post the batch never took (it ended first, or it
// was past the limit) stays with taken != seq. The finisher also publishes the
// level it reached, so the host posts only while a post can still be taken:
// results come back when the whole batch ends, so a source that joins late
// would hold back every result of its batch.
constexpr int JOIN_MAX = 2048;
struct JoinBox {
  int32_t seq;            // written by the host
  int32_t taken;          // written by the device
  int32_t n;              // entries of the post
  int32_t limit;          // deepest level at which the batch takes a post (host)
  int32_t level;          // level the batch has reached (device)
  int32_t pad[3];
  int32_t pos[JOIN_MAX];  // bit position (source slot) in the batch
  int32_t src[JOIN_MAX];  // source vertex
  int32_t row[JOIN_MAX];  // depth row (row_map entry) of the source
};

// Traversal state for one batched run of up to words_for(n_src)*64 sources.
int create_batch_workspace(ent_graph* g, int n_src, BatchWorkspace** out);
// Adds one independent branch (memsets, seed, while{expand, commit,
// if{flush}}, final flush) for workspace w to `graph`.
int append_branch(ent_graph* g, BatchWorkspace* w, cudaGraph_t graph, cudaStream_t cap_stream);
// Uploads sources and output location for the next launch of w's branch.
// With row_map_dev (device, n_src entries) source s writes depth row row_map[s].
// bytes: the rows are uint8 (255 = unreached) instead of int32; depth_dev then
// points at n_src x V bytes.
int stage_request(ent_graph* g, BatchWorkspace* w, const int32_t* src, int32_t n_src, int32_t* depth_dev,
                  cudaStream_t s, const int32_t* row_map_dev, bool bytes = false);
// Gives w's branch a join mailbox (device address of a mapped JoinBox); call
// before append_branch. With one, the batch's n_src may grow while it runs and
// row_map_dev must hold JOIN_MAX entries.
void set_join_box(BatchWorkspace* w, JoinBox* box_dev);
// Sources that joined w's last run (valid after batch_source_stats).
int batch_joined(const BatchWorkspace* w);
int batch_source_stats(BatchWorkspace* w, int32_t n_src, cudaStream_t s, ent_stats* stats);
int batch_max_sources(const BatchWorkspace* w);

// Single-source traversal state with its own instantiated CUDA graph
// (independent of the graph's own workspace, so several run concurrently).
// cluster > 0 sets the CTAs of its small-frontier cluster (else the graph's option).
int create_bfs_workspace(ent_graph* g, BfsWorkspace** out, int32_t cluster = 0);
// Launches one traversal from src writing depth_dev (V int32) on stream s; async.
int launch_bfs_single(BfsWorkspace* w, int32_t src, int32_t* depth_dev, cudaStream_t s);
// Statistics of w's last traversal once it finished (copies on s, synchronises).
int bfs_single_stats(BfsWorkspace* w, cudaStream_t s, ent_stats* stats);
}  // namespace ent
