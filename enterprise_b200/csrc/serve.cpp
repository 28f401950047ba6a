// Serving loop: continuous batching of BFS queries against device-resident
// graphs. No reference counterpart (the reference runs a fixed list of 64
// sources per process, bfs_gpu_opt.cuh:370-432).
//
// Model
//  * Graphs stay resident; each graph has S batch slots. A slot owns a
//    batched-traversal workspace, an instantiated CUDA graph of that
//    traversal, a stream and a completion event.
//  * Per-query state resident in HBM is one depth row (V int32) from a
//    per-graph pool sized by the memory budget. A query is admitted when a
//    row is free; it keeps the row until the client releases it. submit()
//    refuses (ENT_ERR_ADMISSION) once max_pending queries wait.
//  * One scheduler thread loops: it retires finished slots (event query),
//    then for every graph with waiting queries and a free slot it takes up to
//    max_batch of them that have rows, uploads their sources and row map and
//    launches the slot's graph on its stream. Queries that arrive while other
//    batches run join the next batch as soon as a slot and rows free up, and
//    batches of different graphs and slots overlap on the device.
//  * High-diameter graphs are served one source per launch: a probe
//    traversal at creation measures the graph's depth, and a graph at least
//    single_source_levels deep gets single_slots single-source slots instead
//    (each a single-source workspace with its own instantiated CUDA graph,
//    stream and event). A bitwise batch on such a graph would hold every one
//    of its queries for thousands of levels of grid-wide launches; a
//    single-source traversal runs its small frontiers inside one
//    thread-block cluster, so several queries proceed side by side on
//    different SMs and each finishes as soon as its own traversal does.
//  * Every other graph also has fast_slots single-source slots, listed before
//    its batched slots. They take the graph's queries while at most
//    fast_max_waiting wait: one direction-optimising traversal per query ends
//    sooner than a bitwise batch of a few, whose levels each sweep every
//    vertex. When more wait, the batched slots take them.
//  * The single-source slots of deep graphs run their small frontiers in
//    clusters of single_cluster CTAs (8 by default, where a lone traversal
//    would take the largest cluster, 16): with several deep queries in
//    flight, smaller clusters leave SMs to the others and to the batches.
//  * Batched and fast slots run on the highest stream priority and the
//    single-source slots of deep graphs on the lowest, so that the block
//    scheduler hands freed SMs to them before the next cluster of a deep
//    graph's traversal.
//  * Latency = submit to the scheduler observing completion (poll granularity
//    tens of microseconds); queue time = submit to launch.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "batch_internal.h"

using Clock = std::chrono::steady_clock;

namespace {

struct Query {
  int32_t graph = 0;
  int32_t src = 0;
  int32_t row = -1;
  int32_t done = 0;
  Clock::time_point t_submit, t_launch, t_done;
  ent_stats st{};
};

struct Slot {
  ent::BatchWorkspace* ws = nullptr;   // batched slot
  ent::BfsWorkspace* sws = nullptr;    // single-source slot
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  cudaStream_t stream = nullptr;
  cudaEvent_t done = nullptr;
  int32_t* row_map_dev = nullptr;
  std::vector<int64_t> qids;           // the batch's queries, in bit-position order
  bool busy = false;
  bool fast = false;                   // single-source slot of a shallow graph
  // batched slots: queries join the running batch at a level boundary
  ent::JoinBox* box = nullptr;         // mapped host mailbox (device sees box_dev)
  ent::JoinBox* box_dev = nullptr;
  std::vector<int64_t> posted;         // posted, not yet seen taken
  int32_t next_pos = 0;                // next free bit position of the running batch
};

struct GraphState {
  ent_graph* g = nullptr;
  int64_t V = 0;
  int32_t* pool = nullptr;
  int32_t rows = 0;
  std::vector<int32_t> free_rows;
  std::deque<int64_t> pending;
  std::vector<Slot> slots;
  bool single = false;       // served one source per launch
  int32_t probe_levels = 0;  // depth of the probe traversal
};

}  // namespace

struct ent_server {
  ent_server_opts opts{};
  int device = 0;
  std::vector<GraphState> gs;
  std::mutex mu;
  std::condition_variable cv;       // wakes the scheduler
  std::condition_variable cv_done;  // wakes pollers
  std::unordered_map<int64_t, Query> queries;
  std::deque<int64_t> completed;
  std::atomic<bool> stop{false};
  std::thread worker;
  cudaStream_t prep = nullptr;      // fills the rows of joining queries with -1
  int64_t next_id = 1;
  int64_t n_pending = 0;
  ent_server_counters ctr{};
  int worker_error = 0;
  std::string worker_msg;
};

namespace {

using namespace ent;

void free_server(ent_server* s) {
  DeviceGuard dg(s->device);
  for (GraphState& g : s->gs) {
    for (Slot& sl : g.slots) {
      if (sl.stream) cudaStreamSynchronize(sl.stream);
      if (sl.exec) cudaGraphExecDestroy(sl.exec);
      if (sl.graph) cudaGraphDestroy(sl.graph);
      if (sl.ws) destroy_batch_workspace(sl.ws);
      if (sl.sws) destroy_bfs_workspace(sl.sws);
      if (sl.row_map_dev) cudaFree(sl.row_map_dev);
      if (sl.box) cudaFreeHost(sl.box);
      if (sl.done) cudaEventDestroy(sl.done);
      if (sl.stream) cudaStreamDestroy(sl.stream);
    }
    if (g.pool) cudaFree(g.pool);
  }
  if (s->prep) cudaStreamDestroy(s->prep);
  delete s;
}

// Posted joins the batch took move into its query list; host side of the
// mailbox protocol (the device stores taken = seq once it has seeded them).
void confirm_joins(Slot& sl) {
  if (sl.posted.empty()) return;
  if (__atomic_load_n(&sl.box->taken, __ATOMIC_ACQUIRE) != sl.box->seq) return;
  sl.qids.insert(sl.qids.end(), sl.posted.begin(), sl.posted.end());
  sl.posted.clear();
}

// Retires finished slots; returns true if any finished.
bool retire(ent_server* s) {
  bool any = false;
  for (GraphState& g : s->gs) {
    for (Slot& sl : g.slots) {
      if (!sl.busy) continue;
      cudaError_t q = cudaEventQuery(sl.done);
      if (q == cudaErrorNotReady) continue;
      const Clock::time_point now = Clock::now();
      std::vector<int64_t> untaken;  // posted joins the batch ended without
      if (sl.box) {
        confirm_joins(sl);
        untaken.swap(sl.posted);
      }
      std::vector<ent_stats> st(sl.qids.size());
      int rc = q != cudaSuccess ? fail(ENT_ERR_CUDA, "batch failed: %s", cudaGetErrorString(q))
               : sl.sws         ? bfs_single_stats(sl.sws, sl.stream, st.data())
                                : batch_source_stats(sl.ws, (int32_t)sl.qids.size(), sl.stream, st.data());
      std::lock_guard<std::mutex> lk(s->mu);
      if (!sl.sws && rc == ENT_OK && q == cudaSuccess) s->ctr.joined += batch_joined(sl.ws);
      for (auto it = untaken.rbegin(); it != untaken.rend(); ++it) {  // back to the queue's front, in order
        Query& uq = s->queries[*it];
        g.free_rows.push_back(uq.row);
        uq.row = -1;
        g.pending.push_front(*it);
        ++s->n_pending;
        --s->ctr.launched;  // counted again when it launches
      }
      for (size_t i = 0; i < sl.qids.size(); ++i) {
        auto it = s->queries.find(sl.qids[i]);
        if (it == s->queries.end()) continue;
        it->second.st = st[i];
        if (rc != ENT_OK) it->second.st.status = rc;
        it->second.done = 1;
        it->second.t_done = now;
        s->completed.push_back(sl.qids[i]);
      }
      s->ctr.completed += (int64_t)sl.qids.size();
      if ((int64_t)sl.qids.size() > s->ctr.max_batch_seen) s->ctr.max_batch_seen = (int32_t)sl.qids.size();
      if (rc != ENT_OK) {
        s->worker_error = rc;
        s->worker_msg = ent_last_error();
      }
      sl.qids.clear();
      sl.busy = false;
      any = true;
      s->cv_done.notify_all();
    }
  }
  return any;
}

// Launches batches for graphs with waiting queries; returns true if any launched.
bool launch(ent_server* s) {
  bool any = false;
  for (size_t gi = 0; gi < s->gs.size(); ++gi) {
    GraphState& g = s->gs[gi];
    for (Slot& sl : g.slots) {
      if (sl.busy) continue;
      std::vector<int32_t> src, rows;
      {
        std::lock_guard<std::mutex> lk(s->mu);
        if (g.pending.empty() || g.free_rows.empty()) break;
        // a fast slot takes queries only while few wait; else the batched slots do
        if (sl.fast && g.pending.size() > (size_t)s->opts.fast_max_waiting) continue;
        const int cap = sl.sws ? 1 : batch_max_sources(sl.ws);
        const int take = (int)std::min<size_t>({(size_t)s->opts.max_batch, (size_t)cap, g.pending.size(),
                                                g.free_rows.size()});
        const Clock::time_point now = Clock::now();
        for (int i = 0; i < take; ++i) {
          const int64_t qid = g.pending.front();
          g.pending.pop_front();
          --s->n_pending;
          Query& q = s->queries[qid];
          q.row = g.free_rows.back();
          g.free_rows.pop_back();
          q.t_launch = now;
          src.push_back(q.src);
          rows.push_back(q.row);
          sl.qids.push_back(qid);
        }
        s->ctr.batches += 1;
        s->ctr.launched += take;
        if (sl.fast) s->ctr.fast_launches += take;
        if (take > s->ctr.max_batch_seen) s->ctr.max_batch_seen = take;
      }
      const int n = (int)src.size();
      cudaError_t e = cudaSuccess;
      int rc = ENT_OK;
      if (sl.sws) {
        rc = launch_bfs_single(sl.sws, src[0], g.pool + (size_t)rows[0] * g.V, sl.stream);
      } else {
        sl.box->seq = 0;  // the slot is idle: nothing reads the mailbox
        sl.box->taken = 0;
        sl.box->n = 0;
        sl.box->limit = s->opts.join;
        sl.box->level = 0;
        sl.posted.clear();
        sl.next_pos = n;
        e = cudaMemcpyAsync(sl.row_map_dev, rows.data(), sizeof(int32_t) * n, cudaMemcpyHostToDevice, sl.stream);
        rc = e == cudaSuccess ? stage_request(g.g, sl.ws, src.data(), n, g.pool, sl.stream, sl.row_map_dev)
                              : fail(ENT_ERR_CUDA, "row map upload failed");
        if (rc == ENT_OK) e = cudaGraphLaunch(sl.exec, sl.stream);
      }
      if (rc == ENT_OK && e == cudaSuccess) e = cudaEventRecord(sl.done, sl.stream);
      if (rc != ENT_OK || e != cudaSuccess) {
        // the batch never ran: complete its queries with the error status
        std::lock_guard<std::mutex> lk(s->mu);
        s->worker_error = rc != ENT_OK ? rc : ENT_ERR_CUDA;
        s->worker_msg = rc != ENT_OK ? ent_last_error() : cudaGetErrorString(e);
        const Clock::time_point now = Clock::now();
        for (int64_t qid : sl.qids) {
          Query& q = s->queries[qid];
          q.done = 1;
          q.st.status = s->worker_error;
          q.t_done = now;
          s->completed.push_back(qid);
        }
        s->ctr.completed += (int64_t)sl.qids.size();
        sl.qids.clear();
        s->cv_done.notify_all();
        continue;
      }
      sl.busy = true;
      any = true;
    }
  }
  return any;
}

// Queries still waiting join running batches of their graph at the batches'
// next level boundary: into the free bit positions of a busy batched slot
// whose previous post was taken. Their rows are filled with -1 first (a
// window of levels the batch flushed before they joined never writes them).
bool join(ent_server* s) {
  bool any = false;
  for (GraphState& g : s->gs) {
    for (Slot& sl : g.slots) {
      if (!sl.busy || !sl.box) continue;
      confirm_joins(sl);
      if (!sl.posted.empty()) continue;  // one post in flight per batch
      // a post is taken at the next level boundary: only while that is within the limit
      if (__atomic_load_n(&sl.box->level, __ATOMIC_ACQUIRE) >= s->opts.join) continue;
      const int cap = batch_max_sources(sl.ws);
      std::vector<int64_t> qs;
      std::vector<int32_t> rows, srcs;  // copied under the lock: submit() may rehash the query map
      {
        std::lock_guard<std::mutex> lk(s->mu);
        if (g.pending.empty() || g.free_rows.empty() || sl.next_pos >= cap) continue;
        const int take = (int)std::min<size_t>({(size_t)(cap - sl.next_pos), g.pending.size(), g.free_rows.size(),
                                                (size_t)s->opts.max_batch});
        const Clock::time_point now = Clock::now();
        for (int i = 0; i < take; ++i) {
          const int64_t qid = g.pending.front();
          g.pending.pop_front();
          --s->n_pending;
          Query& q = s->queries[qid];
          q.row = g.free_rows.back();
          g.free_rows.pop_back();
          q.t_launch = now;
          qs.push_back(qid);
          rows.push_back(q.row);
          srcs.push_back(q.src);
        }
        s->ctr.launched += take;
      }
      cudaError_t e = cudaSuccess;
      for (size_t i = 0; i < qs.size() && e == cudaSuccess; ++i)
        e = cudaMemsetAsync(g.pool + (size_t)rows[i] * g.V, 0xFF, sizeof(int32_t) * (size_t)g.V, s->prep);
      if (e == cudaSuccess) e = cudaStreamSynchronize(s->prep);
      std::lock_guard<std::mutex> lk(s->mu);
      if (e != cudaSuccess) {  // not posted: back to the queue
        for (auto it = qs.rbegin(); it != qs.rend(); ++it) {
          Query& q = s->queries[*it];
          g.free_rows.push_back(q.row);
          q.row = -1;
          g.pending.push_front(*it);
          ++s->n_pending;
        }
        s->ctr.launched -= (int64_t)qs.size();
        s->worker_error = ENT_ERR_CUDA;
        s->worker_msg = cudaGetErrorString(e);
        continue;
      }
      for (size_t i = 0; i < qs.size(); ++i) {
        sl.box->pos[i] = sl.next_pos + (int32_t)i;
        sl.box->src[i] = srcs[i];
        sl.box->row[i] = rows[i];
      }
      sl.box->n = (int32_t)qs.size();
      __atomic_store_n(&sl.box->seq, sl.box->seq + 1, __ATOMIC_RELEASE);
      sl.next_pos += (int32_t)qs.size();
      sl.posted = qs;
      any = true;
    }
  }
  return any;
}

void scheduler(ent_server* s) {
  cudaSetDevice(s->device);
  while (!s->stop.load()) {
    const bool r = retire(s);
    const bool l = launch(s);
    const bool j = s->opts.join ? join(s) : false;
    if (!r && !l && !j) {
      std::unique_lock<std::mutex> lk(s->mu);
      s->cv.wait_for(lk, std::chrono::microseconds(20));
    }
  }
}

}  // namespace

extern "C" {

void ent_server_opts_default(ent_server_opts* o) {
  if (!o) return;
  o->max_batch = 64;
  o->slots_per_graph = 2;
  o->rows_per_graph = 0;
  o->max_pending = 1 << 20;
  o->hbm_budget_bytes = 0;
  o->single_source_levels = 64;
  o->single_slots = 8;
  o->fast_slots = 2;
  o->fast_max_waiting = 2;
  o->single_cluster = 8;
  o->join = 1;
}

// Depth of one traversal of g from its first non-isolated vertex (0 if the
// first 4096 vertices are all isolated); scratch is a depth row of the pool.
static int probe_depth(ent_graph* g, int32_t* scratch, int32_t* levels) {
  *levels = 0;
  const int64_t n = std::min<int64_t>(g->V, 4096);
  std::vector<int64_t> off(n + 1);
  std::lock_guard<std::mutex> lk(g->mu);
  ENT_CUDA(cudaMemcpyAsync(off.data(), g->off, sizeof(int64_t) * (n + 1), cudaMemcpyDeviceToHost, g->stream));
  ENT_CUDA(cudaStreamSynchronize(g->stream));
  int32_t src = -1;
  for (int64_t v = 0; v < n && src < 0; ++v)
    if (off[v + 1] > off[v]) src = (int32_t)v;
  if (src < 0) return ENT_OK;
  ent_stats st{};
  int rc = run_bfs_single(g, src, scratch, nullptr, g->stream, &st);
  if (rc == ENT_OK) *levels = st.levels;
  return rc;
}

int ent_server_create(ent_graph* const* graphs, int32_t n_graphs, const ent_server_opts* opts, ent_server** out) {
  clear_error();
  if (!graphs || n_graphs < 1 || !out) return fail(ENT_ERR_INVALID_ARG, "bad arguments");
  *out = nullptr;
  ent_server_opts o;
  ent_server_opts_default(&o);
  if (opts) o = *opts;
  if (o.max_batch < 1 || o.max_batch > 2048) return fail(ENT_ERR_INVALID_ARG, "max_batch must be 1..2048");
  if (o.slots_per_graph < 1 || o.slots_per_graph > 16) return fail(ENT_ERR_INVALID_ARG, "slots_per_graph must be 1..16");
  if (o.max_pending < 1) return fail(ENT_ERR_INVALID_ARG, "max_pending must be >= 1");
  if (o.single_source_levels < 0) return fail(ENT_ERR_INVALID_ARG, "single_source_levels must be >= 0");
  if (o.single_slots < 1 || o.single_slots > 64) return fail(ENT_ERR_INVALID_ARG, "single_slots must be 1..64");
  if (o.fast_slots < 0 || o.fast_slots > 16) return fail(ENT_ERR_INVALID_ARG, "fast_slots must be 0..16");
  if (o.fast_max_waiting < 1) return fail(ENT_ERR_INVALID_ARG, "fast_max_waiting must be >= 1");
  if (o.single_cluster < 0 || o.single_cluster > 16) return fail(ENT_ERR_INVALID_ARG, "single_cluster must be 0..16");
  if (o.join < 0) return fail(ENT_ERR_INVALID_ARG, "join must be >= 0");
  const int dev = graphs[0]->device;
  for (int k = 0; k < n_graphs; ++k)
    if (!graphs[k] || graphs[k]->device != dev) return fail(ENT_ERR_INVALID_ARG, "all graphs must be on one GPU");
  DeviceGuard dg(dev);
  ent_server* s = new ent_server();
  s->opts = o;
  s->device = dev;
  size_t free_b = 0, total_b = 0;
  cudaMemGetInfo(&free_b, &total_b);
  const int64_t budget = o.hbm_budget_bytes > 0 ? o.hbm_budget_bytes : (int64_t)(free_b / 4);
  // Batched slots run on the highest stream priority, single-source slots on
  // the lowest: a single-source traversal of a deep graph holds a cluster of
  // SMs for milliseconds, and without priorities the grid-wide kernels of
  // batches queue behind it for SMs.
  if (cudaStreamCreateWithFlags(&s->prep, cudaStreamNonBlocking) != cudaSuccess) {
    free_server(s);
    return fail(ENT_ERR_CUDA, "server stream setup failed");
  }
  int prio_low = 0, prio_high = 0;
  cudaDeviceGetStreamPriorityRange(&prio_low, &prio_high);
  s->gs.resize(n_graphs);
  for (int k = 0; k < n_graphs; ++k) {
    GraphState& g = s->gs[k];
    g.g = graphs[k];
    g.V = graphs[k]->V;
    int64_t rows = o.rows_per_graph > 0 ? o.rows_per_graph : (budget / n_graphs) / (g.V * 4);
    rows = std::max<int64_t>(1, std::min<int64_t>(rows, 1 << 16));
    g.rows = (int32_t)rows;
    cudaError_t e = cudaMalloc(&g.pool, sizeof(int32_t) * (size_t)g.rows * g.V);
    if (e != cudaSuccess) {
      free_server(s);
      return fail(ENT_ERR_OOM, "graph %d: depth pool of %d rows does not fit", k, g.rows);
    }
    for (int r = g.rows - 1; r >= 0; --r) g.free_rows.push_back(r);
    if (o.single_source_levels > 0) {
      int rc = probe_depth(g.g, g.pool, &g.probe_levels);
      if (rc != ENT_OK) {
        free_server(s);
        return rc;
      }
      g.single = g.probe_levels >= o.single_source_levels;
    }
    if (g.single) {
      s->ctr.single_graphs++;
      g.slots.resize(o.single_slots);
      for (Slot& sl : g.slots) {
        int rc;
        {
          std::lock_guard<std::mutex> lk(g.g->mu);
          rc = create_bfs_workspace(g.g, &sl.sws, o.single_cluster);
        }
        if (rc == ENT_OK) {
          cudaError_t e2 = cudaStreamCreateWithPriority(&sl.stream, cudaStreamNonBlocking, prio_low);
          if (e2 == cudaSuccess) e2 = cudaEventCreateWithFlags(&sl.done, cudaEventDisableTiming);
          if (e2 != cudaSuccess) rc = fail(ENT_ERR_CUDA, "slot setup: %s", cudaGetErrorString(e2));
        }
        if (rc != ENT_OK) {
          free_server(s);
          return rc;
        }
      }
      continue;
    }
    g.slots.resize((size_t)o.fast_slots + o.slots_per_graph);
    for (int f = 0; f < o.fast_slots; ++f) {
      Slot& sl = g.slots[f];
      sl.fast = true;
      int rc;
      {
        std::lock_guard<std::mutex> lk(g.g->mu);
        rc = create_bfs_workspace(g.g, &sl.sws);
      }
      if (rc == ENT_OK) {
        cudaError_t e2 = cudaStreamCreateWithPriority(&sl.stream, cudaStreamNonBlocking, prio_high);
        if (e2 == cudaSuccess) e2 = cudaEventCreateWithFlags(&sl.done, cudaEventDisableTiming);
        if (e2 != cudaSuccess) rc = fail(ENT_ERR_CUDA, "slot setup: %s", cudaGetErrorString(e2));
      }
      if (rc != ENT_OK) {
        free_server(s);
        return rc;
      }
    }
    for (size_t b = (size_t)o.fast_slots; b < g.slots.size(); ++b) {
      Slot& sl = g.slots[b];
      int rc = create_batch_workspace(g.g, o.max_batch, &sl.ws);
      if (rc == ENT_OK) {
        cudaError_t e2 = cudaStreamCreateWithPriority(&sl.stream, cudaStreamNonBlocking, prio_high);
        if (e2 == cudaSuccess) e2 = cudaEventCreateWithFlags(&sl.done, cudaEventDisableTiming);
        if (e2 == cudaSuccess) e2 = cudaMalloc(&sl.row_map_dev, sizeof(int32_t) * JOIN_MAX);
        if (e2 == cudaSuccess) e2 = cudaGraphCreate(&sl.graph, 0);
        if (e2 == cudaSuccess) e2 = cudaHostAlloc((void**)&sl.box, sizeof(JoinBox), cudaHostAllocMapped);
        if (e2 == cudaSuccess) {
          memset(sl.box, 0, sizeof(JoinBox));
          e2 = cudaHostGetDevicePointer((void**)&sl.box_dev, sl.box, 0);
        }
        if (e2 != cudaSuccess) rc = fail(ENT_ERR_CUDA, "slot setup: %s", cudaGetErrorString(e2));
      }
      if (rc == ENT_OK && o.join) set_join_box(sl.ws, sl.box_dev);
      if (rc == ENT_OK) rc = append_branch(g.g, sl.ws, sl.graph, sl.stream);
      if (rc == ENT_OK && cudaGraphInstantiate(&sl.exec, sl.graph, 0) != cudaSuccess)
        rc = fail(ENT_ERR_CUDA, "slot graph instantiate failed");
      if (rc != ENT_OK) {
        free_server(s);
        return rc;
      }
    }
  }
  s->worker = std::thread(scheduler, s);
  *out = s;
  return ENT_OK;
}

int ent_server_submit(ent_server* s, int32_t graph, int32_t src, int64_t* query_id) {
  clear_error();
  if (!s || !query_id) return fail(ENT_ERR_INVALID_ARG, "null argument");
  if (graph < 0 || graph >= (int32_t)s->gs.size()) return fail(ENT_ERR_INVALID_ARG, "graph %d out of range", graph);
  if (src < 0 || src >= s->gs[graph].V) return fail(ENT_ERR_INVALID_ARG, "source %d out of range", src);
  std::lock_guard<std::mutex> lk(s->mu);
  if (s->n_pending >= s->opts.max_pending) {
    s->ctr.rejected++;
    return fail(ENT_ERR_ADMISSION, "queue full (%d waiting)", s->opts.max_pending);
  }
  const int64_t id = s->next_id++;
  Query q;
  q.graph = graph;
  q.src = src;
  q.t_submit = Clock::now();
  s->queries.emplace(id, q);
  s->gs[graph].pending.push_back(id);
  s->n_pending++;
  s->ctr.submitted++;
  *query_id = id;
  s->cv.notify_one();
  return ENT_OK;
}

int ent_server_poll(ent_server* s, ent_query_result* out, int32_t max_results, int32_t* n_out, int32_t wait_us) {
  clear_error();
  if (!s || !out || !n_out || max_results < 1) return fail(ENT_ERR_INVALID_ARG, "bad arguments");
  std::unique_lock<std::mutex> lk(s->mu);
  if (s->completed.empty() && wait_us > 0)
    s->cv_done.wait_for(lk, std::chrono::microseconds(wait_us), [&] { return !s->completed.empty(); });
  int n = 0;
  while (n < max_results && !s->completed.empty()) {
    const int64_t id = s->completed.front();
    s->completed.pop_front();
    auto it = s->queries.find(id);
    if (it == s->queries.end()) continue;
    const Query& q = it->second;
    ent_query_result& r = out[n++];
    r.query_id = id;
    r.graph = q.graph;
    r.src = q.src;
    r.reached_vertices = q.st.reached_vertices;
    r.traversed_edges = q.st.traversed_edges;
    r.levels = q.st.levels;
    r.status = q.st.status;
    r.latency_ms = std::chrono::duration<double, std::milli>(q.t_done - q.t_submit).count();
    r.queue_ms = std::chrono::duration<double, std::milli>(q.t_launch - q.t_submit).count();
  }
  *n_out = n;
  if (s->worker_error) return fail(s->worker_error, "%s", s->worker_msg.c_str());
  return ENT_OK;
}

static int find_done(ent_server* s, int64_t id, const GraphState** g, int32_t* row) {
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->queries.find(id);
  if (it == s->queries.end()) return fail(ENT_ERR_INVALID_ARG, "unknown or released query %lld", (long long)id);
  if (!it->second.done) return fail(ENT_ERR_INVALID_ARG, "query %lld has not completed", (long long)id);
  *g = &s->gs[it->second.graph];
  *row = it->second.row;
  return ENT_OK;
}

int ent_server_depth(ent_server* s, int64_t query_id, int32_t* depth_out) {
  clear_error();
  if (!s || !depth_out) return fail(ENT_ERR_INVALID_ARG, "null argument");
  const GraphState* g = nullptr;
  int32_t row = -1;
  int rc = find_done(s, query_id, &g, &row);
  if (rc != ENT_OK) return rc;
  DeviceGuard dg(s->device);
  ENT_CUDA(cudaMemcpy(depth_out, g->pool + (size_t)row * g->V, sizeof(int32_t) * g->V, cudaMemcpyDeviceToHost));
  return ENT_OK;
}

int ent_server_depth_device(ent_server* s, int64_t query_id, const int32_t** depth_dev) {
  clear_error();
  if (!s || !depth_dev) return fail(ENT_ERR_INVALID_ARG, "null argument");
  const GraphState* g = nullptr;
  int32_t row = -1;
  int rc = find_done(s, query_id, &g, &row);
  if (rc != ENT_OK) return rc;
  *depth_dev = g->pool + (size_t)row * g->V;
  return ENT_OK;
}

int ent_server_release(ent_server* s, int64_t query_id) {
  clear_error();
  if (!s) return fail(ENT_ERR_INVALID_ARG, "null server");
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->queries.find(query_id);
  if (it == s->queries.end()) return fail(ENT_ERR_INVALID_ARG, "unknown or released query %lld", (long long)query_id);
  if (!it->second.done) return fail(ENT_ERR_INVALID_ARG, "query %lld has not completed", (long long)query_id);
  s->gs[it->second.graph].free_rows.push_back(it->second.row);
  s->queries.erase(it);
  s->ctr.released++;
  s->cv.notify_one();
  return ENT_OK;
}

int ent_server_get_counters(ent_server* s, ent_server_counters* out) {
  if (!s || !out) return fail(ENT_ERR_INVALID_ARG, "null argument");
  std::lock_guard<std::mutex> lk(s->mu);
  *out = s->ctr;
  out->pending = s->n_pending;
  int64_t rows = 0, free_rows = 0;
  for (const GraphState& g : s->gs) {
    rows += g.rows;
    free_rows += (int64_t)g.free_rows.size();
  }
  out->rows_total = rows;
  out->rows_free = free_rows;
  return ENT_OK;
}

int ent_server_destroy(ent_server* s) {
  if (!s) return ENT_OK;
  s->stop.store(true);
  s->cv.notify_all();
  if (s->worker.joinable()) s->worker.join();
  free_server(s);
  return ENT_OK;
}

}  // extern "C"
