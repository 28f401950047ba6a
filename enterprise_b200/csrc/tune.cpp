// Autotuner for the traversal's thresholds. No reference counterpart: the
// reference fixes its tiers and bins at compile time (sml_shed = 32,
// lrg_shed = 1024, bfs_gpu_opt.cuh:323-324; BIN_SZ, comm.h:155; hub sizes,
// comm.h:176-177; switch ratio 0.3, inspector.cuh:497).
//
// Method: coordinate descent from the current options. For each knob in turn
// every candidate value is applied (ent_graph_set_opts, which rebuilds the
// workspaces and their CUDA graphs), one untimed run warms the new state up,
// then `reps` timed runs over the given sources are taken; the score is the
// smallest total device time (CUDA events) of those runs, and the knob keeps
// its best value. Two sweeps. Any option set yields the same depths, so the
// search can only change speed.
#include <algorithm>
#include <vector>

#include "dev_graph.h"

namespace {

struct Knob {
  const char* name;
  std::vector<double> values;
  void (*set)(ent_bfs_opts&, double);
};

void set_small(ent_bfs_opts& o, double v) { o.small_max = (int32_t)v; }
void set_large(ent_bfs_opts& o, double v) { o.large_min = (int32_t)v; }
void set_chunk(ent_bfs_opts& o, double v) { o.chunk_edges = (int32_t)v; }
void set_hub(ent_bfs_opts& o, double v) { o.hub_slots = (int32_t)v; }
void set_alpha(ent_bfs_opts& o, double v) { o.alpha = v; }
void set_beta(ent_bfs_opts& o, double v) { o.beta = v; }
void set_bps(ent_bfs_opts& o, double v) { o.blocks_per_sm = (int32_t)v; }
void set_balpha(ent_bfs_opts& o, double v) { o.batch_alpha = v; }
void set_bsmall(ent_bfs_opts& o, double v) { o.batch_small_max = (int32_t)v; }
void set_blarge(ent_bfs_opts& o, double v) { o.batch_large_min = (int32_t)v; }
void set_bheavy(ent_bfs_opts& o, double v) { o.batch_heavy = (int32_t)v; }

// Total device time of one evaluation (min over reps); <0 on error.
double score(ent_graph* g, const int32_t* src, int32_t n, int mode, int reps) {
  double best = -1;
  std::vector<ent_stats> st(std::max(n, 1));
  for (int r = -1; r < reps; ++r) {  // r == -1: warm-up
    double t = 0;
    if (mode == 0) {
      for (int i = 0; i < n; ++i) {
        if (ent_bfs(g, src[i], nullptr, nullptr, &st[0]) != ENT_OK) return -1;
        t += st[0].device_ms;
      }
    } else {
      if (ent_bfs_batch(g, src, n, nullptr, st.data()) != ENT_OK) return -1;
      t = st[0].device_ms;
    }
    if (r >= 0 && (best < 0 || t < best)) best = t;
  }
  return best;
}

}  // namespace

extern "C" int ent_autotune(ent_graph* g, const int32_t* src, int32_t n_src, int32_t mode, int32_t reps,
                            ent_bfs_opts* best_out, double* best_ms_out) {
  ent::NvtxRange nvtx_range("ent_autotune");
  ent::clear_error();
  if (!g || !src || n_src < 1 || (mode != 0 && mode != 1) || reps < 1)
    return ent::fail(ENT_ERR_INVALID_ARG, "bad arguments");
  std::vector<Knob> knobs;
  if (mode == 0) {
    knobs = {{"small_max", {16, 32, 64, 128, 256}, set_small}, {"large_min", {128, 256, 512, 1024, 4096}, set_large},
             {"chunk_edges", {256, 512, 1024, 2048, 8192}, set_chunk}, {"hub_slots", {0, 1024}, set_hub},
             {"alpha", {8, 14, 24, 48, 96}, set_alpha}, {"beta", {24, 64, 256, 1024}, set_beta},
             {"blocks_per_sm", {0, 4}, set_bps}};
  } else {
    knobs = {{"batch_alpha", {1, 2, 4, 8, 16}, set_balpha},
             {"batch_small_max", {16, 32, 64}, set_bsmall},
             {"batch_large_min", {512, 1024, 4096}, set_blarge},
             {"batch_heavy", {1024, 4096, 16384}, set_bheavy}};
  }
  ent_bfs_opts best;
  if (ent_graph_get_opts(g, &best) != ENT_OK) return ENT_ERR_INVALID_ARG;
  ent_bfs_opts start = best;
  double best_t = score(g, src, n_src, mode, reps);
  if (best_t < 0) return ENT_ERR_CUDA;
  for (int sweep = 0; sweep < 2; ++sweep) {
    for (const Knob& k : knobs) {
      for (double v : k.values) {
        ent_bfs_opts o = best;
        k.set(o, v);
        if (o.large_min < o.small_max || o.batch_large_min < o.batch_small_max) continue;
        if (ent_graph_set_opts(g, &o) != ENT_OK) continue;
        const double t = score(g, src, n_src, mode, reps);
        if (t >= 0 && t < best_t) {
          best_t = t;
          best = o;
        }
      }
    }
  }
  int rc = ent_graph_set_opts(g, &best);
  if (rc != ENT_OK) {
    ent_graph_set_opts(g, &start);
    return rc;
  }
  if (best_out) *best_out = best;
  if (best_ms_out) *best_ms_out = best_t;
  return ENT_OK;
}
