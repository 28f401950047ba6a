// Device graph: upload (replaces allocator<>::alloc_array, allocator.cuh:35-150),
// on-GPU generation of the seeded synthetic graphs, download and teardown.
//
// The GPU builder produces exactly the CSR of the host builder
// (host_graph.cpp): the same counter-based edge draws, then a radix sort of
// packed (u, v) keys, duplicate removal and offset search. Sorting uses CUB
// (graph construction only; it is not on the traversal path).
#include <cub/cub.cuh>
#include <string.h>
#include <omp.h>
#include <vector>

#include "dev_graph.h"
#include "gen_common.h"

namespace ent {

RmatParams make_rmat_params(int scale, int ef, double a, double b, double c, uint64_t seed);
GridParams make_grid_params(int64_t w, int64_t h, double drop, uint64_t seed);
ErParams make_er_params(int64_t n, double mean_degree, uint64_t seed);

__global__ void k_degrees(const int64_t* __restrict__ off, int32_t* __restrict__ deg, int64_t V) {
  for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < V; v += (int64_t)gridDim.x * blockDim.x)
    deg[v] = (int32_t)(off[v + 1] - off[v]);
}

int graph_alloc(ent_graph* g, int64_t V, int64_t E) {
  g->V = V;
  g->E = E;
  ENT_CUDA(cudaMalloc(&g->off, sizeof(int64_t) * (V + 1)));
  ENT_CUDA(cudaMalloc(&g->adj, sizeof(int32_t) * (E > 0 ? E : 1)));
  ENT_CUDA(cudaMalloc(&g->deg, sizeof(int32_t) * V));
  return ENT_OK;
}

__global__ void k_active_bits(const int32_t* __restrict__ deg, uint32_t* __restrict__ active, int64_t V) {
  const int64_t W = (V + 31) >> 5;
  for (int64_t w = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; w < W; w += (int64_t)gridDim.x * blockDim.x) {
    uint32_t bits = 0;
    for (int b = 0; b < 32; ++b) {
      const int64_t v = w * 32 + b;
      if (v < V && deg[v] > 0) bits |= 1u << b;
    }
    active[w] = bits;
  }
}

// Key that orders a row by descending neighbour degree, then ascending id.
__global__ void k_degree_keys(const int32_t* __restrict__ adj, const int32_t* __restrict__ deg, int64_t E,
                              unsigned long long* __restrict__ keys) {
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < E; e += (int64_t)gridDim.x * blockDim.x) {
    const int32_t u = adj[e];
    keys[e] = ((unsigned long long)(uint32_t)(0x7fffffff - deg[u]) << 32) | (uint32_t)u;
  }
}

__global__ void k_keys_to_ids(const unsigned long long* __restrict__ keys, int64_t E, int32_t* __restrict__ out) {
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < E; e += (int64_t)gridDim.x * blockDim.x)
    out[e] = (int32_t)(uint32_t)keys[e];
}

// lead[v] = the first 4 neighbours of v in the traversal adjacency (its
// highest-degree ones), -1 where the row is shorter.
__global__ void k_lead(const int64_t* __restrict__ off, const int32_t* __restrict__ trav, int64_t V,
                       int4* __restrict__ lead) {
  for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < V; v += (int64_t)gridDim.x * blockDim.x) {
    const int64_t b = off[v], d = off[v + 1] - b;
    lead[v] = make_int4(d > 0 ? trav[b] : -1, d > 1 ? trav[b + 1] : -1, d > 2 ? trav[b + 2] : -1,
                        d > 3 ? trav[b + 3] : -1);
  }
}

// Builds the traversal adjacency (rows by descending neighbour degree).
static int build_traversal_order(ent_graph* g) {
  const int64_t E = g->E, V = g->V;
  if (E == 0 || E > 0x7fffffffll || V > 0x7ffffffell) {
    g->trav = g->adj;  // no re-ordering: traverse the canonical rows
    return ENT_OK;
  }
  ENT_CUDA(cudaMalloc(&g->trav, sizeof(int32_t) * E));
  unsigned long long *k0 = nullptr, *k1 = nullptr;
  void* tmp = nullptr;
  size_t tmp_bytes = 0;
  cudaError_t e = cudaMalloc(&k0, sizeof(unsigned long long) * E);
  if (e == cudaSuccess) e = cudaMalloc(&k1, sizeof(unsigned long long) * E);
  const int blocks = g->num_sms * 16;
  if (e == cudaSuccess) {
    k_degree_keys<<<blocks, 256, 0, g->stream>>>(g->adj, g->deg, E, k0);
    g_kernel_launches++;
    e = cub::DeviceSegmentedSort::SortKeys(nullptr, tmp_bytes, k0, k1, (int)E, (int)V, g->off, g->off + 1,
                                           g->stream);
  }
  if (e == cudaSuccess) e = cudaMalloc(&tmp, tmp_bytes);
  if (e == cudaSuccess)
    e = cub::DeviceSegmentedSort::SortKeys(tmp, tmp_bytes, k0, k1, (int)E, (int)V, g->off, g->off + 1, g->stream);
  if (e == cudaSuccess) {
    k_keys_to_ids<<<blocks, 256, 0, g->stream>>>(k1, E, g->trav);
    g_kernel_launches++;
    e = cudaStreamSynchronize(g->stream);
  }
  if (k0) cudaFree(k0);
  if (k1) cudaFree(k1);
  if (tmp) cudaFree(tmp);
  if (e != cudaSuccess)
    return fail(e == cudaErrorMemoryAllocation ? ENT_ERR_OOM : ENT_ERR_CUDA, "traversal order build failed: %s",
                cudaGetErrorString(e));
  return ENT_OK;
}

int graph_finish(ent_graph* g) {
  ENT_CUDA(cudaDeviceGetAttribute(&g->num_sms, cudaDevAttrMultiProcessorCount, g->device));
  if (!g->stream) ENT_CUDA(cudaStreamCreateWithFlags(&g->stream, cudaStreamNonBlocking));
  int blocks = (int)std::min<int64_t>((g->V + 255) / 256, (int64_t)g->num_sms * 16);
  k_degrees<<<blocks, 256, 0, g->stream>>>(g->off, g->deg, g->V);
  g_kernel_launches++;
  ENT_CUDA(cudaGetLastError());
  const int64_t W = (g->V + 31) >> 5;
  ENT_CUDA(cudaMalloc(&g->active, sizeof(uint32_t) * (W + 1)));
  k_active_bits<<<(int)std::min<int64_t>((W + 255) / 256, (int64_t)g->num_sms * 16), 256, 0, g->stream>>>(
      g->deg, g->active, g->V);
  g_kernel_launches++;
  ENT_CUDA(cudaGetLastError());
  int rc = build_traversal_order(g);
  if (rc != ENT_OK) return rc;
  ENT_CUDA(cudaMalloc(&g->lead, sizeof(int4) * (g->V > 0 ? g->V : 1)));
  k_lead<<<blocks, 256, 0, g->stream>>>(g->off, g->trav, g->V, g->lead);
  g_kernel_launches++;
  ENT_CUDA(cudaGetLastError());
  ENT_CUDA(cudaStreamSynchronize(g->stream));
  ent_bfs_opts_default(&g->opts);
  return ENT_OK;
}

static void graph_free(ent_graph* g) {
  if (!g) return;
  DeviceGuard dg(g->device);
  if (g->ws) destroy_bfs_workspace(g->ws);
  if (g->bws) destroy_batch_workspace(g->bws);
  if (g->lanes) destroy_deep_lanes(g->lanes);
  if (g->stage) cudaFree(g->stage);
  if (g->trav && g->trav != g->adj) cudaFree(g->trav);
  if (g->active) cudaFree(g->active);
  if (g->lead) cudaFree(g->lead);
  if (g->off) cudaFree(g->off);
  if (g->adj) cudaFree(g->adj);
  if (g->deg) cudaFree(g->deg);
  if (g->stream) cudaStreamDestroy(g->stream);
  delete g;
}

// ----------------------------------------------------------- generators ---
// Key layout: (u << b) | v with b = ceil_log2(V); dropped draws and self
// loops get the sentinel (V << b), which sorts after every real key.
struct KeyCodec {
  int b;
  uint64_t V;
  __host__ __device__ uint64_t pack(uint64_t u, uint64_t v) const { return (u << b) | v; }
  __host__ __device__ uint64_t sentinel() const { return V << b; }
};

template <class Draw>
__global__ void k_gen_keys(Draw draw, uint64_t n_draws, KeyCodec kc, uint64_t* __restrict__ keys) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n_draws; i += (uint64_t)gridDim.x * blockDim.x) {
    uint64_t u, v;
    bool keep = draw(i, &u, &v);
    if (!keep || u == v) {
      keys[2 * i] = kc.sentinel();
      keys[2 * i + 1] = kc.sentinel();
    } else {
      keys[2 * i] = kc.pack(u, v);
      keys[2 * i + 1] = kc.pack(v, u);
    }
  }
}

__global__ void k_offsets_from_keys(const uint64_t* __restrict__ keys, int64_t n, KeyCodec kc, int64_t* __restrict__ off,
                                    int64_t V) {
  for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r <= V; r += (int64_t)gridDim.x * blockDim.x) {
    uint64_t target = (uint64_t)r << kc.b;
    int64_t lo = 0, hi = n;
    while (lo < hi) {
      int64_t mid = (lo + hi) >> 1;
      if (keys[mid] < target) lo = mid + 1; else hi = mid;
    }
    off[r] = lo;
  }
}

__global__ void k_adj_from_keys(const uint64_t* __restrict__ keys, int64_t n, uint64_t mask, int32_t* __restrict__ adj) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    adj[i] = (int32_t)(keys[i] & mask);
}

struct RmatDraw {
  RmatParams rp;
  __device__ bool operator()(uint64_t i, uint64_t* u, uint64_t* v) const {
    uint64_t x, y;
    rmat_edge(rp, i, &x, &y);
    *u = perm_pow2(rp.perm, x);
    *v = perm_pow2(rp.perm, y);
    return true;
  }
};
struct GridDraw {
  GridParams gp;
  __device__ bool operator()(uint64_t e, uint64_t* u, uint64_t* v) const {
    uint64_t x, y;
    bool keep = grid_edge(gp, e, &x, &y);
    *u = perm_apply(gp.perm, gp.n, x);
    *v = perm_apply(gp.perm, gp.n, y);
    return keep;
  }
};
struct ErDraw {
  ErParams ep;
  __device__ bool operator()(uint64_t i, uint64_t* u, uint64_t* v) const {
    uint64_t x, y;
    er_edge(ep, i, &x, &y);
    *u = perm_apply(ep.perm, ep.n, x);
    *v = perm_apply(ep.perm, ep.n, y);
    return true;
  }
};

template <class Draw>
static int build_on_device(Draw draw, uint64_t n_draws, int64_t V, int gpu, ent_graph** out) {
  DeviceGuard dg(gpu);
  ent_graph* g = new ent_graph();
  g->device = gpu;
  int nsm = 148;
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, gpu);
  cudaStream_t s;
  if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess) {
    delete g;
    return fail(ENT_ERR_CUDA, "stream create failed");
  }
  g->stream = s;
  KeyCodec kc;
  kc.V = (uint64_t)V;
  kc.b = ceil_log2((uint64_t)V + 1);
  int end_bit = 2 * kc.b + 1;
  if (end_bit > 64) { graph_free(g); return fail(ENT_ERR_UNSUPPORTED, "graph too large for packed keys"); }
  int64_t n_keys = (int64_t)(2 * n_draws);
  uint64_t *k0 = nullptr, *k1 = nullptr;
  void* tmp = nullptr;
  size_t tmp_bytes = 0, tmp2 = 0;
  int64_t* d_nsel = nullptr;
  int rc = ENT_OK;
  auto cleanup = [&]() {
    if (k0) cudaFree(k0);
    if (k1) cudaFree(k1);
    if (tmp) cudaFree(tmp);
    if (d_nsel) cudaFree(d_nsel);
  };
#define GEN_CUDA(call)                                                                          \
  do {                                                                                          \
    cudaError_t _e = (call);                                                                    \
    if (_e != cudaSuccess) {                                                                    \
      rc = fail(_e == cudaErrorMemoryAllocation ? ENT_ERR_OOM : ENT_ERR_CUDA, "%s: %s", #call, \
                cudaGetErrorString(_e));                                                        \
      cleanup();                                                                                \
      graph_free(g);                                                                            \
      return rc;                                                                                \
    }                                                                                           \
  } while (0)
  GEN_CUDA(cudaMalloc(&k0, sizeof(uint64_t) * std::max<int64_t>(n_keys, 1)));
  GEN_CUDA(cudaMalloc(&k1, sizeof(uint64_t) * std::max<int64_t>(n_keys, 1)));
  GEN_CUDA(cudaMalloc(&d_nsel, sizeof(int64_t)));
  int blocks = nsm * 16;
  k_gen_keys<<<blocks, 256, 0, s>>>(draw, n_draws, kc, k0);
  g_kernel_launches++;
  GEN_CUDA(cudaGetLastError());
  cub::DoubleBuffer<uint64_t> db(k0, k1);
  GEN_CUDA(cub::DeviceRadixSort::SortKeys(nullptr, tmp_bytes, db, n_keys, 0, end_bit, s));
  GEN_CUDA(cub::DeviceSelect::Unique(nullptr, tmp2, k0, k1, d_nsel, n_keys, s));
  tmp_bytes = std::max(tmp_bytes, tmp2);
  GEN_CUDA(cudaMalloc(&tmp, tmp_bytes));
  GEN_CUDA(cub::DeviceRadixSort::SortKeys(tmp, tmp_bytes, db, n_keys, 0, end_bit, s));
  uint64_t* sorted = db.Current();
  uint64_t* uniq = db.Alternate();
  GEN_CUDA(cub::DeviceSelect::Unique(tmp, tmp_bytes, sorted, uniq, d_nsel, n_keys, s));
  int64_t n_uniq = 0;
  GEN_CUDA(cudaMemcpyAsync(&n_uniq, d_nsel, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
  GEN_CUDA(cudaStreamSynchronize(s));
  // Drop the sentinel (at most one survives Unique, and it sorts last).
  if (n_uniq > 0) {
    uint64_t last = 0;
    GEN_CUDA(cudaMemcpy(&last, uniq + n_uniq - 1, sizeof(uint64_t), cudaMemcpyDeviceToHost));
    if (last == kc.sentinel()) --n_uniq;
  }
  if (graph_alloc(g, V, n_uniq) != ENT_OK) {
    rc = fail(ENT_ERR_OOM, "device allocation failed for graph (V=%lld E=%lld)", (long long)V, (long long)n_uniq);
    cleanup();
    graph_free(g);
    return rc;
  }
  k_offsets_from_keys<<<blocks, 256, 0, s>>>(uniq, n_uniq, kc, g->off, V);
  k_adj_from_keys<<<blocks, 256, 0, s>>>(uniq, n_uniq, (1ull << kc.b) - 1, g->adj);
  g_kernel_launches += 2;
  GEN_CUDA(cudaGetLastError());
  GEN_CUDA(cudaStreamSynchronize(s));
  cleanup();
  k0 = k1 = nullptr;
  tmp = nullptr;
  d_nsel = nullptr;
  rc = graph_finish(g);
  if (rc != ENT_OK) { graph_free(g); return rc; }
  *out = g;
  return ENT_OK;
#undef GEN_CUDA
}

}  // namespace ent

using namespace ent;

extern "C" {

void ent_bfs_opts_default(ent_bfs_opts* o) {
  if (!o) return;
  o->policy = ENT_POLICY_BEAMER;
  o->loop = ENT_LOOP_GRAPH;
  o->alpha = 24.0;  // measured on B200 (R-MAT s24 and Erdos-Renyi 2^24): Beamer's CPU values 14 / 24
  o->beta = 256.0;  // switch to bottom-up too early and back too early here
  o->ref_ratio = 0.3;
  o->small_max = 32;
  o->large_min = 1024;
  o->hub_slots = 0;
  o->chunk_edges = 2048;
  o->blocks_per_sm = 0;
  o->batch_alpha = 4.0;
  o->batch_small_max = 32;
  o->batch_large_min = 1024;
  o->batch_heavy = 4096;
  o->narrow_max_frontier = 8192;
  o->narrow_max_edges = 131072;
  o->narrow_max_degree = 256;
  o->narrow_cluster = 0;
  o->fault_inject = 0;
  o->batch_deep = 1;
  o->batch_deep_levels = 64;
  o->batch_deep_cluster = 0;
  o->batch_deep_lanes = 0;
}

int ent_graph_create(const int64_t* beg, const int32_t* csr, int64_t V, int64_t E, int32_t gpu, ent_graph** out) {
  ent::NvtxRange nvtx_range("ent_graph_create");
  clear_error();
  if (!beg || (!csr && E > 0) || !out || V < 1 || E < 0) return fail(ENT_ERR_INVALID_ARG, "bad arguments");
  *out = nullptr;
  if (V >= (1ll << 31) - 1) return fail(ENT_ERR_UNSUPPORTED, "V=%lld exceeds int32 ids", (long long)V);
  if (beg[0] != 0 || beg[V] != E) return fail(ENT_ERR_FORMAT, "beg_pos[0] must be 0 and beg_pos[V] must equal E");
  int64_t bad = -1;
#pragma omp parallel for reduction(max : bad)
  for (int64_t i = 0; i < V; ++i)
    if (beg[i + 1] < beg[i]) bad = std::max(bad, i);
  if (bad >= 0) return fail(ENT_ERR_FORMAT, "beg_pos not monotone at %lld", (long long)bad);
#pragma omp parallel for reduction(max : bad)
  for (int64_t k = 0; k < E; ++k)
    if (csr[k] < 0 || csr[k] >= V) bad = std::max(bad, k);
  if (bad >= 0) return fail(ENT_ERR_FORMAT, "csr entry %lld out of range [0,V)", (long long)bad);
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return fail(ENT_ERR_CUDA, "no CUDA device available");
  if (gpu < 0 || gpu >= ndev) return fail(ENT_ERR_INVALID_ARG, "gpu_id %d out of range (%d devices)", gpu, ndev);
  DeviceGuard dg(gpu);
  ent_graph* g = new ent_graph();
  g->device = gpu;
  int rc = graph_alloc(g, V, E);
  if (rc != ENT_OK) { graph_free(g); return rc; }
  // Upload on the graph's stream and wait for it: a cudaMemcpy from pageable
  // memory may return before its DMA lands, and the kernels that read the
  // CSR next run on this non-blocking stream.
  cudaError_t e1 = cudaStreamCreateWithFlags(&g->stream, cudaStreamNonBlocking);
  if (e1 == cudaSuccess)
    e1 = cudaMemcpyAsync(g->off, beg, sizeof(int64_t) * (V + 1), cudaMemcpyHostToDevice, g->stream);
  cudaError_t e2 = (E > 0 && e1 == cudaSuccess)
                       ? cudaMemcpyAsync(g->adj, csr, sizeof(int32_t) * E, cudaMemcpyHostToDevice, g->stream)
                       : cudaSuccess;
  if (e1 == cudaSuccess && e2 == cudaSuccess) e1 = cudaStreamSynchronize(g->stream);
  if (e1 != cudaSuccess || e2 != cudaSuccess) {
    graph_free(g);
    return fail(ENT_ERR_CUDA, "CSR upload failed");
  }
  rc = graph_finish(g);
  if (rc != ENT_OK) { graph_free(g); return rc; }
  *out = g;
  return ENT_OK;
}

int ent_graph_from_csr(const ent_csr* c, int32_t gpu, ent_graph** out) {
  if (!c) return fail(ENT_ERR_INVALID_ARG, "null csr");
  return ent_graph_create(c->off.data(), c->adj.data(), c->V, c->E, gpu, out);
}

static int check_gpu(int gpu) {
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return fail(ENT_ERR_CUDA, "no CUDA device available");
  if (gpu < 0 || gpu >= ndev) return fail(ENT_ERR_INVALID_ARG, "gpu_id %d out of range", gpu);
  return ENT_OK;
}

int ent_graph_gen_rmat(int32_t scale, int32_t ef, double a, double b, double c, uint64_t seed, int32_t gpu,
                       ent_graph** out) {
  ent::NvtxRange nvtx_range("ent_graph_gen_rmat");
  clear_error();
  if (!out || scale < 1 || scale > 30 || ef < 1 || a < 0 || b < 0 || c < 0 || a + b + c > 1.0)
    return fail(ENT_ERR_INVALID_ARG, "bad R-MAT parameters");
  int rc = check_gpu(gpu);
  if (rc) return rc;
  RmatDraw d{make_rmat_params(scale, ef, a, b, c, seed)};
  return build_on_device(d, d.rp.n_edges, 1ll << scale, gpu, out);
}

int ent_graph_gen_grid(int64_t w, int64_t h, double drop, uint64_t seed, int32_t gpu, ent_graph** out) {
  clear_error();
  if (!out || w < 2 || h < 2 || drop < 0 || drop > 1 || w * h >= (1ll << 31) - 1)
    return fail(ENT_ERR_INVALID_ARG, "bad grid parameters");
  int rc = check_gpu(gpu);
  if (rc) return rc;
  GridDraw d{make_grid_params(w, h, drop, seed)};
  return build_on_device(d, d.gp.n_edges, (int64_t)d.gp.n, gpu, out);
}

int ent_graph_gen_er(int64_t n, double mean_degree, uint64_t seed, int32_t gpu, ent_graph** out) {
  clear_error();
  if (!out || n < 2 || n >= (1ll << 31) - 1 || mean_degree < 0) return fail(ENT_ERR_INVALID_ARG, "bad ER parameters");
  int rc = check_gpu(gpu);
  if (rc) return rc;
  ErDraw d{make_er_params(n, mean_degree, seed)};
  return build_on_device(d, d.ep.n_edges, n, gpu, out);
}

namespace ent {
// A caller's edge list already on the device (endpoints checked in range).
struct ListDraw {
  const int64_t* src;
  const int64_t* dst;
  __device__ bool operator()(uint64_t i, uint64_t* u, uint64_t* v) const {
    *u = (uint64_t)src[i];
    *v = (uint64_t)dst[i];
    return true;
  }
};

__global__ void k_first_bad_edge(const int64_t* __restrict__ src, const int64_t* __restrict__ dst, int64_t n,
                                 int64_t V, unsigned long long* first) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    if (src[i] < 0 || src[i] >= V || dst[i] < 0 || dst[i] >= V) atomicMin(first, (unsigned long long)i);
}
}  // namespace ent

int ent_graph_from_edges(const int64_t* src, const int64_t* dst, int64_t n, int64_t V, int32_t gpu,
                         ent_graph** out) {
  ent::NvtxRange nvtx_range("ent_graph_from_edges");
  clear_error();
  if ((!src || !dst) && n > 0) return fail(ENT_ERR_INVALID_ARG, "null edge arrays");
  if (!out || V < 1 || n < 0) return fail(ENT_ERR_INVALID_ARG, "bad arguments");
  if (V >= (1ll << 31) - 1) return fail(ENT_ERR_UNSUPPORTED, "V exceeds int32 ids");
  int rc = check_gpu(gpu);
  if (rc) return rc;
  DeviceGuard dg(gpu);
  int64_t *d_src = nullptr, *d_dst = nullptr;
  unsigned long long* d_bad = nullptr;
  unsigned long long bad = ~0ull;
  cudaStream_t s = nullptr;
  cudaError_t e = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
  const size_t bytes = sizeof(int64_t) * (size_t)std::max<int64_t>(n, 1);
  if (e == cudaSuccess) e = cudaMalloc(&d_src, bytes);
  if (e == cudaSuccess) e = cudaMalloc(&d_dst, bytes);
  if (e == cudaSuccess) e = cudaMalloc(&d_bad, sizeof(bad));
  if (e == cudaSuccess && n > 0) e = cudaMemcpyAsync(d_src, src, sizeof(int64_t) * n, cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess && n > 0) e = cudaMemcpyAsync(d_dst, dst, sizeof(int64_t) * n, cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(d_bad, &bad, sizeof(bad), cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess && n > 0) {
    int nsm = 148;
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, gpu);
    k_first_bad_edge<<<nsm * 8, 256, 0, s>>>(d_src, d_dst, n, V, d_bad);
    g_kernel_launches++;
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpyAsync(&bad, d_bad, sizeof(bad), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) {
    rc = fail(e == cudaErrorMemoryAllocation ? ENT_ERR_OOM : ENT_ERR_CUDA, "edge upload failed: %s",
              cudaGetErrorString(e));
  } else if (bad != ~0ull) {
    rc = fail(ENT_ERR_FORMAT, "edge %lld has an endpoint outside [0,V)", (long long)bad);
  } else {
    rc = build_on_device(ListDraw{d_src, d_dst}, (uint64_t)n, V, gpu, out);
  }
  if (d_src) cudaFree(d_src);
  if (d_dst) cudaFree(d_dst);
  if (d_bad) cudaFree(d_bad);
  if (s) cudaStreamDestroy(s);
  return rc;
}

int64_t ent_graph_vert_count(const ent_graph* g) { return g ? g->V : -1; }
int64_t ent_graph_edge_count(const ent_graph* g) { return g ? g->E : -1; }
int32_t ent_graph_device(const ent_graph* g) { return g ? g->device : -1; }
int64_t ent_graph_device_bytes(const ent_graph* g) {
  if (!g) return -1;
  const int64_t V = g->V, E = g->E, W = (V + 31) >> 5;
  int64_t b = 8 * (V + 1) + 4 * std::max<int64_t>(E, 1) + 4 * V + 4 * (W + 1) + 16 * std::max<int64_t>(V, 1);
  if (g->trav && g->trav != g->adj) b += 4 * E;
  return b;
}

int ent_device_alloc(int32_t gpu, size_t bytes, void** out) {
  clear_error();
  if (!out) return fail(ENT_ERR_INVALID_ARG, "null argument");
  *out = nullptr;
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || gpu < 0 || gpu >= n)
    return fail(ENT_ERR_INVALID_ARG, "no GPU %d (%d present)", gpu, n);
  DeviceGuard dg(gpu);
  void* p = nullptr;
  if (cudaMalloc(&p, bytes ? bytes : 1) != cudaSuccess)
    return fail(ENT_ERR_OOM, "device allocation of %zu bytes on GPU %d failed", bytes, gpu);
  *out = p;
  return ENT_OK;
}

int ent_device_free(void* p) {
  clear_error();
  if (p && cudaFree(p) != cudaSuccess) return fail(ENT_ERR_CUDA, "device free failed");
  return ENT_OK;
}

int ent_graph_download(const ent_graph* g, int64_t* beg, int32_t* csr) {
  clear_error();
  if (!g || !beg || (!csr && g->E > 0)) return fail(ENT_ERR_INVALID_ARG, "null argument");
  DeviceGuard dg(g->device);
  ENT_CUDA(cudaMemcpy(beg, g->off, sizeof(int64_t) * (g->V + 1), cudaMemcpyDeviceToHost));
  if (g->E > 0) ENT_CUDA(cudaMemcpy(csr, g->adj, sizeof(int32_t) * g->E, cudaMemcpyDeviceToHost));
  return ENT_OK;
}

int ent_graph_device_csr(const ent_graph* g, const int64_t** beg, const int32_t** csr) {
  if (!g || !beg || !csr) return fail(ENT_ERR_INVALID_ARG, "null argument");
  *beg = g->off;
  *csr = g->adj;
  return ENT_OK;
}

int ent_graph_set_opts(ent_graph* g, const ent_bfs_opts* o) {
  clear_error();
  if (!g || !o) return fail(ENT_ERR_INVALID_ARG, "null argument");
  if (o->policy < 0 || o->policy > 3) return fail(ENT_ERR_INVALID_ARG, "unknown policy %d", o->policy);
  if (o->loop < 0 || o->loop > 1) return fail(ENT_ERR_INVALID_ARG, "unknown loop mode %d", o->loop);
  if (o->small_max < 1 || o->large_min < o->small_max) return fail(ENT_ERR_INVALID_ARG, "need 1 <= small_max <= large_min");
  if (o->hub_slots < 0 || o->hub_slots > 4096 || (o->hub_slots & (o->hub_slots - 1)))
    return fail(ENT_ERR_INVALID_ARG, "hub_slots must be 0 or a power of two <= 4096");
  if (o->chunk_edges < 32) return fail(ENT_ERR_INVALID_ARG, "chunk_edges must be >= 32");
  if (o->alpha <= 0 || o->beta <= 0 || o->ref_ratio < 0) return fail(ENT_ERR_INVALID_ARG, "alpha/beta must be > 0");
  if (o->blocks_per_sm < 0 || o->blocks_per_sm > 32) return fail(ENT_ERR_INVALID_ARG, "blocks_per_sm out of range");
  if (o->batch_alpha <= 0) return fail(ENT_ERR_INVALID_ARG, "batch_alpha must be > 0");
  if (o->batch_small_max < 1 || o->batch_large_min < o->batch_small_max)
    return fail(ENT_ERR_INVALID_ARG, "need 1 <= batch_small_max <= batch_large_min");
  if (o->batch_heavy < 32) return fail(ENT_ERR_INVALID_ARG, "batch_heavy must be >= 32");
  if (o->narrow_max_frontier < 0 || o->narrow_max_frontier > 16384)
    return fail(ENT_ERR_INVALID_ARG, "narrow_max_frontier must be in [0, 16384]");
  if (o->narrow_max_edges < 0 || o->narrow_max_degree < 1 || o->narrow_max_degree > (1 << 20))
    return fail(ENT_ERR_INVALID_ARG, "need narrow_max_edges >= 0 and 1 <= narrow_max_degree <= 2^20");
  if (o->narrow_cluster < 0 || o->narrow_cluster > 16) return fail(ENT_ERR_INVALID_ARG, "narrow_cluster must be in [0, 16]");
  if (o->fault_inject < 0 || o->fault_inject > 1) return fail(ENT_ERR_INVALID_ARG, "fault_inject must be 0 or 1");
  if (o->batch_deep < 0 || o->batch_deep > 2) return fail(ENT_ERR_INVALID_ARG, "batch_deep must be 0, 1 or 2");
  if (o->batch_deep_levels < 1) return fail(ENT_ERR_INVALID_ARG, "batch_deep_levels must be >= 1");
  if (o->batch_deep_cluster < 0 || o->batch_deep_cluster > 16)
    return fail(ENT_ERR_INVALID_ARG, "batch_deep_cluster must be in [0, 16]");
  if (o->batch_deep_lanes < 0 || o->batch_deep_lanes > 256)
    return fail(ENT_ERR_INVALID_ARG, "batch_deep_lanes must be in [0, 256]");
  std::lock_guard<std::mutex> lk(g->mu);
  g->opts = *o;
  if (g->ws || g->bws || g->lanes) {  // workspaces were built and captured with the old options
    DeviceGuard dg(g->device);
    cudaStreamSynchronize(g->stream);
    destroy_bfs_workspace(g->ws);
    g->ws = nullptr;
    destroy_batch_workspace(g->bws);
    g->bws = nullptr;
    destroy_deep_lanes(g->lanes);  // waits for its lanes' streams
    g->lanes = nullptr;
  }
  return ENT_OK;
}

int ent_graph_get_opts(const ent_graph* g, ent_bfs_opts* o) {
  if (!g || !o) return fail(ENT_ERR_INVALID_ARG, "null argument");
  *o = g->opts;
  return ENT_OK;
}

int ent_graph_destroy(ent_graph* g) {
  clear_error();
  if (!g) return ENT_OK;
  {
    DeviceGuard dg(g->device);
    if (g->stream) cudaStreamSynchronize(g->stream);
  }
  graph_free(g);
  return ENT_OK;
}

}  // extern "C"
