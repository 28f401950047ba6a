// Direction-optimising single-source BFS for sm_100a.
//
// What it replaces (reference bfs_gpu_opt.cuh:40-288 and the kernels it
// drives): a host-driven level loop that per level launches 13-14 kernels
// (inspector over all V, three two-kernel scans, three reapers, three
// expanders) and synchronises the host >= 5 times.
//
// Design here:
//  * Status lives in bitmaps: `vis` (visited, 1 bit/vertex), the graph's
//    `active` bitmap (degree > 0) and two frontier bitmaps fb[level & 1].
//    At s24 each is 2 MB and stays in L2.
//  * Top-down (TD) levels expand classified frontier queues (small: < small_max,
//    warp-cooperative gather; mid: warp per vertex; large: CTA per chunk of
//    chunk_edges edges), claim vertices with atomicOr on `vis`, and append
//    discoveries to a raw queue with warp-aggregated atomics
//    (reference expanders K2-K4, expander.cuh:74-423).
//  * Bottom-up (BU) levels sweep the status bitmaps: a warp owns one word
//    (32 consecutive ids) and checks only unvisited, non-isolated vertices,
//    each lane serially for small degrees, the whole warp together for large
//    ones, stopping at the first neighbour in the frontier bitmap or in a
//    shared-memory hub cache of the frontier's highest-degree vertices
//    (reference K5-K7, expander.cuh:431-819; hub cache comm.h:172-177).
//    Rows are ordered by descending neighbour degree, so the first check
//    usually meets a hub; each vertex's first four neighbours are also kept
//    in a `lead` array read coalesced beside its row offsets, so that check
//    costs no scattered row read.
//  * The inspector (reference K8/K9/K11, inspector.cuh:36-432) classifies the
//    next frontier into small/mid/large queues with one single-pass
//    decoupled look-back scan, order-preserving: from the raw discovery queue
//    after a TD level, from the frontier bitmap (the status array) when a BU
//    level hands over to TD.
//  * The direction policy runs on the device in the inspector's last CTA
//    (reference rule inspector.cuh:486-521 is one option; Beamer alpha/beta
//    with switch-back is the default).
//  * Small frontiers (high-diameter graphs such as grids, and the first and
//    last levels of any traversal) would pay two grid-wide launches per level.
//    While the TD frontier stays small, one thread-block cluster runs level
//    after level inside a single launch instead (k_narrow): the frontier lives
//    in the CTAs' shared memory (read across the cluster through distributed
//    shared memory), levels are separated by the hardware cluster barrier, and
//    each queue entry carries the vertex's row start and degree, read while
//    its visit was being claimed, so a level costs one adjacency read, one
//    status probe and one claim on its critical path.
//  * The whole traversal is one CUDA graph: a reset kernel (which also writes
//    the loop state), then a while node whose body is two copies of
//    [expand, inspect, narrow]; the inspector sets the loop condition and the
//    small-frontier flag, and the cluster kernel leaves at once unless that
//    flag is set. The look-back wait is the only spin: it is bounded, and a
//    classification whose wait ran out ends the traversal with an error bit
//    instead of handing on inconsistent queues.
#include <algorithm>
#include <type_traits>
#include <vector>
#include <string.h>

#include <cooperative_groups.h>

#include "dev_common.cuh"
#include "dev_graph.h"

namespace ent {

constexpr int BT = 256;          // threads per CTA of the level kernels
constexpr int IPT = 4;           // items per thread in an inspector tile
constexpr int TILE = BT * IPT;   // items per inspector tile
constexpr int KS = 4;            // look-back status words per tile
constexpr int WPT = 8;           // bitmap words per thread when classifying a frontier bitmap (two uint4)
constexpr int TD = 0, BU = 1;
constexpr int NWE = 16;          // expansion warps per CTA of the small-frontier kernel
constexpr int NT = 32 * (NWE + 1);  // ... plus one coordinator warp
constexpr int NROUND = 4;        // rounds of 32 edges a warp keeps in flight together
constexpr int NC_MAX = 16;       // CTAs per cluster, at most
constexpr int NQCAP = 4096;      // small-frontier entries per CTA and buffer
constexpr uint32_t NF_HEAVY = 1, NF_SPILL = 2;
constexpr int LCAP = 128;        // vertices a CTA of a listing bottom-up level keeps (then the bitmap is used)
constexpr int BU_ILP = 2;        // bottom-up light path: neighbours checked per step (2 beat 4 and 8)
constexpr int LOOP_UNROLL = 2;   // level-loop bodies per while-node iteration of the CUDA-graph loop

// Device-resident loop state. Written only by the reset kernel's and the
// inspector's last CTA (plus atomics on the acc_* counters and n_raw); read
// by every kernel at start.
struct BfsCtl {
  int32_t src;
  int32_t pad0;
  int32_t* depth;
  int32_t* parent;
  int32_t level;      // the frontier holds the vertices at depth `level`
  int32_t dir;        // direction used to expand `level`
  int32_t qcur;       // ping-pong index of TD queues
  int32_t n_q[3];     // TD frontier queue sizes (small, mid, large)
  int32_t n_chunks;   // chunks of the large TD queue
  int32_t n_raw;      // TD raw next-frontier count (atomic append)
  int32_t done;
  int32_t narrow;     // next level runs in the small-frontier kernel (next to `done`: read together)
  int32_t err;        // bit 1: look-back wait timed out, 2: level overflow, 3: count overflow
  int32_t td_levels;
  int32_t bu_levels;
  int32_t skip;       // the small-frontier kernel already expanded this level
  int32_t narrow_levels;
  int32_t iters;      // inspector launches (level-loop iterations)
  int32_t narrow_runs;
  int32_t narrow_calls;  // launches of the small-frontier kernel, those that left at once included
  uint32_t n_spill;   // small-frontier entries that did not fit in shared memory
  uint32_t acc_maxd;  // maximum degree in the next frontier being classified
  int64_t n_f, m_f;   // frontier size and degree sum
  int64_t n_vis, m_vis;
  unsigned long long acc_n, acc_m;  // next frontier size / degree sum being accumulated
  uint32_t tot[KS];   // chain totals, written by the last tile
  uint32_t tile_ticket;
  uint32_t finished;
  uint32_t epoch;
  int32_t bu_list;    // the bottom-up level being expanded also lists what it finds in raw
  int32_t list_over;  // ... and a CTA found more than it could list: use the frontier bitmap
};

struct LevelArgs {
  BfsCtl* ctl;
  const int64_t* off;
  const int32_t* adj;      // traversal order (descending neighbour degree)
  const int4* lead;        // adj[off[v] .. off[v]+3] per vertex (-1 past the row)
  const int32_t* deg;
  const uint32_t* active;
  int64_t V, E;
  uint32_t* vis;
  uint32_t* fb[2];
  int32_t* q[2][3];
  int32_t* qc[2];
  int32_t* raw;
  unsigned long long* hub[2];
  unsigned long long* tiles;  // [tiles][KS]
  int32_t small_max, large_min, chunk, hub_slots, hub_shift, hub_min_deg;
  int32_t policy;
  double alpha, beta, ref_ratio;
  cudaGraphConditionalHandle cond;
  int32_t use_cond;
  int32_t max_levels;
  // small-frontier mode: enter at <= narrow_f vertices, <= narrow_m edges and
  // no degree above narrow_deg; leave above exit_f vertices or exit_m edges.
  int32_t narrow_f, exit_f, narrow_deg;
  int32_t fault_inject;  // test hook (ent_bfs_opts::fault_inject)
  int64_t narrow_m, exit_m;
};

__device__ __forceinline__ int cls_of(int d, const LevelArgs& a) {
  return d < a.small_max ? 0 : (d > a.large_min ? 2 : 1);
}
__device__ __forceinline__ uint32_t n_chunks_of(int d, const LevelArgs& a) {
  return (uint32_t)((d + a.chunk - 1) / a.chunk);
}
__device__ __forceinline__ uint32_t hub_slot(uint32_t v, int shift) { return (v * 0x9E3779B1u) >> shift; }

// Direct-mapped table of the frontier's highest-degree vertices (the
// reference keeps the max-degree vertex per slot, inspector.cuh:218-224, but
// without atomics). Reading first keeps the atomics to the few keys that win.
__device__ __forceinline__ void hub_insert(const LevelArgs& a, unsigned long long* ht, int v, int d) {
  if (a.hub_slots && d >= a.hub_min_deg) {
    unsigned long long* slot = ht + hub_slot((uint32_t)v, a.hub_shift);
    const unsigned long long key = ((unsigned long long)(uint32_t)d << 32) | (uint32_t)v;
    if (__ldcg(slot) < key) atomicMax(slot, key);
  }
}

template <class T>
__device__ __forceinline__ T block_sum(T x, T* s_red) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(FULL, x, o);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) s_red[warp] = x;
  __syncthreads();
  T r = 0;
  if (threadIdx.x == 0)
    for (int w = 0; w < BT / 32; ++w) r += s_red[w];
  return r;  // valid in thread 0
}

__device__ __forceinline__ uint32_t block_max(uint32_t x, uint32_t* s_red) {
  x = __reduce_max_sync(FULL, x);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) s_red[warp] = x;
  __syncthreads();
  uint32_t r = 0;
  if (threadIdx.x == 0)
    for (int w = 0; w < BT / 32; ++w) r = max(r, s_red[w]);
  return r;  // valid in thread 0
}

// --------------------------------------------------------------- reset ----
// Fills p[0, n) with -1, except p[sp] = sv. The thread that stores the
// element or 16-byte vector holding sp stores sv in it, so nothing has to be
// ordered after the fill to set the source's own entry.
__device__ void fill_neg1(int32_t* p, int64_t n, int64_t tid, int64_t nth, int64_t sp, int32_t sv) {
  uintptr_t addr = (uintptr_t)p;
  int64_t head = (int64_t)(((16 - (addr & 15)) & 15) >> 2);
  if ((addr & 3) != 0) head = n;  // not even 4-byte aligned: scalar path
  if (head > n) head = n;
  for (int64_t i = tid; i < head; i += nth) p[i] = i == sp ? sv : -1;
  int64_t nvec = (n - head) >> 2;
  int4* pv = reinterpret_cast<int4*>(p + head);
  const int64_t vs = sp >= head ? (sp - head) >> 2 : -1;
  const int ks = (int)((sp - head) & 3);
  for (int64_t i = tid; i < nvec; i += nth) {
    const bool at = i == vs;
    pv[i] = make_int4(at && ks == 0 ? sv : -1, at && ks == 1 ? sv : -1, at && ks == 2 ? sv : -1,
                      at && ks == 3 ? sv : -1);
  }
  for (int64_t i = head + nvec * 4 + tid; i < n; i += nth) p[i] = i == sp ? sv : -1;
}

// Byte depths, the reference's depth_t (unsigned char, comm.h:69): depth d
// (0..254) as d, unreached as 255 (INFTY, comm.h:131). Fills p[0, n) with
// 0xFF except p[sp] = sv, as fill_neg1 does.
__device__ void fill_ff(uint8_t* p, int64_t n, int64_t tid, int64_t nth, int64_t sp, uint8_t sv) {
  const uintptr_t addr = (uintptr_t)p;
  int64_t head = (int64_t)((16 - (addr & 15)) & 15);
  if (head > n) head = n;
  for (int64_t i = tid; i < head; i += nth) p[i] = i == sp ? sv : (uint8_t)0xFF;
  const int64_t nvec = (n - head) >> 4;
  uint4* pv = reinterpret_cast<uint4*>(p + head);
  const int64_t vs = sp >= head ? (sp - head) >> 4 : -1;
  const int bs = (int)((sp - head) & 15), ws = bs >> 2, sh = 8 * (bs & 3);
  const uint32_t patched = ~(0xFFu << sh) | ((uint32_t)sv << sh);
  for (int64_t i = tid; i < nvec; i += nth) {
    const bool at = i == vs;
    pv[i] = make_uint4(at && ws == 0 ? patched : ~0u, at && ws == 1 ? patched : ~0u, at && ws == 2 ? patched : ~0u,
                       at && ws == 3 ? patched : ~0u);
  }
  for (int64_t i = head + nvec * 16 + tid; i < n; i += nth) p[i] = i == sp ? sv : (uint8_t)0xFF;
}
__device__ __forceinline__ void fill_unreached(int32_t* p, int64_t n, int64_t tid, int64_t nth, int64_t src) {
  fill_neg1(p, n, tid, nth, src, 0);
}
__device__ __forceinline__ void fill_unreached(uint8_t* p, int64_t n, int64_t tid, int64_t nth, int64_t src) {
  fill_ff(p, n, tid, nth, src, 0);
}

// Loop state for one traversal from src (its frontier: src alone, classified
// by degree). Written by one thread of k_reset while the others fill; no fill
// touches the control block or the queues.
template <class DT>
__device__ void init_state(const LevelArgs& a, int32_t src, DT* depth, int32_t* parent) {
  BfsCtl* c = a.ctl;
  const int d = a.deg[src];
  const int cl = cls_of(d, a);
  a.q[0][cl][0] = src;
  c->src = src;
  c->depth = reinterpret_cast<int32_t*>(depth);  // the level kernels of this DT cast it back
  c->parent = parent;
  c->level = 0;
  c->dir = a.policy == ENT_POLICY_BU_ONLY ? BU : TD;
  c->qcur = 0;
  for (int k = 0; k < 3; ++k) c->n_q[k] = 0;
  c->n_q[cl] = 1;
  if (cl == 2) {
    a.qc[0][0] = 0;
    c->n_chunks = (int32_t)n_chunks_of(d, a);
  } else {
    c->n_chunks = 0;
  }
  c->n_raw = 0;
  c->bu_list = 0;
  c->list_over = 0;
  c->done = 0;
  c->narrow = 0;
  c->err = 0;
  c->td_levels = 0;
  c->bu_levels = 0;
  c->skip = 0;
  c->narrow_levels = 0;
  c->iters = 0;
  c->narrow_runs = 0;
  c->narrow_calls = 0;
  c->n_spill = 0;
  c->acc_maxd = 0;
  c->n_f = 1;
  c->m_f = d;
  c->n_vis = 1;
  c->m_vis = d;
  c->acc_n = c->acc_m = 0;
  for (int k = 0; k < KS; ++k) c->tot[k] = 0;
  c->tile_ticket = 0;
  c->finished = 0;
}

// The first kernel of a traversal: depths unreached but depth[src] = 0,
// parents -1 but parent[src] = src, the visited and frontier-0 bitmaps holding
// src alone, hub tables clear, and the loop state (one thread). The level
// kernels are instantiated for int32 depths and for the reference's byte
// depths (DT = uint8_t: written directly, no conversion pass).
template <class DT>
__global__ void __launch_bounds__(BT) k_reset(LevelArgs a, int32_t src, DT* depth, int32_t* parent) {
  const int64_t tid = blockIdx.x * (int64_t)BT + threadIdx.x, nth = (int64_t)gridDim.x * BT;
  if (tid == 0) init_state(a, src, depth, parent);
  fill_unreached(depth, a.V, tid, nth, src);
  if (parent) fill_neg1(parent, a.V, tid, nth, src, src);
  const int64_t W = (a.V + 31) >> 5, sw = src >> 5;
  const uint32_t sb = 1u << (src & 31);
  for (int64_t i = tid; i < W; i += nth) {
    const uint32_t x = i == sw ? sb : 0u;
    a.vis[i] = x;
    a.fb[0][i] = x;
    a.fb[1][i] = 0;
  }
  for (int64_t i = tid; i < a.hub_slots; i += nth) {
    a.hub[0][i] = 0;
    a.hub[1][i] = 0;
  }
}

// ------------------------------------------------------------ top-down ----
template <class DT>
__device__ __forceinline__ void td_visit(const LevelArgs& a, BfsCtl* c, int v, int u, bool valid, int ln,
                                         DT* depth, int32_t* parent, uint32_t* fbn) {
  bool mine = false;
  if (valid) {
    const uint32_t w = (uint32_t)v >> 5, b = 1u << (v & 31);
    if (!(ld_cg(a.vis + w) & b)) {
      const uint32_t old = atomicOr(a.vis + w, b);
      if (!(old & b)) {
        mine = true;
        depth[v] = (DT)ln;
        if (parent) parent[v] = u;
        red_or(fbn + w, b);
      }
    }
  }
  const unsigned m = __ballot_sync(FULL, mine);
  if (m) {
    const int lane = threadIdx.x & 31;
    const int leader = __ffs(m) - 1;
    int base = 0;
    if (lane == leader) base = atomicAdd(&c->n_raw, __popc(m));
    base = __shfl_sync(FULL, base, leader);
    if (mine) a.raw[base + __popc(m & lanemask_lt())] = v;
  }
}

template <class DT>
__device__ void td_expand(const LevelArgs& a, BfsCtl* c, int L, DT* depth, int32_t* parent) {
  const int qc = c->qcur;
  const int ns = c->n_q[0], nm = c->n_q[1], nl = c->n_q[2], nch = c->n_chunks;
  const int32_t* __restrict__ qs = a.q[qc][0];
  const int32_t* __restrict__ qm = a.q[qc][1];
  const int32_t* __restrict__ ql = a.q[qc][2];
  const int32_t* __restrict__ qch = a.qc[qc];
  uint32_t* fbn = a.fb[(L + 1) & 1];
  const int lane = threadIdx.x & 31;
  const int gw = (int)((blockIdx.x * (int64_t)BT + threadIdx.x) >> 5);
  const int nw = (int)(((int64_t)gridDim.x * BT) >> 5);
  const int ln = L + 1;

  // Large tier: one CTA per chunk of a high-degree vertex.
  __shared__ int s_vi;
  for (int ch = blockIdx.x; ch < nch; ch += gridDim.x) {
    if (threadIdx.x == 0) {
      int lo = 0, hi = nl - 1;
      while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (qch[mid] <= ch) lo = mid; else hi = mid - 1;
      }
      s_vi = lo;
    }
    __syncthreads();
    const int i = s_vi;
    __syncthreads();
    const int u = ql[i];
    const int64_t beg = a.off[u] + (int64_t)(ch - qch[i]) * a.chunk;
    const int64_t end = min(a.off[u + 1], beg + (int64_t)a.chunk);
    for (int64_t e0 = beg; e0 < end; e0 += BT) {
      const int64_t e = e0 + threadIdx.x;
      const bool valid = e < end;
      const int v = valid ? __ldg(a.adj + e) : 0;
      td_visit(a, c, v, u, valid, ln, depth, parent, fbn);
    }
  }
  // Mid tier: one warp per vertex.
  for (int i = gw; i < nm; i += nw) {
    const int u = qm[i];
    const int64_t beg = a.off[u], end = a.off[u + 1];
    for (int64_t e0 = beg; e0 < end; e0 += 32) {
      const int64_t e = e0 + lane;
      const bool valid = e < end;
      const int v = valid ? __ldg(a.adj + e) : 0;
      td_visit(a, c, v, u, valid, ln, depth, parent, fbn);
    }
  }
  // Small tier: a warp gathers the adjacency lists of 32 vertices and
  // processes the concatenation 32 edges at a time.
  for (int base = gw * 32; base < ns; base += nw * 32) {
    const int i = base + lane;
    int u = -1, d = 0;
    int64_t st = 0;
    if (i < ns) {
      u = qs[i];
      st = a.off[u];
      d = (int)(a.off[u + 1] - st);
    }
    int incl = d;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(FULL, incl, o);
      if (lane >= o) incl += y;
    }
    const int total = __shfl_sync(FULL, incl, 31);
    const int excl = incl - d;
    for (int r = 0; r < total; r += 32) {
      const int k = r + lane;
      const bool valid = k < total;
      int j = 0;
#pragma unroll
      for (int step = 16; step > 0; step >>= 1) {
        const int cand = j + step;
        const int ev = __shfl_sync(FULL, excl, cand & 31);
        if (cand < 32 && ev <= k) j = cand;
      }
      const int64_t sj = __shfl_sync(FULL, st, j);
      const int ej = __shfl_sync(FULL, excl, j);
      const int uj = __shfl_sync(FULL, u, j);
      const int v = valid ? __ldg(a.adj + sj + (k - ej)) : 0;
      td_visit(a, c, v, uj, valid, ln, depth, parent, fbn);
    }
  }
}

// ----------------------------------------------------------- bottom-up ----
struct Front {
  const uint32_t* fb;
  const int32_t* hub;
  int hub_slots, shift;
  __device__ __forceinline__ bool operator()(int u) const {
    if (hub_slots && hub[hub_slot((uint32_t)u, shift)] == u) return true;
    return (__ldg(fb + (u >> 5)) >> (u & 31)) & 1u;
  }
};

template <class DT>
__device__ void bu_expand(const LevelArgs& a, BfsCtl* c, int L, DT* depth, int32_t* parent, int32_t* s_hub,
                          unsigned long long* s_red) {
  const uint32_t* fbc = a.fb[L & 1];
  uint32_t* fbn = a.fb[(L + 1) & 1];
  unsigned long long* hub_next = a.hub[(L + 1) & 1];
  if (a.hub_slots) {
    const unsigned long long* ht = a.hub[L & 1];
    for (int i = threadIdx.x; i < a.hub_slots; i += BT) {
      const unsigned long long key = ht[i];
      s_hub[i] = key ? (int)(uint32_t)key : -1;
    }
  }
  // listing levels: this CTA's finds, appended to raw once at the end
  __shared__ uint32_t s_lcnt, s_lbase, s_listing;
  __shared__ int32_t s_list[LCAP];
  if (threadIdx.x == 0) {
    s_lcnt = 0;
    s_listing = c->bu_list;  // read from shared memory where needed: no register held in the loop
  }
  __syncthreads();
  const Front is_front{fbc, s_hub, a.hub_slots, a.hub_shift};
  const int lane = threadIdx.x & 31;
  const int64_t gtid = blockIdx.x * (int64_t)BT + threadIdx.x, nth = (int64_t)gridDim.x * BT;
  const int64_t gw = gtid >> 5, nw = nth >> 5;
  const int ln = L + 1;
  const int64_t W = (a.V + 31) >> 5;
  unsigned long long my_n = 0, my_m = 0;
  // A warp owns one status word: 32 consecutive vertex ids.
  for (int64_t wi = gw; wi < W; wi += nw) {
    const uint32_t todo_mask = a.active[wi] & ~a.vis[wi];
    if (!todo_mask) continue;
    const int64_t v = wi * 32 + lane;
    const bool todo = (todo_mask >> lane) & 1u;
    int64_t e0 = 0;
    int d = 0;
    bool found = false;
    int pu = -1;
    int4 ld = make_int4(-1, -1, -1, -1);
    if (todo) {
      // The lead neighbour (the highest-degree one) is the parent of most
      // vertices found: the first 4 neighbours are read coalesced, beside the
      // row offsets, and the first is probed before anything else, whatever
      // the vertex's degree.
      ld = __ldg(a.lead + v);
      e0 = a.off[v];
      d = (int)(a.off[v + 1] - e0);
      if (is_front(ld.x)) { found = true; pu = ld.x; }
    }
    if (todo && !found && d > 1) {
      // then the other three together
      const bool f1 = is_front(ld.y), f2 = ld.z >= 0 && is_front(ld.z), f3 = ld.w >= 0 && is_front(ld.w);
      if (f1) found = true, pu = ld.y;
      else if (f2) found = true, pu = ld.z;
      else if (f3) found = true, pu = ld.w;
    }
    if (todo && !found && d < a.small_max) {
      // A light vertex that keeps scanning is usually not adjacent to the
      // frontier at all: it checks BU_ILP neighbours per step, their reads
      // and then their frontier probes in flight together.
      for (int k = 4; k < d && !found; k += BU_ILP) {
        int u[BU_ILP];
        bool f[BU_ILP];
#pragma unroll
        for (int i = 0; i < BU_ILP; ++i) u[i] = k + i < d ? __ldg(a.adj + e0 + k + i) : -1;
#pragma unroll
        for (int i = 0; i < BU_ILP; ++i) f[i] = u[i] >= 0 && is_front(u[i]);
#pragma unroll
        for (int i = 0; i < BU_ILP; ++i)
          if (!found && f[i]) { found = true; pu = u[i]; }
      }
    }
    unsigned heavy = __ballot_sync(FULL, todo && !found && d >= a.small_max);
    while (heavy) {
      const int j = __ffs(heavy) - 1;
      heavy &= heavy - 1;
      const int64_t beg = __shfl_sync(FULL, e0, j);
      const int64_t end = beg + __shfl_sync(FULL, d, j);
      int hit = -1;
      for (int64_t b0 = beg; b0 < end; b0 += 32) {
        const int64_t e = b0 + lane;
        const int u = e < end ? __ldg(a.adj + e) : -1;
        const unsigned hm = __ballot_sync(FULL, e < end && is_front(u));
        if (hm) { hit = __shfl_sync(FULL, u, __ffs(hm) - 1); break; }
      }
      if (lane == j && hit >= 0) { found = true; pu = hit; }
    }
    if (found) {
      depth[v] = (DT)ln;
      if (parent) parent[v] = pu;
      my_n++;
      my_m += (unsigned long long)d;
      hub_insert(a, hub_next, (int)v, d);
    }
    const unsigned fm = __ballot_sync(FULL, found);
    if (lane == 0 && fm) {
      // this warp is the only writer of word wi during the level
      a.vis[wi] = a.vis[wi] | fm;
      fbn[wi] = fm;
    }
  }
  if (s_listing) {
    // List this CTA's finds: re-read the next-frontier words its warps wrote
    // (kept out of the loop above, which runs at its register limit). Lane 0
    // wrote them: the warp barrier orders those stores before these loads.
    __syncwarp();
    for (int64_t w0 = gw; w0 < W; w0 += nw * 32) {
      const int64_t wl = w0 + (int64_t)lane * nw;
      const uint32_t fw = wl < W ? __ldcg(fbn + wl) : 0u;
      unsigned any_w = __ballot_sync(FULL, fw != 0);
      while (any_w) {
        const int j = __ffs(any_w) - 1;
        any_w &= any_w - 1;
        const uint32_t fm = __shfl_sync(FULL, fw, j);
        const int64_t wj = w0 + (int64_t)j * nw;
        uint32_t p = 0;
        if (lane == 0) p = atomicAdd(&s_lcnt, (uint32_t)__popc(fm));
        p = __shfl_sync(FULL, p, 0) + __popc(fm & lanemask_lt());
        if (((fm >> lane) & 1u) && p < (uint32_t)LCAP) s_list[p] = (int32_t)(wj * 32 + lane);
      }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      const uint32_t n = s_lcnt;
      s_lbase = 0;
      if (n > (uint32_t)LCAP) c->list_over = 1;
      else if (n) s_lbase = (uint32_t)atomicAdd(&c->n_raw, (int)n);
    }
    __syncthreads();
    if (s_lcnt <= (uint32_t)LCAP)
      for (uint32_t i = threadIdx.x; i < s_lcnt; i += BT) a.raw[s_lbase + i] = s_list[i];
  }
  const int any = __syncthreads_or(my_n != 0);
  if (any) {
    unsigned long long r = block_sum(my_n, s_red);
    if (threadIdx.x == 0) atomicAdd(&c->acc_n, r);
    r = block_sum(my_m, s_red);
    if (threadIdx.x == 0) atomicAdd(&c->acc_m, r);
  }
}

template <class DT>
__global__ void __launch_bounds__(BT, 8) k_expand(LevelArgs a) {
  extern __shared__ int32_t s_hub[];
  __shared__ unsigned long long s_red[BT / 32];
  BfsCtl* c = a.ctl;
  if (c->done || c->skip) return;
  const int L = c->level;
  DT* depth = reinterpret_cast<DT*>(c->depth);
  if (c->dir == TD) td_expand(a, c, L, depth, c->parent);
  else bu_expand(a, c, L, depth, c->parent, s_hub, s_red);
}

// ----------------------------------------------------------- inspector ----
// Reads the items of one tile in blocked order: thread t owns items
// [t*IPT, t*IPT+IPT) of the tile, so per-thread output order = input order.
__device__ __forceinline__ void load_tile(const int32_t* src, int64_t first, int64_t n, int32_t (&v)[IPT]) {
  const int64_t i0 = first + (int64_t)threadIdx.x * IPT;
  if (i0 + IPT <= n && ((((uintptr_t)(src + i0)) & 15) == 0)) {
    const int4 x = *reinterpret_cast<const int4*>(src + i0);
    v[0] = x.x; v[1] = x.y; v[2] = x.z; v[3] = x.w;
  } else {
#pragma unroll
    for (int j = 0; j < IPT; ++j) v[j] = (i0 + j < n) ? src[i0 + j] : -1;
  }
}

__device__ __forceinline__ uint32_t acquire_tile(BfsCtl* c, uint32_t* s_tile) {
  if (threadIdx.x == 0) *s_tile = atomicAdd(&c->tile_ticket, 1u);
  __syncthreads();
  const uint32_t t = *s_tile;
  __syncthreads();
  return t;
}

// Appends one classified vertex to the next TD queues.
struct QueueOut {
  int32_t* q[3];
  int32_t* qc;
  __device__ __forceinline__ void put(const LevelArgs& a, int v, int cl, int d, uint32_t (&pos)[4]) const {
    q[cl][pos[cl]++] = v;
    if (cl == 2) {
      qc[pos[2] - 1] = (int32_t)pos[3];
      pos[3] += n_chunks_of(d, a);
    }
  }
};

__global__ void __launch_bounds__(BT) k_inspect(LevelArgs a) {
  __shared__ uint32_t s_scan[32 * KS];
  __shared__ uint32_t s_excl[KS];
  __shared__ uint32_t s_tile;
  __shared__ int s_last;
  __shared__ unsigned long long s_red[BT / 32];
  __shared__ uint32_t s_redu[BT / 32];
  BfsCtl* c = a.ctl;
  if (c->done) {  // never leave the while node spinning on a finished traversal
    if (blockIdx.x == 0 && threadIdx.x == 0) {
      c->iters = c->iters + 1;
      if (a.use_cond) {
        cudaGraphSetConditional(a.cond, 0u);
      }
    }
    return;
  }
  const int L = c->level, dir = c->dir;
  const uint32_t epoch = c->epoch;
  const int qcur = c->qcur;
  const int64_t gtid = blockIdx.x * (int64_t)BT + threadIdx.x, nth = (int64_t)gridDim.x * BT;
  int* err = &c->err;
  const QueueOut qo{{a.q[qcur ^ 1][0], a.q[qcur ^ 1][1], a.q[qcur ^ 1][2]}, a.qc[qcur ^ 1]};
  // The hub table of frontier L was read by expand(L): clear it for level L+2.
  if (a.hub_slots) {
    unsigned long long* hd = a.hub[L & 1];
    for (int64_t i = gtid; i < a.hub_slots; i += nth) hd[i] = 0;
  }
  uint32_t* fbo = a.fb[L & 1];
  const uint32_t* fbn = a.fb[(L + 1) & 1];
  unsigned long long my_m = 0;
  uint32_t my_maxd = 0;
  bool to_td = false;

  if (dir == TD) {
    // Frontier L is dead: zero its words in fb[L&1] (touching only its vertices).
    for (int k = 0; k < 3; ++k) {
      const int32_t* qk = a.q[qcur][k];
      for (int64_t i = gtid; i < c->n_q[k]; i += nth) fbo[(uint32_t)qk[i] >> 5] = 0;
    }
    // Classify the raw next frontier into q[qcur^1].
    const int64_t n = c->n_raw;
    const uint32_t ntiles = (uint32_t)((n + TILE - 1) / TILE);
    unsigned long long* hub_next = a.hub[(L + 1) & 1];
    while (true) {
      const uint32_t tile = acquire_tile(c, &s_tile);
      if (tile >= ntiles) break;
      int32_t v[IPT];
      load_tile(a.raw, (int64_t)tile * TILE, n, v);
      int dg[IPT], cl[IPT];
      uint32_t cnt[4] = {0, 0, 0, 0};
#pragma unroll
      for (int j = 0; j < IPT; ++j) {
        dg[j] = v[j] >= 0 ? a.deg[v[j]] : 0;
        cl[j] = v[j] >= 0 ? cls_of(dg[j], a) : -1;
        if (cl[j] >= 0) {
          cnt[cl[j]]++;
          my_m += dg[j];
          my_maxd = max(my_maxd, (uint32_t)dg[j]);
          hub_insert(a, hub_next, v[j], dg[j]);
          if (cl[j] == 2) cnt[3] += n_chunks_of(dg[j], a);
        }
      }
      uint32_t pre[4] = {cnt[0], cnt[1], cnt[2], cnt[3]}, agg[4], excl[4];
      block_excl_scan<4>(pre, agg, s_scan);
      lookback<4, KS>(a.tiles, tile, epoch, agg, excl, s_excl, err, a.fault_inject != 0);
      uint32_t pos[4];
#pragma unroll
      for (int k = 0; k < 4; ++k) pos[k] = excl[k] + pre[k];
#pragma unroll
      for (int j = 0; j < IPT; ++j)
        if (cl[j] >= 0) qo.put(a, v[j], cl[j], dg[j], pos);
      if (tile == ntiles - 1 && threadIdx.x == 0) {
        for (int k = 0; k < 4; ++k) c->tot[k] = excl[k] + agg[k];
        __threadfence();
      }
    }
  } else {
    // BU level done: the expander counted the new frontier in acc_n/acc_m.
    const int64_t n_next = (int64_t)c->acc_n;
    to_td = a.policy == ENT_POLICY_BEAMER && n_next > 0 && (double)n_next < (double)a.V / a.beta &&
            n_next < c->n_f;
    const int64_t W = (a.V + 31) >> 5;
    for (int64_t i = gtid; i < W; i += nth) fbo[i] = 0;
    if (to_td && c->bu_list && !c->list_over) {
      // Hand over to TD from the list the expander made: classify raw (its
      // vertices in the order the CTAs listed them) into q[qcur^1].
      const int64_t n = c->n_raw;
      const uint32_t ntiles = (uint32_t)((n + TILE - 1) / TILE);
      while (true) {
        const uint32_t tile = acquire_tile(c, &s_tile);
        if (tile >= ntiles) break;
        int32_t v[IPT];
        load_tile(a.raw, (int64_t)tile * TILE, n, v);
        int dg[IPT], cl[IPT];
        uint32_t cnt[4] = {0, 0, 0, 0};
#pragma unroll
        for (int j = 0; j < IPT; ++j) {
          dg[j] = v[j] >= 0 ? a.deg[v[j]] : 0;
          cl[j] = v[j] >= 0 ? cls_of(dg[j], a) : -1;
          if (cl[j] >= 0) {
            cnt[cl[j]]++;
            my_maxd = max(my_maxd, (uint32_t)dg[j]);
            if (cl[j] == 2) cnt[3] += n_chunks_of(dg[j], a);
          }
        }
        uint32_t pre[4] = {cnt[0], cnt[1], cnt[2], cnt[3]}, agg[4], excl[4];
        block_excl_scan<4>(pre, agg, s_scan);
        lookback<4, KS>(a.tiles, tile, epoch, agg, excl, s_excl, err, a.fault_inject != 0);
        uint32_t pos[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) pos[k] = excl[k] + pre[k];
#pragma unroll
        for (int j = 0; j < IPT; ++j)
          if (cl[j] >= 0) qo.put(a, v[j], cl[j], dg[j], pos);
        if (tile == ntiles - 1 && threadIdx.x == 0) {
          for (int k = 0; k < 4; ++k) c->tot[k] = excl[k] + agg[k];
          __threadfence();
        }
      }
    } else if (to_td) {
      // Hand over to TD: classify the frontier bitmap (ascending ids) into
      // q[qcur^1]. A tile is BT*WPT words, WPT consecutive words per thread
      // (the frontier is sparse here: few look-back tiles, not few words).
      const uint32_t ntiles = (uint32_t)((W + BT * WPT - 1) / (BT * WPT));
      while (true) {
        const uint32_t tile = acquire_tile(c, &s_tile);
        if (tile >= ntiles) break;
        const int64_t w_first = ((int64_t)tile * BT + threadIdx.x) * WPT;
        uint32_t wd[WPT];
        if (w_first + WPT <= W) {  // 32-byte aligned: the slab is 256-byte aligned, w_first % 8 == 0
          const uint4 x = __ldcg(reinterpret_cast<const uint4*>(fbn + w_first));
          const uint4 y = __ldcg(reinterpret_cast<const uint4*>(fbn + w_first) + 1);
          wd[0] = x.x; wd[1] = x.y; wd[2] = x.z; wd[3] = x.w;
          wd[4] = y.x; wd[5] = y.y; wd[6] = y.z; wd[7] = y.w;
        } else {
#pragma unroll
          for (int j = 0; j < WPT; ++j) wd[j] = w_first + j < W ? ld_cg(fbn + w_first + j) : 0u;
        }
        uint32_t cnt[4] = {0, 0, 0, 0};
#pragma unroll
        for (int j = 0; j < WPT; ++j) {
          const int64_t wi = w_first + j;
          for (uint32_t m = wd[j]; m; m &= m - 1) {
            const int v = (int)(wi * 32 + __ffs(m) - 1);
            const int d = a.deg[v];
            const int cl = cls_of(d, a);
            my_maxd = max(my_maxd, (uint32_t)d);
            cnt[cl]++;
            if (cl == 2) cnt[3] += n_chunks_of(d, a);
          }
        }
        uint32_t pre[4] = {cnt[0], cnt[1], cnt[2], cnt[3]}, agg[4], excl[4];
        block_excl_scan<4>(pre, agg, s_scan);
        lookback<4, KS>(a.tiles, tile, epoch, agg, excl, s_excl, err, a.fault_inject != 0);
        uint32_t pos[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) pos[k] = excl[k] + pre[k];
#pragma unroll
        for (int j = 0; j < WPT; ++j) {
          const int64_t wi = w_first + j;
          for (uint32_t m = wd[j]; m; m &= m - 1) {
            const int v = (int)(wi * 32 + __ffs(m) - 1);
            const int d = a.deg[v];
            qo.put(a, v, cls_of(d, a), d, pos);
          }
        }
        if (tile == ntiles - 1 && threadIdx.x == 0) {
          for (int k = 0; k < 4; ++k) c->tot[k] = excl[k] + agg[k];
          __threadfence();
        }
      }
    }
  }

  // Publish this CTA's counters, then the last CTA to finish runs the policy.
  if (dir == TD && __syncthreads_or(my_m != 0)) {
    const unsigned long long r = block_sum(my_m, s_red);
    if (threadIdx.x == 0) atomicAdd(&c->acc_m, r);
  }
  if (a.narrow_f > 0 && __syncthreads_or(my_maxd != 0)) {
    const uint32_t r = block_max(my_maxd, s_redu);
    if (threadIdx.x == 0 && r > ld_cg(&c->acc_maxd)) atomicMax(&c->acc_maxd, r);
  }
  if (threadIdx.x == 0) {
    __threadfence();
    s_last = atomicAdd(&c->finished, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!s_last || threadIdx.x != 0) return;
  __threadfence();
  // Every counter the policy needs is loaded at once (independent L2 loads in
  // flight together), the decision is made in registers, then all is stored:
  // the finisher is on the critical path of every level.
  const auto ld64 = [](const void* p) { return (int64_t)__ldcg(reinterpret_cast<const long long*>(p)); };
  const int32_t n_raw = __ldcg(&c->n_raw), err0 = __ldcg(&c->err), it0 = __ldcg(&c->iters);
  const int32_t tdl = __ldcg(&c->td_levels), bul = __ldcg(&c->bu_levels);
  const int64_t acc_n = ld64(&c->acc_n), acc_m = ld64(&c->acc_m);
  const int64_t n_vis0 = ld64(&c->n_vis), m_vis0 = ld64(&c->m_vis), n_f0 = ld64(&c->n_f);
  const uint32_t maxd = __ldcg(&c->acc_maxd);
  uint32_t tot[KS];
#pragma unroll
  for (int k = 0; k < KS; ++k) tot[k] = __ldcg(&c->tot[k]);
  const int64_t n_next = dir == TD ? (int64_t)n_raw : acc_n;
  const int64_t m_next = acc_m;
  int next_dir = dir;
  bool new_queues = false;
  if (dir == TD) {
    new_queues = true;
    const double m_u = (double)(a.E - (m_vis0 + m_next));
    if (a.policy == ENT_POLICY_BEAMER && (double)m_next > m_u / a.alpha) next_dir = BU;
    if (a.policy == ENT_POLICY_REFERENCE && (double)m_next >= a.ref_ratio * (double)a.E) next_dir = BU;
    if (a.policy == ENT_POLICY_BU_ONLY) next_dir = BU;
  } else if (to_td) {
    next_dir = TD;
    new_queues = true;
  }
  const int64_t n_vis1 = n_vis0 + n_next;
  int done = n_next == 0;
  int err1 = err0;
  if (L + 1 >= a.max_levels && !done) {
    err1 |= 4;
    done = 1;
  }
  if (n_vis1 > a.V) {  // a vertex counted twice: stop instead of looping on
    err1 |= 8;
    done = 1;
  }
  // A look-back wait ran out (bit 2): the positions of this classification
  // came from partial prefixes, so its queues and chunk offsets are not
  // consistent. Stop here: no kernel may expand them.
  if (err1 & 2) done = 1;
  // Small-frontier mode for the next level (top-down only).
  const int narrow = !done && next_dir == TD && a.narrow_f > 0 && n_next <= a.narrow_f &&
                     m_next <= a.narrow_m && (int64_t)maxd <= a.narrow_deg;
  if (dir == TD) c->td_levels = tdl + 1;
  else c->bu_levels = bul + 1;
  if (new_queues) {
    c->qcur = qcur ^ 1;
    for (int k = 0; k < 3; ++k) c->n_q[k] = (int32_t)tot[k];
    c->n_chunks = (int32_t)tot[3];
  }
  c->n_vis = n_vis1;
  c->m_vis = m_vis0 + m_next;
  c->n_f = n_next;
  c->m_f = m_next;
  c->dir = next_dir;
  c->level = L + 1;
  c->err = err1;
  c->done = done;
  c->narrow = narrow;
  // A bottom-up level on a shrinking frontier usually finds few vertices and
  // then hands over to top-down: it also lists them, so the inspector need not
  // scan the frontier bitmap to classify them.
  c->bu_list = !done && next_dir == BU && a.policy == ENT_POLICY_BEAMER && n_next < n_f0;
  c->list_over = 0;
  c->skip = 0;
  c->acc_maxd = 0;
  c->iters = it0 + 1;
  c->n_raw = 0;
  c->acc_n = 0;
  c->acc_m = 0;
  for (int k = 0; k < KS; ++k) c->tot[k] = 0;
  c->tile_ticket = 0;
  c->finished = 0;
  c->epoch = epoch + 1;
  __threadfence();
  if (a.use_cond) {
    cudaGraphSetConditional(a.cond, done ? 0u : 1u);
  }
}

// ------------------------------------------------------ small frontier ----
namespace cg = cooperative_groups;

// A small-frontier queue entry: vertex, degree, row start (16 bytes).
__device__ __forceinline__ int4 nentry(int v, int d, int64_t st) {
  return make_int4(v, d, (int)(uint32_t)st, (int)(uint32_t)((uint64_t)st >> 32));
}

__device__ __forceinline__ void cluster_arrive_relaxed() {
  asm volatile("barrier.cluster.arrive.relaxed.aligned;" ::: "memory");
}
__device__ __forceinline__ void cluster_wait() { asm volatile("barrier.cluster.wait.aligned;" ::: "memory"); }
__device__ __forceinline__ void fence_cluster() { asm volatile("fence.acq_rel.cluster;" ::: "memory"); }
// Named CTA barrier 1 between the expansion warps (arrive) and the coordinator (sync).
__device__ __forceinline__ void bar1_arrive() { asm volatile("bar.arrive 1, %0;" ::"r"(NT) : "memory"); }
__device__ __forceinline__ void bar1_sync() { asm volatile("bar.sync 1, %0;" ::"r"(NT) : "memory"); }

struct NarrowOut {
  int4* q;                   // this CTA's next-frontier buffer
  uint32_t* cnt;             // its append counter (may pass NQCAP: the rest spills)
  unsigned long long* msum;  // degree sum of the appended vertices
  uint32_t* flag;            // NF_HEAVY | NF_SPILL
  int32_t* spill;            // global overflow list
};

// Appends the vertices this warp claimed (mine) to the CTA's next frontier.
__device__ __forceinline__ void narrow_append(const LevelArgs& a, BfsCtl* c, bool mine, int v, int vd, int64_t vst,
                                              const NarrowOut& o) {
  const unsigned m = __ballot_sync(FULL, mine);
  if (!m) return;
  const int lane = threadIdx.x & 31, leader = __ffs(m) - 1;
  uint32_t base = 0;
  if (lane == leader) base = atomicAdd(o.cnt, (uint32_t)__popc(m));
  base = __shfl_sync(FULL, base, leader);
  const unsigned wsum = __reduce_add_sync(FULL, mine ? (unsigned)vd : 0u);
  const bool heavy = __any_sync(FULL, mine && vd > a.narrow_deg);
  if (lane == leader) {
    atomicAdd(o.msum, (unsigned long long)wsum);
    if (heavy) atomicOr(o.flag, NF_HEAVY);
  }
  if (mine) {
    const uint32_t pos = base + __popc(m & lanemask_lt());
    if (pos < (uint32_t)NQCAP) {
      o.q[pos] = nentry(v, vd, vst);
    } else {
      o.spill[atomicAdd(&c->n_spill, 1u)] = v;
      __threadfence();  // read by other CTAs after the (relaxed) cluster barrier
      atomicOr(o.flag, NF_SPILL);
    }
  }
}

// Runs top-down levels of a small frontier inside one launch of one cluster
// (grid = one cluster of nc CTAs). Entered with frontier L0 classified in
// q[qcur] (the state the inspector leaves). Leaves either
//  * done (frontier empty or level limit), or
//  * the state the top-down expander leaves after level Lx-1: frontier Lx in
//    raw[0, n_raw) with its bits in fb[Lx & 1], and `skip` set so that the
//    expander of the next loop iteration does nothing and the inspector
//    classifies raw as usual.
//
// A CTA is NWE expansion warps plus one coordinator warp. Per level:
//  * every warp reads the cluster-wide counts of the frontier from its own
//    shared memory (lane r: CTA r's count) and takes the same exit decision;
//  * expansion warp gw takes k consecutive entries of the cluster-wide
//    frontier (CTA r's entries follow those of CTAs < r; read through
//    distributed shared memory) and walks their concatenated rows, up to
//    NROUND rounds of 32 edges with all loads and claims in flight together.
//    The claim is an atomicOr on the visited bitmap without a probe first,
//    with the claimed vertex's row read beside it, so a level costs one
//    adjacency read and one claim on its critical path;
//  * expansion warps signal the coordinator (named barrier, no wait) and
//    arrive at the cluster barrier relaxed: their global stores (depths) are
//    only read after the kernel, so they never wait for them to drain;
//  * the coordinator pushes its CTA's counts into every CTA's r_* arrays
//    (double-buffered by level parity: a slow CTA may still use the previous
//    level's while a fast one pushes the next), fences at cluster scope
//    (releasing those and, through the named barrier, the expansion warps'
//    shared-memory entries) and arrives.
// Every CTA takes the same decisions from the same counts, so all reach the
// same barriers; there are no spin waits.
template <class DT>
__global__ void __launch_bounds__(NT, 1) k_narrow(LevelArgs a) {
  extern __shared__ int4 s_q[];  // [2][NQCAP]
  __shared__ uint32_t s_cnt[2], s_flag[2];
  __shared__ unsigned long long s_m[2];
  __shared__ uint32_t r_cnt[2][NC_MAX], r_flag[2][NC_MAX];
  __shared__ unsigned long long r_m[2][NC_MAX];
  cg::cluster_group cl = cg::this_cluster();
  BfsCtl* c = a.ctl;
  if (blockIdx.x == 0 && threadIdx.x == 0) c->narrow_calls = c->narrow_calls + 1;
  if (c->done || !c->narrow) return;  // same value in every CTA
  const int nc = (int)cl.num_blocks(), rank = (int)cl.block_rank();
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const bool coord = warp == NWE;
  const int gw = rank * NWE + warp, nwt = nc * NWE;
  DT* depth = reinterpret_cast<DT*>(c->depth);
  int32_t* parent = c->parent;
  const int L0 = c->level;
  const int qcur = c->qcur;
  int32_t* spill = a.q[qcur ^ 1][0];

  // Entry: each CTA loads a slice of frontier L0 (with its rows) into buffer 0
  // and clears the frontier's bits (nothing reads them during the run).
  {
    const int n0 = c->n_q[0], n1 = c->n_q[1], n2 = c->n_q[2];
    const int N0 = n0 + n1 + n2;
    const int lo = (int)((int64_t)N0 * rank / nc), hi = (int)((int64_t)N0 * (rank + 1) / nc);
    uint32_t* fbo = a.fb[L0 & 1];
    for (int i = lo + tid; i < hi; i += NT) {
      const int u = i < n0 ? a.q[qcur][0][i] : (i < n0 + n1 ? a.q[qcur][1][i - n0] : a.q[qcur][2][i - n0 - n1]);
      const int64_t st = a.off[u];
      s_q[i - lo] = nentry(u, (int)(a.off[u + 1] - st), st);
      fbo[(uint32_t)u >> 5] = 0;
    }
    // the hub table of frontier L0 would be stale for a later bottom-up level
    if (a.hub_slots)
      for (int i = rank * NT + tid; i < a.hub_slots; i += nc * NT) a.hub[L0 & 1][i] = 0;
    // every CTA knows every slice size: no push needed for frontier L0
    if (tid < nc) {
      r_cnt[0][tid] = (uint32_t)((int64_t)N0 * (tid + 1) / nc - (int64_t)N0 * tid / nc);
      r_m[0][tid] = 0;
      r_flag[0][tid] = 0;
    }
    if (tid == 0) {
      s_cnt[1] = 0;
      s_m[1] = 0;
      s_flag[1] = 0;
    }
  }
  cl.sync();

  unsigned long long n_vis = (unsigned long long)c->n_vis, m_vis = (unsigned long long)c->m_vis;
  int64_t nf_last = c->n_f, mf_last = c->m_f;
  int L = L0;
  int outcome = 0;  // 1 frontier empty, 2 hand over, 3 level limit
  uint32_t n_all = 0;
  for (int it = 0;; ++it) {
    const int cur = it & 1, nxt = cur ^ 1;
    // Counts of frontier L: lane r holds CTA r's; `incl` is their inclusive
    // prefix, i.e. the end of CTA r's entries in the cluster-wide order.
    uint32_t incl = lane < nc ? r_cnt[cur][lane] : 0u;
    unsigned long long m_all = lane < nc ? r_m[cur][lane] : 0ull;
    const uint32_t flags = __reduce_or_sync(FULL, lane < nc ? r_flag[cur][lane] : 0u);
#pragma unroll
    for (int ofs = 1; ofs < 32; ofs <<= 1) {
      const uint32_t y = __shfl_up_sync(FULL, incl, ofs);
      if (lane >= ofs) incl += y;
      m_all += __shfl_xor_sync(FULL, m_all, ofs);
    }
    n_all = __shfl_sync(FULL, incl, 31);
    if (n_all == 0) outcome = 1;
    else if (it > 0 && (flags || n_all > (uint32_t)a.exit_f || (int64_t)m_all > a.exit_m)) outcome = 2;
    else if (L + 1 >= a.max_levels) outcome = 3;
    if (outcome) break;
    if (it > 0) {
      n_vis += n_all;
      m_vis += m_all;
      nf_last = n_all;
      mf_last = (int64_t)m_all;
    }

    if (!coord) {
      const NarrowOut o{s_q + nxt * NQCAP, &s_cnt[nxt], &s_m[nxt], &s_flag[nxt], spill};
      const int ln = L + 1;
      int k = (int)((n_all + nwt - 1) / nwt);
      if (k > 32) k = 32;
      for (int first = gw * k; first < (int)n_all; first += nwt * k) {
        const int i = first + lane;
        // owner CTA of entry i: the number of CTAs whose entries end at or before i
        int r = 0;
#pragma unroll
        for (int step = NC_MAX / 2; step > 0; step >>= 1) {
          const uint32_t e_end = __shfl_sync(FULL, incl, r + step - 1);
          if (r + step <= nc - 1 && (uint32_t)i >= e_end) r += step;
        }
        const uint32_t base = __shfl_sync(FULL, incl, (r + 31) & 31);  // end of CTA r-1 (unused for r = 0)
        int u = -1, d = 0;
        int64_t st = 0;
        if (lane < k && i < (int)n_all) {
          const int4 e = *(cl.map_shared_rank(s_q + cur * NQCAP, r) + (i - (r ? (int)base : 0)));
          u = e.x;
          d = e.y;
          st = (int64_t)(((uint64_t)(uint32_t)e.w << 32) | (uint32_t)e.z);
        }
        int dincl = d;
#pragma unroll
        for (int ofs = 1; ofs < 32; ofs <<= 1) {
          const int y = __shfl_up_sync(FULL, dincl, ofs);
          if (lane >= ofs) dincl += y;
        }
        const int total = __shfl_sync(FULL, dincl, 31);
        const int excl = dincl - d;
        for (int r0 = 0; r0 < total; r0 += 32 * NROUND) {
          int v[NROUND], uj[NROUND], vd[NROUND];
          int64_t vst[NROUND];
          bool mine[NROUND];
          // adjacency reads of up to NROUND rounds
#pragma unroll
          for (int q = 0; q < NROUND; ++q) {
            v[q] = -1;
            uj[q] = 0;
            if (r0 + 32 * q < total) {  // warp-uniform
              const int kk = r0 + 32 * q + lane;
              int j = 0;
#pragma unroll
              for (int step = 16; step > 0; step >>= 1) {
                const int cand = j + step;
                const int ev = __shfl_sync(FULL, excl, cand & 31);
                if (cand < 32 && ev <= kk) j = cand;
              }
              const int64_t sj = __shfl_sync(FULL, st, j);
              const int ej = __shfl_sync(FULL, excl, j);
              uj[q] = __shfl_sync(FULL, u, j);
              if (kk < total) v[q] = __ldg(a.adj + sj + (kk - ej));
            }
          }
          // claims, with each candidate's row read beside its claim
#pragma unroll
          for (int q = 0; q < NROUND; ++q) {
            mine[q] = false;
            vd[q] = 0;
            vst[q] = 0;
            if (v[q] >= 0) {
              const int x = v[q];
              const int64_t o0 = __ldg(a.off + x), o1 = __ldg(a.off + x + 1);
              const uint32_t b = 1u << (x & 31);
              const uint32_t old = atomicOr(a.vis + ((uint32_t)x >> 5), b);
              if (!(old & b)) {
                mine[q] = true;
                vst[q] = o0;
                vd[q] = (int)(o1 - o0);
                // the next level walks this row: start its first sector towards L2 now
                // (an empty row may start one past the array: nothing to fetch)
                if (o1 > o0) asm volatile("prefetch.global.L2 [%0];" ::"l"(a.adj + o0));
                depth[x] = (DT)ln;
                if (parent) parent[x] = uj[q];
              }
            }
          }
#pragma unroll
          for (int q = 0; q < NROUND; ++q)
            if (r0 + 32 * q < total) narrow_append(a, c, mine[q], v[q], vd[q], vst[q], o);
        }
      }
      bar1_arrive();  // this warp's appends are complete
      cluster_arrive_relaxed();
      cluster_wait();
    } else {
      bar1_sync();  // all expansion warps' appends to buffer nxt are complete
      if (lane < nc) {
        *cl.map_shared_rank(&r_cnt[nxt][rank], lane) = s_cnt[nxt];
        *cl.map_shared_rank(&r_m[nxt][rank], lane) = s_m[nxt];
        *cl.map_shared_rank(&r_flag[nxt][rank], lane) = s_flag[nxt];
      }
      __syncwarp();
      if (lane == 0) {  // buffer cur takes the appends of the next level
        s_cnt[cur] = 0;
        s_m[cur] = 0;
        s_flag[cur] = 0;
      }
      fence_cluster();
      cluster_arrive_relaxed();
      cluster_wait();
    }
    ++L;
  }
  cl.sync();  // no CTA leaves while another may still read its entries

  const int cur = (L - L0) & 1;
  if (outcome == 2) {
    // Hand over frontier L: this CTA's stored entries to raw[base, ...),
    // spilled ones after all stored entries; set their frontier bits.
    uint32_t base = 0, n_stored = 0;
    for (int r = 0; r < nc; ++r) {
      const uint32_t sr = min(r_cnt[cur][r], (uint32_t)NQCAP);
      if (r < rank) base += sr;
      n_stored += sr;
    }
    uint32_t* fbn = a.fb[L & 1];
    const uint32_t mine = min(r_cnt[cur][rank], (uint32_t)NQCAP);
    for (uint32_t j = tid; j < mine; j += NT) {
      const int v = s_q[cur * NQCAP + j].x;
      a.raw[base + j] = v;
      red_or(fbn + ((uint32_t)v >> 5), 1u << (v & 31));
    }
    for (uint32_t j = rank * NT + tid; j < n_all - n_stored; j += nc * NT) {
      const int v = __ldcg(spill + j);
      a.raw[n_stored + j] = v;
      red_or(fbn + ((uint32_t)v >> 5), 1u << (v & 31));
    }
  }
  if (rank != 0 || tid != 0) return;
  c->narrow_levels += L - L0;
  c->narrow_runs += 1;
  c->narrow = 0;
  c->n_spill = 0;
  c->n_vis = (int64_t)n_vis;
  c->m_vis = (int64_t)m_vis;
  if (outcome == 2) {
    c->level = L - 1;  // as if the expander had just run level L-1
    c->td_levels += L - 1 - L0;
    c->n_raw = (int32_t)n_all;
    for (int q = 0; q < 3; ++q) c->n_q[q] = 0;
    c->n_chunks = 0;
    c->n_f = nf_last;
    c->m_f = mf_last;
    c->acc_m = 0;
    c->skip = 1;
  } else {
    c->level = L;
    c->td_levels += L - L0;
    c->n_f = 0;
    c->m_f = 0;
    if (outcome == 3) c->err |= 4;
    c->done = 1;
  }
  __threadfence();
}

// Pulls a finished byte-depth row into L2 (kept there preferentially) before
// its copy to the host: the traversal wrote it as bytes scattered over all its
// levels, mostly evicted since, and the copy engine would otherwise read it
// from DRAM that the next traversal keeps busy (s24, 64 sources: 36.2 against
// 44.9 ms with every row copied; one prefetch per 128-byte line).
__global__ void __launch_bounds__(256) k_row_to_l2(const uint8_t* __restrict__ p, int64_t n) {
  const int64_t step = (int64_t)gridDim.x * blockDim.x * 128;
  for (int64_t i = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) * 128; i < n; i += step)
    asm volatile("prefetch.global.L2::evict_last [%0];" ::"l"(p + i));
}

// ------------------------------------------------------------- host -------
struct BfsWorkspace {
  int device = 0;
  int64_t V = 0;
  BfsCtl* ctl = nullptr;
  BfsCtl* ctl_h = nullptr;  // pinned mirror for stats
  int32_t* depth = nullptr;
  int32_t* parent = nullptr;
  void* slab = nullptr;     // one allocation for all level state
  LevelArgs args;
  int grid_reset = 0, grid_expand = 0, grid_inspect = 0;
  size_t smem_expand = 0;
  int narrow_nc = 0;        // CTAs of the small-frontier cluster (0: mode off)
  size_t smem_narrow = 0;
  // the traversal graph, [0] for int32 depths, [1] for byte depths (built on first use)
  cudaGraph_t graph[2] = {nullptr, nullptr};
  cudaGraphExec_t exec[2] = {nullptr, nullptr};
  cudaGraphNode_t reset_node[2] = {nullptr, nullptr};
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  // ent_bfs_many: a second depth buffer, a copy stream and pinned per-source
  // copies of the control block (created on first use)
  int32_t* depth_b = nullptr;
  uint8_t* depth8[2] = {nullptr, nullptr};  // byte depths (ent_bfs_many_u8)
  cudaStream_t copy_stream = nullptr;
  BfsCtl* many_ctl_h = nullptr;
  int32_t many_cap = 0;
  std::vector<cudaEvent_t> many_ev;          // [2i], [2i+1] bracket traversal i
  cudaEvent_t many_sync[3] = {nullptr, nullptr, nullptr};  // buffer 0 / 1 copied, byte row in L2
};

template <class DT>
constexpr int depth_kind() { return std::is_same<DT, uint8_t>::value ? 1 : 0; }

void destroy_bfs_workspace(BfsWorkspace* w) {
  if (!w) return;
  for (int k = 0; k < 2; ++k) {
    if (w->exec[k]) cudaGraphExecDestroy(w->exec[k]);
    if (w->graph[k]) cudaGraphDestroy(w->graph[k]);
  }
  if (w->slab) cudaFree(w->slab);
  if (w->ctl) cudaFree(w->ctl);
  if (w->ctl_h) cudaFreeHost(w->ctl_h);
  if (w->depth) cudaFree(w->depth);
  if (w->parent) cudaFree(w->parent);
  if (w->ev0) cudaEventDestroy(w->ev0);
  if (w->ev1) cudaEventDestroy(w->ev1);
  if (w->depth_b) cudaFree(w->depth_b);
  for (int i = 0; i < 2; ++i)
    if (w->depth8[i]) cudaFree(w->depth8[i]);
  if (w->copy_stream) cudaStreamDestroy(w->copy_stream);
  if (w->many_ctl_h) cudaFreeHost(w->many_ctl_h);
  for (cudaEvent_t e : w->many_ev) cudaEventDestroy(e);
  for (cudaEvent_t e : w->many_sync)
    if (e) cudaEventDestroy(e);
  delete w;
}

template <class DT>
static int build_graph(ent_graph* g, BfsWorkspace* w) {
  const int k = depth_kind<DT>();
  cudaGraph_t graph;
  ENT_CUDA(cudaGraphCreate(&graph, 0));
  w->graph[k] = graph;
  LevelArgs ra = w->args;
  ra.use_cond = 0;
  int32_t src0 = 0;
  DT* d0 = reinterpret_cast<DT*>(w->depth);  // placeholders: launch_graph sets each launch's
  int32_t* p0 = nullptr;
  void* rargs[4] = {&ra, &src0, &d0, &p0};
  cudaKernelNodeParams kp = {};
  kp.func = (void*)k_reset<DT>;
  kp.gridDim = dim3(w->grid_reset);
  kp.blockDim = dim3(BT);
  kp.sharedMemBytes = 0;
  kp.kernelParams = rargs;
  ENT_CUDA(cudaGraphAddKernelNode(&w->reset_node[k], graph, nullptr, 0, &kp));
  cudaGraphConditionalHandle handle;
  ENT_CUDA(cudaGraphConditionalHandleCreate(&handle, graph, 1, cudaGraphCondAssignDefault));
  cudaGraphNodeParams cp = {};
  cp.type = cudaGraphNodeTypeConditional;
  cp.conditional.handle = handle;
  cp.conditional.type = cudaGraphCondTypeWhile;
  cp.conditional.size = 1;
  cudaGraphNode_t cond_node;
  ENT_CUDA(cudaGraphAddNode(&cond_node, graph, &w->reset_node[k], 1, &cp));
  cudaGraph_t body = cp.conditional.phGraph_out[0];
  // Loop body: LOOP_UNROLL copies of expand -> inspect -> small-frontier
  // cluster, in a chain. Measured on B200 with trivial kernels: a kernel node
  // in a chain costs about 1.7 us, a while-node iteration about 5 us more, so
  // each copy after the first saves that iteration. Every level kernel treats
  // a finished traversal as a no-op (the inspector still counts its launch),
  // so copies after the one that finished only cost their launches.
  // The cluster kernel runs in every copy and leaves at once unless the
  // inspector chose the small-frontier mode (its first read; the same value
  // in every CTA): such a kernel costs less than an IF node that is not
  // taken (about 1.1 against 2.4 us per iteration).
  LevelArgs la = w->args;
  la.cond = handle;
  la.use_cond = 1;
  void* largs[1] = {&la};
  cudaGraphNode_t prev = nullptr;
  for (int u = 0; u < LOOP_UNROLL; ++u) {
    cudaKernelNodeParams bp = {};
    bp.func = (void*)k_expand<DT>;
    bp.gridDim = dim3(w->grid_expand);
    bp.blockDim = dim3(BT);
    bp.sharedMemBytes = (unsigned)w->smem_expand;
    bp.kernelParams = largs;
    cudaGraphNode_t n_expand, n_inspect;
    ENT_CUDA(cudaGraphAddKernelNode(&n_expand, body, prev ? &prev : nullptr, prev ? 1 : 0, &bp));
    bp.func = (void*)k_inspect;
    bp.gridDim = dim3(w->grid_inspect);
    bp.sharedMemBytes = 0;
    ENT_CUDA(cudaGraphAddKernelNode(&n_inspect, body, &n_expand, 1, &bp));
    prev = n_inspect;
    if (w->narrow_nc > 0) {
      cudaGraphNode_t n_narrow;
      bp.func = (void*)k_narrow<DT>;
      bp.gridDim = dim3(w->narrow_nc);
      bp.blockDim = dim3(NT);
      bp.sharedMemBytes = (unsigned)w->smem_narrow;
      ENT_CUDA(cudaGraphAddKernelNode(&n_narrow, body, &n_inspect, 1, &bp));
      cudaLaunchAttributeValue cv = {};
      cv.clusterDim.x = (unsigned)w->narrow_nc;
      cv.clusterDim.y = 1;
      cv.clusterDim.z = 1;
      ENT_CUDA(cudaGraphKernelNodeSetAttribute(n_narrow, cudaLaunchAttributeClusterDimension, &cv));
      prev = n_narrow;
    }
  }
  ENT_CUDA(cudaGraphInstantiate(&w->exec[k], graph, 0));
  return ENT_OK;
}

template <class DT>
static cudaError_t launch_narrow(const BfsWorkspace* w, const LevelArgs& la, cudaStream_t s) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(w->narrow_nc);
  cfg.blockDim = dim3(NT);
  cfg.dynamicSmemBytes = w->smem_narrow;
  cfg.stream = s;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeClusterDimension;
  at[0].val.clusterDim.x = (unsigned)w->narrow_nc;
  at[0].val.clusterDim.y = 1;
  at[0].val.clusterDim.z = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, k_narrow<DT>, la);
}

// Largest cluster (<= limit CTAs, 0 = no limit) of the small-frontier kernel
// that can be resident on this GPU; 0 if none.
static int pick_narrow_cluster(int limit, size_t smem) {
  if (cudaFuncSetAttribute(k_narrow<int32_t>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess ||
      cudaFuncSetAttribute(k_narrow<int32_t>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != cudaSuccess ||
      cudaFuncSetAttribute(k_narrow<uint8_t>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess ||
      cudaFuncSetAttribute(k_narrow<uint8_t>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  for (int nc = NC_MAX; nc >= 1; nc >>= 1) {
    if (limit > 0 && nc > limit) continue;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(nc);
    cfg.blockDim = dim3(NT);
    cfg.dynamicSmemBytes = smem;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = (unsigned)nc;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    int n = 0;
    if (cudaOccupancyMaxActiveClusters(&n, k_narrow<int32_t>, &cfg) == cudaSuccess && n >= 1) return nc;
    cudaGetLastError();
  }
  return 0;
}

static int create_workspace(ent_graph* g, BfsWorkspace** out, bool force_graph = false, int32_t cluster = 0) {
  BfsWorkspace* w = new BfsWorkspace();
  w->device = g->device;
  w->V = g->V;
  const int64_t V = g->V;
  const int64_t W = (V + 31) / 32;
  const int64_t tiles = std::max((V + TILE - 1) / TILE, (W + BT - 1) / BT) + 1;
  const ent_bfs_opts& o = g->opts;
  int hub = o.hub_slots;
  if (hub > 0 && hub < 16) hub = 16;
  // Slab layout (all 256-byte aligned): vis, fb0, fb1, q[2][3], qc[2], raw, hub[2], tiles.
  auto al = [](size_t x) { return (x + 255) & ~(size_t)255; };
  size_t sz_bits = al(sizeof(uint32_t) * (W + 1));
  size_t sz_q = al(sizeof(int32_t) * (V + 4));
  size_t sz_hub = al(sizeof(unsigned long long) * (hub > 0 ? hub : 1));
  size_t sz_tiles = al(sizeof(unsigned long long) * tiles * KS);
  size_t total = 3 * sz_bits + 9 * sz_q + 2 * sz_hub + sz_tiles;
  cudaError_t e = cudaMalloc(&w->slab, total);
  if (e != cudaSuccess) { destroy_bfs_workspace(w); return fail(ENT_ERR_OOM, "workspace allocation (%zu bytes) failed", total); }
  // Initialise on the graph's stream and wait: the traversal runs on
  // non-blocking streams, which a plain cudaMemset (legacy stream, async to
  // the host) would not be ordered against.
  e = cudaMemsetAsync(w->slab, 0, total, g->stream);
  if (e == cudaSuccess) e = cudaMalloc(&w->ctl, sizeof(BfsCtl));
  if (e == cudaSuccess) e = cudaMemsetAsync(w->ctl, 0, sizeof(BfsCtl), g->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(g->stream);
  if (e == cudaSuccess) e = cudaMallocHost(&w->ctl_h, sizeof(BfsCtl));
  if (e == cudaSuccess) e = cudaMalloc(&w->depth, sizeof(int32_t) * V);
  if (e == cudaSuccess) e = cudaMalloc(&w->parent, sizeof(int32_t) * V);
  if (e == cudaSuccess) e = cudaEventCreate(&w->ev0);
  if (e == cudaSuccess) e = cudaEventCreate(&w->ev1);
  if (e != cudaSuccess) { destroy_bfs_workspace(w); return fail(ENT_ERR_OOM, "workspace setup failed: %s", cudaGetErrorString(e)); }
  char* p = (char*)w->slab;
  LevelArgs& a = w->args;
  memset(&a, 0, sizeof(a));
  a.ctl = w->ctl;
  a.off = g->off;
  a.adj = g->trav;
  a.lead = g->lead;
  a.deg = g->deg;
  a.active = g->active;
  a.V = V;
  a.E = g->E;
  a.vis = (uint32_t*)p; p += sz_bits;
  a.fb[0] = (uint32_t*)p; p += sz_bits;
  a.fb[1] = (uint32_t*)p; p += sz_bits;
  for (int i = 0; i < 2; ++i)
    for (int k = 0; k < 3; ++k) { a.q[i][k] = (int32_t*)p; p += sz_q; }
  for (int i = 0; i < 2; ++i) { a.qc[i] = (int32_t*)p; p += sz_q; }
  a.raw = (int32_t*)p; p += sz_q;
  a.hub[0] = (unsigned long long*)p; p += sz_hub;
  a.hub[1] = (unsigned long long*)p; p += sz_hub;
  a.tiles = (unsigned long long*)p; p += sz_tiles;
  a.small_max = o.small_max;
  a.large_min = o.large_min;
  a.chunk = o.chunk_edges;
  a.hub_slots = hub;
  int lg = 0;
  while ((1 << lg) < hub) ++lg;
  a.hub_shift = 32 - lg;
  a.hub_min_deg = o.small_max;
  a.policy = o.policy;
  a.alpha = o.alpha;
  a.beta = o.beta;
  a.ref_ratio = o.ref_ratio;
  a.fault_inject = o.fault_inject;
  a.max_levels = (int32_t)std::min<int64_t>(V + 2, 0x7ffffff0);
  w->smem_expand = sizeof(int32_t) * (hub > 0 ? hub : 1);
  int occ_e = 0, occ_i = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_e, k_expand<int32_t>, BT, w->smem_expand);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_i, k_inspect, BT, 0);
  if (occ_e < 1) occ_e = 1;
  if (occ_i < 1) occ_i = 1;
  if (o.blocks_per_sm > 0) occ_e = std::min(occ_e, o.blocks_per_sm);
  w->grid_expand = g->num_sms * occ_e;
  w->grid_inspect = g->num_sms * std::min(occ_i, 4);
  w->grid_reset = g->num_sms * 4;
  w->smem_narrow = 2 * NQCAP * sizeof(int4);
  w->narrow_nc =
      o.narrow_max_frontier > 0 ? pick_narrow_cluster(cluster > 0 ? cluster : o.narrow_cluster, w->smem_narrow) : 0;
  if (w->narrow_nc > 0) {
    a.narrow_f = std::min(o.narrow_max_frontier, w->narrow_nc * NQCAP / 2);
    a.exit_f = 2 * a.narrow_f;
    a.narrow_m = o.narrow_max_edges;
    a.exit_m = 2 * (int64_t)o.narrow_max_edges;
    a.narrow_deg = o.narrow_max_degree;
  }
  if (o.loop == ENT_LOOP_GRAPH || force_graph) {
    int rc = build_graph<int32_t>(g, w);
    if (rc != ENT_OK) { destroy_bfs_workspace(w); return rc; }
  }
  *out = w;
  return ENT_OK;
}

int create_bfs_workspace(ent_graph* g, BfsWorkspace** out, int32_t cluster) {
  return create_workspace(g, out, true, cluster);
}

static void fill_stats(const BfsCtl& h, float ms, ent_stats* stats) {
  stats->reached_vertices = h.n_vis;
  stats->traversed_edges = h.m_vis;
  stats->levels = h.level;
  stats->td_levels = h.td_levels;
  stats->bu_levels = h.bu_levels;
  stats->status = h.err;
  stats->device_ms = ms;
  stats->narrow_levels = h.narrow_levels;
  stats->launches = 1 + 2 * h.iters + h.narrow_calls;
}

// One launch of the workspace's instantiated traversal graph on stream s.
template <class DT>
static int launch_graph(ent_graph* g, BfsWorkspace* w, int32_t src, DT* depth, int32_t* parent, cudaStream_t s) {
  const int k = depth_kind<DT>();
  if (!w->exec[k]) {  // the byte-depth graph is built on first use
    int rc = build_graph<DT>(g, w);
    if (rc != ENT_OK) return rc;
  }
  LevelArgs ra = w->args;
  ra.use_cond = 0;
  void* rargs[4] = {&ra, &src, &depth, &parent};
  cudaKernelNodeParams kp = {};
  kp.func = (void*)k_reset<DT>;
  kp.gridDim = dim3(w->grid_reset);
  kp.blockDim = dim3(BT);
  kp.sharedMemBytes = 0;
  kp.kernelParams = rargs;
  ENT_CUDA(cudaGraphExecKernelNodeSetParams(w->exec[k], w->reset_node[k], &kp));
  ENT_CUDA(cudaGraphLaunch(w->exec[k], s));
  return ENT_OK;
}

int launch_bfs_single(BfsWorkspace* w, int32_t src, int32_t* depth_dev, cudaStream_t s) {
  g_kernel_launches += 1;  // reset; the level kernels are counted by bfs_single_stats
  return launch_graph(nullptr, w, src, depth_dev, nullptr, s);  // int32 graph: built with the workspace
}

int bfs_single_stats(BfsWorkspace* w, cudaStream_t s, ent_stats* stats) {
  ENT_CUDA(cudaMemcpyAsync(w->ctl_h, w->ctl, sizeof(BfsCtl), cudaMemcpyDeviceToHost, s));
  ENT_CUDA(cudaStreamSynchronize(s));
  fill_stats(*w->ctl_h, 0.f, stats);
  g_kernel_launches += stats->launches - 1;
  if (w->ctl_h->err) return fail(ENT_ERR_TIMEOUT, "device traversal reported error flags 0x%x", w->ctl_h->err);
  return ENT_OK;
}

template <class DT>
static int run_bfs_typed(ent_graph* g, int32_t src, DT* depth, int32_t* parent, cudaStream_t stream, ent_stats* stats) {
  if (!g->ws) {
    int rc = create_workspace(g, &g->ws);
    if (rc != ENT_OK) return rc;
  }
  BfsWorkspace* w = g->ws;
  cudaStream_t s = stream ? stream : g->stream;
  if (stats) ENT_CUDA(cudaEventRecord(w->ev0, s));
  if (g->opts.loop == ENT_LOOP_GRAPH) {
    int rc = launch_graph(g, w, src, depth, parent, s);
    if (rc != ENT_OK) return rc;
  } else {
    LevelArgs la = w->args;
    la.use_cond = 0;
    k_reset<DT><<<w->grid_reset, BT, 0, s>>>(la, src, depth, parent);
    g_kernel_launches += 1;
    ENT_CUDA(cudaGetLastError());
    int32_t* flags_h = &w->ctl_h->done;  // done, narrow
    for (int64_t it = 0;; ++it) {
      k_expand<DT><<<w->grid_expand, BT, w->smem_expand, s>>>(la);
      k_inspect<<<w->grid_inspect, BT, 0, s>>>(la);
      g_kernel_launches += 2;
      ENT_CUDA(cudaGetLastError());
      ENT_CUDA(cudaMemcpyAsync(flags_h, &w->ctl->done, 2 * sizeof(int32_t), cudaMemcpyDeviceToHost, s));
      ENT_CUDA(cudaStreamSynchronize(s));
      if (flags_h[0]) break;
      if (flags_h[1]) {
        ENT_CUDA(launch_narrow<DT>(w, la, s));
        g_kernel_launches += 1;
      }
      if (it > w->V + 2) return fail(ENT_ERR_INTERNAL, "level loop did not terminate");
    }
  }
  if (stats) {
    ENT_CUDA(cudaEventRecord(w->ev1, s));
    ENT_CUDA(cudaMemcpyAsync(w->ctl_h, w->ctl, sizeof(BfsCtl), cudaMemcpyDeviceToHost, s));
    ENT_CUDA(cudaStreamSynchronize(s));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, w->ev0, w->ev1);
    fill_stats(*w->ctl_h, ms, stats);
    if (g->opts.loop == ENT_LOOP_GRAPH) g_kernel_launches += stats->launches;
    if (w->ctl_h->err) return fail(ENT_ERR_TIMEOUT, "device traversal reported error flags 0x%x", w->ctl_h->err);
  } else if (g->opts.loop == ENT_LOOP_GRAPH) {
    g_kernel_launches += 1;  // reset; level kernels are counted when stats are read
  }
  return ENT_OK;
}

int run_bfs_single(ent_graph* g, int32_t src, int32_t* depth, int32_t* parent, cudaStream_t stream, ent_stats* stats) {
  return run_bfs_typed<int32_t>(g, src, depth, parent, stream, stats);
}

int probe_graph_levels(ent_graph* g, const int32_t* src, int32_t n_src, int32_t* levels) {
  *levels = 0;
  if (!g->ws) {
    int rc = create_workspace(g, &g->ws);
    if (rc != ENT_OK) return rc;
  }
  int tried = 0;
  for (int32_t i = 0; i < n_src && tried < 3; ++i) {
    if (i > 0 && src[i] == src[i - 1]) continue;
    ent_stats st{};
    int rc = run_bfs_single(g, src[i], g->ws->depth, nullptr, g->stream, &st);
    if (rc != ENT_OK) return rc;
    ++tried;
    *levels = std::max(*levels, st.levels);
    if (st.reached_vertices * 4 >= g->V) break;  // a source in the bulk of the graph
  }
  return ENT_OK;
}

// ---------------------------------------------------------- deep batches --
// A batch of sources on a deep graph runs as concurrent single-source
// traversals, "lanes": each lane is a workspace with its own instantiated
// CUDA graph and stream, whose small-frontier levels run inside its own
// cluster of batch_deep_cluster CTAs, and the lanes take the sources round
// robin. On such graphs a bitwise batch saves nothing (frontiers of different
// sources are disjoint rings, so per-level work grows with the sources) and
// pays grid-wide launches per level; lanes instead fill the GPU with as many
// clusters as it holds, each paying only its own level chain.
struct DeepLanes {
  int asked = 0;                     // cluster size the lanes were built for
  int cluster = 0;                   // CTAs per lane's cluster as built (the GPU may allow fewer)
  std::vector<BfsWorkspace*> w;
  std::vector<cudaStream_t> s;
  std::vector<cudaEvent_t> done;
  cudaEvent_t start = nullptr, end = nullptr;
  BfsCtl* ctl_h = nullptr;           // pinned: each source's final control block
  int32_t ctl_cap = 0;
};

void destroy_deep_lanes(DeepLanes* l) {
  if (!l) return;
  for (cudaStream_t s : l->s)
    if (s) cudaStreamSynchronize(s);
  for (BfsWorkspace* w : l->w) destroy_bfs_workspace(w);
  for (cudaStream_t s : l->s)
    if (s) cudaStreamDestroy(s);
  for (cudaEvent_t e : l->done)
    if (e) cudaEventDestroy(e);
  if (l->start) cudaEventDestroy(l->start);
  if (l->end) cudaEventDestroy(l->end);
  if (l->ctl_h) cudaFreeHost(l->ctl_h);
  delete l;
}

// Byte depths of one row at any alignment (the rows of a batch start at
// multiples of V bytes): depth d (0..254) as d, unreached (-1) as 255.
__global__ void __launch_bounds__(256) k_depth_u8_row(const int32_t* __restrict__ d, uint8_t* __restrict__ o,
                                                      int64_t V) {
  const int64_t nth = (int64_t)gridDim.x * blockDim.x;
  for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < V; j += nth) {
    const int x = __ldcs(d + j);
    o[j] = (uint8_t)((x < 0 ? 255 : x) & 0xFF);
  }
}

// Lanes the GPU runs at once: as many clusters of the lanes' size as it holds
// (at most 32, each lane's workspace holding about 11 words per vertex), or
// the option's cap.
static int lane_cap(const ent_graph* g, const DeepLanes* l) {
  const int cap = std::max(1, std::min(32, g->num_sms / std::max(1, l->cluster)));
  return g->opts.batch_deep_lanes > 0 ? std::min(g->num_sms, g->opts.batch_deep_lanes) : cap;
}

// Cluster size of the lanes for a batch of n sources: the option, or else the
// largest power of two in [4, 16] with n lanes of it fitting the GPU's SMs
// (measured on the 4096^2 grid: 8 sources run fastest with 8-16 CTAs per
// lane, 32 or more with 4).
static int lane_cluster(const ent_graph* g, int n) {
  if (g->opts.batch_deep_cluster > 0) return g->opts.batch_deep_cluster;
  int c = 16;
  while (c > 4 && (int64_t)c * n > g->num_sms) c >>= 1;
  return c;
}

// Builds lanes up to `want` (at least one, at most lane_cap) for a batch of
// n_src sources; lanes of another cluster size are rebuilt.
static int ensure_lanes(ent_graph* g, int n_src) {
  const int asked = lane_cluster(g, n_src);
  if (g->lanes && g->lanes->asked != asked) {
    destroy_deep_lanes(g->lanes);
    g->lanes = nullptr;
  }
  if (!g->lanes) {
    g->lanes = new DeepLanes();
    g->lanes->asked = asked;
    ENT_CUDA(cudaEventCreate(&g->lanes->start));
    ENT_CUDA(cudaEventCreate(&g->lanes->end));
  }
  DeepLanes* l = g->lanes;
  int want = n_src;
  if (!l->w.empty()) want = std::min(want, lane_cap(g, l));
  while ((int)l->w.size() < want) {
    BfsWorkspace* w = nullptr;
    int rc = create_workspace(g, &w, true, asked);
    if (rc != ENT_OK) return rc;
    l->w.push_back(w);
    cudaStream_t s = nullptr;
    cudaEvent_t e = nullptr;
    ENT_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    l->s.push_back(s);
    ENT_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    l->done.push_back(e);
    if (l->w.size() == 1) {
      l->cluster = std::max(1, w->narrow_nc);
      want = std::min(want, lane_cap(g, l));
    }
  }
  return ENT_OK;
}

int run_bfs_deep(ent_graph* g, const int32_t* src, int32_t n_src, void* depth_dev, bool bytes, cudaStream_t stream,
                 ent_stats* stats) {
  int rc = ensure_lanes(g, n_src);
  if (rc != ENT_OK) return rc;
  DeepLanes* l = g->lanes;
  const int n_lanes = std::min<int>((int)l->w.size(), n_src);
  if (l->ctl_cap < n_src) {
    if (l->ctl_h) cudaFreeHost(l->ctl_h);
    l->ctl_h = nullptr;
    l->ctl_cap = 0;
    ENT_CUDA(cudaMallocHost(&l->ctl_h, sizeof(BfsCtl) * (size_t)n_src));
    l->ctl_cap = n_src;
  }
  cudaStream_t cs = stream ? stream : g->stream;
  const int64_t V = g->V;
  ENT_CUDA(cudaEventRecord(l->start, cs));
  for (int k = 0; k < n_lanes; ++k) ENT_CUDA(cudaStreamWaitEvent(l->s[k], l->start, 0));
  const int pack_blocks = (int)std::min<int64_t>((V + 255) / 256, (int64_t)g->num_sms * 8);
  for (int32_t i = 0; i < n_src; ++i) {
    const int k = i % n_lanes;
    BfsWorkspace* w = l->w[k];
    int32_t* row = bytes ? w->depth : static_cast<int32_t*>(depth_dev) + (size_t)i * V;
    rc = launch_graph(g, w, src[i], row, nullptr, l->s[k]);
    if (rc != ENT_OK) return rc;
    if (bytes)
      k_depth_u8_row<<<pack_blocks, 256, 0, l->s[k]>>>(w->depth, static_cast<uint8_t*>(depth_dev) + (size_t)i * V, V);
    ENT_CUDA(cudaGetLastError());
    ENT_CUDA(cudaMemcpyAsync(l->ctl_h + i, w->ctl, sizeof(BfsCtl), cudaMemcpyDeviceToHost, l->s[k]));
  }
  for (int k = 0; k < n_lanes; ++k) {
    ENT_CUDA(cudaEventRecord(l->done[k], l->s[k]));
    ENT_CUDA(cudaStreamWaitEvent(cs, l->done[k], 0));
  }
  ENT_CUDA(cudaEventRecord(l->end, cs));
  if (!stats) {
    g_kernel_launches += (bytes ? 2 : 1) * (int64_t)n_src;  // reset (+ pack); level kernels uncounted
    return ENT_OK;
  }
  ENT_CUDA(cudaEventSynchronize(l->end));
  float ms = 0.f;
  cudaEventElapsedTime(&ms, l->start, l->end);
  int err = 0, deep = 0;
  for (int32_t i = 0; i < n_src; ++i) {
    fill_stats(l->ctl_h[i], ms, &stats[i]);
    g_kernel_launches += stats[i].launches + (bytes ? 1 : 0);
    err |= l->ctl_h[i].err;
    deep |= stats[i].levels > 255;
  }
  if (err) return fail(ENT_ERR_TIMEOUT, "device traversal reported error flags 0x%x", err);
  if (bytes && deep) return fail(ENT_ERR_UNSUPPORTED, "a source reaches a depth above 254; byte depths hold 0..254");
  return ENT_OK;
}

}  // namespace ent

using namespace ent;

extern "C" {

int ent_bfs_device(ent_graph* g, int32_t src, int32_t* depth_dev, int32_t* parent_dev, void* stream, ent_stats* stats) {
  ent::NvtxRange nvtx_range("ent_bfs_device");
  clear_error();
  if (!g || !depth_dev) return fail(ENT_ERR_INVALID_ARG, "null argument");
  if (src < 0 || src >= g->V) return fail(ENT_ERR_INVALID_ARG, "source %d out of range [0,%lld)", src, (long long)g->V);
  std::lock_guard<std::mutex> lk(g->mu);
  DeviceGuard dg(g->device);
  return run_bfs_single(g, src, depth_dev, parent_dev, (cudaStream_t)stream, stats);
}

int ent_bfs_trace(ent_graph* g, int32_t src, ent_level_trace* out, int32_t max_levels, int32_t* n_levels,
                  ent_stats* stats) {
  ent::NvtxRange nvtx_range("ent_bfs_trace");
  clear_error();
  if (!g || !out || !n_levels || max_levels < 1) return fail(ENT_ERR_INVALID_ARG, "bad arguments");
  if (src < 0 || src >= g->V) return fail(ENT_ERR_INVALID_ARG, "source %d out of range", src);
  std::lock_guard<std::mutex> lk(g->mu);
  DeviceGuard dg(g->device);
  if (!g->ws) {
    int rc = create_workspace(g, &g->ws);
    if (rc != ENT_OK) return rc;
  }
  BfsWorkspace* w = g->ws;
  cudaStream_t s = g->stream;
  cudaEvent_t e[3];
  for (int i = 0; i < 3; ++i) ENT_CUDA(cudaEventCreate(&e[i]));
  LevelArgs la = w->args;
  la.use_cond = 0;
  ENT_CUDA(cudaEventRecord(w->ev0, s));
  k_reset<int32_t><<<w->grid_reset, BT, 0, s>>>(la, src, w->depth, nullptr);
  g_kernel_launches += 1;
  int n = 0;
  for (;;) {
    ENT_CUDA(cudaMemcpyAsync(w->ctl_h, w->ctl, sizeof(BfsCtl), cudaMemcpyDeviceToHost, s));
    ENT_CUDA(cudaStreamSynchronize(s));
    const BfsCtl h = *w->ctl_h;
    if (h.done || n >= max_levels) break;
    ent_level_trace& t = out[n];
    if (h.narrow) {  // one row for a run of the small-frontier kernel (direction 2)
      t.level = h.level;
      t.direction = 2;
      t.bu_sweep = 0;
      t.pad = 0;
      t.frontier_vertices = h.n_f;
      t.frontier_edges = h.m_f;
      t.unvisited_queued = 0;
      ENT_CUDA(cudaEventRecord(e[0], s));
      ENT_CUDA(launch_narrow<int32_t>(w, la, s));
      ENT_CUDA(cudaEventRecord(e[1], s));
      g_kernel_launches += 1;
      ENT_CUDA(cudaEventSynchronize(e[1]));
      float ta = 0;
      cudaEventElapsedTime(&ta, e[0], e[1]);
      t.expand_ms = ta;
      t.inspect_ms = 0;
      ++n;
      continue;
    }
    t.level = h.level;
    t.direction = h.dir;
    t.bu_sweep = h.dir == BU;
    t.pad = 0;
    t.frontier_vertices = h.n_f;
    t.frontier_edges = h.m_f;
    t.unvisited_queued = 0;
    ENT_CUDA(cudaEventRecord(e[0], s));
    k_expand<int32_t><<<w->grid_expand, BT, w->smem_expand, s>>>(la);
    ENT_CUDA(cudaEventRecord(e[1], s));
    k_inspect<<<w->grid_inspect, BT, 0, s>>>(la);
    ENT_CUDA(cudaEventRecord(e[2], s));
    g_kernel_launches += 2;
    ENT_CUDA(cudaGetLastError());
    ENT_CUDA(cudaEventSynchronize(e[2]));
    float ta = 0, tb = 0;
    cudaEventElapsedTime(&ta, e[0], e[1]);
    cudaEventElapsedTime(&tb, e[1], e[2]);
    t.expand_ms = ta;
    t.inspect_ms = tb;
    ++n;
  }
  ENT_CUDA(cudaEventRecord(w->ev1, s));
  ENT_CUDA(cudaStreamSynchronize(s));
  for (int i = 0; i < 3; ++i) cudaEventDestroy(e[i]);
  *n_levels = n;
  const BfsCtl& h = *w->ctl_h;
  if (stats) {
    float ms = 0.f;
    cudaEventElapsedTime(&ms, w->ev0, w->ev1);
    fill_stats(h, ms, stats);
  }
  if (h.err) return fail(ENT_ERR_TIMEOUT, "device traversal reported error flags 0x%x", h.err);
  return ENT_OK;
}

int ent_bfs(ent_graph* g, int32_t src, int32_t* depth_out, int32_t* parent_out, ent_stats* stats) {
  ent::NvtxRange nvtx_range("ent_bfs");
  clear_error();
  if (!g) return fail(ENT_ERR_INVALID_ARG, "null graph");
  if (src < 0 || src >= g->V) return fail(ENT_ERR_INVALID_ARG, "source %d out of range [0,%lld)", src, (long long)g->V);
  std::lock_guard<std::mutex> lk(g->mu);
  DeviceGuard dg(g->device);
  if (!g->ws) {
    int rc = create_workspace(g, &g->ws);
    if (rc != ENT_OK) return rc;
  }
  BfsWorkspace* w = g->ws;
  ent_stats local;
  int rc = run_bfs_single(g, src, w->depth, parent_out ? w->parent : nullptr, g->stream, stats ? stats : &local);
  if (rc != ENT_OK) return rc;
  if (depth_out)
    ENT_CUDA(cudaMemcpyAsync(depth_out, w->depth, sizeof(int32_t) * g->V, cudaMemcpyDeviceToHost, g->stream));
  if (parent_out)
    ENT_CUDA(cudaMemcpyAsync(parent_out, w->parent, sizeof(int32_t) * g->V, cudaMemcpyDeviceToHost, g->stream));
  ENT_CUDA(cudaStreamSynchronize(g->stream));
  return ENT_OK;
}

// The reference's source loop (bfs_gpu_opt.cuh:370-431: per source, reset,
// traverse, copy the depths to the host) as one call, pipelined: traversals
// alternate between two device depth buffers on the graph's stream while a
// copy stream moves the previous source's depths to its host array, so the
// copy of source i overlaps the traversal of source i+1.
static int bfs_many(ent_graph* g, const int32_t* src, int32_t n_src, void* const* depth_out, bool bytes,
                    ent_stats* stats) {
  ent::NvtxRange nvtx_range("ent_bfs_many");
  clear_error();
  if (!g) return fail(ENT_ERR_INVALID_ARG, "null graph");
  if (n_src < 0) return fail(ENT_ERR_INVALID_ARG, "negative source count %d", n_src);
  if (n_src > 0 && !src) return fail(ENT_ERR_INVALID_ARG, "null source list");
  for (int32_t i = 0; i < n_src; ++i)
    if (src[i] < 0 || src[i] >= g->V)
      return fail(ENT_ERR_INVALID_ARG, "source %d (index %d) out of range [0,%lld)", src[i], i, (long long)g->V);
  std::lock_guard<std::mutex> lk(g->mu);
  DeviceGuard dg(g->device);
  if (!g->ws) {
    int rc = create_workspace(g, &g->ws);
    if (rc != ENT_OK) return rc;
  }
  if (n_src == 0) return ENT_OK;
  BfsWorkspace* w = g->ws;
  if (!bytes && !w->depth_b && cudaMalloc(&w->depth_b, sizeof(int32_t) * g->V) != cudaSuccess) {
    w->depth_b = nullptr;
    return fail(ENT_ERR_OOM, "second depth buffer (%lld bytes) failed", (long long)(sizeof(int32_t) * g->V));
  }
  for (int i = 0; bytes && i < 2; ++i)
    if (!w->depth8[i] && cudaMalloc(&w->depth8[i], (size_t)g->V) != cudaSuccess) {
      w->depth8[i] = nullptr;
      return fail(ENT_ERR_OOM, "byte depth buffer (%lld bytes) failed", (long long)g->V);
    }
  if (!w->copy_stream) ENT_CUDA(cudaStreamCreateWithFlags(&w->copy_stream, cudaStreamNonBlocking));
  if (w->many_cap < n_src) {
    if (w->many_ctl_h) cudaFreeHost(w->many_ctl_h);
    w->many_ctl_h = nullptr;
    w->many_cap = 0;
    if (cudaMallocHost(&w->many_ctl_h, sizeof(BfsCtl) * n_src) != cudaSuccess) {
      w->many_ctl_h = nullptr;
      return fail(ENT_ERR_OOM, "pinned control copies failed");
    }
    w->many_cap = n_src;
  }
  const cudaStream_t s = g->stream, cs = w->copy_stream;
  // events (kept in the workspace): two per traversal for its time, and three
  // to order the streams: each depth buffer's latest copy done, a byte row in L2
  while (w->many_ev.size() < 2 * (size_t)n_src) {
    cudaEvent_t e = nullptr;
    if (cudaEventCreate(&e) != cudaSuccess) return fail(ENT_ERR_CUDA, "event creation failed");
    w->many_ev.push_back(e);
  }
  for (cudaEvent_t& e : w->many_sync)
    if (!e && cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) {
      e = nullptr;
      return fail(ENT_ERR_CUDA, "event creation failed");
    }
  const std::vector<cudaEvent_t>& ev = w->many_ev;
  // byte depths are written by the traversal itself (the reference's depth_t)
  void* buf[2] = {bytes ? (void*)w->depth8[0] : (void*)w->depth, bytes ? (void*)w->depth8[1] : (void*)w->depth_b};
  cudaEvent_t freed[2] = {w->many_sync[0], w->many_sync[1]};
  bool copied[2] = {false, false};
  const size_t row_bytes = (bytes ? 1 : sizeof(int32_t)) * g->V;
  int rc = ENT_OK;
  cudaError_t ce = cudaSuccess;
  int32_t done = 0;
  for (int32_t i = 0; i < n_src && rc == ENT_OK && ce == cudaSuccess; ++i) {
    const int b = i & 1;
    if (copied[b]) ce = cudaStreamWaitEvent(s, freed[b], 0);  // source i-2's copy has read buf[b]
    if (ce == cudaSuccess) ce = cudaEventRecord(ev[2 * (size_t)i], s);
    if (ce != cudaSuccess) break;
    rc = bytes ? run_bfs_typed<uint8_t>(g, src[i], (uint8_t*)buf[b], nullptr, s, nullptr)
               : run_bfs_typed<int32_t>(g, src[i], (int32_t*)buf[b], nullptr, s, nullptr);
    if (rc != ENT_OK) break;
    ce = cudaEventRecord(ev[2 * (size_t)i + 1], s);
    if (ce == cudaSuccess)
      ce = cudaMemcpyAsync(&w->many_ctl_h[i], w->ctl, sizeof(BfsCtl), cudaMemcpyDeviceToHost, s);
    if (ce == cudaSuccess && depth_out && depth_out[i]) {
      cudaEvent_t ready = ev[2 * (size_t)i + 1];
      if (bytes) {
        k_row_to_l2<<<(unsigned)((g->V + 128 * 256 - 1) / (128 * 256)), 256, 0, s>>>((const uint8_t*)buf[b], g->V);
        g_kernel_launches += 1;
        ce = cudaGetLastError();
        if (ce == cudaSuccess) ce = cudaEventRecord(w->many_sync[2], s);
        ready = w->many_sync[2];
      }
      if (ce == cudaSuccess) ce = cudaStreamWaitEvent(cs, ready, 0);
      if (ce == cudaSuccess) ce = cudaMemcpyAsync(depth_out[i], buf[b], row_bytes, cudaMemcpyDeviceToHost, cs);
      if (ce == cudaSuccess) ce = cudaEventRecord(freed[b], cs);
      copied[b] = true;
    }
    if (ce == cudaSuccess) done = i + 1;
  }
  const cudaError_t se = cudaStreamSynchronize(s);
  const cudaError_t sc = cudaStreamSynchronize(cs);
  if (rc == ENT_OK && ce == cudaSuccess) ce = se != cudaSuccess ? se : sc;
  if (rc == ENT_OK && ce != cudaSuccess) return fail(ENT_ERR_CUDA, "pipelined traversals: %s", cudaGetErrorString(ce));
  int first_bad = -1, first_deep = -1;
  for (int32_t i = 0; i < done; ++i) {
    const BfsCtl& h = w->many_ctl_h[i];
    ent_stats st;
    float ms = 0.f;
    cudaEventElapsedTime(&ms, ev[2 * (size_t)i], ev[2 * (size_t)i + 1]);
    fill_stats(h, ms, &st);
    if (g->opts.loop == ENT_LOOP_GRAPH) g_kernel_launches += st.launches - 2;
    if (stats) stats[i] = st;
    if (h.err && first_bad < 0) first_bad = i;
    if (bytes && st.levels > 255 && first_deep < 0) first_deep = i;
  }
  if (rc != ENT_OK) return rc;
  if (first_bad >= 0)
    return fail(ENT_ERR_TIMEOUT, "traversal %d (source %d) reported error flags 0x%x", first_bad, src[first_bad],
                w->many_ctl_h[first_bad].err);
  if (first_deep >= 0)
    return fail(ENT_ERR_UNSUPPORTED, "source %d (index %d) reaches depth %d; byte depths hold 0..254",
                src[first_deep], first_deep, w->many_ctl_h[first_deep].level - 1);
  return ENT_OK;
}

int ent_bfs_many(ent_graph* g, const int32_t* src, int32_t n_src, int32_t* const* depth_out, ent_stats* stats) {
  return bfs_many(g, src, n_src, reinterpret_cast<void* const*>(depth_out), false, stats);
}

// The same loop returning the reference's own depth type: one byte per vertex
// (depth_t, comm.h:69; 255 = unreached, comm.h:131), a quarter of the bytes
// to copy to the host.
int ent_bfs_many_u8(ent_graph* g, const int32_t* src, int32_t n_src, uint8_t* const* depth_out, ent_stats* stats) {
  return bfs_many(g, src, n_src, reinterpret_cast<void* const*>(depth_out), true, stats);
}

}  // extern "C"
