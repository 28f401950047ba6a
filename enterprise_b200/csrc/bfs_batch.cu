// Bitwise multi-source BFS (many sources per launch) for sm_100a.
//
// No reference code exists for this path: the reference runs its 64 sources
// one after another (bfs_gpu_opt.cuh:370-432) and only cites the iBFS paper
// (readme.md:79). The design follows the published idea (Liu, Huang, Hu,
// "iBFS: Concurrent Breadth-First Search on GPUs", SIGMOD'16): one bit per
// source in a shared per-vertex status word, so one adjacency read serves
// every source that reaches the vertex at that level.
//
// Layout (per graph, W = words per vertex, a power of two >= n_src/64):
//   X    uint64[V][W]      visited bits
//   log  uint64[K][V][W]   ring of K levels: log[L-base][v] = bits found at level L
//   jf   int32[2][V]       joint frontier (vertices with any new bit), ping-pong
//   heavy int32[2][V]      joint-frontier vertices of degree >= opts.batch_heavy
//   done bit per vertex    every source has visited it (bottom-up skips it)
//   jfb  bit per vertex    [2] joint-frontier membership of levels L and L+1:
//                          dedups top-down claims and lets bottom-up skip the
//                          frontier-word gather of neighbours outside the frontier
//   act  uint64[2][W]      sources with a non-empty frontier at L (and at L+1,
//                          being collected): only their bits are ever needed
// A level is top-down (frontier-driven ORs of new bits, then a commit pass;
// with many frontier edges the ORs are no-return atomics and the commit
// rebuilds the frontier from its bitmap) or bottom-up (every unfinished
// vertex ORs its neighbours' frontier words, stopping once all bits of the
// active sources it lacks are covered; light, mid and large degree tiers).
// Depths are never scattered during the traversal: a flush kernel decodes the
// log into a byte tile per span of vertices, zeroing the slots as it reads
// them, and writes the source-major depth rows with coalesced vector stores.
#include <algorithm>
#include <string.h>
#include <vector>

#include "batch_internal.h"
#include "dev_common.cuh"
#include "dev_graph.h"

namespace ent {

constexpr int BB = 256;        // threads per CTA
constexpr int KMAX = 16;       // log slots (levels per flush window)
constexpr int LOOP_UNROLL = 2; // level-loop bodies per while-node iteration of the CUDA-graph loop
constexpr int SEED_THREADS = 1024;  // the one seeding CTA: a multi-graph plan seeds thousands of entries
constexpr int WMAX = 32;       // words per vertex per launch (2048 sources)

struct BatchCtl {
  int32_t level;     // level of the frontier being expanded
  int32_t dir;       // 0 top-down, 1 bottom-up
  int32_t done;
  int32_t err;
  int32_t cur;       // jf / heavy ping-pong index
  int32_t n_jf[2];
  int32_t n_heavy[2];
  int32_t base;      // level stored in log slot 0
  int32_t windows;   // flush windows completed
  int32_t flush_now; // the window is full: flush before the next level
  int32_t td_levels, bu_levels;
  int32_t n_src;
  int32_t td_scan;   // top-down level of many edges: claims by no-return atomics, the commit rebuilds jf from jfb
  int32_t* depth;    // [n_src][V] output of this run
  const int32_t* row_map;  // optional: source s writes row row_map[s] of depth
  unsigned long long acc_m, acc_mdone;
  int64_t m_f, m_done;
  uint32_t finished;
  int32_t out_bytes;  // depth rows are uint8 (the reference's depth type, 255 = unreached), not int32
  int32_t clear_done; // sources joined: the completion bits no longer hold (k_b_flush clears them)
  int32_t joined;     // sources that joined this run
  int32_t flush_runs;    // level-loop iterations whose flush did work (window flush or joined sources)
  int32_t n_seed;     // entries of the seed list (0: one seed per source, src[s] for source s)
  int32_t iters;      // commit launches (level-loop bodies run, those after the end included)
};

struct BatchArgs {
  BatchCtl* ctl;
  const int64_t* off;
  const int32_t* adj;
  const int4* lead;     // adj[off[v] .. off[v]+3] per vertex (-1 past the row)
  const int32_t* deg;
  const uint32_t* active;
  int64_t V, E;
  int32_t W, lgW;       // words per vertex and log2(W)
  int32_t K;            // log slots in use
  unsigned long long* X;
  unsigned long long* log;
  const unsigned long long* mask;  // [W] valid source bits
  // [2][W] active sources: act[cur] holds the sources whose level-L frontier
  // is non-empty, act[nxt] collects those found at level L+1. A source that
  // is not active can add no bit again, so only its bits are ever needed.
  unsigned long long* act[2];
  uint32_t* donebits;
  uint32_t* jfb[2];
  const uint32_t* lightbits;  // degree in [1, batch_small_max): bottom-up light tier
  const int32_t* mid;         // batch_small_max <= degree < batch_large_min
  const int32_t* large;       // degree >= batch_large_min
  int32_t n_mid, n_large;
  int32_t* jf[2];
  int32_t* heavy[2];
  const int32_t* src;   // [n_src], or the seed vertices of a seed list
  const int32_t* seed_slot;  // source of each seed-list entry (null: entry i seeds source i)
  unsigned long long* st_edges;  // per source: sum of degrees of reached vertices
  unsigned long long* st_verts;  // per source: reached vertices
  int32_t* st_maxd;              // per source: max depth
  int32_t* join;                 // per source: the level of its depth 0 (0 unless it joined later)
  JoinBox* box;                  // mapped mailbox of sources joining at a level boundary, or null
  double alpha;      // bottom-up when frontier edges * alpha > unfinished edges
  int32_t heavy_deg; // top-down: from this degree every CTA takes a slice of a vertex
  cudaGraphConditionalHandle cond;
  int32_t use_cond;
  int32_t max_levels;
};

__device__ __forceinline__ unsigned long long* slot_ptr(const BatchArgs& a, int slot) {
  return a.log + (size_t)slot * (size_t)a.V * a.W;
}

template <class T>
__device__ __forceinline__ T bsum(T x, T* s_red) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(FULL, x, o);
  __syncthreads();
  if ((threadIdx.x & 31) == 0) s_red[threadIdx.x >> 5] = x;
  __syncthreads();
  T r = 0;
  if (threadIdx.x == 0)
    for (int w = 0; w < BB / 32; ++w) r += s_red[w];
  return r;
}

// Warp-aggregated append of v (when `want`) to list, counter *n.
__device__ __forceinline__ void wappend(bool want, int v, int32_t* list, int32_t* n) {
  const unsigned m = __ballot_sync(FULL, want);
  if (!m) return;
  const int lane = threadIdx.x & 31, leader = __ffs(m) - 1;
  int base = 0;
  if (lane == leader) base = atomicAdd(n, __popc(m));
  base = __shfl_sync(FULL, base, leader);
  if (want) list[base + __popc(m & lanemask_lt())] = v;
}

// Adds found source bits to the CTA's active-source word; the atomic is only
// paid for bits the word does not hold yet (a stale read costs an atomic).
__device__ __forceinline__ void note_act(unsigned long long* s_word, unsigned long long bits) {
  if ((*s_word & bits) != bits) atomicOr(s_word, bits);
}

// ORs the CTA's active-source words (s_act, W words) into dst; a word whose
// bits are all present already costs a read, not an atomic.
__device__ __forceinline__ void publish_act(const BatchArgs& a, const unsigned long long* s_act,
                                            unsigned long long* dst) {
  __syncthreads();
  if ((int)threadIdx.x < a.W) {
    const unsigned long long m = s_act[threadIdx.x];
    const unsigned long long have =
        (unsigned long long)__ldcg(reinterpret_cast<const long long*>(dst + threadIdx.x));
    if ((have & m) != m) atomicOr(dst + threadIdx.x, m);
  }
}

// ------------------------------------------------------------ seeding -----
// Runs after X, donebits and both jfb bitmaps are zeroed (memset nodes). One CTA
// of SEED_THREADS threads: each seed is a short chain of dependent atomics, and
// a multi-graph plan's seed list holds thousands (48 graphs x 64 sources).
__global__ void __launch_bounds__(SEED_THREADS) k_b_seed(BatchArgs a) {
  BatchCtl* c = a.ctl;
  unsigned long long* s0 = slot_ptr(a, 0);
  __shared__ int s_n, s_h;
  __shared__ unsigned long long s_m;
  if (threadIdx.x == 0) { s_n = 0; s_h = 0; s_m = 0; }
  __syncthreads();
  // A seed list gives a source several start vertices: a traversal over the
  // disjoint union of many graphs seeds source s in every graph at once.
  // The shared counters take one atomic per warp (ballot, then the leader),
  // not one per seed: thousands of same-address atomics would serialise. The
  // loop runs whole blocks at a time so that every lane takes part.
  const int n_seed = c->n_seed > 0 ? c->n_seed : c->n_src;
  const int lane = threadIdx.x & 31;
  for (int i0 = 0; i0 < n_seed; i0 += blockDim.x) {
    const int i = i0 + threadIdx.x;
    bool fresh = false;
    int v = 0, d = 0;
    if (i < n_seed) {
      v = a.src[i];
      const int s = a.seed_slot ? a.seed_slot[i] : i;
      const unsigned long long bit = 1ull << (s & 63);
      atomicOr(&a.X[(size_t)v * a.W + (s >> 6)], bit);
      atomicOr(&s0[(size_t)v * a.W + (s >> 6)], bit);
      const uint32_t tb = 1u << (v & 31);
      fresh = !(atomicOr(&a.jfb[0][v >> 5], tb) & tb);
      if (fresh) d = a.deg[v];
    }
    const unsigned mf = __ballot_sync(FULL, fresh);
    if (!mf) continue;
    const int leader = __ffs(mf) - 1;
    int at = 0;
    if (lane == leader) at = atomicAdd(&s_n, __popc(mf));
    at = __shfl_sync(FULL, at, leader);
    if (fresh) a.jf[0][at + __popc(mf & lanemask_lt())] = v;
    const bool hv = fresh && d >= a.heavy_deg;
    const unsigned mh = __ballot_sync(FULL, hv);
    if (mh) {
      const int lh = __ffs(mh) - 1;
      int ah = 0;
      if (lane == lh) ah = atomicAdd(&s_h, __popc(mh));
      ah = __shfl_sync(FULL, ah, lh);
      if (hv) a.heavy[0][ah + __popc(mh & lanemask_lt())] = v;
    }
    // degrees are below 2^31: split in 16-bit halves, each sums over 32 lanes without overflow
    const unsigned dlo = __reduce_add_sync(FULL, (unsigned)d & 0xFFFFu);
    const unsigned dhi = __reduce_add_sync(FULL, (unsigned)d >> 16);
    if (lane == leader) atomicAdd(&s_m, ((unsigned long long)dhi << 16) + dlo);
  }
  for (int w = threadIdx.x; w < a.W; w += blockDim.x) {
    a.act[0][w] = a.mask[w];
    a.act[1][w] = 0;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    c->level = 0;
    c->dir = 0;
    c->done = s_n == 0;
    c->err = 0;
    c->cur = 0;
    c->n_jf[0] = s_n;
    c->td_scan = 0;
    c->n_jf[1] = 0;
    c->n_heavy[0] = s_h;
    c->n_heavy[1] = 0;
    c->base = 0;
    c->windows = 0;
    c->flush_now = 0;
    c->td_levels = 0;
    c->bu_levels = 0;
    c->acc_m = 0;
    c->acc_mdone = 0;
    c->m_f = (int64_t)s_m;
    c->m_done = 0;
    c->finished = 0;
    __threadfence();
  }
}

// ----------------------------------------------------------- top-down -----
// Claims the bits of frontier vertex u (frontier words fu) for neighbour v.
// With `scan` (uniform) the words and the frontier bit are ORed by atomics
// whose results are not used, so nothing waits on memory; the commit then
// drops the bits v already had. Otherwise v's visited words filter the bits
// and the first claimant appends v to the next frontier.
__device__ __forceinline__ void td_edge(const BatchArgs& a, BatchCtl* c, const unsigned long long* fu, int v,
                                        bool valid, unsigned long long* nb, int nxt, bool scan) {
  if (scan) {
    if (valid) {
      bool any = false;
      for (int w = 0; w < a.W; ++w) {
        const unsigned long long f = fu[w];
        if (f) {
          atomicOr(nb + (size_t)v * a.W + w, f);
          any = true;
        }
      }
      if (any) atomicOr(&a.jfb[nxt][v >> 5], 1u << (v & 31));
    }
    return;
  }
  bool first = false;
  if (valid) {
    const unsigned long long* xv = a.X + (size_t)v * a.W;
    bool any = false;
    for (int w = 0; w < a.W; ++w) {
      const unsigned long long f = fu[w];
      if (!f) continue;
      const unsigned long long b = f & ~__ldg(xv + w);
      if (b) {
        atomicOr(nb + (size_t)v * a.W + w, b);
        any = true;
      }
    }
    if (any) {
      const uint32_t tb = 1u << (v & 31);
      first = !(atomicOr(&a.jfb[nxt][v >> 5], tb) & tb);
    }
  }
  wappend(first, v, a.jf[nxt], &c->n_jf[nxt]);
}

__device__ void b_td_expand(const BatchArgs& a, BatchCtl* c, unsigned long long* s_f) {
  const int cur = c->cur, nxt = cur ^ 1;
  const int slot = c->level - c->base;
  const unsigned long long* F = slot_ptr(a, slot);
  unsigned long long* NB = slot_ptr(a, slot + 1);
  const bool scan = c->td_scan != 0;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  // Heavy frontier vertices: every CTA takes an interleaved slice of the edges.
  const int nh = c->n_heavy[cur];
  for (int h = 0; h < nh; ++h) {
    const int u = a.heavy[cur][h];
    __syncthreads();
    for (int w = threadIdx.x; w < a.W; w += BB) s_f[w] = F[(size_t)u * a.W + w];
    __syncthreads();
    const int64_t beg = a.off[u], end = a.off[u + 1];
    for (int64_t e0 = beg + (int64_t)blockIdx.x * BB; e0 < end; e0 += (int64_t)gridDim.x * BB) {
      const int64_t e = e0 + threadIdx.x;
      const bool valid = e < end;
      td_edge(a, c, s_f, valid ? __ldg(a.adj + e) : 0, valid, NB, nxt, scan);
    }
  }
  // Light frontier vertices: one warp each; the warp keeps F[u] in shared memory.
  __syncthreads();
  unsigned long long* fw = s_f + (size_t)warp * a.W;
  const int n = c->n_jf[cur];
  const int gw = (blockIdx.x * BB + threadIdx.x) >> 5, nw = (gridDim.x * BB) >> 5;
  for (int i = gw; i < n; i += nw) {
    const int u = a.jf[cur][i];
    const int64_t beg = a.off[u], end = a.off[u + 1];
    if (end - beg >= a.heavy_deg) continue;
    __syncwarp();
    for (int w = lane; w < a.W; w += 32) fw[w] = F[(size_t)u * a.W + w];
    __syncwarp();
    for (int64_t e0 = beg; e0 < end; e0 += 32) {
      const int64_t e = e0 + lane;
      const bool valid = e < end;
      td_edge(a, c, fw, valid ? __ldg(a.adj + e) : 0, valid, NB, nxt, scan);
    }
  }
}

// ----------------------------------------------------------- bottom-up ----
// Reads WPL consecutive frontier words (8*WPL-byte aligned) with 16-byte loads.
template <int WPL>
__device__ __forceinline__ void load_words(const unsigned long long* p, unsigned long long (&f)[WPL]) {
  if constexpr (WPL == 1) {
    f[0] = __ldg(p);
  } else {
#pragma unroll
    for (int j = 0; j < WPL; j += 2) {
      const ulonglong2 x = __ldg(reinterpret_cast<const ulonglong2*>(p + j));
      f[j] = x.x;
      f[j + 1] = x.y;
    }
  }
}

// Records the outcome of one bottom-up vertex (called by the lane that owns
// the vertex): frontier append, counters, completion bit.
__device__ __forceinline__ void bu_finish_vertex(const BatchArgs& a, BatchCtl* c, int v, int nxt, bool gany,
                                                 bool gfull, int64_t d, unsigned long long& my_m,
                                                 unsigned long long& my_md) {
  if (gany) {
    my_m += (unsigned long long)d;
    atomicOr(&a.jfb[nxt][v >> 5], 1u << (v & 31));
    a.jf[nxt][atomicAdd(&c->n_jf[nxt], 1)] = v;
    if (d >= a.heavy_deg) a.heavy[nxt][atomicAdd(&c->n_heavy[nxt], 1)] = v;
  }
  if (gfull) {
    atomicOr(&a.donebits[v >> 5], 1u << (v & 31));
    my_md += (unsigned long long)d;
  }
}

// Gathers the frontier words of two neighbour slots of a row (e and e + step,
// each if below end): both ids, then both status bits, then both word loads
// are in flight together. A thread owns WPT consecutive words (from wofs) of
// every neighbour it visits and ORs them into acc.
template <int WPT>
__device__ __forceinline__ void bu_gather2(const BatchArgs& a, const uint32_t* jfc, const unsigned long long* F,
                                           int64_t e, int64_t step, int64_t end, int wofs,
                                           unsigned long long (&acc)[WPT]) {
  const bool ok0 = e < end, ok1 = e + step < end;
  const int u0 = ok0 ? __ldg(a.adj + e) : 0;
  const int u1 = ok1 ? __ldg(a.adj + e + step) : 0;
  const bool h0 = ok0 && ((__ldg(jfc + (u0 >> 5)) >> (u0 & 31)) & 1u);
  const bool h1 = ok1 && ((__ldg(jfc + (u1 >> 5)) >> (u1 & 31)) & 1u);
  unsigned long long f0[WPT], f1[WPT];
#pragma unroll
  for (int j = 0; j < WPT; ++j) f0[j] = f1[j] = 0;
  if (h0) load_words<WPT>(F + (size_t)u0 * a.W + wofs, f0);
  if (h1) load_words<WPT>(F + (size_t)u1 * a.W + wofs, f1);
#pragma unroll
  for (int j = 0; j < WPT; ++j) acc[j] |= f0[j] | f1[j];
}

// ORs r across the lanes of a warp that own the same words (lanes equal
// modulo G). With G = 1 every lane owns the same words: one redux per half.
template <int WPT>
__device__ __forceinline__ void group_or(unsigned long long (&r)[WPT], int G) {
  if (G == 1) {
#pragma unroll
    for (int j = 0; j < WPT; ++j) {
      const unsigned lo = __reduce_or_sync(FULL, (unsigned)r[j]);
      const unsigned hi = __reduce_or_sync(FULL, (unsigned)(r[j] >> 32));
      r[j] = ((unsigned long long)hi << 32) | lo;
    }
  } else {
#pragma unroll
    for (int j = 0; j < WPT; ++j)
      for (int o = G; o < 32; o <<= 1) r[j] |= __shfl_xor_sync(FULL, r[j], o);
  }
}

// Mid tier (batch_small_max <= degree < batch_large_min): one warp per vertex.
// G = W / WPT lanes cover a neighbour's W words (WPT each, one 8*WPT-byte
// load), so a warp visits 32 / G neighbours per slot and two slots per step,
// reading the row coalesced. Lanes accumulate in registers; the warp tests
// coverage after steps 1, 3, 7, 11, ... (the interval doubles up to 4).
template <int WPT>
__device__ void b_bu_mid(const BatchArgs& a, BatchCtl* c, const unsigned long long* F, unsigned long long* NB,
                         unsigned long long& my_m, unsigned long long& my_md, unsigned long long* s_act) {
  const int W = a.W, G = W / WPT, NS = 32 / G;
  const int lane = threadIdx.x & 31, gl = lane % G, k = lane / G;
  const int nxt = c->cur ^ 1;
  const int gw = (blockIdx.x * BB + threadIdx.x) >> 5, nw = (gridDim.x * BB) >> 5;
  const unsigned long long* ac = a.act[c->cur] + gl * WPT;
  const uint32_t* jfc = a.jfb[c->cur];
  for (int i = gw; i < a.n_mid; i += nw) {
    const int v = a.mid[i];
    if ((a.donebits[v >> 5] >> (v & 31)) & 1u) continue;
    unsigned long long* xv = a.X + (size_t)v * W + gl * WPT;
    unsigned long long need[WPT], acc[WPT];
    bool any = false;
#pragma unroll
    for (int j = 0; j < WPT; ++j) {
      need[j] = ac[j] & ~xv[j];
      acc[j] = 0;
      any |= need[j] != 0;
    }
    if (!__any_sync(FULL, any)) {  // every source it still lacks has finished
      if (lane == 0) bu_finish_vertex(a, c, v, nxt, false, true, a.deg[v], my_m, my_md);
      continue;
    }
    const int64_t beg = a.off[v], end = a.off[v + 1];
    int chk = 1, since = 0;
    for (int64_t b0 = beg; b0 < end; b0 += 2 * NS) {
      bu_gather2<WPT>(a, jfc, F, b0 + k, NS, end, gl * WPT, acc);
      if (++since == chk) {
        since = 0;
        if (chk < 4) chk <<= 1;
        unsigned long long r[WPT];
        bool mine = true;
#pragma unroll
        for (int j = 0; j < WPT; ++j) r[j] = acc[j];
        group_or<WPT>(r, G);
#pragma unroll
        for (int j = 0; j < WPT; ++j) mine &= (r[j] & need[j]) == need[j];
        if (__all_sync(FULL, mine)) break;
      }
    }
    group_or<WPT>(acc, G);
    bool got = false, full = true;
#pragma unroll
    for (int j = 0; j < WPT; ++j) {
      const unsigned long long nw_ = acc[j] & need[j];
      if (nw_) {
        got = true;
        if (k == 0) {
          NB[(size_t)v * W + gl * WPT + j] = nw_;
          xv[j] = xv[j] | nw_;
          note_act(s_act + gl * WPT + j, nw_);
        }
      }
      full &= (need[j] & ~nw_) == 0;
    }
    const bool gany = __any_sync(FULL, got);
    const bool gfull = __all_sync(FULL, full);
    if (lane == 0) bu_finish_vertex(a, c, v, nxt, gany, gfull, end - beg, my_m, my_md);
  }
}

// Large tier (degree >= batch_large_min): one CTA per vertex, the same lane
// layout over BB / G neighbours per slot. Threads accumulate in registers; at
// coverage tests (after steps 1, 3, 7, 15, 23, ...: the interval doubles up to
// 8) each warp folds its words into shared memory and the block votes.
template <int WPT>
__device__ void b_bu_large(const BatchArgs& a, BatchCtl* c, const unsigned long long* F, unsigned long long* NB,
                           unsigned long long& my_m, unsigned long long& my_md, unsigned long long* s_act) {
  __shared__ unsigned long long s_acc[WMAX], s_need[WMAX];
  __shared__ int s_skip;
  const int W = a.W, G = W / WPT, NS = BB / G;
  const int t = threadIdx.x, lane = t & 31, gl = t % G, k = t / G;
  const int nxt = c->cur ^ 1;
  const uint32_t* jfc = a.jfb[c->cur];
  const unsigned long long* ac = a.act[c->cur];
  for (int i = blockIdx.x; i < a.n_large; i += gridDim.x) {
    const int v = a.large[i];
    __syncthreads();
    if (t < W) {
      s_need[t] = ac[t] & ~a.X[(size_t)v * W + t];
      s_acc[t] = 0;
    }
    if (t == 0) s_skip = (a.donebits[v >> 5] >> (v & 31)) & 1u;
    __syncthreads();
    if (s_skip) continue;
    if (!__syncthreads_or(t < W && s_need[t] != 0)) {  // every source it still lacks has finished
      if (t == 0) bu_finish_vertex(a, c, v, nxt, false, true, a.deg[v], my_m, my_md);
      continue;
    }
    unsigned long long need[WPT], acc[WPT];
#pragma unroll
    for (int j = 0; j < WPT; ++j) {
      need[j] = s_need[gl * WPT + j];
      acc[j] = 0;
    }
    const int64_t beg = a.off[v], end = a.off[v + 1];
    int chk = 1, since = 0;
    for (int64_t b0 = beg; b0 < end; b0 += 2 * NS) {
      bu_gather2<WPT>(a, jfc, F, b0 + k, NS, end, gl * WPT, acc);
      if (++since == chk) {
        since = 0;
        if (chk < 8) chk <<= 1;
        unsigned long long r[WPT];
#pragma unroll
        for (int j = 0; j < WPT; ++j) r[j] = acc[j];
        group_or<WPT>(r, G);
        if (lane < G)
#pragma unroll
          for (int j = 0; j < WPT; ++j) note_act(s_acc + gl * WPT + j, r[j] & need[j]);
        __syncthreads();
        const bool open = t < W && (s_acc[t] & s_need[t]) != s_need[t];
        if (!__syncthreads_or(open)) break;
      }
    }
    group_or<WPT>(acc, G);
    if (lane < G)
#pragma unroll
      for (int j = 0; j < WPT; ++j) note_act(s_acc + gl * WPT + j, acc[j] & need[j]);
    __syncthreads();
    bool got = false, full = true;
    if (t < W) {
      const unsigned long long nw_ = s_acc[t] & s_need[t];
      if (nw_) {
        NB[(size_t)v * W + t] = nw_;
        a.X[(size_t)v * W + t] = a.X[(size_t)v * W + t] | nw_;
        note_act(s_act + t, nw_);
        got = true;
      }
      full = (s_need[t] & ~nw_) == 0;
    }
    const bool gany = __syncthreads_or(got);
    const bool gfull = !__syncthreads_or(!full);
    if (t == 0) bu_finish_vertex(a, c, v, nxt, gany, gfull, end - beg, my_m, my_md);
  }
}

// Light tier (degree < batch_small_max): a group of G = W / WPL lanes handles one
// vertex; each lane owns WPL words.
template <int WPL>
__device__ void b_bu_expand(const BatchArgs& a, BatchCtl* c, unsigned long long* s_red, unsigned long long* s_act) {
  const int cur = c->cur, nxt = cur ^ 1;
  const int slot = c->level - c->base;
  const unsigned long long* F = slot_ptr(a, slot);
  unsigned long long* NB = slot_ptr(a, slot + 1);
  const int G = a.W / WPL;  // lanes per vertex (1..32)
  const int VPW = 32 / G;   // vertices per warp round
  const int lane = threadIdx.x & 31;
  const int gl = lane % G;  // lane within group
  const int grp = lane / G;
  const unsigned gmask = (G == 32) ? FULL : (((1u << G) - 1) << (grp * G));
  const int64_t gtid = blockIdx.x * (int64_t)BB + threadIdx.x, nth = (int64_t)gridDim.x * BB;
  const int64_t gw = gtid >> 5, nw = nth >> 5;
  const int64_t Wd = (a.V + 31) >> 5;
  unsigned long long mk[WPL];
#pragma unroll
  for (int j = 0; j < WPL; ++j) mk[j] = a.act[cur][gl * WPL + j];
  const uint32_t* jfc = a.jfb[cur];
  unsigned long long my_m = 0, my_md = 0;
  for (int64_t wi = gw; wi < Wd; wi += nw) {
    const uint32_t todo_word = a.lightbits[wi] & ~a.donebits[wi];
    if (!todo_word) continue;
    uint32_t full_bits = 0, front_bits = 0;
    for (int r = 0; r < G; ++r) {
      const int vl = r * VPW + grp;
      if (!((todo_word >> (r * VPW)) & (VPW == 32 ? FULL : ((1u << VPW) - 1)))) continue;
      const bool todo = (todo_word >> vl) & 1u;
      const int64_t v = wi * 32 + vl;
      unsigned long long need[WPL], acc[WPL];
      bool any_need = false;
      int64_t e0 = 0, e1 = 0;
      int4 ld = make_int4(-1, -1, -1, -1);
      if (todo) {
        ld = __ldg(a.lead + v);  // the row's first four neighbours, read coalesced
        const unsigned long long* xv = a.X + (size_t)v * a.W + gl * WPL;
#pragma unroll
        for (int j = 0; j < WPL; ++j) {
          need[j] = mk[j] & ~xv[j];
          acc[j] = 0;
          any_need |= need[j] != 0;
        }
        e0 = a.off[v];
        e1 = a.off[v + 1];
      }
      // the whole group scans the row together (same trip count)
      if (todo) {
        bool cover = !(__ballot_sync(gmask, any_need) & gmask);
        // two neighbours per step: both gathers are in flight together; the
        // first two steps take their ids from the lead entry instead of the row
        for (int64_t e = e0; e < e1 && !cover; e += 2) {
          const int k = (int)(e - e0);
          int u0, u1;
          if (k == 0) {
            u0 = ld.x;
            u1 = e + 1 < e1 ? ld.y : u0;
          } else if (k == 2) {
            u0 = ld.z;
            u1 = e + 1 < e1 ? ld.w : u0;
          } else {
            u0 = __ldg(a.adj + e);
            u1 = e + 1 < e1 ? __ldg(a.adj + e + 1) : u0;
          }
          unsigned long long f0[WPL], f1[WPL];
#pragma unroll
          for (int j = 0; j < WPL; ++j) f0[j] = f1[j] = 0;
          if ((__ldg(jfc + (u0 >> 5)) >> (u0 & 31)) & 1u) load_words<WPL>(F + (size_t)u0 * a.W + gl * WPL, f0);
          if ((__ldg(jfc + (u1 >> 5)) >> (u1 & 31)) & 1u) load_words<WPL>(F + (size_t)u1 * a.W + gl * WPL, f1);
          bool mine = true;
#pragma unroll
          for (int j = 0; j < WPL; ++j) {
            acc[j] |= f0[j] | f1[j];
            mine &= (acc[j] & need[j]) == need[j];
          }
          cover = (__ballot_sync(gmask, mine) & gmask) == gmask;
        }
        bool got = false, full = true;
        unsigned long long* nbv = NB + (size_t)v * a.W + gl * WPL;
        unsigned long long* xw = a.X + (size_t)v * a.W + gl * WPL;
#pragma unroll
        for (int j = 0; j < WPL; ++j) {
          const unsigned long long nw_ = acc[j] & need[j];
          if (nw_) {
            nbv[j] = nw_;
            xw[j] = (mk[j] & ~need[j]) | nw_ | (xw[j] & ~mk[j]);
            note_act(s_act + gl * WPL + j, nw_);
            got = true;
          }
          full &= (need[j] & ~nw_) == 0;
        }
        const bool gany = (__ballot_sync(gmask, got) & gmask) != 0;
        const bool gfull = (__ballot_sync(gmask, full) & gmask) == gmask;
        if (gl == 0 && gany) my_m += (unsigned long long)(e1 - e0);
        if (gl == 0 && gfull) {
          full_bits |= 1u << vl;
          my_md += (unsigned long long)(e1 - e0);
        }
        if (gl == 0 && gany && e1 - e0 >= a.heavy_deg) {
          const int at = atomicAdd(&c->n_heavy[nxt], 1);
          a.heavy[nxt][at] = (int)v;
        }
        // append v to the next joint frontier (one lane per group)
        if (gl == 0 && gany) {
          const int at = atomicAdd(&c->n_jf[nxt], 1);
          a.jf[nxt][at] = (int)v;
          front_bits |= 1u << vl;
        }
      }
    }
    // vertices found complete (every source) become done
    full_bits = __reduce_or_sync(FULL, full_bits);
    front_bits = __reduce_or_sync(FULL, front_bits);
    if (lane == 0 && full_bits) atomicOr(&a.donebits[wi], full_bits);
    if (lane == 0 && front_bits) atomicOr(&a.jfb[nxt][wi], front_bits);
  }
  b_bu_mid<WPL>(a, c, F, NB, my_m, my_md, s_act);
  b_bu_large<WPL>(a, c, F, NB, my_m, my_md, s_act);
  publish_act(a, s_act, a.act[nxt]);
  const int any = __syncthreads_or(my_m != 0 || my_md != 0);
  if (any) {
    unsigned long long r = bsum(my_m, s_red);
    if (threadIdx.x == 0) atomicAdd(&c->acc_m, r);
    r = bsum(my_md, s_red);
    if (threadIdx.x == 0) atomicAdd(&c->acc_mdone, r);
  }
}

// One instantiation per width class: batches of up to 2 words per vertex fit
// 6 resident CTAs per SM without spills, while 4 words per lane need the
// registers of 4 (capped at 6 they spill, and the bottom-up levels slow down
// more than the occupancy gains: s22/256 5.71 -> 6.37 ms, s22/64 2.66 -> 2.45).
template <bool WIDE>
__global__ void __launch_bounds__(BB, WIDE ? 4 : 6) k_b_expand(BatchArgs a) {
  extern __shared__ unsigned long long s_f[];
  __shared__ unsigned long long s_red[BB / 32], s_act[WMAX];
  BatchCtl* c = a.ctl;
  if (c->done) return;
  if (c->dir == 0) {
    b_td_expand(a, c, s_f);
  } else {
    if ((int)threadIdx.x < WMAX) s_act[threadIdx.x] = 0;
    __syncthreads();
    if (a.W == 1) b_bu_expand<1>(a, c, s_red, s_act);
    else if (a.W == 2) b_bu_expand<2>(a, c, s_red, s_act);
    else if constexpr (WIDE) b_bu_expand<4>(a, c, s_red, s_act);
  }
}

static void* expand_kernel(int W) { return W > 2 ? (void*)k_b_expand<true> : (void*)k_b_expand<false>; }

// ----------------------------------------------------------- commit -------
// Folds v's claimed words NB[v] into X[v] (warp-uniform call; `valid` lanes
// only): the bits v already had are cleared from NB, got = a bit was new,
// full = v now holds every active source. The new words are OR-reduced across
// the warp into the CTA's active-source words.
__device__ __forceinline__ void td_commit_words(const BatchArgs& a, unsigned long long* NB,
                                                const unsigned long long* ac, int v, bool valid,
                                                unsigned long long* s_act, bool& got, bool& full) {
  const int lane = threadIdx.x & 31;
  got = false;
  full = true;
  for (int w = 0; w < a.W; ++w) {
    unsigned long long nn = 0;
    if (valid) {
      const size_t at = (size_t)v * a.W + w;
      const unsigned long long nb = NB[at], x = a.X[at];
      nn = nb & ~x;
      if (nn != nb) NB[at] = nn;
      if (nn) a.X[at] = x | nn;
      got |= nn != 0;
      full &= ((x | nn) & ac[w]) == ac[w];
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) nn |= __shfl_xor_sync(FULL, nn, o);
    if (lane == 0) note_act(s_act + w, nn);
  }
}

// The join mailbox is host memory written by the host while the batch runs.
__device__ __forceinline__ int ld_acquire_sys(const int32_t* p) {
  int v;
  asm volatile("ld.acquire.sys.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release_sys(int32_t* p, int v) {
  asm volatile("st.release.sys.global.b32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Level finisher (one thread, every CTA of the level done): publishes level L
// to the join mailbox and, while L is no deeper than the mailbox's limit,
// starts the sources posted there, at depth 0 on level L. Each takes its bit
// position s: the bit goes into its vertex's visited words and into the slot
// of level L's frontier, the vertex joins that frontier (once), s becomes an
// active source, and its depths are written relative to L (join[s]). Vertices
// marked complete lack the new bits, so their marks are dropped (k_b_flush
// clears them before the next level).
__device__ void join_sources(const BatchArgs& a, volatile BatchCtl* vc, int L, int nxt, int64_t& n_next,
                             int64_t& m_next) {
  JoinBox* box = a.box;
  *(volatile int32_t*)&box->level = L;
  if (L > *(volatile int32_t*)&box->limit) return;
  const int seq = ld_acquire_sys(&box->seq);
  if (seq == *(volatile int32_t*)&box->taken) return;
  const int nj = *(volatile int32_t*)&box->n;
  unsigned long long* F = slot_ptr(a, L - vc->base);
  int32_t* rows = const_cast<int32_t*>(vc->row_map);
  for (int j = 0; j < nj && j < JOIN_MAX; ++j) {
    const int s = *(volatile int32_t*)&box->pos[j];
    const int v = *(volatile int32_t*)&box->src[j];
    const int r = *(volatile int32_t*)&box->row[j];
    if (s < 0 || s >= a.W * 64 || v < 0 || v >= a.V) continue;  // the host never posts these
    const unsigned long long bit = 1ull << (s & 63);
    const size_t at = (size_t)v * a.W + (s >> 6);
    a.X[at] |= bit;
    F[at] |= bit;
    a.act[nxt][s >> 6] |= bit;
    a.join[s] = L;
    if (rows) rows[s] = r;
    if (s + 1 > vc->n_src) vc->n_src = s + 1;
    const uint32_t tb = 1u << (v & 31);
    if (!(a.jfb[nxt][v >> 5] & tb)) {
      a.jfb[nxt][v >> 5] |= tb;
      a.jf[nxt][n_next++] = v;
      const int d = a.deg[v];
      m_next += d;
      if (d >= a.heavy_deg) a.heavy[nxt][vc->n_heavy[nxt]++] = v;
    }
  }
  vc->n_jf[nxt] = (int32_t)n_next;
  vc->joined = vc->joined + nj;
  vc->clear_done = 1;
  vc->m_done = 0;
  __threadfence();
  st_release_sys(&box->taken, seq);
}

// Top-down: fold the claimed bits into X and count. Both directions: clear
// the frontier bitmap of level L (jfb[cur], its words hold only jf[cur]). Then the
// last CTA advances the level and picks the next direction.
__global__ void __launch_bounds__(BB) k_b_commit(BatchArgs a) {
  __shared__ unsigned long long s_red[BB / 32], s_act[WMAX];
  __shared__ int s_last;
  BatchCtl* c = a.ctl;
  if (c->done) {  // never leave the while node spinning on a finished traversal
    if (blockIdx.x == 0 && threadIdx.x == 0) {
      c->iters = c->iters + 1;
      if (a.use_cond) cudaGraphSetConditional(a.cond, 0u);
    }
    return;
  }
  const int cur = c->cur, nxt = cur ^ 1;
  const int dir = c->dir;
  {
    // frontier bitmap of level L: only words of jf[cur] vertices are set
    const int64_t gtid = blockIdx.x * (int64_t)BB + threadIdx.x, nth = (int64_t)gridDim.x * BB;
    const int nc = c->n_jf[cur];
    for (int64_t i = gtid; i < nc; i += nth) a.jfb[cur][(uint32_t)a.jf[cur][i] >> 5] = 0;
  }
  if (dir == 0) {
    const int slot = c->level - c->base;
    unsigned long long* NB = slot_ptr(a, slot + 1);
    const int n = c->n_jf[nxt];
    const unsigned long long* ac = a.act[cur];
    unsigned long long my_m = 0, my_md = 0;
    const int lane = threadIdx.x & 31;
    if ((int)threadIdx.x < WMAX) s_act[threadIdx.x] = 0;
    __syncthreads();
    const int64_t gtid = blockIdx.x * (int64_t)BB + threadIdx.x, nth = (int64_t)gridDim.x * BB;
    // bookkeeping for a vertex that gained a bit (got)
    const auto vertex_done = [&](int v, bool got, bool full) {
      if (!got) return;
      const int d = a.deg[v];
      my_m += d;
      if (full) {
        atomicOr(&a.donebits[v >> 5], 1u << (v & 31));
        my_md += d;
      }
      if (d >= a.heavy_deg) a.heavy[nxt][atomicAdd(&c->n_heavy[nxt], 1)] = v;
    };
    if (c->td_scan) {
      // a warp takes 32 consecutive jfb words (lane = word) and walks their
      // set bits in rounds, one vertex per lane per round
      uint32_t* jn = a.jfb[nxt];
      const int64_t Wd = (a.V + 31) >> 5;
      for (int64_t wb = gtid - lane; wb < Wd; wb += nth) {
        const int64_t wi = wb + lane;
        const uint32_t orig = wi < Wd ? jn[wi] : 0u;
        uint32_t bits = orig, keep = orig;
        while (__any_sync(FULL, bits != 0)) {
          const bool valid = bits != 0;
          const int b = valid ? __ffs(bits) - 1 : 0;
          bits &= bits - 1;
          const int v = (int)(wi * 32 + b);
          bool got, full;
          td_commit_words(a, NB, ac, v, valid, s_act, got, full);
          if (valid && !got) keep &= ~(1u << b);
          wappend(valid && got, v, a.jf[nxt], &c->n_jf[nxt]);
          if (valid) vertex_done(v, got, full);
        }
        if (keep != orig) jn[wi] = keep;
      }
    } else {
      // warp-uniform trip count: the claimed words are OR-reduced across the warp
      for (int64_t i0 = gtid - lane; i0 < n; i0 += nth) {
        const int64_t i = i0 + lane;
        const bool valid = i < n;
        const int v = valid ? a.jf[nxt][i] : 0;
        bool got, full;
        td_commit_words(a, NB, ac, v, valid, s_act, got, full);
        if (valid) vertex_done(v, true, full);
      }
    }
    publish_act(a, s_act, a.act[nxt]);
    if (__syncthreads_or(my_m != 0 || my_md != 0)) {
      unsigned long long r = bsum(my_m, s_red);
      if (threadIdx.x == 0) atomicAdd(&c->acc_m, r);
      r = bsum(my_md, s_red);
      if (threadIdx.x == 0) atomicAdd(&c->acc_mdone, r);
    }
  }
  if (threadIdx.x == 0) {
    __threadfence();
    s_last = atomicAdd(&c->finished, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!s_last || threadIdx.x != 0) return;
  __threadfence();
  volatile BatchCtl* vc = c;
  int64_t n_next = vc->n_jf[nxt];
  int64_t m_next = (int64_t)vc->acc_m;
  vc->m_done = vc->m_done + (int64_t)vc->acc_mdone;
  if (dir == 0) vc->td_levels = vc->td_levels + 1; else vc->bu_levels = vc->bu_levels + 1;
  const int L = vc->level + 1;
  vc->level = L;
  vc->iters = vc->iters + 1;
  if (a.box) join_sources(a, vc, L, nxt, n_next, m_next);
  // level L's active set is spent: it collects level L+2's from here
  for (int w = 0; w < a.W; ++w) a.act[cur][w] = 0;
  vc->cur = nxt;
  vc->n_jf[cur] = 0;
  vc->n_heavy[cur] = 0;
  vc->m_f = m_next;
  const double m_u = (double)(a.E - vc->m_done);
  vc->dir = ((double)m_next * a.alpha > m_u) ? 1 : 0;
  // a top-down level over at least V/4 edges claims without waiting on memory
  vc->td_scan = vc->dir == 0 && m_next * 4 >= a.V;
  int done = n_next == 0;
  if (L >= a.max_levels && !done) {
    vc->err = vc->err | 4;
    done = 1;
  }
  vc->done = done;
  // The next level writes slot L+1-base: flush first if it would not fit.
  vc->flush_now = !done && (L + 1 - vc->base >= a.K);
  vc->acc_m = 0;
  vc->acc_mdone = 0;
  vc->finished = 0;
  __threadfence();
  if (a.use_cond) cudaGraphSetConditional(a.cond, done ? 0u : 1u);
}

// ----------------------------------------------------------- flush --------
// Converts log slots [first, last] (levels base+first .. base+last) into the
// source-major depth rows and recycles the slots in the same pass. A CTA takes
// a span of 1024 vertices and walks the W word columns in groups of
// CG = min(W, 4), VS = 1024 / CG vertices per pass.
// Decode (thread per vertex): the slots of a vertex are disjoint bit sets, so
// the vertex's CG words of every slot fold into a found mask and four bit
// planes of the slot index; a bit-block transpose turns those into one byte
// per source (slot index, 0xFF where not found), stored in a vertex-major
// byte tile [vertex][64*CG sources].
// Each vertex's slot words are zeroed once decoded (a window flush carries the
// last slot, the next window's frontier, into slot 0).
// Write (warp per 4 sources): where every (source, vertex) pair is written
// (the first window: -1 where not found) and the rows allow it, a lane takes
// 4 consecutive vertices and stores each row's 4 depths as one vector;
// otherwise (later windows write only the pairs they found) a lane takes a
// vertex. Reached vertices, the sum of their degrees and the deepest level
// are kept per row.
constexpr int TILE_BYTES = 64 * 1024;  // VS vertices x 64*CG source bytes
constexpr int FLUSH_TILE_BYTES = TILE_BYTES + 1024 * 4;  // + the span's degrees

template <int CG>
__device__ __forceinline__ void load_cols(const unsigned long long* p, unsigned long long (&w)[CG]) {
  if constexpr (CG == 1) {
    w[0] = *p;
  } else {
#pragma unroll
    for (int j = 0; j < CG; j += 2) {
      const ulonglong2 x = *reinterpret_cast<const ulonglong2*>(p + j);
      w[j] = x.x;
      w[j + 1] = x.y;
    }
  }
}

template <int CG>
__device__ __forceinline__ void store_cols(unsigned long long* p, unsigned long long x0, unsigned long long x1,
                                           unsigned long long x2, unsigned long long x3) {
  if constexpr (CG == 1) {
    *p = x0;
  } else {
    *reinterpret_cast<ulonglong2*>(p) = make_ulonglong2(x0, x1);
    if constexpr (CG == 4) *reinterpret_cast<ulonglong2*>(p + 2) = make_ulonglong2(x2, x3);
  }
}

// Tile word c (4 sources) of vertex vi. Rows of 16*CG words, the word index
// XOR-swizzled by the vertex so that both access patterns spread over the
// banks: 32 consecutive vertices (decode, and the write of later windows) hit
// 32 banks, and vertices 4l+t of lanes l = 0..31 (the vector write; the base
// vertex a multiple of 128) hit 32 banks, or 16 when CG == 1.
template <int CG>
__device__ __forceinline__ int tile_word(int vi, int c) {
  if constexpr (CG == 1) return vi * 16 + (c ^ (((vi >> 1) ^ (vi >> 5)) & 15));
  else return vi * 16 * CG + (c ^ ((vi ^ (vi >> 5)) & 31));
}

// One step of an 8x8 bit-block transpose (per byte column of the rows):
// swaps the s-bit blocks that mask selects in b with the blocks s bits above
// them in a.
__device__ __forceinline__ void swap_blocks(uint32_t& a, uint32_t& b, int s, uint32_t mask) {
  const uint32_t t = ((a >> s) ^ b) & mask;
  b ^= t;
  a ^= t << s;
}

// 4x4 byte transpose: t[g] = byte g of a, b, c, d (a in byte 0).
__device__ __forceinline__ void byte_transpose4(uint32_t a, uint32_t b, uint32_t c, uint32_t d, uint32_t& t0,
                                                uint32_t& t1, uint32_t& t2, uint32_t& t3) {
  const uint32_t ab_lo = __byte_perm(a, b, 0x5140u), ab_hi = __byte_perm(a, b, 0x7362u);
  const uint32_t cd_lo = __byte_perm(c, d, 0x5140u), cd_hi = __byte_perm(c, d, 0x7362u);
  t0 = __byte_perm(ab_lo, cd_lo, 0x5410u);
  t1 = __byte_perm(ab_lo, cd_lo, 0x7632u);
  t2 = __byte_perm(ab_hi, cd_hi, 0x5410u);
  t3 = __byte_perm(ab_hi, cd_hi, 0x7632u);
}

// 32 sources' tile words from their found mask f and slot-index bit planes
// h0..h3: byte r of out[n] is the slot index of source 4n+r, 0xFF where not
// found. The rows (h0..h3 each ORed with not-found, then not-found four times)
// are transposed as 8x8 bit blocks per byte column, which turns byte g of row
// c into the 8 bits of source 8g+c; two 4x4 byte transposes then gather each
// word's four consecutive sources.
__device__ __forceinline__ void planes_to_tile_words(uint32_t f, uint32_t h0, uint32_t h1, uint32_t h2, uint32_t h3,
                                                     uint32_t (&out)[8]) {
  const uint32_t nf = ~f;
  uint32_t r0 = h0 | nf, r1 = h1 | nf, r2 = h2 | nf, r3 = h3 | nf, r4 = nf, r5 = nf, r6 = nf, r7 = nf;
  swap_blocks(r0, r1, 1, 0x55555555u);
  swap_blocks(r2, r3, 1, 0x55555555u);
  swap_blocks(r4, r5, 1, 0x55555555u);
  swap_blocks(r6, r7, 1, 0x55555555u);
  swap_blocks(r0, r2, 2, 0x33333333u);
  swap_blocks(r1, r3, 2, 0x33333333u);
  swap_blocks(r4, r6, 2, 0x33333333u);
  swap_blocks(r5, r7, 2, 0x33333333u);
  swap_blocks(r0, r4, 4, 0x0F0F0F0Fu);
  swap_blocks(r1, r5, 4, 0x0F0F0F0Fu);
  swap_blocks(r2, r6, 4, 0x0F0F0F0Fu);
  swap_blocks(r3, r7, 4, 0x0F0F0F0Fu);
  // sources 4n..4n+3 sit in rows 4(n&1)..4(n&1)+3, byte n>>1
  byte_transpose4(r0, r1, r2, r3, out[0], out[2], out[4], out[6]);
  byte_transpose4(r4, r5, r6, r7, out[1], out[3], out[5], out[7]);
}

// Byte j of w as a signed value (a slot index 0..15, or 0xFF -> -1). In its
// default mode prmt copies the selected byte's sign bit into every result
// byte whose selector nibble has its top bit set.
__device__ __forceinline__ int sext_byte(uint32_t w, uint32_t j) {
  const uint32_t sel = j | ((8u + j) * 0x1110u);
  uint32_t r;
  asm("prmt.b32 %0, %1, 0, %2;" : "=r"(r) : "r"(w), "r"(sel));
  return (int)r;
}

// The low bytes of a, b, c, d as one word, a in byte 0.
__device__ __forceinline__ uint32_t pack_low_bytes(int a, int b, int c, int d) {
  return __byte_perm(__byte_perm((uint32_t)a, (uint32_t)b, 0x0040u), __byte_perm((uint32_t)c, (uint32_t)d, 0x0040u),
                     0x5410u);
}

struct FlushState {
  int first, last, base, windows, nsrc;
  bool final_flush;
  bool vec;                 // whole-window rows take 16-byte (int32) or 4-byte (u8) vector stores
  int32_t* depth;
  const int32_t* row_map;
  uint32_t* tile;
  const int* s_deg;         // [1024] degrees of the span
  unsigned* s_cnt;          // [W*64] reached vertices per source
  unsigned long long* s_edg;  // [W*64] their degrees
  int* s_maxd;              // [W*64] deepest level
};

template <int CG, bool BYTES>
__device__ void flush_span(const BatchArgs& a, const FlushState& fs, int64_t v0, int nv) {
  constexpr int VS = 1024 / CG;  // vertices per pass
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int first = fs.first, last = fs.last;
  for (int sub = 0; sub < nv; sub += VS) {
    const int nsub = min(VS, nv - sub);
    for (int cg = 0; cg < a.W; cg += CG) {
      if (cg * 64 >= fs.nsrc) break;  // words of no source: never set, so already zero
      __syncthreads();  // the previous tile has been written out
      for (int vi = threadIdx.x; vi < VS; vi += BB) {
        const bool in = vi < nsub;
        const size_t at = (size_t)(v0 + sub + vi) * a.W + cg;
        unsigned long long f[CG], p0[CG], p1[CG], p2[CG], p3[CG];
#pragma unroll
        for (int cc = 0; cc < CG; ++cc) f[cc] = p0[cc] = p1[cc] = p2[cc] = p3[cc] = 0;
        // loads and folds only: no store or warp-collective may sit between
        // the slot loads, which the compiler then keeps in flight together
        if (in) {
          // slots in groups of four from a multiple of 4: bits 0 and 1 of a
          // slot's index follow from its place in the group, bits 2 and 3 are
          // the group's
          for (int k0 = 0; k0 <= last; k0 += 4) {
#pragma unroll
            for (int h = 0; h < 2; ++h) {
              const int ka = k0 + 2 * h, kb = ka + 1;
              unsigned long long wa[CG], wb[CG];
              if (ka >= first && ka <= last) load_cols<CG>(slot_ptr(a, ka) + at, wa);
              else
#pragma unroll
                for (int cc = 0; cc < CG; ++cc) wa[cc] = 0;
              if (kb >= first && kb <= last) load_cols<CG>(slot_ptr(a, kb) + at, wb);
              else
#pragma unroll
                for (int cc = 0; cc < CG; ++cc) wb[cc] = 0;
#pragma unroll
              for (int cc = 0; cc < CG; ++cc) {
                const unsigned long long u = wa[cc] | wb[cc];
                f[cc] |= u;
                p0[cc] |= wb[cc];
                if (h) p1[cc] |= u;
                if (k0 & 4) p2[cc] |= u;
                if (k0 & 8) p3[cc] |= u;
              }
            }
          }
        }
#pragma unroll
        for (int cc = 0; cc < CG; ++cc) {
#pragma unroll
          for (int hw = 0; hw < 2; ++hw) {
            uint32_t o[8];
            planes_to_tile_words((uint32_t)(f[cc] >> (32 * hw)), (uint32_t)(p0[cc] >> (32 * hw)),
                                 (uint32_t)(p1[cc] >> (32 * hw)), (uint32_t)(p2[cc] >> (32 * hw)),
                                 (uint32_t)(p3[cc] >> (32 * hw)), o);
#pragma unroll
            for (int n = 0; n < 8; ++n) fs.tile[tile_word<CG>(vi, cc * 16 + hw * 8 + n)] = o[n];
          }
        }
        if (in) {
          // recycle: a window flush carries slot K-1 (the next window's
          // frontier) into slot 0 and zeroes slots 1..K-1; the final flush
          // zeroes slots 0..last (slot 0 too after a window flush)
          int z0 = 0;
          if (!fs.final_flush) {
            unsigned long long x[CG];
            load_cols<CG>(slot_ptr(a, last) + at, x);
            store_cols<CG>(slot_ptr(a, 0) + at, x[0], x[CG > 1 ? 1 : 0], x[CG > 2 ? 2 : 0], x[CG > 2 ? 3 : 0]);
            z0 = 1;
          }
          for (int k = z0; k <= last; ++k) store_cols<CG>(slot_ptr(a, k) + at, 0ull, 0ull, 0ull, 0ull);
        }
      }
      __syncthreads();
      for (int r0 = warp * 4; r0 < 64 * CG; r0 += BB / 32 * 4) {
        const int s0 = cg * 64 + r0;
        if (s0 >= fs.nsrc) break;
        const int c4 = r0 >> 2;
        size_t ofs[4];  // element offset of each row's segment (int32 or byte rows)
        bool rv[4];
        int rb[4];      // depth of log slot 0 for the row: the window's base level less the source's start
        bool wide = false;  // a byte row whose depths could pass 254 here: checked one by one
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          rv[j] = s0 + j < fs.nsrc;
          ofs[j] = rv[j] ? (size_t)(fs.row_map ? fs.row_map[s0 + j] : s0 + j) * a.V + v0 + sub : 0;
          rb[j] = fs.base - (rv[j] ? a.join[s0 + j] : 0);
          if (BYTES && rv[j] && rb[j] > 239) wide = true;
        }
        unsigned cnt[4] = {0, 0, 0, 0};
        unsigned long long edg[4] = {0, 0, 0, 0};
        int mx[4] = {-1, -1, -1, -1};
        if (fs.vec && !wide) {
          for (int vi = lane * 4; vi < nsub; vi += 128) {
            uint32_t wv[4];
#pragma unroll
            for (int t = 0; t < 4; ++t) wv[t] = fs.tile[tile_word<CG>(vi + t, c4)];
            const int4 dg = *reinterpret_cast<const int4*>(fs.s_deg + sub + vi);
#pragma unroll
            for (int j = 0; j < 4; ++j) {
              if (!rv[j]) continue;
              int v[4], m[4];
#pragma unroll
              for (int t = 0; t < 4; ++t) {
                const int d = sext_byte(wv[t], j);
                m[t] = d >> 31;  // -1 where not found
                v[t] = d + (rb[j] & ~m[t]);
                cnt[j] += 1 + m[t];
                mx[j] = max(mx[j], v[t]);
              }
              // two degrees below 2^31 each cannot overflow 32 bits
              const uint32_t e01 = (uint32_t)(dg.x & ~m[0]) + (uint32_t)(dg.y & ~m[1]);
              const uint32_t e23 = (uint32_t)(dg.z & ~m[2]) + (uint32_t)(dg.w & ~m[3]);
              edg[j] += (unsigned long long)e01 + e23;
              if constexpr (BYTES)
                *reinterpret_cast<uint32_t*>(reinterpret_cast<uint8_t*>(fs.depth) + ofs[j] + vi) =
                    pack_low_bytes(v[0], v[1], v[2], v[3]);
              else
                *reinterpret_cast<int4*>(fs.depth + ofs[j] + vi) = make_int4(v[0], v[1], v[2], v[3]);
            }
          }
        } else {
          bool deep = false;  // a depth above 254 met in byte rows
          for (int vi = lane; vi < nsub; vi += 32) {
            const uint32_t wv = fs.tile[tile_word<CG>(vi, c4)];
            const int dg = fs.s_deg[sub + vi];
#pragma unroll
            for (int j = 0; j < 4; ++j) {
              if (!rv[j]) continue;
              const int d = sext_byte(wv, j);
              const int m = d >> 31;
              const int v = d + (rb[j] & ~m);
              if (fs.windows == 0 || d >= 0) {
                if constexpr (BYTES) {
                  reinterpret_cast<uint8_t*>(fs.depth)[ofs[j] + vi] = (uint8_t)v;  // -1 -> 255
                  deep |= v > 254;
                } else {
                  fs.depth[ofs[j] + vi] = v;
                }
              }
              cnt[j] += 1 + m;
              edg[j] += (uint32_t)(dg & ~m);
              mx[j] = max(mx[j], v);
            }
          }
          if constexpr (BYTES)
            if (__any_sync(FULL, deep) && lane == 0) atomicOr(&a.ctl->err, 16);
        }
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          // a lane's degree sum is below 2^36 (at most 32 vertices), so both
          // 16-bit-split halves sum over 32 lanes without overflow
          const unsigned c = __reduce_add_sync(FULL, cnt[j]);
          const unsigned elo = __reduce_add_sync(FULL, (unsigned)(edg[j] & 0xFFFFu));
          const unsigned ehi = __reduce_add_sync(FULL, (unsigned)(edg[j] >> 16));
          const int dmax = __reduce_max_sync(FULL, mx[j]);
          if (lane == 0 && rv[j] && c) {  // a source's rows are always this warp's
            fs.s_cnt[s0 + j] += c;
            fs.s_edg[s0 + j] += ((unsigned long long)ehi << 16) + elo;
            fs.s_maxd[s0 + j] = max(fs.s_maxd[s0 + j], dmax);
          }
        }
      }
    }
  }
  __syncthreads();
}

// Runs after a level when the log window is full (flush_now) or sources
// joined (clear_done), and once at the end (final_flush). Joined sources void
// the completion bits, which are cleared. A flush writes the window's depth
// rows and per-source statistics and recycles the slots (flush_span); a window
// flush then moves the window by K-1 levels.
__global__ void __launch_bounds__(BB, 3) k_b_flush(BatchArgs a, int final_flush) {
  extern __shared__ __align__(16) unsigned char s_flush[];
  BatchCtl* c = a.ctl;
  const bool clear = !final_flush && c->clear_done;  // sources joined at this level boundary
  const bool flush = final_flush || c->flush_now;
  if (!flush && !clear) return;
  if (clear) {
    const int64_t tid = blockIdx.x * (int64_t)BB + threadIdx.x, nth = (int64_t)gridDim.x * BB;
    for (int64_t i = tid; i <= (a.V + 31) >> 5; i += nth) a.donebits[i] = 0u;
  }
  if (flush) {
    FlushState fs;
    fs.base = c->base;
    fs.windows = c->windows;
    // final: levels base .. level-1 are in slots 0 .. level-1-base
    fs.last = final_flush ? (c->level - 1 - fs.base) : (a.K - 1);
    fs.first = fs.windows == 0 ? 0 : 1;
    fs.nsrc = c->n_src;
    fs.final_flush = final_flush != 0;
    fs.depth = c->depth;
    fs.row_map = c->row_map;
    const bool bytes = c->out_bytes != 0;
    // vector stores: every pair is written and each row segment (row * V + a
    // multiple of 4) starts 16-byte (int32) or 4-byte (u8) aligned
    fs.vec = fs.windows == 0 && (a.V & 3) == 0 && ((uintptr_t)fs.depth & (bytes ? 3 : 15)) == 0;
    const int NSRC = a.W * 64;
    fs.tile = reinterpret_cast<uint32_t*>(s_flush);
    fs.s_deg = reinterpret_cast<const int*>(s_flush + TILE_BYTES);
    fs.s_cnt = reinterpret_cast<unsigned*>(s_flush + FLUSH_TILE_BYTES);
    fs.s_edg = reinterpret_cast<unsigned long long*>(fs.s_cnt + NSRC);  // NSRC is a multiple of 64: 8-byte aligned
    fs.s_maxd = reinterpret_cast<int*>(fs.s_edg + NSRC);
    int* s_deg = reinterpret_cast<int*>(s_flush + TILE_BYTES);
    for (int i = threadIdx.x; i < NSRC; i += BB) { fs.s_cnt[i] = 0; fs.s_edg[i] = 0; fs.s_maxd[i] = -1; }
    const int64_t units = (a.V + 1023) / 1024;
    for (int64_t u = blockIdx.x; u < units; u += gridDim.x) {
      const int64_t v0 = u * 1024;
      const int nv = (int)min((int64_t)1024, a.V - v0);
      __syncthreads();
      for (int i = threadIdx.x; i < 1024; i += BB) s_deg[i] = i < nv ? a.deg[v0 + i] : 0;
      __syncthreads();
      if (bytes) {
        if (a.W == 1) flush_span<1, true>(a, fs, v0, nv);
        else if (a.W == 2) flush_span<2, true>(a, fs, v0, nv);
        else flush_span<4, true>(a, fs, v0, nv);
      } else {
        if (a.W == 1) flush_span<1, false>(a, fs, v0, nv);
        else if (a.W == 2) flush_span<2, false>(a, fs, v0, nv);
        else flush_span<4, false>(a, fs, v0, nv);
      }
    }
    __syncthreads();
    for (int s = threadIdx.x; s < fs.nsrc; s += BB) {
      if (fs.s_cnt[s]) {
        atomicAdd(&a.st_verts[s], (unsigned long long)fs.s_cnt[s]);
        atomicAdd(&a.st_edges[s], fs.s_edg[s]);
        atomicMax(&a.st_maxd[s], fs.s_maxd[s]);
      }
    }
  }
  if (final_flush) return;
  // the last CTA to finish moves the window
  __shared__ int s_last;
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    s_last = atomicAdd(&c->finished, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!s_last || threadIdx.x != 0) return;
  __threadfence();
  volatile BatchCtl* vc = c;
  if (flush) {
    vc->base = vc->base + a.K - 1;
    vc->windows = vc->windows + 1;
    vc->flush_now = 0;
  }
  vc->clear_done = 0;
  vc->flush_runs = vc->flush_runs + 1;
  vc->finished = 0;
  __threadfence();
}

// Static degree tiers of a graph for the bottom-up pass (degrees never change).
__global__ void k_b_tiers(const int32_t* __restrict__ deg, int64_t V, int small_max, int large_min,
                          uint32_t* __restrict__ lightbits, int32_t* __restrict__ mid, int32_t* __restrict__ large,
                          int32_t* __restrict__ counts) {
  const int lane = threadIdx.x & 31;
  const int64_t nth = (int64_t)gridDim.x * blockDim.x;
  for (int64_t base = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) & ~31ll; base < V; base += nth) {
    const int64_t v = base + lane;
    const int d = v < V ? deg[v] : 0;
    const unsigned lb = __ballot_sync(FULL, d >= 1 && d < small_max);
    if (lane == 0) lightbits[base >> 5] = lb;
    wappend(d >= small_max && d < large_min, (int)v, mid, &counts[0]);
    wappend(d >= large_min, (int)v, large, &counts[1]);
  }
}

// ------------------------------------------------------------- host -------
struct BatchWorkspace {
  int64_t V = 0;
  int W = 0, K = 0, cap_src = 0;
  void* slab = nullptr;
  BatchCtl* ctl = nullptr;
  BatchCtl* ctl_h = nullptr;
  BatchArgs args;
  int grid = 0, grid_flush = 0;
  size_t smem = 0, smem_flush = 0;
  cudaGraphExec_t exec = nullptr;
  cudaGraph_t graph = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  std::vector<unsigned long long> h_edges, h_verts;
  std::vector<int32_t> h_maxd;
  size_t x_bytes = 0, small_bytes = 0, stats_bytes = 0;
  void* x_ptr = nullptr;      // X (memset per run)
  void* small_ptr = nullptr;  // donebits + jfb[0..1] (memset per run)
  void* stats_ptr = nullptr;  // per-source stats (memset per run)
};

void destroy_batch_workspace(BatchWorkspace* w) {
  if (!w) return;
  if (w->exec) cudaGraphExecDestroy(w->exec);
  if (w->graph) cudaGraphDestroy(w->graph);
  if (w->slab) cudaFree(w->slab);
  if (w->ctl) cudaFree(w->ctl);
  if (w->ctl_h) cudaFreeHost(w->ctl_h);
  if (w->ev0) cudaEventDestroy(w->ev0);
  if (w->ev1) cudaEventDestroy(w->ev1);
  delete w;
}

static int words_for(int n_src) {
  int w = 1;
  while (w * 64 < n_src) w <<= 1;
  return w;
}
constexpr int MAX_BATCH = WMAX * 64;

// Appends this graph's whole batched traversal to `graph` as an independent
// branch: memsets -> seed -> while { expand, commit, flush } -> final flush.
int append_branch(ent_graph* g, BatchWorkspace* w, cudaGraph_t graph, cudaStream_t cap_stream) {
  cudaGraphNode_t prev = nullptr;
  auto add_memset = [&](void* p, size_t bytes) -> int {
    cudaMemsetParams mp = {};
    mp.dst = p;
    mp.value = 0;
    mp.elementSize = 1;
    mp.width = bytes;
    mp.height = 1;
    cudaGraphNode_t n;
    ENT_CUDA(cudaGraphAddMemsetNode(&n, graph, prev ? &prev : nullptr, prev ? 1 : 0, &mp));
    prev = n;
    return ENT_OK;
  };
  int rc;
  if ((rc = add_memset(w->x_ptr, w->x_bytes))) return rc;
  if ((rc = add_memset(w->small_ptr, w->small_bytes))) return rc;
  if ((rc = add_memset(w->stats_ptr, w->stats_bytes))) return rc;
  BatchArgs a0 = w->args;
  a0.use_cond = 0;
  {
    void* kargs[1] = {&a0};
    cudaKernelNodeParams kp = {};
    kp.func = (void*)k_b_seed;
    kp.gridDim = dim3(1);
    kp.blockDim = dim3(SEED_THREADS);
    kp.kernelParams = kargs;
    cudaGraphNode_t n;
    ENT_CUDA(cudaGraphAddKernelNode(&n, graph, &prev, 1, &kp));
    prev = n;
  }
  cudaGraphConditionalHandle handle;
  ENT_CUDA(cudaGraphConditionalHandleCreate(&handle, graph, 1, cudaGraphCondAssignDefault));
  cudaGraphNodeParams cp = {};
  cp.type = cudaGraphNodeTypeConditional;
  cp.conditional.handle = handle;
  cp.conditional.type = cudaGraphCondTypeWhile;
  cp.conditional.size = 1;
  cudaGraphNode_t cond_node;
  ENT_CUDA(cudaGraphAddNode(&cond_node, graph, &prev, 1, &cp));
  prev = cond_node;
  cudaGraph_t body = cp.conditional.phGraph_out[0];
  // Loop body: LOOP_UNROLL copies of expand -> commit -> flush in a chain (a
  // while-node iteration costs about 5 us more than the kernel nodes in it on
  // B200; every kernel treats a finished run as a no-op). The flush runs every
  // level and leaves at once unless the window is full or sources joined
  // (flush_now, clear_done): an always-launched kernel that exits costs less
  // than an IF node that is not taken (about 1.1 against 2.4 us).
  BatchArgs la = w->args;
  la.cond = handle;
  la.use_cond = 1;
  {
    int zero = 0;
    void* kl[1] = {&la};
    void* kf[2] = {&la, &zero};
    cudaGraphNode_t chain = nullptr;
    for (int u = 0; u < LOOP_UNROLL; ++u) {
      cudaKernelNodeParams kp = {};
      kp.blockDim = dim3(BB);
      kp.func = expand_kernel(w->W);
      kp.gridDim = dim3(w->grid);
      kp.sharedMemBytes = (unsigned)w->smem;
      kp.kernelParams = kl;
      cudaGraphNode_t n_expand, n_commit, n_flush;
      ENT_CUDA(cudaGraphAddKernelNode(&n_expand, body, chain ? &chain : nullptr, chain ? 1 : 0, &kp));
      kp.func = (void*)k_b_commit;
      kp.sharedMemBytes = 0;
      ENT_CUDA(cudaGraphAddKernelNode(&n_commit, body, &n_expand, 1, &kp));
      kp.func = (void*)k_b_flush;
      kp.gridDim = dim3(w->grid_flush);
      kp.sharedMemBytes = (unsigned)w->smem_flush;
      kp.kernelParams = kf;
      ENT_CUDA(cudaGraphAddKernelNode(&n_flush, body, &n_commit, 1, &kp));
      chain = n_flush;
    }
  }
  (void)cap_stream;
  {
    int fin = 1;
    void* kargs[2] = {&a0, &fin};
    cudaKernelNodeParams kp = {};
    kp.func = (void*)k_b_flush;
    kp.gridDim = dim3(w->grid_flush);
    kp.blockDim = dim3(BB);
    kp.sharedMemBytes = (unsigned)w->smem_flush;
    kp.kernelParams = kargs;
    cudaGraphNode_t n;
    ENT_CUDA(cudaGraphAddKernelNode(&n, graph, &prev, 1, &kp));
    prev = n;
  }
  return ENT_OK;
}

int create_batch_workspace(ent_graph* g, int n_src, BatchWorkspace** out) {
  BatchWorkspace* w = new BatchWorkspace();
  const int64_t V = g->V;
  const int W = words_for(n_src);
  w->V = V;
  w->W = W;
  w->K = KMAX;
  w->cap_src = W * 64;
  const int64_t Wd = (V + 31) / 32;
  auto al = [](size_t x) { return (x + 255) & ~(size_t)255; };
  const size_t sz_x = al(sizeof(unsigned long long) * V * W);
  const size_t sz_log = al(sizeof(unsigned long long) * V * W * (size_t)w->K);
  const size_t sz_bits = al(sizeof(uint32_t) * (Wd + 1));
  const size_t sz_q = al(sizeof(int32_t) * (V + 4));
  const size_t sz_mask = al(sizeof(unsigned long long) * W);
  const size_t sz_src = al(sizeof(int32_t) * w->cap_src);
  const size_t sz_st = al(sizeof(unsigned long long) * w->cap_src) * 2 + 2 * al(sizeof(int32_t) * w->cap_src);
  const size_t total = sz_x + sz_log + 4 * sz_bits + 6 * sz_q + 3 * sz_mask + sz_src + sz_st + 256;
  cudaError_t e = cudaMalloc(&w->slab, total);
  if (e != cudaSuccess) { destroy_batch_workspace(w); return fail(ENT_ERR_OOM, "batch workspace (%zu bytes) failed", total); }
  // Initialise on the graph's stream and wait (see create_workspace in
  // bfs_single.cu): the runs use other, non-blocking streams.
  e = cudaMemsetAsync(w->slab, 0, total, g->stream);
  if (e == cudaSuccess) e = cudaMalloc(&w->ctl, sizeof(BatchCtl));
  if (e == cudaSuccess) e = cudaMemsetAsync(w->ctl, 0, sizeof(BatchCtl), g->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(g->stream);
  if (e == cudaSuccess) e = cudaMallocHost(&w->ctl_h, sizeof(BatchCtl));
  if (e == cudaSuccess) e = cudaEventCreate(&w->ev0);
  if (e == cudaSuccess) e = cudaEventCreate(&w->ev1);
  if (e != cudaSuccess) { destroy_batch_workspace(w); return fail(ENT_ERR_OOM, "batch workspace setup failed"); }
  char* p = (char*)w->slab;
  BatchArgs& a = w->args;
  memset(&a, 0, sizeof(a));
  a.ctl = w->ctl;
  a.off = g->off;
  a.adj = g->trav;
  a.lead = g->lead;
  a.deg = g->deg;
  a.active = g->active;
  a.V = V;
  a.E = g->E;
  a.W = W;
  int lg = 0;
  while ((1 << lg) < W) ++lg;
  a.lgW = lg;
  a.K = w->K;
  a.X = (unsigned long long*)p; w->x_ptr = p; w->x_bytes = sz_x; p += sz_x;
  a.log = (unsigned long long*)p; p += sz_log;
  a.donebits = (uint32_t*)p; w->small_ptr = p; w->small_bytes = 3 * sz_bits; p += sz_bits;
  a.jfb[0] = (uint32_t*)p; p += sz_bits;
  a.jfb[1] = (uint32_t*)p; p += sz_bits;
  for (int i = 0; i < 2; ++i) { a.jf[i] = (int32_t*)p; p += sz_q; }
  for (int i = 0; i < 2; ++i) { a.heavy[i] = (int32_t*)p; p += sz_q; }
  uint32_t* lightbits = (uint32_t*)p; p += sz_bits;
  int32_t* mid = (int32_t*)p; p += sz_q;
  int32_t* large = (int32_t*)p; p += sz_q;
  int32_t* counts = (int32_t*)p; p += 256;
  a.lightbits = lightbits;
  a.mid = mid;
  a.large = large;
  a.mask = (const unsigned long long*)p; p += sz_mask;
  a.act[0] = (unsigned long long*)p; p += sz_mask;
  a.act[1] = (unsigned long long*)p; p += sz_mask;
  a.src = (const int32_t*)p; p += sz_src;
  w->stats_ptr = p;
  w->stats_bytes = sz_st;
  a.st_edges = (unsigned long long*)p; p += al(sizeof(unsigned long long) * w->cap_src);
  a.st_verts = (unsigned long long*)p; p += al(sizeof(unsigned long long) * w->cap_src);
  a.st_maxd = (int32_t*)p; p += al(sizeof(int32_t) * w->cap_src);
  a.join = (int32_t*)p; p += al(sizeof(int32_t) * w->cap_src);  // zeroed with the statistics
  a.box = nullptr;
  a.alpha = g->opts.batch_alpha;
  a.heavy_deg = g->opts.batch_heavy;
  a.max_levels = (int32_t)std::min<int64_t>(V + 2, 0x7ffffff0);
  w->smem = sizeof(unsigned long long) * std::max(W * (BB / 32), W);
  {
    const int blocks = (int)std::min<int64_t>((V + BB - 1) / BB, (int64_t)g->num_sms * 8);
    k_b_tiers<<<blocks, BB, 0, g->stream>>>(g->deg, V, g->opts.batch_small_max, g->opts.batch_large_min, lightbits,
                                             mid, large, counts);
    g_kernel_launches++;
    int32_t hc[2] = {0, 0};
    e = cudaMemcpyAsync(hc, counts, sizeof(hc), cudaMemcpyDeviceToHost, g->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(g->stream);
    if (e != cudaSuccess) { destroy_batch_workspace(w); return fail(ENT_ERR_CUDA, "tier build failed: %s", cudaGetErrorString(e)); }
    a.n_mid = hc[0];
    a.n_large = hc[1];
  }
  int occ = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, expand_kernel(W), BB, w->smem);
  if (occ < 1) occ = 1;
  // small graphs get small grids so that the branches of a multi-graph
  // launch can run side by side
  const int64_t want = std::max<int64_t>(1, (V + BB * 8 - 1) / (BB * 8));
  w->grid = (int)std::min<int64_t>((int64_t)g->num_sms * occ, want);
  w->grid_flush = (int)std::min<int64_t>((int64_t)g->num_sms * 3, std::max<int64_t>(1, (V + 1023) / 1024));
  // tile and degrees; per source: reached vertices, their degree sum, deepest level
  w->smem_flush = FLUSH_TILE_BYTES + (size_t)W * 64 * (4 + 8 + 4) + 16;
  {
    e = cudaFuncSetAttribute(k_b_flush, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)w->smem_flush);
    if (e != cudaSuccess) { destroy_batch_workspace(w); return fail(ENT_ERR_CUDA, "flush smem attribute failed"); }
  }
  w->h_edges.resize(w->cap_src);
  w->h_verts.resize(w->cap_src);
  w->h_maxd.resize(w->cap_src);
  *out = w;
  return ENT_OK;
}

static int ensure_batch(ent_graph* g, int n_src) {
  if (g->bws && g->bws->cap_src >= n_src && g->bws->W == words_for(n_src)) return ENT_OK;
  if (g->bws) {
    cudaStreamSynchronize(g->stream);
    destroy_batch_workspace(g->bws);
    g->bws = nullptr;
  }
  int rc = create_batch_workspace(g, n_src, &g->bws);
  if (rc != ENT_OK) return rc;
  BatchWorkspace* w = g->bws;
  ENT_CUDA(cudaGraphCreate(&w->graph, 0));
  rc = append_branch(g, w, w->graph, g->stream);
  if (rc != ENT_OK) return rc;
  ENT_CUDA(cudaGraphInstantiate(&w->exec, w->graph, 0));
  return ENT_OK;
}

// Kernels one finished graph-driven run launched: seed, final flush, and
// expand, commit and flush per loop body run (the flush leaves at once on
// most levels; bodies after the end only cost their launches).
static int64_t run_launches(const BatchCtl& h) { return 2 + 3 * (int64_t)h.iters; }

// Uploads sources, mask and the output pointer (the kernels read them from
// device memory, so one instantiated graph serves every batch).
int stage_request(ent_graph*, BatchWorkspace* w, const int32_t* src, int32_t n_src, int32_t* depth_dev,
                  cudaStream_t s, const int32_t* row_map_dev, bool bytes) {
  std::vector<unsigned long long> mask(w->W, 0);
  for (int i = 0; i < n_src; ++i) mask[i >> 6] |= 1ull << (i & 63);
  ENT_CUDA(cudaMemcpyAsync((void*)w->args.mask, mask.data(), sizeof(unsigned long long) * w->W, cudaMemcpyHostToDevice, s));
  ENT_CUDA(cudaMemcpyAsync((void*)w->args.src, src, sizeof(int32_t) * n_src, cudaMemcpyHostToDevice, s));
  BatchCtl init = {};
  init.n_src = n_src;
  init.depth = depth_dev;
  init.row_map = row_map_dev;
  init.out_bytes = bytes ? 1 : 0;
  ENT_CUDA(cudaMemcpyAsync(w->ctl, &init, sizeof(BatchCtl), cudaMemcpyHostToDevice, s));
  return ENT_OK;
}

// Status of a finished batch from its device error word: bit 16 = a depth
// above 254 met while writing byte rows (those rows hold its low byte).
static int batch_status(int32_t err) {
  if (err & 16) return fail(ENT_ERR_UNSUPPORTED, "a source reaches a depth above 254; byte depths hold 0..254");
  if (err) return fail(ENT_ERR_TIMEOUT, "batched traversal reported error flags 0x%x", err);
  return ENT_OK;
}

static int read_batch_stats(ent_graph* g, BatchWorkspace* w, int32_t n_src, cudaStream_t s, ent_stats* stats) {
  ENT_CUDA(cudaMemcpyAsync(w->ctl_h, w->ctl, sizeof(BatchCtl), cudaMemcpyDeviceToHost, s));
  ENT_CUDA(cudaMemcpyAsync(w->h_edges.data(), w->args.st_edges, sizeof(unsigned long long) * n_src, cudaMemcpyDeviceToHost, s));
  ENT_CUDA(cudaMemcpyAsync(w->h_verts.data(), w->args.st_verts, sizeof(unsigned long long) * n_src, cudaMemcpyDeviceToHost, s));
  ENT_CUDA(cudaMemcpyAsync(w->h_maxd.data(), w->args.st_maxd, sizeof(int32_t) * n_src, cudaMemcpyDeviceToHost, s));
  ENT_CUDA(cudaStreamSynchronize(s));
  float ms = 0.f;
  cudaEventElapsedTime(&ms, w->ev0, w->ev1);
  for (int i = 0; i < n_src; ++i) {
    stats[i].reached_vertices = (int64_t)w->h_verts[i];
    stats[i].traversed_edges = (int64_t)w->h_edges[i];
    stats[i].levels = w->h_maxd[i] + 1;
    stats[i].td_levels = w->ctl_h->td_levels;
    stats[i].bu_levels = w->ctl_h->bu_levels;
    stats[i].status = w->ctl_h->err;
    stats[i].device_ms = ms;
    stats[i].narrow_levels = 0;
    stats[i].launches = (int32_t)run_launches(*w->ctl_h);  // shared by the batch
  }
  g_kernel_launches += run_launches(*w->ctl_h);
  return batch_status(w->ctl_h->err);
}

// Per-source statistics of a finished run of workspace w (the caller has
// waited for the run; copies on stream s and synchronises it).
int batch_source_stats(BatchWorkspace* w, int32_t n_src, cudaStream_t s, ent_stats* stats) {
  ENT_CUDA(cudaMemcpyAsync(w->ctl_h, w->ctl, sizeof(BatchCtl), cudaMemcpyDeviceToHost, s));
  ENT_CUDA(cudaMemcpyAsync(w->h_edges.data(), w->args.st_edges, sizeof(unsigned long long) * n_src, cudaMemcpyDeviceToHost, s));
  ENT_CUDA(cudaMemcpyAsync(w->h_verts.data(), w->args.st_verts, sizeof(unsigned long long) * n_src, cudaMemcpyDeviceToHost, s));
  ENT_CUDA(cudaMemcpyAsync(w->h_maxd.data(), w->args.st_maxd, sizeof(int32_t) * n_src, cudaMemcpyDeviceToHost, s));
  ENT_CUDA(cudaStreamSynchronize(s));
  for (int i = 0; i < n_src; ++i) {
    stats[i].reached_vertices = (int64_t)w->h_verts[i];
    stats[i].traversed_edges = (int64_t)w->h_edges[i];
    stats[i].levels = w->h_maxd[i] + 1;
    stats[i].td_levels = w->ctl_h->td_levels;
    stats[i].bu_levels = w->ctl_h->bu_levels;
    stats[i].status = w->ctl_h->err;
    stats[i].device_ms = 0;
    stats[i].narrow_levels = 0;
    stats[i].launches = (int32_t)run_launches(*w->ctl_h);  // shared by the batch
  }
  g_kernel_launches += run_launches(*w->ctl_h);
  return batch_status(w->ctl_h->err);
}

int batch_max_sources(const BatchWorkspace* w) { return w->cap_src; }

void set_join_box(BatchWorkspace* w, JoinBox* box_dev) { w->args.box = box_dev; }

int batch_joined(const BatchWorkspace* w) { return w->ctl_h->joined; }

// Whether a batch on g runs as concurrent single-source lanes: by option, and
// in auto mode by the graph's depth, probed once per graph.
static int choose_deep(ent_graph* g, const int32_t* src, int32_t n_src, bool* deep) {
  *deep = false;
  if (g->opts.batch_deep == 0) return ENT_OK;
  if (g->opts.batch_deep == 2) {
    *deep = true;
    return ENT_OK;
  }
  if (g->probe_levels < 0) {
    int32_t lv = 0;
    const int rc = probe_graph_levels(g, src, n_src, &lv);
    if (rc != ENT_OK) return rc;
    g->probe_levels = lv;
  }
  *deep = g->probe_levels >= g->opts.batch_deep_levels;
  return ENT_OK;
}

// One staged run of workspace w driven level by level from the host (the
// kernels of the CUDA-graph loop, launched directly): memsets, seed, then
// expand, commit and flush per level while the run is not done, and the final
// flush. With `out`, one trace row per level (at most max_levels, the final
// flush as level -1 if room is left) and *n_levels rows; with total_ms, the
// device time of the whole run. Synchronises s.
static int host_batch_loop(BatchWorkspace* w, int64_t E, BatchArgs a, cudaStream_t s, ent_level_trace* out,
                           int32_t max_levels, int32_t* n_levels, float* total_ms) {
  ENT_CUDA(cudaMemsetAsync(w->x_ptr, 0, w->x_bytes, s));
  ENT_CUDA(cudaMemsetAsync(w->small_ptr, 0, w->small_bytes, s));
  ENT_CUDA(cudaMemsetAsync(w->stats_ptr, 0, w->stats_bytes, s));
  a.use_cond = 0;
  cudaEvent_t e[4];
  for (int i = 0; i < 4; ++i) ENT_CUDA(cudaEventCreate(&e[i]));
  ENT_CUDA(cudaEventRecord(e[3], s));
  k_b_seed<<<1, SEED_THREADS, 0, s>>>(a);
  int n = 0;
  int64_t iters = 0;  // level-loop iterations: expand, commit and flush launches each
  for (;;) {
    ENT_CUDA(cudaMemcpyAsync(w->ctl_h, w->ctl, sizeof(BatchCtl), cudaMemcpyDeviceToHost, s));
    ENT_CUDA(cudaStreamSynchronize(s));
    const BatchCtl h = *w->ctl_h;
    if (h.done || iters >= max_levels) break;
    ++iters;
    if (out) {
      ent_level_trace& t = out[n];
      t.level = h.level;
      t.direction = h.dir;
      t.bu_sweep = h.dir;
      t.pad = 0;
      t.frontier_vertices = h.n_jf[h.cur];
      t.frontier_edges = h.m_f;
      t.unvisited_queued = E - h.m_done;
    }
    ENT_CUDA(cudaEventRecord(e[0], s));
    if (w->W > 2) k_b_expand<true><<<w->grid, BB, w->smem, s>>>(a);
    else k_b_expand<false><<<w->grid, BB, w->smem, s>>>(a);
    ENT_CUDA(cudaEventRecord(e[1], s));
    k_b_commit<<<w->grid, BB, 0, s>>>(a);
    k_b_flush<<<w->grid_flush, BB, w->smem_flush, s>>>(a, 0);
    ENT_CUDA(cudaEventRecord(e[2], s));
    ENT_CUDA(cudaGetLastError());
    if (out) {
      ENT_CUDA(cudaEventSynchronize(e[2]));
      float ta = 0, tb = 0;
      cudaEventElapsedTime(&ta, e[0], e[1]);
      cudaEventElapsedTime(&tb, e[1], e[2]);
      out[n].expand_ms = ta;
      out[n].inspect_ms = tb;
      ++n;
    }
  }
  ENT_CUDA(cudaEventRecord(e[0], s));
  k_b_flush<<<w->grid_flush, BB, w->smem_flush, s>>>(a, 1);
  ENT_CUDA(cudaEventRecord(e[1], s));
  ENT_CUDA(cudaStreamSynchronize(s));
  float tf = 0, tt = 0;
  cudaEventElapsedTime(&tf, e[0], e[1]);
  cudaEventElapsedTime(&tt, e[3], e[1]);
  if (total_ms) *total_ms = tt;
  if (out && n < max_levels) {
    ent_level_trace& t = out[n];
    memset(&t, 0, sizeof(t));
    t.level = -1;  // the final flush (depth rows + per-source stats)
    t.inspect_ms = tf;
    ++n;
  }
  for (int i = 0; i < 4; ++i) cudaEventDestroy(e[i]);
  g_kernel_launches += 2 + 3 * iters;
  if (n_levels) *n_levels = out ? n : (int32_t)iters;
  if (w->ctl_h->err) return fail(ENT_ERR_TIMEOUT, "batched traversal error flags 0x%x", w->ctl_h->err);
  return ENT_OK;
}

int run_bfs_batch(ent_graph* g, const int32_t* src, int32_t n_src, int32_t* depth_dev, cudaStream_t stream,
                  ent_stats* stats, bool bytes) {
  for (int i = 0; i < n_src; ++i)
    if (src[i] < 0 || src[i] >= g->V) return fail(ENT_ERR_INVALID_ARG, "source %d out of range", src[i]);
  bool deep = false;
  int rc = choose_deep(g, src, n_src, &deep);
  if (rc != ENT_OK) return rc;
  if (deep) return run_bfs_deep(g, src, n_src, depth_dev, bytes, stream, stats);
  rc = ensure_batch(g, n_src);
  if (rc != ENT_OK) return rc;
  BatchWorkspace* w = g->bws;
  cudaStream_t s = stream ? stream : g->stream;
  rc = stage_request(g, w, src, n_src, depth_dev, s, nullptr, bytes);
  if (rc != ENT_OK) return rc;
  ENT_CUDA(cudaEventRecord(w->ev0, s));
  ENT_CUDA(cudaGraphLaunch(w->exec, s));
  ENT_CUDA(cudaEventRecord(w->ev1, s));
  if (stats) return read_batch_stats(g, w, n_src, s, stats);
  g_kernel_launches += 2;
  return ENT_OK;
}

}  // namespace ent

using namespace ent;

extern "C" {

int ent_bfs_batch_device(ent_graph* g, const int32_t* src, int32_t n_src, int32_t* depth_dev, void* stream,
                         ent_stats* stats) {
  ent::NvtxRange nvtx_range("ent_bfs_batch_device");
  clear_error();
  if (!g || !src || !depth_dev || n_src < 1) return fail(ENT_ERR_INVALID_ARG, "bad arguments");
  if (n_src > MAX_BATCH) return fail(ENT_ERR_UNSUPPORTED, "at most %d sources per batch", MAX_BATCH);
  std::lock_guard<std::mutex> lk(g->mu);
  DeviceGuard dg(g->device);
  return run_bfs_batch(g, src, n_src, depth_dev, (cudaStream_t)stream, stats);
}

int ent_bfs_batch_device_u8(ent_graph* g, const int32_t* src, int32_t n_src, uint8_t* depth_dev, void* stream,
                            ent_stats* stats) {
  ent::NvtxRange nvtx_range("ent_bfs_batch_device_u8");
  clear_error();
  if (!g || !src || !depth_dev || n_src < 1) return fail(ENT_ERR_INVALID_ARG, "bad arguments");
  if (n_src > MAX_BATCH) return fail(ENT_ERR_UNSUPPORTED, "at most %d sources per batch", MAX_BATCH);
  std::lock_guard<std::mutex> lk(g->mu);
  DeviceGuard dg(g->device);
  return run_bfs_batch(g, src, n_src, reinterpret_cast<int32_t*>(depth_dev), (cudaStream_t)stream, stats, true);
}

// Host rows of either type: the batch writes them into the graph's staging
// buffer on the device, then one copy brings them back.
static int batch_to_host(ent_graph* g, const int32_t* src, int32_t n_src, void* depth_out, bool bytes,
                         ent_stats* stats) {
  clear_error();
  if (!g || !src || n_src < 1) return fail(ENT_ERR_INVALID_ARG, "bad arguments");
  if (n_src > MAX_BATCH) return fail(ENT_ERR_UNSUPPORTED, "at most %d sources per batch", MAX_BATCH);
  std::lock_guard<std::mutex> lk(g->mu);
  DeviceGuard dg(g->device);
  const size_t need = (bytes ? 1 : sizeof(int32_t)) * (size_t)n_src * g->V;
  if (g->stage_cap < need) {
    if (g->stage) cudaFree(g->stage);
    g->stage = nullptr;
    g->stage_cap = 0;
    ENT_CUDA(cudaMalloc(&g->stage, need));
    g->stage_cap = need;
  }
  std::vector<ent_stats> local(stats ? 0 : n_src);
  int rc = run_bfs_batch(g, src, n_src, static_cast<int32_t*>(g->stage), g->stream, stats ? stats : local.data(), bytes);
  // a byte row past depth 254 still holds the other sources' complete rows
  if (rc != ENT_OK && !(bytes && rc == ENT_ERR_UNSUPPORTED)) return rc;
  if (depth_out) ENT_CUDA(cudaMemcpyAsync(depth_out, g->stage, need, cudaMemcpyDeviceToHost, g->stream));
  ENT_CUDA(cudaStreamSynchronize(g->stream));
  return rc;
}

int ent_bfs_batch(ent_graph* g, const int32_t* src, int32_t n_src, int32_t* depth_out, ent_stats* stats) {
  ent::NvtxRange nvtx_range("ent_bfs_batch");
  return batch_to_host(g, src, n_src, depth_out, false, stats);
}

int ent_bfs_batch_u8(ent_graph* g, const int32_t* src, int32_t n_src, uint8_t* depth_out, ent_stats* stats) {
  ent::NvtxRange nvtx_range("ent_bfs_batch_u8");
  return batch_to_host(g, src, n_src, depth_out, true, stats);
}

// Host-driven run of a batch with CUDA events per level (tracing aid; same
// kernels and results as ent_bfs_batch_device).
int ent_bfs_batch_trace(ent_graph* g, const int32_t* src, int32_t n_src, int32_t* depth_dev, ent_level_trace* out,
                        int32_t max_levels, int32_t* n_levels) {
  clear_error();
  if (!g || !src || !depth_dev || !out || !n_levels || n_src < 1 || max_levels < 1)
    return fail(ENT_ERR_INVALID_ARG, "bad arguments");
  if (n_src > MAX_BATCH) return fail(ENT_ERR_UNSUPPORTED, "at most %d sources per batch", MAX_BATCH);
  for (int i = 0; i < n_src; ++i)
    if (src[i] < 0 || src[i] >= g->V) return fail(ENT_ERR_INVALID_ARG, "source %d out of range", src[i]);
  std::lock_guard<std::mutex> lk(g->mu);
  DeviceGuard dg(g->device);
  int rc = ensure_batch(g, n_src);
  if (rc != ENT_OK) return rc;
  BatchWorkspace* w = g->bws;
  rc = stage_request(g, w, src, n_src, depth_dev, g->stream, nullptr, false);
  if (rc != ENT_OK) return rc;
  return host_batch_loop(w, g->E, w->args, g->stream, out, max_levels, n_levels, nullptr);
}

}  // extern "C"

// Many graphs, one launch. The graphs share no vertex, so one batched
// traversal over their disjoint union computes every graph's rows at once:
// source slot s starts at the s-th source of every graph (a seed list), and a
// slot's bits never leave the graph they started in. Each level then runs one
// expand and one commit for all graphs together, over the whole GPU, instead
// of one small launch chain per graph. The descriptor table (MultiPart) says
// where each graph sits in its union (first vertex, first edge); graph k's
// sources are slots 0 .. n_src[k]-1. Graphs are grouped by the width class of
// their request (64-bit words per vertex), one union per class, so a narrow
// request never carries a wide one's words; each class is one branch of the
// plan's CUDA graph. A graph's slots past its own sources repeat them
// (slot s starts at source s % n_src[k]): every slot then reaches every
// graph's components as in an ordinary batch, and vertices stop needing bits
// exactly as they would there. Those rows are computed and never returned.
struct MultiPart {
  int32_t graph;   // index in the plan's graph list
  int64_t v0, e0;  // first vertex and first edge of the graph in its union
};

struct MultiUnion {
  ent_graph* u = nullptr;    // the union's CSR and traversal arrays
  BatchWorkspace* w = nullptr;
  int32_t* depth = nullptr;  // [slots][u->V]
  int32_t* seeds = nullptr;  // seed vertices [n_seed], then their slots [n_seed]
  int32_t slots = 0, n_seed = 0;
  std::vector<MultiPart> parts;
};

// Uploads a union's run state (its sources are the plan's seed list, already
// on the device) and source mask on stream s.
static int stage_union(const MultiUnion& mu, cudaStream_t s) {
  BatchWorkspace* w = mu.w;
  std::vector<unsigned long long> mask(w->W, 0);
  for (int i = 0; i < mu.slots; ++i) mask[i >> 6] |= 1ull << (i & 63);
  ENT_CUDA(cudaMemcpyAsync((void*)w->args.mask, mask.data(), sizeof(unsigned long long) * w->W, cudaMemcpyHostToDevice, s));
  BatchCtl init = {};
  init.n_src = mu.slots;
  init.n_seed = mu.n_seed;
  init.depth = mu.depth;
  ENT_CUDA(cudaMemcpyAsync(w->ctl, &init, sizeof(BatchCtl), cudaMemcpyHostToDevice, s));
  return ENT_OK;
}

// The union's direction threshold (batch alpha), measured once at creation.
// A union's frontier at level L sums its graphs' level-L frontiers, so the
// threshold that suits one graph alone need not suit the sum: on 48 R-MAT
// graphs of scales 12-20, alpha 4 runs level 1 top-down over 72M frontier
// edges in 6.7 ms where bottom-up takes 2.5 ms. Candidates are the value of
// the member with the most edges and 2..32, each run twice host-driven; the
// lowest time wins. Depths never depend on it. A union deeper than 64 levels
// keeps the member's value: its frontiers are small, and each candidate would
// cost a long host-driven run.
static int tune_union_alpha(MultiUnion& mu, cudaStream_t s) {
  BatchWorkspace* w = mu.w;
  const double own = w->args.alpha;
  std::vector<double> cand = {own};
  for (double c : {2.0, 4.0, 8.0, 16.0, 32.0})
    if (c != own) cand.push_back(c);
  double best = own;
  float best_ms = 0.f;
  for (size_t i = 0; i < cand.size(); ++i) {
    BatchArgs a = w->args;
    a.alpha = cand[i];
    float t = 0.f;
    for (int rep = 0; rep < 2; ++rep) {
      int rc = stage_union(mu, s);
      if (rc != ENT_OK) return rc;
      float ms = 0.f;
      int32_t levels = 0;
      rc = host_batch_loop(w, mu.u->E, a, s, nullptr, INT32_MAX, &levels, &ms);
      if (rc != ENT_OK) return rc;
      if (i == 0 && levels > 64) return ENT_OK;
      t = rep == 0 ? ms : std::min(t, ms);
    }
    if (i == 0 || t < best_ms) {
      best_ms = t;
      best = cand[i];
    }
  }
  w->args.alpha = best;
  return ENT_OK;
}

struct ent_multi {
  std::vector<ent_graph*> graphs;
  std::vector<int32_t> n_src;
  std::vector<int64_t> vcount;  // V of each graph: after creation the plan reads no member graph
  std::vector<MultiUnion> unions;
  std::vector<std::pair<int32_t, int32_t>> where;  // graph k: (union, part)
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  int device = 0;
};

static void multi_free(ent_multi* m) {
  if (!m) return;
  DeviceGuard dg(m->device);
  if (m->stream) cudaStreamSynchronize(m->stream);
  if (m->exec) cudaGraphExecDestroy(m->exec);
  if (m->graph) cudaGraphDestroy(m->graph);
  for (MultiUnion& mu : m->unions) {
    destroy_batch_workspace(mu.w);
    if (mu.depth) cudaFree(mu.depth);
    if (mu.seeds) cudaFree(mu.seeds);
    if (mu.u) ent_graph_destroy(mu.u);
  }
  if (m->ev0) cudaEventDestroy(m->ev0);
  if (m->ev1) cudaEventDestroy(m->ev1);
  if (m->stream) cudaStreamDestroy(m->stream);
  delete m;
}

// Graph k's offsets into the union's, shifted by the edges before it (n = V_k + 1
// entries; the last equals the next graph's first, so the overlap is harmless).
__global__ void k_union_off(const int64_t* __restrict__ off, int64_t n, int64_t e0, int64_t* __restrict__ out) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    out[i] = off[i] + e0;
}

// Graph k's neighbour ids into the union's, shifted by the vertices before it.
__global__ void k_union_adj(const int32_t* __restrict__ adj, int64_t n, int32_t v0, int32_t* __restrict__ out) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    out[i] = adj[i] + v0;
}

// Builds union mu (its parts listed) on the device: CSR by shifted copies of
// the member graphs', then degrees, traversal order and lead entries as for
// any graph. Batch options are those of the member with the most edges.
static int build_union(ent_multi* m, MultiUnion& mu) {
  int64_t V = 0, E = 0;
  int32_t big = mu.parts[0].graph;
  for (MultiPart& p : mu.parts) {
    const ent_graph* g = m->graphs[p.graph];
    p.v0 = V;
    p.e0 = E;
    V += g->V;
    E += g->E;
    if (g->E > m->graphs[big]->E) big = p.graph;
  }
  if (V > (int64_t)INT32_MAX - 64)
    return fail(ENT_ERR_UNSUPPORTED, "graphs of one width class hold %lld vertices together; ids are int32",
                (long long)V);
  ent_graph* u = new ent_graph();
  u->device = m->device;
  mu.u = u;  // freed with the plan on any error below
  int rc = graph_alloc(u, V, E);
  if (rc != ENT_OK) return rc;
  ENT_CUDA(cudaStreamCreateWithFlags(&u->stream, cudaStreamNonBlocking));
  int sms = 0;
  ENT_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, m->device));
  auto blocks = [&](int64_t n) { return (int)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, (int64_t)sms * 16)); };
  for (const MultiPart& p : mu.parts) {
    const ent_graph* g = m->graphs[p.graph];
    k_union_off<<<blocks(g->V + 1), 256, 0, u->stream>>>(g->off, g->V + 1, p.e0, u->off + p.v0);
    g_kernel_launches++;
    if (g->E > 0) {
      k_union_adj<<<blocks(g->E), 256, 0, u->stream>>>(g->adj, g->E, (int32_t)p.v0, u->adj + p.e0);
      g_kernel_launches++;
    }
    ENT_CUDA(cudaGetLastError());
  }
  rc = graph_finish(u);
  if (rc != ENT_OK) return rc;
  u->opts = m->graphs[big]->opts;
  return ENT_OK;
}

extern "C" {

int ent_multi_create(ent_graph* const* graphs, int32_t n_graphs, const int32_t* src, const int32_t* n_src,
                     ent_multi** out) {
  clear_error();
  if (!graphs || !src || !n_src || !out || n_graphs < 1) return fail(ENT_ERR_INVALID_ARG, "bad arguments");
  *out = nullptr;
  for (int k = 0; k < n_graphs; ++k)
    if (!graphs[k]) return fail(ENT_ERR_INVALID_ARG, "graph %d is null", k);
  // a graph may be listed more than once (several source sets): every entry
  // is its own part of a union
  const int dev = graphs[0]->device;
  for (int k = 0; k < n_graphs; ++k) {
    if (graphs[k]->device != dev) return fail(ENT_ERR_INVALID_ARG, "all graphs must be on one GPU");
    if (n_src[k] < 1 || n_src[k] > MAX_BATCH) return fail(ENT_ERR_INVALID_ARG, "graph %d: bad source count", k);
  }
  int64_t at = 0;
  for (int k = 0; k < n_graphs; ++k) {
    for (int i = 0; i < n_src[k]; ++i)
      if (src[at + i] < 0 || src[at + i] >= graphs[k]->V)
        return fail(ENT_ERR_INVALID_ARG, "graph %d: source %d out of range", k, src[at + i]);
    at += n_src[k];
  }
  DeviceGuard dg(dev);
  ent_multi* m = new ent_multi();
  m->device = dev;
  m->graphs.assign(graphs, graphs + n_graphs);
  m->n_src.assign(n_src, n_src + n_graphs);
  for (int k = 0; k < n_graphs; ++k) m->vcount.push_back(graphs[k]->V);
  m->where.resize(n_graphs);
  // one union per width class, graphs in request order within it
  for (int cls = 1; cls <= WMAX; cls <<= 1) {
    MultiUnion mu;
    for (int k = 0; k < n_graphs; ++k)
      if (words_for(n_src[k]) == cls) {
        m->where[k] = {(int32_t)m->unions.size(), (int32_t)mu.parts.size()};
        mu.parts.push_back({k, 0, 0});
        mu.slots = std::max(mu.slots, n_src[k]);
      }
    if (mu.parts.empty()) continue;
    mu.n_seed = mu.slots * (int32_t)mu.parts.size();
    m->unions.push_back(std::move(mu));
  }
  cudaError_t e = cudaStreamCreateWithFlags(&m->stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaEventCreate(&m->ev0);
  if (e == cudaSuccess) e = cudaEventCreate(&m->ev1);
  if (e == cudaSuccess) e = cudaGraphCreate(&m->graph, 0);
  if (e != cudaSuccess) { multi_free(m); return fail(ENT_ERR_CUDA, "multi setup: %s", cudaGetErrorString(e)); }
  std::vector<int64_t> first(n_graphs + 1, 0);
  for (int k = 0; k < n_graphs; ++k) first[k + 1] = first[k] + n_src[k];
  for (MultiUnion& mu : m->unions) {
    int rc = build_union(m, mu);
    if (rc == ENT_OK) rc = create_batch_workspace(mu.u, mu.slots, &mu.w);
    if (rc != ENT_OK) { multi_free(m); return rc; }
    // seed list: slot i of graph k starts at its source i % n_src[k]
    std::vector<int32_t> h(2 * (size_t)mu.n_seed);
    size_t j = 0;
    for (const MultiPart& p : mu.parts) {
      const int32_t n = n_src[p.graph];
      for (int32_t i = 0; i < mu.slots; ++i, ++j) {
        h[j] = (int32_t)p.v0 + src[first[p.graph] + i % n];
        h[mu.n_seed + j] = i;
      }
    }
    e = cudaMalloc(&mu.seeds, sizeof(int32_t) * h.size());
    if (e == cudaSuccess) e = cudaMemcpy(mu.seeds, h.data(), sizeof(int32_t) * h.size(), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMalloc(&mu.depth, sizeof(int32_t) * (size_t)mu.slots * mu.u->V);
    if (e != cudaSuccess) { multi_free(m); return fail(ENT_ERR_OOM, "multi seed list or output allocation failed"); }
    mu.w->args.src = mu.seeds;
    mu.w->args.seed_slot = mu.seeds + mu.n_seed;
    rc = tune_union_alpha(mu, m->stream);
    if (rc == ENT_OK) rc = append_branch(mu.u, mu.w, m->graph, m->stream);
    if (rc != ENT_OK) { multi_free(m); return rc; }
  }
  e = cudaGraphInstantiate(&m->exec, m->graph, 0);
  if (e != cudaSuccess) { multi_free(m); return fail(ENT_ERR_CUDA, "multi instantiate: %s", cudaGetErrorString(e)); }
  *out = m;
  return ENT_OK;
}

int ent_multi_run(ent_multi* m, double* device_ms) {
  ent::NvtxRange nvtx_range("ent_multi_run");
  clear_error();
  if (!m) return fail(ENT_ERR_INVALID_ARG, "null plan");
  DeviceGuard dg(m->device);
  for (MultiUnion& mu : m->unions) {
    const int rc = stage_union(mu, m->stream);
    if (rc != ENT_OK) return rc;
  }
  ENT_CUDA(cudaEventRecord(m->ev0, m->stream));
  ENT_CUDA(cudaGraphLaunch(m->exec, m->stream));
  ENT_CUDA(cudaEventRecord(m->ev1, m->stream));
  ENT_CUDA(cudaStreamSynchronize(m->stream));
  float ms = 0.f;
  cudaEventElapsedTime(&ms, m->ev0, m->ev1);
  if (device_ms) *device_ms = ms;
  for (size_t i = 0; i < m->unions.size(); ++i) {
    BatchWorkspace* w = m->unions[i].w;
    ENT_CUDA(cudaMemcpy(w->ctl_h, w->ctl, sizeof(BatchCtl), cudaMemcpyDeviceToHost));
    g_kernel_launches += run_launches(*w->ctl_h);
    if (w->ctl_h->err) return fail(ENT_ERR_TIMEOUT, "width class %zu: batched traversal error flags 0x%x", i, w->ctl_h->err);
  }
  return ENT_OK;
}

int ent_multi_depths(ent_multi* m, int32_t k, int32_t* depth_out) {
  clear_error();
  if (!m || !depth_out || k < 0 || k >= (int32_t)m->graphs.size()) return fail(ENT_ERR_INVALID_ARG, "bad arguments");
  DeviceGuard dg(m->device);
  const MultiUnion& mu = m->unions[m->where[k].first];
  const MultiPart& p = mu.parts[m->where[k].second];
  const size_t width = sizeof(int32_t) * (size_t)m->vcount[k], pitch = sizeof(int32_t) * (size_t)mu.u->V;
  int max_pitch = 0;
  ENT_CUDA(cudaDeviceGetAttribute(&max_pitch, cudaDevAttrMaxPitch, m->device));
  if (pitch <= (size_t)max_pitch) {
    ENT_CUDA(cudaMemcpy2D(depth_out, width, mu.depth + p.v0, pitch, width, m->n_src[k], cudaMemcpyDeviceToHost));
  } else {
    for (int32_t i = 0; i < m->n_src[k]; ++i)
      ENT_CUDA(cudaMemcpy(depth_out + (size_t)i * m->vcount[k], mu.depth + (size_t)i * mu.u->V + p.v0, width,
                          cudaMemcpyDeviceToHost));
  }
  return ENT_OK;
}

int ent_multi_trace(ent_multi* m, int32_t k, ent_level_trace* out, int32_t max_levels, int32_t* n_levels) {
  clear_error();
  if (!m || !out || !n_levels || max_levels < 1 || k < 0 || k >= (int32_t)m->graphs.size())
    return fail(ENT_ERR_INVALID_ARG, "bad arguments");
  DeviceGuard dg(m->device);
  MultiUnion& mu = m->unions[m->where[k].first];
  const int rc = stage_union(mu, m->stream);
  if (rc != ENT_OK) return rc;
  return host_batch_loop(mu.w, mu.u->E, mu.w->args, m->stream, out, max_levels, n_levels, nullptr);
}

int ent_multi_destroy(ent_multi* m) {
  multi_free(m);
  return ENT_OK;
}

int ent_bfs_multi(ent_graph* const* graphs, int32_t n_graphs, const int32_t* src, const int32_t* n_src,
                  int32_t* const* depth_out) {
  ent::NvtxRange nvtx_range("ent_bfs_multi");
  ent_multi* m = nullptr;
  int rc = ent_multi_create(graphs, n_graphs, src, n_src, &m);
  if (rc != ENT_OK) return rc;
  rc = ent_multi_run(m, nullptr);
  for (int k = 0; rc == ENT_OK && k < n_graphs; ++k)
    if (depth_out && depth_out[k]) rc = ent_multi_depths(m, k, depth_out[k]);
  multi_free(m);
  return rc;
}

}  // extern "C"
