/*
 * CPU oracle for the BFS hot path — TEST INFRASTRUCTURE ONLY (see oracle.h).
 * Never linked into, or called by, the product library.
 */
#include "oracle.h"

#include <omp.h>
#include <stdlib.h>
#include <string.h>

int oracle_max_threads(void) { return omp_get_max_threads(); }

/* Serial queue BFS: the level loop of bfs_gpu_opt.cuh:99-282 in its plainest
 * form. A vertex gets depth L+1 the first time a depth-L vertex reaches it. */
int oracle_bfs(int64_t V, const int64_t* off, const int32_t* adj, int32_t src, int32_t* depth, int32_t* parent) {
  if (V <= 0 || src < 0 || src >= V) return -1;
  int32_t* q = (int32_t*)malloc(sizeof(int32_t) * (size_t)V);
  if (!q) return -2;
  for (int64_t i = 0; i < V; ++i) depth[i] = -1;
  if (parent)
    for (int64_t i = 0; i < V; ++i) parent[i] = -1;
  int64_t head = 0, tail = 0;
  depth[src] = 0;
  if (parent) parent[src] = src;
  q[tail++] = src;
  while (head < tail) {
    const int32_t u = q[head++];
    const int32_t du = depth[u];
    for (int64_t e = off[u]; e < off[u + 1]; ++e) {
      const int32_t v = adj[e];
      if (depth[v] == -1) {
        depth[v] = du + 1;
        if (parent) parent[v] = u;
        q[tail++] = v;
      }
    }
  }
  free(q);
  return 0;
}

/* Level-synchronous top-down BFS with OpenMP; vertices are claimed with a
 * compare-and-swap on their depth word. */
int oracle_bfs_omp(int64_t V, const int64_t* off, const int32_t* adj, int32_t src, int32_t* depth, int32_t* parent,
                   int threads) {
  if (V <= 0 || src < 0 || src >= V) return -1;
  if (threads <= 0) threads = omp_get_max_threads();
  int32_t* cur = (int32_t*)malloc(sizeof(int32_t) * (size_t)V);
  int32_t* nxt = (int32_t*)malloc(sizeof(int32_t) * (size_t)V);
  if (!cur || !nxt) { free(cur); free(nxt); return -2; }
#pragma omp parallel for num_threads(threads) schedule(static)
  for (int64_t i = 0; i < V; ++i) {
    depth[i] = -1;
    if (parent) parent[i] = -1;
  }
  depth[src] = 0;
  if (parent) parent[src] = src;
  cur[0] = src;
  int64_t ncur = 1;
  int32_t level = 0;
  while (ncur > 0) {
    int64_t nnext = 0;
#pragma omp parallel num_threads(threads)
    {
      int32_t buf[1024];
      int nb = 0;
#pragma omp for schedule(dynamic, 64)
      for (int64_t i = 0; i < ncur; ++i) {
        const int32_t u = cur[i];
        for (int64_t e = off[u]; e < off[u + 1]; ++e) {
          const int32_t v = adj[e];
          if (__atomic_load_n(&depth[v], __ATOMIC_RELAXED) != -1) continue;
          int32_t expect = -1;
          if (__atomic_compare_exchange_n(&depth[v], &expect, level + 1, 0, __ATOMIC_RELAXED, __ATOMIC_RELAXED)) {
            if (parent) parent[v] = u;
            buf[nb++] = v;
            if (nb == 1024) {
              int64_t at = __atomic_fetch_add(&nnext, nb, __ATOMIC_RELAXED);
              memcpy(nxt + at, buf, sizeof(int32_t) * nb);
              nb = 0;
            }
          }
        }
      }
      if (nb) {
        int64_t at = __atomic_fetch_add(&nnext, nb, __ATOMIC_RELAXED);
        memcpy(nxt + at, buf, sizeof(int32_t) * nb);
      }
    }
    int32_t* t = cur;
    cur = nxt;
    nxt = t;
    ncur = nnext;
    ++level;
  }
  free(cur);
  free(nxt);
  return 0;
}

/* Direction-optimising BFS (Beamer, Asanovic, Patterson, SC'12) on the CPU:
 * top-down while the frontier's edges are few, bottom-up over a frontier
 * bitmap when m_f > m_u/14, back when n_f < V/24. */
int oracle_bfs_omp_do(int64_t V, const int64_t* off, const int32_t* adj, int32_t src, int32_t* depth, int threads) {
  if (V <= 0 || src < 0 || src >= V) return -1;
  if (threads <= 0) threads = omp_get_max_threads();
  const int64_t W = (V + 63) / 64;
  int32_t* cur = (int32_t*)malloc(sizeof(int32_t) * (size_t)V);
  int32_t* nxt = (int32_t*)malloc(sizeof(int32_t) * (size_t)V);
  uint64_t* fb = (uint64_t*)calloc((size_t)W, sizeof(uint64_t));
  uint64_t* nb_ = (uint64_t*)calloc((size_t)W, sizeof(uint64_t));
  if (!cur || !nxt || !fb || !nb_) { free(cur); free(nxt); free(fb); free(nb_); return -2; }
#pragma omp parallel for num_threads(threads) schedule(static)
  for (int64_t i = 0; i < V; ++i) depth[i] = -1;
  const int64_t E = off[V];
  depth[src] = 0;
  cur[0] = src;
  int64_t ncur = 1, m_vis = off[src + 1] - off[src], m_f = m_vis;
  int32_t level = 0;
  int bottom_up = 0;
  while (ncur > 0) {
    int64_t nnext = 0, mnext = 0;
    if (!bottom_up && (double)m_f > (double)(E - m_vis) / 14.0) {
      bottom_up = 1;
      memset(fb, 0, sizeof(uint64_t) * (size_t)W);
      for (int64_t i = 0; i < ncur; ++i) fb[cur[i] >> 6] |= 1ull << (cur[i] & 63);
    } else if (bottom_up && (double)ncur < (double)V / 24.0) {
      /* convert the bitmap frontier back to a queue */
      bottom_up = 0;
      int64_t n = 0;
      for (int64_t v = 0; v < V; ++v)
        if ((fb[v >> 6] >> (v & 63)) & 1) cur[n++] = (int32_t)v;
      ncur = n;
    }
    if (bottom_up) {
      memset(nb_, 0, sizeof(uint64_t) * (size_t)W);
#pragma omp parallel for num_threads(threads) schedule(dynamic, 1024) reduction(+ : nnext, mnext)
      for (int64_t v = 0; v < V; ++v) {
        if (depth[v] != -1) continue;
        for (int64_t e = off[v]; e < off[v + 1]; ++e) {
          const int32_t u = adj[e];
          if ((fb[u >> 6] >> (u & 63)) & 1) {
            depth[v] = level + 1;
            __atomic_fetch_or(&nb_[v >> 6], 1ull << (v & 63), __ATOMIC_RELAXED);
            nnext++;
            mnext += off[v + 1] - off[v];
            break;
          }
        }
      }
      uint64_t* t = fb;
      fb = nb_;
      nb_ = t;
      ncur = nnext;
    } else {
#pragma omp parallel num_threads(threads) reduction(+ : mnext)
      {
        int32_t buf[1024];
        int nb = 0;
#pragma omp for schedule(dynamic, 64)
        for (int64_t i = 0; i < ncur; ++i) {
          const int32_t u = cur[i];
          for (int64_t e = off[u]; e < off[u + 1]; ++e) {
            const int32_t v = adj[e];
            if (__atomic_load_n(&depth[v], __ATOMIC_RELAXED) != -1) continue;
            int32_t expect = -1;
            if (__atomic_compare_exchange_n(&depth[v], &expect, level + 1, 0, __ATOMIC_RELAXED, __ATOMIC_RELAXED)) {
              mnext += off[v + 1] - off[v];
              buf[nb++] = v;
              if (nb == 1024) {
                int64_t at = __atomic_fetch_add(&nnext, nb, __ATOMIC_RELAXED);
                memcpy(nxt + at, buf, sizeof(int32_t) * nb);
                nb = 0;
              }
            }
          }
        }
        if (nb) {
          int64_t at = __atomic_fetch_add(&nnext, nb, __ATOMIC_RELAXED);
          memcpy(nxt + at, buf, sizeof(int32_t) * nb);
        }
      }
      int32_t* t = cur;
      cur = nxt;
      nxt = t;
      ncur = nnext;
    }
    m_vis += mnext;
    m_f = mnext;
    ++level;
  }
  free(cur);
  free(nxt);
  free(fb);
  free(nb_);
  return 0;
}

void oracle_report(int64_t V, const int64_t* off, const int32_t* depth, int64_t* tr_edges, int64_t* tr_verts) {
  int64_t e = 0, n = 0;
  for (int64_t i = 0; i < V; ++i)
    if (depth[i] != -1) {
      ++n;
      e += off[i + 1] - off[i];
    }
  *tr_edges = e;
  *tr_verts = n;
}

int oracle_check_depths(int64_t V, const int64_t* off, const int32_t* adj, int32_t src, const int32_t* depth,
                        int64_t* bad_vertex) {
  *bad_vertex = -1;
  if (depth[src] != 0) { *bad_vertex = src; return -1; }
  for (int64_t v = 0; v < V; ++v) {
    const int32_t dv = depth[v];
    if (dv < -1) { *bad_vertex = v; return -2; }
    if (dv == 0 && v != src) { *bad_vertex = v; return -3; }
    int has_parent = 0;
    for (int64_t e = off[v]; e < off[v + 1]; ++e) {
      const int32_t du = depth[adj[e]];
      if ((du == -1) != (dv == -1)) { *bad_vertex = v; return -4; }
      if (dv != -1 && (du > dv + 1 || du < dv - 1)) { *bad_vertex = v; return -5; }
      if (dv > 0 && du == dv - 1) has_parent = 1;
    }
    if (dv > 0 && !has_parent) { *bad_vertex = v; return -6; }
  }
  return 0;
}

static int has_edge(const int64_t* off, const int32_t* adj, int32_t p, int32_t v) {
  for (int64_t e = off[p]; e < off[p + 1]; ++e)
    if (adj[e] == v) return 1;
  return 0;
}

int oracle_check_parents(int64_t V, const int64_t* off, const int32_t* adj, int32_t src, const int32_t* depth,
                         const int32_t* parent, int64_t* bad_vertex) {
  *bad_vertex = -1;
  if (parent[src] != src || depth[src] != 0) { *bad_vertex = src; return -1; }
  for (int64_t v = 0; v < V; ++v) {
    if (v == src) continue;
    const int32_t p = parent[v];
    if (depth[v] == -1) {
      if (p != -1) { *bad_vertex = v; return -2; }
      continue;
    }
    if (p < 0 || p >= V) { *bad_vertex = v; return -3; }
    if (depth[p] != depth[v] - 1) { *bad_vertex = v; return -4; }
    if (!has_edge(off, adj, p, (int32_t)v)) { *bad_vertex = v; return -5; }
  }
  return 0;
}
