/*
 * Seeded R-MAT graph and seeded sources for the CPU side of the benchmark —
 * TEST INFRASTRUCTURE ONLY (see oracle.h).
 *
 * The reference ships no generator (its inputs come from its edge-list text
 * converter, tuple_text_to_binary_csr/tuple_text_to_bin.cpp:56-315). The
 * benchmark's CPU arm must traverse the same graph and the same sources as the
 * GPU arm without loading the product library, so this file restates, in C,
 * the published recipe the product's generator implements:
 *  - R-MAT (Chakrabarti, Zhan, Faloutsos, SDM'04) with the Graph500 quadrant
 *    probabilities: per draw, `scale` quadrant choices, each taking the upper
 *    32 bits of a SplitMix64 step (Steele, Lea, Flood, OOPSLA'14) compared
 *    with 32-bit fixed-point thresholds a, a+b, a+b+c;
 *  - vertex ids scrambled by a seeded bijection of [0, 2^scale): three rounds
 *    of (x*odd + c) mod 2^scale followed by x ^= x >> k;
 *  - the undirected CSR: both directions, self loops and duplicates dropped,
 *    rows ascending (a CSR that the edge multiset alone determines);
 *  - sources: draw j is mulhi64(mix64(seed*0x100000001B3 + j), V); the first
 *    `count` distinct vertices of degree > 0 are kept (the reference's rule,
 *    main.cu:55-78, with a seeded hash in place of rand()).
 * tests/test_oracle.py checks both against the product's generator bit for bit.
 */
#include "oracle.h"

#include <omp.h>
#include <stdlib.h>
#include <string.h>

static uint64_t sm64(uint64_t x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}

static uint64_t hi64(uint64_t a, uint64_t b) { return (uint64_t)(((unsigned __int128)a * b) >> 64); }

typedef struct {
  uint64_t mask, mul[3], add[3];
  int sh[3];
} scramble_t;

static scramble_t scramble_make(uint64_t seed, int bits) {
  scramble_t p;
  p.mask = bits >= 64 ? ~0ull : ((1ull << bits) - 1);
  uint64_t s = sm64(seed ^ 0xA5A5F00DCAFEBEEFull);
  for (int r = 0; r < 3; ++r) {
    s = sm64(s);
    p.mul[r] = (s | 1ull) & p.mask;
    if (!p.mul[r]) p.mul[r] = 1;
    s = sm64(s);
    p.add[r] = s & p.mask;
    const int k = bits / (r + 2);
    p.sh[r] = k < 1 ? 1 : k;
  }
  return p;
}

static uint64_t scramble(const scramble_t* p, uint64_t x) {
  for (int r = 0; r < 3; ++r) {
    x = (x * p->mul[r] + p->add[r]) & p->mask;
    x ^= x >> p->sh[r];
  }
  return x;
}

static uint32_t fixed32(double prob) {
  const double x = prob * 4294967296.0;
  if (x <= 0) return 0;
  if (x >= 4294967295.0) return 4294967295u;
  return (uint32_t)x;
}

typedef struct {
  int scale;
  uint32_t ta, tab, tabc;
  uint64_t key;
  scramble_t perm;
} rmat_t;

static void rmat_draw(const rmat_t* r, uint64_t i, uint64_t* u, uint64_t* v) {
  uint64_t st = sm64(r->key + i), a = 0, b = 0;
  for (int k = 0; k < r->scale; ++k) {
    st = sm64(st + (uint64_t)k);
    const uint32_t x = (uint32_t)(st >> 32);
    const uint64_t right = x >= r->ta && (x < r->tab || x >= r->tabc);  /* quadrants b and d */
    const uint64_t down = x >= r->tab;                                 /* quadrants c and d */
    a = (a << 1) | down;
    b = (b << 1) | right;
  }
  *u = scramble(&r->perm, a);
  *v = scramble(&r->perm, b);
}

static int cmp_i32(const void* x, const void* y) {
  const int32_t a = *(const int32_t*)x, b = *(const int32_t*)y;
  return (a > b) - (a < b);
}

int oracle_gen_rmat(int32_t scale, int32_t edge_factor, double a, double b, double c, uint64_t seed,
                    int64_t** off_out, int32_t** adj_out, int64_t* vert_count, int64_t* edge_count) {
  if (scale < 1 || scale > 30 || edge_factor < 1 || !off_out || !adj_out || !vert_count || !edge_count) return -1;
  rmat_t r;
  r.scale = scale;
  r.ta = fixed32(a);
  r.tab = fixed32(a + b);
  r.tabc = fixed32(a + b + c);
  r.key = sm64(seed ^ 0x524D4154ull);
  r.perm = scramble_make(seed, scale);
  const int64_t V = (int64_t)1 << scale;
  const int64_t draws = (int64_t)edge_factor << scale;
  /* pass 1: row lengths with repeats; pass 2: scatter both directions;
     pass 3: sort and drop repeats per row; pass 4: compact */
  int64_t* len = (int64_t*)calloc((size_t)V + 1, sizeof(int64_t));
  if (!len) return -2;
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < draws; ++i) {
    uint64_t u, v;
    rmat_draw(&r, (uint64_t)i, &u, &v);
    if (u == v) continue;
#pragma omp atomic
    len[u]++;
#pragma omp atomic
    len[v]++;
  }
  int64_t* start = (int64_t*)malloc(sizeof(int64_t) * ((size_t)V + 1));
  int64_t* fill = (int64_t*)malloc(sizeof(int64_t) * (size_t)V);
  if (!start || !fill) { free(len); free(start); free(fill); return -2; }
  start[0] = 0;
  for (int64_t i = 0; i < V; ++i) start[i + 1] = start[i] + len[i];
  memcpy(fill, start, sizeof(int64_t) * (size_t)V);
  int32_t* raw = (int32_t*)malloc(sizeof(int32_t) * (size_t)(start[V] > 0 ? start[V] : 1));
  if (!raw) { free(len); free(start); free(fill); return -2; }
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < draws; ++i) {
    uint64_t u, v;
    rmat_draw(&r, (uint64_t)i, &u, &v);
    if (u == v) continue;
    int64_t pu, pv;
#pragma omp atomic capture
    pu = fill[u]++;
#pragma omp atomic capture
    pv = fill[v]++;
    raw[pu] = (int32_t)v;
    raw[pv] = (int32_t)u;
  }
  free(fill);
#pragma omp parallel for schedule(dynamic, 4096)
  for (int64_t x = 0; x < V; ++x) {
    int32_t* row = raw + start[x];
    const int64_t n = start[x + 1] - start[x];
    if (n > 1) qsort(row, (size_t)n, sizeof(int32_t), cmp_i32);
    int64_t k = 0;
    for (int64_t j = 0; j < n; ++j)
      if (k == 0 || row[j] != row[k - 1]) row[k++] = row[j];
    len[x] = k;
  }
  int64_t* off = (int64_t*)malloc(sizeof(int64_t) * ((size_t)V + 1));
  if (!off) { free(len); free(start); free(raw); return -2; }
  off[0] = 0;
  for (int64_t x = 0; x < V; ++x) off[x + 1] = off[x] + len[x];
  int32_t* adj = (int32_t*)malloc(sizeof(int32_t) * (size_t)(off[V] > 0 ? off[V] : 1));
  if (!adj) { free(len); free(start); free(raw); free(off); return -2; }
#pragma omp parallel for schedule(dynamic, 4096)
  for (int64_t x = 0; x < V; ++x) memcpy(adj + off[x], raw + start[x], sizeof(int32_t) * (size_t)len[x]);
  free(len);
  free(start);
  free(raw);
  *off_out = off;
  *adj_out = adj;
  *vert_count = V;
  *edge_count = off[V];
  return 0;
}

int oracle_pick_sources(const int64_t* off, int64_t V, uint64_t seed, int32_t count, int32_t* out) {
  if (!off || !out || V < 1 || count < 0) return -1;
  int64_t live = 0;
  for (int64_t x = 0; x < V; ++x) live += off[x + 1] > off[x];
  if (count > live) return -1;
  unsigned char* seen = (unsigned char*)calloc((size_t)V, 1);
  if (!seen) return -2;
  int32_t k = 0;
  const uint64_t limit = (uint64_t)V * 64 + (1u << 20);
  for (uint64_t j = 0; k < count; ++j) {
    if (j > limit) { free(seen); return -3; }
    const int64_t s = (int64_t)hi64(sm64(seed * 0x100000001B3ull + j), (uint64_t)V);
    if (off[s + 1] == off[s] || seen[s]) continue;
    seen[s] = 1;
    out[k++] = (int32_t)s;
  }
  free(seen);
  return 0;
}

void oracle_free(void* p) { free(p); }
