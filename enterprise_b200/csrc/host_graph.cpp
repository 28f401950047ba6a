// Host side of the graph boundary: error reporting, the reference-format CSR
// loader/writer, the canonical CSR builder and the seeded host generators.
//
// Loader contract follows graph<...>::graph (graph.hpp:33-118): V is derived
// from the beg_pos file size (fsize/8 - 1, graph.hpp:46), beg_pos is int64,
// the csr file is int64 in the reference's format (main.cu:50-52) and is
// narrowed to int32 in memory (graph.hpp:80-88). Unlike the reference, which
// asserts on short reads and never checks ids, every malformed input becomes
// a status code.
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/stat.h>
#include <algorithm>
#include <string>
#include <omp.h>

#include "ent_internal.h"
#include "gen_common.h"

namespace ent {

static thread_local std::string t_last_error;
std::atomic<int64_t> g_kernel_launches{0};

int fail(int code, const char* fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  t_last_error = buf;
  return code;
}

void clear_error() { t_last_error.clear(); }

// ------------------------------------------------------------------------
// Canonical CSR from undirected draws. `draw(i, &u, &v)` returns false for a
// dropped draw. Both directions are inserted; self loops and duplicates are
// removed; rows end up sorted ascending. The result does not depend on the
// thread schedule.
template <class Draw>
static int build_canonical(int64_t V, int64_t n_draws, Draw draw, ent_csr* g) {
  std::vector<int64_t> cnt(V + 1, 0);
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n_draws; ++i) {
    uint64_t u, v;
    if (!draw(i, &u, &v) || u == v) continue;
#pragma omp atomic
    cnt[u]++;
#pragma omp atomic
    cnt[v]++;
  }
  std::vector<int64_t> off(V + 1, 0);
  for (int64_t i = 0; i < V; ++i) off[i + 1] = off[i] + cnt[i];
  std::vector<int32_t> tmp(off[V]);
  std::vector<int64_t> cur(off.begin(), off.end() - 1);
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n_draws; ++i) {
    uint64_t u, v;
    if (!draw(i, &u, &v) || u == v) continue;
    int64_t pu, pv;
#pragma omp atomic capture
    pu = cur[u]++;
#pragma omp atomic capture
    pv = cur[v]++;
    tmp[pu] = (int32_t)v;
    tmp[pv] = (int32_t)u;
  }
  // sort + unique each row
#pragma omp parallel for schedule(dynamic, 1024)
  for (int64_t r = 0; r < V; ++r) {
    int32_t* b = tmp.data() + off[r];
    int32_t* e = tmp.data() + off[r + 1];
    std::sort(b, e);
    cnt[r] = std::unique(b, e) - b;
  }
  g->V = V;
  g->off.assign(V + 1, 0);
  for (int64_t i = 0; i < V; ++i) g->off[i + 1] = g->off[i] + cnt[i];
  g->E = g->off[V];
  g->adj.resize(g->E);
#pragma omp parallel for schedule(dynamic, 1024)
  for (int64_t r = 0; r < V; ++r)
    memcpy(g->adj.data() + g->off[r], tmp.data() + off[r], sizeof(int32_t) * cnt[r]);
  return ENT_OK;
}

RmatParams make_rmat_params(int scale, int ef, double a, double b, double c, uint64_t seed) {
  RmatParams rp;
  rp.scale = scale;
  rp.n_edges = (uint64_t)ef << scale;
  auto fx = [](double p) -> uint32_t {
    double x = p * 4294967296.0;
    if (x <= 0) return 0;
    if (x >= 4294967295.0) return 4294967295u;
    return (uint32_t)x;
  };
  rp.t_a = fx(a);
  rp.t_ab = fx(a + b);
  rp.t_abc = fx(a + b + c);
  rp.key = mix64(seed ^ 0x524D4154ull);
  rp.perm = make_perm(seed, scale);
  return rp;
}

GridParams make_grid_params(int64_t w, int64_t h, double drop, uint64_t seed) {
  GridParams gp;
  gp.w = w;
  gp.h = h;
  gp.n = (uint64_t)w * h;
  gp.n_edges = (uint64_t)h * (w - 1) + (uint64_t)(h - 1) * w;
  double x = drop * 4294967296.0;
  gp.t_drop = x <= 0 ? 0u : (x >= 4294967295.0 ? 4294967295u : (uint32_t)x);
  gp.key = mix64(seed ^ 0x47524944ull);
  gp.perm = make_perm(seed, ceil_log2(gp.n));
  return gp;
}

ErParams make_er_params(int64_t n, double mean_degree, uint64_t seed) {
  ErParams ep;
  ep.n = n;
  ep.n_edges = (uint64_t)(mean_degree * (double)n / 2.0 + 0.5);
  ep.key = mix64(seed ^ 0x45524452ull);
  ep.perm = make_perm(seed, ceil_log2(n));
  return ep;
}

}  // namespace ent

using namespace ent;

extern "C" {

const char* ent_last_error(void) { return t_last_error.c_str(); }
int ent_abi_version(void) { return ENT_ABI_VERSION; }
int64_t ent_kernel_launch_count(void) { return g_kernel_launches.load(); }

static int64_t file_size(const char* p) {
  struct stat st;
  if (stat(p, &st) != 0) return -1;
  return (int64_t)st.st_size;
}

int ent_csr_load(const char* beg_path, const char* csr_path, ent_csr** out) {
  clear_error();
  if (!beg_path || !csr_path || !out) return fail(ENT_ERR_INVALID_ARG, "null argument");
  *out = nullptr;
  int64_t bsz = file_size(beg_path);
  if (bsz < 0) return fail(ENT_ERR_IO, "beg file cannot open: %s", beg_path);
  if (bsz < 16 || bsz % 8 != 0)
    return fail(ENT_ERR_FORMAT, "beg_pos file size %lld is not 8*(V+1) with V>=1", (long long)bsz);
  int64_t csz = file_size(csr_path);
  if (csz < 0) return fail(ENT_ERR_IO, "CSR file cannot open: %s", csr_path);
  int64_t V = bsz / 8 - 1;
  if (V >= (1ll << 31) - 1) return fail(ENT_ERR_UNSUPPORTED, "V=%lld exceeds int32 ids", (long long)V);
  ent_csr* g = new ent_csr();
  g->V = V;
  g->off.resize(V + 1);
  FILE* f = fopen(beg_path, "rb");
  if (!f) { delete g; return fail(ENT_ERR_IO, "beg file cannot open: %s", beg_path); }
  size_t got = fread(g->off.data(), 8, V + 1, f);
  fclose(f);
  if ((int64_t)got != V + 1) { delete g; return fail(ENT_ERR_IO, "short read on %s", beg_path); }
  if (g->off[0] != 0) {
    const long long first = (long long)g->off[0];
    delete g;
    return fail(ENT_ERR_FORMAT, "beg_pos[0]=%lld, expected 0", first);
  }
  for (int64_t i = 0; i < V; ++i)
    if (g->off[i + 1] < g->off[i]) {
      int64_t a = g->off[i], b = g->off[i + 1];
      delete g;
      return fail(ENT_ERR_FORMAT, "beg_pos not monotone at %lld (%lld > %lld)", (long long)i, (long long)a, (long long)b);
    }
  int64_t E = g->off[V];
  int width;
  if (csz == E * 8) width = 8;
  else if (csz == E * 4) width = 4;
  else {
    delete g;
    return fail(ENT_ERR_FORMAT, "csr file size %lld matches neither int64 nor int32 for beg_pos[V]=%lld",
                (long long)csz, (long long)E);
  }
  g->E = E;
  g->adj.resize(E);
  f = fopen(csr_path, "rb");
  if (!f) { delete g; return fail(ENT_ERR_IO, "CSR file cannot open: %s", csr_path); }
  int64_t bad = -1;
  if (width == 4) {
    got = fread(g->adj.data(), 4, E, f);
    if ((int64_t)got != E) { fclose(f); delete g; return fail(ENT_ERR_IO, "short read on %s", csr_path); }
  } else {
    const int64_t CH = 1 << 22;
    std::vector<int64_t> buf(std::min<int64_t>(CH, std::max<int64_t>(E, 1)));
    for (int64_t pos = 0; pos < E; pos += CH) {
      int64_t n = std::min<int64_t>(CH, E - pos);
      got = fread(buf.data(), 8, n, f);
      if ((int64_t)got != n) { fclose(f); delete g; return fail(ENT_ERR_IO, "short read on %s", csr_path); }
      for (int64_t k = 0; k < n; ++k) {
        int64_t x = buf[k];
        if ((x < 0 || x >= V) && bad < 0) bad = pos + k;
        g->adj[pos + k] = (int32_t)x;
      }
    }
  }
  fclose(f);
  if (bad < 0) {
    for (int64_t k = 0; k < E; ++k)
      if (g->adj[k] < 0 || g->adj[k] >= V) { bad = k; break; }
  }
  if (bad >= 0) { delete g; return fail(ENT_ERR_FORMAT, "csr entry %lld out of range [0,V)", (long long)bad); }
  *out = g;
  return ENT_OK;
}

int ent_csr_save(const ent_csr* g, const char* beg_path, const char* csr_path) {
  clear_error();
  if (!g || !beg_path || !csr_path) return fail(ENT_ERR_INVALID_ARG, "null argument");
  FILE* f = fopen(beg_path, "wb");
  if (!f) return fail(ENT_ERR_IO, "cannot write %s", beg_path);
  size_t w = fwrite(g->off.data(), 8, g->V + 1, f);
  fclose(f);
  if ((int64_t)w != g->V + 1) return fail(ENT_ERR_IO, "short write %s", beg_path);
  f = fopen(csr_path, "wb");
  if (!f) return fail(ENT_ERR_IO, "cannot write %s", csr_path);
  const int64_t CH = 1 << 22;
  std::vector<int64_t> buf(std::min<int64_t>(CH, std::max<int64_t>(g->E, 1)));
  for (int64_t pos = 0; pos < g->E; pos += CH) {
    int64_t n = std::min<int64_t>(CH, g->E - pos);
    for (int64_t k = 0; k < n; ++k) buf[k] = g->adj[pos + k];
    if ((int64_t)fwrite(buf.data(), 8, n, f) != n) { fclose(f); return fail(ENT_ERR_IO, "short write %s", csr_path); }
  }
  fclose(f);
  return ENT_OK;
}

int ent_csr_from_arrays(const int64_t* beg, const int32_t* csr, int64_t V, int64_t E, ent_csr** out) {
  clear_error();
  if (!beg || (!csr && E > 0) || !out || V < 1 || E < 0) return fail(ENT_ERR_INVALID_ARG, "bad arguments");
  if (V >= (1ll << 31) - 1) return fail(ENT_ERR_UNSUPPORTED, "V exceeds int32 ids");
  if (beg[0] != 0 || beg[V] != E) return fail(ENT_ERR_FORMAT, "beg_pos[0] must be 0 and beg_pos[V] == E");
  for (int64_t i = 0; i < V; ++i)
    if (beg[i + 1] < beg[i]) return fail(ENT_ERR_FORMAT, "beg_pos not monotone at %lld", (long long)i);
  for (int64_t k = 0; k < E; ++k)
    if (csr[k] < 0 || csr[k] >= V) return fail(ENT_ERR_FORMAT, "csr entry %lld out of range", (long long)k);
  ent_csr* g = new ent_csr();
  g->V = V;
  g->E = E;
  g->off.assign(beg, beg + V + 1);
  g->adj.assign(csr, csr + E);
  *out = g;
  return ENT_OK;
}

int ent_csr_from_edges(const int64_t* src, const int64_t* dst, int64_t n, int64_t V, ent_csr** out) {
  clear_error();
  if ((!src || !dst) && n > 0) return fail(ENT_ERR_INVALID_ARG, "null edge arrays");
  if (!out || V < 1 || n < 0) return fail(ENT_ERR_INVALID_ARG, "bad arguments");
  if (V >= (1ll << 31) - 1) return fail(ENT_ERR_UNSUPPORTED, "V exceeds int32 ids");
  for (int64_t i = 0; i < n; ++i)
    if (src[i] < 0 || src[i] >= V || dst[i] < 0 || dst[i] >= V)
      return fail(ENT_ERR_FORMAT, "edge %lld has an endpoint outside [0,V)", (long long)i);
  ent_csr* g = new ent_csr();
  build_canonical(V, n, [&](int64_t i, uint64_t* u, uint64_t* v) {
    *u = (uint64_t)src[i];
    *v = (uint64_t)dst[i];
    return true;
  }, g);
  *out = g;
  return ENT_OK;
}

int64_t ent_csr_vert_count(const ent_csr* g) { return g ? g->V : -1; }
int64_t ent_csr_edge_count(const ent_csr* g) { return g ? g->E : -1; }
const int64_t* ent_csr_beg_pos(const ent_csr* g) { return g ? g->off.data() : nullptr; }
const int32_t* ent_csr_adj(const ent_csr* g) { return g ? g->adj.data() : nullptr; }
void ent_csr_free(ent_csr* g) { delete g; }

int ent_gen_rmat(int32_t scale, int32_t ef, double a, double b, double c, uint64_t seed, ent_csr** out) {
  clear_error();
  if (!out || scale < 1 || scale > 30 || ef < 1 || a < 0 || b < 0 || c < 0 || a + b + c > 1.0)
    return fail(ENT_ERR_INVALID_ARG, "bad R-MAT parameters");
  RmatParams rp = make_rmat_params(scale, ef, a, b, c, seed);
  int64_t V = 1ll << scale;
  ent_csr* g = new ent_csr();
  build_canonical(V, (int64_t)rp.n_edges, [&](int64_t i, uint64_t* u, uint64_t* v) {
    uint64_t x, y;
    rmat_edge(rp, (uint64_t)i, &x, &y);
    *u = perm_pow2(rp.perm, x);
    *v = perm_pow2(rp.perm, y);
    return true;
  }, g);
  *out = g;
  return ENT_OK;
}

int ent_gen_grid(int64_t w, int64_t h, double drop, uint64_t seed, ent_csr** out) {
  clear_error();
  if (!out || w < 2 || h < 2 || drop < 0 || drop > 1 || w * h >= (1ll << 31) - 1)
    return fail(ENT_ERR_INVALID_ARG, "bad grid parameters");
  GridParams gp = make_grid_params(w, h, drop, seed);
  ent_csr* g = new ent_csr();
  build_canonical((int64_t)gp.n, (int64_t)gp.n_edges, [&](int64_t e, uint64_t* u, uint64_t* v) {
    uint64_t x, y;
    bool keep = grid_edge(gp, (uint64_t)e, &x, &y);
    *u = perm_apply(gp.perm, gp.n, x);
    *v = perm_apply(gp.perm, gp.n, y);
    return keep;
  }, g);
  *out = g;
  return ENT_OK;
}

int ent_gen_er(int64_t n, double mean_degree, uint64_t seed, ent_csr** out) {
  clear_error();
  if (!out || n < 2 || n >= (1ll << 31) - 1 || mean_degree < 0) return fail(ENT_ERR_INVALID_ARG, "bad ER parameters");
  ErParams ep = make_er_params(n, mean_degree, seed);
  ent_csr* g = new ent_csr();
  build_canonical(n, (int64_t)ep.n_edges, [&](int64_t i, uint64_t* u, uint64_t* v) {
    uint64_t x, y;
    er_edge(ep, (uint64_t)i, &x, &y);
    *u = perm_apply(ep.perm, ep.n, x);
    *v = perm_apply(ep.perm, ep.n, y);
    return true;
  }, g);
  *out = g;
  return ENT_OK;
}

int ent_pick_sources(const int64_t* beg, int64_t V, uint64_t seed, int32_t count, int32_t* out) {
  clear_error();
  if (!beg || !out || V < 1 || count < 0) return fail(ENT_ERR_INVALID_ARG, "bad arguments");
  int64_t nonisolated = 0;
  for (int64_t v = 0; v < V; ++v) nonisolated += (beg[v + 1] > beg[v]);
  if (count > nonisolated)
    return fail(ENT_ERR_INVALID_ARG, "asked for %d sources, graph has %lld non-isolated vertices", count, (long long)nonisolated);
  std::vector<uint8_t> taken(V, 0);
  int32_t k = 0;
  uint64_t limit = (uint64_t)V * 64 + (1u << 20);
  for (uint64_t j = 0; k < count; ++j) {
    if (j > limit) return fail(ENT_ERR_INTERNAL, "source draw did not converge");
    int64_t s = (int64_t)source_draw(seed, j, (uint64_t)V);
    if (beg[s + 1] == beg[s] || taken[s]) continue;
    taken[s] = 1;
    out[k++] = (int32_t)s;
  }
  return ENT_OK;
}

int ent_pick_sources_compat(const int64_t* beg, int64_t V, int32_t count, int32_t* out) {
  clear_error();
  if (!beg || !out || V < 1 || count < 0) return fail(ENT_ERR_INVALID_ARG, "bad arguments");
  int64_t nonisolated = 0;
  for (int64_t v = 0; v < V; ++v) nonisolated += (beg[v + 1] > beg[v]);
  if (count > nonisolated)
    return fail(ENT_ERR_INVALID_ARG, "asked for %d sources, graph has %lld non-isolated vertices", count, (long long)nonisolated);
  // Same draw sequence as main.cu:55-78: rand()%vert_count with vert_count an
  // int, rejecting orphans and repeats.
  int vc = (int)V;
  for (int32_t i = 0; i < count; ++i) {
    for (;;) {
      int s = rand() % vc;
      if (beg[s + 1] - beg[s] == 0) continue;
      bool fresh = true;
      for (int32_t j = 0; j < i; ++j)
        if (out[j] == s) { fresh = false; break; }
      if (!fresh) continue;
      out[i] = s;
      break;
    }
  }
  return ENT_OK;
}

}  // extern "C"
