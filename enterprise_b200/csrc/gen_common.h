// Seeded synthetic graph generators shared by the host (g++) and device (nvcc)
// builders. Everything here is integer arithmetic so that the CPU and GPU
// builders produce bit-identical edge lists, and therefore identical CSR.
//
// The reference ships no generator (its inputs come from an edge-list text
// converter, tuple_text_to_binary_csr/tuple_text_to_bin.cpp:56-315); these
// generators stand in for the Graph500 / SNAP inputs it was run on:
//   * R-MAT with the Graph500 quadrant probabilities a/b/c/d (no noise),
//   * a W x H 4-neighbour grid with a seeded fraction of edges dropped,
//   * an Erdos-Renyi G(n, M) graph.
// Vertex ids are scrambled by a seeded bijection so that id locality carries
// no information about the generator.
#pragma once
#include <stdint.h>

#if defined(__CUDACC__)
#define ENT_HD __host__ __device__ __forceinline__
#else
#define ENT_HD inline
#endif

namespace ent {

// SplitMix64 finaliser (Steele, Lea, Flood 2014; Vigna's public-domain
// constants). Used as a counter-based hash: x -> 64 well-mixed bits.
ENT_HD uint64_t mix64(uint64_t x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}

// Upper 64 bits of a 64x64 product: maps a uniform 64-bit word onto [0, n).
ENT_HD uint64_t mulhi64(uint64_t a, uint64_t b) {
#if defined(__CUDA_ARCH__)
  return __umul64hi(a, b);
#else
  return (uint64_t)(((unsigned __int128)a * b) >> 64);
#endif
}

// A seeded bijection on [0, 2^bits). Each round is invertible modulo 2^bits:
// multiply by an odd constant, add a constant, xor-shift right.
struct Perm {
  uint64_t mask;
  uint64_t mul[3];
  uint64_t add[3];
  int sh[3];
  int bits;
};

ENT_HD Perm make_perm(uint64_t seed, int bits) {
  Perm p;
  p.bits = bits;
  p.mask = bits >= 64 ? ~0ull : ((1ull << bits) - 1);
  uint64_t s = mix64(seed ^ 0xA5A5F00DCAFEBEEFull);
  for (int r = 0; r < 3; ++r) {
    s = mix64(s);
    p.mul[r] = (s | 1ull) & p.mask;
    if (p.mul[r] == 0) p.mul[r] = 1;
    s = mix64(s);
    p.add[r] = s & p.mask;
    int k = bits / (r + 2);
    p.sh[r] = k < 1 ? 1 : k;
  }
  return p;
}

ENT_HD uint64_t perm_pow2(const Perm& p, uint64_t x) {
  for (int r = 0; r < 3; ++r) {
    x = (x * p.mul[r] + p.add[r]) & p.mask;
    x ^= x >> p.sh[r];
  }
  return x;
}

// Bijection on [0, n) by cycle walking over the enclosing power of two.
ENT_HD uint64_t perm_apply(const Perm& p, uint64_t n, uint64_t x) {
  do {
    x = perm_pow2(p, x);
  } while (x >= n);
  return x;
}

ENT_HD int ceil_log2(uint64_t n) {
  int b = 0;
  while ((1ull << b) < n) ++b;
  return b;
}

// ---------------------------------------------------------------- R-MAT ---
// Quadrant thresholds are 32-bit fixed point, computed once on the host from
// the probabilities so both builders compare the same integers.
struct RmatParams {
  int scale;
  uint64_t n_edges;  // undirected edge draws = edge_factor << scale
  uint32_t t_a, t_ab, t_abc;
  uint64_t key;      // per-graph stream key
  Perm perm;
};

// One R-MAT draw: `scale` recursive quadrant choices, one 32-bit uniform
// per level. Returns the (unpermuted) endpoints.
ENT_HD void rmat_edge(const RmatParams& rp, uint64_t i, uint64_t* u_out, uint64_t* v_out) {
  uint64_t st = mix64(rp.key + i);
  uint64_t u = 0, v = 0;
  for (int k = 0; k < rp.scale; ++k) {
    st = mix64(st + (uint64_t)k);
    uint32_t r = (uint32_t)(st >> 32);
    uint64_t bu, bv;
    if (r < rp.t_a) { bu = 0; bv = 0; }
    else if (r < rp.t_ab) { bu = 0; bv = 1; }
    else if (r < rp.t_abc) { bu = 1; bv = 0; }
    else { bu = 1; bv = 1; }
    u = (u << 1) | bu;
    v = (v << 1) | bv;
  }
  *u_out = u;
  *v_out = v;
}

// ---------------------------------------------------------------- grid ----
// Edge e of a W x H 4-neighbour grid: horizontal edges first (row-major,
// W-1 per row), then vertical edges (row-major, W per row, H-1 rows).
struct GridParams {
  uint64_t w, h;
  uint64_t n_edges;     // h*(w-1) + (h-1)*w
  uint32_t t_drop;      // drop edge when hash32 < t_drop
  uint64_t key;
  Perm perm;
  uint64_t n;           // w*h
};

ENT_HD bool grid_edge(const GridParams& gp, uint64_t e, uint64_t* u_out, uint64_t* v_out) {
  uint32_t r = (uint32_t)(mix64(gp.key + e) >> 32);
  uint64_t nh = gp.h * (gp.w - 1);
  uint64_t u, v;
  if (e < nh) {
    uint64_t row = e / (gp.w - 1), col = e % (gp.w - 1);
    u = row * gp.w + col;
    v = u + 1;
  } else {
    uint64_t f = e - nh;
    uint64_t row = f / gp.w, col = f % gp.w;
    u = row * gp.w + col;
    v = u + gp.w;
  }
  *u_out = u;
  *v_out = v;
  return r >= gp.t_drop;
}

// ---------------------------------------------------------------- ER ------
struct ErParams {
  uint64_t n;
  uint64_t n_edges;  // undirected draws
  uint64_t key;
  Perm perm;
};

ENT_HD void er_edge(const ErParams& ep, uint64_t i, uint64_t* u_out, uint64_t* v_out) {
  uint64_t a = mix64(ep.key + 2 * i);
  uint64_t b = mix64(ep.key + 2 * i + 1);
  *u_out = mulhi64(a, ep.n);
  *v_out = mulhi64(b, ep.n);
}

// Deterministic seeded sources: draw j is mix64(seed + j) mod n; keep the
// first `count` distinct vertices with degree > 0 (the reference's source
// rule, main.cu:55-78, with a seeded hash in place of rand()).
ENT_HD uint64_t source_draw(uint64_t seed, uint64_t j, uint64_t n) {
  return mulhi64(mix64(seed * 0x100000001B3ull + j), n);
}

}  // namespace ent
