/*
 * CPU oracle for the BFS hot path — TEST INFRASTRUCTURE ONLY.
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline legs may
 * load this code, and only as the checker / the timed CPU baseline. The
 * product path (libenterprise_b200) never calls it.
 *
 * The reference has no CPU BFS: its validate() only spot-checks one random
 * reached vertex (validate.h:34-103) and report() counts reached vertices and
 * their degrees (validate.h:106-127). This file restates
 *  - the traversal the GPU level loop computes (bfs_gpu_opt.cuh:99-282):
 *    depth[src] = 0, a vertex first seen from a frontier vertex at depth L
 *    gets L+1 (top-down rule expander.cuh:162-163; bottom-up rule
 *    expander.cuh:519-523 gives the same depths), unreached = -1 (INFTY,
 *    comm.h:131, widened to int32);
 *  - report() (validate.h:106-127);
 *  - a complete BFS-depth certificate and the Graph500 parent checks.
 * Parity is pinned against the reference's own validate()/report(), compiled
 * from its sources by oracle/Makefile into oracle/_ref/, and against golden
 * depth fixtures under tests/golden/.
 */
#ifndef ENT_ORACLE_H
#define ENT_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Serial FIFO-queue BFS. parent may be NULL; parent = first discoverer. */
int oracle_bfs(int64_t V, const int64_t* off, const int32_t* adj, int32_t src, int32_t* depth, int32_t* parent);

/* Level-synchronous top-down BFS on `threads` OpenMP threads (<=0: all).
 * Same depths as oracle_bfs; parents are any valid BFS parent. */
int oracle_bfs_omp(int64_t V, const int64_t* off, const int32_t* adj, int32_t src, int32_t* depth,
                   int32_t* parent, int threads);

/* Direction-optimising (Beamer) CPU BFS on `threads` threads: the strongest
 * CPU baseline here. Same depths. */
int oracle_bfs_omp_do(int64_t V, const int64_t* off, const int32_t* adj, int32_t src, int32_t* depth,
                      int threads);

/* report(): reached vertices and the sum of their degrees. */
void oracle_report(int64_t V, const int64_t* off, const int32_t* depth, int64_t* tr_edges, int64_t* tr_verts);

/* Complete depth certificate: depth[src]==0; every edge joins two reached or
 * two unreached vertices and spans <= 1 level; every reached v != src has a
 * neighbour one level up. Returns 0 or a negative code; *bad_vertex set. */
int oracle_check_depths(int64_t V, const int64_t* off, const int32_t* adj, int32_t src, const int32_t* depth,
                        int64_t* bad_vertex);

/* Graph500-style parent validation: parent[src]==src; reached v != src has
 * depth[parent[v]] == depth[v]-1 and the edge (parent[v], v) exists;
 * unreached v has parent -1. Returns 0 or a negative code. */
int oracle_check_parents(int64_t V, const int64_t* off, const int32_t* adj, int32_t src, const int32_t* depth,
                         const int32_t* parent, int64_t* bad_vertex);

/* Maximum OpenMP threads on this host. */
int oracle_max_threads(void);

/* Seeded Graph500-parameter R-MAT graph as an undirected CSR (both directions,
 * self loops and duplicates dropped, rows ascending, ids scrambled by a seeded
 * bijection): the same CSR as the product's generator for the same arguments,
 * so the benchmark's CPU arm needs no product code (graph_oracle.c). *off_out
 * (V+1) and *adj_out (E) are malloc'ed; release with oracle_free. */
int oracle_gen_rmat(int32_t scale, int32_t edge_factor, double a, double b, double c, uint64_t seed,
                    int64_t** off_out, int32_t** adj_out, int64_t* vert_count, int64_t* edge_count);
/* The first `count` distinct non-isolated vertices of the seeded hash draw
 * (the product's seeded source rule). */
int oracle_pick_sources(const int64_t* off, int64_t V, uint64_t seed, int32_t count, int32_t* out);
void oracle_free(void* p);

#ifdef __cplusplus
}
#endif
#endif
