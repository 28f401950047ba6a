// Runs the reference's own GPU BFS and writes its depth arrays — TEST
// INFRASTRUCTURE ONLY (golden-vector generation; see tests/golden/).
//
// Built by oracle/Makefile from the reference's sources where they lie
// (-I <reference dir>, with ref_cuda_compat.h force-included). This harness
// does what the reference's entry point bfs_gpu_coalescing_mem does for each
// source (bfs_gpu_opt.cuh:293-410: allocate through allocator<>::alloc_array,
// reset the uint8 depth array to INFTY, run bfs_tdbu_clfy_sort), but instead
// of printing TEPS it copies the depth array back and writes it out.
//
//   ref_bfs_dump <beg_pos.bin> <csr.bin> <sources.txt> <out.bin>
//
// out.bin: for each source, V bytes (the reference's depth_t; 0xFF = unreached).
#include "bfs_gpu_opt.cuh"

#include <cstdio>
#include <vector>

int main(int argc, char** argv) {
  if (argc != 5) {
    fprintf(stderr, "usage: %s beg_pos.bin csr.bin sources.txt out.bin\n", argv[0]);
    return 2;
  }
  typedef int vertex_t;
  typedef int index_t;
  graph<long, long, double, vertex_t, index_t, double>* g =
      new graph<long, long, double, vertex_t, index_t, double>(argv[1], argv[2], NULL);
  std::vector<int> src;
  FILE* f = fopen(argv[3], "r");
  if (!f) return 3;
  int s;
  while (fscanf(f, "%d", &s) == 1) src.push_back(s);
  fclose(f);
  const index_t V = g->vert_count, E = g->edge_count;
  for (int x : src)
    if (x < 0 || x >= V) return 4;

  depth_t* depth_d;
  index_t *adj_card_d, *strt_pos_d;
  vertex_t* adj_list_d;
  vertex_t *ex_q_sml_d, *ex_q_mid_d, *ex_q_lrg_d;
  index_t *ex_cat_sml_sz, *ex_cat_mid_sz, *ex_cat_lrg_sz;
  index_t *ex_cat_sml_off, *ex_cat_mid_off, *ex_cat_lrg_off;
  vertex_t *ex_cat_sml_d, *ex_cat_mid_d, *ex_cat_lrg_d;
  index_t *tr_edges_c_d, *tr_edges_c_h;
  cudaStream_t* stream;
  const index_t bin_sz = BIN_SZ;
  cudaSetDevice(0);
  allocator<vertex_t, index_t, depth_t>::alloc_array(
      depth_d, adj_list_d, adj_card_d, strt_pos_d, ex_q_sml_d, ex_q_mid_d, ex_q_lrg_d, ex_cat_sml_sz, ex_cat_mid_sz,
      ex_cat_lrg_sz, ex_cat_sml_off, ex_cat_mid_off, ex_cat_lrg_off, ex_cat_sml_d, ex_cat_mid_d, ex_cat_lrg_d,
      tr_edges_c_d, tr_edges_c_h, g->beg_pos, g->csr, V, E, stream, bin_sz);
  std::vector<depth_t> inf(V, INFTY), out(V);
  FILE* o = fopen(argv[4], "wb");
  if (!o) return 5;
  for (int x : src) {
    ENABLE_CGU = false;
    ENABLE_BTUP = false;
    agg_tr_edges = 0;
    cudaMemcpy(depth_d, inf.data(), V, cudaMemcpyHostToDevice);
    depth_t level = 0;
    bfs_tdbu_clfy_sort<vertex_t, index_t, depth_t>(x, depth_d, adj_list_d, ex_q_sml_d, ex_q_mid_d, ex_q_lrg_d,
                                                   ex_cat_sml_sz, ex_cat_mid_sz, ex_cat_lrg_sz, ex_cat_sml_off,
                                                   ex_cat_mid_off, ex_cat_lrg_off, ex_cat_sml_d, ex_cat_mid_d,
                                                   ex_cat_lrg_d, V, tr_edges_c_d, tr_edges_c_h, stream, level, 32,
                                                   1024, bin_sz);
    cudaError_t e = cudaDeviceSynchronize();
    if (e != cudaSuccess) {
      fprintf(stderr, "reference BFS failed: %s\n", cudaGetErrorString(e));
      return 6;
    }
    cudaMemcpy(out.data(), depth_d, V, cudaMemcpyDeviceToHost);
    fwrite(out.data(), 1, V, o);
  }
  fclose(o);
  return 0;
}
