// enterprise.bin — drop-in command line for the reference's main.cu:37-88.
//
//   enterprise.bin <beg_pos.bin> <csr.bin> [options]
//
// With only the two positional arguments it behaves like the reference:
// prints the input-format banner, loads the CSR (int64 files, graph.hpp:33-118;
// int32 csr files are accepted too), picks 64 distinct non-isolated sources
// with glibc rand()%V exactly as main.cu:55-78 does (same sequence), and runs
// bfs_gpu_coalescing_mem, printing the reference's per-source lines.
// Options (only after the two paths):
//   --seed S        seeded sources (hash draw) instead of rand()
//   --sources N     number of sources (default 64)
//   --json PATH     append one JSON line per source to PATH
//   --policy P      beamer | reference | td | bu
//   --loop L        graph | host
//   --gpu G         device id (default 0, as main.cu:49)
//   --batch [N]     run the sources as bitwise multi-source batches of up to N
//                   (default 64) sources, one launch per batch; a batch's depth
//                   rows (N x V int32) are held in host memory for the checks
// The csr file may hold int64 (the reference's format) or int32 ids: the
// width follows from its size against beg_pos[V].
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <chrono>
#include <string>
#include <vector>

#include "bfs_gpu_opt.cuh"

int main(int argc, char** argv) {
  printf("Input format: ./exe beg_pos(binary, signed long) csr_file(binary, signed long)\n");
  if (argc < 3) {
    printf("Wrong input\n");
    return -1;
  }
  long long seed = -1;
  int n_sources = 64, gpu = 0, batch = 0;
  const char* json_path = nullptr;
  ent_bfs_opts opts;
  ent_bfs_opts_default(&opts);
  for (int i = 3; i < argc; ++i) {
    std::string a = argv[i];
    auto need = [&](const char* what) -> const char* {
      if (i + 1 >= argc) {
        printf("Wrong input: %s needs a value\n", what);
        exit(255);
      }
      return argv[++i];
    };
    if (a == "--seed") seed = atoll(need("--seed"));
    else if (a == "--sources") n_sources = atoi(need("--sources"));
    else if (a == "--json") json_path = need("--json");
    else if (a == "--gpu") gpu = atoi(need("--gpu"));
    else if (a == "--batch") {
      batch = 64;
      if (i + 1 < argc && argv[i + 1][0] != '-') batch = atoi(argv[++i]);
      if (batch < 1) {
        printf("Wrong input: --batch needs a positive size\n");
        return -1;
      }
    }
    else if (a == "--policy") {
      std::string p = need("--policy");
      if (p == "beamer") opts.policy = ENT_POLICY_BEAMER;
      else if (p == "reference") opts.policy = ENT_POLICY_REFERENCE;
      else if (p == "td") opts.policy = ENT_POLICY_TD_ONLY;
      else if (p == "bu") opts.policy = ENT_POLICY_BU_ONLY;
      else { printf("Wrong input: unknown policy %s\n", p.c_str()); return -1; }
    } else if (a == "--loop") {
      std::string p = need("--loop");
      opts.loop = p == "host" ? ENT_LOOP_HOST : ENT_LOOP_GRAPH;
    } else {
      printf("Wrong input: unknown option %s\n", a.c_str());
      return -1;
    }
  }
  if (n_sources < 1) {
    printf("Wrong input: --sources must be >= 1\n");
    return -1;
  }
  auto t0 = std::chrono::steady_clock::now();
  ent_csr* g = nullptr;
  if (ent_csr_load(argv[1], argv[2], &g) != ENT_OK) {
    printf("Graph load failed: %s\n", ent_last_error());
    return 1;
  }
  const int64_t V = ent_csr_vert_count(g), E = ent_csr_edge_count(g);
  const int64_t* beg = ent_csr_beg_pos(g);
  printf("Possible edge count: %lld\n", (long long)beg[V]);
  double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  printf("Graph load (success): %lld verts, %lld edges %g second(s)\n", (long long)V, (long long)E, secs);
  std::vector<int32_t> src(n_sources);
  int rc = seed >= 0 ? ent_pick_sources(beg, V, (uint64_t)seed, n_sources, src.data())
                     : ent_pick_sources_compat(beg, V, n_sources, src.data());
  if (rc != ENT_OK) {
    printf("Source selection failed: %s\n", ent_last_error());
    ent_csr_free(g);
    return 1;
  }
  FILE* jf = nullptr;
  if (json_path) {
    jf = fopen(json_path, "a");
    if (!jf) {
      printf("Cannot open %s\n", json_path);
      ent_csr_free(g);
      return 1;
    }
  }
  ent_compat::RunOptions ro;
  ro.n_sources = n_sources;
  ro.batch = batch;
  ro.opts = &opts;
  ro.json = jf;
  rc = ent_compat::run(src.data(), beg, ent_csr_adj(g), V, E, gpu, ro);
  if (jf) fclose(jf);
  ent_csr_free(g);
  return rc;
}
