// enterprise.bin — drop-in command line for the reference's main.cu:37-88.
//
//   enterprise.bin <beg_pos.bin> <csr.bin> [options]
//
// With only the two positional arguments it does what the reference does:
// prints the input-format banner, loads the CSR (int64 files, graph.hpp:33-118;
// int32 csr files are accepted too), picks 64 distinct non-isolated sources
// with glibc rand()%V exactly as main.cu:55-78 does (same sequence), runs one
// BFS per source and prints the reference's per-source lines. The files are
// streamed straight to the GPU (ent_graph_load: the CSR never sits in host
// memory; only beg_pos is read on the host, for the source draw), and every
// traversal is validated on the GPU against the whole graph (ent_validate).
// --host-load takes the reference's route to the GPU instead: the CSR loaded
// into host memory and uploaded from there.
// Options (only after the two paths):
//   --seed S        seeded sources (hash draw) instead of rand()
//   --sources N     number of sources (default 64)
//   --json PATH     append one JSON line per source to PATH
//   --policy P      beamer | reference | td | bu
//   --loop L        graph | host
//   --gpu G         device id (default 0, as main.cu:49)
//   --batch [N]     run the sources as bitwise multi-source batches of up to N
//                   (default 64) sources, one launch per batch; a batch's depth
//                   rows (N x V int32) are held in GPU memory
//   --host-load     load through host memory, then upload
// The csr file may hold int64 (the reference's format) or int32 ids: the
// width follows from its size against beg_pos[V].
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <chrono>
#include <string>
#include <vector>

#include "bfs_gpu_opt.cuh"

// beg_pos.bin (int64[V+1], V from the file size as graph.hpp:46-47 derives it).
static bool read_beg_pos(const char* path, std::vector<int64_t>& beg) {
  FILE* f = fopen(path, "rb");
  if (!f) return false;
  bool ok = fseeko(f, 0, SEEK_END) == 0;
  const off_t n = ok ? ftello(f) : -1;
  ok = ok && n >= 16 && n % 8 == 0 && fseeko(f, 0, SEEK_SET) == 0;
  if (ok) {
    beg.resize((size_t)n / 8);
    ok = fread(beg.data(), 8, beg.size(), f) == beg.size();
  }
  fclose(f);
  return ok;
}

int main(int argc, char** argv) {
  printf("Input format: ./exe beg_pos(binary, signed long) csr_file(binary, signed long)\n");
  if (argc < 3) {
    printf("Wrong input\n");
    return -1;
  }
  long long seed = -1;
  int n_sources = 64, gpu = 0, batch = 0;
  bool host_load = false;
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
    else if (a == "--host-load") host_load = true;
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
  ent_csr* hg = nullptr;    // --host-load: the whole CSR in host memory
  ent_graph* dg = nullptr;  // default: the CSR streamed to the GPU
  std::vector<int64_t> beg_host;
  const int64_t* beg = nullptr;
  int64_t V = 0, E = 0;
  if (host_load) {
    if (ent_csr_load(argv[1], argv[2], &hg) != ENT_OK) {
      printf("Graph load failed: %s\n", ent_last_error());
      return 1;
    }
    V = ent_csr_vert_count(hg);
    E = ent_csr_edge_count(hg);
    beg = ent_csr_beg_pos(hg);
  } else {
    if (ent_graph_load(argv[1], argv[2], gpu, &dg) != ENT_OK) {
      printf("Graph load failed: %s\n", ent_last_error());
      return 1;
    }
    V = ent_graph_vert_count(dg);
    E = ent_graph_edge_count(dg);
    if (!read_beg_pos(argv[1], beg_host) || (int64_t)beg_host.size() != V + 1) {
      printf("Graph load failed: cannot reread %s\n", argv[1]);
      ent_graph_destroy(dg);
      return 1;
    }
    beg = beg_host.data();
  }
  const auto release = [&]() {
    if (hg) ent_csr_free(hg);
    if (dg) ent_graph_destroy(dg);
  };
  printf("Possible edge count: %lld\n", (long long)beg[V]);
  printf("Weight file cannot open\n");  // graph.hpp:114: main.cu:52 passes no weight file
  double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  printf("Graph load (success): %lld verts, %lld edges %g second(s)\n", (long long)V, (long long)E, secs);
  std::vector<int32_t> src(n_sources);
  int rc = seed >= 0 ? ent_pick_sources(beg, V, (uint64_t)seed, n_sources, src.data())
                     : ent_pick_sources_compat(beg, V, n_sources, src.data());
  if (rc != ENT_OK) {
    printf("Source selection failed: %s\n", ent_last_error());
    release();
    return 1;
  }
  FILE* jf = nullptr;
  if (json_path) {
    jf = fopen(json_path, "a");
    if (!jf) {
      printf("Cannot open %s\n", json_path);
      release();
      return 1;
    }
  }
  ent_compat::RunOptions ro;
  ro.n_sources = n_sources;
  ro.batch = batch;
  ro.opts = &opts;
  ro.json = jf;
  ro.cpu_bytes = host_load ? (int64_t)(sizeof(int64_t) * (V + 1) + sizeof(int32_t) * E)
                           : (int64_t)(sizeof(int64_t) * beg_host.size());
  rc = host_load ? ent_compat::run(src.data(), beg, ent_csr_adj(hg), V, E, gpu, ro)
                 : ent_compat::run_loaded(dg, src.data(), ro);
  if (jf) fclose(jf);
  release();
  return rc;
}
