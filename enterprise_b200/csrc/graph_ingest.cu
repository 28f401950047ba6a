// Loads a graph in the reference's binary format straight into device memory.
//
// The reference reads beg_pos.bin (int64[V+1]) and csr.bin (int64[E]) into
// host arrays and narrows the column ids to int32 in a serial loop
// (graph.hpp:33-118) before its allocator copies them to the GPU
// (allocator.cuh:107-120). Here the file is streamed to the GPU:
//  * beg_pos is read with parallel pread, checked on the host (beg_pos[0] ==
//    0, monotone) and copied once;
//  * csr.bin is read in chunks by several threads (pread at disjoint offsets)
//    into two pinned buffers in turn; each chunk is copied asynchronously and a
//    kernel narrows int64 ids to int32 (or checks int32 ids) in place in the
//    graph's column array, recording the first id outside [0, V). Reading
//    chunk i+1 overlaps the copy and kernel of chunk i.
// Format rules and error messages are those of ent_csr_load (int64 or int32
// csr.bin, told apart by its size against beg_pos[V]).
#include <fcntl.h>
#include <omp.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <string>
#include <vector>

#include "dev_graph.h"

namespace ent {
namespace {

constexpr int64_t CHUNK = 64ll << 20;  // bytes per streamed chunk of csr.bin

__global__ void k_narrow_ids(const int64_t* __restrict__ in, int64_t n, int64_t V, int64_t first,
                             int32_t* __restrict__ out, unsigned long long* bad) {
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
    const int64_t x = in[k];
    if (x < 0 || x >= V) atomicMin(bad, (unsigned long long)(first + k));
    out[k] = (int32_t)x;
  }
}

__global__ void k_check_ids(const int32_t* __restrict__ ids, int64_t n, int64_t V, int64_t first,
                            unsigned long long* bad) {
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x)
    if (ids[k] < 0 || ids[k] >= V) atomicMin(bad, (unsigned long long)(first + k));
}

int64_t file_bytes(const char* p) {
  struct stat st;
  return stat(p, &st) == 0 ? (int64_t)st.st_size : -1;
}

// Reads n bytes at offset off of fd into dst with up to `threads` parallel
// preads; false on a short read or error.
bool pread_all(int fd, void* dst, int64_t n, int64_t off, int threads) {
  const int64_t piece = std::max<int64_t>(1 << 20, (n + threads - 1) / threads);
  const int64_t pieces = (n + piece - 1) / piece;
  bool ok = true;
#pragma omp parallel for num_threads(threads) reduction(&& : ok)
  for (int64_t i = 0; i < pieces; ++i) {
    int64_t a = i * piece, b = std::min(n, a + piece);
    while (a < b) {
      const ssize_t r = pread(fd, (char*)dst + a, (size_t)(b - a), (off_t)(off + a));
      if (r <= 0) {
        ok = false;
        break;
      }
      a += r;
    }
  }
  return ok;
}

struct Fd {
  int fd = -1;
  ~Fd() {
    if (fd >= 0) close(fd);
  }
};

}  // namespace
}  // namespace ent

using namespace ent;

extern "C" int ent_graph_load(const char* beg_path, const char* csr_path, int32_t gpu, ent_graph** out) {
  ent::NvtxRange nvtx_range("ent_graph_load");
  clear_error();
  if (!beg_path || !csr_path || !out) return fail(ENT_ERR_INVALID_ARG, "null argument");
  *out = nullptr;
  const int64_t bsz = file_bytes(beg_path);
  if (bsz < 0) return fail(ENT_ERR_IO, "beg file cannot open: %s", beg_path);
  if (bsz < 16 || bsz % 8 != 0)
    return fail(ENT_ERR_FORMAT, "beg_pos file size %lld is not 8*(V+1) with V>=1", (long long)bsz);
  const int64_t csz = file_bytes(csr_path);
  if (csz < 0) return fail(ENT_ERR_IO, "CSR file cannot open: %s", csr_path);
  const int64_t V = bsz / 8 - 1;
  if (V >= (1ll << 31) - 1) return fail(ENT_ERR_UNSUPPORTED, "V=%lld exceeds int32 ids", (long long)V);
  const int threads = std::max(1, std::min(8, omp_get_max_threads()));

  // ---- beg_pos: read and checked on the host before any device work, so a
  // malformed file fails the same way with or without a GPU
  Fd fb;
  fb.fd = open(beg_path, O_RDONLY);
  if (fb.fd < 0) return fail(ENT_ERR_IO, "beg file cannot open: %s", beg_path);
  std::vector<int64_t> off_v(V + 1);
  int64_t* off_h = off_v.data();
  if (!pread_all(fb.fd, off_h, bsz, 0, threads)) return fail(ENT_ERR_IO, "short read on %s", beg_path);
  if (off_h[0] != 0) return fail(ENT_ERR_FORMAT, "beg_pos[0]=%lld, expected 0", (long long)off_h[0]);
  int64_t first_dec = V;
#pragma omp parallel for num_threads(threads) reduction(min : first_dec)
  for (int64_t i = 0; i < V; ++i)
    if (off_h[i + 1] < off_h[i]) first_dec = std::min(first_dec, i);
  if (first_dec < V)
    return fail(ENT_ERR_FORMAT, "beg_pos not monotone at %lld (%lld > %lld)", (long long)first_dec,
                (long long)off_h[first_dec], (long long)off_h[first_dec + 1]);
  const int64_t E = off_h[V];
  int width;
  if (csz == E * 8) width = 8;
  else if (csz == E * 4) width = 4;
  else
    return fail(ENT_ERR_FORMAT, "csr file size %lld matches neither int64 nor int32 for beg_pos[V]=%lld",
                (long long)csz, (long long)E);

  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return fail(ENT_ERR_CUDA, "no CUDA device available");
  if (gpu < 0 || gpu >= ndev) return fail(ENT_ERR_INVALID_ARG, "gpu_id %d out of range (%d devices)", gpu, ndev);
  DeviceGuard dg(gpu);

  // ---- device graph and streamed columns
  Fd fc;
  fc.fd = open(csr_path, O_RDONLY);
  if (fc.fd < 0) return fail(ENT_ERR_IO, "CSR file cannot open: %s", csr_path);
  ent_graph* g = new ent_graph();
  g->device = gpu;
  int rc = graph_alloc(g, V, E);
  cudaError_t e = rc == ENT_OK ? cudaStreamCreateWithFlags(&g->stream, cudaStreamNonBlocking) : cudaSuccess;
  void* pin[2] = {nullptr, nullptr};
  int64_t* stage[2] = {nullptr, nullptr};
  cudaEvent_t done[2] = {nullptr, nullptr};
  unsigned long long* d_bad = nullptr;
  unsigned long long bad = ~0ull;
  int nsm = 148;
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, gpu);
  const int64_t chunk = std::min<int64_t>(CHUNK, std::max<int64_t>(E * width, 8));
  for (int b = 0; b < 2 && e == cudaSuccess && rc == ENT_OK; ++b) {
    e = cudaMallocHost(&pin[b], chunk);
    if (e == cudaSuccess && width == 8) e = cudaMalloc(&stage[b], chunk);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&done[b], cudaEventDisableTiming);
  }
  if (e == cudaSuccess && rc == ENT_OK) e = cudaMalloc(&d_bad, sizeof(bad));
  if (e == cudaSuccess && rc == ENT_OK) e = cudaMemcpyAsync(d_bad, &bad, sizeof(bad), cudaMemcpyHostToDevice, g->stream);
  if (e == cudaSuccess && rc == ENT_OK)
    e = cudaMemcpyAsync(g->off, off_h, sizeof(int64_t) * (V + 1), cudaMemcpyHostToDevice, g->stream);
  const int64_t per = chunk / width;  // ids per chunk
  bool short_read = false;
  for (int64_t c = 0, pos = 0; pos < E && e == cudaSuccess && rc == ENT_OK; ++c, pos += per) {
    const int b = (int)(c & 1);
    const int64_t n = std::min(per, E - pos);
    e = cudaEventSynchronize(done[b]);  // the copy and kernel that last used buffer b are done
    if (e != cudaSuccess) break;
    if (!pread_all(fc.fd, pin[b], n * width, pos * width, threads)) {
      short_read = true;
      break;
    }
    const int blocks = (int)std::min<int64_t>((n + 255) / 256, (int64_t)nsm * 8);
    if (width == 8) {
      e = cudaMemcpyAsync(stage[b], pin[b], n * 8, cudaMemcpyHostToDevice, g->stream);
      if (e == cudaSuccess) k_narrow_ids<<<blocks, 256, 0, g->stream>>>(stage[b], n, V, pos, g->adj + pos, d_bad);
    } else {
      e = cudaMemcpyAsync(g->adj + pos, pin[b], n * 4, cudaMemcpyHostToDevice, g->stream);
      if (e == cudaSuccess) k_check_ids<<<blocks, 256, 0, g->stream>>>(g->adj + pos, n, V, pos, d_bad);
    }
    g_kernel_launches++;
    if (e == cudaSuccess) e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaEventRecord(done[b], g->stream);
  }
  if (e == cudaSuccess && rc == ENT_OK && !short_read)
    e = cudaMemcpyAsync(&bad, d_bad, sizeof(bad), cudaMemcpyDeviceToHost, g->stream);
  const cudaError_t es = g->stream ? cudaStreamSynchronize(g->stream) : cudaSuccess;
  for (int b = 0; b < 2; ++b) {
    if (pin[b]) cudaFreeHost(pin[b]);
    if (stage[b]) cudaFree(stage[b]);
    if (done[b]) cudaEventDestroy(done[b]);
  }
  if (d_bad) cudaFree(d_bad);
  if (rc == ENT_OK && short_read) rc = fail(ENT_ERR_IO, "short read on %s", csr_path);
  if (rc == ENT_OK && (e != cudaSuccess || es != cudaSuccess))
    rc = fail(ENT_ERR_CUDA, "graph upload failed: %s", cudaGetErrorString(e != cudaSuccess ? e : es));
  if (rc == ENT_OK && bad != ~0ull) rc = fail(ENT_ERR_FORMAT, "csr entry %lld out of range [0,V)", (long long)bad);
  if (rc == ENT_OK) rc = graph_finish(g);
  if (rc != ENT_OK) {
    const std::string msg = ent_last_error();  // destroying the graph clears the error
    ent_graph_destroy(g);
    return fail(rc, "%s", msg.c_str());
  }
  *out = g;
  return ENT_OK;
}
