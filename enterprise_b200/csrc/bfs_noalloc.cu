// Breadth-first search that allocates no memory at all.
//
// Some callers cannot allocate GPU memory when they need a traversal: code on
// a latency-critical request path, where a cudaMalloc/cudaFree may
// synchronise the whole device and stall unrelated streams; plug-ins inside
// a host process whose GPU memory is already owned by another allocator (a
// framework's caching allocator or a fixed, pre-reserved budget); and code
// that must not fail half-way with an out-of-memory error. For them this file
// provides ent_bfs_noalloc: the caller passes the CSR and the depth output,
// both already on the GPU, and the traversal's scratch lives in a file-scope
// __device__ array that exists on every GPU that loads this library, for the
// lifetime of the process.
//
// The scratch holds a visited bitmap, two frontier queues and two counters
// for at most NOALLOC_MAX_VERTICES vertices (about 8.5 MB per GPU). Larger
// graphs are rejected with ENT_ERR_INVALID_ARG. The traversal is level-
// synchronous top-down; each level's kernel reads one frontier queue and
// appends the next with warp-aggregated atomics, exactly the depths every
// other entry point of this library produces.
//
// Sharing: every call uses the same array and leaves its last contents
// behind; each call clears the visited bitmap and the counters before it
// starts. Two calls whose work overlaps on the same GPU (for example from two
// host threads at once, or on two streams) race on the shared scratch and
// produce wrong results: callers must serialise them.
#include <cuda_runtime.h>
#include <mutex>
#include <stdint.h>
#include <vector>

#include "ent_internal.h"

namespace ent {

constexpr int64_t NOALLOC_MAX_VERTICES = 1 << 20;
constexpr int64_t NOALLOC_WORDS = NOALLOC_MAX_VERTICES / 32;

// Layout inside the scratch array (all offsets 256-byte aligned):
//   [0]                       uint32 visited[NOALLOC_WORDS]
//   [NOALLOC_WORDS*4]         int32  queue[2][NOALLOC_MAX_VERTICES]
//   [.. + 8*MAX]              int32  count[2]  (frontier sizes)
constexpr size_t NA_OFF_QUEUE = NOALLOC_WORDS * 4;
constexpr size_t NA_OFF_COUNT = NA_OFF_QUEUE + 2 * NOALLOC_MAX_VERTICES * 4;
constexpr size_t NA_BYTES = NA_OFF_COUNT + 256;

static __device__ __align__(256) unsigned char g_noalloc_scratch[NA_BYTES];

struct NaView {
  uint32_t* visited;
  int32_t* queue[2];
  int32_t* count;
};

__host__ __device__ inline NaView na_view(unsigned char* base) {
  NaView v;
  v.visited = reinterpret_cast<uint32_t*>(base);
  v.queue[0] = reinterpret_cast<int32_t*>(base + NA_OFF_QUEUE);
  v.queue[1] = v.queue[0] + NOALLOC_MAX_VERTICES;
  v.count = reinterpret_cast<int32_t*>(base + NA_OFF_COUNT);
  return v;
}

// Clears what must start at zero (visited bits, counters) and fills depth with -1.
__global__ void k_na_clear(unsigned char* scratch, int64_t V, int32_t* depth) {
  NaView s = na_view(scratch);
  const int64_t tid = blockIdx.x * (int64_t)blockDim.x + threadIdx.x, nth = (int64_t)gridDim.x * blockDim.x;
  const int64_t W = (V + 31) / 32;
  for (int64_t i = tid; i < W; i += nth) s.visited[i] = 0;
  for (int64_t i = tid; i < V; i += nth) depth[i] = -1;
  if (tid < 2) s.count[tid] = 0;
}

__global__ void k_na_seed(unsigned char* scratch, int32_t src, int32_t* depth) {
  NaView s = na_view(scratch);
  depth[src] = 0;
  s.visited[src >> 5] = 1u << (src & 31);
  s.queue[0][0] = src;
  s.count[0] = 1;
  s.count[1] = 0;
}

// One top-down level: a warp per frontier vertex, lanes over its neighbours.
__global__ void k_na_expand(unsigned char* scratch, const int64_t* __restrict__ off, const int32_t* __restrict__ adj,
                            int cur, int32_t next_level, int32_t* depth) {
  NaView s = na_view(scratch);
  const int32_t* q = s.queue[cur];
  int32_t* qn = s.queue[cur ^ 1];
  int32_t* cn = &s.count[cur ^ 1];
  const int n = s.count[cur];
  const int lane = threadIdx.x & 31;
  const int gw = (int)((blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5);
  const int nw = (int)(((int64_t)gridDim.x * blockDim.x) >> 5);
  for (int i = gw; i < n; i += nw) {
    const int u = q[i];
    const int64_t beg = off[u], end = off[u + 1];
    for (int64_t e0 = beg; e0 < end; e0 += 32) {
      const int64_t e = e0 + lane;
      bool mine = false;
      int v = 0;
      if (e < end) {
        v = adj[e];
        const uint32_t b = 1u << (v & 31);
        if (!(s.visited[v >> 5] & b) && !(atomicOr(&s.visited[v >> 5], b) & b)) {
          mine = true;
          depth[v] = next_level;
        }
      }
      const unsigned m = __ballot_sync(0xffffffffu, mine);
      if (m) {
        const int leader = __ffs(m) - 1;
        int base = 0;
        if (lane == leader) base = atomicAdd(cn, __popc(m));
        base = __shfl_sync(0xffffffffu, base, leader);
        if (mine) qn[base + __popc(m & ((1u << lane) - 1))] = v;
      }
    }
  }
}

// Device address of the scratch array, looked up once per device and CUDA
// context with that device current (in host code the symbol's name is only a
// stand-in). An address is valid only in the context it was looked up in, so
// a caller that switches between the runtime's primary context and a context
// of its own (a driver-API plug-in) gets one lookup in each.
typedef int (*CtxGetCurrentFn)(void**);  // cuCtxGetCurrent, from the driver
struct NaEntry {
  int dev;
  void* ctx;
  unsigned char* ptr;
};
static std::mutex g_na_mu;
static std::vector<NaEntry> g_na_cache;
static CtxGetCurrentFn g_ctx_get = nullptr;

static int na_scratch_for_current_device(unsigned char** out) {
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return fail(ENT_ERR_CUDA, "cudaGetDevice failed: %s", cudaGetErrorString(e));
  std::lock_guard<std::mutex> lk(g_na_mu);
  if (!g_ctx_get) {
    void* fn = nullptr;
    cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
    e = cudaGetDriverEntryPoint("cuCtxGetCurrent", &fn, cudaEnableDefault, &q);
    if (e != cudaSuccess || q != cudaDriverEntryPointSuccess || !fn)
      return fail(ENT_ERR_CUDA, "driver entry point cuCtxGetCurrent unavailable: %s", cudaGetErrorString(e));
    g_ctx_get = reinterpret_cast<CtxGetCurrentFn>(fn);
  }
  void* ctx = nullptr;
  if (g_ctx_get(&ctx) != 0) return fail(ENT_ERR_CUDA, "cuCtxGetCurrent failed on device %d", dev);
  if (ctx)
    for (const NaEntry& n : g_na_cache)
      if (n.dev == dev && n.ctx == ctx) {
        *out = n.ptr;
        return ENT_OK;
      }
  // Not seen in this context (or no context is bound to this thread yet: the
  // lookup binds the device's primary context, as any runtime call does).
  void* p = nullptr;
  e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
  if (e != cudaSuccess || !p)
    return fail(ENT_ERR_CUDA, "cudaGetSymbolAddress(scratch) failed on device %d: %s", dev, cudaGetErrorString(e));
  if (!ctx && (g_ctx_get(&ctx) != 0 || !ctx)) return fail(ENT_ERR_CUDA, "no current CUDA context on device %d", dev);
  g_na_cache.push_back(NaEntry{dev, ctx, static_cast<unsigned char*>(p)});
  *out = static_cast<unsigned char*>(p);
  return ENT_OK;
}

}  // namespace ent

using namespace ent;

extern "C" int ent_bfs_noalloc(const int64_t* beg_pos_dev, const int32_t* csr_dev, int64_t vert_count, int32_t src,
                               int32_t* depth_dev, void* stream) {
  clear_error();
  if (!beg_pos_dev || !csr_dev || !depth_dev) return fail(ENT_ERR_INVALID_ARG, "null device pointer");
  if (vert_count < 1) return fail(ENT_ERR_INVALID_ARG, "vert_count must be >= 1");
  if (vert_count > NOALLOC_MAX_VERTICES)
    return fail(ENT_ERR_INVALID_ARG,
                "vert_count %lld exceeds the no-allocation limit of %lld vertices (use ent_bfs_device instead)",
                (long long)vert_count, (long long)NOALLOC_MAX_VERTICES);
  if (src < 0 || src >= vert_count) return fail(ENT_ERR_INVALID_ARG, "source %d out of range [0,%lld)", src, (long long)vert_count);
  unsigned char* scratch = nullptr;
  int rc = na_scratch_for_current_device(&scratch);
  if (rc != ENT_OK) return rc;
  cudaStream_t s = (cudaStream_t)stream;
  int dev_sms = 148;
  int dev = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&dev_sms, cudaDevAttrMultiProcessorCount, dev);
  const int blocks = dev_sms * 8;
  k_na_clear<<<blocks, 256, 0, s>>>(scratch, vert_count, depth_dev);
  k_na_seed<<<1, 1, 0, s>>>(scratch, src, depth_dev);
  g_kernel_launches += 2;
  NaView view = na_view(scratch);
  int cur = 0;
  for (int64_t level = 0; level <= vert_count; ++level) {
    k_na_expand<<<blocks, 256, 0, s>>>(scratch, beg_pos_dev, csr_dev, cur, (int32_t)(level + 1), depth_dev);
    g_kernel_launches++;
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail(ENT_ERR_CUDA, "level kernel launch failed: %s", cudaGetErrorString(e));
    int32_t next = 0;
    // 4-byte read of the next frontier size into a host variable (no allocation)
    e = cudaMemcpyAsync(&next, view.count + (cur ^ 1), sizeof(int32_t), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return fail(ENT_ERR_CUDA, "level sync failed: %s", cudaGetErrorString(e));
    if (next == 0) return ENT_OK;
    e = cudaMemsetAsync(view.count + cur, 0, sizeof(int32_t), s);
    if (e != cudaSuccess) return fail(ENT_ERR_CUDA, "counter reset failed: %s", cudaGetErrorString(e));
    cur ^= 1;
  }
  return fail(ENT_ERR_INTERNAL, "level loop did not terminate");
}
