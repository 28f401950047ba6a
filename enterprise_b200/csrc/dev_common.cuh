// Device utilities shared by the traversal kernels: acquire/release accessors,
// warp/block scans and the single-pass decoupled look-back prefix sum
// (Merrill & Garland, "Single-pass Parallel Prefix Scan with Decoupled
// Look-back", NVIDIA TR 2016). The look-back replaces the reference's
// two-kernel Blelloch scan over 65,536 per-thread bin counts
// (scan.cuh:484-685, driven by insp_scan, scan.cuh:895-938).
#pragma once
#include <stdint.h>
#include <cuda_runtime.h>

namespace ent {

constexpr unsigned FULL = 0xffffffffu;

__device__ __forceinline__ void st_release(unsigned long long* p, unsigned long long v) {
  asm volatile("st.release.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ unsigned long long ld_acquire(const unsigned long long* p) {
  unsigned long long v;
  asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ uint32_t ld_cg(const uint32_t* p) { return __ldcg(p); }
__device__ __forceinline__ void red_or(uint32_t* p, uint32_t v) {
  asm volatile("red.relaxed.gpu.global.or.b32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ unsigned lanemask_lt() {
  unsigned m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

// Look-back status word: [63:34] epoch, [33:32] flag, [31:0] value.
constexpr unsigned long long LB_INVALID = 0, LB_AGG = 1, LB_PREFIX = 2;
__device__ __forceinline__ unsigned long long lb_pack(uint32_t epoch, unsigned long long flag, uint32_t value) {
  return ((unsigned long long)(epoch & 0x3fffffffu) << 34) | (flag << 32) | value;
}
__device__ __forceinline__ unsigned long long lb_flag(unsigned long long w, uint32_t epoch) {
  return ((uint32_t)(w >> 34) == (epoch & 0x3fffffffu)) ? ((w >> 32) & 3ull) : LB_INVALID;
}

// Spin limit for any wait in these kernels: a wait that exceeds it records
// an error bit and gives up, so a bug can never hang the GPU. An iteration
// (an acquire load, a load of the error word, a short sleep) takes about a
// microsecond, so a wait gives up after roughly a second; a predecessor
// tile is always held by a running CTA and publishes within microseconds.
constexpr int SPIN_LIMIT = 1 << 20;

// Inclusive warp scan of K lanes' values (each lane holds v[k]).
template <int K>
__device__ __forceinline__ void warp_incl_scan(uint32_t (&v)[K]) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
#pragma unroll
    for (int k = 0; k < K; ++k) {
      uint32_t y = __shfl_up_sync(FULL, v[k], o);
      if (lane >= o) v[k] += y;
    }
  }
}

// Exclusive block scan of K values per thread. smem: [32][K] words.
// Returns per-thread exclusive prefix in v and block totals in total.
template <int K>
__device__ __forceinline__ void block_excl_scan(uint32_t (&v)[K], uint32_t (&total)[K], uint32_t* smem) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  uint32_t orig[K];
#pragma unroll
  for (int k = 0; k < K; ++k) orig[k] = v[k];
  warp_incl_scan<K>(v);
  if (lane == 31) {
#pragma unroll
    for (int k = 0; k < K; ++k) smem[warp * K + k] = v[k];
  }
  __syncthreads();
  if (warp == 0) {
    uint32_t w[K];
#pragma unroll
    for (int k = 0; k < K; ++k) w[k] = lane < nw ? smem[lane * K + k] : 0u;
    warp_incl_scan<K>(w);
    if (lane < nw) {
#pragma unroll
      for (int k = 0; k < K; ++k) smem[lane * K + k] = w[k];
    }
  }
  __syncthreads();
#pragma unroll
  for (int k = 0; k < K; ++k) {
    uint32_t before = warp > 0 ? smem[(warp - 1) * K + k] : 0u;
    total[k] = smem[(nw - 1) * K + k];
    v[k] = before + v[k] - orig[k];
  }
  __syncthreads();
}

// Decoupled look-back for tile `tile` with K independent chains. status is
// this segment's array [tiles][KS] (KS >= K). agg: tile aggregates (valid in
// every thread). On return excl[k] (valid in every thread) is the exclusive
// prefix of chain k. *err gets bit 1 set if a wait timed out.
template <int K, int KS>
__device__ void lookback(unsigned long long* status, uint32_t tile, uint32_t epoch, const uint32_t (&agg)[K],
                         uint32_t (&excl)[K], uint32_t* s_excl, int* err, bool hold_first = false) {
  const int lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
    if (tile == 0) {
      if (!hold_first) {  // fault-injection hook: tile 0 never publishes, the others time out
#pragma unroll
        for (int k = 0; k < K; ++k) st_release(status + k, lb_pack(epoch, LB_PREFIX, agg[k]));
      }
    } else {
#pragma unroll
      for (int k = 0; k < K; ++k) st_release(status + (size_t)tile * KS + k, lb_pack(epoch, LB_AGG, agg[k]));
    }
  }
  if (tile == 0) {
#pragma unroll
    for (int k = 0; k < K; ++k) excl[k] = 0;
    return;
  }
  if (threadIdx.x < 32) {
#pragma unroll 1
    for (int k = 0; k < K; ++k) {
      uint32_t acc = 0;
      long pred = (long)tile - 1;
      int spins = 0;
      while (true) {
        long idx = pred - lane;
        unsigned long long w = idx >= 0 ? ld_acquire(status + (size_t)idx * KS + k) : lb_pack(epoch, LB_PREFIX, 0);
        unsigned long long f = idx >= 0 ? lb_flag(w, epoch) : LB_PREFIX;
        if (__any_sync(FULL, f == LB_INVALID)) {
          // give up (warp-uniformly) on timeout or once another tile timed out
          if (__any_sync(FULL, ++spins > SPIN_LIMIT || (*(volatile int*)err & 2))) {
            if (lane == 0) atomicOr(err, 2);
            break;
          }
          __nanosleep(32);
          continue;
        }
        unsigned pmask = __ballot_sync(FULL, f == LB_PREFIX);
        uint32_t val = (uint32_t)w;
        int stop = pmask ? (__ffs(pmask) - 1) : 31;
        uint32_t contrib = lane <= stop ? val : 0u;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) contrib += __shfl_xor_sync(FULL, contrib, o);
        acc += contrib;
        if (pmask) break;
        pred -= 32;
      }
      if (lane == 0) {
        s_excl[k] = acc;
        st_release(status + (size_t)tile * KS + k, lb_pack(epoch, LB_PREFIX, acc + agg[k]));
      }
    }
  }
  __syncthreads();
#pragma unroll
  for (int k = 0; k < K; ++k) excl[k] = s_excl[k];
  __syncthreads();
}

}  // namespace ent
