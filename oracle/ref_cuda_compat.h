// Compatibility layer that lets the reference's GPU BFS (written for CUDA
// 5.5-7.5 and sm_35) compile unmodified with CUDA 12.9 for sm_100a. Force-
// included (nvcc -include) ahead of the reference's own headers by
// oracle/Makefile. TEST INFRASTRUCTURE ONLY: it exists to run the reference
// itself on small graphs and record its depths as golden vectors.
//
// What changed in CUDA since the reference was written, and the stand-in:
//  * texture references (texture<T,1,mode> + cudaBindTexture + tex1Dfetch,
//    comm.h:163-169, allocator.cuh) were removed in CUDA 12. A texture
//    reference becomes a __device__ struct holding the bound pointer;
//    cudaBindTexture stores the pointer into it; tex1Dfetch reads through it.
//  * the unmasked warp votes __any/__all (expander.cuh:48, :616, :645, :663)
//    are invalid from sm_70 on; they become __any_sync/__all_sync over the full
//    warp. The reference reaches every vote with all 32 lanes (its warp loops
//    have warp-uniform trip counts), which the _sync forms require.
//  * cudaThreadSynchronize (inspector.cuh:484, scan.cuh:927) became
//    cudaDeviceSynchronize.
#pragma once
#include <cuda_runtime.h>

template <class T, int dim, enum cudaTextureReadMode mode>
struct ent_compat_tex {
  const T* ptr;
};

#define texture __device__ ent_compat_tex

template <class T, int dim, enum cudaTextureReadMode mode>
__device__ __forceinline__ T tex1Dfetch(const ent_compat_tex<T, dim, mode>& t, int i) {
  return t.ptr[i];
}

template <class T, int dim, enum cudaTextureReadMode mode>
static inline cudaError_t cudaBindTexture(size_t*, const ent_compat_tex<T, dim, mode>& tex, const void* p,
                                          size_t) {
  const T* ptr = static_cast<const T*>(p);
  return cudaMemcpyToSymbol(tex, &ptr, sizeof(ptr));
}

#define __any(x) __any_sync(0xffffffffu, (x))
#define __all(x) __all_sync(0xffffffffu, (x))
#define cudaThreadSynchronize cudaDeviceSynchronize
