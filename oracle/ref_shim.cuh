// ref_shim.cuh -- stand-ins for the CUDA features that the reference's walk
// (code/computeForces.cu) uses and that CUDA 12 removed: legacy texture
// references and cudaBindTexture/cudaUnbindTexture.  Test and baseline
// infrastructure only, included by oracle/ref_walk_main.cu before the
// modified reference files that oracle/make_modref.py writes.
//
// A RefTexture<T> is a __device__ (pointer, length) pair.  bindTexture
// (code/cuda_primitives.h:24-32) sets it through cudaBindTexture below, which
// copies the pair to the device variable; tex1Dfetch reads element i with
// __ldg when 0 <= i < length.  Out of range a texture fetch from linear memory
// returned zero and read nothing; the walk relies on that, because lanes whose
// list entry lies past the current level read stale or unwritten list slots
// and fetch whatever cell index they find (their results are masked off).  So
// an out-of-range fetch reads nothing here either and returns zero -- except
// for the cell-record type (uint4), where it returns an empty leaf
// (first = ~0, pbeg = pend = 0).  Masked lanes discard the record either way;
// the leaf makes sure that a corrupted list could never expand a stale entry
// into a child range and keep a warp walking.
#pragma once
#include <cstddef>
#include <cuda_runtime.h>

template <typename T>
struct RefTexture {
  const T* ptr;
  int n;
  cudaTextureAddressMode addressMode[3];
  cudaTextureFilterMode filterMode;
  int normalized;
};

template <typename T>
__device__ __forceinline__ T ref_texture_outside() {
  return T{};
}
template <>
__device__ __forceinline__ uint4 ref_texture_outside<uint4>() {
  return make_uint4(0u, 0xFFFFFFFFu, 0u, 0u);
}

template <typename T>
__device__ __forceinline__ T tex1Dfetch(const RefTexture<T>& t, const int i) {
  if (i >= 0 && i < t.n) return __ldg(t.ptr + i);
  return ref_texture_outside<T>();
}

// `tex` is the host-side handle of the __device__ RefTexture (what
// cudaMemcpyToSymbol takes); its fields are written on the device only.
template <typename T>
cudaError_t cudaBindTexture(size_t* /*offset*/, RefTexture<T>& tex, const void* ptr, size_t bytes) {
  RefTexture<T> v{};
  v.ptr = static_cast<const T*>(ptr);
  v.n = static_cast<int>(bytes / sizeof(T));
  return cudaMemcpyToSymbol(tex, &v, sizeof(v));
}

template <typename T>
cudaError_t cudaUnbindTexture(RefTexture<T>& tex) {
  const RefTexture<T> v{};
  return cudaMemcpyToSymbol(tex, &v, sizeof(v));
}
