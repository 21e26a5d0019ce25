// walk_common.cuh -- pieces shared by the float walk (walk.cu) and the FP64
// checker walk (walk64.cu), so that both take the same opening decisions.
#pragma once
#include "common.cuh"

namespace bonsai {

// Opening test of split_node_grav_impbh (computeForces.cu:30-54), explicitly
// rounded so that the CPU restatement reproduces it bit for bit.
__device__ __forceinline__ bool open_cell(const float4 co, const float3 gc, const float3 gs) {
  float dx = __fsub_rn(fabsf(__fsub_rn(gc.x, co.x)), gs.x);
  float dy = __fsub_rn(fabsf(__fsub_rn(gc.y, co.y)), gs.y);
  float dz = __fsub_rn(fabsf(__fsub_rn(gc.z, co.z)), gs.z);
  dx = __fmul_rn(__fadd_rn(dx, fabsf(dx)), 0.5f);
  dy = __fmul_rn(__fadd_rn(dy, fabsf(dy)), 0.5f);
  dz = __fmul_rn(__fadd_rn(dz, fabsf(dz)), 0.5f);
  const float ds2 = __fmaf_rn(dz, dz, __fmaf_rn(dy, dy, __fmul_rn(dx, dx)));
  return ds2 < fabsf(co.w);
}

// binary search over the warp's inclusive scan: the lane whose range holds s
__device__ __forceinline__ int find_src(int incl, int s) {
  int src = 0;
#pragma unroll
  for (int step = 16; step >= 1; step >>= 1) {
    const int v = __shfl_sync(kFull, incl, src + step - 1);
    if (v <= s) src += step;
  }
  return src;
}

}  // namespace bonsai
