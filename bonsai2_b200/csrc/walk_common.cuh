// walk_common.cuh -- pieces shared by the float walk (walk.cu) and the FP64
// checker walk (walk64.cu), so that both take the same opening decisions.
#pragma once
#include "common.cuh"

namespace bonsai {

// Squared distance from the group's box to a cell's centre of mass, the
// quantity of split_node_grav_impbh (computeForces.cu:30-54), explicitly
// rounded so that the CPU restatement reproduces it bit for bit.
__device__ __forceinline__ float box_dist2(const float4 co, const float3 gc, const float3 gs) {
  float dx = __fsub_rn(fabsf(__fsub_rn(gc.x, co.x)), gs.x);
  float dy = __fsub_rn(fabsf(__fsub_rn(gc.y, co.y)), gs.y);
  float dz = __fsub_rn(fabsf(__fsub_rn(gc.z, co.z)), gs.z);
  dx = __fmul_rn(__fadd_rn(dx, fabsf(dx)), 0.5f);
  dy = __fmul_rn(__fadd_rn(dy, fabsf(dy)), 0.5f);
  dz = __fmul_rn(__fadd_rn(dz, fabsf(dz)), 0.5f);
  return __fmaf_rn(dz, dz, __fmaf_rn(dy, dy, __fmul_rn(dx, dx)));
}

// Opening test of split_node_grav_impbh: open when ds^2 < cellOp^2.
__device__ __forceinline__ bool open_cell(const float4 co, const float3 gc, const float3 gs) {
  return box_dist2(co, gc, gs) < fabsf(co.w);
}

// Mass-weighted opening test of the relative accuracy mode: a cell that
// passes the geometric test is still opened when the octupole truncation
// error of its quadrupole expansion, of order M l^3 / ds^5, exceeds the
// group's bound tau (tau = alpha |a| of the group: the relative error
// criterion of tree codes with a relative opening rule).  mk = M l^3 as the
// multipole kernel stored it (cell_ls.z).
__device__ __forceinline__ bool open_relative(const float4 co, const float3 gc, const float3 gs, float mk, float tau) {
  const float ds2 = box_dist2(co, gc, gs);
  const float ds5 = __fmul_rn(__fmul_rn(ds2, ds2), __fsqrt_rn(ds2));
  return mk > __fmul_rn(tau, ds5);
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
