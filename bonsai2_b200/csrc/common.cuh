// common.cuh -- shared definitions of the B200 tree-code kernels.
//
// Layout conventions (all device arrays are owned by one Treecode handle):
//   positions   float4 (x, y, z, mass)        -- Particle4<float>, Particle4.h:59-83
//   velocities  float4 (vx, vy, vz, unused)
//   accel       float4 (ax, ay, az, potential) -- computeForces.cu:611-617
//   CellData    uint4  (parent | level<<27, first | (n-1)<<29 or ~0 for a
//                       leaf, pbeg, pend)      -- Treecode.h:45-89
//   cell_open   float4 (com x,y,z, cellOp^2)   -- d_cellSize, computeMultipoles.cu:180
//   cell_stage  3 x float4 per cell, the walk's staged quadrupole record:
//               (COM, -0.5 tr I), (M, -3Ixx, -3Iyy, -3Izz),
//               (-3Ixy, -3Ixz, -3Iyz, -1.5 tr I), I the mass-weighted
//               central second moments (multipoles.cu)
//   GroupData   int2   (pbeg, np)              -- Treecode.h:29-43
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

// sm_100a only: the device code uses sm_100 packed FP32 (FFMA2) and
// redux.sync.f32, and no other target is built.
#if defined(__CUDA_ARCH__) && (__CUDA_ARCH__ != 1000 || !defined(__CUDA_ARCH_FEAT_SM100_ALL))
#error "bonsai_b200 device code is compiled for sm_100a only (-gencode arch=compute_100a,code=sm_100a)"
#endif

namespace bonsai {

constexpr int kMaxLevel = 21;        // 3 bits per level in a 63-bit key
constexpr int kLevels = 32;          // level table size (reference: 32, Treecode.h:171)
constexpr unsigned kFull = 0xffffffffu;

// Device status word bits (sticky; read by the host after a stage).
enum : int {
  kStatusCellCapacity = 1 << 0,   // more cells than the cell arrays hold
  kStatusDepth = 1 << 1,          // a level-21 cell holds more than nLeaf (kept as a fat leaf)
  kStatusWalkStack = 1 << 2,      // a walk level list outgrew its ring
  kStatusNonFinite = 1 << 3,      // NaN/Inf coordinate seen by the box reduction
  kStatusGroupCapacity = 1 << 4,  // more groups than the group array holds
  kStatusBadParam = 1 << 5,
  kStatusSortTimeout = 1 << 6,    // a sort look-back wait hit its bound (results invalid)
};

// Device-resident tree/group bookkeeping: written by the build kernels and
// read by later kernels, so no stage needs a host round trip.
struct TreeInfo {
  int ncells;
  int nleaves;
  int nnodes;
  int nlevels;
  int ngroups;
  int status;
  int npart;  // particles of the build (all systems of an ensemble)
  int pad;
  int level_beg[kLevels];   // half-open [beg, end) cell range of level L
  int level_end[kLevels];
};

// Per-cell FP64 record used by the bottom-up multipole pass (the particle
// bounding box is a separate array, float or double with the positions).
struct MpRec {
  double m, cx, cy, cz;
  double ixx, iyy, izz, ixy, ixz, iyz;
};

struct Box {
  float cx, cy, cz, hsize;
};

__device__ __forceinline__ unsigned lanemask_lt() {
  unsigned m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

__device__ __forceinline__ int lane_id() { return threadIdx.x & 31; }

// sm_100a: single-instruction warp min/max of f32 (redux.sync .f32).
__device__ __forceinline__ float warp_min_f32(float v) {
  float r;
  asm volatile("redux.sync.min.f32 %0, %1, 0xffffffff;" : "=f"(r) : "f"(v));
  return r;
}
__device__ __forceinline__ float warp_max_f32(float v) {
  float r;
  asm volatile("redux.sync.max.f32 %0, %1, 0xffffffff;" : "=f"(r) : "f"(v));
  return r;
}

// inclusive warp scan of ints
__device__ __forceinline__ int warp_incl_scan(int v) {
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int t = __shfl_up_sync(kFull, v, o);
    if (lane_id() >= o) v += t;
  }
  return v;
}

__device__ __forceinline__ int set_status(int* status, int bit) {
  return atomicOr(status, bit);
}

// Bounds-checked build (compiled with -DBONSAI_CHECKS).  BONSAI_IN_RANGE(i, n,
// site) tests 0 <= i < n; a failure is counted in this translation unit's
// word, the first failing site is recorded, and the caller skips the access
// (no trap: the kernel runs on and the host reads the count).  Sites are
// (kernel file << 8) | number.  In the normal build the macro is the constant
// true and the guarded accesses compile exactly as before.
#ifdef BONSAI_CHECKS
static __device__ unsigned g_bounds_word[2];  // violations, first failing site
__device__ __forceinline__ bool in_range_checked(long long i, long long n, unsigned site) {
  if (i >= 0 && i < n) return true;
  if (atomicAdd(&g_bounds_word[0], 1u) == 0u) g_bounds_word[1] = site;
  return false;
}
#define BONSAI_IN_RANGE(i, n, site) ::bonsai::in_range_checked((long long)(i), (long long)(n), (unsigned)(site))
// host accessor of this translation unit's word (after a device synchronise)
#define BONSAI_BOUNDS_ACCESSOR(name)                                                    \
  int name(unsigned* w, bool reset) {                                                   \
    if (cudaMemcpyFromSymbol(w, g_bounds_word, 2 * sizeof(unsigned)) != cudaSuccess)    \
      return -1;                                                                        \
    const unsigned zero[2] = {0u, 0u};                                                  \
    if (reset && cudaMemcpyToSymbol(g_bounds_word, zero, sizeof(zero)) != cudaSuccess) \
      return -1;                                                                        \
    return 0;                                                                           \
  }
#else
#define BONSAI_IN_RANGE(i, n, site) true
#define BONSAI_BOUNDS_ACCESSOR(name) \
  int name(unsigned* w, bool) {      \
    w[0] = w[1] = 0u;                \
    return 0;                        \
  }
#endif

// Ensemble layout: system s owns particles [off[s], off[s+1]) of the state
// arrays; every stage keeps that partition (sorts and gathers stay inside a
// system).  Chunks are the per-block work units of the per-system passes: at
// most kChunk particles of one system, {begin, end, system, 0}.
constexpr int kChunk = 4096;

// largest s in [0, nsys) with off[s] <= i
__device__ __forceinline__ int sys_of(const int* __restrict__ off, int nsys, int i) {
  int lo = 0, hi = nsys;
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (__ldg(off + mid) <= i) lo = mid; else hi = mid;
  }
  return lo;
}

// computeBoundingBox's finalisation (buildTree.cu:145-161) from the particle
// extent [a, b]: hsize = smallest power of two >= the largest half extent
// (floored at max(2^-100, 2^-40 * pow2 >= max|c|), so that a zero-extent
// input still gives a finite box whose centre quantisation fits 64 bits),
// centre quantised to hsize/2^20.
__device__ __forceinline__ Box box_from_extent(const float a[3], const float b[3]) {
  float c[3], h[3];
  for (int k = 0; k < 3; k++) { c[k] = (b[k] + a[k]) * 0.5f; h[k] = (b[k] - a[k]) * 0.5f; }
  const float hm = fmaxf(h[2], fmaxf(h[1], h[0]));
  const float cm = fmaxf(fabsf(c[0]), fmaxf(fabsf(c[1]), fabsf(c[2])));
  float pw = 1.0f;
  while (pw < cm) pw *= 2.0f;
  while (pw * 0.5f >= cm && pw > 7.888609052210118e-31f) pw *= 0.5f;
  const float floor_h = fmaxf(pw * 9.094947017729282e-13f, 7.888609052210118e-31f);
  float hs = 1.0f;
  while (hs > hm && hs > floor_h) hs *= 0.5f;
  while (hs < hm) hs *= 2.0f;
  const float hq = __fdiv_rn(hs, (float)(1 << 20));
  Box bx;
  bx.cx = __fmul_rn(hq, (float)(long long)__fdiv_rn(c[0], hq));
  bx.cy = __fmul_rn(hq, (float)(long long)__fdiv_rn(c[1], hq));
  bx.cz = __fmul_rn(hq, (float)(long long)__fdiv_rn(c[2], hq));
  bx.hsize = hs;
  return bx;
}

// Level (1..21) of the first octant digit where two sorted 63-bit keys
// differ; kMaxLevel+1 when they are equal.
__device__ __forceinline__ int diff_level(unsigned long long a, unsigned long long b) {
  const unsigned long long x = a ^ b;
  if (x == 0ull) return kMaxLevel + 1;
  const int p = 63 - __clzll((long long)x);
  return (62 - p) / 3 + 1;
}

}  // namespace bonsai

#define BONSAI_CUDA_TRY(expr)                       \
  do {                                              \
    cudaError_t _e = (expr);                        \
    if (_e != cudaSuccess) return -(int)_e - 1000;  \
  } while (0)
