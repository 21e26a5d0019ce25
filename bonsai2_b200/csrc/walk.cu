// walk.cu -- the tree walk: one warp per group, FP32, persistent.
//
// Semantics follow treewalk / treewalk_warp (computeForces.cu:229-619):
//   * a warp takes the next group from an atomic counter (:516-522); its
//     particles are held in registers, up to 128 per group (the reference
//     allows 64, :661-694);
//   * group box from the min/max of its particles (:531-555);
//   * breadth-first walk from all level-1 cells (:259-263, :511-512);
//   * a cell is opened when split_node_grav_impbh holds (:30-54) or when it
//     holds fewer than 3 particles (:284-285);
//   * opened nodes push their children to the next level (:291-334);
//     cells that stay closed (leaves too) are quadrupoles (:337-367);
//     opened leaves are evaluated particle by particle, i==j included
//     (:370-430);
//   * acc = (ax, ay, az, potential) in group (PH) order (:611-617), interaction
//     counts per particle (:568-609).
// B200 design:
//   * explicit __shfl_sync / __ballot_sync / redux.sync cooperation, no
//     implicit warp-synchronous shared memory;
//   * range expansion from the warp's inclusive scan: opened nodes write
//     their own children at their offsets; leaf particles are expanded 32 at
//     a time by a shuffle binary search over the scan;
//   * the level lists live in a per-warp pair of buffers in global memory
//     (current level / next level, swapped per level; L1/L2 resident),
//     bounded; overflow sets a status bit, never traps;
//   * accepted cells (their records pre-staged by the multipole kernel in
//     cell_stage) and direct particles are copied by value with cp.async into
//     per-warp shared-memory rings (64 quadrupoles, 128 particles) as they
//     are found, and evaluated 32 at a time when the next 32-cell block
//     starts, so the copies land behind the warp's own traversal and the
//     32-wide evaluation loops read broadcast LDS.128 only;
//   * the quadrupole kernel uses mass-weighted, pre-scaled moments
//     (34 FP32 operations + 1 MUFU per interaction; the reference's
//     formulation, counted as 64 flops by treecode.cu:149-158, is the same
//     algebra), evaluated as packed FFMA2/FMUL2/FADD2 over pairs of a lane's
//     particles.
#include <algorithm>
#include <type_traits>

#include "common.cuh"
#include "kernels.cuh"
#include "walk_common.cuh"

namespace bonsai {

constexpr int kWalkWarps = kWalkThreads / 32;

// Tuning knobs (compile time, like the reference's NWARPS_OCTREE2 / NI
// template switches): half-warp source split, unroll depth of the 32-entry
// evaluation loops (the loop body must stay inside the instruction cache).
#ifndef BONSAI_WALK_SPLIT
#define BONSAI_WALK_SPLIT 1
#endif
#ifndef BONSAI_WALK_UNROLL
#define BONSAI_WALK_UNROLL 4
#endif
#define BONSAI_DO_PRAGMA(x) _Pragma(#x)
#define BONSAI_UNROLL_N(n) BONSAI_DO_PRAGMA(unroll n)

#ifndef BONSAI_WALK_PACKED
#define BONSAI_WALK_PACKED 1
#endif
// children of opened nodes written by their parent's lane (1) or expanded
// 32 at a time by a shuffle search over the warp's scan (0)
#ifndef BONSAI_WALK_CHILD_LOOP
#define BONSAI_WALK_CHILD_LOOP 1
#endif

struct IPart {
  float x, y, z;
};

// Staging knobs (walk at N = 2^24, theta 0.6, one B200):
//   BONSAI_WALK_ASYNC 1: accepted cells' staged records (cell_stage, 48 B)
//     and leaf particles are copied global -> shared by cp.async (LDGSTS,
//     cached in L1), waited for only when their batch is evaluated; 0: loaded
//     into registers and stored (the warp waits one L2 round trip per block);
//   BONSAI_WALK_EVAL_EARLY 1: a 32-cell block first evaluates the full
//     batches that earlier blocks staged, then reads its level-list entries
//     (63.4 ms; register staging with evaluation right after staging: 63.8);
//     0: it evaluates them while its own cell records are in flight (65.0 ms:
//     the records held across the evaluation loop cost it registers).
#ifndef BONSAI_WALK_ASYNC
#define BONSAI_WALK_ASYNC 1
#endif
#ifndef BONSAI_WALK_LIST_AHEAD
#define BONSAI_WALK_LIST_AHEAD 1
#endif
#ifndef BONSAI_WALK_EVAL_EARLY
#define BONSAI_WALK_EVAL_EARLY 1
#endif
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
#if BONSAI_WALK_ASYNC
  const unsigned d = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(gmem) : "memory");
#else
  *static_cast<float4*>(smem) = __ldg(static_cast<const float4*>(gmem));
#endif
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

// direct-source ring per warp (a power of two, >= 64)
constexpr int kDirRing = 128;
// double-single positions: the leaf particles' hi and lo parts are copied by
// cp.async into two rings (64 entries each, to stay within static shared
// memory) and combined into (hi - R) + lo in shared memory right before the
// batch is evaluated, one lane per entry; 0: loaded into registers and
// combined at staging (the warp waits a round trip per 32 particles)
#ifndef BONSAI_WALK_DS_ASYNC
#define BONSAI_WALK_DS_ASYNC 1
#endif

// Interaction arithmetic over V = float (one i-particle) or V = float2 (two
// i-particles of the lane, evaluated by the packed FFMA2/FMUL2/FADD2 of
// sm_100: one instruction per pair, same FP32 pipe rate, half the issue
// slots).  Sources are scalars broadcast into both halves.
__device__ __forceinline__ float vfma(float a, float b, float c) { return fmaf(a, b, c); }
__device__ __forceinline__ float vmul(float a, float b) { return a * b; }
__device__ __forceinline__ float vadd(float a, float b) { return a + b; }
__device__ __forceinline__ float vrsqrt(float a) { return rsqrtf(a); }
__device__ __forceinline__ float vdup(float a, float) { return a; }
__device__ __forceinline__ float2 vfma(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 vmul(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 vadd(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 vrsqrt(float2 a) { return make_float2(rsqrtf(a.x), rsqrtf(a.y)); }
__device__ __forceinline__ float2 vdup(float a, float2) { return make_float2(a, a); }

// i-state: negated coordinates n = -x_i; accumulators (ax, ay, az, -phi)
template <class V>
struct IVec {
  V nx, ny, nz;
};
template <class V>
struct AVec {
  V x, y, z, w;
};

// Staged sources.  Quadrupole (moments negated at staging):
//   a0 = (COM, -0.5 tr I), a1 = (M, -3Ixx, -3Iyy, -3Izz), a2 = (-3Ixy, -3Ixz, -3Iyz, -1.5 tr I)
// With d = COM - x_i = -dr, q = -3I d = 3 I dr and w = q.d = -3 dIdr:
//   phi -= M/r - 0.5 tr/r^3 + 1.5 dIdr/r^5
//   a   += [-M + u (1.5 tr - 7.5 dIdr u)] dr / r^3 + 3 I dr / r^5,   dr = x_i - COM
// is a += [M - u (1.5 tr + 2.5 w u)] d / r^3 + q / r^5 and
// -phi += [M + u (-0.5 tr - 0.5 w u)] / r: 34 FP32 operations + 1 rsqrt.
template <class V>
__device__ __forceinline__ void quad_acc(AVec<V>& acc, const IVec<V>& p, const float4 a0, const float4 a1,
                                         const float4 a2, V eps2) {
  const V dx = vadd(vdup(a0.x, eps2), p.nx), dy = vadd(vdup(a0.y, eps2), p.ny), dz = vadd(vdup(a0.z, eps2), p.nz);
  const V r2 = vfma(dz, dz, vfma(dy, dy, vfma(dx, dx, eps2)));
  const V rinv = vrsqrt(r2);
  const V u = vmul(rinv, rinv);
  const V qx = vfma(vdup(a2.y, eps2), dz, vfma(vdup(a2.x, eps2), dy, vmul(vdup(a1.y, eps2), dx)));
  const V qy = vfma(vdup(a2.z, eps2), dz, vfma(vdup(a1.z, eps2), dy, vmul(vdup(a2.x, eps2), dx)));
  const V qz = vfma(vdup(a1.w, eps2), dz, vfma(vdup(a2.z, eps2), dy, vmul(vdup(a2.y, eps2), dx)));
  const V qrr = vfma(qz, dz, vfma(qy, dy, vmul(qx, dx)));
  const V r3 = vmul(rinv, u);
  const V r5 = vmul(r3, u);
  const V b = vmul(qrr, u);
  const V ca = vmul(vfma(u, vfma(vdup(-2.5f, eps2), b, vdup(a2.w, eps2)), vdup(a1.x, eps2)), r3);
  acc.x = vfma(r5, qx, vfma(ca, dx, acc.x));
  acc.y = vfma(r5, qy, vfma(ca, dy, acc.y));
  acc.z = vfma(r5, qz, vfma(ca, dz, acc.z));
  const V pp = vfma(u, vfma(vdup(-0.5f, eps2), b, vdup(a0.w, eps2)), vdup(a1.x, eps2));
  acc.w = vfma(rinv, pp, acc.w);
}

// monopole (computeForces.cu:58-78): d = x_j - x_i
template <class V>
__device__ __forceinline__ void mono_acc(AVec<V>& acc, const IVec<V>& p, const float4 j, V eps2) {
  const V dx = vadd(vdup(j.x, eps2), p.nx), dy = vadd(vdup(j.y, eps2), p.ny), dz = vadd(vdup(j.z, eps2), p.nz);
  const V r2 = vfma(dz, dz, vfma(dy, dy, vfma(dx, dx, eps2)));
  const V rinv = vrsqrt(r2);
  const V mr = vmul(vdup(j.w, eps2), rinv);
  const V mr3 = vmul(vmul(mr, rinv), rinv);
  acc.w = vadd(acc.w, mr);
  acc.x = vfma(mr3, dx, acc.x);
  acc.y = vfma(mr3, dy, acc.y);
  acc.z = vfma(mr3, dz, acc.z);
}

// NI i-particles of a lane as NV vectors of type V
template <int NI>
struct Lanes {
#if BONSAI_WALK_PACKED
  typedef typename std::conditional<(NI >= 2), float2, float>::type V;
  static constexpr int NV = NI >= 2 ? NI / 2 : NI;
#else
  typedef float V;
  static constexpr int NV = NI;
#endif
};

__device__ __forceinline__ void set_lane(float& v, int, float x) { v = x; }
__device__ __forceinline__ void set_lane(float2& v, int h, float x) {
  if (h) v.y = x; else v.x = x;
}
__device__ __forceinline__ float get_lane(float v, int) { return v; }
__device__ __forceinline__ float get_lane(float2 v, int h) { return h ? v.y : v.x; }

// Particle ownership.  SPLIT: lane l holds particles (l & 15) + 16k, k < NI,
// both half-warps hold the same particles, the two halves evaluate alternate
// entries of every 32-entry batch and their sums are added once per group, so
// each broadcast shared-memory load feeds NI (= 4 for nCrit <= 64)
// interactions.  Otherwise lane l holds l + 32k, k < NI.
// PERGROUP: each group has its own opening angle (1/theta_g in
// group_inv_theta); the opening size is re-formed as (l/theta_g + s)^2 from
// cell_ls with the same rounding as the multipole kernel, so theta_g = theta
// reproduces the fixed-angle walk exactly.
// ENS: the particles form an ensemble of independent systems (sys_off); a
// group walks from its own system's level-1 cells [root_beg[s], root_beg[s+1])
// only, in the order the system alone would.
// DS: positions are double-single (hi in ipos/jpos/cell_open, lo in
// ipos_lo/jpos_lo/cell_lo).  Every coordinate the group uses is taken
// relative to the group's reference point R (its first particle's hi
// position) as (hi - R) + lo: the subtraction is exact for nearby points, so
// separations keep FP32 relative precision however far from the origin the
// group lies.  The interaction loops are unchanged.
template <int NI, bool SPLIT, bool PERGROUP, bool ENS, bool DS>
__global__ void __launch_bounds__(kWalkThreads, kWalkMinBlocks)
    k_walk(const int2* __restrict__ groups, const TreeInfo* __restrict__ info, const float4* __restrict__ ipos,
           const float4* __restrict__ jpos, const uint4* __restrict__ cell_data,
           const float4* __restrict__ cell_open, const float4* __restrict__ cell_stage,
           const float4* __restrict__ cell_ls,
           const float* __restrict__ group_inv_theta, float eps2, float4* __restrict__ acc,
           int* __restrict__ ring_pool, int ring_cap, unsigned* __restrict__ group_counter,
           unsigned long long* __restrict__ stats, int* __restrict__ status, const int* __restrict__ sys_off,
           int nsys, const int* __restrict__ root_beg, const float4* __restrict__ ipos_lo,
           const float4* __restrict__ jpos_lo, const float4* __restrict__ cell_lo,
           uint2* __restrict__ group_counts, const int* __restrict__ group_list,
           const unsigned* __restrict__ group_list_n, const RelativeArgs rel) {
  constexpr int STRIDE = SPLIT ? 16 : 32;
  constexpr int JSTEP = SPLIT ? 2 : 1;
  __shared__ float4 s_a0[kWalkWarps][64];
  __shared__ float4 s_a1[kWalkWarps][64];
  __shared__ float4 s_a2[kWalkWarps][64];
  constexpr bool DSA = DS && BONSAI_WALK_DS_ASYNC;
  constexpr int DRING = DSA ? 64 : kDirRing;
  __shared__ float4 s_d[kWalkWarps][DRING];
  __shared__ float4 s_dlo[kWalkWarps][DSA ? DRING : 1];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int sub = SPLIT ? (lane & 15) : lane;
  const int half = SPLIT ? (lane >> 4) : 0;
  // two halves of the warp's list buffer: the current level is read from one
  // while the next is written to the other, so the hot footprint stays ~2x the
  // widest level (a sweeping ring would push its dirty lines out to HBM)
  int* lists = ring_pool + (size_t)(blockIdx.x * kWalkWarps + w) * (size_t)ring_cap;
  const int half_cap = ring_cap >> 1;
  // group_list (optional): walk only the listed groups (block time steps)
  const int ngroups = group_list ? (int)*group_list_n : info->ngroups;
  int l1b = info->level_beg[1], l1e = info->level_end[1];
  [[maybe_unused]] const int ncells = info->ncells, npart = info->npart, ngroups_all = info->ngroups;
  const unsigned lt = lanemask_lt();
  unsigned long long sum_app = 0, sum_dir = 0;
  unsigned max_app = 0, max_dir = 0;
  // whether this evaluation is the fixed-angle fallback (no previous
  // accelerations when it starts): its statistics are then flagged as those
  // of a walk without the relative test
  bool start_fallback = false;
  if (rel.acc_valid && blockIdx.x == 0 && threadIdx.x == 0) start_fallback = rel.acc_valid[0] == 0;

  while (true) {
    int g = 0;
    if (lane == 0) g = (int)atomicAdd(group_counter, 1u);
    g = __shfl_sync(kFull, g, 0);
    if (g >= ngroups) break;
    if (group_list) g = __ldg(group_list + g);
    if (!BONSAI_IN_RANGE(g, ngroups_all, 0x401)) continue;
    const int2 gd = groups[g];
    const int pbeg = gd.x, np = gd.y;
    if (!BONSAI_IN_RANGE(np - 1, NI * STRIDE, 0x402) || !BONSAI_IN_RANGE(pbeg + np - 1, npart, 0x403) ||
        !BONSAI_IN_RANGE(pbeg, npart, 0x407))
      continue;
    const float inv_theta_g = PERGROUP ? group_inv_theta[g] : 0.0f;
    // relative accuracy mode: the group's bound on a cell's truncation error
    const float tau_g = (PERGROUP && rel.tau) ? rel.tau[g] : 0.0f;
    // per-group statistics for the next evaluation's features (learned mode):
    // cells near the opening boundary (count; mass of the accepted ones) and
    // the force-weighted quadrupole norm of the accepted cells
    unsigned st_near = 0;
    float st_mnear = 0.f, st_macc = 0.f, st_qn = 0.f, st_wm = 0.f;
    if (ENS) {
      const int sy = sys_of(sys_off, nsys, pbeg);
      l1b = __ldg(root_beg + sy);
      l1e = __ldg(root_beg + sy + 1);
    }
    typedef typename Lanes<NI>::V V;
    constexpr int NV = Lanes<NI>::NV;
    IPart pi[NI];
    float3 R = make_float3(0.f, 0.f, 0.f);
    if (DS) {
      const float4 r0 = ipos[pbeg];
      R = make_float3(r0.x, r0.y, r0.z);
    }
    float mnx = 3.0e38f, mny = 3.0e38f, mnz = 3.0e38f, mxx = -3.0e38f, mxy = -3.0e38f, mxz = -3.0e38f;
#pragma unroll
    for (int k = 0; k < NI; k++) {
      const int ii = pbeg + min(k * STRIDE + sub, np - 1);
      const float4 p = ipos[ii];
      if (DS) {
        const float4 lo = ipos_lo[ii];
        pi[k].x = __fadd_rn(__fsub_rn(p.x, R.x), lo.x);
        pi[k].y = __fadd_rn(__fsub_rn(p.y, R.y), lo.y);
        pi[k].z = __fadd_rn(__fsub_rn(p.z, R.z), lo.z);
      } else {
        pi[k].x = p.x; pi[k].y = p.y; pi[k].z = p.z;
      }
      mnx = fminf(mnx, pi[k].x); mny = fminf(mny, pi[k].y); mnz = fminf(mnz, pi[k].z);
      mxx = fmaxf(mxx, pi[k].x); mxy = fmaxf(mxy, pi[k].y); mxz = fmaxf(mxz, pi[k].z);
    }
    mnx = warp_min_f32(mnx); mny = warp_min_f32(mny); mnz = warp_min_f32(mnz);
    mxx = warp_max_f32(mxx); mxy = warp_max_f32(mxy); mxz = warp_max_f32(mxz);
    const float3 gc = make_float3(__fmul_rn(0.5f, __fadd_rn(mxx, mnx)), __fmul_rn(0.5f, __fadd_rn(mxy, mny)),
                                  __fmul_rn(0.5f, __fadd_rn(mxz, mnz)));
    const float3 gs = make_float3(__fmul_rn(0.5f, __fsub_rn(mxx, mnx)), __fmul_rn(0.5f, __fsub_rn(mxy, mny)),
                                  __fmul_rn(0.5f, __fsub_rn(mxz, mnz)));
    const V veps2 = vdup(eps2, V());
    IVec<V> iv[NV];
    AVec<V> av[NV];
#pragma unroll
    for (int k = 0; k < NI; k++) {
      set_lane(iv[k % NV].nx, k / NV, -pi[k].x);
      set_lane(iv[k % NV].ny, k / NV, -pi[k].y);
      set_lane(iv[k % NV].nz, k / NV, -pi[k].z);
    }
#pragma unroll
    for (int v = 0; v < NV; v++) av[v].x = av[v].y = av[v].z = av[v].w = vdup(0.0f, V());

    int cb = 0;  // base of the current level's half; the next level's is cb ^ half_cap
    int ncur = l1e - l1b, nnext = 0;
    bool overflow = ncur > half_cap;
    for (int j = lane; j < ncur && !overflow; j += 32) lists[j] = l1b + j;
    int a_head = 0, a_cnt = 0, d_head = 0, d_cnt = 0;
    unsigned n_app = 0, n_dir = 0;
    __syncwarp();

    // evaluation of the staged 32-entry batches (ring order): the accepted
    // cells' quadrupoles and the opened leaves' particles
    auto eval_app = [&]() {
      const float4* A0 = &s_a0[w][a_head + half];
      const float4* A1 = &s_a1[w][a_head + half];
      const float4* A2 = &s_a2[w][a_head + half];
      BONSAI_UNROLL_N(BONSAI_WALK_UNROLL)
      for (int j = 0; j < 32; j += JSTEP) {
        const float4 a0 = A0[j], a1 = A1[j], a2 = A2[j];
#pragma unroll
        for (int v = 0; v < NV; v++) quad_acc(av[v], iv[v], a0, a1, a2, veps2);
      }
      a_head = (a_head + 32) & 63;
      a_cnt -= 32;
      n_app += 32;
    };
    // DSA: the entries [d_head + first, + count) become (hi - R) + lo (their
    // copies have landed: called after cp_async_wait_all and __syncwarp)
    [[maybe_unused]] auto combine_dir = [&](int first, int count) {
      for (int k = lane; k < count; k += 32) {
        const int sl = (d_head + first + k) & (DRING - 1);
        float4 pj = s_d[w][sl];
        const float4 lo = s_dlo[w][sl];
        pj.x = __fadd_rn(__fsub_rn(pj.x, R.x), lo.x);
        pj.y = __fadd_rn(__fsub_rn(pj.y, R.y), lo.y);
        pj.z = __fadd_rn(__fsub_rn(pj.z, R.z), lo.z);
        s_d[w][sl] = pj;
      }
      __syncwarp();
    };
    auto eval_dir = [&]() {
      if (DSA) combine_dir(0, 32);
      const float4* D = &s_d[w][d_head + half];
      BONSAI_UNROLL_N(BONSAI_WALK_UNROLL)
      for (int j = 0; j < 32; j += JSTEP) {
        const float4 pj = D[j];
#pragma unroll
        for (int v = 0; v < NV; v++) mono_acc(av[v], iv[v], pj, veps2);
      }
      d_head = (d_head + 32) & (DRING - 1);
      d_cnt -= 32;
      n_dir += 32;
    };

    while (ncur > 0 && !overflow) {
#if BONSAI_WALK_LIST_AHEAD
      // the level's list entries are read one 32-cell block ahead
      int cell_ahead = lane < ncur ? lists[cb + lane] : 0;
#endif
      for (int blk = 0; blk < ncur; blk += 32) {
#if BONSAI_WALK_LIST_AHEAD
        const int cell_here = cell_ahead;
        if (blk + 32 < ncur) cell_ahead = blk + 32 + lane < ncur ? lists[cb + blk + 32 + lane] : 0;
#endif
#if BONSAI_WALK_EVAL_EARLY
        if (a_cnt >= 32 || d_cnt >= 32) {
          cp_async_wait_all();
          __syncwarp();
          if (a_cnt >= 32) eval_app();
          while (d_cnt >= 32) eval_dir();
          __syncwarp();
        }
#endif
        const int li = blk + lane;
        const bool inlist = li < ncur;
#if BONSAI_WALK_LIST_AHEAD
        const int cell = inlist ? cell_here : 0;
#else
        const int cell = inlist ? lists[cb + li] : 0;
#endif
        const bool valid = inlist && BONSAI_IN_RANGE(cell, ncells, 0x404);
        uint4 cd = make_uint4(0u, 0xFFFFFFFFu, 0u, 0u);
        float4 co = make_float4(0.f, 0.f, 0.f, 0.f);
        float4 ls = make_float4(0.f, 0.f, 0.f, 0.f);
        [[maybe_unused]] float a0w = 0.f;  // DS: the staged -0.5 tr I, carried by cell_lo.w
        if (valid) {
          cd = __ldg(cell_data + cell);
          co = __ldg(cell_open + cell);
          if (DS) {
            const float4 cl = __ldg(cell_lo + cell);
            co.x = __fadd_rn(__fsub_rn(co.x, R.x), cl.x);
            co.y = __fadd_rn(__fsub_rn(co.y, R.y), cl.y);
            co.z = __fadd_rn(__fsub_rn(co.z, R.z), cl.z);
            a0w = cl.w;
          }
          if (PERGROUP) ls = __ldg(cell_ls + cell);
        }
#if !BONSAI_WALK_EVAL_EARLY
        // (0) while this block's records are in flight, evaluate the full
        // batches that earlier blocks staged (their copies have had at least
        // one block's traversal to land)
        if (a_cnt >= 32 || d_cnt >= 32) {
          cp_async_wait_all();
          __syncwarp();
          if (a_cnt >= 32) eval_app();
          while (d_cnt >= 32) eval_dir();
          __syncwarp();
        }
#endif
        float mk = 0.f;  // M l^3 (relative test)
        if (PERGROUP && valid) {
          const float op = __fmaf_rn(ls.x, inv_theta_g, ls.y);
          co.w = __fmul_rn(op, op);
          mk = ls.z;
        }
        const bool leaf = cd.y == 0xFFFFFFFFu;
        // the squared box-to-COM distance, shared by the geometric test (the
        // same value open_cell forms), the relative test and the statistics
        const float ds2 = box_dist2(co, gc, gs);
        bool split = valid && (ds2 < fabsf(co.w) || ((int)(cd.w - cd.z) < 3));
        bool near = false;
        if (PERGROUP && rel.stats) {
          // ds within ~20 % of the geometric opening distance
          const float w = fabsf(co.w);
          near = valid && ds2 > 0.7f * w && ds2 < 1.45f * w;
        }
        if (PERGROUP && tau_g > 0.0f && valid && !split) {
          // open_relative on the shared ds2
          const float tds5 = __fmul_rn(tau_g, __fmul_rn(__fmul_rn(ds2, ds2), __fsqrt_rn(ds2)));
          split = mk > tds5;
          // within a factor 2 of the relative bound (ds within ~15 %)
          if (rel.stats) near = near || (mk > 0.5f * tds5 && mk < 2.0f * tds5);
        }
        if (PERGROUP && rel.stats) st_near += __popc(__ballot_sync(kFull, near));

        // (1) children of opened nodes -> next level
        const int nch = (split && !leaf) ? (int)(cd.y >> 29) + 1 : 0;
        const int incl = warp_incl_scan(nch);
        const int tot = __shfl_sync(kFull, incl, 31);
        if (nnext + tot > half_cap) { overflow = true; break; }
        const int first = (int)(cd.y & 0x1FFFFFFFu);
#if BONSAI_WALK_CHILD_LOOP
        // each opened node writes its own (at most 8, contiguous) children at
        // its scan offset: the same entries in the same order as the shuffle
        // expansion, without the dependent shuffle search on the critical path
        {
          int* dst = lists + (cb ^ half_cap) + nnext + (incl - nch);
          for (int k = 0; k < nch; k++) dst[k] = BONSAI_IN_RANGE(first + k, ncells, 0x405) ? first + k : 0;
        }
#else
        for (int base = 0; base < tot; base += 32) {
          const int s = base + lane;
          const int src = find_src(incl, s);
          const int f = __shfl_sync(kFull, first, src);
          const int e = __shfl_sync(kFull, incl - nch, src);
          if (s < tot) lists[(cb ^ half_cap) + nnext + s] = BONSAI_IN_RANGE(f + (s - e), ncells, 0x405) ? f + (s - e) : 0;
        }
#endif
        nnext += tot;

        // (2) accepted cells -> approximate ring, copied by value from the
        // staged records (at most 31 + 32 entries pending)
        const bool app = valid && !split;
        const unsigned bal = __ballot_sync(kFull, app);
        if (app) {
          const int slot = (a_head + a_cnt + __popc(bal & lt)) & 63;
          const float4* src = cell_stage + 3 * (size_t)cell;
          if (PERGROUP && rel.stats) {
            // M from M l^3 and l; tr I from 1.5 tr I (cell_ls)
            const float m = __fdividef(ls.z, __fmul_rn(ls.x, __fmul_rn(ls.x, ls.x)));
            const float inv = __frcp_rn(fmaxf(ds2, 1e-30f));
            st_macc += m;
            st_mnear += near ? m : 0.f;
            st_qn += ls.w * (2.0f / 3.0f) * inv * inv;  // tr I / ds^4 = (M / ds^2) (b / ds)^2
            st_wm += m * inv;                           // the cell's force share M / ds^2
          }
          if (DS)  // the COM relative to the group's reference point
            s_a0[w][slot] = make_float4(co.x, co.y, co.z, a0w);
          else
            cp_async16(&s_a0[w][slot], src);
          cp_async16(&s_a1[w][slot], src + 1);
          cp_async16(&s_a2[w][slot], src + 2);
        }
        a_cnt += __popc(bal);

        // (3) particles of opened leaves -> direct ring
        const int nb = (split && leaf) ? (int)(cd.w - cd.z) : 0;
        const int incl2 = warp_incl_scan(nb);
        const int tot2 = __shfl_sync(kFull, incl2, 31);
        const int pb = (int)cd.z;
        for (int base = 0; base < tot2; base += 32) {
          const int s = base + lane;
          const int src = find_src(incl2, s);
          const int f = __shfl_sync(kFull, pb, src);
          const int e = __shfl_sync(kFull, incl2 - nb, src);
          const int cnt = min(32, tot2 - base);
          if (d_cnt + cnt > DRING) {  // no room: evaluate one batch now
            cp_async_wait_all();
            __syncwarp();
            eval_dir();
            __syncwarp();
          }
          if (lane < cnt) {
            const int jj = BONSAI_IN_RANGE(f + (s - e), npart, 0x406) ? f + (s - e) : 0;
            const int dsl = (d_head + d_cnt + lane) & (DRING - 1);
            float4* dst = &s_d[w][dsl];
            if (DSA) {
              cp_async16(dst, jpos + jj);
              cp_async16(&s_dlo[w][dsl], jpos_lo + jj);
            } else if (DS) {
              float4 pj = __ldg(jpos + jj);
              const float4 lo = __ldg(jpos_lo + jj);
              pj.x = __fadd_rn(__fsub_rn(pj.x, R.x), lo.x);
              pj.y = __fadd_rn(__fsub_rn(pj.y, R.y), lo.y);
              pj.z = __fadd_rn(__fsub_rn(pj.z, R.z), lo.z);
              *dst = pj;
            } else {
              cp_async16(dst, jpos + jj);
            }
          }
          d_cnt += cnt;
        }
      }
      cb ^= half_cap;
      ncur = nnext;
      nnext = 0;
      __syncwarp();
    }

    // the remaining batches, full and partial
    cp_async_wait_all();
    __syncwarp();
    for (int j = half; j < a_cnt; j += JSTEP) {
      const int sl = (a_head + j) & 63;
      const float4 a0 = s_a0[w][sl], a1 = s_a1[w][sl], a2 = s_a2[w][sl];
#pragma unroll
      for (int v = 0; v < NV; v++) quad_acc(av[v], iv[v], a0, a1, a2, veps2);
    }
    n_app += a_cnt;
    if (DSA) combine_dir(0, d_cnt);
    for (int j = half; j < d_cnt; j += JSTEP) {
      const float4 pj = s_d[w][(d_head + j) & (DRING - 1)];
#pragma unroll
      for (int v = 0; v < NV; v++) mono_acc(av[v], iv[v], pj, veps2);
    }
    n_dir += d_cnt;
    __syncwarp();
    float4 ai[NI];
#pragma unroll
    for (int k = 0; k < NI; k++)
      ai[k] = make_float4(get_lane(av[k % NV].x, k / NV), get_lane(av[k % NV].y, k / NV),
                          get_lane(av[k % NV].z, k / NV), -get_lane(av[k % NV].w, k / NV));
    if (SPLIT) {
#pragma unroll
      for (int k = 0; k < NI; k++) {
        ai[k].x += __shfl_xor_sync(kFull, ai[k].x, 16);
        ai[k].y += __shfl_xor_sync(kFull, ai[k].y, 16);
        ai[k].z += __shfl_xor_sync(kFull, ai[k].z, 16);
        ai[k].w += __shfl_xor_sync(kFull, ai[k].w, 16);
      }
    }

    if (overflow) {
      if (lane == 0) set_status(status, kStatusWalkStack);
#pragma unroll
      for (int k = 0; k < NI; k++) ai[k] = make_float4(__int_as_float(0x7fc00000), 0.f, 0.f, 0.f);
    }
    if (half == 0) {
#pragma unroll
      for (int k = 0; k < NI; k++) {
        const int idx = k * STRIDE + sub;
        if (idx < np) acc[pbeg + idx] = ai[k];
      }
    }
    // per-group (approximate, direct) interaction counts, for the per-group angle variant
    if (PERGROUP && group_counts && lane == 0) group_counts[g] = make_uint2(n_app, n_dir);
    if (PERGROUP && rel.stats) {
#pragma unroll
      for (int o = 16; o; o >>= 1) {
        st_mnear += __shfl_xor_sync(kFull, st_mnear, o);
        st_macc += __shfl_xor_sync(kFull, st_macc, o);
        st_qn += __shfl_xor_sync(kFull, st_qn, o);
        st_wm += __shfl_xor_sync(kFull, st_wm, o);
      }
      if (lane == 0)
        rel.stats[g] = make_float4((float)st_near, st_macc > 0.f ? st_mnear / st_macc : 0.f,
                                   st_wm > 0.f ? st_qn / st_wm : 0.f, (float)n_app);
      for (int i = lane; i < np; i += 32) rel.part_gid[pbeg + i] = g;
    }
    sum_app += (unsigned long long)n_app * (unsigned long long)np;
    sum_dir += (unsigned long long)n_dir * (unsigned long long)np;
    max_app = max(max_app, n_app);
    max_dir = max(max_dir, n_dir);
  }
  // the accelerations just written are the previous ones of the next evaluation
  if (rel.acc_valid && blockIdx.x == 0 && threadIdx.x == 0) {
    rel.acc_valid[0] = 1;
    rel.acc_valid[1] = rel.stats == nullptr ? 0 : (start_fallback ? 1 : 2);
  }
  if (lane == 0) {
    atomicAdd(stats + 0, sum_app);
    atomicAdd(stats + 1, sum_dir);
    atomicMax(stats + 2, (unsigned long long)max_app);
    atomicMax(stats + 3, (unsigned long long)max_dir);
  }
}

// variants: 0..2 half-warp split with NI = 1, 2, 4 (nCrit <= 16, 32, 64);
// 3..5 full warp with NI = 1, 2, 4 (nCrit <= 32, 64, 128).  layout 0: split
// where nCrit <= 64 (the default); 1: full warp.
int walk_variant(int ncrit, int layout) {
#if BONSAI_WALK_SPLIT
  if (ncrit <= 64 && layout != 1) return ncrit <= 16 ? 0 : (ncrit <= 32 ? 1 : 2);
#endif
  return ncrit <= 32 ? 3 : (ncrit <= 64 ? 4 : 5);
}

template <class K>
static int occupancy(K kernel) {
  int nb = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, kernel, kWalkThreads, 0) != cudaSuccess) nb = 1;
  return nb;
}

// blocks per SM that every instantiation of the variant reaches (the level
// lists are sized for the largest grid)
template <int NI, bool SPLIT>
static int occupancy_of() {
  int nb = occupancy(k_walk<NI, SPLIT, false, false, false>);
  nb = std::min(nb, occupancy(k_walk<NI, SPLIT, true, false, false>));
  nb = std::min(nb, occupancy(k_walk<NI, SPLIT, false, true, false>));
  nb = std::min(nb, occupancy(k_walk<NI, SPLIT, true, true, false>));
  nb = std::min(nb, occupancy(k_walk<NI, SPLIT, false, true, true>));
  nb = std::min(nb, occupancy(k_walk<NI, SPLIT, true, true, true>));
  nb = std::min(nb, occupancy(k_walk<NI, SPLIT, false, false, true>));
  nb = std::min(nb, occupancy(k_walk<NI, SPLIT, true, false, true>));
  return nb < 1 ? 1 : nb;
}

int walk_blocks_per_sm(int variant) {
  switch (variant) {
#if BONSAI_WALK_SPLIT
    case 0: return occupancy_of<1, true>();
    case 1: return occupancy_of<2, true>();
    case 2: return occupancy_of<4, true>();
#endif
    case 3: return occupancy_of<1, false>();
    case 4: return occupancy_of<2, false>();
    default: return occupancy_of<4, false>();
  }
}

void launch_walk(int variant, int nblocks, const int2* groups, const TreeInfo* info, const float4* ipos,
                 const float4* jpos, const uint4* cell_data, const float4* cell_open, const float4* cell_stage,
                 const float4* cell_ls, const float* group_inv_theta, float eps2,
                 float4* acc, int* ring_pool, int ring_cap, unsigned* group_counter, unsigned long long* stats,
                 int* status, const int* sys_off, int nsys, const int* root_beg, const float4* ipos_lo,
                 const float4* jpos_lo, const float4* cell_lo, uint2* group_counts, const int* group_list,
                 const unsigned* group_list_n, const RelativeArgs& rel, cudaStream_t s) {
#define BONSAI_WALK_ARGS                                                                                          \
  groups, info, ipos, jpos, cell_data, cell_open, cell_stage, cell_ls, group_inv_theta, eps2, acc, ring_pool, \
      ring_cap, group_counter, stats, status, sys_off, nsys, root_beg, ipos_lo, jpos_lo, cell_lo, group_counts,  \
      group_list, group_list_n, rel
#define BONSAI_WALK(NI, SP)                                                                \
  do {                                                                                     \
    if (nsys > 1 && ipos_lo && group_inv_theta)                                            \
      k_walk<NI, SP, true, true, true><<<nblocks, kWalkThreads, 0, s>>>(BONSAI_WALK_ARGS);   \
    else if (nsys > 1 && ipos_lo)                                                          \
      k_walk<NI, SP, false, true, true><<<nblocks, kWalkThreads, 0, s>>>(BONSAI_WALK_ARGS);  \
    else if (nsys > 1 && group_inv_theta)                                                  \
      k_walk<NI, SP, true, true, false><<<nblocks, kWalkThreads, 0, s>>>(BONSAI_WALK_ARGS);  \
    else if (nsys > 1)                                                                     \
      k_walk<NI, SP, false, true, false><<<nblocks, kWalkThreads, 0, s>>>(BONSAI_WALK_ARGS); \
    else if (ipos_lo && group_inv_theta)                                                   \
      k_walk<NI, SP, true, false, true><<<nblocks, kWalkThreads, 0, s>>>(BONSAI_WALK_ARGS);  \
    else if (ipos_lo)                                                                      \
      k_walk<NI, SP, false, false, true><<<nblocks, kWalkThreads, 0, s>>>(BONSAI_WALK_ARGS); \
    else if (group_inv_theta)                                                              \
      k_walk<NI, SP, true, false, false><<<nblocks, kWalkThreads, 0, s>>>(BONSAI_WALK_ARGS); \
    else                                                                                   \
      k_walk<NI, SP, false, false, false><<<nblocks, kWalkThreads, 0, s>>>(BONSAI_WALK_ARGS); \
  } while (0)
  switch (variant) {
#if BONSAI_WALK_SPLIT
    case 0: BONSAI_WALK(1, true); break;
    case 1: BONSAI_WALK(2, true); break;
    case 2: BONSAI_WALK(4, true); break;
#endif
    case 3: BONSAI_WALK(1, false); break;
    case 4: BONSAI_WALK(2, false); break;
    default: BONSAI_WALK(4, false); break;
  }
#undef BONSAI_WALK
#undef BONSAI_WALK_ARGS
}

BONSAI_BOUNDS_ACCESSOR(bounds_word_walk)

}  // namespace bonsai
