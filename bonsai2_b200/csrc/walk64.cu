// walk64.cu -- the FP64 walk: a checker with the float walk's interaction
// lists and FP64 arithmetic.
//
// The float walk (walk.cu) evaluates every interaction in FP32.  This kernel
// walks the same tree for the same groups and takes the same opening
// decisions (the float test of walk_common.cuh on the same float operands,
// group-relative in double-single mode, per-group angles likewise), so the
// interaction lists are the float walk's exactly; each interaction is then
// evaluated in FP64 from the FP64 cell records (M, COM, mass-weighted second
// moments of multipoles.cu) and the exact particle positions (hi + lo in
// double-single mode), with the reference's formulas (computeForces.cu:58-78
// monopole, :83-128 quadrupole; Q per unit mass there is I/M here).  The
// difference to the float walk is then rounding alone, and the difference to
// the FP64 direct sum is the multipole truncation alone.  A checker: one warp
// per group, interactions evaluated as they are found, no staging.
#include "common.cuh"
#include "kernels.cuh"
#include "walk_common.cuh"

namespace bonsai {

constexpr int kW64Threads = 256;
constexpr int kW64Warps = kW64Threads / 32;
constexpr int kW64NI = 4;  // 128 particle slots per warp (nCrit <= 128)

__device__ __forceinline__ void quad64(double4& a, const double x, const double y, const double z, const MpRec& c,
                                       double eps2) {
  const double dx = x - c.cx, dy = y - c.cy, dz = z - c.cz;
  const double r2 = dx * dx + dy * dy + dz * dz + eps2;
  const double rinv = 1.0 / sqrt(r2);
  const double r2i = rinv * rinv;
  const double r3i = rinv * r2i, r5i = r3i * r2i, r7i = r5i * r2i;
  const double tr = c.ixx + c.iyy + c.izz;
  const double qx = c.ixx * dx + c.ixy * dy + c.ixz * dz;
  const double qy = c.ixy * dx + c.iyy * dy + c.iyz * dz;
  const double qz = c.ixz * dx + c.iyz * dy + c.izz * dz;
  const double qrr = dx * qx + dy * qy + dz * qz;
  a.w -= c.m * rinv + 0.5 * (-tr * r3i + 3.0 * qrr * r5i);
  const double cf = -c.m * r3i + 0.5 * (3.0 * tr * r5i - 15.0 * qrr * r7i);
  a.x += cf * dx + 3.0 * qx * r5i;
  a.y += cf * dy + 3.0 * qy * r5i;
  a.z += cf * dz + 3.0 * qz * r5i;
}

__device__ __forceinline__ void mono64(double4& a, const double x, const double y, const double z, const double jx,
                                       const double jy, const double jz, const double m, double eps2) {
  const double dx = jx - x, dy = jy - y, dz = jz - z;
  const double r2 = dx * dx + dy * dy + dz * dz + eps2;
  const double rinv = 1.0 / sqrt(r2);
  const double mr = m * rinv;
  const double mr3 = mr * rinv * rinv;
  a.w -= mr;
  a.x += mr3 * dx;
  a.y += mr3 * dy;
  a.z += mr3 * dz;
}

template <bool DS, bool PERGROUP>
__global__ void __launch_bounds__(kW64Threads) k_walk64(
    const int2* __restrict__ groups, const TreeInfo* __restrict__ info, const float4* __restrict__ ipos,
    const float4* __restrict__ ipos_lo, const float4* __restrict__ jpos, const float4* __restrict__ jpos_lo,
    const uint4* __restrict__ cell_data, const float4* __restrict__ cell_open, const float4* __restrict__ cell_lo,
    const float4* __restrict__ cell_ls, const float* __restrict__ group_inv_theta,
    const float* __restrict__ group_tau, const MpRec* __restrict__ rec,
    double eps2, double4* __restrict__ acc, int* __restrict__ ring_pool, int ring_cap,
    unsigned* __restrict__ group_counter, unsigned long long* __restrict__ stats, int* __restrict__ status,
    const int* __restrict__ sys_off, int nsys, const int* __restrict__ root_beg) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  int* lists = ring_pool + (size_t)(blockIdx.x * kW64Warps + w) * (size_t)ring_cap;
  const int half_cap = ring_cap >> 1;
  const int ngroups = info->ngroups;
  int l1b = info->level_beg[1], l1e = info->level_end[1];
  [[maybe_unused]] const int ncells = info->ncells, npart = info->npart;
  unsigned long long sum_app = 0, sum_dir = 0;
  unsigned max_app = 0, max_dir = 0;
  while (true) {
    int g = 0;
    if (lane == 0) g = (int)atomicAdd(group_counter, 1u);
    g = __shfl_sync(kFull, g, 0);
    if (g >= ngroups) break;
    const int2 gd = groups[g];
    const int pbeg = gd.x, np = gd.y;
    if (!BONSAI_IN_RANGE(np - 1, kW64NI * 32, 0x501) || !BONSAI_IN_RANGE(pbeg + np - 1, npart, 0x502) ||
        !BONSAI_IN_RANGE(pbeg, npart, 0x503))
      continue;
    const float inv_theta_g = PERGROUP ? group_inv_theta[g] : 0.0f;
    const float tau_g = (PERGROUP && group_tau) ? group_tau[g] : 0.0f;
    if (nsys > 1) {  // an ensemble: the group's own system's level-1 cells
      const int sy = sys_of(sys_off, nsys, pbeg);
      l1b = __ldg(root_beg + sy);
      l1e = __ldg(root_beg + sy + 1);
    }
    float3 R = make_float3(0.f, 0.f, 0.f);
    if (DS) {
      const float4 r0 = ipos[pbeg];
      R = make_float3(r0.x, r0.y, r0.z);
    }
    double xi[kW64NI], yi[kW64NI], zi[kW64NI];
    double4 ai[kW64NI];
    float mnx = 3.0e38f, mny = 3.0e38f, mnz = 3.0e38f, mxx = -3.0e38f, mxy = -3.0e38f, mxz = -3.0e38f;
#pragma unroll
    for (int k = 0; k < kW64NI; k++) {
      const int ii = pbeg + min(k * 32 + lane, np - 1);
      const float4 p = ipos[ii];
      float fx = p.x, fy = p.y, fz = p.z;
      xi[k] = p.x; yi[k] = p.y; zi[k] = p.z;
      if (DS) {
        const float4 lo = ipos_lo[ii];
        fx = __fadd_rn(__fsub_rn(p.x, R.x), lo.x);
        fy = __fadd_rn(__fsub_rn(p.y, R.y), lo.y);
        fz = __fadd_rn(__fsub_rn(p.z, R.z), lo.z);
        xi[k] += lo.x; yi[k] += lo.y; zi[k] += lo.z;
      }
      ai[k] = make_double4(0.0, 0.0, 0.0, 0.0);
      mnx = fminf(mnx, fx); mny = fminf(mny, fy); mnz = fminf(mnz, fz);
      mxx = fmaxf(mxx, fx); mxy = fmaxf(mxy, fy); mxz = fmaxf(mxz, fz);
    }
    mnx = warp_min_f32(mnx); mny = warp_min_f32(mny); mnz = warp_min_f32(mnz);
    mxx = warp_max_f32(mxx); mxy = warp_max_f32(mxy); mxz = warp_max_f32(mxz);
    const float3 gc = make_float3(__fmul_rn(0.5f, __fadd_rn(mxx, mnx)), __fmul_rn(0.5f, __fadd_rn(mxy, mny)),
                                  __fmul_rn(0.5f, __fadd_rn(mxz, mnz)));
    const float3 gs = make_float3(__fmul_rn(0.5f, __fsub_rn(mxx, mnx)), __fmul_rn(0.5f, __fsub_rn(mxy, mny)),
                                  __fmul_rn(0.5f, __fsub_rn(mxz, mnz)));
    int cb = 0;
    int ncur = l1e - l1b, nnext = 0;
    bool overflow = ncur > half_cap;
    for (int j = lane; j < ncur && !overflow; j += 32) lists[j] = l1b + j;
    unsigned n_app = 0, n_dir = 0;
    __syncwarp();
    while (ncur > 0 && !overflow) {
      for (int blk = 0; blk < ncur; blk += 32) {
        const int li = blk + lane;
        const bool inlist = li < ncur;
        const int cell = inlist ? lists[cb + li] : 0;
        const bool valid = inlist && BONSAI_IN_RANGE(cell, ncells, 0x504);
        uint4 cd = make_uint4(0u, 0xFFFFFFFFu, 0u, 0u);
        float4 co = make_float4(0.f, 0.f, 0.f, 0.f);
        if (valid) {
          cd = __ldg(cell_data + cell);
          co = __ldg(cell_open + cell);
          if (DS) {
            const float4 cl = __ldg(cell_lo + cell);
            co.x = __fadd_rn(__fsub_rn(co.x, R.x), cl.x);
            co.y = __fadd_rn(__fsub_rn(co.y, R.y), cl.y);
            co.z = __fadd_rn(__fsub_rn(co.z, R.z), cl.z);
          }
          if (PERGROUP) {
            const float4 ls = __ldg(cell_ls + cell);
            const float op = __fmaf_rn(ls.x, inv_theta_g, ls.y);
            co.w = __fmul_rn(op, op);
          }
        }
        const bool leaf = cd.y == 0xFFFFFFFFu;
        bool split = valid && (open_cell(co, gc, gs) || ((int)(cd.w - cd.z) < 3));
        // the float walk's relative test on the same float operands
        if (PERGROUP && tau_g > 0.0f && valid && !split)
          split = open_relative(co, gc, gs, __ldg(&cell_ls[cell].z), tau_g);
        // children of opened nodes -> next level
        const int nch = (split && !leaf) ? (int)(cd.y >> 29) + 1 : 0;
        const int incl = warp_incl_scan(nch);
        const int tot = __shfl_sync(kFull, incl, 31);
        if (nnext + tot > half_cap) { overflow = true; break; }
        const int first = (int)(cd.y & 0x1FFFFFFFu);
        for (int base = 0; base < tot; base += 32) {
          const int s = base + lane;
          const int src = find_src(incl, s);
          const int f = __shfl_sync(kFull, first, src);
          const int e = __shfl_sync(kFull, incl - nch, src);
          if (s < tot) lists[(cb ^ half_cap) + nnext + s] = BONSAI_IN_RANGE(f + (s - e), ncells, 0x505) ? f + (s - e) : 0;
        }
        nnext += tot;
        // accepted cells: quadrupoles in FP64 from the cell records
        unsigned acc_mask = __ballot_sync(kFull, valid && !split);
        n_app += __popc(acc_mask);
        while (acc_mask) {
          const int b = __ffs(acc_mask) - 1;
          acc_mask &= acc_mask - 1;
          const int c = __shfl_sync(kFull, cell, b);
          const MpRec r = rec[c];
#pragma unroll
          for (int k = 0; k < kW64NI; k++) quad64(ai[k], xi[k], yi[k], zi[k], r, eps2);
        }
        // opened leaves: their particles directly, in FP64
        unsigned leaf_mask = __ballot_sync(kFull, split && leaf);
        while (leaf_mask) {
          const int b = __ffs(leaf_mask) - 1;
          leaf_mask &= leaf_mask - 1;
          int pb = (int)__shfl_sync(kFull, cd.z, b), pe = (int)__shfl_sync(kFull, cd.w, b);
          if (!BONSAI_IN_RANGE(pe - 1, npart, 0x506) || !BONSAI_IN_RANGE(pb, pe, 0x507)) pb = pe = 0;
          n_dir += (unsigned)(pe - pb);
          for (int j = pb; j < pe; j++) {
            const float4 q = __ldg(jpos + j);
            double jx = q.x, jy = q.y, jz = q.z;
            if (DS) {
              const float4 l = __ldg(jpos_lo + j);
              jx += l.x; jy += l.y; jz += l.z;
            }
#pragma unroll
            for (int k = 0; k < kW64NI; k++) mono64(ai[k], xi[k], yi[k], zi[k], jx, jy, jz, q.w, eps2);
          }
        }
      }
      cb ^= half_cap;
      ncur = nnext;
      nnext = 0;
      __syncwarp();
    }
    if (overflow) {
      if (lane == 0) set_status(status, kStatusWalkStack);
#pragma unroll
      for (int k = 0; k < kW64NI; k++) ai[k] = make_double4(__longlong_as_double(0x7ff8000000000000ll), 0.0, 0.0, 0.0);
    }
#pragma unroll
    for (int k = 0; k < kW64NI; k++) {
      const int idx = k * 32 + lane;
      if (idx < np) acc[pbeg + idx] = ai[k];
    }
    sum_app += (unsigned long long)n_app * (unsigned long long)np;
    sum_dir += (unsigned long long)n_dir * (unsigned long long)np;
    max_app = max(max_app, n_app);
    max_dir = max(max_dir, n_dir);
  }
  if (lane == 0) {
    atomicAdd(stats + 0, sum_app);
    atomicAdd(stats + 1, sum_dir);
    atomicMax(stats + 2, (unsigned long long)max_app);
    atomicMax(stats + 3, (unsigned long long)max_dir);
  }
}

__global__ void __launch_bounds__(256) k_scatter_d4(const int* __restrict__ id, int n, const double4* __restrict__ in,
                                                    double4* __restrict__ out) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) out[id[k]] = in[k];
}

void launch_walk64(int nblocks, const int2* groups, const TreeInfo* info, const float4* ipos, const float4* ipos_lo,
                   const float4* jpos, const float4* jpos_lo, const uint4* cell_data, const float4* cell_open,
                   const float4* cell_lo, const float4* cell_ls, const float* group_inv_theta,
                   const float* group_tau, const MpRec* rec, double eps2, double4* acc, int* ring_pool, int ring_cap, unsigned* group_counter,
                   unsigned long long* stats, int* status, const int* sys_off, int nsys, const int* root_beg,
                   cudaStream_t s) {
#define BONSAI_W64(DS, PG)                                                                                         \
  k_walk64<DS, PG><<<nblocks, kW64Threads, 0, s>>>(groups, info, ipos, ipos_lo, jpos, jpos_lo, cell_data,          \
                                                   cell_open, cell_lo, cell_ls, group_inv_theta, group_tau, rec,  \
                                                   eps2, acc,                                                     \
                                                   ring_pool, ring_cap, group_counter, stats, status, sys_off,    \
                                                   nsys, root_beg)
  if (ipos_lo) {
    if (group_inv_theta) BONSAI_W64(true, true); else BONSAI_W64(true, false);
  } else {
    if (group_inv_theta) BONSAI_W64(false, true); else BONSAI_W64(false, false);
  }
#undef BONSAI_W64
}

void launch_scatter_d4(const int* id, int n, const double4* in, double4* out, int nblocks, cudaStream_t s) {
  k_scatter_d4<<<nblocks, 256, 0, s>>>(id, n, in, out);
}

BONSAI_BOUNDS_ACCESSOR(bounds_word_walk64)

}  // namespace bonsai
