// multipoles.cu -- monopole, quadrupole and opening size of every cell in one
// launch, bottom up.
//
// The reference (computeCellMultipoles, computeMultipoles.cu:81-190) gives a
// warp to every cell and rescans all of that cell's particles, O(N * depth)
// particle reads, with float products summed in double.  Here each leaf is
// reduced from its own particles (one thread per leaf, FP64, two passes:
// centre of mass, then central moments), and every node is combined from its
// children with the parallel-axis theorem by the child that finishes last
// (an arrival counter per cell; no thread waits on another).
// Each particle is read once.  The quantities match the reference's definitions:
//   M, COM; Q = second moment about the COM per unit mass (:148-158);
//   particle bounding box -> l = max(2 max h, 1e-6), s = |cvec - COM|,
//   cellOp = l/theta + s, stored squared (:168-177).
// cell_ls = (l, s) lets a walk with per-group opening angles form
// (l/theta_g + s)^2.  Stored for the walk (mass-weighted, pre-scaled so the
// force kernel needs fewer operations):  cell_q0 = (M, 3Ixx, 3Iyy, 3Izz),
// cell_q1 = (3Ixy, 3Ixz, 3Iyz, 1.5 tr I), with I = M Q.
// Double-single positions (jlo != nullptr): particles enter the FP64 sums as
// hi + lo, and the COM is stored as hi (cell_open) plus lo (cell_lo).
#include "common.cuh"
#include "kernels.cuh"

namespace bonsai {

__device__ __forceinline__ void store_cell(int c, const MpRec& r, float inv_theta, MpRec* __restrict__ rec,
                                           float4* __restrict__ cell_open, float4* __restrict__ cell_q0,
                                           float4* __restrict__ cell_q1, float2* __restrict__ cell_ls,
                                           float4* __restrict__ cell_lo) {
  rec[c] = r;
  const float cx = (float)r.cx, cy = (float)r.cy, cz = (float)r.cz;
  if (cell_lo)
    cell_lo[c] = make_float4((float)(r.cx - (double)cx), (float)(r.cy - (double)cy), (float)(r.cz - (double)cz), 0.f);
  float s, l;
  if (cell_lo) {
    // double-single: extents and centre offsets from the exact box and COM
    double v[3], hm = 0.0, d2 = 0.0;
    const double com[3] = {r.cx, r.cy, r.cz};
    for (int k = 0; k < 3; k++) {
      v[k] = 0.5 * (r.bmax[k] + r.bmin[k]) - com[k];
      hm = fmax(hm, 0.5 * (r.bmax[k] - r.bmin[k]));
      d2 += v[k] * v[k];
    }
    s = (float)sqrt(d2);
    l = fmaxf((float)(2.0 * hm), 1.0e-6f);
  } else {
    const float b0[3] = {(float)r.bmin[0], (float)r.bmin[1], (float)r.bmin[2]};
    const float b1[3] = {(float)r.bmax[0], (float)r.bmax[1], (float)r.bmax[2]};
    const float vx = __fmul_rn(__fadd_rn(b1[0], b0[0]), 0.5f);
    const float vy = __fmul_rn(__fadd_rn(b1[1], b0[1]), 0.5f);
    const float vz = __fmul_rn(__fadd_rn(b1[2], b0[2]), 0.5f);
    const float hx = __fmul_rn(__fsub_rn(b1[0], b0[0]), 0.5f);
    const float hy = __fmul_rn(__fsub_rn(b1[1], b0[1]), 0.5f);
    const float hz = __fmul_rn(__fsub_rn(b1[2], b0[2]), 0.5f);
    const float dx = __fsub_rn(vx, cx), dy = __fsub_rn(vy, cy), dz = __fsub_rn(vz, cz);
    s = __fsqrt_rn(__fmaf_rn(dz, dz, __fmaf_rn(dy, dy, __fmul_rn(dx, dx))));
    l = fmaxf(__fmul_rn(2.0f, fmaxf(hx, fmaxf(hy, hz))), 1.0e-6f);
  }
  const float op = __fmaf_rn(l, inv_theta, s);
  cell_open[c] = make_float4(cx, cy, cz, __fmul_rn(op, op));
  cell_ls[c] = make_float2(l, s);  // per-group opening angles recompute (l/theta_g + s)^2
  const double tr = r.ixx + r.iyy + r.izz;
  cell_q0[c] = make_float4((float)r.m, (float)(3.0 * r.ixx), (float)(3.0 * r.iyy), (float)(3.0 * r.izz));
  cell_q1[c] = make_float4((float)(3.0 * r.ixy), (float)(3.0 * r.ixz), (float)(3.0 * r.iyz), (float)(1.5 * tr));
}

// Arrival on a parent's counter: a fence publishes this child's record, a
// relaxed atomic counts it, and only the last arriver fences again before it
// reads its siblings' records (through L2).  (An acquire-release atomic per
// arrival was measured 16x slower here: a GPU-scope acquire invalidates the
// SM's L1, which the leaf loads of every other warp depend on.)
__device__ __forceinline__ bool arrive_last(int* p, int nch) {
  __threadfence();
  if (atomicAdd(p, 1) != nch - 1) return false;
  __threadfence();
  return true;
}

__device__ __forceinline__ void particle_ds(const float4* __restrict__ jpos, const float4* __restrict__ jlo, int i,
                                            double& x, double& y, double& z, double& w) {
  const float4 p = __ldg(jpos + i);
  x = p.x; y = p.y; z = p.z; w = p.w;
  if (jlo) {
    const float4 l = __ldg(jlo + i);
    x += l.x; y += l.y; z += l.z;
  }
}

// Combines parents bottom-up while this thread is the last child to arrive.
__device__ void climb(int c, const uint4* __restrict__ cell_data, const int* __restrict__ cell_parent,
                      float inv_theta, MpRec* __restrict__ rec, float4* __restrict__ cell_open,
                      float4* __restrict__ cell_q0, float4* __restrict__ cell_q1, float2* __restrict__ cell_ls,
                      int* __restrict__ mp_count, float4* __restrict__ cell_lo) {
  while (true) {
    const int p = cell_parent[c];
    if (p < 0) break;
    const unsigned y = cell_data[p].y;
    const int first = (int)(y & 0x1FFFFFFFu), nch = (int)(y >> 29) + 1;
    if (!arrive_last(mp_count + p, nch)) break;
    double M = 0, X = 0, Y = 0, Z = 0;
    double bmn[3] = {3.0e38, 3.0e38, 3.0e38}, bmx[3] = {-3.0e38, -3.0e38, -3.0e38};
    for (int k = 0; k < nch; k++) {
      const MpRec* ck = rec + first + k;
      const double mk = __ldcg(&ck->m);
      M += mk;
      X += mk * __ldcg(&ck->cx); Y += mk * __ldcg(&ck->cy); Z += mk * __ldcg(&ck->cz);
      for (int a = 0; a < 3; a++) {
        bmn[a] = fmin(bmn[a], __ldcg(&ck->bmin[a]));
        bmx[a] = fmax(bmx[a], __ldcg(&ck->bmax[a]));
      }
    }
    MpRec P;
    if (M > 0.0) { P.cx = X / M; P.cy = Y / M; P.cz = Z / M; }
    else { P.cx = 0.5 * (bmn[0] + bmx[0]); P.cy = 0.5 * (bmn[1] + bmx[1]); P.cz = 0.5 * (bmn[2] + bmx[2]); }
    double I[6] = {0, 0, 0, 0, 0, 0};
    for (int k = 0; k < nch; k++) {
      const MpRec* ck = rec + first + k;
      const double mk = __ldcg(&ck->m);
      const double dx = __ldcg(&ck->cx) - P.cx, dy = __ldcg(&ck->cy) - P.cy, dz = __ldcg(&ck->cz) - P.cz;
      I[0] += __ldcg(&ck->ixx) + mk * dx * dx;
      I[1] += __ldcg(&ck->iyy) + mk * dy * dy;
      I[2] += __ldcg(&ck->izz) + mk * dz * dz;
      I[3] += __ldcg(&ck->ixy) + mk * dx * dy;
      I[4] += __ldcg(&ck->ixz) + mk * dx * dz;
      I[5] += __ldcg(&ck->iyz) + mk * dy * dz;
    }
    P.m = M;
    P.ixx = I[0]; P.iyy = I[1]; P.izz = I[2]; P.ixy = I[3]; P.ixz = I[4]; P.iyz = I[5];
    for (int a = 0; a < 3; a++) { P.bmin[a] = bmn[a]; P.bmax[a] = bmx[a]; }
    store_cell(p, P, inv_theta, rec, cell_open, cell_q0, cell_q1, cell_ls, cell_lo);
    c = p;
  }
}

// One thread per leaf: two passes over the leaf's particles (COM, then
// central moments), then the bottom-up climb.  (Half-warp-cooperative leaves
// with shuffle reductions were measured 16x slower on the B200.)
__global__ void __launch_bounds__(256) k_multipoles(const int* __restrict__ leaf_list, const TreeInfo* __restrict__ info,
                                                    const uint4* __restrict__ cell_data,
                                                    const int* __restrict__ cell_parent,
                                                    const float4* __restrict__ jpos, float inv_theta,
                                                    MpRec* __restrict__ rec, float4* __restrict__ cell_open,
                                                    float4* __restrict__ cell_q0, float4* __restrict__ cell_q1,
                                                    float2* __restrict__ cell_ls, int* __restrict__ mp_count,
                                                    int cell_cap, const float4* __restrict__ jlo,
                                                    float4* __restrict__ cell_lo) {
  const int nleaves = info->nleaves;
  if (info->ncells > cell_cap) return;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < nleaves; t += gridDim.x * blockDim.x) {
    const int c = leaf_list[t];
    const uint4 cd = cell_data[c];
    const int b = (int)cd.z, e = (int)cd.w;
    MpRec r;
    double m = 0, sx = 0, sy = 0, sz = 0;
    double mn[3] = {3.0e38, 3.0e38, 3.0e38}, mx[3] = {-3.0e38, -3.0e38, -3.0e38};
    for (int i = b; i < e; i++) {
      double px, py, pz, w;
      particle_ds(jpos, jlo, i, px, py, pz, w);
      m += w;
      sx += w * px; sy += w * py; sz += w * pz;
      mn[0] = fmin(mn[0], px); mn[1] = fmin(mn[1], py); mn[2] = fmin(mn[2], pz);
      mx[0] = fmax(mx[0], px); mx[1] = fmax(mx[1], py); mx[2] = fmax(mx[2], pz);
    }
    if (m > 0.0) { r.cx = sx / m; r.cy = sy / m; r.cz = sz / m; }
    else { r.cx = 0.5 * (mn[0] + mx[0]); r.cy = 0.5 * (mn[1] + mx[1]); r.cz = 0.5 * (mn[2] + mx[2]); }
    double q[6] = {0, 0, 0, 0, 0, 0};
    for (int i = b; i < e; i++) {
      double px, py, pz, w;
      particle_ds(jpos, jlo, i, px, py, pz, w);
      const double dx = px - r.cx, dy = py - r.cy, dz = pz - r.cz;
      q[0] += w * dx * dx; q[1] += w * dy * dy; q[2] += w * dz * dz;
      q[3] += w * dx * dy; q[4] += w * dx * dz; q[5] += w * dy * dz;
    }
    r.m = m;
    r.ixx = q[0]; r.iyy = q[1]; r.izz = q[2]; r.ixy = q[3]; r.ixz = q[4]; r.iyz = q[5];
    for (int k = 0; k < 3; k++) { r.bmin[k] = mn[k]; r.bmax[k] = mx[k]; }
    store_cell(c, r, inv_theta, rec, cell_open, cell_q0, cell_q1, cell_ls, cell_lo);
    climb(c, cell_data, cell_parent, inv_theta, rec, cell_open, cell_q0, cell_q1, cell_ls, mp_count, cell_lo);
  }
}

// Reference-layout view of the multipoles (debug/parity getter):
// size = (COM, cellOp^2), mono = (COM, M), quad0 = (xx,yy,zz,xy), quad1 = (xz,yz)
// with Q per unit mass (computeMultipoles.cu:180-188).
__global__ void k_multipoles_ref_layout(const TreeInfo* __restrict__ info, const float4* __restrict__ cell_open,
                                        const MpRec* __restrict__ rec, float4* __restrict__ size,
                                        float4* __restrict__ mono, float4* __restrict__ quad0,
                                        float2* __restrict__ quad1) {
  const int nc = info->ncells;
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < nc; c += gridDim.x * blockDim.x) {
    const MpRec r = rec[c];
    const float4 o = cell_open[c];
    const double im = r.m > 0 ? 1.0 / r.m : 0.0;
    size[c] = o;
    mono[c] = make_float4(o.x, o.y, o.z, (float)r.m);
    quad0[c] = make_float4((float)(r.ixx * im), (float)(r.iyy * im), (float)(r.izz * im), (float)(r.ixy * im));
    quad1[c] = make_float2((float)(r.ixz * im), (float)(r.iyz * im));
  }
}

}  // namespace bonsai
