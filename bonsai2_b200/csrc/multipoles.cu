// multipoles.cu -- monopole, quadrupole and opening size of every cell in one
// launch, bottom up.
//
// The reference (computeCellMultipoles, computeMultipoles.cu:81-190) gives a
// warp to every cell and rescans all of that cell's particles, O(N * depth)
// particle reads, with float products summed in double.  Here each leaf is
// reduced from its own particles (one thread per leaf, FP64, one pass: sums
// about the leaf's first particle, shifted to the centre of mass), and every
// node is combined from its
// children with the parallel-axis theorem by the child that finishes last
// (an arrival counter per cell; no thread waits on another).
// Each particle is read once.  The quantities match the reference's definitions:
//   M, COM; Q = second moment about the COM per unit mass (:148-158);
//   particle bounding box -> l = max(2 max h, 1e-6), s = |cvec - COM|,
//   cellOp = l/theta + s, stored squared (:168-177).
// cell_ls = (l, s, M l^3, 1.5 tr I) lets a walk with per-group opening angles
// form (l/theta_g + s)^2.  Stored for the walk as three float4 per cell, in
// the form the force kernel stages them (mass-weighted, pre-scaled and
// negated so that it needs fewer operations; I = M Q):
//   cell_stage[3c]     = (COM, -0.5 tr I)
//   cell_stage[3c + 1] = (M, -3Ixx, -3Iyy, -3Izz)
//   cell_stage[3c + 2] = (-3Ixy, -3Ixz, -3Iyz, -1.5 tr I)
// The FP64 record (MpRec) holds M, COM and the moments; the particle bounding
// box is a separate array, float for float positions and double (DS) for
// double-single positions, where particles enter the FP64 sums as hi + lo,
// extents are exact, and the COM is stored as hi (cell_open) plus lo (cell_lo).
#include <algorithm>

#include "common.cuh"
#include "kernels.cuh"

namespace bonsai {

// leaf moments in one pass over the particles (1) or two (0: centre of mass,
// then central moments)
// parents level by level, one launch per level from the deepest (0: 6.55 ms
// build phase at N = 2^24), or by the last-arriving child's climb with an
// arrival counter per cell (1: 6.99 ms; fences and atomics serialise its
// tail through the top levels); both bit-identical
#ifndef BONSAI_MP_CLIMB
#define BONSAI_MP_CLIMB 0
#endif
#ifndef BONSAI_MP_ONE_PASS
#define BONSAI_MP_ONE_PASS 1
#endif

template <bool DS>
struct BoxOf {
  typedef float T;
};
template <>
struct BoxOf<true> {
  typedef double T;
};

// minimum blocks per SM of the leaf and level passes (1: no bound; 5 or 6
// blocks spill the FP64 sums and were slower: build phase 4.59 / 4.84 ms
// against 4.50 at N = 2^24)
#ifndef BONSAI_MP_MINB
#define BONSAI_MP_MINB 1
#endif
#ifndef BONSAI_MP_BATCH
#define BONSAI_MP_BATCH 4
#endif
constexpr int kMpBatch = BONSAI_MP_BATCH;  // leaf particles loaded ahead of their sums

template <bool DS>
__device__ __forceinline__ void store_cell(int c, const MpRec& r, const typename BoxOf<DS>::T* bmin,
                                           const typename BoxOf<DS>::T* bmax, float inv_theta, MpRec* __restrict__ rec,
                                           typename BoxOf<DS>::T* __restrict__ box, float4* __restrict__ cell_open,
                                           float4* __restrict__ cell_stage,
                                           float4* __restrict__ cell_ls, float4* __restrict__ cell_lo) {
  rec[c] = r;
  for (int k = 0; k < 3; k++) { box[6 * (size_t)c + k] = bmin[k]; box[6 * (size_t)c + 3 + k] = bmax[k]; }
  const float cx = (float)r.cx, cy = (float)r.cy, cz = (float)r.cz;
  float s, l;
  if (DS) {
    // w: the staged record's -0.5 tr I (cell_stage[3c].w), so that the
    // double-single walk, which loads cell_lo for every visited cell, stages
    // an accepted cell without another load
    const float t15d = (float)(1.5 * (r.ixx + r.iyy + r.izz));
    cell_lo[c] = make_float4((float)(r.cx - (double)cx), (float)(r.cy - (double)cy), (float)(r.cz - (double)cz),
                             __fmul_rn(t15d, -1.0f / 3.0f));
    // extents and centre offsets from the exact box and COM
    double hm = 0.0, d2 = 0.0;
    const double com[3] = {r.cx, r.cy, r.cz};
    for (int k = 0; k < 3; k++) {
      const double v = 0.5 * ((double)bmax[k] + (double)bmin[k]) - com[k];
      hm = fmax(hm, 0.5 * ((double)bmax[k] - (double)bmin[k]));
      d2 += v * v;
    }
    s = (float)sqrt(d2);
    l = fmaxf((float)(2.0 * hm), 1.0e-6f);
  } else {
    const float vx = __fmul_rn(__fadd_rn((float)bmax[0], (float)bmin[0]), 0.5f);
    const float vy = __fmul_rn(__fadd_rn((float)bmax[1], (float)bmin[1]), 0.5f);
    const float vz = __fmul_rn(__fadd_rn((float)bmax[2], (float)bmin[2]), 0.5f);
    const float hx = __fmul_rn(__fsub_rn((float)bmax[0], (float)bmin[0]), 0.5f);
    const float hy = __fmul_rn(__fsub_rn((float)bmax[1], (float)bmin[1]), 0.5f);
    const float hz = __fmul_rn(__fsub_rn((float)bmax[2], (float)bmin[2]), 0.5f);
    const float dx = __fsub_rn(vx, cx), dy = __fsub_rn(vy, cy), dz = __fsub_rn(vz, cz);
    s = __fsqrt_rn(__fmaf_rn(dz, dz, __fmaf_rn(dy, dy, __fmul_rn(dx, dx))));
    l = fmaxf(__fmul_rn(2.0f, fmaxf(hx, fmaxf(hy, hz))), 1.0e-6f);
  }
  const float op = __fmaf_rn(l, inv_theta, s);
  cell_open[c] = make_float4(cx, cy, cz, __fmul_rn(op, op));
  // per-group opening angles recompute (l/theta_g + s)^2; the relative test
  // compares M l^3 (formed once here, in float) with tau ds^5
  const float mf = (float)r.m;
  const double tr = r.ixx + r.iyy + r.izz;
  const float t15 = (float)(1.5 * tr);
  // (the relative test's size is the box's l: the mass-weighted rms radius
  // sqrt(tr I / M) in its place ran 3-4 % slower at equal median error)
  const float mk = __fmul_rn(mf, __fmul_rn(l, __fmul_rn(l, l)));
  cell_ls[c] = make_float4(l, s, mk, t15);
  // the walk's staged record, copied to shared memory as it is (moments
  // negated so that every difference in the interaction is one add)
  float4* st = cell_stage + 3 * (size_t)c;
  st[0] = make_float4(cx, cy, cz, __fmul_rn(t15, -1.0f / 3.0f));
  st[1] = make_float4(mf, -(float)(3.0 * r.ixx), -(float)(3.0 * r.iyy), -(float)(3.0 * r.izz));
  st[2] = make_float4(-(float)(3.0 * r.ixy), -(float)(3.0 * r.ixz), -(float)(3.0 * r.iyz), -t15);
}

// Arrival on a parent's counter: a fence publishes this child's record, a
// relaxed atomic counts it, and only the last arriver fences again before it
// reads its siblings' records (through L2).
__device__ __forceinline__ bool arrive_last(int* p, int nch) {
  __threadfence();
  if (atomicAdd(p, 1) != nch - 1) return false;
  __threadfence();
  return true;
}

// A child's record fields.  CACHED (the level passes, whose children were
// written by earlier launches): 16-byte vector loads through L1, so a record
// costs 5 load instructions and its second read hits L1; otherwise (the
// arrival-counter climb, whose siblings wrote them in this launch) 8-byte
// loads from L2.
template <bool CACHED>
__device__ __forceinline__ void load_mass_com(const MpRec* r, double& m, double& x, double& y, double& z) {
  if (CACHED) {
    const double2 a = __ldg(reinterpret_cast<const double2*>(r)), b = __ldg(reinterpret_cast<const double2*>(r) + 1);
    m = a.x; x = a.y; y = b.x; z = b.y;
  } else {
    m = __ldcg(&r->m); x = __ldcg(&r->cx); y = __ldcg(&r->cy); z = __ldcg(&r->cz);
  }
}
template <bool CACHED>
__device__ __forceinline__ MpRec load_rec(const MpRec* r) {
  MpRec o;
  if (CACHED) {
    const double2* q = reinterpret_cast<const double2*>(r);
    const double2 a = __ldg(q), b = __ldg(q + 1), c = __ldg(q + 2), d = __ldg(q + 3), e = __ldg(q + 4);
    o.m = a.x; o.cx = a.y; o.cy = b.x; o.cz = b.y;
    o.ixx = c.x; o.iyy = c.y; o.izz = d.x; o.ixy = d.y; o.ixz = e.x; o.iyz = e.y;
  } else {
    o.m = __ldcg(&r->m); o.cx = __ldcg(&r->cx); o.cy = __ldcg(&r->cy); o.cz = __ldcg(&r->cz);
    o.ixx = __ldcg(&r->ixx); o.iyy = __ldcg(&r->iyy); o.izz = __ldcg(&r->izz);
    o.ixy = __ldcg(&r->ixy); o.ixz = __ldcg(&r->ixz); o.iyz = __ldcg(&r->iyz);
  }
  return o;
}
template <bool CACHED, class B>
__device__ __forceinline__ void load_box(const B* bk, B lo[3], B hi[3]) {
  if (CACHED && sizeof(B) == 4) {
    const float2* q = reinterpret_cast<const float2*>(bk);  // 24 B per cell: 8-byte aligned
    const float2 a = __ldg(q), b = __ldg(q + 1), c = __ldg(q + 2);
    lo[0] = (B)a.x; lo[1] = (B)a.y; lo[2] = (B)b.x; hi[0] = (B)b.y; hi[1] = (B)c.x; hi[2] = (B)c.y;
  } else if (CACHED) {
    const double2* q = reinterpret_cast<const double2*>(bk);  // 48 B per cell: 16-byte aligned
    const double2 a = __ldg(q), b = __ldg(q + 1), c = __ldg(q + 2);
    lo[0] = (B)a.x; lo[1] = (B)a.y; lo[2] = (B)b.x; hi[0] = (B)b.y; hi[1] = (B)c.x; hi[2] = (B)c.y;
  } else {
#pragma unroll
    for (int a = 0; a < 3; a++) { lo[a] = __ldcg(bk + a); hi[a] = __ldcg(bk + 3 + a); }
  }
}

// A parent's moments from its nch contiguous children (parallel-axis
// theorem, FP64), the children taken in index order.
template <bool DS, bool CACHED>
__device__ void combine_children(int p, int first, int nch, float inv_theta, MpRec* __restrict__ rec,
                                 typename BoxOf<DS>::T* __restrict__ box, float4* __restrict__ cell_open,
                                 float4* __restrict__ cell_stage,
                                 float4* __restrict__ cell_ls, float4* __restrict__ cell_lo) {
  typedef typename BoxOf<DS>::T B;
  double M = 0, X = 0, Y = 0, Z = 0;
  B bmn[3] = {(B)3.0e38, (B)3.0e38, (B)3.0e38}, bmx[3] = {(B)-3.0e38, (B)-3.0e38, (B)-3.0e38};
  // the children's records are loaded a batch ahead of their sums, which
  // stay in child order (the moments are the same to the bit)
  constexpr int kB = 4;
  for (int k0 = 0; k0 < nch; k0 += kB) {
    double mb[kB], xb[kB], yb[kB], zb[kB];
    B lo[kB][3], hi[kB][3];
#pragma unroll
    for (int u = 0; u < kB; u++) {
      const int k = min(k0 + u, nch - 1);
      load_mass_com<CACHED>(rec + first + k, mb[u], xb[u], yb[u], zb[u]);
      load_box<CACHED>(box + 6 * (size_t)(first + k), lo[u], hi[u]);
    }
#pragma unroll
    for (int u = 0; u < kB; u++) {
      if (k0 + u >= nch) break;
      const double mk = mb[u];
      M += mk;
      X += mk * xb[u]; Y += mk * yb[u]; Z += mk * zb[u];
#pragma unroll
      for (int a = 0; a < 3; a++) {
        bmn[a] = DS ? (B)fmin((double)bmn[a], (double)lo[u][a]) : (B)fminf((float)bmn[a], (float)lo[u][a]);
        bmx[a] = DS ? (B)fmax((double)bmx[a], (double)hi[u][a]) : (B)fmaxf((float)bmx[a], (float)hi[u][a]);
      }
    }
  }
  MpRec P;
  if (M > 0.0) { P.cx = X / M; P.cy = Y / M; P.cz = Z / M; }
  else {
    P.cx = 0.5 * ((double)bmn[0] + bmx[0]); P.cy = 0.5 * ((double)bmn[1] + bmx[1]);
    P.cz = 0.5 * ((double)bmn[2] + bmx[2]);
  }
  double I[6] = {0, 0, 0, 0, 0, 0};
  constexpr int kB2 = 2;
  for (int k0 = 0; k0 < nch; k0 += kB2) {
    MpRec cb[kB2];
#pragma unroll
    for (int u = 0; u < kB2; u++) {
      cb[u] = load_rec<CACHED>(rec + first + min(k0 + u, nch - 1));
    }
#pragma unroll
    for (int u = 0; u < kB2; u++) {
      if (k0 + u >= nch) break;
      const double mk = cb[u].m;
      const double dx = cb[u].cx - P.cx, dy = cb[u].cy - P.cy, dz = cb[u].cz - P.cz;
      I[0] += cb[u].ixx + mk * dx * dx;
      I[1] += cb[u].iyy + mk * dy * dy;
      I[2] += cb[u].izz + mk * dz * dz;
      I[3] += cb[u].ixy + mk * dx * dy;
      I[4] += cb[u].ixz + mk * dx * dz;
      I[5] += cb[u].iyz + mk * dy * dz;
    }
  }
  P.m = M;
  P.ixx = I[0]; P.iyy = I[1]; P.izz = I[2]; P.ixy = I[3]; P.ixz = I[4]; P.iyz = I[5];
  store_cell<DS>(p, P, bmn, bmx, inv_theta, rec, box, cell_open, cell_stage, cell_ls, cell_lo);
}

// Combines parents bottom-up while this thread is the last child to arrive.
template <bool DS>
__device__ void climb(int c, [[maybe_unused]] int ncells, const uint4* __restrict__ cell_data,
                      const int* __restrict__ cell_parent,
                      float inv_theta, MpRec* __restrict__ rec, typename BoxOf<DS>::T* __restrict__ box,
                      float4* __restrict__ cell_open, float4* __restrict__ cell_stage,
                      float4* __restrict__ cell_ls, int* __restrict__ mp_count, float4* __restrict__ cell_lo) {
  while (true) {
    const int p = cell_parent[c];
    if (p < 0) break;
    if (!BONSAI_IN_RANGE(p, ncells, 0x303)) break;
    const unsigned y = cell_data[p].y;
    const int first = (int)(y & 0x1FFFFFFFu), nch = (int)(y >> 29) + 1;
    if (!BONSAI_IN_RANGE(first + nch - 1, ncells, 0x304) || !BONSAI_IN_RANGE(c - first, nch, 0x305)) break;
    if (!arrive_last(mp_count + p, nch)) break;
    combine_children<DS, false>(p, first, nch, inv_theta, rec, box, cell_open, cell_stage, cell_ls, cell_lo);
    c = p;
  }
}

// The nodes of one level from their children, one thread per cell (leaves
// were done by the leaf pass): the level-by-level form of the climb.
template <bool DS>
__global__ void __launch_bounds__(256, BONSAI_MP_MINB) k_mp_level(int L, const TreeInfo* __restrict__ info,
                                                  const uint4* __restrict__ cell_data, float inv_theta,
                                                  MpRec* __restrict__ rec, typename BoxOf<DS>::T* __restrict__ box,
                                                  float4* __restrict__ cell_open, float4* __restrict__ cell_stage, float4* __restrict__ cell_ls,
                                                  int cell_cap, float4* __restrict__ cell_lo) {
  if (info->ncells > cell_cap) return;
  [[maybe_unused]] const int ncells = info->ncells;
  const int b = info->level_beg[L], e = info->level_end[L];
  for (int c = b + blockIdx.x * blockDim.x + threadIdx.x; c < e; c += gridDim.x * blockDim.x) {
    const unsigned y = cell_data[c].y;
    if (y == 0xFFFFFFFFu) continue;
    const int first = (int)(y & 0x1FFFFFFFu), nch = (int)(y >> 29) + 1;
    if (!BONSAI_IN_RANGE(first + nch - 1, ncells, 0x307)) continue;
    combine_children<DS, true>(c, first, nch, inv_theta, rec, box, cell_open, cell_stage, cell_ls, cell_lo);
  }
}

// One thread per leaf: the leaf's moments (one pass by default), then the
// bottom-up climb.  (Half-warp-cooperative leaves
// with shuffle reductions were measured 13x slower on the B200.)
template <bool DS, bool CLIMB>
__global__ void __launch_bounds__(256, BONSAI_MP_MINB) k_multipoles(const int* __restrict__ leaf_list, const TreeInfo* __restrict__ info,
                                                    const uint4* __restrict__ cell_data,
                                                    const int* __restrict__ cell_parent,
                                                    const float4* __restrict__ jpos, float inv_theta,
                                                    MpRec* __restrict__ rec, typename BoxOf<DS>::T* __restrict__ box,
                                                    float4* __restrict__ cell_open, float4* __restrict__ cell_stage, float4* __restrict__ cell_ls,
                                                    int* __restrict__ mp_count, int cell_cap,
                                                    const float4* __restrict__ jlo, float4* __restrict__ cell_lo) {
  typedef typename BoxOf<DS>::T B;
  const int nleaves = info->nleaves;
  if (info->ncells > cell_cap) return;
  [[maybe_unused]] const int ncells = info->ncells, npart = info->npart;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < nleaves; t += gridDim.x * blockDim.x) {
    const int c = leaf_list[t];
    if (!BONSAI_IN_RANGE(c, ncells, 0x301)) continue;
    const uint4 cd = cell_data[c];
    const int b = (int)cd.z, e = (int)cd.w;
    if (!BONSAI_IN_RANGE(e - 1, npart, 0x302) || !BONSAI_IN_RANGE(b, e, 0x306)) continue;
    MpRec r;
    B mn[3] = {(B)3.0e38, (B)3.0e38, (B)3.0e38}, mx[3] = {(B)-3.0e38, (B)-3.0e38, (B)-3.0e38};
#if BONSAI_MP_ONE_PASS
    // one pass: sums about the leaf's first particle x0 (d = x - x0), then the
    // shift to the centre of mass: COM = x0 + S1/M, I = S2 - S1 S1^T / M; the
    // cancellation is relative to the leaf's extent, not to |x0|
    double x0, y0, z0;
    {
      const float4 p = __ldg(jpos + b);
      x0 = p.x; y0 = p.y; z0 = p.z;
      if (DS) {
        const float4 l = __ldg(jlo + b);
        x0 += l.x; y0 += l.y; z0 += l.z;
      }
    }
    double m = 0, s1x = 0, s1y = 0, s1z = 0, q[6] = {0, 0, 0, 0, 0, 0};
    // four particles' loads in flight before they are summed (in order)
    for (int i0 = b; i0 < e; i0 += kMpBatch) {
      float4 pb[kMpBatch], lb[kMpBatch];
#pragma unroll
      for (int u = 0; u < kMpBatch; u++) {
        const int i = min(i0 + u, e - 1);
        pb[u] = __ldg(jpos + i);
        if (DS) lb[u] = __ldg(jlo + i);
      }
#pragma unroll
      for (int u = 0; u < kMpBatch; u++) {
        if (i0 + u >= e) break;
        const float4 p = pb[u];
        double px = p.x, py = p.y, pz = p.z;
        if (DS) {
          const float4 l = lb[u];
          px += l.x; py += l.y; pz += l.z;
          mn[0] = (B)fmin((double)mn[0], px); mn[1] = (B)fmin((double)mn[1], py); mn[2] = (B)fmin((double)mn[2], pz);
          mx[0] = (B)fmax((double)mx[0], px); mx[1] = (B)fmax((double)mx[1], py); mx[2] = (B)fmax((double)mx[2], pz);
        } else {
          mn[0] = (B)fminf((float)mn[0], p.x); mn[1] = (B)fminf((float)mn[1], p.y); mn[2] = (B)fminf((float)mn[2], p.z);
          mx[0] = (B)fmaxf((float)mx[0], p.x); mx[1] = (B)fmaxf((float)mx[1], p.y); mx[2] = (B)fmaxf((float)mx[2], p.z);
        }
        const double w = p.w, dx = px - x0, dy = py - y0, dz = pz - z0;
        m += w;
        s1x += w * dx; s1y += w * dy; s1z += w * dz;
        q[0] += w * dx * dx; q[1] += w * dy * dy; q[2] += w * dz * dz;
        q[3] += w * dx * dy; q[4] += w * dx * dz; q[5] += w * dy * dz;
      }
    }
    if (m > 0.0) {
      const double ux = s1x / m, uy = s1y / m, uz = s1z / m;
      r.cx = x0 + ux; r.cy = y0 + uy; r.cz = z0 + uz;
      q[0] -= s1x * ux; q[1] -= s1y * uy; q[2] -= s1z * uz;
      q[3] -= s1x * uy; q[4] -= s1x * uz; q[5] -= s1y * uz;
    } else {
      r.cx = 0.5 * ((double)mn[0] + mx[0]); r.cy = 0.5 * ((double)mn[1] + mx[1]); r.cz = 0.5 * ((double)mn[2] + mx[2]);
    }
#else
    double m = 0, sx = 0, sy = 0, sz = 0;
    for (int i = b; i < e; i++) {
      const float4 p = __ldg(jpos + i);
      double px = p.x, py = p.y, pz = p.z;
      if (DS) {
        const float4 l = __ldg(jlo + i);
        px += l.x; py += l.y; pz += l.z;
        mn[0] = (B)fmin((double)mn[0], px); mn[1] = (B)fmin((double)mn[1], py); mn[2] = (B)fmin((double)mn[2], pz);
        mx[0] = (B)fmax((double)mx[0], px); mx[1] = (B)fmax((double)mx[1], py); mx[2] = (B)fmax((double)mx[2], pz);
      } else {
        mn[0] = (B)fminf((float)mn[0], p.x); mn[1] = (B)fminf((float)mn[1], p.y); mn[2] = (B)fminf((float)mn[2], p.z);
        mx[0] = (B)fmaxf((float)mx[0], p.x); mx[1] = (B)fmaxf((float)mx[1], p.y); mx[2] = (B)fmaxf((float)mx[2], p.z);
      }
      m += p.w;
      sx += (double)p.w * px; sy += (double)p.w * py; sz += (double)p.w * pz;
    }
    if (m > 0.0) { r.cx = sx / m; r.cy = sy / m; r.cz = sz / m; }
    else {
      r.cx = 0.5 * ((double)mn[0] + mx[0]); r.cy = 0.5 * ((double)mn[1] + mx[1]); r.cz = 0.5 * ((double)mn[2] + mx[2]);
    }
    double q[6] = {0, 0, 0, 0, 0, 0};
    for (int i = b; i < e; i++) {
      const float4 p = __ldg(jpos + i);
      double px = p.x, py = p.y, pz = p.z;
      if (DS) {
        const float4 l = __ldg(jlo + i);
        px += l.x; py += l.y; pz += l.z;
      }
      const double dx = px - r.cx, dy = py - r.cy, dz = pz - r.cz, w = p.w;
      q[0] += w * dx * dx; q[1] += w * dy * dy; q[2] += w * dz * dz;
      q[3] += w * dx * dy; q[4] += w * dx * dz; q[5] += w * dy * dz;
    }
#endif
    r.m = m;
    r.ixx = q[0]; r.iyy = q[1]; r.izz = q[2]; r.ixy = q[3]; r.ixz = q[4]; r.iyz = q[5];
    store_cell<DS>(c, r, mn, mx, inv_theta, rec, box, cell_open, cell_stage, cell_ls, cell_lo);
    if (CLIMB)
      climb<DS>(c, ncells, cell_data, cell_parent, inv_theta, rec, box, cell_open, cell_stage, cell_ls, mp_count,
                cell_lo);
  }
}

void launch_multipoles(const int* leaf_list, const TreeInfo* info, const uint4* cell_data, const int* cell_parent,
                       const float4* jpos, float inv_theta, MpRec* rec, void* box, float4* cell_open,
                       float4* cell_stage, float4* cell_ls, int* mp_count, int cell_cap,
                       const float4* jlo, float4* cell_lo, int nblocks, cudaStream_t s) {
#if BONSAI_MP_CLIMB
  if (jlo)
    k_multipoles<true, true><<<nblocks, 256, 0, s>>>(leaf_list, info, cell_data, cell_parent, jpos, inv_theta, rec,
                                                     static_cast<double*>(box), cell_open, cell_stage, cell_ls,
                                                     mp_count, cell_cap, jlo, cell_lo);
  else
    k_multipoles<false, true><<<nblocks, 256, 0, s>>>(leaf_list, info, cell_data, cell_parent, jpos, inv_theta, rec,
                                                      static_cast<float*>(box), cell_open, cell_stage, cell_ls,
                                                      mp_count, cell_cap, nullptr, nullptr);
#else
  // leaves, then the nodes level by level from the deepest (levels 20 .. 1)
  const int lb = nblocks;
  if (jlo) {
    k_multipoles<true, false><<<nblocks, 256, 0, s>>>(leaf_list, info, cell_data, cell_parent, jpos, inv_theta, rec,
                                                      static_cast<double*>(box), cell_open, cell_stage, cell_ls,
                                                      mp_count, cell_cap, jlo, cell_lo);
    for (int L = kMaxLevel - 1; L >= 1; L--)
      k_mp_level<true><<<lb, 256, 0, s>>>(L, info, cell_data, inv_theta, rec, static_cast<double*>(box), cell_open,
                                          cell_stage, cell_ls, cell_cap, cell_lo);
  } else {
    k_multipoles<false, false><<<nblocks, 256, 0, s>>>(leaf_list, info, cell_data, cell_parent, jpos, inv_theta,
                                                       rec, static_cast<float*>(box), cell_open, cell_stage,
                                                       cell_ls, mp_count, cell_cap, nullptr, nullptr);
    for (int L = kMaxLevel - 1; L >= 1; L--)
      k_mp_level<false><<<lb, 256, 0, s>>>(L, info, cell_data, inv_theta, rec, static_cast<float*>(box), cell_open,
                                           cell_stage, cell_ls, cell_cap, nullptr);
  }
#endif
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

BONSAI_BOUNDS_ACCESSOR(bounds_word_multipoles)

}  // namespace bonsai
