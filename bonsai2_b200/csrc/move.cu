// move.cu -- leapfrog move with the energy sums fused in, the FP64 direct-sum
// checker, and the scatter back to the caller's particle order.
//
// The reference's moveParticles and computeEnergies are stubs
// (moveParticles.cu:3-7, computeEnergies.cu:3-7); its only energy term is the
// potential sum made inside the walk (computeForces.cu:576-607).  Here the
// move is a kick-drift-kick leapfrog with merged kicks, one HBM pass:
//   closing kick  v += a dt/2   (skipped on the first step)
//   energy sums at the synchronised point (FP64): T, W = 1/2 sum m phi,
//     W without the i==j self term, momentum, mass
//   opening kick  v += a dt/2,  drift x += v dt
// Per-block FP64 partials are folded in a fixed order by the last block, so
// the sums are deterministic.
#include <algorithm>

#include "common.cuh"
#include "kernels.cuh"

namespace bonsai {

constexpr int kNE = 8;

struct EnergySums {
  double T = 0, W = 0, S = 0, px = 0, py = 0, pz = 0, mt = 0;
};

// x_hi + x_lo += d in double-single: exact two-sum of hi and d, the error
// and the old low part folded into lo, renormalised (Dekker 1971; Knuth TAOCP
// vol. 2, 4.2.2)
__device__ __forceinline__ void ds_add(float& hi, float& lo, float d) {
  const float s = __fadd_rn(hi, d);
  const float bb = __fsub_rn(s, hi);
  const float err = __fadd_rn(__fsub_rn(hi, __fsub_rn(s, bb)), __fsub_rn(d, bb));
  const float l = __fadd_rn(lo, err);
  hi = __fadd_rn(s, l);
  lo = __fsub_rn(l, __fsub_rn(hi, s));
}

// one particle: closing kick (hc = 0 on the first step), energy terms at the
// synchronised point, then opening kick and drift when write is set.  lo
// (nullable): double-single low parts of the positions
__device__ __forceinline__ void move_one(float4* __restrict__ pos, float4* __restrict__ vel,
                                         const float4* __restrict__ acc, int i, float dt, float h, float hc,
                                         double ieps, int write, EnergySums& e, float4* __restrict__ lo = nullptr) {
  float4 p = pos[i], v = vel[i];
  const float4 a = acc[i];
  v.x = fmaf(a.x, hc, v.x); v.y = fmaf(a.y, hc, v.y); v.z = fmaf(a.z, hc, v.z);
  const double m = p.w;
  e.T += 0.5 * m * ((double)v.x * v.x + (double)v.y * v.y + (double)v.z * v.z);
  e.W += 0.5 * m * a.w;
  e.S += 0.5 * m * m * ieps;
  e.px += m * v.x; e.py += m * v.y; e.pz += m * v.z; e.mt += m;
  if (write) {
    v.x = fmaf(a.x, h, v.x); v.y = fmaf(a.y, h, v.y); v.z = fmaf(a.z, h, v.z);
    if (lo) {
      float4 l = lo[i];
      ds_add(p.x, l.x, __fmul_rn(v.x, dt));
      ds_add(p.y, l.y, __fmul_rn(v.y, dt));
      ds_add(p.z, l.z, __fmul_rn(v.z, dt));
      lo[i] = l;
    } else {
      p.x = fmaf(v.x, dt, p.x); p.y = fmaf(v.y, dt, p.y); p.z = fmaf(v.z, dt, p.z);
    }
    pos[i] = p;
    vel[i] = v;
  }
}

// block sum of the eight energy terms {T, W, W+S, T+W+S, Px, Py, Pz, M};
// thread k < 8 returns term k
__device__ __forceinline__ double block_energy_sum(const EnergySums& s, double (*sh)[8]) {
  const double e[kNE] = {s.T, s.W, s.W + s.S, s.T + s.W + s.S, s.px, s.py, s.pz, s.mt};
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < kNE; k++) {
    double x = e[k];
#pragma unroll
    for (int o = 16; o >= 1; o >>= 1) x += __shfl_xor_sync(kFull, x, o);
    if (lane == 0) sh[k][w] = x;
  }
  __syncthreads();
  double x = 0;
  if (threadIdx.x < kNE)
    for (int q = 0; q < (int)(blockDim.x >> 5); q++) x += sh[threadIdx.x][q];
  __syncthreads();
  return x;
}

// closing kick taken when *closing is set (device flag: set by every writing
// move, cleared when particles are loaded), so the same captured graph serves
// the first and later steps.  write == 0 computes the energies only.
__global__ void __launch_bounds__(256) k_move(float4* __restrict__ pos, float4* __restrict__ vel,
                                              const float4* __restrict__ acc, int n, float dt,
                                              int* __restrict__ closing, float eps, int write,
                                              double* __restrict__ partial, unsigned* __restrict__ ticket,
                                              double* __restrict__ energies, float4* __restrict__ lo) {
  const float h = 0.5f * dt;
  const float hc = (*closing) ? h : 0.0f;
  const double ieps = eps > 0.f ? 1.0 / (double)eps : 0.0;
  EnergySums e;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    move_one(pos, vel, acc, i, dt, h, hc, ieps, write, e, lo);
  __shared__ double sh[kNE][8];
  __shared__ bool last;
  const double x = block_energy_sum(e, sh);
  if (threadIdx.x < kNE) partial[blockIdx.x * kNE + threadIdx.x] = x;
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    last = (atomicAdd(ticket, 1u) == gridDim.x - 1);
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  if (threadIdx.x < kNE) {
    double y = 0;
    for (int b = 0; b < (int)gridDim.x; b++) y += __ldcg(partial + b * kNE + threadIdx.x);
    energies[threadIdx.x] = y;
  }
  if (threadIdx.x == 0) {
    *ticket = 0u;
    if (write) *closing = 1;
  }
}

// Ensemble move: the same per-particle update, blocks over chunks; each
// chunk's energy terms are kept, and the last block folds them per system
// (chunk order) and in total.
__global__ void __launch_bounds__(256) k_move_sys(float4* __restrict__ pos, float4* __restrict__ vel,
                                                  const float4* __restrict__ acc, const int4* __restrict__ chunks,
                                                  int nchunks, const int* __restrict__ chunk_beg, int nsys, float dt,
                                                  int* __restrict__ closing, float eps, int write,
                                                  double* __restrict__ chunk_part, unsigned* __restrict__ ticket,
                                                  double* __restrict__ energies, double* __restrict__ sys_energies,
                                                  float4* __restrict__ lo) {
  const float h = 0.5f * dt;
  const float hc = (*closing) ? h : 0.0f;
  const double ieps = eps > 0.f ? 1.0 / (double)eps : 0.0;
  __shared__ double sh[kNE][8];
  __shared__ bool last;
  for (int c = blockIdx.x; c < nchunks; c += gridDim.x) {
    const int4 ch = chunks[c];
    EnergySums e;
    for (int i = ch.x + threadIdx.x; i < ch.y; i += blockDim.x)
      move_one(pos, vel, acc, i, dt, h, hc, ieps, write, e, lo);
    const double x = block_energy_sum(e, sh);
    if (threadIdx.x < kNE) chunk_part[(size_t)c * kNE + threadIdx.x] = x;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    last = (atomicAdd(ticket, 1u) == gridDim.x - 1);
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  for (int s = threadIdx.x; s < nsys; s += blockDim.x) {
    double y[kNE] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (int c = chunk_beg[s]; c < chunk_beg[s + 1]; c++)
      for (int k = 0; k < kNE; k++) y[k] += __ldcg(chunk_part + (size_t)c * kNE + k);
    for (int k = 0; k < kNE; k++) sys_energies[(size_t)s * kNE + k] = y[k];
  }
  if (threadIdx.x < kNE) {
    double y = 0;
    for (int c = 0; c < nchunks; c++) y += __ldcg(chunk_part + (size_t)c * kNE + threadIdx.x);
    energies[threadIdx.x] = y;
  }
  if (threadIdx.x == 0) {
    *ticket = 0u;
    if (write) *closing = 1;
  }
}

void launch_move_sys(float4* pos, float4* vel, const float4* acc, const int4* chunks, int nchunks,
                     const int* chunk_beg, int nsys, float dt, int* closing, float eps, int write, double* chunk_part,
                     int nblocks, unsigned* ticket, double* energies, double* sys_energies, cudaStream_t s,
                     float4* lo) {
  k_move_sys<<<nblocks, 256, 0, s>>>(pos, vel, acc, chunks, nchunks, chunk_beg, nsys, dt, closing, eps, write,
                                     chunk_part, ticket, energies, sys_energies, lo);
}

void launch_move(float4* pos, float4* vel, const float4* acc, int n, float dt, int* closing, float eps, int write,
                 double* partial, int nblocks, unsigned* ticket, double* energies, cudaStream_t s, float4* lo) {
  k_move<<<nblocks, 256, 0, s>>>(pos, vel, acc, n, dt, closing, eps, write, partial, ticket, energies, lo);
}

// FP64 direct summation for sample particles (checker): grid (ceil(ns/256),
// nsplit); thread = one sample, block = one slice of the sources.  A sample
// index outside [0, n) reads nothing: its partial sums are NaN, so its output
// row is NaN (the allocation-free entry point passes caller device indices
// that no host code has checked).
__global__ void __launch_bounds__(256) k_direct_fp64(const float4* __restrict__ pos, int n,
                                                     const int* __restrict__ sample, int ns, double eps2,
                                                     int include_self, double* __restrict__ part,
                                                     const float4* __restrict__ lo) {
  __shared__ double4 sj[256];
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  const int nsplit = gridDim.y;
  const int jb = (int)((long long)n * blockIdx.y / nsplit), je = (int)((long long)n * (blockIdx.y + 1) / nsplit);
  const int si = s < ns ? sample[s] : 0;
  const bool valid = si >= 0 && si < n;
  const int i = valid ? si : 0;
  const float4 pi = pos[i];
  double xi = pi.x, yi = pi.y, zi = pi.z;
  if (lo) {
    const float4 l = lo[i];
    xi += l.x; yi += l.y; zi += l.z;
  }
  double ax = 0, ay = 0, az = 0, ph = 0;
  for (int j0 = jb; j0 < je; j0 += 256) {
    __syncthreads();
    const int jj = j0 + threadIdx.x;
    if (jj < je) {
      const float4 p = pos[jj];
      double4 q = make_double4(p.x, p.y, p.z, p.w);
      if (lo) {
        const float4 l = lo[jj];
        q.x += l.x; q.y += l.y; q.z += l.z;
      }
      sj[threadIdx.x] = q;
    }
    __syncthreads();
    const int cnt = min(256, je - j0);
    for (int t = 0; t < cnt; t++) {
      if (j0 + t == i && !include_self) continue;
      const double4 q = sj[t];
      const double dx = q.x - xi, dy = q.y - yi, dz = q.z - zi;
      const double r2 = fma(dz, dz, fma(dy, dy, fma(dx, dx, eps2)));
      const double rinv = rsqrt(r2);
      const double mr = q.w * rinv;
      const double mr3 = mr * rinv * rinv;
      ax = fma(mr3, dx, ax); ay = fma(mr3, dy, ay); az = fma(mr3, dz, az); ph -= mr;
    }
  }
  if (s < ns) {
    if (!valid) ax = ay = az = ph = __longlong_as_double(0x7ff8000000000000LL);
    double* o = part + ((size_t)blockIdx.y * ns + s) * 4;
    o[0] = ax; o[1] = ay; o[2] = az; o[3] = ph;
  }
}

__global__ void k_direct_fold(const double* __restrict__ part, int ns, int nsplit, double* __restrict__ out) {
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < 4 * ns; t += gridDim.x * blockDim.x) {
    double x = 0;
    for (int q = 0; q < nsplit; q++) x += part[(size_t)q * ns * 4 + t];
    out[t] = x;
  }
}

void launch_direct_fp64(const float4* pos, int n, const int* sample, int ns, double eps2, int include_self,
                        double* part, int nsplit, double* out, cudaStream_t s, const float4* lo) {
  dim3 grid((ns + 255) / 256, nsplit);
  k_direct_fp64<<<grid, 256, 0, s>>>(pos, n, sample, ns, eps2, include_self, part, lo);
  k_direct_fold<<<(4 * ns + 255) / 256, 256, 0, s>>>(part, ns, nsplit, out);
}

// The pending closing kick v += a dt/2 (the same operation the move applies
// when the closing flag is set), for checkpoints with synchronised
// velocities; the caller clears the flag afterwards.
__global__ void __launch_bounds__(256) k_closing_kick(float4* __restrict__ vel, const float4* __restrict__ acc, int n,
                                                      float dt, const int* __restrict__ closing) {
  if (!*closing) return;
  const float h = 0.5f * dt;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    float4 v = vel[i];
    const float4 a = acc[i];
    v.x = fmaf(a.x, h, v.x); v.y = fmaf(a.y, h, v.y); v.z = fmaf(a.z, h, v.z);
    vel[i] = v;
  }
}

void launch_closing_kick(float4* vel, const float4* acc, int n, float dt, int* closing, int nblocks, cudaStream_t s) {
  k_closing_kick<<<nblocks, 256, 0, s>>>(vel, acc, n, dt, closing);
  cudaMemsetAsync(closing, 0, sizeof(int), s);
}

// ---------------------------------------------------------------------------
// Block time steps: hierarchical power-of-two levels, kick-drift-kick per
// particle.  Level k steps by dt_k = dt / 2^k; the big step dt is cut into
// 2^K substeps of dt / 2^K.  At substep s a level-k particle starts a step when
// s is a multiple of 2^(K-k) and ends one when s + 1 is.
// ---------------------------------------------------------------------------
__device__ __forceinline__ bool on_boundary(int s, int k, int K) { return (s & ((1 << (K - k)) - 1)) == 0; }

// opening half kick of the particles whose step starts at substep s, then the
// drift of every particle by one substep (double-single when lo is given)
__global__ void __launch_bounds__(256) k_bts_open_drift(float4* __restrict__ pos, float4* __restrict__ vel,
                                                        const float4* __restrict__ acc,
                                                        const unsigned char* __restrict__ lev, int n, float dt, int K,
                                                        int s, float4* __restrict__ lo) {
  const float dmin = ldexpf(dt, -K);
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int k = lev[i];
    float4 p = pos[i], v = vel[i];
    if (on_boundary(s, k, K)) {
      const float h = ldexpf(dt, -k - 1);
      const float4 a = acc[i];
      v.x = fmaf(a.x, h, v.x); v.y = fmaf(a.y, h, v.y); v.z = fmaf(a.z, h, v.z);
      vel[i] = v;
    }
    if (lo) {
      float4 l = lo[i];
      ds_add(p.x, l.x, __fmul_rn(v.x, dmin));
      ds_add(p.y, l.y, __fmul_rn(v.y, dmin));
      ds_add(p.z, l.z, __fmul_rn(v.z, dmin));
      lo[i] = l;
    } else {
      p.x = fmaf(v.x, dmin, p.x); p.y = fmaf(v.y, dmin, p.y); p.z = fmaf(v.z, dmin, p.z);
    }
    pos[i] = p;
  }
}

// Closing half kick of the particles whose step ends at s1 (= s + 1) with
// their new accelerations, then their next level: the smallest k with
// dt / 2^k <= eta sqrt(eps / |a|), no smaller than K - (trailing zeros of s1)
// (a step must start on its own boundary) and than the old level - 1 (a step
// at most doubles).  assign: levels for every particle, no kick (start).
__global__ void __launch_bounds__(256) k_bts_close(float4* __restrict__ vel, const float4* __restrict__ acc,
                                                   unsigned char* __restrict__ lev, int n, float dt, int K, int s1,
                                                   float eta, float eps, int assign) {
  const int sync = (s1 & ((1 << K) - 1)) == 0 ? 0 : K - (__ffs(s1) - 1);
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int k = lev[i];
    if (!assign && !on_boundary(s1, k, K)) continue;
    const float4 a = acc[i];
    if (!assign) {
      const float h = ldexpf(dt, -k - 1);
      float4 v = vel[i];
      v.x = fmaf(a.x, h, v.x); v.y = fmaf(a.y, h, v.y); v.z = fmaf(a.z, h, v.z);
      vel[i] = v;
    }
    const float am = __fsqrt_rn(__fadd_rn(__fadd_rn(__fmul_rn(a.x, a.x), __fmul_rn(a.y, a.y)), __fmul_rn(a.z, a.z)));
    const float dti = am > 0.f ? __fmul_rn(eta, __fsqrt_rn(__fdiv_rn(eps, am))) : 3.0e38f;
    int kn = 0;
    while (kn < K && ldexpf(dt, -kn) > dti) kn++;
    kn = max(kn, sync);
    if (!assign) kn = max(kn, k - 1);
    lev[i] = (unsigned char)kn;
  }
}

// groups holding at least one particle whose step ends at s1, compacted
__global__ void __launch_bounds__(256) k_bts_active_groups(const int2* __restrict__ groups,
                                                           const TreeInfo* __restrict__ info,
                                                           const unsigned char* __restrict__ lev, int K, int s1,
                                                           int* __restrict__ list, unsigned* __restrict__ count) {
  const int ng = info->ngroups;
  for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < ng; g += gridDim.x * blockDim.x) {
    const int2 gd = groups[g];
    bool act = false;
    for (int i = gd.x; i < gd.x + gd.y && !act; i++) act = on_boundary(s1, lev[i], K);
    if (act) {
      const unsigned slot = atomicAdd(count, 1u);
      if (BONSAI_IN_RANGE(slot, ng, 0x701)) list[slot] = g;
    }
  }
}

__global__ void __launch_bounds__(256) k_max_level(const unsigned char* __restrict__ lev, int n,
                                                   int* __restrict__ out) {
  int m = 0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) m = max(m, (int)lev[i]);
  for (int o = 16; o >= 1; o >>= 1) m = max(m, __shfl_xor_sync(kFull, m, o));
  if ((threadIdx.x & 31) == 0 && m > 0) atomicMax(out, m);
}

void launch_max_level(const unsigned char* lev, int n, int* out, int nblocks, cudaStream_t st) {
  cudaMemsetAsync(out, 0, sizeof(int), st);
  k_max_level<<<nblocks, 256, 0, st>>>(lev, n, out);
}

__global__ void __launch_bounds__(256) k_gather_u8(const int* __restrict__ perm, int n,
                                                   const unsigned char* __restrict__ in,
                                                   unsigned char* __restrict__ out) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) out[k] = in[perm[k]];
}

__global__ void __launch_bounds__(256) k_scatter_u8(const int* __restrict__ id, int n,
                                                    const unsigned char* __restrict__ in,
                                                    unsigned char* __restrict__ out) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
    const int d = id[k];
    if (BONSAI_IN_RANGE(d, n, 0x702)) out[d] = in[k];
  }
}

void launch_bts_open_drift(float4* pos, float4* vel, const float4* acc, const unsigned char* lev, int n, float dt,
                           int K, int s, float4* lo, int nblocks, cudaStream_t st) {
  k_bts_open_drift<<<nblocks, 256, 0, st>>>(pos, vel, acc, lev, n, dt, K, s, lo);
}
void launch_bts_close(float4* vel, const float4* acc, unsigned char* lev, int n, float dt, int K, int s1, float eta,
                      float eps, int assign, int nblocks, cudaStream_t st) {
  k_bts_close<<<nblocks, 256, 0, st>>>(vel, acc, lev, n, dt, K, s1, eta, eps, assign);
}
void launch_bts_active_groups(const int2* groups, const TreeInfo* info, const unsigned char* lev, int K, int s1,
                              int* list, unsigned* count, int nblocks, cudaStream_t st) {
  cudaMemsetAsync(count, 0, sizeof(unsigned), st);
  k_bts_active_groups<<<nblocks, 256, 0, st>>>(groups, info, lev, K, s1, list, count);
}
void launch_gather_u8(const int* perm, int n, const unsigned char* in, unsigned char* out, int nblocks,
                      cudaStream_t st) {
  k_gather_u8<<<nblocks, 256, 0, st>>>(perm, n, in, out);
}
void launch_scatter_u8(const int* id, int n, const unsigned char* in, unsigned char* out, int nblocks,
                       cudaStream_t st) {
  k_scatter_u8<<<nblocks, 256, 0, st>>>(id, n, in, out);
}

// Ensemble checker: each sample's force from the particles of its own system
// only (positions in the caller's order, systems contiguous; lo, nullable:
// double-single low parts, positions taken as hi + lo); one block per sample,
// fixed-order block reduction.
__global__ void __launch_bounds__(256) k_direct_fp64_sys(const float4* __restrict__ pos,
                                                         const int* __restrict__ sys_off, int nsys,
                                                         const int* __restrict__ sample, int ns, double eps2,
                                                         int include_self, double* __restrict__ out,
                                                         const float4* __restrict__ lo) {
  __shared__ double sh[4][8];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  for (int s = blockIdx.x; s < ns; s += gridDim.x) {
    const int i = sample[s];
    const int sy = sys_of(sys_off, nsys, i);
    const int jb = sys_off[sy], je = sys_off[sy + 1];
    const float4 pi = pos[i];
    double xi = pi.x, yi = pi.y, zi = pi.z;
    if (lo) {
      const float4 l = lo[i];
      xi += l.x; yi += l.y; zi += l.z;
    }
    double a[4] = {0, 0, 0, 0};
    for (int j = jb + threadIdx.x; j < je; j += blockDim.x) {
      if (j == i && !include_self) continue;
      const float4 q = pos[j];
      double qx = q.x, qy = q.y, qz = q.z;
      if (lo) {
        const float4 l = lo[j];
        qx += l.x; qy += l.y; qz += l.z;
      }
      const double dx = qx - xi, dy = qy - yi, dz = qz - zi;
      const double r2 = fma(dz, dz, fma(dy, dy, fma(dx, dx, eps2)));
      const double rinv = rsqrt(r2);
      const double mr = q.w * rinv;
      const double mr3 = mr * rinv * rinv;
      a[0] = fma(mr3, dx, a[0]); a[1] = fma(mr3, dy, a[1]); a[2] = fma(mr3, dz, a[2]); a[3] -= mr;
    }
#pragma unroll
    for (int k = 0; k < 4; k++) {
      double x = a[k];
#pragma unroll
      for (int o = 16; o >= 1; o >>= 1) x += __shfl_xor_sync(kFull, x, o);
      if (lane == 0) sh[k][w] = x;
    }
    __syncthreads();
    if (threadIdx.x < 4) {
      double x = 0;
      for (int q = 0; q < (int)(blockDim.x >> 5); q++) x += sh[threadIdx.x][q];
      out[(size_t)s * 4 + threadIdx.x] = x;
    }
    __syncthreads();
  }
}

void launch_direct_fp64_sys(const float4* pos, const int* sys_off, int nsys, const int* sample, int ns, double eps2,
                            int include_self, double* out, cudaStream_t s, const float4* lo) {
  k_direct_fp64_sys<<<ns < 65535 ? ns : 65535, 256, 0, s>>>(pos, sys_off, nsys, sample, ns, eps2, include_self, out,
                                                            lo);
}

// out[id[k]] = in[k]
__global__ void k_scatter_by_id(const int* __restrict__ id, int n, const float4* __restrict__ in,
                                float4* __restrict__ out) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) out[id[k]] = in[k];
}

__global__ void k_iota(int* __restrict__ a, int n) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) a[k] = k;
}

}  // namespace bonsai

namespace bonsai {

// FP32 FMA throughput probe: 8 independent dependent-FMA chains per thread,
// the roofline denominator of the walk (which uses no tensor cores).
__global__ void __launch_bounds__(256) k_fma_probe(float* __restrict__ out, int iters, float b, float c) {
  float a[8];
#pragma unroll
  for (int k = 0; k < 8; k++) a[k] = (float)(threadIdx.x + k) * 1e-7f;
  for (int i = 0; i < iters; i++) {
#pragma unroll
    for (int u = 0; u < 16; u++) {
#pragma unroll
      for (int k = 0; k < 8; k++) a[k] = fmaf(a[k], b, c);
    }
  }
  float s = 0.f;
#pragma unroll
  for (int k = 0; k < 8; k++) s += a[k];
  if (s == 1234.5f) out[blockIdx.x] = s;
}

// the same chains as packed pairs (FFMA2: two lanes' worth per instruction)
__global__ void __launch_bounds__(256) k_fma2_probe(float* __restrict__ out, int iters, float b, float c) {
  float2 a[8];
  const float2 b2 = make_float2(b, b), c2 = make_float2(c, c);
#pragma unroll
  for (int k = 0; k < 8; k++) a[k] = make_float2((float)(threadIdx.x + k) * 1e-7f, (float)(threadIdx.x + 2 * k) * 1e-7f);
  for (int i = 0; i < iters; i++) {
#pragma unroll
    for (int u = 0; u < 16; u++) {
#pragma unroll
      for (int k = 0; k < 8; k++) a[k] = __ffma2_rn(a[k], b2, c2);
    }
  }
  float s = 0.f;
#pragma unroll
  for (int k = 0; k < 8; k++) s += a[k].x + a[k].y;
  if (s == 1234.5f) out[blockIdx.x] = s;
}

// FP32 FMA peak: the faster of scalar FFMA and packed FFMA2 chains (the walk
// issues both forms)
double fma_probe_tflops(int nsm, cudaStream_t st, float* scratch) {
  const int iters = 4096, blocks = nsm * 8;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  double best_tf = 0.0;
  for (int packed = 0; packed < 2; packed++) {
    float best = 1e30f;
    for (int r = 0; r < 4; r++) {
      cudaEventRecord(e0, st);
      if (packed) k_fma2_probe<<<blocks, 256, 0, st>>>(scratch, iters, 0.9999999f, 1e-7f);
      else k_fma_probe<<<blocks, 256, 0, st>>>(scratch, iters, 0.9999999f, 1e-7f);
      cudaEventRecord(e1, st);
      cudaEventSynchronize(e1);
      float ms = 0.f;
      cudaEventElapsedTime(&ms, e0, e1);
      if (r > 0 && ms < best) best = ms;
    }
    const double flops = 2.0 * 8 * 16 * (double)iters * blocks * 256 * (packed ? 2 : 1);
    best_tf = std::max(best_tf, flops / (best * 1e-3) / 1e12);
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return best_tf;
}

// The architecture the loaded device code was compiled for (binaryVersion
// 100 = sm_100), read from one of this library's kernels at run time.
int kernel_binary_version(int* binary_version, int* ptx_version) {
  cudaFuncAttributes a;
  const cudaError_t e = cudaFuncGetAttributes(&a, k_fma_probe);
  if (e != cudaSuccess) return -(int)e - 1000;
  *binary_version = a.binaryVersion;
  *ptx_version = a.ptxVersion;
  return 0;
}

// Self-test of the checked build's machinery: index n of a logical length n,
// in a buffer of n + 1 elements (so the write stays inside the allocation in
// every build).  A checked build skips the write and counts it.
__global__ void k_bounds_selftest(int* __restrict__ buf, int n) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    if (BONSAI_IN_RANGE(n, n, 0x7FF)) buf[n] = 1;
  }
}

BONSAI_BOUNDS_ACCESSOR(bounds_word_move)

int bounds_selftest(cudaStream_t s) {
  constexpr int n = 32;
  int* buf = nullptr;
  if (cudaMalloc(&buf, (n + 1) * sizeof(int)) != cudaSuccess) return -1;
  unsigned before[2], after[2];
  int r = -1;
  if (cudaStreamSynchronize(s) == cudaSuccess && bounds_word_move(before, false) == 0) {
    k_bounds_selftest<<<1, 32, 0, s>>>(buf, n);
    if (cudaStreamSynchronize(s) == cudaSuccess && bounds_word_move(after, false) == 0) r = (int)(after[0] - before[0]);
  }
  cudaFree(buf);
  return r;
}

}  // namespace bonsai
