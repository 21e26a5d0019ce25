// keys.cu -- domain box and the two per-particle keys.
//
//  k_box      : one HBM pass, float min/max, last block finalises the Box the
//               way computeBoundingBox does (buildTree.cu:80-166).
//  k_keys     : per particle, in one pass over the positions
//               * tree key: the octant path the reference's recursive
//                 partition gives the particle (Octant/ChildBox,
//                 Particle4.h:129-148, float centres exactly as buildOctant
//                 computes them, buildTree.cu:206-207,237,245);
//               * PH key: makeGroups.cu:108-135 quantisation and the
//                 get_key<21> state machine (makeGroups.cu:19-106), evaluated
//                 through a 48-state x 8-octant table built on the host from
//                 the same rules (build_ph_table).
#include "common.cuh"
#include "kernels.cuh"

namespace bonsai {

// ---------------------------------------------------------------------------
// PH table.  The reference transforms the three quantised coordinates with
// swaps and bitwise complements as it walks the bits (makeGroups.cu:49-81),
// so after any prefix the "current" coordinate k equals original coordinate
// perm[k] xor (all ones if comp[k]).  A state is (perm, comp): 6 x 8 = 48.
// Entry = digit | next_state << 3, indexed by state*8 + original octant bits
// (bx<<2 | by<<1 | bz).
// ---------------------------------------------------------------------------
static const int kPerms[6][3] = {{0, 1, 2}, {0, 2, 1}, {1, 0, 2}, {1, 2, 0}, {2, 0, 1}, {2, 1, 0}};

static int perm_index(const int p[3]) {
  for (int i = 0; i < 6; i++)
    if (kPerms[i][0] == p[0] && kPerms[i][1] == p[1] && kPerms[i][2] == p[2]) return i;
  return -1;
}

void build_ph_table(uint16_t* tab) {
  static const int digit_of[8] = {0, 1, 7, 6, 3, 2, 4, 5};  // makeGroups.cu:28
  for (int pi = 0; pi < 6; pi++)
    for (int c = 0; c < 8; c++)
      for (int o = 0; o < 8; o++) {
        const int b[3] = {(o >> 2) & 1, (o >> 1) & 1, o & 1};
        const int* p = kPerms[pi];
        const int cm[3] = {c & 1, (c >> 1) & 1, (c >> 2) & 1};
        const int t0 = b[p[0]] ^ cm[0], t1 = b[p[1]] ^ cm[1], t2 = b[p[2]] ^ cm[2];
        const int idx = (t0 << 2) | (t1 << 1) | t2;
        int np[3] = {p[0], p[1], p[2]};
        int nc[3] = {cm[0], cm[1], cm[2]};
        if (idx == 0) {                      // swap y,z
          np[1] = p[2]; np[2] = p[1]; nc[1] = cm[2]; nc[2] = cm[1];
        } else if (idx == 1 || idx == 5) {   // swap x,y
          np[0] = p[1]; np[1] = p[0]; nc[0] = cm[1]; nc[1] = cm[0];
        } else if (idx == 4 || idx == 6) {   // complement x,z
          nc[0] ^= 1; nc[2] ^= 1;
        } else if (idx == 3 || idx == 7) {   // x <- ~y, y <- ~x
          np[0] = p[1]; np[1] = p[0]; nc[0] = cm[1] ^ 1; nc[1] = cm[0] ^ 1;
        } else {                             // idx 2: z <- ~y, y <- ~z
          np[1] = p[2]; np[2] = p[1]; nc[1] = cm[2] ^ 1; nc[2] = cm[1] ^ 1;
        }
        const int ns = perm_index(np) * 8 + (nc[0] | (nc[1] << 1) | (nc[2] << 2));
        tab[(pi * 8 + c) * 8 + o] = (uint16_t)(digit_of[idx] | (ns << 3));
      }
}

// ---------------------------------------------------------------------------
// Box: grid-stride min/max, per-block partials, last block folds them.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_box(const float4* __restrict__ pos, int n, float* __restrict__ partial,
                                             unsigned* __restrict__ ticket, Box* __restrict__ box,
                                             int* __restrict__ status) {
  float mn[3] = {1e10f, 1e10f, 1e10f}, mx[3] = {-1e10f, -1e10f, -1e10f};
  bool bad = false;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const float4 p = __ldcs(pos + i);
    bad |= !(isfinite(p.x) && isfinite(p.y) && isfinite(p.z));
    mn[0] = fminf(mn[0], p.x); mn[1] = fminf(mn[1], p.y); mn[2] = fminf(mn[2], p.z);
    mx[0] = fmaxf(mx[0], p.x); mx[1] = fmaxf(mx[1], p.y); mx[2] = fmaxf(mx[2], p.z);
  }
  if (__any_sync(kFull, bad) && lane_id() == 0) set_status(status, kStatusNonFinite);
  __shared__ float sm[6][8];
  __shared__ bool last;
  for (int k = 0; k < 3; k++) {
    const float a = warp_min_f32(mn[k]), b = warp_max_f32(mx[k]);
    if (lane_id() == 0) { sm[k][threadIdx.x >> 5] = a; sm[3 + k][threadIdx.x >> 5] = b; }
  }
  __syncthreads();
  if (threadIdx.x < 32) {
    const int nw = blockDim.x >> 5;
    for (int k = 0; k < 3; k++) {
      const float a = warp_min_f32(threadIdx.x < nw ? sm[k][threadIdx.x] : 1e10f);
      const float b = warp_max_f32(threadIdx.x < nw ? sm[3 + k][threadIdx.x] : -1e10f);
      if (threadIdx.x == 0) { partial[6 * blockIdx.x + k] = a; partial[6 * blockIdx.x + 3 + k] = b; }
    }
    if (threadIdx.x == 0) {
      __threadfence();
      const unsigned t = atomicAdd(ticket, 1u);
      last = (t == gridDim.x - 1);
    }
  }
  __syncthreads();
  if (!last) return;
  if (threadIdx.x < 32) {
    __threadfence();
    float a[3] = {1e10f, 1e10f, 1e10f}, b[3] = {-1e10f, -1e10f, -1e10f};
    for (int j = threadIdx.x; j < (int)gridDim.x; j += 32)
      for (int k = 0; k < 3; k++) {
        a[k] = fminf(a[k], __ldcg(partial + 6 * j + k));
        b[k] = fmaxf(b[k], __ldcg(partial + 6 * j + 3 + k));
      }
    for (int k = 0; k < 3; k++) { a[k] = warp_min_f32(a[k]); b[k] = warp_max_f32(b[k]); }
    if (threadIdx.x == 0) {
      *box = box_from_extent(a, b);
      *ticket = 0u;
    }
  }
}

__device__ __forceinline__ int quantise(float x, float bmin, float inv) {
  // makeGroups.cu:129-131: (x - bmin) * (0.5/hsize) * 2^21, truncated
  return __float2int_rz(__fmul_rn(__fmul_rn(__fsub_rn(x, bmin), inv), 2097152.0f));
}

struct KeyFrame {
  float cx, cy, cz, hsize, inv, bx, by, bz;
};

__device__ __forceinline__ KeyFrame key_frame(const Box b) {
  KeyFrame f;
  f.cx = b.cx; f.cy = b.cy; f.cz = b.cz; f.hsize = b.hsize;
  f.inv = __fdiv_rn(0.5f, b.hsize);
  f.bx = __fsub_rn(b.cx, b.hsize); f.by = __fsub_rn(b.cy, b.hsize); f.bz = __fsub_rn(b.cz, b.hsize);
  return f;
}

__device__ __forceinline__ void particle_keys(const float4 p, const KeyFrame& f, const uint16_t* tab,
                                              unsigned long long& tkey, unsigned long long& pkey) {
  // exact octant path (comparison partition)
  float cx = f.cx, cy = f.cy, cz = f.cz, h = f.hsize;
  unsigned long long tk = 0ull;
#pragma unroll
  for (int L = 0; L < kMaxLevel; L++) {
    const bool ox = cx <= p.x, oy = cy <= p.y, oz = cz <= p.z;
    tk = (tk << 3) | (unsigned long long)((int)ox | ((int)oy << 1) | ((int)oz << 2));
    const float s = __fmul_rn(0.5f, h);
    cx = __fadd_rn(cx, ox ? s : -s);
    cy = __fadd_rn(cy, oy ? s : -s);
    cz = __fadd_rn(cz, oz ? s : -s);
    h = s;
  }
  tkey = tk;
  // Peano-Hilbert key through the state table
  const int qx = quantise(p.x, f.bx, f.inv), qy = quantise(p.y, f.by, f.inv), qz = quantise(p.z, f.bz, f.inv);
  unsigned st = 0;
  unsigned long long pk = 0ull;
#pragma unroll
  for (int L = kMaxLevel - 1; L >= 0; L--) {
    const int o = (((qx >> L) & 1) << 2) | (((qy >> L) & 1) << 1) | ((qz >> L) & 1);
    const unsigned e = tab[st * 8 + o];
    pk = (pk << 3) | (unsigned long long)(e & 7u);
    st = e >> 3;
  }
  pkey = pk;
}

__global__ void __launch_bounds__(256) k_keys(const float4* __restrict__ pos, int n, const Box* __restrict__ boxp,
                                              const uint16_t* __restrict__ ph_table,
                                              unsigned long long* __restrict__ tkey,
                                              unsigned long long* __restrict__ pkey) {
  __shared__ uint16_t tab[384];
  for (int t = threadIdx.x; t < 384; t += blockDim.x) tab[t] = ph_table[t];
  __syncthreads();
  const KeyFrame f = key_frame(*boxp);
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    particle_keys(pos[i], f, tab, tkey[i], pkey[i]);
}

// ---------------------------------------------------------------------------
// Ensembles: every system gets its own box (the same finalisation, so a
// system's box equals the box it gets alone) and its keys are taken in that
// box.  One block per chunk (a chunk never spans two systems).
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_sys_box(const float4* __restrict__ pos, const int4* __restrict__ chunks,
                                                 int nchunks, float* __restrict__ partial,
                                                 int* __restrict__ status) {
  __shared__ float sm[6][8];
  for (int c = blockIdx.x; c < nchunks; c += gridDim.x) {
    const int4 ch = chunks[c];
    float mn[3] = {1e10f, 1e10f, 1e10f}, mx[3] = {-1e10f, -1e10f, -1e10f};
    bool bad = false;
    for (int i = ch.x + threadIdx.x; i < ch.y; i += blockDim.x) {
      const float4 p = __ldcs(pos + i);
      bad |= !(isfinite(p.x) && isfinite(p.y) && isfinite(p.z));
      mn[0] = fminf(mn[0], p.x); mn[1] = fminf(mn[1], p.y); mn[2] = fminf(mn[2], p.z);
      mx[0] = fmaxf(mx[0], p.x); mx[1] = fmaxf(mx[1], p.y); mx[2] = fmaxf(mx[2], p.z);
    }
    if (__any_sync(kFull, bad) && lane_id() == 0) set_status(status, kStatusNonFinite);
    for (int k = 0; k < 3; k++) {
      const float a = warp_min_f32(mn[k]), b = warp_max_f32(mx[k]);
      if (lane_id() == 0) { sm[k][threadIdx.x >> 5] = a; sm[3 + k][threadIdx.x >> 5] = b; }
    }
    __syncthreads();
    if (threadIdx.x < 32) {
      const int nw = blockDim.x >> 5;
      for (int k = 0; k < 3; k++) {
        const float a = warp_min_f32(threadIdx.x < nw ? sm[k][threadIdx.x] : 1e10f);
        const float b = warp_max_f32(threadIdx.x < nw ? sm[3 + k][threadIdx.x] : -1e10f);
        if (threadIdx.x == 0) { partial[6 * c + k] = a; partial[6 * c + 3 + k] = b; }
      }
    }
    __syncthreads();
  }
}

// one warp per system: fold the system's chunk extents, finalise its box
__global__ void __launch_bounds__(256) k_sys_box_final(const float* __restrict__ partial,
                                                       const int* __restrict__ chunk_beg, int nsys,
                                                       Box* __restrict__ boxes) {
  const int lane = threadIdx.x & 31;
  for (int s = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; s < nsys; s += (gridDim.x * blockDim.x) >> 5) {
    float a[3] = {1e10f, 1e10f, 1e10f}, b[3] = {-1e10f, -1e10f, -1e10f};
    for (int c = chunk_beg[s] + lane; c < chunk_beg[s + 1]; c += 32)
      for (int k = 0; k < 3; k++) {
        a[k] = fminf(a[k], partial[6 * c + k]);
        b[k] = fmaxf(b[k], partial[6 * c + 3 + k]);
      }
    for (int k = 0; k < 3; k++) { a[k] = warp_min_f32(a[k]); b[k] = warp_max_f32(b[k]); }
    if (lane == 0) boxes[s] = box_from_extent(a, b);
  }
}

__global__ void __launch_bounds__(256) k_keys_sys(const float4* __restrict__ pos, const int4* __restrict__ chunks,
                                                  int nchunks, const Box* __restrict__ boxes,
                                                  const uint16_t* __restrict__ ph_table,
                                                  unsigned long long* __restrict__ tkey,
                                                  unsigned long long* __restrict__ pkey) {
  __shared__ uint16_t tab[384];
  for (int t = threadIdx.x; t < 384; t += blockDim.x) tab[t] = ph_table[t];
  __syncthreads();
  for (int c = blockIdx.x; c < nchunks; c += gridDim.x) {
    const int4 ch = chunks[c];
    const KeyFrame f = key_frame(boxes[ch.z]);
    for (int i = ch.x + threadIdx.x; i < ch.y; i += blockDim.x) particle_keys(pos[i], f, tab, tkey[i], pkey[i]);
  }
}

void launch_sys_keys(const float4* pos, const int4* chunks, int nchunks, const int* chunk_beg, int nsys,
                     float* box_partial, Box* boxes, const uint16_t* ph_table, unsigned long long* tkey,
                     unsigned long long* pkey, int* status, int nblocks, cudaStream_t s) {
  k_sys_box<<<nblocks, 256, 0, s>>>(pos, chunks, nchunks, box_partial, status);
  k_sys_box_final<<<(nsys + 7) / 8, 256, 0, s>>>(box_partial, chunk_beg, nsys, boxes);
  k_keys_sys<<<nblocks, 256, 0, s>>>(pos, chunks, nchunks, boxes, ph_table, tkey, pkey);
}

}  // namespace bonsai
