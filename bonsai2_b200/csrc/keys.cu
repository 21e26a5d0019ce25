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
//                 through tables built on the host from the same rules
//                 (build_ph_table): 48 states x 8 octants for the top level,
//                 then 48 x 64 for two levels per shared-memory lookup.
//               The kernel is issue-bound (two 21-step chains per particle):
//               two levels per lookup and 32-bit key words took it from
//               0.47 to 0.36 ms at N = 2^24 on one B200.
#include "common.cuh"
#include "kernels.cuh"

namespace bonsai {

// ---------------------------------------------------------------------------
// PH table.  The reference transforms the three quantised coordinates with
// swaps and bitwise complements as it walks the bits (makeGroups.cu:49-81),
// so after any prefix the "current" coordinate k equals original coordinate
// perm[k] xor (all ones if comp[k]).  A state is (perm, comp): 6 x 8 = 48.
// Entry = digit | next_state << 3, indexed by state*8 + original octant bits
// (bx<<2 | by<<1 | bz); a second table composes two levels per lookup.
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
  // two levels per lookup: entry [state * 64 + (ex << 4 | ey << 2 | ez)],
  // e* = the coordinate's bits at levels L (bit 1) and L - 1 (bit 0), holds
  // the two digits (level L's in bits 3..5) and the state after both levels,
  // times 64, in bits 6..11
  uint16_t* tab2 = tab + kPhTable1;
  for (int st = 0; st < 48; st++)
    for (int e = 0; e < 64; e++) {
      const int ex = (e >> 4) & 3, ey = (e >> 2) & 3, ez = e & 3;
      const int ohi = ((ex >> 1) << 2) | ((ey >> 1) << 1) | (ez >> 1);
      const int olo = ((ex & 1) << 2) | ((ey & 1) << 1) | (ez & 1);
      const int e1 = tab[st * 8 + ohi], s1 = e1 >> 3;
      const int e2 = tab[s1 * 8 + olo], s2 = e2 >> 3;
      tab2[st * 64 + e] = (uint16_t)(((e1 & 7) << 3) | (e2 & 7) | (s2 << 6));
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
  // exact octant path (comparison partition); x and y centres advance as one
  // packed add (same rounding as two scalar adds), the 63 key bits are
  // gathered in 32-bit words: levels 0..9 (bits 33..62), 10..19 (3..32), 20
  float2 cxy = make_float2(f.cx, f.cy);
  float cz = f.cz, h = f.hsize;
  unsigned w0 = 0u, w1 = 0u, w2 = 0u;
#pragma unroll
  for (int L = 0; L < kMaxLevel; L++) {
    const bool ox = cxy.x <= p.x, oy = cxy.y <= p.y, oz = cz <= p.z;
    const unsigned o = (unsigned)ox | ((unsigned)oy << 1) | ((unsigned)oz << 2);
    if (L < 10) w0 = w0 * 8u + o;
    else if (L < 20) w1 = w1 * 8u + o;
    else w2 = o;
    const float s = __fmul_rn(0.5f, h);
    cxy = __fadd2_rn(cxy, make_float2(ox ? s : -s, oy ? s : -s));
    cz = __fadd_rn(cz, oz ? s : -s);
    h = s;
  }
  tkey = ((unsigned long long)w0 << 33) | ((unsigned long long)w1 << 3) | w2;
  // Peano-Hilbert key through the state tables: level 20 alone, then the
  // pairs (19, 18) .. (1, 0); digits gathered as level 20 + pairs 1..4
  // (bits 36..62), pairs 5..9 (6..35), pair 10 (0..5)
  const int qx = quantise(p.x, f.bx, f.inv), qy = quantise(p.y, f.by, f.inv), qz = quantise(p.z, f.bz, f.inv);
  const uint16_t* tab2 = tab + kPhTable1;
  const unsigned e0 = tab[(((qx >> 20) & 1) << 2) | (((qy >> 20) & 1) << 1) | ((qz >> 20) & 1)];
  unsigned v0 = e0 & 7u, v1 = 0u, v2 = 0u;
  unsigned st = (e0 >> 3) << 6;
#pragma unroll
  for (int k = 0; k < 10; k++) {
    const int L = 19 - 2 * k;  // this pair's levels L, L - 1
    const unsigned idx = ((unsigned)(qx >> (L - 1)) & 3u) << 4 | ((unsigned)(qy >> (L - 1)) & 3u) << 2 |
                         ((unsigned)(qz >> (L - 1)) & 3u);
    const unsigned e = tab2[st | idx];
    if (k < 4) v0 = (v0 << 6) | (e & 63u);
    else if (k < 9) v1 = (v1 << 6) | (e & 63u);
    else v2 = e & 63u;
    st = e & 0xFC0u;
  }
  pkey = ((unsigned long long)v0 << 36) | ((unsigned long long)v1 << 6) | v2;
}

__global__ void __launch_bounds__(256) k_keys(const float4* __restrict__ pos, int n, const Box* __restrict__ boxp,
                                              const uint16_t* __restrict__ ph_table,
                                              unsigned long long* __restrict__ tkey,
                                              unsigned long long* __restrict__ pkey) {
  __shared__ uint16_t tab[kPhTableSize];
  for (int t = threadIdx.x; t < kPhTableSize; t += blockDim.x) tab[t] = ph_table[t];
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
  __shared__ uint16_t tab[kPhTableSize];
  for (int t = threadIdx.x; t < kPhTableSize; t += blockDim.x) tab[t] = ph_table[t];
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
