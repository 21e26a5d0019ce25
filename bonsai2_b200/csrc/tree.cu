// tree.cu -- octree from the sorted octant-path keys, in three launches and no
// host round trip.
//
// The reference builds the tree by a recursive CUDA-dynamic-parallelism
// partition (buildOctant, buildTree.cu:170-722) and then stable-sorts the
// cells by level (buildTree.cu:725-841,932-958).  Its cell set is defined by
// two rules: the root is always split, and a cell with more than nLeaf
// particles is split (buildTree.cu:394-395,444,541).  With particles sorted
// by the octant path, every cell at level L is a maximal run of equal
// 3L-bit key prefix, so the cell set follows from d(i), the level at which
// keys i-1 and i first differ:
//   * with m(i) = min d(i+1..i+nLeaf) (d = 0 past the end), the level-L run
//     starting at i holds more than nLeaf particles iff d(i) <= L < m(i);
//     all of those runs are nodes, and the chain of cells that start at i
//     runs from max(d(i),1) down to the first level whose run is small
//     (a leaf), or to level 21 (a fat leaf, flagged);
//   * a small run starting at i at level d(i) >= 2 is a leaf iff its parent
//     run (level d(i)-1) holds more than nLeaf particles, which is decided
//     from d inside the window i-nLeaf .. i+nLeaf.
// Launch 1 computes the chains of a 4096-position tile (halo nLeaf) and a
// per-level histogram; launch 2 scans the histograms (one block); launch 3
// writes the cells level-major, key order inside a level (the canonical form
// of the reference's cell order), with children contiguous, the leaf list,
// parent links (a cell's parent is the last cell of the level above that
// starts at or before it, counted from the same prefix sums) and the level
// ranges; then one short launch per level, from the top, gives every cell its
// run end (its next sibling's start, or its parent's end for a last child)
// and every node its child count -- no searches over the keys.
#include "common.cuh"
#include "kernels.cuh"

namespace bonsai {

constexpr int kTreeThreads = 256;
constexpr int kTreeItems = 16;
constexpr int kTreeTile = kTreeThreads * kTreeItems;  // 4096
constexpr int kHalo = 64;                              // max nLeaf
constexpr int kNL = kMaxLevel + 1;                     // rows 0..21 (row 0 unused)

int tree_tiles(int n) { return (n + kTreeTile - 1) / kTreeTile; }

struct Chain {
  int a, b;  // levels [a, b]; a == 0: no cell starts here
};

constexpr int kLen = kTreeTile + 2 * kHalo;  // positions of a tile with its halo

// sd[loc + j] = d(i + j) for j in [-kHalo, kHalo] (0 past n); W[k - 1][x] =
// min of sd over [x, x + 2^k) for 2^k <= wp, wp the largest power of two <=
// nleaf (0 where the window leaves the tile), so that
// m(i) = min d(i+1 .. i+nleaf) = min(W[K][loc + 1], W[K][loc + 1 + nleaf - wp]).
__device__ __forceinline__ uint8_t wmin(const uint8_t* sd, const uint8_t* W, int k, int x) {
  return k == 0 ? sd[x] : W[(k - 1) * kLen + x];
}
__device__ __forceinline__ Chain make_chain(const uint8_t* sd, const uint8_t* W, int K, int wp, int loc, int i, int n,
                                            int nleaf, bool* fat) {
  Chain c{0, 0};
  const int di = (i == 0) ? 0 : (int)sd[loc];
  const int ls = max(di, 1);
  if (ls > kMaxLevel) return c;
  const int m = K == 0 ? min((int)sd[loc + 1], (int)sd[loc + 1 + nleaf - wp])
                       : min((int)W[(K - 1) * kLen + loc + 1], (int)W[(K - 1) * kLen + loc + 1 + nleaf - wp]);
  if (ls < m) {
    c.a = ls;
    c.b = min(m, kMaxLevel);
    *fat = (m > kMaxLevel);
    return c;
  }
  if (ls == 1) {
    c.a = c.b = 1;
    return c;
  }
  // the parent run at level ls-1 containing i is [p, e): p the nearest
  // position <= i - 1 with d <= ls-1 (d = 0 at and before position 0), e the
  // nearest position >= i + 1 with d <= ls-1 (d = 0 at and past n), each
  // looked for within nleaf positions by binary lifting over the window
  // minima; the small run starting here is a leaf iff the parent holds more
  // than nleaf particles (or a bound is not found within nleaf)
  const int l1 = ls - 1;
  int xb = loc;  // [xb, loc - 1] all > l1
  for (int k = K; k >= 0; k--) {
    const int st = 1 << k;
    if (xb - st >= loc - nleaf && (int)wmin(sd, W, k, xb - st) > l1) xb -= st;
  }
  int xf = loc + 1;  // [loc + 1, xf - 1] all > l1
  for (int k = K; k >= 0; k--) {
    const int st = 1 << k;
    if (xf + st - 1 <= loc + nleaf && (int)wmin(sd, W, k, xf) > l1) xf += st;
  }
  const bool found = xb > loc - nleaf && xf <= loc + nleaf;
  // p = i - (loc - xb + 1), e = i + (xf - loc): e - p = xf - xb + 1
  if (!found || xf - xb + 1 > nleaf) c.a = c.b = ls;
  return c;
}

// Loads d for positions [t0-kHalo, t0+kTreeTile+kHalo) into sd, from keys.
// In an ensemble d = 0 at every system start: a system's first particle
// starts a level-1 cell, and no run crosses into the next system (the same
// values d takes at 0 and past n when the system is alone).
__device__ void load_d_from_keys(const unsigned long long* __restrict__ keys, int n, int t0, uint8_t* sd,
                                 unsigned long long* sk, const int* __restrict__ sys_off, int nsys) {
  const int nk = kTreeTile + 2 * kHalo + 1;
  for (int j = threadIdx.x; j < nk; j += blockDim.x) {
    const int g = t0 - kHalo - 1 + j;
    sk[j] = (g >= 0 && g < n) ? keys[g] : 0ull;
  }
  __syncthreads();
  for (int j = threadIdx.x; j < kTreeTile + 2 * kHalo; j += blockDim.x) {
    const int p = t0 - kHalo + j;
    sd[j] = (p <= 0 || p >= n) ? (uint8_t)0 : (uint8_t)diff_level(sk[j], sk[j + 1]);
  }
  __syncthreads();
  if (nsys > 1) {
    const int lo = t0 - kHalo, hi = t0 + kTreeTile + kHalo;
    // systems whose start lies in [lo, hi): few per tile
    if (threadIdx.x == 0) {
      for (int s = sys_of(sys_off, nsys, max(lo, 0)); s < nsys; s++) {
        const int p = sys_off[s];
        if (p >= hi) break;
        if (p >= lo) sd[p - lo] = 0;
      }
    }
    __syncthreads();
  }
}

__global__ void __launch_bounds__(kTreeThreads) k_tree_chains(const unsigned long long* __restrict__ keys, int n,
                                                              int nleaf, uint8_t* __restrict__ dlev,
                                                              uint16_t* __restrict__ chain,
                                                              unsigned* __restrict__ hist, int nb,
                                                              int* __restrict__ status,
                                                              const int* __restrict__ sys_off, int nsys) {
  __shared__ unsigned long long sk[kTreeTile + 2 * kHalo + 1];
  __shared__ uint8_t sd[kTreeTile + 2 * kHalo];
  __shared__ unsigned hc[kNL], hl[kNL];
  const int t0 = blockIdx.x * kTreeTile;
  if (threadIdx.x < kNL) { hc[threadIdx.x] = 0; hl[threadIdx.x] = 0; }
  load_d_from_keys(keys, n, t0, sd, sk, sys_off, nsys);
  for (int j = threadIdx.x; j < kTreeTile; j += blockDim.x)
    if (t0 + j < n) dlev[t0 + j] = sd[kHalo + j];
  // window minima of d by doubling, every level kept (W[k-1]: windows of
  // 2^k), in the key buffer's space (no longer read)
  uint8_t* W = reinterpret_cast<uint8_t*>(sk);
  int wp = 1, K = 0;
  for (; 2 * wp <= nleaf; wp *= 2, K++) {
    const uint8_t* prev = K == 0 ? sd : W + (K - 1) * kLen;
    uint8_t* out = W + K * kLen;
    for (int j = threadIdx.x; j < kLen; j += blockDim.x) out[j] = min(prev[j], j + wp < kLen ? prev[j + wp] : (uint8_t)0);
    __syncthreads();
  }
  bool anyfat = false;
  const int i0 = t0 + threadIdx.x * kTreeItems;
#pragma unroll 1
  for (int k = 0; k < kTreeItems; k++) {
    const int i = i0 + k;
    if (i >= n) break;
    bool fat = false;
    const Chain c = make_chain(sd, W, K, wp, kHalo + (i - t0), i, n, nleaf, &fat);
    anyfat |= fat;
    chain[i] = (uint16_t)(c.a | (c.b << 8));
    if (c.a) {
      for (int L = c.a; L <= c.b; L++) atomicAdd(&hc[L], 1u);
      atomicAdd(&hl[c.b], 1u);
    }
  }
  if (__any_sync(kFull, anyfat) && lane_id() == 0) set_status(status, kStatusDepth);
  __syncthreads();
  if (threadIdx.x < kNL) {
    hist[threadIdx.x * nb + blockIdx.x] = hc[threadIdx.x];
    hist[(kNL + threadIdx.x) * nb + blockIdx.x] = hl[threadIdx.x];
  }
}

// One block: exclusive scan of each histogram row across tiles, rows chained
// so that offsets are global (cells level-major; leaves ordered likewise).
// The rows are independent once their totals are known: each warp sums its
// rows, one thread chains the row totals into row bases (and fills the tree
// info), then each warp scans its rows, four entries per lane per step.
__global__ void __launch_bounds__(1024) k_tree_scan(unsigned* __restrict__ hist, int nb, int cell_cap,
                                                    int leaf_cap, int n, TreeInfo* __restrict__ info) {
  __shared__ unsigned rowtot[2 * kNL], rowbase[2 * kNL];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int row = w; row < 2 * kNL; row += nw) {
    const unsigned* h = hist + (size_t)row * nb;
    unsigned sum = 0;
    if (row % kNL > 0)
      for (int b = lane; b < nb; b += 32) sum += h[b];
#pragma unroll
    for (int o = 16; o; o >>= 1) sum += __shfl_xor_sync(kFull, sum, o);
    if (lane == 0) rowtot[row] = sum;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned tc = 0, tl = 0;
    int nlevels = 0;
    for (int L = 0; L < kNL; L++) {
      rowbase[L] = tc;
      info->level_beg[L] = (int)tc;
      if (L > 0 && rowtot[L] > 0) nlevels = L;
      tc += rowtot[L];
      info->level_end[L] = (int)tc;
    }
    for (int L = 0; L < kNL; L++) {
      rowbase[kNL + L] = tl;
      tl += rowtot[kNL + L];
    }
    for (int L = kNL; L < kLevels; L++) info->level_beg[L] = info->level_end[L] = (int)tc;
    info->ncells = (int)tc;
    info->nleaves = (int)tl;
    info->nnodes = (int)(tc - tl);
    info->nlevels = nlevels;
    info->npart = n;
    if ((int)tc > cell_cap || (int)tl > leaf_cap) set_status(&info->status, kStatusCellCapacity);
  }
  __syncthreads();
  for (int row = w; row < 2 * kNL; row += nw) {
    unsigned* h = hist + (size_t)row * nb;
    const bool live = row % kNL > 0;
    unsigned carry = rowbase[row];
    for (int b0 = 0; b0 < nb; b0 += 128) {
      const int b = b0 + 4 * lane;
      unsigned v[4], s = 0;
#pragma unroll
      for (int q = 0; q < 4; q++) {
        v[q] = (live && b + q < nb) ? h[b + q] : 0u;
        s += v[q];
      }
      const unsigned incl = (unsigned)warp_incl_scan((int)s);
      unsigned run = carry + incl - s;
#pragma unroll
      for (int q = 0; q < 4; q++) {
        if (b + q < nb) h[b + q] = run;
        run += v[q];
      }
      carry += __shfl_sync(kFull, incl, 31);
    }
  }
}

__global__ void __launch_bounds__(kTreeThreads) k_tree_cells(
    const unsigned long long* __restrict__ keys, const uint8_t* __restrict__ dlev,
    const uint16_t* __restrict__ chain, const unsigned* __restrict__ hist, int n, int nleaf, int nb, int cell_cap,
    TreeInfo* __restrict__ info, uint4* __restrict__ cell_data, int* __restrict__ cell_parent,
    int* __restrict__ leaf_list, int* __restrict__ mp_count, const int* __restrict__ sys_off, int nsys,
    int* __restrict__ root_beg) {
  __shared__ uint8_t sd[kTreeTile + 2 * kHalo];
  __shared__ uint16_t cpre[kNL][kTreeThreads];
  __shared__ uint16_t lpre[kNL][kTreeThreads];
  __shared__ unsigned boff[2][kNL];
  if (info->ncells > cell_cap || info->nleaves > cell_cap) return;
  [[maybe_unused]] const int ncells = info->ncells, nleaves = info->nleaves;
  if (nsys > 1 && blockIdx.x == 0 && threadIdx.x == 0) root_beg[nsys] = info->level_end[1];
  const int t0 = blockIdx.x * kTreeTile;
  for (int j = threadIdx.x; j < kTreeTile + 2 * kHalo; j += blockDim.x) {
    const int p = t0 - kHalo + j;
    sd[j] = (p <= 0 || p >= n) ? (uint8_t)0 : dlev[p];
  }
  if (threadIdx.x < kNL) {
    boff[0][threadIdx.x] = hist[threadIdx.x * nb + blockIdx.x];
    boff[1][threadIdx.x] = hist[(kNL + threadIdx.x) * nb + blockIdx.x];
  }
  const int i0 = t0 + threadIdx.x * kTreeItems;
  // per-thread totals per level (cells of the thread's chains; leaves)
  for (int L = 0; L < kNL; L++) {
    cpre[L][threadIdx.x] = 0;
    lpre[L][threadIdx.x] = 0;
  }
#pragma unroll 4
  for (int k = 0; k < kTreeItems; k++) {
    const int i = i0 + k;
    const unsigned c = (i < n) ? (unsigned)chain[i] : 0u;
    const int a = (int)(c & 255u), b = (int)(c >> 8);
    if (!a) continue;
    for (int L = a; L <= b; L++) cpre[L][threadIdx.x]++;
    lpre[b][threadIdx.x]++;
  }
  __syncthreads();
  // exclusive scans of the 2*kNL rows over the 256 threads (one warp per row)
  {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int row = w; row < 2 * kNL; row += kTreeThreads / 32) {
      uint16_t* r = (row < kNL) ? cpre[row] : lpre[row - kNL];
      unsigned v[8], s = 0;
#pragma unroll
      for (int q = 0; q < 8; q++) { v[q] = r[lane * 8 + q]; s += v[q]; }
      const unsigned incl = (unsigned)warp_incl_scan((int)s);
      unsigned run = incl - s;
#pragma unroll
      for (int q = 0; q < 8; q++) { r[lane * 8 + q] = (uint16_t)run; run += v[q]; }
    }
  }
  __syncthreads();
  // cpre[L][t] / lpre[L][t] now hold the thread's first cell / leaf slot at
  // level L (relative to the level's block offset) and advance as its items
  // are written: an item's cells and links read them before it adds its own
#pragma unroll 1
  for (int k = 0; k < kTreeItems; k++) {
    const int i = i0 + k;
    if (i >= n) break;
    const unsigned c = (unsigned)chain[i];  // (the thread's 32 bytes of chain words, cached)
    const int a = (int)(c & 255u), b = (int)(c >> 8);
    if (!a) continue;
    const int loc = kHalo + (i - t0);
    {
      const int leaf_idx = (int)(boff[1][b] + lpre[b][threadIdx.x]);
      if (BONSAI_IN_RANGE(leaf_idx, nleaves, 0x101)) leaf_list[leaf_idx] = (int)(boff[0][b] + cpre[b][threadIdx.x]);
    }
    for (int L = a; L <= b; L++) {
      const int cidx = (int)(boff[0][L] + cpre[L][threadIdx.x]);
      if (!BONSAI_IN_RANGE(cidx, ncells, 0x102)) continue;
      const bool leaf = (L == b);
      uint4 cd;
      int parent = -1;
      if (L == 1) {
        cd.x = (unsigned)(1 << 27);  // level-1 cells: parent 0, as the reference stores them
        // a system's first level-1 cell starts at the system's first particle
        if (nsys > 1 && sd[loc] == 0) root_beg[sys_of(sys_off, nsys, i)] = cidx;
      } else {
        // the parent is the last level-(L-1) cell starting at or before i:
        // the one starting at i when the chain here covers level L-1, else
        // the one before the first level-(L-1) cell that starts after i
        parent = (int)(boff[0][L - 1] + cpre[L - 1][threadIdx.x]) - (a <= L - 1 ? 0 : 1);
        cd.x = (unsigned)parent | ((unsigned)L << 27);
      }
      // nodes: the first child (children are contiguous at level L + 1); the
      // child count and every cell's run end follow in the level passes
      cd.y = leaf ? 0xFFFFFFFFu : (unsigned)((int)(boff[0][L + 1] + cpre[L + 1][threadIdx.x]));
      cd.z = (unsigned)i;
      cd.w = (unsigned)i;
      cell_data[cidx] = cd;
      cell_parent[cidx] = parent;
      mp_count[cidx] = 0;
    }
    for (int L = a; L <= b; L++) cpre[L][threadIdx.x]++;
    lpre[b][threadIdx.x]++;
  }
}

// Run ends and child counts, level by level from the top.  A cell's run ends
// where its next sibling starts (the next cell of the level with the same
// parent) or, for a last child, where its parent's run ends; the last child
// of a node writes the node's child count.  Level-1 cells partition their
// system: a run ends at the next level-1 cell's start (the next system's
// first particle for a system's last cell) or at n.
__global__ void __launch_bounds__(kTreeThreads) k_tree_pass(int L, const TreeInfo* __restrict__ info,
                                                            uint4* __restrict__ cell_data,
                                                            const int* __restrict__ cell_parent, int n,
                                                            int cell_cap) {
  if (info->ncells > cell_cap || info->nleaves > cell_cap) return;
  [[maybe_unused]] const int ncells = info->ncells;
  const int b = info->level_beg[L], e = info->level_end[L];
  for (int c = b + blockIdx.x * blockDim.x + threadIdx.x; c < e; c += gridDim.x * blockDim.x) {
    const bool more = c + 1 < e;
    int pend;
    if (L == 1) {
      pend = more ? (int)cell_data[c + 1].z : n;
    } else {
      const int par = cell_parent[c];
      if (!BONSAI_IN_RANGE(par, ncells, 0x107)) continue;
      const bool sib = more && cell_parent[c + 1] == par;
      pend = sib ? (int)cell_data[c + 1].z : (int)cell_data[par].w;
      if (!sib) {
        const unsigned first = cell_data[par].y & 0x1FFFFFFFu;
        cell_data[par].y = first | ((unsigned)(c - (int)first) << 29);
      }
    }
    const int i = (int)cell_data[c].z;
    if (!BONSAI_IN_RANGE(pend - 1, n, 0x104) || !BONSAI_IN_RANGE(i, pend, 0x105)) pend = min(max(pend, i + 1), n);
    cell_data[c].w = (unsigned)pend;
  }
}

void build_tree(const unsigned long long* sorted_keys, int n, int nleaf, int cell_cap, int leaf_cap,
                uint8_t* dlev, uint16_t* chain, unsigned* hist, TreeInfo* info, uint4* cell_data,
                int* cell_parent, int* leaf_list, int* mp_count, const int* sys_off, int nsys, int* root_beg,
                cudaStream_t s) {
  const int nb = tree_tiles(n);
  k_tree_chains<<<nb, kTreeThreads, 0, s>>>(sorted_keys, n, nleaf, dlev, chain, hist, nb, &info->status, sys_off,
                                            nsys);
  k_tree_scan<<<1, 1024, 0, s>>>(hist, nb, cell_cap, leaf_cap, n, info);
  k_tree_cells<<<nb, kTreeThreads, 0, s>>>(sorted_keys, dlev, chain, hist, n, nleaf, nb, cell_cap, info, cell_data,
                                           cell_parent, leaf_list, mp_count, sys_off, nsys, root_beg);
  const int pb = nb < 512 ? nb : 512;
  for (int L = 1; L <= kMaxLevel; L++)
    k_tree_pass<<<pb, kTreeThreads, 0, s>>>(L, info, cell_data, cell_parent, n, cell_cap);
}

BONSAI_BOUNDS_ACCESSOR(bounds_word_tree)

}  // namespace bonsai
