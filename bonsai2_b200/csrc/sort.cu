// sort.cu -- stable LSD radix sort of (u64 key, int value) pairs and a
// multi-block exclusive scan.
//
// The reference sorts with Thrust (sort_by_key / stable_sort_by_key,
// makeGroups.cu:270-277, buildTree.cu:940-944): a stable radix sort, ties in
// input order.  This is a hand-written replacement with the same semantics:
// 8 passes of 8 bits; per pass an upsweep (per-tile digit counts), one
// exclusive scan over the digit-major count matrix, and a downsweep that
// ranks every key stably inside its 4096-key tile (warp match_any + per-warp
// digit counters in shared memory) and scatters it.
#include "common.cuh"
#include "kernels.cuh"

namespace bonsai {

constexpr int kSortThreads = 256;
constexpr int kSortItems = 16;
constexpr int kSortTile = kSortThreads * kSortItems;  // 4096
constexpr int kScanChunk = 4096;

int sort_tiles(int n) { return (n + kSortTile - 1) / kSortTile; }

// digit-major count matrix: counts[d * ntiles + tile]
__global__ void __launch_bounds__(kSortThreads) k_sort_upsweep(const unsigned long long* __restrict__ keys, int n,
                                                               int shift, unsigned* __restrict__ counts,
                                                               int ntiles) {
  __shared__ unsigned h[256];
  h[threadIdx.x] = 0;
  __syncthreads();
  const int base = blockIdx.x * kSortTile;
#pragma unroll
  for (int k = 0; k < kSortItems; k++) {
    const int i = base + k * kSortThreads + threadIdx.x;
    if (i < n) {
      const unsigned d = (unsigned)(keys[i] >> shift) & 255u;
      // aggregate equal digits within the warp before the shared atomic
      const unsigned peers = __match_any_sync(__activemask(), d);
      if ((peers & lanemask_lt()) == 0) atomicAdd(&h[d], (unsigned)__popc(peers));
    }
  }
  __syncthreads();
  counts[threadIdx.x * ntiles + blockIdx.x] = h[threadIdx.x];
}

__global__ void __launch_bounds__(kSortThreads) k_sort_downsweep(const unsigned long long* __restrict__ keys_in,
                                                                 const int* __restrict__ vals_in, int n, int shift,
                                                                 const unsigned* __restrict__ offsets, int ntiles,
                                                                 unsigned long long* __restrict__ keys_out,
                                                                 int* __restrict__ vals_out) {
  __shared__ unsigned wcnt[kSortThreads / 32][256];
  __shared__ unsigned gofs[256];
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int t = threadIdx.x; t < (kSortThreads / 32) * 256; t += kSortThreads) (&wcnt[0][0])[t] = 0;
  gofs[threadIdx.x] = offsets[threadIdx.x * ntiles + blockIdx.x];
  __syncthreads();
  // warp-striped ownership: item k of warp w is tile index w*512 + k*32 + lane
  const int base = blockIdx.x * kSortTile + w * (32 * kSortItems);
  unsigned long long key[kSortItems];
  int val[kSortItems];
  unsigned rank[kSortItems];
#pragma unroll
  for (int k = 0; k < kSortItems; k++) {
    const int i = base + k * 32 + lane;
    const bool ok = i < n;
    key[k] = ok ? keys_in[i] : 0ull;
    val[k] = ok ? (vals_in ? vals_in[i] : i) : 0;
    const unsigned d = ok ? ((unsigned)(key[k] >> shift) & 255u) : 256u;
    const unsigned peers = __match_any_sync(kFull, d);
    const unsigned before = (unsigned)__popc(peers & lanemask_lt());
    const unsigned cur = ok ? wcnt[w][d] : 0u;
    rank[k] = cur + before;
    __syncwarp();
    if (ok && before == 0) wcnt[w][d] = cur + (unsigned)__popc(peers);
    __syncwarp();
  }
  __syncthreads();
  {  // exclusive prefix over warps for digit threadIdx.x
    unsigned run = 0;
#pragma unroll
    for (int ww = 0; ww < kSortThreads / 32; ww++) {
      const unsigned c = wcnt[ww][threadIdx.x];
      wcnt[ww][threadIdx.x] = run;
      run += c;
    }
  }
  __syncthreads();
#pragma unroll
  for (int k = 0; k < kSortItems; k++) {
    const int i = base + k * 32 + lane;
    if (i < n) {
      const unsigned d = (unsigned)(key[k] >> shift) & 255u;
      const unsigned o = gofs[d] + wcnt[w][d] + rank[k];
      keys_out[o] = key[k];
      vals_out[o] = val[k];
    }
  }
}

// ---------------------------------------------------------------------------
// exclusive scan of unsigned ints (length m known on the host)
// ---------------------------------------------------------------------------
__device__ __forceinline__ unsigned block_excl_scan(unsigned v, unsigned* sh, unsigned* total) {
  // 256 threads
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  unsigned x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const unsigned t = __shfl_up_sync(kFull, x, o);
    if (lane >= o) x += t;
  }
  if (lane == 31) sh[w] = x;
  __syncthreads();
  if (w == 0) {
    unsigned y = lane < (int)(blockDim.x >> 5) ? sh[lane] : 0u;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const unsigned t = __shfl_up_sync(kFull, y, o);
      if (lane >= o) y += t;
    }
    sh[lane] = y;  // inclusive per-warp totals
  }
  __syncthreads();
  const unsigned wprefix = w ? sh[w - 1] : 0u;
  if (total) *total = sh[(blockDim.x >> 5) - 1];
  __syncthreads();
  return wprefix + x - v;
}

__global__ void __launch_bounds__(256) k_scan_reduce(const unsigned* __restrict__ in, int m,
                                                     unsigned* __restrict__ bsum) {
  __shared__ unsigned sh[32];
  const int b0 = blockIdx.x * kScanChunk;
  unsigned s = 0;
  for (int i = b0 + threadIdx.x; i < min(b0 + kScanChunk, m); i += 256) s += in[i];
  unsigned tot;
  block_excl_scan(s, sh, &tot);
  if (threadIdx.x == 0) bsum[blockIdx.x] = tot;
}

__global__ void __launch_bounds__(256) k_scan_top(unsigned* __restrict__ bsum, int nb, unsigned* __restrict__ total) {
  __shared__ unsigned sh[32];
  unsigned carry = 0;
  for (int b0 = 0; b0 < nb; b0 += 256) {
    const int i = b0 + threadIdx.x;
    const unsigned v = i < nb ? bsum[i] : 0u;
    unsigned tot;
    const unsigned e = block_excl_scan(v, sh, &tot);
    if (i < nb) bsum[i] = carry + e;
    carry += tot;
    __syncthreads();
  }
  if (threadIdx.x == 0 && total) *total = carry;
}

__global__ void __launch_bounds__(256) k_scan_down(const unsigned* __restrict__ in, int m,
                                                   const unsigned* __restrict__ bsum, unsigned* __restrict__ out) {
  __shared__ unsigned sh[32];
  const int b0 = blockIdx.x * kScanChunk;
  // each thread owns 16 consecutive elements of the chunk
  const int i0 = b0 + threadIdx.x * 16;
  unsigned v[16];
  unsigned s = 0;
#pragma unroll
  for (int k = 0; k < 16; k++) {
    v[k] = (i0 + k < m) ? in[i0 + k] : 0u;
    s += v[k];
  }
  unsigned run = block_excl_scan(s, sh, nullptr) + bsum[blockIdx.x];
#pragma unroll
  for (int k = 0; k < 16; k++) {
    if (i0 + k < m) out[i0 + k] = run;
    run += v[k];
  }
}

int scan_blocks(int m) { return (m + kScanChunk - 1) / kScanChunk; }

// out may alias in.  bsum needs scan_blocks(m) entries.
void exclusive_scan(const unsigned* in, unsigned* out, int m, unsigned* bsum, unsigned* total, cudaStream_t s) {
  const int nb = scan_blocks(m);
  if (nb == 0) return;
  k_scan_reduce<<<nb, 256, 0, s>>>(in, m, bsum);
  k_scan_top<<<1, 256, 0, s>>>(bsum, nb, total);
  k_scan_down<<<nb, 256, 0, s>>>(in, m, bsum, out);
}

// Stable sort of n (key, value) pairs; values_in == nullptr means 0..n-1.
// Result ends in (keys_a, vals_a) after the 8 passes (even pass count).
void radix_sort_pairs(unsigned long long* keys_a, unsigned long long* keys_b, int* vals_a, int* vals_b,
                      const int* vals_in, int n, unsigned* counts, unsigned* bsum, int passes, cudaStream_t s) {
  if (n <= 0) return;
  const int nt = sort_tiles(n);
  const int m = 256 * nt;
  unsigned long long* kin = keys_a;
  unsigned long long* kout = keys_b;
  int* vin = vals_a;
  int* vout = vals_b;
  for (int p = 0; p < passes; p++) {
    const int shift = 8 * p;
    k_sort_upsweep<<<nt, kSortThreads, 0, s>>>(kin, n, shift, counts, nt);
    exclusive_scan(counts, counts, m, bsum, nullptr, s);
    k_sort_downsweep<<<nt, kSortThreads, 0, s>>>(kin, p == 0 ? vals_in : vin, n, shift, counts, nt, kout, vout);
    unsigned long long* tk = kin; kin = kout; kout = tk;
    int* tv = vin; vin = vout; vout = tv;
  }
}

}  // namespace bonsai
