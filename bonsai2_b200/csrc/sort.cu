// sort.cu -- stable LSD radix sort of (u64 key, int value) pairs and a
// multi-block exclusive scan.
//
// The reference sorts with Thrust (sort_by_key / stable_sort_by_key,
// makeGroups.cu:270-277, buildTree.cu:940-944): a stable radix sort, ties in
// input order.  This is a hand-written replacement with the same semantics:
// 8 passes of 8 bits, one-sweep (below): keys are ranked stably inside each
// 4096-key tile (the lanes of equal digit from bit ballots) with per-warp
// digit counters in shared memory, tile offsets come from a decoupled look-back, and tiles are written
// out through shared memory in contiguous digit runs.  A thread keeps only the
// 16 ranks and packed digits of its keys across the look-back (the keys are
// re-read from L2 for staging): 4 blocks per SM (keeping the keys, 127
// registers and 2 blocks per SM, was 16 % slower per sort than 3 blocks).
#include "common.cuh"
#include "kernels.cuh"

namespace bonsai {

constexpr int kSortThreads = 256;
constexpr int kSortItems = 16;
constexpr int kSortTile = kSortThreads * kSortItems;  // 4096
constexpr int kScanChunk = 4096;

int sort_tiles(int n) { return (n + kSortTile - 1) / kSortTile; }

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

// ---------------------------------------------------------------------------
// One-sweep passes.  One kernel reads the keys once and builds the digit
// histograms of all eight passes; one kernel per pass then ranks each
// 4096-key tile (same stable warp ranking as above), obtains the tile's
// global offset per digit by decoupled look-back over the preceding tiles
// (tiles take ids in launch order from an atomic counter, so a tile only waits
// for tiles that already run; every wait is bounded and sets an error flag
// when the bound is hit), stages the tile in shared memory in digit order and
// writes it out in contiguous runs.  One read and one write of the pairs per
// pass.
// ---------------------------------------------------------------------------
// blocks per SM of the one-sweep pass: the pass is latency-bound, and 4 blocks
// (64 registers, a 40-byte spill) beat 3 (80 registers): build phase at
// N = 2^24 4.49 against 4.71 ms
#ifndef BONSAI_SORT_MINB
#define BONSAI_SORT_MINB 4
#endif
constexpr unsigned kFlagAgg = 1u << 30, kFlagInc = 2u << 30, kValMask = (1u << 30) - 1u;

// The lanes holding the same digit (0..256, 256 = no key): the intersection
// of nine bit ballots (BONSAI_SORT_BALLOT_MATCH, the default), or
// __match_any_sync, which was slower on the B200 (PH sort + group formation at
// N = 2^24: 1.82 against 1.93 ms).  Issuing all items' ballots before the
// chain through the warp's counters was measured no faster.
#ifndef BONSAI_SORT_BALLOT_MATCH
#define BONSAI_SORT_BALLOT_MATCH 1
#endif
__device__ __forceinline__ unsigned digit_peers(unsigned d) {
#if BONSAI_SORT_BALLOT_MATCH
  unsigned m = kFull;
#pragma unroll
  for (int b = 0; b < 9; b++) {
    const unsigned bal = __ballot_sync(kFull, (d >> b) & 1u);
    m &= ((d >> b) & 1u) ? bal : ~bal;
  }
  return m;
#else
  return __match_any_sync(kFull, d);
#endif
}
constexpr int kLookbackSpin = 1 << 22;

__global__ void __launch_bounds__(kSortThreads) k_sort_hist8(const unsigned long long* __restrict__ keys, int n,
                                                             int passes, unsigned* __restrict__ ghist) {
  __shared__ unsigned h[8][256];
  for (int t = threadIdx.x; t < 8 * 256; t += kSortThreads) (&h[0][0])[t] = 0;
  __syncthreads();
  for (int i = blockIdx.x * kSortThreads + threadIdx.x; i < n; i += gridDim.x * kSortThreads) {
    const unsigned long long k = keys[i];
#pragma unroll
    for (int p = 0; p < 8; p++)
      if (p < passes) atomicAdd(&h[p][(unsigned)(k >> (8 * p)) & 255u], 1u);
  }
  __syncthreads();
  for (int t = threadIdx.x; t < passes * 256; t += kSortThreads) {
    const unsigned v = (&h[0][0])[t];
    if (v) atomicAdd(ghist + t, v);
  }
}

// exclusive scan of each 256-entry row in place (one block, 256 threads)
__global__ void __launch_bounds__(256) k_sort_hist_scan(unsigned* __restrict__ ghist, int passes) {
  __shared__ unsigned sh[32];
  for (int p = 0; p < passes; p++) {
    const unsigned v = ghist[p * 256 + threadIdx.x];
    const unsigned e = block_excl_scan(v, sh, nullptr);
    ghist[p * 256 + threadIdx.x] = e;
    __syncthreads();
  }
}

// SYSD: the digit is a byte of the element's system index (sys_of of its
// value, the element's position in the sort's input order), not of its key:
// the passes that make an ensemble sort stable-partition by system last.
template <bool SYSD>
__global__ void __launch_bounds__(kSortThreads, BONSAI_SORT_MINB) k_sort_onesweep(
    const unsigned long long* __restrict__ keys_in, const int* __restrict__ vals_in, int n, int shift,
    const unsigned* __restrict__ gbase, unsigned* __restrict__ status, unsigned* __restrict__ tile_counter,
    unsigned long long* __restrict__ keys_out, int* __restrict__ vals_out, int* __restrict__ err,
    const int* __restrict__ sys_off, int nsys) {
  __shared__ unsigned wcnt[kSortThreads / 32][256];
  __shared__ unsigned tile_off[256];
  __shared__ unsigned dstart[256];
  __shared__ unsigned long long stage[kSortTile];  // keys, then values (as 32-bit) in digit order
  __shared__ unsigned char sdig[kSortTile];
  __shared__ unsigned sh[32];
  __shared__ int tile_sh;
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) tile_sh = (int)atomicAdd(tile_counter, 1u);
  for (int t = threadIdx.x; t < (kSortThreads / 32) * 256; t += kSortThreads) (&wcnt[0][0])[t] = 0;
  __syncthreads();
  const int tile = tile_sh;
  const int base = tile * kSortTile + w * (32 * kSortItems);
  unsigned rank[kSortItems];
  unsigned dpack[kSortItems / 4];
#pragma unroll
  for (int k = 0; k < kSortItems; k++) {
    const int i = base + k * 32 + lane;
    const bool ok = i < n;
    unsigned d;
    if constexpr (SYSD) {
      d = ok ? (((unsigned)sys_of(sys_off, nsys, vals_in ? vals_in[i] : i) >> shift) & 255u) : 256u;
    } else {
      d = ok ? ((unsigned)(keys_in[i] >> shift) & 255u) : 256u;
    }
    if ((k & 3) == 0) dpack[k >> 2] = 0u;
    dpack[k >> 2] |= (d & 255u) << (8 * (k & 3));
    const unsigned peers = digit_peers(d);
    const unsigned before = (unsigned)__popc(peers & lanemask_lt());
    const unsigned cur = ok ? wcnt[w][d] : 0u;
    rank[k] = cur + before;
    __syncwarp();
    if (ok && before == 0) wcnt[w][d] = cur + (unsigned)__popc(peers);
    __syncwarp();
  }
  __syncthreads();
  // per digit: prefix over warps, tile total, tile-local digit offsets
  const unsigned d = threadIdx.x;
  unsigned tot = 0;
#pragma unroll
  for (int ww = 0; ww < kSortThreads / 32; ww++) {
    const unsigned c = wcnt[ww][d];
    wcnt[ww][d] = tot;
    tot += c;
  }
  tile_off[d] = block_excl_scan(tot, sh, nullptr);
  // decoupled look-back for the digit's global offset
  volatile unsigned* st = status;
  if (tile == 0) {
    st[d] = kFlagInc | tot;
    dstart[d] = gbase[d];
  } else {
    st[(size_t)tile * 256 + d] = kFlagAgg | tot;
    unsigned excl = 0;
    for (int t = tile - 1; t >= 0; t--) {
      unsigned v = st[(size_t)t * 256 + d];
      int spin = 0;
      while ((v & ~kValMask) == 0u && spin < kLookbackSpin) {
        __nanosleep(32);
        v = st[(size_t)t * 256 + d];
        spin++;
      }
      if ((v & ~kValMask) == 0u) {  // bound hit: report and give up (results invalid)
        atomicOr(err, kStatusSortTimeout);
        break;
      }
      excl += v & kValMask;
      if ((v & ~kValMask) == kFlagInc) break;
    }
    st[(size_t)tile * 256 + d] = kFlagInc | (excl + tot);
    dstart[d] = gbase[d] + excl;
  }
  __syncthreads();
  // stage keys in digit order (re-read from L2), write contiguous runs
  const int tile_n = min(kSortTile, n - tile * kSortTile);
  unsigned lpos[kSortItems];
#pragma unroll
  for (int k = 0; k < kSortItems; k++) {
    const int i = base + k * 32 + lane;
    if (i < n) {
      const unsigned dd = (dpack[k >> 2] >> (8 * (k & 3))) & 255u;
      lpos[k] = tile_off[dd] + wcnt[w][dd] + rank[k];
      stage[lpos[k]] = keys_in[i];
      sdig[lpos[k]] = (unsigned char)dd;
    }
  }
  __syncthreads();
  for (int j = threadIdx.x; j < tile_n; j += kSortThreads) {
    const unsigned long long kk = stage[j];
    const unsigned dd = sdig[j];
    const unsigned dst = dstart[dd] + (unsigned)j - tile_off[dd];
    if (BONSAI_IN_RANGE(dst, n, 0x601)) keys_out[dst] = kk;
  }
  __syncthreads();
  unsigned* stage32 = reinterpret_cast<unsigned*>(stage);
#pragma unroll
  for (int k = 0; k < kSortItems; k++) {
    const int i = base + k * 32 + lane;
    if (i < n) stage32[lpos[k]] = (unsigned)(vals_in ? vals_in[i] : i);
  }
  __syncthreads();
  for (int j = threadIdx.x; j < tile_n; j += kSortThreads) {
    const unsigned dd = sdig[j];
    const unsigned dst = dstart[dd] + (unsigned)j - tile_off[dd];
    if (BONSAI_IN_RANGE(dst, n, 0x602)) vals_out[dst] = (int)stage32[j];
  }
}

// digit histograms of the two system-index passes, from the system sizes
__global__ void __launch_bounds__(256) k_sort_hist_sys(const int* __restrict__ sys_off, int nsys,
                                                       unsigned* __restrict__ ghist) {
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < nsys; s += gridDim.x * blockDim.x) {
    const unsigned c = (unsigned)(sys_off[s + 1] - sys_off[s]);
    atomicAdd(ghist + (s & 255), c);
    atomicAdd(ghist + 256 + ((s >> 8) & 255), c);
  }
}

constexpr int kMaxPasses = 10;  // 8 key bytes + 2 system-index bytes

size_t sort_status_words(int n) { return (size_t)sort_tiles(n) * 256 * kMaxPasses + kMaxPasses + kMaxPasses * 256; }

// Stable sort of n (key, value) pairs; values_in == nullptr means 0..n-1.
// Result ends in (keys_a, vals_a) after an even number of passes.  work holds
// sort_status_words(n) unsigned ints: look-back status of every pass, the
// tile counters and the digit histograms; kStatusSortTimeout is or-ed into
// *err if a look-back wait hit its bound.  With nsys > 1 (an ensemble laid
// out as sys_off), two more passes order by system index, so each system's
// pairs are sorted by key within the system's own index range, ties in input
// order: the order each system gets when sorted alone.
void radix_sort_pairs(unsigned long long* keys_a, unsigned long long* keys_b, int* vals_a, int* vals_b,
                      const int* vals_in, int n, unsigned* work, int* err, int passes, const int* sys_off, int nsys,
                      cudaStream_t s) {
  if (n <= 0) return;
  const int nt = sort_tiles(n);
  const int sys_passes = nsys > 1 ? 2 : 0;
  unsigned* status = work;
  unsigned* counters = work + (size_t)nt * 256 * kMaxPasses;
  unsigned* ghist = counters + kMaxPasses;
  cudaMemsetAsync(work, 0, sort_status_words(n) * sizeof(unsigned), s);
  k_sort_hist8<<<1184, kSortThreads, 0, s>>>(keys_a, n, passes, ghist);
  if (sys_passes) k_sort_hist_sys<<<(nsys + 255) / 256, 256, 0, s>>>(sys_off, nsys, ghist + 256 * passes);
  k_sort_hist_scan<<<1, 256, 0, s>>>(ghist, passes + sys_passes);
  unsigned long long* kin = keys_a;
  unsigned long long* kout = keys_b;
  int* vin = vals_a;
  int* vout = vals_b;
  for (int p = 0; p < passes + sys_passes; p++) {
    const int* vi = p == 0 ? vals_in : vin;
    unsigned* stp = status + (size_t)p * nt * 256;
    if (p < passes)
      k_sort_onesweep<false><<<nt, kSortThreads, 0, s>>>(kin, vi, n, 8 * p, ghist + 256 * p, stp, counters + p, kout,
                                                         vout, err, nullptr, 0);
    else
      k_sort_onesweep<true><<<nt, kSortThreads, 0, s>>>(kin, vi, n, 8 * (p - passes), ghist + 256 * p, stp,
                                                        counters + p, kout, vout, err, sys_off, nsys);
    unsigned long long* tk = kin; kin = kout; kout = tk;
    int* tv = vin; vin = vout; vout = tv;
  }
}

// Self-test of the look-back bound: one pass over three tiles launched as two
// blocks with the tile counter starting at 1, so tile 0 never runs and tile 1
// waits on a flag that nothing sets.  The wait must end at its bound with
// kStatusSortTimeout in *err, and tile 2 must then finish behind tile 1.
// Returns the status bits (or a CUDA error as -1000 - code).
int sort_timeout_selftest(cudaStream_t s) {
  const int n = 3 * kSortTile, nt = 3;
  unsigned long long *ka = nullptr, *kb = nullptr;
  int *va = nullptr, *err = nullptr;
  unsigned *status = nullptr, *counter = nullptr, *gbase = nullptr;
  cudaError_t e = cudaSuccess;
  if (e == cudaSuccess) e = cudaMalloc(&ka, n * sizeof(unsigned long long));
  if (e == cudaSuccess) e = cudaMalloc(&kb, n * sizeof(unsigned long long));
  if (e == cudaSuccess) e = cudaMalloc(&va, 2 * n * sizeof(int));
  if (e == cudaSuccess) e = cudaMalloc(&err, sizeof(int));
  if (e == cudaSuccess) e = cudaMalloc(&status, (size_t)nt * 256 * sizeof(unsigned));
  if (e == cudaSuccess) e = cudaMalloc(&counter, sizeof(unsigned));
  if (e == cudaSuccess) e = cudaMalloc(&gbase, 256 * sizeof(unsigned));
  int result = 0;
  if (e == cudaSuccess) {
    cudaMemsetAsync(ka, 0, n * sizeof(unsigned long long), s);
    cudaMemsetAsync(status, 0, (size_t)nt * 256 * sizeof(unsigned), s);
    cudaMemsetAsync(gbase, 0, 256 * sizeof(unsigned), s);
    cudaMemsetAsync(err, 0, sizeof(int), s);
    const unsigned one = 1u;
    cudaMemcpyAsync(counter, &one, sizeof(unsigned), cudaMemcpyHostToDevice, s);
    k_sort_onesweep<false><<<nt - 1, kSortThreads, 0, s>>>(ka, nullptr, n, 0, gbase, status, counter, kb, va + n, err,
                                                           nullptr, 0);
    cudaMemcpyAsync(&result, err, sizeof(int), cudaMemcpyDeviceToHost, s);
    e = cudaStreamSynchronize(s);
  }
  cudaFree(ka); cudaFree(kb); cudaFree(va); cudaFree(err); cudaFree(status); cudaFree(counter); cudaFree(gbase);
  return e == cudaSuccess ? result : -(int)e - 1000;
}

BONSAI_BOUNDS_ACCESSOR(bounds_word_sort)

}  // namespace bonsai
