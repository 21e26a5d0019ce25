// groups.cu -- walk groups from the PH-sorted keys, and the gather of the
// particle state into PH order.
//
// The reference (makeGroups.cu:137-223, :259-309) masks the sorted PH keys to
// their top levelSplit octal digits, finds the segments of equal masked key
// with two scan_by_key passes, and cuts every segment into chunks of nCrit
// particles, numbering groups with an atomic counter.  The masked key of a
// sorted key is its top 3*levelSplit bits, i.e. a bin index in
// [0, 8^levelSplit); bins appear in increasing order along the sorted array.
// So the segment of every bin is found where the bin changes (one pass, no
// atomics), one exclusive scan over ceil(size/nCrit) gives the group offsets,
// and groups are written in PH order (deterministic; the reference's
// canonical order).
#include "common.cuh"
#include "kernels.cuh"

namespace bonsai {

// Segment bounds straight from the sorted keys: position i starts the segment
// of bin(i) when bin(i) != bin(i-1), and ends the segment of bin(i-1) there.
// Each bin has one start and one end, so every entry is written by exactly one
// thread (no atomics); empty bins keep [0, 0) from the memset.
__global__ void __launch_bounds__(256) k_group_bounds(const unsigned long long* __restrict__ sorted, int n,
                                                      int shift, unsigned* __restrict__ seg_beg,
                                                      unsigned* __restrict__ seg_end) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const unsigned b = (unsigned)(sorted[i] >> shift);
    const unsigned p = i > 0 ? (unsigned)(sorted[i - 1] >> shift) : ~0u;
    if (b != p) {
      seg_beg[b] = (unsigned)i;
      if (i > 0) seg_end[p] = (unsigned)i;
    }
    if (i == n - 1) seg_end[b] = (unsigned)n;
  }
}

__global__ void k_group_sizes(const unsigned* __restrict__ seg_beg, const unsigned* __restrict__ seg_end, int nbins,
                              int ncrit, unsigned* __restrict__ ng) {
  for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < nbins; b += gridDim.x * blockDim.x)
    ng[b] = (seg_end[b] - seg_beg[b] + (unsigned)ncrit - 1u) / (unsigned)ncrit;
}

// one thread per group: the group's bin is found by binary search over the
// exclusive scan of group counts (bins near a dense core hold 10^5 groups, so
// a thread per bin would serialise them)
__global__ void __launch_bounds__(256) k_group_write(const unsigned* __restrict__ seg_end,
                                                     const unsigned* __restrict__ seg_start,
                                                     const unsigned* __restrict__ goff, int nbins, int ncrit,
                                                     int2* __restrict__ groups, int group_cap,
                                                     TreeInfo* __restrict__ info) {
  const int ng = info->ngroups;
  if (ng > group_cap) {
    if (blockIdx.x == 0 && threadIdx.x == 0) set_status(&info->status, kStatusGroupCapacity);
    return;
  }
  for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < ng; g += gridDim.x * blockDim.x) {
    int lo = 0, hi = nbins;  // last bin with goff <= g
    while (hi - lo > 1) {
      const int mid = (lo + hi) >> 1;
      if ((int)__ldg(goff + mid) <= g) lo = mid; else hi = mid;
    }
    // the last bin with goff <= g is never empty (an empty bin shares its
    // offset with the next bin)
    const int k = g - (int)goff[lo];
    const int off = k * ncrit;
    const int count = (int)(seg_end[lo] - seg_start[lo]);
    groups[g] = make_int2((int)seg_start[lo] + off, min(ncrit, count - off));
  }
}

void make_groups(const unsigned long long* sorted_ph, int n, int level_split, int ncrit, unsigned* seg_end,
                 unsigned* seg_start, unsigned* ng, unsigned* bsum, int2* groups, int group_cap, TreeInfo* info,
                 cudaStream_t s) {
  const int nbins = 1 << (3 * level_split);
  const int shift = 63 - 3 * level_split;
  cudaMemsetAsync(seg_start, 0, sizeof(unsigned) * (size_t)nbins, s);
  cudaMemsetAsync(seg_end, 0, sizeof(unsigned) * (size_t)nbins, s);
  k_group_bounds<<<1184, 256, 0, s>>>(sorted_ph, n, shift, seg_start, seg_end);
  k_group_sizes<<<(nbins + 255) / 256, 256, 0, s>>>(seg_start, seg_end, nbins, ncrit, ng);
  exclusive_scan(ng, ng, nbins, bsum, (unsigned*)&info->ngroups, s);
  k_group_write<<<1184, 256, 0, s>>>(seg_end, seg_start, ng, nbins, ncrit, groups, group_cap, info);
}

// state gather: out[k] = in[perm[k]] for positions, velocities and ids
__global__ void __launch_bounds__(256) k_gather_state(const int* __restrict__ perm, int n,
                                                      const float4* __restrict__ pos, const float4* __restrict__ vel,
                                                      const int* __restrict__ id, float4* __restrict__ pos_o,
                                                      float4* __restrict__ vel_o, int* __restrict__ id_o) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
    const int j = __ldcs(perm + k);
    __stcs(pos_o + k, __ldg(pos + j));
    __stcs(vel_o + k, __ldg(vel + j));
    __stcs(id_o + k, __ldg(id + j));
  }
}

__global__ void __launch_bounds__(256) k_gather_pos(const int* __restrict__ perm, int n,
                                                    const float4* __restrict__ pos, float4* __restrict__ out) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x)
    out[k] = __ldg(pos + __ldcs(perm + k));
}

}  // namespace bonsai
