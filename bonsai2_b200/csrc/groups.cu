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
                                                      int shift, [[maybe_unused]] int nbins,
                                                      unsigned* __restrict__ seg_beg, unsigned* __restrict__ seg_end) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const unsigned b = (unsigned)(sorted[i] >> shift);
    const unsigned p = i > 0 ? (unsigned)(sorted[i - 1] >> shift) : ~0u;
    if (!BONSAI_IN_RANGE(b, nbins, 0x201) || (i > 0 && !BONSAI_IN_RANGE(p, nbins, 0x202))) continue;
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
                                                     TreeInfo* __restrict__ info, [[maybe_unused]] int n) {
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
    // every group holds at least one particle, inside the particle range
    if (!BONSAI_IN_RANGE(off, count, 0x203) || !BONSAI_IN_RANGE((int)seg_start[lo] + count - 1, n, 0x204)) continue;
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
  k_group_bounds<<<1184, 256, 0, s>>>(sorted_ph, n, shift, nbins, seg_start, seg_end);
  k_group_sizes<<<(nbins + 255) / 256, 256, 0, s>>>(seg_start, seg_end, nbins, ncrit, ng);
  exclusive_scan(ng, ng, nbins, bsum, (unsigned*)&info->ngroups, s);
  k_group_write<<<1184, 256, 0, s>>>(seg_end, seg_start, ng, nbins, ncrit, groups, group_cap, info, n);
}

// Ensembles.  Bins repeat from system to system, so segments are numbered by
// position instead: flag[i] = 1 where a segment starts (bin change or system
// start), an exclusive scan gives every start its segment index, and the
// group sizes and offsets follow as above over the segment list (capacity n,
// tail entries sized 0).  Inside a system the segments and groups are those
// the system gets alone.
__global__ void __launch_bounds__(256) k_seg_flags(const unsigned long long* __restrict__ sorted, int n, int shift,
                                                   unsigned* __restrict__ flag) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    flag[i] = (i == 0 || (sorted[i] >> shift) != (sorted[i - 1] >> shift)) ? 1u : 0u;
}

__global__ void k_seg_mark_systems(const int* __restrict__ sys_off, int nsys, unsigned* __restrict__ flag) {
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < nsys; s += gridDim.x * blockDim.x) flag[sys_off[s]] = 1u;
}

// seg_beg/seg_end of every segment (flag is reused for the group counts next)
__global__ void __launch_bounds__(256) k_seg_bounds(const unsigned* __restrict__ flag,
                                                    const unsigned* __restrict__ sid, int n,
                                                    unsigned* __restrict__ seg_beg, unsigned* __restrict__ seg_end) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const unsigned f = flag[i], k = sid[i];
    if (!BONSAI_IN_RANGE(k + f - 1, n, 0x205) || (f && !BONSAI_IN_RANGE(k, n, 0x206))) continue;
    if (f) {
      seg_beg[k] = (unsigned)i;
      if (i > 0) seg_end[k - 1] = (unsigned)i;
    }
    if (i == n - 1) seg_end[k + f - 1] = (unsigned)n;
  }
}

__global__ void __launch_bounds__(256) k_seg_group_sizes(const unsigned* __restrict__ seg_beg,
                                                         const unsigned* __restrict__ seg_end,
                                                         const unsigned* __restrict__ nseg, int m, int ncrit,
                                                         unsigned* __restrict__ ng) {
  const int ns = (int)*nseg;
  for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < m; b += gridDim.x * blockDim.x)
    ng[b] = b < ns ? (seg_end[b] - seg_beg[b] + (unsigned)ncrit - 1u) / (unsigned)ncrit : 0u;
}

void make_groups_sys(const unsigned long long* sorted_ph, int n, int level_split, int ncrit, const int* sys_off,
                     int nsys, unsigned* flag, unsigned* sid, unsigned* seg_beg, unsigned* seg_end, unsigned* nseg,
                     unsigned* bsum, int2* groups, int group_cap, TreeInfo* info, cudaStream_t s) {
  const int shift = 63 - 3 * level_split;
  k_seg_flags<<<1184, 256, 0, s>>>(sorted_ph, n, shift, flag);
  k_seg_mark_systems<<<(nsys + 255) / 256, 256, 0, s>>>(sys_off, nsys, flag);
  exclusive_scan(flag, sid, n, bsum, nseg, s);
  k_seg_bounds<<<1184, 256, 0, s>>>(flag, sid, n, seg_beg, seg_end);
  unsigned* ng = flag;
  k_seg_group_sizes<<<1184, 256, 0, s>>>(seg_beg, seg_end, nseg, n, ncrit, ng);
  exclusive_scan(ng, ng, n, bsum, (unsigned*)&info->ngroups, s);
  k_group_write<<<1184, 256, 0, s>>>(seg_end, seg_beg, ng, n, ncrit, groups, group_cap, info, n);
}

// state gather: out[k] = in[perm[k]] for positions, velocities and ids
__global__ void __launch_bounds__(256) k_gather_state(const int* __restrict__ perm, int n,
                                                      const float4* __restrict__ pos, const float4* __restrict__ vel,
                                                      const int* __restrict__ id, float4* __restrict__ pos_o,
                                                      float4* __restrict__ vel_o, int* __restrict__ id_o) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
    const int j = __ldcs(perm + k);
    if (!BONSAI_IN_RANGE(j, n, 0x207)) continue;
    __stcs(pos_o + k, __ldg(pos + j));
    __stcs(vel_o + k, __ldg(vel + j));
    __stcs(id_o + k, __ldg(id + j));
  }
}

__global__ void __launch_bounds__(256) k_gather_pos(const int* __restrict__ perm, int n,
                                                    const float4* __restrict__ pos, float4* __restrict__ out) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
    const int j = __ldcs(perm + k);
    if (BONSAI_IN_RANGE(j, n, 0x208)) out[k] = __ldg(pos + j);
  }
}

BONSAI_BOUNDS_ACCESSOR(bounds_word_groups)

}  // namespace bonsai
