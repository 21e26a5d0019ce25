// Harness that runs the reference's own GPU group formation,
// Treecode<float>::makeGroups (code/makeGroups.cu:236-340: PH keys, Thrust
// sort_by_key, segment masks and scans, groups), compiled unmodified for
// sm_100a from the reference tree by oracle/build_ref.sh.  Test and baseline
// infrastructure only: it pins the PH-key, sort-order and group rows to the
// reference's own outputs (tests/golden/make_ref_groups.py) and times the
// reference's kernels beside the library's (bench.py --impl reference).
//
// The reference sets the domain box in buildTree (computeBoundingBox,
// buildTree.cu:80-166), which does not build for sm_100; the box is passed in
// (the oracle's restatement of that function computes it).
//
// Guard: mask_keys (makeGroups.cu:165-175) computes the halo index of block 0
// as max(blockIdx.x*blockDim.x - 1, 0), which resolves to the unsigned max, so
// thread 0 of block 0 reads keys[-1], 8 bytes before the key buffer.  The
// harness sizes the key buffer itself (2N ints, which makeGroups' realloc
// keeps) and places it 16 bytes into an allocation of its own, so that read
// stays inside memory the harness owns; the pointer is handed back before the
// reference's destructor would free it.
//
// usage: ref_groups IN N CX CY CZ HSIZE LEVELSPLIT NCRIT REPS [OUTPREFIX]
//   IN: N float4 (x, y, z, m) records.  Writes, when OUTPREFIX is given,
//   OUTPREFIX.rawkeys (N u64: the full 63-bit PH key of every input particle,
//   from the reference's computeKeys<21> launched alone), .keys (N u64: what
//   makeGroups leaves in its key buffer: the sorted keys masked to their top
//   levelSplit digits by mask_keys), .vals (N int32, the sort permutation),
//   .groups (G int2 (pbeg, np), the reference's atomic order); prints one line
//   "REFGROUPS {json}" with the group count and the makeGroups times.
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <vector>

// the reference's translation unit itself, so that its file-local kernels
// (makeGroups::computeKeys) can also be launched on their own
#include "makeGroups.cu"

int main(int argc, char **argv)
{
  if (argc != 10 && argc != 11) {
    fprintf(stderr, "usage: %s IN N CX CY CZ HSIZE LEVELSPLIT NCRIT REPS [OUTPREFIX]\n", argv[0]);
    return 2;
  }
  const int n = atoi(argv[2]);
  const float box[4] = {(float)atof(argv[3]), (float)atof(argv[4]), (float)atof(argv[5]), (float)atof(argv[6])};
  const int level_split = atoi(argv[7]), ncrit = atoi(argv[8]), reps = std::max(1, atoi(argv[9]));
  std::vector<float> in((size_t)4 * n);
  {
    FILE *f = fopen(argv[1], "rb");
    if (!f || fread(in.data(), sizeof(float), in.size(), f) != in.size()) { fprintf(stderr, "read %s\n", argv[1]); return 1; }
    fclose(f);
  }
  Treecode<float> tc(0.01f, 0.75f, ncrit);
  tc.alloc(n);
  // key buffer with a 16-byte lead (see the guard note above)
  tc.d_key.free();
  char *key_base = nullptr;
  if (cudaMalloc(&key_base, 16 + sizeof(int) * 2 * (size_t)n) != cudaSuccess) return 1;
  cudaMemset(key_base, 0, 16);
  tc.d_key.ptr = reinterpret_cast<int *>(key_base + 16);
  tc.d_key.n = 2 * (size_t)n;
  for (int i = 0; i < n; i++) {
    tc.h_ptclPos[i].x() = in[4 * i];
    tc.h_ptclPos[i].y() = in[4 * i + 1];
    tc.h_ptclPos[i].z() = in[4 * i + 2];
    tc.h_ptclPos[i].mass() = in[4 * i + 3];
    tc.h_ptclVel[i].x() = tc.h_ptclVel[i].y() = tc.h_ptclVel[i].z() = tc.h_ptclVel[i].mass() = 0.0f;
  }
  tc.ptcl_h2d();
  if (cudaMemcpy(tc.d_domain.ptr, box, sizeof(box), cudaMemcpyHostToDevice) != cudaSuccess) return 1;

  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  std::vector<float> ms;
  for (int r = 0; r < reps + 1; r++) {  // the first call is a warm-up
    cudaEventRecord(e0, 0);
    tc.makeGroups(level_split, ncrit);
    cudaEventRecord(e1, 0);
    cudaEventSynchronize(e1);
    float t = 0.f;
    cudaEventElapsedTime(&t, e0, e1);
    if (r > 0) ms.push_back(t);
  }
  // the first G entries of the group list partition the particles
  std::vector<int2> groups((size_t)n);
  if (cudaMemcpy(groups.data(), tc.d_groupList.ptr, sizeof(int2) * n, cudaMemcpyDeviceToHost) != cudaSuccess) return 1;
  long covered = 0;
  int ng = 0;
  while (ng < n && covered < n) covered += groups[ng++].y;
  if (covered != n) { fprintf(stderr, "group sizes do not add up to N\n"); return 1; }
  if (argc == 11) {
    // full keys of the input order: computeKeys<21> (makeGroups.cu:108-135) alone
    {
      unsigned long long *raw = nullptr;
      int *idx = nullptr;
      if (cudaMalloc(&raw, sizeof(unsigned long long) * n) != cudaSuccess) return 1;
      if (cudaMalloc(&idx, sizeof(int) * n) != cudaSuccess) return 1;
      makeGroups::computeKeys<21, float><<<(n + 255) / 256, 256>>>(n, tc.d_domain, tc.d_ptclPos, raw, idx);
      std::vector<unsigned long long> h((size_t)n);
      cudaMemcpy(h.data(), raw, sizeof(unsigned long long) * n, cudaMemcpyDeviceToHost);
      FILE *f = fopen((std::string(argv[10]) + ".rawkeys").c_str(), "wb");
      fwrite(h.data(), sizeof(unsigned long long), n, f); fclose(f);
      cudaFree(raw);
      cudaFree(idx);
    }
    std::vector<unsigned long long> keys((size_t)n);
    std::vector<int> vals((size_t)n);
    cudaMemcpy(keys.data(), tc.d_key.ptr, sizeof(unsigned long long) * n, cudaMemcpyDeviceToHost);
    cudaMemcpy(vals.data(), tc.d_value.ptr, sizeof(int) * n, cudaMemcpyDeviceToHost);
    const std::string p(argv[10]);
    FILE *f = fopen((p + ".keys").c_str(), "wb");
    fwrite(keys.data(), sizeof(unsigned long long), n, f); fclose(f);
    f = fopen((p + ".vals").c_str(), "wb");
    fwrite(vals.data(), sizeof(int), n, f); fclose(f);
    f = fopen((p + ".groups").c_str(), "wb");
    fwrite(groups.data(), sizeof(int2), ng, f); fclose(f);
  }
  tc.d_key.ptr = nullptr;  // owned by the harness
  tc.d_key.n = 0;
  cudaFree(key_base);
  std::sort(ms.begin(), ms.end());
  printf("REFGROUPS {\"n\": %d, \"groups\": %d, \"reps\": %d, \"ms_min\": %.4f, \"ms_median\": %.4f}\n", n, ng,
         (int)ms.size(), ms.front(), ms[ms.size() / 2]);
  return cudaGetLastError() == cudaSuccess ? 0 : 1;
}
