// Harness that runs the reference's own multipole and tree-walk code,
// Treecode<float>::computeMultipoles (code/computeMultipoles.cu:81-190,
// 194-231) and Treecode<float>::computeForces (code/computeForces.cu:229-619,
// 622-727), on a tree that the library built.  Test and baseline
// infrastructure only: the "modified reference" that pins the walk and
// multipole rows to the reference's own kernels (tests/golden/make_ref_walk.py)
// and times them beside the library (bench.py --impl reference).
//
// The two files do not build for sm_100 as shipped (legacy textures, pre-Volta
// shuffles, warp-synchronous shared-memory exchanges); oracle/make_modref.py
// writes copies with mechanical shims into oracle/_ref/modref/, and
// oracle/ref_shim.cuh supplies the texture stand-ins.  The reference's tree
// build (buildTree.cu) needs CUDA-12-removed device synchronisation, so the
// cells, level ranges and groups come from the library, which exports them in
// the reference's layout (CellData uint4, Treecode.h:45-89; GroupData int2,
// Treecode.h:29-43; level_begIdx {first, last}).
//
// The input is checked on the host before anything is launched: every node's
// children lie in (cell, ncells), every particle range in [0, n], the level-1
// range and the groups inside their arrays, group sizes in [1, 64] (the
// reference's NI = 2 walk).  A walk over such a tree ends.
//
// usage:
//   ref_walk check IN OUTPREFIX   reference multipoles of the given tree
//       (OUTPREFIX.refmp: size4, mono4, quad0 float4 and quad1 float2 per
//       cell), and the reference walk twice -- with the library's multipoles
//       (OUTPREFIX.acc_lib float4 per particle in group order, .cnt_lib
//       (approx, direct) per group) and with the reference's own (.acc_ref,
//       .cnt_ref).  Per-group counts come from computeForces' own statistics
//       (its maxima) with the group list narrowed to one group per call.
//   ref_walk time IN REPS         times computeMultipoles and computeForces
//       (CUDA events around the public calls; best and median of REPS after
//       one warm-up), the walk on the reference's own multipoles.
// IN: int32 header {magic 0x4b4c5752, n, ncells, ngroups, l1_beg, l1_end
// (exclusive), ncrit, 0}, float32 {theta, eps2}, then cell_data uint4[ncells],
// size4, mono4, quad0 float4[ncells], quad1 float2[ncells], groups int2[ngroups],
// ipos float4[n] (group order), jpos float4[n] (tree order).
#include <algorithm>  // before Treecode.h, whose "#define __out" breaks libstdc++'s <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "ref_shim.cuh"
#include "_ref/modref/computeMultipoles.cu"
#include "_ref/modref/computeForces.cu"

// Access to Treecode's private counts (nCells, nGroups) through explicit
// instantiation, where access checking does not apply ([temp.explicit]).
template <typename Tag, typename Tag::type M>
struct PrivateMember {
  friend typename Tag::type member(Tag) { return M; }
};
struct TcCells { typedef int Treecode<float>::*type; friend type member(TcCells); };
struct TcGroups { typedef int Treecode<float>::*type; friend type member(TcGroups); };
template struct PrivateMember<TcCells, &Treecode<float>::nCells>;
template struct PrivateMember<TcGroups, &Treecode<float>::nGroups>;

namespace {

struct Input {
  int n = 0, ncells = 0, ngroups = 0, l1_beg = 0, l1_end = 0, ncrit = 0;
  float theta = 0.f, eps2 = 0.f;
  std::vector<uint4> cells;
  std::vector<float4> size, mono, q0, ipos, jpos;
  std::vector<float2> q1;
  std::vector<int2> groups;
};

template <typename T>
bool rd(FILE* f, std::vector<T>& v, size_t count) {
  v.resize(count);
  return fread(v.data(), sizeof(T), count, f) == count;
}

const char* read_input(const char* path, Input& in) {
  FILE* f = fopen(path, "rb");
  if (!f) return "cannot open input";
  int hdr[8];
  float fl[2];
  const char* err = nullptr;
  if (fread(hdr, sizeof(int), 8, f) != 8 || fread(fl, sizeof(float), 2, f) != 2) err = "short header";
  else if (hdr[0] != 0x4b4c5752) err = "bad magic";
  if (!err) {
    in.n = hdr[1]; in.ncells = hdr[2]; in.ngroups = hdr[3]; in.l1_beg = hdr[4]; in.l1_end = hdr[5]; in.ncrit = hdr[6];
    in.theta = fl[0]; in.eps2 = fl[1];
    if (in.n < 1 || in.ncells < 1 || in.ngroups < 1) err = "empty input";
  }
  if (!err && !(rd(f, in.cells, in.ncells) && rd(f, in.size, in.ncells) && rd(f, in.mono, in.ncells) &&
                rd(f, in.q0, in.ncells) && rd(f, in.q1, in.ncells) && rd(f, in.groups, in.ngroups) &&
                rd(f, in.ipos, in.n) && rd(f, in.jpos, in.n)))
    err = "short input";
  fclose(f);
  return err;
}

// the tree is walkable: children after their parent and inside the array
const char* validate(const Input& in) {
  if (!(0 <= in.l1_beg && in.l1_beg < in.l1_end && in.l1_end <= in.ncells)) return "level-1 range";
  for (int c = 0; c < in.ncells; c++) {
    const CellData cd(in.cells[c]);
    if (cd.pbeg() < 0 || cd.pend() < cd.pbeg() || cd.pend() > in.n) return "cell particle range";
    if (cd.isNode()) {
      const long first = cd.first(), nch = cd.n();
      if (first <= c || nch < 1 || nch > 8 || first + nch > in.ncells) return "cell children";
    }
  }
  long covered = 0;
  for (const int2& g : in.groups) {
    if (g.x < 0 || g.y < 1 || g.y > 64 || (long)g.x + g.y > in.n) return "group range";
    covered += g.y;
  }
  if (covered != in.n) return "groups do not cover the particles";
  if (in.ncrit < 1 || in.ncrit > 64) return "ncrit";
  return nullptr;
}

template <typename T>
bool h2d(cuda_mem<T>& d, const std::vector<T>& h) {
  d.realloc(h.size());
  return cudaMemcpy(d.ptr, h.data(), sizeof(T) * h.size(), cudaMemcpyHostToDevice) == cudaSuccess;
}

template <typename T>
bool d2h(std::vector<T>& h, const T* d, size_t count) {
  h.resize(count);
  return cudaMemcpy(h.data(), d, sizeof(T) * count, cudaMemcpyDeviceToHost) == cudaSuccess;
}

template <typename T>
void wr(const std::string& path, const std::vector<T>& v) {
  FILE* f = fopen(path.c_str(), "wb");
  if (!f) { fprintf(stderr, "cannot write %s\n", path.c_str()); exit(1); }
  fwrite(v.data(), sizeof(T), v.size(), f);
  fclose(f);
}

bool cuda_ok(const char* where) {
  const cudaError_t e = cudaDeviceSynchronize();
  const cudaError_t e2 = cudaGetLastError();
  if (e != cudaSuccess || e2 != cudaSuccess) {
    fprintf(stderr, "%s: %s\n", where, cudaGetErrorString(e != cudaSuccess ? e : e2));
    return false;
  }
  return true;
}

// the reference object holding the library's tree
bool setup(Treecode<float>& tc, const Input& in) {
  tc.theta = in.theta;
  tc.eps2 = in.eps2;
  tc.alloc(in.n);
  tc.*member(TcCells()) = in.ncells;
  tc.*member(TcGroups()) = in.ngroups;
  std::vector<CellData> cd(in.cells.begin(), in.cells.end());
  tc.d_cellDataList.free();
  std::vector<Particle4<float>> ip(in.n), jp(in.n);
  for (int i = 0; i < in.n; i++) {
    ip[i] = Particle4<float>();
    jp[i] = Particle4<float>();
    ip[i].x() = in.ipos[i].x; ip[i].y() = in.ipos[i].y; ip[i].z() = in.ipos[i].z; ip[i].mass() = in.ipos[i].w;
    jp[i].x() = in.jpos[i].x; jp[i].y() = in.jpos[i].y; jp[i].z() = in.jpos[i].z; jp[i].mass() = in.jpos[i].w;
  }
  std::vector<int2> lev(32, make_int2(0, 0));
  lev[1] = make_int2(in.l1_beg, in.l1_end - 1);  // {first, last}
  std::vector<GroupData> gd(in.groups.begin(), in.groups.end());
  return h2d(tc.d_cellDataList, cd) && h2d(tc.d_ptclPos, jp) && h2d(tc.d_ptclPos_tmp, ip) &&
         cudaMemcpy(tc.d_level_begIdx.ptr, lev.data(), sizeof(int2) * 32, cudaMemcpyHostToDevice) == cudaSuccess &&
         h2d(tc.d_groupList, gd) && cuda_ok("setup");
}

bool set_multipoles(Treecode<float>& tc, const std::vector<float4>& s, const std::vector<float4>& m,
                    const std::vector<float4>& q0, const std::vector<float2>& q1) {
  return h2d(tc.d_cellSize, s) && h2d(tc.d_cellMonopole, m) && h2d(tc.d_cellQuad0, q0) && h2d(tc.d_cellQuad1, q1);
}

// the whole walk, then one call per group for that group's counts
bool walk(Treecode<float>& tc, const Input& in, double4& stats, std::vector<float4>& acc,
          std::vector<unsigned>& counts) {
  stats = tc.computeForces(true);
  if (!cuda_ok("computeForces") || !d2h(acc, reinterpret_cast<float4*>(tc.d_ptclAcc.ptr), in.n)) return false;
  counts.assign(2 * (size_t)in.ngroups, 0u);
  GroupData* base = tc.d_groupList.ptr;
  tc.*member(TcGroups()) = 1;
  bool ok = true;
  for (int g = 0; g < in.ngroups && ok; g++) {
    tc.d_groupList.ptr = base + g;
    const double4 s = tc.computeForces(true);
    ok = cuda_ok("computeForces (one group)");
    counts[2 * g] = (unsigned)s.w;      // approximate interactions of the group
    counts[2 * g + 1] = (unsigned)s.y;  // direct interactions of the group
  }
  tc.d_groupList.ptr = base;
  tc.*member(TcGroups()) = in.ngroups;
  return ok;
}

float elapsed(cudaEvent_t a, cudaEvent_t b) {
  float ms = 0.f;
  cudaEventElapsedTime(&ms, a, b);
  return ms;
}

}  // namespace

int main(int argc, char** argv) {
  if (argc != 4 || (strcmp(argv[1], "check") && strcmp(argv[1], "time"))) {
    fprintf(stderr, "usage: %s check IN OUTPREFIX | time IN REPS\n", argv[0]);
    return 2;
  }
  Input in;
  const char* err = read_input(argv[2], in);
  if (!err) err = validate(in);
  if (err) {
    fprintf(stderr, "ref_walk: %s\n", err);
    return 1;
  }
  Treecode<float> tc(0.01f, in.theta, in.ncrit);
  if (!setup(tc, in)) return 1;

  if (!strcmp(argv[1], "time")) {
    const int reps = std::max(1, atoi(argv[3]));
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    std::vector<float> tm, tw;
    double4 stats = {0, 0, 0, 0};
    for (int r = 0; r <= reps; r++) {
      cudaEventRecord(e0, 0);
      tc.computeMultipoles();
      cudaEventRecord(e1, 0);
      cudaEventSynchronize(e1);
      if (r) tm.push_back(elapsed(e0, e1));
      cudaEventRecord(e0, 0);
      stats = tc.computeForces(true);
      cudaEventRecord(e1, 0);
      cudaEventSynchronize(e1);
      if (r) tw.push_back(elapsed(e0, e1));
      if (!cuda_ok("timed step")) return 1;
    }
    std::sort(tm.begin(), tm.end());
    std::sort(tw.begin(), tw.end());
    printf("REFWALK_TIME {\"n\": %d, \"cells\": %d, \"groups\": %d, \"reps\": %d, "
           "\"multipoles_ms_min\": %.4f, \"multipoles_ms_median\": %.4f, \"walk_ms_min\": %.4f, "
           "\"walk_ms_median\": %.4f, \"direct_mean\": %.4f, \"direct_max\": %.0f, \"approx_mean\": %.4f, "
           "\"approx_max\": %.0f}\n",
           in.n, in.ncells, in.ngroups, reps, tm.front(), tm[tm.size() / 2], tw.front(), tw[tw.size() / 2], stats.x,
           stats.y, stats.z, stats.w);
    return 0;
  }

  const std::string out(argv[3]);
  tc.computeMultipoles();
  if (!cuda_ok("computeMultipoles")) return 1;
  std::vector<float4> rs, rm, rq0;
  std::vector<float2> rq1;
  if (!d2h(rs, tc.d_cellSize.ptr, in.ncells) || !d2h(rm, tc.d_cellMonopole.ptr, in.ncells) ||
      !d2h(rq0, tc.d_cellQuad0.ptr, in.ncells) || !d2h(rq1, tc.d_cellQuad1.ptr, in.ncells))
    return 1;
  {
    FILE* f = fopen((out + ".refmp").c_str(), "wb");
    if (!f) return 1;
    fwrite(rs.data(), sizeof(float4), rs.size(), f);
    fwrite(rm.data(), sizeof(float4), rm.size(), f);
    fwrite(rq0.data(), sizeof(float4), rq0.size(), f);
    fwrite(rq1.data(), sizeof(float2), rq1.size(), f);
    fclose(f);
  }
  double4 sl, sr;
  std::vector<float4> al, ar;
  std::vector<unsigned> cl, cr;
  if (!set_multipoles(tc, in.size, in.mono, in.q0, in.q1) || !walk(tc, in, sl, al, cl)) return 1;
  if (!set_multipoles(tc, rs, rm, rq0, rq1) || !walk(tc, in, sr, ar, cr)) return 1;
  wr(out + ".acc_lib", al);
  wr(out + ".cnt_lib", cl);
  wr(out + ".acc_ref", ar);
  wr(out + ".cnt_ref", cr);
  printf("REFWALK {\"n\": %d, \"cells\": %d, \"groups\": %d, \"lib_multipoles\": [%.6f, %.0f, %.6f, %.0f], "
         "\"ref_multipoles\": [%.6f, %.0f, %.6f, %.0f]}\n",
         in.n, in.ncells, in.ngroups, sl.x, sl.y, sl.z, sl.w, sr.x, sr.y, sr.z, sr.w);
  return 0;
}
