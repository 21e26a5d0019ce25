// treecode.cu -- host side: the Treecode handle behind the C ABI
// (include/bonsai_b200.h).  Owns every device buffer, sequences the stages on
// the handle's stream without host round trips, and captures the whole step
// as a CUDA graph.
//
// Data flow of one step (reference: treecode.cu:137-168):
//   build     : box -> (tree key, PH key) per particle -> sort tree keys ->
//               gather positions into tree order (jpos) -> cells
//   multipoles: bottom-up from jpos
//   groups    : sort PH keys -> groups -> gather the state (pos, vel, id)
//               into PH order, so group particles are contiguous
//   forces    : walk, acc in PH order (= state order)
//   move      : leapfrog + energies on the state
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "../../include/bonsai_b200.h"
#include "common.cuh"
#include "kernels.cuh"

using namespace bonsai;

namespace {

// the learned form's bound tau = kStartAlpha A_g in the one evaluation after
// the fixed-angle fallback (the single-parameter relative walk the training
// tables are recorded after, bonsai2_b200/learned.py ALPHA0)
constexpr float kStartAlpha = 1e-2f;
constexpr int kRingCap = 16384;  // per-warp level lists of the walk (ints): two halves of 8192
constexpr int kMaxLevelSplit = 7;

template <class T>
cudaError_t dalloc(T** p, size_t n) {
  *p = nullptr;
  if (n == 0) n = 1;
  return cudaMalloc((void**)p, n * sizeof(T));
}
template <class T>
void dfree(T** p) {
  if (*p) cudaFree(*p);
  *p = nullptr;
}

struct Handle {
  bonsai_params prm{};
  int dev = 0, nsm = 0;
  cudaStream_t st = nullptr;
  int n = 0, cap_cells = 0;
  // state, double-buffered: [par] holds the live state
  float4* pos[2] = {nullptr, nullptr};
  float4* vel[2] = {nullptr, nullptr};
  int* id[2] = {nullptr, nullptr};
  int par = 0;
  float4* acc = nullptr;
  float4* jpos = nullptr;
  unsigned long long *tkey = nullptr, *pkey = nullptr, *kalt = nullptr;
  int *tperm = nullptr, *pperm = nullptr, *valt = nullptr;
  unsigned *sort_counts = nullptr, *bsum = nullptr;
  // the group branch of a step (PH sort, groups, state gather) runs on st2,
  // beside the tree branch (tree sort, tree, multipoles), with its own sort
  // scratch; ev_fork / ev_join tie it to the handle's stream
  cudaStream_t st2 = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  unsigned long long* kalt2 = nullptr;
  int* valt2 = nullptr;
  unsigned* sort_counts2 = nullptr;
  uint8_t* dlev = nullptr;
  uint16_t* chain = nullptr;
  unsigned* hist = nullptr;
  TreeInfo* info = nullptr;
  uint4* cell_data = nullptr;
  float4 *cell_open = nullptr, *cell_stage = nullptr;  // cell_stage: 3 per cell
  int *cell_parent = nullptr, *leaf_list = nullptr, *mp_count = nullptr;
  MpRec* rec = nullptr;
  double* cell_box = nullptr;  // 6 per cell: floats (float positions) or doubles (double-single)
  float4* cell_ls = nullptr;
  // per-group opening angles (theta mode 1: MLP, 2: caller's array)
  int theta_mode = 0;
  float theta_lo = 0.25f, theta_hi = 1.25f;
  int gcap = 0;
  float* group_inv = nullptr;
  // relative accuracy mode: per-group bound on a cell's truncation error,
  // each group's mean |a| of the previous evaluation, the walk's per-group
  // statistics and the group of every particle (read by the next
  // evaluation's features), and the flag that acc holds valid accelerations
  float* group_tau = nullptr;
  float* group_amag = nullptr;
  float4* group_stats = nullptr;
  int* part_gid = nullptr;
  int* acc_valid = nullptr;  // device: [0] acc is this state's, [1] the walk statistics came with it
  bool tau_on = false;
  float theta_bound = 2.0f;  // geometric safety bound of the relative modes
  float rel_alpha = 1e-2f;   // theta mode 3: tau = rel_alpha * A_g
  float* group_feat = nullptr;
  uint2* group_counts = nullptr;  // per-group (approx, direct) counts of the per-group angle walk
  double4 *acc64 = nullptr, *acc64_tmp = nullptr;  // FP64 checker walk output (group order, caller order)
  float* mlp_w = nullptr;
  void* mlp_wh = nullptr;
  bool mlp_loaded = false;
  int2* groups = nullptr;
  unsigned *g_count = nullptr, *g_seg = nullptr, *g_ng = nullptr;
  int* ring = nullptr;
  int walk_blocks[6] = {0, 0, 0, 0, 0, 0};  // per walk variant (walk_variant)
  int ring_warps = 0;
  unsigned* group_counter = nullptr;
  unsigned long long* stats = nullptr;
  double *move_partial = nullptr, *energies = nullptr;
  unsigned *move_ticket = nullptr, *box_ticket = nullptr;
  int* closing = nullptr;
  Box* box = nullptr;
  float* box_partial = nullptr;
  uint16_t* ph_table = nullptr;
  double *direct_part = nullptr, *direct_out = nullptr;
  int* direct_sample = nullptr;
  int direct_cap = 0;
  int box_blocks = 0, move_blocks = 0;
  int cur_nleaf = 16, cur_ncrit = 64, cur_ls = 5;
  int walk_layout = 0;  // walk_variant layout: 0 half-warp pairs where nCrit <= 64, 1 full warp
  // precision 1: positions double-single, hi in pos/jpos/cell_open, lo in
  // plo/jlo/cell_lo (state, tree and cell order)
  int precision = 0;
  float4* plo[2] = {nullptr, nullptr};
  float4 *jlo = nullptr, *cell_lo = nullptr;
  // ensemble layout (nsys > 1): system s owns particles [off[s], off[s+1]) of
  // the state; every stage works per system in the same launches
  // asynchronous host copies: uploads on st_h2d into staging (in_pos,
  // in_vel), consumed by the handle's stream; downloads of results from two
  // staging slots on st_d2h.  Events order the three streams.
  cudaStream_t st_h2d = nullptr, st_d2h = nullptr;
  float4 *in_pos = nullptr, *in_vel = nullptr;
  float4* out_buf[2][3] = {{nullptr, nullptr, nullptr}, {nullptr, nullptr, nullptr}};  // slot x (pos, vel, acc)
  int out_slot = 0;
  cudaEvent_t ev_in_copied = nullptr, ev_in_consumed = nullptr, ev_out_ready[2] = {nullptr, nullptr},
              ev_out_done[2] = {nullptr, nullptr};
  // block time steps (bts_K >= 0): per-particle level (state order, double
  // buffered like the state), accelerations carried between substeps, and the
  // list of groups walked in a substep
  int bts_K = -1;
  float bts_eta = 0.2f;
  bool bts_ready = false;
  unsigned char* lev[2] = {nullptr, nullptr};
  float4* acc_alt = nullptr;
  int* walk_list = nullptr;
  unsigned* walk_list_n = nullptr;
  int* max_lev = nullptr;  // device: largest level present
  bool walk_list_on = false;
  // acc follows the particles' current (state) order: after a walk, and after
  // a block-step gather; false once a PH gather reorders the particles
  bool acc_in_state_order = false;
  PrevEval prev_eval() const {
    PrevEval p;
    p.acc = acc;
    p.perm = acc_in_state_order ? nullptr : pperm;
    p.acc_valid = acc_valid;
    p.part_gid = part_gid;
    p.stats = group_stats;
    p.stats_cap = gcap;
    return p;
  }
  bool bts_gathering = false;  // inside block_steps: levels and accelerations follow the state
  int nsys = 1, nchunks = 0;
  int *sys_off = nullptr, *chunk_beg = nullptr, *root_beg = nullptr;
  int4* chunks = nullptr;
  Box* sys_box = nullptr;
  float* sys_box_part = nullptr;
  unsigned *seg_beg = nullptr, *seg_end = nullptr, *nseg = nullptr;
  double *chunk_energy = nullptr, *sys_energy = nullptr;
  const int* so() const { return nsys > 1 ? sys_off : nullptr; }
  // stage bookkeeping for the eager API
  bool built = false, mp_done = false, grouped = false, forced = false, moved_after_forces = false;
  bool ever_built = false, ever_mp = false;  // the cell arrays hold a tree / multipoles
  // graphs, one per state parity and phase (0: build+multipoles+groups, 1: walk, 2: move)
  cudaGraphExec_t gexec[2][3] = {{nullptr, nullptr, nullptr}, {nullptr, nullptr, nullptr}};
  int graph_kernels = 0;
  bool graph_ok = false;

  ~Handle() { release(); }

  void release_graphs() {
    for (int p = 0; p < 2; p++)
      for (int k = 0; k < 3; k++)
        if (gexec[p][k]) { cudaGraphExecDestroy(gexec[p][k]); gexec[p][k] = nullptr; }
    graph_ok = false;
  }

  void release_systems() {
    dfree(&sys_off); dfree(&chunk_beg); dfree(&root_beg); dfree(&chunks); dfree(&sys_box); dfree(&sys_box_part);
    dfree(&seg_beg); dfree(&seg_end); dfree(&nseg); dfree(&chunk_energy); dfree(&sys_energy);
    nsys = 1;
    nchunks = 0;
  }

  void release_lo() {
    dfree(&plo[0]); dfree(&plo[1]); dfree(&jlo); dfree(&cell_lo);
  }
  // the low-part arrays of double-single positions (zero: exact float input)
  int alloc_lo() {
    release_lo();
    if (!precision || n == 0) return 0;
    const size_t N = (size_t)n;
    for (int p = 0; p < 2; p++) {
      BONSAI_CUDA_TRY(dalloc(&plo[p], N));
      BONSAI_CUDA_TRY(cudaMemset(plo[p], 0, N * sizeof(float4)));
    }
    BONSAI_CUDA_TRY(dalloc(&jlo, N));
    BONSAI_CUDA_TRY(dalloc(&cell_lo, (size_t)cap_cells));
    return 0;
  }

  void release_staging() {
    if (st_h2d) cudaStreamSynchronize(st_h2d);
    if (st_d2h) cudaStreamSynchronize(st_d2h);
    dfree(&in_pos); dfree(&in_vel);
    for (int k = 0; k < 2; k++)
      for (int a = 0; a < 3; a++) dfree(&out_buf[k][a]);
  }

  void release_bts() {
    dfree(&lev[0]); dfree(&lev[1]); dfree(&acc_alt); dfree(&walk_list); dfree(&walk_list_n); dfree(&max_lev);
    bts_ready = false;
  }
  int alloc_bts() {
    release_bts();
    if (bts_K < 0 || n == 0) return 0;
    for (int p = 0; p < 2; p++) {
      BONSAI_CUDA_TRY(dalloc(&lev[p], (size_t)n));
      BONSAI_CUDA_TRY(cudaMemset(lev[p], 0, (size_t)n));
    }
    BONSAI_CUDA_TRY(dalloc(&acc_alt, (size_t)n));
    BONSAI_CUDA_TRY(dalloc(&walk_list, (size_t)n));
    BONSAI_CUDA_TRY(dalloc(&walk_list_n, 1));
    BONSAI_CUDA_TRY(dalloc(&max_lev, 1));
    return 0;
  }

  void release_particles() {
    release_graphs();
    release_staging();
    release_bts();
    release_systems();
    release_lo();
    for (int p = 0; p < 2; p++) { dfree(&pos[p]); dfree(&vel[p]); dfree(&id[p]); }
    dfree(&acc); dfree(&jpos); dfree(&tkey); dfree(&pkey); dfree(&kalt);
    dfree(&tperm); dfree(&pperm); dfree(&valt); dfree(&sort_counts); dfree(&bsum);
    dfree(&kalt2); dfree(&valt2); dfree(&sort_counts2);
    dfree(&dlev); dfree(&chain); dfree(&hist); dfree(&groups); dfree(&group_inv); dfree(&group_tau); dfree(&group_amag);
    dfree(&group_stats); dfree(&part_gid); dfree(&group_feat);
    dfree(&group_counts); dfree(&acc64); dfree(&acc64_tmp);
    release_cells();
    n = 0;
  }
  void release_cells() {
    dfree(&cell_data); dfree(&cell_open); dfree(&cell_stage);
    dfree(&cell_parent); dfree(&leaf_list); dfree(&mp_count); dfree(&rec); dfree(&cell_ls);
    dfree(&cell_box);
    cap_cells = 0;
  }
  void release() {
    if (st) cudaStreamSynchronize(st);
    release_particles();
    dfree(&info); dfree(&g_count); dfree(&g_seg); dfree(&g_ng); dfree(&ring);
    dfree(&group_counter); dfree(&stats); dfree(&move_partial); dfree(&energies);
    dfree(&move_ticket); dfree(&box_ticket); dfree(&closing); dfree(&acc_valid); dfree(&box); dfree(&box_partial);
    dfree(&ph_table); dfree(&direct_part); dfree(&direct_out); dfree(&direct_sample);
    dfree(&mlp_w);
    if (mlp_wh) { cudaFree(mlp_wh); mlp_wh = nullptr; }
    if (st2) { cudaStreamSynchronize(st2); cudaStreamDestroy(st2); st2 = nullptr; }
    if (ev_fork) { cudaEventDestroy(ev_fork); ev_fork = nullptr; }
    if (ev_join) { cudaEventDestroy(ev_join); ev_join = nullptr; }
    if (st_h2d) { cudaStreamDestroy(st_h2d); st_h2d = nullptr; }
    if (st_d2h) { cudaStreamDestroy(st_d2h); st_d2h = nullptr; }
    cudaEvent_t* evs[6] = {&ev_in_copied, &ev_in_consumed, &ev_out_ready[0], &ev_out_ready[1], &ev_out_done[0],
                           &ev_out_done[1]};
    for (cudaEvent_t* e : evs)
      if (*e) { cudaEventDestroy(*e); *e = nullptr; }
    if (st) { cudaStreamDestroy(st); st = nullptr; }
  }

  int alloc_cells(int cap) {
    release_graphs();
    release_cells();
    cap_cells = cap;
    const size_t C = (size_t)cap;
    BONSAI_CUDA_TRY(dalloc(&cell_data, C));
    BONSAI_CUDA_TRY(dalloc(&cell_open, C));
    BONSAI_CUDA_TRY(dalloc(&cell_stage, 3 * C));
    BONSAI_CUDA_TRY(dalloc(&cell_parent, C));
    BONSAI_CUDA_TRY(dalloc(&leaf_list, C));
    BONSAI_CUDA_TRY(dalloc(&mp_count, C));
    BONSAI_CUDA_TRY(dalloc(&rec, C));
    BONSAI_CUDA_TRY(dalloc(&cell_box, 6 * C));
    BONSAI_CUDA_TRY(dalloc(&cell_ls, C));
    dfree(&cell_lo);
    if (precision) BONSAI_CUDA_TRY(dalloc(&cell_lo, C));
    return 0;
  }

  int init(const bonsai_params* p) {
    prm = *p;
    dev = p->device;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return BONSAI_ERR_NO_DEVICE;
    if (dev < 0 || dev >= ndev) return BONSAI_ERR_ARG;
    BONSAI_CUDA_TRY(cudaSetDevice(dev));
    BONSAI_CUDA_TRY(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    BONSAI_CUDA_TRY(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    BONSAI_CUDA_TRY(cudaStreamCreateWithFlags(&st2, cudaStreamNonBlocking));
    BONSAI_CUDA_TRY(cudaEventCreateWithFlags(&ev_fork, cudaEventDisableTiming));
    BONSAI_CUDA_TRY(cudaEventCreateWithFlags(&ev_join, cudaEventDisableTiming));
    BONSAI_CUDA_TRY(cudaStreamCreateWithFlags(&st_h2d, cudaStreamNonBlocking));
    BONSAI_CUDA_TRY(cudaStreamCreateWithFlags(&st_d2h, cudaStreamNonBlocking));
    {
      cudaEvent_t* evs[6] = {&ev_in_copied, &ev_in_consumed, &ev_out_ready[0], &ev_out_ready[1], &ev_out_done[0],
                             &ev_out_done[1]};
      for (cudaEvent_t* e : evs) BONSAI_CUDA_TRY(cudaEventCreateWithFlags(e, cudaEventDisableTiming));
    }
    box_blocks = nsm * 4;
    move_blocks = nsm * 4;
    BONSAI_CUDA_TRY(dalloc(&info, 1));
    BONSAI_CUDA_TRY(cudaMemset(info, 0, sizeof(TreeInfo)));
    BONSAI_CUDA_TRY(dalloc(&g_count, (size_t)1 << (3 * kMaxLevelSplit)));
    BONSAI_CUDA_TRY(dalloc(&g_seg, (size_t)1 << (3 * kMaxLevelSplit)));
    BONSAI_CUDA_TRY(dalloc(&g_ng, (size_t)1 << (3 * kMaxLevelSplit)));
    for (int k = 0; k < 6; k++) walk_blocks[k] = nsm * walk_blocks_per_sm(k);
    ring_warps = *std::max_element(walk_blocks, walk_blocks + 6) * (kWalkThreads / 32);
    BONSAI_CUDA_TRY(dalloc(&ring, (size_t)ring_warps * kRingCap));
    BONSAI_CUDA_TRY(dalloc(&group_counter, 1));
    BONSAI_CUDA_TRY(dalloc(&stats, 4));
    BONSAI_CUDA_TRY(dalloc(&move_partial, (size_t)move_blocks * 8));
    BONSAI_CUDA_TRY(dalloc(&energies, 8));
    BONSAI_CUDA_TRY(cudaMemset(energies, 0, 8 * sizeof(double)));
    BONSAI_CUDA_TRY(dalloc(&move_ticket, 1));
    BONSAI_CUDA_TRY(dalloc(&box_ticket, 1));
    BONSAI_CUDA_TRY(cudaMemset(move_ticket, 0, sizeof(unsigned)));
    BONSAI_CUDA_TRY(cudaMemset(box_ticket, 0, sizeof(unsigned)));
    BONSAI_CUDA_TRY(dalloc(&closing, 1));
    BONSAI_CUDA_TRY(cudaMemset(closing, 0, sizeof(int)));
    BONSAI_CUDA_TRY(dalloc(&acc_valid, 2));
    BONSAI_CUDA_TRY(cudaMemset(acc_valid, 0, 2 * sizeof(int)));
    BONSAI_CUDA_TRY(dalloc(&box, 1));
    BONSAI_CUDA_TRY(dalloc(&box_partial, (size_t)box_blocks * 6));
    std::vector<uint16_t> tab(kPhTableSize);
    build_ph_table(tab.data());
    BONSAI_CUDA_TRY(dalloc(&ph_table, kPhTableSize));
    BONSAI_CUDA_TRY(cudaMemcpy(ph_table, tab.data(), kPhTableSize * sizeof(uint16_t), cudaMemcpyHostToDevice));
    cur_nleaf = p->nleaf;
    cur_ncrit = p->ncrit;
    cur_ls = p->level_split;
    return 0;
  }

  int alloc(int nn) {
    release_particles();
    n = nn;
    const size_t N = (size_t)nn;
    for (int p = 0; p < 2; p++) {
      BONSAI_CUDA_TRY(dalloc(&pos[p], N));
      BONSAI_CUDA_TRY(dalloc(&vel[p], N));
      BONSAI_CUDA_TRY(dalloc(&id[p], N));
    }
    BONSAI_CUDA_TRY(dalloc(&acc, N));
    BONSAI_CUDA_TRY(cudaMemset(acc, 0, N * sizeof(float4)));
    BONSAI_CUDA_TRY(dalloc(&jpos, N));
    BONSAI_CUDA_TRY(dalloc(&tkey, N));
    BONSAI_CUDA_TRY(dalloc(&pkey, N));
    BONSAI_CUDA_TRY(dalloc(&kalt, N));
    BONSAI_CUDA_TRY(dalloc(&tperm, N));
    BONSAI_CUDA_TRY(dalloc(&pperm, N));
    BONSAI_CUDA_TRY(dalloc(&valt, N));
    BONSAI_CUDA_TRY(dalloc(&sort_counts, sort_status_words(nn)));
    BONSAI_CUDA_TRY(dalloc(&kalt2, N));
    BONSAI_CUDA_TRY(dalloc(&valt2, N));
    BONSAI_CUDA_TRY(dalloc(&sort_counts2, sort_status_words(nn)));
    // scans: group counts per bin (8^7), and per position for ensembles (n)
    const int scan_m = std::max(std::max(256 * sort_tiles(nn), 1 << (3 * kMaxLevelSplit)), nn);
    BONSAI_CUDA_TRY(dalloc(&bsum, (size_t)scan_blocks(scan_m) + 1));
    BONSAI_CUDA_TRY(dalloc(&dlev, N));
    BONSAI_CUDA_TRY(dalloc(&chain, N));
    BONSAI_CUDA_TRY(dalloc(&hist, (size_t)2 * (kMaxLevel + 1) * tree_tiles(nn)));
    BONSAI_CUDA_TRY(dalloc(&groups, N));
    // group-indexed arrays of the per-group angle: at most N/nCrit groups plus
    // one partial group per PH segment (groups.cu)
    gcap = (int)std::min<long long>(N, (long long)N / std::max(1, prm.ncrit) + (1ll << (3 * kMaxLevelSplit)) + 1);
    BONSAI_CUDA_TRY(dalloc(&group_inv, (size_t)gcap));
    BONSAI_CUDA_TRY(dalloc(&group_tau, (size_t)gcap));
    BONSAI_CUDA_TRY(dalloc(&group_amag, (size_t)gcap));
    BONSAI_CUDA_TRY(dalloc(&group_stats, (size_t)gcap));
    BONSAI_CUDA_TRY(cudaMemset(group_stats, 0, (size_t)gcap * sizeof(float4)));
    BONSAI_CUDA_TRY(dalloc(&part_gid, N));
    BONSAI_CUDA_TRY(cudaMemset(part_gid, 0, N * sizeof(int)));
    BONSAI_CUDA_TRY(cudaMemset(acc_valid, 0, 2 * sizeof(int)));
    BONSAI_CUDA_TRY(dalloc(&group_feat, (size_t)gcap * kMlpFeatures));
    BONSAI_CUDA_TRY(dalloc(&group_counts, (size_t)gcap));
    // the reference reserves nPtcl cells (Treecode.h:192); a Plummer tree at
    // nLeaf 16 uses ~0.23 N.  Grown on demand by the eager build.
    int rc = alloc_cells(prm.nleaf >= 8 ? nn / 2 + 4096 : 2 * nn + 4096);
    if (rc) return rc;
    rc = alloc_lo();
    if (rc) return rc;
    rc = alloc_bts();
    if (rc) return rc;
    par = 0;
    built = mp_done = grouped = forced = moved_after_forces = false;
    ever_built = ever_mp = false;
    return 0;
  }

  // ensemble layout from the per-system particle counts (all >= 1)
  int set_systems(const int* counts, int ns) {
    long long tot = 0;
    for (int k = 0; k < ns; k++) {
      if (counts[k] < 1) return BONSAI_ERR_ARG;
      tot += counts[k];
    }
    if (tot > (long long)0x7fffffff - kChunk) return BONSAI_ERR_ARG;
    int rc = alloc((int)tot);
    if (rc) return rc;
    if (ns == 1) return 0;
    std::vector<int> off(ns + 1), cbeg(ns + 1);
    std::vector<int4> ch;
    off[0] = 0;
    for (int k = 0; k < ns; k++) {
      off[k + 1] = off[k] + counts[k];
      cbeg[k] = (int)ch.size();
      for (int b = off[k]; b < off[k + 1]; b += kChunk) ch.push_back(make_int4(b, std::min(b + kChunk, off[k + 1]), k, 0));
    }
    cbeg[ns] = (int)ch.size();
    nsys = ns;
    nchunks = (int)ch.size();
    BONSAI_CUDA_TRY(dalloc(&sys_off, (size_t)ns + 1));
    BONSAI_CUDA_TRY(dalloc(&chunk_beg, (size_t)ns + 1));
    BONSAI_CUDA_TRY(dalloc(&root_beg, (size_t)ns + 1));
    BONSAI_CUDA_TRY(dalloc(&chunks, (size_t)nchunks));
    BONSAI_CUDA_TRY(dalloc(&sys_box, (size_t)ns));
    BONSAI_CUDA_TRY(dalloc(&sys_box_part, (size_t)nchunks * 6));
    BONSAI_CUDA_TRY(dalloc(&seg_beg, (size_t)n));
    BONSAI_CUDA_TRY(dalloc(&seg_end, (size_t)n));
    BONSAI_CUDA_TRY(dalloc(&nseg, 1));
    BONSAI_CUDA_TRY(dalloc(&chunk_energy, (size_t)nchunks * 8));
    BONSAI_CUDA_TRY(dalloc(&sys_energy, (size_t)ns * 8));
    BONSAI_CUDA_TRY(cudaMemcpy(sys_off, off.data(), (ns + 1) * sizeof(int), cudaMemcpyHostToDevice));
    BONSAI_CUDA_TRY(cudaMemcpy(chunk_beg, cbeg.data(), (ns + 1) * sizeof(int), cudaMemcpyHostToDevice));
    BONSAI_CUDA_TRY(cudaMemcpy(chunks, ch.data(), ch.size() * sizeof(int4), cudaMemcpyHostToDevice));
    BONSAI_CUDA_TRY(cudaMemset(sys_energy, 0, (size_t)ns * 8 * sizeof(double)));
    BONSAI_CUDA_TRY(cudaMemset(root_beg, 0, (size_t)(ns + 1) * sizeof(int)));
    theta_mode = 0;  // angles, precision and block steps are set again for the ensemble
    precision = 0;
    release_lo();
    bts_K = -1;
    release_bts();
    return 0;
  }

  // eager build that grows the cell arrays until the tree fits
  int build_checked(int nleaf) {
    for (int attempt = 0; attempt < 4; attempt++) {
      enq_build(nleaf);
      int nc = 0;
      BONSAI_CUDA_TRY(cudaMemcpyAsync(&nc, &info->ncells, sizeof(int), cudaMemcpyDeviceToHost, st));
      BONSAI_CUDA_TRY(cudaStreamSynchronize(st));
      if (nc <= cap_cells) return 0;
      const int rc = alloc_cells(nc + nc / 4 + 4096);
      if (rc) return rc;
      BONSAI_CUDA_TRY(cudaMemsetAsync(&info->status, 0, sizeof(int), st));
    }
    return BONSAI_STATUS_CELL_CAPACITY;
  }

  // ---------------- stages (enqueue only) ----------------
  void enq_build(int nleaf) {
    enq_keys();
    enq_tree(nleaf);
  }
  void enq_keys() {
    if (nsys > 1) {
      launch_sys_keys(pos[par], chunks, nchunks, chunk_beg, nsys, sys_box_part, sys_box, ph_table, tkey, pkey,
                      &info->status, nsm * 8, st);
    } else {
      cudaMemsetAsync(box_ticket, 0, sizeof(unsigned), st);
      k_box<<<box_blocks, 256, 0, st>>>(pos[par], n, box_partial, box_ticket, box, &info->status);
      k_keys<<<nsm * 8, 256, 0, st>>>(pos[par], n, box, ph_table, tkey, pkey);
    }
  }
  void enq_tree(int nleaf) {
    radix_sort_pairs(tkey, kalt, tperm, valt, nullptr, n, sort_counts, &info->status, 8, so(), nsys, st);
    k_gather_pos<<<nsm * 8, 256, 0, st>>>(tperm, n, pos[par], jpos);
    if (precision) k_gather_pos<<<nsm * 8, 256, 0, st>>>(tperm, n, plo[par], jlo);
    build_tree(tkey, n, nleaf, cap_cells, cap_cells, dlev, chain, hist, info, cell_data, cell_parent, leaf_list,
               mp_count, so(), nsys, root_beg, st);
  }
  void enq_multipoles() {
    launch_multipoles(leaf_list, info, cell_data, cell_parent, jpos, 1.0f / prm.theta, rec, cell_box, cell_open,
                      cell_stage, cell_ls, mp_count, cap_cells, precision ? jlo : nullptr,
                      precision ? cell_lo : nullptr, nsm * 8, st);
  }
  void enq_groups(int ls, int ncrit) { enq_groups_on(ls, ncrit, st, kalt, valt, sort_counts); }
  void enq_groups_on(int ls, int ncrit, cudaStream_t s, unsigned long long* ka, int* va, unsigned* work) {
    radix_sort_pairs(pkey, ka, pperm, va, nullptr, n, work, &info->status, 8, so(), nsys, s);
    if (nsys > 1) {
      // ka (8 bytes per particle) is free after the sort: segment flags and indices
      unsigned* flag = reinterpret_cast<unsigned*>(ka);
      make_groups_sys(pkey, n, ls, ncrit, sys_off, nsys, flag, flag + n, seg_beg, seg_end, nseg, bsum, groups,
                      theta_mode ? gcap : n, info, s);
    } else {
      make_groups(pkey, n, ls, ncrit, g_count, g_seg, g_ng, bsum, groups, theta_mode ? gcap : n, info, s);
    }
    const int q = par ^ 1;
    k_gather_state<<<nsm * 8, 256, 0, s>>>(pperm, n, pos[par], vel[par], id[par], pos[q], vel[q], id[q]);
    if (precision) k_gather_pos<<<nsm * 8, 256, 0, s>>>(pperm, n, plo[par], plo[q]);
    acc_in_state_order = false;
    if (bts_K >= 0 && bts_gathering) {
      // levels and the accelerations of inactive particles travel with them
      launch_gather_u8(pperm, n, lev[par], lev[q], nsm * 8, s);
      k_gather_pos<<<nsm * 8, 256, 0, s>>>(pperm, n, acc, acc_alt);
      std::swap(acc, acc_alt);
      acc_in_state_order = true;
    } else {
      bts_ready = false;  // the levels no longer follow the particle order
    }
    par = q;
  }
  // keys, then the tree branch (handle's stream) and the group branch (st2)
  // concurrently; both only read the keys and the current state.  The two
  // sorts run side by side: a one-sweep pass is latency-bound (~30 % of HBM
  // bandwidth), so two at once beat one after the other (build phase at
  // N = 2^24: 5.66 ms, 5.82 ms with the group branch forked after the
  // tree-key sort).
  void enq_build_groups(int nleaf, int ls, int ncrit) {
    enq_keys();
    cudaEventRecord(ev_fork, st);
    cudaStreamWaitEvent(st2, ev_fork, 0);
    enq_tree(nleaf);
    enq_multipoles();
    enq_groups_on(ls, ncrit, st2, kalt2, valt2, sort_counts2);
    cudaEventRecord(ev_join, st2);
    cudaStreamWaitEvent(st, ev_join, 0);
  }
  void enq_forces(int ncrit) {
    const int k = walk_variant(ncrit, walk_layout);
    cudaMemsetAsync(group_counter, 0, sizeof(unsigned), st);
    cudaMemsetAsync(stats, 0, 4 * sizeof(unsigned long long), st);
    const float* ginv = nullptr;
    RelativeArgs rel;
    rel.acc_valid = acc_valid;
    if (theta_mode == 1 || theta_mode == 3) {
      // the previous evaluation's accelerations and statistics, through this
      // step's PH permutation
      const PrevEval prev = prev_eval();
      launch_group_features(groups, info, pos[par], pkey, rec, nsys > 1 ? sys_box : box, n, ncrit, prm.eps,
                            group_feat, so(), nsys, root_beg, prev, group_amag, nsm * 8, st);
      if (theta_mode == 1)
        launch_mlp_infer(group_feat, mlp_wh, info, theta_lo, theta_hi, group_amag, acc_valid, 1.0f / theta_bound,
                         1.0f / prm.theta, kStartAlpha, group_inv, group_tau, nsm * 4, st);
      else
        launch_relative_tau(info, group_amag, acc_valid, rel_alpha, 1.0f / theta_bound, 1.0f / prm.theta,
                            group_inv, group_tau, nsm * 4, st);
      ginv = group_inv;
      rel.tau = group_tau;
    } else if (theta_mode == 2) {
      ginv = group_inv;
      rel.tau = tau_on ? group_tau : nullptr;
    }
    if (ginv && theta_mode != 3) {
      // the per-group statistics feed the learned form's next features (mode
      // 3 has one parameter and no features; mode 2 records them for training)
      rel.stats = group_stats;
      rel.part_gid = part_gid;
    }
    launch_walk(k, walk_blocks[k], groups, info, pos[par], jpos, cell_data, cell_open, cell_stage, cell_ls,
                ginv, prm.eps * prm.eps, acc, ring, kRingCap, group_counter, stats, &info->status, so(), nsys, root_beg,
                precision ? plo[par] : nullptr, jlo, cell_lo, ginv ? group_counts : nullptr,
                walk_list_on ? walk_list : nullptr, walk_list_on ? walk_list_n : nullptr, rel, st);
    acc_in_state_order = true;
  }
  void enq_move(bool write) {
    launch_move_wrapper(write);
  }
  void launch_move_wrapper(bool write);

  void enq_step() {
    enq_build_groups(cur_nleaf, cur_ls, cur_ncrit);
    enq_forces(cur_ncrit);
    enq_move(true);
  }

  void enq_phase(int k) {
    if (k == 0) {
      enq_build_groups(cur_nleaf, cur_ls, cur_ncrit);
    } else if (k == 1) {
      enq_forces(cur_ncrit);
    } else {
      enq_move(true);
    }
  }

  int capture_graphs() {
    release_graphs();
    const int par0 = par;
    graph_kernels = 0;
    for (int p = 0; p < 2; p++) {
      par = p;
      for (int k = 0; k < 3; k++) {
        cudaGraph_t g = nullptr;
        BONSAI_CUDA_TRY(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
        enq_phase(k);
        cudaError_t e = cudaStreamEndCapture(st, &g);
        if (e != cudaSuccess) { par = par0; return -(int)e - 1000; }
        if (p == 0) {
          size_t nn = 0;
          cudaGraphGetNodes(g, nullptr, &nn);
          std::vector<cudaGraphNode_t> nodes(nn);
          cudaGraphGetNodes(g, nodes.data(), &nn);
          for (size_t q = 0; q < nn; q++) {
            cudaGraphNodeType ty;
            cudaGraphNodeGetType(nodes[q], &ty);
            graph_kernels += (ty == cudaGraphNodeTypeKernel);
          }
        }
        e = cudaGraphInstantiate(&gexec[p][k], g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) { par = par0; return -(int)e - 1000; }
      }
    }
    par = par0;
    graph_ok = true;
    return 0;
  }

  int launch_graph_step(cudaEvent_t* ev) {
    for (int k = 0; k < 3; k++) {
      if (ev) BONSAI_CUDA_TRY(cudaEventRecord(ev[k], st));
      BONSAI_CUDA_TRY(cudaGraphLaunch(gexec[par][k], st));
    }
    if (ev) BONSAI_CUDA_TRY(cudaEventRecord(ev[3], st));
    par ^= 1;
    return 0;
  }

  // Times `steps` graph steps (after one warm-up step) of every candidate
  // (nLeaf, nCrit, walk layout) on the current particles, restoring them
  // before each trial and at the end, and keeps the fastest.
  int autotune(const int* nl, int nnl, const int* nc, int nnc, int steps, float* results, int* best) {
    const size_t N = (size_t)n;
    float4 *sp = nullptr, *sv = nullptr, *sl = nullptr;
    int* si = nullptr;
    int closing0 = 0;
    BONSAI_CUDA_TRY(dalloc(&sp, N));
    BONSAI_CUDA_TRY(dalloc(&sv, N));
    BONSAI_CUDA_TRY(dalloc(&si, N));
    if (precision) BONSAI_CUDA_TRY(dalloc(&sl, N));
    BONSAI_CUDA_TRY(cudaMemcpyAsync(sp, pos[par], N * sizeof(float4), cudaMemcpyDeviceToDevice, st));
    BONSAI_CUDA_TRY(cudaMemcpyAsync(sv, vel[par], N * sizeof(float4), cudaMemcpyDeviceToDevice, st));
    BONSAI_CUDA_TRY(cudaMemcpyAsync(si, id[par], N * sizeof(int), cudaMemcpyDeviceToDevice, st));
    if (precision) BONSAI_CUDA_TRY(cudaMemcpyAsync(sl, plo[par], N * sizeof(float4), cudaMemcpyDeviceToDevice, st));
    BONSAI_CUDA_TRY(cudaMemcpyAsync(&closing0, closing, sizeof(int), cudaMemcpyDeviceToHost, st));
    BONSAI_CUDA_TRY(cudaStreamSynchronize(st));
    auto restore = [&]() -> int {
      BONSAI_CUDA_TRY(cudaMemcpyAsync(pos[par], sp, N * sizeof(float4), cudaMemcpyDeviceToDevice, st));
      BONSAI_CUDA_TRY(cudaMemcpyAsync(vel[par], sv, N * sizeof(float4), cudaMemcpyDeviceToDevice, st));
      BONSAI_CUDA_TRY(cudaMemcpyAsync(id[par], si, N * sizeof(int), cudaMemcpyDeviceToDevice, st));
      if (precision) BONSAI_CUDA_TRY(cudaMemcpyAsync(plo[par], sl, N * sizeof(float4), cudaMemcpyDeviceToDevice, st));
      BONSAI_CUDA_TRY(cudaMemcpyAsync(closing, &closing0, sizeof(int), cudaMemcpyHostToDevice, st));
      BONSAI_CUDA_TRY(cudaMemsetAsync(acc_valid, 0, 2 * sizeof(int), st));
      return 0;
    };
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    BONSAI_CUDA_TRY(cudaEventCreate(&e0));
    BONSAI_CUDA_TRY(cudaEventCreate(&e1));
    float best_ms = 3.0e38f;
    int bl = cur_nleaf, bc = cur_ncrit, blay = walk_layout;
    int rc = 0;
    for (int lay = 0; lay < 2 && rc >= 0; lay++)
      for (int a = 0; a < nnl && rc >= 0; a++)
        for (int b = 0; b < nnc && rc >= 0; b++) {
          const int idx = (lay * nnl + a) * nnc + b;
          if (results) results[idx] = -1.0f;
          if (nl[a] < 1 || nl[a] > 64 || nc[b] < 1 || nc[b] > 128) continue;
          if (lay == 0 && nc[b] > 64) continue;  // no half-warp layout above 64: same as layout 1
          rc = restore();
          if (rc) break;
          cur_nleaf = nl[a];
          cur_ncrit = nc[b];
          walk_layout = lay;
          release_graphs();
          rc = build_checked(cur_nleaf);
          if (rc > 0) { rc = read_status(true) < 0 ? -1 : 0; continue; }
          if (rc) break;
          rc = capture_graphs();
          if (rc) break;
          rc = launch_graph_step(nullptr);
          if (rc) break;
          cudaEventRecord(e0, st);
          for (int k = 0; k < steps && !rc; k++) rc = launch_graph_step(nullptr);
          cudaEventRecord(e1, st);
          if (rc) break;
          const int status = read_status(true);
          if (status < 0) { rc = status; break; }
          float ms = 0.f;
          cudaEventElapsedTime(&ms, e0, e1);
          if (status != 0) continue;
          ms /= (float)steps;
          if (results) results[idx] = ms;
          if (ms < best_ms) { best_ms = ms; bl = cur_nleaf; bc = cur_ncrit; blay = lay; }
        }
    if (rc >= 0) rc = restore();
    if (rc >= 0) rc = (int)cudaStreamSynchronize(st) == 0 ? 0 : -1000 - (int)cudaGetLastError();
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    dfree(&sp); dfree(&sv); dfree(&si); dfree(&sl);
    cur_nleaf = bl;
    cur_ncrit = bc;
    walk_layout = blay;
    prm.nleaf = bl;
    prm.ncrit = bc;
    release_graphs();
    built = mp_done = grouped = forced = moved_after_forces = false;
    if (best) { best[0] = bl; best[1] = bc; best[2] = blay; }
    return rc;
  }

  // Block time steps over nsteps big steps of prm.dt (eager launches).
  int block_steps(int nsteps) {
    bts_gathering = true;
    const int rc = block_steps_impl(nsteps);
    bts_gathering = false;
    return rc;
  }
  int block_steps_impl(int nsteps) {
    const int nb = nsm * 8;
    float4* lo_p = nullptr;
    if (!bts_ready) {
      // forces at the start, any pending closing kick, first levels
      int rc = build_checked(cur_nleaf);
      if (rc) return rc;
      enq_multipoles();
      enq_groups(cur_ls, cur_ncrit);
      walk_list_on = false;
      enq_forces(cur_ncrit);
      launch_closing_kick(vel[par], acc, n, prm.dt, closing, nsm * 4, st);
      launch_bts_close(vel[par], acc, lev[par], n, prm.dt, bts_K, 0, bts_eta, prm.eps, 1, nb, st);
      bts_ready = true;
    }
    const int nsub = 1 << bts_K;
    int maxl = bts_K;
    for (int b = 0; b < nsteps; b++) {
      for (int s = 0; s < nsub; s++) {
        lo_p = precision ? plo[par] : nullptr;
        launch_bts_open_drift(pos[par], vel[par], acc, lev[par], n, prm.dt, bts_K, s, lo_p, nb, st);
        // the particles ending at s + 1 have level >= K - tz(s + 1); when none
        // is that fine, the substep is the drift alone (nothing else changes)
        if (bts_K > 0 && s + 1 < nsub) {
          launch_max_level(lev[par], n, max_lev, nb, st);
          BONSAI_CUDA_TRY(cudaMemcpyAsync(&maxl, max_lev, sizeof(int), cudaMemcpyDeviceToHost, st));
          BONSAI_CUDA_TRY(cudaStreamSynchronize(st));
          if (maxl < bts_K - (__builtin_ctz((unsigned)(s + 1)))) continue;
        }
        enq_build_groups(cur_nleaf, cur_ls, cur_ncrit);
        launch_bts_active_groups(groups, info, lev[par], bts_K, s + 1, walk_list, walk_list_n, nb, st);
        walk_list_on = true;
        enq_forces(cur_ncrit);
        walk_list_on = false;
        launch_bts_close(vel[par], acc, lev[par], n, prm.dt, bts_K, s + 1, bts_eta, prm.eps, 0, nb, st);
      }
      // energies at the synchronised end of the big step (closing flag is 0)
      enq_move(false);
    }
    return 0;
  }

  int read_status(bool clear) {
    int s = 0;
    cudaError_t e = cudaMemcpyAsync(&s, &info->status, sizeof(int), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return -(int)e - 1000;
    if (clear && s) {
      e = cudaMemsetAsync(&info->status, 0, sizeof(int), st);
      if (e != cudaSuccess) return -(int)e - 1000;
    }
    return s;
  }
};

void Handle::launch_move_wrapper(bool write) {
  if (nsys > 1)
    launch_move_sys(pos[par], vel[par], acc, chunks, nchunks, chunk_beg, nsys, prm.dt, closing, prm.eps, write ? 1 : 0,
                    chunk_energy, move_blocks, move_ticket, energies, sys_energy, st, precision ? plo[par] : nullptr);
  else
    launch_move(pos[par], vel[par], acc, n, prm.dt, closing, prm.eps, write ? 1 : 0, move_partial, move_blocks,
                move_ticket, energies, st, precision ? plo[par] : nullptr);
}

Handle* H(bonsai_handle h) { return reinterpret_cast<Handle*>(h); }

int check_params(const bonsai_params* p) {
  if (!p) return BONSAI_ERR_ARG;
  // eps > 0: every particle's own term is part of its sum (as in the reference), singular at eps = 0
  if (!(p->theta > 0.f) || !(p->eps > 0.f) || !std::isfinite(p->dt)) return BONSAI_ERR_ARG;
  if (p->nleaf < 1 || p->nleaf > 64) return BONSAI_ERR_ARG;
  if (p->ncrit < 1 || p->ncrit > 128) return BONSAI_ERR_ARG;
  if (p->level_split < 1 || p->level_split > kMaxLevelSplit) return BONSAI_ERR_ARG;
  return 0;
}

int last_cuda(void) {
  const cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? 0 : -(int)e - 1000;
}

}  // namespace

// Plummer initial conditions (host): plummer.cpp
extern "C" int bonsai_plummer_impl(long n, unsigned int seed, float* pos4, float* vel4);
// Tipsy snapshots (host): tipsy.cpp
extern "C" int bonsai_read_tipsy_impl(const char* path, double* time, int* n, float* pos4, float* vel4, int* ids);
extern "C" int bonsai_write_tipsy_impl(const char* path, double time, int n, int ndark, const float* pos4,
                                       const float* vel4, const int* ids);
// composite galaxy and clustered field (host): ics.cpp
extern "C" int bonsai_galaxy_impl(long n, unsigned long long seed, double* pos4, float* vel4);
extern "C" int bonsai_clustered_field_impl(long n, unsigned long long seed, int nclusters, float* pos4, float* vel4);

extern "C" {

void bonsai_default_params(bonsai_params* p) {
  if (!p) return;
  p->theta = 0.75f;
  p->eps = 0.01f;
  p->nleaf = 16;
  p->ncrit = 64;
  p->level_split = 5;
  p->dt = 1.0f / 64.0f;
  p->device = 0;
}

int bonsai_create(const bonsai_params* p, bonsai_handle* out) {
  if (!out) return BONSAI_ERR_ARG;
  *out = nullptr;
  int rc = check_params(p);
  if (rc) return rc;
  Handle* h = new Handle();
  rc = h->init(p);
  if (rc) { delete h; return rc; }
  *out = reinterpret_cast<bonsai_handle>(h);
  return 0;
}

int bonsai_destroy(bonsai_handle hh) {
  Handle* h = H(hh);
  if (!h) return BONSAI_ERR_HANDLE;
  cudaSetDevice(h->dev);
  delete h;
  return 0;
}

int bonsai_alloc(bonsai_handle hh, int n) {
  Handle* h = H(hh);
  if (!h) return BONSAI_ERR_HANDLE;
  if (n < 1) return BONSAI_ERR_ARG;
  BONSAI_CUDA_TRY(cudaSetDevice(h->dev));
  return h->alloc(n);
}

int bonsai_set_params(bonsai_handle hh, const bonsai_params* p) {
  Handle* h = H(hh);
  if (!h) return BONSAI_ERR_HANDLE;
  const int rc = check_params(p);
  if (rc) return rc;
  if (p->device != h->dev) return BONSAI_ERR_ARG;
  h->prm = *p;
  h->cur_nleaf = p->nleaf;
  h->cur_ncrit = p->ncrit;
  h->cur_ls = p->level_split;
  h->release_graphs();
  return 0;
}

static int set_particles_impl(Handle* h, const float* pos4, const float* vel4, int n, cudaMemcpyKind kind) {
  if (!h) return BONSAI_ERR_HANDLE;
  if (!pos4 || !vel4 || n < 1) return BONSAI_ERR_ARG;
  BONSAI_CUDA_TRY(cudaSetDevice(h->dev));
  if (n != h->n) {
    const int rc = h->alloc(n);
    if (rc) return rc;
  }
  const size_t bytes = (size_t)n * sizeof(float4);
  BONSAI_CUDA_TRY(cudaMemcpyAsync(h->pos[h->par], pos4, bytes, kind, h->st));
  BONSAI_CUDA_TRY(cudaMemcpyAsync(h->vel[h->par], vel4, bytes, kind, h->st));
  k_iota<<<h->nsm * 4, 256, 0, h->st>>>(h->id[h->par], n);
  if (h->precision) BONSAI_CUDA_TRY(cudaMemsetAsync(h->plo[h->par], 0, bytes, h->st));  // float input: lo = 0
  BONSAI_CUDA_TRY(cudaMemsetAsync(h->closing, 0, sizeof(int), h->st));
  BONSAI_CUDA_TRY(cudaMemsetAsync(h->acc_valid, 0, 2 * sizeof(int), h->st));  // no previous accelerations
  h->built = h->mp_done = h->grouped = h->forced = h->moved_after_forces = false;
  h->bts_ready = false;
  return last_cuda();
}

int bonsai_set_particles(bonsai_handle hh, const float* pos4, const float* vel4, int n) {
  return set_particles_impl(H(hh), pos4, vel4, n, cudaMemcpyHostToDevice);
}
int bonsai_set_particles_device(bonsai_handle hh, const float* pos4, const float* vel4, int n) {
  return set_particles_impl(H(hh), pos4, vel4, n, cudaMemcpyDeviceToDevice);
}

static int get_particles_impl(Handle* h, float* pos4, float* vel4, float* acc4, cudaMemcpyKind kind) {
  if (!h) return BONSAI_ERR_HANDLE;
  if (h->n == 0) return BONSAI_ERR_NOT_ALLOCATED;
  BONSAI_CUDA_TRY(cudaSetDevice(h->dev));
  const int n = h->n;
  const size_t bytes = (size_t)n * sizeof(float4);
  float4* tmp = h->pos[h->par ^ 1];  // the idle state buffer
  const float4* src[3] = {h->pos[h->par], h->vel[h->par], h->acc};
  float* dst[3] = {pos4, vel4, acc4};
  for (int k = 0; k < 3; k++) {
    if (!dst[k]) continue;
    k_scatter_by_id<<<h->nsm * 8, 256, 0, h->st>>>(h->id[h->par], n, src[k], tmp);
    BONSAI_CUDA_TRY(cudaMemcpyAsync(dst[k], tmp, bytes, kind, h->st));
  }
  BONSAI_CUDA_TRY(cudaStreamSynchronize(h->st));
  return last_cuda();
}

int bonsai_get_particles(bonsai_handle hh, float* pos4, float* vel4, float* acc4) {
  return get_particles_impl(H(hh), pos4, vel4, acc4, cudaMemcpyDeviceToHost);
}
int bonsai_get_particles_device(bonsai_handle hh, float* pos4, float* vel4, float* acc4) {
  return get_particles_impl(H(hh), pos4, vel4, acc4, cudaMemcpyDeviceToDevice);
}

int bonsai_set_particles_async(bonsai_handle hh, const float* pos4, const float* vel4, int n) {
  Handle* h = H(hh);
  if (!h) return BONSAI_ERR_HANDLE;
  if (!pos4 || !vel4 || n < 1) return BONSAI_ERR_ARG;
  if (h->n == 0) return BONSAI_ERR_NOT_ALLOCATED;
  if (n != h->n) return BONSAI_ERR_ARG;  // no reallocation on the asynchronous path
  BONSAI_CUDA_TRY(cudaSetDevice(h->dev));
  const size_t bytes = (size_t)n * sizeof(float4);
  if (!h->in_pos) {
    BONSAI_CUDA_TRY(dalloc(&h->in_pos, (size_t)n));
    BONSAI_CUDA_TRY(dalloc(&h->in_vel, (size_t)n));
  }
  // upload once the previous upload has been consumed
  BONSAI_CUDA_TRY(cudaStreamWaitEvent(h->st_h2d, h->ev_in_consumed, 0));
  BONSAI_CUDA_TRY(cudaMemcpyAsync(h->in_pos, pos4, bytes, cudaMemcpyHostToDevice, h->st_h2d));
  BONSAI_CUDA_TRY(cudaMemcpyAsync(h->in_vel, vel4, bytes, cudaMemcpyHostToDevice, h->st_h2d));
  BONSAI_CUDA_TRY(cudaEventRecord(h->ev_in_copied, h->st_h2d));
  // the handle's stream takes the particles over when they have landed
  BONSAI_CUDA_TRY(cudaStreamWaitEvent(h->st, h->ev_in_copied, 0));
  BONSAI_CUDA_TRY(cudaMemcpyAsync(h->pos[h->par], h->in_pos, bytes, cudaMemcpyDeviceToDevice, h->st));
  BONSAI_CUDA_TRY(cudaMemcpyAsync(h->vel[h->par], h->in_vel, bytes, cudaMemcpyDeviceToDevice, h->st));
  BONSAI_CUDA_TRY(cudaEventRecord(h->ev_in_consumed, h->st));
  k_iota<<<h->nsm * 4, 256, 0, h->st>>>(h->id[h->par], n);
  if (h->precision) BONSAI_CUDA_TRY(cudaMemsetAsync(h->plo[h->par], 0, bytes, h->st));
  BONSAI_CUDA_TRY(cudaMemsetAsync(h->closing, 0, sizeof(int), h->st));
  BONSAI_CUDA_TRY(cudaMemsetAsync(h->acc_valid, 0, 2 * sizeof(int), h->st));
  h->built = h->mp_done = h->grouped = h->forced = h->moved_after_forces = false;
  h->bts_ready = false;
  return last_cuda();
}

int bonsai_get_particles_async(bonsai_handle hh, float* pos4, float* vel4, float* acc4) {
  Handle* h = H(hh);
  if (!h) return BONSAI_ERR_HANDLE;
  if (h->n == 0) return BONSAI_ERR_NOT_ALLOCATED;
  BONSAI_CUDA_TRY(cudaSetDevice(h->dev));
  const int n = h->n;
  const size_t bytes = (size_t)n * sizeof(float4);
  const int slot = h->out_slot;
  h->out_slot ^= 1;
  const float4* src[3] = {h->pos[h->par], h->vel[h->par], h->acc};
  float* dst[3] = {pos4, vel4, acc4};
  // the slot is free once its previous download has finished
  BONSAI_CUDA_TRY(cudaStreamWaitEvent(h->st, h->ev_out_done[slot], 0));
  for (int a = 0; a < 3; a++) {
    if (!dst[a]) continue;
    if (!h->out_buf[slot][a]) BONSAI_CUDA_TRY(dalloc(&h->out_buf[slot][a], (size_t)n));
    k_scatter_by_id<<<h->nsm * 8, 256, 0, h->st>>>(h->id[h->par], n, src[a], h->out_buf[slot][a]);
  }
  BONSAI_CUDA_TRY(cudaEventRecord(h->ev_out_ready[slot], h->st));
  BONSAI_CUDA_TRY(cudaStreamWaitEvent(h->st_d2h, h->ev_out_ready[slot], 0));
  for (int a = 0; a < 3; a++)
    if (dst[a]) BONSAI_CUDA_TRY(cudaMemcpyAsync(dst[a], h->out_buf[slot][a], bytes, cudaMemcpyDeviceToHost, h->st_d2h));
  BONSAI_CUDA_TRY(cudaEventRecord(h->ev_out_done[slot], h->st_d2h));
  return last_cuda();
}

int bonsai_build_tree(bonsai_handle hh, int nleaf) {
  Handle* h = H(hh);
  if (!h) return BONSAI_ERR_HANDLE;
  if (h->n == 0) return BONSAI_ERR_NOT_ALLOCATED;
  if (nleaf < 1 || nleaf > 64) return BONSAI_ERR_ARG;
  BONSAI_CUDA_TRY(cudaSetDevice(h->dev));
  h->cur_nleaf = nleaf;
  {
    const int rc = h->build_checked(nleaf);
    if (rc) return rc;
  }
  h->built = h->ever_built = true;
  h->mp_done = h->grouped = h->forced = h->moved_after_forces = false;
  return last_cuda();
}

int bonsai_compute_multipoles(bonsai_handle hh) {
  Handle* h = H(hh);
  if (!h) return BONSAI_ERR_HANDLE;
  if (!h->built) return BONSAI_ERR_ORDER;
  BONSAI_CUDA_TRY(cudaSetDevice(h->dev));
  h->enq_multipoles();
  h->mp_done = h->ever_mp = true;
  return last_cuda();
}

int bonsai_make_groups(bonsai_handle hh, int level_split, int ncrit) {
  Handle* h = H(hh);
  if (!h) return BONSAI_ERR_HANDLE;
  if (!h->built) return BONSAI_ERR_ORDER;
  level_split = std::max(1, level_split);  // makeGroups.cu:259
  if (level_split > kMaxLevelSplit || ncrit < 1 || ncrit > 128) return BONSAI_ERR_ARG;
  BONSAI_CUDA_TRY(cudaSetDevice(h->dev));
  if (h->grouped) return BONSAI_ERR_ORDER;  // the state was already reordered for this tree
  h->cur_ls = level_split;
  h->cur_ncrit = ncrit;
  h->enq_groups(level_split, ncrit);
  h->grouped = true;
  return last_cuda();
}

int bonsai_compute_forces(bonsai_handle hh, int intcount, double* out) {
  Handle* h = H(hh);
  if (!h) return BONSAI_ERR_HANDLE;
  if (!h->built || !h->mp_done || !h->grouped) return BONSAI_ERR_ORDER;
  BONSAI_CUDA_TRY(cudaSetDevice(h->dev));
  h->enq_forces(h->cur_ncrit);
  h->forced = true;
  h->moved_after_forces = false;
  if (intcount && out) {
    unsigned long long s[4];
    BONSAI_CUDA_TRY(cudaMemcpyAsync(s, h->stats, sizeof(s), cudaMemcpyDeviceToHost, h->st));
    BONSAI_CUDA_TRY(cudaStreamSynchronize(h->st));
    out[0] = (double)s[1] / h->n;  // <direct>
    out[1] = (double)s[3];         // max direct
    out[2] = (double)s[0] / h->n;  // <approx>
    out[3] = (double)s[2];         // max approx
  }
  return last_cuda();
}

int bonsai_move_particles(bonsai_handle hh) {
  Handle* h = H(hh);
  if (!h) return BONSAI_ERR_HANDLE;
  if (!h->forced || h->moved_after_forces) return BONSAI_ERR_ORDER;
  BONSAI_CUDA_TRY(cudaSetDevice(h->dev));
  h->enq_move(true);
  h->moved_after_forces = true;
  h->built = h->mp_done = h->grouped = false;
  return last_cuda();
}

int bonsai_compute_energies(bonsai_handle hh, double* out) {
  Handle* h = H(hh);
  if (!h) return BONSAI_ERR_HANDLE;
  if (h->n == 0) return BONSAI_ERR_NOT_ALLOCATED;
  if (!h->forced) return BONSAI_ERR_ORDER;
  BONSAI_CUDA_TRY(cudaSetDevice(h->dev));
  if (!h->moved_after_forces) h->enq_move(false);
  double e[8];
  BONSAI_CUDA_TRY(cudaMemcpyAsync(e, h->energies, sizeof(e), cudaMemcpyDeviceToHost, h->st));
  BONSAI_CUDA_TRY(cudaStreamSynchronize(h->st));
  if (out) std::memcpy(out, e, sizeof(e));
  return last_cuda();
}

int bonsai_step(bonsai_handle hh, int nsteps, int use_graph) {
  Handle* h = H(hh);
  if (!h) return BONSAI_ERR_HANDLE;
  if (h->n == 0) return BONSAI_ERR_NOT_ALLOCATED;
  if (nsteps < 0) return BONSAI_ERR_ARG;
  BONSAI_CUDA_TRY(cudaSetDevice(h->dev));
  if (use_graph && !h->graph_ok) {
    // size the cell arrays on the current particles before freezing pointers
    int rc = h->build_checked(h->cur_nleaf);
    if (rc) return rc;
    rc = h->capture_graphs();
    if (rc) return rc;
  }
  for (int s = 0; s < nsteps; s++) {
    if (use_graph) {
      const int rc = h->launch_graph_step(nullptr);
      if (rc) return rc;
    } else {
      h->enq_step();
    }
  }
  if (nsteps > 0) {
    h->built = h->mp_done = h->grouped = false;
    h->ever_built = h->ever_mp = true;
    h->forced = h->moved_after_forces = true;
  }
  return last_cuda();
}

int bonsai_step_timed(bonsai_handle hh, int nsteps, float* phase_ms) {
  Handle* h = H(hh);
  if (!h) return BONSAI_ERR_HANDLE;
  if (h->n == 0) return BONSAI_ERR_NOT_ALLOCATED;
  if (nsteps < 1 || !phase_ms) return BONSAI_ERR_ARG;
  BONSAI_CUDA_TRY(cudaSetDevice(h->dev));
  if (!h->graph_ok) {
    int rc = h->build_checked(h->cur_nleaf);
    if (rc) return rc;
    rc = h->capture_graphs();
    if (rc) return rc;
  }
  std::vector<cudaEvent_t> ev((size_t)4 * nsteps);
  for (auto& e : ev) BONSAI_CUDA_TRY(cudaEventCreate(&e));
  int rc = 0;
  for (int s = 0; s < nsteps && !rc; s++) rc = h->launch_graph_step(&ev[(size_t)4 * s]);
  if (!rc) {
    BONSAI_CUDA_TRY(cudaStreamSynchronize(h->st));
    for (int s = 0; s < nsteps; s++) {
      cudaEvent_t* e = &ev[(size_t)4 * s];
      cudaEventElapsedTime(&phase_ms[4 * s + 0], e[0], e[1]);
      cudaEventElapsedTime(&phase_ms[4 * s + 1], e[1], e[2]);
      cudaEventElapsedTime(&phase_ms[4 * s + 2], e[2], e[3]);
      cudaEventElapsedTime(&phase_ms[4 * s + 3], e[0], e[3]);
    }
    cudaEventElapsedTime(&phase_ms[4 * nsteps], ev[0], ev[(size_t)4 * nsteps - 1]);
  }
  for (auto& e : ev) cudaEventDestroy(e);
  h->built = h->mp_done = h->grouped = false;
  h->ever_built = h->ever_mp = true;
  h->forced = h->moved_after_forces = true;
  return rc ? rc : last_cuda();
}

int bonsai_set_systems(bonsai_handle hh, const int* counts, int nsys) {
  Handle* h = H(hh);
  if (!h) return BONSAI_ERR_HANDLE;
  if (!counts || nsys < 1 || nsys > 65536) return BONSAI_ERR_ARG;
  BONSAI_CUDA_TRY(cudaSetDevice(h->dev));
  return h->set_systems(counts, nsys);
}

int bonsai_get_system_energies(bonsai_handle hh, double* out) {
  Handle* h = H(hh);
  if (!h) return BONSAI_ERR_HANDLE;
  if (h->n == 0) return BONSAI_ERR_NOT_ALLOCATED;
  if (!h->forced) return BONSAI_ERR_ORDER;
  if (!out) return BONSAI_ERR_ARG;
  BONSAI_CUDA_TRY(cudaSetDevice(h->dev));
  if (!h->moved_after_forces) h->enq_move(false);
  const double* src = h->nsys > 1 ? h->sys_energy : h->energies;
  BONSAI_CUDA_TRY(cudaMemcpyAsync(out, src, (size_t)h->nsys * 8 * sizeof(double), cudaMemcpyDeviceToHost, h->st));
  BONSAI_CUDA_TRY(cudaStreamSynchronize(h->st));
  return last_cuda();
}

int bonsai_set_precision(bonsai_handle hh, int mode) {
  Handle* h = H(hh);
  if (!h) return BONSAI_ERR_HANDLE;
  if (mode < 0 || mode > 1) return BONSAI_ERR_ARG;
  BONSAI_CUDA_TRY(cudaSetDevice(h->dev));
  BONSAI_CUDA_TRY(cudaStreamSynchronize(h->st));
  h->release_graphs();
  h->precision = mode;
  return h->alloc_lo();
}

int bonsai_set_particles_f64(bonsai_handle hh, const double* pos4, const float* vel4, int n) {
  Handle* h = H(hh);
  if (!h) return BONSAI_ERR_HANDLE;
  if (!pos4 || !vel4 || n < 1) return BONSAI_ERR_ARG;
  const size_t N = (size_t)n;
  std::vector<float4> hi(N), lo(N);
  for (size_t i = 0; i < N; i++) {
    const double x = pos4[4 * i], y = pos4[4 * i + 1], z = pos4[4 * i + 2];
    hi[i] = make_float4((float)x, (float)y, (float)z, (float)pos4[4 * i + 3]);
    lo[i] = make_float4((float)(x - (double)hi[i].x), (float)(y - (double)hi[i].y), (float)(z - (double)hi[i].z), 0.f);
  }
  int rc = set_particles_impl(h, &hi[0].x, vel4, n, cudaMemcpyHostToDevice);
  if (rc) return rc;
  if (h->precision)
    BONSAI_CUDA_TRY(cudaMemcpyAsync(h->plo[h->par], lo.data(), N * sizeof(float4), cudaMemcpyHostToDevice, h->st));
  BONSAI_CUDA_TRY(cudaStreamSynchronize(h->st));  // the host staging vectors go out of scope
  return last_cuda();
}

int bonsai_get_particles_f64(bonsai_handle hh, double* pos4, float* vel4, float* acc4) {
  Handle* h = H(hh);
  if (!h) return BONSAI_ERR_HANDLE;
  if (h->n == 0) return BONSAI_ERR_NOT_ALLOCATED;
  int rc = get_particles_impl(h, nullptr, vel4, acc4, cudaMemcpyDeviceToHost);
  if (rc || !pos4) return rc;
  const size_t N = (size_t)h->n;
  std::vector<float4> hi(N), lo(N, make_float4(0.f, 0.f, 0.f, 0.f));
  rc = get_particles_impl(h, &hi[0].x, nullptr, nullptr, cudaMemcpyDeviceToHost);
  if (rc) return rc;
  if (h->precision) {
    float4* tmp = h->pos[h->par ^ 1];
    k_scatter_by_id<<<h->nsm * 8, 256, 0, h->st>>>(h->id[h->par], h->n, h->plo[h->par], tmp);
    BONSAI_CUDA_TRY(cudaMemcpyAsync(lo.data(), tmp, N * sizeof(float4), cudaMemcpyDeviceToHost, h->st));
    BONSAI_CUDA_TRY(cudaStreamSynchronize(h->st));
  }
  for (size_t i = 0; i < N; i++) {
    pos4[4 * i] = (double)hi[i].x + (double)lo[i].x;
    pos4[4 * i + 1] = (double)hi[i].y + (double)lo[i].y;
    pos4[4 * i + 2] = (double)hi[i].z + (double)lo[i].z;
    pos4[4 * i + 3] = (double)hi[i].w;
  }
  return last_cuda();
}

int bonsai_compute_forces_fp64(bonsai_handle hh, double* acc4, unsigned long long* stats4) {
  Handle* h = H(hh);
  if (!h) return BONSAI_ERR_HANDLE;
  if (!h->built || !h->mp_done || !h->grouped) return BONSAI_ERR_ORDER;
  if (h->theta_mode == 1 && !h->forced) return BONSAI_ERR_ORDER;  // the network's angles come from compute_forces
  if (h->cur_ncrit > 128) return BONSAI_ERR_ARG;
  BONSAI_CUDA_TRY(cudaSetDevice(h->dev));
  if (!h->acc64) {
    BONSAI_CUDA_TRY(dalloc(&h->acc64, (size_t)h->n));
    BONSAI_CUDA_TRY(dalloc(&h->acc64_tmp, (size_t)h->n));
  }
  BONSAI_CUDA_TRY(cudaMemsetAsync(h->group_counter, 0, sizeof(unsigned), h->st));
  BONSAI_CUDA_TRY(cudaMemsetAsync(h->stats, 0, 4 * sizeof(unsigned long long), h->st));
  const double e2 = (double)h->prm.eps * (double)h->prm.eps;
  const int nblocks = h->ring_warps / (256 / 32);
  launch_walk64(nblocks, h->groups, h->info, h->pos[h->par], h->precision ? h->plo[h->par] : nullptr, h->jpos,
                h->jlo, h->cell_data, h->cell_open, h->cell_lo, h->cell_ls, h->theta_mode ? h->group_inv : nullptr,
                (h->theta_mode == 1 || h->theta_mode == 3 || (h->theta_mode == 2 && h->tau_on)) ? h->group_tau : nullptr,
                h->rec, e2, h->acc64, h->ring, kRingCap, h->group_counter, h->stats, &h->info->status, h->so(),
                h->nsys, h->root_beg, h->st);
  if (acc4) {
    launch_scatter_d4(h->id[h->par], h->n, h->acc64, h->acc64_tmp, h->nsm * 8, h->st);
    BONSAI_CUDA_TRY(cudaMemcpyAsync(acc4, h->acc64_tmp, (size_t)h->n * sizeof(double4), cudaMemcpyDeviceToHost, h->st));
  }
  if (stats4) BONSAI_CUDA_TRY(cudaMemcpyAsync(stats4, h->stats, 4 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, h->st));
  BONSAI_CUDA_TRY(cudaStreamSynchronize(h->st));
  return last_cuda();
}

int bonsai_sync_velocities(bonsai_handle hh) {
  Handle* h = H(hh);
  if (!h) return BONSAI_ERR_HANDLE;
  if (h->n == 0) return BONSAI_ERR_NOT_ALLOCATED;
  BONSAI_CUDA_TRY(cudaSetDevice(h->dev));
  int rc = h->build_checked(h->cur_nleaf);
  if (rc) return rc;
  h->enq_multipoles();
  h->enq_groups(h->cur_ls, h->cur_ncrit);
  h->enq_forces(h->cur_ncrit);
  launch_closing_kick(h->vel[h->par], h->acc, h->n, h->prm.dt, h->closing, h->nsm * 4, h->st);
  h->built = h->mp_done = h->grouped = h->forced = true;
  h->ever_built = h->ever_mp = true;
  h->moved_after_forces = false;
  return last_cuda();
}

int bonsai_set_block_steps(bonsai_handle hh, int max_level, float eta) {
  Handle* h = H(hh);
  if (!h) return BONSAI_ERR_HANDLE;
  if (max_level > 16 || (max_level >= 0 && !(eta > 0.f))) return BONSAI_ERR_ARG;
  BONSAI_CUDA_TRY(cudaSetDevice(h->dev));
  BONSAI_CUDA_TRY(cudaStreamSynchronize(h->st));
  h->bts_K = max_level < 0 ? -1 : max_level;
  h->bts_eta = eta;
  h->release_graphs();
  return h->alloc_bts();
}

int bonsai_block_step(bonsai_handle hh, int nsteps) {
  Handle* h = H(hh);
  if (!h) return BONSAI_ERR_HANDLE;
  if (h->n == 0) return BONSAI_ERR_NOT_ALLOCATED;
  if (h->bts_K < 0) return BONSAI_ERR_ORDER;
  if (nsteps < 0) return BONSAI_ERR_ARG;
  BONSAI_CUDA_TRY(cudaSetDevice(h->dev));
  const int rc = h->block_steps(nsteps);
  if (rc) return rc;
  h->built = h->mp_done = h->grouped = false;
  h->ever_built = h->ever_mp = true;
  h->forced = h->moved_after_forces = true;
  return last_cuda();
}

int bonsai_get_levels(bonsai_handle hh, unsigned char* out) {
  Handle* h = H(hh);
  if (!h) return BONSAI_ERR_HANDLE;
  if (!out) return BONSAI_ERR_ARG;
  if (h->bts_K < 0 || !h->bts_ready) return BONSAI_ERR_ORDER;
  BONSAI_CUDA_TRY(cudaSetDevice(h->dev));
  unsigned char* tmp = h->lev[h->par ^ 1];
  launch_scatter_u8(h->id[h->par], h->n, h->lev[h->par], tmp, h->nsm * 8, h->st);
  BONSAI_CUDA_TRY(cudaMemcpyAsync(out, tmp, (size_t)h->n, cudaMemcpyDeviceToHost, h->st));
  BONSAI_CUDA_TRY(cudaStreamSynchronize(h->st));
  return last_cuda();
}

int bonsai_set_walk_layout(bonsai_handle hh, int layout) {
  Handle* h = H(hh);
  if (!h) return BONSAI_ERR_HANDLE;
  if (layout < 0 || layout > 1) return BONSAI_ERR_ARG;
  h->walk_layout = layout;
  h->release_graphs();
  return 0;
}

int bonsai_autotune(bonsai_handle hh, const int* nleaf, int n_nleaf, const int* ncrit, int n_ncrit, int steps,
                    float* results, int* best) {
  Handle* h = H(hh);
  if (!h) return BONSAI_ERR_HANDLE;
  if (h->n == 0) return BONSAI_ERR_NOT_ALLOCATED;
  if (!nleaf || !ncrit || n_nleaf < 1 || n_ncrit < 1 || steps < 1) return BONSAI_ERR_ARG;
  BONSAI_CUDA_TRY(cudaSetDevice(h->dev));
  return h->autotune(nleaf, n_nleaf, ncrit, n_ncrit, steps, results, best);
}

int bonsai_graph_kernel_count(bonsai_handle hh) {
  Handle* h = H(hh);
  if (!h) return BONSAI_ERR_HANDLE;
  if (h->n == 0) return BONSAI_ERR_NOT_ALLOCATED;
  BONSAI_CUDA_TRY(cudaSetDevice(h->dev));
  if (!h->graph_ok) {
    const int rc = h->capture_graphs();
    if (rc) return rc;
  }
  return h->graph_kernels;
}

int bonsai_get_stats(bonsai_handle hh, unsigned long long* out) {
  Handle* h = H(hh);
  if (!h) return BONSAI_ERR_HANDLE;
  if (!out) return BONSAI_ERR_ARG;
  BONSAI_CUDA_TRY(cudaSetDevice(h->dev));
  BONSAI_CUDA_TRY(cudaMemcpyAsync(out, h->stats, 4 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, h->st));
  BONSAI_CUDA_TRY(cudaStreamSynchronize(h->st));
  return 0;
}

int bonsai_synchronize(bonsai_handle hh) {
  Handle* h = H(hh);
  if (!h) return BONSAI_ERR_HANDLE;
  BONSAI_CUDA_TRY(cudaSetDevice(h->dev));
  BONSAI_CUDA_TRY(cudaStreamSynchronize(h->st_h2d));
  BONSAI_CUDA_TRY(cudaStreamSynchronize(h->st_d2h));
  const int c = last_cuda();
  if (c) return c;
  int st = h->read_status(true);
#ifdef BONSAI_CHECKS
  unsigned count = 0, site = 0;
  if (st >= 0 && bonsai_bounds_check(&count, &site, 0) == 1 && count > 0) st |= BONSAI_STATUS_BOUNDS;
#endif
  return st;
}

int bonsai_last_error(bonsai_handle hh) {
  Handle* h = H(hh);
  if (!h) return BONSAI_ERR_HANDLE;
  BONSAI_CUDA_TRY(cudaSetDevice(h->dev));
  const cudaError_t e = cudaPeekAtLastError();
  if (e != cudaSuccess) return -(int)e - 1000;
  return h->read_status(false);
}

int bonsai_step_graph(bonsai_handle hh, int nsteps) { return bonsai_step(hh, nsteps, 1); }

int bonsai_bounds_check(unsigned* count, unsigned* first_site, int reset) {
  unsigned tot = 0, first = 0;
#ifdef BONSAI_CHECKS
  BONSAI_CUDA_TRY(cudaDeviceSynchronize());
  int (*const words[])(unsigned*, bool) = {bounds_word_sort,   bounds_word_tree,   bounds_word_multipoles,
                                           bounds_word_groups, bounds_word_walk,   bounds_word_walk64,
                                           bounds_word_move,   bounds_word_learned};
  for (auto f : words) {
    unsigned w[2] = {0u, 0u};
    if (f(w, reset != 0) != 0) return -(int)cudaErrorUnknown - 1000;
    if (w[0] && !tot) first = w[1];
    tot += w[0];
  }
  if (count) *count = tot;
  if (first_site) *first_site = first;
  return 1;
#else
  (void)reset;
  if (count) *count = tot;
  if (first_site) *first_site = first;
  return 0;
#endif
}

int bonsai_bounds_selftest(int device) {
  BONSAI_CUDA_TRY(cudaSetDevice(device));
  cudaStream_t st;
  BONSAI_CUDA_TRY(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
  const int r = bounds_selftest(st);
  cudaStreamDestroy(st);
  return r;
}

int bonsai_copy_streams(bonsai_handle hh, void** h2d, void** d2h) {
  Handle* h = H(hh);
  if (!h) return BONSAI_ERR_HANDLE;
  if (h2d) *h2d = (void*)h->st_h2d;
  if (d2h) *d2h = (void*)h->st_d2h;
  return 0;
}

void* bonsai_stream(bonsai_handle hh) {
  Handle* h = H(hh);
  return h ? (void*)h->st : nullptr;
}

const char* bonsai_error_string(int code) {
  if (code == 0) return "ok";
  if (code <= -1000) return cudaGetErrorString((cudaError_t)(-(code + 1000)));
  switch (code) {
    case BONSAI_ERR_HANDLE: return "invalid handle";
    case BONSAI_ERR_NOT_ALLOCATED: return "particles not allocated";
    case BONSAI_ERR_ORDER: return "stage called before the stage it depends on";
    case BONSAI_ERR_ARG: return "invalid argument";
    case BONSAI_ERR_NO_DEVICE: return "no CUDA device";
    case BONSAI_ERR_IO: return "file could not be opened, read or written (or is not a Tipsy snapshot)";
    case BONSAI_ERR_TOO_LARGE: return "request exceeds the fixed scratch capacity (bonsai_direct_fp64_noalloc: ns <= 65536)";
    default: break;
  }
  if (code > 0) {
    if (code & BONSAI_STATUS_CELL_CAPACITY) return "cell capacity exceeded";
    if (code & BONSAI_STATUS_WALK_STACK) return "walk level list overflow";
    if (code & BONSAI_STATUS_NONFINITE) return "non-finite particle coordinate";
    if (code & BONSAI_STATUS_GROUP_CAPACITY) return "group capacity exceeded";
    if (code & BONSAI_STATUS_DEPTH) return "tree deeper than 21 levels (fat leaf kept)";
    if (code & BONSAI_STATUS_BAD_PARAM) return "bad parameter";
    if (code & BONSAI_STATUS_SORT_TIMEOUT) return "radix sort look-back wait timed out";
    if (code & BONSAI_STATUS_BOUNDS) return "index out of range (bounds-checked build; access skipped)";
  }
  return "unknown";
}

int bonsai_get_tree_info(bonsai_handle hh, bonsai_tree_info* out) {
  Handle* h = H(hh);
  if (!h) return BONSAI_ERR_HANDLE;
  if (!out) return BONSAI_ERR_ARG;
  BONSAI_CUDA_TRY(cudaSetDevice(h->dev));
  TreeInfo ti;
  BONSAI_CUDA_TRY(cudaMemcpyAsync(&ti, h->info, sizeof(ti), cudaMemcpyDeviceToHost, h->st));
  BONSAI_CUDA_TRY(cudaStreamSynchronize(h->st));
  out->ncells = ti.ncells;
  out->nleaves = ti.nleaves;
  out->nnodes = ti.nnodes;
  out->nlevels = ti.nlevels;
  out->ngroups = ti.ngroups;
  out->status = ti.status;
  for (int L = 0; L < 32; L++) { out->level_beg[L] = ti.level_beg[L]; out->level_end[L] = ti.level_end[L]; }
  return 0;
}

int bonsai_get_box(bonsai_handle hh, float* box4) {
  Handle* h = H(hh);
  if (!h) return BONSAI_ERR_HANDLE;
  if (!box4) return BONSAI_ERR_ARG;
  BONSAI_CUDA_TRY(cudaSetDevice(h->dev));
  const Box* b = h->nsys > 1 ? h->sys_box : h->box;  // an ensemble's first system
  BONSAI_CUDA_TRY(cudaMemcpyAsync(box4, b, 4 * sizeof(float), cudaMemcpyDeviceToHost, h->st));
  BONSAI_CUDA_TRY(cudaStreamSynchronize(h->st));
  return 0;
}

int bonsai_get_keys(bonsai_handle hh, uint64_t* tk, int* tp, uint64_t* pk, int* pp, int* ids) {
  Handle* h = H(hh);
  if (!h) return BONSAI_ERR_HANDLE;
  if (h->n == 0) return BONSAI_ERR_NOT_ALLOCATED;
  BONSAI_CUDA_TRY(cudaSetDevice(h->dev));
  const size_t N = (size_t)h->n;
  if (tk) BONSAI_CUDA_TRY(cudaMemcpyAsync(tk, h->tkey, N * 8, cudaMemcpyDeviceToHost, h->st));
  if (tp) BONSAI_CUDA_TRY(cudaMemcpyAsync(tp, h->tperm, N * 4, cudaMemcpyDeviceToHost, h->st));
  if (pk) BONSAI_CUDA_TRY(cudaMemcpyAsync(pk, h->pkey, N * 8, cudaMemcpyDeviceToHost, h->st));
  if (pp) BONSAI_CUDA_TRY(cudaMemcpyAsync(pp, h->pperm, N * 4, cudaMemcpyDeviceToHost, h->st));
  // ids of the order the build saw: the state buffer before the PH gather
  const int q = h->grouped ? (h->par ^ 1) : h->par;
  if (ids) BONSAI_CUDA_TRY(cudaMemcpyAsync(ids, h->id[q], N * 4, cudaMemcpyDeviceToHost, h->st));
  BONSAI_CUDA_TRY(cudaStreamSynchronize(h->st));
  return 0;
}

int bonsai_get_cells(bonsai_handle hh, uint32_t* cell_data, float* size4, float* mono4, float* quad0, float* quad1,
                     int* leaf_list, int* parent) {
  Handle* h = H(hh);
  if (!h) return BONSAI_ERR_HANDLE;
  if (!h->ever_built) return BONSAI_ERR_ORDER;
  BONSAI_CUDA_TRY(cudaSetDevice(h->dev));
  TreeInfo ti;
  BONSAI_CUDA_TRY(cudaMemcpyAsync(&ti, h->info, sizeof(ti), cudaMemcpyDeviceToHost, h->st));
  BONSAI_CUDA_TRY(cudaStreamSynchronize(h->st));
  const size_t C = (size_t)ti.ncells;
  if (cell_data) BONSAI_CUDA_TRY(cudaMemcpyAsync(cell_data, h->cell_data, C * 16, cudaMemcpyDeviceToHost, h->st));
  if (leaf_list)
    BONSAI_CUDA_TRY(cudaMemcpyAsync(leaf_list, h->leaf_list, (size_t)ti.nleaves * 4, cudaMemcpyDeviceToHost, h->st));
  if (parent) BONSAI_CUDA_TRY(cudaMemcpyAsync(parent, h->cell_parent, C * 4, cudaMemcpyDeviceToHost, h->st));
  if ((size4 || mono4 || quad0 || quad1) && C > 0) {
    if (!h->ever_mp) return BONSAI_ERR_ORDER;
    float4 *s = nullptr, *m = nullptr, *q0 = nullptr;
    float2* q1 = nullptr;
    BONSAI_CUDA_TRY(dalloc(&s, C));
    BONSAI_CUDA_TRY(dalloc(&m, C));
    BONSAI_CUDA_TRY(dalloc(&q0, C));
    BONSAI_CUDA_TRY(dalloc(&q1, C));
    k_multipoles_ref_layout<<<h->nsm * 4, 256, 0, h->st>>>(h->info, h->cell_open, h->rec, s, m, q0, q1);
    if (size4) BONSAI_CUDA_TRY(cudaMemcpyAsync(size4, s, C * 16, cudaMemcpyDeviceToHost, h->st));
    if (mono4) BONSAI_CUDA_TRY(cudaMemcpyAsync(mono4, m, C * 16, cudaMemcpyDeviceToHost, h->st));
    if (quad0) BONSAI_CUDA_TRY(cudaMemcpyAsync(quad0, q0, C * 16, cudaMemcpyDeviceToHost, h->st));
    if (quad1) BONSAI_CUDA_TRY(cudaMemcpyAsync(quad1, q1, C * 8, cudaMemcpyDeviceToHost, h->st));
    BONSAI_CUDA_TRY(cudaStreamSynchronize(h->st));
    dfree(&s); dfree(&m); dfree(&q0); dfree(&q1);
  }
  BONSAI_CUDA_TRY(cudaStreamSynchronize(h->st));
  return last_cuda();
}

int bonsai_get_groups(bonsai_handle hh, int* groups) {
  Handle* h = H(hh);
  if (!h) return BONSAI_ERR_HANDLE;
  if (!h->grouped && !h->forced) return BONSAI_ERR_ORDER;
  if (!groups) return BONSAI_ERR_ARG;
  BONSAI_CUDA_TRY(cudaSetDevice(h->dev));
  int ng = 0;
  BONSAI_CUDA_TRY(cudaMemcpyAsync(&ng, &h->info->ngroups, sizeof(int), cudaMemcpyDeviceToHost, h->st));
  BONSAI_CUDA_TRY(cudaStreamSynchronize(h->st));
  BONSAI_CUDA_TRY(cudaMemcpyAsync(groups, h->groups, (size_t)ng * 8, cudaMemcpyDeviceToHost, h->st));
  BONSAI_CUDA_TRY(cudaStreamSynchronize(h->st));
  return 0;
}

int bonsai_get_walk_arrays(bonsai_handle hh, float* ipos4, float* jpos4, float* acc4, int* ids) {
  Handle* h = H(hh);
  if (!h) return BONSAI_ERR_HANDLE;
  if (h->n == 0) return BONSAI_ERR_NOT_ALLOCATED;
  BONSAI_CUDA_TRY(cudaSetDevice(h->dev));
  const size_t N = (size_t)h->n;
  if (ipos4) BONSAI_CUDA_TRY(cudaMemcpyAsync(ipos4, h->pos[h->par], N * 16, cudaMemcpyDeviceToHost, h->st));
  if (jpos4) BONSAI_CUDA_TRY(cudaMemcpyAsync(jpos4, h->jpos, N * 16, cudaMemcpyDeviceToHost, h->st));
  if (acc4) BONSAI_CUDA_TRY(cudaMemcpyAsync(acc4, h->acc, N * 16, cudaMemcpyDeviceToHost, h->st));
  if (ids) BONSAI_CUDA_TRY(cudaMemcpyAsync(ids, h->id[h->par], N * 4, cudaMemcpyDeviceToHost, h->st));
  BONSAI_CUDA_TRY(cudaStreamSynchronize(h->st));
  return 0;
}

int bonsai_direct_fp64(bonsai_handle hh, const int* sample, int ns, int include_self, double* out) {
  Handle* h = H(hh);
  if (!h) return BONSAI_ERR_HANDLE;
  if (h->n == 0) return BONSAI_ERR_NOT_ALLOCATED;
  if (!sample || !out || ns < 1) return BONSAI_ERR_ARG;
  for (int s = 0; s < ns; s++)
    if (sample[s] < 0 || sample[s] >= h->n) return BONSAI_ERR_ARG;
  BONSAI_CUDA_TRY(cudaSetDevice(h->dev));
  const int nsplit = std::max(1, std::min(512, (h->nsm * 8 * 256) / std::max(ns, 1)));
  if (ns > h->direct_cap || !h->direct_part) {
    dfree(&h->direct_part); dfree(&h->direct_out); dfree(&h->direct_sample);
    BONSAI_CUDA_TRY(dalloc(&h->direct_part, (size_t)512 * ns * 4));
    BONSAI_CUDA_TRY(dalloc(&h->direct_out, (size_t)ns * 4));
    BONSAI_CUDA_TRY(dalloc(&h->direct_sample, (size_t)ns));
    h->direct_cap = ns;
  }
  // positions in caller order into the idle state buffer
  float4* tmp = h->pos[h->par ^ 1];
  k_scatter_by_id<<<h->nsm * 8, 256, 0, h->st>>>(h->id[h->par], h->n, h->pos[h->par], tmp);
  float4* tmp_lo = nullptr;
  if (h->precision) {
    tmp_lo = h->plo[h->par ^ 1];
    k_scatter_by_id<<<h->nsm * 8, 256, 0, h->st>>>(h->id[h->par], h->n, h->plo[h->par], tmp_lo);
  }
  BONSAI_CUDA_TRY(cudaMemcpyAsync(h->direct_sample, sample, (size_t)ns * 4, cudaMemcpyHostToDevice, h->st));
  const double e2 = (double)h->prm.eps * (double)h->prm.eps;
  if (h->nsys > 1)
    launch_direct_fp64_sys(tmp, h->sys_off, h->nsys, h->direct_sample, ns, e2, include_self, h->direct_out, h->st,
                           tmp_lo);
  else
    launch_direct_fp64(tmp, h->n, h->direct_sample, ns, e2, include_self, h->direct_part, nsplit, h->direct_out,
                       h->st, tmp_lo);
  BONSAI_CUDA_TRY(cudaMemcpyAsync(out, h->direct_out, (size_t)ns * 4 * sizeof(double), cudaMemcpyDeviceToHost, h->st));
  BONSAI_CUDA_TRY(cudaStreamSynchronize(h->st));
  return last_cuda();
}

int bonsai_set_theta_mode(bonsai_handle hh, int mode, float lo, float hi) {
  Handle* h = H(hh);
  if (!h) return BONSAI_ERR_HANDLE;
  if (mode < 0 || mode > 3 || !(hi >= lo)) return BONSAI_ERR_ARG;
  if (mode == 3 && !(lo > 0.f)) return BONSAI_ERR_ARG;  // alpha
  if (mode == 1 && !h->mlp_loaded) return BONSAI_ERR_ORDER;
  h->theta_mode = mode;
  h->theta_lo = lo;
  h->theta_hi = hi;
  if (mode == 3) h->rel_alpha = lo;
  h->release_graphs();
  return 0;
}

int bonsai_set_relative_bound(bonsai_handle hh, float theta_bound) {
  Handle* h = H(hh);
  if (!h) return BONSAI_ERR_HANDLE;
  if (!(theta_bound > 0.f) || !(theta_bound < 100.f)) return BONSAI_ERR_ARG;
  h->theta_bound = theta_bound;
  h->release_graphs();
  return 0;
}

int bonsai_set_mlp_weights(bonsai_handle hh, const float* w, int nw) {
  Handle* h = H(hh);
  if (!h) return BONSAI_ERR_HANDLE;
  if (!w || nw != kMlpWeights) return BONSAI_ERR_ARG;
  BONSAI_CUDA_TRY(cudaSetDevice(h->dev));
  if (!h->mlp_w) BONSAI_CUDA_TRY(dalloc(&h->mlp_w, (size_t)kMlpWeights));
  if (!h->mlp_wh) BONSAI_CUDA_TRY(cudaMalloc(&h->mlp_wh, (size_t)kMlpWeights * 2));
  BONSAI_CUDA_TRY(cudaMemcpyAsync(h->mlp_w, w, (size_t)kMlpWeights * 4, cudaMemcpyHostToDevice, h->st));
  launch_weights_to_half(h->mlp_w, h->mlp_wh, h->st);
  BONSAI_CUDA_TRY(cudaStreamSynchronize(h->st));
  h->mlp_loaded = true;
  return last_cuda();
}

int bonsai_set_group_theta(bonsai_handle hh, const float* theta, int ngroups) {
  Handle* h = H(hh);
  if (!h) return BONSAI_ERR_HANDLE;
  if (!h->grouped && !h->forced) return BONSAI_ERR_ORDER;
  if (!theta || ngroups < 1 || ngroups > h->gcap) return BONSAI_ERR_ARG;
  BONSAI_CUDA_TRY(cudaSetDevice(h->dev));
  int ng = 0;
  BONSAI_CUDA_TRY(cudaMemcpyAsync(&ng, &h->info->ngroups, sizeof(int), cudaMemcpyDeviceToHost, h->st));
  BONSAI_CUDA_TRY(cudaStreamSynchronize(h->st));
  if (ng != ngroups) return BONSAI_ERR_ARG;
  float* tmp = reinterpret_cast<float*>(h->group_feat);  // staging: the feature buffer holds >= G floats
  BONSAI_CUDA_TRY(cudaMemcpyAsync(tmp, theta, (size_t)ng * 4, cudaMemcpyHostToDevice, h->st));
  launch_fill_inv_theta(h->info, tmp, 0.f, h->group_inv, h->nsm * 4, h->st);
  BONSAI_CUDA_TRY(cudaStreamSynchronize(h->st));
  return last_cuda();
}

int bonsai_set_group_tau(bonsai_handle hh, const float* tau, int ngroups) {
  Handle* h = H(hh);
  if (!h) return BONSAI_ERR_HANDLE;
  if (!tau) {
    h->tau_on = false;
    h->release_graphs();
    return 0;
  }
  if (!h->grouped && !h->forced) return BONSAI_ERR_ORDER;
  if (ngroups < 1 || ngroups > h->gcap) return BONSAI_ERR_ARG;
  BONSAI_CUDA_TRY(cudaSetDevice(h->dev));
  int ng = 0;
  BONSAI_CUDA_TRY(cudaMemcpyAsync(&ng, &h->info->ngroups, sizeof(int), cudaMemcpyDeviceToHost, h->st));
  BONSAI_CUDA_TRY(cudaStreamSynchronize(h->st));
  if (ng != ngroups) return BONSAI_ERR_ARG;
  BONSAI_CUDA_TRY(cudaMemcpyAsync(h->group_tau, tau, (size_t)ng * 4, cudaMemcpyHostToDevice, h->st));
  BONSAI_CUDA_TRY(cudaStreamSynchronize(h->st));
  h->tau_on = true;
  h->release_graphs();
  return last_cuda();
}

int bonsai_get_group_features(bonsai_handle hh, float* out, int* ngroups) {
  Handle* h = H(hh);
  if (!h) return BONSAI_ERR_HANDLE;
  if (!h->grouped) return BONSAI_ERR_ORDER;
  if (!out || !ngroups) return BONSAI_ERR_ARG;
  BONSAI_CUDA_TRY(cudaSetDevice(h->dev));
  int ng = 0;
  BONSAI_CUDA_TRY(cudaMemcpyAsync(&ng, &h->info->ngroups, sizeof(int), cudaMemcpyDeviceToHost, h->st));
  BONSAI_CUDA_TRY(cudaStreamSynchronize(h->st));
  if (ng > h->gcap) return BONSAI_STATUS_GROUP_CAPACITY;
  launch_group_features(h->groups, h->info, h->pos[h->par], h->pkey, h->rec, h->nsys > 1 ? h->sys_box : h->box, h->n,
                        h->cur_ncrit, h->prm.eps, h->group_feat, h->so(), h->nsys, h->root_beg, h->prev_eval(),
                        h->group_amag, h->nsm * 8, h->st);
  BONSAI_CUDA_TRY(cudaMemcpyAsync(out, h->group_feat, (size_t)ng * kMlpFeatures * 4, cudaMemcpyDeviceToHost, h->st));
  BONSAI_CUDA_TRY(cudaStreamSynchronize(h->st));
  *ngroups = ng;
  return last_cuda();
}

int bonsai_get_group_scale(bonsai_handle hh, float* out) {
  Handle* h = H(hh);
  if (!h) return BONSAI_ERR_HANDLE;
  if (!out) return BONSAI_ERR_ARG;
  if (!h->grouped && !h->forced) return BONSAI_ERR_ORDER;
  BONSAI_CUDA_TRY(cudaSetDevice(h->dev));
  int ng = 0;
  BONSAI_CUDA_TRY(cudaMemcpyAsync(&ng, &h->info->ngroups, sizeof(int), cudaMemcpyDeviceToHost, h->st));
  BONSAI_CUDA_TRY(cudaStreamSynchronize(h->st));
  if (ng > h->gcap) return BONSAI_STATUS_GROUP_CAPACITY;
  BONSAI_CUDA_TRY(cudaMemcpyAsync(out, h->group_amag, (size_t)ng * 4, cudaMemcpyDeviceToHost, h->st));
  BONSAI_CUDA_TRY(cudaStreamSynchronize(h->st));
  return last_cuda();
}

int bonsai_get_group_interactions(bonsai_handle hh, unsigned* out) {
  Handle* h = H(hh);
  if (!h) return BONSAI_ERR_HANDLE;
  if (!out) return BONSAI_ERR_ARG;
  if (h->theta_mode == 0 || !h->forced) return BONSAI_ERR_ORDER;
  BONSAI_CUDA_TRY(cudaSetDevice(h->dev));
  int ng = 0;
  BONSAI_CUDA_TRY(cudaMemcpyAsync(&ng, &h->info->ngroups, sizeof(int), cudaMemcpyDeviceToHost, h->st));
  BONSAI_CUDA_TRY(cudaStreamSynchronize(h->st));
  if (ng > h->gcap) return BONSAI_STATUS_GROUP_CAPACITY;
  BONSAI_CUDA_TRY(cudaMemcpyAsync(out, h->group_counts, (size_t)ng * 8, cudaMemcpyDeviceToHost, h->st));
  BONSAI_CUDA_TRY(cudaStreamSynchronize(h->st));
  return 0;
}

int bonsai_get_group_theta(bonsai_handle hh, float* out) {
  Handle* h = H(hh);
  if (!h) return BONSAI_ERR_HANDLE;
  if (!out) return BONSAI_ERR_ARG;
  if (h->theta_mode == 0) return BONSAI_ERR_ORDER;
  BONSAI_CUDA_TRY(cudaSetDevice(h->dev));
  int ng = 0;
  BONSAI_CUDA_TRY(cudaMemcpyAsync(&ng, &h->info->ngroups, sizeof(int), cudaMemcpyDeviceToHost, h->st));
  BONSAI_CUDA_TRY(cudaStreamSynchronize(h->st));
  BONSAI_CUDA_TRY(cudaMemcpyAsync(out, h->group_inv, (size_t)ng * 4, cudaMemcpyDeviceToHost, h->st));
  BONSAI_CUDA_TRY(cudaStreamSynchronize(h->st));
  for (int g = 0; g < ng; g++) out[g] = 1.0f / out[g];
  return 0;
}

// standalone MLP training helpers (host arrays in and out)
struct MlpJob {
  float *X = nullptr, *y = nullptr, *w = nullptr, *g = nullptr, *m = nullptr, *v = nullptr, *scr = nullptr,
        *pred = nullptr;
  double* loss = nullptr;
  cudaStream_t st = nullptr;
  ~MlpJob() {
    dfree(&X); dfree(&y); dfree(&w); dfree(&g); dfree(&m); dfree(&v); dfree(&scr); dfree(&pred); dfree(&loss);
    if (st) cudaStreamDestroy(st);
  }
  int init(int device, const float* hX, const float* hy, int S, const float* hw) {
    BONSAI_CUDA_TRY(cudaSetDevice(device));
    BONSAI_CUDA_TRY(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    BONSAI_CUDA_TRY(dalloc(&X, (size_t)S * kMlpFeatures));
    BONSAI_CUDA_TRY(dalloc(&y, (size_t)S));
    BONSAI_CUDA_TRY(dalloc(&w, (size_t)kMlpWeights));
    BONSAI_CUDA_TRY(dalloc(&g, (size_t)kMlpWeights));
    BONSAI_CUDA_TRY(dalloc(&m, (size_t)kMlpWeights));
    BONSAI_CUDA_TRY(dalloc(&v, (size_t)kMlpWeights));
    BONSAI_CUDA_TRY(dalloc(&scr, mlp_train_scratch_floats(S)));
    BONSAI_CUDA_TRY(dalloc(&pred, (size_t)S));
    BONSAI_CUDA_TRY(dalloc(&loss, 1));
    BONSAI_CUDA_TRY(cudaMemcpyAsync(X, hX, (size_t)S * kMlpFeatures * 4, cudaMemcpyHostToDevice, st));
    if (hy) BONSAI_CUDA_TRY(cudaMemcpyAsync(y, hy, (size_t)S * 4, cudaMemcpyHostToDevice, st));
    BONSAI_CUDA_TRY(cudaMemcpyAsync(w, hw, (size_t)kMlpWeights * 4, cudaMemcpyHostToDevice, st));
    BONSAI_CUDA_TRY(cudaMemsetAsync(m, 0, (size_t)kMlpWeights * 4, st));
    BONSAI_CUDA_TRY(cudaMemsetAsync(v, 0, (size_t)kMlpWeights * 4, st));
    return 0;
  }
};

int bonsai_mlp_loss_grad(int device, const float* X, const float* y, int S, const float* w, float lo, float hi,
                         float over, float* grad, double* loss) {
  if (!X || !y || !w || S < 1 || !(hi > lo)) return BONSAI_ERR_ARG;
  MlpJob j;
  int rc = j.init(device, X, y, S, w);
  if (rc) return rc;
  mlp_loss_grad(j.X, j.y, S, j.w, lo, hi, over, j.scr, j.g, j.loss, j.st);
  if (grad) BONSAI_CUDA_TRY(cudaMemcpyAsync(grad, j.g, (size_t)kMlpWeights * 4, cudaMemcpyDeviceToHost, j.st));
  double l = 0;
  BONSAI_CUDA_TRY(cudaMemcpyAsync(&l, j.loss, sizeof(double), cudaMemcpyDeviceToHost, j.st));
  BONSAI_CUDA_TRY(cudaStreamSynchronize(j.st));
  if (loss) *loss = l / S;
  return last_cuda();
}

int bonsai_mlp_train(int device, const float* X, const float* y, int S, float* w, int epochs, float lr, float lo,
                     float hi, float over, double* loss) {
  if (!X || !y || !w || S < 1 || epochs < 0 || !(hi > lo)) return BONSAI_ERR_ARG;
  MlpJob j;
  int rc = j.init(device, X, y, S, w);
  if (rc) return rc;
  for (int e = 1; e <= epochs; e++) {
    mlp_loss_grad(j.X, j.y, S, j.w, lo, hi, over, j.scr, j.g, nullptr, j.st);
    mlp_adam_step(j.w, j.g, j.m, j.v, lr, e, j.st);
  }
  mlp_loss_grad(j.X, j.y, S, j.w, lo, hi, over, j.scr, j.g, j.loss, j.st);
  double l = 0;
  BONSAI_CUDA_TRY(cudaMemcpyAsync(w, j.w, (size_t)kMlpWeights * 4, cudaMemcpyDeviceToHost, j.st));
  BONSAI_CUDA_TRY(cudaMemcpyAsync(&l, j.loss, sizeof(double), cudaMemcpyDeviceToHost, j.st));
  BONSAI_CUDA_TRY(cudaStreamSynchronize(j.st));
  if (loss) *loss = l / S;
  return last_cuda();
}

int bonsai_mlp_predict(int device, const float* X, int S, const float* w, float lo, float hi, float* theta) {
  if (!X || !w || !theta || S < 1 || !(hi > lo)) return BONSAI_ERR_ARG;
  MlpJob j;
  int rc = j.init(device, X, nullptr, S, w);
  if (rc) return rc;
  BONSAI_CUDA_TRY(cudaMemsetAsync(j.pred, 0, (size_t)S * 4, j.st));
  mlp_predict(j.X, S, j.w, lo, hi, j.scr, j.pred, j.st);
  BONSAI_CUDA_TRY(cudaMemcpyAsync(theta, j.pred, (size_t)S * 4, cudaMemcpyDeviceToHost, j.st));
  BONSAI_CUDA_TRY(cudaStreamSynchronize(j.st));
  return last_cuda();
}

int bonsai_plummer(long n, unsigned int seed, float* pos4, float* vel4) {
  if (n < 1 || !pos4 || !vel4) return BONSAI_ERR_ARG;
  return bonsai_plummer_impl(n, seed, pos4, vel4);
}

int bonsai_read_tipsy(const char* path, double* time, int* n, float* pos4, float* vel4, int* ids) {
  return bonsai_read_tipsy_impl(path, time, n, pos4, vel4, ids);
}

int bonsai_write_tipsy(const char* path, double time, int n, int ndark, const float* pos4, const float* vel4,
                       const int* ids) {
  return bonsai_write_tipsy_impl(path, time, n, ndark, pos4, vel4, ids);
}

int bonsai_galaxy(long n, unsigned long long seed, double* pos4, float* vel4) {
  return bonsai_galaxy_impl(n, seed, pos4, vel4);
}

int bonsai_clustered_field(long n, unsigned long long seed, int nclusters, float* pos4, float* vel4) {
  return bonsai_clustered_field_impl(n, seed, nclusters, pos4, vel4);
}

int bonsai_selftest_wait_bound(int device) {
  BONSAI_CUDA_TRY(cudaSetDevice(device));
  cudaStream_t st;
  BONSAI_CUDA_TRY(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
  const int r = sort_timeout_selftest(st);
  cudaStreamDestroy(st);
  return r;
}

int bonsai_fp32_peak(int device, double* tflops) {
  if (!tflops) return BONSAI_ERR_ARG;
  BONSAI_CUDA_TRY(cudaSetDevice(device));
  int nsm = 0;
  BONSAI_CUDA_TRY(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device));
  cudaStream_t st;
  BONSAI_CUDA_TRY(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
  float* scratch = nullptr;
  BONSAI_CUDA_TRY(dalloc(&scratch, (size_t)nsm * 8));
  *tflops = fma_probe_tflops(nsm, st, scratch);
  cudaStreamSynchronize(st);
  dfree(&scratch);
  cudaStreamDestroy(st);
  return last_cuda();
}

int bonsai_binary_version(int device, int* binary_version, int* ptx_version) {
  if (!binary_version || !ptx_version) return BONSAI_ERR_ARG;
  BONSAI_CUDA_TRY(cudaSetDevice(device));
  return kernel_binary_version(binary_version, ptx_version);
}

void* bonsai_host_alloc(size_t bytes) {
  void* p = nullptr;
  if (cudaMallocHost(&p, bytes) != cudaSuccess) return nullptr;
  return p;
}

void bonsai_host_free(void* p) {
  if (p) cudaFreeHost(p);
}

}  // extern "C"
