// kernels.cuh -- internal declarations shared by the kernel translation units
// and the host orchestration (treecode.cu).  Not part of the C ABI.
#pragma once
#include "common.cuh"

namespace bonsai {

constexpr int kWalkThreads = 256;
constexpr int kMlpFeatures = 16;
constexpr int kMlpHidden = 64;
constexpr int kMlpWeights = kMlpHidden * kMlpFeatures + kMlpHidden + kMlpHidden * kMlpHidden + kMlpHidden + kMlpHidden + 1;
#ifndef BONSAI_WALK_MINB
#define BONSAI_WALK_MINB 2
#endif
constexpr int kWalkMinBlocks = BONSAI_WALK_MINB;

// keys.cu
// PH state tables: one level per lookup (48 states x 8 octants), then two
// levels per lookup (48 x 64)
constexpr int kPhTable1 = 48 * 8;
constexpr int kPhTableSize = kPhTable1 + 48 * 64;
void build_ph_table(uint16_t* tab);
__global__ void k_box(const float4* __restrict__ pos, int n, float* __restrict__ partial, unsigned* __restrict__ ticket,
                      Box* __restrict__ box, int* __restrict__ status);
__global__ void k_keys(const float4* __restrict__ pos, int n, const Box* __restrict__ boxp,
                       const uint16_t* __restrict__ ph_table, unsigned long long* __restrict__ tkey,
                       unsigned long long* __restrict__ pkey);
// ensemble: per-system boxes (chunk extents folded per system) and keys
void launch_sys_keys(const float4* pos, const int4* chunks, int nchunks, const int* chunk_beg, int nsys,
                     float* box_partial, Box* boxes, const uint16_t* ph_table, unsigned long long* tkey,
                     unsigned long long* pkey, int* status, int nblocks, cudaStream_t s);

// sort.cu
int sort_tiles(int n);
int scan_blocks(int m);
void exclusive_scan(const unsigned* in, unsigned* out, int m, unsigned* bsum, unsigned* total, cudaStream_t s);
size_t sort_status_words(int n);
void radix_sort_pairs(unsigned long long* keys_a, unsigned long long* keys_b, int* vals_a, int* vals_b,
                      const int* vals_in, int n, unsigned* work, int* err, int passes, const int* sys_off, int nsys,
                      cudaStream_t s);

// bounded look-back self-test: returns the status bits of a pass whose first tile never runs
int sort_timeout_selftest(cudaStream_t s);

// tree.cu
int tree_tiles(int n);
void build_tree(const unsigned long long* sorted_keys, int n, int nleaf, int cell_cap, int leaf_cap, uint8_t* dlev,
                uint16_t* chain, unsigned* hist, TreeInfo* info, uint4* cell_data, int* cell_parent, int* leaf_list,
                int* mp_count, const int* sys_off, int nsys, int* root_beg, cudaStream_t s);

// multipoles.cu
// box: 6 floats per cell (float positions) or 6 doubles (jlo != nullptr:
// double-single positions)
void launch_multipoles(const int* leaf_list, const TreeInfo* info, const uint4* cell_data, const int* cell_parent,
                       const float4* jpos, float inv_theta, MpRec* rec, void* box, float4* cell_open,
                       float4* cell_stage, float4* cell_ls, int* mp_count, int cell_cap,
                       const float4* jlo, float4* cell_lo, int nblocks, cudaStream_t s);
__global__ void k_multipoles_ref_layout(const TreeInfo* __restrict__ info, const float4* __restrict__ cell_open,
                                        const MpRec* __restrict__ rec, float4* __restrict__ size,
                                        float4* __restrict__ mono, float4* __restrict__ quad0,
                                        float2* __restrict__ quad1);

// groups.cu
void make_groups(const unsigned long long* sorted_ph, int n, int level_split, int ncrit, unsigned* count,
                 unsigned* seg_start, unsigned* ng, unsigned* bsum, int2* groups, int group_cap, TreeInfo* info,
                 cudaStream_t s);
void make_groups_sys(const unsigned long long* sorted_ph, int n, int level_split, int ncrit, const int* sys_off,
                     int nsys, unsigned* flag, unsigned* sid, unsigned* seg_beg, unsigned* seg_end, unsigned* nseg,
                     unsigned* bsum, int2* groups, int group_cap, TreeInfo* info, cudaStream_t s);
__global__ void k_gather_state(const int* __restrict__ perm, int n, const float4* __restrict__ pos,
                               const float4* __restrict__ vel, const int* __restrict__ id, float4* __restrict__ pos_o,
                               float4* __restrict__ vel_o, int* __restrict__ id_o);
__global__ void k_gather_pos(const int* __restrict__ perm, int n, const float4* __restrict__ pos,
                             float4* __restrict__ out);

// Relative accuracy mode (per-group bound tau on a cell's octupole truncation
// error, M l^3 / ds^5 <= tau) and the statistics the learned features read
// at the next evaluation.
struct RelativeArgs {
  const float* tau = nullptr;  // per-group bounds; null: the geometric test only
  float4* stats = nullptr;     // per-group statistics written by the walk (null: none)
  int* part_gid = nullptr;     // group of each particle, written with the statistics
  int* acc_valid = nullptr;    // [0] set to 1 by the walk once acc holds this evaluation's
                               // accelerations, [1] to where its statistics came from: 0 none,
                               // 1 a walk without the relative test (the fallback), 2 a relative walk
};

// What the learned features read of the previous evaluation.
struct PrevEval {
  const float4* acc = nullptr;    // its accelerations, in its particle order
  const int* perm = nullptr;      // current position -> index in that order (null: the same order)
  const int* acc_valid = nullptr; // device flags: [0] acc is valid, [1] stats and part_gid came with it
                                  // (1: from the fixed-angle fallback, 2: from a relative walk)
  const int* part_gid = nullptr;  // group of each particle in that evaluation (its order)
  const float4* stats = nullptr;  // its per-group statistics
  int stats_cap = 0;              // capacity of stats
};

// walk.cu
int walk_variant(int ncrit, int layout);
int walk_blocks_per_sm(int variant);
// group_inv_theta == nullptr: the fixed opening angle baked into cell_open.w;
// else 1/theta per group with (l, s) from cell_ls
void launch_walk(int variant, int nblocks, const int2* groups, const TreeInfo* info, const float4* ipos, const float4* jpos,
                 const uint4* cell_data, const float4* cell_open, const float4* cell_stage,
                 const float4* cell_ls, const float* group_inv_theta, float eps2, float4* acc, int* ring_pool,
                 int ring_cap, unsigned* group_counter, unsigned long long* stats, int* status, const int* sys_off,
                 int nsys, const int* root_beg, const float4* ipos_lo, const float4* jpos_lo, const float4* cell_lo,
                 uint2* group_counts, const int* group_list, const unsigned* group_list_n, const RelativeArgs& rel,
                 cudaStream_t s);

// walk64.cu: the FP64 checker walk (same interaction lists as the float walk)
void launch_walk64(int nblocks, const int2* groups, const TreeInfo* info, const float4* ipos, const float4* ipos_lo,
                   const float4* jpos, const float4* jpos_lo, const uint4* cell_data, const float4* cell_open,
                   const float4* cell_lo, const float4* cell_ls, const float* group_inv_theta,
                   const float* group_tau, const MpRec* rec, double eps2, double4* acc, int* ring_pool, int ring_cap,
                   unsigned* group_counter,
                   unsigned long long* stats, int* status, const int* sys_off, int nsys, const int* root_beg,
                   cudaStream_t s);
void launch_scatter_d4(const int* id, int n, const double4* in, double4* out, int nblocks, cudaStream_t s);

// move.cu
// lo (nullable): double-single position low parts, drifted with the high parts
void launch_move(float4* pos, float4* vel, const float4* acc, int n, float dt, int* closing, float eps, int write,
                 double* partial, int nblocks, unsigned* ticket, double* energies, cudaStream_t s,
                 float4* lo = nullptr);
// ensemble move: energies per chunk, folded per system and in total (lo as launch_move)
void launch_move_sys(float4* pos, float4* vel, const float4* acc, const int4* chunks, int nchunks,
                     const int* chunk_beg, int nsys, float dt, int* closing, float eps, int write, double* chunk_part,
                     int nblocks, unsigned* ticket, double* energies, double* sys_energies, cudaStream_t s,
                     float4* lo = nullptr);
// block time steps (hierarchical levels, kick-drift-kick per particle)
void launch_bts_open_drift(float4* pos, float4* vel, const float4* acc, const unsigned char* lev, int n, float dt,
                           int K, int s, float4* lo, int nblocks, cudaStream_t st);
void launch_bts_close(float4* vel, const float4* acc, unsigned char* lev, int n, float dt, int K, int s1, float eta,
                      float eps, int assign, int nblocks, cudaStream_t st);
void launch_bts_active_groups(const int2* groups, const TreeInfo* info, const unsigned char* lev, int K, int s1,
                              int* list, unsigned* count, int nblocks, cudaStream_t st);
// largest level present (into *out)
void launch_max_level(const unsigned char* lev, int n, int* out, int nblocks, cudaStream_t st);
void launch_gather_u8(const int* perm, int n, const unsigned char* in, unsigned char* out, int nblocks,
                      cudaStream_t st);
void launch_scatter_u8(const int* id, int n, const unsigned char* in, unsigned char* out, int nblocks,
                       cudaStream_t st);
// pending closing kick applied in place, then the closing flag cleared
void launch_closing_kick(float4* vel, const float4* acc, int n, float dt, int* closing, int nblocks, cudaStream_t s);
// FP64 direct sum inside each sample's own system (one block per sample; lo as launch_direct_fp64)
void launch_direct_fp64_sys(const float4* pos, const int* sys_off, int nsys, const int* sample, int ns, double eps2,
                            int include_self, double* out, cudaStream_t s, const float4* lo = nullptr);
// lo (nullable): double-single low parts, positions taken as hi + lo
void launch_direct_fp64(const float4* pos, int n, const int* sample, int ns, double eps2, int include_self,
                        double* part, int nsplit, double* out, cudaStream_t s, const float4* lo = nullptr);
__global__ void k_scatter_by_id(const int* __restrict__ id, int n, const float4* __restrict__ in,
                                float4* __restrict__ out);
__global__ void k_iota(int* __restrict__ a, int n);
double fma_probe_tflops(int nsm, cudaStream_t st, float* scratch);
int kernel_binary_version(int* binary_version, int* ptx_version);

// Bounds-checked builds (-DBONSAI_CHECKS): the violation word (count, first
// failing site) of each translation unit with guarded accesses; reset clears
// it.  Zeros in the normal build.
int bounds_word_sort(unsigned* w, bool reset);
int bounds_word_tree(unsigned* w, bool reset);
int bounds_word_multipoles(unsigned* w, bool reset);
int bounds_word_groups(unsigned* w, bool reset);
int bounds_word_walk(unsigned* w, bool reset);
int bounds_word_walk64(unsigned* w, bool reset);
int bounds_word_move(unsigned* w, bool reset);
int bounds_word_learned(unsigned* w, bool reset);
// checked-build self-test (move.cu): one guarded write at the logical end of
// a buffer that has a spare element, so the access is inside the allocation
// in every build; returns the violations it recorded (1 in a checked build)
int bounds_selftest(cudaStream_t s);

// learned.cu
size_t mlp_train_scratch_floats(int S);
void mlp_loss_grad(const float* X, const float* y, int S, const float* w, float lo, float hi, float over,
                   float* scratch, float* grad, double* loss_out, cudaStream_t st);
void mlp_adam_step(float* w, const float* grad, float* m, float* v, float lr, int step, cudaStream_t st);
void mlp_predict(const float* X, int S, const float* w, float lo, float hi, float* scratch, float* pred,
                 cudaStream_t st);
// box: the domain box, or an ensemble's per-system boxes (nsys > 1, with
// sys_off and the systems' level-1 cell ranges root_beg)
// amag: each group's mean |a| of the previous evaluation (0 without one)
void launch_group_features(const int2* groups, const TreeInfo* info, const float4* ipos,
                           const unsigned long long* ph_sorted, const MpRec* rec, const Box* box, int n, int ncrit,
                           float eps, float* feat, const int* sys_off, int nsys, const int* root_beg,
                           const PrevEval& prev, float* amag, int nblocks, cudaStream_t st);
// the network's output y in [lo, hi] per group: tau = amag 10^y, 1/theta =
// inv_bound; without previous accelerations the fixed angle (tau = 0,
// 1/theta = inv_fixed)
// start_alpha: the bound tau = start_alpha amag used instead of the network
// when the previous walk recorded no relative-walk statistics (acc_valid[1]
// != 2: the fixed-angle fallback, or a walk in another theta mode)
void launch_mlp_infer(const float* feat, const void* wh, const TreeInfo* info, float lo, float hi, const float* amag,
                      const int* acc_valid, float inv_bound, float inv_fixed, float start_alpha, float* inv, float* tau,
                      int nblocks, cudaStream_t st);
// relative mode with one accuracy parameter: tau = alpha amag (fallback as above)
void launch_relative_tau(const TreeInfo* info, const float* amag, const int* acc_valid, float alpha, float inv_bound,
                         float inv_fixed, float* inv, float* tau, int nblocks, cudaStream_t st);
void launch_weights_to_half(const float* w, void* wh, cudaStream_t st);
void launch_fill_inv_theta(const TreeInfo* info, const float* theta, float c, float* inv, int nblocks,
                           cudaStream_t st);

}  // namespace bonsai
