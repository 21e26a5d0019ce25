/*
 * bonsai_b200.h -- C ABI of the B200 tree code (libbonsai_b200.so).
 *
 * Drop-in for the per-step path of Bonsai2's Treecode<float>
 * (code/Treecode.h:123-223, instantiated for float only in
 * code/TreecodeInstances.h:3).  Every entry point names the reference member
 * it replaces.  Plain pointers and sizes only; all state lives in an opaque
 * handle (one CUDA stream per handle, no globals), so handles are
 * independent and a process may hold several.
 *
 * Return codes: 0 = OK; > 0 = bit set of device-detected data conditions
 * (BONSAI_STATUS_*), reported after the stage that raised them; < 0 = API
 * misuse (BONSAI_ERR_*) or a CUDA error (-1000 - cudaError_t).  Nothing
 * aborts, asserts or traps (the reference aborts through CUDA_SAFE_CALL and
 * device assert, Treecode.h:18-27, computeForces.cu:565).
 *
 * Particle order: positions/velocities are passed in and returned in the
 * caller's order (index i of the arrays given to bonsai_set_particles).
 * Internally particles are kept in Peano-Hilbert order and reordered every
 * step; bonsai_get_particles scatters them back.
 */
#ifndef BONSAI_B200_H
#define BONSAI_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* device status bits (returned as positive codes) */
#define BONSAI_STATUS_CELL_CAPACITY 1  /* tree has more cells than allocated (retry with bonsai_alloc) */
#define BONSAI_STATUS_DEPTH 2          /* a level-21 cell holds more than nLeaf: kept as one leaf */
#define BONSAI_STATUS_WALK_STACK 4     /* a walk level list outgrew its ring: forces of that group are NaN */
#define BONSAI_STATUS_NONFINITE 8      /* NaN/Inf coordinate in the input */
#define BONSAI_STATUS_GROUP_CAPACITY 16
#define BONSAI_STATUS_BAD_PARAM 32
#define BONSAI_STATUS_SORT_TIMEOUT 64  /* a radix-sort look-back wait hit its bound: results invalid */
#define BONSAI_STATUS_BOUNDS 128       /* bounds-checked build only: a guarded index was out of range (access skipped) */

/* API errors */
#define BONSAI_ERR_HANDLE (-1)
#define BONSAI_ERR_NOT_ALLOCATED (-2)
#define BONSAI_ERR_ORDER (-3)     /* a stage was called before the stage it needs */
#define BONSAI_ERR_ARG (-4)
#define BONSAI_ERR_NO_DEVICE (-5)
#define BONSAI_ERR_TOO_LARGE (-6) /* request beyond a fixed capacity (bonsai_direct_fp64_noalloc) */
#define BONSAI_ERR_IO (-7)        /* snapshot file could not be opened, read or written */

typedef struct bonsai_handle_s *bonsai_handle;

typedef struct bonsai_params {
  float theta;      /* opening angle: Treecode::theta (Treecode.h:133,167) */
  float eps;        /* softening > 0: Treecode::eps2 = eps*eps (Treecode.h:133,166); the i == j term is summed */
  int nleaf;        /* max particles per leaf, 1..64: buildTree(nLeaf) (Treecode.h:216) */
  int ncrit;        /* max particles per group, 1..128: makeGroups(levelSplit, nCrit) (Treecode.h:218) */
  int level_split;  /* PH octal digits per group segment, 1..7 (Treecode.h:218; treecode.cu:142 passes 5) */
  float dt;         /* leapfrog step; the reference's moveParticles is a stub (moveParticles.cu:3-7) */
  int device;       /* CUDA device ordinal */
} bonsai_params;

typedef struct bonsai_tree_info {
  int ncells, nleaves, nnodes, nlevels, ngroups, status;
  int level_beg[32]; /* cells of level L are [level_beg[L], level_end[L]);   */
  int level_end[32]; /* the reference stores inclusive int2 ranges (buildTree.cu:748-780) */
} bonsai_tree_info;

/* Defaults of the Treecode constructor (Treecode.h:164: eps 0.01, theta 0.75,
 * nCrit 64), buildTree's nLeaf 16 (Treecode.h:216), the driver's
 * levelSplit 5 (treecode.cu:142), dt 1/64, device 0. */
void bonsai_default_params(bonsai_params *p);

/* Treecode(eps, theta, ncrit) -- Treecode.h:164-173 */
int bonsai_create(const bonsai_params *p, bonsai_handle *out);
/* ~Treecode (cuda_mem destructors, cudamem.h:13) */
int bonsai_destroy(bonsai_handle h);
/* Treecode::alloc(nPtcl) -- Treecode.h:175-198 */
int bonsai_alloc(bonsai_handle h, int n);
/* update theta / eps / dt between steps (the reference's public theta, eps2 fields, Treecode.h:133) */
int bonsai_set_params(bonsai_handle h, const bonsai_params *p);

/* Treecode::ptcl_h2d -- Treecode.h:207-214.  pos4 = (x,y,z,m), vel4 = (vx,vy,vz,*),
 * n floats4 each, host memory (pinned memory from bonsai_host_alloc is fastest).
 * Velocities are taken as synchronised with positions (first step: no closing kick). */
int bonsai_set_particles(bonsai_handle h, const float *pos4, const float *vel4, int n);
/* same, from device memory */
int bonsai_set_particles_device(bonsai_handle h, const float *d_pos4, const float *d_vel4, int n);
/* Treecode::ptcl_d2h -- Treecode.h:200-204, plus the accelerations (d_ptclAcc,
 * computeForces.cu:611-617); caller order; any pointer may be NULL. */
int bonsai_get_particles(bonsai_handle h, float *pos4, float *vel4, float *acc4);
int bonsai_get_particles_device(bonsai_handle h, float *d_pos4, float *d_vel4, float *d_acc4);
/* Asynchronous forms (no counterpart in the reference, whose copies are
 * synchronous): they return at once, so one step's uploads and downloads can
 * overlap other steps' compute.  bonsai_set_particles_async uploads on a copy
 * stream into device staging and the handle's stream takes the particles over
 * when they have landed (n must equal the allocated n; the host arrays must
 * stay unchanged until the next bonsai_synchronize).  bonsai_get_particles_async
 * captures the current state on the handle's stream into one of two staging
 * slots and downloads it on a second copy stream; the host arrays hold the
 * result after bonsai_synchronize (at most two downloads in flight; a third
 * waits for the first).  Pinned host memory (bonsai_host_alloc) is needed for
 * real overlap. */
int bonsai_set_particles_async(bonsai_handle h, const float *pos4, const float *vel4, int n);
int bonsai_get_particles_async(bonsai_handle h, float *pos4, float *vel4, float *acc4);

/* Treecode::buildTree(nLeaf) -- Treecode.h:216, buildTree.cu:845-1108 (box, tree, level order, leaves) */
int bonsai_build_tree(bonsai_handle h, int nleaf);
/* Treecode::computeMultipoles() -- Treecode.h:217, computeMultipoles.cu:194-234 */
int bonsai_compute_multipoles(bonsai_handle h);
/* Treecode::makeGroups(levelSplit, nCrit) -- Treecode.h:218, makeGroups.cu:236-341 */
int bonsai_make_groups(bonsai_handle h, int level_split, int ncrit);
/* Treecode::computeForces(INTCOUNT) -- Treecode.h:219, computeForces.cu:622-727.
 * If intcount and stats != NULL: stats = {<direct>, max direct, <approx>, max approx}
 * per particle (the reference's double4), and the call waits for the walk. */
int bonsai_compute_forces(bonsai_handle h, int intcount, double *stats);
/* Treecode::moveParticles() -- Treecode.h:220 (reference stub, moveParticles.cu:3-7):
 * kick-drift-kick leapfrog with merged kicks; energies of the synchronised
 * point are summed in the same pass. */
int bonsai_move_particles(bonsai_handle h);
/* Treecode::computeEnergies() -- Treecode.h:221 (reference stub, computeEnergies.cu:3-7;
 * potential sum of computeForces.cu:576-607).  out (may be NULL) =
 * {T, W, W without the i==j self term, T + W_noself, Px, Py, Pz, M}, FP64,
 * at the time of the last force evaluation.  Waits for the device. */
int bonsai_compute_energies(bonsai_handle h, double *out);

/* The whole step of treecode.cu:137-168 (build, multipoles, groups, forces,
 * move) nsteps times; use_graph != 0 replays it as a captured CUDA graph.
 * Asynchronous: call bonsai_synchronize for the status. */
int bonsai_step(bonsai_handle h, int nsteps, int use_graph);
/* bonsai_step with use_graph = 1 and CUDA events recorded on the handle's
 * stream between the phases of every step; waits, then writes
 * phase_ms[4*s + k] = {build+multipoles+groups, walk, move, whole step} (ms),
 * and phase_ms[4*nsteps] = device time from the first step's start to the
 * last step's end (phase_ms holds 4*nsteps+1 floats). */
int bonsai_step_timed(bonsai_handle h, int nsteps, float *phase_ms);
/* number of kernel nodes in the captured graphs of one step */
int bonsai_graph_kernel_count(bonsai_handle h);
/* interaction statistics of the last walk (computeForces.cu:568-609):
 * {sum over particles of n_approx, of n_direct, max n_approx, max n_direct} */
int bonsai_get_stats(bonsai_handle h, unsigned long long *out4);
/* Failure-detection self-test (no counterpart in the reference, whose waits
 * are unbounded): runs one radix-sort pass whose first tile never starts, so
 * the next tile's look-back waits on a flag nothing sets; the wait must end at
 * its bound and report.  Returns the status bits (BONSAI_STATUS_SORT_TIMEOUT
 * expected) after a fraction of a second; the device stays usable. */
int bonsai_selftest_wait_bound(int device);
/* Bounds-checked builds (the library compiled with -DBONSAI_CHECKS, e.g.
 * `python -m bonsai2_b200.build --checks`): every guarded index of the kernels
 * (cell, leaf, group, particle and scatter indexes) is tested, and an
 * out-of-range one skips its access and is counted; bonsai_synchronize then
 * reports BONSAI_STATUS_BOUNDS.  No reference counterpart (its kernels
 * assert).  Waits for the device, writes the number of violations since the
 * last reset and the first failing site ((kernel file << 8) | site), and
 * clears them when reset != 0.  Returns 1 in a checked build, 0 in the normal
 * build (count 0, no device access), < 0 on a CUDA error. */
int bonsai_bounds_check(unsigned *count, unsigned *first_site, int reset);
/* Runs one guarded access at the logical end of a buffer with a spare element
 * (inside the allocation in every build) and returns the violations it
 * recorded: 1 in a checked build, 0 in the normal build. */
int bonsai_bounds_selftest(int device);
/* measured FP32 FMA throughput of the device (TFLOP/s; the faster of scalar
 * FFMA and packed FFMA2 chains): the walk's roofline */
int bonsai_fp32_peak(int device, double *tflops);
/* the architecture of the device code loaded on `device`, read at run time
 * from one of the library's kernels (cudaFuncGetAttributes): binary_version
 * 100 = sm_100 SASS; ptx_version 0 when no PTX was embedded */
int bonsai_binary_version(int device, int *binary_version, int *ptx_version);
/* Wait for the handle's stream and its copy streams; returns the sticky device
 * status (and clears it). */
int bonsai_synchronize(bonsai_handle h);
/* The last error the handle has seen, without clearing anything: a pending
 * CUDA error (< 0) if there is one, else the sticky device status bits
 * (BONSAI_STATUS_*, 0 = none) after waiting for the handle's stream.  API
 * argument and order errors are returned by the call that made them. */
int bonsai_last_error(bonsai_handle h);
/* bonsai_step(h, nsteps, 1): nsteps steps replayed as captured CUDA graphs. */
int bonsai_step_graph(bonsai_handle h, int nsteps);
/* the copy streams (cudaStream_t) of the asynchronous set / get, for callers
 * that order their own work or events after them */
int bonsai_copy_streams(bonsai_handle h, void **h2d, void **d2h);
/* the handle's CUDA stream (cudaStream_t) */
void *bonsai_stream(bonsai_handle h);
const char *bonsai_error_string(int code);

/* ---- inspection (parity tests; the reference keeps these in device globals
 * and cuda_mem members: d_domain, d_cellDataList, d_level_begIdx, d_leafList,
 * d_key/d_value, d_groupList, d_cellSize, d_cellMonopole, d_cellQuad0/1) ---- */
int bonsai_get_tree_info(bonsai_handle h, bonsai_tree_info *out);
/* domain box {cx, cy, cz, hsize} (d_domain, buildTree.cu:161) */
int bonsai_get_box(bonsai_handle h, float *box4);
/* keys of the last build, sorted, and the sort permutations (indices into the
 * particle order the build saw); ids_at_build maps that order to caller order.
 * Any pointer may be NULL.  n entries each. */
int bonsai_get_keys(bonsai_handle h, uint64_t *tree_keys, int *tree_perm, uint64_t *ph_keys, int *ph_perm,
                    int *ids_at_build);
/* cells in the reference layout: cell_data uint32[4C] (CellData packing,
 * Treecode.h:45-89), size4/mono4/quad0 float[4C], quad1 float[2C],
 * leaf_list int[nleaves], parent int[C] (-1 for level 1).  Any may be NULL. */
int bonsai_get_cells(bonsai_handle h, uint32_t *cell_data, float *size4, float *mono4, float *quad0, float *quad1,
                     int *leaf_list, int *parent);
/* groups int[2G] = (pbeg, np) in PH order (GroupData, Treecode.h:29-43) */
int bonsai_get_groups(bonsai_handle h, int *groups);
/* walk inputs/outputs in internal order: ipos4 (PH/group order), jpos4 (tree
 * order), acc4 (PH order), ids (caller index of each PH-order particle) */
int bonsai_get_walk_arrays(bonsai_handle h, float *ipos4, float *jpos4, float *acc4, int *ids);

/* FP64 direct summation for ns sample particles (caller indices) against all
 * particles -- the force checker.  out double[4*ns] = (ax, ay, az, phi). */
int bonsai_direct_fp64(bonsai_handle h, const int *sample, int ns, int include_self, double *out);

/* The FP64 direct-sum checker for callers that cannot allocate device memory
 * (their GPU memory belongs to another framework's allocator, or their loop
 * must not pay cudaMalloc's device-wide synchronisation).  No counterpart in
 * the reference.  All pointers are device memory: d_pos4 = n float4 (x,y,z,m),
 * d_sample = ns particle indices, each in [0, n) (an index outside that range
 * reads nothing and gets a NaN output row), d_out = double[4*ns] (ax, ay, az,
 * phi); eps2 = softening squared, > 0 when include_self is set (the i == j
 * term; eps2 <= 0 then returns BONSAI_ERR_ARG); stream = a cudaStream_t
 * (NULL: the legacy default stream).  Allocates nothing: its scratch is a
 * fixed 2 MiB device array in the library, so ns <= 65536 (larger:
 * BONSAI_ERR_TOO_LARGE).  Calls share that array: calls that overlap on the
 * GPU race and must be serialised.  Every call looks the array up on the
 * current device (cudaGetSymbolAddress); the first call on a device may load
 * the library's device code, so make it before any stream capture on that
 * device.  Asynchronous on `stream`. */
int bonsai_direct_fp64_noalloc(const float *d_pos4, int n, const int *d_sample, int ns, double eps2,
                               int include_self, double *d_out, void *stream);

/* ---- per-group opening criteria (learned form; no counterpart in the
 * reference, whose angle is one number baked into every cell's opening size,
 * computeMultipoles.cu:168-177) ----
 * The walk opens a cell when the group's box is inside its geometric opening
 * sphere at the group's angle theta_g (split_node_grav_impbh,
 * computeForces.cu:30-54), and -- in the relative modes -- also when the cell's
 * octupole truncation error, M l^3 / ds^5 (M = cell mass, l = cell size,
 * ds = box-to-centre-of-mass distance), exceeds the group's bound tau_g.
 * Relative modes take tau_g from A_g, the group's mean |a| of the previous
 * force evaluation (read through this step's PH permutation); while there is
 * none (the first evaluation after particles are loaded) every group walks at
 * the fixed angle, exactly as mode 0.  theta_g is then the safety bound of
 * bonsai_set_relative_bound. */
#define BONSAI_MLP_FEATURES 16
#define BONSAI_MLP_WEIGHTS 5313 /* W1[64][16], b1[64], W2[64][64], b2[64], w3[64], b3 */
/* mode 0: fixed theta (params);
 * 1 (learned): tau_g = A_g 10^y_g, y_g = lo + (hi-lo)*sigmoid(MLP(features_g))
 *   from the weights of bonsai_set_mlp_weights; the features include
 *   statistics of the previous walk, and when that walk left none of a
 *   relative walk (the fixed-angle evaluation after a load, or a walk in
 *   another mode) the evaluation takes tau_g = 1e-2 A_g instead of the
 *   network, the relative walk the training tables are recorded after;
 * 2: theta_g from bonsai_set_group_theta, tau_g from bonsai_set_group_tau;
 * 3 (relative, one parameter): tau_g = lo * A_g (lo = alpha > 0; hi >= lo).
 * Features are clamped to [-10, 10] (degenerate groups, e.g. of a one-particle
 * system, would otherwise give inf or NaN). */
int bonsai_set_theta_mode(bonsai_handle h, int mode, float lo, float hi);
/* geometric bound theta_g of the relative modes 1 and 3 (default 2.0) */
int bonsai_set_relative_bound(bonsai_handle h, float theta_bound);
int bonsai_set_mlp_weights(bonsai_handle h, const float *w, int nw);
/* host array of ngroups angles for the current groups (after bonsai_make_groups) */
int bonsai_set_group_theta(bonsai_handle h, const float *theta, int ngroups);
/* theta mode 2: host array of ngroups bounds tau_g for the current groups
 * (tau = NULL: the geometric test only) */
int bonsai_set_group_tau(bonsai_handle h, const float *tau, int ngroups);
/* features of the current groups, host float[ngroups * 16] */
int bonsai_get_group_features(bonsai_handle h, float *out, int *ngroups);
/* A_g of the current groups as the last feature computation (a relative-mode
 * walk or bonsai_get_group_features) found it, host float[ngroups]; 0 when
 * there were no previous accelerations */
int bonsai_get_group_scale(bonsai_handle h, float *out);
/* angles used by the last walk in mode 1, 2 or 3, host float[ngroups] */
int bonsai_get_group_theta(bonsai_handle h, float *out);
/* per-group interaction counts of the last walk with per-group criteria (theta
 * mode 1, 2 or 3): out[2g] = approximate (cell) and out[2g+1] = direct (particle)
 * interactions of group g (the per-group form of computeForces.cu:568-609) */
int bonsai_get_group_interactions(bonsai_handle h, unsigned *out);
/* MLP on the GPU, host arrays: loss (mean of 0.5 (theta - y)^2 (1 + over [theta > y]))
 * and its gradient; Adam training for `epochs` full-batch steps (w in/out);
 * prediction of theta for S feature rows. */
int bonsai_mlp_loss_grad(int device, const float *X, const float *y, int S, const float *w, float lo, float hi,
                         float over, float *grad, double *loss);
int bonsai_mlp_train(int device, const float *X, const float *y, int S, float *w, int epochs, float lr, float lo,
                     float hi, float over, double *loss);
int bonsai_mlp_predict(int device, const float *X, int S, const float *w, float lo, float hi, float *theta);

/* FP64 checker walk (the FP64 option; no counterpart in the reference, whose
 * tree-build experiments have a -DFP64 switch, treebuild/readme:8-9): after
 * the stages up to makeGroups (and compute_forces for theta mode 1), walks the
 * same tree for the same groups with the float walk's opening decisions, so the
 * interaction lists are identical, and evaluates every interaction in FP64
 * from the FP64 cell records and the exact positions.  acc4 (optional):
 * n x (ax, ay, az, phi) doubles in caller order; stats4 (optional): as
 * bonsai_get_stats.  Against the float walk the difference is rounding alone;
 * against bonsai_direct_fp64 it is multipole truncation alone.  Slow (a
 * checker).  nCrit <= 128; in an ensemble each group walks its own system. */
int bonsai_compute_forces_fp64(bonsai_handle h, double *acc4, unsigned long long *stats4);

/* ---- Double-single positions (precision form) ----
 * No counterpart in the reference (float positions throughout).  mode 1
 * keeps every position as a float pair hi + lo: the tree, keys and groups are
 * built from hi; multipoles sum hi + lo in FP64 and store the centre of mass
 * as a pair; the walk takes every coordinate relative to the group's first
 * particle, (hi - R) + lo, so separations keep FP32 relative precision far
 * from the origin; the drift adds in double-single; the FP64 checker
 * (bonsai_direct_fp64) uses hi + lo.  Interactions stay FP32.  Set it before
 * loading particles (the low parts start at zero) and, for an ensemble, after
 * bonsai_set_systems (each system then advances bit for bit as it does
 * alone).  mode 0 (default) = float positions. */
int bonsai_set_precision(bonsai_handle h, int mode);
/* bonsai_set_particles from double positions pos4 = (x, y, z, m): split into
 * hi = (float)x and lo = (float)(x - hi) (lo dropped in mode 0) */
int bonsai_set_particles_f64(bonsai_handle h, const double *pos4, const float *vel4, int n);
/* bonsai_get_particles with positions returned as hi + lo in double */
int bonsai_get_particles_f64(bonsai_handle h, double *pos4, float *vel4, float *acc4);

/* ---- Ensembles of independent systems (batching) ----
 * No counterpart in the reference, which holds one tree per process (its stage
 * state lives in file-scope device globals, buildTree.cu:23-36).
 * bonsai_set_systems lays the handle's particles out as nsys independent
 * systems: system s owns the counts[s] >= 1 particles that follow system
 * s-1's in the arrays given to bonsai_set_particles.  It allocates like
 * bonsai_alloc(h, sum of counts); bonsai_alloc and a bonsai_set_particles
 * with another n return to one system.  Every stage then treats each system
 * as if it were alone (own box, keys, tree and groups; no force between
 * systems) in the same kernel launches for all systems, so the positions,
 * velocities and accelerations of each system are bit-identical to those of a
 * handle that holds that system alone with the same parameters.
 * bonsai_compute_energies then sums over all systems; bonsai_get_box returns
 * system 0's box; bonsai_direct_fp64 sums inside each sample's system.
 * Per-group opening angles (bonsai_set_theta_mode, set after this call) work
 * inside an ensemble: the network's features are normalised per system, so a
 * system's angles, and with them its forces, are those it gets alone.
 * Double-single positions (bonsai_set_precision, set after this call) work
 * inside an ensemble too, and so do block time steps (bonsai_set_block_steps,
 * set after this call).  nsys <= 65536. */
int bonsai_set_systems(bonsai_handle h, const int *counts, int nsys);
/* energies of every system, 8 doubles per system in the layout and with the
 * timing rules of bonsai_compute_energies (a single system: its 8 values) */
int bonsai_get_system_energies(bonsai_handle h, double *out);
/* walk thread layout, the analogue of the reference's warps-per-group
 * choice (NWARPS_OCTREE2 / NI, computeForces.cu:475-619): 0 (default) = two
 * half-warps per group, each holding all the group's particles and taking
 * alternate sources (nCrit <= 64; above that as 1); 1 = one warp per group,
 * one lane per particle slot. */
int bonsai_set_walk_layout(bonsai_handle h, int layout);
/* Autotuner (no counterpart in the reference): on the handle's current
 * particles, for every walk layout L in {0, 1}, nleaf[a] and ncrit[b],
 * builds, captures and times one warm-up plus `steps` graph steps, restoring
 * the particles before each trial and at the end.  results (optional,
 * 2 * n_nleaf * n_ncrit floats, index (L*n_nleaf + a)*n_ncrit + b) receives
 * ms per step, or -1 for a skipped or failed candidate (layout 0 with
 * nCrit > 64, a value out of range, a device status).  The fastest candidate
 * becomes the handle's nLeaf / nCrit / layout; best (optional, 3 ints)
 * receives them.  Allocates a copy of the particle state while it runs. */
int bonsai_autotune(bonsai_handle h, const int *nleaf, int n_nleaf, const int *ncrit, int n_ncrit, int steps,
                    float *results, int *best);

/* Plummer sphere initial conditions on the host: the algorithm of
 * code/plummer.h:9-138 (glibc rand(), same stream), converted to float4 like
 * treecode.cu:65-87: pos4 = (x,y,z,m), vel4 = (vx,vy,vz,m).  n >= 1. */
int bonsai_plummer(long n, unsigned int seed, float *pos4, float *vel4);

/* Tipsy snapshots (host; ReadTipsy, read_tipsy.h:108-160, records of
 * tipsydefs.h): native-order header {double time; int nbodies, ndim, nsph,
 * ndark, nstar} (32 bytes), ndark dark records {mass, pos[3], vel[3], eps,
 * int phi}, then nbodies - ndark star records {mass, pos[3], vel[3], metals,
 * tform, eps, int phi}, as the reference reads them (nsph ignored).  pos4 =
 * (x, y, z, mass), vel4 = (vx, vy, vz, eps), ids = phi.
 * bonsai_read_tipsy with pos4, vel4 and ids all NULL returns the particle count
 * in *n (and the time); otherwise *n is the capacity of the arrays on entry and
 * the count on return.  bonsai_write_tipsy writes the same layout (ids NULL:
 * 0..n-1; nsph 0, nstar = n - ndark), which the reference's reader reads back. */
int bonsai_read_tipsy(const char *path, double *time, int *n, float *pos4, float *vel4, int *ids);
int bonsai_write_tipsy(const char *path, double time, int n, int ndark, const float *pos4, const float *vel4,
                       const int *ids);
/* Checkpoints: after a step the velocities are half a step ahead of the
 * positions (kick-drift-kick with merged kicks).  This evaluates the forces at
 * the current positions and applies the pending closing kick in place, so that
 * bonsai_get_particles returns synchronised (x, v) that a restart loads with
 * bonsai_set_particles and continues exactly (the next move skips the kick it
 * would have applied). */
int bonsai_sync_velocities(bonsai_handle h);

/* Block time steps (no counterpart in the reference; Bonsai proper's
 * per-particle steps).  max_level = K >= 0 enables them: levels 0..K, a
 * level-k particle steps by dt/2^k (dt from bonsai_params), kick-drift-kick
 * per particle; its level is the smallest k with dt/2^k <= eta sqrt(eps/|a|),
 * taken at the end of each of its steps, never before its boundary (a step
 * starts where a step of its length may) and at most doubling the step at a
 * time.  max_level < 0 turns them off.  In an ensemble (set after
 * bonsai_set_systems) every particle keeps its own level and each system
 * advances as it does alone; a substep rebuilds the tree when a particle of
 * any system ends a step there. */
int bonsai_set_block_steps(bonsai_handle h, int max_level, float eta);
/* nsteps big steps of dt, each 2^K substeps: per substep the opening kicks of
 * the particles whose step starts, the drift of all particles, a tree of all
 * particles, a walk of only the groups holding a particle whose step ends, and
 * those particles' closing kicks and new levels.  The first call evaluates all
 * forces and applies any pending closing kick.  All particles are
 * synchronised at the end of every big step (bonsai_compute_energies then
 * returns that time's energies).  With K = 0 this is the bonsai_step
 * sequence, bit for bit. */
int bonsai_block_step(bonsai_handle h, int nsteps);
/* current levels in the caller's particle order (n bytes) */
int bonsai_get_levels(bonsai_handle h, unsigned char *levels);

/* Composite galaxy on the host (no counterpart in the reference): 60 % NFW-like
 * halo (r_s 10, truncated at 200), 30 % exponential disk (R_d 3, sech^2
 * z_d 0.3), 10 % Hernquist bulge (a 0.5) by particle index; log-normal masses
 * (sigma 0.5) normalised to 1; pos4 = (x, y, z, m) in double, vel4 = (vx, vy,
 * vz, m).  Seeded per particle: the result is independent of thread count. */
int bonsai_galaxy(long n, unsigned long long seed, double *pos4, float *vel4);
/* Clustered field on the host (no counterpart in the reference): 80 % of the
 * particles in nclusters Plummer subclusters (masses log-uniform over two
 * decades, scale radii log-uniform in [0.01, 0.2], centres uniform in the
 * unit cube), 20 % uniform in the unit cube; equal masses 1/n. */
int bonsai_clustered_field(long n, unsigned long long seed, int nclusters, float *pos4, float *vel4);

/* pinned host memory (host_mem<T>, cudamem.h:64-96) */
void *bonsai_host_alloc(size_t bytes);
void bonsai_host_free(void *p);

#ifdef __cplusplus
}
#endif

#endif /* BONSAI_B200_H */
