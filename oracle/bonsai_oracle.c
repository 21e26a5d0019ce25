/*
 * bonsai_oracle.c -- CPU restatement of the Bonsai2 per-step hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker for the CUDA path in
 * bonsai2_b200/csrc; it is loaded only by tests/, by __graft_entry__.smoke()
 * and by the cpu_baseline / reference leg of bench.py.  The product never
 * links, loads or calls it.
 *
 * Every function states the reference lines it restates (paths relative to
 * the Bonsai2 source tree).  Parity pinning:
 *   - oracle_plummer is pinned bit-exactly against the reference's own
 *     code/plummer.h, compiled unmodified from the reference tree by
 *     oracle/build_ref.sh (fixture tests/golden/plummer_*.bin).
 *   - oracle_ph_keys, oracle_argsort_u64 and oracle_make_groups are pinned
 *     bit-exactly against the reference's own GPU group formation
 *     (code/makeGroups.cu, compiled unmodified for sm_100a by
 *     oracle/build_ref.sh and run on a B200; fixture
 *     tests/golden/ref_groups.json: full PH keys, sorted order including a
 *     2000-way tie, groups, over four inputs).
 *   - tree keys, tree topology and walk decisions are restated from the cited
 *     CUDA sources (buildTree.cu and computeForces.cu do not build for
 *     sm_100, and the reference ships no golden vectors for them); the
 *     topology is also checked against the tree shape the reference
 *     publishes for its own N = 20,000,000 build.  Forces are additionally
 *     judged against the FP64 direct sum below.
 *
 * Build: gcc -O2 -fopenmp -fPIC -shared (no -ffast-math, no -march: the
 * Plummer generator must round exactly as the reference's g++ build does).
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <math.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define OR_MAXL 21 /* 3 bits per level, 63-bit keys (makeGroups.cu:253) */

/* ------------------------------------------------------------------------ */
/* Plummer sphere: restates code/plummer.h:9-138 (glibc rand(), Henon units,
 * R<100 cut, speed by rejection, centre-of-mass and mean-velocity removal).
 * The on-disk cache of plummer.h (plummer.dat) is not reproduced.          */
/* ------------------------------------------------------------------------ */
static double or_rand01(void) { return rand() / (1. + RAND_MAX); }

void oracle_plummer(long n, unsigned int seed, double *mass, double *pos, double *vel)
{
  srand(seed);
  long i = 0;
  while (i < n) {
    double X1 = or_rand01();
    double X2 = or_rand01();
    double X3 = or_rand01();
    double R = 1.0 / sqrt((pow(X1, -2.0 / 3.0) - 1.0));
    if (R < 100.0) {
      double Z = (1.0 - 2.0 * X2) * R;
      double X = sqrt(R * R - Z * Z) * cos(2.0 * M_PI * X3);
      double Y = sqrt(R * R - Z * Z) * sin(2.0 * M_PI * X3);
      double Ve = sqrt(2.0) * pow((1.0 + R * R), -0.25);
      double X4 = 0.0, X5 = 0.0;
      while (0.1 * X5 >= X4 * X4 * pow((1.0 - X4 * X4), 3.5)) {
        X4 = or_rand01();
        X5 = or_rand01();
      }
      double V = Ve * X4;
      double X6 = or_rand01();
      double X7 = or_rand01();
      double Vz = (1.0 - 2.0 * X6) * V;
      double Vx = sqrt(V * V - Vz * Vz) * cos(2.0 * M_PI * X7);
      double Vy = sqrt(V * V - Vz * Vz) * sin(2.0 * M_PI * X7);
      double conv = 3.0 * M_PI / 16.0;
      X *= conv; Y *= conv; Z *= conv;
      Vx /= sqrt(conv); Vy /= sqrt(conv); Vz /= sqrt(conv);
      mass[i] = 1.0 / n;
      pos[3 * i + 0] = X; pos[3 * i + 1] = Y; pos[3 * i + 2] = Z;
      vel[3 * i + 0] = Vx; vel[3 * i + 1] = Vy; vel[3 * i + 2] = Vz;
      i++;
    }
  }
  double mcm = 0.0, xcm[3] = {0, 0, 0}, vcm[3] = {0, 0, 0};
  for (i = 0; i < n; i++) {
    mcm += mass[i];
    for (int k = 0; k < 3; k++) {
      xcm[k] += mass[i] * pos[3 * i + k];
      vcm[k] += mass[i] * vel[3 * i + k];
    }
  }
  for (int k = 0; k < 3; k++) { xcm[k] /= mcm; vcm[k] /= mcm; }
  for (i = 0; i < n; i++)
    for (int k = 0; k < 3; k++) {
      pos[3 * i + k] -= xcm[k];
      vel[3 * i + k] -= vcm[k];
    }
}

/* ------------------------------------------------------------------------ */
/* Domain box: restates code/buildTree.cu:80-166 (float min/max; hsize is the
 * smallest power of two >= the largest half-extent; centre truncated to a
 * multiple of hsize/2^20).  The halving loop is floored at
 * max(2^-100, 2^-40 * max|centre|) (powers of two) so that a zero-extent input
 * (one particle, all particles coincident) gives a finite box whose centre
 * quantisation fits 64 bits; the reference halves to hsize == 0 there and
 * divides by zero.  The floor never binds for extents above 2^-40 of the
 * coordinates.
 * Returns 1 when any coordinate is NaN/Inf, else 0.                        */
/* ------------------------------------------------------------------------ */
int oracle_bbox(int n, const float *p4, float *box)
{
  float bmin[3] = {1e10f, 1e10f, 1e10f}, bmax[3] = {-1e10f, -1e10f, -1e10f};
  int bad = 0;
  for (int i = 0; i < n; i++)
    for (int k = 0; k < 3; k++) {
      float x = p4[4 * i + k];
      if (!isfinite(x)) bad = 1;
      bmin[k] = fminf(bmin[k], x);
      bmax[k] = fmaxf(bmax[k], x);
    }
  float c[3], h[3];
  for (int k = 0; k < 3; k++) {
    c[k] = (bmax[k] + bmin[k]) * 0.5f;
    h[k] = (bmax[k] - bmin[k]) * 0.5f;
  }
  const float hm = fmaxf(h[2], fmaxf(h[1], h[0]));
  /* floor for hsize: max(2^-100, 2^-40 * (power of two >= max |centre|)),
   * so that centre/hquant fits a 64-bit integer when the extent is ~0 */
  const float cm = fmaxf(fabsf(c[0]), fmaxf(fabsf(c[1]), fabsf(c[2])));
  float pw = 1.0f;
  while (pw < cm) pw *= 2.0f;
  while (pw * 0.5f >= cm && pw > 7.888609052210118e-31f) pw *= 0.5f;
  const float floor_h = fmaxf(pw * 9.094947017729282e-13f, 7.888609052210118e-31f); /* 2^-40, 2^-100 */
  float hsize = 1.0f;
  while (hsize > hm && hsize > floor_h) hsize *= 0.5f;
  while (hsize < hm) hsize *= 2.0f;
  const float hquant = hsize / (float)(1 << 20);
  for (int k = 0; k < 3; k++) {
    const long long q = (long long)(c[k] / hquant);
    box[k] = hquant * (float)q;
  }
  box[3] = hsize;
  return bad;
}

/* ------------------------------------------------------------------------ */
/* Exact octant-path key: the sequence of octants the reference's recursive
 * partition assigns to a particle.  Octant() is Particle4.h:129-136
 * ((centre <= x) bits x,y,z -> 0,1,2) and the child box is ChildBox()
 * Particle4.h:138-148 (centre +- hsize/2, float); the root uses the domain
 * box (buildTree.cu:237) and every level the child box of the previous one
 * (buildTree.cu:206-207,245).  Digit of level L sits in bits 62-3L+3..60-3L+3
 * (level 1 most significant).                                              */
/* ------------------------------------------------------------------------ */
static uint64_t or_tree_key1(float x, float y, float z, const float *box)
{
  float cx = box[0], cy = box[1], cz = box[2], h = box[3];
  uint64_t key = 0;
  for (int L = 1; L <= OR_MAXL; L++) {
    const int oct = (cx <= x) | ((cy <= y) << 1) | ((cz <= z) << 2);
    key = (key << 3) | (uint64_t)oct;
    const float s = 0.5f * h;
    cx = cx + s * ((oct & 1) ? 1.0f : -1.0f);
    cy = cy + s * ((oct & 2) ? 1.0f : -1.0f);
    cz = cz + s * ((oct & 4) ? 1.0f : -1.0f);
    h = s;
  }
  return key;
}

void oracle_tree_keys(int n, const float *p4, const float *box, uint64_t *keys)
{
#pragma omp parallel for schedule(static)
  for (int i = 0; i < n; i++)
    keys[i] = or_tree_key1(p4[4 * i], p4[4 * i + 1], p4[4 * i + 2], box);
}

/* ------------------------------------------------------------------------ */
/* Peano-Hilbert key: restates makeGroups.cu:108-135 (float quantisation of
 * (x - bmin) * (0.5/hsize) * 2^21, truncation to int) and the 21-step
 * state machine get_key<21> makeGroups.cu:19-106 (digit table at :28, axis
 * swaps / complements at :49-81).                                          */
/* ------------------------------------------------------------------------ */
static uint64_t or_ph_digits(int cx, int cy, int cz)
{
  static const int C[8] = {0, 1, 7, 6, 3, 2, 4, 5};
  uint64_t key = 0;
  int mask = 1 << (OR_MAXL - 1);
  for (int i = 0; i < OR_MAXL; i++, mask >>= 1) {
    const int xi = (cx & mask) ? 1 : 0;
    const int yi = (cy & mask) ? 1 : 0;
    const int zi = (cz & mask) ? 1 : 0;
    const int idx = (xi << 2) + (yi << 1) + zi;
    int d, t;
    if (idx == 0) {
      t = cz; cz = cy; cy = t; d = C[0];
    } else if (idx == 1 || idx == 5) {
      t = cx; cx = cy; cy = t; d = (idx == 1) ? C[1] : C[5];
    } else if (idx == 4 || idx == 6) {
      cx = ~cx; cz = ~cz; d = (idx == 4) ? C[4] : C[6];
    } else if (idx == 7 || idx == 3) {
      t = ~cx; cx = ~cy; cy = t; d = (idx == 3) ? C[3] : C[7];
    } else {
      t = ~cz; cz = ~cy; cy = t; d = C[2];
    }
    key = (key << 3) + (uint64_t)d;
  }
  return key;
}

static int or_quant(float x, float bmin, float inv)
{
  const float v = (x - bmin) * inv * (float)(1 << OR_MAXL);
  /* CUDA's float->int conversion truncates toward zero and saturates (NaN
   * gives 0); C leaves out-of-range undefined, so saturate explicitly. */
  if (!(v == v)) return 0;
  if (v >= 2147483647.0f) return 2147483647;
  if (v <= -2147483648.0f) return (int)0x80000000;
  return (int)v;
}

void oracle_ph_keys(int n, const float *p4, const float *box, uint64_t *keys)
{
  const float inv = 0.5f / box[3];
  const float bx = box[0] - box[3], by = box[1] - box[3], bz = box[2] - box[3];
#pragma omp parallel for schedule(static)
  for (int i = 0; i < n; i++)
    keys[i] = or_ph_digits(or_quant(p4[4 * i], bx, inv), or_quant(p4[4 * i + 1], by, inv),
                           or_quant(p4[4 * i + 2], bz, inv));
}

/* ------------------------------------------------------------------------ */
/* Stable sort of 64-bit keys, ties by input position: the semantics of the
 * Thrust radix sort_by_key the reference calls (makeGroups.cu:270-277).
 * Plain LSD radix, 8 passes of 8 bits, OpenMP-parallel histograms.          */
/* ------------------------------------------------------------------------ */
void oracle_argsort_u64(int n, const uint64_t *keys_in, int *perm)
{
  uint64_t *k0 = (uint64_t *)malloc(sizeof(uint64_t) * (size_t)(n > 0 ? n : 1));
  uint64_t *k1 = (uint64_t *)malloc(sizeof(uint64_t) * (size_t)(n > 0 ? n : 1));
  int *v0 = perm;
  int *v1 = (int *)malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
  memcpy(k0, keys_in, sizeof(uint64_t) * (size_t)n);
  for (int i = 0; i < n; i++) v0[i] = i;
  int nt = 1;
#ifdef _OPENMP
  nt = omp_get_max_threads();
#endif
  size_t *hist = (size_t *)malloc(sizeof(size_t) * 256 * (size_t)nt);
  for (int pass = 0; pass < 8; pass++) {
    const int sh = 8 * pass;
    memset(hist, 0, sizeof(size_t) * 256 * (size_t)nt);
#pragma omp parallel num_threads(nt)
    {
      int t = 0, T = 1;
#ifdef _OPENMP
      t = omp_get_thread_num();
      T = omp_get_num_threads();
#endif
      const long b = (long)n * t / T, e = (long)n * (t + 1) / T;
      size_t *h = hist + 256 * (size_t)t;
      for (long i = b; i < e; i++) h[(k0[i] >> sh) & 255]++;
#pragma omp barrier
#pragma omp single
      {
        size_t run = 0;
        for (int d = 0; d < 256; d++)
          for (int u = 0; u < T; u++) {
            const size_t c = hist[256 * (size_t)u + d];
            hist[256 * (size_t)u + d] = run;
            run += c;
          }
      }
      for (long i = b; i < e; i++) {
        const int d = (int)((k0[i] >> sh) & 255);
        const size_t o = h[d]++;
        k1[o] = k0[i];
        v1[o] = v0[i];
      }
    }
    uint64_t *tk = k0; k0 = k1; k1 = tk;
    int *tv = v0; v0 = v1; v1 = tv;
  }
  /* 8 passes: v0 is back at perm */
  free(k0); free(k1); free(v1); free(hist);
}

/* ------------------------------------------------------------------------ */
/* Octree by comparison partition, breadth first.  Restates the semantics of
 * buildOctant/buildOctree (buildTree.cu:170-722) and the level sort that
 * follows (buildTree.cu:725-841, :932-958):
 *   - the root (level 0) is always split and is not stored; level-1 cells
 *     start at index 0 (buildTree.cu:424,696-703);
 *   - a child with more than nleaf particles is split (:394,:444), one with
 *     1..nleaf particles is a leaf (:395,:541-549); empty octants make no cell;
 *   - cells are stored level by level; within a level in parent order and
 *     octant order (the reference's order there is atomicAdd order; this is
 *     its canonical form);
 *   - particles inside a cell keep input order (stable partition).
 * A cell at level 21 with more than nleaf particles is kept as a leaf and
 * *overflow is set (the reference recurses without a depth limit).
 * Outputs: perm[n] (tree position -> input index), per cell: level, pbeg,
 * pend, first child, nchild (0 for leaves), parent (-1 for level 1).
 * level_beg[L], level_end[L] (half-open, L=0..31).  Returns ncells, or -1
 * when cap is too small.                                                    */
/* ------------------------------------------------------------------------ */
typedef struct { float c[3], h; } or_box_t;

int oracle_build_tree(int n, const float *p4, const float *box, int nleaf, int cap, int *perm,
                      int *level, int *pbeg, int *pend, int *first, int *nchild, int *parent,
                      int *level_beg, int *level_end, int *overflow)
{
  *overflow = 0;
  for (int L = 0; L < 32; L++) level_beg[L] = level_end[L] = 0;
  int *tmp = (int *)malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
  or_box_t *cbox = (or_box_t *)malloc(sizeof(or_box_t) * (size_t)(cap > 0 ? cap : 1));
  for (int i = 0; i < n; i++) perm[i] = i;
  /* node work list of the current level: (range, box, cell index or -1 for root) */
  typedef struct { int b, e, cell; or_box_t box; } node_t;
  node_t *cur = (node_t *)malloc(sizeof(node_t));
  int ncur = 1;
  cur[0].b = 0; cur[0].e = n; cur[0].cell = -1;
  memcpy(cur[0].box.c, box, 3 * sizeof(float));
  cur[0].box.h = box[3];
  int ncells = 0;
  int L = 0;
  while (ncur > 0 && n > 0) {
    /* children counts per node (sequential so that the numbering is the
     * canonical BFS order) */
    int *cnt = (int *)malloc(sizeof(int) * 8 * (size_t)ncur);
#pragma omp parallel for schedule(dynamic, 1)
    for (int k = 0; k < ncur; k++) {
      const node_t nd = cur[k];
      int c8[8] = {0, 0, 0, 0, 0, 0, 0, 0};
      for (int i = nd.b; i < nd.e; i++) {
        const float *p = p4 + 4 * (size_t)perm[i];
        const int oct = (nd.box.c[0] <= p[0]) | ((nd.box.c[1] <= p[1]) << 1) | ((nd.box.c[2] <= p[2]) << 2);
        c8[oct]++;
      }
      int off[8], run = nd.b;
      for (int o = 0; o < 8; o++) { off[o] = run; run += c8[o]; cnt[8 * k + o] = c8[o]; }
      for (int i = nd.b; i < nd.e; i++) {
        const int id = perm[i];
        const float *p = p4 + 4 * (size_t)id;
        const int oct = (nd.box.c[0] <= p[0]) | ((nd.box.c[1] <= p[1]) << 1) | ((nd.box.c[2] <= p[2]) << 2);
        tmp[off[oct]++] = id;
      }
      memcpy(perm + nd.b, tmp + nd.b, sizeof(int) * (size_t)(nd.e - nd.b));
    }
    /* emit children of this level */
    const int lev = L + 1;
    level_beg[lev] = ncells;
    int nnext = 0;
    for (int k = 0; k < ncur; k++)
      for (int o = 0; o < 8; o++)
        if (cnt[8 * k + o] > 0) nnext += (cnt[8 * k + o] > nleaf && lev < OR_MAXL);
    node_t *next = (node_t *)malloc(sizeof(node_t) * (size_t)(nnext > 0 ? nnext : 1));
    int inext = 0;
    for (int k = 0; k < ncur; k++) {
      const node_t nd = cur[k];
      int run = nd.b, firstc = ncells, nc = 0;
      for (int o = 0; o < 8; o++) {
        const int c = cnt[8 * k + o];
        if (c == 0) continue;
        if (ncells >= cap) {
          free(cnt); free(next); free(cur); free(tmp); free(cbox);
          return -1;
        }
        const float s = 0.5f * nd.box.h;
        or_box_t cb;
        cb.c[0] = nd.box.c[0] + s * ((o & 1) ? 1.0f : -1.0f);
        cb.c[1] = nd.box.c[1] + s * ((o & 2) ? 1.0f : -1.0f);
        cb.c[2] = nd.box.c[2] + s * ((o & 4) ? 1.0f : -1.0f);
        cb.h = s;
        const int ci = ncells++;
        level[ci] = lev; pbeg[ci] = run; pend[ci] = run + c; parent[ci] = nd.cell;
        first[ci] = -1; nchild[ci] = 0;
        cbox[ci] = cb;
        if (c > nleaf) {
          if (lev < OR_MAXL) {
            next[inext].b = run; next[inext].e = run + c; next[inext].cell = ci; next[inext].box = cb;
            inext++;
          } else {
            *overflow = 1;
          }
        }
        run += c;
        nc++;
      }
      if (nd.cell >= 0) { first[nd.cell] = firstc; nchild[nd.cell] = nc; }
    }
    level_end[lev] = ncells;
    free(cnt);
    free(cur);
    cur = next;
    ncur = nnext;
    L++;
  }
  free(cur); free(tmp); free(cbox);
  return ncells;
}

/* ------------------------------------------------------------------------ */
/* Multipoles, reference arithmetic: restates computeCellMultipoles
 * (computeMultipoles.cu:81-190).  Per cell, particles in chunks of 32 (the
 * warp); lanes past the end reuse the last particle with mass 0 (:130-132);
 * per-lane float products m*x, m*x*x, ... (:20,:45-50) summed with the xor
 * butterfly (:22-28,:52-60) in float, added to double accumulators (:30-33,
 * :62-67); then COM = S1/M, Q = S2/M - COM COM^T in double (:148-158); the
 * opening size from the particle bounding box: l = max(2 max h, 1e-6),
 * s = |cvec - com|, cellOp = l*inv_theta + s (:168-177).
 * Outputs in the reference layout: size4 (com, cellOp^2), mono4 (com, M),
 * quad0 (xx,yy,zz,xy), quad1 (xz,yz).                                        */
/* ------------------------------------------------------------------------ */
static float or_warp_sum(const float v[32])
{
  float a[32];
  for (int l = 0; l < 32; l++) a[l] = v[l];
  for (int s = 16; s >= 1; s >>= 1) {
    float b[32];
    for (int l = 0; l < 32; l++) b[l] = a[l] + a[l ^ s];
    for (int l = 0; l < 32; l++) a[l] = b[l];
  }
  return a[0];
}

void oracle_multipoles_ref(int ncells, const int *pbeg, const int *pend, const float *jpos4,
                           float inv_theta, float *size4, float *mono4, float *quad0, float *quad1)
{
#pragma omp parallel for schedule(dynamic, 64)
  for (int c = 0; c < ncells; c++) {
    const int b = pbeg[c], e = pend[c];
    float rmin[3] = {1e10f, 1e10f, 1e10f}, rmax[3] = {-1e10f, -1e10f, -1e10f};
    double M[4] = {0, 0, 0, 0}, Q[6] = {0, 0, 0, 0, 0, 0};
    for (int i = b; i < e; i += 32) {
      float mx[32], my[32], mz[32], mm[32], qxx[32], qyy[32], qzz[32], qxy[32], qxz[32], qyz[32];
      for (int l = 0; l < 32; l++) {
        const int j = (i + l < e) ? i + l : e - 1;
        const float x = jpos4[4 * (size_t)j], y = jpos4[4 * (size_t)j + 1], z = jpos4[4 * (size_t)j + 2];
        const float m = (i + l < e) ? jpos4[4 * (size_t)j + 3] : 0.0f;
        rmin[0] = fminf(rmin[0], x); rmin[1] = fminf(rmin[1], y); rmin[2] = fminf(rmin[2], z);
        rmax[0] = fmaxf(rmax[0], x); rmax[1] = fmaxf(rmax[1], y); rmax[2] = fmaxf(rmax[2], z);
        mx[l] = m * x; my[l] = m * y; mz[l] = m * z; mm[l] = m;
        qxx[l] = m * x * x; qyy[l] = m * y * y; qzz[l] = m * z * z;
        qxy[l] = m * x * y; qxz[l] = m * x * z; qyz[l] = m * y * z;
      }
      M[0] += or_warp_sum(mx); M[1] += or_warp_sum(my); M[2] += or_warp_sum(mz); M[3] += or_warp_sum(mm);
      Q[0] += or_warp_sum(qxx); Q[1] += or_warp_sum(qyy); Q[2] += or_warp_sum(qzz);
      Q[3] += or_warp_sum(qxy); Q[4] += or_warp_sum(qxz); Q[5] += or_warp_sum(qyz);
    }
    const double inv_mass = 1.0 / M[3];
    M[0] *= inv_mass; M[1] *= inv_mass; M[2] *= inv_mass;
    Q[0] = Q[0] * inv_mass - M[0] * M[0];
    Q[1] = Q[1] * inv_mass - M[1] * M[1];
    Q[2] = Q[2] * inv_mass - M[2] * M[2];
    Q[3] = Q[3] * inv_mass - M[0] * M[1];
    Q[4] = Q[4] * inv_mass - M[0] * M[2];
    Q[5] = Q[5] * inv_mass - M[1] * M[2];
    const float cv[3] = {(rmax[0] + rmin[0]) * 0.5f, (rmax[1] + rmin[1]) * 0.5f, (rmax[2] + rmin[2]) * 0.5f};
    const float hv[3] = {(rmax[0] - rmin[0]) * 0.5f, (rmax[1] - rmin[1]) * 0.5f, (rmax[2] - rmin[2]) * 0.5f};
    const float com[3] = {(float)M[0], (float)M[1], (float)M[2]};
    const float dx = cv[0] - com[0], dy = cv[1] - com[1], dz = cv[2] - com[2];
    const float s = sqrtf(dx * dx + dy * dy + dz * dz);
    const float l = fmaxf(2.0f * fmaxf(hv[0], fmaxf(hv[1], hv[2])), 1.0e-6f);
    const float op = l * inv_theta + s;
    size4[4 * (size_t)c + 0] = com[0]; size4[4 * (size_t)c + 1] = com[1];
    size4[4 * (size_t)c + 2] = com[2]; size4[4 * (size_t)c + 3] = op * op;
    mono4[4 * (size_t)c + 0] = com[0]; mono4[4 * (size_t)c + 1] = com[1];
    mono4[4 * (size_t)c + 2] = com[2]; mono4[4 * (size_t)c + 3] = (float)M[3];
    quad0[4 * (size_t)c + 0] = (float)Q[0]; quad0[4 * (size_t)c + 1] = (float)Q[1];
    quad0[4 * (size_t)c + 2] = (float)Q[2]; quad0[4 * (size_t)c + 3] = (float)Q[3];
    quad1[2 * (size_t)c + 0] = (float)Q[4]; quad1[2 * (size_t)c + 1] = (float)Q[5];
  }
}

/* Exact per-cell moments in FP64, two passes (COM first, then central
 * moments): the yardstick the CUDA multipoles are judged against.
 * out[16*c]: M, com x,y,z, Qxx,Qyy,Qzz,Qxy,Qxz,Qyz (per unit mass),
 * bbox min x,y,z, max x,y,z.                                               */
void oracle_multipoles_fp64(int ncells, const int *pbeg, const int *pend, const float *jpos4, double *out)
{
#pragma omp parallel for schedule(dynamic, 64)
  for (int c = 0; c < ncells; c++) {
    const int b = pbeg[c], e = pend[c];
    double m = 0, sx = 0, sy = 0, sz = 0;
    double mn[3] = {1e300, 1e300, 1e300}, mx[3] = {-1e300, -1e300, -1e300};
    for (int i = b; i < e; i++) {
      const float *p = jpos4 + 4 * (size_t)i;
      m += p[3]; sx += (double)p[3] * p[0]; sy += (double)p[3] * p[1]; sz += (double)p[3] * p[2];
      for (int k = 0; k < 3; k++) { if (p[k] < mn[k]) mn[k] = p[k]; if (p[k] > mx[k]) mx[k] = p[k]; }
    }
    const double cx = sx / m, cy = sy / m, cz = sz / m;
    double q[6] = {0, 0, 0, 0, 0, 0};
    for (int i = b; i < e; i++) {
      const float *p = jpos4 + 4 * (size_t)i;
      const double dx = p[0] - cx, dy = p[1] - cy, dz = p[2] - cz, w = p[3];
      q[0] += w * dx * dx; q[1] += w * dy * dy; q[2] += w * dz * dz;
      q[3] += w * dx * dy; q[4] += w * dx * dz; q[5] += w * dy * dz;
    }
    double *o = out + 16 * (size_t)c;
    o[0] = m; o[1] = cx; o[2] = cy; o[3] = cz;
    for (int k = 0; k < 6; k++) o[4 + k] = q[k] / m;
    for (int k = 0; k < 3; k++) { o[10 + k] = mn[k]; o[13 + k] = mx[k]; }
  }
}

/* ------------------------------------------------------------------------ */
/* Groups: restates makeGroups.cu:137-223 and :259-309.  Keys sorted by PH
 * order are masked to their top level_split octal digits (mask :259-266,
 * level_split clamped to >= 1 as at :259); segments of equal masked key are
 * cut into chunks of ncrit particles (:208-221).  Groups come out ordered by
 * first particle (the reference's order is atomicAdd order).  Returns G.   */
/* ------------------------------------------------------------------------ */
int oracle_make_groups(int n, const uint64_t *sorted_keys, int level_split, int ncrit, int *gbeg, int *gnp)
{
  if (level_split < 1) level_split = 1;
  uint64_t mask = 0;
  for (int i = 0; i < OR_MAXL; i++) {
    mask <<= 3;
    if (i < level_split) mask |= 0x7;
  }
  int g = 0, seg = 0;
  for (int i = 0; i < n; i++) {
    if (i == 0 || (sorted_keys[i] & mask) != (sorted_keys[i - 1] & mask)) seg = i;
    if ((i - seg) % ncrit == 0) {
      int e = i + 1;
      while (e < n && e - i < ncrit && (sorted_keys[e] & mask) == (sorted_keys[i] & mask)) e++;
      gbeg[g] = i;
      gnp[g] = e - i;
      g++;
    }
  }
  return g;
}

/* ------------------------------------------------------------------------ */
/* Tree walk: restates treewalk/treewalk_warp (computeForces.cu:229-619) for
 * one group at a time.  Group box from the min/max of its particles
 * (:539-555); breadth-first from all level-1 cells (:259-263,:511-512);
 * a cell is opened when split_node_grav_impbh (:30-54) says so or when it
 * holds fewer than 3 particles (:284-285); opened nodes push their children
 * to the next level (:291-334); cells that are not opened (leaves too) are
 * evaluated as quadrupoles (:337-367, add_acc :83-128); opened leaves are
 * evaluated particle by particle (:370-430, add_acc :58-78), i==j included.
 * The open test is computed with explicitly rounded operations
 * (fmaf for the distance) so that it reproduces the CUDA path's decisions
 * bit for bit on identical inputs.  Forces are accumulated in float in list
 * order (the CUDA path accumulates in 32-wide batches, so forces agree to
 * float rounding, not bit for bit).
 * cell_data is the reference's CellData packing (Treecode.h:45-89):
 * x = parent | level<<27, y = first | (n-1)<<29 or 0xFFFFFFFF for a leaf,
 * z = pbeg, w = pend.  gsel (may be NULL) selects a subset of groups.
 * Returns 0, or 1 when a level list outgrows its buffer.                   */
/* ------------------------------------------------------------------------ */
static int or_open(const float *cs, const float gc[3], const float gs[3])
{
  float d[3];
  for (int k = 0; k < 3; k++) {
    float v = fabsf(gc[k] - cs[k]) - gs[k];
    v += fabsf(v);
    v *= 0.5f;
    d[k] = v;
  }
  const float ds2 = fmaf(d[2], d[2], fmaf(d[1], d[1], d[0] * d[0]));
  return ds2 < fabsf(cs[3]);
}

int oracle_walk(int ngroups_sel, const int *gsel, const int *gbeg, const int *gnp, const float *ipos4,
                const uint32_t *cell_data, const float *cell_size4, const float *mono4, const float *quad0,
                const float *quad1, int l1_beg, int l1_end, const float *jpos4, float eps2, float *acc4,
                long long *napprox, long long *ndirect)
{
  int err = 0;
#pragma omp parallel reduction(| : err)
  {
    int cap = 1 << 16;
    int *list = (int *)malloc(sizeof(int) * (size_t)cap);
    int *nxt = (int *)malloc(sizeof(int) * (size_t)cap);
    int *appx = (int *)malloc(sizeof(int) * (size_t)cap);
    int *dirp = (int *)malloc(sizeof(int) * (size_t)cap * 16);
#pragma omp for schedule(dynamic, 4)
    for (int s = 0; s < ngroups_sel; s++) {
      const int g = gsel ? gsel[s] : s;
      const int b = gbeg[g], np = gnp[g];
      float mn[3], mx[3];
      for (int k = 0; k < 3; k++) mn[k] = mx[k] = ipos4[4 * (size_t)b + k];
      for (int i = b; i < b + np; i++)
        for (int k = 0; k < 3; k++) {
          mn[k] = fminf(mn[k], ipos4[4 * (size_t)i + k]);
          mx[k] = fmaxf(mx[k], ipos4[4 * (size_t)i + k]);
        }
      float gc[3], gs[3];
      for (int k = 0; k < 3; k++) { gc[k] = 0.5f * (mx[k] + mn[k]); gs[k] = 0.5f * (mx[k] - mn[k]); }
      int nl = 0, na = 0, nd = 0;
      for (int c = l1_beg; c < l1_end; c++) list[nl++] = c;
      while (nl > 0) {
        int nn = 0;
        for (int k = 0; k < nl; k++) {
          const int c = list[k];
          const uint32_t *cd = cell_data + 4 * (size_t)c;
          const int pb = (int)cd[2], pe = (int)cd[3];
          const int split = or_open(cell_size4 + 4 * (size_t)c, gc, gs) || (pe - pb < 3);
          const int isleaf = cd[1] == 0xFFFFFFFFu;
          if (!split) {
            if (na >= cap) { err = 1; continue; }
            appx[na++] = c;
          } else if (!isleaf) {
            const int f = (int)(cd[1] & 0x1FFFFFFFu), nch = (int)(cd[1] >> 29) + 1;
            if (nn + nch > cap) { err = 1; continue; }
            for (int q = 0; q < nch; q++) nxt[nn++] = f + q;
          } else {
            if (nd + (pe - pb) > cap * 16) { err = 1; continue; }
            for (int j = pb; j < pe; j++) dirp[nd++] = j;
          }
        }
        int *t = list; list = nxt; nxt = t;
        nl = nn;
      }
      napprox[g] = na;
      ndirect[g] = nd;
      for (int i = b; i < b + np; i++) {
        const float px = ipos4[4 * (size_t)i], py = ipos4[4 * (size_t)i + 1], pz = ipos4[4 * (size_t)i + 2];
        float ax = 0, ay = 0, az = 0, ph = 0;
        for (int k = 0; k < na; k++) {
          const int c = appx[k];
          const float *m = mono4 + 4 * (size_t)c;
          const float *q0 = quad0 + 4 * (size_t)c, *q1 = quad1 + 2 * (size_t)c;
          const float dx = px - m[0], dy = py - m[1], dz = pz - m[2];
          const float r2 = dx * dx + dy * dy + dz * dz + eps2;
          const float rinv = 1.0f / sqrtf(r2);
          const float rinv2 = rinv * rinv;
          const float mrinv = m[3] * rinv;
          const float mrinv3 = rinv2 * mrinv;
          const float mrinv5 = rinv2 * mrinv3;
          const float mrinv7 = rinv2 * mrinv5;
          const float D0 = mrinv, D1 = -mrinv3, D2 = mrinv5 * 3.0f, D3 = mrinv7 * (-15.0f);
          const float q11 = q0[0], q22 = q0[1], q33 = q0[2], q12 = q0[3], q13 = q1[0], q23 = q1[1];
          const float qq = q11 + q22 + q33;
          const float qRx = q11 * dx + q12 * dy + q13 * dz;
          const float qRy = q12 * dx + q22 * dy + q23 * dz;
          const float qRz = q13 * dx + q23 * dy + q33 * dz;
          const float qRR = qRx * dx + qRy * dy + qRz * dz;
          ph -= D0 + 0.5f * (D1 * qq + D2 * qRR);
          const float C = D1 + 0.5f * (D2 * qq + D3 * qRR);
          ax += C * dx + D2 * qRx;
          ay += C * dy + D2 * qRy;
          az += C * dz + D2 * qRz;
        }
        for (int k = 0; k < nd; k++) {
          const float *pj = jpos4 + 4 * (size_t)dirp[k];
          const float dx = pj[0] - px, dy = pj[1] - py, dz = pj[2] - pz;
          const float r2 = dx * dx + dy * dy + dz * dz + eps2;
          const float rinv = 1.0f / sqrtf(r2);
          const float rinv2 = rinv * rinv;
          const float mrinv = pj[3] * rinv;
          const float mrinv3 = mrinv * rinv2;
          ph -= mrinv;
          ax += mrinv3 * dx; ay += mrinv3 * dy; az += mrinv3 * dz;
        }
        acc4[4 * (size_t)i + 0] = ax; acc4[4 * (size_t)i + 1] = ay;
        acc4[4 * (size_t)i + 2] = az; acc4[4 * (size_t)i + 3] = ph;
      }
    }
    free(list); free(nxt); free(appx); free(dirp);
  }
  return err;
}

/* ------------------------------------------------------------------------ */
/* FP64 direct summation (the force oracle): for each sample i, sum over all
 * j of m_j (x_j - x_i) / (r^2+eps^2)^(3/2) and -m_j / sqrt(r^2+eps^2); the
 * i==j term (0 force, -m_i/eps potential, as computeForces.cu:58-78 includes
 * it) is added only when include_self is set.  out[4*s] = ax, ay, az, phi. */
/* ------------------------------------------------------------------------ */
void oracle_direct_fp64(int n, const float *pos4, int nsample, const int *sample, double eps2,
                        int include_self, double *out)
{
#pragma omp parallel for schedule(dynamic, 1)
  for (int s = 0; s < nsample; s++) {
    const int i = sample[s];
    const double xi = pos4[4 * (size_t)i], yi = pos4[4 * (size_t)i + 1], zi = pos4[4 * (size_t)i + 2];
    double ax = 0, ay = 0, az = 0, ph = 0;
    for (int j = 0; j < n; j++) {
      if (j == i && !include_self) continue;
      const double dx = pos4[4 * (size_t)j] - xi, dy = pos4[4 * (size_t)j + 1] - yi, dz = pos4[4 * (size_t)j + 2] - zi;
      const double r2 = dx * dx + dy * dy + dz * dz + eps2;
      const double rinv = 1.0 / sqrt(r2);
      const double mr = pos4[4 * (size_t)j + 3] * rinv;
      const double mr3 = mr * rinv * rinv;
      ax += mr3 * dx; ay += mr3 * dy; az += mr3 * dz; ph -= mr;
    }
    out[4 * (size_t)s + 0] = ax; out[4 * (size_t)s + 1] = ay;
    out[4 * (size_t)s + 2] = az; out[4 * (size_t)s + 3] = ph;
  }
}

/* ------------------------------------------------------------------------ */
/* Leapfrog move + energies.  The reference's moveParticles/computeEnergies
 * are stubs (moveParticles.cu:3-7, computeEnergies.cu:3-7); this restates
 * the project's kick-drift-kick definition with merged kicks:
 *   if closing: v += a dt/2         (closing kick of the previous step)
 *   energies at the synchronised point (FP64 sums)
 *   v += a dt/2; x += v dt          (opening kick + drift)
 * acc4 w holds the potential (computeForces.cu:72,119).  Float updates use
 * fmaf like the CUDA kernel.  e[0]=T, e[1]=W=1/2 sum m phi, e[2]=W without
 * the i==j self term (W + 1/2 sum m^2/eps), e[3]=T+e[2], e[4..6]=momentum,
 * e[7]=total mass.                                                          */
/* ------------------------------------------------------------------------ */
void oracle_move(int n, float *pos4, float *vel4, const float *acc4, float dt, int closing, float eps,
                 double *e)
{
  const float h = 0.5f * dt;
  double T = 0, W = 0, S = 0, px = 0, py = 0, pz = 0, mt = 0;
#pragma omp parallel for schedule(static) reduction(+ : T, W, S, px, py, pz, mt)
  for (int i = 0; i < n; i++) {
    float *p = pos4 + 4 * (size_t)i, *v = vel4 + 4 * (size_t)i;
    const float *a = acc4 + 4 * (size_t)i;
    if (closing)
      for (int k = 0; k < 3; k++) v[k] = fmaf(a[k], h, v[k]);
    const double m = p[3];
    T += 0.5 * m * ((double)v[0] * v[0] + (double)v[1] * v[1] + (double)v[2] * v[2]);
    W += 0.5 * m * a[3];
    S += 0.5 * m * m / eps;
    px += m * v[0]; py += m * v[1]; pz += m * v[2]; mt += m;
    for (int k = 0; k < 3; k++) v[k] = fmaf(a[k], h, v[k]);
    for (int k = 0; k < 3; k++) p[k] = fmaf(v[k], dt, p[k]);
  }
  e[0] = T; e[1] = W; e[2] = W + S; e[3] = T + W + S;
  e[4] = px; e[5] = py; e[6] = pz; e[7] = mt;
}

int oracle_num_threads(void)
{
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}
