// learned.cu -- per-group opening bounds from a small MLP.
//
// The walk opens a cell when the group is inside its geometric opening
// sphere (computeForces.cu:30-54) at the group's angle theta_g, or -- in the
// relative accuracy mode -- when the cell's octupole truncation error, of
// order M l^3 / ds^5, exceeds the group's bound tau_g.  A single angle must
// suit the worst group; per-group angles alone gain little (their best
// allocation is a few tens of percent and cannot be predicted from group
// features), while a bound on each cell's truncation error relative to the
// group's own acceleration puts the error budget where it matters.  Here a
// 16 -> 64 -> 64 -> 1 network maps group features to y_g = log10(tau_g / A_g),
// A_g being the group's mean |a| of the previous force evaluation; it is
// trained on pairs (features, y label) that the walk and the FP64 direct sum
// generate (bonsai2_b200/learned.py: each group's error and cost over a grid
// of y; the label is the cost-optimal y for the error budget, or the y at
// which the group's error meets the target), with this file's own forward
// and backward kernels.  theta_g is then a fixed safety bound.  Without previous
// accelerations (the first evaluation after particles are loaded) every
// group walks at the fixed angle (theta mode 0's walk, bit for bit).
//
// Features (per group, normalised logs clamped to [-10, 10]): size, radius,
// tree depth (common PH-key prefix), distance from and mass share of its
// system, density, shape, system size, softening over radius, the previous
// acceleration scale A_g and its spread over the group, and -- recorded by
// the previous walk of the group holding the group's middle particle -- the
// number of cells near the opening boundary, the mass share of the accepted
// cells near it, and the force-weighted quadrupole norm of the accepted
// cells.
//
// Weight vector layout (kMlpWeights floats): W1[64][16], b1[64], W2[64][64],
// b2[64], w3[64], b3.  Hidden activations tanh; output
// y = lo + (hi - lo) * sigmoid(z).
#include "common.cuh"
#include "kernels.cuh"

#include <cuda_fp16.h>

namespace bonsai {

constexpr int kF = kMlpFeatures, kH = kMlpHidden;
constexpr int oW1 = 0, oB1 = oW1 + kH * kF, oW2 = oB1 + kH, oB2 = oW2 + kH * kH, oW3 = oB2 + kH, oB3 = oW3 + kH;
static_assert(oB3 + 1 == kMlpWeights, "weight layout");

__device__ __forceinline__ float safe_log10(float x) { return log10f(fmaxf(x, 1e-30f)); }

// ---------------------------------------------------------------------------
// Group features (one warp per group; groups are contiguous in PH order).
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_group_features(const int2* __restrict__ groups,
                                                        const TreeInfo* __restrict__ info,
                                                        const float4* __restrict__ ipos,
                                                        const unsigned long long* __restrict__ ph_sorted,
                                                        const MpRec* __restrict__ rec, const Box* __restrict__ box,
                                                        int n, int ncrit, float eps, float* __restrict__ feat,
                                                        const int* __restrict__ sys_off, int nsys,
                                                        const int* __restrict__ root_beg, const PrevEval prev,
                                                        float* __restrict__ amag) {
  const int lane = threadIdx.x & 31;
  const int ng = info->ngroups;
  const bool have_prev = prev.acc_valid && *prev.acc_valid;
  // the group's system: its centre of mass and mass from its level-1 cells,
  // its box and its size (an ensemble's systems each have their own)
  int sys = -1;
  float mtot = 0.f, cx = 0.f, cy = 0.f, cz = 0.f, hs = 0.f;
  int ns = n;
  const int nw = (gridDim.x * blockDim.x) >> 5;
  for (int g = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; g < ng; g += nw) {
    const int2 gd = groups[g];
    const int pb = gd.x, np = gd.y;
    const int s = nsys > 1 ? sys_of(sys_off, nsys, pb) : 0;
    if (s != sys) {
      sys = s;
      const int c0 = nsys > 1 ? root_beg[s] : info->level_beg[1];
      const int c1 = nsys > 1 ? root_beg[s + 1] : info->level_end[1];
      double M = 0, X = 0, Y = 0, Z = 0;
      for (int c = c0; c < c1; c++) {
        const double m = rec[c].m;
        M += m; X += m * rec[c].cx; Y += m * rec[c].cy; Z += m * rec[c].cz;
      }
      mtot = (float)M;
      cx = M > 0 ? (float)(X / M) : 0.f; cy = M > 0 ? (float)(Y / M) : 0.f; cz = M > 0 ? (float)(Z / M) : 0.f;
      hs = box[s].hsize;
      ns = nsys > 1 ? sys_off[s + 1] - sys_off[s] : n;
    }
    float mn[3] = {3e38f, 3e38f, 3e38f}, mx[3] = {-3e38f, -3e38f, -3e38f};
    float mg = 0.f, am = 0.f, al = 0.f, al2 = 0.f;
    for (int i = lane; i < np; i += 32) {
      const float4 p = ipos[pb + i];
      mn[0] = fminf(mn[0], p.x); mn[1] = fminf(mn[1], p.y); mn[2] = fminf(mn[2], p.z);
      mx[0] = fmaxf(mx[0], p.x); mx[1] = fmaxf(mx[1], p.y); mx[2] = fmaxf(mx[2], p.z);
      mg += p.w;
      if (have_prev) {
        const int k = pb + i;
        const int j = prev.perm ? __ldg(prev.perm + k) : k;
        const float4 a = BONSAI_IN_RANGE(j, n, 0x501) ? __ldg(prev.acc + j) : make_float4(0.f, 0.f, 0.f, 0.f);
        const float m = sqrtf(a.x * a.x + a.y * a.y + a.z * a.z);
        const float lm = safe_log10(m);
        am += m; al += lm; al2 += lm * lm;
      }
    }
    for (int k = 0; k < 3; k++) { mn[k] = warp_min_f32(mn[k]); mx[k] = warp_max_f32(mx[k]); }
#pragma unroll
    for (int o = 16; o; o >>= 1) {
      mg += __shfl_xor_sync(kFull, mg, o);
      am += __shfl_xor_sync(kFull, am, o);
      al += __shfl_xor_sync(kFull, al, o);
      al2 += __shfl_xor_sync(kFull, al2, o);
    }
    const float gx = 0.5f * (mx[0] + mn[0]), gy = 0.5f * (mx[1] + mn[1]), gz = 0.5f * (mx[2] + mn[2]);
    const float sx = 0.5f * (mx[0] - mn[0]), sy = 0.5f * (mx[1] - mn[1]), sz = 0.5f * (mx[2] - mn[2]);
    const float rg = fmaxf(sqrtf(sx * sx + sy * sy + sz * sz), 1e-12f * hs);
    if (lane == 0) {
      const float dg = sqrtf((gx - cx) * (gx - cx) + (gy - cy) * (gy - cy) + (gz - cz) * (gz - cz));
      const int lvl = diff_level(ph_sorted[pb], ph_sorted[pb + np - 1]) - 1;  // common PH prefix (levels)
      const float vol = rg * rg * rg;
      // the previous evaluation: acceleration scale (floored at 1e-4 of the
      // system's M / hsize^2, so that a group at an exact balance point does not
      // open everything) and the statistics of the group that held the
      // group's middle particle
      const float afloor = 1e-4f * mtot / fmaxf(hs * hs, 1e-30f);
      float A = 0.f, spread = 0.f;
      float4 st = make_float4(0.f, 0.f, 0.f, 0.f);
      if (have_prev) {
        A = fmaxf(am / (float)np, afloor);
        const float mu = al / (float)np;
        spread = sqrtf(fmaxf(al2 / (float)np - mu * mu, 0.f));
        const int k = pb + np / 2;
        const int j = prev.perm ? __ldg(prev.perm + k) : k;
        if (prev.acc_valid[1] && BONSAI_IN_RANGE(j, n, 0x502)) {
          const int og = __ldg(prev.part_gid + j);
          if (og >= 0 && og < prev.stats_cap) st = __ldg(prev.stats + og);
        }
      }
      amag[g] = A;
      float f[kF];
      f[0] = (float)np / (float)ncrit;                               // group size
      f[1] = safe_log10(rg / hs) / 6.f;                              // radius
      f[2] = (float)min(lvl, kMaxLevel) / (float)kMaxLevel;          // tree depth
      f[3] = safe_log10(dg / hs + 1e-7f) / 6.f;                      // distance from the system's centre
      f[4] = safe_log10(mg / fmaxf(mtot, 1e-30f)) / 8.f;             // mass share
      f[5] = safe_log10((float)np / vol * hs * hs * hs / (float)ns) / 8.f;  // density
      f[6] = sx / rg; f[7] = sy / rg; f[8] = sz / rg;                // shape
      f[9] = log10f((float)ns) / 8.f;                                // system size
      f[10] = safe_log10(fmaxf(eps, 1e-12f) / rg) / 3.f;             // softening / radius
      f[11] = have_prev ? safe_log10(A * hs * hs / fmaxf(mtot, 1e-30f)) / 3.f : 0.f;  // acceleration scale
      f[12] = spread;                                                // its spread (dex)
      f[13] = log10f(1.0f + st.x) / 4.f;                             // cells near the opening boundary
      f[14] = st.y;                                                  // accepted mass near it
      f[15] = have_prev ? safe_log10(st.z + 1e-12f) / 3.f : 0.f;     // quadrupole norm of accepted cells
      // degenerate groups (a one-particle system's box and radius are floored
      // near 1e-12, so the density's float products under- and overflow) give
      // inf or NaN; the features are normalised logs well inside [-10, 10], and
      // fmaxf returns its other operand for a NaN
      float* o = feat + (size_t)g * kF;
#pragma unroll
      for (int k = 0; k < kF; k++) o[k] = fminf(fmaxf(f[k], -10.0f), 10.0f);
    }
  }
}

// ---------------------------------------------------------------------------
// Inference: FP16 weights in shared memory, FP32 accumulation; one warp per
// group (lane holds hidden units lane and lane+32) writes 1/theta_g.  W1 and
// W2 are staged transposed (input-major), so that the 32 lanes of a step read
// 32 consecutive weights: row-major, lane j's row starts j * 128 bytes apart
// and every lane of the warp hits the same bank.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_mlp_infer(const float* __restrict__ feat, const __half* __restrict__ wh,
                                                   const TreeInfo* __restrict__ info, float lo, float hi,
                                                   const float* __restrict__ amag, const int* __restrict__ acc_valid,
                                                   float inv_bound, float inv_fixed, float start_alpha,
                                                   float* __restrict__ group_inv_theta, float* __restrict__ group_tau) {
  __shared__ __half sw[kMlpWeights + 1];
  __shared__ float sh[8][kH];
  for (int t = threadIdx.x; t < kMlpWeights; t += blockDim.x) {
    int d = t;
    if (t < oB1) d = oW1 + (t % kF) * kH + t / kF;                          // W1[j][k] -> [k][j]
    else if (t >= oW2 && t < oB2) d = oW2 + ((t - oW2) % kH) * kH + (t - oW2) / kH;  // W2[j][i] -> [i][j]
    sw[d] = wh[t];
  }
  __syncthreads();
  const int lane = threadIdx.x & 31, wi = threadIdx.x >> 5;
  const int ng = info->ngroups;
  const int nw = (gridDim.x * blockDim.x) >> 5;
  for (int g = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; g < ng; g += nw) {
    const float xk = lane < kF ? feat[(size_t)g * kF + lane] : 0.f;
#pragma unroll
    for (int u = 0; u < 2; u++) {
      const int j = lane + 32 * u;
      float a = __half2float(sw[oB1 + j]);
#pragma unroll
      for (int k = 0; k < kF; k++) a = fmaf(__half2float(sw[oW1 + k * kH + j]), __shfl_sync(kFull, xk, k), a);
      sh[wi][j] = tanhf(a);
    }
    __syncwarp();
    float z = 0.f;
#pragma unroll
    for (int u = 0; u < 2; u++) {
      const int j = lane + 32 * u;
      float a = __half2float(sw[oB2 + j]);
#pragma unroll 8
      for (int i = 0; i < kH; i++) a = fmaf(__half2float(sw[oW2 + i * kH + j]), sh[wi][i], a);
      z = fmaf(__half2float(sw[oW3 + j]), tanhf(a), z);
    }
#pragma unroll
    for (int o = 16; o; o >>= 1) z += __shfl_xor_sync(kFull, z, o);
    z += __half2float(sw[oB3]);
    if (lane == 0) {
      if (acc_valid[0] && acc_valid[1] != 2) {
        // the previous walk was not a relative walk with statistics (the
        // fixed-angle fallback, or another theta mode): the network never
        // saw such statistics in training, so one evaluation takes the
        // single-parameter bound, the relative walk the training tables were
        // recorded after (after the fallback, the network's own bounds
        // overshot the error target by ~2x in this evaluation)
        group_tau[g] = start_alpha * amag[g];
        group_inv_theta[g] = inv_bound;
      } else if (acc_valid[0]) {
        const float y = lo + (hi - lo) / (1.0f + expf(-z));
        group_tau[g] = amag[g] * exp10f(y);
        group_inv_theta[g] = inv_bound;
      } else {  // no previous accelerations: the fixed angle
        group_tau[g] = 0.0f;
        group_inv_theta[g] = inv_fixed;
      }
    }
    __syncwarp();
  }
}

__global__ void k_relative_tau(const TreeInfo* __restrict__ info, const float* __restrict__ amag,
                               const int* __restrict__ acc_valid, float alpha, float inv_bound, float inv_fixed,
                               float* __restrict__ inv, float* __restrict__ tau) {
  const int ng = info->ngroups;
  const bool v = *acc_valid != 0;
  for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < ng; g += gridDim.x * blockDim.x) {
    tau[g] = v ? alpha * amag[g] : 0.0f;
    inv[g] = v ? inv_bound : inv_fixed;
  }
}

__global__ void k_weights_to_half(const float* __restrict__ w, __half* __restrict__ wh) {
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < kMlpWeights; t += gridDim.x * blockDim.x)
    wh[t] = __float2half_rn(w[t]);
}

__global__ void k_fill_inv_theta(const TreeInfo* __restrict__ info, const float* __restrict__ theta, float c,
                                 float* __restrict__ inv) {
  const int ng = info->ngroups;
  for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < ng; g += gridDim.x * blockDim.x)
    inv[g] = 1.0f / (theta ? theta[g] : c);
}

// ---------------------------------------------------------------------------
// Training.  Loss per sample: 0.5 (theta - y)^2 (1 + over [theta > y]), mean
// over the S samples (over-prediction costs accuracy, so it is weighted).
// k_mlp_fwd_bwd: one warp per sample (lane holds hidden units lane, lane+32),
// stores the activations and back-propagated deltas; the weight gradients are
// then fixed-order sums over samples (deterministic).
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_mlp_fwd_bwd(const float* __restrict__ X, const float* __restrict__ y, int S,
                                                     const float* __restrict__ w, float lo, float hi, float over,
                                                     float* __restrict__ H1, float* __restrict__ D1,
                                                     float* __restrict__ H2, float* __restrict__ D2,
                                                     float* __restrict__ G, float* __restrict__ loss,
                                                     float* __restrict__ pred) {
  __shared__ float sh[8][2][kH];
  // weights staged once per block: W1 and W2 transposed for the forward pass
  // (lanes read consecutive hidden units), W2 row-major for the backward pass
  // (lanes read consecutive inputs); the rest as they are
  __shared__ float sw1t[kF * kH], sw2t[kH * kH], sw2[kH * kH], sb1[kH], sb2[kH], sw3[kH], sb3;
  for (int t = threadIdx.x; t < kH * kF; t += blockDim.x) sw1t[(t % kF) * kH + t / kF] = w[oW1 + t];
  for (int t = threadIdx.x; t < kH * kH; t += blockDim.x) {
    const float v = w[oW2 + t];
    sw2[t] = v;
    sw2t[(t % kH) * kH + t / kH] = v;
  }
  for (int t = threadIdx.x; t < kH; t += blockDim.x) { sb1[t] = w[oB1 + t]; sb2[t] = w[oB2 + t]; sw3[t] = w[oW3 + t]; }
  if (threadIdx.x == 0) sb3 = w[oB3];
  __syncthreads();
  const int lane = threadIdx.x & 31, wi = threadIdx.x >> 5;
  const int nw = (gridDim.x * blockDim.x) >> 5;
  for (int s = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; s < S; s += nw) {
    float x[kF];
#pragma unroll
    for (int k = 0; k < kF; k++) x[k] = X[(size_t)s * kF + k];
    float h1[2], h2[2];
#pragma unroll
    for (int u = 0; u < 2; u++) {
      const int j = lane + 32 * u;
      float a = sb1[j];
#pragma unroll
      for (int k = 0; k < kF; k++) a = fmaf(sw1t[k * kH + j], x[k], a);
      h1[u] = tanhf(a);
      sh[wi][0][j] = h1[u];
    }
    __syncwarp();
#pragma unroll
    for (int u = 0; u < 2; u++) {
      const int j = lane + 32 * u;
      float a = sb2[j];
      for (int i = 0; i < kH; i++) a = fmaf(sw2t[i * kH + j], sh[wi][0][i], a);
      h2[u] = tanhf(a);
    }
    float z = sw3[lane] * h2[0] + sw3[lane + 32] * h2[1];
#pragma unroll
    for (int o = 16; o; o >>= 1) z += __shfl_xor_sync(kFull, z, o);
    z += sb3;
    const float sg = 1.0f / (1.0f + expf(-z));
    const float th = lo + (hi - lo) * sg;
    const float e = th - y[s];
    const float wgt = e > 0.f ? 1.0f + over : 1.0f;
    const float gz = e * wgt * (hi - lo) * sg * (1.0f - sg) / (float)S;  // d(mean loss)/dz
    float d2[2];
#pragma unroll
    for (int u = 0; u < 2; u++) {
      const int j = lane + 32 * u;
      d2[u] = gz * sw3[j] * (1.0f - h2[u] * h2[u]);
      sh[wi][1][j] = d2[u];
    }
    __syncwarp();
#pragma unroll
    for (int u = 0; u < 2; u++) {
      const int i = lane + 32 * u;
      float a = 0.f;
      for (int j = 0; j < kH; j++) a = fmaf(sw2[j * kH + i], sh[wi][1][j], a);
      const float d1 = a * (1.0f - h1[u] * h1[u]);
      H1[(size_t)s * kH + i] = h1[u];
      D1[(size_t)s * kH + i] = d1;
      H2[(size_t)s * kH + i] = h2[u];
      D2[(size_t)s * kH + i] = d2[u];
    }
    if (lane == 0) {
      G[s] = gz;
      loss[s] = 0.5f * e * e * wgt;
      pred[s] = th;
    }
    __syncwarp();
  }
}

// Weight gradients as fixed-order sums over the samples, in two levels:
// block (x, c) sums samples [c * chunk, (c + 1) * chunk) in order for 256
// weights into part[c][t]; k_mlp_grad_fold then adds the chunks in order.
constexpr int kGradChunks = 32;
__global__ void __launch_bounds__(256) k_mlp_grad(const float* __restrict__ X, int S, const float* __restrict__ H1,
                                                  const float* __restrict__ D1, const float* __restrict__ H2,
                                                  const float* __restrict__ D2, const float* __restrict__ G,
                                                  float* __restrict__ part) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= kMlpWeights) return;
  const int chunk = (S + kGradChunks - 1) / kGradChunks;
  const int s0 = blockIdx.y * chunk, s1 = min(S, s0 + chunk);
  float acc = 0.f;
  if (t < oB1) {  // W1[j][k] = sum d1[j] x[k]
    const int j = t / kF, k = t % kF;
    for (int s = s0; s < s1; s++) acc = fmaf(D1[(size_t)s * kH + j], X[(size_t)s * kF + k], acc);
  } else if (t < oW2) {
    const int j = t - oB1;
    for (int s = s0; s < s1; s++) acc += D1[(size_t)s * kH + j];
  } else if (t < oB2) {  // W2[j][i] = sum d2[j] h1[i]
    const int j = (t - oW2) / kH, i = (t - oW2) % kH;
    for (int s = s0; s < s1; s++) acc = fmaf(D2[(size_t)s * kH + j], H1[(size_t)s * kH + i], acc);
  } else if (t < oW3) {
    const int j = t - oB2;
    for (int s = s0; s < s1; s++) acc += D2[(size_t)s * kH + j];
  } else if (t < oB3) {  // w3[j] = sum g h2[j]
    const int j = t - oW3;
    for (int s = s0; s < s1; s++) acc = fmaf(G[s], H2[(size_t)s * kH + j], acc);
  } else {
    for (int s = s0; s < s1; s++) acc += G[s];
  }
  part[(size_t)blockIdx.y * kMlpWeights + t] = acc;
}

__global__ void k_mlp_grad_fold(const float* __restrict__ part, float* __restrict__ grad) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= kMlpWeights) return;
  float acc = 0.f;
  for (int c = 0; c < kGradChunks; c++) acc += part[(size_t)c * kMlpWeights + t];
  grad[t] = acc;
}

__global__ void k_adam(float* __restrict__ w, const float* __restrict__ grad, float* __restrict__ m,
                       float* __restrict__ v, float lr, float b1, float b2, float c1, float c2) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= kMlpWeights) return;
  const float g = grad[t];
  const float mt = b1 * m[t] + (1.f - b1) * g;
  const float vt = b2 * v[t] + (1.f - b2) * g * g;
  m[t] = mt;
  v[t] = vt;
  w[t] -= lr * (mt / c1) / (sqrtf(vt / c2) + 1e-8f);
}

__global__ void k_sum_f(const float* __restrict__ a, int S, double* __restrict__ out) {
  // one block: fixed-order partials, then lane 0 folds them
  __shared__ double sh[256];
  double s = 0;
  for (int i = threadIdx.x; i < S; i += blockDim.x) s += a[i];
  sh[threadIdx.x] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0;
    for (int i = 0; i < (int)blockDim.x; i++) t += sh[i];
    *out = t;
  }
}

// scratch for training: H1, D1, H2, D2 (S x kH each), G, loss, pred (S each),
// the gradient partials (kGradChunks x kMlpWeights)
size_t mlp_train_scratch_floats(int S) { return (size_t)S * (4 * kH + 3) + (size_t)kGradChunks * kMlpWeights; }

void mlp_loss_grad(const float* X, const float* y, int S, const float* w, float lo, float hi, float over,
                   float* scratch, float* grad, double* loss_out, cudaStream_t st) {
  float* H1 = scratch;
  float* D1 = H1 + (size_t)S * kH;
  float* H2 = D1 + (size_t)S * kH;
  float* D2 = H2 + (size_t)S * kH;
  float* G = D2 + (size_t)S * kH;
  float* L = G + S;
  float* P = L + S;
  float* part = P + S;
  const int blocks = (S + 7) / 8 < 512 ? (S + 7) / 8 : 512;
  k_mlp_fwd_bwd<<<blocks, 256, 0, st>>>(X, y, S, w, lo, hi, over, H1, D1, H2, D2, G, L, P);
  k_mlp_grad<<<dim3((kMlpWeights + 255) / 256, kGradChunks), 256, 0, st>>>(X, S, H1, D1, H2, D2, G, part);
  k_mlp_grad_fold<<<(kMlpWeights + 255) / 256, 256, 0, st>>>(part, grad);
  if (loss_out) k_sum_f<<<1, 256, 0, st>>>(L, S, loss_out);
}

void mlp_adam_step(float* w, const float* grad, float* m, float* v, float lr, int step, cudaStream_t st) {
  const float b1 = 0.9f, b2 = 0.999f;
  const float c1 = 1.f - powf(b1, (float)step), c2 = 1.f - powf(b2, (float)step);
  k_adam<<<(kMlpWeights + 255) / 256, 256, 0, st>>>(w, grad, m, v, lr, b1, b2, c1, c2);
}

void mlp_predict(const float* X, int S, const float* w, float lo, float hi, float* scratch, float* pred,
                 cudaStream_t st) {
  // reuse the training forward with zero targets; pred is the last scratch row
  float* H1 = scratch;
  float* D1 = H1 + (size_t)S * kH;
  float* H2 = D1 + (size_t)S * kH;
  float* D2 = H2 + (size_t)S * kH;
  float* G = D2 + (size_t)S * kH;
  float* L = G + S;
  const int blocks = (S + 7) / 8 < 512 ? (S + 7) / 8 : 512;
  k_mlp_fwd_bwd<<<blocks, 256, 0, st>>>(X, pred, S, w, lo, hi, 0.f, H1, D1, H2, D2, G, L, pred);
}

void launch_group_features(const int2* groups, const TreeInfo* info, const float4* ipos,
                           const unsigned long long* ph_sorted, const MpRec* rec, const Box* box, int n, int ncrit,
                           float eps, float* feat, const int* sys_off, int nsys, const int* root_beg,
                           const PrevEval& prev, float* amag, int nblocks, cudaStream_t st) {
  k_group_features<<<nblocks, 256, 0, st>>>(groups, info, ipos, ph_sorted, rec, box, n, ncrit, eps, feat, sys_off,
                                            nsys, root_beg, prev, amag);
}

void launch_mlp_infer(const float* feat, const void* wh, const TreeInfo* info, float lo, float hi, const float* amag,
                      const int* acc_valid, float inv_bound, float inv_fixed, float start_alpha, float* inv, float* tau,
                      int nblocks, cudaStream_t st) {
  k_mlp_infer<<<nblocks, 256, 0, st>>>(feat, static_cast<const __half*>(wh), info, lo, hi, amag, acc_valid,
                                       inv_bound, inv_fixed, start_alpha, inv, tau);
}

void launch_relative_tau(const TreeInfo* info, const float* amag, const int* acc_valid, float alpha, float inv_bound,
                         float inv_fixed, float* inv, float* tau, int nblocks, cudaStream_t st) {
  k_relative_tau<<<nblocks, 256, 0, st>>>(info, amag, acc_valid, alpha, inv_bound, inv_fixed, inv, tau);
}

void launch_weights_to_half(const float* w, void* wh, cudaStream_t st) {
  k_weights_to_half<<<(kMlpWeights + 255) / 256, 256, 0, st>>>(w, static_cast<__half*>(wh));
}

void launch_fill_inv_theta(const TreeInfo* info, const float* theta, float c, float* inv, int nblocks,
                           cudaStream_t st) {
  k_fill_inv_theta<<<nblocks, 256, 0, st>>>(info, theta, c, inv);
}

BONSAI_BOUNDS_ACCESSOR(bounds_word_learned)

}  // namespace bonsai
