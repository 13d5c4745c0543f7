// kc_mlp.cuh — the learned initial guess of the implicit solve: a 16 -> 64 ->
// 64 -> 4 MLP (ReLU) that predicts, from a cell's pre-solve state, the four
// primitives the Newton iteration solves for (the start fluid's energy density
// and 3-velocity). Inference runs on the tensor cores with BF16 weights and
// activations and FP32 accumulation (mma.sync m16n8k16, one warp per 32 cells);
// training runs FP32 forward/backward kernels with the weights rounded to BF16
// in the forward pass, so the trained network is the one inference evaluates.
// The prediction only seeds the solve: the same FP64 Newton iteration finishes
// it to the same tolerance, and the plain path (bisection warm start + ladder)
// runs when the seeded ladder fails.
#pragma once
#include <cuda_bf16.h>

#include "kc_dev.cuh"

namespace kc {

using namespace kp;

enum : int { MLP_IN = 16, MLP_H = 64, MLP_OUT = 4 };
// weight blob (floats): input mean/std, output mean/std, W1 [64][16], b1, W2
// [64][64], b2, W3 [4][64], b3 — row-major [out][in]
enum : int {
  MLP_OFF_IMEAN = 0,
  MLP_OFF_ISTD = MLP_OFF_IMEAN + MLP_IN,
  MLP_OFF_OMEAN = MLP_OFF_ISTD + MLP_IN,
  MLP_OFF_OSTD = MLP_OFF_OMEAN + MLP_OUT,
  MLP_OFF_W1 = MLP_OFF_OSTD + MLP_OUT,
  MLP_OFF_B1 = MLP_OFF_W1 + MLP_H * MLP_IN,
  MLP_OFF_W2 = MLP_OFF_B1 + MLP_H,
  MLP_OFF_B2 = MLP_OFF_W2 + MLP_H * MLP_H,
  MLP_OFF_W3 = MLP_OFF_B2 + MLP_H,
  MLP_OFF_B3 = MLP_OFF_W3 + MLP_OUT * MLP_H,
  MLP_NW = MLP_OFF_B3 + MLP_OUT
};

// Standardisation guards. A feature that barely varies over the training
// pairs (a velocity component or field that is ~0 at early times, say) would
// otherwise turn a later, ordinary value into a huge standardised input: the
// feature deviations are floored at MLP_FEATURE_STD_MIN (the features are
// logs and asinh-compressed values, O(1) in scale), and standardised inputs
// and outputs are clipped to +-MLP_STD_CLIP, in training and in inference.
constexpr float MLP_FEATURE_STD_MIN = 1.0e-2f;
constexpr float MLP_STD_CLIP = 8.0f;
KC_HD float mlp_clip(float z) { return z > MLP_STD_CLIP ? MLP_STD_CLIP : (z < -MLP_STD_CLIP ? -MLP_STD_CLIP : z); }

// Raw (unstandardised) features of a cell's pre-solve state: log10 of rho,
// u_int, E_rad, dt, sqrt(-g); asinh-compressed velocities (scale 1e-3) and B
// (scale 1e-12); the start fluid (+1 gas, -1 radiation) in place of the entropy
// slot; the lapse. Computed in FP64, stored as FP32.
KC_HD void mlp_features_raw(const double pp[NV], double dt, double gdet, double alpha, int startwith, float f[MLP_IN]) {
  f[0] = (float)kmath::log(pp[RHO]) * 0.43429448190325176f;
  f[1] = (float)kmath::log(pp[UU]) * 0.43429448190325176f;
  for (int k = 0; k < 3; ++k) f[2 + k] = (float)::asinh(pp[VX + k] * 1.0e3);
  f[5] = startwith == PRIM_MHD ? 1.0f : -1.0f;
  for (int k = 0; k < 3; ++k) f[6 + k] = (float)::asinh(pp[B1 + k] * 1.0e12);
  f[9] = (float)kmath::log(pp[EE]) * 0.43429448190325176f;
  for (int k = 0; k < 3; ++k) f[10 + k] = (float)::asinh(pp[FX + k] * 1.0e3);
  f[13] = (float)kmath::log(dt) * 0.43429448190325176f;
  f[14] = (float)kmath::log(gdet) * 0.43429448190325176f;
  f[15] = (float)alpha;
}
// the index of the start fluid's energy slot (the Newton unknowns are
// pp[sh .. sh+3]), implicit.zig:642
KC_HD int mlp_sh(int startwith) { return startwith == PRIM_MHD ? UU : EE; }
// Targets are the changes the Newton iteration makes, in the units of its
// convergence test (koral/solve/implicit.zig:880: relative energy change,
// velocity change over max(eps, |v|) with eps = 1e-6), asinh-compressed with
// scales 1e-7 (energy) and 1e-9 (velocities): the changes span eight decades,
// and the compression lets the fit resolve the small ones (most cells) to
// below the 1e-8 convergence tolerance while still following the large ones.
constexpr double MLP_SCALE_E = 1.0e-7, MLP_SCALE_V = 1.0e-9, MLP_V_FLOOR = 1.0e-6;
KC_HD double mlp_sinh(double y) { return 0.5 * (kmath::exp(y) - kmath::exp(-y)); }
KC_HD void mlp_targets_raw(const double pp00[NV], const double sol[NV], int startwith, float t[MLP_OUT]) {
  int sh = mlp_sh(startwith);
  t[0] = (float)::asinh(kmath::log(sol[sh] / pp00[sh]) / MLP_SCALE_E);
  for (int k = 1; k < 4; ++k)
    t[k] = (float)::asinh((sol[sh + k] - pp00[sh + k]) / kmath::fmax(MLP_V_FLOOR, kmath::fabs(pp00[sh + k])) /
                          MLP_SCALE_V);
}
// the guess from a (destandardised) network output
KC_HD void mlp_apply(const double pp00[NV], const float y[MLP_OUT], int startwith, double guess[NV]) {
  int sh = mlp_sh(startwith);
  for (int i = 0; i < NV; ++i) guess[i] = pp00[i];
  guess[sh] = pp00[sh] * kmath::exp(MLP_SCALE_E * mlp_sinh((double)y[0]));
  for (int k = 1; k < 4; ++k)
    guess[sh + k] = pp00[sh + k] + MLP_SCALE_V * mlp_sinh((double)y[k]) * kmath::fmax(MLP_V_FLOOR, kmath::fabs(pp00[sh + k]));
}

#if defined(__CUDACC__)
__device__ __forceinline__ unsigned pack_bf16(float lo, float hi) {
  __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<unsigned*>(&v);
}
// D = A (16x16 bf16, row) * B (16x8 bf16, col) + C, FP32 accumulate
__device__ __forceinline__ void mma_bf16(float d[4], const unsigned a[4], const unsigned b[2]) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

// Network weights for inference: BF16 copies of W1, W2, W3 (W3 padded to 8
// rows) and FP32 biases and normalisation, as built by mlp_pack.
struct MlpDev {
  const __nv_bfloat16* w1;  // [64][16]
  const __nv_bfloat16* w2;  // [64][64]
  const __nv_bfloat16* w3;  // [8][64], rows 4..7 zero
  const float* blob;        // the FP32 blob (biases, normalisation)
};
__global__ void k_mlp_pack(const float* blob, __nv_bfloat16* w1, __nv_bfloat16* w2, __nv_bfloat16* w3) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < MLP_H * MLP_IN) w1[t] = __float2bfloat16_rn(blob[MLP_OFF_W1 + t]);
  if (t < MLP_H * MLP_H) w2[t] = __float2bfloat16_rn(blob[MLP_OFF_W2 + t]);
  if (t < 8 * MLP_H) w3[t] = __float2bfloat16_rn(t < MLP_OUT * MLP_H ? blob[MLP_OFF_W3 + t] : 0.0f);
}

// B fragment of W (row-major [out][in]) for n-tile nt and k-step kk
__device__ __forceinline__ void wfrag(const __nv_bfloat16* w, int in, int nt, int kk, int lane, unsigned b[2]) {
  int g = lane >> 2, t = lane & 3;
  const __nv_bfloat16* row = w + (long)(nt * 8 + g) * in + kk * 16 + 2 * t;
  b[0] = *reinterpret_cast<const unsigned*>(row);
  b[1] = *reinterpret_cast<const unsigned*>(row + 8);
}

// The forward pass of one warp over 32 cells. xs: the warp's standardised
// features [32][16] in shared memory (FP32); ys: [32][4] standardised outputs.
__device__ void mlp_forward_warp(const MlpDev& m, const float* xs, float* ys) {
  int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
  const float* b1 = m.blob + MLP_OFF_B1;
  const float* b2 = m.blob + MLP_OFF_B2;
  const float* b3 = m.blob + MLP_OFF_B3;
  for (int mt = 0; mt < 2; ++mt) {
    const float* x0 = xs + (mt * 16 + g) * MLP_IN;
    const float* x8 = xs + (mt * 16 + g + 8) * MLP_IN;
    unsigned a[4] = {pack_bf16(x0[2 * t], x0[2 * t + 1]), pack_bf16(x8[2 * t], x8[2 * t + 1]),
                     pack_bf16(x0[2 * t + 8], x0[2 * t + 9]), pack_bf16(x8[2 * t + 8], x8[2 * t + 9])};
    float h1[8][4];
    for (int nt = 0; nt < 8; ++nt) {
      unsigned b[2];
      wfrag(m.w1, MLP_IN, nt, 0, lane, b);
      h1[nt][0] = h1[nt][1] = h1[nt][2] = h1[nt][3] = 0.0f;
      mma_bf16(h1[nt], a, b);
      float bl = b1[nt * 8 + 2 * t], bh = b1[nt * 8 + 2 * t + 1];
      h1[nt][0] = fmaxf(h1[nt][0] + bl, 0.0f);
      h1[nt][1] = fmaxf(h1[nt][1] + bh, 0.0f);
      h1[nt][2] = fmaxf(h1[nt][2] + bl, 0.0f);
      h1[nt][3] = fmaxf(h1[nt][3] + bh, 0.0f);
    }
    float h2[8][4];
    for (int nt = 0; nt < 8; ++nt) h2[nt][0] = h2[nt][1] = h2[nt][2] = h2[nt][3] = 0.0f;
    for (int kk = 0; kk < 4; ++kk) {
      // the layer-1 accumulators of n-tiles 2kk and 2kk+1 are this k-step's A fragment
      unsigned a2[4] = {pack_bf16(h1[2 * kk][0], h1[2 * kk][1]), pack_bf16(h1[2 * kk][2], h1[2 * kk][3]),
                        pack_bf16(h1[2 * kk + 1][0], h1[2 * kk + 1][1]), pack_bf16(h1[2 * kk + 1][2], h1[2 * kk + 1][3])};
      for (int nt = 0; nt < 8; ++nt) {
        unsigned b[2];
        wfrag(m.w2, MLP_H, nt, kk, lane, b);
        mma_bf16(h2[nt], a2, b);
      }
    }
    for (int nt = 0; nt < 8; ++nt) {
      float bl = b2[nt * 8 + 2 * t], bh = b2[nt * 8 + 2 * t + 1];
      h2[nt][0] = fmaxf(h2[nt][0] + bl, 0.0f);
      h2[nt][1] = fmaxf(h2[nt][1] + bh, 0.0f);
      h2[nt][2] = fmaxf(h2[nt][2] + bl, 0.0f);
      h2[nt][3] = fmaxf(h2[nt][3] + bh, 0.0f);
    }
    float o[4] = {0.0f, 0.0f, 0.0f, 0.0f};
    for (int kk = 0; kk < 4; ++kk) {
      unsigned a3[4] = {pack_bf16(h2[2 * kk][0], h2[2 * kk][1]), pack_bf16(h2[2 * kk][2], h2[2 * kk][3]),
                        pack_bf16(h2[2 * kk + 1][0], h2[2 * kk + 1][1]), pack_bf16(h2[2 * kk + 1][2], h2[2 * kk + 1][3])};
      unsigned b[2];
      wfrag(m.w3, MLP_H, 0, kk, lane, b);
      mma_bf16(o, a3, b);
    }
    if (t < 2) {
      ys[(mt * 16 + g) * MLP_OUT + 2 * t] = o[0] + b3[2 * t];
      ys[(mt * 16 + g) * MLP_OUT + 2 * t + 1] = o[1] + b3[2 * t + 1];
      ys[(mt * 16 + g + 8) * MLP_OUT + 2 * t] = o[2] + b3[2 * t];
      ys[(mt * 16 + g + 8) * MLP_OUT + 2 * t + 1] = o[3] + b3[2 * t + 1];
    }
  }
  __syncwarp();
}

// ---- training (FP32, one minibatch per launch pair) ---------------------------
__device__ __forceinline__ float bf16r(float x) { return __bfloat162float(__float2bfloat16_rn(x)); }

// Per sample of the batch: the forward pass with BF16-rounded weights, inputs
// and hidden activations (the values inference sees), the squared error
// against the standardised target, and the back-propagated signals. Stores
// x, h1, h2, dy, dh1, dh2 for k_mlp_train_grad. Loss sum into *loss.
__global__ void __launch_bounds__(128) k_mlp_train_fwd(const float* blob, const float* X, const float* T,
                                                       const long* idx, long nb, float* act, float* loss) {
  __shared__ float w[MLP_NW];
  for (int i = threadIdx.x; i < MLP_NW; i += blockDim.x) {
    bool weight = (i >= MLP_OFF_W1 && i < MLP_OFF_B1) || (i >= MLP_OFF_W2 && i < MLP_OFF_B2) ||
                  (i >= MLP_OFF_W3 && i < MLP_OFF_B3);
    w[i] = weight ? bf16r(blob[i]) : blob[i];
  }
  __syncthreads();
  long s = (long)blockIdx.x * blockDim.x + threadIdx.x;
  float l = 0.0f;
  if (s < nb) {
    long src = idx ? idx[s] : s;
    float x[MLP_IN], h1[MLP_H], h2[MLP_H], y[MLP_OUT], dy[MLP_OUT];
    for (int k = 0; k < MLP_IN; ++k) x[k] = bf16r(X[src * MLP_IN + k]);
    for (int i = 0; i < MLP_H; ++i) {
      float a = 0.0f;
      for (int k = 0; k < MLP_IN; ++k) a += w[MLP_OFF_W1 + i * MLP_IN + k] * x[k];
      h1[i] = bf16r(fmaxf(a + w[MLP_OFF_B1 + i], 0.0f));
    }
    for (int i = 0; i < MLP_H; ++i) {
      float a = 0.0f;
      for (int k = 0; k < MLP_H; ++k) a += w[MLP_OFF_W2 + i * MLP_H + k] * h1[k];
      h2[i] = bf16r(fmaxf(a + w[MLP_OFF_B2 + i], 0.0f));
    }
    for (int o = 0; o < MLP_OUT; ++o) {
      float a = 0.0f;
      for (int k = 0; k < MLP_H; ++k) a += w[MLP_OFF_W3 + o * MLP_H + k] * h2[k];
      y[o] = a + w[MLP_OFF_B3 + o];
      float e = y[o] - T[src * MLP_OUT + o];
      l += e * e;
      dy[o] = 2.0f * e / (float)(nb * MLP_OUT);
    }
    float* r = act + s * (MLP_IN + 4 * MLP_H + MLP_OUT);
    float* dh2 = r + MLP_IN + 2 * MLP_H;
    float* dh1 = dh2 + MLP_H;
    for (int k = 0; k < MLP_IN; ++k) r[k] = x[k];
    for (int i = 0; i < MLP_H; ++i) {
      r[MLP_IN + i] = h1[i];
      r[MLP_IN + MLP_H + i] = h2[i];
    }
    for (int i = 0; i < MLP_H; ++i) {
      float a = 0.0f;
      for (int o = 0; o < MLP_OUT; ++o) a += w[MLP_OFF_W3 + o * MLP_H + i] * dy[o];
      dh2[i] = h2[i] > 0.0f ? a : 0.0f;
    }
    for (int i = 0; i < MLP_H; ++i) {
      float a = 0.0f;
      for (int k = 0; k < MLP_H; ++k) a += w[MLP_OFF_W2 + k * MLP_H + i] * dh2[k];
      dh1[i] = h1[i] > 0.0f ? a : 0.0f;
    }
    for (int o = 0; o < MLP_OUT; ++o) r[MLP_IN + 4 * MLP_H + o] = dy[o];
  }
  for (int o = 16; o > 0; o >>= 1) l += __shfl_down_sync(0xffffffffu, l, o);
  if ((threadIdx.x & 31) == 0) atomicAdd(loss, l);
}
// One thread per weight or bias entry: its gradient summed over the batch in
// sample order (deterministic).
__global__ void __launch_bounds__(128) k_mlp_train_grad(const float* act, long nb, float* grad) {
  int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e < MLP_OFF_W1 || e >= MLP_NW) return;
  const int stride = MLP_IN + 4 * MLP_H + MLP_OUT;
  const int X0 = 0, H1 = MLP_IN, H2 = MLP_IN + MLP_H, DH2 = MLP_IN + 2 * MLP_H, DH1 = DH2 + MLP_H,
            DY = MLP_IN + 4 * MLP_H;
  int a, b;  // grad = sum_s act[a] * (b >= 0 ? act[b] : 1)
  if (e < MLP_OFF_B1) {
    int i = (e - MLP_OFF_W1) / MLP_IN, k = (e - MLP_OFF_W1) % MLP_IN;
    a = DH1 + i;
    b = X0 + k;
  } else if (e < MLP_OFF_W2) {
    a = DH1 + (e - MLP_OFF_B1);
    b = -1;
  } else if (e < MLP_OFF_B2) {
    int i = (e - MLP_OFF_W2) / MLP_H, k = (e - MLP_OFF_W2) % MLP_H;
    a = DH2 + i;
    b = H1 + k;
  } else if (e < MLP_OFF_W3) {
    a = DH2 + (e - MLP_OFF_B2);
    b = -1;
  } else if (e < MLP_OFF_B3) {
    int o = (e - MLP_OFF_W3) / MLP_H, k = (e - MLP_OFF_W3) % MLP_H;
    a = DY + o;
    b = H2 + k;
  } else {
    a = DY + (e - MLP_OFF_B3);
    b = -1;
  }
  float g = 0.0f;
  for (long s = 0; s < nb; ++s) {
    const float* r = act + s * stride;
    g += r[a] * (b >= 0 ? r[b] : 1.0f);
  }
  grad[e] = g;
}
// Adam (beta1 0.9, beta2 0.999, eps 1e-8) on the weight and bias entries
__global__ void k_mlp_adam(float* blob, const float* grad, float* m1, float* m2, float lr, float bc1, float bc2) {
  int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e < MLP_OFF_W1 || e >= MLP_NW) return;
  float g = grad[e];
  m1[e] = 0.9f * m1[e] + 0.1f * g;
  m2[e] = 0.999f * m2[e] + 0.001f * g * g;
  blob[e] -= lr * (m1[e] / bc1) / (sqrtf(m2[e] / bc2) + 1.0e-8f);
}
#endif

}  // namespace kc
