// kc_mixed.cuh — the FP32 pieces of the mixed-precision step form: the PPM
// face reconstruction (koral/fv/recon.zig:107, C finite.c:210, non-uniform
// widths) on stencil deviations, the LAXF dissipation (koral/fv/laxf.zig:13)
// and the flux-CT corner averages (koral/sim/ct.zig:38) in single precision;
// KC_MIXED takes the LAXF and CT pieces (the reconstruction is a piece of its
// own: it moves the floor-level accretion rate by 9e-3 over 1000 steps).
// Everything else — floors, the one-sided fluxes with their metric
// contractions, p2u, u2p, the implicit solve and the metric cache — stays
// FP64. The FP64 form does not use this file.
#pragma once
#include "kc_dev.cuh"

namespace kc {

struct FacesF {
  float left, right;
};

__device__ __forceinline__ float sign_pm_f(float x) { return (x >= 0.0f) ? 1.0f : -1.0f; }

// PPM with non-uniform widths in FP32, the formula of kp::recon_ppm
__device__ __forceinline__ FacesF recon_ppm_f(const float u[5], const float dx[5]) {
  float dxm2 = dx[0], dxm1 = dx[1], dx0 = dx[2], dxp1 = dx[3], dxp2 = dx[4];
  float dxp2_plus_dxp1_inv = 1.0f / (dxp2 + dxp1);
  float dxp1_plus_dx0 = dxp1 + dx0;
  float dxp1_plus_dx0_inv = 1.0f / dxp1_plus_dx0;
  float dx0_plus_dxm1 = dx0 + dxm1;
  float dx0_plus_dxm1_inv = 1.0f / dx0_plus_dxm1;
  float dxm1_plus_dxm2 = dxm1 + dxm2;
  float dxm1_plus_dxm2_inv = 1.0f / dxm1_plus_dxm2;
  float dxm1_plus_dx0_plus_dxp1_inv = 1.0f / (dxm1 + dx0 + dxp1);
  float dx0_plus_dxp1_plus_dxp2_inv = 1.0f / (dx0 + dxp1 + dxp2);
  float dxm2_plus_dxm1_plus_dx0_inv = 1.0f / (dxm2 + dxm1 + dx0);
  float dx0_plus_twodxm1 = dx0 + 2.0f * dxm1;
  float dxp1_plus_twodx0 = dxp1 + 2.0f * dx0;
  float dxm1_plus_twodxm2 = dxm1 + 2.0f * dxm2;
  float twodxp1_plus_dx0 = 2.0f * dxp1 + dx0;
  float twodxp2_plus_dxp1 = 2.0f * dxp2 + dxp1;
  float twodx0_plus_dxm1 = 2.0f * dx0 + dxm1;

  float dri = dx0 * dxm1_plus_dx0_plus_dxp1_inv *
              (dx0_plus_twodxm1 * dxp1_plus_dx0_inv * (u[3] - u[2]) + twodxp1_plus_dx0 * dx0_plus_dxm1_inv * (u[2] - u[1]));
  float drip1 = dxp1 * dx0_plus_dxp1_plus_dxp2_inv *
                (dxp1_plus_twodx0 * dxp2_plus_dxp1_inv * (u[4] - u[3]) + twodxp2_plus_dxp1 * dxp1_plus_dx0_inv * (u[3] - u[2]));
  float drim1 = dxm1 * dxm2_plus_dxm1_plus_dx0_inv *
                (dxm1_plus_twodxm2 * dx0_plus_dxm1_inv * (u[2] - u[1]) + twodx0_plus_dxm1 * dxm1_plus_dxm2_inv * (u[1] - u[0]));
  dri = ((u[3] - u[2]) * (u[2] - u[1]) > 0.0f)
            ? fminf(fabsf(dri), fminf(2.0f * fabsf(u[2] - u[1]), 2.0f * fabsf(u[2] - u[3]))) * sign_pm_f(dri)
            : 0.0f;
  drip1 = ((u[4] - u[3]) * (u[3] - u[2]) > 0.0f)
              ? fminf(fabsf(drip1), fminf(2.0f * fabsf(u[3] - u[2]), 2.0f * fabsf(u[3] - u[4]))) * sign_pm_f(drip1)
              : 0.0f;
  drim1 = ((u[2] - u[1]) * (u[1] - u[0]) > 0.0f)
              ? fminf(fabsf(drim1), fminf(2.0f * fabsf(u[1] - u[0]), 2.0f * fabsf(u[1] - u[2]))) * sign_pm_f(drim1)
              : 0.0f;

  float z1 = dx0_plus_dxm1 / dxp1_plus_twodx0;
  float z2 = (dxp2 + dxp1) / twodxp1_plus_dx0;
  float dx_inv = 1.0f / (dxm1 + dx0 + dxp1 + dxp2);
  float right = u[2] + dx0 * dxp1_plus_dx0_inv * (u[3] - u[2]) +
                dx_inv * ((2.0f * dxp1 * dx0) * dxp1_plus_dx0_inv * (z1 - z2) * (u[3] - u[2]) - dx0 * z1 * drip1 +
                          dxp1 * z2 * dri);
  z1 = dxm1_plus_dxm2 / dx0_plus_twodxm1;
  z2 = dxp1_plus_dx0 / twodx0_plus_dxm1;
  dx_inv = 1.0f / (dxm2 + dxm1 + dx0 + dxp1);
  float left = u[1] + dxm1 * dx0_plus_dxm1_inv * (u[2] - u[1]) +
               dx_inv * ((2.0f * dx0 * dxm1) * dx0_plus_dxm1_inv * (z1 - z2) * (u[2] - u[1]) - dxm1 * z1 * dri +
                         dx0 * z2 * drim1);
  if ((right - u[2]) * (u[2] - left) <= 0.0f) {
    left = u[2];
    right = u[2];
  }
  if ((right - left) * (left - (3.0f * u[2] - 2.0f * right)) < 0.0f) left = 3.0f * u[2] - 2.0f * right;
  if ((right - left) * ((3.0f * u[2] - 2.0f * left) - right) < 0.0f) right = 3.0f * u[2] - 2.0f * left;
  FacesF f;
  f.left = left;
  f.right = right;
  return f;
}

// PPM of a 5-cell stencil on its deviations from the centre value: the
// differences are taken in FP64 and the PPM arithmetic runs in FP32 on them.
// PPM is translation-invariant (differences, linear combinations and
// comparisons of differences), so the FP32 rounding is relative to the local
// variation, not to the value itself; a near-hydrostatic torus, whose flux
// divergence is a tiny fraction of the fluxes, stays balanced.
__device__ __forceinline__ Faces recon_ppm_mixed(const double v[5], const double dx[5]) {
  float d[5], dxf[5];
  for (int k = 0; k < 5; ++k) {
    d[k] = (float)(v[k] - v[2]);
    dxf[k] = (float)dx[k];
  }
  FacesF f = recon_ppm_f(d, dxf);
  Faces o;
  o.left = v[2] + (double)f.left;
  o.right = v[2] + (double)f.right;
  return o;
}

// F* = (F_R + F_L)/2 - a (U_R - U_L)/2: the averages and the conserved jump in
// FP64 (their cancellation is the flux divergence), the dissipation product in FP32
__device__ __forceinline__ double laxf_f(double fl, double fr, double ul, double ur, double ag) {
  double jump = ur - ul;
  return 0.5 * (fr + fl) - (double)(0.5f * (float)ag * (float)jump);
}

}  // namespace kc
