// kks_pointwise.cuh - FP64 pointwise formulas shared by the field kernels of
// the cuFFT step (kks_fields.cu) and the fused FP64 passes (kks_fft64.cu).
#pragma once

#include <math.h>

#include "kks_internal.cuh"

namespace kks_pw {

// Free energy of one point: G_s, G_eta_s, h'(c_a - c_t) and df_alpha/dc
// (pf_kks/free_energy.py:21-71). FP64: the reference's operation order.
struct FreeEnergy {
  double G, G_eta, G_flux, mu;
};

__device__ __forceinline__ FreeEnergy free_energy(double ca, double ct, double eta, const KksPar& q) {
  FreeEnergy r;
  const double fa_s = q.A_alp_s * (ca * ca) + q.B_alp_s * ca + q.C_alp_s;
  const double fa_ca_s = 2 * q.A_alp_s * ca + q.B_alp_s;
  const double ft_s = q.A_thet_s * (ct * ct) + q.B_thet_s * ct + q.C_thet_s;
  const double e2 = eta * eta, e3 = e2 * eta;
  const double h = 3.0 * e2 - 2 * e3;
  const double h_eta = 6.0 * eta - 6 * e2;
  const double g = e2 - 2 * e3 + e2 * e2;
  const double g_eta = 2.0 * eta - 6.0 * e2 + 4.0 * e3;
  r.G = (1 - h) * fa_s + h * ft_s + q.w_s * g;
  r.G_eta = -h_eta * (fa_s - ft_s - (ca - ct) * fa_ca_s) + q.w_s * g_eta;
  r.G_flux = h_eta * (ca - ct);
  r.mu = fa_ca_s;
  return r;
}

// Elastic strain multipliers 0.5((N k)_h k_k + (N k)_k k_h), N = inverse of
// the 2x2 acoustic tensor of the stiffness normalised by C44(T0); 0 at k = 0
// (pf_kks/elasticity.py:60-94 with k_z = 0).
template <typename T>
__device__ __forceinline__ void strain_multipliers(T kx, T ky, T c11, T c12, T& oxx, T& oyy, T& oxy) {
  const T Kxx = c11 * kx * kx + ky * ky;
  const T Kyy = kx * kx + c11 * ky * ky;
  const T Kxy = (c12 + T(1)) * kx * ky;
  const T det = Kxx * Kyy - Kxy * Kxy;
  if (det == T(0)) {
    oxx = oyy = oxy = T(0);
    return;
  }
  const T inv = T(1) / det;
  const T Nxx = Kyy * inv, Nyy = Kxx * inv, Nxy = -Kxy * inv;
  const T Nkx = Nxx * kx + Nxy * ky;
  const T Nky = Nxy * kx + Nyy * ky;
  oxx = Nkx * kx;
  oyy = Nky * ky;
  oxy = T(0.5) * (Nky * kx + Nkx * ky);
}

// Closed-form phase compositions with the reference's non-finite guards.
__device__ __forceinline__ void phase_comp(double Xo, double eb, const KksPar& q, double& xal, double& xth) {
  const double h = 3.0 * (eb * eb) - 2 * (eb * eb * eb);
  xal = (Xo - h * q.pc_shift) / ((1 - h) + h * q.pc_ratio);
  if (isinf(xal)) xal = xal > 0 ? 1e-6 : -1e-6;
  if (isnan(xal)) xal = 1e-6;
  xth = q.pc_ratio * xal + q.pc_shift;
  if (isinf(xth)) xth = xth > 0 ? 1e-6 : -1e-6;
  if (isnan(xth)) xth = 1e-6;
}

}  // namespace kks_pw
