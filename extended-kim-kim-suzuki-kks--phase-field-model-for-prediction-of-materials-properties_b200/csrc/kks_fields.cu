// kks_fields.cu - field kernels of one attempt of the semi-implicit KKS step.
//
// An attempt (pf_kks/solver.py:178-276) is, on the device:
//
//   square          eta -> eta^2                                  (R2C batch input)
//   [cuFFT R2C x3]  FT(eta), FT(X), FT(eta^2)
//   spectral_mid    Khachaturyan strain spectra eps_xx, eps_yy, eps_xy from
//                   FT(eta^2) (pf_kks/elasticity.py:107-163, closed 2-D form)
//                   and i k_a FT(eta) (pf_kks/solver.py:258-262)
//   [cuFFT C2R x5]
//   pre_pointwise   free_energy_terms of the old state (pf_kks/free_energy.py:21-71),
//                   elastic energy and its eta derivative, Allen-Cahn drive and
//                   Cahn-Hilliard fluxes; sums for the energy and histories
//   [cuFFT R2C x3]
//   spectral_update semi-implicit Allen-Cahn and Cahn-Hilliard divisions
//                   (pf_kks/solver.py:249-264)
//   [cuFFT C2R x2]  -> candidate eta_b, X_b written into the other state buffer
//   post_pointwise  phase_compositions (pf_kks/free_energy.py:74-95), new free
//                   energy and diffusion potential, np.gradient energy term,
//                   residual field sums (pf_kks/residual.py:48-66), histories
//   restore         only after a rejection: keep the rejected pair entry and
//                   copy the step's input back into the candidate buffer
//
// Each kernel is one coalesced pass over its arrays (HBM-bound: no stage is a
// dense contraction). Reductions are per-block partial sums in FP64, finished
// in a fixed order by the decide kernel, so results are deterministic.

#include <math.h>

#include "kks_internal.cuh"

namespace {

template <typename R>
struct Cplx;
template <>
struct Cplx<double> {
  using T = double2;
};
template <>
struct Cplx<float> {
  using T = float2;
};

constexpr int kThreads = 256;

// Reduce NV per-thread values over the block; thread 0 writes them to out[0..NV).
template <int NV>
__device__ __forceinline__ void block_reduce_store(double (&v)[NV], double* out) {
  __shared__ double sh[NV][kThreads / 32];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < NV; ++k) {
    double x = v[k];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
    if (lane == 0) sh[k][wid] = x;
  }
  __syncthreads();
  if (wid == 0) {
#pragma unroll
    for (int k = 0; k < NV; ++k) {
      double x = lane < kThreads / 32 ? sh[k][lane] : 0.0;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
      if (lane == 0) out[k] = x;
    }
  }
}

__device__ __forceinline__ bool in_iface(double e) { return e >= 0.1 && e <= 0.9; }

// ---------------------------------------------------------------------------
// Free energy of one point: G_s, G_eta_s, h'(c_a - c_t) and df_alpha/dc
// (pf_kks/free_energy.py:21-71). FP64: the reference's operation order.
// FP32: the two parabolas in vertex form A (c - v)^2 + f0 with v, f0 from the
// FP64 prologue, which avoids the cancellation of A c^2 + B c + C near the
// vertex (the precipitate parabola has its vertex at c ~ 1).
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

struct FreeEnergyF {
  float G, G_eta, G_flux, mu;
};

__device__ __forceinline__ FreeEnergyF free_energy(float ca, float ct, float eta, float A_a, float va, float fa0,
                                                   float A_t, float vt, float ft0, float w_s) {
  FreeEnergyF r;
  const float da = ca - va, dt_ = ct - vt;
  const float fa_s = A_a * da * da + fa0;
  const float fa_ca_s = 2.0f * A_a * da;
  const float ft_s = A_t * dt_ * dt_ + ft0;
  const float e2 = eta * eta, e3 = e2 * eta;
  const float h = 3.0f * e2 - 2.0f * e3;
  const float h_eta = 6.0f * eta - 6.0f * e2;
  const float g = e2 - 2.0f * e3 + e2 * e2;
  const float g_eta = 2.0f * eta - 6.0f * e2 + 4.0f * e3;
  r.G = (1.0f - h) * fa_s + h * ft_s + w_s * g;
  r.G_eta = -h_eta * (fa_s - ft_s - (ca - ct) * fa_ca_s) + w_s * g_eta;
  r.G_flux = h_eta * (ca - ct);
  r.mu = fa_ca_s;
  return r;
}

// ---------------------------------------------------------------------------
template <typename R>
__global__ void __launch_bounds__(kThreads) k_square(const KksPar* __restrict__ par, R* __restrict__ state, int N,
                                                     int Np) {
  if (!par->active) return;
  const R* eta = state;
  R* eta2 = state + 2 * (size_t)Np;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
    const R e = eta[i];
    eta2[i] = e * e;
  }
}

// Elastic strain multipliers 0.5((N k)_h k_k + (N k)_k k_h), N = inverse of
// the 2x2 acoustic tensor of the stiffness normalised by C44(T0); 0 at k = 0.
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

template <typename R>
__global__ void __launch_bounds__(kThreads)
    k_spectral_mid(const KksConst* __restrict__ c, const KksPar* __restrict__ par,
                   const typename Cplx<R>::T* __restrict__ spec_a, typename Cplx<R>::T* __restrict__ spec_b,
                   const double* __restrict__ kxs, const double* __restrict__ kys) {
  using C = typename Cplx<R>::T;
  if (!par->active) return;
  const int NC = c->NC, NCp = c->NCp, nyh = c->nyh;
  const R inv_N = (R)c->inv_N;
  const R a = (R)(par->epsX * c->c3) * inv_N;
  const R c11 = (R)c->c11, c12 = (R)c->c12;
  const C* eta_h = spec_a;
  const C* eta2_h = spec_a + 2 * (size_t)NCp;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < NC; k += gridDim.x * blockDim.x) {
    const int ix = k / nyh;
    const int iy = k - ix * nyh;
    const R kx = (R)kxs[ix], ky = (R)kys[iy];
    R oxx, oyy, oxy;
    strain_multipliers<R>(kx, ky, c11, c12, oxx, oyy, oxy);
    const C e2 = eta2_h[k];
    const C eh = eta_h[k];
    const R sx = a * oxx, sy = a * oyy, sxy = a * oxy;
    C o;
    o.x = sx * e2.x; o.y = sx * e2.y;
    spec_b[k] = o;
    o.x = sy * e2.x; o.y = sy * e2.y;
    spec_b[NCp + k] = o;
    o.x = sxy * e2.x; o.y = sxy * e2.y;
    spec_b[2 * (size_t)NCp + k] = o;
    const R kxn = kx * inv_N, kyn = ky * inv_N;
    o.x = -kxn * eh.y; o.y = kxn * eh.x;
    spec_b[3 * (size_t)NCp + k] = o;
    o.x = -kyn * eh.y; o.y = kyn * eh.x;
    spec_b[4 * (size_t)NCp + k] = o;
  }
}

// ---------------------------------------------------------------------------
// Old-state pointwise pass (FP64 path).
__global__ void __launch_bounds__(kThreads)
    k_pre_pointwise_f64(const KksConst* __restrict__ c, const KksPar* __restrict__ par,
                        const double* __restrict__ state, const double* __restrict__ real_b,
                        double* __restrict__ real_c, double* g0, double* g1, double* g2,
                        double* __restrict__ partials) {
  if (!par->active) return;
  const KksPar q = *par;
  const int N = c->N, Np = c->Np, nx = c->nx, ny = c->ny;
  const double* eta = state;
  const double* X = state + Np;
  const double* Xal = state + 3 * (size_t)Np;
  const double* Xth = state + 4 * (size_t)Np;
  const double* exx_a = real_b;
  const double* eyy_a = real_b + Np;
  const double* exy_a = real_b + 2 * (size_t)Np;
  const double* gx_a = real_b + 3 * (size_t)Np;
  const double* gy_a = real_b + 4 * (size_t)Np;
  double* drive = real_c;
  double* fx = real_c + Np;
  double* fy = real_c + 2 * (size_t)Np;
  double* gs_buf = q.gs == 0 ? g0 : (q.gs == 1 ? g1 : g2);
  const double C11 = c->C11_0, C12 = c->C12_0, C44_0 = c->C44_0;
  const double c3u = C11 + 2 * C12;
  const double epsX = q.epsX, C44 = q.C44;
  double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
    const double e = eta[i];
    const double x = X[i];
    const FreeEnergy f = free_energy(Xal[i], Xth[i], e, q);
    // elastic energy density and its eta derivative (frozen stiffness, current epsX)
    const double exx = exx_a[i], eyy = eyy_a[i], exy = exy_a[i];
    const double a = epsX * (e * e);
    const double e_xx = exx - a, e_yy = eyy - a, e_zz = -a;
    const double s_xx = C11 * e_xx + C12 * (e_yy + e_zz);
    const double s_yy = C11 * e_yy + C12 * (e_xx + e_zz);
    const double s_zz = C11 * e_zz + C12 * (e_xx + e_yy);
    const double s_xy = 2 * C44_0 * exy;
    const double el = 0.5 * (s_xx * e_xx + s_yy * e_yy + s_zz * e_zz + 2 * s_xy * exy);
    const double el_eta = 2 * epsX * e * c3u * (3 * epsX * (e * e) - (exx + eyy));
    const double el_s = el / C44;
    drive[i] = f.G_eta + el_eta / C44;
    fx[i] = f.G_flux * gx_a[i];
    fy[i] = f.G_flux * gy_a[i];
    if (q.armed_write) gs_buf[i] = f.G;
    acc[0] += f.G;
    acc[1] += f.G + el_s;
    acc[2] += e;
    if (e < 0.05) { acc[3] += x; acc[4] += 1.0; }
    if (e > 0.95) { acc[5] += x; acc[6] += 1.0; }
    if (q.surface) {
      const int ix = i / ny, iy = i - ix * ny;
      if (ix < nx - 1 && iy < ny - 1 && in_iface(e) && in_iface(eta[i + ny]) && in_iface(eta[i + ny + 1]) &&
          in_iface(eta[i + 1]))
        acc[7] += 1.0;
    }
  }
  block_reduce_store<8>(acc, partials + (size_t)blockIdx.x * KKS_NPART + P3_G);
}

// Old-state pointwise pass (mixed path: FP32 fields, FP64 sums).
__global__ void __launch_bounds__(kThreads)
    k_pre_pointwise_f32(const KksConst* __restrict__ c, const KksPar* __restrict__ par,
                        const float* __restrict__ state, const float* __restrict__ real_b, float* __restrict__ real_c,
                        float* g0, float* g1, float* g2, double* __restrict__ partials) {
  if (!par->active) return;
  const KksPar q = *par;
  const int N = c->N, Np = c->Np, nx = c->nx, ny = c->ny;
  const float* eta = state;
  const float* X = state + Np;
  const float* Xal = state + 3 * (size_t)Np;
  const float* Xth = state + 4 * (size_t)Np;
  const float* exx_a = real_b;
  const float* eyy_a = real_b + Np;
  const float* exy_a = real_b + 2 * (size_t)Np;
  const float* gx_a = real_b + 3 * (size_t)Np;
  const float* gy_a = real_b + 4 * (size_t)Np;
  float* drive = real_c;
  float* fx = real_c + Np;
  float* fy = real_c + 2 * (size_t)Np;
  float* gs_buf = q.gs == 0 ? g0 : (q.gs == 1 ? g1 : g2);
  // stiffness normalised by C44(T): el_s and el_eta_s directly in units of C44
  const float c11 = (float)(c->C11_0 * q.inv_C44), c12 = (float)(c->C12_0 * q.inv_C44);
  const float c44 = (float)(c->C44_0 * q.inv_C44);
  const float c3 = (float)((c->C11_0 + 2 * c->C12_0) * q.inv_C44);
  const float epsX = (float)q.epsX;
  const float A_a = (float)q.A_alp_s, va = (float)q.va, fa0 = (float)q.fa0;
  const float A_t = (float)q.A_thet_s, vt = (float)q.vt, ft0 = (float)q.ft0, w_s = (float)q.w_s;
  const double x_mean = q.x_mean;
  double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
    const float e = eta[i];
    const FreeEnergyF f = free_energy(Xal[i], Xth[i], e, A_a, va, fa0, A_t, vt, ft0, w_s);
    const float exx = exx_a[i], eyy = eyy_a[i], exy = exy_a[i];
    const float a = epsX * (e * e);
    const float e_xx = exx - a, e_yy = eyy - a, e_zz = -a;
    const float s_xx = c11 * e_xx + c12 * (e_yy + e_zz);
    const float s_yy = c11 * e_yy + c12 * (e_xx + e_zz);
    const float s_zz = c11 * e_zz + c12 * (e_xx + e_yy);
    const float s_xy = 2.0f * c44 * exy;
    const float el_s = 0.5f * (s_xx * e_xx + s_yy * e_yy + s_zz * e_zz + 2.0f * s_xy * exy);
    const float el_eta_s = 2.0f * epsX * e * c3 * (3.0f * epsX * (e * e) - (exx + eyy));
    drive[i] = f.G_eta + el_eta_s;
    fx[i] = f.G_flux * gx_a[i];
    fy[i] = f.G_flux * gy_a[i];
    if (q.armed_write) gs_buf[i] = f.G;
    const double ed = (double)e;
    const double xd = (double)X[i] + x_mean;
    acc[0] += (double)f.G;
    acc[1] += (double)f.G + (double)el_s;
    acc[2] += ed;
    if (ed < 0.05) { acc[3] += xd; acc[4] += 1.0; }
    if (ed > 0.95) { acc[5] += xd; acc[6] += 1.0; }
    if (q.surface) {
      const int ix = i / ny, iy = i - ix * ny;
      if (ix < nx - 1 && iy < ny - 1 && in_iface(ed) && in_iface((double)eta[i + ny]) &&
          in_iface((double)eta[i + ny + 1]) && in_iface((double)eta[i + 1]))
        acc[7] += 1.0;
    }
  }
  block_reduce_store<8>(acc, partials + (size_t)blockIdx.x * KKS_NPART + P3_G);
}

// ---------------------------------------------------------------------------
template <typename R>
__global__ void __launch_bounds__(kThreads)
    k_spectral_update(const KksConst* __restrict__ c, const KksPar* __restrict__ par,
                      const typename Cplx<R>::T* __restrict__ spec_a, typename Cplx<R>::T* __restrict__ spec_bcd,
                      const double* __restrict__ kxs, const double* __restrict__ kys) {
  using C = typename Cplx<R>::T;
  if (!par->active) return;
  const int NC = c->NC, NCp = c->NCp, nyh = c->nyh;
  const R inv_N = (R)c->inv_N;
  const R ac_mul = (R)par->ac_mul, ac_den = (R)par->ac_den, ch_mul = (R)par->ch_mul;
  const R dt = (R)par->dt, D_s = (R)par->D_s;
  const int zero_dc = c->zero_dc;
  const C* eta_h = spec_a;
  const C* X_h = spec_a + NCp;
  const C* D_h = spec_bcd;
  const C* Fx_h = spec_bcd + NCp;
  const C* Fy_h = spec_bcd + 2 * (size_t)NCp;
  C* eta_b = spec_bcd + 3 * (size_t)NCp;
  C* X_b = spec_bcd + 4 * (size_t)NCp;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < NC; k += gridDim.x * blockDim.x) {
    const int ix = k / nyh;
    const int iy = k - ix * nyh;
    const R kx = (R)kxs[ix], ky = (R)kys[iy];
    const R k2 = kx * kx + ky * ky;
    const C eh = eta_h[k], dh = D_h[k], xh = X_h[k], fxh = Fx_h[k], fyh = Fy_h[k];
    // Allen-Cahn: (eta^ - dt L FT(drive)) / (1 + dt L kappa^2 k^2)
    const R den_e = R(1) + ac_den * k2;
    C o;
    o.x = (ac_mul * dh.x + eh.x) / den_e * inv_N;
    o.y = (ac_mul * dh.y + eh.y) / den_e * inv_N;
    eta_b[k] = o;
    // Cahn-Hilliard: (X^ + dt D sum_a i k_a FT(flux_a)) / (1 + dt k^2 D)
    const R flx = -(kx * fxh.y) - ky * fyh.y;
    const R fly = kx * fxh.x + ky * fyh.x;
    const R den_x = R(1) + dt * k2 * D_s;
    o.x = (ch_mul * flx + xh.x) / den_x * inv_N;
    o.y = (ch_mul * fly + xh.y) / den_x * inv_N;
    if (zero_dc && k == 0) o.x = o.y = R(0);
    X_b[k] = o;
  }
}

// ---------------------------------------------------------------------------
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

// np.gradient of eta along x (rows) and y (columns): central differences
// inside, one-sided differences on the two edges (non-periodic).
template <typename R>
__device__ __forceinline__ void np_gradient(const R* e, int i, int ix, int iy, int nx, int ny, double& gx,
                                            double& gy) {
  if (ix == 0) gx = (double)e[i + ny] - (double)e[i];
  else if (ix == nx - 1) gx = (double)e[i] - (double)e[i - ny];
  else gx = ((double)e[i + ny] - (double)e[i - ny]) / 2.0;
  if (iy == 0) gy = (double)e[i + 1] - (double)e[i];
  else if (iy == ny - 1) gy = (double)e[i] - (double)e[i - 1];
  else gy = ((double)e[i + 1] - (double)e[i - 1]) / 2.0;
}

template <typename R>
__global__ void __launch_bounds__(kThreads)
    k_post_pointwise(const KksConst* __restrict__ c, const KksPar* __restrict__ par, const R* __restrict__ state_in,
                     R* __restrict__ state_out, const R* __restrict__ eta_m, const R* __restrict__ X_m,
                     R* __restrict__ mu, R* g0, R* g1, R* g2, double* __restrict__ partials) {
  if (!par->active) return;
  const KksPar q = *par;
  const int N = c->N, Np = c->Np, nx = c->nx, ny = c->ny;
  const R* eta_b = state_out;
  const R* X_b = state_out + Np;
  R* Xal_b = state_out + 3 * (size_t)Np;
  R* Xth_b = state_out + 4 * (size_t)Np;
  const R* eta_o = state_in;
  const R* X_o = state_in + Np;
  R* gb_buf = q.gb == 0 ? g0 : (q.gb == 1 ? g1 : g2);
  const R* gm_buf = q.gm == 0 ? g0 : (q.gm == 1 ? g1 : g2);
  const R* eta_minus = q.minus_is_state ? eta_o : eta_m;
  const R* X_minus = q.minus_is_state ? X_o : X_m;
  const double x_mean = q.x_mean;
  const double dt = q.dt;
  double acc[11] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
    const int ix = i / ny, iy = i - ix * ny;
    const double eb = (double)eta_b[i];
    const double xb = (double)X_b[i] + x_mean;
    const double xo = (double)X_o[i] + x_mean;
    double xal, xth;
    phase_comp(xo, eb, q, xal, xth);
    Xal_b[i] = (R)xal;
    Xth_b[i] = (R)xth;
    double G_b, mu_b;
    if (sizeof(R) == 8) {
      const FreeEnergy f = free_energy(xal, xth, eb, q);
      G_b = f.G;
      mu_b = f.mu;
    } else {
      const FreeEnergyF f = free_energy((float)xal, (float)xth, (float)eb, (float)q.A_alp_s, (float)q.va,
                                        (float)q.fa0, (float)q.A_thet_s, (float)q.vt, (float)q.ft0, (float)q.w_s);
      G_b = f.G;
      mu_b = f.mu;
    }
    double gx, gy;
    np_gradient<R>(eta_b, i, ix, iy, nx, ny, gx, gy);
    acc[0] += gx * gx + gy * gy;
    if (eb < 0.05) { acc[1] += xb; acc[2] += 1.0; }
    if (eb > 0.95) { acc[3] += xb; acc[4] += 1.0; }
    acc[5] += eb;
    if (q.surface && ix < nx - 1 && iy < ny - 1 && in_iface(eb) && in_iface((double)eta_b[i + ny]) &&
        in_iface((double)eta_b[i + ny + 1]) && in_iface((double)eta_b[i + 1]))
      acc[6] += 1.0;
    if (q.armed_write) {
      if (q.armed_residual) {
        const double mum = (double)mu[i];
        const double em = (double)eta_minus[i];
        double dX;
        if (sizeof(R) == 8) dX = xb - ((double)X_minus[i] + x_mean);
        else dX = (double)X_b[i] - (double)X_minus[i];
        const double dXdt = dX / dt;
        const double mu_mean = (mu_b + mum) / 2;
        const double diffusion = dXdt * mu_mean;
        const double detadt = (eb - em) / dt;
        const double allen_cahn = q.inv_Ls * (detadt * detadt);
        const double temperature = (G_b - (double)gm_buf[i]) / dt;
        acc[7] += diffusion;
        acc[8] += allen_cahn;
        acc[9] += temperature;
        acc[10] += -1 * diffusion + allen_cahn - temperature;
      }
      mu[i] = (R)mu_b;
      gb_buf[i] = (R)G_b;
    }
  }
  block_reduce_store<11>(acc, partials + (size_t)blockIdx.x * KKS_NPART + P5_GRAD2);
}

// After a rejection: the rejected candidate becomes the pair's minus entry and
// the step's input is copied back into the candidate buffer.
template <typename R>
__global__ void __launch_bounds__(kThreads)
    k_restore(const KksConst* __restrict__ c, const KksCtl* __restrict__ ctl, const R* __restrict__ state_in,
              R* __restrict__ state_out, R* __restrict__ eta_m, R* __restrict__ X_m) {
  if (!ctl->restore || ctl->status != KKS_STATUS_OK) return;
  const int N = c->N, Np = c->Np;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
    eta_m[i] = state_out[i];
    X_m[i] = state_out[Np + i];
    state_out[i] = state_in[i];
    state_out[Np + i] = state_in[Np + i];
    state_out[3 * (size_t)Np + i] = state_in[3 * (size_t)Np + i];
    state_out[4 * (size_t)Np + i] = state_in[4 * (size_t)Np + i];
  }
}

// Stress and elastic strain returned by solve_elasticity (components xx, yy, zz, xy).
template <typename R>
__global__ void __launch_bounds__(kThreads)
    k_elastic_out(const KksConst* __restrict__ c, const KksPar* __restrict__ par, const R* __restrict__ eta,
                  const R* __restrict__ real_b, double* __restrict__ sig4, double* __restrict__ eps4) {
  const int N = c->N, Np = c->Np;
  const double C11 = c->C11_0, C12 = c->C12_0, C44_0 = c->C44_0, epsX = par->epsX;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
    const double e = (double)eta[i];
    const double exx = (double)real_b[i], eyy = (double)real_b[Np + i], exy = (double)real_b[2 * (size_t)Np + i];
    const double a = epsX * (e * e);
    const double e_xx = exx - a, e_yy = eyy - a, e_zz = -a;
    sig4[i] = C11 * e_xx + C12 * (e_yy + e_zz);
    sig4[N + i] = C11 * e_yy + C12 * (e_xx + e_zz);
    sig4[2 * (size_t)N + i] = C11 * e_zz + C12 * (e_xx + e_yy);
    sig4[3 * (size_t)N + i] = 2 * C44_0 * exy;
    eps4[i] = e_xx;
    eps4[N + i] = e_yy;
    eps4[2 * (size_t)N + i] = e_zz;
    eps4[3 * (size_t)N + i] = exy;
  }
}

template <typename R>
__global__ void k_to_real(const double* __restrict__ src, R* __restrict__ dst, int n, double shift) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) dst[i] = (R)(src[i] - shift);
}

template <typename R>
__global__ void k_to_double(const R* __restrict__ src, double* __restrict__ dst, int n, double shift) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    dst[i] = (double)src[i] + shift;
}

int grid_for(int n, int cap) {
  int g = (n + kThreads - 1) / kThreads;
  return g < cap ? (g > 0 ? g : 1) : cap;
}

}  // namespace

int kks_field_blocks(int N, int num_sms) { return grid_for(N, num_sms * 4); }

template <typename R>
void kks_launch_square(const KksConst* hc, const KksPar* par, R* state, int nblocks, cudaStream_t s) {
  k_square<R><<<nblocks, kThreads, 0, s>>>(par, state, hc->N, hc->Np);
}

template <typename R>
void kks_launch_spectral_mid(const KksConst* hc, const KksConst* dc, const KksPar* par, const KksFieldPtrs& f,
                             cudaStream_t s) {
  using C = typename Cplx<R>::T;
  const int g = grid_for(hc->NC, 148 * 8);
  k_spectral_mid<R><<<g, kThreads, 0, s>>>(dc, par, (const C*)f.spec_a, (C*)f.spec_bcd, f.kx, f.ky);
}

template <>
void kks_launch_pre_pointwise<double>(const KksConst* hc, const KksConst* dc, const KksPar* par,
                                      const KksFieldPtrs& f, int parity, int nblocks, cudaStream_t s) {
  k_pre_pointwise_f64<<<nblocks, kThreads, 0, s>>>(dc, par, (const double*)f.state[parity], (const double*)f.real_b,
                                                   (double*)f.real_c, (double*)f.g[0], (double*)f.g[1],
                                                   (double*)f.g[2], f.partials3);
  (void)hc;
}

template <>
void kks_launch_pre_pointwise<float>(const KksConst* hc, const KksConst* dc, const KksPar* par, const KksFieldPtrs& f,
                                     int parity, int nblocks, cudaStream_t s) {
  k_pre_pointwise_f32<<<nblocks, kThreads, 0, s>>>(dc, par, (const float*)f.state[parity], (const float*)f.real_b,
                                                   (float*)f.real_c, (float*)f.g[0], (float*)f.g[1], (float*)f.g[2],
                                                   f.partials3);
  (void)hc;
}

template <typename R>
void kks_launch_spectral_update(const KksConst* hc, const KksConst* dc, const KksPar* par, const KksFieldPtrs& f,
                                cudaStream_t s) {
  using C = typename Cplx<R>::T;
  const int g = grid_for(hc->NC, 148 * 8);
  k_spectral_update<R><<<g, kThreads, 0, s>>>(dc, par, (const C*)f.spec_a, (C*)f.spec_bcd, f.kx, f.ky);
}

template <typename R>
void kks_launch_post_pointwise(const KksConst* hc, const KksConst* dc, const KksPar* par, const KksFieldPtrs& f,
                               int parity, int nblocks, cudaStream_t s) {
  k_post_pointwise<R><<<nblocks, kThreads, 0, s>>>(dc, par, (const R*)f.state[parity], (R*)f.state[1 - parity],
                                                   (const R*)f.eta_m, (const R*)f.X_m, (R*)f.mu, (R*)f.g[0],
                                                   (R*)f.g[1], (R*)f.g[2], f.partials5);
  (void)hc;
}

template <typename R>
void kks_launch_restore(const KksConst* hc, const KksConst* dc, const KksCtl* ctl, const KksFieldPtrs& f, int parity,
                        int nblocks, cudaStream_t s) {
  (void)hc;
  k_restore<R><<<nblocks, kThreads, 0, s>>>(dc, ctl, (const R*)f.state[parity], (R*)f.state[1 - parity], (R*)f.eta_m,
                                            (R*)f.X_m);
}

template <typename R>
void kks_launch_elastic_out(const KksConst* hc, const KksConst* dc, const KksPar* par, const R* eta, const R* real_b,
                            double* sig4, double* eps4, int nblocks, cudaStream_t s) {
  (void)hc;
  k_elastic_out<R><<<nblocks, kThreads, 0, s>>>(dc, par, eta, real_b, sig4, eps4);
}

template <typename R>
void kks_launch_to_real(const double* src, R* dst, int n, double shift, cudaStream_t s) {
  k_to_real<R><<<grid_for(n, 148 * 8), kThreads, 0, s>>>(src, dst, n, shift);
}

template <typename R>
void kks_launch_to_double(const R* src, double* dst, int n, double shift, cudaStream_t s) {
  k_to_double<R><<<grid_for(n, 148 * 8), kThreads, 0, s>>>(src, dst, n, shift);
}

#define KKS_INSTANTIATE(R)                                                                                        \
  template void kks_launch_square<R>(const KksConst*, const KksPar*, R*, int, cudaStream_t);                    \
  template void kks_launch_spectral_mid<R>(const KksConst*, const KksConst*, const KksPar*, const KksFieldPtrs&, \
                                           cudaStream_t);                                                        \
  template void kks_launch_spectral_update<R>(const KksConst*, const KksConst*, const KksPar*,                   \
                                              const KksFieldPtrs&, cudaStream_t);                                \
  template void kks_launch_post_pointwise<R>(const KksConst*, const KksConst*, const KksPar*, const KksFieldPtrs&, \
                                             int, int, cudaStream_t);                                            \
  template void kks_launch_restore<R>(const KksConst*, const KksConst*, const KksCtl*, const KksFieldPtrs&, int, \
                                      int, cudaStream_t);                                                        \
  template void kks_launch_elastic_out<R>(const KksConst*, const KksConst*, const KksPar*, const R*, const R*,   \
                                          double*, double*, int, cudaStream_t);                                  \
  template void kks_launch_to_real<R>(const double*, R*, int, double, cudaStream_t);                             \
  template void kks_launch_to_double<R>(const R*, double*, int, double, cudaStream_t);

KKS_INSTANTIATE(double)
KKS_INSTANTIATE(float)
