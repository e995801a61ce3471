// kks_fields.cu - field kernels of one attempt of the semi-implicit KKS step.
//
// An attempt (pf_kks/solver.py:178-276) is, on the device:
//
//   prep            eta -> eta^2 (FP64: in the state buffer; mixed: FP32 copies
//                   of eta, X and eta^2 for the transforms)
//   [cuFFT R2C x3]  FT(eta), FT(X), FT(eta^2)
//   spectral_mid    trace of the Khachaturyan strain, tr eps^ = epsX (C11+2C12)
//                   (Oxx + Oyy) FT(eta^2) (pf_kks/elasticity.py:107-163 in its
//                   closed 2-D form), i k_a FT(eta) (pf_kks/solver.py:258-262),
//                   and the Parseval sums that give the elastic energy sum
//   [cuFFT C2R x3]
//   pre_pointwise   free_energy_terms of the old state (pf_kks/free_energy.py:21-71),
//                   elastic eta-derivative, Allen-Cahn drive and Cahn-Hilliard
//                   fluxes; sums for the energy and the histories
//   [cuFFT R2C x3]
//   spectral_update semi-implicit Allen-Cahn and Cahn-Hilliard divisions
//                   (pf_kks/solver.py:249-264); the mixed path forms the
//                   increments d_eta^, d_X^ instead of the new spectra
//   [cuFFT C2R x2]
//   post_pointwise  new state, phase_compositions (pf_kks/free_energy.py:74-95),
//                   new free energy and diffusion potential, np.gradient energy
//                   term, residual field sums (pf_kks/residual.py:48-66), histories
//   restore         only after a rejection: keep the rejected pair entry and
//                   copy the step's input back into the candidate buffer
//
// Only the elastic energy *sum* enters the step (total_energy), so the strain
// components never need to exist in real space during the step: their sum of
// squares comes from Parseval's theorem on FT(eta^2), and only tr eps is
// transformed back. Each kernel is one coalesced pass over its arrays
// (HBM-bound: no stage is a dense contraction). Reductions are per-block
// partial sums in FP64 finished in a fixed order by the decide kernel, so
// results are deterministic.

#include <math.h>

#include <type_traits>

#include "kks_internal.cuh"
#include "kks_pointwise.cuh"

namespace {

using kks_pw::FreeEnergy;
using kks_pw::free_energy;
using kks_pw::phase_comp;
using kks_pw::strain_multipliers;

template <bool MIXED>
struct Tr;
template <>
struct Tr<false> {
  using R = double;
  using C = double2;
};
template <>
struct Tr<true> {
  using R = float;
  using C = float2;
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

// FP32: the two parabolas in vertex form A (c - v)^2 + f0 with v, f0 from the
// FP64 prologue, which avoids the cancellation of A c^2 + B c + C near the
// vertex (the precipitate parabola has its vertex at c ~ 1).
struct FreeEnergyF {
  float G, G_eta, G_flux, mu;
};

struct ParF {
  float A_a, va, fa0, A_t, vt, ft0, w_s;
};

__device__ __forceinline__ ParF par_f(const KksPar& q) {
  ParF p;
  p.A_a = (float)q.A_alp_s;
  p.va = (float)q.va;
  p.fa0 = (float)q.fa0;
  p.A_t = (float)q.A_thet_s;
  p.vt = (float)q.vt;
  p.ft0 = (float)q.ft0;
  p.w_s = (float)q.w_s;
  return p;
}

__device__ __forceinline__ FreeEnergyF free_energy_f(float ca, float ct, float eta, const ParF& p) {
  FreeEnergyF r;
  const float da = ca - p.va, dt_ = ct - p.vt;
  const float fa_s = p.A_a * da * da + p.fa0;
  const float fa_ca_s = 2.0f * p.A_a * da;
  const float ft_s = p.A_t * dt_ * dt_ + p.ft0;
  const float e2 = eta * eta, e3 = e2 * eta;
  const float h = 3.0f * e2 - 2.0f * e3;
  const float h_eta = 6.0f * eta - 6.0f * e2;
  const float g = e2 - 2.0f * e3 + e2 * e2;
  const float g_eta = 2.0f * eta - 6.0f * e2 + 4.0f * e3;
  r.G = (1.0f - h) * fa_s + h * ft_s + p.w_s * g;
  r.G_eta = -h_eta * (fa_s - ft_s - (ca - ct) * fa_ca_s) + p.w_s * g_eta;
  r.G_flux = h_eta * (ca - ct);
  r.mu = fa_ca_s;
  return r;
}

// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kThreads) k_prep_f64(const KksPar* __restrict__ par, double* __restrict__ state,
                                                       int N, int Np) {
  if (!par->active) return;
  const double* eta = state;
  double* eta2 = state + 2 * (size_t)Np;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
    const double e = eta[i];
    eta2[i] = e * e;
  }
}

__global__ void __launch_bounds__(kThreads) k_prep_mixed(const KksPar* __restrict__ par,
                                                         const double* __restrict__ eta,
                                                         const double* __restrict__ X, float* __restrict__ fin,
                                                         int N, int Np) {
  if (!par->active) return;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
    const double e = eta[i];
    fin[i] = (float)e;
    fin[Np + i] = (float)X[i];
    fin[2 * (size_t)Np + i] = (float)(e * e);
  }
}

template <bool MIXED>
__global__ void __launch_bounds__(kThreads)
    k_spectral_mid(const KksConst* __restrict__ c, const KksPar* __restrict__ par,
                   const typename Tr<MIXED>::C* __restrict__ spec_a, typename Tr<MIXED>::C* __restrict__ spec_b,
                   const double* __restrict__ kxs, const double* __restrict__ kys, double* __restrict__ partials) {
  using R = typename Tr<MIXED>::R;
  using C = typename Tr<MIXED>::C;
  if (!par->active) return;
  const int NC = c->NC, NCp = c->NCp, nyh = c->nyh, ny = c->ny;
  const R inv_N = (R)c->inv_N;
  const R a = (R)(par->epsX * c->c3) * inv_N;
  const R c11 = (R)c->c11, c12 = (R)c->c12;
  const C* eta_h = spec_a;
  const C* eta2_h = spec_a + 2 * (size_t)NCp;
  double acc[6] = {0, 0, 0, 0, 0, 0};
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < NC; k += gridDim.x * blockDim.x) {
    const int ix = k / nyh;
    const int iy = k - ix * nyh;
    const R kx = (R)kxs[ix], ky = (R)kys[iy];
    R oxx, oyy, oxy;
    strain_multipliers<R>(kx, ky, c11, c12, oxx, oyy, oxy);
    const C e2 = eta2_h[k];
    const C eh = eta_h[k];
    const R st = a * (oxx + oyy);
    C o;
    o.x = st * e2.x;
    o.y = st * e2.y;
    spec_b[k] = o;
    const R kxn = kx * inv_N, kyn = ky * inv_N;
    o.x = -kxn * eh.y;
    o.y = kxn * eh.x;
    spec_b[NCp + k] = o;
    o.x = -kyn * eh.y;
    o.y = kyn * eh.x;
    spec_b[2 * (size_t)NCp + k] = o;
    // Parseval sums (half spectrum: interior bins of the y axis count twice)
    const double w = (iy == 0 || (2 * iy == ny)) ? 1.0 : 2.0;
    const double p = w * ((double)e2.x * (double)e2.x + (double)e2.y * (double)e2.y);
    const double dxx = (double)oxx, dyy = (double)oyy, dxy = (double)oxy;
    acc[0] += p * dxx * dxx;
    acc[1] += p * dyy * dyy;
    acc[2] += p * dxx * dyy;
    acc[3] += p * dxy * dxy;
    acc[4] += p * (dxx + dyy);
    acc[5] += p;
  }
  block_reduce_store<6>(acc, partials + (size_t)blockIdx.x * KKS_NPART + P2_OXX2);
}

// The three strain spectra (only for the elastic fields returned at the end).
template <bool MIXED>
__global__ void __launch_bounds__(kThreads)
    k_strain_spectra(const KksConst* __restrict__ c, const KksPar* __restrict__ par,
                     const typename Tr<MIXED>::C* __restrict__ spec_a, typename Tr<MIXED>::C* __restrict__ spec_b,
                     const double* __restrict__ kxs, const double* __restrict__ kys) {
  using R = typename Tr<MIXED>::R;
  using C = typename Tr<MIXED>::C;
  const int NC = c->NC, NCp = c->NCp, nyh = c->nyh;
  const R a = (R)(par->epsX * c->c3) * (R)c->inv_N;
  const R c11 = (R)c->c11, c12 = (R)c->c12;
  const C* eta2_h = spec_a + 2 * (size_t)NCp;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < NC; k += gridDim.x * blockDim.x) {
    const int ix = k / nyh;
    const int iy = k - ix * nyh;
    R oxx, oyy, oxy;
    strain_multipliers<R>((R)kxs[ix], (R)kys[iy], c11, c12, oxx, oyy, oxy);
    const C e2 = eta2_h[k];
    const R m[3] = {a * oxx, a * oyy, a * oxy};
    for (int s = 0; s < 3; ++s) {
      C o;
      o.x = m[s] * e2.x;
      o.y = m[s] * e2.y;
      spec_b[s * (size_t)NCp + k] = o;
    }
  }
}

// ---------------------------------------------------------------------------
// Old-state pointwise pass.
template <bool MIXED>
__global__ void __launch_bounds__(kThreads)
    k_pre_pointwise(const KksConst* __restrict__ c, const KksPar* __restrict__ par, const double* __restrict__ eta,
                    const double* __restrict__ X, const typename Tr<MIXED>::R* __restrict__ Xal,
                    const typename Tr<MIXED>::R* __restrict__ Xth, const typename Tr<MIXED>::R* __restrict__ real_b,
                    typename Tr<MIXED>::R* __restrict__ real_c, typename Tr<MIXED>::R* g0,
                    typename Tr<MIXED>::R* g1, typename Tr<MIXED>::R* g2, double* __restrict__ partials) {
  using R = typename Tr<MIXED>::R;
  if (!par->active) return;
  const KksPar q = *par;
  const int N = c->N, Np = c->Np, nx = c->nx, ny = c->ny;
  const R* tr_a = real_b;
  const R* gx_a = real_b + Np;
  const R* gy_a = real_b + 2 * (size_t)Np;
  R* drive = real_c;
  R* fx = real_c + Np;
  R* fy = real_c + 2 * (size_t)Np;
  R* gs_buf = q.gs == 0 ? g0 : (q.gs == 1 ? g1 : g2);
  const double c3u = c->C11_0 + 2 * c->C12_0;
  const double epsX = q.epsX, C44 = q.C44;
  const ParF pf = par_f(q);
  const float epsXf = (float)epsX;
  const float c3f = (float)(c3u * q.inv_C44);
  double acc[7] = {0, 0, 0, 0, 0, 0, 0};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
    const double e = eta[i];
    const double x = X[i];
    double G;
    if (!MIXED) {
      const FreeEnergy f = free_energy((double)Xal[i], (double)Xth[i], e, q);
      const double tr = (double)tr_a[i];
      const double el_eta = 2 * epsX * e * c3u * (3 * epsX * (e * e) - tr);
      drive[i] = (R)(f.G_eta + el_eta / C44);
      fx[i] = (R)(f.G_flux * (double)gx_a[i]);
      fy[i] = (R)(f.G_flux * (double)gy_a[i]);
      G = f.G;
    } else {
      const float ef = (float)e;
      const FreeEnergyF f = free_energy_f((float)Xal[i], (float)Xth[i], ef, pf);
      const float el_eta_s = 2.0f * epsXf * ef * c3f * (3.0f * epsXf * (ef * ef) - (float)tr_a[i]);
      drive[i] = (R)(f.G_eta + el_eta_s);
      fx[i] = (R)(f.G_flux * (float)gx_a[i]);
      fy[i] = (R)(f.G_flux * (float)gy_a[i]);
      G = (double)f.G;
    }
    if (q.armed_write) gs_buf[i] = (R)G;
    acc[0] += G;
    acc[1] += e;
    if (e < 0.05) { acc[2] += x; acc[3] += 1.0; }
    if (e > 0.95) { acc[4] += x; acc[5] += 1.0; }
    if (q.surface) {
      const int ix = i / ny, iy = i - ix * ny;
      if (ix < nx - 1 && iy < ny - 1 && in_iface(e) && in_iface(eta[i + ny]) && in_iface(eta[i + ny + 1]) &&
          in_iface(eta[i + 1]))
        acc[6] += 1.0;
    }
  }
  block_reduce_store<7>(acc, partials + (size_t)blockIdx.x * KKS_NPART + P3_G);
}

// ---------------------------------------------------------------------------
template <bool MIXED>
__global__ void __launch_bounds__(kThreads)
    k_spectral_update(const KksConst* __restrict__ c, const KksPar* __restrict__ par,
                      const typename Tr<MIXED>::C* __restrict__ spec_a, typename Tr<MIXED>::C* __restrict__ spec_bcd,
                      const double* __restrict__ kxs, const double* __restrict__ kys) {
  using R = typename Tr<MIXED>::R;
  using C = typename Tr<MIXED>::C;
  if (!par->active) return;
  const int NC = c->NC, NCp = c->NCp, nyh = c->nyh;
  const R inv_N = (R)c->inv_N;
  const R ac_mul = (R)par->ac_mul, ac_den = (R)par->ac_den, ch_mul = (R)par->ch_mul;
  const R dt = (R)par->dt, D_s = (R)par->D_s;
  const C* eta_h = spec_a;
  const C* X_h = spec_a + NCp;
  const C* D_h = spec_bcd;
  const C* Fx_h = spec_bcd + NCp;
  const C* Fy_h = spec_bcd + 2 * (size_t)NCp;
  C* eta_o = spec_bcd + 3 * (size_t)NCp;
  C* X_o = spec_bcd + 4 * (size_t)NCp;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < NC; k += gridDim.x * blockDim.x) {
    const int ix = k / nyh;
    const int iy = k - ix * nyh;
    const R kx = (R)kxs[ix], ky = (R)kys[iy];
    const R k2 = kx * kx + ky * ky;
    const C eh = eta_h[k], dh = D_h[k], xh = X_h[k], fxh = Fx_h[k], fyh = Fy_h[k];
    const R den_e = R(1) + ac_den * k2;
    const R flx = -(kx * fxh.y) - ky * fyh.y;  // sum_a i k_a FT(flux_a)
    const R fly = kx * fxh.x + ky * fyh.x;
    const R den_x = R(1) + dt * k2 * D_s;
    C o, p;
    if (!MIXED) {
      // Allen-Cahn: (eta^ - dt L FT(drive)) / (1 + dt L kappa^2 k^2)
      o.x = (ac_mul * dh.x + eh.x) / den_e * inv_N;
      o.y = (ac_mul * dh.y + eh.y) / den_e * inv_N;
      // Cahn-Hilliard: (X^ + dt D sum_a i k_a FT(flux_a)) / (1 + dt k^2 D)
      p.x = (ch_mul * flx + xh.x) / den_x * inv_N;
      p.y = (ch_mul * fly + xh.y) / den_x * inv_N;
    } else {
      // the same updates written as increments of the old spectra
      const R ak = ac_den * k2, bk = dt * k2 * D_s;
      o.x = (ac_mul * dh.x - ak * eh.x) / den_e * inv_N;
      o.y = (ac_mul * dh.y - ak * eh.y) / den_e * inv_N;
      p.x = (ch_mul * flx - bk * xh.x) / den_x * inv_N;
      p.y = (ch_mul * fly - bk * xh.y) / den_x * inv_N;
    }
    eta_o[k] = o;
    X_o[k] = p;
  }
}

// New order parameter at point j: the C2R output (FP64) or the old value plus
// the transformed increment (mixed).
template <bool MIXED>
struct EtaNew {
  const double* base;
  const typename Tr<MIXED>::R* incr;
  __device__ __forceinline__ double operator()(int j) const {
    return MIXED ? base[j] + (double)incr[j] : base[j];
  }
};

template <bool MIXED>
__global__ void __launch_bounds__(kThreads)
    k_post_pointwise(const KksConst* __restrict__ c, const KksPar* __restrict__ par,
                     const double* __restrict__ eta_o, const double* __restrict__ X_o,
                     double* __restrict__ eta_b, double* __restrict__ X_b, typename Tr<MIXED>::R* __restrict__ Xal_b,
                     typename Tr<MIXED>::R* __restrict__ Xth_b, const typename Tr<MIXED>::R* __restrict__ d_eta,
                     const typename Tr<MIXED>::R* __restrict__ d_X, const double* __restrict__ eta_m,
                     const double* __restrict__ X_m, typename Tr<MIXED>::R* __restrict__ mu,
                     typename Tr<MIXED>::R* g0, typename Tr<MIXED>::R* g1, typename Tr<MIXED>::R* g2,
                     double* __restrict__ partials) {
  using R = typename Tr<MIXED>::R;
  if (!par->active) return;
  const KksPar q = *par;
  const int N = c->N, nx = c->nx, ny = c->ny;
  R* gb_buf = q.gb == 0 ? g0 : (q.gb == 1 ? g1 : g2);
  const R* gm_buf = q.gm == 0 ? g0 : (q.gm == 1 ? g1 : g2);
  const double* eta_minus = q.minus_is_state ? eta_o : eta_m;
  const double* X_minus = q.minus_is_state ? X_o : X_m;
  const double dt = q.dt;
  const ParF pf = par_f(q);
  EtaNew<MIXED> en{MIXED ? eta_o : eta_b, d_eta};
  double acc[11] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
    const int ix = i / ny, iy = i - ix * ny;
    const double xo = X_o[i];
    double eb, xb;
    if (MIXED) {
      eb = eta_o[i] + (double)d_eta[i];
      xb = xo + (double)d_X[i];
      eta_b[i] = eb;
      X_b[i] = xb;
    } else {
      eb = eta_b[i];
      xb = X_b[i];
    }
    double xal, xth;
    phase_comp(xo, eb, q, xal, xth);
    Xal_b[i] = (R)xal;
    Xth_b[i] = (R)xth;
    double G_b, mu_b;
    if (!MIXED) {
      const FreeEnergy f = free_energy(xal, xth, eb, q);
      G_b = f.G;
      mu_b = f.mu;
    } else {
      const FreeEnergyF f = free_energy_f((float)xal, (float)xth, (float)eb, pf);
      G_b = f.G;
      mu_b = f.mu;
    }
    // np.gradient: central differences inside, one-sided on the edges
    double gx, gy;
    if (ix == 0) gx = en(i + ny) - eb;
    else if (ix == nx - 1) gx = eb - en(i - ny);
    else gx = (en(i + ny) - en(i - ny)) / 2.0;
    if (iy == 0) gy = en(i + 1) - eb;
    else if (iy == ny - 1) gy = eb - en(i - 1);
    else gy = (en(i + 1) - en(i - 1)) / 2.0;
    acc[0] += gx * gx + gy * gy;
    if (eb < 0.05) { acc[1] += xb; acc[2] += 1.0; }
    if (eb > 0.95) { acc[3] += xb; acc[4] += 1.0; }
    acc[5] += eb;
    if (q.surface && ix < nx - 1 && iy < ny - 1 && in_iface(eb) && in_iface(en(i + ny)) &&
        in_iface(en(i + ny + 1)) && in_iface(en(i + 1)))
      acc[6] += 1.0;
    if (q.armed_write) {
      if (q.armed_residual) {
        const double mum = (double)mu[i];
        const double dXdt = (xb - X_minus[i]) / dt;
        const double mu_mean = (mu_b + mum) / 2;
        const double diffusion = dXdt * mu_mean;
        const double detadt = (eb - eta_minus[i]) / dt;
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
template <bool MIXED>
__global__ void __launch_bounds__(kThreads)
    k_restore(const KksConst* __restrict__ c, const KksCtl* __restrict__ ctl, const double* __restrict__ eta_i,
              const double* __restrict__ X_i, const typename Tr<MIXED>::R* __restrict__ Xal_i,
              const typename Tr<MIXED>::R* __restrict__ Xth_i, double* __restrict__ eta_o,
              double* __restrict__ X_o, typename Tr<MIXED>::R* __restrict__ Xal_o,
              typename Tr<MIXED>::R* __restrict__ Xth_o, double* __restrict__ eta_m, double* __restrict__ X_m) {
  if (!ctl->restore || ctl->status != KKS_STATUS_OK) return;
  using R = typename Tr<MIXED>::R;
  using R2 = typename std::conditional<MIXED, float2, double2>::type;
  const int N = c->N;
  const int stride = gridDim.x * blockDim.x;
  int start = 0;
  // two points per access where every array allows it (16-byte double pairs,
  // 8- or 16-byte pairs of the composition type): a copy of ~80 bytes per
  // point, bound by HBM, wants the wide accesses and their bytes in flight
  const uintptr_t a8 = (uintptr_t)eta_i | (uintptr_t)X_i | (uintptr_t)eta_o | (uintptr_t)X_o |
                       (uintptr_t)eta_m | (uintptr_t)X_m;
  const uintptr_t ar = (uintptr_t)Xal_i | (uintptr_t)Xth_i | (uintptr_t)Xal_o | (uintptr_t)Xth_o;
  if ((a8 & 15u) == 0 && (ar & (2 * sizeof(R) - 1)) == 0) {
    const int N2 = N / 2;
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < N2; j += stride) {
      const double2 eo = ((const double2*)eta_o)[j], xo = ((const double2*)X_o)[j];
      const double2 ei = ((const double2*)eta_i)[j], xi = ((const double2*)X_i)[j];
      const R2 ai = ((const R2*)Xal_i)[j], ti = ((const R2*)Xth_i)[j];
      ((double2*)eta_m)[j] = eo;
      ((double2*)X_m)[j] = xo;
      ((double2*)eta_o)[j] = ei;
      ((double2*)X_o)[j] = xi;
      ((R2*)Xal_o)[j] = ai;
      ((R2*)Xth_o)[j] = ti;
    }
    start = 2 * N2;
  }
  for (int i = start + blockIdx.x * blockDim.x + threadIdx.x; i < N; i += stride) {
    eta_m[i] = eta_o[i];
    X_m[i] = X_o[i];
    eta_o[i] = eta_i[i];
    X_o[i] = X_i[i];
    Xal_o[i] = Xal_i[i];
    Xth_o[i] = Xth_i[i];
  }
}

// Stress and elastic strain returned by solve_elasticity (components xx, yy, zz, xy).
template <bool MIXED>
__global__ void __launch_bounds__(kThreads)
    k_elastic_out(const KksConst* __restrict__ c, const KksPar* __restrict__ par, const double* __restrict__ eta,
                  const typename Tr<MIXED>::R* __restrict__ real_b, double* __restrict__ sig4,
                  double* __restrict__ eps4) {
  const int N = c->N, Np = c->Np;
  const double C11 = c->C11_0, C12 = c->C12_0, C44_0 = c->C44_0, epsX = par->epsX;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
    const double e = eta[i];
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
__global__ void k_to_real(const double* __restrict__ src, R* __restrict__ dst, int n) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) dst[i] = (R)src[i];
}

template <typename R>
__global__ void k_to_double(const R* __restrict__ src, double* __restrict__ dst, int n) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) dst[i] = (double)src[i];
}

int grid_for(int n, int cap) {
  int g = (n + kThreads - 1) / kThreads;
  return g < cap ? (g > 0 ? g : 1) : cap;
}

}  // namespace

int kks_field_blocks(int N, int num_sms) { return grid_for(N, num_sms * 4); }

template <bool MIXED>
void kks_launch_prep(const KksConst* hc, const KksPar* par, const KksFieldPtrs& f, int p, int nblocks,
                     cudaStream_t s) {
  if (!MIXED) {
    k_prep_f64<<<nblocks, kThreads, 0, s>>>(par, (double*)f.eta[p], hc->N, hc->Np);
  } else {
    k_prep_mixed<<<nblocks, kThreads, 0, s>>>(par, (const double*)f.eta[p], (const double*)f.X[p],
                                              (float*)f.fft_in[p], hc->N, hc->Np);
  }
}

template <bool MIXED>
void kks_launch_spectral_mid(const KksConst* hc, const KksConst* dc, const KksPar* par, const KksFieldPtrs& f,
                             int nblocks, cudaStream_t s) {
  using C = typename Tr<MIXED>::C;
  (void)hc;
  k_spectral_mid<MIXED><<<nblocks, kThreads, 0, s>>>(dc, par, (const C*)f.spec_a, (C*)f.spec_bcd, f.kx, f.ky,
                                                     f.partials);
}

template <bool MIXED>
void kks_launch_strain_spectra(const KksConst* hc, const KksConst* dc, const KksPar* par, const KksFieldPtrs& f,
                               int nblocks, cudaStream_t s) {
  using C = typename Tr<MIXED>::C;
  (void)hc;
  k_strain_spectra<MIXED><<<nblocks, kThreads, 0, s>>>(dc, par, (const C*)f.spec_a, (C*)f.spec_bcd, f.kx, f.ky);
}

template <bool MIXED>
void kks_launch_pre_pointwise(const KksConst* hc, const KksConst* dc, const KksPar* par, const KksFieldPtrs& f,
                              int p, int nblocks, cudaStream_t s) {
  using R = typename Tr<MIXED>::R;
  (void)hc;
  k_pre_pointwise<MIXED><<<nblocks, kThreads, 0, s>>>(dc, par, (const double*)f.eta[p], (const double*)f.X[p],
                                                      (const R*)f.X_al[p], (const R*)f.X_th[p], (const R*)f.real_b,
                                                      (R*)f.real_c, (R*)f.g[0], (R*)f.g[1], (R*)f.g[2], f.partials);
}

template <bool MIXED>
void kks_launch_spectral_update(const KksConst* hc, const KksConst* dc, const KksPar* par, const KksFieldPtrs& f,
                                int nblocks, cudaStream_t s) {
  using C = typename Tr<MIXED>::C;
  (void)hc;
  k_spectral_update<MIXED><<<nblocks, kThreads, 0, s>>>(dc, par, (const C*)f.spec_a, (C*)f.spec_bcd, f.kx, f.ky);
}

template <bool MIXED>
void kks_launch_post_pointwise(const KksConst* hc, const KksConst* dc, const KksPar* par, const KksFieldPtrs& f,
                               int p, int nblocks, cudaStream_t s) {
  using R = typename Tr<MIXED>::R;
  const int q = 1 - p;
  const R* d_eta = MIXED ? (const R*)f.real_c : nullptr;
  const R* d_X = MIXED ? (const R*)f.real_c + hc->Np : nullptr;
  k_post_pointwise<MIXED><<<nblocks, kThreads, 0, s>>>(
      dc, par, (const double*)f.eta[p], (const double*)f.X[p], (double*)f.eta[q], (double*)f.X[q], (R*)f.X_al[q],
      (R*)f.X_th[q], d_eta, d_X, (const double*)f.eta_m, (const double*)f.X_m, (R*)f.mu, (R*)f.g[0], (R*)f.g[1],
      (R*)f.g[2], f.partials);
}

template <bool MIXED>
void kks_launch_restore(const KksConst* hc, const KksConst* dc, const KksCtl* ctl, const KksFieldPtrs& f, int p,
                        int nblocks, cudaStream_t s) {
  using R = typename Tr<MIXED>::R;
  (void)hc;
  const int q = 1 - p;
  k_restore<MIXED><<<nblocks, kThreads, 0, s>>>(dc, ctl, (const double*)f.eta[p], (const double*)f.X[p],
                                                (const R*)f.X_al[p], (const R*)f.X_th[p], (double*)f.eta[q],
                                                (double*)f.X[q], (R*)f.X_al[q], (R*)f.X_th[q], (double*)f.eta_m,
                                                (double*)f.X_m);
}

template <bool MIXED>
void kks_launch_elastic_out(const KksConst* hc, const KksConst* dc, const KksPar* par, const KksFieldPtrs& f, int p,
                            double* sig4, double* eps4, int nblocks, cudaStream_t s) {
  using R = typename Tr<MIXED>::R;
  (void)hc;
  k_elastic_out<MIXED><<<nblocks, kThreads, 0, s>>>(dc, par, (const double*)f.eta[p], (const R*)f.real_b, sig4,
                                                    eps4);
}

template <typename R>
void kks_launch_to_real(const double* src, R* dst, int n, cudaStream_t s) {
  k_to_real<R><<<grid_for(n, 148 * 8), kThreads, 0, s>>>(src, dst, n);
}

template <typename R>
void kks_launch_to_double(const R* src, double* dst, int n, cudaStream_t s) {
  k_to_double<R><<<grid_for(n, 148 * 8), kThreads, 0, s>>>(src, dst, n);
}

#define KKS_INSTANTIATE(M)                                                                                         \
  template void kks_launch_prep<M>(const KksConst*, const KksPar*, const KksFieldPtrs&, int, int, cudaStream_t);   \
  template void kks_launch_spectral_mid<M>(const KksConst*, const KksConst*, const KksPar*, const KksFieldPtrs&,  \
                                           int, cudaStream_t);                                                    \
  template void kks_launch_strain_spectra<M>(const KksConst*, const KksConst*, const KksPar*, const KksFieldPtrs&, \
                                             int, cudaStream_t);                                                  \
  template void kks_launch_pre_pointwise<M>(const KksConst*, const KksConst*, const KksPar*, const KksFieldPtrs&, \
                                            int, int, cudaStream_t);                                              \
  template void kks_launch_spectral_update<M>(const KksConst*, const KksConst*, const KksPar*,                    \
                                              const KksFieldPtrs&, int, cudaStream_t);                            \
  template void kks_launch_post_pointwise<M>(const KksConst*, const KksConst*, const KksPar*,                     \
                                             const KksFieldPtrs&, int, int, cudaStream_t);                        \
  template void kks_launch_restore<M>(const KksConst*, const KksConst*, const KksCtl*, const KksFieldPtrs&, int,  \
                                      int, cudaStream_t);                                                         \
  template void kks_launch_elastic_out<M>(const KksConst*, const KksConst*, const KksPar*, const KksFieldPtrs&,   \
                                          int, double*, double*, int, cudaStream_t);

KKS_INSTANTIATE(false)
KKS_INSTANTIATE(true)
template void kks_launch_to_real<float>(const double*, float*, int, cudaStream_t);
template void kks_launch_to_real<double>(const double*, double*, int, cudaStream_t);
template void kks_launch_to_double<float>(const float*, double*, int, cudaStream_t);
template void kks_launch_to_double<double>(const double*, double*, int, cudaStream_t);
