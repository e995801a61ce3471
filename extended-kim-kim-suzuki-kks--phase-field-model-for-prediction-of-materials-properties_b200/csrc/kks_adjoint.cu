// kks_adjoint.cu - the fixed-dt FP64 step with explicit per-step coefficients,
// and its hand-written vector-Jacobian product (adjoint).
//
// A fixed-dt step is the unarmed branch of the attempt loop
// (pf_kks/solver.py:176-290 with flag == 0): no residual, no decision. Its
// coefficients (dt, L_s, kappa^2_s, D_s, w_s, the two parabolas, epsX, C44 and
// the phase-composition constants) depend only on the schedule and the kinetic
// parameters, not on the fields, so a step is the map
//   (eta, X, X_al, X_th; c) -> (eta_b, X_b, X_al_b, X_th_b)
//   trtr   = IFT[ epsX c3 / C44_0 (Oxx + Oyy) FT(eta^2) ]                 elasticity.py:140-163
//   drive  = G_eta_s(X_al, X_th, eta) + 2 epsX eta (C11_0+2C12_0)(3 epsX eta^2 - trtr) / C44
//   eta_b  = IFT[ (FT eta - dt L_s FT drive) / (1 + dt L_s kappa^2 k^2) ]   solver.py:249-254
//   flux_a = h'(eta)(X_al - X_th) IFT[i k_a FT eta]
//   X_b    = IFT[ (FT X + dt D_s sum_a i k_a FT flux_a) / (1 + dt D_s k^2) ] solver.py:256-264
//   X_al_b, X_th_b = phase_compositions(X, eta_b)                         free_energy.py:74-95
// with the reference's wave vectors (Nyquist entries 0) and the stiffness
// frozen at T(t = 0). The adjoint takes the cotangents of the four outputs and
// returns those of the four inputs and the gradient of <cotangent, output>
// with respect to the 15 coefficients. Every spectral multiplier is real and
// even in k, so the operators IFT m(k) FT are self-adjoint and i k_a is
// anti-self-adjoint; the pointwise parts are differentiated by hand. The
// phase-composition guards (+/-inf, NaN) are treated as inactive.
//
// Mixed precision (kks_adj_set_precision): every transform runs in FP32 (the
// real input rounded to float, cuFFT R2C / C2R in single precision, the
// output widened back), everything else stays FP64, and, as in the main mixed
// step, the semi-implicit updates carry only the increments through the FP32
// transforms: eta_b = eta + IFT[(-dt L_s FT drive - dt L_s kappa^2 k^2 FT eta)
// / (1 + dt L_s kappa^2 k^2)] and X_b = X + IFT[(dt D_s S^ - dt D_s k^2 FT X) /
// (1 + dt D_s k^2)], so that the FP32 rounding scales with the step's change,
// not with the fields. The backward pass writes the adjoint operators the same
// way: A[l] = l + IFT[(A(k) - 1) FT l].

#include <cuda_runtime.h>
#include <cufft.h>
#include <math.h>

#include <string>
#include <vector>

#include "kks.h"

int kks_set_error(int code, const std::string& msg);

namespace {

constexpr int kT = 256;
constexpr int kBlocks = 296;  // 2 x 148 SMs
constexpr int kNS = 16;       // partial-sum slots

enum { S_GP = 0, S_GK, S_GQ, S_W, S_AA, S_BA, S_CA, S_AT, S_BT, S_CT, S_EPSX, S_C44, S_PCS, S_PCR };

struct Coef {
  double dt, Ls, kappa2, Ds, w, Aa, Ba, Ca, At, Bt, Ct, epsX, C44, pcs, pcr;
};

struct Spec {
  int nx, ny, nyh, N, NC;
  double invN;
  double cc;       // C11_0 + 2 C12_0
  double c3n;      // (C11_0 + 2 C12_0) / C44_0
  double c11, c12; // C11_0 / C44_0, C12_0 / C44_0
};

__device__ __forceinline__ double2 cm(double2 a, double s) { return make_double2(a.x * s, a.y * s); }
__device__ __forceinline__ double2 cmi(double2 a, double s) { return make_double2(-a.y * s, a.x * s); }  // i s a

__device__ double otr(double kx, double ky, double c11, double c12) {
  const double Kxx = c11 * kx * kx + ky * ky, Kyy = kx * kx + c11 * ky * ky, Kxy = (c12 + 1.0) * kx * ky;
  const double det = Kxx * Kyy - Kxy * Kxy;
  if (det == 0.0) return 0.0;
  const double inv = 1.0 / det;
  const double Nxx = Kyy * inv, Nyy = Kxx * inv, Nxy = -Kxy * inv;
  return (Nxx * kx + Nxy * ky) * kx + (Nxy * kx + Nyy * ky) * ky;
}

// multiplier kinds applied to a half spectrum (all include the 1/N of the inverse)
enum { M_TR = 0, M_DX, M_DY, M_AETA, M_AX, M_LAP, M_AETA_INC, M_AX_INC };

// in and out may be the same array (an in-place multiply)
__global__ void k_spec_mul(const double2* in, double2* out, Spec s, const double* kx, const double* ky, int kind,
                           double p0, double p1) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < s.NC; i += gridDim.x * blockDim.x) {
    const int ix = i / s.nyh, iy = i - ix * s.nyh;
    const double a = kx[ix], b = ky[iy], k2 = a * a + b * b;
    const double2 v = in[i];
    double2 r;
    switch (kind) {
      case M_TR: r = cm(v, p0 * otr(a, b, s.c11, s.c12) * s.invN); break;   // p0 = epsX c3n
      case M_DX: r = cmi(v, a * p0 * s.invN); break;                          // p0 scale
      case M_DY: r = cmi(v, b * p0 * s.invN); break;
      case M_AETA: r = cm(v, s.invN / (1.0 + p0 * p1 * k2)); break;          // p0 = dt L_s, p1 = kappa^2
      case M_AX: r = cm(v, s.invN / (1.0 + p0 * k2)); break;                  // p0 = dt D_s
      case M_AETA_INC: r = cm(v, -p0 * p1 * k2 / (1.0 + p0 * p1 * k2) * s.invN); break;  // M_AETA - 1
      case M_AX_INC: r = cm(v, -p0 * k2 / (1.0 + p0 * k2) * s.invN); break;              // M_AX - 1
      default: r = cm(v, -k2 * s.invN); break;                                // Laplacian
    }
    out[i] = r;
  }
}

// eta_b^ and X_b^ / N from FT eta, FT drive, FT X, FT flux_x, FT flux_y; with
// lap = 1 the outputs are instead IFT-ready -k^2 eta_b^ / N and (S^ - k^2 X_b^) / N,
// with lap = 2 the increments (eta_b^ - eta^) / N and (X_b^ - X^) / N.
__global__ void k_spec_update(const double2* __restrict__ e, const double2* __restrict__ d,
                              const double2* __restrict__ x, const double2* __restrict__ fx,
                              const double2* __restrict__ fy, double2* __restrict__ eb, double2* __restrict__ xb,
                              Spec s, const double* kx, const double* ky, Coef c, int lap) {
  const double p = c.dt * c.Ls, q = c.dt * c.Ds;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < s.NC; i += gridDim.x * blockDim.x) {
    const int ix = i / s.nyh, iy = i - ix * s.nyh;
    const double a = kx[ix], b = ky[iy], k2 = a * a + b * b;
    const double2 E = e[i], D = d[i], X = x[i], Fx = fx[i], Fy = fy[i];
    // S^ = i kx Fx + i ky Fy
    const double2 S = make_double2(-(a * Fx.y) - b * Fy.y, a * Fx.x + b * Fy.x);
    const double de = 1.0 + p * c.kappa2 * k2, dx = 1.0 + q * k2;
    const double2 Eb = make_double2((E.x - p * D.x) / de, (E.y - p * D.y) / de);
    const double2 Xb = make_double2((X.x + q * S.x) / dx, (X.y + q * S.y) / dx);
    if (lap == 2) {  // increments
      eb[i] = make_double2((Eb.x - E.x) * s.invN, (Eb.y - E.y) * s.invN);
      xb[i] = make_double2((Xb.x - X.x) * s.invN, (Xb.y - X.y) * s.invN);
    } else if (!lap) {
      eb[i] = cm(Eb, s.invN);
      xb[i] = cm(Xb, s.invN);
    } else {
      eb[i] = cm(Eb, -k2 * s.invN);
      xb[i] = make_double2((S.x - k2 * Xb.x) * s.invN, (S.y - k2 * Xb.y) * s.invN);
    }
  }
}

__global__ void k_narrow(const double* __restrict__ in, float* __restrict__ out, int n) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) out[i] = (float)in[i];
}
__global__ void k_widen(const float* __restrict__ in, double* __restrict__ out, int n) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) out[i] = (double)in[i];
}
// out = a + b (FP64 state plus an increment); out may be b
__global__ void k_add(const double* a, const double* b, double* out, int n) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) out[i] = a[i] + b[i];
}

__global__ void k_square(const double* __restrict__ e, double* __restrict__ sq, int N) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) sq[i] = e[i] * e[i];
}

// drive and fluxes of the old state (free_energy.py:21-71 terms, elasticity el_eta)
__global__ void k_fwd_pointwise(const double* __restrict__ e_, const double* __restrict__ ca_,
                                const double* __restrict__ ct_, const double* __restrict__ tr,
                                const double* __restrict__ gx, const double* __restrict__ gy,
                                double* __restrict__ drive, double* __restrict__ fx, double* __restrict__ fy, Spec s,
                                Coef c) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < s.N; i += gridDim.x * blockDim.x) {
    const double e = e_[i], ca = ca_[i], ct = ct_[i];
    const double fa = c.Aa * ca * ca + c.Ba * ca + c.Ca, fa1 = 2 * c.Aa * ca + c.Ba;
    const double ft = c.At * ct * ct + c.Bt * ct + c.Ct;
    const double h1 = 6.0 * e - 6 * e * e;
    const double g1 = 2.0 * e - 6.0 * e * e + 4.0 * e * e * e;
    const double Geta = -h1 * (fa - ft - (ca - ct) * fa1) + c.w * g1;
    const double el = 2 * c.epsX * e * s.cc * (3 * c.epsX * e * e - tr[i]) / c.C44;
    drive[i] = Geta + el;
    const double fl = h1 * (ca - ct);
    fx[i] = fl * gx[i];
    fy[i] = fl * gy[i];
  }
}

// phase compositions of (X_old, eta_b) (free_energy.py:74-95, guards included)
__global__ void k_phase(const double* __restrict__ X, const double* __restrict__ eb, double* __restrict__ ca,
                        double* __restrict__ ct, int N, Coef c) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
    const double e = eb[i];
    const double h = 3.0 * (e * e) - 2 * (e * e * e);
    double a = (X[i] - h * c.pcs) / ((1 - h) + h * c.pcr);
    if (isinf(a)) a = a > 0 ? 1e-6 : -1e-6;
    if (isnan(a)) a = 1e-6;
    double t = c.pcr * a + c.pcs;
    if (isinf(t)) t = t > 0 ? 1e-6 : -1e-6;
    if (isnan(t)) t = 1e-6;
    ca[i] = a;
    ct[i] = t;
  }
}

template <int NV>
__device__ void block_sums(double (&v)[NV], double* out) {
  __shared__ double sh[NV][kT / 32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  for (int k = 0; k < NV; ++k) {
    double x = v[k];
    for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
    if (lane == 0) sh[k][w] = x;
  }
  __syncthreads();
  if (threadIdx.x < NV) {
    double x = 0;
    for (int j = 0; j < kT / 32; ++j) x += sh[threadIdx.x][j];
    out[threadIdx.x] = x;
  }
}

// back through the phase compositions: cotangent of eta_b in full, the part
// of X's cotangent from X_al_b / X_th_b, and the pc_s / pc_r sums
__global__ void k_back_phase(const double* __restrict__ X, const double* __restrict__ eb,
                             const double* __restrict__ cab, const double* __restrict__ leb,
                             const double* __restrict__ lcab, const double* __restrict__ lctb,
                             double* __restrict__ leb_tot, double* __restrict__ lx_pc, int N, Coef c,
                             double* __restrict__ partials) {
  double acc[2] = {0, 0};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
    const double e = eb[i];
    const double h = 3.0 * (e * e) - 2 * (e * e * e), h1 = 6.0 * e - 6 * e * e;
    const double num = X[i] - h * c.pcs, den = (1 - h) + h * c.pcr;
    const double lt = lctb[i];
    const double la = lcab[i] + c.pcr * lt;  // X_th_b = r X_al_b + s
    const double dadh = (-c.pcs * den - num * (c.pcr - 1)) / (den * den);
    leb_tot[i] = leb[i] + la * dadh * h1;
    lx_pc[i] = la / den;
    acc[0] += la * (-h / den) + lt;                     // d / d pc_s
    acc[1] += la * (-num * h / (den * den)) + lt * cab[i];  // d / d pc_r
  }
  block_sums<2>(acc, partials + (size_t)blockIdx.x * kNS + S_PCS);
}

// the main pointwise back pass (see the header comment for the chain)
__global__ void k_back_main(const double* __restrict__ e_, const double* __restrict__ ca_,
                            const double* __restrict__ ct_, const double* __restrict__ tr,
                            const double* __restrict__ gx, const double* __restrict__ gy,
                            const double* __restrict__ drive, const double* __restrict__ mu_e,
                            const double* __restrict__ mu_x, const double* __restrict__ lfx,
                            const double* __restrict__ lfy, const double* __restrict__ lap_eb,
                            const double* __restrict__ sx_b, double* __restrict__ ltr, double* __restrict__ lgx,
                            double* __restrict__ lgy, double* __restrict__ le_part, double* __restrict__ lca,
                            double* __restrict__ lct, Spec s, Coef c, double* __restrict__ partials) {
  double acc[12] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
  const double p = c.dt * c.Ls;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < s.N; i += gridDim.x * blockDim.x) {
    const double e = e_[i], ca = ca_[i], ct = ct_[i], dc = ca - ct;
    const double fa = c.Aa * ca * ca + c.Ba * ca + c.Ca, fa1 = 2 * c.Aa * ca + c.Ba;
    const double ft = c.At * ct * ct + c.Bt * ct + c.Ct, ft1 = 2 * c.At * ct + c.Bt;
    const double h1 = 6.0 * e - 6 * e * e, h2 = 6.0 - 12.0 * e;
    const double g1 = 2.0 * e - 6.0 * e * e + 4.0 * e * e * e, g2 = 2.0 - 12.0 * e + 12.0 * e * e;
    const double m = mu_e[i];
    const double lG = -p * m;  // cotangent of the drive (G_eta_s and el_eta_s alike)
    const double k_el = 2 * s.cc / c.C44;
    const double el = k_el * c.epsX * e * (3 * c.epsX * e * e - tr[i]);
    // Allen-Cahn coefficient sums: d/dp and d/dkappa^2 of <lambda, eta_b>
    acc[S_GP] += -m * (drive[i] - c.kappa2 * lap_eb[i]);
    acc[S_GK] += p * m * lap_eb[i];
    acc[S_GQ] += mu_x[i] * sx_b[i];
    // free-energy coefficients
    acc[S_W] += lG * g1;
    acc[S_AA] += lG * (-h1 * (ca * ca - 2 * ca * dc));
    acc[S_BA] += lG * (-h1 * ct);
    acc[S_CA] += lG * (-h1);
    acc[S_AT] += lG * (h1 * ct * ct);
    acc[S_BT] += lG * (h1 * ct);
    acc[S_CT] += lG * h1;
    acc[S_EPSX] += lG * k_el * (6 * c.epsX * e * e * e - 2 * e * tr[i]);
    acc[S_C44] += -lG * el / c.C44;
    // fields
    const double lf_x = lfx[i], lf_y = lfy[i], g_x = gx[i], g_y = gy[i];
    const double lh1 = dc * (g_x * lf_x + g_y * lf_y);
    const double ldc = h1 * (g_x * lf_x + g_y * lf_y);
    lgx[i] = h1 * dc * lf_x;
    lgy[i] = h1 * dc * lf_y;
    ltr[i] = -k_el * c.epsX * e * lG;
    const double dG_de = -h2 * (fa - ft - dc * fa1) + c.w * g2;
    const double del_de = k_el * (9 * c.epsX * c.epsX * e * e - c.epsX * tr[i]);
    le_part[i] = m + lh1 * h2 + lG * (dG_de + del_de);
    lca[i] = ldc + lG * (2 * c.Aa * h1 * dc);
    lct[i] = -ldc + lG * (-h1 * (fa1 - ft1));
  }
  block_sums<12>(acc, partials + (size_t)blockIdx.x * kNS + S_GP);
}

__global__ void k_back_final(const double* __restrict__ e, const double* __restrict__ le_part,
                             const double* __restrict__ lsq, const double* __restrict__ dv,
                             const double* __restrict__ mu_x, const double* __restrict__ lx_pc,
                             double* __restrict__ le, double* __restrict__ lx, int N) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
    le[i] = le_part[i] + 2 * e[i] * lsq[i] - dv[i];
    lx[i] = mu_x[i] + lx_pc[i];
  }
}

__global__ void k_finish(const double* __restrict__ partials, int nb, double* __restrict__ out) {
  const int k = threadIdx.x;
  if (k >= kNS) return;
  double v = 0;
  for (int b = 0; b < nb; ++b) v += partials[(size_t)b * kNS + k];
  out[k] = v;
}

// The gradient of <lam_out, state_out> with respect to the coefficient row
// from the finished sums g (one thread; the same expressions as the host
// version in kks_adj_backward).
__device__ __host__ inline void dcoef_of(const double* g, const Coef& c, double* d) {
  for (int k = 0; k < KKS_COEF_COUNT; ++k) d[k] = 0.0;
  d[KKS_COEF_DT] = c.Ls * g[S_GP] + c.Ds * g[S_GQ];
  d[KKS_COEF_LS] = c.dt * g[S_GP];
  d[KKS_COEF_KAPPA2] = g[S_GK];
  d[KKS_COEF_DS] = c.dt * g[S_GQ];
  d[KKS_COEF_W] = g[S_W];
  d[KKS_COEF_A_ALP] = g[S_AA];
  d[KKS_COEF_B_ALP] = g[S_BA];
  d[KKS_COEF_C_ALP] = g[S_CA];
  d[KKS_COEF_A_THET] = g[S_AT];
  d[KKS_COEF_B_THET] = g[S_BT];
  d[KKS_COEF_C_THET] = g[S_CT];
  d[KKS_COEF_EPSX] = g[S_EPSX];
  d[KKS_COEF_C44] = g[S_C44];
  d[KKS_COEF_PC_SHIFT] = g[S_PCS];
  d[KKS_COEF_PC_RATIO] = g[S_PCR];
}

__global__ void k_dcoef(const double* __restrict__ g, Coef c, double* __restrict__ d) {
  if (threadIdx.x == 0) dcoef_of(g, c, d);
}

// i kx A + i ky B (both half spectra), times 1/N
__global__ void k_spec_div(const double2* __restrict__ A, const double2* __restrict__ B, double2* __restrict__ out,
                           Spec s, const double* kx, const double* ky) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < s.NC; i += gridDim.x * blockDim.x) {
    const int ix = i / s.nyh, iy = i - ix * s.nyh;
    const double a = kx[ix], b = ky[iy];
    const double2 u = A[i], v = B[i];
    out[i] = make_double2((-(a * u.y) - b * v.y) * s.invN, (a * u.x + b * v.x) * s.invN);
  }
}

void wave_numbers(int n, std::vector<double>& out, int count) {
  // angular wave numbers of a unit-spacing axis, Nyquist entry of an even axis 0
  std::vector<double> lin(n, 0.0);
  if (n % 2 == 1) {
    const int half = (int)((n - 1) / 2.0 + 1);
    for (int j = 0; j < half; ++j) lin[j] = (double)j * 2 * M_PI / (n * 1.0);
    for (int j = half, v = (int)(-(n + 1) / 2.0 + 1); j < n; ++j, ++v) lin[j] = (double)v * 2 * M_PI / (n * 1.0);
  } else {
    for (int j = 0; j < n / 2; ++j) lin[j] = (double)j * 2 * M_PI / (n * 1.0);
    for (int j = n / 2 + 1, v = -n / 2 + 1; j < n; ++j, ++v) lin[j] = (double)v * 2 * M_PI / (n * 1.0);
  }
  out.assign(lin.begin(), lin.begin() + count);
}

}  // namespace

struct kks_adj {
  int device = 0;
  int mixed = 0;  // 1: FP32 transforms (kks_adj_set_precision)
  Spec s{};
  cudaStream_t stream = nullptr;  // the stream the calls run on (own, or bound by kks_adj_set_stream)
  cudaStream_t own = nullptr;     // the handle's own stream
  bool bound = false;             // calls run on a caller's stream and return without waiting
  cufftHandle r2c = 0, c2r = 0;
  cufftHandle r2c32 = 0, c2r32 = 0;
  float* fbuf = nullptr;   // FP32 real transform buffer (N)
  float* zbuf = nullptr;   // FP32 half-spectrum buffer (2 NC)
  double *kx = nullptr, *ky = nullptr;
  double* f = nullptr;      // real work fields
  double2* z = nullptr;     // half-spectrum work
  double* partials = nullptr;
  double* sums = nullptr;
  double* h_sums = nullptr;  // pinned
};

namespace {

constexpr int kFields = 20;
constexpr int kSpectra = 8;

#define ACK(expr)                                                                                    \
  do {                                                                                               \
    cudaError_t _e = (expr);                                                                         \
    if (_e != cudaSuccess) return kks_set_error(KKS_ERR_CUDA, std::string(#expr) + ": " + cudaGetErrorString(_e)); \
  } while (0)
#define AFK(expr)                                                                                    \
  do {                                                                                               \
    if ((expr) != CUFFT_SUCCESS) return kks_set_error(KKS_ERR_CUFFT, std::string(#expr));            \
  } while (0)

Coef coef_of(const double* c) {
  Coef k;
  k.dt = c[KKS_COEF_DT]; k.Ls = c[KKS_COEF_LS]; k.kappa2 = c[KKS_COEF_KAPPA2]; k.Ds = c[KKS_COEF_DS];
  k.w = c[KKS_COEF_W]; k.Aa = c[KKS_COEF_A_ALP]; k.Ba = c[KKS_COEF_B_ALP]; k.Ca = c[KKS_COEF_C_ALP];
  k.At = c[KKS_COEF_A_THET]; k.Bt = c[KKS_COEF_B_THET]; k.Ct = c[KKS_COEF_C_THET]; k.epsX = c[KKS_COEF_EPSX];
  k.C44 = c[KKS_COEF_C44]; k.pcs = c[KKS_COEF_PC_SHIFT]; k.pcr = c[KKS_COEF_PC_RATIO];
  return k;
}

double* fld(kks_adj* h, int k) { return h->f + (size_t)k * h->s.N; }
double2* spc(kks_adj* h, int k) { return h->z + (size_t)k * h->s.NC; }

// Forward / inverse real transforms of the step: FP64 cuFFT, or in mixed
// precision FP32 cuFFT on the rounded input with the output widened back.
int r2c(kks_adj* h, const double* in, double2* out) {
  if (!h->mixed) {
    AFK(cufftExecD2Z(h->r2c, (double*)in, (cufftDoubleComplex*)out));
    return KKS_OK;
  }
  const Spec& s = h->s;
  k_narrow<<<kBlocks, kT, 0, h->stream>>>(in, h->fbuf, s.N);
  AFK(cufftExecR2C(h->r2c32, h->fbuf, (cufftComplex*)h->zbuf));
  k_widen<<<kBlocks, kT, 0, h->stream>>>(h->zbuf, (double*)out, 2 * s.NC);
  return KKS_OK;
}

int c2r(kks_adj* h, double2* in, double* out) {
  if (!h->mixed) {
    AFK(cufftExecZ2D(h->c2r, (cufftDoubleComplex*)in, out));
    return KKS_OK;
  }
  const Spec& s = h->s;
  k_narrow<<<kBlocks, kT, 0, h->stream>>>((const double*)in, h->zbuf, 2 * s.NC);
  AFK(cufftExecC2R(h->c2r32, (cufftComplex*)h->zbuf, h->fbuf));
  k_widen<<<kBlocks, kT, 0, h->stream>>>(h->fbuf, out, s.N);
  return KKS_OK;
}

#define XF(expr)                        \
  do {                                  \
    const int _rc = (expr);             \
    if (_rc != KKS_OK) return _rc;      \
  } while (0)

// Shared front part of the forward and the backward pass: drive, fluxes and
// the spectra of eta, drive, X, flux_x, flux_y.
//   fields: 0 eta^2 / tr, 1 gx, 2 gy, 3 drive, 4 fx, 5 fy
//   spectra: 0 FT eta, 1 FT drive, 2 FT X, 3 FT fx, 4 FT fy, 5 scratch
int front(kks_adj* h, const double* in, const Coef& c) {
  const Spec& s = h->s;
  cudaStream_t st = h->stream;
  const double* e = in;
  const double* X = in + s.N;
  const double* ca = in + 2 * (size_t)s.N;
  const double* ct = in + 3 * (size_t)s.N;
  k_square<<<kBlocks, kT, 0, st>>>(e, fld(h, 0), s.N);
  XF(r2c(h, fld(h, 0), spc(h, 5)));
  k_spec_mul<<<kBlocks, kT, 0, st>>>(spc(h, 5), spc(h, 5), s, h->kx, h->ky, M_TR, c.epsX * s.c3n, 0.0);
  XF(c2r(h, spc(h, 5), fld(h, 0)));  // tr eps
  XF(r2c(h, e, spc(h, 0)));
  k_spec_mul<<<kBlocks, kT, 0, st>>>(spc(h, 0), spc(h, 5), s, h->kx, h->ky, M_DX, 1.0, 0.0);
  XF(c2r(h, spc(h, 5), fld(h, 1)));
  k_spec_mul<<<kBlocks, kT, 0, st>>>(spc(h, 0), spc(h, 5), s, h->kx, h->ky, M_DY, 1.0, 0.0);
  XF(c2r(h, spc(h, 5), fld(h, 2)));
  k_fwd_pointwise<<<kBlocks, kT, 0, st>>>(e, ca, ct, fld(h, 0), fld(h, 1), fld(h, 2), fld(h, 3), fld(h, 4), fld(h, 5),
                                          s, c);
  XF(r2c(h, fld(h, 3), spc(h, 1)));
  XF(r2c(h, X, spc(h, 2)));
  XF(r2c(h, fld(h, 4), spc(h, 3)));
  XF(r2c(h, fld(h, 5), spc(h, 4)));
  ACK(cudaGetLastError());
  return KKS_OK;
}

}  // namespace

extern "C" {

int kks_adj_create(int32_t nx, int32_t ny, double C11_0, double C12_0, double C44_0, int device, kks_adj** out) {
  if (!out || nx < 2 || ny < 2 || !(C44_0 > 0)) return kks_set_error(KKS_ERR_ARG, "bad argument");
  *out = nullptr;
  ACK(cudaSetDevice(device));
  kks_adj* h = new (std::nothrow) kks_adj();
  if (!h) return kks_set_error(KKS_ERR_ARG, "out of host memory");
  h->device = device;
  Spec& s = h->s;
  s.nx = nx; s.ny = ny; s.nyh = ny / 2 + 1; s.N = nx * ny; s.NC = nx * s.nyh;
  s.invN = 1.0 / (double)s.N;
  s.cc = C11_0 + 2 * C12_0;
  s.c3n = s.cc / C44_0;
  s.c11 = C11_0 / C44_0;
  s.c12 = C12_0 / C44_0;
  auto fail = [&](int rc) { kks_adj_destroy(h); return rc; };
  if (cudaStreamCreateWithFlags(&h->own, cudaStreamNonBlocking) != cudaSuccess)
    return fail(kks_set_error(KKS_ERR_CUDA, "stream"));
  h->stream = h->own;
  std::vector<double> kx, ky;
  wave_numbers(nx, kx, nx);
  wave_numbers(ny, ky, s.nyh);
  if (cudaMalloc(&h->kx, nx * sizeof(double)) != cudaSuccess || cudaMalloc(&h->ky, s.nyh * sizeof(double)) != cudaSuccess ||
      cudaMalloc(&h->f, (size_t)kFields * s.N * sizeof(double)) != cudaSuccess ||
      cudaMalloc(&h->z, (size_t)kSpectra * s.NC * sizeof(double2)) != cudaSuccess ||
      cudaMalloc(&h->partials, (size_t)kBlocks * kNS * sizeof(double)) != cudaSuccess ||
      cudaMalloc(&h->sums, kNS * sizeof(double)) != cudaSuccess ||
      cudaMallocHost(&h->h_sums, kNS * sizeof(double)) != cudaSuccess)
    return fail(kks_set_error(KKS_ERR_CUDA, "allocation"));
  cudaMemcpy(h->kx, kx.data(), nx * sizeof(double), cudaMemcpyHostToDevice);
  cudaMemcpy(h->ky, ky.data(), s.nyh * sizeof(double), cudaMemcpyHostToDevice);
  cudaMemset(h->partials, 0, (size_t)kBlocks * kNS * sizeof(double));
  if (cufftPlan2d(&h->r2c, nx, ny, CUFFT_D2Z) != CUFFT_SUCCESS || cufftPlan2d(&h->c2r, nx, ny, CUFFT_Z2D) != CUFFT_SUCCESS ||
      cufftSetStream(h->r2c, h->stream) != CUFFT_SUCCESS || cufftSetStream(h->c2r, h->stream) != CUFFT_SUCCESS)
    return fail(kks_set_error(KKS_ERR_CUFFT, "plans"));
  if (cudaDeviceSynchronize() != cudaSuccess) return fail(kks_set_error(KKS_ERR_CUDA, "set-up"));
  *out = h;
  return KKS_OK;
}

int kks_adj_forward(kks_adj* h, const double* state_in, const double* coef, double* state_out) {
  if (!h || !state_in || !coef || !state_out) return kks_set_error(KKS_ERR_ARG, "null argument");
  ACK(cudaSetDevice(h->device));
  const Spec& s = h->s;
  const Coef c = coef_of(coef);
  cudaStream_t st = h->stream;
  int rc = front(h, state_in, c);
  if (rc != KKS_OK) return rc;
  k_spec_update<<<kBlocks, kT, 0, st>>>(spc(h, 0), spc(h, 1), spc(h, 2), spc(h, 3), spc(h, 4), spc(h, 6), spc(h, 7),
                                        s, h->kx, h->ky, c, h->mixed ? 2 : 0);
  double* eb = state_out;
  double* xb = state_out + s.N;
  if (h->mixed) {  // FP32 transforms of the increments, added to the FP64 state
    XF(c2r(h, spc(h, 6), fld(h, 6)));
    XF(c2r(h, spc(h, 7), fld(h, 7)));
    k_add<<<kBlocks, kT, 0, st>>>(state_in, fld(h, 6), eb, s.N);
    k_add<<<kBlocks, kT, 0, st>>>(state_in + s.N, fld(h, 7), xb, s.N);
  } else {
    XF(c2r(h, spc(h, 6), eb));
    XF(c2r(h, spc(h, 7), xb));
  }
  k_phase<<<kBlocks, kT, 0, st>>>(state_in + s.N, eb, state_out + 2 * (size_t)s.N, state_out + 3 * (size_t)s.N, s.N, c);
  ACK(cudaGetLastError());
  if (!h->bound) ACK(cudaStreamSynchronize(st));
  return KKS_OK;
}

}  // extern "C"

// The backward pass up to the finished sums in h->sums (on h->stream).
static int backward_sums(kks_adj* h, const double* state_in, const double* state_out, const Coef& c,
                         const double* lam_out, double* lam_in) {
  const Spec& s = h->s;
  cudaStream_t st = h->stream;
  const size_t N = s.N;
  int rc = front(h, state_in, c);  // fields 0 tr, 1 gx, 2 gy, 3 drive, 4 fx, 5 fy; spectra 0-4
  if (rc != KKS_OK) return rc;
  // laplacian of eta_b and S + laplacian X_b from the same spectra
  k_spec_update<<<kBlocks, kT, 0, st>>>(spc(h, 0), spc(h, 1), spc(h, 2), spc(h, 3), spc(h, 4), spc(h, 6), spc(h, 7),
                                        s, h->kx, h->ky, c, 1);
  XF(c2r(h, spc(h, 6), fld(h, 6)));   // lap eta_b
  XF(c2r(h, spc(h, 7), fld(h, 7)));   // S + lap X_b
  // phase compositions
  k_back_phase<<<kBlocks, kT, 0, st>>>(state_in + N, state_out, state_out + 2 * N, lam_out, lam_out + 2 * N,
                                       lam_out + 3 * N, fld(h, 8), fld(h, 9), s.N, c, h->partials);
  // mu_eta = A_eta[lambda eta_b], mu_X = A_X[lambda X_b]
  XF(r2c(h, fld(h, 8), spc(h, 5)));
  k_spec_mul<<<kBlocks, kT, 0, st>>>(spc(h, 5), spc(h, 5), s, h->kx, h->ky, h->mixed ? M_AETA_INC : M_AETA,
                                     c.dt * c.Ls, c.kappa2);
  XF(c2r(h, spc(h, 5), fld(h, 10)));  // mu_eta (mixed: its increment over the cotangent)
  if (h->mixed) k_add<<<kBlocks, kT, 0, st>>>(fld(h, 8), fld(h, 10), fld(h, 10), s.N);
  XF(r2c(h, (lam_out + N), spc(h, 5)));
  k_spec_mul<<<kBlocks, kT, 0, st>>>(spc(h, 5), spc(h, 5), s, h->kx, h->ky, h->mixed ? M_AX_INC : M_AX,
                                     c.dt * c.Ds, 0.0);
  XF(c2r(h, spc(h, 5), fld(h, 11)));  // mu_X (mixed: its increment over the cotangent)
  if (h->mixed) k_add<<<kBlocks, kT, 0, st>>>(lam_out + N, fld(h, 11), fld(h, 11), s.N);
  // lambda flux_a = -dt D_s d_a mu_X
  XF(r2c(h, fld(h, 11), spc(h, 5)));
  k_spec_mul<<<kBlocks, kT, 0, st>>>(spc(h, 5), spc(h, 6), s, h->kx, h->ky, M_DX, -c.dt * c.Ds, 0.0);
  XF(c2r(h, spc(h, 6), fld(h, 12)));
  k_spec_mul<<<kBlocks, kT, 0, st>>>(spc(h, 5), spc(h, 6), s, h->kx, h->ky, M_DY, -c.dt * c.Ds, 0.0);
  XF(c2r(h, spc(h, 6), fld(h, 13)));
  // main pointwise back pass
  double* lam_e = lam_in;
  double* lam_x = lam_in + N;
  k_back_main<<<kBlocks, kT, 0, st>>>(state_in, state_in + 2 * N, state_in + 3 * N, fld(h, 0), fld(h, 1), fld(h, 2),
                                      fld(h, 3), fld(h, 10), fld(h, 11), fld(h, 12), fld(h, 13), fld(h, 6), fld(h, 7),
                                      fld(h, 14), fld(h, 15), fld(h, 16), fld(h, 17), lam_in + 2 * N, lam_in + 3 * N, s,
                                      c, h->partials);
  // lambda of eta^2 = epsX c3n T[lambda tr]; divergence of lambda g
  XF(r2c(h, fld(h, 14), spc(h, 5)));
  k_spec_mul<<<kBlocks, kT, 0, st>>>(spc(h, 5), spc(h, 5), s, h->kx, h->ky, M_TR, c.epsX * s.c3n, 0.0);
  XF(c2r(h, spc(h, 5), fld(h, 18)));
  XF(r2c(h, fld(h, 15), spc(h, 5)));
  XF(r2c(h, fld(h, 16), spc(h, 6)));
  k_spec_div<<<kBlocks, kT, 0, st>>>(spc(h, 5), spc(h, 6), spc(h, 7), s, h->kx, h->ky);
  XF(c2r(h, spc(h, 7), fld(h, 19)));
  k_back_final<<<kBlocks, kT, 0, st>>>(state_in, fld(h, 17), fld(h, 18), fld(h, 19), fld(h, 11), fld(h, 9), lam_e,
                                       lam_x, s.N);
  k_finish<<<1, 32, 0, st>>>(h->partials, kBlocks, h->sums);
  ACK(cudaGetLastError());
  return KKS_OK;
}

extern "C" {

int kks_adj_backward(kks_adj* h, const double* state_in, const double* state_out, const double* coef,
                     const double* lam_out, double* lam_in, double* dcoef) {
  if (!h || !state_in || !state_out || !coef || !lam_out || !lam_in || !dcoef)
    return kks_set_error(KKS_ERR_ARG, "null argument");
  ACK(cudaSetDevice(h->device));
  const Coef c = coef_of(coef);
  int rc = backward_sums(h, state_in, state_out, c, lam_out, lam_in);
  if (rc != KKS_OK) return rc;
  ACK(cudaMemcpyAsync(h->h_sums, h->sums, kNS * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  ACK(cudaStreamSynchronize(h->stream));
  dcoef_of(h->h_sums, c, dcoef);
  return KKS_OK;
}

int kks_adj_backward_device(kks_adj* h, const double* state_in, const double* state_out, const double* coef,
                            const double* lam_out, double* lam_in, double* dcoef_device) {
  if (!h || !state_in || !state_out || !coef || !lam_out || !lam_in || !dcoef_device)
    return kks_set_error(KKS_ERR_ARG, "null argument");
  ACK(cudaSetDevice(h->device));
  const Coef c = coef_of(coef);
  int rc = backward_sums(h, state_in, state_out, c, lam_out, lam_in);
  if (rc != KKS_OK) return rc;
  k_dcoef<<<1, 32, 0, h->stream>>>(h->sums, c, dcoef_device);
  ACK(cudaGetLastError());
  if (!h->bound) ACK(cudaStreamSynchronize(h->stream));
  return KKS_OK;
}

int kks_adj_set_stream(kks_adj* h, void* stream) {
  if (!h) return kks_set_error(KKS_ERR_ARG, "null handle");
  ACK(cudaSetDevice(h->device));
  cudaStream_t want = stream ? (cudaStream_t)stream : h->own;
  if (want == h->stream) {
    h->bound = stream != nullptr;
    return KKS_OK;
  }
  // work already queued on the old stream comes before anything on the new one
  ACK(cudaStreamSynchronize(h->stream));
  h->stream = want;
  h->bound = stream != nullptr;
  for (cufftHandle p : {h->r2c, h->c2r, h->r2c32, h->c2r32})
    if (p && cufftSetStream(p, h->stream) != CUFFT_SUCCESS) return kks_set_error(KKS_ERR_CUFFT, "plan stream");
  return KKS_OK;
}

int kks_adj_set_precision(kks_adj* h, int precision) {
  if (!h || (precision != KKS_PRECISION_FP64 && precision != KKS_PRECISION_MIXED))
    return kks_set_error(KKS_ERR_ARG, "precision must be KKS_PRECISION_FP64 or KKS_PRECISION_MIXED");
  ACK(cudaSetDevice(h->device));
  ACK(cudaStreamSynchronize(h->stream));
  if (precision == KKS_PRECISION_MIXED && !h->r2c32) {
    const Spec& s = h->s;
    ACK(cudaMalloc(&h->fbuf, (size_t)s.N * sizeof(float)));
    ACK(cudaMalloc(&h->zbuf, (size_t)2 * s.NC * sizeof(float)));
    cufftHandle a = 0, b = 0;
    if (cufftPlan2d(&a, s.nx, s.ny, CUFFT_R2C) != CUFFT_SUCCESS) return kks_set_error(KKS_ERR_CUFFT, "FP32 plans");
    h->r2c32 = a;
    if (cufftPlan2d(&b, s.nx, s.ny, CUFFT_C2R) != CUFFT_SUCCESS) return kks_set_error(KKS_ERR_CUFFT, "FP32 plans");
    h->c2r32 = b;
    AFK(cufftSetStream(h->r2c32, h->stream));
    AFK(cufftSetStream(h->c2r32, h->stream));
  }
  h->mixed = precision == KKS_PRECISION_MIXED;
  return KKS_OK;
}

int kks_adj_destroy(kks_adj* h) {
  if (!h) return KKS_OK;
  cudaSetDevice(h->device);
  if (h->r2c) cufftDestroy(h->r2c);
  if (h->c2r) cufftDestroy(h->c2r);
  if (h->r2c32) cufftDestroy(h->r2c32);
  if (h->c2r32) cufftDestroy(h->c2r32);
  cudaFree(h->fbuf);
  cudaFree(h->zbuf);
  cudaFree(h->kx);
  cudaFree(h->ky);
  cudaFree(h->f);
  cudaFree(h->z);
  cudaFree(h->partials);
  cudaFree(h->sums);
  if (h->h_sums) cudaFreeHost(h->h_sums);
  if (h->bound && h->stream) cudaStreamSynchronize(h->stream);
  if (h->own) cudaStreamDestroy(h->own);
  delete h;
  return KKS_OK;
}

}  // extern "C"
