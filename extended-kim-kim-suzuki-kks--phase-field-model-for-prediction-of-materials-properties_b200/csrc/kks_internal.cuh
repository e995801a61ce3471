// kks_internal.cuh - device-side state shared by the scalar kernels
// (kks_scalar.cu), the field kernels (kks_fields.cu) and the host runtime
// (kks_abi.cu).
//
// Layout in HBM of one cell (Np = nx*ny rounded up to 64 elements,
// NCp = nx*(ny/2+1) rounded up to 32; R = double on the FP64 path, float on
// the mixed path):
//
// FP64 path (the reference's formulation: new fields are inverse transforms of
// the updated spectra)
//   state[p], p = 0, 1 : double[5*Np]  eta | X | eta^2 | X_al | X_th
//       (eta | X | eta^2 is the batch-3 R2C input; the batch-2 C2R writes the
//        candidate eta_b | X_b straight into state[1-p])
// mixed path (increment formulation: the FP32 transforms only carry the
// step's increments, the state itself is kept in FP64)
//   state[p]           : double eta[Np] | double X[Np] | float X_al[Np] | float X_th[Np]
//   fft_in             : float[3*Np]   eta | X | eta^2 (batch-3 R2C input)
//   the batch-2 C2R writes d_eta | d_X into real_c
// both paths
//   spec_a             : C[3*NCp]  FT(eta) | FT(X) | FT(eta^2)
//   real_b             : R[3*Np]   tr eps | d_x eta | d_y eta
//   real_c             : R[3*Np]   drive | flux_x | flux_y   (mixed: then d_eta | d_X)
//   spec_bcd           : C[5*NCp]  slots 0-2: B spectra, then C spectra; slots 3-4: D spectra
//   eta_m, X_m         : S[Np]     residual pair "minus" entry (S = double on both paths)
//   mu, g[3]           : R[Np]     diffusion potential, free-energy buffers rotated by index
//   partials           : double[nblocks * KKS_NPART] block sums of the reductions
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "kks.h"

#define KKS_NPART 32
// slots of the partial sums (every field kernel is launched with the same grid)
enum {
  // spectral_mid: Parseval sums of the elastic energy, weight w = 1 or 2 per
  // half-spectrum bin, p = w |FT(eta^2)|^2, O = strain multipliers
  P2_OXX2 = 0,   // sum p Oxx^2
  P2_OYY2,       // sum p Oyy^2
  P2_OXXYY,      // sum p Oxx Oyy
  P2_OXY2,       // sum p Oxy^2
  P2_OTR,        // sum p (Oxx + Oyy)
  P2_P,          // sum p
  // pre_pointwise (old state)
  P3_G,          // sum G_s
  P3_ETA,        // sum eta
  P3_XLO,        // sum X[eta < 0.05]
  P3_NLO,        // count eta < 0.05
  P3_XHI,        // sum X[eta > 0.95]
  P3_NHI,        // count eta > 0.95
  P3_IFACE,      // interface cells of eta (surface steps)
  // post_pointwise (new state)
  P5_GRAD2,      // sum (d_x eta_b)^2 + (d_y eta_b)^2 (np.gradient stencil)
  P5_XLO,        // sum X_b[eta_b < 0.05]
  P5_NLO,
  P5_XHI,        // sum X_b[eta_b > 0.95]
  P5_NHI,
  P5_ETA,        // sum eta_b
  P5_IFACE,      // interface cells of eta_b (surface steps)
  P5_DIFF,       // sum dX/dt * mu_mean
  P5_AC,         // sum (1/L) (deta/dt)^2
  P5_TEMP,       // sum (G+ - G-)/dt
  P5_COMB,       // sum (-diff + ac - temp)
  P_COUNT
};
static_assert(P_COUNT <= KKS_NPART, "partials slots");

// Loop state of the cell (the scalar variables of pf_kks/solver.py:118-175),
// read and written only by the single-thread prologue and decide kernels.
struct KksCtl {
  int32_t istep, iteration, flag, good_step, status, target_step;
  int32_t minus_is_state, gm, gs, gb, restore, surf_valid, surf_b_valid, T_b_valid;
  int32_t error_istep, error_iteration;
  long long attempts, n_rec, n_row;
  double t, t_s, t_b, ttime, Xv, dtime_s, D_0, Meta_0;
  double surf, surf_b, T_b;
  double E_prev, ts_prev, ed_sum, ed_comp;
  int32_t ed_n;
  int32_t parity;  // state buffer of the next attempt's input (flipped by every attempt that runs)
  double error_dtime_s;
  // residual terms of the last attempt of the current step (history row)
  double res[5];
  int32_t res_valid, pad1;
};

// Per-attempt coefficients, written by the prologue, read by every field kernel.
struct KksPar {
  int32_t active, istep, iteration, surface;
  int32_t armed_write, armed_residual, minus_is_state, gm, gs, gb;
  int32_t parity;  // state buffer of this attempt's input
  int32_t pad_par;
  double T, D, Meta, L, Vm;
  double dt, L_s, kappa2_s, D_s, w_s;
  double A_alp_s, B_alp_s, C_alp_s, A_thet_s, B_thet_s, C_thet_s;
  double A_alp, B_alp, A_thet, B_thet;
  double C44, epsX;
  // derived
  double inv_C44;
  double pc_shift;   // (B_alp - B_thet) / (2 A_thet)
  double pc_ratio;   // A_alp / A_thet
  double ac_mul;     // -dtime_s * L_s
  double ac_den;     // dtime_s * L_s * kappa2_s
  double ch_mul;     // dtime_s * D_s
  double inv_dt, inv_Ls;
  // vertex forms of the two parabolas, for the FP32 path: f = A (c - v)^2 + f0
  double va, fa0, vt, ft0;
};

// Run constants in device memory.
struct KksConst {
  kks_params p;
  int32_t nx, ny, nyh, N, NC, Np, NCp, n_steps;
  double dtime_s_min;
  double inv_N;
  // frozen stiffness at T0 (pf_kks/solver.py:152-154), and normalised by C44(T0)
  double c11, c12, c3;   // C11/C44_0, C12/C44_0, (C11 + 2 C12)/C44_0
  double C11_0, C12_0, C44_0;
  int32_t mixed;
  int32_t pad;
};

// ---------------------------------------------------------------------------
// launchers (kks_scalar.cu)
void kks_launch_prologue(const KksConst* c, KksCtl* ctl, KksPar* par, const uint8_t* step_flags, kks_record* ring,
                         long long ring_cap, cudaStream_t s);
void kks_launch_decide(const KksConst* c, KksCtl* ctl, const KksPar* par, const double* partials, int nblocks,
                       kks_record* ring, long long ring_cap, kks_step_row* rows, long long row_cap, cudaStream_t s);

// Device buffers of one cell (typed per path in kks_fields.cu).
struct KksFieldPtrs {
  void* eta[2];
  void* X[2];
  void* X_al[2];
  void* X_th[2];
  void* fft_in[2];  // batch-3 R2C input (eta | X | eta^2) for an attempt of parity p
  void* fft_out[2]; // batch-2 C2R output for an attempt of parity p
  void* spec_a;
  void* real_b;
  void* real_c;
  void* spec_bcd;
  void* eta_m;
  void* X_m;
  void* mu;
  void* g[3];
  double* partials;
  const double* kx;
  const double* ky;
};

int kks_field_blocks(int N, int num_sms);

// Field kernels of one attempt. MIXED selects the FP32 increment path.
template <bool MIXED>
void kks_launch_prep(const KksConst* hc, const KksPar* par, const KksFieldPtrs& f, int parity, int nblocks,
                     cudaStream_t s);
template <bool MIXED>
void kks_launch_spectral_mid(const KksConst* hc, const KksConst* dc, const KksPar* par, const KksFieldPtrs& f,
                             int nblocks, cudaStream_t s);
template <bool MIXED>
void kks_launch_pre_pointwise(const KksConst* hc, const KksConst* dc, const KksPar* par, const KksFieldPtrs& f,
                              int parity, int nblocks, cudaStream_t s);
template <bool MIXED>
void kks_launch_spectral_update(const KksConst* hc, const KksConst* dc, const KksPar* par, const KksFieldPtrs& f,
                                int nblocks, cudaStream_t s);
template <bool MIXED>
void kks_launch_post_pointwise(const KksConst* hc, const KksConst* dc, const KksPar* par, const KksFieldPtrs& f,
                               int parity, int nblocks, cudaStream_t s);
template <bool MIXED>
void kks_launch_restore(const KksConst* hc, const KksConst* dc, const KksCtl* ctl, const KksFieldPtrs& f,
                        int parity, int nblocks, cudaStream_t s);
// elastic fields of the state of parity p (pf_kks/elasticity.py:107-163): the
// three strain spectra into spec_bcd slots 0-2 (then C2R into real_b), and the
// stress / elastic strain components xx, yy, zz, xy.
template <bool MIXED>
void kks_launch_strain_spectra(const KksConst* hc, const KksConst* dc, const KksPar* par, const KksFieldPtrs& f,
                               int nblocks, cudaStream_t s);
template <bool MIXED>
void kks_launch_elastic_out(const KksConst* hc, const KksConst* dc, const KksPar* par, const KksFieldPtrs& f,
                            int parity, double* sig4, double* eps4, int nblocks, cudaStream_t s);
template <typename R>
void kks_launch_to_real(const double* src, R* dst, int n, cudaStream_t s);
template <typename R>
void kks_launch_to_double(const R* src, double* dst, int n, cudaStream_t s);

// Initial state on the device (kks_init.cu). Selection buffers: cnt holds
// kks_init_chunks(N) counts, off kks_init_chunks(N) + 1 offsets (off[last] =
// total). parts holds n * kks_init_particle_bytes().
int kks_init_chunks(int N);
size_t kks_init_particle_bytes();
void kks_init_labels(const double* seeds, int ns, int nx, int ny, int32_t* labels, cudaStream_t s);
void kks_init_count_edges(const int32_t* labels, int nx, int ny, long long* cnt, long long* off, cudaStream_t s);
void kks_init_count_below(const double* eta, double thr, int N, long long* cnt, long long* off, cudaStream_t s);
void kks_init_select_edges(const int32_t* labels, int nx, int ny, const long long* off, const long long* ranks,
                           int n, long long* flat, cudaStream_t s);
void kks_init_select_below(const double* eta, double thr, int N, const long long* off, const long long* ranks, int n,
                           long long* flat, cudaStream_t s);
void kks_init_eta(const long long* flat, int n, int nx, int ny, const double* jitter, const double* radii, double w,
                  void* parts, double* eta, cudaStream_t s);
template <typename R>
void kks_init_fields(int N, const uint64_t state[2], const uint64_t inc[2], double x_matrix, double low, double range,
                     double x_particle, double pc_shift, double pc_ratio, const double* eta, double* X, R* X_al,
                     R* X_th, cudaStream_t s);
template <typename R>
void kks_init_place(bool add, int nx, int ny, double dx, double dy, const double* prm, int n, double x_matrix,
                    double x_precipitate, double* eta, double* X, R* X_mat, R* X_pre, cudaStream_t s);
void kks_init_set_eta(const long long* flat, int n, double value, double* eta, cudaStream_t s);
