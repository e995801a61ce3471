// kks_scalar.cu - the scalar part of an attempt, on the device.
//
// Two small stages bracket the field kernels of every attempt:
//
//  * kks_prologue (one warp: the table interpolations in parallel, the rest on
//    one thread): temperature from the heat-treatment schedule, vacancy
//    model, Si diffusivity, interface mobility, Allen-Cahn coefficient, table
//    interpolation and the dimensionless parameter set
//    (pf_kks/solver.py:179-240, pf_kks/kinetics.py:9-107, pf_kks/materials.py:57-59);
//  * kks_decide (one block finishes the block reductions, then one thread):
//    forms the total energy and the energy residual, and takes the reject /
//    accept / enlarge decision and the end-of-step bookkeeping
//    (pf_kks/solver.py:270-404, pf_kks/residual.py:26-66).
//
// This file is compiled with -fmad=false: every scalar expression is evaluated
// with the same operation order and roundings as the reference's float64
// Python, so the scalars (and the log lines printed from them) follow the
// reference; only the libm-level exp may differ by an ulp.

#include <math.h>

#include "kks_internal.cuh"
#include "kks_fft.cuh"

namespace {

// Constants of pf_kks/constants.py:6-21.
__device__ const double kR = 8.314472;
__device__ const double kHF1VA = 63680;
__device__ const double kSF1VA = 2.49;
__device__ const double kHB = 10613;
__device__ const double kSB_KB = 42453;
__device__ const double kZ = 12;
__device__ const double kD0_AL = 1.7e-4;
__device__ const double kQ_AL = 142e3;
__device__ const double kD0_SI = 3.66e-6;
__device__ const double kQ_SI = 110958;

// np.interp for a scalar abscissa (numpy's arr_interp: binary search, slope
// times offset plus left value, end values outside the table).
__device__ double interp(double x, const double* xp, const double* fp, int n) {
  if (n == 1) return fp[0];
  if (x < xp[0]) return fp[0];
  if (x > xp[n - 1]) return fp[n - 1];
  if (x == xp[n - 1]) return fp[n - 1];
  int lo = 0, hi = n - 1;  // xp[lo] <= x < xp[hi]
  while (hi - lo > 1) {
    int mid = (lo + hi) >> 1;
    if (x >= xp[mid]) lo = mid; else hi = mid;
  }
  if (xp[lo] == x) return fp[lo];
  double slope = (fp[lo + 1] - fp[lo]) / (xp[lo + 1] - xp[lo]);
  double r = slope * (x - xp[lo]) + fp[lo];
  if (isnan(r)) {
    r = slope * (x - xp[lo + 1]) + fp[lo + 1];
    if (isnan(r) && fp[lo] == fp[lo + 1]) r = fp[lo];
  }
  return r;
}

__device__ double tab(const kks_params& p, int k, double T) {
  return interp(T, p.table_T, p.table[k], p.n_table);
}

// pf_kks/kinetics.py:9-14
__device__ double equilibrium_vacancy_fraction(double T) {
  return exp(-(kHF1VA - T * kSF1VA) / (kR * T)) *
         (1 - kZ * 0.01 + kZ * 0.01 * exp((kHB - T * kSB_KB) / (kR * T)));
}

// pf_kks/kinetics.py:24-38
__device__ double si_diffusivity(double T, double Xv, double Xve, double D0, double QD, double cap) {
  double factor = fabs(1 + (Xv - Xve) / Xve);
  double D;
  if (factor > cap) D = cap * D0 * exp(-QD / (kR * T));
  else D = factor * D0 * exp(-QD / (kR * T));
  if (factor < 1) D = D0 * exp(-QD / (kR * T));
  return D;
}

// pf_kks/kinetics.py:41-45
__device__ double effective_vacancy_diffusivity(double T, double Xv, double Xve) {
  double D_Al = kD0_AL * exp(-kQ_AL / (kR * T));
  double D_Si = kD0_SI * exp(-kQ_SI / (kR * T));
  return fabs(1 + (Xv - Xve) / Xve) * (0.03 * D_Si + 0.97 * D_Al);
}

// Copy a read-only struct into shared memory with all threads of the block
// (independent 8-byte loads), so that the single-thread chains below read it
// at shared-memory latency instead of one L2 round trip per cache line.
template <typename T>
__device__ __forceinline__ void stage_struct(T* dst, const T* src) {
  static_assert(sizeof(T) % 8 == 0 && alignof(T) >= 8, "8-byte words");
  const long long* s = reinterpret_cast<const long long*>(src);
  long long* d = reinterpret_cast<long long*>(dst);
  // eight loads in flight per thread: the one-warp prologue copies the ~5 KB
  // run constants in three rounds of L2 latency instead of twenty
  constexpr int n = (int)(sizeof(T) / 8), U = 8;
  for (int i0 = threadIdx.x; i0 < n; i0 += U * blockDim.x) {
    long long v[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int i = i0 + u * blockDim.x;
      if (i < n) v[u] = s[i];
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int i = i0 + u * blockDim.x;
      if (i < n) d[i] = v[u];
    }
  }
}

__device__ void push_record(KksCtl* ctl, kks_record* ring, long long cap, const kks_record& r) {
  ring[ctl->n_rec % cap] = r;
  ctl->n_rec += 1;
}

// An attempt that runs takes KksCtl::parity as its input buffer and flips it,
// so the device always knows which buffer holds the current state (attempts
// that do not run, after the target step or a stop, leave it alone).
__device__ __forceinline__ void prologue_body(const KksConst* __restrict__ c, KksCtl* ctl, KksPar* par,
                                              const uint8_t* __restrict__ step_flags, kks_record* ring,
                                              long long ring_cap) {
  // one warp: lane 0 runs the scalar chain; the material tables are
  // interpolated at T by one lane each (same expressions, same roundings)
  __shared__ int s_go;
  __shared__ double s_T, s_tab[KKS_NTAB];
  __shared__ KksConst sc;
  stage_struct(&sc, c);
  __syncwarp();
  c = &sc;
  const kks_params& p = sc.p;
  const int lane = threadIdx.x;
  if (lane == 0) {
    s_go = ctl->status == KKS_STATUS_OK && ctl->istep < ctl->target_step;
    if (!s_go) par->active = 0;
    else s_T = interp(ctl->t, p.sched_time, p.sched_temp, p.n_sched);
  }
  __syncwarp();
  if (!s_go) return;
  if (lane < KKS_NTAB) s_tab[lane] = tab(p, lane, s_T);
  __syncwarp();
  if (lane != 0) return;
  const int istep = ctl->istep;
  const double T = s_T;
  const int surface = step_flags[istep] & 1;

  double Xv = ctl->Xv;
  const double Xve = equilibrium_vacancy_fraction(T);
  const double D = si_diffusivity(T, Xv, Xve, p.D0, p.QD, p.diffusion_enhancement_cap);
  const double Meta = p.Meta0 * exp(-p.QMeta / (kR * T));
  const double Deff = effective_vacancy_diffusivity(T, Xv, Xve);
  if (istep == 0) {
    ctl->D_0 = D;
    ctl->Meta_0 = Meta;
    ctl->dtime_s = p.dtime_s;
  }
  double dtime_s = ctl->dtime_s;
  if (dtime_s > p.dtime_max) dtime_s = p.dtime_max;
  if (dtime_s < c->dtime_s_min) dtime_s = c->dtime_s_min;
  ctl->dtime_s = dtime_s;
  const double D_0 = ctl->D_0;
  const double Meta_0 = ctl->Meta_0;
  const double dx2 = p.dx * p.dx;
  const double dtime = (dx2 / D_0) * p.dtime_s;  // ttime and Xv use the initial step (quirk of the reference)
  ctl->ttime = ctl->ttime + dtime;
  {
    double dXv = (1 - exp(-dtime * (Deff / p.Lv2))) * (Xve - Xv);
    ctl->Xv = Xv + dXv;
  }

  const double A_alp = s_tab[KKS_TAB_A_ALP];
  const double B_alp = s_tab[KKS_TAB_B_ALP];
  const double C_alp = s_tab[KKS_TAB_C_ALP];
  const double C44 = s_tab[KKS_TAB_C44];
  const double A_thet = s_tab[KKS_TAB_A_THET];
  const double B_thet = s_tab[KKS_TAB_B_THET];
  const double C_thet = s_tab[KKS_TAB_C_THET];
  const double sigma = s_tab[KKS_TAB_GAMMA];
  const double Omega0 = s_tab[KKS_TAB_VM];
  const double epsX = s_tab[KKS_TAB_EPSX];
  const double X_Si_fcc = s_tab[KKS_TAB_X_SI_FCC];

  // pf_kks/kinetics.py:60-80
  const double kappa2 = 2 * p.lambd * sigma * 3 / p.alpha;
  const double w = (sigma * 3 * p.alpha) / p.lambd;
  const double kappa = sqrt(kappa2);
  const double xi = (19.0 / 30.0) * (1 / Omega0) * 2 * A_alp * ((X_Si_fcc - 0.9999) * (X_Si_fcc - 0.9999));
  const double L = (sigma / (kappa * kappa)) * (1 / (1 / Meta + kappa * xi / (D * sqrt(2 * w)))) * 0.01;

  if (istep % 100 == 0) {
    kks_record r;
    r.kind = KKS_REC_STATE;
    r.istep = istep;
    r.iteration = ctl->iteration;
    r.good_step = ctl->flag ? ctl->good_step : -1;
    r.T = T; r.D = D; r.L = L; r.Meta = Meta; r.Vm = Omega0; r.dtime_s = dtime_s;
    r.res_total = r.res_energy_derivative = r.res_diffusion = r.res_allen_cahn = r.res_temperature = 0;
    r.energy_s = 0;
    push_record(ctl, ring, ring_cap, r);
  }

  // pf_kks/kinetics.py:83-107 (normalize)
  KksPar q;
  q.active = 1;
  q.istep = istep;
  q.iteration = ctl->iteration;
  q.surface = surface;
  q.armed_write = ctl->flag == 1;
  q.armed_residual = (ctl->flag == 1) && (istep >= ctl->good_step + 2);
  q.minus_is_state = ctl->minus_is_state;
  q.gm = ctl->gm;
  q.gs = ctl->gs;
  q.gb = ctl->gb;
  q.parity = ctl->parity;
  q.pad_par = 0;
  ctl->parity = q.parity ^ 1;
  q.T = T; q.D = D; q.Meta = Meta; q.L = L; q.Vm = Omega0;
  q.dt = dtime_s;
  q.L_s = (L * C44 * dx2) / D_0;
  const double kappa2_norm = 2 * p.lambd * sigma * 3 / p.alpha;
  const double w_norm = (sigma * 3 * p.alpha) / p.lambd;
  q.kappa2_s = kappa2_norm / (C44 * dx2);
  q.D_s = D / D_0;
  q.w_s = w_norm / (C44);
  q.A_thet_s = A_thet / (C44 * Omega0);
  q.B_thet_s = B_thet / (C44 * Omega0);
  q.C_thet_s = C_thet / (C44 * Omega0);
  q.A_alp_s = A_alp / (C44 * Omega0);
  q.B_alp_s = B_alp / (C44 * Omega0);
  q.C_alp_s = C_alp / (C44 * Omega0);
  (void)Meta_0;
  q.A_alp = A_alp; q.B_alp = B_alp; q.A_thet = A_thet; q.B_thet = B_thet;
  q.C44 = C44;
  q.epsX = epsX;
  q.inv_C44 = 1.0 / C44;
  q.pc_shift = (B_alp - B_thet) / (2 * A_thet);
  q.pc_ratio = A_alp / A_thet;
  q.ac_mul = -dtime_s * q.L_s;
  q.ac_den = dtime_s * q.L_s * q.kappa2_s;
  q.ch_mul = dtime_s * q.D_s;
  q.inv_dt = 1.0 / dtime_s;
  q.inv_Ls = 1 / q.L_s;
  q.va = -q.B_alp_s / (2 * q.A_alp_s);
  q.fa0 = q.C_alp_s - q.B_alp_s * q.B_alp_s / (4 * q.A_alp_s);
  q.vt = -q.B_thet_s / (2 * q.A_thet_s);
  q.ft0 = q.C_thet_s - q.B_thet_s * q.B_thet_s / (4 * q.A_thet_s);
  *par = q;
  ctl->attempts += 1;
}

__global__ void kks_prologue(const KksConst* __restrict__ c, KksCtl* ctl, KksPar* par,
                             const uint8_t* __restrict__ step_flags, kks_record* ring, long long ring_cap) {
  prologue_body(c, ctl, par, step_flags, ring, ring_cap);
}

// one warp per cell of a batch
__global__ void kks_prologue_batch(const KksCellDesc* __restrict__ cells) {
  const KksCellDesc& d = cells[blockIdx.x];
  prologue_body(d.dc, d.ctl, d.par, d.step_flags, d.ring, d.ring_cap);
}

// The partial sums of all blocks are finished in a fixed order (deterministic).
constexpr int kDecideWarps = 16;  // warps of the decide block (one row group each)
static_assert(KKS_NPART == 32, "one lane per partial-sum slot");

__device__ __forceinline__ void decide_body(const KksConst* __restrict__ c, KksCtl* ctl, const KksPar* __restrict__ par,
                                            const double* __restrict__ partials, int nblocks, kks_record* ring,
                                            long long ring_cap, kks_step_row* rows, long long row_cap) {
  __shared__ double S[P_COUNT];
  __shared__ double G[kDecideWarps][KKS_NPART + 1];
  __shared__ KksConst sc;
  __shared__ KksPar sp;
  if (!par->active) return;
  stage_struct(&sc, c);
  stage_struct(&sp, par);
  // warp w sums rows w, w + W, ...: lane k reads slot k, so a warp reads one
  // whole row per load, kU rows in flight; the W row groups are then added in
  // a fixed order
  {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    constexpr int kU = 8;
    double v = 0;
    for (int b0 = w; b0 < nblocks; b0 += kU * kDecideWarps) {
      double r[kU];
#pragma unroll
      for (int u = 0; u < kU; ++u) {
        const int b = b0 + u * kDecideWarps;
        r[u] = b < nblocks ? partials[(size_t)b * KKS_NPART + lane] : 0.0;
      }
#pragma unroll
      for (int u = 0; u < kU; ++u) v += r[u];
    }
    G[w][lane] = v;
    __syncthreads();
    if (threadIdx.x < P_COUNT) {
      double t = 0;
      for (int g = 0; g < kDecideWarps; ++g) t += G[g][threadIdx.x];
      S[threadIdx.x] = t;
    }
    __syncthreads();
  }
  if (threadIdx.x != 0) return;

  c = &sc;
  par = &sp;
  const kks_params& p = sc.p;
  const double Nd = (double)c->N;
  const int istep = par->istep;
  const int iteration = ctl->iteration;
  double dtime_s = ctl->dtime_s;

  // Elastic energy sum from Parseval's theorem: eps_ab^ = epsX c3 O_ab FT(eta^2)
  // and a = epsX eta^2, so every sum of products of eps_xx, eps_yy, eps_xy and a
  // is a weighted sum of |FT(eta^2)|^2 (sum_x f g = 1/N sum_k f^ conj(g^)).
  const double eX = par->epsX;
  const double A2 = (eX * c->c3) * (eX * c->c3) / Nd;
  const double Sxx = A2 * S[P2_OXX2], Syy = A2 * S[P2_OYY2], Sxxyy = A2 * S[P2_OXXYY], Sxy2 = A2 * S[P2_OXY2];
  const double Stra = eX * eX * c->c3 / Nd * S[P2_OTR];  // sum (eps_xx + eps_yy) a
  const double Saa = eX * eX / Nd * S[P2_P];             // sum a^2
  const double el_sum = 0.5 * (c->C11_0 * (Sxx + Syy - 2 * Stra + 3 * Saa) +
                               2 * c->C12_0 * (Sxxyy - 2 * Stra + 3 * Saa) + 4 * c->C44_0 * Sxy2);

  // total_energy (pf_kks/free_energy.py:98-110): both gradient components carry G and el
  const double energy_s = (S[P3_G] + el_sum / par->C44) * 2.0 + (0.5 * par->kappa2_s) * S[P5_GRAD2];
  if (par->surface) {  // interface measure of the step's input state (pf_kks/solver.py:180-181)
    ctl->surf = S[P3_IFACE] * p.surf_scale;
    ctl->surf_valid = 1;
  }

  if (iteration == p.max_iterations) {  // pf_kks/solver.py:292-295
    ctl->status = KKS_STATUS_MAX_ITER;
    ctl->error_istep = istep;
    ctl->error_iteration = iteration;
    ctl->error_dtime_s = dtime_s;
    return;
  }

  int outcome = 0;  // 0: no residual, 1: rejected, 2: accepted, 3: enlarged
  if (par->armed_residual) {
    // kks_residual (pf_kks/residual.py:26-66); energy derivative = running
    // mean over the completed steps since good_step
    const double ed = ctl->ed_sum / (double)ctl->ed_n;
    const double total = ed + S[P5_COMB];
    if (!isfinite(total)) {  // pf_kks/solver.py:312-313
      ctl->status = KKS_STATUS_NONFINITE;
      ctl->error_istep = istep;
      ctl->error_iteration = iteration;
      ctl->error_dtime_s = dtime_s;
      return;
    }
    ctl->res[0] = total;
    ctl->res[1] = ed;
    ctl->res[2] = S[P5_DIFF];
    ctl->res[3] = S[P5_AC];
    ctl->res[4] = S[P5_TEMP];
    ctl->res_valid = 1;
    kks_record r;
    r.istep = istep;
    r.iteration = iteration;
    r.good_step = ctl->good_step;
    r.T = par->T; r.D = par->D; r.L = par->L; r.Meta = par->Meta; r.Vm = par->Vm;
    r.res_total = total;
    r.res_energy_derivative = ed;
    r.res_diffusion = S[P5_DIFF];
    r.res_allen_cahn = S[P5_AC];
    r.res_temperature = S[P5_TEMP];
    r.energy_s = energy_s;
    if (fabs(total) > p.residual_max) {
      dtime_s /= p.step_factor;
      r.kind = KKS_REC_REJECTED;
      outcome = 1;
    } else if (fabs(total) > p.residual_min) {
      r.kind = KKS_REC_ACCEPTED;
      outcome = 2;
    } else {
      r.kind = KKS_REC_ENLARGED;
      outcome = 3;
    }
    r.dtime_s = dtime_s;
    push_record(ctl, ring, ring_cap, r);
    if (outcome == 3) dtime_s *= p.step_factor;
  }
  ctl->dtime_s = dtime_s;

  const int gm = par->gm, gs = par->gs, gb = par->gb;
  if (outcome == 1) {
    // The rejected attempt becomes the "minus" entry of the pair; the host
    // graph then restores the step's input state into the candidate buffer.
    ctl->iteration = iteration + 1;
    ctl->restore = 1;
    ctl->minus_is_state = 0;
    ctl->gm = gb;
    ctl->gs = gm;
    ctl->gb = gs;
    return;
  }

  // ---- end of step (pf_kks/solver.py:353-404)
  ctl->restore = 0;
  ctl->minus_is_state = 1;
  ctl->gm = gs;  // post-loop overwrite: the pair keeps the pre-update free energy
  ctl->gs = gm;
  ctl->gb = gb;

  const double dx2 = p.dx * p.dx;
  const double t = ctl->t;
  const double t_s = ctl->t_s + dtime_s;
  const double dtime = (dx2 / ctl->D_0) * dtime_s;
  const double t_b = ctl->t_b + (dx2 / ctl->D_0) * dtime_s;
  ctl->t_s = t_s;
  ctl->t_b = t_b;
  if (par->surface) {
    ctl->T_b = interp(t_b, p.sched_time, p.sched_temp, p.n_sched);
    ctl->T_b_valid = 1;
    ctl->surf_b = S[P5_IFACE] * p.surf_scale;
    ctl->surf_b_valid = 1;
  }

  // running sum of the energy derivative terms (pf_kks/residual.py:48-60)
  if (ctl->flag == 1 && istep >= ctl->good_step + 1) {
    const double term = (energy_s - ctl->E_prev) / (t_s - ctl->ts_prev);
    const double y = term - ctl->ed_comp;
    const double tt = ctl->ed_sum + y;
    ctl->ed_comp = (tt - ctl->ed_sum) - y;
    ctl->ed_sum = tt;
    ctl->ed_n += 1;
  }
  ctl->E_prev = energy_s;
  ctl->ts_prev = t_s;

  const double X_al_mean = S[P3_XLO] / S[P3_NLO];
  const double X_th_mean = S[P3_XHI] / S[P3_NHI];
  const int armed_before = ctl->flag;
  if (X_al_mean <= p.x_equilibrium && ctl->flag == 0 && istep > 1) {  // pf_kks/solver.py:375-378
    ctl->good_step = istep + p.good_step_offset;
    ctl->flag = 1;
  }
  (void)armed_before;

  kks_step_row row;
  for (int k = 0; k < 32; ++k) row.v[k] = 0;
  row.v[KKS_H_X_AL_MEAN] = X_al_mean;
  row.v[KKS_H_X_TH_MEAN] = X_th_mean;
  row.v[KKS_H_X_MEAN] = X_th_mean;  // mask (eta > 0.05) & (eta > 0.95) is eta > 0.95
  row.v[KKS_H_DX_AL_MEAN] = S[P5_XLO] / S[P5_NLO] - S[P3_XLO] / S[P3_NLO];
  row.v[KKS_H_DX_TH_MEAN] = S[P5_XHI] / S[P5_NHI] - S[P3_XHI] / S[P3_NHI];
  row.v[KKS_H_DETA_MEAN] = S[P5_ETA] / Nd - S[P3_ETA] / Nd;
  row.v[KKS_H_DT] = ctl->T_b - par->T;
  row.v[KKS_H_ETA_MEAN] = S[P3_ETA] / Nd;
  row.v[KKS_H_G_MEAN] = S[P3_G] / Nd;
  row.v[KKS_H_SURF] = ctl->surf_b;
  row.v[KKS_H_DSURF] = ctl->surf_b - ctl->surf;
  row.v[KKS_H_T] = par->T;
  row.v[KKS_H_DTIME] = dtime;
  row.v[KKS_H_TIME] = t;
  row.v[KKS_H_TIME_S] = t_s;
  row.v[KKS_H_L] = par->L;
  row.v[KKS_H_ENERGY_S] = energy_s;
  row.v[KKS_H_DTIME_S] = dtime_s;
  if (par->armed_residual) {
    for (int k = 0; k < 5; ++k) row.v[KKS_H_RES_TOTAL + k] = ctl->res[k];
  }
  row.v[KKS_H_TTIME] = ctl->ttime;
  row.v[KKS_H_ISTEP] = (double)istep;
  row.v[KKS_H_SURF_VALID] = (double)(ctl->surf_b_valid + 2 * ctl->surf_valid);
  row.v[KKS_H_D] = par->D;
  row.v[KKS_H_XV] = ctl->Xv;
  rows[ctl->n_row % row_cap] = row;
  ctl->n_row += 1;

  ctl->t = t_b;
  ctl->istep = istep + 1;
  ctl->iteration = 1;
  ctl->res_valid = 0;
}

__global__ void __launch_bounds__(32 * kDecideWarps)
    kks_decide(const KksConst* __restrict__ c, KksCtl* ctl, const KksPar* __restrict__ par,
               const double* __restrict__ partials, int nblocks, kks_record* ring, long long ring_cap,
               kks_step_row* rows, long long row_cap) {
  decide_body(c, ctl, par, partials, nblocks, ring, ring_cap, rows, row_cap);
}

// one block per cell of a batch
__global__ void __launch_bounds__(32 * kDecideWarps) kks_decide_batch(const KksCellDesc* __restrict__ cells) {
  const KksCellDesc& d = cells[blockIdx.x];
  decide_body(d.dc, d.ctl, d.par, d.partials, d.part_rows, d.ring, d.ring_cap, d.rows, d.row_cap);
}

}  // namespace

void kks_launch_prologue(const KksConst* c, KksCtl* ctl, KksPar* par, const uint8_t* step_flags, kks_record* ring,
                         long long ring_cap, cudaStream_t s) {
  kks_prologue<<<1, 32, 0, s>>>(c, ctl, par, step_flags, ring, ring_cap);
}

void kks_launch_decide(const KksConst* c, KksCtl* ctl, const KksPar* par, const double* partials, int nblocks,
                       kks_record* ring, long long ring_cap, kks_step_row* rows, long long row_cap, cudaStream_t s) {
  kks_decide<<<1, 32 * kDecideWarps, 0, s>>>(c, ctl, par, partials, nblocks, ring, ring_cap, rows, row_cap);
}

void kks_launch_prologue_batch(const KksCellDesc* cells, int n, cudaStream_t s) {
  kks_prologue_batch<<<n, 32, 0, s>>>(cells);
}

void kks_launch_decide_batch(const KksCellDesc* cells, int n, cudaStream_t s) {
  kks_decide_batch<<<n, 32 * kDecideWarps, 0, s>>>(cells);
}
