// kks_fft.cu - the mixed-path attempt with hand-written shared-memory FFTs.
//
// cuFFT runs every 2-D transform as several factor passes over the whole batch
// (1420 = 4*5*71: eight kernels per transform, its prime-71 factor
// compute-bound), and the pointwise stages of the step are separate passes
// between the transforms. Here each 2-D transform is split into a row pass and
// a column pass, every 1-D transform runs in shared memory, and the pointwise
// stages are fused into the passes around them:
//
//   rows_A    read eta, X (f64)   -> eta, X, eta^2 row spectra (RA)      + old-state history sums
//   cols_AB   RA columns: forward FFT -> FT(eta), FT(X) kept (SA); tr eps^, i k_x FT(eta),
//             i k_y FT(eta) -> inverse FFT -> row spectra (RB)          + Parseval sums
//   rows_BC   RB rows: inverse FFT -> tr eps, d_x eta, d_y eta; free energy, drive, fluxes
//             (pointwise, old state) -> forward FFT -> row spectra (RC) + sum G
//   cols_CD   RC columns: forward FFT; with SA the semi-implicit increments d_eta^, d_X^
//             -> inverse FFT -> row spectra (RD)
//   rows_D    RD rows: inverse FFT -> d_eta, d_X; new state, phase compositions, new free
//             energy, residual sums, new-state history sums
//   extras    np.gradient energy of the new state and, at surface steps, interface counts
//
// so that the spectra never make a round trip through HBM between a transform
// and the operation that consumes it. Rows are transformed in pairs as one
// complex sequence (row a + i row b) and split / merged with the Hermitian
// symmetry; row spectra hold the ny/2+1 non-negative y frequencies in natural
// order, one row per x. Each 1-D transform is an in-place mixed-radix DIF
// (natural order in, digit-reversed out) for forward transforms and the
// matching DIT (digit-reversed in, natural out) for inverse ones, so spectra
// inside a column pass are indexed through a slot -> frequency table and no
// permutation pass exists. Radices 2, 3, 4, 5, 7 are butterflies with
// compile-time constants; one larger prime factor (71 for 1420) is a direct
// DFT in registers using the symmetry of its cosine / sine matrix (a pair of
// outputs per 35 x 4 FMA), as the last DIF stage where it needs no twiddles.
// Only the mixed path uses these kernels (FP32 transforms on the increments of
// an FP64 state; see kks_fields.cu); the FP64 path keeps cuFFT.

#include <math.h>

#include "kks_internal.cuh"
#include "kks_fft.cuh"

namespace {

constexpr int kThreads = 128;

__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ float2 cmulc(float2 a, float2 b) {  // a * conj(b)
  return make_float2(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}

// cos / sin (2 pi m / R) of the small odd radices, m = 0..R-1 (compile-time after unrolling).
template <int R>
__device__ __forceinline__ constexpr float tc(int m);
template <int R>
__device__ __forceinline__ constexpr float ts(int m);
template <>
__device__ __forceinline__ constexpr float tc<3>(int m) {
  return m == 0 ? 1.0f : -0.5f;
}
template <>
__device__ __forceinline__ constexpr float ts<3>(int m) {
  return m == 0 ? 0.0f : (m == 1 ? 0.866025403784438647f : -0.866025403784438647f);
}
template <>
__device__ __forceinline__ constexpr float tc<5>(int m) {
  return m == 0 ? 1.0f : ((m == 1 || m == 4) ? 0.309016994374947424f : -0.809016994374947424f);
}
template <>
__device__ __forceinline__ constexpr float ts<5>(int m) {
  return m == 0 ? 0.0f
                : (m == 1 ? 0.951056516295153572f
                          : (m == 2 ? 0.587785252292473129f : (m == 3 ? -0.587785252292473129f : -0.951056516295153572f)));
}
template <>
__device__ __forceinline__ constexpr float tc<7>(int m) {
  return m == 0 ? 1.0f
                : ((m == 1 || m == 6) ? 0.623489801858733531f
                                      : ((m == 2 || m == 5) ? -0.222520933956314404f : -0.900968867902419126f));
}
template <>
__device__ __forceinline__ constexpr float ts<7>(int m) {
  return m == 0 ? 0.0f
                : (m == 1 ? 0.781831482468029809f
                          : (m == 2 ? 0.974927912181823607f
                                    : (m == 3 ? 0.433883739117558120f
                                              : (m == 4 ? -0.433883739117558120f
                                                        : (m == 5 ? -0.974927912181823607f : -0.781831482468029809f)))));
}

// Small DFT in registers: y_k = sum_m x_m exp(DIR 2 pi i m k / R), DIR = -1 (forward) or +1.
template <int R, int DIR>
__device__ __forceinline__ void dft_small(float2 (&x)[R]) {
  if constexpr (R == 2) {
    const float2 a = x[0], b = x[1];
    x[0] = cadd(a, b);
    x[1] = csub(a, b);
  } else if constexpr (R == 4) {
    const float2 t0 = cadd(x[0], x[2]), t1 = csub(x[0], x[2]);
    const float2 t2 = cadd(x[1], x[3]), t3 = csub(x[1], x[3]);
    x[0] = cadd(t0, t2);
    x[2] = csub(t0, t2);
    // -i t3 (forward) / +i t3 (inverse)
    const float2 it3 = DIR < 0 ? make_float2(t3.y, -t3.x) : make_float2(-t3.y, t3.x);
    x[1] = cadd(t1, it3);
    x[3] = csub(t1, it3);
  } else {
    constexpr int H = (R - 1) / 2;
    float2 s[H], d[H];
    float2 sum = x[0];
#pragma unroll
    for (int n = 1; n <= H; ++n) {
      s[n - 1] = cadd(x[n], x[R - n]);
      d[n - 1] = csub(x[n], x[R - n]);
      sum = cadd(sum, s[n - 1]);
    }
    const float2 x0 = x[0];
    float2 y[R];
    y[0] = sum;
#pragma unroll
    for (int k = 1; k <= H; ++k) {
      float2 A = x0, B = make_float2(0.f, 0.f);
#pragma unroll
      for (int n = 1; n <= H; ++n) {
        const int m = (n * k) % R;
        A.x += s[n - 1].x * tc<R>(m);
        A.y += s[n - 1].y * tc<R>(m);
        B.x += d[n - 1].x * ts<R>(m);
        B.y += d[n - 1].y * ts<R>(m);
      }
      if (DIR < 0) {
        y[k] = make_float2(A.x + B.y, A.y - B.x);
        y[R - k] = make_float2(A.x - B.y, A.y + B.x);
      } else {
        y[k] = make_float2(A.x - B.y, A.y + B.x);
        y[R - k] = make_float2(A.x + B.y, A.y - B.x);
      }
    }
#pragma unroll
    for (int k = 0; k < R; ++k) x[k] = y[k];
  }
}

// One in-place radix-R butterfly at base, stride q, twiddle row tw[j*R + m]
// (cos, sin of 2 pi j m / L). DIF (forward): twiddle after the DFT with
// exp(-i ...); DIT (inverse): twiddle before the DFT with exp(+i ...).
template <int R, int DIR>
__device__ __forceinline__ void bfly_small(float2* base, int q, int j, const float2* __restrict__ tw) {
  float2 x[R];
#pragma unroll
  for (int m = 0; m < R; ++m) x[m] = base[m * q];
  if (DIR > 0 && j != 0) {
    const float2* w = tw + j * R;
#pragma unroll
    for (int m = 1; m < R; ++m) x[m] = cmul(x[m], __ldg(w + m));
  }
  dft_small<R, DIR>(x);
  if (DIR < 0 && j != 0) {
    const float2* w = tw + j * R;
#pragma unroll
    for (int m = 1; m < R; ++m) x[m] = cmulc(x[m], __ldg(w + m));
  }
#pragma unroll
  for (int m = 0; m < R; ++m) base[m * q] = x[m];
}

// Direct DFT of prime length P on P consecutive elements (q = 1, no twiddles):
// the inputs are folded into s_n = x_n + x_{P-n}, d_n = x_n - x_{P-n} (in
// registers) and each output pair (k, P-k) costs H complex-by-real FMAs on s
// and d with cos / sin (2 pi n k / P) read from the table prow (row k-1, H
// float2 padded to an even count, broadcast to the warp).
template <int P, int DIR>
__device__ __forceinline__ void bfly_prime(float2* base, const float4* __restrict__ prow) {
  constexpr int H = (P - 1) / 2;
  constexpr int H2 = (H + 1) / 2;  // float4 per table row
  float2 s[H], d[H];
  const float2 x0 = base[0];
  float2 sum = x0;
#pragma unroll
  for (int n = 1; n <= H; ++n) {
    const float2 a = base[n], b = base[P - n];
    s[n - 1] = cadd(a, b);
    d[n - 1] = csub(a, b);
    sum = cadd(sum, s[n - 1]);
  }
#pragma unroll 1
  for (int k = 1; k <= H; ++k) {
    const float4* row = prow + (k - 1) * H2;
    float2 A = x0, B = make_float2(0.f, 0.f);
#pragma unroll
    for (int h = 0; h < H2; ++h) {
      const float4 w = __ldg(row + h);
      const int n0 = 2 * h;
      A.x += s[n0].x * w.x;
      A.y += s[n0].y * w.x;
      B.x += d[n0].x * w.y;
      B.y += d[n0].y * w.y;
      if (n0 + 1 < H) {
        A.x += s[n0 + 1].x * w.z;
        A.y += s[n0 + 1].y * w.z;
        B.x += d[n0 + 1].x * w.w;
        B.y += d[n0 + 1].y * w.w;
      }
    }
    if (DIR < 0) {
      base[k] = make_float2(A.x + B.y, A.y - B.x);
      base[P - k] = make_float2(A.x - B.y, A.y + B.x);
    } else {
      base[k] = make_float2(A.x - B.y, A.y + B.x);
      base[P - k] = make_float2(A.x + B.y, A.y - B.x);
    }
  }
  base[0] = sum;
}

// nseq in-place transforms of length ax.n, sequence s at buf + s * sstride.
// DIR = -1: forward DIF (natural -> digit-reversed); DIR = +1: inverse DIT
// (digit-reversed -> natural), unnormalised. P: the large prime of the axis
// (0 if none); its stage is the last DIF stage (q = 1).
template <int DIR, int P>
__device__ void fft_run(float2* buf, int nseq, int sstride, const KksFftAxis& ax) {
  for (int si = 0; si < ax.nst; ++si) {
    const int s = DIR < 0 ? si : ax.nst - 1 - si;
    const int r = ax.r[s], L = ax.L[s], q = ax.q[s];
    const int per = ax.n / r;
    const int total = nseq * per;
    const float2* tw = ax.tw + ax.tw_off[s];
    for (int t = threadIdx.x; t < total; t += blockDim.x) {
      const int seq = t / per;
      const int rem = t - seq * per;
      const int b = rem / q, j = rem - b * q;
      float2* base = buf + (size_t)seq * sstride + b * L + j;
      switch (r) {
        case 2: bfly_small<2, DIR>(base, q, j, tw); break;
        case 3: bfly_small<3, DIR>(base, q, j, tw); break;
        case 4: bfly_small<4, DIR>(base, q, j, tw); break;
        case 5: bfly_small<5, DIR>(base, q, j, tw); break;
        case 7: bfly_small<7, DIR>(base, q, j, tw); break;
        default:
          if constexpr (P > 7) bfly_prime<P, DIR>(base, (const float4*)ax.prow);
          break;
      }
    }
    __syncthreads();
  }
}

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
  if (threadIdx.x < 32) {
    const int lane2 = threadIdx.x;
#pragma unroll
    for (int k = 0; k < NV; ++k) {
      double x = lane2 < kThreads / 32 ? sh[k][lane2] : 0.0;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
      if (lane2 == 0) out[k] = x;
    }
  }
}

__device__ __forceinline__ bool in_iface(double e) { return e >= 0.1 && e <= 0.9; }

// Split the transform of (row a + i row b) into the half spectra of a and b
// and write them to rows ix0, ix0+1 of field f of a row-spectrum array.
__device__ __forceinline__ void split_store(const float2* z, const KksFftAxis& ay, float2* dst, int ix0, bool has1,
                                            int nyh) {
  const int ny = ay.n;
  for (int k = threadIdx.x; k < nyh; k += blockDim.x) {
    const float2 Zk = z[ay.slot[k]];
    const float2 Zm = z[ay.slot[k == 0 ? 0 : ny - k]];
    // A = (Z_k + conj Z_{-k}) / 2, B = (Z_k - conj Z_{-k}) / (2i)
    dst[(size_t)ix0 * nyh + k] = make_float2(0.5f * (Zk.x + Zm.x), 0.5f * (Zk.y - Zm.y));
    if (has1) dst[(size_t)(ix0 + 1) * nyh + k] = make_float2(0.5f * (Zk.y + Zm.y), -0.5f * (Zk.x - Zm.x));
  }
}

// Inverse of split_store: z (digit-reversed) = A + i B with the Hermitian
// extension. The y = 0 and Nyquist bins of a real row are real: their
// imaginary round-off is dropped (as a C2R transform does), so that it cannot
// leak into the other row of the pair.
__device__ __forceinline__ void merge_load(float2* z, const KksFftAxis& ay, const float2* src, int ix0, bool has1,
                                           int nyh) {
  const int ny = ay.n;
  for (int k = threadIdx.x; k < ny; k += blockDim.x) {
    float2 A, B;
    if (k < nyh) {
      A = src[(size_t)ix0 * nyh + k];
      B = has1 ? src[(size_t)(ix0 + 1) * nyh + k] : make_float2(0.f, 0.f);
      if (k == 0 || 2 * k == ny) {
        A.y = 0.f;
        B.y = 0.f;
      }
    } else {
      const float2 a = src[(size_t)ix0 * nyh + (ny - k)];
      const float2 b = has1 ? src[(size_t)(ix0 + 1) * nyh + (ny - k)] : make_float2(0.f, 0.f);
      A = make_float2(a.x, -a.y);
      B = make_float2(b.x, -b.y);
    }
    z[ay.slot[k]] = make_float2(A.x - B.y, A.y + B.x);
  }
}

// ---------------------------------------------------------------------------
// pass 1: eta, X rows -> row spectra of eta, X, eta^2; old-state history sums
template <int PY>
__global__ void __launch_bounds__(kThreads) kf_rows_A(const KksConst* __restrict__ c, const KksPar* __restrict__ par,
                                                      const KksFftConst* __restrict__ fc,
                                                      const double* __restrict__ eta, const double* __restrict__ X,
                                                      float2* __restrict__ RA, double* __restrict__ partials) {
  if (!par->active) return;
  extern __shared__ float2 sm[];
  const KksFftAxis& ay = fc->ay;
  const int nx = c->nx, ny = c->ny, nyh = c->nyh;
  const int ix0 = 2 * blockIdx.x;
  const bool has1 = ix0 + 1 < nx;
  double acc[5] = {0, 0, 0, 0, 0};
  for (int y = threadIdx.x; y < ny; y += blockDim.x) {
    const double e0 = eta[(size_t)ix0 * ny + y], x0 = X[(size_t)ix0 * ny + y];
    const double e1 = has1 ? eta[(size_t)(ix0 + 1) * ny + y] : 0.0, x1 = has1 ? X[(size_t)(ix0 + 1) * ny + y] : 0.0;
    sm[y] = make_float2((float)e0, (float)e1);
    sm[ny + y] = make_float2((float)x0, (float)x1);
    sm[2 * ny + y] = make_float2((float)(e0 * e0), (float)(e1 * e1));
    acc[0] += e0;
    if (e0 < 0.05) { acc[1] += x0; acc[2] += 1.0; }
    if (e0 > 0.95) { acc[3] += x0; acc[4] += 1.0; }
    if (has1) {
      acc[0] += e1;
      if (e1 < 0.05) { acc[1] += x1; acc[2] += 1.0; }
      if (e1 > 0.95) { acc[3] += x1; acc[4] += 1.0; }
    }
  }
  __syncthreads();
  fft_run<-1, PY>(sm, 3, ny, ay);
  const size_t fs = (size_t)nx * nyh;
  for (int f = 0; f < 3; ++f) split_store(sm + f * ny, ay, RA + f * fs, ix0, has1, nyh);
  block_reduce_store<5>(acc, partials + (size_t)blockIdx.x * KKS_NPART + P3_ETA);
}

// column tile: C consecutive y-frequency columns, every x
template <int C>
__device__ __forceinline__ void col_load(float2* sm, const float2* __restrict__ src, int nx, int nyh, int ky0,
                                         int ncol) {
  for (int idx = threadIdx.x; idx < nx * C; idx += blockDim.x) {
    const int p = idx / C, cc = idx - p * C;
    sm[cc * nx + p] = cc < ncol ? src[(size_t)p * nyh + ky0 + cc] : make_float2(0.f, 0.f);
  }
}

template <int C>
__device__ __forceinline__ void col_store(const float2* sm, float2* __restrict__ dst, int nx, int nyh, int ky0,
                                          int ncol) {
  for (int idx = threadIdx.x; idx < nx * C; idx += blockDim.x) {
    const int p = idx / C, cc = idx - p * C;
    if (cc < ncol) dst[(size_t)p * nyh + ky0 + cc] = sm[cc * nx + p];
  }
}

// pass 2: columns of RA. blockIdx.y: 0 eta -> keep FT(eta), i k_x FT(eta);
// 1 eta -> i k_y FT(eta); 2 eta^2 -> tr eps^ (+ Parseval sums); 3 X -> keep FT(X).
template <int PX, int C>
__global__ void __launch_bounds__(kThreads) kf_cols_AB(const KksConst* __restrict__ c,
                                                       const KksPar* __restrict__ par,
                                                       const KksFftConst* __restrict__ fc,
                                                       const float2* __restrict__ RA, float2* __restrict__ SA,
                                                       float2* __restrict__ RB, const double* __restrict__ kys,
                                                       double* __restrict__ partials) {
  if (!par->active) return;
  extern __shared__ float2 sm[];
  const KksFftAxis& ax = fc->ax;
  const int nx = c->nx, ny = c->ny, nyh = c->nyh;
  const size_t fs = (size_t)nx * nyh;
  const int g = blockIdx.y;
  const int ky0 = blockIdx.x * C;
  const int ncol = min(C, nyh - ky0);
  const int src_field = g < 2 ? 0 : (g == 2 ? 2 : 1);
  col_load<C>(sm, RA + src_field * fs, nx, nyh, ky0, ncol);
  __syncthreads();
  fft_run<-1, PX>(sm, C, nx, ax);
  if (g == 3) {
    col_store<C>(sm, SA + fs, nx, nyh, ky0, ncol);
    return;
  }
  if (g == 0) col_store<C>(sm, SA, nx, nyh, ky0, ncol);
  const float inv_N = (float)c->inv_N;
  const float a = (float)(par->epsX * c->c3) * inv_N;
  const float c11 = (float)c->c11, c12 = (float)c->c12;
  double acc[6] = {0, 0, 0, 0, 0, 0};
  for (int idx = threadIdx.x; idx < nx * C; idx += blockDim.x) {
    const int cc = idx / nx, p = idx - cc * nx;
    if (cc >= ncol) continue;
    const float kx = fc->kx_slot[p];
    const int iy = ky0 + cc;
    const float ky = (float)kys[iy];
    float2 v = sm[idx];
    if (g == 0) {
      v = make_float2(-kx * inv_N * v.y, kx * inv_N * v.x);
    } else if (g == 1) {
      v = make_float2(-ky * inv_N * v.y, ky * inv_N * v.x);
    } else {
      // strain multipliers of the 2x2 acoustic tensor (stiffness / C44(T0)), 0 at k = 0
      const float Kxx = c11 * kx * kx + ky * ky, Kyy = kx * kx + c11 * ky * ky, Kxy = (c12 + 1.f) * kx * ky;
      const float det = Kxx * Kyy - Kxy * Kxy;
      float oxx = 0.f, oyy = 0.f, oxy = 0.f;
      if (det != 0.f) {
        const float inv = 1.f / det;
        const float Nxx = Kyy * inv, Nyy = Kxx * inv, Nxy = -Kxy * inv;
        const float Nkx = Nxx * kx + Nxy * ky, Nky = Nxy * kx + Nyy * ky;
        oxx = Nkx * kx;
        oyy = Nky * ky;
        oxy = 0.5f * (Nky * kx + Nkx * ky);
      }
      const double w = (iy == 0 || 2 * iy == ny) ? 1.0 : 2.0;
      const double pw = w * ((double)v.x * v.x + (double)v.y * v.y);
      const double dxx = oxx, dyy = oyy, dxy = oxy;
      acc[0] += pw * dxx * dxx;
      acc[1] += pw * dyy * dyy;
      acc[2] += pw * dxx * dyy;
      acc[3] += pw * dxy * dxy;
      acc[4] += pw * (dxx + dyy);
      acc[5] += pw;
      const float st = a * (oxx + oyy);
      v = make_float2(st * v.x, st * v.y);
    }
    sm[idx] = v;
  }
  if (g == 2) block_reduce_store<6>(acc, partials + (size_t)blockIdx.x * KKS_NPART + P2_OXX2);
  __syncthreads();
  fft_run<+1, PX>(sm, C, nx, ax);
  const int dst_field = g == 2 ? 0 : (g == 0 ? 1 : 2);
  col_store<C>(sm, RB + dst_field * fs, nx, nyh, ky0, ncol);
}

// pass 3: RB rows -> tr eps, d_x eta, d_y eta; pointwise old-state free
// energy, Allen-Cahn drive and Cahn-Hilliard fluxes -> row spectra RC
template <int PY>
__global__ void __launch_bounds__(kThreads)
    kf_rows_BC(const KksConst* __restrict__ c, const KksPar* __restrict__ par, const KksFftConst* __restrict__ fc,
               const float2* __restrict__ RB, float2* __restrict__ RC, const double* __restrict__ eta,
               const float* __restrict__ Xal, const float* __restrict__ Xth, float* g0, float* g1, float* g2,
               double* __restrict__ partials) {
  if (!par->active) return;
  extern __shared__ float2 sm[];
  const KksFftAxis& ay = fc->ay;
  const int nx = c->nx, ny = c->ny, nyh = c->nyh;
  const size_t fs = (size_t)nx * nyh;
  const int ix0 = 2 * blockIdx.x;
  const bool has1 = ix0 + 1 < nx;
  for (int f = 0; f < 3; ++f) merge_load(sm + f * ny, ay, RB + f * fs, ix0, has1, nyh);
  __syncthreads();
  fft_run<+1, PY>(sm, 3, ny, ay);
  const KksPar q = *par;
  float* gs_buf = q.gs == 0 ? g0 : (q.gs == 1 ? g1 : g2);
  const float A_a = (float)q.A_alp_s, va = (float)q.va, fa0 = (float)q.fa0;
  const float A_t = (float)q.A_thet_s, vt = (float)q.vt, ft0 = (float)q.ft0, w_s = (float)q.w_s;
  const float epsX = (float)q.epsX;
  const float c3 = (float)((c->C11_0 + 2 * c->C12_0) * q.inv_C44);
  double accG = 0.0;
  for (int y = threadIdx.x; y < ny; y += blockDim.x) {
    const float2 tr = sm[y], gx = sm[ny + y], gy = sm[2 * ny + y];
    float dr[2], fxv[2], fyv[2];
#pragma unroll
    for (int r = 0; r < 2; ++r) {
      dr[r] = fxv[r] = fyv[r] = 0.f;
      if (r == 1 && !has1) continue;
      const size_t i = (size_t)(ix0 + r) * ny + y;
      const float e = (float)eta[i];
      const float ca = Xal[i], ct = Xth[i];
      const float da = ca - va, dtt = ct - vt;
      const float fa_s = A_a * da * da + fa0;
      const float fa_ca_s = 2.0f * A_a * da;
      const float ft_s = A_t * dtt * dtt + ft0;
      const float e2 = e * e, e3 = e2 * e;
      const float h = 3.0f * e2 - 2.0f * e3;
      const float h_eta = 6.0f * e - 6.0f * e2;
      const float gw = e2 - 2.0f * e3 + e2 * e2;
      const float g_eta = 2.0f * e - 6.0f * e2 + 4.0f * e3;
      const float G = (1.0f - h) * fa_s + h * ft_s + w_s * gw;
      const float G_eta = -h_eta * (fa_s - ft_s - (ca - ct) * fa_ca_s) + w_s * g_eta;
      const float flux = h_eta * (ca - ct);
      const float trv = r == 0 ? tr.x : tr.y;
      const float el_eta_s = 2.0f * epsX * e * c3 * (3.0f * epsX * e2 - trv);
      dr[r] = G_eta + el_eta_s;
      fxv[r] = flux * (r == 0 ? gx.x : gx.y);
      fyv[r] = flux * (r == 0 ? gy.x : gy.y);
      if (q.armed_write) gs_buf[i] = G;
      accG += (double)G;
    }
    sm[y] = make_float2(dr[0], dr[1]);
    sm[ny + y] = make_float2(fxv[0], fxv[1]);
    sm[2 * ny + y] = make_float2(fyv[0], fyv[1]);
  }
  __syncthreads();
  fft_run<-1, PY>(sm, 3, ny, ay);
  for (int f = 0; f < 3; ++f) split_store(sm + f * ny, ay, RC + f * fs, ix0, has1, nyh);
  double acc[1] = {accG};
  block_reduce_store<1>(acc, partials + (size_t)blockIdx.x * KKS_NPART + P3_G);
}

// pass 4: columns of RC. blockIdx.y: 0 -> d_eta^ from FT(drive) and FT(eta);
// 1 -> d_X^ from FT(flux_x), FT(flux_y) and FT(X). Output row spectra RD.
template <int PX, int C>
__global__ void __launch_bounds__(kThreads) kf_cols_CD(const KksConst* __restrict__ c,
                                                       const KksPar* __restrict__ par,
                                                       const KksFftConst* __restrict__ fc,
                                                       const float2* __restrict__ RC, const float2* __restrict__ SA,
                                                       float2* __restrict__ RD, const double* __restrict__ kys) {
  if (!par->active) return;
  extern __shared__ float2 sm[];
  const KksFftAxis& ax = fc->ax;
  const int nx = c->nx, nyh = c->nyh;
  const size_t fs = (size_t)nx * nyh;
  const int g = blockIdx.y;
  const int ky0 = blockIdx.x * C;
  const int ncol = min(C, nyh - ky0);
  const float inv_N = (float)c->inv_N;
  const float ac_mul = (float)par->ac_mul, ac_den = (float)par->ac_den, ch_mul = (float)par->ch_mul;
  const float dtD = (float)(par->dt * par->D_s);
  if (g == 0) {
    col_load<C>(sm, RC, nx, nyh, ky0, ncol);
    __syncthreads();
    fft_run<-1, PX>(sm, C, nx, ax);
    for (int idx = threadIdx.x; idx < nx * C; idx += blockDim.x) {
      const int cc = idx / nx, p = idx - cc * nx;
      if (cc >= ncol) continue;
      const float kx = fc->kx_slot[p], ky = (float)kys[ky0 + cc];
      const float k2 = kx * kx + ky * ky;
      const float2 dh = sm[idx];
      const float2 eh = SA[(size_t)p * nyh + ky0 + cc];
      const float ak = ac_den * k2, den = 1.f + ak;
      sm[idx] = make_float2((ac_mul * dh.x - ak * eh.x) / den * inv_N, (ac_mul * dh.y - ak * eh.y) / den * inv_N);
    }
    __syncthreads();
    fft_run<+1, PX>(sm, C, nx, ax);
    col_store<C>(sm, RD, nx, nyh, ky0, ncol);
  } else {
    col_load<C>(sm, RC + fs, nx, nyh, ky0, ncol);
    col_load<C>(sm + C * nx, RC + 2 * fs, nx, nyh, ky0, ncol);
    __syncthreads();
    fft_run<-1, PX>(sm, 2 * C, nx, ax);
    for (int idx = threadIdx.x; idx < nx * C; idx += blockDim.x) {
      const int cc = idx / nx, p = idx - cc * nx;
      if (cc >= ncol) continue;
      const float kx = fc->kx_slot[p], ky = (float)kys[ky0 + cc];
      const float k2 = kx * kx + ky * ky;
      const float2 fx = sm[idx], fy = sm[C * nx + idx];
      const float flx = -(kx * fx.y) - ky * fy.y;
      const float fly = kx * fx.x + ky * fy.x;
      const float2 xh = SA[fs + (size_t)p * nyh + ky0 + cc];
      const float bk = dtD * k2, den = 1.f + bk;
      sm[idx] = make_float2((ch_mul * flx - bk * xh.x) / den * inv_N, (ch_mul * fly - bk * xh.y) / den * inv_N);
    }
    __syncthreads();
    fft_run<+1, PX>(sm, C, nx, ax);
    col_store<C>(sm, RD + fs, nx, nyh, ky0, ncol);
  }
}

// pass 5: RD rows -> d_eta, d_X; new state, phase compositions, new free
// energy and diffusion potential, residual and history sums
template <int PY>
__global__ void __launch_bounds__(kThreads)
    kf_rows_D(const KksConst* __restrict__ c, const KksPar* __restrict__ par, const KksFftConst* __restrict__ fc,
              const float2* __restrict__ RD, const double* __restrict__ eta_o, const double* __restrict__ X_o,
              double* __restrict__ eta_b, double* __restrict__ X_b, float* __restrict__ Xal_b,
              float* __restrict__ Xth_b, const double* __restrict__ eta_m, const double* __restrict__ X_m,
              float* __restrict__ mu, float* g0, float* g1, float* g2, double* __restrict__ partials) {
  if (!par->active) return;
  extern __shared__ float2 sm[];
  const KksFftAxis& ay = fc->ay;
  const int nx = c->nx, ny = c->ny, nyh = c->nyh;
  const size_t fs = (size_t)nx * nyh;
  const int ix0 = 2 * blockIdx.x;
  const bool has1 = ix0 + 1 < nx;
  merge_load(sm, ay, RD, ix0, has1, nyh);
  merge_load(sm + ny, ay, RD + fs, ix0, has1, nyh);
  __syncthreads();
  fft_run<+1, PY>(sm, 2, ny, ay);
  const KksPar q = *par;
  float* gb_buf = q.gb == 0 ? g0 : (q.gb == 1 ? g1 : g2);
  const float* gm_buf = q.gm == 0 ? g0 : (q.gm == 1 ? g1 : g2);
  const double* eta_minus = q.minus_is_state ? eta_o : eta_m;
  const double* X_minus = q.minus_is_state ? X_o : X_m;
  const float A_a = (float)q.A_alp_s, va = (float)q.va, fa0 = (float)q.fa0;
  const float A_t = (float)q.A_thet_s, vt = (float)q.vt, ft0 = (float)q.ft0, w_s = (float)q.w_s;
  const double dt = q.dt;
  double acc[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  for (int y = threadIdx.x; y < ny; y += blockDim.x) {
    const float2 de = sm[y], dX = sm[ny + y];
#pragma unroll
    for (int r = 0; r < 2; ++r) {
      if (r == 1 && !has1) continue;
      const size_t i = (size_t)(ix0 + r) * ny + y;
      const double xo = X_o[i];
      const double eb = eta_o[i] + (double)(r == 0 ? de.x : de.y);
      const double xb = xo + (double)(r == 0 ? dX.x : dX.y);
      eta_b[i] = eb;
      X_b[i] = xb;
      // closed-form phase compositions in FP64 with the reference's guards
      const double h = 3.0 * (eb * eb) - 2 * (eb * eb * eb);
      double xal = (xo - h * q.pc_shift) / ((1 - h) + h * q.pc_ratio);
      if (isinf(xal)) xal = xal > 0 ? 1e-6 : -1e-6;
      if (isnan(xal)) xal = 1e-6;
      double xth = q.pc_ratio * xal + q.pc_shift;
      if (isinf(xth)) xth = xth > 0 ? 1e-6 : -1e-6;
      if (isnan(xth)) xth = 1e-6;
      Xal_b[i] = (float)xal;
      Xth_b[i] = (float)xth;
      if (eb < 0.05) { acc[0] += xb; acc[1] += 1.0; }
      if (eb > 0.95) { acc[2] += xb; acc[3] += 1.0; }
      acc[4] += eb;
      if (q.armed_write) {
        const float ca = (float)xal, ct = (float)xth, e = (float)eb;
        const float da = ca - va, dtt = ct - vt;
        const float fa_s = A_a * da * da + fa0;
        const float mu_b = 2.0f * A_a * da;
        const float ft_s = A_t * dtt * dtt + ft0;
        const float e2 = e * e, e3 = e2 * e;
        const float hh = 3.0f * e2 - 2.0f * e3;
        const float gw = e2 - 2.0f * e3 + e2 * e2;
        const float G_b = (1.0f - hh) * fa_s + hh * ft_s + w_s * gw;
        if (q.armed_residual) {
          const double mum = (double)mu[i];
          const double dXdt = (xb - X_minus[i]) / dt;
          const double mu_mean = ((double)mu_b + mum) / 2;
          const double diffusion = dXdt * mu_mean;
          const double detadt = (eb - eta_minus[i]) / dt;
          const double allen_cahn = q.inv_Ls * (detadt * detadt);
          const double temperature = ((double)G_b - (double)gm_buf[i]) / dt;
          acc[5] += diffusion;
          acc[6] += allen_cahn;
          acc[7] += temperature;
          acc[8] += -1 * diffusion + allen_cahn - temperature;
        }
        mu[i] = mu_b;
        gb_buf[i] = G_b;
      }
    }
  }
  // slots P5_XLO, NLO, XHI, NHI, ETA are consecutive; DIFF, AC, TEMP, COMB follow P5_IFACE
  double a5[5] = {acc[0], acc[1], acc[2], acc[3], acc[4]};
  block_reduce_store<5>(a5, partials + (size_t)blockIdx.x * KKS_NPART + P5_XLO);
  __syncthreads();
  double a4[4] = {acc[5], acc[6], acc[7], acc[8]};
  block_reduce_store<4>(a4, partials + (size_t)blockIdx.x * KKS_NPART + P5_DIFF);
}

// np.gradient energy sum of a state (mode bit 0) and, at surface steps, its
// interface cell count (mode bit 1) into the given partial slots.
__global__ void __launch_bounds__(kThreads)
    kf_extras(const KksConst* __restrict__ c, const KksPar* __restrict__ par, const double* __restrict__ eta,
              int mode, int slot_grad, int slot_iface, double* __restrict__ partials) {
  if (!par->active) return;
  const bool do_grad = mode & 1;
  const bool do_iface = (mode & 2) && par->surface;
  if (!do_grad && !do_iface) return;
  const int N = c->N, nx = c->nx, ny = c->ny;
  double acc[2] = {0, 0};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
    const int ix = i / ny, iy = i - ix * ny;
    const double e = eta[i];
    if (do_grad) {
      double gx, gy;
      if (ix == 0) gx = eta[i + ny] - e;
      else if (ix == nx - 1) gx = e - eta[i - ny];
      else gx = (eta[i + ny] - eta[i - ny]) / 2.0;
      if (iy == 0) gy = eta[i + 1] - e;
      else if (iy == ny - 1) gy = e - eta[i - 1];
      else gy = (eta[i + 1] - eta[i - 1]) / 2.0;
      acc[0] += gx * gx + gy * gy;
    }
    if (do_iface && ix < nx - 1 && iy < ny - 1 && in_iface(e) && in_iface(eta[i + ny]) &&
        in_iface(eta[i + ny + 1]) && in_iface(eta[i + 1]))
      acc[1] += 1.0;
  }
  double a1[1] = {acc[0]};
  double a2[1] = {acc[1]};
  if (do_grad) block_reduce_store<1>(a1, partials + (size_t)blockIdx.x * KKS_NPART + slot_grad);
  __syncthreads();
  if (do_iface) block_reduce_store<1>(a2, partials + (size_t)blockIdx.x * KKS_NPART + slot_iface);
}

template <int PY>
void launch_rows(const KksFftLaunch& L, int p, int stage, cudaStream_t s) {
  const KksConst* dc = L.dc;
  const KksPar* par = L.par;
  const KksFieldPtrs& f = *L.f;
  const int q = 1 - p;
  const int npairs = (L.nx + 1) / 2;
  const size_t row_smem3 = 3 * (size_t)L.ny * sizeof(float2);
  const size_t row_smem2 = 2 * (size_t)L.ny * sizeof(float2);
  float2* RA = (float2*)L.RA;
  float2* RB = (float2*)L.RB;
  if (stage == 0) {
    kf_rows_A<PY><<<npairs, kThreads, row_smem3, s>>>(dc, par, L.fc, (const double*)f.eta[p], (const double*)f.X[p],
                                                      RA, f.partials);
  } else if (stage == 1) {
    kf_rows_BC<PY><<<npairs, kThreads, row_smem3, s>>>(dc, par, L.fc, RB, RA, (const double*)f.eta[p],
                                                       (const float*)f.X_al[p], (const float*)f.X_th[p],
                                                       (float*)f.g[0], (float*)f.g[1], (float*)f.g[2], f.partials);
  } else {
    kf_rows_D<PY><<<npairs, kThreads, row_smem2, s>>>(
        dc, par, L.fc, RB, (const double*)f.eta[p], (const double*)f.X[p], (double*)f.eta[q], (double*)f.X[q],
        (float*)f.X_al[q], (float*)f.X_th[q], (const double*)f.eta_m, (const double*)f.X_m, (float*)f.mu,
        (float*)f.g[0], (float*)f.g[1], (float*)f.g[2], f.partials);
  }
}

template <int PX>
void launch_cols(const KksFftLaunch& L, int stage, cudaStream_t s) {
  constexpr int C = KKS_FFT_COLS;
  const int ntiles = (L.nyh + C - 1) / C;
  const size_t col_smem1 = (size_t)C * L.nx * sizeof(float2);
  float2* RA = (float2*)L.RA;
  float2* RB = (float2*)L.RB;
  float2* SA = (float2*)L.SA;
  if (stage == 0) {
    kf_cols_AB<PX, C><<<dim3(ntiles, 4), kThreads, col_smem1, s>>>(L.dc, L.par, L.fc, RA, SA, RB, L.f->ky,
                                                                    L.f->partials);
  } else {
    kf_cols_CD<PX, C><<<dim3(ntiles, 2), kThreads, 2 * col_smem1, s>>>(L.dc, L.par, L.fc, RA, SA, RB, L.f->ky);
  }
}

template <int PY>
int set_row_attrs(int ny) {
  const int row3 = 3 * ny * (int)sizeof(float2);
  const int row2 = 2 * ny * (int)sizeof(float2);
  cudaError_t e = cudaFuncSetAttribute(kf_rows_A<PY>, cudaFuncAttributeMaxDynamicSharedMemorySize, row3);
  if (e == cudaSuccess) e = cudaFuncSetAttribute(kf_rows_BC<PY>, cudaFuncAttributeMaxDynamicSharedMemorySize, row3);
  if (e == cudaSuccess) e = cudaFuncSetAttribute(kf_rows_D<PY>, cudaFuncAttributeMaxDynamicSharedMemorySize, row2);
  return (int)e;
}

template <int PX>
int set_col_attrs(int nx) {
  constexpr int C = KKS_FFT_COLS;
  const int col1 = C * nx * (int)sizeof(float2);
  cudaError_t e = cudaFuncSetAttribute(kf_cols_AB<PX, C>, cudaFuncAttributeMaxDynamicSharedMemorySize, col1);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(kf_cols_CD<PX, C>, cudaFuncAttributeMaxDynamicSharedMemorySize, 2 * col1);
  return (int)e;
}

#define KKS_FFT_DISPATCH(PVAL, CALL) \
  switch (PVAL) {                    \
    case 0: CALL(0); break;          \
    case 11: CALL(11); break;        \
    case 19: CALL(19); break;        \
    case 71: CALL(71); break;        \
    default: break;                  \
  }

}  // namespace

int kks_fft_partial_rows(int nx, int ny, int nbx) {
  const int npairs = (nx + 1) / 2;
  const int ntiles = (ny / 2 + 1 + KKS_FFT_COLS - 1) / KKS_FFT_COLS;
  int m = npairs > ntiles ? npairs : ntiles;
  return m > nbx ? m : nbx;
}

// The large prime of each axis selects the kernel instantiation.
int kks_fft_set_attributes(const KksFftLaunch& L) {
  int rc = -1, rc2 = -1;
#define KKS_ROWS_ATTR(P) rc = set_row_attrs<P>(L.ny)
#define KKS_COLS_ATTR(P) rc2 = set_col_attrs<P>(L.nx)
  KKS_FFT_DISPATCH(L.PY, KKS_ROWS_ATTR)
  KKS_FFT_DISPATCH(L.PX, KKS_COLS_ATTR)
#undef KKS_ROWS_ATTR
#undef KKS_COLS_ATTR
  return rc != 0 ? rc : rc2;
}

void kks_fft_launch_attempt(const KksFftLaunch& L, int p, cudaStream_t s) {
  const KksFieldPtrs& f = *L.f;
  kf_extras<<<L.nbx, kThreads, 0, s>>>(L.dc, L.par, (const double*)f.eta[p], 2, 0, P3_IFACE, f.partials);
#define KKS_ROWS(P) launch_rows<P>(L, p, stage, s)
#define KKS_COLS(P) launch_cols<P>(L, stage, s)
  int stage = 0;
  KKS_FFT_DISPATCH(L.PY, KKS_ROWS)
  KKS_FFT_DISPATCH(L.PX, KKS_COLS)
  stage = 1;
  KKS_FFT_DISPATCH(L.PY, KKS_ROWS)
  KKS_FFT_DISPATCH(L.PX, KKS_COLS)
  stage = 2;
  KKS_FFT_DISPATCH(L.PY, KKS_ROWS)
#undef KKS_ROWS
#undef KKS_COLS
  kf_extras<<<L.nbx, kThreads, 0, s>>>(L.dc, L.par, (const double*)f.eta[1 - p], 3, P5_GRAD2, P5_IFACE,
                                       f.partials);
}
