// kks_fft64.cu - the fused shared-memory FFT pipeline of the FP64 step.
//
// The FP64 step runs, per attempt, the six passes of the mixed step's fused
// pipeline (kks_fft.cu: rows_A, cols_AB, rows_BC, cols_CD_eta, cols_CD_X,
// rows_D; then the shared extras kernel) with every value in double precision:
// sequences of double2 in shared memory, twiddle and prime-stage factor tables
// computed on the host in double, the FP64 path's pointwise formulas
// (kks_pointwise.cuh, the reference's operation order), and the semi-implicit
// updates formed as the new spectra, as the cuFFT FP64 step does
// (pf_kks/solver.py:249-264). One attempt replaces eleven cuFFT FP64 2-D
// transforms and the five pointwise kernels between them; the FP64 result is
// the same to round-off (the step's parity bar is 1e-10).
//
// Differences from the mixed kernels, all for the doubled width of a value:
// spectra move between passes with plain loads and stores (a row pair's two
// values of one frequency are 32 contiguous bytes; a column is contiguous), so
// no tensor maps or bulk copies; the prime stage gives each lane 5 output pairs
// (7 groups over seven-warp blocks) to keep its FP64 accumulators in registers;
// a column tile defaults to one column.

#include <cuda_runtime.h>
#include <math.h>

#include <algorithm>

#include "kks_fft.cuh"
#include "kks_pointwise.cuh"

namespace {

using kks_pw::FreeEnergy;
using kks_pw::free_energy;
using kks_pw::phase_comp;
using kks_pw::strain_multipliers;

// Threads of a pass block: seven warps on axes with a large prime (one per
// output group of the prime stage), four otherwise.
template <int P>
__host__ __device__ constexpr int nt64() {
  return P > 7 ? 224 : 128;
}
template <int P>
__host__ __device__ constexpr int minb64() {
  return P > 7 ? 2 : 4;
}

__device__ __forceinline__ double2 zadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 zsub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double2 zmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 zmulc(double2 a, double2 b) {  // a * conj(b)
  return make_double2(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}

// cos / sin (2 pi m / R) of the small odd radices (exact values to double precision).
template <int R>
__device__ __forceinline__ constexpr double zc(int m);
template <int R>
__device__ __forceinline__ constexpr double zs(int m);
template <>
__device__ __forceinline__ constexpr double zc<3>(int m) {
  return m == 0 ? 1.0 : -0.5;
}
template <>
__device__ __forceinline__ constexpr double zs<3>(int m) {
  return m == 0 ? 0.0 : (m == 1 ? 0.86602540378443864676 : -0.86602540378443864676);
}
template <>
__device__ __forceinline__ constexpr double zc<5>(int m) {
  return m == 0 ? 1.0 : ((m == 1 || m == 4) ? 0.30901699437494742410 : -0.80901699437494742410);
}
template <>
__device__ __forceinline__ constexpr double zs<5>(int m) {
  return m == 0 ? 0.0
                : (m == 1 ? 0.95105651629515357212
                          : (m == 2 ? 0.58778525229247312917
                                    : (m == 3 ? -0.58778525229247312917 : -0.95105651629515357212)));
}
template <>
__device__ __forceinline__ constexpr double zc<7>(int m) {
  return m == 0 ? 1.0
                : ((m == 1 || m == 6) ? 0.62348980185873353053
                                      : ((m == 2 || m == 5) ? -0.22252093395631440429 : -0.90096886790241912624));
}
template <>
__device__ __forceinline__ constexpr double zs<7>(int m) {
  return m == 0 ? 0.0
                : (m == 1 ? 0.78183148246802980871
                          : (m == 2 ? 0.97492791218182360702
                                    : (m == 3 ? 0.43388373911755812048
                                              : (m == 4 ? -0.43388373911755812048
                                                        : (m == 5 ? -0.97492791218182360702
                                                                  : -0.78183148246802980871)))));
}

// Small DFT in registers: y_k = sum_m x_m exp(DIR 2 pi i m k / R).
template <int R, int DIR>
__device__ __forceinline__ void zdft_small(double2 (&x)[R]) {
  if constexpr (R == 2) {
    const double2 a = x[0], b = x[1];
    x[0] = zadd(a, b);
    x[1] = zsub(a, b);
  } else if constexpr (R == 4) {
    const double2 t0 = zadd(x[0], x[2]), t1 = zsub(x[0], x[2]);
    const double2 t2 = zadd(x[1], x[3]), t3 = zsub(x[1], x[3]);
    x[0] = zadd(t0, t2);
    x[2] = zsub(t0, t2);
    const double2 it3 = DIR < 0 ? make_double2(t3.y, -t3.x) : make_double2(-t3.y, t3.x);
    x[1] = zadd(t1, it3);
    x[3] = zsub(t1, it3);
  } else {
    constexpr int H = (R - 1) / 2;
    double2 s[H], d[H];
    double2 sum = x[0];
#pragma unroll
    for (int n = 1; n <= H; ++n) {
      s[n - 1] = zadd(x[n], x[R - n]);
      d[n - 1] = zsub(x[n], x[R - n]);
      sum = zadd(sum, s[n - 1]);
    }
    const double2 x0 = x[0];
    double2 y[R];
    y[0] = sum;
#pragma unroll
    for (int k = 1; k <= H; ++k) {
      double2 A = x0, B = make_double2(0.0, 0.0);
#pragma unroll
      for (int n = 1; n <= H; ++n) {
        const int m = (n * k) % R;
        A.x += s[n - 1].x * zc<R>(m);
        A.y += s[n - 1].y * zc<R>(m);
        B.x += d[n - 1].x * zs<R>(m);
        B.y += d[n - 1].y * zs<R>(m);
      }
      if (DIR < 0) {
        y[k] = make_double2(A.x + B.y, A.y - B.x);
        y[R - k] = make_double2(A.x - B.y, A.y + B.x);
      } else {
        y[k] = make_double2(A.x - B.y, A.y + B.x);
        y[R - k] = make_double2(A.x + B.y, A.y - B.x);
      }
    }
#pragma unroll
    for (int k = 0; k < R; ++k) x[k] = y[k];
  }
}

// One in-place radix-R butterfly at base, stride q, twiddles tw[j R + m].
template <int R, int DIR>
__device__ __forceinline__ void zbfly(double2* base, int q, int j, const double2* __restrict__ tw) {
  double2 x[R];
#pragma unroll
  for (int m = 0; m < R; ++m) x[m] = base[m * q];
  if (DIR > 0 && j != 0) {
    const double2* w = tw + j * R;
#pragma unroll
    for (int m = 1; m < R; ++m) x[m] = zmul(x[m], __ldg(w + m));
  }
  zdft_small<R, DIR>(x);
  if (DIR < 0 && j != 0) {
    const double2* w = tw + j * R;
#pragma unroll
    for (int m = 1; m < R; ++m) x[m] = zmulc(x[m], __ldg(w + m));
  }
#pragma unroll
  for (int m = 0; m < R; ++m) base[m * q] = x[m];
}

// Prime stages in FP64: the H = (P-1)/2 output pairs split into NG groups of
// G; the table holds (cos, sin)(2 pi ((n k) mod P) / P) at [(g H + n - 1) G + j]
// for output k = g G + j + 1 and input n = 1..H (kks_fft64_prime_table).
template <int P>
struct ZPrime {
  static constexpr int H = (P - 1) / 2;
  static constexpr int G = P == 71 ? 5 : (P == 19 ? 3 : H);
  static constexpr int NG = H / G;
  static constexpr int TABLE = NG * H * G;
  static constexpr int FOLD = (H + NG - 1) / NG;
  static_assert(NG * G == H, "prime group size must divide (P-1)/2");
  static_assert(NG <= nt64<P>() / 32, "a round needs one warp per group");
};
static_assert(ZPrime<71>::TABLE <= KKS_FFT64_PRIME_TABLE_MAX && ZPrime<19>::TABLE <= KKS_FFT64_PRIME_TABLE_MAX &&
                  ZPrime<11>::TABLE <= KKS_FFT64_PRIME_TABLE_MAX,
              "FP64 prime table size");

__shared__ __align__(16) double2 s_zp11[ZPrime<11>::TABLE];
__shared__ __align__(16) double2 s_zp19[ZPrime<19>::TABLE];
__shared__ __align__(16) double2 s_zp71[ZPrime<71>::TABLE];

template <int P>
__device__ __forceinline__ double2* zprime_smem() {
  if constexpr (P == 11) return s_zp11;
  else if constexpr (P == 19) return s_zp19;
  else return s_zp71;
}

// Copy the axis's FP64 prime table into shared memory (before the first barrier).
template <int P>
__device__ __forceinline__ void zprime_fill(const double2* __restrict__ src) {
  if constexpr (P > 7) {
    double2* dst = zprime_smem<P>();
    for (int i = threadIdx.x; i < ZPrime<P>::TABLE; i += blockDim.x) dst[i] = __ldg(src + i);
  }
}

// The prime stage of nseq sequences of length n, in place: a warp takes 32
// DFTs (one per lane) and one output group; the input pairs are folded first
// (x[n] + x[P-n], x[n] - x[P-n]); outputs stay in registers until every warp
// of the round has read its inputs.
template <int P, int DIR>
__device__ __forceinline__ void zprime_stage(int nseq, int n, uint32_t pm) {
  using S = ZPrime<P>;
  constexpr int H = S::H, G = S::G, NG = S::NG;
  constexpr int W = nt64<P>() / 32, R = W / NG;
  extern __shared__ double2 zsm[];
  const int per = n / P;
  const int D = nseq * per;
  const int LG = (D + 31) >> 5;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int g = warp % NG;
  for (int lg0 = 0; lg0 < LG; lg0 += R) {
    const int lg = lg0 + warp / NG;
    const int d = (lg << 5) + lane;
    const bool has = warp < R * NG && lg < LG && d < D;
    double2* x = zsm;
    if (has) {
      const int sq = per == 1 ? d : (int)__umulhi((uint32_t)d, pm);
      x = zsm + sq * n + (d - sq * per) * P;
#pragma unroll
      for (int f = 0; f < S::FOLD; ++f) {
        const int nn = g * S::FOLD + f + 1;
        if (nn <= H) {
          const double2 a = x[nn], c = x[P - nn];
          x[nn] = zadd(a, c);
          x[P - nn] = zsub(a, c);
        }
      }
    }
    __syncthreads();
    double2 A[G], B[G], x0 = make_double2(0.0, 0.0), sum = make_double2(0.0, 0.0);
    if (has) {
      x0 = x[0];
      sum = x0;
#pragma unroll
      for (int j = 0; j < G; ++j) {
        A[j] = make_double2(0.0, 0.0);
        B[j] = make_double2(0.0, 0.0);
      }
      const double2* tw = zprime_smem<P>() + g * (H * G);
#pragma unroll 5
      for (int nn = 1; nn <= H; ++nn) {
        const double2 s = x[nn], dd = x[P - nn];
        if (g == 0) sum = zadd(sum, s);
#pragma unroll
        for (int j = 0; j < G; ++j) {
          const double2 w = tw[(nn - 1) * G + j];
          A[j].x += s.x * w.x;
          A[j].y += s.y * w.x;
          B[j].x += dd.x * w.y;
          B[j].y += dd.y * w.y;
        }
      }
    }
    __syncthreads();
    if (has) {
#pragma unroll
      for (int j = 0; j < G; ++j) {
        const int k = g * G + j + 1;
        const double ax = x0.x + A[j].x, ay = x0.y + A[j].y;
        if (DIR < 0) {
          x[k] = make_double2(ax + B[j].y, ay - B[j].x);
          x[P - k] = make_double2(ax - B[j].y, ay + B[j].x);
        } else {
          x[k] = make_double2(ax - B[j].y, ay + B[j].x);
          x[P - k] = make_double2(ax + B[j].y, ay - B[j].x);
        }
      }
      if (g == 0) x[0] = sum;
    }
  }
}

__device__ __forceinline__ int zfdiv(int x, int d, uint32_t m) {
  return d == 1 ? x : (int)__umulhi((uint32_t)x, m);
}

// nseq in-place transforms of length ax.n at the start of the block's dynamic
// shared memory: DIR = -1 forward DIF (natural -> digit-reversed), DIR = +1
// inverse DIT (digit-reversed -> natural), unnormalised. Ends with a barrier.
template <int DIR, int P>
__device__ __forceinline__ void zfft_run(int nseq, const KksFftAxis& ax) {
  extern __shared__ double2 zsm[];
  double2* buf = zsm;
  const int n = ax.n;
  for (int si = 0; si < ax.nst; ++si) {
    const int s = DIR < 0 ? si : ax.nst - 1 - si;
    const int r = ax.r[s];
    if constexpr (P > 7) {
      if (r == P) {
        zprime_stage<P, DIR>(nseq, n, ax.pm[s]);
        __syncthreads();
        continue;
      }
    }
    const int L = ax.L[s], q = ax.q[s];
    const int per = n / r;
    const uint32_t qm = ax.qm[s], pm = ax.pm[s];
    const double2* tw = ax.tw64 + ax.tw_off[s];
    const int total = nseq * per;
    for (int t = threadIdx.x; t < total; t += nt64<P>()) {
      const int sq = nseq == 1 ? 0 : zfdiv(t, per, pm);
      const int bt = t - sq * per;
      const int b = zfdiv(bt, q, qm);
      const int j = bt - b * q;
      double2* base = buf + sq * n + b * L + j;
      switch (r) {
        case 2: zbfly<2, DIR>(base, q, j, tw); break;
        case 3: zbfly<3, DIR>(base, q, j, tw); break;
        case 4: zbfly<4, DIR>(base, q, j, tw); break;
        case 5: zbfly<5, DIR>(base, q, j, tw); break;
        case 7: zbfly<7, DIR>(base, q, j, tw); break;
        default: break;
      }
    }
    __syncthreads();
  }
}

template <int NV, int NT>
__device__ __forceinline__ void zreduce_store(double (&v)[NV], double* out) {
  __shared__ double sh[NV][NT / 32];
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
#pragma unroll
    for (int k = 0; k < NV; ++k) {
      double x = lane < NT / 32 ? sh[k][lane] : 0.0;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
      if (lane == 0) out[k] = x;
    }
  }
}

__device__ __forceinline__ bool zin_iface(double e) { return e >= 0.1 && e <= 0.9; }

// Ask L2 for `bytes` (a multiple of 16) from a 16-byte aligned global address
// (one bulk prefetch, no data returned): the state rows a row pass reads
// after its transforms arrive in L2 while the transforms run.
__device__ __forceinline__ void zprefetch_l2(const void* p, uint32_t bytes) {
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(p), "r"(bytes) : "memory");
}

// Split the transform of (row a + i row b) (digit-reversed) into the half
// spectra of rows ix0 (a) and ix0+1 (b) of a column-major spectrum field.
template <int NT>
__device__ __forceinline__ void zsplit_store(const double2* z, const KksFftAxis& ay, double2* __restrict__ dst, int ix0,
                                             bool has1, int nx, int nyh) {
  const int ny = ay.n;
  for (int k = threadIdx.x; k < nyh; k += NT) {
    const double2 Zk = z[__ldg(ay.slot + k)];
    const double2 Zm = z[__ldg(ay.slot + (k == 0 ? 0 : ny - k))];
    double2* d = dst + (size_t)k * nx + ix0;
    d[0] = make_double2(0.5 * (Zk.x + Zm.x), 0.5 * (Zk.y - Zm.y));
    if (has1) d[1] = make_double2(0.5 * (Zk.y + Zm.y), -0.5 * (Zk.x - Zm.x));
  }
}

// Inverse of zsplit_store for F fields of a spectrum buffer (field f at src +
// f fs, into z + f ny; the y = 0 and Nyquist bins of a real row are real), the loads of U frequencies of every field issued before any
// store: each load is a 32-byte row-pair value from its own memory row, so
// several in flight per thread hide their latency.
template <int NT, int F>
__device__ __forceinline__ void zmerge_fields(double2* z, const KksFftAxis& ay, const double2* __restrict__ src,
                                              size_t fs, int ix0, bool has1, int nx, int nyh) {
  constexpr int U = 2;
  const int ny = ay.n;
  for (int k0 = threadIdx.x; k0 < nyh; k0 += U * NT) {
    double2 A[U][F], B[U][F];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int k = k0 + u * NT;
#pragma unroll
      for (int f = 0; f < F; ++f) {
        A[u][f] = make_double2(0.0, 0.0);
        B[u][f] = make_double2(0.0, 0.0);
        if (k < nyh) {
          const double2* sp = src + f * fs + (size_t)k * nx + ix0;
          A[u][f] = sp[0];
          if (has1) B[u][f] = sp[1];
        }
      }
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int k = k0 + u * NT;
      if (k >= nyh) continue;
      const bool self = k == 0 || 2 * k == ny;
      const int sk = __ldg(ay.slot + k);
      const int sm = self ? 0 : __ldg(ay.slot + (ny - k));
#pragma unroll
      for (int f = 0; f < F; ++f) {
        double2 a = A[u][f], b = B[u][f];
        if (self) {
          a.y = 0.0;
          b.y = 0.0;
        }
        z[f * ny + sk] = make_double2(a.x - b.y, a.y + b.x);
        if (!self) z[f * ny + sm] = make_double2(a.x + b.y, b.x - a.y);
      }
    }
  }
}

// d[0, n) = s[0, n) (global -> shared), four loads in flight per thread.
template <int NT>
__device__ __forceinline__ void zcopy_in(double2* d, const double2* __restrict__ s, int n) {
  constexpr int U = 4;
  for (int i0 = threadIdx.x; i0 < n; i0 += U * NT) {
    double2 v[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int i = i0 + u * NT;
      if (i < n) v[u] = s[i];
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int i = i0 + u * NT;
      if (i < n) d[i] = v[u];
    }
  }
}

// ---------------------------------------------------------------------------
// pass 1: one row pair: eta, X, eta^2 -> row spectra RA; old-state history
// sums and, at surface steps, the interface cells of rows ix0, ix0 + 1
// (pf_kks/microstructure.py:117-128; the same slots as the mixed rows_A).
template <int PY>
__global__ void __launch_bounds__(nt64<PY>(), minb64<PY>())
    kz_rows_A(const KksConst* __restrict__ c, const KksPar* __restrict__ par, const KksFftConst* __restrict__ fc,
              const double* __restrict__ eta, const double* __restrict__ X, double2* __restrict__ RA,
              double* __restrict__ partials) {
  constexpr int NT = nt64<PY>();
  if (!par->active) return;
  zprime_fill<PY>(fc->ay.ptw64);
  extern __shared__ double2 zsm[];
  const KksFftAxis& ay = fc->ay;
  const int nx = c->nx, ny = c->ny, nyh = c->nyh;
  const int bx = blockIdx.x, ix0 = 2 * bx;
  const bool has1 = ix0 + 1 < nx;
  const size_t i0 = (size_t)ix0 * ny;
  const bool surface = par->surface;
  double acc[6] = {0, 0, 0, 0, 0, 0};
  for (int y = threadIdx.x; y < ny; y += NT) {
    const double e0 = eta[i0 + y], x0 = X[i0 + y];
    const double e1 = has1 ? eta[i0 + ny + y] : 0.0, x1 = has1 ? X[i0 + ny + y] : 0.0;
    if (surface && y < ny - 1 && ix0 < nx - 1) {
      const double e0n = eta[i0 + y + 1], e1n = eta[i0 + ny + y + 1];
      const bool m1 = zin_iface(e1) && zin_iface(e1n);
      if (m1 && zin_iface(e0) && zin_iface(e0n)) acc[5] += 1.0;
      if (m1 && ix0 + 1 < nx - 1 && zin_iface(eta[i0 + 2 * ny + y]) && zin_iface(eta[i0 + 2 * ny + y + 1]))
        acc[5] += 1.0;
    }
    zsm[y] = make_double2(e0, e1);
    zsm[ny + y] = make_double2(x0, x1);
    zsm[2 * ny + y] = make_double2(e0 * e0, e1 * e1);
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
  zfft_run<-1, PY>(3, ay);
  const size_t fs = (size_t)nx * nyh;
  for (int f = 0; f < 3; ++f) zsplit_store<NT>(zsm + f * ny, ay, RA + f * fs, ix0, has1, nx, nyh);
  static_assert(P3_IFACE == P3_ETA + 5, "rows_A writes P3_ETA .. P3_IFACE");
  zreduce_store<6, NT>(acc, partials + (size_t)bx * KKS_NPART + P3_ETA);
}

// pass 2: fc->cols adjacent y-frequency columns of RA. Role by: 0 eta -> keep
// FT(eta), i k_x FT(eta) and i k_y FT(eta); 1 eta^2 -> tr eps^ (+ Parseval
// sums); 2 X -> keep FT(X) (k_spectral_mid<false> of kks_fields.cu, per column).
template <int PX>
__global__ void __launch_bounds__(nt64<PX>(), minb64<PX>())
    kz_cols_AB(const KksConst* __restrict__ c, const KksPar* __restrict__ par, const KksFftConst* __restrict__ fc,
               const double2* __restrict__ RA, double2* __restrict__ SA, double2* __restrict__ RB,
               const double* __restrict__ kys, double* __restrict__ partials) {
  constexpr int NT = nt64<PX>();
  if (!par->active) return;
  zprime_fill<PX>(fc->ax.ptw64);
  extern __shared__ double2 zsm[];
  const KksFftAxis& ax = fc->ax;
  const int nx = c->nx, ny = c->ny, nyh = c->nyh;
  const size_t fs = (size_t)nx * nyh;
  const int bx = blockIdx.x, g = blockIdx.y;
  const int cols = fc->cols;
  const int ky0 = bx * cols;
  const int ncol = min(cols, nyh - ky0);
  const int nv = ncol * nx;
  const int src_field = g == 0 ? 0 : (g == 1 ? 2 : 1);
  const double2* col = RA + src_field * fs + (size_t)ky0 * nx;
  zcopy_in<NT>(zsm, col, nv);
  __syncthreads();
  zfft_run<-1, PX>(ncol, ax);
  if (g != 1) {
    double2* dst = SA + (g == 2 ? fs : 0) + (size_t)ky0 * nx;
    for (int i = threadIdx.x; i < nv; i += NT) dst[i] = zsm[i];
    if (g == 2) return;
    __syncthreads();  // the columns are rewritten in place below by other threads
  }
  const double inv_N = c->inv_N;
  const double a = (par->epsX * c->c3) * inv_N;
  const double c11 = c->c11, c12 = c->c12;
  double acc[6] = {0, 0, 0, 0, 0, 0};
  for (int cc = 0; cc < ncol; ++cc) {
    const int iy = ky0 + cc;
    const double ky = kys[iy];
    const double w = (iy == 0 || 2 * iy == ny) ? 1.0 : 2.0;
    double2* z = zsm + cc * nx;
    for (int p = threadIdx.x; p < nx; p += NT) {
      const double kx = __ldg(fc->kx_slot64 + p);
      const double2 v = z[p];
      if (g == 0) {
        const double kxn = kx * inv_N, kyn = ky * inv_N;
        z[p] = make_double2(-kxn * v.y, kxn * v.x);
        z[nv + p] = make_double2(-kyn * v.y, kyn * v.x);
      } else {
        double oxx, oyy, oxy;
        strain_multipliers<double>(kx, ky, c11, c12, oxx, oyy, oxy);
        const double pw = w * (v.x * v.x + v.y * v.y);
        acc[0] += pw * oxx * oxx;
        acc[1] += pw * oyy * oyy;
        acc[2] += pw * oxx * oyy;
        acc[3] += pw * oxy * oxy;
        acc[4] += pw * (oxx + oyy);
        acc[5] += pw;
        const double st = a * (oxx + oyy);
        z[p] = make_double2(st * v.x, st * v.y);
      }
    }
  }
  if (g == 1) zreduce_store<6, NT>(acc, partials + (size_t)bx * KKS_NPART + P2_OXX2);
  __syncthreads();
  zfft_run<+1, PX>(g == 0 ? 2 * ncol : ncol, ax);
  if (g == 0) {
    double2* dx = RB + fs + (size_t)ky0 * nx;
    double2* dy = RB + 2 * fs + (size_t)ky0 * nx;
    for (int i = threadIdx.x; i < nv; i += NT) {
      dx[i] = zsm[i];
      dy[i] = zsm[nv + i];
    }
  } else {
    double2* dst = RB + (size_t)ky0 * nx;
    for (int i = threadIdx.x; i < nv; i += NT) dst[i] = zsm[i];
  }
}

// pass 3: one row pair of RB (tr eps, d_x eta, d_y eta) -> inverse FFT ->
// free_energy_terms of the old state, the Allen-Cahn drive and the
// Cahn-Hilliard fluxes (k_pre_pointwise<false>) -> forward FFT -> RC; sum G.
template <int PY>
__global__ void __launch_bounds__(nt64<PY>(), minb64<PY>())
    kz_rows_BC(const KksConst* __restrict__ c, const KksPar* __restrict__ par, const KksFftConst* __restrict__ fc,
               const double2* __restrict__ RB, double2* __restrict__ RC, const double* __restrict__ eta,
               const double* __restrict__ Xal, const double* __restrict__ Xth, double* g0, double* g1, double* g2,
               double* __restrict__ partials) {
  constexpr int NT = nt64<PY>();
  if (!par->active) return;
  zprime_fill<PY>(fc->ay.ptw64);
  extern __shared__ double2 zsm[];
  const KksFftAxis& ay = fc->ay;
  const int nx = c->nx, ny = c->ny, nyh = c->nyh;
  const size_t fs = (size_t)nx * nyh;
  const int bx = blockIdx.x, ix0 = 2 * bx;
  const bool has1 = ix0 + 1 < nx;
  if (threadIdx.x == 0) {  // rows ix0, ix0 + 1 of eta, X_al, X_th for the pointwise phase
    const size_t i0 = (size_t)ix0 * ny;
    const uint32_t bytes = (has1 ? 16u : 8u) * (uint32_t)ny;
    if ((bytes & 15u) == 0) {
      zprefetch_l2(eta + i0, bytes);
      zprefetch_l2(Xal + i0, bytes);
      zprefetch_l2(Xth + i0, bytes);
    }
  }
  zmerge_fields<NT, 3>(zsm, ay, RB, fs, ix0, has1, nx, nyh);
  __syncthreads();
  zfft_run<+1, PY>(3, ay);
  const KksPar q = *par;
  double* gs_buf = q.gs == 0 ? g0 : (q.gs == 1 ? g1 : g2);
  const double c3u = c->C11_0 + 2 * c->C12_0;
  const double epsX = q.epsX, C44 = q.C44;
  double accG = 0.0;
  for (int y = threadIdx.x; y < ny; y += NT) {
    const double2 tr = zsm[y], gx = zsm[ny + y], gy = zsm[2 * ny + y];
    double dr[2] = {0.0, 0.0}, fxv[2] = {0.0, 0.0}, fyv[2] = {0.0, 0.0};
#pragma unroll
    for (int r = 0; r < 2; ++r) {
      if (r == 1 && !has1) continue;
      const size_t i = (size_t)(ix0 + r) * ny + y;
      const double e = eta[i];
      const FreeEnergy f = free_energy(Xal[i], Xth[i], e, q);
      const double trv = r == 0 ? tr.x : tr.y;
      const double el_eta = 2 * epsX * e * c3u * (3 * epsX * (e * e) - trv);
      dr[r] = f.G_eta + el_eta / C44;
      fxv[r] = f.G_flux * (r == 0 ? gx.x : gx.y);
      fyv[r] = f.G_flux * (r == 0 ? gy.x : gy.y);
      if (q.armed_write) gs_buf[i] = f.G;
      accG += f.G;
    }
    zsm[y] = make_double2(dr[0], dr[1]);
    zsm[ny + y] = make_double2(fxv[0], fxv[1]);
    zsm[2 * ny + y] = make_double2(fyv[0], fyv[1]);
  }
  __syncthreads();
  zfft_run<-1, PY>(3, ay);
  for (int f = 0; f < 3; ++f) zsplit_store<NT>(zsm + f * ny, ay, RC + f * fs, ix0, has1, nx, nyh);
  double acc[1] = {accG};
  zreduce_store<1, NT>(acc, partials + (size_t)bx * KKS_NPART + P3_G);
}

// pass 4a: fc->cols columns of RC field 0 (FT of the drive) with FT(eta) from
// SA -> the new eta spectrum (eta^ + dt L FT(drive) ... / (1 + dt L kappa^2 k^2),
// k_spectral_update<false>) -> inverse x FFT -> RD field 0.
template <int PX>
__global__ void __launch_bounds__(nt64<PX>(), minb64<PX>())
    kz_cols_CD_eta(const KksConst* __restrict__ c, const KksPar* __restrict__ par, const KksFftConst* __restrict__ fc,
                   const double2* __restrict__ RC, const double2* __restrict__ SA, double2* __restrict__ RD,
                   const double* __restrict__ kys) {
  constexpr int NT = nt64<PX>();
  if (!par->active) return;
  zprime_fill<PX>(fc->ax.ptw64);
  extern __shared__ double2 zsm[];
  const KksFftAxis& ax = fc->ax;
  const int nx = c->nx, nyh = c->nyh;
  const int cols = fc->cols;
  const int ky0 = blockIdx.x * cols;
  const int ncol = min(cols, nyh - ky0);
  const int nv = ncol * nx;
  const double2* col = RC + (size_t)ky0 * nx;
  zcopy_in<NT>(zsm, col, nv);
  __syncthreads();
  zfft_run<-1, PX>(ncol, ax);
  const double inv_N = c->inv_N;
  const double ac_mul = par->ac_mul, ac_den = par->ac_den;
  for (int cc = 0; cc < ncol; ++cc) {
    const double ky = kys[ky0 + cc];
    const double2* ecol = SA + (size_t)(ky0 + cc) * nx;
    double2* z = zsm + cc * nx;
    for (int p = threadIdx.x; p < nx; p += NT) {
      const double kx = __ldg(fc->kx_slot64 + p);
      const double k2 = kx * kx + ky * ky;
      const double2 dh = z[p], eh = ecol[p];
      const double den = 1.0 + ac_den * k2;
      z[p] = make_double2((ac_mul * dh.x + eh.x) / den * inv_N, (ac_mul * dh.y + eh.y) / den * inv_N);
    }
  }
  __syncthreads();
  zfft_run<+1, PX>(ncol, ax);
  double2* dst = RD + (size_t)ky0 * nx;
  for (int i = threadIdx.x; i < nv; i += NT) dst[i] = zsm[i];
}

// pass 4b: the flux columns (RC fields 1, 2) with FT(X) from SA -> the new X
// spectrum (X^ + dt D sum_a i k_a FT(flux_a)) / (1 + dt k^2 D) -> RD field 1.
template <int PX>
__global__ void __launch_bounds__(nt64<PX>(), minb64<PX>())
    kz_cols_CD_X(const KksConst* __restrict__ c, const KksPar* __restrict__ par, const KksFftConst* __restrict__ fc,
                 const double2* __restrict__ RC, const double2* __restrict__ SA, double2* __restrict__ RD,
                 const double* __restrict__ kys) {
  constexpr int NT = nt64<PX>();
  if (!par->active) return;
  zprime_fill<PX>(fc->ax.ptw64);
  extern __shared__ double2 zsm[];
  const KksFftAxis& ax = fc->ax;
  const int nx = c->nx, nyh = c->nyh;
  const size_t fs = (size_t)nx * nyh;
  const int cols = fc->cols;
  const int ky0 = blockIdx.x * cols;
  const int ncol = min(cols, nyh - ky0);
  const int nv = ncol * nx;
  const double2* cx = RC + fs + (size_t)ky0 * nx;
  const double2* cy = RC + 2 * fs + (size_t)ky0 * nx;
  zcopy_in<NT>(zsm, cx, nv);
  zcopy_in<NT>(zsm + nv, cy, nv);
  __syncthreads();
  zfft_run<-1, PX>(2 * ncol, ax);
  const double inv_N = c->inv_N;
  const double ch_mul = par->ch_mul, dt = par->dt, D_s = par->D_s;
  for (int cc = 0; cc < ncol; ++cc) {
    const double ky = kys[ky0 + cc];
    const double2* xcol = SA + fs + (size_t)(ky0 + cc) * nx;
    double2* z = zsm + cc * nx;
    const double2* zy = zsm + nv + cc * nx;
    for (int p = threadIdx.x; p < nx; p += NT) {
      const double kx = __ldg(fc->kx_slot64 + p);
      const double k2 = kx * kx + ky * ky;
      const double2 fx = z[p], fy = zy[p];
      const double flx = -(kx * fx.y) - ky * fy.y;
      const double fly = kx * fx.x + ky * fy.x;
      const double2 xh = xcol[p];
      const double den = 1.0 + dt * k2 * D_s;
      z[p] = make_double2((ch_mul * flx + xh.x) / den * inv_N, (ch_mul * fly + xh.y) / den * inv_N);
    }
  }
  __syncthreads();
  zfft_run<+1, PX>(ncol, ax);
  double2* dst = RD + fs + (size_t)ky0 * nx;
  for (int i = threadIdx.x; i < nv; i += NT) dst[i] = zsm[i];
}

// pass 5: one row pair of RD -> eta_b, X_b (the new fields themselves); phase
// compositions, new free energy and diffusion potential, residual and history
// sums (k_post_pointwise<false>; the gradient-energy and interface sums of
// the new state come from the extras kernel, as in the mixed pipeline).
template <int PY>
__global__ void __launch_bounds__(nt64<PY>(), minb64<PY>())
    kz_rows_D(const KksConst* __restrict__ c, const KksPar* __restrict__ par, const KksFftConst* __restrict__ fc,
              const double2* __restrict__ RD, const double* __restrict__ X_o, double* __restrict__ eta_b,
              double* __restrict__ X_b, double* __restrict__ Xal_b, double* __restrict__ Xth_b,
              const double* __restrict__ eta_o, const double* __restrict__ eta_m, const double* __restrict__ X_m,
              double* __restrict__ mu, double* g0, double* g1, double* g2, double* __restrict__ partials) {
  constexpr int NT = nt64<PY>();
  if (!par->active) return;
  zprime_fill<PY>(fc->ay.ptw64);
  extern __shared__ double2 zsm[];
  const KksFftAxis& ay = fc->ay;
  const int nx = c->nx, ny = c->ny, nyh = c->nyh;
  const size_t fs = (size_t)nx * nyh;
  const int bx = blockIdx.x, ix0 = 2 * bx;
  const bool has1 = ix0 + 1 < nx;
  if (threadIdx.x == 0) {  // rows ix0, ix0 + 1 of the old X for the pointwise phase
    const uint32_t bytes = (has1 ? 16u : 8u) * (uint32_t)ny;
    const size_t i0 = (size_t)ix0 * ny;
    if ((bytes & 15u) == 0) {
      zprefetch_l2(X_o + i0, bytes);
      // armed attempts also read the pair's rows of mu, G- and the minus state
      const KksPar& qa = *par;
      if (qa.armed_write) zprefetch_l2(mu + i0, bytes);
      if (qa.armed_residual) {
        zprefetch_l2((qa.gm == 0 ? g0 : (qa.gm == 1 ? g1 : g2)) + i0, bytes);
        if (!qa.minus_is_state) {
          zprefetch_l2(eta_m + i0, bytes);
          zprefetch_l2(X_m + i0, bytes);
        }
      }
    }
  }
  zmerge_fields<NT, 2>(zsm, ay, RD, fs, ix0, has1, nx, nyh);
  __syncthreads();
  zfft_run<+1, PY>(2, ay);
  const KksPar q = *par;
  double* gb_buf = q.gb == 0 ? g0 : (q.gb == 1 ? g1 : g2);
  const double* gm_buf = q.gm == 0 ? g0 : (q.gm == 1 ? g1 : g2);
  const double* eta_minus = q.minus_is_state ? eta_o : eta_m;
  const double* X_minus = q.minus_is_state ? X_o : X_m;
  const double dt = q.dt;
  double acc[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  for (int y = threadIdx.x; y < ny; y += NT) {
    const double2 en = zsm[y], xn = zsm[ny + y];
#pragma unroll
    for (int r = 0; r < 2; ++r) {
      if (r == 1 && !has1) continue;
      const size_t i = (size_t)(ix0 + r) * ny + y;
      const double xo = X_o[i];
      const double eb = r == 0 ? en.x : en.y;
      const double xb = r == 0 ? xn.x : xn.y;
      eta_b[i] = eb;
      X_b[i] = xb;
      double xal, xth;
      phase_comp(xo, eb, q, xal, xth);
      Xal_b[i] = xal;
      Xth_b[i] = xth;
      if (eb < 0.05) { acc[0] += xb; acc[1] += 1.0; }
      if (eb > 0.95) { acc[2] += xb; acc[3] += 1.0; }
      acc[4] += eb;
      if (q.armed_write) {
        const FreeEnergy f = free_energy(xal, xth, eb, q);
        const double G_b = f.G, mu_b = f.mu;
        if (q.armed_residual) {
          const double mum = mu[i];
          const double dXdt = (xb - X_minus[i]) / dt;
          const double mu_mean = (mu_b + mum) / 2;
          const double diffusion = dXdt * mu_mean;
          const double detadt = (eb - eta_minus[i]) / dt;
          const double allen_cahn = q.inv_Ls * (detadt * detadt);
          const double temperature = (G_b - gm_buf[i]) / dt;
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
  double a5[5] = {acc[0], acc[1], acc[2], acc[3], acc[4]};
  zreduce_store<5, NT>(a5, partials + (size_t)bx * KKS_NPART + P5_XLO);
  __syncthreads();
  double a4[4] = {acc[5], acc[6], acc[7], acc[8]};
  zreduce_store<4, NT>(a4, partials + (size_t)bx * KKS_NPART + P5_DIFF);
}

// ---------------------------------------------------------------------------
// host side

// dynamic shared memory of each pass: its sequences, transformed in place
inline size_t zseq_smem(int n, int nseq) { return (size_t)nseq * n * sizeof(double2); }

template <int PY>
void zlaunch_rows(const KksFftLaunch& L, int p, int stage, cudaStream_t s) {
  const KksFieldPtrs& f = *L.f;
  const int q = 1 - p;
  const int npairs = kks_fft_row_blocks(L.nx);
  double2* RA = (double2*)L.RA;
  double2* RB = (double2*)L.RB;
  double* g0 = (double*)f.g[0];
  double* g1 = (double*)f.g[1];
  double* g2 = (double*)f.g[2];
  if (stage == 0) {
    kz_rows_A<PY><<<npairs, nt64<PY>(), zseq_smem(L.ny, 3), s>>>(L.dc, L.par, L.fc, (const double*)f.eta[p],
                                                                (const double*)f.X[p], RA, f.partials);
  } else if (stage == 1) {
    kz_rows_BC<PY><<<npairs, nt64<PY>(), zseq_smem(L.ny, 3), s>>>(
        L.dc, L.par, L.fc, RB, RA, (const double*)f.eta[p], (const double*)f.X_al[p], (const double*)f.X_th[p], g0,
        g1, g2, f.partials);
  } else {
    kz_rows_D<PY><<<npairs, nt64<PY>(), zseq_smem(L.ny, 2), s>>>(
        L.dc, L.par, L.fc, RB, (const double*)f.X[p], (double*)f.eta[q], (double*)f.X[q], (double*)f.X_al[q],
        (double*)f.X_th[q], (const double*)f.eta[p], (const double*)f.eta_m, (const double*)f.X_m, (double*)f.mu, g0,
        g1, g2, f.partials);
  }
}

template <int PX>
void zlaunch_cols(const KksFftLaunch& L, int stage, cudaStream_t s) {
  double2* RA = (double2*)L.RA;
  double2* RB = (double2*)L.RB;
  double2* SA = (double2*)L.SA;
  const int nb = kks_fft_col_blocks(L.nyh, L.cols);
  if (stage == 0) {
    kz_cols_AB<PX><<<dim3(nb, 3), nt64<PX>(), zseq_smem(L.nx, 2 * L.cols), s>>>(L.dc, L.par, L.fc, RA, SA, RB,
                                                                                 L.f->ky, L.f->partials);
  } else {
    kz_cols_CD_eta<PX><<<nb, nt64<PX>(), zseq_smem(L.nx, L.cols), s>>>(L.dc, L.par, L.fc, RA, SA, RB, L.f->ky);
    kz_cols_CD_X<PX><<<nb, nt64<PX>(), zseq_smem(L.nx, 2 * L.cols), s>>>(L.dc, L.par, L.fc, RA, SA, RB, L.f->ky);
  }
}

// The dynamic shared-memory limit of a kernel is process-wide and only raised.
template <typename K>
cudaError_t zset_attr(K* kernel, size_t smem) {
  cudaFuncAttributes fa;
  cudaError_t e = cudaFuncGetAttributes(&fa, kernel);
  if (e == cudaSuccess && (size_t)fa.maxDynamicSharedSizeBytes < smem)
    e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(kernel, cudaFuncAttributePreferredSharedMemoryCarveout, cudaSharedmemCarveoutMaxShared);
  return e;
}

template <int PY>
int zset_row_attrs(int ny) {
  cudaError_t e = zset_attr(kz_rows_A<PY>, zseq_smem(ny, 3));
  if (e == cudaSuccess) e = zset_attr(kz_rows_BC<PY>, zseq_smem(ny, 3));
  if (e == cudaSuccess) e = zset_attr(kz_rows_D<PY>, zseq_smem(ny, 2));
  return (int)e;
}

template <int PX>
int zset_col_attrs(int nx, int cols) {
  cudaError_t e = zset_attr(kz_cols_AB<PX>, zseq_smem(nx, 2 * cols));
  if (e == cudaSuccess) e = zset_attr(kz_cols_CD_eta<PX>, zseq_smem(nx, cols));
  if (e == cudaSuccess) e = zset_attr(kz_cols_CD_X<PX>, zseq_smem(nx, 2 * cols));
  return (int)e;
}

#define KKS_FFT64_DISPATCH(PVAL, CALL) \
  switch (PVAL) {                      \
    case 0: CALL(0); break;            \
    case 11: CALL(11); break;          \
    case 19: CALL(19); break;          \
    case 71: CALL(71); break;          \
    default: break;                    \
  }

template <int P>
int zprime_table(double2* t) {
  using S = ZPrime<P>;
  for (int g = 0; g < S::NG; ++g)
    for (int n = 1; n <= S::H; ++n)
      for (int j = 0; j < S::G; ++j) {
        const int k = g * S::G + j + 1;
        const double th = 2.0 * M_PI * (double)((n * k) % P) / (double)P;
        t[(g * S::H + n - 1) * S::G + j] = make_double2(cos(th), sin(th));
      }
  return S::TABLE;
}

}  // namespace

size_t kks_fft64_smem_bytes(int nx, int ny, int cols) {
  const size_t r = zseq_smem(ny, 3);
  const size_t c = zseq_smem(nx, 2 * cols);
  // + reduction scratch and the prime table
  return std::max(r, c) + 1024 + KKS_FFT64_PRIME_TABLE_MAX * sizeof(double2);
}

int kks_fft64_set_attributes(const KksFftLaunch& L) {
  int rc = -1, rc2 = -1;
#define KKS_ROWS_ATTR(P) rc = zset_row_attrs<P>(L.ny)
#define KKS_COLS_ATTR(P) rc2 = zset_col_attrs<P>(L.nx, L.cols)
  KKS_FFT64_DISPATCH(L.PY, KKS_ROWS_ATTR)
  KKS_FFT64_DISPATCH(L.PX, KKS_COLS_ATTR)
#undef KKS_ROWS_ATTR
#undef KKS_COLS_ATTR
  return rc != 0 ? rc : rc2;
}

int kks_fft64_prime_table(int P, double2* out) {
  switch (P) {
    case 11: return zprime_table<11>(out);
    case 19: return zprime_table<19>(out);
    case 71: return zprime_table<71>(out);
    default: return 0;
  }
}

void kks_fft64_launch_passes(const KksFftLaunch& L, int p, cudaStream_t s) {
#define KKS_ROWS(P) zlaunch_rows<P>(L, p, stage, s)
#define KKS_COLS(P) zlaunch_cols<P>(L, stage, s)
  int stage = 0;
  KKS_FFT64_DISPATCH(L.PY, KKS_ROWS)
  KKS_FFT64_DISPATCH(L.PX, KKS_COLS)
  stage = 1;
  KKS_FFT64_DISPATCH(L.PY, KKS_ROWS)
  KKS_FFT64_DISPATCH(L.PX, KKS_COLS)
  stage = 2;
  KKS_FFT64_DISPATCH(L.PY, KKS_ROWS)
#undef KKS_ROWS
#undef KKS_COLS
}
