// kks_fft.cu - the mixed-path attempt with hand-written shared-memory FFTs.
//
// cuFFT runs every 2-D transform as several factor passes over the whole batch
// (1420 = 4*5*71: eight kernels per transform, its prime-71 factor
// compute-bound), and the pointwise stages of the step are separate passes
// between the transforms. Here each 2-D transform is split into a row pass and
// a column pass, every 1-D transform runs in shared memory, and the pointwise
// stages are fused into the passes around them:
//
//   rows_A    eta, X (f64) rows -> eta, X, eta^2 row spectra (RA)       + old-state history sums
//   cols_AB   RA columns: forward FFT -> FT(eta), FT(X) kept (SA); tr eps^, i k_x FT(eta),
//             i k_y FT(eta) -> inverse FFT -> row spectra (RB)         + Parseval sums
//   rows_BC   RB rows: inverse FFT -> tr eps, d_x eta, d_y eta; Allen-Cahn drive and
//             Cahn-Hilliard fluxes (pointwise, old state) -> forward FFT -> RC  + sum G
//   cols_CD   RC columns: forward FFT; with SA the semi-implicit increments d_eta^, d_X^
//             -> inverse FFT -> row spectra (RD)
//   rows_D    RD rows: inverse FFT -> d_eta, d_X; new state, phase compositions, new free
//             energy, residual sums, new-state history sums
//   extras    np.gradient energy of the new state and, at surface steps, interface counts
//
// so that the spectra never make a round trip through HBM between a transform
// and the operation that consumes it. A row-pass block owns one pair of rows
// (all fields of the pass), each field's pair transformed as one complex
// sequence (row a + i row b) and split / merged with the Hermitian symmetry; a
// column-pass block owns fc->cols adjacent y-frequency columns (a launch shape,
// KKS_FFT_COLS unless tuned). A block has
// ten warps for two to six sequences, so that every stage (butterflies, the
// prime DFTs, loads and stores) has several warps of independent work. Spectra
// between passes are column-major (x fastest): a column pass moves one
// contiguous run, a row pass one 16-byte pair per frequency.
//
// Each 1-D transform is an in-place mixed-radix DIF (natural order in,
// digit-reversed out) for forward transforms and the matching DIT
// (digit-reversed in, natural out) for inverse ones, so spectra inside a
// column pass are indexed through a slot -> frequency table and no
// permutation pass exists. Radices 2, 3, 4, 5, 7 are butterflies with
// compile-time constants. One larger prime factor P (71 for 1420) is the last
// DIF stage (no twiddles): a direct DFT that folds its inputs into
// s_n = x_n + x_{P-n}, d_n = x_n - x_{P-n} and forms each output pair (k, P-k)
// from H = (P-1)/2 real-by-complex products on s and d. It runs as warp tasks:
// the lanes of a warp take 32 DFTs and one group of G output pairs, the warp's
// cos / sin factors come from a table in shared memory (one broadcast read per
// factor, uniform across the warp), and
// the outputs wait in registers for a block barrier before they overwrite the
// inputs, so the stage is in place and no thread holds the whole folded input.
// Only the mixed path uses these kernels (FP32 transforms on the increments of
// an FP64 state; see kks_fields.cu); the FP64 path keeps cuFFT.

#include <math.h>

#include <algorithm>
#include <vector>

#include <cuda.h>

#include "kks_internal.cuh"
#include "kks_fft.cuh"
#include "kks_check.cuh"

namespace {

// sites of the bounds-check build (kks_check.cuh): pass * 10 + check
enum {
  kSiteRowsA = 10, kSiteColsAB = 20, kSiteRowsBC = 30, kSiteColsCDeta = 40, kSiteColsCDX = 50, kSiteRowsD = 60,
  kSiteExtras = 70, kSiteFFT = 80
};

// The rows ix0 and ix0 + 1 (if any) of a row-pass block lie in the grid and its
// partial-sum row in the buffer.
__device__ __forceinline__ bool row_block_in_range(const KksConst* c, const KksFftConst* fc, int ix0, int bx, int site) {
  return KKS_IN((long long)(ix0 + 1 < c->nx ? ix0 + 1 : ix0) * c->ny + c->ny - 1, c->N, site) &&
         KKS_IN(bx, fc->part_cap, site + 1);
}

// The columns ky0 .. ky0 + ncol - 1 of a column-pass block lie in the half
// spectrum, its nseq columns in the launch's dynamic shared memory, and its
// partial-sum row in the buffer.
__device__ __forceinline__ bool col_block_in_range(const KksConst* c, const KksFftConst* fc, int ky0, int ncol, int nseq,
                                                   int bx, int site) {
  return KKS_IN(ky0 + ncol - 1, c->nyh, site) && KKS_IN((long long)nseq * c->nx * 8 - 1, kks_dyn_smem_bytes(), site + 1) &&
         KKS_IN(bx, fc->part_cap, site + 2);
}

constexpr int kThreads = KKS_FFT_THREADS;
// blocks per SM the register allocation must allow
constexpr int kMinBlocks = 2;
// Passes of grids without a large prime factor (small cells, whose blocks are
// short and latency-bound) ask for eight blocks of four warps per SM (64
// registers); the prime-stage passes keep two blocks of ten warps (their warp
// tasks need 96 registers), and rows_D keeps 96 registers (its FP64 pointwise
// phase would spill). A batched pass and its single-cell twin use
// the same bound, so that both compile to the same arithmetic.
template <int P>
__host__ __device__ constexpr int pass_min_blocks() {
  return P > 7 ? kMinBlocks : 8;
}
// Threads of a pass block: ten warps where a prime stage needs one warp per
// output group; four for grids without a large prime factor, whose rows and
// columns are short (a radix-4 stage of three 128-point sequences has 96
// butterflies), so that more, smaller blocks share an SM (measured on the
// 48-cell ensemble: 8 warps 1.20, 5 warps 0.84, 4 warps 0.81 ms per batch
// attempt).
template <int P>
__host__ __device__ constexpr int pass_threads() {
  return P > 7 ? kThreads : 128;
}
// rows_D (96 registers: its FP64 pointwise phase) keeps 20 warps per SM.
template <int P>
__host__ __device__ constexpr int rows_d_min_blocks() {
  return P > 7 ? kMinBlocks : 5;
}

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
  } else if constexpr (R == 8) {
    // two 4-point DFTs of the even and the odd values, combined with
    // w^k = exp(DIR 2 pi i k / 8): X_k = E_k + w^k O_k, X_{k+4} = E_k - w^k O_k
    float2 e[4] = {x[0], x[2], x[4], x[6]}, o[4] = {x[1], x[3], x[5], x[7]};
    dft_small<4, DIR>(e);
    dft_small<4, DIR>(o);
    constexpr float h = 0.707106781186547524f;  // sqrt(1/2)
    const float2 w1o = make_float2(h * (o[1].x - DIR * o[1].y), h * (o[1].y + DIR * o[1].x));
    const float2 w2o = DIR < 0 ? make_float2(o[2].y, -o[2].x) : make_float2(-o[2].y, o[2].x);
    const float2 w3o = make_float2(h * (-o[3].x - DIR * o[3].y), h * (-o[3].y + DIR * o[3].x));
    x[0] = cadd(e[0], o[0]);
    x[4] = csub(e[0], o[0]);
    x[1] = cadd(e[1], w1o);
    x[5] = csub(e[1], w1o);
    x[2] = cadd(e[2], w2o);
    x[6] = csub(e[2], w2o);
    x[3] = cadd(e[3], w3o);
    x[7] = csub(e[3], w3o);
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

// The butterfly of a stage with stride q = 1 (the last DIF / first DIT stage
// when the last radix is 2 or 4): its R values are contiguous and j = 0 (no
// twiddles), so they move as 16-byte pairs: one shared-memory access per pair
// instead of two 8-byte ones 16 or 32 bytes apart across the warp's lanes.
template <int R, int DIR>
__device__ __forceinline__ void bfly_contig(float2* base) {
  static_assert(R == 2 || R == 4, "pairs of values");
  float2 x[R];
  float4* b4 = reinterpret_cast<float4*>(base);
#pragma unroll
  for (int m = 0; m < R / 2; ++m) {
    const float4 v = b4[m];
    x[2 * m] = make_float2(v.x, v.y);
    x[2 * m + 1] = make_float2(v.z, v.w);
  }
  dft_small<R, DIR>(x);
#pragma unroll
  for (int m = 0; m < R / 2; ++m) b4[m] = make_float4(x[2 * m].x, x[2 * m].y, x[2 * m + 1].x, x[2 * m + 1].y);
}

// ---------------------------------------------------------------------------
// Prime stages. The H = (P-1)/2 output pairs (k, P-k) of a DFT are split into
// NG groups of G; the table of prime P holds (cos, sin)(2 pi ((n k) mod P) / P)
// at [(g H + n - 1) GP + j] for output k = g G + j + 1 and input n = 1..H, rows
// padded to an even GP so that a warp reads two (cos, sin) pairs per 16-byte
// load (computed on the host in double precision, see kks_fft_prime_table).
// Every pass kernel copies it into shared memory at entry: the warps of the
// five groups read different parts of the 11.2 KB table for P = 71, more than
// the constant cache holds, while a shared-memory read by a whole warp at one
// address is a single broadcast.
template <int P>
struct PrimeShape {
  static constexpr int H = (P - 1) / 2;
  static constexpr int G = P == 71 ? 7 : (P == 19 ? 3 : H);
  static constexpr int NG = H / G;
  static constexpr int GP = (G + 1) & ~1;
  static constexpr int TABLE = NG * H * GP;        // float2 entries
  static constexpr int FOLD = (H + NG - 1) / NG;   // input pairs each group's warp folds
  static_assert(NG * G == H, "prime group size must divide (P-1)/2");
  static_assert(NG <= kThreads / 32, "a round needs one warp per group");
};
static_assert(PrimeShape<71>::TABLE <= KKS_FFT_PRIME_TABLE_MAX && PrimeShape<19>::TABLE <= KKS_FFT_PRIME_TABLE_MAX &&
                  PrimeShape<11>::TABLE <= KKS_FFT_PRIME_TABLE_MAX,
              "prime table size");

__shared__ __align__(16) float2 s_ptw11[PrimeShape<11>::TABLE];
__shared__ __align__(16) float2 s_ptw19[PrimeShape<19>::TABLE];
__shared__ __align__(16) float2 s_ptw71[PrimeShape<71>::TABLE];

template <int P>
__device__ __forceinline__ float2* prime_tw_smem() {
  if constexpr (P == 11) return s_ptw11;
  else if constexpr (P == 19) return s_ptw19;
  else return s_ptw71;
}

// Copy the axis's prime table into shared memory (before the kernel's first
// barrier; nothing for axes without a prime stage).
template <int P>
__device__ __forceinline__ void prime_table_fill(const float2* __restrict__ src) {
  if constexpr (P > 7) {
    float4* dst = reinterpret_cast<float4*>(prime_tw_smem<P>());
    const float4* s4 = reinterpret_cast<const float4*>(src);
    for (int i = threadIdx.x; i < PrimeShape<P>::TABLE / 2; i += blockDim.x) dst[i] = __ldg(s4 + i);
  }
}

// The prime stage of nseq sequences of length n at the start of the block's
// dynamic shared memory, in place. DFT d = (sequence d / per, block d % per)
// covers d's P consecutive values. A warp takes 32 DFTs (one per lane) and one
// group g of output pairs; with W warps a round covers W / NG lane groups.
// First the input pairs are folded in place, x[n] <- x[n] + x[P-n] and
// x[P-n] <- x[n] - x[P-n] (each group's warp folds FOLD of them), so that the
// products read each folded value once per group; the outputs stay in
// registers until every warp of the round has read its inputs, then
// overwrite them.
template <int P, int DIR>
__device__ __forceinline__ void prime_stage(int nseq, int n, uint32_t pm) {
  using S = PrimeShape<P>;
  constexpr int H = S::H, G = S::G, NG = S::NG, GP = S::GP;
  constexpr int W = kThreads / 32, R = W / NG;
  extern __shared__ float2 sm[];
  const int per = n / P;
  const int D = nseq * per;
  const int LG = (D + 31) >> 5;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int g = warp % NG;
  for (int lg0 = 0; lg0 < LG; lg0 += R) {
    const int lg = lg0 + warp / NG;
    const int d = (lg << 5) + lane;
    const bool has = warp < R * NG && lg < LG && d < D;
    float2* x = sm;
    if (has) {
      const int sq = per == 1 ? d : (int)__umulhi((uint32_t)d, pm);
      x = sm + sq * n + (d - sq * per) * P;
#pragma unroll
      for (int f = 0; f < S::FOLD; ++f) {
        const int nn = g * S::FOLD + f + 1;
        if (nn <= H) {
          const float2 a = x[nn], c = x[P - nn];
          x[nn] = cadd(a, c);
          x[P - nn] = csub(a, c);
        }
      }
    }
    __syncthreads();
    float2 A[G], B[G], x0 = make_float2(0.f, 0.f), sum = make_float2(0.f, 0.f);
    if (has) {
      x0 = x[0];
      sum = x0;
#pragma unroll
      for (int j = 0; j < G; ++j) {
        A[j] = make_float2(0.f, 0.f);
        B[j] = make_float2(0.f, 0.f);
      }
      const float4* tw = reinterpret_cast<const float4*>(prime_tw_smem<P>() + g * (H * GP));
#pragma unroll
      for (int nn = 1; nn <= H; ++nn) {
        const float2 s = x[nn], dd = x[P - nn];
        if (g == 0) sum = cadd(sum, s);
#pragma unroll
        for (int jj = 0; jj < GP / 2; ++jj) {
          const float4 w = tw[(nn - 1) * (GP / 2) + jj];
          A[2 * jj].x += s.x * w.x;
          A[2 * jj].y += s.y * w.x;
          B[2 * jj].x += dd.x * w.y;
          B[2 * jj].y += dd.y * w.y;
          if (2 * jj + 1 < G) {
            A[2 * jj + 1].x += s.x * w.z;
            A[2 * jj + 1].y += s.y * w.z;
            B[2 * jj + 1].x += dd.x * w.w;
            B[2 * jj + 1].y += dd.y * w.w;
          }
        }
      }
    }
    __syncthreads();
    if (has) {
#pragma unroll
      for (int j = 0; j < G; ++j) {
        const int k = g * G + j + 1;
        const float ax = x0.x + A[j].x, ay = x0.y + A[j].y;
        if (DIR < 0) {
          x[k] = make_float2(ax + B[j].y, ay - B[j].x);
          x[P - k] = make_float2(ax - B[j].y, ay + B[j].x);
        } else {
          x[k] = make_float2(ax - B[j].y, ay + B[j].x);
          x[P - k] = make_float2(ax + B[j].y, ay - B[j].x);
        }
      }
      if (g == 0) x[0] = sum;
    }
  }
}

__device__ __forceinline__ int fdiv(int x, int d, uint32_t m) {
  return d == 1 ? x : (int)__umulhi((uint32_t)x, m);
}

// ---------------------------------------------------------------------------
// Bulk copies (global -> shared, completion counted on an mbarrier): a row
// pass stages the state rows its pointwise phase needs at kernel entry, so the
// loads overlap the merge and the inverse FFT. Source, destination and size
// are multiples of 16 bytes (the host enables this only for ny % 4 == 0).
constexpr int kWaitLimit = KKS_FFT_WAIT_POLLS;  // try_wait polls before a wait is declared lost

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(bar)) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}

__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// Wait for the phase of bar with the given parity, with a bounded number of
// polls (`polls`, the cell's KksFftConst::wait_polls). If it runs out the
// cell's status becomes KKS_STATUS_TIMEOUT (the host stops the run and reports
// it) and the block waits once more, bounded by kWaitLimit, for its copies in
// flight, so that no copy lands in shared memory after the block has moved on.
__device__ __forceinline__ void bulk_wait(uint64_t* bar, uint32_t parity, KksCtl* ctl, int polls) {
  bool done = false;
  for (int i = 0; i < polls && !done; ++i) done = mbar_try_wait(bar, parity);
  if (!done) {
    atomicCAS(&ctl->status, KKS_STATUS_OK, KKS_STATUS_TIMEOUT);
    for (int i = 0; i < kWaitLimit && !done; ++i) done = mbar_try_wait(bar, parity);
  }
}

// Orders this thread's generic shared-memory accesses before later bulk /
// tensor copies that read or overwrite the same bytes.
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// Tensor copies of a row pair's half spectra. A spectrum buffer is viewed as a
// 3-D tensor of 8-byte elements (x: nx, ky: nyh, field: F) and a box is
// {2, kb, F}: rows ix0, ix0 + 1 of kb consecutive frequencies of every field.
// Box b lands at stage + b * F * kb * 2 (float2 units) as [field][ky][x].
__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, int x, int y, int z, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
      "[%5];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
      : "memory");
}

__device__ __forceinline__ void tma_store_3d(const CUtensorMap* map, int x, int y, int z, const void* src) {
  asm volatile("cp.async.bulk.tensor.3d.global.shared::cta.tile.bulk_group [%0, {%1, %2, %3}], [%4];" ::"l"(
                   reinterpret_cast<uint64_t>(map)),
               "r"(x), "r"(y), "r"(z), "r"(smem_u32(src))
               : "memory");
}

// Commit the bulk stores issued by this thread and wait until they are done.
__device__ __forceinline__ void bulk_store_drain() {
  asm volatile("cp.async.bulk.commit_group;" ::: "memory");
  asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");
}

// Position of (frequency k, field f, row xi) in a staged box set with box
// height kb (256, or nyh when a single box holds them all).
__device__ __forceinline__ int stage_at(int k, int f, int F, int kb, int xi) {
  const int b = kb == 256 ? (k >> 8) : 0;
  return ((b * F + f) * kb + (k - b * kb)) * 2 + xi;
}

// The staging area: 128-byte aligned, after `seq_bytes` of sequences.
__device__ __forceinline__ char* stage_base(void* sm, uint32_t seq_bytes) {
  const uint32_t base = smem_u32(sm);
  const uint32_t off = ((base + seq_bytes + 127u) & ~127u) - base;
  return (char*)sm + off;
}

// nseq in-place transforms of length ax.n, sequence s at offset s * n of the
// block's dynamic shared memory. DIR = -1: forward DIF (natural ->
// digit-reversed); DIR = +1: inverse DIT (digit-reversed -> natural),
// unnormalised. P: the large prime of the axis (0 if none). Ends with a barrier.
template <int DIR, int P>
__device__ __forceinline__ void fft_run(int nseq, const KksFftAxis& ax) {
  extern __shared__ float2 sm[];
  float2* buf = sm;
  const int n = ax.n;
  // the sequences must lie in the launch's dynamic shared memory (a uniform
  // condition: the whole block skips the transform)
  if (!KKS_IN((long long)nseq * n * 8 - 1, kks_dyn_smem_bytes(), kSiteFFT)) {
    __syncthreads();
    return;
  }
  for (int si = 0; si < ax.nst; ++si) {
    const int s = DIR < 0 ? si : ax.nst - 1 - si;
    const int r = ax.r[s];
    if constexpr (P > 7) {
      if (r == P) {
        prime_stage<P, DIR>(nseq, n, ax.pm[s]);
        __syncthreads();
        continue;
      }
    }
    const int L = ax.L[s], q = ax.q[s];
    const int per = n / r;
    const uint32_t qm = ax.qm[s], pm = ax.pm[s];
    const float2* tw = ax.tw + ax.tw_off[s];
    const int total = nseq * per;
    // stride-1 stages of radix 2 / 4 on 16-byte aligned sequences: paired
    // loads (n even keeps every sequence and butterfly 16-byte aligned once the
    // dynamic shared memory is)
    if (q == 1 && (r == 2 || r == 4) && (n & 1) == 0 && (smem_u32(sm) & 15u) == 0) {
      for (int t = threadIdx.x; t < total; t += pass_threads<P>()) {
        const int sq = nseq == 1 ? 0 : fdiv(t, per, pm);
        float2* base = buf + sq * n + (t - sq * per) * r;
        if (r == 2) bfly_contig<2, DIR>(base);
        else bfly_contig<4, DIR>(base);
      }
      __syncthreads();
      continue;
    }
    for (int t = threadIdx.x; t < total; t += pass_threads<P>()) {
      const int sq = nseq == 1 ? 0 : fdiv(t, per, pm);
      const int bt = t - sq * per;
      const int b = fdiv(bt, q, qm);
      const int j = bt - b * q;
      float2* base = buf + sq * n + b * L + j;
      switch (r) {
        case 2: bfly_small<2, DIR>(base, q, j, tw); break;
        case 3: bfly_small<3, DIR>(base, q, j, tw); break;
        case 4: bfly_small<4, DIR>(base, q, j, tw); break;
        case 5: bfly_small<5, DIR>(base, q, j, tw); break;
        case 7: bfly_small<7, DIR>(base, q, j, tw); break;
        case 8:
          if constexpr (P <= 7) bfly_small<8, DIR>(base, q, j, tw);  // (axes with a large prime: radix <= 7)
          break;
        default: break;
      }
    }
    __syncthreads();
  }
}

template <int NV, int NT = kThreads>
__device__ __forceinline__ void block_reduce_store(double (&v)[NV], double* out) {
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
    const int lane2 = threadIdx.x;
#pragma unroll
    for (int k = 0; k < NV; ++k) {
      double x = lane2 < NT / 32 ? sh[k][lane2] : 0.0;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
      if (lane2 == 0) out[k] = x;
    }
  }
}

__device__ __forceinline__ bool in_iface(double e) { return e >= 0.1 && e <= 0.9; }

// Split the transform of (row a + i row b) (digit-reversed) into the half
// spectra of rows ix0 (a) and ix0+1 (b) of a column-major row-spectrum field.
template <int NT>
__device__ __forceinline__ void split_store(const float2* z, const KksFftAxis& ay, float2* __restrict__ dst, int ix0,
                                            bool has1, int nx, int nyh) {
  const int ny = ay.n;
  for (int k = threadIdx.x; k < nyh; k += NT) {
    const float2 Zk = z[__ldg(ay.slot + k)];
    const float2 Zm = z[__ldg(ay.slot + (k == 0 ? 0 : ny - k))];
    // A = (Z_k + conj Z_{-k}) / 2, B = (Z_k - conj Z_{-k}) / (2i)
    float2* d = dst + (size_t)k * nx + ix0;
    d[0] = make_float2(0.5f * (Zk.x + Zm.x), 0.5f * (Zk.y - Zm.y));
    if (has1) d[1] = make_float2(0.5f * (Zk.y + Zm.y), -0.5f * (Zk.x - Zm.x));
  }
}

// Inverse of split_store: z (digit-reversed) = A + i B over all ny
// frequencies, the negative ones from the Hermitian extension. The y = 0 and
// Nyquist bins of a real row are real: their imaginary round-off is dropped
// (as a C2R transform does), so that it cannot leak into the other row.
template <int NT>
__device__ __forceinline__ void merge_load(float2* z, const KksFftAxis& ay, const float2* __restrict__ src, int ix0,
                                           bool has1, int nx, int nyh) {
  const int ny = ay.n;
  for (int k = threadIdx.x; k < nyh; k += NT) {
    const float2* s = src + (size_t)k * nx + ix0;
    float2 A = s[0];
    float2 B = has1 ? s[1] : make_float2(0.f, 0.f);
    const bool self = k == 0 || 2 * k == ny;
    if (self) {
      A.y = 0.f;
      B.y = 0.f;
    }
    z[__ldg(ay.slot + k)] = make_float2(A.x - B.y, A.y + B.x);
    // conj(A) + i conj(B) at -k
    if (!self) z[__ldg(ay.slot + (ny - k))] = make_float2(A.x + B.y, B.x - A.y);
  }
}

// split_store / merge_load against a staged box set (field f of F) instead of
// global memory; the tensor copies move the boxes.
template <int NT>
__device__ __forceinline__ void split_stage(const float2* z, const KksFftAxis& ay, float2* stage, int f, int F,
                                            int kb, int nyh) {
  const int ny = ay.n;
  for (int k = threadIdx.x; k < nyh; k += NT) {
    const float2 Zk = z[__ldg(ay.slot + k)];
    const float2 Zm = z[__ldg(ay.slot + (k == 0 ? 0 : ny - k))];
    // rows x = 0, 1 of frequency k: one 16-byte store (the staging area is
    // 128-byte aligned and i is even)
    const int i = stage_at(k, f, F, kb, 0);
    *reinterpret_cast<float4*>(stage + i) =
        make_float4(0.5f * (Zk.x + Zm.x), 0.5f * (Zk.y - Zm.y), 0.5f * (Zk.y + Zm.y), -0.5f * (Zk.x - Zm.x));
  }
}

template <int NT>
__device__ __forceinline__ void merge_stage(float2* z, const KksFftAxis& ay, const float2* stage, int f, int F, int kb,
                                            int nyh) {
  const int ny = ay.n;
  for (int k = threadIdx.x; k < nyh; k += NT) {
    const int i = stage_at(k, f, F, kb, 0);
    const float4 v = *reinterpret_cast<const float4*>(stage + i);
    float2 A = make_float2(v.x, v.y), B = make_float2(v.z, v.w);
    const bool self = k == 0 || 2 * k == ny;
    if (self) {
      A.y = 0.f;
      B.y = 0.f;
    }
    z[__ldg(ay.slot + k)] = make_float2(A.x - B.y, A.y + B.x);
    if (!self) z[__ldg(ay.slot + (ny - k))] = make_float2(A.x + B.y, B.x - A.y);
  }
}

// Issue the tensor loads of all boxes of a row pair (thread 0) on bar.
__device__ __forceinline__ void stage_load(float2* stage, const CUtensorMap* map, int ix0, int F, int kb, int nb,
                                           uint64_t* bar) {
  mbar_expect_tx(bar, (uint32_t)(nb * F * kb * 16));
  for (int b = 0; b < nb; ++b) tma_load_3d(stage + b * F * kb * 2, map, ix0, b * kb, 0, bar);
}

// Store all boxes of a row pair (thread 0, after a fence and a barrier).
__device__ __forceinline__ void stage_store(const CUtensorMap* map, const float2* stage, int ix0, int F, int kb,
                                            int nb) {
  for (int b = 0; b < nb; ++b) tma_store_3d(map, ix0, b * kb, 0, stage + b * F * kb * 2);
  bulk_store_drain();
}

// ---------------------------------------------------------------------------
// pass 1: one row pair; the sequences are eta, X, eta^2 -> row spectra RA;
// old-state history sums and, at surface steps, the interface cells of rows
// ix0 and ix0 + 1 (corners in rows ix0 .. ix0 + 2; pf_kks/microstructure.py:117-128).
template <int PY>
__device__ __forceinline__ void rows_A_body(const KksConst* __restrict__ c, const KksPar* __restrict__ par, const KksFftConst* __restrict__ fc,
              const double* __restrict__ eta, const double* __restrict__ X, float2* __restrict__ RA,
              double* __restrict__ partials, KksCtl* ctl, int bulk, const CUtensorMap* map_RA, int bx) {
  constexpr int NT = pass_threads<PY>();
  if (!par->active) return;
  prime_table_fill<PY>(fc->ay.ptw);
  extern __shared__ float2 sm[];
  __shared__ __align__(8) uint64_t bar;
  const KksFftAxis& ay = fc->ay;
  const int nx = c->nx, ny = c->ny, nyh = c->nyh;
  const int ix0 = 2 * bx;
  const bool has1 = ix0 + 1 < nx;
  if (!row_block_in_range(c, fc, ix0, bx, kSiteRowsA)) return;
  const size_t i0 = (size_t)ix0 * ny;
  // staging after the three sequences: rows ix0, ix0+1 of eta and X, later
  // the three split half spectra of the pair
  char* stage = stage_base(sm, 3u * ny * (uint32_t)sizeof(float2));
  const double* s_eta = (const double*)stage;
  const double* s_X = s_eta + 2 * ny;
  if (bulk) {
    if (threadIdx.x == 0) mbar_init(&bar);
    __syncthreads();
    if (threadIdx.x == 0) {
      mbar_expect_tx(&bar, 32u * (uint32_t)ny);
      bulk_g2s((void*)s_eta, eta + i0, 16u * ny, &bar);
      bulk_g2s((void*)s_X, X + i0, 16u * ny, &bar);
    }
    bulk_wait(&bar, 0, ctl, fc->wait_polls);
  }
  const bool surface = par->surface;
  double acc[6] = {0, 0, 0, 0, 0, 0};
  for (int y = threadIdx.x; y < ny; y += NT) {
    double e0, x0, e1, x1;
    if (bulk) {
      e0 = s_eta[y], x0 = s_X[y], e1 = s_eta[ny + y], x1 = s_X[ny + y];
    } else {
      e0 = eta[i0 + y], x0 = X[i0 + y];
      e1 = has1 ? eta[i0 + ny + y] : 0.0, x1 = has1 ? X[i0 + ny + y] : 0.0;
    }
    if (surface && y < ny - 1 && ix0 < nx - 1) {  // ix0 < nx - 1: row ix0 + 1 exists
      const double e0n = bulk ? s_eta[y + 1] : eta[i0 + y + 1];
      const double e1n = bulk ? s_eta[ny + y + 1] : eta[i0 + ny + y + 1];
      const bool m1 = in_iface(e1) && in_iface(e1n);
      if (m1 && in_iface(e0) && in_iface(e0n)) acc[5] += 1.0;
      if (m1 && ix0 + 1 < nx - 1 && in_iface(eta[i0 + 2 * ny + y]) && in_iface(eta[i0 + 2 * ny + y + 1]))
        acc[5] += 1.0;
    }
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
  fft_run<-1, PY>(3, ay);
  const size_t fs = (size_t)nx * nyh;
  if (bulk) {
    const int kb = nyh < 256 ? nyh : 256, nb = (nyh + kb - 1) / kb;
    float2* st = (float2*)stage;
    for (int f = 0; f < 3; ++f) split_stage<NT>(sm + f * ny, ay, st, f, 3, kb, nyh);
    fence_async_smem();
    __syncthreads();
    if (threadIdx.x == 0) stage_store(map_RA, st, ix0, 3, kb, nb);
  } else {
    for (int f = 0; f < 3; ++f) split_store<NT>(sm + f * ny, ay, RA + f * fs, ix0, has1, nx, nyh);
  }
  static_assert(P3_IFACE == P3_ETA + 5, "rows_A writes P3_ETA .. P3_IFACE");
  block_reduce_store<6, NT>(acc, partials + (size_t)bx * KKS_NPART + P3_ETA);
}

template <int PY>
__global__ void __launch_bounds__(pass_threads<PY>(), pass_min_blocks<PY>())
    kf_rows_A(const KksConst* __restrict__ c, const KksPar* __restrict__ par, const KksFftConst* __restrict__ fc,
              const double* __restrict__ eta, const double* __restrict__ X, float2* __restrict__ RA,
              double* __restrict__ partials, KksCtl* ctl, int bulk, const __grid_constant__ CUtensorMap map_RA) {
  rows_A_body<PY>(c, par, fc, eta, X, RA, partials, ctl, bulk, &map_RA, (int)blockIdx.x);
}

// pass 2: fc->cols adjacent y-frequency columns of RA. Role by: 0 eta -> keep
// FT(eta), i k_x FT(eta) and i k_y FT(eta) (one forward, two inverse
// transforms); 1 eta^2 -> tr eps^ (+ Parseval sums); 2 X -> keep FT(X).
template <int PX>
__device__ __forceinline__ void cols_AB_body(const KksConst* __restrict__ c, const KksPar* __restrict__ par, const KksFftConst* __restrict__ fc,
               const float2* __restrict__ RA, float2* __restrict__ SA, float2* __restrict__ RB,
               const double* __restrict__ kys, double* __restrict__ partials, KksCtl* ctl, int bulk, int bx, int by) {
  constexpr int NT = pass_threads<PX>();
  if (!par->active) return;
  prime_table_fill<PX>(fc->ax.ptw);
  extern __shared__ float2 sm[];
  __shared__ __align__(8) uint64_t bar;
  bulk = bulk && (smem_u32(sm) & 15u) == 0;  // bulk destinations need 16-byte alignment
  const KksFftAxis& ax = fc->ax;
  const int nx = c->nx, ny = c->ny, nyh = c->nyh;
  const size_t fs = (size_t)nx * nyh;
  const int g = by;
  const int cols = fc->cols;
  const int ky0 = bx * cols;
  const int ncol = min(cols, nyh - ky0);
  const int nv = ncol * nx;
  if (!col_block_in_range(c, fc, ky0, ncol, g == 0 ? 2 * ncol : ncol, bx, kSiteColsAB)) return;
  const int src_field = g == 0 ? 0 : (g == 1 ? 2 : 1);
  const float2* col = RA + src_field * fs + (size_t)ky0 * nx;
  if (bulk) {  // the block's columns are one contiguous run: one bulk copy
    if (threadIdx.x == 0) {
      mbar_init(&bar);
      mbar_expect_tx(&bar, 8u * nv);
      bulk_g2s(sm, col, 8u * nv, &bar);
    }
    __syncthreads();
    bulk_wait(&bar, 0, ctl, fc->wait_polls);
  } else {
    for (int i = threadIdx.x; i < nv; i += NT) sm[i] = col[i];
    __syncthreads();
  }
  fft_run<-1, PX>(ncol, ax);
  if (g != 1) {
    float2* dst = SA + (g == 2 ? fs : 0) + (size_t)ky0 * nx;
    for (int i = threadIdx.x; i < nv; i += NT) dst[i] = sm[i];
    if (g == 2) return;
    // the eta role rewrites these columns in place below, element cc nx + p by
    // thread p % NT, which is not the thread that copied it unless NT divides
    // nx: every copy must have read its value first
    __syncthreads();
  }
  const float inv_N = (float)c->inv_N;
  const float a = (float)(par->epsX * c->c3) * inv_N;
  const float c11 = (float)c->c11, c12 = (float)c->c12;
  double acc[6] = {0, 0, 0, 0, 0, 0};
  for (int cc = 0; cc < ncol; ++cc) {
    const int iy = ky0 + cc;
    const float ky = (float)kys[iy];
    const double w = (iy == 0 || 2 * iy == ny) ? 1.0 : 2.0;
    float2* z = sm + cc * nx;
    for (int p = threadIdx.x; p < nx; p += NT) {
      const float kx = __ldg(fc->kx_slot + p);
      const float2 v = z[p];
      if (g == 0) {
        z[p] = make_float2(-kx * inv_N * v.y, kx * inv_N * v.x);
        z[nv + p] = make_float2(-ky * inv_N * v.y, ky * inv_N * v.x);
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
        const double pw = w * ((double)v.x * v.x + (double)v.y * v.y);
        const double dxx = oxx, dyy = oyy, dxy = oxy;
        acc[0] += pw * dxx * dxx;
        acc[1] += pw * dyy * dyy;
        acc[2] += pw * dxx * dyy;
        acc[3] += pw * dxy * dxy;
        acc[4] += pw * (dxx + dyy);
        acc[5] += pw;
        const float st = a * (oxx + oyy);
        z[p] = make_float2(st * v.x, st * v.y);
      }
    }
  }
  if (g == 1) block_reduce_store<6, NT>(acc, partials + (size_t)bx * KKS_NPART + P2_OXX2);
  __syncthreads();
  // g = 0: the i k_x columns at [0, nv), the i k_y columns at [nv, 2 nv)
  fft_run<+1, PX>(g == 0 ? 2 * ncol : ncol, ax);
  if (g == 0) {
    float2* dx = RB + fs + (size_t)ky0 * nx;
    float2* dy = RB + 2 * fs + (size_t)ky0 * nx;
    for (int i = threadIdx.x; i < nv; i += NT) {
      dx[i] = sm[i];
      dy[i] = sm[nv + i];
    }
  } else {
    float2* dst = RB + (size_t)ky0 * nx;
    for (int i = threadIdx.x; i < nv; i += NT) dst[i] = sm[i];
  }
}

template <int PX>
__global__ void __launch_bounds__(pass_threads<PX>(), pass_min_blocks<PX>())
    kf_cols_AB(const KksConst* __restrict__ c, const KksPar* __restrict__ par, const KksFftConst* __restrict__ fc,
               const float2* __restrict__ RA, float2* __restrict__ SA, float2* __restrict__ RB,
               const double* __restrict__ kys, double* __restrict__ partials, KksCtl* ctl, int bulk) {
  cols_AB_body<PX>(c, par, fc, RA, SA, RB, kys, partials, ctl, bulk, (int)blockIdx.x, (int)blockIdx.y);
}

// pass 3: one row pair of RB (tr eps, d_x eta, d_y eta) -> inverse FFT ->
// pointwise with the old state: the Allen-Cahn drive (free energy + elastic)
// and the Cahn-Hilliard fluxes -> forward FFT -> row spectra RC; sum G.
template <int PY>
__device__ __forceinline__ void rows_BC_body(const KksConst* __restrict__ c, const KksPar* __restrict__ par, const KksFftConst* __restrict__ fc,
               const float2* __restrict__ RB, float2* __restrict__ RC, const double* __restrict__ eta,
               const float* __restrict__ Xal, const float* __restrict__ Xth, float* g0, float* g1, float* g2,
               double* __restrict__ partials, KksCtl* ctl, int bulk, const CUtensorMap* map_RB,
               const CUtensorMap* map_RC, int bx) {
  constexpr int NT = pass_threads<PY>();
  if (!par->active) return;
  prime_table_fill<PY>(fc->ay.ptw);
  extern __shared__ float2 sm[];
  __shared__ __align__(8) uint64_t bar;
  const KksFftAxis& ay = fc->ay;
  const int nx = c->nx, ny = c->ny, nyh = c->nyh;
  const size_t fs = (size_t)nx * nyh;
  const int ix0 = 2 * bx;
  const bool has1 = ix0 + 1 < nx;
  if (!row_block_in_range(c, fc, ix0, bx, kSiteRowsBC)) return;
  const int kb = nyh < 256 ? nyh : 256, nb = (nyh + kb - 1) / kb;
  // staging after the three sequences: the pair's three half spectra (tensor
  // load), then rows ix0, ix0+1 of eta, X_al, X_th (bulk copies, overlapping
  // the inverse FFT), then the three split half spectra (tensor store)
  char* stage = stage_base(sm, 3u * ny * (uint32_t)sizeof(float2));
  float2* st = (float2*)stage;
  const double* s_eta = (const double*)stage;
  const float* s_al = (const float*)(s_eta + 2 * ny);
  const float* s_th = s_al + 2 * ny;
  if (bulk) {
    if (threadIdx.x == 0) {
      mbar_init(&bar);
      stage_load(st, map_RB, ix0, 3, kb, nb, &bar);
    }
    __syncthreads();
    bulk_wait(&bar, 0, ctl, fc->wait_polls);
    for (int f = 0; f < 3; ++f) merge_stage<NT>(sm + f * ny, ay, st, f, 3, kb, nyh);
    __syncthreads();
    if (threadIdx.x == 0) {
      const size_t i0 = (size_t)ix0 * ny;
      fence_async_smem();
      mbar_expect_tx(&bar, 32u * (uint32_t)ny);
      bulk_g2s((void*)s_eta, eta + i0, 16u * ny, &bar);
      bulk_g2s((void*)s_al, Xal + i0, 8u * ny, &bar);
      bulk_g2s((void*)s_th, Xth + i0, 8u * ny, &bar);
    }
  } else {
    for (int f = 0; f < 3; ++f) merge_load<NT>(sm + f * ny, ay, RB + f * fs, ix0, has1, nx, nyh);
    __syncthreads();
  }
  fft_run<+1, PY>(3, ay);
  if (bulk) bulk_wait(&bar, 1, ctl, fc->wait_polls);
  const KksPar q = *par;
  float* gs_buf = q.gs == 0 ? g0 : (q.gs == 1 ? g1 : g2);
  const float A_a = (float)q.A_alp_s, va = (float)q.va, fa0 = (float)q.fa0;
  const float A_t = (float)q.A_thet_s, vt = (float)q.vt, ft0 = (float)q.ft0, w_s = (float)q.w_s;
  const float epsX = (float)q.epsX;
  const float c3 = (float)((c->C11_0 + 2 * c->C12_0) * q.inv_C44);
  double accG = 0.0;
  for (int y = threadIdx.x; y < ny; y += NT) {
    const float2 tr = sm[y], gx = sm[ny + y], gy = sm[2 * ny + y];
    float dr[2], fxv[2], fyv[2];
#pragma unroll
    for (int r = 0; r < 2; ++r) {
      dr[r] = fxv[r] = fyv[r] = 0.f;
      if (r == 1 && !has1) continue;
      const size_t i = (size_t)(ix0 + r) * ny + y;
      const int is = r * ny + y;
      const float e = (float)(bulk ? s_eta[is] : eta[i]);
      const float ca = bulk ? s_al[is] : Xal[i], ct = bulk ? s_th[is] : Xth[i];
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
  fft_run<-1, PY>(3, ay);
  if (bulk) {
    for (int f = 0; f < 3; ++f) split_stage<NT>(sm + f * ny, ay, st, f, 3, kb, nyh);
    fence_async_smem();
    __syncthreads();
    if (threadIdx.x == 0) stage_store(map_RC, st, ix0, 3, kb, nb);
  } else {
    for (int f = 0; f < 3; ++f) split_store<NT>(sm + f * ny, ay, RC + f * fs, ix0, has1, nx, nyh);
  }
  double acc[1] = {accG};
  block_reduce_store<1, NT>(acc, partials + (size_t)bx * KKS_NPART + P3_G);
}

template <int PY>
__global__ void __launch_bounds__(pass_threads<PY>(), pass_min_blocks<PY>())
    kf_rows_BC(const KksConst* __restrict__ c, const KksPar* __restrict__ par, const KksFftConst* __restrict__ fc,
               const float2* __restrict__ RB, float2* __restrict__ RC, const double* __restrict__ eta,
               const float* __restrict__ Xal, const float* __restrict__ Xth, float* g0, float* g1, float* g2,
               double* __restrict__ partials, KksCtl* ctl, int bulk, const __grid_constant__ CUtensorMap map_RB,
               const __grid_constant__ CUtensorMap map_RC) {
  rows_BC_body<PY>(c, par, fc, RB, RC, eta, Xal, Xth, g0, g1, g2, partials, ctl, bulk, &map_RB, &map_RC, (int)blockIdx.x);
}

// pass 4a: fc->cols columns of FT(drive) with FT(eta) -> d_eta^ -> row spectra RD[0]
template <int PX>
__device__ __forceinline__ void cols_CD_eta_body(const KksConst* __restrict__ c, const KksPar* __restrict__ par, const KksFftConst* __restrict__ fc,
                   const float2* __restrict__ RC, const float2* __restrict__ SA, float2* __restrict__ RD,
                   const double* __restrict__ kys, KksCtl* ctl, int bulk, int bx) {
  constexpr int NT = pass_threads<PX>();
  if (!par->active) return;
  prime_table_fill<PX>(fc->ax.ptw);
  extern __shared__ float2 sm[];
  __shared__ __align__(8) uint64_t bar;
  bulk = bulk && (smem_u32(sm) & 15u) == 0;  // bulk destinations need 16-byte alignment
  const KksFftAxis& ax = fc->ax;
  const int nx = c->nx, nyh = c->nyh;
  const int cols = fc->cols;
  const int ky0 = bx * cols;
  const int ncol = min(cols, nyh - ky0);
  const int nv = ncol * nx;
  if (!col_block_in_range(c, fc, ky0, ncol, ncol, bx, kSiteColsCDeta)) return;
  const float2* col = RC + (size_t)ky0 * nx;
  // FT(eta) of the same columns, staged during the forward FFT
  float2* s_sa = (float2*)stage_base(sm, (uint32_t)(cols * nx * sizeof(float2)));
  if (bulk) {
    if (threadIdx.x == 0) {
      mbar_init(&bar);
      mbar_expect_tx(&bar, 8u * nv);
      bulk_g2s(sm, col, 8u * nv, &bar);
    }
    __syncthreads();
    bulk_wait(&bar, 0, ctl, fc->wait_polls);
    // every thread has seen phase 0 complete before the barrier is armed for
    // phase 1: a thread still polling parity 0 once phase 1 has completed too
    // would find phase 2 (parity 0) open and wait until its poll limit
    __syncthreads();
    if (threadIdx.x == 0) {
      mbar_expect_tx(&bar, 8u * nv);
      bulk_g2s(s_sa, SA + (size_t)ky0 * nx, 8u * nv, &bar);
    }
  } else {
    for (int i = threadIdx.x; i < nv; i += NT) sm[i] = col[i];
    __syncthreads();
  }
  fft_run<-1, PX>(ncol, ax);
  if (bulk) bulk_wait(&bar, 1, ctl, fc->wait_polls);
  const float inv_N = (float)c->inv_N;
  const float ac_mul = (float)par->ac_mul, ac_den = (float)par->ac_den;
  for (int cc = 0; cc < ncol; ++cc) {
    const float ky = (float)kys[ky0 + cc];
    const float2* ecol = bulk ? s_sa + cc * nx : SA + (size_t)(ky0 + cc) * nx;
    float2* z = sm + cc * nx;
    for (int p = threadIdx.x; p < nx; p += NT) {
      const float kx = __ldg(fc->kx_slot + p);
      const float k2 = kx * kx + ky * ky;
      const float2 dh = z[p];
      const float2 eh = ecol[p];
      const float ak = ac_den * k2, den = 1.f + ak;
      z[p] = make_float2((ac_mul * dh.x - ak * eh.x) / den * inv_N, (ac_mul * dh.y - ak * eh.y) / den * inv_N);
    }
  }
  __syncthreads();
  fft_run<+1, PX>(ncol, ax);
  float2* dst = RD + (size_t)ky0 * nx;
  for (int i = threadIdx.x; i < nv; i += NT) dst[i] = sm[i];
}

template <int PX>
__global__ void __launch_bounds__(pass_threads<PX>(), pass_min_blocks<PX>())
    kf_cols_CD_eta(const KksConst* __restrict__ c, const KksPar* __restrict__ par, const KksFftConst* __restrict__ fc,
                   const float2* __restrict__ RC, const float2* __restrict__ SA, float2* __restrict__ RD,
                   const double* __restrict__ kys, KksCtl* ctl, int bulk) {
  cols_CD_eta_body<PX>(c, par, fc, RC, SA, RD, kys, ctl, bulk, (int)blockIdx.x);
}

// pass 4b: fc->cols columns of FT(flux_x), FT(flux_y) with FT(X) -> d_X^ -> row spectra RD[1]
template <int PX>
__device__ __forceinline__ void cols_CD_X_body(const KksConst* __restrict__ c, const KksPar* __restrict__ par, const KksFftConst* __restrict__ fc,
                 const float2* __restrict__ RC, const float2* __restrict__ SA, float2* __restrict__ RD,
                 const double* __restrict__ kys, KksCtl* ctl, int bulk, int bx) {
  constexpr int NT = pass_threads<PX>();
  if (!par->active) return;
  prime_table_fill<PX>(fc->ax.ptw);
  extern __shared__ float2 sm[];
  __shared__ __align__(8) uint64_t bar;
  bulk = bulk && (smem_u32(sm) & 15u) == 0;  // bulk destinations need 16-byte alignment
  const KksFftAxis& ax = fc->ax;
  const int nx = c->nx, nyh = c->nyh;
  const size_t fs = (size_t)nx * nyh;
  const int cols = fc->cols;
  const int ky0 = bx * cols;
  const int ncol = min(cols, nyh - ky0);
  const int nv = ncol * nx;
  if (!col_block_in_range(c, fc, ky0, ncol, 2 * ncol, bx, kSiteColsCDX)) return;
  // flux_x columns at [0, nv), flux_y columns at [nv, 2 nv); FT(X) of the same
  // columns staged during the forward FFT
  const float2* cx = RC + fs + (size_t)ky0 * nx;
  const float2* cy = RC + 2 * fs + (size_t)ky0 * nx;
  float2* s_sa = (float2*)stage_base(sm, (uint32_t)(2 * cols * nx * sizeof(float2)));
  if (bulk) {
    if (threadIdx.x == 0) {
      mbar_init(&bar);
      mbar_expect_tx(&bar, 16u * nv);
      bulk_g2s(sm, cx, 8u * nv, &bar);
      bulk_g2s(sm + nv, cy, 8u * nv, &bar);
    }
    __syncthreads();
    bulk_wait(&bar, 0, ctl, fc->wait_polls);
    __syncthreads();  // phase 0 seen by every thread before phase 1 is armed (as in cols_CD_eta)
    if (threadIdx.x == 0) {
      mbar_expect_tx(&bar, 8u * nv);
      bulk_g2s(s_sa, SA + fs + (size_t)ky0 * nx, 8u * nv, &bar);
    }
  } else {
    for (int i = threadIdx.x; i < nv; i += NT) {
      sm[i] = cx[i];
      sm[nv + i] = cy[i];
    }
    __syncthreads();
  }
  fft_run<-1, PX>(2 * ncol, ax);
  if (bulk) bulk_wait(&bar, 1, ctl, fc->wait_polls);
  const float inv_N = (float)c->inv_N;
  const float ch_mul = (float)par->ch_mul;
  const float dtD = (float)(par->dt * par->D_s);
  for (int cc = 0; cc < ncol; ++cc) {
    const float ky = (float)kys[ky0 + cc];
    const float2* xcol = bulk ? s_sa + cc * nx : SA + fs + (size_t)(ky0 + cc) * nx;
    float2* z = sm + cc * nx;
    const float2* zy = sm + nv + cc * nx;
    for (int p = threadIdx.x; p < nx; p += NT) {
      const float kx = __ldg(fc->kx_slot + p);
      const float k2 = kx * kx + ky * ky;
      const float2 fx = z[p], fy = zy[p];
      const float flx = -(kx * fx.y) - ky * fy.y;
      const float fly = kx * fx.x + ky * fy.x;
      const float2 xh = xcol[p];
      const float bk = dtD * k2, den = 1.f + bk;
      z[p] = make_float2((ch_mul * flx - bk * xh.x) / den * inv_N, (ch_mul * fly - bk * xh.y) / den * inv_N);
    }
  }
  __syncthreads();
  fft_run<+1, PX>(ncol, ax);
  float2* dst = RD + fs + (size_t)ky0 * nx;
  for (int i = threadIdx.x; i < nv; i += NT) dst[i] = sm[i];
}

template <int PX>
__global__ void __launch_bounds__(pass_threads<PX>(), pass_min_blocks<PX>())
    kf_cols_CD_X(const KksConst* __restrict__ c, const KksPar* __restrict__ par, const KksFftConst* __restrict__ fc,
                 const float2* __restrict__ RC, const float2* __restrict__ SA, float2* __restrict__ RD,
                 const double* __restrict__ kys, KksCtl* ctl, int bulk) {
  cols_CD_X_body<PX>(c, par, fc, RC, SA, RD, kys, ctl, bulk, (int)blockIdx.x);
}

// Bulk prefetch of a contiguous range into L2 (no data returned), issued only
// where the range starts on a 16-byte boundary and spans whole 16-byte units,
// as the instruction requires; otherwise the later loads go to memory.
__device__ __forceinline__ void prefetch_rows_l2(const void* p, uint32_t bytes) {
  if ((((uintptr_t)p | bytes) & 15u) != 0 || bytes == 0) return;
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(p), "r"(bytes) : "memory");
}

// pass 5: one row pair of RD -> d_eta, d_X; new state, phase compositions,
// new free energy and diffusion potential, residual and history sums
template <int PY>
__device__ __forceinline__ void rows_D_body(const KksConst* __restrict__ c, const KksPar* __restrict__ par, const KksFftConst* __restrict__ fc,
              const float2* __restrict__ RD, const double* __restrict__ eta_o, const double* __restrict__ X_o,
              double* __restrict__ eta_b, double* __restrict__ X_b, float* __restrict__ Xal_b,
              float* __restrict__ Xth_b, const double* __restrict__ eta_m, const double* __restrict__ X_m,
              float* __restrict__ mu, float* g0, float* g1, float* g2, double* __restrict__ partials, KksCtl* ctl,
              int bulk, const CUtensorMap* map_RD, int bx) {
  constexpr int NT = pass_threads<PY>();
  if (!par->active) return;
  prime_table_fill<PY>(fc->ay.ptw);
  extern __shared__ float2 sm[];
  __shared__ __align__(8) uint64_t bar;
  const KksFftAxis& ay = fc->ay;
  const int nx = c->nx, ny = c->ny, nyh = c->nyh;
  const size_t fs = (size_t)nx * nyh;
  const int ix0 = 2 * bx;
  const bool has1 = ix0 + 1 < nx;
  if (!row_block_in_range(c, fc, ix0, bx, kSiteRowsD)) return;
  if (threadIdx.x == 0 && par->armed_write) {
    // armed attempts read the pair's rows of mu, G- and the minus state after
    // the transforms: bring them into L2 while the transforms run
    const KksPar& qa = *par;
    const size_t i0 = (size_t)ix0 * ny;
    const uint32_t rows = has1 ? 2u : 1u;
    prefetch_rows_l2(mu + i0, rows * 4u * (uint32_t)ny);
    if (qa.armed_residual) {
      const float* gm = qa.gm == 0 ? g0 : (qa.gm == 1 ? g1 : g2);
      prefetch_rows_l2(gm + i0, rows * 4u * (uint32_t)ny);
      if (!qa.minus_is_state) {
        prefetch_rows_l2(eta_m + i0, rows * 8u * (uint32_t)ny);
        prefetch_rows_l2(X_m + i0, rows * 8u * (uint32_t)ny);
      }
    }
  }
  // staging after the two sequences: the pair's two half spectra (tensor
  // load), then rows ix0, ix0+1 of the old eta and X (bulk copies,
  // overlapping the inverse FFT)
  char* stage = stage_base(sm, 2u * ny * (uint32_t)sizeof(float2));
  const double* s_eta = (const double*)stage;
  const double* s_X = s_eta + 2 * ny;
  if (bulk) {
    const int kb = nyh < 256 ? nyh : 256, nb = (nyh + kb - 1) / kb;
    float2* st = (float2*)stage;
    if (threadIdx.x == 0) {
      mbar_init(&bar);
      stage_load(st, map_RD, ix0, 2, kb, nb, &bar);
    }
    __syncthreads();
    bulk_wait(&bar, 0, ctl, fc->wait_polls);
    merge_stage<NT>(sm, ay, st, 0, 2, kb, nyh);
    merge_stage<NT>(sm + ny, ay, st, 1, 2, kb, nyh);
    __syncthreads();
    if (threadIdx.x == 0) {
      const size_t i0 = (size_t)ix0 * ny;
      fence_async_smem();
      mbar_expect_tx(&bar, 32u * (uint32_t)ny);
      bulk_g2s((void*)s_eta, eta_o + i0, 16u * ny, &bar);
      bulk_g2s((void*)s_X, X_o + i0, 16u * ny, &bar);
    }
  } else {
    merge_load<NT>(sm, ay, RD, ix0, has1, nx, nyh);
    merge_load<NT>(sm + ny, ay, RD + fs, ix0, has1, nx, nyh);
    __syncthreads();
  }
  fft_run<+1, PY>(2, ay);
  if (bulk) bulk_wait(&bar, 1, ctl, fc->wait_polls);
  const KksPar q = *par;
  float* gb_buf = q.gb == 0 ? g0 : (q.gb == 1 ? g1 : g2);
  const float* gm_buf = q.gm == 0 ? g0 : (q.gm == 1 ? g1 : g2);
  const double* eta_minus = q.minus_is_state ? eta_o : eta_m;
  const double* X_minus = q.minus_is_state ? X_o : X_m;
  const float A_a = (float)q.A_alp_s, va = (float)q.va, fa0 = (float)q.fa0;
  const float A_t = (float)q.A_thet_s, vt = (float)q.vt, ft0 = (float)q.ft0, w_s = (float)q.w_s;
  const double dt = q.dt;
  double acc[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  for (int y = threadIdx.x; y < ny; y += NT) {
    const float2 de = sm[y], dX = sm[ny + y];
#pragma unroll
    for (int r = 0; r < 2; ++r) {
      if (r == 1 && !has1) continue;
      const size_t i = (size_t)(ix0 + r) * ny + y;
      const int is = r * ny + y;
      // the residual's inputs first, so that their loads overlap the
      // phase-composition math (neither buffer is written before its use)
      float mu_m = 0.0f, g_m = 0.0f;
      double x_m = 0.0, e_m = 0.0;
      if (q.armed_residual) {
        mu_m = mu[i];
        g_m = gm_buf[i];
        x_m = X_minus[i];
        e_m = eta_minus[i];
      }
      const double xo = bulk ? s_X[is] : X_o[i];
      const double eb = (bulk ? s_eta[is] : eta_o[i]) + (double)(r == 0 ? de.x : de.y);
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
          const double mum = (double)mu_m;
          const double dXdt = (xb - x_m) / dt;
          const double mu_mean = ((double)mu_b + mum) / 2;
          const double diffusion = dXdt * mu_mean;
          const double detadt = (eb - e_m) / dt;
          const double allen_cahn = q.inv_Ls * (detadt * detadt);
          const double temperature = ((double)G_b - (double)g_m) / dt;
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
  block_reduce_store<5, NT>(a5, partials + (size_t)bx * KKS_NPART + P5_XLO);
  __syncthreads();
  double a4[4] = {acc[5], acc[6], acc[7], acc[8]};
  block_reduce_store<4, NT>(a4, partials + (size_t)bx * KKS_NPART + P5_DIFF);
}

template <int PY>
__global__ void __launch_bounds__(pass_threads<PY>(), rows_d_min_blocks<PY>())
    kf_rows_D(const KksConst* __restrict__ c, const KksPar* __restrict__ par, const KksFftConst* __restrict__ fc,
              const float2* __restrict__ RD, const double* __restrict__ eta_o, const double* __restrict__ X_o,
              double* __restrict__ eta_b, double* __restrict__ X_b, float* __restrict__ Xal_b,
              float* __restrict__ Xth_b, const double* __restrict__ eta_m, const double* __restrict__ X_m,
              float* __restrict__ mu, float* g0, float* g1, float* g2, double* __restrict__ partials, KksCtl* ctl,
              int bulk, const __grid_constant__ CUtensorMap map_RD) {
  rows_D_body<PY>(c, par, fc, RD, eta_o, X_o, eta_b, X_b, Xal_b, Xth_b, eta_m, X_m, mu, g0, g1, g2, partials, ctl, bulk, &map_RD, (int)blockIdx.x);
}

// np.gradient energy sum of a state (mode bit 0) and, at surface steps, its
// interface cell count (mode bit 1) into the given partial slots.
constexpr int kExtrasThreads = 256;

__device__ __forceinline__ void extras_body(const KksConst* __restrict__ c, const KksPar* __restrict__ par,
                                            const double* __restrict__ eta, int mode, int slot_grad, int slot_iface,
                                            double* __restrict__ partials, int bx, int nbk) {
  if (!par->active) return;
  const bool do_grad = mode & 1;
  const bool do_iface = (mode & 2) && par->surface;
  if (!do_grad && !do_iface) return;
  const int N = c->N, nx = c->nx, ny = c->ny;
  double acc[2] = {0, 0};
  // kU points per thread and iteration, their stencil loads issued together
  constexpr int kU = 4;
  const int stride = nbk * blockDim.x;
  for (int i0 = bx * blockDim.x + threadIdx.x; i0 < N; i0 += kU * stride) {
    double e[kU], xm[kU], xp[kU], ym[kU], yp[kU];
#pragma unroll
    for (int u = 0; u < kU; ++u) {
      const int i = i0 + u * stride;
      if (i < N) {
        const int ix = i / ny, iy = i - ix * ny;
        e[u] = eta[i];
        xm[u] = ix > 0 ? eta[i - ny] : 0.0;
        xp[u] = ix < nx - 1 ? eta[i + ny] : 0.0;
        ym[u] = iy > 0 ? eta[i - 1] : 0.0;
        yp[u] = iy < ny - 1 ? eta[i + 1] : 0.0;
      }
    }
#pragma unroll
    for (int u = 0; u < kU; ++u) {
      const int i = i0 + u * stride;
      if (i >= N) break;
      const int ix = i / ny, iy = i - ix * ny;
      if (do_grad) {
        double gx, gy;
        if (ix == 0) gx = xp[u] - e[u];
        else if (ix == nx - 1) gx = e[u] - xm[u];
        else gx = (xp[u] - xm[u]) / 2.0;
        if (iy == 0) gy = yp[u] - e[u];
        else if (iy == ny - 1) gy = e[u] - ym[u];
        else gy = (yp[u] - ym[u]) / 2.0;
        acc[0] += gx * gx + gy * gy;
      }
      if (do_iface && ix < nx - 1 && iy < ny - 1 && in_iface(e[u]) && in_iface(xp[u]) &&
          in_iface(eta[i + ny + 1]) && in_iface(yp[u]))
        acc[1] += 1.0;
    }
  }
  double a1[1] = {acc[0]};
  double a2[1] = {acc[1]};
  if (do_grad) block_reduce_store<1, kExtrasThreads>(a1, partials + (size_t)bx * KKS_NPART + slot_grad);
  __syncthreads();
  if (do_iface) block_reduce_store<1, kExtrasThreads>(a2, partials + (size_t)bx * KKS_NPART + slot_iface);
}

__global__ void __launch_bounds__(kExtrasThreads)
    kf_extras(const KksConst* __restrict__ c, const KksPar* __restrict__ par, const double* __restrict__ eta,
              int mode, int slot_grad, int slot_iface, double* __restrict__ partials) {
  extras_body(c, par, eta, mode, slot_grad, slot_iface, partials, (int)blockIdx.x, (int)gridDim.x);
}

// ---------------------------------------------------------------------------
// Batched passes (KksBatchLaunch): one launch covers every cell of a batch.
// Block b works on cell map[b].x as block map[b].y of that cell's own grid,
// with the cell's pointers from its descriptor and its state parity from the
// attempt's parameters (written by the batched prologue); a cell that takes
// no part in this attempt (target reached, or stopped) returns at once.

// Orders the host's writes of a tensor map held in global memory (a cell
// descriptor) before its use by tensor copies.
__device__ __forceinline__ void tensormap_acquire(const CUtensorMap* map) {
  asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;" ::"l"(map) : "memory");
}

template <int PY>
__global__ void __launch_bounds__(pass_threads<PY>(), pass_min_blocks<PY>())
    kfb_rows_A(const KksCellDesc* __restrict__ cells, const int2* __restrict__ bmap) {
  const int2 m = bmap[blockIdx.x];
  const KksCellDesc* d = cells + m.x;
  const int p = d->par->parity;
  if (threadIdx.x == 0 && d->bulk_rows) tensormap_acquire(&d->map_RA3);
  rows_A_body<PY>(d->dc, d->par, d->fc, d->eta[p], d->X[p], d->RA, d->partials, d->ctl, d->bulk_rows, &d->map_RA3,
                  m.y);
}

template <int PX>
__global__ void __launch_bounds__(pass_threads<PX>(), pass_min_blocks<PX>())
    kfb_cols_AB(const KksCellDesc* __restrict__ cells, const int2* __restrict__ bmap) {
  const int2 m = bmap[blockIdx.x];
  const KksCellDesc* d = cells + m.x;
  cols_AB_body<PX>(d->dc, d->par, d->fc, d->RA, d->SA, d->RB, d->ky, d->partials, d->ctl, d->bulk_cols,
                   m.y & 0xffff, m.y >> 16);
}

template <int PY>
__global__ void __launch_bounds__(pass_threads<PY>(), pass_min_blocks<PY>())
    kfb_rows_BC(const KksCellDesc* __restrict__ cells, const int2* __restrict__ bmap) {
  const int2 m = bmap[blockIdx.x];
  const KksCellDesc* d = cells + m.x;
  const int p = d->par->parity;
  if (threadIdx.x == 0 && d->bulk_rows) {
    tensormap_acquire(&d->map_RB3);
    tensormap_acquire(&d->map_RA3);
  }
  rows_BC_body<PY>(d->dc, d->par, d->fc, d->RB, d->RA, d->eta[p], d->X_al[p], d->X_th[p], d->g[0], d->g[1], d->g[2],
                   d->partials, d->ctl, d->bulk_rows, &d->map_RB3, &d->map_RA3, m.y);
}

template <int PX>
__global__ void __launch_bounds__(pass_threads<PX>(), pass_min_blocks<PX>())
    kfb_cols_CD_eta(const KksCellDesc* __restrict__ cells, const int2* __restrict__ bmap) {
  const int2 m = bmap[blockIdx.x];
  const KksCellDesc* d = cells + m.x;
  cols_CD_eta_body<PX>(d->dc, d->par, d->fc, d->RA, d->SA, d->RB, d->ky, d->ctl, d->bulk_cols, m.y);
}

template <int PX>
__global__ void __launch_bounds__(pass_threads<PX>(), pass_min_blocks<PX>())
    kfb_cols_CD_X(const KksCellDesc* __restrict__ cells, const int2* __restrict__ bmap) {
  const int2 m = bmap[blockIdx.x];
  const KksCellDesc* d = cells + m.x;
  cols_CD_X_body<PX>(d->dc, d->par, d->fc, d->RA, d->SA, d->RB, d->ky, d->ctl, d->bulk_cols, m.y);
}

template <int PY>
__global__ void __launch_bounds__(pass_threads<PY>(), rows_d_min_blocks<PY>())
    kfb_rows_D(const KksCellDesc* __restrict__ cells, const int2* __restrict__ bmap) {
  const int2 m = bmap[blockIdx.x];
  const KksCellDesc* d = cells + m.x;
  const int p = d->par->parity, q = p ^ 1;
  if (threadIdx.x == 0 && d->bulk_rows) tensormap_acquire(&d->map_RB2);
  rows_D_body<PY>(d->dc, d->par, d->fc, d->RB, d->eta[p], d->X[p], d->eta[q], d->X[q], d->X_al[q], d->X_th[q],
                  d->eta_m, d->X_m, d->mu, d->g[0], d->g[1], d->g[2], d->partials, d->ctl, d->bulk_rows, &d->map_RB2,
                  m.y);
}

// np.gradient energy and interface count of the candidate state
__global__ void __launch_bounds__(kExtrasThreads)
    kfb_extras(const KksCellDesc* __restrict__ cells, const int2* __restrict__ bmap) {
  const int2 m = bmap[blockIdx.x];
  const KksCellDesc* d = cells + m.x;
  const int q = d->par->parity ^ 1;
  extras_body(d->dc, d->par, d->eta[q], 3, P5_GRAD2, P5_IFACE, d->partials, m.y, d->nbx);
}

// After a rejection (decided by this attempt): the rejected candidate becomes
// the pair's minus entry and the step's input is copied back into the
// candidate buffer (k_restore of the single-cell attempt, per cell).
__global__ void __launch_bounds__(kExtrasThreads)
    kfb_restore(const KksCellDesc* __restrict__ cells, const int2* __restrict__ bmap) {
  const int2 m = bmap[blockIdx.x];
  const KksCellDesc* d = cells + m.x;
  const KksCtl* ctl = d->ctl;
  if (!d->par->active || !ctl->restore || ctl->status != KKS_STATUS_OK) return;
  const int p = d->par->parity, q = p ^ 1;
  const double* __restrict__ eta_i = d->eta[p];
  const double* __restrict__ X_i = d->X[p];
  const float* __restrict__ Xal_i = d->X_al[p];
  const float* __restrict__ Xth_i = d->X_th[p];
  double* __restrict__ eta_o = d->eta[q];
  double* __restrict__ X_o = d->X[q];
  float* __restrict__ Xal_o = d->X_al[q];
  float* __restrict__ Xth_o = d->X_th[q];
  double* __restrict__ eta_m = d->eta_m;
  double* __restrict__ X_m = d->X_m;
  const int N = d->N;
  for (int i = m.y * kExtrasThreads + threadIdx.x; i < N; i += d->nbx * kExtrasThreads) {
    eta_m[i] = eta_o[i];
    X_m[i] = X_o[i];
    eta_o[i] = eta_i[i];
    X_o[i] = X_i[i];
    Xal_o[i] = Xal_i[i];
    Xth_o[i] = Xth_i[i];
  }
}

// shared memory of each pass (bytes): its sequences, transformed in place,
// and for rows_BC / rows_D the staged state rows of the pair
inline size_t seq_smem(int n, int nseq) { return (size_t)nseq * n * sizeof(float2); }
// staging of a row pass: the larger of the pair's state rows (32 ny bytes)
// and its F staged half spectra (boxes of 2 x kb x F 8-byte elements), plus
// 128 bytes of alignment slack
inline size_t row_stage_bytes(int ny, int F) {
  const int nyh = ny / 2 + 1, kb = nyh < 256 ? nyh : 256, nb = (nyh + kb - 1) / kb;
  const size_t spec = (size_t)nb * F * kb * 16, rows = (size_t)32 * ny;
  return (spec > rows ? spec : rows) + 128;
}
inline size_t rows_a_smem(int ny) { return seq_smem(ny, 3) + row_stage_bytes(ny, 3); }
inline size_t rows_bc_smem(int ny) { return seq_smem(ny, 3) + row_stage_bytes(ny, 3); }
inline size_t rows_d_smem(int ny) { return seq_smem(ny, 2) + row_stage_bytes(ny, 2); }
// column increment passes: m x cols columns, and cols staged SA columns
inline size_t cols_cd_smem(int nx, int m, int cols) { return seq_smem(nx, m * cols) + 128 + seq_smem(nx, cols); }
inline int col_blocks(int nyh, int cols) { return (nyh + cols - 1) / cols; }

template <int PY>
void launch_rows(const KksFftLaunch& L, int p, int stage, cudaStream_t s) {
  const KksConst* dc = L.dc;
  const KksPar* par = L.par;
  const KksFieldPtrs& f = *L.f;
  const int q = 1 - p;
  const int npairs = kks_fft_row_blocks(L.nx);
  float2* RA = (float2*)L.RA;
  float2* RB = (float2*)L.RB;
  if (stage == 0) {
    kf_rows_A<PY><<<npairs, pass_threads<PY>(), rows_a_smem(L.ny), s>>>(dc, par, L.fc, (const double*)f.eta[p],
                                                               (const double*)f.X[p], RA, f.partials, L.ctl,
                                                               L.bulk_rows, L.map_RA3);
  } else if (stage == 1) {
    kf_rows_BC<PY><<<npairs, pass_threads<PY>(), rows_bc_smem(L.ny), s>>>(
        dc, par, L.fc, RB, RA, (const double*)f.eta[p], (const float*)f.X_al[p], (const float*)f.X_th[p],
        (float*)f.g[0], (float*)f.g[1], (float*)f.g[2], f.partials, L.ctl, L.bulk_rows, L.map_RB3, L.map_RA3);
  } else {
    kf_rows_D<PY><<<npairs, pass_threads<PY>(), rows_d_smem(L.ny), s>>>(
        dc, par, L.fc, RB, (const double*)f.eta[p], (const double*)f.X[p], (double*)f.eta[q], (double*)f.X[q],
        (float*)f.X_al[q], (float*)f.X_th[q], (const double*)f.eta_m, (const double*)f.X_m, (float*)f.mu,
        (float*)f.g[0], (float*)f.g[1], (float*)f.g[2], f.partials, L.ctl, L.bulk_rows, L.map_RB2);
  }
}

template <int PX>
void launch_cols(const KksFftLaunch& L, int stage, cudaStream_t s) {
  float2* RA = (float2*)L.RA;
  float2* RB = (float2*)L.RB;
  float2* SA = (float2*)L.SA;
  const int nb = col_blocks(L.nyh, L.cols);
  if (stage == 0) {
    kf_cols_AB<PX><<<dim3(nb, 3), pass_threads<PX>(), seq_smem(L.nx, 2 * L.cols), s>>>(
        L.dc, L.par, L.fc, RA, SA, RB, L.f->ky, L.f->partials, L.ctl, L.bulk_cols);
  } else {
    kf_cols_CD_eta<PX><<<nb, pass_threads<PX>(), cols_cd_smem(L.nx, 1, L.cols), s>>>(L.dc, L.par, L.fc, RA, SA, RB, L.f->ky,
                                                                            L.ctl, L.bulk_cols);
    kf_cols_CD_X<PX><<<nb, pass_threads<PX>(), cols_cd_smem(L.nx, 2, L.cols), s>>>(L.dc, L.par, L.fc, RA, SA, RB, L.f->ky,
                                                                          L.ctl, L.bulk_cols);
  }
}

// The dynamic shared-memory limit of a kernel is process-wide: it is only
// ever raised, so that a smaller cell created later does not lower the limit
// that the graphs of a larger one rely on.
template <typename K>
cudaError_t set_attr(K* kernel, size_t smem) {
  cudaFuncAttributes fa;
  cudaError_t e = cudaFuncGetAttributes(&fa, kernel);
  if (e == cudaSuccess && (size_t)fa.maxDynamicSharedSizeBytes < smem)
    e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(kernel, cudaFuncAttributePreferredSharedMemoryCarveout, cudaSharedmemCarveoutMaxShared);
  return e;
}

template <int PY>
void launch_rows_batch(const KksBatchLaunch& B, int stage, cudaStream_t s) {
  if (stage == 0)
    kfb_rows_A<PY><<<B.n_rows, pass_threads<PY>(), B.smem_rows_a, s>>>(B.cells, B.map_rows);
  else if (stage == 1)
    kfb_rows_BC<PY><<<B.n_rows, pass_threads<PY>(), B.smem_rows_bc, s>>>(B.cells, B.map_rows);
  else
    kfb_rows_D<PY><<<B.n_rows, pass_threads<PY>(), B.smem_rows_d, s>>>(B.cells, B.map_rows);
}

template <int PX>
void launch_cols_batch(const KksBatchLaunch& B, int stage, cudaStream_t s) {
  if (stage == 0) {
    kfb_cols_AB<PX><<<B.n_cols3, pass_threads<PX>(), B.smem_cols_ab, s>>>(B.cells, B.map_cols3);
  } else {
    kfb_cols_CD_eta<PX><<<B.n_cols, pass_threads<PX>(), B.smem_cols_cd1, s>>>(B.cells, B.map_cols);
    kfb_cols_CD_X<PX><<<B.n_cols, pass_threads<PX>(), B.smem_cols_cd2, s>>>(B.cells, B.map_cols);
  }
}

template <int PY>
int set_row_batch_attrs(const KksBatchLaunch& B) {
  cudaError_t e = set_attr(kfb_rows_A<PY>, B.smem_rows_a);
  if (e == cudaSuccess) e = set_attr(kfb_rows_BC<PY>, B.smem_rows_bc);
  if (e == cudaSuccess) e = set_attr(kfb_rows_D<PY>, B.smem_rows_d);
  return (int)e;
}

template <int PX>
int set_col_batch_attrs(const KksBatchLaunch& B) {
  cudaError_t e = set_attr(kfb_cols_AB<PX>, B.smem_cols_ab);
  if (e == cudaSuccess) e = set_attr(kfb_cols_CD_eta<PX>, B.smem_cols_cd1);
  if (e == cudaSuccess) e = set_attr(kfb_cols_CD_X<PX>, B.smem_cols_cd2);
  return (int)e;
}

template <int PY>
int set_row_attrs(int ny) {
  cudaError_t e = set_attr(kf_rows_A<PY>, rows_a_smem(ny));
  if (e == cudaSuccess) e = set_attr(kf_rows_BC<PY>, rows_bc_smem(ny));
  if (e == cudaSuccess) e = set_attr(kf_rows_D<PY>, rows_d_smem(ny));
  return (int)e;
}

template <int PX>
int set_col_attrs(int nx, int cols) {
  cudaError_t e = set_attr(kf_cols_AB<PX>, seq_smem(nx, 2 * cols));
  if (e == cudaSuccess) e = set_attr(kf_cols_CD_eta<PX>, cols_cd_smem(nx, 1, cols));
  if (e == cudaSuccess) e = set_attr(kf_cols_CD_X<PX>, cols_cd_smem(nx, 2, cols));
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

template <int P>
int prime_table(float2* t) {
  using S = PrimeShape<P>;
  for (int i = 0; i < S::TABLE; ++i) t[i] = make_float2(0.f, 0.f);
  for (int g = 0; g < S::NG; ++g)
    for (int n = 1; n <= S::H; ++n)
      for (int j = 0; j < S::G; ++j) {
        const int k = g * S::G + j + 1;
        const double th = 2.0 * M_PI * (double)((n * k) % P) / (double)P;
        t[(g * S::H + n - 1) * S::GP + j] = make_float2((float)cos(th), (float)sin(th));
      }
  return S::TABLE;
}

}  // namespace

size_t kks_fft_smem_bytes(int nx, int ny, int cols) {
  const size_t r = rows_bc_smem(ny) > rows_d_smem(ny) ? rows_bc_smem(ny) : rows_d_smem(ny);
  const size_t c = std::max(cols_cd_smem(nx, 2, cols), seq_smem(nx, 2 * cols));
  return (r > c ? r : c) + 1024 + KKS_FFT_PRIME_TABLE_MAX * sizeof(float2);  // + reduction scratch and prime table
}

int kks_fft_row_blocks(int nx) { return (nx + 1) / 2; }

int kks_fft_partial_rows(int nx, int ny, int nbx) {
  int m = kks_fft_row_blocks(nx);
  const int cb = col_blocks(ny / 2 + 1, 1);  // the column pass that writes sums, at its finest tile
  if (cb > m) m = cb;
  return m > nbx ? m : nbx;
}

// The large prime of each axis selects the kernel instantiation.
int kks_fft_set_attributes(const KksFftLaunch& L) {
  if (L.f64) return kks_fft64_set_attributes(L);
  int rc = -1, rc2 = -1;
#define KKS_ROWS_ATTR(P) rc = set_row_attrs<P>(L.ny)
#define KKS_COLS_ATTR(P) rc2 = set_col_attrs<P>(L.nx, L.cols)
  KKS_FFT_DISPATCH(L.PY, KKS_ROWS_ATTR)
  KKS_FFT_DISPATCH(L.PX, KKS_COLS_ATTR)
#undef KKS_ROWS_ATTR
#undef KKS_COLS_ATTR
  return rc != 0 ? rc : rc2;
}

int kks_fft_bounds_word(unsigned long long* first, int reset) {
  *first = 0;
#ifdef KKS_BOUNDS_CHECK
  if (cudaMemcpyFromSymbol(first, g_kks_oob, sizeof(unsigned long long)) != cudaSuccess) return -1;
  if (reset) {
    const unsigned long long zero = 0;
    if (cudaMemcpyToSymbol(g_kks_oob, &zero, sizeof(zero)) != cudaSuccess) return -1;
  }
  return 1;
#else
  (void)reset;
  return 0;
#endif
}

int kks_fft_prime_table(int P, float2* out) {
  switch (P) {
    case 11: return prime_table<11>(out);
    case 19: return prime_table<19>(out);
    case 71: return prime_table<71>(out);
    default: return 0;
  }
}

void kks_fft_launch_attempt(const KksFftLaunch& L, int p, cudaStream_t s) {
  const KksFieldPtrs& f = *L.f;
  if (L.f64) {
    kks_fft64_launch_passes(L, p, s);
  } else {
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
  }
  // the stencil pass is bound by load latency: give it at least one block per
  // row pair (the decide kernel reduces that many partial-sum rows anyway)
  const int ge = std::max(L.nbx, kks_fft_row_blocks(L.nx));
  kf_extras<<<ge, kExtrasThreads, 0, s>>>(L.dc, L.par, (const double*)f.eta[1 - p], 3, P5_GRAD2, P5_IFACE,
                                          f.partials);
}

int kks_fft_col_blocks(int nyh, int cols) { return col_blocks(nyh, cols); }

int kks_fft_batch_prepare(KksBatchLaunch& B, const int* nx, const int* ny, const int* cols, int n) {
  size_t ra = 0, rbc = 0, rd = 0, cab = 0, ccd1 = 0, ccd2 = 0;
  for (int i = 0; i < n; ++i) {
    ra = std::max(ra, rows_a_smem(ny[i]));
    rbc = std::max(rbc, rows_bc_smem(ny[i]));
    rd = std::max(rd, rows_d_smem(ny[i]));
    cab = std::max(cab, seq_smem(nx[i], 2 * cols[i]));
    ccd1 = std::max(ccd1, cols_cd_smem(nx[i], 1, cols[i]));
    ccd2 = std::max(ccd2, cols_cd_smem(nx[i], 2, cols[i]));
  }
  B.smem_rows_a = ra;
  B.smem_rows_bc = rbc;
  B.smem_rows_d = rd;
  B.smem_cols_ab = cab;
  B.smem_cols_cd1 = ccd1;
  B.smem_cols_cd2 = ccd2;
  int rc = -1, rc2 = -1;
#define KKS_ROWS_ATTR(P) rc = set_row_batch_attrs<P>(B)
#define KKS_COLS_ATTR(P) rc2 = set_col_batch_attrs<P>(B)
  KKS_FFT_DISPATCH(B.PY, KKS_ROWS_ATTR)
  KKS_FFT_DISPATCH(B.PX, KKS_COLS_ATTR)
#undef KKS_ROWS_ATTR
#undef KKS_COLS_ATTR
  if (rc == 0 && rc2 == 0) {
    cudaError_t e = cudaFuncSetAttribute(kfb_extras, cudaFuncAttributePreferredSharedMemoryCarveout,
                                         cudaSharedmemCarveoutMaxShared);
    rc = (int)e;
  }
  return rc != 0 ? rc : rc2;
}

void kks_fft_launch_attempt_batch(const KksBatchLaunch& B, cudaStream_t s) {
  kks_launch_prologue_batch(B.cells, B.n_cells, s);
#define KKS_ROWS(P) launch_rows_batch<P>(B, stage, s)
#define KKS_COLS(P) launch_cols_batch<P>(B, stage, s)
  int stage = 0;
  KKS_FFT_DISPATCH(B.PY, KKS_ROWS)
  KKS_FFT_DISPATCH(B.PX, KKS_COLS)
  stage = 1;
  KKS_FFT_DISPATCH(B.PY, KKS_ROWS)
  KKS_FFT_DISPATCH(B.PX, KKS_COLS)
  stage = 2;
  KKS_FFT_DISPATCH(B.PY, KKS_ROWS)
#undef KKS_ROWS
#undef KKS_COLS
  kfb_extras<<<B.n_extras, kExtrasThreads, 0, s>>>(B.cells, B.map_extras);
  kks_launch_decide_batch(B.cells, B.n_cells, s);
  kfb_restore<<<B.n_extras, kExtrasThreads, 0, s>>>(B.cells, B.map_extras);
}
