// kks_init.cu - initial state of a cell written on the device.
//
// The fields are created where the step reads them instead of being built on
// the host and copied in:
//   * the seeded synthetic microstructure of the benchmark workloads: periodic
//     Voronoi labels and their edge pixels, particles centred on ranked edge
//     pixels, a diffuse order parameter (max over particles of a tanh profile
//     stamped in a periodic window), a noisy matrix composition and the closed
//     KKS phase compositions (pf_kks/free_energy.py:74-95). The host keeps the
//     few draws of numpy's PCG64 stream that are per particle; the per-point
//     matrix noise is drawn here from the same stream by jumping the 128-bit
//     LCG ahead (Brown, "Random number generation with arbitrary strides",
//     1994), so the arrays equal the host generator's;
//   * sharp precipitates and nuclei (pf_kks/microstructure.py:7-74);
//   * nuclei at ranked candidate points (pf_kks/nucleation.py:103-111).
//
// Ordered selection ("the k-th point, in C order, that satisfies a predicate",
// numpy's flatnonzero(mask)[k]) is done without compacting the whole mask:
// per-chunk counts, one exclusive scan over the chunks, then one block per
// rank scans its chunk.
//
// Compiled with -fmad=false: every product and sum rounds on its own, as in
// numpy, so the integer outcomes (labels, edge pixels, inside tests) and the
// noise equal the host's bit for bit.

#include <math.h>

#include "kks_internal.cuh"

namespace {

constexpr int kT = 256;
constexpr int kChunk = 1024;  // points per chunk of the ordered selection (kT x 4)
constexpr int kTileX = 16, kTileY = 64;  // eta tile: 16 rows (x) x 64 columns (y)
constexpr int kBatch = 256;  // particles or seeds staged in shared memory at a time

typedef unsigned __int128 u128;

// PCG64 (XSL-RR 128/64) as numpy.random.PCG64 runs it: step the LCG, then
// output from the new state. The LCG multiplier is O'Neill's default 128-bit one.
__device__ __forceinline__ u128 pcg_mult() { return ((u128)0x2360ED051FC65DA4ull << 64) | (u128)0x4385DF649FCCF645ull; }

__device__ __forceinline__ uint64_t pcg_output(u128 s) {
  const uint64_t x = (uint64_t)(s >> 64) ^ (uint64_t)s;
  const unsigned rot = (unsigned)(s >> 122);
  return (x >> rot) | (x << ((64u - rot) & 63u));
}

// The affine map of d LCG steps, s -> mult * s + plus.
__device__ void lcg_jump(unsigned long long d, u128 inc, u128& mult, u128& plus) {
  u128 cm = pcg_mult(), cp = inc, am = 1, ap = 0;
  while (d) {
    if (d & 1ull) {
      am *= cm;
      ap = ap * cm + cp;
    }
    cp = (cm + 1) * cp;
    cm *= cm;
    d >>= 1;
  }
  mult = am;
  plus = ap;
}

__device__ __forceinline__ int pmod(int a, int n) {
  const int r = a % n;
  return r < 0 ? r + n : r;
}

// Minimum-image difference a - n * round_half_even(a / n).
__device__ __forceinline__ double periodic_delta(double a, double n) { return a - n * rint(a / n); }

// ---------------------------------------------------------------------------
// Voronoi labels: nearest seed under the periodic metric, the first seed on a
// tie (strict <, seeds in order).
__global__ void __launch_bounds__(kT) k_labels(const double* __restrict__ seeds, int ns, int nx, int ny,
                                               int32_t* __restrict__ labels) {
  __shared__ double s_xy[2 * kBatch];
  const int N = nx * ny;
  const int i = blockIdx.x * kT + threadIdx.x;
  const double xs = (double)(i / ny), ys = (double)(i % ny);
  const double fnx = (double)nx, fny = (double)ny;
  double best = INFINITY;
  int32_t lab = 0;
  for (int base = 0; base < ns; base += kBatch) {
    const int m = min(kBatch, ns - base);
    __syncthreads();
    for (int k = threadIdx.x; k < 2 * m; k += kT) s_xy[k] = seeds[2 * base + k];
    __syncthreads();
    if (i < N) {
      for (int k = 0; k < m; ++k) {
        const double ddx = periodic_delta(xs - s_xy[2 * k], fnx);
        const double ddy = periodic_delta(ys - s_xy[2 * k + 1], fny);
        const double d2 = ddx * ddx + ddy * ddy;
        if (d2 < best) {
          best = d2;
          lab = base + k;
        }
      }
    }
  }
  if (i < N) labels[i] = lab;
}

// Predicates of the ordered selection.
struct EdgePred {
  const int32_t* lab;
  int nx, ny;
  // the right (x + 1) or lower (y + 1) periodic neighbour carries another label
  __device__ bool operator()(int i) const {
    const int x = i / ny, y = i - x * ny;
    const int32_t l = lab[i];
    const int right = (x + 1 == nx ? 0 : x + 1) * ny + y;
    const int lower = x * ny + (y + 1 == ny ? 0 : y + 1);
    return l != lab[right] || l != lab[lower];
  }
};

struct BelowPred {
  const double* eta;
  double thr;
  __device__ bool operator()(int i) const { return eta[i] < thr; }
};

template <class Pred>
__global__ void __launch_bounds__(kT) k_chunk_count(Pred pred, int N, long long* __restrict__ cnt) {
  const int base = blockIdx.x * kChunk;
  int c = 0;
#pragma unroll
  for (int k = 0; k < kChunk / kT; ++k) {
    const int i = base + k * kT + threadIdx.x;
    c += __syncthreads_count(i < N && pred(i));
  }
  if (threadIdx.x == 0) cnt[blockIdx.x] = c;
}

// Exclusive scan of cnt[0..n) into off[0..n], off[n] = total; one block.
__global__ void __launch_bounds__(1024) k_chunk_scan(const long long* __restrict__ cnt, int n,
                                                     long long* __restrict__ off) {
  __shared__ long long s_warp[32];
  __shared__ long long s_carry;
  const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
  if (t == 0) s_carry = 0;
  __syncthreads();
  for (int base = 0; base < n; base += 1024) {
    const long long v = base + t < n ? cnt[base + t] : 0;
    long long incl = v;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      const long long o = __shfl_up_sync(0xffffffffu, incl, d);
      if (lane >= d) incl += o;
    }
    if (lane == 31) s_warp[warp] = incl;
    __syncthreads();
    if (warp == 0) {
      long long w = s_warp[lane];
#pragma unroll
      for (int d = 1; d < 32; d <<= 1) {
        const long long o = __shfl_up_sync(0xffffffffu, w, d);
        if (lane >= d) w += o;
      }
      s_warp[lane] = w;  // inclusive over warps
    }
    __syncthreads();
    const long long carry = s_carry;
    const long long excl = carry + (warp ? s_warp[warp - 1] : 0) + incl - v;
    if (base + t < n) off[base + t] = excl;
    __syncthreads();
    if (t == 1023) s_carry = excl + v;
    __syncthreads();
  }
  if (t == 0) off[n] = s_carry;
}

// flat[j] = the ranks[j]-th point (C order) satisfying pred, -1 if the rank is
// out of range. One block per rank (grid-stride over ranks); thread t owns the
// four consecutive points 4t .. 4t+3 of the chunk.
template <class Pred>
__global__ void __launch_bounds__(kT) k_select(Pred pred, int N, const long long* __restrict__ off, int nchunks,
                                               const long long* __restrict__ ranks, int n,
                                               long long* __restrict__ flat) {
  __shared__ int s_chunk;
  __shared__ int s_warp[kT / 32];
  const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
  const long long total = off[nchunks];
  for (int j = blockIdx.x; j < n; j += gridDim.x) {
    const long long r = ranks[j];
    if (r < 0 || r >= total) {
      if (t == 0) flat[j] = -1;
      continue;  // uniform across the block
    }
    if (t == 0) {
      int lo = 0, hi = nchunks - 1;  // last chunk c with off[c] <= r
      while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (off[mid] <= r) lo = mid;
        else hi = mid - 1;
      }
      s_chunk = lo;
    }
    __syncthreads();
    const int c = s_chunk;
    const long long local = r - off[c];
    const int p0 = c * kChunk + 4 * t;
    bool hit[4];
    int mine = 0;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      hit[k] = p0 + k < N && pred(p0 + k);
      mine += hit[k];
    }
    int incl = mine;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      const int o = __shfl_up_sync(0xffffffffu, incl, d);
      if (lane >= d) incl += o;
    }
    if (lane == 31) s_warp[warp] = incl;
    __syncthreads();
    int before = incl - mine;
    for (int w = 0; w < warp; ++w) before += s_warp[w];
    if (local >= before && local < before + mine) {
      int k = 0, seen = before;
      for (; k < 4; ++k) {
        if (hit[k]) {
          if (seen == local) break;
          ++seen;
        }
      }
      flat[j] = p0 + k;
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// Particles of the synthetic microstructure.
struct Particle {
  double cx, cy, R;
  int xlo, ylo, lenx, leny;
};

// Centre = picked pixel + jitter; window [floor(c) - reach, floor(c) + reach]
// per axis with reach = ceil(R + 8 w) + 1.
__global__ void __launch_bounds__(kT) k_particles(const long long* __restrict__ flat, int n, int ny,
                                                  const double* __restrict__ jitter, const double* __restrict__ radii,
                                                  double w, Particle* __restrict__ out) {
  const int j = blockIdx.x * kT + threadIdx.x;
  if (j >= n) return;
  const long long e = flat[j];
  const long long px = e / ny, py = e - px * ny;
  Particle p;
  p.cx = (double)px + jitter[2 * j];
  p.cy = (double)py + jitter[2 * j + 1];
  p.R = radii[j];
  const int reach = (int)ceil(p.R + 8.0 * w) + 1;
  p.xlo = (int)floor(p.cx) - reach;
  p.ylo = (int)floor(p.cy) - reach;
  p.lenx = p.leny = 2 * reach + 1;
  out[j] = p;
}

// Does the periodic window [lo, lo + len) meet the rows [t0, t1) of an axis of n?
__device__ __forceinline__ bool window_meets(int lo, int len, int t0, int t1, int n) {
  if (len >= n) return true;
  const int s = pmod(lo, n);
  return pmod(t0 - s, n) < len || pmod(s - t0, n) < t1 - t0;
}

// eta = max over particles and over the window images of a point of
// 1/2 [1 - tanh((r - R) / w)]; 0 where no window reaches.
__global__ void __launch_bounds__(kT) k_eta(const Particle* __restrict__ parts, int n, int nx, int ny, double w,
                                            double* __restrict__ eta) {
  __shared__ int s_list[kBatch];
  __shared__ int s_n;
  const int tilesy = (ny + kTileY - 1) / kTileY;
  const int tx0 = (blockIdx.x / tilesy) * kTileX, ty0 = (blockIdx.x % tilesy) * kTileY;
  const int tx1 = min(tx0 + kTileX, nx), ty1 = min(ty0 + kTileY, ny);
  const int gy = ty0 + (threadIdx.x & (kTileY - 1));
  const int xr = threadIdx.x / kTileY;  // 0..3
  double v[kTileX / 4];
#pragma unroll
  for (int k = 0; k < kTileX / 4; ++k) v[k] = 0.0;
  for (int base = 0; base < n; base += kBatch) {
    if (threadIdx.x == 0) s_n = 0;
    __syncthreads();
    const int j = base + threadIdx.x;
    if (j < n) {
      const Particle p = parts[j];
      if (window_meets(p.xlo, p.lenx, tx0, tx1, nx) && window_meets(p.ylo, p.leny, ty0, ty1, ny))
        s_list[atomicAdd(&s_n, 1)] = j;
    }
    __syncthreads();
    const int m = s_n;
    if (gy < ny) {
      for (int q = 0; q < m; ++q) {
        const Particle p = parts[s_list[q]];
        const int yfirst = p.ylo + pmod(gy - p.ylo, ny), yhi = p.ylo + p.leny - 1;
#pragma unroll
        for (int k = 0; k < kTileX / 4; ++k) {
          const int gx = tx0 + xr + 4 * k;
          if (gx >= nx) continue;
          const int xhi = p.xlo + p.lenx - 1;
          for (int ix = p.xlo + pmod(gx - p.xlo, nx); ix <= xhi; ix += nx) {
            const double dxs = (double)ix - p.cx;
            for (int iy = yfirst; iy <= yhi; iy += ny) {
              const double dys = (double)iy - p.cy;
              const double r = sqrt(dxs * dxs + dys * dys);
              const double prof = 0.5 * (1.0 - tanh((r - p.R) / w));
              v[k] = fmax(v[k], prof);
            }
          }
        }
      }
    }
    __syncthreads();
  }
  if (gy < ny) {
#pragma unroll
    for (int k = 0; k < kTileX / 4; ++k) {
      const int gx = tx0 + xr + 4 * k;
      if (gx < nx) eta[(size_t)gx * ny + gy] = v[k];
    }
  }
}

// X = eta x_particle + (1 - eta) (x_matrix + low + range u_i), u_i the i-th
// double of the PCG64 stream after (state, inc); then the KKS phase
// compositions. Thread g owns the points g, g + G, g + 2G, ... (G threads).
template <typename R>
__global__ void __launch_bounds__(kT) k_fields(int N, uint64_t st_lo, uint64_t st_hi, uint64_t inc_lo,
                                               uint64_t inc_hi, double x_matrix, double low, double range,
                                               double x_particle, double pc_shift, double pc_ratio,
                                               const double* __restrict__ eta, double* __restrict__ X,
                                               R* __restrict__ X_al, R* __restrict__ X_th) {
  const int G = gridDim.x * kT;
  const int g = blockIdx.x * kT + threadIdx.x;
  if (g >= N) return;
  const u128 inc = ((u128)inc_hi << 64) | inc_lo;
  u128 am, ap, gm, gp;
  lcg_jump((unsigned long long)g + 1ull, inc, am, ap);  // draw i comes from the state after i + 1 steps
  lcg_jump((unsigned long long)G, inc, gm, gp);
  u128 s = am * (((u128)st_hi << 64) | st_lo) + ap;
  for (int i = g; i < N; i += G) {
    const double u = (double)(pcg_output(s) >> 11) * (1.0 / 9007199254740992.0);
    const double xm = x_matrix + (low + range * u);
    const double e = eta[i];
    const double x = e * x_particle + (1.0 - e) * xm;
    const double h = 3.0 * (e * e) - 2.0 * (e * e * e);
    const double xa = (x - h * pc_shift) / ((1.0 - h) + h * pc_ratio);
    X[i] = x;
    X_al[i] = (R)xa;
    X_th[i] = (R)(pc_ratio * xa + pc_shift);
    s = gm * s + gp;
  }
}

// Sharp spheres (circles, z = 0): inside = any_i |o_i - x| <= r_i, the norm
// summed in the reference's order (x, y, z).
template <typename R, bool ADD>
__global__ void __launch_bounds__(kT) k_place(int nx, int ny, double dx, double dy, const double* __restrict__ prm,
                                              int n, double x_matrix, double x_precipitate, double* __restrict__ eta,
                                              double* __restrict__ X, R* __restrict__ X_mat, R* __restrict__ X_pre) {
  __shared__ double s_p[4 * kBatch];  // r, ox, oy, oz
  const int N = nx * ny;
  const int i = blockIdx.x * kT + threadIdx.x;
  const double x = (double)(i / ny) * dx, y = (double)(i % ny) * dy, z = 0.0;
  bool inside = false;
  for (int base = 0; base < n; base += kBatch) {
    const int m = min(kBatch, n - base);
    __syncthreads();
    for (int k = threadIdx.x; k < m; k += kT) {
#pragma unroll
      for (int c = 0; c < 4; ++c) s_p[4 * k + c] = prm[c * (size_t)n + base + k];
    }
    __syncthreads();
    for (int k = 0; k < m && !inside; ++k) {
      const double ax = s_p[4 * k + 1] - x, ay = s_p[4 * k + 2] - y, az = s_p[4 * k + 3] - z;
      inside = sqrt(ax * ax + ay * ay + az * az) <= s_p[4 * k];
    }
  }
  if (i >= N) return;
  if (!ADD) {
    eta[i] = inside ? 1.0 : 0.0;
    X[i] = inside ? x_precipitate : x_matrix;
    X_mat[i] = (R)(inside ? 0.0 : x_matrix);
    X_pre[i] = (R)(inside ? x_precipitate : 0.0);
  } else if (inside) {
    eta[i] = 1.0;
    X[i] = 0.99999;
    X_mat[i] = (R)0.0;
    X_pre[i] = (R)0.99999;
  }
}

__global__ void k_set_eta(const long long* __restrict__ flat, int n, double value, double* __restrict__ eta) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j < n && flat[j] >= 0) eta[flat[j]] = value;
}

int blocks_for(long long n) { return (int)((n + kT - 1) / kT); }

}  // namespace

// ---------------------------------------------------------------------------
// launchers

int kks_init_chunks(int N) { return (N + kChunk - 1) / kChunk; }

size_t kks_init_particle_bytes() { return sizeof(Particle); }

void kks_init_labels(const double* seeds, int ns, int nx, int ny, int32_t* labels, cudaStream_t s) {
  k_labels<<<blocks_for((long long)nx * ny), kT, 0, s>>>(seeds, ns, nx, ny, labels);
}

void kks_init_count_edges(const int32_t* labels, int nx, int ny, long long* cnt, long long* off, cudaStream_t s) {
  const int N = nx * ny, nc = kks_init_chunks(N);
  k_chunk_count<<<nc, kT, 0, s>>>(EdgePred{labels, nx, ny}, N, cnt);
  k_chunk_scan<<<1, 1024, 0, s>>>(cnt, nc, off);
}

void kks_init_count_below(const double* eta, double thr, int N, long long* cnt, long long* off, cudaStream_t s) {
  const int nc = kks_init_chunks(N);
  k_chunk_count<<<nc, kT, 0, s>>>(BelowPred{eta, thr}, N, cnt);
  k_chunk_scan<<<1, 1024, 0, s>>>(cnt, nc, off);
}

void kks_init_select_edges(const int32_t* labels, int nx, int ny, const long long* off, const long long* ranks,
                           int n, long long* flat, cudaStream_t s) {
  const int N = nx * ny;
  if (n <= 0) return;
  k_select<<<min(n, 148 * 8), kT, 0, s>>>(EdgePred{labels, nx, ny}, N, off, kks_init_chunks(N), ranks, n, flat);
}

void kks_init_select_below(const double* eta, double thr, int N, const long long* off, const long long* ranks, int n,
                           long long* flat, cudaStream_t s) {
  if (n <= 0) return;
  k_select<<<min(n, 148 * 8), kT, 0, s>>>(BelowPred{eta, thr}, N, off, kks_init_chunks(N), ranks, n, flat);
}

void kks_init_eta(const long long* flat, int n, int nx, int ny, const double* jitter, const double* radii, double w,
                  void* parts, double* eta, cudaStream_t s) {
  if (n > 0) k_particles<<<blocks_for(n), kT, 0, s>>>(flat, n, ny, jitter, radii, w, (Particle*)parts);
  const int tiles = ((nx + kTileX - 1) / kTileX) * ((ny + kTileY - 1) / kTileY);
  k_eta<<<tiles, kT, 0, s>>>((const Particle*)parts, n, nx, ny, w, eta);
}

template <typename R>
void kks_init_fields(int N, const uint64_t state[2], const uint64_t inc[2], double x_matrix, double low, double range,
                     double x_particle, double pc_shift, double pc_ratio, const double* eta, double* X, R* X_al,
                     R* X_th, cudaStream_t s) {
  const int nb = min(blocks_for(N), 148 * 8);
  k_fields<R><<<nb, kT, 0, s>>>(N, state[0], state[1], inc[0], inc[1], x_matrix, low, range, x_particle, pc_shift,
                                pc_ratio, eta, X, X_al, X_th);
}

template <typename R>
void kks_init_place(bool add, int nx, int ny, double dx, double dy, const double* prm, int n, double x_matrix,
                    double x_precipitate, double* eta, double* X, R* X_mat, R* X_pre, cudaStream_t s) {
  const int nb = blocks_for((long long)nx * ny);
  if (add)
    k_place<R, true><<<nb, kT, 0, s>>>(nx, ny, dx, dy, prm, n, x_matrix, x_precipitate, eta, X, X_mat, X_pre);
  else
    k_place<R, false><<<nb, kT, 0, s>>>(nx, ny, dx, dy, prm, n, x_matrix, x_precipitate, eta, X, X_mat, X_pre);
}

void kks_init_set_eta(const long long* flat, int n, double value, double* eta, cudaStream_t s) {
  if (n > 0) k_set_eta<<<blocks_for(n), kT, 0, s>>>(flat, n, value, eta);
}

template void kks_init_fields<double>(int, const uint64_t*, const uint64_t*, double, double, double, double, double,
                                      double, const double*, double*, double*, double*, cudaStream_t);
template void kks_init_fields<float>(int, const uint64_t*, const uint64_t*, double, double, double, double, double,
                                     double, const double*, double*, float*, float*, cudaStream_t);
template void kks_init_place<double>(bool, int, int, double, double, const double*, int, double, double, double*,
                                     double*, double*, double*, cudaStream_t);
template void kks_init_place<float>(bool, int, int, double, double, const double*, int, double, double, double*,
                                    double*, float*, float*, cudaStream_t);
