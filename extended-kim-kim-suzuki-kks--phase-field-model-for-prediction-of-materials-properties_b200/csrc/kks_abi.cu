// kks_abi.cu - host runtime of one KKS cell behind the C ABI of include/kks.h.
//
// Execution model. An attempt is a fixed sequence of kernels and cuFFT
// executions with no host decision inside it: the prologue reads the loop
// state from device memory, the decide kernel writes it back (including the
// reject / accept / enlarge outcome, pf_kks/solver.py:330-351), and a
// rejection is handled on the device by restoring the step's input into the
// candidate buffer. Consecutive attempts therefore alternate between the two
// state buffers unconditionally, and the attempt for each parity is captured
// once as a CUDA graph. kks_run launches as many attempt graphs as there are
// steps left, synchronises once, reads the step counter, and launches again
// for the steps that rejections consumed: one host synchronisation per batch
// of steps, none per attempt.

#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>
#include <cufft.h>
#include <math.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <new>
#include <string>
#include <vector>

#include <nvtx3/nvToolsExt.h>

#include "kks_fft.cuh"
#include "kks_internal.cuh"

// NVTX ranges around the library's calls (header-only NVTX v3: free when no
// profiler is attached), so that a timeline shows which call a device span
// belongs to; the attempt graphs' kernels carry their own names.
namespace {
struct NvtxRange {
  explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
  ~NvtxRange() { nvtxRangePop(); }
};
}  // namespace
#define KKS_RANGE(name) NvtxRange kks_nvtx_range_(name)

static thread_local std::string g_last_error;

static int set_error(int code, const std::string& msg) {
  g_last_error = msg;
  return code;
}

int kks_set_error(int code, const std::string& msg) { return set_error(code, msg); }

#define CK(expr)                                                                                          \
  do {                                                                                                    \
    cudaError_t _e = (expr);                                                                              \
    if (_e != cudaSuccess)                                                                                \
      return set_error(KKS_ERR_CUDA, std::string(#expr) + ": " + cudaGetErrorString(_e));                \
  } while (0)

#define CKF(expr)                                                                                        \
  do {                                                                                                   \
    cufftResult _r = (expr);                                                                             \
    if (_r != CUFFT_SUCCESS) return set_error(KKS_ERR_CUFFT, std::string(#expr) + ": cufft error " +      \
                                              std::to_string((int)_r));                                  \
  } while (0)

struct kks_handle {
  int device = 0, precision = 0, rsize = 8;
  cudaStream_t stream = nullptr;
  KksConst hc{};
  KksConst* dc = nullptr;
  KksCtl* d_ctl = nullptr;
  KksPar* d_par = nullptr;
  KksCtl* h_ctl = nullptr;  // pinned mirror
  int32_t* h_target = nullptr;
  uint8_t* d_flags = nullptr;
  kks_record* d_ring = nullptr;
  long long ring_cap = 0;
  kks_step_row* d_rows = nullptr;
  long long row_cap = 0;
  double* d_kx = nullptr;
  double* d_ky = nullptr;
  double* d_xfer = nullptr;
  void* arena = nullptr;
  size_t arena_bytes = 0, state_bytes = 0;
  KksFieldPtrs f{};
  int nblocks = 0;      // grid of the grid-stride field kernels (a launch shape)
  int nblocks_cap = 0;  // largest grid the partial-sum buffers hold
  int nsm = 148;
  int in_batch = 0;     // batches that hold this cell (its launch shape is then fixed)
  cufftHandle plan_r2c3 = 0, plan_c2r3 = 0, plan_c2r2 = 0;
  bool plans_made = false;
  void* fft_work = nullptr;
  cudaGraphExec_t graph[2] = {nullptr, nullptr};
  int parity = 0;
  bool uploaded = false;
  long long rec_read = 0, row_read = 0;
  std::vector<kks_record> recs;
  std::vector<kks_step_row> rows;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  double device_ms = 0.0;
  long long timed_attempts = 0;
  long long attempts_launched = 0;
  // shared-memory FFT pipeline of the mixed path (kks_fft.cu)
  bool fused = false;     // the attempt runs the fused passes (KKS_PRECISION_MIXED)
  bool fused_ok = false;  // the fused passes are set up for this cell
  void* fft_arena = nullptr;
  KksFftConst* d_fc = nullptr;
  KksFftLaunch fl{};
  double* partials_fused = nullptr;
  int nb_fused = 0;        // partial-sum rows of the current launch shape
  int part_cap_fused = 0;  // rows allocated
  // initial state on the device (kks_init.cu): chunk counts and offsets of the
  // ordered selection, and a per-call buffer for particles and ranks
  long long* sel = nullptr;
  void* init_buf = nullptr;
  size_t init_bytes = 0;
  bool edges_ready = false;
  long long n_edges = 0;
};

static size_t round_up(size_t v, size_t m) { return (v + m - 1) / m * m; }

// Angular wave numbers of pf_kks/grid.py:6-20 (Nyquist entry of an even axis
// left at 0), same arithmetic as the reference: j * 2 * pi / (n * 1).
static void frequencies(int n, std::vector<double>& out, int count) {
  out.assign(count, 0.0);
  std::vector<double> lin(n, 0.0);
  if (n % 2 == 1) {
    int half = (int)((n - 1) / 2.0 + 1);
    for (int j = 0; j < half; ++j) lin[j] = (double)j * 2 * M_PI / (n * 1.0);
    int start = (int)(-(n + 1) / 2.0 + 1);
    for (int j = half, v = start; j < n; ++j, ++v) lin[j] = (double)v * 2 * M_PI / (n * 1.0);
  } else {
    for (int j = 0; j < n / 2; ++j) lin[j] = (double)j * 2 * M_PI / (n * 1.0);
    for (int j = n / 2 + 1, v = -n / 2 + 1; j < n; ++j, ++v) lin[j] = (double)v * 2 * M_PI / (n * 1.0);
  }
  for (int j = 0; j < count; ++j) out[j] = lin[j];
}

// np.interp at a scalar, host side (the stiffness is frozen at T(t = 0)).
static double interp_host(double x, const double* xp, const double* fp, int n) {
  if (n == 1 || x <= xp[0]) return fp[0];
  if (x >= xp[n - 1]) return fp[n - 1];
  int lo = 0, hi = n - 1;
  while (hi - lo > 1) {
    int mid = (lo + hi) / 2;
    if (x >= xp[mid]) lo = mid; else hi = mid;
  }
  if (xp[lo] == x) return fp[lo];
  double slope = (fp[lo + 1] - fp[lo]) / (xp[lo + 1] - xp[lo]);
  return slope * (x - xp[lo]) + fp[lo];
}

template <bool MIXED>
static int enqueue_attempt(kks_handle* h, int p) {
  cudaStream_t s = h->stream;
  KksFieldPtrs& f = h->f;
  const size_t NCp = h->hc.NCp;
  const int nb = h->nblocks;
  kks_launch_prologue(h->dc, h->d_ctl, h->d_par, h->d_flags, h->d_ring, h->ring_cap, s);
  kks_launch_prep<MIXED>(&h->hc, h->d_par, f, p, nb, s);
  if (!MIXED) {
    CKF(cufftExecD2Z(h->plan_r2c3, (double*)f.fft_in[p], (cufftDoubleComplex*)f.spec_a));
  } else {
    CKF(cufftExecR2C(h->plan_r2c3, (float*)f.fft_in[p], (cufftComplex*)f.spec_a));
  }
  kks_launch_spectral_mid<MIXED>(&h->hc, h->dc, h->d_par, f, nb, s);
  if (!MIXED) {
    CKF(cufftExecZ2D(h->plan_c2r3, (cufftDoubleComplex*)f.spec_bcd, (double*)f.real_b));
  } else {
    CKF(cufftExecC2R(h->plan_c2r3, (cufftComplex*)f.spec_bcd, (float*)f.real_b));
  }
  kks_launch_pre_pointwise<MIXED>(&h->hc, h->dc, h->d_par, f, p, nb, s);
  if (!MIXED) {
    CKF(cufftExecD2Z(h->plan_r2c3, (double*)f.real_c, (cufftDoubleComplex*)f.spec_bcd));
  } else {
    CKF(cufftExecR2C(h->plan_r2c3, (float*)f.real_c, (cufftComplex*)f.spec_bcd));
  }
  kks_launch_spectral_update<MIXED>(&h->hc, h->dc, h->d_par, f, nb, s);
  if (!MIXED) {
    CKF(cufftExecZ2D(h->plan_c2r2, (cufftDoubleComplex*)f.spec_bcd + 3 * NCp, (double*)f.fft_out[p]));
  } else {
    CKF(cufftExecC2R(h->plan_c2r2, (cufftComplex*)f.spec_bcd + 3 * NCp, (float*)f.fft_out[p]));
  }
  kks_launch_post_pointwise<MIXED>(&h->hc, h->dc, h->d_par, f, p, nb, s);
  kks_launch_decide(h->dc, h->d_ctl, h->d_par, f.partials, nb, h->d_ring, h->ring_cap, h->d_rows, h->row_cap, s);
  kks_launch_restore<MIXED>(&h->hc, h->dc, h->d_ctl, f, p, nb, s);
  CK(cudaGetLastError());
  return KKS_OK;
}

static int enqueue_fused(kks_handle* h, int p) {
  cudaStream_t s = h->stream;
  kks_launch_prologue(h->dc, h->d_ctl, h->d_par, h->d_flags, h->d_ring, h->ring_cap, s);
  kks_fft_launch_attempt(h->fl, p, s);
  kks_launch_decide(h->dc, h->d_ctl, h->d_par, h->partials_fused, h->nb_fused, h->d_ring, h->ring_cap, h->d_rows,
                    h->row_cap, s);
  if (h->fl.f64) kks_launch_restore<false>(&h->hc, h->dc, h->d_ctl, h->f, p, h->nblocks, s);
  else kks_launch_restore<true>(&h->hc, h->dc, h->d_ctl, h->f, p, h->nblocks, s);
  CK(cudaGetLastError());
  return KKS_OK;
}

static int enqueue(kks_handle* h, int p) {
  if (h->fused) return enqueue_fused(h, p);
  return h->precision == KKS_PRECISION_FP64 ? enqueue_attempt<false>(h, p) : enqueue_attempt<true>(h, p);
}

// ---------------------------------------------------------------------------
// Plans of the shared-memory FFT (kks_fft.cu): radices 4, 2, 3, 5, 7 and at
// most one larger prime from KKS_FFT_PRIMES as the last DIF stage.
struct AxisTables {
  std::vector<float2> tw;
  std::vector<double2> tw64;  // the same twiddles in double (FP64 step)
  std::vector<int> slot;
};

// ceil(2^32 / d) for the device's x / d == __umulhi(x, m) (x, d < 2^16); 0 for d = 1
static uint32_t div_magic(int d) {
  return d <= 1 ? 0u : (uint32_t)((((uint64_t)1 << 32) + (uint64_t)d - 1) / (uint64_t)d);
}

static bool build_axis(int n, KksFftAxis& ax, AxisTables& t, bool radix8) {
  std::vector<int> rad;
  int m = n;
  // radix-8 stages first where the sides allow them (fewer passes over shared
  // memory, barriers and index computations) on axes without a large prime
  // (their kernels are built without radix 8); the FP64 passes keep radix 4
  int rest = n;
  for (int r : {2, 3, 5, 7})
    while (rest % r == 0) rest /= r;
  if (radix8 && rest == 1)
    while (m % 8 == 0) { rad.push_back(8); m /= 8; }
  for (int r : {4, 2, 3, 5, 7})
    while (m % r == 0) { rad.push_back(r); m /= r; }
  int P = 0;
  if (m > 1) {
    bool ok = false;
    for (int p : KKS_FFT_PRIMES) ok = ok || (m == p);
    if (!ok) return false;
    P = m;
    rad.push_back(m);
  }
  if ((int)rad.size() > KKS_FFT_MAXST || rad.empty() || n > KKS_FFT_MAXN) return false;
  memset(&ax, 0, sizeof(ax));
  ax.n = n;
  ax.nst = (int)rad.size();
  ax.P = P;
  int L = n;
  t.tw.clear();
  t.tw64.clear();
  for (int s = 0; s < ax.nst; ++s) {
    const int r = rad[s], q = L / r;
    ax.r[s] = r;
    ax.L[s] = L;
    ax.q[s] = q;
    ax.tw_off[s] = (int)t.tw.size();
    ax.qm[s] = div_magic(q);
    ax.pm[s] = div_magic(n / r);
    if (q > 1)
      for (int j = 0; j < q; ++j)
        for (int mm = 0; mm < r; ++mm) {
          const double th = 2.0 * M_PI * (double)((long long)j * mm % L) / (double)L;
          t.tw.push_back(make_float2((float)cos(th), (float)sin(th)));
          t.tw64.push_back(make_double2(cos(th), sin(th)));
        }
    L = q;
  }
  if (t.tw.empty()) {
    t.tw.push_back(make_float2(1.f, 0.f));
    t.tw64.push_back(make_double2(1.0, 0.0));
  }
  // position of frequency k after the DIF: digits d_s of the position (weights q_s)
  // are the digits of k read with weights r_0 r_1 ... r_{s-1}
  t.slot.assign(n, 0);
  for (int pos = 0; pos < n; ++pos) {
    int rem = pos, k = 0, w = 1;
    for (int s = 0; s < ax.nst; ++s) {
      const int d = rem / ax.q[s];
      rem = rem % ax.q[s];
      k += d * w;
      w *= ax.r[s];
    }
    t.slot[k] = pos;
  }
  return true;
}

// cuTensorMapEncodeTiled through the runtime's driver entry point (no link
// against libcuda); nullptr when the driver does not provide it.
static PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
  void* fn = nullptr;
  cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
  if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) != cudaSuccess ||
      q != cudaDriverEntryPointSuccess)
    return nullptr;
  return (PFN_cuTensorMapEncodeTiled_v12000)fn;
}

// Tensor map of F column-major row-spectrum fields at base (kks_fft.cuh).
static bool encode_spectrum_map(CUtensorMap* map, void* base, int nx, int nyh, int F) {
  PFN_cuTensorMapEncodeTiled_v12000 enc = tensor_map_encoder();
  if (!enc) return false;
  const cuuint64_t dims[3] = {(cuuint64_t)nx, (cuuint64_t)nyh, (cuuint64_t)F};
  const cuuint64_t strides[2] = {(cuuint64_t)nx * 8, (cuuint64_t)nx * nyh * 8};
  const cuuint32_t box[3] = {2, (cuuint32_t)(nyh < 256 ? nyh : 256), (cuuint32_t)F};
  const cuuint32_t estr[3] = {1, 1, 1};
  return enc(map, CU_TENSOR_MAP_DATA_TYPE_UINT64, 3, base, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
             CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

template <typename T>
static int upload_vec(const std::vector<T>& v, T** dst) {
  CK(cudaMalloc(dst, v.size() * sizeof(T)));
  CK(cudaMemcpy(*dst, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice));
  return KKS_OK;
}

// Partial-sum rows the fused attempt writes under the cell's launch shape.
static int fused_rows(const kks_handle* h) {
  return std::max(std::max(kks_fft_row_blocks(h->hc.nx), kks_fft_col_blocks(h->hc.nyh, h->fl.cols)), h->nblocks);
}

// The fused passes of a mixed cell (kks_fft.cu) or of an FP64 cell
// (kks_fft64.cu): the same plans and buffers, in single or double precision.
static int setup_fused(kks_handle* h, const std::vector<double>& kx) {
  KksConst& c = h->hc;
  const bool f64 = h->precision == KKS_PRECISION_FP64;
  KksFftConst fc;
  memset(&fc, 0, sizeof(fc));
  AxisTables tx, ty;
  if (!build_axis(c.nx, fc.ax, tx, !f64) || !build_axis(c.ny, fc.ay, ty, !f64)) return KKS_OK;  // not supported: cuFFT
  int optin = 0;
  CK(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, h->device));
  fc.cols = f64 ? 1 : KKS_FFT_COLS;
  const size_t need = f64 ? kks_fft64_smem_bytes(c.nx, c.ny, fc.cols) : kks_fft_smem_bytes(c.nx, c.ny, fc.cols);
  if (need > (size_t)optin) return KKS_OK;
  fc.wait_polls = KKS_FFT_WAIT_POLLS;
  std::vector<float> kx_slot(c.nx);
  std::vector<double> kx_slot64(c.nx);
  for (int k = 0; k < c.nx; ++k) {
    kx_slot[tx.slot[k]] = (float)kx[k];
    kx_slot64[tx.slot[k]] = kx[k];
  }
  // device tables and buffers in one allocation
  const size_t elem = f64 ? sizeof(double2) : sizeof(float2);
  const size_t fs = (size_t)c.nx * c.nyh * elem;
  auto al = [](size_t b) { return (b + 255) / 256 * 256; };
  const size_t b_twx = al(tx.tw.size() * sizeof(float2)), b_twy = al(ty.tw.size() * sizeof(float2));
  const size_t b_slx = al(tx.slot.size() * sizeof(int)), b_sly = al(ty.slot.size() * sizeof(int));
  const size_t b_kxs = al(kx_slot.size() * sizeof(float));
  // prime-stage factor tables of the two axes
  std::vector<float2> ptx(KKS_FFT_PRIME_TABLE_MAX), pty(KKS_FFT_PRIME_TABLE_MAX);
  const int npx = kks_fft_prime_table(fc.ax.P, ptx.data()), npy = kks_fft_prime_table(fc.ay.P, pty.data());
  const size_t b_ptx = al(std::max(npx, 1) * sizeof(float2)), b_pty = al(std::max(npy, 1) * sizeof(float2));
  // the FP64 step's tables
  std::vector<double2> ztx(KKS_FFT64_PRIME_TABLE_MAX), zty(KKS_FFT64_PRIME_TABLE_MAX);
  int nzx = 0, nzy = 0;
  size_t b_64 = 0;
  if (f64) {
    nzx = kks_fft64_prime_table(fc.ax.P, ztx.data());
    nzy = kks_fft64_prime_table(fc.ay.P, zty.data());
    b_64 = al(tx.tw64.size() * sizeof(double2)) + al(ty.tw64.size() * sizeof(double2)) +
           al(kx_slot64.size() * sizeof(double)) + al(std::max(nzx, 1) * sizeof(double2)) +
           al(std::max(nzy, 1) * sizeof(double2));
  }
  const size_t b_spec = al(3 * fs) * 2 + al(2 * fs);
  const size_t total = b_twx + b_twy + b_slx + b_sly + b_kxs + b_ptx + b_pty + b_64 + b_spec;
  CK(cudaMalloc(&h->fft_arena, total));
  char* a = (char*)h->fft_arena;
  cudaError_t put_err = cudaSuccess;
  auto put = [&](const void* src, size_t n, size_t b) -> char* {
    char* p = a;
    const cudaError_t e = cudaMemcpy(p, src, n, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) put_err = e;
    a += b;
    return p;
  };
  fc.ax.tw = (const float2*)put(tx.tw.data(), tx.tw.size() * sizeof(float2), b_twx);
  fc.ay.tw = (const float2*)put(ty.tw.data(), ty.tw.size() * sizeof(float2), b_twy);
  fc.ax.slot = (const int*)put(tx.slot.data(), tx.slot.size() * sizeof(int), b_slx);
  fc.ay.slot = (const int*)put(ty.slot.data(), ty.slot.size() * sizeof(int), b_sly);
  fc.kx_slot = (const float*)put(kx_slot.data(), kx_slot.size() * sizeof(float), b_kxs);
  fc.ax.ptw = (const float2*)put(ptx.data(), std::max(npx, 1) * sizeof(float2), b_ptx);
  fc.ay.ptw = (const float2*)put(pty.data(), std::max(npy, 1) * sizeof(float2), b_pty);
  if (f64) {
    fc.ax.tw64 = (const double2*)put(tx.tw64.data(), tx.tw64.size() * sizeof(double2),
                                     al(tx.tw64.size() * sizeof(double2)));
    fc.ay.tw64 = (const double2*)put(ty.tw64.data(), ty.tw64.size() * sizeof(double2),
                                     al(ty.tw64.size() * sizeof(double2)));
    fc.kx_slot64 = (const double*)put(kx_slot64.data(), kx_slot64.size() * sizeof(double),
                                      al(kx_slot64.size() * sizeof(double)));
    fc.ax.ptw64 = (const double2*)put(ztx.data(), std::max(nzx, 1) * sizeof(double2),
                                      al(std::max(nzx, 1) * sizeof(double2)));
    fc.ay.ptw64 = (const double2*)put(zty.data(), std::max(nzy, 1) * sizeof(double2),
                                      al(std::max(nzy, 1) * sizeof(double2)));
  }
  CK(put_err);
  void* RA = a; a += al(3 * fs);
  void* RB = a; a += al(3 * fs);
  void* SA = a; a += al(2 * fs);
  CK(cudaMemset(RA, 0, b_spec));
  // every kernel of the pipeline writes one partial-sum row per block: the
  // buffer holds the largest grid of them (row pairs, column tiles, extras)
  // under any launch shape; the decide kernel reads the rows of the current one
  fc.part_cap = std::max(kks_fft_partial_rows(c.nx, c.ny, h->nblocks_cap), h->nblocks_cap);
  CK(cudaMalloc(&h->d_fc, sizeof(KksFftConst)));
  CK(cudaMemcpy(h->d_fc, &fc, sizeof(KksFftConst), cudaMemcpyHostToDevice));
  KksFftLaunch& L = h->fl;
  L.dc = h->dc;
  L.par = h->d_par;
  L.ctl = h->d_ctl;
  L.fc = h->d_fc;
  L.f = &h->f;
  L.RA = RA;
  L.RB = RB;
  L.SA = SA;
  L.nx = c.nx;
  L.ny = c.ny;
  L.nyh = c.nyh;
  L.nbx = h->nblocks;
  L.cols = fc.cols;
  L.PX = fc.ax.P;
  L.PY = fc.ay.P;
  L.f64 = f64 ? 1 : 0;
  // bulk copies of whole row pairs need 16-byte multiples for the f32 rows, the
  // tensor maps 16-byte strides (nx even; every pair then has both rows)
  // column runs start at multiples of nx * 8 bytes: bulk copies need nx even
  // (the FP64 passes move their spectra with plain loads and stores)
  L.bulk_cols = (!f64 && c.nx % 2 == 0) ? 1 : 0;
  L.bulk_rows = 0;
  if (!f64 && c.nx % 2 == 0 && c.ny % 4 == 0 && encode_spectrum_map(&L.map_RA3, RA, c.nx, c.nyh, 3) &&
      encode_spectrum_map(&L.map_RB3, RB, c.nx, c.nyh, 3) && encode_spectrum_map(&L.map_RB2, RB, c.nx, c.nyh, 2))
    L.bulk_rows = 1;
  if (kks_fft_set_attributes(L) != 0) return set_error(KKS_ERR_CUDA, "fft kernel attributes");
  h->part_cap_fused = fc.part_cap;
  h->nb_fused = fused_rows(h);
  CK(cudaMalloc(&h->partials_fused, (size_t)h->part_cap_fused * KKS_NPART * sizeof(double)));
  CK(cudaMemset(h->partials_fused, 0, (size_t)h->part_cap_fused * KKS_NPART * sizeof(double)));
  h->f.partials = h->partials_fused;
  h->fused = true;
  h->fused_ok = true;
  return KKS_OK;
}

static int make_plans(kks_handle* h) {
  const int nx = h->hc.nx, ny = h->hc.ny, nyh = h->hc.nyh;
  int n[2] = {nx, ny};
  int rembed[2] = {nx, ny};
  int cembed[2] = {nx, nyh};
  const bool d = h->precision == KKS_PRECISION_FP64;
  size_t ws[3] = {0, 0, 0};
  CKF(cufftCreate(&h->plan_r2c3));
  CKF(cufftCreate(&h->plan_c2r3));
  CKF(cufftCreate(&h->plan_c2r2));
  h->plans_made = true;
  for (cufftHandle p : {h->plan_r2c3, h->plan_c2r3, h->plan_c2r2}) CKF(cufftSetAutoAllocation(p, 0));
  CKF(cufftMakePlanMany(h->plan_r2c3, 2, n, rembed, 1, h->hc.Np, cembed, 1, h->hc.NCp, d ? CUFFT_D2Z : CUFFT_R2C, 3,
                        &ws[0]));
  CKF(cufftMakePlanMany(h->plan_c2r3, 2, n, cembed, 1, h->hc.NCp, rembed, 1, h->hc.Np, d ? CUFFT_Z2D : CUFFT_C2R, 3,
                        &ws[1]));
  CKF(cufftMakePlanMany(h->plan_c2r2, 2, n, cembed, 1, h->hc.NCp, rembed, 1, h->hc.Np, d ? CUFFT_Z2D : CUFFT_C2R, 2,
                        &ws[2]));
  size_t w = std::max(ws[0], std::max(ws[1], ws[2]));
  if (w > 0) CK(cudaMalloc(&h->fft_work, w));
  for (cufftHandle p : {h->plan_r2c3, h->plan_c2r3, h->plan_c2r2}) {
    CKF(cufftSetWorkArea(p, h->fft_work));
    CKF(cufftSetStream(p, h->stream));
  }
  return KKS_OK;
}

static int capture_graphs(kks_handle* h) {
  for (int p = 0; p < 2; ++p) {
    cudaGraph_t g = nullptr;
    CK(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
    int rc = enqueue(h, p);
    cudaError_t e = cudaStreamEndCapture(h->stream, &g);
    if (rc != KKS_OK) {
      if (g) cudaGraphDestroy(g);
      return rc;
    }
    if (e != cudaSuccess) return set_error(KKS_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(e));
    e = cudaGraphInstantiate(&h->graph[p], g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return set_error(KKS_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(e));
  }
  return KKS_OK;
}

static void free_handle(kks_handle* h) {
  if (!h) return;
  if (h->stream) cudaStreamSynchronize(h->stream);
  for (int p = 0; p < 2; ++p)
    if (h->graph[p]) cudaGraphExecDestroy(h->graph[p]);
  if (h->plans_made) {
    cufftDestroy(h->plan_r2c3);
    cufftDestroy(h->plan_c2r3);
    cufftDestroy(h->plan_c2r2);
  }
  cudaFree(h->fft_work);
  cudaFree(h->fft_arena);
  cudaFree(h->d_fc);
  cudaFree(h->partials_fused);
  cudaFree(h->arena);
  cudaFree(h->dc);
  cudaFree(h->d_ctl);
  cudaFree(h->d_par);
  cudaFree(h->d_flags);
  cudaFree(h->d_ring);
  cudaFree(h->d_rows);
  cudaFree(h->d_kx);
  cudaFree(h->d_ky);
  cudaFree(h->d_xfer);
  cudaFree(h->sel);
  cudaFree(h->init_buf);
  if (h->h_ctl) cudaFreeHost(h->h_ctl);
  if (h->h_target) cudaFreeHost(h->h_target);
  if (h->ev0) cudaEventDestroy(h->ev0);
  if (h->ev1) cudaEventDestroy(h->ev1);
  if (h->stream) cudaStreamDestroy(h->stream);
  delete h;
}

static int create_impl(kks_handle* h, const kks_params* prm, int32_t n_steps, const uint8_t* step_flags) {
  CK(cudaSetDevice(h->device));
  CK(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));
  CK(cudaEventCreate(&h->ev0));
  CK(cudaEventCreate(&h->ev1));
  KksConst& c = h->hc;
  c.p = *prm;
  c.nx = prm->nx;
  c.ny = prm->ny;
  c.nyh = prm->ny / 2 + 1;
  c.N = prm->nx * prm->ny;
  c.NC = prm->nx * c.nyh;
  c.Np = (int)round_up((size_t)c.N, 64);
  c.NCp = (int)round_up((size_t)c.NC, 32);
  c.n_steps = n_steps;
  c.dtime_s_min = prm->dtime_s / prm->dtime_min_divisor;
  c.inv_N = 1.0 / (double)c.N;
  const double T0 = interp_host(0.0, prm->sched_time, prm->sched_temp, prm->n_sched);
  c.C11_0 = interp_host(T0, prm->table_T, prm->table[KKS_TAB_C11], prm->n_table);
  c.C12_0 = interp_host(T0, prm->table_T, prm->table[KKS_TAB_C12], prm->n_table);
  c.C44_0 = interp_host(T0, prm->table_T, prm->table[KKS_TAB_C44], prm->n_table);
  c.c11 = c.C11_0 / c.C44_0;
  c.c12 = c.C12_0 / c.C44_0;
  c.c3 = (c.C11_0 + 2 * c.C12_0) / c.C44_0;
  h->rsize = h->precision == KKS_PRECISION_FP64 ? 8 : 4;
  c.mixed = h->precision != KKS_PRECISION_FP64;

  int nsm = 148;
  CK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, h->device));
  h->nsm = nsm;
  h->nblocks = kks_field_blocks(c.N, nsm);
  h->nblocks_cap = kks_field_blocks(c.N, 2 * nsm);  // up to 8 blocks per SM

  // arena (layout in kks_internal.cuh)
  const bool mixed = h->precision != KKS_PRECISION_FP64;
  c.mixed = mixed;
  const size_t R = h->rsize, Np = c.Np, NCp = c.NCp, D = sizeof(double);
  const size_t sz_state = mixed ? 2 * Np * D + 2 * Np * R : 5 * Np * D;
  const size_t sz_fin = mixed ? 3 * Np * R : 0;
  const size_t sz_spec_a = 3 * NCp * 2 * R, sz_real_b = 3 * Np * R, sz_real_c = 3 * Np * R,
               sz_spec_bcd = 5 * NCp * 2 * R, sz_one = Np * R;
  const size_t sz_part = round_up((size_t)h->nblocks_cap * KKS_NPART * sizeof(double), 256);
  size_t total = 2 * sz_state + sz_fin + sz_spec_a + sz_real_b + sz_real_c + sz_spec_bcd + 2 * Np * D + 4 * sz_one +
                 sz_part;
  CK(cudaMalloc(&h->arena, total));
  CK(cudaMemset(h->arena, 0, total));
  h->arena_bytes = total;
  char* a = (char*)h->arena;
  char* state[2];
  state[0] = a; a += sz_state;
  state[1] = a; a += sz_state;
  h->state_bytes = sz_state;
  char* fin = a; a += sz_fin;
  h->f.spec_a = a; a += sz_spec_a;
  h->f.real_b = a; a += sz_real_b;
  h->f.real_c = a; a += sz_real_c;
  h->f.spec_bcd = a; a += sz_spec_bcd;
  h->f.eta_m = a; a += Np * D;
  h->f.X_m = a; a += Np * D;
  h->f.mu = a; a += sz_one;
  for (int k = 0; k < 3; ++k) { h->f.g[k] = a; a += sz_one; }
  h->f.partials = (double*)a; a += sz_part;
  for (int p = 0; p < 2; ++p) {
    h->f.eta[p] = state[p];
    h->f.X[p] = state[p] + Np * D;
    if (mixed) {
      h->f.X_al[p] = state[p] + 2 * Np * D;
      h->f.X_th[p] = state[p] + 2 * Np * D + Np * R;
    } else {
      h->f.X_al[p] = state[p] + 3 * Np * D;
      h->f.X_th[p] = state[p] + 4 * Np * D;
    }
  }
  for (int p = 0; p < 2; ++p) {
    h->f.fft_in[p] = mixed ? fin : state[p];           // eta | X | eta^2
    h->f.fft_out[p] = mixed ? h->f.real_c : state[1 - p];  // eta_b | X_b, or d_eta | d_X
  }

  std::vector<double> kx, ky;
  frequencies(c.nx, kx, c.nx);
  frequencies(c.ny, ky, c.nyh);
  CK(cudaMalloc(&h->d_kx, c.nx * sizeof(double)));
  CK(cudaMalloc(&h->d_ky, c.nyh * sizeof(double)));
  CK(cudaMemcpy(h->d_kx, kx.data(), c.nx * sizeof(double), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(h->d_ky, ky.data(), c.nyh * sizeof(double), cudaMemcpyHostToDevice));
  h->f.kx = h->d_kx;
  h->f.ky = h->d_ky;

  CK(cudaMalloc(&h->dc, sizeof(KksConst)));
  CK(cudaMemcpy(h->dc, &c, sizeof(KksConst), cudaMemcpyHostToDevice));
  CK(cudaMalloc(&h->d_ctl, sizeof(KksCtl)));
  CK(cudaMemset(h->d_ctl, 0, sizeof(KksCtl)));
  CK(cudaMalloc(&h->d_par, sizeof(KksPar)));
  CK(cudaMemset(h->d_par, 0, sizeof(KksPar)));
  CK(cudaMallocHost(&h->h_ctl, sizeof(KksCtl)));
  memset(h->h_ctl, 0, sizeof(KksCtl));
  CK(cudaMallocHost(&h->h_target, sizeof(int32_t)));
  CK(cudaMalloc(&h->d_flags, std::max(n_steps, 1)));
  CK(cudaMemset(h->d_flags, 0, std::max(n_steps, 1)));
  if (n_steps > 0) CK(cudaMemcpy(h->d_flags, step_flags, n_steps, cudaMemcpyHostToDevice));
  CK(cudaMalloc(&h->d_ring, h->ring_cap * sizeof(kks_record)));
  CK(cudaMalloc(&h->d_rows, h->row_cap * sizeof(kks_step_row)));
  CK(cudaMalloc(&h->d_xfer, (size_t)c.N * sizeof(double)));

  int rc = make_plans(h);
  if (rc != KKS_OK) return rc;
  if (h->precision != KKS_PRECISION_MIXED_CUFFT) {  // the cuFFT comparison path has no fused passes
    rc = setup_fused(h, kx);
    if (rc != KKS_OK) return rc;
  }
  rc = capture_graphs(h);
  if (rc != KKS_OK) return rc;
  CK(cudaStreamSynchronize(h->stream));
  return KKS_OK;
}

extern "C" {

const char* kks_last_error(void) { return g_last_error.c_str(); }

const char* kks_version(void) { return "kks_b200 1.0 (sm_100a, cuFFT)"; }

int kks_create(const kks_params* params, int precision, int device, int32_t n_steps, const uint8_t* step_flags,
               int64_t record_capacity, kks_handle** out) {
  KKS_RANGE("kks_create");
  if (!params || !out) return set_error(KKS_ERR_ARG, "null argument");
  *out = nullptr;
  if (params->nx < 2 || params->ny < 2) return set_error(KKS_ERR_ARG, "nx and ny must be >= 2 (np.gradient)");
  if ((long long)params->nx * params->ny > (1LL << 30)) return set_error(KKS_ERR_ARG, "grid too large");
  if (precision != KKS_PRECISION_FP64 && precision != KKS_PRECISION_MIXED && precision != KKS_PRECISION_MIXED_CUFFT)
    return set_error(KKS_ERR_ARG, "precision must be KKS_PRECISION_FP64, _MIXED or _MIXED_CUFFT");
  if (params->n_sched < 1 || params->n_sched > KKS_MAX_SCHED)
    return set_error(KKS_ERR_ARG, "schedule length out of range");
  if (params->n_table < 1 || params->n_table > KKS_MAX_TABLE)
    return set_error(KKS_ERR_ARG, "table length out of range");
  if (n_steps < 0 || (n_steps > 0 && !step_flags)) return set_error(KKS_ERR_ARG, "bad step schedule");
  kks_handle* h = new (std::nothrow) kks_handle();
  if (!h) return set_error(KKS_ERR_ARG, "out of host memory");
  h->device = device;
  h->precision = precision;
  h->ring_cap = record_capacity > 64 ? record_capacity : 64;
  h->row_cap = 4096;
  int rc = create_impl(h, params, n_steps, step_flags);
  if (rc != KKS_OK) {
    std::string msg = g_last_error;
    free_handle(h);
    g_last_error = msg;
    return rc;
  }
  *out = h;
  return KKS_OK;
}

// Host float64 field -> device field of type R (state fields eta and X are
// float64 on both paths; X_al, X_th follow the path's precision).
static int put_field(kks_handle* h, void* dst, bool is_double, const double* src) {
  const int N = h->hc.N;
  if (is_double) {
    CK(cudaMemcpyAsync(dst, src, N * sizeof(double), cudaMemcpyHostToDevice, h->stream));
  } else {
    CK(cudaMemcpyAsync(h->d_xfer, src, N * sizeof(double), cudaMemcpyHostToDevice, h->stream));
    kks_launch_to_real<float>(h->d_xfer, (float*)dst, N, h->stream);
    CK(cudaGetLastError());
  }
  return KKS_OK;
}

static int get_field(kks_handle* h, double* dst, const void* src, bool is_double) {
  const int N = h->hc.N;
  if (is_double) {
    CK(cudaMemcpyAsync(dst, src, N * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  } else {
    kks_launch_to_double<float>((const float*)src, h->d_xfer, N, h->stream);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(dst, h->d_xfer, N * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  }
  CK(cudaStreamSynchronize(h->stream));
  return KKS_OK;
}

static int reset_loop(kks_handle* h);

int kks_upload(kks_handle* h, const double* eta, const double* X, const double* X_al, const double* X_th) {
  KKS_RANGE("kks_upload");
  if (!h || !eta || !X || !X_al || !X_th) return set_error(KKS_ERR_ARG, "null argument");
  CK(cudaSetDevice(h->device));
  const bool d = h->precision == KKS_PRECISION_FP64;
  int rc;
  if ((rc = put_field(h, h->f.eta[0], true, eta)) != KKS_OK) return rc;
  if ((rc = put_field(h, h->f.X[0], true, X)) != KKS_OK) return rc;
  if ((rc = put_field(h, h->f.X_al[0], d, X_al)) != KKS_OK) return rc;
  if ((rc = put_field(h, h->f.X_th[0], d, X_th)) != KKS_OK) return rc;
  return reset_loop(h);
}

// Initial loop state (pf_kks/solver.py:118-175) once state[0] holds the fields.
static int reset_loop(kks_handle* h) {
  KksCtl* c = h->h_ctl;
  memset(c, 0, sizeof(KksCtl));
  c->iteration = 1;
  c->minus_is_state = 1;
  c->gm = 0; c->gs = 1; c->gb = 2;
  c->Xv = h->hc.p.Xv0;
  c->dtime_s = h->hc.p.dtime_s;
  CK(cudaMemcpyAsync(h->d_ctl, c, sizeof(KksCtl), cudaMemcpyHostToDevice, h->stream));
  CK(cudaMemsetAsync(h->d_par, 0, sizeof(KksPar), h->stream));
  CK(cudaStreamSynchronize(h->stream));
  h->parity = 0;
  h->rec_read = h->row_read = 0;
  h->recs.clear();
  h->rows.clear();
  h->uploaded = true;
  h->attempts_launched = 0;
  return KKS_OK;
}

static int drain_device(kks_handle* h) {
  const KksCtl* c = h->h_ctl;
  while (h->rec_read < c->n_rec) {
    long long start = h->rec_read % h->ring_cap;
    long long n = std::min(c->n_rec - h->rec_read, h->ring_cap - start);
    size_t old = h->recs.size();
    h->recs.resize(old + n);
    CK(cudaMemcpy(h->recs.data() + old, h->d_ring + start, n * sizeof(kks_record), cudaMemcpyDeviceToHost));
    h->rec_read += n;
  }
  while (h->row_read < c->n_row) {
    long long start = h->row_read % h->row_cap;
    long long n = std::min(c->n_row - h->row_read, h->row_cap - start);
    size_t old = h->rows.size();
    h->rows.resize(old + n);
    CK(cudaMemcpy(h->rows.data() + old, h->d_rows + start, n * sizeof(kks_step_row), cudaMemcpyDeviceToHost));
    h->row_read += n;
  }
  return KKS_OK;
}

int kks_run(kks_handle* h, int32_t n_steps, int32_t* status) {
  KKS_RANGE("kks_run");
  if (!h || n_steps < 0) return set_error(KKS_ERR_ARG, "bad argument");
  if (!h->uploaded) return set_error(KKS_ERR_STATE, "kks_run before kks_upload");
  CK(cudaSetDevice(h->device));
  KksCtl* c = h->h_ctl;
  if (c->status != KKS_STATUS_OK) {
    if (status) *status = c->status;
    return KKS_OK;
  }
  const long long target = (long long)c->istep + n_steps;
  if (target > h->hc.n_steps) return set_error(KKS_ERR_ARG, "run beyond the scheduled number of steps");
  *h->h_target = (int32_t)target;
  CK(cudaMemcpyAsync(&h->d_ctl->target_step, h->h_target, sizeof(int32_t), cudaMemcpyHostToDevice, h->stream));
  CK(cudaEventRecord(h->ev0, h->stream));
  const long long max_batch = std::max(1LL, std::min(h->ring_cap / 2 - 1, h->row_cap - 1));
  long long launched = 0;
  while (c->istep < target && c->status == KKS_STATUS_OK) {
    long long todo = std::min(target - c->istep, max_batch);
    KKS_RANGE("attempt graphs");
    for (long long a = 0; a < todo; ++a) {
      CK(cudaGraphLaunch(h->graph[h->parity], h->stream));
      h->parity ^= 1;
    }
    launched += todo;
    CK(cudaMemcpyAsync(c, h->d_ctl, sizeof(KksCtl), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    int rc = drain_device(h);
    if (rc != KKS_OK) return rc;
  }
  CK(cudaEventRecord(h->ev1, h->stream));
  CK(cudaEventSynchronize(h->ev1));
  float ms = 0.f;
  CK(cudaEventElapsedTime(&ms, h->ev0, h->ev1));
  h->device_ms += ms;
  h->timed_attempts += launched;
  h->attempts_launched += launched;
  // attempts launched after a stop did not run: the device's parity is the state's
  h->parity = c->parity;
  if (status) *status = c->status;
  return KKS_OK;
}

int kks_run_many(kks_handle** cells, int32_t n_cells, const int32_t* n_steps, int32_t* status) {
  KKS_RANGE("kks_run_many");
  if (!cells || n_cells < 0 || (n_cells > 0 && !n_steps)) return set_error(KKS_ERR_ARG, "bad argument");
  std::vector<long long> target(n_cells), launched(n_cells, 0);
  for (int i = 0; i < n_cells; ++i) {
    kks_handle* h = cells[i];
    if (!h || n_steps[i] < 0) return set_error(KKS_ERR_ARG, "bad cell or step count");
    if (!h->uploaded) return set_error(KKS_ERR_STATE, "kks_run_many before kks_upload");
    if (i > 0 && h->device != cells[0]->device) return set_error(KKS_ERR_ARG, "cells must share one device");
    target[i] = (long long)h->h_ctl->istep + n_steps[i];
    if (target[i] > h->hc.n_steps) return set_error(KKS_ERR_ARG, "run beyond the scheduled number of steps");
  }
  if (n_cells == 0) return KKS_OK;
  CK(cudaSetDevice(cells[0]->device));
  for (int i = 0; i < n_cells; ++i) {
    kks_handle* h = cells[i];
    *h->h_target = (int32_t)target[i];
    CK(cudaMemcpyAsync(&h->d_ctl->target_step, h->h_target, sizeof(int32_t), cudaMemcpyHostToDevice, h->stream));
    CK(cudaEventRecord(h->ev0, h->stream));
  }
  for (;;) {
    bool any = false;
    for (int i = 0; i < n_cells; ++i) {
      kks_handle* h = cells[i];
      KksCtl* c = h->h_ctl;
      if (c->istep >= target[i] || c->status != KKS_STATUS_OK) continue;
      const long long max_batch = std::max(1LL, std::min(h->ring_cap / 2 - 1, h->row_cap - 1));
      const long long todo = std::min(target[i] - c->istep, max_batch);
      for (long long a = 0; a < todo; ++a) {
        CK(cudaGraphLaunch(h->graph[h->parity], h->stream));
        h->parity ^= 1;
      }
      launched[i] += todo;
      CK(cudaMemcpyAsync(c, h->d_ctl, sizeof(KksCtl), cudaMemcpyDeviceToHost, h->stream));
      any = true;
    }
    if (!any) break;
    for (int i = 0; i < n_cells; ++i) {
      CK(cudaStreamSynchronize(cells[i]->stream));
      int rc = drain_device(cells[i]);
      if (rc != KKS_OK) return rc;
    }
  }
  for (int i = 0; i < n_cells; ++i) {
    kks_handle* h = cells[i];
    CK(cudaEventRecord(h->ev1, h->stream));
    CK(cudaEventSynchronize(h->ev1));
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, h->ev0, h->ev1));
    h->device_ms += ms;
    h->timed_attempts += launched[i];
    h->attempts_launched += launched[i];
    h->parity = h->h_ctl->parity;
    if (status) status[i] = h->h_ctl->status;
  }
  return KKS_OK;
}

// ---------------------------------------------------------------------------
// Batches: cells of one device on the fused mixed pipeline, advanced together.
// One attempt of the batch is one launch per kernel for all cells (block maps
// built here, largest cells first), captured once as a CUDA graph; each cell's
// state parity, target step, dt and rejections stay on the device, so cells
// of different sizes and schedules advance in lockstep without a host
// decision, and a cell that has reached its target or stopped sits out.
// A batch may split its cells into groups of about equal cost, each with its
// own stream and graph: the groups' passes overlap, so that one group's pass
// tails and scalar kernels run beside another group's work.
struct BatchGroup {
  std::vector<int> idx;  // cells of the batch in this group
  cudaStream_t stream = nullptr;
  cudaGraphExec_t graph = nullptr;
  cudaEvent_t done = nullptr;
  KksCellDesc* d_cells = nullptr;
  int2* d_maps = nullptr;
  KksBatchLaunch L{};
};

struct kks_batch {
  std::vector<kks_handle*> cells;
  std::vector<BatchGroup> groups;
  int device = 0;
  int32_t* h_stage = nullptr;  // pinned: target step per cell
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  double device_ms = 0.0;
  long long attempts = 0;
  long long max_batch = 1;
};

static void free_batch(kks_batch* b) {
  if (!b) return;
  for (BatchGroup& g : b->groups) {
    if (g.stream) cudaStreamSynchronize(g.stream);
    if (g.graph) cudaGraphExecDestroy(g.graph);
    cudaFree(g.d_cells);
    cudaFree(g.d_maps);
    if (g.done) cudaEventDestroy(g.done);
    if (g.stream) cudaStreamDestroy(g.stream);
  }
  if (b->h_stage) cudaFreeHost(b->h_stage);
  if (b->ev0) cudaEventDestroy(b->ev0);
  if (b->ev1) cudaEventDestroy(b->ev1);
  delete b;
}

static void fill_desc(KksCellDesc& d, const kks_handle* h) {
  memset(&d, 0, sizeof(d));
  const KksFftLaunch& L = h->fl;
  const KksFieldPtrs& f = h->f;
  d.map_RA3 = L.map_RA3;
  d.map_RB3 = L.map_RB3;
  d.map_RB2 = L.map_RB2;
  d.dc = h->dc;
  d.par = h->d_par;
  d.ctl = h->d_ctl;
  d.fc = h->d_fc;
  for (int p = 0; p < 2; ++p) {
    d.eta[p] = (double*)f.eta[p];
    d.X[p] = (double*)f.X[p];
    d.X_al[p] = (float*)f.X_al[p];
    d.X_th[p] = (float*)f.X_th[p];
  }
  d.eta_m = (double*)f.eta_m;
  d.X_m = (double*)f.X_m;
  d.mu = (float*)f.mu;
  for (int k = 0; k < 3; ++k) d.g[k] = (float*)f.g[k];
  d.RA = (float2*)L.RA;
  d.RB = (float2*)L.RB;
  d.SA = (float2*)L.SA;
  d.partials = h->partials_fused;
  d.ky = h->d_ky;
  d.step_flags = h->d_flags;
  d.ring = h->d_ring;
  d.ring_cap = h->ring_cap;
  d.rows = h->d_rows;
  d.row_cap = h->row_cap;
  d.N = h->hc.N;
  d.nbx = h->nblocks;
  d.part_rows = h->nb_fused;
  d.bulk_rows = L.bulk_rows;
  d.bulk_cols = L.bulk_cols;
}

static int group_create(kks_batch* b, BatchGroup& G) {
  const int n = (int)G.idx.size();
  CK(cudaStreamCreateWithFlags(&G.stream, cudaStreamNonBlocking));
  CK(cudaEventCreateWithFlags(&G.done, cudaEventDisableTiming));
  std::vector<KksCellDesc> desc(n);
  std::vector<int> nx(n), ny(n), tile(n);
  for (int i = 0; i < n; ++i) {
    const kks_handle* h = b->cells[G.idx[i]];
    fill_desc(desc[i], h);
    nx[i] = h->hc.nx;
    ny[i] = h->hc.ny;
    tile[i] = h->fl.cols;
  }
  // largest cells first, so that the small ones fill the last wave of a pass
  std::vector<int> order(n);
  for (int i = 0; i < n; ++i) order[i] = i;
  std::stable_sort(order.begin(), order.end(), [&](int a, int c) { return nx[a] * ny[a] > nx[c] * ny[c]; });
  std::vector<int2> rows, cols, cols3, extras;
  for (int i : order) {
    const int nr = kks_fft_row_blocks(nx[i]), nc = kks_fft_col_blocks(ny[i] / 2 + 1, tile[i]);
    for (int k = 0; k < nr; ++k) rows.push_back(make_int2(i, k));
    for (int k = 0; k < nc; ++k) cols.push_back(make_int2(i, k));
    for (int r = 0; r < 3; ++r)
      for (int k = 0; k < nc; ++k) cols3.push_back(make_int2(i, (r << 16) | k));
    for (int k = 0; k < desc[i].nbx; ++k) extras.push_back(make_int2(i, k));
  }
  KksBatchLaunch& L = G.L;
  L.n_cells = n;
  L.PX = b->cells[0]->fl.PX;
  L.PY = b->cells[0]->fl.PY;
  L.n_rows = (int)rows.size();
  L.n_cols = (int)cols.size();
  L.n_cols3 = (int)cols3.size();
  L.n_extras = (int)extras.size();
  CK(cudaMalloc(&G.d_cells, n * sizeof(KksCellDesc)));
  CK(cudaMemcpy(G.d_cells, desc.data(), n * sizeof(KksCellDesc), cudaMemcpyHostToDevice));
  const size_t nm = rows.size() + cols.size() + cols3.size() + extras.size();
  CK(cudaMalloc(&G.d_maps, nm * sizeof(int2)));
  int2* m = G.d_maps;
  for (const std::vector<int2>* v : {&rows, &cols, &cols3, &extras}) {
    CK(cudaMemcpy(m, v->data(), v->size() * sizeof(int2), cudaMemcpyHostToDevice));
    if (v == &rows) L.map_rows = m;
    else if (v == &cols) L.map_cols = m;
    else if (v == &cols3) L.map_cols3 = m;
    else L.map_extras = m;
    m += v->size();
  }
  L.cells = G.d_cells;
  if (kks_fft_batch_prepare(L, nx.data(), ny.data(), tile.data(), n) != 0)
    return set_error(KKS_ERR_CUDA, "batched fft kernel attributes");
  cudaGraph_t g = nullptr;
  CK(cudaStreamBeginCapture(G.stream, cudaStreamCaptureModeThreadLocal));
  kks_fft_launch_attempt_batch(L, G.stream);
  const cudaError_t le = cudaGetLastError();
  cudaError_t e = cudaStreamEndCapture(G.stream, &g);
  if (le != cudaSuccess) e = le;
  if (e != cudaSuccess) {
    if (g) cudaGraphDestroy(g);
    return set_error(KKS_ERR_CUDA, std::string("batch graph capture: ") + cudaGetErrorString(e));
  }
  e = cudaGraphInstantiate(&G.graph, g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) return set_error(KKS_ERR_CUDA, std::string("batch graph instantiate: ") + cudaGetErrorString(e));
  return KKS_OK;
}

static int batch_create_impl(kks_batch* b, int n_groups) {
  const int n = (int)b->cells.size();
  CK(cudaSetDevice(b->device));
  CK(cudaEventCreate(&b->ev0));
  CK(cudaEventCreate(&b->ev1));
  CK(cudaMallocHost(&b->h_stage, n * sizeof(int32_t)));
  // longest-processing-time split by N log N (the transforms' cost)
  std::vector<int> order(n);
  for (int i = 0; i < n; ++i) order[i] = i;
  auto cost = [&](int i) { const double N = b->cells[i]->hc.N; return N * std::log2(std::max(N, 2.0)); };
  std::stable_sort(order.begin(), order.end(), [&](int a, int c) { return cost(a) > cost(c); });
  b->groups.resize(n_groups);
  std::vector<double> load(n_groups, 0.0);
  for (int i : order) {
    const int g = (int)(std::min_element(load.begin(), load.end()) - load.begin());
    b->groups[g].idx.push_back(i);
    load[g] += cost(i);
  }
  for (BatchGroup& G : b->groups) {
    std::sort(G.idx.begin(), G.idx.end());
    const int rc = group_create(b, G);
    if (rc != KKS_OK) return rc;
  }
  b->max_batch = 1LL << 30;
  for (kks_handle* h : b->cells)
    b->max_batch = std::min(b->max_batch, std::max(1LL, std::min(h->ring_cap / 2 - 1, h->row_cap - 1)));
  return KKS_OK;
}

int kks_batch_create(kks_handle* const* cells, int32_t n_cells, int32_t groups, kks_batch** out) {
  KKS_RANGE("kks_batch_create");
  if (!cells || !out || n_cells < 1 || groups < 1) return set_error(KKS_ERR_ARG, "bad argument");
  *out = nullptr;
  for (int i = 0; i < n_cells; ++i) {
    const kks_handle* h = cells[i];
    if (!h) return set_error(KKS_ERR_ARG, "null cell");
    if (!h->fused || h->fl.f64)
      return set_error(KKS_ERR_ARG, "batched cells must use the fused mixed pipeline (KKS_PRECISION_MIXED, supported sizes)");
    if (h->device != cells[0]->device) return set_error(KKS_ERR_ARG, "cells must share one device");
    if (h->fl.PX != cells[0]->fl.PX || h->fl.PY != cells[0]->fl.PY)
      return set_error(KKS_ERR_ARG, "batched cells must share the large prime factor of each axis");
    for (int j = 0; j < i; ++j)
      if (cells[j] == h) return set_error(KKS_ERR_ARG, "a cell appears twice in the batch");
  }
  kks_batch* b = new (std::nothrow) kks_batch();
  if (!b) return set_error(KKS_ERR_ARG, "out of host memory");
  b->cells.assign(cells, cells + n_cells);
  b->device = cells[0]->device;
  const int rc = batch_create_impl(b, std::min(groups, n_cells));
  if (rc != KKS_OK) {
    std::string msg = g_last_error;
    free_batch(b);
    g_last_error = msg;
    return rc;
  }
  for (kks_handle* h : b->cells) h->in_batch += 1;
  *out = b;
  return KKS_OK;
}

int kks_batch_run(kks_batch* b, const int32_t* n_steps, int32_t* status) {
  KKS_RANGE("kks_batch_run");
  if (!b || !n_steps) return set_error(KKS_ERR_ARG, "bad argument");
  const int n = (int)b->cells.size();
  std::vector<long long> target(n);
  for (int i = 0; i < n; ++i) {
    kks_handle* h = b->cells[i];
    if (n_steps[i] < 0) return set_error(KKS_ERR_ARG, "negative step count");
    if (!h->uploaded) return set_error(KKS_ERR_STATE, "kks_batch_run before kks_upload of every cell");
    target[i] = (long long)h->h_ctl->istep + n_steps[i];
    if (target[i] > h->hc.n_steps) return set_error(KKS_ERR_ARG, "run beyond the scheduled number of steps");
  }
  CK(cudaSetDevice(b->device));
  cudaStream_t s0 = b->groups[0].stream;
  for (BatchGroup& G : b->groups) {
    for (int i : G.idx) {
      kks_handle* h = b->cells[i];
      CK(cudaStreamSynchronize(h->stream));  // the cell's own work (uploads, runs) is done
      b->h_stage[i] = (int32_t)target[i];
      CK(cudaMemcpyAsync(&h->d_ctl->target_step, &b->h_stage[i], sizeof(int32_t), cudaMemcpyHostToDevice,
                         G.stream));
    }
  }
  CK(cudaEventRecord(b->ev0, s0));
  for (size_t g = 1; g < b->groups.size(); ++g) CK(cudaStreamWaitEvent(b->groups[g].stream, b->ev0, 0));
  long long launched = 0;
  for (;;) {
    long long most = 0;
    for (BatchGroup& G : b->groups) {
      long long todo = 0;
      for (int i : G.idx) {
        const KksCtl* c = b->cells[i]->h_ctl;
        if (c->status == KKS_STATUS_OK && c->istep < target[i]) todo = std::max(todo, target[i] - c->istep);
      }
      todo = std::min(todo, b->max_batch);
      for (long long a = 0; a < todo; ++a) CK(cudaGraphLaunch(G.graph, G.stream));
      if (todo > 0)
        for (int i : G.idx) {
          kks_handle* h = b->cells[i];
          CK(cudaMemcpyAsync(h->h_ctl, h->d_ctl, sizeof(KksCtl), cudaMemcpyDeviceToHost, G.stream));
        }
      most = std::max(most, todo);
    }
    if (most == 0) break;
    launched += most;
    for (BatchGroup& G : b->groups) CK(cudaStreamSynchronize(G.stream));
    for (int i = 0; i < n; ++i) {
      int rc = drain_device(b->cells[i]);
      if (rc != KKS_OK) return rc;
    }
  }
  for (size_t g = 1; g < b->groups.size(); ++g) {
    CK(cudaEventRecord(b->groups[g].done, b->groups[g].stream));
    CK(cudaStreamWaitEvent(s0, b->groups[g].done, 0));
  }
  CK(cudaEventRecord(b->ev1, s0));
  CK(cudaEventSynchronize(b->ev1));
  float ms = 0.f;
  CK(cudaEventElapsedTime(&ms, b->ev0, b->ev1));
  b->device_ms += ms;
  b->attempts += launched;
  for (int i = 0; i < n; ++i) {
    kks_handle* h = b->cells[i];
    h->parity = h->h_ctl->parity;
    if (status) status[i] = h->h_ctl->status;
  }
  return KKS_OK;
}

int kks_batch_timing(const kks_batch* b, double* device_ms, int64_t* attempts) {
  if (!b) return set_error(KKS_ERR_ARG, "null batch");
  if (device_ms) *device_ms = b->device_ms;
  if (attempts) *attempts = b->attempts;
  return KKS_OK;
}

int kks_batch_destroy(kks_batch* b) {
  if (!b) return KKS_OK;
  CK(cudaSetDevice(b->device));
  for (kks_handle* h : b->cells) h->in_batch -= 1;
  free_batch(b);
  return KKS_OK;
}

int kks_drain(kks_handle* h, kks_record* records, int64_t record_cap, int64_t* n_records, kks_step_row* rows,
              int64_t row_cap, int64_t* n_rows) {
  KKS_RANGE("kks_drain");
  if (!h) return set_error(KKS_ERR_ARG, "null handle");
  if (n_records) {
    if (!records && record_cap > 0) return set_error(KKS_ERR_ARG, "null record buffer");
    int64_t n = std::min<int64_t>(record_cap, (int64_t)h->recs.size());
    if (n > 0) memcpy(records, h->recs.data(), n * sizeof(kks_record));
    h->recs.erase(h->recs.begin(), h->recs.begin() + n);
    *n_records = n;
  }
  if (n_rows) {
    if (!rows && row_cap > 0) return set_error(KKS_ERR_ARG, "null row buffer");
    int64_t n = std::min<int64_t>(row_cap, (int64_t)h->rows.size());
    if (n > 0) memcpy(rows, h->rows.data(), n * sizeof(kks_step_row));
    h->rows.erase(h->rows.begin(), h->rows.begin() + n);
    *n_rows = n;
  }
  return KKS_OK;
}

int kks_get_state(kks_handle* h, kks_run_state* s) {
  if (!h || !s) return set_error(KKS_ERR_ARG, "null argument");
  const KksCtl* c = h->h_ctl;
  s->istep = c->istep;
  s->iteration = c->iteration;
  s->flag = c->flag;
  s->good_step = c->good_step;
  s->status = c->status;
  s->parity = h->parity;
  s->attempts = c->attempts;
  s->n_records = (int64_t)h->recs.size();
  s->n_rows = (int64_t)h->rows.size();
  s->t = c->t;
  s->t_s = c->t_s;
  s->t_b = c->t_b;
  s->ttime = c->ttime;
  s->Xv = c->Xv;
  s->dtime_s = c->dtime_s;
  s->D_0 = c->D_0;
  s->Meta_0 = c->Meta_0;
  s->surf = c->surf;
  s->surf_b = c->surf_b;
  s->T_b = c->T_b;
  s->error_istep = c->error_istep;
  s->error_iteration = c->error_iteration;
  s->error_dtime_s = c->error_dtime_s;
  return KKS_OK;
}

int kks_download(kks_handle* h, double* eta, double* X, double* X_al, double* X_th) {
  KKS_RANGE("kks_download");
  if (!h) return set_error(KKS_ERR_ARG, "null handle");
  if (!h->uploaded) return set_error(KKS_ERR_STATE, "kks_download before kks_upload");
  CK(cudaSetDevice(h->device));
  const bool d = h->precision == KKS_PRECISION_FP64;
  const int p = h->parity;
  int rc;
  if (eta && (rc = get_field(h, eta, h->f.eta[p], true)) != KKS_OK) return rc;
  if (X && (rc = get_field(h, X, h->f.X[p], true)) != KKS_OK) return rc;
  if (X_al && (rc = get_field(h, X_al, h->f.X_al[p], d)) != KKS_OK) return rc;
  if (X_th && (rc = get_field(h, X_th, h->f.X_th[p], d)) != KKS_OK) return rc;
  return KKS_OK;
}

int kks_bounds_report(int device, int32_t* checked, uint64_t* first) {
  if (!checked || !first) return set_error(KKS_ERR_ARG, "null argument");
  CK(cudaSetDevice(device));
  unsigned long long w = 0;
  const int rc = kks_fft_bounds_word(&w, 1);
  if (rc < 0) return set_error(KKS_ERR_CUDA, "reading the bounds-check word");
  *checked = rc;
  *first = (uint64_t)w;
  return KKS_OK;
}

int kks_set_wait_polls(kks_handle* h, int32_t polls) {
  if (!h) return set_error(KKS_ERR_ARG, "null handle");
  if (!h->fused_ok || !h->d_fc || h->fl.f64)
    return set_error(KKS_ERR_STATE, "the cell has no bulk copies in its passes (nothing waits)");
  const int v = polls < 0 ? KKS_FFT_WAIT_POLLS : polls;
  CK(cudaSetDevice(h->device));
  CK(cudaStreamSynchronize(h->stream));
  CK(cudaMemcpy(&h->d_fc->wait_polls, &v, sizeof(int), cudaMemcpyHostToDevice));
  return KKS_OK;
}

int kks_download_pair(kks_handle* h, double* eta_m, double* X_m, double* mu_m, double* G_m) {
  KKS_RANGE("kks_download_pair");
  if (!h) return set_error(KKS_ERR_ARG, "null handle");
  if (!h->uploaded) return set_error(KKS_ERR_STATE, "kks_download_pair before kks_upload");
  CK(cudaSetDevice(h->device));
  const KksCtl* c = h->h_ctl;
  const bool d = h->precision == KKS_PRECISION_FP64;
  // after an accepted step the minus entry is the step's input state itself;
  // after a rejection it is the saved copy of the rejected attempt
  const void* e = c->minus_is_state ? h->f.eta[h->parity] : h->f.eta_m;
  const void* x = c->minus_is_state ? h->f.X[h->parity] : h->f.X_m;
  if (c->gm < 0 || c->gm > 2) return set_error(KKS_ERR_STATE, "residual pair not set");
  int rc;
  if (eta_m && (rc = get_field(h, eta_m, e, true)) != KKS_OK) return rc;
  if (X_m && (rc = get_field(h, X_m, x, true)) != KKS_OK) return rc;
  if (mu_m && (rc = get_field(h, mu_m, h->f.mu, d)) != KKS_OK) return rc;
  if (G_m && (rc = get_field(h, G_m, h->f.g[c->gm], d)) != KKS_OK) return rc;
  return KKS_OK;
}

// ---------------------------------------------------------------------------
// Initial state on the device (kks_init.cu).

static int ensure_sel(kks_handle* h) {
  if (!h->sel) CK(cudaMalloc(&h->sel, (2 * (size_t)kks_init_chunks(h->hc.N) + 1) * sizeof(long long)));
  return KKS_OK;
}

static int ensure_init_buf(kks_handle* h, size_t bytes) {
  if (bytes <= h->init_bytes) return KKS_OK;
  CK(cudaStreamSynchronize(h->stream));
  cudaFree(h->init_buf);
  h->init_buf = nullptr;
  h->init_bytes = 0;
  CK(cudaMalloc(&h->init_buf, bytes));
  h->init_bytes = bytes;
  return KKS_OK;
}

// chunk counts at sel[0..nc), offsets at sel[nc..2nc]
static long long* sel_cnt(kks_handle* h) { return h->sel; }
static long long* sel_off(kks_handle* h) { return h->sel + kks_init_chunks(h->hc.N); }

static int sel_total(kks_handle* h, long long* total) {
  CK(cudaMemcpyAsync(total, sel_off(h) + kks_init_chunks(h->hc.N), sizeof(long long), cudaMemcpyDeviceToHost,
                     h->stream));
  CK(cudaStreamSynchronize(h->stream));
  return KKS_OK;
}

static size_t align256(size_t v) { return (v + 255) / 256 * 256; }

int kks_voronoi_edges(kks_handle* h, int32_t n_seeds, const double* seeds, int64_t* n_edges) {
  KKS_RANGE("kks_voronoi_edges");
  if (!h || !seeds || !n_edges) return set_error(KKS_ERR_ARG, "null argument");
  if (n_seeds < 1) return set_error(KKS_ERR_ARG, "kks_voronoi_edges: n_seeds < 1");
  CK(cudaSetDevice(h->device));
  int rc;
  if ((rc = ensure_sel(h)) != KKS_OK) return rc;
  if ((rc = ensure_init_buf(h, align256(2 * (size_t)n_seeds * sizeof(double)))) != KKS_OK) return rc;
  h->edges_ready = false;
  CK(cudaMemcpyAsync(h->init_buf, seeds, 2 * (size_t)n_seeds * sizeof(double), cudaMemcpyHostToDevice, h->stream));
  // labels live in the parity-1 eta buffer until the first attempt overwrites it
  int32_t* labels = (int32_t*)h->f.eta[1];
  kks_init_labels((const double*)h->init_buf, n_seeds, h->hc.nx, h->hc.ny, labels, h->stream);
  kks_init_count_edges(labels, h->hc.nx, h->hc.ny, sel_cnt(h), sel_off(h), h->stream);
  CK(cudaGetLastError());
  long long total = 0;
  if ((rc = sel_total(h, &total)) != KKS_OK) return rc;
  h->n_edges = total;
  h->edges_ready = true;
  *n_edges = total;
  return KKS_OK;
}

int kks_generate_fields(kks_handle* h, const kks_gen_args* a) {
  KKS_RANGE("kks_generate_fields");
  if (!h || !a) return set_error(KKS_ERR_ARG, "null argument");
  const int n = a->n_particles;
  if (n < 0 || (n > 0 && (!a->pick || !a->jitter || !a->radii)))
    return set_error(KKS_ERR_ARG, "kks_generate_fields: bad particle arrays");
  if (!(a->w > 0.0)) return set_error(KKS_ERR_ARG, "kks_generate_fields: w <= 0");
  const long long range = a->picks_are_points ? (long long)h->hc.N : h->n_edges;
  if (!a->picks_are_points && !h->edges_ready)
    return set_error(KKS_ERR_STATE, "kks_generate_fields before kks_voronoi_edges");
  // windows reach ceil(R + 8 w) + 1 cells: keep them within int range
  if (!(a->w <= 1e6)) return set_error(KKS_ERR_ARG, "kks_generate_fields: w > 1e6");
  for (int j = 0; j < n; ++j) {
    if (a->pick[j] < 0 || a->pick[j] >= range) return set_error(KKS_ERR_ARG, "kks_generate_fields: pick out of range");
    if (!(fabs(a->radii[j]) <= 1e6) || !(fabs(a->jitter[2 * j]) <= 1e6) || !(fabs(a->jitter[2 * j + 1]) <= 1e6))
      return set_error(KKS_ERR_ARG, "kks_generate_fields: radius or jitter not finite or above 1e6 cells");
  }
  CK(cudaSetDevice(h->device));
  const size_t ids = align256(n * sizeof(long long));
  const size_t o_rank = 0, o_flat = ids, o_jit = 2 * ids, o_rad = o_jit + align256(2 * (size_t)n * sizeof(double)),
               o_part = o_rad + align256(n * sizeof(double)),
               total = o_part + align256(n * kks_init_particle_bytes()) + 256;
  int rc;
  if ((rc = ensure_init_buf(h, total)) != KKS_OK) return rc;
  char* b = (char*)h->init_buf;
  long long* ranks = (long long*)(b + o_rank);
  long long* flat = (long long*)(b + o_flat);
  double* jit = (double*)(b + o_jit);
  double* rad = (double*)(b + o_rad);
  if (n > 0) {
    CK(cudaMemcpyAsync(ranks, a->pick, n * sizeof(long long), cudaMemcpyHostToDevice, h->stream));
    CK(cudaMemcpyAsync(jit, a->jitter, 2 * (size_t)n * sizeof(double), cudaMemcpyHostToDevice, h->stream));
    CK(cudaMemcpyAsync(rad, a->radii, n * sizeof(double), cudaMemcpyHostToDevice, h->stream));
    if (a->picks_are_points) {
      CK(cudaMemcpyAsync(flat, ranks, n * sizeof(long long), cudaMemcpyDeviceToDevice, h->stream));
    } else {
      kks_init_select_edges((const int32_t*)h->f.eta[1], h->hc.nx, h->hc.ny, sel_off(h), ranks, n, flat, h->stream);
    }
  }
  double* eta = (double*)h->f.eta[0];
  kks_init_eta(flat, n, h->hc.nx, h->hc.ny, jit, rad, a->w, b + o_part, eta, h->stream);
  if (h->precision == KKS_PRECISION_FP64) {
    kks_init_fields<double>(h->hc.N, a->rng_state, a->rng_inc, a->x_matrix, a->noise_low, a->noise_range,
                            a->x_particle, a->pc_shift, a->pc_ratio, eta, (double*)h->f.X[0],
                            (double*)h->f.X_al[0], (double*)h->f.X_th[0], h->stream);
  } else {
    kks_init_fields<float>(h->hc.N, a->rng_state, a->rng_inc, a->x_matrix, a->noise_low, a->noise_range,
                           a->x_particle, a->pc_shift, a->pc_ratio, eta, (double*)h->f.X[0], (float*)h->f.X_al[0],
                           (float*)h->f.X_th[0], h->stream);
  }
  CK(cudaGetLastError());
  h->edges_ready = false;
  return reset_loop(h);
}

static int place_impl(kks_handle* h, bool add, double dx, double dy, double x_matrix, double x_precipitate,
                      int32_t n, const double* r, const double* ox, const double* oy, const double* oz) {
  if (!h) return set_error(KKS_ERR_ARG, "null handle");
  if (n < 0 || (n > 0 && (!r || !ox || !oy || !oz))) return set_error(KKS_ERR_ARG, "bad precipitate arrays");
  if (add && !h->uploaded) return set_error(KKS_ERR_STATE, "kks_add_nuclei before the fields are set");
  CK(cudaSetDevice(h->device));
  int rc;
  if ((rc = ensure_init_buf(h, align256(4 * (size_t)std::max(n, 1) * sizeof(double)))) != KKS_OK) return rc;
  double* prm = (double*)h->init_buf;
  const double* src[4] = {r, ox, oy, oz};
  for (int c = 0; c < 4 && n > 0; ++c)
    CK(cudaMemcpyAsync(prm + (size_t)c * n, src[c], n * sizeof(double), cudaMemcpyHostToDevice, h->stream));
  const int p = add ? h->parity : 0;
  double* eta = (double*)h->f.eta[p];
  double* X = (double*)h->f.X[p];
  if (h->precision == KKS_PRECISION_FP64)
    kks_init_place<double>(add, h->hc.nx, h->hc.ny, dx, dy, prm, n, x_matrix, x_precipitate, eta, X,
                           (double*)h->f.X_al[p], (double*)h->f.X_th[p], h->stream);
  else
    kks_init_place<float>(add, h->hc.nx, h->hc.ny, dx, dy, prm, n, x_matrix, x_precipitate, eta, X,
                          (float*)h->f.X_al[p], (float*)h->f.X_th[p], h->stream);
  CK(cudaGetLastError());
  if (!add) return reset_loop(h);
  CK(cudaStreamSynchronize(h->stream));
  return KKS_OK;
}

int kks_place_precipitates(kks_handle* h, double dx, double dy, double x_matrix, double x_precipitate, int32_t n,
                           const double* r, const double* ox, const double* oy, const double* oz) {
  KKS_RANGE("kks_place_precipitates");
  return place_impl(h, false, dx, dy, x_matrix, x_precipitate, n, r, ox, oy, oz);
}

int kks_add_nuclei(kks_handle* h, double dx, double dy, int32_t n, const double* r, const double* ox,
                   const double* oy, const double* oz) {
  KKS_RANGE("kks_add_nuclei");
  return place_impl(h, true, dx, dy, 0.0, 0.0, n, r, ox, oy, oz);
}

static int count_below(kks_handle* h, double eta_below, long long* count) {
  int rc;
  if ((rc = ensure_sel(h)) != KKS_OK) return rc;
  kks_init_count_below((const double*)h->f.eta[h->parity], eta_below, h->hc.N, sel_cnt(h), sel_off(h), h->stream);
  CK(cudaGetLastError());
  return sel_total(h, count);
}

int kks_count_below(kks_handle* h, double eta_below, int64_t* count) {
  if (!h || !count) return set_error(KKS_ERR_ARG, "null argument");
  if (!h->uploaded) return set_error(KKS_ERR_STATE, "kks_count_below before the fields are set");
  CK(cudaSetDevice(h->device));
  long long c = 0;
  int rc = count_below(h, eta_below, &c);
  *count = c;
  return rc;
}

int kks_insert_nuclei(kks_handle* h, double eta_below, int32_t n, const int64_t* ranks) {
  KKS_RANGE("kks_insert_nuclei");
  if (!h || (n > 0 && !ranks)) return set_error(KKS_ERR_ARG, "null argument");
  if (n < 0) return set_error(KKS_ERR_ARG, "kks_insert_nuclei: n < 0");
  if (!h->uploaded) return set_error(KKS_ERR_STATE, "kks_insert_nuclei before the fields are set");
  if (n == 0) return KKS_OK;
  CK(cudaSetDevice(h->device));
  long long c = 0;
  int rc;
  if ((rc = count_below(h, eta_below, &c)) != KKS_OK) return rc;
  for (int j = 0; j < n; ++j)
    if (ranks[j] < 0 || ranks[j] >= c) return set_error(KKS_ERR_ARG, "kks_insert_nuclei: rank out of range");
  if ((rc = ensure_init_buf(h, 2 * align256(n * sizeof(long long)))) != KKS_OK) return rc;
  long long* d_rank = (long long*)h->init_buf;
  long long* d_flat = (long long*)((char*)h->init_buf + align256(n * sizeof(long long)));
  CK(cudaMemcpyAsync(d_rank, ranks, n * sizeof(long long), cudaMemcpyHostToDevice, h->stream));
  double* eta = (double*)h->f.eta[h->parity];
  kks_init_select_below(eta, eta_below, h->hc.N, sel_off(h), d_rank, n, d_flat, h->stream);
  kks_init_set_eta(d_flat, n, 1.0, eta, h->stream);
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(h->stream));
  return KKS_OK;
}

}  // extern "C"

template <bool MIXED>
static int elastic_impl(kks_handle* h, int p, double* d_out) {
  KksFieldPtrs& f = h->f;
  cudaStream_t s = h->stream;
  kks_launch_prep<MIXED>(&h->hc, h->d_par, f, p, h->nblocks, s);
  if (!MIXED) {
    CKF(cufftExecD2Z(h->plan_r2c3, (double*)f.fft_in[p], (cufftDoubleComplex*)f.spec_a));
  } else {
    CKF(cufftExecR2C(h->plan_r2c3, (float*)f.fft_in[p], (cufftComplex*)f.spec_a));
  }
  kks_launch_strain_spectra<MIXED>(&h->hc, h->dc, h->d_par, f, h->nblocks, s);
  if (!MIXED) {
    CKF(cufftExecZ2D(h->plan_c2r3, (cufftDoubleComplex*)f.spec_bcd, (double*)f.real_b));
  } else {
    CKF(cufftExecC2R(h->plan_c2r3, (cufftComplex*)f.spec_bcd, (float*)f.real_b));
  }
  kks_launch_elastic_out<MIXED>(&h->hc, h->dc, h->d_par, f, p, d_out, d_out + 4 * (size_t)h->hc.N, h->nblocks, s);
  CK(cudaGetLastError());
  return KKS_OK;
}

extern "C" {

int kks_elastic_fields(kks_handle* h, double* sig4, double* eps4) {
  KKS_RANGE("kks_elastic_fields");
  if (!h || !sig4 || !eps4) return set_error(KKS_ERR_ARG, "null argument");
  if (!h->uploaded || h->attempts_launched == 0) return set_error(KKS_ERR_STATE, "no attempt has run yet");
  CK(cudaSetDevice(h->device));
  const int p = h->parity ^ 1;  // the last attempt read its input from the other buffer
  const size_t N = h->hc.N;
  double* d_out = nullptr;
  CK(cudaMalloc(&d_out, 8 * N * sizeof(double)));
  int one = 1;
  cudaError_t e = cudaMemcpyAsync(&h->d_par->active, &one, sizeof(int), cudaMemcpyHostToDevice, h->stream);
  int rc = e == cudaSuccess ? KKS_OK : set_error(KKS_ERR_CUDA, cudaGetErrorString(e));
  if (rc == KKS_OK)
    rc = h->precision == KKS_PRECISION_FP64 ? elastic_impl<false>(h, p, d_out) : elastic_impl<true>(h, p, d_out);
  if (rc == KKS_OK) {
    e = cudaMemcpyAsync(sig4, d_out, 4 * N * sizeof(double), cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(eps4, d_out + 4 * N, 4 * N * sizeof(double), cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) rc = set_error(KKS_ERR_CUDA, std::string("elastic fields: ") + cudaGetErrorString(e));
  }
  cudaStreamSynchronize(h->stream);
  cudaFree(d_out);
  return rc;
}

// checkpoint blob: header | KksCtl | state[0] | state[1] | eta_m | X_m | mu | g[0..2]
struct CkptHeader {
  char magic[8];
  int32_t nx, ny, precision, parity;
  uint64_t bytes;
};

static size_t ckpt_bytes(kks_handle* h) {
  const size_t Np = h->hc.Np;
  return sizeof(CkptHeader) + sizeof(KksCtl) + 2 * h->state_bytes + 2 * Np * sizeof(double) + 4 * Np * h->rsize;
}

static void ckpt_regions(kks_handle* h, void** ptr, size_t* len) {
  const size_t Np = h->hc.Np;
  ptr[0] = h->f.eta[0]; len[0] = h->state_bytes;
  ptr[1] = h->f.eta[1]; len[1] = h->state_bytes;
  ptr[2] = h->f.eta_m; len[2] = Np * sizeof(double);
  ptr[3] = h->f.X_m; len[3] = Np * sizeof(double);
  ptr[4] = h->f.mu; len[4] = Np * h->rsize;
  for (int k = 0; k < 3; ++k) { ptr[5 + k] = h->f.g[k]; len[5 + k] = Np * h->rsize; }
}

int kks_checkpoint(kks_handle* h, void* buf, size_t cap, size_t* size) {
  KKS_RANGE("kks_checkpoint");
  if (!h || !size) return set_error(KKS_ERR_ARG, "null argument");
  const size_t need = ckpt_bytes(h);
  *size = need;
  if (!buf) return KKS_OK;
  if (cap < need) return set_error(KKS_ERR_CAPACITY, "checkpoint buffer too small");
  if (!h->uploaded) return set_error(KKS_ERR_STATE, "nothing to checkpoint");
  CK(cudaSetDevice(h->device));
  CK(cudaStreamSynchronize(h->stream));
  char* o = (char*)buf;
  CkptHeader hd;
  memcpy(hd.magic, "KKSCKPT2", 8);
  hd.nx = h->hc.nx; hd.ny = h->hc.ny; hd.precision = h->precision; hd.parity = h->parity;
  hd.bytes = need;
  memcpy(o, &hd, sizeof(hd)); o += sizeof(hd);
  CK(cudaMemcpy(o, h->d_ctl, sizeof(KksCtl), cudaMemcpyDeviceToHost)); o += sizeof(KksCtl);
  void* ptr[8];
  size_t len[8];
  ckpt_regions(h, ptr, len);
  for (int k = 0; k < 8; ++k) { CK(cudaMemcpy(o, ptr[k], len[k], cudaMemcpyDeviceToHost)); o += len[k]; }
  return KKS_OK;
}

int kks_restore(kks_handle* h, const void* buf, size_t size) {
  KKS_RANGE("kks_restore");
  if (!h || !buf) return set_error(KKS_ERR_ARG, "null argument");
  const size_t need = ckpt_bytes(h);
  if (size < need) return set_error(KKS_ERR_CAPACITY, "checkpoint blob too small");
  const char* o = (const char*)buf;
  CkptHeader hd;
  memcpy(&hd, o, sizeof(hd)); o += sizeof(hd);
  if (memcmp(hd.magic, "KKSCKPT2", 8) != 0 || hd.nx != h->hc.nx || hd.ny != h->hc.ny ||
      hd.precision != h->precision || hd.bytes != need)
    return set_error(KKS_ERR_ARG, "checkpoint does not match this cell");
  CK(cudaSetDevice(h->device));
  CK(cudaStreamSynchronize(h->stream));
  memcpy(h->h_ctl, o, sizeof(KksCtl)); o += sizeof(KksCtl);
  h->h_ctl->target_step = h->h_ctl->istep;
  CK(cudaMemcpy(h->d_ctl, h->h_ctl, sizeof(KksCtl), cudaMemcpyHostToDevice));
  void* ptr[8];
  size_t len[8];
  ckpt_regions(h, ptr, len);
  for (int k = 0; k < 8; ++k) { CK(cudaMemcpy(ptr[k], o, len[k], cudaMemcpyHostToDevice)); o += len[k]; }
  CK(cudaMemset(h->d_par, 0, sizeof(KksPar)));
  h->parity = hd.parity;
  h->rec_read = h->h_ctl->n_rec;
  h->row_read = h->h_ctl->n_row;
  h->recs.clear();
  h->rows.clear();
  h->uploaded = true;
  h->attempts_launched = 0;
  return KKS_OK;
}

// ---------------------------------------------------------------------------
// Launch shapes and the autotuner.

static int apply_shape(kks_handle* h, const kks_launch_shape& s) {
  if (h->in_batch) return set_error(KKS_ERR_STATE, "the cell belongs to a batch: its launch shape is fixed");
  if (s.pipeline != 0 && s.pipeline != 1) return set_error(KKS_ERR_ARG, "pipeline must be 0 (cuFFT) or 1 (fused)");
  if (s.pipeline == 1 && !h->fused_ok)
    return set_error(KKS_ERR_ARG, "the fused passes are not available for this cell (precision or size)");
  if (s.field_blocks < 1 || s.field_blocks > h->nblocks_cap)
    return set_error(KKS_ERR_ARG, "field_blocks out of range (1 .. " + std::to_string(h->nblocks_cap) + ")");
  if (h->fused_ok) {
    if (s.cols < 1 || s.cols > KKS_FFT_COLS_MAX) return set_error(KKS_ERR_ARG, "cols out of range (1 .. 4)");
    int optin = 0;
    CK(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, h->device));
    const size_t need = h->fl.f64 ? kks_fft64_smem_bytes(h->hc.nx, h->hc.ny, s.cols)
                                  : kks_fft_smem_bytes(h->hc.nx, h->hc.ny, s.cols);
    if (need > (size_t)optin) return set_error(KKS_ERR_CAPACITY, "column tile does not fit shared memory");
  }
  CK(cudaSetDevice(h->device));
  CK(cudaStreamSynchronize(h->stream));
  for (int p = 0; p < 2; ++p) {
    if (h->graph[p]) cudaGraphExecDestroy(h->graph[p]);
    h->graph[p] = nullptr;
  }
  h->fused = s.pipeline == 1;
  h->nblocks = s.field_blocks;
  size_t rows = (size_t)h->nblocks_cap;
  if (h->fused_ok) {
    h->fl.cols = s.cols;
    h->fl.nbx = h->nblocks;
    CK(cudaMemcpy(&h->d_fc->cols, &h->fl.cols, sizeof(int), cudaMemcpyHostToDevice));
    if (kks_fft_set_attributes(h->fl) != 0) return set_error(KKS_ERR_CUDA, "fft kernel attributes");
    h->nb_fused = fused_rows(h);
    rows = (size_t)h->part_cap_fused;
  }
  // rows that the new shape does not write must read as zero
  CK(cudaMemset(h->f.partials, 0, rows * KKS_NPART * sizeof(double)));
  return capture_graphs(h);
}

static void current_shape(const kks_handle* h, kks_launch_shape* s) {
  s->pipeline = h->fused ? 1 : 0;
  s->cols = h->fused_ok ? h->fl.cols : 0;
  s->field_blocks = h->nblocks;
  s->pad = 0;
}

int kks_get_launch_shape(const kks_handle* h, kks_launch_shape* shape) {
  if (!h || !shape) return set_error(KKS_ERR_ARG, "null argument");
  current_shape(h, shape);
  return KKS_OK;
}

int kks_set_launch_shape(kks_handle* h, const kks_launch_shape* shape) {
  KKS_RANGE("kks_set_launch_shape");
  if (!h || !shape) return set_error(KKS_ERR_ARG, "null argument");
  return apply_shape(h, *shape);
}

// Candidates: the field-kernel grid at 1, 2, 4 and 8 blocks per SM (as far as
// the cell has points for), crossed with the column tiles 1..4 of the fused
// passes, and the cuFFT passes (unless only batchable shapes are wanted).
static std::vector<kks_launch_shape> candidate_shapes(const kks_handle* h, bool batchable) {
  std::vector<int> grids;
  for (int m : {1, 2, 4, 8}) {
    const int g = std::min(m * h->nsm, h->nblocks_cap);
    if (std::find(grids.begin(), grids.end(), g) == grids.end()) grids.push_back(g);
  }
  std::vector<kks_launch_shape> out;
  for (int g : grids) {
    if (h->fused_ok)
      for (int cols = 1; cols <= KKS_FFT_COLS_MAX; ++cols) out.push_back({1, cols, g, 0});
    if (!(batchable && h->fused_ok)) out.push_back({0, h->fused_ok ? h->fl.cols : 0, g, 0});
  }
  return out;
}

int kks_autotune(kks_handle* h, int32_t attempts, int32_t flags, kks_launch_shape* best,
                 double* best_ms_per_attempt) {
  KKS_RANGE("kks_autotune");
  if (!h || attempts < 1 || (flags & ~KKS_TUNE_BATCHABLE)) return set_error(KKS_ERR_ARG, "bad argument");
  if (!h->uploaded) return set_error(KKS_ERR_STATE, "kks_autotune before kks_upload");
  if (h->in_batch) return set_error(KKS_ERR_STATE, "the cell belongs to a batch: its launch shape is fixed");
  CK(cudaSetDevice(h->device));
  CK(cudaStreamSynchronize(h->stream));
  const KksCtl* c = h->h_ctl;
  if (c->status != KKS_STATUS_OK) return set_error(KKS_ERR_STATE, "the cell has stopped");
  const long long left = (long long)h->hc.n_steps - c->istep;
  const int warm = (int)std::min<long long>(3, left / 4);
  const int timed = (int)std::min<long long>(attempts, left - warm);
  if (timed < 1 || left < 2) return set_error(KKS_ERR_STATE, "too few scheduled steps left to time an attempt");
  // everything an attempt changes, saved and put back after every candidate
  size_t size = 0;
  int rc = kks_checkpoint(h, nullptr, 0, &size);
  if (rc != KKS_OK) return rc;
  std::vector<char> blob(size);
  if ((rc = kks_checkpoint(h, blob.data(), size, &size)) != KKS_OK) return rc;
  const std::vector<kks_record> recs = h->recs;
  const std::vector<kks_step_row> rows = h->rows;
  const long long rec_read = h->rec_read, row_read = h->row_read, launched = h->attempts_launched;
  const long long timed_attempts = h->timed_attempts;
  const double device_ms = h->device_ms;
  kks_launch_shape start;
  current_shape(h, &start);
  kks_launch_shape win = start;
  double win_ms = -1.0;
  const int32_t target = c->istep + warm + timed;
  for (const kks_launch_shape& cand : candidate_shapes(h, (flags & KKS_TUNE_BATCHABLE) != 0)) {
    if (apply_shape(h, cand) != KKS_OK) continue;  // e.g. a tile that does not fit
    if ((rc = kks_restore(h, blob.data(), size)) != KKS_OK) return rc;
    *h->h_target = target;
    CK(cudaMemcpyAsync(&h->d_ctl->target_step, h->h_target, sizeof(int32_t), cudaMemcpyHostToDevice, h->stream));
    for (int a = 0; a < warm; ++a) {
      CK(cudaGraphLaunch(h->graph[h->parity], h->stream));
      h->parity ^= 1;
    }
    CK(cudaEventRecord(h->ev0, h->stream));
    for (int a = 0; a < timed; ++a) {
      CK(cudaGraphLaunch(h->graph[h->parity], h->stream));
      h->parity ^= 1;
    }
    CK(cudaEventRecord(h->ev1, h->stream));
    CK(cudaMemcpyAsync(h->h_ctl, h->d_ctl, sizeof(KksCtl), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaEventSynchronize(h->ev1));
    CK(cudaStreamSynchronize(h->stream));
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, h->ev0, h->ev1));
    if (h->h_ctl->status != KKS_STATUS_OK) continue;  // a stop inside the trial: attempts did not all run
    const double per = ms / timed;
    if (win_ms < 0 || per < win_ms) {
      win_ms = per;
      win = cand;
    }
  }
  if ((rc = apply_shape(h, win)) != KKS_OK) return rc;
  if ((rc = kks_restore(h, blob.data(), size)) != KKS_OK) return rc;
  h->recs = recs;
  h->rows = rows;
  h->rec_read = rec_read;
  h->row_read = row_read;
  h->attempts_launched = launched;
  h->timed_attempts = timed_attempts;
  h->device_ms = device_ms;
  if (best) *best = win;
  if (best_ms_per_attempt) *best_ms_per_attempt = win_ms;
  return win_ms < 0 ? set_error(KKS_ERR_STATE, "no candidate shape completed its trial attempts") : KKS_OK;
}

int kks_timing(kks_handle* h, double* device_ms, int64_t* attempts) {
  if (!h) return set_error(KKS_ERR_ARG, "null handle");
  if (device_ms) *device_ms = h->device_ms;
  if (attempts) *attempts = h->timed_attempts;
  return KKS_OK;
}

int kks_pipeline(kks_handle* h, int32_t* fused, int32_t* kernels) {
  if (!h) return set_error(KKS_ERR_ARG, "null handle");
  if (fused) *fused = h->fused ? 1 : 0;
  // fused: prologue, rows A, cols AB, rows BC, cols CD (2), rows D, extras
  // (new state), decide, restore; cuFFT pipeline: prologue, prep,
  // spectral_mid, pre_pointwise, spectral_update, post_pointwise, decide,
  // restore
  if (kernels) *kernels = h->fused ? 10 : 8;
  return KKS_OK;
}

int kks_destroy(kks_handle* h) {
  KKS_RANGE("kks_destroy");
  free_handle(h);
  return KKS_OK;
}

}  // extern "C"
