// kks_noalloc.cu - state reductions for callers that cannot allocate device memory.
//
// kks_state_sums_noalloc computes, for a state already in the caller's device
// memory, the sums behind the per-step histories of the old state (mean eta,
// mean X of the matrix and of the precipitates) and the interface cell count.
// The step's own pre-update kernel computes the same sums inside kks_run.
//
// Some callers cannot call cudaMalloc: a framework that hands this library
// buffers from its own pooled allocator and forbids raw allocations, or a
// latency-critical loop that must not call into the allocator, because
// cudaMalloc / cudaFree may synchronise the whole device. This entry point
// allocates nothing. Its scratch (one row of partial sums per thread block) is
// a fixed file-scope device array, kKksNoallocBlocks x kKksNoallocSlots
// doubles (48 KiB), that every GPU that loads this library holds until the
// process exits.
//
// Host code cannot use the array's name as a device address (it is a host
// stand-in), so the first call on each device looks the address up with
// cudaGetSymbolAddress while that device is current and caches it, together
// with the device's current context; make that first call before any stream
// capture. A call that finds another context current (after cudaDeviceReset,
// or a primary context released and created again, the module is loaded anew
// and the array may sit elsewhere) looks the address up again. All calls share the one array and it
// keeps the last call's contents: every block overwrites its own row before
// the final kernel reads it, so nothing has to start at zero, but calls that
// overlap on the GPU (two streams, or two host threads) race on the array and
// must be serialised by the caller.

#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "kks.h"

// Sets the message returned by kks_last_error (kks_abi.cu).
int kks_set_error(int code, const std::string& msg);

namespace {

constexpr int kThreads = 256;
constexpr int kKksNoallocBlocks = KKS_NOALLOC_MAX_BLOCKS;
constexpr int kKksNoallocSlots = 6;

static __device__ __align__(256) double g_noalloc_scratch[kKksNoallocBlocks * kKksNoallocSlots];

// Per-device address of the scratch array and the context it belongs to,
// filled on the first call on the device (and again after a context change).
constexpr int kMaxDevices = 64;
double* g_scratch_addr[kMaxDevices] = {nullptr};
CUcontext g_scratch_ctx[kMaxDevices] = {nullptr};
std::mutex g_scratch_mu;

// cuCtxGetCurrent through the runtime's driver entry point (no link to libcuda).
PFN_cuCtxGetCurrent_v4000 ctx_getter() {
  static PFN_cuCtxGetCurrent_v4000 fn = nullptr;
  if (!fn) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = (PFN_cuCtxGetCurrent_v4000)p;
  }
  return fn;
}

__device__ __forceinline__ bool in_iface(double e) { return e >= 0.1 && e <= 0.9; }

__global__ void __launch_bounds__(kThreads)
    k_state_partials(const double* __restrict__ eta, const double* __restrict__ X, int nx, int ny,
                     double* __restrict__ scratch) {
  __shared__ double sh[kKksNoallocSlots][kThreads / 32];
  const int N = nx * ny;
  double acc[kKksNoallocSlots] = {0, 0, 0, 0, 0, 0};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
    const double e = eta[i], x = X[i];
    acc[0] += e;
    if (e < 0.05) { acc[1] += x; acc[2] += 1.0; }
    if (e > 0.95) { acc[3] += x; acc[4] += 1.0; }
    const int ix = i / ny, iy = i - ix * ny;
    if (ix < nx - 1 && iy < ny - 1 && in_iface(e) && in_iface(eta[i + ny]) && in_iface(eta[i + ny + 1]) &&
        in_iface(eta[i + 1]))
      acc[5] += 1.0;
  }
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < kKksNoallocSlots; ++k) {
    double v = acc[k];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if (lane == 0) sh[k][wid] = v;
  }
  __syncthreads();
  if (threadIdx.x < kKksNoallocSlots) {
    double v = 0;
    for (int w = 0; w < kThreads / 32; ++w) v += sh[threadIdx.x][w];
    scratch[blockIdx.x * kKksNoallocSlots + threadIdx.x] = v;  // every row is overwritten: no clearing needed
  }
}

__global__ void k_state_finish(const double* __restrict__ scratch, int nblocks, double* __restrict__ out) {
  const int k = threadIdx.x;
  if (k >= kKksNoallocSlots) return;
  double v = 0;
  for (int b = 0; b < nblocks; ++b) v += scratch[b * kKksNoallocSlots + k];
  out[k] = v;
}

int fail(int code, const std::string& msg) { return kks_set_error(code, msg); }

}  // namespace

extern "C" int kks_state_sums_noalloc(const double* eta, const double* X, int32_t nx, int32_t ny, double* out,
                                      void* stream) {
  if (!eta || !X || !out) return fail(KKS_ERR_ARG, "kks_state_sums_noalloc: null device pointer");
  if (nx < 2 || ny < 2) return fail(KKS_ERR_ARG, "kks_state_sums_noalloc: nx and ny must be >= 2");
  if ((long long)nx * ny > KKS_NOALLOC_MAX_POINTS)
    return fail(KKS_ERR_CAPACITY, "kks_state_sums_noalloc: nx*ny exceeds KKS_NOALLOC_MAX_POINTS (2^26)");
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices)
    return fail(KKS_ERR_CUDA, "kks_state_sums_noalloc: no current CUDA device");
  double* scratch;
  {
    std::lock_guard<std::mutex> lock(g_scratch_mu);
    PFN_cuCtxGetCurrent_v4000 get_ctx = ctx_getter();
    CUcontext ctx = nullptr;
    if (!get_ctx || get_ctx(&ctx) != CUDA_SUCCESS)
      return fail(KKS_ERR_CUDA, "kks_state_sums_noalloc: cannot read the current CUDA context");
    if (!ctx || !g_scratch_addr[dev] || g_scratch_ctx[dev] != ctx) {
      // set-up for this device and context (the lookup also makes the
      // device's primary context current when no context was yet)
      void* p = nullptr;
      cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
      if (e != cudaSuccess || !p)
        return fail(KKS_ERR_CUDA, std::string("kks_state_sums_noalloc: cudaGetSymbolAddress: ") +
                                      cudaGetErrorString(e));
      if (!ctx && (get_ctx(&ctx) != CUDA_SUCCESS || !ctx))
        return fail(KKS_ERR_CUDA, "kks_state_sums_noalloc: no current CUDA context");
      g_scratch_addr[dev] = (double*)p;
      g_scratch_ctx[dev] = ctx;
    }
    scratch = g_scratch_addr[dev];
  }
  const int N = nx * ny;
  int nblocks = (N + kThreads - 1) / kThreads;
  if (nblocks > kKksNoallocBlocks) nblocks = kKksNoallocBlocks;
  cudaStream_t s = (cudaStream_t)stream;
  k_state_partials<<<nblocks, kThreads, 0, s>>>(eta, X, nx, ny, scratch);
  k_state_finish<<<1, 32, 0, s>>>(scratch, nblocks, out);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return fail(KKS_ERR_CUDA, std::string("kks_state_sums_noalloc: launch: ") +
                                                      cudaGetErrorString(e));
  return KKS_OK;
}
