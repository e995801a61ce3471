// kks_check.cuh - non-trapping bounds checks of the debug build.
//
// Built with -DKKS_BOUNDS_CHECK (python -m pf_kks_gpu.build --bounds-check,
// libkks_b200_check.so), the fused passes check the ranges each block works
// on (its rows or columns against the grid, its partial-sum row against the
// buffer, its sequences against the dynamic shared memory of the launch)
// before touching memory. A failed check records the first offender of this
// translation unit in a device word (site in bits 44..63, index in bits
// 0..43), and the block skips its work instead of faulting; the host reads
// the word with kks_bounds_report. Release builds compile the checks away.
// The substitute for a memory checker where none can run: out-of-range
// indices show up as a recorded site, never as a GPU fault.
#pragma once

#ifdef KKS_BOUNDS_CHECK
static __device__ unsigned long long g_kks_oob = 0ull;

__device__ __forceinline__ bool kks_in_range(long long i, long long n, int site) {
  if (i >= 0 && i < n) return true;
  atomicCAS(&g_kks_oob, 0ull, ((unsigned long long)(site & 0xFFFFF) << 44) | ((unsigned long long)i & 0xFFFFFFFFFFFull));
  return false;
}
#define KKS_IN(i, n, site) kks_in_range((long long)(i), (long long)(n), (site))
#define KKS_CHECKED_BUILD 1
#else
#define KKS_IN(i, n, site) true
#define KKS_CHECKED_BUILD 0
#endif

// Bytes of dynamic shared memory of the running launch.
__device__ __forceinline__ unsigned kks_dyn_smem_bytes() {
  unsigned v;
  asm volatile("mov.u32 %0, %%dynamic_smem_size;" : "=r"(v));
  return v;
}
