// kks_fft.cuh - plans and launch description of the shared-memory FFT
// pipeline of the mixed path (kks_fft.cu).
#pragma once

#include <cuda_runtime.h>

#include "kks_internal.cuh"

#define KKS_FFT_MAXST 16
#define KKS_FFT_COLS 4  // y-frequency columns per column-pass block

// In-place mixed-radix transform of length n along one axis. Stage s has radix
// r[s], current sub-transform length L[s] and stride q[s] = L[s] / r[s]; the
// DIF runs the stages in order, the DIT in reverse. tw + tw_off[s] holds
// (cos, sin)(2 pi j m / L[s]) at [j * r[s] + m] (stages with q = 1 have none).
// A large prime factor P (> 7) is the last stage; prow holds its cos / sin
// table. slot[k] is the position of frequency k after the DIF.
struct KksFftAxis {
  int n, nst, P;
  int r[KKS_FFT_MAXST], L[KKS_FFT_MAXST], q[KKS_FFT_MAXST], tw_off[KKS_FFT_MAXST];
  const float2* tw;
  const float2* prow;
  const int* slot;
};

struct KksFftConst {
  KksFftAxis ax;         // x axis (column passes)
  KksFftAxis ay;         // y axis (row passes)
  const float* kx_slot;  // k_x of the frequency held at each x slot after the DIF
};

struct KksFftLaunch {
  const KksConst* dc;
  const KksPar* par;
  const KksFftConst* fc;  // device copy
  const KksFieldPtrs* f;
  void* RA;  // 3 row-spectrum fields (also RC)
  void* RB;  // 3 row-spectrum fields (also RD)
  void* SA;  // 2 full spectra FT(eta), FT(X)
  int nx, ny, nyh;
  int nbx;   // grid of the pointwise extras kernel
  int PX, PY;
};

// Largest prime factors with a register-resident direct DFT; other sizes use cuFFT.
#define KKS_FFT_PRIMES {11, 19, 71}

// Number of partial-sum rows the pipeline writes (the decide kernel reduces them).
int kks_fft_partial_rows(int nx, int ny, int nbx);
int kks_fft_set_attributes(const KksFftLaunch& L);
void kks_fft_launch_attempt(const KksFftLaunch& L, int parity, cudaStream_t s);
