// kks_fft.cuh - plans and launch description of the shared-memory FFT
// pipeline of the mixed path (kks_fft.cu).
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "kks_internal.cuh"

#define KKS_FFT_MAXST 16
#define KKS_FFT_THREADS 320   // threads of every pass block (ten warps)
#define KKS_FFT_COLS 3        // y-frequency columns per column-pass block
#define KKS_FFT_MAXN 8192     // longest axis of the pipeline (shared memory and 32-bit index magic)

// In-place mixed-radix transform of length n along one axis. Stage s has radix
// r[s], current sub-transform length L[s] and stride q[s] = L[s] / r[s]; the
// DIF runs the stages in order, the DIT in reverse. tw + tw_off[s] holds
// (cos, sin)(2 pi j m / L[s]) at [j * r[s] + m] (stages with q = 1 have none).
// qm[s] / pm[s] are ceil(2^32 / q[s]) and ceil(2^32 / (n / r[s])) (0 for a
// divisor of 1): x / d == __umulhi(x, m) for x, d < 2^16. A large prime factor
// P (> 7) is the last DIF stage (q = 1). slot[k] is the position of frequency k
// after the DIF.
struct KksFftAxis {
  int n, nst, P;
  int r[KKS_FFT_MAXST], L[KKS_FFT_MAXST], q[KKS_FFT_MAXST], tw_off[KKS_FFT_MAXST];
  uint32_t qm[KKS_FFT_MAXST], pm[KKS_FFT_MAXST];
  const float2* tw;
  const int* slot;
  const float2* ptw;  // prime DFT factors, (cos, sin) pairs (see kks_fft_prime_table); null if P = 0
};

struct KksFftConst {
  KksFftAxis ax;         // x axis (column passes)
  KksFftAxis ay;         // y axis (row passes)
  const float* kx_slot;  // k_x of the frequency held at each x slot after the DIF
};

// Spectrum buffers are column-major: element (ix, ky) of field f at
// f * nx * nyh + ky * nx + ix, so that a column pass reads and writes one
// contiguous run of nx values and a row pass one 16-byte pair per frequency.
struct KksFftLaunch {
  const KksConst* dc;
  const KksPar* par;
  KksCtl* ctl;            // status word (a bounded wait that runs out sets KKS_STATUS_TIMEOUT)
  const KksFftConst* fc;  // device copy
  const KksFieldPtrs* f;
  void* RA;  // 3 row-spectrum fields (also RC)
  void* RB;  // 3 row-spectrum fields (also RD)
  void* SA;  // 2 full spectra FT(eta), FT(X), x in DIF slot order
  int nx, ny, nyh;
  int nbx;   // grid of the pointwise extras kernel
  int PX, PY;
  int bulk_rows;  // 1: row passes move their spectra with tensor copies and stage their state
                  // rows with bulk copies (needs nx % 2 == 0, ny % 4 == 0 and encoded maps)
  int bulk_cols;  // 1: column passes load their columns with bulk copies (needs nx % 2 == 0)
  // tensor maps (x: nx, ky: nyh, field: F; 8-byte elements; box {2, min(nyh, 256), F})
  CUtensorMap map_RA3;  // RA (also RC), F = 3
  CUtensorMap map_RB3;  // RB, F = 3
  CUtensorMap map_RB2;  // RB as RD, F = 2
};

// Largest prime factors with a direct DFT stage; other sizes use cuFFT.
#define KKS_FFT_PRIMES {11, 19, 71}

// Shared memory of the largest pass block for an nx x ny grid (bytes).
size_t kks_fft_smem_bytes(int nx, int ny);
// Blocks of a row pass, and the number of partial-sum rows the pipeline
// writes (the decide kernel reduces them).
int kks_fft_row_blocks(int nx);
int kks_fft_partial_rows(int nx, int ny, int nbx);
int kks_fft_set_attributes(const KksFftLaunch& L);
// The prime-stage factor table of prime P (11, 19 or 71), rows padded to an
// even length: at most KKS_FFT_PRIME_TABLE_MAX pairs written to out; returns
// the count, or 0 for an unsupported P.
#define KKS_FFT_PRIME_TABLE_MAX (5 * 35 * 8)
int kks_fft_prime_table(int P, float2* out);
void kks_fft_launch_attempt(const KksFftLaunch& L, int parity, cudaStream_t s);
