// kks_fft.cuh - plans and launch description of the shared-memory FFT
// pipeline of the mixed path (kks_fft.cu).
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "kks_internal.cuh"

#define KKS_FFT_MAXST 16
#define KKS_FFT_THREADS 320   // threads of every pass block (ten warps)
#define KKS_FFT_COLS 3        // default y-frequency columns per column-pass block (a launch shape)
#define KKS_FFT_COLS_MAX 4    // largest column tile a launch shape may choose
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
  // the FP64 step's tables (kks_fft64.cu): the same twiddles in double, and
  // its prime factors (kks_fft64_prime_table); null in a mixed cell
  const double2* tw64;
  const double2* ptw64;
};

struct KksFftConst {
  KksFftAxis ax;         // x axis (column passes)
  KksFftAxis ay;         // y axis (row passes)
  const float* kx_slot;  // k_x of the frequency held at each x slot after the DIF
  const double* kx_slot64;  // the same in double (FP64 step)
  int cols;              // y-frequency columns per column-pass block (1..KKS_FFT_COLS_MAX)
  int wait_polls;        // polls of the first wait for a block's bulk / tensor copies (KKS_FFT_WAIT_POLLS;
                         // kks_set_wait_polls changes it for fault-path tests)
  int part_cap;          // partial-sum rows allocated (the bounds-check build checks each block's row)
};

#define KKS_FFT_WAIT_POLLS (1 << 20)

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
  int cols;  // y-frequency columns per column-pass block (the device copy is fc->cols)
  int PX, PY;
  int f64;        // 1: the FP64 step's passes (kks_fft64.cu; plain loads, no tensor maps)
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

// Shared memory of the largest pass block for an nx x ny grid with column
// tiles of `cols` (bytes).
size_t kks_fft_smem_bytes(int nx, int ny, int cols);
// Blocks of a row pass, and an upper bound of the partial-sum rows the
// pipeline writes with any column tile (the decide kernel reduces them).
int kks_fft_row_blocks(int nx);
int kks_fft_partial_rows(int nx, int ny, int nbx);
int kks_fft_set_attributes(const KksFftLaunch& L);
// The prime-stage factor table of prime P (11, 19 or 71), rows padded to an
// even length: at most KKS_FFT_PRIME_TABLE_MAX pairs written to out; returns
// the count, or 0 for an unsupported P.
#define KKS_FFT_PRIME_TABLE_MAX (5 * 35 * 8)
int kks_fft_prime_table(int P, float2* out);
// The first out-of-range index recorded by the bounds-check build's kernels of
// kks_fft.cu on the current device (0: none; site << 44 | index), cleared when
// reset is nonzero. Returns 1 in a bounds-check build, 0 otherwise (*first = 0).
int kks_fft_bounds_word(unsigned long long* first, int reset);
void kks_fft_launch_attempt(const KksFftLaunch& L, int parity, cudaStream_t s);

// The FP64 step's passes (kks_fft64.cu). Prime tables: at most
// KKS_FFT64_PRIME_TABLE_MAX (cos, sin) pairs in double, layout of ZPrime there.
#define KKS_FFT64_PRIME_TABLE_MAX (7 * 35 * 5)
size_t kks_fft64_smem_bytes(int nx, int ny, int cols);
int kks_fft64_set_attributes(const KksFftLaunch& L);
int kks_fft64_prime_table(int P, double2* out);
void kks_fft64_launch_passes(const KksFftLaunch& L, int parity, cudaStream_t s);

// ---------------------------------------------------------------------------
// Batched launches: the cells of an ensemble advance together, every kernel of
// the attempt launched once for all of them. A cell is described in device
// memory (its tensor maps first, 64-byte aligned as TMA requires); a pass
// block finds its cell and its block index within the cell in the pass's
// block map. The state parity of each cell lives on the device (KksCtl::parity,
// flipped by the prologue of every attempt the cell takes part in), so cells
// that have reached their target, or stopped, skip attempts without losing
// track of their buffers.
struct __align__(64) KksCellDesc {
  CUtensorMap map_RA3, map_RB3, map_RB2;
  const KksConst* dc;
  KksPar* par;
  KksCtl* ctl;
  const KksFftConst* fc;
  double* eta[2];
  double* X[2];
  float* X_al[2];
  float* X_th[2];
  double* eta_m;
  double* X_m;
  float* mu;
  float* g[3];
  float2* RA;
  float2* RB;
  float2* SA;
  double* partials;
  const double* ky;
  const uint8_t* step_flags;
  kks_record* ring;
  long long ring_cap;
  kks_step_row* rows;
  long long row_cap;
  int N, nbx, part_rows, bulk_rows, bulk_cols, pad;
};

// Block map entry: x = cell, y = block within the cell (for the first column
// pass: role << 16 | column tile).
struct KksBatchLaunch {
  const KksCellDesc* cells;
  int n_cells;
  int PX, PY;
  const int2* map_rows;    // row pairs
  const int2* map_cols;    // column tiles
  const int2* map_cols3;   // column tiles x 3 roles (first column pass)
  const int2* map_extras;  // blocks of the extras and restore kernels (nbx per cell)
  int n_rows, n_cols, n_cols3, n_extras;
  size_t smem_rows_a, smem_rows_bc, smem_rows_d, smem_cols_ab, smem_cols_cd1, smem_cols_cd2;
};

// Fill the block maps' sizes and the passes' shared memory for cells of the
// given grids (host; the maps themselves are built by the caller in the order
// of its choice) and raise the kernels' shared-memory limits to match.
int kks_fft_batch_prepare(KksBatchLaunch& B, const int* nx, const int* ny, const int* cols, int n);
// Column tiles of a column pass.
int kks_fft_col_blocks(int nyh, int cols);
// prologue, fused passes, extras, decide and restore of one attempt of every cell
void kks_fft_launch_attempt_batch(const KksBatchLaunch& B, cudaStream_t s);
// batched scalar kernels (kks_scalar.cu)
void kks_launch_prologue_batch(const KksCellDesc* cells, int n, cudaStream_t s);
void kks_launch_decide_batch(const KksCellDesc* cells, int n, cudaStream_t s);
