/*
 * kks.h - C ABI of the B200-native extended-KKS phase-field step.
 *
 * One handle owns one simulation cell on one GPU: its fields stay resident in
 * device memory, every attempt of the semi-implicit step (KKS free energy,
 * Khachaturyan elasticity, spectral Allen-Cahn / Cahn-Hilliard updates, phase
 * compositions, energy residual and the accept / enlarge / reject decision)
 * runs on the device, and the host only launches work, drains log records and
 * moves fields at the boundary.
 *
 * The reference (pf_kks, pure Python) has no FFI; its one entry point for this
 * path is `pf_kks.solver.run(cfg, eta, X, X_al, X_th, out_dir, base_dir,
 * write_logs, verbose)` (pf_kks/solver.py:76-414). The functions below are the
 * pieces that call decomposes into; each names the reference lines it replaces.
 *
 * Conventions: every function returns 0 (KKS_OK) or a negative error code;
 * kks_last_error() gives a message. No exception crosses the ABI. A handle
 * uses one CUDA stream and is not thread-safe. Field arrays are C-order
 * (nx, ny) float64 on the host, y fastest, as the reference's (nx, ny, 1).
 */
#ifndef KKS_H
#define KKS_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define KKS_OK 0
#define KKS_ERR_ARG (-1)      /* invalid argument (size, pointer, option) */
#define KKS_ERR_CUDA (-2)     /* CUDA runtime error */
#define KKS_ERR_CUFFT (-3)    /* cuFFT error */
#define KKS_ERR_STATE (-4)    /* call out of order (e.g. run before upload) */
#define KKS_ERR_CAPACITY (-5) /* host buffer too small */

/* Run status of a cell, set on the device (pf_kks/solver.py:292-295, 312-313). */
#define KKS_STATUS_OK 0
#define KKS_STATUS_MAX_ITER 1   /* AdaptiveStepError: no admissible step after max_iterations attempts */
#define KKS_STATUS_NONFINITE 2  /* AdaptiveStepError: non-finite energy residual */
#define KKS_STATUS_TIMEOUT 3    /* a bounded device wait (bulk-copy completion) ran out; state undefined */

#define KKS_PRECISION_FP64 0  /* all-FP64 step */
#define KKS_PRECISION_MIXED 1 /* FP32 transforms and pointwise math on the step increments; FP64 state, scalars,
                                 phase compositions and sums; hand-written shared-memory FFTs where the grid
                                 factors into 2, 3, 4, 5, 7 and at most one of 11, 19, 71, else cuFFT */
#define KKS_PRECISION_MIXED_CUFFT 2 /* the mixed step with cuFFT transforms (comparison path) */

#define KKS_MAX_SCHED 64
#define KKS_MAX_TABLE 32
#define KKS_NTAB 13
/* Order of the material tables in kks_params.table (pf_kks/materials.py:17-31). */
enum {
  KKS_TAB_A_ALP = 0, KKS_TAB_B_ALP, KKS_TAB_C_ALP, KKS_TAB_A_THET, KKS_TAB_B_THET, KKS_TAB_C_THET,
  KKS_TAB_C11, KKS_TAB_C12, KKS_TAB_C44, KKS_TAB_EPSX, KKS_TAB_VM, KKS_TAB_GAMMA, KKS_TAB_X_SI_FCC
};

/* Run constants: SimulationConfig (pf_kks/config.py:12-90) after the scaling
 * that solver.run applies at its start (pf_kks/solver.py:101-116), plus the
 * tables of final_export.npz (pf_kks/materials.py:33-55, already scaled by
 * c_gamma / c_eps0). */
typedef struct kks_params {
  int32_t nx, ny;
  int32_t max_iterations, good_step_offset;
  double dx;          /* grid spacing [m] */
  double lambd;       /* half interface width [m] = half_width_cells * dx */
  double alpha;       /* interface-width constant */
  double D0, QD;      /* Si diffusion prefactor (x c_D) [m^2/s], activation energy [J/mol] */
  double Meta0, QMeta;/* interface mobility prefactor (x c_Meta), activation energy */
  double Lv2;         /* vacancy_sink_distance^2 [m^2] */
  double diffusion_enhancement_cap;
  double Xv0;         /* initial vacancy site fraction = quenched_vacancy_fraction(T_quench) */
  double dtime_s, dtime_max, dtime_min_divisor;
  double residual_max, residual_min, step_factor;
  double x_equilibrium;
  double surf_scale;  /* dx^2 / (2 lambd) (pf_kks/microstructure.py:128) */
  int32_t n_sched, n_table;
  double sched_time[KKS_MAX_SCHED], sched_temp[KKS_MAX_SCHED];
  double table_T[KKS_MAX_TABLE];
  double table[KKS_NTAB][KKS_MAX_TABLE];
} kks_params;

/* One log record, emitted on the device in program order
 * (pf_kks/runlog.py:32-140 formats them). */
#define KKS_REC_STATE 1     /* RunLog.state: every attempt of a step multiple of 100 */
#define KKS_REC_REJECTED 2  /* RunLog.rejected (dtime_s already divided) */
#define KKS_REC_ACCEPTED 3  /* RunLog.accepted */
#define KKS_REC_ENLARGED 4  /* RunLog.enlarged (dtime_s not yet multiplied) */
typedef struct kks_record {
  int32_t kind, istep, iteration, good_step;
  double T, D, L, Meta, Vm, dtime_s;
  double res_total, res_energy_derivative, res_diffusion, res_allen_cahn, res_temperature;
  double energy_s;
} kks_record;

/* Per-step history row (pf_kks/solver.py:375-395 and the energy / dt /
 * residual arrays of :166-170, 410-413). */
enum {
  KKS_H_X_AL_MEAN = 0, KKS_H_X_TH_MEAN, KKS_H_X_MEAN, KKS_H_DX_AL_MEAN, KKS_H_DX_TH_MEAN, KKS_H_DETA_MEAN,
  KKS_H_DT, KKS_H_ETA_MEAN, KKS_H_G_MEAN, KKS_H_SURF, KKS_H_DSURF, KKS_H_T, KKS_H_DTIME, KKS_H_TIME,
  KKS_H_TIME_S, KKS_H_L, KKS_H_ENERGY_S, KKS_H_DTIME_S, KKS_H_RES_TOTAL, KKS_H_RES_ENERGY_DERIVATIVE,
  KKS_H_RES_DIFFUSION, KKS_H_RES_ALLEN_CAHN, KKS_H_RES_TEMPERATURE, KKS_H_TTIME, KKS_H_ISTEP,
  KKS_H_SURF_VALID,
  KKS_H_D,   /* Si diffusivity of the accepted attempt [m^2/s] (pf_kks/kinetics.py:24-37, solver.py:184) */
  KKS_H_XV,  /* vacancy site fraction after the step (pf_kks/kinetics.py:52-60, solver.py:201) */
  KKS_H_COUNT
};
typedef struct kks_step_row {
  double v[32];
} kks_step_row;

/* Scalar run state (the loop variables of pf_kks/solver.py:118-175). */
typedef struct kks_run_state {
  int32_t istep, iteration, flag, good_step, status, parity;
  int64_t attempts, n_records, n_rows;
  double t, t_s, t_b, ttime, Xv, dtime_s, D_0, Meta_0, surf, surf_b, T_b;
  int32_t error_istep, error_iteration;
  double error_dtime_s;
} kks_run_state;

typedef struct kks_handle kks_handle;

/* Create a cell: allocate its device arena, plan the batched cuFFT R2C/C2R
 * transforms and capture the attempt graphs. Replaces the set-up of
 * pf_kks/solver.py:99-175 (tables, FFT plans, wave vectors, frozen-stiffness
 * Green operator, initial scalars). precision: KKS_PRECISION_*.
 * step_flags[i] bit 0: step i+1 is a surface-sampling step
 * (Schedule.surface_steps, pf_kks/solver.py:46-53); n_steps entries. */
int kks_create(const kks_params* params, int precision, int device, int32_t n_steps, const uint8_t* step_flags,
               int64_t record_capacity, kks_handle** out);

/* Upload the initial fields (host float64, nx*ny each). Replaces the arrays
 * handed to pf_kks/solver.py:76. */
int kks_upload(kks_handle* h, const double* eta, const double* X, const double* X_al, const double* X_th);

/* Advance up to n_steps accepted steps (attempt loop of pf_kks/solver.py:176-404)
 * without a host synchronisation per attempt; returns when the steps are done
 * or the device status is not OK. *status receives KKS_STATUS_*. */
int kks_run(kks_handle* h, int32_t n_steps, int32_t* status);

/* Advance several cells together (an ensemble): cell i by n_steps[i] steps.
 * Each cell keeps its own stream, graphs, adaptive dt and rejections; the
 * batches of all cells are launched before one synchronisation, so small
 * cells run concurrently on the GPU. status[i] receives KKS_STATUS_* per cell.
 * Replaces running pf_kks.solver.run (pf_kks/solver.py:76-414) once per cell. */
int kks_run_many(kks_handle** cells, int32_t n_cells, const int32_t* n_steps, int32_t* status);

/* A batch: cells of one device (KKS_PRECISION_MIXED on the shared-memory FFT
 * pipeline, all with the same large prime factor per axis, e.g. any mix of
 * 128..512 power-of-two / 3*2^k sides) advanced together. One attempt of the
 * batch launches every kernel once for all cells over the cells' device
 * descriptors (one CUDA graph); each cell keeps its own adaptive dt,
 * rejections, step target and buffer parity on the device, so cells of
 * different size, seed and schedule advance in lockstep and a cell that has
 * reached its target sits out. Results equal kks_run of each cell up to the
 * rounding of separately compiled FP32 kernels. `groups` (>= 1) splits the
 * cells into that many groups of about equal cost, each a graph on its own
 * stream, so that the groups' passes overlap. The cells must outlive the
 * batch. Replaces running pf_kks.solver.run (pf_kks/solver.py:76-414) once per
 * instance. */
typedef struct kks_batch kks_batch;
int kks_batch_create(kks_handle* const* cells, int32_t n_cells, int32_t groups, kks_batch** out);
/* Advance cell i by n_steps[i] steps; status[i] receives KKS_STATUS_*. */
int kks_batch_run(kks_batch* b, const int32_t* n_steps, int32_t* status);
/* Device time of all kks_batch_run calls (CUDA events) and batch attempts launched. */
int kks_batch_timing(const kks_batch* b, double* device_ms, int64_t* attempts);
int kks_batch_destroy(kks_batch* b);

/* Launch shape of a cell's attempt. The mixed precision can run the fused
 * shared-memory FFT passes or the cuFFT passes; the fused column passes take
 * `cols` y-frequency columns per block; the grid-stride field kernels
 * (interface / gradient sums, restore, the cuFFT pipeline's pointwise
 * kernels) run `field_blocks` blocks. kks_create picks a default; the
 * autotuner below times the candidates. No counterpart in the reference (a
 * numpy program has no launch shapes). */
typedef struct kks_launch_shape {
  int32_t pipeline;     /* 1: fused passes (KKS_PRECISION_MIXED only), 0: cuFFT passes */
  int32_t cols;         /* fused column tile, 1..4 */
  int32_t field_blocks; /* 1 .. the cell's maximum (8 blocks per SM) */
  int32_t pad;
} kks_launch_shape;
int kks_get_launch_shape(const kks_handle* h, kks_launch_shape* shape);
/* Re-captures the attempt graphs; KKS_ERR_STATE while the cell belongs to a batch. */
int kks_set_launch_shape(kks_handle* h, const kks_launch_shape* shape);
/* Time every candidate shape on `attempts` attempts of the cell's current
 * state (which is saved first and restored afterwards: the run continues as if
 * nothing had happened), keep the fastest and return it with its device time
 * per attempt. Needs at least 2 scheduled steps left. flags: 0, or
 * KKS_TUNE_BATCHABLE to consider only shapes that can join a batch. */
#define KKS_TUNE_BATCHABLE 1
int kks_autotune(kks_handle* h, int32_t attempts, int32_t flags, kks_launch_shape* best,
                 double* best_ms_per_attempt);

/* Copy the log records and history rows produced since the last drain. */
int kks_drain(kks_handle* h, kks_record* records, int64_t record_cap, int64_t* n_records, kks_step_row* rows,
              int64_t row_cap, int64_t* n_rows);

/* Scalar loop state. */
int kks_get_state(kks_handle* h, kks_run_state* state);

/* Download the current fields (host float64, nx*ny each); any pointer may be NULL. */
int kks_download(kks_handle* h, double* eta, double* X, double* X_al, double* X_th);

/* Debug aid; no counterpart in the reference. The library built with
 * -DKKS_BOUNDS_CHECK (libkks_b200_check.so) checks, in the fused passes, the
 * range each block works on (its rows or columns against the grid, its
 * partial-sum row against the buffer, its sequences against the launch's
 * shared memory) and, instead of faulting, records the first failed check and
 * skips that block's work. *checked = 1 for that build (0 otherwise: nothing
 * is checked); *first = the first recorded failure on `device` since the last
 * report (site << 44 | index; 0 = none), which the call clears. */
int kks_bounds_report(int device, int32_t* checked, uint64_t* first);

/* Fault-path test hook; no counterpart in the reference. The fused passes of
 * the mixed path wait for their bulk and tensor copies on an mbarrier with a
 * bounded number of polls; when a wait runs out, the cell's status becomes
 * KKS_STATUS_TIMEOUT, the block still waits (bounded again) for its copies in
 * flight, and kks_run stops after that attempt. This sets the poll count of the
 * first wait of a cell's passes (0: every such wait gives up at once; < 0: the
 * default, 2^20). KKS_ERR_STATE for a cell without fused passes. */
int kks_set_wait_polls(kks_handle* h, int32_t polls);

/* The "minus" entry of the energy residual's pair (the second-to-last element
 * of the reference's pair lists, pf_kks/solver.py:172-173, 278-290, 353-365):
 * eta- and X- (after an accepted step the current state, after a rejection the
 * rejected attempt's fields), the diffusion potential mu- of the last attempt
 * and the free energy G- (after an accepted step the step's pre-update G_s),
 * each host float64, nx*ny, in the units of the normalised step. With the
 * current state and kks_get_state this is the whole loop state of the
 * reference's solver at a step boundary. Any pointer may be NULL. */
int kks_download_pair(kks_handle* h, double* eta_m, double* X_m, double* mu_m, double* G_m);

/* Elastic stress and strain of the last attempt (returned by solve_elasticity,
 * pf_kks/elasticity.py:107-163; SimulationResult.sig_el / eps_el). Components
 * xx, yy, zz, xy (xz = yz = 0 in 2-D), nx*ny each: sig4 and eps4 hold 4*nx*ny. */
int kks_elastic_fields(kks_handle* h, double* sig4, double* eps4);

/* Exact restart point: every device buffer and scalar that carries state from
 * one attempt to the next (the reference has none: pf_kks/io.py:6-8). With
 * buf == NULL, *size receives the size in bytes. */
int kks_checkpoint(kks_handle* h, void* buf, size_t cap, size_t* size);
int kks_restore(kks_handle* h, const void* buf, size_t size);

/* Device milliseconds spent in kks_run since creation (CUDA events on the
 * handle's stream) and the attempts they covered. */
int kks_timing(kks_handle* h, double* device_ms, int64_t* attempts);

/* No counterpart in the reference. The attempt pipeline of the handle:
 * *fused = 1 for the shared-memory FFT passes of the mixed path, 0 for the
 * cuFFT pipeline; *kernels = kernels of this library one attempt launches
 * (cuFFT's own kernels not counted). Either pointer may be NULL. */
int kks_pipeline(kks_handle* h, int32_t* fused, int32_t* kernels);

int kks_destroy(kks_handle* h);

/* No counterpart in the reference. For callers that cannot allocate device
 * memory (a framework that owns all device memory through its own pool, or a
 * latency-critical loop that must not call cudaMalloc / cudaFree because they
 * may synchronise the device): the sums behind the old-state histories of one
 * step (pf_kks/solver.py:380-395) and the interface cell count
 * (pf_kks/microstructure.py:117-128) of a state already in device memory, with
 * no allocation. eta, X: device float64, nx*ny each (C order); out: device
 * float64[6] = { sum eta, sum X[eta < 0.05], count(eta < 0.05),
 * sum X[eta > 0.95], count(eta > 0.95), cells with 4 corners in [0.1, 0.9] }.
 * Runs asynchronously on `stream` (a cudaStream_t, NULL = default stream).
 * Its scratch is a fixed device array of KKS_NOALLOC_MAX_BLOCKS x 6 doubles
 * (48 KiB) held by every GPU that loads the library; nx*ny above
 * KKS_NOALLOC_MAX_POINTS is rejected with KKS_ERR_CAPACITY, and nx or ny below
 * 2 with KKS_ERR_ARG (the interface count needs 2 x 2 corners). The first call
 * on a device looks up that array's address (make it before any stream
 * capture); a call that finds another context current than the one of that
 * lookup (after cudaDeviceReset, for instance) looks it up again. Calls share
 * the array: calls that overlap on the GPU race and must be serialised by the
 * caller. */
#define KKS_NOALLOC_MAX_BLOCKS 1024
#define KKS_NOALLOC_MAX_POINTS (1 << 26)
int kks_state_sums_noalloc(const double* eta, const double* X, int32_t nx, int32_t ny, double* out, void* stream);

/* Fixed-dt step with explicit coefficients, and its adjoint. No counterpart in
 * the reference: they make the step differentiable (gradients of history
 * functionals such as a simulated DSC with respect to the kinetic parameters).
 * A fixed-dt step is the unarmed branch of the attempt loop
 * (pf_kks/solver.py:176-290 with flag == 0), all in FP64, with the per-step
 * coefficients given by the caller instead of the prologue:
 * coef[KKS_COEF_COUNT] = { dtime_s, L_s, kappa2_s, D_s, w_s, A_alp_s, B_alp_s,
 * C_alp_s, A_thet_s, B_thet_s, C_thet_s, epsX, C44(T), (B_alp - B_thet) /
 * (2 A_thet), A_alp / A_thet } (pf_kks/kinetics.py:83-107,
 * pf_kks/free_energy.py:74-95). State buffers are device float64 arrays of
 * 4*nx*ny: eta | X | X_al | X_th, each C-order (nx, ny). The stiffness is
 * frozen at C11_0, C12_0, C44_0 (pf_kks/solver.py:152-154). Calls run on the
 * handle's own stream and return after it has finished, unless the handle is
 * bound to a caller's stream (kks_adj_set_stream). */
enum {
  KKS_COEF_DT = 0, KKS_COEF_LS, KKS_COEF_KAPPA2, KKS_COEF_DS, KKS_COEF_W, KKS_COEF_A_ALP, KKS_COEF_B_ALP,
  KKS_COEF_C_ALP, KKS_COEF_A_THET, KKS_COEF_B_THET, KKS_COEF_C_THET, KKS_COEF_EPSX, KKS_COEF_C44,
  KKS_COEF_PC_SHIFT, KKS_COEF_PC_RATIO, KKS_COEF_COUNT
};
typedef struct kks_adj kks_adj;
int kks_adj_create(int32_t nx, int32_t ny, double C11_0, double C12_0, double C44_0, int device, kks_adj** out);
/* state_out = step(state_in; coef). */
int kks_adj_forward(kks_adj* h, const double* state_in, const double* coef, double* state_out);
/* Vector-Jacobian product of one step: given state_in, its step state_out and
 * the cotangent lam_out of state_out, lam_in receives the cotangent of
 * state_in and dcoef[KKS_COEF_COUNT] the gradient of <lam_out, state_out>
 * with respect to coef (host array). */
int kks_adj_backward(kks_adj* h, const double* state_in, const double* state_out, const double* coef,
                     const double* lam_out, double* lam_in, double* dcoef);
/* kks_adj_backward with dcoef[KKS_COEF_COUNT] written to device memory by the
 * stream, so that a run of backward steps needs no host round trip. */
int kks_adj_backward_device(kks_adj* h, const double* state_in, const double* state_out, const double* coef,
                            const double* lam_out, double* lam_in, double* dcoef_device);
/* Run the handle's calls on the caller's CUDA stream (a cudaStream_t; the
 * calls then return once their work is queued, ordered after earlier work on
 * that stream), or, with stream = NULL, on the handle's own stream, returning
 * after it has finished (the default). The legacy default stream is named
 * cudaStreamLegacy here, since NULL selects the handle's own stream.
 * Switching waits for queued work. */
int kks_adj_set_stream(kks_adj* h, void* stream);
/* Precision of the handle's step and adjoint: KKS_PRECISION_FP64 (default)
 * or KKS_PRECISION_MIXED: every transform in FP32 (cuFFT R2C / C2R on the
 * rounded input, output widened back), all pointwise work, the state and the
 * sums in FP64, and the semi-implicit updates (and their adjoints) carrying
 * only the increments through the FP32 transforms, as the main mixed step
 * does. */
int kks_adj_set_precision(kks_adj* h, int precision);
int kks_adj_destroy(kks_adj* h);

/* Initial state written on the device. No nx*ny host array crosses the ABI:
 * the fields go straight into the cell's state, and the functions that set a
 * whole state reset the loop state as kks_upload does.
 *
 * The seeded synthetic microstructure of the benchmark workloads (no
 * counterpart in the reference, which places sharp circles read from a file,
 * pf_kks/microstructure.py:7-52) is made in two calls around the host's draws
 * from numpy.random.Generator(PCG64(seed)), which keep their order:
 *   1. kks_voronoi_edges: seeds (host, n_seeds x {x, y} in cells, drawn
 *      uniformly in the box) -> nearest-seed labels under the periodic metric
 *      and *n_edges = the pixels whose right or lower periodic neighbour has
 *      another label;
 *   2. the host draws the particle picks (ranks among the edge pixels in C
 *      order; flat point indices when n_edges == 0), jitters and radii, then
 *      kks_generate_fields: eta = max over particles of
 *      1/2 [1 - tanh((r - R)/w)] in a periodic window of reach ceil(R + 8w) + 1
 *      around each centre, X = eta x_particle + (1 - eta)(x_matrix + low +
 *      range u_i) with u_i the i-th double of the PCG64 stream from rng_state
 *      (the 128-bit LCG jumped ahead on the device), and the KKS phase
 *      compositions X_al = (X - h pc_shift) / ((1 - h) + h pc_ratio),
 *      X_th = pc_ratio X_al + pc_shift, h = 3 eta^2 - 2 eta^3
 *      (pf_kks/free_energy.py:74-95). */
typedef struct kks_gen_args {
  int32_t n_particles;
  int32_t picks_are_points;  /* 1: pick[] are flat point indices, not edge-pixel ranks */
  const int64_t* pick;       /* host, n_particles */
  const double* jitter;      /* host, 2 per particle: x, y [cells] */
  const double* radii;       /* host, n_particles [cells] */
  double w;                  /* width of the tanh profile [cells] */
  double x_matrix, noise_low, noise_range, x_particle;
  uint64_t rng_state[2];     /* PCG64 LCG state before the matrix noise: {low 64 bits, high 64 bits} */
  uint64_t rng_inc[2];       /* PCG64 increment: {low, high} */
  double pc_shift;           /* (B_alp - B_thet) / (2 A_thet) at the initial temperature */
  double pc_ratio;           /* A_alp / A_thet */
} kks_gen_args;
int kks_voronoi_edges(kks_handle* h, int32_t n_seeds, const double* seeds, int64_t* n_edges);
int kks_generate_fields(kks_handle* h, const kks_gen_args* args);

/* Sharp circular precipitates in a uniform matrix: the state becomes
 * (eta, X, X_matrix, X_precipitate) of pf_kks/microstructure.py:7-52
 * (`place_precipitates`, the CLI's initial state, pf_kks/cli.py:46-49), with
 * nz = 1: a point at (i dx, j dy, 0) is inside when
 * sqrt((ox-x)^2 + (oy-y)^2 + (oz-0)^2) <= r. r, ox, oy, oz: host float64[n] in
 * metres. */
int kks_place_precipitates(kks_handle* h, double dx, double dy, double x_matrix, double x_precipitate, int32_t n,
                           const double* r, const double* ox, const double* oy, const double* oz);
/* Nuclei into the current state, in place (pf_kks/microstructure.py:55-74,
 * `add_nuclei`): inside points get eta = 1, X = X_th = 0.99999, X_al = 0. */
int kks_add_nuclei(kks_handle* h, double dx, double dy, int32_t n, const double* r, const double* ox,
                   const double* oy, const double* oz);
/* Random nucleation on the current state (pf_kks/nucleation.py:103-111,
 * `insert_random_nucleus`, with the candidates of the original put_nucle: the
 * points with eta < eta_below, in C order). kks_count_below gives their number;
 * kks_insert_nuclei sets eta = 1 at the ranks[j]-th candidate of each j (ranks
 * taken before any of the n insertions; a rank out of range is KKS_ERR_ARG). */
int kks_count_below(kks_handle* h, double eta_below, int64_t* count);
int kks_insert_nuclei(kks_handle* h, double eta_below, int32_t n, const int64_t* ranks);

/* Message of the last error of this thread. */
const char* kks_last_error(void);

/* Library version string. */
const char* kks_version(void);

#ifdef __cplusplus
}
#endif

#endif /* KKS_H */
