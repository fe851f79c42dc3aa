/*
 * hgpm_c.h — C-ABI of the B200-native particle-mesh step (drop-in for the
 * serial path of HACC_GPM).
 *
 * Plain C types only: opaque context handle, plain pointers and sizes, int
 * status returns (HGPM_OK == 0), no exits.  Every call is stream-ordered on
 * the context's CUDA stream; calls that take HOST pointers synchronise that
 * stream before returning.  Error text for the last failure on a context is
 * available from hgpm_last_error().
 *
 * Each entry point names the reference interface it replaces
 * (file:line within the HACC_GPM project).
 */
#ifndef HGPM_C_H
#define HGPM_C_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
#define HGPM_OK 0
#define HGPM_ERR_ARG 1         /* invalid argument or unsupported size     */
#define HGPM_ERR_CUDA 2        /* CUDA runtime error (message has details) */
#define HGPM_ERR_IO 3          /* file missing / malformed                  */
#define HGPM_ERR_OOM 4         /* device allocation failed                  */
#define HGPM_ERR_STATE 5       /* call order violated (e.g. no particles)   */

#define HGPM_MAX_STEPS 1000    /* src/haccgpm.hpp:106 */
#define HGPM_MAX_NG 1024       /* largest grid side (10-bit packed cell)    */
#define HGPM_PATH_MAX 300      /* char[300] fields of HACCGPM::Params       */

/* ---- run parameters ----------------------------------------------------
 * Mirror of HACCGPM::Params (src/haccgpm.hpp:118-174), serial fields only.
 * Cosmology values are stored as double after float rounding, exactly as
 * read_params does (params.cpp:109 `float val = atof(value)`).            */
typedef struct hgpm_params {
    char fname[HGPM_PATH_MAX];
    char prefix[HGPM_PATH_MAX];     /* OUTPUT_BASE_NAME */
    char ipk[HGPM_PATH_MAX];        /* IPK */
    int ng, np;
    double rl;
    int block_size;
    int seed;
    double z_ini, z_fin;
    int nsteps;
    int last_step;                  /* LAST_STEP (defaults to nsteps) */
    int pk_folds;
    int pk_bins;                    /* PK_BINS (new key; reference fixes 221) */
    int pk_log;                     /* PK_LOG (new key; 1 = log-spaced bins)  */
    double ol;
    int overload;
    double hubble, omega_cdm, omega_nu, deut, ss8, ns, w_de, wa_de, t_cmb;
    double neff_massless, neff_massive;
    /* derived (params.cpp:237-245) */
    double omega_baryon, omega_cb, omega_matter, omega_radiation;
    double f_nu_massless, f_nu_massive;
    unsigned char pks[HGPM_MAX_STEPS];
    unsigned char dumps[HGPM_MAX_STEPS];
    int dump_init, dump_final;
    int ref_quirks;                 /* 1 (default): float dtdy / float growth
                                       exactly as the reference; 0: FP64    */
    /* analysis hook (params.cpp:195-214): DO_ANALYSIS, ANALYSIS_STEPS,
       ANALYSIS_DIR, ANALYSIS_PY */
    int do_analysis;
    unsigned char analysis[HGPM_MAX_STEPS];
    char analysis_dir[HGPM_PATH_MAX];
    char analysis_py[HGPM_PATH_MAX];
    /* NOISE (new key): white-noise source of hgpm_ic_generate.
       HGPM_NOISE_CURAND (default): the reference's own draws,
       curand_init(SEED, cell, 0) then curand_normal_double per cell
       (rng_initializer.cu:38-49), so a SEED gives the reference's universe;
       HGPM_NOISE_PHILOX: counter-based Philox4x32-10 (Box-Muller).      */
    int noise;
} hgpm_params;

#define HGPM_NOISE_CURAND 0
#define HGPM_NOISE_PHILOX 1

/* Replaces HACCGPM::read_params (src/simulation/params.cpp:72-250).
 * Does not print or write the .params echo; see hgpm_params_save.        */
int hgpm_params_read(const char* path, hgpm_params* out, char* err, size_t errlen);
/* Parse params from a string (same grammar as hgpm_params_read).          */
int hgpm_params_parse(const char* text, hgpm_params* out, char* err, size_t errlen);
/* Recompute derived fields (params.cpp:237-245).                          */
void hgpm_params_derive(hgpm_params* p);
/* Replaces save_params (src/simulation/params.cpp:6-39): writes
 * "<prefix>.params" byte-compatible with the reference.                   */
int hgpm_params_save(const hgpm_params* p);

/* ---- time stepper ------------------------------------------------------
 * Replaces HACCGPM::Timestepper (src/simulation/timestepper.cpp:31-68),
 * get_adot (:13-21) and get_fscal (:23-28).  Host-side FP64.              */
typedef struct hgpm_timestepper {
    double aa, z, deltaT, adot, fscal;
    hgpm_params params;
} hgpm_timestepper;

void hgpm_ts_init(hgpm_timestepper* ts, const hgpm_params* p);
void hgpm_ts_set_initial_z(hgpm_timestepper* ts, double z);
void hgpm_ts_advance_half(hgpm_timestepper* ts);
void hgpm_ts_reverse_half(hgpm_timestepper* ts);
/* pm_actions.cpp:291: float prefactor = deltaT/(a*a*adot)*frac            */
float hgpm_ts_drift_prefactor(const hgpm_timestepper* ts, float frac);
double hgpm_get_adot(double aa, const hgpm_params* p);
double hgpm_get_fscal(double aa, double adot, double omega_cb, int ref_quirks);

/* Linear growth and its derivative at the IC epochs.
 * Replaces CosmoClass::get_delta_and_dotDelta (cosmo.cpp:133-139).        */
void hgpm_growth(const hgpm_params* p, double z, double z_vel, double* delta, double* dot_delta);

/* ---- context (device memory + stream) ----------------------------------
 * Replaces serial::MemoryManager (src/simulation/cuda/mmanager.cu:93-179)
 * and serial::fft_cache_plan (src/fft_tools/cuda/ffts.cu:136).            */
typedef struct hgpm_ctx hgpm_ctx;

int hgpm_create(const hgpm_params* p, int device, hgpm_ctx** out);
void hgpm_destroy(hgpm_ctx* ctx);
const char* hgpm_last_error(const hgpm_ctx* ctx);
/* Device bytes a context of this size holds (mem_calc.py:41-95 analogue). */
size_t hgpm_footprint_bytes(int ng, int np);
/* The CUDA stream (cudaStream_t) all work of this context is ordered on.   */
void* hgpm_stream(hgpm_ctx* ctx);
int hgpm_sync(hgpm_ctx* ctx);
int hgpm_ng(const hgpm_ctx* ctx);
int hgpm_np(const hgpm_ctx* ctx);

/* ---- particle state ------------------------------------------------------
 * Host buffers in the reference layout: float3 x[np^3], float3 v[np^3]
 * (particle_t = float3, src/haccgpm.hpp:76-80), grid units, x in [0, ng).
 * Inside the context positions are an int32 packed cell plus an FP32
 * in-cell offset, so precision does not degrade with the box side.        */
int hgpm_load_state(hgpm_ctx* ctx, const float* x_host, const float* v_host);
int hgpm_store_state(hgpm_ctx* ctx, float* x_host, float* v_host);
/* Same as above, but pointers are DEVICE pointers (stream-ordered).        */
int hgpm_load_state_device(hgpm_ctx* ctx, const float* x_dev, const float* v_dev);
int hgpm_store_state_device(hgpm_ctx* ctx, float* x_dev, float* v_dev);
/* The rows PyAnalysis hands to the analysis code (py_analysis.cu:10-22):
 * per particle, in lattice order, 7 floats (tag, x, y, z, vx, vy, vz), tag
 * the particle's lattice index (exact as a float up to 2^24 particles).   */
int hgpm_analysis_rows(hgpm_ctx* ctx, float* rows_host);
/* Linear cell index (ix*ng+iy)*ng+iz of every particle's CIC base cell
 * (the reference's `int i = x` truncation, cic_pm.cu:52-54).              */
int hgpm_get_cells(hgpm_ctx* ctx, int32_t* cells_host);
/* Restart from a particle dump: reads the file serial::writeOutput writes
 * (io.cu:12-44: raw float3 x[np^3] then float3 v[np^3]) into the context,
 * like hgpm_load_state.  Positions re-split from float3 as on any load.   */
int hgpm_read_output(hgpm_ctx* ctx, const char* fname);
/* Checkpoints (no counterpart in the reference): the exact device state
 * (packed cells, offsets, velocities) and a time stepper, to and from a
 * host buffer of hgpm_checkpoint_bytes(ctx).  A run of s steps,
 * checkpointed, loaded into a context of the same NG/NP and continued for n
 * steps with the saved stepper is bit-identical to s + n steps run at once
 * (resume after pre-emption; the float3 dump above is not exact).         */
size_t hgpm_checkpoint_bytes(const hgpm_ctx* ctx);
int hgpm_checkpoint_save(hgpm_ctx* ctx, const hgpm_timestepper* ts, void* host_buf, size_t bytes);
int hgpm_checkpoint_load(hgpm_ctx* ctx, hgpm_timestepper* ts_out, const void* host_buf, size_t bytes);

/* ---- PM phases -----------------------------------------------------------*/
/* serial::UpdatePositions (pm_actions.cpp:287-314, update_positions_pm.cu:3-20) */
int hgpm_drift(hgpm_ctx* ctx, float prefactor);
/* serial::CIC (pm_actions.cpp:221-258, cic_pm.cu:46-87): deterministic
 * fixed-point int64 deposit; the density is bit-exact run to run.         */
int hgpm_deposit(hgpm_ctx* ctx);
/* Density after hgpm_deposit, float ng^3 (Re of the reference's d_grid).  */
int hgpm_get_density(hgpm_ctx* ctx, float* rho_host);
/* serial::SolveGradient (solver.cpp:144-170): R2C FFT, fused Green's
 * function and -i sin(k) gradient, 3 C2R FFTs -> force grids.            */
int hgpm_solve_gradient(hgpm_ctx* ctx);
/* Force grids, float 3*ng^3 (x, y, z components; d_grad.xyz).             */
int hgpm_get_force(hgpm_ctx* ctx, float* force_host);
/* serial::UpdateVelocities (pm_actions.cpp:260-285, icic_pm.cu:72-127).    */
int hgpm_kick(hgpm_ctx* ctx, double deltaT, double fscal);
/* Fused CIC gather + kick + ndrift (0..2) drifts with prefactors pf_a, pf_b:
 * the reference's UpdateVelocities followed by UpdatePositions calls.     */
int hgpm_kick_drift(hgpm_ctx* ctx, double deltaT, double fscal, float pf_a, float pf_b, int ndrift);
/* nsteps whole DKD steps (driver_pm.cpp:114-125), advancing *ts exactly as
 * the reference's loop does; consecutive drifts are fused.                */
int hgpm_run_steps(hgpm_ctx* ctx, hgpm_timestepper* ts, int nsteps);
/* One step with the particle state in HOST buffers (reference layout):
 * copies in, runs hgpm_run_steps(ctx, ts, 1), copies out.                 */
int hgpm_step_host(hgpm_ctx* ctx, hgpm_timestepper* ts, float* x_host, float* v_host);

/* ---- power spectrum ------------------------------------------------------
 * serial::GetPowerSpectrum fold 0 (power.cu:152-246 with scale_power.cu,
 * filter_power.cu, bin_power.cu): nbins bins (linear as the reference, or
 * log-spaced when log_bins), FP64 shell sums, deterministic.  Outputs are
 * host arrays of nbins: bin centre k, P(k) (0 where empty), mode count.  */
int hgpm_power_spectrum(hgpm_ctx* ctx, int nbins, int log_bins, double* k_host,
                        double* pk_host, int64_t* count_host);
/* Writes "<fname>.fold.0" lines "%g,%g,%d" (power.cu:13-28).               */
int hgpm_write_pk(const char* fname, int nbins, const double* k, const double* pk,
                  const int64_t* count);
/* One fold of GetPowerSpectrum's PK_FOLDS loop (power.cu:189-227): the
 * positions folded `fold` times (x -> 2x mod ng per axis each time,
 * fold_particles_power.cu:3-27; exact on the packed positions) in a box of
 * side rl / 2^fold.  ref_quirks = 1 (default) keeps the reference's choices:
 * bin edges from rl / 2^max(PK_FOLDS, fold) for every fold and the power
 * scaled with the unfolded rl; modes below the first edge by more than one
 * bin, which the reference writes before its bin arrays (bin_power.cu:12-16),
 * are dropped.  ref_quirks = 0: bins and scale from the fold's own box.
 * fold 0 is hgpm_power_spectrum.  fold <= 9.                               */
int hgpm_power_spectrum_fold(hgpm_ctx* ctx, int fold, int nbins, int log_bins, double* k_host,
                             double* pk_host, int64_t* count_host);
/* writePkOutput for any fold: "<fname>.fold.<fold>".                        */
int hgpm_write_pk_fold(const char* fname, int fold, int nbins, const double* k, const double* pk,
                       const int64_t* count);
/* serial::writeOutput (io.cu:12-44): raw float3 x then float3 v.           */
int hgpm_write_output(hgpm_ctx* ctx, const char* fname);

/* ---- initial conditions -------------------------------------------------
 * serial::GenerateDisplacementIC (initializer.cpp:65-166).  The table is the
 * .ipk P(k) body (read by hgpm_read_ipk), k_delta its spacing.
 * hgpm_ic_generate draws the white noise with a counter-based Philox4x32-10
 * generator keyed by params.seed; hgpm_ic_from_noise takes the noise grid
 * (float np^3, host) instead, e.g. the reference's own cuRAND draw.        */
int hgpm_read_ipk(const char* path, double* header20, double* table, int max_bins, int* nbins);
int hgpm_ic_generate(hgpm_ctx* ctx, const double* table, int nbins, double k_delta);
int hgpm_ic_from_noise(hgpm_ctx* ctx, const float* noise_host, const double* table,
                       int nbins, double k_delta);
/* The Philox white-noise grid hgpm_ic_generate would use (float np^3).     */
int hgpm_ic_noise(hgpm_ctx* ctx, float* noise_host);

/* ---- phase timing --------------------------------------------------------
 * When enabled, phases record CUDA events; hgpm_phase_times returns the
 * accumulated milliseconds per phase and launch counts since the last reset.
 * One phase per kernel of the step: 0 drift, 1 deposit, 2 fft_z_fwd,
 * 3 fft_y_fwd, 4 poisson_x (x pass fused with Green's function, gradient
 * and inverse x), 5 fft_y_inv, 6 fft_z_inv, 7 kick_drift, 8 pk.           */
#define HGPM_NPHASE 9
int hgpm_enable_timing(hgpm_ctx* ctx, int on);
int hgpm_phase_times(hgpm_ctx* ctx, double* ms, int64_t* launches);
/* Number of kernels this context launched since creation / last reset.    */
int64_t hgpm_kernel_launches(hgpm_ctx* ctx, int reset);

/* ---- batched ensembles ------------------------------------------------------
 * No counterpart in the reference (its driver runs one box per process,
 * driver_pm.cpp:32-163).  An ensemble holds size classes; class i is
 * nslots[i] boxes of one (ng[i], np[i]).  hgpm_ens_step advances every
 * running box by one PM step with ONE launch per phase per class (the slot
 * is a grid dimension), classes on parallel streams, optionally replayed
 * from one CUDA graph.  Per box the results are bit-identical to
 * hgpm_run_steps on a single context.
 *
 * Life of a slot: hgpm_ens_slot binds params (NG/NP of the class, any RL,
 * cosmology and seed) and returns the slot as a context ("view", owned by
 * the ensemble, never passed to hgpm_destroy) for ICs, state I/O and P(k);
 * hgpm_ens_start queues its nsteps-step run; hgpm_ens_step / hgpm_ens_sync /
 * hgpm_ens_status advance and observe it; hgpm_ens_release frees the slot
 * once it has finished.  All work is ordered on the ensemble's stream.   */
typedef struct hgpm_ensemble hgpm_ensemble;

int hgpm_ens_create(int nclass, const int* ng, const int* np, const int* nslots, int device,
                    hgpm_ensemble** out);
void hgpm_ens_destroy(hgpm_ensemble* ens);
const char* hgpm_ens_last_error(const hgpm_ensemble* ens);
/* Device bytes of one class of nslots boxes (admission by footprint).     */
size_t hgpm_ens_footprint_bytes(int ng, int np, int nslots);
void* hgpm_ens_stream(hgpm_ensemble* ens);
int hgpm_ens_slot(hgpm_ensemble* ens, int cls, int slot, const hgpm_params* p, hgpm_ctx** view);
/* *ts as hgpm_run_steps takes it; returns advanced through nsteps.        */
int hgpm_ens_start(hgpm_ensemble* ens, int cls, int slot, hgpm_timestepper* ts, int nsteps);
int hgpm_ens_release(hgpm_ensemble* ens, int cls, int slot);
/* nsteps batched steps (slots that finish go idle on the device).         */
int hgpm_ens_step(hgpm_ensemble* ens, int nsteps);
int hgpm_ens_use_graph(hgpm_ensemble* ens, int on);
/* hgpm_ens_step launches each phase once for ALL classes (one launch per
 * phase over every class's and slot's work units; the kick gathering the
 * paired potential; ten launches per step) when `on` (the default),
 * the ensemble has at most 8 classes and every class has 16^3 particle
 * blocks (np a multiple of 16, ng <= np) and ng in {32, 48, 64, 96, 128,
 * 192, 256}; otherwise once per phase per class, the classes on their own
 * streams.  Results are bit-identical either way.  Returns 1 if the
 * multi-class form applies to this ensemble, 0 if not, < 0 on error.     */
int hgpm_ens_multi_launch(hgpm_ensemble* ens, int on);
/* Wait for queued work; refresh the host copy of every slot's status.     */
int hgpm_ens_sync(hgpm_ensemble* ens);
int hgpm_ens_status(hgpm_ensemble* ens, int cls, int slot, int* running, int* steps_done);
int64_t hgpm_ens_kernel_launches(hgpm_ensemble* ens, int reset);
/* One class at a time, for a serving loop whose classes advance at their
 * own pace (no counterpart in the reference either): hgpm_ens_step_class
 * queues nsteps steps of class cls on the class's own stream, after the
 * slot set-up queued so far, and returns; hgpm_ens_class_done sets *done to
 * 1 once they have run (a poll, no wait); hgpm_ens_sync_class waits for
 * them and refreshes that class's hgpm_ens_status.  While steps of a class
 * are queued, make no slot call on that class (hgpm_ens_slot, _start,
 * _release, or work on its views, whose deposit shares per-slot spill
 * counters with the class step); the other classes are free meanwhile.   */
/* Class streams carry stream priorities, smaller boxes higher.           */
int hgpm_ens_step_class(hgpm_ensemble* ens, int cls, int nsteps);
int hgpm_ens_class_done(hgpm_ensemble* ens, int cls, int* done);
int hgpm_ens_sync_class(hgpm_ensemble* ens, int cls);

/* ---- 3D FFT of a caller's grid ----------------------------------------------
 * serial::forward_fft / backward_fft on a single-precision complex grid
 * (ffts.cu:244-294 and :397-445 with a cufftComplex grid): the unnormalised
 * 3D complex-to-complex transform of data_dev ([ng][ng][ng] float2, z
 * fastest, the reference's get_index order) in place, forward
 * (exp(-2 pi i k.x / ng), CUFFT_FORWARD) or inverse (exp(+...),
 * CUFFT_INVERSE), for ng among the supported sides.  The first call for an
 * ng on a device uploads its twiddle table (kept until exit).  Stream-
 * ordered on `stream` (a cudaStream_t); with NULL it runs on the legacy
 * stream and returns when the transform is done (as the reference's
 * cufftExecC2C + cudaDeviceSynchronize).  Double-precision grids (the
 * reference's deviceFFT_t) are not supported.                             */
int hgpm_fft_c2c(void* data_dev, int ng, int inverse, void* stream);

/* ---- allocation-free density ------------------------------------------------
 * No counterpart in the reference.  For callers that cannot allocate device
 * memory (a host framework that owns every device allocation, or a run that
 * must never allocate after start-up): the CIC density of np_side^3 particles
 * (device float3 positions, grid units, reference layout) on an ng^3 grid,
 * written as float into rho_dev (device, ng^3), bit-identical to
 * hgpm_deposit + hgpm_get_density.  It allocates nothing: the int64
 * accumulation grid is a built-in device array of 128^3 cells (16 MiB, held
 * by every GPU that loads the library until exit), so ng > 128 is rejected
 * with HGPM_ERR_ARG.  The array is cleared at the start of every call and
 * keeps the last call's contents; calls on one device share it, so calls
 * whose work overlaps on the GPU (different streams, or different host
 * threads) race.  The first call on each device looks up the array's device
 * address (cudaGetSymbolAddress) and should be made before any stream
 * capture; the address is kept for the life of the process, so after a
 * cudaDeviceReset of a device this entry point must not be called on that
 * device again.  Stream-ordered on `stream` (a cudaStream_t, NULL = legacy). */
int hgpm_cic_density_noalloc(const float* x_dev, int np_side, int ng, float* rho_dev, void* stream);

/* ---- autotuner --------------------------------------------------------------
 * No counterpart in the reference, whose one launch knob is BLOCK_SIZE
 * (params.cpp:164, applied to every kernel by InvokeGPUKernel,
 * haccgpm.hpp:59).  Each knob below has candidates that give bit-identical
 * results and differ only in speed:
 *   HGPM_TUNE_DEPOSIT  deposit window kernel / CTA shape / window cap,
 *   HGPM_TUNE_KICK     kick gather scheme / CTA shape / units per CTA turn,
 *   HGPM_TUNE_YPASS    1 = TMA-fed persistent y pass, 0 = plain strided,
 *   HGPM_TUNE_XPASS    2 = plain x pass with twice the columns per CTA (the
 *                      default), 1 = TMA-fed persistent, 0 = plain.
 * hgpm_autotune times every candidate `reps` times on the context's current
 * particle state (which it leaves unchanged), keeps a knob's default unless
 * another candidate is faster by more than 2 %, applies the winners to the
 * context and, when `store`, appends them to the cache file
 * ($HGPM_TUNE_CACHE, else tune_cache.txt beside the library) under (device
 * name, SM count, ng, np).  hgpm_create applies the last cached entry for
 * its size and device unless HGPM_NO_TUNE_CACHE is set (or the knob's
 * environment variable HGPM_DEPOSIT / HGPM_KICK / HGPM_NO_TMA / HGPM_XTMA
 * pins it).  choices / best_ms (may be NULL) receive the picks and their
 * ms per launch.  HGPM_PLANE=1 (not tuned; sides 256, 512, 1024) runs the
 * z and y passes of the step's transforms as one kernel with an 8-CTA
 * thread-block cluster per x plane: bit-identical, slower than the
 * separate passes on B200.                                                */
#define HGPM_TUNE_KNOBS 4
#define HGPM_TUNE_DEPOSIT 0
#define HGPM_TUNE_KICK 1
#define HGPM_TUNE_YPASS 2
#define HGPM_TUNE_XPASS 3
int hgpm_autotune(hgpm_ctx* ctx, int reps, int store, int choices[HGPM_TUNE_KNOBS], double best_ms[HGPM_TUNE_KNOBS]);
/* The knobs a context uses now (after env, cache or tuning).              */
int hgpm_tuned_choices(const hgpm_ctx* ctx, int choices[HGPM_TUNE_KNOBS]);
/* The tuner's pick: the fastest of n timings (ms <= 0: not measured),
 * unless the default `def` is within a fraction `tol` of it.              */
int hgpm_tune_pick(const double* ms, int n, int def, double tol);
/* Cache file access (host only): lookup returns 1 and fills choices when a
 * line for (device, sms, ng, np) exists (the last one wins), else 0;
 * store appends one line.  device: one token without blanks.              */
int hgpm_tune_cache_lookup(const char* path, const char* device, int sms, int ng, int np,
                           int choices[HGPM_TUNE_KNOBS]);
int hgpm_tune_cache_store(const char* path, const char* device, int sms, int ng, int np,
                          const int choices[HGPM_TUNE_KNOBS], const double ms[HGPM_TUNE_KNOBS]);

/* ---- time-out path, for tests ------------------------------------------------
 * No counterpart in the reference.  Every mbarrier wait of the TMA-fed
 * passes is bounded; on time-out the pass sets an error flag and returns,
 * and the next hgpm_sync reports HGPM_ERR_CUDA ("... timed out ...") and
 * clears the flag, with the context still usable.  This queues a one-thread
 * kernel whose bounded wait (polls <= 2^20) nothing completes, so a test can
 * take that path without a fault.                                         */
int hgpm_test_wait_timeout(hgpm_ctx* ctx, unsigned polls);

/* ---- ABI checks ------------------------------------------------------------
 * sizeof of the public structs, for bindings that mirror them.            */
size_t hgpm_sizeof_params(void);
size_t hgpm_sizeof_timestepper(void);

#ifdef __cplusplus
}
#endif
#endif /* HGPM_C_H */
