// hgpm_internal.h — declarations shared by the CUDA translation units and
// the host runtime of the PM step.  Not part of the public C-ABI.
#pragma once
#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

#include "hgpm_device.cuh"

namespace hgpm {

// Arguments of the fused x pass that bins P(k).
struct PkArgs {
    const float* kf;     // float(signed(i) * 2 pi / rl), one per grid index
    const float* filt;   // per-axis CIC window factor
    int nbins;
    int log_bins;
    double min_k;
    double bin_delta;    // linear: width; log: width in ln k
    double scale;        // (1/ng^3) * (rl/ng), scale_power.cu:8
};

// Grid sides with compiled FFT passes: 2^a 3^b 5^c multiples of 8 up to 1024
// (the reference's sizing tool, mem_calc.py:6-22, picks such sides; the
// Lagrangian particle blocks need multiples of 8 and the packed cell index
// 10 bits per axis).
#define HGPM_SIZES(X)                                                                                       \
    X(16) X(24) X(32) X(40) X(48) X(64) X(80) X(96) X(120) X(128) X(160) X(192) X(200) X(240) X(256) X(320) \
    X(384) X(400) X(480) X(512) X(640) X(768) X(800) X(960) X(1000) X(1024)
#define HGPM_SIZES_TEXT                                                                                     \
    "16,24,32,40,48,64,80,96,120,128,160,192,200,240,256,320,384,400,480,512,640,768,800,960,1000,1024"
bool fft_size_supported(int ng);
// cudaFuncAttributeMaxDynamicSharedMemorySize for `func` on the current
// device, set once per (device, kernel) rather than before every launch.
cudaError_t smem_attr_once(const void* func, int bytes);
// Resident CTAs per SM of `func` at this block size and shared memory
// (occupancy query made once per (device, kernel)).
int blocks_per_sm_once(const void* func, int threads, int smem);
int pk_max_bins();

// Launchers of the step's kernels.  `sl`/`nslots` batch the launch over
// nslots boxes of one size class (Slots in hgpm_device.cuh); the defaults
// launch one box.
cudaError_t launch_zfwd(int ng, void* in, bool fixed, float2* out, int nlines, int zs, double mean,
                        const float2* tw, cudaStream_t s, const Slots& sl = Slots{}, int nslots = 1);
cudaError_t launch_zinv(int ng, const float2* in, float* out, int nlines, int zs, size_t in_cs, size_t out_cs,
                        int ncomp, float scale, const float2* tw, cudaStream_t s, const Slots& sl = Slots{},
                        int nslots = 1);
// Unnormalised 3D complex-to-complex FFT of a [ng][ng][ng] float2 grid (z
// fastest), in place; tw: the ng-point table exp(-2 pi i k / ng).
cudaError_t launch_fft_c2c(int ng, float2* data, bool inv, const float2* tw, cudaStream_t s);
// The C2R z pass of one box writing the paired potential (2 ng^3 floats:
// cell z of a line holds (phi(z), phi(z+1 mod ng))).
cudaError_t launch_zinv_pair(int ng, const float2* in, float* out, int zs, const float2* tw, cudaStream_t s);
// The z and y passes of one box with a thread-block cluster per x plane
// (sides in HGPM_PLANE_SIZES): the forward R2C z + y passes of the int64
// density (zeroed) into the half spectrum, and the inverse y + C2R z passes
// of a half spectrum (y-inverted in place) into the paired potential;
// bit-identical to launch_zfwd + the y pass and the y pass +
// launch_zinv_pair.  Measured slower than the separate passes (512^3: 0.77
// against 0.65 ms forward, 0.77 against 0.49 inverse), so opt-in.
#define HGPM_PLANE_SIZES(X) X(256) X(512) X(1024)
bool plane_fft_supported(int ng);
cudaError_t launch_zy_fwd(int ng, unsigned long long* rho, float2* spec, int zs, double mean, const float2* tw,
                          cudaStream_t s);
cudaError_t launch_yz_inv_pair(int ng, float2* spec, float* out, int zs, const float2* tw, cudaStream_t s);
cudaError_t launch_strided(int ng, bool inv, float2* data, int ncols, size_t rs, size_t ps, int nplanes, size_t cs,
                           int ncomp, const float2* tw, cudaStream_t s, const Slots& sl = Slots{}, int nslots = 1);
// x pass fused with the Green's function: the potential's spectrum
// G rho_k, transformed back along x, into out (one half-spectrum buffer).
cudaError_t launch_xpotential(int ng, const float2* in, float2* out, int ncols, size_t rs, size_t ps, int nplanes,
                              const float2* tw, const double* cosq, double coeff, cudaStream_t s,
                              const Slots& sl = Slots{}, int nslots = 1);
// The same pass with twice the columns per CTA (x pass choice 2).
cudaError_t launch_xpotential_wide(int ng, const float2* in, float2* out, int ncols, size_t rs, size_t ps,
                                   int nplanes, const float2* tw, const double* cosq, double coeff, cudaStream_t s);
// Force grid (F_x, F_y, F_z, 0) from the real potential by central
// differences (the reference's -i sin(k) gradient, applied in real space).
cudaError_t launch_gradient(int ng, const float* phi, float4* f, cudaStream_t s, const Slots& sl = Slots{},
                            int nslots = 1);
cudaError_t launch_xic(int n, const float2* in, float2* out, int ncols, size_t rs, size_t ps, int nplanes,
                       size_t out_cs, const float2* tw, const double* table, int nbins, double k_delta,
                       double pkscale, double inv_delta, const float* kf, int* err, cudaStream_t s);
cudaError_t launch_xpk(int ng, const float2* in, int ncols, size_t rs, size_t ps, const float2* tw, const PkArgs& a,
                       double* part_sum, unsigned long long* part_cnt, int nparts, double* sum,
                       unsigned long long* cnt, cudaStream_t s);

// Persistent TMA-fed strided pass over a half-spectrum buffer (y lines, or x
// lines when isx); err is set if a bounded mbarrier wait times out.
cudaError_t launch_strided_tma(int ng, bool inv, bool isx, float2* data, int ncols, int zs, size_t cs, int ncomp,
                               const float2* tw, int* err, cudaStream_t s);
// A bounded mbarrier wait that nothing completes (tests of the time-out
// path): sets *err after `polls` polls.
cudaError_t launch_wait_timeout_probe(int* err, unsigned polls, cudaStream_t s);
// Persistent TMA-fed launch_xpotential (single box).
cudaError_t launch_xpotential_tma(int ng, float2* in, float2* out, int ncols, int zs, const float2* tw,
                                  const double* cosq, double coeff, int* err, cudaStream_t s);

cudaError_t launch_load_state(const float* x, const float* v, const ParticleSoA& p, int np_side, int B, int ng,
                              cudaStream_t s);
cudaError_t launch_store_state(const ParticleSoA& p, float* x, float* v, int np_side, int B, int ng,
                               cudaStream_t s);
cudaError_t launch_drift(const ParticleSoA& p, size_t n, int ng, float pf, cudaStream_t s);
// CIC (int64 fixed point, global atomics) of the positions folded `fold`
// times (x -> 2x mod ng per axis, each time), for folded P(k).
cudaError_t launch_deposit_folded(const ParticleSoA& p, size_t n, int ng, int fold, float mass,
                                  unsigned long long* rho, cudaStream_t s);
int deposit_cap_cells(int np_side, int ng);
// The deposit writes every block's CIC window (kWinRec ints per block); the
// kick reads it back when have_rec (positions unchanged since the deposit),
// else measures and writes it.
int window_records(int np_side, int ng);  // ints per box
// Kick configurations: every candidate gives bit-identical results.
// kick_candidates: how many; kick_kernels: kernels one launch_kick_drift
// call of candidate `choice` launches (the windowed one two: windowed + spill).
int kick_candidates(int np_side, int ng);
int kick_kernels(int choice, int np_side, int ng);
// Candidates that gather the real potential instead of the float4 force
// grid (the step then skips gradient_kernel).
bool kick_uses_phi(int choice);
// the kick gathers the paired potential (zpass_c2r with pair: cell z holds
// (phi(z), phi(z+1)), 8 bytes per cell, in the force grid's space)
bool kick_uses_phi2(int choice);
// Deposit configurations (bit-identical int64 grids): how many, and the
// default (used when the choice is -1).
int deposit_candidates(int np_side, int ng);
int deposit_default(int np_side, int ng);
// Built-in kick candidate (without tuning): the paired potential for 16^3
// blocks, the real potential for 8^3 blocks.
int kick_default(int np_side, int ng);
// Blocks too wide for a kernel's window are queued in `spill` (the deposit's
// and the kick's own lists) and run one particle per thread after the
// windowed pass, inside the same launcher.
cudaError_t launch_deposit(const ParticleSoA& p, int np_side, int ng, float mass, unsigned long long* rho,
                           int* blkwin, const SpillList& spill, cudaStream_t s, const Slots& sl = Slots{},
                           int nslots = 1, int choice = -1);
// f: the float4 (F_x, F_y, F_z, 0) force grid; phi (may be null): the real
// potential, for the candidates that gather it (with phi null they fall
// back to candidate 0).  choice: kick candidate (0 = default).
cudaError_t launch_kick_drift(const ParticleSoA& p, int np_side, int ng, const float4* f, double deltaT,
                              double fscal, float pf_a, float pf_b, int ndrift, int choice, int* blkwin,
                              bool have_rec, const SpillList& spill, cudaStream_t s, const Slots& sl = Slots{},
                              const KickSched& ks = KickSched{}, int nslots = 1, const float* phi = nullptr);
// Batched step bookkeeping: each active slot's step counter advances and a
// slot that has run nsteps[slot] steps goes idle.
cudaError_t launch_slots_advance(int* active, int* step, const int* nsteps, int nslots, cudaStream_t s);
cudaError_t launch_density(const unsigned long long* rho64, float* rho, size_t n, cudaStream_t s);
cudaError_t launch_ktables(int ng, double* cosq, float* sk, float* pkw, cudaStream_t s);
// White noise of the ICs: kind HGPM_NOISE_CURAND (curand_init(seed, i, 0) +
// curand_normal_double, as the reference) or HGPM_NOISE_PHILOX.
cudaError_t launch_noise(float* out, size_t n, int seed, int kind, cudaStream_t s);
cudaError_t launch_place(const float* sgrid, size_t scomp, const ParticleSoA& p, int np_side, int ng, float delta_f,
                         float velmul, cudaStream_t s);

}  // namespace hgpm
