// haccgpm.hpp — C++ drop-in for the serial path of HACC_GPM, over the C-ABI
// of include/hgpm_c.h.
//
// The names, argument meanings and call order are those of the reference's
// public header (src/haccgpm.hpp): HACCGPM::Params (:118-174),
// HACCGPM::read_params, HACCGPM::Timestepper (:178-198),
// HACCGPM::CosmoClass (:200-254) and namespace HACCGPM::serial (:385-506),
// so a caller written against the reference's serial() loop
// (src/driver_pm.cpp:32-163) compiles against this header unchanged in the
// calls it makes.  Error behaviour is the reference's: a failing call prints
// the message and exits the process (the reference's gpuErrchk/cudaCall).
//
// Differences a caller can see:
//   * MemoryManager holds an opaque context instead of raw d_pos / d_vel /
//     d_grid / d_grad pointers (the state lives in HBM as packed cell + FP32
//     offset; hgpm_store_state_device gives the reference's float3 layout).
//   * forward_fft / backward_fft take single-precision cufftComplex grids
//     (floatFFT_t); the reference's double-precision overloads (deviceFFT_t)
//     and out-of-place forms have no counterpart.
//   * InitGreens and fft_cache_plan are no-ops (the Green's function is
//     computed inside the fused Poisson pass; there are no plans).
//   * GetPowerSpectrum writes folds 0..PK_FOLDS; modes that the reference's
//     BinPower would index before its bin arrays (bin_power.cu:12-16, folds
//     > 0) are dropped (REF_QUIRKS 0: each fold binned in its own box).
#pragma once

// the headers the reference's haccgpm.hpp brings to its callers (the
// driver calls cudaFree(0) and strlen through them)
#include <cuComplex.h>
#include <cuda_runtime.h>
#include <stdio.h>
#include <cstdint>
#include <cstring>
#include <functional>

#include "hgpm_c.h"

// Wall-clock timer as the reference declares it, at global scope
// (src/haccgpm.hpp:18): microseconds since an arbitrary origin.
typedef unsigned long long CPUTimer_t;
CPUTimer_t CPUTimer();

// src/haccgpm.hpp:28: the single-precision complex grid type (cufftComplex
// is cuFloatComplex)
#ifndef floatFFT_t
#define floatFFT_t cuFloatComplex
#endif

namespace HACCGPM {

using ::CPUTimer;
using ::CPUTimer_t;

// src/haccgpm.hpp:118-174, the fields the serial path reads.  `c` holds the
// same values in the C-ABI layout; every call re-derives it from the named
// fields, so a caller may edit them between read_params and use.
struct Params {
    char fname[HGPM_PATH_MAX];
    int ng, np;
    double rl;
    int blockSize;
    int seed;
    double z_ini, z_fin;
    int nsteps;
    char prefix[HGPM_PATH_MAX];
    double m_hubble, m_omega_cdm, m_omega_nu, m_deut, m_ss8, m_ns, m_w_de, m_wa_de, m_Tcmb;
    double m_neff_massless, m_neff_massive;
    double m_omega_baryon, m_omega_cb, m_omega_matter, m_omega_radiation;
    double m_f_nu_massless, m_f_nu_massive;
    bool pks[HGPM_MAX_STEPS];
    bool dumps[HGPM_MAX_STEPS];
    char ipk[HGPM_PATH_MAX];
    bool do_analysis;
    bool analysis[HGPM_MAX_STEPS];
    char analysis_dir[HGPM_PATH_MAX];
    char analysis_py[HGPM_PATH_MAX];
    int lastStep;
    int pkFolds;
    int world_rank, world_size;
    // the one-rank decomposition (the multi-rank fields of the reference's
    // struct): a single 1x1x1 grid of ranks holding the whole ng^3 grid
    int local_grid_size[3];
    int grid_dims[3];
    int grid_coords[3];
    bool dump_init, dump_final;
    double ol;
    int overload;
    int pk_bins;
    bool pk_log;
    hgpm_params c;
};

// params.cpp:201-250: parse, print (print_params) and write the
// "<prefix>.params" echo (save_params).
Params read_params(const char* fname);
hgpm_params to_c(const Params& p);

// timestepper.cpp:31-68
class Timestepper {
   public:
    Params params;
    double aa, z, deltaT, adot, fscal;
    int world_rank;
    explicit Timestepper(Params iparams);
    void setInitialA(double a);
    void setInitialZ(double z);
    void advanceHalfStep();
    void reverseHalfStep();
    hgpm_timestepper to_c() const;

   private:
    void from_c(const hgpm_timestepper& t);
};

// cosmo.cpp:11-79: the serial path uses it only to find and read the .ipk
class CosmoClass {
   public:
    double Omega_m, Omega_cb, h;
    char ipk[HGPM_PATH_MAX];
    CosmoClass() {}
    explicit CosmoClass(Params& params);
    // cosmo.cpp:26-79; *out is new[]-allocated, the caller delete[]s it
    void read_ipk(double** out, int* nbins, double* k_delta, double* k_max, double* k_min, int calls = 0);
};

namespace serial {

// mmanager.cu:93-179: owns the device state of one box
class MemoryManager {
   public:
    hgpm_ctx* ctx = nullptr;
    explicit MemoryManager(Params params);
    ~MemoryManager();
    MemoryManager(const MemoryManager&) = delete;
    MemoryManager& operator=(const MemoryManager&) = delete;
};

void fft_cache_plan(int ng);
// ffts.cu:244-294 / :397-445 with a floatFFT_t grid: the unnormalised 3D C2C
// transform of d_grid ([ng][ng][ng], device) in place, on the legacy stream,
// returning when done as the reference's cufftExecC2C + cudaDeviceSynchronize.
void forward_fft(floatFFT_t* d_grid, int ng, int calls = 0);
void backward_fft(floatFFT_t* d_grid, int ng, int calls = 0);
void InitGreens(Params& params, MemoryManager& mem, int calls = 0);
void GenerateDisplacementIC(MemoryManager& mem, CosmoClass& cosmo, Params& params, Timestepper& ts, int calls = 0);
void UpdatePositions(Params& params, MemoryManager& mem, Timestepper ts, float frac, int calls = 0);
void CIC(Params& params, MemoryManager& mem, int calls = 0);
void SolveGradient(Params& params, MemoryManager& mem, int calls = 0);
void UpdateVelocities(Params& params, MemoryManager& mem, Timestepper ts, int calls = 0);
void GetPowerSpectrum(Params& params, MemoryManager& mem, const char* fname, int calls = 0);
void writeOutput(Params& params, MemoryManager& mem, char* fname, int calls = 0);
double get_fscal(double m_aa, double m_adot, double m_omega_cb);
void printTimers(CPUTimer_t init, CPUTimer_t total);

// Not in the reference: nsteps whole steps with the drifts fused into the
// kick (bit-identical to the UpdatePositions/CIC/SolveGradient/
// UpdateVelocities/UpdatePositions sequence); ts advances as that loop does.
void RunSteps(Params& params, MemoryManager& mem, Timestepper& ts, int nsteps);

// PyAnalysis (py_analysis.cu:3-27): with DO_ANALYSIS, at every step that
// ANALYSIS_STEPS marks, the particles' rows (tag, x, y, z, vx, vy, vz; tag
// the lattice index) go to the analysis code with the step, a and z.  The
// reference passes them to Python through pycosmotools (a submodule absent
// here); here the receiver is any callable.
using AnalysisHook = std::function<void(const float* rows, int64_t n, int ncols, int step, double aa, double z)>;
void Analysis(Params& params, MemoryManager& mem, Timestepper& ts, int step, const AnalysisHook& hook);
// The driver's receiver: the rows as raw float32 [n][ncols] in
// "<dir>/analysis.<step>" (dir "." when ANALYSIS_DIR is unset).
void WriteAnalysisRows(const char* dir, const float* rows, int64_t n, int ncols, int step);

}  // namespace serial
}  // namespace HACCGPM
