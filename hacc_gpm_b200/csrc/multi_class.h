// multi_class.h — one launch per PM phase across the size classes of an
// ensemble.
//
// A batched step of an ensemble normally launches each phase once per size
// class (ensemble.cu).  The multi-class step launches each phase ONCE for all
// classes: the launch's work units are the concatenation of every class's
// units (deposit: Lagrangian blocks of every slot; FFT passes: line groups or
// column tiles of every slot; kick: particle units of every slot).  A CTA
// finds its unit's class in the table below and runs that class's code for
// that unit: the same device bodies the single-class kernels run
// (bit-identical results), the FFT ones dispatched on the class's grid side.
// The deposit and the kick are persistent grids walking the units; the FFT
// passes launch one CTA per unit.  Per step: a counter reset, the deposit,
// its spill pass, the five FFT passes (z, y, x with the Green's function, y,
// and z to the paired potential), the kick gathering the paired potential
// with both drifts, and the slot advance: ten launches whatever the number of
// classes.
#pragma once

#include "hgpm_device.cuh"
#include "hgpm_internal.h"

namespace hgpm {

constexpr int kMaxMC = 8;  // classes per multi-class launch

// Grid sides the multi-class FFT passes are compiled for: those of the
// ensemble and serving workloads (2^a 3^b from 32 to 256).  Each side is a
// case of one kernel per pass; more cases push the kernels into spills.
#define HGPM_MC_SIZES(X) X(32) X(48) X(64) X(96) X(128) X(192) X(256)

struct MCClass {
    int ng = 0, np = 0, nslots = 0, nblocks = 0, zs = 0;
    float mass = 1.f;
    double mean = 0.0;
    int* active = nullptr;   // [nslots] 1 while the slot has steps to run
    int* step = nullptr;     // [nslots] steps done
    const int* nsteps = nullptr;
    ParticleSoA p{};         // slot 0; slot s at s * part_stride
    size_t part_stride = 0;
    unsigned long long* rho64 = nullptr;  // slot s at s * ncell
    size_t ncell = 0;
    float2* spec = nullptr;   // forward spectrum, slot s at s * spec_elems
    float2* fspec = nullptr;  // potential spectrum (slot stride 3 * spec_elems)
    size_t spec_elems = 0;
    float* force = nullptr;   // force grid space (slot stride force_elems floats):
                              // the paired potential the kick gathers
    size_t force_elems = 0;
    int* blkwin = nullptr;    // window records, slot stride win_stride
    size_t win_stride = 0;
    SpillList spill{};
    const float2* tw = nullptr;
    const double* cosq = nullptr;
    const float4* sched = nullptr;  // [nslots][pitch] kick / drift scalars
    int pitch = 0;
};

struct MCTable {
    int n = 0;
    int u0[kMaxMC + 1] = {};  // first global work unit of each class (per phase)
    int per[kMaxMC] = {};     // units per slot of each class (FFT passes)
    MCClass c[kMaxMC];
};

// Classes the multi-class step takes: 16^3 particle blocks and a grid side
// among HGPM_MC_SIZES.
bool mc_class_supported(int ng, int np);

cudaError_t mc_step(const MCTable& t, cudaStream_t s);
// The FFT passes of mc_step (fft_passes.cu): z forward from the int64
// density, y forward, x with the Green's function, y inverse, z inverse to
// the real potential.
cudaError_t mc_launch_fft_passes(const MCTable& t, cudaStream_t s);
// Kernel launches of one mc_step.
constexpr int kMCStepLaunches = 10;

}  // namespace hgpm
