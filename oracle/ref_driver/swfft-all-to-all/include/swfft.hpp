// swfft.hpp — stand-in for the SWFFT submodule header that the reference's
// driver (src/driver_pm.cpp) includes.  TEST INFRASTRUCTURE ONLY.  The
// driver's parallel() branch (multi-rank: SWFFT, MPI, particle transfer) is
// out of scope for the drop-in; its HACCGPM::parallel:: calls are declared
// here so the driver compiles unchanged, and each aborts if reached (the
// one-rank mpi.h stand-in sends main() to serial()).
#pragma once
#include <cstdio>
#include <cstdlib>

namespace HACCGPM {
namespace parallel {
[[noreturn]] inline void not_in_drop_in(const char* what) {
    fprintf(stderr, "ref_driver: HACCGPM::parallel::%s is the multi-rank path, outside the drop-in\n", what);
    abort();
}
class MemoryManager {
   public:
    explicit MemoryManager(HACCGPM::Params) { not_in_drop_in("MemoryManager"); }
};
inline void init_swfft(HACCGPM::Params&) { not_in_drop_in("init_swfft"); }
inline void finalize_swfft() { not_in_drop_in("finalize_swfft"); }
inline void GenerateDisplacementIC(MemoryManager&, HACCGPM::CosmoClass&, HACCGPM::Params&, HACCGPM::Timestepper&,
                                   int = 0) { not_in_drop_in("GenerateDisplacementIC"); }
inline void TransferParticles(HACCGPM::Params&, MemoryManager&, int = 0) { not_in_drop_in("TransferParticles"); }
inline void InitGreens(HACCGPM::Params&, MemoryManager&, int = 0) { not_in_drop_in("InitGreens"); }
inline void GetPowerSpectrum(HACCGPM::Params&, MemoryManager&, int, const char*, int = 0) {
    not_in_drop_in("GetPowerSpectrum");
}
inline void UpdatePositions(HACCGPM::Params&, MemoryManager&, HACCGPM::Timestepper, float, int = 0) {
    not_in_drop_in("UpdatePositions");
}
inline void CIC(HACCGPM::Params&, MemoryManager&, int = 0) { not_in_drop_in("CIC"); }
inline void SolveGradient(HACCGPM::Params&, MemoryManager&, int = 0) { not_in_drop_in("SolveGradient"); }
inline void UpdateVelocities(HACCGPM::Params&, MemoryManager&, HACCGPM::Timestepper, int = 0) {
    not_in_drop_in("UpdateVelocities");
}
inline void printTimers(HACCGPM::CPUTimer_t, HACCGPM::CPUTimer_t, int) { not_in_drop_in("printTimers"); }
}  // namespace parallel
}  // namespace HACCGPM
